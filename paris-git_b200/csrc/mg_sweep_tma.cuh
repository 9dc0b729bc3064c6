// mg_sweep_tma.cuh -- the fused red-black sweep of mg_sweep.cuh with its planes
// staged by the Tensor Memory Accelerator (FP32 levels; included by mg_fast.cu
// after mg_sweep.cuh).
//
// The arithmetic, the tiles, the wavefront of two planes per step and the ring
// slots are those of k_rb_sweep2_cfg; only the staging differs.  One thread
// issues, for every step, one cp.async.bulk.tensor box per array plane (the
// tile plus its ring, 40 x 20 cells) into the slot the plane occupies, and the
// boxes of a step complete on one mbarrier (transaction bytes).  The block
// waits on that barrier instead of on cp.async groups, and the 16-byte chunks
// that every thread used to stage (address arithmetic, 10 cp.async per step)
// disappear from the update threads.
//
// Out-of-range boxes are zero-filled by the copy engine: the wall ghosts of the
// multigrid are zero, as they are for the cp.async staging.  Where a direction
// is periodic, the ring columns and rows that leave the domain come from the
// other side: the block fetches those elements (at most one per thread) with
// plain loads one step ahead and writes them over the zeros once the box has
// landed.  The tiles need n0 % 32 == 0 and n1 % TY == 0 (checked on the host),
// so only the first and last tiles of a row or column have such elements.
//
// The tensor maps cover this GPU's own level arrays, are loaded without
// multicast, and only the single-GPU solver launches this kernel.
//
// Every wait on an mbarrier is bounded (kTmaWaitCycles); a wait that runs out
// sets *err (mapped host memory), and the block finishes its steps without
// waiting again, so the host sees the error instead of a hung kernel.
#pragma once
#include <cuda.h>

struct SwTmaMaps {
    CUtensorMap x, cx, cy, b, cz;   // level arrays as 3-D tensors (n0, n1, n2), box (kSwTX + 8, TY + 4, 1)
};

__device__ inline uint32_t sw_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ inline void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ inline bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ inline void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
// generic-proxy writes to shared memory before the copy engine overwrites it
__device__ inline void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ inline void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

static constexpr long long kTmaWaitCycles = 4000000000LL;   // about two seconds at the B200's clocks

// wait for the phase of parity `parity` of the barrier; false when it did not
// complete within kTmaWaitCycles
__device__ inline bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kTmaWaitCycles) return false;
    return true;
}

// the configuration of the TMA-staged sweep (its own, whatever the cp.async
// sweep uses): 32x16 tiles, one step staged ahead, two blocks per SM
using SwTmaCfg = SwCfg<float, 16, 1, 320, 2>;

// the ring slots, two mbarriers, and 128 bytes to align the slots (a box's
// destination must start on a 128-byte boundary)
template <class C>
static constexpr size_t sweep_tma_smem() {
    return sizeof(float) * (size_t)Sw2<C>::RP * Sw2<C>::SLOTS + sizeof(uint64_t) * 2 + 128;
}

// the array planes of one staging group: NE entries in a fixed order (so that
// they live in registers), each with its ring slot, array (0 x, 1 cx, 2 cy,
// 3 b, 4 cz), plane and whether the step needs it
template <int NE>
struct SwGroup {
    uint32_t slot[NE];   // byte offset of the plane's slot from the ring base
    int arr[NE];
    int k[NE];
    bool ok[NE];
};

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB)
    k_rb_sweep_tma(const LV<float> v, const float* __restrict__ xin, const __grid_constant__ SwTmaMaps M,
                   float* __restrict__ xout, const float* __restrict__ xc, const Bnd B, int first, int zc,
                   int* __restrict__ err) {
    using T = float;
    using G = Sw2<C>;
    constexpr int NT = G::NT;
    constexpr int RX = G::RX, RY = G::RY, RP = G::RP, TY = G::TY;
    static_assert(C::D == 1 && C::TX == kSwTX, "one step of planes staged ahead, 32-wide tiles");
    constexpr int NB = 2;   // groups in flight at most: one barrier each
    constexpr uint32_t BOX_BYTES = sizeof(T) * RP;
    static_assert(2 * (RX * 2) + 2 * (RY - 4) * 4 <= NT, "one ring element to wrap per thread");
    extern __shared__ __align__(128) unsigned char sw_dyn[];
    // slot 0 on a 128-byte boundary of the shared window; every slot is a
    // multiple of 128 bytes (BOX_BYTES)
    static_assert(BOX_BYTES % 128 == 0, "slots keep the 128-byte alignment of the boxes");
    unsigned char* const sw_raw = sw_dyn + ((128u - (sw_smem_u32(sw_dyn) & 127u)) & 127u);
    T* const sm = reinterpret_cast<T*>(sw_raw);
    T* const rx_ = sm;
    T* const rcx = sm + G::XS * RP;
    T* const rcy = rcx + G::CS * RP;
    T* const rb = rcy + G::CS * RP;
    T* const rcz = rb + G::CS * RP;
    uint64_t* const bars = reinterpret_cast<uint64_t*>(rcz + G::ZS * RP);
    const uint32_t s_base = sw_smem_u32(sm);
    const uint32_t s_bar0 = sw_smem_u32(bars);

    const int tid = threadIdx.x;
    const int n0 = v.n0, n1 = v.n1, n2 = v.n2;
    const long plane = (long)n0 * n1;
    const int x0 = blockIdx.x * kSwTX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, n2);
    const int kb = z0 - 2;
    auto slot = [&](int k, int S) { return (k - kb) % S; };
    const bool have_x = xin != nullptr;
    bool bad = false;

    if (tid == 0) {
        for (int q = 0; q < NB; q++) mbar_init(s_bar0 + 8 * q, 1);
        fence_mbar_init();
    }

    // the ring element this thread copies from the other side of a periodic
    // direction (candidates: rows 0, 1, RY-2, RY-1 over all columns, and
    // columns 0..3, RX-4..RX-1 over the other rows)
    long woff = -1;
    int wsm = 0;
    {
        int r = -1, cc = -1;
        if (tid < 4 * RX) {
            const int q = tid / RX;
            r = q < 2 ? q : RY - 4 + q;
            cc = tid % RX;
        } else if (tid < 4 * RX + 8 * (RY - 4)) {
            const int t = tid - 4 * RX;
            r = 2 + t / 8;
            const int q = t % 8;
            cc = q < 4 ? q : RX - 8 + q;
        }
        if (r >= 0) {
            const int gi0 = x0 - 4 + cc, gj0 = y0 - 2 + r;
            const bool out = gi0 < 0 || gi0 >= n0 || gj0 < 0 || gj0 >= n1;
            const int gi = sw_wrap(gi0, n0, B.per[0]), gj = sw_wrap(gj0, n1, B.per[1]);
            if (out && gi >= 0 && gj >= 0) {
                woff = gi + (long)n0 * gj;
                wsm = r * RX + cc;
            }
        }
    }
    float wv[13];

    const T* const garr[5] = {xin, v.cx, v.cy, v.b, v.cz};
    const CUtensorMap* const maps[5] = {&M.x, &M.cx, &M.cy, &M.b, &M.cz};
    const uint32_t ring_off[5] = {0u, (uint32_t)(sizeof(T) * G::XS * RP),
                                  (uint32_t)(sizeof(T) * (G::XS + G::CS) * RP),
                                  (uint32_t)(sizeof(T) * (G::XS + 2 * G::CS) * RP),
                                  (uint32_t)(sizeof(T) * (G::XS + 3 * G::CS) * RP)};
    auto set_x = [&](auto& g, int e, int k, int sx) {
        g.slot[e] = ring_off[0] + BOX_BYTES * sx;
        g.arr[e] = 0;
        g.k[e] = k;
        g.ok[e] = k <= z1 + 1;
    };
    auto set_c = [&](auto& g, int e, int a, int k, int s) {   // a = 1..4
        g.slot[e] = ring_off[a] + BOX_BYTES * s;
        g.arr[e] = a;
        g.k[e] = k;
        g.ok[e] = k <= z1;
    };
    // issue a group (thread 0), zero its iterate slots when there is no input
    // iterate, and fetch this thread's wrapped elements of the group
    auto issue = [&](const auto& g, int gi) {
        constexpr int NE = sizeof(g.k) / sizeof(int);
        const uint32_t bar = s_bar0 + 8 * (gi % NB);
        if (tid == 0) {
            uint32_t bytes = 0;
#pragma unroll
            for (int e = 0; e < NE; e++)
                if (g.ok[e] && (g.arr[e] != 0 || have_x)) bytes += BOX_BYTES;
            mbar_arrive_expect_tx(bar, bytes);
#pragma unroll
            for (int e = 0; e < NE; e++) {
                if (!g.ok[e] || (g.arr[e] == 0 && !have_x)) continue;
                const int gk = sw_wrap(g.k[e], n2, B.per[2]);
                tma_load_3d(s_base + g.slot[e], maps[g.arr[e]], x0 - 4, y0 - 2, gk >= 0 ? gk : g.k[e], bar);
            }
        }
        if (!have_x) {
#pragma unroll
            for (int e = 0; e < NE; e++)
                if (g.ok[e] && g.arr[e] == 0) {
                    T* d = reinterpret_cast<T*>(sw_raw + g.slot[e]);
                    for (int q = tid; q < RP; q += NT) d[q] = (T)0;
                }
        }
#pragma unroll
        for (int e = 0; e < NE; e++) {
            wv[e] = (T)0;
            if (g.ok[e] && woff >= 0 && (g.arr[e] != 0 || have_x)) {
                const int gk = sw_wrap(g.k[e], n2, B.per[2]);
                if (gk >= 0) wv[e] = garr[g.arr[e]][woff + plane * gk];
            }
        }
    };
    // wait for a group, then write the wrapped elements over the zero fill
    auto land = [&](const auto& g, int gi) {
        constexpr int NE = sizeof(g.k) / sizeof(int);
        if (!bad && !mbar_wait_bounded(s_bar0 + 8 * (gi % NB), (uint32_t)((gi / NB) & 1))) {
            bad = true;
            *(volatile int*)err = 1;
        }
        if (woff >= 0) {
#pragma unroll
            for (int e = 0; e < NE; e++)
                if (g.ok[e] && (g.arr[e] != 0 || have_x)) reinterpret_cast<T*>(sw_raw + g.slot[e])[wsm] = wv[e];
        }
    };

    int fr0[G::FPER], fpar[G::FPER], fok[G::FPER];
#pragma unroll
    for (int q = 0; q < G::FPER; q++) {
        int t = tid + q * NT;
        fr0[q] = -1;
        fpar[q] = 0;
        fok[q] = 0;
        if (t < G::FCELLS) {
            int fry = 1 + t / G::FROW, fcol = t % G::FROW;
            int gj = y0 - 2 + fry;
            if (sw_wrap(gj, n1, B.per[1]) >= 0) {
                fr0[q] = 3 + 2 * fcol + RX * fry;
                fpar[q] = (x0 - 1 + gj + first) & 1;
                fok[q] = (sw_wrap(x0 - 1 + 2 * fcol, n0, B.per[0]) >= 0 ? 1 : 0) |
                         (sw_wrap(x0 + 2 * fcol, n0, B.per[0]) >= 0 ? 2 : 0);
            }
        }
    }
    const int sry = 2 + tid / (kSwTX / 2);
    const int scol = tid % (kSwTX / 2);
    const int sgi = x0 + 2 * scol, sgj = y0 + sry - 2;
    const bool s_out = tid < G::SCELLS && sgi < n0 && sgj < n1;
    const int srl = 4 + 2 * scol + RX * sry;
    const int spar = (sgj + first) & 1;

    int coff[G::CPER];
    T cval[2][G::CPER];
    const int cn0 = n0 >> 1;
    const long cplane = (long)cn0 * (n1 >> 1);
#pragma unroll
    for (int q = 0; q < G::CPER; q++) {
        coff[q] = -1;
        cval[0][q] = cval[1][q] = (T)0;
        int e = tid + q * NT;
        if (xc && e < RP) {
            int gi = sw_wrap(x0 - 4 + e % RX, n0, B.per[0]);
            int gj = sw_wrap(y0 - 2 + e / RX, n1, B.per[1]);
            if (gi >= 0 && gj >= 0) coff[q] = (gi >> 1) + cn0 * (gj >> 1);
        }
    }
    auto fetch_coarse = [&](int h, int k) {
        int gk = sw_wrap(k, n2, B.per[2]);
        const T* cp = xc + cplane * (gk >> 1);
#pragma unroll
        for (int q = 0; q < G::CPER; q++) cval[h][q] = (gk >= 0 && coff[q] >= 0) ? cp[coff[q]] : (T)0;
    };
    auto add_coarse = [&](int h, int k) {
        T* d = rx_ + slot(k, G::XS) * RP;
#pragma unroll
        for (int q = 0; q < G::CPER; q++) {
            int e = tid + q * NT;
            if (e < RP) d[e] += cval[h][q];
        }
    };
    auto update = [&](int r, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk,
                      const T* czk, const T* czm) {
        T a1 = cxk[r - 1], a2 = cxk[r], a3 = cyk[r - RX], a4 = cyk[r], a5 = czm[r], a6 = czk[r];
        T out;
        const T x0 = v.omega != (T)1 ? xk[r] : (T)0;
        if (SwUpd<T>::apply(a1, a2, a3, a4, a5, a6, xk[r - 1], xk[r + 1], xk[r - RX], xk[r + RX], xm[r], xp[r], bk[r],
                            x0, v.omega, out))
            xk[r] = out;
    };
    auto f_at = [&](int k, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk, const T* czk,
                    const T* czm) {
        if (sw_wrap(k, n2, B.per[2]) < 0) return;
#pragma unroll
        for (int q = 0; q < G::FPER; q++) {
            if (fr0[q] < 0) continue;
            const int off = fpar[q] ^ (k & 1);
            if ((fok[q] >> off) & 1) update(fr0[q] + off, xk, xm, xp, cxk, cyk, bk, czk, czm);
        }
    };
    auto s_at = [&](int k, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk, const T* czk,
                    const T* czm) {
        if (k < z0 || k >= z1 || !s_out) return;
        const int rS = srl + ((spar ^ (k & 1)) ? 0 : 1);
        update(rS, xk, xm, xp, cxk, cyk, bk, czk, czm);
        float2 pr;
        pr.x = xk[srl];
        pr.y = xk[srl + 1];
        *reinterpret_cast<float2*>(xout + sgi + (long)n0 * sgj + plane * k) = pr;
    };

    __syncthreads();   // barriers initialised
    // prologue, waited for at once: group 0 = iterate z0-2..z0+1, cz z0-2,
    // coefficients z0-1 and z0
    {
        SwGroup<13> g0;
        for (int q = 0; q < 4; q++) set_x(g0, q, z0 - 2 + q, slot(z0 - 2 + q, G::XS));
        set_c(g0, 4, 4, z0 - 2, 0);
        for (int a = 1; a <= 4; a++) {
            set_c(g0, 4 + a, a, z0 - 1, 1);
            set_c(g0, 8 + a, a, z0, 2);
        }
        issue(g0, 0);
        land(g0, 0);
    }
    // step s waits for group s, issued by step s-1 with its wrapped elements
    // kept in registers
    SwGroup<10> gnext;
    int xb = G::XS - 1, cb = 0, zb = G::ZS - 1;
    int step = 0;
    for (int f0 = z0 - 1; f0 <= z1; f0 += 2, step++) {
        if (step > 0) land(gnext, step);
        __syncthreads();
        // slots of planes f0+3, f0+4 (iterate) and f0+2, f0+3 (coefficients):
        // those of planes f0-4, f0-3 and f0-3, f0-2
        set_x(gnext, 0, f0 + 3, sw_add(xb, -2, G::XS));
        set_x(gnext, 1, f0 + 4, sw_add(xb, -1, G::XS));
        for (int a = 1; a <= 3; a++) {
            set_c(gnext, 1 + a, a, f0 + 2, sw_add(cb, -2, G::CS));
            set_c(gnext, 5 + a, a, f0 + 3, sw_add(cb, -1, G::CS));
        }
        set_c(gnext, 5, 4, f0 + 2, sw_add(zb, -2, G::ZS));
        set_c(gnext, 9, 4, f0 + 3, sw_add(zb, -1, G::ZS));
        issue(gnext, step + 1);
        if (xc) {   // the iterate planes that arrived: group 0's, then two per step
            if (f0 == z0 - 1) {
                for (int k = z0 - 2; k <= z0 + 1; k++) {
                    fetch_coarse(0, k);
                    add_coarse(0, k);
                }
            } else {
                if (f0 + 1 <= z1 + 1) add_coarse(0, f0 + 1);
                if (f0 + 2 <= z1 + 1) add_coarse(1, f0 + 2);
            }
            fetch_coarse(0, f0 + 3);
            fetch_coarse(1, f0 + 4);
            __syncthreads();
        }
        T* const xm2 = rx_ + xb * RP;
        T* const xm1 = rx_ + sw_add(xb, 1, G::XS) * RP;
        T* const x0p = rx_ + sw_add(xb, 2, G::XS) * RP;
        T* const x1p = rx_ + sw_add(xb, 3, G::XS) * RP;
        T* const x2p = rx_ + sw_add(xb, 4, G::XS) * RP;
        const int c0 = sw_add(cb, 1, G::CS), c1 = sw_add(cb, 2, G::CS);
        const T* const zm2 = rcz + zb * RP;
        const T* const zm1 = rcz + sw_add(zb, 1, G::ZS) * RP;
        const T* const z0p = rcz + sw_add(zb, 2, G::ZS) * RP;
        const T* const z1p = rcz + sw_add(zb, 3, G::ZS) * RP;
        f_at(f0, x0p, xm1, x1p, rcx + c0 * RP, rcy + c0 * RP, rb + c0 * RP, z0p, zm1);
        if (f0 + 1 <= z1) f_at(f0 + 1, x1p, x0p, x2p, rcx + c1 * RP, rcy + c1 * RP, rb + c1 * RP, z1p, z0p);
        __syncthreads();
        s_at(f0 - 1, xm1, xm2, x0p, rcx + cb * RP, rcy + cb * RP, rb + cb * RP, zm1, zm2);
        s_at(f0, x0p, xm1, x1p, rcx + c0 * RP, rcy + c0 * RP, rb + c0 * RP, z0p, zm1);
        xb = sw_add(xb, 2, G::XS);
        cb = sw_add(cb, 2, G::CS);
        zb = sw_add(zb, 2, G::ZS);
        // the slots written above are overwritten by the copy engine later
        fence_proxy_async_smem();
    }
    // drain the last group issued (an empty one completes at once)
    if (!bad && !mbar_wait_bounded(s_bar0 + 8 * (step % NB), (uint32_t)((step / NB) & 1))) *(volatile int*)err = 1;
}
