// mg_sweep.cuh -- fused red-black Gauss-Seidel sweep of the B200 multigrid
// (included by mg_fast.cu after LV<T>).
//
// One full sweep (colour F = `first`, then the other colour S) in one pass
// over memory.  A block owns a kSwTX x kSwTY column of cells and marches up a
// chunk of planes with a wavefront:
//   step kk:  F at plane kk on the tile plus a one-cell ring (from the old
//             iterate), then S at plane kk-1 on the tile (from the new F
//             values of planes kk-2..kk); plane kk-1 is then final.
// Planes of the iterate (tile + ring) and of the coefficients are staged in
// shared memory with 16-byte cp.async, kSwDepth steps ahead of their use, so
// that enough bytes are in flight per SM to cover the HBM latency; each array
// is read from HBM once per sweep (the ring re-reads hit L2).  The iterate is
// read from `xin` (nullptr: zero) and written to `xout`, never in place, so
// blocks never see each other's new values and the sweep computes exactly the
// two colour passes of k_fast_smooth.  With `xc`, the coarse-grid correction
// (injection from the level below) is added to the iterate as it arrives.
//
// Requirements (checked by the host): n0 a multiple of 16 / sizeof(T) and all
// dimensions even (true of every level above the coarsest).
#pragma once

static constexpr int kSwTX = 32, kSwTY = 8;
static constexpr int kSwThreads = kSwTX * kSwTY;
static constexpr int kSwRX = kSwTX + 8;            // region: x0-4 .. x0+TX+3 (16-byte aligned rows)
static constexpr int kSwRY = kSwTY + 4;            // y0-2 .. y0+TY+1
static constexpr int kSwRP = kSwRX * kSwRY;
static constexpr int kSwDepth = 3;                 // planes staged ahead of use
// live planes: iterate kk-2..kk+1 (+ Depth in flight), coefficients kk-1..kk
// (+ Depth), cz kk-2..kk (+ Depth)
static constexpr int kSwXSlots = kSwDepth + 4, kSwCSlots = kSwDepth + 2, kSwZSlots = kSwDepth + 3;
static constexpr int kSwSlots = kSwXSlots + 3 * kSwCSlots + kSwZSlots;
static constexpr int kSwFCells = (kSwTX + 2) / 2 * (kSwTY + 2);   // F cells of tile + ring per plane (170)
static constexpr int kSwSCells = kSwTX / 2 * kSwTY;               // S cells of the tile per plane (128)
static constexpr int kSwCoarsePer = (kSwRP + kSwThreads - 1) / kSwThreads;

template <typename T>
static constexpr size_t sweep_smem() {
    return sizeof(T) * (size_t)kSwRP * kSwSlots;
}

template <typename T>
struct SwVec;
template <>
struct SwVec<float> { using V2 = float2; };
template <>
struct SwVec<double> { using V2 = double2; };

__device__ inline void cp_async16(uint32_t saddr, const void* g, int src_size) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(g), "r"(src_size) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ inline void cp_async_wait_all_groups() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// all but the newest kSwDepth-1 groups complete
__device__ inline void cp_async_wait_pipe() { asm volatile("cp.async.wait_group %0;\n" ::"n"(kSwDepth - 1) : "memory"); }

// wrap a coordinate into [0,n) (periodic) or return -1 outside a wall
__device__ inline int sw_wrap(int a, int n, int per) {
    if (a >= 0 && a < n) return a;
    if (!per) return -1;
    a %= n;
    return a < 0 ? a + n : a;
}

template <typename T>
__global__ void __launch_bounds__(kSwThreads, sizeof(T) == 4 ? 4 : 2)
    k_rb_sweep(const LV<T> v, const T* __restrict__ xin, T* __restrict__ xout, const T* __restrict__ xc, const Bnd B,
               int first, int zc) {
    constexpr int VEC = 16 / sizeof(T);             // elements per 16-byte chunk
    constexpr int RXC = kSwRX / VEC;                // chunks per region row
    constexpr int CH = RXC * kSwRY;                 // chunks per array plane
    constexpr int NA = 5;                           // arrays staged: x, cx, cy, b, cz
    constexpr int LPER = (NA * CH + kSwThreads - 1) / kSwThreads;
    extern __shared__ __align__(16) unsigned char sw_raw[];
    T* const sm = reinterpret_cast<T*>(sw_raw);
    // slot bases: iterate, then cx, cy, b (kSwCSlots each), then cz
    auto xslot = [&](int s) { return sm + s * kSwRP; };
    auto cslot = [&](int a, int s) { return sm + (kSwXSlots + (a - 1) * kSwCSlots + s) * kSwRP; };
    auto zslot = [&](int s) { return sm + (kSwXSlots + 3 * kSwCSlots + s) * kSwRP; };

    const int tid = threadIdx.x;
    const int n0 = v.n0, n1 = v.n1, n2 = v.n2;
    const long plane = (long)n0 * n1;
    const int x0 = blockIdx.x * kSwTX, y0 = blockIdx.y * kSwTY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, n2);
    const int kb = z0 - 2;   // planes are >= kb: slot of plane k = (k - kb) % slots

    // this thread's staged chunks, resolved once: the global address of the
    // chunk in plane 0 (nullptr: zero fill), the shared address of the chunk
    // in slot 0 of its ring, and the ring (0 iterate, 1 cx/cy/b, 2 cz)
    const T* gptr[LPER];
    uint32_t sdst[LPER];
    int kind[LPER];
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
#pragma unroll
    for (int q = 0; q < LPER; q++) {
        int idx = tid + q * kSwThreads;
        gptr[q] = nullptr;
        sdst[q] = 0;
        kind[q] = -1;
        if (idx < NA * CH) {
            int a = idx / CH, c = idx % CH;
            int ry = c / RXC, cxq = c % RXC;
            int gi = sw_wrap(x0 - 4 + VEC * cxq, n0, B.per[0]);
            int gj = sw_wrap(y0 - 2 + ry, n1, B.per[1]);
            const T* src = a == 0 ? xin : (a == 1 ? v.cx : (a == 2 ? v.cy : (a == 3 ? v.b : v.cz)));
            if (src && gi >= 0 && gj >= 0) gptr[q] = src + gi + (long)n0 * gj;
            int ring0 = a == 0 ? 0 : (a == 4 ? kSwXSlots + 3 * kSwCSlots : kSwXSlots + (a - 1) * kSwCSlots);
            sdst[q] = sbase + (uint32_t)(sizeof(T) * (ring0 * kSwRP + ry * kSwRX + VEC * cxq));
            kind[q] = a == 0 ? 0 : (a == 4 ? 2 : 1);
        }
    }
    constexpr uint32_t kSlotBytes = sizeof(T) * kSwRP;
    // issue the loads of iterate plane kx (if kx_on) and of the coefficients
    // of plane kc (cx, cy, b and cz if kc_on; cz alone if cz_only)
    auto stage = [&](int kx, bool kx_on, int kc, bool kc_on, bool cz_only) {
        const int gkx = sw_wrap(kx, n2, B.per[2]), gkc = sw_wrap(kc, n2, B.per[2]);
        const uint32_t offx = kSlotBytes * (uint32_t)((kx - kb) % kSwXSlots);
        const uint32_t offc = kSlotBytes * (uint32_t)((kc - kb) % kSwCSlots);
        const uint32_t offz = kSlotBytes * (uint32_t)((kc - kb) % kSwZSlots);
        const long px = plane * gkx, pc = plane * gkc;
#pragma unroll
        for (int q = 0; q < LPER; q++) {
            const int kd = kind[q];
            if (kd < 0) continue;
            if (kd == 0 ? !kx_on : (!kc_on || (cz_only && kd != 2))) continue;
            const bool ok = gptr[q] != nullptr && (kd == 0 ? gkx : gkc) >= 0;
            const T* g = ok ? gptr[q] + (kd == 0 ? px : pc) : v.b;
            cp_async16(sdst[q] + (kd == 0 ? offx : (kd == 1 ? offc : offz)), g, ok ? 16 : 0);
        }
    };

    // F cell of this thread (one per plane): ring row fry; the column of the
    // first F cell of the row depends on the plane's parity
    const bool fon = tid < kSwFCells;
    const int fry = 1 + tid / ((kSwTX + 2) / 2);     // region row 1..TY+2
    const int fcol = tid % ((kSwTX + 2) / 2);
    const int fgj = y0 - 2 + fry;
    const bool fj_ok = fon && sw_wrap(fgj, n1, B.per[1]) >= 0;
    // S cell: one of the pair of tile columns 2c, 2c+1 in tile row sry
    const bool son = tid < kSwSCells;
    const int sry = 2 + tid / (kSwTX / 2);
    const int sc = tid % (kSwTX / 2);
    const int sgi = x0 + 2 * sc, sgj = y0 + sry - 2;
    const bool s_out = son && sgi < n0 && sgj < n1;

    // parent offsets for the coarse-grid correction of the staged iterate
    long coff[kSwCoarsePer];
    const int cn0 = n0 >> 1;
    const long cplane = (long)cn0 * (n1 >> 1);
    if (xc) {
#pragma unroll
        for (int q = 0; q < kSwCoarsePer; q++) {
            int e = tid + q * kSwThreads;
            coff[q] = -1;
            if (e < kSwRP) {
                int gi = sw_wrap(x0 - 4 + e % kSwRX, n0, B.per[0]);
                int gj = sw_wrap(y0 - 2 + e / kSwRX, n1, B.per[1]);
                if (gi >= 0 && gj >= 0) coff[q] = (gi >> 1) + (long)cn0 * (gj >> 1);
            }
        }
    }
    auto add_coarse = [&](int k) {
        int gk = sw_wrap(k, n2, B.per[2]);
        if (gk < 0) return;
        T* d = xslot((k - kb) % kSwXSlots);
        const T* cp = xc + cplane * (gk >> 1);
#pragma unroll
        for (int q = 0; q < kSwCoarsePer; q++) {
            int e = tid + q * kSwThreads;
            if (e < kSwRP && coff[q] >= 0) d[e] += cp[coff[q]];
        }
    };

    // point update of region cell r of plane xk (same formula and operation
    // order as smooth_cell)
    auto update = [&](int r, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk,
                      const T* czk, const T* czm) {
        T a1 = cxk[r - 1], a2 = cxk[r], a3 = cyk[r - kSwRX], a4 = cyk[r], a5 = czm[r], a6 = czk[r];
        T d = a1 + a2 + a3 + a4 + a5 + a6;
        T s = a1 * xk[r - 1] + a2 * xk[r + 1] + a3 * xk[r - kSwRX] + a4 * xk[r + kSwRX] + a5 * xm[r] + a6 * xp[r] +
              bk[r];
        if (d > (T)0) xk[r] = s / d;
    };

    // prologue.  Group 0: iterate planes z0-2..z0, coefficients of plane z0-1,
    // cz of plane z0-2.  Groups 1..Depth-1: iterate plane z0+j, coefficients
    // of plane z0-1+j (what step kk issues for kk = z0-1-Depth+j).
    stage(z0 - 2, true, z0 - 2, true, true);
    stage(z0 - 1, true, z0 - 1, true, false);
    stage(z0, true, 0, false, false);
    cp_async_commit();
#pragma unroll
    for (int j = 1; j < kSwDepth; j++) {
        stage(z0 + j, z0 + j <= z1 + 1, z0 - 1 + j, z0 - 1 + j <= z1, false);
        cp_async_commit();
    }

    for (int kk = z0 - 1; kk <= z1; kk++) {
        cp_async_wait_pipe();   // the group carrying iterate kk+1 and coefficients kk
        __syncthreads();
        stage(kk + 1 + kSwDepth, kk + 1 + kSwDepth <= z1 + 1, kk + kSwDepth, kk + kSwDepth <= z1, false);
        cp_async_commit();
        if (xc) {   // the planes that arrived: group 0's, then one per step
            if (kk == z0 - 1)
                for (int k = z0 - 2; k <= z0; k++) add_coarse(k);
            else
                add_coarse(kk + 1);
            __syncthreads();
        }
        const int o = kk - kb;   // >= 1
        T* xkm1 = xslot((o - 1) % kSwXSlots);
        T* xk = xslot(o % kSwXSlots);
        T* xkp1 = xslot((o + 1) % kSwXSlots);
        // F at plane kk on the tile + ring
        const int gk = sw_wrap(kk, n2, B.per[2]);
        if (gk >= 0 && fj_ok) {
            int off = ((x0 - 1 + fgj + kk + first) & 1);   // is column x0-1 of this row F?
            int rx = 3 + 2 * fcol + off;
            if (sw_wrap(x0 - 4 + rx, n0, B.per[0]) >= 0) {
                const int c1 = o % kSwCSlots;
                update(rx + kSwRX * fry, xk, xkm1, xkp1, cslot(1, c1), cslot(2, c1), cslot(3, c1),
                       zslot(o % kSwZSlots), zslot((o - 1) % kSwZSlots));
            }
        }
        __syncthreads();
        // S at plane kk-1 on the tile; store the finished pair of plane kk-1
        const int ks = kk - 1;
        if (ks >= z0 && s_out) {
            const int os = o - 1;
            T* xs_ = xslot(os % kSwXSlots);
            int rl = 4 + 2 * sc + kSwRX * sry;                     // left cell of the pair
            int rS = rl + (((sgj + ks + first) & 1) ? 0 : 1);      // the S cell of the pair
            const int c2 = os % kSwCSlots;
            update(rS, xs_, xslot((os - 1) % kSwXSlots), xk, cslot(1, c2), cslot(2, c2), cslot(3, c2),
                   zslot(os % kSwZSlots), zslot((os - 1) % kSwZSlots));
            using V2 = typename SwVec<T>::V2;
            V2 pr;
            pr.x = xs_[rl];
            pr.y = xs_[rl + 1];
            *reinterpret_cast<V2*>(xout + sgi + (long)n0 * sgj + plane * ks) = pr;
        }
    }
    cp_async_wait_all_groups();
}
