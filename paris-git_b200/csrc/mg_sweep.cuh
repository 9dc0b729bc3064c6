// mg_sweep.cuh -- fused red-black Gauss-Seidel sweep of the B200 multigrid
// (included by mg_fast.cu after LV<T>).
//
// One full sweep (colour F = `first`, then the other colour S) in one pass
// over memory.  A block owns a kSwTX x TY column of cells and marches up a
// chunk of planes with a wavefront:
//   step kk:  F at plane kk on the tile plus a one-cell ring (from the old
//             iterate), then S at plane kk-1 on the tile (from the new F
//             values of planes kk-2..kk); plane kk-1 is then final.
// Planes of the iterate (tile + two-cell ring) and of the coefficients are
// staged in shared memory with 16-byte cp.async, D steps ahead of their use,
// so that enough bytes are in flight per SM to cover the HBM latency; each
// array is read from HBM once per sweep (the ring re-reads hit L2).  The
// iterate is read from `xin` (nullptr: zero) and written to `xout`, never in
// place, so blocks never see each other's new values and the sweep computes
// exactly the two colour passes of k_fast_smooth.  With `xc`, the coarse-grid
// correction (injection from the level below) is added to the iterate as it
// arrives.  Ring-buffer slots rotate with the step; the per-step work outside
// the point updates is a handful of integer operations per thread.
//
// Requirements (checked by the host): n0 a multiple of 16 / sizeof(T) and all
// dimensions even (true of every level above the coarsest).
#pragma once

static constexpr int kSwTX = 32;

// a configuration: element type, tile height, planes staged ahead, threads
// per block and blocks per SM the registers are budgeted for
template <typename T_, int TY_, int D_, int NT_, int MINB_>
struct SwCfg {
    using type = T_;
    static constexpr int TY = TY_, D = D_, NT = NT_, MINB = MINB_;
};
// the configurations the solver uses
template <typename T>
struct SwGeo;
template <>
struct SwGeo<float> {
    using Cfg = SwCfg<float, 16, 2, 320, 3>;   // 512 cells per plane step, three blocks per SM
};
template <>
struct SwGeo<double> {
    using Cfg = SwCfg<double, 8, 3, 256, 2>;   // two blocks per SM within shared memory
};

template <class C>
struct Sw {
    using T = typename C::type;
    static constexpr int NT = C::NT;
    static constexpr int TY = C::TY;
    static constexpr int D = C::D;                    // planes staged ahead of use
    static constexpr int RX = kSwTX + 8;              // region x0-4 .. x0+TX+3 (16-byte aligned rows)
    static constexpr int RY = TY + 4;                 // y0-2 .. y0+TY+1
    static constexpr int RP = RX * RY;
    // live planes: iterate kk-2..kk+1, coefficients kk-1..kk, cz kk-2..kk,
    // each plus D in flight
    static constexpr int XS = D + 4, CS = D + 2, ZS = D + 3;
    static constexpr int SLOTS = XS + 3 * CS + ZS;
    static constexpr int FROW = (kSwTX + 2) / 2;      // F cells per ring row
    static constexpr int FCELLS = FROW * (TY + 2);
    static constexpr int FPER = (FCELLS + NT - 1) / NT;
    static constexpr int SCELLS = kSwTX / 2 * TY;     // S cells (= output pairs) of the tile
    static constexpr int VEC = 16 / sizeof(T);
    static constexpr int RXC = RX / VEC;
    static constexpr int CH = RXC * RY;               // 16-byte chunks per array plane
    static constexpr int CPER = (RP + NT - 1) / NT;
    static constexpr uint32_t SLOT_BYTES = sizeof(T) * RP;
    static_assert(SCELLS <= NT, "one output pair per thread");
};

template <class C>
static constexpr size_t sweep_smem_cfg() {
    return sizeof(typename C::type) * (size_t)Sw<C>::RP * Sw<C>::SLOTS;
}

template <typename T>
static constexpr size_t sweep_smem() {
    return sweep_smem_cfg<typename SwGeo<T>::Cfg>();
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
// all but the newest N groups complete
template <int N>
__device__ inline void cp_async_wait_newest() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// wrap a coordinate into [0,n) (periodic) or return -1 outside a wall
__device__ inline int sw_wrap(int a, int n, int per) {
    if (a >= 0 && a < n) return a;
    if (!per) return -1;
    a %= n;
    return a < 0 ? a + n : a;
}

__device__ inline int sw_next(int s, int S) { return s + 1 == S ? 0 : s + 1; }
// (s + d) mod S for |d| < S
__device__ inline int sw_add(int s, int d, int S) {
    s += d;
    return s >= S ? s - S : (s < 0 ? s + S : s);
}

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB)
    k_rb_sweep_cfg(const LV<typename C::type> v, const typename C::type* __restrict__ xin,
                   typename C::type* __restrict__ xout, const typename C::type* __restrict__ xc, const Bnd B, int first,
                   int zc) {
    using T = typename C::type;
    using G = Sw<C>;
    constexpr int NT = G::NT;
    constexpr int RX = G::RX, RP = G::RP, TY = G::TY, VEC = G::VEC;
    static_assert(G::CH <= NT, "one chunk of each array per thread");
    extern __shared__ __align__(16) unsigned char sw_raw[];
    T* const sm = reinterpret_cast<T*>(sw_raw);
    // rings: iterate (XS slots), cx, cy, b (CS slots each), cz (ZS slots)
    T* const rx_ = sm;
    T* const rcx = sm + G::XS * RP;
    T* const rcy = rcx + G::CS * RP;
    T* const rb = rcy + G::CS * RP;
    T* const rcz = rb + G::CS * RP;

    const int tid = threadIdx.x;
    const int n0 = v.n0, n1 = v.n1, n2 = v.n2;
    const long plane = (long)n0 * n1;
    const int x0 = blockIdx.x * kSwTX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, n2);
    const int kb = z0 - 2;   // first staged plane: slot of plane k = (k - kb) mod ring size

    // the 16-byte chunk this thread stages of every array plane: its byte
    // offset within a slot and its in-plane element offset (-1: zero fill)
    const bool ld = tid < G::CH;
    uint32_t creg = 0;
    long cin = -1;
    if (ld) {
        int ry = tid / G::RXC, cxq = tid % G::RXC;
        int gi = sw_wrap(x0 - 4 + VEC * cxq, n0, B.per[0]);
        int gj = sw_wrap(y0 - 2 + ry, n1, B.per[1]);
        creg = (uint32_t)(sizeof(T) * (ry * RX + VEC * cxq));
        if (gi >= 0 && gj >= 0) cin = gi + (long)n0 * gj;
    }
    const uint32_t s_x = (uint32_t)__cvta_generic_to_shared(rx_) + creg;
    const uint32_t s_cx = (uint32_t)__cvta_generic_to_shared(rcx) + creg;
    const uint32_t s_cy = (uint32_t)__cvta_generic_to_shared(rcy) + creg;
    const uint32_t s_b = (uint32_t)__cvta_generic_to_shared(rb) + creg;
    const uint32_t s_cz = (uint32_t)__cvta_generic_to_shared(rcz) + creg;
    auto copy = [&](uint32_t sa, const T* base, int gk) {
        bool ok = base != nullptr && cin >= 0 && gk >= 0;
        cp_async16(sa, ok ? base + cin + plane * gk : v.b, ok ? 16 : 0);
    };
    // issue the loads of iterate plane kx into slot sx (if kx_on) and of the
    // coefficients of plane kc into slots sc (cx, cy, b) and sz (cz)
    // (if kc_on; cz alone if cz_only)
    auto stage = [&](int kx, int sx, bool kx_on, int kc, int sc, int sz, bool kc_on, bool cz_only) {
        if (!ld) return;
        if (kx_on) copy(s_x + G::SLOT_BYTES * sx, xin, sw_wrap(kx, n2, B.per[2]));
        if (kc_on) {
            const int gk = sw_wrap(kc, n2, B.per[2]);
            if (!cz_only) {
                const uint32_t oc = G::SLOT_BYTES * sc;
                copy(s_cx + oc, v.cx, gk);
                copy(s_cy + oc, v.cy, gk);
                copy(s_b + oc, v.b, gk);
            }
            copy(s_cz + G::SLOT_BYTES * sz, v.cz, gk);
        }
    };

    // F cells of this thread (FPER per plane): region index of the even
    // candidate column, parity of (x0-1, row) against `first`, and which of
    // the two candidate columns is a real cell (bit 0: even, bit 1: odd)
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
    // the output pair of this thread: tile columns 2c, 2c+1 of tile row sry
    const int sry = 2 + tid / (kSwTX / 2);
    const int scol = tid % (kSwTX / 2);
    const int sgi = x0 + 2 * scol, sgj = y0 + sry - 2;
    const bool s_out = tid < G::SCELLS && sgi < n0 && sgj < n1;
    const int srl = 4 + 2 * scol + RX * sry;           // left cell of the pair
    const int spar = (sgj + first) & 1;

    // coarse-grid correction: parents of the iterate elements of this thread
    // (in-plane offset, -1 outside a wall), fetched into registers one step
    // before the plane is added to
    int coff[G::CPER];
    T cval[G::CPER];
    const int cn0 = n0 >> 1;
    const long cplane = (long)cn0 * (n1 >> 1);
#pragma unroll
    for (int q = 0; q < G::CPER; q++) {
        coff[q] = -1;
        cval[q] = (T)0;
        int e = tid + q * NT;
        if (xc && e < RP) {
            int gi = sw_wrap(x0 - 4 + e % RX, n0, B.per[0]);
            int gj = sw_wrap(y0 - 2 + e / RX, n1, B.per[1]);
            if (gi >= 0 && gj >= 0) coff[q] = (gi >> 1) + cn0 * (gj >> 1);
        }
    }
    auto fetch_coarse = [&](int k) {
        int gk = sw_wrap(k, n2, B.per[2]);
        const T* cp = xc + cplane * (gk >> 1);
#pragma unroll
        for (int q = 0; q < G::CPER; q++) cval[q] = (gk >= 0 && coff[q] >= 0) ? cp[coff[q]] : (T)0;
    };
    auto add_coarse = [&](int slot) {
        T* d = rx_ + slot * RP;
#pragma unroll
        for (int q = 0; q < G::CPER; q++) {
            int e = tid + q * NT;
            if (e < RP) d[e] += cval[q];
        }
    };

    // point update of region cell r in plane xk (formula and operation order
    // of smooth_cell)
    auto update = [&](int r, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk,
                      const T* czk, const T* czm) {
        T a1 = cxk[r - 1], a2 = cxk[r], a3 = cyk[r - RX], a4 = cyk[r], a5 = czm[r], a6 = czk[r];
        T d = a1 + a2 + a3 + a4 + a5 + a6;
        T s = a1 * xk[r - 1] + a2 * xk[r + 1] + a3 * xk[r - RX] + a4 * xk[r + RX] + a5 * xm[r] + a6 * xp[r] + bk[r];
        if (d > (T)0) xk[r] = s / d;
    };

    // prologue.  Group 0: iterate planes z0-2..z0 (slots 0..2), coefficients
    // of plane z0-1 (slot 1), cz of plane z0-2 (slot 0).  Groups 1..D-1:
    // iterate plane z0+j and coefficients of plane z0-1+j, as a step issues.
    stage(z0 - 2, 0, true, z0 - 2, 0, 0, true, true);
    stage(z0 - 1, 1, true, z0 - 1, 1, 1, true, false);
    stage(z0, 2, true, 0, 0, 0, false, false);
    cp_async_commit();
#pragma unroll
    for (int j = 1; j < G::D; j++) {
        stage(z0 + j, (j + 2) % G::XS, z0 + j <= z1 + 1, z0 - 1 + j, (j + 1) % G::CS, (j + 1) % G::ZS, z0 - 1 + j <= z1,
              false);
        cp_async_commit();
    }

    // ring positions of plane kk-1 in the iterate, coefficient and cz rings
    int xs1 = 0, cs1 = 0, zs1 = 0;
    for (int kk = z0 - 1; kk <= z1; kk++) {
        cp_async_wait_newest<G::D - 1>();   // the group carrying iterate kk+1 and coefficients kk
        __syncthreads();
        // iterate plane kk+1+D and coefficients of plane kk+D into the slots
        // freed by planes kk-3 (iterate, cz) and kk-2 (coefficients)
        stage(kk + 1 + G::D, sw_add(xs1, -2, G::XS), kk + 1 + G::D <= z1 + 1, kk + G::D, sw_add(cs1, -1, G::CS),
              sw_add(zs1, -2, G::ZS), kk + G::D <= z1, false);
        cp_async_commit();
        const int xk0 = sw_next(xs1, G::XS), xkp = sw_add(xs1, 2, G::XS);
        if (xc) {   // the planes that arrived: group 0's, then one per step
            if (kk == z0 - 1) {
                for (int k = 0; k < 3; k++) {
                    fetch_coarse(z0 - 2 + k);
                    add_coarse(k);
                }
            } else {
                add_coarse(xkp);
            }
            fetch_coarse(kk + 2);   // for the plane that arrives next step
            __syncthreads();
        }
        T* const xm1 = rx_ + xs1 * RP;       // plane kk-1
        T* const xk = rx_ + xk0 * RP;        // plane kk
        // F at plane kk on the tile + ring
        if (sw_wrap(kk, n2, B.per[2]) >= 0) {
            const int ck = sw_next(cs1, G::CS);
            const T* cxk = rcx + ck * RP;
            const T* cyk = rcy + ck * RP;
            const T* bk = rb + ck * RP;
            const T* czk = rcz + sw_next(zs1, G::ZS) * RP;
            const T* czm = rcz + zs1 * RP;
            const T* xp = rx_ + xkp * RP;
#pragma unroll
            for (int q = 0; q < G::FPER; q++) {
                if (fr0[q] < 0) continue;
                const int off = fpar[q] ^ (kk & 1);
                if ((fok[q] >> off) & 1) update(fr0[q] + off, xk, xm1, xp, cxk, cyk, bk, czk, czm);
            }
        }
        __syncthreads();
        // S at plane kk-1 on the tile; store the finished pair of plane kk-1
        const int ks = kk - 1;
        if (ks >= z0 && s_out) {
            const T* xm2 = rx_ + sw_add(xs1, -1, G::XS) * RP;   // plane kk-2
            const int rS = srl + ((spar ^ (ks & 1)) ? 0 : 1);
            update(rS, xm1, xm2, xk, rcx + cs1 * RP, rcy + cs1 * RP, rb + cs1 * RP, rcz + zs1 * RP,
                   rcz + sw_add(zs1, -1, G::ZS) * RP);
            using V2 = typename SwVec<T>::V2;
            V2 pr;
            pr.x = xm1[srl];
            pr.y = xm1[srl + 1];
            *reinterpret_cast<V2*>(xout + sgi + (long)n0 * sgj + plane * ks) = pr;
        }
        xs1 = xk0;
        cs1 = sw_next(cs1, G::CS);
        zs1 = sw_next(zs1, G::ZS);
    }
    cp_async_wait_all_groups();
}
