// mg_sweep.cuh -- fused red-black Gauss-Seidel sweep of the B200 multigrid
// (included by mg_fast.cu after LV<T>).
//
// One full sweep (colour F = `first`, then the other colour S) in one pass
// over memory.  A block owns a TX x TY column of cells and marches up a
// chunk of planes with a wavefront, two planes per step:
//   step (f0, f1 = f0+1):  F at planes f0 and f1 on the tile plus a one-cell
//             ring (from the old iterate), then S at planes f0-1 and f0 on the
//             tile (from the new F values of the planes around them); planes
//             f0-1 and f0 are then final and stored.
// Planes of the iterate (tile + two-cell ring) and of the coefficients are
// staged in shared memory with 16-byte cp.async, D steps ahead of their use,
// so that enough bytes are in flight per SM to cover the HBM latency; each
// array is read from HBM once per sweep (the ring re-reads hit L2).  The
// iterate is read from `xin` (nullptr: zero) and written to `xout`, never in
// place, so blocks never see each other's new values and the sweep computes
// the two colour passes of k_fast_smooth (in FP64 exactly; in FP32 with the
// update arithmetic of SwUpd<float>).  With `xc`, the coarse-grid
// correction (injection from the level below) is added to the iterate as it
// arrives, fetched into registers one step ahead.  Ring-buffer slots rotate
// with the step.
//
// With bx_part, the sweep also sums b x over the cells it stores (in FP64) and
// writes one partial per block: on the last sweep of a V-cycle on the finest
// level that is r.z, the dot product the CG needs next.
//
// Requirements (checked by the host): n0 a multiple of 16 / sizeof(T) and all
// dimensions even (true of every level above the coarsest).
#pragma once

static constexpr int kSwTX = 32;

// a configuration: element type, tile height, steps staged ahead, threads
// per block, blocks per SM the registers are budgeted for, tile width
template <typename T_, int TY_, int D_, int NT_, int MINB_, int TX_ = kSwTX>
struct SwCfg {
    using type = T_;
    static constexpr int TY = TY_, D = D_, NT = NT_, MINB = MINB_, TX = TX_;
};
// the configurations the solver uses
template <typename T>
struct SwGeo;
template <>
struct SwGeo<float> {
    using Cfg = SwCfg<float, 16, 1, 320, 2>;   // 32x16 tiles, two planes staged ahead, two blocks per SM
};
template <>
struct SwGeo<double> {
    using Cfg = SwCfg<double, 8, 1, 256, 2>;   // 32x8 tiles: two blocks per SM within shared memory
};
// the merged-phase form (FP32, opt-in): its deeper rings fit two blocks per
// SM with 32x12 or 32x14 tiles
using SwMCfg12 = SwCfg<float, 12, 1, 256, 2>;
using SwMCfg14 = SwCfg<float, 14, 1, 288, 2>;

template <class C, bool M = false>
static constexpr size_t sweep2_smem_cfg();
template <typename T>
static constexpr size_t sweep_smem() {
    return sweep2_smem_cfg<typename SwGeo<T>::Cfg>();
}

// VEC/2 coarse values of a staged chunk, loaded together
template <typename T, int N>
struct SwCVec;
template <>
struct SwCVec<float, 2> {
    using V = float2;
    __device__ static V zero() { return make_float2(0.f, 0.f); }
};
template <>
struct SwCVec<double, 1> {
    using V = double;
    __device__ static V zero() { return 0.0; }
};

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

// The Gauss-Seidel update x = s / d of one cell.  FP32 (the inner cycle of
// the mixed solver): the sums as trees of depth three instead of chains of
// seven dependent adds, and the fast division (two ulps); the smoother only
// has to reduce the error, the FP64 outer loop keeps the residual exact.
// FP64: the sums in the order of A1..A6 and the IEEE division.
template <typename T>
struct SwUpd {
    __device__ static inline bool apply(T a1, T a2, T a3, T a4, T a5, T a6, T x1, T x2, T x3, T x4, T x5, T x6, T b,
                                        T x0, T w, T& out) {
        T d = a1 + a2 + a3 + a4 + a5 + a6;
        T s = a1 * x1 + a2 * x2 + a3 * x3 + a4 * x4 + a5 * x5 + a6 * x6 + b;
        if (d > (T)0) { out = relax(s / d, x0, w); return true; }
        return false;
    }
};
template <>
struct SwUpd<float> {
    __device__ static inline bool apply(float a1, float a2, float a3, float a4, float a5, float a6, float x1,
                                        float x2, float x3, float x4, float x5, float x6, float b, float x0, float w,
                                        float& out) {
        const float d = ((a1 + a2) + (a3 + a4)) + (a5 + a6);
        const float s = ((a1 * x1 + a2 * x2) + (a3 * x3 + a4 * x4)) + ((a5 * x5 + a6 * x6) + b);
        if (d > 0.f) { out = relax(__fdividef(s, d), x0, w); return true; }
        return false;
    }
};

__device__ inline int sw_next(int s, int S) { return s + 1 == S ? 0 : s + 1; }
// (s + d) mod S for |d| < S
__device__ inline int sw_add(int s, int d, int S) {
    s += d;
    return s >= S ? s - S : (s < 0 ? s + S : s);
}

// ---------------------------------------------------------------------------
// Step s works on f0 = z0-1+2s and f1 = f0+1; the barriers and the ring
// bookkeeping of a step are shared by two planes, and each thread has two
// independent updates per phase.  Live planes: iterate f0-2..f1+1,
// coefficients f0-1..f1, cz f0-2..f1, each plus 2D staged ahead.
//
// M (merged phases): the second colour of step s-1 (planes f0-3, f0-2) and
// the first colour of step s (planes f0, f0+1) run in one phase between two
// barriers.  They touch disjoint cells: the first colour writes its cells of
// planes f0, f0+1 and reads second-colour cells of planes f0-1..f0+2, which
// the second colour of step s-1 does not write; that one writes its cells of
// planes f0-3, f0-2 and reads first-colour cells of planes f0-4..f0-1, final
// since the phases before.  One barrier per step instead of two, for a ring
// two planes deeper (iterate f0-4..f0+2, coefficients f0-3..f0+1, cz
// f0-4..f0+1, plus 2D staged ahead).
template <class C, bool M = false>
struct Sw2 {
    using T = typename C::type;
    static constexpr int NT = C::NT, TY = C::TY, D = C::D;
    static constexpr int TX = C::TX;
    static constexpr int RX = TX + 8, RY = TY + 4, RP = RX * RY;
    static constexpr int XS = (M ? 7 : 5) + 2 * D, CS = (M ? 5 : 3) + 2 * D, ZS = (M ? 6 : 4) + 2 * D;
    static constexpr int SLOTS = XS + 3 * CS + ZS;
    static constexpr int FROW = (TX + 2) / 2;
    static constexpr int FCELLS = FROW * (TY + 2);
    static constexpr int FPER = (FCELLS + NT - 1) / NT;
    static constexpr int SCELLS = TX / 2 * TY;
    static constexpr int VEC = 16 / sizeof(T);
    static constexpr int RXC = RX / VEC;
    static constexpr int CH = RXC * RY;
    static constexpr int CPER = (RP + NT - 1) / NT;
    static constexpr uint32_t SLOT_BYTES = sizeof(T) * RP;
    static_assert(SCELLS <= NT, "one output pair per thread");
    static_assert(CH <= NT, "one chunk of each array per thread");
};

template <class C, bool M>
static constexpr size_t sweep2_smem_cfg() {
    return sizeof(typename C::type) * (size_t)Sw2<C, M>::RP * Sw2<C, M>::SLOTS;
}

template <class C, bool M = false>
__global__ void __launch_bounds__(C::NT, C::MINB)
    k_rb_sweep2_cfg(const LV<typename C::type> v, const typename C::type* __restrict__ xin,
                    typename C::type* __restrict__ xout, const typename C::type* __restrict__ xc, const Bnd B,
                    int first, int zc, double* __restrict__ bx_part) {
    using T = typename C::type;
    using G = Sw2<C, M>;
    constexpr int NT = G::NT;
    constexpr int RX = G::RX, RP = G::RP, TY = G::TY, VEC = G::VEC;
    extern __shared__ __align__(16) unsigned char sw_raw[];
    T* const sm = reinterpret_cast<T*>(sw_raw);
    T* const rx_ = sm;
    T* const rcx = sm + G::XS * RP;
    T* const rcy = rcx + G::CS * RP;
    T* const rb = rcy + G::CS * RP;
    T* const rcz = rb + G::CS * RP;

    const int tid = threadIdx.x;
    const int n0 = v.n0, n1 = v.n1, n2 = v.n2;
    const long plane = (long)n0 * n1;
    const int x0 = blockIdx.x * G::TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, n2);
    const int kb = z0 - 2;   // slot of plane k in a ring of S slots: (k - kb) % S
    auto slot = [&](int k, int S) { return (k - kb) % S; };

    // the 16-byte chunk this thread stages of every array plane: shared
    // address in slot 0 of each ring and global address in plane 0 (valid
    // only when the chunk lies in the domain or its periodic image)
    const bool ld = tid < G::CH;
    uint32_t creg = 0;
    long cin = 0;
    bool cok = false;
    if (ld) {
        int ry = tid / G::RXC, cxq = tid % G::RXC;
        int gi = sw_wrap(x0 - 4 + VEC * cxq, n0, B.per[0]);
        int gj = sw_wrap(y0 - 2 + ry, n1, B.per[1]);
        creg = (uint32_t)(sizeof(T) * (ry * RX + VEC * cxq));
        if (gi >= 0 && gj >= 0) {
            cin = gi + (long)n0 * gj;
            cok = true;
        }
    }
    const uint32_t s_x = (uint32_t)__cvta_generic_to_shared(rx_) + creg;
    const uint32_t s_cx = (uint32_t)__cvta_generic_to_shared(rcx) + creg;
    const uint32_t s_cy = (uint32_t)__cvta_generic_to_shared(rcy) + creg;
    const uint32_t s_b = (uint32_t)__cvta_generic_to_shared(rb) + creg;
    const uint32_t s_cz = (uint32_t)__cvta_generic_to_shared(rcz) + creg;
    const T* const g_x = xin ? xin + cin : v.b;
    const T* const g_cx = v.cx + cin;
    const T* const g_cy = v.cy + cin;
    const T* const g_b = v.b + cin;
    const T* const g_cz = v.cz + cin;
    const bool xok = cok && xin != nullptr;
    // iterate plane k into slot sx (k above z1+1 is never needed)
    auto stage_x = [&](int k, int sx) {
        if (!ld || k > z1 + 1) return;
        const int gk = sw_wrap(k, n2, B.per[2]);
        const bool ok = xok && gk >= 0;
        cp_async16(s_x + G::SLOT_BYTES * sx, ok ? g_x + plane * gk : v.b, ok ? 16 : 0);
    };
    // coefficients of plane k into slot sc (cx, cy, b) and sz (cz), or cz alone
    auto stage_c = [&](int k, int sc, int sz, bool cz_only) {
        if (!ld || k > z1) return;
        const int gk = sw_wrap(k, n2, B.per[2]);
        const bool ok = cok && gk >= 0;
        const long po = ok ? plane * gk : 0;
        const int nb = ok ? 16 : 0;
        if (!cz_only) {
            const uint32_t oc = G::SLOT_BYTES * sc;
            cp_async16(s_cx + oc, ok ? g_cx + po : v.b, nb);
            cp_async16(s_cy + oc, ok ? g_cy + po : v.b, nb);
            cp_async16(s_b + oc, ok ? g_b + po : v.b, nb);
        }
        cp_async16(s_cz + G::SLOT_BYTES * sz, ok ? g_cz + po : v.b, nb);
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
    const int sry = 2 + tid / (G::TX / 2);
    const int scol = tid % (G::TX / 2);
    const int sgi = x0 + 2 * scol, sgj = y0 + sry - 2;
    const bool s_out = tid < G::SCELLS && sgi < n0 && sgj < n1;
    const int srl = 4 + 2 * scol + RX * sry;
    const int spar = (sgj + first) & 1;

    // coarse-grid correction of the chunks this thread stages: VEC/2 coarse
    // values per chunk and plane (a chunk starts at an even cell and stays in
    // one row), fetched one step ahead and added to the thread's own chunks as
    // they arrive, before the barrier that publishes them
    constexpr int CV = VEC / 2;
    using CVec = typename SwCVec<T, CV>::V;
    const bool cload = xc != nullptr && ld && cok;
    const int cn0 = n0 >> 1;
    const long cplane = (long)cn0 * (n1 >> 1);
    long ccoff = 0;
    if (cload) ccoff = ((cin % n0) >> 1) + (long)cn0 * ((cin / n0) >> 1);
    CVec cval[2];
    auto fetch_coarse = [&](int h, int k) {
        const int gk = sw_wrap(k, n2, B.per[2]);
        if (cload && gk >= 0)
            cval[h] = *reinterpret_cast<const CVec*>(xc + cplane * (gk >> 1) + ccoff);
        else
            cval[h] = SwCVec<T, CV>::zero();
    };
    auto add_coarse = [&](int h, int k) {
        if (!cload) return;
        T* d = rx_ + slot(k, G::XS) * RP + creg / sizeof(T);
        const T* c = reinterpret_cast<const T*>(&cval[h]);
#pragma unroll
        for (int e = 0; e < VEC; e++) d[e] += c[e >> 1];
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
    // F at plane k (tile + ring) and S at plane k (tile) with its output; the
    // slot pointers of the planes involved are passed in
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
    double bx = 0.0;   // with bx_part: sum of b x over the cells this thread stores
    auto s_at = [&](int k, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk, const T* czk,
                    const T* czm) {
        if (k < z0 || k >= z1 || !s_out) return;
        const int rS = srl + ((spar ^ (k & 1)) ? 0 : 1);
        update(rS, xk, xm, xp, cxk, cyk, bk, czk, czm);
        using V2 = typename SwVec<T>::V2;
        V2 pr;
        pr.x = xk[srl];
        pr.y = xk[srl + 1];
        *reinterpret_cast<V2*>(xout + sgi + (long)n0 * sgj + plane * k) = pr;
        if (bx_part) bx += (double)bk[srl] * (double)pr.x + (double)bk[srl + 1] * (double)pr.y;
    };

    // prologue: group 0 = iterate z0-2..z0+1, coefficients z0-1, z0, cz z0-2;
    // group g (1..D-1) = iterate z0+2g, z0+2g+1 and coefficients z0-1+2g, z0+2g
    for (int k = z0 - 2; k <= z0 + 1; k++) stage_x(k, slot(k, G::XS));
    stage_c(z0 - 2, 0, 0, true);
    stage_c(z0 - 1, 1, 1, false);
    stage_c(z0, 2, 2, false);
    cp_async_commit();
#pragma unroll
    for (int g = 1; g < G::D; g++) {
        stage_x(z0 + 2 * g, slot(z0 + 2 * g, G::XS));
        stage_x(z0 + 2 * g + 1, slot(z0 + 2 * g + 1, G::XS));
        stage_c(z0 - 1 + 2 * g, slot(z0 - 1 + 2 * g, G::CS), slot(z0 - 1 + 2 * g, G::ZS), false);
        stage_c(z0 + 2 * g, slot(z0 + 2 * g, G::CS), slot(z0 + 2 * g, G::ZS), false);
        cp_async_commit();
    }
    // the coarse correction of the iterate planes that arrived for step f0:
    // group 0's, then two per step
    auto coarse_step = [&](int f0) {
        if (f0 == z0 - 1) {
            for (int k = z0 - 2; k <= z0 + 1; k++) {
                fetch_coarse(0, k);
                add_coarse(0, k);
            }
        } else {
            if (f0 + 1 <= z1 + 1) add_coarse(0, f0 + 1);   // planes above z1+1 are never staged
            if (f0 + 2 <= z1 + 1) add_coarse(1, f0 + 2);
        }
        fetch_coarse(0, f0 + 3);
        fetch_coarse(1, f0 + 4);
    };
    if constexpr (M) {
        // slot of plane k >= kb - S in a ring of S slots
        auto sl = [&](int k, int S) { return (k - kb + S) % S; };
        auto X = [&](int k) { return rx_ + sl(k, G::XS) * RP; };
        auto CX = [&](int k) { return rcx + sl(k, G::CS) * RP; };
        auto CY = [&](int k) { return rcy + sl(k, G::CS) * RP; };
        auto BB = [&](int k) { return rb + sl(k, G::CS) * RP; };
        auto CZ = [&](int k) { return rcz + sl(k, G::ZS) * RP; };
        for (int f0 = z0 - 1; f0 <= z1 + 2; f0 += 2) {
            cp_async_wait_newest<G::D - 1>();
            if (xc) coarse_step(f0);
            __syncthreads();
            stage_x(f0 + 2 * G::D + 1, sl(f0 + 2 * G::D + 1, G::XS));
            stage_x(f0 + 2 * G::D + 2, sl(f0 + 2 * G::D + 2, G::XS));
            stage_c(f0 + 2 * G::D, sl(f0 + 2 * G::D, G::CS), sl(f0 + 2 * G::D, G::ZS), false);
            stage_c(f0 + 2 * G::D + 1, sl(f0 + 2 * G::D + 1, G::CS), sl(f0 + 2 * G::D + 1, G::ZS), false);
            cp_async_commit();
            s_at(f0 - 3, X(f0 - 3), X(f0 - 4), X(f0 - 2), CX(f0 - 3), CY(f0 - 3), BB(f0 - 3), CZ(f0 - 3), CZ(f0 - 4));
            s_at(f0 - 2, X(f0 - 2), X(f0 - 3), X(f0 - 1), CX(f0 - 2), CY(f0 - 2), BB(f0 - 2), CZ(f0 - 2), CZ(f0 - 3));
            if (f0 <= z1) f_at(f0, X(f0), X(f0 - 1), X(f0 + 1), CX(f0), CY(f0), BB(f0), CZ(f0), CZ(f0 - 1));
            if (f0 + 1 <= z1)
                f_at(f0 + 1, X(f0 + 1), X(f0), X(f0 + 2), CX(f0 + 1), CY(f0 + 1), BB(f0 + 1), CZ(f0 + 1), CZ(f0));
        }
    }
    // ring positions of plane f0-2 (iterate, cz) and f0-1 (coefficients),
    // advanced by two each step (plane z0-2 sits in slot 0 of every ring)
    int xb = G::XS - 1, cb = 0, zb = G::ZS - 1;
    for (int f0 = z0 - 1; f0 <= z1 && !M; f0 += 2) {
        cp_async_wait_newest<G::D - 1>();
        if (xc) {   // the iterate planes that arrived: group 0's, then two per step
            if (f0 == z0 - 1) {
                for (int k = z0 - 2; k <= z0 + 1; k++) {
                    fetch_coarse(0, k);
                    add_coarse(0, k);
                }
            } else {
                if (f0 + 1 <= z1 + 1) add_coarse(0, f0 + 1);   // planes above z1+1 are never staged
                if (f0 + 2 <= z1 + 1) add_coarse(1, f0 + 2);
            }
            fetch_coarse(0, f0 + 3);
            fetch_coarse(1, f0 + 4);
        }
        __syncthreads();
        // slots of planes f0+2D+1, f0+2D+2 (iterate) and f0+2D, f0+2D+1
        // (coefficients): those of planes f0-4, f0-3 and f0-3, f0-2
        stage_x(f0 + 2 * G::D + 1, sw_add(xb, -2, G::XS));
        stage_x(f0 + 2 * G::D + 2, sw_add(xb, -1, G::XS));
        stage_c(f0 + 2 * G::D, sw_add(cb, -2, G::CS), sw_add(zb, -2, G::ZS), false);
        stage_c(f0 + 2 * G::D + 1, sw_add(cb, -1, G::CS), sw_add(zb, -1, G::ZS), false);
        cp_async_commit();
        // iterate planes f0-2 .. f0+2, coefficient planes f0-1 .. f0+1, cz f0-2 .. f0+1
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
    }
    cp_async_wait_all_groups();
    if (bx_part) {   // b.x of the block: one partial per block, in launch order
        __shared__ double bsh[32];
        bx = block_sum<G::NT>(bx, bsh);
        if (tid == 0) bx_part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bx;
    }
}
