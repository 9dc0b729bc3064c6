// mg_sweep4.cuh -- two consecutive red-black Gauss-Seidel sweeps of the B200
// multigrid in one pass over memory (included by mg_fast.cu after
// mg_sweep.cuh).
//
// Sweep A (colour X = `first`, then Y) and sweep B (X, then Y again) on the
// iterate, as two calls of k_rb_sweep2_cfg would compute them, with the
// iterate, the coefficients and the right-hand side read from HBM once for
// the pair.  A block owns a TX x TY column of cells and marches up a chunk of
// planes two at a time; at step f (planes f, f+1):
//   P1  A.X at planes f, f+1 on the tile plus a three-cell ring (old values);
//   P2  A.Y at planes f-1, f on the tile plus a two-cell ring;
//   P3  B.X at planes f-2, f-1 on the tile plus a one-cell ring;
//   P4  B.Y at planes f-3, f-2 on the tile, whose planes are then final and
//       stored.
// Each phase reads only values that the phases before it have finished: a
// ring shrinks by one cell per phase, and each phase lags the one before by
// one plane, so every update reads exactly the neighbour values of the two
// separate sweeps and the result is the same to the bit.  The staged region
// is the tile plus a four-cell ring; the ring slots rotate as in
// k_rb_sweep2_cfg, with the plane window four planes wider.  With `xc`, the
// coarse-grid correction is added to the iterate as it arrives (the first
// sweep of the post-smoothing pair).
#pragma once

// the configurations the solver uses
template <typename T>
struct SwGeo4;
template <>
struct SwGeo4<float> {
    using Cfg = SwCfg<float, 16, 1, 448, 1>;   // 32x16 tiles, 146 KB of staged planes, one block per SM
};
template <>
struct SwGeo4<double> {
    using Cfg = SwCfg<double, 8, 1, 320, 1>;   // 32x8 tiles, 190 KB of staged planes, one block per SM
};

template <class C>
struct Sw4 {
    using T = typename C::type;
    static constexpr int NT = C::NT, TY = C::TY, TX = C::TX, D = C::D;
    static constexpr int RX = TX + 8, RY = TY + 8, RP = RX * RY;
    static constexpr int XS = 7 + 2 * D, CS = 5 + 2 * D, ZS = 6 + 2 * D;
    static constexpr int SLOTS = XS + 3 * CS + ZS;
    static constexpr int VEC = 16 / sizeof(T);
    static constexpr int RXC = RX / VEC;
    static constexpr int CH = RXC * RY;
    static constexpr int CPER = (RP + NT - 1) / NT;
    static constexpr uint32_t SLOT_BYTES = sizeof(T) * RP;
    // pairs of cells per plane on the tile plus a ring of r cells
    static constexpr int pairs(int r) { return (TX + 2 * r) * (TY + 2 * r) / 2; }
    static_assert(D == 1, "one step of planes staged ahead");
    static_assert(TX % 2 == 0 && TY % 2 == 0, "pairs of cells");
    static_assert(pairs(3) <= NT, "one pair of each ring per thread");
    static_assert(CH <= NT, "one chunk of each array per thread");
};

template <class C>
static constexpr size_t sweep4_smem_cfg() {
    return sizeof(typename C::type) * (size_t)Sw4<C>::RP * Sw4<C>::SLOTS;
}

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB)
    k_rb_sweep4_cfg(const LV<typename C::type> v, const typename C::type* __restrict__ xin,
                    typename C::type* __restrict__ xout, const typename C::type* __restrict__ xc, const Bnd B,
                    int first, int zc) {
    using T = typename C::type;
    using G = Sw4<C>;
    constexpr int NT = G::NT;
    constexpr int RX = G::RX, RP = G::RP, TY = G::TY, TX = G::TX, VEC = G::VEC;
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
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc, z1 = min(z0 + zc, n2);
    const int kb = z0 - 4;   // slot of plane k in a ring of S slots: (k - kb) % S
    auto slot = [&](int k, int S) { return (k - kb) % S; };

    // staging: the 16-byte chunk of every array plane this thread loads
    const bool ld = tid < G::CH;
    uint32_t creg = 0;
    long cin = 0;
    bool cok = false;
    if (ld) {
        int ry = tid / G::RXC, cxq = tid % G::RXC;
        int gi = sw_wrap(x0 - 4 + VEC * cxq, n0, B.per[0]);
        int gj = sw_wrap(y0 - 4 + ry, n1, B.per[1]);
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
    // iterate plane k (needed up to z1+3) and coefficient plane k (up to z1+2)
    auto stage_x = [&](int k, int sx) {
        if (!ld || k > z1 + 3) return;
        const int gk = sw_wrap(k, n2, B.per[2]);
        const bool ok = xok && gk >= 0;
        cp_async16(s_x + G::SLOT_BYTES * sx, ok ? g_x + plane * gk : v.b, ok ? 16 : 0);
    };
    auto stage_c = [&](int k, int sc, int sz, bool cz_only) {
        if (!ld || k > z1 + 2) return;
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

    // the pair of cells this thread updates on the tile plus a ring of r
    // cells (r = 3, 2, 1, 0): its first cell in the staged plane (-1: none),
    // the parity of that cell without the plane (x + y + first), and which of
    // the two cells lie in the domain or its periodic image
    int pr0[4], ppar[4], pok[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int w = (TX + 2 * r) / 2;
        pr0[r] = -1;
        ppar[r] = 0;
        pok[r] = 0;
        if (tid < (TX + 2 * r) * (TY + 2 * r) / 2) {
            const int sr = 4 - r + tid / w, p = tid % w;
            const int gx = x0 - r + 2 * p, gy = y0 - 4 + sr;
            if (sw_wrap(gy, n1, B.per[1]) >= 0) {
                pr0[r] = sr * RX + 4 - r + 2 * p;
                ppar[r] = (gx + gy + first) & 1;
                pok[r] = (sw_wrap(gx, n0, B.per[0]) >= 0 ? 1 : 0) | (sw_wrap(gx + 1, n0, B.per[0]) >= 0 ? 2 : 0);
            }
        }
    }
    // the tile pair this thread stores
    const bool s_out = pr0[0] >= 0 && tid < TX * TY / 2 && x0 + 2 * (tid % (TX / 2)) < n0 &&
                       y0 + tid / (TX / 2) < n1;
    const long s_g = (x0 + 2 * (tid % (TX / 2))) + (long)n0 * (y0 + tid / (TX / 2));

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
            int gj = sw_wrap(y0 - 4 + e / RX, n1, B.per[1]);
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
    // one colour (0: X, 1: Y) at plane k on the ring of this thread's pair,
    // when k lies in [klo, khi] and in the domain or its periodic image
    auto phase = [&](int ring, int colour, int k, int klo, int khi, T* xk, const T* xm, const T* xp, const T* cxk,
                     const T* cyk, const T* bk, const T* czk, const T* czm) {
        if (k < klo || k > khi || pr0[ring] < 0 || sw_wrap(k, n2, B.per[2]) < 0) return;
        const int off = ppar[ring] ^ (k & 1) ^ colour;
        if ((pok[ring] >> off) & 1) update(pr0[ring] + off, xk, xm, xp, cxk, cyk, bk, czk, czm);
    };

    // prologue: group 0 = iterate z0-4..z0-1, cz z0-4, coefficients z0-3, z0-2
    for (int k = z0 - 4; k <= z0 - 1; k++) stage_x(k, slot(k, G::XS));
    stage_c(z0 - 4, 0, 0, true);
    stage_c(z0 - 3, 1, 1, false);
    stage_c(z0 - 2, 2, 2, false);
    cp_async_commit();
    // ring positions of the oldest live planes: iterate f-4, coefficients
    // f-3, cz f-4 (at f = z0-3: planes z0-7, z0-6, z0-7)
    int xb = G::XS - 3, cb = G::CS - 2, zb = G::ZS - 3;
    for (int f = z0 - 3; f <= z1 + 2; f += 2) {
        cp_async_wait_newest<0>();
        __syncthreads();
        // planes f+3, f+4 (iterate) and f+2, f+3 (coefficients) into the slots
        // of planes f-6, f-5 and f-5, f-4, no longer live
        stage_x(f + 3, sw_add(xb, -2, G::XS));
        stage_x(f + 4, sw_add(xb, -1, G::XS));
        stage_c(f + 2, sw_add(cb, -2, G::CS), sw_add(zb, -2, G::ZS), false);
        stage_c(f + 3, sw_add(cb, -1, G::CS), sw_add(zb, -1, G::ZS), false);
        cp_async_commit();
        if (xc) {   // the iterate planes that arrived: group 0's, then two per step
            if (f == z0 - 3) {
                for (int k = z0 - 4; k <= z0 - 1; k++) {
                    fetch_coarse(0, k);
                    add_coarse(0, k);
                }
            } else {
                if (f + 1 <= z1 + 3) add_coarse(0, f + 1);
                if (f + 2 <= z1 + 3) add_coarse(1, f + 2);
            }
            fetch_coarse(0, f + 3);
            fetch_coarse(1, f + 4);
            __syncthreads();
        }
        // iterate planes f-4 .. f+2, coefficient planes f-3 .. f+1, cz f-4 .. f+1
        T* xs[7];
#pragma unroll
        for (int q = 0; q < 7; q++) xs[q] = rx_ + sw_add(xb, q, G::XS) * RP;   // plane f-4+q
        const T *cxs[5], *cys[5], *bs[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {   // plane f-3+q
            const int sc = sw_add(cb, q, G::CS) * RP;
            cxs[q] = rcx + sc;
            cys[q] = rcy + sc;
            bs[q] = rb + sc;
        }
        const T* czs[6];
#pragma unroll
        for (int q = 0; q < 6; q++) czs[q] = rcz + sw_add(zb, q, G::ZS) * RP;   // plane f-4+q
        // the phase at plane k = f + o uses xs[o+4], coefficients [o+3], cz [o+4] (top) and [o+3] (bottom)
#define SW4_PH(ring, colour, o, klo, khi) \
    phase(ring, colour, f + (o), klo, khi, xs[(o) + 4], xs[(o) + 3], xs[(o) + 5], cxs[(o) + 3], cys[(o) + 3], \
          bs[(o) + 3], czs[(o) + 4], czs[(o) + 3])
        SW4_PH(3, 0, 0, z0 - 3, z1 + 2);
        SW4_PH(3, 0, 1, z0 - 3, z1 + 2);
        __syncthreads();
        SW4_PH(2, 1, -1, z0 - 2, z1 + 1);
        SW4_PH(2, 1, 0, z0 - 2, z1 + 1);
        __syncthreads();
        SW4_PH(1, 0, -2, z0 - 1, z1);
        SW4_PH(1, 0, -1, z0 - 1, z1);
        __syncthreads();
        SW4_PH(0, 1, -3, z0, z1 - 1);
        SW4_PH(0, 1, -2, z0, z1 - 1);
#undef SW4_PH
        // planes f-3 and f-2 of the tile are final
        if (s_out) {
            using V2 = typename SwVec<T>::V2;
#pragma unroll
            for (int o = -3; o <= -2; o++) {
                const int k = f + o;
                if (k < z0 || k >= z1) continue;
                const T* xk = xs[o + 4];
                V2 pr;
                pr.x = xk[pr0[0]];
                pr.y = xk[pr0[0] + 1];
                *reinterpret_cast<V2*>(xout + s_g + plane * k) = pr;
            }
        }
        xb = sw_add(xb, 2, G::XS);
        cb = sw_add(cb, 2, G::CS);
        zb = sw_add(zb, 2, G::ZS);
    }
    cp_async_wait_all_groups();
}
