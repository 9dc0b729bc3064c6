// mg_sweep_rs.cuh -- the last pre-smoothing sweep of a level fused with the
// residual and its restriction to the level below (included by mg_fast.cu
// after mg_sweep.cuh).
//
// One full red-black sweep as k_rb_sweep2_cfg computes it (same updates, same
// arithmetic), and in the same pass the residual r = b - A x of the swept
// iterate on every cell and the coarse right-hand side, the mean of each 2x2x2
// block of residuals, as k_fast_restrict2 forms it (same operations in the
// same order), so the level's restriction kernel does not run.  The residual
// of a cell needs the final iterate of its six neighbours, so the wavefront is
// one ring wider than the plain sweep's: at step f (planes f, f+1)
//   F   the first colour at planes f, f+1 on the tile plus a two-cell ring;
//   S   the second colour at planes f-1, f on the tile plus a one-cell ring;
//   R   planes f-1, f of the tile are final: stored; the residuals of planes
//       f-2, f-1 of the tile (their neighbours up to f are final), summed over
//       2x2 cells across lanes, and over the plane pair (f-2, f-1) into the
//       coarse cell, whose right-hand side is then written.
// The block's chunk of planes is even and starts on an even plane, so the
// plane pairs of the coarse cells never cross chunks; F runs on z0-2..z1+1,
// S on z0-1..z1, R on z0..z1-1.  Planes of the iterate (tile plus a
// three-cell ring across y, four across x) and of the coefficients are staged
// by 16-byte cp.async one step ahead, as in k_rb_sweep2_cfg.
#pragma once

// the configuration: 32x8 tiles, 224 threads, three blocks per SM (74 KB of
// staged planes each)
using SwRsCfg = SwCfg<float, 8, 1, 224, 3>;

template <class C>
struct SwRs {
    using T = typename C::type;
    static constexpr int NT = C::NT, TY = C::TY, TX = C::TX;
    static constexpr int RX = TX + 8, RY = TY + 6, RP = RX * RY;
    // live planes at step f: iterate f-3..f+2, coefficients f-2..f+1, cz f-3..f+1; plus two staged ahead
    static constexpr int XS = 8, CS = 6, ZS = 7;
    static constexpr int SLOTS = XS + 3 * CS + ZS;
    static constexpr int VEC = 16 / sizeof(T);
    static constexpr int RXC = RX / VEC;
    static constexpr int CH = RXC * RY;
    static constexpr int FROW = (TX + 4) / 2, FCELLS = FROW * (TY + 4);   // pairs, tile + 2-cell ring
    static constexpr int SROW = (TX + 2) / 2, SCELLS = SROW * (TY + 2);   // pairs, tile + 1-cell ring
    static constexpr int TPAIRS = TX / 2 * TY;                           // pairs of the tile
    static constexpr uint32_t SLOT_BYTES = sizeof(T) * RP;
    static_assert(C::D == 1, "one step staged ahead");
    static_assert(TX == 32 && TY % 2 == 0, "32-wide tiles, even height");
    static_assert(CH <= NT && FCELLS <= NT && SCELLS <= NT && TPAIRS <= NT, "one unit of each kind per thread");
};

template <class C>
static constexpr size_t sweep_rs_smem() {
    return sizeof(typename C::type) * (size_t)SwRs<C>::RP * SwRs<C>::SLOTS;
}

// v: the level (b its right-hand side); cb: the right-hand side of the level
// below (n0/2 x n1/2 x n2/2), written; zc even.
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB)
    k_rb_sweep_rs(const LV<typename C::type> v, const typename C::type* __restrict__ xin,
                  typename C::type* __restrict__ xout, typename C::type* __restrict__ cb, const Bnd B, int first,
                  int zc) {
    using T = typename C::type;
    using G = SwRs<C>;
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
    const int kb = z0 - 3;   // slot of plane k in a ring of S slots: (k - kb) % S
    auto slot = [&](int k, int S) { return (k - kb) % S; };

    // staging: rows y0-3 .. y0+TY+2, columns x0-4 .. x0+TX+3
    const bool ld = tid < G::CH;
    uint32_t creg = 0;
    long cin = 0;
    bool cok = false;
    if (ld) {
        int ry = tid / G::RXC, cxq = tid % G::RXC;
        int gi = sw_wrap(x0 - 4 + VEC * cxq, n0, B.per[0]);
        int gj = sw_wrap(y0 - 3 + ry, n1, B.per[1]);
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
    auto stage_x = [&](int k, int sx) {   // iterate planes z0-3 .. z1+2
        if (!ld || k > z1 + 2) return;
        const int gk = sw_wrap(k, n2, B.per[2]);
        const bool ok = xok && gk >= 0;
        cp_async16(s_x + G::SLOT_BYTES * sx, ok ? g_x + plane * gk : v.b, ok ? 16 : 0);
    };
    auto stage_c = [&](int k, int sc, int sz, bool cz_only) {   // coefficient planes up to z1+1
        if (!ld || k > z1 + 1) return;
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

    // the F pair of this thread (tile + 2-cell ring): staged cell, parity,
    // which of its two cells lie in the domain or its periodic image
    int fr0 = -1, fpar = 0, fok = 0;
    if (tid < G::FCELLS) {
        const int fry = 1 + tid / G::FROW, fcol = tid % G::FROW;   // staged row 1..TY+4
        const int gy = y0 - 3 + fry, gx = x0 - 2 + 2 * fcol;
        if (sw_wrap(gy, n1, B.per[1]) >= 0) {
            fr0 = 2 + 2 * fcol + RX * fry;
            fpar = (gx + gy + first) & 1;
            fok = (sw_wrap(gx, n0, B.per[0]) >= 0 ? 1 : 0) | (sw_wrap(gx + 1, n0, B.per[0]) >= 0 ? 2 : 0);
        }
    }
    // the S pair (tile + 1-cell ring)
    int sr0 = -1, spar = 0, sok = 0;
    if (tid < G::SCELLS) {
        const int sry = 2 + tid / G::SROW, scol = tid % G::SROW;   // staged row 2..TY+3
        const int gy = y0 - 3 + sry, gx = x0 - 1 + 2 * scol;
        if (sw_wrap(gy, n1, B.per[1]) >= 0) {
            sr0 = 3 + 2 * scol + RX * sry;
            spar = (gx + gy + first) & 1;
            sok = (sw_wrap(gx, n0, B.per[0]) >= 0 ? 1 : 0) | (sw_wrap(gx + 1, n0, B.per[0]) >= 0 ? 2 : 0);
        }
    }
    // the tile pair (2i, 2i+1) of row j this thread stores and forms residuals
    // for; lanes l and l+16 of a warp hold rows 2cj and 2cj+1 of a coarse cell
    const int tcol = tid % (TX / 2), trow = tid / (TX / 2);
    const int tgi = x0 + 2 * tcol, tgj = y0 + trow;
    const bool t_in = tid < G::TPAIRS && tgi < n0 && tgj < n1;
    const int trl = 4 + 2 * tcol + RX * (3 + trow);
    const int cn0 = n0 >> 1, cn1 = n1 >> 1;
    T acc = (T)0;   // coarse-cell sum over its first fine plane (lanes of even rows)

    auto update = [&](int r, T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk,
                      const T* czk, const T* czm) {
        T a1 = cxk[r - 1], a2 = cxk[r], a3 = cyk[r - RX], a4 = cyk[r], a5 = czm[r], a6 = czk[r];
        T out;
        const T x0v = v.omega != (T)1 ? xk[r] : (T)0;
        if (SwUpd<T>::apply(a1, a2, a3, a4, a5, a6, xk[r - 1], xk[r + 1], xk[r - RX], xk[r + RX], xm[r], xp[r], bk[r],
                            x0v, v.omega, out))
            xk[r] = out;
    };
    // one colour (0: F, 1: S) at plane k for this thread's pair r0
    auto colour = [&](int r0, int par, int okm, int col, int k, T* xk, const T* xm, const T* xp, const T* cxk,
                      const T* cyk, const T* bk, const T* czk, const T* czm) {
        if (r0 < 0 || sw_wrap(k, n2, B.per[2]) < 0) return;
        const int off = par ^ (k & 1) ^ col;
        if ((okm >> off) & 1) update(r0 + off, xk, xm, xp, cxk, cyk, bk, czk, czm);
    };
    // residuals of the tile pair at plane k (the operations of k_fast_restrict2)
    auto pair_resid = [&](const T* xk, const T* xm, const T* xp, const T* cxk, const T* cyk, const T* bk,
                          const T* czk, const T* czm) {
        const int r = trl;
        const T a1w = cxk[r - 1], xw = xk[r - 1], xe = xk[r + 2];
        const T Xx = xk[r], Xy = xk[r + 1], CXx = cxk[r], CXy = cxk[r + 1], CYx = cyk[r], CYy = cyk[r + 1];
        const T CZx = czk[r], CZy = czk[r + 1], BBx = bk[r], BBy = bk[r + 1];
        const T XSx = xk[r - RX], XSy = xk[r + 1 - RX], XNx = xk[r + RX], XNy = xk[r + 1 + RX];
        const T XBx = xm[r], XBy = xm[r + 1], XTx = xp[r], XTy = xp[r + 1];
        const T CYSx = cyk[r - RX], CYSy = cyk[r + 1 - RX], CZBx = czm[r], CZBy = czm[r + 1];
        T d = a1w + CXx + CYSx + CYx + CZBx + CZx;
        const T rA = BBx - d * Xx + a1w * xw + CXx * Xy + CYSx * XSx + CYx * XNx + CZBx * XBx + CZx * XTx;
        d = CXx + CXy + CYSy + CYy + CZBy + CZy;
        const T rB = BBy - d * Xy + CXx * Xx + CXy * xe + CYSy * XSy + CYy * XNy + CZBy * XBy + CZy * XTy;
        return rA + rB;
    };

    // prologue: iterate z0-3..z0, coefficients z0-2, z0-1, cz z0-3..z0-1
    for (int k = z0 - 3; k <= z0; k++) stage_x(k, slot(k, G::XS));
    stage_c(z0 - 3, 0, 0, true);
    stage_c(z0 - 2, slot(z0 - 2, G::CS), slot(z0 - 2, G::ZS), false);
    stage_c(z0 - 1, slot(z0 - 1, G::CS), slot(z0 - 1, G::ZS), false);
    cp_async_commit();
    for (int f = z0 - 2; f <= z1; f += 2) {
        cp_async_wait_newest<0>();
        __syncthreads();
        // planes f+3, f+4 (iterate) and f+2, f+3 (coefficients) into the slots
        // of planes f-5, f-4 and f-4, f-3 / f-5, f-4 (cz), no longer live
        stage_x(f + 3, slot(f + 3, G::XS));
        stage_x(f + 4, slot(f + 4, G::XS));
        stage_c(f + 2, slot(f + 2, G::CS), slot(f + 2, G::ZS), false);
        stage_c(f + 3, slot(f + 3, G::CS), slot(f + 3, G::ZS), false);
        cp_async_commit();
        // slot pointers of planes f-3 .. f+2
        T* xs[6];
        const T *cxs[6], *cys[6], *bs[6], *czs[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int k = f - 3 + q;
            xs[q] = rx_ + slot(k, G::XS) * RP;
            const int sc = slot(k, G::CS) * RP;   // coefficient planes f-2..f+1 are the ones read
            cxs[q] = rcx + sc;
            cys[q] = rcy + sc;
            bs[q] = rb + sc;
            czs[q] = rcz + slot(k, G::ZS) * RP;
        }
        // plane k = f - 3 + q: x xs[q], neighbours xs[q-1], xs[q+1]; top face czs[q], bottom czs[q-1]
#define SWRS_AT(q) xs[q], xs[(q) - 1], xs[(q) + 1], cxs[q], cys[q], bs[q], czs[q], czs[(q) - 1]
        // F at f, f+1 (q = 3, 4) on the tile + 2-cell ring
        colour(fr0, fpar, fok, 0, f, SWRS_AT(3));   // f <= z1 here
        if (f + 1 <= z1 + 1) colour(fr0, fpar, fok, 0, f + 1, SWRS_AT(4));
        __syncthreads();
        // S at f-1, f (q = 2, 3) on the tile + 1-cell ring
        if (f - 1 >= z0 - 1) colour(sr0, spar, sok, 1, f - 1, SWRS_AT(2));
        if (f >= z0 - 1 && f <= z1) colour(sr0, spar, sok, 1, f, SWRS_AT(3));
        __syncthreads();
        // R: store planes f-1, f of the tile; residuals of planes f-2 (even) and f-1 (odd)
        if (t_in) {
#pragma unroll
            for (int q = 2; q <= 3; q++) {
                const int k = f - 3 + q;
                if (k < z0 || k >= z1) continue;
                const T* xk = xs[q];
                float2 pr;
                pr.x = xk[trl];
                pr.y = xk[trl + 1];
                *reinterpret_cast<float2*>(xout + tgi + (long)n0 * tgj + plane * k) = pr;
            }
        }
#pragma unroll
        for (int q = 1; q <= 2; q++) {   // planes f-2, f-1
            const int k = f - 3 + q;
            const bool live = k >= z0 && k < z1;   // uniform over the block
            T p = (T)0;
            if (live && t_in) p = pair_resid(SWRS_AT(q));
            const T p1 = __shfl_down_sync(0xffffffffu, p, 16);   // the odd row of the coarse cell
            if (live && t_in && (trow & 1) == 0) {
                if ((k & 1) == 0) {
                    acc = p + p1;
                } else {
                    acc = (acc + p) + p1;
                    const int ci = tgi >> 1, cj = tgj >> 1, ck = k >> 1;
                    if (ci < cn0 && cj < cn1) cb[ci + (long)cn0 * (cj + (long)cn1 * ck)] = (T)0.125 * acc;
                }
            }
        }
#undef SWRS_AT
    }
    cp_async_wait_all_groups();
}
