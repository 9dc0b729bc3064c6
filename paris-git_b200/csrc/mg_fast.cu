// mg_fast.cu -- the B200 multigrid for the variable-density pressure
// equation (PARIS_MG_FP64 / PARIS_MG_MIXED).  It solves the system that
// SetupPoisson builds (modules.f90:2735-2745), using that A is symmetric on
// the uniform grid (A2(i) == A1(i+1)), so one coefficient per face is stored:
//   level 0 faces = A2, A4, A6 of each cell; coarse face = (sum of the four
//   fine faces across it) / 16; restriction = mean of the 8 children;
//   prolongation = injection; red-black Gauss-Seidel V(nu1,nu2) cycles with
//   the colours reversed after the coarse correction (symmetric cycle).
// The inner cycle runs in T = float (mixed) or double; the outer loop is FP64:
// defect correction p += V(b - A p), or CG preconditioned by the V-cycle.
// Levels at or below kCoarseCells cells run in one single-block kernel.
#include <stdlib.h>
#include <string.h>
#include <type_traits>

#include "ctx.cuh"

static constexpr long kCoarseCells = 4096;   // 16^3
static constexpr int kMaxLevels = 16;
static constexpr int kCoarseSweeps = 8;
static constexpr long kWarpCells = 64;   // coarse levels of at most 4^3 cells run in one warp
static constexpr long kFusedCells = 1L << 15;
// device-side scalars of the CG loop (paris_ctx::cg_scal): r.z of the two
// latest preconditioned residuals (alternating), d.q, and r.r, sum |r|, r.z_old
// from the update
static constexpr int kScRZ0 = 0, kScDQ = 2, kScRR = 3, kScRZold = 5;
static constexpr size_t kCoarseSmemMax = 227 * 1024;   // opt-in shared memory per block   // levels of at least 64^3 cells use the fused sweep

template <typename T>
struct LV {
    const T *cx, *cy, *cz;
    T *b, *x;
    int n0, n1, n2;
    long N;
    T omega;   // relaxation factor of the red-black smoother (1: Gauss-Seidel)
};

// sweeps of a smoothing pass on level L: nu, or nuc on the levels cf..ct
// (ct <= 0: every level from cf down)
__host__ __device__ inline int nu_at(int L, int nu, int nuc, int cf, int ct) {
    return nuc > 0 && L >= cf && (ct <= 0 || L <= ct) ? nuc : nu;
}

// x_new of a relaxed cell: the Gauss-Seidel value g, over-relaxed by w
template <typename T>
__device__ inline T relax(T g, T x0, T w) {
    return w == (T)1 ? g : x0 + w * (g - x0);
}

template <typename T>
struct LVSet {
    LV<T> l[kMaxLevels];
};

// west/south/bottom face coefficient of cell (i,j,k)
template <typename T>
__device__ inline void west_coefs(const LV<T>& v, const Bnd& B, int i, int j, int k, long m, T& a1, T& a3, T& a5) {
    a1 = i > 0 ? v.cx[m - 1] : (B.per[0] ? v.cx[m + v.n0 - 1] : (T)0);
    a3 = j > 0 ? v.cy[m - v.n0] : (B.per[1] ? v.cy[m + (long)v.n0 * (v.n1 - 1)] : (T)0);
    a5 = k > 0 ? v.cz[m - (long)v.n0 * v.n1] : (B.per[2] ? v.cz[m + (long)v.n0 * v.n1 * (v.n2 - 1)] : (T)0);
}

template <typename T>
__device__ inline void nbrs(const LV<T>& v, const T* __restrict__ x, const Bnd& B, int i, int j, int k, long m, T& xw,
                            T& xe, T& xs, T& xn, T& xb, T& xt) {
    long sy = v.n0, sz = (long)v.n0 * v.n1;
    xw = i > 0 ? x[m - 1] : (B.per[0] ? x[m + v.n0 - 1] : (T)0);
    xe = i < v.n0 - 1 ? x[m + 1] : (B.per[0] ? x[m - (v.n0 - 1)] : (T)0);
    xs = j > 0 ? x[m - sy] : (B.per[1] ? x[m + sy * (v.n1 - 1)] : (T)0);
    xn = j < v.n1 - 1 ? x[m + sy] : (B.per[1] ? x[m - sy * (v.n1 - 1)] : (T)0);
    xb = k > 0 ? x[m - sz] : (B.per[2] ? x[m + sz * (v.n2 - 1)] : (T)0);
    xt = k < v.n2 - 1 ? x[m + sz] : (B.per[2] ? x[m - sz * (v.n2 - 1)] : (T)0);
}

template <typename T>
__device__ inline void smooth_cell(const LV<T>& v, const Bnd& B, int i, int j, int k) {
    long m = cidx(v.n0, v.n1, i, j, k);
    T a1, a3, a5, xw, xe, xs, xn, xb, xt;
    west_coefs(v, B, i, j, k, m, a1, a3, a5);
    T a2 = v.cx[m], a4 = v.cy[m], a6 = v.cz[m];
    nbrs(v, v.x, B, i, j, k, m, xw, xe, xs, xn, xb, xt);
    T d = a1 + a2 + a3 + a4 + a5 + a6;
    T s = a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt + v.b[m];
    if (d > (T)0) v.x[m] = relax(s / d, v.omega != (T)1 ? v.x[m] : (T)0, v.omega);
}

template <typename T>
__device__ inline T resid_cell(const LV<T>& v, const Bnd& B, int i, int j, int k) {
    long m = cidx(v.n0, v.n1, i, j, k);
    T a1, a3, a5, xw, xe, xs, xn, xb, xt;
    west_coefs(v, B, i, j, k, m, a1, a3, a5);
    T a2 = v.cx[m], a4 = v.cy[m], a6 = v.cz[m];
    nbrs(v, v.x, B, i, j, k, m, xw, xe, xs, xn, xb, xt);
    T d = a1 + a2 + a3 + a4 + a5 + a6;
    return v.b[m] - d * v.x[m] + a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt;
}

// coarse rhs = mean of the 8 fine residuals
template <typename T>
__device__ inline void restrict_cell(const LV<T>& f, const LV<T>& c, const Bnd& B, int i, int j, int k) {
    T s = 0;
    for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) s += resid_cell(f, B, 2 * i + di, 2 * j + dj, 2 * k + dk);
    c.b[cidx(c.n0, c.n1, i, j, k)] = (T)0.125 * s;
}

// grid (ceil(n/128), n1, n2), block 128: one thread per cell of the colour
template <typename T>
__global__ void k_fast_smooth(const LV<T> v, const Bnd B, int color) {
    int ih = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    int i = 2 * ih + ((j + k + color) & 1);
    if (i < v.n0) smooth_cell(v, B, i, j, k);
}

// Residual and restriction with one warp per 32 coarse cells of a fine row:
// threadIdx.y = dj + 2 dk picks the fine row of the 2x2x2 block, and each
// lane computes the residuals of its fine pair (2i, 2i+1) from pair loads
// (x, the east/north/top coefficients, b, and the rows and planes around),
// the west neighbours of the pair by a shuffle from the lane to its left
// (scalar loads at the tile edge).  The four rows of a coarse cell are summed
// in shared memory.  Needs an even fine n0 (every level above the coarsest).
template <typename T>
__global__ void __launch_bounds__(128) k_fast_restrict2(const LV<T> f, const LV<T> c, const Bnd B) {
    using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
    __shared__ T part[4][32];
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int ci = blockIdx.x * 32 + lane, cj = blockIdx.y, ck = blockIdx.z;
    const int n0 = f.n0, n1 = f.n1, n2 = f.n2;
    const long sy = n0, sz = (long)n0 * n1;
    const int i0 = 2 * ci, j = 2 * cj + (ty & 1), k = 2 * ck + (ty >> 1);
    const bool ok = ci < c.n0;
    const long m = i0 + sy * j + sz * k;
    auto ld2 = [&](const T* a, long q) { return *reinterpret_cast<const V2*>(a + q); };
    const V2 zero2 = {(T)0, (T)0};
    V2 X = zero2, CX = zero2, CY = zero2, CZ = zero2, BB = zero2, XS = zero2, XN = zero2, XB = zero2, XT = zero2,
       CYS = zero2, CZB = zero2;
    if (ok) {
        X = ld2(f.x, m);
        CX = ld2(f.cx, m);
        CY = ld2(f.cy, m);
        CZ = ld2(f.cz, m);
        BB = ld2(f.b, m);
        if (j > 0) { XS = ld2(f.x, m - sy); CYS = ld2(f.cy, m - sy); }
        else if (B.per[1]) { XS = ld2(f.x, m + sy * (n1 - 1)); CYS = ld2(f.cy, m + sy * (n1 - 1)); }
        if (j < n1 - 1) XN = ld2(f.x, m + sy);
        else if (B.per[1]) XN = ld2(f.x, m - sy * (n1 - 1));
        if (k > 0) { XB = ld2(f.x, m - sz); CZB = ld2(f.cz, m - sz); }
        else if (B.per[2]) { XB = ld2(f.x, m + sz * (n2 - 1)); CZB = ld2(f.cz, m + sz * (n2 - 1)); }
        if (k < n2 - 1) XT = ld2(f.x, m + sz);
        else if (B.per[2]) XT = ld2(f.x, m - sz * (n2 - 1));
    }
    // west of the pair: x and cx of fine cell i0-1; east: x of fine cell i0+2
    T xw = __shfl_up_sync(0xffffffffu, X.y, 1), a1w = __shfl_up_sync(0xffffffffu, CX.y, 1);
    T xe = __shfl_down_sync(0xffffffffu, X.x, 1);
    if (ok && (lane == 0 || i0 == 0)) {
        if (i0 > 0) { xw = f.x[m - 1]; a1w = f.cx[m - 1]; }
        else if (B.per[0]) { xw = f.x[m + n0 - 1]; a1w = f.cx[m + n0 - 1]; }
        else { xw = (T)0; a1w = (T)0; }
    }
    if (ok && (lane == 31 || ci == c.n0 - 1)) {
        if (i0 + 2 < n0) xe = f.x[m + 2];
        else xe = B.per[0] ? f.x[m + 2 - n0] : (T)0;
    }
    T s = (T)0;
    if (ok) {
        // the fine cell i0, then i0+1 (the arithmetic of resid_cell)
        T d = a1w + CX.x + CYS.x + CY.x + CZB.x + CZ.x;
        const T rA = BB.x - d * X.x + a1w * xw + CX.x * X.y + CYS.x * XS.x + CY.x * XN.x + CZB.x * XB.x + CZ.x * XT.x;
        d = CX.x + CX.y + CYS.y + CY.y + CZB.y + CZ.y;
        const T rB = BB.y - d * X.y + CX.x * X.x + CX.y * xe + CYS.y * XS.y + CY.y * XN.y + CZB.y * XB.y + CZ.y * XT.y;
        s = rA + rB;
    }
    part[ty][lane] = s;
    __syncthreads();
    if (ty == 0 && ok)
        c.b[cidx(c.n0, c.n1, ci, cj, ck)] = (T)0.125 * (((part[0][lane] + part[1][lane]) + part[2][lane]) + part[3][lane]);
}

template <typename T>
__global__ void k_fast_prolong(const LV<T> f, const LV<T> c) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= f.n0) return;
    f.x[cidx(f.n0, f.n1, i, j, k)] += c.x[cidx(c.n0, c.n1, i >> 1, j >> 1, k >> 1)];
}

static inline dim3 row_grid(long n0, int n1, int n2) { return dim3(div_up(n0, 128), n1, n2); }

#include "mg_sweep.cuh"
#include "mg_sweep_tma.cuh"
#include "mg_sweep4.cuh"
#include "mg_sweep_rs.cuh"

// 32-bit forms of smooth_cell / resid_cell / restrict_cell for the levels of
// the single-block coarse cycle (at most a few thousand cells): the same
// operations on the same values, with int instead of long index arithmetic.
template <typename T>
__device__ inline void nbrs32(const LV<T>& v, const T* x, const Bnd& B, int i, int j, int k, int m, T& a1, T& a3,
                              T& a5, T& xw, T& xe, T& xs, T& xn, T& xb, T& xt) {
    const int n0 = v.n0, n1 = v.n1, n2 = v.n2, sy = n0, sz = n0 * n1;
    a1 = i > 0 ? v.cx[m - 1] : (B.per[0] ? v.cx[m + n0 - 1] : (T)0);
    a3 = j > 0 ? v.cy[m - sy] : (B.per[1] ? v.cy[m + sy * (n1 - 1)] : (T)0);
    a5 = k > 0 ? v.cz[m - sz] : (B.per[2] ? v.cz[m + sz * (n2 - 1)] : (T)0);
    xw = i > 0 ? x[m - 1] : (B.per[0] ? x[m + n0 - 1] : (T)0);
    xe = i < n0 - 1 ? x[m + 1] : (B.per[0] ? x[m - (n0 - 1)] : (T)0);
    xs = j > 0 ? x[m - sy] : (B.per[1] ? x[m + sy * (n1 - 1)] : (T)0);
    xn = j < n1 - 1 ? x[m + sy] : (B.per[1] ? x[m - sy * (n1 - 1)] : (T)0);
    xb = k > 0 ? x[m - sz] : (B.per[2] ? x[m + sz * (n2 - 1)] : (T)0);
    xt = k < n2 - 1 ? x[m + sz] : (B.per[2] ? x[m - sz * (n2 - 1)] : (T)0);
}

template <typename T>
__device__ inline void smooth_cell32(const LV<T>& v, const Bnd& B, int i, int j, int k) {
    const int m = i + v.n0 * (j + v.n1 * k);
    T a1, a3, a5, xw, xe, xs, xn, xb, xt;
    nbrs32(v, v.x, B, i, j, k, m, a1, a3, a5, xw, xe, xs, xn, xb, xt);
    T a2 = v.cx[m], a4 = v.cy[m], a6 = v.cz[m];
    T d = a1 + a2 + a3 + a4 + a5 + a6;
    T s = a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt + v.b[m];
    if (d > (T)0) v.x[m] = relax(s / d, v.omega != (T)1 ? v.x[m] : (T)0, v.omega);
}

template <typename T>
__device__ inline T resid_cell32(const LV<T>& v, const Bnd& B, int i, int j, int k) {
    const int m = i + v.n0 * (j + v.n1 * k);
    T a1, a3, a5, xw, xe, xs, xn, xb, xt;
    nbrs32(v, v.x, B, i, j, k, m, a1, a3, a5, xw, xe, xs, xn, xb, xt);
    T a2 = v.cx[m], a4 = v.cy[m], a6 = v.cz[m];
    T d = a1 + a2 + a3 + a4 + a5 + a6;
    return v.b[m] - d * v.x[m] + a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt;
}

template <typename T>
__device__ inline void restrict_cell32(const LV<T>& f, const LV<T>& c, const Bnd& B, int i, int j, int k) {
    T s = 0;
    for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) s += resid_cell32(f, B, 2 * i + di, 2 * j + dj, 2 * k + dk);
    c.b[i + c.n0 * (j + c.n1 * k)] = (T)0.125 * s;
}

// t / d for 0 <= t, d < 2^22 (exact): a float estimate within one of the
// quotient, corrected
__device__ inline int div_small(int t, int d, float rd) {
    int q = __float2int_rz((float)t * rd);
    const int r = t - q * d;
    if (r < 0) q--;
    else if (r >= d) q++;
    return q;
}

// The V-cycle from level L0 down to the coarsest, in one block, on copies of
// those levels in shared memory: the coefficients of every level and the
// right-hand side of level L0 are loaded, the cycle runs, and the iterate of
// level L0 is written back.
template <typename T>
__global__ void __launch_bounds__(1024) k_fast_coarse_cycle(const LVSet<T> G, int L0, int nl, const Bnd B, int nu1,
                                                            int nu2, int nuc, int cf, int ct, int in_smem) {
    const int tid = threadIdx.x, nt = blockDim.x;
    extern __shared__ __align__(16) unsigned char cc_raw[];
    __shared__ LV<T> S[kMaxLevels];   // level views, read by value in every phase
    if (tid == 0) {
        T* p = reinterpret_cast<T*>(cc_raw);
        for (int L = L0; L < nl; L++) {
            LV<T> l = G.l[L];
            if (in_smem) {
                T* cx = p;
                l.cx = cx; l.cy = cx + l.N; l.cz = cx + 2 * l.N;
                l.b = cx + 3 * l.N;
                l.x = cx + 4 * l.N;
                p = cx + 5 * l.N;
            }
            S[L] = l;
        }
    }
    __syncthreads();
    if (in_smem) {
        for (int L = L0; L < nl; L++) {
            const LV<T> g = G.l[L], l = S[L];
            T* cx = const_cast<T*>(l.cx);
            T* cy = const_cast<T*>(l.cy);
            T* cz = const_cast<T*>(l.cz);
            for (int t = tid; t < (int)g.N; t += nt) {
                cx[t] = g.cx[t]; cy[t] = g.cy[t]; cz[t] = g.cz[t];
                if (L == L0) l.b[t] = g.b[t];
            }
        }
        __syncthreads();
    }
    // 32-bit index arithmetic throughout (levels here have at most a few
    // thousand cells; 64-bit division would dominate every phase).  Levels of
    // at most kWarpCells cells are worked by warp 0 alone with warp barriers.
    const int lane = tid & 31;
    auto smooth = [&](const LV<T> v, int color, bool warp) {
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const int h0 = (v.n0 + 1) >> 1, hn = h0 * v.n1;
        const int tot = hn * v.n2;
        const float rhn = 1.0f / (float)hn, rh0 = 1.0f / (float)h0;
        for (int t = t0; t < tot; t += st) {
            int k = div_small(t, hn, rhn), r = t - k * hn;
            int j = div_small(r, h0, rh0), ih = r - j * h0;
            int i = 2 * ih + ((j + k + color) & 1);
            if (i < v.n0) smooth_cell32(v, B, i, j, k);
        }
        if (warp) __syncwarp();
        else __syncthreads();
    };
    auto down = [&](int L, bool warp) {   // zero, pre-smooth and restrict level L, or solve the coarsest
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const LV<T> v = S[L];
        for (int t = t0; t < (int)v.N; t += st) v.x[t] = (T)0;
        if (warp) __syncwarp();
        else __syncthreads();
        if (L == nl - 1) {
            for (int s = 0; s < kCoarseSweeps; s++) { smooth(v, 0, warp); smooth(v, 1, warp); }
            for (int s = 0; s < kCoarseSweeps; s++) { smooth(v, 1, warp); smooth(v, 0, warp); }
            return;
        }
        for (int s = 0; s < nu_at(L, nu1, nuc, cf, ct); s++) { smooth(v, 0, warp); smooth(v, 1, warp); }
        const LV<T> c = S[L + 1];
        const int cn = c.n0 * c.n1;
        const float rcn = 1.0f / (float)cn, rc0 = 1.0f / (float)c.n0;
        for (int t = t0; t < (int)c.N; t += st) {
            int k = div_small(t, cn, rcn), r = t - k * cn;
            int j = div_small(r, c.n0, rc0), i = r - j * c.n0;
            restrict_cell32(v, c, B, i, j, k);
        }
        if (warp) __syncwarp();
        else __syncthreads();
    };
    auto up = [&](int L, bool warp) {     // prolong into level L and post-smooth it
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const LV<T> v = S[L], c = S[L + 1];
        const int fn = v.n0 * v.n1;
        const float rfn = 1.0f / (float)fn, rf0 = 1.0f / (float)v.n0;
        for (int t = t0; t < (int)v.N; t += st) {
            int k = div_small(t, fn, rfn), r = t - k * fn;
            int j = div_small(r, v.n0, rf0), i = r - j * v.n0;
            v.x[t] += c.x[(i >> 1) + c.n0 * ((j >> 1) + c.n1 * (k >> 1))];
        }
        if (warp) __syncwarp();
        else __syncthreads();
        for (int s = 0; s < nu_at(L, nu2, nuc, cf, ct); s++) { smooth(v, 1, warp); smooth(v, 0, warp); }
    };
    int Lw = L0;   // first level worked by warp 0
    while (Lw < nl && S[Lw].N > kWarpCells) Lw++;
    for (int L = L0; L < Lw; L++) down(L, false);
    if (Lw < nl) {
        if (tid < 32) {
            for (int L = Lw; L < nl; L++) down(L, true);
            for (int L = nl - 2; L >= Lw; L--) up(L, true);
        }
        __syncthreads();
    }
    for (int L = min(Lw, nl - 1) - 1; L >= L0; L--) up(L, false);
    if (in_smem) {
        const LV<T> g = G.l[L0], l = S[L0];
        for (int t = tid; t < (int)g.N; t += nt) g.x[t] = l.x[t];
    }
}

// ---- the coarse cycle in shared memory ------------------------------------
// The same cycle as k_fast_coarse_cycle, with every level of at most 16^3
// cells held in the block's shared memory and addressed by element offsets
// from one shared array (shared-memory loads rather than generic ones), the
// neighbours of a cell taken branch-free (the wrapped or clamped index always
// loaded, the value dropped at a wall), the cell indices of each thread
// decomposed once per pass, and the restriction split into a pass over the
// fine cells (their residuals into a scratch array) and one over the coarse
// cells (the 8 residuals summed in the order restrict_cell32 sums them).
// The arithmetic of every update, residual and sum is that of
// smooth_cell32 / resid_cell32 / restrict_cell32.
struct CcLvl {
    int n0, n1, n2, N;
    int cx, cy, cz, b, x;   // element offsets of the arrays in shared memory
};

struct CcNb {   // a cell's index and its six neighbours' (always valid), and which exist
    int m, mw, me, ms, mn, mb, mt;
    bool hw, he, hs, hn, hb, ht;
};

__device__ inline CcNb cc_nb(const CcLvl& l, const Bnd& B, int i, int j, int k) {
    const int n0 = l.n0, n1 = l.n1, n2 = l.n2, sy = n0, sz = n0 * n1;
    CcNb q;
    q.m = i + sy * j + sz * k;
    q.mw = i > 0 ? q.m - 1 : q.m + n0 - 1;
    q.me = i < n0 - 1 ? q.m + 1 : q.m - (n0 - 1);
    q.ms = j > 0 ? q.m - sy : q.m + sy * (n1 - 1);
    q.mn = j < n1 - 1 ? q.m + sy : q.m - sy * (n1 - 1);
    q.mb = k > 0 ? q.m - sz : q.m + sz * (n2 - 1);
    q.mt = k < n2 - 1 ? q.m + sz : q.m - sz * (n2 - 1);
    q.hw = i > 0 || B.per[0];
    q.he = i < n0 - 1 || B.per[0];
    q.hs = j > 0 || B.per[1];
    q.hn = j < n1 - 1 || B.per[1];
    q.hb = k > 0 || B.per[2];
    q.ht = k < n2 - 1 || B.per[2];
    return q;
}

template <typename T>
__device__ inline void cc_terms(const T* sm, const CcLvl& l, const CcNb& q, T& a1, T& a2, T& a3, T& a4, T& a5, T& a6,
                                T& xw, T& xe, T& xs, T& xn, T& xb, T& xt) {
    const T* x = sm + l.x;
    const T c1 = sm[l.cx + q.mw], c3 = sm[l.cy + q.ms], c5 = sm[l.cz + q.mb];
    const T vw = x[q.mw], ve = x[q.me], vs = x[q.ms], vn = x[q.mn], vb = x[q.mb], vt = x[q.mt];
    a1 = q.hw ? c1 : (T)0;
    a3 = q.hs ? c3 : (T)0;
    a5 = q.hb ? c5 : (T)0;
    xw = q.hw ? vw : (T)0;
    xe = q.he ? ve : (T)0;
    xs = q.hs ? vs : (T)0;
    xn = q.hn ? vn : (T)0;
    xb = q.hb ? vb : (T)0;
    xt = q.ht ? vt : (T)0;
    a2 = sm[l.cx + q.m];
    a4 = sm[l.cy + q.m];
    a6 = sm[l.cz + q.m];
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_cycle_smem(const LVSet<T> G, int L0, int nl, const Bnd B, int nu1,
                                                            int nu2, int nuc, int cf, int ct, int scratch) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    extern __shared__ __align__(16) unsigned char cc_raw[];
    T* const sm = reinterpret_cast<T*>(cc_raw);
    __shared__ CcLvl S[kMaxLevels];
    __shared__ T omg[kMaxLevels];
    if (tid == 0) {
        int off = 0;
        for (int L = L0; L < nl; L++) {
            const LV<T>& g = G.l[L];
            const int N = (int)g.N;
            S[L] = CcLvl{g.n0, g.n1, g.n2, N, off, off + N, off + 2 * N, off + 3 * N, off + 4 * N};
            omg[L] = g.omega;
            off += 5 * N;
        }
    }
    __syncthreads();
    // the coefficients of every level and the right-hand side of L0, four
    // loads in flight per thread and array
    for (int L = L0; L < nl; L++) {
        const LV<T>& g = G.l[L];
        const CcLvl l = S[L];
        for (int t0 = tid; t0 < l.N; t0 += 4 * nt) {
            T v[4][4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int t = t0 + u * nt;
                if (t < l.N) {
                    v[u][0] = g.cx[t];
                    v[u][1] = g.cy[t];
                    v[u][2] = g.cz[t];
                    v[u][3] = L == L0 ? g.b[t] : (T)0;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int t = t0 + u * nt;
                if (t < l.N) {
                    sm[l.cx + t] = v[u][0];
                    sm[l.cy + t] = v[u][1];
                    sm[l.cz + t] = v[u][2];
                    if (L == L0) sm[l.b + t] = v[u][3];
                }
            }
        }
    }
    __syncthreads();
    auto sync = [&](bool warp) {
        if (warp) __syncwarp();
        else __syncthreads();
    };
    // one colour pass of red-black Gauss-Seidel over level l
    auto smooth = [&](const CcLvl& l, T w, int color, bool warp) {
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const int h0 = (l.n0 + 1) >> 1, hn = h0 * l.n1;
        const int tot = hn * l.n2;
        const float rhn = 1.0f / (float)hn, rh0 = 1.0f / (float)h0;
        for (int t = t0; t < tot; t += st) {
            const int k = div_small(t, hn, rhn), r = t - k * hn;
            const int j = div_small(r, h0, rh0), ih = r - j * h0;
            const int i = 2 * ih + ((j + k + color) & 1);
            if (i >= l.n0) continue;
            const CcNb q = cc_nb(l, B, i, j, k);
            T a1, a2, a3, a4, a5, a6, xw, xe, xs, xn, xb, xt;
            cc_terms(sm, l, q, a1, a2, a3, a4, a5, a6, xw, xe, xs, xn, xb, xt);
            T d = a1 + a2 + a3 + a4 + a5 + a6;
            T s = a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt + sm[l.b + q.m];
            T* x = sm + l.x;
            if (d > (T)0) x[q.m] = relax(s / d, w != (T)1 ? x[q.m] : (T)0, w);
        }
        sync(warp);
    };
    auto down = [&](int L, bool warp) {   // zero, pre-smooth and restrict level L, or solve the coarsest
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const CcLvl l = S[L];
        const T w = omg[L];
        for (int t = t0; t < l.N; t += st) sm[l.x + t] = (T)0;
        sync(warp);
        if (L == nl - 1) {
            for (int s = 0; s < kCoarseSweeps; s++) { smooth(l, w, 0, warp); smooth(l, w, 1, warp); }
            for (int s = 0; s < kCoarseSweeps; s++) { smooth(l, w, 1, warp); smooth(l, w, 0, warp); }
            return;
        }
        for (int s = 0; s < nu_at(L, nu1, nuc, cf, ct); s++) { smooth(l, w, 0, warp); smooth(l, w, 1, warp); }
        // residuals of the fine cells into the scratch array
        {
            const int fn = l.n0 * l.n1;
            const float rfn = 1.0f / (float)fn, rf0 = 1.0f / (float)l.n0;
            for (int t = t0; t < l.N; t += st) {
                const int k = div_small(t, fn, rfn), r = t - k * fn;
                const int j = div_small(r, l.n0, rf0), i = r - j * l.n0;
                const CcNb q = cc_nb(l, B, i, j, k);
                T a1, a2, a3, a4, a5, a6, xw, xe, xs, xn, xb, xt;
                cc_terms(sm, l, q, a1, a2, a3, a4, a5, a6, xw, xe, xs, xn, xb, xt);
                T d = a1 + a2 + a3 + a4 + a5 + a6;
                sm[scratch + q.m] =
                    sm[l.b + q.m] - d * sm[l.x + q.m] + a1 * xw + a2 * xe + a3 * xs + a4 * xn + a5 * xb + a6 * xt;
            }
        }
        sync(warp);
        // the coarse right-hand side: the mean of each 2x2x2 block
        {
            const CcLvl c = S[L + 1];
            const int cn = c.n0 * c.n1;
            const float rcn = 1.0f / (float)cn, rc0 = 1.0f / (float)c.n0;
            const int sy = l.n0, sz = l.n0 * l.n1;
            for (int t = t0; t < c.N; t += st) {
                const int k = div_small(t, cn, rcn), r = t - k * cn;
                const int j = div_small(r, c.n0, rc0), i = r - j * c.n0;
                const int f = 2 * i + sy * (2 * j) + sz * (2 * k);
                T s = 0;
                for (int dk = 0; dk < 2; dk++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int di = 0; di < 2; di++) s += sm[scratch + f + di + sy * dj + sz * dk];
                sm[c.b + t] = (T)0.125 * s;
            }
        }
        sync(warp);
    };
    auto up = [&](int L, bool warp) {     // prolong into level L and post-smooth it
        const int t0 = warp ? lane : tid, st = warp ? 32 : nt;
        const CcLvl l = S[L], c = S[L + 1];
        const T w = omg[L];
        const int fn = l.n0 * l.n1;
        const float rfn = 1.0f / (float)fn, rf0 = 1.0f / (float)l.n0;
        for (int t = t0; t < l.N; t += st) {
            const int k = div_small(t, fn, rfn), r = t - k * fn;
            const int j = div_small(r, l.n0, rf0), i = r - j * l.n0;
            sm[l.x + t] += sm[c.x + (i >> 1) + c.n0 * ((j >> 1) + c.n1 * (k >> 1))];
        }
        sync(warp);
        for (int s = 0; s < nu_at(L, nu2, nuc, cf, ct); s++) { smooth(l, w, 1, warp); smooth(l, w, 0, warp); }
    };
    int Lw = L0;   // first level worked by warp 0
    while (Lw < nl && S[Lw].N > kWarpCells) Lw++;
    for (int L = L0; L < Lw; L++) down(L, false);
    if (Lw < nl) {
        if (tid < 32) {
            for (int L = Lw; L < nl; L++) down(L, true);
            for (int L = nl - 2; L >= Lw; L--) up(L, true);
        }
        __syncthreads();
    }
    for (int L = min(Lw, nl - 1) - 1; L >= L0; L--) up(L, false);
    {
        const LV<T>& g = G.l[L0];
        const CcLvl l = S[L0];
        for (int t = tid; t < l.N; t += nt) g.x[t] = sm[l.x + t];
    }
}

// shared memory of k_fast_coarse_cycle: five arrays per level from L0 down
template <typename T>
static size_t coarse_smem(const std::vector<FastLevel<T>>& lv, int L0) {
    size_t n = 0;
    for (int L = L0; L < (int)lv.size(); L++) n += 5 * (size_t)lv[L].N;
    return n * sizeof(T);
}

// level-0 coefficients from the FP64 compact matrix
template <typename T>
__global__ void k_fast_coef0(const double* __restrict__ cx, const double* __restrict__ cy,
                             const double* __restrict__ cz, T* ox, T* oy, T* oz, long N) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= N) return;
    ox[t] = (T)cx[t]; oy[t] = (T)cy[t]; oz[t] = (T)cz[t];
}

// coarse face = (sum of the four fine faces on it) / 16
template <typename T>
__global__ void k_fast_coarsen(const LV<T> f, const LV<T> c, T* ccx, T* ccy, T* ccz) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= c.N) return;
    // a coarse level holds fewer than 2^32 cells: 32-bit index arithmetic
    const unsigned tt = (unsigned)t, r = tt / (unsigned)c.n0;
    const int i = (int)(tt - r * (unsigned)c.n0), k = (int)(r / (unsigned)c.n1), j = (int)(r - (unsigned)k * c.n1);
    int I = 2 * i, J = 2 * j, K = 2 * k;
    ccx[t] = (T)0.0625 * (f.cx[cidx(f.n0, f.n1, I + 1, J, K)] + f.cx[cidx(f.n0, f.n1, I + 1, J + 1, K)] +
                          f.cx[cidx(f.n0, f.n1, I + 1, J, K + 1)] + f.cx[cidx(f.n0, f.n1, I + 1, J + 1, K + 1)]);
    ccy[t] = (T)0.0625 * (f.cy[cidx(f.n0, f.n1, I, J + 1, K)] + f.cy[cidx(f.n0, f.n1, I + 1, J + 1, K)] +
                          f.cy[cidx(f.n0, f.n1, I, J + 1, K + 1)] + f.cy[cidx(f.n0, f.n1, I + 1, J + 1, K + 1)]);
    ccz[t] = (T)0.0625 * (f.cz[cidx(f.n0, f.n1, I, J, K + 1)] + f.cz[cidx(f.n0, f.n1, I + 1, J, K + 1)] +
                          f.cz[cidx(f.n0, f.n1, I, J + 1, K + 1)] + f.cz[cidx(f.n0, f.n1, I + 1, J + 1, K + 1)]);
}

// ---- FP64 outer loop --------------------------------------------------------
// the six neighbours of interior cell (i,j,k) of a ghosted field, at offsets
// from its index n: the periodic image across a boundary, 0 at a wall
__device__ inline void pnbrs(const double* __restrict__ p, const Layout& L, const Bnd& B, int i, int j, int k, long n,
                             double& xw, double& xe, double& xs, double& xn, double& xb, double& xt) {
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    const long sy = L.pitch, sz = L.plane;
    xw = i > 0 ? p[n - 1] : (B.per[0] ? p[n + n0 - 1] : 0.0);
    xe = i < n0 - 1 ? p[n + 1] : (B.per[0] ? p[n - (n0 - 1)] : 0.0);
    xs = j > 0 ? p[n - sy] : (B.per[1] ? p[n + sy * (n1 - 1)] : 0.0);
    xn = j < n1 - 1 ? p[n + sy] : (B.per[1] ? p[n - sy * (n1 - 1)] : 0.0);
    xb = k > 0 ? p[n - sz] : (B.per[2] ? p[n + sz * (n2 - 1)] : 0.0);
    xt = k < n2 - 1 ? p[n + sz] : (B.per[2] ? p[n - sz * (n2 - 1)] : 0.0);
}

// (A x)_m with the symmetric face form: A1 = cx(i-1), A2 = cx(i), ...
// The FP64 outer loop applies A in flux form, sum_f a_f (x_f - x_c): a
// constant x gives exactly 0 (constants are the null space of the singular
// system), and only neighbour differences are rounded, not coef * |x|.  A
// warm-started pressure carries the hydrostatic field (|p| ~ 1e4 at density
// ratio 1000 and g = 9.81); with the d*x form its rounding, coef * |p| * eps
// per cell, was above the 1e-10 relative residual at h = 1/512.
struct Mat64 {
    const double *cx, *cy, *cz, *rhs;
};

__device__ inline double ax_compact(const Mat64& A, const double* __restrict__ x, const Layout& L, const Bnd& B,
                                    int i, int j, int k, long m) {
    LV<double> v{A.cx, A.cy, A.cz, nullptr, nullptr, L.n[0], L.n[1], L.n[2], 0, 1.0};
    double a1, a3, a5, xw, xe, xs, xn, xb, xt;
    west_coefs(v, B, i, j, k, m, a1, a3, a5);
    double a2 = A.cx[m], a4 = A.cy[m], a6 = A.cz[m];
    nbrs(v, x, B, i, j, k, m, xw, xe, xs, xn, xb, xt);
    const double xc = x[m];
    return -(a1 * (xw - xc) + a2 * (xe - xc) + a3 * (xs - xc) + a4 * (xn - xc) + a5 * (xb - xc) + a6 * (xt - xc));
}

// r = b - A p on the ghosted p (wrap in the kernel); writes r as T into the
// level-0 right-hand side (and as double into r64 when given).
// slots: 0 = sum r^2, 1 = sum |r|, 2 = sum b^2
template <typename T>
__global__ void k_fast_residual64(const Mat64 A, const double* __restrict__ p, const Layout L, const Bnd B,
                                  T* __restrict__ rT, double* __restrict__ r64, double* part) {
    __shared__ double sh[32];
    double s2 = 0.0, s1 = 0.0, sb = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        long m = cidx(L.n[0], L.n[1], i, j, k);
        double a1 = i > 0 ? A.cx[m - 1] : (B.per[0] ? A.cx[m + L.n[0] - 1] : 0.0);
        double a3 = j > 0 ? A.cy[m - L.n[0]] : (B.per[1] ? A.cy[m + (long)L.n[0] * (L.n[1] - 1)] : 0.0);
        long sz = (long)L.n[0] * L.n[1];
        double a5 = k > 0 ? A.cz[m - sz] : (B.per[2] ? A.cz[m + sz * (L.n[2] - 1)] : 0.0);
        double a2 = A.cx[m], a4 = A.cy[m], a6 = A.cz[m];
        long n = lidx(L, i, j, k);
        double b = A.rhs[m];
        const double pc = p[n];
        double xw, xe, xs, xn, xb, xt;
        pnbrs(p, L, B, i, j, k, n, xw, xe, xs, xn, xb, xt);
        double r = b + (a1 * (xw - pc) + a2 * (xe - pc) + a3 * (xs - pc) + a4 * (xn - pc) + a5 * (xb - pc) +
                        a6 * (xt - pc));
        if (rT) rT[m] = (T)r;
        if (r64) r64[m] = r;
        s2 += r * r;
        s1 += fabs(r);
        sb += b * b;
    ROWS_END
    s2 = block_sum<256>(s2, sh);
    s1 = block_sum<256>(s1, sh);
    sb = block_sum<256>(sb, sh);
    if (linear_tid() == 0) {
        part[blockIdx.x] = s2;
        part[kRedBlocks + blockIdx.x] = s1;
        part[2 * kRedBlocks + blockIdx.x] = sb;
    }
}

// p += x (the level-0 correction) on the ghosted field
template <typename T>
__global__ void k_fast_correct(double* __restrict__ p, const T* __restrict__ x, const Layout L, double alpha) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.n[0]) return;
    long n = lidx(L, i, j, k);
    p[n] = p[n] + alpha * (double)x[cidx(L.n[0], L.n[1], i, j, k)];
}

// ---- PCG helpers (FP64 compact vectors) --------------------------------------
// q = A d ; slot 0 = d.q
__global__ void k_pcg_matvec(const Mat64 A, const double* __restrict__ d, double* __restrict__ q, const Layout L,
                             const Bnd B, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        long m = cidx(L.n[0], L.n[1], i, j, k);
        double v = ax_compact(A, d, L, B, i, j, k, m);
        q[m] = v;
        s += d[m] * v;
    ROWS_END
    s = block_sum<256>(s, sh);
    if (linear_tid() == 0) part[blockIdx.x] = s;
}

// p += alpha d (ghosted p), r -= alpha q, and the right-hand side of the next
// V-cycle rT = (T) r.  slots: 0 = r.r, 1 = sum |r|, 2 = r.zold (zold: the
// last preconditioned residual, still in the V-cycle's output buffer)
template <typename T>
__global__ void k_pcg_update(double* __restrict__ p, double* __restrict__ r, const double* __restrict__ d,
                             const double* __restrict__ q, T* __restrict__ rT, const T* __restrict__ zold,
                             const double* __restrict__ sc, int rzs, const Layout L, double* part) {
    __shared__ double sh[32];
    // alpha = r.z / d.q from the device-side scalars; when d.q is not positive
    // nothing is written and the host leaves the loop with p and r as they were
    const double dq = sc[kScDQ];
    if (!(dq > 0.0)) return;
    const double alpha = sc[rzs] / dq;
    double s2 = 0.0, s1 = 0.0, sz = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        long m = cidx(L.n[0], L.n[1], i, j, k);
        long n = lidx(L, i, j, k);
        p[n] = p[n] + alpha * d[m];
        double rr = r[m] - alpha * q[m];
        r[m] = rr;
        rT[m] = (T)rr;
        s2 += rr * rr;
        s1 += fabs(rr);
        sz += rr * (double)zold[m];
    ROWS_END
    s2 = block_sum<256>(s2, sh);
    s1 = block_sum<256>(s1, sh);
    sz = block_sum<256>(sz, sh);
    if (linear_tid() == 0) {
        part[blockIdx.x] = s2;
        part[kRedBlocks + blockIdx.x] = s1;
        part[2 * kRedBlocks + blockIdx.x] = sz;
    }
}

// slot 0 = r.z with z the V-cycle's output
template <typename T>
__global__ void k_pcg_rz(const T* __restrict__ z, const double* __restrict__ r, long N, double* part) {
    __shared__ double sh[32];
    double s0 = 0.0;
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < N; m += (long)gridDim.x * blockDim.x)
        s0 += r[m] * (double)z[m];
    s0 = block_sum<256>(s0, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s0;
}

// d = z + beta d, beta = (r.z_new - r.z_old) / r.z (flexible Polak-Ribiere)
// from the device-side scalars, or 0 when rzs_old < 0 (a fresh start)
template <typename T>
__global__ void k_pcg_dir(double* __restrict__ d, const T* __restrict__ z, const double* __restrict__ sc, int rzs_new,
                          int rzs_old, long N) {
    const double beta = rzs_old < 0 ? 0.0 : (sc[rzs_new] - sc[kScRZold]) / sc[rzs_old];
    long m = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (m < N) d[m] = (double)z[m] + beta * d[m];
}

// the partials of slot blockIdx.x summed in the fixed order of k_reduce_slots,
// into dev[slot] and, when host is given (mapped memory), host[slot]
__global__ void k_cg_reduce(const double* __restrict__ part, double* dev, double* host, int nb) {
    __shared__ double sh[32];
    const int slot = blockIdx.x;
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v = v + part[(long)slot * kRedBlocks + b];
    v = block_sum<256>(v, sh);
    if (threadIdx.x == 0) {
        dev[slot] = v;
        if (host) host[slot] = v;
    }
}

// ---- host side ---------------------------------------------------------------
// profile label of a kernel instantiated for T (stable strings)
template <typename T>
static const char* kname(const char* base);
template <>
const char* kname<float>(const char* base) {
    static const char* names[] = {"mg_smooth_f32", "mg_restrict_f32", "mg_prolong_f32", "mg_coarse_cycle_f32",
                                  "mg_correct_f32", "mg_residual_fp64(r32)", "mg_sweep_f32", "mg_sweep_zero_f32",
                                  "pcg_update_fp64(z32)", "pcg_rz(z32)", "pcg_dir(z32)", "mg_sweep_lower_f32",
                                  "mg_sweep_pair_f32", "mg_sweep_pair_zero_f32", "mg_sweep_pair_lower_f32"};
    static const char* keys[] = {"mg_smooth", "mg_restrict", "mg_prolong", "mg_coarse_cycle", "mg_correct",
                                 "mg_residual_fp64", "mg_sweep", "mg_sweep_zero", "pcg_update", "pcg_rz", "pcg_dir",
                                 "mg_sweep_lower", "mg_sweep_pair", "mg_sweep_pair_zero", "mg_sweep_pair_lower"};
    for (int q = 0; q < 15; q++)
        if (!strcmp(base, keys[q])) return names[q];
    return base;
}
template <>
const char* kname<double>(const char* base) {
    static const char* names[] = {"mg_smooth_f64", "mg_restrict_f64", "mg_prolong_f64", "mg_coarse_cycle_f64",
                                  "mg_correct_f64", "mg_residual_fp64(r64)", "mg_sweep_f64", "mg_sweep_zero_f64",
                                  "pcg_update_fp64(z64)", "pcg_rz(z64)", "pcg_dir(z64)", "mg_sweep_lower_f64",
                                  "mg_sweep_pair_f64", "mg_sweep_pair_zero_f64", "mg_sweep_pair_lower_f64"};
    static const char* keys[] = {"mg_smooth", "mg_restrict", "mg_prolong", "mg_coarse_cycle", "mg_correct",
                                 "mg_residual_fp64", "mg_sweep", "mg_sweep_zero", "pcg_update", "pcg_rz", "pcg_dir",
                                 "mg_sweep_lower", "mg_sweep_pair", "mg_sweep_pair_zero", "mg_sweep_pair_lower"};
    for (int q = 0; q < 15; q++)
        if (!strcmp(base, keys[q])) return names[q];
    return base;
}
template <typename T>
static std::vector<FastLevel<T>>& levels(paris_ctx* c);
template <>
std::vector<FastLevel<float>>& levels<float>(paris_ctx* c) { return c->fl32; }
template <>
std::vector<FastLevel<double>>& levels<double>(paris_ctx* c) { return c->fl64; }

static int fast_depth(const paris_ctx* c) {
    int n0[3] = {c->d.nx, c->d.ny, c->d.nz};
    int nl = 1;
    while (nl < kMaxLevels) {
        bool even = true, big = true;
        for (int a = 0; a < 3; a++) {
            if ((n0[a] >> (nl - 1)) % 2) even = false;
            if ((n0[a] >> nl) < 2) big = false;
        }
        if (!even || !big) break;
        nl++;
    }
    return nl;
}

// ---- tensor maps of the TMA-staged sweep (FP32 levels) --------------------
struct LevelTma {
    SwTmaMaps m;     // .x: the iterate buffer x
    CUtensorMap x2;  // the iterate buffer x2
};

using TmEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to
// the driver library); null when the driver does not provide it
static TmEncodeFn tm_encode_fn() {
    static TmEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TmEncodeFn)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// a level array as the 3-D tensor (n0, n1, n2), boxes of a tile and its ring;
// out-of-range elements of a box read as zero
static bool tm_encode(CUtensorMap* m, const float* base, const int n[3]) {
    TmEncodeFn fn = tm_encode_fn();
    if (!fn) return false;
    using Cfg = SwTmaCfg;
    const cuuint64_t dims[3] = {(cuuint64_t)n[0], (cuuint64_t)n[1], (cuuint64_t)n[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)n[0] * sizeof(float), (cuuint64_t)n[0] * n[1] * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)(kSwTX + 8), (cuuint32_t)(Cfg::TY + 4), 1u};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// The TMA staging is opt-in (PARIS_SWEEP_TMA=1 in the environment when a
// handle first builds its FP32 levels), and only where the tiles fit the
// level exactly in x and y (the wrapped ring is then only at the first and
// last tile of a row or column).  Measured on a B200 at 256^3 it ran at 207 us
// per sweep against 147 us for the cp.async staging, so cp.async is the
// default.
static bool tma_wanted() {
    const char* e = getenv("PARIS_SWEEP_TMA");
    return e && e[0] == '1';
}

static void level_maps(FastLevel<float>& l) {
    using Cfg = SwTmaCfg;
    if (!l.x2 || l.n[0] % kSwTX || l.n[1] % Cfg::TY || !tma_wanted()) return;
    LevelTma* t = new LevelTma();
    bool ok = tm_encode(&t->m.x, l.x, l.n) && tm_encode(&t->x2, l.x2, l.n) && tm_encode(&t->m.cx, l.cx, l.n) &&
              tm_encode(&t->m.cy, l.cy, l.n) && tm_encode(&t->m.b, l.b, l.n) && tm_encode(&t->m.cz, l.cz, l.n);
    if (ok)
        l.tma = t;
    else
        delete t;
}

// Two consecutive sweeps of a smoothing pass run as one pass over memory
// (k_rb_sweep4_cfg) when PARIS_SWEEP_PAIRS=1 is in the environment as a
// handle first builds its levels; the two forms give the same iterate to the
// bit.
static bool pairs_wanted() {
    const char* e = getenv("PARIS_SWEEP_PAIRS");
    return e && e[0] == '1';
}

// The last pre-smoothing sweep of a fused FP32 level can also form the
// residual and the coarse right-hand side (k_rb_sweep_rs): on the finest level
// (PARIS_SWEEP_RS=1 in the environment when a handle first builds its levels)
// or on every fused level (2).  It gives the same iterates to the bit, but
// measured on a B200 at 256^3 the fused sweep took 291 us against 148 us for
// the sweep plus 75 us for the restriction kernel (its wider rings and the
// 32x8 tiles that fit three blocks per SM), so it is off by default.
static int rs_levels() {
    const char* e = getenv("PARIS_SWEEP_RS");
    if (!e) return 0;
    return e[0] == '1' ? 1 : (e[0] == '2' ? 2 : 0);
}

// The FP32 fused sweep with one barrier per step (the merged phases of
// k_rb_sweep2_cfg<C, true>) when PARIS_SWEEP_MERGED=1 (32x12 tiles) or 2
// (32x14 tiles) is in the environment as a handle first builds its levels;
// the same iterate to the bit.
static int merged_wanted() {
    const char* e = getenv("PARIS_SWEEP_MERGED");
    if (!e) return 0;
    return e[0] == '1' ? 1 : (e[0] == '2' ? 2 : 0);
}

void mg_fast_free_maps(paris_ctx* c) {
    for (auto& l : c->fl32) {
        delete static_cast<LevelTma*>(l.tma);
        l.tma = nullptr;
    }
}

template <typename T>
static int fast_alloc(paris_ctx* c) {
    auto& lv = levels<T>(c);
    if (!lv.empty()) return PARIS_OK;
    int nl = fast_depth(c);
    c->fast_nl = nl;
    lv.resize(nl);
    for (int L = 0; L < nl; L++) {
        FastLevel<T>& l = lv[L];
        l.n[0] = c->d.nx >> L; l.n[1] = c->d.ny >> L; l.n[2] = c->d.nz >> L;
        l.N = (long)l.n[0] * l.n[1] * l.n[2];
        for (T** p : {&l.cx, &l.cy, &l.cz, &l.b, &l.x}) PARIS_CUDA_TRY(c, cudaMalloc(p, l.N * sizeof(T)));
        // the fused sweep stages 16-byte row chunks and pairs cells by parity
        l.x2 = nullptr;
        bool fusable = l.N >= kFusedCells && l.N > kCoarseCells && l.n[0] % 4 == 0 && l.n[1] % 2 == 0 &&
                       l.n[2] % 2 == 0 && L < nl - 1;
        if (fusable) PARIS_CUDA_TRY(c, cudaMalloc(&l.x2, l.N * sizeof(T)));
        l.pairs = fusable && pairs_wanted();
        l.rs = fusable && std::is_same<T, float>::value && (rs_levels() == 2 || (rs_levels() == 1 && L == 0));
        l.merged = fusable && std::is_same<T, float>::value ? merged_wanted() : 0;
        if constexpr (std::is_same<T, float>::value) level_maps(l);
    }
    return PARIS_OK;
}

template <typename T>
static LV<T> view(const FastLevel<T>& l) {
    return LV<T>{l.cx, l.cy, l.cz, l.b, l.x, l.n[0], l.n[1], l.n[2], l.N, (T)l.omega};
}

template <typename T>
static int fast_coefs(paris_ctx* c) {
    auto& lv = levels<T>(c);
    PARIS_LAUNCH_N(c, "mg_coef0", c->N, k_fast_coef0<T>, div_up(c->N, 256), 256, 0, c->cx, c->cy, c->cz, lv[0].cx, lv[0].cy, lv[0].cz,
                 c->N);
    for (int L = 1; L < (int)lv.size(); L++)
        PARIS_LAUNCH_N(c, "mg_coarsen", lv[L].N, k_fast_coarsen<T>, div_up(lv[L].N, 256), 256, 0, view(lv[L - 1]), view(lv[L]), lv[L].cx,
                     lv[L].cy, lv[L].cz);
    return PARIS_OK;
}

// Planes per block of the fused sweep: enough blocks for one wave of resident
// blocks, at least 4 planes per block (2 where that leaves fewer blocks than
// SMs).
template <class Cfg, bool M, typename T>
static int sweep_chunk_cfg(paris_ctx* c, const FastLevel<T>& l) {
    constexpr size_t smem = sweep2_smem_cfg<Cfg, M>();
    static int per_sm = 0;   // resident blocks per SM (the same on every B200)
    if (!per_sm) {
        cudaFuncSetAttribute(k_rb_sweep2_cfg<Cfg, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_sweep2_cfg<Cfg, M>, Cfg::NT, smem) !=
                cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    long tiles = (long)div_up(l.n[0], Cfg::TX) * div_up(l.n[1], Cfg::TY);
    long nbz = (long)per_sm * c->nsm / tiles;
    long cap = l.n[2] / 4;
    if (tiles * cap < c->nsm) cap = l.n[2] / 2;   // small levels (64^3, 32^3): two planes per block
    if (nbz > cap) nbz = cap;
    if (nbz < 1) nbz = 1;
    return (int)div_up(l.n[2], nbz);
}
template <typename T>
static int sweep_chunk(paris_ctx* c, const FastLevel<T>& l) {
    return sweep_chunk_cfg<typename SwGeo<T>::Cfg, false>(c, l);
}

// the merged-phase sweep of an FP32 level with configuration Cfg
template <class Cfg>
static int sweep_merged(paris_ctx* c, const FastLevel<float>& l, const char* label, const float* xin, float* xout,
                        const float* xc, int first, double* bx_part, int* bx_blocks) {
    const int zc = sweep_chunk_cfg<Cfg, true>(c, l);
    dim3 grid(div_up(l.n[0], Cfg::TX), div_up(l.n[1], Cfg::TY), div_up(l.n[2], zc));
    if (bx_part && (long)grid.x * grid.y * grid.z > kRedBlocks) bx_part = nullptr;
    auto* const kern = &k_rb_sweep2_cfg<Cfg, true>;
    constexpr size_t smem = sweep2_smem_cfg<Cfg, true>();
    PARIS_LAUNCH_N(c, kname<float>(label), l.N, kern, grid, Cfg::NT, smem, view(l), xin, xout, xc, c->bnd, first, zc,
                   bx_part);
    if (bx_part && bx_blocks) *bx_blocks = (int)(grid.x * grid.y * grid.z);
    return PARIS_OK;
}

// planes per block of the TMA-staged sweep, as sweep_chunk
static int sweep_tma_chunk(paris_ctx* c, const FastLevel<float>& l) {
    using Cfg = SwTmaCfg;
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_rb_sweep_tma<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep_tma_smem<Cfg>());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_sweep_tma<Cfg>, Cfg::NT,
                                                          sweep_tma_smem<Cfg>()) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    long tiles = (long)div_up(l.n[0], Cfg::TX) * div_up(l.n[1], Cfg::TY);
    long nbz = (long)per_sm * c->nsm / tiles;
    long cap = l.n[2] / 4;
    if (nbz > cap) nbz = cap;
    if (nbz < 1) nbz = 1;
    return (int)div_up(l.n[2], nbz);
}

// bx_part: also write the per-block partials of b.x (see k_rb_sweep2_cfg);
// *bx_blocks receives their count (0 when this form of the sweep cannot)
template <typename T>
static int sweep_fused(paris_ctx* c, int L, const FastLevel<T>& l, const T* xin, T* xout, const T* xc, int first,
                       double* bx_part = nullptr, int* bx_blocks = nullptr) {
    using Cfg = typename SwGeo<T>::Cfg;
    // level 0 streams from HBM; the lower levels are resident in L2
    const char* label = L > 0 ? "mg_sweep_lower" : (xin ? "mg_sweep" : "mg_sweep_zero");
    if (bx_blocks) *bx_blocks = 0;
    if constexpr (std::is_same<T, float>::value) {
        if (l.tma) {
            const LevelTma* t = static_cast<const LevelTma*>(l.tma);
            SwTmaMaps M = t->m;
            if (xin == l.x2) M.x = t->x2;
            using TC = SwTmaCfg;
            const int zc = sweep_tma_chunk(c, l);
            dim3 grid(div_up(l.n[0], TC::TX), div_up(l.n[1], TC::TY), div_up(l.n[2], zc));
            PARIS_LAUNCH_N(c, kname<T>(label), l.N, k_rb_sweep_tma<TC>, grid, TC::NT, sweep_tma_smem<TC>(),
                           view(l), xin, M, xout, xc, c->bnd, first, zc, c->err_dev);
            return PARIS_OK;
        }
        if (l.merged == 1) return sweep_merged<SwMCfg12>(c, l, label, xin, xout, xc, first, bx_part, bx_blocks);
        if (l.merged == 2) return sweep_merged<SwMCfg14>(c, l, label, xin, xout, xc, first, bx_part, bx_blocks);
    }
    int zc = sweep_chunk<T>(c, l);
    dim3 grid(div_up(l.n[0], Cfg::TX), div_up(l.n[1], Cfg::TY), div_up(l.n[2], zc));
    if (bx_part && (long)grid.x * grid.y * grid.z > kRedBlocks) bx_part = nullptr;
    PARIS_LAUNCH_N(c, kname<T>(label), l.N, k_rb_sweep2_cfg<Cfg>, grid, Cfg::NT,
                   sweep_smem<T>(), view(l), xin, xout, xc, c->bnd, first, zc, bx_part);
    if (bx_part && bx_blocks) *bx_blocks = (int)(grid.x * grid.y * grid.z);
    return PARIS_OK;
}

// planes per block of the fused-restriction sweep: one wave of resident
// blocks, an even number of planes, at least 4
static int sweep_rs_chunk(paris_ctx* c, const FastLevel<float>& l) {
    using Cfg = SwRsCfg;
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_rb_sweep_rs<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep_rs_smem<Cfg>());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_sweep_rs<Cfg>, Cfg::NT,
                                                          sweep_rs_smem<Cfg>()) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    long tiles = (long)div_up(l.n[0], Cfg::TX) * div_up(l.n[1], Cfg::TY);
    long nbz = (long)per_sm * c->nsm / tiles;
    long cap = l.n[2] / 4;
    if (nbz > cap) nbz = cap;
    if (nbz < 1) nbz = 1;
    int zc = (int)div_up(l.n[2], nbz);
    return zc + (zc & 1);
}

// the last pre-smoothing sweep of level L with the restriction into the
// right-hand side of level L+1
static int sweep_rs(paris_ctx* c, const FastLevel<float>& l, const FastLevel<float>& lc, const float* xin,
                    float* xout, int first) {
    using Cfg = SwRsCfg;
    const int zc = sweep_rs_chunk(c, l);
    dim3 grid(div_up(l.n[0], Cfg::TX), div_up(l.n[1], Cfg::TY), div_up(l.n[2], zc));
    PARIS_LAUNCH_N(c, "mg_sweep_restrict_f32", l.N, k_rb_sweep_rs<Cfg>, grid, Cfg::NT, sweep_rs_smem<Cfg>(), view(l),
                   xin, xout, lc.b, c->bnd, first, zc);
    return PARIS_OK;
}

// planes per block of the pair sweep: as sweep_chunk, at least 8 planes per
// block (a block recomputes three planes on either side of its chunk)
template <typename T>
static int sweep4_chunk(paris_ctx* c, const FastLevel<T>& l) {
    using Cfg = typename SwGeo4<T>::Cfg;
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_rb_sweep4_cfg<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep4_smem_cfg<Cfg>());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_sweep4_cfg<Cfg>, Cfg::NT,
                                                          sweep4_smem_cfg<Cfg>()) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    long tiles = (long)div_up(l.n[0], Cfg::TX) * div_up(l.n[1], Cfg::TY);
    long nbz = (long)per_sm * c->nsm / tiles;
    long cap = l.n[2] / 8;
    if (nbz > cap) nbz = cap;
    if (nbz < 1) nbz = 1;
    return (int)div_up(l.n[2], nbz);
}

// two sweeps (colour `first`, then the other; twice) from xin to xout
template <typename T>
static int sweep_pair(paris_ctx* c, int L, const FastLevel<T>& l, const T* xin, T* xout, const T* xc, int first) {
    using Cfg = typename SwGeo4<T>::Cfg;
    const char* label = L > 0 ? "mg_sweep_pair_lower" : (xin ? "mg_sweep_pair" : "mg_sweep_pair_zero");
    int zc = sweep4_chunk<T>(c, l);
    dim3 grid(div_up(l.n[0], Cfg::TX), div_up(l.n[1], Cfg::TY), div_up(l.n[2], zc));
    PARIS_LAUNCH_N(c, kname<T>(label), l.N, k_rb_sweep4_cfg<Cfg>, grid, Cfg::NT, sweep4_smem_cfg<Cfg>(), view(l), xin,
                   xout, xc, c->bnd, first, zc);
    return PARIS_OK;
}

template <typename T>
static LV<T> view_x(const FastLevel<T>& l, T* x) {
    LV<T> v = view(l);
    v.x = x;
    return v;
}

// one V(nu1,nu2) cycle on level 0 from x0 = 0 with the right-hand side in b0
// (nuc sweeps each way instead on the levels cf..ct, when nuc > 0);
// *x0 receives the buffer holding the level-0 result (lv[0].x or lv[0].x2)
template <typename T>
static int vcycle(paris_ctx* c, int nu1_, int nu2_, T** x0) {
    const int nuc = c->fast_nuc, cf = c->fast_cf, ct = c->fast_ct;
    auto& lv = levels<T>(c);
    int nl = (int)lv.size();
    int Lc = 0;
    while (Lc < nl - 1 && lv[Lc].N > kCoarseCells) Lc++;
    T* cur[kMaxLevels];
    for (int L = 0; L < Lc; L++) {
        const FastLevel<T>& l = lv[L];
        const int nu1 = nu_at(L, nu1_, nuc, cf, ct);
        bool restricted = false;   // the last pre-smoothing sweep formed lv[L+1].b
        if (l.x2 && nu1 > 0) {
            const T* in = nullptr;
            T* out = l.x;
            for (int s = 0; s < nu1;) {
                if (l.pairs && s + 1 < nu1) {
                    PARIS_CHECK(sweep_pair<T>(c, L, l, in, out, nullptr, 0));
                    s += 2;
                } else if (l.rs && s + 1 == nu1) {
                    if constexpr (std::is_same<T, float>::value) PARIS_CHECK(sweep_rs(c, l, lv[L + 1], in, out, 0));
                    restricted = true;
                    s += 1;
                } else {
                    PARIS_CHECK(sweep_fused<T>(c, L, l, in, out, nullptr, 0));
                    s += 1;
                }
                in = out;
                out = out == l.x ? l.x2 : l.x;
            }
            cur[L] = (T*)in;
        } else {
            PARIS_CUDA_TRY(c, cudaMemsetAsync(l.x, 0, l.N * sizeof(T), c->stream));
            LV<T> v = view(l);
            for (int s = 0; s < nu1; s++) {
                PARIS_LAUNCH_N(c, kname<T>("mg_smooth"), v.N, k_fast_smooth<T>, row_grid((v.n0 + 1) / 2, v.n1, v.n2), 128, 0, v, c->bnd, 0);
                PARIS_LAUNCH_N(c, kname<T>("mg_smooth"), v.N, k_fast_smooth<T>, row_grid((v.n0 + 1) / 2, v.n1, v.n2), 128, 0, v, c->bnd, 1);
            }
            cur[L] = l.x;
        }
        LV<T> cv = view(lv[L + 1]);
        if (!restricted)
            PARIS_LAUNCH_N(c, kname<T>("mg_restrict"), l.N, k_fast_restrict2<T>,
                           dim3(div_up(cv.n0, 32), cv.n1, cv.n2), dim3(32, 4), 0, view_x(l, cur[L]), cv, c->bnd);
    }
    LVSet<T> S;
    for (int L = 0; L < nl; L++) S.l[L] = view(lv[L]);
    // the levels run in shared memory when they fit (always for L0 <= 16^3)
    // (the shared-memory cycle adds a scratch array of the largest restricted level)
    const size_t scratch = coarse_smem(lv, Lc) / sizeof(T);
    size_t csm = coarse_smem(lv, Lc) + (Lc < nl - 1 ? (size_t)lv[Lc].N * sizeof(T) : 0);
    const int in_smem = csm <= kCoarseSmemMax ? 1 : 0;
    if (!in_smem) csm = 0;
    if (in_smem) {
        static size_t csm_set = 0;   // opt-in size set for this instantiation
        if (csm > csm_set) {
            PARIS_CUDA_TRY(c, cudaFuncSetAttribute(k_coarse_cycle_smem<T>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
            csm_set = csm;
        }
        PARIS_LAUNCH_N(c, kname<T>("mg_coarse_cycle"), lv[Lc].N, k_coarse_cycle_smem<T>, 1, 1024, csm, S, Lc, nl,
                       c->bnd, nu1_, nu2_, nuc, cf, ct, (int)scratch);
    } else {
        PARIS_LAUNCH_N(c, kname<T>("mg_coarse_cycle"), lv[Lc].N, k_fast_coarse_cycle<T>, 1, 1024, 0, S, Lc, nl,
                       c->bnd, nu1_, nu2_, nuc, cf, ct, 0);
    }
    cur[Lc] = lv[Lc].x;
    for (int L = Lc - 1; L >= 0; L--) {
        const FastLevel<T>& l = lv[L];
        const int nu2 = nu_at(L, nu2_, nuc, cf, ct);
        if (l.x2 && nu2 > 0) {
            T* in = cur[L];
            for (int s = 0; s < nu2;) {
                T* out = in == l.x ? l.x2 : l.x;
                const T* xc = s == 0 ? cur[L + 1] : nullptr;
                if (l.pairs && s + 1 < nu2) {
                    PARIS_CHECK(sweep_pair<T>(c, L, l, in, out, xc, 1));
                    s += 2;
                } else {
                    // the last sweep of the cycle on the finest level also forms
                    // the partials of r.z for the CG, when asked to
                    const bool last = L == 0 && s + 1 == nu2 && c->bx_part;
                    int nb = 0;
                    PARIS_CHECK(sweep_fused<T>(c, L, l, in, out, xc, 1, last ? c->bx_part : nullptr, &nb));
                    if (last && nb > 0) c->bx_blocks = nb;
                    s += 1;
                }
                in = out;
            }
            cur[L] = in;
        } else {
            LV<T> v = view_x(l, cur[L]);
            PARIS_LAUNCH_N(c, kname<T>("mg_prolong"), v.N, k_fast_prolong<T>, row_grid(v.n0, v.n1, v.n2), 128, 0, v,
                           view_x(lv[L + 1], cur[L + 1]));
            for (int s = 0; s < nu2; s++) {
                PARIS_LAUNCH_N(c, kname<T>("mg_smooth"), v.N, k_fast_smooth<T>, row_grid((v.n0 + 1) / 2, v.n1, v.n2), 128, 0, v, c->bnd, 1);
                PARIS_LAUNCH_N(c, kname<T>("mg_smooth"), v.N, k_fast_smooth<T>, row_grid((v.n0 + 1) / 2, v.n1, v.n2), 128, 0, v, c->bnd, 0);
            }
        }
    }
    *x0 = cur[0];
    return PARIS_OK;
}

static bool converged(const paris_solve_opts* o, double s2, double s1, double bn2, long N, double* tres,
                      double* rel) {
    *rel = bn2 > 0.0 ? sqrt(s2 / bn2) : sqrt(s2);
    *tres = o->norm == 1 ? s1 / (double)N : sqrt(s2 / (double)N);
    if (o->rel_tol > 0.0) return *rel < o->rel_tol;
    return *tres < o->max_error;
}

template <typename T>
static int solve_dc(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* res, const double* rhs, double* p) {
    auto& lv = levels<T>(c);
    Mat64 A{c->cx, c->cy, c->cz, rhs};
    double s[3], tres, rel;
    PARIS_LAUNCH_N(c, kname<T>("mg_residual_fp64"), c->N, k_fast_residual64<T>, red_grid(c, k_fast_residual64<T>, 256), kRowBlock, 0, A, p, c->L, c->bnd, lv[0].b, (double*)nullptr,
                 c->red_part);
    PARIS_CHECK(ctx_reduce_finish(c, 3, s));
    double bn2 = s[2];
    bool done = converged(o, s[0], s[1], bn2, c->N, &tres, &rel);
    res->res0 = tres;
    int it = 0;
    int nu1 = o->nu1 > 0 ? o->nu1 : 2, nu2 = o->nu2 > 0 ? o->nu2 : 2;
    while (!done && it < o->maxit) {
        T* x0;
        PARIS_CHECK(vcycle<T>(c, nu1, nu2, &x0));
        PARIS_LAUNCH_N(c, kname<T>("mg_correct"), c->N, k_fast_correct<T>, row_grid(c->d.nx, c->d.ny, c->d.nz), 128, 0, p, x0, c->L, 1.0);
        PARIS_LAUNCH_N(c, kname<T>("mg_residual_fp64"), c->N, k_fast_residual64<T>, red_grid(c, k_fast_residual64<T>, 256), kRowBlock, 0, A, p, c->L, c->bnd, lv[0].b, (double*)nullptr,
                     c->red_part);
        PARIS_CHECK(ctx_reduce_finish(c, 3, s));
        it++;
        done = converged(o, s[0], s[1], bn2, c->N, &tres, &rel);
        if (tres != tres) {
            ctx_set_error(c, "pressure residual is NaN after %d cycles", it);
            res->it = it; res->res = tres; res->rel_res = rel;
            return PARIS_NAN_DETECTED;
        }
    }
    res->it = done ? it : o->maxit + 1;
    res->res = tres;
    res->rel_res = rel;
    return done ? PARIS_OK : PARIS_NOT_CONVERGED;
}

// a PCG vector, zero on allocation: the first direction d = z + 0*d must not
// read uninitialised memory (0 * NaN is NaN)
static int alloc_vec(paris_ctx* c, double** p) {
    if (!*p) {
        PARIS_CUDA_TRY(c, cudaMalloc(p, c->N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMemsetAsync(*p, 0, c->N * sizeof(double), c->stream));
    }
    return PARIS_OK;
}

// z = V(rT): one V-cycle on the right-hand side already in lv[0].b; returns
// the buffer holding z; r.z goes to the device-side scalar slot rzs
template <typename T>
static int precondition(paris_ctx* c, int nu1, int nu2, T** z, int rzs) {
    // r.z from the cycle's last finest-level sweep (r as the FP32 right-hand
    // side it smooths, rT; the same FP64 r in the FP64 cycle), or a pass of its own
    c->bx_part = c->red_part;
    c->bx_blocks = 0;
    PARIS_CHECK(vcycle<T>(c, nu1, nu2, z));
    c->bx_part = nullptr;
    if (c->bx_blocks > 0) {
        c->red_nb = c->bx_blocks;
    } else {
        PARIS_LAUNCH_N(c, kname<T>("pcg_rz"), c->N, k_pcg_rz<T>, red_grid(c, k_pcg_rz<T>, 256), 256, 0, *z,
                       c->fast_r64, c->N, c->red_part);
    }
    PARIS_LAUNCH(c, k_cg_reduce, 1, 256, 0, c->red_part, c->cg_scal + rzs, (double*)nullptr, c->red_nb);
    return PARIS_OK;
}

// Flexible CG (Polak-Ribiere beta) preconditioned by one V-cycle, in FP64.
// z stays in the V-cycle's output buffer until the next V-cycle starts: the
// update kernel forms r.zold before that.  The residual is updated
// recursively; when it meets the tolerance the true residual b - A p is
// formed and checked, and CG restarts from it (at most kMaxRestarts times)
// when rounding has let the two drift apart, so the residual reported is the
// true one.
static constexpr int kMaxRestarts = 2;
template <typename T>
static int solve_pcg(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* res, const double* rhs, double* p) {
    auto& lv = levels<T>(c);
    for (double** v : {&c->fast_r64, &c->fast_d64, &c->fast_q64}) PARIS_CHECK(alloc_vec(c, v));
    Mat64 A{c->cx, c->cy, c->cz, rhs};
    double s[3], tres, rel;
    PARIS_LAUNCH_N(c, kname<T>("mg_residual_fp64"), c->N, k_fast_residual64<T>, red_grid(c, k_fast_residual64<T>, 256), kRowBlock, 0, A, p, c->L, c->bnd, lv[0].b, c->fast_r64,
                 c->red_part);
    PARIS_CHECK(ctx_reduce_finish(c, 3, s));
    double bn2 = s[2];
    bool done = converged(o, s[0], s[1], bn2, c->N, &tres, &rel);
    res->res0 = tres;
    int it = 0;
    int nu1 = o->nu1 > 0 ? o->nu1 : 2, nu2 = o->nu2 > 0 ? o->nu2 : 2;
    // The scalars alpha and beta are formed on the device from the reduced
    // dot products (cg_scal), so an iteration waits on the host once, for the
    // residual norms after the update; r.z alternates between two slots.
    int rzs = kScRZ0;
    T* z = nullptr;
    double* const sc = c->cg_scal;
    if (!done) {
        PARIS_CHECK(precondition<T>(c, nu1, nu2, &z, rzs));
        PARIS_LAUNCH_N(c, kname<T>("pcg_dir"), c->N, k_pcg_dir<T>, div_up(c->N, 256), 256, 0, c->fast_d64, z, sc, rzs,
                       -1, c->N);
    }
    int restarts = 0;
    while (!done && it < o->maxit) {
        PARIS_LAUNCH_N(c, "pcg_matvec_fp64", c->N, k_pcg_matvec, red_grid(c, k_pcg_matvec, 256), kRowBlock, 0, A, c->fast_d64, c->fast_q64, c->L, c->bnd, c->red_part);
        PARIS_LAUNCH(c, k_cg_reduce, 1, 256, 0, c->red_part, sc + kScDQ, c->red_host_dev + 3, c->red_nb);
        PARIS_LAUNCH_N(c, kname<T>("pcg_update"), c->N, k_pcg_update<T>, red_grid(c, k_pcg_update<T>, 256), kRowBlock, 0, p, c->fast_r64, c->fast_d64, c->fast_q64, lv[0].b, z, sc, rzs, c->L,
                     c->red_part);
        PARIS_LAUNCH(c, k_cg_reduce, 3, 256, 0, c->red_part, sc + kScRR, c->red_host_dev, c->red_nb);
        PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        const double dq = c->red_host[3];
        for (int q = 0; q < 3; q++) s[q] = c->red_host[q];
        if (!(dq > 0.0)) break;   // the update wrote nothing: p and r are as they were
        it++;
        done = converged(o, s[0], s[1], bn2, c->N, &tres, &rel);
        if (tres != tres) {
            ctx_set_error(c, "pressure residual is NaN after %d iterations", it);
            res->it = it; res->res = tres; res->rel_res = rel;
            return PARIS_NAN_DETECTED;
        }
        if (done) {
            // the true residual (also the right-hand side of a restart)
            PARIS_LAUNCH_N(c, kname<T>("mg_residual_fp64"), c->N, k_fast_residual64<T>,
                           red_grid(c, k_fast_residual64<T>, 256), kRowBlock, 0, A, p, c->L, c->bnd, lv[0].b,
                           c->fast_r64, c->red_part);
            PARIS_CHECK(ctx_reduce_finish(c, 3, s));
            done = converged(o, s[0], s[1], bn2, c->N, &tres, &rel);
            if (done || restarts == kMaxRestarts) break;
            restarts++;
            rzs = kScRZ0 + 1 - rzs;
            PARIS_CHECK(precondition<T>(c, nu1, nu2, &z, rzs));
            PARIS_LAUNCH_N(c, kname<T>("pcg_dir"), c->N, k_pcg_dir<T>, div_up(c->N, 256), 256, 0, c->fast_d64, z, sc,
                           rzs, -1, c->N);
            continue;
        }
        const int rzs_new = kScRZ0 + 1 - rzs;
        PARIS_CHECK(precondition<T>(c, nu1, nu2, &z, rzs_new));
        PARIS_LAUNCH_N(c, kname<T>("pcg_dir"), c->N, k_pcg_dir<T>, div_up(c->N, 256), 256, 0, c->fast_d64, z, sc,
                       rzs_new, rzs, c->N);
        rzs = rzs_new;
    }
    res->it = done ? it : o->maxit + 1;
    res->res = tres;
    res->rel_res = rel;
    return done ? PARIS_OK : PARIS_NOT_CONVERGED;
}

// Interior sum of a ghosted field (slot 0 of the reduction buffer).
__global__ void k_interior_sum(const double* __restrict__ x, const Layout L, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        s += x[lidx(L, i, j, k)];
    ROWS_END
    s = block_sum<256>(s, sh);
    if (linear_tid() == 0) part[blockIdx.x] = s;
}

__global__ void k_interior_shift(double* __restrict__ x, const Layout L, double m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const long n = lidx(L, i, blockIdx.y, blockIdx.z);
    x[n] = x[n] + m;
}

// Walls (shear walls included) and periodic boundaries leave the pressure
// equation singular: constants are its null space.
static bool singular(const paris_ctx* c) {
    for (int a = 0; a < 3; a++)
        if (!c->bnd.per[a] && !(c->bnd.wall_lo[a] && c->bnd.wall_hi[a])) return false;
    return true;
}

int mg_fast_solve_into(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* res, const double* rhs,
                       double* x) {
    if (!c->have_matrix) return PARIS_BAD_ARGS;
    if (o->nu_coarse < 0 || o->coarse_from < 0 || o->coarse_to < 0) {
        ctx_set_error(c, "NewSolver: negative nu_coarse, coarse_from or coarse_to");
        return PARIS_BAD_ARGS;
    }
    // A singular system is solved from its initial guess with the mean taken
    // out, and the mean is put back afterwards.  A warm start with a large
    // constant part (the hydrostatic pressure of the previous step) otherwise
    // leaves a rounding-sized mean in r = b - A x: the inconsistent part of
    // the singular system, which the V-cycle's coarsest level turns into a
    // growing constant in the search direction, and PCG stalls.
    double shift = 0.0;
    if (singular(c)) {
        PARIS_LAUNCH_N(c, "mean_shift", c->N, k_interior_sum, red_grid(c, k_interior_sum, 256), kRowBlock, 0, x, c->L,
                       c->red_part);
        double sum;
        PARIS_CHECK(ctx_reduce_finish(c, 1, &sum));
        shift = sum / (double)c->N;
        if (shift != 0.0 && shift == shift)
            PARIS_LAUNCH_N(c, "mean_shift", c->N, k_interior_shift, row_grid(c->d.nx, c->d.ny, c->d.nz), 128, 0, x,
                           c->L, -shift);
        else
            shift = 0.0;
    }
    // the smoother's relaxation factor: the reference's BETA of RedBlackRelax
    // on the finest level, beta_coarse (when given) below it
    const double omega = o->beta > 0.0 ? o->beta : 1.0;
    const double omega_c = o->beta_coarse > 0.0 ? o->beta_coarse : omega;
    // sweeps on the coarser levels (coarse_from..coarse_to) when nu_coarse > 0
    c->fast_nuc = o->nu_coarse;
    c->fast_cf = o->coarse_from > 0 ? o->coarse_from : 1;
    c->fast_ct = o->coarse_to;
    int st;
    if (o->mode == PARIS_MG_MIXED) {
        PARIS_CHECK(fast_alloc<float>(c));
        PARIS_CHECK(fast_coefs<float>(c));
        for (size_t L = 0; L < c->fl32.size(); L++) c->fl32[L].omega = L == 0 ? omega : omega_c;
        st = o->pcg ? solve_pcg<float>(c, o, res, rhs, x) : solve_dc<float>(c, o, res, rhs, x);
    } else {
        PARIS_CHECK(fast_alloc<double>(c));
        PARIS_CHECK(fast_coefs<double>(c));
        for (size_t L = 0; L < c->fl64.size(); L++) c->fl64[L].omega = L == 0 ? omega : omega_c;
        st = o->pcg ? solve_pcg<double>(c, o, res, rhs, x) : solve_dc<double>(c, o, res, rhs, x);
    }
    if (c->err_host && *c->err_host) {   // the kernels before the last reduction have completed
        *c->err_host = 0;
        ctx_set_error(c, "a staging wait of the fused multigrid sweep ran out");
        return PARIS_CUDA_ERROR;
    }
    if (shift != 0.0)
        PARIS_LAUNCH_N(c, "mean_shift", c->N, k_interior_shift, row_grid(c->d.nx, c->d.ny, c->d.nz), 128, 0, x, c->L,
                       shift);
    if (st == PARIS_OK || st == PARIS_NOT_CONVERGED) PARIS_CHECK(ctx_ghost_fill(c, x));
    return st;
}

int mg_fast_solve(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* res) {
    return mg_fast_solve_into(c, o, res, c->rhs, c->fld[PARIS_FIELD_P]);
}
