// mg_ref.cu -- the reference multigrid, step for step, in FP64 on the B200
// (PARIS_MG_REFERENCE): NewSolverMG / MG_iteration / get_MGmatrix_coef /
// fill_coefficients / coarse_from_fine / coarse_fine_interp / get_residual /
// compute_residual (MGsolver.f90:84-405) with RedBlackRelax and apply_BC_MG
// (newsolver.f90:192-247).  Levels are interior-only arrays: the one-layer
// halo of pMG/EMG is resolved in the kernels by periodic wrap, and is zero on
// walls, where ghost_MG_* never writes and the arrays are zeroed.  Every
// colour of a red-black pass only reads the other colour, so one thread per
// cell reproduces the sequential loop exactly.  Built with -fmad=false.
#include "ctx.cuh"

struct LvlDims {
    int n0, n1, n2;
    long N;
};

__device__ inline double nbr(const double* __restrict__ x, const LvlDims& d, const Bnd& B, int i, int j, int k) {
    if (i < 0 || i >= d.n0) { if (!B.per[0]) return 0.0; i = i < 0 ? i + d.n0 : i - d.n0; }
    if (j < 0 || j >= d.n1) { if (!B.per[1]) return 0.0; j = j < 0 ? j + d.n1 : j - d.n1; }
    if (k < 0 || k >= d.n2) { if (!B.per[2]) return 0.0; k = k < 0 ? k + d.n2 : k - d.n2; }
    return x[cidx(d.n0, d.n1, i, j, k)];
}

// RedBlackRelax, one colour: (i+j+k+color) even cells (local indices).
__global__ void k_ref_relax(const double* __restrict__ K, double* __restrict__ p, const LvlDims d, const Bnd B,
                            double beta, int color) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int h0 = (d.n0 + 1) / 2;
    if (t >= (long)h0 * d.n1 * d.n2) return;
    int ih = (int)(t % h0), j = (int)((t / h0) % d.n1), k = (int)(t / ((long)h0 * d.n1));
    int i = 2 * ih + ((j + k + color) & 1);
    if (i >= d.n0) return;
    long m = cidx(d.n0, d.n1, i, j, k);
    long N = d.N;
    p[m] = (1.0 - beta) * p[m] +
           beta / K[6 * N + m] *
               (K[0 * N + m] * nbr(p, d, B, i - 1, j, k) + K[1 * N + m] * nbr(p, d, B, i + 1, j, k) +
                K[2 * N + m] * nbr(p, d, B, i, j - 1, k) + K[3 * N + m] * nbr(p, d, B, i, j + 1, k) +
                K[4 * N + m] * nbr(p, d, B, i, j, k - 1) + K[5 * N + m] * nbr(p, d, B, i, j, k + 1) + K[7 * N + m]);
}

__device__ inline double powabs(double r, int norm) {
    double a = fabs(r);
    return norm == 2 ? a * a : (norm == 1 ? a : pow(a, (double)norm));
}

// get_residual: K8 <- K8 - K7 p + sum K_n p_n (in place); optional sum |r|^norm
__global__ void k_ref_get_residual(double* __restrict__ K, const double* __restrict__ p, const LvlDims d,
                                   const Bnd B, int norm, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    long N = d.N;
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < N; m += (long)gridDim.x * blockDim.x) {
        int i = (int)(m % d.n0), j = (int)((m / d.n0) % d.n1), k = (int)(m / ((long)d.n0 * d.n1));
        double r = K[7 * N + m] - K[6 * N + m] * p[m] + K[0 * N + m] * nbr(p, d, B, i - 1, j, k) +
                   K[1 * N + m] * nbr(p, d, B, i + 1, j, k) + K[2 * N + m] * nbr(p, d, B, i, j - 1, k) +
                   K[3 * N + m] * nbr(p, d, B, i, j + 1, k) + K[4 * N + m] * nbr(p, d, B, i, j, k - 1) +
                   K[5 * N + m] * nbr(p, d, B, i, j, k + 1);
        K[7 * N + m] = r;
        if (part) s += powabs(r, norm);
    }
    if (part) {
        s = block_sum<256>(s, sh);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

// compute_residual on the finest level with the caller's A and the ghosted p
__global__ void k_ref_compute_residual(const double* __restrict__ A, const double* __restrict__ p, const Layout L,
                                       int norm, double* part) {
    __shared__ double sh[32];
    double s = 0.0;
    long N = (long)L.n[0] * L.n[1] * L.n[2];
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < N; m += (long)gridDim.x * blockDim.x) {
        int i = (int)(m % L.n[0]), j = (int)((m / L.n[0]) % L.n[1]), k = (int)(m / ((long)L.n[0] * L.n[1]));
        long n = lidx(L, i, j, k);
        double r = A[7 * N + m] - A[6 * N + m] * p[n] + A[0 * N + m] * p[n - 1] + A[1 * N + m] * p[n + 1] +
                   A[2 * N + m] * p[n - L.pitch] + A[3 * N + m] * p[n + L.pitch] +
                   A[4 * N + m] * p[n - L.plane] + A[5 * N + m] * p[n + L.plane];
        s += powabs(r, norm);
    }
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// fill_coefficients: 0.125*(sum of the 8 children in the Fortran order)
__global__ void k_ref_fill_coef(const double* __restrict__ Kf, const LvlDims f, double* __restrict__ Kc,
                                const LvlDims c) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= 8 * c.N) return;
    int comp = (int)(t / c.N);
    long m = t % c.N;
    int i = (int)(m % c.n0), j = (int)((m / c.n0) % c.n1), k = (int)(m / ((long)c.n0 * c.n1));
    const double* F = Kf + comp * f.N;
    int I = 2 * i, J = 2 * j, Kk = 2 * k;
    double s = F[cidx(f.n0, f.n1, I, J, Kk)] + F[cidx(f.n0, f.n1, I, J + 1, Kk)] + F[cidx(f.n0, f.n1, I, J, Kk + 1)] +
               F[cidx(f.n0, f.n1, I, J + 1, Kk + 1)] + F[cidx(f.n0, f.n1, I + 1, J, Kk)] +
               F[cidx(f.n0, f.n1, I + 1, J + 1, Kk)] + F[cidx(f.n0, f.n1, I + 1, J, Kk + 1)] +
               F[cidx(f.n0, f.n1, I + 1, J + 1, Kk + 1)];
    Kc[comp * c.N + m] = 0.125 * s;
}

// coarse_from_fine: Ac8 = 0; Ac8 += Af8*0.125 with k1 fastest, then j1, i1
__global__ void k_ref_coarse_from_fine(const double* __restrict__ Kf, const LvlDims f, double* __restrict__ Kc,
                                       const LvlDims c) {
    long m = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (m >= c.N) return;
    int i = (int)(m % c.n0), j = (int)((m / c.n0) % c.n1), k = (int)(m / ((long)c.n0 * c.n1));
    const double* F = Kf + 7 * f.N;
    double s = 0.0;
    for (int i1 = 0; i1 < 2; i1++)
        for (int j1 = 0; j1 < 2; j1++)
            for (int k1 = 0; k1 < 2; k1++) s = s + F[cidx(f.n0, f.n1, 2 * i + i1, 2 * j + j1, 2 * k + k1)] * 0.125;
    Kc[7 * c.N + m] = s;
}

// coarse_fine_interp: injection (sym_MG: weights |pf| of the children)
__global__ void k_ref_interp(double* __restrict__ ef, const LvlDims f, const double* __restrict__ pc,
                             const LvlDims c, int sym) {
    long m = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (m >= c.N) return;
    int i = (int)(m % c.n0), j = (int)((m / c.n0) % c.n1), k = (int)(m / ((long)c.n0 * c.n1));
    double v = pc[m];
    long q[8];
    int t = 0;
    for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) q[t++] = cidx(f.n0, f.n1, 2 * i + di, 2 * j + dj, 2 * k + dk);
    if (sym) {
        double rt = fabs(ef[q[0]]) + fabs(ef[q[1]]) + fabs(ef[q[2]]) + fabs(ef[q[3]]) + fabs(ef[q[4]]) +
                    fabs(ef[q[5]]) + fabs(ef[q[6]]) + fabs(ef[q[7]]) + 1.e-15;
        for (int s = 0; s < 8; s++) ef[q[s]] = fabs(ef[q[s]]) / rt * v;
    } else {
        for (int s = 0; s < 8; s++) ef[q[s]] = v;
    }
}

__global__ void k_ref_add(double* __restrict__ a, const double* __restrict__ b, long N) {
    long m = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (m < N) a[m] = a[m] + b[m];
}

// pMG(LMG) <- p (interior) and p <- p + pMG(LMG)
__global__ void k_ref_field_io(double* __restrict__ pf, double* __restrict__ pm, const Layout L, int add) {
    long m = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long N = (long)L.n[0] * L.n[1] * L.n[2];
    if (m >= N) return;
    int i = (int)(m % L.n[0]), j = (int)((m / L.n[0]) % L.n[1]), k = (int)(m / ((long)L.n[0] * L.n[1]));
    long n = lidx(L, i, j, k);
    if (add) pf[n] = pf[n] + pm[m];
    else pm[m] = pf[n];
}

static LvlDims dims(const RefLevel& l) { return LvlDims{l.n[0], l.n[1], l.n[2], l.N}; }

static int ref_alloc(paris_ctx* c) {
    if (!c->ref.empty()) return PARIS_OK;
    int nd[3] = {c->d.nx, c->d.ny, c->d.nz};
    int lmg = 1000;
    for (int a = 0; a < 3; a++) {
        if (nd[a] & (nd[a] - 1)) {
            ctx_set_error(c, "multigrid requires 2^n cells per direction (MGsolver.f90:43-46)");
            return PARIS_BAD_ARGS;
        }
        int L = 0;
        while ((1 << (L + 1)) <= nd[a]) L++;
        lmg = L < lmg ? L : lmg;
    }
    if (lmg < 2) return PARIS_BAD_ARGS;
    c->ref_lmg = lmg;
    c->ref.resize(lmg + 1);
    for (int L = lmg; L >= 1; L--) {
        RefLevel& l = c->ref[L];
        for (int a = 0; a < 3; a++) l.n[a] = nd[a] >> (lmg - L);
        l.N = (long)l.n[0] * l.n[1] * l.n[2];
        PARIS_CUDA_TRY(c, cudaMalloc(&l.K, 8 * l.N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&l.p, l.N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&l.e, l.N * sizeof(double)));
    }
    return PARIS_OK;
}

static int relax(paris_ctx* c, RefLevel& l, double* x, double beta) {
    LvlDims d = dims(l);
    long nt = (long)((d.n0 + 1) / 2) * d.n1 * d.n2;
    PARIS_LAUNCH(c, k_ref_relax, div_up(nt, 256), 256, 0, l.K, x, d, c->bnd, beta, 0);
    PARIS_LAUNCH(c, k_ref_relax, div_up(nt, 256), 256, 0, l.K, x, d, c->bnd, beta, 1);
    return PARIS_OK;
}

static int get_residual(paris_ctx* c, RefLevel& l, double* x) {
    LvlDims d = dims(l);
    unsigned g = div_up(d.N, 256);
    if (g > 65535u) g = 65535u;
    PARIS_LAUNCH(c, k_ref_get_residual, g, 256, 0, l.K, x, d, c->bnd, 2, (double*)nullptr);
    return PARIS_OK;
}

// MG_iteration, MGsolver.f90:253-320
static int mg_iteration(paris_ctx* c, double beta, int nrelax, int sym) {
    int lmg = c->ref_lmg;
    for (int L = lmg; L >= 2; L--) {
        RefLevel& l = c->ref[L];
        PARIS_CUDA_TRY(c, cudaMemsetAsync(l.p, 0, l.N * sizeof(double), c->stream));
        for (int r = 0; r < nrelax; r++) PARIS_CHECK(relax(c, l, l.p, beta));
        PARIS_CHECK(get_residual(c, l, l.p));
        RefLevel& lc = c->ref[L - 1];
        PARIS_LAUNCH(c, k_ref_coarse_from_fine, div_up(lc.N, 256), 256, 0, l.K, dims(l), lc.K, dims(lc));
    }
    PARIS_CHECK(relax(c, c->ref[2], c->ref[2].p, beta));
    for (int L = 3; L <= lmg; L++) {
        RefLevel& l = c->ref[L];
        RefLevel& lc = c->ref[L - 1];
        PARIS_CUDA_TRY(c, cudaMemsetAsync(l.e, 0, l.N * sizeof(double), c->stream));
        PARIS_LAUNCH(c, k_ref_interp, div_up(lc.N, 256), 256, 0, l.e, dims(l), lc.p, dims(lc), sym);
        PARIS_CHECK(get_residual(c, l, l.e));
        PARIS_LAUNCH(c, k_ref_add, div_up(l.N, 256), 256, 0, l.p, l.e, l.N);
        PARIS_CUDA_TRY(c, cudaMemsetAsync(l.e, 0, l.N * sizeof(double), c->stream));
        for (int r = 0; r < nrelax; r++) PARIS_CHECK(relax(c, l, l.e, beta));
        PARIS_LAUNCH(c, k_ref_add, div_up(l.N, 256), 256, 0, l.p, l.e, l.N);
        PARIS_CHECK(get_residual(c, l, l.e));
    }
    return PARIS_OK;
}

// NewSolverMG, MGsolver.f90:346-405
int mg_ref_solve(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* res) {
    PARIS_CHECK(ref_alloc(c));
    if (!c->A_valid) PARIS_CHECK(poisson_build_full_A(c));
    int lmg = c->ref_lmg;
    RefLevel& lf = c->ref[lmg];
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(lf.K, c->A, 8 * lf.N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    for (int L = lmg - 1; L >= 1; L--)
        PARIS_LAUNCH(c, k_ref_fill_coef, div_up(8 * c->ref[L].N, 256), 256, 0, c->ref[L + 1].K, dims(c->ref[L + 1]),
                     c->ref[L].K, dims(c->ref[L]));
    double* p = c->fld[PARIS_FIELD_P];
    PARIS_LAUNCH(c, k_ref_field_io, div_up(lf.N, 256), 256, 0, p, lf.p, c->L, 0);
    PARIS_LAUNCH(c, k_ref_get_residual, red_grid(c, k_ref_get_residual, 256), 256, 0, lf.K, lf.p, dims(lf), c->bnd, o->norm, c->red_part);
    double s;
    PARIS_CHECK(ctx_reduce_finish(c, 1, &s));
    double nxyz = (double)c->d.nx * (double)c->d.ny * (double)c->d.nz;
    double tres2 = s / nxyz;
    res->res0 = o->norm == 2 ? sqrt(tres2) : tres2;
    PARIS_CUDA_TRY(c, cudaMemsetAsync(lf.p, 0, lf.N * sizeof(double), c->stream));
    int nrelax = c->d.nrelax > 0 ? c->d.nrelax : 3;
    int it;
    for (it = 1; it <= o->maxit; it++) {
        PARIS_CHECK(mg_iteration(c, o->beta, nrelax, c->d.sym_mg));
        PARIS_LAUNCH(c, k_ref_field_io, div_up(lf.N, 256), 256, 0, p, lf.p, c->L, 1);
        PARIS_CHECK(ctx_ghost_fill(c, p));
        PARIS_LAUNCH(c, k_ref_compute_residual, red_grid(c, k_ref_compute_residual, 256), 256, 0, c->A, p, c->L, o->norm, c->red_part);
        PARIS_CHECK(ctx_reduce_finish(c, 1, &s));
        tres2 = s / nxyz;
        if (o->norm == 2) tres2 = sqrt(tres2);
        if (tres2 != tres2) {
            res->it = it; res->res = tres2;
            ctx_set_error(c, "pressure residual is NaN after %d cycles", it);
            return PARIS_NAN_DETECTED;
        }
        if (tres2 < o->max_error) break;
    }
    res->it = it;
    res->res = tres2;
    return it == o->maxit + 1 ? PARIS_NOT_CONVERGED : PARIS_OK;
}
