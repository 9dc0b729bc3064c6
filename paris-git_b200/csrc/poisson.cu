// poisson.cu -- assembly of the variable-density pressure equation and the
// velocity correction: SetPressureBC + SetupPoisson + check_poisson_setup
// (modules.f90:916-949,2722-2892; newsolver.f90:275-344), Setup_testMG
// (modules.f90:3160-3192), calcResiduals (modules.f90:3313-3387),
// get_MGtest_err (MGsolver.f90:407-426) and project_velocity
// (paris.f90:882-909).  Built with -fmad=false: every expression keeps the
// reference's operation order, so A and u agree bit for bit with the FP64
// restatement of the reference.
#include "ctx.cuh"

#define CELL_LOOP_HEAD(L)                                                        \
    int i = blockIdx.x * blockDim.x + threadIdx.x;                               \
    int j = blockIdx.y * blockDim.y + threadIdx.y;                               \
    int k = blockIdx.z;                                                          \
    if (i >= (L).n[0] || j >= (L).n[1] || k >= (L).n[2]) return;

static inline dim3 cell_block() { return dim3(128, 2, 1); }
static inline dim3 cell_grid(const Layout& L) {
    return dim3(div_up(L.n[0], 128), div_up(L.n[1], 2), L.n[2]);
}

// mask of face f (interior-relative index of u(f), the face f+1/2) in
// direction d: zero on wall faces (SetPressureBC, modules.f90:916-949)
__device__ inline double face_mask(const Bnd& B, const Layout& L, int d, int f) {
    if (f == -1 && B.wall_lo[d]) return 0.0;
    if (f == L.n[d] - 1 && B.wall_hi[d]) return 0.0;
    return 1.0;
}

struct Metric {
    const double *dx, *dxh, *dy, *dyh, *dz, *dzh;   // index i + ng
};

// SetupPoisson in the compact form used by the solvers: the east/north/top
// coefficients A2, A4, A6 and the right-hand side A8 of every cell, plus the
// checks of check_and_debug_Poisson / check_poisson_setup.
// part slots: 0 = sum A8, 1 = number of cells failing a check
// x / d of the divergence, or x * rd where every d of the axis is the same
// power of two: 1/d is then exact and the product is the same double
template <bool R>
__device__ inline double div_metric(double x, double d, double rd) {
    return R ? x * rd : x / d;
}

// num / den is a number >= 0 (no NaN; -0 counts as 0) whenever den is
// nonzero, num is zero or of den's sign, and not both are infinite
__device__ inline bool quot_nonneg(double num, double den) {
    if (isinf(num) && isinf(den)) return false;
    return (num >= 0.0 && den > 0.0) || (num <= 0.0 && den < 0.0);
}

// A1, A3, A5 (the west, south and bottom faces) are stored by the
// neighbours as their A2, A4, A6; here they only enter the check of the cell.
// When all six coefficients are numbers >= 0, A7 = A1 + .. + A6 is at least
// the largest of them (each rounded partial sum of non-negative terms is at
// least its last term), so A2, A4 and A6 decide the check whenever one of
// them is >= 1e-50, and the three quotients are formed only otherwise.
template <bool R>
__global__ void __launch_bounds__(256, 3) k_setup_poisson(const double* __restrict__ u, const double* __restrict__ v,
                                const double* __restrict__ w, const double* __restrict__ rho,
                                double* __restrict__ cx, double* __restrict__ cy, double* __restrict__ cz,
                                double* __restrict__ rhs, const Layout L, const Bnd B, const Metric M,
                                double rdx, double rdy, double rdz, double dt, double volsrc, double* part) {
    __shared__ double sh[32];
    double s_rhs = 0.0, s_bad = 0.0;
    const int g = L.ng;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        long t = cidx(L.n[0], L.n[1], i, j, k);
        long n = lidx(L, i, j, k);
        double r0 = rho[n];
        const double n1 = 2.0 * dt * face_mask(B, L, 0, i - 1), d1 = M.dx[i + g] * M.dxh[i - 1 + g] * (rho[n - 1] + r0);
        const double n2 = 2.0 * dt * face_mask(B, L, 0, i), d2 = M.dx[i + g] * M.dxh[i + g] * (rho[n + 1] + r0);
        const double n3 = 2.0 * dt * face_mask(B, L, 1, j - 1),
                     d3 = M.dy[j + g] * M.dyh[j - 1 + g] * (rho[n - L.pitch] + r0);
        const double n4 = 2.0 * dt * face_mask(B, L, 1, j), d4 = M.dy[j + g] * M.dyh[j + g] * (rho[n + L.pitch] + r0);
        const double n5 = 2.0 * dt * face_mask(B, L, 2, k - 1),
                     d5 = M.dz[k + g] * M.dzh[k - 1 + g] * (rho[n - L.plane] + r0);
        const double n6 = 2.0 * dt * face_mask(B, L, 2, k), d6 = M.dz[k + g] * M.dzh[k + g] * (rho[n + L.plane] + r0);
        const double a2 = n2 / d2, a4 = n4 / d4, a6 = n6 / d6;
        double a8 = -(volsrc + div_metric<R>(u[n] - u[n - 1], M.dx[i + g], rdx) +
                      div_metric<R>(v[n] - v[n - L.pitch], M.dy[j + g], rdy) +
                      div_metric<R>(w[n] - w[n - L.plane], M.dz[k + g], rdz));
        cx[t] = a2; cy[t] = a4; cz[t] = a6; rhs[t] = a8;
        bool bad = a8 != a8;
        const bool decided = quot_nonneg(n1, d1) && quot_nonneg(n3, d3) && quot_nonneg(n5, d5) && a2 >= 0.0 &&
                             a4 >= 0.0 && a6 >= 0.0 && fmax(a2, fmax(a4, a6)) >= 1e-50;
        if (!decided) {
            const double a1 = n1 / d1, a3 = n3 / d3, a5 = n5 / d5;
            const double a7 = a1 + a2 + a3 + a4 + a5 + a6;
            bad = bad || a1 != a1 || a2 != a2 || a3 != a3 || a4 != a4 || a5 != a5 || a6 != a6 || a7 != a7;
            if (a7 < 1e-50) bad = true;   // no solid cells on this grid: A7 tiny is an error
        }
        s_rhs += a8;
        s_bad += bad ? 1.0 : 0.0;
    ROWS_END
    s_rhs = block_sum<256>(s_rhs, sh);
    s_bad = block_sum<256>(s_bad, sh);
    if (linear_tid() == 0) {
        part[blockIdx.x] = s_rhs;
        part[kRedBlocks + blockIdx.x] = s_bad;
    }
}

// The full A(is:ie,js:je,ks:ke,8) of the reference from rho and the stored
// right-hand side (same formulas as k_setup_poisson; A1,A3,A5 with the
// dx(i)*dxh(i-1) metric of the cell itself).
__global__ void k_full_A(const double* __restrict__ rho, const double* __restrict__ rhs, double* __restrict__ A,
                         const Layout L, const Bnd B, const Metric M, double dt, int with_mask) {
    CELL_LOOP_HEAD(L)
    const int g = L.ng;
    long n = lidx(L, i, j, k);
    long N = (long)L.n[0] * L.n[1] * L.n[2];
    long m = cidx(L.n[0], L.n[1], i, j, k);
    double r0 = rho[n];
    double f1 = with_mask ? 2.0 * dt * face_mask(B, L, 0, i - 1) : 2.0;
    double f2 = with_mask ? 2.0 * dt * face_mask(B, L, 0, i) : 2.0;
    double f3 = with_mask ? 2.0 * dt * face_mask(B, L, 1, j - 1) : 2.0;
    double f4 = with_mask ? 2.0 * dt * face_mask(B, L, 1, j) : 2.0;
    double f5 = with_mask ? 2.0 * dt * face_mask(B, L, 2, k - 1) : 2.0;
    double f6 = with_mask ? 2.0 * dt * face_mask(B, L, 2, k) : 2.0;
    double a1 = f1 / (M.dx[i + g] * M.dxh[i - 1 + g] * (rho[n - 1] + r0));
    double a2 = f2 / (M.dx[i + g] * M.dxh[i + g] * (rho[n + 1] + r0));
    double a3 = f3 / (M.dy[j + g] * M.dyh[j - 1 + g] * (rho[n - L.pitch] + r0));
    double a4 = f4 / (M.dy[j + g] * M.dyh[j + g] * (rho[n + L.pitch] + r0));
    double a5 = f5 / (M.dz[k + g] * M.dzh[k - 1 + g] * (rho[n - L.plane] + r0));
    double a6 = f6 / (M.dz[k + g] * M.dzh[k + g] * (rho[n + L.plane] + r0));
    A[0 * N + m] = a1; A[1 * N + m] = a2; A[2 * N + m] = a3;
    A[3 * N + m] = a4; A[4 * N + m] = a5; A[5 * N + m] = a6;
    A[6 * N + m] = a1 + a2 + a3 + a4 + a5 + a6;
    A[7 * N + m] = rhs[m];
}

static Metric metric(const paris_ctx* c) { return Metric{c->dx, c->dxh, c->dy, c->dyh, c->dz, c->dzh}; }

// every interior spacing d[g..g+n) of an axis (host copy, the doubles the
// device holds) is the same power of two: *r = its exact reciprocal
static bool uniform_pow2(const std::vector<double>& d, int n, int g, double* r) {
    if ((int)d.size() < n + g) return false;
    for (int i = g; i < n + g; i++)
        if (d[i] != d[g]) return false;
    int e;
    const double m = std::frexp(d[g], &e);
    if (m != 0.5) return false;
    *r = 1.0 / d[g];
    return true;
}

int poisson_build_full_A(paris_ctx* c) {
    if (c->A_from_upload) { c->A_valid = 1; return PARIS_OK; }
    if (!c->A) PARIS_CUDA_TRY(c, cudaMalloc(&c->A, 8 * c->N * sizeof(double)));
    int with_mask = c->setup_dt != 0.0 ? 1 : 0;
    PARIS_LAUNCH(c, k_full_A, cell_grid(c->L), cell_block(), 0, c->fld[PARIS_FIELD_RHO], c->rhs, c->A, c->L,
                 c->bnd, metric(c), c->setup_dt, with_mask);
    c->A_valid = 1;
    return PARIS_OK;
}

extern "C" int paris_setup_poisson(paris_handle_t c, double dt, double volume_source) {
    if (!c) return PARIS_BAD_ARGS;
    if (!(dt > 0.0)) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_ensure_matrix(c));
    double rd[3];
    if (uniform_pow2(c->h_dx, c->d.nx, c->L.ng, &rd[0]) && uniform_pow2(c->h_dy, c->d.ny, c->L.ng, &rd[1]) &&
        uniform_pow2(c->h_dz, c->d.nz, c->L.ng, &rd[2]))
        PARIS_LAUNCH_N(c, "setup_poisson", c->N, k_setup_poisson<true>, red_grid(c, k_setup_poisson<true>, 256),
                       kRowBlock, 0, c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W],
                       c->fld[PARIS_FIELD_RHO], c->cx, c->cy, c->cz, c->rhs, c->L, c->bnd, metric(c), rd[0], rd[1],
                       rd[2], dt, volume_source, c->red_part);
    else
        PARIS_LAUNCH_N(c, "setup_poisson", c->N, k_setup_poisson<false>, red_grid(c, k_setup_poisson<false>, 256),
                       kRowBlock, 0, c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W],
                       c->fld[PARIS_FIELD_RHO], c->cx, c->cy, c->cz, c->rhs, c->L, c->bnd, metric(c), 0.0, 0.0, 0.0,
                       dt, volume_source, c->red_part);
    double out[2];
    PARIS_CHECK(ctx_reduce_finish(c, 2, out));
    c->have_matrix = 1;
    c->A_valid = 0;
    c->A_from_upload = 0;
    c->setup_dt = dt;
    if (out[1] > 0.0) {
        ctx_set_error(c, "SetupPoisson: %g cells with NaN in A or A7 tiny outside a solid", out[1]);
        return PARIS_SETUP_ERROR;
    }
    if (out[0] / (double)c->N > 1e-10) {
        ctx_set_error(c, "SetupPoisson: large volume source %g", out[0] / (double)c->N);
        return PARIS_SETUP_ERROR;
    }
    return PARIS_OK;
}

// Setup_testMG: no dt, no masks, RHS 3(2 pi)^2 sin sin sin with the
// single-precision literal pi = 3.14159265359 held in real(8)
__global__ void k_test_rhs(double* __restrict__ rhs, const Layout L, const double* __restrict__ xc,
                           const double* __restrict__ yc, const double* __restrict__ zc) {
    CELL_LOOP_HEAD(L)
    const double pi = (double)3.14159265359f;
    const int g = L.ng;
    rhs[cidx(L.n[0], L.n[1], i, j, k)] =
        3.0 * ((2.0 * pi) * (2.0 * pi)) * sin(2. * pi * xc[i + g]) * sin(2. * pi * yc[j + g]) * sin(2. * pi * zc[k + g]);
}

__global__ void k_compact_from_A(const double* __restrict__ A, double* cx, double* cy, double* cz, long N) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= N) return;
    cx[t] = A[1 * N + t]; cy[t] = A[3 * N + t]; cz[t] = A[5 * N + t];
}

extern "C" int paris_setup_test_mg(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_ensure_matrix(c));
    PARIS_LAUNCH(c, k_test_rhs, cell_grid(c->L), cell_block(), 0, c->rhs, c->L, c->xc, c->yc, c->zc);
    c->setup_dt = 0.0;   // marks "no dt, no mask" for the full-A builder
    c->A_from_upload = 0;
    PARIS_CHECK(poisson_build_full_A(c));
    PARIS_LAUNCH(c, k_compact_from_A, div_up(c->N, 256), 256, 0, c->A, c->cx, c->cy, c->cz, c->N);
    c->have_matrix = 1;
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return PARIS_OK;
}

// calcResidual for NormOrder 1, 2 and 100 at once; slots: sum|r|, sum r^2, max|r|
__global__ void k_calc_residuals(const double* __restrict__ A, const double* __restrict__ p, const Layout L,
                                 double* part) {
    __shared__ double sh[32];
    long N = (long)L.n[0] * L.n[1] * L.n[2];
    double s1 = 0.0, s2 = 0.0, smax = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        long t = cidx(L.n[0], L.n[1], i, j, k);
        long n = lidx(L, i, j, k);
        double r = fabs(-p[n] * A[6 * N + t] + A[0 * N + t] * p[n - 1] + A[1 * N + t] * p[n + 1] +
                        A[2 * N + t] * p[n - L.pitch] + A[3 * N + t] * p[n + L.pitch] +
                        A[4 * N + t] * p[n - L.plane] + A[5 * N + t] * p[n + L.plane] + A[7 * N + t]);
        s1 += r;
        s2 += r * r;
        smax = fmax(smax, r);
    ROWS_END
    s1 = block_sum<256>(s1, sh);
    s2 = block_sum<256>(s2, sh);
    smax = block_max<256>(smax, sh);
    if (linear_tid() == 0) {
        part[blockIdx.x] = s1;
        part[kRedBlocks + blockIdx.x] = s2;
        part[2 * kRedBlocks + blockIdx.x] = smax;
    }
}

extern "C" int paris_calc_residuals(paris_handle_t c, double* out3) {
    if (!c || !out3 || !c->have_matrix) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    if (!c->A_valid) PARIS_CHECK(poisson_build_full_A(c));
    PARIS_LAUNCH(c, k_calc_residuals, red_grid(c, k_calc_residuals, 256), kRowBlock, 0, c->A, c->fld[PARIS_FIELD_P], c->L, c->red_part);
    double s[2], mx[1];
    PARIS_CHECK(ctx_reduce_finish(c, 2, s));
    // the max slot is reduced separately
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->red_part, c->red_part + 2 * kRedBlocks, kRedBlocks * sizeof(double),
                                      cudaMemcpyDeviceToDevice, c->stream));
    PARIS_CHECK(ctx_reduce_finish(c, 1, mx, 1));
    double n = (double)c->d.nx * (double)c->d.ny * (double)c->d.nz;
    out3[0] = s[0] / (double)c->d.nx / (double)c->d.ny / (double)c->d.nz;
    out3[1] = sqrt(s[1] / (double)c->d.nx / (double)c->d.ny / (double)c->d.nz);
    out3[2] = mx[0];
    (void)n;
    return PARIS_OK;
}

__global__ void k_mgtest_err(const double* __restrict__ p, const Layout L, const double* __restrict__ xc,
                             const double* __restrict__ yc, const double* __restrict__ zc, double* part) {
    __shared__ double sh[32];
    const double pi = (double)3.14159265359f;
    const int g = L.ng;
    long N = (long)L.n[0] * L.n[1] * L.n[2];
    double sr = 0.0, sf = 0.0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < N; t += (long)gridDim.x * blockDim.x) {
        int i = (int)(t % L.n[0]), j = (int)((t / L.n[0]) % L.n[1]), k = (int)(t / ((long)L.n[0] * L.n[1]));
        double s = sin(2. * pi * xc[i + g]) * sin(2. * pi * yc[j + g]) * sin(2. * pi * zc[k + g]);
        sr += fabs(p[lidx(L, i, j, k)] - s);
        sf += fabs(s);
    }
    sr = block_sum<256>(sr, sh);
    sf = block_sum<256>(sf, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sr;
        part[kRedBlocks + blockIdx.x] = sf;
    }
}

extern "C" int paris_mg_test_err(paris_handle_t c, double* err) {
    if (!c || !err) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_LAUNCH(c, k_mgtest_err, red_grid(c, k_mgtest_err, 256), 256, 0, c->fld[PARIS_FIELD_P], c->L, c->xc, c->yc, c->zc, c->red_part);
    double s[2];
    PARIS_CHECK(ctx_reduce_finish(c, 2, s));
    *err = s[0] / s[1];
    return PARIS_OK;
}

// project_velocity, paris.f90:898-909: the faces is..ieu (jev, kew) of every
// cell, ieu = ie-1 when x is not periodic.
__global__ void k_project(double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                          const double* __restrict__ p, const double* __restrict__ rho, const Layout L,
                          const Bnd B, const Metric M, double dt) {
    CELL_LOOP_HEAD(L)
    const int g = L.ng;
    long n = lidx(L, i, j, k);
    double p0 = p[n], r0 = rho[n];
    if (i < L.n[0] - 1 || B.per[0])
        u[n] = u[n] - dt * (2.0 * face_mask(B, L, 0, i) / M.dxh[i + g]) * (p[n + 1] - p0) / (rho[n + 1] + r0);
    if (j < L.n[1] - 1 || B.per[1])
        v[n] = v[n] - dt * (2.0 * face_mask(B, L, 1, j) / M.dyh[j + g]) * (p[n + L.pitch] - p0) / (rho[n + L.pitch] + r0);
    if (k < L.n[2] - 1 || B.per[2])
        w[n] = w[n] - dt * (2.0 * face_mask(B, L, 2, k) / M.dzh[k + g]) * (p[n + L.plane] - p0) / (rho[n + L.plane] + r0);
}

extern "C" int paris_project_velocity(paris_handle_t c, double dt) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_LAUNCH_N(c, "project_velocity", c->N, k_project, cell_grid(c->L), cell_block(), 0, c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V],
                 c->fld[PARIS_FIELD_W], c->fld[PARIS_FIELD_P], c->fld[PARIS_FIELD_RHO], c->L, c->bnd, metric(c), dt);
    // SetVelocityBC + do_ghost_vector follow the projection (paris.f90:590-591)
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_U]));
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_V]));
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_W]));
    return PARIS_OK;
}
