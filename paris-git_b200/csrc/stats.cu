// stats.cu -- time-step control and flow statistics on the device:
// TimeStepSize without a free surface (paris.f90:968-1041) and
// get_cfl_and_check (paris.f90:1045-1074) as one max reduction of
// u^2+v^2+w^2 over the interior, and calcStats (paris.f90:1116-1267) as one
// pass over the interior cells that keeps the 25 column sums in registers.
//
// The reductions are deterministic: per-block tree sums, then the block
// partials added in block order by one block per column.  The max is
// order-independent, so the time step equals the reference's bit for bit;
// the sums differ from its k,j,i loop order only by rounding.
#include "ctx.cuh"
#include "plic.cuh"

namespace {

constexpr int kNS = PARIS_NSTATS;
constexpr int kThreads = 256;   // kRowBlock

__global__ void __launch_bounds__(kThreads) k_vmax2(const double* __restrict__ u, const double* __restrict__ v,
                                                    const double* __restrict__ w, const Layout L, double* part) {
    __shared__ double sh[32];
    double m = 0.0;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        const long n = lidx(L, i, j, k);
        const double a = u[n] * u[n] + v[n] * v[n] + w[n] * w[n];
        m = fmax(m, a);
    ROWS_END
    m = block_max<kThreads>(m, sh);
    if (linear_tid() == 0) part[blockIdx.x] = m;
}

struct StatsArgs {
    const double *u, *v, *w, *rho, *p, *cvof, *mu;
    const int8_t* flag;
    const double *x, *y, *z;                            // cell centres, index i+ng
    const double *dx, *dxh, *dy, *dyh, *dz, *dzh;       // widths, index i+ng
    double dpdx, dpdy, dpdz, gx, gy, gz, rro;
    double top_layer;                                   // xLength*zLength*(yLength-height4Stats)
    int force, bubble, phase_inv, turb;
    int per[3];
};

// PLIC interface area of a mixed cell (mycs normal + AREA3D,
// paris.f90:1193-1201); kept out of line so the 27-entry block does not
// crowd the accumulators of the main loop.
__device__ __noinline__ double cell_area(const double* __restrict__ c, long n, const Layout L) {
    double st[27], m[3];
#pragma unroll
    for (int kk = 0; kk < 3; kk++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++)
#pragma unroll
            for (int ii = 0; ii < 3; ii++)
                st[ii + 3 * jj + 9 * kk] = c[n + (ii - 1) + (jj - 1) * L.pitch + (kk - 1) * L.plane];
    plic::mycs(st, m);
    if (m[0] != 0.0 || m[1] != 0.0 || m[2] != 0.0) return plic::area3d(m, c[n]);
    return 0.0;
}

// calcStats main loop, paris.f90:1136-1239; s[q-1] is mystats(q)
__global__ void __launch_bounds__(kThreads) k_calc_stats(const StatsArgs a, const Layout L, double* part) {
    __shared__ double sh[32];
    double s[kNS];
#pragma unroll
    for (int q = 0; q < kNS; q++) s[q] = 0.0;
    const long e = 1, nn = L.pitch, t = L.plane;
    const int g = L.ng;
    ROWS_BEGIN(L.n[0], L.n[1], L.n[2])
        const long n = lidx(L, i, j, k);
        const int I = i + g, J = j + g, K = k + g;
        const double vol = a.dx[I] * a.dy[J] * a.dz[K];
        const double un = a.u[n], vn = a.v[n], wn = a.w[n], rn = a.rho[n], cc = a.cvof[n];
        s[1] = s[1] + un * vol;
        if (a.force) {
            if (i < L.n[0] - 1 || a.per[0]) {
                double fx = 0.0 - a.dpdx + (0.5 * (a.rho[n + e] + rn) - a.rro) * a.gx;
                s[2] = s[2] + fx * a.dxh[I] * a.dy[J] * a.dz[K];
            }
            if (j < L.n[1] - 1 || a.per[1]) {
                double fy = 0.0 - a.dpdy + (0.5 * (a.rho[n + nn] + rn) - a.rro) * a.gy;
                s[3] = s[3] + fy * a.dx[I] * a.dyh[J] * a.dz[K];
            }
            if (k < L.n[2] - 1 || a.per[2]) {
                double fz = 0.0 - a.dpdz + (0.5 * (a.rho[n + t] + rn) - a.rro) * a.gz;
                s[4] = s[4] + fz * a.dx[I] * a.dy[J] * a.dzh[K];
            }
        }
        s[5] = s[5] + rn * vol;
        s[6] = s[6] + a.p[n] * vol;
        const double rf = 0.5 * (rn + a.rho[n + e]);
        s[7] = s[7] + rf * un * vol;
        // s[8]: rho_face*uold*vol with uold = 0 under the explicit scheme
        s[9] = s[9] + cc * vol;
        s[10] = s[10] + cc * vol * a.x[I];
        if (a.bubble) s[23] = s[23] + 0.50 * (a.u[n - e] + un) * cc * vol;
        const double a1 = 0.5 * (un + a.u[n + e]), a2 = 0.5 * (vn + a.v[n + nn]), a3 = 0.5 * (wn + a.w[n + t]);
        const double ke = 0.5 * (a1 * a1 + a2 * a2 + a3 * a3);
        s[11] = s[11] + rn * ke * vol * cc;
        s[12] = s[12] + rn * ke * vol * (1.0 - cc);
        if (a.turb) {
            const double b1 = (-un + a.u[n + e]) / a.dx[I], b2 = (-vn + a.v[n + nn]) / a.dy[J];
            s[13] = s[13] + b1 * b1 * vol;
            s[14] = s[14] + b2 * b2 * vol;
        } else {
            s[13] = s[13] + rn * 0.5 * (vn + a.v[n + nn]) * vol * (cc);
            s[14] = s[14] + rn * 0.5 * (vn + a.v[n + nn]) * vol * (1.0 - cc);
        }
        if (cc > 0.0 && cc < 1.0) s[18] = s[18] + cell_area(a.cvof, n, L);
        if (a.phase_inv) {
            s[19] = s[19] + rn * a.gy * a.y[J] * vol * cc;
            s[20] = s[20] + rn * a.gy * a.y[J] * vol * (1.0 - cc);
        }
        const double dyc = a.y[J + 1] - a.y[J - 1], dzc = a.z[K + 1] - a.z[K - 1], dxc = a.x[I + 1] - a.x[I - 1];
        const double d1 = 0.5 * (a.w[n + nn] + a.w[n + nn + t] - a.w[n - nn] - a.w[n - nn + t]) / dyc -
                          0.5 * (a.v[n + t] + a.v[n + nn + t] - a.v[n - t] - a.v[n + nn - t]) / dzc;
        const double d2 = 0.5 * (a.u[n + t] + a.u[n + e + t] - a.u[n - t] - a.u[n + e - t]) / dzc -
                          0.5 * (a.w[n + e] + a.w[n + e + t] - a.w[n - e] - a.w[n - e + t]) / dxc;
        const double d3 = 0.5 * (a.v[n + e] + a.v[n + e + nn] - a.v[n - e] - a.v[n - e + nn]) / dxc -
                          0.5 * (a.u[n + nn] + a.u[n + e + nn] - a.u[n - nn] - a.u[n + e - nn]) / dyc;
        const double ens = 0.5 * (d1 * d1 + d2 * d2 + d3 * d3);
        s[21] = s[21] + ens * vol * cc;
        s[22] = s[22] + ens * vol * (1.0 - cc);
        if (a.flag[n] == 2) s[24] = s[24] + 1.0;
        if (a.phase_inv && a.y[J] > 0.875) s[23] = s[23] + vol * cc / a.top_layer;
        // shear stress on y = 0 and y = Ly (paris.f90:1242-1251)
        if (j == 0) s[0] = s[0] + a.mu[n] * un * a.dx[I] * a.dz[K] / (a.dy[J] / 2.0);
        if (j == L.n[1] - 1) s[0] = s[0] + a.mu[n] * un * a.dx[I] * a.dz[K] / (a.dy[J] / 2.0);
    ROWS_END
#pragma unroll
    for (int q = 0; q < kNS; q++) {
        double b = block_sum<kThreads>(s[q], sh);
        if (linear_tid() == 0) part[(long)q * kRedBlocks + blockIdx.x] = b;
    }
}

// one block per column: the block partials in block order
__global__ void k_stats_finish(const double* __restrict__ part, double* out, int nb) {
    __shared__ double sh[32];
    const int q = blockIdx.x;
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v += part[(long)q * kRedBlocks + b];
    v = block_sum<kThreads>(v, sh);
    if (threadIdx.x == 0) out[q] = v;
}

double min_dx(const paris_ctx* c) {
    double h = c->h_dx[0];
    for (double d : c->h_dx) h = d < h ? d : h;
    return h;
}

int vmax_interior(paris_ctx* c, double* vmax) {
    for (int f : {PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W}) PARIS_CHECK(ctx_alloc_field(c, f));
    PARIS_LAUNCH_N(c, "vmax", c->N, k_vmax2, red_grid(c, k_vmax2, kThreads), kRowBlock, 0, c->fld[PARIS_FIELD_U],
                   c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W], c->L, c->red_part);
    double m2;
    PARIS_CHECK(ctx_reduce_finish(c, 1, &m2, 1));
    *vmax = sqrt(m2);   // sqrt is monotone: max of the roots = root of the max
    return PARIS_OK;
}

}  // namespace

extern "C" int paris_time_step_size(paris_handle_t c, double cfl, double max_dt, double u_inject, double* dt,
                                    double* vmax_out) {
    if (!c || !dt) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    double vmax;
    PARIS_CHECK(vmax_interior(c, &vmax));
    const double vmax_phys = fmax(1e-3, u_inject);
    const double h = min_dx(c);
    const double dtadv = h / (vmax_phys > vmax ? vmax_phys : vmax);
    double mydt = cfl * dtadv;
    *dt = mydt < max_dt ? mydt : max_dt;
    if (vmax_out) *vmax_out = vmax;
    return PARIS_OK;
}

extern "C" int paris_get_cfl_and_check(paris_handle_t c, double dt, double cflmax_allowed, double* cfl) {
    if (!c || !cfl) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    double vmax;
    PARIS_CHECK(vmax_interior(c, &vmax));
    *cfl = vmax * dt / min_dx(c);
    if (*cfl > cflmax_allowed) {
        ctx_set_error(c, "get_cfl_and_check: CFL too large (%g > %g)", *cfl, cflmax_allowed);
        return PARIS_CFL_TOO_LARGE;
    }
    return PARIS_OK;
}

extern "C" int paris_calc_stats(paris_handle_t c, const paris_stats_opts* opts, double* stats) {
    if (!c || !stats) return PARIS_BAD_ARGS;
    paris_stats_opts o{};
    if (opts) o = *opts;
    double rro = 0.0;
    switch (o.buoyancy_case) {
        case 0: rro = 0.0; break;
        case 1: rro = c->d.rho1; break;
        case 2: rro = c->d.rho2; break;
        case 3: rro = o.rho_ave; break;
        default:
            ctx_set_error(c, "volumeForce: invalid buoyancy option %d", o.buoyancy_case);
            return PARIS_BAD_ARGS;
    }
    cudaSetDevice(c->dev);
    for (int f : {PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_RHO, PARIS_FIELD_P, PARIS_FIELD_CVOF,
                  PARIS_FIELD_MU, PARIS_FIELD_VOF_FLAG})
        PARIS_CHECK(ctx_alloc_field(c, f));
    if (!c->stats_part) {
        PARIS_CUDA_TRY(c, cudaMalloc(&c->stats_part, (long)kNS * kRedBlocks * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->stats_out, kNS * sizeof(double)));
    }
    const paris_grid_desc& d = c->d;
    StatsArgs a;
    a.u = c->fld[PARIS_FIELD_U]; a.v = c->fld[PARIS_FIELD_V]; a.w = c->fld[PARIS_FIELD_W];
    a.rho = c->fld[PARIS_FIELD_RHO]; a.p = c->fld[PARIS_FIELD_P]; a.cvof = c->fld[PARIS_FIELD_CVOF];
    a.mu = c->fld[PARIS_FIELD_MU]; a.flag = c->flag;
    a.x = c->xc; a.y = c->yc; a.z = c->zc;
    a.dx = c->dx; a.dxh = c->dxh; a.dy = c->dy; a.dyh = c->dyh; a.dz = c->dz; a.dzh = c->dzh;
    a.dpdx = o.dpdx; a.dpdy = o.dpdy; a.dpdz = o.dpdz; a.gx = o.gx; a.gy = o.gy; a.gz = o.gz; a.rro = rro;
    a.top_layer = d.xlength * d.zlength * (d.ylength - 0.875);
    a.force = o.force_valid != 0;
    a.bubble = (o.test_flags & PARIS_STATS_RISING_BUBBLE) != 0;
    a.phase_inv = (o.test_flags & PARIS_STATS_PHASE_INVERSION) != 0;
    a.turb = (o.test_flags & PARIS_STATS_TURB) != 0;
    for (int q = 0; q < 3; q++) a.per[q] = c->bnd.per[q];
    const unsigned nb = red_grid(c, k_calc_stats, kThreads);
    PARIS_LAUNCH_N(c, "calc_stats", c->N, k_calc_stats, nb, kRowBlock, 0, a, c->L, c->stats_part);
    PARIS_LAUNCH(c, k_stats_finish, kNS, kThreads, 0, c->stats_part, c->stats_out, (int)nb);
    double ms[kNS];
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(ms, c->stats_out, sizeof ms, cudaMemcpyDeviceToHost, c->stream));
    // pressure at entry and exit: p(ng+1, ny/2+ng, nz/2+ng) and p(ng+nx, ny/2+ng, nz/2+ng)
    const int jp = d.ny / 2 - 1, kp = d.nz / 2 - 1;
    const double* P = c->fld[PARIS_FIELD_P];
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(&ms[16], P + lidx(c->L, 0, jp, kp), sizeof(double), cudaMemcpyDeviceToHost,
                                      c->stream));
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(&ms[17], P + lidx(c->L, d.nx - 1, jp, kp), sizeof(double),
                                      cudaMemcpyDeviceToHost, c->stream));
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const double V = d.xlength * d.ylength * d.zlength;
    for (int q = 1; q < 11; q++) ms[q] = ms[q] / V;
    ms[0] = ms[0] / (d.xlength * d.zlength * 2.0);
    if (a.bubble) {
        ms[9] = ms[9] * V;
        ms[10] = ms[10] * V;
        if (ms[9] > 1e-15) {
            ms[10] = ms[10] / ms[9];
            ms[23] = ms[23] / ms[9];
        }
    }
    for (int q = 0; q < kNS; q++) stats[q] = ms[q];
    return PARIS_OK;
}
