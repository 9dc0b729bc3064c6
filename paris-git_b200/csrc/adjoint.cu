// adjoint.cu -- reverse mode of one pressure projection: SetupPoisson
// (modules.f90:2722-2753) -> NewSolver -> project_velocity
// (paris.f90:898-909).  The reference has no adjoint; this file is its exact
// transpose on the faces the projection updates.
//
// Forward, per face f between cells L = f and R = f+1 of one direction:
//     B_f  = 2 / (rho_L + rho_R)
//     L(B) p = -D u*                 (A7 p - sum A_n p_n = A8 of SetupPoisson)
//     u_f  = u*_f - dt B_f (p_R - p_L) / dxh_f
// with (D v)_c = sum_d (v_c - v_{c-1}) / dx_c, L(B) = -D dt B G and G the
// face gradient.  Given g = dL/du on the updated faces:
//     L lambda = G^T (dt B g)        (L is symmetric: the same multigrid)
//     dL/du*_f = g_f + lambda_L / dx_L - lambda_R / dx_R      (= g + D^T lambda)
//     dL/dB_f  = -dt (p_R - p_L) / dxh_f * dL/du*_f
// The faces are those project_velocity updates: every face of a periodic
// direction (face n-1 joining cell n-1 to cell 0), the interior faces of a
// wall-bounded one.  Ghost entries are images of those faces (periodic) or
// constants of the boundary conditions (wall faces), so the gradients of the
// images are folded into the faces they copy and the other entries of the
// outputs are zero.
#include "ctx.cuh"

namespace {

struct Met {
    const double *dx[3], *dxh[3];
};

__device__ inline long step_of(const Layout& L, int d) { return d == 0 ? 1 : (d == 1 ? L.pitch : L.plane); }

// right-hand side of the transpose solve, compact: G^T (dt B g)
__global__ void k_adj_rhs(const double* __restrict__ gu, const double* __restrict__ gv,
                          const double* __restrict__ gw, const double* __restrict__ rho,
                          double* __restrict__ rhs, const Layout L, const Bnd B, const Met M, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const double* gf[3] = {gu, gv, gw};
    int ix[3] = {i, j, k};
    long n = lidx(L, i, j, k);
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long st = step_of(L, d);
        const int a = ix[d], nd = L.n[d];
        // east face of the cell
        if (a < nd - 1 || B.per[d])
            s -= dt * (2.0 / M.dxh[d][a + g]) * gf[d][n] / (rho[n + st] + rho[n]);
        // west face: face a-1, or face nd-1 across the periodic seam
        if (a > 0 || B.per[d]) {
            int fa = a > 0 ? a - 1 : nd - 1;
            long nf = n + (long)(fa - a) * st;
            s += dt * (2.0 / M.dxh[d][fa + g]) * gf[d][nf] / (rho[nf + st] + rho[nf]);
        }
    }
    rhs[cidx(L.n[0], L.n[1], i, j, k)] = s;
}

// dL/du* and dL/dB on the updated faces (outputs zeroed beforehand)
__global__ void k_adj_grad(const double* __restrict__ gu, const double* __restrict__ gv,
                           const double* __restrict__ gw, const double* __restrict__ lam,
                           const double* __restrict__ p, double* __restrict__ su, double* __restrict__ sv,
                           double* __restrict__ sw, double* __restrict__ bu, double* __restrict__ bv,
                           double* __restrict__ bw, const Layout L, const Bnd B, const Met M, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const double* gf[3] = {gu, gv, gw};
    double* so[3] = {su, sv, sw};
    double* bo[3] = {bu, bv, bw};
    int ix[3] = {i, j, k};
    long n = lidx(L, i, j, k);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long st = step_of(L, d);
        const int a = ix[d], nd = L.n[d];
        if (!(a < nd - 1 || B.per[d])) continue;
        int ar = a < nd - 1 ? a + 1 : 0;                 // east cell, wrapped
        long nr = n + (long)(ar - a) * st;
        double gs = gf[d][n] + lam[n] / M.dx[d][a + g] - lam[nr] / M.dx[d][ar + g];
        so[d][n] = gs;
        // the forward reads p east of the face through the ghost layer
        bo[d][n] = -dt * (p[n + st] - p[n]) / M.dxh[d][a + g] * gs;
    }
}

inline dim3 cblock() { return dim3(128, 2, 1); }
inline dim3 cgrid(const Layout& L) { return dim3(div_up(L.n[0], 128), div_up(L.n[1], 2), L.n[2]); }

}  // namespace

extern "C" int paris_projection_adjoint(paris_handle_t c, double dt, const double* gu, const double* gv,
                                        const double* gw, double* gus, double* gvs, double* gws, double* gbx,
                                        double* gby, double* gbz, const paris_solve_opts* opts) {
    if (!c) return PARIS_BAD_ARGS;
    if (!gu || !gv || !gw) {
        ctx_set_error(c, "paris_projection_adjoint: gu, gv and gw are required");
        return PARIS_BAD_ARGS;
    }
    if (!c->have_matrix || c->A_from_upload || c->setup_dt == 0.0) {
        ctx_set_error(c, "paris_projection_adjoint: the matrix must come from paris_setup_poisson");
        return PARIS_BAD_ARGS;
    }
    if (!(dt > 0.0) || fabs(dt - c->setup_dt) > 1e-12 * c->setup_dt) {
        ctx_set_error(c, "paris_projection_adjoint: dt %g differs from the SetupPoisson dt %g", dt, c->setup_dt);
        return PARIS_BAD_ARGS;
    }
    if (!c->fld[PARIS_FIELD_P] || !c->fld[PARIS_FIELD_RHO]) {
        ctx_set_error(c, "paris_projection_adjoint: P and RHO must hold the forward state");
        return PARIS_BAD_ARGS;
    }
    paris_solve_opts o;
    if (opts) {
        o = *opts;
        if (o.maxit < 0 || (o.norm != 1 && o.norm != 2) || o.mode < PARIS_MG_REFERENCE || o.mode > PARIS_MG_MIXED)
            return PARIS_BAD_ARGS;
        if (o.mode == PARIS_MG_REFERENCE) o.mode = PARIS_MG_FP64;
    } else {
        o = paris_solve_opts{};
        o.rel_tol = 1e-12;
        o.beta = 1.0;
        o.maxit = 100;
        o.norm = 2;
        o.mode = PARIS_MG_FP64;
        o.nu1 = 2;
        o.nu2 = 2;
        o.pcg = 1;
    }
    cudaSetDevice(c->dev);
    const long T = c->L.total;
    if (!c->adj) PARIS_CUDA_TRY(c, cudaMalloc(&c->adj, (10 * T + c->N) * sizeof(double)));
    double* w[3] = {c->adj, c->adj + T, c->adj + 2 * T};
    double* lam = c->adj + 3 * T;
    double* so[3] = {c->adj + 4 * T, c->adj + 5 * T, c->adj + 6 * T};
    double* bo[3] = {c->adj + 7 * T, c->adj + 8 * T, c->adj + 9 * T};
    double* rhs = c->adj + 10 * T;
    const size_t bytes = (size_t)T * sizeof(double);
    const double* gin[3] = {gu, gv, gw};
    // host or device pointers alike (unified addressing)
    for (int d = 0; d < 3; d++)
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(w[d], gin[d], bytes, cudaMemcpyDefault, c->stream));
    PARIS_CUDA_TRY(c, cudaMemsetAsync(lam, 0, bytes, c->stream));
    PARIS_CUDA_TRY(c, cudaMemsetAsync(so[0], 0, 6 * bytes, c->stream));
    Met M{{c->dx, c->dy, c->dz}, {c->dxh, c->dyh, c->dzh}};
    const double* rho = c->fld[PARIS_FIELD_RHO];
    PARIS_LAUNCH_N(c, "adjoint_rhs", c->N, k_adj_rhs, cgrid(c->L), cblock(), 0, w[0], w[1], w[2], rho, rhs, c->L,
                   c->bnd, M, dt);
    paris_solve_result r{};
    int st = mg_fast_solve_into(c, &o, &r, rhs, lam);
    if (st != PARIS_OK && st != PARIS_NOT_CONVERGED) return st;
    PARIS_LAUNCH_N(c, "adjoint_grad", c->N, k_adj_grad, cgrid(c->L), cblock(), 0, w[0], w[1], w[2], lam,
                   c->fld[PARIS_FIELD_P], so[0], so[1], so[2], bo[0], bo[1], bo[2], c->L, c->bnd, M, dt);
    double* outs[6] = {gus, gvs, gws, gbx, gby, gbz};
    double* srcs[6] = {so[0], so[1], so[2], bo[0], bo[1], bo[2]};
    for (int q = 0; q < 6; q++)
        if (outs[q]) PARIS_CUDA_TRY(c, cudaMemcpyAsync(outs[q], srcs[q], bytes, cudaMemcpyDefault, c->stream));
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (st == PARIS_NOT_CONVERGED)
        ctx_set_error(c, "paris_projection_adjoint: transpose solve not converged (rel. residual %g after %d cycles)",
                      r.rel_res, o.maxit);
    return st;
}
