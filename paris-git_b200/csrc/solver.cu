// solver.cu -- NewSolver(A,p,maxError,beta,maxit,it,ierr,norm)
// (newsolver.f90:34-57): dispatch to the reference multigrid or to the B200
// multigrid, and the reference's return convention (it = maxit+1 when the
// tolerance was not reached).
#include "ctx.cuh"

extern "C" int paris_new_solver(paris_handle_t c, const paris_solve_opts* o, paris_solve_result* r) {
    if (!c || !o || !r) return PARIS_BAD_ARGS;
    if (!c->have_matrix) {
        ctx_set_error(c, "no matrix: call paris_setup_poisson, paris_setup_test_mg or upload A first");
        return PARIS_BAD_ARGS;
    }
    if (o->maxit < 0 || (o->norm != 1 && o->norm != 2) || o->mode < PARIS_MG_REFERENCE || o->mode > PARIS_MG_MIXED)
        return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    *r = paris_solve_result{};
    if (o->mode == PARIS_MG_REFERENCE) return mg_ref_solve(c, o, r);
    return mg_fast_solve(c, o, r);
}
