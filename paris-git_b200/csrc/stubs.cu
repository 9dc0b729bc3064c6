// stubs.cu -- entry points declared in paris_b200.h whose kernels are not in
// this build yet; they fail loudly.
#include "ctx.cuh"

extern "C" int paris_projection_adjoint(paris_handle_t c, double, const double*, const double*, const double*, double*,
                                        double*, double*, double*, double*, double*, const paris_solve_opts*) {
    if (c) ctx_set_error(c, "paris_projection_adjoint: not implemented in this build");
    return PARIS_BAD_ARGS;
}
