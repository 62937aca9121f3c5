// adjoint.cu -- differentiable form (placeholder until the adjoint kernels land).
#include "md_state.h"
#include "tinymd_b200.h"

using namespace tmd;

extern "C" {
int md_adjoint_configure(int, int, double, double, double, int) {
    set_error(MD_ERR_UNSUPPORTED, "adjoint form not built");
    return -1;
}
int md_adjoint_forward(double const*, double, double, double*) { return -1; }
int md_adjoint_backward(double*, double*, double*) { return -1; }
int md_adjoint_times(double*, double*) { return -1; }
}
