// tp_adjoint.cu -- adjoint (reverse-mode) and one-turn Jacobian entry points.
#include <cuda_runtime.h>

#include "tp_internal.h"

extern "C" {

TP_API int tp_ringpass_adjoint(tp_ctx*, const tp_lattice*, const double*, int64_t, const int64_t*, double, int32_t,
                               double, double, int32_t, const int32_t*, int32_t, const tp_loss_spec*, int32_t,
                               double*, double*, double*, int64_t*, const tp_opts*) {
    return TP_EUNSUPPORTED;
}

TP_API int tp_ringpass_adjoint_batched(tp_ctx*, tp_batch*, const double*, const int64_t*, const int64_t*,
                                       const double*, int32_t, double, double, int32_t, const int32_t*,
                                       const int32_t*, const tp_loss_spec*, int32_t, double*, double*,
                                       const tp_opts*) {
    return TP_EUNSUPPORTED;
}

TP_API int tp_one_turn_jacobian(tp_ctx*, const tp_lattice*, const double*, int64_t, double, int32_t, int32_t,
                                double*, double*, const tp_opts*) {
    return TP_EUNSUPPORTED;
}

}  // extern "C"
