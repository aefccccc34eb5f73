// Batched solver placeholder: solves each parameter value in turn.
#include "momed_internal.cuh"

using namespace momed;

int momed_batch_solve_impl(momed_handle* h, const momed_solve_opts* o, const double* u, int32_t nu, double* vals,
                           double* resid, double* vecs, momed_info* info) {
    (void)h; (void)o; (void)u; (void)nu; (void)vals; (void)resid; (void)vecs; (void)info;
    throw Error{MOMED_EINVAL, "batched solver not built yet"};
}
