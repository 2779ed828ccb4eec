// Mixed-precision instantiation: reconstruction, fluxes, sources, metrics, Res, dt, Lc, Lv in
// FP32 (fused multiply-add allowed); U, DU, the LU-SGS diagonal and divide, the limiter test,
// norms and forces in FP64.
#include "runner.cuh"

namespace ocfd {
Runner* make_runner_mixed(const Arena<float>& A, const RunInfo& I) { return make_runner_t<float>(A, I); }
}  // namespace ocfd
