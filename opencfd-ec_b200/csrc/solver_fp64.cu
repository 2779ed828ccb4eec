// FP64 instantiation of the solver kernels (compiled with --fmad=false: each a*b+c is two rounded
// operations, as in the FP64 Fortran reference, so the residual history can be compared with a
// CPU FP64 evaluation to round-off).
#include "runner.cuh"

namespace ocfd {
Runner* make_runner_fp64(const Arena<double>& A, const RunInfo& I) { return make_runner_t<double>(A, I); }
}  // namespace ocfd
