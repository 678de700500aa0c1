// prec_bf16.cu -- instantiates the cavity solver for __nv_bfloat16 population storage.
#include "solver.cuh"

namespace cav {
Solver* make_solver_bf16() { return new Impl<__nv_bfloat16>; }
}  // namespace cav
