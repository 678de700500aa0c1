// prec_f16.cu -- instantiates the cavity solver for __half population storage.
#include "solver.cuh"

namespace cav {
Solver* make_solver_f16() { return new Impl<__half>; }
}  // namespace cav
