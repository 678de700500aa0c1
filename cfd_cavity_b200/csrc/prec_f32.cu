// prec_f32.cu -- instantiates the cavity solver for float population storage.
#include "solver.cuh"

namespace cav {
Solver* make_solver_f32() { return new Impl<float>; }
}  // namespace cav
