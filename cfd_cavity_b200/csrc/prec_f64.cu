// prec_f64.cu -- instantiates the cavity solver for double population storage.
#include "solver.cuh"

namespace cav {
Solver* make_solver_f64() { return new Impl<double>; }
}  // namespace cav
