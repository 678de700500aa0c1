// prec_f64.cu -- instantiates the cavity solver for double population storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f64() { return new Impl<double>; }
BatchBase* make_batch_f64() { return new Batch<double>; }
}  // namespace cav
