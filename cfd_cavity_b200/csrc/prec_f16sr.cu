// prec_f16sr.cu -- instantiates the cavity solver for binary16 f - w and g, stochastically rounded storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f16sr() { return new Impl<Half16SR>; }
BatchBase* make_batch_f16sr() { return new Batch<Half16SR>; }
}  // namespace cav
