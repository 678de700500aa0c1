// prec_f16.cu -- instantiates the cavity solver for binary16 f - w and g storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f16() { return new Impl<Half16>; }
BatchBase* make_batch_f16() { return new Batch<Half16>; }
}  // namespace cav
