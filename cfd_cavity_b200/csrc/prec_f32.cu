// prec_f32.cu -- instantiates the cavity solver for float population storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f32() { return new Impl<float>; }
BatchBase* make_batch_f32() { return new Batch<float>; }
}  // namespace cav
