// prec_bf16.cu -- instantiates the cavity solver for bfloat16 f - w and g storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_bf16() { return new Impl<Bf16>; }
BatchBase* make_batch_bf16() { return new Batch<Bf16>; }
}  // namespace cav
