// prec_bf16sr.cu -- instantiates the cavity solver for bfloat16 f - w and g, stochastically rounded storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_bf16sr() { return new Impl<Bf16SR>; }
BatchBase* make_batch_bf16sr() { return new Batch<Bf16SR>; }
}  // namespace cav
