// prec_f16gsr.cu -- instantiates the cavity solver for binary16 f - w and fixed-point g, stochastically rounded storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f16gsr() { return new Impl<Mix16SR>; }
BatchBase* make_batch_f16gsr() { return new Batch<Mix16SR>; }
}  // namespace cav
