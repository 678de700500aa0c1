// prec_f16g.cu -- instantiates the cavity solver for binary16 f - w, fixed-point g storage.
#include "batch.cuh"

namespace cav {
Solver* make_solver_f16g() { return new Impl<Mix16>; }
BatchBase* make_batch_f16g() { return new Batch<Mix16>; }
}  // namespace cav
