// oct_f64.cu -- the octree cavity with FP64 storage on every level (built
// without fused multiply-add: bit-identical to the FP64 oracle).
#include "octree.cuh"

namespace cav {
namespace oct {
Octree* make_octree_f64() { return new OctImpl<double, double>; }
}  // namespace oct
}  // namespace cav
