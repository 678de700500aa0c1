// oct_f16.cu -- the octree cavity with FP32 arithmetic, FP32 storage on the
// coarse level and binary16 (stochastically rounded) storage on L1 / L2,
// the g populations either binary16 or 16-bit fixed point.
#include "octree.cuh"

namespace cav {
namespace oct {
Octree* make_octree_f32_f16() { return new OctImpl<float, Half16SR>; }
Octree* make_octree_f32_f16g() { return new OctImpl<float, Mix16SR>; }
}  // namespace oct
}  // namespace cav
