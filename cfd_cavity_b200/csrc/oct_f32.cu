// oct_f32.cu -- the octree cavity with FP32 arithmetic and storage.
#include "octree.cuh"

namespace cav {
namespace oct {
Octree* make_octree_f32() { return new OctImpl<float, float>; }
}  // namespace oct
}  // namespace cav
