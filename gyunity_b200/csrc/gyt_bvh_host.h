// Host construction of the binary BVH traversed by the CUDA kernels.
//
// Layout (one node = 4 x float4 = 64 bytes, both child boxes in the parent so
// a traversal step is one 64-byte fetch):
//   n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   n3 = (child0, child1, 0, 0) as int bits; child >= 0 is an inner node,
//        child < 0 is a leaf ~((first << 3) | (count - 1)) into the
//        leaf-ordered triangle array.
// Child boxes are padded outward by a few ulps so the slab test never culls a
// ray that the watertight triangle test would accept.
//
// Replaces the reference's BVHAccel build (accelerator/BVHAccel.cpp:154-393):
// binned SAH as there (12 buckets, cost 0.125 + ...), here 16 bins per axis
// and up to 8 triangles per leaf.
#pragma once
#include <stdint.h>
#include <vector>

namespace gyt {

struct BvhHost {
  std::vector<float> nodes;       // 16 floats per node
  std::vector<uint32_t> order;    // leaf order -> triangle id
  uint32_t max_depth = 0;
};

// vertices: nv*3, indices: nt*3. Returns false on invalid input.
bool build_bvh_host(const float* vertices, uint32_t nv, const uint32_t* indices, uint32_t nt, BvhHost* out);

}  // namespace gyt
