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

// vertices: nv*3, indices: nt*3. Returns false on invalid input. max_leaf
// bounds the triangles per leaf (at most 8).
bool build_bvh_host(const float* vertices, uint32_t nv, const uint32_t* indices, uint32_t nt, BvhHost* out,
                    int max_leaf = 8);

// 8-wide BVH with quantized child boxes, collapsed from the binary tree.
//
// Node = 5 x uint4 = 80 bytes:
//   [0] origin p (3 x f32), exponents ex, ey, ez (int8 each, scale 2^e) and
//       the inner-child mask in byte 3 of .w
//   [1] child_base (first inner child node), tri_base (first triangle of the
//       node's leaves), meta[0..7] (one byte per child slot)
//   [2] qlo.x[0..7], qhi.x[0..7]   [3] the same for y   [4] the same for z
// Child slot i: inner if bit i of the mask is set, node index child_base +
// popcount(mask & ((1 << i) - 1)); a leaf if meta[i] != 0: (count << 5) |
// offset, 1..3 triangles starting at tri_base + offset; empty otherwise.
// Child box = p + q * 2^e per axis (q in 0..255), rounded outwards.
struct WideBvhHost {
  std::vector<uint32_t> nodes;    // 20 words per node
  std::vector<uint32_t> order;    // leaf order -> triangle id
  uint32_t max_depth = 0;         // wide levels
};

bool build_wide_bvh_host(const float* vertices, uint32_t nv, const uint32_t* indices, uint32_t nt,
                         WideBvhHost* out);

}  // namespace gyt
