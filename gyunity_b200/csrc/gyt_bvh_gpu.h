// Device construction of the binary BVH (node layout of gyt_bvh_host.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace gyt {

struct GpuBvh {
  float4* nodes = nullptr;   // 4 float4 per node, n_slots nodes (cudaMalloc'd)
  uint32_t* order = nullptr; // leaf order -> triangle id, nt entries (cudaMalloc'd)
  uint32_t n_slots = 0;      // node slots allocated (at most nt)
  uint32_t n_inner = 0;      // inner nodes in the tree
  uint32_t max_depth = 0;    // levels, counted as the host builder counts them
};

// Binned-SAH build on `stream` from device vertices (nv x 3 floats) and
// indices (nt x 3, every index < nv: checked by the caller). The tree is the
// one build_bvh_host(max_leaf) makes: the same split rule, the same float
// arithmetic, the same leaves (as triangle sets) and child boxes; only node
// numbering differs (each leaf's triangles are in ascending id order in
// both). Returns 0, or 2 (CUDA error), 3 (out of memory), 4 (unsupported
// input) with *err set. On success the caller owns out->nodes and
// out->order (cudaFree).
int build_bvh_gpu(cudaStream_t stream, const float* d_vertices, const uint32_t* d_indices, uint32_t nt, GpuBvh* out,
                  std::string* err, int max_leaf = 8);

struct GpuWideBvh {
  uint4* nodes = nullptr;    // 5 uint4 per node (the layout of gyt_bvh_host.h), n_nodes nodes (cudaMalloc'd)
  uint32_t* order = nullptr; // leaf order -> triangle id, nt entries (cudaMalloc'd)
  uint32_t n_nodes = 0;
  uint32_t max_depth = 0;    // wide levels
};

// The 8-wide BVH with quantized child boxes that build_wide_bvh_host makes,
// built on the device: build_bvh_gpu(max_leaf = 3), then the collapse one
// level of wide nodes at a time (one thread per wide node: the greedy
// expansion to eight children by largest area, the octant slot order, the
// margin and the quantization, with the host's float and double operations;
// node and triangle offsets from prefix sums over the level, which gives the
// host's breadth-first numbering). The result equals the host build word for
// word. Returns as build_bvh_gpu; the caller owns out->nodes and out->order.
int build_wide_bvh_gpu(cudaStream_t stream, const float* d_vertices, const uint32_t* d_indices, uint32_t nt,
                       GpuWideBvh* out, std::string* err);

}  // namespace gyt
