// Binned-SAH BVH construction on the GPU (replaces BVHAccel's recursive build,
// accelerator/BVHAccel.cpp:154-372), writing the binary node layout of
// gyt_bvh_host.h so the traversal kernels serve both builders.
//
// The tree is the host builder's tree: the same 16-bin SAH, evaluated with
// the same IEEE float operations in the same order (explicit _rn intrinsics,
// no FMA contraction), so every split, leaf and child box comes out the same.
//
// Level-synchronous top-down build over "tasks", contiguous ranges of the
// triangle index array. Per level, for the tasks of more than kSmall triangles:
//   k_bin      every triangle adds itself to its task's 3 x 16 bins (count and
//              box; shared-memory bins for the block's first task, global
//              atomics for the rest)
//   k_split    one thread per task: SAH over the 3 x 15 bin borders, the
//              task's node and both child boxes (unions of bins), child tasks
//   k_flag, an exclusive scan, k_scatter
//              stable partition of every task's range into its left and right
//              parts (deterministic leaf order), with the children's task ids
//              and centroid bounds
// Tasks of at most kSmall triangles are finished by one thread each (k_small)
// with the host builder's recursion, in place, in a node range reserved for
// them (count - 1 slots: enough for any binary tree over count triangles), so
// each such subtree is laid out contiguously in depth-first order.
#include "gyt_bvh_gpu.h"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

namespace gyt {
namespace {

constexpr int kBins = 16;
constexpr int kSmall = 32;
constexpr int kMaxLeaf = 8;
constexpr int kTB = 256;
constexpr int kBinWords = 7;                          // count, lo.xyz, hi.xyz
constexpr int kTaskBinWords = 3 * kBins * kBinWords;  // 336
constexpr uint32_t kOrdMax = 0xffffffffu;             // orderable +inf side
constexpr uint32_t kOrdMin = 0u;

struct Task {
  uint32_t start, count;
  int parent, slot;  // node and child slot that link to this task
  uint32_t depth;    // root 0
  uint32_t nbase;    // first reserved node slot (small tasks)
  float clo[3], chi[3];  // centroid bounds
};

struct Counters {
  uint32_t nodes;      // node slots handed out
  uint32_t next;       // big tasks of the next level
  uint32_t nsmall;     // small tasks so far
  uint32_t max_count;  // largest next-level task
  uint32_t inner;      // inner nodes written
  uint32_t depth;      // levels (host builder's count)
  uint32_t overflow;   // capacity or stack overflow
};

// float <-> uint with the same order, for integer atomic min/max
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Box::area of the host builder: 2 (dx dy + dy dz + dz dx), dx = max(0, hi - lo)
__device__ __forceinline__ float area_rn(const float lo[3], const float hi[3]) {
  float d0 = fmaxf(0.f, __fsub_rn(hi[0], lo[0]));
  float d1 = fmaxf(0.f, __fsub_rn(hi[1], lo[1]));
  float d2 = fmaxf(0.f, __fsub_rn(hi[2], lo[2]));
  return __fmul_rn(2.f, __fadd_rn(__fadd_rn(__fmul_rn(d0, d1), __fmul_rn(d1, d2)), __fmul_rn(d2, d0)));
}
__device__ __forceinline__ float sah_rn(float al, uint32_t l, float ar, uint32_t r) {
  return __fadd_rn(__fmul_rn(al, (float)l), __fmul_rn(ar, (float)r));
}
__device__ __forceinline__ float bin_scale(float lo, float hi) { return __fdiv_rn((float)kBins, __fsub_rn(hi, lo)); }
__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
  return min(kBins - 1, (int)__fmul_rn(__fsub_rn(c, lo), scale));
}
__device__ __forceinline__ float axis(float4 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Child box and link of the binary layout (16 floats per node), padded as the
// host builder pads: e = max|coordinate| * 4e-7 + 1e-30.
__device__ void write_child(float4* nodes, int node, int slot, const float lo0[3], const float hi0[3], int link) {
  float m = 0.f;
  for (int a = 0; a < 3; ++a) m = fmaxf(m, fmaxf(fabsf(lo0[a]), fabsf(hi0[a])));
  float e = __fadd_rn(__fmul_rn(m, 4.0e-7f), 1e-30f);
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = __fsub_rn(lo0[a], e);
    hi[a] = __fadd_rn(hi0[a], e);
  }
  float4* n = nodes + (size_t)node * 4;
  n[slot] = make_float4(lo[0], hi[0], lo[1], hi[1]);
  float* z = reinterpret_cast<float*>(&n[2]);
  z[2 * slot] = lo[2];
  z[2 * slot + 1] = hi[2];
  reinterpret_cast<int*>(&n[3])[slot] = link;
}
__device__ __forceinline__ void set_link(float4* nodes, int node, int slot, int link) {
  reinterpret_cast<int*>(&nodes[(size_t)node * 4 + 3])[slot] = link;
}
__device__ __forceinline__ int leaf_code(uint32_t first, uint32_t count) { return (int)~((first << 3) | (count - 1)); }

__global__ void k_prim_boxes(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t nt,
                             float4* __restrict__ blo, float4* __restrict__ bhi, float4* __restrict__ cen,
                             uint32_t* __restrict__ idx, uint32_t* __restrict__ root) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < nt;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX}, c[3] = {0.f, 0.f, 0.f};
  if (valid) {
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = I[3 * (size_t)t + k];
      for (int a = 0; a < 3; ++a) {
        const float x = V[3 * (size_t)v + a];
        lo[a] = fminf(lo[a], x);
        hi[a] = fmaxf(hi[a], x);
      }
    }
    for (int a = 0; a < 3; ++a) c[a] = __fmul_rn(0.5f, __fadd_rn(lo[a], hi[a]));
    blo[t] = make_float4(lo[0], lo[1], lo[2], 0.f);
    bhi[t] = make_float4(hi[0], hi[1], hi[2], 0.f);
    cen[t] = make_float4(c[0], c[1], c[2], 0.f);
    idx[t] = t;
  }
  // root: centroid bounds (0..5) and box (6..11), one atomic per warp and word
  for (int a = 0; a < 3; ++a) {
    const uint32_t v0 = __reduce_min_sync(0xffffffffu, valid ? f2o(c[a]) : kOrdMax);
    const uint32_t v1 = __reduce_max_sync(0xffffffffu, valid ? f2o(c[a]) : kOrdMin);
    const uint32_t v2 = __reduce_min_sync(0xffffffffu, valid ? f2o(lo[a]) : kOrdMax);
    const uint32_t v3 = __reduce_max_sync(0xffffffffu, valid ? f2o(hi[a]) : kOrdMin);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&root[a], v0);
      atomicMax(&root[3 + a], v1);
      atomicMin(&root[6 + a], v2);
      atomicMax(&root[9 + a], v3);
    }
  }
}

__global__ void k_bins_init(uint32_t* __restrict__ bins, uint32_t words) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= words) return;
  const uint32_t f = i % kBinWords;
  bins[i] = f == 0 ? 0u : (f <= 3 ? kOrdMax : kOrdMin);
}

__device__ __forceinline__ void bin_add(uint32_t* w, const float4& lo, const float4& hi) {
  atomicAdd(w, 1u);
  atomicMin(w + 1, f2o(lo.x));
  atomicMin(w + 2, f2o(lo.y));
  atomicMin(w + 3, f2o(lo.z));
  atomicMax(w + 4, f2o(hi.x));
  atomicMax(w + 5, f2o(hi.y));
  atomicMax(w + 6, f2o(hi.z));
}

__global__ void __launch_bounds__(kTB) k_bin(uint32_t n, const uint32_t* __restrict__ idx,
                                             const int* __restrict__ ptask, const Task* __restrict__ tasks,
                                             const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                             const float4* __restrict__ cen, uint32_t* __restrict__ bins) {
  __shared__ uint32_t sb[kTaskBinWords];
  __shared__ int stk;
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  const int tk = pos < n ? ptask[pos] : -1;
  if (threadIdx.x == 0) stk = tk;
  for (int i = threadIdx.x; i < kTaskBinWords; i += blockDim.x) {
    const int f = i % kBinWords;
    sb[i] = f == 0 ? 0u : (f <= 3 ? kOrdMax : kOrdMin);
  }
  __syncthreads();
  const int tk0 = stk;
  if (tk >= 0) {
    const Task& T = tasks[tk];
    const uint32_t p = idx[pos];
    const float4 c = cen[p], lo = blo[p], hi = bhi[p];
    uint32_t* base = tk == tk0 ? sb : bins + (size_t)tk * kTaskBinWords;
    for (int a = 0; a < 3; ++a) {
      // an axis without centroid extent is not split on; its bin 0 still
      // collects the task's box
      const float clo = T.clo[a], chi = T.chi[a];
      const int b = __fsub_rn(chi, clo) > 0.f ? bin_of(axis(c, a), clo, bin_scale(clo, chi)) : 0;
      bin_add(base + (a * kBins + b) * kBinWords, lo, hi);
    }
  }
  __syncthreads();
  if (tk0 >= 0) {
    uint32_t* g = bins + (size_t)tk0 * kTaskBinWords;
    for (int i = threadIdx.x; i < kTaskBinWords; i += blockDim.x) {
      const int f = i % kBinWords;
      if (sb[i - f] == 0) continue;  // empty bin
      const uint32_t v = sb[i];
      if (f == 0) atomicAdd(&g[i], v);
      else if (f <= 3) atomicMin(&g[i], v);
      else atomicMax(&g[i], v);
    }
  }
}

// Exact SAH choice over one task's bins, in the host builder's order: axes
// 0..2, borders from the right, strict improvement.
struct Split {
  float cost;
  int axis, border;
  uint32_t nl, nr;
};

__device__ void choose_split(const uint32_t* __restrict__ B, const float clo[3], const float chi[3], Split* s) {
  s->cost = FLT_MAX;
  s->axis = -1;
  s->border = -1;
  s->nl = s->nr = 0;
  for (int a = 0; a < 3; ++a) {
    if (!(__fsub_rn(chi[a], clo[a]) > 0.f)) continue;
    float al[kBins];
    uint32_t lc[kBins];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    uint32_t c = 0;
    for (int b = 0; b < kBins; ++b) {
      const uint32_t* w = B + (a * kBins + b) * kBinWords;
      if (w[0]) {
        c += w[0];
        for (int k = 0; k < 3; ++k) {
          lo[k] = fminf(lo[k], o2f(w[1 + k]));
          hi[k] = fmaxf(hi[k], o2f(w[4 + k]));
        }
      }
      al[b] = area_rn(lo, hi);
      lc[b] = c;
    }
    float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    uint32_t rc = 0;
    for (int b = kBins - 1; b > 0; --b) {
      const uint32_t* w = B + (a * kBins + b) * kBinWords;
      if (w[0]) {
        rc += w[0];
        for (int k = 0; k < 3; ++k) {
          rlo[k] = fminf(rlo[k], o2f(w[1 + k]));
          rhi[k] = fmaxf(rhi[k], o2f(w[4 + k]));
        }
      }
      const uint32_t l = lc[b - 1];
      if (l == 0 || rc == 0) continue;
      const float cost = sah_rn(al[b - 1], l, area_rn(rlo, rhi), rc);
      if (cost < s->cost) {
        s->cost = cost;
        s->axis = a;
        s->border = b;
        s->nl = l;
        s->nr = rc;
      }
    }
  }
}

// union of the bins [b0, b1) of one axis
__device__ void bins_box(const uint32_t* __restrict__ B, int a, int b0, int b1, float lo[3], float hi[3]) {
  for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
  for (int b = b0; b < b1; ++b) {
    const uint32_t* w = B + (a * kBins + b) * kBinWords;
    if (!w[0]) continue;
    for (int k = 0; k < 3; ++k) {
      lo[k] = fminf(lo[k], o2f(w[1 + k]));
      hi[k] = fmaxf(hi[k], o2f(w[4 + k]));
    }
  }
}

__global__ void k_split(uint32_t ntasks, const Task* __restrict__ tasks, const uint32_t* __restrict__ bins,
                        float4* __restrict__ nodes, uint32_t node_cap, Task* __restrict__ next, uint32_t next_cap,
                        uint32_t* __restrict__ next_cb, Task* __restrict__ small, uint32_t small_cap,
                        int* __restrict__ split, int* __restrict__ child, Counters* __restrict__ cnt) {
  const uint32_t tk = blockIdx.x * blockDim.x + threadIdx.x;
  if (tk >= ntasks) return;
  const Task T = tasks[tk];
  const uint32_t* B = bins + (size_t)tk * kTaskBinWords;
  Split s;
  choose_split(B, T.clo, T.chi, &s);
  int node = 0;
  if (T.parent >= 0) {
    const uint32_t id = atomicAdd(&cnt->nodes, 1u);
    if (id >= node_cap) {  // cannot happen: a tree over nt triangles has at most nt - 1 inner nodes
      atomicOr(&cnt->overflow, 8u);
      split[2 * tk] = -1;
      child[2 * tk] = child[2 * tk + 1] = -1;
      return;
    }
    node = (int)id;
    set_link(nodes, T.parent, T.slot, node);
  }
  atomicAdd(&cnt->inner, 1u);
  float lo[2][3], hi[2][3];
  uint32_t ns[2];
  if (s.axis >= 0) {
    bins_box(B, s.axis, 0, s.border, lo[0], hi[0]);
    bins_box(B, s.axis, s.border, kBins, lo[1], hi[1]);
    ns[0] = s.nl;
    ns[1] = s.nr;
  } else {
    // every centroid is the same point (no axis was binned): halves of the
    // range by position, both with the box of the whole task
    bins_box(B, 0, 0, kBins, lo[0], hi[0]);
    for (int k = 0; k < 3; ++k) { lo[1][k] = lo[0][k]; hi[1][k] = hi[0][k]; }
    ns[0] = T.count / 2;
    ns[1] = T.count - ns[0];
  }
  split[2 * tk] = s.axis;
  split[2 * tk + 1] = s.border;
  for (int side = 0; side < 2; ++side) {
    write_child(nodes, node, side, lo[side], hi[side], 0);
    Task c;
    c.start = side == 0 ? T.start : T.start + ns[0];
    c.count = ns[side];
    c.parent = node;
    c.slot = side;
    c.depth = T.depth + 1;
    c.nbase = 0;
    for (int k = 0; k < 3; ++k) { c.clo[k] = 0.f; c.chi[k] = 0.f; }
    if (c.count <= (uint32_t)kSmall) {
      const uint32_t id = atomicAdd(&cnt->nsmall, 1u);
      c.nbase = atomicAdd(&cnt->nodes, c.count - 1);
      if (id < small_cap && c.nbase + c.count - 1 <= node_cap) small[id] = c;
      else atomicOr(&cnt->overflow, 1u);
      child[2 * tk + side] = -1;
    } else {
      const uint32_t id = atomicAdd(&cnt->next, 1u);
      if (id < next_cap) {
        next[id] = c;
        uint32_t* cb = next_cb + 6 * (size_t)id;
        cb[0] = cb[1] = cb[2] = kOrdMax;
        cb[3] = cb[4] = cb[5] = kOrdMin;
        child[2 * tk + side] = (int)id;
        atomicMax(&cnt->max_count, c.count);
      } else {
        atomicOr(&cnt->overflow, 2u);
        child[2 * tk + side] = -1;
      }
    }
  }
}

// flag[pos] = 1 for the left part of a split task; flag[n] = 0 (scan total)
__global__ void k_flag(uint32_t n, const uint32_t* __restrict__ idx, const int* __restrict__ ptask,
                       const Task* __restrict__ tasks, const float4* __restrict__ cen, const int* __restrict__ split,
                       uint32_t* __restrict__ flag) {
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos > n) return;
  uint32_t f = 0;
  if (pos < n) {
    const int tk = ptask[pos];
    if (tk >= 0) {
      const Task& T = tasks[tk];
      const int ax = split[2 * tk];
      if (ax >= 0) {
        const float lo = T.clo[ax], hi = T.chi[ax];
        f = bin_of(axis(cen[idx[pos]], ax), lo, bin_scale(lo, hi)) < split[2 * tk + 1] ? 1u : 0u;
      } else {
        f = (pos - T.start) < T.count / 2 ? 1u : 0u;
      }
    }
  }
  flag[pos] = f;
}

// Stable partition by the scan of the flags, with the next level's task id
// per position and the big children's centroid bounds (warp-aggregated).
__global__ void __launch_bounds__(kTB) k_scatter(uint32_t n, const uint32_t* __restrict__ idx_in,
                                                 uint32_t* __restrict__ idx_out, const int* __restrict__ ptask_in,
                                                 int* __restrict__ ptask_out, const Task* __restrict__ tasks,
                                                 const uint32_t* __restrict__ flag, const uint32_t* __restrict__ excl,
                                                 const int* __restrict__ child, const float4* __restrict__ cen,
                                                 uint32_t* __restrict__ next_cb) {
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  int c = -1;
  float4 cc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (pos < n) {
    const int tk = ptask_in[pos];
    const uint32_t p = idx_in[pos];
    if (tk < 0) {
      idx_out[pos] = p;
      ptask_out[pos] = -1;
    } else {
      const Task& T = tasks[tk];
      const uint32_t base = excl[T.start];
      const uint32_t lrank = excl[pos] - base;
      const uint32_t nl = excl[T.start + T.count] - base;
      const bool left = flag[pos] != 0;
      const uint32_t dst = left ? T.start + lrank : T.start + nl + (pos - T.start - lrank);
      c = child[2 * tk + (left ? 0 : 1)];
      idx_out[dst] = p;
      ptask_out[dst] = c;
      if (c >= 0) cc = cen[p];
    }
  }
  // one set of atomics per distinct child in the warp (at most 4: a warp
  // spans at most two tasks of more than 32 triangles)
  bool pending = c >= 0;
  const int lane = (int)(threadIdx.x & 31);
  while (__any_sync(0xffffffffu, pending)) {
    const unsigned m = __ballot_sync(0xffffffffu, pending);
    const int leader = __ffs(m) - 1;
    const int cl = __shfl_sync(0xffffffffu, c, leader);
    const bool mine = pending && c == cl;
    uint32_t v[6];
    v[0] = __reduce_min_sync(0xffffffffu, mine ? f2o(cc.x) : kOrdMax);
    v[1] = __reduce_min_sync(0xffffffffu, mine ? f2o(cc.y) : kOrdMax);
    v[2] = __reduce_min_sync(0xffffffffu, mine ? f2o(cc.z) : kOrdMax);
    v[3] = __reduce_max_sync(0xffffffffu, mine ? f2o(cc.x) : kOrdMin);
    v[4] = __reduce_max_sync(0xffffffffu, mine ? f2o(cc.y) : kOrdMin);
    v[5] = __reduce_max_sync(0xffffffffu, mine ? f2o(cc.z) : kOrdMin);
    if (lane == leader) {
      uint32_t* cb = next_cb + 6 * (size_t)cl;
      for (int k = 0; k < 3; ++k) {
        atomicMin(&cb[k], v[k]);
        atomicMax(&cb[3 + k], v[3 + k]);
      }
    }
    if (mine) pending = false;
  }
}

__global__ void k_cb_final(uint32_t ntasks, Task* __restrict__ tasks, const uint32_t* __restrict__ next_cb) {
  const uint32_t tk = blockIdx.x * blockDim.x + threadIdx.x;
  if (tk >= ntasks) return;
  const uint32_t* cb = next_cb + 6 * (size_t)tk;
  for (int k = 0; k < 3; ++k) {
    tasks[tk].clo[k] = o2f(cb[k]);
    tasks[tk].chi[k] = o2f(cb[3 + k]);
  }
}

// A leaf's triangles in ascending id order (the host builder's order too), so
// both builders break equal-distance ties between triangles the same way.
__device__ void leaf_sort(uint32_t* __restrict__ idx, uint32_t start, uint32_t count) {
  for (uint32_t a = start + 1; a < start + count; ++a) {
    const uint32_t v = idx[a];
    uint32_t b = a;
    while (b > start && idx[b - 1] > v) {
      idx[b] = idx[b - 1];
      --b;
    }
    idx[b] = v;
  }
}

// One thread per small task: the host builder's recursion on the task's
// range (leaf at <= 2 triangles, or at <= max_leaf when no split beats the
// leaf cost), depth-first, nodes from the task's reserved range.
__global__ void k_small(uint32_t nsmall, const Task* __restrict__ small, uint32_t* __restrict__ idx,
                        const float4* __restrict__ blo, const float4* __restrict__ bhi,
                        const float4* __restrict__ cen, float4* __restrict__ nodes, Counters* __restrict__ cnt,
                        uint32_t max_leaf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsmall) return;
  struct Job {
    uint32_t start, count;
    int parent, slot;
    uint32_t depth;
  };
  constexpr int kStack = kSmall + 2;
  Job stack[kStack];
  int sp = 0;
  const Task T = small[i];
  uint32_t nnext = T.nbase;
  const uint32_t nend = T.nbase + (T.count > 0 ? T.count - 1 : 0);
  stack[sp++] = Job{T.start, T.count, T.parent, T.slot, T.depth};
  uint32_t maxd = 0, inner = 0;
  while (sp) {
    const Job j = stack[--sp];
    maxd = max(maxd, j.depth + 1);
    if (j.count <= min(2u, max_leaf)) {
      leaf_sort(idx, j.start, j.count);
      set_link(nodes, j.parent, j.slot, leaf_code(j.start, j.count));
      continue;
    }
    float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = j.start; k < j.start + j.count; ++k) {
      const uint32_t p = idx[k];
      const float4 l = blo[p], h = bhi[p], c = cen[p];
      nlo[0] = fminf(nlo[0], l.x); nlo[1] = fminf(nlo[1], l.y); nlo[2] = fminf(nlo[2], l.z);
      nhi[0] = fmaxf(nhi[0], h.x); nhi[1] = fmaxf(nhi[1], h.y); nhi[2] = fmaxf(nhi[2], h.z);
      clo[0] = fminf(clo[0], c.x); clo[1] = fminf(clo[1], c.y); clo[2] = fminf(clo[2], c.z);
      chi[0] = fmaxf(chi[0], c.x); chi[1] = fmaxf(chi[1], c.y); chi[2] = fmaxf(chi[2], c.z);
    }
    float best = FLT_MAX;
    int bax = -1, bsp = -1;
    for (int a = 0; a < 3; ++a) {
      if (!(__fsub_rn(chi[a], clo[a]) > 0.f)) continue;
      const float scale = bin_scale(clo[a], chi[a]);
      uint32_t bc[kBins];
      float bl[kBins][3], bh[kBins][3];
      for (int b = 0; b < kBins; ++b) {
        bc[b] = 0;
        for (int k = 0; k < 3; ++k) { bl[b][k] = FLT_MAX; bh[b][k] = -FLT_MAX; }
      }
      for (uint32_t k = j.start; k < j.start + j.count; ++k) {
        const uint32_t p = idx[k];
        const float4 l = blo[p], h = bhi[p];
        const int b = bin_of(axis(cen[p], a), clo[a], scale);
        bc[b]++;
        bl[b][0] = fminf(bl[b][0], l.x); bl[b][1] = fminf(bl[b][1], l.y); bl[b][2] = fminf(bl[b][2], l.z);
        bh[b][0] = fmaxf(bh[b][0], h.x); bh[b][1] = fmaxf(bh[b][1], h.y); bh[b][2] = fmaxf(bh[b][2], h.z);
      }
      float al[kBins];
      uint32_t lc[kBins];
      float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      uint32_t c = 0;
      for (int b = 0; b < kBins; ++b) {
        c += bc[b];
        for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], bl[b][k]); hi[k] = fmaxf(hi[k], bh[b][k]); }
        al[b] = area_rn(lo, hi);
        lc[b] = c;
      }
      float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      uint32_t rc = 0;
      for (int b = kBins - 1; b > 0; --b) {
        rc += bc[b];
        for (int k = 0; k < 3; ++k) { rlo[k] = fminf(rlo[k], bl[b][k]); rhi[k] = fmaxf(rhi[k], bh[b][k]); }
        const uint32_t l = lc[b - 1];
        if (l == 0 || rc == 0) continue;
        const float cost = sah_rn(al[b - 1], l, area_rn(rlo, rhi), rc);
        if (cost < best) { best = cost; bax = a; bsp = b; }
      }
    }
    const float an = area_rn(nlo, nhi);
    if (j.count <= max_leaf && (bax < 0 || __fadd_rn(best, an) >= __fmul_rn(an, (float)j.count))) {
      leaf_sort(idx, j.start, j.count);
      set_link(nodes, j.parent, j.slot, leaf_code(j.start, j.count));
      continue;
    }
    uint32_t mid;
    if (bax < 0) {
      mid = j.start + j.count / 2;
    } else {
      const float scale = bin_scale(clo[bax], chi[bax]);
      uint32_t l = j.start, r = j.start + j.count;
      while (l < r) {
        if (bin_of(axis(cen[idx[l]], bax), clo[bax], scale) < bsp) {
          ++l;
        } else {
          --r;
          const uint32_t t = idx[l];
          idx[l] = idx[r];
          idx[r] = t;
        }
      }
      mid = l;
      if (mid == j.start || mid == j.start + j.count) mid = j.start + j.count / 2;
    }
    if (nnext >= nend || sp + 2 > kStack) {
      atomicOr(&cnt->overflow, 4u);
      return;
    }
    const int node = (int)nnext++;
    ++inner;
    set_link(nodes, j.parent, j.slot, node);
    for (int side = 0; side < 2; ++side) {
      const uint32_t s0 = side == 0 ? j.start : mid, s1 = side == 0 ? mid : j.start + j.count;
      float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (uint32_t k = s0; k < s1; ++k) {
        const uint32_t p = idx[k];
        const float4 l = blo[p], h = bhi[p];
        lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
        hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
      }
      write_child(nodes, node, side, lo, hi, 0);
    }
    // right pushed first: the left subtree is laid out first
    stack[sp++] = Job{mid, j.start + j.count - mid, node, 1, j.depth + 1};
    stack[sp++] = Job{j.start, mid - j.start, node, 0, j.depth + 1};
  }
  atomicAdd(&cnt->inner, inner);
  atomicMax(&cnt->depth, maxd);
}

float o2f_host(uint32_t u) {
  const uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  std::memcpy(&f, &v, 4);
  return f;
}

inline uint32_t blocks(uint64_t n, uint32_t tb) { return (uint32_t)((n + tb - 1) / tb); }

// device allocations freed together unless released
struct Bufs {
  std::vector<void*> v;
  ~Bufs() {
    for (void* p : v) cudaFree(p);
  }
  template <class T>
  cudaError_t get(T** p, size_t count) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) v.push_back(*p);
    return e;
  }
  void release(void* p) { v.erase(std::find(v.begin(), v.end(), p)); }
};

}  // namespace

#define GYT_BCK(call)                                                               \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      *err = std::string("build_bvh_gpu: ") + #call + ": " + cudaGetErrorString(e_); \
      return e_ == cudaErrorMemoryAllocation ? 3 : 2;                               \
    }                                                                               \
  } while (0)

int build_bvh_gpu(cudaStream_t st, const float* dV, const uint32_t* dI, uint32_t nt, GpuBvh* out, std::string* err,
                  int max_leaf_in) {
  *out = GpuBvh{};
  if (nt == 0) return 0;
  const uint32_t max_leaf = (uint32_t)std::min(kMaxLeaf, std::max(1, max_leaf_in));
  if ((uint64_t)nt >= (1ull << 28)) {
    *err = "build_bvh_gpu: more than 2^28 triangles";
    return 4;
  }
  Bufs B;  // temporaries, freed on every return; the outputs are released from it
  const uint32_t next_cap = nt / (kSmall + 1) + 2;  // disjoint tasks of more than kSmall triangles
  uint32_t small_cap = std::min<uint32_t>(nt, 2 * next_cap + 64);
  float4 *blo, *bhi, *cen, *nodes;
  uint32_t *idx0, *idx1, *root, *bins, *flag, *excl, *next_cb;
  int *pt0, *pt1, *split, *child;
  Task *ta, *tb, *small;
  Counters* cnt;
  GYT_BCK(B.get(&blo, nt));
  GYT_BCK(B.get(&bhi, nt));
  GYT_BCK(B.get(&cen, nt));
  GYT_BCK(B.get(&idx0, nt));
  GYT_BCK(B.get(&idx1, nt));
  GYT_BCK(B.get(&pt0, nt));
  GYT_BCK(B.get(&pt1, nt));
  GYT_BCK(B.get(&flag, (size_t)nt + 1));
  GYT_BCK(B.get(&excl, (size_t)nt + 1));
  GYT_BCK(B.get(&root, 12));
  GYT_BCK(B.get(&ta, next_cap));
  GYT_BCK(B.get(&tb, next_cap));
  GYT_BCK(B.get(&next_cb, 6 * (size_t)next_cap));
  GYT_BCK(B.get(&split, 2 * (size_t)next_cap));
  GYT_BCK(B.get(&child, 2 * (size_t)next_cap));
  GYT_BCK(B.get(&bins, (size_t)next_cap * kTaskBinWords));
  GYT_BCK(B.get(&small, small_cap));
  GYT_BCK(B.get(&cnt, 1));
  GYT_BCK(B.get(&nodes, 4 * (size_t)nt));
  size_t scan_bytes = 0;
  GYT_BCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flag, excl, (int)nt + 1, st));
  uint8_t* scan_tmp;
  GYT_BCK(B.get(&scan_tmp, scan_bytes));

  uint32_t rinit[12];
  for (int a = 0; a < 3; ++a) {
    rinit[a] = kOrdMax;
    rinit[3 + a] = kOrdMin;
    rinit[6 + a] = kOrdMax;
    rinit[9 + a] = kOrdMin;
  }
  GYT_BCK(cudaMemcpyAsync(root, rinit, sizeof(rinit), cudaMemcpyHostToDevice, st));
  k_prim_boxes<<<blocks(nt, kTB), kTB, 0, st>>>(dV, dI, nt, blo, bhi, cen, idx0, root);
  GYT_BCK(cudaGetLastError());
  uint32_t rh[12];
  GYT_BCK(cudaMemcpyAsync(rh, root, sizeof(rh), cudaMemcpyDeviceToHost, st));
  GYT_BCK(cudaStreamSynchronize(st));

  if (nt <= max_leaf) {
    // one leaf under the root and an inverted (never hit) box in the other
    // slot, as the host builder makes it
    float lo[3], hi[3], m = 0.f;
    for (int a = 0; a < 3; ++a) {
      lo[a] = o2f_host(rh[6 + a]);
      hi[a] = o2f_host(rh[9 + a]);
      m = std::max(m, std::max(std::fabs(lo[a]), std::fabs(hi[a])));
    }
    const float e = m * 4.0e-7f + 1e-30f;
    float n[16] = {lo[0] - e, hi[0] + e, lo[1] - e, hi[1] + e, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX,
                   lo[2] - e, hi[2] + e, FLT_MAX, -FLT_MAX, 0.f, 0.f, 0.f, 0.f};
    const int code = (int)~(nt - 1);
    std::memcpy(&n[12], &code, 4);
    std::memcpy(&n[13], &code, 4);
    GYT_BCK(cudaMemcpyAsync(nodes, n, sizeof(n), cudaMemcpyHostToDevice, st));
    GYT_BCK(cudaStreamSynchronize(st));
    B.release(nodes);
    B.release(idx0);
    out->nodes = nodes;
    out->order = idx0;
    out->n_slots = 1;
    out->n_inner = 1;
    out->max_depth = 1;
    return 0;
  }

  Task rt{};
  rt.start = 0;
  rt.count = nt;
  rt.parent = -1;
  rt.slot = 0;
  rt.depth = 0;
  for (int a = 0; a < 3; ++a) {
    rt.clo[a] = o2f_host(rh[a]);
    rt.chi[a] = o2f_host(rh[3 + a]);
  }
  GYT_BCK(cudaMemcpyAsync(ta, &rt, sizeof(Task), cudaMemcpyHostToDevice, st));
  Counters c0{};
  c0.nodes = 1;  // node 0 is the root
  GYT_BCK(cudaMemcpyAsync(cnt, &c0, sizeof(c0), cudaMemcpyHostToDevice, st));
  GYT_BCK(cudaMemsetAsync(pt0, 0, nt * sizeof(int), st));
  uint32_t ntasks = 1, levels = 0, nsmall = 0;
  uint32_t *idx_cur = idx0, *idx_alt = idx1;
  int *pt_cur = pt0, *pt_alt = pt1;
  while (ntasks > 0) {
    if (++levels > 64) {
      *err = "build_bvh_gpu: more than 64 levels of large tasks";
      return 4;
    }
    if (nsmall + 2 * ntasks > small_cap) {
      const uint32_t cap = std::min<uint32_t>(nt, std::max(2 * small_cap, nsmall + 2 * ntasks));
      Task* grown;
      GYT_BCK(B.get(&grown, cap));
      GYT_BCK(cudaMemcpyAsync(grown, small, (size_t)nsmall * sizeof(Task), cudaMemcpyDeviceToDevice, st));
      GYT_BCK(cudaStreamSynchronize(st));
      B.release(small);
      cudaFree(small);
      small = grown;
      small_cap = cap;
    }
    const uint32_t words = ntasks * kTaskBinWords;
    k_bins_init<<<blocks(words, kTB), kTB, 0, st>>>(bins, words);
    k_bin<<<blocks(nt, kTB), kTB, 0, st>>>(nt, idx_cur, pt_cur, ta, blo, bhi, cen, bins);
    GYT_BCK(cudaMemsetAsync(&cnt->next, 0, sizeof(uint32_t), st));
    GYT_BCK(cudaMemsetAsync(&cnt->max_count, 0, sizeof(uint32_t), st));
    k_split<<<blocks(ntasks, 64), 64, 0, st>>>(ntasks, ta, bins, nodes, nt, tb, next_cap, next_cb, small,
                                                small_cap, split, child, cnt);
    k_flag<<<blocks((uint64_t)nt + 1, kTB), kTB, 0, st>>>(nt, idx_cur, pt_cur, ta, cen, split, flag);
    GYT_BCK(cudaGetLastError());
    GYT_BCK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flag, excl, (int)nt + 1, st));
    k_scatter<<<blocks(nt, kTB), kTB, 0, st>>>(nt, idx_cur, idx_alt, pt_cur, pt_alt, ta, flag, excl, child, cen,
                                               next_cb);
    GYT_BCK(cudaGetLastError());
    Counters ch;
    GYT_BCK(cudaMemcpyAsync(&ch, cnt, sizeof(ch), cudaMemcpyDeviceToHost, st));
    GYT_BCK(cudaStreamSynchronize(st));
    if (ch.overflow) {
      *err = "build_bvh_gpu: task capacity exceeded";
      return 4;
    }
    std::swap(idx_cur, idx_alt);
    std::swap(pt_cur, pt_alt);
    std::swap(ta, tb);
    ntasks = ch.next;
    nsmall = ch.nsmall;
    if (ntasks) k_cb_final<<<blocks(ntasks, kTB), kTB, 0, st>>>(ntasks, ta, next_cb);
  }
  if (nsmall)
    k_small<<<blocks(nsmall, 64), 64, 0, st>>>(nsmall, small, idx_cur, blo, bhi, cen, nodes, cnt, max_leaf);
  GYT_BCK(cudaGetLastError());
  Counters ch;
  GYT_BCK(cudaMemcpyAsync(&ch, cnt, sizeof(ch), cudaMemcpyDeviceToHost, st));
  GYT_BCK(cudaStreamSynchronize(st));
  if (ch.overflow || ch.nodes > nt) {
    *err = "build_bvh_gpu: node range or stack overflow";
    return 4;
  }
  B.release(nodes);
  B.release(idx_cur);
  out->nodes = nodes;
  out->order = idx_cur;
  out->n_slots = ch.nodes;
  out->n_inner = ch.inner;
  out->max_depth = ch.depth;
  return 0;
}


// ------------------------------------------------ 8-wide collapse ---
namespace {

// A child of a binary node: its box (the padded box its parent stores) and
// either the inner node it is or the leaf range it holds.
struct WElem {
  float lo[3], hi[3];
  int node;  // binary inner node, or -1 for a leaf (or an empty slot)
  uint32_t first, count;
};

__device__ WElem welem_child(const float4* __restrict__ nodes, int node, int slot) {
  const float4* n = nodes + (size_t)node * 4;
  const float4 a = n[slot], z = n[2];
  const int4 l = *reinterpret_cast<const int4*>(n + 3);
  WElem e;
  e.lo[0] = a.x; e.hi[0] = a.y; e.lo[1] = a.z; e.hi[1] = a.w;
  e.lo[2] = slot == 0 ? z.x : z.z;
  e.hi[2] = slot == 0 ? z.y : z.w;
  const int c = slot == 0 ? l.x : l.y;
  if (c >= 0) {
    e.node = c;
    e.first = e.count = 0;
  } else {
    const uint32_t code = ~(uint32_t)c;
    e.node = -1;
    e.first = code >> 3;
    e.count = (code & 7u) + 1u;
  }
  return e;
}

__device__ __forceinline__ void welem_empty(WElem& e) {
  for (int a = 0; a < 3; ++a) {
    e.lo[a] = FLT_MAX;
    e.hi[a] = -FLT_MAX;
  }
  e.node = -1;
  e.first = e.count = 0;
}

// One wide node from its seed (the binary node whose two children it starts
// from), as build_wide_bvh_host makes it: ch receives the eight child slots
// in slot order, boxes widened by the node's margin; words the node's 20
// words with child_base and tri_base still to fill. Returns the number of
// inner children; *ntris the triangles of its leaves. root: the binary root,
// whose second child is dropped when it is the inverted box of a one-leaf
// tree. Float and double operations as the host's (no contraction).
__device__ uint32_t wide_node(const float4* __restrict__ bin, int seed, bool root, WElem ch[8], uint32_t words[20],
                              uint32_t* ntris, bool* bad) {
  // the greedy expansion: the inner child of largest surface area is replaced
  // by its two children until there are eight
  int n = 2;
  ch[0] = welem_child(bin, seed, 0);
  ch[1] = welem_child(bin, seed, 1);
  if (root && ch[1].node < 0 && ch[1].count > 0 && !(ch[1].lo[0] <= ch[1].hi[0])) n = 1;
  while (n < 8) {
    int best = -1;
    float area = -1.f;
    for (int k = 0; k < n; ++k)
      if (ch[k].node >= 0) {
        const float ak = area_rn(ch[k].lo, ch[k].hi);
        if (ak > area) {
          area = ak;
          best = k;
        }
      }
    if (best < 0) break;
    const int b = ch[best].node;
    const WElem c = welem_child(bin, b, 1);
    ch[best] = welem_child(bin, b, 0);
    if (c.node >= 0 || c.count > 0) ch[n++] = c;
  }
  // slot order: the (child, free slot) pair whose child centre lies furthest
  // along the slot's octant direction from the node centre goes first
  float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int k = 0; k < n; ++k)
    for (int a = 0; a < 3; ++a) {
      nlo[a] = fminf(nlo[a], ch[k].lo[a]);
      nhi[a] = fmaxf(nhi[a], ch[k].hi[a]);
    }
  float cc[3];
  for (int a = 0; a < 3; ++a) cc[a] = __fmul_rn(0.5f, __fadd_rn(nlo[a], nhi[a]));
  WElem sl[8];
  for (int k = 0; k < 8; ++k) welem_empty(sl[k]);
  uint32_t placed = 0u, used = 0u;
  for (int round = 0; round < n; ++round) {
    float best = -INFINITY;
    int bc = -1, bs = -1;
    for (int k = 0; k < n; ++k) {
      if ((placed >> k) & 1u) continue;
      float off[3];
      for (int a = 0; a < 3; ++a) off[a] = __fsub_rn(__fmul_rn(0.5f, __fadd_rn(ch[k].lo[a], ch[k].hi[a])), cc[a]);
      for (int q = 0; q < 8; ++q) {
        if ((used >> q) & 1u) continue;
        float score = 0.f;
        for (int a = 0; a < 3; ++a) score = __fadd_rn(score, ((q >> a) & 1) ? off[a] : -off[a]);
        if (score > best) {
          best = score;
          bc = k;
          bs = q;
        }
      }
    }
    if (bc < 0) {  // non-finite centres: first unplaced child into the first free slot
      for (bc = 0; (placed >> bc) & 1u; ++bc) {}
      for (bs = 0; (used >> bs) & 1u; ++bs) {}
    }
    placed |= 1u << bc;
    used |= 1u << bs;
    sl[bs] = ch[bc];
  }
  // margin of the node's size so that FP32 rounding in the slab test can
  // never cull a boundary hit (every slot, empty ones included, as the host)
  float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int k = 0; k < 8; ++k)
    for (int a = 0; a < 3; ++a) {
      rlo[a] = fminf(rlo[a], sl[k].lo[a]);
      rhi[a] = fmaxf(rhi[a], sl[k].hi[a]);
    }
  float mext = 0.f, mabs = 0.f;
  for (int a = 0; a < 3; ++a) {
    mext = fmaxf(mext, __fsub_rn(rhi[a], rlo[a]));
    mabs = fmaxf(mabs, fmaxf(fabsf(rlo[a]), fabsf(rhi[a])));
  }
  const float margin = __fadd_rn(__fadd_rn(__fmul_rn(1e-5f, mext), __fmul_rn(1e-6f, mabs)), 1e-30f);
  for (int k = 0; k < 8; ++k)
    for (int a = 0; a < 3; ++a) {
      sl[k].lo[a] = __fsub_rn(sl[k].lo[a], margin);
      sl[k].hi[a] = __fadd_rn(sl[k].hi[a], margin);
    }
  float blo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int k = 0; k < 8; ++k)
    for (int a = 0; a < 3; ++a) {
      blo[a] = fminf(blo[a], sl[k].lo[a]);
      bhi[a] = fmaxf(bhi[a], sl[k].hi[a]);
    }
  // per axis the power-of-two scale: the smallest e (at least -100) with
  // 255 2^e >= extent (1 + 1e-6), which is what the host's log2 estimate and
  // its correction loop give
  double p[3], sc[3];
  int ex[3];
  for (int a = 0; a < 3; ++a) {
    p[a] = (double)blo[a];
    const double ext = __dsub_rn((double)bhi[a], (double)blo[a]);
    const double need = __dmul_rn(ext, 1.0 + 1e-6);
    int e = ext > 0 ? (int)ceil(log2(__ddiv_rn(ext, 255.0))) : -100;
    if (e < -100) e = -100;
    while (ldexp(255.0, e) < need) ++e;
    while (e > -100 && ldexp(255.0, e - 1) >= need) --e;
    ex[a] = e;
    sc[a] = ldexp(1.0, e);
  }
  for (int k = 0; k < 20; ++k) words[k] = 0u;
  words[0] = __float_as_uint(blo[0]);
  words[1] = __float_as_uint(blo[1]);
  words[2] = __float_as_uint(blo[2]);
  uint32_t imask = 0u, inner = 0u, tris = 0u;
  for (int k = 0; k < 8; ++k) {
    const WElem& e = sl[k];
    if (e.node < 0 && e.count == 0) continue;  // empty slot
    for (int a = 0; a < 3; ++a) {
      const double lo = floor(__dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)e.lo[a], p[a]), sc[a]), 1.0 - 1e-6), 1e-6));
      const double hi = ceil(__dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn((double)e.hi[a], p[a]), sc[a]), 1.0 + 1e-6), 1e-6));
      const uint32_t ql = (uint32_t)fmin(255.0, fmax(0.0, lo)), qh = (uint32_t)fmin(255.0, fmax(0.0, hi));
      words[8 + 4 * a + (k >> 2)] |= ql << (8 * (k & 3));
      words[10 + 4 * a + (k >> 2)] |= qh << (8 * (k & 3));
    }
    if (e.node >= 0) {
      imask |= 1u << k;
      ++inner;
    } else {
      if (e.count > 3 || tris + e.count > 32) *bad = true;
      const uint32_t meta = (e.count << 5) | tris;
      words[6 + (k >> 2)] |= (meta & 0xffu) << (8 * (k & 3));
      tris += e.count;
    }
  }
  words[3] = (uint32_t)(uint8_t)(int8_t)ex[0] | ((uint32_t)(uint8_t)(int8_t)ex[1] << 8) |
             ((uint32_t)(uint8_t)(int8_t)ex[2] << 16) | (imask << 24);
  for (int k = 0; k < 8; ++k) ch[k] = sl[k];
  *ntris = tris;
  return inner;
}

// Pass 1 of a level: inner children and leaf triangles of every wide node,
// packed (inner << 32 | triangles) for one prefix sum.
__global__ void k_wide_count(const float4* __restrict__ bin, const int* __restrict__ seeds, uint32_t n, bool root,
                             unsigned long long* __restrict__ counts, uint32_t* __restrict__ bad) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n) return;
  WElem ch[8];
  uint32_t words[20], tris;
  bool b = false;
  const uint32_t inner = wide_node(bin, seeds[w], root, ch, words, &tris, &b);
  counts[w] = ((unsigned long long)inner << 32) | tris;
  if (b) atomicOr(bad, 1u);
}

// Pass 2: the node words, the next level's seeds (inner children in slot
// order from child_base) and the leaves' triangles (from tri_base). first_node
// is the level's first node index, next_first the next level's.
__global__ void k_wide_write(const float4* __restrict__ bin, const uint32_t* __restrict__ bin_order,
                             const int* __restrict__ seeds, uint32_t n, bool root,
                             const unsigned long long* __restrict__ excl, uint32_t first_node, uint32_t next_first,
                             uint32_t tri_first, uint4* __restrict__ out, int* __restrict__ next_seeds,
                             uint32_t* __restrict__ order) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n) return;
  WElem ch[8];
  uint32_t words[20], tris;
  bool b = false;
  wide_node(bin, seeds[w], root, ch, words, &tris, &b);
  const uint32_t ibase = (uint32_t)(excl[w] >> 32), tbase = tri_first + (uint32_t)(excl[w] & 0xffffffffull);
  words[4] = next_first + ibase;
  words[5] = tbase;
  uint32_t rank = 0, t = 0;
  for (int k = 0; k < 8; ++k) {
    const WElem& e = ch[k];
    if (e.node >= 0) {
      next_seeds[ibase + rank++] = e.node;
    } else {
      for (uint32_t j = 0; j < e.count; ++j) order[tbase + t + j] = bin_order[e.first + j];
      t += e.count;
    }
  }
  uint4* o = out + 5 * (size_t)(first_node + w);
  for (int q = 0; q < 5; ++q) o[q] = make_uint4(words[4 * q], words[4 * q + 1], words[4 * q + 2], words[4 * q + 3]);
}

}  // namespace

int build_wide_bvh_gpu(cudaStream_t st, const float* dV, const uint32_t* dI, uint32_t nt, GpuWideBvh* out,
                       std::string* err) {
  *out = GpuWideBvh{};
  if (nt == 0) return 0;
  GpuBvh g;
  int rc = build_bvh_gpu(st, dV, dI, nt, &g, err, 3);
  if (rc) return rc;
  Bufs B;
  B.v.push_back(g.nodes);
  B.v.push_back(g.order);
  // every wide node has its own binary inner node as seed
  const uint32_t cap = std::max<uint32_t>(g.n_inner, 1);
  uint4* wn;
  uint32_t *order, *bad;
  int *seeds0, *seeds1;
  unsigned long long *counts, *excl;
  GYT_BCK(B.get(&wn, 5 * (size_t)cap));
  GYT_BCK(B.get(&order, nt));
  GYT_BCK(B.get(&seeds0, cap));
  GYT_BCK(B.get(&seeds1, cap));
  GYT_BCK(B.get(&counts, (size_t)cap + 1));
  GYT_BCK(B.get(&excl, (size_t)cap + 1));
  GYT_BCK(B.get(&bad, 1));
  size_t scan_bytes = 0;
  GYT_BCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, excl, (int)cap + 1, st));
  uint8_t* scan_tmp;
  GYT_BCK(B.get(&scan_tmp, scan_bytes));
  GYT_BCK(cudaMemsetAsync(seeds0, 0, sizeof(int), st));  // the binary root
  GYT_BCK(cudaMemsetAsync(bad, 0, sizeof(uint32_t), st));
  uint32_t level_first = 0, level_n = 1, tri_first = 0, levels = 0;
  int *cur = seeds0, *nxt = seeds1;
  while (level_n > 0) {
    if (++levels > 64 || level_first + level_n > cap) {
      *err = "build_wide_bvh_gpu: node capacity or depth exceeded";
      return 4;
    }
    const bool root = level_first == 0;
    k_wide_count<<<blocks(level_n, 128), 128, 0, st>>>(g.nodes, cur, level_n, root, counts, bad);
    GYT_BCK(cudaMemsetAsync(counts + level_n, 0, sizeof(unsigned long long), st));
    GYT_BCK(cudaGetLastError());
    GYT_BCK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, excl, (int)level_n + 1, st));
    unsigned long long tot;
    GYT_BCK(cudaMemcpyAsync(&tot, excl + level_n, sizeof(tot), cudaMemcpyDeviceToHost, st));
    GYT_BCK(cudaStreamSynchronize(st));
    const uint32_t next_n = (uint32_t)(tot >> 32), ntris = (uint32_t)(tot & 0xffffffffull);
    if ((uint64_t)level_first + level_n + next_n > cap || (uint64_t)tri_first + ntris > nt) {
      *err = "build_wide_bvh_gpu: node or triangle capacity exceeded";
      return 4;
    }
    k_wide_write<<<blocks(level_n, 128), 128, 0, st>>>(g.nodes, g.order, cur, level_n, root, excl, level_first,
                                                        level_first + level_n, tri_first, wn, nxt, order);
    GYT_BCK(cudaGetLastError());
    level_first += level_n;
    tri_first += ntris;
    level_n = next_n;
    std::swap(cur, nxt);
  }
  uint32_t hbad = 0;
  GYT_BCK(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
  GYT_BCK(cudaStreamSynchronize(st));
  if (hbad || tri_first != nt) {
    *err = "build_wide_bvh_gpu: a leaf does not fit the 8-wide node layout";
    return 4;
  }
  // the exact node count: move the nodes into an allocation of that size
  uint4* exact;
  GYT_BCK(B.get(&exact, 5 * (size_t)level_first));
  GYT_BCK(cudaMemcpyAsync(exact, wn, 5 * (size_t)level_first * sizeof(uint4), cudaMemcpyDeviceToDevice, st));
  GYT_BCK(cudaStreamSynchronize(st));
  B.release(exact);
  B.release(order);
  out->nodes = exact;
  out->order = order;
  out->n_nodes = level_first;
  out->max_depth = levels;
  return 0;
}

}  // namespace gyt
