// Binned-SAH binary BVH builder on the host (see gyt_bvh_host.h for the layout).
#include "gyt_bvh_host.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace gyt {
namespace {

struct Box {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const Box& b) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
  }
  void grow(const float* p) {
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
  }
  float area() const {
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = std::max(0.f, hi[a] - lo[a]);
    return 2.f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
  bool valid() const { return lo[0] <= hi[0]; }
};

constexpr int kBins = 16;
constexpr int kMaxLeaf = 8;

// Widen a box by a few ulps of its largest coordinate magnitude so that
// rounding in the slab test cannot cull a boundary hit.
void pad(Box& b) {
  float m = 0.f;
  for (int a = 0; a < 3; ++a) m = std::max(m, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
  float e = m * 4.0e-7f + 1e-30f;
  for (int a = 0; a < 3; ++a) { b.lo[a] -= e; b.hi[a] += e; }
}

}  // namespace

bool build_bvh_host(const float* V, uint32_t nv, const uint32_t* I, uint32_t nt, BvhHost* out) {
  out->nodes.clear();
  out->order.clear();
  out->max_depth = 0;
  if (nt == 0) return true;
  std::vector<Box> pb(nt);
  std::vector<float> cen((size_t)nt * 3);
  for (uint32_t t = 0; t < nt; ++t) {
    for (int k = 0; k < 3; ++k) {
      uint32_t v = I[3 * t + k];
      if (v >= nv) return false;
      pb[t].grow(&V[3 * v]);
    }
    for (int a = 0; a < 3; ++a) cen[3 * t + a] = 0.5f * (pb[t].lo[a] + pb[t].hi[a]);
  }
  std::vector<uint32_t> idx(nt);
  for (uint32_t t = 0; t < nt; ++t) idx[t] = t;

  struct Job { uint32_t start, count; int parent, slot; uint32_t depth; };
  std::vector<Job> stack;
  std::vector<float>& nodes = out->nodes;
  auto new_node = [&]() {
    size_t id = nodes.size() / 16;
    nodes.resize(nodes.size() + 16, 0.f);
    return (int)id;
  };
  auto set_child = [&](int parent, int slot, const Box& b0, int child) {
    Box b = b0;
    pad(b);
    float* n = &nodes[(size_t)parent * 16];
    if (slot == 0) {
      n[0] = b.lo[0]; n[1] = b.hi[0]; n[2] = b.lo[1]; n[3] = b.hi[1];
      n[8] = b.lo[2]; n[9] = b.hi[2];
    } else {
      n[4] = b.lo[0]; n[5] = b.hi[0]; n[6] = b.lo[1]; n[7] = b.hi[1];
      n[10] = b.lo[2]; n[11] = b.hi[2];
    }
    std::memcpy(&n[12 + slot], &child, 4);
  };
  auto leaf_code = [&](uint32_t first, uint32_t count) { return (int)~((first << 3) | (count - 1)); };

  // The root is always an inner node; a scene that fits one leaf gets an
  // empty (inverted-box, never hit) second child.
  int root = new_node();
  Box all;
  for (uint32_t t = 0; t < nt; ++t) all.grow(pb[t]);
  if (nt <= (uint32_t)kMaxLeaf) {
    out->order = idx;
    set_child(root, 0, all, leaf_code(0, nt));
    float* n = &nodes[0];
    n[4] = n[6] = n[10] = FLT_MAX;
    n[5] = n[7] = n[11] = -FLT_MAX;
    int code = leaf_code(0, nt);
    std::memcpy(&n[13], &code, 4);
    out->max_depth = 1;
    return true;
  }
  stack.push_back({0, nt, -1, 0, 0});
  std::vector<Box> binb(kBins * 3), left(kBins), right(kBins);
  std::vector<uint32_t> binc(kBins * 3);
  out->order.reserve(nt);
  while (!stack.empty()) {
    Job j = stack.back();
    stack.pop_back();
    out->max_depth = std::max(out->max_depth, j.depth + 1);
    Box nb, cb;
    for (uint32_t k = j.start; k < j.start + j.count; ++k) {
      uint32_t t = idx[k];
      nb.grow(pb[t]);
      cb.grow(&cen[3 * t]);
    }
    auto make_leaf = [&](uint32_t start, uint32_t count, int parent, int slot) {
      uint32_t first = (uint32_t)out->order.size();
      for (uint32_t k = start; k < start + count; ++k) out->order.push_back(idx[k]);
      Box b;
      for (uint32_t k = start; k < start + count; ++k) b.grow(pb[idx[k]]);
      set_child(parent, slot, b, leaf_code(first, count));
    };
    if (j.parent >= 0 && j.count <= (uint32_t)kMaxLeaf && j.count <= 2) {
      make_leaf(j.start, j.count, j.parent, j.slot);
      continue;
    }
    // binned SAH over the longest usable axes
    float best = FLT_MAX;
    int best_axis = -1, best_split = -1;
    for (int a = 0; a < 3; ++a) {
      float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.f)) continue;
      float scale = kBins / ext;
      for (int b = 0; b < kBins; ++b) { binb[b] = Box(); binc[b] = 0; }
      for (uint32_t k = j.start; k < j.start + j.count; ++k) {
        uint32_t t = idx[k];
        int b = std::min(kBins - 1, (int)((cen[3 * t + a] - cb.lo[a]) * scale));
        binb[b].grow(pb[t]);
        binc[b]++;
      }
      Box acc;
      uint32_t cnt = 0;
      std::vector<uint32_t> lc(kBins);
      for (int b = 0; b < kBins; ++b) {
        acc.grow(binb[b]);
        cnt += binc[b];
        left[b] = acc;
        lc[b] = cnt;
      }
      acc = Box();
      cnt = 0;
      for (int b = kBins - 1; b > 0; --b) {
        acc.grow(binb[b]);
        cnt += binc[b];
        uint32_t l = lc[b - 1];
        if (l == 0 || cnt == 0) continue;
        float cost = left[b - 1].area() * l + acc.area() * cnt;
        if (cost < best) { best = cost; best_axis = a; best_split = b; }
      }
    }
    float leaf_cost = nb.area() * j.count;
    int parent = j.parent, slot = j.slot;
    if (parent >= 0 && j.count <= (uint32_t)kMaxLeaf && (best_axis < 0 || best * 1.0f + nb.area() * 1.0f >= leaf_cost)) {
      make_leaf(j.start, j.count, parent, slot);
      continue;
    }
    uint32_t mid;
    if (best_axis < 0) {
      mid = j.start + j.count / 2;  // all centroids coincide: split by count
    } else {
      float scale = kBins / (cb.hi[best_axis] - cb.lo[best_axis]);
      auto it = std::partition(idx.begin() + j.start, idx.begin() + j.start + j.count, [&](uint32_t t) {
        int b = std::min(kBins - 1, (int)((cen[3 * t + best_axis] - cb.lo[best_axis]) * scale));
        return b < best_split;
      });
      mid = (uint32_t)(it - idx.begin());
      if (mid == j.start || mid == j.start + j.count) mid = j.start + j.count / 2;
    }
    int node;
    if (parent < 0) {
      node = root;
    } else {
      node = new_node();
      set_child(parent, slot, nb, node);
    }
    // push right first so the left subtree is laid out first (depth-first)
    stack.push_back({mid, j.start + j.count - mid, node, 1, j.depth + 1});
    stack.push_back({j.start, mid - j.start, node, 0, j.depth + 1});
  }
  return true;
}

}  // namespace gyt
