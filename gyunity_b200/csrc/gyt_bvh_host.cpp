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

// Widen a box by a few ulps of its largest coordinate magnitude so that
// rounding in the slab test cannot cull a boundary hit.
void pad(Box& b) {
  float m = 0.f;
  for (int a = 0; a < 3; ++a) m = std::max(m, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
  float e = m * 4.0e-7f + 1e-30f;
  for (int a = 0; a < 3; ++a) { b.lo[a] -= e; b.hi[a] += e; }
}

}  // namespace

bool build_bvh_host(const float* V, uint32_t nv, const uint32_t* I, uint32_t nt, BvhHost* out, int max_leaf) {
  const int kMaxLeaf = std::min(8, std::max(1, max_leaf));
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
      // triangles of a leaf in ascending id order (the device builder's order too)
      std::sort(idx.begin() + start, idx.begin() + start + count);
      uint32_t first = (uint32_t)out->order.size();
      for (uint32_t k = start; k < start + count; ++k) out->order.push_back(idx[k]);
      Box b;
      for (uint32_t k = start; k < start + count; ++k) b.grow(pb[idx[k]]);
      set_child(parent, slot, b, leaf_code(first, count));
    };
    if (j.parent >= 0 && j.count <= (uint32_t)kMaxLeaf && j.count <= 2u) {
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

namespace {

struct Elem {
  Box box;
  int node;           // binary inner node, or -1 for a leaf
  uint32_t first, count;
};

Elem child_elem(const std::vector<float>& nodes, int node, int slot) {
  const float* n = &nodes[(size_t)node * 16];
  Elem e;
  if (slot == 0) {
    e.box.lo[0] = n[0]; e.box.hi[0] = n[1]; e.box.lo[1] = n[2]; e.box.hi[1] = n[3];
    e.box.lo[2] = n[8]; e.box.hi[2] = n[9];
  } else {
    e.box.lo[0] = n[4]; e.box.hi[0] = n[5]; e.box.lo[1] = n[6]; e.box.hi[1] = n[7];
    e.box.lo[2] = n[10]; e.box.hi[2] = n[11];
  }
  int c;
  std::memcpy(&c, &n[12 + slot], 4);
  if (c >= 0) {
    e.node = c;
    e.first = e.count = 0;
  } else {
    uint32_t code = ~(uint32_t)c;
    e.node = -1;
    e.first = code >> 3;
    e.count = (code & 7u) + 1u;
  }
  return e;
}

// Child slots as in Ylitie, Karras and Laine (HPG 2017): slot s faces the
// octant direction d_s (component a is +1 when bit a of s is set, else -1);
// greedily, the (child, free slot) pair whose child centre lies furthest along
// d_s from the node centre is placed first. A ray whose negative direction
// axes are the bits o then meets the children roughly in increasing order of
// slot ^ o. Returns 8 entries; empty slots are leaves with no triangles.
std::vector<Elem> slot_order(const std::vector<Elem>& ch) {
  Box nb;
  for (const Elem& e : ch) nb.grow(e.box);
  float c[3];
  for (int a = 0; a < 3; ++a) c[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
  std::vector<Elem> slots(8);
  for (Elem& e : slots) { e.node = -1; e.first = e.count = 0; }
  std::vector<bool> placed(ch.size(), false), used(8, false);
  for (size_t round = 0; round < ch.size(); ++round) {
    float best = -INFINITY;
    int bc = -1, bs = -1;
    for (size_t k = 0; k < ch.size(); ++k) {
      if (placed[k]) continue;
      float off[3];
      for (int a = 0; a < 3; ++a) off[a] = 0.5f * (ch[k].box.lo[a] + ch[k].box.hi[a]) - c[a];
      for (int sl = 0; sl < 8; ++sl) {
        if (used[sl]) continue;
        float score = 0.f;
        for (int a = 0; a < 3; ++a) score += ((sl >> a) & 1) ? off[a] : -off[a];
        if (score > best) { best = score; bc = (int)k; bs = sl; }
      }
    }
    if (bc < 0) {  // non-finite centres: first unplaced child into the first free slot
      for (bc = 0; placed[bc]; ++bc) {}
      for (bs = 0; used[bs]; ++bs) {}
    }
    placed[bc] = true;
    used[bs] = true;
    slots[bs] = ch[bc];
  }
  return slots;
}

}  // namespace

bool build_wide_bvh_host(const float* V, uint32_t nv, const uint32_t* I, uint32_t nt, WideBvhHost* out) {
  out->nodes.clear();
  out->order.clear();
  out->max_depth = 0;
  if (nt == 0) return true;
  BvhHost bin;
  if (!build_bvh_host(V, nv, I, nt, &bin, 3)) return false;
  // the binary root's own box is not stored: build it from its two children
  struct Pending { std::vector<Elem> children; uint32_t depth; };
  std::vector<std::vector<Elem>> todo;  // children of each wide node, in node order
  std::vector<uint32_t> depth;
  auto expand = [&](std::vector<Elem> ch) {
    while (ch.size() < 8) {
      int best = -1;
      float area = -1.f;
      for (size_t k = 0; k < ch.size(); ++k)
        if (ch[k].node >= 0 && ch[k].box.area() > area) { area = ch[k].box.area(); best = (int)k; }
      if (best < 0) break;
      int b = ch[best].node;
      Elem a = child_elem(bin.nodes, b, 0), c = child_elem(bin.nodes, b, 1);
      ch[best] = a;
      if (c.node >= 0 || c.count > 0) ch.push_back(c);
    }
    return ch;
  };
  std::vector<Elem> root = {child_elem(bin.nodes, 0, 0), child_elem(bin.nodes, 0, 1)};
  if (root[1].node < 0 && root[1].count > 0 && !(root[1].box.lo[0] <= root[1].box.hi[0])) root.pop_back();
  todo.push_back(expand(root));
  depth.push_back(1);
  for (size_t w = 0; w < todo.size(); ++w) {
    std::vector<Elem> ch = slot_order(todo[w]);
    // inner children first get consecutive node indices
    uint32_t child_base = (uint32_t)todo.size();
    uint32_t tri_base = (uint32_t)out->order.size();
    // widen every child box by a margin of the node's size so that FP32
    // rounding in the slab test can never cull a boundary hit
    Box raw;
    for (const Elem& e : ch) raw.grow(e.box);
    float mext = 0.f, mabs = 0.f;
    for (int a = 0; a < 3; ++a) {
      mext = std::max(mext, raw.hi[a] - raw.lo[a]);
      mabs = std::max(mabs, std::max(std::fabs(raw.lo[a]), std::fabs(raw.hi[a])));
    }
    const float margin = 1e-5f * mext + 1e-6f * mabs + 1e-30f;
    for (Elem& e : ch)
      for (int a = 0; a < 3; ++a) { e.box.lo[a] -= margin; e.box.hi[a] += margin; }
    Box nb;
    for (const Elem& e : ch) nb.grow(e.box);
    double p[3], sc[3];
    int ex[3];
    for (int a = 0; a < 3; ++a) {
      p[a] = nb.lo[a];
      double ext = (double)nb.hi[a] - (double)nb.lo[a];
      int e = ext > 0 ? (int)std::ceil(std::log2(ext / 255.0)) : -100;
      if (e < -100) e = -100;
      // one ulp of headroom so the outward rounding below always fits in 255
      while (std::ldexp(255.0, e) < ext * (1.0 + 1e-6)) ++e;
      ex[a] = e;
      sc[a] = std::ldexp(1.0, e);
    }
    uint32_t words[20] = {};
    float pf[3] = {nb.lo[0], nb.lo[1], nb.lo[2]};
    std::memcpy(&words[0], &pf[0], 4);
    std::memcpy(&words[1], &pf[1], 4);
    std::memcpy(&words[2], &pf[2], 4);
    uint32_t imask = 0;
    uint8_t meta[8] = {}, qlo[3][8] = {}, qhi[3][8] = {};
    uint32_t inner_rank = 0;
    for (size_t k = 0; k < ch.size(); ++k) {
      const Elem& e = ch[k];
      if (e.node < 0 && e.count == 0) continue;  // empty slot
      for (int a = 0; a < 3; ++a) {
        double lo = std::floor(((double)e.box.lo[a] - p[a]) / sc[a] * (1.0 - 1e-6) - 1e-6);
        double hi = std::ceil(((double)e.box.hi[a] - p[a]) / sc[a] * (1.0 + 1e-6) + 1e-6);
        qlo[a][k] = (uint8_t)std::min(255.0, std::max(0.0, lo));
        qhi[a][k] = (uint8_t)std::min(255.0, std::max(0.0, hi));
      }
      if (e.node >= 0) {
        imask |= 1u << k;
        std::vector<Elem> sub = {child_elem(bin.nodes, e.node, 0), child_elem(bin.nodes, e.node, 1)};
        todo.push_back(expand(sub));
        depth.push_back(depth[w] + 1);
        ++inner_rank;
      } else {
        uint32_t off = (uint32_t)out->order.size() - tri_base;
        if (e.count > 3 || off + e.count > 32) return false;
        for (uint32_t t = 0; t < e.count; ++t) out->order.push_back(bin.order[e.first + t]);
        meta[k] = (uint8_t)((e.count << 5) | off);
      }
    }
    out->max_depth = std::max(out->max_depth, depth[w]);
    words[3] = (uint32_t)(uint8_t)(int8_t)ex[0] | ((uint32_t)(uint8_t)(int8_t)ex[1] << 8) |
               ((uint32_t)(uint8_t)(int8_t)ex[2] << 16) | (imask << 24);
    words[4] = child_base;
    words[5] = tri_base;
    std::memcpy(&words[6], meta, 8);
    for (int a = 0; a < 3; ++a) {
      std::memcpy(&words[8 + 4 * a], qlo[a], 8);
      std::memcpy(&words[10 + 4 * a], qhi[a], 8);
    }
    out->nodes.insert(out->nodes.end(), words, words + 20);
  }
  return out->order.size() == nt;
}

}  // namespace gyt
