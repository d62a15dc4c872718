// Host BVH builder (binned SAH, multi-threaded over large subtrees) and
// converters to the device layouts.
//
// The reference builds its tree with a full sweep over every split position
// (build_bvh, main.py:437-507), which is quadratic per node and takes minutes
// beyond ~10k triangles.  Binning the centroids (Wald, "On fast construction
// of SAH-based bounding volume hierarchies", 2007) gives trees of comparable
// quality in O(n log n); closest-hit results do not depend on the tree.
#include "bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <thread>

#include "limits.h"

namespace ts {

namespace {

struct Prim {
  float lo[3], hi[3], c[3];
};

struct BNode {
  float lo[3], hi[3];
  int32_t left, right;  // child indices within the same vector; -1 for leaves
  int32_t first, count;
};

// Flat boxes make the strict t_enter < t_exit slab test fail for rays that hit
// the face they lie in, so a zero extent is widened (the reference adds 1e-6,
// main.py:456-460; here at least a few ulps of the coordinate as well).
inline void pad_box(float lo[3], float hi[3]) {
  for (int a = 0; a < 3; ++a) {
    if (lo[a] == hi[a]) {
      const float p = std::max(1e-6f, std::fabs(lo[a]) * 4.8e-7f);
      lo[a] -= p;
      hi[a] += p;
    }
  }
}

inline double half_area(const float lo[3], const float hi[3]) {
  const double dx = std::max(0.0, (double)hi[0] - lo[0]);
  const double dy = std::max(0.0, (double)hi[1] - lo[1]);
  const double dz = std::max(0.0, (double)hi[2] - lo[2]);
  return dx * dy + dy * dz + dz * dx;
}

struct Builder {
  const std::vector<Prim> &prims;
  std::vector<int32_t> &idx;
  BvhParams p;

  void bounds(int b, int e, float lo[3], float hi[3], float clo[3], float chi[3]) const {
    for (int a = 0; a < 3; ++a) {
      lo[a] = clo[a] = INFINITY;
      hi[a] = chi[a] = -INFINITY;
    }
    for (int i = b; i < e; ++i) {
      const Prim &q = prims[idx[i]];
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], q.lo[a]);
        hi[a] = std::max(hi[a], q.hi[a]);
        clo[a] = std::min(clo[a], q.c[a]);
        chi[a] = std::max(chi[a], q.c[a]);
      }
    }
  }

  int median_split(int b, int e, const float clo[3], const float chi[3]) {
    int ax = 0;
    for (int a = 1; a < 3; ++a)
      if (chi[a] - clo[a] > chi[ax] - clo[ax]) ax = a;
    const int mid = b + (e - b) / 2;
    std::nth_element(idx.begin() + b, idx.begin() + mid, idx.begin() + e,
                     [&](int32_t x, int32_t y) { return prims[x].c[ax] < prims[y].c[ax]; });
    return mid;
  }

  // Fills node's box; returns the split position or -1 for a leaf.
  int decide(int b, int e, int depth, BNode &node) {
    float clo[3], chi[3];
    bounds(b, e, node.lo, node.hi, clo, chi);
    pad_box(node.lo, node.hi);
    const int n = e - b;
    node.left = node.right = -1;
    node.first = b;
    node.count = n;
    if (n <= 1) return -1;
    const int hard_max = std::min(p.leaf_max, kLeafMax);
    if (depth >= p.sah_depth) return n <= hard_max ? -1 : median_split(b, e, clo, chi);
    const int K = std::max(2, std::min(p.bins, 256));
    double best = INFINITY;
    int best_axis = -1, best_bin = -1;
    std::vector<float> blo(3 * K), bhi(3 * K), rlo(3 * K), rhi(3 * K);
    std::vector<int> bc(K);
    std::vector<double> racc(K);
    std::vector<int> rcnt(K);
    for (int a = 0; a < 3; ++a) {
      const float ext = chi[a] - clo[a];
      if (!(ext > 0.f)) continue;
      const float k = (float)K * (1.0f - 1e-6f) / ext;
      std::fill(bc.begin(), bc.end(), 0);
      for (int i = 0; i < K; ++i)
        for (int d = 0; d < 3; ++d) {
          blo[3 * i + d] = INFINITY;
          bhi[3 * i + d] = -INFINITY;
        }
      for (int i = b; i < e; ++i) {
        const Prim &q = prims[idx[i]];
        int bi = (int)((q.c[a] - clo[a]) * k);
        bi = std::min(std::max(bi, 0), K - 1);
        bc[bi]++;
        for (int d = 0; d < 3; ++d) {
          blo[3 * bi + d] = std::min(blo[3 * bi + d], q.lo[d]);
          bhi[3 * bi + d] = std::max(bhi[3 * bi + d], q.hi[d]);
        }
      }
      // right-to-left accumulation
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      int cnt = 0;
      for (int i = K - 1; i > 0; --i) {
        for (int d = 0; d < 3; ++d) {
          lo[d] = std::min(lo[d], blo[3 * i + d]);
          hi[d] = std::max(hi[d], bhi[3 * i + d]);
        }
        cnt += bc[i];
        rcnt[i] = cnt;
        racc[i] = cnt ? half_area(lo, hi) * cnt : 0.0;
      }
      for (int d = 0; d < 3; ++d) { lo[d] = INFINITY; hi[d] = -INFINITY; }
      cnt = 0;
      for (int i = 0; i < K - 1; ++i) {
        for (int d = 0; d < 3; ++d) {
          lo[d] = std::min(lo[d], blo[3 * i + d]);
          hi[d] = std::max(hi[d], bhi[3 * i + d]);
        }
        cnt += bc[i];
        if (cnt == 0 || rcnt[i + 1] == 0) continue;
        const double c = half_area(lo, hi) * cnt + racc[i + 1];
        if (c < best) { best = c; best_axis = a; best_bin = i; }
      }
    }
    if (best_axis < 0) return n <= kLeafMax ? -1 : median_split(b, e, clo, chi);
    const double A = half_area(node.lo, node.hi);
    const double split_cost = p.cost_trav + p.cost_tri * (A > 0 ? best / A : (double)n);
    const double leaf_cost = p.cost_tri * n;
    if (n <= hard_max && leaf_cost <= split_cost) return -1;
    const float ext = chi[best_axis] - clo[best_axis];
    const float k = (float)K * (1.0f - 1e-6f) / ext;
    auto it = std::partition(idx.begin() + b, idx.begin() + e, [&](int32_t t) {
      int bi = (int)((prims[t].c[best_axis] - clo[best_axis]) * k);
      bi = std::min(std::max(bi, 0), K - 1);
      return bi <= best_bin;
    });
    int mid = (int)(it - idx.begin());
    if (mid == b || mid == e) mid = median_split(b, e, clo, chi);
    return mid;
  }

  int rec(std::vector<BNode> &out, int b, int e, int depth) {
    const int me = (int)out.size();
    out.push_back(BNode{});
    BNode node;
    const int mid = decide(b, e, depth, node);
    out[me] = node;
    if (mid < 0) return me;
    const int l = rec(out, b, mid, depth + 1);
    const int r = rec(out, mid, e, depth + 1);
    out[me].left = l;
    out[me].right = r;
    return me;
  }

  std::vector<BNode> task(int b, int e, int depth, int par_levels) {
    std::vector<BNode> out;
    if (par_levels <= 0 || e - b < 65536) {
      out.reserve((size_t)(2 * (e - b) / 3 + 16));
      rec(out, b, e, depth);
      return out;
    }
    BNode root;
    const int mid = decide(b, e, depth, root);
    if (mid < 0) {
      out.push_back(root);
      return out;
    }
    auto fl = std::async(std::launch::async, [&, b, mid]() { return task(b, mid, depth + 1, par_levels - 1); });
    std::vector<BNode> r = task(mid, e, depth + 1, par_levels - 1);
    std::vector<BNode> l = fl.get();
    out.reserve(1 + l.size() + r.size());
    out.push_back(root);
    auto append = [&](const std::vector<BNode> &v, int off) {
      for (BNode x : v) {
        if (x.left >= 0) { x.left += off; x.right += off; }
        out.push_back(x);
      }
    };
    out[0].left = 1;
    out[0].right = 1 + (int)l.size();
    append(l, 1);
    append(r, 1 + (int)l.size());
    return out;
  }
};

inline int32_t leaf_code(int first, int count) { return ~((first << 4) | (count - 1)); }

// Split leaves larger than kLeafMax into index chunks (new nodes appended).
void expand_big_leaves(std::vector<BNode> &tree, const std::vector<Prim> &prims, const std::vector<int32_t> &perm) {
  for (size_t i = 0; i < tree.size(); ++i) {
    BNode nd = tree[i];
    if (nd.left < 0 && nd.count > kLeafMax) {
      const int half = nd.count / 2;
      BNode a{}, c{};
      for (int s = 0; s < 2; ++s) {
        BNode &ch = s ? c : a;
        ch.first = s ? nd.first + half : nd.first;
        ch.count = s ? nd.count - half : half;
        ch.left = ch.right = -1;
        for (int d = 0; d < 3; ++d) { ch.lo[d] = INFINITY; ch.hi[d] = -INFINITY; }
        for (int k = ch.first; k < ch.first + ch.count; ++k)
          for (int d = 0; d < 3; ++d) {
            ch.lo[d] = std::min(ch.lo[d], prims[perm[k]].lo[d]);
            ch.hi[d] = std::max(ch.hi[d], prims[perm[k]].hi[d]);
          }
        pad_box(ch.lo, ch.hi);
      }
      tree[i].left = (int)tree.size();
      tree.push_back(a);
      tree[i].right = (int)tree.size();
      tree.push_back(c);
    }
  }
}

// Wide layout: collapse the binary tree greedily (an inner child with the
// largest surface area is replaced by its two children until a node has
// `width` children) and store each node's child boxes as SoA float4 rows:
//   width 4: lo.x hi.x lo.y hi.y lo.z hi.z refs pad         (8 float4, 128 B)
//   width 8: each of the six rows and the refs as two float4 (16 float4, 256 B)
// Empty child slots have NaN boxes, which no slab test accepts.  Returns false
// (out untouched) if the traversal stack bound would be exceeded.
// Quantized wide node (layout ids 5 and 9): the node's origin (the low corner
// of its children's union) and one power-of-two scale per axis; each child
// box as bytes q with bound = origin + q * scale, rounded outwards so that the
// decoded box -- computed on the device as one float multiply (exact: q < 256
// times a power of two) and one float add -- contains the exact box:
//   float4 0: origin.xyz, (biased scale exponents x, y, z, child count) as bytes
//   W/4 float4: child refs
//   then the bytes lo.x[W] hi.x[W] lo.y[W] hi.y[W] lo.z[W] hi.z[W] (4-wide: 24 B + 8 B pad)
// Returns false if a box cannot be covered (the caller keeps full precision).
static float q_decode(float origin, int q, float scale) { return origin + (float)q * scale; }

static bool quantize_node(const std::vector<BNode> &tree, const int *ch, int n, const int *ref, int W,
                          float4 *dst) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int k = 0; k < n; ++k)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], tree[ch[k]].lo[a]);
      hi[a] = std::max(hi[a], tree[ch[k]].hi[a]);
    }
  float scale[3];
  int ebias[3];
  for (int a = 0; a < 3; ++a) {
    const double ext = (double)hi[a] - (double)lo[a];
    int e = -126;
    while (e < 127 && std::ldexp(254.0, e) < ext) ++e;  // extent within 254 steps: one step of margin
    scale[a] = std::ldexp(1.0f, e);
    ebias[a] = e + 127;
  }
  unsigned char qb[6][8];
  std::memset(qb, 0, sizeof qb);
  for (int k = 0; k < n; ++k) {
    const BNode &c = tree[ch[k]];
    for (int a = 0; a < 3; ++a) {
      double ql = std::floor(((double)c.lo[a] - (double)lo[a]) / scale[a]);
      double qh = std::ceil(((double)c.hi[a] - (double)lo[a]) / scale[a]);
      int il = (int)std::max(0.0, std::min(255.0, ql)), ih = (int)std::max(0.0, std::min(255.0, qh));
      while (il > 0 && q_decode(lo[a], il, scale[a]) > c.lo[a]) --il;
      while (ih < 255 && q_decode(lo[a], ih, scale[a]) < c.hi[a]) ++ih;
      if (q_decode(lo[a], il, scale[a]) > c.lo[a] || q_decode(lo[a], ih, scale[a]) < c.hi[a]) return false;
      qb[2 * a][k] = (unsigned char)il;
      qb[2 * a + 1][k] = (unsigned char)ih;
    }
  }
  uint32_t meta = (uint32_t)ebias[0] | (uint32_t)ebias[1] << 8 | (uint32_t)ebias[2] << 16 | (uint32_t)n << 24;
  float mf;
  std::memcpy(&mf, &meta, 4);
  dst[0] = make_float4(lo[0], lo[1], lo[2], mf);
  const int per = W / 4;
  for (int q = 0; q < per; ++q) {
    int4 l = make_int4(ref[4 * q], ref[4 * q + 1], ref[4 * q + 2], ref[4 * q + 3]);
    std::memcpy(&dst[1 + q], &l, sizeof(int4));
  }
  unsigned char bytes[48];
  std::memset(bytes, 0, sizeof bytes);
  for (int r = 0; r < 6; ++r)
    for (int k = 0; k < W; ++k) bytes[r * W + k] = qb[r][k];
  std::memcpy(&dst[1 + per], bytes, (size_t)(W == 8 ? 48 : 32));
  return true;
}

bool flatten_wide(const std::vector<BNode> &tree, int W, BvhOut &out, bool quantize = false) {
  struct WN {
    int ch[8];
    int n;
  };
  std::vector<WN> wn;
  std::vector<int> wmap(tree.size(), -1);
  int max_stack = 0;
  // iterative DFS over binary inner nodes that start a wide node
  struct Item {
    int b, stack_below;
  };
  std::vector<Item> todo;
  const bool root_leaf = tree[0].left < 0;
  if (root_leaf) {
    WN w{};
    w.n = 1;
    w.ch[0] = 0;
    wn.push_back(w);
  } else {
    todo.push_back({0, 0});
  }
  std::vector<std::pair<int, int>> order;  // (binary node, wide index) in creation order
  while (!todo.empty()) {
    const Item it = todo.back();
    todo.pop_back();
    WN w{};
    int ch[8] = {tree[it.b].left, tree[it.b].right};
    int n = 2;
    while (n < W) {
      int best = -1;
      double ba = -1.0;
      for (int k = 0; k < n; ++k) {
        if (tree[ch[k]].left < 0) continue;
        const double a = half_area(tree[ch[k]].lo, tree[ch[k]].hi);
        if (a > ba) { ba = a; best = k; }
      }
      if (best < 0) break;
      const int b = ch[best];
      ch[best] = tree[b].left;
      ch[n++] = tree[b].right;
    }
    w.n = n;
    for (int k = 0; k < n; ++k) w.ch[k] = ch[k];
    const int me = (int)wn.size();
    wn.push_back(w);
    wmap[it.b] = me;
    const int need = it.stack_below + (n - 1);
    max_stack = std::max(max_stack, need);
    for (int k = n - 1; k >= 0; --k)
      if (tree[ch[k]].left >= 0) todo.push_back({ch[k], need});
  }
  if (max_stack > kWideStack) return false;
  if (quantize) {
    const int F = node_float4s(W, true);
    std::vector<float4> nodes((size_t)F * wn.size());
    for (size_t i = 0; i < wn.size(); ++i) {
      int ref[8];
      for (int k = 0; k < 8; ++k) ref[k] = leaf_code(0, 1);
      for (int k = 0; k < wn[i].n; ++k) {
        const BNode &c = tree[wn[i].ch[k]];
        ref[k] = c.left >= 0 ? wmap[wn[i].ch[k]] : leaf_code(c.first, c.count);
      }
      if (!quantize_node(tree, wn[i].ch, wn[i].n, ref, W, nodes.data() + (size_t)F * i)) return false;
    }
    out.node2.swap(nodes);
    out.width = W;
    out.quantized = true;
    out.stack_need = max_stack;
    return true;
  }
  const int F = node_float4s(W);
  std::vector<float4> nodes((size_t)F * wn.size());
  const float qnan = std::nanf("");
  for (size_t i = 0; i < wn.size(); ++i) {
    float row[6][8];
    int ref[8];
    for (int k = 0; k < 8; ++k) {
      for (int r = 0; r < 6; ++r) row[r][k] = qnan;
      ref[k] = leaf_code(0, 1);
    }
    for (int k = 0; k < wn[i].n; ++k) {
      const BNode &c = tree[wn[i].ch[k]];
      row[0][k] = c.lo[0]; row[1][k] = c.hi[0];
      row[2][k] = c.lo[1]; row[3][k] = c.hi[1];
      row[4][k] = c.lo[2]; row[5][k] = c.hi[2];
      ref[k] = c.left >= 0 ? wmap[wn[i].ch[k]] : leaf_code(c.first, c.count);
    }
    float4 *dst = nodes.data() + (size_t)F * i;
    const int per = W / 4;  // float4s per row
    for (int r = 0; r < 6; ++r)
      for (int q = 0; q < per; ++q) dst[r * per + q] = make_float4(row[r][4 * q], row[r][4 * q + 1], row[r][4 * q + 2], row[r][4 * q + 3]);
    for (int q = 0; q < per; ++q) {
      int4 l = make_int4(ref[4 * q], ref[4 * q + 1], ref[4 * q + 2], ref[4 * q + 3]);
      std::memcpy(&dst[6 * per + q], &l, sizeof(int4));
    }
  }
  out.node2.swap(nodes);
  out.width = W;
  out.stack_need = max_stack;
  return true;
}

// Flatten a preorder BNode tree into the device layout (two-child, or wide
// with `width` 4 or 8).  Returns false on a malformed tree.
bool flatten_two_child(std::vector<BNode> tree, const std::vector<Prim> &prims, const std::vector<int32_t> &perm,
                       BvhOut &out, std::string &err, int width = 2, bool quantize = false) {
  expand_big_leaves(tree, prims, perm);
  const int N = (int)tree.size();
  if (N == 0) {
    out.node2.clear();
    return true;
  }
  // number the inner nodes (depth-first, children in left/right order)
  std::vector<int> map(N, -1), depth(N, 0);
  std::vector<int> stack = {0};
  int inner = 0, leaves = 0, maxd = 0;
  std::vector<char> seen(N, 0);
  while (!stack.empty()) {
    const int i = stack.back();
    stack.pop_back();
    if (i < 0 || i >= N || seen[i]) {
      err = "BVH: malformed tree (bad or repeated child index)";
      return false;
    }
    seen[i] = 1;
    maxd = std::max(maxd, depth[i]);
    if (tree[i].left >= 0) {
      map[i] = inner++;
      const int l = tree[i].left, r = tree[i].right;
      if (l < 0 || l >= N || r < 0 || r >= N) {
        err = "BVH: child index out of range";
        return false;
      }
      depth[l] = depth[r] = depth[i] + 1;
      stack.push_back(r);
      stack.push_back(l);
    } else {
      ++leaves;
    }
  }
  if (maxd + 1 >= kStackDepth) {
    err = "BVH: tree depth " + std::to_string(maxd) + " exceeds the traversal stack";
    return false;
  }
  const bool root_leaf = tree[0].left < 0;
  const int nodes = root_leaf ? 1 : inner;
  out.node2.assign((size_t)4 * nodes, make_float4(0.f, 0.f, 0.f, 0.f));
  auto child_ref = [&](int c) { return tree[c].left >= 0 ? map[c] : leaf_code(tree[c].first, tree[c].count); };
  auto put = [&](int slot, int c0, int c1, bool c1_empty) {
    const BNode &A = tree[c0];
    const float nanf_ = std::nanf("");
    float b1[6];
    if (c1_empty) {
      for (float &x : b1) x = nanf_;
    } else {
      const BNode &Bn = tree[c1];
      b1[0] = Bn.lo[0]; b1[1] = Bn.hi[0]; b1[2] = Bn.lo[1]; b1[3] = Bn.hi[1]; b1[4] = Bn.lo[2]; b1[5] = Bn.hi[2];
    }
    out.node2[4 * slot + 0] = make_float4(A.lo[0], A.hi[0], A.lo[1], A.hi[1]);
    out.node2[4 * slot + 1] = make_float4(b1[0], b1[1], b1[2], b1[3]);
    out.node2[4 * slot + 2] = make_float4(A.lo[2], A.hi[2], b1[4], b1[5]);
    int4 link = make_int4(child_ref(c0), c1_empty ? child_ref(c0) : child_ref(c1), 0, 0);
    std::memcpy(&out.node2[4 * slot + 3], &link, sizeof(int4));
  };
  if (root_leaf) {
    put(0, 0, 0, true);
  } else {
    for (int i = 0; i < N; ++i)
      if (tree[i].left >= 0) put(map[i], tree[i].left, tree[i].right, false);
  }
  out.max_depth = maxd;
  out.leaves = leaves;
  out.width = 2;
  out.stack_need = maxd;
  // keeps the two-child layout if the wide one cannot be built
  if (width == 4 || width == 8)
    if (!flatten_wide(tree, width, out, quantize) && quantize) flatten_wide(tree, width, out, false);
  return true;
}

std::vector<Prim> make_prims(int T, const float *v0, const float *v1, const float *v2) {
  std::vector<Prim> prims(T);
  for (int t = 0; t < T; ++t) {
    Prim &q = prims[t];
    for (int a = 0; a < 3; ++a) {
      const float x = v0[3 * t + a], y = v1[3 * t + a], z = v2[3 * t + a];
      q.lo[a] = std::min(std::min(x, y), z);
      q.hi[a] = std::max(std::max(x, y), z);
      q.c[a] = ((x + y) + z) / 3.0f;
    }
  }
  return prims;
}

}  // namespace

bool build_bvh_binned(int T, const float *v0, const float *v1, const float *v2, const BvhParams &p, BvhOut &out,
                      std::string &err) {
  out = BvhOut{};
  if (T < 0 || T >= (1 << 27)) {
    err = "BVH: triangle count out of range (0 .. 2^27-1)";
    return false;
  }
  out.perm.resize(T);
  for (int i = 0; i < T; ++i) out.perm[i] = i;
  if (T == 0) return true;
  std::vector<Prim> prims = make_prims(T, v0, v1, v2);
  Builder b{prims, out.perm, p};
  unsigned hw = p.threads > 0 ? (unsigned)p.threads : std::max(1u, std::thread::hardware_concurrency());
  int par_levels = 0;
  while ((1u << par_levels) < hw && par_levels < 6) ++par_levels;
  std::vector<BNode> tree = b.task(0, T, 0, par_levels);
  // reference layout: same preorder numbering
  const int N = (int)tree.size();
  out.ref_min.resize(3 * (size_t)N);
  out.ref_max.resize(3 * (size_t)N);
  out.ref_link.resize(N);
  double cost = 0.0;
  const double root_area = half_area(tree[0].lo, tree[0].hi);
  for (int i = 0; i < N; ++i) {
    const BNode &nd = tree[i];
    for (int a = 0; a < 3; ++a) {
      out.ref_min[3 * i + a] = nd.lo[a];
      out.ref_max[3 * i + a] = nd.hi[a];
    }
    const double a = root_area > 0 ? half_area(nd.lo, nd.hi) / root_area : 1.0;
    if (nd.left >= 0) {
      out.ref_link[i] = make_int4(nd.left, nd.right, 0, 0);
      cost += p.cost_trav * a;
    } else {
      out.ref_link[i] = make_int4(-1, -1, nd.count, nd.first);
      cost += p.cost_tri * a * nd.count;
    }
  }
  out.sah_cost = cost;
  return flatten_two_child(std::move(tree), prims, out.perm, out, err, p.width, p.quantize);
}

bool bvh_from_reference(int T, const float *v0, const float *v1, const float *v2, int N, const float *nmin,
                        const float *nmax, const int32_t *left, const int32_t *right, const int32_t *ntris,
                        const int32_t *tstart, const int32_t *perm, BvhOut &out, std::string &err, int width,
                        bool quantize) {
  out = BvhOut{};
  if (T < 0 || T >= (1 << 27) || N < 0 || (T > 0 && N == 0)) {
    err = "BVH: bad triangle or node count";
    return false;
  }
  out.perm.assign(perm, perm + T);
  {
    std::vector<char> used(T, 0);
    for (int i = 0; i < T; ++i) {
      if (perm[i] < 0 || perm[i] >= T || used[perm[i]]) {
        err = "BVH: permutation is not a permutation of the triangles";
        return false;
      }
      used[perm[i]] = 1;
    }
  }
  if (T == 0) return true;
  std::vector<Prim> prims = make_prims(T, v0, v1, v2);
  std::vector<BNode> tree(N);
  out.ref_min.assign(nmin, nmin + 3 * (size_t)N);
  out.ref_max.assign(nmax, nmax + 3 * (size_t)N);
  out.ref_link.resize(N);
  for (int i = 0; i < N; ++i) {
    BNode &b = tree[i];
    for (int a = 0; a < 3; ++a) {
      b.lo[a] = nmin[3 * i + a];
      b.hi[a] = nmax[3 * i + a];
    }
    if (ntris[i] > 0) {
      if (tstart[i] < 0 || tstart[i] + ntris[i] > T) {
        err = "BVH: leaf triangle range out of bounds";
        return false;
      }
      b.left = b.right = -1;
      b.first = tstart[i];
      b.count = ntris[i];
      out.ref_link[i] = make_int4(-1, -1, ntris[i], tstart[i]);
    } else {
      if (left[i] < 0 || left[i] >= N || right[i] < 0 || right[i] >= N) {
        err = "BVH: inner node child out of range";
        return false;
      }
      b.left = left[i];
      b.right = right[i];
      b.first = b.count = 0;
      out.ref_link[i] = make_int4(left[i], right[i], 0, 0);
    }
  }
  return flatten_two_child(std::move(tree), prims, out.perm, out, err, width, quantize);
}

}  // namespace ts
