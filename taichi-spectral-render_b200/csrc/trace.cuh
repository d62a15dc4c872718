// Closest-hit BVH traversal on the device.
//
// Semantics follow trace() in main.py:831-864 of the reference: a triangle is
// accepted when its Moller-Trumbore distance t satisfies EPSILON < t < best
// (strict, so the first-visited of two exactly equal distances wins), a box
// is entered when t_enter < t_exit && t_exit > 0 (main.py:797-805), and the
// miss distance is 1e9.  Box and triangle tests use one IEEE rounding per
// operation (no FMA contraction) so that distances are bit-identical to the
// CPU oracle's.
//
// trace_closest() is the fast path: two-child 64-byte nodes, nearest child
// first, and boxes whose entry distance lies beyond the current best hit (by
// a relative margin of 2^-16, far larger than the rounding error of the box
// and triangle distances) are skipped.  The reference never skips boxes, so
// the closest hit differs only where two triangles' distances tie within the
// margin -- the "near tie" case the parity tests count.
//
// trace_reference_order() walks the reference-layout node table exactly like
// the reference: explicit 64-entry stack, left pushed before right (so right
// is popped first), no distance culling.
#pragma once
#include <climits>

#include "common.cuh"

namespace ts {

struct Hit {
  float t, u, v;
  int slot;  // triangle slot (BVH order); -1 on miss
};

// intersect_triangle (main.py:807-829): returns t, or -1 on miss.
TS_D float tri_hit(float3 o, float3 d, float4 A, float4 E1, float4 E2, float eps, float &u, float &v) {
  const float3 e1 = xyz(E1), e2 = xyz(E2);
  const float3 p = xcross(d, e2);
  const float det = xdot(e1, p);
  if (!(fabsf(det) > 1e-8f)) return -1.f;
  const float inv_det = __frcp_rn(det);
  const float3 tv = xsub3(o, xyz(A));
  const float uu = xmul(xdot(tv, p), inv_det);
  if (!(uu >= 0.f && uu <= 1.f)) return -1.f;
  const float3 q = xcross(tv, e1);
  const float vv = xmul(xdot(d, q), inv_det);
  if (!(vv >= 0.f && xadd(uu, vv) <= 1.f)) return -1.f;
  const float tt = xmul(xdot(e2, q), inv_det);
  if (!(tt > eps)) return -1.f;
  u = uu;
  v = vv;
  return tt;
}

// slab test for one box; returns entry/exit distances
TS_D void box_hit(float lox, float hix, float loy, float hiy, float loz, float hiz, float3 o, float3 inv,
                  float &te, float &tx) {
  const float ax = xmul(xsub(lox, o.x), inv.x), bx = xmul(xsub(hix, o.x), inv.x);
  const float ay = xmul(xsub(loy, o.y), inv.y), by = xmul(xsub(hiy, o.y), inv.y);
  const float az = xmul(xsub(loz, o.z), inv.z), bz = xmul(xsub(hiz, o.z), inv.z);
  te = fmaxf(fminf(ax, bx), fmaxf(fminf(ay, by), fminf(az, bz)));
  tx = fminf(fmaxf(ax, bx), fminf(fmaxf(ay, by), fmaxf(az, bz)));
}

TS_D float cull_bound(float best) { return best + best * (1.0f / 65536.0f); }

// Work counters of one traversal (compiled out unless a kernel asks for them).
struct TraceCount {
  uint32_t nodes = 0, tris = 0;
};

// Resumable fast traversal.  The state lives in registers; the stack of
// (node, entry-distance bits) pairs is owned by the caller so that a lane can
// stop after a budget of steps and resume later (the persistent trace kernel
// refills idle lanes between budgets).
constexpr int kTravDone = -2147483647 - 1;  // never a leaf code: first slot < 2^27 - 1

struct Traversal {
  float3 o, d, inv;
  float tcull;
  Hit h;
  int node, sp;
};

// bound: distance beyond which hits do not matter to the caller.  Boxes past
// it are skipped; a hit beyond it may still be returned (callers treat such a
// hit like a miss), so results are the same as with bound = 1e9.
TS_D void trav_begin(const DevScene &s, Traversal &t, float3 o, float3 d, float bound) {
  t.o = o;
  t.d = d;
  t.inv = f3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
  t.h.t = 1e9f;
  t.h.u = t.h.v = 0.f;
  t.h.slot = -1;
  t.tcull = cull_bound(fminf(bound, 1e9f));
  t.node = s.num_nodes > 0 ? 0 : kTravDone;
  t.sp = 0;
}

// Advance by at most `budget` steps (one inner node, or one leaf and the pop
// that follows).  Returns true once the traversal has finished.
template <bool kCount = false>
TS_D bool trav_steps(const DevScene &s, Traversal &t, int2 *stack, float eps, int budget, uint32_t &errbits,
                     TraceCount *tc = nullptr) {
  for (int it = 0; it < budget; ++it) {
    if (t.node == kTravDone) return true;
    if (t.node >= 0) {
      const float4 *n = s.node + 4 * (size_t)t.node;
      if (kCount) tc->nodes++;
      const float4 a = __ldg(n + 0), b = __ldg(n + 1), c = __ldg(n + 2);
      const int4 l = __ldg(reinterpret_cast<const int4 *>(n) + 3);
      float e0, x0, e1, x1;
      box_hit(a.x, a.y, a.z, a.w, c.x, c.y, t.o, t.inv, e0, x0);
      box_hit(b.x, b.y, b.z, b.w, c.z, c.w, t.o, t.inv, e1, x1);
      const bool h0 = e0 < x0 && x0 > 0.f && e0 <= t.tcull;
      const bool h1 = e1 < x1 && x1 > 0.f && e1 <= t.tcull;
      if (h0 && h1) {
        int nr = l.x, fr = l.y;
        float fe = e1;
        if (e1 < e0) { nr = l.y; fr = l.x; fe = e0; }
        if (t.sp < kStackDepth) {
          stack[t.sp++] = make_int2(fr, __float_as_int(fe));
        } else {
          errbits |= kErrStackOverflow;
        }
        t.node = nr;
        continue;
      }
      if (h0) { t.node = l.x; continue; }
      if (h1) { t.node = l.y; continue; }
    } else {
      const int code = ~t.node;
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float tt = tri_hit(t.o, t.d, A, E1, E2, eps, u, v);
        if (tt > eps && tt < t.h.t) {
          t.h.t = tt;
          t.h.u = u;
          t.h.v = v;
          t.h.slot = first + i;
          t.tcull = fminf(t.tcull, cull_bound(tt));
        }
      }
    }
    // pop the next box that is still closer than the cull bound
    for (;;) {
      if (t.sp == 0) {
        t.node = kTravDone;
        return true;
      }
      const int2 e = stack[--t.sp];
      if (__int_as_float(e.y) <= t.tcull) {
        t.node = e.x;
        break;
      }
    }
  }
  return t.node == kTravDone;
}

// Speculative while-while traversal of the two-child layout (Aila & Laine,
// "Understanding the efficiency of ray traversal on GPUs", HPG 2009): a lane
// that reaches a leaf postpones it and keeps descending, and the warp tests
// leaves only once every active lane holds one (or has finished), so leaf
// tests and inner-node steps are not interleaved across the warp.  Same
// results as trav_steps.
template <bool kCount = false>
TS_D bool trav_steps_spec(const DevScene &s, Traversal &t, int2 *stack, float eps, int budget, uint32_t &errbits,
                          TraceCount *tc = nullptr) {
  int leaf = 0;  // postponed leaf code (< 0), or 0
  for (int it = 0; it < budget; ++it) {
    if (t.node == kTravDone && leaf == 0) return true;
    // ---- inner nodes
    while (t.node >= 0) {
      const float4 *n = s.node + 4 * (size_t)t.node;
      if (kCount) tc->nodes++;
      const float4 a = __ldg(n + 0), b = __ldg(n + 1), c = __ldg(n + 2);
      const int4 l = __ldg(reinterpret_cast<const int4 *>(n) + 3);
      float e0, x0, e1, x1;
      box_hit(a.x, a.y, a.z, a.w, c.x, c.y, t.o, t.inv, e0, x0);
      box_hit(b.x, b.y, b.z, b.w, c.z, c.w, t.o, t.inv, e1, x1);
      const bool h0 = e0 < x0 && x0 > 0.f && e0 <= t.tcull;
      const bool h1 = e1 < x1 && x1 > 0.f && e1 <= t.tcull;
      if (h0 && h1) {
        int nr = l.x, fr = l.y;
        float fe = e1;
        if (e1 < e0) { nr = l.y; fr = l.x; fe = e0; }
        if (t.sp < kStackDepth) stack[t.sp++] = make_int2(fr, __float_as_int(fe));
        else errbits |= kErrStackOverflow;
        t.node = nr;
      } else if (h0) {
        t.node = l.x;
      } else if (h1) {
        t.node = l.y;
      } else {
        t.node = kTravDone;
        while (t.sp > 0) {
          const int2 e = stack[--t.sp];
          if (__int_as_float(e.y) <= t.tcull) { t.node = e.x; break; }
        }
      }
      // postpone the first leaf found and keep descending from the stack
      if (t.node < 0 && t.node != kTravDone && leaf == 0) {
        leaf = t.node;
        t.node = kTravDone;
        while (t.sp > 0) {
          const int2 e = stack[--t.sp];
          if (__int_as_float(e.y) <= t.tcull) { t.node = e.x; break; }
        }
      }
      if (!__any_sync(__activemask(), leaf == 0)) break;
    }
    // ---- leaves
    for (;;) {
      int code = 0;
      if (leaf < 0) {
        code = ~leaf;
        leaf = 0;
      } else if (t.node < 0 && t.node != kTravDone) {
        code = ~t.node;
        t.node = kTravDone;
        while (t.sp > 0) {
          const int2 e = stack[--t.sp];
          if (__int_as_float(e.y) <= t.tcull) { t.node = e.x; break; }
        }
      } else {
        break;
      }
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float tt = tri_hit(t.o, t.d, A, E1, E2, eps, u, v);
        if (tt > eps && tt < t.h.t) {
          t.h.t = tt;
          t.h.u = u;
          t.h.v = v;
          t.h.slot = first + i;
          t.tcull = fminf(t.tcull, cull_bound(tt));
        }
      }
    }
    if (t.node == kTravDone && leaf == 0) return true;
  }
  return t.node == kTravDone && leaf == 0;
}

// ---- wide nodes (4 or 8 children) ---------------------------------------
template <int W>
TS_D void cswap(float *k, int *r, int i, int j) {
  if (k[j] < k[i]) {
    const float tk = k[i];
    k[i] = k[j];
    k[j] = tk;
    const int tr = r[i];
    r[i] = r[j];
    r[j] = tr;
  }
}

// Sort W (entry distance, link) pairs ascending (misses carry +inf):
// 5-comparator network for 4, Batcher's 19-comparator network for 8.
template <int W>
TS_D void sort_children(float *k, int *r) {
  if (W == 4) {
    cswap<W>(k, r, 0, 1); cswap<W>(k, r, 2, 3); cswap<W>(k, r, 0, 2); cswap<W>(k, r, 1, 3); cswap<W>(k, r, 1, 2);
  } else {
    cswap<W>(k, r, 0, 1); cswap<W>(k, r, 2, 3); cswap<W>(k, r, 4, 5); cswap<W>(k, r, 6, 7);
    cswap<W>(k, r, 0, 2); cswap<W>(k, r, 1, 3); cswap<W>(k, r, 4, 6); cswap<W>(k, r, 5, 7);
    cswap<W>(k, r, 1, 2); cswap<W>(k, r, 5, 6);
    cswap<W>(k, r, 0, 4); cswap<W>(k, r, 1, 5); cswap<W>(k, r, 2, 6); cswap<W>(k, r, 3, 7);
    cswap<W>(k, r, 2, 4); cswap<W>(k, r, 3, 5);
    cswap<W>(k, r, 1, 2); cswap<W>(k, r, 3, 4); cswap<W>(k, r, 5, 6);
  }
}

// Traversal stacks of (node, entry-distance bits): a plain per-lane array
// (local memory, kept in L1), or a short stack whose newest S entries of each
// lane sit in a shared-memory column laid out [entry][thread] -- consecutive
// threads, consecutive 8-byte words, so a warp touches no bank twice at any
// mix of depths -- with older entries spilled to the lane's local array.
TS_D void spush(int2 *st, Traversal &t, int2 e) { st[t.sp++] = e; }
TS_D int2 spop(int2 *st, Traversal &t) { return st[--t.sp]; }

template <int S>
struct ShortStack {
  static_assert((S & (S - 1)) == 0, "ring size must be a power of two");
  int2 *sm;    // shared: [S][stride] entries
  int2 *loc;   // local: entries by absolute position (the older ones)
  int stride;  // threads per block
  int lane;    // this thread's column
  int ins;     // top entries held in shared memory (0 after trav_begin)
};
template <int S>
TS_D void spush(ShortStack<S> &st, Traversal &t, int2 e) {
  const int pos = t.sp;
  if (st.ins > pos) st.ins = pos;  // a new traversal (trav_begin) emptied the stack
  if (st.ins == S) {  // ring full: the oldest shared entry moves to local memory
    const int old = pos - S;
    st.loc[old] = st.sm[(old & (S - 1)) * st.stride + st.lane];
    --st.ins;
  }
  st.sm[(pos & (S - 1)) * st.stride + st.lane] = e;
  ++st.ins;
  ++t.sp;
}
template <int S>
TS_D int2 spop(ShortStack<S> &st, Traversal &t) {
  const int pos = --t.sp;
  if (st.ins > 0) {
    --st.ins;
    return st.sm[(pos & (S - 1)) * st.stride + st.lane];
  }
  return st.loc[pos];
}

// Same contract as trav_steps, for the wide layout: the children a node's
// ray enters are sorted by entry distance; the nearest is visited next and
// the others are pushed (farthest first) with their entry distances.
template <int W, bool kCount = false, class Stk = int2 *>
TS_D bool trav_steps_wide(const DevScene &s, Traversal &t, Stk &stack, float eps, int budget, uint32_t &errbits,
                          TraceCount *tc = nullptr) {
  constexpr int P = W / 4;  // float4s per row
  for (int it = 0; it < budget; ++it) {
    if (t.node == kTravDone) return true;
    if (t.node >= 0) {
      const float4 *n = s.node + (size_t)(6 * P + P + (W == 4 ? 1 : 2)) * t.node;
      if (kCount) tc->nodes++;
      float row[6][W];
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int q = 0; q < P; ++q) {
          const float4 v = __ldg(n + r * P + q);
          row[r][4 * q + 0] = v.x; row[r][4 * q + 1] = v.y; row[r][4 * q + 2] = v.z; row[r][4 * q + 3] = v.w;
        }
      int ref[W];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const int4 l = __ldg(reinterpret_cast<const int4 *>(n + 6 * P + q));
        ref[4 * q + 0] = l.x; ref[4 * q + 1] = l.y; ref[4 * q + 2] = l.z; ref[4 * q + 3] = l.w;
      }
      float key[W];
      int nh = 0;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        float te, tx;
        box_hit(row[0][k], row[1][k], row[2][k], row[3][k], row[4][k], row[5][k], t.o, t.inv, te, tx);
        const bool h = te < tx && tx > 0.f && te <= t.tcull;
        key[k] = h ? te : INFINITY;
        nh += h;
      }
      if (nh > 0) {
        sort_children<W>(key, ref);
        if (t.sp + nh - 1 <= kWideStack) {
#pragma unroll
          for (int k = W - 1; k >= 1; --k)
            if (k < nh) spush(stack, t, make_int2(ref[k], __float_as_int(key[k])));
        } else {
          errbits |= kErrStackOverflow;
        }
        t.node = ref[0];
        continue;
      }
    } else {
      const int code = ~t.node;
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float tt = tri_hit(t.o, t.d, A, E1, E2, eps, u, v);
        if (tt > eps && tt < t.h.t) {
          t.h.t = tt;
          t.h.u = u;
          t.h.v = v;
          t.h.slot = first + i;
          t.tcull = fminf(t.tcull, cull_bound(tt));
        }
      }
    }
    for (;;) {
      if (t.sp == 0) {
        t.node = kTravDone;
        return true;
      }
      const int2 e = spop(stack, t);
      if (__int_as_float(e.y) <= t.tcull) {
        t.node = e.x;
        break;
      }
    }
  }
  return t.node == kTravDone;
}

// Speculative while-while traversal of the wide layout (Aila & Laine, HPG
// 2009, as trav_steps_spec does for two-child nodes): a lane that reaches a
// leaf postpones it and keeps descending; the warp tests leaves only once
// every active lane holds one (or has finished).  Same results as
// trav_steps_wide.
template <int W, bool kCount = false>
TS_D bool trav_steps_wide_spec(const DevScene &s, Traversal &t, int2 *stack, float eps, int budget,
                               uint32_t &errbits, TraceCount *tc = nullptr) {
  constexpr int P = W / 4;  // float4s per row
  int leaf = 0;             // postponed leaf code (< 0), or 0
  auto pop = [&]() {
    t.node = kTravDone;
    while (t.sp > 0) {
      const int2 e = stack[--t.sp];
      if (__int_as_float(e.y) <= t.tcull) {
        t.node = e.x;
        break;
      }
    }
  };
  for (int it = 0; it < budget; ++it) {
    if (t.node == kTravDone && leaf == 0) return true;
    // ---- inner nodes
    while (t.node >= 0) {
      const float4 *n = s.node + (size_t)(6 * P + P + (W == 4 ? 1 : 2)) * t.node;
      if (kCount) tc->nodes++;
      float row[6][W];
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int q = 0; q < P; ++q) {
          const float4 v = __ldg(n + r * P + q);
          row[r][4 * q + 0] = v.x; row[r][4 * q + 1] = v.y; row[r][4 * q + 2] = v.z; row[r][4 * q + 3] = v.w;
        }
      int ref[W];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const int4 l = __ldg(reinterpret_cast<const int4 *>(n + 6 * P + q));
        ref[4 * q + 0] = l.x; ref[4 * q + 1] = l.y; ref[4 * q + 2] = l.z; ref[4 * q + 3] = l.w;
      }
      float key[W];
      int nh = 0;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        float te, tx;
        box_hit(row[0][k], row[1][k], row[2][k], row[3][k], row[4][k], row[5][k], t.o, t.inv, te, tx);
        const bool h = te < tx && tx > 0.f && te <= t.tcull;
        key[k] = h ? te : INFINITY;
        nh += h;
      }
      if (nh > 0) {
        sort_children<W>(key, ref);
        if (t.sp + nh - 1 <= kWideStack) {
#pragma unroll
          for (int k = W - 1; k >= 1; --k)
            if (k < nh) stack[t.sp++] = make_int2(ref[k], __float_as_int(key[k]));
        } else {
          errbits |= kErrStackOverflow;
        }
        t.node = ref[0];
      } else {
        pop();
      }
      // postpone the first leaf found and keep descending from the stack
      if (t.node < 0 && t.node != kTravDone && leaf == 0) {
        leaf = t.node;
        pop();
      }
      if (!__any_sync(__activemask(), leaf == 0)) break;
    }
    // ---- leaves
    for (;;) {
      int code = 0;
      if (leaf < 0) {
        code = ~leaf;
        leaf = 0;
      } else if (t.node < 0 && t.node != kTravDone) {
        code = ~t.node;
        pop();
      } else {
        break;
      }
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float tt = tri_hit(t.o, t.d, A, E1, E2, eps, u, v);
        if (tt > eps && tt < t.h.t) {
          t.h.t = tt;
          t.h.u = u;
          t.h.v = v;
          t.h.slot = first + i;
          t.tcull = fminf(t.tcull, cull_bound(tt));
        }
      }
    }
    if (t.node == kTravDone && leaf == 0) return true;
  }
  return t.node == kTravDone && leaf == 0;
}

// ---- quantized wide nodes (layout ids 5: 4 children in 64 B, 9: 8 children in 96 B)
// float4 0 = (origin.xyz, biased scale exponents x, y, z and the child count as
// bytes); then the child refs; then the child boxes as bytes q per plane
// (lo.x hi.x lo.y hi.y lo.z hi.z, one byte per child) with bound = origin + q *
// 2^e, decoded with one IEEE multiply (exact) and one add.  The host rounded
// every byte outwards against exactly this decode, so a decoded box contains
// the exact one: the slab test accepts at least the rays the exact box would,
// entry distances are no larger, and culling stays conservative -- the
// closest hit is the same as with full-precision boxes.
template <int WQ, bool kCount = false>
TS_D bool trav_steps_q(const DevScene &s, Traversal &t, int2 *stack, float eps, int budget, uint32_t &errbits,
                       TraceCount *tc = nullptr) {
  constexpr int N = WQ == 9 ? 8 : 4;  // children per node
  constexpr int R = N / 4;            // float4s of refs (and 32-bit words per byte plane)
  constexpr int F = WQ == 9 ? 6 : 4;  // float4s per node
  for (int it = 0; it < budget; ++it) {
    if (t.node == kTravDone) return true;
    if (t.node >= 0) {
      const float4 *n = s.node + (size_t)F * t.node;
      if (kCount) tc->nodes++;
      const float4 h = __ldg(n);
      const uint32_t meta = __float_as_uint(h.w);
      const float sx = __uint_as_float((meta & 0xffu) << 23);
      const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
      const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
      const int nc = (int)(meta >> 24);
      int ref[N];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int4 l = __ldg(reinterpret_cast<const int4 *>(n + 1 + q));
        ref[4 * q + 0] = l.x; ref[4 * q + 1] = l.y; ref[4 * q + 2] = l.z; ref[4 * q + 3] = l.w;
      }
      uint32_t wq[6 * R];  // plane r, children 4j..4j+3 in word r * R + j
      {
        const uint4 *b = reinterpret_cast<const uint4 *>(n + 1 + R);
#pragma unroll
        for (int i = 0; i < (6 * R + 3) / 4; ++i) {
          const uint4 v = __ldg(b + i);
          if (4 * i + 0 < 6 * R) wq[4 * i + 0] = v.x;
          if (4 * i + 1 < 6 * R) wq[4 * i + 1] = v.y;
          if (4 * i + 2 < 6 * R) wq[4 * i + 2] = v.z;
          if (4 * i + 3 < 6 * R) wq[4 * i + 3] = v.w;
        }
      }
      float key[N];
      int nh = 0;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const int j = k >> 2, sh = 8 * (k & 3);
        const float lox = xadd(h.x, xmul((float)((wq[0 * R + j] >> sh) & 0xffu), sx));
        const float hix = xadd(h.x, xmul((float)((wq[1 * R + j] >> sh) & 0xffu), sx));
        const float loy = xadd(h.y, xmul((float)((wq[2 * R + j] >> sh) & 0xffu), sy));
        const float hiy = xadd(h.y, xmul((float)((wq[3 * R + j] >> sh) & 0xffu), sy));
        const float loz = xadd(h.z, xmul((float)((wq[4 * R + j] >> sh) & 0xffu), sz));
        const float hiz = xadd(h.z, xmul((float)((wq[5 * R + j] >> sh) & 0xffu), sz));
        float te, tx;
        box_hit(lox, hix, loy, hiy, loz, hiz, t.o, t.inv, te, tx);
        const bool hit = k < nc && te < tx && tx > 0.f && te <= t.tcull;
        key[k] = hit ? te : INFINITY;
        nh += hit;
      }
      if (nh > 0) {
        sort_children<N>(key, ref);
        if (t.sp + nh - 1 <= kWideStack) {
#pragma unroll
          for (int k = N - 1; k >= 1; --k)
            if (k < nh) stack[t.sp++] = make_int2(ref[k], __float_as_int(key[k]));
        } else {
          errbits |= kErrStackOverflow;
        }
        t.node = ref[0];
        continue;
      }
    } else {
      const int code = ~t.node;
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float tt = tri_hit(t.o, t.d, A, E1, E2, eps, u, v);
        if (tt > eps && tt < t.h.t) {
          t.h.t = tt;
          t.h.u = u;
          t.h.v = v;
          t.h.slot = first + i;
          t.tcull = fminf(t.tcull, cull_bound(tt));
        }
      }
    }
    for (;;) {
      if (t.sp == 0) {
        t.node = kTravDone;
        return true;
      }
      const int2 e = stack[--t.sp];
      if (__int_as_float(e.y) <= t.tcull) {
        t.node = e.x;
        break;
      }
    }
  }
  return t.node == kTravDone;
}

// Dispatch on the node layout (a compile-time choice of each kernel instance).
// W = 2: two-child if-if loop; W = 3: two-child speculative while-while (same
// layout); W = 4 / 8: wide nodes; W = 5 / 9: quantized 4- / 8-wide nodes.
template <int W, bool kCount = false>
TS_D bool trav_advance(const DevScene &s, Traversal &t, int2 *stack, float eps, int budget, uint32_t &errbits,
                       TraceCount *tc = nullptr) {
  if (W == 2) return trav_steps<kCount>(s, t, stack, eps, budget, errbits, tc);
  if (W == 3) return trav_steps_spec<kCount>(s, t, stack, eps, budget, errbits, tc);
  if (W == 5 || W == 9) return trav_steps_q<W, kCount>(s, t, stack, eps, budget, errbits, tc);
#ifdef TS_WIDE_SPECULATIVE
  return trav_steps_wide_spec<W, kCount>(s, t, stack, eps, budget, errbits, tc);
#else
  return trav_steps_wide<W, kCount>(s, t, stack, eps, budget, errbits, tc);
#endif
}

template <int W>
struct StackSize {
  static constexpr int value = W <= 3 ? kStackDepth : kWideStack;
};

// Fast closest hit in one go (local-memory stack).  errbits gets
// kErrStackOverflow if the tree is deeper than the stack (the builder bounds
// the depth below it, so this is a guard only).
// Not inlined: one copy of the traversal per kernel instead of one per call
// site keeps the megakernels' instruction footprint small (instruction-fetch
// stalls dominated them when inlined).
template <int W, bool kCount = false>
__device__ __noinline__ Hit trace_closest(const DevScene &s, float3 o, float3 d, float eps, uint32_t &errbits,
                                          TraceCount *tc = nullptr, float bound = 1e9f) {
  Traversal t;
  int2 stack[StackSize<W>::value];
  trav_begin(s, t, o, d, bound);
  trav_advance<W, kCount>(s, t, stack, eps, 0x7fffffff, errbits, tc);
  return t.h;
}

// Exact reference-order closest hit on the reference-layout table.
TS_D Hit trace_reference_order(const DevScene &s, float3 o, float3 d, float eps, uint32_t &errbits) {
  Hit h;
  h.t = 1e9f;
  h.u = h.v = 0.f;
  h.slot = -1;
  if (s.num_ref_nodes <= 0) return h;
  const float3 inv = f3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
  int stack[kStackDepth];
  int sp = 1;
  stack[0] = 0;
  while (sp > 0) {
    const int ni = stack[--sp];
    float te, tx;
    const float *mn = s.ref_min + 3 * (size_t)ni;
    const float *mx = s.ref_max + 3 * (size_t)ni;
    box_hit(mn[0], mx[0], mn[1], mx[1], mn[2], mx[2], o, inv, te, tx);
    if (!(te < tx && tx > 0.f)) continue;
    const int4 l = s.ref_link[ni];
    if (l.z > 0) {
      for (int i = 0; i < l.z; ++i) {
        const int slot = l.w + i;
        const float4 *tp = s.tri + 3 * (size_t)slot;
        float u, v;
        const float t = tri_hit(o, d, tp[0], tp[1], tp[2], eps, u, v);
        if (t > eps && t < h.t) {
          h.t = t;
          h.u = u;
          h.v = v;
          h.slot = slot;
        }
      }
    } else {
      if (sp + 2 > kStackDepth) {
        errbits |= kErrStackOverflow;
        continue;
      }
      stack[sp++] = l.x;
      stack[sp++] = l.y;
    }
  }
  return h;
}

// Hit-record completion (main.py:860-863): geometric normal, interpolated
// shading normal, front-face flag, material.
struct SurfaceInfo {
  float3 ng, ns;
  int front, mat;
};
TS_D SurfaceInfo surface_info(const DevScene &s, const Hit &h, float3 d) {
  SurfaceInfo r;
  const float4 s0 = __ldg(s.shade + 3 * (size_t)h.slot + 0);
  const float4 s1 = __ldg(s.shade + 3 * (size_t)h.slot + 1);
  const float4 s2 = __ldg(s.shade + 3 * (size_t)h.slot + 2);
  r.ng = f3(s0.w, s1.w, s2.w);
  const float w = 1.0f - h.u - h.v;
  r.ns = normalize(w * xyz(s0) + h.u * xyz(s1) + h.v * xyz(s2));
  r.front = dot(d, r.ng) < 0.f ? 1 : 0;
  r.mat = __float_as_int(__ldg(s.tri + 3 * (size_t)h.slot + 1).w);
  return r;
}

}  // namespace ts
