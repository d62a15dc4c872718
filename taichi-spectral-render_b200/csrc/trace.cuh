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

// Fast closest hit.  stack: kStackDepth entries of (node, entry-distance bits)
// in local memory.  errbits gets kErrStackOverflow if the tree is deeper than
// the stack (the builder caps depth below it, so this is a guard only).
template <bool kCount = false>
TS_D Hit trace_closest(const DevScene &s, float3 o, float3 d, float eps, uint32_t &errbits, TraceCount *tc = nullptr) {
  Hit h;
  h.t = 1e9f;
  h.u = h.v = 0.f;
  h.slot = -1;
  if (s.num_nodes <= 0) return h;
  const float3 inv = f3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
  int2 stack[kStackDepth];
  int sp = 0;
  int node = 0;
  float tcull = cull_bound(h.t);
  for (;;) {
    if (node >= 0) {
      const float4 *n = s.node + 4 * (size_t)node;
      if (kCount) tc->nodes++;
      const float4 a = __ldg(n + 0), b = __ldg(n + 1), c = __ldg(n + 2);
      const int4 l = __ldg(reinterpret_cast<const int4 *>(n) + 3);
      float e0, x0, e1, x1;
      box_hit(a.x, a.y, a.z, a.w, c.x, c.y, o, inv, e0, x0);
      box_hit(b.x, b.y, b.z, b.w, c.z, c.w, o, inv, e1, x1);
      const bool h0 = e0 < x0 && x0 > 0.f && e0 <= tcull;
      const bool h1 = e1 < x1 && x1 > 0.f && e1 <= tcull;
      if (h0 && h1) {
        int nr = l.x, fr = l.y;
        float fe = e1;
        if (e1 < e0) { nr = l.y; fr = l.x; fe = e0; }
        if (sp < kStackDepth) {
          stack[sp++] = make_int2(fr, __float_as_int(fe));
        } else {
          errbits |= kErrStackOverflow;
        }
        node = nr;
        continue;
      }
      if (h0) { node = l.x; continue; }
      if (h1) { node = l.y; continue; }
    } else {
      const int code = ~node;
      const int first = code >> 4;
      const int cnt = (code & 15) + 1;
      if (kCount) tc->tris += cnt;
      for (int i = 0; i < cnt; ++i) {
        const float4 *tp = s.tri + 3 * (size_t)(first + i);
        const float4 A = __ldg(tp + 0), E1 = __ldg(tp + 1), E2 = __ldg(tp + 2);
        float u, v;
        const float t = tri_hit(o, d, A, E1, E2, eps, u, v);
        if (t > eps && t < h.t) {
          h.t = t;
          h.u = u;
          h.v = v;
          h.slot = first + i;
          tcull = cull_bound(t);
        }
      }
    }
    // pop the next box that is still closer than the best hit
    for (;;) {
      if (sp == 0) return h;
      const int2 e = stack[--sp];
      if (__int_as_float(e.y) <= tcull) { node = e.x; break; }
    }
  }
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
