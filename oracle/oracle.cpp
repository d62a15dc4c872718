// CPU oracle for the spectral path-tracing hot path -- TEST INFRASTRUCTURE ONLY.
//
// A line-by-line restatement of the reference estimator
// (Xyzonox/taichi-spectral-render main.py:682-1629), templated on the scalar
// type so that one source gives the FP32 checker (built with
// -ffp-contract=off, IEEE per operation) and the FP64 converged-image oracle.
// Only the tests, the package smoke check and bench.py's CPU-baseline leg use
// it; the product never links it.  See oracle.h for the parity status.
//
// One deliberate departure from the reference: a path whose throughput has
// become exactly zero is ended (see render_pixel); the reference keeps
// tracing it, which changes nothing except that 0 * NaN from a later
// degenerate event can poison the pixel.
//
// The reference draws its random numbers from Taichi's ti.random(); here each
// path owns a Philox-4x32-10 stream keyed (seed, pass) with counter
// (pixel, draw/4, scene, 0), consumed in the reference's draw order, so the
// GPU renderer can replay exactly the same sample sequence.

#include "oracle.h"

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using std::acos;
using std::cos;
using std::exp;
using std::fabs;
using std::fmax;
using std::fmin;
using std::log;
using std::max;
using std::min;
using std::sin;
using std::sqrt;
using std::tan;

// ---------------------------------------------------------------- forward-mode duals
// The adjoint oracle instantiates the estimator with Dual<double, kDualN>: a
// value and its partial derivatives with respect to up to kDualN selected
// material / EEM parameters.  Branches compare values only, so the value part
// follows the FP64 estimator operation for operation.
constexpr int kDualN = 16;
template <class T, int K> struct Dual {
  T v;
  T d[K];
  Dual() : v(0) { for (int i = 0; i < K; ++i) d[i] = 0; }
  template <class S, class = typename std::enable_if<std::is_arithmetic<S>::value>::type>
  Dual(S x) : v(T(x)) { for (int i = 0; i < K; ++i) d[i] = 0; }
  explicit operator double() const { return double(v); }
  explicit operator float() const { return float(v); }
  friend Dual operator+(const Dual &a, const Dual &b) {
    Dual r; r.v = a.v + b.v; for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i]; return r;
  }
  friend Dual operator-(const Dual &a, const Dual &b) {
    Dual r; r.v = a.v - b.v; for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i]; return r;
  }
  friend Dual operator-(const Dual &a) {
    Dual r; r.v = -a.v; for (int i = 0; i < K; ++i) r.d[i] = -a.d[i]; return r;
  }
  friend Dual operator*(const Dual &a, const Dual &b) {
    Dual r; r.v = a.v * b.v; for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r;
  }
  friend Dual operator/(const Dual &a, const Dual &b) {
    Dual r; r.v = a.v / b.v; for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v; return r;
  }
  Dual &operator+=(const Dual &b) { return *this = *this + b; }
  Dual &operator-=(const Dual &b) { return *this = *this - b; }
  Dual &operator*=(const Dual &b) { return *this = *this * b; }
  friend bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
  friend bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
  friend bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
  friend bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
  friend bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
  friend bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }
  // chain rule for a unary function with value fv and derivative df at a.v
  static Dual chain(const Dual &a, T fv, T df) {
    Dual r; r.v = fv; for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * df; return r;
  }
  friend Dual sqrt(const Dual &a) {
    const T r = std::sqrt(a.v);
    return chain(a, r, r > T(0) ? T(0.5) / r : T(0));
  }
  friend Dual exp(const Dual &a) { const T e = std::exp(a.v); return chain(a, e, e); }
  friend Dual log(const Dual &a) { return chain(a, std::log(a.v), T(1) / a.v); }
  friend Dual acos(const Dual &a) {
    const T q = T(1) - a.v * a.v;
    return chain(a, std::acos(a.v), q > T(0) ? -T(1) / std::sqrt(q) : T(0));
  }
  friend Dual cos(const Dual &a) { return chain(a, std::cos(a.v), -std::sin(a.v)); }
  friend Dual sin(const Dual &a) { return chain(a, std::sin(a.v), std::cos(a.v)); }
  friend Dual tan(const Dual &a) { const T t = std::tan(a.v); return chain(a, t, T(1) + t * t); }
  friend Dual fabs(const Dual &a) { return a.v < T(0) ? -a : a; }
  friend Dual max(const Dual &a, const Dual &b) { return a < b ? b : a; }
  friend Dual min(const Dual &a, const Dual &b) { return b < a ? b : a; }
  friend Dual fmax(const Dual &a, const Dual &b) { return (b.v > a.v || a.v != a.v) ? b : a; }
  friend Dual fmin(const Dual &a, const Dual &b) { return (b.v < a.v || a.v != a.v) ? b : a; }
};
template <class R> struct is_dual : std::false_type {};
template <class T, int K> struct is_dual<Dual<T, K>> : std::true_type {};

// A sampled value enters the estimator as a fixed number: its dependence on
// the parameters is accounted for by the score of its density instead.
template <class R> inline R detach(const R &a) {
  if constexpr (is_dual<R>::value) return R(a.v);
  else return a;
}
// Score factor of a sampling decision with probability (density) p: value
// exactly 1, derivative d log p.  Multiplied into the estimate of the event,
// it adds d log p times every later deposit.  Plain types: no factor at all.
template <class R> inline void apply_score(R &est, const R &p) {
  if constexpr (is_dual<R>::value) {
    if (!(p.v > 0)) return;
    R s(1.0);
    for (int i = 0; i < kDualN; ++i) s.d[i] = p.d[i] / p.v;
    est = est * s;
  } else {
    (void)est;
    (void)p;
  }
}

// ---------------------------------------------------------------- Philox
inline void philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

struct Rng {
  uint32_t key[2];
  uint32_t pix, scene, n = 0;
  uint32_t buf[4];
  // function-level checks replay a given list of draws instead (0.5 past its end;
  // the caller compares the count consumed)
  const float *fixed = nullptr;
  uint32_t nfixed = 0;
  Rng(uint32_t seed, uint32_t pass, uint32_t pixel, uint32_t scene_id)
      : pix(pixel), scene(scene_id) { key[0] = seed; key[1] = pass; }
  // uniform in [0, 1) with 24 random bits (exactly representable in f32)
  float next() {
    if (fixed) {
      const float v = n < nfixed ? fixed[n] : 0.5f;
      ++n;
      return v;
    }
    if ((n & 3u) == 0) {
      const uint32_t c[4] = {pix, n >> 2, scene, 0u};
      philox_block(c, key, buf);
    }
    const uint32_t x = buf[n & 3u];
    ++n;
    return (float)(x >> 8) * (1.0f / 16777216.0f);
  }
};

// ---------------------------------------------------------------- vectors
template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> mk(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R norm(V3<R> a) { return sqrt(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) { return a / norm(a); }
// GLSL reflect / refract as taichi.math defines them
template <class R> inline V3<R> reflect(V3<R> x, V3<R> n) { return x - (R(2) * dot(n, x)) * n; }
template <class R> inline V3<R> refract(V3<R> x, V3<R> n, R eta) {
  const R dxn = dot(x, n);
  const R k = R(1) - eta * eta * (R(1) - dxn * dxn);
  if (k >= R(0)) return eta * x - (eta * dxn + sqrt(k)) * n;
  return {R(0), R(0), R(0)};
}
template <class R> inline V3<R> load3(const float *p, int64_t i) {
  return {R(p[3 * i]), R(p[3 * i + 1]), R(p[3 * i + 2])};
}
template <class R> inline R clampr(R x, R lo, R hi) { return min(max(x, lo), hi); }
template <class R> inline V3<R> detach3(V3<R> a) { return {detach(a.x), detach(a.y), detach(a.z)}; }

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- scene view
template <class R> struct Ctx {
  const orc_scene *s;
  const orc_config *c;
  int B;
  R eps, escape;
  R lmin_m, step, lmin_nm;
  R pi, four_pi, two_pi;
  Ctx(const orc_scene *s_, const orc_config *c_) : s(s_), c(c_), B(c_->bands) {
    eps = R(c->epsilon);
    escape = R(c->escape);
    lmin_m = R(double(c->lambda_min_nm) * 1e-9);
    step = R(c->lambda_step_nm);
    lmin_nm = R(c->lambda_min_nm);
    pi = R(kPi);
    four_pi = R(4.0 * kPi);
    two_pi = R(2.0 * kPi);
  }
  // 4*pi*k / lambda[m] as scatter_volume / scatter_surface / shadow_transmittance
  // write it (main.py:1057, :1203, :1462)
  R absorb(R k, int band) const { return (four_pi * k) / (lmin_m + (R(band) * step) * R(1e-9)); }
  // the evaluate_bsdf form (main.py:1394): 4*pi*k*1e9 / lambda[nm]
  R absorb_nm(R k, int band) const { return (four_pi * k * R(1e9)) / (lmin_nm + R(band) * step); }
  // adjoint oracle: derivative slot of each parameter (-1 = not selected),
  // material table [M][6][B] then EEM [E][B][B]
  const int32_t *slot = nullptr;
  int64_t pmat = 0;
};

// A parameter value as the estimator reads it; the adjoint oracle seeds the
// derivative of a selected parameter with 1.
template <class R> inline R param(const Ctx<R> &x, float value, int64_t idx) {
  R r(value);
  if constexpr (is_dual<R>::value) {
    if (x.slot) {
      const int k = x.slot[idx];
      if (k >= 0) r.d[k] = 1.0;
    }
  }
  (void)x;
  (void)idx;
  return r;
}

template <class R> struct Mat {
  R n, k, rough, sigma_s, emission, g;
  int is_vol, surf_emis, eem;
};
// get_mat, main.py:980-996
template <class R> inline Mat<R> get_mat(const Ctx<R> &x, int m, int band) {
  const int B = x.B;
  const float *f = x.s->mat_f32 + (int64_t)m * 6 * B;
  const int32_t *i = x.s->mat_i32 + (int64_t)m * 2 * B;
  Mat<R> r;
  const int64_t base = (int64_t)m * 6 * B + band;
  r.n = param(x, f[0 * B + band], base + 0 * B);
  r.k = param(x, f[1 * B + band], base + 1 * B);
  r.rough = param(x, f[2 * B + band], base + 2 * B);
  r.sigma_s = param(x, f[3 * B + band], base + 3 * B);
  r.emission = param(x, f[4 * B + band], base + 4 * B);
  r.g = param(x, f[5 * B + band], base + 5 * B);
  r.is_vol = i[0 * B + band];
  r.surf_emis = i[1 * B + band];
  r.eem = x.s->mat_eem[m];
  return r;
}
template <class R> inline R eem_at(const Ctx<R> &x, int eem, int row, int col) {
  const int64_t i = ((int64_t)eem * x.B + row) * x.B + col;
  return param(x, x.s->eem[i], x.pmat + i);
}

// ---------------------------------------------------------------- sampling
// random_in_unit_sphere, main.py:682-687
template <class R> V3<R> random_in_unit_sphere(const Ctx<R> &x, Rng &rng) {
  const R z = R(rng.next()) * R(2) - R(1);
  const R rxy = sqrt(max(R(0), R(1) - z * z));
  const R phi = R(rng.next()) * R(2) * x.pi;
  return {rxy * cos(phi), rxy * sin(phi), z};
}
template <class R> inline void onb(V3<R> n, V3<R> &t, V3<R> &b) {
  const V3<R> up = fabs(n.y) < R(0.999) ? mk<R>(0, 1, 0) : mk<R>(1, 0, 0);
  t = normalize(cross(up, n));
  b = cross(n, t);
}
// cosine_weighted_hemisphere_direction, main.py:689-705
template <class R> V3<R> cosine_hemisphere(const Ctx<R> &x, V3<R> n, Rng &rng) {
  const R r1 = R(rng.next());
  const R r2 = R(rng.next());
  const R phi = x.two_pi * r1;
  const R ct = sqrt(R(1) - r2);
  const R st = sqrt(r2);
  V3<R> t, b;
  onb(n, t, b);
  return t * cos(phi) * st + b * sin(phi) * st + n * ct;
}
// evaluate_henyey_greenstein, main.py:758-766
template <class R> R hg_eval(const Ctx<R> &x, R cos_t, R g) {
  const R g2 = g * g;
  const R denom = R(1) + g2 - R(2) * g * cos_t;
  return (R(1) - g2) / (x.four_pi * denom * sqrt(denom) + R(1e-6));
}
// sample_henyey_greenstein, main.py:768-792
template <class R> V3<R> hg_sample(const Ctx<R> &x, V3<R> w, R g, Rng &rng, R *ct_out = nullptr) {
  R ct;
  if (fabs(g) < R(1e-4)) {
    ct = R(2) * R(rng.next()) - R(1);
  } else {
    const R rs = (R(1) - g * g) / (R(1) - g + R(2) * g * R(rng.next()));
    ct = (R(1) + g * g - rs * rs) / (R(2) * g);
  }
  if (ct_out) *ct_out = ct;
  const R st = sqrt(max(R(0), R(1) - ct * ct));
  const R phi = x.two_pi * R(rng.next());
  V3<R> u, v;
  onb(w, u, v);
  return u * cos(phi) * st + v * sin(phi) * st + w * ct;
}

// ---------------------------------------------------------------- intersection
// intersect_aabb, main.py:797-805 (fmin/fmax: NaN-ignoring, like the min/max of
// Taichi's backends)
template <class R> inline bool hit_aabb(V3<R> o, V3<R> inv, V3<R> mn, V3<R> mx) {
  const R ax = (mn.x - o.x) * inv.x, bx = (mx.x - o.x) * inv.x;
  const R ay = (mn.y - o.y) * inv.y, by = (mx.y - o.y) * inv.y;
  const R az = (mn.z - o.z) * inv.z, bz = (mx.z - o.z) * inv.z;
  const R te = fmax(fmin(ax, bx), fmax(fmin(ay, by), fmin(az, bz)));
  const R tx = fmin(fmax(ax, bx), fmin(fmax(ay, by), fmax(az, bz)));
  return te < tx && tx > R(0);
}
// intersect_triangle (Moller-Trumbore), main.py:807-829; returns t=-1 on miss
template <class R> inline void hit_tri(V3<R> o, V3<R> d, V3<R> v0, V3<R> e1, V3<R> e2, R eps,
                                       R &t, R &u, R &v) {
  t = R(-1); u = R(-1); v = R(-1);
  const V3<R> p = cross(d, e2);
  const R det = dot(e1, p);
  if (fabs(det) > R(1e-8)) {
    const R inv_det = R(1) / det;
    const V3<R> tv = o - v0;
    const R ut = dot(tv, p) * inv_det;
    if (ut >= R(0) && ut <= R(1)) {
      const V3<R> q = cross(tv, e1);
      const R vt = dot(d, q) * inv_det;
      if (vt >= R(0) && ut + vt <= R(1)) {
        const R tt = dot(e2, q) * inv_det;
        if (tt > eps) { t = tt; u = ut; v = vt; }
      }
    }
  }
}

template <class R> struct Hit {
  R t;
  V3<R> normal, shading_normal;
  int mat, is_hit, front, tri;
  R u, v;
};

// trace, main.py:831-864.  The reference keeps a 64-entry stack without a
// bound check; overflow is counted here instead.
template <class R> Hit<R> trace(const Ctx<R> &x, V3<R> pos, V3<R> dir, int64_t *overflow) {
  const orc_scene *s = x.s;
  Hit<R> h{};
  h.t = R(1e9);
  h.is_hit = 0;
  h.tri = -1;
  h.mat = 0;
  h.u = h.v = R(0);
  h.normal = h.shading_normal = mk<R>(0, 0, 0);
  h.front = 0;
  const V3<R> inv = {R(1) / dir.x, R(1) / dir.y, R(1) / dir.z};
  int stack[64];
  int sp = 1;
  stack[0] = 0;
  if (s->num_nodes <= 0) return h;
  while (sp > 0) {
    --sp;
    const int ni = stack[sp];
    if (!hit_aabb(pos, inv, load3<R>(s->node_min, ni), load3<R>(s->node_max, ni))) continue;
    const int nt = s->node_num_tris[ni];
    if (nt > 0) {
      const int t0 = s->node_tri_start[ni];
      for (int i = 0; i < nt; ++i) {
        const int ti = t0 + i;
        const V3<R> v0 = load3<R>(s->v0, ti);
        // e1/e2 are formed in the working precision from the stored vertices
        const V3<R> e1 = load3<R>(s->v1, ti) - v0;
        const V3<R> e2 = load3<R>(s->v2, ti) - v0;
        R t, u, v;
        hit_tri(pos, dir, v0, e1, e2, x.eps, t, u, v);
        if (t > x.eps && t < h.t) {
          h.is_hit = 1;
          h.t = t;
          h.mat = s->mat_id[ti];
          h.tri = ti;
          h.u = u;
          h.v = v;
        }
      }
    } else {
      if (sp + 2 > 64) { if (overflow) ++*overflow; continue; }
      stack[sp++] = s->node_left[ni];
      stack[sp++] = s->node_right[ni];
    }
  }
  if (h.is_hit) {
    h.normal = load3<R>(s->normal, h.tri);
    const R w = R(1) - h.u - h.v;
    h.shading_normal = normalize(w * load3<R>(s->n0, h.tri) + h.u * load3<R>(s->n1, h.tri) +
                                 h.v * load3<R>(s->n2, h.tri));
    h.front = dot(dir, h.normal) < R(0) ? 1 : 0;
  }
  return h;
}

// ---------------------------------------------------------------- Fresnel / GGX
template <class R> struct C2 { R re, im; };
template <class R> inline C2<R> cmul(C2<R> a, C2<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R> inline C2<R> cdiv(C2<R> a, C2<R> b) {  // main.py:874-880
  const C2<R> bc = {b.re, -b.im};
  const R m = b.re * b.re + b.im * b.im;
  const C2<R> p = cmul(a, bc);
  return {p.re / m, p.im / m};
}
template <class R> inline R cmod2(C2<R> a) { return a.re * a.re + a.im * a.im; }
template <class R> inline C2<R> csqrt(C2<R> z) {  // main.py:887-896
  const R mod = sqrt(z.re * z.re + z.im * z.im);
  const R re = sqrt((mod + z.re) / R(2));
  const R sg = z.im > R(0) ? R(1) : (z.im < R(0) ? R(-1) : R(0));
  R im = sg * sqrt((mod - z.re) / R(2));
  if (z.im == R(0)) im = R(0);
  return {re, im};
}
// fresnel_spectral, main.py:925-966
template <class R> R fresnel(R cos_i, R ni, R ki, R nt, R kt) {
  const R ang = acos(clampr(cos_i, R(-1), R(1)));
  const C2<R> e_in = {ni * ni - ki * ki, R(2) * ni * ki};
  const C2<R> e_tr = {nt * nt - kt * kt, R(2) * nt * kt};
  const R ct = cos(ang);
  const R s = sin(ang);
  const R s2 = s * s;
  C2<R> left = cmul(csqrt(e_in), C2<R>{ct, R(0)});
  const C2<R> es = cmul(e_in, C2<R>{s2, R(0)});
  C2<R> right = csqrt(C2<R>{e_tr.re - es.re, e_tr.im - es.im});
  const C2<R> rs = cdiv(C2<R>{left.re - right.re, left.im - right.im},
                        C2<R>{left.re + right.re, left.im + right.im});
  left = cmul(e_tr, left);
  right = cmul(e_in, right);
  const C2<R> rp = cdiv(C2<R>{left.re - right.re, left.im - right.im},
                        C2<R>{left.re + right.re, left.im + right.im});
  return R(0.5) * (cmod2(rs) + cmod2(rp));
}
// normaldistrobution_ggx, main.py:900-907 (alpha = roughness^2)
template <class R> inline R ggx_d(const Ctx<R> &x, R ndh, R rough) {
  const R a = rough * rough;
  const R a2 = a * a;
  const R d = ndh * ndh * (a2 - R(1)) + R(1);
  return a2 / (x.pi * d * d);
}
// geometry_smith_ggx, main.py:909-923
template <class R> inline R ggx_g(V3<R> n, V3<R> v, V3<R> l, R rough) {
  const R ndv = max(dot(n, v), R(0));
  R a = rough * rough;
  a = max(a, R(1e-4));
  const R k = a * a / R(2);
  const R gv = ndv / (ndv * (R(1) - k) + k + R(1e-7));
  const R ndl = max(dot(n, l), R(0));
  const R gl = ndl / (ndl * (R(1) - k) + k + R(1e-7));
  return gv * gl;
}
// importance_sample_ggx, main.py:968-978 (called with alpha = roughness)
template <class R> V3<R> ggx_sample(const Ctx<R> &x, R xi0, R xi1, V3<R> n, R alpha) {
  const R a2 = alpha * alpha;
  const R phi = x.two_pi * xi0;
  const R ct = sqrt((R(1) - xi1) / (R(1) + (a2 - R(1)) * xi1));
  const R st = sqrt(R(1) - ct * ct);
  V3<R> t, b;
  onb(n, t, b);
  return normalize(t * (cos(phi) * st) + b * (sin(phi) * st) + n * ct);
}

// ---------------------------------------------------------------- events
template <class R> struct Ray {
  V3<R> pos, dir;
  R thr;
  int active, transport, plen, term, vol;
  R spdf;
  int pen, refl;
};
template <class R> struct VolEvent {
  int action;
  R travel, est;
  V3<R> normal, snormal;
  int front, hit_mat, tri;
  V3<R> dir;
  int new_wl, pen;
};
template <class R> struct SurfEvent {
  int did_reflect;
  V3<R> dir;
  R est, pdf;
  int new_wl;
};

template <class R> inline R eem_row_max(const Ctx<R> &x, int eem, int row) {
  R q = R(0);
  for (int j = 0; j < x.B; ++j) {
    const R e = eem_at(x, eem, row, j);
    if (e > q) q = e;
  }
  return q;
}
template <class R> inline R eem_row_sum(const Ctx<R> &x, int eem, int row) {
  R norm = R(0);
  for (int j = 0; j < x.B; ++j) norm += eem_at(x, eem, row, j);
  return norm;
}
template <class R> inline int eem_pick(const Ctx<R> &x, int eem, int row, R xi) {
  R norm = R(0);
  for (int j = 0; j < x.B; ++j) norm += eem_at(x, eem, row, j);
  R cum = R(0);
  for (int j = 0; j < x.B; ++j) {
    cum += eem_at(x, eem, row, j) / norm;
    if (xi < cum) return j;
  }
  return row;
}

// scatter_surface, main.py:1000-1188
template <class R> SurfEvent<R> scatter_surface(const Ctx<R> &x, const Ray<R> &ray,
                                                const VolEvent<R> &ev, Rng &rng) {
  SurfEvent<R> r{};
  r.dir = mk<R>(0, 0, 0);
  const Mat<R> sm = get_mat(x, ev.hit_mat, ray.active);
  const Mat<R> vm = get_mat(x, ray.vol, ray.active);
  const V3<R> V = -ray.dir;
  const V3<R> N = ev.snormal;
  const R ni = vm.n, ki = vm.k, nt = sm.n, kt = sm.k;
  const R xi0 = R(rng.next());
  const R xi1 = R(rng.next());
  // the half vector is a sample: its density enters through its score
  const V3<R> H = detach3(ggx_sample(x, xi0, xi1, N, sm.rough));
  const R cin = max(R(1e-4), dot(V, H));
  const R F = fresnel(cin, ni, ki, nt, kt);
  const R pick = clampr(R(rng.next()), R(0), R(0.99));
  R sc(1.0);  // product of the score factors of this event (adjoint oracle only)
  if constexpr (is_dual<R>::value) {
    if (sm.rough > R(0)) {
      // sampler density a2 c / (pi (c^2 (a2 - 1) + 1)^2) with a2 = roughness^2; at the
      // sampled c, c^2 = (1 - xi1) / (1 + (a2 - 1) xi1), so d log p / d roughness =
      // (4 xi1 - 2) / roughness (the closed form avoids the cancellation near c = 1)
      R s(1.0);
      const auto k = (R(4) * xi1 - R(2)).v / sm.rough.v;
      for (int i = 0; i < kDualN; ++i) s.d[i] = sm.rough.d[i] * k;
      sc = sc * s;
    }
    if (pick < F) {
      if (F <= R(0.99)) apply_score(sc, F);
    } else {
      apply_score(sc, R(1) - F);
    }
  }
  auto glossy_reflect = [&](bool abs_cos) {
    const V3<R> L = reflect(ray.dir, H);
    if (sm.rough < R(0.008)) {
      r.dir = L; r.did_reflect = 1; r.est = F; r.pdf = R(1e9);
    } else {
      const R ndl = max(R(1e-4), dot(N, L));
      const R ndh = max(R(1e-4), dot(N, H));
      const R ndv = max(R(1e-4), dot(N, V));
      const R D = ggx_d(x, ndh, sm.rough);
      const R G = ggx_g(N, V, L, sm.rough);
      const R bsdf = (D * G * F) / (R(4) * ndl * ndv);
      const R pdf = (D * ndh) / (R(4) * cin);
      r.dir = L; r.did_reflect = 1;
      const R c = abs_cos ? fabs(dot(N, L)) : max(R(0), dot(N, L));
      r.est = (bsdf * c) / pdf;
      r.pdf = pdf;
    }
  };
  if (pick < F) {
    glossy_reflect(false);
  } else {
    R absorb = x.absorb(kt, ray.active);
    const R sig_t = sm.sigma_s + absorb + R(1e-6);
    const R dist = detach(-log(-R(rng.next()) + R(1) + R(1e-7)) / sig_t);
    if (!sm.is_vol) {
      r.did_reflect = 1;
      const V3<R> S = cosine_hemisphere(x, N, rng);
      const R ndl = max(R(1e-4), dot(N, S));
      const R ndv = max(R(1e-4), dot(N, V));
      const R albedo = sm.sigma_s / (sm.sigma_s + absorb + R(1e-6));
      const R sigma = sm.rough * x.pi / R(2);
      const R s2 = sigma * sigma;
      const R A = R(1) - s2 / (R(2) * (s2 + R(0.33)));
      const R Bc = R(0.45) * s2 / (s2 + R(0.09));
      const R th_i = acos(ndl), th_o = acos(ndv);
      const R al = max(th_i, th_o), be = min(th_i, th_o);
      R cphi = R(0);
      if (ndl > R(1e-4) && ndv > R(1e-4)) {
        const V3<R> pi_ = normalize(S - N * ndl);
        const V3<R> po = normalize(V - N * ndv);
        cphi = max(R(0), dot(pi_, po));
      }
      R bsdf = (R(1) - F) * (albedo / x.pi) * (A + Bc * cphi * sin(al) * tan(be));
      const R pdf = R(0.318309886184) * ndl;
      r.new_wl = ray.active;
      const int eem = sm.eem;
      if (eem > 0) {
        const R qy = eem_row_max(x, eem, ray.active);
        const R xi3 = R(rng.next());
        if (qy > R(0) && xi3 < qy) {
          const R xi4 = R(rng.next());
          const int nw = eem_pick(x, eem, ray.active, xi4);
          apply_score(sc, qy);
          apply_score(sc, eem_at(x, eem, ray.active, nw) / eem_row_sum(x, eem, ray.active));
          apply_score(sc, sig_t * exp(-sig_t * dist));  // the penetration distance is used now
          r.new_wl = nw;
          const Mat<R> smf = get_mat(x, ev.hit_mat, nw);
          absorb = x.absorb(smf.k, nw);
          bsdf *= exp(-absorb * dist);
        } else {
          apply_score(sc, R(1) - qy);
        }
      }
      r.est = (bsdf * ndl) / pdf;
      r.pdf = pdf;
      r.dir = S;
    } else {
      const R eta = ni / nt;
      const V3<R> T = refract(ray.dir, H, eta);
      if (dot(T, T) < R(1e-4)) {
        glossy_reflect(true);
      } else {
        r.did_reflect = 0;
        r.dir = T;
        if (sm.rough < R(0.0018)) {
          r.est = R(1) - F;
          r.pdf = R(1e9);
        } else {
          const R ldh = dot(T, H), vdh = dot(V, H);
          const R ndh = max(R(1e-4), dot(N, H));
          const R ndl = max(R(1e-4), fabs(dot(N, T)));
          const R ndv = max(R(1e-4), fabs(dot(N, V)));
          const R G = ggx_g(N, V, T, sm.rough);
          const R D = ggx_d(x, ndh, sm.rough);
          const R den = ni * vdh + nt * ldh;
          const R den2 = den * den;
          const R t1 = fabs(ldh * vdh) / (ndl * ndv);
          const R t2 = (nt * nt * (R(1) - F) * D * G) / den2;
          const R bsdf = t1 * t2;
          const R pdf = (D * ndh * (R(1) - F) * nt * nt * fabs(ldh)) / den2;
          r.est = (bsdf * ndl) / pdf;
          r.pdf = pdf;
        }
      }
    }
  }
  if constexpr (is_dual<R>::value) r.est = r.est * sc;
  return r;
}

// scatter_volume, main.py:1190-1292
template <class R> VolEvent<R> scatter_volume(const Ctx<R> &x, const Ray<R> &ray, Rng &rng,
                                              orc_stats *st) {
  VolEvent<R> r{};
  const Mat<R> vm = get_mat(x, ray.vol, ray.active);
  r.new_wl = ray.active;
  r.dir = ray.dir;
  r.pen = ray.pen;
  const R absorb = x.absorb(vm.k, ray.active);
  const R sig_t = vm.sigma_s + absorb + R(1e-6);
  // the free-flight distance is a sample: its density enters through its score
  const R dvol = detach(-log(-R(rng.next()) + R(1) - R(1e-7)) / sig_t);
  st->traces++;
  const Hit<R> hit = trace(x, ray.pos, ray.dir, &st->stack_overflow);
  const R dsurf = hit.t;
  R travel = R(-1);
  if (dsurf < x.escape) {
    travel = dsurf;
    r.pen = hit.tri;
    if (dvol + x.eps < travel) travel = dvol;
  }
  r.travel = travel;
  r.front = hit.front;
  const R f = R(hit.front);
  r.normal = hit.normal * f - hit.normal * (R(1) - f);
  r.snormal = hit.shading_normal * f - hit.shading_normal * (R(1) - f);
  const R T = exp(-(absorb + vm.sigma_s) * travel);
  const R emit = ((-T + R(1)) * vm.emission) / (absorb + R(1e-6));
  const R att = T + emit;
  if (travel == dsurf) {
    r.est = att / (R(1) + R(1e-6));
    r.action = 1;
    r.hit_mat = hit.mat;
    r.tri = hit.tri;
    // P(free flight >= d_surf - eps)
    apply_score(r.est, exp(-sig_t * detach(max(R(0), dsurf - x.eps))));
  } else if (travel >= R(0)) {
    r.hit_mat = -1;
    r.tri = -1;
    const R xe = R(rng.next());
    const R kind = absorb / (vm.sigma_s + absorb + R(1e-6));
    if (xe <= kind) {
      if (vm.eem > 0) {
        const R qy = eem_row_max(x, vm.eem, ray.active);
        const R xf = R(rng.next());
        if (qy > R(0) && xf < qy) {
          r.action = 3;
          const R x2 = R(rng.next());
          const int nw = eem_pick(x, vm.eem, ray.active, x2);
          r.new_wl = nw;
          r.dir = random_in_unit_sphere(x, rng);
          const R em2 = ((-(R(1) - T) + R(1)) * get_mat(x, ray.vol, nw).emission) / (absorb + R(1e-6));
          r.est = (R(1) - T) + em2;
          apply_score(r.est, qy);
          apply_score(r.est, eem_at(x, vm.eem, ray.active, nw) / eem_row_sum(x, vm.eem, ray.active));
        } else {
          r.est = att;
          apply_score(r.est, R(1) - qy);
        }
      } else {
        r.est = att / (R(1) + R(1e-6));
      }
      apply_score(r.est, kind);
    } else {
      r.action = 2;
      R ct(0.0);
      r.dir = detach3(hg_sample(x, ray.dir, vm.g, rng, &ct));
      r.est = att;
      apply_score(r.est, R(1) - kind);
      if (fabs(vm.g) >= R(1e-4)) {  // the HG density the sampler draws from (no 1e-6 term)
        const R g2 = vm.g * vm.g;
        const R c = detach(ct);
        const R den = R(1) + g2 - R(2) * vm.g * c;
        apply_score(r.est, (R(1) - g2) / (x.four_pi * den * sqrt(den)));
      }
    }
    apply_score(r.est, sig_t * exp(-sig_t * travel));  // free-flight density at the event
  }
  return r;
}

// evaluate_bsdf, main.py:1360-1444
template <class R> void evaluate_bsdf(const Ctx<R> &x, int vol, int surf, V3<R> V, V3<R> L, V3<R> N,
                                      int wl, R &bsdf, R &pdf) {
  const Mat<R> vm = get_mat(x, vol, wl);
  const Mat<R> sm = get_mat(x, surf, wl);
  const R ni = vm.n, ki = vm.k, nt = sm.n, kt = sm.k;
  const R ndl = max(R(1e-4), dot(N, L));
  const R ndv = max(R(1e-4), dot(N, V));
  const bool reflected = ndv * ndl > R(0);
  bsdf = R(0);
  pdf = R(0);
  if (reflected) {
    V3<R> H = normalize(V + L);
    if (dot(H, N) < R(0)) H = -H;
    const R vdh = max(R(1e-4), dot(V, H));
    const R F = fresnel(vdh, ni, ki, nt, kt);
    if (sm.rough > R(0.008)) {
      const R ndh = max(R(1e-4), dot(N, H));
      const R D = ggx_d(x, ndh, sm.rough);
      const R G = ggx_g(N, V, L, sm.rough);
      bsdf += (D * G * F) / (R(4) * ndl * ndv);
      pdf += (D * ndh * F) / (R(4) * vdh);
    }
    const R absorb = x.absorb_nm(kt, wl);
    const R albedo = sm.sigma_s / (sm.sigma_s + absorb + R(1e-6));
    const R sigma = sm.rough * x.pi / R(2);
    const R s2 = sigma * sigma;
    const R A = R(1) - s2 / (R(2) * (s2 + R(0.33)));
    const R Bc = R(0.45) * s2 / (s2 + R(0.09));
    const R th_i = acos(ndl), th_o = acos(ndv);
    const R al = max(th_i, th_o), be = min(th_i, th_o);
    R cphi = R(0);
    if (ndl > R(1e-4) && ndv > R(1e-4)) {
      const V3<R> pi_ = normalize(L - N * ndl);
      const V3<R> po = normalize(V - N * ndv);
      cphi = max(R(0), dot(pi_, po));
    }
    const R nv = R(1) - R(sm.is_vol);
    bsdf += (R(1) - F) * nv * (albedo / x.pi) * (A + Bc * cphi * sin(al) * tan(be));
    pdf += ndl * R(0.318309886184) * (R(1) - F) * nv;
  } else if (sm.rough > R(0.008)) {
    // transmission lobe; unreachable because both cosines are clamped to >= 1e-4
    V3<R> H = -normalize(V * ni + L * nt);
    if (dot(H, N) < R(0)) H = -H;
    const R vdh = dot(V, H), ldh = dot(L, H);
    const R ndh = max(R(1e-4), dot(N, H));
    if (vdh * ldh < R(0)) {
      const R F = fresnel(fabs(vdh), ni, ki, nt, kt);
      const R D = ggx_d(x, ndh, sm.rough);
      const R G = ggx_g(N, V, L, sm.rough);
      const R den = ni * vdh + nt * ldh;
      const R den2 = den * den;
      bsdf += (fabs(ldh * vdh) / fabs(ndl * ndv)) * ((nt * nt * (R(1) - F) * D * G) / den2);
      pdf += (D * ndh * (R(1) - F) * nt * nt * fabs(ldh)) / den2;
    }
  }
}

// shadow_transmittance, main.py:1446-1499.  The segment origin is always the
// shading point plus the LAST segment's length (current_pos never advances),
// exactly as the reference writes it.
template <class R> R shadow_transmittance(const Ctx<R> &x, V3<R> origin, V3<R> dir, R max_dist,
                                          int light_tri, int vol, int wl, orc_stats *st) {
  R total = R(1);
  R traveled = R(0);
  V3<R> pos = origin;
  int cur_vol = vol;
  for (int i = 0; i < x.c->scatter_bounces; ++i) {
    st->traces++;
    const Hit<R> hit = trace(x, pos, dir, &st->stack_overflow);
    const R dsurf = hit.t;
    const Mat<R> vm = get_mat(x, cur_vol, wl);
    const R absorb = x.absorb(vm.k, wl);
    total *= exp(-(absorb + vm.sigma_s) * hit.t);
    if (hit.t >= (max_dist - traveled) || hit.tri == light_tri) {
      total *= exp(-(absorb + vm.sigma_s) * (max_dist - traveled));
      break;
    }
    const Mat<R> sm = get_mat(x, hit.mat, wl);
    const R ni = vm.n;
    R nt = sm.n;
    if (!hit.front) nt = get_mat(x, 0, wl).n;
    const R f = R(hit.front);
    const V3<R> inc = hit.shading_normal * f - hit.shading_normal * (R(1) - f);
    const V3<R> T = refract(dir, inc, ni / nt);
    const R rt = (dot(dir, T) - R(1)) * R(37.9743);
    const R rt2 = rt * rt;
    const R angle = R(1) / (R(1) + rt2 * rt2 * (R(3) - R(2) * rt));
    total *= angle;
    if (total < R(1e-6) || !sm.is_vol) {
      total = R(0);
      break;
    }
    traveled += dsurf + x.eps;
    pos = origin + dir * (dsurf + x.eps);
    cur_vol = hit.mat * hit.front;
  }
  return total;
}

template <class R> struct Nee { R factor, emission, weight; };

// sample_direct_light, main.py:1296-1358
template <class R> Nee<R> sample_direct_light(const Ctx<R> &x, const Ray<R> &ray, V3<R> N, int surf,
                                              Rng &rng, orc_stats *st) {
  Nee<R> r{R(0), R(0), R(0)};
  const orc_scene *s = x.s;
  const int wl = ray.active;
  const int nl = s->num_lights[wl];
  if (nl <= 0) return r;
  const R xl = R(rng.next());
  int lt = 0;
  for (int i = 0; i < nl; ++i) {
    if (xl < R(s->light_cdf[(int64_t)wl * s->max_lights + i])) {
      lt = s->light_idx[(int64_t)wl * s->max_lights + i];
      break;
    }
  }
  R bx = R(rng.next());
  R by = R(rng.next());
  if (bx + by > R(1)) { bx = R(1) - bx; by = R(1) - by; }
  const V3<R> v0 = load3<R>(s->v0, lt);
  const V3<R> P = v0 + bx * (load3<R>(s->v1, lt) - v0) + by * (load3<R>(s->v2, lt) - v0);
  const V3<R> Ldir = normalize(P - ray.pos);
  const R dist = norm(P - ray.pos);
  const R T = shadow_transmittance(x, ray.pos, Ldir, dist, lt, ray.vol, wl, st);
  if (T > R(1e-6)) {
    const int lmat = s->mat_id[lt];
    const V3<R> ln = load3<R>(s->normal, lt);
    const R cosl = max(R(0), dot(ln, -Ldir));
    const R dsq = dist * dist;
    const R G = cosl / (dsq + R(1e-4));
    R bsdf, pdf, c;
    if (surf != -1) {
      c = max(R(0), dot(N, Ldir));
      evaluate_bsdf(x, ray.vol, surf, -ray.dir, Ldir, N, wl, bsdf, pdf);
    } else {
      c = max(R(0), dot(ray.dir, Ldir));
      bsdf = hg_eval(x, c, get_mat(x, ray.vol, wl).g);
      pdf = bsdf;
    }
    const R area = R(s->light_area[wl]);
    r.factor = bsdf * c * T * G * area;
    r.emission = get_mat(x, lmat, ray.transport).emission;
    const R pl = dsq / (max(R(1e-6), cosl) * area);
    r.weight = (pl * pl) / (pl * pl + pdf * pdf + R(1e-6));
  }
  return r;
}

// cast_rays body for one pixel, main.py:1502-1590
// Film deposit of the plain estimators: the value into the pixel's band.
struct FilmSink {
  double *acc;
  template <class R> void operator()(int band, const R &v) { acc[band] += double(v); }
};
// Adjoint oracle: the value into the film (if any) and w[band] * d value into grad.
struct GradSink {
  double *acc;
  const double *w;
  double *grad;
  int n;
  template <class R> void operator()(int band, const R &v) {
    if (acc) acc[band] += double(v.v);
    for (int i = 0; i < n; ++i) grad[i] += w[band] * double(v.d[i]);
  }
};

template <class R, class Sink> void render_pixel(const Ctx<R> &x, uint32_t pass, int band, int pid, Sink &sink,
                                                 orc_stats *st) {
  const orc_config *c = x.c;
  const orc_scene *s = x.s;
  const int W = c->width, Hh = c->height;
  const int i = pid % W, j = pid / W;
  Rng rng(c->seed, pass, (uint32_t)pid, c->scene_id);
  const R u = (R(i) + R(rng.next())) / R(W);
  const R v = (R(j) + R(rng.next())) / R(Hh);
  int active_px = band;
  const V3<R> cu = {R(s->cam_u[0]), R(s->cam_u[1]), R(s->cam_u[2])};
  const V3<R> cv = {R(s->cam_v[0]), R(s->cam_v[1]), R(s->cam_v[2])};
  const V3<R> cw = {R(s->cam_w[0]), R(s->cam_w[1]), R(s->cam_w[2])};
  const V3<R> co = {R(s->cam_origin[0]), R(s->cam_origin[1]), R(s->cam_origin[2])};
  const R fov = R(c->fov_scale);
  Ray<R> ray{};
  ray.dir = normalize(cu * ((u * R(2) - R(1)) * R(c->aspect_ratio) * fov) + cv * ((v * R(2) - R(1)) * fov) -
                      cw * R(2));
  ray.pos = co;
  ray.active = band;
  ray.transport = band;
  ray.vol = 0;
  ray.thr = R(1);
  ray.plen = 0;
  ray.term = 0;
  ray.spdf = R(1);
  ray.pen = 0;
  ray.refl = 0;
  st->paths++;
  for (int k = 0; k < c->max_path_length; ++k) {
    if (ray.term) break;
    R direct = R(0), indirect = R(0);
    const VolEvent<R> ev = scatter_volume(x, ray, rng, st);
    if (ev.travel < R(0)) break;
    st->vertices++;
    ray.pos = ray.pos + ray.dir * ev.travel;
    ray.thr *= ev.est;
    ray.pen = ev.pen;
    if (ev.action == 1) {
      const Mat<R> sm = get_mat(x, ev.hit_mat, ray.transport);
      if (sm.surf_emis) {
        const R dsq = ev.travel * ev.travel;
        const R cosl = max(R(0), dot(load3<R>(s->normal, ev.tri), -ray.dir));
        const R pl = (dsq * min(R(1), R(ray.plen))) /
                     (cosl * R(s->light_area[ray.active]) + R(1e-6));
        const R w = (ray.spdf * ray.spdf) / (pl * pl + ray.spdf * ray.spdf + R(1e-6));
        indirect = ray.thr * sm.emission * w;
        ray.term = 1;
      } else {
        const Nee<R> ne = sample_direct_light(x, ray, ev.snormal, ev.hit_mat, rng, st);
        direct = ray.thr * ne.emission * ne.factor * ne.weight;
        ray.plen++;
        const SurfEvent<R> se = scatter_surface(x, ray, ev, rng);
        ray.spdf = se.pdf;
        ray.dir = se.dir;
        ray.thr *= se.est;
        const R sgn = R(se.did_reflect) - (R(1) - R(se.did_reflect));
        ray.pos = ray.pos + ev.normal * x.eps * sgn;
        ray.vol = ev.hit_mat * ev.front * (1 - se.did_reflect) + ray.vol * se.did_reflect;
        ray.refl = se.did_reflect;
      }
    } else {
      const Nee<R> ne = sample_direct_light(x, ray, ev.snormal, ev.hit_mat, rng, st);
      direct = ray.thr * ne.emission * ne.factor * ne.weight;
      if (ev.action == 2) {
        ray.dir = ev.dir;
        ray.plen++;
      } else if (ev.action == 3) {
        ray.dir = ev.dir;
        ray.active = ev.new_wl;
        active_px = ray.active;
        ray.plen++;
      }
    }
    sink(active_px, indirect);
    sink(active_px, direct);
    // A path whose throughput is exactly zero can only deposit zeros from
    // here on -- or NaN, where a later degenerate event computes 0/0 (the
    // rough-dielectric exit of an index-matched interface does).  Such paths
    // end here, in the oracle and on the GPU alike.
    if (ray.thr == R(0)) break;
  }
}

template <class R>
void render_pass_t(const orc_scene *s, const orc_config *c, uint32_t pass, int band, const int32_t *pix,
                   int npix, double *out, int nthreads, orc_stats *stats) {
  const Ctx<R> x(s, c);
  orc_stats tot{0, 0, 0, 0};
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    orc_stats st{0, 0, 0, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int p = 0; p < npix; ++p) {
      FilmSink sink{out + (int64_t)p * c->bands};
      render_pixel(x, pass, band, pix[p], sink, &st);
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      tot.paths += st.paths;
      tot.vertices += st.vertices;
      tot.traces += st.traces;
      tot.stack_overflow += st.stack_overflow;
    }
  }
  if (stats) *stats = tot;
}

// Forward-mode adjoint of one pass for up to kDualN parameters at a time.
template <class T>
void adjoint_pass_t(const orc_scene *s, const orc_config *c, uint32_t pass, int band, const int32_t *pix, int npix,
                    const double *adj, int nparams, const int64_t *ids, double *grad, double *out, int nthreads) {
  using DR = Dual<T, kDualN>;
  const int B = c->bands;
  const int64_t pmat = (int64_t)s->num_materials * 6 * B;
  const int64_t ptot = pmat + (int64_t)s->num_eems * B * B;
  std::vector<int32_t> slot(ptot, -1);
  for (int p0 = 0; p0 < nparams; p0 += kDualN) {
    const int n = std::min(kDualN, nparams - p0);
    std::fill(slot.begin(), slot.end(), -1);
    for (int i = 0; i < n; ++i)
      if (ids[p0 + i] >= 0 && ids[p0 + i] < ptot) slot[ids[p0 + i]] = i;
    Ctx<DR> x(s, c);
    x.slot = slot.data();
    x.pmat = pmat;
    double *film = p0 == 0 ? out : nullptr;
#ifdef _OPENMP
    const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
      std::vector<double> g(n, 0.0);
      orc_stats st{0, 0, 0, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
      for (int p = 0; p < npix; ++p) {
        GradSink sink{film ? film + (int64_t)p * B : nullptr, adj + (int64_t)p * B, g.data(), n};
        render_pixel(x, pass, band, pix[p], sink, &st);
      }
#ifdef _OPENMP
#pragma omp critical
#endif
      for (int i = 0; i < n; ++i) grad[p0 + i] += g[i];
    }
  }
}

// ---------------------------------------------------------------- BVH sweep builder
struct SweepBuilder {
  int n;
  std::vector<float> cen[3], tmin[3], tmax[3];
  std::vector<float> nmin, nmax;
  std::vector<int> left, right, ntris, tstart, perm;
  int reorder = 0;

  static void pad(float mn[3], float mx[3]) {
    for (int a = 0; a < 3; ++a)
      if (mn[a] == mx[a]) { mn[a] = mn[a] - 1e-6f; mx[a] = mx[a] + 1e-6f; }
  }
  static float area(const float mn[3], const float mx[3]) {
    const float d0 = mx[0] - mn[0], d1 = mx[1] - mn[1], d2 = mx[2] - mn[2];
    return 2.0f * (d0 * d1 + d1 * d2 + d2 * d0);
  }
  void box_of(const std::vector<int> &idx, float mn[3], float mx[3]) const {
    for (int a = 0; a < 3; ++a) { mn[a] = INFINITY; mx[a] = -INFINITY; }
    for (int t : idx)
      for (int a = 0; a < 3; ++a) {
        mn[a] = std::min(mn[a], tmin[a][t]);
        mx[a] = std::max(mx[a], tmax[a][t]);
      }
    pad(mn, mx);
  }
  void make_leaf(int node, const std::vector<int> &idx) {
    tstart[node] = reorder;
    ntris[node] = (int)idx.size();
    left[node] = right[node] = -1;
    for (int t : idx) perm[reorder++] = t;
  }
  int build(std::vector<int> idx) {
    const int node = (int)ntris.size();
    nmin.resize(nmin.size() + 3);
    nmax.resize(nmax.size() + 3);
    left.push_back(-1); right.push_back(-1); ntris.push_back(0); tstart.push_back(0);
    float mn[3], mx[3];
    box_of(idx, mn, mx);
    std::copy(mn, mn + 3, &nmin[3 * node]);
    std::copy(mx, mx + 3, &nmax[3 * node]);
    const int m = (int)idx.size();
    if (m <= 10) { make_leaf(node, idx); return node; }
    int best_axis = -1, best_pos = -1;
    float best = INFINITY;
    const float parent = area(mn, mx);
    std::vector<int> sorted(idx);
    std::vector<float> pre(6 * m), suf(6 * m);
    for (int a = 0; a < 3; ++a) {
      sorted = idx;
      std::stable_sort(sorted.begin(), sorted.end(),
                       [&](int p, int q) { return cen[a][p] < cen[a][q]; });
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int i = 0; i < m; ++i) {
        for (int b = 0; b < 3; ++b) {
          lo[b] = std::min(lo[b], tmin[b][sorted[i]]);
          hi[b] = std::max(hi[b], tmax[b][sorted[i]]);
          pre[6 * i + b] = lo[b];
          pre[6 * i + 3 + b] = hi[b];
        }
      }
      for (int b = 0; b < 3; ++b) { lo[b] = INFINITY; hi[b] = -INFINITY; }
      for (int i = m - 1; i >= 0; --i) {
        for (int b = 0; b < 3; ++b) {
          lo[b] = std::min(lo[b], tmin[b][sorted[i]]);
          hi[b] = std::max(hi[b], tmax[b][sorted[i]]);
          suf[6 * i + b] = lo[b];
          suf[6 * i + 3 + b] = hi[b];
        }
      }
      for (int i = 1; i < m; ++i) {
        float lmn[3], lmx[3], rmn[3], rmx[3];
        for (int b = 0; b < 3; ++b) {
          lmn[b] = pre[6 * (i - 1) + b]; lmx[b] = pre[6 * (i - 1) + 3 + b];
          rmn[b] = suf[6 * i + b]; rmx[b] = suf[6 * i + 3 + b];
        }
        pad(lmn, lmx);
        pad(rmn, rmx);
        const float cost = (area(lmn, lmx) * (float)i + area(rmn, rmx) * (float)(m - i)) / parent;
        if (cost < best) { best = cost; best_axis = a; best_pos = i; }
      }
    }
    if (!(best < (float)m)) { make_leaf(node, idx); return node; }
    sorted = idx;
    std::stable_sort(sorted.begin(), sorted.end(),
                     [&](int p, int q) { return cen[best_axis][p] < cen[best_axis][q]; });
    std::vector<int> li(sorted.begin(), sorted.begin() + best_pos);
    std::vector<int> ri(sorted.begin() + best_pos, sorted.end());
    idx.clear();
    idx.shrink_to_fit();
    const int l = build(std::move(li));
    const int r = build(std::move(ri));
    left[node] = l;
    right[node] = r;
    ntris[node] = 0;
    return node;
  }
};

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  philox_block(ctr, key, out);
}

double orc_fresnel(double cos_i, double ni, double ki, double nt, double kt, int32_t use_double) {
  if (use_double) return fresnel<double>(cos_i, ni, ki, nt, kt);
  return fresnel<float>((float)cos_i, (float)ni, (float)ki, (float)nt, (float)kt);
}

double orc_ggx_d(double ndh, double rough, int32_t use_double) {
  orc_config c{};
  c.bands = 1;
  if (use_double) return ggx_d(Ctx<double>(nullptr, &c), ndh, rough);
  return ggx_d(Ctx<float>(nullptr, &c), (float)ndh, (float)rough);
}

double orc_hg_eval(double cos_t, double g, int32_t use_double) {
  orc_config c{};
  c.bands = 1;
  if (use_double) return hg_eval(Ctx<double>(nullptr, &c), cos_t, g);
  return hg_eval(Ctx<float>(nullptr, &c), (float)cos_t, (float)g);
}

void orc_trace(const orc_scene *s, const orc_config *c, const float *rays, int32_t n, int32_t *tri,
               float *t, float *u, float *v, int32_t use_double) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int i = 0; i < n; ++i) {
    const float *r = rays + 6 * (int64_t)i;
    if (use_double) {
      const Ctx<double> x(s, c);
      const Hit<double> h = trace(x, V3<double>{r[0], r[1], r[2]}, V3<double>{r[3], r[4], r[5]}, nullptr);
      tri[i] = h.tri; t[i] = (float)h.t; u[i] = (float)h.u; v[i] = (float)h.v;
    } else {
      const Ctx<float> x(s, c);
      const Hit<float> h = trace(x, V3<float>{r[0], r[1], r[2]}, V3<float>{r[3], r[4], r[5]}, nullptr);
      tri[i] = h.tri; t[i] = h.t; u[i] = h.u; v[i] = h.v;
    }
  }
}

void orc_trace_brute(const orc_scene *s, const orc_config *c, const float *rays, int32_t n, int32_t *tri,
                     float *t) {
  const float eps = c->epsilon;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int i = 0; i < n; ++i) {
    const float *r = rays + 6 * (int64_t)i;
    const V3<float> o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
    float best = 1e9f;
    int bi = -1;
    for (int k = 0; k < s->num_tris; ++k) {
      const V3<float> v0 = load3<float>(s->v0, k);
      float tt, uu, vv;
      hit_tri(o, d, v0, load3<float>(s->v1, k) - v0, load3<float>(s->v2, k) - v0, eps, tt, uu, vv);
      if (tt > eps && tt < best) { best = tt; bi = k; }
    }
    tri[i] = bi;
    t[i] = best;
  }
}

// Function-level evaluation of the restated reference functions on given
// inputs and random draws (checked against fixtures that the reference's own
// functions computed).  Row layouts of `in` / `out` per kind are listed in
// oracle.h.
void orc_eval(const orc_scene *s, const orc_config *c, int32_t kind, int32_t n, const float *in, int32_t in_stride,
              const float *draws, int32_t draw_stride, float *out, int32_t out_stride, int32_t *draws_used) {
  const Ctx<float> x(s, c);
  using F = float;
  using V = V3<float>;
  auto v3 = [](const float *p) { return V{p[0], p[1], p[2]}; };
  auto put3 = [](float *p, V v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; };
  for (int i = 0; i < n; ++i) {
    const float *a = in ? in + (int64_t)i * in_stride : nullptr;
    float *o = out + (int64_t)i * out_stride;
    Rng rng(0, 0, 0, 0);
    rng.fixed = draws ? draws + (int64_t)i * draw_stride : nullptr;
    rng.nfixed = draws ? (uint32_t)draw_stride : 0;
    if (!rng.fixed) { static const float none = 0.5f; rng.fixed = &none; rng.nfixed = 0; }
    orc_stats st{0, 0, 0, 0};
    switch (kind) {
      case ORC_EVAL_TRIANGLE: {  // main.py:807-829
        const V v0 = v3(a + 6);
        F t, u, vv;
        hit_tri(v3(a), v3(a + 3), v0, v3(a + 9) - v0, v3(a + 12) - v0, x.eps, t, u, vv);
        o[0] = t; o[1] = u; o[2] = vv;
        break;
      }
      case ORC_EVAL_AABB:  // main.py:797-805
        o[0] = hit_aabb(v3(a), v3(a + 3), v3(a + 6), v3(a + 9)) ? 1.f : 0.f;
        break;
      case ORC_EVAL_TRACE: {  // main.py:831-864
        const Hit<F> h = trace(x, v3(a), v3(a + 3), nullptr);
        o[0] = h.t; put3(o + 1, h.normal); put3(o + 4, h.shading_normal); o[7] = (F)h.mat;
        o[8] = h.u; o[9] = h.v; o[10] = (F)h.is_hit; o[11] = (F)h.front; o[12] = (F)h.tri;
        break;
      }
      case ORC_EVAL_COMPLEX: {  // main.py:868-896
        const C2<F> r1 = csqrt(C2<F>{a[0], a[1]});
        const C2<F> r2 = cdiv(C2<F>{a[0], a[1]}, C2<F>{a[2], a[3]});
        o[0] = r1.re; o[1] = r1.im; o[2] = r2.re; o[3] = r2.im;
        break;
      }
      case ORC_EVAL_FRESNEL:  // main.py:925-966
        o[0] = fresnel<F>(a[0], a[1], a[2], a[3], a[4]);
        break;
      case ORC_EVAL_GGX_D:  // main.py:900-907
        o[0] = ggx_d(x, a[0], a[1]);
        break;
      case ORC_EVAL_GGX_G:  // main.py:909-923
        o[0] = ggx_g(v3(a), v3(a + 3), v3(a + 6), a[9]);
        break;
      case ORC_EVAL_GGX_SAMPLE:  // main.py:968-978
        put3(o, ggx_sample(x, a[0], a[1], v3(a + 2), a[5]));
        break;
      case ORC_EVAL_HG:  // main.py:758-766
        o[0] = hg_eval(x, a[0], a[1]);
        break;
      case ORC_EVAL_HG_SAMPLE:  // main.py:768-792
        put3(o, hg_sample(x, v3(a), a[3], rng));
        break;
      case ORC_EVAL_COS_HEMISPHERE:  // main.py:689-705
        put3(o, cosine_hemisphere(x, v3(a), rng));
        break;
      case ORC_EVAL_SPHERE:  // main.py:682-687
        put3(o, random_in_unit_sphere(x, rng));
        break;
      case ORC_EVAL_BSDF: {  // main.py:1360-1444
        F b, p;
        evaluate_bsdf(x, (int)a[0], (int)a[1], v3(a + 2), v3(a + 5), v3(a + 8), (int)a[11], b, p);
        o[0] = b; o[1] = p;
        break;
      }
      case ORC_EVAL_SHADOW:  // main.py:1446-1499
        o[0] = shadow_transmittance(x, v3(a), v3(a + 3), a[6], (int)a[7], (int)a[8], (int)a[9], &st);
        break;
      case ORC_EVAL_NEE: {  // main.py:1296-1358
        Ray<F> ray{};
        ray.pos = v3(a); ray.dir = v3(a + 3); ray.active = (int)a[6]; ray.transport = (int)a[7];
        ray.vol = (int)a[8]; ray.thr = 1.f; ray.spdf = 1.f;
        const Nee<F> r = sample_direct_light(x, ray, v3(a + 9), (int)a[12], rng, &st);
        o[0] = r.factor; o[1] = r.emission; o[2] = r.weight;
        break;
      }
      case ORC_EVAL_SURFACE: {  // main.py:1000-1188
        Ray<F> ray{};
        ray.pos = V{0.f, 0.f, 0.f}; ray.dir = v3(a); ray.active = (int)a[3]; ray.transport = (int)a[3];
        ray.vol = (int)a[4]; ray.thr = 1.f; ray.spdf = 1.f;
        VolEvent<F> ev{};
        ev.hit_mat = (int)a[5]; ev.snormal = v3(a + 6); ev.normal = ev.snormal; ev.front = 1;
        const SurfEvent<F> r = scatter_surface(x, ray, ev, rng);
        o[0] = (F)r.did_reflect; put3(o + 1, r.dir); o[4] = r.est; o[5] = r.pdf; o[6] = (F)r.new_wl;
        break;
      }
      case ORC_EVAL_VOLUME: {  // main.py:1190-1292
        Ray<F> ray{};
        ray.pos = v3(a); ray.dir = v3(a + 3); ray.active = (int)a[6]; ray.transport = (int)a[6];
        ray.vol = (int)a[7]; ray.thr = 1.f; ray.spdf = 1.f; ray.pen = -1;
        const VolEvent<F> e = scatter_volume(x, ray, rng, &st);
        o[0] = (F)e.action; o[1] = e.travel; o[2] = e.est; put3(o + 3, e.normal); put3(o + 6, e.snormal);
        o[9] = (F)e.front; o[10] = (F)e.hit_mat; o[11] = (F)e.tri; put3(o + 12, e.dir); o[15] = (F)e.new_wl;
        o[16] = (F)e.pen;
        break;
      }
      default:
        break;
    }
    if (draws_used) draws_used[i] = (int32_t)rng.n;
  }
}

void orc_render_pass(const orc_scene *s, const orc_config *c, uint32_t pass_idx, int32_t band,
                     const int32_t *pixel_ids, int32_t npix, double *out, int32_t use_double,
                     int32_t nthreads, orc_stats *stats) {
  if (use_double)
    render_pass_t<double>(s, c, pass_idx, band, pixel_ids, npix, out, nthreads, stats);
  else
    render_pass_t<float>(s, c, pass_idx, band, pixel_ids, npix, out, nthreads, stats);
}

void orc_adjoint_pass(const orc_scene *s, const orc_config *c, uint32_t pass_idx, int32_t band,
                      const int32_t *pixel_ids, int32_t npix, const double *adj, int32_t nparams,
                      const int64_t *param_ids, double *grad, double *out, int32_t use_double, int32_t nthreads) {
  if (use_double)
    adjoint_pass_t<double>(s, c, pass_idx, band, pixel_ids, npix, adj, nparams, param_ids, grad, out, nthreads);
  else
    adjoint_pass_t<float>(s, c, pass_idx, band, pixel_ids, npix, adj, nparams, param_ids, grad, out, nthreads);
}

int32_t orc_build_bvh_sweep(int32_t num_tris, const float *v0, const float *v1, const float *v2,
                            int32_t max_nodes, float *node_min, float *node_max, int32_t *left,
                            int32_t *right, int32_t *num_tris_node, int32_t *tri_start, int32_t *perm) {
  if (num_tris <= 0) return 0;
  SweepBuilder b;
  b.n = num_tris;
  for (int a = 0; a < 3; ++a) {
    b.cen[a].resize(num_tris);
    b.tmin[a].resize(num_tris);
    b.tmax[a].resize(num_tris);
  }
  for (int t = 0; t < num_tris; ++t)
    for (int a = 0; a < 3; ++a) {
      const float p = v0[3 * t + a], q = v1[3 * t + a], r = v2[3 * t + a];
      b.cen[a][t] = ((p + q) + r) / 3.0f;  // (v0 + v1 + v2) / 3.0 in float32
      b.tmin[a][t] = std::min(std::min(p, q), r);
      b.tmax[a][t] = std::max(std::max(p, q), r);
    }
  b.perm.assign(num_tris, -1);
  std::vector<int> all(num_tris);
  std::iota(all.begin(), all.end(), 0);
  b.build(std::move(all));
  const int N = (int)b.ntris.size();
  if (N > max_nodes) return -1;
  std::memcpy(node_min, b.nmin.data(), sizeof(float) * 3 * N);
  std::memcpy(node_max, b.nmax.data(), sizeof(float) * 3 * N);
  std::memcpy(left, b.left.data(), sizeof(int) * N);
  std::memcpy(right, b.right.data(), sizeof(int) * N);
  std::memcpy(num_tris_node, b.ntris.data(), sizeof(int) * N);
  std::memcpy(tri_start, b.tstart.data(), sizeof(int) * N);
  std::memcpy(perm, b.perm.data(), sizeof(int) * num_tris);
  return N;
}

}  // extern "C"
