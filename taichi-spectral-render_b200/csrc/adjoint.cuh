// Partial derivatives of the estimator's factors with respect to the material
// parameters, for the path-replay adjoint (adjoint.cu).
//
// Differentiable parameters are the entries of the material table
// [M][6][B] (main.py:545-561) except the refractive index -- extinction k,
// roughness, scattering sigma_s, emission and HG anisotropy g -- plus the EEM
// entries [E][B][B].  Index of (material m, property prop, band b):
// (m * 6 + prop) * B + b; EEM entry (e, row, col): M * 6 * B + (e * B + row) * B + col.
//
// The reference's sampling decisions depend on these parameters (free-flight
// distances on sigma_t, the absorb/scatter choice, the Fresnel branch choice,
// the GGX half vector on the roughness, HG directions on g, the EEM quantum
// yield and emission-band choice).  Sampled values are held fixed and every
// decision contributes the derivative of the log of its probability (score
// function), so the gradient is that of the expected value of the reference's
// estimator.  Refractive indices are not differentiable here: they bend rays.
#pragma once
#include "estimator.cuh"

namespace ts {

enum { kPropN = 0, kPropK = 1, kPropRough = 2, kPropSigmaS = 3, kPropEmission = 4, kPropG = 5 };
constexpr int kAdjMaxSeg = 16;  // shadow segments recorded per NEE query (scatter_bounces bound)

TS_D int pidx(int B, int m, int prop, int band) { return (m * 6 + prop) * B + band; }

// Gradient sink: material-table entries go to a block-shared FP64 table when
// it fits (flushed once per block), everything else to the global FP64 array.
struct Grad {
  double *sh;
  double *gl;
  int pm_shared;  // entries held in shared memory (0 = none)
  TS_D void add(int idx, float v) const {
    if (v == 0.f) return;
    if (idx < pm_shared) atomicAdd(sh + idx, (double)v);
    else atomicAdd(gl + idx, (double)v);
  }
};

// Derivative of the MIS pdf carried from a surface scatter to the emitter hit
// that may follow it (main.py:1556-1557 reads surface_pdf there).
struct SpdfGrad {
  int ms, mv, band;
  float dr, dks, dkv;  // d spdf / d (roughness_s, k_s, k_v)
  TS_D void reset() { ms = mv = band = 0; dr = dks = dkv = 0.f; }
};

// ---------------------------------------------------------------- duals
// value + partials with respect to (k_incident, k_transmitted)
struct D2 { float v, a, b; };
TS_D D2 d2c(float v) { return {v, 0.f, 0.f}; }
TS_D D2 operator+(D2 x, D2 y) { return {x.v + y.v, x.a + y.a, x.b + y.b}; }
TS_D D2 operator-(D2 x, D2 y) { return {x.v - y.v, x.a - y.a, x.b - y.b}; }
TS_D D2 operator-(D2 x) { return {-x.v, -x.a, -x.b}; }
TS_D D2 operator*(D2 x, D2 y) { return {x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b}; }
TS_D D2 operator*(D2 x, float s) { return {x.v * s, x.a * s, x.b * s}; }
TS_D D2 operator/(D2 x, D2 y) {
  const float q = x.v / y.v;
  return {q, (x.a - q * y.a) / y.v, (x.b - q * y.b) / y.v};
}
TS_D D2 dsqrt(D2 x) {
  const float r = sqrtf(x.v);
  const float h = r > 0.f ? 0.5f / r : 0.f;
  return {r, x.a * h, x.b * h};
}
struct CD { D2 re, im; };
TS_D CD cmul(CD a, CD b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
TS_D CD cdiv(CD a, CD b) {
  const CD p = cmul(a, CD{b.re, -b.im});
  const D2 m = b.re * b.re + b.im * b.im;
  return {p.re / m, p.im / m};
}
TS_D CD csqrt(CD z) {
  const D2 mod = dsqrt(z.re * z.re + z.im * z.im);
  const D2 re = dsqrt((mod + z.re) * 0.5f);
  const float sg = z.im.v > 0.f ? 1.f : (z.im.v < 0.f ? -1.f : 0.f);
  D2 im = dsqrt((mod - z.re) * 0.5f) * sg;
  if (z.im.v == 0.f) im = d2c(0.f);
  return {re, im};
}
// fresnel() with its partials d/dki (.a) and d/dkt (.b)
TS_D D2 fresnel_d(float cos_i, float ni, float ki, float nt, float kt) {
  const float ang = acosf(fminf(fmaxf(cos_i, -1.f), 1.f));
  const D2 Ki = {ki, 1.f, 0.f}, Kt = {kt, 0.f, 1.f};
  const D2 Ni = d2c(ni), Nt = d2c(nt);
  const CD e_in = {Ni * Ni - Ki * Ki, Ni * Ki * 2.0f};
  const CD e_tr = {Nt * Nt - Kt * Kt, Nt * Kt * 2.0f};
  float s, ct;
  sincosf(ang, &s, &ct);
  const float s2 = s * s;
  CD left = cmul(csqrt(e_in), CD{d2c(ct), d2c(0.f)});
  const CD es = cmul(e_in, CD{d2c(s2), d2c(0.f)});
  CD right = csqrt(CD{e_tr.re - es.re, e_tr.im - es.im});
  const CD rs = cdiv(CD{left.re - right.re, left.im - right.im}, CD{left.re + right.re, left.im + right.im});
  left = cmul(e_tr, left);
  right = cmul(e_in, right);
  const CD rp = cdiv(CD{left.re - right.re, left.im - right.im}, CD{left.re + right.re, left.im + right.im});
  return ((rs.re * rs.re + rs.im * rs.im) + (rp.re * rp.re + rp.im * rp.im)) * 0.5f;
}

// ---------------------------------------------------------------- closed-form partials
// ggx_d and d/d roughness (alpha = roughness^2, main.py:900-907)
TS_D float ggx_d_dr(float ndh, float r, float &dd) {
  const float a = r * r;
  const float a2 = a * a;
  const float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  const float D = a2 / (kPiF * d * d);
  const float dDda2 = (d - 2.0f * a2 * ndh * ndh) / (kPiF * d * d * d);
  dd = dDda2 * 4.0f * a * r;
  return D;
}
// ggx_g and d/d roughness (main.py:909-923)
TS_D float ggx_g_dr(float3 n, float3 v, float3 l, float r, float &dg) {
  const float ndv = fmaxf(dot(n, v), 0.f);
  const float a = fmaxf(r * r, 1e-4f);
  const float k = a * a / 2.0f;
  const float dv = ndv * (1.0f - k) + k + 1e-7f;
  const float gv = ndv / dv;
  const float ndl = fmaxf(dot(n, l), 0.f);
  const float dl = ndl * (1.0f - k) + k + 1e-7f;
  const float gl = ndl / dl;
  const float dk = r * r > 1e-4f ? a * 2.0f * r : 0.f;  // dk/dr = a * da/dr
  const float dgv = -gv * (1.0f - ndv) / dv;            // d gv / dk
  const float dgl = -gl * (1.0f - ndl) / dl;
  dg = (dgv * gl + gv * dgl) * dk;
  return gv * gl;
}
// Oren-Nayar angular term A + B * X and its derivative in the roughness
// (sigma = roughness * pi / 2, main.py:1068-1088)
TS_D float oren_nayar_dr(float3 n, float3 l, float3 v, float ndl, float ndv, float r, float &don) {
  const float sigma = r * kPiF / 2.0f;
  const float s2 = sigma * sigma;
  const float A = 1.0f - s2 / (2.0f * (s2 + 0.33f));
  const float B = 0.45f * s2 / (s2 + 0.09f);
  const float th_i = acosf(ndl), th_o = acosf(ndv);
  const float al = fmaxf(th_i, th_o), be = fminf(th_i, th_o);
  float cphi = 0.f;
  if (ndl > 1e-4f && ndv > 1e-4f) {
    const float3 pi_ = normalize(l - n * ndl);
    const float3 po = normalize(v - n * ndv);
    cphi = fmaxf(0.f, dot(pi_, po));
  }
  const float X = cphi * sinf(al) * tanf(be);
  const float dA = -0.33f / (2.0f * (s2 + 0.33f) * (s2 + 0.33f));
  const float dB = 0.45f * 0.09f / ((s2 + 0.09f) * (s2 + 0.09f));
  don = (dA + dB * X) * (r * kPiF * kPiF / 2.0f);
  return A + B * X;
}
// d hg_eval / d g (the phase function with its 1e-6, main.py:758-766)
TS_D float hg_eval_dg(float c, float g) {
  const float g2 = g * g;
  const float den = 1.0f + g2 - 2.0f * g * c;
  const float sq = sqrtf(den);
  const float q = kFourPiF * den * sq + 1e-6f;
  return (-2.0f * g * q - (1.0f - g2) * kFourPiF * 1.5f * sq * (2.0f * g - 2.0f * c)) / (q * q);
}
// d log p / d g of the HG density the sampler draws from (main.py:768-792)
TS_D float hg_score(float c, float g) {
  const float g2 = g * g;
  return -2.0f * g / (1.0f - g2) - 1.5f * (2.0f * g - 2.0f * c) / (1.0f + g2 - 2.0f * g * c);
}

// evaluate_bsdf (main.py:1360-1444) partials with respect to
// x = (k_v, k_s, roughness_s, sigma_s_s): dbsdf[x], dpdf[x]
TS_D void evaluate_bsdf_d(const DevScene &s, const DevConfig &c, int vol, int surf, float3 V, float3 L, float3 N,
                          int wl, float dbsdf[4], float dpdf[4]) {
  const Mat vm = get_mat(s, c.B, vol, wl);
  const Mat sm = get_mat(s, c.B, surf, wl);
  const float ndl = fmaxf(1e-4f, dot(N, L));
  const float ndv = fmaxf(1e-4f, dot(N, V));
  for (int i = 0; i < 4; ++i) dbsdf[i] = dpdf[i] = 0.f;
  float3 H = normalize(V + L);
  if (dot(H, N) < 0.f) H = -H;
  const float vdh = fmaxf(1e-4f, dot(V, H));
  const D2 F = fresnel_d(vdh, vm.n, vm.k, sm.n, sm.k);
  if (sm.rough > 0.008f) {
    const float ndh = fmaxf(1e-4f, dot(N, H));
    float dD, dG;
    const float D = ggx_d_dr(ndh, sm.rough, dD);
    const float G = ggx_g_dr(N, V, L, sm.rough, dG);
    const float k0 = 1.0f / (4.0f * ndl * ndv), p0 = ndh / (4.0f * vdh);
    dbsdf[0] += D * G * F.a * k0;
    dbsdf[1] += D * G * F.b * k0;
    dbsdf[2] += (dD * G + D * dG) * F.v * k0;
    dpdf[0] += D * F.a * p0;
    dpdf[1] += D * F.b * p0;
    dpdf[2] += dD * F.v * p0;
  }
  const float nv = 1.0f - (float)sm.is_vol;
  if (nv == 0.f) return;
  const float ab = absorb_nm(c, sm.k, wl);
  const float cA = absorb_nm(c, 1.0f, wl);
  const float den = sm.sigma_s + ab + 1e-6f;
  const float alb = sm.sigma_s / den;
  const float dalb_s = (ab + 1e-6f) / (den * den);
  const float dalb_k = -sm.sigma_s * cA / (den * den);
  float don;
  const float on = oren_nayar_dr(N, L, V, ndl, ndv, sm.rough, don);
  const float ip = 1.0f / kPiF;
  dbsdf[0] += -F.a * nv * alb * ip * on;
  dbsdf[1] += (-F.b * alb + (1.0f - F.v) * dalb_k) * nv * ip * on;
  dbsdf[2] += (1.0f - F.v) * nv * alb * ip * don;
  dbsdf[3] += (1.0f - F.v) * nv * dalb_s * ip * on;
  dpdf[0] += -ndl * 0.318309886184f * F.a * nv;
  dpdf[1] += -ndl * 0.318309886184f * F.b * nv;
}

}  // namespace ts
