// The reference's spectral estimator as device functions (FP32).
//
// Every function follows the reference renderer (main.py of
// Xyzonox/taichi-spectral-render) line for line in what it computes and in
// the order it draws random numbers; the structure is reorganised so that the
// megakernel and the wavefront stages can share it:
//   volume_event()   = scatter_volume after its trace, main.py:1190-1292
//   nee_setup()      = sample_direct_light up to its shadow query, main.py:1296-1358
//   shadow_segment() = one iteration of shadow_transmittance, main.py:1446-1499
//   scatter_surface()= main.py:1000-1188
// Quirks of the reference that are kept on purpose: the surface-fluorescence
// wavelength is drawn but never applied; shadow segments restart from the
// shading point plus the last segment length; Fresnel selection without
// dividing by F; the light CDF may end below 1 and then selects slot 0 --
// here: light slot 0 of the band table is whatever triangle the reference's
// "index 0" denotes (triangle 0 of the BVH order).
#pragma once
#include "common.cuh"
#include "trace.cuh"

namespace ts {

struct Mat {
  float n, k, rough, sigma_s, emission, g;
  int is_vol, surf_emis, eem;
};

TS_D Mat get_mat(const DevScene &s, int B, int m, int band) {  // main.py:980-996
  const float4 a = __ldg(s.mat + ((size_t)m * B + band) * 2 + 0);
  const float4 b = __ldg(s.mat + ((size_t)m * B + band) * 2 + 1);
  Mat r;
  r.n = a.x; r.k = a.y; r.rough = a.z; r.sigma_s = a.w;
  r.emission = b.x; r.g = b.y;
  r.is_vol = __float_as_int(b.z);
  r.surf_emis = __float_as_int(b.w);
  r.eem = __ldg(s.mat_eem + m);
  return r;
}

// 4*pi*k / lambda[m] (main.py:1057, 1203, 1462)
TS_D float absorb_m(const DevConfig &c, float k, int band) {
  return (kFourPiF * k) / (c.lmin_m + ((float)band * c.step_nm) * 1e-9f);
}
// 4*pi*k*1e9 / lambda[nm] (main.py:1394)
TS_D float absorb_nm(const DevConfig &c, float k, int band) {
  return (kFourPiF * k * 1e9f) / (c.lmin_nm + (float)band * c.step_nm);
}

TS_D void onb(float3 n, float3 &t, float3 &b) {
  const float3 up = fabsf(n.y) < 0.999f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
  t = normalize(cross(up, n));
  b = cross(n, t);
}

TS_D float3 random_in_unit_sphere(Rng &rng) {  // main.py:682-687
  const float z = rng.next() * 2.0f - 1.0f;
  const float rxy = sqrtf(fmaxf(0.f, 1.0f - z * z));
  const float phi = rng.next() * 2.0f * kPiF;
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return f3(rxy * cp, rxy * sp, z);
}

TS_D float3 cosine_hemisphere(float3 n, Rng &rng) {  // main.py:689-705
  const float r1 = rng.next();
  const float r2 = rng.next();
  const float phi = kTwoPiF * r1;
  const float ct = sqrtf(1.0f - r2);
  const float st = sqrtf(r2);
  float3 t, b;
  onb(n, t, b);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return t * cp * st + b * sp * st + n * ct;
}

TS_D float hg_eval(float cos_t, float g) {  // main.py:758-766
  const float g2 = g * g;
  const float denom = 1.0f + g2 - 2.0f * g * cos_t;
  return (1.0f - g2) / (kFourPiF * denom * sqrtf(denom) + 1e-6f);
}

TS_D float3 hg_sample(float3 w, float g, Rng &rng, float *ct_out = nullptr) {  // main.py:768-792
  float ct;
  if (fabsf(g) < 1e-4f) {
    ct = 2.0f * rng.next() - 1.0f;
  } else {
    const float rs = (1.0f - g * g) / (1.0f - g + 2.0f * g * rng.next());
    ct = (1.0f + g * g - rs * rs) / (2.0f * g);
  }
  if (ct_out) *ct_out = ct;
  const float st = sqrtf(fmaxf(0.f, 1.0f - ct * ct));
  const float phi = kTwoPiF * rng.next();
  float3 u, v;
  onb(w, u, v);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return u * cp * st + v * sp * st + w * ct;
}

// ------------------------------------------------------------ Fresnel / GGX
struct Cx { float re, im; };
TS_D Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
TS_D Cx cdiv(Cx a, Cx b) {
  const Cx p = cmul(a, Cx{b.re, -b.im});
  const float m = b.re * b.re + b.im * b.im;
  return {p.re / m, p.im / m};
}
TS_D Cx csqrt(Cx z) {  // main.py:887-896
  const float mod = sqrtf(z.re * z.re + z.im * z.im);
  const float re = sqrtf((mod + z.re) / 2.0f);
  const float sg = z.im > 0.f ? 1.f : (z.im < 0.f ? -1.f : 0.f);
  float im = sg * sqrtf((mod - z.re) / 2.0f);
  if (z.im == 0.f) im = 0.f;
  return {re, im};
}
// fresnel_spectral, main.py:925-966 (unpolarised, complex permittivities)
TS_D float fresnel(float cos_i, float ni, float ki, float nt, float kt) {
  const float ang = acosf(fminf(fmaxf(cos_i, -1.f), 1.f));
  const Cx e_in = {ni * ni - ki * ki, 2.0f * ni * ki};
  const Cx e_tr = {nt * nt - kt * kt, 2.0f * nt * kt};
  float s, ct;
  sincosf(ang, &s, &ct);
  const float s2 = s * s;
  Cx left = cmul(csqrt(e_in), Cx{ct, 0.f});
  const Cx es = cmul(e_in, Cx{s2, 0.f});
  Cx right = csqrt(Cx{e_tr.re - es.re, e_tr.im - es.im});
  const Cx rs = cdiv(Cx{left.re - right.re, left.im - right.im}, Cx{left.re + right.re, left.im + right.im});
  left = cmul(e_tr, left);
  right = cmul(e_in, right);
  const Cx rp = cdiv(Cx{left.re - right.re, left.im - right.im}, Cx{left.re + right.re, left.im + right.im});
  return 0.5f * ((rs.re * rs.re + rs.im * rs.im) + (rp.re * rp.re + rp.im * rp.im));
}
TS_D float ggx_d(float ndh, float rough) {  // main.py:900-907, alpha = roughness^2
  const float a = rough * rough;
  const float a2 = a * a;
  const float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
  return a2 / (kPiF * d * d);
}
TS_D float ggx_g(float3 n, float3 v, float3 l, float rough) {  // main.py:909-923
  const float ndv = fmaxf(dot(n, v), 0.f);
  const float a = fmaxf(rough * rough, 1e-4f);
  const float k = a * a / 2.0f;
  const float gv = ndv / (ndv * (1.0f - k) + k + 1e-7f);
  const float ndl = fmaxf(dot(n, l), 0.f);
  const float gl = ndl / (ndl * (1.0f - k) + k + 1e-7f);
  return gv * gl;
}
TS_D float3 ggx_sample(float xi0, float xi1, float3 n, float alpha) {  // main.py:968-978
  const float a2 = alpha * alpha;
  const float phi = kTwoPiF * xi0;
  const float ct = sqrtf((1.0f - xi1) / (1.0f + (a2 - 1.0f) * xi1));
  const float st = sqrtf(1.0f - ct * ct);
  float3 t, b;
  onb(n, t, b);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return normalize(t * (cp * st) + b * (sp * st) + n * ct);
}
TS_D void oren_nayar_terms(float rough, float &A, float &B) {
  const float sigma = rough * kPiF / 2.0f;
  const float s2 = sigma * sigma;
  A = 1.0f - s2 / (2.0f * (s2 + 0.33f));
  B = 0.45f * s2 / (s2 + 0.09f);
}
TS_D float oren_nayar_angular(float3 n, float3 l, float3 v, float ndl, float ndv, float A, float B) {
  const float th_i = acosf(ndl), th_o = acosf(ndv);
  const float al = fmaxf(th_i, th_o), be = fminf(th_i, th_o);
  float cphi = 0.f;
  if (ndl > 1e-4f && ndv > 1e-4f) {
    const float3 pi_ = normalize(l - n * ndl);
    const float3 po = normalize(v - n * ndv);
    cphi = fmaxf(0.f, dot(pi_, po));
  }
  return A + B * cphi * sinf(al) * tanf(be);
}

// ------------------------------------------------------------ path state
struct PathState {
  float3 pos, dir;
  float thr, spdf;
  int active, active_px, plen, vol;
};

// camera ray of cast_rays, main.py:1505-1529 (fov_scale = 1 is the reference),
// from the camera origin o and basis (cu, cv, cw)
TS_D void camera_ray(float3 o, float3 cu, float3 cv, float3 cw, const DevConfig &c, int i, int j, Rng &rng,
                     PathState &p, int band) {
  const float u = ((float)i + rng.next()) / (float)c.W;
  const float v = ((float)j + rng.next()) / (float)c.H;
  p.dir = normalize(cu * ((u * 2.0f - 1.0f) * c.aspect * c.fov) + cv * ((v * 2.0f - 1.0f) * c.fov) - cw * 2.0f);
  p.pos = o;
  p.thr = 1.0f;
  p.spdf = 1.0f;
  p.active = band;
  p.active_px = band;
  p.plen = 0;
  p.vol = 0;
}

TS_D void camera_ray(const DevScene &s, const DevConfig &c, int i, int j, Rng &rng, PathState &p, int band) {
  camera_ray(s.cam_o, s.cam_u, s.cam_v, s.cam_w, c, i, j, rng, p, band);
}

struct VolEvent {
  int action;  // 0 none/absorbed, 1 surface, 2 scattered, 3 fluoresced
  float travel, est;
  float3 normal, snormal, dir;
  int front, hit_mat, tri, new_wl;
  float dsurf;   // distance to the closest surface (1e9 on a miss)
  float hg_ct;   // sampled phase cosine of a scattering event
};

TS_D float eem_cdf_pick(const DevScene &s, int B, int eem, int row, float xi) {
  const float *cdf = s.eem_cdf + ((size_t)eem * B + row) * B;
  for (int j = 0; j < B; ++j)
    if (xi < __ldg(cdf + j)) return (float)j;
  return (float)row;
}

// scatter_volume after its trace (main.py:1190-1292).  The free-flight draw
// comes first in the path's stream, exactly as in the reference where it
// precedes the trace.
TS_D VolEvent volume_event(const DevScene &s, const DevConfig &c, const PathState &p, const Hit &hit,
                           Rng &rng) {
  VolEvent r;
  r.action = 0;
  r.est = 0.f;
  r.new_wl = p.active;
  r.dir = p.dir;
  r.hit_mat = 0;
  r.tri = -1;
  const Mat vm = get_mat(s, c.B, p.vol, p.active);
  const float absorb = absorb_m(c, vm.k, p.active);
  const float dvol = -logf(-rng.next() + 1.0f - 1e-7f) / (vm.sigma_s + absorb + 1e-6f);
  const float dsurf = hit.t;
  float travel = -1.f;
  if (dsurf < c.escape) {
    travel = dsurf;
    if (dvol + c.eps < travel) travel = dvol;
  }
  r.travel = travel;
  r.dsurf = dsurf;
  r.hg_ct = 1.f;
  SurfaceInfo si;
  if (hit.slot >= 0) {
    si = surface_info(s, hit, p.dir);
  } else {
    si.ng = si.ns = f3(0.f, 0.f, 0.f);
    si.front = 0;
    si.mat = 0;
  }
  r.front = si.front;
  const float f = (float)si.front;
  r.normal = si.ng * f - si.ng * (1.0f - f);
  r.snormal = si.ns * f - si.ns * (1.0f - f);
  const float T = expf(-(absorb + vm.sigma_s) * travel);
  const float emit = ((-T + 1.0f) * vm.emission) / (absorb + 1e-6f);
  const float att = T + emit;
  if (travel == dsurf) {
    r.est = att / (1.0f + 1e-6f);
    r.action = 1;
    r.hit_mat = si.mat;
    r.tri = hit.slot;
  } else if (travel >= 0.f) {
    r.hit_mat = -1;
    const float xe = rng.next();
    const float kind = absorb / (vm.sigma_s + absorb + 1e-6f);
    if (xe <= kind) {
      if (vm.eem > 0) {
        const float qy = __ldg(s.eem_qy + (size_t)vm.eem * c.B + p.active);
        const float xf = rng.next();
        if (qy > 0.f && xf < qy) {
          r.action = 3;
          const int nw = (int)eem_cdf_pick(s, c.B, vm.eem, p.active, rng.next());
          r.new_wl = nw;
          r.dir = random_in_unit_sphere(rng);
          const float em2 = ((-(1.0f - T) + 1.0f) * get_mat(s, c.B, p.vol, nw).emission) / (absorb + 1e-6f);
          r.est = (1.0f - T) + em2;
        } else {
          r.est = att;
        }
      } else {
        r.est = att / (1.0f + 1e-6f);
      }
    } else {
      r.action = 2;
      r.dir = hg_sample(p.dir, vm.g, rng, &r.hg_ct);
      r.est = att;
    }
  }
  return r;
}

// evaluate_bsdf, main.py:1360-1444.  Both cosines are clamped to >= 1e-4
// before the reflect/transmit test, so only the reflection lobe is reachable.
TS_D void evaluate_bsdf(const DevScene &s, const DevConfig &c, int vol, int surf, float3 V, float3 L, float3 N,
                        int wl, float &bsdf, float &pdf) {
  const Mat vm = get_mat(s, c.B, vol, wl);
  const Mat sm = get_mat(s, c.B, surf, wl);
  const float ndl = fmaxf(1e-4f, dot(N, L));
  const float ndv = fmaxf(1e-4f, dot(N, V));
  bsdf = 0.f;
  pdf = 0.f;
  float3 H = normalize(V + L);
  if (dot(H, N) < 0.f) H = -H;
  const float vdh = fmaxf(1e-4f, dot(V, H));
  const float F = fresnel(vdh, vm.n, vm.k, sm.n, sm.k);
  if (sm.rough > 0.008f) {
    const float ndh = fmaxf(1e-4f, dot(N, H));
    const float D = ggx_d(ndh, sm.rough);
    const float G = ggx_g(N, V, L, sm.rough);
    bsdf += (D * G * F) / (4.0f * ndl * ndv);
    pdf += (D * ndh * F) / (4.0f * vdh);
  }
  const float absorb = absorb_nm(c, sm.k, wl);
  const float albedo = sm.sigma_s / (sm.sigma_s + absorb + 1e-6f);
  float A, B;
  oren_nayar_terms(sm.rough, A, B);
  const float nv = 1.0f - (float)sm.is_vol;
  bsdf += (1.0f - F) * nv * (albedo / kPiF) * oren_nayar_angular(N, L, V, ndl, ndv, A, B);
  pdf += ndl * 0.318309886184f * (1.0f - F) * nv;
}

// Shadow query produced by next-event estimation.
struct ShadowQuery {
  float3 origin, dir;
  float max_dist;
  int light_slot, vol, band;
  float contrib;  // everything of the direct term except the transmittance
  // factors of contrib, kept for the adjoint: contrib = thr * em * bsdf * cs * ga * weight
  float em, bsdf, pdf, cs, ga, pl;
  int lmat;
};

// sample_direct_light up to the shadow test (main.py:1296-1358).  Returns
// false when the band has no lights (no draws are made then).  The BSDF /
// phase evaluation does not depend on the transmittance, so it is done here;
// the deposit is contrib * T when T > 1e-6.
TS_D bool nee_setup(const DevScene &s, const DevConfig &c, const PathState &p, int transport, float3 N,
                    int surf, Rng &rng, ShadowQuery &q) {
  const int wl = p.active;
  const int nl = __ldg(s.num_lights + wl);
  if (nl <= 0) return false;
  const float xl = rng.next();
  int lt = 0;
  for (int i = 0; i < nl; ++i) {
    if (xl < __ldg(s.light_cdf + (size_t)wl * s.max_lights + i)) {
      lt = __ldg(s.light_slot + (size_t)wl * s.max_lights + i);
      break;
    }
  }
  float bx = rng.next();
  float by = rng.next();
  if (bx + by > 1.0f) { bx = 1.0f - bx; by = 1.0f - by; }
  const float4 A = __ldg(s.tri + 3 * (size_t)lt + 0);
  const float4 E1 = __ldg(s.tri + 3 * (size_t)lt + 1);
  const float4 E2 = __ldg(s.tri + 3 * (size_t)lt + 2);
  const float3 P = xyz(A) + bx * xyz(E1) + by * xyz(E2);
  const float3 toL = P - p.pos;
  q.dir = normalize(toL);
  q.max_dist = length(toL);
  q.origin = p.pos;
  q.light_slot = lt;
  q.vol = p.vol;
  const int lmat = __float_as_int(E1.w);
  const float4 s0 = __ldg(s.shade + 3 * (size_t)lt + 0);
  const float4 s1 = __ldg(s.shade + 3 * (size_t)lt + 1);
  const float4 s2 = __ldg(s.shade + 3 * (size_t)lt + 2);
  const float3 ln = f3(s0.w, s1.w, s2.w);
  const float cosl = fmaxf(0.f, dot(ln, -q.dir));
  const float dsq = q.max_dist * q.max_dist;
  const float G = cosl / (dsq + 1e-4f);
  float bsdf, pdf, cs;
  if (surf != -1) {
    cs = fmaxf(0.f, dot(N, q.dir));
    evaluate_bsdf(s, c, p.vol, surf, -p.dir, q.dir, N, wl, bsdf, pdf);
  } else {
    cs = fmaxf(0.f, dot(p.dir, q.dir));
    bsdf = hg_eval(cs, get_mat(s, c.B, p.vol, wl).g);
    pdf = bsdf;
  }
  const float area = __ldg(s.light_area + wl);
  const float emission = get_mat(s, c.B, lmat, transport).emission;
  const float pl = dsq / (fmaxf(1e-6f, cosl) * area);
  const float weight = (pl * pl) / (pl * pl + pdf * pdf + 1e-6f);
  q.contrib = p.thr * emission * (bsdf * cs * G * area) * weight;
  q.em = emission;
  q.bsdf = bsdf;
  q.pdf = pdf;
  q.cs = cs;
  q.ga = G * area;
  q.pl = pl;
  q.lmat = lmat;
  return true;
}

// One iteration of shadow_transmittance (main.py:1446-1499) given the trace
// of the current segment.  Returns true when the chain is finished.
struct ShadowState {
  float3 pos;
  float total, traveled;
  int vol, seg;
};

// Distance bound for the trace of the next shadow segment.  In a medium that
// neither absorbs nor scatters at this band (air), hits beyond the light do
// not change the transmittance -- exp(-0 * t) = 1 for any t, and such a hit
// counts as reaching the light -- so the traversal may stop at the light.  In
// any other medium the reference attenuates over the distance to the next
// surface even beyond the light (main.py:1459-1462), which needs the true
// closest hit.
TS_D float shadow_bound(const DevScene &s, const DevConfig &c, const ShadowQuery &q, const ShadowState &st,
                        int band) {
  const Mat vm = get_mat(s, c.B, st.vol, band);
  return absorb_m(c, vm.k, band) + vm.sigma_s == 0.f ? q.max_dist - st.traveled : 1e9f;
}
TS_D bool shadow_segment(const DevScene &s, const DevConfig &c, const ShadowQuery &q, const Hit &hit, int band,
                         ShadowState &st) {
  const Mat vm = get_mat(s, c.B, st.vol, band);
  const float absorb = absorb_m(c, vm.k, band);
  st.total *= expf(-(absorb + vm.sigma_s) * hit.t);
  if (hit.t >= (q.max_dist - st.traveled) || hit.slot == q.light_slot) {
    st.total *= expf(-(absorb + vm.sigma_s) * (q.max_dist - st.traveled));
    return true;
  }
  const SurfaceInfo si = surface_info(s, hit, q.dir);
  const Mat sm = get_mat(s, c.B, si.mat, band);
  float nt = sm.n;
  if (!si.front) nt = get_mat(s, c.B, 0, band).n;
  const float f = (float)si.front;
  const float3 inc = si.ns * f - si.ns * (1.0f - f);
  const float3 T = refract(q.dir, inc, vm.n / nt);
  const float rt = (dot(q.dir, T) - 1.0f) * 37.9743f;
  const float rt2 = rt * rt;
  st.total *= 1.0f / (1.0f + rt2 * rt2 * (3.0f - 2.0f * rt));
  if (st.total < 1e-6f || !sm.is_vol) {
    st.total = 0.f;
    return true;
  }
  st.traveled += hit.t + c.eps;
  st.pos = q.origin + q.dir * (hit.t + c.eps);
  st.vol = si.mat * si.front;
  return ++st.seg >= c.scatter_bounces;
}

struct SurfEvent {
  int did_reflect;
  float3 dir;
  float est, pdf;
  // sampling record, kept for the adjoint
  float3 H;      // sampled GGX half vector
  float xi1;     // its polar random number (the sampler's density follows from it exactly)
  float F, cin;  // Fresnel term at cin = max(1e-4, V.H)
  float dist;    // penetration distance (used by surface fluorescence)
  int branch;    // kSurfGlossy, kSurfDiffuse, kSurfTransmit, kSurfTir
  int fl;        // surface fluorescence: -1 no test, -2 rejected, >= 0 accepted band
};
enum { kSurfGlossy = 0, kSurfDiffuse = 1, kSurfTransmit = 2, kSurfTir = 3 };

// scatter_surface, main.py:1000-1188
TS_D SurfEvent scatter_surface(const DevScene &s, const DevConfig &c, const PathState &p, const VolEvent &ev,
                               Rng &rng) {
  SurfEvent r;
  r.did_reflect = 0;
  r.dir = f3(0.f, 0.f, 0.f);
  r.est = 0.f;
  r.pdf = 0.f;
  const Mat sm = get_mat(s, c.B, ev.hit_mat, p.active);
  const Mat vm = get_mat(s, c.B, p.vol, p.active);
  const float3 V = -p.dir;
  const float3 N = ev.snormal;
  const float xi0 = rng.next();
  const float xi1 = rng.next();
  const float3 H = ggx_sample(xi0, xi1, N, sm.rough);
  const float cin = fmaxf(1e-4f, dot(V, H));
  const float F = fresnel(cin, vm.n, vm.k, sm.n, sm.k);
  const float pick = fminf(fmaxf(rng.next(), 0.f), 0.99f);
  r.H = H;
  r.xi1 = xi1;
  r.F = F;
  r.cin = cin;
  r.dist = 0.f;
  r.fl = -1;
  r.branch = kSurfGlossy;
  bool glossy = false, abs_cos = false;
  if (pick < F) {
    glossy = true;
  } else {
    const float absorb = absorb_m(c, sm.k, p.active);
    const float dist = -logf(-rng.next() + 1.0f + 1e-7f) / (sm.sigma_s + absorb + 1e-6f);
    r.dist = dist;
    if (!sm.is_vol) {
      r.branch = kSurfDiffuse;
      r.did_reflect = 1;
      const float3 S = cosine_hemisphere(N, rng);
      const float ndl = fmaxf(1e-4f, dot(N, S));
      const float ndv = fmaxf(1e-4f, dot(N, V));
      const float albedo = sm.sigma_s / (sm.sigma_s + absorb + 1e-6f);
      float A, B;
      oren_nayar_terms(sm.rough, A, B);
      float bsdf = (1.0f - F) * (albedo / kPiF) * oren_nayar_angular(N, S, V, ndl, ndv, A, B);
      const float pdf = 0.318309886184f * ndl;
      if (sm.eem > 0) {
        const float qy = __ldg(s.eem_qy + (size_t)sm.eem * c.B + p.active);
        const float xi3 = rng.next();
        r.fl = -2;
        if (qy > 0.f && xi3 < qy) {
          const int nw = (int)eem_cdf_pick(s, c.B, sm.eem, p.active, rng.next());
          r.fl = nw;
          const Mat smf = get_mat(s, c.B, ev.hit_mat, nw);
          bsdf *= expf(-absorb_m(c, smf.k, nw) * dist);
        }
      }
      r.est = (bsdf * ndl) / pdf;
      r.pdf = pdf;
      r.dir = S;
    } else {
      const float3 T = refract(p.dir, H, vm.n / sm.n);
      if (dot(T, T) < 1e-4f) {
        glossy = true;
        abs_cos = true;
        r.branch = kSurfTir;
      } else {
        r.branch = kSurfTransmit;
        r.did_reflect = 0;
        r.dir = T;
        if (sm.rough < 0.0018f) {
          r.est = 1.0f - F;
          r.pdf = 1e9f;
        } else {
          const float ldh = dot(T, H), vdh = dot(V, H);
          const float ndh = fmaxf(1e-4f, dot(N, H));
          const float ndl = fmaxf(1e-4f, fabsf(dot(N, T)));
          const float ndv = fmaxf(1e-4f, fabsf(dot(N, V)));
          const float G = ggx_g(N, V, T, sm.rough);
          const float D = ggx_d(ndh, sm.rough);
          const float den = vm.n * vdh + sm.n * ldh;
          const float den2 = den * den;
          const float bsdf = (fabsf(ldh * vdh) / (ndl * ndv)) * ((sm.n * sm.n * (1.0f - F) * D * G) / den2);
          const float pdf = (D * ndh * (1.0f - F) * sm.n * sm.n * fabsf(ldh)) / den2;
          r.est = (bsdf * ndl) / pdf;
          r.pdf = pdf;
        }
      }
    }
  }
  if (glossy) {
    const float3 L = reflect(p.dir, H);
    r.dir = L;
    r.did_reflect = 1;
    if (sm.rough < 0.008f) {
      r.est = F;
      r.pdf = 1e9f;
    } else {
      const float ndl = fmaxf(1e-4f, dot(N, L));
      const float ndh = fmaxf(1e-4f, dot(N, H));
      const float ndv = fmaxf(1e-4f, dot(N, V));
      const float D = ggx_d(ndh, sm.rough);
      const float G = ggx_g(N, V, L, sm.rough);
      const float bsdf = (D * G * F) / (4.0f * ndl * ndv);
      const float pdf = (D * ndh) / (4.0f * cin);
      const float cs = abs_cos ? fabsf(dot(N, L)) : fmaxf(0.f, dot(N, L));
      r.est = (bsdf * cs) / pdf;
      r.pdf = pdf;
    }
  }
  return r;
}

// Direct hit on an emitter (main.py:1548-1559)
TS_D float emitter_hit(const DevScene &s, const DevConfig &c, const PathState &p, const VolEvent &ev,
                       float emission, float *w_out = nullptr, float *pl_out = nullptr) {
  const float4 s0 = __ldg(s.shade + 3 * (size_t)ev.tri + 0);
  const float4 s1 = __ldg(s.shade + 3 * (size_t)ev.tri + 1);
  const float4 s2 = __ldg(s.shade + 3 * (size_t)ev.tri + 2);
  const float3 ln = f3(s0.w, s1.w, s2.w);
  const float dsq = ev.travel * ev.travel;
  const float cosl = fmaxf(0.f, dot(ln, -p.dir));
  const float pl = (dsq * fminf(1.0f, (float)p.plen)) / (cosl * __ldg(s.light_area + p.active) + 1e-6f);
  const float w = (p.spdf * p.spdf) / (pl * pl + p.spdf * p.spdf + 1e-6f);
  if (w_out) *w_out = w;
  if (pl_out) *pl_out = pl;
  return p.thr * emission * w;
}

// After scatter_surface: main.py:1569-1574
TS_D void apply_surface(const DevConfig &c, PathState &p, const VolEvent &ev, const SurfEvent &se) {
  p.spdf = se.pdf;
  p.dir = se.dir;
  p.thr *= se.est;
  const float sgn = (float)se.did_reflect - (1.0f - (float)se.did_reflect);
  p.pos = p.pos + ev.normal * c.eps * sgn;
  p.vol = ev.hit_mat * ev.front * (1 - se.did_reflect) + p.vol * se.did_reflect;
}

}  // namespace ts
