// Path-replay adjoint of one sample pass: gradients of an image loss with
// respect to the spectral material parameters (differentiation is a new
// capability; the reference renderer, main.py of Xyzonox/taichi-spectral-render,
// has none).
//
// Each path of cast_rays (main.py:1502-1590) runs twice from its Philox
// stream (path replay, no tape), in two launches of the same persistent kernel:
//   replay 0: the path as the forward pass rendered it, summing its deposits
//             weighted by the adjoint film, A = sum_v w(pixel, band_v) D_v,
//             stored per path (4 bytes);
//   replay 1: the same path again.  A_rem starts at A and drops by w D_v at
//             each deposit.  Every multiplicative factor f of the throughput
//             and every sampling decision with probability p adds
//             A_rem * d log f (or d log p) at the moment it is applied -- A_rem
//             is then exactly the weighted radiance the factor scales -- and
//             every deposit adds w * dD_v for its own factors (emission,
//             BSDF / phase function, MIS weight, shadow transmittance).
// The phase is a template parameter: replay 0 carries no gradient code and
// every lane of a replay-1 warp executes the gradient code (one launch mixing
// the phases per lane ran them divergently).  Path arithmetic is FP32 like the
// forward kernels (the same event functions, so the replays take the forward
// pass's branches); gradient sums are FP64, per block in shared memory, then
// across blocks with global atomics.
#include "adjoint.cuh"
#include "kernels.cuh"

namespace ts {

namespace {

// Scores of an EEM decision (main.py:1247-1272 volume, :1090-1121 surface):
// accept with probability qy = row maximum, then pick column nw with
// probability e[nw] / sum(row).  outcome: -2 rejected, >= 0 accepted band.
__device__ void grad_eem_choice(const DevScene &s, int B, int pmat, int e, int row, int outcome, float arem,
                                const Grad &g) {
  const float *r = s.eem + ((size_t)e * B + row) * B;
  float q = 0.f, sum = 0.f;
  int jm = 0;
  for (int j = 0; j < B; ++j) {
    const float v = __ldg(r + j);
    if (v > q) { q = v; jm = j; }
    sum += v;
  }
  const int base = pmat + (e * B + row) * B;
  if (outcome < 0) {
    if (q < 1.f) g.add(base + jm, -arem / (1.f - q));
    return;
  }
  if (q > 0.f) g.add(base + jm, arem / q);
  if (sum > 0.f) {
    for (int j = 0; j < B; ++j) g.add(base + j, -arem / sum);
    const float v = __ldg(r + outcome);
    if (v > 0.f) g.add(base + outcome, arem / v);
  }
}

// Volume event (scatter_volume, main.py:1190-1292): free-flight decision,
// absorb / scatter choice, EEM choice, phase-direction density and the
// attenuation factor.  p: path state before the event; arem: weighted
// radiance of this and all later deposits.
__device__ void grad_volume(const DevScene &s, const DevConfig &c, int pmat, const PathState &p, const VolEvent &ev,
                            float arem, const Grad &g) {
  if (arem == 0.f) return;
  const int B = c.B, b = p.active, m = p.vol;
  const Mat vm = get_mat(s, B, m, b);
  const float cA = absorb_m(c, 1.0f, b);  // d absorb / d k
  const float ab = absorb_m(c, vm.k, b);
  const float st = vm.sigma_s + ab + 1e-6f;
  const float d = ev.travel;
  const float T = expf(-(ab + vm.sigma_s) * d);
  const float ap = ab + 1e-6f;
  const float emit = ((1.0f - T) * vm.emission) / ap;
  const float att = T + emit;
  const float dT_k = -d * T * cA, dT_s = -d * T;
  float gk = 0.f, gs = 0.f, ge = 0.f, gg = 0.f;
  bool att_factor = true;
  if (ev.action == 1) {
    // surface reached: P(free flight >= d_surf - eps) = exp(-sigma_t x)
    const float x = fmaxf(0.f, ev.dsurf - c.eps);
    gk -= x * cA;
    gs -= x;
  } else {
    // medium event at d: density sigma_t exp(-sigma_t d)
    gk += cA / st - d * cA;
    gs += 1.0f / st - d;
    const float kind = ab / st;
    const float dkind_k = cA * (vm.sigma_s + 1e-6f) / (st * st);
    const float dkind_s = -ab / (st * st);
    if (ev.action == 2) {
      const float q = 1.0f - kind;
      if (q > 0.f) { gk -= dkind_k / q; gs -= dkind_s / q; }
      if (fabsf(vm.g) >= 1e-4f) gg += hg_score(ev.hg_ct, vm.g);
    } else {
      if (kind > 0.f) { gk += dkind_k / kind; gs += dkind_s / kind; }
      if (vm.eem > 0) {
        grad_eem_choice(s, B, pmat, vm.eem, b, ev.action == 3 ? ev.new_wl : -2, arem, g);
        if (ev.action == 3) {
          att_factor = false;
          const float em2 = get_mat(s, B, m, ev.new_wl).emission;
          const float e3 = (1.0f - T) + (T * em2) / ap;
          if (e3 != 0.f) {
            gk += (-dT_k + (dT_k * em2) / ap - (T * em2 * cA) / (ap * ap)) / e3;
            gs += (-dT_s + (dT_s * em2) / ap) / e3;
            g.add(pidx(B, m, kPropEmission, ev.new_wl), arem * (T / ap) / e3);
          }
        }
      }
    }
  }
  if (att_factor && att != 0.f) {
    gk += (dT_k * (1.0f - vm.emission / ap) - emit * cA / ap) / att;
    gs += (dT_s * (1.0f - vm.emission / ap)) / att;
    ge += ((1.0f - T) / ap) / att;
  }
  g.add(pidx(B, m, kPropK, b), arem * gk);
  g.add(pidx(B, m, kPropSigmaS, b), arem * gs);
  g.add(pidx(B, m, kPropEmission, b), arem * ge);
  g.add(pidx(B, m, kPropG, b), arem * gg);
}

// Surface event (scatter_surface, main.py:1000-1188): half-vector density,
// Fresnel branch choice, surface-fluorescence choices and the estimate.
// p: path state before the event.  Sets sp to d spdf of the new path pdf.
__device__ void grad_surface(const DevScene &s, const DevConfig &c, int pmat, const PathState &p, const VolEvent &ev,
                             const SurfEvent &se, float arem, const Grad &g, SpdfGrad &sp) {
  const int B = c.B, b = p.active, ms = ev.hit_mat, mv = p.vol;
  sp.reset();
  sp.ms = ms;
  sp.mv = mv;
  sp.band = b;
  const Mat sm = get_mat(s, B, ms, b);
  const Mat vm = get_mat(s, B, mv, b);
  const float3 N = ev.snormal, V = -p.dir;
  const float r = sm.rough;
  float gr = 0.f, gks = 0.f, gkv = 0.f, gss = 0.f;
  // GGX half vector, drawn with alpha = roughness: density a2 c / (pi (c^2 (a2 - 1) + 1)^2),
  // a2 = r^2.  Its log-derivative at the sampled c, 2/r - 4 r c^2 / (c^2 (a2 - 1) + 1), equals
  // (4 xi1 - 2) / r because c^2 = (1 - xi1) / (1 + (a2 - 1) xi1) -- free of cancellation.
  if (r > 0.f) gr += (4.0f * se.xi1 - 2.0f) / r;
  const D2 F = fresnel_d(se.cin, vm.n, vm.k, sm.n, sm.k);
  const float Fv = se.F, q = 1.0f - Fv;
  if (se.branch == kSurfGlossy) {
    if (Fv <= 0.99f && Fv > 0.f) { gkv += F.a / Fv; gks += F.b / Fv; }
  } else if (q > 0.f) {
    gkv -= F.a / q;
    gks -= F.b / q;
  }
  if (se.branch == kSurfGlossy || se.branch == kSurfTir) {
    if (Fv > 0.f) { gkv += F.a / Fv; gks += F.b / Fv; }
    if (r >= 0.008f) {
      float dG, dD;
      const float G = ggx_g_dr(N, V, se.dir, r, dG);
      if (G > 0.f) gr += dG / G;
      const float ndh = fmaxf(1e-4f, dot(N, se.H));
      ggx_d_dr(ndh, r, dD);
      sp.dr = dD * ndh / (4.0f * se.cin);
    }
  } else if (se.branch == kSurfDiffuse) {
    if (q > 0.f) { gkv -= F.a / q; gks -= F.b / q; }
    const float cA = absorb_m(c, 1.0f, b);
    const float ab = absorb_m(c, sm.k, b);
    const float den = sm.sigma_s + ab + 1e-6f;
    if (sm.sigma_s > 0.f) {
      gss += (ab + 1e-6f) / (den * sm.sigma_s);
      gks += -cA / den;
    }
    const float ndl = fmaxf(1e-4f, dot(N, se.dir));
    const float ndv = fmaxf(1e-4f, dot(N, V));
    float don;
    const float on = oren_nayar_dr(N, se.dir, V, ndl, ndv, r, don);
    if (on != 0.f) gr += don / on;
    if (se.fl != -1) {
      grad_eem_choice(s, B, pmat, sm.eem, b, se.fl, arem, g);
      if (se.fl >= 0) {
        // penetration distance ~ sigma_t exp(-sigma_t dist), then exp(-absorb(k(nw)) dist)
        gks += cA / den - se.dist * cA;
        gss += 1.0f / den - se.dist;
        g.add(pidx(B, ms, kPropK, se.fl), arem * (-se.dist * absorb_m(c, 1.0f, se.fl)));
      }
    }
  } else {  // kSurfTransmit
    if (r < 0.0018f) {
      if (q > 0.f) { gkv -= F.a / q; gks -= F.b / q; }
    } else {
      float dG, dD;
      const float G = ggx_g_dr(N, V, se.dir, r, dG);
      if (G > 0.f) gr += dG / G;
      const float ndh = fmaxf(1e-4f, dot(N, se.H));
      const float D = ggx_d_dr(ndh, r, dD);
      if (D > 0.f) sp.dr = se.pdf * dD / D;
      if (q > 0.f) {
        sp.dks = -se.pdf * F.b / q;
        sp.dkv = -se.pdf * F.a / q;
      }
    }
  }
  if (arem == 0.f) return;
  g.add(pidx(B, ms, kPropRough, b), arem * gr);
  g.add(pidx(B, ms, kPropK, b), arem * gks);
  g.add(pidx(B, mv, kPropK, b), arem * gkv);
  g.add(pidx(B, ms, kPropSigmaS, b), arem * gss);
}

}  // namespace

namespace {

template <int W, int kPhase>
__global__ void __launch_bounds__(128, kPhase ? 4 : 5) k_adjoint(DevScene s, DevConfig c, uint32_t pass0, int npass, int band0,
                                                 const double *__restrict__ adj, double *__restrict__ grad,
                                                 float *__restrict__ weight, int pm_shared, int pmat,
                                                 int *__restrict__ counter, uint32_t *__restrict__ err,
                                                 const float *__restrict__ rec) {
  extern __shared__ double sh_grad[];
  for (int i = threadIdx.x; i < pm_shared; i += blockDim.x) sh_grad[i] = 0.0;
  __syncthreads();
  const Grad g{sh_grad, grad, pm_shared};
  const int lane = threadIdx.x & 31;
  const int npix = c.W * c.H;
  const int total = npix * npass;
  const int B = c.B;
  uint32_t errbits = 0;
  int pix = -1;
  uint32_t pass = 0;
  int band = 0;
  bool exhausted = false;
  constexpr bool phase = kPhase == 1;
  int item = 0;
  PathState p;
  Rng rng;
  SpdfGrad sp;
  int k = 0;
  float atot = 0.f, arem = 0.f;
  int seg_m[kAdjMaxSeg];
  float seg_l[kAdjMaxSeg];
  for (;;) {
    const bool need = pix < 0 && !exhausted;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(counter, __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(m & ((1u << lane) - 1u));
        if (idx < total) {
          const int po = idx / npix;
          pix = idx - po * npix;
          pass = pass0 + (uint32_t)po;
          band = (band0 + po) % B;
          item = idx;
          atot = 0.f;
          const float r = !phase && rec ? rec[idx] : -1.f;
          if (r >= 0.f) {
            // the forward pass recorded this path's total deposit, all of it in
            // its own band: A = w(pixel, band) * total, no replay needed
            weight[idx] = (float)__ldg(adj + (size_t)band * npix + pix) * r;
            pix = -1;
          } else {
            if (phase) arem = weight[idx];
            rng.init(c.seed, pass, (uint32_t)pix, c.scene_id);
            camera_ray(s, c, pix % c.W, pix / c.W, rng, p, band);
            sp.reset();
            k = 0;
          }
        } else {
          exhausted = true;
        }
      }
    }
    // lanes that took a recorded item fetch again; stop when every lane is idle and out of items
    if (__ballot_sync(0xffffffffu, pix >= 0 || !exhausted) == 0) break;
    if (pix < 0) continue;

    // ---- one path vertex, exactly as the forward megakernel takes it
    bool done = false;
    const Hit h = trace_closest<W, false>(s, p.pos, p.dir, c.eps, errbits, nullptr, c.escape);
    const VolEvent ev = volume_event(s, c, p, h, rng);
    if (ev.travel < 0.f) {
      done = true;
    } else {
      p.pos = p.pos + p.dir * ev.travel;
      if (phase) grad_volume(s, c, pmat, p, ev, arem, g);
      p.thr *= ev.est;
      float indirect = 0.f, direct = 0.f, ew = 0.f, epl = 0.f;
      bool nee = false, emitter = false;
      ShadowQuery q;
      if (ev.action == 1) {
        const Mat sm = get_mat(s, B, ev.hit_mat, band);
        if (sm.surf_emis) {
          indirect = emitter_hit(s, c, p, ev, sm.emission, &ew, &epl);
          emitter = true;
          done = true;
        } else {
          nee = nee_setup(s, c, p, band, ev.snormal, ev.hit_mat, rng, q);
        }
      } else {
        nee = nee_setup(s, c, p, band, ev.snormal, -1, rng, q);
      }
      int nseg = 0;
      float tsh = 0.f;
      if (nee) {
        ShadowState ss;
        ss.pos = q.origin;
        ss.total = 1.f;
        ss.traveled = 0.f;
        ss.vol = q.vol;
        ss.seg = 0;
        for (;;) {
          // the gradient replay needs true segment lengths even where the forward
          // pass could stop at the light (non-attenuating media): no bound there
          const Hit sh = trace_closest<W, false>(s, ss.pos, q.dir, c.eps, errbits, nullptr,
                                                 phase ? 1e9f : shadow_bound(s, c, q, ss, p.active));
          if (phase && nseg < kAdjMaxSeg) {
            const float left = q.max_dist - ss.traveled;
            const bool reach = sh.t >= left || sh.slot == q.light_slot;
            seg_m[nseg] = ss.vol;
            seg_l[nseg] = reach ? sh.t + left : sh.t;
            ++nseg;
          }
          if (shadow_segment(s, c, q, sh, p.active, ss)) break;
        }
        if (ss.total > 1e-6f) {
          tsh = ss.total;
          direct = q.contrib * ss.total;
        }
      }
      // deposits of this vertex go to the band the path carries after it
      const int bdep = ev.action == 3 ? ev.new_wl : p.active_px;
      const float w = (float)__ldg(adj + (size_t)bdep * npix + pix);
      if (phase == 0) {
        atot += w * indirect;
        atot += w * direct;
      } else {
        if (emitter && w != 0.f) {
          // indirect = thr * em * mis, mis = spdf^2 / (pl^2 + spdf^2 + 1e-6)
          g.add(pidx(B, ev.hit_mat, kPropEmission, band), w * p.thr * ew);
          const float den = epl * epl + p.spdf * p.spdf + 1e-6f;
          const float dmis = 2.0f * p.spdf * (epl * epl + 1e-6f) / (den * den);
          const float em = get_mat(s, B, ev.hit_mat, band).emission;
          const float f = w * p.thr * em * dmis;
          g.add(pidx(B, sp.ms, kPropRough, sp.band), f * sp.dr);
          g.add(pidx(B, sp.ms, kPropK, sp.band), f * sp.dks);
          g.add(pidx(B, sp.mv, kPropK, sp.band), f * sp.dkv);
        }
        if (tsh > 0.f && w != 0.f) {
          // direct = thr * em * bsdf * cs * ga * weight * T
          const int wl = p.active;
          const float kk = p.thr * q.cs * q.ga * tsh;
          const float den = q.pl * q.pl + q.pdf * q.pdf + 1e-6f;
          const float weight = (q.pl * q.pl) / den;
          const float dweight = -2.0f * q.pl * q.pl * q.pdf / (den * den);
          g.add(pidx(B, q.lmat, kPropEmission, band), w * kk * q.bsdf * weight);
          const float wd = w * direct;
          const float cA = absorb_m(c, 1.0f, wl);
          for (int i = 0; i < nseg; ++i) {
            g.add(pidx(B, seg_m[i], kPropK, wl), -wd * seg_l[i] * cA);
            g.add(pidx(B, seg_m[i], kPropSigmaS, wl), -wd * seg_l[i]);
          }
          const float f = w * kk * q.em;
          if (ev.action == 1) {
            float db[4], dp[4];
            evaluate_bsdf_d(s, c, p.vol, ev.hit_mat, -p.dir, q.dir, ev.snormal, wl, db, dp);
            const int ids[4] = {pidx(B, p.vol, kPropK, wl), pidx(B, ev.hit_mat, kPropK, wl),
                                pidx(B, ev.hit_mat, kPropRough, wl), pidx(B, ev.hit_mat, kPropSigmaS, wl)};
            for (int i = 0; i < 4; ++i) g.add(ids[i], f * (db[i] * weight + q.bsdf * dweight * dp[i]));
          } else {
            const float gv = get_mat(s, B, p.vol, wl).g;
            const float dh = hg_eval_dg(q.cs, gv);
            g.add(pidx(B, p.vol, kPropG, wl), f * (dh * weight + q.bsdf * dweight * dh));
          }
        }
        arem -= w * indirect;
        arem -= w * direct;
      }
      if (ev.action == 1 && !done) {
        p.plen++;
        const SurfEvent se = scatter_surface(s, c, p, ev, rng);
        if (phase) grad_surface(s, c, pmat, p, ev, se, arem, g, sp);
        apply_surface(c, p, ev, se);
      } else if (ev.action == 2) {
        p.dir = ev.dir;
        p.plen++;
      } else if (ev.action == 3) {
        p.dir = ev.dir;
        p.active = ev.new_wl;
        p.active_px = ev.new_wl;
        p.plen++;
      }
      if (++k >= c.max_depth || p.thr == 0.f) done = true;
    }
    if (done) {
      if (!phase) weight[item] = atot;  // replay 1 starts from this
      pix = -1;
    }
  }
  if (errbits) atomicOr(err, errbits);
  __syncthreads();
  for (int i = threadIdx.x; i < pm_shared; i += blockDim.x)
    if (sh_grad[i] != 0.0) atomicAdd(grad + i, sh_grad[i]);
}

}  // namespace

int adjoint_shared_params(int pmat) { return pmat <= kAdjSharedMax ? pmat : 0; }

namespace {
template <int W>
void launch_pair(const DevScene &s, const DevConfig &c, uint32_t pass, int npass, int band, const double *adj,
                 double *grad, float *weight, int psh, int pmat, int *counter, uint32_t *err, int grid,
                 cudaStream_t st, const float *rec) {
  const int block = 128;
  k_adjoint<W, 0><<<grid, block, 0, st>>>(s, c, pass, npass, band, adj, grad, weight, 0, pmat, counter, err, rec);
  k_adjoint<W, 1><<<grid, block, (size_t)psh * sizeof(double), st>>>(s, c, pass, npass, band, adj, grad, weight, psh,
                                                                     pmat, counter + 1, err, nullptr);
}
}  // namespace

cudaError_t launch_adjoint(const DevScene &s, const DevConfig &c, uint32_t pass, int band, const double *adj,
                           double *grad, float *weight, int *counter, uint32_t *err, int grid, cudaStream_t st,
                           int npass, const float *rec) {
  cudaError_t e = cudaMemsetAsync(counter, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int pmat = s.num_materials * 6 * c.B;
  const int psh = adjoint_shared_params(pmat);
  if (s.node_width == 9) launch_pair<9>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  else if (s.node_width == 5)
    launch_pair<5>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  else if (s.node_width == 8)
    launch_pair<8>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  else if (s.node_width == 4)
    launch_pair<4>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  else if (c.speculative)
    launch_pair<3>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  else launch_pair<2>(s, c, pass, npass, band, adj, grad, weight, psh, pmat, counter, err, grid, st, rec);
  return cudaGetLastError();
}

// ---- material / EEM refresh from device tables (parameter updates of an optimiser)
namespace {

__global__ void k_pack_materials(float4 *__restrict__ mat, const float *__restrict__ f, int M, int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * B) return;
  const int m = i / B, b = i % B;
  const float *r = f + (size_t)m * 6 * B;
  const float4 old = mat[(size_t)i * 2 + 1];  // keeps the is_true_volume / surface_emission bits
  mat[(size_t)i * 2 + 0] = make_float4(r[0 * B + b], r[1 * B + b], r[2 * B + b], r[3 * B + b]);
  mat[(size_t)i * 2 + 1] = make_float4(r[4 * B + b], r[5 * B + b], old.z, old.w);
}

// row maximum and running CDF, float32 in the order the host upload uses
__global__ void k_eem_tables(const float *__restrict__ eem, float *__restrict__ qy, float *__restrict__ cdf, int E,
                             int B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E * B) return;
  const float *row = eem + (size_t)i * B;
  float q = 0.f, norm = 0.f;
  for (int j = 0; j < B; ++j) {
    if (row[j] > q) q = row[j];
    norm += row[j];
  }
  qy[i] = q;
  float cum = 0.f;
  for (int j = 0; j < B; ++j) {
    cum += row[j] / norm;
    cdf[(size_t)i * B + j] = norm != 0.f ? cum : 0.f;
  }
}

}  // namespace

cudaError_t launch_update_materials(float4 *mat, const float *mat_f32, int M, int B, float *eem, float *qy,
                                    float *cdf, const float *eem_src, int E, cudaStream_t st) {
  if (mat_f32) k_pack_materials<<<(M * B + 127) / 128, 128, 0, st>>>(mat, mat_f32, M, B);
  if (eem_src && E > 0) {
    cudaError_t e = cudaMemcpyAsync(eem, eem_src, sizeof(float) * (size_t)E * B * B, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    k_eem_tables<<<(E * B + 127) / 128, 128, 0, st>>>(eem, qy, cdf, E, B);
  }
  return cudaGetLastError();
}

}  // namespace ts
