// Film kernels (average_and_reset_block, color_rays, clear_pixel_space,
// visualize_normals of the reference, main.py:1592-1674) and the batched
// closest-hit query used by parity checks.
#include "estimator.cuh"
#include "kernels.cuh"

namespace ts {

namespace {

constexpr int kThreads = 256;

inline int grid_for(size_t n) {
  size_t g = (n + kThreads - 1) / kThreads;
  if (g > (1u << 20)) g = 1u << 20;
  return (int)(g ? g : 1);
}

// average_and_reset_block, main.py:1592-1607: running mean over blocks, and
// the per-cell sum of squared block values for the Monte Carlo error.
__global__ void k_accumulate(Film f, int n) {
  const size_t total = (size_t)f.W * f.H * f.B;
  const double inv_n = 1.0 / (double)n;
  const double nm1 = (double)(n - 1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const double b = f.block[i];
    f.mean[i] = (f.mean[i] * nm1 + b) * inv_n;
    f.m2[i] += b * b;
    f.block[i] = 0.0;
  }
}

__global__ void k_clear(Film f) {
  const size_t total = (size_t)f.W * f.H * f.B;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    f.block[i] = 0.0;
    f.mean[i] = 0.0;
    f.m2[i] = 0.0;
  }
}

// XYZ half of color_rays (main.py:1617-1620): sum_k mean_k * cmf_k * scale,
// scale = step / normalisation.  Output [j][i][3] float32 at render resolution.
__global__ void k_resolve_xyz(Film f, const float *__restrict__ cmf, double scale, float *__restrict__ xyz) {
  const int npix = f.W * f.H;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    double X = 0.0, Y = 0.0, Z = 0.0;
    for (int k = 0; k < f.B; ++k) {
      const double a = f.mean[(size_t)k * npix + p];
      X += a * (double)cmf[3 * k + 0];
      Y += a * (double)cmf[3 * k + 1];
      Z += a * (double)cmf[3 * k + 2];
    }
    xyz[3 * (size_t)p + 0] = (float)(X * scale);
    xyz[3 * (size_t)p + 1] = (float)(Y * scale);
    xyz[3 * (size_t)p + 2] = (float)(Z * scale);
  }
}

// Whole color_rays (main.py:1609-1629): nearest-neighbour upscale to the image
// resolution, XYZ -> RGB, Reinhard with exposure, gamma.  Output [j][i][3].
__global__ void k_resolve_rgb(Film f, const float *__restrict__ cmf, double scale, const float *__restrict__ M,
                              float exposure, float gamma, int iw, int ih, float *__restrict__ rgb) {
  const int npix = f.W * f.H;
  const int n = iw * ih;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int i = p % iw, j = p / iw;
    const int ri = (int)((float)i / (float)iw * (float)f.W);
    const int rj = (int)((float)j / (float)ih * (float)f.H);
    const int rp = rj * f.W + ri;
    double X = 0.0, Y = 0.0, Z = 0.0;
    for (int k = 0; k < f.B; ++k) {
      const double a = f.mean[(size_t)k * npix + rp];
      X += a * (double)cmf[3 * k + 0];
      Y += a * (double)cmf[3 * k + 1];
      Z += a * (double)cmf[3 * k + 2];
    }
    const float x = (float)(X * scale), y = (float)(Y * scale), z = (float)(Z * scale);
    for (int ch = 0; ch < 3; ++ch) {
      const float h = M[3 * ch + 0] * x + M[3 * ch + 1] * y + M[3 * ch + 2] * z;
      const float e = exposure * h;
      const float mapped = e / (e + 1.0f);
      rgb[3 * (size_t)p + ch] = powf(mapped, 1.0f / gamma);
    }
  }
}

// visualize_normals, main.py:1631-1659 (render-resolution part)
template <int W>
__global__ void k_normals(DevScene s, DevConfig c, float *__restrict__ out, uint32_t *err) {
  const int npix = c.W * c.H;
  uint32_t eb = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    const int i = p % c.W, j = p / c.W;
    const float u = ((float)i + 0.5f) / (float)c.W;
    const float v = ((float)j + 0.5f) / (float)c.H;
    const float3 d = normalize(s.cam_u * ((u * 2.0f - 1.0f) * c.aspect * c.fov) +
                               s.cam_v * ((v * 2.0f - 1.0f) * c.fov) - s.cam_w * 2.0f);
    const Hit h = trace_closest<W>(s, s.cam_o, d, c.eps, eb);
    float3 col = f3(0.f, 0.f, 0.f);
    if (h.slot >= 0) col = surface_info(s, h, d).ns * 0.5f + f3(0.5f, 0.5f, 0.5f);
    out[3 * (size_t)p + 0] = col.x;
    out[3 * (size_t)p + 1] = col.y;
    out[3 * (size_t)p + 2] = col.z;
  }
  if (eb) atomicOr(err, eb);
}

template <int kMode, int W>
__global__ void k_trace_batch(DevScene s, float eps, const float *__restrict__ rays, int n,
                              int32_t *__restrict__ tri_orig, float *__restrict__ t, float *__restrict__ u,
                              float *__restrict__ v, uint32_t *err) {
  uint32_t eb = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const float *q = rays + 6 * (size_t)r;
    const float3 o = f3(q[0], q[1], q[2]), d = f3(q[3], q[4], q[5]);
    const Hit h = kMode == 0 ? trace_closest<W>(s, o, d, eps, eb) : trace_reference_order(s, o, d, eps, eb);
    tri_orig[r] = h.slot >= 0 ? __float_as_int(__ldg(s.tri + 3 * (size_t)h.slot).w) : -1;
    t[r] = h.t;
    if (u) u[r] = h.u;
    if (v) v[r] = h.v;
  }
  if (eb) atomicOr(err, eb);
}

}  // namespace

cudaError_t launch_accumulate_block(Film f, int n, cudaStream_t st) {
  k_accumulate<<<grid_for((size_t)f.W * f.H * f.B), kThreads, 0, st>>>(f, n);
  return cudaGetLastError();
}
cudaError_t launch_clear_film(Film f, cudaStream_t st) {
  k_clear<<<grid_for((size_t)f.W * f.H * f.B), kThreads, 0, st>>>(f);
  return cudaGetLastError();
}
cudaError_t launch_resolve_xyz(Film f, const float *cmf, double scale, float *xyz, cudaStream_t st) {
  k_resolve_xyz<<<grid_for((size_t)f.W * f.H), kThreads, 0, st>>>(f, cmf, scale, xyz);
  return cudaGetLastError();
}
cudaError_t launch_resolve_rgb(Film f, const float *cmf, double scale, const float *M, float exposure, float gamma,
                               int iw, int ih, float *rgb, cudaStream_t st) {
  k_resolve_rgb<<<grid_for((size_t)iw * ih), kThreads, 0, st>>>(f, cmf, scale, M, exposure, gamma, iw, ih, rgb);
  return cudaGetLastError();
}
cudaError_t launch_render_normals(const DevScene &s, const DevConfig &c, float *out, uint32_t *err,
                                  cudaStream_t st) {
  const int g = grid_for((size_t)c.W * c.H);
  if (s.node_width == 9) k_normals<9><<<g, kThreads, 0, st>>>(s, c, out, err);
  else if (s.node_width == 5) k_normals<5><<<g, kThreads, 0, st>>>(s, c, out, err);
  else if (s.node_width == 8) k_normals<8><<<g, kThreads, 0, st>>>(s, c, out, err);
  else if (s.node_width == 4) k_normals<4><<<g, kThreads, 0, st>>>(s, c, out, err);
  else k_normals<2><<<g, kThreads, 0, st>>>(s, c, out, err);
  return cudaGetLastError();
}
cudaError_t launch_trace_batch(const DevScene &s, float eps, const float *rays, int n, int mode, int32_t *tri_orig,
                               float *t, float *u, float *v, uint32_t *err, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for((size_t)n);
  if (mode != 0) k_trace_batch<1, 2><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  else if (s.node_width == 9) k_trace_batch<0, 9><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  else if (s.node_width == 5) k_trace_batch<0, 5><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  else if (s.node_width == 8) k_trace_batch<0, 8><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  else if (s.node_width == 4) k_trace_batch<0, 4><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  else k_trace_batch<0, 2><<<g, kThreads, 0, st>>>(s, eps, rays, n, tri_orig, t, u, v, err);
  return cudaGetLastError();
}

}  // namespace ts
