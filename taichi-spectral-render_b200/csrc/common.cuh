// Shared device-side definitions: scene/config views, vector helpers,
// IEEE-exact arithmetic helpers for the intersection tests, Philox RNG.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "limits.h"

#define TS_HD __host__ __device__ __forceinline__
#define TS_D __device__ __forceinline__

namespace ts {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr float kFourPiF = 12.5663706143591729539f;

// error bits reported through the context's device status word
enum : uint32_t {
  kErrStackOverflow = 1u << 0,
  kErrQueueOverflow = 1u << 1,
  kErrIterationCap = 1u << 2,
};

struct DevConfig {
  int32_t W, H, B;
  float lmin_m;     // lambda_min in metres (rounded once from double)
  float lmin_nm;    // lambda_min in nm
  float step_nm;    // band spacing in nm
  float eps, escape;
  int32_t max_depth, scatter_bounces;
  float aspect, fov;
  uint32_t seed, scene_id;
  int32_t speculative;  // two-child layout: speculative while-while traversal
};

// Device scene.  Triangles are in BVH leaf order ("slot" order).
//   tri[3*s+0] = (v0.xyz, orig_id bits)
//   tri[3*s+1] = (e1.xyz, material bits)     e1 = v1 - v0 (float32)
//   tri[3*s+2] = (e2.xyz, 0)                 e2 = v2 - v0 (float32)
//   shade[3*s+k] = (n_k.xyz, geometric_normal[k])
// Wide nodes (width 4 / 8): six rows of child-box bounds (lo.x hi.x lo.y hi.y
// lo.z hi.z, one float per child) followed by the child links, 128 / 256 B.
// Two-child BVH nodes, 64 B each:
//   node[4*i+0] = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   node[4*i+1] = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   node[4*i+2] = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   node[4*i+3] = (child0, child1, -, -) as int; child >= 0 is an inner node,
//                 child < 0 is a leaf: ~child = (first_slot << 4) | (count - 1)
// Reference-layout nodes (main.py:267-275) are kept for the exact-order
// traversal used by parity checks.
struct DevScene {
  const float4 *__restrict__ node;    // device BVH layout (node_width children per node)
  const float4 *__restrict__ tri;
  const float4 *__restrict__ shade;
  int32_t num_nodes, num_tris;
  int32_t node_width;                 // 2, 4 or 8
  const float *__restrict__ ref_min;
  const float *__restrict__ ref_max;
  const int4 *__restrict__ ref_link;  // (left, right, num_tris, tri_start)
  int32_t num_ref_nodes;
  const float4 *__restrict__ mat;     // [(m*B+band)*2 + 0/1]: (n,k,rough,sigma_s), (emission,g,is_vol,surf_emis)
  const int32_t *__restrict__ mat_eem;
  const float *__restrict__ eem;      // [E][B][B]
  const float *__restrict__ eem_qy;   // [E][B] row maximum
  const float *__restrict__ eem_cdf;  // [E][B][B] running sum of e/row_sum (float32, in order)
  int32_t num_materials, num_eems;
  const float *__restrict__ light_cdf;  // [B][L]
  const int32_t *__restrict__ light_slot;  // [B][L]
  const int32_t *__restrict__ num_lights;  // [B]
  const float *__restrict__ light_area;    // [B]
  int32_t max_lights;
  float3 cam_o, cam_u, cam_v, cam_w;
};

// ------------------------------------------------------------ float3 helpers
TS_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
TS_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
TS_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
TS_HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
TS_HD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
TS_HD float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
TS_HD float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
TS_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
TS_HD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
TS_D float length(float3 a) { return sqrtf(dot(a, a)); }
TS_D float3 normalize(float3 a) { return a / sqrtf(dot(a, a)); }
TS_D float3 reflect(float3 x, float3 n) { return x - (2.0f * dot(n, x)) * n; }
TS_D float3 refract(float3 x, float3 n, float eta) {
  const float dxn = dot(x, n);
  const float k = 1.0f - eta * eta * (1.0f - dxn * dxn);
  if (k >= 0.0f) return eta * x - (eta * dxn + sqrtf(k)) * n;
  return f3(0.f, 0.f, 0.f);
}
TS_D float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }

// ------------------------------------------------------------ IEEE per-op helpers
// The intersection tests must round like the CPU oracle (one rounding per
// operation, no fused multiply-add), so they are written with the _rn
// intrinsics, which the compiler never contracts.
TS_D float xmul(float a, float b) { return __fmul_rn(a, b); }
TS_D float xadd(float a, float b) { return __fadd_rn(a, b); }
TS_D float xsub(float a, float b) { return __fsub_rn(a, b); }
TS_D float3 xsub3(float3 a, float3 b) { return f3(xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)); }
TS_D float xdot(float3 a, float3 b) { return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z)); }
TS_D float3 xcross(float3 a, float3 b) {
  return f3(xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
            xsub(xmul(a.x, b.y), xmul(a.y, b.x)));
}

// ------------------------------------------------------------ Philox-4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11.  Counter = (pixel, draw/4, scene, 0), key = (seed, pass).
TS_HD uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k.x += 0x9E3779B9u; k.y += 0xBB67AE85u; }
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}

// Per-path stream.  Draw n is word (n & 3) of block n >> 2, so a path's
// sequence depends only on (seed, pass, pixel, scene) and the draw index; the
// state that must survive between kernels is just the draw index.
struct Rng {
  uint2 key;
  uint32_t pix, scene, n;
  uint4 buf;
  TS_D void init(uint32_t seed, uint32_t pass, uint32_t pixel, uint32_t scene_id, uint32_t draw = 0) {
    key = make_uint2(seed, pass);
    pix = pixel;
    scene = scene_id;
    n = draw;
    if (n & 3u) buf = philox4x32_10(make_uint4(pix, n >> 2, scene, 0u), key);
  }
  TS_D float next() {
    if ((n & 3u) == 0) buf = philox4x32_10(make_uint4(pix, n >> 2, scene, 0u), key);
    const uint32_t w = n & 3u;
    const uint32_t x = w == 0 ? buf.x : (w == 1 ? buf.y : (w == 2 ? buf.z : buf.w));
    ++n;
    return (float)(x >> 8) * (1.0f / 16777216.0f);
  }
};

}  // namespace ts
