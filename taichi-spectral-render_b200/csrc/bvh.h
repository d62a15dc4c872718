// Host-side BVH construction and conversion to the device layouts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace ts {

struct BvhParams {
  int bins = 32;          // SAH bins per axis
  float cost_trav = 1.0f; // SAH traversal cost (relative to one triangle test)
  float cost_tri = 1.0f;
  int leaf_max = 8;       // largest leaf the SAH may choose (hard cap 16)
  int sah_depth = 40;     // below this depth, object-median splits only (bounds the tree depth)
  int threads = 0;        // 0 = hardware concurrency
  int width = 2;          // node width of the device layout: 2, 4 or 8
  bool quantize = false;  // 4- / 8-wide: child boxes as 8-bit conservative offsets (64 / 96 B per node)
};

struct BvhOut {
  std::vector<int32_t> perm;   // slot -> original triangle index
  std::vector<float4> node2;   // device layout: width 2 -> 4 float4 per node, 4 -> 8, 8 -> 16
  int width = 2;               // node width of node2 (a wide layout falls back to 2 if its stack bound is exceeded)
  bool quantized = false;      // node2 holds quantized wide nodes
  int stack_need = 0;          // deepest traversal stack the device layout can require
  std::vector<float> ref_min, ref_max;  // reference layout, [N][3]
  std::vector<int4> ref_link;           // (left, right, num_tris, tri_start)
  int max_depth = 0;
  int leaves = 0;
  double sah_cost = 0.0;
};

// Binned-SAH build over the triangles' bounding boxes and centroids.
bool build_bvh_binned(int T, const float *v0, const float *v1, const float *v2, const BvhParams &p, BvhOut &out,
                      std::string &err);

// float4s per node of the device layout for a node width (quantized: child
// boxes as bytes relative to the node's origin -- 4 float4 for 4-wide, 6 for 8-wide).
inline int node_float4s(int width, bool quantized = false) {
  if (quantized) return width == 8 ? 6 : 4;
  return width == 8 ? 16 : (width == 4 ? 8 : 4);
}
// the device layout id: the node width, plus one for quantized child boxes (5, 9)
inline int layout_id(int width, bool quantized) { return quantized && width >= 4 ? width + 1 : width; }

// Adopt a tree given in the reference layout (e.g. produced by the reference's
// own build_bvh, main.py:437-507): perm[slot] = original triangle index.
bool bvh_from_reference(int T, const float *v0, const float *v1, const float *v2, int N, const float *nmin,
                        const float *nmax, const int32_t *left, const int32_t *right, const int32_t *ntris,
                        const int32_t *tstart, const int32_t *perm, BvhOut &out, std::string &err,
                        int width = 2, bool quantize = false);

}  // namespace ts
