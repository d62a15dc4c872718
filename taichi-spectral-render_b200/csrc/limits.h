// Structural limits shared by the host builder and the device traversal.
#pragma once

namespace ts {
constexpr int kStackDepth = 64;  // traversal stack entries per ray (bounds the tree depth)
constexpr int kLeafMax = 16;     // triangles per leaf in the two-child layout (4-bit count)
constexpr int kMaxBlock = 256;   // largest thread block of the render kernels
constexpr int kWideStack = 96;   // traversal stack entries for 4- and 8-wide nodes
}  // namespace ts
