// Binned-SAH build of the static scene's BVH on the host (once per context).
#pragma once

#include <cstdint>

namespace upbp_host {

// Builds a binary BVH over n boxes (6 floats each: lo.xyz, hi.xyz) with one
// primitive per leaf, in the device's node layout (16 words per node: the
// left child's lo.xyz, hi.xyz, the right child's lo.xyz, hi.xyz, then the
// left and right links and primitive counts as int32; a link >= 0 is an
// internal node, a leaf link is ~position).  Node 0 is the root; a subtree of
// m primitives occupies m - 1 consecutive node slots, its root first.
// order[k] receives the primitive at leaf position k.  Splits minimise the
// surface-area heuristic over 16 centroid bins per axis; from depth 48 on,
// or where all centroids coincide, a subtree is split at its middle.  Up to
// `threads` threads build the upper subtrees in parallel.  n >= 2.
void sah_build(const float* boxes, uint32_t n, float* nodes, uint32_t* order, int threads);

}  // namespace upbp_host
