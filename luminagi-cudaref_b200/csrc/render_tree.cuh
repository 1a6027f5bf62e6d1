// render_tree.cuh -- the binary tree the traversal records are built from (see render_tree.cu).
#pragma once
#include <cstddef>

#include <cuda_runtime.h>

#include "lumina.h"

namespace lg
{
// Scratch for any mode over a BVH of n_nodes nodes and n_tris triangles.
size_t render_tree_scratch_bytes(int n_nodes, int n_tris);
// Nodes of the render tree of `mode` (n_nodes, or 2 * n_tris - 1 for mode 2).
int render_tree_nodes(int n_nodes, int n_tris, int mode);
// mode 0: d_nodes re-sorted by depth; mode 1: d_nodes' leaves regrouped by
// PLOC; mode 2: PLOC over the triangles (d_tris, BVH order), one per leaf;
// all sorted by depth.  d_out holds render_tree_nodes(...) records, root
// first.  Returns an LG_* status (the message in lg_last_error).
int build_render_tree(const lg_bvh_node* d_nodes, int n_nodes, const lg_triangle* d_tris, int n_tris, int mode,
                      lg_bvh_node* d_out, void* scratch, size_t scratch_bytes, cudaStream_t stream);
}  // namespace lg
