// render_tree.cuh -- the binary tree the traversal records are built from (see render_tree.cu).
#pragma once
#include <cstddef>

#include <cuda_runtime.h>

#include "lumina.h"

namespace lg
{
size_t render_tree_scratch_bytes(int n_nodes, int n_tris);
// mode 0: d_nodes re-sorted by depth; mode 1: d_nodes' leaves regrouped by
// PLOC, sorted by depth.  d_out holds n_nodes records, root first.  Returns
// an LG_* status (the message in lg_last_error).
int build_render_tree(const lg_bvh_node* d_nodes, int n_nodes, int n_tris, int mode, lg_bvh_node* d_out,
                      void* scratch, size_t scratch_bytes, cudaStream_t stream);
}  // namespace lg
