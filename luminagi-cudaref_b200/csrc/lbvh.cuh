// lbvh.cuh -- device LBVH build (see lbvh.cu).
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "lumina.h"

namespace lg
{
// Scratch bytes for n triangles; tris_in_scratch when the sorted triangles
// cannot be written straight to a separate output buffer (in-place or no
// triangle output).
size_t lbvh_scratch_bytes(int n_tris, bool tris_in_scratch);

// Builds the reference BVH for d_tris[0..n) on `stream`.  d_nodes must hold
// max(2n-1, 1) nodes.  d_perm_out / d_tris_out may be null; d_tris_out may
// equal d_tris.  Synchronises the stream to return the node count.
int lbvh_build(const lg_triangle* d_tris, int n, lg_bvh_node* d_nodes, int* n_nodes_host, int32_t* d_perm_out,
               lg_triangle* d_tris_out, void* scratch, size_t scratch_bytes, cudaStream_t stream);
}  // namespace lg
