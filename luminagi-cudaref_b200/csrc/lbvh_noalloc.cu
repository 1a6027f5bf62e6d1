// lbvh_noalloc.cu -- a BVH build entry point that never allocates device memory.
//
// lg_build_bvh_device() takes its scratch (Morton codes, sort buffers, the
// radix-tree arrays, the breadth-first keys) from a pool that grows with
// cudaMalloc.  Some callers cannot allow that: an engine that refreshes the
// BVH inside its frame loop cannot absorb the device-wide synchronisation a
// cudaMalloc/cudaFree may cause, and a host application that reserves all
// device memory up front through its own allocator leaves no room for
// allocations it does not control.  lg_build_bvh_device_noalloc() serves
// them: its scratch is one fixed array in device global memory, defined
// below, so the build itself allocates nothing.
//
// The array holds LG_NOALLOC_MAX_TRIS triangles' worth of scratch (about
// 14 MB); every GPU that loads it keeps it until the process exits.  When it
// is loaded depends on CUDA's module loading: eagerly (CUDA_MODULE_LOADING=
// EAGER) with the library's other device code at context creation; lazily
// (the default since CUDA 12.2) on the first call on each device, when its
// address is looked up.  A host that later reserves all device memory for
// its own allocator should therefore make one call on each device first.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "common.h"
#include "lbvh.cuh"

namespace
{
// Bytes of scratch the build needs for LG_NOALLOC_MAX_TRIS triangles with the
// sorted triangles staged in scratch (the largest layout), rounded up.
constexpr size_t kNoAllocScratchBytes = 14u << 20;

// The shared scratch.  Host code must not use this name as a device address:
// on the host it names a stand-in object.  The device address comes from
// cudaGetSymbolAddress (see scratch_on_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, looked up with the device current on
// the first call on that device and kept once found.  A failed lookup (e.g.
// no memory left for a lazily loaded module) is not kept: the next call on
// that device tries again.
struct DeviceSlot
{
    std::mutex mu;
    void* ptr = nullptr;
};
DeviceSlot g_slots[64];

int scratch_on_device(void** out)
{
    int dev = 0;
    LG_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return lg::set_error(LG_ERR_INVALID, "device ordinal %d not supported", dev);
    DeviceSlot& s = g_slots[dev];
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.ptr)
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
        {
            cudaGetLastError();  // the lookup's error is reported here, not left to a later call
            return lg::set_error(LG_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch): %s", cudaGetErrorString(e));
        }
        s.ptr = p;
    }
    *out = s.ptr;
    return LG_OK;
}
}  // namespace

extern "C" int lg_build_bvh_device_noalloc(const lg_triangle* d_tris, int32_t n_tris, lg_bvh_node* d_nodes_out,
                                           int32_t* n_nodes_out, int32_t* d_perm_out, lg_triangle* d_tris_out,
                                           void* stream)
{
    if (!n_nodes_out || n_tris < 0 || (n_tris > 0 && (!d_tris || !d_nodes_out)))
        return lg::set_error(LG_ERR_INVALID, "lg_build_bvh_device_noalloc: bad argument");
    if (n_tris > LG_NOALLOC_MAX_TRIS)
        return lg::set_error(LG_ERR_CAPACITY,
                             "lg_build_bvh_device_noalloc: %d triangles exceed the fixed scratch limit of %d; "
                             "use lg_build_bvh_device",
                             n_tris, LG_NOALLOC_MAX_TRIS);
    const bool tris_in_scratch = d_tris_out == nullptr || d_tris_out == d_tris;
    const size_t need = lg::lbvh_scratch_bytes(n_tris, tris_in_scratch);
    if (need > kNoAllocScratchBytes)
        return lg::set_error(LG_ERR_CAPACITY, "lg_build_bvh_device_noalloc: needs %zu scratch bytes, has %zu", need,
                             kNoAllocScratchBytes);
    void* scratch = nullptr;
    LG_TRY(scratch_on_device(&scratch));
    int count = 0;
    LG_TRY(lg::lbvh_build(d_tris, n_tris, d_nodes_out, &count, d_perm_out, d_tris_out, scratch,
                          kNoAllocScratchBytes, (cudaStream_t)stream));
    *n_nodes_out = count;
    return LG_OK;
}
