// tild_noalloc.cu -- device scratch for the allocation-free density read-back.
//
// tild_box_get_density_noalloc serves callers that cannot allocate device memory (a
// pool allocator already holds the device's memory, or a cudaFree would synchronise
// streams the caller keeps busy).  It needs the same device scratch as
// tild_box_get_density (a density accumulator, a slot-of-particle table and the group's
// site list) but takes it from one file-scope __device__ array instead of cudaMalloc.
// Every call on a device shares that one array and finds the previous call's contents in
// it; calls that overlap on the same device (two boxes or two host threads) race on it.
#include "tild_device.h"

#include <mutex>

namespace tild {

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Address of g_static_scratch on `device`, looked up once per device (the first call on
// a device makes the lookup, which may load the module: make it outside stream capture).
cudaError_t static_scratch(int device, void **ptr)
{
    constexpr int kMaxDevices = 64;
    static void *addr[kMaxDevices] = {};
    static std::mutex mu;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        addr[device] = p;
    }
    *ptr = addr[device];
    return cudaSuccess;
}

// slot_of[orig[s]] = s: inverse of the slot -> original-id permutation of the sort
__global__ void k_slot_of(const int *__restrict__ orig, int n, int *__restrict__ slot_of)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) slot_of[orig[s]] = s;
}

// sites[k] (original particle ids) -> their current slots
__global__ void k_sites_to_slots(int *__restrict__ sites, int ns, const int *__restrict__ slot_of)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) sites[k] = slot_of[sites[k]];
}

cudaError_t launch_slot_map(const int *orig, int n, int *slot_of, int *sites, int ns, cudaStream_t st)
{
    if (n > 0) k_slot_of<<<(n + 255) / 256, 256, 0, st>>>(orig, n, slot_of);
    if (ns > 0) k_sites_to_slots<<<(ns + 255) / 256, 256, 0, st>>>(sites, ns, slot_of);
    return cudaGetLastError();
}

}  // namespace tild
