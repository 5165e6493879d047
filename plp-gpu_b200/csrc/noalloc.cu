// noalloc.cu -- the fixed device scratch of plp_decode_noalloc.
//
// Some callers cannot allocate device memory: code that runs while another
// framework's caching allocator owns the whole device, plugins hosted by a
// runtime that forbids allocation on its request path, or latency-critical
// loops that must not enter the allocator. For them the decoder's scratch
// (instance tables, work list, counters and flags, multi-pass placement rows)
// lives in this file-scope array instead of allocated memory. Every GPU that
// loads the library holds the array until the process exits.
#include <map>
#include <mutex>

#include "device_common.cuh"

namespace plpb {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)8 << 20;   // 8 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of the scratch on the current device. In host code the
// array's name is only a host-side stand-in, so the address is taken with
// cudaGetSymbolAddress once per device (with that device current) and cached.
cudaError_t noalloc_scratch(void** ptr, size_t* bytes) {
    static std::mutex mu;
    static std::map<int, void*> addr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    auto it = addr.find(dev);
    if (it == addr.end()) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        it = addr.emplace(dev, p).first;
    }
    *ptr = it->second;
    *bytes = NOALLOC_SCRATCH_BYTES;
    return cudaSuccess;
}

}  // namespace plpb
