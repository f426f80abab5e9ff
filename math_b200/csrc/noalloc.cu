// Rendering without device allocation (nt_render_noalloc, include/ntrace.h).
//
// The ordinary nt_render allocates its wavefront path pool with cudaMalloc on first use.  Some
// callers cannot allow that: applications that own every byte of device memory through their own
// allocator or a budget fixed at start-up, plugins running inside such hosts, and frame loops where an
// allocation (which may synchronise the device, or fail under memory pressure) is not permitted
// between frames.  For them this entry point keeps the wavefront's scratch (path queues, hit records,
// shadow-ray queue and counters) in one file-scope __device__ array of NT_NOALLOC_SCRATCH_BYTES; the
// scene's arrays (built beforehand) are the inputs and the caller's accumulator is the output.
// Nothing here calls cudaMalloc, cudaFree, cudaMallocHost, or creates a stream or an event.
//
// Every GPU that loads the library holds the array until the process exits.  With CUDA's lazy module
// loading (the default since CUDA 12.2) the module holding the array is loaded, and its 64 MiB
// reserved, by the first cudaGetSymbolAddress on a device, which the first call on that device makes:
// callers with a fixed budget make that call once at start-up.  All calls share the array and it
// keeps the previous call's contents: the counters are cleared at the start of every call, the
// queues are always written before they are read, and calls that overlap on the GPU (two streams,
// two threads) race on it.
#include "ntrace.h"

#include "device_types.h"
#include "kernels.h"

#include <mutex>
#include <string>

namespace
{
static __device__ __align__(256) unsigned char g_noalloc_scratch[NT_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_lock;
void* g_scratch_ptr[MAX_DEVICES] = {};

// Device address of the scratch array for the current device, looked up once per device with that
// device current (in host code the name g_noalloc_scratch is not a device address).
cudaError_t scratch_for_current_device(void** out)
{
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess)
        {
                return e;
        }
        if (dev < 0 || dev >= MAX_DEVICES)
        {
                return cudaErrorInvalidDevice;
        }
        std::lock_guard lg(g_setup_lock);
        if (!g_scratch_ptr[dev])
        {
                void* p = nullptr;
                e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
                if (e != cudaSuccess)
                {
                        return e;
                }
                g_scratch_ptr[dev] = p;
        }
        *out = g_scratch_ptr[dev];
        return cudaSuccess;
}
}

namespace ntrace
{
// Implemented beside the ordinary render (scene.cpp): checks the scene and options, fills the pass
// constants and runs the wavefront on the given working memory.
int render_with_scratch(nt_scene* scene, const nt_render_opts* opts, double* d_accum, int64_t sample_offset,
                        cudaStream_t stream, void* scratch, size_t scratch_bytes, nt_stats* stats);
int report_error(int code, const std::string& message);
}

extern "C" int nt_render_noalloc(nt_scene* scene, const nt_render_opts* opts, double* d_accum, int64_t sample_offset,
                                 void* stream, nt_stats* stats)
{
        void* scratch = nullptr;
        cudaError_t e = scratch_for_current_device(&scratch);
        if (e != cudaSuccess)
        {
                return ntrace::report_error(NT_ECUDA, std::string("no-alloc scratch set-up (cudaGetSymbolAddress): ") +
                                                              cudaGetErrorString(e));
        }
        return ntrace::render_with_scratch(scene, opts, d_accum, sample_offset, (cudaStream_t)stream, scratch,
                                           NT_NOALLOC_SCRATCH_BYTES, stats);
}
