// Peak probes for the rooflines of the tree-walk kernels (nt_probe_peaks, include/ntrace.h).
//
// The walk kernels keep most of their working set (tree nodes, facet records) in the 126 MB L2, and
// their arithmetic is FP32, so besides the HBM copy peak their rooflines need two more ceilings that
// no vendor file states for this part: the L2 read bandwidth and the FP32 FMA rate.  Both are
// measured here with kernels of this library, timed with CUDA events.
//
//  * L2 read: every CTA streams 16-byte loads over a buffer that fits in L2 (32 MiB, read once before
//    the timed launches so it is resident); the loads bypass L1 (ld.global.cg), so every byte comes
//    from L2.  Bytes read / time.
//  * FP32 FMA: every thread runs 8 independent chains of fmaf; 2 flops per FMA / time.
#include "ntrace.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace
{
constexpr int PROBE_BLOCK = 512;

__global__ void k_l2_read(const uint4* __restrict__ buf, long long n16, int passes, unsigned long long* sink)
{
        uint32_t acc = 0;
        const long long stride = (long long)gridDim.x * blockDim.x;
        for (int p = 0; p < passes; ++p)
        {
                for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride)
                {
                        uint4 v;
                        asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
                                     : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                                     : "l"(buf + i));
                        acc ^= v.x ^ v.y ^ v.z ^ v.w;
                }
        }
        if (acc == 0x9e3779b9u)
        {
                atomicAdd(sink, 1ull);  // keeps the loads; practically never taken
        }
}

__global__ void k_fma(int iters, float seed, float* sink)
{
        float a[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
                a[j] = seed + (float)(threadIdx.x + j);
        }
        const float m = 0.999999f, c = 1e-7f;
        for (int i = 0; i < iters; ++i)
        {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                {
                        a[j] = fmaf(a[j], m, c);
                }
        }
        float s = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
                s += a[j];
        }
        if (s == 12345.678f)
        {
                sink[0] = s;
        }
}

struct Events
{
        cudaEvent_t a = nullptr, b = nullptr;
        ~Events()
        {
                if (a)
                {
                        cudaEventDestroy(a);
                }
                if (b)
                {
                        cudaEventDestroy(b);
                }
        }
};
}

namespace ntrace
{
int report_error(int code, const std::string& message);
}

extern "C" int nt_probe_peaks(nt_peaks* out)
{
        if (!out)
        {
                return ntrace::report_error(NT_EINVAL, "nt_probe_peaks: out is NULL");
        }
        int dev = 0, sms = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess)
        {
                e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        }
        const long long bytes = 32ll << 20;
        void* buf = nullptr;
        unsigned long long* sink = nullptr;
        Events ev;
        if (e == cudaSuccess)
        {
                e = cudaMalloc(&buf, bytes);
        }
        if (e == cudaSuccess)
        {
                e = cudaMalloc((void**)&sink, 64);
        }
        if (e == cudaSuccess)
        {
                e = cudaMemset(buf, 1, bytes);
        }
        if (e == cudaSuccess)
        {
                e = cudaEventCreate(&ev.a);
        }
        if (e == cudaSuccess)
        {
                e = cudaEventCreate(&ev.b);
        }
        float l2_ms = 0, fma_ms = 0;
        const int passes = 20;
        const unsigned l2_grid = (unsigned)(std::max(1, sms) * 4);
        const int fma_iters = 1 << 16;
        const unsigned fma_grid = (unsigned)(std::max(1, sms) * 8);
        if (e == cudaSuccess)
        {
                // warm: the buffer resident in L2, the kernels loaded
                k_l2_read<<<l2_grid, PROBE_BLOCK>>>((const uint4*)buf, bytes / 16, 2, sink);
                k_fma<<<fma_grid, PROBE_BLOCK>>>(1 << 10, 1.0f, (float*)sink);
                cudaEventRecord(ev.a);
                k_l2_read<<<l2_grid, PROBE_BLOCK>>>((const uint4*)buf, bytes / 16, passes, sink);
                cudaEventRecord(ev.b);
                e = cudaEventSynchronize(ev.b);
        }
        if (e == cudaSuccess)
        {
                e = cudaEventElapsedTime(&l2_ms, ev.a, ev.b);
        }
        if (e == cudaSuccess)
        {
                cudaEventRecord(ev.a);
                k_fma<<<fma_grid, PROBE_BLOCK>>>(fma_iters, 1.0f, (float*)sink);
                cudaEventRecord(ev.b);
                e = cudaEventSynchronize(ev.b);
        }
        if (e == cudaSuccess)
        {
                e = cudaEventElapsedTime(&fma_ms, ev.a, ev.b);
        }
        if (buf)
        {
                cudaFree(buf);
        }
        if (sink)
        {
                cudaFree(sink);
        }
        if (e != cudaSuccess)
        {
                return ntrace::report_error(NT_ECUDA, std::string("nt_probe_peaks: ") + cudaGetErrorString(e));
        }
        out->l2_read_gbs = (double)bytes * passes / (l2_ms * 1e-3) / 1e9;
        out->fp32_fma_tflops = 2.0 * 8.0 * fma_iters * (double)fma_grid * PROBE_BLOCK / (fma_ms * 1e-3) / 1e12;
        out->l2_ms = l2_ms;
        out->fma_ms = fma_ms;
        return NT_OK;
}
