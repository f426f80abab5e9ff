// Host-side entry points into the sm_100a kernels (kernels.cu).
#pragma once

#include "device_types.h"

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ntrace
{
// Per-kernel device time of one render, measured with CUDA events on the render stream.
struct KernelTimes
{
        double raygen_ms = 0;
        double extend_ms = 0;
        double shade_ms = 0;
        double shadow_ms = 0;
        double plan_ms = 0;  // the plan-and-compact kernels of one-mesh scenes
        long long launches = 0;
        long long extend_launches = 0;
        long long shadow_launches = 0;
        long long extend_rays = 0;
        long long shadow_rays = 0;
};

// Grid sizes of an iteration's kernels (resident blocks on the whole device).
struct LaunchSizes
{
        long long extend_blocks = 1;
        long long shadow_blocks = 1;
        long long extend_refill_blocks[3] = {1, 1, 1};  // per staging chunk: 1, 2, 4 rounds of 32 tests
        long long shadow_refill_blocks[3] = {1, 1, 1};
        long long stream_blocks = 1;
};

// Wavefront path pool: path state A/B (double-buffered, compacted every bounce), the hit record and
// the shadow-ray queue, all carved out of one caller-provided device allocation.
template <int N>
struct Wavefront
{
        long long Q = 0;
        int lights = 1;
        float* fA = nullptr;
        float* fB = nullptr;
        uint32_t* pixA = nullptr;
        uint32_t* pixB = nullptr;
        uint32_t* smpA = nullptr;
        uint32_t* smpB = nullptr;
        int* lvlA = nullptr;
        int* lvlB = nullptr;
        float* hit_t = nullptr;
        int* hit_obj = nullptr;
        int* hit_facet = nullptr;
        float* sq_f = nullptr;
        uint32_t* sq_pix = nullptr;
        // one-mesh scenes: queue indices of the extension rays that walk the tree, and the object plan
        // k_plan_extend found for each (32 bytes), so that the walk kernel does not work it out again
        // (the shadow queue holds only rays that walk, with their entry distance: k_shade plans them)
        int* walk_ext = nullptr;
        void* plan_ext = nullptr;
        // smooth-normal shadow queue (only when some mesh has vertex normals and smooth_normal is set)
        float* sm_f = nullptr;
        uint32_t* sm_pix = nullptr;

        static size_t bytes_for(long long Q, int lights, bool smooth = false);
        void carve(char* base, long long Q, int lights, bool smooth = false);

        // Traces total_paths camera paths starting at P.path_begin into accum (3 doubles per pixel).
        // counters: C_COUNT device int64 (work counters and the wavefront control); host_counters:
        // pinned host mirror of all of them.
        // times: launch counts always, per-kernel device times when timing (events around every
        // launch); stop: optional host flag polled once per wavefront iteration (between launches).
        // The iterations run in batches of `batch` captured as one CUDA graph (use_graph; else enqueued
        // directly), the host reading the done flag after each batch.
        cudaError_t run(const DevScene<N>& S, PassDev P, double* accum, unsigned long long* counters,
                        unsigned long long* host_counters, long long total_paths, cudaStream_t st, KernelTimes* times,
                        bool timing, const volatile int* stop, bool use_graph = true, int batch = 4);

        // One wavefront iteration on stream st (k_iter_begin .. k_iter_end; the queue sizes live in
        // counters, so nothing waits for the host).  parity selects which double-buffered queue is
        // current; ev (8 events, optional) are recorded around the kernel kinds.  Capturable.
        void enqueue_iteration(const DevScene<N>& S, const PassDev& P, double* accum, unsigned long long* counters,
                               long long total_paths, int parity, cudaStream_t st, KernelTimes* times,
                               cudaEvent_t* ev) const;
        static int iteration_launches(bool smooth, bool one_mesh)
        {
                return 6 + (smooth ? 1 : 0) + (one_mesh ? 1 : 0);
        }

        // The iteration kernels' attributes (dynamic shared memory of the walk kernels) and grid sizes,
        // set up on the first call for this dimension.  Call it before capturing iterations into a
        // graph (run() and the batch do).
        static const LaunchSizes& prepare();
};

// Denoiser inputs: first-hit normal and depth of every pixel-centre camera ray; per-pixel mean and
// variance of the mean from a pass rendered with per-path sums (PassDev::moments).
template <int N>
cudaError_t launch_aux(const DevScene<N>& S, long long npix, float* normal, float* depth, cudaStream_t st);
cudaError_t launch_moments_reduce(long long npix, int spp, const double* rad, float* mean, float* var, cudaStream_t st);

// out[j] = rec[idx[j]] for count records of f4 float4s each (the leaves' records in leaf-list order).
cudaError_t launch_gather_records(const float4* rec, const int* idx, long long count, int f4, float4* out,
                                  cudaStream_t st);

// Mean colour per pixel (floats) from the per-pixel sums.
cudaError_t launch_mean(long long n3, const double* sums, long long samples, float* out, cudaStream_t st);

// Viewer feed: width x height words 0x00RRGGBB (sRGB) of the slice whose first pixel is `base`.
cudaError_t launch_srgb_slice(const double* accum, long long samples, long long base, int width, int height,
                              long long row_stride, uint32_t* out, cudaStream_t st);

template <int N>
cudaError_t launch_trace_closest(const MeshDev<N>& M, const float* org, const float* dir, long long nrays, int retest,
                                 int* facet, float* t, unsigned long long* counters, cudaStream_t st);
}
