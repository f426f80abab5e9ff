// sm_100a kernels of the n-space path tracer: the fixed-ray-set closest-hit query and the
// wavefront (ray generation, extension, shading, shadow rays, accumulation) with path and shadow
// queues compacted by warp ballot plus block prefix sums.
#include "device.cuh"
#include "kernels.h"

#include <cuda_runtime.h>

namespace ntrace
{
namespace
{
constexpr int BLOCK = WALK_BLOCK;  // every wavefront kernel's block size
// resident blocks per SM asked of the tree-walk kernels, which caps their registers at 65536 / (5 x
// 128): a few spilled registers at n >= 4 cost less than the extra warps gain (with 256-thread blocks,
// 2 blocks without spills measured faster than 3 or 4 with them)
#ifndef NT_WALK_MIN_BLOCKS
#define NT_WALK_MIN_BLOCKS 5
#endif
constexpr int WALK_MIN_BLOCKS = NT_WALK_MIN_BLOCKS;
// resident blocks per SM asked of the shading kernel (a build-time option): 8 blocks of 128 caps it at
// 64 registers, 32 warps per SM instead of 16 at the 108 it takes uncapped; the kernel is bound by
// latency at that occupancy (ncu: 47 % issue, 13 % of DRAM bandwidth), and the n = 4 frame measured
// 40.5 -> 38.3 ms with the cap despite a few spilled registers
#ifndef NT_SHADE_MIN_BLOCKS
#define NT_SHADE_MIN_BLOCKS 8
#endif
constexpr int SHADE_MIN_BLOCKS = NT_SHADE_MIN_BLOCKS;
// at n = 6 the walk state is larger: one block fewer, so that 128 registers fit without spills
template <int N>
constexpr int walk_min_blocks()
{
        return (N >= 6 && WALK_MIN_BLOCKS > 1) ? WALK_MIN_BLOCKS - 1 : WALK_MIN_BLOCKS;
}
// fill rounds per iteration of the lane-refill walks (1 measured faster than 2, 4, 8 or 16: a lane
// whose new ray needs no walk waits for the next iteration rather than holding up the warp)
#ifndef NT_FILL_ROUNDS
#define NT_FILL_ROUNDS 1
#endif
constexpr int FILL_ROUNDS = NT_FILL_ROUNDS;

__device__ __forceinline__ unsigned lanemask_lt()
{
        unsigned m;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
        return m;
}

// Block-wide stream compaction slot: every thread of the block must call it (flag may be false).
// Warp ballot + popc give the in-warp prefix, a shared-memory scan over warps gives the block
// offset, and one atomic per block reserves the block's range in the output queue.
__device__ __forceinline__ long long compact_slot(bool flag, unsigned long long* counter, int* s_warp, long long* s_base)
{
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        unsigned ballot = __ballot_sync(0xffffffffu, flag);
        if (lane == 0)
        {
                s_warp[warp] = __popc(ballot);
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
                int total = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                {
                        int c = s_warp[w];
                        s_warp[w] = total;
                        total += c;
                }
                *s_base = total ? (long long)atomicAdd(counter, (unsigned long long)total) : 0;
        }
        __syncthreads();
        long long slot = *s_base + s_warp[warp] + __popc(ballot & lanemask_lt());
        __syncthreads();
        return flag ? slot : -1;
}

template <bool SHADOW_KERNEL>
__device__ __forceinline__ void flush_stats(unsigned long long* counters, const WalkStats& ws, long long rays,
                                            long long shadow_rays)
{
        if (!counters)
        {
                return;
        }
        warp_add(counters + (SHADOW_KERNEL ? C_SH_FACET_TESTS : C_FACET_TESTS), ws.facet_tests);
        warp_add(counters + (SHADOW_KERNEL ? C_SH_BOX_STEPS : C_BOX_STEPS), ws.box_steps);
        warp_add(counters + (SHADOW_KERNEL ? C_SH_RETESTS : C_RETESTS), ws.retests);
        warp_add(counters + (SHADOW_KERNEL ? C_SH_DESCENT : C_DESCENT), ws.descent);
        warp_add(counters + C_RAYS, rays);
        warp_add(counters + C_SHADOW_RAYS, shadow_rays);
        if (ws.error)
        {
                atomicOr((unsigned long long*)(counters + C_ERROR), (unsigned long long)ws.error);
        }
}

// ------------------------------------------------------------------------------------------------
// Fixed ray set: closest facet per ray through Mesh::intersect_approximate + intersect_precise
// (the query of src/painter/shapes/test/test_mesh.cpp:139-152).

template <int N>
__global__ void __launch_bounds__(BLOCK) k_trace_closest(__grid_constant__ const MeshDev<N> M, const float* __restrict__ org,
                                                         const float* __restrict__ dir, long long nrays, int retest,
                                                         int* __restrict__ facet_out, float* __restrict__ t_out,
                                                         unsigned long long* counters)
{
        const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        WalkStats ws{0, 0, 0, 0, 0};
        // one ray per lane; the warp walks until all its lanes are done (no early exit: the leaf
        // step is warp-cooperative)
        bool walking = false;
        Walk<N> w;
        w.pc.reset();
        if (i < nrays)
        {
                float o[N], d[N];
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        o[k] = org[i * N + k];
                        d[k] = dir[i * N + k];
                }
                Ray<N> r;
                ray_set<N>(r, o, d);
                float first, second;
                if (root_slabs<N>(M, r.org, r.dir, &first, &second))
                {
                        walk_begin<N>(w, r, (first > 0) ? first : second, FLT_MAX);
                        w.raw = i;
                        walking = true;
                }
                else
                {
                        facet_out[i] = -1;
                        t_out[i] = 0;
                }
        }
        while (__any_sync(0xffffffffu, walking))
        {
                float t = 0;
                int f = -1;
                const int status = walk_step_warp<N>(M, w, walking, retest, org, dir, &t, &f, &ws);
                if (walking && status != W_RUNNING)
                {
                        walking = false;
                        if (status == W_HIT)
                        {
                                if (retest)
                                {
                                        // report the distance of the chosen facet in FP64 (rounded once)
                                        double t64 = retest_facet<N>(M.rec64 + (size_t)f * Rec64<N>::DOUBLES, w.ray,
                                                                     Ray64Source<N>{org, dir, i});
                                        if (t64 > 0)
                                        {
                                                t = (float)t64;
                                        }
                                }
                                facet_out[i] = f;
                                t_out[i] = t;
                        }
                        else
                        {
                                facet_out[i] = -1;
                                t_out[i] = 0;
                        }
                }
        }
        flush_stats<false>(counters, ws, i < nrays ? 1 : 0, 0);
}

// ------------------------------------------------------------------------------------------------
// Wavefront

template <int N>
struct PathView
{
        float* f;        // (2N + 4) x Q: org[N], dir[N], beta[3], color_level
        uint32_t* pix;   // Q
        uint32_t* smp;   // Q: sample index of the pixel (pass offset included)
        int* level;      // Q: bounce level; level > 0 means the ray is a diffuse bounce
        long long Q;

        __device__ __forceinline__ float& at(int field, long long i) const
        {
                return f[field * Q + i];
        }
};

template <int N>
struct HitView
{
        float* t;
        int* obj;
        int* facet;
};

template <int N>
struct ShadowView
{
        float* f;        // (2N + 5) x Q: org[N], dir[N], tmax, contrib[3], entry (scenes with one mesh: the
                         // distance at which the ray enters the mesh's root box)
        uint32_t* pix;
        long long Q;

        __device__ __forceinline__ float& at(int field, long long i) const
        {
                return f[field * Q + i];
        }
};

// paint_pixels: stratified jittered sample -> projector ray (painter.cpp:410-448,
// sampler.h:26-64, engine.h:86-156)
template <int N>
__device__ __forceinline__ void raygen_one(const DevScene<N>& S, const PassDev& P, const PathView<N>& A, long long g,
                                           long long slot)
{
        const long long entry = g / P.spp_eff;
        int s = (int)(g - entry * P.spp_eff);
        const long long pixel = P.list ? P.list[entry] : entry;
        long long sample = P.sample_offset + s;
        unsigned long long path = (unsigned long long)sample * (unsigned long long)P.npix + (unsigned long long)pixel;

        int px[N - 1];
        long long rem = pixel;
#pragma unroll
        for (int j = 0; j < N - 1; ++j)
        {
                px[j] = (int)(rem % S.proj.screen[j]);
                rem /= S.proj.screen[j];
        }
        float u[8];
        float4 a = rng4(P.key0, P.key1, path, 0, 0);
        u[0] = a.x;
        u[1] = a.y;
        u[2] = a.z;
        u[3] = a.w;
        if constexpr (N - 1 > 4)
        {
                float4 b = rng4(P.key0, P.key1, path, 0, 1);
                u[4] = b.x;
        }
        float point[N - 1];
        int r = s;
#pragma unroll
        for (int j = 0; j < N - 1; ++j)
        {
                int digit = r % P.k1d;
                r /= P.k1d;
                float offset = __fdiv_rn((float)digit, (float)P.k1d);
                float sample_j = offset + u[j] * P.recip_k;
                point[j] = (float)px[j] + sample_j;
        }
        Ray<N> ray;
        projector_ray<N>(S.proj, point, ray);
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                A.at(k, slot) = ray.org[k];
                A.at(N + k, slot) = ray.dir[k];
        }
        A.at(2 * N + 0, slot) = 1.0f;
        A.at(2 * N + 1, slot) = 1.0f;
        A.at(2 * N + 2, slot) = 1.0f;
        A.at(2 * N + 3, slot) = 1.0f;
        A.pix[slot] = P.moments ? (uint32_t)g : (uint32_t)entry;
        A.smp[slot] = (uint32_t)sample;
        A.level[slot] = 0;
}

template <int N>
__global__ void __launch_bounds__(BLOCK) k_raygen(__grid_constant__ const DevScene<N> S, const PassDev P, PathView<N> A,
                                                  const unsigned long long* __restrict__ ctl)
{
        // this iteration's fresh paths (k_iter_begin): queue slots base.., pass paths first..
        const long long fresh = (long long)ctl[C_Q_FRESH];
        const long long base = (long long)ctl[C_Q_BASE];
        const long long first = (long long)ctl[C_Q_NEXT] - fresh;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < fresh; i += (long long)gridDim.x * blockDim.x)
        {
                raygen_one<N>(S, P, A, P.path_begin + first + i, base + i);
        }
}

// Persistent warps take 32 consecutive rays at a time from a device counter until the queue is
// exhausted: no block waits for another block's slowest ray, and the grid is sized to the SMs.
__device__ __forceinline__ long long warp_take(unsigned long long* work)
{
        long long base = 0;
        if ((threadIdx.x & 31) == 0)
        {
                base = (long long)atomicAdd(work, 32ull);
        }
        return __shfl_sync(0xffffffffu, base, 0);
}

// extension: closest object per path (ray_intersection over objects, ray_intersection.h:26-105)
template <int N>
__global__ void __launch_bounds__(BLOCK, walk_min_blocks<N>()) k_extend(__grid_constant__ const DevScene<N> S, PathView<N> A, HitView<N> H,
                                                  unsigned long long* counters)
{
        const long long count = (long long)counters[C_Q_ACTIVE];
        WalkStats ws{0, 0, 0, 0, 0};
        long long rays = 0;
        for (long long base = warp_take(counters + C_WORK_EXT); base < count; base = warp_take(counters + C_WORK_EXT))
        {
                long long i = base + (threadIdx.x & 31);
                if (i < count)
                {
                        Ray<N> r;
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                r.org[k] = A.at(k, i);
                                r.dir[k] = A.at(N + k, i);
                        }
                        float t;
                        int obj, facet;
                        if (scene_closest<N>(S, r, &t, &obj, &facet, &ws))
                        {
                                H.t[i] = t;
                                H.obj[i] = obj;
                                H.facet[i] = facet;
                        }
                        else
                        {
                                H.obj[i] = -1;
                        }
                        ++rays;
                }
        }
        flush_stats<false>(counters, ws, rays, 0);
}

__device__ __forceinline__ void accumulate(double* accum, uint32_t pixel, float r, float g, float b)
{
        double* p = accum + (size_t)pixel * 3;
        atomicAdd(p + 0, (double)r);
        atomicAdd(p + 1, (double)g);
        atomicAdd(p + 2, (double)b);
}

// shading: trace_path / direct_diffuse_lighting / diffuse_lighting (painter.cpp:197-397).  A miss
// or an emitting hit adds its colour to the pixel; a diffuse hit emits one shadow ray per light into
// the shadow queue and, below the depth cap, writes its continuation into the next path queue.
template <int N>
__global__ void __launch_bounds__(BLOCK, SHADE_MIN_BLOCKS) k_shade(__grid_constant__ const DevScene<N> S, const PassDev P, PathView<N> A, HitView<N> H,
                                                 PathView<N> B, ShadowView<N> SQ, ShadowView<N> SM, double* accum,
                                                 unsigned long long* counters)
{
        const long long count = (long long)counters[C_Q_ACTIVE];
        __shared__ int s_warp[BLOCK / 32];
        __shared__ long long s_base;
        const bool one_mesh = S.nmesh == 1;
        long long shadow_rays = 0;  // shadow rays planned here (scenes with one mesh)
        const long long tiles = (count + blockDim.x - 1) / blockDim.x;
        for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        {
                long long i = tile * blockDim.x + threadIdx.x;
                bool lit = false;  // diffuse hit whose direct lighting is evaluated
                float beta[3] = {0, 0, 0};
                float sc[3] = {0, 0, 0};
                float ncl = 0;
                float p[N], gn[N], sn[N];
                bool mesh = false;
                bool smooth = false;  // sn holds the interpolated vertex normal (before the flip)
                uint32_t pixel = 0, sample = 0;
                int level = 0;
                int err = 0;
                if (i < count)
                {
                        pixel = A.pix[i];
                        sample = A.smp[i];
                        level = A.level[i];
                        beta[0] = A.at(2 * N + 0, i);
                        beta[1] = A.at(2 * N + 1, i);
                        beta[2] = A.at(2 * N + 2, i);
                        float color_level = A.at(2 * N + 3, i);
                        Ray<N> ray;
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                ray.org[k] = A.at(k, i);
                                ray.dir[k] = A.at(N + k, i);
                        }
                        int obj = H.obj[i];
                        bool diffuse_reflection = level > 0;
                        if (obj < 0)
                        {
                                const float* c = (S.bg_light && diffuse_reflection) ? S.bg_light_color : S.bg_color;
                                accumulate(accum, pixel, beta[0] * c[0], beta[1] * c[1], beta[2] * c[2]);
                        }
                        else
                        {
                                ray_point<N>(ray, H.t[i], p);
                                const ObjDev& ob = S.obj[obj];
                                if (ob.kind == OBJ_MESH)
                                {
                                        const MeshDev<N>& MM = S.mesh[ob.index];
                                        const int facet = H.facet[i];
                                        const float4* rec = MM.rec32 + (size_t)facet * Rec32<N>::F4;
                                        float f4[(N + 3) / 4 * 4];
#pragma unroll
                                        for (int q = 0; q < (N + 3) / 4; ++q)
                                        {
                                                float4 v = __ldg(rec + q);
                                                f4[4 * q + 0] = v.x;
                                                f4[4 * q + 1] = v.y;
                                                f4[4 * q + 2] = v.z;
                                                f4[4 * q + 3] = v.w;
                                        }
#pragma unroll
                                        for (int k = 0; k < N; ++k)
                                        {
                                                gn[k] = f4[k];
                                        }
                                        if (S.smooth_normal && MM.ntype)
                                        {
                                                smooth = smooth_normal<N>(MM, facet, p, sn);
                                        }
                                }
                                else if (ob.kind == OBJ_PLT)
                                {
                                        plt_normal<N>(S.plt[ob.index], p, gn);
                                }
                                else
                                {
#pragma unroll
                                        for (int k = 0; k < N; ++k)
                                        {
                                                gn[k] = S.hplt[ob.index].normal[k];
                                        }
                                }
                                vnormalize<N>(gn);
                                mesh = ob.kind == OBJ_MESH;
                                float dd = vdot<N>(ray.dir, gn);
                                if (!(fabsf(dd) <= 0))
                                {
                                        if (ob.light_source)
                                        {
                                                const float* c = diffuse_reflection ? ob.light_color : ob.color;
                                                accumulate(accum, pixel, beta[0] * c[0], beta[1] * c[1], beta[2] * c[2]);
                                        }
                                        else
                                        {
                                                // only the geometric normal decides the side; the shading
                                                // normal turns with it (painter.cpp:369-373)
                                                if (dd > 0)
                                                {
#pragma unroll
                                                        for (int k = 0; k < N; ++k)
                                                        {
                                                                gn[k] = -gn[k];
                                                                sn[k] = -sn[k];
                                                        }
                                                }
                                                if (!smooth)
                                                {
#pragma unroll
                                                        for (int k = 0; k < N; ++k)
                                                        {
                                                                sn[k] = gn[k];
                                                        }
                                                }
                                                if (ob.diffuse > 0)
                                                {
                                                        sc[0] = ob.diffuse * ob.color[0];
                                                        sc[1] = ob.diffuse * ob.color[1];
                                                        sc[2] = ob.diffuse * ob.color[2];
                                                        ncl = color_level * cmax3(sc);
                                                        lit = ncl >= 1e-4f;
                                                }
                                        }
                                }
                        }
                }

                // direct lighting: one shadow ray per light (block-uniform loop, compacted per light)
                for (int l = 0; l < S.nlights; ++l)
                {
                        bool shadow = false;
                        bool behind = false;  // smooth-normal branch (painter.cpp:238-284)
                        float sh_org[N], sh_dir[N], sh_tmax = 0, sh_c[3] = {0, 0, 0};
                        if (lit)
                        {
                                float lc[3], vec[N];
                                light_properties<N>(S.lights[l], p, lc, vec);
                                if (!(cmax3(lc) < 1e-4f))
                                {
                                        Ray<N> lr;
                                        ray_set<N>(lr, p, vec);
                                        float dln = vdot<N>(lr.dir, sn);
                                        if (dln > 0)
                                        {
                                                // a smooth-shaded mesh point whose geometric side faces away
                                                // from the light takes the smooth-normal branch
                                                behind = mesh && S.smooth_normal && vdot<N>(lr.dir, gn) < 0;
                                                ray_move<N>(lr, S.ray_offset);
                                                float w = S.diffuse_coef * dln;
                                                shadow = !behind;
#pragma unroll
                                                for (int k = 0; k < N; ++k)
                                                {
                                                        sh_org[k] = lr.org[k];
                                                        sh_dir[k] = lr.dir[k];
                                                }
                                                sh_tmax = __fsqrt_rn(vdot<N>(vec, vec));
                                                sh_c[0] = beta[0] * sc[0] * (lc[0] * w);
                                                sh_c[1] = beta[1] * sc[1] * (lc[1] * w);
                                                sh_c[2] = beta[2] * sc[2] * (lc[2] * w);
                                        }
                                }
                        }
                        // scenes with one mesh: the shadow ray's object plan here, on the ray in registers (as
                        // closest_plan does for extension rays): a non-mesh object nearer than the light
                        // occludes it; a ray whose mesh root box starts beyond the light (or is missed) reaches
                        // the light and adds its share now; only the rays that must walk the mesh are queued,
                        // with the distance at which they enter its root box
                        float sh_entry = 0;
                        if (one_mesh && shadow)
                        {
                                ++shadow_rays;
                                Ray<N> r;
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        r.org[k] = sh_org[k];
                                        r.dir[k] = sh_dir[k];
                                }
                                bool occluded = false;
                                bool walk = false;
                                for (int o = 0; o < S.nobj; ++o)
                                {
                                        float a;
                                        if (!obj_approx<N>(S, o, r, &a) || !(a < sh_tmax))
                                        {
                                                continue;
                                        }
                                        if (S.obj[o].kind == OBJ_MESH)
                                        {
                                                walk = true;
                                                sh_entry = a;
                                        }
                                        else
                                        {
                                                occluded = true;
                                        }
                                }
                                walk = walk && !occluded;
                                if (!occluded && !walk)
                                {
                                        accumulate(accum, pixel, sh_c[0], sh_c[1], sh_c[2]);
                                }
                                shadow = walk;
                        }
                        long long qo = compact_slot(shadow, counters + C_SHADOW, s_warp, &s_base);
                        if (shadow)
                        {
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        SQ.at(k, qo) = sh_org[k];
                                        SQ.at(N + k, qo) = sh_dir[k];
                                }
                                SQ.at(2 * N + 0, qo) = sh_tmax;
                                SQ.at(2 * N + 1, qo) = sh_c[0];
                                SQ.at(2 * N + 2, qo) = sh_c[1];
                                SQ.at(2 * N + 3, qo) = sh_c[2];
                                SQ.at(2 * N + 4, qo) = sh_entry;
                                SQ.pix[qo] = pixel;
                        }
                        if (S.smooth_normal)
                        {
                                // block-uniform: every thread of the block takes part in the compaction
                                long long bo = compact_slot(behind, counters + C_SMOOTH, s_warp, &s_base);
                                if (behind)
                                {
#pragma unroll
                                        for (int k = 0; k < N; ++k)
                                        {
                                                SM.at(k, bo) = sh_org[k];
                                                SM.at(N + k, bo) = sh_dir[k];
                                        }
                                        SM.at(2 * N + 0, bo) = sh_tmax;
                                        SM.at(2 * N + 1, bo) = sh_c[0];
                                        SM.at(2 * N + 2, bo) = sh_c[1];
                                        SM.at(2 * N + 3, bo) = sh_c[2];
                                        SM.pix[bo] = pixel;
                                }
                        }
                }

                // diffuse continuation (diffuse_lighting, painter.cpp:298-323)
                bool survive = false;
                float nr_org[N], nr_dir[N];
                if (lit && level < S.max_depth)
                {
                        const unsigned long long px = P.moments ? pixel / (uint32_t)P.spp_eff
                                                                : (P.list ? (unsigned long long)P.list[pixel] : pixel);
                        unsigned long long path = (unsigned long long)sample * (unsigned long long)P.npix + px;
                        float d[N];
                        if (cosine_hemisphere<N>(P.key0, P.key1, path, (uint32_t)(1 + level), sn, d))
                        {
                                Ray<N> dr;
                                ray_set<N>(dr, p, d);
                                if (!(mesh && vdot<N>(dr.dir, gn) <= 0))
                                {
                                        ray_move<N>(dr, S.ray_offset);
                                        survive = true;
#pragma unroll
                                        for (int k = 0; k < N; ++k)
                                        {
                                                nr_org[k] = dr.org[k];
                                                nr_dir[k] = dr.dir[k];
                                        }
                                }
                        }
                        else
                        {
                                err |= ERR_SAMPLING_LIMIT;
                        }
                }
                long long so = compact_slot(survive, counters + C_ACTIVE_OUT, s_warp, &s_base);
                if (survive)
                {
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                B.at(k, so) = nr_org[k];
                                B.at(N + k, so) = nr_dir[k];
                        }
                        B.at(2 * N + 0, so) = beta[0] * sc[0];
                        B.at(2 * N + 1, so) = beta[1] * sc[1];
                        B.at(2 * N + 2, so) = beta[2] * sc[2];
                        B.at(2 * N + 3, so) = ncl;
                        B.pix[so] = pixel;
                        B.smp[so] = sample;
                        B.level[so] = level + 1;
                }
                if (err)
                {
                        atomicOr((unsigned long long*)(counters + C_ERROR), (unsigned long long)err);
                }
        }
        if (one_mesh)
        {
                warp_add(counters + C_SHADOW_RAYS, shadow_rays);
        }
}

// shadow rays: light_source_is_visible (painter.cpp:172-186); visible -> add the light's share
template <int N>
__global__ void __launch_bounds__(BLOCK, walk_min_blocks<N>()) k_shadow(__grid_constant__ const DevScene<N> S, ShadowView<N> SQ, double* accum,
                                                  unsigned long long* counters)
{
        const long long count = (long long)counters[C_SHADOW];
        WalkStats ws{0, 0, 0, 0, 0};
        long long rays = 0;
        for (long long base = warp_take(counters + C_WORK_SH); base < count; base = warp_take(counters + C_WORK_SH))
        {
                long long i = base + (threadIdx.x & 31);
                if (i < count)
                {
                        Ray<N> r;
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                r.org[k] = SQ.at(k, i);
                                r.dir[k] = SQ.at(N + k, i);
                        }
                        float tmax = SQ.at(2 * N, i);
                        if (scene_visible<N>(S, r, tmax, &ws))
                        {
                                accumulate(accum, SQ.pix[i], SQ.at(2 * N + 1, i), SQ.at(2 * N + 2, i), SQ.at(2 * N + 3, i));
                        }
                        ++rays;
                }
        }
        flush_stats<true>(counters, ws, 0, rays);
}

// The smooth-normal branch of direct_diffuse_lighting (painter.cpp:238-284): a smooth-shaded mesh
// point whose geometric side faces away from the light.  The ray to the light (already moved by the
// ray offset) must hit something before the light; the reverse ray must not hit anything nearer than
// that; the light is then tested from just beyond that first hit.  Rare (only meshes with vertex
// normals, only with smooth_normal), so one ray per thread through the general scene functions.
template <int N>
__global__ void __launch_bounds__(BLOCK) k_shadow_smooth(__grid_constant__ const DevScene<N> S, ShadowView<N> SM,
                                                         double* accum, unsigned long long* counters)
{
        WalkStats ws{0, 0, 0, 0, 0};
        long long rays = 0;
        const long long count = (long long)counters[C_SMOOTH];
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        {
                Ray<N> r;
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        r.org[k] = SM.at(k, i);
                        r.dir[k] = SM.at(N + k, i);
                }
                const float dist = SM.at(2 * N, i);
                float t, t_rev;
                int obj, facet;
                rays += 1;
                bool lit = false;
                if (scene_closest<N>(S, r, &t, &obj, &facet, &ws) && t < dist)
                {
                        Ray<N> rev;
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                rev.org[k] = r.org[k];
                                rev.dir[k] = -r.dir[k];
                        }
                        ray_move<N>(rev, 2 * S.ray_offset);
                        rays += 1;
                        if (!(scene_closest<N>(S, rev, &t_rev, &obj, &facet, &ws) && t_rev < t))
                        {
                                ray_move<N>(r, t + S.ray_offset);
                                rays += 1;
                                lit = scene_visible<N>(S, r, dist - t, &ws);
                        }
                }
                if (lit)
                {
                        accumulate(accum, SM.pix[i], SM.at(2 * N + 1, i), SM.at(2 * N + 2, i), SM.at(2 * N + 3, i));
                }
        }
        flush_stats<true>(counters, ws, 0, rays);
}

// Lane-level refill: every lane that has no ray takes the next one from the queue (one atomic per
// warp for all of them), and every lane with a ray advances it by one tree leaf.  Returns, for each
// lane, the queue index it took (-1: none); the warp knows the queue is drained when `exhausted`.
__device__ __forceinline__ long long lane_refill(bool idle, unsigned long long* work, long long count, bool* exhausted)
{
        const unsigned full = 0xffffffffu;
        unsigned need = __ballot_sync(full, idle);
        if (!need || *exhausted)
        {
                return -1;
        }
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(need) - 1;
        const int cnt = __popc(need);
        long long base = 0;
        if (lane == leader)
        {
                base = (long long)atomicAdd(work, (unsigned long long)cnt);
        }
        base = __shfl_sync(full, base, leader);
        if (base + cnt >= count)
        {
                *exhausted = true;
        }
        if (!idle)
        {
                return -1;
        }
        long long j = base + __popc(need & lanemask_lt());
        return j < count ? j : -1;
}

// Appends this lane's queue index to a walk list when `walk` (one atomic per warp; the lanes of a warp
// keep their order) and returns its list position (-1 without `walk`).  Every lane of the warp calls it.
__device__ __forceinline__ long long list_append(bool walk, long long i, int* list, unsigned long long* count)
{
        const unsigned m = __ballot_sync(0xffffffffu, walk);
        if (!m)
        {
                return -1;
        }
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(m) - 1;
        unsigned long long base = 0;
        if (lane == leader)
        {
                base = atomicAdd(count, (unsigned long long)__popc(m));
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        if (!walk)
        {
                return -1;
        }
        const long long q = (long long)base + __popc(m & lanemask_lt());
        list[q] = (int)i;
        return q;
}

static_assert(sizeof(ClosestPlan) <= 32, "a listed ray's plan takes 32 bytes");

// Extension rays of a scene with one mesh, first pass: every ray's objects (closest_plan); the rays
// that need no tree walk are finished here (their hit record written), the others are compacted into
// the walk list for k_extend_refill, so that its lanes only ever hold rays that walk.
template <int N>
__global__ void __launch_bounds__(BLOCK) k_plan_extend(__grid_constant__ const DevScene<N> S, PathView<N> A, HitView<N> H,
                                                       int* __restrict__ list, ClosestPlan* __restrict__ plans,
                                                       unsigned long long* counters)
{
        const long long count = (long long)counters[C_Q_ACTIVE];
        const int lane = threadIdx.x & 31;
        const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
        long long rays = 0;
        for (long long w0 = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; w0 < count;
             w0 += warps * 32)
        {
                const long long i = w0 + lane;
                bool walk = false;
                ClosestPlan plan;
                if (i < count)
                {
                        ++rays;
                        Ray<N> r;
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                r.org[k] = A.at(k, i);
                                r.dir[k] = A.at(N + k, i);
                        }
                        closest_plan<N>(S, r, &plan);
                        walk = plan.walk;
                        if (!walk)
                        {
                                if (plan.pre_obj >= 0)
                                {
                                        H.t[i] = plan.pre_t;
                                        H.obj[i] = plan.pre_obj;
                                        H.facet[i] = -1;
                                }
                                else
                                {
                                        H.obj[i] = -1;
                                }
                        }
                }
                const long long q = list_append(walk, i, list, counters + C_WALK_EXT);
                if (q >= 0)
                {
                        plans[q] = plan;
                }
        }
        warp_add(counters + C_RAYS, rays);
}

// Extension rays of a scene with one mesh that walk the tree (the plan kernel's list, with each ray's
// closest_plan beside it), one leaf per iteration.
// R: rounds of 32 pooled facet tests staged per warp chunk (Stage<N, R>).
template <int N, int R>
__global__ void __launch_bounds__(BLOCK, walk_min_blocks<N>())
        k_extend_refill(__grid_constant__ const DevScene<N> S, PathView<N> A, HitView<N> H, const int* __restrict__ list,
                        const ClosestPlan* __restrict__ plans, unsigned long long* counters)
{
        const long long count = (long long)counters[C_WALK_EXT];
        const MeshDev<N>& M = S.mesh[0];
        WalkStats ws{0, 0, 0, 0, 0};
        long long rays = 0;
        long long i = -1;
        bool exhausted = false;
        Walk<N> w;
        w.pc.reset();
        ClosestPlan plan;
        while (true)
        {
                // fill: every listed ray walks (the plan kernel finished the others), so one round fills
                // every idle lane while rays remain
                for (int round = 0; round < FILL_ROUNDS; ++round)
                {
                        const long long q = lane_refill(i < 0, counters + C_WORK_EXT, count, &exhausted);
                        if (q >= 0)
                        {
                                const long long j = list[q];
                                Ray<N> r;
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        r.org[k] = A.at(k, j);
                                        r.dir[k] = A.at(N + k, j);
                                }
                                plan = plans[q];  // listed rays have plan.walk set
                                walk_begin<N>(w, r, plan.mesh_t, FLT_MAX);
                                i = j;
                        }
                        if (exhausted || !__any_sync(0xffffffffu, i < 0))
                        {
                                break;
                        }
                }
                if (!__any_sync(0xffffffffu, i >= 0))
                {
                        if (exhausted)
                        {
                                break;
                        }
                        continue;
                }
                {
                        float t = 0;
                        int f = -1;
                        int status = walk_step_warp<N, R>(M, w, i >= 0, S.retest, nullptr, nullptr, &t, &f, &ws, S.walk_small);
                        if (i >= 0 && status != W_RUNNING)
                        {
                                float tt;
                                int obj, fct;
                                closest_finish(plan, status == W_HIT, t, f, &tt, &obj, &fct);
                                if (obj >= 0)
                                {
                                        H.t[i] = tt;
                                        H.obj[i] = obj;
                                        H.facet[i] = fct;
                                }
                                else
                                {
                                        H.obj[i] = -1;
                                }
                                i = -1;
                        }
                }
        }
        flush_stats<false>(counters, ws, rays, 0);
}

// Shadow rays of a scene with one mesh that walk the tree (k_shade queued only those, with the distance
// at which each ray enters the mesh's root box): the walk runs up to the light's distance.
template <int N, int R>
__global__ void __launch_bounds__(BLOCK, walk_min_blocks<N>())
        k_shadow_refill(__grid_constant__ const DevScene<N> S, ShadowView<N> SQ, double* accum, unsigned long long* counters)
{
        const long long count = (long long)counters[C_SHADOW];
        const MeshDev<N>& M = S.mesh[0];
        WalkStats ws{0, 0, 0, 0, 0};
        long long rays = 0;
        long long i = -1;
        bool exhausted = false;
        Walk<N> w;
        w.pc.reset();
        float dist = 0;
        while (true)
        {
                for (int round = 0; round < FILL_ROUNDS; ++round)
                {
                        const long long q = lane_refill(i < 0, counters + C_WORK_SH, count, &exhausted);
                        if (q >= 0)
                        {
                                const long long j = q;
                                Ray<N> r;
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        r.org[k] = SQ.at(k, j);
                                        r.dir[k] = SQ.at(N + k, j);
                                }
                                // queued by k_shade: nothing nearer than the light occludes it, and the mesh's
                                // root box starts before the light at the stored entry distance
                                const float dj = SQ.at(2 * N, j);
                                walk_begin<N>(w, r, SQ.at(2 * N + 4, j), dj);
                                dist = dj;
                                i = j;
                        }
                        if (exhausted || !__any_sync(0xffffffffu, i < 0))
                        {
                                break;
                        }
                }
                if (!__any_sync(0xffffffffu, i >= 0))
                {
                        if (exhausted)
                        {
                                break;
                        }
                        continue;
                }
                {
                        float t = 0;
                        int f = -1;
                        int status = walk_step_warp<N, R>(M, w, i >= 0, S.retest, nullptr, nullptr, &t, &f, &ws, S.walk_small);
                        if (i >= 0 && status != W_RUNNING)
                        {
                                if (!(status == W_HIT && t < dist))
                                {
                                        accumulate(accum, SQ.pix[i], SQ.at(2 * N + 1, i), SQ.at(2 * N + 2, i),
                                                   SQ.at(2 * N + 3, i));
                                }
                                i = -1;
                        }
                }
        }
        flush_stats<true>(counters, ws, 0, rays);
}

// ------------------------------------------------------------------------------------------------
// Denoiser inputs

// First hit of the pixel-centre camera ray: geometric normal turned towards the camera (as the
// shading normal of trace_path, painter.cpp:369-373) and distance; zeros on a miss.
template <int N>
__global__ void __launch_bounds__(BLOCK) k_aux(__grid_constant__ const DevScene<N> S, long long npix,
                                               float* __restrict__ normal, float* __restrict__ depth)
{
        const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        WalkStats ws{0, 0, 0, 0, 0};
        if (i >= npix)
        {
                return;
        }
        float point[N - 1];
        long long rem = i;
#pragma unroll
        for (int j = 0; j < N - 1; ++j)
        {
                point[j] = (float)(rem % S.proj.screen[j]) + 0.5f;
                rem /= S.proj.screen[j];
        }
        Ray<N> ray;
        projector_ray<N>(S.proj, point, ray);
        float t;
        int obj, facet;
        float gn[N];
        float d = 0;
        if (scene_closest<N>(S, ray, &t, &obj, &facet, &ws))
        {
                float p[N];
                ray_point<N>(ray, t, p);
                const ObjDev& ob = S.obj[obj];
                if (ob.kind == OBJ_MESH)
                {
                        const float4* rec = S.mesh[ob.index].rec32 + (size_t)facet * Rec32<N>::F4;
                        float f4[(N + 3) / 4 * 4];
#pragma unroll
                        for (int q = 0; q < (N + 3) / 4; ++q)
                        {
                                float4 v = __ldg(rec + q);
                                f4[4 * q + 0] = v.x;
                                f4[4 * q + 1] = v.y;
                                f4[4 * q + 2] = v.z;
                                f4[4 * q + 3] = v.w;
                        }
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                gn[k] = f4[k];
                        }
                }
                else if (ob.kind == OBJ_PLT)
                {
                        plt_normal<N>(S.plt[ob.index], p, gn);
                }
                else
                {
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                gn[k] = S.hplt[ob.index].normal[k];
                        }
                }
                vnormalize<N>(gn);
                if (vdot<N>(ray.dir, gn) > 0)
                {
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                gn[k] = -gn[k];
                        }
                }
                d = t;
        }
        else
        {
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        gn[k] = 0;
                }
        }
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                normal[i * N + k] = gn[k];
        }
        depth[i] = d;
}

// Per-pixel mean and variance of the mean from per-path sums (path index pixel * spp + sample):
// mean = sum / spp, var = (sum of squares - spp mean^2) / (spp - 1) / spp (0 for one sample).
__global__ void k_moments_reduce(long long npix, int spp, const double* __restrict__ rad, float* __restrict__ mean,
                                 float* __restrict__ var)
{
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix * 3; i += (long long)gridDim.x * blockDim.x)
        {
                const long long p = i / 3;
                const int c = (int)(i - p * 3);
                double s1 = 0, s2 = 0;
                for (int k = 0; k < spp; ++k)
                {
                        const double v = rad[((size_t)p * spp + k) * 3 + c];
                        s1 += v;
                        s2 += v * v;
                }
                const double m = s1 / spp;
                mean[i] = (float)m;
                var[i] = spp > 1 ? (float)(fmax(s2 - spp * m * m, 0.0) / (spp - 1) / spp) : 0.0f;
        }
}

// Start of a wavefront iteration (one thread): refill the queue with fresh paths up to Q and clear the
// per-iteration counters.
__global__ void k_iter_begin(unsigned long long* c, long long total, long long Q)
{
        const long long active = (long long)c[C_Q_ACTIVE];
        const long long next = (long long)c[C_Q_NEXT];
        long long fresh = Q - active < total - next ? Q - active : total - next;
        fresh = fresh > 0 ? fresh : 0;
        c[C_Q_BASE] = (unsigned long long)active;
        c[C_Q_FRESH] = (unsigned long long)fresh;
        c[C_Q_ACTIVE] = (unsigned long long)(active + fresh);
        c[C_Q_NEXT] = (unsigned long long)(next + fresh);
        c[C_WORK_EXT] = 0;
        c[C_WORK_SH] = 0;
        c[C_ACTIVE_OUT] = 0;
        c[C_SHADOW] = 0;
        c[C_SMOOTH] = 0;
        c[C_WALK_EXT] = 0;
        if (active + fresh > 0)
        {
                c[C_ITERS] += 1;
        }
}

// End of an iteration (one thread): the continuations become the queue; done once every path of the
// pass has been generated and finished.
__global__ void k_iter_end(unsigned long long* c, long long total)
{
        const long long survivors = (long long)c[C_ACTIVE_OUT];
        c[C_Q_ACTIVE] = (unsigned long long)survivors;
        c[C_DONE] = (survivors == 0 && (long long)c[C_Q_NEXT] >= total) ? 1ull : 0ull;
}

// ------------------------------------------------------------------------------------------------
// Viewer feed: the running mean of a 2-D slice of the screen as 0x00RRGGBB words, as the painter
// window stores a pixel (PainterWindow::set_pixel, painter_window.cpp:140-153) with
// rgb_float_to_srgb_uint8 (com/color/conversion.cpp:35-42,211-230,344-347); the window's row order
// (pixel[1] = height - 1 - y, painter_window.cpp:126-131) puts screen row height - 1 first.

__device__ __forceinline__ unsigned srgb8(float c)
{
        float s;
        if (c >= 1.0f)
        {
                s = 1.0f;
        }
        else if (c >= 0.0031308f)
        {
                s = 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
        }
        else if (c > 0.0f)
        {
                s = c * 12.92f;
        }
        else
        {
                s = 0.0f;
        }
        return (unsigned)(unsigned char)(s * 255.0f + 0.5f);
}

__global__ void k_srgb_slice(const double* __restrict__ accum, double inv_samples, long long base, int width, int height,
                             long long row_stride, uint32_t* __restrict__ out)
{
        const long long count = (long long)width * height;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        {
                const int x = (int)(i % width);
                const int y = (int)(i / width);
                const long long p = base + x + (long long)(height - 1 - y) * row_stride;
                const float r = (float)(accum[p * 3] * inv_samples);
                const float g = (float)(accum[p * 3 + 1] * inv_samples);
                const float b = (float)(accum[p * 3 + 2] * inv_samples);
                out[i] = (srgb8(r) << 16) | (srgb8(g) << 8) | srgb8(b);
        }
}

template <int N>
long long grid_for(long long count)
{
        return (count + BLOCK - 1) / BLOCK;
}

// Resident blocks of a persistent kernel on this device (all SMs, as many blocks per SM as its
// registers and shared memory allow).
template <typename K>
long long resident_blocks(K kernel, int dynamic_smem = 0)
{
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (dynamic_smem > 0)
        {
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dynamic_smem);
        }
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, BLOCK, dynamic_smem);
        return (long long)std::max(1, sms) * std::max(1, per_sm);
}
}

// ------------------------------------------------------------------------------------------------
// Host-side launchers

template <int N>
size_t Wavefront<N>::bytes_for(long long Q, int lights, bool smooth)
{
        size_t per_path = sizeof(float) * (2 * N + 4) * 2  // path state A and B
                          + sizeof(uint32_t) * 2 * 2 + sizeof(int) * 2
                          + sizeof(float) + sizeof(int) * 2  // hit record
                          + (sizeof(float) * (2 * N + 5) + sizeof(uint32_t)) * (size_t)lights * (smooth ? 2 : 1)  // shadow queues
                          + sizeof(int) + 32;  // the extension walk list and its rays' plans
        return per_path * (size_t)Q + 20 * 256;
}

template <int N>
void Wavefront<N>::carve(char* base, long long Q, int lights, bool smooth)
{
        this->Q = Q;
        this->lights = lights;
        auto take = [&](size_t bytes) {
                char* p = base;
                base += (bytes + 255) / 256 * 256;
                return p;
        };
        fA = (float*)take(sizeof(float) * (2 * N + 4) * Q);
        fB = (float*)take(sizeof(float) * (2 * N + 4) * Q);
        pixA = (uint32_t*)take(sizeof(uint32_t) * Q);
        pixB = (uint32_t*)take(sizeof(uint32_t) * Q);
        smpA = (uint32_t*)take(sizeof(uint32_t) * Q);
        smpB = (uint32_t*)take(sizeof(uint32_t) * Q);
        lvlA = (int*)take(sizeof(int) * Q);
        lvlB = (int*)take(sizeof(int) * Q);
        hit_t = (float*)take(sizeof(float) * Q);
        hit_obj = (int*)take(sizeof(int) * Q);
        hit_facet = (int*)take(sizeof(int) * Q);
        sq_f = (float*)take(sizeof(float) * (2 * N + 5) * Q * lights);
        sq_pix = (uint32_t*)take(sizeof(uint32_t) * Q * lights);
        walk_ext = (int*)take(sizeof(int) * Q);
        plan_ext = take(32 * Q);
        if (smooth)
        {
                sm_f = (float*)take(sizeof(float) * (2 * N + 5) * Q * lights);
                sm_pix = (uint32_t*)take(sizeof(uint32_t) * Q * lights);
        }
        else
        {
                sm_f = nullptr;
                sm_pix = nullptr;
        }
}

// The walk kernels' variant when the options leave it open: facet records read straight from global
// memory (measured faster than staging them through shared memory on the configuration scenes, whose
// leaves hold one or two facets per visit on average, so a warp's pooled list rarely fills a chunk).
template <int N>
constexpr int DEFAULT_WALK_ROUNDS = -1;

// Resident blocks of every kernel of an iteration, and the dynamic shared memory of the walk kernels
// (they stage facet records there, leaf_closest_warp): computed once per dimension, on the first call,
// which the host makes before any capture (prepare_pass, nt_render_noalloc).
template <int N>
const LaunchSizes& Wavefront<N>::prepare()
{
        static const LaunchSizes sizes = []() {
                LaunchSizes z;
                z.extend_blocks = resident_blocks(k_extend<N>);
                z.shadow_blocks = resident_blocks(k_shadow<N>);
                z.extend_refill_blocks[0] = resident_blocks(k_extend_refill<N, 0>, Stage<N, 0>::BYTES);
                z.extend_refill_blocks[1] = resident_blocks(k_extend_refill<N, 1>, Stage<N, 1>::BYTES);
                z.extend_refill_blocks[2] = resident_blocks(k_extend_refill<N, 2>, Stage<N, 2>::BYTES);
                z.extend_refill_blocks[3] = resident_blocks(k_extend_refill<N, 4>, Stage<N, 4>::BYTES);
                z.shadow_refill_blocks[0] = resident_blocks(k_shadow_refill<N, 0>, Stage<N, 0>::BYTES);
                z.shadow_refill_blocks[1] = resident_blocks(k_shadow_refill<N, 1>, Stage<N, 1>::BYTES);
                z.shadow_refill_blocks[2] = resident_blocks(k_shadow_refill<N, 2>, Stage<N, 2>::BYTES);
                z.shadow_refill_blocks[3] = resident_blocks(k_shadow_refill<N, 4>, Stage<N, 4>::BYTES);
                z.stream_blocks = resident_blocks(k_shade<N>);
                return z;
        }();
        return sizes;
}

template <int N>
void Wavefront<N>::enqueue_iteration(const DevScene<N>& S, const PassDev& P, double* accum, unsigned long long* counters,
                                     long long total_paths, int parity, cudaStream_t st, KernelTimes* times,
                                     cudaEvent_t* ev) const
{
        const LaunchSizes& L = prepare();
        const long long extend_blocks = L.extend_blocks;
        const long long shadow_blocks = L.shadow_blocks;
        // the walk kernels' variant: records read directly (walk_rounds -1), or staged in chunks of 1, 2
        // or 4 rounds of 32 pooled tests per warp
        const int rounds = S.walk_rounds != 0 ? S.walk_rounds : DEFAULT_WALK_ROUNDS<N>;
        const int vi = rounds < 0 ? 0 : (rounds >= 4 ? 3 : (rounds >= 2 ? 2 : 1));
        const long long extend_refill_blocks = L.extend_refill_blocks[vi];
        const long long shadow_refill_blocks = L.shadow_refill_blocks[vi];
        const long long stream_blocks = L.stream_blocks;
        // scenes with exactly one mesh use the lane-refill walk kernels
        const bool one_mesh = S.nmesh == 1;
        const bool smooth = S.smooth_normal != 0;
        const long long walk_cap = std::max<long long>(1, (Q * lights + BLOCK - 1) / BLOCK);
        const unsigned ext_grid = (unsigned)std::min(one_mesh ? extend_refill_blocks : extend_blocks, walk_cap);
        const unsigned sh_grid = (unsigned)std::min(one_mesh ? shadow_refill_blocks : shadow_blocks, walk_cap);
        const unsigned str_grid = (unsigned)std::min(stream_blocks * 2, walk_cap);
        const bool flip = parity != 0;
        float* fa = flip ? fB : fA;
        float* fb = flip ? fA : fB;
        PathView<N> A{fa, flip ? pixB : pixA, flip ? smpB : smpA, flip ? lvlB : lvlA, Q};
        PathView<N> B{fb, flip ? pixA : pixB, flip ? smpA : smpB, flip ? lvlA : lvlB, Q};
        HitView<N> H{hit_t, hit_obj, hit_facet};
        ShadowView<N> SQ{sq_f, sq_pix, Q * lights};
        ShadowView<N> SM{sm_f, sm_pix, Q * lights};
        k_iter_begin<<<1, 1, 0, st>>>(counters, total_paths, Q);
        if (ev)
        {
                cudaEventRecord(ev[0], st);
        }
        k_raygen<N><<<str_grid, BLOCK, 0, st>>>(S, P, A, counters);
        if (ev)
        {
                cudaEventRecord(ev[1], st);
        }
        if (one_mesh)
        {
                // rays that need no walk are finished by the plan kernel; the walk kernel takes the rest
                k_plan_extend<N><<<str_grid, BLOCK, 0, st>>>(S, A, H, walk_ext, (ClosestPlan*)plan_ext, counters);
        }
        if (ev)
        {
                cudaEventRecord(ev[2], st);
        }
        if (one_mesh)
        {
                if (vi == 0)
                {
                        k_extend_refill<N, 0><<<ext_grid, BLOCK, 0, st>>>(S, A, H, walk_ext, (const ClosestPlan*)plan_ext, counters);
                }
                else if (vi == 1)
                {
                        k_extend_refill<N, 1><<<ext_grid, BLOCK, Stage<N, 1>::BYTES, st>>>(S, A, H, walk_ext, (const ClosestPlan*)plan_ext, counters);
                }
                else if (vi == 2)
                {
                        k_extend_refill<N, 2><<<ext_grid, BLOCK, Stage<N, 2>::BYTES, st>>>(S, A, H, walk_ext, (const ClosestPlan*)plan_ext, counters);
                }
                else
                {
                        k_extend_refill<N, 4><<<ext_grid, BLOCK, Stage<N, 4>::BYTES, st>>>(S, A, H, walk_ext, (const ClosestPlan*)plan_ext, counters);
                }
        }
        else
        {
                k_extend<N><<<ext_grid, BLOCK, 0, st>>>(S, A, H, counters);
        }
        if (ev)
        {
                cudaEventRecord(ev[3], st);
        }
        k_shade<N><<<str_grid, BLOCK, 0, st>>>(S, P, A, H, B, SQ, SM, accum, counters);
        if (ev)
        {
                cudaEventRecord(ev[4], st);
        }
        if (ev)
        {
                cudaEventRecord(ev[5], st);
        }
        if (one_mesh)
        {
                if (vi == 0)
                {
                        k_shadow_refill<N, 0><<<sh_grid, BLOCK, 0, st>>>(S, SQ, accum, counters);
                }
                else if (vi == 1)
                {
                        k_shadow_refill<N, 1><<<sh_grid, BLOCK, Stage<N, 1>::BYTES, st>>>(S, SQ, accum, counters);
                }
                else if (vi == 2)
                {
                        k_shadow_refill<N, 2><<<sh_grid, BLOCK, Stage<N, 2>::BYTES, st>>>(S, SQ, accum, counters);
                }
                else
                {
                        k_shadow_refill<N, 4><<<sh_grid, BLOCK, Stage<N, 4>::BYTES, st>>>(S, SQ, accum, counters);
                }
        }
        else
        {
                k_shadow<N><<<sh_grid, BLOCK, 0, st>>>(S, SQ, accum, counters);
        }
        if (smooth)
        {
                k_shadow_smooth<N><<<str_grid, BLOCK, 0, st>>>(S, SM, accum, counters);
        }
        if (ev)
        {
                cudaEventRecord(ev[6], st);
        }
        k_iter_end<<<1, 1, 0, st>>>(counters, total_paths);
        if (times)
        {
                times->launches += iteration_launches(smooth, one_mesh);
                times->extend_launches += 1;
                times->shadow_launches += 1;
        }
}

template <int N>
cudaError_t Wavefront<N>::run(const DevScene<N>& S, PassDev P, double* accum, unsigned long long* counters,
                              unsigned long long* host_counters, long long total_paths, cudaStream_t st, KernelTimes* times,
                              bool timing, const volatile int* stop, bool use_graph, int batch)
{
        const bool smooth = S.smooth_normal != 0;
        if (smooth && !sm_f)
        {
                return cudaErrorInvalidValue;  // the pool was carved without the smooth-normal queue
        }
        prepare();  // kernel attributes and occupancy, outside the capture below
        // iterations between host checks of the done flag (a pass takes tens of iterations; the few
        // that run after it is done find empty queues and return at once)
        const int BATCH = std::max(1, batch);
        cudaError_t e = cudaMemsetAsync(counters + C_Q_ACTIVE, 0, (C_COUNT - C_Q_ACTIVE) * sizeof(unsigned long long), st);
        if (e != cudaSuccess)
        {
                return e;
        }
        cudaGraphExec_t exec = nullptr;
        if (use_graph && !timing)
        {
                // the BATCH iterations are captured once per pass and replayed as one graph launch
                // (BATCH even, so that the queue parity is the same at the start of every replay)
                const int even = BATCH + (BATCH & 1);
                cudaGraph_t graph = nullptr;
                e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess)
                {
                        for (int k = 0; k < even; ++k)
                        {
                                enqueue_iteration(S, P, accum, counters, total_paths, k & 1, st, nullptr, nullptr);
                        }
                        e = cudaStreamEndCapture(st, &graph);
                        if (e == cudaSuccess)
                        {
                                e = cudaGraphInstantiate(&exec, graph, 0);
                                cudaGraphDestroy(graph);
                        }
                }
                if (e != cudaSuccess)
                {
                        // capture unavailable (e.g. the caller's stream is itself being captured):
                        // enqueue the iterations directly
                        cudaGetLastError();
                        exec = nullptr;
                        e = cudaSuccess;
                }
        }
        cudaEvent_t ev[8];
        if (timing)
        {
                for (auto& v : ev)
                {
                        cudaEventCreate(&v);
                }
        }
        const int per_replay = BATCH + (BATCH & 1);
        int parity = 0;
        while (true)
        {
                if (stop && *stop)
                {
                        break;
                }
                if (timing)
                {
                        for (int k = 0; k < BATCH; ++k)
                        {
                                enqueue_iteration(S, P, accum, counters, total_paths, parity, st, times, ev);
                                parity ^= 1;
                                cudaEventRecord(ev[7], st);
                                cudaEventSynchronize(ev[7]);
                                float ms;
                                cudaEventElapsedTime(&ms, ev[0], ev[1]);
                                times->raygen_ms += ms;
                                cudaEventElapsedTime(&ms, ev[1], ev[2]);
                                times->plan_ms += ms;
                                cudaEventElapsedTime(&ms, ev[2], ev[3]);
                                times->extend_ms += ms;
                                cudaEventElapsedTime(&ms, ev[3], ev[4]);
                                times->shade_ms += ms;
                                cudaEventElapsedTime(&ms, ev[4], ev[5]);
                                times->plan_ms += ms;
                                cudaEventElapsedTime(&ms, ev[5], ev[6]);
                                times->shadow_ms += ms;
                        }
                }
                else if (exec)
                {
                        e = cudaGraphLaunch(exec, st);
                        if (e != cudaSuccess)
                        {
                                break;
                        }
                        times->launches += (long long)per_replay * iteration_launches(smooth, S.nmesh == 1);
                        times->extend_launches += per_replay;
                        times->shadow_launches += per_replay;
                }
                else
                {
                        for (int k = 0; k < BATCH; ++k)
                        {
                                enqueue_iteration(S, P, accum, counters, total_paths, parity, st, times, nullptr);
                                parity ^= 1;
                        }
                }
                e = cudaMemcpyAsync(host_counters, counters, C_COUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess)
                {
                        e = cudaStreamSynchronize(st);
                }
                if (e != cudaSuccess || host_counters[C_DONE] || host_counters[C_ERROR])
                {
                        break;
                }
        }
        if (exec)
        {
                cudaGraphExecDestroy(exec);
        }
        if (timing)
        {
                for (auto& v : ev)
                {
                        cudaEventDestroy(v);
                }
        }
        if (e != cudaSuccess)
        {
                return e;
        }
        return cudaGetLastError();
}

template <int N>
cudaError_t launch_trace_closest(const MeshDev<N>& M, const float* org, const float* dir, long long nrays, int retest,
                                 int* facet, float* t, unsigned long long* counters, cudaStream_t st)
{
        if (nrays <= 0)
        {
                return cudaSuccess;
        }
        static const bool smem_set =
                cudaFuncSetAttribute(k_trace_closest<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, Stage<N>::BYTES) ==
                cudaSuccess;
        if (!smem_set)
        {
                return cudaErrorInvalidValue;
        }
        k_trace_closest<N><<<(unsigned)grid_for<N>(nrays), BLOCK, Stage<N>::BYTES, st>>>(M, org, dir, nrays, retest, facet, t,
                                                                                         counters);
        return cudaGetLastError();
}

template <int N>
cudaError_t launch_aux(const DevScene<N>& S, long long npix, float* normal, float* depth, cudaStream_t st)
{
        if (npix <= 0)
        {
                return cudaSuccess;
        }
        k_aux<N><<<(unsigned)grid_for<N>(npix), BLOCK, 0, st>>>(S, npix, normal, depth);
        return cudaGetLastError();
}

// out[j] = rec[idx[j]] for records of f4 float4s (the leaves' records in leaf-list order)
__global__ void k_gather_records(const float4* __restrict__ rec, const int* __restrict__ idx, long long count, int f4,
                                 float4* __restrict__ out)
{
        const long long total = count * f4;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
                const long long j = i / f4;
                const int q = (int)(i - j * f4);
                out[i] = __ldg(rec + (size_t)__ldg(idx + j) * f4 + q);
        }
}

cudaError_t launch_gather_records(const float4* rec, const int* idx, long long count, int f4, float4* out,
                                  cudaStream_t st)
{
        if (count > 0)
        {
                const unsigned g = (unsigned)std::min<long long>((count * f4 + BLOCK - 1) / BLOCK, 148LL * 64);
                k_gather_records<<<g, BLOCK, 0, st>>>(rec, idx, count, f4, out);
        }
        return cudaGetLastError();
}

cudaError_t launch_moments_reduce(long long npix, int spp, const double* rad, float* mean, float* var, cudaStream_t st)
{
        const unsigned g = (unsigned)std::min<long long>((npix * 3 + BLOCK - 1) / BLOCK, 148LL * 32);
        if (npix > 0)
        {
                k_moments_reduce<<<g, BLOCK, 0, st>>>(npix, spp, rad, mean, var);
        }
        return cudaGetLastError();
}

cudaError_t launch_srgb_slice(const double* accum, long long samples, long long base, int width, int height,
                              long long row_stride, uint32_t* out, cudaStream_t st)
{
        const long long count = (long long)width * height;
        if (count <= 0)
        {
                return cudaSuccess;
        }
        const unsigned g = (unsigned)std::min<long long>((count + BLOCK - 1) / BLOCK, 148LL * 32);
        k_srgb_slice<<<g, BLOCK, 0, st>>>(accum, samples > 0 ? 1.0 / (double)samples : 0.0, base, width, height, row_stride,
                                          out);
        return cudaGetLastError();
}

// per-pixel sums (doubles) -> mean colour (floats), for the accumulator read-back
__global__ void k_mean(long long n3, const double* __restrict__ sums, double inv, float* __restrict__ out)
{
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
        {
                out[i] = (float)(sums[i] * inv);
        }
}

cudaError_t launch_mean(long long n3, const double* sums, long long samples, float* out, cudaStream_t st)
{
        if (n3 <= 0)
        {
                return cudaSuccess;
        }
        const unsigned g = (unsigned)std::min<long long>((n3 + BLOCK - 1) / BLOCK, 148LL * 32);
        k_mean<<<g, BLOCK, 0, st>>>(n3, sums, samples > 0 ? 1.0 / (double)samples : 0.0, out);
        return cudaGetLastError();
}

#define NT_INSTANTIATE(N)                                                                                         \
        template struct Wavefront<N>;                                                                             \
        template cudaError_t launch_trace_closest<N>(const MeshDev<N>&, const float*, const float*, long long, int, \
                                                     int*, float*, unsigned long long*, cudaStream_t);          \
        template cudaError_t launch_aux<N>(const DevScene<N>&, long long, float*, float*, cudaStream_t);
NT_INSTANTIATE(3)
NT_INSTANTIATE(4)
NT_INSTANTIATE(5)
NT_INSTANTIATE(6)
#undef NT_INSTANTIATE
}
