// Device functions of the n-space path tracer (sm_100a).  Compiled with -fmad=false: every fused
// multiply-add below is explicit (__fmaf_rn / __fma_rn, where the reference's dot product uses
// std::fma, src/com/vec.h:259-266); divisions and square roots are IEEE round-to-nearest.
#pragma once

#include "device_types.h"

#include <cfloat>
#include <cstdint>

#ifndef NT_FACET_FULL_LOAD
#define NT_FACET_FULL_LOAD 1
#endif

namespace ntrace
{
// ------------------------------------------------------------------------------------------------
// small vector helpers

template <int N>
__device__ __forceinline__ float vdot(const float* a, const float* b)
{
        float r = a[0] * b[0];
#pragma unroll
        for (int i = 1; i < N; ++i)
        {
                r = __fmaf_rn(a[i], b[i], r);
        }
        return r;
}

template <int N>
__device__ __forceinline__ double vdot64(const double* a, const double* b)
{
        double r = a[0] * b[0];
#pragma unroll
        for (int i = 1; i < N; ++i)
        {
                r = __fma_rn(a[i], b[i], r);
        }
        return r;
}

template <int N>
__device__ __forceinline__ void vnormalize(float* a)
{
        float len = __fsqrt_rn(vdot<N>(a, a));
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                a[i] = __fdiv_rn(a[i], len);
        }
}

__device__ __forceinline__ float smaxf(float a, float b)
{
        return (a < b) ? b : a;
}
__device__ __forceinline__ float sminf(float a, float b)
{
        return (b < a) ? b : a;
}

// ------------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011)

__device__ __forceinline__ uint4 philox(uint32_t k0, uint32_t k1, uint4 c)
{
        const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
        for (int r = 0; r < 10; ++r)
        {
                uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
                uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
                c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
                k0 += W0;
                k1 += W1;
        }
        return c;
}

__device__ __forceinline__ float u01(uint32_t x)
{
        return (float)(x >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float4 rng4(uint32_t k0, uint32_t k1, unsigned long long path, uint32_t stream, uint32_t draw)
{
        uint4 o = philox(k0, k1, make_uint4((uint32_t)path, (uint32_t)(path >> 32), stream, draw));
        return make_float4(u01(o.x), u01(o.y), u01(o.z), u01(o.w));
}

// ------------------------------------------------------------------------------------------------
// Rays

template <int N>
struct Ray
{
        float org[N];
        float dir[N];
};

// Ray(org, dir) normalises dir (src/com/ray.h:34-36)
template <int N>
__device__ __forceinline__ void ray_set(Ray<N>& r, const float* org, const float* dir)
{
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r.org[i] = org[i];
                r.dir[i] = dir[i];
        }
        vnormalize<N>(r.dir);
}

template <int N>
__device__ __forceinline__ void ray_point(const Ray<N>& r, float t, float* p)
{
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                p[i] = r.org[i] + r.dir[i] * t;
        }
}

template <int N>
__device__ __forceinline__ void ray_move(Ray<N>& r, float t)
{
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r.org[i] = r.org[i] + r.dir[i] * t;
        }
}

// ------------------------------------------------------------------------------------------------
// Orthogonal box slabs (ParallelotopeOrtho::intersect_impl, parallelotope_ortho.h:254-300)

template <int N>
__device__ __forceinline__ bool box_slabs(const float* org_box, const float* size, const float* ro, const float* rd,
                                          float* first, float* second)
{
        float f_max = -FLT_MAX;
        float b_min = FLT_MAX;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                float d1 = org_box[i] + size[i];
                float d2 = -org_box[i];
                float s = rd[i];
                float d = ro[i];
                if (s == 0)
                {
                        if (d - d1 > 0 || -d - d2 > 0)
                        {
                                return false;
                        }
                        continue;
                }
                float alpha1 = __fdiv_rn(d1 - d, s);
                float alpha2 = __fdiv_rn(d2 + d, -s);
                if (s < 0)
                {
                        f_max = smaxf(alpha1, f_max);
                        b_min = sminf(alpha2, b_min);
                }
                else
                {
                        b_min = sminf(alpha1, b_min);
                        f_max = smaxf(alpha2, f_max);
                }
                if (b_min <= 0 || b_min < f_max)
                {
                        return false;
                }
        }
        *first = f_max;
        *second = b_min;
        return true;
}

// root box, given directly by its d1 planes
template <int N>
__device__ __forceinline__ bool root_slabs(const MeshDev<N>& M, const float* ro, const float* rd, float* first,
                                           float* second)
{
        float f_max = -FLT_MAX;
        float b_min = FLT_MAX;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                float d1 = M.root_d1[i];
                float d2 = -M.root_org[i];
                float s = rd[i];
                float d = ro[i];
                if (s == 0)
                {
                        if (d - d1 > 0 || -d - d2 > 0)
                        {
                                return false;
                        }
                        continue;
                }
                float alpha1 = __fdiv_rn(d1 - d, s);
                float alpha2 = __fdiv_rn(d2 + d, -s);
                if (s < 0)
                {
                        f_max = smaxf(alpha1, f_max);
                        b_min = sminf(alpha2, b_min);
                }
                else
                {
                        b_min = sminf(alpha1, b_min);
                        f_max = smaxf(alpha2, f_max);
                }
                if (b_min <= 0 || b_min < f_max)
                {
                        return false;
                }
        }
        *first = f_max;
        *second = b_min;
        return true;
}

// nearest-face normal (parallelotope_ortho.h:337-362): returns the axis and sign
template <int N>
__device__ __forceinline__ void box_normal_axis(const float* org_box, const float* d1, const float* p, int* axis,
                                                float* sign)
{
        float mn = FLT_MAX;
        int ax = 0;
        float sg = 1;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                float l = fabsf(p[i] - d1[i]);
                if (l < mn)
                {
                        mn = l;
                        ax = i;
                        sg = 1;
                }
                l = fabsf(p[i] + (-org_box[i]));
                if (l < mn)
                {
                        mn = l;
                        ax = i;
                        sg = -1;
                }
        }
        *axis = ax;
        *sign = sg;
}

// ------------------------------------------------------------------------------------------------
// 2^N-tree point location (SpatialSubdivisionTree::find_box_for_point, tree.h:441-463).
// The reference tries children in index order with closed intervals and backtracks when a child
// contains the point but none of its children does.  The fast path picks, per axis, the lower half
// whenever the point is in it (which is what index order gives) and falls back to the exact
// backtracking search only when some axis was ambiguous (point exactly on a split plane) and the
// greedy descent then failed.

template <int N>
struct Leaf
{
        int node;  // -1: no leaf contains the point
        int level;
        float org[N];
};

template <int N>
struct Point
{
        float v[N];
};

// Out of line and by value: the caller's walk state is not address-taken, so it stays in registers.
template <int N>
__device__ __noinline__ Leaf<N> find_leaf_dfs(const MeshDev<N>& M, const Point<N> pt)
{
        const float* p = pt.v;
        Leaf<N> res;
        res.node = -1;
        res.level = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                res.org[i] = 0;
        }
        Leaf<N>* out = &res;
        struct Frame
        {
                int node;
                int next;
                float org[N];
        };
        Frame st[MAX_LEVELS + 1];
        int top = 0;
        st[0].node = 0;
        st[0].next = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                st[0].org[i] = M.root_org[i];
        }
        while (top >= 0)
        {
                Frame& f = st[top];
                int2 nd = M.nodes[f.node];
                if (nd.y >= 0)
                {
                        out->node = f.node;
                        out->level = top;
                        for (int i = 0; i < N; ++i)
                        {
                                out->org[i] = f.org[i];
                        }
                        return res;
                }
                bool pushed = false;
                while (f.next < (1 << N) && top < MAX_LEVELS)
                {
                        int c = f.next++;
                        float co[N];
                        bool inside = true;
                        for (int i = 0; i < N; ++i)
                        {
                                float h = M.size[top + 1][i];
                                co[i] = (c & (1 << i)) ? f.org[i] + h : f.org[i];
                                float d1 = co[i] + h;
                                if (!(p[i] <= d1) || !(-p[i] <= -co[i]))
                                {
                                        inside = false;
                                }
                        }
                        if (inside)
                        {
                                Frame& g = st[top + 1];
                                g.node = nd.x + c;
                                g.next = 0;
                                for (int i = 0; i < N; ++i)
                                {
                                        g.org[i] = co[i];
                                }
                                ++top;
                                pushed = true;
                                break;
                        }
                }
                if (!pushed)
                {
                        --top;
                }
        }
        return res;
}

// Threads per block of every kernel that walks a tree: the path caches' per-level slots are laid
// out in shared memory with this stride.  A build-time option (NT_BLOCK, with NT_WALK_MIN_BLOCKS the
// occupancy asked of the walk kernels); 128 threads and 5 blocks per SM measured 8 % faster on the
// n = 4 frame than 256 threads and 2 blocks (20 warps per SM instead of 16, at 96 registers instead
// of 120), and 256 x 4 was slower.
#ifndef NT_BLOCK
#define NT_BLOCK 128
#endif
constexpr int WALK_BLOCK = NT_BLOCK;

// The root-to-leaf path of the previous point location of the same walk.  Consecutive leaves of a
// walk share most of their ancestors; the child chosen at each level depends only on the point and
// the box origins above it, so while the new point picks the same children the node records are
// known and are not read again.  The leaf found is the one a full descent finds.
struct PathCache
{
        int depth;                 // level of the cached leaf; -1: empty
        int2 leaf;                 // the cached leaf's record
        // the first child of the internal node at each level of the path, and the child chosen there,
        // are kept in shared memory (path_cache_slots, path_cache_child)

        __device__ __forceinline__ void reset()
        {
                depth = -1;
        }
};

// This thread's column of the block's path-cache slots (MAX_LEVELS x WALK_BLOCK ints).
__device__ __forceinline__ int* path_cache_slots()
{
        __shared__ int s_fc[MAX_LEVELS * WALK_BLOCK];
        return s_fc + threadIdx.x;
}

// This thread's column of the child indices chosen along the cached path (MAX_LEVELS x WALK_BLOCK
// bytes; consecutive threads share 32-bit words, which costs no bank conflicts).
__device__ __forceinline__ unsigned char* path_cache_child()
{
        __shared__ unsigned char s_child[MAX_LEVELS * WALK_BLOCK];
        return s_child + threadIdx.x;
}

template <int N>
__device__ __forceinline__ bool find_leaf_cached(const MeshDev<N>& M, const float* p, PathCache& pc, Leaf<N>* out,
                                                 int2* leaf_rec, unsigned* descent)
{
        int* const fc = path_cache_slots();
        unsigned char* const cc = path_cache_child();
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                if (!(p[i] <= M.root_d1[i]) || !(-p[i] <= -M.root_org[i]))
                {
                        return false;
                }
        }
        float o[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                o[i] = M.root_org[i];
        }
        int node = 0;
        bool ambiguous = false;
        bool same = pc.depth >= 0;
        for (int lvl = 0; lvl < MAX_LEVELS; ++lvl)
        {
                int2 nd;
                if (same)
                {
                        nd = (lvl == pc.depth) ? pc.leaf : make_int2(fc[lvl * WALK_BLOCK], -1);
                }
                else
                {
                        nd = __ldg(&M.nodes[node]);
                }
                ++*descent;
                if (nd.y >= 0)
                {
                        out->node = node;
                        out->level = lvl;
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                out->org[i] = o[i];
                        }
                        *leaf_rec = nd;
                        pc.depth = lvl;
                        pc.leaf = nd;
                        return true;
                }
                if (!same)
                {
                        fc[lvl * WALK_BLOCK] = nd.x;
                }
                int child = 0;
                bool fail = false;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        float h = M.size[lvl + 1][i];
                        float mid = o[i] + h;
                        bool lo_ok = p[i] <= mid;
                        bool hi_ok = (-p[i] <= -mid) && (p[i] <= mid + h);
                        if (lo_ok)
                        {
                                ambiguous |= hi_ok;
                        }
                        else if (hi_ok)
                        {
                                child |= 1 << i;
                                o[i] = mid;
                        }
                        else
                        {
                                fail = true;
                        }
                }
                if (fail)
                {
                        pc.depth = -1;
                        if (ambiguous)
                        {
                                Point<N> pt;
#pragma unroll
                                for (int i = 0; i < N; ++i)
                                {
                                        pt.v[i] = p[i];
                                }
                                *out = find_leaf_dfs<N>(M, pt);
                                if (out->node >= 0)
                                {
                                        *leaf_rec = __ldg(&M.nodes[out->node]);
                                        return true;
                                }
                        }
                        return false;
                }
                if (!same || (int)cc[lvl * WALK_BLOCK] != child)
                {
                        same = false;
                        cc[lvl * WALK_BLOCK] = (unsigned char)child;
                }
                node = nd.x + child;
        }
        pc.depth = -1;
        return false;
}

// ------------------------------------------------------------------------------------------------
// Ray versus (N-1)-simplex.
//
// FP32 test on the Gaussian-elimination planes with a forward error bound; a test whose outcome the
// bound cannot decide is re-run in FP64 with the reference's own formulation
// (HyperplaneSimplexGeometry::intersect, hyperplane_geometry.h:40-52,181-204).

enum TestResult : int
{
        T_MISS = 0,
        T_HIT = 1,
        T_UNSURE = 2
};

// STAGED: the record lies in shared memory (staged by cp.async, leaf_closest_warp) and is read with
// plain loads; otherwise it is read from global memory through the read-only path.
template <int N, bool STAGED = false>
__device__ __forceinline__ int facet_test32(const float4* rec, const Ray<N>& r, float ao, float* t_out)
{
        constexpr float EPS = 5.9604645e-08f;  // 2^-24
        // the whole record is read at once (one memory round trip; measured faster than reading each
        // barycentric plane only once the tests before it have passed, NT_FACET_FULL_LOAD=0, which
        // saves bytes but waits up to N times)
#if NT_FACET_FULL_LOAD
        constexpr int HEAD4 = Rec32<N>::F4;
#else
        constexpr int HEAD4 = (Rec32<N>::OFF_PLANES + 3) / 4;
#endif
        float f[Rec32<N>::FLOATS];
#pragma unroll
        for (int q = 0; q < HEAD4; ++q)
        {
                float4 v = STAGED ? rec[q] : __ldg(rec + q);
                f[4 * q + 0] = v.x;
                f[4 * q + 1] = v.y;
                f[4 * q + 2] = v.z;
                f[4 * q + 3] = v.w;
        }
        const float* nrm = f;
        float s = vdot<N>(nrm, r.dir);
        float d0 = f[Rec32<N>::OFF_D0];
        float num = d0 - vdot<N>(nrm, r.org);
        float as = fabsf(s);
        float e_num = 8.0f * EPS * (fabsf(d0) + N * ao);
        if (as < 1e-6f)
        {
                // grazing: the reference tests s != 0 in FP64; decide there (without the re-test the
                // FP32 distance stands, and a ray parallel to the plane gets none)
                *t_out = (as > 0) ? __fdiv_rn(num, s) : -1.0f;
                return (as == 0 && fabsf(num) > e_num) ? T_MISS : T_UNSURE;
        }
        float t = __fdiv_rn(num, s);
        float e_t = __fdiv_rn(e_num, as) + 2.0f * EPS * fabsf(t);
        if (t < -e_t)
        {
                return T_MISS;
        }
        bool unsure = !(t > e_t);
        float p[N];
        float ap = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                p[i] = r.org[i] + r.dir[i] * t;
                ap = fmaxf(ap, fabsf(p[i]));
        }
        float e_p = e_t + 2.0f * EPS * (ao + fabsf(t));
        float B = f[Rec32<N>::OFF_B];
        float D = f[Rec32<N>::OFF_D];
        float e_b = 4.0f * (B * (e_p + 2.0f * N * EPS * ap) + 2.0f * EPS * D);
        float sum = 0;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                const int staged4 = (Rec32<N>::OFF_PLANES + i * (N + 1) + 3) / 4;
                const int first4 = (i == 0 || staged4 < HEAD4) ? HEAD4 : staged4;
                const int need4 = (Rec32<N>::OFF_PLANES + (i + 1) * (N + 1) + 3) / 4;
#pragma unroll
                for (int q = first4; q < need4; ++q)
                {
                        float4 v = STAGED ? rec[q] : __ldg(rec + q);
                        f[4 * q + 0] = v.x;
                        f[4 * q + 1] = v.y;
                        f[4 * q + 2] = v.z;
                        f[4 * q + 3] = v.w;
                }
                const float* pl = f + Rec32<N>::OFF_PLANES + i * (N + 1);
                float b = vdot<N>(p, pl) - pl[N];
                if (b <= -e_b || b >= 1.0f + e_b)
                {
                        return T_MISS;
                }
                unsure |= !(b > e_b && b < 1.0f - e_b);
                sum += b;
        }
        float last = 1.0f - sum;
        float e_last = N * e_b;
        if (last <= -e_last)
        {
                return T_MISS;
        }
        unsure |= !(last > e_last);
        *t_out = t;
        return unsure ? T_UNSURE : T_HIT;
}

template <int N>
struct Ray64
{
        double org[N];
        double dir[N];
};

template <int N>
__device__ __forceinline__ bool facet_test64(const double* rec, const Ray64<N>& r, double* t_out)
{
        double v0[N], nrm[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                v0[i] = rec[i];
                nrm[i] = rec[Rec64<N>::OFF_NORMAL + i];
        }
        double s = vdot64<N>(nrm, r.dir);
        if (!(s != 0))
        {
                return false;
        }
        double diff[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                diff[i] = v0[i] - r.org[i];
        }
        double t = __ddiv_rn(vdot64<N>(diff, nrm), s);
        if (!(t > 0))
        {
                return false;
        }
        double p[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                p[i] = r.org[i] + r.dir[i] * t;
        }
        double coords[N - 1];
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                const double* pl = rec + Rec64<N>::OFF_PLANES + i * (N + 1);
                double pn[N];
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        pn[k] = pl[k];
                }
                coords[i] = vdot64<N>(p, pn) - pl[N];
                if (coords[i] <= 0 || coords[i] >= 1)
                {
                        return false;
                }
        }
        double rr = 1;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                rr -= coords[i];
        }
        if (!(rr > 0))
        {
                return false;
        }
        *t_out = t;
        return true;
}

// How the FP64 re-test obtains its ray: promoted from the FP32 ray (rendering), or normalised in
// double from the caller's raw input (the fixed-ray-set parity entry point).
template <int N>
struct Ray64Source
{
        const float* raw_org;  // null: promote
        const float* raw_dir;
        long long index;

        __device__ __forceinline__ void get(const Ray<N>& r, Ray64<N>* out) const
        {
                if (raw_org)
                {
                        double len2;
                        double d[N];
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                out->org[i] = (double)raw_org[index * N + i];
                                d[i] = (double)raw_dir[index * N + i];
                        }
                        len2 = vdot64<N>(d, d);
                        double len = __dsqrt_rn(len2);
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                out->dir[i] = __ddiv_rn(d[i], len);
                        }
                }
                else
                {
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                out->org[i] = (double)r.org[i];
                                out->dir[i] = (double)r.dir[i];
                        }
                }
        }
};

// Per-thread work counters of one launch (flushed to the 64-bit device counters at the end).
struct WalkStats
{
        unsigned facet_tests;
        unsigned box_steps;
        unsigned retests;
        unsigned descent;
        int error;
};

// FP64 re-test of one facet, kept out of line so that its double-precision state does not occupy
// registers of the hot FP32 walk; arguments by value so that the caller's ray is not address-taken.
// Returns the FP64 distance, or -1 when the facet is missed.
template <int N>
__device__ __noinline__ double retest_facet(const double* rec, const Ray<N> ray, const Ray64Source<N> src)
{
        Ray64<N> r64;
        src.get(ray, &r64);
        double t;
        return facet_test64<N>(rec, r64, &t) ? t : -1.0;
}

// Closest facet of one leaf (ray_intersection over indices, ray_intersection.h:134-159: strict <
// in list order).  Returns the facet or -1 and its distance.
// The FP32 record of leaf-list entry pos: from the leaf-ordered copy when the mesh has one, else
// through the leaf's index list (the copy is left out when it would take more than a quarter of the
// free device memory; the branch is uniform, on a kernel parameter).
template <int N>
__device__ __forceinline__ const float4* leaf_record(const MeshDev<N>& M, long long pos)
{
        return M.leaf_rec32 ? M.leaf_rec32 + (size_t)pos * Rec32<N>::F4
                            : M.rec32 + (size_t)__ldg(&M.leaf_idx[pos]) * Rec32<N>::F4;
}

template <int N>
__device__ __forceinline__ int leaf_closest(const MeshDev<N>& M, int2 leaf, const Ray<N>& ray, float ao,
                                            const Ray64Source<N>& src, int retest, float* t_best, WalkStats* ws)
{
        int best = -1;
        float bt = FLT_MAX;
        double bt64 = 0;
        bool b64 = false;
        for (int q = 0; q < leaf.y; ++q)
        {
                ++ws->facet_tests;
                float t;
                int res = facet_test32<N>(leaf_record<N>(M, leaf.x + q), ray, ao, &t);
                if (res == T_MISS)
                {
                        continue;
                }
                // the facet's index only for the tests that did not miss
                const int f = __ldg(&M.leaf_idx[leaf.x + q]);
                double t64 = 0;
                bool is64 = false;
                if (res == T_UNSURE)
                {
                        if (!retest)
                        {
                                // without the re-test an uncertain FP32 hit counts when its
                                // distance is positive and the test did not reject it
                                if (!(t > 0))
                                {
                                        continue;
                                }
                        }
                        else
                        {
                                ++ws->retests;
                                t64 = retest_facet<N>(M.rec64 + (size_t)f * Rec64<N>::DOUBLES, ray, src);
                                if (!(t64 > 0))
                                {
                                        continue;
                                }
                                t = (float)t64;
                                is64 = true;
                        }
                }
                // comparison with the best so far; near-ties are settled in FP64
                bool closer;
                float tol = 1e-5f * (fabsf(t) + ao) + 1e-30f;
                if (retest && best >= 0 && fabsf(t - bt) <= tol)
                {
                        if (!is64)
                        {
                                ++ws->retests;
                                t64 = retest_facet<N>(M.rec64 + (size_t)f * Rec64<N>::DOUBLES, ray, src);
                                if (!(t64 > 0))
                                {
                                        continue;
                                }
                                is64 = true;
                        }
                        if (!b64)
                        {
                                ++ws->retests;
                                double tb = retest_facet<N>(M.rec64 + (size_t)best * Rec64<N>::DOUBLES, ray, src);
                                if (tb > 0)
                                {
                                        bt64 = tb;
                                        b64 = true;
                                }
                                else
                                {
                                        // the incumbent fails in FP64: the newcomer wins
                                        best = f;
                                        bt = (float)t64;
                                        bt64 = t64;
                                        b64 = true;
                                        continue;
                                }
                        }
                        closer = t64 < bt64;
                }
                else
                {
                        closer = t < bt;
                }
                if (closer)
                {
                        best = f;
                        bt = t;
                        bt64 = t64;
                        b64 = is64;
                }
        }
        *t_best = bt;
        return best;
}

// Mesh::intersect_precise through SpatialSubdivisionTree::trace_ray (mesh.cpp:143-166,
// tree.h:534-590).  tmax: the walk may stop once the current leaf starts beyond tmax (used by shadow
// rays, whose answer only depends on hits nearer than the light).
template <int N>
__device__ bool mesh_closest(const MeshDev<N>& M, const Ray<N>& ray, float root_t, const Ray64Source<N>& src, int retest,
                             float tmax, float* t_out, int* facet_out, WalkStats* ws)
{
        float ao = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                ao = fmaxf(ao, fabsf(ray.org[i]));
        }
        float cur[N];
        float probe[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                cur[i] = ray.org[i];
                probe[i] = ray.org[i];
        }
        float travelled = 0;
        bool first = true;
        PathCache pc;
        pc.reset();
        // a ray crosses at most (boxes per axis) x N leaves of a 2^N-tree at most 2^9 boxes wide;
        // the bound leaves ample margin and turns a walk that does not advance into an error flag
        for (int step = 0; step < 16384; ++step)
        {
                Leaf<N> lf;
                int2 nd;
                if (find_leaf_cached<N>(M, probe, pc, &lf, &nd, &ws->descent))
                {
                        ++ws->box_steps;
                        const float* sz = M.size[lf.level];
                        if (travelled > tmax * 1.00001f + 1e-6f)
                        {
                                return false;
                        }
                        if (nd.y > 0)
                        {
                                float t;
                                int f = leaf_closest<N>(M, nd, ray, ao, src, retest, &t, ws);
                                if (f >= 0)
                                {
                                        float pt[N];
                                        ray_point<N>(ray, t, pt);
                                        bool inside = true;
#pragma unroll
                                        for (int i = 0; i < N; ++i)
                                        {
                                                float d1 = lf.org[i] + sz[i];
                                                if (!(pt[i] <= d1) || !(-pt[i] <= -lf.org[i]))
                                                {
                                                        inside = false;
                                                }
                                        }
                                        if (inside)
                                        {
                                                *t_out = t;
                                                *facet_out = f;
                                                return true;
                                        }
                                }
                        }
                        float first_t, second_t;
                        if (!box_slabs<N>(lf.org, sz, cur, ray.dir, &first_t, &second_t))
                        {
                                return false;
                        }
                        float ip[N], d1[N];
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                ip[i] = cur[i] + ray.dir[i] * second_t;
                                d1[i] = lf.org[i] + sz[i];
                        }
                        int ax;
                        float sg;
                        box_normal_axis<N>(lf.org, d1, ip, &ax, &sg);
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                cur[i] = ip[i];
                                probe[i] = (i == ax) ? ip[i] + M.dist * sg : ip[i] + M.dist * 0.0f;
                        }
                        travelled += second_t;
                }
                else
                {
                        if (!first)
                        {
                                return false;
                        }
                        float ip[N];
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                ip[i] = cur[i] + ray.dir[i] * root_t;
                        }
                        int ax;
                        float sg;
                        box_normal_axis<N>(M.root_org, M.root_d1, ip, &ax, &sg);
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                cur[i] = ip[i];
                                probe[i] = (i == ax) ? ip[i] - M.dist * sg : ip[i] - M.dist * 0.0f;
                        }
                        travelled = root_t;
                }
                first = false;
        }
        ws->error |= ERR_WALK_LIMIT;
        return false;
}

// ------------------------------------------------------------------------------------------------
// General parallelotope (Parallelotope::intersect_impl / normal, parallelotope.h:190-310)

template <int N>
__device__ __forceinline__ bool plt_intersect(const PltDev<N>& P, const Ray<N>& r, float* t)
{
        float f_max = -FLT_MAX;
        float b_min = FLT_MAX;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                float s = vdot<N>(r.dir, P.n[i]);
                float d = vdot<N>(r.org, P.n[i]);
                if (s == 0)
                {
                        if (d - P.d1[i] > 0 || -d - P.d2[i] > 0)
                        {
                                return false;
                        }
                        continue;
                }
                float alpha1 = __fdiv_rn(P.d1[i] - d, s);
                float alpha2 = __fdiv_rn(P.d2[i] + d, -s);
                if (s < 0)
                {
                        f_max = smaxf(alpha1, f_max);
                        b_min = sminf(alpha2, b_min);
                }
                else
                {
                        b_min = sminf(alpha1, b_min);
                        f_max = smaxf(alpha2, f_max);
                }
                if (b_min <= 0 || b_min < f_max)
                {
                        return false;
                }
        }
        *t = (f_max > 0) ? f_max : b_min;
        return true;
}

template <int N>
__device__ __forceinline__ void plt_normal(const PltDev<N>& P, const float* p, float* nrm)
{
        float mn = FLT_MAX;
        int best = 0;
        float sg = 1;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                float d = vdot<N>(p, P.n[i]);
                float l = fabsf(d - P.d1[i]);
                if (l < mn)
                {
                        mn = l;
                        best = i;
                        sg = 1;
                }
                l = fabsf(-d - P.d2[i]);
                if (l < mn)
                {
                        mn = l;
                        best = i;
                        sg = -1;
                }
        }
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                nrm[k] = sg * P.n[best][k];
        }
}

// Hyperplane parallelotope (HyperplaneParallelotopeGeometry::intersect, hyperplane_geometry.h:236-260)
template <int N>
__device__ __forceinline__ bool hplt_intersect(const HpltDev<N>& H, const Ray<N>& r, float* t_out)
{
        float s = vdot<N>(H.normal, r.dir);
        if (!(s != 0))
        {
                return false;
        }
        float diff[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                diff[i] = H.org[i] - r.org[i];
        }
        float t = __fdiv_rn(vdot<N>(diff, H.normal), s);
        if (!(t > 0))
        {
                return false;
        }
        float p[N];
        ray_point<N>(r, t, p);
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                float b = vdot<N>(p, H.planes[i]) - H.planes[i][N];
                if (b <= 0 || b >= 1)
                {
                        return false;
                }
        }
        *t_out = t;
        return true;
}

// ------------------------------------------------------------------------------------------------
// Objects and the scene (GenericObject / ray_intersection, objects.h:141-172, ray_intersection.h:26-105)

template <int N>
__device__ __forceinline__ bool obj_approx(const DevScene<N>& S, int o, const Ray<N>& r, float* t)
{
        const ObjDev& ob = S.obj[o];
        if (ob.kind == OBJ_MESH)
        {
                float first, second;
                if (root_slabs<N>(S.mesh[ob.index], r.org, r.dir, &first, &second))
                {
                        *t = (first > 0) ? first : second;
                        return true;
                }
                return false;
        }
        if (ob.kind == OBJ_PLT)
        {
                return plt_intersect<N>(S.plt[ob.index], r, t);
        }
        return hplt_intersect<N>(S.hplt[ob.index], r, t);
}

template <int N>
__device__ __forceinline__ bool obj_precise(const DevScene<N>& S, int o, const Ray<N>& r, float approx, float tmax,
                                            float* t, int* facet, WalkStats* ws)
{
        const ObjDev& ob = S.obj[o];
        if (ob.kind == OBJ_MESH)
        {
                Ray64Source<N> src{nullptr, nullptr, 0};
                return mesh_closest<N>(S.mesh[ob.index], r, approx, src, S.retest, tmax, t, facet, ws);
        }
        *t = approx;
        *facet = -1;
        return true;
}

template <int N>
__device__ bool scene_closest(const DevScene<N>& S, const Ray<N>& r, float* t_out, int* obj_out, int* facet_out,
                              WalkStats* ws)
{
        if (S.nobj == 1)
        {
                float a, t;
                int f;
                if (obj_approx<N>(S, 0, r, &a) && obj_precise<N>(S, 0, r, a, FLT_MAX, &t, &f, ws))
                {
                        *t_out = t;
                        *obj_out = 0;
                        *facet_out = f;
                        return true;
                }
                return false;
        }
        float ad[MAX_OBJECTS];
        int ao[MAX_OBJECTS];
        int na = 0;
        for (int o = 0; o < S.nobj; ++o)
        {
                float a;
                if (obj_approx<N>(S, o, r, &a))
                {
                        // insertion keeps equal distances in object order
                        int k = na++;
                        while (k > 0 && a < ad[k - 1])
                        {
                                ad[k] = ad[k - 1];
                                ao[k] = ao[k - 1];
                                --k;
                        }
                        ad[k] = a;
                        ao[k] = o;
                }
        }
        float min_distance = FLT_MAX;
        bool found = false;
        for (int q = 0; q < na; ++q)
        {
                if (min_distance < ad[q])
                {
                        break;
                }
                float d;
                int f;
                if (obj_precise<N>(S, ao[q], r, ad[q], FLT_MAX, &d, &f, ws) && d < min_distance)
                {
                        min_distance = d;
                        *obj_out = ao[q];
                        *facet_out = f;
                        found = true;
                }
        }
        if (found)
        {
                *t_out = min_distance;
        }
        return found;
}

// light_source_is_visible / object_is_obstacle_to_light (painter.cpp:142-186)
template <int N>
__device__ bool scene_visible(const DevScene<N>& S, const Ray<N>& r, float dist, WalkStats* ws)
{
        for (int o = 0; o < S.nobj; ++o)
        {
                float d;
                if (!obj_approx<N>(S, o, r, &d))
                {
                        continue;
                }
                if (d >= dist)
                {
                        continue;
                }
                int f;
                if (!obj_precise<N>(S, o, r, d, dist, &d, &f, ws))
                {
                        continue;
                }
                if (d >= dist)
                {
                        continue;
                }
                return false;
        }
        return true;
}

// ------------------------------------------------------------------------------------------------
// Resumable tree walk for scenes with exactly one mesh.
//
// The same walk as mesh_closest, cut at leaf granularity: each call of walk_step_warp visits one
// leaf (descent, leaf facets, exit) and says whether the walk has ended.  A lane whose walk ends
// takes the next ray at once while the other lanes of its warp continue theirs, so warps stay full
// even though rays visit very different numbers of leaves (the per-ray loop leaves most lanes idle).
// The decisions around the walk are those of ray_intersection (ray_intersection.h:26-105) and
// light_source_is_visible (painter.cpp:142-186) specialised to one mesh plus non-mesh objects, whose
// precise distance equals their approximate one.
//
// The state is kept small (it stays in registers across the pooled facet tests): the probe point is
// the current point nudged along one axis, stored as that axis and direction; the root-box entry
// distance sits in `travelled` until the first step.

template <int N>
struct Walk
{
        Ray<N> ray;
        float cur[N];
        float travelled;
        float tmax;
        float ao;
        int steps;
        int nudge;      // 0: the probe is cur; +-(axis + 1): cur nudged by +-dist along axis
        long long raw;  // index of the caller's raw ray (fixed-ray-set query), for the FP64 re-test
        PathCache pc;

        __device__ __forceinline__ void probe(float dist, float* p) const
        {
                const int ax = (nudge > 0 ? nudge : -nudge) - 1;
                const float s = nudge > 0 ? dist : -dist;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        p[i] = (i == ax) ? cur[i] + s : cur[i];
                }
        }
};

enum WalkStatus : int
{
        W_RUNNING = 0,
        W_HIT = 1,
        W_MISS = 2
};

template <int N>
__device__ __forceinline__ void walk_begin(Walk<N>& w, const Ray<N>& ray, float root_t, float tmax)
{
        w.ray = ray;
        w.ao = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                w.ao = fmaxf(w.ao, fabsf(ray.org[i]));
                w.cur[i] = ray.org[i];
        }
        w.travelled = root_t;
        w.tmax = tmax;
        w.steps = 0;
        w.nudge = 0;
        w.raw = 0;
        // the path cache describes a root-to-leaf path of the tree, not the ray: it stays valid
        // from one ray of the lane to the next (neighbouring rays share their upper levels), so it
        // is reset once per lane (w.pc.reset()) and not here
}

// ------------------------------------------------------------------------------------------------
// Warp-cooperative leaf step.
//
// The leaves that the 32 lanes of a warp stand in hold different numbers of facets (0 to a few
// dozen), so a per-lane loop over them leaves most lanes idle.  Here the warp pools its facet tests:
// the lanes' facet lists are laid end to end (warp prefix sum of the counts) and every lane tests
// every 32nd entry of the pooled list against the owning lane's ray, fetched by shuffle.  Each
// outcome (FP32 hit, or hit after the FP64 re-test) goes to a per-warp shared-memory slot; the owner
// then reads its own slots in leaf-list order and makes the same sequential choice as leaf_closest
// (strict < in list order, near-ties settled in FP64), so the result is the per-lane loop's.

constexpr int POOL_SLOTS = 128;  // pooled tests per warp and round, at most
constexpr int SMALL_LEAF = 2;  // default: leaves this small are tested per lane, not pooled

struct PoolSlot
{
        float t;      // FP32 distance (the rounded FP64 one after a re-test)
        int facet;    // -1: missed
        double t64;   // FP64 distance when re-tested; -1 otherwise
};

// The warp's outcome slots, SLOTS of them (a kernel variant's chunk size: 32 to POOL_SLOTS).
template <int SLOTS>
__device__ __forceinline__ PoolSlot* warp_pool()
{
        __shared__ PoolSlot s_pool[(WALK_BLOCK / 32) * SLOTS];
        return s_pool + (threadIdx.x >> 5) * SLOTS;
}

// Facet records staged through shared memory.  A warp handles its pooled tests in chunks of
// Stage<N>::SLOTS: it first reads the chunk's facet indices (ROUNDS independent loads per lane), then
// copies their records into its staging slots with cp.async (ROUNDS x F4 16-byte copies per lane in
// flight at once), waits once, and tests from shared memory.  A chunk costs two memory round trips
// instead of two per 32 tests.  The buffer is dynamic shared memory (Stage<N>::BYTES per block of
// WALK_BLOCK threads), at most 8 KB per warp.
// Other chunk sizes (R = 1, 2 or 4 rounds) are compiled as kernel variants that the autotuner
// chooses from (nt_render_opts.walk_chunk).
template <int N>
struct StageFit
{
        static constexpr int REC_BYTES = Rec32<N>::F4 * 16;
        static constexpr int FIT = 8192 / (32 * REC_BYTES);
        static constexpr int ROUNDS = FIT < 1 ? 1 : (FIT > 4 ? 4 : (FIT == 3 ? 2 : FIT));
};

// R = 0: no staging; the records are read straight from global memory, 32 tests per round.
template <int N, int R = StageFit<N>::ROUNDS>
struct Stage
{
        static constexpr int REC_BYTES = Rec32<N>::F4 * 16;
        static constexpr int ROUNDS = R > 0 ? R : 1;
        static constexpr int SLOTS = 32 * ROUNDS;
        static constexpr int BYTES = R > 0 ? (WALK_BLOCK / 32) * SLOTS * REC_BYTES : 0;
        static_assert(SLOTS <= POOL_SLOTS, "a chunk's outcomes must fit the warp's pool");
};

__device__ __forceinline__ float4* stage_base()
{
        extern __shared__ float4 g_walk_stage[];
        return g_walk_stage;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
        const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Closest facet of this lane's leaf (facets leaf_idx[start .. start + cnt)); every lane of the warp
// calls it, lanes without a leaf with cnt = 0.  raw_org/raw_dir: the caller's raw rays for the
// FP64 re-test of the fixed-ray-set query (null when rendering: the FP32 ray is promoted).
template <int N, int RR = StageFit<N>::ROUNDS>
__device__ __forceinline__ int leaf_closest_warp(const MeshDev<N>& M, int start, int cnt, const Ray<N>& ray, float ao,
                                                 long long raw, const float* raw_org, const float* raw_dir, int retest,
                                                 float* t_best, WalkStats* ws, int small_leaf = SMALL_LEAF)
{
        const unsigned full = 0xffffffffu;
        const int lane = threadIdx.x & 31;
        // small leaves (at most small_leaf facets in every lane's leaf, the common case: a walk step tests
        // one or two facets on average) are tested by each lane on its own, in list order: the pooling's
        // scan, owner search, shuffles and second pass would cost more than the idle lanes they save
        if ((int)__reduce_max_sync(full, (unsigned)cnt) <= small_leaf)
        {
                return leaf_closest<N>(M, make_int2(start, cnt), ray, ao, Ray64Source<N>{raw_org, raw_dir, raw}, retest,
                                       t_best, ws);
        }
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
                int v = __shfl_up_sync(full, incl, d);
                if (lane >= d)
                {
                        incl += v;
                }
        }
        const int total = __shfl_sync(full, incl, 31);
        const int excl = incl - cnt;
        int best = -1;
        float bt = FLT_MAX;
        double bt64 = 0;
        bool b64 = false;
        if (total == 0)
        {
                *t_best = bt;
                return best;
        }
        PoolSlot* pool = warp_pool<Stage<N, RR>::SLOTS>();
        constexpr bool STAGED = RR > 0;
        constexpr int R = Stage<N, RR>::ROUNDS;
        constexpr int F4 = Rec32<N>::F4;
        float4* const stage = stage_base() + (size_t)(threadIdx.x >> 5) * Stage<N, RR>::SLOTS * F4;
        const Ray64Source<N> own_src{raw_org, raw_dir, raw};
        for (int cb = 0; cb < total; cb += Stage<N, RR>::SLOTS)
        {
                const int ce = min(total, cb + Stage<N, RR>::SLOTS);
                // the chunk's entries (positions in the leaf lists, whose records lie in that order in
                // leaf_rec32), then, staged, their records into the staging slots (all copies in flight
                // at once); a facet's index is read only for the tests that do not miss
                int own[R];
                int pos[R];
#pragma unroll
                for (int r = 0; r < R; ++r)
                {
                        const int k = cb + 32 * r + lane;
                        // owner: the last lane whose list starts at or before k
                        int o = 0;
#pragma unroll
                        for (int step = 16; step > 0; step >>= 1)
                        {
                                int v = __shfl_sync(full, excl, o + step);
                                if (v <= k)
                                {
                                        o += step;
                                }
                        }
                        own[r] = o;
                        const int o_start = __shfl_sync(full, start, o);
                        const int o_excl = __shfl_sync(full, excl, o);
                        pos[r] = (k < ce) ? o_start + (k - o_excl) : -1;
                }
                if constexpr (STAGED)
                {
#pragma unroll
                        for (int r = 0; r < R; ++r)
                        {
                                if (pos[r] >= 0)
                                {
                                        const float4* src = leaf_record<N>(M, pos[r]);
                                        float4* dst = stage + (size_t)(32 * r + lane) * F4;
#pragma unroll
                                        for (int q = 0; q < F4; ++q)
                                        {
                                                cp_async16(dst + q, src + q);
                                        }
                                }
                        }
                        cp_async_wait_all();
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
                {
                        const int k = cb + 32 * r + lane;
                        const int o = own[r];
                        const float o_ao = __shfl_sync(full, ao, o);
                        Ray<N> rr;
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                rr.org[i] = __shfl_sync(full, ray.org[i], o);
                                rr.dir[i] = __shfl_sync(full, ray.dir[i], o);
                        }
                        const long long o_raw = raw_org ? __shfl_sync(full, raw, o) : 0;
                        if (k < ce)
                        {
                                ++ws->facet_tests;
                                float t = -1.0f;
                                double t64 = -1.0;
                                int keep = -1;
                                int res = STAGED ? facet_test32<N, true>(stage + (size_t)(32 * r + lane) * F4, rr, o_ao, &t)
                                                 : facet_test32<N, false>(leaf_record<N>(M, pos[r]), rr, o_ao, &t);
                                const int f = res != T_MISS ? __ldg(&M.leaf_idx[pos[r]]) : -1;
                                if (res == T_HIT)
                                {
                                        keep = f;
                                }
                                else if (res == T_UNSURE)
                                {
                                        if (!retest)
                                        {
                                                // without the re-test an uncertain FP32 hit counts when
                                                // its distance is positive
                                                if (t > 0)
                                                {
                                                        keep = f;
                                                }
                                        }
                                        else
                                        {
                                                ++ws->retests;
                                                t64 = retest_facet<N>(M.rec64 + (size_t)f * Rec64<N>::DOUBLES, rr,
                                                                      Ray64Source<N>{raw_org, raw_dir, o_raw});
                                                if (t64 > 0)
                                                {
                                                        keep = f;
                                                        t = (float)t64;
                                                }
                                                else
                                                {
                                                        t64 = -1.0;
                                                }
                                        }
                                }
                                PoolSlot& s = pool[k - cb];
                                s.t = t;
                                s.facet = keep;
                                s.t64 = t64;
                        }
                }
                __syncwarp();
                // the owner's sequential choice over its slots of this round, in list order
                const int q0 = max(excl, cb);
                const int q1 = min(excl + cnt, ce);
                for (int q = q0; q < q1; ++q)
                {
                        const PoolSlot s = pool[q - cb];
                        if (s.facet < 0)
                        {
                                continue;
                        }
                        const int f = s.facet;
                        float t = s.t;
                        double t64 = s.t64;
                        bool is64 = t64 > 0;
                        bool closer;
                        float tol = 1e-5f * (fabsf(t) + ao) + 1e-30f;
                        if (retest && best >= 0 && fabsf(t - bt) <= tol)
                        {
                                if (!is64)
                                {
                                        ++ws->retests;
                                        t64 = retest_facet<N>(M.rec64 + (size_t)f * Rec64<N>::DOUBLES, ray, own_src);
                                        if (!(t64 > 0))
                                        {
                                                continue;
                                        }
                                        is64 = true;
                                }
                                if (!b64)
                                {
                                        ++ws->retests;
                                        double tb = retest_facet<N>(M.rec64 + (size_t)best * Rec64<N>::DOUBLES, ray, own_src);
                                        if (tb > 0)
                                        {
                                                bt64 = tb;
                                                b64 = true;
                                        }
                                        else
                                        {
                                                // the incumbent fails in FP64: the newcomer wins
                                                best = f;
                                                bt = (float)t64;
                                                bt64 = t64;
                                                b64 = true;
                                                continue;
                                        }
                                }
                                closer = t64 < bt64;
                        }
                        else
                        {
                                closer = t < bt;
                        }
                        if (closer)
                        {
                                best = f;
                                bt = t;
                                bt64 = t64;
                                b64 = is64;
                        }
                }
                __syncwarp();
        }
        *t_best = bt;
        return best;
}

// walk_step with the leaf's facets tested by leaf_closest_warp.  Every lane of the warp calls it
// (active = false for lanes without a walk, whose result is ignored).
template <int N, int RR = StageFit<N>::ROUNDS>
__device__ __forceinline__ int walk_step_warp(const MeshDev<N>& M, Walk<N>& w, bool active, int retest,
                                              const float* raw_org, const float* raw_dir, float* t_out, int* facet_out,
                                              WalkStats* ws, int small_leaf = SMALL_LEAF)
{
        int status = W_MISS;
        bool leaf = false;
        Leaf<N> lf;
        int2 nd = make_int2(0, 0);
        if (active)
        {
                status = W_RUNNING;
                float probe[N];
                w.probe(M.dist, probe);
                if (++w.steps > 16384)
                {
                        ws->error |= ERR_WALK_LIMIT;
                        status = W_MISS;
                }
                else if (find_leaf_cached<N>(M, probe, w.pc, &lf, &nd, &ws->descent))
                {
                        ++ws->box_steps;
                        if (w.steps == 1)
                        {
                                // the origin is inside the tree: nothing travelled yet
                                w.travelled = 0;
                        }
                        if (w.travelled > w.tmax * 1.00001f + 1e-6f)
                        {
                                status = W_MISS;
                        }
                        else
                        {
                                leaf = true;
                        }
                }
        }
        const int cnt = (leaf && nd.y > 0) ? nd.y : 0;
        float t = FLT_MAX;
        const int f = leaf_closest_warp<N, RR>(M, nd.x, cnt, w.ray, w.ao, w.raw, raw_org, raw_dir, retest, &t, ws,
                                                small_leaf);
        if (status != W_RUNNING)
        {
                return status;
        }
        if (leaf)
        {
                const float* sz = M.size[lf.level];
                if (f >= 0)
                {
                        float pt[N];
                        ray_point<N>(w.ray, t, pt);
                        bool inside = true;
#pragma unroll
                        for (int i = 0; i < N; ++i)
                        {
                                float d1 = lf.org[i] + sz[i];
                                if (!(pt[i] <= d1) || !(-pt[i] <= -lf.org[i]))
                                {
                                        inside = false;
                                }
                        }
                        if (inside)
                        {
                                *t_out = t;
                                *facet_out = f;
                                return W_HIT;
                        }
                }
                float first_t, second_t;
                if (!box_slabs<N>(lf.org, sz, w.cur, w.ray.dir, &first_t, &second_t))
                {
                        return W_MISS;
                }
                float ip[N], d1[N];
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        ip[i] = w.cur[i] + w.ray.dir[i] * second_t;
                        d1[i] = lf.org[i] + sz[i];
                }
                int ax;
                float sg;
                box_normal_axis<N>(lf.org, d1, ip, &ax, &sg);
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        w.cur[i] = ip[i];
                }
                // next probe: ip + dist * sg along the exit face's axis
                w.nudge = sg > 0 ? ax + 1 : -(ax + 1);
                w.travelled += second_t;
        }
        else
        {
                if (w.steps != 1)
                {
                        return W_MISS;
                }
                // outside the tree at the start: enter through the root box (travelled holds the
                // entry distance)
                float ip[N];
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        ip[i] = w.cur[i] + w.ray.dir[i] * w.travelled;
                }
                int ax;
                float sg;
                box_normal_axis<N>(M.root_org, M.root_d1, ip, &ax, &sg);
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        w.cur[i] = ip[i];
                }
                // next probe: ip - dist * sg along the entry face's axis
                w.nudge = sg > 0 ? -(ax + 1) : ax + 1;
        }
        return W_RUNNING;
}

// What ray_intersection decides around the one mesh: the objects' approximate distances in stable
// order; the walk is needed unless a non-mesh object is strictly nearer than the mesh's root box
// (then the loop breaks before the mesh).  pre: the choice made before the mesh entry; post: the
// nearest non-mesh entry after it, compared with the walk's result.
struct __align__(16) ClosestPlan  // 32 bytes: two vector loads when stored in a walk list
{
        int mesh_obj;        // object index of the mesh
        float mesh_t;        // its approximate distance (root box)
        bool walk;
        float pre_t;         // FLT_MAX: none
        int pre_obj;
        float post_t;        // FLT_MAX: none
        int post_obj;
};

template <int N>
__device__ __forceinline__ void closest_plan(const DevScene<N>& S, const Ray<N>& r, ClosestPlan* p)
{
        p->mesh_obj = -1;
        p->walk = false;
        p->pre_t = FLT_MAX;
        p->pre_obj = -1;
        p->post_t = FLT_MAX;
        p->post_obj = -1;
        float a_m = FLT_MAX;
        bool mesh_hit = false;
        for (int o = 0; o < S.nobj; ++o)
        {
                if (S.obj[o].kind == OBJ_MESH)
                {
                        p->mesh_obj = o;
                        mesh_hit = obj_approx<N>(S, o, r, &a_m);
                        break;
                }
        }
        // entries before the mesh in the stable ascending order: a < a_m, or a == a_m with a smaller
        // object index; after it: a > a_m, or a == a_m with a larger index
        float best_pre = FLT_MAX, best_post = FLT_MAX;
        int pre_obj = -1, post_obj = -1;
        for (int o = 0; o < S.nobj; ++o)
        {
                if (o == p->mesh_obj)
                {
                        continue;
                }
                float a;
                if (!obj_approx<N>(S, o, r, &a))
                {
                        continue;
                }
                bool before = !mesh_hit || a < a_m || (a == a_m && o < p->mesh_obj);
                if (before)
                {
                        if (a < best_pre)
                        {
                                best_pre = a;
                                pre_obj = o;
                        }
                }
                else if (a < best_post)
                {
                        best_post = a;
                        post_obj = o;
                }
        }
        p->mesh_t = a_m;
        if (!mesh_hit)
        {
                p->pre_t = best_pre;
                p->pre_obj = pre_obj;
                return;
        }
        if (pre_obj >= 0 && best_pre < a_m)
        {
                // the loop takes the nearest entry and breaks at the mesh
                p->pre_t = best_pre;
                p->pre_obj = pre_obj;
                return;
        }
        p->walk = true;
        p->pre_t = best_pre;  // a tie at a_m, or none
        p->pre_obj = pre_obj;
        p->post_t = best_post;
        p->post_obj = post_obj;
}

// The loop's choice once the walk has given (hit, d) for the mesh.
__device__ __forceinline__ void closest_finish(const ClosestPlan& p, bool hit, float d, int facet, float* t_out,
                                               int* obj_out, int* facet_out)
{
        float mn = p.pre_t;
        int obj = p.pre_obj;
        int fct = -1;
        if (hit && d < mn)
        {
                mn = d;
                obj = p.mesh_obj;
                fct = facet;
        }
        if (p.post_obj >= 0 && !(mn < p.post_t) && p.post_t < mn)
        {
                mn = p.post_t;
                obj = p.post_obj;
                fct = -1;
        }
        *t_out = mn;
        *obj_out = obj;
        *facet_out = fct;
}

// ------------------------------------------------------------------------------------------------
// Shading normal of a mesh facet with vertex normals (MeshHyperplaneSimplex::shading_normal,
// mesh_hyperplane_simplex.cpp:157-186): the vertex normals (reversed where the facet's type says so)
// interpolated with the barycentric coordinates of the point (HyperplaneSimplexGeometry::
// barycentric_coordinates / interpolate, hyperplane_geometry.h:169-219), normalised.  Returns false
// for a flat facet (NormalType::None: the shading normal is the geometric one).

template <int N>
__device__ __forceinline__ bool smooth_normal(const MeshDev<N>& M, int facet, const float* p, float* sn)
{
        const int type = M.ntype[facet];
        if ((type & 3) == 0)
        {
                return false;
        }
        const float4* rec = M.rec32 + (size_t)facet * Rec32<N>::F4;
        float f[Rec32<N>::FLOATS];
#pragma unroll
        for (int q = 0; q < Rec32<N>::F4; ++q)
        {
                float4 v = __ldg(rec + q);
                f[4 * q + 0] = v.x;
                f[4 * q + 1] = v.y;
                f[4 * q + 2] = v.z;
                f[4 * q + 3] = v.w;
        }
        float bc[N];
        bc[N - 1] = 1.0f;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                const float* pl = f + Rec32<N>::OFF_PLANES + i * (N + 1);
                bc[i] = vdot<N>(p, pl) - pl[N];
                bc[N - 1] -= bc[i];
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                const float* vn = M.vnormals + (size_t)__ldg(&M.fnormals[(size_t)facet * N + i]) * N;
                const bool rev = (type & 3) == 2 && (type & (1 << (2 + i)));
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        const float c = rev ? -__ldg(vn + k) : __ldg(vn + k);
                        sn[k] = (i == 0) ? bc[0] * c : sn[k] + bc[i] * c;
                }
        }
        vnormalize<N>(sn);
        return true;
}

// ------------------------------------------------------------------------------------------------
// Sampling (sphere.h:87-116, complement.h:71-200)

template <int N>
__device__ __forceinline__ void ortho_nn_dev(const float (*v)[N], float* r);

template <>
__device__ __forceinline__ void ortho_nn_dev<4>(const float (*v)[4], float* r)
{
        r[0] = +v[0][1] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) - v[0][2] * (v[1][1] * v[2][3] - v[1][3] * v[2][1]) +
               v[0][3] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]);
        r[1] = -v[0][0] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) + v[0][2] * (v[1][0] * v[2][3] - v[1][3] * v[2][0]) -
               v[0][3] * (v[1][0] * v[2][2] - v[1][2] * v[2][0]);
        r[2] = +v[0][0] * (v[1][1] * v[2][3] - v[1][3] * v[2][1]) - v[0][1] * (v[1][0] * v[2][3] - v[1][3] * v[2][0]) +
               v[0][3] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
        r[3] = -v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) + v[0][1] * (v[1][0] * v[2][2] - v[1][2] * v[2][0]) -
               v[0][2] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
}

__device__ __forceinline__ void cross3(const float* a, const float* b, float* r)
{
        r[0] = +(a[1] * b[2] - a[2] * b[1]);
        r[1] = -(a[0] * b[2] - a[2] * b[0]);
        r[2] = +(a[0] * b[1] - a[1] * b[0]);
}

template <int N>
__device__ __forceinline__ void complement(const float* u, float (*basis)[N])
{
        const float LIMIT = 0.1f;
        if constexpr (N == 3)
        {
                float nc[3] = {0, 0, 0};
                if (fabsf(u[0]) > LIMIT)
                {
                        nc[1] = 1;
                }
                else
                {
                        nc[0] = 1;
                }
                cross3(u, nc, basis[0]);
                vnormalize<3>(basis[0]);
                cross3(u, basis[0], basis[1]);
        }
        else if constexpr (N == 4)
        {
                int exclude_axis = 0;
                for (; exclude_axis < N - 2; ++exclude_axis)
                {
                        if (fabsf(u[exclude_axis]) > LIMIT)
                        {
                                break;
                        }
                }
                float sb[N - 1][N];
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        sb[N - 2][k] = u[k];
                }
                int num = 0;
                for (int i = 0; num < N - 2; ++i)
                {
                        if (i != exclude_axis)
                        {
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        sb[num][k] = (k == i) ? 1.0f : 0.0f;
                                }
                                ++num;
                        }
                }
#pragma unroll
                for (int i = 0; i < N - 2; ++i)
                {
                        float o[N];
                        ortho_nn_dev<N>(sb, o);
                        vnormalize<N>(o);
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                sb[i][k] = o[k];
                        }
                }
                float o[N];
                ortho_nn_dev<N>(sb, o);
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        sb[N - 2][k] = o[k];
                }
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                basis[i][k] = sb[i][k];
                        }
                }
        }
        else
        {
                int exclude_axis = 0;
                for (; exclude_axis < N - 1; ++exclude_axis)
                {
                        if (fabsf(u[exclude_axis]) > LIMIT)
                        {
                                break;
                        }
                }
                float ob[N][N];
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        ob[0][k] = u[k];
                }
                // basis vectors after u: the unit axes except exclude_axis, in order
#pragma unroll
                for (int i = 1; i < N; ++i)
                {
                        int axis = (i - 1 < exclude_axis) ? i - 1 : i;
                        float b[N];
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                b[k] = (k == axis) ? 1.0f : 0.0f;
                        }
                        float sum[N];
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                sum[k] = 0;
                        }
#pragma unroll
                        for (int q = 0; q < i; ++q)
                        {
                                float d = vdot<N>(b, ob[q]);
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        sum[k] = sum[k] + d * ob[q][k];
                                }
                        }
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                ob[i][k] = b[k] - sum[k];
                        }
                        vnormalize<N>(ob[i]);
                }
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
#pragma unroll
                        for (int k = 0; k < N; ++k)
                        {
                                basis[i][k] = ob[i + 1][k];
                        }
                }
        }
}

// pow(len2, 0.5 (0.5 N - 1.5)) for N = 4, 5, 6 through square roots in double
template <int N>
__device__ __forceinline__ float radial_scale(float len2)
{
        double x = (double)len2;
        if constexpr (N == 4)
        {
                return (float)__dsqrt_rn(__dsqrt_rn(x));
        }
        else if constexpr (N == 5)
        {
                return (float)__dsqrt_rn(x);
        }
        else
        {
                return (float)(__dsqrt_rn(x) * __dsqrt_rn(__dsqrt_rn(x)));
        }
}

// random_cosine_weighted_on_hemisphere with the ball point by rejection; false if the attempt
// bound ran out (probability < 1e-19 per call)
template <int N>
__device__ bool cosine_hemisphere(uint32_t k0, uint32_t k1, unsigned long long path, uint32_t stream, const float* normal,
                                  float* res)
{
        constexpr int M = N - 1;
        float v[M];
        float len2 = 0;
        bool ok = false;
        for (uint32_t attempt = 0; attempt < 256; ++attempt)
        {
                float u[8];
                if constexpr (M <= 4)
                {
                        float4 a = rng4(k0, k1, path, stream, attempt);
                        u[0] = a.x;
                        u[1] = a.y;
                        u[2] = a.z;
                        u[3] = a.w;
                }
                else
                {
                        float4 a = rng4(k0, k1, path, stream, 2 * attempt);
                        float4 b = rng4(k0, k1, path, stream, 2 * attempt + 1);
                        u[0] = a.x;
                        u[1] = a.y;
                        u[2] = a.z;
                        u[3] = a.w;
                        u[4] = b.x;
                }
#pragma unroll
                for (int j = 0; j < M; ++j)
                {
                        v[j] = 2.0f * u[j] - 1.0f;
                }
                len2 = vdot<M>(v, v);
                if (len2 <= 1 && len2 > 0)
                {
                        ok = true;
                        break;
                }
        }
        if (!ok)
        {
                return false;
        }
        if constexpr (N >= 4)
        {
                float k = radial_scale<N>(len2);
#pragma unroll
                for (int j = 0; j < M; ++j)
                {
                        v[j] *= k;
                }
                len2 *= k * k;
        }
        float nz = __fsqrt_rn(1.0f - len2);
        float basis[N - 1][N];
        complement<N>(normal, basis);
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                res[k] = nz * normal[k];
        }
#pragma unroll
        for (int j = 0; j < M; ++j)
        {
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        res[k] = res[k] + v[j] * basis[j][k];
                }
        }
        return true;
}

// Projector::ray (projector.h:102-275)
template <int N>
__device__ __forceinline__ void projector_ray(const ProjDev<N>& P, const float* point, Ray<N>& r)
{
        float sp[N - 1];
#pragma unroll
        for (int j = 0; j < N - 1; ++j)
        {
                sp[j] = P.screen_org[j] + point[j];
        }
        float sd[N];
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                sd[k] = P.axes[0][k] * sp[0];
        }
#pragma unroll
        for (int j = 1; j < N - 1; ++j)
        {
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        sd[k] = sd[k] + P.axes[j][k] * sp[j];
                }
        }
        float org[N], dir[N];
        if (P.kind == 0)
        {
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        org[k] = P.cam_org[k] + sd[k];
                        dir[k] = P.cam_dir[k];
                }
        }
        else if (P.kind == 1)
        {
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        org[k] = P.cam_org[k];
                        dir[k] = P.cam_dir[k] + sd[k];
                }
        }
        else
        {
                float radicand = P.square_radius - vdot<N - 1>(sp, sp);
                float z = __fsqrt_rn(radicand > 0 ? radicand : 0.0f);
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        org[k] = P.cam_org[k];
                        dir[k] = P.cam_dir[k] * z + sd[k];
                }
        }
        ray_set<N>(r, org, dir);
}

// PointLight / ConstantLight::properties (light_source.h:42-77)
template <int N>
__device__ __forceinline__ void light_properties(const LightDev& L, const float* p, float* color, float* vec)
{
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                vec[k] = L.pos[k] - p[k];
        }
        if (L.kind == 1)
        {
                color[0] = L.color[0];
                color[1] = L.color[1];
                color[2] = L.color[2];
                return;
        }
        float sq = vdot<N>(vec, vec);
        float denom;
        if constexpr (N == 3)
        {
                denom = sq;
        }
        else if constexpr (N == 4)
        {
                denom = sq * __fsqrt_rn(sq);
        }
        else if constexpr (N == 5)
        {
                denom = sq * sq;
        }
        else
        {
                denom = sq * sq * __fsqrt_rn(sq);
        }
        float k = __fdiv_rn(L.coef, denom);
        color[0] = L.color[0] * k;
        color[1] = L.color[1] * k;
        color[2] = L.color[2] * k;
}

__device__ __forceinline__ float cmax3(const float* c)
{
        float a = (c[0] < c[1]) ? c[1] : c[0];
        return (c[2] < a) ? a : c[2];
}

// warp-aggregated counter increment
__device__ __forceinline__ void warp_add(unsigned long long* counter, long long v)
{
        unsigned mask = __activemask();
        if (mask == 0xffffffffu)
        {
                long long sum = v;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                {
                        sum += __shfl_xor_sync(0xffffffffu, sum, o);
                }
                if ((threadIdx.x & 31) == 0 && sum != 0)
                {
                        atomicAdd(counter, (unsigned long long)sum);
                }
        }
        else if (v != 0)
        {
                atomicAdd(counter, (unsigned long long)v);
        }
}
}
