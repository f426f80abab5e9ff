// Host side of the C ABI (include/ntrace.h): scene assembly, per-facet setup, the multithreaded
// 2^N-tree build, device packing, the wavefront render driver and the fixed-ray-set query.
#include "ntrace.h"

#include "device_types.h"
#include "geometry.hpp"
#include "kernels.h"
#include "treebuild.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace
{
thread_local std::string g_error;

struct NtError : std::runtime_error
{
        int code;
        NtError(int c, const std::string& m) : std::runtime_error(m), code(c)
        {
        }
};

[[noreturn]] void fail(int code, const std::string& msg)
{
        throw NtError(code, msg);
}

void check_cuda(cudaError_t e, const char* what)
{
        if (e != cudaSuccess)
        {
                fail(e == cudaErrorMemoryAllocation ? NT_ENOMEM : NT_ECUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
        }
}

template <typename F>
int guarded(F&& f)
{
        try
        {
                f();
                return NT_OK;
        }
        catch (const NtError& e)
        {
                g_error = e.what();
                return e.code;
        }
        catch (const std::bad_alloc&)
        {
                g_error = "host allocation failed";
                return NT_ENOMEM;
        }
        catch (const std::exception& e)
        {
                g_error = e.what();
                return NT_EINVAL;
        }
}

unsigned hardware_threads()
{
        unsigned t = std::thread::hardware_concurrency();
        return t ? t : 1;
}

// Runs f(i) for i in [0, count) on `threads` threads (dynamic scheduling).
template <typename F>
void parallel_for(long long count, unsigned threads, F&& f)
{
        if (count <= 0)
        {
                return;
        }
        threads = (unsigned)std::min<long long>(threads, count);
        if (threads <= 1)
        {
                for (long long i = 0; i < count; ++i)
                {
                        f(i);
                }
                return;
        }
        std::atomic<long long> next{0};
        std::exception_ptr err;
        std::mutex err_lock;
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; ++t)
        {
                pool.emplace_back([&]() {
                        try
                        {
                                while (true)
                                {
                                        long long i = next.fetch_add(1);
                                        if (i >= count)
                                        {
                                                break;
                                        }
                                        f(i);
                                }
                        }
                        catch (...)
                        {
                                std::lock_guard lg(err_lock);
                                if (!err)
                                {
                                        err = std::current_exception();
                                }
                                next.store(count);
                        }
                });
        }
        for (auto& th : pool)
        {
                th.join();
        }
        if (err)
        {
                std::rethrow_exception(err);
        }
}

// device buffer owning a cudaMalloc'd region
struct DevBuf
{
        void* p = nullptr;
        size_t bytes = 0;

        DevBuf() = default;
        DevBuf(const DevBuf&) = delete;
        DevBuf& operator=(const DevBuf&) = delete;
        DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes)
        {
                o.p = nullptr;
                o.bytes = 0;
        }
        DevBuf& operator=(DevBuf&& o) noexcept
        {
                if (this != &o)
                {
                        reset();
                        p = o.p;
                        bytes = o.bytes;
                        o.p = nullptr;
                        o.bytes = 0;
                }
                return *this;
        }
        ~DevBuf()
        {
                reset();
        }
        void reset()
        {
                if (p)
                {
                        cudaFree(p);
                }
                p = nullptr;
                bytes = 0;
        }
        void alloc(size_t b)
        {
                reset();
                if (b == 0)
                {
                        return;
                }
                check_cuda(cudaMalloc(&p, b), "cudaMalloc");
                bytes = b;
        }
        template <typename T>
        void upload(const std::vector<T>& v, cudaStream_t st)
        {
                alloc(v.size() * sizeof(T));
                if (bytes)
                {
                        check_cuda(cudaMemcpyAsync(p, v.data(), bytes, cudaMemcpyHostToDevice, st), "upload");
                }
        }
        template <typename T>
        T* as() const
        {
                return static_cast<T*>(p);
        }
};

int tree_max_depth(int n)
{
        switch (n)
        {
        case 3:
                return 10;
        case 4:
                return 8;
        case 5:
                return 6;
        default:
                return 5;
        }
}

constexpr int TREE_MIN_OBJECTS_PER_BOX = 10;       // mesh.cpp:33
constexpr int DISTANCE_FROM_FACET_IN_EPSILONS = 20;  // tree.h:416

struct MeshHost
{
        std::vector<float> vertices;
        std::vector<int32_t> facets;
        nt_surface surface;
        std::vector<float> normals;           // vertex normals (optional)
        std::vector<int32_t> facet_normals;   // N normal indices per facet
        // built
        std::vector<float> rec32;
        std::vector<double> rec64;
        std::vector<int32_t> nodes;  // int2 pairs
        std::vector<int32_t> leaf_idx;
        std::vector<float> level_sizes;  // (levels) x n
        std::vector<float> root_org, root_d1;
        float dist = 0;
        std::vector<float> vmin, vmax;
        long long leaf_count = 0;
        long long degenerate = 0;
        double build_seconds = 0;
        std::vector<int32_t> ntype;  // per facet: NormalType and reversed-vertex bits (MeshDev::ntype)
        DevBuf d_rec32, d_rec64, d_nodes, d_idx;
        DevBuf d_leafrec;  // rec32 gathered in leaf-list order (made on the device from d_rec32, d_idx)
        DevBuf d_normals, d_fnormals, d_ntype;
        // device staging copy of the four arrays (nt_scene_upload_begin / _commit)
        DevBuf d_stage;
        // pinned host copy of the four device arrays, back to back (re-upload, nt_scene_upload)
        void* pinned = nullptr;
        size_t pinned_bytes = 0;
        // facet setup and tree done / device arrays current: a rebuild after edits that leave the
        // mesh unchanged (lights, surfaces, projector) reuses both
        bool ready = false;
        bool uploaded = false;

        MeshHost() = default;
        MeshHost(const MeshHost&) = delete;
        MeshHost& operator=(const MeshHost&) = delete;
        MeshHost(MeshHost&& o) noexcept
                : vertices(std::move(o.vertices)), facets(std::move(o.facets)), surface(o.surface),
                  normals(std::move(o.normals)), facet_normals(std::move(o.facet_normals)), rec32(std::move(o.rec32)),
                  rec64(std::move(o.rec64)), nodes(std::move(o.nodes)), leaf_idx(std::move(o.leaf_idx)),
                  level_sizes(std::move(o.level_sizes)), root_org(std::move(o.root_org)), root_d1(std::move(o.root_d1)),
                  dist(o.dist), vmin(std::move(o.vmin)), vmax(std::move(o.vmax)), leaf_count(o.leaf_count),
                  degenerate(o.degenerate), build_seconds(o.build_seconds), ntype(std::move(o.ntype)),
                  d_rec32(std::move(o.d_rec32)), d_rec64(std::move(o.d_rec64)), d_nodes(std::move(o.d_nodes)),
                  d_idx(std::move(o.d_idx)), d_leafrec(std::move(o.d_leafrec)), d_normals(std::move(o.d_normals)),
                  d_fnormals(std::move(o.d_fnormals)),
                  d_ntype(std::move(o.d_ntype)), d_stage(std::move(o.d_stage)),
                  pinned(o.pinned), pinned_bytes(o.pinned_bytes), ready(o.ready), uploaded(o.uploaded)
        {
                o.pinned = nullptr;
                o.pinned_bytes = 0;
        }
        ~MeshHost()
        {
                if (pinned)
                {
                        cudaFreeHost(pinned);
                }
        }
};

struct PltHost
{
        std::vector<float> org, edges;
        nt_surface surface;
        std::vector<float> pn, d1, d2, vmin, vmax;
};

struct HpltHost
{
        std::vector<float> org, edges;
        nt_surface surface;
        std::vector<float> normal, planes, vmin, vmax;
};

struct LightHost
{
        int kind;
        std::vector<float> pos;
        float color[3];
        float unit;
};

struct ObjRef
{
        int kind;
        int index;
};
}

struct nt_scene
{
        int n;
        std::vector<MeshHost> meshes;
        std::vector<PltHost> plts;
        std::vector<HpltHost> hplts;
        std::vector<ObjRef> objects;
        std::vector<LightHost> lights;
        bool has_projector = false;
        int proj_kind = 0;
        std::vector<float> cam_org, cam_dir, axes;
        float proj_param = 0;
        std::vector<int> screen;
        nt_surface background{{0, 0, 0}, 1, 0, {0, 0, 0}};
        bool built = false;       // built and uploaded: renderable
        bool built_host = false;  // facet setup and trees built on the host only
        int leaf_records = 0;     // nt_build_opts.leaf_records
        float ray_offset = 0;
        // device
        cudaStream_t stream = nullptr;
        DevBuf accum;
        DevBuf pool;
        long long pool_paths = 0;
        int pool_lights = 0;
        bool pool_smooth = false;
        DevBuf counters;
        DevBuf moments;  // per-path sums of nt_render_moments
        DevBuf mean_buf; // mean colours for nt_accum_read and nt_render_pixels
        DevBuf list_buf; // nt_render_pixels: the pixel list, then its per-entry sums
        unsigned long long* host_counters = nullptr;
        long long samples_done = 0;
        std::vector<unsigned char> dev_scene;  // packed DevScene<N>
        // double-buffered upload: the copy stream fills the meshes' staging buffers; `staged` marks the
        // end of that copy, `consumed` the end of the device copies out of staging
        cudaStream_t copy_stream = nullptr;
        cudaEvent_t staged = nullptr;
        cudaEvent_t consumed = nullptr;
        bool consumed_recorded = false;
        bool upload_staged = false;

        ~nt_scene()
        {
                if (copy_stream)
                {
                        cudaStreamSynchronize(copy_stream);
                        cudaStreamDestroy(copy_stream);
                }
                if (staged)
                {
                        cudaEventDestroy(staged);
                }
                if (consumed)
                {
                        cudaEventDestroy(consumed);
                }
                if (host_counters)
                {
                        cudaFreeHost(host_counters);
                }
                if (stream)
                {
                        cudaStreamDestroy(stream);
                }
        }

        long long pixel_count() const
        {
                long long p = 1;
                for (int s : screen)
                {
                        p *= s;
                }
                return p;
        }
};

namespace
{
using namespace ntrace;

// ------------------------------------------------------------------------------------------------
// Mesh setup and tree build

template <int N>
void build_mesh(MeshHost& m, unsigned threads, bool tree_on_gpu, cudaStream_t stream)
{
        using V32 = Vec<N, float>;
        using V64 = Vec<N, double>;
        auto t0 = std::chrono::steady_clock::now();
        const long long nf = (long long)m.facets.size() / N;
        const long long nv = (long long)m.vertices.size() / N;
        if (nf < 1)
        {
                fail(NT_EINVAL, "No facets found in mesh");
        }
        for (int32_t v : m.facets)
        {
                if (v < 0 || v >= nv)
                {
                        fail(NT_EINVAL, "facet vertex index out of range");
                }
        }
        for (float x : m.vertices)
        {
                if (!std::isfinite(x))
                {
                        fail(NT_EINVAL, "mesh vertex is not finite");
                }
        }
        // per-facet setup (MeshHyperplaneSimplex ctor, mesh_hyperplane_simplex.cpp:59-143)
        std::vector<SimplexShape<N, float>> shapes(nf);
        m.rec32.assign((size_t)nf * Rec32<N>::FLOATS, 0.0f);
        m.rec64.assign((size_t)nf * Rec64<N>::DOUBLES, 0.0);
        std::atomic<long long> degenerate{0};
        std::atomic<long long> bad{-1};
        const bool has_normals = !m.normals.empty();
        if (has_normals)
        {
                m.ntype.assign(nf, 0);
        }
        else
        {
                m.ntype.clear();
        }
        parallel_for((nf + 1023) / 1024, threads, [&](long long chunk) {
                long long end = std::min(nf, (chunk + 1) * 1024);
                for (long long f = chunk * 1024; f < end; ++f)
                {
                        std::array<V32, N> v32;
                        std::array<V64, N> v64;
                        for (int i = 0; i < N; ++i)
                        {
                                const float* p = &m.vertices[(size_t)m.facets[f * N + i] * N];
                                for (int k = 0; k < N; ++k)
                                {
                                        v32[i][k] = p[k];
                                        v64[i][k] = p[k];
                                }
                        }
                        if (!shapes[f].init(v32))
                        {
                                long long expected = -1;
                                bad.compare_exchange_strong(expected, f);
                                continue;
                        }
                        // FP64 record in the reference formulation
                        std::array<V64, N - 1> vec;
                        for (int i = 0; i < N - 1; ++i)
                        {
                                for (int k = 0; k < N; ++k)
                                {
                                        vec[i][k] = v64[i + 1][k] - v64[0][k];
                                }
                        }
                        V64 n64 = normalize<N, double>(ortho_nn<N, double>(vec));
                        bool finite = true;
                        for (int k = 0; k < N; ++k)
                        {
                                finite &= std::isfinite(n64[k]);
                        }
                        if (!finite)
                        {
                                long long expected = -1;
                                bad.compare_exchange_strong(expected, f);
                                continue;
                        }
                        std::array<std::array<double, N + 1>, N - 1> pl64;
                        reference_planes<N, double>(n64, v64, &pl64);
                        double* r64 = &m.rec64[(size_t)f * Rec64<N>::DOUBLES];
                        for (int k = 0; k < N; ++k)
                        {
                                r64[k] = v64[0][k];
                                r64[Rec64<N>::OFF_NORMAL + k] = n64[k];
                        }
                        for (int i = 0; i < N - 1; ++i)
                        {
                                for (int k = 0; k <= N; ++k)
                                {
                                        r64[Rec64<N>::OFF_PLANES + i * (N + 1) + k] = pl64[i][k];
                                }
                        }
                        // FP32 record: planes by partial-pivot Gaussian elimination in FP64
                        std::array<std::array<double, N + 1>, N - 1> ge;
                        double cond = gauss_planes<N>(n64, v64, &ge);
                        float* r32 = &m.rec32[(size_t)f * Rec32<N>::FLOATS];
                        double d0 = 0;
                        for (int k = 0; k < N; ++k)
                        {
                                r32[k] = (float)n64[k];
                                d0 += n64[k] * v64[0][k];
                        }
                        r32[Rec32<N>::OFF_D0] = (float)d0;
                        float B = 0, D = 0;
                        for (int i = 0; i < N - 1; ++i)
                        {
                                float l1 = 0;
                                for (int k = 0; k <= N; ++k)
                                {
                                        float x = (float)ge[i][k];
                                        r32[Rec32<N>::OFF_PLANES + i * (N + 1) + k] = x;
                                        if (k < N)
                                        {
                                                l1 += std::fabs(x);
                                        }
                                }
                                B = std::max(B, l1);
                                D = std::max(D, std::fabs((float)ge[i][N]));
                        }
                        bool ok = std::isfinite(B) && std::isfinite(D) && cond > 1e-9;
                        if (!ok)
                        {
                                B = INFINITY;
                                D = 0;
                                degenerate.fetch_add(1);
                        }
                        r32[Rec32<N>::OFF_B] = B;
                        r32[Rec32<N>::OFF_D] = D;
                        if (has_normals && m.facet_normals[f * N] >= 0)
                        {
                                // NormalType (mesh_hyperplane_simplex.cpp:96-143); LIMIT_COSINE = 0.7
                                double dots[N];
                                bool flat = false, all_pos = true, all_neg = true;
                                for (int i = 0; i < N; ++i)
                                {
                                        const float* vn = &m.normals[(size_t)m.facet_normals[f * N + i] * N];
                                        double d = 0;
                                        for (int k = 0; k < N; ++k)
                                        {
                                                d += (double)vn[k] * n64[k];
                                        }
                                        dots[i] = d;
                                        flat |= std::fabs(d) < 0.7;
                                        all_pos &= d > 0;
                                        all_neg &= d < 0;
                                }
                                int type = 0;
                                if (!flat && all_pos)
                                {
                                        type = 1;
                                }
                                else if (!flat && all_neg)
                                {
                                        // the facet normal is reversed to agree with the vertex normals (the
                                        // intersection distance does not depend on its sign)
                                        type = 1;
                                        for (int k = 0; k <= N; ++k)
                                        {
                                                if (k < N)
                                                {
                                                        r64[Rec64<N>::OFF_NORMAL + k] = -r64[Rec64<N>::OFF_NORMAL + k];
                                                }
                                                r32[k] = -r32[k];
                                        }
                                }
                                else if (!flat)
                                {
                                        type = 2;
                                        for (int i = 0; i < N; ++i)
                                        {
                                                if (dots[i] < 0)
                                                {
                                                        type |= 1 << (2 + i);
                                                }
                                        }
                                }
                                m.ntype[f] = type;
                        }
                }
        });
        if (bad.load() >= 0)
        {
                fail(NT_EDEGENERATE, "Simplex normal is not finite (facet " + std::to_string(bad.load()) + ")");
        }
        m.degenerate = degenerate.load();

        // bounds for compute_ray_offset (Mesh::m_min/m_max over facet vertices, mesh.cpp:82-93)
        m.vmin.assign(N, std::numeric_limits<float>::max());
        m.vmax.assign(N, std::numeric_limits<float>::lowest());
        for (long long f = 0; f < nf; ++f)
        {
                for (int i = 0; i < N; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                float x = shapes[f].v[i][k];
                                m.vmin[k] = std::min(m.vmin[k], x);
                                m.vmax[k] = std::max(m.vmax[k], x);
                        }
                }
        }

        // ---- 2^N-tree (SpatialSubdivisionTree::decompose, tree.h:466-525) ----
        const int max_depth = tree_max_depth(N);
        const int max_divisions = 1 << (max_depth - 1);
        V32 mn, mx;
        for (int k = 0; k < N; ++k)
        {
                mn[k] = std::numeric_limits<float>::max();
                mx[k] = std::numeric_limits<float>::lowest();
        }
        for (long long f = 0; f < nf; ++f)
        {
                for (int i = 0; i < N; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                mn[k] = smin(shapes[f].v[i][k], mn[k]);
                                mx[k] = smax(shapes[f].v[i][k], mx[k]);
                        }
                }
        }
        for (int k = 0; k < N; ++k)
        {
                if (!(mn[k] < mx[k]))
                {
                        fail(NT_EDEGENERATE, "Objects for (2^N)-tree don't form N-dimensional object");
                }
        }
        float all_max = std::numeric_limits<float>::lowest();
        for (int k = 0; k < N; ++k)
        {
                float abs_max = smax(std::fabs(mn[k]), std::fabs(mx[k]));
                float guard = abs_max * (DISTANCE_FROM_FACET_IN_EPSILONS * std::numeric_limits<float>::epsilon());
                mn[k] -= guard;
                mx[k] += guard;
                all_max = smax(abs_max, all_max);
        }
        const float dist = all_max * (DISTANCE_FROM_FACET_IN_EPSILONS * std::numeric_limits<float>::epsilon());
        for (int k = 0; k < N; ++k)
        {
                float half_min_box = (mx[k] - mn[k]) / max_divisions / 2;
                if (dist >= half_min_box)
                {
                        fail(NT_EDEGENERATE, "The minimal distance from facets is greater than one half of the minimum box size");
                }
        }
        V32 size0;
        for (int k = 0; k < N; ++k)
        {
                size0[k] = mx[k] - mn[k];
                if (!(size0[k] > 0))
                {
                        fail(NT_EDEGENERATE, "Error orthogonal parallelotope sizes");
                }
        }
        m.dist = dist;
        m.root_org.assign(mn.begin(), mn.end());
        m.root_d1.resize(N);
        for (int k = 0; k < N; ++k)
        {
                m.root_d1[k] = mn[k] + size0[k];
        }
        m.level_sizes.resize((size_t)(max_depth + 1) * N);
        {
                V32 s = size0;
                for (int lvl = 0; lvl <= max_depth; ++lvl)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                m.level_sizes[lvl * N + k] = s[k];
                                s[k] = s[k] / 2;
                        }
                }
        }

        if (tree_on_gpu)
        {
                TreeResult tr;
                build_tree_gpu<N>(shapes, mn, m.level_sizes, max_depth, TREE_MIN_OBJECTS_PER_BOX, stream, &tr);
                if (tr.error != cudaSuccess)
                {
                        fail(tr.error == cudaErrorMemoryAllocation ? NT_ENOMEM : NT_ECUDA, "GPU tree build: " + tr.message);
                }
                m.nodes.swap(tr.nodes);
                m.leaf_idx.swap(tr.leaf_idx);
                m.leaf_count = tr.leaf_count;
                m.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                return;
        }
        // breadth-first: level by level; children of a split box are contiguous
        struct Work
        {
                long long node;
                V32 org;
                std::vector<int32_t> list;
        };
        std::vector<Work> cur(1);
        cur[0].node = 0;
        cur[0].org = mn;
        cur[0].list.resize(nf);
        for (long long f = 0; f < nf; ++f)
        {
                cur[0].list[f] = (int32_t)f;
        }
        std::vector<int32_t> nodes(2, 0);
        struct LeafRef
        {
                long long node;
                std::vector<int32_t> list;
        };
        std::vector<LeafRef> leaves;
        long long node_count = 1;
        for (int depth = 1; !cur.empty(); ++depth)
        {
                std::vector<long long> split;
                for (long long i = 0; i < (long long)cur.size(); ++i)
                {
                        if (depth >= max_depth || (long long)cur[i].list.size() <= TREE_MIN_OBJECTS_PER_BOX)
                        {
                                leaves.push_back({cur[i].node, std::move(cur[i].list)});
                        }
                        else
                        {
                                split.push_back(i);
                        }
                }
                const int C = 1 << N;
                std::vector<Work> next(split.size() * C);
                nodes.resize((size_t)(node_count + (long long)split.size() * C) * 2, 0);
                for (size_t s = 0; s < split.size(); ++s)
                {
                        long long first = node_count + (long long)s * C;
                        nodes[cur[split[s]].node * 2 + 0] = (int32_t)first;
                        nodes[cur[split[s]].node * 2 + 1] = -1;
                }
                const float* half = &m.level_sizes[depth * N];
                parallel_for((long long)split.size() * C, threads, [&](long long w) {
                        const Work& parent = cur[split[w / C]];
                        int c = (int)(w % C);
                        Work& child = next[w];
                        child.node = node_count + w;
                        for (int k = 0; k < N; ++k)
                        {
                                float org_plus_half = parent.org[k] + half[k];
                                child.org[k] = (c & (1 << k)) ? org_plus_half : parent.org[k];
                        }
                        V32 hs;
                        for (int k = 0; k < N; ++k)
                        {
                                hs[k] = half[k];
                        }
                        Box<N, float> box = Box<N, float>::make(child.org, hs);
                        for (int32_t f : parent.list)
                        {
                                if (box_simplex_overlap<N, float>(box, shapes[f]))
                                {
                                        child.list.push_back(f);
                                }
                        }
                });
                node_count += (long long)split.size() * C;
                if (node_count > (1ll << 31) - 1)
                {
                        fail(NT_EINVAL, "tree too large");
                }
                cur.swap(next);
        }
        std::sort(leaves.begin(), leaves.end(), [](const LeafRef& a, const LeafRef& b) { return a.node < b.node; });
        m.leaf_idx.clear();
        for (auto& lf : leaves)
        {
                nodes[lf.node * 2 + 0] = (int32_t)m.leaf_idx.size();
                nodes[lf.node * 2 + 1] = (int32_t)lf.list.size();
                m.leaf_idx.insert(m.leaf_idx.end(), lf.list.begin(), lf.list.end());
        }
        if (m.leaf_idx.empty())
        {
                m.leaf_idx.push_back(0);
        }
        m.nodes.swap(nodes);
        m.leaf_count = (long long)leaves.size();
        m.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// General parallelotope in float (Parallelotope::create_planes, parallelotope.h:160-185)
template <int N>
void build_plt(PltHost& p)
{
        std::array<Vec<N, float>, N> e;
        Vec<N, float> org;
        for (int k = 0; k < N; ++k)
        {
                org[k] = p.org[k];
                for (int i = 0; i < N; ++i)
                {
                        e[i][k] = p.edges[i * N + k];
                }
        }
        p.pn.assign(N * N, 0);
        p.d1.assign(N, 0);
        p.d2.assign(N, 0);
        for (int i = 0; i < N; ++i)
        {
                std::array<Vec<N, float>, N - 1> sub;
                for (int j = 0, c = 0; j < N; ++j)
                {
                        if (j != i)
                        {
                                sub[c++] = e[j];
                        }
                }
                Vec<N, float> nn = normalize<N, float>(ortho_nn<N, float>(sub));
                for (int k = 0; k < N; ++k)
                {
                        if (!std::isfinite(nn[k]))
                        {
                                fail(NT_EDEGENERATE, "degenerate parallelotope");
                        }
                }
                float d1 = dot<N, float>(org, nn);
                Vec<N, float> oe;
                for (int k = 0; k < N; ++k)
                {
                        oe[k] = org[k] + e[i][k];
                }
                float d2 = -dot<N, float>(oe, nn);
                if (dot<N, float>(nn, e[i]) > 0)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                nn[k] = -nn[k];
                        }
                        d1 = -d1;
                        d2 = -d2;
                }
                for (int k = 0; k < N; ++k)
                {
                        p.pn[i * N + k] = nn[k];
                }
                p.d1[i] = d1;
                p.d2[i] = d2;
        }
        // vertex_min_max over parallelotope_vertices (parallelotope_algorithm.h:64-86)
        p.vmin.assign(N, 0);
        p.vmax.assign(N, 0);
        for (int v = 0; v < (1 << N); ++v)
        {
                Vec<N, float> x = org;
                for (int i = N - 1; i >= 0; --i)
                {
                        if (v & (1 << i))
                        {
                                for (int k = 0; k < N; ++k)
                                {
                                        x[k] = x[k] + e[i][k];
                                }
                        }
                }
                for (int k = 0; k < N; ++k)
                {
                        p.vmin[k] = v == 0 ? x[k] : smin(x[k], p.vmin[k]);
                        p.vmax[k] = v == 0 ? x[k] : smax(x[k], p.vmax[k]);
                }
        }
}

// Hyperplane parallelotope in float (HyperplaneParallelotope::set_data, hyperplane_parallelotope.h:76-82)
template <int N>
void build_hplt(HpltHost& h)
{
        std::array<Vec<N, float>, N - 1> e;
        Vec<N, float> org;
        for (int k = 0; k < N; ++k)
        {
                org[k] = h.org[k];
                for (int i = 0; i < N - 1; ++i)
                {
                        e[i][k] = h.edges[i * N + k];
                }
        }
        Vec<N, float> nn = normalize<N, float>(ortho_nn<N, float>(e));
        for (int k = 0; k < N; ++k)
        {
                if (!std::isfinite(nn[k]))
                {
                        fail(NT_EDEGENERATE, "degenerate hyperplane parallelotope");
                }
        }
        std::array<Vec<N, float>, N> pts;
        for (int i = 0; i < N - 1; ++i)
        {
                for (int k = 0; k < N; ++k)
                {
                        pts[i][k] = org[k] + e[i][k];
                }
        }
        pts[N - 1] = org;
        std::array<std::array<float, N + 1>, N - 1> pl;
        reference_planes<N, float>(nn, pts, &pl);
        h.normal.assign(nn.begin(), nn.end());
        h.planes.assign((N - 1) * (N + 1), 0);
        for (int i = 0; i < N - 1; ++i)
        {
                for (int k = 0; k <= N; ++k)
                {
                        h.planes[i * (N + 1) + k] = pl[i][k];
                }
        }
        h.vmin.assign(N, 0);
        h.vmax.assign(N, 0);
        for (int v = 0; v < (1 << (N - 1)); ++v)
        {
                Vec<N, float> x = org;
                for (int i = N - 2; i >= 0; --i)
                {
                        if (v & (1 << i))
                        {
                                for (int k = 0; k < N; ++k)
                                {
                                        x[k] = x[k] + e[i][k];
                                }
                        }
                }
                for (int k = 0; k < N; ++k)
                {
                        h.vmin[k] = v == 0 ? x[k] : smin(x[k], h.vmin[k]);
                        h.vmax[k] = v == 0 ? x[k] : smax(x[k], h.vmax[k]);
                }
        }
}

void copy_obj(ObjDev* o, int kind, int index, const nt_surface& s)
{
        o->kind = kind;
        o->index = index;
        for (int c = 0; c < 3; ++c)
        {
                o->color[c] = s.color[c];
                o->light_color[c] = s.light_color[c];
        }
        o->diffuse = s.diffuse;
        o->light_source = s.light_source;
}

// FP32 record size in float4s at dimension n (Rec32<n>::F4).
int rec32_f4(int n)
{
        return (n * n + n + 2 + 3) / 4;
}

// The leaves' records in leaf-list order, gathered on the device from the uploaded record and index
// arrays (after every upload of those, on the scene's stream).  The copy repeats a facet's record in
// every leaf that lists it (about 50 times at n = 4), so it is made only while it takes at most a
// quarter of the free device memory; without it the kernels read a leaf's records through its index
// list (leaf_record), with the same results.
void gather_leaf_records(MeshHost& m, int n, cudaStream_t st, int policy)
{
        const long long count = (long long)(m.d_idx.bytes / sizeof(int32_t));
        const size_t bytes = std::max<size_t>((size_t)count * rec32_f4(n) * 16, 16);
        if (policy < 0)
        {
                m.d_leafrec.reset();
                return;
        }
        if (m.d_leafrec.bytes != bytes)
        {
                m.d_leafrec.reset();
                size_t free_b = 0, total_b = 0;
                check_cuda(cudaMemGetInfo(&free_b, &total_b), "memory info");
                if (bytes > free_b / 4)
                {
                        return;
                }
                m.d_leafrec.alloc(bytes);
        }
        check_cuda(launch_gather_records(m.d_rec32.as<float4>(), m.d_idx.as<int>(), count, rec32_f4(n),
                                         m.d_leafrec.as<float4>(), st),
                   "gather leaf records");
}

template <int N>
MeshDev<N> mesh_dev(const MeshHost& m)
{
        MeshDev<N> d{};
        d.rec32 = m.d_rec32.as<float4>();
        d.rec64 = m.d_rec64.as<double>();
        d.nodes = m.d_nodes.as<int2>();
        d.leaf_idx = m.d_idx.as<int>();
        d.leaf_rec32 = m.d_leafrec.as<float4>();
        d.vnormals = m.ntype.empty() ? nullptr : m.d_normals.as<float>();
        d.fnormals = m.ntype.empty() ? nullptr : m.d_fnormals.as<int>();
        d.ntype = m.ntype.empty() ? nullptr : m.d_ntype.as<int>();
        d.nfacets = (int)(m.facets.size() / N);
        d.levels = (int)(m.level_sizes.size() / N);
        for (int k = 0; k < N; ++k)
        {
                d.root_org[k] = m.root_org[k];
                d.root_d1[k] = m.root_d1[k];
        }
        for (int l = 0; l < MAX_LEVELS; ++l)
        {
                for (int k = 0; k < N; ++k)
                {
                        d.size[l][k] = l < d.levels ? m.level_sizes[l * N + k] : 0.0f;
                }
        }
        d.dist = m.dist;
        return d;
}

template <int N>
void check_orthogonal(const Vec<N, float>& dir, const std::array<Vec<N, float>, N - 1>& axes)
{
        // projector_implementation::check_vectors_orthogonal (projector.h:29-50)
        const float LIMIT_COS = std::numeric_limits<float>::epsilon() * 100;
        for (int i = 0; i < N - 1; ++i)
        {
                if (!(std::fabs(dot<N, float>(axes[i], dir)) <= LIMIT_COS))
                {
                        fail(NT_EINVAL, "The screen axis " + std::to_string(i) + " is not orthogonal to the camera direction");
                }
                for (int j = i + 1; j < N - 1; ++j)
                {
                        if (!(std::fabs(dot<N, float>(axes[i], axes[j])) <= LIMIT_COS))
                        {
                                fail(NT_EINVAL, "The screen axis " + std::to_string(i) + " is not orthogonal to the screen axis " +
                                                        std::to_string(j));
                        }
                }
        }
}

template <int N>
void build_scene(nt_scene* s, unsigned threads, bool host_only, bool tree_on_gpu)
{
        if (s->objects.empty())
        {
                fail(NT_EINVAL, "scene has no objects");
        }
        if (s->lights.empty())
        {
                fail(NT_EINVAL, "scene has no light sources");
        }
        if (!s->has_projector)
        {
                fail(NT_EINVAL, "scene has no projector");
        }
        if (!host_only && !s->stream)
        {
                check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        }
        for (auto& m : s->meshes)
        {
                if (!m.ready)
                {
                        build_mesh<N>(m, threads, tree_on_gpu && !host_only, s->stream);
                        m.ready = true;
                        m.uploaded = false;
                }
                if (!host_only && !m.uploaded)
                {
                        m.d_rec32.upload(m.rec32, s->stream);
                        m.d_rec64.upload(m.rec64, s->stream);
                        m.d_nodes.upload(m.nodes, s->stream);
                        m.d_idx.upload(m.leaf_idx, s->stream);
                        gather_leaf_records(m, N, s->stream, s->leaf_records);
                        if (!m.ntype.empty())
                        {
                                m.d_normals.upload(m.normals, s->stream);
                                m.d_fnormals.upload(m.facet_normals, s->stream);
                                m.d_ntype.upload(m.ntype, s->stream);
                        }
                        check_cuda(cudaStreamSynchronize(s->stream), "upload");
                        if (m.pinned)
                        {
                                cudaFreeHost(m.pinned);
                                m.pinned = nullptr;
                        }
                        m.pinned_bytes = m.d_rec32.bytes + m.d_rec64.bytes + m.d_nodes.bytes + m.d_idx.bytes;
                        check_cuda(cudaMallocHost(&m.pinned, m.pinned_bytes), "cudaMallocHost");
                        char* p = static_cast<char*>(m.pinned);
                        std::memcpy(p, m.rec32.data(), m.d_rec32.bytes);
                        p += m.d_rec32.bytes;
                        std::memcpy(p, m.rec64.data(), m.d_rec64.bytes);
                        p += m.d_rec64.bytes;
                        std::memcpy(p, m.nodes.data(), m.d_nodes.bytes);
                        p += m.d_nodes.bytes;
                        std::memcpy(p, m.leaf_idx.data(), m.d_idx.bytes);
                        m.uploaded = true;
                }
        }
        for (auto& p : s->plts)
        {
                build_plt<N>(p);
        }
        for (auto& h : s->hplts)
        {
                build_hplt<N>(h);
        }

        auto D = std::make_unique<DevScene<N>>();
        std::memset(D.get(), 0, sizeof(DevScene<N>));
        D->nobj = (int)s->objects.size();
        for (size_t i = 0; i < s->objects.size(); ++i)
        {
                const ObjRef& o = s->objects[i];
                const nt_surface& surf = o.kind == OBJ_MESH ? s->meshes[o.index].surface
                                         : o.kind == OBJ_PLT ? s->plts[o.index].surface
                                                             : s->hplts[o.index].surface;
                copy_obj(&D->obj[i], o.kind, o.index, surf);
        }
        D->nmesh = (int)s->meshes.size();
        for (size_t i = 0; i < s->meshes.size(); ++i)
        {
                D->mesh[i] = mesh_dev<N>(s->meshes[i]);
        }
        D->nplt = (int)s->plts.size();
        for (size_t i = 0; i < s->plts.size(); ++i)
        {
                for (int a = 0; a < N; ++a)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                D->plt[i].n[a][k] = s->plts[i].pn[a * N + k];
                        }
                        D->plt[i].d1[a] = s->plts[i].d1[a];
                        D->plt[i].d2[a] = s->plts[i].d2[a];
                }
        }
        D->nhplt = (int)s->hplts.size();
        for (size_t i = 0; i < s->hplts.size(); ++i)
        {
                for (int k = 0; k < N; ++k)
                {
                        D->hplt[i].normal[k] = s->hplts[i].normal[k];
                        D->hplt[i].org[k] = s->hplts[i].org[k];
                }
                for (int a = 0; a < N - 1; ++a)
                {
                        for (int k = 0; k <= N; ++k)
                        {
                                D->hplt[i].planes[a][k] = s->hplts[i].planes[a * (N + 1) + k];
                        }
                }
        }
        D->nlights = (int)s->lights.size();
        for (size_t i = 0; i < s->lights.size(); ++i)
        {
                const LightHost& L = s->lights[i];
                D->lights[i].kind = L.kind;
                for (int k = 0; k < N; ++k)
                {
                        D->lights[i].pos[k] = L.pos[k];
                }
                for (int c = 0; c < 3; ++c)
                {
                        D->lights[i].color[c] = L.color[c];
                }
                // PointLight: m_coef = pow(unit_intensity_distance, N - 1) (light_source.h:37)
                D->lights[i].coef = (float)std::pow(L.unit, N - 1);
        }
        // projector (projector.h:52-81,102-275)
        {
                ProjDev<N>& P = D->proj;
                P.kind = s->proj_kind;
                Vec<N, float> cd;
                std::array<Vec<N, float>, N - 1> ax;
                for (int k = 0; k < N; ++k)
                {
                        P.cam_org[k] = s->cam_org[k];
                        cd[k] = s->cam_dir[k];
                }
                cd = normalize<N, float>(cd);
                for (int j = 0; j < N - 1; ++j)
                {
                        Vec<N, float> a;
                        for (int k = 0; k < N; ++k)
                        {
                                a[k] = s->axes[j * N + k];
                        }
                        ax[j] = normalize<N, float>(a);
                }
                check_orthogonal<N>(cd, ax);
                for (int j = 0; j < N - 1; ++j)
                {
                        if (s->screen[j] < 1)
                        {
                                fail(NT_EINVAL, "Projection size " + std::to_string(j) + " is not positive");
                        }
                        P.screen[j] = s->screen[j];
                        P.screen_org[j] = -s->screen[j] * (1.0f / 2);
                }
                const float PI = 3.14159265358979323846f;
                if (P.kind == NT_PROJECTOR_PARALLEL)
                {
                        if (!(s->proj_param > 0))
                        {
                                fail(NT_EINVAL, "Error units per pixel for parallel projection");
                        }
                        for (int j = 0; j < N - 1; ++j)
                        {
                                for (int k = 0; k < N; ++k)
                                {
                                        ax[j][k] *= s->proj_param;
                                }
                        }
                }
                else if (P.kind == NT_PROJECTOR_PERSPECTIVE)
                {
                        if (!(s->proj_param > 0 && s->proj_param < 180))
                        {
                                fail(NT_EINVAL, "Perspective projection: error view angle");
                        }
                        float half_angle = s->proj_param * 0.5f * PI / 180;
                        float dir_length = s->screen[0] * 0.5f * std::tan(PI / 2 - half_angle);
                        for (int k = 0; k < N; ++k)
                        {
                                cd[k] *= dir_length;
                        }
                }
                else
                {
                        if (!(s->proj_param > 0))
                        {
                                fail(NT_EINVAL, "Spherical projection view angle is not positive");
                        }
                        float half_angle = s->proj_param * 0.5f * PI / 180;
                        float sin_alpha = std::sin(half_angle);
                        float k = sin_alpha / s->screen[0];
                        float r = sin_alpha * sin_alpha;
                        for (int j = 1; j < N - 1; ++j)
                        {
                                r += (k * s->screen[j]) * (k * s->screen[j]);
                        }
                        if (!(r < 1))
                        {
                                fail(NT_EINVAL, "Spherical projection view angle is too big");
                        }
                        float rad = s->screen[0] * 0.5f / sin_alpha;
                        P.square_radius = rad * rad;
                }
                for (int k = 0; k < N; ++k)
                {
                        P.cam_dir[k] = cd[k];
                }
                for (int j = 0; j < N - 1; ++j)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                P.axes[j][k] = ax[j][k];
                        }
                }
        }
        for (int c = 0; c < 3; ++c)
        {
                D->bg_color[c] = s->background.color[c];
                D->bg_light_color[c] = s->background.light_color[c];
        }
        D->bg_light = s->background.light_source;
        // compute_ray_offset (painter.cpp:539-558)
        float all_max = std::numeric_limits<float>::lowest();
        auto fold = [&](const std::vector<float>& a, const std::vector<float>& b) {
                for (int k = 0; k < N; ++k)
                {
                        all_max = std::max(all_max, std::max(std::fabs(a[k]), std::fabs(b[k])));
                }
        };
        for (const ObjRef& o : s->objects)
        {
                if (o.kind == OBJ_MESH)
                {
                        fold(s->meshes[o.index].vmin, s->meshes[o.index].vmax);
                }
                else if (o.kind == OBJ_PLT)
                {
                        fold(s->plts[o.index].vmin, s->plts[o.index].vmax);
                }
                else
                {
                        fold(s->hplts[o.index].vmin, s->hplts[o.index].vmax);
                }
        }
        s->ray_offset = all_max * (1000 * std::numeric_limits<float>::epsilon());
        D->ray_offset = s->ray_offset;
        {
                // cosine_sphere_coefficient(N) (coefficient/cosine_sphere.h:97-162)
                double c = nt_cosine_sphere_coefficient(N);
                D->diffuse_coef = (float)c;
        }
        D->max_depth = 100;
        D->retest = 1;
        s->dev_scene.resize(sizeof(DevScene<N>));
        std::memcpy(s->dev_scene.data(), D.get(), sizeof(DevScene<N>));
        if (host_only)
        {
                s->built_host = true;
                return;
        }

        long long npix = s->pixel_count();
        s->accum.alloc((size_t)npix * 3 * sizeof(double));
        check_cuda(cudaMemsetAsync(s->accum.p, 0, s->accum.bytes, s->stream), "memset");
        s->samples_done = 0;
        s->counters.alloc(C_COUNT * sizeof(unsigned long long));
        if (!s->host_counters)
        {
                check_cuda(cudaMallocHost(&s->host_counters, C_COUNT * sizeof(unsigned long long)), "cudaMallocHost");
        }
        check_cuda(cudaStreamSynchronize(s->stream), "build sync");
        s->built = true;
}

int one_dimension_size(int n, int spp)
{
        // StratifiedJitteredSampler::one_dimension_size (sampler.h:31-52)
        int m = n - 1;
        double v = std::pow(spp, 1.0 / m);
        unsigned f = (unsigned)std::floor(v);
        unsigned long long p = 1;
        for (int i = 0; i < m; ++i)
        {
                p *= f;
        }
        if (p >= (unsigned long long)spp)
        {
                return (int)f;
        }
        return (int)std::ceil(v);
}

// smooth_normal matters only for meshes with vertex normals (without them the shading normal is the
// geometric one, as in the reference); then the wavefront carries the smooth-normal shadow queue
bool smooth_shading(const nt_scene* s, const nt_render_opts& o)
{
        if (!o.smooth_normal)
        {
                return false;
        }
        for (const MeshHost& m : s->meshes)
        {
                if (!m.ntype.empty())
                {
                        return true;
                }
        }
        return false;
}

// A pass of one scene prepared for the wavefront: checks, the pass constants, the path pool.  Type-
// erased over N so that passes of scenes of different dimensions can run side by side
// (nt_render_batch).
struct PassJob
{
        nt_scene* s = nullptr;
        long long total = 0;
        long long spp_eff = 0;
        bool smooth = false;
        bool counts_samples = true;  // the pass adds to the scene's accumulator (its sample count grows)
        bool one_mesh = false;       // the scene has one mesh (plan-and-compact kernels run)
        KernelTimes times;
        std::chrono::steady_clock::time_point t0;
        virtual ~PassJob() = default;
        // one wavefront iteration of this pass on stream st
        virtual void enqueue(int parity, cudaStream_t st) = 0;
        // the whole pass on the scene's stream
        virtual cudaError_t run(const nt_render_opts& o) = 0;
};

template <int N>
struct PassJobN final : PassJob
{
        DevScene<N> S;
        PassDev P{};
        Wavefront<N> W;
        double* accum = nullptr;
        void enqueue(int parity, cudaStream_t st) override
        {
                W.enqueue_iteration(S, P, accum, s->counters.as<unsigned long long>(), total, parity, st, nullptr, nullptr);
        }
        cudaError_t run(const nt_render_opts& o) override
        {
                return W.run(S, P, accum, s->counters.as<unsigned long long>(), s->host_counters, total, s->stream, &times,
                             o.timing != 0, o.stop, true, o.graph_iterations > 0 ? o.graph_iterations : 4);
        }
};

// The walk kernels' variant (nt_render_opts.walk_chunk): -1 unstaged, else the staging chunk in rounds
// of 32 tests; 0: the default.
int walk_rounds(const nt_render_opts& o)
{
        if (o.walk_chunk != 0 && o.walk_chunk != 1 && o.walk_chunk != 32 && o.walk_chunk != 64 && o.walk_chunk != 128)
        {
                fail(NT_EINVAL, "walk_chunk must be 0, 1, 32, 64 or 128");
        }
        return o.walk_chunk == 1 ? -1 : o.walk_chunk / 32;
}

// The walk kernels' small-leaf threshold (nt_render_opts.walk_small_leaf; 0: the default).
int walk_small(const nt_render_opts& o)
{
        if (o.walk_small_leaf < -1 || o.walk_small_leaf > 64)
        {
                fail(NT_EINVAL, "walk_small_leaf must be -1..64");
        }
        return o.walk_small_leaf == 0 ? 2 : (o.walk_small_leaf < 0 ? 0 : o.walk_small_leaf);
}

// Where a pass's radiance goes when it is not the scene's per-pixel accumulator.
struct PassTarget
{
        double* moments = nullptr;        // per-path sums (pixel * spp_eff + sample, 3 doubles each, zeroed by
                                          // the caller): nt_render_moments
        const long long* list = nullptr;  // device pixel list: nt_render_pixels ...
        long long list_count = 0;
        double* list_accum = nullptr;     // ... and its per-entry sums (3 doubles each, zeroed by the caller)
        long long first_sample = -1;      // >= 0: the pass's first sample index; < 0: from opts / the scene
};

// The first sample index of an ordinary pass: opts.sample_offset when positive, else the samples
// already accumulated (progressive passes).
long long pass_first_sample(const nt_scene* s, const nt_render_opts& o)
{
        return o.sample_offset > 0 ? (long long)o.sample_offset : s->samples_done;
}

template <int N>
std::unique_ptr<PassJob> prepare_pass(nt_scene* s, const nt_render_opts& o, const PassTarget& target = PassTarget())
{
        double* const moments_accum = target.moments;
        Wavefront<N>::prepare();  // kernel attributes before any capture of the pass's iterations
        auto job = std::make_unique<PassJobN<N>>();
        job->t0 = std::chrono::steady_clock::now();
        job->s = s;
        job->counts_samples = !target.moments && !target.list;
        job->one_mesh = s->meshes.size() == 1;
        if (o.samples_per_pixel < 1)
        {
                fail(NT_EINVAL, "Stratified jittered sample count is not a positive integer");
        }
        if (o.max_depth < 0)
        {
                fail(NT_EINVAL, "max_depth must be >= 0");
        }
        const int k = one_dimension_size(N, o.samples_per_pixel);
        long long spp_eff = 1;
        for (int i = 0; i < N - 1; ++i)
        {
                spp_eff *= k;
        }
        DevScene<N>& S = job->S;
        std::memcpy(&S, s->dev_scene.data(), sizeof(S));
        S.max_depth = o.max_depth;
        S.retest = o.retest;
        S.walk_rounds = walk_rounds(o);
        S.walk_small = walk_small(o);
        const bool smooth = smooth_shading(s, o);
        S.smooth_normal = smooth ? 1 : 0;
        const long long npix = s->pixel_count();
        const long long first_sample = target.first_sample >= 0 ? target.first_sample : pass_first_sample(s, o);
        const long long total = (target.list ? target.list_count : npix) * spp_eff;
        if ((first_sample + spp_eff) * npix >= (1ll << 62) || first_sample + spp_eff > 0xffffffffll)
        {
                fail(NT_EINVAL, "sample count overflow");
        }
        if (target.list && target.list_count > 0xffffffffll)
        {
                fail(NT_EINVAL, "too many pixels in one list");
        }
        const int lights = (int)s->lights.size();
        // default pool: 4 Mi paths (fewer wavefront iterations, so less per-launch tail), at most 1 GiB
        const long long per_path =
                (long long)(Wavefront<N>::bytes_for(1, lights, smooth) - Wavefront<N>::bytes_for(0, lights, smooth));
        long long Q = o.pool_paths > 0 ? o.pool_paths : std::min<long long>(1ll << 22, (1ll << 30) / per_path);
        Q = std::max<long long>(256, std::min(Q, total));
        if (Q > s->pool_paths || lights > s->pool_lights || (smooth && !s->pool_smooth))
        {
                s->pool.alloc(Wavefront<N>::bytes_for(Q, lights, smooth));
                s->pool_paths = Q;
                s->pool_lights = lights;
                s->pool_smooth = smooth;
        }
        // the pool may be larger than this pass asks for: carve the pass's Q from it
        job->W.carve(s->pool.as<char>(), Q, s->pool_lights, smooth);

        PassDev& P = job->P;
        P.key0 = (uint32_t)o.seed;
        P.key1 = (uint32_t)(o.seed >> 32);
        P.spp_eff = (int)spp_eff;
        P.k1d = k;
        P.recip_k = 1.0f / k;
        P.npix = npix;
        P.sample_offset = first_sample;
        P.path_begin = 0;
        P.path_end = total;
        P.moments = moments_accum ? 1 : 0;
        P.list = target.list;
        if (moments_accum && total > 0xffffffffll)
        {
                fail(NT_EINVAL, "too many paths in one moments pass");
        }
        job->accum = moments_accum ? moments_accum : (target.list ? target.list_accum : s->accum.as<double>());
        job->total = total;
        job->spp_eff = spp_eff;
        job->smooth = smooth;
        check_cuda(cudaMemsetAsync(s->counters.p, 0, s->counters.bytes, s->stream), "memset counters");
        return job;
}

// After a pass: counters to the host (already there after a batch), statistics, state.
void finish_pass(PassJob& job, const nt_render_opts& o, nt_stats* st, bool copy_counters)
{
        nt_scene* s = job.s;
        if (copy_counters)
        {
                check_cuda(cudaMemcpyAsync(s->host_counters, s->counters.p, C_COUNT * sizeof(unsigned long long),
                                           cudaMemcpyDeviceToHost, s->stream),
                           "counters");
        }
        check_cuda(cudaStreamSynchronize(s->stream), "render sync");
        const bool stopped = (o.stop && *o.stop) || !s->host_counters[C_DONE];
        s->samples_done += (stopped || !job.counts_samples) ? 0 : job.spp_eff;
        if (st)
        {
                const KernelTimes& times = job.times;
                std::memset(st, 0, sizeof(*st));
                st->paths = job.total;
                st->rays = (int64_t)s->host_counters[C_RAYS];
                st->shadow_rays = (int64_t)s->host_counters[C_SHADOW_RAYS];
                st->facet_tests = (int64_t)s->host_counters[C_FACET_TESTS];
                st->box_steps = (int64_t)s->host_counters[C_BOX_STEPS];
                st->retests = (int64_t)s->host_counters[C_RETESTS];
                st->descent_levels = (int64_t)s->host_counters[C_DESCENT];
                st->error_bits = (int64_t)s->host_counters[C_ERROR];
                st->spp_effective = (int)job.spp_eff;
                st->raygen_ms = times.raygen_ms;
                st->extend_ms = times.extend_ms;
                st->shade_ms = times.shade_ms;
                st->shadow_ms = times.shadow_ms;
                st->plan_ms = times.plan_ms;
                st->launches = times.launches;
                st->extend_launches = times.extend_launches;
                st->shadow_launches = times.shadow_launches;
                st->shadow_facet_tests = (int64_t)s->host_counters[C_SH_FACET_TESTS];
                st->shadow_box_steps = (int64_t)s->host_counters[C_SH_BOX_STEPS];
                st->shadow_retests = (int64_t)s->host_counters[C_SH_RETESTS];
                st->shadow_descent_levels = (int64_t)s->host_counters[C_SH_DESCENT];
                st->iterations = (int64_t)s->host_counters[C_ITERS];
                st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - job.t0).count();
        }
        if (s->host_counters[C_ERROR])
        {
                fail(NT_ETIMEOUT, "a bounded device loop ran out (error bits " + std::to_string(s->host_counters[C_ERROR]) + ")");
        }
        if (stopped)
        {
                fail(NT_ESTOPPED, "render stopped");
        }
}

template <int N>
void render(nt_scene* s, const nt_render_opts& o, nt_stats* st, const PassTarget& target = PassTarget())
{
        std::unique_ptr<PassJob> job = prepare_pass<N>(s, o, target);
        check_cuda(job->run(o), "render");
        finish_pass(*job, o, st, true);
}

// One pass of the wavefront on caller-provided working memory (nt_render_noalloc): the scratch holds
// the device counters (first 256 bytes) and the path pool; the pass's sums are added to d_accum.
template <int N>
void render_noalloc(nt_scene* s, const nt_render_opts& o, double* d_accum, long long sample_offset, cudaStream_t st,
                    void* scratch, size_t scratch_bytes, nt_stats* out)
{
        auto t0 = std::chrono::steady_clock::now();
        if (o.samples_per_pixel < 1)
        {
                fail(NT_EINVAL, "Stratified jittered sample count is not a positive integer");
        }
        if (o.max_depth < 0)
        {
                fail(NT_EINVAL, "max_depth must be >= 0");
        }
        if (!d_accum)
        {
                fail(NT_EINVAL, "the accumulator is NULL");
        }
        if (sample_offset < 0)
        {
                fail(NT_EINVAL, "sample_offset must be >= 0");
        }
        const int k = one_dimension_size(N, o.samples_per_pixel);
        long long spp_eff = 1;
        for (int i = 0; i < N - 1; ++i)
        {
                spp_eff *= k;
        }
        const long long npix = s->pixel_count();
        const long long total = npix * spp_eff;
        if ((sample_offset + spp_eff) * npix >= (1ll << 62) || sample_offset + spp_eff > 0xffffffffll)
        {
                fail(NT_EINVAL, "sample count overflow");
        }
        const int lights = (int)s->lights.size();
        const bool smooth = smooth_shading(s, o);
        const size_t fixed = Wavefront<N>::bytes_for(0, lights, smooth);
        const size_t per_path = Wavefront<N>::bytes_for(1, lights, smooth) - fixed;
        const size_t head = 256;  // device counters
        const long long capacity =
                scratch_bytes > head + fixed ? (long long)((scratch_bytes - head - fixed) / per_path) : 0;
        if (capacity < 256)
        {
                fail(NT_EINVAL, "the no-alloc scratch is too small for this scene");
        }
        if (o.pool_paths > capacity)
        {
                fail(NT_EINVAL, "pool_paths " + std::to_string(o.pool_paths) + " exceeds the no-alloc scratch capacity of " +
                                        std::to_string(capacity) + " paths (n = " + std::to_string(N) + ", " +
                                        std::to_string(lights) + " light(s), " + std::to_string(scratch_bytes) +
                                        " bytes)");
        }
        long long Q = o.pool_paths > 0 ? o.pool_paths : capacity;
        Q = std::max<long long>(1, std::min(Q, total));
        DevScene<N> S;
        std::memcpy(&S, s->dev_scene.data(), sizeof(S));
        S.max_depth = o.max_depth;
        S.retest = o.retest;
        S.smooth_normal = smooth ? 1 : 0;
        S.walk_rounds = walk_rounds(o);
        S.walk_small = walk_small(o);
        unsigned long long* counters = static_cast<unsigned long long*>(scratch);
        Wavefront<N> W;
        W.carve(static_cast<char*>(scratch) + head, Q, lights, smooth);
        PassDev P{};
        P.key0 = (uint32_t)o.seed;
        P.key1 = (uint32_t)(o.seed >> 32);
        P.spp_eff = (int)spp_eff;
        P.k1d = k;
        P.recip_k = 1.0f / k;
        P.npix = npix;
        P.sample_offset = sample_offset;
        P.path_begin = 0;
        P.path_end = total;
        check_cuda(cudaMemsetAsync(counters, 0, C_COUNT * sizeof(unsigned long long), st), "memset counters");
        unsigned long long host_counters[C_COUNT] = {};
        KernelTimes times;
        // the iterations are enqueued directly, not through a CUDA graph: instantiating a graph may allocate
        check_cuda(W.run(S, P, d_accum, counters, host_counters, total, st, &times, false, o.stop, false), "render");
        check_cuda(cudaMemcpyAsync(host_counters, counters, C_COUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
                   "counters");
        check_cuda(cudaStreamSynchronize(st), "render sync");
        bool stopped = o.stop && *o.stop;
        if (out)
        {
                std::memset(out, 0, sizeof(*out));
                out->paths = total;
                out->rays = (int64_t)host_counters[C_RAYS];
                out->shadow_rays = (int64_t)host_counters[C_SHADOW_RAYS];
                out->facet_tests = (int64_t)host_counters[C_FACET_TESTS];
                out->box_steps = (int64_t)host_counters[C_BOX_STEPS];
                out->retests = (int64_t)host_counters[C_RETESTS];
                out->descent_levels = (int64_t)host_counters[C_DESCENT];
                out->error_bits = (int64_t)host_counters[C_ERROR];
                out->spp_effective = (int)spp_eff;
                out->launches = times.launches;
                out->extend_launches = times.extend_launches;
                out->shadow_launches = times.shadow_launches;
                out->shadow_facet_tests = (int64_t)host_counters[C_SH_FACET_TESTS];
                out->shadow_box_steps = (int64_t)host_counters[C_SH_BOX_STEPS];
                out->shadow_retests = (int64_t)host_counters[C_SH_RETESTS];
                out->shadow_descent_levels = (int64_t)host_counters[C_SH_DESCENT];
                out->iterations = (int64_t)host_counters[C_ITERS];
                out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        if (stopped)
        {
                fail(NT_ESTOPPED, "render stopped");
        }
        if (host_counters[C_ERROR])
        {
                fail(NT_ETIMEOUT, "a bounded device loop ran out (error bits " + std::to_string(host_counters[C_ERROR]) + ")");
        }
}

template <int N>
struct NoallocF
{
        static void run(nt_scene* s, const nt_render_opts& o, double* acc, long long off, cudaStream_t st, void* scratch,
                        size_t bytes, nt_stats* out)
        {
                render_noalloc<N>(s, o, acc, off, st, scratch, bytes, out);
        }
};

template <int N>
void trace_closest(nt_scene* s, int mesh_index, const float* d_org, const float* d_dir, long long nrays, int retest,
                   int* d_facet, float* d_t, cudaStream_t st, unsigned long long* counters)
{
        MeshDev<N> M = mesh_dev<N>(s->meshes[mesh_index]);
        check_cuda(launch_trace_closest<N>(M, d_org, d_dir, nrays, retest, d_facet, d_t, counters, st), "trace_closest");
}

template <template <int> class F, typename... A>
void dispatch(int n, A&&... a)
{
        switch (n)
        {
        case 3:
                F<3>::run(a...);
                break;
        case 4:
                F<4>::run(a...);
                break;
        case 5:
                F<5>::run(a...);
                break;
        case 6:
                F<6>::run(a...);
                break;
        default:
                fail(NT_EINVAL, "n must be 3..6");
        }
}

template <int N>
struct BuildF
{
        static void run(nt_scene* s, unsigned threads, bool host_only, bool tree_on_gpu)
        {
                build_scene<N>(s, threads, host_only, tree_on_gpu);
        }
};
template <int N>
struct RenderF
{
        static void run(nt_scene* s, const nt_render_opts& o, nt_stats* st)
        {
                render<N>(s, o, st);
        }
};
template <int N>
struct PrepareF
{
        static void run(nt_scene* s, const nt_render_opts& o, std::unique_ptr<PassJob>* out)
        {
                *out = prepare_pass<N>(s, o);
        }
};
template <int N>
struct TargetF
{
        static void run(nt_scene* s, const nt_render_opts& o, nt_stats* st, const PassTarget* target)
        {
                render<N>(s, o, st, *target);
        }
};
template <int N>
struct AuxF
{
        static void run(nt_scene* s, float* normal, float* depth, cudaStream_t st)
        {
                DevScene<N> S;
                std::memcpy(&S, s->dev_scene.data(), sizeof(S));
                check_cuda(launch_aux<N>(S, s->pixel_count(), normal, depth, st), "aux");
        }
};
template <int N>
struct TraceF
{
        static void run(nt_scene* s, int mi, const float* o, const float* d, long long nr, int rt, int* f, float* t,
                        cudaStream_t st, unsigned long long* c)
        {
                trace_closest<N>(s, mi, o, d, nr, rt, f, t, st, c);
        }
};

void need_scene(nt_scene* s)
{
        if (!s)
        {
                fail(NT_EINVAL, "scene is NULL");
        }
}

void need_built(nt_scene* s)
{
        need_scene(s);
        if (!s->built)
        {
                fail(NT_ESTATE, s->built_host ? "scene was built for the host only" : "scene is not built");
        }
}

void need_inspectable(nt_scene* s)
{
        need_scene(s);
        if (!s->built && !s->built_host)
        {
                fail(NT_ESTATE, "scene is not built");
        }
}

std::vector<float> vec_copy(const float* p, size_t count, const char* what)
{
        if (!p)
        {
                fail(NT_EINVAL, std::string(what) + " is NULL");
        }
        std::vector<float> v(p, p + count);
        for (float x : v)
        {
                if (!std::isfinite(x))
                {
                        fail(NT_EINVAL, std::string(what) + " is not finite");
                }
        }
        return v;
}

nt_surface surface_or_default(const nt_surface* s)
{
        if (s)
        {
                return *s;
        }
        return nt_surface{{1, 1, 1}, 1, 0, {0, 0, 0}};
}
}

namespace ntrace
{
int report_error(int code, const std::string& message)
{
        g_error = message;
        return code;
}

int render_with_scratch(nt_scene* scene, const nt_render_opts* opts, double* d_accum, int64_t sample_offset,
                        cudaStream_t stream, void* scratch, size_t scratch_bytes, nt_stats* stats)
{
        return guarded([&]() {
                need_built(scene);
                if (!opts)
                {
                        fail(NT_EINVAL, "opts is NULL");
                }
                dispatch<NoallocF>(scene->n, scene, *opts, d_accum, (long long)sample_offset, stream ? stream : scene->stream,
                                   scratch, scratch_bytes, stats);
        });
}
}

// ------------------------------------------------------------------------------------------------
// C ABI

extern "C" {

const char* nt_last_error_message(void)
{
        return g_error.c_str();
}

int nt_effective_spp(int n, int samples_per_pixel)
{
        if (n < 3 || n > 6 || samples_per_pixel < 1)
        {
                return -1;
        }
        int k = one_dimension_size(n, samples_per_pixel);
        int p = 1;
        for (int i = 0; i < n - 1; ++i)
        {
                p *= k;
        }
        return p;
}

double nt_cosine_sphere_coefficient(int n)
{
        // pi/2 (n-1)(n-3).../((n-2)(n-4)...) for even n, (n-1)(n-3).../((n-2)(n-4)...) for odd n
        long double p = (n & 1) == 0 ? 0.5L : 1.0L;
        for (int i = n - 1; i > 1; i -= 2)
        {
                p *= i;
                if (i > 2)
                {
                        p /= (i - 1);
                }
        }
        if ((n & 1) == 0)
        {
                p *= 3.1415926535897932384626433832795028841971693993751L;
        }
        return (double)p;
}

int nt_scene_create(int n, nt_scene** out)
{
        return guarded([&]() {
                if (!out)
                {
                        fail(NT_EINVAL, "out is NULL");
                }
                if (n < 3 || n > 6)
                {
                        fail(NT_EINVAL, "n must be 3..6");
                }
                auto s = std::make_unique<nt_scene>();
                s->n = n;
                *out = s.release();
        });
}

int nt_scene_destroy(nt_scene* scene)
{
        return guarded([&]() { delete scene; });
}

int nt_scene_add_mesh(nt_scene* scene, const float* vertices, int64_t vertex_count, const int32_t* facets,
                      int64_t facet_count, const nt_surface* surface)
{
        return guarded([&]() {
                need_scene(scene);
                if (scene->meshes.size() >= (size_t)MAX_MESHES || scene->objects.size() >= (size_t)MAX_OBJECTS)
                {
                        fail(NT_EINVAL, "too many objects");
                }
                if (vertex_count < 1 || facet_count < 1 || !facets)
                {
                        fail(NT_EINVAL, "No facets found in mesh");
                }
                const int n = scene->n;
                MeshHost m;
                m.vertices = vec_copy(vertices, (size_t)vertex_count * n, "vertices");
                m.facets.assign(facets, facets + (size_t)facet_count * n);
                m.surface = surface_or_default(surface);
                scene->meshes.push_back(std::move(m));
                scene->objects.push_back({OBJ_MESH, (int)scene->meshes.size() - 1});
                scene->built = false;
        });
}

int nt_scene_set_mesh_normals(nt_scene* scene, int object, const float* normals, int64_t normal_count,
                              const int32_t* facet_normals)
{
        return guarded([&]() {
                need_scene(scene);
                if (object < 0 || object >= (int)scene->objects.size() || scene->objects[object].kind != OBJ_MESH)
                {
                        fail(NT_EINVAL, "object is not a mesh");
                }
                if (!normals || normal_count < 1)
                {
                        fail(NT_EINVAL, "no normals");
                }
                const int n = scene->n;
                MeshHost& m = scene->meshes[scene->objects[object].index];
                std::vector<float> nv = vec_copy(normals, (size_t)normal_count * n, "normals");
                std::vector<int32_t> fn = facet_normals ? std::vector<int32_t>(facet_normals, facet_normals + m.facets.size())
                                                        : m.facets;
                for (size_t f = 0; f < fn.size() / n; ++f)
                {
                        const bool none = fn[f * n] < 0;
                        for (int i = 0; i < n; ++i)
                        {
                                const int32_t x = fn[f * n + i];
                                if (none ? x != -1 : (x < 0 || x >= normal_count))
                                {
                                        fail(NT_EINVAL, "facet normal index out of range");
                                }
                        }
                }
                m.normals = std::move(nv);
                m.facet_normals = std::move(fn);
                m.ready = false;
                scene->built = false;
        });
}

int nt_scene_add_parallelotope(nt_scene* scene, const float* org, const float* edges, const nt_surface* surface)
{
        return guarded([&]() {
                need_scene(scene);
                if (scene->plts.size() >= (size_t)MAX_PLT || scene->objects.size() >= (size_t)MAX_OBJECTS)
                {
                        fail(NT_EINVAL, "too many objects");
                }
                const int n = scene->n;
                PltHost p;
                p.org = vec_copy(org, n, "org");
                p.edges = vec_copy(edges, (size_t)n * n, "edges");
                p.surface = surface_or_default(surface);
                scene->plts.push_back(std::move(p));
                scene->objects.push_back({OBJ_PLT, (int)scene->plts.size() - 1});
                scene->built = false;
        });
}

int nt_scene_add_hyperplane_parallelotope(nt_scene* scene, const float* org, const float* edges,
                                          const nt_surface* surface)
{
        return guarded([&]() {
                need_scene(scene);
                if (scene->hplts.size() >= (size_t)MAX_HPLT || scene->objects.size() >= (size_t)MAX_OBJECTS)
                {
                        fail(NT_EINVAL, "too many objects");
                }
                const int n = scene->n;
                HpltHost h;
                h.org = vec_copy(org, n, "org");
                h.edges = vec_copy(edges, (size_t)(n - 1) * n, "edges");
                h.surface = surface_or_default(surface);
                scene->hplts.push_back(std::move(h));
                scene->objects.push_back({OBJ_HPLT, (int)scene->hplts.size() - 1});
                scene->built = false;
        });
}

int nt_scene_add_point_light(nt_scene* scene, const float* location, const float* rgb, float unit_intensity_distance)
{
        return guarded([&]() {
                need_scene(scene);
                if (scene->lights.size() >= (size_t)MAX_LIGHTS)
                {
                        fail(NT_EINVAL, "too many light sources");
                }
                LightHost L;
                L.kind = 0;
                L.pos = vec_copy(location, scene->n, "location");
                std::vector<float> c = vec_copy(rgb, 3, "rgb");
                std::copy(c.begin(), c.end(), L.color);
                if (!(unit_intensity_distance > 0))
                {
                        fail(NT_EINVAL, "unit intensity distance must be positive");
                }
                L.unit = unit_intensity_distance;
                scene->lights.push_back(L);
                scene->built = false;
        });
}

int nt_scene_add_constant_light(nt_scene* scene, const float* location, const float* rgb)
{
        return guarded([&]() {
                need_scene(scene);
                if (scene->lights.size() >= (size_t)MAX_LIGHTS)
                {
                        fail(NT_EINVAL, "too many light sources");
                }
                LightHost L;
                L.kind = 1;
                L.pos = vec_copy(location, scene->n, "location");
                std::vector<float> c = vec_copy(rgb, 3, "rgb");
                std::copy(c.begin(), c.end(), L.color);
                L.unit = 1;
                scene->lights.push_back(L);
                scene->built = false;
        });
}

int nt_scene_set_projector(nt_scene* scene, int kind, const float* camera_org, const float* camera_dir,
                           const float* screen_axes, float param, const int32_t* screen_size)
{
        return guarded([&]() {
                need_scene(scene);
                if (kind < 0 || kind > 2)
                {
                        fail(NT_EINVAL, "unknown projector kind");
                }
                const int n = scene->n;
                if (!screen_size)
                {
                        fail(NT_EINVAL, "screen_size is NULL");
                }
                long long pix = 1;
                std::vector<int> sz(screen_size, screen_size + n - 1);
                for (int v : sz)
                {
                        if (v < 1 || v > 32767)
                        {
                                fail(NT_EINVAL, "screen size must be in [1, 32767]");
                        }
                        pix *= v;
                }
                if (pix > (1ll << 31))
                {
                        fail(NT_EINVAL, "screen has too many pixels");
                }
                scene->cam_org = vec_copy(camera_org, n, "camera_org");
                scene->cam_dir = vec_copy(camera_dir, n, "camera_dir");
                scene->axes = vec_copy(screen_axes, (size_t)(n - 1) * n, "screen_axes");
                scene->proj_kind = kind;
                scene->proj_param = param;
                scene->screen = sz;
                scene->has_projector = true;
                scene->built = false;
        });
}

int nt_scene_set_background(nt_scene* scene, const nt_surface* surface)
{
        return guarded([&]() {
                need_scene(scene);
                if (!surface)
                {
                        fail(NT_EINVAL, "surface is NULL");
                }
                scene->background = *surface;
                scene->built = false;
        });
}

int nt_scene_dimension(nt_scene* scene)
{
        return scene ? scene->n : -1;
}

int nt_scene_object_count(nt_scene* scene)
{
        return scene ? (int)scene->objects.size() : -1;
}

int nt_scene_clear_lights(nt_scene* scene)
{
        return guarded([&]() {
                need_scene(scene);
                scene->lights.clear();
                scene->built = false;
        });
}

int nt_scene_set_object_surface(nt_scene* scene, int object, const nt_surface* surface)
{
        return guarded([&]() {
                need_scene(scene);
                if (!surface || object < 0 || object >= (int)scene->objects.size())
                {
                        fail(NT_EINVAL, "bad object index or surface");
                }
                const ObjRef& o = scene->objects[object];
                if (o.kind == OBJ_MESH)
                {
                        scene->meshes[o.index].surface = *surface;
                }
                else if (o.kind == OBJ_PLT)
                {
                        scene->plts[o.index].surface = *surface;
                }
                else
                {
                        scene->hplts[o.index].surface = *surface;
                }
                scene->built = false;
        });
}

int nt_scene_build(nt_scene* scene, const nt_build_opts* opts)
{
        return guarded([&]() {
                need_scene(scene);
                unsigned threads = (opts && opts->threads > 0) ? (unsigned)opts->threads : hardware_threads();
                bool host_only = opts && opts->host_only;
                bool tree_on_gpu = opts && opts->tree_on_gpu;
                scene->leaf_records = opts ? opts->leaf_records : 0;
                scene->built = false;
                scene->built_host = false;
                // an upload staged before the build is of the old scene: a commit now is refused
                scene->upload_staged = false;
                if (scene->copy_stream)
                {
                        check_cuda(cudaStreamSynchronize(scene->copy_stream), "sync");
                }
                dispatch<BuildF>(scene->n, scene, threads, host_only, tree_on_gpu);
        });
}

int nt_scene_mesh_info(nt_scene* scene, int mesh_index, nt_mesh_info* info)
{
        return guarded([&]() {
                need_inspectable(scene);
                if (mesh_index < 0 || mesh_index >= (int)scene->meshes.size() || !info)
                {
                        fail(NT_EINVAL, "bad mesh index");
                }
                const MeshHost& m = scene->meshes[mesh_index];
                info->facet_count = (int64_t)(m.facets.size() / scene->n);
                info->node_count = (int64_t)(m.nodes.size() / 2);
                info->leaf_count = m.leaf_count;
                info->index_count = 0;
                for (size_t i = 0; i < m.nodes.size() / 2; ++i)
                {
                        if (m.nodes[2 * i + 1] >= 0)
                        {
                                info->index_count += m.nodes[2 * i + 1];
                        }
                }
                info->max_depth = tree_max_depth(scene->n);
                info->distance_from_facet = m.dist;
                info->degenerate_facets = m.degenerate;
                info->build_seconds = m.build_seconds;
                info->device_bytes =
                        (int64_t)(m.d_rec32.bytes + m.d_rec64.bytes + m.d_nodes.bytes + m.d_idx.bytes + m.d_leafrec.bytes);
        });
}

int nt_scene_tree_export(nt_scene* scene, int mesh_index, int32_t* nodes, int32_t* indices, float* level_sizes,
                         float* root_org)
{
        return guarded([&]() {
                need_inspectable(scene);
                if (mesh_index < 0 || mesh_index >= (int)scene->meshes.size())
                {
                        fail(NT_EINVAL, "bad mesh index");
                }
                const MeshHost& m = scene->meshes[mesh_index];
                if (nodes)
                {
                        std::memcpy(nodes, m.nodes.data(), m.nodes.size() * sizeof(int32_t));
                }
                if (indices)
                {
                        long long cnt = 0;
                        for (size_t i = 0; i < m.nodes.size() / 2; ++i)
                        {
                                if (m.nodes[2 * i + 1] >= 0)
                                {
                                        cnt += m.nodes[2 * i + 1];
                                }
                        }
                        std::memcpy(indices, m.leaf_idx.data(), (size_t)cnt * sizeof(int32_t));
                }
                if (level_sizes)
                {
                        std::memcpy(level_sizes, m.level_sizes.data(), m.level_sizes.size() * sizeof(float));
                }
                if (root_org)
                {
                        std::memcpy(root_org, m.root_org.data(), m.root_org.size() * sizeof(float));
                }
        });
}

int nt_scene_upload(nt_scene* scene, int64_t* bytes)
{
        return guarded([&]() {
                need_built(scene);
                int64_t total = 0;
                for (auto& m : scene->meshes)
                {
                        const char* p = static_cast<const char*>(m.pinned);
                        DevBuf* bufs[4] = {&m.d_rec32, &m.d_rec64, &m.d_nodes, &m.d_idx};
                        for (DevBuf* b : bufs)
                        {
                                if (b->bytes)
                                {
                                        check_cuda(cudaMemcpyAsync(b->p, p, b->bytes, cudaMemcpyHostToDevice, scene->stream),
                                                   "upload");
                                }
                                p += b->bytes;
                                total += (int64_t)b->bytes;
                        }
                        gather_leaf_records(m, scene->n, scene->stream, scene->leaf_records);
                }
                check_cuda(cudaStreamSynchronize(scene->stream), "upload sync");
                if (bytes)
                {
                        *bytes = total;
                }
        });
}

int nt_scene_upload_begin(nt_scene* scene, int64_t* bytes)
{
        return guarded([&]() {
                need_built(scene);
                if (!scene->copy_stream)
                {
                        check_cuda(cudaStreamCreateWithFlags(&scene->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
                        check_cuda(cudaEventCreateWithFlags(&scene->staged, cudaEventDisableTiming), "cudaEventCreate");
                        check_cuda(cudaEventCreateWithFlags(&scene->consumed, cudaEventDisableTiming), "cudaEventCreate");
                }
                // the previous commit's device copies still read the staging buffers
                if (scene->consumed_recorded)
                {
                        check_cuda(cudaStreamWaitEvent(scene->copy_stream, scene->consumed, 0), "wait");
                }
                int64_t total = 0;
                for (auto& m : scene->meshes)
                {
                        const size_t b = m.d_rec32.bytes + m.d_rec64.bytes + m.d_nodes.bytes + m.d_idx.bytes;
                        if (m.d_stage.bytes != b)
                        {
                                // a resize frees the old buffer: nothing may still use it
                                check_cuda(cudaStreamSynchronize(scene->copy_stream), "sync");
                                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
                                m.d_stage.alloc(b);
                        }
                        if (b)
                        {
                                check_cuda(cudaMemcpyAsync(m.d_stage.p, m.pinned, b, cudaMemcpyHostToDevice, scene->copy_stream),
                                           "upload");
                        }
                        total += (int64_t)b;
                }
                check_cuda(cudaEventRecord(scene->staged, scene->copy_stream), "record");
                scene->upload_staged = true;
                if (bytes)
                {
                        *bytes = total;
                }
        });
}

int nt_scene_upload_commit(nt_scene* scene)
{
        return guarded([&]() {
                need_built(scene);
                if (!scene->upload_staged)
                {
                        fail(NT_ESTATE, "no staged upload (nt_scene_upload_begin)");
                }
                check_cuda(cudaStreamWaitEvent(scene->stream, scene->staged, 0), "wait");
                for (auto& m : scene->meshes)
                {
                        const char* p = static_cast<const char*>(m.d_stage.p);
                        DevBuf* bufs[4] = {&m.d_rec32, &m.d_rec64, &m.d_nodes, &m.d_idx};
                        size_t off = 0;
                        for (DevBuf* b : bufs)
                        {
                                if (off + b->bytes > m.d_stage.bytes)
                                {
                                        fail(NT_ESTATE, "the scene changed since nt_scene_upload_begin");
                                }
                                if (b->bytes)
                                {
                                        check_cuda(cudaMemcpyAsync(b->p, p + off, b->bytes, cudaMemcpyDeviceToDevice, scene->stream),
                                                   "commit");
                                }
                                off += b->bytes;
                        }
                }
                check_cuda(cudaEventRecord(scene->consumed, scene->stream), "record");
                // the leaf-ordered records are made from the live arrays, after the staging buffer is free
                for (auto& m : scene->meshes)
                {
                        gather_leaf_records(m, scene->n, scene->stream, scene->leaf_records);
                }
                scene->consumed_recorded = true;
                scene->upload_staged = false;
        });
}

void* nt_scene_stream(nt_scene* scene)
{
        return scene ? (void*)scene->stream : nullptr;
}

int64_t nt_scene_pixel_count(nt_scene* scene)
{
        if (!scene || !scene->has_projector)
        {
                return -1;
        }
        return scene->pixel_count();
}

int nt_render(nt_scene* scene, const nt_render_opts* opts, nt_stats* stats)
{
        return guarded([&]() {
                need_built(scene);
                if (!opts)
                {
                        fail(NT_EINVAL, "opts is NULL");
                }
                dispatch<RenderF>(scene->n, scene, *opts, stats);
        });
}

int nt_render_pixels(nt_scene* scene, const nt_render_opts* opts, const int64_t* pixels, int64_t count,
                     float* rgb_mean, nt_stats* stats)
{
        return guarded([&]() {
                need_built(scene);
                if (!opts || !pixels || !rgb_mean || count < 1)
                {
                        fail(NT_EINVAL, "bad pixel-list arguments");
                }
                const long long npix = scene->pixel_count();
                for (int64_t i = 0; i < count; ++i)
                {
                        if (pixels[i] < 0 || pixels[i] >= npix)
                        {
                                fail(NT_EINVAL, "pixel index " + std::to_string(pixels[i]) + " out of range");
                        }
                }
                const int spp = nt_effective_spp(scene->n, opts->samples_per_pixel);
                if (spp < 1)
                {
                        fail(NT_EINVAL, "Stratified jittered sample count is not a positive integer");
                }
                const size_t list_bytes = (size_t)count * sizeof(long long);
                const size_t sum_bytes = (size_t)count * 3 * sizeof(double);
                if (scene->list_buf.bytes < list_bytes + sum_bytes)
                {
                        scene->list_buf.alloc(list_bytes + sum_bytes);
                }
                if (scene->mean_buf.bytes < (size_t)count * 3 * sizeof(float))
                {
                        scene->mean_buf.alloc((size_t)count * 3 * sizeof(float));
                }
                long long* d_list = scene->list_buf.as<long long>();
                double* d_sums = reinterpret_cast<double*>(scene->list_buf.as<char>() + list_bytes);
                check_cuda(cudaMemcpyAsync(d_list, pixels, list_bytes, cudaMemcpyHostToDevice, scene->stream), "copy pixels");
                check_cuda(cudaMemsetAsync(d_sums, 0, sum_bytes, scene->stream), "memset");
                PassTarget target;
                target.list = d_list;
                target.list_count = count;
                target.list_accum = d_sums;
                target.first_sample = std::max<long long>(opts->sample_offset, 0);
                nt_stats one{};
                dispatch<TargetF>(scene->n, scene, *opts, &one, &target);
                check_cuda(launch_mean(count * 3, d_sums, spp, scene->mean_buf.as<float>(), scene->stream), "mean");
                check_cuda(cudaMemcpyAsync(rgb_mean, scene->mean_buf.p, (size_t)count * 3 * sizeof(float),
                                           cudaMemcpyDeviceToHost, scene->stream),
                           "copy mean");
                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
                if (stats)
                {
                        *stats = one;
                }
        });
}

int nt_render_aux(nt_scene* scene, float* d_normal, float* d_depth, void* stream)
{
        return guarded([&]() {
                need_built(scene);
                if (!d_normal || !d_depth)
                {
                        fail(NT_EINVAL, "null output array");
                }
                cudaStream_t st = stream ? (cudaStream_t)stream : scene->stream;
                dispatch<AuxF>(scene->n, scene, d_normal, d_depth, st);
                check_cuda(cudaStreamSynchronize(st), "aux sync");
        });
}

int nt_render_moments(nt_scene* scene, const nt_render_opts* opts, int64_t sample_offset, float* d_mean, float* d_var,
                      nt_stats* stats)
{
        return guarded([&]() {
                need_built(scene);
                if (!opts || sample_offset < 0 || !d_mean || !d_var)
                {
                        fail(NT_EINVAL, "bad moments arguments");
                }
                const long long npix = scene->pixel_count();
                const int spp = nt_effective_spp(scene->n, opts->samples_per_pixel);
                if (spp < 1)
                {
                        fail(NT_EINVAL, "Stratified jittered sample count is not a positive integer");
                }
                const size_t bytes = (size_t)npix * spp * 3 * sizeof(double);
                if (scene->moments.bytes < bytes)
                {
                        scene->moments.alloc(bytes);
                }
                check_cuda(cudaMemsetAsync(scene->moments.p, 0, bytes, scene->stream), "memset");
                PassTarget target;
                target.moments = scene->moments.as<double>();
                target.first_sample = sample_offset;
                nt_stats one{};
                dispatch<TargetF>(scene->n, scene, *opts, &one, &target);
                check_cuda(launch_moments_reduce(npix, spp, scene->moments.as<double>(), d_mean, d_var, scene->stream),
                           "moments");
                check_cuda(cudaStreamSynchronize(scene->stream), "moments sync");
                if (stats)
                {
                        *stats = one;
                }
        });
}

int nt_render_batch(nt_scene* const* scenes, int count, const nt_render_opts* opts, nt_stats* stats)
{
        cudaStream_t master = nullptr;
        std::vector<cudaEvent_t> events;
        cudaGraphExec_t exec = nullptr;
        auto cleanup = [&]() {
                if (exec)
                {
                        cudaGraphExecDestroy(exec);
                }
                for (cudaEvent_t e : events)
                {
                        cudaEventDestroy(e);
                }
                if (master)
                {
                        cudaStreamDestroy(master);
                }
        };
        int rc = guarded([&]() {
                if (count < 1 || !scenes || !opts)
                {
                        fail(NT_EINVAL, "bad batch arguments");
                }
                for (int i = 0; i < count; ++i)
                {
                        need_built(scenes[i]);
                        for (int j = 0; j < i; ++j)
                        {
                                if (scenes[j] == scenes[i])
                                {
                                        fail(NT_EINVAL, "a scene appears twice in the batch");
                                }
                        }
                }
                std::vector<std::unique_ptr<PassJob>> jobs(count);
                for (int i = 0; i < count; ++i)
                {
                        dispatch<PrepareF>(scenes[i]->n, scenes[i], opts[i], &jobs[i]);
                }
                for (int i = 0; i < count; ++i)
                {
                        check_cuda(cudaStreamSynchronize(scenes[i]->stream), "batch sync");
                }
                // one graph: fork from a master stream to every scene's stream, `per` iterations of
                // each pass, its counters to the host, join back
                const int batch = opts[0].graph_iterations > 0 ? opts[0].graph_iterations : 4;
                const int per = batch + (batch & 1);
                check_cuda(cudaStreamCreateWithFlags(&master, cudaStreamNonBlocking), "cudaStreamCreate");
                events.resize(count + 1);
                for (cudaEvent_t& e : events)
                {
                        check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
                }
                check_cuda(cudaStreamBeginCapture(master, cudaStreamCaptureModeThreadLocal), "capture");
                cudaGraph_t graph = nullptr;
                cudaError_t e = cudaEventRecord(events[count], master);
                for (int i = 0; i < count && e == cudaSuccess; ++i)
                {
                        nt_scene* s = scenes[i];
                        e = cudaStreamWaitEvent(s->stream, events[count], 0);
                        for (int k = 0; k < per && e == cudaSuccess; ++k)
                        {
                                jobs[i]->enqueue(k & 1, s->stream);
                        }
                        if (e == cudaSuccess)
                        {
                                e = cudaMemcpyAsync(s->host_counters, s->counters.p, C_COUNT * sizeof(unsigned long long),
                                                    cudaMemcpyDeviceToHost, s->stream);
                        }
                        if (e == cudaSuccess)
                        {
                                e = cudaEventRecord(events[i], s->stream);
                        }
                        if (e == cudaSuccess)
                        {
                                e = cudaStreamWaitEvent(master, events[i], 0);
                        }
                }
                cudaError_t e2 = cudaStreamEndCapture(master, &graph);
                check_cuda(e != cudaSuccess ? e : e2, "batch capture");
                e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                check_cuda(e, "batch graph");
                for (int i = 0; i < count; ++i)
                {
                        for (int c = C_Q_ACTIVE; c < C_COUNT; ++c)
                        {
                                scenes[i]->host_counters[c] = 0;
                        }
                }
                const volatile int* stop = opts[0].stop;
                while (true)
                {
                        if (stop && *stop)
                        {
                                break;
                        }
                        check_cuda(cudaGraphLaunch(exec, master), "batch launch");
                        check_cuda(cudaStreamSynchronize(master), "batch sync");
                        bool all = true, err = false;
                        for (int i = 0; i < count; ++i)
                        {
                                all &= scenes[i]->host_counters[C_DONE] != 0;
                                err |= scenes[i]->host_counters[C_ERROR] != 0;
                                jobs[i]->times.launches +=
                                        (long long)per * Wavefront<3>::iteration_launches(jobs[i]->smooth, jobs[i]->one_mesh);
                                jobs[i]->times.extend_launches += per;
                                jobs[i]->times.shadow_launches += per;
                        }
                        if (all || err)
                        {
                                break;
                        }
                }
                for (int i = 0; i < count; ++i)
                {
                        finish_pass(*jobs[i], opts[i], stats ? stats + i : nullptr, false);
                }
        });
        cleanup();
        return rc;
}

int nt_autotune(nt_scene* scene, const nt_render_opts* base, nt_render_opts* tuned, double* best_ms)
{
        return guarded([&]() {
                need_built(scene);
                if (!base || !tuned)
                {
                        fail(NT_EINVAL, "null options");
                }
                const long long total = scene->pixel_count() * (long long)nt_effective_spp(scene->n, base->samples_per_pixel);
                std::vector<long long> pools;
                for (long long q = 1ll << 20; q <= (1ll << 25); q <<= 1)
                {
                        if (q < 2 * total || pools.empty())
                        {
                                pools.push_back(std::min(q, std::max<long long>(256, total)));
                        }
                }
                const int iters[] = {2, 4, 8, 16};
                nt_render_opts best = *base;
                double best_t = 1e300;
                for (long long q : pools)
                {
                        for (int it : iters)
                        {
                                nt_render_opts o = *base;
                                o.pool_paths = q;
                                o.graph_iterations = it;
                                o.timing = 0;
                                o.stop = nullptr;
                                // one warm pass, one timed
                                for (int rep = 0; rep < 2; ++rep)
                                {
                                        auto t0 = std::chrono::steady_clock::now();
                                        dispatch<RenderF>(scene->n, scene, o, (nt_stats*)nullptr);
                                        const double ms =
                                                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                                        if (rep == 1 && ms < best_t)
                                        {
                                                best_t = ms;
                                                best = o;
                                        }
                                }
                        }
                }
                // then the walk kernels' variant and small-leaf threshold at the best pool and iterations
                const nt_render_opts at = best;
                for (int v = 0; v < 7; ++v)
                {
                        nt_render_opts o = at;
                        static const int chunks[7] = {1, 32, 64, 128, 1, 1, 1};
                        static const int smalls[7] = {2, 2, 2, 2, -1, 1, 4};
                        o.walk_chunk = chunks[v];
                        o.walk_small_leaf = smalls[v];
                        o.timing = 0;
                        o.stop = nullptr;
                        for (int rep = 0; rep < 2; ++rep)
                        {
                                auto t0 = std::chrono::steady_clock::now();
                                dispatch<RenderF>(scene->n, scene, o, (nt_stats*)nullptr);
                                const double ms =
                                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                                if (rep == 1 && ms < best_t)
                                {
                                        best_t = ms;
                                        best = o;
                                }
                        }
                }
                check_cuda(cudaMemsetAsync(scene->accum.p, 0, scene->accum.bytes, scene->stream), "memset");
                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
                scene->samples_done = 0;
                best.timing = base->timing;
                best.stop = base->stop;
                *tuned = best;
                if (best_ms)
                {
                        *best_ms = best_t;
                }
        });
}

int nt_accum_read_srgb_slice(nt_scene* scene, const int32_t* slice, uint32_t* out, int device_out)
{
        return guarded([&]() {
                need_built(scene);
                if (!out || (scene->n > 3 && !slice))
                {
                        fail(NT_EINVAL, "null argument");
                }
                const int width = scene->screen[0];
                const int height = scene->screen[1];
                long long base = 0;
                long long stride = 1;
                for (int j = 0; j < scene->n - 1; ++j)
                {
                        if (j >= 2)
                        {
                                const int v = slice[j - 2];
                                if (v < 0 || v >= scene->screen[j])
                                {
                                        fail(NT_EINVAL, "slice position out of the screen");
                                }
                                base += (long long)v * stride;
                        }
                        stride *= scene->screen[j];
                }
                const size_t bytes = (size_t)width * height * sizeof(uint32_t);
                DevBuf tmp;
                uint32_t* dst = out;
                if (!device_out)
                {
                        tmp.alloc(bytes);
                        dst = tmp.as<uint32_t>();
                }
                check_cuda(launch_srgb_slice(scene->accum.as<double>(), scene->samples_done, base, width, height, width, dst,
                                             scene->stream),
                           "srgb slice");
                if (!device_out)
                {
                        check_cuda(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, scene->stream), "copy");
                }
                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
        });
}

int nt_accum_clear(nt_scene* scene)
{
        return guarded([&]() {
                need_built(scene);
                check_cuda(cudaMemsetAsync(scene->accum.p, 0, scene->accum.bytes, scene->stream), "memset");
                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
                scene->samples_done = 0;
        });
}

int nt_accum_read(nt_scene* scene, float* rgb_mean, int64_t* samples_per_pixel)
{
        return guarded([&]() {
                need_built(scene);
                const long long npix = scene->pixel_count();
                if (samples_per_pixel)
                {
                        *samples_per_pixel = scene->samples_done;
                }
                if (!rgb_mean)
                {
                        return;
                }
                // the mean is formed on the device (the same double product, rounded once), so half the
                // bytes cross to the host, straight into the caller's array
                const size_t bytes = (size_t)npix * 3 * sizeof(float);
                if (scene->mean_buf.bytes < bytes)
                {
                        scene->mean_buf.alloc(bytes);
                }
                check_cuda(launch_mean(npix * 3, scene->accum.as<double>(), scene->samples_done, scene->mean_buf.as<float>(),
                                       scene->stream),
                           "mean");
                check_cuda(cudaMemcpyAsync(rgb_mean, scene->mean_buf.p, bytes, cudaMemcpyDeviceToHost, scene->stream),
                           "read accumulator");
                check_cuda(cudaStreamSynchronize(scene->stream), "sync");
        });
}

int nt_trace_closest_device(nt_scene* scene, int mesh_index, const float* d_org, const float* d_dir, int64_t ray_count,
                            int retest, int32_t* d_facet, float* d_t, void* stream)
{
        return guarded([&]() {
                need_built(scene);
                if (mesh_index < 0 || mesh_index >= (int)scene->meshes.size())
                {
                        fail(NT_EINVAL, "bad mesh index");
                }
                if (ray_count < 0)
                {
                        fail(NT_EINVAL, "negative ray count");
                }
                cudaStream_t st = stream ? (cudaStream_t)stream : scene->stream;
                dispatch<TraceF>(scene->n, scene, mesh_index, d_org, d_dir, (long long)ray_count, retest, (int*)d_facet, d_t,
                                 st, (unsigned long long*)nullptr);
        });
}

int nt_trace_closest(nt_scene* scene, int mesh_index, const float* org, const float* dir, int64_t ray_count, int retest,
                     int32_t* facet, float* t, nt_stats* stats)
{
        return guarded([&]() {
                need_built(scene);
                if (mesh_index < 0 || mesh_index >= (int)scene->meshes.size())
                {
                        fail(NT_EINVAL, "bad mesh index");
                }
                if (ray_count < 0 || (ray_count > 0 && (!org || !dir || !facet || !t)))
                {
                        fail(NT_EINVAL, "bad ray arrays");
                }
                auto t0 = std::chrono::steady_clock::now();
                const int n = scene->n;
                if (ray_count == 0)
                {
                        return;
                }
                DevBuf d_org, d_dir, d_facet, d_t;
                size_t vb = (size_t)ray_count * n * sizeof(float);
                d_org.alloc(vb);
                d_dir.alloc(vb);
                d_facet.alloc((size_t)ray_count * sizeof(int32_t));
                d_t.alloc((size_t)ray_count * sizeof(float));
                cudaStream_t st = scene->stream;
                check_cuda(cudaMemcpyAsync(d_org.p, org, vb, cudaMemcpyHostToDevice, st), "copy org");
                check_cuda(cudaMemcpyAsync(d_dir.p, dir, vb, cudaMemcpyHostToDevice, st), "copy dir");
                check_cuda(cudaMemsetAsync(scene->counters.p, 0, scene->counters.bytes, st), "memset counters");
                dispatch<TraceF>(n, scene, mesh_index, d_org.as<float>(), d_dir.as<float>(), (long long)ray_count, retest,
                                 d_facet.as<int>(), d_t.as<float>(), st, scene->counters.as<unsigned long long>());
                check_cuda(cudaMemcpyAsync(facet, d_facet.p, d_facet.bytes, cudaMemcpyDeviceToHost, st), "copy facet");
                check_cuda(cudaMemcpyAsync(t, d_t.p, d_t.bytes, cudaMemcpyDeviceToHost, st), "copy t");
                check_cuda(cudaMemcpyAsync(scene->host_counters, scene->counters.p, C_COUNT * sizeof(unsigned long long),
                                           cudaMemcpyDeviceToHost, st),
                           "counters");
                check_cuda(cudaStreamSynchronize(st), "trace sync");
                if (stats)
                {
                        std::memset(stats, 0, sizeof(*stats));
                        stats->rays = ray_count;
                        stats->facet_tests = (int64_t)scene->host_counters[C_FACET_TESTS];
                        stats->box_steps = (int64_t)scene->host_counters[C_BOX_STEPS];
                        stats->retests = (int64_t)scene->host_counters[C_RETESTS];
                        stats->descent_levels = (int64_t)scene->host_counters[C_DESCENT];
                        stats->error_bits = (int64_t)scene->host_counters[C_ERROR];
                        stats->launches = 1;
                        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                }
                if (scene->host_counters[C_ERROR])
                {
                        fail(NT_ETIMEOUT, "a tree walk exceeded its step bound");
                }
        });
}
}
