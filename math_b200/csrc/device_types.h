// Device-side scene description shared by the host packer and the sm_100a kernels.
// Everything a kernel needs arrives as one by-value parameter (DevScene<N>, < 4 KB) plus device
// pointers; per-N templates keep the per-ray state in registers.
#pragma once

#include <cstdint>
#include <vector_types.h>

namespace ntrace
{
constexpr int MAX_MESHES = 2;
constexpr int MAX_PLT = 4;      // general n-parallelotopes
constexpr int MAX_HPLT = 2;     // hyperplane (n-1)-parallelotopes
constexpr int MAX_OBJECTS = 8;
constexpr int MAX_LIGHTS = 4;
constexpr int MAX_LEVELS = 11;  // tree depth 10 (n = 3) plus the root

enum ObjectKind : int
{
        OBJ_MESH = 0,
        OBJ_PLT = 1,
        OBJ_HPLT = 2
};

// FP32 facet record, float4-aligned:
//   [normal (N)] [d0 = dot(normal, v0)] [B = max_i |n_i|_1] [D = max_i |d_i|] [(n_i (N), d_i) x (N-1)]
// planes from the double-precision Gaussian elimination, rounded to float.  B = +inf marks a
// near-degenerate facet whose every test is decided in FP64.
template <int N>
struct Rec32
{
        static constexpr int RAW = N * N + N + 2;
        static constexpr int FLOATS = (RAW + 3) / 4 * 4;
        static constexpr int F4 = FLOATS / 4;
        static constexpr int OFF_D0 = N;
        static constexpr int OFF_B = N + 1;
        static constexpr int OFF_D = N + 2;
        static constexpr int OFF_PLANES = N + 3;
};

// FP64 facet record in the reference's own formulation (used by the FP64 re-test):
//   [v0 (N)] [normal (N)] [(n_i (N), d_i) x (N-1)]  (hyperplane_geometry.h:83-115,181-204)
template <int N>
struct Rec64
{
        static constexpr int RAW = N * N + 2 * N - 1;
        static constexpr int DOUBLES = (RAW + 1) / 2 * 2;
        static constexpr int OFF_NORMAL = N;
        static constexpr int OFF_PLANES = 2 * N;
};

template <int N>
struct MeshDev
{
        const float4* rec32;
        const double* rec64;
        const int2* nodes;     // internal: {first_child, -1}; leaf: {index offset, count}
        const int* leaf_idx;
        const float4* leaf_rec32;  // the leaves' FP32 records in leaf-list order (rec32 gathered through
                                   // leaf_idx): a leaf's records are read without its index list first;
                                   // null when the copy did not fit the memory budget (leaf_record)
        // vertex normals (null without them): normals (count x N), per-facet normal indices (N per
        // facet) and per-facet NormalType: 0 None, 1 Use, 2 Reverse with bit 2 + i set when vertex i's
        // normal is reversed (mesh_hyperplane_simplex.cpp:96-143)
        const float* vnormals;
        const int* fnormals;
        const int* ntype;
        int nfacets;
        int levels;
        float root_org[N];
        float root_d1[N];
        float size[MAX_LEVELS][N];  // box size at depth k (root k = 0)
        float dist;                 // distance_from_facet of the tree (tree.h:419)
};

template <int N>
struct PltDev
{
        float n[N][N];  // outward plane normals
        float d1[N];
        float d2[N];
};

template <int N>
struct HpltDev
{
        float normal[N];
        float org[N];
        float planes[N - 1][N + 1];
};

struct ObjDev
{
        int kind;
        int index;
        float color[3];
        float diffuse;
        int light_source;
        float light_color[3];
};

struct LightDev
{
        int kind;  // 0 point, 1 constant
        float pos[6];
        float color[3];
        float coef;  // unit_intensity_distance^(N-1)
};

template <int N>
struct ProjDev
{
        int kind;  // 0 parallel, 1 perspective, 2 spherical
        float cam_org[N];
        float cam_dir[N];
        float axes[N - 1][N];
        float screen_org[N - 1];
        int screen[N - 1];
        float square_radius;
};

template <int N>
struct DevScene
{
        int nobj;
        ObjDev obj[MAX_OBJECTS];
        int nmesh;
        MeshDev<N> mesh[MAX_MESHES];
        int nplt;
        PltDev<N> plt[MAX_PLT];
        int nhplt;
        HpltDev<N> hplt[MAX_HPLT];
        int nlights;
        LightDev lights[MAX_LIGHTS];
        ProjDev<N> proj;
        float bg_color[3];
        float bg_light_color[3];
        int bg_light;
        float ray_offset;
        float diffuse_coef;  // cosine_sphere_coefficient(N)
        int smooth_normal;
        int max_depth;
        int retest;          // 1: FP64 re-test of uncertain facet tests
        int walk_rounds;     // walk kernels: rounds of 32 pooled facet tests staged per warp chunk (1, 2
                             // or 4; 0: the default for N); host-side choice of the kernel variant
        int walk_small;      // walk kernels: leaves of at most this many facets (in every lane of a warp)
                             // are tested per lane instead of pooled across the warp
};

// Render-pass constants.
struct PassDev
{
        uint32_t key0, key1;      // Philox key (seed)
        int spp_eff;              // k^(N-1)
        int k1d;                  // strata per screen axis
        float recip_k;            // 1/k
        long long npix;
        long long sample_offset;  // first sample index of this pass (progressive passes)
        long long path_begin;     // first path of this launch window
        long long path_end;
        int moments;              // 1: radiance is summed per path (index pixel * spp_eff + sample of
                                  // the pass) instead of per pixel; the path queues then carry that
                                  // index in place of the pixel
        const long long* list;    // non-null: the pass paints these pixels (linear indices) only; path g
                                  // is sample g % spp_eff of list entry g / spp_eff, and the queues carry
                                  // the entry (the accumulator has one slot per entry)
};

// Device-wide counters (one int64 each).
enum Counter : int
{
        C_ACTIVE_OUT = 0,
        C_SHADOW = 1,
        C_ERROR = 2,
        C_RAYS = 3,
        C_FACET_TESTS = 4,
        C_BOX_STEPS = 5,
        C_RETESTS = 6,
        C_SHADOW_RAYS = 7,
        C_DESCENT = 8,
        // the shadow kernel's own walk counters (C_FACET_TESTS.. above hold the extension kernel's)
        C_SH_FACET_TESTS = 9,
        C_SH_BOX_STEPS = 10,
        C_SH_DESCENT = 11,
        C_SH_RETESTS = 12,
        // work cursors of the persistent extension and shadow kernels
        C_WORK_EXT = 13,
        C_WORK_SH = 14,
        C_SMOOTH = 15,     // entries of the smooth-normal shadow queue
        // wavefront control, kept on the device so that iterations need no host round trip
        C_Q_ACTIVE = 16,   // paths in the current queue
        C_Q_NEXT = 17,     // next fresh path of the pass (relative to PassDev::path_begin)
        C_Q_FRESH = 18,    // fresh paths generated by this iteration
        C_Q_BASE = 19,     // queue slot of the first fresh path
        C_DONE = 20,       // 1 once every path of the pass has finished
        C_ITERS = 21,      // iterations that had work
        // one-mesh scenes: extension rays that need the tree walk, compacted by k_plan_extend (the
        // shadow rays that need it are the shadow queue itself, C_SHADOW)
        C_WALK_EXT = 22,
        C_COUNT = 23
};

enum ErrorBits : int
{
        ERR_WALK_LIMIT = 1,      // a tree walk exceeded its step bound
        ERR_SAMPLING_LIMIT = 2,  // a rejection sampler exceeded its attempt bound
        ERR_QUEUE_OVERFLOW = 4
};
}
