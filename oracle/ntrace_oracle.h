/*
 * ntrace oracle: a plain-C restatement of the reference n-space path tracer (templeblock/math,
 * src/painter), used ONLY as a checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg.  The product never links, loads or calls it.
 *
 * Every routine follows a reference function, cited at its definition in ntrace_oracle_core.inc.
 * The core is compiled twice: once in double ("_f64", the FP64 oracle that mirrors Mesh<N,double>
 * and paint<N,double>) and once in float ("_f32", mirroring Mesh<N,float> / paint<N,float>).
 * Arithmetic follows the reference's operation order (dot products as an fma chain,
 * src/com/vec.h:259-266; normalisation as a/sqrt(dot(a,a)), src/com/vec.h:281-290) and the file is
 * compiled with -ffp-contract=off.
 *
 * The one deliberate difference from the reference is the random-number source: the reference seeds
 * an mt19937_64 per thread from the OS (src/painter/painter.cpp:460), so its images are not
 * reproducible.  The oracle instead draws from the same counter-based Philox4x32-10 stream as the
 * product (keyed by seed, counter = path id, stream, draw), so the oracle and the GPU trace the same
 * paths.  Pinning: the closest-hit results of ort_mesh_trace are checked bit-for-bit against the
 * compiled reference (oracle/_ref) and against committed golden fixtures; radiance is checked against
 * the compiled reference statistically.
 */
#ifndef NTRACE_ORACLE_H
#define NTRACE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORT_NMAX 6

/* Same layout as the bridge's refb_scene so that one Python description feeds both checkers. */
typedef struct ort_scene
{
        int n;
        int dbl;
        const float* verts;
        long nverts;
        const int* facets;
        long nfacets;
        float mesh_color[3];
        float mesh_diffuse;
        int has_floor;
        float floor_org[6];
        float floor_edges[36];
        float floor_color[3];
        float floor_diffuse;
        int light_kind;
        float light_pos[6];
        float light_color[3];
        float light_unit_distance;
        int projector_kind;
        float cam_org[6];
        float cam_dir[6];
        float screen_axes[30];
        float proj_param;
        int screen[5];
        float bg_color[3];
        float bg_light_color[3];
        int bg_is_light;
        int smooth_normal;
        int tree_threads;
        /* optional vertex normals of the mesh (nnormals == 0: none); facet_normals NULL: vertex indices */
        const float* normals;
        long nnormals;
        const int* facet_normals;
        /* optional second mesh (nfacets2 == 0: none), after the first in object order */
        const float* verts2;
        long nverts2;
        const int* facets2;
        long nfacets2;
        float mesh2_color[3];
        float mesh2_diffuse;
        /* optional (n-1)-parallelotope in a hyperplane (has_hplt == 0: none), last in object order */
        int has_hplt;
        float hplt_org[6];
        float hplt_edges[30];
        float hplt_color[3];
        float hplt_diffuse;
} ort_scene;

typedef struct ort_stats
{
        long long paths;           /* camera samples traced */
        long long rays;            /* object-level intersection calls, counted as the reference does */
        long long facet_tests;     /* ray-simplex tests */
        long long box_steps;       /* leaves visited by tree walks */
        long long descent_levels;  /* node levels visited by root-to-leaf descents */
        long long shadow_rays;     /* shadow rays cast */
        double seconds;
} ort_stats;

/* Mesh with its 2^N-tree (the reference's Mesh<N,T>).  dbl selects the FP64 or FP32 core. */
void* ort_mesh_build(int n, int dbl, const float* verts, long nverts, const int* facets, long nfacets, char* err,
                     int errlen);
void ort_mesh_destroy(void* mesh);

/* Closest hit per ray: facet (-1 = miss) and distance, as intersect_approximate + intersect_precise. */
int ort_mesh_trace(void* mesh, const float* org, const float* dir, long nrays, int* facet_out, double* t_out,
                   ort_stats* stats);

/* Tree export: boxes in breadth-first order, children of a box contiguous.
 * info: box_count, index_count, max_depth, distance_from_facet. */
int ort_mesh_tree_info(void* mesh, long* box_count, long* index_count, double* distance_from_facet);
int ort_mesh_tree_export(void* mesh, double* org, double* size, int* first_child, int* depth, long* index_offset,
                         int* indices);

/* Per-facet setup export (reference formulation): normal (n), barycentric planes ((n-1) x (n+1)). */
int ort_mesh_facet_export(void* mesh, double* normal, double* planes);

/* Path tracing (paint<N,T>) with the Philox stream.  pixels == NULL: whole screen, rgb_out dense
 * (x0 fastest); otherwise the listed pixels.  sample_offset shifts the sample index (progressive
 * passes): sample s of pixel p (linear index, x0 fastest) uses
 * path id = (sample_offset + s) * pixel_count + p. */
int ort_paint(const ort_scene* scene, int spp, int max_depth, uint64_t seed, int threads, const int* pixels,
              long npix, long long sample_offset, float* rgb_out, ort_stats* stats, char* err, int errlen);

/* Effective samples per pixel: ceil-or-floor stratification of spp over n-1 screen dimensions. */
int ort_effective_spp(int n, int spp);

/* Philox4x32-10 block (test hook). */
void ort_philox(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4]);

/* cosine_sphere_coefficient(n) (test hook). */
double ort_cosine_sphere_coefficient(int n);

/* One cosine-weighted hemisphere direction for unit normal (test hook, FP64 core). */
int ort_cosine_hemisphere(int n, const double* normal, uint64_t seed, uint64_t path, uint32_t stream, double* out);

#ifdef __cplusplus
}
#endif

#endif
