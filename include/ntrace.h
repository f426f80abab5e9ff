/*
 * ntrace: B200 (sm_100a) n-space path tracer, C ABI.
 *
 * Drop-in boundary for the CPU painter of templeblock/math (src/painter).  The reference is
 * in-process C++: a caller assembles a PaintObjects<N,T> (objects, light sources, projector, default
 * surface; src/painter/objects.h:141-223) and calls
 *     paint<N,T>(notifier, samples_per_pixel, paint_objects, paintbrush, thread_count, stop, smooth_normal)
 * (src/painter/painter.h:40-42, src/painter/painter.cpp:599-625).  This header exposes the same scene
 * vocabulary as plain C: one nt_scene per PaintObjects, one add_* call per visible object or light,
 * nt_render for paint().  The C++ header math_b200/paint.hpp rebuilds the reference's template
 * interface on top of it.
 *
 * Conventions: n is the space dimension (3..6); the screen has n-1 dimensions; every vector is n
 * floats, every edge list is row-major; pixels are linear with x0 fastest (GlobalIndex,
 * src/com/global_index.h:45-147).  Host arrays are copied by the call that receives them.  Every
 * function returns an NT_* status; nt_last_error_message() describes the last failure on the
 * calling thread.  Nothing throws across the ABI (the reference's paint() is noexcept and reports
 * through its notifier, painter.cpp:598-625).  One scene must not be used by two threads at once;
 * separate scenes may render concurrently (each owns a CUDA stream).
 */
#ifndef NTRACE_H
#define NTRACE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NT_OK 0
#define NT_EINVAL 1       /* invalid argument or scene */
#define NT_EDEGENERATE 2  /* degenerate geometry (e.g. a simplex whose normal is not finite) */
#define NT_ECUDA 3        /* CUDA runtime error */
#define NT_ETIMEOUT 4     /* a bounded device loop ran out (walk or sampler bound) */
#define NT_ESTOPPED 5     /* stopped through the stop flag */
#define NT_ENOMEM 6       /* device allocation failed */
#define NT_ESTATE 7       /* call out of order (e.g. render before build) */

typedef struct nt_scene nt_scene;

/* SurfaceProperties subset used by the painter (src/painter/objects.h:26-133). */
typedef struct nt_surface
{
        float color[3];        /* linear RGB */
        float diffuse;         /* diffuse coefficient; 0 disables direct and indirect lighting */
        int light_source;      /* the surface emits light_color */
        float light_color[3];
} nt_surface;

/* Projector kinds (src/painter/projectors/projector.h). */
#define NT_PROJECTOR_PARALLEL 0     /* param: units per pixel */
#define NT_PROJECTOR_PERSPECTIVE 1  /* param: width view angle, degrees */
#define NT_PROJECTOR_SPHERICAL 2    /* param: width view angle, degrees */

typedef struct nt_build_opts
{
        int threads;   /* host threads for the tree build; <= 0: all hardware threads */
        int host_only; /* 1: facet setup and tree build only, no device upload (inspection on hosts
                          without a GPU; render and trace calls then fail with NT_ESTATE) */
        int tree_on_gpu; /* 1: build the 2^n-trees on the GPU (the same trees, box for box, as the host
                            build; much faster for large meshes and for n >= 5); ignored with host_only */
        int leaf_records; /* 0: keep a copy of the FP32 facet records in leaf-list order (a facet's record
                             once per leaf that lists it) when it takes at most a quarter of the free
                             device memory, so that a leaf's records are read without its index list;
                             -1: never (records read through the index lists).  Same results either way. */
} nt_build_opts;

typedef struct nt_render_opts
{
        int samples_per_pixel;  /* rounded up to k^(n-1) as StratifiedJitteredSampler does (sampler.h:31-52) */
        int max_depth;          /* MAX_RECURSION_LEVEL (painter.cpp:42); the reference value is 100 */
        uint64_t seed;          /* Philox key; path id = (sample index) * pixel_count + pixel */
        int retest;             /* 1: re-test uncertain FP32 facet tests in FP64 (default); 0: FP32 only */
        int smooth_normal;      /* paint()'s smooth_normal; meshes without vertex normals ignore it */
        int64_t pool_paths;     /* wavefront path pool size; <= 0: automatic */
        int timing;             /* 1: per-kernel CUDA-event times in nt_stats (iterations enqueued one by one) */
        const volatile int* stop; /* optional host stop flag, polled between batches of wavefront iterations */
        int graph_iterations;   /* wavefront iterations per CUDA-graph launch (the host checks for the end of
                                   the pass after each); <= 0: 4.  nt_autotune picks it with pool_paths. */
        int64_t sample_offset;  /* > 0: index of this pass's first sample per pixel (a sample range of its own,
                                   e.g. one rank's share of a frame rendered on several GPUs: samples
                                   [sample_offset, sample_offset + effective spp) trace the same paths whichever
                                   process renders them); 0: continue after the samples already accumulated
                                   (progressive passes).  The accumulator's sample count grows by the pass's
                                   samples either way. */
        int walk_chunk;         /* tree-walk kernels: 1: facet records read straight from global memory, 32
                                   pooled tests per round; 32, 64 or 128: that many pooled tests per warp
                                   have their records staged in shared memory at once (cp.async); 0: the
                                   default (1).  A tuning choice only: every variant makes the same
                                   decisions.  nt_autotune picks it. */
        int walk_small_leaf;    /* tree-walk kernels: a warp whose lanes' leaves hold at most this many facets each
                                   tests them lane by lane instead of pooling them across the warp; 0: the default
                                   (2); -1: always pooled.  A tuning choice only.  nt_autotune picks it. */
} nt_render_opts;

typedef struct nt_stats
{
        int64_t paths;            /* camera samples traced (BarPaintbrush sample_count) */
        int64_t rays;             /* extension rays traced */
        int64_t shadow_rays;      /* shadow rays traced */
        int64_t facet_tests;      /* ray-simplex tests */
        int64_t box_steps;        /* tree leaves visited */
        int64_t retests;          /* FP64 re-tests */
        int64_t descent_levels;   /* tree nodes visited by point location */
        int64_t error_bits;       /* device error flags (bounded loops that ran out) */
        int spp_effective;        /* samples per pixel actually traced */
        double seconds;           /* host wall time of the call */
        double raygen_ms;         /* device times per kernel kind (timing = 1) */
        double extend_ms;
        double shade_ms;
        double shadow_ms;
        int64_t launches;         /* kernel launches issued by the call */
        int64_t extend_launches;
        int64_t shadow_launches;
        /* the shadow kernel's walk counters (facet_tests .. descent_levels above count extension rays) */
        int64_t shadow_facet_tests;
        int64_t shadow_box_steps;
        int64_t shadow_retests;
        int64_t shadow_descent_levels;
        int64_t iterations;       /* wavefront iterations that had work */
        double plan_ms;           /* device time of the extension rays' plan-and-compact kernel of one-mesh
                                     scenes (timing = 1): it finishes the rays that need no tree walk and lists
                                     the others (the shadow rays' plan runs inside the shading kernel, shade_ms) */
} nt_stats;

typedef struct nt_mesh_info
{
        int64_t facet_count;
        int64_t node_count;       /* tree boxes */
        int64_t leaf_count;
        int64_t index_count;      /* facet references held by leaves */
        int max_depth;            /* tree_max_depth (src/painter/shapes/mesh.cpp:35-58) */
        double distance_from_facet;
        int64_t degenerate_facets; /* facets decided in FP64 only (ill-conditioned barycentric solve) */
        double build_seconds;
        int64_t device_bytes;
} nt_mesh_info;

/* ---- scene assembly (PaintObjects) ---- */

/* Replaces constructing a PaintObjects<N,T> (objects.h:211-223); n = 3..6. */
int nt_scene_create(int n, nt_scene** out);
int nt_scene_destroy(nt_scene* scene);

/* Mesh of (n-1)-simplices: Mesh<N,T>(obj, ...) + VisibleSharedMesh (mesh.cpp:61-135,
 * visible_shapes.h:119-168).  vertices: vertex_count x n; facets: facet_count x n vertex indices. */
int nt_scene_add_mesh(nt_scene* scene, const float* vertices, int64_t vertex_count, const int32_t* facets,
                      int64_t facet_count, const nt_surface* surface);

/* Vertex normals of mesh object `object` (the Obj's normals and per-facet normal indices that
 * MeshHyperplaneSimplex takes, mesh_hyperplane_simplex.cpp:59-143): normals is normal_count x n;
 * facet_normals is facet_count x n indices into normals (all n of a facet -1: that facet has none and
 * is flat), or NULL for the facet's vertex indices.  Each
 * facet is classified as the reference does: any |cos(vertex normal, facet normal)| < 0.7 -> flat;
 * all positive -> interpolated; all negative -> interpolated with the facet normal reversed; mixed ->
 * interpolated with the negative ones reversed.  Used when nt_render_opts.smooth_normal is set. */
int nt_scene_set_mesh_normals(nt_scene* scene, int object, const float* normals, int64_t normal_count,
                              const int32_t* facet_normals);

/* Mesh from an OBJ (n = 3) or OBJ-n (n > 3) file, as the reference's loader reads its geometry
 * (src/obj/file/file_load.cpp): "v" lines of n coordinates, "vn" lines of n normal components, "f"
 * lines of vertex[/texture[/normal]] groups (1-based, negative counted back from the end), facets of
 * more than n groups split into a fan around the first; texture coordinates, materials and other
 * lines are skipped.  Added as a mesh object with `surface`; its vertex normals (if any facet has
 * them) as by nt_scene_set_mesh_normals. */
int nt_scene_add_obj_file(nt_scene* scene, const char* path, const nt_surface* surface);

/* The scene's dimension n, and the number of objects added so far (-1 for a NULL scene). */
int nt_scene_dimension(nt_scene* scene);
int nt_scene_object_count(nt_scene* scene);

/* n-parallelotope: VisibleParallelotope(org, e0..e(n-1)) (visible_shapes.h:75-117).  edges: n x n. */
int nt_scene_add_parallelotope(nt_scene* scene, const float* org, const float* edges, const nt_surface* surface);

/* (n-1)-parallelotope in a hyperplane: VisibleHyperplaneParallelotope (visible_shapes.h:31-73).
 * edges: (n-1) x n. */
int nt_scene_add_hyperplane_parallelotope(nt_scene* scene, const float* org, const float* edges,
                                          const nt_surface* surface);

/* VisiblePointLight(location, color, unit_intensity_distance) (visible_lights.h:24-39,
 * light_source.h:26-57). */
int nt_scene_add_point_light(nt_scene* scene, const float* location, const float* rgb, float unit_intensity_distance);

/* VisibleConstantLight(location, color) (visible_lights.h:41-55, light_source.h:59-78). */
int nt_scene_add_constant_light(nt_scene* scene, const float* location, const float* rgb);

/* Visible{Parallel,Perspective,Spherical}Projector (visible_projectors.h:24-94).  screen_axes:
 * (n-1) x n; screen_size: n-1 ints. */
int nt_scene_set_projector(nt_scene* scene, int kind, const float* camera_org, const float* camera_dir,
                           const float* screen_axes, float param, const int32_t* screen_size);

/* PaintObjects::default_surface_properties (objects.h:222): what a ray that hits nothing returns. */
int nt_scene_set_background(nt_scene* scene, const nt_surface* surface);

/* Removes every light source (add the new ones before the next nt_scene_build).  No counterpart in
 * the reference, where a PaintObjects is assembled once; here it lets one scene be relit without
 * rebuilding its meshes' trees. */
int nt_scene_clear_lights(nt_scene* scene);

/* Replaces the surface of object `object` (objects numbered in the order they were added).  No
 * counterpart in the reference (see nt_scene_clear_lights). */
int nt_scene_set_object_surface(nt_scene* scene, int object, const nt_surface* surface);

/* Facet setup, 2^n-tree build and upload to the device (the work of Mesh's constructor).  A rebuild
 * after edits that leave the meshes unchanged (lights, surfaces, projector, background) reuses the
 * meshes' facet setup, trees and device arrays. */
int nt_scene_build(nt_scene* scene, const nt_build_opts* opts);

int nt_scene_mesh_info(nt_scene* scene, int mesh_index, nt_mesh_info* info);

/* ---- painting (paint<N,T>) ---- */

/* One pass: samples_per_pixel (stratified, effective count k^(n-1)) more samples for every pixel
 * of the screen, added to the scene's accumulator; successive calls continue the sample sequence
 * (or start at opts->sample_offset). */
int nt_render(nt_scene* scene, const nt_render_opts* opts, nt_stats* stats);

/* paint_pixels over a list of pixels (src/painter/painter.cpp:410-448 with a Paintbrush that hands out
 * exactly these pixels, paintbrush.h:26-233): samples_per_pixel (effective k^(n-1)) samples of each
 * listed pixel, samples [max(opts->sample_offset, 0), + effective spp), the same paths as a whole-frame
 * pass with that sample range traces for those pixels.  pixels: count linear pixel indices (x0 fastest,
 * each in [0, pixel count); repeats allowed) in host memory; rgb_mean: count x 3 host floats, the mean
 * colour of each listed pixel over the pass.  The scene's accumulator is not touched.  Used for
 * converged-radiance checks on pixel subsets and for partial re-renders. */
int nt_render_pixels(nt_scene* scene, const nt_render_opts* opts, const int64_t* pixels, int64_t count,
                     float* rgb_mean, nt_stats* stats);

/* nt_render for callers that cannot allocate device memory: applications that own all device memory
 * through their own allocator or a budget fixed at start-up, plugins inside such hosts, and frame
 * loops where an allocation (which may synchronise the device or fail) is not allowed.  No counterpart
 * in the reference, whose painter runs on host memory.
 *
 * One pass of samples_per_pixel over the built scene, like nt_render, but the wavefront's working
 * memory is one file-scope device array of NT_NOALLOC_SCRATCH_BYTES inside the library, and the pass's
 * per-pixel sums (red, green, blue as doubles, x0 fastest) are ADDED to the caller's d_accum
 * (pixel_count x 3 doubles of device memory; zero it before the first pass).  sample_offset is the
 * index of the pass's first sample per pixel (0, then the effective samples of the passes before);
 * opts->sample_offset is not used here.  stream: a cudaStream_t, NULL for the scene's stream.
 * The call allocates nothing: no cudaMalloc, cudaFree, cudaMallocHost, stream or event.  Its first
 * call on a device does a one-time set-up for that device: it looks up the array's device address
 * (cudaGetSymbolAddress), and under CUDA's lazy module loading (the default since CUDA 12.2) that
 * look-up is also what loads the library's module holding the array, so the array's 64 MiB are
 * reserved on the device then.  Make that first call (a warm-up pass) at start-up, while device
 * memory is still available, and before any stream capture.  The array holds at most the path pool
 * that fits in it: opts->pool_paths above that capacity is rejected with NT_EINVAL (0 uses the
 * capacity).  The iterations are enqueued one by one with no events: opts->timing and
 * opts->graph_iterations are ignored and the *_ms fields of stats stay 0.  Every GPU that loads the
 * library keeps the array until the process exits; all calls share it and it keeps the last call's
 * contents (each call clears its counters), so calls that overlap on the GPU race and must be
 * serialised by the caller.  A stream other than the scene's must be ordered by the caller (an event
 * recorded on nt_scene_stream) after every earlier asynchronous update of the scene's device arrays:
 * nt_scene_build and nt_scene_upload finish theirs before they return, but nt_scene_upload_commit
 * only enqueues its copies on the scene's stream, and so does any later call documented as
 * asynchronous on that stream. */
#define NT_NOALLOC_SCRATCH_BYTES (64u << 20)
int nt_render_noalloc(nt_scene* scene, const nt_render_opts* opts, double* d_accum, int64_t sample_offset,
                      void* stream, nt_stats* stats);

int nt_accum_clear(nt_scene* scene);

/* ---- batches and tuning (no counterpart in the reference, which paints one scene per call) ---- */

/* One pass of each of `count` built scenes (distinct; any mix of dimensions), opts[i] for scene i,
 * run side by side: the wavefront iterations of all the passes, each on its scene's stream, are
 * captured into one CUDA graph, and the graph is launched until every pass has finished (a pass
 * that ends first idles through empty iterations).  stats: count entries, or NULL. */
int nt_render_batch(nt_scene* const* scenes, int count, const nt_render_opts* opts, nt_stats* stats);

/* Times probe passes of `base` (its samples per pixel) over candidate path-pool sizes and iterations
 * per graph launch, then over the walk kernels' variants (walk_chunk 1, 32, 64, 128) and small-leaf
 * thresholds (walk_small_leaf -1, 1, 2, 4) at the best of those, and returns the fastest in *tuned (a
 * copy of base with pool_paths, graph_iterations, walk_chunk and walk_small_leaf set) and its pass time
 * in *best_ms (may be NULL).  The probe passes go to the scene's
 * accumulator, which is cleared afterwards. */
int nt_autotune(nt_scene* scene, const nt_render_opts* base, nt_render_opts* tuned, double* best_ms);

/* ---- denoiser inputs (no counterpart in the reference; see include/ntrace_denoise.h) ---- */

/* First hit of every pixel-centre camera ray: the unit geometric normal turned towards the camera
 * (pixel_count x n floats, zeros on a miss) and the hit distance (pixel_count floats, 0 on a miss),
 * into device arrays.  stream: a cudaStream_t, NULL for the scene's stream. */
int nt_render_aux(nt_scene* scene, float* d_normal, float* d_depth, void* stream);

/* One pass of opts->samples_per_pixel (stratified, as nt_render; sample indices from sample_offset)
 * with the radiance of every sample kept apart, then per pixel the mean radiance and the variance of
 * that mean (sample variance / samples; 0 for one sample) into device arrays of pixel_count x 3
 * floats.  The scene's accumulator is not touched. */
int nt_render_moments(nt_scene* scene, const nt_render_opts* opts, int64_t sample_offset, float* d_mean, float* d_var,
                      nt_stats* stats);

/* Mean colour per pixel (pixel_count x 3 floats, x0 fastest) and the samples behind it. */
int nt_accum_read(nt_scene* scene, float* rgb_mean, int64_t* samples_per_pixel);

int64_t nt_scene_pixel_count(nt_scene* scene);

/* Viewer feed: the running mean of one 2-D slice of the screen as the painter window shows it
 * (PainterWindow::set_pixel and its row order, src/ui/painter_window/painter_window.cpp:120-153; sRGB
 * conversion rgb_float_to_srgb_uint8, src/com/color/conversion.cpp:35-42,211-230,344-347): screen
 * axes 0 and 1 span the slice, slice[j] fixes screen axis j + 2 (n - 3 entries; NULL for n = 3), and
 * out receives width x height words 0x00RRGGBB, row 0 being the screen's last row.  out is device
 * memory when device_out, else host memory. */
int nt_accum_read_srgb_slice(nt_scene* scene, const int32_t* slice, uint32_t* out, int device_out);

/* Copies the scene's device arrays again from the pinned host copy the build kept (a scene whose
 * data arrive from the host for every frame); *bytes: host-to-device bytes moved.  No counterpart in
 * the reference, whose scene lives in host memory. */
int nt_scene_upload(nt_scene* scene, int64_t* bytes);

/* The same upload, double-buffered, so that the next frame's data cross PCIe while the current frame
 * renders.  nt_scene_upload_begin queues the copy of the pinned host copy into a device staging
 * buffer (one per mesh, allocated at the first call, the size of the mesh's arrays) on the scene's own
 * copy stream and returns at once; *bytes: host-to-device bytes queued.  nt_scene_upload_commit makes
 * the scene's stream wait for that copy and then copies the staged arrays into the live ones (device
 * to device), so that the next nt_render on the scene's stream sees them; it fails with NT_ESTATE
 * without a begin since the last commit, or when the scene was built in between.  A begin waits on
 * the GPU for the previous commit's copies out of staging.  The commit's copies are ordered only on
 * the scene's stream: a render on another stream (nt_render_noalloc's) must be ordered after them by
 * the caller (an event recorded on nt_scene_stream).  No counterpart in the reference. */
int nt_scene_upload_begin(nt_scene* scene, int64_t* bytes);
int nt_scene_upload_commit(nt_scene* scene);

/* The scene's CUDA stream (cudaStream_t), on which nt_render and nt_trace_closest launch. */
void* nt_scene_stream(nt_scene* scene);

/* ---- fixed-ray-set closest hit (parity checks) ---- */

/* Closest facet of mesh mesh_index for each ray, as Mesh::intersect_approximate followed by
 * Mesh::intersect_precise (mesh.cpp:137-166; the query of shapes/test/test_mesh.cpp:139-152).
 * org, dir: ray_count x n host floats (dir need not be unit); facet: -1 for a miss; t: distance
 * from org along the unit direction.  retest = 1 settles uncertain FP32 decisions in FP64. */
int nt_trace_closest(nt_scene* scene, int mesh_index, const float* org, const float* dir, int64_t ray_count,
                     int retest, int32_t* facet, float* t, nt_stats* stats);

/* Same with device pointers on the caller's stream (cudaStream_t; NULL = the scene's stream). */
int nt_trace_closest_device(nt_scene* scene, int mesh_index, const float* d_org, const float* d_dir,
                            int64_t ray_count, int retest, int32_t* d_facet, float* d_t, void* stream);

/* Tree export (host copies) for checks: node_count int2 nodes ({first_child, -1} or {offset, count}),
 * index_count leaf facet indices, per-level box sizes ((max_depth + 1) x n) and root origin (n). */
int nt_scene_tree_export(nt_scene* scene, int mesh_index, int32_t* nodes, int32_t* indices, float* level_sizes,
                         float* root_org);

/* ---- convex hull (the meshes of the measured scenes) ---- */

/* Boundary facets of the convex hull of `count` points in n = 3..6 dimensions, computed exactly as the
 * reference's integer hull prepares its input (src/geometry/core/convex_hull.cpp:657-707: shuffled with
 * mt19937_64(count), scaled to integers in [0, 2^30 - 1], duplicates dropped) with exact integer
 * predicates.  Facets index the input points (n per facet). */
typedef struct nt_hull nt_hull;
int nt_convex_hull(int n, const float* points, int64_t count, nt_hull** out);
int64_t nt_hull_facet_count(nt_hull* hull);
int nt_hull_facets(nt_hull* hull, int32_t* facets);
int nt_hull_destroy(nt_hull* hull);

/* ---- peaks of this GPU for the rooflines (no counterpart in the reference) ---- */

typedef struct nt_peaks
{
        double l2_read_gbs;      /* L2 read bandwidth: 16-byte loads bypassing L1 over a 32 MiB resident buffer */
        double fp32_fma_tflops;  /* FP32 FMA rate: eight independent fmaf chains per thread, 2 flops per FMA */
        double l2_ms;            /* the timed launches */
        double fma_ms;
} nt_peaks;

/* Measures the two ceilings of the tree-walk kernels besides the HBM copy rate with kernels of this
 * library, timed with CUDA events on the current device (allocates and frees 32 MiB). */
int nt_probe_peaks(nt_peaks* out);

/* ---- misc ---- */

const char* nt_last_error_message(void);

/* Samples per pixel that samples_per_pixel becomes in n dimensions. */
int nt_effective_spp(int n, int samples_per_pixel);

/* cosine_sphere_coefficient(n) (src/painter/coefficient/cosine_sphere.h:97-162). */
double nt_cosine_sphere_coefficient(int n);

#ifdef __cplusplus
}
#endif

#endif
