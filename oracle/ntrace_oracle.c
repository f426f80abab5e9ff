/*
 * ntrace oracle: CPU restatement of the reference n-space path tracer (templeblock/math src/painter).
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * as the checker; never linked into or called by the product.  See ntrace_oracle.h.
 */
#define _GNU_SOURCE

#include "ntrace_oracle.h"

#include <unistd.h>

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define ORT_PI 3.14159265358979323846
#ifndef M_PI
#define M_PI ORT_PI
#endif

/* Philox4x32-10 (Salmon et al., SC 2011): 10 rounds of
 *   (hi0, lo0) = M0 * c0, (hi1, lo1) = M1 * c2,
 *   c = (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0),  key += (W0, W1). */
void ort_philox(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4])
{
        const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
        uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
        uint32_t k0 = key0, k1 = key1;
        for (int r = 0; r < 10; ++r)
        {
                uint64_t p0 = (uint64_t)M0 * c0;
                uint64_t p1 = (uint64_t)M1 * c2;
                uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
                uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
                c0 = hi1 ^ c1 ^ k0;
                c1 = lo1;
                c2 = hi0 ^ c3 ^ k1;
                c3 = lo0;
                k0 += W0;
                k1 += W1;
        }
        out[0] = c0;
        out[1] = c1;
        out[2] = c2;
        out[3] = c3;
}

/* cosine_sphere_coefficient (src/painter/coefficient/cosine_sphere.h:97-162): ratio of the integrals
 * of 1 and of cos over the hemisphere, pi/2 * (n-1)(n-3).../((n-2)(n-4)...) for even n and
 * (n-1)(n-3).../((n-2)(n-4)...) for odd n. */
double ort_cosine_sphere_coefficient(int n)
{
        unsigned long long divident = 1;
        unsigned long long divisor = (n & 1) == 0 ? 2 : 1;
        for (int i = n - 1; i > 1; i -= 2)
        {
                divident *= (unsigned long long)i;
                if (i > 2)
                {
                        divisor *= (unsigned long long)(i - 1);
                }
                unsigned long long a = divident, b = divisor;
                while (b)
                {
                        unsigned long long t = a % b;
                        a = b;
                        b = t;
                }
                if (a > 1)
                {
                        divident /= a;
                        divisor /= a;
                }
        }
        long double p = (long double)divident / (long double)divisor;
        if ((n & 1) == 0)
        {
                p *= 3.1415926535897932384626433832795028841971693993751L;
        }
        return (double)p;
}

int ort_effective_spp(int n, int spp)
{
        int m = n - 1;
        if (spp < 1)
        {
                return -1;
        }
        double v = pow(spp, 1.0 / m);
        unsigned f = (unsigned)floor(v);
        unsigned long long p = 1;
        for (int i = 0; i < m; ++i)
        {
                p *= f;
        }
        if (p >= (unsigned long long)spp)
        {
                return (int)p;
        }
        unsigned c = (unsigned)ceil(v);
        p = 1;
        for (int i = 0; i < m; ++i)
        {
                p *= c;
        }
        return (int)p;
}

static int one_dimension_size(int n, int spp)
{
        int m = n - 1;
        double v = pow(spp, 1.0 / m);
        unsigned f = (unsigned)floor(v);
        unsigned long long p = 1;
        for (int i = 0; i < m; ++i)
        {
                p *= f;
        }
        if (p >= (unsigned long long)spp)
        {
                return (int)f;
        }
        return (int)ceil(v);
}

/* ---- double core ---- */
#define REAL double
#define SFX(x) x##_f64
#define FMA fma
#define SQRT sqrt
#define REAL_EPS DBL_EPSILON
#define REAL_MAX DBL_MAX
#define REAL_LOWEST (-DBL_MAX)
#include "ntrace_oracle_core.inc"
#undef REAL
#undef SFX
#undef FMA
#undef SQRT
#undef REAL_EPS
#undef REAL_MAX
#undef REAL_LOWEST
#undef SFX_LP_M
#undef SFX_TREE_MIN_OBJECTS

/* ---- float core ---- */
#define REAL float
#define SFX(x) x##_f32
#define FMA fmaf
#define SQRT sqrtf
#define REAL_EPS FLT_EPSILON
#define REAL_MAX FLT_MAX
#define REAL_LOWEST (-FLT_MAX)
#include "ntrace_oracle_core.inc"
#undef REAL
#undef SFX
#undef FMA
#undef SQRT
#undef REAL_EPS
#undef REAL_MAX
#undef REAL_LOWEST

/* ---- public API ---- */

typedef struct
{
        int n;
        int dbl;
        void* m;
} OrtMesh;

void* ort_mesh_build(int n, int dbl, const float* verts, long nverts, const int* facets, long nfacets, char* err,
                     int errlen)
{
        if (n < 3 || n > 6)
        {
                snprintf(err, errlen, "n must be 3..6");
                return NULL;
        }
        if (nfacets < 1)
        {
                snprintf(err, errlen, "No facets found in obj");
                return NULL;
        }
        void* m = dbl ? (void*)mesh_build_f64(n, verts, nverts, facets, nfacets, err, errlen)
                      : (void*)mesh_build_f32(n, verts, nverts, facets, nfacets, err, errlen);
        if (!m)
        {
                return NULL;
        }
        OrtMesh* h = malloc(sizeof(OrtMesh));
        h->n = n;
        h->dbl = dbl;
        h->m = m;
        return h;
}

void ort_mesh_destroy(void* mesh)
{
        OrtMesh* h = (OrtMesh*)mesh;
        if (!h)
        {
                return;
        }
        if (h->dbl)
        {
                mesh_free_f64(h->m);
        }
        else
        {
                mesh_free_f32(h->m);
        }
        free(h);
}

int ort_mesh_trace(void* mesh, const float* org, const float* dir, long nrays, int* facet_out, double* t_out,
                   ort_stats* stats)
{
        OrtMesh* h = (OrtMesh*)mesh;
        int n = h->n;
        long long ft = 0, bs = 0, dl = 0;
        for (long r = 0; r < nrays; ++r)
        {
                if (h->dbl)
                {
                        Mesh_f64* m = h->m;
                        Counters_f64 cnt = {0};
                        double o[ORT_NMAX], d[ORT_NMAX];
                        for (int k = 0; k < n; ++k)
                        {
                                o[k] = org[r * n + k];
                                d[k] = dir[r * n + k];
                        }
                        Ray_f64 ray;
                        ray_make_f64(n, o, d, &ray);
                        double a, t;
                        long f;
                        if (mesh_intersect_root_f64(m, &ray, &a) && mesh_intersect_precise_f64(m, &ray, a, &t, &f, &cnt))
                        {
                                facet_out[r] = (int)f;
                                t_out[r] = t;
                        }
                        else
                        {
                                facet_out[r] = -1;
                                t_out[r] = 0;
                        }
                        ft += cnt.facet_tests;
                        bs += cnt.box_steps;
                        dl += cnt.descent_levels;
                }
                else
                {
                        Mesh_f32* m = h->m;
                        Counters_f32 cnt = {0};
                        float o[ORT_NMAX], d[ORT_NMAX];
                        for (int k = 0; k < n; ++k)
                        {
                                o[k] = org[r * n + k];
                                d[k] = dir[r * n + k];
                        }
                        Ray_f32 ray;
                        ray_make_f32(n, o, d, &ray);
                        float a, t;
                        long f;
                        if (mesh_intersect_root_f32(m, &ray, &a) && mesh_intersect_precise_f32(m, &ray, a, &t, &f, &cnt))
                        {
                                facet_out[r] = (int)f;
                                t_out[r] = t;
                        }
                        else
                        {
                                facet_out[r] = -1;
                                t_out[r] = 0;
                        }
                        ft += cnt.facet_tests;
                        bs += cnt.box_steps;
                        dl += cnt.descent_levels;
                }
        }
        if (stats)
        {
                memset(stats, 0, sizeof(*stats));
                stats->facet_tests = ft;
                stats->box_steps = bs;
                stats->descent_levels = dl;
                stats->rays = nrays;
        }
        return 0;
}

int ort_mesh_tree_info(void* mesh, long* box_count, long* index_count, double* distance_from_facet)
{
        OrtMesh* h = (OrtMesh*)mesh;
        if (h->dbl)
        {
                Mesh_f64* m = h->m;
                *box_count = m->nboxes;
                *index_count = m->boff[m->nboxes];
                *distance_from_facet = m->distance_from_facet;
        }
        else
        {
                Mesh_f32* m = h->m;
                *box_count = m->nboxes;
                *index_count = m->boff[m->nboxes];
                *distance_from_facet = m->distance_from_facet;
        }
        return 0;
}

int ort_mesh_tree_export(void* mesh, double* org, double* size, int* first_child, int* depth, long* index_offset,
                         int* indices)
{
        OrtMesh* h = (OrtMesh*)mesh;
        int n = h->n;
        if (h->dbl)
        {
                Mesh_f64* m = h->m;
                for (long i = 0; i < m->nboxes * n; ++i)
                {
                        org[i] = m->borg[i];
                        size[i] = m->bsize[i];
                }
                memcpy(first_child, m->bfirst, sizeof(int) * (size_t)m->nboxes);
                memcpy(depth, m->bdepth, sizeof(int) * (size_t)m->nboxes);
                memcpy(index_offset, m->boff, sizeof(long) * (size_t)(m->nboxes + 1));
                memcpy(indices, m->bidx, sizeof(int) * (size_t)m->boff[m->nboxes]);
        }
        else
        {
                Mesh_f32* m = h->m;
                for (long i = 0; i < m->nboxes * n; ++i)
                {
                        org[i] = m->borg[i];
                        size[i] = m->bsize[i];
                }
                memcpy(first_child, m->bfirst, sizeof(int) * (size_t)m->nboxes);
                memcpy(depth, m->bdepth, sizeof(int) * (size_t)m->nboxes);
                memcpy(index_offset, m->boff, sizeof(long) * (size_t)(m->nboxes + 1));
                memcpy(indices, m->bidx, sizeof(int) * (size_t)m->boff[m->nboxes]);
        }
        return 0;
}

int ort_mesh_facet_export(void* mesh, double* normal, double* planes)
{
        OrtMesh* h = (OrtMesh*)mesh;
        int n = h->n;
        if (h->dbl)
        {
                Mesh_f64* m = h->m;
                for (long i = 0; i < m->nfacets * n; ++i)
                {
                        normal[i] = m->normal[i];
                }
                for (long i = 0; i < m->nfacets * (n - 1) * (n + 1); ++i)
                {
                        planes[i] = m->planes[i];
                }
        }
        else
        {
                Mesh_f32* m = h->m;
                for (long i = 0; i < m->nfacets * n; ++i)
                {
                        normal[i] = m->normal[i];
                }
                for (long i = 0; i < m->nfacets * (n - 1) * (n + 1); ++i)
                {
                        planes[i] = m->planes[i];
                }
        }
        return 0;
}

static double now_seconds(void)
{
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        return ts.tv_sec + ts.tv_nsec * 1e-9;
}

#define ORT_PAINT_IMPL(S)                                                                                         \
        static int paint_##S(const ort_scene* in, int spp, int max_depth, uint64_t seed, int threads,           \
                             const int* pixels, long npix, long long sample_offset, float* rgb_out,              \
                             ort_stats* stats, char* err, int errlen)                                            \
        {                                                                                                         \
                int n = in->n;                                                                                    \
                Mesh_##S* mesh = NULL;                                                                            \
                Mesh_##S* mesh2 = NULL;                                                                           \
                if (in->nfacets > 0)                                                                              \
                {                                                                                                 \
                        mesh = mesh_build_##S(n, in->verts, in->nverts, in->facets, in->nfacets, err, errlen);   \
                        if (!mesh)                                                                                \
                        {                                                                                         \
                                return 1;                                                                         \
                        }                                                                                         \
                }                                                                                                 \
                if (in->nfacets2 > 0)                                                                             \
                {                                                                                                 \
                        mesh2 = mesh_build_##S(n, in->verts2, in->nverts2, in->facets2, in->nfacets2, err,       \
                                               errlen);                                                           \
                        if (!mesh2)                                                                               \
                        {                                                                                         \
                                mesh_free_##S(mesh);                                                              \
                                return 1;                                                                         \
                        }                                                                                         \
                }                                                                                                 \
                Scene_##S scene;                                                                                  \
                if (scene_make_##S(in, mesh, mesh2, max_depth, &scene, err, errlen))                              \
                {                                                                                                 \
                        mesh_free_##S(mesh);                                                                      \
                        mesh_free_##S(mesh2);                                                                     \
                        return 1;                                                                                 \
                }                                                                                                 \
                PaintJob_##S job;                                                                                 \
                memset(&job, 0, sizeof(job));                                                                     \
                job.s = &scene;                                                                                   \
                job.spp = spp;                                                                                    \
                job.k1d = one_dimension_size(n, spp);                                                             \
                job.spp_eff = ort_effective_spp(n, spp);                                                          \
                job.seed = seed;                                                                                  \
                job.pixels = pixels;                                                                              \
                long total = 1;                                                                                   \
                for (int j = 0; j < n - 1; ++j)                                                                   \
                {                                                                                                 \
                        total *= in->screen[j];                                                                   \
                }                                                                                                 \
                job.npix = pixels ? npix : total;                                                                 \
                job.total_pixels = total;                                                                         \
                job.sample_offset = sample_offset;                                                                \
                job.out = rgb_out;                                                                                \
                pthread_mutex_init(&job.lock, NULL);                                                              \
                double t0 = now_seconds();                                                                        \
                if (threads <= 1)                                                                                 \
                {                                                                                                 \
                        paint_worker_##S(&job);                                                                   \
                }                                                                                                 \
                else                                                                                              \
                {                                                                                                 \
                        pthread_t* th = malloc(sizeof(pthread_t) * (size_t)threads);                              \
                        for (int i = 0; i < threads; ++i)                                                         \
                        {                                                                                         \
                                pthread_create(&th[i], NULL, paint_worker_##S, &job);                             \
                        }                                                                                         \
                        for (int i = 0; i < threads; ++i)                                                         \
                        {                                                                                         \
                                pthread_join(th[i], NULL);                                                        \
                        }                                                                                         \
                        free(th);                                                                                 \
                }                                                                                                 \
                double t1 = now_seconds();                                                                        \
                pthread_mutex_destroy(&job.lock);                                                                 \
                if (stats)                                                                                        \
                {                                                                                                 \
                        stats->paths = (long long)job.npix * job.spp_eff;                                         \
                        stats->rays = job.total.rays;                                                             \
                        stats->facet_tests = job.total.facet_tests;                                               \
                        stats->box_steps = job.total.box_steps;                                                   \
                        stats->descent_levels = job.total.descent_levels;                                         \
                        stats->shadow_rays = job.total.shadow_rays;                                               \
                        stats->seconds = t1 - t0;                                                                 \
                }                                                                                                 \
                free(scene.ntype);                                                                                \
                free(scene.nsign);                                                                                \
                mesh_free_##S(mesh);                                                                              \
                mesh_free_##S(mesh2);                                                                             \
                return 0;                                                                                         \
        }

ORT_PAINT_IMPL(f64)
ORT_PAINT_IMPL(f32)

int ort_paint(const ort_scene* scene, int spp, int max_depth, uint64_t seed, int threads, const int* pixels,
              long npix, long long sample_offset, float* rgb_out, ort_stats* stats, char* err, int errlen)
{
        if (!scene || scene->n < 3 || scene->n > 6)
        {
                snprintf(err, errlen, "n must be 3..6");
                return 2;
        }
        if (spp < 1)
        {
                snprintf(err, errlen, "samples per pixel must be positive");
                return 2;
        }
        if (scene->dbl)
        {
                return paint_f64(scene, spp, max_depth, seed, threads, pixels, npix, sample_offset, rgb_out, stats,
                                 err, errlen);
        }
        return paint_f32(scene, spp, max_depth, seed, threads, pixels, npix, sample_offset, rgb_out, stats, err,
                         errlen);
}

int ort_cosine_hemisphere(int n, const double* normal, uint64_t seed, uint64_t path, uint32_t stream, double* out)
{
        Rng_f64 g;
        g.k0 = (uint32_t)seed;
        g.k1 = (uint32_t)(seed >> 32);
        g.path = path;
        return cosine_hemisphere_f64(n, &g, stream, normal, out);
}
