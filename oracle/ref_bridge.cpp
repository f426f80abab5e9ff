// Test infrastructure: a C bridge onto the reference painter, compiled from the reference's own
// sources where they lie (templeblock/math src/painter, src/com, src/obj).  Only tests, smoke() and
// bench.py's CPU-baseline leg load the library built from this file; the product never does.
//
// What the bridge exposes, and which reference code it drives:
//   refb_mesh_create / refb_mesh_trace  - Mesh<N,T> (src/painter/shapes/mesh.cpp:61-166) built from an
//       Obj made by create_obj_for_facets (src/obj/create/facets.cpp:244-262), and the closest-hit query
//       intersect_approximate + intersect_precise exactly as src/painter/shapes/test/test_mesh.cpp:139-152.
//   refb_mesh_tree_*                    - the 2^N-tree that Mesh built (src/painter/space/tree.h:390-525).
//   refb_paint                          - paint<N,T>() (src/painter/painter.cpp:599-625) on a scene made of
//       the reference's own VisibleSharedMesh (one or two), VisibleParallelotope,
//       VisibleHyperplaneParallelotope, VisiblePointLight/ConstantLight and
//       VisibleParallel/Perspective/SphericalProjector (src/painter/visible_*.h).
//
// Two constants of painter.cpp are made adjustable without editing that file.  painter.cpp is
// included textually below; its functions live in an unnamed namespace, and an unqualified name used
// there is looked up in that namespace before the global one.  Declaring MAX_RECURSION_LEVEL and
// RandomEngineWithSeed in the unnamed namespace first therefore replaces, for painter.cpp's own code,
//   - the recursion cap (painter.cpp:42,303; the reference value is 100), and
//   - the OS-seeded per-thread engine (painter.cpp:460, src/com/random/engine.h:24-60) by a seeded one,
// while the global definitions of the same names (painter.cpp:42, engine.h:26) still compile unchanged.

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

namespace
{
int MAX_RECURSION_LEVEL = 100;

std::atomic<unsigned long long> g_engine_seed{0};

template <typename E>
class RandomEngineWithSeed
{
        E m_engine;

public:
        using result_type = typename E::result_type;

        RandomEngineWithSeed() : m_engine(g_engine_seed.fetch_add(1))
        {
        }

        operator E&()
        {
                return m_engine;
        }

        result_type operator()()
        {
                return m_engine();
        }

        static constexpr result_type min()
        {
                return E::min();
        }

        static constexpr result_type max()
        {
                return E::max();
        }
};
}

#include "painter/painter.cpp"

#include "com/log.h"
#include "obj/create/facets.h"
#include "painter/shapes/mesh.h"
#include "painter/visible_lights.h"
#include "painter/visible_projectors.h"
#include "painter/visible_shapes.h"
#include "painter/visible_paintbrush.h"
#include "progress/progress.h"

// ---------------------------------------------------------------------------------------------
// Access to Mesh<N,T>::m_facets, Mesh<N,T>::m_tree and SpatialSubdivisionTree::m_boxes.  The names
// are private; an explicit instantiation may name private members ([temp.explicit]/12), which is
// how the member pointers below are obtained.  Read-only use.

namespace refb_access
{
template <typename Tag, typename Tag::type M>
struct Rob
{
        friend typename Tag::type get(Tag)
        {
                return M;
        }
};

template <size_t N, typename T>
struct FacetsTag
{
        using type = std::vector<MeshHyperplaneSimplex<N, T>> Mesh<N, T>::*;
        friend type get(FacetsTag);
};

template <size_t N, typename T>
struct TreeTag
{
        using type = SpatialSubdivisionTree<ParallelotopeOrtho<N, T>> Mesh<N, T>::*;
        friend type get(TreeTag);
};

template <size_t N, typename T>
using BoxT = spatial_subdivision_tree_implementation::Box<ParallelotopeOrtho<N, T>>;

template <size_t N, typename T>
struct BoxesTag
{
        using type = std::vector<BoxT<N, T>> SpatialSubdivisionTree<ParallelotopeOrtho<N, T>>::*;
        friend type get(BoxesTag);
};

template <size_t N, typename T>
struct DistanceTag
{
        using type = T SpatialSubdivisionTree<ParallelotopeOrtho<N, T>>::*;
        friend type get(DistanceTag);
};

#define REFB_ROB(N, T)                                                                                         \
        template struct Rob<FacetsTag<N, T>, &Mesh<N, T>::m_facets>;                                          \
        template struct Rob<TreeTag<N, T>, &Mesh<N, T>::m_tree>;                                              \
        template struct Rob<BoxesTag<N, T>, &SpatialSubdivisionTree<ParallelotopeOrtho<N, T>>::m_boxes>;      \
        template struct Rob<DistanceTag<N, T>, &SpatialSubdivisionTree<ParallelotopeOrtho<N, T>>::m_distance_from_facet>;

REFB_ROB(3, float)
REFB_ROB(4, float)
REFB_ROB(5, float)
REFB_ROB(6, float)
REFB_ROB(3, double)
REFB_ROB(4, double)
REFB_ROB(5, double)
REFB_ROB(6, double)
#undef REFB_ROB
}

namespace
{
std::once_flag g_log_once;

void ensure_log()
{
        std::call_once(g_log_once, []() { log_init(); });
}

void copy_error(const std::string& s, char* err, int errlen)
{
        if (err && errlen > 0)
        {
                std::strncpy(err, s.c_str(), errlen - 1);
                err[errlen - 1] = 0;
        }
}

class NullProgress
{
};

struct MeshHandleBase
{
        int n;
        int dbl;
        virtual ~MeshHandleBase() = default;
};

template <size_t N, typename T>
struct MeshHandle final : MeshHandleBase
{
        std::shared_ptr<const Mesh<N, T>> mesh;
};

// An Obj<N> (src/obj/obj.h) holding the caller's vertices, vertex normals and facets as given (the
// reference's create_obj_for_facets with normals averages them with the face normals; the mesh with
// vertex normals here must take them unchanged, as the product's nt_scene_set_mesh_normals does).
template <size_t N>
class NormalsObj final : public Obj<N>
{
        std::vector<Vector<N, float>> m_vertices;
        std::vector<Vector<N, float>> m_normals;
        std::vector<Vector<N - 1, float>> m_texcoords;
        std::vector<typename Obj<N>::Facet> m_facets;
        std::vector<typename Obj<N>::Point> m_points;
        std::vector<typename Obj<N>::Line> m_lines;
        std::vector<typename Obj<N>::Material> m_materials;
        std::vector<typename Obj<N>::Image> m_images;

public:
        NormalsObj(const float* verts, long nverts, const int* facets, long nfacets, const float* normals, long nnormals,
                   const int* facet_normals)
                : m_vertices(nverts), m_normals(nnormals), m_facets(nfacets)
        {
                for (long i = 0; i < nverts; ++i)
                {
                        for (unsigned k = 0; k < N; ++k)
                        {
                                m_vertices[i][k] = verts[i * N + k];
                        }
                }
                for (long i = 0; i < nnormals; ++i)
                {
                        for (unsigned k = 0; k < N; ++k)
                        {
                                m_normals[i][k] = normals[i * N + k];
                        }
                }
                for (long f = 0; f < nfacets; ++f)
                {
                        typename Obj<N>::Facet& fc = m_facets[f];
                        fc.material = -1;
                        fc.has_texcoord = false;
                        fc.has_normal = !(facet_normals && facet_normals[f * N] < 0);
                        for (unsigned i = 0; i < N; ++i)
                        {
                                fc.vertices[i] = facets[f * N + i];
                                fc.normals[i] = facet_normals ? facet_normals[f * N + i] : facets[f * N + i];
                                fc.texcoords[i] = -1;
                        }
                }
        }
        const std::vector<Vector<N, float>>& vertices() const override
        {
                return m_vertices;
        }
        const std::vector<Vector<N, float>>& normals() const override
        {
                return m_normals;
        }
        const std::vector<Vector<N - 1, float>>& texcoords() const override
        {
                return m_texcoords;
        }
        const std::vector<typename Obj<N>::Facet>& facets() const override
        {
                return m_facets;
        }
        const std::vector<typename Obj<N>::Point>& points() const override
        {
                return m_points;
        }
        const std::vector<typename Obj<N>::Line>& lines() const override
        {
                return m_lines;
        }
        const std::vector<typename Obj<N>::Material>& materials() const override
        {
                return m_materials;
        }
        const std::vector<typename Obj<N>::Image>& images() const override
        {
                return m_images;
        }
        Vector<N, float> center() const override
        {
                return Vector<N, float>(0);
        }
        float length() const override
        {
                return 1;
        }
};

template <size_t N, typename T>
MeshHandleBase* mesh_create(const float* verts, long nverts, const int* facets, long nfacets, int threads,
                            const float* normals = nullptr, long nnormals = 0, const int* facet_normals = nullptr)
{
        if (normals && nnormals > 0)
        {
                NormalsObj<N> obj(verts, nverts, facets, nfacets, normals, nnormals, facet_normals);
                ProgressRatio progress(nullptr);
                constexpr Matrix<N + 1, N + 1, T> matrix(1);
                auto h = std::make_unique<MeshHandle<N, T>>();
                h->n = N;
                h->dbl = std::is_same_v<T, double>;
                h->mesh = std::make_shared<const Mesh<N, T>>(&obj, matrix, threads, &progress);
                return h.release();
        }
        std::vector<Vector<N, float>> points(nverts);
        for (long i = 0; i < nverts; ++i)
        {
                for (unsigned k = 0; k < N; ++k)
                {
                        points[i][k] = verts[i * N + k];
                }
        }
        std::vector<std::array<int, N>> fs(nfacets);
        for (long i = 0; i < nfacets; ++i)
        {
                for (unsigned k = 0; k < N; ++k)
                {
                        fs[i][k] = facets[i * N + k];
                }
        }
        std::unique_ptr<Obj<N>> obj = create_obj_for_facets(points, fs);
        ProgressRatio progress(nullptr);
        constexpr Matrix<N + 1, N + 1, T> matrix(1);
        auto h = std::make_unique<MeshHandle<N, T>>();
        h->n = N;
        h->dbl = std::is_same_v<T, double>;
        h->mesh = std::make_shared<const Mesh<N, T>>(obj.get(), matrix, threads, &progress);
        return h.release();
}

template <size_t N, typename T>
void mesh_trace(const MeshHandleBase* hb, const float* org, const float* dir, long nrays, int* facet_out, double* t_out)
{
        const Mesh<N, T>& mesh = *static_cast<const MeshHandle<N, T>*>(hb)->mesh;
        const auto& facets = mesh.*get(refb_access::FacetsTag<N, T>());
        const MeshHyperplaneSimplex<N, T>* base = facets.data();
        for (long r = 0; r < nrays; ++r)
        {
                Vector<N, T> o, d;
                for (unsigned k = 0; k < N; ++k)
                {
                        o[k] = org[r * N + k];
                        d[k] = dir[r * N + k];
                }
                Ray<N, T> ray(o, d);
                T approximate, precise;
                const void* data;
                if (mesh.intersect_approximate(ray, &approximate) &&
                    mesh.intersect_precise(ray, approximate, &precise, &data))
                {
                        facet_out[r] = static_cast<int>(static_cast<const MeshHyperplaneSimplex<N, T>*>(data) - base);
                        t_out[r] = precise;
                }
                else
                {
                        facet_out[r] = -1;
                        t_out[r] = 0;
                }
        }
}

template <size_t N, typename T>
void mesh_tree_info(const MeshHandleBase* hb, long* box_count, long* index_count, double* distance)
{
        const Mesh<N, T>& mesh = *static_cast<const MeshHandle<N, T>*>(hb)->mesh;
        const auto& tree = mesh.*get(refb_access::TreeTag<N, T>());
        const auto& boxes = tree.*get(refb_access::BoxesTag<N, T>());
        long idx = 0;
        for (const auto& b : boxes)
        {
                idx += b.object_index_count();
        }
        *box_count = static_cast<long>(boxes.size());
        *index_count = idx;
        *distance = tree.*get(refb_access::DistanceTag<N, T>());
}

template <size_t N, typename T>
void mesh_tree_export(const MeshHandleBase* hb, double* org, double* size, int* children, long* index_offset,
                      int* indices)
{
        const Mesh<N, T>& mesh = *static_cast<const MeshHandle<N, T>*>(hb)->mesh;
        const auto& tree = mesh.*get(refb_access::TreeTag<N, T>());
        const auto& boxes = tree.*get(refb_access::BoxesTag<N, T>());
        constexpr int C = 1 << N;
        long off = 0;
        for (size_t i = 0; i < boxes.size(); ++i)
        {
                const auto& p = boxes[i].parallelotope();
                for (unsigned k = 0; k < N; ++k)
                {
                        org[i * N + k] = p.org()[k];
                        size[i * N + k] = p.e(k)[k];
                }
                for (int c = 0; c < C; ++c)
                {
                        children[i * C + c] = boxes[i].childs()[c];
                }
                index_offset[i] = off;
                for (int v : boxes[i].object_indices())
                {
                        indices[off++] = v;
                }
        }
        index_offset[boxes.size()] = off;
}
}

// ---------------------------------------------------------------------------------------------
// Scene description shared with the tests (all arrays are row-major, n = space dimension).

extern "C" {

struct refb_scene
{
        int n;
        int dbl;
        // mesh (nfacets == 0: no mesh)
        const float* verts;
        long nverts;
        const int* facets;
        long nfacets;
        float mesh_color[3];
        float mesh_diffuse;
        // general parallelotope (the floor slab); has_floor == 0: none
        int has_floor;
        float floor_org[6];
        float floor_edges[36];
        float floor_color[3];
        float floor_diffuse;
        // light: kind 0 point (PointLight), 1 constant (ConstantLight)
        int light_kind;
        float light_pos[6];
        float light_color[3];
        float light_unit_distance;
        // projector: kind 0 parallel, 1 perspective, 2 spherical
        int projector_kind;
        float cam_org[6];
        float cam_dir[6];
        float screen_axes[30];
        float proj_param;
        int screen[5];
        // background (default surface properties)
        float bg_color[3];
        float bg_light_color[3];
        int bg_is_light;
        int smooth_normal;
        int tree_threads;
        // optional vertex normals of the mesh (nnormals == 0: none); facet_normals NULL: vertex indices
        const float* normals;
        long nnormals;
        const int* facet_normals;
        // optional second mesh (nfacets2 == 0: none), after the first in object order
        const float* verts2;
        long nverts2;
        const int* facets2;
        long nfacets2;
        float mesh2_color[3];
        float mesh2_diffuse;
        // optional (n-1)-parallelotope in a hyperplane (has_hplt == 0: none), last in object order
        int has_hplt;
        float hplt_org[6];
        float hplt_edges[30];
        float hplt_color[3];
        float hplt_diffuse;
};

struct refb_stats
{
        long long pass_count;
        long long pixel_count;
        long long ray_count;
        long long sample_count;
        double seconds;
};
}

namespace
{
template <size_t N, typename T>
Vector<N, T> vec_from(const float* p)
{
        Vector<N, T> v;
        for (unsigned k = 0; k < N; ++k)
        {
                v[k] = p[k];
        }
        return v;
}

Color color_from(const float* c)
{
        return Color(Vector<3, float>(c[0], c[1], c[2]));
}

template <size_t N, typename T>
class BridgeScene final : public PaintObjects<N, T>
{
        std::unique_ptr<VisibleSharedMesh<N, T>> m_mesh;
        std::unique_ptr<VisibleSharedMesh<N, T>> m_mesh2;
        std::unique_ptr<VisibleParallelotope<N, T>> m_floor;
        std::unique_ptr<VisibleHyperplaneParallelotope<N, T>> m_hplt;
        std::unique_ptr<const LightSource<N, T>> m_light;
        std::unique_ptr<const Projector<N, T>> m_projector;
        SurfaceProperties<N, T> m_default;
        std::vector<const GenericObject<N, T>*> m_objects;
        std::vector<const LightSource<N, T>*> m_lights;

        template <size_t... I>
        static std::unique_ptr<VisibleParallelotope<N, T>> make_floor(const Vector<N, T>& org,
                                                                     const std::array<Vector<N, T>, N>& e,
                                                                     std::index_sequence<I...>)
        {
                return std::make_unique<VisibleParallelotope<N, T>>(org, e[I]...);
        }

        template <size_t... I>
        static std::unique_ptr<VisibleHyperplaneParallelotope<N, T>> make_hplt(const Vector<N, T>& org,
                                                                              const std::array<Vector<N, T>, N - 1>& e,
                                                                              std::index_sequence<I...>)
        {
                return std::make_unique<VisibleHyperplaneParallelotope<N, T>>(org, e[I]...);
        }

public:
        BridgeScene(const refb_scene& s, std::shared_ptr<const Mesh<N, T>> mesh,
                    std::shared_ptr<const Mesh<N, T>> mesh2 = nullptr)
        {
                if (mesh)
                {
                        m_mesh = std::make_unique<VisibleSharedMesh<N, T>>(mesh);
                        m_mesh->set_color(color_from(s.mesh_color));
                        m_mesh->set_diffuse_and_fresnel(s.mesh_diffuse, 0);
                        m_mesh->set_light_source(false);
                        m_objects.push_back(m_mesh.get());
                }
                if (mesh2)
                {
                        m_mesh2 = std::make_unique<VisibleSharedMesh<N, T>>(mesh2);
                        m_mesh2->set_color(color_from(s.mesh2_color));
                        m_mesh2->set_diffuse_and_fresnel(s.mesh2_diffuse, 0);
                        m_mesh2->set_light_source(false);
                        m_objects.push_back(m_mesh2.get());
                }
                if (s.has_floor)
                {
                        std::array<Vector<N, T>, N> e;
                        for (unsigned i = 0; i < N; ++i)
                        {
                                e[i] = vec_from<N, T>(s.floor_edges + i * N);
                        }
                        m_floor = make_floor(vec_from<N, T>(s.floor_org), e, std::make_index_sequence<N>());
                        m_floor->set_color(color_from(s.floor_color));
                        m_floor->set_diffuse_and_fresnel(s.floor_diffuse, 0);
                        m_floor->set_light_source(false);
                        m_objects.push_back(m_floor.get());
                }
                if (s.has_hplt)
                {
                        std::array<Vector<N, T>, N - 1> e;
                        for (unsigned i = 0; i < N - 1; ++i)
                        {
                                e[i] = vec_from<N, T>(s.hplt_edges + i * N);
                        }
                        m_hplt = make_hplt(vec_from<N, T>(s.hplt_org), e, std::make_index_sequence<N - 1>());
                        m_hplt->set_color(color_from(s.hplt_color));
                        m_hplt->set_diffuse_and_fresnel(s.hplt_diffuse, 0);
                        m_hplt->set_light_source(false);
                        m_objects.push_back(m_hplt.get());
                }
                if (s.light_kind == 0)
                {
                        m_light = std::make_unique<const VisiblePointLight<N, T>>(
                                vec_from<N, T>(s.light_pos), color_from(s.light_color), s.light_unit_distance);
                }
                else
                {
                        m_light = std::make_unique<const VisibleConstantLight<N, T>>(vec_from<N, T>(s.light_pos),
                                                                                   color_from(s.light_color));
                }
                m_lights.push_back(m_light.get());

                std::array<Vector<N, T>, N - 1> axes;
                std::array<int, N - 1> screen;
                for (unsigned i = 0; i < N - 1; ++i)
                {
                        axes[i] = vec_from<N, T>(s.screen_axes + i * N);
                        screen[i] = s.screen[i];
                }
                if (s.projector_kind == 0)
                {
                        m_projector = std::make_unique<const VisibleParallelProjector<N, T>>(
                                vec_from<N, T>(s.cam_org), vec_from<N, T>(s.cam_dir), axes, s.proj_param, screen);
                }
                else if (s.projector_kind == 1)
                {
                        m_projector = std::make_unique<const VisiblePerspectiveProjector<N, T>>(
                                vec_from<N, T>(s.cam_org), vec_from<N, T>(s.cam_dir), axes, s.proj_param, screen);
                }
                else
                {
                        m_projector = std::make_unique<const VisibleSphericalProjector<N, T>>(
                                vec_from<N, T>(s.cam_org), vec_from<N, T>(s.cam_dir), axes, s.proj_param, screen);
                }

                m_default.set_color(color_from(s.bg_color));
                m_default.set_diffuse_and_fresnel(1, 0);
                m_default.set_light_source(s.bg_is_light != 0);
                m_default.set_light_source_color(color_from(s.bg_light_color));
        }

        const std::vector<const GenericObject<N, T>*>& objects() const override
        {
                return m_objects;
        }
        const std::vector<const LightSource<N, T>*>& light_sources() const override
        {
                return m_lights;
        }
        const Projector<N, T>& projector() const override
        {
                return *m_projector;
        }
        const SurfaceProperties<N, T>& default_surface_properties() const override
        {
                return m_default;
        }
};

// A Paintbrush that hands out a fixed list of pixels once (a pixel subset of the screen).
template <size_t M>
class ListPaintbrush final : public Paintbrush<M>
{
        std::array<int, M> m_size;
        std::vector<std::array<int_least16_t, M>> m_pixels;
        std::mutex m_lock;
        size_t m_next = 0;
        long long m_pixel_count = 0, m_ray_count = 0, m_sample_count = 0;

public:
        ListPaintbrush(const std::array<int, M>& size, std::vector<std::array<int_least16_t, M>>&& pixels)
                : m_size(size), m_pixels(std::move(pixels))
        {
        }
        void first_pass() noexcept override
        {
        }
        bool next_pixel(int rays, int samples, std::array<int_least16_t, M>* pixel) noexcept override
        {
                std::lock_guard lg(m_lock);
                m_ray_count += rays;
                m_sample_count += samples;
                if (m_next < m_pixels.size())
                {
                        *pixel = m_pixels[m_next++];
                        ++m_pixel_count;
                        return true;
                }
                return false;
        }
        bool next_pass() noexcept override
        {
                return false;
        }
        const std::array<int, M>& screen_size() const noexcept override
        {
                return m_size;
        }
        void statistics(long long* pass_count, long long* pixel_count, long long* ray_count, long long* sample_count,
                        double* previous_pass_duration) const noexcept override
        {
                *pass_count = 1;
                *pixel_count = m_pixel_count;
                *ray_count = m_ray_count;
                *sample_count = m_sample_count;
                *previous_pass_duration = 0;
        }
};

template <size_t M>
class StoreNotifier final : public PainterNotifier<M>
{
        std::array<int, M> m_size;
        float* m_out;
        std::unordered_map<long long, long> m_position;
        bool m_dense;

        long long linear(const std::array<int_least16_t, M>& p) const
        {
                long long idx = 0, stride = 1;
                for (unsigned i = 0; i < M; ++i)
                {
                        idx += stride * p[i];
                        stride *= m_size[i];
                }
                return idx;
        }

public:
        std::string error;

        StoreNotifier(const std::array<int, M>& size, float* out, const std::vector<std::array<int_least16_t, M>>* subset)
                : m_size(size), m_out(out), m_dense(subset == nullptr)
        {
                if (subset)
                {
                        for (size_t i = 0; i < subset->size(); ++i)
                        {
                                m_position[linear((*subset)[i])] = static_cast<long>(i);
                        }
                }
        }
        void painter_pixel_before(const std::array<int_least16_t, M>&) noexcept override
        {
        }
        void painter_pixel_after(const std::array<int_least16_t, M>& pixel, const Color& c) noexcept override
        {
                if (!m_out)
                {
                        return;
                }
                long long idx = m_dense ? linear(pixel) : m_position.at(linear(pixel));
                m_out[idx * 3 + 0] = c.red();
                m_out[idx * 3 + 1] = c.green();
                m_out[idx * 3 + 2] = c.blue();
        }
        void painter_error_message(const std::string& msg) noexcept override
        {
                error = msg;
        }
};

template <size_t N, typename T>
int paint_impl(const refb_scene& s, int spp, int max_depth, unsigned long long seed, int threads, const int* pixels,
               long npix, int bar_height, float* rgb_out, refb_stats* st, char* err, int errlen)
{
        constexpr size_t M = N - 1;
        std::shared_ptr<const Mesh<N, T>> mesh;
        if (s.nfacets > 0)
        {
                std::unique_ptr<MeshHandleBase> h(mesh_create<N, T>(s.verts, s.nverts, s.facets, s.nfacets,
                                                                    std::max(1, s.tree_threads), s.normals, s.nnormals,
                                                                    s.facet_normals));
                mesh = static_cast<MeshHandle<N, T>*>(h.get())->mesh;
        }
        std::shared_ptr<const Mesh<N, T>> mesh2;
        if (s.nfacets2 > 0)
        {
                std::unique_ptr<MeshHandleBase> h(
                        mesh_create<N, T>(s.verts2, s.nverts2, s.facets2, s.nfacets2, std::max(1, s.tree_threads)));
                mesh2 = static_cast<MeshHandle<N, T>*>(h.get())->mesh;
        }
        BridgeScene<N, T> scene(s, mesh, mesh2);

        std::array<int, M> size;
        for (unsigned i = 0; i < M; ++i)
        {
                size[i] = s.screen[i];
        }

        MAX_RECURSION_LEVEL = max_depth;
        g_engine_seed.store(seed);

        std::atomic_bool stop = false;
        std::unique_ptr<Paintbrush<M>> brush;
        std::vector<std::array<int_least16_t, M>> subset;
        std::unique_ptr<StoreNotifier<M>> notifier;
        if (pixels)
        {
                subset.resize(npix);
                for (long i = 0; i < npix; ++i)
                {
                        for (unsigned k = 0; k < M; ++k)
                        {
                                subset[i][k] = static_cast<int_least16_t>(pixels[i * M + k]);
                        }
                }
                notifier = std::make_unique<StoreNotifier<M>>(size, rgb_out, &subset);
                brush = std::make_unique<ListPaintbrush<M>>(size, std::vector(subset));
        }
        else
        {
                notifier = std::make_unique<StoreNotifier<M>>(size, rgb_out, nullptr);
                brush = std::make_unique<VisibleBarPaintbrush<M>>(size, bar_height, 1);
        }

        auto t0 = std::chrono::steady_clock::now();
        paint(notifier.get(), spp, scene, brush.get(), threads, &stop, s.smooth_normal != 0);
        auto t1 = std::chrono::steady_clock::now();

        if (st)
        {
                double prev;
                brush->statistics(&st->pass_count, &st->pixel_count, &st->ray_count, &st->sample_count, &prev);
                st->seconds = std::chrono::duration<double>(t1 - t0).count();
        }
        if (!notifier->error.empty())
        {
                copy_error(notifier->error, err, errlen);
                return 1;
        }
        return 0;
}

template <template <size_t, typename> class F, typename... A>
auto dispatch(int n, int dbl, A&&... a)
{
        switch (n * 2 + (dbl ? 1 : 0))
        {
        case 6:
                return F<3, float>::run(a...);
        case 7:
                return F<3, double>::run(a...);
        case 8:
                return F<4, float>::run(a...);
        case 9:
                return F<4, double>::run(a...);
        case 10:
                return F<5, float>::run(a...);
        case 11:
                return F<5, double>::run(a...);
        case 12:
                return F<6, float>::run(a...);
        default:
                return F<6, double>::run(a...);
        }
}

template <size_t N, typename T>
struct CreateF
{
        static MeshHandleBase* run(const float* v, long nv, const int* f, long nf, int th)
        {
                return mesh_create<N, T>(v, nv, f, nf, th);
        }
};
template <size_t N, typename T>
struct TraceF
{
        static int run(const MeshHandleBase* h, const float* o, const float* d, long nr, int* fo, double* to)
        {
                mesh_trace<N, T>(h, o, d, nr, fo, to);
                return 0;
        }
};
template <size_t N, typename T>
struct InfoF
{
        static int run(const MeshHandleBase* h, long* bc, long* ic, double* dist)
        {
                mesh_tree_info<N, T>(h, bc, ic, dist);
                return 0;
        }
};
template <size_t N, typename T>
struct ExportF
{
        static int run(const MeshHandleBase* h, double* org, double* size, int* ch, long* off, int* idx)
        {
                mesh_tree_export<N, T>(h, org, size, ch, off, idx);
                return 0;
        }
};
template <size_t N, typename T>
struct PaintF
{
        static int run(const refb_scene& s, int spp, int md, unsigned long long seed, int th, const int* px, long np,
                       int bar, float* out, refb_stats* st, char* err, int errlen)
        {
                return paint_impl<N, T>(s, spp, md, seed, th, px, np, bar, out, st, err, errlen);
        }
};

bool valid_n(int n)
{
        return n >= 3 && n <= 6;
}
}

extern "C" {

// Builds Mesh<n, float or double>; returns NULL and fills err on failure.
void* refb_mesh_create(int n, int dbl, const float* verts, long nverts, const int* facets, long nfacets, int threads,
                       char* err, int errlen)
{
        ensure_log();
        if (!valid_n(n))
        {
                copy_error("n must be 3..6", err, errlen);
                return nullptr;
        }
        try
        {
                return dispatch<CreateF>(n, dbl, verts, nverts, facets, nfacets, std::max(1, threads));
        }
        catch (const std::exception& e)
        {
                copy_error(e.what(), err, errlen);
                return nullptr;
        }
}

void refb_mesh_destroy(void* h)
{
        delete static_cast<MeshHandleBase*>(h);
}

// Closest hit of each ray: facet index (-1 = miss) and distance from the ray origin.
int refb_mesh_trace(void* h, const float* org, const float* dir, long nrays, int* facet_out, double* t_out)
{
        const MeshHandleBase* m = static_cast<const MeshHandleBase*>(h);
        return dispatch<TraceF>(m->n, m->dbl, m, org, dir, nrays, facet_out, t_out);
}

int refb_mesh_tree_info(void* h, long* box_count, long* index_count, double* distance_from_facet)
{
        const MeshHandleBase* m = static_cast<const MeshHandleBase*>(h);
        return dispatch<InfoF>(m->n, m->dbl, m, box_count, index_count, distance_from_facet);
}

// org/size: box_count x n; children: box_count x 2^n (-1 = none); index_offset: box_count + 1.
int refb_mesh_tree_export(void* h, double* org, double* size, int* children, long* index_offset, int* indices)
{
        const MeshHandleBase* m = static_cast<const MeshHandleBase*>(h);
        return dispatch<ExportF>(m->n, m->dbl, m, org, size, children, index_offset, indices);
}

// paint<N,T>() on the scene.  pixels == NULL paints the whole screen with the reference's own
// BarPaintbrush (paint height bar_height, one pass) and writes rgb_out densely (x0 fastest);
// otherwise only the listed pixels (npix x (n-1)) are painted and rgb_out follows the list order.
// rgb_out may be NULL (timing only).  max_depth replaces MAX_RECURSION_LEVEL; seed seeds the
// per-thread engines (thread k gets seed + k), so one thread gives a reproducible image.
int refb_paint(const refb_scene* s, int spp, int max_depth, unsigned long long seed, int threads, const int* pixels,
               long npix, int bar_height, float* rgb_out, refb_stats* st, char* err, int errlen)
{
        ensure_log();
        if (!s || !valid_n(s->n))
        {
                copy_error("n must be 3..6", err, errlen);
                return 2;
        }
        try
        {
                return dispatch<PaintF>(s->n, s->dbl, *s, spp, max_depth, seed, std::max(1, threads), pixels, npix,
                                        std::max(1, bar_height), rgb_out, st, err, errlen);
        }
        catch (const std::exception& e)
        {
                copy_error(e.what(), err, errlen);
                return 1;
        }
}
}
