// Header-only C++ drop-in for the reference painter's interface (templeblock/math src/painter),
// running on the B200 library through the C ABI in include/ntrace.h.
//
// The reference's caller builds a PaintObjects<N,T> from visible shapes, lights, a projector and a
// default surface (src/painter/objects.h:141-223) and calls
//     paint<N,T>(notifier, samples_per_pixel, paint_objects, paintbrush, thread_count, stop, smooth_normal)
// (src/painter/painter.h:40-42).  This header keeps those names and that call.  Each visible type
// below exports itself into an nt_scene (the reference builds with -fno-rtti, so the export is a
// virtual function rather than a type switch); paint() builds the scene, renders one pass per
// paintbrush pass on the GPU and hands every pixel's running mean to the notifier in the paintbrush's
// order.  Errors go to painter_error_message, as in the reference (painter.cpp:598-625).
#pragma once

#include "ntrace.h"

#include <array>
#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace ntrace
{
template <std::size_t N, typename T>
using Vector = std::array<T, N>;

struct Color
{
        float r = 0, g = 0, b = 0;
};

// SurfaceProperties subset used by the painter (objects.h:26-133).
struct SurfaceProperties
{
        Color color{1, 1, 1};
        float diffuse = 1;
        bool light_source = false;
        Color light_source_color{};

        nt_surface to_c() const
        {
                return nt_surface{{color.r, color.g, color.b}, diffuse, light_source ? 1 : 0,
                                  {light_source_color.r, light_source_color.g, light_source_color.b}};
        }
};

template <std::size_t N, typename T>
struct GenericObject
{
        virtual ~GenericObject() = default;
        // adds this object to the scene; returns an NT_* status
        virtual int export_to(nt_scene* scene) const = 0;
};

template <std::size_t N, typename T>
struct LightSource
{
        virtual ~LightSource() = default;
        virtual int export_to(nt_scene* scene) const = 0;
};

template <std::size_t N, typename T>
struct Projector
{
        virtual ~Projector() = default;
        virtual const std::array<int, N - 1>& screen_size() const = 0;
        virtual int export_to(nt_scene* scene) const = 0;
};

template <std::size_t N>
struct Paintbrush
{
        virtual ~Paintbrush() = default;
        virtual void first_pass() noexcept = 0;
        virtual bool next_pixel(int previous_pixel_ray_count, int previous_pixel_sample_count,
                                std::array<int_least16_t, N>* pixel) noexcept = 0;
        virtual bool next_pass() noexcept = 0;
        virtual const std::array<int, N>& screen_size() const noexcept = 0;
        virtual void statistics(long long* pass_count, long long* pixel_count, long long* ray_count,
                                long long* sample_count, double* previous_pass_duration) const noexcept = 0;
};

template <std::size_t N, typename T>
struct PaintObjects
{
        virtual ~PaintObjects() = default;
        virtual const std::vector<const GenericObject<N, T>*>& objects() const = 0;
        virtual const std::vector<const LightSource<N, T>*>& light_sources() const = 0;
        virtual const Projector<N, T>& projector() const = 0;
        virtual const SurfaceProperties& default_surface_properties() const = 0;
};

template <std::size_t N>
struct PainterNotifier
{
protected:
        virtual ~PainterNotifier() = default;

public:
        virtual void painter_pixel_before(const std::array<int_least16_t, N>& pixel) noexcept = 0;
        virtual void painter_pixel_after(const std::array<int_least16_t, N>& pixel, const Color& c) noexcept = 0;
        virtual void painter_error_message(const std::string& msg) noexcept = 0;
};

// ---- visible objects (visible_shapes.h) ----

template <std::size_t N, typename T>
class VisibleSharedMesh final : public GenericObject<N, T>, public SurfaceProperties
{
        std::vector<float> m_vertices;
        std::vector<int32_t> m_facets;

public:
        // vertices: N coordinates per vertex; facets: N vertex indices per (N-1)-simplex
        VisibleSharedMesh(const std::vector<Vector<N, T>>& vertices, const std::vector<std::array<int, N>>& facets)
        {
                for (const auto& v : vertices)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                m_vertices.push_back(static_cast<float>(v[k]));
                        }
                }
                for (const auto& f : facets)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                m_facets.push_back(f[k]);
                        }
                }
        }
        int export_to(nt_scene* scene) const override
        {
                nt_surface s = to_c();
                return nt_scene_add_mesh(scene, m_vertices.data(), (int64_t)(m_vertices.size() / N), m_facets.data(),
                                         (int64_t)(m_facets.size() / N), &s);
        }
};

template <std::size_t N, typename T>
class VisibleParallelotope final : public GenericObject<N, T>, public SurfaceProperties
{
        std::array<float, N> m_org;
        std::array<float, N * N> m_edges;

public:
        VisibleParallelotope(const Vector<N, T>& org, const std::array<Vector<N, T>, N>& edges)
        {
                for (std::size_t k = 0; k < N; ++k)
                {
                        m_org[k] = static_cast<float>(org[k]);
                        for (std::size_t i = 0; i < N; ++i)
                        {
                                m_edges[i * N + k] = static_cast<float>(edges[i][k]);
                        }
                }
        }
        int export_to(nt_scene* scene) const override
        {
                nt_surface s = to_c();
                return nt_scene_add_parallelotope(scene, m_org.data(), m_edges.data(), &s);
        }
};

template <std::size_t N, typename T>
class VisibleHyperplaneParallelotope final : public GenericObject<N, T>, public SurfaceProperties
{
        std::array<float, N> m_org;
        std::array<float, (N - 1) * N> m_edges;

public:
        VisibleHyperplaneParallelotope(const Vector<N, T>& org, const std::array<Vector<N, T>, N - 1>& edges)
        {
                for (std::size_t k = 0; k < N; ++k)
                {
                        m_org[k] = static_cast<float>(org[k]);
                        for (std::size_t i = 0; i + 1 < N; ++i)
                        {
                                m_edges[i * N + k] = static_cast<float>(edges[i][k]);
                        }
                }
        }
        int export_to(nt_scene* scene) const override
        {
                nt_surface s = to_c();
                return nt_scene_add_hyperplane_parallelotope(scene, m_org.data(), m_edges.data(), &s);
        }
};

// ---- lights (visible_lights.h) ----

template <std::size_t N, typename T>
class VisiblePointLight final : public LightSource<N, T>
{
        std::array<float, N> m_location;
        std::array<float, 3> m_color;
        float m_unit;

public:
        VisiblePointLight(const Vector<N, T>& location, const Color& color, T unit_intensity_distance)
                : m_color{color.r, color.g, color.b}, m_unit(static_cast<float>(unit_intensity_distance))
        {
                for (std::size_t k = 0; k < N; ++k)
                {
                        m_location[k] = static_cast<float>(location[k]);
                }
        }
        int export_to(nt_scene* scene) const override
        {
                return nt_scene_add_point_light(scene, m_location.data(), m_color.data(), m_unit);
        }
};

template <std::size_t N, typename T>
class VisibleConstantLight final : public LightSource<N, T>
{
        std::array<float, N> m_location;
        std::array<float, 3> m_color;

public:
        VisibleConstantLight(const Vector<N, T>& location, const Color& color) : m_color{color.r, color.g, color.b}
        {
                for (std::size_t k = 0; k < N; ++k)
                {
                        m_location[k] = static_cast<float>(location[k]);
                }
        }
        int export_to(nt_scene* scene) const override
        {
                return nt_scene_add_constant_light(scene, m_location.data(), m_color.data());
        }
};

// ---- projectors (visible_projectors.h) ----

template <std::size_t N, typename T, int KIND>
class VisibleProjector final : public Projector<N, T>
{
        std::array<float, N> m_org, m_dir;
        std::array<float, (N - 1) * N> m_axes;
        float m_param;
        std::array<int, N - 1> m_screen;

public:
        VisibleProjector(const Vector<N, T>& camera_org, const Vector<N, T>& camera_dir,
                         const std::array<Vector<N, T>, N - 1>& screen_axes, T param, const std::array<int, N - 1>& screen_size)
                : m_param(static_cast<float>(param)), m_screen(screen_size)
        {
                for (std::size_t k = 0; k < N; ++k)
                {
                        m_org[k] = static_cast<float>(camera_org[k]);
                        m_dir[k] = static_cast<float>(camera_dir[k]);
                        for (std::size_t i = 0; i + 1 < N; ++i)
                        {
                                m_axes[i * N + k] = static_cast<float>(screen_axes[i][k]);
                        }
                }
        }
        const std::array<int, N - 1>& screen_size() const override
        {
                return m_screen;
        }
        int export_to(nt_scene* scene) const override
        {
                return nt_scene_set_projector(scene, KIND, m_org.data(), m_dir.data(), m_axes.data(), m_param,
                                              m_screen.data());
        }
};

template <std::size_t N, typename T>
using VisibleParallelProjector = VisibleProjector<N, T, NT_PROJECTOR_PARALLEL>;
template <std::size_t N, typename T>
using VisiblePerspectiveProjector = VisibleProjector<N, T, NT_PROJECTOR_PERSPECTIVE>;
template <std::size_t N, typename T>
using VisibleSphericalProjector = VisibleProjector<N, T, NT_PROJECTOR_SPHERICAL>;

// ---- a paintbrush visiting every pixel once per pass, x0 fastest (BarPaintbrush, paintbrush.h) ----

template <std::size_t M>
class VisibleBarPaintbrush final : public Paintbrush<M>
{
        std::array<int, M> m_size;
        int m_max_pass_count;
        long long m_next = 0;
        long long m_total = 1;
        long long m_pass_count = 1, m_pixel_count = 0, m_ray_count = 0, m_sample_count = 0;
        mutable std::mutex m_lock;

public:
        // max_pass_count: -1 = unlimited (paintbrush.h:129-132)
        VisibleBarPaintbrush(const std::array<int, M>& screen_size, int max_pass_count)
                : m_size(screen_size), m_max_pass_count(max_pass_count)
        {
                for (int s : m_size)
                {
                        m_total *= s;
                }
        }
        void first_pass() noexcept override
        {
        }
        bool next_pixel(int rays, int samples, std::array<int_least16_t, M>* pixel) noexcept override
        {
                std::lock_guard lg(m_lock);
                m_ray_count += rays;
                m_sample_count += samples;
                if (m_next >= m_total)
                {
                        return false;
                }
                long long rem = m_next++;
                for (std::size_t j = 0; j < M; ++j)
                {
                        (*pixel)[j] = static_cast<int_least16_t>(rem % m_size[j]);
                        rem /= m_size[j];
                }
                ++m_pixel_count;
                return true;
        }
        bool next_pass() noexcept override
        {
                std::lock_guard lg(m_lock);
                m_next = 0;
                if (m_pass_count == m_max_pass_count)
                {
                        return false;
                }
                ++m_pass_count;
                return true;
        }
        const std::array<int, M>& screen_size() const noexcept override
        {
                return m_size;
        }
        void statistics(long long* pass_count, long long* pixel_count, long long* ray_count, long long* sample_count,
                        double* previous_pass_duration) const noexcept override
        {
                std::lock_guard lg(m_lock);
                *pass_count = m_pass_count;
                *pixel_count = m_pixel_count;
                *ray_count = m_ray_count;
                *sample_count = m_sample_count;
                *previous_pass_duration = 0;
        }
};

// Recursion cap used by paint() (MAX_RECURSION_LEVEL, painter.cpp:42).
inline int& paint_max_depth()
{
        static int depth = 100;
        return depth;
}

// paint<N,T> (painter.h:40-42).  thread_count must be positive, as in the reference
// (check_thread_count, painter.cpp:521-527); the GPU does not use it.
template <std::size_t N, typename T>
void paint(PainterNotifier<N - 1>* notifier, int samples_per_pixel, const PaintObjects<N, T>& paint_objects,
           Paintbrush<N - 1>* paintbrush, int thread_count, std::atomic_bool* stop, bool smooth_normal) noexcept
{
        nt_scene* scene = nullptr;
        auto report = [&](const std::string& what) {
                notifier->painter_error_message("Painter error:\n" + what + ": " + nt_last_error_message());
        };
        try
        {
                if (thread_count < 1)
                {
                        notifier->painter_error_message("Painter error:\nPainter thread count (" + std::to_string(thread_count) +
                                                        ") must be greater than 0");
                        return;
                }
                if (paintbrush->screen_size() != paint_objects.projector().screen_size())
                {
                        notifier->painter_error_message(
                                "Painter error:\nThe paintbrush screen size is not equal to the projector screen size");
                        return;
                }
                if (nt_scene_create((int)N, &scene) != NT_OK)
                {
                        report("scene");
                        return;
                }
                std::unique_ptr<nt_scene, int (*)(nt_scene*)> guard(scene, nt_scene_destroy);
                for (const GenericObject<N, T>* o : paint_objects.objects())
                {
                        if (o->export_to(scene) != NT_OK)
                        {
                                report("object");
                                return;
                        }
                }
                for (const LightSource<N, T>* l : paint_objects.light_sources())
                {
                        if (l->export_to(scene) != NT_OK)
                        {
                                report("light source");
                                return;
                        }
                }
                nt_surface bg = paint_objects.default_surface_properties().to_c();
                if (paint_objects.projector().export_to(scene) != NT_OK || nt_scene_set_background(scene, &bg) != NT_OK)
                {
                        report("projector");
                        return;
                }
                nt_build_opts bopts{0, 0};
                if (nt_scene_build(scene, &bopts) != NT_OK)
                {
                        report("build");
                        return;
                }
                const int64_t npix = nt_scene_pixel_count(scene);
                std::vector<float> rgb((std::size_t)npix * 3);
                std::array<int, N - 1> size = paintbrush->screen_size();
                volatile int stop_flag = 0;
                nt_render_opts opts{};
                opts.samples_per_pixel = samples_per_pixel;
                opts.max_depth = paint_max_depth();
                opts.seed = 0;
                opts.retest = 1;
                opts.smooth_normal = smooth_normal ? 1 : 0;
                opts.stop = &stop_flag;
                paintbrush->first_pass();
                do
                {
                        stop_flag = stop->load() ? 1 : 0;
                        nt_stats st{};
                        int code = nt_render(scene, &opts, &st);
                        if (code == NT_ESTOPPED)
                        {
                                return;
                        }
                        if (code != NT_OK || nt_accum_read(scene, rgb.data(), nullptr) != NT_OK)
                        {
                                report("render");
                                return;
                        }
                        std::array<int_least16_t, N - 1> pixel;
                        long long rays_per_pixel = npix > 0 ? st.rays / npix : 0;
                        while (!*stop && paintbrush->next_pixel((int)rays_per_pixel, st.spp_effective, &pixel))
                        {
                                notifier->painter_pixel_before(pixel);
                                long long idx = 0, stride = 1;
                                for (std::size_t j = 0; j < N - 1; ++j)
                                {
                                        idx += stride * pixel[j];
                                        stride *= size[j];
                                }
                                notifier->painter_pixel_after(pixel, Color{rgb[3 * idx], rgb[3 * idx + 1], rgb[3 * idx + 2]});
                        }
                } while (!*stop && paintbrush->next_pass());
        }
        catch (const std::exception& e)
        {
                notifier->painter_error_message(std::string("Painter error:\n") + e.what());
        }
        catch (...)
        {
                notifier->painter_error_message("Unknown painter error");
        }
}
}
