// Test program for math_b200/paint.hpp: paints a floor scene with the reference-style interface
// (PaintObjects, VisibleSharedMesh, VisibleParallelotope, VisiblePointLight, VisibleParallelProjector,
// BarPaintbrush, PainterNotifier) and writes the final image.
//
// usage: paint_dropin <mesh.bin> <out.bin> <screen> <spp> <max_depth> <passes>
//   mesh.bin: int32 vertex_count, int32 facet_count, float32 vertices (x3), int32 facets (x3)
//   out.bin:  float32 rgb per pixel (x0 fastest) after the last pass
#include "../../math_b200/paint.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace ntrace;

namespace
{
class Scene final : public PaintObjects<3, float>
{
        std::vector<std::unique_ptr<GenericObject<3, float>>> m_owned;
        std::vector<const GenericObject<3, float>*> m_objects;
        std::unique_ptr<LightSource<3, float>> m_light;
        std::vector<const LightSource<3, float>*> m_lights;
        std::unique_ptr<Projector<3, float>> m_projector;
        SurfaceProperties m_background;

public:
        Scene(const std::vector<Vector<3, float>>& v, const std::vector<std::array<int, 3>>& f, int screen)
        {
                auto mesh = std::make_unique<VisibleSharedMesh<3, float>>(v, f);
                mesh->color = Color{0.7f, 0.7f, 0.7f};
                mesh->diffuse = 1;
                auto floor = std::make_unique<VisibleParallelotope<3, float>>(
                        Vector<3, float>{-4, -4, -1.1f},
                        std::array<Vector<3, float>, 3>{Vector<3, float>{8, 0, 0}, Vector<3, float>{0, 8, 0},
                                                        Vector<3, float>{0, 0, 0.1f}});
                floor->color = Color{0.7f, 0.7f, 0.7f};
                floor->diffuse = 1;
                m_objects = {mesh.get(), floor.get()};
                m_owned.push_back(std::move(mesh));
                m_owned.push_back(std::move(floor));
                const float unit = (float)std::sqrt(17.0);  // |(2, 2, 3)|: irradiance 1 at the origin
                m_light = std::make_unique<VisiblePointLight<3, float>>(Vector<3, float>{2, 2, 3}, Color{1, 1, 1}, unit);
                m_lights = {m_light.get()};
                m_projector = std::make_unique<VisibleParallelProjector<3, float>>(
                        Vector<3, float>{0, 0, 10}, Vector<3, float>{0, 0, -1},
                        std::array<Vector<3, float>, 2>{Vector<3, float>{1, 0, 0}, Vector<3, float>{0, 1, 0}},
                        8.0f / screen, std::array<int, 2>{screen, screen});
                m_background.color = Color{0.30f, 0.35f, 0.40f};
                m_background.light_source = true;
                m_background.light_source_color = Color{0.343f, 0.343f, 0.343f};
        }
        const std::vector<const GenericObject<3, float>*>& objects() const override
        {
                return m_objects;
        }
        const std::vector<const LightSource<3, float>*>& light_sources() const override
        {
                return m_lights;
        }
        const Projector<3, float>& projector() const override
        {
                return *m_projector;
        }
        const SurfaceProperties& default_surface_properties() const override
        {
                return m_background;
        }
};

class Store final : public PainterNotifier<2>
{
        int m_width;

public:
        std::vector<float> rgb;
        std::string error;
        explicit Store(int width) : m_width(width), rgb((std::size_t)width * width * 3)
        {
        }
        void painter_pixel_before(const std::array<int_least16_t, 2>&) noexcept override
        {
        }
        void painter_pixel_after(const std::array<int_least16_t, 2>& p, const Color& c) noexcept override
        {
                std::size_t i = (std::size_t)p[0] + (std::size_t)p[1] * m_width;
                rgb[3 * i] = c.r;
                rgb[3 * i + 1] = c.g;
                rgb[3 * i + 2] = c.b;
        }
        void painter_error_message(const std::string& msg) noexcept override
        {
                error = msg;
        }
};
}

int main(int argc, char** argv)
{
        if (argc != 7)
        {
                std::fprintf(stderr, "usage: paint_dropin mesh.bin out.bin screen spp max_depth passes\n");
                return 2;
        }
        FILE* in = std::fopen(argv[1], "rb");
        if (!in)
        {
                return 2;
        }
        int32_t nv = 0, nf = 0;
        if (std::fread(&nv, 4, 1, in) != 1 || std::fread(&nf, 4, 1, in) != 1)
        {
                return 2;
        }
        std::vector<Vector<3, float>> v(nv);
        std::vector<std::array<int, 3>> f(nf);
        if (std::fread(v.data(), sizeof(float) * 3, nv, in) != (size_t)nv ||
            std::fread(f.data(), sizeof(int) * 3, nf, in) != (size_t)nf)
        {
                return 2;
        }
        std::fclose(in);
        const int screen = std::atoi(argv[3]);
        const int spp = std::atoi(argv[4]);
        paint_max_depth() = std::atoi(argv[5]);
        const int passes = std::atoi(argv[6]);
        Scene scene(v, f, screen);
        Store store(screen);
        VisibleBarPaintbrush<2> brush({screen, screen}, passes);
        std::atomic_bool stop = false;
        paint<3, float>(&store, spp, scene, &brush, 1, &stop, false);
        if (!store.error.empty())
        {
                std::fprintf(stderr, "%s\n", store.error.c_str());
                return 1;
        }
        long long pass_count, pixel_count, ray_count, sample_count;
        double dur;
        brush.statistics(&pass_count, &pixel_count, &ray_count, &sample_count, &dur);
        std::printf("passes %lld pixels %lld samples %lld\n", pass_count, pixel_count, sample_count);
        FILE* out = std::fopen(argv[2], "wb");
        std::fwrite(store.rgb.data(), sizeof(float), store.rgb.size(), out);
        std::fclose(out);
        return 0;
}
