/*
 * CPU test oracle: a C-ABI driver around the reference painter.
 *
 * This file is test infrastructure.  It is compiled together with the
 * reference's own sources (see Makefile) into oracle/_ref/libnbpt_oracle.so,
 * which the tests, the golden-fixture generator and bench.py's CPU baseline
 * load through ctypes.  Nothing in the accelerated library links it.
 *
 * Everything here calls the reference's public constructors and functions:
 *   scenes   shapes::HyperplaneParallelotope / Parallelotope / create_mesh,
 *            lights::ParallelotopeLight / BallLight, projectors::Perspective/
 *            ParallelProjector, scenes::create_storage_scene
 *            (src/painter/scenes/storage.h:40-47, shapes/*.h, lights/*.h)
 *   render   integrators::bpt::bpt (src/painter/integrators/bpt/bpt.h:31-36)
 *            with per-path seeded PCG streams, and pixels::Pixels for the
 *            filtered, trimmed image (src/painter/pixels/pixels.cpp:69-166)
 *   baseline painter::create_painter, unmodified (src/painter/painter.h:149-157)
 *   geometry the mesh BVH and facet records the mesh shape builds
 *            (src/painter/shapes/mesh.cpp:172-210, mesh/data.cpp:277-310)
 *
 * Random streams.  The reference seeds one PCG per worker thread from the OS
 * (src/painter/painting/integrator_bpt.cpp:130), so its images are not
 * reproducible.  This driver gives every pixel and every path its own stream,
 * seeded through std::seed_seq (src/com/random/pcg.cpp:84-87):
 *     stratified sub-pixel points of pixel p in pass k: seed_seq{seed, k, p, 0}
 *     path i of pixel p in pass k:                      seed_seq{seed, k, p, i+1}
 * The accelerated library derives the same streams, so the two compute the
 * same paths sample for sample.
 */

#include <src/color/color.h>
#include <src/color/samples/rgb_samples.h>
#include <src/color/samples/xyz_samples.h>
#include <src/com/random/pcg.h>
#include <src/geometry/accelerators/bvh.h>
#include <src/geometry/accelerators/bvh_object.h>
#include <src/geometry/spatial/bounding_box.h>
#include <src/geometry/spatial/hyperplane_parallelotope.h>
#include <src/geometry/spatial/hyperplane_simplex.h>
#include <src/geometry/spatial/parallelotope.h>
#include <src/geometry/spatial/ray_intersection.h>
#include <src/geometry/shapes/ball_volume.h>
#include <src/geometry/shapes/sphere_integral.h>
#include <src/geometry/spatial/point_offset.h>
#include <src/sampling/sphere_cosine.h>
#include <src/sampling/sphere_uniform.h>
#include <src/image/image.h>
#include <src/model/mesh.h>
#include <src/model/mesh/create_facets.h>
#include <src/model/mesh/file/load_obj.h>
#include <src/model/mesh/file/load_stl.h>
#include <src/model/mesh_object.h>
#include <src/numerical/matrix.h>
#include <src/numerical/ray.h>
#include <src/numerical/vector.h>
#include <src/painter/integrators/bpt/bpt.h>
#include <src/painter/integrators/bpt/light_distribution.h>
#include <src/painter/integrators/pt/pt.h>
#include <src/painter/lights/ball_light.h>
#include <src/painter/lights/parallelotope_light.h>
#include <src/painter/objects.h>
#include <src/painter/painter.h>
#include <src/painter/painting/sampler.h>
#include <src/painter/pixels/pixels.h>
#include <src/painter/projectors/parallel_projector.h>
#include <src/painter/projectors/perspective_projector.h>
#include <src/painter/scenes/storage.h>
#include <src/painter/shapes/hyperplane_parallelotope.h>
#include <src/painter/shapes/mesh.h>
#include <src/painter/shapes/mesh/data.h>
#include <src/painter/shapes/parallelotope.h>
#include <src/progress/progress.h>
#include <src/shading/ggx/brdf.h>
#include <src/shading/ggx/f1_albedo.h>
#include <src/shading/ggx/metalness.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <memory>
#include <optional>
#include <random>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

// Path depth of bpt(): the build-time copy of bpt.cpp reads this variable
// instead of its compile-time MAX_DEPTH = 5 (src/painter/integrators/bpt/bpt.cpp:58).
int nbpt_oracle_max_depth = 5;

namespace
{
namespace painter = ns::painter;
namespace numerical = ns::numerical;
namespace spatial = ns::geometry::spatial;
namespace accelerators = ns::geometry::accelerators;

thread_local std::string g_last_error;

// ---------------------------------------------------------------------------
// Read access to private members the reference has no accessor for (the BVH
// arrays and the simplex plane records).  Explicit instantiation may name
// private members; the friend function it defines hands out the pointer.

template <typename Tag, typename Tag::type MEMBER>
struct Expose final
{
        friend typename Tag::type member_pointer(Tag)
        {
                return MEMBER;
        }
};

template <std::size_t N, typename T>
struct BvhNodesTag final
{
        using type = std::vector<accelerators::bvh_implementation::Node<N, T>> accelerators::Bvh<N, T>::*;
        friend type member_pointer(BvhNodesTag);
};

template <std::size_t N, typename T>
struct BvhIndicesTag final
{
        using type = std::vector<unsigned> accelerators::Bvh<N, T>::*;
        friend type member_pointer(BvhIndicesTag);
};

template <std::size_t N, typename T>
struct SimplexPlaneTag final
{
        using type = spatial::Hyperplane<N, T> spatial::HyperplaneSimplex<N, T>::*;
        friend type member_pointer(SimplexPlaneTag);
};

template <std::size_t N, typename T>
struct SimplexPlanesTag final
{
        using type = std::array<spatial::Hyperplane<N, T>, N - 1> spatial::HyperplaneSimplex<N, T>::*;
        friend type member_pointer(SimplexPlanesTag);
};

template <typename Derived, std::size_t K>
struct SamplesDataTag final
{
        using type = numerical::Vector<K, float> ns::color::Samples<Derived, K, float>::*;
        friend type member_pointer(SamplesDataTag);
};

template struct Expose<SamplesDataTag<ns::color::Color, 3>, &ns::color::Samples<ns::color::Color, 3, float>::data_>;
template struct Expose<
        SamplesDataTag<ns::color::Spectrum, 64>,
        &ns::color::Samples<ns::color::Spectrum, 64, float>::data_>;

#define NBPT_EXPOSE(N, T)                                                                                  \
        template struct Expose<BvhNodesTag<N, T>, &accelerators::Bvh<N, T>::nodes_>;                       \
        template struct Expose<BvhIndicesTag<N, T>, &accelerators::Bvh<N, T>::object_indices_>;            \
        template struct Expose<SimplexPlaneTag<N, T>, &spatial::HyperplaneSimplex<N, T>::plane_>;          \
        template struct Expose<SimplexPlanesTag<N, T>, &spatial::HyperplaneSimplex<N, T>::planes_>;

NBPT_EXPOSE(3, float)
NBPT_EXPOSE(3, double)
NBPT_EXPOSE(4, float)
NBPT_EXPOSE(4, double)
NBPT_EXPOSE(5, float)
NBPT_EXPOSE(5, double)

// The facet's simplex is a private member too, but Facet::intersect() and
// geometric_normal() are public; the simplex is rebuilt from the facet's
// vertices with the same constructor instead (the records are then identical
// because the constructor is deterministic).

// ---------------------------------------------------------------------------

template <std::size_t M>
class CollectNotifier final : public painter::Notifier<M>
{
        painter::Images<M> images_;

public:
        void thread_busy(unsigned, const std::array<int, M>&) override
        {
        }
        void thread_free(unsigned) override
        {
        }
        void pixel_set(const std::array<int, M>&, const numerical::Vector<3, float>&) override
        {
        }
        painter::Images<M>* images(long long) override
        {
                return &images_;
        }
        void pass_done(long long) override
        {
        }
        void error_message(const std::string& msg) override
        {
                error = msg;
        }

        std::string error;

        void copy_rgb(float* const out) const
        {
                const painter::ImagesReading<M> lock(&images_);
                const auto& image = lock.image_with_background();
                std::memcpy(out, image.pixels.data(), image.pixels.size());
        }

        void copy_rgba(float* const out) const
        {
                const painter::ImagesReading<M> lock(&images_);
                const auto& image = lock.image_without_background();
                std::memcpy(out, image.pixels.data(), image.pixels.size());
        }
};

std::unique_ptr<ns::PCG> make_engine(const std::initializer_list<std::uint32_t> words)
{
        std::seed_seq seq(words);
        return std::make_unique<ns::PCG>(seq);
}

template <typename Color>
Color surface_color(const float* const rgb)
{
        return Color(rgb[0], rgb[1], rgb[2]);
}

template <typename Color>
Color light_color(const float* const rgb)
{
        return Color::illuminant(rgb[0], rgb[1], rgb[2]);
}

template <typename Color>
constexpr int channels()
{
        if constexpr (std::is_same_v<Color, ns::color::Spectrum>)
        {
                return 64;
        }
        else
        {
                return 3;
        }
}

// Channel k of a colour (3 for RGB, 64 for Spectrum).
template <typename Color>
float& channel(Color& c, const int k)
{
        constexpr std::size_t K = channels<Color>();
        using Base = ns::color::Samples<Color, K, float>;
        return (static_cast<Base&>(c).*member_pointer(SamplesDataTag<Color, K>{}))[k];
}

template <typename Color>
float channel(const Color& c, const int k)
{
        return channel(const_cast<Color&>(c), k);
}

template <std::size_t N, typename T>
numerical::Vector<N, T> vec(const double* const p)
{
        numerical::Vector<N, T> v;
        for (std::size_t i = 0; i < N; ++i)
        {
                v[i] = p[i];
        }
        return v;
}

template <std::size_t N, typename T, std::size_t M>
std::array<numerical::Vector<N, T>, M> vecs(const double* const p)
{
        std::array<numerical::Vector<N, T>, M> res;
        for (std::size_t i = 0; i < M; ++i)
        {
                res[i] = vec<N, T>(p + i * N);
        }
        return res;
}

template <std::size_t M>
std::array<int, M> pixel_of(long long index, const std::array<int, M>& size)
{
        std::array<int, M> res;
        for (std::size_t i = 0; i < M; ++i)
        {
                res[i] = index % size[i];
                index /= size[i];
        }
        return res;
}

template <typename F>
void parallel_for(const long long count, int threads, const F& f)
{
        threads = std::max(1, threads);
        std::atomic<long long> next = 0;
        std::vector<std::thread> pool;
        std::exception_ptr failure;
        std::atomic_bool failed = false;
        for (int t = 0; t < threads; ++t)
        {
                pool.emplace_back(
                        [&]
                        {
                                try
                                {
                                        while (!failed)
                                        {
                                                const long long i = next.fetch_add(64);
                                                if (i >= count)
                                                {
                                                        break;
                                                }
                                                const long long end = std::min(count, i + 64);
                                                for (long long k = i; k < end; ++k)
                                                {
                                                        f(k);
                                                }
                                        }
                                }
                                catch (...)
                                {
                                        if (!failed.exchange(true))
                                        {
                                                failure = std::current_exception();
                                        }
                                }
                        });
        }
        for (std::thread& t : pool)
        {
                t.join();
        }
        if (failure)
        {
                std::rethrow_exception(failure);
        }
}

// ---------------------------------------------------------------------------

struct SceneBase
{
        virtual ~SceneBase() = default;

        virtual int dimension() const = 0;
        virtual int add_hyperplane_parallelotope(double, double, const float*, double, const double*, const double*) = 0;
        virtual int add_parallelotope(double, double, const float*, double, const double*, const double*) = 0;
        virtual int add_mesh_object(const float*, long, const int*, long, const double*, double, double, const float*, double) = 0;
        virtual int add_mesh_file(const char*, const double*, double, double, const float*, double) = 0;
        virtual int add_mesh() = 0;
        virtual int add_parallelotope_light(int, const double*, const float*) = 0;
        virtual int add_ball_light(const double*, const double*, double, const float*) = 0;
        virtual void set_perspective(const double*, const double*, const double*, double, const int*) = 0;
        virtual void set_parallel(const double*, const double*, const double*, double, const int*) = 0;
        virtual void finalize(const float*) = 0;
        virtual long long pixel_count() const = 0;
        virtual int actual_spp(int) const = 0;
        virtual void set_integrator(int) = 0;
        virtual void set_flat_shading(bool) = 0;
        virtual void render_samples(int, int, unsigned, unsigned, long long, long long, int, double*, float*, unsigned char*) = 0;
        virtual void render_image(int, int, unsigned, int, int, long long, long long, float*, float*) = 0;
        virtual void paint(int, int, int, int, double*, float*) = 0;
        virtual void mesh_info(int, long long*) = 0;
        virtual void mesh_dump(int, double*, double*, int*, int*, double*, float*, double*, double*, unsigned*, unsigned*) = 0;
        virtual void mesh_trace(int, const double*, long long, double, int, int*, double*, unsigned char*, int) = 0;
        virtual void scene_trace(const double*, long long, int, double*, double*, double*, unsigned char*) = 0;
        virtual void brdf(double, double, const float*, const double*, const double*, const double*, float*, double*) = 0;
        virtual void brdf_sample(double, double, const float*, const double*, const double*, const unsigned*, int, double*, double*, float*) = 0;
        virtual void light_sample(int, int, const unsigned*, int, const double*, const double*, double*, float*) = 0;
};

template <std::size_t N, typename T, typename Color>
class Scene final : public SceneBase
{
        static constexpr int C = channels<Color>();

        using Shape = painter::Shape<N, T, Color>;
        using Light = painter::LightSource<N, T, Color>;

        struct MeshRecord final
        {
                int shape_index;
                std::vector<std::unique_ptr<ns::model::mesh::MeshObject<N>>> objects;
                painter::shapes::mesh::MeshData<N, T, Color> data;
                std::unique_ptr<accelerators::Bvh<N, T>> bvh;
        };

        std::vector<std::unique_ptr<Shape>> pending_shapes_;
        std::vector<painter::shapes::HyperplaneParallelotope<N, T, Color>*> flat_shapes_;
        std::vector<std::unique_ptr<Light>> pending_lights_;
        std::unique_ptr<painter::Projector<N, T>> projector_;
        std::vector<std::unique_ptr<ns::model::mesh::MeshObject<N>>> mesh_objects_;
        std::vector<MeshRecord> meshes_;
        std::optional<painter::scenes::StorageScene<N, T, Color>> storage_;
        ns::progress::Ratio progress_{nullptr};

        const painter::Scene<N, T, Color>& scene() const
        {
                if (!storage_)
                {
                        throw std::runtime_error("scene is not finalized");
                }
                return *storage_->scene;
        }

        MeshRecord& mesh(const int shape)
        {
                for (MeshRecord& m : meshes_)
                {
                        if (m.shape_index == shape)
                        {
                                return m;
                        }
                }
                throw std::runtime_error("shape " + std::to_string(shape) + " is not a mesh");
        }

        int push_shape(std::unique_ptr<Shape>&& shape)
        {
                if (storage_)
                {
                        throw std::runtime_error("scene is finalized");
                }
                pending_shapes_.push_back(std::move(shape));
                return pending_shapes_.size() - 1;
        }

public:
        int dimension() const override
        {
                return N;
        }

        int add_hyperplane_parallelotope(
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double alpha,
                const double* const org,
                const double* const vectors) override
        {
                auto shape = std::make_unique<painter::shapes::HyperplaneParallelotope<N, T, Color>>(
                        metalness, roughness, surface_color<Color>(rgb), alpha, vec<N, T>(org),
                        vecs<N, T, N - 1>(vectors));
                auto* const raw = shape.get();
                const int index = push_shape(std::move(shape));
                flat_shapes_.resize(pending_shapes_.size(), nullptr);
                flat_shapes_[index] = raw;
                return index;
        }

        int add_parallelotope(
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double alpha,
                const double* const org,
                const double* const vectors) override
        {
                return push_shape(
                        std::make_unique<painter::shapes::Parallelotope<N, T, Color>>(
                                metalness, roughness, surface_color<Color>(rgb), alpha, vec<N, T>(org),
                                vecs<N, T, N>(vectors)));
        }

        int add_mesh_object(
                const float* const points,
                const long n_points,
                const int* const facets,
                const long n_facets,
                const double* const matrix,
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double alpha) override
        {
                std::vector<numerical::Vector<N, float>> p(n_points);
                for (long i = 0; i < n_points; ++i)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                p[i][k] = points[i * N + k];
                        }
                }
                std::vector<std::array<int, N>> f(n_facets);
                for (long i = 0; i < n_facets; ++i)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                f[i][k] = facets[i * N + k];
                        }
                }
                numerical::Matrix<N + 1, N + 1, double> m;
                for (std::size_t r = 0; r < N + 1; ++r)
                {
                        for (std::size_t c = 0; c < N + 1; ++c)
                        {
                                m.row(r)[c] = matrix[r * (N + 1) + c];
                        }
                }
                auto object = std::make_unique<ns::model::mesh::MeshObject<N>>(
                        ns::model::mesh::create_mesh_for_facets(p, f, /*write_log=*/false), m, "oracle");
                {
                        ns::model::mesh::Writing<N> writing(object.get());
                        writing.set_metalness(metalness);
                        writing.set_roughness(roughness);
                        writing.set_alpha(alpha);
                        writing.set_color(ns::color::Color(rgb[0], rgb[1], rgb[2]));
                }
                mesh_objects_.push_back(std::move(object));
                return mesh_objects_.size() - 1;
        }

        // model::mesh::load (src/model/mesh/file.cpp:86-104) of an OBJ or STL file
        // of this dimension, as one mesh object
        int add_mesh_file(
                const char* const path,
                const double* const matrix,
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double alpha) override
        {
                const std::filesystem::path file(path);
                std::string ext = file.extension().string();
                for (char& c : ext)
                {
                        c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
                }
                const std::string n_text = N == 3 ? "" : std::to_string(N);
                std::unique_ptr<ns::model::mesh::Mesh<N>> mesh;
                if (ext == ".obj" + n_text || (N == 3 && ext == ".obj3"))
                {
                        mesh = ns::model::mesh::file::load_from_obj_file<N>(file, &progress_);
                }
                else if (ext == ".stl" + n_text || (N == 3 && ext == ".stl3"))
                {
                        mesh = ns::model::mesh::file::load_from_stl_file<N>(file, &progress_, false);
                }
                else
                {
                        throw std::runtime_error("not an OBJ or STL file of this dimension: " + file.string());
                }
                numerical::Matrix<N + 1, N + 1, double> m;
                for (std::size_t r = 0; r < N + 1; ++r)
                {
                        for (std::size_t c = 0; c < N + 1; ++c)
                        {
                                m.row(r)[c] = matrix[r * (N + 1) + c];
                        }
                }
                auto object = std::make_unique<ns::model::mesh::MeshObject<N>>(std::move(mesh), m, "oracle");
                {
                        ns::model::mesh::Writing<N> writing(object.get());
                        writing.set_metalness(metalness);
                        writing.set_roughness(roughness);
                        writing.set_alpha(alpha);
                        writing.set_color(ns::color::Color(rgb[0], rgb[1], rgb[2]));
                }
                mesh_objects_.push_back(std::move(object));
                return mesh_objects_.size() - 1;
        }

        int add_mesh() override
        {
                if (mesh_objects_.empty())
                {
                        throw std::runtime_error("no mesh objects");
                }
                std::vector<const ns::model::mesh::MeshObject<N>*> objects;
                for (const auto& o : mesh_objects_)
                {
                        objects.push_back(o.get());
                }

                MeshRecord record;
                record.data = painter::shapes::mesh::create_mesh_data<N, T, Color>(objects, std::nullopt, false);

                // The same objects the mesh shape builds its BVH from
                // (src/painter/shapes/mesh.cpp:172-188).
                std::vector<accelerators::BvhObject<N, T>> bvh_objects;
                bvh_objects.reserve(record.data.mesh.facets.size());
                for (std::size_t i = 0; i < record.data.mesh.facets.size(); ++i)
                {
                        bvh_objects.emplace_back(
                                spatial::BoundingBox<N, T>(
                                        record.data.mesh.vertices, record.data.facet_vertex_indices[i]),
                                record.data.mesh.facets[i].intersection_cost(), i);
                }
                record.bvh = std::make_unique<accelerators::Bvh<N, T>>(std::move(bvh_objects), &progress_);

                const int index = push_shape(
                        painter::shapes::create_mesh<N, T, Color>(objects, std::nullopt, false, &progress_));
                record.shape_index = index;
                record.objects = std::move(mesh_objects_);
                mesh_objects_.clear();
                meshes_.push_back(std::move(record));
                return index;
        }

        int add_parallelotope_light(const int shape, const double* const direction, const float* const rgb) override
        {
                if (shape < 0 || shape >= static_cast<int>(flat_shapes_.size()) || !flat_shapes_[shape])
                {
                        throw std::runtime_error("light carrier is not a hyperplane parallelotope");
                }
                auto light = std::make_unique<painter::lights::ParallelotopeLight<N, T, Color>>(
                        flat_shapes_[shape]->hyperplane_parallelotope(), vec<N, T>(direction), light_color<Color>(rgb));
                flat_shapes_[shape]->set_light_source(light.get());
                pending_lights_.push_back(std::move(light));
                return pending_lights_.size() - 1;
        }

        int add_ball_light(
                const double* const center,
                const double* const direction,
                const double radius,
                const float* const rgb) override
        {
                pending_lights_.push_back(
                        std::make_unique<painter::lights::BallLight<N, T, Color>>(
                                vec<N, T>(center), vec<N, T>(direction), radius, light_color<Color>(rgb)));
                return pending_lights_.size() - 1;
        }

        void set_perspective(
                const double* const org,
                const double* const dir,
                const double* const axes,
                const double fov,
                const int* const size) override
        {
                std::array<int, N - 1> s;
                std::copy(size, size + N - 1, s.begin());
                projector_ = std::make_unique<painter::projectors::PerspectiveProjector<N, T>>(
                        vec<N, T>(org), vec<N, T>(dir), vecs<N, T, N - 1>(axes), fov, s);
        }

        void set_parallel(
                const double* const org,
                const double* const dir,
                const double* const axes,
                const double units_per_pixel,
                const int* const size) override
        {
                std::array<int, N - 1> s;
                std::copy(size, size + N - 1, s.begin());
                projector_ = std::make_unique<painter::projectors::ParallelProjector<N, T>>(
                        vec<N, T>(org), vec<N, T>(dir), vecs<N, T, N - 1>(axes), units_per_pixel, s);
        }

        void finalize(const float* const background) override
        {
                if (!projector_)
                {
                        throw std::runtime_error("no projector");
                }
                std::vector<std::unique_ptr<const Shape>> shapes;
                for (auto& s : pending_shapes_)
                {
                        shapes.push_back(std::move(s));
                }
                std::vector<std::unique_ptr<Light>> lights = std::move(pending_lights_);
                storage_ = painter::scenes::create_storage_scene<N, T>(
                        light_color<Color>(background), std::nullopt, std::move(projector_), std::move(lights),
                        std::move(shapes), &progress_);
        }

        long long pixel_count() const override
        {
                long long res = 1;
                for (const int s : scene().projector().screen_size())
                {
                        res *= s;
                }
                return res;
        }

        int actual_spp(const int spp) const override
        {
                const painter::painting::StratifiedJitteredSampler<N - 1, T> sampler(spp);
                ns::PCG engine(0u);
                std::vector<numerical::Vector<N - 1, T>> points;
                sampler.generate(engine, &points);
                return points.size();
        }

        int integrator_ = 0;
        bool flat_shading_ = false;

        // create_painter's flat_shading: bpt<true> / pt<true>, which shade
        // with the geometric normal (integrators/com/normals.h:45-64)
        void set_flat_shading(const bool flat) override
        {
                flat_shading_ = flat;
        }

        void set_integrator(const int integrator) override
        {
                if (integrator != 0 && integrator != 1)
                {
                        throw std::runtime_error("integrator must be 0 (BPT) or 1 (PT)");
                }
                integrator_ = integrator;
        }

        // One pass of per-path seeded BPT (or PT) over pixels [begin, end).
        // points: [pixel][sample][N-1] double; colors: [pixel][sample][C] float;
        // valid: [pixel][sample] 1 if bpt() / pt() returned a colour, 0 for a
        // background sample (std::nullopt).
        void render_samples(
                const int spp,
                const int max_depth,
                const unsigned seed,
                const unsigned pass,
                const long long begin,
                const long long end,
                const int threads,
                double* const points_out,
                float* const colors_out,
                unsigned char* const valid_out) override
        {
                const painter::Scene<N, T, Color>& sc = scene();
                nbpt_oracle_max_depth = max_depth;
                const int count = actual_spp(spp);
                const painter::painting::StratifiedJitteredSampler<N - 1, T> sampler(spp);
                const std::array<int, N - 1> size = sc.projector().screen_size();

                parallel_for(
                        end - begin, threads,
                        [&](const long long k)
                        {
                                thread_local std::optional<painter::integrators::bpt::LightDistribution<N, T, Color>>
                                        distribution;
                                thread_local const void* distribution_scene = nullptr;
                                if (distribution_scene != &sc)
                                {
                                        distribution.emplace(sc.light_sources());
                                        distribution_scene = &sc;
                                }

                                const long long p = begin + k;
                                const std::array<int, N - 1> pixel = pixel_of<N - 1>(p, size);
                                const numerical::Vector<N - 1, T> pixel_org = numerical::to_vector<T>(pixel);

                                std::vector<numerical::Vector<N - 1, T>> points;
                                {
                                        const auto engine = make_engine({seed, pass, static_cast<std::uint32_t>(p), 0u});
                                        sampler.generate(*engine, &points);
                                }
                                for (int i = 0; i < count; ++i)
                                {
                                        const auto engine = make_engine(
                                                {seed, pass, static_cast<std::uint32_t>(p),
                                                 static_cast<std::uint32_t>(i + 1)});
                                        const numerical::Ray<N, T> ray = sc.projector().ray(pixel_org + points[i]);
                                        const std::optional<Color> color =
                                                integrator_ == 1
                                                        ? (flat_shading_
                                                                   ? painter::integrators::pt::pt<true>(sc, ray, *engine)
                                                                   : painter::integrators::pt::pt<false>(sc, ray, *engine))
                                                        : (flat_shading_ ? painter::integrators::bpt::bpt<true>(
                                                                                   sc, ray, *distribution, *engine)
                                                                         : painter::integrators::bpt::bpt<false>(
                                                                                   sc, ray, *distribution, *engine));
                                        const long long s = k * count + i;
                                        for (std::size_t d = 0; d < N - 1; ++d)
                                        {
                                                points_out[s * (N - 1) + d] = points[i][d];
                                        }
                                        valid_out[s] = color.has_value();
                                        for (int c = 0; c < C; ++c)
                                        {
                                                colors_out[s * C + c] = color ? channel(*color, c) : 0.0f;
                                        }
                                }
                        });
        }

        // Seeded passes accumulated by the reference's pixels::Pixels.
        // Samples are added pixel by pixel in index order, so the result does
        // not depend on the thread count.
        // the samples of the pixels [source_begin, source_end) (all of them
        // when source_end < 0) added to one pixels::Pixels in increasing pixel
        // order, which is the order a receiving pixel takes its sources in
        void render_image(
                const int spp,
                const int max_depth,
                const unsigned seed,
                const int passes,
                const int threads,
                const long long source_begin,
                const long long source_end,
                float* const rgb_out,
                float* const rgba_out) override
        {
                const painter::Scene<N, T, Color>& sc = scene();
                const long long pixels_count = source_end < 0 ? pixel_count() : source_end;
                const int count = actual_spp(spp);
                CollectNotifier<N - 1> notifier;
                painter::pixels::Pixels<N - 1, T, Color> pixels(
                        sc.projector().screen_size(), sc.background_color(), &notifier);

                constexpr long long CHUNK = 1 << 14;
                std::vector<double> points(CHUNK * count * (N - 1));
                std::vector<float> colors(CHUNK * count * C);
                std::vector<unsigned char> valid(CHUNK * count);
                for (int pass = 0; pass < passes; ++pass)
                {
                        for (long long b = source_begin; b < pixels_count; b += CHUNK)
                        {
                                const long long e = std::min(pixels_count, b + CHUNK);
                                render_samples(
                                        spp, max_depth, seed, pass, b, e, threads, points.data(), colors.data(),
                                        valid.data());
                                std::vector<numerical::Vector<N - 1, T>> pts(count);
                                std::vector<std::optional<Color>> cols(count);
                                for (long long p = b; p < e; ++p)
                                {
                                        for (int i = 0; i < count; ++i)
                                        {
                                                const long long s = (p - b) * count + i;
                                                for (std::size_t d = 0; d < N - 1; ++d)
                                                {
                                                        pts[i][d] = points[s * (N - 1) + d];
                                                }
                                                if (valid[s])
                                                {
                                                        Color c(0);
                                                        for (int k = 0; k < C; ++k)
                                                        {
                                                                channel(c, k) = colors[s * C + k];
                                                        }
                                                        cols[i] = c;
                                                }
                                                else
                                                {
                                                        cols[i].reset();
                                                }
                                        }
                                        pixels.add_samples(
                                                pixel_of<N - 1>(p, sc.projector().screen_size()), pts, cols);
                                }
                        }
                }
                ns::image::Image<N - 1> rgb;
                ns::image::Image<N - 1> rgba;
                pixels.images(&rgb, &rgba);
                std::memcpy(rgb_out, rgb.pixels.data(), rgb.pixels.size());
                if (rgba_out)
                {
                        std::memcpy(rgba_out, rgba.pixels.data(), rgba.pixels.size());
                }
        }

        // The unmodified reference painter (create_painter, BPT, OS-seeded
        // per-thread streams), timed.  stats: [sample_count, ray_count,
        // previous_pass_duration, wall seconds, pass_number].
        void paint(
                const int spp,
                const int max_depth,
                const int passes,
                const int threads,
                double* const stats,
                float* const rgb_out) override
        {
                const painter::Scene<N, T, Color>& sc = scene();
                nbpt_oracle_max_depth = max_depth;
                CollectNotifier<N - 1> notifier;
                const auto start = std::chrono::steady_clock::now();
                std::unique_ptr<painter::Painter> p = painter::create_painter<N, T, Color>(
                        integrator_ == 1 ? painter::Integrator::PT : painter::Integrator::BPT, &notifier, spp, passes,
                        &sc, threads, flat_shading_);
                p->wait();
                const double wall =
                        std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
                if (!notifier.error.empty())
                {
                        throw std::runtime_error(notifier.error);
                }
                const painter::Statistics s = p->statistics();
                stats[0] = s.sample_count;
                stats[1] = s.ray_count;
                stats[2] = s.previous_pass_duration;
                stats[3] = wall;
                stats[4] = s.pass_number;
                if (rgb_out)
                {
                        notifier.copy_rgb(rgb_out);
                }
        }

        // counts: vertices, normals, facets, materials, nodes, indices
        void mesh_info(const int shape, long long* const counts) override
        {
                MeshRecord& m = mesh(shape);
                counts[0] = m.data.mesh.vertices.size();
                counts[1] = m.data.mesh.normals.size();
                counts[2] = m.data.mesh.facets.size();
                counts[3] = m.data.mesh.materials.size();
                counts[4] = (m.bvh.get()->*member_pointer(BvhNodesTag<N, T>{})).size();
                counts[5] = (m.bvh.get()->*member_pointer(BvhIndicesTag<N, T>{})).size();
        }

        // planes: per facet the simplex hyperplane (n[N], d) followed by the
        // N-1 barycentric hyperplanes (n[N], d), as built by HyperplaneSimplex
        // (src/geometry/spatial/hyperplane_simplex.h:82-111); the facet's normal
        // is reversed where its vertex normals all point the other way
        // (src/painter/shapes/mesh/facet.cpp:113-118), read back here through
        // the public geometric_normal().
        void mesh_dump(
                const int shape,
                double* const vertices,
                double* const normals,
                int* const facet_vertices,
                int* const facet_materials,
                double* const material_params,
                float* const material_colors,
                double* const planes,
                double* const node_bounds,
                unsigned* const node_info,
                unsigned* const indices) override
        {
                MeshRecord& m = mesh(shape);
                const auto& mesh = m.data.mesh;
                for (std::size_t i = 0; i < mesh.vertices.size(); ++i)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                vertices[i * N + k] = mesh.vertices[i][k];
                        }
                }
                for (std::size_t i = 0; i < mesh.normals.size(); ++i)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                normals[i * N + k] = mesh.normals[i][k];
                        }
                }
                for (std::size_t f = 0; f < mesh.facets.size(); ++f)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                facet_vertices[f * N + k] = m.data.facet_vertex_indices[f][k];
                        }
                        facet_materials[f] = mesh.facets[f].material();

                        std::array<numerical::Vector<N, T>, N> v;
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                v[k] = mesh.vertices[m.data.facet_vertex_indices[f][k]];
                        }
                        const spatial::HyperplaneSimplex<N, T> simplex(v);
                        const auto& plane = simplex.*member_pointer(SimplexPlaneTag<N, T>{});
                        const auto& ps = simplex.*member_pointer(SimplexPlanesTag<N, T>{});
                        double* const out = planes + f * N * (N + 1);
                        const numerical::Vector<N, T> n = mesh.facets[f].geometric_normal();
                        const bool reversed = !(n == plane.n);
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                out[k] = n[k];
                        }
                        out[N] = reversed ? -plane.d : plane.d;
                        for (std::size_t j = 0; j < N - 1; ++j)
                        {
                                for (std::size_t k = 0; k < N; ++k)
                                {
                                        out[(j + 1) * (N + 1) + k] = ps[j].n[k];
                                }
                                out[(j + 1) * (N + 1) + N] = ps[j].d;
                        }
                }
                for (std::size_t i = 0; i < mesh.materials.size(); ++i)
                {
                        const auto& material = mesh.materials[i];
                        material_params[i * 3 + 0] = material.metalness();
                        material_params[i * 3 + 1] = material.roughness();
                        material_params[i * 3 + 2] = material.alpha();
                        for (int c = 0; c < C; ++c)
                        {
                                material_colors[i * C + c] = channel(material.color(), c);
                        }
                }
                const auto& nodes = m.bvh.get()->*member_pointer(BvhNodesTag<N, T>{});
                for (std::size_t i = 0; i < nodes.size(); ++i)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                node_bounds[i * 2 * N + k] = nodes[i].bounds.min()[k];
                                node_bounds[i * 2 * N + N + k] = nodes[i].bounds.max()[k];
                        }
                        node_info[i * 3 + 0] = nodes[i].object_offset;
                        node_info[i * 3 + 1] = nodes[i].object_count;
                        node_info[i * 3 + 2] = nodes[i].axis;
                }
                const auto& idx = m.bvh.get()->*member_pointer(BvhIndicesTag<N, T>{});
                std::copy(idx.begin(), idx.end(), indices);
        }

        // Closest hit (any == 0) or any hit (any == 1) of rays against one
        // mesh, with the mesh shape's own traversal and facet test
        // (src/painter/shapes/mesh.cpp:231-268).  rays: [n][2N] (org, dir; the
        // direction is normalised by Ray as in the reference).
        void mesh_trace(
                const int shape,
                const double* const rays,
                const long long n,
                const double max_distance,
                const int any,
                int* const facet_out,
                double* const t_out,
                unsigned char* const any_out,
                const int threads) override
        {
                MeshRecord& m = mesh(shape);
                const auto& facets = m.data.mesh.facets;
                const accelerators::Bvh<N, T>& bvh = *m.bvh;
                parallel_for(
                        n, threads,
                        [&](const long long i)
                        {
                                const numerical::Ray<N, T> ray(
                                        vec<N, T>(rays + i * 2 * N), vec<N, T>(rays + i * 2 * N + N));
                                const T max = max_distance;
                                if (any)
                                {
                                        any_out[i] = bvh.intersect(
                                                ray, max,
                                                [&](const auto& indices, const auto& max_d) -> bool
                                                {
                                                        return spatial::ray_intersection_any(facets, indices, ray, max_d);
                                                });
                                        return;
                                }
                                using Facet = std::remove_cvref_t<decltype(facets.front())>;
                                const auto hit = bvh.intersect(
                                        ray, max,
                                        [&](const auto& indices,
                                            const auto& max_d) -> std::optional<std::tuple<T, const Facet*>>
                                        {
                                                const std::tuple<T, const Facet*> info =
                                                        spatial::ray_intersection(facets, indices, ray, max_d);
                                                if (std::get<1>(info))
                                                {
                                                        return info;
                                                }
                                                return std::nullopt;
                                        });
                                if (hit)
                                {
                                        facet_out[i] = std::get<1>(*hit) - facets.data();
                                        t_out[i] = std::get<0>(*hit);
                                }
                                else
                                {
                                        facet_out[i] = -1;
                                        t_out[i] = 0;
                                }
                        });
        }

        // Closest hit through the whole scene (Scene::intersect,
        // src/painter/scenes/scene.cpp:161-167) without an origin offset.
        void scene_trace(
                const double* const rays,
                const long long n,
                const int threads,
                double* const t_out,
                double* const point_out,
                double* const normal_out,
                unsigned char* const hit_out) override
        {
                const painter::Scene<N, T, Color>& sc = scene();
                parallel_for(
                        n, threads,
                        [&](const long long i)
                        {
                                const numerical::Ray<N, T> ray(
                                        vec<N, T>(rays + i * 2 * N), vec<N, T>(rays + i * 2 * N + N));
                                const painter::SurfaceIntersection<N, T, Color> s = sc.intersect(std::nullopt, ray);
                                hit_out[i] = static_cast<bool>(s);
                                if (!s)
                                {
                                        t_out[i] = 0;
                                        return;
                                }
                                t_out[i] = s.distance();
                                const numerical::Vector<N, T> g = s.geometric_normal();
                                for (std::size_t k = 0; k < N; ++k)
                                {
                                        point_out[i * N + k] = s.point()[k];
                                        normal_out[i * N + k] = g[k];
                                }
                        });
        }

        // GGX brdf f and pdf (src/shading/ggx/brdf.h:146-194) for a surface of
        // the given colour and metalness.
        void brdf(
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double* const n,
                const double* const v,
                const double* const l,
                float* const f_out,
                double* const pdf_out) override
        {
                const auto colors = ns::shading::ggx::compute_metalness(surface_color<Color>(rgb), T(metalness));
                const Color f = ns::shading::ggx::brdf::f(
                        T(roughness), colors, vec<N, T>(n), vec<N, T>(v), vec<N, T>(l));
                for (int c = 0; c < C; ++c)
                {
                        f_out[c] = channel(f, c);
                }
                *pdf_out = ns::shading::ggx::brdf::pdf(T(roughness), vec<N, T>(n), vec<N, T>(v), vec<N, T>(l));
        }

        // One sample_f (src/shading/ggx/brdf.h:196-238) from a seed_seq stream.
        void brdf_sample(
                const double metalness,
                const double roughness,
                const float* const rgb,
                const double* const n,
                const double* const v,
                const unsigned* const seed,
                const int seed_words,
                double* const l_out,
                double* const pdf_out,
                float* const f_out) override
        {
                std::seed_seq seq(seed, seed + seed_words);
                ns::PCG engine(seq);
                const auto colors = ns::shading::ggx::compute_metalness(surface_color<Color>(rgb), T(metalness));
                const auto s = ns::shading::ggx::brdf::sample_f(
                        engine, T(roughness), colors, vec<N, T>(n), vec<N, T>(v));
                *pdf_out = s.pdf;
                if (s.pdf > 0)
                {
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                l_out[k] = s.l[k];
                        }
                        for (int c = 0; c < C; ++c)
                        {
                                f_out[c] = channel(s.brdf, c);
                        }
                }
        }

        // One leave_sample (kind 0) or arrive_sample (kind 1) of light `light`
        // from a seed_seq stream (src/painter/lights/*_light.cpp).
        // out: leave: [org N, dir N, n N, pdf_pos, pdf_dir]; arrive: [l N, pdf,
        // distance or -1]; radiance: C channels.
        void light_sample(
                const int light,
                const int kind,
                const unsigned* const seed,
                const int seed_words,
                const double* const point,
                const double* const n,
                double* const out,
                float* const radiance) override
        {
                if (!storage_ || light < 0 || light >= static_cast<int>(storage_->light_sources.size()))
                {
                        throw std::runtime_error("no such light");
                }
                const Light& l = *storage_->light_sources[light];
                std::seed_seq seq(seed, seed + seed_words);
                ns::PCG engine(seq);
                if (kind == 0)
                {
                        const auto s = l.leave_sample(engine);
                        for (std::size_t k = 0; k < N; ++k)
                        {
                                out[k] = s.ray.org()[k];
                                out[N + k] = s.ray.dir()[k];
                                out[2 * N + k] = s.n ? (*s.n)[k] : 0;
                        }
                        out[3 * N] = s.pdf_pos;
                        out[3 * N + 1] = s.pdf_dir;
                        for (int c = 0; c < C; ++c)
                        {
                                radiance[c] = channel(s.radiance, c);
                        }
                        return;
                }
                const auto s = l.arrive_sample(engine, vec<N, T>(point), vec<N, T>(n));
                for (std::size_t k = 0; k < N; ++k)
                {
                        out[k] = s.pdf > 0 ? s.l[k] : 0;
                }
                out[N] = s.pdf;
                out[N + 1] = s.distance ? *s.distance : -1;
                for (int c = 0; c < C; ++c)
                {
                        radiance[c] = s.pdf > 0 ? channel(s.radiance, c) : 0;
                }
        }
};

template <std::size_t N>
std::unique_ptr<SceneBase> make_scene(const int use_double, const int spectrum)
{
        if (use_double)
        {
                if (spectrum)
                {
                        return std::make_unique<Scene<N, double, ns::color::Spectrum>>();
                }
                return std::make_unique<Scene<N, double, ns::color::Color>>();
        }
        if (spectrum)
        {
                return std::make_unique<Scene<N, float, ns::color::Spectrum>>();
        }
        return std::make_unique<Scene<N, float, ns::color::Color>>();
}

template <typename F>
int guarded(const F& f)
{
        try
        {
                f();
                return 0;
        }
        catch (const std::exception& e)
        {
                g_last_error = e.what();
        }
        catch (...)
        {
                g_last_error = "unknown exception";
        }
        return -1;
}

SceneBase* as_scene(void* const p)
{
        if (!p)
        {
                throw std::runtime_error("null scene");
        }
        return static_cast<SceneBase*>(p);
}

template <std::size_t N, typename T>
void f1_tables(float* const table, float* const average)
{
        const auto [size2, data2] = ns::shading::ggx::f1_albedo_cosine_roughness_data<N, T>();
        const auto [size1, data1] = ns::shading::ggx::f1_albedo_cosine_weighted_average_data<N, T>();
        if (size2[0] * size2[1] != 32 * 32 || size1[0] != 32)
        {
                throw std::runtime_error("unexpected f1 albedo table size");
        }
        std::copy(data2.begin(), data2.end(), table);
        std::copy(data1.begin(), data1.end(), average);
}
}

extern "C"
{
const char* oracle_last_error()
{
        return g_last_error.c_str();
}

void* oracle_scene_new(const int n, const int use_double, const int spectrum)
{
        try
        {
                switch (n)
                {
                case 3:
                        return make_scene<3>(use_double, spectrum).release();
                case 4:
                        return make_scene<4>(use_double, spectrum).release();
                case 5:
                        return make_scene<5>(use_double, spectrum).release();
                default:
                        g_last_error = "dimension must be 3, 4 or 5";
                        return nullptr;
                }
        }
        catch (const std::exception& e)
        {
                g_last_error = e.what();
                return nullptr;
        }
}

void oracle_scene_free(void* const scene)
{
        delete static_cast<SceneBase*>(scene);
}

int oracle_scene_add_hyperplane_parallelotope(
        void* const scene,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double alpha,
        const double* const org,
        const double* const vectors)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_hyperplane_parallelotope(
                                metalness, roughness, rgb, alpha, org, vectors);
                });
        return r < 0 ? r : index;
}

int oracle_scene_add_parallelotope(
        void* const scene,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double alpha,
        const double* const org,
        const double* const vectors)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_parallelotope(metalness, roughness, rgb, alpha, org, vectors);
                });
        return r < 0 ? r : index;
}

int oracle_scene_add_mesh_object(
        void* const scene,
        const float* const points,
        const long n_points,
        const int* const facets,
        const long n_facets,
        const double* const matrix,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double alpha)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_mesh_object(
                                points, n_points, facets, n_facets, matrix, metalness, roughness, rgb, alpha);
                });
        return r < 0 ? r : index;
}

int oracle_scene_add_mesh_file(
        void* const scene,
        const char* const path,
        const double* const matrix,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double alpha)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_mesh_file(path, matrix, metalness, roughness, rgb, alpha);
                });
        return r < 0 ? r : index;
}

// model::mesh::file::load_from_obj_file / load_from_stl_file alone:
// counts[0] vertices, [1] normals, [2] facets
int oracle_load_mesh_file(const char* const path, const int n, const int stl, long long* const counts)
{
        return guarded(
                [&]
                {
                        ns::progress::Ratio progress(nullptr);
                        const std::filesystem::path file(path);
                        const auto fill = [&](const auto& mesh)
                        {
                                counts[0] = mesh->vertices.size();
                                counts[1] = mesh->normals.size();
                                counts[2] = mesh->facets.size();
                        };
                        if (n == 3)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<3>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<3>(file, &progress));
                        }
                        else if (n == 4)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<4>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<4>(file, &progress));
                        }
                        else if (n == 5)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<5>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<5>(file, &progress));
                        }
                        else
                        {
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                });
}

// model::mesh::file::load_from_obj_file / load_from_stl_file alone, as
// arrays: counts[0] vertices, [1] normals, [2] facets; with non-null
// buffers also the vertices [V][n], the normals [M][n], and per facet its n
// vertex indices, its n normal indices (-1 where it has none), has_normal
// and its material (-1: none)
int oracle_mesh_file_arrays(
        const char* const path,
        const int n,
        const int stl,
        long long* const counts,
        float* const vertices,
        float* const normals,
        int* const facet_vertices,
        int* const facet_normals,
        unsigned char* const has_normal,
        int* const facet_material)
{
        return guarded(
                [&]
                {
                        ns::progress::Ratio progress(nullptr);
                        const std::filesystem::path file(path);
                        const auto fill = [&](const auto& mesh)
                        {
                                const int M = n;
                                counts[0] = mesh->vertices.size();
                                counts[1] = mesh->normals.size();
                                counts[2] = mesh->facets.size();
                                if (vertices == nullptr)
                                {
                                        return;
                                }
                                for (std::size_t i = 0; i < mesh->vertices.size(); ++i)
                                {
                                        for (int d = 0; d < M; ++d)
                                        {
                                                vertices[i * M + d] = mesh->vertices[i][d];
                                        }
                                }
                                for (std::size_t i = 0; i < mesh->normals.size(); ++i)
                                {
                                        for (int d = 0; d < M; ++d)
                                        {
                                                normals[i * M + d] = mesh->normals[i][d];
                                        }
                                }
                                for (std::size_t f = 0; f < mesh->facets.size(); ++f)
                                {
                                        const auto& facet = mesh->facets[f];
                                        for (int k = 0; k < M; ++k)
                                        {
                                                facet_vertices[f * M + k] = facet.vertices[k];
                                                facet_normals[f * M + k] = facet.has_normal ? facet.normals[k] : -1;
                                        }
                                        has_normal[f] = facet.has_normal ? 1 : 0;
                                        facet_material[f] = facet.material;
                                }
                        };
                        if (n == 3)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<3>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<3>(file, &progress));
                        }
                        else if (n == 4)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<4>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<4>(file, &progress));
                        }
                        else if (n == 5)
                        {
                                stl ? fill(ns::model::mesh::file::load_from_stl_file<5>(file, &progress, false))
                                    : fill(ns::model::mesh::file::load_from_obj_file<5>(file, &progress));
                        }
                        else
                        {
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                });
}

int oracle_scene_add_mesh(void* const scene)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_mesh();
                });
        return r < 0 ? r : index;
}

int oracle_scene_add_parallelotope_light(
        void* const scene,
        const int shape,
        const double* const direction,
        const float* const rgb)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_parallelotope_light(shape, direction, rgb);
                });
        return r < 0 ? r : index;
}

int oracle_scene_add_ball_light(
        void* const scene,
        const double* const center,
        const double* const direction,
        const double radius,
        const float* const rgb)
{
        int index = -1;
        const int r = guarded(
                [&]
                {
                        index = as_scene(scene)->add_ball_light(center, direction, radius, rgb);
                });
        return r < 0 ? r : index;
}

int oracle_scene_set_perspective(
        void* const scene,
        const double* const org,
        const double* const dir,
        const double* const axes,
        const double fov,
        const int* const size)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->set_perspective(org, dir, axes, fov, size);
                });
}

int oracle_scene_set_parallel(
        void* const scene,
        const double* const org,
        const double* const dir,
        const double* const axes,
        const double units_per_pixel,
        const int* const size)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->set_parallel(org, dir, axes, units_per_pixel, size);
                });
}

int oracle_scene_finalize(void* const scene, const float* const background)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->finalize(background);
                });
}

long long oracle_scene_pixel_count(void* const scene)
{
        long long res = -1;
        guarded(
                [&]
                {
                        res = as_scene(scene)->pixel_count();
                });
        return res;
}

int oracle_scene_actual_spp(void* const scene, const int spp)
{
        int res = -1;
        guarded(
                [&]
                {
                        res = as_scene(scene)->actual_spp(spp);
                });
        return res;
}

int oracle_scene_set_flat_shading(void* const scene, const int flat)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->set_flat_shading(flat != 0);
                });
}

int oracle_scene_set_integrator(void* const scene, const int integrator)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->set_integrator(integrator);
                });
}

int oracle_render_samples(
        void* const scene,
        const int spp,
        const int max_depth,
        const unsigned seed,
        const unsigned pass,
        const long long begin,
        const long long end,
        const int threads,
        double* const points,
        float* const colors,
        unsigned char* const valid)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->render_samples(
                                spp, max_depth, seed, pass, begin, end, threads, points, colors, valid);
                });
}

int oracle_render_image(
        void* const scene,
        const int spp,
        const int max_depth,
        const unsigned seed,
        const int passes,
        const int threads,
        float* const rgb,
        float* const rgba)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->render_image(spp, max_depth, seed, passes, threads, 0, -1, rgb, rgba);
                });
}

int oracle_render_image_range(
        void* const scene,
        const int spp,
        const int max_depth,
        const unsigned seed,
        const int passes,
        const int threads,
        const long long source_begin,
        const long long source_end,
        float* const rgb,
        float* const rgba)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->render_image(
                                spp, max_depth, seed, passes, threads, source_begin, source_end, rgb, rgba);
                });
}

int oracle_paint(
        void* const scene,
        const int spp,
        const int max_depth,
        const int passes,
        const int threads,
        double* const stats,
        float* const rgb)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->paint(spp, max_depth, passes, threads, stats, rgb);
                });
}

int oracle_mesh_info(void* const scene, const int shape, long long* const counts)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->mesh_info(shape, counts);
                });
}

int oracle_mesh_dump(
        void* const scene,
        const int shape,
        double* const vertices,
        double* const normals,
        int* const facet_vertices,
        int* const facet_materials,
        double* const material_params,
        float* const material_colors,
        double* const planes,
        double* const node_bounds,
        unsigned* const node_info,
        unsigned* const indices)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->mesh_dump(
                                shape, vertices, normals, facet_vertices, facet_materials, material_params,
                                material_colors, planes, node_bounds, node_info, indices);
                });
}

int oracle_mesh_trace(
        void* const scene,
        const int shape,
        const double* const rays,
        const long long n,
        const double max_distance,
        const int any,
        int* const facet,
        double* const t,
        unsigned char* const any_hit,
        const int threads)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->mesh_trace(shape, rays, n, max_distance, any, facet, t, any_hit, threads);
                });
}

int oracle_scene_trace(
        void* const scene,
        const double* const rays,
        const long long n,
        const int threads,
        double* const t,
        double* const point,
        double* const normal,
        unsigned char* const hit)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->scene_trace(rays, n, threads, t, point, normal, hit);
                });
}

int oracle_brdf(
        void* const scene,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double* const n,
        const double* const v,
        const double* const l,
        float* const f,
        double* const pdf)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->brdf(metalness, roughness, rgb, n, v, l, f, pdf);
                });
}

int oracle_brdf_sample(
        void* const scene,
        const double metalness,
        const double roughness,
        const float* const rgb,
        const double* const n,
        const double* const v,
        const unsigned* const seed,
        const int seed_words,
        double* const l,
        double* const pdf,
        float* const f)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->brdf_sample(metalness, roughness, rgb, n, v, seed, seed_words, l, pdf, f);
                });
}

// Raw PCG32 output of a seed_seq stream (src/com/random/pcg.h:53-62).
int oracle_pcg(const unsigned* const seed, const int seed_words, const int count, unsigned* const out)
{
        return guarded(
                [&]
                {
                        std::seed_seq seq(seed, seed + seed_words);
                        ns::PCG engine(seq);
                        for (int i = 0; i < count; ++i)
                        {
                                out[i] = engine();
                        }
                });
}

// std::uniform_real_distribution<T>(0, 1) draws from a seed_seq stream.
int oracle_canonical(
        const unsigned* const seed,
        const int seed_words,
        const int count,
        const int use_double,
        double* const out)
{
        return guarded(
                [&]
                {
                        std::seed_seq seq(seed, seed + seed_words);
                        ns::PCG engine(seq);
                        if (use_double)
                        {
                                std::uniform_real_distribution<double> urd(0, 1);
                                for (int i = 0; i < count; ++i)
                                {
                                        out[i] = urd(engine);
                                }
                        }
                        else
                        {
                                std::uniform_real_distribution<float> urd(0, 1);
                                for (int i = 0; i < count; ++i)
                                {
                                        out[i] = urd(engine);
                                }
                        }
                });
}

// Stratified jittered points of one pixel (src/sampling/sj_sampler.h:187-205),
// returned as [count][dimension] doubles; the return value is the count.
int oracle_sj_points(
        const int dimension,
        const int use_double,
        const int spp,
        const unsigned* const seed,
        const int seed_words,
        double* const out)
{
        int count = -1;
        const int r = guarded(
                [&]
                {
                        std::seed_seq seq(seed, seed + seed_words);
                        ns::PCG engine(seq);
                        const auto run = [&]<std::size_t M, typename T>()
                        {
                                const ns::painter::painting::StratifiedJitteredSampler<M, T> sampler(spp);
                                std::vector<numerical::Vector<M, T>> points;
                                sampler.generate(engine, &points);
                                count = points.size();
                                if (out)
                                {
                                        for (std::size_t i = 0; i < points.size(); ++i)
                                        {
                                                for (std::size_t d = 0; d < M; ++d)
                                                {
                                                        out[i * M + d] = points[i][d];
                                                }
                                        }
                                }
                        };
                        switch (dimension * 2 + (use_double ? 1 : 0))
                        {
                        case 4:
                                run.template operator()<2, float>();
                                break;
                        case 5:
                                run.template operator()<2, double>();
                                break;
                        case 6:
                                run.template operator()<3, float>();
                                break;
                        case 7:
                                run.template operator()<3, double>();
                                break;
                        case 8:
                                run.template operator()<4, float>();
                                break;
                        case 9:
                                run.template operator()<4, double>();
                                break;
                        default:
                                throw std::runtime_error("screen dimension must be 2, 3 or 4");
                        }
                });
        return r < 0 ? r : count;
}

// The 32x32 (cosine, roughness) and 32-entry (roughness) f1 albedo tables the
// GGX multiple-bounce term interpolates (src/shading/ggx/f1_albedo.cpp).
int oracle_f1_albedo_tables(const int n, const int use_double, float* const table, float* const average)
{
        return guarded(
                [&]
                {
                        (void)use_double;
                        switch (n)
                        {
                        case 3:
                                f1_tables<3, float>(table, average);
                                break;
                        case 4:
                                f1_tables<4, float>(table, average);
                                break;
                        case 5:
                                f1_tables<5, float>(table, average);
                                break;
                        default:
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                });
}

int oracle_f1_albedo_tables_double(const int n, double* const table, double* const average)
{
        return guarded(
                [&]
                {
                        const auto copy = [&]<std::size_t N>()
                        {
                                const auto [s2, d2] = ns::shading::ggx::f1_albedo_cosine_roughness_data<N, double>();
                                const auto [s1, d1] =
                                        ns::shading::ggx::f1_albedo_cosine_weighted_average_data<N, double>();
                                std::copy(d2.begin(), d2.end(), table);
                                std::copy(d1.begin(), d1.end(), average);
                        };
                        switch (n)
                        {
                        case 3:
                                copy.template operator()<3>();
                                break;
                        case 4:
                                copy.template operator()<4>();
                                break;
                        case 5:
                                copy.template operator()<5>();
                                break;
                        default:
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                });
}

// The 64-bin spectral basis the reference's Spectrum type builds at start-up
// (src/color/color.h:156-210): x, y, z colour matching functions, then the
// seven reflectance and seven D65 illumination Smits basis spectra
// (white, cyan, magenta, yellow, red, green, blue).  out: [17][64].
int oracle_spectrum_functions(double* const out)
{
        return guarded(
                [&]
                {
                        namespace s = ns::color::samples;
                        constexpr int FROM = 380;
                        constexpr int TO = 720;
                        constexpr int COUNT = 64;
                        const std::vector<std::vector<double>> rows = {
                                s::cie_x_samples<s::XYZ_31>(FROM, TO, COUNT),
                                s::cie_y_samples<s::XYZ_31>(FROM, TO, COUNT),
                                s::cie_z_samples<s::XYZ_31>(FROM, TO, COUNT),
                                s::rgb_reflectance_white_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_cyan_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_magenta_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_yellow_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_red_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_green_samples(FROM, TO, COUNT),
                                s::rgb_reflectance_blue_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_white_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_cyan_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_magenta_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_yellow_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_red_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_green_samples(FROM, TO, COUNT),
                                s::rgb_illumination_d65_blue_samples(FROM, TO, COUNT)};
                        for (std::size_t r = 0; r < rows.size(); ++r)
                        {
                                if (rows[r].size() != COUNT)
                                {
                                        throw std::runtime_error("unexpected spectrum size");
                                }
                                std::copy(rows[r].begin(), rows[r].end(), out + r * COUNT);
                        }
                });
}

// A material colour as the painter stores it: Color(r, g, b) for surfaces and
// Color::illuminant(r, g, b) for lights, as float channels (3 or 64).
int oracle_color(const int spectrum, const int illuminant, const float* const rgb, float* const out)
{
        return guarded(
                [&]
                {
                        const auto copy = [&]<typename Color>()
                        {
                                const Color c = illuminant ? light_color<Color>(rgb) : surface_color<Color>(rgb);
                                for (int i = 0; i < channels<Color>(); ++i)
                                {
                                        out[i] = channel(c, i);
                                }
                        };
                        if (spectrum)
                        {
                                copy.template operator()<ns::color::Spectrum>();
                        }
                        else
                        {
                                copy.template operator()<ns::color::Color>();
                        }
                });
}
int oracle_light_sample(
        void* const scene,
        const int light,
        const int kind,
        const unsigned* const seed,
        const int seed_words,
        const double* const point,
        const double* const n,
        double* const out,
        float* const radiance)
{
        return guarded(
                [&]
                {
                        as_scene(scene)->light_sample(light, kind, seed, seed_words, point, n, out, radiance);
                });
}

// Compile-time constants of the path, as the reference computes them for
// dimension n and precision T (double if use_double, else float), returned as
// doubles: [0] hemisphere cosine integral K (sphere_integral.h), [1] cosine
// hemisphere pdf factor 1/K (sphere_cosine.h:82-92), [2] uniform (n-1)-ball
// pdf factor (sphere_uniform.h:198-203), [3] ray origin offset
// (point_offset.h:32), [4] visibility distance factor (visibility.h:36-43),
// [5] directed-outside cosine (visibility.h:45-50), [6] 1/K as the diffuse
// term stores it (subsurface.h:71), [7] K as the multiple-bounce term stores
// it (multiple_bounce.h:44).
int oracle_constants(const int n, const int use_double, double* const out)
{
        return guarded(
                [&]
                {
                        const auto fill = [&]<std::size_t N, typename T>()
                        {
                                namespace g = ns::geometry::shapes;
                                out[0] = static_cast<T>(g::SPHERE_INTEGRATE_COSINE_FACTOR_OVER_HEMISPHERE<N, T>);
                                out[1] = ns::sampling::cosine_on_hemisphere_pdf<N, T>(T{1});
                                out[2] = ns::sampling::uniform_in_sphere_pdf<N - 1, T>(T{1});
                                out[3] = spatial::point_offset_implementation::OFFSET<T>;
                                out[4] = static_cast<T>(1 - 1000 * ns::Limits<T>::epsilon()) * T{1};
                                out[5] = 100 * ns::Limits<T>::epsilon();
                                out[6] = static_cast<T>(
                                        1 / g::SPHERE_INTEGRATE_COSINE_FACTOR_OVER_HEMISPHERE<N, long double>);
                                out[7] = static_cast<T>(g::SPHERE_INTEGRATE_COSINE_FACTOR_OVER_HEMISPHERE<N, long double>);
                        };
                        switch (n * 2 + (use_double ? 1 : 0))
                        {
                        case 6:
                                fill.template operator()<3, float>();
                                break;
                        case 7:
                                fill.template operator()<3, double>();
                                break;
                        case 8:
                                fill.template operator()<4, float>();
                                break;
                        case 9:
                                fill.template operator()<4, double>();
                                break;
                        case 10:
                                fill.template operator()<5, float>();
                                break;
                        case 11:
                                fill.template operator()<5, double>();
                                break;
                        default:
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                });
}
}
