// Type-erased interface between the C-ABI (capi.cpp) and the templated
// scene/painter implementations compiled once per space dimension
// (painter_n3.cu, painter_n4.cu, painter_n5.cu).
#pragma once

#include <cstdint>
#include <memory>

namespace nbpt
{
struct Statistics final
{
        long long pass_number;
        long long pixel_count;
        long long ray_count;
        long long sample_count;
        double previous_pass_duration; // seconds, device time of the last pass
        double paths_seconds;          // device time of the path kernel, last pass
        unsigned long long nodes;      // BVH nodes visited, last pass
        unsigned long long facets;     // facet records tested, last pass
        unsigned long long shapes;     // other shapes tested, last pass
        long long kernel_launches;     // kernels launched by the last pass
        long long nonfinite_samples;   // samples with a NaN or infinite colour, all passes
        long long stack_overflows;     // ray queries cut short by a full traversal stack, all passes
};

// painter::Integrator (src/painter/painter.h:143-147), same order
enum class Integrator : int
{
        BPT = 0,
        PT = 1
};

// the type of a painter's per-pixel sums (create_painter's pixel_sums)
inline constexpr int PIXEL_SUMS_DEFAULT = 0;
inline constexpr int PIXEL_SUMS_FLOAT = 1;
inline constexpr int PIXEL_SUMS_DOUBLE = 2;

class Painter
{
public:
        virtual ~Painter() = default;
        virtual void enqueue_passes(int passes) = 0;
        virtual void wait() = 0;
        virtual void images(float* rgb, float* rgba) = 0;
        // resolves the images of the passes so far and copies them to host
        // memory on the painter's stream, without waiting (the copy overlaps
        // later work when the host memory is pinned)
        virtual void enqueue_images(float* rgb, float* rgba) = 0;
        virtual int device() const = 0;
        virtual void samples(double* points, float* colors, unsigned char* valid) = 0;
        virtual Statistics statistics() = 0;
        virtual void* stream() = 0;
        // device bytes of the painter's buffers plus those of its scene
        virtual long long device_bytes() const = 0;
        // Asks the passes in flight to take no more paths, as the reference's
        // painter threads test their stop flag before every pixel
        // (src/painter/painting/integrator_bpt.cpp:90-93); callable from any
        // thread while a pass runs.  The pass ends early with an incomplete
        // image, the next wait() reports the cancellation, and the painter
        // takes no more passes.
        virtual void cancel() = 0;
        virtual bool cancelled() const = 0;
        // After the passes enqueued so far (it waits for them): gives the
        // per-chunk path buffers back to the library's buffer cache and
        // returns their bytes; the next enqueue_passes allocates them again.
        // Images, samples and statistics stay.
        virtual long long release_scratch() = 0;
        // Progress within a pass: after the paths of each chunk of pixels are
        // traced, `callback(user, pass, pixels_done, pixels)` runs on a CUDA
        // host-callback thread (pass counted from 1; pixels: the pixels whose
        // paths the pass renders).  It must return quickly and call no CUDA
        // function.  nullptr: none.  Applies to the passes enqueued after it.
        using ProgressCallback = void (*)(void* user, long long pass, long long pixels_done, long long pixels);
        virtual void set_progress(ProgressCallback callback, void* user) = 0;
};

class Scene
{
public:
        virtual ~Scene() = default;

        virtual int dimension() const = 0;
        virtual int channels() const = 0;
        virtual bool double_precision() const = 0;

        virtual int add_hyperplane_parallelotope(double metalness, double roughness, const float* rgb, double alpha,
                                                 const double* org, const double* vectors) = 0;
        virtual int add_parallelotope(double metalness, double roughness, const float* rgb, double alpha,
                                      const double* org, const double* vectors) = 0;
        virtual int add_mesh_object(const float* points, long long point_count, const int* facets,
                                    long long facet_count, const double* matrix, const float* normals,
                                    float metalness, float roughness, const float* rgb, float alpha) = 0;
        virtual int add_mesh_file(const char* path, const double* matrix, float metalness, float roughness,
                                  const float* rgb, float alpha) = 0;
        virtual int add_mesh() = 0;
        virtual int add_mesh_data(long long vertex_count, const double* vertices, const double* normals,
                                  long long facet_count, const int* facets, const int* facet_materials,
                                  int material_count, const double* material_params, const float* material_colors) = 0;
        virtual int add_parallelotope_light(int shape, const double* direction, const float* rgb) = 0;
        virtual int add_ball_light(const double* center, const double* direction, double radius, const float* rgb) = 0;
        virtual void set_perspective_projector(const double* org, const double* dir, const double* axes,
                                               double fov_degrees, const int* size) = 0;
        virtual void set_parallel_projector(const double* org, const double* dir, const double* axes,
                                            double units_per_pixel, const int* size) = 0;
        virtual void set_background(const float* rgb) = 0;
        // 0: mesh BVHs built on the GPU (the default), 1: on the host
        virtual void set_bvh_builder(int builder) = 0;
        virtual void finalize() = 0;

        virtual long long pixel_count() const = 0;
        virtual int actual_spp(int samples_per_pixel) const = 0;
        virtual long long device_bytes() const = 0;
        virtual long long upload_bytes() const = 0;
        // host seconds of the build: [mesh ingestion, BVH builds, the rest of
        // finalize (device uploads, facet setup), total]
        virtual void build_seconds(double* out) const = 0;

        // max_depth bounds the BPT subpaths; the PT integrator ends its paths
        // by Russian roulette and ignores it
        // slab_end >= 0: a painter of the rows [slab_begin, slab_end) of the
        // last screen axis only (its paths, those of the rows either side,
        // and the estimator of its own pixels); its images are the slab's
        // pixel_sums: the type of the per-pixel radiance and weight sums,
        // PIXEL_SUMS_FLOAT (the reference's), PIXEL_SUMS_DOUBLE, or
        // PIXEL_SUMS_DEFAULT: float for a double-precision scene (its images
        // are the reference's), double for a single-precision one
        virtual std::unique_ptr<Painter> create_painter(int samples_per_pixel, int max_depth, std::uint32_t seed,
                                                        Integrator integrator = Integrator::BPT, int slab_begin = 0,
                                                        int slab_end = -1, bool flat_shading = false,
                                                        long long chunk_budget = 0, int pixel_sums = 0) = 0;
        // device bytes create_painter would allocate.  chunk_budget: bytes
        // for the buffers of one chunk of paths (0: a fifth of the device's
        // memory within [4, 32] GiB); the job server gives each of its slots
        // a share of its memory budget
        virtual long long painter_bytes(int samples_per_pixel, int max_depth,
                                        Integrator integrator = Integrator::BPT,
                                        long long chunk_budget = 0, int pixel_sums = 0) const = 0;

        // verification: closest hit (any == 0) or any hit of rays [n][2N]
        virtual void trace(const double* rays, long long count, int any, int* kind, int* index, double* t,
                           double* point) = 0;
        // the same query on device buffers the caller provides: launches the
        // query kernel on the legacy default stream and returns without
        // waiting; allocates nothing
        virtual void trace_device(const double* rays, long long count, int any, int* kind, int* index, double* t,
                                  double* point) const = 0;
        virtual void mesh_export(int mesh, long long* counts, double* planes, double* node_lo, double* node_hi,
                                 unsigned* node_info, unsigned* indices, int* normal_info) = 0;
        // the ingested mesh `mesh` on the host (no GPU needed): counts =
        // (vertices, facets, normals); vertices and normals [V][N] as the
        // painter keeps them, facets [F][N]; any pointer may be NULL
        virtual void ingested_mesh(int mesh, long long* counts, double* vertices, double* normals,
                                   int* facets) const = 0;
        virtual void brdf(int material, const double* n, const double* v, const double* l, float* f,
                          double* pdf) = 0;
        virtual void brdf_sample(int material, const double* n, const double* v, const std::uint32_t* seed,
                                 int seed_words, double* l, double* pdf, float* f) = 0;
        virtual void light_sample(int light, int kind, const std::uint32_t* seed, int seed_words,
                                  const double* point, double* out, float* radiance) = 0;
};

std::unique_ptr<Scene> make_scene_3(bool double_precision, bool spectrum);
std::unique_ptr<Scene> make_scene_4(bool double_precision, bool spectrum);
std::unique_ptr<Scene> make_scene_5(bool double_precision, bool spectrum);

// random-number kernels for verification (capi.cpp)
void test_pcg(const std::uint32_t* seed, int seed_words, int count, std::uint32_t* out);
void test_canonical(const std::uint32_t* seed, int seed_words, int count, int use_double, double* out);
int test_sj_points(int dimension, int use_double, int spp, const std::uint32_t* seed, int seed_words, double* out);
} // namespace nbpt
