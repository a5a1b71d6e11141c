// C ABI of the painter (include/nbpt.h): argument checks, error codes and
// the thread-local error message around the C++ scene/painter classes.
#include "../../include/nbpt.h"

#include "bvh_build.h"
#include "core.cuh"
#include "cuda_error.h"
#include "device_pool.h"
#include "mesh_files.h"
#include "painter_api.h"
#include "pass_stream.h"
#include "server.h"

#include <cuda_runtime.h>

#include <cmath>
#include <exception>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

struct nbpt_scene
{
        std::unique_ptr<nbpt::Scene> impl;
};

struct nbpt_painter
{
        std::unique_ptr<nbpt::Painter> impl;
        // pinned images of the pass worker, kept from one start to the next
        std::unique_ptr<nbpt::PassBuffers> buffers;
        // passes on a worker thread (nbpt_painter_start); destroyed first
        std::unique_ptr<nbpt::PassStream> stream;
};

struct nbpt_server
{
        std::unique_ptr<nbpt::Server> impl;
};

namespace
{
thread_local std::string g_error;

template <typename F>
int guarded(const F& f)
{
        try
        {
                return f();
        }
        catch (const nbpt::CudaError& e)
        {
                g_error = e.what();
                cudaGetLastError(); // a non-sticky error is cleared for the next call
                return NBPT_CUDA_ERROR;
        }
        catch (const std::exception& e)
        {
                g_error = e.what();
                return NBPT_ERROR;
        }
        catch (...)
        {
                g_error = "unknown error";
                return NBPT_ERROR;
        }
}

nbpt::Scene& scene_of(nbpt_scene* s)
{
        if (!s || !s->impl)
        {
                throw std::runtime_error("null scene");
        }
        return *s->impl;
}

nbpt::Painter& painter_of(nbpt_painter* p)
{
        if (!p || !p->impl)
        {
                throw std::runtime_error("null painter");
        }
        if (p->stream && p->stream->running())
        {
                throw std::runtime_error("the painter is running passes on its worker thread");
        }
        return *p->impl;
}

void require(const void* p, const char* what)
{
        if (!p)
        {
                throw std::runtime_error(std::string("null ") + what);
        }
}

nbpt::Server& server_of(nbpt_server* s)
{
        if (!s || !s->impl)
        {
                throw std::runtime_error("null server");
        }
        return *s->impl;
}

void copy_info(const nbpt::JobInfo& j, nbpt_job_info* info)
{
        if (!info)
        {
                return;
        }
        info->state = static_cast<int>(j.state);
        info->passes = j.passes;
        info->passes_done = j.passes_done;
        info->footprint = j.footprint;
        info->submitted = j.submitted;
        info->started = j.started;
        info->finished = j.finished;
        info->device_started = j.device_started;
        info->device_finished = j.device_finished;
}

void copy_statistics(const nbpt::Statistics& s, nbpt_statistics* statistics)
{
        statistics->pass_number = s.pass_number;
        statistics->pixel_count = s.pixel_count;
        statistics->ray_count = s.ray_count;
        statistics->sample_count = s.sample_count;
        statistics->previous_pass_duration = s.previous_pass_duration;
        statistics->paths_seconds = s.paths_seconds;
        statistics->nodes = s.nodes;
        statistics->facets = s.facets;
        statistics->shapes = s.shapes;
        statistics->kernel_launches = s.kernel_launches;
        statistics->nonfinite_samples = s.nonfinite_samples;
        statistics->stack_overflows = s.stack_overflows;
}

void require_device()
{
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        {
                cudaGetLastError();
                throw std::runtime_error("no CUDA device");
        }
}

__global__ void pcg_kernel(const std::uint32_t* seed, const int words, const int count, std::uint32_t* out)
{
        nbpt::Pcg g = nbpt::seed_seq_pcg(seed, words);
        for (int i = 0; i < count; ++i)
        {
                out[i] = g();
        }
}

__global__ void canonical_kernel(const std::uint32_t* seed, const int words, const int count, const int use_double,
                                 double* out)
{
        nbpt::Pcg g = nbpt::seed_seq_pcg(seed, words);
        for (int i = 0; i < count; ++i)
        {
                out[i] = use_double ? nbpt::uniform<double>(g, 0.0, 1.0)
                                    : static_cast<double>(nbpt::uniform<float>(g, 0.0f, 1.0f));
        }
}

template <typename T>
__global__ void sj_kernel(const std::uint32_t* seed, const int words, const int dimension, const int k,
                          const T* offsets, double* out)
{
        nbpt::Pcg g = nbpt::seed_seq_pcg(seed, words);
        int count = 1;
        for (int d = 0; d < dimension; ++d)
        {
                count *= k;
        }
        for (int s = 0; s < count; ++s)
        {
                int rest = s;
                for (int d = 0; d < dimension; ++d)
                {
                        const int idx = rest % k;
                        rest /= k;
                        const T a = offsets[idx];
                        const T b = offsets[idx + 1];
                        T v;
                        do
                        {
                                v = nbpt::uniform<T>(g, a, b);
                        } while (!(v < b));
                        out[s * dimension + d] = static_cast<double>(v);
                }
        }
}

template <typename X>
struct Buffer final
{
        X* p = nullptr;
        explicit Buffer(const std::size_t n)
        {
                nbpt::cuda_check(cudaMalloc(&p, n * sizeof(X)), "cudaMalloc");
        }
        ~Buffer()
        {
                cudaFree(p);
        }
};

template <typename T>
int sj_points(const int dimension, const int spp, const std::uint32_t* seed, const int words, double* out)
{
        const double v = std::pow(spp, 1.0 / dimension);
        int k = static_cast<int>(std::floor(v));
        long long p = 1;
        for (int i = 0; i < dimension; ++i)
        {
                p *= k;
        }
        if (p < spp)
        {
                k = static_cast<int>(std::ceil(v));
        }
        int count = 1;
        for (int i = 0; i < dimension; ++i)
        {
                count *= k;
        }
        if (!out)
        {
                return count;
        }
        std::vector<T> offsets(k + 1);
        const T size = (T(1) - T(0)) / static_cast<T>(k);
        offsets[0] = 0;
        for (int i = 1; i < k; ++i)
        {
                offsets[i] = T(0) + static_cast<T>(i) * size;
        }
        offsets[k] = 1;
        Buffer<std::uint32_t> d_seed(words);
        Buffer<T> d_offsets(k + 1);
        Buffer<double> d_out(static_cast<std::size_t>(count) * dimension);
        cudaMemcpy(d_seed.p, seed, words * sizeof(std::uint32_t), cudaMemcpyHostToDevice);
        cudaMemcpy(d_offsets.p, offsets.data(), (k + 1) * sizeof(T), cudaMemcpyHostToDevice);
        sj_kernel<T><<<1, 1>>>(d_seed.p, words, dimension, k, d_offsets.p, d_out.p);
        nbpt::cuda_check(cudaDeviceSynchronize(), "sj kernel");
        cudaMemcpy(out, d_out.p, static_cast<std::size_t>(count) * dimension * sizeof(double), cudaMemcpyDeviceToHost);
        return count;
}
} // namespace

extern "C"
{
const char* nbpt_last_error(void)
{
        return g_error.c_str();
}

long long nbpt_release_cached_memory(void)
{
        long long r = NBPT_ERROR;
        guarded(
                [&]
                {
                        r = static_cast<long long>(nbpt::pool::trim());
                        return 0;
                });
        return r;
}

int nbpt_device_count(void)
{
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess)
        {
                cudaGetLastError();
                return 0;
        }
        return count;
}

nbpt_scene* nbpt_scene_create(const int dimension, const int precision, const int color)
{
        nbpt_scene* out = nullptr;
        guarded(
                [&]
                {
                        if (precision != NBPT_FLOAT && precision != NBPT_DOUBLE)
                        {
                                throw std::runtime_error("precision must be NBPT_FLOAT or NBPT_DOUBLE");
                        }
                        if (color != NBPT_RGB && color != NBPT_SPECTRUM)
                        {
                                throw std::runtime_error("color must be NBPT_RGB or NBPT_SPECTRUM");
                        }
                        const bool d = precision == NBPT_DOUBLE;
                        const bool s = color == NBPT_SPECTRUM;
                        auto scene = std::make_unique<nbpt_scene>();
                        switch (dimension)
                        {
                        case 3:
                                scene->impl = nbpt::make_scene_3(d, s);
                                break;
                        case 4:
                                scene->impl = nbpt::make_scene_4(d, s);
                                break;
                        case 5:
                                scene->impl = nbpt::make_scene_5(d, s);
                                break;
                        default:
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                        out = scene.release();
                        return 0;
                });
        return out;
}

void nbpt_scene_destroy(nbpt_scene* scene)
{
        delete scene;
}

int nbpt_scene_add_hyperplane_parallelotope(
        nbpt_scene* scene,
        const double metalness,
        const double roughness,
        const float* rgb,
        const double alpha,
        const double* org,
        const double* vectors)
{
        return guarded(
                [&]
                {
                        require(rgb, "color");
                        require(org, "org");
                        require(vectors, "vectors");
                        return scene_of(scene).add_hyperplane_parallelotope(metalness, roughness, rgb, alpha, org, vectors);
                });
}

int nbpt_scene_add_parallelotope(
        nbpt_scene* scene,
        const double metalness,
        const double roughness,
        const float* rgb,
        const double alpha,
        const double* org,
        const double* vectors)
{
        return guarded(
                [&]
                {
                        require(rgb, "color");
                        require(org, "org");
                        require(vectors, "vectors");
                        return scene_of(scene).add_parallelotope(metalness, roughness, rgb, alpha, org, vectors);
                });
}

int nbpt_scene_add_mesh_object(
        nbpt_scene* scene,
        const float* points,
        const long long point_count,
        const int* facets,
        const long long facet_count,
        const double* matrix,
        const float* normals,
        const float metalness,
        const float roughness,
        const float* rgb,
        const float alpha)
{
        return guarded(
                [&]
                {
                        require(points, "points");
                        require(facets, "facets");
                        require(matrix, "matrix");
                        require(rgb, "color");
                        return scene_of(scene).add_mesh_object(
                                points, point_count, facets, facet_count, matrix, normals, metalness, roughness, rgb,
                                alpha);
                });
}

int nbpt_scene_add_mesh_file(
        nbpt_scene* scene,
        const char* path,
        const double* matrix,
        const float metalness,
        const float roughness,
        const float* rgb,
        const float alpha)
{
        return guarded(
                [&]
                {
                        require(path, "path");
                        require(matrix, "matrix");
                        require(rgb, "color");
                        return scene_of(scene).add_mesh_file(path, matrix, metalness, roughness, rgb, alpha);
                });
}

int nbpt_mesh_file_dimension(const char* path)
{
        return guarded(
                [&]
                {
                        require(path, "path");
                        const int n = nbpt::host::mesh_file_dimension(path);
                        if (n == 0)
                        {
                                throw std::runtime_error(std::string("Not an OBJ or STL file name: ") + path);
                        }
                        return n;
                });
}

int nbpt_scene_add_mesh(nbpt_scene* scene)
{
        return guarded(
                [&]
                {
                        return scene_of(scene).add_mesh();
                });
}

int nbpt_scene_add_mesh_data(
        nbpt_scene* scene,
        const long long vertex_count,
        const double* vertices,
        const double* normals,
        const long long facet_count,
        const int* facets,
        const int* facet_materials,
        const int material_count,
        const double* material_params,
        const float* material_colors)
{
        return guarded(
                [&]
                {
                        require(vertices, "vertices");
                        require(facets, "facets");
                        require(facet_materials, "facet materials");
                        require(material_params, "material parameters");
                        require(material_colors, "material colors");
                        return scene_of(scene).add_mesh_data(
                                vertex_count, vertices, normals, facet_count, facets, facet_materials, material_count,
                                material_params, material_colors);
                });
}

int nbpt_scene_add_parallelotope_light(nbpt_scene* scene, const int shape, const double* direction, const float* rgb)
{
        return guarded(
                [&]
                {
                        require(direction, "direction");
                        require(rgb, "radiance");
                        return scene_of(scene).add_parallelotope_light(shape, direction, rgb);
                });
}

int nbpt_scene_add_ball_light(
        nbpt_scene* scene,
        const double* center,
        const double* direction,
        const double radius,
        const float* rgb)
{
        return guarded(
                [&]
                {
                        require(center, "center");
                        require(direction, "direction");
                        require(rgb, "radiance");
                        return scene_of(scene).add_ball_light(center, direction, radius, rgb);
                });
}

int nbpt_scene_set_perspective_projector(
        nbpt_scene* scene,
        const double* org,
        const double* dir,
        const double* axes,
        const double fov_degrees,
        const int* size)
{
        return guarded(
                [&]
                {
                        require(org, "org");
                        require(dir, "dir");
                        require(axes, "axes");
                        require(size, "size");
                        scene_of(scene).set_perspective_projector(org, dir, axes, fov_degrees, size);
                        return 0;
                });
}

int nbpt_scene_set_parallel_projector(
        nbpt_scene* scene,
        const double* org,
        const double* dir,
        const double* axes,
        const double units_per_pixel,
        const int* size)
{
        return guarded(
                [&]
                {
                        require(org, "org");
                        require(dir, "dir");
                        require(axes, "axes");
                        require(size, "size");
                        scene_of(scene).set_parallel_projector(org, dir, axes, units_per_pixel, size);
                        return 0;
                });
}

int nbpt_scene_set_background(nbpt_scene* scene, const float* rgb)
{
        return guarded(
                [&]
                {
                        require(rgb, "background");
                        scene_of(scene).set_background(rgb);
                        return 0;
                });
}

int nbpt_scene_finalize(nbpt_scene* scene)
{
        return guarded(
                [&]
                {
                        require_device();
                        scene_of(scene).finalize();
                        return 0;
                });
}

long long nbpt_scene_pixel_count(const nbpt_scene* scene)
{
        long long r = NBPT_ERROR;
        guarded(
                [&]
                {
                        r = scene_of(const_cast<nbpt_scene*>(scene)).pixel_count();
                        return 0;
                });
        return r;
}

int nbpt_scene_actual_spp(const nbpt_scene* scene, const int samples_per_pixel)
{
        return guarded(
                [&]
                {
                        return scene_of(const_cast<nbpt_scene*>(scene)).actual_spp(samples_per_pixel);
                });
}

long long nbpt_scene_device_bytes(const nbpt_scene* scene)
{
        long long r = NBPT_ERROR;
        guarded(
                [&]
                {
                        r = scene_of(const_cast<nbpt_scene*>(scene)).device_bytes();
                        return 0;
                });
        return r;
}

long long nbpt_scene_upload_bytes(const nbpt_scene* scene)
{
        long long r = NBPT_ERROR;
        guarded(
                [&]
                {
                        r = scene_of(const_cast<nbpt_scene*>(scene)).upload_bytes();
                        return 0;
                });
        return r;
}

int nbpt_scene_set_bvh_builder(nbpt_scene* scene, const int builder)
{
        return guarded(
                [&]
                {
                        scene_of(scene).set_bvh_builder(builder);
                        return 0;
                });
}

int nbpt_scene_build_seconds(const nbpt_scene* scene, double* seconds)
{
        return guarded(
                [&]
                {
                        if (!seconds)
                        {
                                throw std::runtime_error("null output");
                        }
                        scene_of(const_cast<nbpt_scene*>(scene)).build_seconds(seconds);
                        return 0;
                });
}

nbpt_painter* nbpt_painter_create(nbpt_scene* scene, const int samples_per_pixel, const int max_depth, const unsigned seed)
{
        nbpt_painter* out = nullptr;
        guarded(
                [&]
                {
                        auto p = std::make_unique<nbpt_painter>();
                        p->impl = scene_of(scene).create_painter(samples_per_pixel, max_depth, seed);
                        out = p.release();
                        return 0;
                });
        return out;
}

nbpt_painter* nbpt_painter_create_integrator(
        nbpt_scene* scene,
        const int integrator,
        const int samples_per_pixel,
        const int max_depth,
        const unsigned seed)
{
        return nbpt_painter_create_slab(scene, integrator, samples_per_pixel, max_depth, seed, 0, -1);
}

nbpt_painter* nbpt_painter_create_options(nbpt_scene* scene, const nbpt_painter_options* options)
{
        nbpt_painter* out = nullptr;
        guarded(
                [&]
                {
                        require(options, "options");
                        const nbpt_painter_options& o = *options;
                        if (o.integrator != NBPT_INTEGRATOR_BPT && o.integrator != NBPT_INTEGRATOR_PT)
                        {
                                throw std::runtime_error("Unknown integrator " + std::to_string(o.integrator));
                        }
                        if (o.chunk_budget < 0)
                        {
                                throw std::runtime_error("chunk budget " + std::to_string(o.chunk_budget) +
                                                         " is negative");
                        }
                        auto p = std::make_unique<nbpt_painter>();
                        p->impl = scene_of(scene).create_painter(o.samples_per_pixel, o.max_depth, o.seed,
                                                                 static_cast<nbpt::Integrator>(o.integrator),
                                                                 o.slab_begin, o.slab_end, o.flat_shading != 0,
                                                                 o.chunk_budget, o.pixel_sums);
                        out = p.release();
                        return 0;
                });
        return out;
}

nbpt_painter* nbpt_painter_create_slab(
        nbpt_scene* scene,
        const int integrator,
        const int samples_per_pixel,
        const int max_depth,
        const unsigned seed,
        const int slab_begin,
        const int slab_end)
{
        nbpt_painter* out = nullptr;
        guarded(
                [&]
                {
                        if (integrator != NBPT_INTEGRATOR_BPT && integrator != NBPT_INTEGRATOR_PT)
                        {
                                throw std::runtime_error("Unknown integrator " + std::to_string(integrator));
                        }
                        auto p = std::make_unique<nbpt_painter>();
                        p->impl = scene_of(scene).create_painter(samples_per_pixel, max_depth, seed,
                                                                 static_cast<nbpt::Integrator>(integrator), slab_begin,
                                                                 slab_end, false);
                        out = p.release();
                        return 0;
                });
        return out;
}

int nbpt_painter_start(
        nbpt_painter* painter,
        const int max_pass_count,
        const nbpt_pass_callback on_pass,
        const nbpt_error_callback on_error,
        void* const user)
{
        return guarded(
                [&]
                {
                        nbpt::Painter& p = painter_of(painter);
                        if (!on_pass)
                        {
                                throw std::runtime_error("null pass callback");
                        }
                        if (max_pass_count < 0)
                        {
                                throw std::runtime_error("pass count must not be negative");
                        }
                        painter->stream.reset();
                        if (!painter->buffers)
                        {
                                painter->buffers = std::make_unique<nbpt::PassBuffers>(p.statistics().pixel_count);
                        }
                        painter->stream = std::make_unique<nbpt::PassStream>(
                                &p, painter->buffers.get(), max_pass_count, on_pass, on_error, user);
                        return 0;
                });
}

int nbpt_painter_stop(nbpt_painter* painter)
{
        return guarded(
                [&]
                {
                        if (!painter)
                        {
                                throw std::runtime_error("null painter");
                        }
                        if (painter->stream)
                        {
                                painter->stream->stop();
                        }
                        return 0;
                });
}

int nbpt_painter_join(nbpt_painter* painter)
{
        return guarded(
                [&]
                {
                        if (!painter)
                        {
                                throw std::runtime_error("null painter");
                        }
                        if (painter->stream)
                        {
                                painter->stream->join();
                        }
                        return 0;
                });
}

int nbpt_painter_is_running(const nbpt_painter* painter)
{
        if (!painter)
        {
                g_error = "null painter";
                return NBPT_ERROR;
        }
        return painter->stream && painter->stream->running() ? 1 : 0;
}

void nbpt_painter_destroy(nbpt_painter* painter)
{
        delete painter;
}

int nbpt_painter_enqueue(nbpt_painter* painter, const int passes)
{
        return guarded(
                [&]
                {
                        if (passes < 1)
                        {
                                throw std::runtime_error("pass count must be greater than 0");
                        }
                        painter_of(painter).enqueue_passes(passes);
                        return 0;
                });
}

int nbpt_painter_wait(nbpt_painter* painter)
{
        return guarded(
                [&]
                {
                        painter_of(painter).wait();
                        return 0;
                });
}

int nbpt_painter_images(nbpt_painter* painter, float* rgb, float* rgba)
{
        return guarded(
                [&]
                {
                        painter_of(painter).images(rgb, rgba);
                        return 0;
                });
}

int nbpt_painter_samples(nbpt_painter* painter, double* points, float* colors, unsigned char* valid)
{
        return guarded(
                [&]
                {
                        painter_of(painter).samples(points, colors, valid);
                        return 0;
                });
}

int nbpt_painter_statistics(nbpt_painter* painter, nbpt_statistics* statistics)
{
        return guarded(
                [&]
                {
                        require(statistics, "statistics");
                        copy_statistics(painter_of(painter).statistics(), statistics);
                        return 0;
                });
}

void* nbpt_painter_stream(nbpt_painter* painter)
{
        void* s = nullptr;
        guarded(
                [&]
                {
                        s = painter_of(painter).stream();
                        return 0;
                });
        return s;
}

int nbpt_painter_set_progress(nbpt_painter* painter, const nbpt_progress_callback on_chunk, void* const user)
{
        return guarded(
                [&]
                {
                        painter_of(painter).set_progress(on_chunk, user);
                        return 0;
                });
}

int nbpt_painter_cancel(nbpt_painter* painter)
{
        return guarded(
                [&]
                {
                        if (!painter || !painter->impl)
                        {
                                throw std::runtime_error("null painter");
                        }
                        // allowed while the worker runs: Painter::cancel is thread safe
                        if (painter->stream)
                        {
                                painter->stream->request_stop();
                        }
                        painter->impl->cancel();
                        return 0;
                });
}

nbpt_server* nbpt_server_create(const int max_jobs, const long long memory_budget)
{
        nbpt_server* out = nullptr;
        guarded(
                [&]
                {
                        require_device();
                        auto s = std::make_unique<nbpt_server>();
                        s->impl = std::make_unique<nbpt::Server>(max_jobs, memory_budget);
                        out = s.release();
                        return 0;
                });
        return out;
}

void nbpt_server_destroy(nbpt_server* server)
{
        delete server;
}


long long nbpt_server_submit(nbpt_server* server, nbpt_painter* painter, const int passes)
{
        long long id = NBPT_ERROR;
        guarded(
                [&]
                {
                        id = server_of(server).submit(&painter_of(painter), passes);
                        return 0;
                });
        return id;
}

long long nbpt_server_submit_render(nbpt_server* server, nbpt_scene* scene, const int samples_per_pixel,
                                    const int max_depth, const unsigned seed, const int passes)
{
        long long id = NBPT_ERROR;
        guarded(
                [&]
                {
                        id = server_of(server).submit_render(&scene_of(scene), samples_per_pixel, max_depth, seed,
                                                             passes);
                        return 0;
                });
        return id;
}

int nbpt_server_images(nbpt_server* server, const long long job, float* rgb, float* rgba)
{
        return guarded(
                [&]
                {
                        server_of(server).images(job, rgb, rgba);
                        return 0;
                });
}

int nbpt_server_statistics(nbpt_server* server, const long long job, nbpt_statistics* statistics)
{
        return guarded(
                [&]
                {
                        require(statistics, "statistics");
                        copy_statistics(server_of(server).statistics(job), statistics);
                        return 0;
                });
}

int nbpt_server_release(nbpt_server* server, const long long job)
{
        return guarded(
                [&]
                {
                        server_of(server).release(job);
                        return 0;
                });
}

int nbpt_server_job(nbpt_server* server, const long long job, nbpt_job_info* info)
{
        return guarded(
                [&]
                {
                        require(info, "info");
                        copy_info(server_of(server).info(job), info);
                        return 0;
                });
}

int nbpt_server_wait(nbpt_server* server, const long long job, nbpt_job_info* info)
{
        return guarded(
                [&]
                {
                        const nbpt::JobInfo j = server_of(server).wait(job);
                        copy_info(j, info);
                        if (j.state == nbpt::JobState::FAILED)
                        {
                                throw std::runtime_error("job " + std::to_string(job) + " failed: " + j.error);
                        }
                        return 0;
                });
}

double nbpt_server_time(nbpt_server* server)
{
        double t = -1;
        guarded(
                [&]
                {
                        t = server_of(server).now();
                        return 0;
                });
        return t;
}

int nbpt_server_cancel(nbpt_server* server, const long long job)
{
        return guarded(
                [&]
                {
                        server_of(server).cancel(job);
                        return 0;
                });
}

int nbpt_server_set_chunk_budget(nbpt_server* server, const long long bytes)
{
        return guarded(
                [&]
                {
                        server_of(server).set_chunk_budget(bytes);
                        return 0;
                });
}

long long nbpt_server_chunk_budget(const nbpt_server* server)
{
        long long out = -1;
        guarded(
                [&]
                {
                        out = server_of(const_cast<nbpt_server*>(server)).chunk_budget();
                        return 0;
                });
        return out;
}

int nbpt_test_server_hold(nbpt_server* server, const int hold)
{
        return guarded(
                [&]
                {
                        server_of(server).hold_admission(hold != 0);
                        return 0;
                });
}

int nbpt_test_server_fail_allocations(nbpt_server* server, const int count)
{
        return guarded(
                [&]
                {
                        server_of(server).fail_next_creations(count);
                        return 0;
                });
}

int nbpt_scene_trace(
        nbpt_scene* scene,
        const double* rays,
        const long long count,
        const int any,
        int* kind,
        int* index,
        double* t,
        double* point)
{
        return guarded(
                [&]
                {
                        require(rays, "rays");
                        require(kind, "kind");
                        if (!any)
                        {
                                require(index, "index");
                                require(t, "t");
                                require(point, "point");
                        }
                        scene_of(scene).trace(rays, count, any, kind, index, t, point);
                        return 0;
                });
}

// ---------------------------------------------------------------------------
// Ray queries without allocation (nbpt_scene_trace_noalloc)
//
// The rays and results of one call pass through a fixed scratch array in
// device memory, defined here at file scope, instead of buffers allocated per
// call.  Its layout holds NBPT_TRACE_NOALLOC_MAX_RAYS rays of the largest
// dimension (5): origins and directions, then kind, index, distance and
// point, each part starting on a 256-byte boundary.  Nothing in it needs to
// start at zero: for every one of the `count` rays of a call the query
// kernel writes each result slot that is read back.

namespace
{
constexpr long long NOALLOC_MAX_N = 5;
constexpr long long NOALLOC_RAYS = NBPT_TRACE_NOALLOC_MAX_RAYS;

constexpr long long align256(const long long bytes)
{
        return (bytes + 255) / 256 * 256;
}

constexpr long long NOALLOC_RAYS_OFFSET = 0;
constexpr long long NOALLOC_KIND_OFFSET = NOALLOC_RAYS_OFFSET + align256(NOALLOC_RAYS * 2 * NOALLOC_MAX_N * 8);
constexpr long long NOALLOC_INDEX_OFFSET = NOALLOC_KIND_OFFSET + align256(NOALLOC_RAYS * 4);
constexpr long long NOALLOC_T_OFFSET = NOALLOC_INDEX_OFFSET + align256(NOALLOC_RAYS * 4);
constexpr long long NOALLOC_POINT_OFFSET = NOALLOC_T_OFFSET + align256(NOALLOC_RAYS * 8);
constexpr long long NOALLOC_BYTES = NOALLOC_POINT_OFFSET + align256(NOALLOC_RAYS * NOALLOC_MAX_N * 8);
static_assert(NOALLOC_BYTES == 2228224, "the scratch size stated in nbpt.h");

// one copy per device (each device's context loads the module's own copy)
static __device__ __align__(256) unsigned char g_trace_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_trace_scratch_mutex;
unsigned char* g_trace_scratch_address[NOALLOC_MAX_DEVICES] = {};

// The scratch's device address on the current device, looked up once per
// device (cudaGetSymbolAddress) and cached.
unsigned char* trace_scratch()
{
        int device = 0;
        const cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess)
        {
                throw nbpt::CudaError("cudaGetDevice", e);
        }
        if (device < 0 || device >= NOALLOC_MAX_DEVICES)
        {
                throw std::runtime_error("nbpt_scene_trace_noalloc: device ordinal " + std::to_string(device) +
                                         " beyond the " + std::to_string(NOALLOC_MAX_DEVICES) + " devices it serves");
        }
        const std::lock_guard lock(g_trace_scratch_mutex);
        if (!g_trace_scratch_address[device])
        {
                void* address = nullptr;
                const cudaError_t r = cudaGetSymbolAddress(&address, g_trace_scratch);
                if (r != cudaSuccess || !address)
                {
                        throw nbpt::CudaError("cudaGetSymbolAddress of the trace scratch",
                                              r != cudaSuccess ? r : cudaErrorInvalidSymbol);
                }
                g_trace_scratch_address[device] = static_cast<unsigned char*>(address);
        }
        return g_trace_scratch_address[device];
}

void copy_checked(void* to, const void* from, const long long bytes, const cudaMemcpyKind kind)
{
        const cudaError_t e = cudaMemcpy(to, from, static_cast<std::size_t>(bytes), kind);
        if (e != cudaSuccess)
        {
                throw nbpt::CudaError("cudaMemcpy", e);
        }
}
} // namespace

int nbpt_scene_trace_noalloc(
        nbpt_scene* scene,
        const double* rays,
        const long long count,
        const int any,
        int* kind,
        int* index,
        double* t,
        double* point)
{
        return guarded(
                [&]
                {
                        const nbpt::Scene& sc = scene_of(scene);
                        require(rays, "rays");
                        require(kind, "kind");
                        if (!any)
                        {
                                require(index, "index");
                                require(t, "t");
                                require(point, "point");
                        }
                        if (count < 0)
                        {
                                throw std::runtime_error("nbpt_scene_trace_noalloc: negative ray count");
                        }
                        if (count > NOALLOC_RAYS)
                        {
                                throw std::runtime_error(
                                        "nbpt_scene_trace_noalloc: " + std::to_string(count) +
                                        " rays exceed its fixed scratch of " + std::to_string(NOALLOC_RAYS) +
                                        " rays per call; split the batch or use nbpt_scene_trace");
                        }
                        if (count == 0)
                        {
                                return 0;
                        }
                        const long long n = sc.dimension();
                        unsigned char* const base = trace_scratch();
                        double* const d_rays = reinterpret_cast<double*>(base + NOALLOC_RAYS_OFFSET);
                        int* const d_kind = reinterpret_cast<int*>(base + NOALLOC_KIND_OFFSET);
                        int* const d_index = reinterpret_cast<int*>(base + NOALLOC_INDEX_OFFSET);
                        double* const d_t = reinterpret_cast<double*>(base + NOALLOC_T_OFFSET);
                        double* const d_point = reinterpret_cast<double*>(base + NOALLOC_POINT_OFFSET);

                        copy_checked(d_rays, rays, count * 2 * n * 8, cudaMemcpyHostToDevice);
                        sc.trace_device(d_rays, count, any, d_kind, d_index, d_t, d_point);
                        // copies on the legacy default stream wait for the query kernel
                        copy_checked(kind, d_kind, count * 4, cudaMemcpyDeviceToHost);
                        if (!any)
                        {
                                copy_checked(index, d_index, count * 4, cudaMemcpyDeviceToHost);
                                copy_checked(t, d_t, count * 8, cudaMemcpyDeviceToHost);
                                copy_checked(point, d_point, count * n * 8, cudaMemcpyDeviceToHost);
                        }
                        return 0;
                });
}

int nbpt_scene_ingested_mesh(nbpt_scene* scene, const int mesh, long long* counts, double* vertices, double* normals,
                             int* facets)
{
        return guarded(
                [&]
                {
                        scene_of(scene).ingested_mesh(mesh, counts, vertices, normals, facets);
                        return 0;
                });
}

int nbpt_scene_mesh_export(
        nbpt_scene* scene,
        const int mesh,
        long long* counts,
        double* planes,
        double* node_lo,
        double* node_hi,
        unsigned* node_info,
        unsigned* indices,
        int* normal_info)
{
        return guarded(
                [&]
                {
                        require(counts, "counts");
                        scene_of(scene).mesh_export(mesh, counts, planes, node_lo, node_hi, node_info, indices, normal_info);
                        return 0;
                });
}

int nbpt_scene_brdf(
        nbpt_scene* scene,
        const int material,
        const double* n,
        const double* v,
        const double* l,
        float* f,
        double* pdf)
{
        return guarded(
                [&]
                {
                        scene_of(scene).brdf(material, n, v, l, f, pdf);
                        return 0;
                });
}

int nbpt_scene_brdf_sample(
        nbpt_scene* scene,
        const int material,
        const double* n,
        const double* v,
        const unsigned* seed,
        const int seed_words,
        double* l,
        double* pdf,
        float* f)
{
        return guarded(
                [&]
                {
                        scene_of(scene).brdf_sample(material, n, v, seed, seed_words, l, pdf, f);
                        return 0;
                });
}

int nbpt_scene_light_sample(
        nbpt_scene* scene,
        const int light,
        const int kind,
        const unsigned* seed,
        const int seed_words,
        const double* point,
        double* out,
        float* radiance)
{
        return guarded(
                [&]
                {
                        scene_of(scene).light_sample(light, kind, seed, seed_words, point, out, radiance);
                        return 0;
                });
}

int nbpt_test_pcg(const unsigned* seed, const int seed_words, const int count, unsigned* out)
{
        return guarded(
                [&]
                {
                        require_device();
                        Buffer<std::uint32_t> d_seed(seed_words);
                        Buffer<std::uint32_t> d_out(count);
                        cudaMemcpy(d_seed.p, seed, seed_words * sizeof(std::uint32_t), cudaMemcpyHostToDevice);
                        pcg_kernel<<<1, 1>>>(d_seed.p, seed_words, count, d_out.p);
                        nbpt::cuda_check(cudaDeviceSynchronize(), "pcg kernel");
                        cudaMemcpy(out, d_out.p, count * sizeof(std::uint32_t), cudaMemcpyDeviceToHost);
                        return 0;
                });
}

int nbpt_test_canonical(const unsigned* seed, const int seed_words, const int count, const int use_double, double* out)
{
        return guarded(
                [&]
                {
                        require_device();
                        Buffer<std::uint32_t> d_seed(seed_words);
                        Buffer<double> d_out(count);
                        cudaMemcpy(d_seed.p, seed, seed_words * sizeof(std::uint32_t), cudaMemcpyHostToDevice);
                        canonical_kernel<<<1, 1>>>(d_seed.p, seed_words, count, use_double, d_out.p);
                        nbpt::cuda_check(cudaDeviceSynchronize(), "canonical kernel");
                        cudaMemcpy(out, d_out.p, count * sizeof(double), cudaMemcpyDeviceToHost);
                        return 0;
                });
}

int nbpt_test_sj_points(
        const int dimension,
        const int use_double,
        const int spp,
        const unsigned* seed,
        const int seed_words,
        double* out)
{
        return guarded(
                [&]
                {
                        if (dimension < 2 || dimension > 4 || spp < 1)
                        {
                                throw std::runtime_error("bad sampler arguments");
                        }
                        if (out)
                        {
                                require_device();
                        }
                        return use_double ? sj_points<double>(dimension, spp, seed, seed_words, out)
                                          : sj_points<float>(dimension, spp, seed, seed_words, out);
                });
}
}

namespace
{
template <int N, typename T>
void host_bvh_depth(const double* vertices, const long long vertex_count, const int* facets,
                    const long long facet_count, long long* nodes, int* depth)
{
        std::vector<T> v(static_cast<std::size_t>(vertex_count) * N);
        for (std::size_t i = 0; i < v.size(); ++i)
        {
                v[i] = static_cast<T>(vertices[i]);
        }
        std::vector<int> f(facets, facets + facet_count * N);
        for (const int k : f)
        {
                if (k < 0 || k >= vertex_count)
                {
                        throw std::runtime_error("facet vertex index out of range");
                }
        }
        const nbpt::host::BuiltBvh<N, T> bvh = nbpt::host::build_facet_bvh<N, T>(v, f);
        if (nodes)
        {
                *nodes = static_cast<long long>(bvh.count.size());
        }
        if (depth)
        {
                *depth = bvh.depth;
        }
}
} // namespace

int nbpt_test_bvh_build(const int dimension, const int precision, const double* vertices, const long long vertex_count,
                        const int* facets, const long long facet_count, long long* nodes, int* depth)
{
        return guarded(
                [&]
                {
                        require(vertices, "vertices");
                        require(facets, "facets");
                        if (facet_count <= 0 || vertex_count <= 0)
                        {
                                throw std::runtime_error("No objects to build BVH");
                        }
                        const bool d = precision == NBPT_DOUBLE;
                        switch (dimension)
                        {
                        case 3:
                                d ? host_bvh_depth<3, double>(vertices, vertex_count, facets, facet_count, nodes, depth)
                                  : host_bvh_depth<3, float>(vertices, vertex_count, facets, facet_count, nodes, depth);
                                break;
                        case 4:
                                d ? host_bvh_depth<4, double>(vertices, vertex_count, facets, facet_count, nodes, depth)
                                  : host_bvh_depth<4, float>(vertices, vertex_count, facets, facet_count, nodes, depth);
                                break;
                        case 5:
                                d ? host_bvh_depth<5, double>(vertices, vertex_count, facets, facet_count, nodes, depth)
                                  : host_bvh_depth<5, float>(vertices, vertex_count, facets, facet_count, nodes, depth);
                                break;
                        default:
                                throw std::runtime_error("dimension must be 3, 4 or 5");
                        }
                        return 0;
                });
}
