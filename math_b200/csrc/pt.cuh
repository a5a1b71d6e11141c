// Path tracing with next-event estimation for one path: the reference
// painter's other integrator (Integrator::PT).
//
// Mirrors src/painter/integrators/pt/{pt.cpp, direct_lighting.cpp} and
// src/painter/integrators/com/surface_sample.cpp, with the parallelotope and
// ball lights' arrive_info (src/painter/lights/parallelotope_light.cpp:92-115,
// ball_light.cpp:90-113).  Russian roulette weighs the path by the
// luminance of all its colour channels, so a path carries its full colour
// (one thread per path; no channel-0 tape as for BPT).
#pragma once

#include "bpt.cuh"
#include "core.cuh"
#include "geometry.cuh"
#include "kernels.cuh"
#include "scene.cuh"
#include "shading.cuh"

namespace nbpt
{
// std::bernoulli_distribution(p)(engine): one canonical double below p
NBPT_HD bool bernoulli(Pcg& g, const double p)
{
        return canonical<double>(g) < p;
}

// sampling::mis::power_heuristic with one sample each (src/sampling/mis.h:34-58)
template <typename T>
NBPT_HD T power_heuristic(const T f_pdf, const T g_pdf)
{
        const T f = square(1 * f_pdf);
        const T g = square(1 * g_pdf);
        return f / (f + g);
}

// A path longer than this many bounces is cut (Russian roulette ends a path
// with probability at least 0.05 per bounce from the fourth on, so no path
// of the reference gets near it).
inline constexpr int PT_MAX_BOUNCES = 100000;

template <int N, typename T, int C>
struct Pt final
{
        const SceneQueries<N, T, C>& q;
        const DeviceScene<N, T, C>& s;
        Pcg& g;
        const float* cie_y;
        Bpt<N, T, C> b; // light samples and visibility

        // LightSource::arrive_info: the light seen from `point` in direction
        // `l`; false when not usable.
        __device__ bool arrive_info(const Light<N, T, C>& light, const Vec<N, T>& point, const Vec<N, T>& l, T& pdf,
                                    T& distance) const
        {
                if (!(dot(light.normal, point - light.org) > 0))
                {
                        return false;
                }
                const Ray<N, T> ray = Ray<N, T>::make(point, l);
                T t;
                if (light.type == static_cast<int>(LightType::PARALLELOTOPE))
                {
                        t = s.flat[light.shape].shape.intersect(ray);
                        if (!(t > 0))
                        {
                                return false;
                        }
                }
                else
                {
                        // HyperplaneBall::intersect (src/geometry/spatial/hyperplane_ball.h:54-69)
                        Plane<N, T> plane;
                        plane.n = light.normal;
                        plane.d = dot(plane.n, light.org);
                        t = plane.intersect(ray);
                        if (!(t > 0))
                        {
                                return false;
                        }
                        const Vec<N, T> p = ray.point(t);
                        if (!((p - light.org).norm_squared() < light.radius_squared))
                        {
                                return false;
                        }
                }
                const T cos = -dot(ray.dir, light.normal);
                pdf = area_pdf_to_solid_angle_pdf<N>(light.pdf, cos, t);
                distance = t;
                return pdf > 0 && !light.radiance.is_black();
        }

        // sample_light_with_mis (direct_lighting.cpp:59-99); the lights here
        // are area lights (is_delta() false)
        NBPT_CALL bool light_with_mis(const Light<N, T, C>& light, const Hit<N, T>& surface, const Vec<N, T>& v,
                                      const Normals<N, T>& normals, Color<C>& out) const
        {
                const Vec<N, T>& n = normals.shading;
                const ArriveSample<N, T, C> sample = b.arrive_sample(light, surface.point);
                if (!sample.usable())
                {
                        return false;
                }
                const Vec<N, T>& l = sample.l;
                const T n_l = dot(n, l);
                if (!(n_l > 0))
                {
                        return false;
                }
                if (b.occluded_ray(normals, Ray<N, T>::make(surface.point, l), sample.distance))
                {
                        return false;
                }
                const Material<T, C>& m = s.materials[q.material(surface)];
                const Color<C> brdf = brdf_f(s.shading, m.roughness, m.f0, m.rho_ss, n, v, l);
                const T pdf = brdf_pdf(s.shading, m.roughness, n, v, l);
                const T weight = power_heuristic(sample.pdf, pdf);
                out = brdf * sample.radiance * static_cast<float>(weight * n_l / sample.pdf);
                return true;
        }

        // sample_surface_with_mis (direct_lighting.cpp:101-147); no shape
        // here is specular
        NBPT_CALL bool surface_with_mis(const Light<N, T, C>& light, const Hit<N, T>& surface, const Vec<N, T>& v,
                                        const Normals<N, T>& normals, Color<C>& out) const
        {
                const Vec<N, T>& n = normals.shading;
                const Material<T, C>& m = s.materials[q.material(surface)];
                const BrdfSample<N, C, T> sample = brdf_sample<N>(g, s.shading, m.roughness, m.f0, m.rho_ss, n, v);
                if (!(sample.pdf > 0 && !sample.brdf.is_black()))
                {
                        return false;
                }
                const Vec<N, T>& l = sample.l;
                const T n_l = dot(n, l);
                if (!(n_l > 0))
                {
                        return false;
                }
                T light_pdf;
                T distance;
                if (!arrive_info(light, surface.point, l, light_pdf, distance))
                {
                        return false;
                }
                if (b.occluded_ray(normals, Ray<N, T>::make(surface.point, l), distance))
                {
                        return false;
                }
                const T weight = power_heuristic(sample.pdf, light_pdf);
                out = sample.brdf * light.radiance * static_cast<float>(weight * n_l / sample.pdf);
                return true;
        }

        // terminate (pt.cpp:43-66)
        __device__ bool terminate(const int depth, Color<C>& beta) const
        {
                if (depth < 4)
                {
                        return false;
                }
                const float lum = luminance(beta, cie_y);
                if (!(lum > 0))
                {
                        return true;
                }
                constexpr float MIN = 0.05f;
                constexpr float MAX = 0.95f;
                const float x = 1 - lum;
                const float p = (x < MIN) ? MIN : ((MAX < x) ? MAX : x);
                if (bernoulli(g, p))
                {
                        return true;
                }
                const float k = 1 - p;
#pragma unroll 8
                for (int i = 0; i < C; ++i)
                {
                        beta.c[i] /= k;
                }
                return false;
        }

        // one bounce (pt.cpp:68-111): false when the path ends
        NBPT_CALL bool step(const int depth, Ray<N, T>& ray, Hit<N, T>& surface, Normals<N, T>& normals,
                            Color<C>& color, Color<C>& beta) const
        {
                const Vec<N, T> v = -ray.dir;
                if (dot(normals.shading, v) <= 0)
                {
                        return false;
                }

                // direct_lighting (direct_lighting.cpp:150-167): both
                // estimates of every light, summed in that order
                bool lit = false;
                Color<C> direct;
                for (int k = 0; k < s.light_count; ++k)
                {
                        const Light<N, T, C>& light = s.lights[k];
                        Color<C> c;
                        if (light_with_mis(light, surface, v, normals, c))
                        {
                                direct = lit ? direct + c : c;
                                lit = true;
                        }
                        if (surface_with_mis(light, surface, v, normals, c))
                        {
                                direct = lit ? direct + c : c;
                                lit = true;
                        }
                }
                if (lit)
                {
#pragma unroll 8
                        for (int i = 0; i < C; ++i)
                        {
                                color.c[i] += beta.c[i] * direct.c[i];
                        }
                }

                // com::surface_sample (surface_sample.cpp:31-70)
                const Vec<N, T>& n = normals.shading;
                const Material<T, C>& m = s.materials[q.material(surface)];
                const BrdfSample<N, C, T> sample = brdf_sample<N>(g, s.shading, m.roughness, m.f0, m.rho_ss, n, v);
                if (!(sample.pdf > 0 && !sample.brdf.is_black()))
                {
                        return false;
                }
                if (dot(sample.l, normals.geometric) <= 0)
                {
                        return false;
                }
                const T n_l = dot(n, sample.l);
                if (n_l <= 0)
                {
                        return false;
                }
                beta *= sample.brdf * static_cast<float>(n_l / sample.pdf);

                if (terminate(depth, beta))
                {
                        return false;
                }

                ray = Ray<N, T>::make(surface.point, sample.l);
                const Vec<N, T> gn = normals.geometric;
                surface = q.scene_intersect(&gn, ray, normals);
                return static_cast<bool>(surface);
        }

        // pt() (pt.cpp:138-170): false for a background sample (nullopt)
        __device__ bool run(const Ray<N, T>& primary, Color<C>& out) const
        {
                Ray<N, T> ray = primary;
                Normals<N, T> normals;
                Hit<N, T> surface = q.scene_intersect(nullptr, ray, normals);
                if (!surface)
                {
                        return false;
                }
                Color<C> color = Color<C>::filled(0);
                const int li = q.light(surface);
                if (li >= 0)
                {
                        // LightSource::leave_radiance(-dir)
                        const Light<N, T, C>& light = s.lights[li];
                        if (dot(-ray.dir, light.normal) > 0)
                        {
                                color = light.radiance;
                        }
                }
                Color<C> beta = Color<C>::filled(1);
                for (int depth = 0; depth < PT_MAX_BOUNCES; ++depth)
                {
                        if (!step(depth, ray, surface, normals, color, beta))
                        {
                                break;
                        }
                }
                out = color;
                return true;
        }
};

#ifndef NBPT_PT_MIN_BLOCKS
#define NBPT_PT_MIN_BLOCKS 4
#endif

// One path of the PT integrator per thread, persistent: the threads take
// paths from a shared counter.  The sample points, the path's ray and its
// random stream are those of the BPT kernels (the same stratified points,
// seed_seq{seed, pass, pixel, sample + 1}); the reference's painter draws
// them the same way whichever integrator it runs (painting.cpp:225-257).
template <int N, typename T, int C>
__global__ void __launch_bounds__(128, NBPT_PT_MIN_BLOCKS) pt_paths_kernel(
        const DeviceScene<N, T, C> scene,
        const long long begin,
        const long long end,
        const int spp,
        const std::uint32_t seed,
        const std::uint32_t pass,
        const T* __restrict__ points,
        float* __restrict__ colors,
        float* __restrict__ lum,
        unsigned char* __restrict__ valid,
        unsigned* __restrict__ next_path,
        PathStats* __restrict__ stats,
        const float* __restrict__ cie_y)
{
        const long long paths = (end - begin) * spp;
        QueryCounters counters{0, 0, 0, 0};
        while (true)
        {
                const long long i = reserve_together(next_path, 1);
                if (i >= paths)
                {
                        break;
                }
                const long long local_pixel = i / spp;
                const int sample = static_cast<int>(i - local_pixel * spp);
                const long long p = begin + local_pixel;

                Vec<N - 1, T> point;
                {
                        long long rest = p;
#pragma unroll
                        for (int d = 0; d < N - 1; ++d)
                        {
                                const int size = scene.projector.size[d];
                                const long long q = rest / size;
                                point[d] = static_cast<T>(static_cast<int>(rest - q * size)) + points[i * (N - 1) + d];
                                rest = q;
                        }
                }
                const Ray<N, T> ray = scene.projector.ray(point);

                const std::uint32_t words[4] = {seed, pass, static_cast<std::uint32_t>(p),
                                                static_cast<std::uint32_t>(sample + 1)};
                Pcg g = seed_seq_pcg(words, 4);
                const SceneQueries<N, T, C> q{scene, counters};
                const Pt<N, T, C> pt{q, scene, g, cie_y, Bpt<N, T, C>{q, scene, g, 0, nullptr, nullptr}};
                Color<C> color;
                const bool has = pt.run(ray, color);
                float* const out = colors + i * C;
#pragma unroll 8
                for (int k = 0; k < C; ++k)
                {
                        out[k] = has ? color.c[k] : 0.0f;
                }
                lum[i] = has ? luminance(color, cie_y) : 0.0f;
                valid[i] = has ? 1 : 0;
        }
        add_counters(counters, stats);
}

} // namespace nbpt
