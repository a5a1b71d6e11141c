// Path tracing with next-event estimation for one path: the reference
// painter's other integrator (Integrator::PT).
//
// Mirrors src/painter/integrators/pt/{pt.cpp, direct_lighting.cpp} and
// src/painter/integrators/com/surface_sample.cpp, with the parallelotope and
// ball lights' arrive_info (src/painter/lights/parallelotope_light.cpp:92-115,
// ball_light.cpp:90-113).  Russian roulette weighs the path by the
// luminance of all its colour channels, so each thread carries its path's
// full throughput (beta) while it traces.
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

// One direct-lighting estimate of a bounce, colour-free: its channel c is
// (brdf_c * radiance_c) * scale, brdf_c from the terms (0 when the BRDF's
// own checks fail) and radiance_c the light's.
struct PtEstimate final
{
        BrdfTerms terms;
        float scale;
        int light;
        int zero;
};

// The sampled continuation of a bounce (com::surface_sample): beta_c is
// multiplied by brdf_c * scale.
template <int N, typename T>
struct PtContinuation final
{
        BrdfTerms terms;
        float scale;
        Vec<N, T> l;
};

// Tracing and sampling run on the channel-0 view of the scene (the
// reference's Color::is_black() and usable() look at channel 0 only, so
// every decision is the same); the colour arithmetic runs per channel from
// the recorded BRDF terms, in the reference's operation order.
template <int N, typename T>
struct Pt final
{
        const SceneQueries<N, T, 1>& q;
        const DeviceScene<N, T, 1>& s;
        Pcg& g;
        Bpt<N, T, 1> b; // light samples and visibility

        // LightSource::arrive_info: the light seen from `point` in direction
        // `l`; false when not usable.
        __device__ bool arrive_info(const Light<N, T, 1>& light, const Vec<N, T>& point, const Vec<N, T>& l, T& pdf,
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
        NBPT_CALL bool light_with_mis(const int k, const Hit<N, T>& surface, const Vec<N, T>& v,
                                      const Normals<N, T>& normals, PtEstimate& out) const
        {
                const Light<N, T, 1>& light = s.lights[k];
                const Vec<N, T>& n = normals.shading;
                const ArriveSample<N, T, 1> sample = b.arrive_sample(light, surface.point);
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
                const Material<T, 1>& m = s.materials[q.material(surface)];
                // brdf::f's own checks (brdf.h:146-171), then its terms
                out.zero = (dot(n, v) <= 0 || dot(n, l) <= 0) ? 1 : 0;
                if (!out.zero)
                {
                        out.terms = brdf_terms<N>(s.shading, m.roughness, n, v, l);
                }
                const T pdf = brdf_pdf(s.shading, m.roughness, n, v, l);
                const T weight = power_heuristic(sample.pdf, pdf);
                out.scale = static_cast<float>(weight * n_l / sample.pdf);
                out.light = k;
                return true;
        }

        // sample_surface_with_mis (direct_lighting.cpp:101-147); no shape
        // here is specular
        NBPT_CALL bool surface_with_mis(const int k, const Hit<N, T>& surface, const Vec<N, T>& v,
                                        const Normals<N, T>& normals, PtEstimate& out) const
        {
                const Light<N, T, 1>& light = s.lights[k];
                const Vec<N, T>& n = normals.shading;
                const Material<T, 1>& m = s.materials[q.material(surface)];
                const BrdfSample<N, 1, T> sample =
                        brdf_sample<N>(g, s.shading, m.roughness, m.f0, m.rho_ss, n, v, &out.terms);
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
                out.scale = static_cast<float>(weight * n_l / sample.pdf);
                out.light = k;
                out.zero = 0;
                return true;
        }

        // com::surface_sample (surface_sample.cpp:31-70)
        NBPT_CALL bool continuation(const Hit<N, T>& surface, const Vec<N, T>& v, const Normals<N, T>& normals,
                                    PtContinuation<N, T>& out) const
        {
                const Vec<N, T>& n = normals.shading;
                const Material<T, 1>& m = s.materials[q.material(surface)];
                const BrdfSample<N, 1, T> sample =
                        brdf_sample<N>(g, s.shading, m.roughness, m.f0, m.rho_ss, n, v, &out.terms);
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
                out.scale = static_cast<float>(n_l / sample.pdf);
                out.l = sample.l;
                return true;
        }
};

template <typename T, int C>
__device__ float pt_brdf_channel(const BrdfTerms& t, const int zero, const Material<T, C>& m, const int c,
                                 const ShadingConstants<T>& sc)
{
        return zero ? 0.0f : brdf_channel(t, m.f0.c[c], m.rho_ss.c[c], sc.fresnel_a, sc.fresnel_b);
}

#ifndef NBPT_PT_MIN_BLOCKS
#define NBPT_PT_MIN_BLOCKS 16
#endif

// The PT integrator's paths (pt.cpp:113-170), one lane per path at a time
// and one bounce per iteration of a persistent loop: every lane traces one
// ray and processes its hit in each iteration, and a lane whose path ends
// writes it out and takes the next path from a shared counter, so the
// warp's lanes run together however many bounces Russian roulette gives
// their paths.  The sample points, the path's ray and its random stream are
// those of the BPT kernels (the same stratified points, seed_seq{seed, pass,
// pixel, sample + 1}); the reference's painter draws them the same way
// whichever integrator it runs (painting.cpp:225-257).  Each lane keeps its
// path's beta (all C channels: in registers for RGB, in the thread's local
// memory for a spectrum) and, for RGB, its colour; a spectrum accumulates in
// the output row.  `estimates` holds 2 * light_count records per thread of
// the grid.
template <int N, typename T, int C>
__global__ void __launch_bounds__(128, NBPT_PT_MIN_BLOCKS) pt_paths_kernel(
        const DeviceScene<N, T, 1> scene,
        const Material<T, C>* __restrict__ materials,
        const Light<N, T, C>* __restrict__ lights,
        const long long begin,
        const long long end,
        const int spp,
        const std::uint32_t seed,
        const std::uint32_t pass,
        const T* __restrict__ points,
        float* __restrict__ colors,
        float* __restrict__ lum,
        unsigned char* __restrict__ valid,
        PtEstimate* __restrict__ estimates,
        unsigned* __restrict__ next_path,
        PathStats* __restrict__ stats,
        const float* __restrict__ cie_y,
        const unsigned* __restrict__ cancel)
{
        constexpr bool IN_REGISTERS = C <= 4;
        const long long paths = (end - begin) * spp;
        PtEstimate* const est =
                estimates + (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) * 2 * scene.light_count;
        const ShadingConstants<T>& sc = scene.shading;
        QueryCounters counters{0, 0, 0, 0};
        const SceneQueries<N, T, 1> q{scene, counters};
        Pcg g{0, 0};
        const Pt<N, T> pt{q, scene, g, Bpt<N, T, 1>{q, scene, g, 0, nullptr, nullptr}};
        Ray<N, T> ray;
        Vec<N, T> gn;
        Color<IN_REGISTERS ? C : 1> reg;
        Color<C> beta;
        int depth = -1;   // the bounce whose hit is traced next; -1: the primary ray
        long long i = -1; // the lane's path; -1 when it takes the next one
        while (true)
        {
                if (i < 0)
                {
                        if (cancelled(cancel))
                        {
                                break;
                        }
                        i = reserve_together(next_path, 1);
                        if (i >= paths)
                        {
                                break;
                        }
                        // 32-bit index arithmetic: a chunk's path index and a
                        // screen's pixel index fit in 31 bits (the painter's chunk
                        // limits and its screen check), and a 64-bit division costs
                        // several times a 32-bit one
                        const unsigned local_pixel = static_cast<unsigned>(i) / static_cast<unsigned>(spp);
                        const int sample = static_cast<int>(static_cast<unsigned>(i) - local_pixel * spp);
                        const unsigned p = static_cast<unsigned>(begin) + local_pixel;
                        Vec<N - 1, T> point;
                        {
                                unsigned rest = p;
#pragma unroll
                                for (int d = 0; d < N - 1; ++d)
                                {
                                        const unsigned size = static_cast<unsigned>(scene.projector.size[d]);
                                        const unsigned r = rest / size;
                                        point[d] = static_cast<T>(static_cast<int>(rest - r * size)) +
                                                   points[i * (N - 1) + d];
                                        rest = r;
                                }
                        }
                        ray = scene.projector.ray(point);
                        const std::uint32_t words[4] = {seed, pass, static_cast<std::uint32_t>(p),
                                                        static_cast<std::uint32_t>(sample + 1)};
                        g = seed_seq_pcg(words, 4);
                        depth = -1;
                }

                float* const out = colors + i * C;
                Normals<N, T> normals;
                const Hit<N, T> surface = q.scene_intersect(depth < 0 ? nullptr : &gn, ray, normals);
                if (depth < 0)
                {
                        if (!surface)
                        {
#pragma unroll 8
                                for (int c = 0; c < C; ++c)
                                {
                                        out[c] = 0.0f;
                                }
                                lum[i] = 0.0f;
                                valid[i] = 0;
                                i = -1;
                                continue;
                        }
                        // the emitted radiance seen by the primary ray
                        // (LightSource::leave_radiance(-dir))
                        const int li = q.light(surface);
                        const bool emits = li >= 0 && dot(-ray.dir, scene.lights[li].normal) > 0;
#pragma unroll 8
                        for (int c = 0; c < C; ++c)
                        {
                                const float e = emits ? lights[li].radiance.c[c] : 0.0f;
                                if constexpr (IN_REGISTERS)
                                {
                                        reg.c[c] = e;
                                }
                                else
                                {
                                        out[c] = e;
                                }
                        }
                        beta = Color<C>::filled(1);
                        depth = 0;
                }

                // one bounce (pt.cpp:68-111); the path ends where the
                // reference's loop breaks
                bool go_on = static_cast<bool>(surface);
                const Vec<N, T> v = -ray.dir;
                if (go_on)
                {
                        go_on = !(dot(normals.shading, v) <= 0);
                }
                if (go_on)
                {
                        // direct_lighting (direct_lighting.cpp:150-167): both
                        // estimates of every light, summed in that order
                        int count = 0;
                        for (int k = 0; k < scene.light_count; ++k)
                        {
                                count += pt.light_with_mis(k, surface, v, normals, est[count]) ? 1 : 0;
                                count += pt.surface_with_mis(k, surface, v, normals, est[count]) ? 1 : 0;
                        }
                        const Material<T, C>& m = materials[q.material(surface)];
                        if (count > 0)
                        {
#pragma unroll 4
                                for (int c = 0; c < C; ++c)
                                {
                                        float d = 0.0f;
                                        for (int e = 0; e < count; ++e)
                                        {
                                                const PtEstimate& r = est[e];
                                                const float brdf = pt_brdf_channel(r.terms, r.zero, m, c, sc);
                                                const float x = (brdf * lights[r.light].radiance.c[c]) * r.scale;
                                                d = e == 0 ? x : d + x;
                                        }
                                        if constexpr (IN_REGISTERS)
                                        {
                                                reg.c[c] += beta.c[c] * d;
                                        }
                                        else
                                        {
                                                out[c] += beta.c[c] * d;
                                        }
                                }
                        }

                        PtContinuation<N, T> next;
                        go_on = pt.continuation(surface, v, normals, next);
                        if (go_on)
                        {
#pragma unroll 8
                                for (int c = 0; c < C; ++c)
                                {
                                        beta.c[c] *= pt_brdf_channel(next.terms, 0, m, c, sc) * next.scale;
                                }

                                // terminate (pt.cpp:43-66)
                                if (depth >= 4)
                                {
                                        const float y = luminance(beta, cie_y);
                                        go_on = y > 0;
                                        if (go_on)
                                        {
                                                constexpr float MIN = 0.05f;
                                                constexpr float MAX = 0.95f;
                                                const float x = 1 - y;
                                                const float rr = (x < MIN) ? MIN : ((MAX < x) ? MAX : x);
                                                go_on = !bernoulli(g, rr);
                                                if (go_on)
                                                {
                                                        const float k = 1 - rr;
#pragma unroll 8
                                                        for (int c = 0; c < C; ++c)
                                                        {
                                                                beta.c[c] /= k;
                                                        }
                                                }
                                        }
                                }
                                // after the last bounce the path ends without
                                // the next ray, whose hit the reference never uses
                                if (go_on && ++depth < PT_MAX_BOUNCES)
                                {
                                        ray = Ray<N, T>::make(surface.point, next.l);
                                        gn = normals.geometric;
                                        continue;
                                }
                        }
                }

                // the path is done
                if constexpr (IN_REGISTERS)
                {
#pragma unroll
                        for (int c = 0; c < C; ++c)
                        {
                                out[c] = reg.c[c];
                        }
                        lum[i] = luminance(reg, cie_y);
                        if (!all_finite(reg.c))
                        {
                                atomicAdd(&stats->nonfinite, 1ull);
                        }
                }
                else
                {
                        Color<C> final_color;
#pragma unroll 8
                        for (int c = 0; c < C; ++c)
                        {
                                final_color.c[c] = out[c];
                        }
                        lum[i] = luminance(final_color, cie_y);
                        if (!all_finite(final_color.c))
                        {
                                atomicAdd(&stats->nonfinite, 1ull);
                        }
                }
                valid[i] = 1;
                i = -1;
        }
        add_counters(counters, stats);
}

} // namespace nbpt
