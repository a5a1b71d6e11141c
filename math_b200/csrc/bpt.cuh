// Bidirectional path tracing with multiple importance sampling for one path:
// camera subpath, light subpath and every (s, t) connection strategy.
//
// Mirrors src/painter/integrators/bpt/{bpt.cpp, connect.cpp, mis.cpp,
// vertex_pdf.h, vertex/*.h}, src/painter/integrators/com/{visibility.h,
// normals.h, surface_sample.cpp} and the parallelotope and ball lights
// (src/painter/lights/parallelotope_light.cpp, ball_light.cpp), with one
// random stream per path consumed in the reference's order.
#pragma once

#include "core.cuh"
#include "geometry.cuh"
#include "scene.cuh"
#include "shading.cuh"
#include "tape.cuh"

namespace nbpt
{
// Longest subpath: MAX_DEPTH + 1 vertices for a maximum depth of 8.
inline constexpr int MAX_PATH_VERTICES = 9;

enum class VertexType : int
{
        SURFACE = 0,
        CAMERA = 1,
        LIGHT = 2,
        INFINITE = 3
};

template <int N, typename T, int C>
struct PathVertex final
{
        int type;
        int material; // surface
        int light;    // surface: attached light or -1; light vertex: the light
        bool has_pos; // light vertex
        bool has_normal;
        Vec<N, T> pos;     // surface point or light position
        Normals<N, T> nrm; // surface normals; light vertex: emission normal in .shading
        Vec<N, T> dir;     // surface: to previous vertex; camera: to camera; light: direction
        Color<C> beta;
        T pdf_fwd;
        T pdf_rev;
};

template <int N, typename T, int C>
struct LeaveSample final
{
        Ray<N, T> ray;
        Vec<N, T> n;
        T pdf_pos;
        T pdf_dir;
        Color<C> radiance;
};

template <int N, typename T, int C>
struct ArriveSample final
{
        Vec<N, T> l;
        T pdf;
        Color<C> radiance;
        T distance;

        NBPT_HD bool usable() const
        {
                return pdf > 0 && !radiance.is_black();
        }
};

// RECORD: trace with channel 0 only (C == 1) and write the path's colour
// factors to `tape` (tape.cuh); the colours are then formed for all
// channels by replaying the tape.
template <int N, typename T, int C, bool RECORD = false>
struct Bpt final
{
        const SceneQueries<N, T, C>& q;
        const DeviceScene<N, T, C>& s;
        Pcg& g;
        int max_depth;
        // the subpaths: max_depth + 1 vertices each, in local or global memory
        PathVertex<N, T, C>* camera;
        PathVertex<N, T, C>* light;
        int camera_size = 0;
        int light_size = 0;
        mutable TapeWriter tape{};

        // -----------------------------------------------------------------
        // lights

        __device__ Vec<N, T> sample_location(const Light<N, T, C>& l) const
        {
                if (l.type == static_cast<int>(LightType::PARALLELOTOPE))
                {
                        return l.org + uniform_in_parallelotope(g, l.vectors);
                }
                return l.org + uniform_in_ball_spanned(g, l.vectors);
        }

        // leave_sample: the emission direction is drawn before the point
        NBPT_CALL LeaveSample<N, T, C> leave_sample(const Light<N, T, C>& l) const
        {
                const Vec<N, T> dir = cosine_on_hemisphere(g, l.normal);
                const Vec<N, T> org = sample_location(l);
                LeaveSample<N, T, C> r;
                r.ray = Ray<N, T>::make(org, dir);
                const T cos = dot(l.normal, r.ray.dir);
                r.n = l.normal;
                r.pdf_pos = l.pdf;
                r.pdf_dir = cosine_on_hemisphere_pdf(cos, s.shading.k_inv);
                r.radiance = l.radiance;
                return r;
        }

        NBPT_CALL ArriveSample<N, T, C> arrive_sample(const Light<N, T, C>& l, const Vec<N, T>& point) const
        {
                ArriveSample<N, T, C> r;
                if (!(dot(l.normal, point - l.org) > 0))
                {
                        r.pdf = 0;
                        r.radiance = Color<C>::filled(0);
                        return r;
                }
                const Vec<N, T> direction = sample_location(l) - point;
                const T distance = direction.norm();
                r.l = direction / distance;
                const T cos = -dot(r.l, l.normal);
                r.pdf = area_pdf_to_solid_angle_pdf<N>(l.pdf, cos, distance);
                r.radiance = l.radiance;
                r.distance = distance;
                return r;
        }

        __device__ T leave_pdf_dir(const Light<N, T, C>& l, const Vec<N, T>& dir) const
        {
                return cosine_on_hemisphere_pdf(dot(l.normal, dir), s.shading.k_inv);
        }

        // light distribution: uniform choice (light_distribution.cpp:36-65);
        // one light consumes no random numbers (std::discrete_distribution).
        __device__ int sample_light() const
        {
                if (s.light_count <= 1)
                {
                        return 0;
                }
                const double p = canonical<double>(g);
                int i = 0;
                while (i < s.light_count - 1 && s.lights[i].cumulative < p)
                {
                        ++i;
                }
                return i;
        }

        // -----------------------------------------------------------------
        // area pdfs (vertex/area_pdf.h)

        __device__ static T area_pdf_pos(const Vec<N, T>& prev_pos, const T angle_pdf, const Vec<N, T>& next_pos,
                                         const Vec<N, T>* next_normal)
        {
                const Vec<N, T> v = prev_pos - next_pos;
                const T distance = v.norm();
                const T cosine = next_normal ? (abs_value(dot(v, *next_normal)) / distance) : T(1);
                return solid_angle_pdf_to_area_pdf<N>(angle_pdf, cosine, distance);
        }

        __device__ static T area_pdf_dir(const T angle_pdf, const Vec<N, T>& next_dir, const T next_distance,
                                         const Vec<N, T>* next_normal)
        {
                const T cosine = next_normal ? abs_value(dot(next_dir, *next_normal)) : T(1);
                return solid_angle_pdf_to_area_pdf<N>(angle_pdf, cosine, next_distance);
        }

        // -----------------------------------------------------------------
        // vertex methods

        __device__ T angle_pdf(const PathVertex<N, T, C>& v, const Vec<N, T>& dv, const Vec<N, T>& dl) const
        {
                return brdf_pdf(s.shading, s.materials[v.material].roughness, v.nrm.shading, dv, dl);
        }

        __device__ Color<C> vertex_brdf(const PathVertex<N, T, C>& v, const Vec<N, T>& dv, const Vec<N, T>& dl,
                                        BrdfTerms* const terms = nullptr) const
        {
                const Material<T, C>& m = s.materials[v.material];
                return brdf_f(s.shading, m.roughness, m.f0, m.rho_ss, v.nrm.shading, dv, dl, terms);
        }

        // prev.area_pdf(angle_pdf, next_pos, next_normal) for the vertex kinds
        // that can precede a surface (vertex_pdf.h:35-60)
        __device__ T prev_area_pdf(const PathVertex<N, T, C>& prev, const T angle, const Vec<N, T>& next_pos,
                                   const Vec<N, T>& next_normal) const
        {
                switch (static_cast<VertexType>(prev.type))
                {
                case VertexType::CAMERA:
                        return 1;
                case VertexType::LIGHT:
                        return area_pdf_pos(prev.pos, angle, next_pos, &next_normal);
                default:
                        return area_pdf_pos(prev.pos, angle, next_pos, &next_normal);
                }
        }

        // Light vertex: pdf of reaching `next_pos` from the light (light.h:108-120)
        __device__ T light_vertex_area_pdf(const PathVertex<N, T, C>& lv, const Vec<N, T>& next_pos,
                                           const Vec<N, T>& next_normal) const
        {
                const Vec<N, T> l_dir = next_pos - lv.pos;
                const T l_distance = l_dir.norm();
                const Vec<N, T> l = l_dir / l_distance;
                const T pdf = leave_pdf_dir(s.lights[lv.light], l);
                return area_pdf_dir(pdf, l, l_distance, &next_normal);
        }

        // Surface vertex that carries a light: surface.h:97-107
        __device__ T surface_light_area_pdf(const PathVertex<N, T, C>& sv, const Vec<N, T>& next_pos,
                                            const Vec<N, T>& next_normal) const
        {
                const Vec<N, T> l_dir = next_pos - sv.pos;
                const T l_distance = l_dir.norm();
                const Vec<N, T> l = l_dir / l_distance;
                const T pdf = leave_pdf_dir(s.lights[sv.light], l);
                return area_pdf_dir(pdf, l, l_distance, &next_normal);
        }

        __device__ Vec<N, T> dir_to_light(const PathVertex<N, T, C>& lv, const Vec<N, T>& point) const
        {
                if (lv.has_pos)
                {
                        return (lv.pos - point).normalized();
                }
                return -lv.dir;
        }

        // compute_pdf (vertex_pdf.h:141-190)
        NBPT_CALL T compute_pdf(const PathVertex<N, T, C>& prev, const PathVertex<N, T, C>& v,
                                 const PathVertex<N, T, C>& next) const
        {
                Vec<N, T> to_prev;
                switch (static_cast<VertexType>(prev.type))
                {
                case VertexType::CAMERA:
                        to_prev = prev.dir;
                        break;
                case VertexType::LIGHT:
                        to_prev = dir_to_light(prev, v.pos);
                        break;
                default:
                        to_prev = (prev.pos - v.pos).normalized();
                        break;
                }
                if (next.type == static_cast<int>(VertexType::LIGHT))
                {
                        const Vec<N, T> to_next = dir_to_light(next, v.pos);
                        const T a = angle_pdf(v, to_prev, to_next);
                        return area_pdf_pos(v.pos, a, next.pos, next.has_normal ? &next.nrm.shading : nullptr);
                }
                const Vec<N, T> l_dir = next.pos - v.pos;
                const T l_distance = l_dir.norm();
                const Vec<N, T> l = l_dir / l_distance;
                const T pdf = angle_pdf(v, to_prev, l);
                return area_pdf_dir(pdf, l, l_distance, &next.nrm.shading);
        }

        // compute_light_pdf (vertex_pdf.h:88-115)
        NBPT_CALL T compute_light_pdf(const PathVertex<N, T, C>& lv, const PathVertex<N, T, C>& next) const
        {
                if (lv.type == static_cast<int>(VertexType::LIGHT))
                {
                        return light_vertex_area_pdf(lv, next.pos, next.nrm.shading);
                }
                return surface_light_area_pdf(lv, next.pos, next.nrm.shading);
        }

        // -----------------------------------------------------------------
        // visibility (com/visibility.h)

        __device__ static T visibility_distance(const T d)
        {
                constexpr T K = 1 - 1000 * Limits<T>::EPSILON;
                return K * d;
        }

        __device__ static bool directed_outside(const T cosine)
        {
                constexpr T EPSILON = 100 * Limits<T>::EPSILON;
                return cosine > EPSILON;
        }

        NBPT_CALL bool move_and_intersect_any(const Vec<N, T>& gn, const Ray<N, T>& ray, const T distance) const
        {
                const Hit<N, T> h = q.intersect(&gn, ray, distance);
                if (!h)
                {
                        return false;
                }
                const T d = distance - h.distance;
                if (d > 0)
                {
                        const Vec<N, T> hg = q.geometric_normal(h);
                        Ray<N, T> r2 = ray;
                        r2.org = h.point;
                        return q.intersect_any(&hg, r2, d);
                }
                return false;
        }

        // occluded(scene, normals, ray, distance) (visibility.h:99-123)
        NBPT_CALL bool occluded_ray(const Normals<N, T>& normals, const Ray<N, T>& ray, const T distance) const
        {
                if (!directed_outside(dot(ray.dir, normals.shading)))
                {
                        return true;
                }
                const T d = visibility_distance(distance);
                const bool visible = dot(ray.dir, normals.geometric) >= 0;
                if (visible)
                {
                        return q.intersect_any(&normals.geometric, ray, d);
                }
                return move_and_intersect_any(normals.geometric, ray, d);
        }

        // occluded(scene, p1, n1, p2, n2) (visibility.h:125-172)
        NBPT_CALL bool occluded_points(const Vec<N, T>& p1, const Normals<N, T>& n1, const Vec<N, T>& p2,
                                        const Normals<N, T>& n2) const
        {
                const Vec<N, T> direction_1 = p2 - p1;
                const Ray<N, T> ray_1 = Ray<N, T>::make(p1, direction_1);
                if (!directed_outside(dot(ray_1.dir, n1.shading)) || !directed_outside(-dot(ray_1.dir, n2.shading)))
                {
                        return true;
                }
                const bool visible_1 = dot(ray_1.dir, n1.geometric) >= 0;
                const bool visible_2 = dot(ray_1.dir, n2.geometric) <= 0;
                T distance = visibility_distance(direction_1.norm());
                if (visible_1 && visible_2)
                {
                        return q.intersect_any(&n1.geometric, ray_1, distance);
                }
                if (!visible_1)
                {
                        const Hit<N, T> h = q.intersect(&n1.geometric, ray_1, distance);
                        if (!h)
                        {
                                return false;
                        }
                        const T d = distance - h.distance;
                        if (!(d > 0))
                        {
                                return false;
                        }
                        distance = d;
                }
                Ray<N, T> ray_2;
                ray_2.org = p2;
                ray_2.dir = -ray_1.dir;
                if (!visible_2)
                {
                        return move_and_intersect_any(n2.geometric, ray_2, distance);
                }
                return q.intersect_any(&n2.geometric, ray_2, distance);
        }

        // -----------------------------------------------------------------
        // subpaths (bpt.cpp:60-264)

        __device__ void set_surface(PathVertex<N, T, C>& v, const Hit<N, T>& h, const Normals<N, T>& normals,
                                    const Color<C>& beta, const Vec<N, T>& dir_to_prev) const
        {
                v.type = static_cast<int>(VertexType::SURFACE);
                v.material = q.material(h);
                v.light = q.light(h);
                v.has_pos = true;
                v.has_normal = true;
                v.pos = h.point;
                v.nrm = normals;
                v.dir = dir_to_prev;
                v.beta = beta;
                v.pdf_fwd = 0;
                v.pdf_rev = 0;
        }

        __device__ static T correct_normals(const Normals<N, T>& n, const Vec<N, T>& v, const Vec<N, T>& l)
        {
                const T denominator = dot(v, n.geometric) * dot(l, n.shading);
                if (denominator == 0)
                {
                        return 0;
                }
                const T numerator = dot(v, n.shading) * dot(l, n.geometric);
                return abs_value(numerator / denominator);
        }

        // A subpath walk in progress (walk, bpt.cpp:184-212): the throughput,
        // the forward pdf, the ray to trace next and the bounces done.
        struct Walk final
        {
                Color<C> beta;
                T pdf_forward;
                Ray<N, T> ray;
                int depth;
                bool camera;
        };

        // process_intersection (bpt.cpp:136-178) for the closest hit of
        // w.ray: the vertex added to the walk's subpath, and true with w.ray
        // set to the next ray (to be traced from normals.geometric) when the
        // walk goes on.  The reference intersects the next ray of the last
        // bounce as well and never uses the hit; the walk ends there instead,
        // with the same vertices, random stream and tape.
        NBPT_CALL bool walk_step(Walk& w, const Hit<N, T>& surface, const Normals<N, T>& normals)
        {
                PathVertex<N, T, C>* const path = w.camera ? camera : light;
                int& size = w.camera ? camera_size : light_size;
                const Vec<N, T> v = -w.ray.dir;
                // surface_found (bpt.cpp:60-67)
                if (!(surface && dot(normals.shading, v) > 0))
                {
                        // surface_not_found (bpt.cpp:84-100)
                        if (w.camera)
                        {
                                path[size].type = static_cast<int>(VertexType::INFINITE);
                                ++size;
                        }
                        return false;
                }

                // surface_sample_with_pdf (surface_sample.cpp:39-82)
                const int material = q.material(surface);
                const Material<T, C>& m = s.materials[material];
                const Vec<N, T>& n = normals.shading;
                BrdfTerms terms;
                const BrdfSample<N, C, T> bs =
                        brdf_sample<N>(g, s.shading, m.roughness, m.f0, m.rho_ss, n, v, RECORD ? &terms : nullptr);
                bool ok = bs.pdf > 0 && !bs.brdf.is_black();
                T n_l = 0;
                if (ok)
                {
                        ok = dot(bs.l, normals.geometric) > 0;
                }
                if (ok)
                {
                        n_l = dot(n, bs.l);
                        ok = n_l > 0;
                }
                if (!ok)
                {
                        // sample_not_found (bpt.cpp:102-117)
                        if (q.light(surface) >= 0)
                        {
                                PathVertex<N, T, C>& next = path[size];
                                set_surface(next, surface, normals, w.beta, v);
                                next.pdf_fwd = prev_area_pdf(path[size - 1], w.pdf_forward, next.pos, next.nrm.shading);
                                ++size;
                        }
                        return false;
                }
                const float sample_k = static_cast<float>(n_l / bs.pdf);
                const Color<C> sample_beta = bs.brdf * sample_k;
                const T pdf_reversed = brdf_pdf(s.shading, m.roughness, n, bs.l, v);

                // add_sample (bpt.cpp:119-134)
                {
                        PathVertex<N, T, C>& next = path[size];
                        set_surface(next, surface, normals, w.beta, v);
                        PathVertex<N, T, C>& prev = path[size - 1];
                        next.pdf_fwd = prev_area_pdf(prev, w.pdf_forward, next.pos, next.nrm.shading);
                        if (prev.type == static_cast<int>(VertexType::SURFACE))
                        {
                                prev.pdf_rev = area_pdf_pos(next.pos, pdf_reversed, prev.pos, &prev.nrm.shading);
                        }
                        else if (prev.type == static_cast<int>(VertexType::LIGHT))
                        {
                                prev.pdf_rev = area_pdf_pos(next.pos, pdf_reversed, prev.pos,
                                                            prev.has_normal ? &prev.nrm.shading : nullptr);
                        }
                        ++size;
                }

                w.pdf_forward = bs.pdf;
                w.beta *= sample_beta;
                float normals_k = 1;
                if (!w.camera)
                {
                        normals_k = static_cast<float>(correct_normals(normals, bs.l, v));
                        w.beta *= normals_k;
                }
                if constexpr (RECORD)
                {
                        tape.put(static_cast<int>(w.camera ? TapeRecord::CAMERA_BOUNCE : TapeRecord::LIGHT_BOUNCE));
                        tape.put(material);
                        tape.put(terms);
                        tape.put(sample_k);
                        if (!w.camera)
                        {
                                tape.put(normals_k);
                        }
                }
                if (w.beta.is_black() || ++w.depth == max_depth)
                {
                        return false;
                }
                w.ray = Ray<N, T>::make(surface.point, bs.l);
                return true;
        }

        // generate_camera_path (bpt.cpp:213-229) up to its first ray.
        __device__ Walk camera_start(const Ray<N, T>& ray)
        {
                camera_size = 1;
                camera[0].type = static_cast<int>(VertexType::CAMERA);
                camera[0].dir = -ray.dir;
                camera[0].has_pos = false;
                camera[0].has_normal = false;
                return Walk{Color<C>::filled(1), T(1), ray, 0, true};
        }

        // generate_light_path (bpt.cpp:231-264) up to its first ray: false,
        // with no light subpath, when the light sample is unusable.
        __device__ bool light_start(Walk& w)
        {
                light_size = 0;
                const int li = sample_light();
                const Light<N, T, C>& l = s.lights[li];
                const LeaveSample<N, T, C> ls = leave_sample(l);
                if (!(ls.pdf_pos > 0 && ls.pdf_dir > 0 && !ls.radiance.is_black()))
                {
                        return false;
                }
                const T dpdf = l.distribution_pdf;
                PathVertex<N, T, C>& v = light[0];
                v.type = static_cast<int>(VertexType::LIGHT);
                v.light = li;
                v.has_pos = true;
                v.has_normal = true;
                v.pos = ls.ray.org;
                v.dir = ls.ray.dir.normalized();
                v.nrm.shading = ls.n;
                v.nrm.geometric = ls.n;
                v.pdf_fwd = dpdf * ls.pdf_pos;
                v.pdf_rev = 0;
                light_size = 1;

                const T pdf = dpdf * ls.pdf_pos * ls.pdf_dir;
                const T k = max_value(T(0), dot(ls.n, ls.ray.dir));
                const float start_k = static_cast<float>(k / pdf);
                if constexpr (RECORD)
                {
                        tape.put(static_cast<int>(TapeRecord::LIGHT_START));
                        tape.put(li);
                        tape.put(start_k);
                }
                w = Walk{ls.radiance * start_k, ls.pdf_dir, ls.ray, 0, false};
                return true;
        }

        // -----------------------------------------------------------------
        // MIS (mis.cpp:48-235)

        __device__ static T map(const T v)
        {
                return v != 0 ? v : T(1);
        }

        // The light subpath is `lp` (light[] or the single resampled light
        // vertex of an s = 1 strategy).
        NBPT_CALL T mis_weight(const PathVertex<N, T, C>* lp, const int s_count, const int t_count) const
        {
                if (s_count + t_count == 2)
                {
                        return 1;
                }
                T lf[MAX_PATH_VERTICES];
                T lr[MAX_PATH_VERTICES];
                T cf[MAX_PATH_VERTICES];
                T cr[MAX_PATH_VERTICES];
                for (int i = 0; i < s_count; ++i)
                {
                        lf[i] = lp[i].pdf_fwd;
                        lr[i] = lp[i].pdf_rev;
                }
                for (int i = 0; i < t_count; ++i)
                {
                        if (camera[i].type == static_cast<int>(VertexType::CAMERA))
                        {
                                cf[i] = -1;
                                cr[i] = -1;
                        }
                        else
                        {
                                cf[i] = camera[i].pdf_fwd;
                                cr[i] = camera[i].pdf_rev;
                        }
                }

                // set_reversed (mis.cpp:107-146)
                if (s_count == 0)
                {
                        cr[t_count - 1] = s.lights[camera[t_count - 1].light].pdf;
                        cr[t_count - 2] = compute_light_pdf(camera[t_count - 1], camera[t_count - 2]);
                }
                else
                {
                        lr[s_count - 1] = compute_pdf(camera[t_count - 2], camera[t_count - 1], lp[s_count - 1]);
                        if (t_count > 2)
                        {
                                cr[t_count - 2] = compute_pdf(lp[s_count - 1], camera[t_count - 1], camera[t_count - 2]);
                        }
                        if (s_count == 1)
                        {
                                cr[t_count - 1] = compute_light_pdf(lp[0], camera[t_count - 1]);
                        }
                        else
                        {
                                lr[s_count - 2] = compute_pdf(camera[t_count - 1], lp[s_count - 1], lp[s_count - 2]);
                                cr[t_count - 1] = compute_pdf(lp[s_count - 2], lp[s_count - 1], camera[t_count - 1]);
                        }
                }

                // every vertex of these scenes is connectible (no specular
                // surfaces, no delta lights)
                T light_sum = 0;
                if (s_count > 0)
                {
                        T ri = 1;
                        for (int i = s_count - 1; i > 0; --i)
                        {
                                ri *= map(lr[i]) / map(lf[i]);
                                light_sum += ri;
                        }
                        ri *= map(lr[0]) / map(lf[0]);
                        light_sum += ri;
                }
                T camera_sum = 0;
                if (t_count > 1)
                {
                        T ri = 1;
                        for (int i = t_count - 1; i > 1; --i)
                        {
                                ri *= map(cr[i]) / map(cf[i]);
                                camera_sum += ri;
                        }
                        ri *= map(cr[1]) / map(cf[1]);
                        camera_sum += ri;
                }
                return 1 / (1 + light_sum + camera_sum);
        }

        // -----------------------------------------------------------------
        // connections (connect.cpp:48-375)

        // The s = 1 strategy in two parts (connect.cpp:135-185): the light
        // sample, the only part that draws from the path's random stream, and
        // the connection to it.  false: the sample is unusable.
        __device__ bool light_arrival(const int t_count, int& li, ArriveSample<N, T, C>& as) const
        {
                const PathVertex<N, T, C>& cv = camera[t_count - 1];
                li = sample_light();
                as = arrive_sample(s.lights[li], cv.pos);
                return as.usable();
        }

        NBPT_CALL bool connect_light(const int t_count, const int li, const ArriveSample<N, T, C>& as,
                                     Color<C>& out) const
        {
                const PathVertex<N, T, C>& cv = camera[t_count - 1];
                const Light<N, T, C>& l = s.lights[li];
                PathVertex<N, T, C> lv;
                lv.type = static_cast<int>(VertexType::LIGHT);
                lv.light = li;
                lv.has_pos = true;
                lv.has_normal = false;
                lv.pos = cv.pos + as.l * as.distance;
                lv.dir = (-as.l).normalized();
                lv.pdf_fwd = l.distribution_pdf * l.pdf;
                lv.pdf_rev = 0;

                const Ray<N, T> ray_to_light = Ray<N, T>::make(cv.pos, as.l);
                const T n_l = dot(cv.nrm.shading, ray_to_light.dir);
                if (!(n_l > 0))
                {
                        return false;
                }
                BrdfTerms terms;
                const float light_k = static_cast<float>(n_l / (as.pdf * l.distribution_pdf));
                const Color<C> c = cv.beta * vertex_brdf(cv, cv.dir, ray_to_light.dir, RECORD ? &terms : nullptr) *
                                   as.radiance * light_k;
                if (c.is_black())
                {
                        return false;
                }
                if (occluded_ray(cv.nrm, ray_to_light, as.distance))
                {
                        return false;
                }
                const float mis = static_cast<float>(mis_weight(&lv, 1, t_count));
                out = c * mis;
                if constexpr (RECORD)
                {
                        tape.n = tape_slot_offset(max_depth, t_count, 1);
                        tape.put(static_cast<int>(TapeRecord::STRATEGY_LIGHT));
                        tape.put(t_count);
                        tape.put(cv.material);
                        tape.put(terms);
                        tape.put(li);
                        tape.put(light_k);
                        tape.put(mis);
                }
                return true;
        }

        NBPT_CALL bool connect_strategy(const int s_count, const int t_count, Color<C>& out)
        {
                const PathVertex<N, T, C>& cv = camera[t_count - 1];
                if (s_count == 0)
                {
                        if (cv.type != static_cast<int>(VertexType::SURFACE) || cv.light < 0)
                        {
                                return false;
                        }
                        const Light<N, T, C>& l = s.lights[cv.light];
                        if (!(dot(cv.dir, l.normal) > 0))
                        {
                                return false;
                        }
                        const Color<C> c = l.radiance * cv.beta;
                        if (c.is_black())
                        {
                                return false;
                        }
                        const float mis = static_cast<float>(mis_weight(light, 0, t_count));
                        out = c * mis;
                        if constexpr (RECORD)
                        {
                                tape.n = tape_slot_offset(max_depth, t_count, s_count);
                                tape.put(static_cast<int>(TapeRecord::STRATEGY_EMITTED));
                                tape.put(t_count);
                                tape.put(cv.light);
                                tape.put(mis);
                        }
                        return true;
                }
                if (cv.type == static_cast<int>(VertexType::INFINITE))
                {
                        return false;
                }
                if (s_count == 1)
                {
                        int li;
                        ArriveSample<N, T, C> as;
                        if (!light_arrival(t_count, li, as))
                        {
                                return false;
                        }
                        return connect_light(t_count, li, as, out);
                }

                const PathVertex<N, T, C>& lv = light[s_count - 1];
                // compute_color (connect.cpp:187-221)
                const Vec<N, T> v = lv.pos - cv.pos;
                const T distance = v.norm();
                const Vec<N, T> from_camera_to_light = v / distance;
                const T camera_n_l = dot(cv.nrm.shading, from_camera_to_light);
                if (!(camera_n_l > 0))
                {
                        return false;
                }
                const Vec<N, T> light_l = -from_camera_to_light;
                const T light_n_l = dot(lv.nrm.shading, light_l);
                if (!(light_n_l > 0))
                {
                        return false;
                }
                BrdfTerms camera_terms;
                BrdfTerms light_terms;
                const Color<C> c0 = cv.beta * vertex_brdf(cv, cv.dir, from_camera_to_light, RECORD ? &camera_terms : nullptr) *
                                    vertex_brdf(lv, lv.dir, light_l, RECORD ? &light_terms : nullptr) * lv.beta;
                const T geometry = camera_n_l * light_n_l / power<N - 1>(distance);
                const float geometry_k = static_cast<float>(geometry);
                const Color<C> c = c0 * geometry_k;
                if (c.is_black())
                {
                        return false;
                }
                if (occluded_points(cv.pos, cv.nrm, lv.pos, lv.nrm))
                {
                        return false;
                }
                const float mis = static_cast<float>(mis_weight(light, s_count, t_count));
                out = c * mis;
                if constexpr (RECORD)
                {
                        tape.n = tape_slot_offset(max_depth, t_count, s_count);
                        tape.put(static_cast<int>(TapeRecord::STRATEGY_CONNECT));
                        tape.put(s_count);
                        tape.put(t_count);
                        tape.put(cv.material);
                        tape.put(camera_terms);
                        tape.put(lv.material);
                        tape.put(light_terms);
                        tape.put(geometry_k);
                        tape.put(mis);
                }
                return true;
        }

        // bpt() (bpt.cpp:267-292) after the camera subpath: BACKGROUND for a
        // camera ray that leaves the scene (the reference's nullopt), NO_LIGHT
        // when the camera subpath is the camera alone (black), CONNECT when
        // the light subpath is traced and the strategies follow.
        enum class Subpaths : int
        {
                BACKGROUND = 0,
                NO_LIGHT = 1,
                CONNECT = 2
        };

        __device__ Subpaths camera_outcome() const
        {
                if (camera_size == 1)
                {
                        return Subpaths::NO_LIGHT;
                }
                if (camera_size == 2 && camera[1].type == static_cast<int>(VertexType::INFINITE))
                {
                        return Subpaths::BACKGROUND;
                }
                return Subpaths::CONNECT;
        }
};
} // namespace nbpt
