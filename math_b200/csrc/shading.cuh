// n-D GGX microfacet BRDF with multiple-bounce and Disney-style diffuse
// terms, its sampling, and the n-sphere / parallelotope sampling routines.
//
// Follows src/shading/ggx/{brdf.h, ggx.h, multiple_bounce.h, subsurface.h,
// fresnel.h, metalness.h, f1_albedo.cpp} and src/sampling/{sphere_uniform.h,
// sphere_cosine.h, parallelotope_uniform.h, pdf.h}.
//
// Random-number order.  Where the reference draws several random numbers as
// arguments of one constructor call, C++ leaves their order to the compiler;
// the reference build (GCC) evaluates such arguments right to left, so
//   * a random vector (sphere_uniform.h:54-62) fills its last component first;
//   * a light's leave sample (lights/*_light.cpp leave_sample) draws the
//     emission direction before the emission point.
// The accelerated path consumes random numbers in that same order.
#pragma once

#include "core.cuh"
#include "geometry.cuh"

namespace nbpt
{
// Per-dimension constants the reference computes at compile time in long
// double and stores in the path's precision T:
//   k: integral of the cosine over the hemisphere (sphere_integral.h),
//   k_inv: 1 / k, the cosine-hemisphere pdf factor (sphere_cosine.h:82-92),
//   ball_pdf: 1 / volume of the unit (N-1)-ball (sphere_uniform.h:198-203).
// Fresnel average a * f0 + b (fresnel.h:50-87) is in float (colour precision).
template <typename T>
struct ShadingConstants final
{
        T k;
        T k_inv;
        T ball_pdf;
        float fresnel_a;
        float fresnel_b;
        const T* f1_albedo;  // [32 roughness][32 cosine]
        const T* f1_average; // [32]
};

// ---------------------------------------------------------------------------
// sampling

// Uniform point in the unit M-ball by rejection (sphere_uniform.h:66-82);
// components drawn last-to-first.
template <int M, typename T>
NBPT_HD void uniform_in_ball(Pcg& g, Vec<M, T>& v, T& length_square)
{
        while (true)
        {
#pragma unroll
                for (int i = M - 1; i >= 0; --i)
                {
                        v[i] = uniform<T>(g, T(-1), T(1));
                }
                length_square = dot(v, v);
                if (length_square <= 1 && length_square > 0)
                {
                        break;
                }
        }
}

// Cosine-weighted direction about `normal` from a point `v` drawn uniformly
// in the unit (N-1)-ball, given the orthonormal complement of `normal`
// (sphere_cosine.h:41-80).
template <int N, typename T>
NBPT_HD Vec<N, T> cosine_from_ball(const Vec<N, T>& normal, const Vec<N, T>* basis, const Vec<N - 1, T>& v,
                                   const T length_square)
{
        const T h = sqrt_value(1 - length_square);
        Vec<N, T> r = normal * h;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                r.multiply_add(basis[i], v[i]);
        }
        return r;
}

// Cosine-weighted direction about `normal` (sphere_cosine.h:41-80).
template <int N, typename T>
NBPT_HD Vec<N, T> cosine_on_hemisphere(Pcg& g, const Vec<N, T>& normal)
{
        Vec<N, T> basis[N - 1];
        orthogonal_complement_of_unit_vector(normal, basis);
        Vec<N - 1, T> v;
        T length_square;
        uniform_in_ball<N - 1>(g, v, length_square);
        const T h = sqrt_value(1 - length_square);
        Vec<N, T> r = normal * h;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                r.multiply_add(basis[i], v[i]);
        }
        return r;
}

template <typename T>
NBPT_HD T cosine_on_hemisphere_pdf(const T n_v, const T k_inv)
{
        return n_v > 0 ? n_v * k_inv : T(0);
}

// sum_i vectors[i] * u_i with u_i uniform in [0, 1) (parallelotope_uniform.h:44-58)
template <int N, typename T>
NBPT_HD Vec<N, T> uniform_in_parallelotope(Pcg& g, const Vec<N, T>* vectors)
{
        Vec<N, T> r = vectors[0] * uniform<T>(g, T(0), T(1));
#pragma unroll
        for (int i = 1; i < N - 1; ++i)
        {
                r.multiply_add(vectors[i], uniform<T>(g, T(0), T(1)));
        }
        return r;
}

// Uniform point in the (N-1)-ball spanned by orthogonal `vectors`
// (sphere_uniform.h:179-196).
template <int N, typename T>
NBPT_HD Vec<N, T> uniform_in_ball_spanned(Pcg& g, const Vec<N, T>* vectors)
{
        Vec<N - 1, T> v;
        T length_square;
        uniform_in_ball<N - 1>(g, v, length_square);
        Vec<N, T> r = vectors[0] * v[0];
#pragma unroll
        for (int i = 1; i < N - 1; ++i)
        {
                r.multiply_add(vectors[i], v[i]);
        }
        return r;
}

// sampling/pdf.h:27-75
template <int N, typename T>
NBPT_HD T reflected_pdf(const T pdf, const T cosine)
{
        if (cosine > 0)
        {
                return pdf / (T(1 << (N - 1)) * power<N - 2>(cosine));
        }
        return 0;
}

template <int N, typename T>
NBPT_HD T area_pdf_to_solid_angle_pdf(const T pdf, const T cosine, const T distance)
{
        if (cosine > 0)
        {
                return pdf * power<N - 1>(distance) / cosine;
        }
        return 0;
}

template <int N, typename T>
NBPT_HD T solid_angle_pdf_to_area_pdf(const T pdf, const T cosine, const T distance)
{
        if (cosine > 0)
        {
                return pdf * cosine / power<N - 1>(distance);
        }
        return 0;
}

// ---------------------------------------------------------------------------
// GGX (ggx.h)

template <typename T>
NBPT_HD T ggx_lambda(const T n_v, const T alpha)
{
        const T n_v_2 = square(n_v);
        const T t = square(alpha) * (1 - n_v_2) / n_v_2;
        return (sqrt_value(1 + t) - 1) / 2;
}

template <typename T>
NBPT_HD T ggx_g1(const T n_v, const T alpha)
{
        return 1 / (1 + ggx_lambda(n_v, alpha));
}

template <typename T>
NBPT_HD T ggx_g2(const T n_v, const T n_l, const T alpha)
{
        return 1 / (1 + ggx_lambda(n_v, alpha) + ggx_lambda(n_l, alpha));
}

template <int N, typename T>
NBPT_HD T ggx_d(const T n_h, const T alpha, const T k)
{
        if (n_h > 0)
        {
                const T alpha_2 = square(alpha);
                const T v = 1 + square(n_h) * (alpha_2 - 1);
                T v_power = power<(N + 1) / 2>(v);
                if constexpr (((N + 1) & 1) == 1)
                {
                        v_power *= sqrt_value(v);
                }
                return alpha_2 / (k * v_power);
        }
        return 0;
}

template <int N, typename T>
NBPT_HD T ggx_visible_normals_h_pdf(const T n_v, const T n_h, const T h_v, const T alpha, const T k)
{
        if (n_v > 0 && n_h > 0 && h_v > 0)
        {
                return ggx_g1(n_v, alpha) * h_v * ggx_d<N>(n_h, alpha, k) / n_v;
        }
        return 0;
}

template <int N, typename T>
NBPT_HD T ggx_visible_normals_l_pdf(const T n_v, const T n_h, const T h_v, const T alpha, const T k)
{
        return reflected_pdf<N>(ggx_visible_normals_h_pdf<N>(n_v, n_h, h_v, alpha, k), h_v);
}

// Orthonormal basis whose last vector is orthogonal to the others and to vh
// (ggx.h:139-171).
template <int N, typename T>
NBPT_HD void ggx_basis(const Vec<N, T>& vh, Vec<N, T>* res)
{
        T length_s = 0;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                length_s += square(vh[i]);
        }
        if (length_s > 0)
        {
                const T length = sqrt_value(length_s);
                Vec<N - 1, T> plane_v;
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        plane_v[i] = vh[i] / length;
                }
                Vec<N - 1, T> plane_basis[N - 2];
                orthogonal_complement_of_unit_vector(plane_v, plane_basis);
#pragma unroll
                for (int i = 0; i < N - 2; ++i)
                {
#pragma unroll
                        for (int k = 0; k < N - 1; ++k)
                        {
                                res[i][k] = plane_basis[i][k];
                        }
                        res[i][N - 1] = 0;
                }
        }
        else
        {
#pragma unroll
                for (int i = 0; i < N - 2; ++i)
                {
                        res[i] = Vec<N, T>::filled(0);
                        res[i][i] = 1;
                }
        }
        res[N - 2] = vh;
        res[N - 2] = orthogonal_complement(res);
        if (res[N - 2][N - 1] < 0)
        {
                res[N - 2] = -res[N - 2];
        }
}

// Visible-normal sample in the local frame (ggx.h:173-233), from the point
// `t` drawn uniformly in the unit (N-1)-ball (the sample's only random draw)
// and its squared length.
template <int N, typename T>
NBPT_HD Vec<N, T> ggx_vn_from_ball(const Vec<N, T>& ve, const T alpha, Vec<N - 1, T> t, const T length_square)
{
        Vec<N, T> t0;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                t0[i] = alpha * ve[i];
        }
        t0[N - 1] = ve[N - 1];
        const Vec<N, T> vh = t0.normalized();

        Vec<N, T> basis[N - 1];
        ggx_basis(vh, basis);

        static_cast<void>(length_square);
        const T s = T(0.5) * (1 + vh[N - 1]);
        T sum = 0;
#pragma unroll
        for (int i = 0; i < N - 2; ++i)
        {
                sum += square(t[i]);
        }
        const T a = sqrt_value(1 - sum);
        t[N - 2] = interpolation(a, t[N - 2], s);

        Vec<N, T> nh = vh * sqrt_value(max_value(T(0), 1 - dot(t, t)));
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                nh.multiply_add(basis[i], t[i]);
        }

        Vec<N, T> ne;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                ne[i] = alpha * nh[i];
        }
        ne[N - 1] = max_value(T(0), nh[N - 1]);
        return ne.normalized();
}

// the visible-normal half vector about `normal` (ggx.h:235-260), given the
// orthonormal complement of `normal` and the ball point of ggx_vn_from_ball
template <int N, typename T>
NBPT_HD Vec<N, T> ggx_visible_normals_h(const Vec<N, T>& normal, const Vec<N, T>* basis, const Vec<N, T>& v,
                                        const T alpha, const Vec<N - 1, T>& ball, const T ball_length_square)
{
        Vec<N, T> ve;
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                ve[i] = dot(v, basis[i]);
        }
        ve[N - 1] = dot(v, normal);
        const Vec<N, T> ne = ggx_vn_from_ball(ve, alpha, ball, ball_length_square);
        Vec<N, T> r = normal * ne[N - 1];
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
                r.multiply_add(basis[i], ne[i]);
        }
        return r;
}

// (2 * dot(v, n)) * n - v  (numerical/optics.h:46-51)
template <int N, typename T>
NBPT_HD Vec<N, T> reflect_vn(const Vec<N, T>& v, const Vec<N, T>& n)
{
        return n * (2 * dot(v, n)) - v;
}

// ---------------------------------------------------------------------------
// f1 albedo interpolation (f1_albedo.cpp:614-635, numerical/interpolation.h)

template <typename T>
NBPT_HD void interpolation_cell(const T p, int& x0, int& x1, T& x)
{
        const T v = p * T(32) - T(0.5);
        const T f = floor_value(v);
        x = v - f;
        x0 = static_cast<int>(f);
        x1 = x0 + 1;
        x0 = x0 < 0 ? 0 : (x0 > 31 ? 31 : x0);
        x1 = x1 < 0 ? 0 : (x1 > 31 ? 31 : x1);
}

template <typename T>
NBPT_HD T f1_albedo(const ShadingConstants<T>& sc, const T roughness, const T cosine)
{
        int c0, c1, r0, r1;
        T xc, xr;
        interpolation_cell(cosine, c0, c1, xc);
        interpolation_cell(roughness, r0, r1, xr);
        const T* d = sc.f1_albedo;
        const T t0 = interpolation(d[c0 + 32 * r0], d[c1 + 32 * r0], xc);
        const T t1 = interpolation(d[c0 + 32 * r1], d[c1 + 32 * r1], xc);
        return interpolation(t0, t1, xr);
}

template <typename T>
NBPT_HD T f1_albedo_average(const ShadingConstants<T>& sc, const T roughness)
{
        int r0, r1;
        T xr;
        interpolation_cell(roughness, r0, r1, xr);
        return interpolation(sc.f1_average[r0], sc.f1_average[r1], xr);
}

// ---------------------------------------------------------------------------
// BRDF terms

// The scalar factors of one evaluation of brdf::f.  Every term of the BRDF
// is a colour-channel-wise function of f0 and rho_ss with these factors,
// converted to float as the reference converts them; brdf_channel() applies
// them to one channel.  Both the full-colour evaluation below and the
// channel-parallel evaluation of recorded paths go through brdf_channel(),
// so they give the same floats.
struct BrdfTerms final
{
        float fresnel_t; // float(power<5>(1 - h.l)), Schlick Fresnel (fresnel.h:37-45)
        float ggx;       // float(D * G2 / divisor), the GGX term without Fresnel
        float bounce_d;  // multiple-bounce numerator factor (multiple_bounce.h:40-64)
        float bounce_m;  // float(1 - average f1 albedo)
        float diffuse;   // float(c / k), diffuse_disney_ws (subsurface.h:67-78)
        int ggx_on;      // n.v > 0, n.l > 0 and h.l > 0: the GGX term is present
};

template <int N, typename T>
NBPT_HD_CALL BrdfTerms brdf_terms(
        const ShadingConstants<T>& sc,
        const T roughness,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        const Vec<N, T>& l)
{
        const Vec<N, T> h = (l + v).normalized();
        const T n_l = dot(n, l);
        const T h_l = dot(h, l);
        const T n_v = dot(n, v);
        const T n_h = dot(n, h);
        BrdfTerms r;
        // ggx_brdf (ggx.h:360-380)
        r.ggx_on = (n_v > 0 && n_l > 0 && h_l > 0) ? 1 : 0;
        r.fresnel_t = 0;
        r.ggx = 0;
        if (r.ggx_on)
        {
                const T alpha = square(roughness);
                const T d = ggx_d<N>(n_h, alpha, sc.k);
                const T g2 = ggx_g2(n_v, n_l, alpha);
                const T divisor = (n_v * n_l * T(1 << (N - 1)) * power<N - 3>(h_l));
                r.fresnel_t = static_cast<float>(power<5>(1 - h_l));
                r.ggx = static_cast<float>(d * g2 / divisor);
        }
        // multiple_bounce_surface_reflection (multiple_bounce.h:40-64)
        const T rs_f1 = f1_albedo_average(sc, roughness);
        const T rs_f1_l = f1_albedo(sc, roughness, n_l);
        const T rs_f1_v = f1_albedo(sc, roughness, n_v);
        r.bounce_d = static_cast<float>(rs_f1 * (1 - rs_f1_l) * (1 - rs_f1_v) / (sc.k * (1 - rs_f1)));
        r.bounce_m = static_cast<float>(1 - rs_f1);
        // diffuse_disney_ws
        const T lp = power<5>(1 - n_l);
        const T vp = power<5>(1 - n_v);
        const T f_d90 = 2 * roughness * square(h_l);
        const T c = (1 + (f_d90 - 1) * lp) * (1 + (f_d90 - 1) * vp);
        r.diffuse = static_cast<float>(c * sc.k_inv);
        return r;
}

// One channel of ggx + multiple bounce + diffuse, summed in that order
// (brdf.h:48-71).
NBPT_HD float brdf_channel(const BrdfTerms& t, const float f0, const float rho_ss, const float fresnel_a,
                           const float fresnel_b)
{
        float r = 0.0f;
        if (t.ggx_on)
        {
                const float fresnel = (1 - t.fresnel_t) * f0 + t.fresnel_t * 1.0f;
                r = fresnel * t.ggx;
        }
        const float f = f0 * fresnel_a + fresnel_b;
        const float d = f * t.bounce_d;
        const float m = f * t.bounce_m;
        r += d / (1.0f - m);
        r += ((1.0f - f0) * t.diffuse) * rho_ss;
        return r;
}

template <int C, typename T>
NBPT_HD Color<C> brdf_color(const ShadingConstants<T>& sc, const BrdfTerms& t, const Color<C>& f0,
                            const Color<C>& rho_ss)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = brdf_channel(t, f0.c[i], rho_ss.c[i], sc.fresnel_a, sc.fresnel_b);
        }
        return r;
}

template <int N, int C, typename T>
NBPT_HD Color<C> brdf_f_unchecked(
        const ShadingConstants<T>& sc,
        const T roughness,
        const Color<C>& f0,
        const Color<C>& rho_ss,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        const Vec<N, T>& l,
        BrdfTerms* const terms = nullptr)
{
        const BrdfTerms t = brdf_terms<N>(sc, roughness, n, v, l);
        if (terms)
        {
                *terms = t;
        }
        return brdf_color<C>(sc, t, f0, rho_ss);
}

// brdf::f (brdf.h:146-171)
template <int N, int C, typename T>
NBPT_HD Color<C> brdf_f(
        const ShadingConstants<T>& sc,
        const T roughness,
        const Color<C>& f0,
        const Color<C>& rho_ss,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        const Vec<N, T>& l,
        BrdfTerms* const terms = nullptr)
{
        if (dot(n, v) <= 0)
        {
                return Color<C>::filled(0);
        }
        if (dot(n, l) <= 0)
        {
                return Color<C>::filled(0);
        }
        return brdf_f_unchecked<N>(sc, roughness, f0, rho_ss, n, v, l, terms);
}

template <int N, typename T>
NBPT_HD T pdf_ggx_cosine(
        const ShadingConstants<T>& sc,
        const T alpha,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        const Vec<N, T>& l,
        const Vec<N, T>& h)
{
        const T pdf_ggx = ggx_visible_normals_l_pdf<N>(dot(n, v), dot(n, h), dot(h, l), alpha, sc.k);
        const T pdf_cosine = cosine_on_hemisphere_pdf(dot(n, l), sc.k_inv);
        return T(0.5) * (pdf_cosine + pdf_ggx);
}

// brdf::pdf (brdf.h:173-194)
template <int N, typename T>
NBPT_HD_CALL T brdf_pdf(
        const ShadingConstants<T>& sc,
        const T roughness,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        const Vec<N, T>& l)
{
        if (dot(n, v) <= 0)
        {
                return 0;
        }
        const T alpha = square(roughness);
        return pdf_ggx_cosine(sc, alpha, n, v, l, (v + l).normalized());
}

template <int N, int C, typename T>
struct BrdfSample final
{
        Vec<N, T> l;
        T pdf;
        Color<C> brdf;
};

// brdf::sample_f (brdf.h:109-141, 196-238): a 50/50 mix of GGX
// visible-normal and cosine sampling.
template <int N, int C, typename T>
NBPT_HD_CALL BrdfSample<N, C, T> brdf_sample(
        Pcg& g,
        const ShadingConstants<T>& sc,
        const T roughness,
        const Color<C>& f0,
        const Color<C>& rho_ss,
        const Vec<N, T>& n,
        const Vec<N, T>& v,
        BrdfTerms* const terms = nullptr)
{
        BrdfSample<N, C, T> s;
        s.pdf = 0;
        if (dot(n, v) <= 0)
        {
                return s;
        }
        const T alpha = square(roughness);
        Vec<N, T> l;
        Vec<N, T> h;
        // Both ways draw one point in the unit (N-1)-ball after the choice
        // and work in the complement of n (ggx.h:235-260,
        // sphere_cosine.h:41-80), so the complement and the draw are shared
        // and only the arithmetic between them diverges.
        const bool ggx = bernoulli_half(g);
        Vec<N, T> basis[N - 1];
        orthogonal_complement_of_unit_vector(n, basis);
        Vec<N - 1, T> ball;
        T ball_length_square;
        uniform_in_ball<N - 1>(g, ball, ball_length_square);
        if (ggx)
        {
                h = ggx_visible_normals_h(n, basis, v, alpha, ball, ball_length_square);
                l = reflect_vn(v, h);
        }
        else
        {
                l = cosine_from_ball(n, basis, ball, ball_length_square);
                h = (v + l).normalized();
        }
        const T pdf = pdf_ggx_cosine(sc, alpha, n, v, l, h);
        s.l = l;
        s.pdf = pdf;
        if (pdf <= 0)
        {
                s.pdf = 0;
                return s;
        }
        if (dot(n, l) <= 0)
        {
                s.brdf = Color<C>::filled(0);
                return s;
        }
        s.brdf = brdf_f_unchecked<N>(sc, roughness, f0, rho_ss, n, v, l, terms);
        return s;
}
} // namespace nbpt
