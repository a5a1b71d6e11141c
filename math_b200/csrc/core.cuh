// Core numeric types of the accelerated n-D painter: fixed-size vectors,
// colours, the PCG32 engine with seed_seq seeding, and the floating-point
// distributions the path consumes random numbers through.
//
// Arithmetic order.  Every operation here reproduces the reference's order of
// floating-point operations (src/numerical/vector.h:164-173 left-to-right dot
// products; vector_object.h:201-247 norm and normalisation by division;
// src/com/exponent.h power<>), and the library is compiled without
// multiply-add contraction, so that double-precision results are bit-identical
// to the reference's on the same inputs.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define NBPT_HD __host__ __device__ __forceinline__
// Large functions called from several places of the path kernels are kept
// out of line: inlined at every call site they multiply the kernel's code
// beyond the instruction cache.
#define NBPT_HD_CALL __host__ __device__ __noinline__
#define NBPT_CALL __device__ __noinline__
#else
#define NBPT_HD inline
#define NBPT_HD_CALL inline
#define NBPT_CALL inline
#endif

namespace nbpt
{
// ---------------------------------------------------------------------------
// scalar helpers

template <typename T>
NBPT_HD T square(const T v)
{
        return v * v;
}

template <typename T>
NBPT_HD T abs_value(const T v)
{
        return v < 0 ? -v : (v == 0 ? T(0) : v);
}

NBPT_HD float sqrt_value(const float v)
{
#if defined(__CUDA_ARCH__)
        return __fsqrt_rn(v);
#else
        return __builtin_sqrtf(v);
#endif
}

NBPT_HD double sqrt_value(const double v)
{
#if defined(__CUDA_ARCH__)
        return __dsqrt_rn(v);
#else
        return __builtin_sqrt(v);
#endif
}

NBPT_HD float floor_value(const float v)
{
#if defined(__CUDA_ARCH__)
        return floorf(v);
#else
        return __builtin_floorf(v);
#endif
}

NBPT_HD double floor_value(const double v)
{
#if defined(__CUDA_ARCH__)
        return floor(v);
#else
        return __builtin_floor(v);
#endif
}

// std::max / std::min as the reference uses them: max(a, b) returns a unless
// a < b (src/com/exponent.h sqrt_s, std::max in brdf and spectrum code).
template <typename T>
NBPT_HD T max_value(const T a, const T b)
{
        return (a < b) ? b : a;
}

template <typename T>
NBPT_HD T min_value(const T a, const T b)
{
        return (b < a) ? b : a;
}

// power<E>(x) with the reference's multiplication tree (src/com/exponent.h:38-105).
template <unsigned E, typename T>
NBPT_HD T power(const T base)
{
        if constexpr (E == 0)
        {
                return T(1);
        }
        else if constexpr (E == 1)
        {
                return base;
        }
        else if constexpr (E == 2)
        {
                return base * base;
        }
        else if constexpr (E == 3)
        {
                return base * base * base;
        }
        else if constexpr (E == 4)
        {
                const T t = base * base;
                return t * t;
        }
        else if constexpr (E == 5)
        {
                const T t = base * base;
                return t * t * base;
        }
        else if constexpr (E == 6)
        {
                const T t = base * base;
                return t * t * t;
        }
        else if constexpr (E == 7)
        {
                const T t = base * base;
                return t * t * t * base;
        }
        else if constexpr (E == 8)
        {
                const T t = base * base;
                const T t2 = t * t;
                return t2 * t2;
        }
        else
        {
                T res = (E & 1) ? base : T(1);
                T b = base;
                unsigned e = E >> 1;
                while (e)
                {
                        b *= b;
                        if (e & 1)
                        {
                                res *= b;
                        }
                        e >>= 1;
                }
                return res;
        }
}

// (1 - t) * a + t * b  (src/com/interpolation.h:27-30)
template <typename T>
NBPT_HD T interpolation(const T a, const T b, const T t)
{
        return (1 - t) * a + t * b;
}

template <typename T>
struct Limits;

template <>
struct Limits<float>
{
        static constexpr float EPSILON = 1.1920928955078125e-07f;
        static constexpr float MAX = 3.40282346638528859812e+38f;
};

template <>
struct Limits<double>
{
        static constexpr double EPSILON = 2.220446049250313080847e-16;
        static constexpr double MAX = 1.79769313486231570815e+308;
};

template <typename T>
NBPT_HD T infinity();

template <>
NBPT_HD float infinity<float>()
{
        return __builtin_huge_valf();
}

template <>
NBPT_HD double infinity<double>()
{
        return __builtin_huge_val();
}

// ---------------------------------------------------------------------------
// vectors

template <int N, typename T>
struct Vec final
{
        T v[N];

        NBPT_HD T& operator[](const int i)
        {
                return v[i];
        }

        NBPT_HD const T& operator[](const int i) const
        {
                return v[i];
        }

        NBPT_HD static Vec filled(const T x)
        {
                Vec r;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        r.v[i] = x;
                }
                return r;
        }

        NBPT_HD T norm_squared() const
        {
                T s = v[0] * v[0];
#pragma unroll
                for (int i = 1; i < N; ++i)
                {
                        s += v[i] * v[i];
                }
                return s;
        }

        NBPT_HD T norm() const
        {
                return sqrt_value(norm_squared());
        }

        NBPT_HD Vec normalized() const
        {
                const T n = norm();
                Vec r;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        r.v[i] = v[i] / n;
                }
                return r;
        }

        // this[i] += a[i] * b  (vector_object.h:160-166)
        NBPT_HD void multiply_add(const Vec& a, const T b)
        {
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        v[i] += a.v[i] * b;
                }
        }
};

template <int N, typename T>
NBPT_HD T dot(const Vec<N, T>& a, const Vec<N, T>& b)
{
        T r = a[0] * b[0];
#pragma unroll
        for (int i = 1; i < N; ++i)
        {
                r += a[i] * b[i];
        }
        return r;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator+(const Vec<N, T>& a, const Vec<N, T>& b)
{
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = a[i] + b[i];
        }
        return r;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator-(const Vec<N, T>& a, const Vec<N, T>& b)
{
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = a[i] - b[i];
        }
        return r;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator-(const Vec<N, T>& a)
{
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = -a[i];
        }
        return r;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator*(const Vec<N, T>& a, const T b)
{
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = a[i] * b;
        }
        return r;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator*(const T b, const Vec<N, T>& a)
{
        return a * b;
}

template <int N, typename T>
NBPT_HD Vec<N, T> operator/(const Vec<N, T>& a, const T b)
{
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = a[i] / b;
        }
        return r;
}

template <int N, typename T>
NBPT_HD bool operator==(const Vec<N, T>& a, const Vec<N, T>& b)
{
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                if (!(a[i] == b[i]))
                {
                        return false;
                }
        }
        return true;
}

// ---------------------------------------------------------------------------
// colours: 3 (RGB) or 64 (spectrum) float channels; the reference keeps colour
// in float whatever the geometry precision (src/color/color.h:416-417).

template <int C>
struct Color final
{
        float c[C];

        NBPT_HD static Color filled(const float x)
        {
                Color r;
#pragma unroll
                for (int i = 0; i < C; ++i)
                {
                        r.c[i] = x;
                }
                return r;
        }

        // The reference's is_black() inspects channel 0 only
        // (src/color/samples.h:109-119); this keeps that behaviour.
        NBPT_HD bool is_black() const
        {
                return c[0] <= 0;
        }

        NBPT_HD Color& operator+=(const Color& b)
        {
#pragma unroll
                for (int i = 0; i < C; ++i)
                {
                        c[i] += b.c[i];
                }
                return *this;
        }

        NBPT_HD Color& operator*=(const Color& b)
        {
#pragma unroll
                for (int i = 0; i < C; ++i)
                {
                        c[i] *= b.c[i];
                }
                return *this;
        }

        NBPT_HD Color& operator*=(const float b)
        {
#pragma unroll
                for (int i = 0; i < C; ++i)
                {
                        c[i] *= b;
                }
                return *this;
        }
};

template <int C>
NBPT_HD Color<C> operator+(const Color<C>& a, const Color<C>& b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] + b.c[i];
        }
        return r;
}

template <int C>
NBPT_HD Color<C> operator-(const Color<C>& a, const Color<C>& b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] - b.c[i];
        }
        return r;
}

template <int C>
NBPT_HD Color<C> operator*(const Color<C>& a, const Color<C>& b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] * b.c[i];
        }
        return r;
}

// Colour times scalar: the scalar is first converted to float, as the
// reference's Samples::operator*(const Derived&, const T&) with T = float
// receives it.
template <int C>
NBPT_HD Color<C> operator*(const Color<C>& a, const float b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] * b;
        }
        return r;
}

template <int C>
NBPT_HD Color<C> operator/(const Color<C>& a, const Color<C>& b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] / b.c[i];
        }
        return r;
}

template <int C>
NBPT_HD Color<C> operator/(const Color<C>& a, const float b)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = a.c[i] / b;
        }
        return r;
}

template <int C>
NBPT_HD Color<C> color_interpolation(const Color<C>& a, const Color<C>& b, const float t)
{
        Color<C> r;
#pragma unroll
        for (int i = 0; i < C; ++i)
        {
                r.c[i] = interpolation(a.c[i], b.c[i], t);
        }
        return r;
}

// ---------------------------------------------------------------------------
// random numbers

// PCG-XSH-RR 64/32 (src/com/random/pcg.h:53-62).
struct Pcg final
{
        std::uint64_t state;
        std::uint64_t increment;

        NBPT_HD std::uint32_t operator()()
        {
                constexpr std::uint64_t MULTIPLIER = 6364136223846793005ULL;
                const std::uint64_t x = state;
                state = x * MULTIPLIER + increment;
                const std::uint32_t s = static_cast<std::uint32_t>(((x >> 18) ^ x) >> 27);
                const std::uint32_t r = static_cast<std::uint32_t>(x >> 59);
                return (s >> r) | (s << ((32u - r) & 31u));
        }
};

// std::seed_seq::generate for four output words from `count` input words
// (the algorithm of the C++ standard, [rand.util.seedseq]), and the PCG state
// the reference builds from those four words (src/com/random/pcg.cpp:57-77).
NBPT_HD Pcg seed_seq_pcg(const std::uint32_t* const in, const int count)
{
        constexpr int n = 4;
        constexpr int t = 1; // (n - 1) / 2 for n < 7
        constexpr int p = (n - t) / 2;
        constexpr int q = p + t;
        std::uint32_t b[n] = {0x8b8b8b8bu, 0x8b8b8b8bu, 0x8b8b8b8bu, 0x8b8b8b8bu};
        const int m = (count + 1 > n) ? count + 1 : n;
        for (int k = 0; k < m; ++k)
        {
                std::uint32_t x = b[k % n] ^ b[(k + p) % n] ^ b[(k + n - 1) % n];
                x = x ^ (x >> 27);
                const std::uint32_t r1 = 1664525u * x;
                const std::uint32_t r2 =
                        r1 + (k == 0 ? static_cast<std::uint32_t>(count)
                                     : (k <= count ? static_cast<std::uint32_t>(k % n) + in[k - 1]
                                                   : static_cast<std::uint32_t>(k % n)));
                b[(k + p) % n] += r1;
                b[(k + q) % n] += r2;
                b[k % n] = r2;
        }
        for (int k = m; k < m + n; ++k)
        {
                std::uint32_t x = b[k % n] + b[(k + p) % n] + b[(k + n - 1) % n];
                x = x ^ (x >> 27);
                const std::uint32_t r3 = 1566083941u * x;
                const std::uint32_t r4 = r3 - static_cast<std::uint32_t>(k % n);
                b[(k + p) % n] ^= r3;
                b[(k + q) % n] ^= r4;
                b[k % n] = r4;
        }
        Pcg g;
        g.state = static_cast<std::uint64_t>(b[0]) | (static_cast<std::uint64_t>(b[1]) << 32);
        g.increment = static_cast<std::uint64_t>(b[2]) | (static_cast<std::uint64_t>(b[3]) << 32) | 1u;
        return g;
}

// std::generate_canonical<T, digits(T)> over a 32-bit engine: one draw for
// float, two for double; a result of 1 is replaced by the largest value
// below 1 (the algorithm of [rand.util.canonical] as libstdc++ implements it).
template <typename T>
NBPT_HD T canonical(Pcg& g);

template <>
NBPT_HD float canonical<float>(Pcg& g)
{
        const float sum = static_cast<float>(g());
        const float r = sum / 4294967296.0f;
        return r >= 1.0f ? 0.99999994f : r;
}

template <>
NBPT_HD double canonical<double>(Pcg& g)
{
        double sum = static_cast<double>(g());
        sum += static_cast<double>(g()) * 4294967296.0;
        const double r = sum / 18446744073709551616.0;
        return r >= 1.0 ? 0.99999999999999989 : r;
}

// std::uniform_real_distribution<T>(a, b): canonical * (b - a) + a.
template <typename T>
NBPT_HD T uniform(Pcg& g, const T a, const T b)
{
        return (canonical<T>(g) * (b - a)) + a;
}

// std::bernoulli_distribution(0.5): one double canonical draw < 0.5.
NBPT_HD bool bernoulli_half(Pcg& g)
{
        return canonical<double>(g) < 0.5;
}
} // namespace nbpt
