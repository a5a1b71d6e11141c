// Host-side scene preparation arithmetic: compile-time constants of the
// path, colour conversions and material colours, each computed the way the
// reference computes them so that the uploaded values are identical.
#pragma once

#include "tables.inc"

#include <array>
#include <cmath>
#include <stdexcept>
#include <vector>

namespace nbpt::host
{
inline constexpr long double PI_L = 3.1415926535897932384626433832795028841971693993751L;

// Area of the unit (n-1)-sphere in n-space (src/geometry/shapes/sphere_area.h:28-68).
inline long double sphere_area(const int n)
{
        const int m = n / 2;
        if ((n & 1) == 0)
        {
                long double res = 2;
                res *= PI_L;
                if (m >= 2)
                {
                        res *= PI_L;
                }
                for (int i = m - 1; i > 1; --i)
                {
                        res /= i;
                        res *= PI_L;
                }
                return res;
        }
        long double res = 2;
        for (int i = 2 * m; i > m; --i)
        {
                res /= i;
                res *= 4;
                res *= PI_L;
        }
        return res;
}

// Integral of the cosine over the hemisphere in n-space
// (src/geometry/shapes/sphere_integral.h: SPHERE_AREA<n-1> / (n-1)).
inline long double hemisphere_cosine_integral(const int n)
{
        if (n == 2)
        {
                return 2.0L;
        }
        return sphere_area(n - 1) / (n - 1);
}

// Volume of the unit m-ball (src/geometry/shapes/ball_volume.h:28-35).
inline long double ball_volume(const int m)
{
        return sphere_area(m) / m;
}

// a * f0 + b: cosine-weighted average of Schlick's Fresnel term
// (src/shading/ggx/fresnel.h:50-87), evaluated in float.
inline std::array<float, 2> fresnel_average(const int n)
{
        constexpr float PI_F = static_cast<float>(PI_L);
        switch (n)
        {
        case 3:
                return {20.0f / 21, 1.0f / 21};
        case 4:
                return {495 * PI_F / 256 - 36.0f / 7, 43.0f / 7 - 495 * PI_F / 256};
        case 5:
                return {115.0f / 126, 11.0f / 126};
        default:
                throw std::runtime_error("dimension must be 3, 4 or 5");
        }
}

// ---------------------------------------------------------------------------
// colours

enum SpectrumRow
{
        CIE_X = 0,
        CIE_Y = 1,
        CIE_Z = 2,
        REFLECTANCE = 3,
        ILLUMINATION = 10
};

// basis colour order inside a reflectance or illumination block
enum Basis
{
        WHITE = 0,
        CYAN = 1,
        MAGENTA = 2,
        YELLOW = 3,
        RED = 4,
        GREEN = 5,
        BLUE = 6
};

inline const std::vector<float>& spectrum_row(const int row)
{
        static const std::vector<std::vector<float>> rows = []
        {
                std::vector<std::vector<float>> r(17, std::vector<float>(64));
                for (int i = 0; i < 17; ++i)
                {
                        for (int k = 0; k < 64; ++k)
                        {
                                r[i][k] = static_cast<float>(tables::SPECTRUM[i][k]);
                        }
                }
                return r;
        }();
        return rows[row];
}

inline float max0(const float v)
{
        return (0.0f < v) ? v : 0.0f;
}

// s += basis * k  (vector multiply_add order)
inline void add_scaled(std::vector<float>& s, const int row, const float k)
{
        const std::vector<float>& b = spectrum_row(row);
        for (int i = 0; i < 64; ++i)
        {
                s[i] += b[i] * k;
        }
}

// Smits RGB to spectrum (src/color/color.h:212-310), float arithmetic.
inline std::vector<float> rgb_to_spectrum(float r, float g, float b, const int block)
{
        r = max0(r);
        g = max0(g);
        b = max0(b);
        std::vector<float> s(64, 0.0f);
        if (r <= g && r <= b)
        {
                add_scaled(s, block + WHITE, r);
                if (g <= b)
                {
                        add_scaled(s, block + CYAN, g - r);
                        add_scaled(s, block + BLUE, b - g);
                }
                else
                {
                        add_scaled(s, block + CYAN, b - r);
                        add_scaled(s, block + GREEN, g - b);
                }
        }
        else if (g <= r && g <= b)
        {
                add_scaled(s, block + WHITE, g);
                if (r <= b)
                {
                        add_scaled(s, block + MAGENTA, r - g);
                        add_scaled(s, block + BLUE, b - r);
                }
                else
                {
                        add_scaled(s, block + MAGENTA, b - g);
                        add_scaled(s, block + RED, r - b);
                }
        }
        else if (b <= r && b <= g)
        {
                add_scaled(s, block + WHITE, b);
                if (r <= g)
                {
                        add_scaled(s, block + YELLOW, r - b);
                        add_scaled(s, block + GREEN, g - r);
                }
                else
                {
                        add_scaled(s, block + YELLOW, g - b);
                        add_scaled(s, block + RED, r - g);
                }
        }
        for (float& v : s)
        {
                v = (v < 0.0f) ? 0.0f : v;
        }
        return s;
}

// Color(r, g, b) for a surface: RGB clamps at 0, a spectrum uses the
// reflectance basis.
inline std::vector<float> surface_color(const int channels, const float* rgb)
{
        if (channels == 3)
        {
                return {max0(rgb[0]), max0(rgb[1]), max0(rgb[2])};
        }
        return rgb_to_spectrum(rgb[0], rgb[1], rgb[2], REFLECTANCE);
}

// Color::illuminant(r, g, b) for a light.
inline std::vector<float> illuminant_color(const int channels, const float* rgb)
{
        if (channels == 3)
        {
                return {max0(rgb[0]), max0(rgb[1]), max0(rgb[2])};
        }
        return rgb_to_spectrum(rgb[0], rgb[1], rgb[2], ILLUMINATION);
}

inline float clamp01(const float v)
{
        return (v < 0.0f) ? 0.0f : ((1.0f < v) ? 1.0f : v);
}

// f0 and rho_ss of the GGX material (src/shading/ggx/metalness.h:34-44):
// f0 = interpolation(0.05, colour, metalness), rho_ss = interpolation(colour, 0, metalness).
inline void metalness_colors(const std::vector<float>& color, const float metalness, std::vector<float>& f0,
                             std::vector<float>& rho_ss)
{
        f0.resize(color.size());
        rho_ss.resize(color.size());
        for (std::size_t i = 0; i < color.size(); ++i)
        {
                f0[i] = (1 - metalness) * 0.05f + metalness * color[i];
                rho_ss[i] = (1 - metalness) * color[i] + metalness * 0.0f;
        }
}
} // namespace nbpt::host
