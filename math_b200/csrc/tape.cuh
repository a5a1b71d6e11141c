// Path tapes: spectral paths traced with one colour channel, then coloured
// channel-parallel.
//
// Every colour of a BPT path is built from per-channel products of a few
// kinds of factors: BRDF values (brdf_channel of a material's f0 and rho_ss
// with scalar BrdfTerms), light radiances, and float scalars (cosines over
// pdfs, geometry terms, MIS weights).  The control flow of the path (which
// bounces happen, which strategies contribute) depends on colours only
// through channel 0 (Color::is_black, as in the reference).  So a path is
// traced once with channel 0 alone, recording every factor on a tape in the
// order the full-colour path multiplies them; a second kernel replays the
// tape for all channels at once, one warp per path and the channels across
// the lanes.  Replaying performs, per channel, the same float operations in
// the same order as the full-colour path, so the colours are identical.
#pragma once

#include "core.cuh"
#include "shading.cuh"

#include <cstdint>

namespace nbpt
{
enum class TapeRecord : int
{
        CAMERA_BOUNCE = 1,    // material, terms, s:     beta *= brdf * s
        LIGHT_START = 2,      // light, s:               beta = radiance * s
        LIGHT_BOUNCE = 3,     // material, terms, s, cn: beta *= brdf * s; beta *= cn
        STRATEGY_EMITTED = 4, // t, light, mis:          (radiance * beta_t) * mis
        STRATEGY_LIGHT = 5,   // t, material, terms, light, x, mis
        STRATEGY_CONNECT = 6  // s, t, material_c, terms_c, material_l, terms_l, g, mis
};

// header: end of the bounce records, valid (not a background sample),
// camera subpath size, light subpath size
inline constexpr int TAPE_HEADER = 4;
inline constexpr int TAPE_TERMS = 6;  // words of a BrdfTerms
inline constexpr int TAPE_CAMERA_BOUNCE = 3 + TAPE_TERMS;
inline constexpr int TAPE_LIGHT_START = 3;
inline constexpr int TAPE_LIGHT_BOUNCE = 4 + TAPE_TERMS;
inline constexpr int TAPE_STRATEGY_EMITTED = 4;
inline constexpr int TAPE_STRATEGY_LIGHT = 6 + TAPE_TERMS;
inline constexpr int TAPE_STRATEGY_CONNECT = 7 + 2 * TAPE_TERMS;

// Layout of one path's tape for a maximum depth D: the header; the bounce
// records in the order they happen (at most D per subpath and the light
// start); then one fixed slot of TAPE_STRATEGY_CONNECT words per (s, t)
// strategy with 2 <= t <= D + 1, 0 <= s and s + t - 2 <= D, in the
// reference's loop order (t outer, s inner).  A slot whose first word is 0
// holds no contribution.
NBPT_HD constexpr int tape_slots_begin(const int max_depth)
{
        return TAPE_HEADER + max_depth * TAPE_CAMERA_BOUNCE + TAPE_LIGHT_START + max_depth * TAPE_LIGHT_BOUNCE;
}

NBPT_HD constexpr int tape_slot_count(const int max_depth)
{
        return (max_depth + 1) * (max_depth + 2) / 2 - 1;
}

// index of strategy (s, t): slots of t' = 2 .. t - 1 (D + 3 - t' each), then s
NBPT_HD constexpr int tape_slot(const int max_depth, const int t, const int s)
{
        return (t - 2) * (max_depth + 3) - ((t - 1) * t / 2 - 1) + s;
}

NBPT_HD constexpr int tape_slot_offset(const int max_depth, const int t, const int s)
{
        return tape_slots_begin(max_depth) + tape_slot(max_depth, t, s) * TAPE_STRATEGY_CONNECT;
}

NBPT_HD constexpr int tape_words(const int max_depth)
{
        return tape_slots_begin(max_depth) + tape_slot_count(max_depth) * TAPE_STRATEGY_CONNECT;
}

static_assert(tape_slot(6, 2, 6) == 6 && tape_slot(6, 3, 0) == 7 && tape_slot(6, 7, 1) == tape_slot_count(6) - 1);

// Appends records to one path's tape (a contiguous slot of 32-bit words).
struct TapeWriter final
{
        std::uint32_t* w = nullptr;
        int n = TAPE_HEADER;

        NBPT_HD void put(const int v)
        {
                w[n++] = static_cast<std::uint32_t>(v);
        }

        NBPT_HD void put(const float v)
        {
                w[n++] = bits_of(v);
        }

        NBPT_HD void put(const BrdfTerms& t)
        {
                put(t.fresnel_t);
                put(t.ggx);
                put(t.bounce_d);
                put(t.bounce_m);
                put(t.diffuse);
                put(t.ggx_on);
        }

        NBPT_HD static std::uint32_t bits_of(const float v)
        {
                std::uint32_t u;
                __builtin_memcpy(&u, &v, sizeof(u));
                return u;
        }
};

// Reads one path's tape.
struct TapeReader final
{
        const std::uint32_t* w;
        int n = TAPE_HEADER;

        NBPT_HD int get_int()
        {
                return static_cast<int>(w[n++]);
        }

        NBPT_HD float get_float()
        {
                const std::uint32_t u = w[n++];
                float v;
                __builtin_memcpy(&v, &u, sizeof(v));
                return v;
        }

        NBPT_HD BrdfTerms get_terms()
        {
                BrdfTerms t;
                t.fresnel_t = get_float();
                t.ggx = get_float();
                t.bounce_d = get_float();
                t.bounce_m = get_float();
                t.diffuse = get_float();
                t.ggx_on = get_int();
                return t;
        }
};
} // namespace nbpt
