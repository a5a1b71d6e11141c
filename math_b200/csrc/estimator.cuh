// The painter's per-pixel estimator on the GPU: filtered, trimmed, with the
// reference's exact merge semantics.
//
// Every sample of a source pixel is splatted into its 3^(n-1) neighbours with
// the truncated Gaussian weight (src/painter/pixels/pixel_filter.h:32-70,
// gaussian.h:38-78).  For one (receiving pixel, source pixel) pair the
// weighted samples form a group; the group's two lowest and two highest
// weighted luminances are held out and the rest summed
// (samples/create.cpp:147-250); the group is merged into the receiving
// pixel's state keeping the two lowest and two highest of the union
// (samples/merge.cpp:78-223, com/merge.h:34-233).  Background samples (paths
// that escape at the first hit) keep their own held-out weights.
//
// Which of several equal keys is held out, and the order of the float sums,
// follow the reference step for step: groups are ordered with the same
// insertion-sort and binary-heap selection the reference's sort and
// partial_sort perform, sources are merged into a receiving pixel in
// increasing pixel index, and all sums are in float as the reference keeps
// them.  From the same samples the image is therefore the reference's, bit
// for bit.  One thread gathers for one receiving pixel, so no atomics are
// needed.
//
// The same merges run with the radiance and weight sums in double (the sum
// type S of the sets): the single-precision trace keeps its per-pixel sums
// in double, so that long renders do not lose the small late contributions
// to float rounding.  Held-out samples are float in both forms.
#pragma once

#include "core.cuh"
#include "group_order.h"

#include <cstdint>

namespace nbpt
{

// largest number of samples per pixel a pass can gather in one group
inline constexpr int MAX_GROUP = 256;

// ---------------------------------------------------------------------------
// sample sets (samples/color.h, samples/background.h)

// S is the type of the sums: float as the reference keeps them (the
// bit-exact mode), or double (the radiance sums of the single-precision
// trace kept in double); held-out entries are float samples in both.
template <int C, typename S = float>
struct ColorSet final
{
        S color_sum[C];
        S weight_sum;
        float colors[HELD_OUT][C];
        float weights[HELD_OUT];
        float contributions[HELD_OUT];
        int count; // held-out entries in use
        int full;  // more than HELD_OUT samples seen: the sums are valid
};

template <typename S = float>
struct BackgroundSet final
{
        S weight_sum;
        float weights[HELD_OUT];
        int count;
        int full;
};

template <int C, typename S = float>
struct PixelState final
{
        ColorSet<C, S> color;
        BackgroundSet<S> background;
};

// A group of one source pixel's samples for one receiving pixel: sample
// indices in the source pixel and their float weights; colours are read
// from global memory and weighted on use (sample.color = weight * colour).
template <int C>
struct ColorGroup final
{
        const float* colors; // the source pixel's sample colours [spp][stride]
        const float* weights;
        const float* contributions;
        const int* order;
        int n;
        // channel c of this group is channel c * step + offset of the colours
        // (one thread per pixel: all channels, step 1; one warp per pixel: a
        // lane's channels, step 32 and offset the lane)
        int stride;
        int step;
        int offset;

        NBPT_HD float color(const int k, const int c) const
        {
                const int i = order[k];
                return weights[i] * colors[i * stride + c * step + offset];
        }
};

// ---- merges (com/merge.h) ------------------------------------------------

// Entry accessor over a set or a group, in the set's (sorted) order.
template <int C, typename S>
struct SetView final
{
        const ColorSet<C, S>* s;
        const ColorGroup<C>* g; // when merging a fresh group
        int g_full;
        // group held-out positions: 0, 1 -> order[0], order[1]; 2, 3 -> order[n-2], order[n-1]

        NBPT_HD int count() const
        {
                if (s)
                {
                        return s->full ? HELD_OUT : s->count;
                }
                return g_full ? HELD_OUT : g->n;
        }

        NBPT_HD int group_position(const int k) const
        {
                if (!g_full)
                {
                        return k;
                }
                return k < HELD_OUT / 2 ? k : g->n - HELD_OUT + k;
        }

        NBPT_HD float contribution(const int k) const
        {
                if (s)
                {
                        return s->contributions[k];
                }
                return g->contributions[g->order[group_position(k)]];
        }

        NBPT_HD float weight(const int k) const
        {
                if (s)
                {
                        return s->weights[k];
                }
                return g->weights[g->order[group_position(k)]];
        }

        NBPT_HD float color(const int k, const int c) const
        {
                if (s)
                {
                        return s->colors[k][c];
                }
                return g->color(group_position(k), c);
        }
};

template <int C, typename S>
NBPT_HD void copy_entry(ColorSet<C, S>& out, const int to, const SetView<C, S>& from, const int k)
{
#pragma unroll 8
        for (int c = 0; c < C; ++c)
        {
                out.colors[to][c] = from.color(k, c);
        }
        out.weights[to] = from.weight(k);
        out.contributions[to] = from.contribution(k);
}

template <int C, typename S>
NBPT_HD void sum_entry(S* color_sum, S& weight_sum, const SetView<C, S>& from, const int k)
{
#pragma unroll 8
        for (int c = 0; c < C; ++c)
        {
                color_sum[c] += from.color(k, c);
        }
        weight_sum += from.weight(k);
}

// merge_with_sum (com/merge.h:199-233, samples/merge.cpp:109-145)
template <int C, typename S>
NBPT_HD void merge_colors_with_sum(const SetView<C, S>& a, const SetView<C, S>& b, const S* a_sum, S a_wsum,
                                   const S* b_sum, S b_wsum, const bool a_full, const bool b_full,
                                   ColorSet<C, S>& out)
{
        // samples_color_sum / samples_weight_sum (samples/merge.cpp:37-76)
        S sum[C];
        S wsum;
        if (a_full && b_full)
        {
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        sum[c] = a_sum[c] + b_sum[c];
                }
                wsum = a_wsum + b_wsum;
        }
        else if (a_full)
        {
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        sum[c] = a_sum[c];
                }
                wsum = a_wsum;
        }
        else if (b_full)
        {
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        sum[c] = b_sum[c];
                }
                wsum = b_wsum;
        }
        else
        {
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        sum[c] = 0;
                }
                wsum = 0;
        }

        const int a_size = a.count();
        const int b_size = b.count();
        ColorSet<C, S> r;
        if (a_size == HELD_OUT && b_size == HELD_OUT)
        {
                int ai = 0;
                int bi = 0;
                for (int i = 0; i < HELD_OUT / 2; ++i)
                {
                        if (a.contribution(ai) < b.contribution(bi))
                        {
                                copy_entry(r, i, a, ai++);
                        }
                        else
                        {
                                copy_entry(r, i, b, bi++);
                        }
                }
                while (ai < HELD_OUT / 2)
                {
                        sum_entry(sum, wsum, a, ai++);
                }
                while (bi < HELD_OUT / 2)
                {
                        sum_entry(sum, wsum, b, bi++);
                }
                ai = HELD_OUT - 1;
                bi = HELD_OUT - 1;
                for (int i = HELD_OUT - 1; i >= HELD_OUT / 2; --i)
                {
                        if (a.contribution(ai) > b.contribution(bi))
                        {
                                copy_entry(r, i, a, ai--);
                        }
                        else
                        {
                                copy_entry(r, i, b, bi--);
                        }
                }
                while (ai >= HELD_OUT / 2)
                {
                        sum_entry(sum, wsum, a, ai--);
                }
                while (bi >= HELD_OUT / 2)
                {
                        sum_entry(sum, wsum, b, bi--);
                }
        }
        else
        {
                int ai = 0;
                int bi = 0;
                int i = 0;
                while (i < HELD_OUT / 2 && ai < a_size && bi < b_size)
                {
                        if (a.contribution(ai) < b.contribution(bi))
                        {
                                copy_entry(r, i++, a, ai++);
                        }
                        else
                        {
                                copy_entry(r, i++, b, bi++);
                        }
                }
                while (i < HELD_OUT / 2 && ai < a_size)
                {
                        copy_entry(r, i++, a, ai++);
                }
                while (i < HELD_OUT / 2 && bi < b_size)
                {
                        copy_entry(r, i++, b, bi++);
                }
                const int a_low = ai;
                const int b_low = bi;
                int aj = a_size - 1;
                int bj = b_size - 1;
                int j = HELD_OUT - 1;
                while (j >= HELD_OUT / 2 && aj >= a_low && bj >= b_low)
                {
                        if (a.contribution(aj) > b.contribution(bj))
                        {
                                copy_entry(r, j--, a, aj--);
                        }
                        else
                        {
                                copy_entry(r, j--, b, bj--);
                        }
                }
                while (j >= HELD_OUT / 2 && aj >= a_low)
                {
                        copy_entry(r, j--, a, aj--);
                }
                while (j >= HELD_OUT / 2 && bj >= b_low)
                {
                        copy_entry(r, j--, b, bj--);
                }
                for (int k = a_low; k <= aj; ++k)
                {
                        sum_entry(sum, wsum, a, k);
                }
                for (int k = b_low; k <= bj; ++k)
                {
                        sum_entry(sum, wsum, b, k);
                }
        }
#pragma unroll 8
        for (int c = 0; c < C; ++c)
        {
                r.color_sum[c] = sum[c];
        }
        r.weight_sum = wsum;
        r.count = HELD_OUT;
        r.full = 1;
        out = r;
}

// Merge a fresh group into a pixel's colour set (samples/merge.cpp:198-223).
template <int C, typename S>
NBPT_HD void merge_color_group(ColorSet<C, S>& s, const ColorGroup<C>& g, const S* g_sum, const S g_wsum,
                               const bool g_full)
{
        const SetView<C, S> a{&s, nullptr, 0};
        const SetView<C, S> b{nullptr, &g, g_full ? 1 : 0};
        const int a_count = a.count();
        const int b_count = b.count();
        if (a_count + b_count > HELD_OUT)
        {
                merge_colors_with_sum(a, b, s.color_sum, s.weight_sum, g_sum, g_wsum, s.full != 0, g_full, s);
                return;
        }
        if (b_count == 0)
        {
                return;
        }
        if (a_count == 0)
        {
                // the group as created, held-out entries and sums
                ColorSet<C, S> r;
                for (int k = 0; k < b_count; ++k)
                {
                        copy_entry(r, k, b, k);
                }
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        r.color_sum[c] = g_full ? g_sum[c] : S(0);
                }
                r.weight_sum = g_full ? g_wsum : S(0);
                r.count = b_count;
                r.full = g_full ? 1 : 0;
                s = r;
                return;
        }
        // merge (com/merge.h:235-271): sorted merge of two small sets
        ColorSet<C, S> r;
        int i = 0;
        int ai = 0;
        int bi = 0;
        while (ai < a_count && bi < b_count)
        {
                if (a.contribution(ai) < b.contribution(bi))
                {
                        copy_entry(r, i++, a, ai++);
                }
                else
                {
                        copy_entry(r, i++, b, bi++);
                }
        }
        while (ai < a_count)
        {
                copy_entry(r, i++, a, ai++);
        }
        while (bi < b_count)
        {
                copy_entry(r, i++, b, bi++);
        }
        r.count = a_count + b_count;
        r.full = 0;
        s = r;
}

// Background sets: the same merges on weights only.
template <typename S>
NBPT_HD void merge_background_group(BackgroundSet<S>& s, const float* gw, const int n)
{
        // gw: the group's weights, already ordered (order_group on values)
        const bool g_full = n > HELD_OUT;
        float held[HELD_OUT];
        S g_sum = 0;
        int g_count = n;
        if (g_full)
        {
                held[0] = gw[0];
                held[1] = gw[1];
                for (int k = 2; k < n - 2; ++k)
                {
                        g_sum += gw[k];
                }
                held[2] = gw[n - 2];
                held[3] = gw[n - 1];
                g_count = HELD_OUT;
        }
        else
        {
                for (int k = 0; k < n; ++k)
                {
                        held[k] = gw[k];
                }
        }
        const int a_count = s.full ? HELD_OUT : s.count;
        if (a_count + g_count > HELD_OUT)
        {
                S wsum;
                if (s.full && g_full)
                {
                        wsum = s.weight_sum + g_sum;
                }
                else if (s.full)
                {
                        wsum = s.weight_sum;
                }
                else if (g_full)
                {
                        wsum = g_sum;
                }
                else
                {
                        wsum = 0;
                }
                float out[HELD_OUT];
                const float* a = s.weights;
                const float* b = held;
                const int a_size = a_count;
                const int b_size = g_count;
                if (a_size == HELD_OUT && b_size == HELD_OUT)
                {
                        int ai = 0;
                        int bi = 0;
                        for (int i = 0; i < HELD_OUT / 2; ++i)
                        {
                                out[i] = (a[ai] < b[bi]) ? a[ai++] : b[bi++];
                        }
                        while (ai < HELD_OUT / 2)
                        {
                                wsum += a[ai++];
                        }
                        while (bi < HELD_OUT / 2)
                        {
                                wsum += b[bi++];
                        }
                        ai = HELD_OUT - 1;
                        bi = HELD_OUT - 1;
                        for (int i = HELD_OUT - 1; i >= HELD_OUT / 2; --i)
                        {
                                out[i] = (a[ai] > b[bi]) ? a[ai--] : b[bi--];
                        }
                        while (ai >= HELD_OUT / 2)
                        {
                                wsum += a[ai--];
                        }
                        while (bi >= HELD_OUT / 2)
                        {
                                wsum += b[bi--];
                        }
                }
                else
                {
                        int ai = 0;
                        int bi = 0;
                        int i = 0;
                        while (i < HELD_OUT / 2 && ai < a_size && bi < b_size)
                        {
                                out[i++] = (a[ai] < b[bi]) ? a[ai++] : b[bi++];
                        }
                        while (i < HELD_OUT / 2 && ai < a_size)
                        {
                                out[i++] = a[ai++];
                        }
                        while (i < HELD_OUT / 2 && bi < b_size)
                        {
                                out[i++] = b[bi++];
                        }
                        const int a_low = ai;
                        const int b_low = bi;
                        int aj = a_size - 1;
                        int bj = b_size - 1;
                        int j = HELD_OUT - 1;
                        while (j >= HELD_OUT / 2 && aj >= a_low && bj >= b_low)
                        {
                                out[j--] = (a[aj] > b[bj]) ? a[aj--] : b[bj--];
                        }
                        while (j >= HELD_OUT / 2 && aj >= a_low)
                        {
                                out[j--] = a[aj--];
                        }
                        while (j >= HELD_OUT / 2 && bj >= b_low)
                        {
                                out[j--] = b[bj--];
                        }
                        for (int k = a_low; k <= aj; ++k)
                        {
                                wsum += a[k];
                        }
                        for (int k = b_low; k <= bj; ++k)
                        {
                                wsum += b[k];
                        }
                }
                for (int k = 0; k < HELD_OUT; ++k)
                {
                        s.weights[k] = out[k];
                }
                s.weight_sum = wsum;
                s.count = HELD_OUT;
                s.full = 1;
                return;
        }
        if (g_count == 0)
        {
                return;
        }
        if (a_count == 0)
        {
                for (int k = 0; k < g_count; ++k)
                {
                        s.weights[k] = held[k];
                }
                s.weight_sum = g_full ? g_sum : S(0);
                s.count = g_count;
                s.full = g_full ? 1 : 0;
                return;
        }
        float out[HELD_OUT];
        int i = 0;
        int ai = 0;
        int bi = 0;
        while (ai < a_count && bi < g_count)
        {
                out[i++] = (s.weights[ai] < held[bi]) ? s.weights[ai++] : held[bi++];
        }
        while (ai < a_count)
        {
                out[i++] = s.weights[ai++];
        }
        while (bi < g_count)
        {
                out[i++] = held[bi++];
        }
        for (int k = 0; k < i; ++k)
        {
                s.weights[k] = out[k];
        }
        s.count = i;
        s.full = 0;
}

// ---------------------------------------------------------------------------
// accumulation kernel: one thread per receiving pixel

template <int N>
struct Screen final
{
        int size[N - 1];
        // a slab of the screen: the receiving pixels are [first, first +
        // pixel_count) in global index, and the sample arrays hold the pixels
        // from source_first on (0 and 0 for the whole screen)
        long long first = 0;
        long long source_first = 0;
};

// Merge one pass's samples of the 3^(n-1) neighbours into receiving pixel t
// (global index).
template <int N, typename T, int C, typename S>
NBPT_HD void accumulate_pixel(
        const Screen<N>& screen,
        const long long t,
        const int spp,
        const T* __restrict__ points,
        const float* __restrict__ colors,
        const float* __restrict__ lum,
        const unsigned char* __restrict__ valid,
        const T alpha,
        const T exp_radius,
        PixelState<C, S>& st)
{
        int tc[N - 1];
        {
                long long rest = t;
#pragma unroll
                for (int d = 0; d < N - 1; ++d)
                {
                        tc[d] = static_cast<int>(rest % screen.size[d]);
                        rest /= screen.size[d];
                }
        }

        float w[MAX_GROUP];
        float contribution[MAX_GROUP];
        int color_order[MAX_GROUP];
        float background[MAX_GROUP];

        int neighbours = 1;
#pragma unroll
        for (int d = 0; d < N - 1; ++d)
        {
                neighbours *= 3;
        }
        // sources in increasing pixel index: the last screen axis outermost
        for (int nb = 0; nb < neighbours; ++nb)
        {
                int pc[N - 1];
                bool inside = true;
                {
                        int rest = nb;
#pragma unroll
                        for (int d = 0; d < N - 1; ++d)
                        {
                                pc[d] = tc[d] + (rest % 3) - 1;
                                rest /= 3;
                                inside = inside && pc[d] >= 0 && pc[d] < screen.size[d];
                        }
                }
                if (!inside)
                {
                        continue;
                }
                long long p = 0;
#pragma unroll
                for (int d = N - 2; d >= 0; --d)
                {
                        p = p * screen.size[d] + pc[d];
                }

                // weights (pixel_filter.h:57-69, gaussian.h:66-77) and the
                // selection of colour and background samples (com/select.h:28-47)
                int nc = 0;
                int nbg = 0;
                for (int j = 0; j < spp; ++j)
                {
                        const long long sidx = (p - screen.source_first) * spp + j;
                        const T x0 = (static_cast<T>(tc[0] - pc[0]) + T(0.5)) - points[sidx * (N - 1)];
                        T weight = max_value(T(0), exp(alpha * x0 * x0) - exp_radius);
#pragma unroll
                        for (int d = 1; d < N - 1; ++d)
                        {
                                const T x = (static_cast<T>(tc[d] - pc[d]) + T(0.5)) - points[sidx * (N - 1) + d];
                                weight *= max_value(T(0), exp(alpha * x * x) - exp_radius);
                        }
                        if (!(weight > 0))
                        {
                                continue;
                        }
                        const float wf = static_cast<float>(weight);
                        if (valid[sidx])
                        {
                                w[j] = wf;
                                contribution[j] = wf * lum[sidx];
                                color_order[nc++] = j;
                        }
                        else
                        {
                                background[nbg++] = wf;
                        }
                }

                if (nc > 0)
                {
                        order_group(color_order, nc, [&](const int i) { return contribution[i]; });
                        const ColorGroup<C> g{colors + (p - screen.source_first) * spp * C, w, contribution, color_order, nc, C, 1, 0};
                        S g_sum[C];
                        S g_wsum = 0;
#pragma unroll 8
                        for (int c = 0; c < C; ++c)
                        {
                                g_sum[c] = 0;
                        }
                        const bool g_full = nc > HELD_OUT;
                        if (g_full)
                        {
                                // create_with_sum (samples/com/create.h:28-55)
                                for (int k = HELD_OUT / 2; k < nc - HELD_OUT / 2; ++k)
                                {
#pragma unroll 8
                                        for (int c = 0; c < C; ++c)
                                        {
                                                g_sum[c] += g.color(k, c);
                                        }
                                        g_wsum += w[color_order[k]];
                                }
                        }
                        merge_color_group(st.color, g, g_sum, g_wsum, g_full);
                }
                if (nbg > 0)
                {
                        // background samples are ordered by value
                        int order[MAX_GROUP];
                        for (int k = 0; k < nbg; ++k)
                        {
                                order[k] = k;
                        }
                        order_group(order, nbg, [&](const int i) { return background[i]; });
                        float sorted[MAX_GROUP];
                        for (int k = 0; k < nbg; ++k)
                        {
                                sorted[k] = background[order[k]];
                        }
                        merge_background_group(st.background, sorted, nbg);
                }
        }
}

// accumulation kernel: one thread per receiving pixel, no atomics
template <int N, typename T, int C, typename S>
__global__ void __launch_bounds__(128) accumulate_kernel(
        const Screen<N> screen,
        const long long pixel_count,
        const int spp,
        const T* __restrict__ points,
        const float* __restrict__ colors,
        const float* __restrict__ lum,
        const unsigned char* __restrict__ valid,
        const T alpha,
        const T exp_radius,
        PixelState<C, S>* __restrict__ state)
{
        const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        if (t >= pixel_count)
        {
                return;
        }
        PixelState<C, S> st = state[t];
        accumulate_pixel<N, T, C, S>(screen, screen.first + t, spp, points, colors, lum, valid, alpha, exp_radius, st);
        state[t] = st;
}

// Spectral colours: one warp per receiving pixel.  The lanes compute the
// filter weights of a source's samples in parallel; lane 0 selects and
// orders the group (the scalar part, in shared memory); then every lane runs
// the same merge on the same scalars for its own channels (lane, lane + 32,
// ...), so the merge decisions are the single-thread kernel's and each
// channel's sums are formed in the same order.
template <int N, typename T, int C, typename S>
__global__ void __launch_bounds__(128) accumulate_warp_kernel(
        const Screen<N> screen,
        const long long pixel_count,
        const int spp,
        const T* __restrict__ points,
        const float* __restrict__ colors,
        const float* __restrict__ lum,
        const unsigned char* __restrict__ valid,
        const T alpha,
        const T exp_radius,
        PixelState<C, S>* __restrict__ state)
{
        static_assert(C % 32 == 0);
        constexpr int K = C / 32;
        constexpr int WARPS = 4;
        __shared__ float s_weight[WARPS][MAX_GROUP];
        __shared__ float s_contribution[WARPS][MAX_GROUP];
        __shared__ int s_kind[WARPS][MAX_GROUP]; // 0 none, 1 colour, 2 background
        __shared__ int s_order[WARPS][MAX_GROUP];
        __shared__ float s_background[WARPS][MAX_GROUP];
        __shared__ float s_sorted[WARPS][MAX_GROUP];
        __shared__ int s_counts[WARPS][2];

        const int warp = threadIdx.x / 32;
        const int lane = threadIdx.x & 31;
        const long long t = blockIdx.x * static_cast<long long>(WARPS) + warp;
        if (t >= pixel_count)
        {
                return; // the whole warp
        }
        float* const w = s_weight[warp];
        float* const contribution = s_contribution[warp];
        int* const kind = s_kind[warp];
        int* const order = s_order[warp];
        float* const background = s_background[warp];
        float* const sorted = s_sorted[warp];

        // this lane's channels of the pixel state, and its scalars
        PixelState<C, S>& global = state[t];
        ColorSet<K, S> cs;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                cs.color_sum[k] = global.color.color_sum[lane + 32 * k];
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        cs.colors[j][k] = global.color.colors[j][lane + 32 * k];
                }
        }
        cs.weight_sum = global.color.weight_sum;
#pragma unroll
        for (int j = 0; j < HELD_OUT; ++j)
        {
                cs.weights[j] = global.color.weights[j];
                cs.contributions[j] = global.color.contributions[j];
        }
        cs.count = global.color.count;
        cs.full = global.color.full;
        BackgroundSet<S> bs = global.background;

        int tc[N - 1];
        {
                long long rest = screen.first + t;
#pragma unroll
                for (int d = 0; d < N - 1; ++d)
                {
                        tc[d] = static_cast<int>(rest % screen.size[d]);
                        rest /= screen.size[d];
                }
        }
        int neighbours = 1;
#pragma unroll
        for (int d = 0; d < N - 1; ++d)
        {
                neighbours *= 3;
        }
        for (int nb = 0; nb < neighbours; ++nb)
        {
                int pc[N - 1];
                bool inside = true;
                {
                        int rest = nb;
#pragma unroll
                        for (int d = 0; d < N - 1; ++d)
                        {
                                pc[d] = tc[d] + (rest % 3) - 1;
                                rest /= 3;
                                inside = inside && pc[d] >= 0 && pc[d] < screen.size[d];
                        }
                }
                if (!inside)
                {
                        continue;
                }
                long long p = 0;
#pragma unroll
                for (int d = N - 2; d >= 0; --d)
                {
                        p = p * screen.size[d] + pc[d];
                }
                // weights and selection (pixel_filter.h:57-69, com/select.h:28-47)
                for (int j = lane; j < spp; j += 32)
                {
                        const long long sidx = (p - screen.source_first) * spp + j;
                        const T x0 = (static_cast<T>(tc[0] - pc[0]) + T(0.5)) - points[sidx * (N - 1)];
                        T weight = max_value(T(0), exp(alpha * x0 * x0) - exp_radius);
#pragma unroll
                        for (int d = 1; d < N - 1; ++d)
                        {
                                const T x = (static_cast<T>(tc[d] - pc[d]) + T(0.5)) - points[sidx * (N - 1) + d];
                                weight *= max_value(T(0), exp(alpha * x * x) - exp_radius);
                        }
                        int k = 0;
                        if (weight > 0)
                        {
                                const float wf = static_cast<float>(weight);
                                w[j] = wf;
                                if (valid[sidx])
                                {
                                        contribution[j] = wf * lum[sidx];
                                        k = 1;
                                }
                                else
                                {
                                        k = 2;
                                }
                        }
                        kind[j] = k;
                }
                __syncwarp();
                if (lane == 0)
                {
                        int nc = 0;
                        int nbg = 0;
                        for (int j = 0; j < spp; ++j)
                        {
                                if (kind[j] == 1)
                                {
                                        order[nc++] = j;
                                }
                                else if (kind[j] == 2)
                                {
                                        background[nbg++] = w[j];
                                }
                        }
                        order_group(order, nc, [&](const int i) { return contribution[i]; });
                        if (nbg > 1)
                        {
                                // background samples are ordered by value; reuse
                                // `kind` as the index array of the ordering
                                int* const index = kind;
                                for (int j = 0; j < nbg; ++j)
                                {
                                        index[j] = j;
                                }
                                order_group(index, nbg, [&](const int i) { return background[i]; });
                                for (int j = 0; j < nbg; ++j)
                                {
                                        sorted[j] = background[index[j]];
                                }
                        }
                        else if (nbg == 1)
                        {
                                sorted[0] = background[0];
                        }
                        s_counts[warp][0] = nc;
                        s_counts[warp][1] = nbg;
                }
                __syncwarp();
                const int nc = s_counts[warp][0];
                const int nbg = s_counts[warp][1];
                if (nc > 0)
                {
                        const ColorGroup<K> g{colors + (p - screen.source_first) * spp * C, w, contribution, order, nc, C, 32, lane};
                        S g_sum[K];
                        S g_wsum = 0;
#pragma unroll
                        for (int k = 0; k < K; ++k)
                        {
                                g_sum[k] = 0;
                        }
                        const bool g_full = nc > HELD_OUT;
                        if (g_full)
                        {
                                for (int k = HELD_OUT / 2; k < nc - HELD_OUT / 2; ++k)
                                {
#pragma unroll
                                        for (int c = 0; c < K; ++c)
                                        {
                                                g_sum[c] += g.color(k, c);
                                        }
                                        g_wsum += w[order[k]];
                                }
                        }
                        merge_color_group(cs, g, g_sum, g_wsum, g_full);
                }
                if (nbg > 0)
                {
                        merge_background_group(bs, sorted, nbg);
                }
                __syncwarp();
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                global.color.color_sum[lane + 32 * k] = cs.color_sum[k];
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        global.color.colors[j][lane + 32 * k] = cs.colors[j][k];
                }
        }
        if (lane == 0)
        {
                global.color.weight_sum = cs.weight_sum;
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        global.color.weights[j] = cs.weights[j];
                        global.color.contributions[j] = cs.contributions[j];
                }
                global.color.count = cs.count;
                global.color.full = cs.full;
                global.background = bs;
        }
}

// The same merge with the scalar work of the neighbours done side by side,
// for up to 32 samples per pixel: one warp per receiving pixel; first the
// weights of every neighbour's samples (lanes over samples), then every
// neighbour's group ordered on its own lane, then the groups merged in
// increasing pixel index with the channels across the lanes, as
// accumulate_warp_kernel merges them.
inline constexpr int SMALL_GROUP = 32;

template <int N, typename T, int C, typename S>
__global__ void __launch_bounds__(128) accumulate_warp_small_kernel(
        const Screen<N> screen,
        const long long pixel_count,
        const int spp,
        const T* __restrict__ points,
        const float* __restrict__ colors,
        const float* __restrict__ lum,
        const unsigned char* __restrict__ valid,
        const T alpha,
        const T exp_radius,
        PixelState<C, S>* __restrict__ state)
{
        static_assert(C % 32 == 0);
        constexpr int K = C / 32;
        constexpr int WARPS = 4;
        static_assert(N <= 4, "the shared-memory tables hold 3^(N-1) <= 27 neighbours");
        constexpr int NB = N == 3 ? 9 : 27;
        __shared__ float s_weight[WARPS][NB][SMALL_GROUP];
        __shared__ float s_contribution[WARPS][NB][SMALL_GROUP];
        __shared__ unsigned char s_kind[WARPS][NB][SMALL_GROUP]; // 0 none, 1 colour, 2 background
        __shared__ unsigned char s_order[WARPS][NB][SMALL_GROUP];
        __shared__ unsigned char s_order_bg[WARPS][NB][SMALL_GROUP];
        __shared__ int s_counts[WARPS][NB][2];
        __shared__ int s_order_int[WARPS][SMALL_GROUP];
        __shared__ float s_sorted[WARPS][SMALL_GROUP];

        const int warp = threadIdx.x / 32;
        const int lane = threadIdx.x & 31;
        const long long t = blockIdx.x * static_cast<long long>(WARPS) + warp;
        if (t >= pixel_count)
        {
                return; // the whole warp
        }

        int tc[N - 1];
        {
                long long rest = screen.first + t;
#pragma unroll
                for (int d = 0; d < N - 1; ++d)
                {
                        tc[d] = static_cast<int>(rest % screen.size[d]);
                        rest /= screen.size[d];
                }
        }
        // neighbour nb's pixel, or -1 outside the screen
        const auto neighbour = [&](const int nb, int* pc) -> long long
        {
                int rest = nb;
                bool inside = true;
#pragma unroll
                for (int d = 0; d < N - 1; ++d)
                {
                        pc[d] = tc[d] + (rest % 3) - 1;
                        rest /= 3;
                        inside = inside && pc[d] >= 0 && pc[d] < screen.size[d];
                }
                if (!inside)
                {
                        return -1;
                }
                long long p = 0;
#pragma unroll
                for (int d = N - 2; d >= 0; --d)
                {
                        p = p * screen.size[d] + pc[d];
                }
                return p;
        };

        // weights and kinds (pixel_filter.h:57-69), lanes over the samples
        for (int nb = 0; nb < NB; ++nb)
        {
                int pc[N - 1];
                const long long p = neighbour(nb, pc);
                if (p < 0 || lane >= spp)
                {
                        continue;
                }
                const int j = lane;
                const long long sidx = (p - screen.source_first) * spp + j;
                const T x0 = (static_cast<T>(tc[0] - pc[0]) + T(0.5)) - points[sidx * (N - 1)];
                T weight = max_value(T(0), exp(alpha * x0 * x0) - exp_radius);
#pragma unroll
                for (int d = 1; d < N - 1; ++d)
                {
                        const T x = (static_cast<T>(tc[d] - pc[d]) + T(0.5)) - points[sidx * (N - 1) + d];
                        weight *= max_value(T(0), exp(alpha * x * x) - exp_radius);
                }
                unsigned char k = 0;
                if (weight > 0)
                {
                        const float wf = static_cast<float>(weight);
                        s_weight[warp][nb][j] = wf;
                        if (valid[sidx])
                        {
                                s_contribution[warp][nb][j] = wf * lum[sidx];
                                k = 1;
                        }
                        else
                        {
                                k = 2;
                        }
                }
                s_kind[warp][nb][j] = k;
        }
        __syncwarp();

        // every neighbour's group ordered on its own lane (com/select.h:28-47,
        // samples/com/sort.h:26-46)
        if (lane < NB)
        {
                const int nb = lane;
                int pc[N - 1];
                const long long p = neighbour(nb, pc);
                int nc = 0;
                int nbg = 0;
                if (p >= 0)
                {
                        int order[SMALL_GROUP];
                        int order_bg[SMALL_GROUP];
                        for (int j = 0; j < spp; ++j)
                        {
                                const unsigned char k = s_kind[warp][nb][j];
                                if (k == 1)
                                {
                                        order[nc++] = j;
                                }
                                else if (k == 2)
                                {
                                        order_bg[nbg++] = j;
                                }
                        }
                        const float* const contribution = s_contribution[warp][nb];
                        const float* const w = s_weight[warp][nb];
                        order_group(order, nc, [&](const int i) { return contribution[i]; });
                        order_group(order_bg, nbg, [&](const int i) { return w[i]; });
                        for (int k = 0; k < nc; ++k)
                        {
                                s_order[warp][nb][k] = static_cast<unsigned char>(order[k]);
                        }
                        for (int k = 0; k < nbg; ++k)
                        {
                                s_order_bg[warp][nb][k] = static_cast<unsigned char>(order_bg[k]);
                        }
                }
                s_counts[warp][nb][0] = nc;
                s_counts[warp][nb][1] = nbg;
        }
        __syncwarp();

        // this lane's channels of the pixel state, and its scalars
        PixelState<C, S>& global = state[t];
        ColorSet<K, S> cs;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                cs.color_sum[k] = global.color.color_sum[lane + 32 * k];
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        cs.colors[j][k] = global.color.colors[j][lane + 32 * k];
                }
        }
        cs.weight_sum = global.color.weight_sum;
#pragma unroll
        for (int j = 0; j < HELD_OUT; ++j)
        {
                cs.weights[j] = global.color.weights[j];
                cs.contributions[j] = global.color.contributions[j];
        }
        cs.count = global.color.count;
        cs.full = global.color.full;
        BackgroundSet<S> bs = global.background;

        int* const order = s_order_int[warp];
        float* const sorted = s_sorted[warp];
        for (int nb = 0; nb < NB; ++nb)
        {
                const int nc = s_counts[warp][nb][0];
                const int nbg = s_counts[warp][nb][1];
                if (nc == 0 && nbg == 0)
                {
                        continue;
                }
                int pc[N - 1];
                const long long p = neighbour(nb, pc);
                const float* const w = s_weight[warp][nb];
                if (lane < nc)
                {
                        order[lane] = s_order[warp][nb][lane];
                }
                if (lane < nbg)
                {
                        sorted[lane] = w[s_order_bg[warp][nb][lane]];
                }
                __syncwarp();
                if (nc > 0)
                {
                        const ColorGroup<K> g{colors + (p - screen.source_first) * spp * C, w, s_contribution[warp][nb], order, nc, C, 32, lane};
                        S g_sum[K];
                        S g_wsum = 0;
#pragma unroll
                        for (int k = 0; k < K; ++k)
                        {
                                g_sum[k] = 0;
                        }
                        const bool g_full = nc > HELD_OUT;
                        if (g_full)
                        {
                                for (int k = HELD_OUT / 2; k < nc - HELD_OUT / 2; ++k)
                                {
#pragma unroll
                                        for (int c = 0; c < K; ++c)
                                        {
                                                g_sum[c] += g.color(k, c);
                                        }
                                        g_wsum += w[order[k]];
                                }
                        }
                        merge_color_group(cs, g, g_sum, g_wsum, g_full);
                }
                if (nbg > 0)
                {
                        merge_background_group(bs, sorted, nbg);
                }
                __syncwarp();
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                global.color.color_sum[lane + 32 * k] = cs.color_sum[k];
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        global.color.colors[j][lane + 32 * k] = cs.colors[j][k];
                }
        }
        if (lane == 0)
        {
                global.color.weight_sum = cs.weight_sum;
#pragma unroll
                for (int j = 0; j < HELD_OUT; ++j)
                {
                        global.color.weights[j] = cs.weights[j];
                        global.color.contributions[j] = cs.contributions[j];
                }
                global.color.count = cs.count;
                global.color.full = cs.full;
                global.background = bs;
        }
}

// ---------------------------------------------------------------------------
// image resolve: merge_color / merge_color_alpha (samples/merge_color.cpp:45-177)
// and the RGB of the colour (src/color/color.h rgb32).  The background is
// black: its colour and contribution are 0.

template <int C, typename S>
struct Resolved final
{
        bool has;
        S color[C];
        S color_weight;
        S background_weight;
};

template <int C, typename S>
NBPT_HD Resolved<C, S> resolve_pixel(const PixelState<C, S>& st)
{
        Resolved<C, S> res;
        res.has = false;
        const ColorSet<C, S>& a = st.color;
        const BackgroundSet<S>& b = st.background;
        const int a_size = a.full ? HELD_OUT : a.count;
        const int b_size = b.full ? HELD_OUT : b.count;
        if (a_size + b_size <= HELD_OUT)
        {
                if (a_size == 0 || b_size != 0 || !a.full)
                {
                        return res;
                }
                res.has = true;
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        res.color[c] = a.color_sum[c];
                }
                res.color_weight = a.weight_sum;
                res.background_weight = 0;
                return res;
        }
        res.has = true;
#pragma unroll 8
        for (int c = 0; c < C; ++c)
        {
                res.color[c] = a.full ? a.color_sum[c] : S(0);
        }
        res.color_weight = a.full ? a.weight_sum : S(0);
        res.background_weight = b.full ? b.weight_sum : S(0);

        const auto a_key = [&](const int i)
        {
                return a.contributions[i];
        };
        const auto b_key = [&](const int i)
        {
                return b.weights[i] * 0.0f;
        };
        const auto sum_a = [&](const int i)
        {
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        res.color[c] += a.colors[i][c];
                }
                res.color_weight += a.weights[i];
        };
        const auto sum_b = [&](const int i)
        {
                res.background_weight += b.weights[i];
        };
        if (a_size == HELD_OUT && b_size == HELD_OUT)
        {
                int ai = 0;
                int bi = 0;
                for (int i = 0; i < HELD_OUT / 2; ++i)
                {
                        if (a_key(ai) < b_key(bi))
                        {
                                ++ai;
                        }
                        else
                        {
                                ++bi;
                        }
                }
                while (ai < HELD_OUT / 2)
                {
                        sum_a(ai++);
                }
                while (bi < HELD_OUT / 2)
                {
                        sum_b(bi++);
                }
                ai = HELD_OUT - 1;
                bi = HELD_OUT - 1;
                for (int i = HELD_OUT - 1; i >= HELD_OUT / 2; --i)
                {
                        if (a_key(ai) > b_key(bi))
                        {
                                --ai;
                        }
                        else
                        {
                                --bi;
                        }
                }
                while (ai >= HELD_OUT / 2)
                {
                        sum_a(ai--);
                }
                while (bi >= HELD_OUT / 2)
                {
                        sum_b(bi--);
                }
                return res;
        }
        int ai = 0;
        int bi = 0;
        int i = 0;
        while (i < HELD_OUT / 2 && ai < a_size && bi < b_size)
        {
                if (a_key(ai) < b_key(bi))
                {
                        ++ai;
                }
                else
                {
                        ++bi;
                }
                ++i;
        }
        while (i < HELD_OUT / 2 && ai < a_size)
        {
                ++ai;
                ++i;
        }
        while (i < HELD_OUT / 2 && bi < b_size)
        {
                ++bi;
                ++i;
        }
        const int a_low = ai;
        const int b_low = bi;
        int aj = a_size - 1;
        int bj = b_size - 1;
        int j = HELD_OUT - 1;
        while (j >= HELD_OUT / 2 && aj >= a_low && bj >= b_low)
        {
                if (a_key(aj) > b_key(bj))
                {
                        --aj;
                }
                else
                {
                        --bj;
                }
                --j;
        }
        while (j >= HELD_OUT / 2 && aj >= a_low)
        {
                --aj;
                --j;
        }
        while (j >= HELD_OUT / 2 && bj >= b_low)
        {
                --bj;
                --j;
        }
        for (int k = a_low; k <= aj; ++k)
        {
                sum_a(k);
        }
        for (int k = b_low; k <= bj; ++k)
        {
                sum_b(k);
        }
        return res;
}

// The pixel's RGB and premultiplied RGBA (pixel.h:51-88, color.h rgb32); with
// double sums the division by the weight is in double and the colour is then
// rounded to float.
template <int C, typename S>
NBPT_HD void resolve_rgb(const PixelState<C, S>& state, const float* xyz, float* rgb, float* rgba)
{
        const Resolved<C, S> r = resolve_pixel(state);
        float out[3] = {0.0f, 0.0f, 0.0f};
        float out_a[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (r.has)
        {
                const S sum = r.color_weight + r.background_weight;
                float color[C];
#pragma unroll 8
                for (int c = 0; c < C; ++c)
                {
                        color[c] = static_cast<float>(r.color[c] / sum);
                }
                float c_rgb[3];
                if constexpr (C == 3)
                {
                        c_rgb[0] = max_value(0.0f, color[0]);
                        c_rgb[1] = max_value(0.0f, color[1]);
                        c_rgb[2] = max_value(0.0f, color[2]);
                }
                else
                {
                        float v[3];
                        for (int k = 0; k < 3; ++k)
                        {
                                const float* f = xyz + k * 64;
                                float s = max_value(0.0f, color[0]) * f[0];
                                for (int c = 1; c < C; ++c)
                                {
                                        s += max_value(0.0f, color[c]) * f[c];
                                }
                                v[k] = s;
                        }
                        c_rgb[0] = max_value(0.0f, 3.2406255f * v[0] + -1.5372080f * v[1] + -0.4986286f * v[2]);
                        c_rgb[1] = max_value(0.0f, -0.9689307f * v[0] + 1.8757561f * v[1] + 0.0415175f * v[2]);
                        c_rgb[2] = max_value(0.0f, 0.0557101f * v[0] + -0.2040211f * v[1] + 1.0569959f * v[2]);
                }
                const bool background_only =
                        !(r.color_weight == sum || (r.color_weight / sum) == 1) &&
                        (r.background_weight == sum || (r.background_weight / sum) == 1);
                if (!background_only)
                {
                        out[0] = c_rgb[0];
                        out[1] = c_rgb[1];
                        out[2] = c_rgb[2];
                }
                if (r.color_weight != 0)
                {
                        out_a[0] = c_rgb[0];
                        out_a[1] = c_rgb[1];
                        out_a[2] = c_rgb[2];
                        out_a[3] = static_cast<float>(r.color_weight / sum);
                }
        }
        rgb[0] = out[0];
        rgb[1] = out[1];
        rgb[2] = out[2];
        if (rgba)
        {
                rgba[0] = out_a[0];
                rgba[1] = out_a[1];
                rgba[2] = out_a[2];
                rgba[3] = out_a[3];
        }
}

template <int C, typename S>
__global__ void resolve_kernel(
        const long long pixel_count,
        const PixelState<C, S>* __restrict__ state,
        const float* __restrict__ xyz, // [3][64] colour matching functions (spectrum only)
        float* __restrict__ rgb,
        float* __restrict__ rgba)
{
        const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        if (t >= pixel_count)
        {
                return;
        }
        resolve_rgb<C, S>(state[t], xyz, rgb + t * 3, rgba ? rgba + t * 4 : nullptr);
}
} // namespace nbpt
