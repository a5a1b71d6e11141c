// CUDA kernels of the painter: facet setup, stratified sub-pixel samples,
// the path kernel, the filtered trimmed accumulation and image resolve, and
// ray-query and per-function kernels used for verification.
#pragma once

#include "bpt.cuh"
#include "core.cuh"
#include "geometry.cuh"
#include "scene.cuh"
#include "shading.cuh"
#include "tape.cuh"

#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>
#include <cstdint>
#include <type_traits>

namespace nbpt
{
namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// facet setup at scene load, in double precision (hyperplane_simplex.h:82-111,
// mesh/facet.cpp:83-125), stored in the path precision T.

template <int N, typename T>
__global__ void facet_setup_kernel(
        const double* __restrict__ vertices,
        const double* __restrict__ normals, // nullptr: no vertex normals
        const unsigned char* __restrict__ flat, // nullptr, or 1 for a facet without vertex normals
        const int* __restrict__ facet_vertices,
        const int* __restrict__ facet_materials,
        const long long count,
        Facet<N, T>* __restrict__ out,
        int* __restrict__ error)
{
        const long long f = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        if (f >= count)
        {
                return;
        }
        Vec<N, double> v[N];
        int idx[N];
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                idx[k] = facet_vertices[f * N + k];
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        v[k][d] = vertices[static_cast<long long>(idx[k]) * N + d];
                }
        }
        Simplex<N, double> s;
        if (!s.set(v))
        {
                atomicMax(error, 1);
                return;
        }
        int normal_type = static_cast<int>(NormalType::NONE);
        unsigned reverse_mask = 0;
        if (normals && !(flat && flat[f]))
        {
                double dots[N];
                bool unidirectional = true;
                bool positive = true;
                bool negative = true;
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                        Vec<N, double> n;
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                n[d] = normals[static_cast<long long>(idx[k]) * N + d];
                        }
                        dots[k] = dot(n, s.plane.n);
                        const double a = abs_value(dots[k]);
                        if (!(dots[k] - dots[k] == 0 && a >= 0.7))
                        {
                                unidirectional = false;
                        }
                        positive = positive && dots[k] > 0;
                        negative = negative && dots[k] < 0;
                }
                if (unidirectional)
                {
                        if (positive)
                        {
                                normal_type = static_cast<int>(NormalType::USE);
                        }
                        else if (negative)
                        {
                                normal_type = static_cast<int>(NormalType::USE);
                                s.plane.n = -s.plane.n;
                                s.plane.d = -s.plane.d;
                        }
                        else
                        {
                                normal_type = static_cast<int>(NormalType::REVERSE);
#pragma unroll
                                for (int k = 0; k < N; ++k)
                                {
                                        if (dots[k] < 0)
                                        {
                                                reverse_mask |= 1u << k;
                                        }
                                }
                        }
                }
        }
        Facet<N, T> r;
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                r.simplex.plane.n[d] = static_cast<T>(s.plane.n[d]);
        }
        r.simplex.plane.d = static_cast<T>(s.plane.d);
#pragma unroll
        for (int i = 0; i < N - 1; ++i)
        {
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        r.simplex.planes[i].n[d] = static_cast<T>(s.planes[i].n[d]);
                }
                r.simplex.planes[i].d = static_cast<T>(s.planes[i].d);
        }
        r.material = facet_materials[f];
        r.normal_type = normal_type;
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
                r.normals[k] = idx[k];
        }
        r.reverse_mask = reverse_mask;
        out[f] = r;
}

// ---------------------------------------------------------------------------
// stratified jittered sub-pixel points (src/sampling/sj_sampler.h:51-205),
// one thread per pixel, from the pixel's stream seed_seq{seed, pass, p, 0}.

template <int M, typename T>
__global__ void sj_points_kernel(
        const long long begin,
        const long long end,
        const std::uint32_t seed,
        const std::uint32_t pass,
        const int k, // strata per dimension
        const T* __restrict__ offsets,
        T* __restrict__ points)
{
        const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        if (i >= end - begin)
        {
                return;
        }
        const long long p = begin + i;
        const std::uint32_t words[4] = {seed, pass, static_cast<std::uint32_t>(p), 0u};
        Pcg g = seed_seq_pcg(words, 4);
        int count = 1;
#pragma unroll
        for (int d = 0; d < M; ++d)
        {
                count *= k;
        }
        T* const out = points + i * count * M;
        for (int s = 0; s < count; ++s)
        {
                int rest = s;
#pragma unroll
                for (int d = 0; d < M; ++d)
                {
                        const int idx = rest % k;
                        rest /= k;
                        const T a = offsets[idx];
                        const T b = offsets[idx + 1];
                        T v;
                        do
                        {
                                v = uniform<T>(g, a, b);
                        } while (!(v < b));
                        out[s * M + d] = v;
                }
        }
}

// Minimum resident blocks of 128 threads per SM asked of the compiler for
// the path kernels, which caps their registers (65536 / (128 * blocks)), per
// dimension and precision, from launch-bound sweeps of the mixed-scene
// batch's jobs on a B200 (one pass each, best of three):
//   float: 16 blocks (32 registers) in 3-, 4- and 5-space; 12 and 8 blocks
//          were 1-8 % slower;
//   double: 8 blocks (64 registers) in 4- and 5-space, 7-8 % faster than 16;
//          12 blocks in 3-space, 5 % faster than 16.
// NBPT_PATHS_MIN_BLOCKS, when defined, sets every kernel's (for sweeps).
template <int N, typename T>
struct PathsMinBlocks final
{
#ifdef NBPT_PATHS_MIN_BLOCKS
        static constexpr int value = NBPT_PATHS_MIN_BLOCKS;
#else
        static constexpr int value = std::is_same_v<T, double> ? (N == 3 ? 12 : 8) : 16;
#endif
};

// ---------------------------------------------------------------------------
// Paths: one per pixel sample, with the random stream seed_seq{seed, pass,
// p, i + 1}.  A chunk of pixels runs through four kernels:
//   paths_walk_kernel     one lane per path, one bounce per iteration: the
//                         camera and light subpaths traced with colour
//                         channel 0 (tape.cuh), their
//                         vertices kept in global memory, the bounce records
//                         on the path's tape, and one task queued per
//                         strategy with s != 1;
//   paths_light_kernel    one thread per path: the light samples of the
//                         s = 1 strategies in t order, since each draws from
//                         the path's stream where the light subpath left it;
//                         the usable ones are kept and their strategies
//                         queued;
//   paths_connect_kernel  one thread per queued strategy: its contribution
//                         factors written to the strategy's tape slot;
//   paths_replay_kernel   the colours of all channels from the tapes.
// Strategies of one path are independent apart from that random stream, so
// evaluating them on separate threads changes no result; the replay sums
// them in the reference's order.

struct PathStats final
{
        unsigned long long queries;
        unsigned long long nodes;
        unsigned long long facets;
        unsigned long long shapes;
        unsigned long long overflows; // ray queries ended on a full traversal stack (an error)
        unsigned long long nonfinite; // samples whose colour has a NaN or infinite channel
};

template <int C>
NBPT_HD float luminance(const Color<C>& c, const float* y)
{
        if constexpr (C == 3)
        {
                const float r = max_value(0.0f, c.c[0]);
                const float g = max_value(0.0f, c.c[1]);
                const float b = max_value(0.0f, c.c[2]);
                return 0.2126f * r + 0.7152f * g + 0.0722f * b;
        }
        else
        {
                float s = max_value(0.0f, c.c[0]) * y[0];
#pragma unroll 8
                for (int i = 1; i < C; ++i)
                {
                        s += max_value(0.0f, c.c[i]) * y[i];
                }
                return s;
        }
}

// Warp-aggregated statistics; every thread of the block must call it.
__device__ inline void add_counters(const QueryCounters& counters, PathStats* const stats)
{
        unsigned long long a = counters.queries;
        unsigned long long b = counters.nodes;
        unsigned long long c = counters.facets;
        unsigned long long d = counters.shapes;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
                a += __shfl_down_sync(0xffffffffu, a, o);
                b += __shfl_down_sync(0xffffffffu, b, o);
                c += __shfl_down_sync(0xffffffffu, c, o);
                d += __shfl_down_sync(0xffffffffu, d, o);
        }
        if ((threadIdx.x & 31) == 0 && (a | b | c | d) != 0)
        {
                atomicAdd(&stats->queries, a);
                atomicAdd(&stats->nodes, b);
                atomicAdd(&stats->facets, c);
                atomicAdd(&stats->shapes, d);
        }
        if (counters.overflows != 0)
        {
                atomicAdd(&stats->overflows, static_cast<unsigned long long>(counters.overflows));
        }
}

// A sample colour with a NaN or infinite channel is counted, as the
// reference logs it (src/painter/pixels/pixels.cpp:107-113), and kept.
template <int K>
__device__ inline bool all_finite(const float (&c)[K])
{
        bool ok = true;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                ok = ok && isfinite(c[k]);
        }
        return ok;
}

// The painter's cancel word, written by the host on another stream while a
// pass runs (Painter::cancel); read from L2 on every test.
__device__ inline bool cancelled(const unsigned* const cancel)
{
        return *static_cast<const volatile unsigned*>(cancel) != 0;
}

// A queued strategy: the path's index in its chunk, t and s.
inline constexpr int TASK_PATH_SHIFT = 8;
inline constexpr long long TASK_MAX_PATHS = 1LL << (32 - TASK_PATH_SHIFT);

NBPT_HD constexpr std::uint32_t make_task(const long long path, const int t, const int s)
{
        return (static_cast<std::uint32_t>(path) << TASK_PATH_SHIFT) | (static_cast<std::uint32_t>(t) << 4) |
               static_cast<std::uint32_t>(s);
}

// Queued strategies, one queue per kind so that the warps of the connect
// kernel run one kind of strategy at a time: s = 0 (emission at a camera
// vertex), s = 1 (a resampled light) and s >= 2 (a vertex-vertex connection).
// The queues are regions of one buffer with a counter each.
struct TaskQueues final
{
        enum Kind : int
        {
                CONNECT = 0,
                LIGHT = 1,
                EMITTED = 2
        };
        std::uint32_t* base[3];
        unsigned* count; // [3]

        __device__ std::uint32_t& task(const int kind, const unsigned k) const
        {
                return base[kind][k];
        }
};

// Reserves `n` consecutive slots of a counter for each calling thread with
// one atomic per group of threads that call it together.
__device__ inline unsigned reserve_together(unsigned* const counter, const unsigned n)
{
        const cg::coalesced_group g = cg::coalesced_threads();
        const unsigned before = cg::exclusive_scan(g, n);
        unsigned base = 0;
        if (g.thread_rank() == g.size() - 1)
        {
                const unsigned total = before + n;
                base = total > 0 ? atomicAdd(counter, total) : 0;
        }
        base = g.shfl(base, g.size() - 1);
        return base + before;
}

// Persistent, one bounce per iteration: every lane traces one ray and
// processes its hit (Bpt::walk_step) in each iteration of the loop, whether
// the ray belongs to a camera or a light subpath, so the warp's lanes run the
// intersection and the shading together however their paths' lengths
// differ.  A lane whose camera subpath ends starts its light subpath
// (bpt.cpp:273-289) in the same iteration, and a lane whose path ends
// finishes it and takes the next path from a shared counter until the chunk
// is done.  Each path's random stream, vertices and tape are those of the
// reference's sequential order (camera subpath, light sample, light
// subpath).
template <int N, typename T>
__global__ void __launch_bounds__(128, (PathsMinBlocks<N, T>::value)) paths_walk_kernel(
        const DeviceScene<N, T, 1> scene,
        const long long begin,
        const long long end,
        const int spp,
        const int max_depth,
        const std::uint32_t seed,
        const std::uint32_t pass,
        const T* __restrict__ points,
        PathVertex<N, T, 1>* __restrict__ vertices,
        Pcg* __restrict__ rng,
        std::uint32_t* __restrict__ tape,
        const int words_per_path,
        unsigned char* __restrict__ valid,
        const TaskQueues queues,
        unsigned* __restrict__ next_path,
        PathStats* __restrict__ stats,
        const unsigned* __restrict__ cancel)
{
        using B = Bpt<N, T, 1, true>;
        using S = typename B::Subpaths;
        const long long paths = (end - begin) * spp;
        QueryCounters counters{0, 0, 0, 0};
        const SceneQueries<N, T, 1> q{scene, counters};
        Pcg g{0, 0};
        B bpt{q, scene, g, max_depth, nullptr, nullptr};
        typename B::Walk w;
        Vec<N, T> gn;
        bool from_surface = false;
        long long i = -1; // the lane's path; -1 when it takes the next one
        while (true)
        {
                if (i < 0)
                {
                        if (cancelled(cancel))
                        {
                                break; // the paths not taken keep no tape: the later kernels skip the chunk
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
                        const std::uint32_t words[4] = {seed, pass, static_cast<std::uint32_t>(p),
                                                        static_cast<std::uint32_t>(sample + 1)};
                        g = seed_seq_pcg(words, 4);
                        bpt.camera = vertices + i * 2 * (max_depth + 1);
                        bpt.light = bpt.camera + max_depth + 1;
                        bpt.light_size = 0;
                        bpt.tape.w = tape + i * static_cast<long long>(words_per_path);
                        bpt.tape.n = TAPE_HEADER;
                        w = bpt.camera_start(scene.projector.ray(point));
                        from_surface = false;
                }

                Normals<N, T> normals;
                const Hit<N, T> surface = q.scene_intersect(from_surface ? &gn : nullptr, w.ray, normals);
                if (bpt.walk_step(w, surface, normals))
                {
                        gn = normals.geometric;
                        from_surface = true;
                        continue;
                }
                if (w.camera && bpt.camera_outcome() == S::CONNECT && bpt.light_start(w))
                {
                        from_surface = false;
                        continue;
                }

                // the path's subpaths are done
                const S r = bpt.camera_outcome();
                const bool connect = r == S::CONNECT;
                std::uint32_t* const tw = bpt.tape.w;
                tw[0] = static_cast<std::uint32_t>(bpt.tape.n);
                tw[1] = r != S::BACKGROUND ? 1u : 0u;
                tw[2] = static_cast<std::uint32_t>(connect ? bpt.camera_size : 1);
                tw[3] = static_cast<std::uint32_t>(connect ? bpt.light_size : 0);
                valid[i] = r != S::BACKGROUND ? 1 : 0;
                rng[i] = g;
                if (connect)
                {
                        const int camera_size = bpt.camera_size;
                        const int light_size = bpt.light_size;
                        // s = 0 strategies: one per t
                        unsigned k = reserve_together(&queues.count[TaskQueues::EMITTED], camera_size - 1);
                        for (int t = 2; t <= camera_size; ++t)
                        {
                                queues.task(TaskQueues::EMITTED, k++) = make_task(i, t, 0);
                        }
                        // s >= 2 strategies
                        unsigned task_n = 0;
                        for (int t = 2; t <= camera_size; ++t)
                        {
                                for (int sc = 2; sc <= light_size; ++sc)
                                {
                                        task_n += (t + sc - 2 <= max_depth) ? 1 : 0;
                                }
                        }
                        k = reserve_together(&queues.count[TaskQueues::CONNECT], task_n);
                        for (int t = 2; t <= camera_size; ++t)
                        {
                                for (int sc = 2; sc <= light_size; ++sc)
                                {
                                        if (t + sc - 2 <= max_depth)
                                        {
                                                queues.task(TaskQueues::CONNECT, k++) = make_task(i, t, sc);
                                        }
                                }
                        }
                }
                i = -1;
        }
        add_counters(counters, stats);
}

// The light sample of an s = 1 strategy (Bpt::light_arrival), kept for the
// connect kernel.
template <int N, typename T>
struct Arrival final
{
        Vec<N, T> l;
        T pdf;
        T distance;
        int light;
};

// Persistent: the grid strides over the queued strategies.
template <int N, typename T>
__global__ void __launch_bounds__(128, (PathsMinBlocks<N, T>::value)) paths_connect_kernel(
        const DeviceScene<N, T, 1> scene,
        const int max_depth,
        PathVertex<N, T, 1>* __restrict__ vertices,
        std::uint32_t* __restrict__ tape,
        const int words_per_path,
        const Arrival<N, T>* __restrict__ arrivals,
        const TaskQueues queues,
        PathStats* __restrict__ stats)
{
        QueryCounters counters{0, 0, 0, 0};
        const unsigned n0 = queues.count[0];
        const unsigned n1 = queues.count[1];
        const unsigned total = n0 + n1 + queues.count[2];
        const unsigned stride = gridDim.x * blockDim.x;
        for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride)
        {
                const std::uint32_t task =
                        k < n0 ? queues.base[0][k] : (k < n0 + n1 ? queues.base[1][k - n0] : queues.base[2][k - n0 - n1]);
                const long long i = task >> TASK_PATH_SHIFT;
                const int t = static_cast<int>((task >> 4) & 15u);
                const int sc = static_cast<int>(task & 15u);
                PathVertex<N, T, 1>* const v = vertices + i * 2 * (max_depth + 1);
                std::uint32_t* const w = tape + i * static_cast<long long>(words_per_path);
                Pcg unused{0, 0}; // the random numbers of s = 1 were drawn by paths_light_kernel
                const SceneQueries<N, T, 1> q{scene, counters};
                Bpt<N, T, 1, true> bpt{q, scene, unused, max_depth, v, v + max_depth + 1};
                bpt.camera_size = static_cast<int>(w[2]);
                bpt.light_size = static_cast<int>(w[3]);
                bpt.tape.w = w;
                Color<1> c;
                bool contributes;
                if (sc == 1)
                {
                        const Arrival<N, T>& a = arrivals[i * max_depth + (t - 2)];
                        ArriveSample<N, T, 1> as;
                        as.l = a.l;
                        as.pdf = a.pdf;
                        as.distance = a.distance;
                        as.radiance = scene.lights[a.light].radiance;
                        contributes = bpt.connect_light(t, a.light, as, c);
                }
                else
                {
                        contributes = bpt.connect_strategy(sc, t, c);
                }
                if (!contributes)
                {
                        w[tape_slot_offset(max_depth, t, sc)] = 0;
                }
        }
        add_counters(counters, stats);
}

// One thread per path: the light samples of the s = 1 strategies, drawn in
// t order from the path's stream where the light subpath left it; each
// usable sample is kept and its strategy queued for the connect kernel.
template <int N, typename T>
__global__ void __launch_bounds__(128, (PathsMinBlocks<N, T>::value)) paths_light_kernel(
        const DeviceScene<N, T, 1> scene,
        const long long paths,
        const int max_depth,
        PathVertex<N, T, 1>* __restrict__ vertices,
        const Pcg* __restrict__ rng,
        std::uint32_t* __restrict__ tape,
        const int words_per_path,
        Arrival<N, T>* __restrict__ arrivals,
        const TaskQueues queues,
        const unsigned* __restrict__ cancel)
{
        const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        unsigned queued = 0; // bit t - 2: strategy (1, t) queued
        // a cancelled pass has paths without tapes (see paths_replay_kernel)
        if (i < paths && !cancelled(cancel))
        {
                std::uint32_t* const w = tape + i * static_cast<long long>(words_per_path);
                const int camera_size = static_cast<int>(w[2]);
                const int light_size = static_cast<int>(w[3]);
                if (w[1] != 0 && light_size >= 1)
                {
                        Pcg g = rng[i];
                        PathVertex<N, T, 1>* const v = vertices + i * 2 * (max_depth + 1);
                        QueryCounters counters{0, 0, 0, 0};
                        const SceneQueries<N, T, 1> q{scene, counters};
                        Bpt<N, T, 1, true> bpt{q, scene, g, max_depth, v, v + max_depth + 1};
                        bpt.camera_size = camera_size;
                        bpt.light_size = light_size;
                        for (int t = 2; t <= camera_size; ++t)
                        {
                                if (t - 1 > max_depth)
                                {
                                        continue;
                                }
                                int li = 0;
                                ArriveSample<N, T, 1> as;
                                if (v[t - 1].type == static_cast<int>(VertexType::INFINITE) ||
                                    !bpt.light_arrival(t, li, as))
                                {
                                        w[tape_slot_offset(max_depth, t, 1)] = 0;
                                        continue;
                                }
                                Arrival<N, T>& a = arrivals[i * max_depth + (t - 2)];
                                a.l = as.l;
                                a.pdf = as.pdf;
                                a.distance = as.distance;
                                a.light = li;
                                queued |= 1u << (t - 2);
                        }
                }
        }
        // reserve this warp's task range with one atomic
        const int task_n = __popc(queued);
        const int lane = threadIdx.x & 31;
        int offset = task_n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
                const int x = __shfl_up_sync(0xffffffffu, offset, o);
                offset += lane >= o ? x : 0;
        }
        const int total = __shfl_sync(0xffffffffu, offset, 31);
        unsigned base = 0;
        if (lane == 31 && total > 0)
        {
                base = atomicAdd(&queues.count[TaskQueues::LIGHT], static_cast<unsigned>(total));
        }
        base = __shfl_sync(0xffffffffu, base, 31);
        unsigned k = base + static_cast<unsigned>(offset - task_n);
        while (queued != 0)
        {
                const int b = __ffs(queued) - 1;
                queued &= queued - 1;
                queues.task(TaskQueues::LIGHT, k++) = make_task(i, b + 2, 1);
        }
}

// Colours from the tapes: LANES threads per path (32: one warp per path,
// lane l forms channels l, l + 32, ...; 1: one thread per path).  Every
// channel goes through the float operations of Bpt::walk, light_path and
// connect_strategy in the recorded order, the strategies summed in the
// reference's (t, s) order; then the luminance by the reference's
// left-to-right dot product.
template <int N, typename T, int C, int LANES>
__global__ void __launch_bounds__(128) paths_replay_kernel(
        const Material<T, C>* __restrict__ materials,
        const Light<N, T, C>* __restrict__ lights,
        const float fresnel_a,
        const float fresnel_b,
        const int max_depth,
        const long long paths,
        const std::uint32_t* __restrict__ tape,
        const int words_per_path,
        float* __restrict__ colors,
        float* __restrict__ lum,
        const float* __restrict__ cie_y,
        PathStats* __restrict__ stats,
        const unsigned* __restrict__ cancel)
{
        static_assert(C % LANES == 0 && 32 % LANES == 0);
        constexpr int K = C / LANES;
        // a cancelled pass has paths without tapes: no thread reads them (a
        // walk that stopped early wrote the word before this launch began)
        if (__shfl_sync(0xffffffffu, cancelled(cancel) ? 1 : 0, 0) != 0)
        {
                return;
        }
        const long long i = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) / LANES;
        const int lane = static_cast<int>(threadIdx.x % LANES);
        if (i >= paths)
        {
                return; // all LANES threads of the path
        }
        TapeReader r{tape + i * static_cast<long long>(words_per_path)};
        const int used = static_cast<int>(r.w[0]);
        const bool has = r.w[1] != 0;
        const int camera_size = static_cast<int>(r.w[2]);
        const int light_size = static_cast<int>(r.w[3]);

        float camera_beta[MAX_PATH_VERTICES + 1][K];
        float light_beta[MAX_PATH_VERTICES + 1][K];
        float color[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                camera_beta[1][k] = 1.0f;
                color[k] = 0.0f;
        }
        int camera_vertex = 1;
        int light_vertex = 1;
        r.n = TAPE_HEADER;
        while (r.n < used)
        {
                const TapeRecord kind = static_cast<TapeRecord>(r.get_int());
                if (kind == TapeRecord::CAMERA_BOUNCE)
                {
                        const Material<T, C>& m = materials[r.get_int()];
                        const BrdfTerms t = r.get_terms();
                        const float sk = r.get_float();
#pragma unroll
                        for (int k = 0; k < K; ++k)
                        {
                                const int ch = lane + LANES * k;
                                const float b = brdf_channel(t, m.f0.c[ch], m.rho_ss.c[ch], fresnel_a, fresnel_b);
                                camera_beta[camera_vertex + 1][k] = camera_beta[camera_vertex][k] * (b * sk);
                        }
                        ++camera_vertex;
                }
                else if (kind == TapeRecord::LIGHT_START)
                {
                        const Light<N, T, C>& l = lights[r.get_int()];
                        const float sk = r.get_float();
#pragma unroll
                        for (int k = 0; k < K; ++k)
                        {
                                light_beta[1][k] = l.radiance.c[lane + LANES * k] * sk;
                        }
                        light_vertex = 1;
                }
                else if (kind == TapeRecord::LIGHT_BOUNCE)
                {
                        const Material<T, C>& m = materials[r.get_int()];
                        const BrdfTerms t = r.get_terms();
                        const float sk = r.get_float();
                        const float nk = r.get_float();
#pragma unroll
                        for (int k = 0; k < K; ++k)
                        {
                                const int ch = lane + LANES * k;
                                const float b = brdf_channel(t, m.f0.c[ch], m.rho_ss.c[ch], fresnel_a, fresnel_b);
                                const float beta = light_beta[light_vertex][k] * (b * sk);
                                light_beta[light_vertex + 1][k] = beta * nk;
                        }
                        ++light_vertex;
                }
                else
                {
                        break; // not a bounce record: tapes are written by paths_walk_kernel only
                }
        }
        for (int t_count = 2; t_count <= camera_size; ++t_count)
        {
                for (int s_count = 0; s_count <= light_size; ++s_count)
                {
                        if (t_count + s_count - 2 > max_depth)
                        {
                                continue;
                        }
                        r.n = tape_slot_offset(max_depth, t_count, s_count);
                        const int kind = r.get_int();
                        if (kind == static_cast<int>(TapeRecord::STRATEGY_EMITTED))
                        {
                                r.get_int(); // t
                                const Light<N, T, C>& l = lights[r.get_int()];
                                const float mis = r.get_float();
#pragma unroll
                                for (int k = 0; k < K; ++k)
                                {
                                        const float c = l.radiance.c[lane + LANES * k] * camera_beta[t_count - 1][k];
                                        color[k] += c * mis;
                                }
                        }
                        else if (kind == static_cast<int>(TapeRecord::STRATEGY_LIGHT))
                        {
                                r.get_int(); // t
                                const Material<T, C>& m = materials[r.get_int()];
                                const BrdfTerms t = r.get_terms();
                                const Light<N, T, C>& l = lights[r.get_int()];
                                const float lk = r.get_float();
                                const float mis = r.get_float();
#pragma unroll
                                for (int k = 0; k < K; ++k)
                                {
                                        const int ch = lane + LANES * k;
                                        const float b = brdf_channel(t, m.f0.c[ch], m.rho_ss.c[ch], fresnel_a, fresnel_b);
                                        const float c = ((camera_beta[t_count - 1][k] * b) * l.radiance.c[ch]) * lk;
                                        color[k] += c * mis;
                                }
                        }
                        else if (kind == static_cast<int>(TapeRecord::STRATEGY_CONNECT))
                        {
                                r.get_int(); // s
                                r.get_int(); // t
                                const Material<T, C>& mc = materials[r.get_int()];
                                const BrdfTerms tc = r.get_terms();
                                const Material<T, C>& ml = materials[r.get_int()];
                                const BrdfTerms tl = r.get_terms();
                                const float gk = r.get_float();
                                const float mis = r.get_float();
#pragma unroll
                                for (int k = 0; k < K; ++k)
                                {
                                        const int ch = lane + LANES * k;
                                        const float bc =
                                                brdf_channel(tc, mc.f0.c[ch], mc.rho_ss.c[ch], fresnel_a, fresnel_b);
                                        const float bl =
                                                brdf_channel(tl, ml.f0.c[ch], ml.rho_ss.c[ch], fresnel_a, fresnel_b);
                                        const float c0 =
                                                ((camera_beta[t_count - 1][k] * bc) * bl) * light_beta[s_count - 1][k];
                                        const float c = c0 * gk;
                                        color[k] += c * mis;
                                }
                        }
                }
        }
        float* const out = colors + i * C;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
                out[lane + LANES * k] = has ? color[k] : 0.0f;
        }
        if constexpr (LANES == 1)
        {
                Color<C> c;
#pragma unroll
                for (int k = 0; k < C; ++k)
                {
                        c.c[k] = color[k];
                }
                lum[i] = has ? luminance(c, cie_y) : 0.0f;
                if (has && !all_finite(color))
                {
                        atomicAdd(&stats->nonfinite, 1ull);
                }
        }
        else
        {
                static_assert(LANES == 32);
                // max(0, c_j) * y_j summed for j = 0, 1, ..., C - 1 in order
                float sum = 0.0f;
#pragma unroll
                for (int k = 0; k < K; ++k)
                {
                        const float mine = max_value(0.0f, color[k]) * cie_y[lane + 32 * k];
                        for (int j = 0; j < 32; ++j)
                        {
                                const float v = __shfl_sync(0xffffffffu, mine, j);
                                sum = (k == 0 && j == 0) ? v : sum + v;
                        }
                }
                if (lane == 0)
                {
                        lum[i] = has ? sum : 0.0f;
                }
                const bool bad = __any_sync(0xffffffffu, !all_finite(color));
                if (lane == 0 && has && bad)
                {
                        atomicAdd(&stats->nonfinite, 1ull);
                }
        }
}

} // namespace nbpt
