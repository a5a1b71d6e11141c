// The single-precision path kernels, compiled in their own unit
// (painter_paths_f.cu) with multiply-add contraction, denormals flushed to
// zero and approximate division and square root.  The library's other units
// compile with none of these, so that double precision follows the
// reference's operation order bit for bit; single precision is checked
// against the reference statistically (relative RMSE, z-tests), and these
// options make its path kernels about 15 % faster.  The painter launches them
// through these pointers, so no other unit instantiates them.
#pragma once

#include "kernels.cuh"
#include "pt.cuh"

namespace nbpt
{
template <int N>
struct FloatPathKernels final
{
        decltype(&paths_walk_kernel<N, float>) walk;
        decltype(&paths_light_kernel<N, float>) light;
        decltype(&paths_connect_kernel<N, float>) connect;
        decltype(&paths_replay_kernel<N, float, 3, 1>) replay_rgb;
        decltype(&paths_replay_kernel<N, float, 64, 32>) replay_spectrum;
        decltype(&pt_paths_kernel<N, float, 3>) pt_rgb;
        decltype(&pt_paths_kernel<N, float, 64>) pt_spectrum;
};

template <int N>
const FloatPathKernels<N>& float_path_kernels();

extern template const FloatPathKernels<3>& float_path_kernels<3>();
extern template const FloatPathKernels<4>& float_path_kernels<4>();
extern template const FloatPathKernels<5>& float_path_kernels<5>();
} // namespace nbpt
