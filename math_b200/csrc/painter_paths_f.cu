// Single-precision path kernels with multiply-add contraction, denormals
// flushed and approximate division and square root (float_paths.h; the
// Makefile compiles this unit with -fmad=true -ftz=true -prec-div=false
// -prec-sqrt=false).
#include "float_paths.h"

namespace nbpt
{
template <int N>
const FloatPathKernels<N>& float_path_kernels()
{
        static const FloatPathKernels<N> kernels{
                &paths_walk_kernel<N, float>,          &paths_light_kernel<N, float>,
                &paths_connect_kernel<N, float>,       &paths_replay_kernel<N, float, 3, 1>,
                &paths_replay_kernel<N, float, 64, 32>, &pt_paths_kernel<N, float, 3>,
                &pt_paths_kernel<N, float, 64>};
        return kernels;
}

template const FloatPathKernels<3>& float_path_kernels<3>();
template const FloatPathKernels<4>& float_path_kernels<4>();
template const FloatPathKernels<5>& float_path_kernels<5>();
} // namespace nbpt
