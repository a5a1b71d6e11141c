/*
 * Test-oracle build only.
 *
 * The reference measures the cost of one primitive intersection with a
 * micro-benchmark the first time the cost is needed
 * (src/geometry/spatial/bounding_box.cpp:32-69, hyperplane_simplex.cpp:32-43,
 * hyperplane_parallelotope.cpp, hyperplane_ball.cpp, parallelotope.cpp) and
 * feeds it to the SAH BVH build (src/geometry/accelerators/bvh_build.h:106,
 * bvh_split.h:215-239).  Timed costs make the BVH shape differ from run to run.
 * The oracle replaces those five translation units with the fixed costs below
 * so that its BVH, and therefore every tie broken by traversal order, is the
 * same on every run and every machine.  The accelerated library's own BVH
 * builder uses the same constants (math_b200/csrc/bvh_build.cpp).
 *
 * A cost is seconds per intersection; only ratios matter to the SAH.
 */

#include <src/geometry/spatial/bounding_box.h>
#include <src/geometry/spatial/hyperplane_ball.h>
#include <src/geometry/spatial/hyperplane_parallelotope.h>
#include <src/geometry/spatial/hyperplane_simplex.h>
#include <src/geometry/spatial/parallelotope.h>
#include <src/settings/instantiation.h>

#include <cstddef>

namespace ns::geometry::spatial
{
namespace
{
// intersections per second of one primitive, per unit of space dimension
constexpr double BOX_RATE = 1.6e9;
constexpr double BOX_VOLUME_RATE = 1.2e9;
constexpr double BOX_R_RATE = 2.4e9;
constexpr double SIMPLEX_RATE = 0.8e9;
constexpr double HYPERPLANE_PARALLELOTOPE_RATE = 0.8e9;
constexpr double HYPERPLANE_BALL_RATE = 1.0e9;
constexpr double PARALLELOTOPE_RATE = 0.5e9;

template <std::size_t N>
constexpr double cost(const double rate)
{
        return static_cast<double>(N) / rate;
}
}

template <std::size_t N, typename T>
T BoundingBox<N, T>::intersection_cost()
{
        return cost<N>(BOX_RATE);
}

template <std::size_t N, typename T>
T BoundingBox<N, T>::intersection_volume_cost()
{
        return cost<N>(BOX_VOLUME_RATE);
}

template <std::size_t N, typename T>
T BoundingBox<N, T>::intersection_r_cost()
{
        return cost<N>(BOX_R_RATE);
}

template <std::size_t N, typename T>
T HyperplaneSimplex<N, T>::intersection_cost()
{
        return cost<N>(SIMPLEX_RATE);
}

template <std::size_t N, typename T>
T HyperplaneParallelotope<N, T>::intersection_cost()
{
        return cost<N>(HYPERPLANE_PARALLELOTOPE_RATE);
}

template <std::size_t N, typename T>
T HyperplaneBall<N, T>::intersection_cost()
{
        return cost<N>(HYPERPLANE_BALL_RATE);
}

template <std::size_t N, typename T>
T Parallelotope<N, T>::intersection_cost()
{
        return cost<N>(PARALLELOTOPE_RATE);
}

#define NBPT_ORACLE_COSTS(N, T)                                      \
        template T BoundingBox<(N), T>::intersection_cost();         \
        template T BoundingBox<(N), T>::intersection_volume_cost();  \
        template T BoundingBox<(N), T>::intersection_r_cost();       \
        template T HyperplaneSimplex<(N), T>::intersection_cost();   \
        template T HyperplaneParallelotope<(N), T>::intersection_cost(); \
        template T HyperplaneBall<(N), T>::intersection_cost();      \
        template T Parallelotope<(N), T>::intersection_cost();

TEMPLATE_INSTANTIATION_N_T_2(NBPT_ORACLE_COSTS)
}
