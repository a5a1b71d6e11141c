// C entry point of the reference's own convex hull (compute_convex_hull,
// src/geometry/core/convex_hull.h:95-98, compiled from its sources into
// _ref/libnbpt_hull.so), for the tests that check that the scene generators'
// hulls have the reference's facets.  Test infrastructure only.

#include <src/geometry/core/convex_hull.h>
#include <src/numerical/vector.h>
#include <src/progress/progress.h>

#include <exception>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_error;

template <std::size_t N>
long long hull(const float* points, const long long count, int* facets, const long long capacity)
{
        std::vector<ns::numerical::Vector<N, float>> p(count);
        for (long long i = 0; i < count; ++i)
        {
                for (std::size_t d = 0; d < N; ++d)
                {
                        p[i][d] = points[i * N + d];
                }
        }
        ns::progress::Ratio progress(nullptr);
        const auto simplices = ns::geometry::core::compute_convex_hull(p, &progress, false);
        const long long n = static_cast<long long>(simplices.size());
        if (facets && n <= capacity)
        {
                for (long long f = 0; f < n; ++f)
                {
                        for (std::size_t d = 0; d < N; ++d)
                        {
                                facets[f * N + d] = simplices[f].vertices()[d];
                        }
                }
        }
        return n;
}
}

extern "C" {
// facets of the hull of count points [count][n] (n = 3, 4 or 5): returns the
// facet count (facets written when it is at most capacity), -1 on error
long long oracle_convex_hull(const int n, const float* points, const long long count, int* facets,
                             const long long capacity)
{
        try
        {
                if (n == 3)
                {
                        return hull<3>(points, count, facets, capacity);
                }
                if (n == 4)
                {
                        return hull<4>(points, count, facets, capacity);
                }
                if (n == 5)
                {
                        return hull<5>(points, count, facets, capacity);
                }
                g_error = "convex hull: dimension " + std::to_string(n) + " is not built (3, 4 and 5 only)";
        }
        catch (const std::exception& e)
        {
                g_error = e.what();
        }
        return -1;
}

const char* oracle_hull_error()
{
        return g_error.c_str();
}
}
