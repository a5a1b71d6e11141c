/*
 * Oracle build override of the reference's template-instantiation lists for
 * its convex hull alone (src/geometry/core/convex_hull.cpp, compiled into
 * _ref/libnbpt_hull.so).  The hull computes in exact integers whose width
 * grows with the dimension: 30 * N + log2(N!) bits, 93 in 3-space and 125 in
 * 4-space, which fit the compiler's 128-bit integers; 5-space and above need
 * GMP, which is not installed here.  So the convex hull is instantiated for
 * 3- and 4-space only, and the Delaunay triangulation that shares the file
 * for 2- and 3-space (a hull in one dimension more, at most 127 bits).
 */
#pragma once

#define TEMPLATE_INSTANTIATION_N_2(X) X(2) X(3)
#define TEMPLATE_INSTANTIATION_N_2_A(X) X(3) X(4)
