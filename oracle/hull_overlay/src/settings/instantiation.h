/*
 * Oracle build override of the reference's template-instantiation lists for
 * its convex hull alone (src/geometry/core/convex_hull.cpp, compiled into
 * _ref/libnbpt_hull.so).  The hull computes in exact integers whose width
 * grows with the dimension: 30 * N + log2(N!) bits, 93 in 3-space and 125 in
 * 4-space, which fit the compiler's 128-bit integers, 157 in 5-space, which
 * takes GMP (hull_gmp/ over the system's libgmp).  So the convex hull is
 * instantiated for 3-, 4- and 5-space, and the Delaunay triangulation that
 * shares the file for 2- and 3-space only (a hull in one dimension more).
 */
#pragma once

#define TEMPLATE_INSTANTIATION_N_2(X) X(2) X(3)
#define TEMPLATE_INSTANTIATION_N_2_A(X) X(3) X(4) X(5)
