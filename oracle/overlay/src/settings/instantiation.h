/*
 * Oracle build override of the reference's template-instantiation lists.
 *
 * The reference instantiates its painter for space dimensions 3..6.  The
 * accelerated path covers dimensions 3..5, so this header (found before the
 * reference's own copy on the include path) keeps the same macro names and the
 * same float/double x RGB/Spectrum product but drops dimension 6 from the
 * painter lists, which cuts the oracle's compile time by a quarter.  The
 * geometry-only lists keep their full ranges.
 */
#pragma once

#include <src/color/color.h>

#define TEMPLATE_INSTANTIATION_N(X) X(3) X(4) X(5)
#define TEMPLATE_INSTANTIATION_N_2(X) X(2) X(3) X(4) X(5) X(6)
#define TEMPLATE_INSTANTIATION_N_2_A(X) X(2) X(3) X(4) X(5) X(6) X(7)
#define TEMPLATE_INSTANTIATION_N_M(X) \
        X(3, 1) X(3, 2) X(4, 1) X(4, 2) X(4, 3) X(5, 1) X(5, 2) X(5, 3) X(5, 4) X(6, 1) X(6, 2) X(6, 3) X(6, 4) X(6, 5)

#define NBPT_ORACLE_N_T(N, X) X((N), float) X((N), double)
#define TEMPLATE_INSTANTIATION_N_T(X) NBPT_ORACLE_N_T(3, X) NBPT_ORACLE_N_T(4, X) NBPT_ORACLE_N_T(5, X)
#define TEMPLATE_INSTANTIATION_N_T_2(X) \
        NBPT_ORACLE_N_T(2, X) NBPT_ORACLE_N_T(3, X) NBPT_ORACLE_N_T(4, X) NBPT_ORACLE_N_T(5, X) NBPT_ORACLE_N_T(6, X)

#define TEMPLATE_INSTANTIATION_C(X) X(::ns::color::Color) X(::ns::color::Spectrum)

#define NBPT_ORACLE_T_C(T, X) X(T, ::ns::color::Color) X(T, ::ns::color::Spectrum)
#define TEMPLATE_INSTANTIATION_T_C(X) NBPT_ORACLE_T_C(float, X) NBPT_ORACLE_T_C(double, X)

#define NBPT_ORACLE_N_T_C2(N, T, X) X((N), T, ::ns::color::Color) X((N), T, ::ns::color::Spectrum)
#define NBPT_ORACLE_N_T_C(N, X) NBPT_ORACLE_N_T_C2(N, float, X) NBPT_ORACLE_N_T_C2(N, double, X)
#define TEMPLATE_INSTANTIATION_N_T_C(X) NBPT_ORACLE_N_T_C(3, X) NBPT_ORACLE_N_T_C(4, X) NBPT_ORACLE_N_T_C(5, X)
