// n-D geometry of the painter: rays, hyperplanes, orthogonal complements,
// (n-1)-simplex facets, flat (n-1)-parallelotopes, solid n-parallelotopes and
// axis-aligned boxes, each with the reference's arithmetic order.
#pragma once

#include "core.cuh"

namespace nbpt
{
// Ray with a normalised direction (src/numerical/ray.h: the constructor
// normalises; point(t) = dir * t + org).
template <int N, typename T>
struct Ray final
{
        Vec<N, T> org;
        Vec<N, T> dir;

        NBPT_HD static Ray make(const Vec<N, T>& o, const Vec<N, T>& d)
        {
                return Ray{o, d.normalized()};
        }

        NBPT_HD Vec<N, T> point(const T t) const
        {
                Vec<N, T> p;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        p[i] = dir[i] * t + org[i];
                }
                return p;
        }
};

// ---------------------------------------------------------------------------
// orthogonal complement of N-1 vectors: the cofactor expansion the reference
// uses (src/numerical/complement.h:45-101, determinant.h:33-118).

template <typename T>
NBPT_HD Vec<3, T> orthogonal_complement(const Vec<3, T>* v)
{
        Vec<3, T> r;
        r[0] = v[0][1] * v[1][2] - v[0][2] * v[1][1];
        r[1] = v[0][2] * v[1][0] - v[0][0] * v[1][2];
        r[2] = v[0][0] * v[1][1] - v[0][1] * v[1][0];
        return r;
}

template <typename T>
NBPT_HD Vec<4, T> orthogonal_complement(const Vec<4, T>* v)
{
        Vec<4, T> r;
        r[0] = +v[0][1] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) - v[0][2] * (v[1][1] * v[2][3] - v[1][3] * v[2][1])
               + v[0][3] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]);
        r[1] = -v[0][0] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) + v[0][2] * (v[1][0] * v[2][3] - v[1][3] * v[2][0])
               - v[0][3] * (v[1][0] * v[2][2] - v[1][2] * v[2][0]);
        r[2] = +v[0][0] * (v[1][1] * v[2][3] - v[1][3] * v[2][1]) - v[0][1] * (v[1][0] * v[2][3] - v[1][3] * v[2][0])
               + v[0][3] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
        r[3] = -v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) + v[0][1] * (v[1][0] * v[2][2] - v[1][2] * v[2][0])
               - v[0][2] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
        return r;
}

// 3x3 minor with rows r0..r2 and columns c0..c2 (determinant.h:60-85)
template <typename T>
NBPT_HD T minor3(const Vec<5, T>* v, const int r0, const int r1, const int r2, const int c0, const int c1, const int c2)
{
        const T v00 = v[r0][c0];
        const T v01 = v[r0][c1];
        const T v02 = v[r0][c2];
        const T v10 = v[r1][c0];
        const T v11 = v[r1][c1];
        const T v12 = v[r1][c2];
        const T v20 = v[r2][c0];
        const T v21 = v[r2][c1];
        const T v22 = v[r2][c2];
        const T d0 = v00 * (v11 * v22 - v12 * v21);
        const T d1 = v01 * (v10 * v22 - v12 * v20);
        const T d2 = v02 * (v10 * v21 - v11 * v20);
        return d0 - d1 + d2;
}

// 4x4 determinant of rows 0..3 and the given columns, expanded along row 0
// (determinant.h:87-118: det = 0; det += / -= entry * minor).
template <typename T>
NBPT_HD T minor4(const Vec<5, T>* v, const int* cols)
{
        T det = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
                int c[3];
                int k = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                        if (j != i)
                        {
                                c[k++] = cols[j];
                        }
                }
                const T entry = v[0][cols[i]];
                const T m = minor3(v, 1, 2, 3, c[0], c[1], c[2]);
                if (i & 1)
                {
                        det -= entry * m;
                }
                else
                {
                        det += entry * m;
                }
        }
        return det;
}

template <typename T>
NBPT_HD Vec<5, T> orthogonal_complement(const Vec<5, T>* v)
{
        Vec<5, T> r;
#pragma unroll
        for (int i = 0; i < 5; ++i)
        {
                int cols[4];
                int k = 0;
#pragma unroll
                for (int j = 0; j < 5; ++j)
                {
                        if (j != i)
                        {
                                cols[k++] = j;
                        }
                }
                const T d = minor4(v, cols);
                r[i] = (i & 1) ? -d : d;
        }
        return r;
}

// Index of the largest |component|, first one on ties (complement.h:186-202).
template <int N, typename T>
NBPT_HD int closest_axis(const Vec<N, T>& v)
{
        int index = 0;
        T m = abs_value(v[0]);
#pragma unroll
        for (int i = 1; i < N; ++i)
        {
                const T a = abs_value(v[i]);
                if (a > m)
                {
                        index = i;
                        m = a;
                }
        }
        return index;
}

template <typename T>
NBPT_HD Vec<3, T> cross(const Vec<3, T>& a, const Vec<3, T>& b)
{
        Vec<3, T> r;
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
        return r;
}

// Orthonormal basis of the complement of a unit vector
// (complement.h:213-251 for N = 3 and N = 4; Gram-Schmidt, 253-289, for N = 5).
template <int N, typename T>
NBPT_HD void orthogonal_complement_of_unit_vector(const Vec<N, T>& u, Vec<N, T>* basis)
{
        if constexpr (N == 2)
        {
                basis[0][0] = u[1];
                basis[0][1] = -u[0];
        }
        else if constexpr (N == 3)
        {
                Vec<3, T> v = Vec<3, T>::filled(0);
                if (abs_value(u[0]) > T(0.5))
                {
                        v[1] = 1;
                }
                else
                {
                        v[0] = 1;
                }
                const Vec<3, T> e0 = cross(u, v).normalized();
                basis[0] = e0;
                basis[1] = cross(u, e0);
        }
        else if constexpr (N == 4)
        {
                const int excluded = closest_axis(u);
                int num = 0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        if (i != excluded && num < N - 2)
                        {
                                basis[num] = Vec<N, T>::filled(0);
                                basis[num][i] = 1;
                                ++num;
                        }
                }
                basis[N - 2] = u;
#pragma unroll
                for (int i = 0; i < N - 2; ++i)
                {
                        basis[i] = orthogonal_complement(basis).normalized();
                }
                basis[N - 2] = orthogonal_complement(basis);
        }
        else
        {
                const int excluded = closest_axis(u);
                Vec<N, T> b[N];
                b[0] = u;
                int num = 1;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        if (i != excluded && num < N)
                        {
                                b[num] = Vec<N, T>::filled(0);
                                b[num][i] = 1;
                                ++num;
                        }
                }
                Vec<N, T> o[N];
                o[0] = b[0];
#pragma unroll
                for (int i = 1; i < N; ++i)
                {
                        Vec<N, T> sum = Vec<N, T>::filled(0);
                        for (int k = 0; k < i; ++k)
                        {
                                const T d = dot(b[i], o[k]);
                                sum.multiply_add(o[k], d);
                        }
                        o[i] = (b[i] - sum).normalized();
                }
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        basis[i] = o[i + 1];
                }
        }
}

// ---------------------------------------------------------------------------
// hyperplane n.x - d = 0 (src/geometry/spatial/hyperplane.h:27-74)

template <int N, typename T>
struct Plane final
{
        Vec<N, T> n;
        T d;

        NBPT_HD T intersect(const Ray<N, T>& r) const
        {
                return (d - dot(n, r.org)) / dot(n, r.dir);
        }

        NBPT_HD T distance(const Vec<N, T>& p) const
        {
                return dot(n, p) - d;
        }

        NBPT_HD Vec<N, T> project(const Vec<N, T>& p) const
        {
                return p - n * distance(p);
        }
};

// Ray origin moved off a surface along +-normal by |org| * 64 eps
// (src/geometry/spatial/point_offset.h:35-50).
template <int N, typename T>
NBPT_HD Vec<N, T> offset_ray_org(const Vec<N, T>& normal, const Ray<N, T>& ray)
{
        constexpr T OFFSET = 64 * Limits<T>::EPSILON;
        const T ray_offset = (dot(normal, ray.dir) < 0) ? -OFFSET : OFFSET;
        Vec<N, T> r;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                r[i] = ray.org[i] + abs_value(ray.org[i]) * ray_offset * normal[i];
        }
        return r;
}

// ---------------------------------------------------------------------------
// (n-1)-simplex facet: its hyperplane and N-1 barycentric hyperplanes through
// vertex N-1 scaled so that vertex i is at distance 1 from plane i
// (src/geometry/spatial/hyperplane_simplex.h:82-111, intersect 177-207).

template <int N, typename T>
struct Simplex final
{
        Plane<N, T> plane;
        Plane<N, T> planes[N - 1];

        // Returns false if the facet is degenerate (non-finite normal).
        NBPT_HD bool set(const Vec<N, T>* vertices)
        {
                Vec<N, T> vectors[N - 1];
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        vectors[i] = vertices[i] - vertices[N - 1];
                }
                plane.n = orthogonal_complement(vectors).normalized();
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        const T x = plane.n[i];
                        if (!(x - x == 0))
                        {
                                return false;
                        }
                }
                plane.d = dot(plane.n, vertices[N - 1]);
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        const Vec<N, T> vi = vectors[i];
                        vectors[i] = plane.n;
                        planes[i].n = orthogonal_complement(vectors);
                        vectors[i] = vi;
                        planes[i].d = dot(vertices[N - 1], planes[i].n);
                        const T distance = planes[i].distance(vertices[i]);
                        planes[i].n = planes[i].n / distance;
                        planes[i].d /= distance;
                }
                return true;
        }

        // Hit distance, or 0 for no hit (a hit has t > 0).
        NBPT_HD T intersect(const Ray<N, T>& r) const
        {
                const T t = plane.intersect(r);
                if (!(t > 0))
                {
                        return 0;
                }
                const Vec<N, T> p = r.point(t);
                T bc[N - 1];
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        bc[i] = planes[i].distance(p);
                        if (!(bc[i] > 0 && bc[i] < 1))
                        {
                                return 0;
                        }
                }
                T sum = bc[0];
#pragma unroll
                for (int i = 1; i < N - 1; ++i)
                {
                        sum += bc[i];
                }
                return (sum < 1) ? t : T(0);
        }

        // barycentric coordinates (hyperplane_simplex.h:70-80)
        NBPT_HD void barycentric(const Vec<N, T>& p, T* bc) const
        {
                bc[N - 1] = 1;
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        bc[i] = planes[i].distance(p);
                        bc[N - 1] -= bc[i];
                }
        }
};

// ---------------------------------------------------------------------------
// flat (n-1)-parallelotope in a hyperplane
// (src/geometry/spatial/hyperplane_parallelotope.h:99-189)

template <int N, typename T>
struct FlatParallelotope final
{
        Plane<N, T> plane;
        Plane<N, T> planes[N - 1];

        NBPT_HD bool set(const Vec<N, T>& org, const Vec<N, T>* vectors_in)
        {
                Vec<N, T> vectors[N - 1];
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        vectors[i] = vectors_in[i];
                }
                plane.n = orthogonal_complement(vectors).normalized();
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        const T x = plane.n[i];
                        if (!(x - x == 0))
                        {
                                return false;
                        }
                }
                plane.d = dot(plane.n, org);
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        const Vec<N, T> vi = vectors[i];
                        vectors[i] = plane.n;
                        planes[i].n = orthogonal_complement(vectors);
                        vectors[i] = vi;
                        if (dot(planes[i].n, vectors[i]) < 0)
                        {
                                planes[i].n = -planes[i].n;
                        }
                        planes[i].d = dot(org, planes[i].n);
                        const T distance = planes[i].distance(org + vectors[i]);
                        planes[i].n = planes[i].n / distance;
                        planes[i].d /= distance;
                }
                return true;
        }

        NBPT_HD T intersect(const Ray<N, T>& r) const
        {
                const T t = plane.intersect(r);
                if (!(t > 0))
                {
                        return 0;
                }
                const Vec<N, T> p = r.point(t);
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        const T d = planes[i].distance(p);
                        if (!(d > 0 && d < 1))
                        {
                                return 0;
                        }
                }
                return t;
        }
};

// ---------------------------------------------------------------------------
// solid n-parallelotope: N slabs between d1 and d2 along outward unit normals
// (src/geometry/spatial/parallelotope.h:192-379)

template <int N, typename T>
struct SolidParallelotope final
{
        Vec<N, T> n[N];
        T d1[N];
        T d2[N];

        NBPT_HD void set(const Vec<N, T>& org, const Vec<N, T>* vectors)
        {
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        Vec<N, T> others[N - 1];
                        int k = 0;
#pragma unroll
                        for (int j = 0; j < N; ++j)
                        {
                                if (j != i)
                                {
                                        others[k++] = vectors[j];
                                }
                        }
                        n[i] = orthogonal_complement(others).normalized();
                        if (dot(n[i], vectors[i]) < 0)
                        {
                                n[i] = -n[i];
                        }
                        d1[i] = dot(org, n[i]);
                        d2[i] = dot(org + vectors[i], n[i]);
                }
        }

        // intersect_volume: entry distance (0 from inside), or -1 for no hit.
        NBPT_HD T intersect_volume(const Ray<N, T>& r, const T max_distance) const
        {
                T near = 0;
                T far = max_distance;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        const T s = dot(r.dir, n[i]);
                        const T d = dot(r.org, n[i]);
                        if (s == 0)
                        {
                                if (d < d1[i] || d > d2[i])
                                {
                                        return -1;
                                }
                                continue;
                        }
                        const T rec = 1 / s;
                        const T a0 = (d1[i] - d) * rec;
                        const T a1 = (d2[i] - d) * rec;
                        const T an = (s < 0) ? a1 : a0;
                        const T af = (s < 0) ? a0 : a1;
                        near = max_value(near, an);
                        far = min_value(far, af);
                        if (far < near)
                        {
                                return -1;
                        }
                }
                return near;
        }

        // normal of the face closest to the point
        NBPT_HD Vec<N, T> normal(const Vec<N, T>& p) const
        {
                T min_distance = Limits<T>::MAX;
                Vec<N, T> res = n[0];
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        const T d = dot(p, n[i]);
                        {
                                const T distance = abs_value(d - d1[i]);
                                if (distance < min_distance)
                                {
                                        min_distance = distance;
                                        res = -n[i];
                                }
                        }
                        {
                                const T distance = abs_value(d - d2[i]);
                                if (distance < min_distance)
                                {
                                        min_distance = distance;
                                        res = n[i];
                                }
                        }
                }
                return res;
        }

        NBPT_HD Vec<N, T> project(const Vec<N, T>& p) const
        {
                T min_distance = Limits<T>::MAX;
                int index = 0;
                T plane_distance = 0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        const T d = dot(p, n[i]);
                        {
                                const T distance = d - d1[i];
                                const T a = abs_value(distance);
                                if (a < min_distance)
                                {
                                        min_distance = a;
                                        index = i;
                                        plane_distance = distance;
                                }
                        }
                        {
                                const T distance = d - d2[i];
                                const T a = abs_value(distance);
                                if (a < min_distance)
                                {
                                        min_distance = a;
                                        index = i;
                                        plane_distance = distance;
                                }
                        }
                }
                return p - n[index] * plane_distance;
        }
};

// ---------------------------------------------------------------------------
// axis-aligned box tests (src/geometry/spatial/bounding_box.h:121-194)

// Traversal test with the precomputed reciprocal direction and signs.
template <int N, typename T>
NBPT_HD bool box_hit(
        const T* lo,
        const T* hi,
        const Vec<N, T>& org,
        const Vec<N, T>& rec,
        const unsigned neg_mask,
        const T max_distance)
{
        T near = 0;
        T far = max_distance;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                const bool negative = (neg_mask >> i) & 1u;
                const T d = org[i];
                const T r = rec[i];
                const T a1 = ((negative ? hi[i] : lo[i]) - d) * r;
                const T a2 = ((negative ? lo[i] : hi[i]) - d) * r;
                near = a1 > near ? a1 : near;
                far = a2 < far ? a2 : far;
                if (far < near)
                {
                        return false;
                }
        }
        return true;
}

// Volume test: entry distance (0 from inside) or -1 for no hit.
template <int N, typename T>
NBPT_HD T box_volume(const T* lo, const T* hi, const Ray<N, T>& r, const T max_distance)
{
        T near = 0;
        T far = max_distance;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                const T dir = r.dir[i];
                const T d = r.org[i];
                if (dir == 0)
                {
                        if (!(d >= lo[i] && d <= hi[i]))
                        {
                                return -1;
                        }
                        continue;
                }
                const bool negative = dir < 0;
                const T rr = 1 / dir;
                const T a1 = ((negative ? hi[i] : lo[i]) - d) * rr;
                const T a2 = ((negative ? lo[i] : hi[i]) - d) * rr;
                near = a1 > near ? a1 : near;
                far = a2 < far ? a2 : far;
                if (!(far >= near))
                {
                        return -1;
                }
        }
        return near;
}
} // namespace nbpt
