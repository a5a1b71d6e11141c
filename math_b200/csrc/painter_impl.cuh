// Templated scene and painter implementation (one instantiation per space
// dimension N, path precision T and colour channel count C).
//
// Scene preparation (host): shapes, meshes, lights and the projector are
// turned into the device records of scene.cuh with the reference's
// arithmetic (src/painter/shapes/*.cpp, lights/*.cpp, projectors/*.cpp,
// shapes/mesh/data.cpp); the mesh BVH is built on the host (bvh_build.cpp)
// and the facet records in double precision on the GPU (facet_setup_kernel).
//
// Painter: one pass renders every pixel's stratified samples through the path
// kernel and folds them into the per-pixel estimator on the device.
#pragma once

#include "bvh_build.h"
#include "bvh_device.cuh"
#include "cuda_error.h"
#include "mesh_files.h"
#include "device_pool.h"
#include "estimator.cuh"
#include "float_paths.h"
#include "host_math.h"
#include "kernels.cuh"
#include "painter_api.h"
#include "pt.cuh"
#include "tables.inc"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <thread>
#include <atomic>
#include <exception>
#include <mutex>
#include <vector>

namespace nbpt
{
#define NBPT_CUDA(x) ::nbpt::cuda_check((x), #x)

template <typename X>
class DeviceArray final
{
        X* ptr_ = nullptr;
        std::size_t size_ = 0;
        int device_ = 0;

        void release()
        {
                if (ptr_)
                {
                        pool::release(ptr_, size_ * sizeof(X), device_);
                        ptr_ = nullptr;
                }
        }

public:
        DeviceArray() = default;
        DeviceArray(const DeviceArray&) = delete;
        DeviceArray& operator=(const DeviceArray&) = delete;

        // gives the buffer back to the library's cache; returns its bytes
        std::size_t free()
        {
                const std::size_t b = ptr_ ? size_ * sizeof(X) : 0;
                release();
                size_ = 0;
                return b;
        }

        ~DeviceArray()
        {
                release();
        }

        void allocate(const std::size_t n)
        {
                release();
                size_ = n;
                if (n > 0)
                {
                        ptr_ = static_cast<X*>(pool::allocate(n * sizeof(X), &device_));
                }
        }

        void upload(const std::vector<X>& v)
        {
                allocate(v.size());
                if (!v.empty())
                {
                        NBPT_CUDA(cudaMemcpy(ptr_, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
                }
        }

        void upload(const X* data, const std::size_t n)
        {
                allocate(n);
                if (n > 0)
                {
                        NBPT_CUDA(cudaMemcpy(ptr_, data, n * sizeof(X), cudaMemcpyHostToDevice));
                }
        }

        // copies on `stream` and waits for them (no legacy default stream, so
        // painters driven from different host threads do not order each other)
        void upload_on(const std::vector<X>& v, const cudaStream_t stream)
        {
                allocate(v.size());
                if (!v.empty())
                {
                        NBPT_CUDA(cudaMemcpyAsync(ptr_, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, stream));
                        NBPT_CUDA(cudaStreamSynchronize(stream));
                }
        }

        void download_on(X* out, const std::size_t n, const cudaStream_t stream) const
        {
                if (n > 0)
                {
                        NBPT_CUDA(cudaMemcpyAsync(out, ptr_, n * sizeof(X), cudaMemcpyDeviceToHost, stream));
                        NBPT_CUDA(cudaStreamSynchronize(stream));
                }
        }

        void download(X* out, const std::size_t n) const
        {
                if (n > 0)
                {
                        NBPT_CUDA(cudaMemcpy(out, ptr_, n * sizeof(X), cudaMemcpyDeviceToHost));
                }
        }

        [[nodiscard]] X* get() const
        {
                return ptr_;
        }

        [[nodiscard]] std::size_t size() const
        {
                return size_;
        }

        [[nodiscard]] std::size_t bytes() const
        {
                return size_ * sizeof(X);
        }
};

inline unsigned blocks_for(const long long n, const int threads)
{
        return static_cast<unsigned>((n + threads - 1) / threads);
}

template <int N, typename T>
NBPT_HD Vec<N, T> to_vec(const double* p)
{
        Vec<N, T> v;
        for (int i = 0; i < N; ++i)
        {
                v[i] = static_cast<T>(p[i]);
        }
        return v;
}

// Inverse of an M x M matrix (row major) in T as the reference computes it
// (src/numerical/solve.h:159-172): for M <= 3 the adjugate over the
// determinant (Leon, Linear Algebra with Applications, 2.3), for M >= 4
// Gaussian elimination with partial pivoting on [A | I] and back substitution
// (Karniadakis and Kirby, Parallel Scientific Computing in C++ and MPI;
// src/numerical/gauss.h:142-280), with the same operation order.
template <int M, typename T>
std::array<T, M * M> inverse(std::array<T, M * M> a)
{
        const auto at = [&](const int r, const int c) -> T&
        {
                return a[r * M + c];
        };
        std::array<T, M * M> b{};
        if constexpr (M == 1)
        {
                b[0] = T{1} / a[0];
        }
        else if constexpr (M == 2)
        {
                const T d = at(0, 0) * at(1, 1) - at(0, 1) * at(1, 0);
                b[0] = at(1, 1) / d;
                b[1] = -at(0, 1) / d;
                b[2] = -at(1, 0) / d;
                b[3] = at(0, 0) / d;
        }
        else if constexpr (M == 3)
        {
                const T c00 = at(1, 1) * at(2, 2) - at(1, 2) * at(2, 1);
                const T c10 = at(0, 2) * at(2, 1) - at(0, 1) * at(2, 2);
                const T c20 = at(0, 1) * at(1, 2) - at(0, 2) * at(1, 1);
                const T d = at(0, 0) * c00 + at(1, 0) * c10 + at(2, 0) * c20;
                b[0] = c00 / d;
                b[1] = c10 / d;
                b[2] = c20 / d;
                b[3] = (at(1, 2) * at(2, 0) - at(1, 0) * at(2, 2)) / d;
                b[4] = (at(0, 0) * at(2, 2) - at(0, 2) * at(2, 0)) / d;
                b[5] = (at(0, 2) * at(1, 0) - at(0, 0) * at(1, 2)) / d;
                b[6] = (at(1, 0) * at(2, 1) - at(1, 1) * at(2, 0)) / d;
                b[7] = (at(0, 1) * at(2, 0) - at(0, 0) * at(2, 1)) / d;
                b[8] = (at(0, 0) * at(1, 1) - at(0, 1) * at(1, 0)) / d;
        }
        else
        {
                for (int i = 0; i < M; ++i)
                {
                        b[i * M + i] = 1;
                }
                // rows are exchanged whole, which is what exchanging the
                // reference's row pointers does
                const auto swap_rows = [](std::array<T, M * M>& m, const int r0, const int r1)
                {
                        for (int c = 0; c < M; ++c)
                        {
                                std::swap(m[r0 * M + c], m[r1 * M + c]);
                        }
                };
                for (int k = 0; k < M - 1; ++k)
                {
                        T largest = abs_value(at(k, k));
                        int pivot = k;
                        for (int r = k + 1; r < M; ++r)
                        {
                                const T v = abs_value(at(r, k));
                                if (v > largest)
                                {
                                        largest = v;
                                        pivot = r;
                                }
                        }
                        if (pivot != k)
                        {
                                swap_rows(a, pivot, k);
                                swap_rows(b, pivot, k);
                        }
                        for (int i = k + 1; i < M; ++i)
                        {
                                const T l_ik = at(i, k) / at(k, k);
                                for (int j = k; j < M; ++j)
                                {
                                        at(i, j) -= l_ik * at(k, j);
                                }
                                for (int m = 0; m < M; ++m)
                                {
                                        b[i * M + m] -= l_ik * b[k * M + m];
                                }
                        }
                }
                for (int m = 0; m < M; ++m)
                {
                        b[(M - 1) * M + m] /= at(M - 1, M - 1);
                }
                for (int k = M - 2; k >= 0; --k)
                {
                        for (int j = k + 1; j < M; ++j)
                        {
                                const T u = -at(k, j);
                                for (int m = 0; m < M; ++m)
                                {
                                        b[k * M + m] += b[j * M + m] * u;
                                }
                        }
                        for (int m = 0; m < M; ++m)
                        {
                                b[k * M + m] /= at(k, k);
                        }
                }
        }
        for (const T x : b)
        {
                if (!std::isfinite(x))
                {
                        throw std::runtime_error("mesh matrix is singular");
                }
        }
        return b;
}

// Runs f(begin, end) over [0, count) split across the host's threads.
template <typename F>
void parallel_ranges(const std::size_t count, const F& f, const std::size_t grain = 4096)
{
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const std::size_t parts = std::min<std::size_t>(hw, std::max<std::size_t>(1, count / grain));
        if (parts <= 1)
        {
                f(std::size_t{0}, count);
                return;
        }
        std::vector<std::thread> threads;
        threads.reserve(parts - 1);
        const std::size_t step = (count + parts - 1) / parts;
        std::exception_ptr error;
        std::mutex error_mutex;
        const auto run = [&](const std::size_t b, const std::size_t e)
        {
                try
                {
                        f(b, e);
                }
                catch (...)
                {
                        const std::lock_guard lock(error_mutex);
                        error = std::current_exception();
                }
        };
        for (std::size_t p = 1; p < parts; ++p)
        {
                const std::size_t b = std::min(count, p * step);
                const std::size_t e = std::min(count, b + step);
                threads.emplace_back(
                        [&run, b, e]
                        {
                                run(b, e);
                        });
        }
        run(std::size_t{0}, std::min(count, step));
        for (std::thread& t : threads)
        {
                t.join();
        }
        if (error)
        {
                std::rethrow_exception(error);
        }
}

// f(begin, end) over [0, count): in parts on the host threads, or at once
template <typename F>
void ranges(const bool parallel, const std::size_t count, const F& f, const std::size_t grain = 4096)
{
        if (parallel)
        {
                parallel_ranges(count, f, grain);
        }
        else
        {
                f(std::size_t{0}, count);
        }
}

// f(i) for i in [0, count), the indices shared out among the host threads
template <typename F>
void parallel_items(const std::size_t count, const F& f)
{
        const unsigned threads = std::min<std::size_t>(std::max(1u, std::thread::hardware_concurrency()), count);
        std::atomic<std::size_t> next{0};
        std::vector<std::thread> pool;
        std::exception_ptr error;
        std::mutex error_mutex;
        const auto work = [&]
        {
                try
                {
                        for (std::size_t i = next++; i < count; i = next++)
                        {
                                f(i);
                        }
                }
                catch (...)
                {
                        const std::lock_guard lock(error_mutex);
                        error = std::current_exception();
                }
        };
        for (unsigned t = 1; t < threads; ++t)
        {
                pool.emplace_back(work);
        }
        work();
        for (std::thread& t : pool)
        {
                t.join();
        }
        if (error)
        {
                std::rethrow_exception(error);
        }
}

// Adds the seconds from its construction to its destruction to `total`.
class Stopwatch final
{
        double& total_;
        std::chrono::steady_clock::time_point start_;

public:
        explicit Stopwatch(double& total)
                : total_(total),
                  start_(std::chrono::steady_clock::now())
        {
        }

        ~Stopwatch()
        {
                total_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count();
        }

        Stopwatch(const Stopwatch&) = delete;
        Stopwatch& operator=(const Stopwatch&) = delete;
};

// The normal of a point set as the reference computes it for a vertex's
// vicinity (src/numerical/normal.h:46-103): the eigenvector of the smallest
// eigenvalue of the point set's covariance, found as the orthogonal
// complement of the other N - 1 eigenvectors.  The eigenvectors come from
// the cyclic Jacobi method with a threshold (Kiusalaas, Numerical Methods in
// Engineering with Python 3, section 9.2; src/numerical/eigen.h), on the
// upper triangle, with the reference's tolerance and at most 20 sweeps.
// Only the sign of this normal reaches the mesh (the vertex normal is the
// sum of its facets' normals, each turned towards it), but that sign decides
// which way a facet's geometric normal faces (facet.cpp:104-117), so the
// steps follow the reference's for the same eigenvector signs.
template <int N>
Vec<N, double> point_normal(const std::vector<Vec<N, double>>& points)
{
        if (points.size() < static_cast<std::size_t>(N))
        {
                throw std::runtime_error("At least " + std::to_string(N) + " points are required for point normal");
        }
        // covariance (numerical/covariance.h:38-66), upper triangle
        Vec<N, double> average = Vec<N, double>::filled(0);
        for (const Vec<N, double>& p : points)
        {
                average = average + p;
        }
        average = average / static_cast<double>(points.size());
        double a[N][N] = {};
        for (const Vec<N, double>& p : points)
        {
                const Vec<N, double> v = p - average;
                for (int i = 0; i < N; ++i)
                {
                        for (int j = i; j < N; ++j)
                        {
                                a[i][j] += v[i] * v[j];
                        }
                }
        }
        double largest = std::numeric_limits<double>::lowest();
        for (int i = 0; i < N - 1; ++i)
        {
                for (int j = i + 1; j < N; ++j)
                {
                        largest = std::max(largest, std::abs(a[i][j]));
                }
        }
        const double tolerance = largest * (100 * std::numeric_limits<double>::epsilon());
        // eigenvectors as rows, from the identity
        Vec<N, double> vectors[N];
        for (int i = 0; i < N; ++i)
        {
                vectors[i] = Vec<N, double>::filled(0);
                vectors[i][i] = 1;
        }
        const auto rotate = [&](const int k, const int l)
        {
                const double diff = a[l][l] - a[k][k];
                const double phi = diff / (2 * a[k][l]);
                const double phi_s = phi * phi + 1;
                double t;
                if (phi_s <= std::numeric_limits<double>::max())
                {
                        t = std::copysign(1 / (std::abs(phi) + std::sqrt(phi_s)), phi);
                }
                else
                {
                        t = 1 / (2 * phi);
                }
                const double c = 1 / std::sqrt(t * t + 1);
                const double s = t * c;
                const double tau = s / (1 + c);
                const double a_kl = a[k][l];
                a[k][l] = 0;
                a[k][k] = a[k][k] - t * a_kl;
                a[l][l] = a[l][l] + t * a_kl;
                for (int i = 0; i < k; ++i)
                {
                        const double a_ik = a[i][k];
                        const double a_il = a[i][l];
                        a[i][k] = a_ik - s * (a_il + tau * a_ik);
                        a[i][l] = a_il + s * (a_ik - tau * a_il);
                }
                for (int i = k + 1; i < l; ++i)
                {
                        const double a_ki = a[k][i];
                        const double a_il = a[i][l];
                        a[k][i] = a_ki - s * (a_il + tau * a_ki);
                        a[i][l] = a_il + s * (a_ki - tau * a_il);
                }
                for (int i = l + 1; i < N; ++i)
                {
                        const double a_ki = a[k][i];
                        const double a_li = a[l][i];
                        a[k][i] = a_ki - s * (a_li + tau * a_ki);
                        a[l][i] = a_li + s * (a_ki - tau * a_li);
                }
                for (int i = 0; i < N; ++i)
                {
                        const double p_ik = vectors[k][i];
                        const double p_il = vectors[l][i];
                        vectors[k][i] = p_ik - s * (p_il + tau * p_ik);
                        vectors[l][i] = p_il + s * (p_ik - tau * p_il);
                }
        };
        bool converged = false;
        for (int sweep = 0; sweep < 20 && !converged; ++sweep)
        {
                double sum = 0;
                for (int i = 0; i < N - 1; ++i)
                {
                        for (int j = i + 1; j < N; ++j)
                        {
                                sum += std::abs(a[i][j]);
                        }
                }
                const double mu = 0.5 * sum / (N * (N - 1));
                for (int k = 0; k < N - 1; ++k)
                {
                        for (int l = k + 1; l < N; ++l)
                        {
                                if (std::abs(a[k][l]) >= mu)
                                {
                                        rotate(k, l);
                                }
                        }
                }
                converged = mu <= tolerance;
        }
        if (!converged)
        {
                throw std::runtime_error("Jacobi method did not converge");
        }
        int smallest = 0;
        for (int i = 1; i < N; ++i)
        {
                if (a[i][i] < a[smallest][smallest])
                {
                        smallest = i;
                }
        }
        Vec<N, double> others[N - 1];
        for (int i = 0, k = 0; i < N; ++i)
        {
                if (i != smallest)
                {
                        others[k++] = vectors[i];
                }
        }
        return orthogonal_complement(others).normalized();
}

// Solid angle at a facet's corner for the corner's weight (3-space: the
// angle; 4-space: the spherical triangle's excess, src/geometry/shapes/
// sphere_simplex.h:88-156), 0 for a degenerate corner.
template <int N>
double corner_weight(Vec<N, double> (&e)[N - 1])
{
        double norm[N - 1];
        for (int j = 0; j < N - 1; ++j)
        {
                norm[j] = e[j].norm();
                if (norm[j] == 0)
                {
                        return 0;
                }
        }
        if constexpr (N == 3)
        {
                const double cosine = dot(e[0] / norm[0], e[1] / norm[1]);
                return std::acos(std::clamp(cosine, -1.0, 1.0));
        }
        else
        {
                static_assert(N == 4);
                const Vec<N, double> a = e[0] / norm[0];
                const Vec<N, double> b = e[1] / norm[1];
                const Vec<N, double> c = e[2] / norm[2];
                const double cos_a = dot(b, c);
                const double cos_b = dot(a, c);
                const double cos_c = dot(a, b);
                const double sin_a_2 = 1 - cos_a * cos_a;
                const double sin_b_2 = 1 - cos_b * cos_b;
                const double sin_c_2 = 1 - cos_c * cos_c;
                const double dihedral_cosine_a = (cos_a - cos_b * cos_c) / std::sqrt(sin_b_2 * sin_c_2);
                const double dihedral_cosine_b = (cos_b - cos_a * cos_c) / std::sqrt(sin_a_2 * sin_c_2);
                const double dihedral_cosine_c = (cos_c - cos_a * cos_b) / std::sqrt(sin_a_2 * sin_b_2);
                const double dihedral_a = std::acos(std::clamp(dihedral_cosine_a, -1.0, 1.0));
                const double dihedral_b = std::acos(std::clamp(dihedral_cosine_b, -1.0, 1.0));
                const double dihedral_c = std::acos(std::clamp(dihedral_cosine_c, -1.0, 1.0));
                const double area = dihedral_a + dihedral_b + dihedral_c - 3.141592653589793238462643383279502884;
                return std::max(0.0, area);
        }
}

// Vertex normals of a simplex mesh as src/model/mesh/normals.cpp:46-195
// computes them: per vertex, the facet normals around it weighted by the
// facet's solid angle at the vertex (n = 3, 4) or 1 (n >= 5), each turned
// towards the normal of the vertex's vicinity (point_normal), summed in facet
// order and normalised, then rounded to float.  Facet normals and angles are
// computed in parallel, and so are the vertices.
template <int N>
std::vector<float> vertex_normals(const std::vector<float>& points, const std::vector<int>& facets,
                                  const bool parallel = true)
{
        const std::size_t vcount = points.size() / N;
        const std::size_t fcount = facets.size() / N;
        std::vector<Vec<N, double>> fn(fcount);
        std::vector<double> weight(fcount * N, 1.0);
        ranges(
                parallel, fcount,
                [&](const std::size_t begin, const std::size_t end)
                {
                        for (std::size_t f = begin; f < end; ++f)
                        {
                                Vec<N, double> e[N - 1];
                                const int i0 = facets[f * N];
                                for (int k = 0; k < N - 1; ++k)
                                {
                                        for (int d = 0; d < N; ++d)
                                        {
                                                e[k][d] = static_cast<double>(
                                                                  points[facets[f * N + k + 1] * static_cast<std::size_t>(N) + d]) -
                                                          static_cast<double>(points[i0 * static_cast<std::size_t>(N) + d]);
                                        }
                                }
                                fn[f] = orthogonal_complement(e).normalized();
                                if constexpr (N == 3 || N == 4)
                                {
                                        // normals.cpp:46-72: the corner's edges in the facet's
                                        // cyclic order from the corner
                                        for (int k = 0; k < N; ++k)
                                        {
                                                const int v = facets[f * N + k];
                                                Vec<N, double> a[N - 1];
                                                for (int j = 0; j < N - 1; ++j)
                                                {
                                                        const int o = facets[f * N + (k + 1 + j) % N];
                                                        for (int d = 0; d < N; ++d)
                                                        {
                                                                a[j][d] = static_cast<double>(points[o * static_cast<std::size_t>(N) + d]) -
                                                                          static_cast<double>(points[v * static_cast<std::size_t>(N) + d]);
                                                        }
                                                }
                                                weight[f * N + k] = corner_weight<N>(a);
                                        }
                                }
                        }
                });
        // the corners of every vertex in facet order, then each vertex's sum in
        // that order (the vertices in parallel).  The corner lists are built by
        // parts of the facets: each part counts its corners per vertex, and a
        // vertex's corners from part k follow those from parts before k.
        const std::size_t corner_count = fcount * N;
        const unsigned parts = parallel ? std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(),
                                                                          static_cast<unsigned>(corner_count / 16384)))
                                        : 1u;
        const std::size_t step = (corner_count + parts - 1) / parts;
        std::vector<std::vector<int>> part_count(parts, std::vector<int>(vcount, 0));
        const auto each_part = [&](const auto& f)
        {
                if (parts == 1)
                {
                        f(0u);
                        return;
                }
                std::vector<std::thread> pool;
                for (unsigned k = 1; k < parts; ++k)
                {
                        pool.emplace_back([&f, k] { f(k); });
                }
                f(0u);
                for (std::thread& t : pool)
                {
                        t.join();
                }
        };
        each_part(
                [&](const unsigned k)
                {
                        std::vector<int>& count = part_count[k];
                        const std::size_t e = std::min(corner_count, (k + 1) * step);
                        for (std::size_t c = k * step; c < e; ++c)
                        {
                                ++count[facets[c]];
                        }
                });
        std::vector<int> first(vcount + 1, 0);
        for (std::size_t v = 0; v < vcount; ++v)
        {
                int offset = first[v];
                for (unsigned k = 0; k < parts; ++k)
                {
                        const int n = part_count[k][v];
                        part_count[k][v] = offset; // where part k's corners of v go
                        offset += n;
                }
                first[v + 1] = offset;
        }
        std::vector<int> corners(corner_count);
        each_part(
                [&](const unsigned k)
                {
                        std::vector<int>& fill = part_count[k];
                        const std::size_t e = std::min(corner_count, (k + 1) * step);
                        for (std::size_t c = k * step; c < e; ++c)
                        {
                                corners[fill[facets[c]]++] = static_cast<int>(c);
                        }
                });
        std::vector<float> out(vcount * N, 0.0f);
        ranges(
                parallel, vcount,
                [&](const std::size_t begin, const std::size_t end)
                {
                        std::vector<int> vicinity_ids;
                        std::vector<Vec<N, double>> vicinity;
                        for (std::size_t v = begin; v < end; ++v)
                        {
                                if (first[v] == first[v + 1])
                                {
                                        continue;
                                }
                                // the vicinity: every vertex of the vertex's facets, in
                                // increasing index (normals.cpp:98-135)
                                vicinity_ids.clear();
                                for (int i = first[v]; i < first[v + 1]; ++i)
                                {
                                        const std::size_t f = static_cast<std::size_t>(corners[i]) / N;
                                        for (int k = 0; k < N; ++k)
                                        {
                                                vicinity_ids.push_back(facets[f * N + k]);
                                        }
                                }
                                std::sort(vicinity_ids.begin(), vicinity_ids.end());
                                vicinity_ids.erase(std::unique(vicinity_ids.begin(), vicinity_ids.end()),
                                                   vicinity_ids.end());
                                if (vicinity_ids.size() < static_cast<std::size_t>(N))
                                {
                                        throw std::runtime_error("Vertex has " + std::to_string(vicinity_ids.size()) +
                                                                 " vertices in its vicinity, required minimum is " +
                                                                 std::to_string(N) + " vertices");
                                }
                                vicinity.resize(vicinity_ids.size());
                                for (std::size_t i = 0; i < vicinity_ids.size(); ++i)
                                {
                                        for (int d = 0; d < N; ++d)
                                        {
                                                vicinity[i][d] = static_cast<double>(
                                                        points[static_cast<std::size_t>(vicinity_ids[i]) * N + d]);
                                        }
                                }
                                const Vec<N, double> reference = point_normal<N>(vicinity);
                                Vec<N, double> sum = Vec<N, double>::filled(0);
                                for (int i = first[v]; i < first[v + 1]; ++i)
                                {
                                        const std::size_t c = static_cast<std::size_t>(corners[i]);
                                        const Vec<N, double>& n = fn[c / N];
                                        const Vec<N, double> wn = n * weight[c];
                                        if (dot(n, reference) >= 0)
                                        {
                                                sum = sum + wn;
                                        }
                                        else
                                        {
                                                sum = sum - wn;
                                        }
                                }
                                const Vec<N, double> n = sum.normalized();
                                for (int d = 0; d < N; ++d)
                                {
                                        out[v * N + d] = static_cast<float>(n[d]);
                                }
                        }
                },
                512);
        return out;
}

// ---------------------------------------------------------------------------

// Builds the BVH of `count` facets (global vertex indices `facets`, N per
// facet, into `vertices`) on the GPU (bvh_device.cuh); returns the node
// count.  nodes: depth-first records, interior offsets and leaf index slots
// local to the mesh; indices: the facet of every leaf slot.
template <int N, typename T>
int build_device_bvh(
        const double* vertices,
        const int* facets,
        const int count,
        const double* uniform_sums,
        const T interior_cost,
        DeviceArray<BvhNode<N, T>>& nodes,
        DeviceArray<std::uint32_t>& indices)
{
        using K = typename BvhKey<T>::K;
        if (count <= 0)
        {
                throw std::runtime_error("No objects to build BVH");
        }
        const int task_capacity = count / (BVH_SMALL + 1) + 1;
        const int chunk_capacity = count / BVH_CHUNK + task_capacity + 1;
        DeviceArray<BvhObject<N, T>> objects;
        objects.allocate(count);
        DeviceArray<unsigned char> buckets;
        buckets.allocate(count);
        DeviceArray<int> first;
        first.allocate(count);
        DeviceArray<int> second;
        second.allocate(count);
        DeviceArray<BvhBuildNode<N, T>> leaves;
        leaves.allocate(count);
        DeviceArray<BvhBuildNode<N, T>> inner;
        inner.allocate(count);
        DeviceArray<int> leaf_list;
        leaf_list.allocate(count);
        DeviceArray<int> inner_list;
        inner_list.allocate(count);
        DeviceArray<BvhTask<N, T>> tasks[2];
        DeviceArray<BvhChunk> chunks[2];
        for (int i = 0; i < 2; ++i)
        {
                tasks[i].allocate(task_capacity);
                chunks[i].allocate(chunk_capacity);
        }
        DeviceArray<int2> chunk_counts;
        chunk_counts.allocate(chunk_capacity);
        DeviceArray<int2> chunk_offsets;
        chunk_offsets.allocate(chunk_capacity);
        DeviceArray<BvhSmallTask<N, T>> small;
        small.allocate(count);
        DeviceArray<BvhCounters> counters;
        counters.allocate(1);
        DeviceArray<K> root_keys;
        root_keys.allocate(2 * N);

        NBPT_CUDA(cudaMemset(counters.get(), 0, sizeof(BvhCounters)));
        NBPT_CUDA(cudaMemset(root_keys.get(), 0xff, N * sizeof(K)));
        NBPT_CUDA(cudaMemset(root_keys.get() + N, 0, N * sizeof(K)));
        bvh_objects_kernel<N, T><<<blocks_for(count, 256), 256>>>(vertices, facets, count, objects.get(), root_keys.get());
        NBPT_CUDA(cudaGetLastError());
        bvh_root_kernel<N, T><<<1, 1>>>(count, root_keys.get(), tasks[0].get(), chunks[0].get(), small.get(),
                                          counters.get());
        NBPT_CUDA(cudaGetLastError());
        BvhCounters h{};
        NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
        int cur = 0;
        while (h.tasks > 0)
        {
                const int task_count = h.tasks;
                const int chunk_count = h.chunks;
                if (task_count > task_capacity || chunk_count > chunk_capacity)
                {
                        throw std::runtime_error("BVH build: level larger than its buffers");
                }
                BvhTask<N, T>* const t = tasks[cur].get();
                const BvhChunk* const c = chunks[cur].get();
                bvh_center_kernel<N, T><<<chunk_count, BVH_THREADS>>>(t, c, objects.get());
                bvh_bin_kernel<N, T><<<chunk_count, BVH_THREADS>>>(t, c, objects.get(), buckets.get());
                NBPT_CUDA(cudaMemset(counters.get(), 0, 2 * sizeof(int))); // next level: tasks, chunks
                bvh_split_kernel<N, T><<<blocks_for(task_count, 128), 128>>>(
                        t, task_count, uniform_sums, interior_cost, tasks[1 - cur].get(), chunks[1 - cur].get(),
                        small.get(), leaves.get(), inner.get(), leaf_list.get(), inner_list.get(), counters.get());
                bvh_misplaced_kernel<N, T><<<chunk_count, BVH_THREADS>>>(
                        t, c, buckets.get(), chunk_counts.get(), nullptr, first.get(), second.get());
                bvh_offsets_kernel<N, T><<<blocks_for(task_count, 128), 128>>>(
                        t, task_count, chunk_counts.get(), chunk_offsets.get(), counters.get());
                bvh_misplaced_kernel<N, T><<<chunk_count, BVH_THREADS>>>(
                        t, c, buckets.get(), chunk_counts.get(), chunk_offsets.get(), first.get(), second.get());
                bvh_swap_kernel<N, T><<<chunk_count, BVH_THREADS>>>(t, c, first.get(), second.get(), objects.get());
                NBPT_CUDA(cudaGetLastError());
                NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
                if (h.error)
                {
                        break;
                }
                cur = 1 - cur;
        }
        if (h.small > 0 && !h.error)
        {
                bvh_small_kernel<N, T><<<(h.small + 3) / 4, 128>>>(
                        small.get(), h.small, uniform_sums, interior_cost, objects.get(), leaves.get(), inner.get(),
                        leaf_list.get(), inner_list.get(), counters.get());
                NBPT_CUDA(cudaGetLastError());
                NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
        }
        if (h.error == 2)
        {
                throw std::runtime_error("BVH leaf too large");
        }
        if (h.error)
        {
                throw std::runtime_error("BVH split produced an empty side");
        }
        bvh_sizes_kernel<N, T><<<blocks_for(h.leaves, 128), 128>>>(leaf_list.get(), h.leaves, leaves.get(), inner.get(),
                                                                    counters.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
        if (h.root_size != h.leaves + h.inner)
        {
                throw std::runtime_error("BVH build: the tree does not reach every node");
        }
        bvh_preorder_kernel<N, T><<<blocks_for(h.leaves + h.inner, 128), 128>>>(
                leaf_list.get(), h.leaves, inner_list.get(), h.inner, leaves.get(), inner.get(), counters.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
        if (h.depth > host::BVH_MAX_DEPTH)
        {
                throw std::runtime_error("BVH depth " + std::to_string(h.depth) + " exceeds the traversal stack of " +
                                         std::to_string(host::BVH_MAX_DEPTH) + " entries (a degenerate mesh)");
        }
        const int node_count = h.leaves + h.inner;
        nodes.allocate(node_count);
        bvh_write_kernel<N, T><<<blocks_for(node_count, 128), 128>>>(
                leaf_list.get(), h.leaves, inner_list.get(), h.inner, leaves.get(), inner.get(), nodes.get(),
                counters.get());
        NBPT_CUDA(cudaGetLastError());
        indices.allocate(count);
        bvh_indices_kernel<N, T><<<blocks_for(count, 256), 256>>>(objects.get(), count, indices.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaMemcpy(&h, counters.get(), sizeof(h), cudaMemcpyDeviceToHost));
        if (h.error)
        {
                throw std::runtime_error("BVH build: a node outside the depth-first order");
        }
        return node_count;
}

template <int N, typename T, int C>
class PainterT;

template <int N, typename T, int C>
class SceneT final : public Scene
{
        friend class PainterT<N, T, C>;

        enum class ShapeKind
        {
                FLAT,
                SOLID,
                MESH
        };

        struct ShapeRef final
        {
                ShapeKind kind;
                int index;
        };

        struct FlatHost final
        {
                Vec<N, T> org;
                Vec<N, T> vectors[N - 1];
        };

        struct MeshObjectHost final
        {
                std::vector<float> points;
                std::vector<int> facets;
                std::array<double, (N + 1) * (N + 1)> matrix;
                std::vector<float> normals;
                float metalness;
                float roughness;
                float alpha;
                float rgb[3];
                // mesh files: the normals are the file's (none: a flat facet),
                // and facets may name materials of their own
                bool file = false;
                std::vector<unsigned char> flat;               // [F]
                std::vector<int> facet_material;               // [F], -1: the object's colour
                std::vector<std::array<float, 3>> colors;      // the file's materials
        };

        struct MeshHost final
        {
                std::vector<T> vertices; // [V][N]
                std::vector<T> normals;  // [V][N] or empty
                std::vector<int> facets;
                std::vector<int> facet_materials;
                std::vector<unsigned char> flat; // [F]: no vertex normals
                int node_count = 0;
                int facet_offset = 0;
                int node_offset = 0;
                int index_offset = 0;
                int vertex_offset = 0;
        };

        std::vector<ShapeRef> shapes_;
        std::vector<FlatShape<N, T>> flat_;
        std::vector<FlatHost> flat_host_;
        std::vector<SolidShape<N, T>> solid_;
        std::vector<Material<T, C>> materials_;
        std::vector<MeshObjectHost> pending_;
        std::vector<MeshHost> meshes_;
        std::vector<Light<N, T, C>> lights_;
        Projector<N, T> projector_{};
        bool has_projector_ = false;
        bool finalized_ = false;
        int bvh_builder_ = 0; // 0: on the GPU, 1: on the host

        DeviceArray<FlatShape<N, T>> d_flat_;
        DeviceArray<SolidShape<N, T>> d_solid_;
        DeviceArray<MeshShape<N, T>> d_meshes_;
        DeviceArray<BvhNode<N, T>> d_nodes_;
        DeviceArray<std::uint32_t> d_indices_;
        DeviceArray<Facet<N, T>> d_facets_;
        DeviceArray<Vec<N, T>> d_normals_;
        DeviceArray<Material<T, C>> d_materials_;
        DeviceArray<Light<N, T, C>> d_lights_;
        DeviceArray<T> d_f1_albedo_;
        DeviceArray<T> d_f1_average_;
        DeviceArray<float> d_cie_; // x, y, z colour matching functions
        std::vector<MeshShape<N, T>> mesh_records_;
        long long facet_total_ = 0;
        long long upload_bytes_ = 0;
        // host seconds of the scene build: mesh ingestion (add_mesh,
        // add_mesh_data), BVH builds, the rest of finalize
        double ingest_seconds_ = 0;
        double bvh_seconds_ = 0;
        double finalize_seconds_ = 0;
        long long node_total_ = 0;

        DeviceScene<N, T, C> device_{};
        // channel-0 view of the materials and lights, for tracing paths with
        // one colour channel (tape.cuh)
        DeviceArray<Material<T, 1>> d_materials_1_;
        DeviceArray<Light<N, T, 1>> d_lights_1_;
        DeviceScene<N, T, 1> device_1_{};

        void check_open() const
        {
                if (finalized_)
                {
                        throw std::runtime_error("the scene is finalized");
                }
        }

        int add_material(const std::vector<float>& color, const float metalness, const T roughness)
        {
                std::vector<float> f0;
                std::vector<float> rho;
                host::metalness_colors(color, metalness, f0, rho);
                Material<T, C> m;
                m.roughness = roughness;
                for (int c = 0; c < C; ++c)
                {
                        m.f0.c[c] = f0[c];
                        m.rho_ss.c[c] = rho[c];
                }
                materials_.push_back(m);
                return static_cast<int>(materials_.size()) - 1;
        }

        static T clamp_t(const T v)
        {
                return (v < T(0)) ? T(0) : ((T(1) < v) ? T(1) : v);
        }

        std::vector<float> clamped_surface_color(const float* rgb) const
        {
                std::vector<float> c = host::surface_color(C, rgb);
                for (float& v : c)
                {
                        v = host::clamp01(v);
                }
                return c;
        }

        Vec<N, T> box_lo(const Vec<N, T>* pts, const int count) const
        {
                Vec<N, T> r = pts[0];
                for (int k = 1; k < count; ++k)
                {
                        for (int d = 0; d < N; ++d)
                        {
                                r[d] = (pts[k][d] < r[d]) ? pts[k][d] : r[d];
                        }
                }
                return r;
        }

        Vec<N, T> box_hi(const Vec<N, T>* pts, const int count) const
        {
                Vec<N, T> r = pts[0];
                for (int k = 1; k < count; ++k)
                {
                        for (int d = 0; d < N; ++d)
                        {
                                r[d] = (r[d] < pts[k][d]) ? pts[k][d] : r[d];
                        }
                }
                return r;
        }

public:
        int dimension() const override
        {
                return N;
        }

        int channels() const override
        {
                return C;
        }

        bool double_precision() const override
        {
                return std::is_same_v<T, double>;
        }

        // shapes/hyperplane_parallelotope.cpp:175-188
        int add_hyperplane_parallelotope(
                const double metalness,
                const double roughness,
                const float* rgb,
                const double alpha,
                const double* org,
                const double* vectors) override
        {
                check_open();
                (void)alpha;
                FlatHost h;
                h.org = to_vec<N, T>(org);
                for (int i = 0; i < N - 1; ++i)
                {
                        h.vectors[i] = to_vec<N, T>(vectors + i * N);
                }
                FlatShape<N, T> s;
                if (!s.shape.set(h.org, h.vectors))
                {
                        throw std::runtime_error("hyperplane parallelotope normal is not finite");
                }
                // bounding box of the 2^(N-1) vertices
                Vec<N, T> pts[1 << (N - 1)];
                for (int m = 0; m < (1 << (N - 1)); ++m)
                {
                        Vec<N, T> p = h.org;
                        for (int i = 0; i < N - 1; ++i)
                        {
                                if ((m >> i) & 1)
                                {
                                        p = p + h.vectors[i];
                                }
                        }
                        pts[m] = p;
                }
                const Vec<N, T> lo = box_lo(pts, 1 << (N - 1));
                const Vec<N, T> hi = box_hi(pts, 1 << (N - 1));
                for (int d = 0; d < N; ++d)
                {
                        s.lo[d] = lo[d];
                        s.hi[d] = hi[d];
                }
                const T m = clamp_t(static_cast<T>(metalness));
                s.material = add_material(clamped_surface_color(rgb), static_cast<float>(m),
                                          clamp_t(static_cast<T>(roughness)));
                s.light = -1;
                flat_.push_back(s);
                flat_host_.push_back(h);
                shapes_.push_back({ShapeKind::FLAT, static_cast<int>(flat_.size()) - 1});
                return static_cast<int>(shapes_.size()) - 1;
        }

        // shapes/parallelotope.cpp:174-187
        int add_parallelotope(
                const double metalness,
                const double roughness,
                const float* rgb,
                const double alpha,
                const double* org,
                const double* vectors) override
        {
                check_open();
                (void)alpha;
                const Vec<N, T> o = to_vec<N, T>(org);
                Vec<N, T> v[N];
                for (int i = 0; i < N; ++i)
                {
                        v[i] = to_vec<N, T>(vectors + i * N);
                }
                SolidShape<N, T> s;
                s.shape.set(o, v);
                Vec<N, T> pts[1 << N];
                for (int m = 0; m < (1 << N); ++m)
                {
                        Vec<N, T> p = o;
                        for (int i = 0; i < N; ++i)
                        {
                                if ((m >> i) & 1)
                                {
                                        p = p + v[i];
                                }
                        }
                        pts[m] = p;
                }
                const Vec<N, T> lo = box_lo(pts, 1 << N);
                const Vec<N, T> hi = box_hi(pts, 1 << N);
                for (int d = 0; d < N; ++d)
                {
                        s.lo[d] = lo[d];
                        s.hi[d] = hi[d];
                }
                const T m = clamp_t(static_cast<T>(metalness));
                s.material = add_material(clamped_surface_color(rgb), static_cast<float>(m),
                                          clamp_t(static_cast<T>(roughness)));
                solid_.push_back(s);
                shapes_.push_back({ShapeKind::SOLID, static_cast<int>(solid_.size()) - 1});
                return static_cast<int>(shapes_.size()) - 1;
        }

        int add_mesh_object(
                const float* points,
                const long long point_count,
                const int* facets,
                const long long facet_count,
                const double* matrix,
                const float* normals,
                const float metalness,
                const float roughness,
                const float* rgb,
                const float alpha) override
        {
                check_open();
                if (point_count <= 0 || facet_count <= 0)
                {
                        throw std::runtime_error("No facets for facet object");
                }
                MeshObjectHost o;
                // only the points the facets use, numbered in the order the
                // facets first reach them (model/mesh/optimize.cpp:48-62,
                // 168-205, which the reference applies to every mesh object)
                std::vector<int> map(point_count, -1);
                int used = 0;
                o.facets.resize(facet_count * N);
                for (long long k = 0; k < facet_count * N; ++k)
                {
                        const int i = facets[k];
                        if (i < 0 || i >= point_count)
                        {
                                throw std::runtime_error("facet vertex index out of range");
                        }
                        if (map[i] < 0)
                        {
                                map[i] = used++;
                        }
                        o.facets[k] = map[i];
                }
                o.points.resize(static_cast<std::size_t>(used) * N);
                if (normals)
                {
                        o.normals.resize(static_cast<std::size_t>(used) * N);
                }
                for (long long i = 0; i < point_count; ++i)
                {
                        if (map[i] < 0)
                        {
                                continue;
                        }
                        for (int d = 0; d < N; ++d)
                        {
                                o.points[static_cast<std::size_t>(map[i]) * N + d] = points[i * N + d];
                                if (normals)
                                {
                                        o.normals[static_cast<std::size_t>(map[i]) * N + d] = normals[i * N + d];
                                }
                        }
                }
                std::copy(matrix, matrix + (N + 1) * (N + 1), o.matrix.begin());
                o.metalness = metalness;
                o.roughness = roughness;
                o.alpha = alpha;
                std::copy(rgb, rgb + 3, o.rgb);
                pending_.push_back(std::move(o));
                return static_cast<int>(pending_.size()) - 1;
        }

        // A mesh object read from an OBJ or STL file (model/mesh/file.cpp:86-104):
        // every distinct (vertex, normal) corner of its facets becomes a point,
        // numbered by first use; facets without normals are flat.
        int add_mesh_file(
                const char* path,
                const double* matrix,
                const float metalness,
                const float roughness,
                const float* rgb,
                const float alpha) override
        {
                check_open();
                const host::MeshFile file = host::load_mesh_file(path, N);
                MeshObjectHost o;
                o.file = true;
                const std::size_t facet_count = file.has_normal.size();
                const long long normal_slots = static_cast<long long>(file.normals.size() / N) + 1;
                // the first corner of each vertex in a table, the others in a map
                const std::size_t vertex_count = file.vertices.size() / N;
                std::vector<int> first_normal(vertex_count, -2);
                std::vector<int> first_id(vertex_count, -1);
                std::unordered_map<long long, int> other;
                o.facets.resize(facet_count * N);
                const auto new_point = [&](const int v, const int nm)
                {
                        const int id = static_cast<int>(o.points.size() / N);
                        for (int d = 0; d < N; ++d)
                        {
                                o.points.push_back(file.vertices[static_cast<std::size_t>(v) * N + d]);
                                o.normals.push_back(nm < 0 ? 0.0f : file.normals[static_cast<std::size_t>(nm) * N + d]);
                        }
                        return id;
                };
                for (std::size_t f = 0; f < facet_count; ++f)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                const int v = file.facet_vertices[f * N + k];
                                const int nm = file.has_normal[f] ? file.facet_normals[f * N + k] : -1;
                                int id;
                                if (first_normal[v] == -2)
                                {
                                        first_normal[v] = nm;
                                        id = first_id[v] = new_point(v, nm);
                                }
                                else if (first_normal[v] == nm)
                                {
                                        id = first_id[v];
                                }
                                else
                                {
                                        const long long key = static_cast<long long>(v) * normal_slots + (nm + 1);
                                        const auto it = other.find(key);
                                        if (it != other.end())
                                        {
                                                id = it->second;
                                        }
                                        else
                                        {
                                                id = new_point(v, nm);
                                                other.emplace(key, id);
                                        }
                                }
                                o.facets[f * N + k] = id;
                        }
                }
                o.flat.resize(facet_count);
                for (std::size_t f = 0; f < facet_count; ++f)
                {
                        o.flat[f] = file.has_normal[f] ? 0 : 1;
                }
                o.facet_material = file.facet_material;
                o.colors = file.material_colors;
                std::copy(matrix, matrix + (N + 1) * (N + 1), o.matrix.begin());
                o.metalness = metalness;
                o.roughness = roughness;
                o.alpha = alpha;
                std::copy(rgb, rgb + 3, o.rgb);
                pending_.push_back(std::move(o));
                return static_cast<int>(pending_.size()) - 1;
        }

        // shapes/mesh/data.cpp:88-310: transform the objects' vertices and
        // normals, one material per object
        int add_mesh() override
        {
                check_open();
                const Stopwatch watch(ingest_seconds_);
                if (pending_.empty())
                {
                        throw std::runtime_error("No objects to paint");
                }
                // objects in order: offsets and materials; then every object's
                // normals and transforms, the objects shared out among the host
                // threads when there are many, each object's work shared out
                // when there are few
                MeshHost mesh;
                std::vector<MeshObjectHost*> objects;
                std::vector<std::size_t> vertex_base;
                std::vector<std::size_t> facet_base;
                std::vector<int> materials;            // the object's colour
                std::vector<std::vector<int>> file_materials; // the file's materials
                std::size_t vertex_total = 0;
                std::size_t facet_total = 0;
                for (MeshObjectHost& o : pending_)
                {
                        const T alpha = clamp_t(static_cast<T>(o.alpha));
                        if (alpha == 0)
                        {
                                continue;
                        }
                        objects.push_back(&o);
                        vertex_base.push_back(vertex_total);
                        facet_base.push_back(facet_total);
                        vertex_total += o.points.size() / N;
                        facet_total += o.facets.size() / N;
                        const auto color_of = [&](const float* rgb)
                        {
                                std::vector<float> c = host::surface_color(C, rgb);
                                for (float& x : c)
                                {
                                        x = host::clamp01(x);
                                }
                                return c;
                        };
                        const float metalness = static_cast<float>(clamp_t(static_cast<T>(o.metalness)));
                        const T roughness = clamp_t(static_cast<T>(o.roughness));
                        // the file's materials, then the object's colour
                        // (shapes/mesh/data.cpp:113-161)
                        std::vector<int> own;
                        for (const std::array<float, 3>& c : o.colors)
                        {
                                own.push_back(add_material(color_of(c.data()), metalness, roughness));
                        }
                        file_materials.push_back(std::move(own));
                        materials.push_back(add_material(color_of(o.rgb), metalness, roughness));
                }
                mesh.vertices.resize(vertex_total * N);
                mesh.normals.resize(vertex_total * N);
                mesh.facets.resize(facet_total * N);
                mesh.facet_materials.resize(facet_total);
                mesh.flat.assign(facet_total, 0);
                const bool per_object = objects.size() >= 4;
                const auto ingest = [&](const std::size_t k)
                {
                        MeshObjectHost& o = *objects[k];
                        const bool inner_parallel = !per_object;
                        const std::size_t vcount = o.points.size() / N;
                        if (o.normals.empty() && !o.file)
                        {
                                o.normals = vertex_normals<N>(o.points, o.facets, inner_parallel);
                        }
                        // vertices: M * (v, 1)  (numerical/transform.h:83-119)
                        const std::size_t vbase = vertex_base[k] * N;
                        ranges(
                                inner_parallel, vcount,
                                [&](const std::size_t begin, const std::size_t end)
                                {
                                        for (std::size_t v = begin; v < end; ++v)
                                        {
                                                for (int r = 0; r < N; ++r)
                                                {
                                                        T x = static_cast<T>(o.matrix[r * (N + 1) + 0]) *
                                                              static_cast<T>(o.points[v * N + 0]);
                                                        for (int c = 1; c < N; ++c)
                                                        {
                                                                x += static_cast<T>(o.matrix[r * (N + 1) + c]) *
                                                                     static_cast<T>(o.points[v * N + c]);
                                                        }
                                                        x += static_cast<T>(o.matrix[r * (N + 1) + N]);
                                                        mesh.vertices[vbase + v * N + r] = x;
                                                }
                                        }
                                });
                        // normals: inverse transpose of the linear part
                        std::array<T, N * N> lin;
                        for (int r = 0; r < N; ++r)
                        {
                                for (int c = 0; c < N; ++c)
                                {
                                        lin[r * N + c] = static_cast<T>(o.matrix[r * (N + 1) + c]);
                                }
                        }
                        const std::array<T, N * N> inv = inverse<N, T>(lin);
                        ranges(
                                inner_parallel, vcount,
                                [&](const std::size_t begin, const std::size_t end)
                                {
                                        for (std::size_t v = begin; v < end; ++v)
                                        {
                                                for (int r = 0; r < N; ++r)
                                                {
                                                        // row r of the transpose = column r of the inverse
                                                        T x = inv[0 * N + r] * static_cast<T>(o.normals[v * N + 0]);
                                                        for (int c = 1; c < N; ++c)
                                                        {
                                                                x += inv[c * N + r] * static_cast<T>(o.normals[v * N + c]);
                                                        }
                                                        mesh.normals[vbase + v * N + r] = x;
                                                }
                                        }
                                });
                        const std::size_t fbase = facet_base[k];
                        const int vertex_offset = static_cast<int>(vertex_base[k]);
                        for (std::size_t i = 0; i < o.facets.size(); ++i)
                        {
                                mesh.facets[fbase * N + i] = o.facets[i] + vertex_offset;
                        }
                        const std::size_t fcount = o.facets.size() / N;
                        for (std::size_t f = 0; f < fcount; ++f)
                        {
                                const int own = o.facet_material.empty() ? -1 : o.facet_material[f];
                                mesh.facet_materials[fbase + f] = own < 0 ? materials[k] : file_materials[k][own];
                                mesh.flat[fbase + f] = o.flat.empty() ? 0 : o.flat[f];
                        }
                };
                if (per_object)
                {
                        parallel_items(objects.size(), ingest);
                }
                else
                {
                        for (std::size_t k = 0; k < objects.size(); ++k)
                        {
                                ingest(k);
                        }
                }
                pending_.clear();
                if (mesh.facets.empty())
                {
                        throw std::runtime_error("No facets found in meshes");
                }
                meshes_.push_back(std::move(mesh));
                shapes_.push_back({ShapeKind::MESH, static_cast<int>(meshes_.size()) - 1});
                return static_cast<int>(shapes_.size()) - 1;
        }

        // A mesh given as the painter's mesh data (shapes/mesh/data.h:34-50):
        // transformed vertices and normals, facet vertex indices, per-facet
        // material index; material_params [metalness, roughness, alpha] and
        // material_colors [C] per material.
        int add_mesh_data(
                const long long vertex_count,
                const double* vertices,
                const double* normals,
                const long long facet_count,
                const int* facets,
                const int* facet_materials,
                const int material_count,
                const double* material_params,
                const float* material_colors) override
        {
                check_open();
                const Stopwatch watch(ingest_seconds_);
                if (facet_count <= 0)
                {
                        throw std::runtime_error("No facets found in meshes");
                }
                MeshHost mesh;
                mesh.vertices.resize(vertex_count * N);
                for (long long i = 0; i < vertex_count * N; ++i)
                {
                        mesh.vertices[i] = static_cast<T>(vertices[i]);
                }
                if (normals)
                {
                        mesh.normals.resize(vertex_count * N);
                        for (long long i = 0; i < vertex_count * N; ++i)
                        {
                                mesh.normals[i] = static_cast<T>(normals[i]);
                        }
                }
                const int base = static_cast<int>(materials_.size());
                for (int m = 0; m < material_count; ++m)
                {
                        std::vector<float> color(material_colors + m * C, material_colors + (m + 1) * C);
                        add_material(color, static_cast<float>(static_cast<T>(material_params[m * 3 + 0])),
                                     static_cast<T>(material_params[m * 3 + 1]));
                }
                mesh.facets.assign(facets, facets + facet_count * N);
                for (const int i : mesh.facets)
                {
                        if (i < 0 || i >= vertex_count)
                        {
                                throw std::runtime_error("facet vertex index out of range");
                        }
                }
                mesh.facet_materials.resize(facet_count);
                for (long long f = 0; f < facet_count; ++f)
                {
                        if (facet_materials[f] < 0 || facet_materials[f] >= material_count)
                        {
                                throw std::runtime_error("facet material index out of range");
                        }
                        mesh.facet_materials[f] = base + facet_materials[f];
                }
                meshes_.push_back(std::move(mesh));
                shapes_.push_back({ShapeKind::MESH, static_cast<int>(meshes_.size()) - 1});
                return static_cast<int>(shapes_.size()) - 1;
        }

        // lights/parallelotope_light.cpp:183-193 (normal turned towards
        // `direction`, pdf 1 / area)
        int add_parallelotope_light(const int shape, const double* direction, const float* rgb) override
        {
                check_open();
                if (shape < 0 || shape >= static_cast<int>(shapes_.size()) || shapes_[shape].kind != ShapeKind::FLAT)
                {
                        throw std::runtime_error("light carrier is not a hyperplane parallelotope");
                }
                const int fi = shapes_[shape].index;
                const FlatHost& h = flat_host_[fi];
                Light<N, T, C> l{};
                l.type = static_cast<int>(LightType::PARALLELOTOPE);
                l.org = h.org;
                for (int i = 0; i < N - 1; ++i)
                {
                        l.vectors[i] = h.vectors[i];
                }
                l.normal = flat_[fi].shape.plane.n;
                const Vec<N, T> dir = to_vec<N, T>(direction);
                if (dot(l.normal, dir) < 0)
                {
                        l.normal = -l.normal;
                }
                Vec<N, T> vv[N - 1];
                for (int i = 0; i < N - 1; ++i)
                {
                        vv[i] = h.vectors[i];
                }
                l.pdf = 1 / orthogonal_complement(vv).norm();
                const std::vector<float> rad = host::illuminant_color(C, rgb);
                for (int c = 0; c < C; ++c)
                {
                        l.radiance.c[c] = rad[c];
                }
                l.shape = fi;
                lights_.push_back(l);
                flat_[fi].light = static_cast<int>(lights_.size()) - 1;
                return static_cast<int>(lights_.size()) - 1;
        }

        // lights/ball_light.cpp:181-202
        int add_ball_light(const double* center, const double* direction, const double radius, const float* rgb) override
        {
                check_open();
                const T r = static_cast<T>(radius);
                if (!(r > 0))
                {
                        throw std::runtime_error("Ball light radius must be positive");
                }
                Light<N, T, C> l{};
                l.type = static_cast<int>(LightType::BALL);
                l.org = to_vec<N, T>(center);
                l.normal = to_vec<N, T>(direction).normalized();
                orthogonal_complement_of_unit_vector(l.normal, l.vectors);
                for (int i = 0; i < N - 1; ++i)
                {
                        for (int d = 0; d < N; ++d)
                        {
                                l.vectors[i][d] *= r;
                        }
                }
                const T pdf_unit = static_cast<T>(1 / host::ball_volume(N - 1));
                l.pdf = pdf_unit / power<N - 1>(r);
                l.radius_squared = square(r);
                const std::vector<float> rad = host::illuminant_color(C, rgb);
                for (int c = 0; c < C; ++c)
                {
                        l.radiance.c[c] = rad[c];
                }
                lights_.push_back(l);
                return static_cast<int>(lights_.size()) - 1;
        }

        // projectors/perspective_projector.cpp:37-90
        void set_perspective_projector(
                const double* org,
                const double* dir,
                const double* axes,
                const double fov_degrees,
                const int* size) override
        {
                check_open();
                const T fov = static_cast<T>(fov_degrees);
                if (!(fov > 0 && fov < 180))
                {
                        throw std::runtime_error("Perspective projection: error view angle");
                }
                Projector<N, T> p{};
                p.type = static_cast<int>(ProjectorType::PERSPECTIVE);
                p.org = to_vec<N, T>(org);
                for (int i = 0; i < N - 1; ++i)
                {
                        if (size[i] < 1)
                        {
                                throw std::runtime_error("Screen size is not positive");
                        }
                        p.size[i] = size[i];
                        p.axes[i] = to_vec<N, T>(axes + i * N).normalized();
                        p.screen_org[i] = static_cast<T>(-size[i]) * (static_cast<T>(1) / 2);
                }
                const T pi = static_cast<T>(host::PI_L);
                const T half_angle = (fov * T(0.5)) * (pi / 180);
                const T dir_length = static_cast<T>(size[0]) * T(0.5) * std::tan(pi / 2 - half_angle);
                p.dir = to_vec<N, T>(dir).normalized() * dir_length;
                projector_ = p;
                has_projector_ = true;
        }

        // projectors/parallel_projector.cpp:35-88
        void set_parallel_projector(
                const double* org,
                const double* dir,
                const double* axes,
                const double units_per_pixel,
                const int* size) override
        {
                check_open();
                const T u = static_cast<T>(units_per_pixel);
                if (!(u > 0))
                {
                        throw std::runtime_error("Error units per pixel for parallel projection");
                }
                Projector<N, T> p{};
                p.type = static_cast<int>(ProjectorType::PARALLEL);
                p.org = to_vec<N, T>(org);
                p.dir = to_vec<N, T>(dir).normalized();
                for (int i = 0; i < N - 1; ++i)
                {
                        if (size[i] < 1)
                        {
                                throw std::runtime_error("Screen size is not positive");
                        }
                        p.size[i] = size[i];
                        p.axes[i] = to_vec<N, T>(axes + i * N).normalized();
                        for (int d = 0; d < N; ++d)
                        {
                                p.axes[i][d] *= u;
                        }
                        p.screen_org[i] = static_cast<T>(-size[i]) * (static_cast<T>(1) / 2);
                }
                projector_ = p;
                has_projector_ = true;
        }

        void set_background(const float* rgb) override
        {
                check_open();
                if (rgb[0] != 0 || rgb[1] != 0 || rgb[2] != 0)
                {
                        throw std::runtime_error(
                                "non-black backgrounds (an infinite area light) are not supported by this painter");
                }
        }

        void set_bvh_builder(const int builder) override
        {
                check_open();
                if (builder != 0 && builder != 1)
                {
                        throw std::runtime_error("BVH builder must be 0 (GPU) or 1 (host)");
                }
                bvh_builder_ = builder;
        }

        void finalize() override
        {
                check_open();
                const Stopwatch watch(finalize_seconds_);
                if (!has_projector_)
                {
                        throw std::runtime_error("no projector");
                }
                if (lights_.empty())
                {
                        throw std::runtime_error("No light sources");
                }
                if (shapes_.empty())
                {
                        throw std::runtime_error("No objects to paint");
                }
                // light distribution: equal power (light_distribution.cpp:36-111)
                {
                        const int count = static_cast<int>(lights_.size());
                        double cumulative = 0;
                        for (int i = 0; i < count; ++i)
                        {
                                const double p = 1.0 / static_cast<double>(count);
                                lights_[i].distribution_pdf = static_cast<T>(p);
                                cumulative += p;
                                lights_[i].cumulative = (i == count - 1) ? 1.0 : cumulative;
                        }
                }

                // meshes: vertices, normals and facets of all meshes in one
                // set of arrays; BVHs built on the GPU (or the host); facet
                // records set up on the GPU
                std::vector<double> all_vertices;
                std::vector<T> all_normals;
                std::vector<int> all_facets;
                std::vector<int> all_materials;
                std::vector<unsigned char> all_flat;
                bool any_normals = false;
                bool any_flat = false;
                std::size_t max_facets = 0;
                for (const MeshHost& m : meshes_)
                {
                        any_normals = any_normals || !m.normals.empty();
                        any_flat = any_flat || std::find(m.flat.begin(), m.flat.end(), 1) != m.flat.end();
                        max_facets = std::max(max_facets, m.facets.size() / N);
                }
                {
                        std::size_t vertex_total = 0;
                        std::size_t facet_total = 0;
                        for (MeshHost& m : meshes_)
                        {
                                m.facet_offset = static_cast<int>(facet_total);
                                m.index_offset = static_cast<int>(facet_total);
                                m.vertex_offset = static_cast<int>(vertex_total);
                                vertex_total += m.vertices.size() / N;
                                facet_total += m.facets.size() / N;
                        }
                        all_vertices.resize(vertex_total * N);
                        all_facets.resize(facet_total * N);
                        all_materials.resize(facet_total);
                        if (any_flat)
                        {
                                all_flat.assign(facet_total, 0);
                        }
                        if (any_normals)
                        {
                                all_normals.assign(vertex_total * N, T(0));
                        }
                        for (const MeshHost& m : meshes_)
                        {
                                const std::size_t vo = static_cast<std::size_t>(m.vertex_offset) * N;
                                const std::size_t fo = static_cast<std::size_t>(m.facet_offset) * N;
                                parallel_ranges(
                                        m.vertices.size(),
                                        [&](const std::size_t b, const std::size_t e)
                                        {
                                                for (std::size_t i = b; i < e; ++i)
                                                {
                                                        all_vertices[vo + i] = static_cast<double>(m.vertices[i]);
                                                }
                                        });
                                if (!m.normals.empty())
                                {
                                        std::copy(m.normals.begin(), m.normals.end(), all_normals.begin() + vo);
                                }
                                parallel_ranges(
                                        m.facets.size(),
                                        [&](const std::size_t b, const std::size_t e)
                                        {
                                                for (std::size_t i = b; i < e; ++i)
                                                {
                                                        all_facets[fo + i] = m.facets[i] + m.vertex_offset;
                                                }
                                        });
                                std::copy(m.facet_materials.begin(), m.facet_materials.end(),
                                          all_materials.begin() + m.facet_offset);
                                if (any_flat && !m.flat.empty())
                                {
                                        std::copy(m.flat.begin(), m.flat.end(), all_flat.begin() + m.facet_offset);
                                }
                        }
                }
                facet_total_ = static_cast<long long>(all_facets.size() / N);

                DeviceArray<double> dv;
                DeviceArray<int> df;
                if (facet_total_ > 0)
                {
                        dv.upload(all_vertices);
                        df.upload(all_facets);
                }

                // BVHs: per mesh, nodes and leaf index slots local to the mesh
                std::vector<std::unique_ptr<DeviceArray<BvhNode<N, T>>>> mesh_nodes;
                std::vector<std::unique_ptr<DeviceArray<std::uint32_t>>> mesh_indices;
                {
                        const Stopwatch bvh_watch(bvh_seconds_);
                        const T facet_cost = static_cast<T>(static_cast<double>(N) / host::SIMPLEX_RATE);
                        const T box_r_cost = static_cast<T>(static_cast<double>(N) / host::BOX_R_RATE);
                        const T interior_cost = static_cast<T>(2 * box_r_cost);
                        DeviceArray<double> uniform_sums;
                        if (bvh_builder_ == 0 && max_facets > 0)
                        {
                                // the running sums of the one facet cost (bvh_build.cpp)
                                std::vector<double> sums(max_facets + 1);
                                sums[0] = 0;
                                sums[1] = facet_cost;
                                for (std::size_t k = 2; k <= max_facets; ++k)
                                {
                                        sums[k] = sums[k - 1] + facet_cost;
                                }
                                uniform_sums.upload(sums);
                        }
                        for (MeshHost& m : meshes_)
                        {
                                const int count = static_cast<int>(m.facets.size() / N);
                                auto nodes = std::make_unique<DeviceArray<BvhNode<N, T>>>();
                                auto indices = std::make_unique<DeviceArray<std::uint32_t>>();
                                if (bvh_builder_ == 0)
                                {
                                        m.node_count = build_device_bvh<N, T>(
                                                dv.get(), df.get() + static_cast<std::size_t>(m.facet_offset) * N, count,
                                                uniform_sums.get(), interior_cost, *nodes, *indices);
                                }
                                else
                                {
                                        const host::BuiltBvh<N, T> bvh = host::build_facet_bvh<N, T>(m.vertices, m.facets);
                                        const std::size_t node_count = bvh.count.size();
                                        std::vector<BvhNode<N, T>> host_nodes(node_count);
                                        for (std::size_t i = 0; i < node_count; ++i)
                                        {
                                                BvhNode<N, T>& b = host_nodes[i];
                                                for (int d = 0; d < N; ++d)
                                                {
                                                        b.lo[d] = bvh.lo[i * N + d];
                                                        b.hi[d] = bvh.hi[i * N + d];
                                                }
                                                b.offset = bvh.offset[i];
                                                b.count = static_cast<std::uint16_t>(bvh.count[i]);
                                                b.axis = static_cast<std::uint16_t>(bvh.axis[i]);
                                                if (bvh.count[i] > 0xffff)
                                                {
                                                        throw std::runtime_error("BVH leaf too large");
                                                }
                                        }
                                        nodes->upload(host_nodes);
                                        indices->upload(bvh.indices);
                                        m.node_count = static_cast<int>(node_count);
                                }
                                mesh_nodes.push_back(std::move(nodes));
                                mesh_indices.push_back(std::move(indices));
                        }
                }
                long long node_total = 0;
                for (MeshHost& m : meshes_)
                {
                        m.node_offset = static_cast<int>(node_total);
                        node_total += m.node_count;
                }
                node_total_ = node_total;
                d_nodes_.allocate(node_total);
                d_indices_.allocate(facet_total_);
                mesh_records_.clear();
                for (std::size_t k = 0; k < meshes_.size(); ++k)
                {
                        const MeshHost& m = meshes_[k];
                        const std::size_t count = m.facets.size() / N;
                        NBPT_CUDA(cudaMemcpy(d_nodes_.get() + m.node_offset, mesh_nodes[k]->get(),
                                             static_cast<std::size_t>(m.node_count) * sizeof(BvhNode<N, T>),
                                             cudaMemcpyDeviceToDevice));
                        NBPT_CUDA(cudaMemcpy(d_indices_.get() + m.index_offset, mesh_indices[k]->get(),
                                             count * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice));
                        BvhNode<N, T> root;
                        NBPT_CUDA(cudaMemcpy(&root, mesh_nodes[k]->get(), sizeof(root), cudaMemcpyDeviceToHost));
                        MeshShape<N, T> rec;
                        for (int d = 0; d < N; ++d)
                        {
                                rec.lo[d] = root.lo[d];
                                rec.hi[d] = root.hi[d];
                        }
                        rec.node_offset = m.node_offset;
                        rec.index_offset = m.index_offset;
                        rec.facet_offset = m.facet_offset;
                        mesh_records_.push_back(rec);
                }
                mesh_nodes.clear();
                mesh_indices.clear();

                d_flat_.upload(flat_);
                d_solid_.upload(solid_);
                d_meshes_.upload(mesh_records_);
                d_materials_.upload(materials_);
                d_lights_.upload(lights_);
                upload_bytes_ = static_cast<long long>(d_flat_.bytes() + d_solid_.bytes() + d_meshes_.bytes() +
                                                       d_materials_.bytes() + d_lights_.bytes() + dv.bytes() +
                                                       df.bytes());
                if (bvh_builder_ != 0)
                {
                        upload_bytes_ += static_cast<long long>(d_nodes_.bytes() + d_indices_.bytes());
                }

                if (facet_total_ > 0)
                {
                        DeviceArray<double> dn;
                        if (any_normals)
                        {
                                std::vector<double> normals_double(all_normals.begin(), all_normals.end());
                                dn.upload(normals_double);
                        }
                        DeviceArray<int> dm;
                        dm.upload(all_materials);
                        DeviceArray<unsigned char> dflat;
                        if (any_flat)
                        {
                                dflat.upload(all_flat);
                        }
                        DeviceArray<int> derr;
                        std::vector<int> zero(1, 0);
                        derr.upload(zero);
                        upload_bytes_ += static_cast<long long>(dn.bytes() + dm.bytes() + derr.bytes() + dflat.bytes());
                        d_facets_.allocate(facet_total_);
                        facet_setup_kernel<N, T><<<blocks_for(facet_total_, 128), 128>>>(
                                dv.get(), any_normals ? dn.get() : nullptr, any_flat ? dflat.get() : nullptr, df.get(),
                                dm.get(), facet_total_, d_facets_.get(), derr.get());
                        NBPT_CUDA(cudaGetLastError());
                        NBPT_CUDA(cudaDeviceSynchronize());
                        int err = 0;
                        derr.download(&err, 1);
                        if (err)
                        {
                                throw std::runtime_error("Hyperplane simplex normal is not finite");
                        }
                        if (any_normals)
                        {
                                std::vector<Vec<N, T>> nv(all_normals.size() / N);
                                for (std::size_t i = 0; i < nv.size(); ++i)
                                {
                                        for (int d = 0; d < N; ++d)
                                        {
                                                nv[i][d] = all_normals[i * N + d];
                                        }
                                }
                                d_normals_.upload(nv);
                                upload_bytes_ += static_cast<long long>(d_normals_.bytes());
                        }
                }

                // shading constants and tables
                std::vector<T> f1(1024);
                std::vector<T> f1a(32);
                for (int i = 0; i < 1024; ++i)
                {
                        if constexpr (std::is_same_v<T, double>)
                        {
                                f1[i] = N == 3 ? tables::F1_ALBEDO_3_D[i] : (N == 4 ? tables::F1_ALBEDO_4_D[i] : tables::F1_ALBEDO_5_D[i]);
                        }
                        else
                        {
                                f1[i] = N == 3 ? tables::F1_ALBEDO_3_F[i] : (N == 4 ? tables::F1_ALBEDO_4_F[i] : tables::F1_ALBEDO_5_F[i]);
                        }
                }
                for (int i = 0; i < 32; ++i)
                {
                        if constexpr (std::is_same_v<T, double>)
                        {
                                f1a[i] = N == 3 ? tables::F1_AVERAGE_3_D[i] : (N == 4 ? tables::F1_AVERAGE_4_D[i] : tables::F1_AVERAGE_5_D[i]);
                        }
                        else
                        {
                                f1a[i] = N == 3 ? tables::F1_AVERAGE_3_F[i] : (N == 4 ? tables::F1_AVERAGE_4_F[i] : tables::F1_AVERAGE_5_F[i]);
                        }
                }
                d_f1_albedo_.upload(f1);
                d_f1_average_.upload(f1a);
                std::vector<float> cie;
                for (int r = 0; r < 3; ++r)
                {
                        const std::vector<float>& row = host::spectrum_row(r);
                        cie.insert(cie.end(), row.begin(), row.end());
                }
                d_cie_.upload(cie);

                device_.flat = d_flat_.get();
                device_.flat_count = static_cast<int>(flat_.size());
                device_.solid = d_solid_.get();
                device_.solid_count = static_cast<int>(solid_.size());
                device_.meshes = d_meshes_.get();
                device_.mesh_count = static_cast<int>(mesh_records_.size());
                device_.nodes = d_nodes_.get();
                device_.indices = d_indices_.get();
                device_.facets = d_facets_.get();
                device_.normals = d_normals_.get();
                device_.materials = d_materials_.get();
                device_.lights = d_lights_.get();
                device_.light_count = static_cast<int>(lights_.size());
                device_.projector = projector_;
                const long double k = host::hemisphere_cosine_integral(N);
                device_.shading.k = static_cast<T>(k);
                device_.shading.k_inv = static_cast<T>(1 / k);
                device_.shading.ball_pdf = static_cast<T>(1 / host::ball_volume(N - 1));
                const std::array<float, 2> fa = host::fresnel_average(N);
                device_.shading.fresnel_a = fa[0];
                device_.shading.fresnel_b = fa[1];
                device_.shading.f1_albedo = d_f1_albedo_.get();
                device_.shading.f1_average = d_f1_average_.get();

                {
                        std::vector<Material<T, 1>> m1(materials_.size());
                        for (std::size_t i = 0; i < materials_.size(); ++i)
                        {
                                m1[i].roughness = materials_[i].roughness;
                                m1[i].f0.c[0] = materials_[i].f0.c[0];
                                m1[i].rho_ss.c[0] = materials_[i].rho_ss.c[0];
                        }
                        std::vector<Light<N, T, 1>> l1(lights_.size());
                        for (std::size_t i = 0; i < lights_.size(); ++i)
                        {
                                const Light<N, T, C>& l = lights_[i];
                                Light<N, T, 1>& o = l1[i];
                                o.type = l.type;
                                o.org = l.org;
                                for (int k = 0; k < N - 1; ++k)
                                {
                                        o.vectors[k] = l.vectors[k];
                                }
                                o.normal = l.normal;
                                o.pdf = l.pdf;
                                o.radiance.c[0] = l.radiance.c[0];
                                o.distribution_pdf = l.distribution_pdf;
                                o.cumulative = l.cumulative;
                                o.shape = l.shape;
                                o.radius_squared = l.radius_squared;
                        }
                        d_materials_1_.upload(m1);
                        d_lights_1_.upload(l1);
                        upload_bytes_ += static_cast<long long>(d_materials_1_.bytes() + d_lights_1_.bytes());
                        device_1_.flat = device_.flat;
                        device_1_.flat_count = device_.flat_count;
                        device_1_.solid = device_.solid;
                        device_1_.solid_count = device_.solid_count;
                        device_1_.meshes = device_.meshes;
                        device_1_.mesh_count = device_.mesh_count;
                        device_1_.nodes = device_.nodes;
                        device_1_.indices = device_.indices;
                        device_1_.facets = device_.facets;
                        device_1_.normals = device_.normals;
                        device_1_.materials = d_materials_1_.get();
                        device_1_.lights = d_lights_1_.get();
                        device_1_.light_count = device_.light_count;
                        device_1_.projector = device_.projector;
                        device_1_.shading = device_.shading;
                }
                finalized_ = true;
        }

        const DeviceScene<N, T, 1>& device_channel_0() const
        {
                device(); // throws if not finalized
                return device_1_;
        }

        const Material<T, C>* device_materials() const
        {
                return d_materials_.get();
        }

        const Light<N, T, C>* device_lights() const
        {
                return d_lights_.get();
        }

        long long pixel_count() const override
        {
                if (!has_projector_)
                {
                        throw std::runtime_error("no projector");
                }
                long long r = 1;
                for (int i = 0; i < N - 1; ++i)
                {
                        r *= projector_.size[i];
                }
                return r;
        }

        // strata per screen dimension (sj_sampler.h:51-73)
        static int strata(const int spp)
        {
                if (spp < 1)
                {
                        throw std::runtime_error("Painter samples per pixel must be greater than 0");
                }
                const double v = std::pow(spp, 1.0 / (N - 1));
                const unsigned f = static_cast<unsigned>(std::floor(v));
                unsigned p = 1;
                for (int i = 0; i < N - 1; ++i)
                {
                        p *= f;
                }
                if (p >= static_cast<unsigned>(spp))
                {
                        return static_cast<int>(f);
                }
                const unsigned c = static_cast<unsigned>(std::ceil(v));
                return static_cast<int>(c);
        }

        int actual_spp(const int spp) const override
        {
                const int k = strata(spp);
                int r = 1;
                for (int i = 0; i < N - 1; ++i)
                {
                        r *= k;
                }
                return r;
        }

        void build_seconds(double* out) const override
        {
                out[0] = ingest_seconds_;
                out[1] = bvh_seconds_;
                out[2] = finalize_seconds_ - bvh_seconds_;
                out[3] = ingest_seconds_ + finalize_seconds_;
        }

        long long upload_bytes() const override
        {
                return upload_bytes_;
        }

        long long device_bytes() const override
        {
                return static_cast<long long>(d_flat_.bytes() + d_solid_.bytes() + d_meshes_.bytes() + d_nodes_.bytes() +
                                              d_indices_.bytes() + d_facets_.bytes() + d_normals_.bytes() +
                                              d_materials_.bytes() + d_lights_.bytes());
        }

        const DeviceScene<N, T, C>& device() const
        {
                if (!finalized_)
                {
                        throw std::runtime_error("the scene is not finalized");
                }
                return device_;
        }

        const float* cie() const
        {
                return d_cie_.get();
        }

        std::unique_ptr<Painter> create_painter(int spp, int max_depth, std::uint32_t seed,
                                                Integrator integrator, int slab_begin, int slab_end,
                                                bool flat_shading, long long chunk_budget, int pixel_sums) override;
        long long painter_bytes(int spp, int max_depth, Integrator integrator, long long chunk_budget,
                                int pixel_sums) const override;

        void trace(const double* rays, long long count, int any, int* kind, int* index, double* t, double* point) override;
        void trace_device(const double* rays, long long count, int any, int* kind, int* index, double* t,
                          double* point) const override;
        void mesh_export(int mesh, long long* counts, double* planes, double* node_lo, double* node_hi,
                         unsigned* node_info, unsigned* indices, int* normal_info) override;

        void ingested_mesh(const int mesh, long long* counts, double* vertices, double* normals,
                           int* facets) const override
        {
                if (mesh < 0 || mesh >= static_cast<int>(meshes_.size()))
                {
                        throw std::runtime_error("no mesh " + std::to_string(mesh));
                }
                const MeshHost& m = meshes_[mesh];
                if (counts)
                {
                        counts[0] = static_cast<long long>(m.vertices.size() / N);
                        counts[1] = static_cast<long long>(m.facets.size() / N);
                        counts[2] = static_cast<long long>(m.normals.size() / N);
                }
                if (vertices)
                {
                        std::copy(m.vertices.begin(), m.vertices.end(), vertices);
                }
                if (normals)
                {
                        std::copy(m.normals.begin(), m.normals.end(), normals);
                }
                if (facets)
                {
                        std::copy(m.facets.begin(), m.facets.end(), facets);
                }
        }
        void brdf(int material, const double* n, const double* v, const double* l, float* f, double* pdf) override;
        void brdf_sample(int material, const double* n, const double* v, const std::uint32_t* seed, int seed_words,
                         double* l, double* pdf, float* f) override;
        void light_sample(int light, int kind, const std::uint32_t* seed, int seed_words, const double* point,
                          double* out, float* radiance) override;
};

// ---------------------------------------------------------------------------
// verification kernels

template <int N, typename T, int C>
__global__ void trace_kernel(
        const DeviceScene<N, T, C> scene,
        const double* __restrict__ rays,
        const long long count,
        const int any,
        int* __restrict__ kind,
        int* __restrict__ index,
        double* __restrict__ t,
        double* __restrict__ point)
{
        const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
        if (i >= count)
        {
                return;
        }
        Vec<N, T> o;
        Vec<N, T> d;
        for (int k = 0; k < N; ++k)
        {
                o[k] = static_cast<T>(rays[i * 2 * N + k]);
                d[k] = static_cast<T>(rays[i * 2 * N + N + k]);
        }
        const Ray<N, T> ray = Ray<N, T>::make(o, d);
        QueryCounters counters{0, 0, 0, 0};
        const SceneQueries<N, T, C> q{scene, counters};
        if (any)
        {
                kind[i] = q.intersect_any(nullptr, ray, infinity<T>()) ? 1 : 0;
                return;
        }
        const Hit<N, T> h = q.intersect(nullptr, ray, infinity<T>());
        kind[i] = h.kind;
        index[i] = h.index;
        t[i] = h ? static_cast<double>(h.distance) : 0.0;
        for (int k = 0; k < N; ++k)
        {
                point[i * N + k] = h ? static_cast<double>(h.point[k]) : 0.0;
        }
}

template <int N, typename T, int C>
__global__ void brdf_kernel(
        const DeviceScene<N, T, C> scene,
        const int material,
        const double* in, // n, v, l
        float* f,
        double* pdf)
{
        const Vec<N, T> n = to_vec<N, T>(in);
        const Vec<N, T> v = to_vec<N, T>(in + N);
        const Vec<N, T> l = to_vec<N, T>(in + 2 * N);
        const Material<T, C>& m = scene.materials[material];
        const Color<C> c = brdf_f(scene.shading, m.roughness, m.f0, m.rho_ss, n, v, l);
        for (int k = 0; k < C; ++k)
        {
                f[k] = c.c[k];
        }
        *pdf = static_cast<double>(brdf_pdf(scene.shading, m.roughness, n, v, l));
}

template <int N, typename T, int C>
__global__ void brdf_sample_kernel(
        const DeviceScene<N, T, C> scene,
        const int material,
        const double* in, // n, v
        const std::uint32_t* seed,
        const int seed_words,
        double* l,
        double* pdf,
        float* f)
{
        const Vec<N, T> n = to_vec<N, T>(in);
        const Vec<N, T> v = to_vec<N, T>(in + N);
        const Material<T, C>& m = scene.materials[material];
        Pcg g = seed_seq_pcg(seed, seed_words);
        const BrdfSample<N, C, T> s = brdf_sample<N>(g, scene.shading, m.roughness, m.f0, m.rho_ss, n, v);
        *pdf = static_cast<double>(s.pdf);
        if (s.pdf > 0)
        {
                for (int k = 0; k < N; ++k)
                {
                        l[k] = static_cast<double>(s.l[k]);
                }
                for (int k = 0; k < C; ++k)
                {
                        f[k] = s.brdf.c[k];
                }
        }
}

// leave (kind 0): out = [org N, dir N, n N, pdf_pos, pdf_dir];
// arrive (kind 1): out = [l N, pdf, distance or -1]
template <int N, typename T, int C>
__global__ void light_sample_kernel(
        const DeviceScene<N, T, C> scene,
        const int light,
        const int kind,
        const std::uint32_t* seed,
        const int seed_words,
        const double* point,
        double* out,
        float* radiance)
{
        Pcg g = seed_seq_pcg(seed, seed_words);
        QueryCounters counters{0, 0, 0, 0};
        const SceneQueries<N, T, C> q{scene, counters};
        const Bpt<N, T, C> b{q, scene, g, 1, nullptr, nullptr};
        const Light<N, T, C>& l = scene.lights[light];
        if (kind == 0)
        {
                const LeaveSample<N, T, C> s = b.leave_sample(l);
                for (int k = 0; k < N; ++k)
                {
                        out[k] = static_cast<double>(s.ray.org[k]);
                        out[N + k] = static_cast<double>(s.ray.dir[k]);
                        out[2 * N + k] = static_cast<double>(s.n[k]);
                }
                out[3 * N] = static_cast<double>(s.pdf_pos);
                out[3 * N + 1] = static_cast<double>(s.pdf_dir);
                for (int c = 0; c < C; ++c)
                {
                        radiance[c] = s.radiance.c[c];
                }
                return;
        }
        const ArriveSample<N, T, C> s = b.arrive_sample(l, to_vec<N, T>(point));
        for (int k = 0; k < N; ++k)
        {
                out[k] = s.pdf > 0 ? static_cast<double>(s.l[k]) : 0.0;
        }
        out[N] = static_cast<double>(s.pdf);
        out[N + 1] = s.pdf > 0 ? static_cast<double>(s.distance) : -1.0;
        for (int c = 0; c < C; ++c)
        {
                radiance[c] = s.pdf > 0 ? s.radiance.c[c] : 0.0f;
        }
}

// ---------------------------------------------------------------------------
// painter: one render of one scene

template <int N, typename T, int C>
class PainterT final : public Painter
{
        const SceneT<N, T, C>* scene_;
        bool flat_shading_;
        long long chunk_budget_; // bytes for the chunk buffers, 0: chunk_budget()
        int spp_request_;
        int spp_;
        int strata_;
        int max_depth_;
        std::uint32_t seed_;
        Integrator integrator_;
        int device_ = 0;
        long long pixels_;      // receiving pixels: the screen, or a slab of it
        long long first_ = 0;   // global index of the first receiving pixel
        long long sources_ = 0; // pixels whose paths a pass renders: the slab and its one-row halo
        long long source_first_ = 0;
        long long pass_ = 0;
        long long passes_done_ = 0;
        cudaStream_t stream_ = nullptr;
        cudaEvent_t ev_start_ = nullptr;
        cudaEvent_t ev_paths_ = nullptr;
        cudaEvent_t ev_paths_end_ = nullptr;
        cudaEvent_t ev_end_ = nullptr;

        DeviceArray<T> offsets_;
        DeviceArray<T> points_;
        DeviceArray<float> colors_;
        DeviceArray<float> lum_;
        DeviceArray<unsigned char> valid_;
        bool double_sums_ = false;
        // set_progress: the callback and one note per chunk enqueued since
        // the last wait (a deque: host callbacks hold pointers to its notes)
        struct ProgressNote
        {
                ProgressCallback callback;
                void* user;
                long long pass;
                long long done;
                long long total;
                std::atomic<long long>* completed;
        };
        ProgressCallback progress_ = nullptr;
        void* progress_user_ = nullptr;
        std::deque<ProgressNote> progress_notes_;
        std::atomic<long long> progress_completed_{0}; // notes whose callback has run, in stream order
        long long progress_dropped_ = 0;              // notes removed from the front of the deque

        static void CUDART_CB progress_host(void* data)
        {
                const ProgressNote* const n = static_cast<const ProgressNote*>(data);
                n->callback(n->user, n->pass, n->done, n->total);
                n->completed->fetch_add(1, std::memory_order_release);
        }

        void note_progress(const std::uint32_t pass, const long long end)
        {
                if (!progress_)
                {
                        return;
                }
                // the notes of callbacks that have run are no longer referenced
                const long long completed = progress_completed_.load(std::memory_order_acquire);
                while (!progress_notes_.empty() && progress_dropped_ < completed)
                {
                        progress_notes_.pop_front();
                        ++progress_dropped_;
                }
                progress_notes_.push_back({progress_, progress_user_, static_cast<long long>(pass) + 1,
                                           end - source_first_, sources_, &progress_completed_});
                NBPT_CUDA(cudaLaunchHostFunc(stream_, &progress_host, &progress_notes_.back()));
        }
        DeviceArray<PixelState<C, float>> state_;    // float sums
        DeviceArray<PixelState<C, double>> state64_; // double sums
        DeviceArray<PathStats> stats_;
        DeviceArray<unsigned> cancel_; // nonzero: the passes take no more paths
        bool scratch_ready_ = false;   // the per-chunk path buffers are allocated
        cudaStream_t cancel_stream_ = nullptr;
        std::mutex cancel_mutex_;
        std::atomic<bool> cancelled_{false};
        DeviceArray<float> rgb_;
        DeviceArray<float> rgba_;
        // per-path buffers of one chunk of pixels: subpath vertices, random
        // stream states, tapes (tape.cuh) and the queued strategies
        int tape_words_ = 0;
        long long chunk_pixels_ = 0;
        DeviceArray<PathVertex<N, T, 1>> vertices_;
        DeviceArray<Pcg> rng_;
        DeviceArray<std::uint32_t> tape_;
        DeviceArray<std::uint32_t> tasks_;
        DeviceArray<unsigned> task_count_;
        DeviceArray<unsigned> next_path_;
        DeviceArray<Arrival<N, T>> arrivals_;
        DeviceArray<PtEstimate> pt_estimates_;
        int connect_blocks_ = 0;
        long long launches_ = 0;
        Statistics statistics_{};

        // Device memory for the per-path buffers of one chunk.  The walk and
        // connect kernels are persistent over a chunk, and every chunk ends in
        // a tail in which the last, longest paths run on an emptying GPU;
        // larger chunks make the tails rarer.  Measured on five jobs of the
        // mixed batch (3/4/5-space, one pass each): 4 -> 16 GiB 1.09-1.41x
        // faster per pass, 4 -> 32 GiB 1.11-1.53x.  A fifth of the device's
        // memory, within [4, 32] GiB (NBPT_CHUNK_BUDGET_GB, when defined, sets
        // it for sweeps).
        static long long chunk_budget()
        {
#ifdef NBPT_CHUNK_BUDGET_GB
                return static_cast<long long>(NBPT_CHUNK_BUDGET_GB) << 30;
#else
                static std::atomic<long long> by_device[64] = {};
                int device = 0;
                if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64)
                {
                        cudaGetLastError();
                        return 4LL << 30;
                }
                long long b = by_device[device].load();
                if (b == 0)
                {
                        std::size_t free = 0;
                        std::size_t total = 0;
                        NBPT_CUDA(cudaMemGetInfo(&free, &total));
                        b = std::min(32LL << 30, std::max(4LL << 30, static_cast<long long>(total / 5)));
                        by_device[device] = b;
                }
                return b;
#endif
        }

        // device bytes of one path's buffers in a chunk (vertices, tape,
        // random stream state, strategy tasks)
        static long long chunk_path_bytes(const int max_depth)
        {
                return static_cast<long long>(tape_words(max_depth)) * 4 +
                       2LL * (max_depth + 1) * sizeof(PathVertex<N, T, 1>) + sizeof(Pcg) +
                       4LL * tape_slot_count(max_depth) + static_cast<long long>(max_depth) * sizeof(Arrival<N, T>);
        }

        // the PT kernel keeps nothing per path; its chunks only bound the
        // 32-bit path counter
        static constexpr long long PT_CHUNK_PATHS = 1LL << 30;

        // budget: bytes for the chunk buffers, 0 for chunk_budget()
        static long long chunk_pixels(const long long pixels, const int spp, const int max_depth,
                                      const Integrator integrator, const long long budget = 0)
        {
                if (integrator == Integrator::PT)
                {
                        return std::max(1LL, std::min(pixels, PT_CHUNK_PATHS / spp));
                }
                const long long per_pixel = chunk_path_bytes(max_depth) * spp;
                const long long b = budget > 0 ? std::min(budget, chunk_budget()) : chunk_budget();
                long long c = std::max(1LL, std::min(pixels, b / per_pixel));
                return std::min(c, (TASK_MAX_PATHS - 1) / spp);
        }

public:
        static bool double_sums(const int pixel_sums)
        {
                if (pixel_sums != PIXEL_SUMS_DEFAULT && pixel_sums != PIXEL_SUMS_FLOAT &&
                    pixel_sums != PIXEL_SUMS_DOUBLE)
                {
                        throw std::runtime_error("Unknown pixel sums " + std::to_string(pixel_sums));
                }
                return pixel_sums == PIXEL_SUMS_DOUBLE ||
                       (pixel_sums == PIXEL_SUMS_DEFAULT && std::is_same_v<T, float>);
        }

        // device bytes a painter of these parameters allocates
        static long long estimate_bytes(const long long pixels, const int spp, const int max_depth, const int strata,
                                        const Integrator integrator, const long long budget = 0,
                                        const bool sums_in_double = false)
        {
                const long long samples = pixels * spp;
                const long long per_sample = (N - 1) * sizeof(T) + C * 4 + 4 + 1;
                const long long per_pixel =
                        (sums_in_double ? sizeof(PixelState<C, double>) : sizeof(PixelState<C, float>)) + 12 + 16;
                const long long chunk = integrator == Integrator::PT
                                                ? 4 // the path counter; the direct-lighting records are small
                                                : chunk_pixels(pixels, spp, max_depth, integrator, budget) * spp *
                                                          chunk_path_bytes(max_depth);
                return (strata + 1) * sizeof(T) + samples * per_sample + pixels * per_pixel + sizeof(PathStats) +
                       chunk;
        }

        // slab_end < 0: the whole screen; else the rows [slab_begin, slab_end)
        // of the last screen axis, with their paths, the paths of the rows
        // either side (the filter reaches one pixel) and the estimator of the
        // slab's own pixels
        PainterT(const SceneT<N, T, C>* scene, const int spp, const int max_depth, const std::uint32_t seed,
                 const Integrator integrator, const int slab_begin = 0, const int slab_end = -1,
                 const bool flat_shading = false, const long long chunk_budget = 0, const int pixel_sums = 0)
                : scene_(scene),
                  flat_shading_(flat_shading),
                  double_sums_(double_sums(pixel_sums)),
                  chunk_budget_(chunk_budget),
                  spp_request_(spp),
                  max_depth_(max_depth),
                  seed_(seed),
                  integrator_(integrator)
        {
                if (spp < 1)
                {
                        throw std::runtime_error("Painter samples per pixel must be greater than 0");
                }
                if (integrator != Integrator::BPT && integrator != Integrator::PT)
                {
                        throw std::runtime_error("Unknown integrator " + std::to_string(static_cast<int>(integrator)));
                }
                if (integrator == Integrator::BPT && (max_depth < 1 || max_depth > MAX_PATH_VERTICES - 1))
                {
                        throw std::runtime_error("Painter maximum depth must be in [1, 8]");
                }
                scene_->device(); // throws if not finalized
                strata_ = SceneT<N, T, C>::strata(spp);
                spp_ = scene_->actual_spp(spp);
                if (spp_ > MAX_GROUP)
                {
                        throw std::runtime_error(
                                "Painter samples per pixel " + std::to_string(spp_) + " exceed the maximum "
                                + std::to_string(MAX_GROUP) + " of one pass");
                }
                pixels_ = scene_->pixel_count();
                if (pixels_ >= (1LL << 31))
                {
                        throw std::runtime_error("a screen of " + std::to_string(pixels_) +
                                                 " pixels: at most 2^31 - 1 are supported");
                }
                sources_ = pixels_;
                if (slab_end >= 0)
                {
                        const int rows = scene_->device().projector.size[N - 2];
                        if (slab_begin < 0 || slab_begin >= slab_end || slab_end > rows)
                        {
                                throw std::runtime_error("slab rows [" + std::to_string(slab_begin) + ", " +
                                                         std::to_string(slab_end) + ") outside the screen's " +
                                                         std::to_string(rows) + " rows");
                        }
                        const long long row = pixels_ / rows;
                        const int source_begin = std::max(0, slab_begin - 1);
                        const int source_end = std::min(rows, slab_end + 1);
                        first_ = slab_begin * row;
                        pixels_ = (slab_end - slab_begin) * row;
                        source_first_ = source_begin * row;
                        sources_ = (source_end - source_begin) * row;
                }

                NBPT_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));

                // offsets of the strata (sj_sampler.h:75-114)
                std::vector<T> offsets(strata_ + 1);
                const T offset_size = (T(1) - T(0)) / static_cast<T>(strata_);
                offsets[0] = 0;
                for (int i = 1; i < strata_; ++i)
                {
                        offsets[i] = T(0) + static_cast<T>(i) * offset_size;
                }
                offsets[strata_] = 1;
                offsets_.upload_on(offsets, stream_);

                const long long samples = sources_ * spp_;
                points_.allocate(samples * (N - 1));
                colors_.allocate(samples * C);
                lum_.allocate(samples);
                valid_.allocate(samples);
                if (double_sums_)
                {
                        state64_.allocate(pixels_);
                }
                else
                {
                        state_.allocate(pixels_);
                }
                stats_.allocate(1);
                NBPT_CUDA(cudaMemsetAsync(stats_.get(), 0, sizeof(PathStats), stream_));
                cancel_.allocate(1);
                NBPT_CUDA(cudaMemsetAsync(cancel_.get(), 0, sizeof(unsigned), stream_));
                rgb_.allocate(pixels_ * 3);
                rgba_.allocate(pixels_ * 4);
                int device = 0;
                int sms = 0;
                NBPT_CUDA(cudaGetDevice(&device));
                device_ = device;
                NBPT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
                chunk_pixels_ = chunk_pixels(sources_, spp_, max_depth_, integrator_, chunk_budget_);
                if (integrator_ == Integrator::PT)
                {
                        next_path_.allocate(1);
                        connect_blocks_ = sms * NBPT_PT_MIN_BLOCKS;
                        // direct-lighting records: 2 per light per thread
                        pt_estimates_.allocate(std::max(1LL, static_cast<long long>(connect_blocks_) * 128 * 2 *
                                                                     scene_->device().light_count));
                }
                else
                {
                        tape_words_ = tape_words(max_depth_);
                        allocate_scratch();
                        task_count_.allocate(3);
                        next_path_.allocate(1);
                        connect_blocks_ = sms * PathsMinBlocks<N, T>::value;
                }

                NBPT_CUDA(cudaEventCreate(&ev_start_));
                NBPT_CUDA(cudaEventCreate(&ev_paths_));
                NBPT_CUDA(cudaEventCreate(&ev_paths_end_));
                NBPT_CUDA(cudaEventCreate(&ev_end_));
                if (double_sums_)
                {
                        NBPT_CUDA(cudaMemsetAsync(state64_.get(), 0, state64_.bytes(), stream_));
                }
                else
                {
                        NBPT_CUDA(cudaMemsetAsync(state_.get(), 0, state_.bytes(), stream_));
                }
                statistics_.pixel_count = pixels_;
        }

        ~PainterT() override
        {
                if (stream_)
                {
                        cudaStreamSynchronize(stream_);
                        cudaStreamDestroy(stream_);
                }
                if (cancel_stream_)
                {
                        cudaStreamSynchronize(cancel_stream_);
                        cudaStreamDestroy(cancel_stream_);
                }
                for (cudaEvent_t e : {ev_start_, ev_paths_, ev_paths_end_, ev_end_})
                {
                        if (e)
                        {
                                cudaEventDestroy(e);
                        }
                }
        }

        long long device_bytes() const override
        {
                const std::size_t own = offsets_.bytes() + points_.bytes() + colors_.bytes() + lum_.bytes() +
                                        valid_.bytes() + state_.bytes() + state64_.bytes() + stats_.bytes() +
                                        rgb_.bytes() +
                                        rgba_.bytes() + vertices_.bytes() + rng_.bytes() + tape_.bytes() +
                                        tasks_.bytes() + task_count_.bytes() + arrivals_.bytes() +
                                        next_path_.bytes() + pt_estimates_.bytes();
                return static_cast<long long>(own) + scene_->device_bytes();
        }

        void* stream() override
        {
                return stream_;
        }

        // The path kernels of this precision: single precision's come from
        // their own unit, compiled with multiply-add contraction
        // (float_paths.h); double precision's are compiled here, without it.
        static auto walk_kernel()
        {
                if constexpr (std::is_same_v<T, float>)
                {
                        return float_path_kernels<N>().walk;
                }
                else
                {
                        return &paths_walk_kernel<N, T>;
                }
        }
        static auto light_kernel()
        {
                if constexpr (std::is_same_v<T, float>)
                {
                        return float_path_kernels<N>().light;
                }
                else
                {
                        return &paths_light_kernel<N, T>;
                }
        }
        static auto connect_kernel()
        {
                if constexpr (std::is_same_v<T, float>)
                {
                        return float_path_kernels<N>().connect;
                }
                else
                {
                        return &paths_connect_kernel<N, T>;
                }
        }
        static auto replay_kernel()
        {
                constexpr int LANES = C % 32 == 0 ? 32 : 1;
                if constexpr (std::is_same_v<T, float>)
                {
                        static_assert(C == 3 || C == 64);
                        if constexpr (C == 3)
                        {
                                return float_path_kernels<N>().replay_rgb;
                        }
                        else
                        {
                                return float_path_kernels<N>().replay_spectrum;
                        }
                }
                else
                {
                        return &paths_replay_kernel<N, T, C, LANES>;
                }
        }
        static auto pt_kernel()
        {
                if constexpr (std::is_same_v<T, float>)
                {
                        static_assert(C == 3 || C == 64);
                        if constexpr (C == 3)
                        {
                                return float_path_kernels<N>().pt_rgb;
                        }
                        else
                        {
                                return float_path_kernels<N>().pt_spectrum;
                        }
                }
                else
                {
                        return &pt_paths_kernel<N, T, C>;
                }
        }

        // the per-chunk buffers of the BPT path kernels
        void allocate_scratch()
        {
                const long long paths = chunk_pixels_ * spp_;
                tape_.allocate(paths * tape_words_);
                vertices_.allocate(paths * 2 * (max_depth_ + 1));
                rng_.allocate(paths);
                tasks_.allocate(paths * tape_slot_count(max_depth_));
                arrivals_.allocate(paths * max_depth_);
                scratch_ready_ = true;
        }

        long long release_scratch() override
        {
                NBPT_CUDA(cudaStreamSynchronize(stream_));
                if (integrator_ == Integrator::PT || !scratch_ready_)
                {
                        return 0;
                }
                scratch_ready_ = false;
                return static_cast<long long>(tape_.free() + vertices_.free() + rng_.free() + tasks_.free() +
                                              arrivals_.free());
        }

        void cancel() override
        {
                const std::lock_guard lock(cancel_mutex_);
                if (cancelled_)
                {
                        return;
                }
                if (!cancel_stream_)
                {
                        NBPT_CUDA(cudaStreamCreateWithFlags(&cancel_stream_, cudaStreamNonBlocking));
                }
                // on its own stream, so the word changes while the pass runs
                NBPT_CUDA(cudaMemsetAsync(cancel_.get(), 1, 1, cancel_stream_));
                cancelled_ = true;
        }

        bool cancelled() const override
        {
                return cancelled_;
        }

        void enqueue_passes(const int passes) override
        {
                if (cancelled_)
                {
                        throw std::runtime_error("the painter was cancelled");
                }
                if (integrator_ == Integrator::BPT && !scratch_ready_)
                {
                        allocate_scratch();
                }
                const DeviceScene<N, T, C>& scene = scene_->device();
                for (int k = 0; k < passes; ++k)
                {
                        const std::uint32_t pass = static_cast<std::uint32_t>(pass_++);
                        // per-pass counters; overflows and nonfinite count over the
                        // painter's life
                        NBPT_CUDA(cudaMemsetAsync(stats_.get(), 0, offsetof(PathStats, overflows), stream_));
                        NBPT_CUDA(cudaEventRecord(ev_start_, stream_));
                        sj_points_kernel<N - 1, T><<<blocks_for(sources_, 128), 128, 0, stream_>>>(
                                source_first_, source_first_ + sources_, seed_, pass, strata_, offsets_.get(),
                                points_.get());
                        NBPT_CUDA(cudaGetLastError());
                        NBPT_CUDA(cudaEventRecord(ev_paths_, stream_));
                        long long launches = 2;
                        DeviceScene<N, T, 1> scene_1 = scene_->device_channel_0();
                        scene_1.flat_shading = flat_shading_ ? 1 : 0;
                        if (integrator_ == Integrator::PT)
                        {
                                // one launch per chunk: whole paths (pt.cuh)
                                for (long long b = source_first_; b < source_first_ + sources_; b += chunk_pixels_)
                                {
                                        const long long e = std::min(source_first_ + sources_, b + chunk_pixels_);
                                        const long long o = b - source_first_; // the chunk in the sample arrays
                                        const long long n = (e - b) * spp_;
                                        NBPT_CUDA(cudaMemsetAsync(next_path_.get(), 0, sizeof(unsigned), stream_));
                                        pt_kernel()
                                                <<<std::min<long long>(connect_blocks_, blocks_for(n, 128)), 128, 0, stream_>>>(
                                                        scene_1, scene_->device_materials(),
                                                        scene_->device_lights(), b, e, spp_, seed_, pass,
                                                        points_.get() + o * spp_ * (N - 1), colors_.get() + o * spp_ * C,
                                                        lum_.get() + o * spp_, valid_.get() + o * spp_,
                                                        pt_estimates_.get(), next_path_.get(), stats_.get(),
                                                        scene_->cie() + 64, cancel_.get());
                                        NBPT_CUDA(cudaGetLastError());
                                        launches += 1;
                                        note_progress(pass, e);
                                }
                        }
                        else
                        {
                                // per chunk of pixels: subpaths, strategies, the s = 1
                                // strategies, then the colours (kernels.cuh)
                                for (long long b = source_first_; b < source_first_ + sources_; b += chunk_pixels_)
                                {
                                        const long long e = std::min(source_first_ + sources_, b + chunk_pixels_);
                                        const long long o = b - source_first_; // the chunk in the sample arrays
                                        const long long n = (e - b) * spp_;
                                        NBPT_CUDA(cudaMemsetAsync(task_count_.get(), 0, 3 * sizeof(unsigned), stream_));
                                        // queue regions: s >= 2, then s = 1 and s = 0 (at most
                                        // max_depth each per path)
                                        TaskQueues queues;
                                        queues.base[TaskQueues::CONNECT] = tasks_.get();
                                        queues.base[TaskQueues::LIGHT] =
                                                tasks_.get() + n * (tape_slot_count(max_depth_) - 2 * max_depth_);
                                        queues.base[TaskQueues::EMITTED] =
                                                tasks_.get() + n * (tape_slot_count(max_depth_) - max_depth_);
                                        queues.count = task_count_.get();
                                        NBPT_CUDA(cudaMemsetAsync(next_path_.get(), 0, sizeof(unsigned), stream_));
                                        walk_kernel()<<<std::min<long long>(connect_blocks_, blocks_for(n, 128)), 128, 0,
                                                                  stream_>>>(
                                                scene_1, b, e, spp_, max_depth_, seed_, pass, points_.get() + o * spp_ * (N - 1),
                                                vertices_.get(), rng_.get(), tape_.get(), tape_words_, valid_.get() + o * spp_,
                                                queues, next_path_.get(), stats_.get(), cancel_.get());
                                        NBPT_CUDA(cudaGetLastError());
                                        light_kernel()<<<blocks_for(n, 128), 128, 0, stream_>>>(
                                                scene_1, n, max_depth_, vertices_.get(), rng_.get(), tape_.get(), tape_words_,
                                                arrivals_.get(), queues, cancel_.get());
                                        NBPT_CUDA(cudaGetLastError());
                                        connect_kernel()<<<connect_blocks_, 128, 0, stream_>>>(
                                                scene_1, max_depth_, vertices_.get(), tape_.get(), tape_words_, arrivals_.get(),
                                                queues, stats_.get());
                                        NBPT_CUDA(cudaGetLastError());
                                        constexpr int LANES = C % 32 == 0 ? 32 : 1;
                                        replay_kernel()<<<blocks_for(n * LANES, 128), 128, 0, stream_>>>(
                                                scene_->device_materials(), scene_->device_lights(),
                                                scene.shading.fresnel_a, scene.shading.fresnel_b, max_depth_, n, tape_.get(),
                                                tape_words_, colors_.get() + o * spp_ * C, lum_.get() + o * spp_,
                                                scene_->cie() + 64, stats_.get(), cancel_.get());
                                        NBPT_CUDA(cudaGetLastError());
                                        launches += 4;
                                        note_progress(pass, e);
                                }
                        }
                        NBPT_CUDA(cudaEventRecord(ev_paths_end_, stream_));
                        Screen<N> screen;
                        for (int i = 0; i < N - 1; ++i)
                        {
                                screen.size[i] = scene.projector.size[i];
                        }
                        screen.first = first_;
                        screen.source_first = source_first_;
                        const T radius = T(1.5);
                        const T width = radius / T(2.5);
                        const T alpha = -1 / (2 * width * width);
                        const T exp_radius = std::exp(alpha * radius * radius);
                        if (double_sums_)
                        {
                                accumulate(screen, alpha, exp_radius, state64_.get());
                        }
                        else
                        {
                                accumulate(screen, alpha, exp_radius, state_.get());
                        }
                        NBPT_CUDA(cudaGetLastError());
                        NBPT_CUDA(cudaEventRecord(ev_end_, stream_));
                        launches_ = launches;
                }
                passes_done_ += passes;
        }

        void set_progress(const ProgressCallback callback, void* const user) override
        {
                progress_ = callback;
                progress_user_ = user;
        }

        void wait() override
        {
                NBPT_CUDA(cudaStreamSynchronize(stream_));
                // every host callback has run
                progress_dropped_ += static_cast<long long>(progress_notes_.size());
                progress_notes_.clear();
                if (cancelled_)
                {
                        throw std::runtime_error("cancelled: the pass in flight ended early and its image is incomplete");
                }
                PathStats s{};
                stats_.download_on(&s, 1, stream_);
                float ms = 0;
                float paths_ms = 0;
                NBPT_CUDA(cudaEventElapsedTime(&ms, ev_start_, ev_end_));
                NBPT_CUDA(cudaEventElapsedTime(&paths_ms, ev_paths_, ev_paths_end_));
                statistics_.pass_number = passes_done_;
                statistics_.ray_count = static_cast<long long>(s.queries);
                statistics_.sample_count = sources_ * spp_;
                statistics_.previous_pass_duration = ms * 1e-3;
                statistics_.paths_seconds = paths_ms * 1e-3;
                statistics_.nodes = s.nodes;
                statistics_.facets = s.facets;
                statistics_.shapes = s.shapes;
                statistics_.kernel_launches = launches_;
                statistics_.nonfinite_samples = static_cast<long long>(s.nonfinite);
                statistics_.stack_overflows = static_cast<long long>(s.overflows);
                if (s.overflows != 0)
                {
                        throw std::runtime_error(std::to_string(s.overflows) +
                                                 " ray queries found the BVH traversal stack full; the image is "
                                                 "incomplete");
                }
        }

        template <typename S>
        void accumulate(const Screen<N>& screen, const T alpha, const T exp_radius, PixelState<C, S>* const state)
        {
                if constexpr (C % 32 == 0 && N <= 4)
                {
                        if (spp_ <= SMALL_GROUP)
                        {
                                accumulate_warp_small_kernel<N, T, C, S><<<blocks_for(pixels_ * 32, 128), 128, 0, stream_>>>(
                                        screen, pixels_, spp_, points_.get(), colors_.get(), lum_.get(), valid_.get(),
                                        alpha, exp_radius, state);
                        }
                        else
                        {
                                accumulate_warp_kernel<N, T, C, S><<<blocks_for(pixels_ * 32, 128), 128, 0, stream_>>>(
                                        screen, pixels_, spp_, points_.get(), colors_.get(), lum_.get(), valid_.get(),
                                        alpha, exp_radius, state);
                        }
                }
                else if constexpr (C % 32 == 0)
                {
                        accumulate_warp_kernel<N, T, C, S><<<blocks_for(pixels_ * 32, 128), 128, 0, stream_>>>(
                                screen, pixels_, spp_, points_.get(), colors_.get(), lum_.get(), valid_.get(), alpha,
                                exp_radius, state);
                }
                else
                {
                        accumulate_kernel<N, T, C, S><<<blocks_for(pixels_, 128), 128, 0, stream_>>>(
                                screen, pixels_, spp_, points_.get(), colors_.get(), lum_.get(), valid_.get(), alpha,
                                exp_radius, state);
                }
        }

        void resolve()
        {
                if (double_sums_)
                {
                        resolve_kernel<C, double><<<blocks_for(pixels_, 128), 128, 0, stream_>>>(
                                pixels_, state64_.get(), scene_->cie(), rgb_.get(), rgba_.get());
                }
                else
                {
                        resolve_kernel<C, float><<<blocks_for(pixels_, 128), 128, 0, stream_>>>(
                                pixels_, state_.get(), scene_->cie(), rgb_.get(), rgba_.get());
                }
        }

        void images(float* rgb, float* rgba) override
        {
                resolve();
                NBPT_CUDA(cudaGetLastError());
                NBPT_CUDA(cudaStreamSynchronize(stream_));
                if (rgb)
                {
                        rgb_.download_on(rgb, pixels_ * 3, stream_);
                }
                if (rgba)
                {
                        rgba_.download_on(rgba, pixels_ * 4, stream_);
                }
        }

        void enqueue_images(float* rgb, float* rgba) override
        {
                resolve();
                NBPT_CUDA(cudaGetLastError());
                if (rgb)
                {
                        NBPT_CUDA(cudaMemcpyAsync(rgb, rgb_.get(), pixels_ * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                                                  stream_));
                }
                if (rgba)
                {
                        NBPT_CUDA(cudaMemcpyAsync(rgba, rgba_.get(), pixels_ * 4 * sizeof(float),
                                                  cudaMemcpyDeviceToHost, stream_));
                }
        }

        int device() const override
        {
                return device_;
        }

        void samples(double* points, float* colors, unsigned char* valid) override
        {
                NBPT_CUDA(cudaStreamSynchronize(stream_));
                const long long samples = sources_ * spp_;
                if (points)
                {
                        std::vector<T> p(samples * (N - 1));
                        points_.download_on(p.data(), p.size(), stream_);
                        for (std::size_t i = 0; i < p.size(); ++i)
                        {
                                points[i] = static_cast<double>(p[i]);
                        }
                }
                if (colors)
                {
                        colors_.download_on(colors, samples * C, stream_);
                }
                if (valid)
                {
                        valid_.download_on(valid, samples, stream_);
                }
        }

        Statistics statistics() override
        {
                return statistics_;
        }
};

template <int N, typename T, int C>
std::unique_ptr<Painter> SceneT<N, T, C>::create_painter(
        const int spp,
        const int max_depth,
        const std::uint32_t seed,
        const Integrator integrator,
        const int slab_begin,
        const int slab_end,
        const bool flat_shading,
        const long long chunk_budget,
        const int pixel_sums)
{
        return std::make_unique<PainterT<N, T, C>>(this, spp, max_depth, seed, integrator, slab_begin, slab_end,
                                                   flat_shading, chunk_budget, pixel_sums);
}

template <int N, typename T, int C>
long long SceneT<N, T, C>::painter_bytes(const int spp, const int max_depth, const Integrator integrator,
                                         const long long chunk_budget, const int pixel_sums) const
{
        if (spp < 1 || (integrator == Integrator::BPT && max_depth < 1))
        {
                throw std::runtime_error("painter samples per pixel and maximum depth must be positive");
        }
        return PainterT<N, T, C>::estimate_bytes(pixel_count(), actual_spp(spp), max_depth, strata(spp), integrator,
                                                 chunk_budget, PainterT<N, T, C>::double_sums(pixel_sums));
}

template <int N, typename T, int C>
void SceneT<N, T, C>::trace(
        const double* rays,
        const long long count,
        const int any,
        int* kind,
        int* index,
        double* t,
        double* point)
{
        const DeviceScene<N, T, C>& s = device();
        DeviceArray<double> d_rays;
        d_rays.upload(rays, count * 2 * N);
        DeviceArray<int> d_kind;
        d_kind.allocate(count);
        DeviceArray<int> d_index;
        d_index.allocate(count);
        DeviceArray<double> d_t;
        d_t.allocate(count);
        DeviceArray<double> d_point;
        d_point.allocate(count * N);
        trace_kernel<N, T, C><<<blocks_for(count, 128), 128>>>(s, d_rays.get(), count, any, d_kind.get(), d_index.get(),
                                                               d_t.get(), d_point.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaDeviceSynchronize());
        d_kind.download(kind, count);
        if (!any)
        {
                d_index.download(index, count);
                d_t.download(t, count);
                d_point.download(point, count * N);
        }
}

template <int N, typename T, int C>
void SceneT<N, T, C>::trace_device(
        const double* rays,
        const long long count,
        const int any,
        int* kind,
        int* index,
        double* t,
        double* point) const
{
        const DeviceScene<N, T, C>& s = device();
        trace_kernel<N, T, C><<<blocks_for(count, 128), 128>>>(s, rays, count, any, kind, index, t, point);
        NBPT_CUDA(cudaGetLastError());
}

// counts: facets, nodes, indices; planes [F][N][N+1]; node_lo/hi [nodes][N];
// node_info [nodes][3] (offset, count, axis); normal_info [F][2] (type, reverse mask)
template <int N, typename T, int C>
void SceneT<N, T, C>::mesh_export(
        const int mesh,
        long long* counts,
        double* planes,
        double* node_lo,
        double* node_hi,
        unsigned* node_info,
        unsigned* indices,
        int* normal_info)
{
        device();
        if (mesh < 0 || mesh >= static_cast<int>(meshes_.size()))
        {
                throw std::runtime_error("no such mesh");
        }
        const MeshHost& m = meshes_[mesh];
        const long long facets = static_cast<long long>(m.facets.size() / N);
        const long long nodes = m.node_count;
        counts[0] = facets;
        counts[1] = nodes;
        counts[2] = facets;
        if (!planes)
        {
                return;
        }
        std::vector<Facet<N, T>> f(facets);
        NBPT_CUDA(cudaMemcpy(f.data(), d_facets_.get() + m.facet_offset, facets * sizeof(Facet<N, T>),
                             cudaMemcpyDeviceToHost));
        for (long long i = 0; i < facets; ++i)
        {
                double* out = planes + i * N * (N + 1);
                for (int d = 0; d < N; ++d)
                {
                        out[d] = static_cast<double>(f[i].simplex.plane.n[d]);
                }
                out[N] = static_cast<double>(f[i].simplex.plane.d);
                for (int j = 0; j < N - 1; ++j)
                {
                        for (int d = 0; d < N; ++d)
                        {
                                out[(j + 1) * (N + 1) + d] = static_cast<double>(f[i].simplex.planes[j].n[d]);
                        }
                        out[(j + 1) * (N + 1) + N] = static_cast<double>(f[i].simplex.planes[j].d);
                }
                normal_info[i * 2] = f[i].normal_type;
                normal_info[i * 2 + 1] = static_cast<int>(f[i].reverse_mask);
        }
        std::vector<BvhNode<N, T>> b(nodes);
        NBPT_CUDA(cudaMemcpy(b.data(), d_nodes_.get() + m.node_offset, nodes * sizeof(BvhNode<N, T>),
                             cudaMemcpyDeviceToHost));
        for (long long i = 0; i < nodes; ++i)
        {
                for (int d = 0; d < N; ++d)
                {
                        node_lo[i * N + d] = static_cast<double>(b[i].lo[d]);
                        node_hi[i * N + d] = static_cast<double>(b[i].hi[d]);
                }
                node_info[i * 3] = b[i].offset;
                node_info[i * 3 + 1] = b[i].count;
                node_info[i * 3 + 2] = b[i].axis;
        }
        NBPT_CUDA(cudaMemcpy(indices, d_indices_.get() + m.index_offset, facets * sizeof(std::uint32_t),
                             cudaMemcpyDeviceToHost));
}

template <int N, typename T, int C>
void SceneT<N, T, C>::brdf(const int material, const double* n, const double* v, const double* l, float* f, double* pdf)
{
        const DeviceScene<N, T, C>& s = device();
        if (material < 0 || material >= static_cast<int>(materials_.size()))
        {
                throw std::runtime_error("no such material");
        }
        std::vector<double> in(3 * N);
        std::copy(n, n + N, in.begin());
        std::copy(v, v + N, in.begin() + N);
        std::copy(l, l + N, in.begin() + 2 * N);
        DeviceArray<double> d_in;
        d_in.upload(in);
        DeviceArray<float> d_f;
        d_f.allocate(C);
        DeviceArray<double> d_pdf;
        d_pdf.allocate(1);
        brdf_kernel<N, T, C><<<1, 1>>>(s, material, d_in.get(), d_f.get(), d_pdf.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaDeviceSynchronize());
        d_f.download(f, C);
        d_pdf.download(pdf, 1);
}

template <int N, typename T, int C>
void SceneT<N, T, C>::brdf_sample(
        const int material,
        const double* n,
        const double* v,
        const std::uint32_t* seed,
        const int seed_words,
        double* l,
        double* pdf,
        float* f)
{
        const DeviceScene<N, T, C>& s = device();
        if (material < 0 || material >= static_cast<int>(materials_.size()))
        {
                throw std::runtime_error("no such material");
        }
        std::vector<double> in(2 * N);
        std::copy(n, n + N, in.begin());
        std::copy(v, v + N, in.begin() + N);
        DeviceArray<double> d_in;
        d_in.upload(in);
        DeviceArray<std::uint32_t> d_seed;
        d_seed.upload(seed, seed_words);
        DeviceArray<double> d_l;
        d_l.allocate(N);
        DeviceArray<double> d_pdf;
        d_pdf.allocate(1);
        DeviceArray<float> d_f;
        d_f.allocate(C);
        brdf_sample_kernel<N, T, C><<<1, 1>>>(s, material, d_in.get(), d_seed.get(), seed_words, d_l.get(), d_pdf.get(),
                                              d_f.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaDeviceSynchronize());
        d_pdf.download(pdf, 1);
        d_l.download(l, N);
        d_f.download(f, C);
}

template <int N, typename T, int C>
void SceneT<N, T, C>::light_sample(
        const int light,
        const int kind,
        const std::uint32_t* seed,
        const int seed_words,
        const double* point,
        double* out,
        float* radiance)
{
        const DeviceScene<N, T, C>& s = device();
        if (light < 0 || light >= static_cast<int>(lights_.size()))
        {
                throw std::runtime_error("no such light");
        }
        DeviceArray<std::uint32_t> d_seed;
        d_seed.upload(seed, seed_words);
        std::vector<double> p(point, point + N);
        DeviceArray<double> d_point;
        d_point.upload(p);
        DeviceArray<double> d_out;
        d_out.allocate(3 * N + 2);
        DeviceArray<float> d_rad;
        d_rad.allocate(C);
        light_sample_kernel<N, T, C><<<1, 1>>>(s, light, kind, d_seed.get(), seed_words, d_point.get(), d_out.get(),
                                               d_rad.get());
        NBPT_CUDA(cudaGetLastError());
        NBPT_CUDA(cudaDeviceSynchronize());
        d_out.download(out, 3 * N + 2);
        d_rad.download(radiance, C);
}

template <int N>
std::unique_ptr<Scene> make_scene_n(const bool double_precision, const bool spectrum)
{
        if (double_precision)
        {
                if (spectrum)
                {
                        return std::make_unique<SceneT<N, double, 64>>();
                }
                return std::make_unique<SceneT<N, double, 3>>();
        }
        if (spectrum)
        {
                return std::make_unique<SceneT<N, float, 64>>();
        }
        return std::make_unique<SceneT<N, float, 3>>();
}
} // namespace nbpt
