#include "bvh_build.h"

#include <algorithm>
#include <array>
#include <thread>
#include <future>
#include <memory>
#include <limits>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

namespace nbpt::host
{
namespace
{
constexpr unsigned BUCKET_COUNT = 32;

// Nodes of at least this many objects are binned by several threads.
constexpr std::size_t PARALLEL_BINNING = 32768;
constexpr unsigned THREADS = 8;

// f(thread, begin, end) over [0, count) in THREADS parts
template <typename F>
void run_parallel(const std::size_t count, const F& f)
{
        std::vector<std::thread> threads;
        const std::size_t step = (count + THREADS - 1) / THREADS;
        for (unsigned t = 1; t < THREADS; ++t)
        {
                const std::size_t b = std::min(count, t * step);
                const std::size_t e = std::min(count, b + step);
                threads.emplace_back([&f, t, b, e] { f(t, b, e); });
        }
        f(0, 0, std::min(count, step));
        for (std::thread& th : threads)
        {
                th.join();
        }
}

template <int N, typename T>
struct Box final
{
        std::array<T, N> lo;
        std::array<T, N> hi;

        static Box point(const T* p)
        {
                Box b;
                for (int i = 0; i < N; ++i)
                {
                        b.lo[i] = p[i];
                        b.hi[i] = p[i];
                }
                return b;
        }

        // std::min / std::max per component (bounding_box.h:307-332)
        void merge(const T* p)
        {
                for (int i = 0; i < N; ++i)
                {
                        lo[i] = (p[i] < lo[i]) ? p[i] : lo[i];
                        hi[i] = (hi[i] < p[i]) ? p[i] : hi[i];
                }
        }

        void merge(const Box& b)
        {
                for (int i = 0; i < N; ++i)
                {
                        lo[i] = (b.lo[i] < lo[i]) ? b.lo[i] : lo[i];
                        hi[i] = (hi[i] < b.hi[i]) ? b.hi[i] : hi[i];
                }
        }

        [[nodiscard]] Box merged(const Box& b) const
        {
                Box r = *this;
                r.merge(b);
                return r;
        }

        [[nodiscard]] std::array<T, N> center() const
        {
                std::array<T, N> c;
                for (int i = 0; i < N; ++i)
                {
                        c[i] = (lo[i] + hi[i]) * T(0.5);
                }
                return c;
        }

        [[nodiscard]] unsigned maximum_extent() const
        {
                T m = hi[0] - lo[0];
                unsigned r = 0;
                for (int i = 1; i < N; ++i)
                {
                        const T d = hi[i] - lo[i];
                        if (d > m)
                        {
                                m = d;
                                r = i;
                        }
                }
                return r;
        }

        // bounding_box.h:43-103
        static T volume_impl(const T* d, const int m)
        {
                if (m == 1)
                {
                        return d[0];
                }
                if (m == 2)
                {
                        return d[0] * d[1];
                }
                if (m == 3)
                {
                        return d[0] * d[1] * d[2];
                }
                return d[m - 1] * volume_impl(d, m - 1);
        }

        static T surface_impl(const T* d, const int m)
        {
                if (m == 2)
                {
                        return d[0] + d[1];
                }
                if (m == 3)
                {
                        return d[0] * d[1] + d[2] * (d[0] + d[1]);
                }
                return volume_impl(d, m - 1) + d[m - 1] * surface_impl(d, m - 1);
        }

        [[nodiscard]] T surface() const
        {
                std::array<T, N> d;
                for (int i = 0; i < N; ++i)
                {
                        d[i] = hi[i] - lo[i];
                }
                return 2 * surface_impl(d.data(), N);
        }
};

template <int N, typename T>
struct Object final
{
        Box<N, T> bounds;
        std::array<T, N> center;
        T cost;
        unsigned index;
};

template <int N, typename T>
struct Bucket final
{
        Box<N, T> bounds;
        T cost;
};

template <int N, typename T>
struct CenterBounds final
{
        Box<N, T> box;
        unsigned axis;
        T length_r;
        T min;

        explicit CenterBounds(const std::span<const Object<N, T>> objects)
        {
                box = Box<N, T>::point(objects[0].center.data());
                if (objects.size() >= PARALLEL_BINNING)
                {
                        // component-wise min and max: the order of merging does not matter
                        std::vector<Box<N, T>> part(THREADS, box);
                        run_parallel(objects.size(), [&](const unsigned t, const std::size_t b, const std::size_t e)
                                     {
                                             for (std::size_t i = b; i < e; ++i)
                                             {
                                                     part[t].merge(objects[i].center.data());
                                             }
                                     });
                        for (const Box<N, T>& p : part)
                        {
                                box.merge(p);
                        }
                }
                else
                {
                        for (std::size_t i = 1; i < objects.size(); ++i)
                        {
                                box.merge(objects[i].center.data());
                        }
                }
                axis = box.maximum_extent();
                length_r = 1 / (box.hi[axis] - box.lo[axis]);
                min = box.lo[axis];
        }

        [[nodiscard]] bool is_point() const
        {
                return box.lo[axis] == box.hi[axis];
        }

        [[nodiscard]] unsigned bucket(const Object<N, T>& o) const
        {
                const unsigned n = static_cast<unsigned>(static_cast<T>(BUCKET_COUNT) * ((o.center[axis] - min) * length_r));
                return n < BUCKET_COUNT - 1 ? n : BUCKET_COUNT - 1;
        }
};

template <int N, typename T>
struct Split final
{
        std::size_t middle;
        Box<N, T> bounds_min;
        Box<N, T> bounds_max;
        unsigned axis;
};

// bvh_split.h:273-314
// uniform_sums: when every object has the same cost c, uniform_sums[k] is
// the double sum of k copies of c added one at a time (the value the
// sequential loop below forms for k objects), which lets large nodes be
// binned in parallel with the same sums.
template <int N, typename T>
std::optional<Split<N, T>> split(std::span<Object<N, T>> objects, const Box<N, T>& bounds, const T interior_cost,
                                 const std::vector<double>* const uniform_sums)
{
        if (objects.size() == 1)
        {
                return std::nullopt;
        }
        const CenterBounds<N, T> cb{std::span<const Object<N, T>>(objects.data(), objects.size())};
        if (cb.is_point())
        {
                return std::nullopt;
        }

        std::array<double, BUCKET_COUNT> sum{};
        std::array<std::optional<Bucket<N, T>>, BUCKET_COUNT> buckets;
        double total = 0;
        if (uniform_sums && objects.size() >= PARALLEL_BINNING)
        {
                // per-thread buckets over contiguous ranges, merged in range
                // order: each bucket's bounds are the same component-wise min
                // and max, its count the same, and its cost sum is looked up
                struct Part final
                {
                        std::array<std::optional<Box<N, T>>, BUCKET_COUNT> bounds;
                        std::array<std::size_t, BUCKET_COUNT> count{};
                };
                std::vector<Part> parts(THREADS);
                run_parallel(objects.size(), [&](const unsigned t, const std::size_t b, const std::size_t e)
                             {
                                     Part& part = parts[t];
                                     for (std::size_t k = b; k < e; ++k)
                                     {
                                             const Object<N, T>& o = objects[k];
                                             const unsigned i = cb.bucket(o);
                                             if (part.bounds[i])
                                             {
                                                     part.bounds[i]->merge(o.bounds);
                                             }
                                             else
                                             {
                                                     part.bounds[i] = o.bounds;
                                             }
                                             ++part.count[i];
                                     }
                             });
                std::array<std::size_t, BUCKET_COUNT> count{};
                for (const Part& part : parts)
                {
                        for (unsigned i = 0; i < BUCKET_COUNT; ++i)
                        {
                                if (!part.bounds[i])
                                {
                                        continue;
                                }
                                if (buckets[i])
                                {
                                        buckets[i]->bounds.merge(*part.bounds[i]);
                                }
                                else
                                {
                                        buckets[i].emplace();
                                        buckets[i]->bounds = *part.bounds[i];
                                }
                                count[i] += part.count[i];
                        }
                }
                for (unsigned i = 0; i < BUCKET_COUNT; ++i)
                {
                        sum[i] = (*uniform_sums)[count[i]];
                }
                total = (*uniform_sums)[objects.size()];
        }
        else
        {
                for (const Object<N, T>& o : objects)
                {
                        total += o.cost;
                        const unsigned i = cb.bucket(o);
                        if (buckets[i])
                        {
                                buckets[i]->bounds.merge(o.bounds);
                                sum[i] += o.cost;
                        }
                        else
                        {
                                buckets[i].emplace();
                                buckets[i]->bounds = o.bounds;
                                sum[i] = o.cost;
                        }
                }
        }
        for (unsigned i = 0; i < BUCKET_COUNT; ++i)
        {
                if (buckets[i])
                {
                        buckets[i]->cost = static_cast<T>(sum[i]);
                }
        }
        const T cost = static_cast<T>(total);

        std::array<Bucket<N, T>, BUCKET_COUNT - 1> forward;
        forward[0] = *buckets[0];
        for (unsigned i = 1; i < BUCKET_COUNT - 1; ++i)
        {
                if (!buckets[i])
                {
                        forward[i] = forward[i - 1];
                        continue;
                }
                forward[i] = Bucket<N, T>{forward[i - 1].bounds.merged(buckets[i]->bounds), forward[i - 1].cost + buckets[i]->cost};
        }
        std::array<Bucket<N, T>, BUCKET_COUNT - 1> backward;
        backward[BUCKET_COUNT - 2] = *buckets[BUCKET_COUNT - 1];
        for (unsigned i = BUCKET_COUNT - 2; i > 0; --i)
        {
                if (!buckets[i])
                {
                        backward[i - 1] = backward[i];
                        continue;
                }
                backward[i - 1] = Bucket<N, T>{backward[i].bounds.merged(buckets[i]->bounds), backward[i].cost + buckets[i]->cost};
        }

        const T surface_r = 1 / bounds.surface();
        T split_cost = std::numeric_limits<T>::max();
        unsigned index = std::numeric_limits<unsigned>::max();
        for (unsigned i = 0; i < BUCKET_COUNT - 1; ++i)
        {
                const T f = forward[i].cost * forward[i].bounds.surface();
                const T b = backward[i].cost * backward[i].bounds.surface();
                const T c = interior_cost + (f + b) * surface_r;
                if (c < split_cost)
                {
                        split_cost = c;
                        index = i;
                }
        }
        if (split_cost >= cost)
        {
                return std::nullopt;
        }

        // std::partition (libstdc++ bidirectional algorithm)
        std::size_t first = 0;
        std::size_t last = objects.size();
        const auto pred = [&](const std::size_t k)
        {
                return cb.bucket(objects[k]) <= index;
        };
        while (true)
        {
                bool done = false;
                while (true)
                {
                        if (first == last)
                        {
                                done = true;
                                break;
                        }
                        if (pred(first))
                        {
                                ++first;
                        }
                        else
                        {
                                break;
                        }
                }
                if (done)
                {
                        break;
                }
                --last;
                while (true)
                {
                        if (first == last)
                        {
                                done = true;
                                break;
                        }
                        if (!pred(last))
                        {
                                --last;
                        }
                        else
                        {
                                break;
                        }
                }
                if (done)
                {
                        break;
                }
                std::swap(objects[first], objects[last]);
                ++first;
        }
        if (first == 0 || first == objects.size())
        {
                throw std::runtime_error("BVH split produced an empty side");
        }
        return Split<N, T>{first, forward[index].bounds, backward[index].bounds, cb.axis};
}

// The tree is built with subtrees of large nodes on separate threads (a
// node's split depends only on its own objects, and sibling subtrees
// partition disjoint ranges), then laid out depth first in one pass, so the
// result is the same node for node as a sequential depth-first build.
template <int N, typename T>
struct TreeNode final
{
        Box<N, T> bounds;
        unsigned axis = 0;
        std::unique_ptr<TreeNode> first;
        std::unique_ptr<TreeNode> second;
        std::span<Object<N, T>> objects; // leaves
};

inline constexpr std::size_t PARALLEL_OBJECTS = 8192;
inline constexpr int PARALLEL_DEPTH = 5; // up to 2^5 concurrent subtrees

template <int N, typename T>
std::unique_ptr<TreeNode<N, T>> build_tree(
        const std::span<Object<N, T>> objects,
        const Box<N, T>& bounds,
        const T interior_cost,
        const std::vector<double>* const uniform_sums,
        const int depth)
{
        auto node = std::make_unique<TreeNode<N, T>>();
        node->bounds = bounds;
        const std::optional<Split<N, T>> s = split(objects, bounds, interior_cost, uniform_sums);
        if (!s)
        {
                node->objects = objects;
                return node;
        }
        node->axis = s->axis;
        const std::span<Object<N, T>> a = objects.subspan(0, s->middle);
        const std::span<Object<N, T>> b = objects.subspan(s->middle);
        if (depth < PARALLEL_DEPTH && objects.size() >= PARALLEL_OBJECTS)
        {
                std::future<std::unique_ptr<TreeNode<N, T>>> f = std::async(
                        std::launch::async, [&]
                        {
                                return build_tree(a, s->bounds_min, interior_cost, uniform_sums, depth + 1);
                        });
                node->second = build_tree(b, s->bounds_max, interior_cost, uniform_sums, depth + 1);
                node->first = f.get();
        }
        else
        {
                node->first = build_tree(a, s->bounds_min, interior_cost, uniform_sums, depth + 1);
                node->second = build_tree(b, s->bounds_max, interior_cost, uniform_sums, depth + 1);
        }
        return node;
}

// Depth-first layout (bvh.cpp:35-67): a node, its first subtree, its second
// subtree; an interior node stores the index of its second child.
template <int N, typename T>
struct Layout final
{
        BuiltBvh<N, T>* out;

        unsigned push_node(const Box<N, T>& b)
        {
                const unsigned index = out->count.size();
                for (int i = 0; i < N; ++i)
                {
                        out->lo.push_back(b.lo[i]);
                        out->hi.push_back(b.hi[i]);
                }
                out->offset.push_back(0);
                out->count.push_back(0);
                out->axis.push_back(0);
                return index;
        }

        unsigned place(const TreeNode<N, T>& t, const int depth)
        {
                const unsigned node = push_node(t.bounds);
                if (!t.first)
                {
                        out->depth = std::max(out->depth, depth);
                        out->offset[node] = out->indices.size();
                        out->count[node] = t.objects.size();
                        for (const Object<N, T>& o : t.objects)
                        {
                                out->indices.push_back(o.index);
                        }
                        return node;
                }
                out->axis[node] = t.axis;
                place(*t.first, depth + 1);
                const unsigned second = place(*t.second, depth + 1);
                out->offset[node] = second;
                return node;
        }
};
} // namespace

template <int N, typename T>
BuiltBvh<N, T> build_facet_bvh(const std::vector<T>& vertices, const std::vector<int>& facets)
{
        const std::size_t count = facets.size() / N;
        if (count == 0)
        {
                throw std::runtime_error("No objects to build BVH");
        }
        const T facet_cost = static_cast<T>(static_cast<double>(N) / SIMPLEX_RATE);
        const T box_r_cost = static_cast<T>(static_cast<double>(N) / BOX_R_RATE);

        std::vector<Object<N, T>> objects(count);
        for (std::size_t f = 0; f < count; ++f)
        {
                Box<N, T> b = Box<N, T>::point(&vertices[static_cast<std::size_t>(facets[f * N]) * N]);
                for (int k = 1; k < N; ++k)
                {
                        b.merge(&vertices[static_cast<std::size_t>(facets[f * N + k]) * N]);
                }
                objects[f].bounds = b;
                objects[f].center = b.center();
                objects[f].cost = facet_cost;
                objects[f].index = static_cast<unsigned>(f);
        }
        Box<N, T> root = objects[0].bounds;
        for (std::size_t f = 1; f < count; ++f)
        {
                root.merge(objects[f].bounds);
        }

        // every facet costs the same: the running sums of that cost
        std::vector<double> uniform_sums(count + 1);
        uniform_sums[0] = 0;
        uniform_sums[1] = facet_cost;
        for (std::size_t k = 2; k <= count; ++k)
        {
                uniform_sums[k] = uniform_sums[k - 1] + facet_cost;
        }
        const std::unique_ptr<TreeNode<N, T>> tree = build_tree(
                std::span<Object<N, T>>(objects), root, static_cast<T>(2 * box_r_cost), &uniform_sums, 0);
        BuiltBvh<N, T> out;
        out.indices.reserve(count);
        out.lo.reserve(4 * count * N);
        out.hi.reserve(4 * count * N);
        Layout<N, T> layout{&out};
        layout.place(*tree, 0);
        if (out.depth > BVH_MAX_DEPTH)
        {
                throw std::runtime_error(
                        "BVH depth " + std::to_string(out.depth) + " exceeds the traversal stack of " +
                        std::to_string(BVH_MAX_DEPTH) + " entries (a degenerate mesh)");
        }
        return out;
}

template BuiltBvh<3, float> build_facet_bvh<3, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<3, double> build_facet_bvh<3, double>(const std::vector<double>&, const std::vector<int>&);
template BuiltBvh<4, float> build_facet_bvh<4, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<4, double> build_facet_bvh<4, double>(const std::vector<double>&, const std::vector<int>&);
template BuiltBvh<5, float> build_facet_bvh<5, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<5, double> build_facet_bvh<5, double>(const std::vector<double>&, const std::vector<int>&);
} // namespace nbpt::host
