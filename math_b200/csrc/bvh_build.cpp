#include "bvh_build.h"

#include <array>
#include <limits>
#include <optional>
#include <span>
#include <stdexcept>
#include <vector>

namespace nbpt::host
{
namespace
{
constexpr unsigned BUCKET_COUNT = 32;

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
                for (std::size_t i = 1; i < objects.size(); ++i)
                {
                        box.merge(objects[i].center.data());
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
template <int N, typename T>
std::optional<Split<N, T>> split(std::span<Object<N, T>> objects, const Box<N, T>& bounds, const T interior_cost)
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

template <int N, typename T>
struct Builder final
{
        T interior_cost;
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

        // Builds the subtree of `objects` in depth-first order and returns its
        // root node index (bvh.cpp:35-67).
        unsigned build(const std::span<Object<N, T>> objects, const Box<N, T>& bounds)
        {
                const unsigned node = push_node(bounds);
                const std::optional<Split<N, T>> s = split(objects, bounds, interior_cost);
                if (!s)
                {
                        out->offset[node] = out->indices.size();
                        out->count[node] = objects.size();
                        for (const Object<N, T>& o : objects)
                        {
                                out->indices.push_back(o.index);
                        }
                        return node;
                }
                out->axis[node] = s->axis;
                build(objects.subspan(0, s->middle), s->bounds_min);
                const unsigned second = build(objects.subspan(s->middle), s->bounds_max);
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

        BuiltBvh<N, T> out;
        out.indices.reserve(count);
        Builder<N, T> builder{static_cast<T>(2 * box_r_cost), &out};
        builder.build(std::span<Object<N, T>>(objects), root);
        return out;
}

template BuiltBvh<3, float> build_facet_bvh<3, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<3, double> build_facet_bvh<3, double>(const std::vector<double>&, const std::vector<int>&);
template BuiltBvh<4, float> build_facet_bvh<4, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<4, double> build_facet_bvh<4, double>(const std::vector<double>&, const std::vector<int>&);
template BuiltBvh<5, float> build_facet_bvh<5, float>(const std::vector<float>&, const std::vector<int>&);
template BuiltBvh<5, double> build_facet_bvh<5, double>(const std::vector<double>&, const std::vector<int>&);
} // namespace nbpt::host
