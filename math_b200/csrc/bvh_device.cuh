// Binned-SAH BVH build for mesh facets on the GPU.
//
// The same tree as the reference's sequential build
// (src/geometry/accelerators/bvh_build.h:79-221, bvh_split.h:47-315,
// bvh.cpp:35-86) and as the host builder (bvh_build.cpp): 32 buckets on the
// axis of largest centroid extent, SAH costs from the pinned intersection
// costs, a leaf when no split is cheaper, objects partitioned with the
// element order of libstdc++'s bidirectional std::partition, nodes laid out
// depth first.
//
// The build runs level by level.  A node of more than BVH_SMALL objects is a
// task of the level: blocks over chunks of its objects reduce the centroid
// bounds and the bucket bounds and counts with atomic min / max on
// order-preserving integer keys, one thread per task takes the SAH decision,
// and the partition pairs the i-th misplaced object from the left with the
// i-th misplaced object from the right, which is the pairing std::partition's
// two scans produce.  A node of at most BVH_SMALL objects is built whole by
// one warp, one object per lane.  Nodes are named by their object range
// (a leaf by its first object, an interior node by its split position), the
// subtree sizes are summed bottom up, and every node finds its depth-first
// position from the sizes on its path to the root.
//
// Bucket sums of the costs use the running sums of the one facet cost, so
// they equal the sequential loop's.  Bounds are exact minima and maxima; the
// one difference from a sequential merge is the sign of a zero bound when a
// box holds both +0 and -0 in one coordinate (the sequential merge keeps the
// first it meets, the keys order -0 below +0).  The sign of such a zero
// changes no intersection, distance or SAH decision.
#pragma once

#include "core.cuh"
#include "scene.cuh"

#include <cstdint>

namespace nbpt
{
inline constexpr int BVH_BUCKETS = 32;
inline constexpr int BVH_SMALL = 32;   // nodes of at most this many objects: one warp
inline constexpr int BVH_CHUNK = 2048; // objects per block in the per-level kernels
inline constexpr int BVH_THREADS = 256;

// order-preserving integer keys of finite floating-point values
template <typename T>
struct BvhKey;

template <>
struct BvhKey<float> final
{
        using K = unsigned;
        static constexpr K LOW = 0u;
        static constexpr K HIGH = 0xffffffffu;

        __device__ static K key(const float f)
        {
                const unsigned b = __float_as_uint(f);
                return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        }

        __device__ static float value(const K k)
        {
                const unsigned b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
                return __uint_as_float(b);
        }
};

template <>
struct BvhKey<double> final
{
        using K = unsigned long long;
        static constexpr K LOW = 0ull;
        static constexpr K HIGH = 0xffffffffffffffffull;

        __device__ static K key(const double f)
        {
                const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(f));
                return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
        }

        __device__ static double value(const K k)
        {
                const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
                return __longlong_as_double(static_cast<long long>(b));
        }
};

template <int N, typename T>
struct BvhObject final
{
        T lo[N];
        T hi[N];
        T c[N];
        unsigned index;
};

// A node while building: a leaf is named by its first object, an interior
// node by its split position - 1.  Child references are id * 2 + (1 for a
// leaf).
template <int N, typename T>
struct BvhBuildNode final
{
        T lo[N];
        T hi[N];
        int axis;
        int child[2];
        int parent; // interior id, -1 for the root
        int side;   // 0: first child of the parent, 1: second
        int begin;  // leaves: first object
        int count;  // leaves: objects
        int size[2]; // interior: node counts of the two subtrees
        int visits;
        int preorder;
};

template <int N, typename T>
struct BvhTask final
{
        using K = typename BvhKey<T>::K;
        int begin;
        int end;
        int parent;
        int side;
        int chunk_begin;
        int chunk_count;
        T lo[N];
        T hi[N];
        K center_lo[N];
        K center_hi[N];
        K bucket_lo[BVH_BUCKETS][N];
        K bucket_hi[BVH_BUCKETS][N];
        unsigned bucket_count[BVH_BUCKETS];
        int split;  // bucket index of the split, -1: leaf
        int middle; // objects of the first child
        int swaps;  // misplaced pairs
};

struct BvhChunk final
{
        int task;
        int begin;
        int end;
};

template <int N, typename T>
struct BvhSmallTask final
{
        int begin;
        int end;
        int parent;
        int side;
        T lo[N];
        T hi[N];
};

struct BvhCounters final
{
        int tasks;       // tasks of the next level
        int chunks;      // chunks of the next level
        int small;       // small tasks
        int leaves;      // leaf ids
        int inner;       // interior ids
        int error;       // 1: an empty side, 2: a leaf of more than 65535 objects, 3: pairing mismatch,
                         // 4: a depth-first position out of range
        int root;        // reference of the root
        int root_size;
        int depth;       // of the deepest leaf, the root at 0
};

// ---------------------------------------------------------------------------
// box arithmetic of the reference (bounding_box.h:43-103, bvh_split.h)

template <int N, typename T>
__device__ T bvh_surface(const T* lo, const T* hi)
{
        T d[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                d[i] = hi[i] - lo[i];
        }
        // surface_impl(d, N), volume_impl(d, m) unrolled in the same order
        T s = d[0] * d[1] + d[2] * (d[0] + d[1]); // m = 3
        if constexpr (N == 3)
        {
                return 2 * s;
        }
        T v = d[0] * d[1] * d[2]; // volume_impl(d, 3)
#pragma unroll
        for (int m = 4; m <= N; ++m)
        {
                s = v + d[m - 1] * s;
                v = d[m - 1] * v;
        }
        return 2 * s;
}

template <int N, typename T>
__device__ void bvh_merge(T* lo, T* hi, const T* blo, const T* bhi)
{
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
                lo[i] = (blo[i] < lo[i]) ? blo[i] : lo[i];
                hi[i] = (hi[i] < bhi[i]) ? bhi[i] : hi[i];
        }
}

// CenterBounds: axis of largest extent, its minimum and reciprocal length
template <int N, typename T>
struct BvhAxis final
{
        int axis;
        T min;
        T length_r;
        bool point;

        __device__ static BvhAxis from(const T* lo, const T* hi)
        {
                BvhAxis r;
                T m = hi[0] - lo[0];
                r.axis = 0;
#pragma unroll
                for (int i = 1; i < N; ++i)
                {
                        const T d = hi[i] - lo[i];
                        if (d > m)
                        {
                                m = d;
                                r.axis = i;
                        }
                }
                r.length_r = 1 / (hi[r.axis] - lo[r.axis]);
                r.min = lo[r.axis];
                r.point = lo[r.axis] == hi[r.axis];
                return r;
        }

        __device__ int bucket(const T c) const
        {
                const unsigned n = static_cast<unsigned>(static_cast<T>(BVH_BUCKETS) * ((c - min) * length_r));
                return n < BVH_BUCKETS - 1 ? static_cast<int>(n) : BVH_BUCKETS - 1;
        }
};

// The SAH decision of bvh_split.h:273-314 from the buckets' bounds and
// counts: the split bucket, or -1 for a leaf.
template <int N, typename T>
__device__ int bvh_decide(
        const T (*bucket_lo)[N],
        const T (*bucket_hi)[N],
        const unsigned* bucket_count,
        const unsigned count,
        const T* lo,
        const T* hi,
        const double* uniform_sums,
        const T interior_cost,
        T* first_lo,
        T* first_hi,
        T* second_lo,
        T* second_hi)
{
        const T cost = static_cast<T>(uniform_sums[count]);
        // backward[i]: buckets i + 1 .. 31
        T back_lo[BVH_BUCKETS - 1][N];
        T back_hi[BVH_BUCKETS - 1][N];
        T back_cost[BVH_BUCKETS - 1];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                back_lo[BVH_BUCKETS - 2][d] = bucket_lo[BVH_BUCKETS - 1][d];
                back_hi[BVH_BUCKETS - 2][d] = bucket_hi[BVH_BUCKETS - 1][d];
        }
        back_cost[BVH_BUCKETS - 2] = static_cast<T>(uniform_sums[bucket_count[BVH_BUCKETS - 1]]);
        for (int i = BVH_BUCKETS - 2; i > 0; --i)
        {
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        back_lo[i - 1][d] = back_lo[i][d];
                        back_hi[i - 1][d] = back_hi[i][d];
                }
                back_cost[i - 1] = back_cost[i];
                if (bucket_count[i] > 0)
                {
                        bvh_merge<N>(back_lo[i - 1], back_hi[i - 1], bucket_lo[i], bucket_hi[i]);
                        back_cost[i - 1] = back_cost[i] + static_cast<T>(uniform_sums[bucket_count[i]]);
                }
        }
        const T surface_r = 1 / bvh_surface<N>(lo, hi);
        T split_cost = Limits<T>::MAX;
        int index = -1;
        T f_lo[N];
        T f_hi[N];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                f_lo[d] = bucket_lo[0][d];
                f_hi[d] = bucket_hi[0][d];
        }
        T f_cost = static_cast<T>(uniform_sums[bucket_count[0]]);
        T best_lo[N];
        T best_hi[N];
        for (int i = 0; i < BVH_BUCKETS - 1; ++i)
        {
                if (i > 0 && bucket_count[i] > 0)
                {
                        bvh_merge<N>(f_lo, f_hi, bucket_lo[i], bucket_hi[i]);
                        f_cost = f_cost + static_cast<T>(uniform_sums[bucket_count[i]]);
                }
                const T f = f_cost * bvh_surface<N>(f_lo, f_hi);
                const T b = back_cost[i] * bvh_surface<N>(back_lo[i], back_hi[i]);
                const T c = interior_cost + (f + b) * surface_r;
                if (c < split_cost)
                {
                        split_cost = c;
                        index = i;
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                best_lo[d] = f_lo[d];
                                best_hi[d] = f_hi[d];
                        }
                }
        }
        if (split_cost >= cost)
        {
                return -1;
        }
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                first_lo[d] = best_lo[d];
                first_hi[d] = best_hi[d];
                second_lo[d] = back_lo[index][d];
                second_hi[d] = back_hi[index][d];
        }
        return index;
}

// ---------------------------------------------------------------------------
// block reductions of keys

template <typename K>
__device__ K bvh_warp_min(K v)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
                const K w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w < v ? w : v;
        }
        return v;
}

template <typename K>
__device__ K bvh_warp_max(K v)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
                const K w = __shfl_xor_sync(0xffffffffu, v, o);
                v = v < w ? w : v;
        }
        return v;
}

// ---------------------------------------------------------------------------
// set-up: object bounds and centres, the root bounds

template <int N, typename T>
__global__ void bvh_objects_kernel(
        const double* __restrict__ vertices,
        const int* __restrict__ facets, // global vertex indices, N per facet
        const int count,
        BvhObject<N, T>* __restrict__ objects,
        typename BvhKey<T>::K* __restrict__ root_keys) // [2N]: lo, hi
{
        using Key = BvhKey<T>;
        using K = typename Key::K;
        const int f = blockIdx.x * blockDim.x + threadIdx.x;
        K lo_key[N];
        K hi_key[N];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                lo_key[d] = Key::HIGH;
                hi_key[d] = Key::LOW;
        }
        if (f < count)
        {
                BvhObject<N, T> o;
                {
                        const long long v = facets[static_cast<long long>(f) * N];
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                o.lo[d] = static_cast<T>(vertices[v * N + d]);
                                o.hi[d] = o.lo[d];
                        }
                }
#pragma unroll
                for (int k = 1; k < N; ++k)
                {
                        const long long v = facets[static_cast<long long>(f) * N + k];
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                const T p = static_cast<T>(vertices[v * N + d]);
                                o.lo[d] = (p < o.lo[d]) ? p : o.lo[d];
                                o.hi[d] = (o.hi[d] < p) ? p : o.hi[d];
                        }
                }
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        o.c[d] = (o.lo[d] + o.hi[d]) * T(0.5);
                        lo_key[d] = Key::key(o.lo[d]);
                        hi_key[d] = Key::key(o.hi[d]);
                }
                o.index = static_cast<unsigned>(f);
                objects[f] = o;
        }
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                const K a = bvh_warp_min(lo_key[d]);
                const K b = bvh_warp_max(hi_key[d]);
                if ((threadIdx.x & 31) == 0)
                {
                        atomicMin(&root_keys[d], a);
                        atomicMax(&root_keys[N + d], b);
                }
        }
}

template <int N, typename T>
__device__ void bvh_init_task(BvhTask<N, T>& t)
{
        using Key = BvhKey<T>;
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                t.center_lo[d] = Key::HIGH;
                t.center_hi[d] = Key::LOW;
        }
        for (int b = 0; b < BVH_BUCKETS; ++b)
        {
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        t.bucket_lo[b][d] = Key::HIGH;
                        t.bucket_hi[b][d] = Key::LOW;
                }
                t.bucket_count[b] = 0;
        }
        t.split = -1;
        t.middle = 0;
        t.swaps = 0;
}

// A node of [begin, end) with its bounds, child `side` of interior node
// `parent`: a task of the next level, or a small task.
template <int N, typename T>
__device__ void bvh_emit(
        const int begin,
        const int end,
        const int parent,
        const int side,
        const T* lo,
        const T* hi,
        BvhTask<N, T>* next_tasks,
        BvhChunk* next_chunks,
        BvhSmallTask<N, T>* small,
        BvhCounters* counters)
{
        const int count = end - begin;
        if (count <= BVH_SMALL)
        {
                const int s = atomicAdd(&counters->small, 1);
                BvhSmallTask<N, T>& st = small[s];
                st.begin = begin;
                st.end = end;
                st.parent = parent;
                st.side = side;
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        st.lo[d] = lo[d];
                        st.hi[d] = hi[d];
                }
                return;
        }
        const int ti = atomicAdd(&counters->tasks, 1);
        const int chunk_count = (count + BVH_CHUNK - 1) / BVH_CHUNK;
        const int cb = atomicAdd(&counters->chunks, chunk_count);
        BvhTask<N, T>& t = next_tasks[ti];
        t.begin = begin;
        t.end = end;
        t.parent = parent;
        t.side = side;
        t.chunk_begin = cb;
        t.chunk_count = chunk_count;
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                t.lo[d] = lo[d];
                t.hi[d] = hi[d];
        }
        bvh_init_task(t);
        for (int c = 0; c < chunk_count; ++c)
        {
                BvhChunk& ch = next_chunks[cb + c];
                ch.task = ti;
                ch.begin = begin + c * BVH_CHUNK;
                ch.end = min(end, begin + (c + 1) * BVH_CHUNK);
        }
}

template <int N, typename T>
__device__ void bvh_set_child(BvhBuildNode<N, T>* inner, const int parent, const int side, const int ref,
                              BvhCounters* counters)
{
        if (parent < 0)
        {
                counters->root = ref;
        }
        else
        {
                inner[parent].child[side] = ref;
        }
}

template <int N, typename T>
__device__ void bvh_write_leaf(
        const int begin,
        const int end,
        const int parent,
        const int side,
        const T* lo,
        const T* hi,
        BvhBuildNode<N, T>* leaves,
        BvhBuildNode<N, T>* inner,
        int* leaf_list,
        BvhCounters* counters)
{
        BvhBuildNode<N, T>& n = leaves[begin];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                n.lo[d] = lo[d];
                n.hi[d] = hi[d];
        }
        n.axis = 0;
        n.parent = parent;
        n.side = side;
        n.begin = begin;
        n.count = end - begin;
        if (end - begin > 0xffff)
        {
                atomicMax(&counters->error, 2);
        }
        leaf_list[atomicAdd(&counters->leaves, 1)] = begin;
        bvh_set_child(inner, parent, side, begin * 2 + 1, counters);
}

template <int N, typename T>
__device__ void bvh_write_inner(
        const int id,
        const int axis,
        const int parent,
        const int side,
        const T* lo,
        const T* hi,
        BvhBuildNode<N, T>* inner,
        int* inner_list,
        BvhCounters* counters)
{
        BvhBuildNode<N, T>& n = inner[id];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                n.lo[d] = lo[d];
                n.hi[d] = hi[d];
        }
        n.axis = axis;
        n.parent = parent;
        n.side = side;
        n.visits = 0;
        inner_list[atomicAdd(&counters->inner, 1)] = id;
        bvh_set_child(inner, parent, side, id * 2, counters);
}

// the root: a task, a small task or (one object) a leaf
template <int N, typename T>
__global__ void bvh_root_kernel(
        const int count,
        const typename BvhKey<T>::K* __restrict__ root_keys,
        BvhTask<N, T>* tasks,
        BvhChunk* chunks,
        BvhSmallTask<N, T>* small,
        BvhCounters* counters)
{
        T lo[N];
        T hi[N];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                lo[d] = BvhKey<T>::value(root_keys[d]);
                hi[d] = BvhKey<T>::value(root_keys[N + d]);
        }
        bvh_emit<N, T>(0, count, -1, 0, lo, hi, tasks, chunks, small, counters);
}

// ---------------------------------------------------------------------------
// one level of the large nodes

// centroid bounds of each task
template <int N, typename T>
__global__ void __launch_bounds__(BVH_THREADS) bvh_center_kernel(
        BvhTask<N, T>* __restrict__ tasks,
        const BvhChunk* __restrict__ chunks,
        const BvhObject<N, T>* __restrict__ objects)
{
        using Key = BvhKey<T>;
        using K = typename Key::K;
        __shared__ K s_lo[BVH_THREADS / 32][N];
        __shared__ K s_hi[BVH_THREADS / 32][N];
        const BvhChunk ch = chunks[blockIdx.x];
        K lo[N];
        K hi[N];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                lo[d] = Key::HIGH;
                hi[d] = Key::LOW;
        }
        for (int p = ch.begin + threadIdx.x; p < ch.end; p += BVH_THREADS)
        {
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        const K k = Key::key(objects[p].c[d]);
                        lo[d] = k < lo[d] ? k : lo[d];
                        hi[d] = hi[d] < k ? k : hi[d];
                }
        }
        const int warp = threadIdx.x / 32;
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                const K a = bvh_warp_min(lo[d]);
                const K b = bvh_warp_max(hi[d]);
                if ((threadIdx.x & 31) == 0)
                {
                        s_lo[warp][d] = a;
                        s_hi[warp][d] = b;
                }
        }
        __syncthreads();
        if (threadIdx.x < N)
        {
                const int d = threadIdx.x;
                K a = s_lo[0][d];
                K b = s_hi[0][d];
                for (int w = 1; w < BVH_THREADS / 32; ++w)
                {
                        a = s_lo[w][d] < a ? s_lo[w][d] : a;
                        b = b < s_hi[w][d] ? s_hi[w][d] : b;
                }
                BvhTask<N, T>& t = tasks[ch.task];
                atomicMin(&t.center_lo[d], a);
                atomicMax(&t.center_hi[d], b);
        }
}

template <int N, typename T>
__device__ BvhAxis<N, T> bvh_task_axis(const BvhTask<N, T>& t)
{
        T lo[N];
        T hi[N];
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                lo[d] = BvhKey<T>::value(t.center_lo[d]);
                hi[d] = BvhKey<T>::value(t.center_hi[d]);
        }
        return BvhAxis<N, T>::from(lo, hi);
}

// bucket of every object, bucket bounds and counts of each task
template <int N, typename T>
__global__ void __launch_bounds__(BVH_THREADS) bvh_bin_kernel(
        BvhTask<N, T>* __restrict__ tasks,
        const BvhChunk* __restrict__ chunks,
        const BvhObject<N, T>* __restrict__ objects,
        unsigned char* __restrict__ buckets)
{
        using Key = BvhKey<T>;
        using K = typename Key::K;
        __shared__ K s_lo[BVH_BUCKETS][N];
        __shared__ K s_hi[BVH_BUCKETS][N];
        __shared__ unsigned s_count[BVH_BUCKETS];
        const BvhChunk ch = chunks[blockIdx.x];
        BvhTask<N, T>& t = tasks[ch.task];
        const BvhAxis<N, T> ax = bvh_task_axis(t);
        if (ax.point)
        {
                return; // a leaf: the whole block
        }
        for (int i = threadIdx.x; i < BVH_BUCKETS * N; i += BVH_THREADS)
        {
                s_lo[i / N][i % N] = Key::HIGH;
                s_hi[i / N][i % N] = Key::LOW;
        }
        if (threadIdx.x < BVH_BUCKETS)
        {
                s_count[threadIdx.x] = 0;
        }
        __syncthreads();
        for (int p = ch.begin + threadIdx.x; p < ch.end; p += BVH_THREADS)
        {
                const BvhObject<N, T>& o = objects[p];
                const int b = ax.bucket(o.c[ax.axis]);
                buckets[p] = static_cast<unsigned char>(b);
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        atomicMin(&s_lo[b][d], Key::key(o.lo[d]));
                        atomicMax(&s_hi[b][d], Key::key(o.hi[d]));
                }
                atomicAdd(&s_count[b], 1u);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < BVH_BUCKETS * N; i += BVH_THREADS)
        {
                const int b = i / N;
                const int d = i % N;
                if (s_count[b] > 0)
                {
                        atomicMin(&t.bucket_lo[b][d], s_lo[b][d]);
                        atomicMax(&t.bucket_hi[b][d], s_hi[b][d]);
                }
        }
        if (threadIdx.x < BVH_BUCKETS && s_count[threadIdx.x] > 0)
        {
                atomicAdd(&t.bucket_count[threadIdx.x], s_count[threadIdx.x]);
        }
}

// the SAH decision of every task; children to the next level
template <int N, typename T>
__global__ void bvh_split_kernel(
        BvhTask<N, T>* __restrict__ tasks,
        const int task_count,
        const double* __restrict__ uniform_sums,
        const T interior_cost,
        BvhTask<N, T>* __restrict__ next_tasks,
        BvhChunk* __restrict__ next_chunks,
        BvhSmallTask<N, T>* __restrict__ small,
        BvhBuildNode<N, T>* __restrict__ leaves,
        BvhBuildNode<N, T>* __restrict__ inner,
        int* __restrict__ leaf_list,
        int* __restrict__ inner_list,
        BvhCounters* __restrict__ counters)
{
        const int ti = blockIdx.x * blockDim.x + threadIdx.x;
        if (ti >= task_count)
        {
                return;
        }
        BvhTask<N, T>& t = tasks[ti];
        const BvhAxis<N, T> ax = bvh_task_axis(t);
        int split = -1;
        T first_lo[N];
        T first_hi[N];
        T second_lo[N];
        T second_hi[N];
        if (!ax.point)
        {
                T blo[BVH_BUCKETS][N];
                T bhi[BVH_BUCKETS][N];
                for (int b = 0; b < BVH_BUCKETS; ++b)
                {
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                blo[b][d] = BvhKey<T>::value(t.bucket_lo[b][d]);
                                bhi[b][d] = BvhKey<T>::value(t.bucket_hi[b][d]);
                        }
                }
                split = bvh_decide<N, T>(blo, bhi, t.bucket_count, static_cast<unsigned>(t.end - t.begin), t.lo, t.hi,
                                         uniform_sums, interior_cost, first_lo, first_hi, second_lo, second_hi);
        }
        t.split = split;
        if (split < 0)
        {
                bvh_write_leaf<N, T>(t.begin, t.end, t.parent, t.side, t.lo, t.hi, leaves, inner, leaf_list, counters);
                return;
        }
        int middle = 0;
        for (int b = 0; b <= split; ++b)
        {
                middle += static_cast<int>(t.bucket_count[b]);
        }
        t.middle = middle;
        if (middle == 0 || middle == t.end - t.begin)
        {
                atomicMax(&counters->error, 1);
                return;
        }
        const int id = t.begin + middle - 1;
        bvh_write_inner<N, T>(id, ax.axis, t.parent, t.side, t.lo, t.hi, inner, inner_list, counters);
        bvh_emit<N, T>(t.begin, t.begin + middle, id, 0, first_lo, first_hi, next_tasks, next_chunks, small,
                       counters);
        bvh_emit<N, T>(t.begin + middle, t.end, id, 1, second_lo, second_hi, next_tasks, next_chunks, small,
                       counters);
}

// Per chunk of a splitting task: the objects on the wrong side, counted
// (rank == nullptr) or ranked into `first` / `second` by position.
template <int N, typename T>
__global__ void __launch_bounds__(BVH_THREADS) bvh_misplaced_kernel(
        BvhTask<N, T>* __restrict__ tasks,
        const BvhChunk* __restrict__ chunks,
        const unsigned char* __restrict__ buckets,
        int2* __restrict__ chunk_counts, // per chunk: misplaced in the first part, in the second part
        const int2* __restrict__ chunk_offsets,
        int* __restrict__ first,  // positions of the misplaced objects of the first part, by rank
        int* __restrict__ second) // those of the second part, by rank from the left
{
        constexpr int PER = BVH_CHUNK / BVH_THREADS;
        __shared__ int s_a[BVH_THREADS / 32];
        __shared__ int s_b[BVH_THREADS / 32];
        const BvhChunk ch = chunks[blockIdx.x];
        const BvhTask<N, T>& t = tasks[ch.task];
        if (t.split < 0)
        {
                return;
        }
        const int boundary = t.begin + t.middle;
        // this thread's PER consecutive objects
        const int p0 = ch.begin + threadIdx.x * PER;
        unsigned fa = 0; // bit j: object p0 + j belongs to the second part but lies in the first
        unsigned fb = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j)
        {
                const int p = p0 + j;
                if (p < ch.end)
                {
                        const bool in_first = buckets[p] <= t.split;
                        if (p < boundary && !in_first)
                        {
                                fa |= 1u << j;
                        }
                        if (p >= boundary && in_first)
                        {
                                fb |= 1u << j;
                        }
                }
        }
        const int ca = __popc(fa);
        const int cb = __popc(fb);
        // exclusive block scans of ca and cb
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x / 32;
        int sa = ca;
        int sb = cb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
                const int xa = __shfl_up_sync(0xffffffffu, sa, o);
                const int xb = __shfl_up_sync(0xffffffffu, sb, o);
                if (lane >= o)
                {
                        sa += xa;
                        sb += xb;
                }
        }
        if (lane == 31)
        {
                s_a[warp] = sa;
                s_b[warp] = sb;
        }
        __syncthreads();
        int wa = 0;
        int wb = 0;
        int ta = 0;
        int tb = 0;
        for (int w = 0; w < BVH_THREADS / 32; ++w)
        {
                if (w < warp)
                {
                        wa += s_a[w];
                        wb += s_b[w];
                }
                ta += s_a[w];
                tb += s_b[w];
        }
        if (!chunk_offsets)
        {
                if (threadIdx.x == 0)
                {
                        chunk_counts[blockIdx.x] = make_int2(ta, tb);
                }
                return;
        }
        int ra = chunk_offsets[blockIdx.x].x + wa + sa - ca;
        int rb = chunk_offsets[blockIdx.x].y + wb + sb - cb;
#pragma unroll
        for (int j = 0; j < PER; ++j)
        {
                if (fa & (1u << j))
                {
                        first[t.begin + ra++] = p0 + j;
                }
                if (fb & (1u << j))
                {
                        second[t.begin + rb++] = p0 + j;
                }
        }
}

// per task: offsets of its chunks' counts, and the number of pairs
template <int N, typename T>
__global__ void bvh_offsets_kernel(
        BvhTask<N, T>* __restrict__ tasks,
        const int task_count,
        const int2* __restrict__ chunk_counts,
        int2* __restrict__ chunk_offsets,
        BvhCounters* __restrict__ counters)
{
        const int ti = blockIdx.x * blockDim.x + threadIdx.x;
        if (ti >= task_count)
        {
                return;
        }
        BvhTask<N, T>& t = tasks[ti];
        if (t.split < 0)
        {
                return;
        }
        int a = 0;
        int b = 0;
        for (int c = 0; c < t.chunk_count; ++c)
        {
                const int2 n = chunk_counts[t.chunk_begin + c];
                chunk_offsets[t.chunk_begin + c] = make_int2(a, b);
                a += n.x;
                b += n.y;
        }
        if (a != b)
        {
                atomicMax(&counters->error, 3);
        }
        t.swaps = a;
}

// the i-th misplaced object of the first part swaps with the i-th of the
// second part counted from the right
template <int N, typename T>
__global__ void __launch_bounds__(BVH_THREADS) bvh_swap_kernel(
        const BvhTask<N, T>* __restrict__ tasks,
        const BvhChunk* __restrict__ chunks,
        const int* __restrict__ first,
        const int* __restrict__ second,
        BvhObject<N, T>* __restrict__ objects)
{
        const BvhChunk ch = chunks[blockIdx.x];
        const BvhTask<N, T>& t = tasks[ch.task];
        if (t.split < 0)
        {
                return;
        }
        for (int p = ch.begin + threadIdx.x; p < ch.end; p += BVH_THREADS)
        {
                const int i = p - t.begin;
                if (i < t.swaps)
                {
                        const int a = first[t.begin + i];
                        const int b = second[t.begin + t.swaps - 1 - i];
                        const BvhObject<N, T> x = objects[a];
                        objects[a] = objects[b];
                        objects[b] = x;
                }
        }
}

// ---------------------------------------------------------------------------
// small nodes: one warp builds the whole subtree, one object per lane

// position of the n-th (from 0) set bit of `mask`
__device__ inline int bvh_nth_bit(unsigned mask, const int n)
{
        for (int i = 0; i < n; ++i)
        {
                mask &= mask - 1u;
        }
        return __ffs(static_cast<int>(mask)) - 1;
}

template <int N, typename T>
struct BvhStackEntry final
{
        int begin; // relative to the task
        int end;
        int parent;
        int side;
        T lo[N];
        T hi[N];
};

template <int N, typename T>
__global__ void __launch_bounds__(128) bvh_small_kernel(
        const BvhSmallTask<N, T>* __restrict__ small,
        const int small_count,
        const double* __restrict__ uniform_sums,
        const T interior_cost,
        BvhObject<N, T>* __restrict__ objects,
        BvhBuildNode<N, T>* __restrict__ leaves,
        BvhBuildNode<N, T>* __restrict__ inner,
        int* __restrict__ leaf_list,
        int* __restrict__ inner_list,
        BvhCounters* __restrict__ counters)
{
        using Key = BvhKey<T>;
        using K = typename Key::K;
        constexpr int WARPS = 4;
        __shared__ BvhStackEntry<N, T> s_stack[WARPS][BVH_SMALL];
        const int warp = threadIdx.x / 32;
        const int lane = threadIdx.x & 31;
        const int si = blockIdx.x * WARPS + warp;
        if (si >= small_count)
        {
                return;
        }
        const BvhSmallTask<N, T> task = small[si];
        const int count = task.end - task.begin;
        BvhObject<N, T> o;
        if (lane < count)
        {
                o = objects[task.begin + lane];
        }
        BvhStackEntry<N, T>* const stack = s_stack[warp];
        int top = 0;
        if (lane == 0)
        {
                BvhStackEntry<N, T>& e = stack[0];
                e.begin = 0;
                e.end = count;
                e.parent = task.parent;
                e.side = task.side;
#pragma unroll
                for (int d = 0; d < N; ++d)
                {
                        e.lo[d] = task.lo[d];
                        e.hi[d] = task.hi[d];
                }
        }
        top = 1;
        __syncwarp();
        while (top > 0)
        {
                --top;
                const BvhStackEntry<N, T> e = stack[top];
                __syncwarp();
                const int n = e.end - e.begin;
                const bool active = lane >= e.begin && lane < e.end;
                int split = -1;
                int middle = 0;
                int axis = 0;
                T first_lo[N];
                T first_hi[N];
                T second_lo[N];
                T second_hi[N];
                if (n > 1)
                {
                        // centroid bounds
                        T clo[N];
                        T chi[N];
#pragma unroll
                        for (int d = 0; d < N; ++d)
                        {
                                const K k = Key::key(o.c[d]);
                                clo[d] = Key::value(bvh_warp_min(active ? k : Key::HIGH));
                                chi[d] = Key::value(bvh_warp_max(active ? k : Key::LOW));
                        }
                        const BvhAxis<N, T> ax = BvhAxis<N, T>::from(clo, chi);
                        axis = ax.axis;
                        if (!ax.point)
                        {
                                const int my_bucket = active ? ax.bucket(o.c[ax.axis]) : -1;
                                // lane b gathers bucket b in object order
                                T blo[N];
                                T bhi[N];
                                unsigned bcount = 0;
                                for (int j = e.begin; j < e.end; ++j)
                                {
                                        const int bj = __shfl_sync(0xffffffffu, my_bucket, j);
#pragma unroll
                                        for (int d = 0; d < N; ++d)
                                        {
                                                const T l = __shfl_sync(0xffffffffu, o.lo[d], j);
                                                const T h = __shfl_sync(0xffffffffu, o.hi[d], j);
                                                if (bj == lane)
                                                {
                                                        if (bcount == 0)
                                                        {
                                                                blo[d] = l;
                                                                bhi[d] = h;
                                                        }
                                                        else
                                                        {
                                                                blo[d] = (l < blo[d]) ? l : blo[d];
                                                                bhi[d] = (bhi[d] < h) ? h : bhi[d];
                                                        }
                                                }
                                        }
                                        if (bj == lane)
                                        {
                                                ++bcount;
                                        }
                                }
                                // every lane takes the decision on all buckets
                                T all_lo[BVH_BUCKETS][N];
                                T all_hi[BVH_BUCKETS][N];
                                unsigned all_count[BVH_BUCKETS];
                                for (int b = 0; b < BVH_BUCKETS; ++b)
                                {
#pragma unroll
                                        for (int d = 0; d < N; ++d)
                                        {
                                                all_lo[b][d] = __shfl_sync(0xffffffffu, blo[d], b);
                                                all_hi[b][d] = __shfl_sync(0xffffffffu, bhi[d], b);
                                        }
                                        all_count[b] = __shfl_sync(0xffffffffu, bcount, b);
                                }
                                split = bvh_decide<N, T>(all_lo, all_hi, all_count, static_cast<unsigned>(n), e.lo, e.hi,
                                                         uniform_sums, interior_cost, first_lo, first_hi, second_lo,
                                                         second_hi);
                                if (split >= 0)
                                {
                                        for (int b = 0; b <= split; ++b)
                                        {
                                                middle += static_cast<int>(all_count[b]);
                                        }
                                        // the partition: misplaced objects pair up
                                        const int boundary = e.begin + middle;
                                        const bool in_first = my_bucket <= split;
                                        const unsigned fa =
                                                __ballot_sync(0xffffffffu, active && lane < boundary && !in_first);
                                        const unsigned fb =
                                                __ballot_sync(0xffffffffu, active && lane >= boundary && in_first);
                                        const unsigned below = (1u << lane) - 1u;
                                        const int k = __popc(fa);
                                        int partner = lane;
                                        if (fa & (1u << lane))
                                        {
                                                partner = bvh_nth_bit(fb, k - 1 - __popc(fa & below));
                                        }
                                        else if (fb & (1u << lane))
                                        {
                                                partner = bvh_nth_bit(fa, k - 1 - __popc(fb & below));
                                        }
                                        BvhObject<N, T> x;
#pragma unroll
                                        for (int d = 0; d < N; ++d)
                                        {
                                                x.lo[d] = __shfl_sync(0xffffffffu, o.lo[d], partner);
                                                x.hi[d] = __shfl_sync(0xffffffffu, o.hi[d], partner);
                                                x.c[d] = __shfl_sync(0xffffffffu, o.c[d], partner);
                                        }
                                        x.index = __shfl_sync(0xffffffffu, o.index, partner);
                                        o = x;
                                }
                        }
                }
                const int abs_begin = task.begin + e.begin;
                if (split < 0)
                {
                        if (lane == 0)
                        {
                                bvh_write_leaf<N, T>(abs_begin, task.begin + e.end, e.parent, e.side, e.lo, e.hi, leaves,
                                                     inner, leaf_list, counters);
                        }
                }
                else
                {
                        const int id = abs_begin + middle - 1;
                        if (lane == 0)
                        {
                                bvh_write_inner<N, T>(id, axis, e.parent, e.side, e.lo, e.hi, inner, inner_list,
                                                      counters);
                                BvhStackEntry<N, T>& second = stack[top];
                                second.begin = e.begin + middle;
                                second.end = e.end;
                                second.parent = id;
                                second.side = 1;
                                BvhStackEntry<N, T>& first = stack[top + 1];
                                first.begin = e.begin;
                                first.end = e.begin + middle;
                                first.parent = id;
                                first.side = 0;
#pragma unroll
                                for (int d = 0; d < N; ++d)
                                {
                                        second.lo[d] = second_lo[d];
                                        second.hi[d] = second_hi[d];
                                        first.lo[d] = first_lo[d];
                                        first.hi[d] = first_hi[d];
                                }
                        }
                        top += 2;
                }
                __syncwarp();
        }
        if (lane < count)
        {
                objects[task.begin + lane] = o;
        }
}

// ---------------------------------------------------------------------------
// layout: subtree sizes bottom up, depth-first positions, the records

template <int N, typename T>
__global__ void bvh_sizes_kernel(
        const int* __restrict__ leaf_list,
        const int leaf_count,
        const BvhBuildNode<N, T>* __restrict__ leaves,
        BvhBuildNode<N, T>* inner,
        BvhCounters* counters)
{
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= leaf_count)
        {
                return;
        }
        const BvhBuildNode<N, T>& leaf = leaves[leaf_list[i]];
        int size = 1;
        int parent = leaf.parent;
        int side = leaf.side;
        while (parent >= 0)
        {
                BvhBuildNode<N, T>& p = inner[parent];
                volatile int* const sizes = p.size;
                sizes[side] = size;
                __threadfence();
                if (atomicAdd(&p.visits, 1) == 0)
                {
                        return; // the sibling's thread goes on
                }
                __threadfence();
                size = 1 + sizes[0] + sizes[1];
                side = p.side;
                parent = p.parent;
        }
        counters->root_size = size;
}

template <int N, typename T>
__device__ int bvh_preorder(int parent, int side, const BvhBuildNode<N, T>* inner, int* depth)
{
        int index = 0;
        int d = 0;
        while (parent >= 0)
        {
                const BvhBuildNode<N, T>& p = inner[parent];
                index += 1 + (side == 1 ? p.size[0] : 0);
                side = p.side;
                parent = p.parent;
                ++d;
        }
        *depth = d;
        return index;
}

template <int N, typename T>
__global__ void bvh_preorder_kernel(
        const int* __restrict__ leaf_list,
        const int leaf_count,
        const int* __restrict__ inner_list,
        const int inner_count,
        BvhBuildNode<N, T>* __restrict__ leaves,
        BvhBuildNode<N, T>* __restrict__ inner,
        BvhCounters* __restrict__ counters)
{
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        int depth = 0;
        if (i < leaf_count)
        {
                BvhBuildNode<N, T>& n = leaves[leaf_list[i]];
                n.preorder = bvh_preorder<N, T>(n.parent, n.side, inner, &depth);
                atomicMax(&counters->depth, depth);
        }
        else if (i < leaf_count + inner_count)
        {
                BvhBuildNode<N, T>& n = inner[inner_list[i - leaf_count]];
                n.preorder = bvh_preorder<N, T>(n.parent, n.side, inner, &depth);
        }
}

template <int N, typename T>
__global__ void bvh_write_kernel(
        const int* __restrict__ leaf_list,
        const int leaf_count,
        const int* __restrict__ inner_list,
        const int inner_count,
        const BvhBuildNode<N, T>* __restrict__ leaves,
        const BvhBuildNode<N, T>* __restrict__ inner,
        BvhNode<N, T>* __restrict__ out,
        BvhCounters* __restrict__ counters)
{
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= leaf_count + inner_count)
        {
                return;
        }
        const bool leaf = i < leaf_count;
        const BvhBuildNode<N, T>& n = leaf ? leaves[leaf_list[i]] : inner[inner_list[i - leaf_count]];
        BvhNode<N, T> r;
#pragma unroll
        for (int d = 0; d < N; ++d)
        {
                r.lo[d] = n.lo[d];
                r.hi[d] = n.hi[d];
        }
        if (leaf)
        {
                r.offset = static_cast<std::uint32_t>(n.begin);
                r.count = static_cast<std::uint16_t>(n.count);
                r.axis = 0;
        }
        else
        {
                const int c = n.child[1];
                const BvhBuildNode<N, T>& second = (c & 1) ? leaves[c >> 1] : inner[c >> 1];
                r.offset = static_cast<std::uint32_t>(second.preorder);
                r.count = 0;
                r.axis = static_cast<std::uint16_t>(n.axis);
        }
        if (n.preorder < 0 || n.preorder >= leaf_count + inner_count)
        {
                atomicMax(&counters->error, 4);
                return;
        }
        out[n.preorder] = r;
}

template <int N, typename T>
__global__ void bvh_indices_kernel(const BvhObject<N, T>* __restrict__ objects, const int count,
                                   std::uint32_t* __restrict__ indices)
{
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < count)
        {
                indices[i] = objects[i].index;
        }
}
} // namespace nbpt
