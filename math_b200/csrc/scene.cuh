// Device-resident scene of the n-D painter and its ray queries.
//
// Layout in HBM (all arrays device pointers, one scene per render job):
//   flat[]      flat (n-1)-parallelotopes (walls, light carriers): hyperplane,
//               N-1 slab planes, bounding box, material, attached light
//   solid[]     solid n-parallelotopes: N slabs, bounding box, material
//   meshes[]    one record per mesh shape: root box, node/index/facet offsets
//   nodes[]     binary BVH nodes in depth-first order, as the reference lays
//               them out (src/geometry/accelerators/bvh.h:49-62, bvh.cpp:35-67):
//               box, second-child or first-object offset, object count, axis
//   indices[]   facet index per leaf slot
//   facets[]    (n-1)-simplex records (hyperplane + N-1 barycentric planes),
//               material and vertex-normal indices
//   normals[]   mesh vertex normals (for interpolated shading normals)
//   materials[] roughness and the two GGX colours (f0, rho_ss)
//   lights[]    parallelotope and ball lights
//
// The queries follow src/painter/scenes/scene.cpp:70-189 (origin offset,
// closest hit, any hit) and src/painter/shapes/*.cpp (per-shape tests).
#pragma once

#include "bvh_build.h"
#include "core.cuh"
#include "geometry.cuh"
#include "shading.cuh"

#include <cstdint>

namespace nbpt
{
enum class NormalType : int
{
        NONE = 0,
        USE = 1,
        REVERSE = 2
};

template <int N, typename T>
struct FlatShape final
{
        FlatParallelotope<N, T> shape;
        T lo[N];
        T hi[N];
        int material;
        int light; // index into lights[] or -1
};

template <int N, typename T>
struct SolidShape final
{
        SolidParallelotope<N, T> shape;
        T lo[N];
        T hi[N];
        int material;
};

template <int N, typename T>
struct Facet final
{
        Simplex<N, T> simplex; // plane possibly reversed (facet.cpp:113-118)
        int material;
        int normal_type;
        int normals[N];
        unsigned reverse_mask;
};

template <int N, typename T>
struct BvhNode final
{
        T lo[N];
        T hi[N];
        std::uint32_t offset; // leaf: first index slot; interior: second child
        std::uint16_t count;  // 0 for interior nodes
        std::uint16_t axis;
};

template <int N, typename T>
struct MeshShape final
{
        T lo[N];
        T hi[N];
        int node_offset;
        int index_offset;
        int facet_offset;
};

template <typename T, int C>
struct Material final
{
        T roughness;
        Color<C> f0;
        Color<C> rho_ss;
};

enum class LightType : int
{
        PARALLELOTOPE = 0,
        BALL = 1
};

template <int N, typename T, int C>
struct Light final
{
        int type;
        Vec<N, T> org;             // parallelotope origin or ball centre
        Vec<N, T> vectors[N - 1]; // parallelotope edges or radius-scaled ball basis
        Vec<N, T> normal;          // emission side
        T pdf;                     // 1 / area
        Color<C> radiance;
        T distribution_pdf; // probability of choosing this light
        double cumulative;  // discrete-distribution cumulative probability
        int shape;          // parallelotope: the flat shape that carries it
        T radius_squared;   // ball: square of the radius
};

enum class ProjectorType : int
{
        PERSPECTIVE = 0,
        PARALLEL = 1
};

template <int N, typename T>
struct Projector final
{
        int type;
        Vec<N, T> org;
        Vec<N, T> dir;            // perspective: scaled camera direction; parallel: unit
        Vec<N, T> axes[N - 1];    // normalised screen axes (parallel: times units per pixel)
        Vec<N - 1, T> screen_org; // -size / 2
        int size[N - 1];

        // src/painter/projectors/perspective_projector.cpp:63-69, parallel_projector.cpp:61-67
        NBPT_HD Ray<N, T> ray(const Vec<N - 1, T>& point) const
        {
                Vec<N - 1, T> sp;
#pragma unroll
                for (int i = 0; i < N - 1; ++i)
                {
                        sp[i] = screen_org[i] + point[i];
                }
                Vec<N, T> screen_dir = axes[0] * sp[0];
#pragma unroll
                for (int i = 1; i < N - 1; ++i)
                {
                        screen_dir.multiply_add(axes[i], sp[i]);
                }
                if (type == static_cast<int>(ProjectorType::PERSPECTIVE))
                {
                        return Ray<N, T>::make(org, dir + screen_dir);
                }
                return Ray<N, T>::make(org + screen_dir, dir);
        }
};

template <int N, typename T, int C>
struct DeviceScene final
{
        const FlatShape<N, T>* flat;
        int flat_count;
        const SolidShape<N, T>* solid;
        int solid_count;
        const MeshShape<N, T>* meshes;
        int mesh_count;
        const BvhNode<N, T>* nodes;
        const std::uint32_t* indices;
        const Facet<N, T>* facets;
        const Vec<N, T>* normals;
        const Material<T, C>* materials;
        const Light<N, T, C>* lights;
        int light_count;
        Projector<N, T> projector;
        ShadingConstants<T> shading;
        // create_painter's flat_shading: shade with the geometric normal, not
        // the facets' interpolated vertex normals (a painter's copy sets it)
        int flat_shading = 0;
};

// ---------------------------------------------------------------------------
// hits

enum class HitKind : int
{
        NONE = 0,
        FLAT = 1,
        SOLID = 2,
        FACET = 3
};

// A surface intersection: what was hit, at which distance, and the hit point
// computed from the (offset) ray the way SurfaceIntersection does
// (src/painter/objects.h:108-116).
template <int N, typename T>
struct Hit final
{
        int kind;
        int index; // flat/solid shape index or global facet index
        T distance;
        Vec<N, T> point;

        NBPT_HD explicit operator bool() const
        {
                return kind != static_cast<int>(HitKind::NONE);
        }
};

template <int N, typename T>
struct Normals final
{
        Vec<N, T> geometric;
        Vec<N, T> shading;
};

// Statistics counted per query for the roofline: BVH nodes visited, facet
// records tested and other shapes tested.
struct QueryCounters final
{
        std::uint32_t queries;
        std::uint32_t nodes;
        std::uint32_t facets;
        std::uint32_t shapes;
        std::uint32_t overflows; // queries that ended on a full traversal stack
};

template <int N, typename T, int C>
struct SceneQueries final
{
        const DeviceScene<N, T, C>& s;
        QueryCounters& counters;

        // Closest facet of one mesh hit by the ray with t < max_distance
        // (bvh.h:108-149 traversal, spatial/ray_intersection.h:30-54 leaves).
        NBPT_CALL int mesh_closest(const MeshShape<N, T>& mesh, const Ray<N, T>& ray, T& distance) const
        {
                Vec<N, T> rec;
                unsigned neg = 0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        rec[i] = (ray.dir[i] == 0) ? infinity<T>() : (1 / ray.dir[i]);
                        if (ray.dir[i] < 0)
                        {
                                neg |= 1u << i;
                        }
                }
                const BvhNode<N, T>* const nodes = s.nodes + mesh.node_offset;
                const std::uint32_t* const indices = s.indices + mesh.index_offset;
                const Facet<N, T>* const facets = s.facets + mesh.facet_offset;

                std::uint32_t stack[host::BVH_MAX_DEPTH];
                int top = 0;
                std::uint32_t node_index = 0;
                int result = -1;
                while (true)
                {
                        const BvhNode<N, T>& node = nodes[node_index];
                        ++counters.nodes;
                        bool descend = false;
                        if (box_hit<N>(node.lo, node.hi, ray.org, rec, neg, distance))
                        {
                                if (node.count == 0)
                                {
                                        if (top == host::BVH_MAX_DEPTH)
                                        {
                                                // the builders refuse trees this deep; end the
                                                // query rather than write past the stack
                                                ++counters.overflows;
                                                break;
                                        }
                                        if ((neg >> node.axis) & 1u)
                                        {
                                                stack[top++] = node_index + 1;
                                                node_index = node.offset;
                                        }
                                        else
                                        {
                                                stack[top++] = node.offset;
                                                ++node_index;
                                        }
                                        descend = true;
                                }
                                else
                                {
                                        T min_distance = distance;
                                        int closest = -1;
                                        for (int k = 0; k < node.count; ++k)
                                        {
                                                const std::uint32_t f = indices[node.offset + k];
                                                ++counters.facets;
                                                const T t = facets[f].simplex.intersect(ray);
                                                if (t > 0 && t < min_distance)
                                                {
                                                        min_distance = t;
                                                        closest = f;
                                                }
                                        }
                                        if (closest >= 0)
                                        {
                                                distance = min_distance;
                                                result = closest;
                                        }
                                }
                        }
                        if (!descend)
                        {
                                if (top == 0)
                                {
                                        break;
                                }
                                node_index = stack[--top];
                        }
                }
                return result < 0 ? -1 : result + mesh.facet_offset;
        }

        NBPT_CALL bool mesh_any(const MeshShape<N, T>& mesh, const Ray<N, T>& ray, const T max_distance) const
        {
                Vec<N, T> rec;
                unsigned neg = 0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                        rec[i] = (ray.dir[i] == 0) ? infinity<T>() : (1 / ray.dir[i]);
                        if (ray.dir[i] < 0)
                        {
                                neg |= 1u << i;
                        }
                }
                const BvhNode<N, T>* const nodes = s.nodes + mesh.node_offset;
                const std::uint32_t* const indices = s.indices + mesh.index_offset;
                const Facet<N, T>* const facets = s.facets + mesh.facet_offset;

                std::uint32_t stack[host::BVH_MAX_DEPTH];
                int top = 0;
                std::uint32_t node_index = 0;
                while (true)
                {
                        const BvhNode<N, T>& node = nodes[node_index];
                        ++counters.nodes;
                        bool descend = false;
                        if (box_hit<N>(node.lo, node.hi, ray.org, rec, neg, max_distance))
                        {
                                if (node.count == 0)
                                {
                                        if (top == host::BVH_MAX_DEPTH)
                                        {
                                                // the builders refuse trees this deep; end the
                                                // query rather than write past the stack
                                                ++counters.overflows;
                                                return false;
                                        }
                                        if ((neg >> node.axis) & 1u)
                                        {
                                                stack[top++] = node_index + 1;
                                                node_index = node.offset;
                                        }
                                        else
                                        {
                                                stack[top++] = node.offset;
                                                ++node_index;
                                        }
                                        descend = true;
                                }
                                else
                                {
                                        for (int k = 0; k < node.count; ++k)
                                        {
                                                ++counters.facets;
                                                const T t = facets[indices[node.offset + k]].simplex.intersect(ray);
                                                if (t > 0 && t < max_distance)
                                                {
                                                        return true;
                                                }
                                        }
                                }
                        }
                        if (!descend)
                        {
                                if (top == 0)
                                {
                                        return false;
                                }
                                node_index = stack[--top];
                        }
                }
        }

        // Closest hit of the ray against every shape with t < max_distance,
        // after moving the origin off the surface it leaves
        // (scene.cpp:70-95, 97-123, 161-178).
        NBPT_CALL Hit<N, T> intersect(const Vec<N, T>* geometric_normal, Ray<N, T> ray, T max_distance) const
        {
                ++counters.queries;
                if (geometric_normal)
                {
                        ray.org = offset_ray_org(*geometric_normal, ray);
                }
                Hit<N, T> hit;
                hit.kind = static_cast<int>(HitKind::NONE);
                hit.index = -1;
                T best = max_distance;
                for (int i = 0; i < s.flat_count; ++i)
                {
                        ++counters.shapes;
                        const T t = s.flat[i].shape.intersect(ray);
                        if (t > 0 && t < best)
                        {
                                best = t;
                                hit.kind = static_cast<int>(HitKind::FLAT);
                                hit.index = i;
                        }
                }
                for (int i = 0; i < s.solid_count; ++i)
                {
                        ++counters.shapes;
                        const T t = s.solid[i].shape.intersect_volume(ray, best);
                        if (t >= 0 && t < best)
                        {
                                best = t;
                                hit.kind = static_cast<int>(HitKind::SOLID);
                                hit.index = i;
                        }
                }
                for (int i = 0; i < s.mesh_count; ++i)
                {
                        const MeshShape<N, T>& mesh = s.meshes[i];
                        // the mesh's bound is its root box entry (shapes/mesh.cpp:225-229)
                        if (box_volume<N>(mesh.lo, mesh.hi, ray, best) < 0)
                        {
                                continue;
                        }
                        T distance = best;
                        const int f = mesh_closest(mesh, ray, distance);
                        if (f >= 0)
                        {
                                best = distance;
                                hit.kind = static_cast<int>(HitKind::FACET);
                                hit.index = f;
                        }
                }
                if (!hit)
                {
                        return hit;
                }
                hit.distance = best;
                const Vec<N, T> p = ray.point(best);
                switch (static_cast<HitKind>(hit.kind))
                {
                case HitKind::FLAT:
                        hit.point = s.flat[hit.index].shape.plane.project(p);
                        break;
                case HitKind::SOLID:
                        hit.point = s.solid[hit.index].shape.project(p);
                        break;
                default:
                        hit.point = s.facets[hit.index].simplex.plane.project(p);
                        break;
                }
                return hit;
        }

        // Any hit with t < max_distance (scene.cpp:125-133, 180-189).
        NBPT_CALL bool intersect_any(const Vec<N, T>* geometric_normal, Ray<N, T> ray, const T max_distance) const
        {
                ++counters.queries;
                if (geometric_normal)
                {
                        ray.org = offset_ray_org(*geometric_normal, ray);
                }
                for (int i = 0; i < s.flat_count; ++i)
                {
                        ++counters.shapes;
                        const T t = s.flat[i].shape.intersect(ray);
                        if (t > 0 && t < max_distance)
                        {
                                return true;
                        }
                }
                for (int i = 0; i < s.solid_count; ++i)
                {
                        ++counters.shapes;
                        const T t = s.solid[i].shape.intersect_volume(ray, max_distance);
                        if (t >= 0 && t < max_distance)
                        {
                                return true;
                        }
                }
                for (int i = 0; i < s.mesh_count; ++i)
                {
                        const MeshShape<N, T>& mesh = s.meshes[i];
                        if (box_volume<N>(mesh.lo, mesh.hi, ray, max_distance) < 0)
                        {
                                continue;
                        }
                        if (mesh_any(mesh, ray, max_distance))
                        {
                                return true;
                        }
                }
                return false;
        }

        // ---------------------------------------------------------------
        // surface properties

        __device__ Vec<N, T> geometric_normal(const Hit<N, T>& h) const
        {
                switch (static_cast<HitKind>(h.kind))
                {
                case HitKind::FLAT:
                        return s.flat[h.index].shape.plane.n;
                case HitKind::SOLID:
                        return s.solid[h.index].shape.normal(h.point);
                default:
                        return s.facets[h.index].simplex.plane.n;
                }
        }

        // Interpolated vertex normal of a facet (facet.h:96-126); flat and
        // solid parallelotopes have no shading normal.
        __device__ bool shading_normal(const Hit<N, T>& h, Vec<N, T>& out) const
        {
                if (h.kind != static_cast<int>(HitKind::FACET))
                {
                        return false;
                }
                const Facet<N, T>& f = s.facets[h.index];
                if (f.normal_type == static_cast<int>(NormalType::NONE))
                {
                        out = f.simplex.plane.n;
                        return true;
                }
                T bc[N];
                f.simplex.barycentric(h.point, bc);
                Vec<N, T> r;
                {
                        Vec<N, T> n0 = s.normals[f.normals[0]];
                        if ((f.reverse_mask & 1u) != 0)
                        {
                                n0 = -n0;
                        }
                        r = n0 * bc[0];
                }
#pragma unroll
                for (int i = 1; i < N; ++i)
                {
                        Vec<N, T> ni = s.normals[f.normals[i]];
                        if (((f.reverse_mask >> i) & 1u) != 0)
                        {
                                ni = -ni;
                        }
                        r.multiply_add(ni, bc[i]);
                }
                out = r.normalized();
                return true;
        }

        __device__ int material(const Hit<N, T>& h) const
        {
                switch (static_cast<HitKind>(h.kind))
                {
                case HitKind::FLAT:
                        return s.flat[h.index].material;
                case HitKind::SOLID:
                        return s.solid[h.index].material;
                default:
                        return s.facets[h.index].material;
                }
        }

        __device__ int light(const Hit<N, T>& h) const
        {
                return h.kind == static_cast<int>(HitKind::FLAT) ? s.flat[h.index].light : -1;
        }

        // integrators/com/normals.h:45-64; with flat shading the shading
        // normal is the geometric one, which also ends scene_intersect at its
        // first hit (visibility.h:187-190: the flipped geometric normal never
        // faces the ray)
        __device__ Normals<N, T> compute_normals(const Hit<N, T>& h, const Vec<N, T>& ray_dir) const
        {
                const Vec<N, T> g = geometric_normal(h);
                const bool flip = dot(ray_dir, g) >= 0;
                Normals<N, T> r;
                r.geometric = flip ? -g : g;
                Vec<N, T> sn;
                if (s.flat_shading == 0 && shading_normal(h, sn))
                {
                        r.shading = flip ? -sn : sn;
                }
                else
                {
                        r.shading = r.geometric;
                }
                return r;
        }

        // integrators/com/visibility.h:174-204: a hit whose shading normal
        // faces away from the ray is re-cast up to two more times.
        NBPT_CALL Hit<N, T> scene_intersect(const Vec<N, T>* geometric_normal, const Ray<N, T>& ray, Normals<N, T>& normals)
                const
        {
                Hit<N, T> h = intersect(geometric_normal, ray, infinity<T>());
                if (!h)
                {
                        return h;
                }
                normals = compute_normals(h, ray.dir);
                if (dot(ray.dir, normals.shading) <= 0)
                {
                        return h;
                }
                for (int i = 0; i < 2; ++i)
                {
                        const Vec<N, T> g = geometric_normal_of(h);
                        Ray<N, T> r2 = ray;
                        r2.org = h.point;
                        h = intersect(&g, r2, infinity<T>());
                        if (!h)
                        {
                                return h;
                        }
                }
                normals = compute_normals(h, ray.dir);
                return h;
        }

        __device__ Vec<N, T> geometric_normal_of(const Hit<N, T>& h) const
        {
                return geometric_normal(h);
        }
};
} // namespace nbpt
