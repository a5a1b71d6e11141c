/*
 * nbpt: C ABI of the B200 n-dimensional bidirectional path tracer.
 *
 * This is the drop-in boundary for the CPU painter of cppd/math: it replaces
 * the render path behind the reference's painter API
 *   create_painter(Integrator::BPT, notifier, samples_per_pixel,
 *                  max_pass_count, scene, thread_count, flat_shading)
 *   (src/painter/painter.h:149-157, src/painter/painter.cpp:139-151)
 * and the scene factories it renders
 *   scenes::create_storage_scene      (src/painter/scenes/storage.h:40-47)
 *   shapes::HyperplaneParallelotope   (src/painter/shapes/hyperplane_parallelotope.h:66-77)
 *   shapes::Parallelotope             (src/painter/shapes/parallelotope.h:65-71)
 *   shapes::create_mesh               (src/painter/shapes/mesh.h:32-37)
 *   lights::ParallelotopeLight        (src/painter/lights/parallelotope_light.h:73-83)
 *   lights::BallLight                 (src/painter/lights/ball_light.h:76-90)
 *   projectors::PerspectiveProjector  (src/painter/projectors/perspective_projector.h)
 *   projectors::ParallelProjector     (src/painter/projectors/parallel_projector.h)
 * The reference's Scene interface exposes no geometry (src/painter/objects.h:330-359),
 * so a drop-in re-implements the factories: every scene object is described
 * through the calls below and rendered on the GPU.
 *
 * Conventions: plain pointers and sizes; vectors are arrays of `dimension`
 * doubles; arrays of vectors are row-major.  Functions return 0 (or a
 * non-negative index) on success and a negative status on error, with the
 * message in nbpt_last_error() (thread-local).  No exception crosses the ABI.
 * Objects are not thread-safe; use one object from one thread at a time.
 */
#ifndef NBPT_H
#define NBPT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nbpt_scene nbpt_scene;
typedef struct nbpt_painter nbpt_painter;

enum nbpt_status
{
        NBPT_OK = 0,
        NBPT_ERROR = -1,        /* invalid argument or state, see nbpt_last_error() */
        NBPT_CUDA_ERROR = -2,   /* CUDA runtime error, see nbpt_last_error() */
        NBPT_NO_DEVICE = -3     /* no usable GPU */
};

enum nbpt_precision
{
        NBPT_FLOAT = 0, /* geometry, pdfs and MIS in float (the reference's float instantiation) */
        NBPT_DOUBLE = 1 /* geometry, pdfs and MIS in double */
};

enum nbpt_color
{
        NBPT_RGB = 0,     /* color::Color = RGB<float> */
        NBPT_SPECTRUM = 1 /* color::Spectrum = 64 samples over 380-720 nm */
};

/* Statistics of the painter, as painter::Statistics (src/painter/painter.h:120-132)
 * plus counters of the last pass for the roofline. */
typedef struct nbpt_statistics
{
        long long pass_number;
        long long pixel_count;
        long long ray_count;    /* scene queries of the last pass */
        long long sample_count; /* paths of the last pass (actual samples) */
        double previous_pass_duration; /* seconds, device time of the last pass */
        double paths_seconds;          /* device time of the path kernel, last pass */
        unsigned long long nodes;      /* BVH nodes visited, last pass */
        unsigned long long facets;     /* facet records tested, last pass */
        unsigned long long shapes;     /* other shapes tested, last pass */
        long long kernel_launches;     /* kernels launched by the last pass */
        /* samples of all passes whose colour has a NaN or infinite channel:
         * kept in the image and counted, as the reference logs them
         * (src/painter/pixels/pixels.cpp:107-113) */
        long long nonfinite_samples;
        /* ray queries of all passes that found the BVH traversal stack full
         * (none for trees the scene build accepts); nbpt_painter_wait fails
         * when this is not zero */
        long long stack_overflows;
} nbpt_statistics;

const char* nbpt_last_error(void);
int nbpt_device_count(void);

/* Device buffers released by scenes and painters are cached by the library
 * and reused by later scenes and painters of the same sizes, which spares
 * jobs that follow one another the cost of cudaMalloc and cudaFree.  This
 * returns the cached buffers to the driver; returns the bytes freed. */
long long nbpt_release_cached_memory(void);

/* ---- scene (scenes::create_storage_scene and the shape/light/projector factories) ---- */

nbpt_scene* nbpt_scene_create(int dimension, int precision, int color);
void nbpt_scene_destroy(nbpt_scene* scene);

/* shapes::HyperplaneParallelotope(metalness, roughness, color, alpha, org, vectors[N-1]);
 * returns the shape index. */
int nbpt_scene_add_hyperplane_parallelotope(
        nbpt_scene* scene, double metalness, double roughness, const float* rgb, double alpha,
        const double* org, const double* vectors);

/* shapes::Parallelotope(metalness, roughness, color, alpha, org, vectors[N]) */
int nbpt_scene_add_parallelotope(
        nbpt_scene* scene, double metalness, double roughness, const float* rgb, double alpha,
        const double* org, const double* vectors);

/* One model::mesh::MeshObject<N> of a mesh shape: points [point_count][N],
 * simplex facets [facet_count][N] (vertex indices), the (N+1)x(N+1)
 * object matrix, optional per-point normals (NULL: computed as
 * model::mesh::create_mesh_for_facets does), and the object's material.
 * Objects accumulate until nbpt_scene_add_mesh(). */
int nbpt_scene_add_mesh_object(
        nbpt_scene* scene, const float* points, long long point_count, const int* facets, long long facet_count,
        const double* matrix, const float* normals, float metalness, float roughness, const float* rgb, float alpha);

/* A mesh object read from an n-dimensional OBJ (v, vn, f, usemtl, mtllib
 * with Kd) or STL (ASCII or binary) file, as model::mesh::load reads it
 * (src/model/mesh/file.cpp:86-104, file/load_obj.cpp, file/load_stl.cpp):
 * .obj / .stl are 3-space files, .objN / .stlN N-space ones.  Facets with
 * normals in the file keep them; facets without are flat.  Facets that name a
 * material take its Kd colour, the others the object's colour. */
int nbpt_scene_add_mesh_file(
        nbpt_scene* scene, const char* path, const double* matrix, float metalness, float roughness, const float* rgb,
        float alpha);
/* the dimension of an OBJ or STL file from its name (file_type.cpp) */
int nbpt_mesh_file_dimension(const char* path);

/* shapes::create_mesh(mesh_objects, no clip plane, ...): one mesh shape from
 * the accumulated objects; returns the shape index. */
int nbpt_scene_add_mesh(nbpt_scene* scene);

/* A mesh shape given as the painter's mesh data (src/painter/shapes/mesh/data.h:34-50):
 * transformed vertices and normals [vertex_count][N] (normals may be NULL),
 * facets [facet_count][N], facet_materials [facet_count],
 * material_params [material_count][3] = (metalness, roughness, alpha),
 * material_colors [material_count][channels]. */
int nbpt_scene_add_mesh_data(
        nbpt_scene* scene, long long vertex_count, const double* vertices, const double* normals,
        long long facet_count, const int* facets, const int* facet_materials, int material_count,
        const double* material_params, const float* material_colors);

/* lights::ParallelotopeLight on the hyperplane parallelotope `shape`
 * (hyperplane_parallelotope().set_light_source); returns the light index. */
int nbpt_scene_add_parallelotope_light(nbpt_scene* scene, int shape, const double* direction, const float* rgb);

/* lights::BallLight(center, direction, radius, radiance) */
int nbpt_scene_add_ball_light(
        nbpt_scene* scene, const double* center, const double* direction, double radius, const float* rgb);

/* projectors::PerspectiveProjector(org, dir, screen_axes[N-1], width_view_angle_degrees, screen_size[N-1]) */
int nbpt_scene_set_perspective_projector(
        nbpt_scene* scene, const double* org, const double* dir, const double* axes, double fov_degrees,
        const int* size);

/* projectors::ParallelProjector(org, dir, screen_axes[N-1], units_per_pixel, screen_size[N-1]) */
int nbpt_scene_set_parallel_projector(
        nbpt_scene* scene, const double* org, const double* dir, const double* axes, double units_per_pixel,
        const int* size);

/* background colour (only black is supported) */
int nbpt_scene_set_background(nbpt_scene* scene, const float* rgb);

/* Where nbpt_scene_finalize builds the mesh BVHs (geometry::accelerators::Bvh,
 * src/geometry/accelerators/bvh.cpp:35-86): NBPT_BVH_DEVICE (the default) on
 * the GPU, NBPT_BVH_HOST on the host threads; both give the reference's tree */
#define NBPT_BVH_DEVICE 0
#define NBPT_BVH_HOST 1
int nbpt_scene_set_bvh_builder(nbpt_scene* scene, int builder);

/* Builds the acceleration structures and uploads the scene to the GPU. */
int nbpt_scene_finalize(nbpt_scene* scene);

long long nbpt_scene_pixel_count(const nbpt_scene* scene);
/* samples per pixel actually rendered: spp rounded up to a power of the screen dimension */
int nbpt_scene_actual_spp(const nbpt_scene* scene, int samples_per_pixel);
/* bytes of scene data the scene keeps on the GPU */
long long nbpt_scene_device_bytes(const nbpt_scene* scene);
/* bytes finalize copied from host to device (shapes, BVH, vertices, facets) */
long long nbpt_scene_upload_bytes(const nbpt_scene* scene);
/* host seconds of the scene build, as the reference logs its mesh and BVH
 * build times (src/painter/shapes/mesh.cpp:190-209): seconds[0] mesh
 * ingestion, [1] BVH builds, [2] the rest of nbpt_scene_finalize (device
 * uploads, facet setup on the GPU), [3] the total */
int nbpt_scene_build_seconds(const nbpt_scene* scene, double* seconds);

/* ---- painter (painter::create_painter with Integrator::BPT) ---- */

/* A render of a finalized scene.  Every pass renders samples_per_pixel
 * stratified samples per pixel with per-path random streams derived from
 * (seed, pass, pixel, sample) and accumulates the filtered, trimmed pixel
 * estimator.  max_depth is the reference's MAX_DEPTH (1..8). */
nbpt_painter* nbpt_painter_create(nbpt_scene* scene, int samples_per_pixel, int max_depth, unsigned seed);
/* painter::create_painter(Integrator, ...) (src/painter/painter.h:143-157):
 * NBPT_INTEGRATOR_BPT as nbpt_painter_create; NBPT_INTEGRATOR_PT runs the
 * path tracer with next-event estimation and Russian roulette
 * (src/painter/integrators/pt/pt.cpp:138-170), which ignores max_depth */
#define NBPT_INTEGRATOR_BPT 0
#define NBPT_INTEGRATOR_PT 1
nbpt_painter* nbpt_painter_create_integrator(
        nbpt_scene* scene, int integrator, int samples_per_pixel, int max_depth, unsigned seed);
/* A painter of one slab of the screen, for renders split across GPUs: the
 * rows [slab_begin, slab_end) of the last screen axis.  No reference function
 * (the reference's painter threads share one screen; its pixel order is
 * src/painter/painting/paintbrush.h:162-205).  A pass renders the paths of
 * the slab and of the row on either side (the pixel filter reaches one
 * pixel) and accumulates the slab's own pixels; every path's stream is fixed
 * by (seed, pass, pixel, sample), so the slab's pixels are bit for bit those
 * of the whole-screen painter, and the slabs of a split put together are its
 * image.  Images and samples cover the slab (samples: the slab with its
 * halo rows); sample_count counts every path rendered.  slab_end < 0: the
 * whole screen. */
nbpt_painter* nbpt_painter_create_slab(
        nbpt_scene* scene, int integrator, int samples_per_pixel, int max_depth, unsigned seed, int slab_begin,
        int slab_end);
/* Every painter argument at once: create_painter's integrator, samples per
 * pixel and flat_shading (src/painter/painter.h:149-157; flat shading shades
 * with the geometric normal instead of the facets' interpolated vertex
 * normals, src/painter/integrators/com/normals.h:45-64), the BPT maximum
 * depth, the random streams' seed, the slab as nbpt_painter_create_slab
 * (slab_end < 0: the whole screen), and the type of the per-pixel radiance
 * and weight sums of the estimator (src/painter/pixels/pixels.cpp:83-95,
 * samples/com/merge.h:199-233):
 *   NBPT_PIXEL_SUMS_FLOAT   float, as the reference's Color keeps them
 *                           (src/color/color.h:416-417): the images of a
 *                           double-precision scene are the reference's;
 *   NBPT_PIXEL_SUMS_DOUBLE  double; held-out samples stay float;
 *   NBPT_PIXEL_SUMS_DEFAULT float for a double-precision scene, double for a
 *                           single-precision one (the single-precision trace
 *                           keeps its radiance sums in double).
 * The other painter constructors take NBPT_PIXEL_SUMS_DEFAULT. */
#define NBPT_PIXEL_SUMS_DEFAULT 0
#define NBPT_PIXEL_SUMS_FLOAT 1
#define NBPT_PIXEL_SUMS_DOUBLE 2
typedef struct nbpt_painter_options
{
        int integrator; /* NBPT_INTEGRATOR_BPT or NBPT_INTEGRATOR_PT */
        int samples_per_pixel;
        int max_depth;
        unsigned seed;
        int flat_shading; /* 0 or 1 */
        int slab_begin;
        int slab_end;
        int pixel_sums; /* NBPT_PIXEL_SUMS_* */
        /* device bytes of the per-chunk path buffers (0: a fifth of the
         * device's memory within [4, 32] GiB); a pass runs its paths in
         * chunks of as many as they hold, with the same images whatever the
         * size */
        long long chunk_budget;
} nbpt_painter_options;
nbpt_painter* nbpt_painter_create_options(nbpt_scene* scene, const nbpt_painter_options* options);
void nbpt_painter_destroy(nbpt_painter* painter);

/* ---- passes on a worker thread (the reference painter's thread and its
 * Notifier: src/painter/painter.cpp:77-134, painter.h:36-78) ---- */

/* called on the painter's worker thread after each pass with that pass's
 * images (as nbpt_painter_images), valid until the callback returns; `pass`
 * counts from 1 (Notifier::pass_done, Notifier::images) */
typedef void (*nbpt_pass_callback)(void* user, long long pass, const float* rgb, const float* rgba,
                                   long long pixel_count);
/* Progress within a pass, the GPU's counterpart of the reference's per-pixel
 * notifications (Notifier::pixel_set and thread_busy / thread_free,
 * src/painter/pixels/pixels.cpp:95, painting/thread_notifier.h:27-50): a
 * pass traces its paths in chunks of pixels and calls this after each chunk
 * with the pixels traced so far (the pixel estimate of a pass is formed
 * after all its chunks, so no pixel value changes before the pass's images).
 * `pass` counts from 1; `pixels` is the pixels whose paths the pass renders.
 * It runs on a CUDA host-callback thread: it must return quickly and call no
 * CUDA function. */
typedef void (*nbpt_progress_callback)(void* user, long long pass, long long pixels_done, long long pixels);
/* sets (or, with NULL, removes) the painter's progress callback for the
 * passes enqueued from now on, with nbpt_painter_enqueue or on the worker */
int nbpt_painter_set_progress(nbpt_painter* painter, nbpt_progress_callback on_chunk, void* user);
/* called on the worker thread when a pass fails (Notifier::error_message);
 * the worker then ends */
typedef void (*nbpt_error_callback)(void* user, const char* message);
/* starts max_pass_count passes (0: until nbpt_painter_stop) on a worker
 * thread and returns; while pass k + 1 renders, the images of pass k go to
 * on_pass.  Until the worker ends, the painter's other calls fail. */
int nbpt_painter_start(nbpt_painter* painter, int max_pass_count, nbpt_pass_callback on_pass,
                       nbpt_error_callback on_error, void* user);
/* asks the worker to stop after the pass in flight and waits for it */
int nbpt_painter_stop(nbpt_painter* painter);
/* waits for the worker to end (Painter::wait) */
int nbpt_painter_join(nbpt_painter* painter);
/* 1 while the worker runs, else 0 */
int nbpt_painter_is_running(const nbpt_painter* painter);
/* enqueues `passes` passes on the painter's CUDA stream and returns */
int nbpt_painter_enqueue(nbpt_painter* painter, int passes);
/* waits for the enqueued passes and updates the statistics */
int nbpt_painter_wait(nbpt_painter* painter);
/* images as Pixels::images (src/painter/pixels/pixels.cpp:123-166):
 * rgb [pixels][3] with background, rgba [pixels][4] premultiplied; either may be NULL */
int nbpt_painter_images(nbpt_painter* painter, float* rgb, float* rgba);
/* per-sample output of the last pass: points [pixels][spp][N-1], colors
 * [pixels][spp][channels], valid [pixels][spp] (0: background sample); any may be NULL */
int nbpt_painter_samples(nbpt_painter* painter, double* points, float* colors, unsigned char* valid);
int nbpt_painter_statistics(nbpt_painter* painter, nbpt_statistics* statistics);
/* the CUDA stream (cudaStream_t) the painter's passes run on, for callers
 * that order their own work or events with it */
void* nbpt_painter_stream(nbpt_painter* painter);
/* Stops the painter as the reference's Painter destructor does (stop flag,
 * src/painter/painter.cpp:129-134), from any thread and without waiting: the
 * pass in flight takes no more paths (its image stays incomplete), a worker
 * started by nbpt_painter_start ends after it and reports "cancelled"
 * through on_error, nbpt_painter_wait returns NBPT_ERROR, and the painter
 * takes no more passes. */
int nbpt_painter_cancel(nbpt_painter* painter);

/* ---- job server: continuous batching of renders on one GPU ----
 *
 * No single reference function: the reference runs one painter per render,
 * each with its own worker threads (src/painter/painter.cpp:77-134).  The
 * server runs the passes of many painters at once, each on its own CUDA
 * stream, keeping one pass of every admitted job in flight; jobs submitted
 * while others run are admitted as soon as a slot and device memory allow.
 * Results do not depend on what runs beside a job. */
typedef struct nbpt_server nbpt_server;

enum nbpt_job_state
{
        NBPT_JOB_QUEUED = 0,
        NBPT_JOB_RUNNING = 1,
        NBPT_JOB_DONE = 2,
        NBPT_JOB_FAILED = 3
};

typedef struct nbpt_job_info
{
        int state;            /* nbpt_job_state */
        int passes;
        int passes_done;
        long long footprint;  /* device bytes of the painter and its scene */
        double submitted;     /* seconds since the server started */
        double started;       /* admitted; -1 while queued */
        double finished;      /* done or failed; -1 before */
        /* device clock (CUDA events on the job's stream) of the start of its
         * first pass and the end of its last, in seconds after the server's
         * creation; -1 until the job is done */
        double device_started;
        double device_finished;
} nbpt_job_info;

/* max_jobs jobs run at once within memory_budget device bytes (0: 80 % of
 * the free device memory); a job larger than the budget runs alone. */
nbpt_server* nbpt_server_create(int max_jobs, long long memory_budget);
/* finishes the running jobs, fails the queued ones */
void nbpt_server_destroy(nbpt_server* server);
/* queues `passes` passes of a painter; returns the job id.  The painter and
 * its scene must stay alive and unused by the caller until the job is done. */
long long nbpt_server_submit(nbpt_server* server, nbpt_painter* painter, int passes);
/* queues a render (nbpt_painter_create's arguments and `passes` passes) that
 * the server creates when it admits the job, so a queued job holds no device
 * memory; the scene must stay alive until the job is released */
long long nbpt_server_submit_render(
        nbpt_server* server, nbpt_scene* scene, int samples_per_pixel, int max_depth, unsigned seed, int passes);
/* images and statistics of a done job (nbpt_painter_images / _statistics) */
int nbpt_server_images(nbpt_server* server, long long job, float* rgb, float* rgba);
int nbpt_server_statistics(nbpt_server* server, long long job, nbpt_statistics* statistics);
/* forgets a done or failed job and frees the render the server created for
 * it; until then a done render keeps its device memory */
int nbpt_server_release(nbpt_server* server, long long job);
int nbpt_server_job(nbpt_server* server, long long job, nbpt_job_info* info);
/* Device bytes of per-chunk path buffers for each render the server creates
 * from now on (renders already submitted keep theirs); 0 restores the
 * default, an equal share of the memory budget per job slot and at least
 * 4 GiB.  A pass's paths run in chunks of as many paths as these buffers
 * hold, and each chunk ends in a tail where the persistent path kernels run
 * out of paths; larger chunks shorten the tails, while fewer renders fit in
 * the memory budget at once.  math_b200.tuning picks it by measurement.
 * No reference counterpart: the reference's painter keeps one path per
 * thread (src/painter/painting/painting.cpp:181-206). */
int nbpt_server_set_chunk_budget(nbpt_server* server, long long bytes);
/* the chunk budget of the renders submitted next (bytes), -1 on error */
long long nbpt_server_chunk_budget(const nbpt_server* server);
/* blocks until the job is done or failed; NBPT_ERROR (with the message) if it failed */
int nbpt_server_wait(nbpt_server* server, long long job, nbpt_job_info* info);
/* seconds since the server started, on the clock of nbpt_job_info */
double nbpt_server_time(nbpt_server* server);
/* nbpt_job_cancel: a queued job fails at once with the error "cancelled"; a
 * running job's pass in flight takes no more paths (the reference's painter
 * threads test their stop flag before each pixel,
 * src/painter/painting/integrator_bpt.cpp:90-93), then the job fails the
 * same way; a finished job is left as it is.  Returns without waiting. */
int nbpt_server_cancel(nbpt_server* server, long long job);

/* ---- verification entry points (same arithmetic as the render path) ---- */

/* closest hit (any = 0): kind (0 none, 1 flat, 2 solid, 3 facet), index,
 * distance, point [count][N]; any hit (any = 1): kind = 0/1.
 * rays [count][2N] = (origin, direction). */
int nbpt_scene_trace(
        nbpt_scene* scene, const double* rays, long long count, int any, int* kind, int* index, double* t,
        double* point);

/* Ray queries that allocate nothing.  No counterpart in the reference: an
 * addition for callers that must not allocate device memory while they run,
 * such as a caller whose own allocator or memory pool already holds the
 * free device memory (an allocation here could fail), or a caller on a
 * latency-critical thread (cudaFree synchronizes the whole device, stalling
 * work on every stream).  Same arguments, results and arithmetic as
 * nbpt_scene_trace, which allocates device buffers for every call.
 *
 * The rays and results pass through one fixed scratch array in device
 * memory (2,228,224 bytes per device, part of the library image), so a call
 * takes at most NBPT_TRACE_NOALLOC_MAX_RAYS rays; more are rejected with
 * NBPT_ERROR and a message, before any device work.  Nothing in the scratch
 * needs to start at zero.  The first call on each device looks up the
 * scratch's device address (cudaGetSymbolAddress), which can initialise the
 * CUDA context; make that first call before any stream capture begins.
 * The address is kept for the life of the process: calls after the caller
 * has run cudaDeviceReset on that device are not supported (the reset
 * unloads the module the address belongs to).
 * Calls share the scratch: two calls that overlap on one device, from two
 * host threads, race on it and corrupt each other's results, so serialise
 * them.  The call returns when the results are in the host arrays. */
#define NBPT_TRACE_NOALLOC_MAX_RAYS 16384
int nbpt_scene_trace_noalloc(
        nbpt_scene* scene, const double* rays, long long count, int any, int* kind, int* index, double* t,
        double* point);

/* facet records and BVH of mesh `mesh` (order of creation among meshes):
 * counts = (facets, nodes, indices); planes [facets][N][N+1] (facet
 * hyperplane then N-1 barycentric hyperplanes, each n[N], d);
 * node_lo/node_hi [nodes][N]; node_info [nodes][3] (offset, count, axis);
 * indices [indices]; normal_info [facets][2] (normal type, reverse mask).
 * With planes == NULL only the counts are returned. */
int nbpt_scene_mesh_export(
        nbpt_scene* scene, int mesh, long long* counts, double* planes, double* node_lo, double* node_hi,
        unsigned* node_info, unsigned* indices, int* normal_info);

/* the mesh `mesh` (order of creation among meshes) as ingested on the host,
 * before or after nbpt_scene_finalize, no GPU needed: counts = (vertices,
 * facets, normals); vertices and normals [V][N] transformed as the painter's
 * mesh data (src/painter/shapes/mesh/data.cpp:88-111), the normals computed
 * as src/model/mesh/normals.cpp does when a mesh object has none; facets
 * [F][N].  Any output pointer may be NULL. */
int nbpt_scene_ingested_mesh(nbpt_scene* scene, int mesh, long long* counts, double* vertices, double* normals,
                             int* facets);

/* GGX brdf f and pdf of material `material` (src/shading/ggx/brdf.h:146-194) */
int nbpt_scene_brdf(
        nbpt_scene* scene, int material, const double* n, const double* v, const double* l, float* f, double* pdf);
/* one brdf sample from the stream seed_seq(seed[0..seed_words)) */
int nbpt_scene_brdf_sample(
        nbpt_scene* scene, int material, const double* n, const double* v, const unsigned* seed, int seed_words,
        double* l, double* pdf, float* f);
/* one leave (kind 0) or arrive (kind 1) sample of light `light`;
 * leave: out = [org N, dir N, normal N, pdf_pos, pdf_dir];
 * arrive: out = [l N, pdf, distance] */
int nbpt_scene_light_sample(
        nbpt_scene* scene, int light, int kind, const unsigned* seed, int seed_words, const double* point,
        double* out, float* radiance);

/* test hook: the next `count` renders the server creates at admission fail as
 * if cudaMalloc had run out of device memory (the server puts them back at the
 * head of its queue in arrival order) */
int nbpt_test_server_fail_allocations(nbpt_server* server, int count);
/* test hook: while hold is 1 the server admits no job (queued jobs wait) */
int nbpt_test_server_hold(nbpt_server* server, int hold);
/* raw PCG32 draws and uniform [0, 1) draws of a seed_seq stream, computed on the GPU */
int nbpt_test_pcg(const unsigned* seed, int seed_words, int count, unsigned* out);
int nbpt_test_canonical(const unsigned* seed, int seed_words, int count, int use_double, double* out);
/* the host BVH build alone (no GPU needed): node count and the depth of the
 * deepest leaf of the facet BVH of a mesh (vertices [vertex_count][dimension],
 * facets [facet_count][dimension]); NBPT_ERROR when the tree is deeper than the
 * traversal stack (64 entries, the reference's BvhStack:
 * src/geometry/accelerators/bvh_stack.h:26), as nbpt_scene_finalize reports */
int nbpt_test_bvh_build(int dimension, int precision, const double* vertices, long long vertex_count,
                        const int* facets, long long facet_count, long long* nodes, int* depth);
/* stratified jittered points of one pixel; returns the point count */
int nbpt_test_sj_points(int dimension, int use_double, int spp, const unsigned* seed, int seed_words, double* out);

#ifdef __cplusplus
}
#endif

#endif
