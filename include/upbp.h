/*
 * upbp.h -- C ABI of the B200 UPBP renderer (libupbp_b200.so).
 *
 * Drop-in boundary for the reference's render path.  The reference's only
 * plugin boundary is `struct Renderer` (gpuupbp/renderer/renderer.hpp:46-149):
 *     int32_t init(const SceneLoader*, const Config*, Framebuffer*);  // 0 ok, -1 fail
 *     void run_iteration(int iteration);                              // adds into Framebuffer
 *     void cleanup();
 * called from main (gpuupbp/gpuupbp.cpp:85-135) after parse_commandline
 * (gpuupbp/misc/config.cpp:735-1370) and SceneLoader::load_scene
 * (gpuupbp/misc/scene_loader.hpp:44-76).  Each entry point below names the
 * reference interface it replaces.  Plain pointers and sizes only.
 *
 * Return codes: 0 ok; < 0 host or CUDA errors (UPBP_ERR_*);
 * upbp_run_iteration returns > 0 when the iteration set device status bits
 * (UPBP_STATUS_*: paths that the reference, too, ends early or beams it
 * drops), and the iteration's image is complete all the same.  No
 * exception crosses the ABI.
 * Devices and threads: a context belongs to the device that was current at
 * upbp_create; every entry point works on that device, whichever device the
 * calling thread has current (and leaves the caller's current device as it
 * was).  A context is driven by one host thread at a time; several contexts
 * may be driven from several threads and then run concurrently on the GPU,
 * each on its own stream: a call that launches kernels leases one of 48
 * launch-parameter slots of the device for its duration (a 49th concurrent
 * call waits for a slot).  The caller owns host buffers, the library owns
 * device memory.
 */
#ifndef UPBP_B200_H
#define UPBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
#define UPBP_OK 0
#define UPBP_ERR_ARGS (-1)       /* invalid argument or command line */
#define UPBP_ERR_IO (-2)         /* file could not be read or written */
#define UPBP_ERR_CUDA (-3)       /* a CUDA call failed; see upbp_last_error */
#define UPBP_ERR_NO_DEVICE (-4)  /* no CUDA device / extension not usable */
#define UPBP_ERR_SCENE (-5)      /* scene description is inconsistent */
#define UPBP_ERR_HOST (-6)       /* host memory or thread failure; see upbp_last_error */
#define UPBP_HELP 1              /* the command line asked for help */

/* Device status bits, the reference's RETURN_WITH_ERR codes
 * (gpuupbp/kernel/defs.cuh:36-48) turned into bits, plus capacity bits. */
#define UPBP_STATUS_BOUNDARY_STACK (1u << 0)
#define UPBP_STATUS_INTERSECTION_ARRAY (1u << 1)
#define UPBP_STATUS_VOL_SEGMENT_ARRAY (1u << 2)
#define UPBP_STATUS_INTERSECTION_STACK (1u << 3)
#define UPBP_STATUS_BEAM_CAPACITY (1u << 4)
#define UPBP_STATUS_TRAVERSAL_STACK (1u << 5)

/* -------------------------------------------------- estimator selection */
/* Same bit values as the reference (gpuupbp/shared/shared_enums.h:28-58). */
#define UPBP_BPT (1u << 2)
#define UPBP_SURF (1u << 3)
#define UPBP_PP3D (1u << 4)
#define UPBP_PB2D (1u << 5)
#define UPBP_BB1D (1u << 6)
#define UPBP_BP2D (1u << 7)
#define UPBP_PREVIOUS (1u << 9)
#define UPBP_COMPATIBLE (1u << 10)
#define UPBP_SPECULAR_ONLY (1u << 12)
#define UPBP_SHORT_BEAM 1
#define UPBP_LONG_BEAM 2

/* Mirror of the reference's Config (gpuupbp/misc/config.hpp:44-120), POD. */
typedef struct upbp_config {
    int scene_id;                 /* -1: OBJ file in scene_path */
    char scene_path[1024];
    uint32_t algorithm_flags;     /* UPBP_BPT | UPBP_SURF | ... */
    int iteration_count;
    float max_time;               /* seconds, < 0 if unused */
    char output_name[1024];
    uint32_t res_x, res_y;
    uint32_t max_path_length, min_path_length;
    float path_count_per_iter;    /* resolved to an absolute count by the parser */
    int query_beam_type;          /* UPBP_SHORT_BEAM / UPBP_LONG_BEAM */
    int photon_beam_type;
    float bb1d_radius_initial, bb1d_radius_alpha, bb1d_used_light_subpath_count;
    float bp2d_radius_initial, bp2d_radius_alpha;
    float pb2d_radius_initial, pb2d_radius_alpha;
    float pp3d_radius_initial, pp3d_radius_alpha;
    float surf_radius_initial, surf_radius_alpha;
    int continuous_output;
    int ignore_fully_spec_paths;
    int gpu_assert;
    uint64_t iteration_offset;
    int do_log;
    int use_shading_normal;
    /* Not in the reference (command line -mis_exact): 1 makes the MIS
     * weights equal the balance heuristic over the full path where the
     * reference's recursion departs from it -- photon-beam merges (BB1D,
     * BP2D) measure the light-side distance from the light vertex instead of
     * the beam's origin, first-segment BB1D beams of finite lights convert to
     * area measure like every other beam, and next-event estimation counts
     * the camera-side sampling pdf of the media its light ray crosses.  0
     * (the default) keeps the reference's weights. */
    int mis_exact;
    /* Not in the reference (command line -guide <n>): when n > 0, a learned
     * proposal guides the scattering of camera subpaths in media -- an MLP
     * (position under a 12-band frequency encoding, direction of travel,
     * one-hot medium -> 8-lobe von Mises-Fisher mixture, blended 50/50 with
     * Henyey-Greenstein), trained on the GPU from the light subpaths'
     * medium vertices after the light passes of iterations 0..n-1 and used
     * from iteration 1 on; its pdf enters every camera-direction pdf of the
     * MIS recursion.  0 (the default): the plain method. */
    int guide_train_iterations;
    /* Not in the reference (command line -checkpoint <file>, -resume <file>):
     * the executable writes a checkpoint (upbp_save_checkpoint) after its
     * last iteration and at every continuous output, and resumes from one
     * (upbp_load_checkpoint) before its first; empty: none. */
    char checkpoint_path[1024];
    char resume_path[1024];
} upbp_config;

/* ------------------------------------------------------ scene records */
typedef struct upbp_material {   /* gpuupbp/shared/material.h:42-61 */
    float diffuse[3];
    float phong[3];
    float phong_exponent;
    float mirror[3];
    float ior;
    int priority;
    int real;
    int medium;                  /* -1 if none */
} upbp_material;

typedef struct upbp_medium {     /* gpuupbp/host/medium.hpp init_homogeneous_medium inputs */
    float absorption[3];
    float emission[3];
    float scattering[3];
    float continuation_prob;
    float mean_cosine;
} upbp_medium;

#define UPBP_LIGHT_AREA 0
#define UPBP_LIGHT_BACKGROUND 1
#define UPBP_LIGHT_DIRECTIONAL 2
#define UPBP_LIGHT_POINT 3
typedef struct upbp_light {      /* gpuupbp/shared/light.h:34-81 */
    int type;
    int mat_id, med_id;          /* enclosing material / medium, -1 for global */
    float p0[3], p1[3], p2[3];   /* area light triangle */
    float intensity[3];          /* area/point/directional intensity; background colour */
    float position[3];           /* point light position; directional light direction */
    float scale;                 /* background scale */
} upbp_light;

typedef struct upbp_camera_desc {  /* gpuupbp/host/camera.hpp init_camera inputs */
    float origin[3], target[3], roll[3];
    float horizontal_fov_deg;
    float focal_dist;
    int mat_id, med_id;
} upbp_camera_desc;

/* Whole scene as flat host arrays (the reference's Scene + Record[],
 * gpuupbp/shared/scene.h:98-129 and scene_loader.hpp:104-108).  Triangle i
 * uses verts[9i..9i+8], normals[12i..12i+11] (three vertex normals then the
 * face normal) and material/light ids; real vs imaginary follows the
 * material's `real` flag. */
typedef struct upbp_scene_desc {
    uint32_t triangle_count;
    const float* verts;
    const float* normals;
    const int32_t* tri_material;
    const int32_t* tri_light;    /* -1 if the triangle is not an emitter */
    uint32_t material_count;
    const upbp_material* materials;
    uint32_t medium_count;
    const upbp_medium* media;
    int32_t global_medium;       /* index into media */
    uint32_t light_count;
    const upbp_light* lights;
    int32_t background_light;    /* index into lights, -1 if none */
    upbp_camera_desc camera;
    uint32_t res_x, res_y;
    float bbox_min[3], bbox_max[3];
    /* Analytic spheres (the reference's Spheres, gpuupbp/shared/scene.h:62-75;
     * only the predefined scenes have them): centre xyz and radius per
     * sphere, and its material.  Real vs imaginary follows the material's
     * `real` flag, as for triangles.  Spheres are never emitters (no loader
     * of the reference gives them a light).  At most UPBP_MAX_SPHERES. */
    uint32_t sphere_count;
    const float* spheres;
    const int32_t* sph_material;
    /* Environment map of the background light `background_light`
     * (light_background_em, gpuupbp/host/env_map.hpp): env_width x env_height
     * RGB floats, rows top to bottom, already scaled and rotated as the
     * reference's loader leaves them; NULL for a constant background.
     * env_width must be at least 2 * env_height (the reference's sampling
     * distribution spans 2 * height columns). */
    uint32_t env_width, env_height;
    const float* env_rgb;
} upbp_scene_desc;

#define UPBP_MAX_SPHERES 64
#define UPBP_PREDEFINED_SCENES 41

typedef struct upbp_scene upbp_scene;   /* host scene owned by the library */
typedef struct upbp_ctx upbp_ctx;       /* device renderer state */

#define UPBP_KERNEL_KINDS 9

typedef struct upbp_stats {
    uint32_t light_vertices, surface_vertices, medium_vertices, light_beams;
    uint32_t light_paths, camera_paths;
    uint32_t status;              /* OR of UPBP_STATUS_* seen so far */
    uint32_t iterations_done;
    double ms_light, ms_build, ms_camera;   /* last iteration, CUDA events; camera = extend, connection and query kernels */
    uint64_t triangle_count;
    double scene_radius;
    /* Work counters of the last iteration, light pass then camera pass, in
     * the order: BVH node visits, triangle tests, rays cast, photon-point
     * candidates, accepted point merges, beam-chunk candidates, accepted beam
     * merges, light-vertex records read by BPT connections. */
    uint64_t work_light[8];
    uint64_t work_camera[8];
    uint32_t beam_chunks;         /* leaves of the last beam map */
    uint32_t kernel_launches;     /* this library's kernel launches in the last iteration */
    uint32_t h2d_bytes;           /* host->device bytes of the last iteration (launch parameters, counter pointers) */
    uint32_t d2h_bytes;           /* device->host bytes of the last iteration (counters that size the next launches) */
    /* Pass times summed over the iterations run since the previous
     * upbp_get_stats call (at most the last 64), and their count. */
    double ms_light_sum, ms_build_sum, ms_camera_sum;
    uint32_t timed_iterations;
    /* Radii of the last iteration: bb1d, bp2d, pb2d, pp3d, surf, and the beam
     * radius used for the beam map (max of bb1d and bp2d when enabled). */
    float radius[6];
    /* Per kernel kind -- light pass, camera extend, PB2D, BB1D, SURF, PP3D,
     * BP2D queries, NEE and BPT connections -- work counters of the last
     * iteration and kernel times summed like the pass times above. */
    uint64_t work[UPBP_KERNEL_KINDS][8];
    double ms_kernel_sum[UPBP_KERNEL_KINDS];
    uint32_t segment_queries, point_queries;   /* query records of the last camera pass */
    uint32_t nee_samples, bpt_pairs;           /* deferred connections of the last camera pass */
    /* Training of the learned proposal (its steps and the table bake) in
     * the last iteration and summed like the pass times; zero without it.
     * ms_light excludes it. */
    double ms_guide, ms_guide_sum;
    /* Device time of the scene BVH builds (both classes of triangles) in
     * upbp_create, including the host's orchestration of their levels. */
    double ms_scene_bvh;
    /* Clustering passes (many-cluster passes and the final block's
     * iterations) that built the last iteration's beam map; 0: the
     * Morton-split LBVH (UPBP_BEAM_MAP=lbvh, or the clustering fell back:
     * its passes ran out -- UPBP_PLOC_PASSES caps them -- or its layout
     * check failed). */
    uint32_t beam_map_passes;
} upbp_stats;

/* Replaces: parse_commandline (gpuupbp/misc/config.cpp:735-1370).  Same
 * flags, defaults and errors; returns UPBP_HELP after printing help. */
int upbp_parse_command_line(int argc, const char** argv, upbp_config* out);

/* Replaces: SceneLoader::load_from_obj (gpuupbp/misc/scene_loader_obj.cpp:926-1104)
 * with the reference's OBJ+MTL+AUX semantics. */
int upbp_scene_load_obj(const char* obj_path, uint32_t res_x, uint32_t res_y, upbp_scene** out);
/* Replaces: SceneLoader::load_predefined (gpuupbp/misc/scene_loader_predef.cpp:126).
 * Builds predefined scene scene_id (0 .. UPBP_PREDEFINED_SCENES - 1, the
 * reference's table in gpuupbp/misc/config.cpp:100-548) with the same
 * records as the reference; UPBP_ERR_ARGS for other ids.  Scenes 3, 4, 9
 * and 10 (emitting media, which the renderer does not add on camera paths)
 * are built although the command line refuses them, as the reference's. */
int upbp_scene_load_predefined(int scene_id, uint32_t res_x, uint32_t res_y, upbp_scene** out);
const upbp_scene_desc* upbp_scene_get_desc(const upbp_scene* scene);
void upbp_scene_free(upbp_scene* scene);

/* Replaces: Renderer::init (gpuupbp/renderer/renderer_init.cpp:675-929).
 * The range-query hit list grows with the work up to 2^32 - 2^21 entries (8
 * bytes each); an iteration with more hits runs its searches in rounds.  The
 * environment variable UPBP_MAX_HITS, read here, sets a smaller limit
 * (entries) for hosts with less device memory to spare; it must exceed the
 * neighbours of any single query, or upbp_run_iteration fails with
 * UPBP_ERR_CUDA ("range search made no progress"). */
int upbp_create(const upbp_scene_desc* scene, const upbp_config* config, upbp_ctx** out);
/* Replaces: Renderer::run_iteration (gpuupbp/renderer/renderer.cpp:37-418).
 * Renders iteration `iteration` and adds it to the device accumulation.
 * Synchronous like the reference's: returns when the iteration's work on
 * the device is done, with UPBP_OK, the iteration's UPBP_STATUS_* bits
 * (> 0; upbp_stats.status keeps the OR over all iterations), or an error. */
int upbp_run_iteration(upbp_ctx* ctx, int iteration);
/* Replaces the D->H framebuffer copy + add_framebuffer of run_iteration
 * (renderer.cpp:381-392): adds scale * (device accumulation) into rgb. */
int upbp_accumulate_to_host(upbp_ctx* ctx, float* rgb, double scale);
/* Copies the last iteration's image (W*H*3 floats, not accumulated). */
int upbp_read_iteration(upbp_ctx* ctx, float* rgb);
int upbp_get_stats(upbp_ctx* ctx, upbp_stats* out);
/* Replaces: Renderer::cleanup (gpuupbp/renderer/renderer.cpp:420-508). */
void upbp_destroy(upbp_ctx* ctx);

/* Replaces: save(fb, name) -> tinyexr_wrapper::save_exr
 * (gpuupbp/host/framebuffer.cpp:114-127, misc/tinyexr_wrapper.cpp:34-95):
 * half-float B,G,R channels, uncompressed scanlines. */
int upbp_write_exr(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* Replaces: save_bmp (gpuupbp/host/framebuffer.cpp:129-202): 24-bit BGR,
 * rows bottom up, bytes of min(255, max(0, pow(c, 1/gamma) * 255)) truncated,
 * the reference's 52-byte header after "BM" and no row padding. */
int upbp_write_bmp(const char* path, const float* rgb, uint32_t width, uint32_t height, float gamma);
/* Replaces: save_hdr (gpuupbp/host/framebuffer.cpp:204-233): Radiance RGBE,
 * uncompressed pixels after the "-Y h +X w" line. */
int upbp_write_hdr(const char* path, const float* rgb, uint32_t width, uint32_t height);
/* Replaces: save(fb, name, gamma) (gpuupbp/host/framebuffer.cpp:114-127):
 * the writer chosen by the name's last three characters (bmp, hdr, exr);
 * UPBP_ERR_ARGS for any other. */
int upbp_write_image(const char* path, const float* rgb, uint32_t width, uint32_t height, float gamma);

/* ---- diagnostics (no counterpart in the reference; used by the parity tests)
 * upbp_debug_photons: the last iteration's photon map contents.  kind 0/1:
 * surface/medium photons as 4 floats (x, y, z, vertex-slot bits) in map
 * order; kind 2: beams as 8 floats (origin xyz, length, direction xyz,
 * light-path index bits).  *count receives the total; at most `capacity`
 * records are written.
 * upbp_debug_query: neighbour sets through the estimators' own range
 * queries for the last iteration's maps and radii.  Each query is 8 floats
 * (x y z dx dy dz tmin tmax).  kind 0 SURF and 1 PP3D (points within the
 * radius of x), 2 PB2D (medium photons along the segment), 3 BB1D (beams
 * near the segment), 4 BP2D (beams near x).  counts[i] = set size, ids =
 * up to ids_per_query vertex slots (0-2) or beam indices (3-4) per query. */
int upbp_debug_photons(upbp_ctx* ctx, int kind, float* out, uint32_t capacity, uint32_t* count);
/* upbp_debug_scene_bvh: the static scene's BVH of one class of triangles
 * (real 1: surfaces, 0: imaginary medium boundaries), built on the device in
 * upbp_create (a binned-SAH tree; the reference builds an OptiX GAS,
 * renderer/renderer_init.cpp:134-289): up to node_capacity floats of nodes
 * (16 words each: left box lo.xyz hi.xyz, right box, left and right links,
 * left and right primitive counts; *count - 1 nodes) and up to tri_capacity
 * floats of triangles in leaf order (12 each: v0 with the original index's
 * bits in w, e1, e2); *count receives the triangle count. */
int upbp_debug_scene_bvh(upbp_ctx* ctx, int real, float* nodes, uint64_t node_capacity, float* tris,
                         uint64_t tri_capacity, uint32_t* count);
int upbp_debug_query(upbp_ctx* ctx, int kind, const float* queries, uint32_t n, uint32_t* counts, uint32_t* ids,
                     uint32_t ids_per_query);

/* Same neighbour-set query as upbp_debug_query, for callers that cannot
 * allocate device memory per call (a fixed device-memory budget, or other
 * streams that must not be stalled by the device-wide synchronisation of
 * cudaFree).  No counterpart in the reference.  Allocates nothing: queries,
 * counts and ids are staged in one static device array of about 4.2 MB that
 * every GPU loading the library holds until exit.  Limits: n <= 4096 queries
 * and ids_per_query <= 256, otherwise UPBP_ERR_ARGS.  The array's device
 * address on the context's device is looked up once, in upbp_create (so a
 * context created after a cudaDeviceReset gets the new one); the call
 * itself resolves nothing.  All calls share the array:
 * calls that overlap on the GPU (several threads, or contexts on one device)
 * race and must be serialised by the caller.  Nothing in the array has to
 * start at zero: every call writes all n counts and clears its own n x
 * ids_per_query id slots before the search, so id slots beyond counts[i]
 * are returned as 0 whatever an earlier call left there. */
int upbp_debug_query_static(upbp_ctx* ctx, int kind, const float* queries, uint32_t n, uint32_t* counts,
                            uint32_t* ids, uint32_t ids_per_query);

/* MIS records of the last iteration, for the FP64 full-path weight check
 * (oracle/mis_fp64.py).  No counterpart in the reference.  Only the
 * recording build of the library, libupbp_b200_misdbg.so (the same sources
 * compiled with UPBP_MIS_DEBUG), keeps them; the production library returns
 * UPBP_ERR_ARGS.  which: 0 light-subpath vertices and 1 camera-subpath
 * vertices (per subpath max_verts records of vtx_words float4, see
 * gpuupbp_b200/csrc/upbp_misdbg.cuh), 2 contributions (ev_words float4
 * each: technique, the FP32 weight applied, the two subpaths and the points
 * where they meet), 3 a header of 64 floats: max_verts, light paths, camera
 * paths, contributions, capacity, vtx_words, ev_words, segments per record,
 * camera origin xyz, direction xyz, image-plane distance, resolution x y,
 * MIS factors surf pp3d pb2d bp2d bb1d, BPT subpath count, light subpaths,
 * photon and query beam types, light count, mis_exact, light tracing from
 * surfaces, max and min path length, scene radius.  *count receives the
 * number of floats; at most `capacity` are written.  The recording build
 * keeps up to 2^20 contributions per iteration (environment variable
 * UPBP_MIS_EVENTS, read by upbp_create, sets another limit). */
int upbp_debug_mis_records(upbp_ctx* ctx, int which, float* out, uint64_t capacity, uint64_t* count);

/* The learned proposal (upbp_config.guide_train_iterations; not in the
 * reference).  upbp_guide_info writes up to n floats: training iterations,
 * Adam steps taken, mean weighted loss of the last batch, training records
 * collected, proposal-table rows, cells per axis, direction bins per axis,
 * media slots, table in use (-1: none yet).
 * upbp_guide_gradients runs the network's FP16 tensor-core forward and
 * backward kernels once on the current device for given FP32 parameters
 * (the layout of gpuupbp_b200/csrc/upbp_guide.cuh: four row-major [in][out]
 * weight matrices 96x64, 64x64, 64x64, 64x48, then their biases; n_params
 * must be their count, 17648, or UPBP_ERR_ARGS is returned), `rows`
 * inputs of 96 floats and targets of 5 floats (unit direction, weight, the
 * phase function's pdf of the direction); it writes the gradient sums of
 * the weighted negative log-likelihood of the target under the sampled
 * blend (1 - a) phase + a mixture (weights normalised to a batch mean of 1;
 * outputs 0-39 the 8-lobe mixture, 40 the logit of a = 0.9 sigmoid) with
 * respect to every parameter, the rows x 48 outputs when `outputs` is not
 * NULL, and the summed loss. */
int upbp_guide_info(upbp_ctx* ctx, float* out, uint32_t n);
int upbp_guide_gradients(const float* params, uint32_t n_params, const float* x, const float* t, uint32_t rows,
                         float* grads, float* outputs, float* loss);

/* Batched rendering of many independent jobs (config 3 of the benchmark
 * spec; no counterpart in the reference, which renders one scene): each job
 * is a context of its own (scene, view, configuration), and
 * upbp_run_batch renders iteration `iteration` of all n of them
 * concurrently -- `workers` host threads (0: 16) take jobs from a shared
 * counter and drive each on the job's own stream and launch-parameter slot,
 * so one job's kernels and host synchronisations overlap the others' -- and
 * returns once every job's iteration is done: the OR of their status bits,
 * or the first job's error.  upbp_set_grid_limit caps the blocks of any of a
 * context's launches (0: no cap; the persistent kernels otherwise fill the
 * GPU), so that kernels of concurrent jobs share the SMs; the batch
 * autotuner in gpuupbp_b200/batch.py picks workers and the cap by timing. */
int upbp_run_batch(upbp_ctx* const* ctxs, uint32_t n, int iteration, int workers);
int upbp_set_grid_limit(upbp_ctx* ctx, uint32_t max_blocks);

/* Checkpoints (not in the reference, which has none): upbp_save_checkpoint
 * writes the context's FP64 accumulation, the number of iterations it has
 * rendered, the status bits seen and, with a learned proposal, its network,
 * Adam state, training records and whether a table is in use, with a
 * fingerprint of the configuration and scene; upbp_load_checkpoint restores
 * them into a context created from the same scene and configuration
 * (UPBP_ERR_ARGS with the reason otherwise, UPBP_ERR_IO if the file cannot
 * be read or written).  Random numbers and radii depend only on the
 * iteration index, so a caller that continues with iteration index =
 * iterations rendered (upbp_stats.iterations_done) renders what the
 * uninterrupted run would have, up to the order of float additions. */
int upbp_save_checkpoint(upbp_ctx* ctx, const char* path);
int upbp_load_checkpoint(upbp_ctx* ctx, const char* path);

/* The CUDA stream (cudaStream_t) all of a context's work is issued on, so a
 * caller can order its own work or time the library with events. */
void* upbp_get_stream(upbp_ctx* ctx);
/* The device index the context was created on (UPBP_ERR_ARGS for NULL). */
int upbp_get_device(const upbp_ctx* ctx);

const char* upbp_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
