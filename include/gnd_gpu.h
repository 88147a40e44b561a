/*
 * gnd_gpu.h -- C ABI of the B200 radiance path (BVH4 traversal + path/volpath
 * wavefront integrators) for Gianduia-style scenes.
 *
 * The library (gianduia_b200/_lib/libgianduia_b200.so) exports two groups:
 *
 *  1. gnd_gpu_*  : the device boundary. Plain pointers and sizes; no C++ types.
 *                  A reference-side integrator plugin binds exactly these.
 *  2. gnd_host_* : the host scene framework (XML + OBJ loading through the same plugin
 *                  names as the reference, SAH BVH build, BVH4 collapse, flattening to
 *                  the device layout) that produces the gnd_scene_desc the device
 *                  boundary consumes.
 *
 * Every function returns a gnd_status (0 = success). On failure the message is
 * available from gnd_last_error() (thread-local). No C++ exception crosses the ABI.
 * Calls on one context are serialised internally, except that a scene upload's copies
 * overlap the other calls (gnd_gpu_scene_upload); contexts are independent.
 */
#ifndef GND_GPU_H
#define GND_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gnd_status;
enum {
    GND_OK = 0,
    GND_ERR_INVALID = 1,      /* bad argument or handle */
    GND_ERR_CUDA = 2,         /* CUDA runtime error (message has the CUDA text) */
    GND_ERR_OOM = 3,          /* device allocation failed */
    GND_ERR_DEVICE_CHECK = 4, /* a kernel's bounds/stack/iteration check tripped */
    GND_ERR_TIMEOUT = 5,      /* a bounded wait ran out */
    GND_ERR_PARSE = 6,        /* scene file could not be loaded */
    GND_ERR_CANCELLED = 7,    /* render or job cancelled */
    GND_ERR_BUDGET = 8,       /* admission refused: over the HBM budget */
    GND_ERR_NO_DEVICE = 9     /* no CUDA device / extension not usable */
};

/* Message of the last failing call on this thread (never NULL). */
const char* gnd_last_error(void);
/* Library version string. */
const char* gnd_version(void);

/* ------------------------------------------------------------------ rays and hits */
/* A ray as the reference's Ray (ray.h:12-33): origin, tMin, direction, tMax. */
typedef struct gnd_ray {
    float o[3];
    float tmin;
    float d[3];
    float tmax;
} gnd_ray;

/* Closest hit (the fields SurfaceInteraction gets from Shape::rayIntersect):
 * t, barycentric u/v (meshes) and the primitive: inst = index of the <primitive> in
 * scene-file order, prim = triangle index within its mesh (-1 for analytic shapes).
 * A miss has inst = -1 and t = +inf. */
typedef struct gnd_hit {
    float t, u, v;
    int32_t inst;
    int32_t prim;
} gnd_hit;

/* ------------------------------------------------------------------ scene description */
/* Flattened scene in the device layout (see gianduia_b200/csrc/include/gnd/layout.h for
 * the record formats). All arrays are host memory owned by the caller; upload copies. */
typedef struct gnd_scene_desc {
    const void* nodes;            /* 128-byte BVH4 nodes, top level and every mesh */
    int64_t num_nodes;
    const void* tris;             /* 48-byte leaf-ordered triangles */
    const void* tri_attrs;        /* 64-byte per-triangle shading attributes */
    int64_t num_tris;
    const void* inst_trav;        /* 64-byte per-instance traversal records */
    const void* inst_shade;       /* 96-byte per-instance shading records */
    int32_t num_instances;
    uint32_t tlas_root;           /* root node of the top level (0xFFFFFFFF: empty) */
    const uint32_t* tlas_list;    /* top-level leaf entries -> instance index */
    int64_t tlas_list_len;
    const void* materials;        /* material records */
    int32_t num_materials;
    int32_t num_emitters;
    const void* emitters;         /* emitter records */
    const void* media;            /* homogeneous media */
    int32_t num_media;
    int32_t num_meshes;
    const void* meshes;           /* mesh records (area sampling) */
    const float* cdf;             /* concatenated per-mesh area CDFs */
    int64_t cdf_len;
    const uint32_t* orig_to_leaf; /* per mesh: original triangle -> leaf slot */
    int64_t orig_to_leaf_len;
    const void* camera;           /* camera record */
    /* render settings read from the scene file */
    int32_t width, height, spp, max_depth;
    int32_t integrator;           /* 0 path_gpu, 1 volpath_gpu */
    int32_t filter;               /* 0 box (radius 0.5), 1 gaussian */
    float filter_radius[2];
    float filter_alpha;
    /* 1: the mesh trees are left to the device: `nodes` holds only the top-level tree,
     * tris / tri_attrs / orig_to_leaf are in original triangle order (orig_to_leaf the
     * identity) and instance blasRoot fields are unset; gnd_gpu_scene_upload builds the
     * mesh trees on the GPU (gnd_host_load_xml_ex, GND_HOST_DEVICE_BLAS) */
    int32_t blas_on_device;
    /* environment map (environment.cpp), or env_emitter = -1: texels width x height x 3
     * floats (row = polar angle from +z, column = azimuth), then its sampling tables
     * (distribution.cpp) in env_dist: marginal func (height), marginal cdf (height + 1),
     * conditional funcs (height x width), conditional cdfs (height x (width + 1)),
     * conditional integrals (height) */
    int32_t env_emitter;          /* index in the emitter list */
    int32_t env_width, env_height;
    float env_marginal_integral;
    float env_strength;
    int32_t pad2;
    const float* env_texels;
    const float* env_dist;
    /* motion blur (animated.cpp): num_instances motion records (gnd::InstMotion, 192
     * bytes) when any instance has a toWorldEnd, else NULL; an instance moves when its
     * traversal record's kind has bit 31 set */
    const void* inst_motion;
    /* textures other than constant and checkerboard (textures/perlin.h, marble.h, wood.h,
     * cellular.h, domainWarp.h, imageTexture.cpp): a color slot of kind 2 evaluates node
     * `node` of tex_nodes (96-byte gnd::TexNode records); image texels are rgba floats,
     * num_tex_texels of them, row 0 the image's bottom row */
    const void* tex_nodes;
    int32_t num_tex_nodes;
    int32_t pad3;
    const float* tex_texels;
    int64_t num_tex_texels;
} gnd_scene_desc;

/* ------------------------------------------------------------------ host framework */
typedef struct gnd_host_scene gnd_host_scene;

/* Parser::loadFromXML + Scene::activate (parser.cpp:220-235, scene.cpp:46-62): parses the
 * scene file, loads meshes, builds every BVH and flattens them. */
gnd_status gnd_host_load_xml(const char* path, gnd_host_scene** out);
/* As gnd_host_load_xml / gnd_host_from_triangles; flags GND_HOST_DEVICE_BLAS: build only
 * the top-level tree on the host and leave the mesh trees (the SAH build of
 * bvhBuilder.cpp:59-262) to the device at upload (an LBVH, see gnd_gpu_scene_upload). */
#define GND_HOST_DEVICE_BLAS 1
gnd_status gnd_host_load_xml_ex(const char* path, int32_t flags, gnd_host_scene** out);
gnd_status gnd_host_from_triangles_ex(const float* tris, int64_t ntri, int32_t flags, gnd_host_scene** out);
/* One mesh primitive with an identity transform from a triangle soup (ntri x 9 floats),
 * default camera; used for traversal-only workloads. */
gnd_status gnd_host_from_triangles(const float* tris, int64_t ntri, gnd_host_scene** out);
gnd_status gnd_host_scene_desc(const gnd_host_scene* s, const gnd_scene_desc** out);
gnd_status gnd_host_free(gnd_host_scene* s);

/* ------------------------------------------------------------------ device boundary */
typedef struct gnd_gpu_ctx gnd_gpu_ctx;
typedef uint64_t gnd_scene_id;

/* One context per GPU (device ordinal). Fails with GND_ERR_NO_DEVICE when no CUDA
 * device is usable: there is no CPU fallback. */
gnd_status gnd_gpu_create(int device, gnd_gpu_ctx** out);
gnd_status gnd_gpu_destroy(gnd_gpu_ctx* ctx);

/* Integrator::preprocess (integrator.h:23, called at scene.cpp:61): copies a flattened
 * scene to HBM; the scene stays resident until gnd_gpu_scene_free. With
 * desc->blas_on_device the mesh trees are built here on the GPU (replacing the host build
 * of bvhBuilder.cpp:59-262): a linear BVH over 3D Morton codes of the triangle
 * centroids, leaves chosen by the surface area heuristic, collapsed to the same 4-wide
 * nodes. Closest hits equal those through a host-built tree except between triangles at
 * exactly the same distance.
 * An upload copies, builds and validates on a stream of its own and may run on another
 * host thread while a render or the serving thread uses the context: the transfer
 * overlaps the render, and only publishing the finished scene waits for the context.
 * Uploads on one context run one at a time. */
gnd_status gnd_gpu_scene_upload(gnd_gpu_ctx* ctx, const gnd_scene_desc* desc, gnd_scene_id* out);
gnd_status gnd_gpu_scene_free(gnd_gpu_ctx* ctx, gnd_scene_id scene);
/* Largest leaf (1..16 triangles, default 4) of the mesh trees that later uploads build on
 * the GPU; a subtree up to that size becomes a leaf where the surface area heuristic
 * prefers it. Changes the tree, and so which triangle wins an exact-distance tie. */
gnd_status gnd_gpu_set_build_leaf_max(gnd_gpu_ctx* ctx, int32_t leaf_max);
/* Page-locks (pin = 1) or releases (pin = 0) the large host arrays of a scene
 * description (BVH nodes, triangles, triangle attributes) so that gnd_gpu_scene_upload
 * copies them by DMA at full link speed. Release before the description is freed. */
gnd_status gnd_gpu_host_register(const gnd_scene_desc* desc, int32_t pin);
/* Bytes of HBM the scene occupies. */
gnd_status gnd_gpu_scene_bytes(gnd_gpu_ctx* ctx, gnd_scene_id scene, uint64_t* bytes);

/* Sizes and build record of an uploaded scene. */
typedef struct gnd_scene_info {
    int64_t num_nodes;          /* BVH4 nodes, the top-level tree first */
    int64_t num_tris;
    int32_t num_instances;
    int32_t blas_on_device;     /* 1: the mesh trees were built on the GPU at upload */
    int32_t fast_boxes;         /* 1: every node bound is finite (fast slab test) */
    int32_t num_meshes;
    double build_ms;            /* device time of the mesh-tree build; 0 when built on the host */
    uint64_t bytes;             /* device bytes held by the scene */
} gnd_scene_info;
gnd_status gnd_gpu_scene_info(gnd_gpu_ctx* ctx, gnd_scene_id scene, gnd_scene_info* info);

/* Copies one device array of an uploaded scene into host memory `dst` of `capacity`
 * bytes (GND_ERR_INVALID when the array does not fit): the layout records of
 * gnd/layout.h. With it a tree built on the GPU can be kept as a host scene
 * description (blas_on_device 0) and uploaded again without a build. */
#define GND_ARRAY_NODES 0          /* Node4, 128 bytes each, num_nodes */
#define GND_ARRAY_TRIS 1           /* Tri, 48 bytes, leaf order */
#define GND_ARRAY_TRI_ATTRS 2      /* TriAttr, 64 bytes, leaf order */
#define GND_ARRAY_ORIG_TO_LEAF 3   /* uint32 per triangle: original index -> leaf slot */
#define GND_ARRAY_INST_TRAV 4      /* InstTrav, 64 bytes, per instance */
gnd_status gnd_gpu_scene_download(gnd_gpu_ctx* ctx, gnd_scene_id scene, int32_t array, void* dst, int64_t capacity);

/* BVH refit for a deforming mesh (no counterpart in the reference, whose scenes are
 * static after Scene::activate; it replaces rebuilding the tree with bvhBuilder.cpp:59-262
 * for the same triangles): mesh `mesh` of an uploaded scene takes new object-space
 * positions, num_tris x 9 floats in the mesh's original triangle order (num_tris must
 * be the mesh's triangle count). Its tree keeps its topology and every box is recomputed
 * on the GPU, then the instance bounds and the top-level tree; normals and uvs stay as
 * loaded. Refused for scenes with moving instances and for meshes carrying an area
 * light. The first refit of a scene walks its trees once (a few synchronous steps);
 * device_ms (may be NULL) receives the device time of the refit kernels. Renders of the
 * context finish before the refit starts (both hold the context and run on its stream);
 * a scene named by a queued or running served job is refused (GND_ERR_INVALID), and ray
 * batches the caller queued on its own streams must have finished. */
gnd_status gnd_gpu_scene_refit_mesh(gnd_gpu_ctx* ctx, gnd_scene_id scene, int32_t mesh, const float* positions,
                                    int64_t num_tris, float* device_ms);

/* Scene::rayIntersect(ray, isect) (scene.cpp:64-66, bvh.cpp:38-66) for n rays in HOST
 * memory: closest hit per ray, world tMax shrinking as hits are found. */
gnd_status gnd_gpu_trace_closest(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* rays, int64_t n,
                                 gnd_hit* hits);
/* Scene::rayIntersect(ray) (scene.cpp:68-71): occlusion (any hit) per ray, 1/0. */
gnd_status gnd_gpu_trace_any(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* rays, int64_t n,
                             uint8_t* occluded);
/* The same on DEVICE buffers, asynchronous on `stream` (a cudaStream_t, NULL = the
 * context's stream). */
gnd_status gnd_gpu_trace_closest_dev(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* d_rays, int64_t n,
                                     gnd_hit* d_hits, void* stream);
gnd_status gnd_gpu_trace_any_dev(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* d_rays, int64_t n,
                                 uint8_t* d_occluded, void* stream);
/* Per-ray traversal work of the closest-hit kernel (instrumented variant): node visits
 * and triangle tests, DEVICE buffers. Used for the roofline byte counts. */
gnd_status gnd_gpu_trace_count_dev(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* d_rays, int64_t n,
                                   uint32_t* d_nodes, uint32_t* d_tris, void* stream);
/* gnd_gpu_trace_closest without any device allocation. No counterpart in the reference.
 * Rays, hits and the kernel's fetch counter live in a fixed module-scope device array
 * (3.25 MiB per device), so n may be at most GND_TRACE_FIXED_MAX_RAYS; larger batches
 * are rejected with GND_ERR_INVALID. Returns after the hits are in `hits` (HOST
 * memory). The first call on a device looks the array up (cudaGetSymbolAddress), which
 * may load the module; make that first call before any stream capture begins. The
 * array is shared by every context of the process on the device: calls that overlap in
 * time on one device race on it. */
#define GND_TRACE_FIXED_MAX_RAYS 65536
gnd_status gnd_gpu_trace_closest_fixed(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_ray* rays, int64_t n,
                                       gnd_hit* hits);

/* Read bandwidth of the device in GB/s: `reps` passes of 16-byte L2-cached loads over
 * a buffer of `bytes` (allocated and freed by the call). A buffer well inside L2 gives
 * the L2 bandwidth, one far larger than L2 the HBM bandwidth: the denominators of the
 * traversal roofline. Diagnostics; no counterpart in the reference. */
gnd_status gnd_gpu_read_bandwidth(gnd_gpu_ctx* ctx, uint64_t bytes, int32_t reps, double* gbps);

/* ------------------------------------------------------------------ image outputs */
/* The reference's post-processing (PostProcessor::render, postProcessor.cpp:148-235, and
 * its shaders tonemap.frag, bloom_*.frag, gammaCorrect.frag) and the 8-bit conversion of
 * Film::savePNG (film.cpp:154-171), run as CUDA kernels on a linear RGB image
 * (width x height x 3 floats, row-major) instead of through OpenGL. Defaults of
 * PostProcessor: tonemapper 0, exposure 0, bloom off, threshold 1, radius 1, intensity
 * 0.04, 6 mips. */
typedef struct gnd_post_params {
    int32_t tonemapper;       /* 0 linear, 1 Reinhard, 2 Uncharted 2, 3 ACES, 4 Khronos PBR
                                 neutral, 5 AgX, 6 AgX punchy (TonemapOperator) */
    float exposure;           /* stops: colour *= exp2(exposure) */
    int32_t bloom;            /* 1: bloom pyramid added before the exposure */
    float bloom_threshold;    /* prefilter: keep texels whose brightest channel exceeds it */
    float bloom_radius;       /* upsample tent radius in source texels */
    float bloom_intensity;    /* weight of the bloom in the sum */
    int32_t bloom_mips;       /* pyramid levels used, 1..6 */
    int32_t output;           /* 8-bit conversion: 0 Film::savePNG (sRGB, x255 + 0.5,
                                 truncate), 1 display pass (gammaCorrect.frag, rounded) */
} gnd_post_params;
/* Host buffers: `rgb` in; `hdr` (tonemapped floats, w x h x 3) and `rgb8` (w x h x 3
 * bytes) out, each optional (NULL). */
gnd_status gnd_gpu_post(gnd_gpu_ctx* ctx, const float* rgb, int32_t width, int32_t height,
                        const gnd_post_params* params, float* hdr, uint8_t* rgb8);
/* The same on device buffers, enqueued on `stream` (cudaStream_t; 0 = legacy stream). */
gnd_status gnd_gpu_post_dev(gnd_gpu_ctx* ctx, const float* d_rgb, int32_t width, int32_t height,
                            const gnd_post_params* params, float* d_hdr, uint8_t* d_rgb8, void* stream);
/* Film::savePNG / Film::saveEXR (film.cpp:154-195) as files: an 8-bit RGB PNG (zlib
 * compressed) and a 32-bit float RGB OpenEXR image (scanline, uncompressed; channels
 * B, G, R as the format orders them). */
gnd_status gnd_image_write_png(const char* path, const uint8_t* rgb8, int32_t width, int32_t height);
gnd_status gnd_image_write_exr(const char* path, const float* rgb, int32_t width, int32_t height);
/* Reads a scanline OpenEXR image (compression none, ZIPS or ZIP; HALF or FLOAT channels)
 * as rgb floats: the reader the environment map uses (image2d.h:100-135). With rgb = NULL
 * only the size is returned; otherwise `capacity` bytes must hold width x height x 3
 * floats. */
gnd_status gnd_image_read_exr(const char* path, float* rgb, int64_t capacity, int32_t* width, int32_t* height);

/* ------------------------------------------------------------------ rendering */
/* Progress callback, the reference's Integrator::setCallback / notifyUpdate
 * (integrator.h:25-35, 148-149): called after each completed sample pass with the film
 * accumulated so far (height x width x 7 floats, see gnd_gpu_render). */
typedef void (*gnd_progress_fn)(void* user, int32_t sample_index, const float* film, int32_t width, int32_t height);

typedef struct gnd_render_params {
    int32_t spp;              /* passes (samples per pixel); <= 0: the scene file's value */
    int32_t first_pass;       /* sample index of the first pass (it keys the seeds) */
    int32_t max_depth;        /* <= 0: the scene file's value */
    int32_t integrator;       /* -1: the scene file's; 0 path_gpu; 1 volpath_gpu */
    int32_t window[4];        /* pixel window x0, y0, x1, y1; all zero: the full image */
    int32_t batched;          /* 0: one pass in flight at a time (plain); 1: every pass
                                 shares the path pool, refilled as paths finish */
    int32_t profile;          /* bit0: time the closest-hit (extend) launches with events;
                                 bit1: count BVH node visits / triangle tests in extend */
    gnd_progress_fn callback; /* optional (plain mode only) */
    void* user;
    int32_t width, height;    /* film size; <= 0: the scene file's (the camera keeps its
                                 field of view; the aspect ratio follows the film) */
} gnd_render_params;

typedef struct gnd_render_stats {
    int64_t paths;            /* camera samples traced */
    int64_t rays;             /* closest-hit + shadow queries */
    int32_t passes_done;
    int32_t pad;
    double ms;                /* device time of the render */
    int64_t extend_rays;      /* closest-hit queries of the extend kernel */
    int64_t shadow_rays;      /* shadow queries */
    int64_t extend_nodes;     /* profile bit1: BVH4 node visits in extend */
    int64_t extend_tris;      /* profile bit1: triangle tests in extend */
    double extend_ms;         /* profile bit0: summed device time of the extend launches */
    int64_t iterations;       /* wavefront iterations (bounce steps) */
    int64_t launches;         /* kernels the render launched */
    /* profile bit1: the extend traversal's phases (a warp alternates inner-node steps and
     * leaf steps): warp steps of the node phase, lane steps and warp steps of the leaf
     * phase; lanes busy per step = extend_nodes / (32 x extend_node_warp_steps) and
     * extend_leaf_steps / (32 x extend_leaf_warp_steps) */
    int64_t extend_node_warp_steps;
    int64_t extend_leaf_steps;
    int64_t extend_leaf_warp_steps;
} gnd_render_stats;

/* Integrator::render (integrator.h:49-155) for path_gpu / volpath_gpu: renders the
 * passes [first_pass, first_pass + spp) and ADDS them into `film` (host memory,
 * height x width x 7 floats per pixel: sum of w*L (r, g, b), sum of w, sum of w*L^2
 * (r, g, b); the image is sum(w*L) / sum(w)). Per-pixel sample keys, draw order and film
 * splatting follow the reference render loop. Cancelled renders (gnd_gpu_cancel) stop
 * after the current pass and return GND_ERR_CANCELLED with the partial film added. */
gnd_status gnd_gpu_render(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_render_params* params, float* film,
                          gnd_render_stats* stats);
/* Integrator::cancel (integrator.h:22): asks a running gnd_gpu_render on this context
 * to stop after its current pass. Safe to call from another thread. */
gnd_status gnd_gpu_cancel(gnd_gpu_ctx* ctx);

/* gnd_gpu_render with the film in the exact form the device accumulates it. No
 * counterpart in the reference, whose film holds float sums (film.h:110-124); it serves
 * callers that add up films of several renders (sample passes sharded over GPUs or
 * processes) and want the total to equal one render of all the passes bit for bit.
 * `sum` (height x width x 4 uint64: sum of w*L r, g, b and sum of w, in units of 2^-24)
 * and `sq` (height x width x 3 floats: sum of w*L^2) are HOST buffers; the render ADDS
 * into them (the integer sums modulo 2^64). Integer sums do not depend on the order of
 * the additions, so passes split over any number of calls or ranks give the same `sum`
 * as one call; `sq` is a float sum and agrees to rounding. Image = sum[0..2] / sum[3]. */
gnd_status gnd_gpu_render_fixed(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_render_params* params, uint64_t* sum,
                                float* sq, gnd_render_stats* stats);

/* Work counters of a context (diagnostics; no counterpart in the reference, which keeps
 * none). Sums since the context was created or the counters were last reset:
 *   trace_*  the ray batches of gnd_gpu_trace_closest / _any / _count_dev / _closest_fixed
 *            and their _dev forms (rays queued on another stream are counted once the
 *            device has run them: the call synchronises the device);
 *   the node visits and triangle tests of the batches that count them
 *            (gnd_gpu_trace_count_dev);
 *   render   gnd_gpu_render / gnd_gpu_render_fixed calls: camera paths, closest-hit and
 *            shadow queries, wavefront iterations, kernel launches, device time, and the
 *            extend kernel's node visits and triangle tests for renders that count them
 *            (gnd_render_params.profile bit1);
 *   last     the statistics of the last render.
 * reset != 0 clears the sums after reading them. */
typedef struct gnd_counters {
    int64_t trace_batches;    /* batches with at least one ray */
    int64_t trace_rays;
    int64_t counted_rays;     /* rays of the counting batches */
    int64_t counted_nodes;    /* BVH4 node visits of those rays */
    int64_t counted_tris;     /* triangle tests of those rays */
    int64_t renders;
    int64_t paths;
    int64_t extend_rays;
    int64_t shadow_rays;
    int64_t extend_nodes;     /* renders with profile bit1 only */
    int64_t extend_tris;
    int64_t iterations;
    int64_t launches;
    double render_ms;
    gnd_render_stats last;
} gnd_counters;
gnd_status gnd_gpu_counters(gnd_gpu_ctx* ctx, gnd_counters* out, int32_t reset);

/* ------------------------------------------------------------------ tuning */
/* Engine settings of a scene's renders. They change speed only: every setting renders
 * the same film sums. No counterpart in the reference. */
typedef struct gnd_tune {
    int32_t pool_log2;        /* path slots of a batched render: 2^pool_log2 (16..26) */
    int32_t round_iters;      /* wavefront iterations per host round, batched (2..64, even) */
    int32_t trav_blocks;      /* persistent traversal blocks of 128 threads per SM (1..10; 9
                                 and 10 run the plain closest-hit and shadow kernels
                                 compiled to fit them, with fewer registers per thread) */
    int32_t material_sort;    /* 1: classify hits and shade per material class; 0: one kernel */
    int32_t stack_smem;       /* traversal stack entries in shared memory: 16 or 32 */
    int32_t graphs;           /* 1: replay pairs of iterations as CUDA graphs */
    int32_t sample_film;      /* 1: batched renders write one record per sample and build the
                                 film from them afterwards (no film atomics; 16 bytes of HBM
                                 per sample, 24 with the Gaussian filter, whose film is then
                                 gathered per pixel from the records around it); 0: atomics */
    int32_t spec_extend;      /* 1: closest-hit traversal lets a ray that holds a leaf keep
                                 visiting inner nodes until it is blocked (speculative);
                                 default 0 */
    int32_t spec_shadow;      /* the same for the shadow (occlusion) traversal */
    int32_t ray_sort;         /* bit 0: before each closest-hit launch the active paths are
                                 reordered by a ray key (origin cell and direction bin) so
                                 that a warp's rays visit the same nodes; bit 1: the path
                                 tracer's shadow queries likewise; bit 2: ray batches of at
                                 least 65,536 rays (gnd_gpu_trace_*, except the _fixed
                                 form) are traversed in key order, results still in input
                                 order; default 0 */
    int32_t leaf_batch;       /* closest-hit traversal of renders (1..32): a warp leaves its
                                 inner-node phase for its leaf phase once this many of its
                                 rays hold a leaf; the others resume their traversal
                                 afterwards (32: only when no ray can take another
                                 inner-node step, the default) */
    int32_t trace_leaf_batch; /* the same for the scene's ray batches (gnd_gpu_trace_*,
                                 except the _fixed form); default 12 */
    int32_t shadow_leaf_batch; /* the same for the path tracer's shadow queries; default 32 */
    int32_t trace_blocks;     /* persistent blocks of 128 threads per SM for the scene's ray
                                 batches (1..10, as trav_blocks; default 8) */
} gnd_tune;
gnd_status gnd_gpu_get_tune(gnd_gpu_ctx* ctx, gnd_scene_id scene, gnd_tune* tune);
gnd_status gnd_gpu_set_tune(gnd_gpu_ctx* ctx, gnd_scene_id scene, const gnd_tune* tune);
/* Chooses the settings for a scene by measurement: coordinate descent from the current
 * settings over every field, each candidate timed on the device with a batched render of
 * `spp` passes (<= 0: 8) at the scene's film size, depth and integrator, until about
 * budget_ms of wall time is spent. Keeps a change when it is at least 2% faster, or
 * when a candidate between 0.3% and 2% faster stays at least 0.5% faster over three
 * renders alternating with the current settings. Stores the result as the scene's
 * settings; returns it and its Mpaths/s. */
gnd_status gnd_gpu_autotune(gnd_gpu_ctx* ctx, gnd_scene_id scene, int32_t spp, int32_t budget_ms, gnd_tune* best,
                            double* mpaths_per_s);

/* ------------------------------------------------------------------ serving */
/* A stream of render jobs on one context. No counterpart in the reference, whose
 * Integrator::render renders one scene per call (integrator.h:49-155); each job renders
 * exactly what gnd_gpu_render renders for the same arguments (same samples, same film
 * sums), but jobs share one pool of path slots: they are admitted first-come
 * first-served while the job table (64 running jobs) and the HBM budget allow, and the
 * slots freed by finishing paths take the oldest running job's next samples. */
typedef uint64_t gnd_job_id;

typedef struct gnd_job_desc {
    gnd_scene_id scene;
    int32_t width, height;    /* film size; <= 0: the scene file's */
    int32_t spp;              /* <= 0: the scene file's */
    int32_t max_depth;        /* <= 0: the scene file's */
    int32_t integrator;       /* -1: the scene file's; 0 path_gpu; 1 volpath_gpu */
    int32_t first_pass;       /* sample index of the first pass (it keys the seeds) */
} gnd_job_desc;

enum { GND_JOB_QUEUED = 0, GND_JOB_RUNNING = 1, GND_JOB_DONE = 2, GND_JOB_CANCELLED = 3, GND_JOB_FAILED = 4 };

typedef struct gnd_job_status {
    int32_t state;            /* GND_JOB_* */
    int32_t pad;
    int64_t samples_total;    /* width * height * spp */
    int64_t samples_done;     /* samples retired into the film */
    double submit_ms;         /* host steady clock, ms since the server started */
    double admit_ms;          /* 0 while queued */
    double done_ms;           /* film resolved into host memory; 0 while unfinished */
} gnd_job_status;

/* HBM admission budget in bytes for the context (scenes + path pool + films of running
 * jobs); 0 = no budget beyond the device's free memory. Jobs over budget wait in the
 * queue; a job that cannot fit even alone is refused at submit with GND_ERR_BUDGET. */
gnd_status gnd_gpu_set_hbm_budget(gnd_gpu_ctx* ctx, uint64_t bytes);
/* Order in which running jobs' samples are handed to free path slots:
 * GND_SERVE_FIFO: the oldest running job first;
 * GND_SERVE_SRPT: the job with the fewest samples left to hand out first;
 * GND_SERVE_DEADLINE (default): earliest deadline first, a job's deadline being its
 *   submission time plus 4x its estimated render time alone (samples / the server's
 *   measured sample rate): small jobs overtake large ones, but a large job waits at
 *   most a bounded multiple of its own render time.
 * Admission is first-come first-served under every policy. */
enum { GND_SERVE_FIFO = 0, GND_SERVE_SRPT = 1, GND_SERVE_DEADLINE = 2 };
gnd_status gnd_gpu_serve_policy(gnd_gpu_ctx* ctx, int32_t policy);
/* Engine settings of the serving thread (gnd_tune; pool_log2 and round_iters are the
 * server's own: its pool of path slots, default 2^22, takes the new size when no job is
 * running; material_sort is always on because jobs of both integrators share launches).
 * Like a scene's settings they change speed, never results. */
gnd_status gnd_gpu_serve_tune(gnd_gpu_ctx* ctx, const gnd_tune* tune);
/* Queues a job; returns at once with its id. The scene may not be freed while a job
 * that names it is queued or running (gnd_gpu_scene_free fails with GND_ERR_INVALID). */
gnd_status gnd_gpu_serve_submit(gnd_gpu_ctx* ctx, const gnd_job_desc* job, gnd_job_id* id);
/* Current state of a job (does not block). */
gnd_status gnd_gpu_serve_poll(gnd_gpu_ctx* ctx, gnd_job_id id, gnd_job_status* status);
/* Blocks until the job has finished, copies its film (height x width x 7 floats, laid
 * out as gnd_gpu_render's) into `film` (may be NULL) and releases the job id. Returns
 * GND_ERR_CANCELLED for a cancelled job (with the samples that were retired) and the
 * job's error for a failed one. timeout_ms < 0 waits without limit; when it runs out the
 * call returns GND_ERR_TIMEOUT and the job stays valid. */
gnd_status gnd_gpu_serve_wait(gnd_gpu_ctx* ctx, gnd_job_id id, float* film, gnd_job_status* status,
                              int64_t timeout_ms);
/* Asks a job to stop: a queued job is dropped, a running one hands out no further
 * samples and finishes when its paths in flight have retired. */
gnd_status gnd_gpu_serve_cancel(gnd_gpu_ctx* ctx, gnd_job_id id);

#ifdef __cplusplus
}
#endif
#endif /* GND_GPU_H */
