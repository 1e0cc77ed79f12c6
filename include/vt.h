/*
 * vt.h -- C ABI of libvt.so, the B200 (sm_100a) isosurface ray caster with
 * the capabilities of carlosduelo/visualTur.
 *
 * Conventions (all entry points):
 *   - every call returns a vt_status; nothing calls exit(); vt_last_error()
 *     gives a message for the calling thread's last failure;
 *   - device buffers passed in are borrowed and owned by the caller;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default);
 *     work is stream-ordered, calls return once it is enqueued unless the
 *     entry point says it synchronises;
 *   - a handle belongs to one host thread at a time; the caller serialises
 *     calls from other threads;
 *   - voxel layout: x slowest, z fastest (index z + y*dz + x*dy*dz), as the
 *     reference's HDF5 datasets ([x][y][z], src/FileManager.cu:86-167).
 *
 * Reference citations are path:line in carlosduelo/visualTur.
 */
#ifndef VT_H
#define VT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VT_API_VERSION 2

typedef enum {
    VT_OK = 0,
    VT_ERR_INVALID = 1,      /* bad argument or inconsistent parameters */
    VT_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    VT_ERR_IO = 3,           /* file could not be opened/read/written */
    VT_ERR_FORMAT = 4,       /* bad octree magic / volume header */
    VT_ERR_NOMEM = 5,        /* host or device allocation failed */
    VT_ERR_TIMEOUT = 6,      /* a bounded device wait or frame loop gave up */
    VT_ERR_STACK = 7,        /* a ray's traversal stack overflowed */
    VT_ERR_UNSUPPORTED = 8,  /* valid request the library does not handle */
    VT_ERR_STATE = 9         /* call not valid in the handle's state */
} vt_status;

const char* vt_status_string(vt_status s);
const char* vt_last_error(void);
int vt_api_version(void);

/* Voxel types.  The reference stores float32 only (H5T_IEEE_F32LE,
 * src/FileManager.cu:155); uint8 is an extension for 4096^3 volumes. */
enum { VT_F32 = 0, VT_U8 = 1 };

/* ------------------------------------------------------------------------ */
/* Volume I/O (replaces class FileManager, inc/FileManager.hpp:12-35)       */
/* ------------------------------------------------------------------------ */
typedef struct vt_volume vt_volume;

/* FileManager::FileManager (src/FileManager.cu:11-37).  Opens a project raw
 * volume file ("VTVOL001" header) or an HDF5 file holding a contiguous or
 * compact 3-D dataset; `dataset` is its path in the file ("value",
 * "/grp/value"; ignored for raw files).  float32 and uint8 datasets are
 * memory-mapped; other little-endian integer or float datasets are
 * converted to float32 in memory, as the reference's H5Dread to
 * H5T_IEEE_F32LE converts them (src/FileManager.cu:155). */
vt_status vt_volume_open(const char* path, const char* dataset, vt_volume** out);
/* Wraps caller-owned host memory as a volume (no copy; must outlive it). */
vt_status vt_volume_wrap(const void* data, int vtype, const int64_t dims[3], vt_volume** out);
/* A volume read through a caller's function (no reference counterpart):
 * read(user, s, e, out) fills out with the voxels [s,e) as vt_volume_read
 * would (|e-s| per axis, x slowest, zeros outside the volume, the volume's
 * voxel type) and returns 0, or returns non-zero when the read failed (a
 * short read, a missing brick file).  Brick-cache misses call it from
 * several host threads at once.  A failed read makes the render call
 * return VT_ERR_IO -- where the reference exit(0)s on an HDF5 error
 * (src/FileManager.cu:15-36) -- and leaves the renderer usable: the next
 * frame requests the brick again.  Volumes of this kind serve the brick
 * cache and vt_volume_read only (not resident renderers or the builder). */
typedef int (*vt_read_fn)(void* user, const int s[3], const int e[3], void* out);
vt_status vt_volume_from_reader(vt_read_fn read, void* user, int vtype, const int64_t dims[3], vt_volume** out);
void      vt_volume_close(vt_volume* v);
vt_status vt_volume_info(const vt_volume* v, int64_t dims[3], int* vtype);
/* FileManager::readHDF5_Voxel_Array (src/FileManager.cu:86-167): reads
 * voxels [s,e) into out (|e-s| per axis, float32); parts outside the volume
 * are 0. */
vt_status vt_volume_read(const vt_volume* v, const int s[3], const int e[3], float* out);
/* FileManager::readHDF5 (src/FileManager.cu:71-84): whole dataset. */
vt_status vt_volume_read_all(const vt_volume* v, void* out);
/* FileManager::CreateFile (src/FileManager.cu:169-243).  format 0 = raw,
 * 1 = HDF5 (contiguous dataset named `dataset`). */
vt_status vt_volume_write(const char* path, const char* dataset, int format, const void* data,
                          int vtype, const int64_t dims[3]);

/* HDF5 dataset inspection (no reference counterpart): how libvt's reader
 * sees the dataset `dataset` of the HDF5 file `path`.  type_class: 0 fixed
 * point, 1 IEEE float; offset: file offset of the first element. */
typedef struct {
    int rank;
    int64_t dims[32];
    int type_class, type_size, is_signed, big_endian;
    uint64_t offset, bytes;
} vt_h5_info;
vt_status vt_h5_describe(const char* path, const char* dataset, vt_h5_info* out);

/* Seeded synthetic volumes (no reference counterpart).
 *   VT_GEN_SPHERE: |x-c| + 0.25*g, g ~ N(0,1) by 4-term Irwin-Hall;
 *                  params[0..2] = c; params[3] = noise sigma
 *   VT_GEN_BLOBS:  sum of params[0] anisotropic Gaussian blobs, sigma in
 *                  [params[1],params[2]], amplitude [params[3],params[4]],
 *                  plus 4-octave value noise of amplitude params[5]
 *   VT_GEN_FRACTAL_U8: 6-octave value noise in [0,255] with params[0]
 *                  spheres of value params[3], radius [params[1],params[2]]
 * Host generation writes `out` (host); device generation writes `dev_out`. */
enum { VT_GEN_SPHERE = 0, VT_GEN_BLOBS = 1, VT_GEN_FRACTAL_U8 = 2 };
vt_status vt_generate_volume(int kind, uint64_t seed, const int64_t dims[3], const float* params,
                             int nparams, void* out);
vt_status vt_generate_volume_device(int kind, uint64_t seed, const int64_t dims[3],
                                    const float* params, int nparams, void* dev_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Octree (replaces class Octree, inc/Octree.hpp:12-42, and OctreeM,        */
/* inc/CreateOctree.hpp:12-89)                                              */
/* ------------------------------------------------------------------------ */
typedef struct vt_octree vt_octree;

/* Octree::Octree file reading (src/Octree.cu:769-813). */
vt_status vt_octree_load(const char* path, vt_octree** out);
void      vt_octree_free(vt_octree* o);
vt_status vt_octree_info(const vt_octree* o, float* iso, int* dimension, int realDim[3], int* nLevels);
/* Number of uint64 words of level `level` and a copy of them. */
vt_status vt_octree_level(const vt_octree* o, int level, int64_t* n, uint64_t* words);
/* OctreeM::OctreeM + writeToFile (src/CreateOctree.cu:300-371) on the GPU:
 * builds the octree of `v` for isovalue `iso` and writes the file. */
vt_status vt_octree_build(const vt_volume* v, float iso, const char* out_path, void* stream);
/* Same for a volume already in device memory (dims[0]*dims[1]*dims[2]
 * voxels of vtype, x slowest). */
vt_status vt_octree_build_device(const void* dev_vol, int vtype, const int64_t dims[3], float iso,
                                 const char* out_path, void* stream);

/* ------------------------------------------------------------------------ */
/* Camera rays and single-brick rendering (class Camera, rayCaster)         */
/* ------------------------------------------------------------------------ */
typedef struct {
    int W, H;
    float distance;          /* screen distance (Screen, src/Screen.cpp:11-20) */
    float h, w;              /* screen extent in world units */
    float look[3], up[3], right[3], position[3];
} vt_camera;

/* Camera(...) initial state (src/Camera.cu:12-29): fov_H/fov_W act as
 * half-angles, h = 2*d*tanf(fov_H*pi/180). */
vt_status vt_camera_init(vt_camera* c, int H, int W, float distance, float fov_H, float fov_W);
/* Camera::Move/RotateX/RotateY/RotateZ/MoveForward/MoveUpward/StrafeRight
 * (src/Camera.cu:85-156), including the reference's axis naming. op:
 * 0 move(x,y,z) 1 rotX 2 rotY 3 rotZ 4 forward 5 upward 6 strafe. */
vt_status vt_camera_op(vt_camera* c, int op, float a, float b, float cc);
/* cuda_updateRays (src/Camera.cu:39-83): W*H float3 directions. */
vt_status vt_camera_rays(const vt_camera* c, float* dev_dirs, void* stream);
/* rayCaster::renderCube / cuda_rayCasterCube (src/rayCaster.cu:267-394):
 * renders one brick of (cubeDim+2*cubeInc) voxels (float32, on device)
 * whose interior starts at minBox, into dev_rgba (W*H*4 floats). */
vt_status vt_render_cube(const vt_camera* c, const float* dev_cube, const int minBox[3],
                         const int cubeDim[3], const int cubeInc[3], float iso, const float light[3],
                         float* dev_rgba, void* stream);

/* ------------------------------------------------------------------------ */
/* Renderer (replaces class visualTur, inc/visualTur.hpp:12-80)              */
/* ------------------------------------------------------------------------ */
/* visualTurParams_t (inc/visualTur.hpp:12-33). */
typedef struct {
    int W, H;
    float distance, fov_H, fov_W;
    int numRayPx;                 /* must be 1: the reference writes W*H rays only */
    int maxElementsCache;         /* device brick slots */
    int maxElementsCache_CPU;     /* pinned host brick slots */
    int dimCubeCache[3];          /* brick edge; must equal 2^(nLevels-levelCubes) */
    int cubeInc;                  /* apron; >= 3 so every tap stays in the brick */
    int levelCubes;
    const char* hdf5File;
    const char* dataset_name;
    const char* octreeFile;
    int octreeLevel;
} vt_params;

/* Renderer options (no reference counterpart). */
typedef struct {
    int resident;          /* 1: whole volume in HBM, no brick cache; 0: brick cache */
    int tile_w, tile_h;    /* pixels per CTA tile (autotuned) */
    int unroll;            /* march unroll (autotuned) */
    int lookahead;         /* bricks a suspended ray may request ahead (0..4) */
    int max_passes;        /* bound on demand passes per frame */
    int host_threads;      /* host tier fill threads (0 = hardware) */
    int record_trace;      /* log per-frame touched coarse nodes */
    int trace_level;       /* octree level of the logged nodes (4 in C4) */
    int record_hits;       /* keep per-ray hit node/brick/t/normal for vt_debug_hits */
    int persistent;        /* 1: persistent ray-queue kernel with warp refill */
    int blocks_per_sm;     /* persistent grid: CTAs per SM (autotuned) */
    int pops;              /* persistent: traversal steps between warp refills */
    int preload;           /* 1: load every needed brick at create when they fit */
    int use_graph;         /* 1: pass 0 of a frame replays a captured CUDA graph */
    int refine;            /* isovalue crossing refinement: 0 = one linear step, as the
                              reference (src/rayCaster.cu:227-228); k in 1..16 = k
                              bisection steps on the bracketing samples, then the
                              linear step.  Node and brick ids do not depend on it. */
    int skip;              /* 0..4: candidates whose brick is absent a ray may set aside
                              (requesting the brick) to march later ones in the same
                              pass; a hit found past them waits for them, so the image
                              is the in-order one.  0 = stop at the first absent brick,
                              as the reference.  Off while record_trace is on. */
    /* Bounds of a pass's queues (0 = sized so they never fill).  Requests
     * past max_requests wait for the next pass (the reference's per-pass
     * admission cap, src/lruCache.cu:184-192); more than max_suspended rays
     * waiting on bricks fail the frame with VT_ERR_STATE; a suspended ray
     * whose stack does not fit the pool of pool_per_ray entries per ray
     * restarts from the root next pass (same pixel). */
    int max_suspended, max_requests, pool_per_ray;
    /* 1: lookahead requests are queued and their bricks load on a side
     * stream into never-filled device slots while later passes run (demand
     * requests never wait for them); 0: they load with the demand requests
     * of the same service, into slots the frame has not used. */
    int spec_async;
    /* 0: one trace kernel per pass (traversal and march fused); k in 1..8:
     * wavefront passes -- k rounds of a traversal kernel that queues each
     * ray's next resident candidate, binned by brick, and a march kernel
     * that stages each binned brick into shared memory with one bulk copy
     * and marches its rays from there; then the fused kernel finishes the
     * rays still waiting.  Same image.  Slab mode, in-order traversal
     * (skip 0) only. */
    int wavefront;
    /* 1: a demand load copies a brick's x and y aprons from the slots of
     * resident neighbours (whose middles hold the same voxels) and reads
     * and transfers only the rest; 0: every load reads and transfers the
     * whole brick.  Same bricks either way. */
    int shared_aprons;
    /* with spec_async: a pass's service loads at most this many demand
     * bricks itself while never-filled slots can take them all (a cold
     * start) and hands the rest to the side stream, which loads them while
     * the next pass runs (0: no bound).  Same images. */
    int demand_batch;
} vt_options;

typedef struct vt_handle vt_handle;
/* the learned-prefetch network (vt_mlp_*, below) */
typedef struct vt_mlp vt_mlp;

void      vt_default_options(vt_options* o);
/* visualTur::visualTur (src/visualTur.cu:10-35). */
vt_status vt_create(const vt_params* p, const vt_options* opt, vt_handle** out);
/* Same, with an already-open volume and loaded octree (borrowed). */
vt_status vt_create_from(const vt_params* p, const vt_options* opt, vt_volume* v, vt_octree* o,
                         vt_handle** out);
void      vt_destroy(vt_handle* h);

/* visualTur::camera_* (src/visualTur.cu:124-165); op codes as vt_camera_op. */
vt_status vt_camera_update(vt_handle* h, int op, float a, float b, float c);
/* Sets/reads the full camera state (extension: poses set directly). */
vt_status vt_set_camera(vt_handle* h, const vt_camera* c);
vt_status vt_get_camera(vt_handle* h, vt_camera* c);
/* visualTur::changeScreen / changeNumRays / changeCacheParameters
 * (src/visualTur.cu:83-122). */
vt_status vt_change_screen(vt_handle* h, int W, int H, float fovW, float fovH, float distance);
vt_status vt_change_num_rays(vt_handle* h, int numRayPx);
vt_status vt_change_cache(vt_handle* h, int maxElements, const int cubeDim[3], int cubeInc);

/* Kernel schedule knobs of a live handle (autotuner): ray-tile shape,
 * march unroll, persistent ray queue, traversal steps between refills,
 * persistent CTAs per SM, lookahead requests, graph replay, absent-brick
 * candidates set aside per pass, side-stream lookahead loads, wavefront
 * rounds, shared aprons, demand batch. */
typedef struct {
    int tile_w, tile_h, unroll, persistent, pops, blocks_per_sm, lookahead, use_graph, skip, spec_async, wavefront,
        shared_aprons, demand_batch;
} vt_tuning;
vt_status vt_set_tuning(vt_handle* h, const vt_tuning* t);
vt_status vt_get_tuning(vt_handle* h, vt_tuning* t);

/* visualTur::updateVisibleCubes (src/visualTur.cu:167-228): renders the
 * current camera into dev_rgba (W*H*4 floats, pixel i*W+j) and, if not
 * NULL, dev_rgb8 (W*H*3 bytes, (uint8)(clamp(v,0,1)*255)). */
vt_status vt_render(vt_handle* h, float* dev_rgba, uint8_t* dev_rgb8, void* stream);
/* Same with host output buffers (copies included); synchronises. */
vt_status vt_render_host(vt_handle* h, float* host_rgba, uint8_t* host_rgb8);

/* Many views in one persistent ray-queue launch (no reference counterpart). */
typedef struct {
    vt_camera cam;
    float* dev_rgba;        /* W*H*4 floats, may be NULL if dev_rgb8 given */
    uint8_t* dev_rgb8;      /* W*H*3 bytes, may be NULL */
} vt_view;
vt_status vt_render_batch(vt_handle* h, const vt_view* views, int n, void* stream);

/* Coarse-node access trace of the last frame (record_trace): bit k of
 * `bits` = node 8^trace_level + k was marched.  nwords = 8^trace_level/32;
 * the call synchronises. */
vt_status vt_get_trace(vt_handle* h, uint32_t* bits, int64_t nwords);

/* Loads the given bricks (codes at levelCubes) into the device cache ahead
 * of demand, on `stream`; bricks used by the current frame are never
 * evicted.  Returns the number loaded in *loaded (may be NULL). */
vt_status vt_prefetch(vt_handle* h, const uint64_t* bricks, int64_t n, int64_t* loaded, void* stream);

/* Learned prefetch on the device (no reference counterpart): for the n
 * poses `cams` (the frames about to be rendered), computes the network's 12
 * pose features (position relative to the volume centre over `vol_edge`,
 * look, up, fov_deg / 90, near and far distance to the volume's bounding
 * sphere over `vol_edge`), runs the network m (its outputs: one probability
 * per node of an octree level, 8^level of them, level <= levelCubes) and
 * requests, speculatively, every absent brick holding candidates whose
 * node's largest probability over the poses exceeds `threshold`.  Work is
 * enqueued on `stream` (no synchronisation, nothing copied back but the
 * list of requested bricks); the next vt_render / vt_render_batch queues
 * those bricks ahead of its lookahead requests, and they load as
 * spec_async loads them (or as a vt_prefetch_hint when spec_async is 0).
 * Demand paging stays the fallback: a wrong prediction costs transfers,
 * never a pixel. */
vt_status vt_prefetch_predict(vt_handle* h, vt_mlp* m, const vt_camera* cams, int n, float vol_edge, float fov_deg,
                              float threshold, void* stream);

/* Prefetch hint for the frame after the next vt_render: during that call
 * the bricks' host-tier reads run while its first pass renders (in hint
 * order, as many as finish before the pass does; the rest are dropped),
 * and their device fill follows its last pass (never evicting bricks it
 * used). */
vt_status vt_prefetch_hint(vt_handle* h, const uint64_t* bricks, int64_t n);

/* Bricks (codes at levelCubes) that hold candidate nodes of the octree,
 * sorted; n in/out: capacity / count. */
vt_status vt_brick_list(vt_handle* h, uint64_t* bricks, int64_t* n);

/* Per-ray diagnostics of the last vt_render (host buffers, W*H entries,
 * any may be NULL): hit node Morton code at octreeLevel (0 = none), brick
 * code at levelCubes, hit distance along the ray, unit normal. */
vt_status vt_debug_hits(vt_handle* h, uint64_t* node_id, uint64_t* brick_id, float* t, float* normal);

/* Copies the device-cache slot of brick `code` (Morton code at levelCubes)
 * into host_out: (edge + 2*cubeInc)^3 voxels of the volume's type, the
 * zero-padded box [min - cubeInc, min + edge + cubeInc) x slowest, as
 * lruCache's bricks (src/lruCache.cu:224-226).  *resident = 0, and nothing
 * is copied, when the brick has no slot (or the renderer is resident).
 * Synchronises the device. */
vt_status vt_debug_slot(vt_handle* h, uint64_t code, void* host_out, int* resident);

typedef struct {
    int64_t frames, rays, hits, samples, normal_samples, candidates, expansions;
    int64_t passes;                 /* demand passes in the last frame */
    int64_t bricks_requested, bricks_loaded_host, bricks_loaded_disk, bricks_prefetched;
    int64_t device_hits, device_misses, host_hits, host_misses;
    int64_t max_stack;
    int64_t launches;               /* libvt kernels launched (cumulative) */
    int64_t bricks_hinted;          /* bricks named by vt_prefetch and by hints a frame consumed */
    int64_t bricks_staged;          /* of those, absent from the device cache when staged */
    int64_t bricks_speculative;     /* lookahead requests among bricks_requested */
    double  ms_last_frame, ms_stall_last_frame, bytes_h2d_last_frame;
    double  ms_trace_last_frame;    /* device time of the trace kernels of the last frame */
    double  ms_prefetch_last_frame; /* host time of the hinted prefetch's device fill */
    double  ms_host_read_total;     /* cumulative host time reading bricks into the host tier */
    double  ms_fill_wait_total;     /* cumulative host time waiting for device fills to finish */
    double  ms_wait_last_frame;     /* host time of the last frame blocked on its passes' results */
    int64_t requests_deferred;      /* brick requests past max_requests, retried a pass later */
    int64_t bricks_spec_loaded;     /* lookahead bricks loaded on the side stream (spec_async) */
} vt_stats;
vt_status vt_get_stats(vt_handle* h, vt_stats* s);
/* Empties the brick cache (both tiers): the next frame starts cold.
 * Synchronises the device. */
vt_status vt_drop_cache(vt_handle* h);
vt_status vt_reset_stats(vt_handle* h);

/* ------------------------------------------------------------------------ */
/* Learned brick prefetch (no reference counterpart)                       */
/* ------------------------------------------------------------------------ */
/* Multi-layer perceptron in -> h1 -> h2 -> out (ReLU, ReLU, sigmoid) with
 * BF16 weights, FP32 master weights and FP32 accumulation; He-initialised
 * from `seed`.  Used as pose (12 features) -> per-coarse-node probability
 * that a frame from that pose marches the node. */
vt_status vt_mlp_create(int in, int h1, int h2, int out, uint64_t seed, vt_mlp** m);
void      vt_mlp_free(vt_mlp* m);
/* probabilities of `batch` rows of dev_x (batch x in floats) into dev_p */
vt_status vt_mlp_forward(vt_mlp* m, const float* dev_x, int batch, float* dev_p, void* stream);
/* one Adam step on the mean binary cross-entropy against dev_y (batch x
 * out targets in {0,1}); *loss (host, may be NULL) gets the batch loss and
 * the call then synchronises */
vt_status vt_mlp_train_step(vt_mlp* m, const float* dev_x, const float* dev_y, int batch, float lr,
                            float* loss, void* stream);
/* gradients of the batch loss without updating (host buffer laid out as
 * the weights); synchronises */
vt_status vt_mlp_gradients(vt_mlp* m, const float* dev_x, const float* dev_y, int batch, float* host_grads,
                           float* loss);
/* GEMMs on the tensor cores (tcgen05; the default, GEMM inputs rounded to
 * BF16) or, with on = 0, on the SIMT FMA pipes (FP32 activations) */
vt_status vt_mlp_use_tensor_cores(vt_mlp* m, int on);
/* the network's layer widths: in, h1, h2, out */
vt_status vt_mlp_info(const vt_mlp* m, int dims[4]);
/* FP32 master weights, layer by layer: W (in x out, row-major) then b */
vt_status vt_mlp_get_weights(vt_mlp* m, float* host, int64_t* n);
vt_status vt_mlp_set_weights(vt_mlp* m, const float* host, int64_t n);
/* vt_mlp_forward without any allocation (no counterpart in the reference).
 * For callers that cannot allocate GPU memory where they run inference --
 * a render loop in a host that owns the device's memory budget, or a frame
 * thread that must not call cudaMalloc (it synchronises the device).  The
 * hidden activations use a fixed 1 MiB device array built into libvt.so,
 * so batch * (h1 + h2) must be at most 262144 floats (e.g. batch 256 for
 * 512 + 512 hidden units); larger batches return VT_ERR_INVALID.  The first
 * call on each device looks the array's address up (cudaGetSymbolAddress):
 * make that first call before any stream capture.  After a cudaDeviceReset
 * the next call looks it up again, so make that call outside a capture too.
 * All calls on a device
 * share the array: calls that overlap on the GPU (other streams, threads)
 * race and must be serialised by the caller. */
vt_status vt_mlp_forward_noalloc(vt_mlp* m, const float* dev_x, int batch, float* dev_p, void* stream);

#ifdef __cplusplus
}
#endif
#endif
