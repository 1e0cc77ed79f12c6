/*
 * vt_kernels.h -- argument blocks shared by the host runtime and the CUDA
 * kernels of libvt.so (internal header; the public ABI is include/vt.h).
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define VT_MAX_LEVELS 20
#define VT_STACK 64          /* per-ray DFS stack entries (reference: 32) */
#define VT_SKIP_MAX 4        /* absent-brick candidates a ray may pass over in one pass */

/* error bits reported by kernels through DevCtl::err */
#define VT_KERR_STACK 1u        /* a ray's stack overflowed */
#define VT_KERR_NOTRESIDENT 2u  /* resident mode met a brick with no slot */
#define VT_KERR_SUSPEND_FULL 4u /* suspended-ray list overflowed */
#define VT_KERR_STAGE 8u        /* a bounded wait for a staged brick gave up */
#define VT_KERR_WAVE 16u        /* a wavefront round ran out of item room (cannot happen: one item a ray) */
/* page-table states besides a slot index: -1 absent, and */
#define VT_PAGE_REQUESTED (-2)     /* a ray waits on the brick */
#define VT_PAGE_SPECULATIVE (-3)   /* requested ahead of need (lookahead) */
#define VT_REQ_SPECULATIVE (1ull << 63)   /* request-list tag of a speculative request */

/* counter slots in DevCtl::counters */
enum {
    VT_C_RAYS = 0, VT_C_HITS, VT_C_SAMPLES, VT_C_NSAMPLES, VT_C_CANDIDATES, VT_C_EXPANSIONS,
    VT_C_MAXSTACK, VT_C_SUSPENDED, VT_C_REQUESTS, VT_C_DEVHITS, VT_C_DEVMISSES, VT_C_REQDEFER, VT_C_COUNT
};

struct DevCamera {
    float3 look, up, right, pos;
    float h, w, dist;
    int W, H;
};

/* Flattened octree: records of the reachable nodes of levels 0..Lo-1 in
 * one array, level after level.  node.x = array index of the first child,
 * node.y = 8-bit child mask (bit k = child (code<<3)+k accepted by the
 * reference's range search); children of a node are contiguous. */
struct DevOctree {
    int nLevels, Lo, Lc, rootValid;
    const uint2* nodes;
};

/* DFS stack entry (8 bytes): node array index, level, and the node's
 * coordinates in units of its own size (each < 2^level). */
#define VT_E_COORD_BITS 11
#define VT_E_LEVEL_SHIFT 33
#define VT_E_INDEX_SHIFT 37
#define VT_MAX_OCTREE_LEVEL 11                 /* coordinates fit 11 bits */
#define VT_MAX_INNER_NODES (1u << 27)          /* index field */

/* Brick storage.  Dense: the whole zero-padded volume, P voxels of zeros on
 * every side; index ((x+P)*ey + (y+P))*ez + (z+P).  Slab: bricks of D^3
 * voxels (edge + 2*inc) in slots; page[(bx << 2Lc) | (by << Lc) | bz] =
 * slot or < 0, (bx,by,bz) the brick's coordinates in bricks. */
struct DevBricks {
    const void* vol;  long long vsx, vsy; int P; int ve;   /* ve: padded edge */
    int* page; unsigned long long pageBase; const void* slab; int D; long long brickVol;
    int inc; int vtype;
    unsigned int* stamp;   /* per slot: last pass that used it (slab mode) */
    unsigned int pass;
};

/* Per-ray diagnostics, pixel-indexed for view 0 (single-view renders). */
struct DevOut {
    unsigned long long* node;
    unsigned long long* brick;
    float* t;
    float* n;
};

/* One camera view of a batch.  Rays are numbered in tile order: view v owns
 * the padded ray indices [rayBase, rayBase + tilesX*tilesY*tw*th). */
#define VT_MAX_VIEWS 64
struct DevView {
    DevCamera cam;
    float4* rgba;
    uint8_t* rgb8;
    unsigned int rayBase;
    unsigned int tilesX;
};
struct DevViews {
    const DevView* v;
    int n;
    unsigned int totalRays;
};

/* A suspended ray: padded global ray index, saved stack depth (0 = restart
 * from the root) and offset of its entries in the stack pool. */
/* A suspended ray: its pool entries at `off` are its passed-over
 * candidates (depth bits 8-10), then its DFS stack (bits 0-7); bit 11: its
 * pixel already holds a hit found past those candidates. */
struct SuspRec {
    unsigned int ray;
    unsigned int depth;
    unsigned long long off;
};

/* Per-pass control: counters, error bits, work queue, demand paging. */
struct DevCtl {
    unsigned long long* counters;
    unsigned int* err;
    unsigned int* work;                         /* persistent-kernel work counter */
    const SuspRec* in; unsigned int n_in;      /* rays to resume (NULL: pass 0) */
    const unsigned int* n_in_dev;               /* if set: the count, in device memory (n_in bounds it) */
    const unsigned long long* pool_in;
    SuspRec* out; unsigned int* n_out; unsigned int out_cap;
    unsigned long long* pool_out; unsigned long long* pool_used; unsigned long long pool_cap;
    unsigned long long* req; unsigned int* n_req; unsigned int req_cap;
    int lookahead;                              /* bricks a suspended ray may request ahead */
    int skip;                                   /* absent-brick candidates a ray may pass over */
    unsigned int* touched; int touch_shift;     /* optional bitmask of coarse nodes used (trace log) */
    unsigned long long touch_base;
};

struct TraceArgs {
    DevViews views;
    DevOctree oct;
    DevBricks br;
    DevOut out;
    DevCtl ctl;
    float iso;
    float3 light;
    int tile_w, tile_h;
    int pops;                                   /* pops between warp refills (persistent) */
    int unroll;                                 /* march samples fetched per round: 1, 2, 4, 8 */
    int refine;                                 /* bisection steps before the linear refinement */
};

/* Wavefront passes (slab mode): a traversal kernel walks each ray's DFS to
 * its next candidate whose brick is resident and queues (ray, candidate)
 * as a march item, binned by brick slot; a march kernel stages each binned
 * slot into shared memory with one bulk copy and marches its items from
 * there.  Rays whose candidate missed wait (their stack in a wait pool) for
 * the next traversal round. */
struct MarchItem {
    unsigned long long entry;   /* the candidate's stack entry */
    unsigned int rec;           /* the ray's wait record (its remaining stack) */
    int slot;                   /* brick slot */
    float tn;                   /* candidate slab entry parameter */
    int maxStep;                /* march steps */
    unsigned int g;             /* padded global ray index */
    unsigned int rank;          /* position among the slot's items */
    float dx, dy, dz;           /* ray direction */
    unsigned int pad;
};
struct WaveRound {
    /* input of this round: the pass's rays (in == NULL in a first pass: ray
     * indices 0..count) or the previous round's waiting records */
    const SuspRec* in; const unsigned int* n_in; unsigned int n_in_host; const unsigned long long* pool_in;
    /* waiting rays of this round */
    SuspRec* wait; unsigned int* n_wait; unsigned long long* pool_wait; unsigned long long* pool_wait_used;
    unsigned long long pool_wait_cap; unsigned int wait_cap;
    /* march items, binned by slot */
    MarchItem* items; unsigned int* n_items; MarchItem* sorted; unsigned int items_cap;
    unsigned int* binCount; unsigned int* binStart; unsigned int* touched; unsigned int* n_touched;
    /* rays whose candidate missed: the next round's input */
    SuspRec* next; unsigned int* n_next;
    unsigned int* work;         /* persistent work counter */
    int last;                   /* last round: misses join the pass's suspended list instead */
};

/* launchers (render.cu) */
cudaError_t vt_launch_trace(const TraceArgs& a, bool slab, bool persistent, int blocks_per_sm, cudaStream_t s);
cudaError_t vt_launch_wave_round(const TraceArgs& a, const WaveRound& w, int blocks_per_sm, size_t slotBytes,
                                 cudaStream_t s);
cudaError_t vt_launch_rays(const DevCamera& c, float* dirs, cudaStream_t s);
cudaError_t vt_launch_cube(const DevCamera& c, const float* cube, int3 minBox, int3 cubeDim,
                           int3 cubeInc, float iso, float3 light, float4* rgba, cudaStream_t s);
/* learned prefetch: speculative requests of the leaf bricks whose coarse
 * node (at `level`) has a largest probability over `ncams` rows above thr */
cudaError_t vt_launch_predict_requests(int* page, const unsigned int* leafPages, int nLeaf, const float* probs,
                                       int ncams, int level, int Lc, float thr, unsigned int* list,
                                       unsigned int* count, unsigned int cap, cudaStream_t s);
cudaError_t vt_launch_fill_dense(void* dst, int vtype, const void* src, long long nx, long long ny,
                                 long long nz, int P, long long ey, long long ez, cudaStream_t s);
