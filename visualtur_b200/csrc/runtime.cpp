/*
 * runtime.cpp -- the renderer handle of libvt.so: camera state (class
 * Camera/Screen), octree flattening and upload (class Octree), brick
 * residency (class lruCache) and the frame loop (visualTur::
 * updateVisibleCubes, src/visualTur.cu:167-228), behind the C ABI.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <stddef.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vt_kernels.h"
#include "vt_runtime.h"
#include "cache.h"
#include "vt_math.cuh"

using namespace vtrt;

namespace vtrt { const char* last_error(); }

extern "C" const char* vt_last_error(void) { return vtrt::last_error(); }
extern "C" int vt_api_version(void) { return VT_API_VERSION; }
extern "C" const char* vt_status_string(vt_status s) {
    switch (s) {
        case VT_OK: return "ok";
        case VT_ERR_INVALID: return "invalid argument";
        case VT_ERR_CUDA: return "CUDA error";
        case VT_ERR_IO: return "I/O error";
        case VT_ERR_FORMAT: return "bad file format";
        case VT_ERR_NOMEM: return "out of memory";
        case VT_ERR_TIMEOUT: return "timeout";
        case VT_ERR_STACK: return "traversal stack overflow";
        case VT_ERR_UNSUPPORTED: return "unsupported";
        case VT_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(VT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

/* ======================================================================== */
/* Camera (src/Camera.cu, src/Screen.cpp)                                   */
/* ======================================================================== */
static float3 mk3(const float* a) { return make_float3(a[0], a[1], a[2]); }
static void put3(float* a, float3 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }
static float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
static float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

static void screen_extent(float d, float fh, float fw, float* h, float* w) {   /* Screen.cpp:18-19 */
    *h = 2 * d * tanf(fh * (M_PI / 180.0));
    *w = 2 * d * tanf(fw * (M_PI / 180.0));
}

extern "C" vt_status vt_camera_init(vt_camera* c, int H, int W, float d, float fh, float fw) {
    clear_error();
    if (!c || H <= 0 || W <= 0) return fail(VT_ERR_INVALID, "vt_camera_init: bad arguments");
    memset(c, 0, sizeof(*c));
    c->H = H; c->W = W; c->distance = d;
    screen_extent(d, fh, fw, &c->h, &c->w);
    float3 look = make_float3(0.0f, 0.0f, -1.0f), up = make_float3(0.0f, 1.0f, 0.0f);   /* Camera.cu:17-20 */
    put3(c->look, look); put3(c->up, up);
    put3(c->right, cross3(look, up));
    put3(c->position, make_float3(0.0f, 0.0f, 0.0f));
    return VT_OK;
}

extern "C" vt_status vt_camera_op(vt_camera* c, int op, float a, float b, float cc) {
    clear_error();
    if (!c) return fail(VT_ERR_INVALID, "null camera");
    float3 look = mk3(c->look), up = mk3(c->up), right = mk3(c->right), pos = mk3(c->position);
    switch (op) {
        case 0: pos = add3(pos, make_float3(a, b, cc)); break;                  /* Move :85-89 */
        case 1: {                                                                /* RotateX :91-106 */
            float s = sin(a * (M_PI / 180.0)), co = cos(a * (M_PI / 180.0));
            look = add3(mul3(look, co), mul3(up, s));
            up = mul3(cross3(look, right), -1.0f);
            break;
        }
        case 2: {                                                                /* RotateY :108-122 */
            float s = sin(a * (M_PI / 180.0)), co = cos(a * (M_PI / 180.0));
            look = sub3(mul3(look, co), mul3(right, s));
            right = cross3(look, up);
            break;
        }
        case 3: {                                                                /* RotateZ :124-138 */
            float s = sin(a * (M_PI / 180.0)), co = cos(a * (M_PI / 180.0));
            right = add3(mul3(right, co), mul3(up, s));
            up = mul3(cross3(look, right), -1.0f);
            break;
        }
        case 4: pos = add3(pos, mul3(look, -a)); break;                        /* MoveForward :140-144 */
        case 5: pos = add3(pos, mul3(right, a)); break;                        /* MoveUpward :146-150 */
        case 6: pos = add3(pos, mul3(up, a)); break;                           /* StrafeRight :152-156 */
        default: return fail(VT_ERR_INVALID, "unknown camera op %d", op);
    }
    put3(c->look, look); put3(c->up, up); put3(c->right, right); put3(c->position, pos);
    return VT_OK;
}

static DevCamera dev_camera(const vt_camera& c) {
    DevCamera d;
    d.look = mk3(c.look); d.up = mk3(c.up); d.right = mk3(c.right); d.pos = mk3(c.position);
    d.h = c.h; d.w = c.w; d.dist = c.distance; d.W = c.W; d.H = c.H;
    return d;
}

extern "C" vt_status vt_camera_rays(const vt_camera* c, float* dev_dirs, void* stream) {
    clear_error();
    if (!c || !dev_dirs) return fail(VT_ERR_INVALID, "vt_camera_rays: null argument");
    CK(vt_launch_rays(dev_camera(*c), dev_dirs, (cudaStream_t)stream));
    return VT_OK;
}

extern "C" vt_status vt_render_cube(const vt_camera* c, const float* dev_cube, const int minBox[3],
                                    const int cubeDim[3], const int cubeInc[3], float iso, const float light[3],
                                    float* dev_rgba, void* stream) {
    clear_error();
    if (!c || !dev_cube || !minBox || !cubeDim || !cubeInc || !dev_rgba) return fail(VT_ERR_INVALID, "vt_render_cube: null argument");
    float3 l = light ? mk3(light) : make_float3(0.0f, 512.0f, 0.0f);
    CK(vt_launch_cube(dev_camera(*c), dev_cube, make_int3(minBox[0], minBox[1], minBox[2]),
                      make_int3(cubeDim[0], cubeDim[1], cubeDim[2]), make_int3(cubeInc[0], cubeInc[1], cubeInc[2]),
                      iso, l, (float4*)dev_rgba, (cudaStream_t)stream));
    return VT_OK;
}

/* ======================================================================== */
/* Renderer handle                                                          */
/* ======================================================================== */
/* control block: one memset clears a pass's counters */
struct CtlBlock {
    unsigned long long counters[VT_C_COUNT];
    unsigned int err;
    unsigned int n_out, n_req, work;       /* reset every pass */
    unsigned long long pool_used;
};

struct vt_handle {
    vt_params p;
    vt_options opt;
    vt_volume* vol = nullptr; bool ownVol = false;
    vt_octree* oct = nullptr; bool ownOct = false;
    vt_camera cam;
    float fovH = 0, fovW = 0;
    int nLevels = 0, Lo = 0, Lc = 0, inc = 3, edge = 0, D = 0;
    /* flattened octree */
    uint2* d_nodes = nullptr;
    size_t nodeCount = 0;
    int rootValid = 0;
    std::vector<uint64_t> leafBricks;   /* bricks holding reachable candidate nodes */
    /* dense residency */
    void* d_vol = nullptr; int P = 4; long long ve = 0;
    /* brick cache */
    vtrt::BrickCache* cache = nullptr;
    /* single-view output buffers */
    int nRays = 0;
    float4* d_rgba = nullptr; uint8_t* d_rgb8 = nullptr;
    unsigned long long* d_node = nullptr; unsigned long long* d_brick = nullptr; float* d_t = nullptr; float* d_n = nullptr;
    /* control */
    CtlBlock* d_ctl = nullptr; CtlBlock* h_ctl = nullptr;
    DevView* d_views = nullptr; DevView* h_views = nullptr;
    unsigned int* d_touched = nullptr; size_t touchedWords = 0;
    /* suspended rays (ping-pong) */
    unsigned int susp_cap = 0; unsigned long long pool_cap = 0;
    SuspRec* d_susp[2] = {nullptr, nullptr};
    unsigned long long* d_pool[2] = {nullptr, nullptr};
    unsigned long long* d_req = nullptr; unsigned int req_cap = 0;
    /* timing and the pass-0 graph */
    std::vector<cudaEvent_t> ev;
    cudaGraphExec_t graph = nullptr;
    int passKernels = 1;                   /* kernels of the last pass enqueued */
    cudaStream_t s_int = nullptr;
    std::vector<uint64_t> hint;            /* bricks to load for the next frame */
    /* wavefront passes: per-round waiting rays (ping-pong), march items and bins */
    struct WaveCtl { unsigned int n_wait, n_items, n_touched, n_next; unsigned long long pool_wait_used; };
    unsigned int wave_cap = 0;
    SuspRec* d_wwait[2] = {nullptr, nullptr}; SuspRec* d_wnext[2] = {nullptr, nullptr};
    unsigned long long* d_wpool[2] = {nullptr, nullptr}; unsigned long long wpool_cap = 0;
    MarchItem* d_witems = nullptr; MarchItem* d_wsorted = nullptr;
    unsigned int* d_wbins = nullptr;    /* count, start per slot; touched list */
    WaveCtl* d_wctl = nullptr;          /* [2] */
    /* learned prefetch on the device (vt_prefetch_predict) */
    unsigned int* d_leafPages = nullptr; int nLeaf = 0;
    float* d_feat = nullptr; float* h_feat = nullptr; float* d_probs = nullptr; int predCap = 0; int probsCap = 0;
    unsigned int* d_pred = nullptr; unsigned int* h_pred = nullptr;   /* [0] = count, then pages */
    cudaEvent_t predDone = nullptr; bool predPending = false;
    vt_stats stats;
    bool lastValid = false;
};

static void free_ray_buffers(vt_handle* h) {
    cudaFree(h->d_rgba); cudaFree(h->d_rgb8); cudaFree(h->d_node); cudaFree(h->d_brick); cudaFree(h->d_t); cudaFree(h->d_n);
    h->d_rgba = nullptr; h->d_rgb8 = nullptr; h->d_node = nullptr; h->d_brick = nullptr; h->d_t = nullptr; h->d_n = nullptr;
}

static vt_status alloc_ray_buffers(vt_handle* h) {
    free_ray_buffers(h);
    h->nRays = h->cam.W * h->cam.H;
    size_t n = (size_t)h->nRays;
    CK(cudaMalloc(&h->d_rgba, n * sizeof(float4)));
    CK(cudaMalloc(&h->d_rgb8, n * 3));
    if (h->opt.record_hits) {
        CK(cudaMalloc(&h->d_node, n * 8)); CK(cudaMalloc(&h->d_brick, n * 8));
        CK(cudaMalloc(&h->d_t, n * 4)); CK(cudaMalloc(&h->d_n, n * 12));
    }
    h->lastValid = false;
    return VT_OK;
}

/* suspended-ray records for `rays` rays and a stack pool of 12 entries per
 * ray on average (pool_per_ray; rays whose stack does not fit restart from
 * the root) */
static vt_status ensure_suspend_buffers(vt_handle* h, unsigned int rays) {
    if (h->susp_cap >= rays) return VT_OK;
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_susp[i]); cudaFree(h->d_pool[i]);
        h->d_susp[i] = nullptr; h->d_pool[i] = nullptr;
    }
    /* grow by half again at least: a caller that adds views one at a time
     * reallocates (and synchronises the device) only a few times */
    rays = (unsigned int)std::min<unsigned long long>(0xFFFFFFFFull,
                                                      std::max<unsigned long long>(rays, h->susp_cap + h->susp_cap / 2ull));
    h->susp_cap = rays;
    h->pool_cap = (unsigned long long)rays * (unsigned long long)(h->opt.pool_per_ray > 0 ? h->opt.pool_per_ray : 12);
    for (int i = 0; i < 2; i++) {
        CK(cudaMalloc(&h->d_susp[i], (size_t)rays * sizeof(SuspRec)));
        CK(cudaMalloc(&h->d_pool[i], (size_t)h->pool_cap * 8));
    }
    return VT_OK;
}

/* Octree flattening: keeps the nodes reachable from the root through the
 * reference's traversal (src/Octree.cu:620-739) and records, per node, the
 * children its range search accepts -- a property of the node alone.  All
 * levels 0..Lo-1 go into one array; a record holds the array index of its
 * node's first child. */
static vt_status flatten_octree(vt_handle* h) {
    const vt_octree* o = h->oct;
    const int Lo = h->Lo;
    if (Lo > VT_MAX_OCTREE_LEVEL) return fail(VT_ERR_UNSUPPORTED, "octreeLevel %d > %d", Lo, VT_MAX_OCTREE_LEVEL);
    const std::vector<uint64_t>& l0 = o->levels[0];
    h->rootValid = (l0.size() >= 2 && (l0[0] == 1 || l0[1] == 1 || (l0[0] < 1 && l0[1] > 1))) ? 1 : 0;
    std::vector<uint64_t> codes(1, 1ull), next;
    std::vector<uint2> all;
    for (int l = 0; l < Lo; l++) {
        const std::vector<uint64_t>& e = o->levels[l + 1];
        std::vector<int> mask(codes.size());
#pragma omp parallel for schedule(dynamic, 4096)
        for (long long i = 0; i < (long long)codes.size(); i++)
            mask[i] = children_mask(e.data(), (int)e.size(), codes[i]);
        const uint64_t nextBase = all.size() + codes.size();   /* level l+1 starts after level l */
        next.clear();
        uint64_t run = 0;
        for (size_t i = 0; i < codes.size(); i++) {
            uint2 r;
            r.x = (unsigned int)(nextBase + run);
            r.y = (unsigned int)mask[i];
            all.push_back(r);
            for (int k = 0; k < 8; k++)
                if ((mask[i] >> k) & 1) next.push_back((codes[i] << 3) + (uint64_t)k);
            run += __builtin_popcount(mask[i]);
        }
        if (l + 1 < Lo && all.size() + next.size() > VT_MAX_INNER_NODES)
            return fail(VT_ERR_UNSUPPORTED, "octree has more than %u inner nodes", VT_MAX_INNER_NODES);
        codes.swap(next);
    }
    h->nodeCount = all.size();
    CK(cudaMalloc(&h->d_nodes, std::max<size_t>(all.size(), 1) * sizeof(uint2)));
    CK(cudaMemcpy(h->d_nodes, all.data(), all.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    /* bricks that hold reachable candidates, as Morton codes at levelCubes */
    const int shift = 3 * (Lo - h->Lc);
    h->leafBricks.clear();
    for (size_t i = 0; i < codes.size(); i++) {
        uint64_t b = codes[i] >> shift;
        if (h->leafBricks.empty() || h->leafBricks.back() != b) h->leafBricks.push_back(b);
    }
    return VT_OK;
}

/* brick Morton code at levelCubes <-> page-table index (bx << 2Lc | by << Lc | bz) */
static inline uint64_t code_to_page(uint64_t code, int Lc) {
    int3 c = vt::min_box(code, Lc, Lc);
    return ((uint64_t)c.x << (2 * Lc)) | ((uint64_t)c.y << Lc) | (uint64_t)c.z;
}
static inline uint64_t page_to_code(uint64_t p, int Lc) {
    uint64_t m = (1ull << Lc) - 1;
    return vt::node_code((uint32_t)(p >> (2 * Lc)), (uint32_t)((p >> Lc) & m), (uint32_t)(p & m), Lc);
}
static std::vector<uint64_t> to_pages(const std::vector<uint64_t>& codes, int Lc) {
    std::vector<uint64_t> p(codes.size());
    for (size_t i = 0; i < codes.size(); i++) p[i] = code_to_page(codes[i], Lc);
    return p;
}

static vt_status upload_dense(vt_handle* h) {
    const vt_volume* v = h->vol;
    if (!v->data) return fail(VT_ERR_UNSUPPORTED, "a resident renderer needs the volume in memory, not a read function");
    h->ve = (long long)(1 << h->nLevels) + 2 * h->P;
    for (int a = 0; a < 3; a++)
        if (v->dims[a] > (1 << h->nLevels)) return fail(VT_ERR_INVALID, "volume larger than the octree");
    size_t es = v->esize();
    size_t bytes = (size_t)h->ve * h->ve * h->ve * es;
    CK(cudaMalloc(&h->d_vol, bytes));
    CK(cudaMemset(h->d_vol, 0, bytes));
    /* stream the volume through a mapped pinned staging buffer, x-slab by x-slab */
    const long long nx = v->dims[0], ny = v->dims[1], nz = v->dims[2];
    long long slab = std::max<long long>(1, (256ll << 20) / (ny * nz * (long long)es));
    void* stage = nullptr;
    void* dstage = nullptr;
    CK(cudaHostAlloc(&stage, (size_t)(slab * ny * nz) * es, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(&dstage, stage, 0));
    for (long long x0 = 0; x0 < nx; x0 += slab) {
        long long cnt = std::min(slab, nx - x0);
        memcpy(stage, v->data + (size_t)(x0 * ny * nz) * es, (size_t)(cnt * ny * nz) * es);
        char* dst = (char*)h->d_vol + (size_t)(x0 * h->ve * h->ve) * es;
        cudaError_t e = vt_launch_fill_dense(dst, v->vtype, dstage, cnt, ny, nz, h->P, h->ve, h->ve, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { cudaFreeHost(stage); return fail(VT_ERR_CUDA, "dense upload: %s", cudaGetErrorString(e)); }
    }
    cudaFreeHost(stage);
    return VT_OK;
}

extern "C" void vt_default_options(vt_options* o) {
    memset(o, 0, sizeof(*o));
    o->resident = 0;
    o->tile_w = 8; o->tile_h = 4;
    o->unroll = 1;
    o->lookahead = 0;
    o->max_passes = 4096;
    o->host_threads = 0;
    o->record_trace = 0;
    o->trace_level = 4;
    o->record_hits = 1;
    o->persistent = 0;
    o->blocks_per_sm = 8;
    o->pops = 32;
    o->preload = 1;
    o->use_graph = 1;
    o->refine = 0;
    o->skip = 0;
    o->max_suspended = 0;
    o->max_requests = 0;
    o->pool_per_ray = 0;
    o->spec_async = 1;
    o->wavefront = 0;
    o->shared_aprons = 1;
    o->demand_batch = 0;
}

static vt_status validate(const vt_params* p, const vt_octree* o, const vt_options* opt) {
    if (p->W <= 0 || p->H <= 0) return fail(VT_ERR_INVALID, "screen size must be positive");
    if (p->numRayPx != 1) return fail(VT_ERR_UNSUPPORTED, "numRayPx must be 1 (the reference generates W*H rays only)");
    if (p->octreeLevel < 1 || p->octreeLevel > o->nLevels) return fail(VT_ERR_INVALID, "octreeLevel %d outside 1..%d", p->octreeLevel, o->nLevels);
    if (p->levelCubes < 0 || p->levelCubes > p->octreeLevel) return fail(VT_ERR_INVALID, "levelCubes must be in 0..octreeLevel");
    if (p->levelCubes > 9) return fail(VT_ERR_UNSUPPORTED, "levelCubes > 9: brick table too large");
    int b = 1 << (o->nLevels - p->levelCubes);
    if (p->dimCubeCache[0] != b || p->dimCubeCache[1] != b || p->dimCubeCache[2] != b)
        return fail(VT_ERR_INVALID, "dimCubeCache must be %d^3 for levelCubes %d of a %d-level octree", b, p->levelCubes, o->nLevels);
    if (p->cubeInc < 3) return fail(VT_ERR_INVALID, "cubeInc must be >= 3 so every trilinear and normal tap stays in the brick");
    if (opt) {
        int tw = opt->tile_w, th = opt->tile_h;
        if (tw <= 0 || th <= 0 || tw * th > 4096) return fail(VT_ERR_INVALID, "tile %dx%d: 1..4096 rays", tw, th);
        if (opt->unroll != 1 && opt->unroll != 2 && opt->unroll != 4 && opt->unroll != 8)
            return fail(VT_ERR_INVALID, "unroll must be 1, 2, 4 or 8");
        if (opt->refine < 0 || opt->refine > 16) return fail(VT_ERR_INVALID, "refine must be in 0..16");
        if (opt->skip < 0 || opt->skip > VT_SKIP_MAX) return fail(VT_ERR_INVALID, "skip must be in 0..%d", VT_SKIP_MAX);
        if (opt->max_passes < 1) return fail(VT_ERR_INVALID, "max_passes must be >= 1");
        if (opt->max_suspended < 0 || opt->max_requests < 0 || opt->pool_per_ray < 0)
            return fail(VT_ERR_INVALID, "queue bounds must be >= 0 (0 = default)");
        if (opt->wavefront < 0 || opt->wavefront > 8) return fail(VT_ERR_INVALID, "wavefront rounds must be in 0..8");
        if (opt->demand_batch < 0) return fail(VT_ERR_INVALID, "demand_batch must be >= 0");
        if (opt->record_trace && (opt->trace_level < 1 || opt->trace_level > p->octreeLevel || opt->trace_level > 8))
            return fail(VT_ERR_INVALID, "trace_level must be in 1..min(octreeLevel, 8)");
    }
    return VT_OK;
}

static vt_status init_handle(vt_handle* h) {
    vt_status s;
    const vt_params& p = h->p;
    h->nLevels = h->oct->nLevels; h->Lo = p.octreeLevel; h->Lc = p.levelCubes; h->inc = p.cubeInc;
    h->edge = 1 << (h->nLevels - h->Lc);
    h->D = h->edge + 2 * h->inc;
    h->fovH = p.fov_H; h->fovW = p.fov_W;
    if ((s = vt_camera_init(&h->cam, p.H, p.W, p.distance, p.fov_H, p.fov_W)) != VT_OK) return s;
    if ((s = flatten_octree(h)) != VT_OK) return s;
    CK(cudaStreamCreateWithFlags(&h->s_int, cudaStreamNonBlocking));
    CK(cudaMalloc(&h->d_ctl, sizeof(CtlBlock)));
    CK(cudaHostAlloc(&h->h_ctl, sizeof(CtlBlock), cudaHostAllocDefault));
    CK(cudaMalloc(&h->d_views, VT_MAX_VIEWS * sizeof(DevView)));
    CK(cudaHostAlloc(&h->h_views, VT_MAX_VIEWS * sizeof(DevView), cudaHostAllocDefault));
    if (h->opt.record_trace) {
        h->touchedWords = std::max<size_t>(1, ((size_t)1 << (3 * h->opt.trace_level)) / 32);
        CK(cudaMalloc(&h->d_touched, h->touchedWords * 4));
        CK(cudaMemset(h->d_touched, 0, h->touchedWords * 4));
    }
    if (h->opt.resident) {
        if ((s = upload_dense(h)) != VT_OK) return s;
    } else {
        vtrt::CacheConfig cc;
        cc.vol = h->vol; cc.nLevels = h->nLevels; cc.Lc = h->Lc; cc.inc = h->inc; cc.edge = h->edge;
        cc.deviceSlots = p.maxElementsCache; cc.hostSlots = p.maxElementsCache_CPU;
        cc.hostThreads = h->opt.host_threads;
        cc.asyncSpec = h->opt.spec_async != 0;
        cc.sharedAprons = h->opt.shared_aprons != 0;
        cc.demandBatch = h->opt.demand_batch;
        h->cache = new vtrt::BrickCache();
        if ((s = h->cache->init(cc)) != VT_OK) return s;
        if (h->opt.preload && (size_t)p.maxElementsCache >= h->leafBricks.size()) {
            if ((s = h->cache->preload(to_pages(h->leafBricks, h->Lc))) != VT_OK) return s;
        }
        /* a page enters the list at most twice per pass: speculatively, then
         * upgraded to a demand request */
        h->req_cap = (unsigned int)std::max<size_t>(2 * h->leafBricks.size(), 1);
        if (h->opt.max_requests > 0) h->req_cap = std::min<unsigned int>(h->req_cap, (unsigned int)h->opt.max_requests);
        CK(cudaMalloc(&h->d_req, (size_t)h->req_cap * 8));
    }
    if ((s = alloc_ray_buffers(h)) != VT_OK) return s;
    memset(&h->stats, 0, sizeof(h->stats));
    return VT_OK;
}

extern "C" vt_status vt_create_from(const vt_params* p, const vt_options* opt, vt_volume* v, vt_octree* o,
                                    vt_handle** out) {
    clear_error();
    if (!p || !v || !o || !out) return fail(VT_ERR_INVALID, "vt_create_from: null argument");
    vt_options dopt;
    vt_default_options(&dopt);
    vt_status s = validate(p, o, opt ? opt : &dopt);
    if (s != VT_OK) return s;
    vt_handle* h = new vt_handle();
    h->p = *p;
    h->opt = opt ? *opt : dopt;
    h->vol = v; h->oct = o;
    if ((s = init_handle(h)) != VT_OK) { vt_destroy(h); return s; }
    *out = h;
    return VT_OK;
}

extern "C" vt_status vt_create(const vt_params* p, const vt_options* opt, vt_handle** out) {
    clear_error();
    if (!p || !out || !p->octreeFile || !p->hdf5File) return fail(VT_ERR_INVALID, "vt_create: null argument");
    vt_octree* o = nullptr;
    vt_volume* v = nullptr;
    vt_status s = vt_octree_load(p->octreeFile, &o);
    if (s != VT_OK) return s;
    if ((s = vt_volume_open(p->hdf5File, p->dataset_name, &v)) != VT_OK) { vt_octree_free(o); return s; }
    vt_handle* h = nullptr;
    if ((s = vt_create_from(p, opt, v, o, &h)) != VT_OK) { vt_octree_free(o); vt_volume_close(v); return s; }
    h->ownVol = true; h->ownOct = true;
    *out = h;
    return VT_OK;
}

extern "C" void vt_destroy(vt_handle* h) {
    if (!h) return;
    if (h->s_int) cudaStreamSynchronize(h->s_int);
    cudaDeviceSynchronize();
    free_ray_buffers(h);
    cudaFree(h->d_nodes);
    for (int i = 0; i < 2; i++) { cudaFree(h->d_susp[i]); cudaFree(h->d_pool[i]); }
    cudaFree(h->d_vol); cudaFree(h->d_ctl); cudaFree(h->d_views); cudaFree(h->d_req); cudaFree(h->d_touched);
    if (h->h_ctl) cudaFreeHost(h->h_ctl);
    if (h->h_views) cudaFreeHost(h->h_views);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    cudaFree(h->d_leafPages); cudaFree(h->d_feat); cudaFree(h->d_probs); cudaFree(h->d_pred);
    for (int i = 0; i < 2; i++) { cudaFree(h->d_wwait[i]); cudaFree(h->d_wnext[i]); cudaFree(h->d_wpool[i]); }
    cudaFree(h->d_witems); cudaFree(h->d_wsorted); cudaFree(h->d_wbins); cudaFree(h->d_wctl);
    if (h->h_feat) cudaFreeHost(h->h_feat);
    if (h->h_pred) cudaFreeHost(h->h_pred);
    if (h->predDone) cudaEventDestroy(h->predDone);
    if (h->s_int) cudaStreamDestroy(h->s_int);
    delete h->cache;
    if (h->ownVol) vt_volume_close(h->vol);
    if (h->ownOct) vt_octree_free(h->oct);
    delete h;
}

/* ---- camera / parameter changes (src/visualTur.cu:83-165) -------------- */
extern "C" vt_status vt_camera_update(vt_handle* h, int op, float a, float b, float c) {
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    h->lastValid = false;
    return vt_camera_op(&h->cam, op, a, b, c);
}
extern "C" vt_status vt_set_camera(vt_handle* h, const vt_camera* c) {
    clear_error();
    if (!h || !c) return fail(VT_ERR_INVALID, "null argument");
    if (c->W != h->cam.W || c->H != h->cam.H) return fail(VT_ERR_INVALID, "vt_set_camera cannot resize; use vt_change_screen");
    h->cam = *c;
    h->lastValid = false;
    return VT_OK;
}
extern "C" vt_status vt_get_camera(vt_handle* h, vt_camera* c) {
    clear_error();
    if (!h || !c) return fail(VT_ERR_INVALID, "null argument");
    *c = h->cam;
    return VT_OK;
}
extern "C" vt_status vt_change_screen(vt_handle* h, int W, int H, float fovW, float fovH, float d) {
    clear_error();
    if (!h || W <= 0 || H <= 0) return fail(VT_ERR_INVALID, "bad screen");
    h->cam.W = W; h->cam.H = H; h->cam.distance = d; h->fovW = fovW; h->fovH = fovH;
    screen_extent(d, fovH, fovW, &h->cam.h, &h->cam.w);
    return alloc_ray_buffers(h);
}
extern "C" vt_status vt_change_num_rays(vt_handle* h, int nRP) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    if (nRP != 1) return fail(VT_ERR_UNSUPPORTED, "numRayPx must be 1 (the reference generates W*H rays only)");
    return VT_OK;
}
extern "C" vt_status vt_change_cache(vt_handle* h, int nE, const int cDim[3], int cInc) {
    clear_error();
    if (!h || !cDim) return fail(VT_ERR_INVALID, "null argument");
    if (cDim[0] != h->edge || cDim[1] != h->edge || cDim[2] != h->edge)
        return fail(VT_ERR_INVALID, "brick edge is fixed by levelCubes (%d)", h->edge);
    if (cInc < 3) return fail(VT_ERR_INVALID, "cubeInc must be >= 3");
    if (h->opt.resident) { h->p.maxElementsCache = nE; return VT_OK; }
    vt_status s;
    CK(cudaDeviceSynchronize());
    h->p.maxElementsCache = nE; h->p.cubeInc = cInc; h->inc = cInc; h->D = h->edge + 2 * cInc;
    delete h->cache;
    vtrt::CacheConfig cc;
    cc.vol = h->vol; cc.nLevels = h->nLevels; cc.Lc = h->Lc; cc.inc = h->inc; cc.edge = h->edge;
    cc.deviceSlots = nE; cc.hostSlots = h->p.maxElementsCache_CPU; cc.hostThreads = h->opt.host_threads;
    cc.asyncSpec = h->opt.spec_async != 0;
    cc.sharedAprons = h->opt.shared_aprons != 0;
    cc.demandBatch = h->opt.demand_batch;
    h->cache = new vtrt::BrickCache();
    if ((s = h->cache->init(cc)) != VT_OK) return s;
    if (h->opt.preload && (size_t)nE >= h->leafBricks.size() &&
        (s = h->cache->preload(to_pages(h->leafBricks, h->Lc))) != VT_OK) return s;
    h->lastValid = false;
    return VT_OK;
}

/* ---- frame ---------------------------------------------------------------- */
static void fill_args(vt_handle* h, TraceArgs& a, int nViews, unsigned int totalRays) {
    memset(&a, 0, sizeof(a));
    a.views.v = h->d_views; a.views.n = nViews; a.views.totalRays = totalRays;
    a.oct.nLevels = h->nLevels; a.oct.Lo = h->Lo; a.oct.Lc = h->Lc; a.oct.rootValid = h->rootValid;
    a.oct.nodes = h->d_nodes;
    a.br.vtype = h->vol->vtype; a.br.inc = h->inc;
    if (h->opt.resident) {
        a.br.vol = h->d_vol; a.br.P = h->P; a.br.ve = (int)h->ve;
        a.br.vsx = h->ve * h->ve; a.br.vsy = h->ve;
    } else {
        h->cache->fill_args(a.br);
    }
    if (nViews == 1) { a.out.node = h->d_node; a.out.brick = h->d_brick; a.out.t = h->d_t; a.out.n = h->d_n; }
    CtlBlock* c = h->d_ctl;
    a.ctl.counters = c->counters; a.ctl.err = &c->err; a.ctl.work = &c->work;
    a.ctl.n_out = &c->n_out; a.ctl.n_req = &c->n_req; a.ctl.pool_used = &c->pool_used;
    a.ctl.req = h->d_req; a.ctl.req_cap = h->req_cap;
    a.ctl.lookahead = h->opt.lookahead;
    a.ctl.skip = h->opt.skip;
    if (h->d_touched) {
        a.ctl.touched = h->d_touched;
        a.ctl.touch_shift = 3 * (h->Lo - h->opt.trace_level);
        a.ctl.touch_base = 1ull << (3 * h->opt.trace_level);
    }
    a.iso = h->oct->iso;
    a.light = make_float3(0.0f, 512.0f, 0.0f);   /* src/visualTur.cu:30 */
    a.tile_w = h->opt.tile_w; a.tile_h = h->opt.tile_h;
    a.pops = h->opt.pops > 0 ? h->opt.pops : 8;
    a.unroll = h->opt.unroll;
    a.refine = h->opt.refine;
}

static vt_status collect_counters(vt_handle* h, cudaStream_t s) {
    CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(CtlBlock), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const unsigned long long* c = h->h_ctl->counters;
    vt_stats& st = h->stats;
    st.rays += c[VT_C_RAYS]; st.hits += c[VT_C_HITS]; st.samples += c[VT_C_SAMPLES];
    st.normal_samples += c[VT_C_NSAMPLES]; st.candidates += c[VT_C_CANDIDATES]; st.expansions += c[VT_C_EXPANSIONS];
    st.device_hits += c[VT_C_DEVHITS]; st.device_misses += c[VT_C_DEVMISSES];
    st.max_stack = std::max<int64_t>(st.max_stack, (int64_t)c[VT_C_MAXSTACK]);
    st.requests_deferred += c[VT_C_REQDEFER];
    unsigned int err = h->h_ctl->err;
    if (err & VT_KERR_STACK) return fail(VT_ERR_STACK, "a ray's traversal stack overflowed (%d entries)", VT_STACK);
    if (err & VT_KERR_NOTRESIDENT) return fail(VT_ERR_STATE, "resident render met a brick with no slot");
    if (err & VT_KERR_STAGE) return fail(VT_ERR_TIMEOUT, "a staged brick did not arrive within its wait bound");
    if (err & VT_KERR_WAVE) return fail(VT_ERR_STATE, "a wavefront round ran out of march-item room");
    if (err & VT_KERR_SUSPEND_FULL) return fail(VT_ERR_STATE, "suspended-ray list overflow (more than %u rays waiting on bricks)", h->opt.max_suspended > 0 ? std::min<unsigned int>(h->susp_cap, (unsigned int)h->opt.max_suspended) : h->susp_cap);
    return VT_OK;
}

/* trace launch of pass `k`, between events 2k and 2k+1 */
static vt_status ensure_events(vt_handle* h, int k) {
    while ((int)h->ev.size() < 2 * (k + 1)) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h->ev.push_back(e);
    }
    return VT_OK;
}

/* wavefront passes apply: slab mode, in-order traversal, no trace log */
static bool use_wave(const vt_handle* h, bool slabMode) {
    return slabMode && h->opt.wavefront > 0 && h->opt.skip == 0 && !h->d_touched;
}

/* buffers of wavefront passes over up to `rays` rays */
static vt_status ensure_wave_buffers(vt_handle* h, unsigned int rays) {
    if (h->wave_cap >= rays && h->d_wbins) return VT_OK;
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_wwait[i]); cudaFree(h->d_wnext[i]); cudaFree(h->d_wpool[i]);
        h->d_wwait[i] = h->d_wnext[i] = nullptr; h->d_wpool[i] = nullptr;
    }
    cudaFree(h->d_witems); cudaFree(h->d_wsorted);
    h->d_witems = h->d_wsorted = nullptr;
    rays = (unsigned int)std::max<unsigned long long>(rays, h->wave_cap + h->wave_cap / 2ull);
    h->wave_cap = rays;
    h->wpool_cap = (unsigned long long)rays * 12ull;
    for (int i = 0; i < 2; i++) {
        CK(cudaMalloc(&h->d_wwait[i], (size_t)rays * sizeof(SuspRec)));
        CK(cudaMalloc(&h->d_wnext[i], (size_t)rays * sizeof(SuspRec)));
        CK(cudaMalloc(&h->d_wpool[i], (size_t)h->wpool_cap * 8));
    }
    CK(cudaMalloc(&h->d_witems, (size_t)rays * sizeof(MarchItem)));
    CK(cudaMalloc(&h->d_wsorted, (size_t)rays * sizeof(MarchItem)));
    if (!h->d_wbins) {
        const size_t ns = (size_t)h->cache->device_slots();
        CK(cudaMalloc(&h->d_wbins, ns * 3 * sizeof(unsigned int)));
        CK(cudaMemset(h->d_wbins, 0, ns * 3 * sizeof(unsigned int)));
        CK(cudaMalloc(&h->d_wctl, 2 * sizeof(vt_handle::WaveCtl)));
    }
    return VT_OK;
}

/* One pass's kernels: the fused trace kernel, or wavefront rounds then the
 * fused kernel (persistent, its ray count read on the device) for the rays
 * still waiting.  `bound`: rays the pass can hold (wavefront buffers). */
static cudaError_t launch_pass(vt_handle* h, const TraceArgs& a0, bool slabMode, cudaStream_t s, int* kernels) {
    if (!use_wave(h, slabMode)) {
        *kernels = 1;
        return vt_launch_trace(a0, slabMode, h->opt.persistent != 0, h->opt.blocks_per_sm, s);
    }
    const int rounds = h->opt.wavefront;
    const unsigned int bound = h->wave_cap;
    const size_t ns = (size_t)h->cache->device_slots();
    TraceArgs a = a0;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < rounds && e == cudaSuccess; r++) {
        const int p = r & 1, q = p ^ 1;
        if (r > 0) {
            a.ctl.in = h->d_wnext[q]; a.ctl.n_in = bound; a.ctl.pool_in = h->d_wpool[q];
            a.ctl.n_in_dev = &h->d_wctl[q].n_next;
        }
        WaveRound w;
        memset(&w, 0, sizeof(w));
        w.wait = h->d_wwait[p]; w.n_wait = &h->d_wctl[p].n_wait;
        w.pool_wait = h->d_wpool[p]; w.pool_wait_used = &h->d_wctl[p].pool_wait_used;
        w.pool_wait_cap = h->wpool_cap; w.wait_cap = bound;
        w.items = h->d_witems; w.n_items = &h->d_wctl[p].n_items; w.sorted = h->d_wsorted; w.items_cap = bound;
        w.binCount = h->d_wbins; w.binStart = h->d_wbins + ns; w.touched = h->d_wbins + 2 * ns;
        w.n_touched = &h->d_wctl[p].n_touched;
        w.next = h->d_wnext[p]; w.n_next = &h->d_wctl[p].n_next;
        e = cudaMemsetAsync(&h->d_wctl[p], 0, sizeof(vt_handle::WaveCtl), s);
        if (e == cudaSuccess) e = vt_launch_wave_round(a, w, h->opt.blocks_per_sm, h->cache->slot_bytes(), s);
    }
    if (e != cudaSuccess) return e;
    const int p = (rounds - 1) & 1;
    a.ctl.in = h->d_wnext[p]; a.ctl.n_in = bound; a.ctl.pool_in = h->d_wpool[p]; a.ctl.n_in_dev = &h->d_wctl[p].n_next;
    *kernels = 4 * rounds + 1;
    return vt_launch_trace(a, slabMode, true, h->opt.blocks_per_sm, s);
}

/* pass 0: clear the control block (and trace log), upload the view table,
 * launch the trace kernel -- captured once as a CUDA graph and replayed */
static vt_status pass0(vt_handle* h, const TraceArgs& a, int nViews, bool slabMode, cudaStream_t s) {
    auto enqueue = [&](cudaStream_t q) -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(h->d_ctl, 0, sizeof(CtlBlock), q);
        if (e == cudaSuccess && h->d_touched) e = cudaMemsetAsync(h->d_touched, 0, h->touchedWords * 4, q);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_views, h->h_views, (size_t)nViews * sizeof(DevView), cudaMemcpyHostToDevice, q);
        if (e == cudaSuccess) e = launch_pass(h, a, slabMode, q, &h->passKernels);
        return e;
    };
    if (!h->opt.use_graph || s == 0) {
        CK(enqueue(s));
        return VT_OK;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue(s);
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(VT_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    bool ok = false;
    if (h->graph) {
        cudaGraphExecUpdateResultInfo info;
        ok = cudaGraphExecUpdate(h->graph, g, &info) == cudaSuccess;
        if (!ok) { cudaGetLastError(); cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    }
    if (!ok) {
        e = cudaGraphInstantiate(&h->graph, g, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(g); return fail(VT_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    }
    cudaGraphDestroy(g);
    CK(cudaGraphLaunch(h->graph, s));
    return VT_OK;
}

struct ViewReq { vt_camera cam; float4* rgba; uint8_t* rgb8; };

static vt_status render_views_inner(vt_handle* h, const ViewReq* vr, int n, cudaStream_t s);

/* A frame that ends in an error (a failed brick read, a full queue, the
 * pass bound) leaves pages its last pass requested but nobody will load:
 * they go back to absent, so the next frame requests them again. */
static vt_status render_views(vt_handle* h, const ViewReq* vr, int n, cudaStream_t s) {
    vt_status st = render_views_inner(h, vr, n, s);
    if (st != VT_OK && h->cache && st != VT_ERR_CUDA) {
        std::string msg = vt_last_error();
        h->cache->cancel_requests(s);
        /* wavefront bins start empty (a failed round may have left counts) */
        if (h->d_wbins) cudaMemsetAsync(h->d_wbins, 0, (size_t)h->cache->device_slots() * 4, s);
        fail(st, "%s", msg.c_str());
    }
    return st;
}

static vt_status render_views_inner(vt_handle* h, const ViewReq* vr, int n, cudaStream_t s) {
    auto t0 = std::chrono::steady_clock::now();
    if (n < 1 || n > VT_MAX_VIEWS) return fail(VT_ERR_INVALID, "1..%d views per call", VT_MAX_VIEWS);
    const int tw = h->opt.tile_w, th = h->opt.tile_h;
    unsigned long long base = 0, real = 0;
    for (int k = 0; k < n; k++) {
        const vt_camera& c = vr[k].cam;
        if (c.W <= 0 || c.H <= 0) return fail(VT_ERR_INVALID, "view %d has no pixels", k);
        DevView& v = h->h_views[k];
        v.cam = dev_camera(c);
        v.rgba = vr[k].rgba; v.rgb8 = vr[k].rgb8;
        v.rayBase = (unsigned int)base;
        v.tilesX = (unsigned int)((c.W + tw - 1) / tw);
        base += (unsigned long long)v.tilesX * ((c.H + th - 1) / th) * (unsigned long long)(tw * th);
        real += (unsigned long long)c.W * c.H;
    }
    if (base > 0xFFFFFFFFull) return fail(VT_ERR_UNSUPPORTED, "more than 2^32 rays in one call");
    TraceArgs a;
    fill_args(h, a, n, (unsigned int)base);
    const bool slabMode = !h->opt.resident;
    const bool allResident = h->opt.resident || h->cache->all_resident();
    vt_status st;
    if (!allResident && (st = ensure_suspend_buffers(h, (unsigned int)real)) != VT_OK) return st;
    const unsigned int outCap =
        h->opt.max_suspended > 0 ? std::min<unsigned int>(h->susp_cap, (unsigned int)h->opt.max_suspended) : h->susp_cap;
    a.ctl.out_cap = outCap; a.ctl.pool_cap = h->pool_cap;
    a.ctl.out = h->d_susp[0]; a.ctl.pool_out = h->d_pool[0];
    if (slabMode) { h->cache->begin_frame(); a.br.pass = h->cache->next_pass(); }
    if ((st = ensure_events(h, 0)) != VT_OK) return st;
    CK(cudaEventRecord(h->ev[0], s));
    if (use_wave(h, slabMode) && (st = ensure_wave_buffers(h, std::max<unsigned int>((unsigned int)base, h->susp_cap))) != VT_OK)
        return st;
    if ((st = pass0(h, a, n, slabMode, s)) != VT_OK) return st;
    CK(cudaEventRecord(h->ev[1], s));
    h->stats.launches += h->passKernels;
    int passes = 1;
    double stall = 0, h2d = 0, wait = 0;
    /* prefetch hint for the next frame: host-tier loads overlap this frame's kernel */
    std::vector<uint64_t> staged;
    std::vector<int> stagedSlots;
    if (slabMode && !h->hint.empty()) {
        /* stage in small parts only while pass 0 still runs on the GPU: the
         * host-tier reads then never lengthen the frame; the rest of the
         * hint is dropped */
        const size_t kPart = 1024;
        const uint64_t protect = h->cache->host_tick() + 1;
        for (size_t p0 = 0; p0 < h->hint.size(); p0 += kPart) {
            std::vector<uint64_t> part(h->hint.begin() + p0, h->hint.begin() + std::min(h->hint.size(), p0 + kPart));
            if ((st = h->cache->prefetch_stage(part, staged, stagedSlots, true, protect)) != VT_OK) return st;
            if (cudaEventQuery(h->ev[1]) != cudaErrorNotReady) break;
        }
        if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();   /* the query's answer, not a fault */
        h->hint.clear();
    }
    /* bricks the network predicted for these frames join the side stream's
     * queue ahead of the lookahead requests */
    if (slabMode && h->predPending) {
        h->predPending = false;
        CK(cudaEventSynchronize(h->predDone));
        const unsigned int np = std::min<unsigned int>(h->h_pred[0], (unsigned int)h->nLeaf);
        if (h->cache->async_spec()) {
            h->cache->spec_hint(h->h_pred + 1, np);
        } else {
            h->hint.assign(h->h_pred + 1, h->h_pred + 1 + np);
        }
    }
    /* queued lookahead bricks load on the cache's side stream while the pass runs */
    if (slabMode && (st = h->cache->spec_work(h->ev[1], nullptr)) != VT_OK) return st;
    if (!allResident) {
        int cur = 0;
        for (;;) {
            CK(cudaMemcpyAsync(&h->h_ctl->n_out, &h->d_ctl->n_out, 8, cudaMemcpyDeviceToHost, s));
            const auto tw = std::chrono::steady_clock::now();
            CK(cudaStreamSynchronize(s));
            wait += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
            unsigned int nOut = h->h_ctl->n_out, nReq = std::min(h->h_ctl->n_req, h->req_cap);
            if (nOut == 0) break;
            if (nOut > outCap)
                return fail(VT_ERR_STATE, "suspended-ray list overflow (%u rays waiting on bricks, room for %u)", nOut, outCap);
            if (passes >= h->opt.max_passes)
                return fail(VT_ERR_TIMEOUT, "frame did not finish in %d passes (max_passes)", passes);
            auto ts = std::chrono::steady_clock::now();
            if ((st = h->cache->service(h->d_req, nReq, s, &h2d)) != VT_OK) return st;
            stall += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
            a.ctl.in = h->d_susp[cur]; a.ctl.n_in = nOut; a.ctl.pool_in = h->d_pool[cur];
            cur ^= 1;
            a.ctl.out = h->d_susp[cur]; a.ctl.pool_out = h->d_pool[cur];
            a.br.pass = h->cache->next_pass();
            CK(cudaMemsetAsync(&h->d_ctl->n_out, 0, offsetof(CtlBlock, pool_used) + 8 - offsetof(CtlBlock, n_out), s));
            if ((st = ensure_events(h, passes)) != VT_OK) return st;
            CK(cudaEventRecord(h->ev[2 * passes], s));
            int nk = 1;
            CK(launch_pass(h, a, slabMode, s, &nk));
            CK(cudaEventRecord(h->ev[2 * passes + 1], s));
            h->stats.launches += nk;
            passes++;
            if ((st = h->cache->spec_work(h->ev[2 * passes - 1], nullptr)) != VT_OK) return st;
        }
    }
    if ((st = collect_counters(h, s)) != VT_OK) return st;
    if (!staged.empty()) {
        auto tp = std::chrono::steady_clock::now();
        int64_t got = 0;
        if ((st = h->cache->prefetch_commit(staged, stagedSlots, s, &got)) != VT_OK) return st;
        CK(cudaStreamSynchronize(s));
        h->stats.ms_prefetch_last_frame =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count();
    } else {
        h->stats.ms_prefetch_last_frame = 0;
    }
    double tk = 0;
    for (int k = 0; k < passes; k++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, h->ev[2 * k], h->ev[2 * k + 1]));
        tk += ms;
    }
    h->stats.ms_trace_last_frame = tk;
    h->stats.frames++;
    h->stats.passes = passes;
    h->stats.ms_stall_last_frame = stall;
    h->stats.ms_wait_last_frame = wait;
    h->stats.bytes_h2d_last_frame = h2d;
    if (h->cache) h->cache->fold_stats(h->stats);
    h->stats.ms_last_frame = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    h->lastValid = n == 1;
    return VT_OK;
}

extern "C" vt_status vt_render(vt_handle* h, float* dev_rgba, uint8_t* dev_rgb8, void* stream) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    ViewReq v = {h->cam, dev_rgba ? (float4*)dev_rgba : (dev_rgb8 ? nullptr : h->d_rgba), dev_rgb8};
    return render_views(h, &v, 1, (cudaStream_t)stream);
}

extern "C" vt_status vt_render_host(vt_handle* h, float* host_rgba, uint8_t* host_rgb8) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    ViewReq v = {h->cam, host_rgba ? h->d_rgba : nullptr, host_rgb8 ? h->d_rgb8 : nullptr};
    if (!v.rgba && !v.rgb8) v.rgba = h->d_rgba;
    vt_status s = render_views(h, &v, 1, h->s_int);
    if (s != VT_OK) return s;
    size_t n = (size_t)h->nRays;
    if (host_rgba) CK(cudaMemcpyAsync(host_rgba, h->d_rgba, n * 16, cudaMemcpyDeviceToHost, h->s_int));
    if (host_rgb8) CK(cudaMemcpyAsync(host_rgb8, h->d_rgb8, n * 3, cudaMemcpyDeviceToHost, h->s_int));
    CK(cudaStreamSynchronize(h->s_int));
    return VT_OK;
}

extern "C" vt_status vt_render_batch(vt_handle* h, const vt_view* views, int n, void* stream) {
    clear_error();
    if (!h || !views || n < 1) return fail(VT_ERR_INVALID, "vt_render_batch: bad arguments");
    std::vector<ViewReq> vr(n);
    for (int k = 0; k < n; k++) {
        if (!views[k].dev_rgba && !views[k].dev_rgb8) return fail(VT_ERR_INVALID, "view %d has no output buffer", k);
        vr[k].cam = views[k].cam; vr[k].rgba = (float4*)views[k].dev_rgba; vr[k].rgb8 = views[k].dev_rgb8;
    }
    return render_views(h, vr.data(), n, (cudaStream_t)stream);
}

extern "C" vt_status vt_debug_hits(vt_handle* h, uint64_t* node, uint64_t* brick, float* t, float* n) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    if (!h->opt.record_hits) return fail(VT_ERR_STATE, "record_hits is off");
    if (!h->lastValid) return fail(VT_ERR_STATE, "no single-view frame rendered since the last change");
    size_t N = (size_t)h->nRays;
    CK(cudaDeviceSynchronize());
    if (node) CK(cudaMemcpy(node, h->d_node, N * 8, cudaMemcpyDeviceToHost));
    if (brick) CK(cudaMemcpy(brick, h->d_brick, N * 8, cudaMemcpyDeviceToHost));
    if (t) CK(cudaMemcpy(t, h->d_t, N * 4, cudaMemcpyDeviceToHost));
    if (n) CK(cudaMemcpy(n, h->d_n, N * 12, cudaMemcpyDeviceToHost));
    return VT_OK;
}

extern "C" vt_status vt_get_trace(vt_handle* h, uint32_t* bits, int64_t nwords) {
    clear_error();
    if (!h || !bits) return fail(VT_ERR_INVALID, "null argument");
    if (!h->d_touched) return fail(VT_ERR_STATE, "record_trace is off");
    if ((size_t)nwords < h->touchedWords) return fail(VT_ERR_INVALID, "need %zu words", h->touchedWords);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(bits, h->d_touched, h->touchedWords * 4, cudaMemcpyDeviceToHost));
    return VT_OK;
}

extern "C" vt_status vt_prefetch(vt_handle* h, const uint64_t* bricks, int64_t n, int64_t* loaded, void* stream) {
    clear_error();
    if (!h || (!bricks && n > 0)) return fail(VT_ERR_INVALID, "null argument");
    if (loaded) *loaded = 0;
    if (h->opt.resident || n <= 0) return VT_OK;
    uint64_t lo = 1ull << (3 * h->Lc), hi = lo << 3;
    std::vector<uint64_t> b;
    b.reserve((size_t)n);
    for (int64_t i = 0; i < n; i++) {
        if (bricks[i] < lo || bricks[i] >= hi) return fail(VT_ERR_INVALID, "brick code %llu not at levelCubes", (unsigned long long)bricks[i]);
        b.push_back(code_to_page(bricks[i], h->Lc));
    }
    int64_t got = 0;
    vt_status s = h->cache->prefetch(b, stream ? (cudaStream_t)stream : h->s_int, &got);
    if (loaded) *loaded = got;
    h->cache->fold_stats(h->stats);
    return s;
}

extern "C" vt_status vt_set_tuning(vt_handle* h, const vt_tuning* t) {
    clear_error();
    if (!h || !t) return fail(VT_ERR_INVALID, "null argument");
    vt_options o = h->opt;
    o.tile_w = t->tile_w; o.tile_h = t->tile_h; o.unroll = t->unroll; o.persistent = t->persistent;
    o.pops = t->pops; o.blocks_per_sm = t->blocks_per_sm; o.lookahead = t->lookahead; o.use_graph = t->use_graph;
    o.skip = t->skip;
    o.spec_async = t->spec_async;
    o.wavefront = t->wavefront;
    o.shared_aprons = t->shared_aprons;
    o.demand_batch = t->demand_batch;
    vt_status s = validate(&h->p, h->oct, &o);
    if (s != VT_OK) return s;
    if (o.lookahead < 0 || o.lookahead > 64 || o.pops < 1 || o.blocks_per_sm < 1 || o.blocks_per_sm > 32)
        return fail(VT_ERR_INVALID, "lookahead 0..64, pops >= 1, blocks_per_sm 1..32");
    h->opt = o;
    if (h->cache) {
        h->cache->set_async_spec(o.spec_async != 0);
        h->cache->set_shared_aprons(o.shared_aprons != 0);
        h->cache->set_demand_batch(o.demand_batch);
    }
    return VT_OK;
}

extern "C" vt_status vt_get_tuning(vt_handle* h, vt_tuning* t) {
    clear_error();
    if (!h || !t) return fail(VT_ERR_INVALID, "null argument");
    t->tile_w = h->opt.tile_w; t->tile_h = h->opt.tile_h; t->unroll = h->opt.unroll; t->persistent = h->opt.persistent;
    t->pops = h->opt.pops; t->blocks_per_sm = h->opt.blocks_per_sm; t->lookahead = h->opt.lookahead;
    t->use_graph = h->opt.use_graph;
    t->skip = h->opt.skip;
    t->spec_async = h->opt.spec_async;
    t->wavefront = h->opt.wavefront;
    t->shared_aprons = h->opt.shared_aprons;
    t->demand_batch = h->opt.demand_batch;
    return VT_OK;
}

extern "C" vt_status vt_prefetch_hint(vt_handle* h, const uint64_t* bricks, int64_t n) {
    clear_error();
    if (!h || (!bricks && n > 0)) return fail(VT_ERR_INVALID, "null argument");
    uint64_t lo = 1ull << (3 * h->Lc), hi = lo << 3;
    h->hint.clear();
    for (int64_t i = 0; i < n; i++) {
        if (bricks[i] < lo || bricks[i] >= hi) return fail(VT_ERR_INVALID, "brick code %llu not at levelCubes", (unsigned long long)bricks[i]);
        h->hint.push_back(code_to_page(bricks[i], h->Lc));
    }
    return VT_OK;
}

extern "C" vt_status vt_prefetch_predict(vt_handle* h, vt_mlp* m, const vt_camera* cams, int n, float vol_edge,
                                         float fov_deg, float threshold, void* stream) {
    clear_error();
    if (!h || !m || !cams || n < 1 || vol_edge <= 0) return fail(VT_ERR_INVALID, "vt_prefetch_predict: bad arguments");
    if (h->opt.resident || !h->cache) return VT_OK;
    int d[4];
    vt_status st = vt_mlp_info(m, d);
    if (st != VT_OK) return st;
    int level = 0;
    while (level < 10 && (1 << (3 * level)) < d[3]) level++;
    if (d[0] != 12 || (1 << (3 * level)) != d[3] || level > h->Lc)
        return fail(VT_ERR_INVALID, "the network must map 12 pose features to 8^level outputs, level <= levelCubes (%d)",
                    h->Lc);
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->d_leafPages) {
        std::vector<unsigned int> pages(h->leafBricks.size());
        for (size_t i = 0; i < pages.size(); i++) pages[i] = (unsigned int)code_to_page(h->leafBricks[i], h->Lc);
        h->nLeaf = (int)pages.size();
        CK(cudaMalloc(&h->d_leafPages, std::max<size_t>(1, pages.size()) * 4));
        CK(cudaMemcpy(h->d_leafPages, pages.data(), pages.size() * 4, cudaMemcpyHostToDevice));
        CK(cudaMalloc(&h->d_pred, ((size_t)h->nLeaf + 1) * 4));
        CK(cudaHostAlloc(&h->h_pred, ((size_t)h->nLeaf + 1) * 4, cudaHostAllocDefault));
        CK(cudaEventCreateWithFlags(&h->predDone, cudaEventDisableTiming));
    }
    if (h->predPending) CK(cudaEventSynchronize(h->predDone));   /* its buffers are reused */
    if (n > h->predCap) {
        cudaFree(h->d_feat);
        if (h->h_feat) cudaFreeHost(h->h_feat);
        h->d_feat = nullptr; h->h_feat = nullptr;
        CK(cudaMalloc(&h->d_feat, (size_t)n * 12 * 4));
        CK(cudaHostAlloc(&h->h_feat, (size_t)n * 12 * 4, cudaHostAllocDefault));
        h->predCap = n;
    }
    if ((long long)n * d[3] > h->probsCap) {
        cudaFree(h->d_probs);
        h->d_probs = nullptr;
        CK(cudaMalloc(&h->d_probs, (size_t)n * d[3] * 4));
        h->probsCap = n * d[3];
    }
    /* pose features, as the network was trained on them */
    const double c = (vol_edge - 1.0) / 2.0, rad = std::sqrt(3.0) * vol_edge / 2.0;
    for (int k = 0; k < n; k++) {
        float* f = h->h_feat + 12 * k;
        const vt_camera& cm = cams[k];
        double dd = 0;
        for (int a = 0; a < 3; a++) {
            const double r = (double)cm.position[a] - c;
            f[a] = (float)(r / vol_edge);
            dd += r * r;
            f[3 + a] = cm.look[a];
            f[6 + a] = cm.up[a];
        }
        dd = std::sqrt(dd);
        f[9] = (float)(fov_deg / 90.0);
        f[10] = (float)(std::max(dd - rad, 0.0) / vol_edge);
        f[11] = (float)((dd + rad) / vol_edge);
    }
    CK(cudaMemcpyAsync(h->d_feat, h->h_feat, (size_t)n * 12 * 4, cudaMemcpyHostToDevice, s));
    if ((st = vt_mlp_forward(m, h->d_feat, n, h->d_probs, stream)) != VT_OK) return st;
    CK(cudaMemsetAsync(h->d_pred, 0, 4, s));
    DevBricks b;
    h->cache->fill_args(b);
    CK(vt_launch_predict_requests(b.page, h->d_leafPages, h->nLeaf, h->d_probs, n, level, h->Lc, threshold,
                                  h->d_pred + 1, h->d_pred, (unsigned int)h->nLeaf, s));
    h->stats.launches++;
    CK(cudaMemcpyAsync(h->h_pred, h->d_pred, ((size_t)h->nLeaf + 1) * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(h->predDone, s));
    h->predPending = true;
    return VT_OK;
}

extern "C" vt_status vt_brick_list(vt_handle* h, uint64_t* bricks, int64_t* n) {
    clear_error();
    if (!h || !n) return fail(VT_ERR_INVALID, "null argument");
    int64_t cap = *n;
    *n = (int64_t)h->leafBricks.size();
    if (bricks) memcpy(bricks, h->leafBricks.data(), (size_t)std::min<int64_t>(cap, *n) * 8);
    return VT_OK;
}

extern "C" vt_status vt_debug_slot(vt_handle* h, uint64_t code, void* host_out, int* resident) {
    clear_error();
    if (!h || !host_out || !resident) return fail(VT_ERR_INVALID, "null argument");
    *resident = 0;
    if (!h->cache) return VT_OK;
    return h->cache->copy_slot(code_to_page(code, h->Lc), host_out, resident);
}

extern "C" vt_status vt_drop_cache(vt_handle* h) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    h->hint.clear();
    if (h->predPending) { cudaEventSynchronize(h->predDone); h->predPending = false; }
    if (!h->cache) return VT_OK;
    return h->cache->drop();
}

extern "C" vt_status vt_get_stats(vt_handle* h, vt_stats* s) {
    clear_error();
    if (!h || !s) return fail(VT_ERR_INVALID, "null argument");
    *s = h->stats;
    return VT_OK;
}
extern "C" vt_status vt_reset_stats(vt_handle* h) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    memset(&h->stats, 0, sizeof(h->stats));
    if (h->cache) h->cache->reset_stats();
    return VT_OK;
}
