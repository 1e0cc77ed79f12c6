/*
 * runtime.cpp -- the renderer handle of libvt.so: camera state (class
 * Camera/Screen), octree flattening and upload (class Octree), brick
 * residency (class lruCache) and the frame loop (visualTur::
 * updateVisibleCubes, src/visualTur.cu:167-228), behind the C ABI.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include <cuda_runtime.h>

#include "vt_kernels.h"
#include "vt_runtime.h"
#include "cache.h"

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
struct vt_handle {
    vt_params p;
    vt_options opt;
    std::string volPath, dsName, octPath;
    vt_volume* vol = nullptr; bool ownVol = false;
    vt_octree* oct = nullptr; bool ownOct = false;
    vt_camera cam;
    float fovH = 0, fovW = 0;
    int nLevels = 0, Lo = 0, Lc = 0, inc = 3, edge = 0, D = 0;
    /* flattened octree */
    std::vector<uint2*> d_nodes;
    int rootValid = 0;
    std::vector<uint64_t> leafBricks;   /* bricks holding reachable candidate nodes */
    /* dense residency */
    void* d_vol = nullptr; int P = 4; long long ve = 0;
    /* brick cache */
    vtrt::BrickCache* cache = nullptr;
    /* per-ray buffers */
    int nRays = 0;
    float4* d_rgba = nullptr; uint8_t* d_rgb8 = nullptr;
    unsigned long long* d_node = nullptr; unsigned long long* d_brick = nullptr; float* d_t = nullptr; float* d_n = nullptr;
    /* control */
    unsigned long long* d_counters = nullptr;
    unsigned int* d_err = nullptr;
    unsigned int* d_nout = nullptr;       /* [0] n_out, [1] n_req */
    unsigned long long* h_counters = nullptr;   /* pinned */
    unsigned int* h_small = nullptr;             /* pinned: err, n_out, n_req */
    /* suspended-ray ping-pong buffers */
    unsigned int susp_cap = 0;
    unsigned int* d_susp[2] = {nullptr, nullptr};
    unsigned long long* d_stk[2] = {nullptr, nullptr};
    unsigned char* d_top[2] = {nullptr, nullptr};
    unsigned long long* d_req = nullptr; unsigned int req_cap = 0;
    std::vector<cudaEvent_t> ev;          /* start/stop pairs around trace launches */
    vt_stats stats;
    bool lastValid = false;
};

static void free_ray_buffers(vt_handle* h) {
    cudaFree(h->d_rgba); cudaFree(h->d_rgb8); cudaFree(h->d_node); cudaFree(h->d_brick); cudaFree(h->d_t); cudaFree(h->d_n);
    h->d_rgba = nullptr; h->d_rgb8 = nullptr; h->d_node = nullptr; h->d_brick = nullptr; h->d_t = nullptr; h->d_n = nullptr;
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_susp[i]); cudaFree(h->d_stk[i]); cudaFree(h->d_top[i]);
        h->d_susp[i] = nullptr; h->d_stk[i] = nullptr; h->d_top[i] = nullptr;
    }
    h->susp_cap = 0;
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

static vt_status ensure_suspend_buffers(vt_handle* h, unsigned int cap) {
    if (h->susp_cap >= cap) return VT_OK;
    for (int i = 0; i < 2; i++) {
        cudaFree(h->d_susp[i]); cudaFree(h->d_stk[i]); cudaFree(h->d_top[i]);
        CK(cudaMalloc(&h->d_susp[i], (size_t)cap * 4));
        CK(cudaMalloc(&h->d_stk[i], (size_t)cap * VT_STACK * 8));
        CK(cudaMalloc(&h->d_top[i], (size_t)cap));
    }
    h->susp_cap = cap;
    return VT_OK;
}

/* Octree flattening: keeps the nodes reachable from the root through the
 * reference's traversal (src/Octree.cu:620-739) and records, per node, the
 * children its range search accepts -- a property of the node alone. */
static vt_status flatten_octree(vt_handle* h) {
    const vt_octree* o = h->oct;
    const int Lo = h->Lo;
    const std::vector<uint64_t>& l0 = o->levels[0];
    h->rootValid = (l0.size() >= 2 && (l0[0] == 1 || l0[1] == 1 || (l0[0] < 1 && l0[1] > 1))) ? 1 : 0;
    std::vector<uint64_t> codes(1, 1ull), next;
    h->d_nodes.assign(Lo, nullptr);
    const int codeBits = 3 * Lo + 1;
    for (int l = 0; l < Lo; l++) {
        const std::vector<uint64_t>& e = o->levels[l + 1];
        std::vector<uint2> rec(codes.size());
        std::vector<int> mask(codes.size());
#pragma omp parallel for schedule(dynamic, 4096)
        for (long long i = 0; i < (long long)codes.size(); i++)
            mask[i] = children_mask(e.data(), (int)e.size(), codes[i]);
        next.clear();
        uint64_t base = 0;
        for (size_t i = 0; i < codes.size(); i++) {
            rec[i].x = (unsigned int)base;
            rec[i].y = (unsigned int)mask[i];
            for (int k = 0; k < 8; k++)
                if ((mask[i] >> k) & 1) next.push_back((codes[i] << 3) + (uint64_t)k);
            base += __builtin_popcount(mask[i]);
        }
        if (l + 1 < Lo && next.size() >= (1ull << (64 - codeBits)))
            return fail(VT_ERR_UNSUPPORTED, "level %d has %zu nodes, more than the stack entry encodes", l + 1, next.size());
        if (next.size() > 0xFFFFFFFFull) return fail(VT_ERR_UNSUPPORTED, "level %d too large", l + 1);
        CK(cudaMalloc(&h->d_nodes[l], std::max<size_t>(rec.size(), 1) * sizeof(uint2)));
        CK(cudaMemcpy(h->d_nodes[l], rec.data(), rec.size() * sizeof(uint2), cudaMemcpyHostToDevice));
        codes.swap(next);
    }
    /* bricks that hold reachable candidates */
    const int shift = 3 * (Lo - h->Lc);
    h->leafBricks.clear();
    for (size_t i = 0; i < codes.size(); i++) {
        uint64_t b = codes[i] >> shift;
        if (h->leafBricks.empty() || h->leafBricks.back() != b) h->leafBricks.push_back(b);
    }
    return VT_OK;
}

static vt_status upload_dense(vt_handle* h) {
    const vt_volume* v = h->vol;
    h->ve = (long long)(1 << h->nLevels) + 2 * h->P;
    for (int a = 0; a < 3; a++)
        if (v->dims[a] > (1 << h->nLevels)) return fail(VT_ERR_INVALID, "volume larger than the octree");
    size_t es = v->esize();
    size_t bytes = (size_t)h->ve * h->ve * h->ve * es;
    CK(cudaMalloc(&h->d_vol, bytes));
    CK(cudaMemset(h->d_vol, 0, bytes));
    /* stream the volume through a pinned staging buffer, x-slab by x-slab */
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
}

static vt_status validate(const vt_params* p, const vt_octree* o) {
    if (p->W <= 0 || p->H <= 0) return fail(VT_ERR_INVALID, "screen size must be positive");
    if (p->numRayPx != 1) return fail(VT_ERR_UNSUPPORTED, "numRayPx must be 1 (the reference generates W*H rays only)");
    if (p->octreeLevel < 1 || p->octreeLevel > o->nLevels) return fail(VT_ERR_INVALID, "octreeLevel %d outside 1..%d", p->octreeLevel, o->nLevels);
    if (p->levelCubes < 0 || p->levelCubes > p->octreeLevel) return fail(VT_ERR_INVALID, "levelCubes must be in 0..octreeLevel");
    if (p->levelCubes > 9) return fail(VT_ERR_UNSUPPORTED, "levelCubes > 9: brick table too large");
    int b = 1 << (o->nLevels - p->levelCubes);
    if (p->dimCubeCache[0] != b || p->dimCubeCache[1] != b || p->dimCubeCache[2] != b)
        return fail(VT_ERR_INVALID, "dimCubeCache must be %d^3 for levelCubes %d of a %d-level octree", b, p->levelCubes, o->nLevels);
    if (p->cubeInc < 3) return fail(VT_ERR_INVALID, "cubeInc must be >= 3 so every trilinear and normal tap stays in the brick");
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
    CK(cudaMalloc(&h->d_counters, VT_C_COUNT * 8));
    CK(cudaMalloc(&h->d_err, 4));
    CK(cudaMalloc(&h->d_nout, 8));
    CK(cudaHostAlloc(&h->h_counters, VT_C_COUNT * 8, cudaHostAllocDefault));
    CK(cudaHostAlloc(&h->h_small, 16, cudaHostAllocDefault));
    if (h->opt.resident) {
        if ((s = upload_dense(h)) != VT_OK) return s;
    } else {
        vtrt::CacheConfig cc;
        cc.vol = h->vol; cc.nLevels = h->nLevels; cc.Lc = h->Lc; cc.inc = h->inc; cc.edge = h->edge;
        cc.deviceSlots = p.maxElementsCache; cc.hostSlots = p.maxElementsCache_CPU;
        cc.hostThreads = h->opt.host_threads;
        h->cache = new vtrt::BrickCache();
        if ((s = h->cache->init(cc)) != VT_OK) return s;
        /* preload when every needed brick fits */
        if ((size_t)p.maxElementsCache >= h->leafBricks.size()) {
            if ((s = h->cache->preload(h->leafBricks)) != VT_OK) return s;
        }
        h->req_cap = (unsigned int)std::max<size_t>(h->leafBricks.size(), 1);
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
    vt_status s = validate(p, o);
    if (s != VT_OK) return s;
    vt_handle* h = new vt_handle();
    h->p = *p;
    if (opt) h->opt = *opt; else vt_default_options(&h->opt);
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
    free_ray_buffers(h);
    for (uint2* p : h->d_nodes) cudaFree(p);
    cudaFree(h->d_vol); cudaFree(h->d_counters); cudaFree(h->d_err); cudaFree(h->d_nout); cudaFree(h->d_req);
    if (h->h_counters) cudaFreeHost(h->h_counters);
    if (h->h_small) cudaFreeHost(h->h_small);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
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
    h->p.maxElementsCache = nE; h->p.cubeInc = cInc; h->inc = cInc; h->D = h->edge + 2 * cInc;
    delete h->cache;
    vtrt::CacheConfig cc;
    cc.vol = h->vol; cc.nLevels = h->nLevels; cc.Lc = h->Lc; cc.inc = h->inc; cc.edge = h->edge;
    cc.deviceSlots = nE; cc.hostSlots = h->p.maxElementsCache_CPU; cc.hostThreads = h->opt.host_threads;
    h->cache = new vtrt::BrickCache();
    if ((s = h->cache->init(cc)) != VT_OK) return s;
    if ((size_t)nE >= h->leafBricks.size() && (s = h->cache->preload(h->leafBricks)) != VT_OK) return s;
    h->lastValid = false;
    return VT_OK;
}

/* ---- frame ---------------------------------------------------------------- */
static void fill_args(vt_handle* h, TraceArgs& a, float4* rgba, uint8_t* rgb8) {
    memset(&a, 0, sizeof(a));
    a.cam = dev_camera(h->cam);
    a.oct.nLevels = h->nLevels; a.oct.Lo = h->Lo; a.oct.Lc = h->Lc; a.oct.rootValid = h->rootValid;
    for (int l = 0; l < h->Lo; l++) a.oct.nodes[l] = h->d_nodes[l];
    a.br.vtype = h->vol->vtype; a.br.inc = h->inc;
    if (h->opt.resident) {
        a.br.vol = h->d_vol; a.br.P = h->P; a.br.ve = (int)h->ve;
        a.br.vsx = h->ve * h->ve; a.br.vsy = h->ve;
    } else {
        h->cache->fill_args(a.br);
    }
    a.out.rgba = rgba; a.out.rgb8 = rgb8;
    a.out.node = h->d_node; a.out.brick = h->d_brick; a.out.t = h->d_t; a.out.n = h->d_n;
    a.ctl.counters = h->d_counters; a.ctl.err = h->d_err;
    a.ctl.n_out = h->d_nout; a.ctl.n_req = h->d_nout + 1;
    a.ctl.req = h->d_req; a.ctl.req_cap = h->req_cap;
    a.ctl.lookahead = h->opt.lookahead;
    a.iso = h->oct->iso;
    a.light = make_float3(0.0f, 512.0f, 0.0f);   /* src/visualTur.cu:30 */
    a.tile_w = h->opt.tile_w; a.tile_h = h->opt.tile_h;
}

static vt_status collect_counters(vt_handle* h, cudaStream_t s) {
    CK(cudaMemcpyAsync(h->h_counters, h->d_counters, VT_C_COUNT * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->h_small, h->d_err, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const unsigned long long* c = h->h_counters;
    vt_stats& st = h->stats;
    st.rays += c[VT_C_RAYS]; st.hits += c[VT_C_HITS]; st.samples += c[VT_C_SAMPLES];
    st.normal_samples += c[VT_C_NSAMPLES]; st.candidates += c[VT_C_CANDIDATES]; st.expansions += c[VT_C_EXPANSIONS];
    st.device_hits += c[VT_C_DEVHITS]; st.device_misses += c[VT_C_DEVMISSES];
    st.max_stack = std::max<int64_t>(st.max_stack, (int64_t)c[VT_C_MAXSTACK]);
    unsigned int err = h->h_small[0];
    if (err & VT_KERR_STACK) return fail(VT_ERR_STACK, "a ray's traversal stack overflowed (%d entries)", VT_STACK);
    if (err & VT_KERR_NOTRESIDENT) return fail(VT_ERR_STATE, "resident render met a brick with no slot");
    if (err & (VT_KERR_SUSPEND_FULL | VT_KERR_REQUEST_FULL)) return fail(VT_ERR_STATE, "demand-paging queue overflow (%u)", err);
    return VT_OK;
}

/* records the launch of pass `k` between events 2k and 2k+1 */
static vt_status timed_trace(vt_handle* h, const TraceArgs& a, bool slabMode, cudaStream_t s, int k) {
    while ((int)h->ev.size() < 2 * (k + 1)) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        h->ev.push_back(e);
    }
    CK(cudaEventRecord(h->ev[2 * k], s));
    CK(vt_launch_trace(a, slabMode, s));
    CK(cudaEventRecord(h->ev[2 * k + 1], s));
    h->stats.launches++;
    return VT_OK;
}

static vt_status render_frame(vt_handle* h, float4* rgba, uint8_t* rgb8, cudaStream_t s) {
    auto t0 = std::chrono::steady_clock::now();
    TraceArgs a;
    fill_args(h, a, rgba, rgb8);
    CK(cudaMemsetAsync(h->d_counters, 0, VT_C_COUNT * 8, s));
    CK(cudaMemsetAsync(h->d_err, 0, 4, s));
    CK(cudaMemsetAsync(h->d_nout, 0, 8, s));
    const bool slabMode = !h->opt.resident;
    const bool allResident = h->opt.resident || h->cache->all_resident();
    if (!allResident) {
        vt_status st = ensure_suspend_buffers(h, (unsigned int)h->nRays);
        if (st != VT_OK) return st;
    }
    if (slabMode) h->cache->begin_frame();
    a.ctl.susp_cap = h->susp_cap;
    a.ctl.susp_out = h->d_susp[0]; a.ctl.stk_out = h->d_stk[0]; a.ctl.top_out = h->d_top[0];
    if (slabMode) a.br.pass = h->cache->next_pass();
    vt_status st0 = timed_trace(h, a, slabMode, s, 0);
    if (st0 != VT_OK) return st0;
    int passes = 1;
    double stall = 0, h2d = 0;
    vt_status st;
    if (!allResident) {
        int cur = 0;
        for (;;) {
            CK(cudaMemcpyAsync(h->h_small, h->d_nout, 8, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            unsigned int nOut = h->h_small[0], nReq = h->h_small[1];
            if (nOut == 0) break;
            if (passes >= h->opt.max_passes) return fail(VT_ERR_TIMEOUT, "frame did not finish in %d passes", passes);
            auto ts = std::chrono::steady_clock::now();
            if ((st = h->cache->service(h->d_req, nReq, s, &h2d)) != VT_OK) return st;
            stall += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
            /* resume the suspended rays */
            a.ctl.susp_in = h->d_susp[cur]; a.ctl.n_in = nOut;
            a.ctl.stk_in = h->d_stk[cur]; a.ctl.top_in = h->d_top[cur];
            cur ^= 1;
            a.ctl.susp_out = h->d_susp[cur]; a.ctl.stk_out = h->d_stk[cur]; a.ctl.top_out = h->d_top[cur];
            a.br.pass = h->cache->next_pass();
            CK(cudaMemsetAsync(h->d_nout, 0, 8, s));
            if ((st = timed_trace(h, a, slabMode, s, passes)) != VT_OK) return st;
            passes++;
        }
    }
    if ((st = collect_counters(h, s)) != VT_OK) return st;
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
    h->stats.bytes_h2d_last_frame = h2d;
    if (h->cache) h->cache->fold_stats(h->stats);
    h->stats.ms_last_frame = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    h->lastValid = true;
    return VT_OK;
}

extern "C" vt_status vt_render(vt_handle* h, float* dev_rgba, uint8_t* dev_rgb8, void* stream) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    if (!dev_rgba && !dev_rgb8) { dev_rgba = (float*)h->d_rgba; }
    return render_frame(h, (float4*)dev_rgba, dev_rgb8, (cudaStream_t)stream);
}

extern "C" vt_status vt_render_host(vt_handle* h, float* host_rgba, uint8_t* host_rgb8) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    vt_status s = render_frame(h, h->d_rgba, host_rgb8 ? h->d_rgb8 : nullptr, 0);
    if (s != VT_OK) return s;
    size_t n = (size_t)h->nRays;
    if (host_rgba) CK(cudaMemcpy(host_rgba, h->d_rgba, n * 16, cudaMemcpyDeviceToHost));
    if (host_rgb8) CK(cudaMemcpy(host_rgb8, h->d_rgb8, n * 3, cudaMemcpyDeviceToHost));
    return VT_OK;
}

extern "C" vt_status vt_debug_hits(vt_handle* h, uint64_t* node, uint64_t* brick, float* t, float* n) {
    clear_error();
    if (!h) return fail(VT_ERR_INVALID, "null handle");
    if (!h->opt.record_hits) return fail(VT_ERR_STATE, "record_hits is off");
    if (!h->lastValid) return fail(VT_ERR_STATE, "no frame rendered since the last change");
    size_t N = (size_t)h->nRays;
    CK(cudaDeviceSynchronize());
    if (node) CK(cudaMemcpy(node, h->d_node, N * 8, cudaMemcpyDeviceToHost));
    if (brick) CK(cudaMemcpy(brick, h->d_brick, N * 8, cudaMemcpyDeviceToHost));
    if (t) CK(cudaMemcpy(t, h->d_t, N * 4, cudaMemcpyDeviceToHost));
    if (n) CK(cudaMemcpy(n, h->d_n, N * 12, cudaMemcpyDeviceToHost));
    return VT_OK;
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

extern "C" vt_status vt_render_batch(vt_handle* h, const vt_view* views, int n, void* stream) {
    clear_error();
    if (!h || (!views && n > 0)) return fail(VT_ERR_INVALID, "null argument");
    return fail(VT_ERR_UNSUPPORTED, "vt_render_batch is not built yet");
}
