/*
 * vt_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY, never the product).
 *
 * A literal single-precision restatement of the reference algorithm of
 * carlosduelo/visualTur for the isosurface ray-casting path.  Built with
 * -ffp-contract=off so every float operation rounds exactly once, in the
 * order the reference source writes it.  The reference's own device code is
 * compiled separately (oracle/ref_build.sh) to pin this file; see the header.
 */
#include "vt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <fstream>
#include <map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* ---- float3 helpers with the semantics the reference relies on ---------- */
struct V3 { float x, y, z; };
struct I3 { int x, y, z; };
static inline V3 mk(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(float s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* normalize(v) = v * rsqrtf(dot(v,v)); host rsqrtf(x) = 1/sqrtf(x). */
static inline V3 normalize(V3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
static inline V3 fromf3(orc_f3 a) { return mk(a.x, a.y, a.z); }
static inline orc_f3 tof3(V3 a) { orc_f3 r = {a.x, a.y, a.z}; return r; }

/* ---- Morton utilities: inc/mortonCodeUtil.hpp --------------------------- */
/* dilateInteger (:31-40): bit b of x moves to bit 3b (21-bit inputs). */
static inline uint64_t dilate(uint64_t x) {
    uint64_t r = 0;
    for (int b = 0; b < 21; b++) r |= ((x >> b) & 1ull) << (3 * b);
    return r;
}
/* getIndexLevel (:42-86). */
static inline int index_level(uint64_t index) {
    if (index == 1) return 0;
    if (index < 8) return -1;
    int l = 0;
    while (l < 19 && (index >> (3 * (l + 1))) != 0) l++;
    return l;
}
/* getMinBoxIndex2 (:120-144). */
static inline I3 min_box(uint64_t index, int level, int nLevels) {
    I3 m = {0, 0, 0};
    if (index == 1) return m;
    for (int l = level; l > 0; l--) {
        m.z += (int)((index & 1ull) << (nLevels - l)); index >>= 1;
        m.y += (int)((index & 1ull) << (nLevels - l)); index >>= 1;
        m.x += (int)((index & 1ull) << (nLevels - l)); index >>= 1;
    }
    return m;
}
/* coordinateToIndex (:146-169). */
static inline uint64_t coord_to_index(int x, int y, int z, int level, int nLevels) {
    if (level == 0) return 1;
    uint64_t code = 1ull << (nLevels * 3);
    code |= dilate((uint64_t)x) << 2;
    code |= dilate((uint64_t)y) << 1;
    code |= dilate((uint64_t)z);
    code >>= (nLevels - level) * 3;
    return code;
}
/* updateCoordinates (:172-202). */
static inline I3 update_coordinates(int maxLevel, int cLevel, uint64_t cIndex, int nLevel,
                                    uint64_t nIndex, I3 m) {
    if (nIndex == 0) { I3 z = {0, 0, 0}; return z; }
    if (cLevel < nLevel) {
        m.z += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
        m.y += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
        m.x += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
        return m;
    } else if (cLevel > nLevel) {
        return min_box(nIndex, nLevel, maxLevel);
    }
    m.z += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
    m.y += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
    m.x += (int)((nIndex & 1ull) << (maxLevel - nLevel)); nIndex >>= 1;
    m.z -= (int)((cIndex & 1ull) << (maxLevel - cLevel)); cIndex >>= 1;
    m.y -= (int)((cIndex & 1ull) << (maxLevel - cLevel)); cIndex >>= 1;
    m.x -= (int)((cIndex & 1ull) << (maxLevel - cLevel)); cIndex >>= 1;
    return m;
}

/* ---- Range membership, device variant: src/Octree.cu -------------------- */
/* Reads past the end only happen in the terminating iteration of the closer
 * search, where they cannot change the returned index; they read 0 here. */
static inline uint64_t at(const uint64_t* e, int size, int i) {
    return (i >= 0 && i < size) ? e[i] : 0ull;
}
/* _cuda_checkRange (:15-20). */
static inline bool check_range(const uint64_t* e, int size, uint64_t index, int mn, int mx) {
    uint64_t a = at(e, size, mn), b = at(e, size, mx);
    return index == a || index == b || (a < index && b > index);
}
/* _cuda_binary_search_closer, active branch (:78-99). */
static int closer_dev(const uint64_t* e, int size, uint64_t index, int mn, int mx) {
    bool end = false, found = false;
    int middle = 0;
    while (!end && !found) {
        int diff = mx - mn;
        middle = mn + (diff / 2);
        if (middle % 2 == 1) middle--;
        end = diff <= 1;
        found = check_range(e, size, index, middle, middle + 1);
        if (index < at(e, size, middle)) mx = middle - 1;
        else mn = middle + 2;
    }
    return middle;
}
/* _cuda_searchSecuential (:134-142). */
static bool seq_dev(const uint64_t* e, int size, uint64_t index, int mn, int mx) {
    bool find = false;
    for (int i = mn; i < mx; i += 2)
        if (check_range(e, size, index, i, i + 1)) find = true;
    return find;
}
/* Membership part of _cuda_searchChildrenValidAndHit2 (:385-530). */
static int children_mask_dev(const uint64_t* e, int size, uint64_t father) {
    uint64_t c0 = father << 3;
    int mask = 0;
    if (size == 2) {
        for (int k = 0; k < 8; k++)
            if (check_range(e, size, c0 + k, 0, 1)) mask |= 1 << k;
        return mask;
    }
    unsigned int closer1 = (unsigned int)closer_dev(e, size, c0, 0, size - 1);
    unsigned int closer8 = (unsigned int)closer_dev(e, size, c0 + 7, (int)closer1, size - 1) + 1;
    if (closer8 >= (unsigned int)size) closer8 = (unsigned int)(size - 1);
    for (int k = 0; k < 8; k++)
        if (seq_dev(e, size, c0 + k, (int)closer1, (int)closer8)) mask |= 1 << k;
    return mask;
}

/* ---- Slab tests --------------------------------------------------------- */
/* _cuda_RayAABB2 (src/Octree.cu:258-330) and _cuda_RayAABB
 * (src/rayCaster.cu:12-79): identical arithmetic on an explicit box. */
static inline bool ray_aabb(V3 o, V3 d, float* tnear, float* tfar, I3 minB, I3 maxB) {
    bool hit = true;
    float tmin, tmax, tymin, tymax, tzmin, tzmax;
    float divx = 1 / d.x;
    if (divx >= 0) { tmin = ((float)minB.x - o.x) * divx; tmax = ((float)maxB.x - o.x) * divx; }
    else { tmin = ((float)maxB.x - o.x) * divx; tmax = ((float)minB.x - o.x) * divx; }
    float divy = 1 / d.y;
    if (divy >= 0) { tymin = ((float)minB.y - o.y) * divy; tymax = ((float)maxB.y - o.y) * divy; }
    else { tymin = ((float)maxB.y - o.y) * divy; tymax = ((float)minB.y - o.y) * divy; }
    if ((tmin > tymax) || (tymin > tmax)) hit = false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float divz = 1 / d.z;
    if (divz >= 0) { tzmin = ((float)minB.z - o.z) * divz; tzmax = ((float)maxB.z - o.z) * divz; }
    else { tzmin = ((float)maxB.z - o.z) * divz; tzmax = ((float)minB.z - o.z) * divz; }
    if ((tmin > tzmax) || (tzmin > tmax)) hit = false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    if (tmin < 0.0) *tnear = 0.0f; else *tnear = tmin;
    *tfar = tmax;
    return hit;
}
static inline bool ray_aabb_level(V3 o, V3 d, float* tn, float* tf, int nLevels, I3 mn, int level) {
    int dim = 1 << (nLevels - level);
    I3 mx = {mn.x + dim, mn.y + dim, mn.z + dim};
    return ray_aabb(o, d, tn, tf, mn, mx);
}

/* float -> int conversion as the GPU performs it (NaN -> 0, saturating);
 * the reference's conversions run on the GPU. */
static inline int f2i(float v) {
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    if (v <= -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
}
static inline int d2i(double v) {
    if (v != v) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (-2147483647 - 1);
    return (int)v;
}

/* ---- Volume access ------------------------------------------------------ */
struct Volume {
    const void* data; int vtype; int dx, dy, dz;
    inline float get(int x, int y, int z) const {   /* zero-padded, src/FileManager.cu:90-112 */
        if (x < 0 || y < 0 || z < 0 || x >= dx || y >= dy || z >= dz) return 0.0f;
        size_t i = (size_t)z + (size_t)y * dz + (size_t)x * dy * dz;
        if (vtype == ORC_U8) return (float)((const uint8_t*)data)[i];
        return ((const float*)data)[i];
    }
};

/* Brick of (cubeDim + 2*inc)^3 voxels whose element (0,0,0) is global voxel
 * `org`, read zero-padded from the volume (src/lruCache.cu:223-226).  An
 * element index outside the brick is an out-of-bounds read in the
 * reference; it is counted and reads 0. */
struct Brick {
    const Volume* v; I3 org; int D; int64_t* oob;
    inline float get(int x, int y, int z) const {
        if (x < 0 || y < 0 || z < 0 || x >= D || y >= D || z >= D) { (*oob)++; return 0.0f; }
        return v->get(org.x + x, org.y + y, org.z + z);
    }
};

/* getElementInterpolate (src/rayCaster.cu:86-106), brick-relative. */
template <class B>
static inline float interp(V3 pos, const B& data, I3 minBox) {
    float rx, ry, rz;
    float px = modff(pos.x, &rx), py = modff(pos.y, &ry), pz = modff(pos.z, &rz);
    int x0 = f2i(rx - (float)minBox.x);
    int y0 = f2i(ry - (float)minBox.y);
    int z0 = f2i(rz - (float)minBox.z);
    int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    float c00 = data.get(x0, y0, z0) * (1.0f - px) + data.get(x1, y0, z0) * px;
    float c01 = data.get(x0, y0, z1) * (1.0f - px) + data.get(x1, y0, z1) * px;
    float c10 = data.get(x0, y1, z0) * (1.0f - px) + data.get(x1, y1, z0) * px;
    float c11 = data.get(x0, y1, z1) * (1.0f - px) + data.get(x1, y1, z1) * px;
    float c0 = c00 * (1.0f - py) + c10 * py;
    float c1 = c01 * (1.0f - py) + c11 * py;
    return c0 * (1.0f - pz) + c1 * pz;
}
/* getNormal (src/rayCaster.cu:131-137). */
template <class B>
static inline V3 normal_at(V3 p, const B& d, I3 mb) {
    return normalize(mk(
        (interp(mk(p.x - 1.0f, p.y, p.z), d, mb) - interp(mk(p.x + 1.0f, p.y, p.z), d, mb)) / 2.0f,
        (interp(mk(p.x, p.y - 1.0f, p.z), d, mb) - interp(mk(p.x, p.y + 1.0f, p.z), d, mb)) / 2.0f,
        (interp(mk(p.x, p.y, p.z - 1.0f), d, mb) - interp(mk(p.x, p.y, p.z + 1.0f), d, mb)) / 2.0f));
}

/* The march loop shared by cuda_rayCaster (:166-237) and
 * cuda_rayCasterCube (:285-328); TSteps is int or float.
 *
 * refine > 0 is the renderer's bisection mode (an extension: the
 * reference's own refinement loop at :214-226 is compiled out): before the
 * linear step, the pair (previous sample, crossing sample) is halved
 * `refine` times; a midpoint whose iso - value is strictly on the same side
 * as the previous sample's replaces the previous sample, otherwise it
 * replaces the crossing sample.  Every midpoint counts as a sample. */
template <class B, class TSteps>
static inline bool march(V3 origin, V3 ray, float tnear, TSteps maxStep, const B& data, I3 minBox,
                         float iso, V3* Xhit, int64_t* nsamp, int refine = 0) {
    bool hit = false;
    V3 Xnear = origin + tnear * ray;
    V3 Xfar = Xnear, Xnew = Xnear;
    bool primera = true;
    float ant = 0.0f, sig = 0.0f;
    TSteps steps = 0;
    V3 vStep = 0.5f * ray;
    while (steps <= maxStep) {
        if (primera) {
            primera = false;
            ant = interp(Xnear, data, minBox); (*nsamp)++;
            Xfar = Xnear;
        } else {
            sig = interp(Xnear, data, minBox); (*nsamp)++;
            if ((((iso - ant) < 0.0) && ((iso - sig) < 0.0)) ||
                (((iso - ant) > 0.0) && ((iso - sig) > 0.0))) {
                ant = sig;
                Xfar = Xnear;
            } else {
                V3 lo = Xfar, hi = Xnear;
                for (int k = 0; k < refine; k++) {
                    V3 mid = (lo + hi) * 0.5f;
                    float vm = interp(mid, data, minBox); (*nsamp)++;
                    bool same = (((iso - ant) < 0.0) && ((iso - vm) < 0.0)) ||
                                (((iso - ant) > 0.0) && ((iso - vm) > 0.0));
                    if (same) { lo = mid; ant = vm; }
                    else { hi = mid; sig = vm; }
                }
                float a = (iso - ant) / (sig - ant);
                Xnew = lo * (1.0f - a) + hi * a;
                hit = true;
                steps = maxStep;
            }
        }
        Xnear = Xnear + vStep;
        steps++;
    }
    *Xhit = Xnew;
    return hit;
}

static inline uint8_t to_u8(float v) {
    float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)(c * 255.0f);
}

}  // namespace

/* ======================================================================== */
/* Camera (src/Camera.cu, src/Screen.cpp)                                   */
/* ======================================================================== */
static void screen_extent(orc_camera* c) {   /* src/Screen.cpp:18-19 */
    c->h = 2 * c->distance * tanf(c->fov_h * (M_PI / 180.0));
    c->w = 2 * c->distance * tanf(c->fov_w * (M_PI / 180.0));
}

extern "C" void orc_camera_init(orc_camera* c, int nRP, int H, int W, float d, float fh, float fw) {
    memset(c, 0, sizeof(*c));
    c->H = H; c->W = W; c->numRayPixel = nRP;
    c->distance = d; c->fov_h = fh; c->fov_w = fw;
    screen_extent(c);
    V3 look = mk(0.0f, 0.0f, -1.0f), up = mk(0.0f, 1.0f, 0.0f);   /* src/Camera.cu:17-20 */
    c->look = tof3(look); c->up = tof3(up);
    c->position = tof3(mk(0.0f, 0.0f, 0.0f));
    c->right = tof3(cross(look, up));
}
extern "C" void orc_camera_move(orc_camera* c, orc_f3 d) {          /* :85-89 */
    c->position = tof3(fromf3(c->position) + fromf3(d));
}
extern "C" void orc_camera_rotate_x(orc_camera* c, float angle) {   /* :91-106 */
    float s = sin(angle * (M_PI / 180.0)), co = cos(angle * (M_PI / 180.0));
    c->rotX += angle;
    V3 look = fromf3(c->look) * co + fromf3(c->up) * s;
    c->look = tof3(look);
    c->up = tof3((-1.0f) * cross(look, fromf3(c->right)));
}
extern "C" void orc_camera_rotate_y(orc_camera* c, float angle) {   /* :108-122 */
    float s = sin(angle * (M_PI / 180.0)), co = cos(angle * (M_PI / 180.0));
    c->rotY += angle;
    V3 look = fromf3(c->look) * co - fromf3(c->right) * s;
    c->look = tof3(look);
    c->right = tof3(cross(look, fromf3(c->up)));
}
extern "C" void orc_camera_rotate_z(orc_camera* c, float angle) {   /* :124-138 */
    float s = sin(angle * (M_PI / 180.0)), co = cos(angle * (M_PI / 180.0));
    c->rotZ += angle;
    V3 right = fromf3(c->right) * co + fromf3(c->up) * s;
    c->right = tof3(right);
    c->up = tof3((-1.0f) * cross(fromf3(c->look), right));
}
extern "C" void orc_camera_move_forward(orc_camera* c, float dist) {   /* :140-144 */
    c->position = tof3(fromf3(c->position) + fromf3(c->look) * (-dist));
}
extern "C" void orc_camera_move_upward(orc_camera* c, float dist) {    /* :146-150 (along right) */
    c->position = tof3(fromf3(c->position) + fromf3(c->right) * dist);
}
extern "C" void orc_camera_strafe_right(orc_camera* c, float dist) {   /* :152-156 (along up) */
    c->position = tof3(fromf3(c->position) + fromf3(c->up) * dist);
}
extern "C" void orc_camera_change_screen(orc_camera* c, int W, int H, float fovW, float fovH, float d) {
    c->W = W; c->H = H; c->fov_w = fovW; c->fov_h = fovH; c->distance = d;
    screen_extent(c);
}
static inline V3 ray_dir(const orc_camera* c, int id) {   /* src/Camera.cu:59-72 */
    int i = id / c->W, j = id % c->W;
    float ih = c->h / c->H, iw = c->w / c->W;
    V3 A = fromf3(c->look) * c->distance;
    A = A + fromf3(c->up) * (-(c->h / 2.0f) + (ih * ((float)i + 0.5f)));
    A = A + fromf3(c->right) * (-(c->w / 2.0f) + (iw * ((float)j + 0.5f)));
    return normalize(A);
}
extern "C" void orc_camera_rays(const orc_camera* c, orc_f3* out) {
    int n = c->W * c->H;
    for (int id = 0; id < n; id++) out[id] = tof3(ray_dir(c, id));
}

/* ======================================================================== */
/* Morton exports                                                          */
/* ======================================================================== */
extern "C" uint64_t orc_coordinate_to_index(int x, int y, int z, int level, int nLevels) {
    return coord_to_index(x, y, z, level, nLevels);
}
extern "C" int orc_index_level(uint64_t index) { return index_level(index); }
extern "C" void orc_min_box(uint64_t index, int level, int nLevels, int out[3]) {
    I3 m = min_box(index, level, nLevels);
    out[0] = m.x; out[1] = m.y; out[2] = m.z;
}

/* ======================================================================== */
/* Octree file (src/Octree.cu:769-813)                                      */
/* ======================================================================== */
struct orc_octree {
    float iso; int dimension; int realDim[3]; int nLevels;
    std::vector<std::vector<uint64_t> > levels;
};

extern "C" int orc_octree_load(const char* path, orc_octree** out) {
    std::ifstream f(path, std::ifstream::binary);
    if (!f) return -1;
    int magic = 0;
    f.read((char*)&magic, 4);
    if (!f || magic != 919278872) return -2;
    orc_octree* o = new orc_octree();
    f.read((char*)&o->iso, 4);
    f.read((char*)&o->dimension, 4);
    f.read((char*)&o->realDim[0], 4);
    f.read((char*)&o->realDim[1], 4);
    f.read((char*)&o->realDim[2], 4);
    f.read((char*)&o->nLevels, 4);
    if (!f || o->nLevels < 0 || o->nLevels > 19) { delete o; return -3; }
    o->levels.resize(o->nLevels + 1);
    for (int i = o->nLevels; i >= 0; i--) {
        int n = 0;
        f.read((char*)&n, 4);
        if (!f || n < 0) { delete o; return -4; }
        o->levels[i].resize(n);
        if (n) f.read((char*)o->levels[i].data(), (std::streamsize)n * 8);
        if (!f) { delete o; return -5; }
    }
    *out = o;
    return 0;
}
extern "C" void orc_octree_free(orc_octree* o) { delete o; }
extern "C" void orc_octree_info(const orc_octree* o, float* iso, int* dim, int rd[3], int* nl) {
    if (iso) *iso = o->iso;
    if (dim) *dim = o->dimension;
    if (rd) { rd[0] = o->realDim[0]; rd[1] = o->realDim[1]; rd[2] = o->realDim[2]; }
    if (nl) *nl = o->nLevels;
}
extern "C" int orc_octree_level_size(const orc_octree* o, int l) {
    return (l < 0 || l > o->nLevels) ? -1 : (int)o->levels[l].size();
}
extern "C" const uint64_t* orc_octree_level(const orc_octree* o, int l) {
    return (l < 0 || l > o->nLevels) ? 0 : o->levels[l].data();
}
extern "C" int orc_children_mask(const uint64_t* e, int size, uint64_t father) {
    return children_mask_dev(e, size, father);
}

/* ======================================================================== */
/* Traversal + march (src/Octree.cu:620-739, src/rayCaster.cu:139-265)       */
/* ======================================================================== */
namespace {
struct RayStack {              /* GstackIndex / GstackLevel / GstackActual */
    std::vector<uint64_t> idx; std::vector<int> lvl; int top; int maxDepth;
};

/* _cuda_getFirtsVoxel (src/Octree.cu:620-720) for one ray; returns true and
 * the candidate id when a node of finalLevel is reached. */
static bool first_voxel(const orc_octree* o, V3 origin, V3 ray, int finalLevel, RayStack& st,
                        uint64_t* id, int64_t* expansions) {
    if (st.top < 0) return false;
    const int nLevels = o->nLevels;
    int top = st.top;
    int currentLevel = st.lvl[top];
    uint64_t current = st.idx[top];
    I3 minBox = min_box(current, currentLevel, nLevels);
    uint64_t children[8]; float tnears[8], tfars[8];
    while (top >= 0) {
        if (st.lvl[top] == finalLevel) {
            *id = st.idx[top];
            st.top = top - 1;
            return true;
        }
        minBox = update_coordinates(nLevels, currentLevel, current, st.lvl[top], st.idx[top], minBox);
        current = st.idx[top];
        currentLevel = st.lvl[top];
        top--;
        (*expansions)++;
        /* _cuda_searchChildrenValidAndHit2 (:375-532) */
        const int level = currentLevel + 1;
        const std::vector<uint64_t>& e = o->levels[level];
        int mask = children_mask_dev(e.data(), (int)e.size(), current);
        int dim = 1 << (nLevels - level);
        int nValid = 0;
        for (int k = 0; k < 8; k++) {
            I3 cb = {minBox.x + ((k >> 2) & 1) * dim, minBox.y + ((k >> 1) & 1) * dim,
                     minBox.z + (k & 1) * dim};
            if (ray_aabb_level(origin, ray, &tnears[nValid], &tfars[nValid], nLevels, cb, level) &&
                tfars[nValid] >= 0.0 && ((mask >> k) & 1)) {
                children[nValid] = (current << 3) + (uint64_t)k;
                nValid++;
            }
        }
        /* bubble sort by (tnear, tfar) (:665-706) */
        int n = nValid;
        while (n != 0) {
            int newn = 0;
            for (int i = 1; i < nValid; i++) {
                if (tnears[i - 1] > tnears[i] ||
                    (tnears[i - 1] == tnears[i] && tfars[i - 1] > tfars[i])) {
                    std::swap(children[i], children[i - 1]);
                    std::swap(tnears[i], tnears[i - 1]);
                    std::swap(tfars[i], tfars[i - 1]);
                    newn = i;
                }
            }
            n = newn;
        }
        for (int i = nValid - 1; i >= 0; i--) {
            top++;
            if ((int)st.idx.size() <= top) { st.idx.resize(top + 16); st.lvl.resize(top + 16); }
            st.idx[top] = children[i];
            st.lvl[top] = currentLevel + 1;
        }
        if (top + 1 > st.maxDepth) st.maxDepth = top + 1;
    }
    st.top = top;
    return false;
}
}  // namespace

extern "C" int orc_render_frame(const orc_octree* o, const void* vol, int vtype, const int realDim[3],
                                const orc_camera* cam, const orc_render_params* p, orc_render_out* out) {
    const int nLevels = o->nLevels;
    if (p->levelO < 1 || p->levelO > nLevels || p->levelC < 0 || p->levelC > p->levelO) return -1;
    const int numRays = cam->W * cam->H;
    const int rb = p->ray_begin < 0 ? 0 : p->ray_begin;
    const int re = (p->ray_end <= 0 || p->ray_end > numRays) ? numRays : p->ray_end;
    const int rs = p->ray_stride <= 0 ? 1 : p->ray_stride;
    Volume V = {vol, vtype, realDim[0], realDim[1], realDim[2]};
    const V3 origin = fromf3(cam->position);
    const V3 light = fromf3(p->light);
    const int cubeDim = 1 << (nLevels - p->levelC);
    const int D = cubeDim + 2 * p->cubeInc;
    const int dimO = (int)powf(2, (float)(nLevels - p->levelO));   /* src/rayCaster.cu:161 */
    const bool rootValid = o->levels[0].size() >= 2 && check_range(o->levels[0].data(),
                           (int)o->levels[0].size(), 1, 0, 1);
    int64_t a_rays = 0, a_hits = 0, a_samp = 0, a_nsamp = 0, a_cand = 0, a_exp = 0;
    int64_t a_maxstack = 0, a_overflow = 0, a_oob = 0;
    const int nIter = (re > rb) ? (re - rb + rs - 1) / rs : 0;
#ifdef _OPENMP
    int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nth) \
    reduction(+ : a_rays, a_hits, a_samp, a_nsamp, a_cand, a_exp, a_overflow, a_oob) \
    reduction(max : a_maxstack)
#endif
    for (int it = 0; it < nIter; it++) {
        const int id = rb + it * rs;
        const V3 ray = p->dirs ? fromf3(p->dirs[id]) : ray_dir(cam, id);
        int64_t samp = 0, nsamp = 0, cand = 0, exps = 0, oob = 0;
        uint64_t hitNode = 0, hitBrick = 0;
        bool hit = false;
        V3 X = mk(0, 0, 0), n = mk(0, 0, 0);
        float rgba[4] = {1.0f, 1.0f, 1.0f, 1.0f};
        RayStack st;
        st.idx.assign(32, 0); st.lvl.assign(32, 0);
        st.top = 0; st.idx[0] = 1; st.lvl[0] = 0; st.maxDepth = 1;   /* cuda_resetState :750-760 */
        float tn, tf;
        I3 z0 = {0, 0, 0}, zr = {1 << nLevels, 1 << nLevels, 1 << nLevels};
        /* root test (src/Octree.cu:729) */
        if (rootValid && ray_aabb(origin, ray, &tn, &tf, z0, zr)) {
            uint64_t cid;
            while (first_voxel(o, origin, ray, p->levelO, st, &cid, &exps)) {
                cand++;
                I3 mb = min_box(cid, p->levelO, nLevels);
                I3 mx = {mb.x + dimO, mb.y + dimO, mb.z + dimO};
                if (!ray_aabb(origin, ray, &tn, &tf, mb, mx)) continue;  /* never: traversal accepted it */
                uint64_t cubeID = cid >> (3 * (p->levelO - p->levelC));   /* src/lruCache.cu:177 */
                I3 bm = min_box(cubeID, p->levelC, nLevels);
                I3 minBox = {bm.x - p->cubeInc, bm.y - p->cubeInc, bm.z - p->cubeInc};
                Brick B = {&V, minBox, D, &oob};
                int maxStep = d2i(ceil((tf - tn) / 0.5));
                V3 Xh;
                if (march(origin, ray, tn, maxStep, B, minBox, p->iso, &Xh, &samp, p->refine)) {
                    hit = true; hitNode = cid; hitBrick = cubeID; X = Xh;
                    n = normal_at(X, B, minBox);
                    nsamp += 6;
                    V3 l = normalize(X - light);
                    float dif = fabsf(n.x * l.x + n.y * l.y + n.z * l.z);
                    float a = X.y / 256.0f;
                    rgba[0] = (1 - a) * dif; rgba[1] = a * dif; rgba[2] = 0.0f * dif; rgba[3] = 1.0f;
                    break;
                }
            }
        }
        if (out->node_id) out->node_id[id] = hitNode;
        if (out->brick_id) out->brick_id[id] = hitBrick;
        if (out->t) out->t[id] = hit ? dot(X - origin, ray) : -1.0f;
        if (out->normal) { out->normal[3 * id] = n.x; out->normal[3 * id + 1] = n.y; out->normal[3 * id + 2] = n.z; }
        if (out->rgba) for (int c = 0; c < 4; c++) out->rgba[4 * id + c] = rgba[c];
        if (out->rgb8) for (int c = 0; c < 3; c++) out->rgb8[3 * id + c] = to_u8(rgba[c]);
        a_rays++; a_hits += hit; a_samp += samp; a_nsamp += nsamp; a_cand += cand; a_exp += exps;
        a_oob += oob;
        if (st.maxDepth > a_maxstack) a_maxstack = st.maxDepth;
        if (st.maxDepth > 32) a_overflow++;
    }
    out->rays = a_rays; out->hits = a_hits; out->samples = a_samp; out->normal_samples = a_nsamp;
    out->candidates = a_cand; out->expansions = a_exp; out->max_stack = a_maxstack;
    out->stack_overflow_rays = a_overflow; out->oob_taps = a_oob;
    return 0;
}

/* ======================================================================== */
/* renderCube (src/rayCaster.cu:267-357)                                    */
/* ======================================================================== */
namespace {
struct RawCube {   /* data[z + y*D + x*D*D] with D = dims.x, bounded by the allocation */
    const float* d; int D; int64_t total; int64_t* oob;
    inline float get(int x, int y, int z) const {
        int64_t i = (int64_t)z + (int64_t)y * D + (int64_t)x * D * D;
        if (i < 0 || i >= total) { (*oob)++; return 0.0f; }
        return d[i];
    }
};
}
extern "C" void orc_render_cube(const orc_camera* cam, const float* cube, const int pmin[3],
                                const int cdim[3], const int cinc[3], float iso, orc_f3 lightp,
                                float* rgba, int64_t* oob_taps) {
    const int n = cam->W * cam->H;
    const V3 origin = fromf3(cam->position), light = fromf3(lightp);
    const I3 D = {cdim[0] + 2 * cinc[0], cdim[1] + 2 * cinc[1], cdim[2] + 2 * cinc[2]};
    int64_t oob = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : oob)
#endif
    for (int tid = 0; tid < n; tid++) {
        V3 ray = ray_dir(cam, tid);
        I3 minBox = {pmin[0], pmin[1], pmin[2]};
        I3 maxBox = {minBox.x + cdim[0], minBox.y + cdim[1], minBox.z + cdim[2]};
        float tn, tf;
        bool hit = false;
        V3 X = mk(0, 0, 0);
        int64_t ns = 0, lo = 0;
        RawCube C = {cube, D.x, (int64_t)D.x * D.y * D.z, &lo};
        if (ray_aabb(origin, ray, &tn, &tf, minBox, maxBox)) {
            minBox.x -= cinc[0]; minBox.y -= cinc[1]; minBox.z -= cinc[2];
            float maxStep = (float)((tf - tn) / 0.5);
            hit = march(origin, ray, tn, maxStep, C, minBox, iso, &X, &ns);
        }
        float* px = rgba + 4 * (size_t)tid;
        if (hit) {
            V3 nn = normal_at(X, C, minBox);
            V3 l = normalize(X - light);
            float dif = fabsf(dot(nn, l));
            float a = X.y / (float)cdim[1];
            px[0] = (1 - a) * dif; px[1] = a * dif; px[2] = 0.0f * dif; px[3] = 1.0f;
        } else {
            px[0] = px[1] = px[2] = px[3] = 1.0f;
        }
        oob += lo;
    }
    if (oob_taps) *oob_taps = oob;
}

/* ======================================================================== */
/* FileManager::readHDF5_Voxel_Array (src/FileManager.cu:86-167)            */
/* ======================================================================== */
extern "C" void orc_read_voxels(const float* vol, const int dims[3], const int s[3], const int e[3],
                                float* out) {
    int64_t dim[3] = {labs((long)(e[0] - s[0])), labs((long)(e[1] - s[1])), labs((long)(e[2] - s[2]))};
    memset(out, 0, (size_t)(dim[0] * dim[1] * dim[2]) * sizeof(float));
    if (s[0] >= dims[0] || s[1] >= dims[1] || s[2] >= dims[2] || e[0] < 0 || e[1] < 0 || e[2] < 0)
        return;
    int64_t off_out[3], off[3], dimR[3];
    for (int a = 0; a < 3; a++) {
        off_out[a] = s[a] < 0 ? -(int64_t)s[a] : 0;
        off[a] = s[a] < 0 ? 0 : s[a];
        dimR[a] = e[a] > dims[a] ? dims[a] - off[a] : e[a] - off[a];
        if (dimR[a] <= 0) return;
    }
    for (int64_t a = 0; a < dimR[0]; a++)
        for (int64_t b = 0; b < dimR[1]; b++) {
            const float* src = vol + ((off[0] + a) * dims[1] + (off[1] + b)) * (int64_t)dims[2] + off[2];
            float* dst = out + ((off_out[0] + a) * dim[1] + (off_out[1] + b)) * dim[2] + off_out[2];
            memcpy(dst, src, (size_t)dimR[2] * sizeof(float));
        }
}

/* ======================================================================== */
/* OctreeM builder (src/CreateOctree.cu)                                     */
/* ======================================================================== */
namespace {
/* OctreeLevel (:16-284) */
struct Level {
    std::vector<uint64_t> e; bool has = false; bool status = false; uint64_t next = 0;
    void insert(uint64_t index) {                    /* :79-116 */
        if (has && index < next) return;
        if (!has) { has = true; e.push_back(index); status = false; next = index + 1; return; }
        if (next == index) { next++; return; }
        e.push_back(next - 1); e.push_back(index); status = false; next = index + 1;
    }
    void complete() {                                /* :118-128 */
        if (!has) status = false;
        else { e.push_back(next - 1); status = true; }
    }
    bool check(uint64_t index, int mn, int mx) const {   /* :130-139 */
        return (e.at(mn) < index && e.at(mx) > index) || index == e.at(mn) || index == e.at(mx);
    }
    int closer(uint64_t index, int mn, int mx) const {   /* :182-221 */
        int diff = mx - mn;
        unsigned int middle = mn + (diff / 2);
        if (diff <= 1) { if (middle % 2 == 1) middle--; return (int)middle; }
        if (middle % 2 == 1) middle--;
        if (check(index, (int)middle, (int)middle + 1)) return (int)middle;
        else if (index < e.at(middle)) return closer(index, mn, (int)middle - 1);
        else if (index > e.at(middle + 1)) return closer(index, (int)middle + 2, mx);
        return 0;
    }
    bool seq(uint64_t index, int mn, int mx) const {     /* :223-244, up=true */
        for (int i = mn; i < mx; i += 2) {
            if (check(index, i, i + 1)) return true;
            if (index < e.at(i + 1)) break;
        }
        return false;
    }
    int search_children(uint64_t father) const {         /* :247-284 */
        if (!status) return 0;
        uint64_t c = father << 3;
        int num = 0;
        if (e.size() == 2) {
            for (int i = 0; i < 8; i++) { if (check(c, 0, 1)) num++; c++; }
            return num;
        }
        unsigned int closer1 = (unsigned int)closer(c, 0, (int)e.size());
        unsigned int closer8 = (unsigned int)closer(c + 7, (int)closer1, (int)e.size()) + 1;
        if (closer8 >= e.size()) closer8 = (unsigned int)(e.size() - 1);
        for (int i = 0; i < 8; i++) { if (seq(c, (int)closer1, (int)closer8)) num++; c++; }
        return num;
    }
};
}  // namespace

extern "C" int orc_build_octree(const void* vol, int vtype, const int realDim[3], float iso,
                                const char* path) {
    /* :300-334 */
    int dimension;
    if (realDim[0] > realDim[1] && realDim[0] > realDim[2]) dimension = realDim[0];
    else if (realDim[1] > realDim[2]) dimension = realDim[1];
    else dimension = realDim[2];
    float aux = logf((float)dimension) / logf(2.0);
    float aux2 = aux - floorf(aux);
    int nLevels = aux2 > 0.0 ? (int)(aux + 1) : (int)aux;
    dimension = (int)pow(2, nLevels);
    Volume V = {vol, vtype, realDim[0], realDim[1], realDim[2]};
    std::vector<Level> oct(nLevels + 1);

    /* Leaf level (:430-531): every cell code in Morton order; a cell is
     * valid when its 8 zero-padded corners straddle iso. */
    {
        const uint64_t first = coord_to_index(0, 0, 0, nLevels, nLevels);
        const uint64_t ncell = (uint64_t)dimension * dimension * dimension;
        std::vector<uint8_t> valid(ncell);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
        for (int64_t k = 0; k < (int64_t)ncell; k++) {
            I3 c = min_box(first + (uint64_t)k, nLevels, nLevels);
            float v[8];
            v[0] = V.get(c.x, c.y, c.z);         v[1] = V.get(c.x, c.y, c.z + 1);
            v[2] = V.get(c.x, c.y + 1, c.z);     v[3] = V.get(c.x, c.y + 1, c.z + 1);
            v[4] = V.get(c.x + 1, c.y, c.z);     v[5] = V.get(c.x + 1, c.y, c.z + 1);
            v[6] = V.get(c.x + 1, c.y + 1, c.z); v[7] = V.get(c.x + 1, c.y + 1, c.z + 1);
            bool has = false;
            bool sign = (v[0] - iso) < 0;
            for (int i = 1; i < 8 && !has; ++i)
                if (((v[i] - iso) < 0) != sign) has = true;
            valid[k] = has;
        }
        for (uint64_t k = 0; k < ncell; k++)
            if (valid[k]) oct[nLevels].insert(first + k);
        oct[nLevels].complete();
    }
    /* Inner levels (:541-571): `while(inicio!=fin)` visits every code of the
     * level except the last.  A node can only be accepted when a child is
     * truly inside a range (checkRange is exact), so only parents of
     * existing children are searched. */
    for (int level = nLevels - 1; level >= 1; level--) {
        const Level& below = oct[level + 1];
        const uint64_t fin = coord_to_index(dimension - 1, dimension - 1, dimension - 1, level, nLevels);
        Level& L = oct[level];
        uint64_t lastParent = 0;
        bool any = false;
        for (size_t r = 0; r + 1 < below.e.size(); r += 2) {
            uint64_t p0 = below.e[r] >> 3, p1 = below.e[r + 1] >> 3;
            if (any && p0 <= lastParent) p0 = lastParent + 1;
            for (uint64_t p = p0; p <= p1; p++) {
                any = true; lastParent = p;
                if (p == fin) continue;
                if (below.search_children(p) > 0) L.insert(p);
            }
        }
        L.complete();
    }
    /* Level 0 (:532-540) */
    if (nLevels >= 1 && oct[1].search_children(1) > 0) { oct[0].insert(1); oct[0].complete(); }

    /* writeToFile (:342-371) */
    FILE* f = fopen(path, "wb");
    if (!f) return -1;
    int magic = 919278872;
    fwrite(&magic, 4, 1, f);
    fwrite(&iso, 4, 1, f);
    fwrite(&dimension, 4, 1, f);
    fwrite(&realDim[0], 4, 1, f); fwrite(&realDim[1], 4, 1, f); fwrite(&realDim[2], 4, 1, f);
    fwrite(&nLevels, 4, 1, f);
    for (int i = nLevels; i >= 0; i--) {
        int n = (int)oct[i].e.size();
        fwrite(&n, 4, 1, f);
        if (n) fwrite(oct[i].e.data(), 8, (size_t)n, f);
    }
    fclose(f);
    return 0;
}

/* ======================================================================== */
/* lruCache state machine (src/lruCache.cu)                                  */
/* ======================================================================== */
namespace {
struct LNode { LNode* after; LNode* before; unsigned int element; uint64_t cubeID; };
struct LList {                                   /* LinkedList (:7-99) */
    std::vector<LNode> mem; LNode* list; LNode* last;
    explicit LList(int size) : mem(size) {
        for (int i = 0; i < size; i++) {
            mem[i].after = (i + 1 < size) ? &mem[i + 1] : 0;
            mem[i].before = i > 0 ? &mem[i - 1] : 0;
            mem[i].element = (unsigned)i; mem[i].cubeID = 0;
        }
        list = &mem[0]; last = &mem[size - 1];
    }
    LNode* get_first(uint64_t newID, uint64_t* removed) {   /* :44-62 */
        LNode* first = list;
        list = first->after; list->before = 0;
        first->after = 0; first->before = last;
        last->after = first; last = first;
        *removed = last->cubeID; last->cubeID = newID;
        return first;
    }
    LNode* move_last(LNode* node) {                  /* :64-99 */
        if (node->before == 0) {
            LNode* first = list;
            list = first->after; list->before = 0;
            first->after = 0; first->before = last;
            last->after = first; last = first;
            return first;
        } else if (node->after == 0) {
            return node;
        }
        node->before->after = node->after;
        node->after->before = node->before;
        last->after = node; node->before = last; node->after = 0; last = node;
        return node;
    }
};
static inline uint64_t int_key(uint64_t k) { return (uint64_t)(int64_t)(int32_t)(uint32_t)k; }
}  // namespace

struct orc_lru {
    int numElements, numElementsCPU, levelOctree, levelCube;
    LList gpu, cpu;
    std::map<uint64_t, LNode*> stored, storedCPU;
    int64_t access = 0, hitsCPU = 0, missCPU = 0, hitsGPU = 0, missGPU = 0;
    orc_lru(int ne, int nc, int lo, int lc)
        : numElements(ne), numElementsCPU(nc), levelOctree(lo), levelCube(lc), gpu(ne), cpu(nc) {}
};

extern "C" orc_lru* orc_lru_create(int ne, int nc, int lo, int lc) {
    if (ne < 2 || nc < 2) return 0;   /* LinkedList(1) dereferences past its array */
    return new orc_lru(ne, nc, lo, lc);
}
extern "C" void orc_lru_free(orc_lru* c) { delete c; }
extern "C" int orc_lru_update(orc_lru* c, int num, const uint64_t* id, uint8_t* state, int* slot,
                              uint64_t* cubeID, uint64_t* loads) {
    int newC = 0, newG = 0, nloads = 0;               /* updateCache (:298-313) */
    for (int i = 0; i < num; i++) {
        if (!(state[i] == 1 || state[i] == 8)) continue;
        /* updateCube (:168-296) */
        c->access++;
        uint64_t idCube = id[i] >> (3 * (c->levelOctree - c->levelCube));
        std::map<uint64_t, LNode*>::iterator it = c->stored.find(idCube);
        if (it == c->stored.end()) {
            if (newG >= c->numElements) { state[i] = 1; cubeID[i] = 0; slot[i] = -1; continue; }
            std::map<uint64_t, LNode*>::iterator itc = c->storedCPU.find(idCube);
            if (itc == c->storedCPU.end()) {
                if (newC >= c->numElementsCPU) { state[i] = 1; cubeID[i] = 0; slot[i] = -1; continue; }
                c->missCPU++;
                uint64_t removed = 0;
                LNode* node = c->cpu.get_first(idCube, &removed);
                c->storedCPU.insert(std::make_pair(int_key(idCube), node));
                if (removed != 0) {
                    std::map<uint64_t, LNode*>::iterator r = c->storedCPU.find(removed);
                    if (r != c->storedCPU.end()) c->storedCPU.erase(r);
                }
                loads[nloads++] = idCube;
                newC++;
            } else {
                c->hitsCPU++; c->missCPU++;
                c->cpu.move_last(itc->second);
            }
            uint64_t removed = 0;
            LNode* node = c->gpu.get_first(idCube, &removed);
            c->stored.insert(std::make_pair(int_key(idCube), node));
            if (removed != 0) {
                std::map<uint64_t, LNode*>::iterator r = c->stored.find(removed);
                if (r != c->stored.end()) c->stored.erase(r);
            }
            slot[i] = (int)node->element; state[i] = 2; cubeID[i] = idCube;
            newG++;
            c->missGPU++;
        } else {
            c->hitsGPU++;
            LNode* node = it->second;
            c->gpu.move_last(node);
            slot[i] = (int)node->element; state[i] = 2; cubeID[i] = idCube;
        }
    }
    return nloads;
}
extern "C" void orc_lru_stats(const orc_lru* c, int64_t out[5]) {
    out[0] = c->access; out[1] = c->hitsCPU; out[2] = c->missCPU; out[3] = c->hitsGPU; out[4] = c->missGPU;
}
