/*
 * vt_math.cuh -- device arithmetic of the ray-casting path.
 *
 * Every function performs the same IEEE single-precision operations, in the
 * same order, as the reference source it cites (carlosduelo/visualTur).
 * The library is compiled with --fmad=false (no contraction), IEEE division
 * and square root, so results are bit-identical to a host evaluation of the
 * same expressions.  normalize() uses 1/sqrtf, the reference's host
 * definition of rsqrtf (inc/cutil_math.h).
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define VT_HD __host__ __device__ __forceinline__

namespace vt {

VT_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
VT_HD float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
VT_HD float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
VT_HD float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
VT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VT_HD float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
VT_HD float3 normalize(float3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return mul(v, inv); }

/* Pixel direction of cuda_updateRays (src/Camera.cu:59-72); i = row. */
VT_HD float3 ray_dir(float3 look, float3 up, float3 right, float distance, float h, float w, int H,
                     int W, int i, int j) {
    float ih = h / H, iw = w / W;
    float3 A = mul(look, distance);
    A = add(A, mul(up, -(h / 2.0f) + (ih * ((float)i + 0.5f))));
    A = add(A, mul(right, -(w / 2.0f) + (iw * ((float)j + 0.5f))));
    return normalize(A);
}

/* Per-ray reciprocal directions: the reference evaluates `1 / dir.x` in
 * every slab test (src/Octree.cu:268); the value is the same each time. */
struct RayInv { float3 o; float dx, dy, dz; };

/* _cuda_RayAABB2 / _cuda_RayAABB (src/Octree.cu:258-330,
 * src/rayCaster.cu:12-79).  Conditional min/max exactly as written, so
 * NaN operands behave as in the reference. */
__device__ __forceinline__ bool slab(const RayInv& r, int mnx, int mny, int mnz, int mxx, int mxy,
                                     int mxz, float* tnear, float* tfar) {
    bool hit = true;
    float tmin, tmax, tymin, tymax, tzmin, tzmax;
    if (r.dx >= 0) { tmin = ((float)mnx - r.o.x) * r.dx; tmax = ((float)mxx - r.o.x) * r.dx; }
    else { tmin = ((float)mxx - r.o.x) * r.dx; tmax = ((float)mnx - r.o.x) * r.dx; }
    if (r.dy >= 0) { tymin = ((float)mny - r.o.y) * r.dy; tymax = ((float)mxy - r.o.y) * r.dy; }
    else { tymin = ((float)mxy - r.o.y) * r.dy; tymax = ((float)mny - r.o.y) * r.dy; }
    if ((tmin > tymax) || (tymin > tmax)) hit = false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    if (r.dz >= 0) { tzmin = ((float)mnz - r.o.z) * r.dz; tzmax = ((float)mxz - r.o.z) * r.dz; }
    else { tzmin = ((float)mxz - r.o.z) * r.dz; tzmax = ((float)mnz - r.o.z) * r.dz; }
    if ((tmin > tzmax) || (tzmin > tmax)) hit = false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    *tnear = (tmin < 0.0f) ? 0.0f : tmin;
    *tfar = tmax;
    return hit;
}

/* The comparison half of slab(): per-axis entry/exit parameters already
 * ordered by the direction's sign.  slab() == slab_t() on the same planes. */
__device__ __forceinline__ bool slab_t(float tmin, float tmax, float tymin, float tymax, float tzmin, float tzmax,
                                       float* tnear, float* tfar) {
    bool hit = true;
    if ((tmin > tymax) || (tymin > tmax)) hit = false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    if ((tmin > tzmax) || (tzmin > tmax)) hit = false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    *tnear = (tmin < 0.0f) ? 0.0f : tmin;
    *tfar = tmax;
    return hit;
}

/* Level of a sentinel-bit Morton code (getIndexLevel,
 * inc/mortonCodeUtil.hpp:42-86) for valid codes (>= 1). */
VT_HD int code_level(uint64_t c) {
#ifdef __CUDA_ARCH__
    return (63 - __clzll((long long)c)) / 3;
#else
    return (63 - __builtin_clzll(c)) / 3;
#endif
}

/* Inverse of the 3-way bit dilation: bit 3k of v -> bit k. */
VT_HD uint32_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ull;
    v = (v ^ (v >> 4)) & 0x100F00F00F00F00Full;
    v = (v ^ (v >> 8)) & 0x001F0000FF0000FFull;
    v = (v ^ (v >> 16)) & 0x001F00000000FFFFull;
    v = (v ^ (v >> 32)) & 0x00000000001FFFFFull;
    return (uint32_t)v;
}
/* 3-way bit dilation (dilateInteger, inc/mortonCodeUtil.hpp:31-40): bit k
 * of v -> bit 3k, for 21-bit v. */
VT_HD uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}
/* coordinateToIndex (inc/mortonCodeUtil.hpp:146-169) from node coordinates
 * at `level` (each in [0, 2^level)): sentinel bit 3*level, x in bit 2 of
 * each triplet. */
VT_HD uint64_t node_code(uint32_t x, uint32_t y, uint32_t z, int level) {
    return (1ull << (3 * level)) | (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
}

/* getMinBoxIndex2 (inc/mortonCodeUtil.hpp:120-144): min corner of node
 * `code` at `level` of an nLevels tree (x in bit 2 of each triplet). */
VT_HD int3 min_box(uint64_t code, int level, int nLevels) {
    if (level == 0) return make_int3(0, 0, 0);
    uint64_t c = code & ((1ull << (3 * level)) - 1ull);
    int s = nLevels - level;
    return make_int3((int)(compact3(c >> 2) << s), (int)(compact3(c >> 1) << s),
                     (int)(compact3(c) << s));
}

/* float -> int as the reference's device code converts (cvt.rzi: NaN -> 0,
 * saturating); explicit so host and device agree. */
VT_HD int f2i(float v) {
#ifdef __CUDA_ARCH__
    return __float2int_rz(v);
#else
    if (v != v) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    if (v <= -2147483648.0f) return (-2147483647 - 1);
    return (int)v;
#endif
}

/* int maxStep = ceil((tfar-tnear)/0.5) (src/rayCaster.cu:182): the double
 * quotient is an exact doubling, so ceilf of the float doubling is equal. */
VT_HD int max_steps(float tnear, float tfar) { return f2i(ceilf((tfar - tnear) * 2.0f)); }

VT_HD uint8_t to_u8(float v) {
    float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)(c * 255.0f);
}

}  // namespace vt
