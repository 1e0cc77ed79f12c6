/*
 * vt_search.h -- the reference's two range-list searches, usable from host
 * and device code of libvt.so.
 *
 * A level of the octree file is a sorted array of inclusive Morton ranges
 * [s0,e0,s1,e1,...].  The reference asks "which children of node p does
 * this level hold" with two different procedures:
 *   - the renderer's device variant (src/Octree.cu:15-20, :78-99,
 *     :134-142, :375-532), used to flatten the octree for traversal;
 *   - the builder's host variant (src/CreateOctree.cu:130-284), used to
 *     decide which inner nodes exist.
 * Both can miss a child that a range holds (never report one it does not),
 * so they are restated step by step rather than replaced by a plain binary
 * search.
 */
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define VT_SHD __host__ __device__ inline
#else
#define VT_SHD inline
#endif

namespace vtsearch {

/* device variant: reads past the end only happen in the terminating
 * iteration of the closer search and cannot change its result; they read 0 */
VT_SHD uint64_t el(const uint64_t* e, int n, int i) { return (i >= 0 && i < n) ? e[i] : 0ull; }
VT_SHD bool in_pair(const uint64_t* e, int n, uint64_t c, int a, int b) {
    uint64_t lo = el(e, n, a), hi = el(e, n, b);
    return c == lo || c == hi || (lo < c && hi > c);
}
VT_SHD int closer_device(const uint64_t* e, int n, uint64_t c, int lo, int hi) {
    bool end = false, found = false;
    int mid = 0;
    while (!end && !found) {
        int diff = hi - lo;
        mid = lo + diff / 2;
        if (mid % 2 == 1) mid--;
        end = diff <= 1;
        found = in_pair(e, n, c, mid, mid + 1);
        if (c < el(e, n, mid)) hi = mid - 1;
        else lo = mid + 2;
    }
    return mid;
}
/* 8-bit mask of the children of `father` the renderer's search accepts */
VT_SHD int children_mask_device(const uint64_t* e, int n, uint64_t father) {
    const uint64_t c0 = father << 3;
    int mask = 0;
    if (n == 2) {
        for (int k = 0; k < 8; k++)
            if (in_pair(e, n, c0 + k, 0, 1)) mask |= 1 << k;
        return mask;
    }
    unsigned int w0 = (unsigned int)closer_device(e, n, c0, 0, n - 1);
    unsigned int w1 = (unsigned int)closer_device(e, n, c0 + 7, (int)w0, n - 1) + 1;
    if (w1 >= (unsigned int)n) w1 = (unsigned int)(n - 1);
    for (int k = 0; k < 8; k++) {
        bool found = false;
        for (int i = (int)w0; i < (int)w1; i += 2)
            if (in_pair(e, n, c0 + k, i, i + 1)) found = true;
        if (found) mask |= 1 << k;
    }
    return mask;
}

/* host (builder) variant */
VT_SHD bool hpair(const uint64_t* e, uint64_t c, int64_t a, int64_t b) {
    return (e[a] < c && e[b] > c) || c == e[a] || c == e[b];
}
VT_SHD int64_t closer_host(const uint64_t* e, uint64_t c, int64_t lo, int64_t hi) {
    for (;;) {
        int64_t diff = hi - lo;
        uint32_t mid = (uint32_t)(lo + diff / 2);
        if (diff <= 1) { if (mid % 2 == 1) mid--; return (int32_t)mid; }
        if (mid % 2 == 1) mid--;
        if (hpair(e, c, mid, (int64_t)mid + 1)) return mid;
        if (c < e[mid]) hi = (int64_t)mid - 1;
        else if (c > e[mid + 1]) lo = (int64_t)mid + 2;
        else return 0;
    }
}
/* number of children of `father` the builder's search finds (>0 = node
 * exists); n = 0 is a level without elements (status false) */
VT_SHD int search_children_host(const uint64_t* e, int64_t n, uint64_t father) {
    if (n <= 0) return 0;
    uint64_t c = father << 3;
    int num = 0;
    if (n == 2) {
        for (int i = 0; i < 8; i++, c++) if (hpair(e, c, 0, 1)) num++;
        return num;
    }
    uint32_t w0 = (uint32_t)closer_host(e, c, 0, n);
    uint32_t w1 = (uint32_t)closer_host(e, c + 7, (int32_t)w0, n) + 1;
    if ((uint64_t)w1 >= (uint64_t)n) w1 = (uint32_t)(n - 1);
    for (int k = 0; k < 8; k++, c++) {
        for (int64_t i = (int32_t)w0; i < (int32_t)w1; i += 2) {
            if (hpair(e, c, i, i + 1)) { num++; break; }
            if (c < e[i + 1]) break;
        }
    }
    return num;
}

}  // namespace vtsearch
