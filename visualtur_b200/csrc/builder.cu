/*
 * builder.cu -- GPU octree builder writing the reference's octree file
 * (OctreeM, src/CreateOctree.cu:300-573, writeToFile :342-371).
 *
 * Reference semantics, restated level by level:
 *   nLevels  = ceil(log2(max extent)) computed as the reference does in
 *              float (:316-319); dimension = 2^nLevels;
 *   leaf     = every cell code of level nLevels (inclusive range, :452),
 *              valid when the 8 zero-padded corner voxels straddle iso with
 *              the test ((v-iso)<0) != ((v0-iso)<0) (:497-501);
 *   inner l  = every code of level l except the last (`while(inicio!=fin)`,
 *              :550) whose children the builder's range search finds in
 *              level l+1 (:553, searchChildren :247-284);
 *   root     = {1,1} when level 1 has children of node 1 (:532-540);
 *   a level  = its valid codes as sorted inclusive runs [s,e] (insert /
 *              completeLevel, :79-128).
 * The GPU version keeps each level as a bitmask over its Morton codes, turns
 * runs of ones into [s,e] pairs with two prefix sums, and runs the builder's
 * search only for parents that have a set child byte (the search never
 * finds a child a range does not hold).  Output is byte-identical to the
 * reference's volumeToOctree.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <cub/cub.cuh>
#include <vector>

#include "../../include/vt.h"
#include "vt_math.cuh"
#include "vt_runtime.h"
#include "vt_search.h"

namespace vtb {

#define CKB(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) { st = vtrt::fail(VT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); goto done; } \
    } while (0)

template <int VTYPE>
__device__ __forceinline__ float vox(const void* v, long long dx, long long dy, long long dz, long long x, long long y,
                                     long long z) {
    if (x >= dx || y >= dy || z >= dz) return 0.0f;   /* zero padding (x,y,z >= 0 here) */
    long long i = (x * dy + y) * dz + z;
    if (VTYPE == 0) return __ldg((const float*)v + i);
    return (float)__ldg((const unsigned char*)v + i);
}

/* leaf cells: bit b of word w = cell with Morton offset 32w+b (src/CreateOctree.cu:471-517) */
template <int VTYPE>
__global__ void k_leaf(const void* v, long long dx, long long dy, long long dz, float iso, uint32_t* bits,
                       long long nwords) {
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        uint32_t m = 0;
        for (int b = 0; b < 32; b++) {
            uint64_t off = (uint64_t)w * 32 + b;
            long long x = vt::compact3(off >> 2), y = vt::compact3(off >> 1), z = vt::compact3(off);
            float c[8];
            c[0] = vox<VTYPE>(v, dx, dy, dz, x, y, z);         c[1] = vox<VTYPE>(v, dx, dy, dz, x, y, z + 1);
            c[2] = vox<VTYPE>(v, dx, dy, dz, x, y + 1, z);     c[3] = vox<VTYPE>(v, dx, dy, dz, x, y + 1, z + 1);
            c[4] = vox<VTYPE>(v, dx, dy, dz, x + 1, y, z);     c[5] = vox<VTYPE>(v, dx, dy, dz, x + 1, y, z + 1);
            c[6] = vox<VTYPE>(v, dx, dy, dz, x + 1, y + 1, z); c[7] = vox<VTYPE>(v, dx, dy, dz, x + 1, y + 1, z + 1);
            bool sign = (c[0] - iso) < 0;
            bool has = false;
            for (int i = 1; i < 8; i++) has |= (((c[i] - iso) < 0) != sign);
            m |= (uint32_t)has << b;
        }
        bits[w] = m;
    }
}

/* inner level: parent p exists when it has a set child byte, is not the
 * level's last code, and the builder's search over level l+1 finds a child */
__global__ void k_inner(const uint32_t* childBits, const uint64_t* e, long long n, uint64_t base, uint64_t lastOff,
                        uint32_t* bits, long long nwords, long long nparents) {
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        uint32_t m = 0;
        for (int b = 0; b < 32; b++) {
            long long p = w * 32 + b;
            if (p >= nparents || (uint64_t)p == lastOff) continue;
            uint32_t byte = (childBits[p >> 2] >> (8 * (p & 3))) & 0xFFu;
            if (!byte) continue;
            if (vtsearch::search_children_host(e, n, base + (uint64_t)p) > 0) m |= 1u << b;
        }
        bits[w] = m;
    }
}

/* run starts / ends per word (bit i of the level = Morton offset i) */
__global__ void k_runcount(const uint32_t* bits, long long nwords, uint32_t* cs, uint32_t* ce) {
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        uint32_t m = bits[w];
        uint32_t prev = w > 0 ? bits[w - 1] >> 31 : 0u;
        uint32_t next = w + 1 < nwords ? bits[w + 1] & 1u : 0u;
        uint32_t starts = m & ~((m << 1) | prev);
        uint32_t ends = m & ~((m >> 1) | (next << 31));
        cs[w] = __popc(starts);
        ce[w] = __popc(ends);
    }
}
__global__ void k_runwrite(const uint32_t* bits, long long nwords, const unsigned long long* os,
                           const unsigned long long* oe, uint64_t base, uint64_t* out) {
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        uint32_t m = bits[w];
        uint32_t prev = w > 0 ? bits[w - 1] >> 31 : 0u;
        uint32_t next = w + 1 < nwords ? bits[w + 1] & 1u : 0u;
        uint32_t starts = m & ~((m << 1) | prev);
        uint32_t ends = m & ~((m >> 1) | (next << 31));
        unsigned long long k = os[w];
        while (starts) {
            int b = __ffs(starts) - 1;
            starts &= starts - 1;
            out[2 * k++] = base + (uint64_t)w * 32 + b;
        }
        k = oe[w];
        while (ends) {
            int b = __ffs(ends) - 1;
            ends &= ends - 1;
            out[2 * k++ + 1] = base + (uint64_t)w * 32 + b;
        }
    }
}
__global__ void k_widen(const uint32_t* a, unsigned long long* b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i];
}

static unsigned int grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned int)(g < 148 * 32 ? (g < 1 ? 1 : g) : 148 * 32);
}

__global__ void k_addc(unsigned long long* a, long long n, unsigned long long c) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] += c;
}

/* exclusive prefix sums of two u32 count arrays into u64 offsets, in chunks
 * of 2^30 items (cub's item count is an int) with carried totals */
static cudaError_t scan2(uint32_t* cs, uint32_t* ce, unsigned long long* os, unsigned long long* oe, long long n,
                         cudaStream_t s, unsigned long long* ts, unsigned long long* te) {
    cudaError_t e = cudaSuccess;
    const long long CH = 1ll << 30;
    k_widen<<<grid_for(n), 256, 0, s>>>(cs, os, n);
    k_widen<<<grid_for(n), 256, 0, s>>>(ce, oe, n);
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, os, os, (int)(n < CH ? n : CH), s);
    void* d_tmp = nullptr;
    if ((e = cudaMalloc(&d_tmp, tmp + 16)) != cudaSuccess) return e;
    unsigned long long carry[2] = {0, 0};
    unsigned long long* h = nullptr;
    if ((e = cudaMallocHost(&h, 4 * 8)) != cudaSuccess) { cudaFree(d_tmp); return e; }
    for (long long o = 0; o < n && e == cudaSuccess; o += CH) {
        int m = (int)(n - o < CH ? n - o : CH);
        cudaMemcpyAsync(h + 0, os + o + m - 1, 8, cudaMemcpyDeviceToHost, s);   /* last counts */
        cudaMemcpyAsync(h + 1, oe + o + m - 1, 8, cudaMemcpyDeviceToHost, s);
        cub::DeviceScan::ExclusiveSum(d_tmp, tmp, os + o, os + o, m, s);
        cub::DeviceScan::ExclusiveSum(d_tmp, tmp, oe + o, oe + o, m, s);
        cudaMemcpyAsync(h + 2, os + o + m - 1, 8, cudaMemcpyDeviceToHost, s);   /* last offsets */
        cudaMemcpyAsync(h + 3, oe + o + m - 1, 8, cudaMemcpyDeviceToHost, s);
        if (carry[0]) k_addc<<<grid_for(m), 256, 0, s>>>(os + o, m, carry[0]);
        if (carry[1]) k_addc<<<grid_for(m), 256, 0, s>>>(oe + o, m, carry[1]);
        e = cudaStreamSynchronize(s);
        carry[0] += h[2] + h[0];
        carry[1] += h[3] + h[1];
    }
    cudaFree(d_tmp);
    cudaFreeHost(h);
    *ts = carry[0];
    *te = carry[1];
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

/* bitmask -> device range array of the level; returns words (2 * runs) */
static vt_status encode(const uint32_t* bits, long long nwords, uint64_t base, cudaStream_t s, uint64_t** out,
                        long long* nout) {
    vt_status st = VT_OK;
    uint32_t *cs = nullptr, *ce = nullptr;
    unsigned long long *os = nullptr, *oe = nullptr;
    unsigned long long ts = 0, te = 0;
    *out = nullptr;
    *nout = 0;
    CKB(cudaMalloc(&cs, nwords * 4));
    CKB(cudaMalloc(&ce, nwords * 4));
    CKB(cudaMalloc(&os, nwords * 8));
    CKB(cudaMalloc(&oe, nwords * 8));
    k_runcount<<<grid_for(nwords), 256, 0, s>>>(bits, nwords, cs, ce);
    CKB(cudaGetLastError());
    CKB(scan2(cs, ce, os, oe, nwords, s, &ts, &te));
    if (ts != te) { st = vtrt::fail(VT_ERR_STATE, "run encoding mismatch (%llu starts, %llu ends)", ts, te); goto done; }
    if (2 * ts > 0x7FFFFFFFull) { st = vtrt::fail(VT_ERR_UNSUPPORTED, "level with %llu ranges exceeds the file format", ts); goto done; }
    if (ts) {
        CKB(cudaMalloc(out, 2 * ts * 8));
        k_runwrite<<<grid_for(nwords), 256, 0, s>>>(bits, nwords, os, oe, base, *out);
        CKB(cudaGetLastError());
    }
    *nout = (long long)(2 * ts);
done:
    cudaFree(cs); cudaFree(ce); cudaFree(os); cudaFree(oe);
    return st;
}

}  // namespace vtb

using namespace vtb;

extern "C" vt_status vt_octree_build_device(const void* dev_vol, int vtype, const int64_t dims[3], float iso,
                                            const char* out_path, void* stream) {
    vtrt::clear_error();
    if (!dev_vol || !dims || !out_path) return vtrt::fail(VT_ERR_INVALID, "vt_octree_build_device: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    vt_status st = VT_OK;
    /* nLevels exactly as the reference computes it (src/CreateOctree.cu:308-319) */
    int rd[3] = {(int)dims[0], (int)dims[1], (int)dims[2]};
    int dimension;
    if (rd[0] > rd[1] && rd[0] > rd[2]) dimension = rd[0];
    else if (rd[1] > rd[2]) dimension = rd[1];
    else dimension = rd[2];
    float aux = logf((float)dimension) / logf(2.0);
    float aux2 = aux - floorf(aux);
    int nLevels = aux2 > 0.0 ? (int)(aux + 1) : (int)aux;
    dimension = (int)pow(2, nLevels);
    if (nLevels < 1 || nLevels > 13) return vtrt::fail(VT_ERR_UNSUPPORTED, "volume extent gives %d levels", nLevels);
    std::vector<std::vector<uint64_t> > levels(nLevels + 1);
    uint32_t* childBits = nullptr;
    uint64_t* childRanges = nullptr;
    long long childN = 0;
    {
        const long long ncell = 1ll << (3 * nLevels);
        const long long nwords = (ncell + 31) / 32;
        CKB(cudaMalloc(&childBits, nwords * 4));
        if (vtype == VT_U8) k_leaf<1><<<grid_for(nwords), 256, 0, s>>>(dev_vol, dims[0], dims[1], dims[2], iso, childBits, nwords);
        else k_leaf<0><<<grid_for(nwords), 256, 0, s>>>(dev_vol, dims[0], dims[1], dims[2], iso, childBits, nwords);
        CKB(cudaGetLastError());
        if ((st = encode(childBits, nwords, 1ull << (3 * nLevels), s, &childRanges, &childN)) != VT_OK) goto done;
        levels[nLevels].resize(childN);
        if (childN) CKB(cudaMemcpyAsync(levels[nLevels].data(), childRanges, childN * 8, cudaMemcpyDeviceToHost, s));
        CKB(cudaStreamSynchronize(s));
    }
    for (int l = nLevels - 1; l >= 1; l--) {
        const long long np = 1ll << (3 * l);
        const long long nwords = (np + 31) / 32;
        uint32_t* bits = nullptr;
        uint64_t* ranges = nullptr;
        long long n = 0;
        CKB(cudaMalloc(&bits, nwords * 4));
        k_inner<<<grid_for(nwords), 256, 0, s>>>(childBits, childRanges, childN, 1ull << (3 * l), (uint64_t)(np - 1),
                                                 bits, nwords, np);
        CKB(cudaGetLastError());
        st = encode(bits, nwords, 1ull << (3 * l), s, &ranges, &n);
        cudaFree(childBits);
        cudaFree(childRanges);
        childBits = bits;
        childRanges = ranges;
        childN = n;
        if (st != VT_OK) goto done;
        levels[l].resize(n);
        if (n) CKB(cudaMemcpyAsync(levels[l].data(), ranges, n * 8, cudaMemcpyDeviceToHost, s));
        CKB(cudaStreamSynchronize(s));
    }
    /* root (src/CreateOctree.cu:532-540) */
    if (vtsearch::search_children_host(levels[1].data(), (int64_t)levels[1].size(), 1ull) > 0) levels[0] = {1ull, 1ull};
    {
        FILE* f = fopen(out_path, "wb");
        if (!f) { st = vtrt::fail(VT_ERR_IO, "unable to write %s", out_path); goto done; }
        int magic = 919278872;
        bool ok = fwrite(&magic, 4, 1, f) == 1 && fwrite(&iso, 4, 1, f) == 1 && fwrite(&dimension, 4, 1, f) == 1 &&
                  fwrite(rd, 4, 3, f) == 3 && fwrite(&nLevels, 4, 1, f) == 1;
        for (int l = nLevels; ok && l >= 0; l--) {
            int n = (int)levels[l].size();
            ok = fwrite(&n, 4, 1, f) == 1 && (n == 0 || fwrite(levels[l].data(), 8, (size_t)n, f) == (size_t)n);
        }
        if (fclose(f) != 0) ok = false;
        if (!ok) st = vtrt::fail(VT_ERR_IO, "short write to %s", out_path);
    }
done:
    cudaFree(childBits);
    cudaFree(childRanges);
    return st;
}

extern "C" vt_status vt_octree_build(const vt_volume* v, float iso, const char* out_path, void* stream) {
    vtrt::clear_error();
    if (!v || !out_path) return vtrt::fail(VT_ERR_INVALID, "vt_octree_build: null argument");
    if (!v->data) return vtrt::fail(VT_ERR_UNSUPPORTED, "vt_octree_build: the volume is read through a function");
    size_t bytes = v->voxels() * v->esize();
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return vtrt::fail(VT_ERR_NOMEM, "octree build: %s", cudaGetErrorString(e));
    e = cudaMemcpy(d, v->data, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(d); return vtrt::fail(VT_ERR_CUDA, "octree build upload: %s", cudaGetErrorString(e)); }
    vt_status st = vt_octree_build_device(d, v->vtype, v->dims, iso, out_path, stream);
    cudaFree(d);
    return st;
}
