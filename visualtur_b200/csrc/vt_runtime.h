/*
 * vt_runtime.h -- internal host-side declarations of libvt.so.
 */
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/vt.h"

namespace vtrt {

/* Thread-local error message + status helper. */
vt_status fail(vt_status s, const char* fmt, ...);
void clear_error();

/* splitmix64 (Steele, Lea, Flood 2014): the counter-based generator behind
 * every seeded volume, identical on host and device. */
inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace vtrt

/* Host volume: memory-mapped file, wrapped caller memory or owned buffer. */
struct vt_volume {
    int vtype = VT_F32;
    int64_t dims[3] = {0, 0, 0};
    const unsigned char* data = nullptr;   /* first voxel */
    void* map_base = nullptr;
    size_t map_len = 0;
    std::vector<unsigned char> owned;
    std::string path;
    vt_read_fn reader = nullptr;           /* caller's read function (no voxels in memory) */
    void* user = nullptr;
    size_t esize() const { return vtype == VT_U8 ? 1 : 4; }
    size_t voxels() const { return (size_t)dims[0] * dims[1] * dims[2]; }
};

/* Octree as stored in the file (levels 0..nLevels of sorted inclusive
 * Morton ranges). */
struct vt_octree {
    float iso = 0;
    int dimension = 0;
    int realDim[3] = {0, 0, 0};
    int nLevels = 0;
    std::vector<std::vector<uint64_t> > levels;
};

namespace vtrt {
/* zero-padded hyperslab read, float32 output (FileManager semantics);
 * false when a reader-backed volume's read failed */
bool volume_read(const vt_volume* v, const int s[3], const int e[3], float* out);
/* same, native voxel type, into a buffer of (e-s) voxels */
bool volume_read_native(const vt_volume* v, const int s[3], const int e[3], void* out);
/* copies `bytes` (a multiple of 16) to a 16-byte aligned `dst` with stores
 * that bypass the caches (the destination is not read first); the calling
 * thread ends its run of such copies with stream_fence() */
void stream_copy(void* dst, const void* src, size_t bytes);
void stream_fence();
/* the same for any alignment and size (the unaligned head and tail by
 * ordinary stores) */
void stream_copy_any(void* dst, const void* src, size_t bytes);
/* reference device-variant child membership (src/Octree.cu:375-532) */
int children_mask(const uint64_t* e, int size, uint64_t father);
/* reference host-variant child count (src/CreateOctree.cu:247-284) */
int search_children_host(const uint64_t* e, int64_t size, uint64_t father);
/* h5lite: a dataset of an HDF5 file as stored */
struct H5Dataset {
    int rank = 0;
    int64_t dims[32] = {0};
    int type_class = -1;        /* 0 fixed point, 1 IEEE float */
    int type_size = 0;          /* bytes per element */
    bool is_signed = false, big_endian = false;
    uint64_t offset = 0;        /* file offset of element 0 */
    uint64_t bytes = 0;         /* storage size */
    bool offset_is_addr = false;
};
bool h5_describe(const unsigned char* file, size_t len, const char* path, H5Dataset* d, std::string* why);
bool h5_write(const char* path, const char* dataset, const void* data, int vtype, const int64_t dims[3],
              std::string* why);
}  // namespace vtrt
