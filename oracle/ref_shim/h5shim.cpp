/*
 * h5shim.cpp -- implementation of the hdf5.h stand-in (test infrastructure
 * for building the reference into oracle/_ref/).  Raw volume files only:
 * 64-byte header "VTVOL001", u32 version (1), u32 voxel type (0 = float32),
 * i64 dims[3], u64 data offset, then voxels with z fastest.
 */
#include "hdf5.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

namespace {
struct Space { int rank; hsize_t dims[3]; hsize_t start[3]; hsize_t count[3]; bool sel; };
struct File { FILE* f; std::string name; bool write; };
struct Dset { hid_t file; hsize_t dims[3]; uint64_t off; };
std::map<hid_t, File> g_files;
std::map<hid_t, Dset> g_dsets;
std::map<hid_t, Space> g_spaces;
hid_t g_next = 100;

bool read_header(FILE* f, hsize_t dims[3], uint64_t* off) {
    unsigned char h[64];
    if (fseek(f, 0, SEEK_SET) != 0 || fread(h, 1, 64, f) != 64) return false;
    if (memcmp(h, "VTVOL001", 8) != 0) return false;
    uint32_t vtype; memcpy(&vtype, h + 12, 4);
    if (vtype != 0) return false;
    int64_t d[3]; memcpy(d, h + 16, 24);
    memcpy(off, h + 40, 8);
    for (int i = 0; i < 3; i++) dims[i] = (hsize_t)d[i];
    return true;
}
}  // namespace

extern "C" hid_t H5Fopen(const char* name, unsigned, hid_t) {
    FILE* f = fopen(name, "rb");
    if (!f) return -1;
    hid_t id = g_next++;
    g_files[id] = File{f, name, false};
    return id;
}
extern "C" hid_t H5Fcreate(const char* name, unsigned, hid_t, hid_t) {
    FILE* f = fopen(name, "wb");
    if (!f) return -1;
    hid_t id = g_next++;
    g_files[id] = File{f, name, true};
    return id;
}
extern "C" herr_t H5Fclose(hid_t id) {
    std::map<hid_t, File>::iterator it = g_files.find(id);
    if (it == g_files.end()) return -1;
    fclose(it->second.f);
    g_files.erase(it);
    return 0;
}
extern "C" hid_t H5Dopen1(hid_t fid, const char*) {
    std::map<hid_t, File>::iterator it = g_files.find(fid);
    if (it == g_files.end()) return -1;
    Dset d; d.file = fid;
    if (!read_header(it->second.f, d.dims, &d.off)) return -1;
    hid_t id = g_next++;
    g_dsets[id] = d;
    return id;
}
extern "C" hid_t H5Dget_space(hid_t did) {
    std::map<hid_t, Dset>::iterator it = g_dsets.find(did);
    if (it == g_dsets.end()) return -1;
    Space s; s.rank = 3; s.sel = false;
    for (int i = 0; i < 3; i++) { s.dims[i] = it->second.dims[i]; s.start[i] = 0; s.count[i] = s.dims[i]; }
    hid_t id = g_next++;
    g_spaces[id] = s;
    return id;
}
extern "C" herr_t H5Dclose(hid_t did) { return g_dsets.erase(did) ? 0 : -1; }
extern "C" int H5Sget_simple_extent_dims(hid_t sid, hsize_t dims[], hsize_t maxdims[]) {
    std::map<hid_t, Space>::iterator it = g_spaces.find(sid);
    if (it == g_spaces.end()) return -1;
    for (int i = 0; i < it->second.rank; i++) {
        dims[i] = it->second.dims[i];
        if (maxdims) maxdims[i] = it->second.dims[i];
    }
    return it->second.rank;
}
extern "C" herr_t H5Sselect_hyperslab(hid_t sid, H5S_seloper_t, const hsize_t start[], const hsize_t*,
                                      const hsize_t count[], const hsize_t*) {
    std::map<hid_t, Space>::iterator it = g_spaces.find(sid);
    if (it == g_spaces.end()) return -1;
    for (int i = 0; i < 3; i++) {
        if (start[i] + count[i] > it->second.dims[i]) return -1;
        it->second.start[i] = start[i]; it->second.count[i] = count[i];
    }
    it->second.sel = true;
    return 0;
}
extern "C" hid_t H5Screate_simple(int rank, const hsize_t dims[], const hsize_t*) {
    if (rank != 3) return -1;
    Space s; s.rank = 3; s.sel = false;
    for (int i = 0; i < 3; i++) { s.dims[i] = dims[i]; s.start[i] = 0; s.count[i] = dims[i]; }
    hid_t id = g_next++;
    g_spaces[id] = s;
    return id;
}
extern "C" herr_t H5Sclose(hid_t sid) { return g_spaces.erase(sid) ? 0 : -1; }
extern "C" herr_t H5Dread(hid_t did, hid_t, hid_t msid, hid_t fsid, hid_t, void* buf) {
    std::map<hid_t, Dset>::iterator d = g_dsets.find(did);
    if (d == g_dsets.end()) return -1;
    FILE* f = g_files[d->second.file].f;
    const hsize_t* D = d->second.dims;
    Space fs, ms;
    if (fsid == H5S_ALL || !g_spaces.count(fsid)) {
        fs.rank = 3; for (int i = 0; i < 3; i++) { fs.dims[i] = D[i]; fs.start[i] = 0; fs.count[i] = D[i]; }
    } else fs = g_spaces[fsid];
    if (msid == H5S_ALL || !g_spaces.count(msid)) ms = fs;
    else ms = g_spaces[msid];
    for (int i = 0; i < 3; i++) if (fs.count[i] != ms.count[i]) return -1;
    std::vector<float> row(fs.count[2]);
    float* out = (float*)buf;
    for (hsize_t a = 0; a < fs.count[0]; a++)
        for (hsize_t b = 0; b < fs.count[1]; b++) {
            uint64_t src = ((fs.start[0] + a) * D[1] + (fs.start[1] + b)) * D[2] + fs.start[2];
            if (fseek(f, (long)(d->second.off + src * 4), SEEK_SET) != 0) return -1;
            if (fread(row.data(), 4, fs.count[2], f) != fs.count[2]) return -1;
            uint64_t dst = ((ms.start[0] + a) * ms.dims[1] + (ms.start[1] + b)) * ms.dims[2] + ms.start[2];
            memcpy(out + dst, row.data(), fs.count[2] * 4);
        }
    return 0;
}
extern "C" hid_t H5Tcopy(hid_t t) { return t; }
extern "C" herr_t H5Tset_order(hid_t, H5T_order_t) { return 0; }
extern "C" herr_t H5Tclose(hid_t) { return 0; }
extern "C" hid_t H5Dcreate2(hid_t fid, const char*, hid_t, hid_t sid, hid_t, hid_t, hid_t) {
    std::map<hid_t, File>::iterator it = g_files.find(fid);
    if (it == g_files.end() || !g_spaces.count(sid)) return -1;
    Dset d; d.file = fid; d.off = 64;
    for (int i = 0; i < 3; i++) d.dims[i] = g_spaces[sid].dims[i];
    unsigned char h[64]; memset(h, 0, 64);
    memcpy(h, "VTVOL001", 8);
    uint32_t ver = 1, vt = 0; memcpy(h + 8, &ver, 4); memcpy(h + 12, &vt, 4);
    int64_t dd[3] = {(int64_t)d.dims[0], (int64_t)d.dims[1], (int64_t)d.dims[2]};
    memcpy(h + 16, dd, 24); memcpy(h + 40, &d.off, 8);
    fwrite(h, 1, 64, it->second.f);
    hid_t id = g_next++;
    g_dsets[id] = d;
    return id;
}
extern "C" herr_t H5Dwrite(hid_t did, hid_t, hid_t, hid_t, hid_t, const void* buf) {
    std::map<hid_t, Dset>::iterator d = g_dsets.find(did);
    if (d == g_dsets.end()) return -1;
    FILE* f = g_files[d->second.file].f;
    uint64_t n = d->second.dims[0] * d->second.dims[1] * d->second.dims[2];
    fseek(f, (long)d->second.off, SEEK_SET);
    return fwrite(buf, 4, n, f) == n ? 0 : -1;
}
