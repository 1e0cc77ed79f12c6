/*
 * octree.cpp -- octree file I/O (class Octree, src/Octree.cu:769-813) and the
 * host entry points of the range searches in vt_search.h.
 */
#include <stdio.h>
#include <string.h>

#include <fstream>

#include "vt_runtime.h"
#include "vt_search.h"

namespace vtrt {
int children_mask(const uint64_t* e, int n, uint64_t father) { return vtsearch::children_mask_device(e, n, father); }
int search_children_host(const uint64_t* e, int64_t n, uint64_t father) {
    return vtsearch::search_children_host(e, n, father);
}
}  // namespace vtrt

using namespace vtrt;

extern "C" vt_status vt_octree_load(const char* path, vt_octree** out) {
    clear_error();
    if (!path || !out) return fail(VT_ERR_INVALID, "vt_octree_load: null argument");
    std::ifstream f(path, std::ifstream::binary);
    if (!f) return fail(VT_ERR_IO, "unable to open octree file %s", path);
    int magic = 0;
    f.read((char*)&magic, 4);
    if (!f || magic != 919278872) return fail(VT_ERR_FORMAT, "Error, invalid file format: %s", path);
    vt_octree* o = new vt_octree();
    f.read((char*)&o->iso, 4);
    f.read((char*)&o->dimension, 4);
    f.read((char*)o->realDim, 12);
    f.read((char*)&o->nLevels, 4);
    if (!f || o->nLevels < 1 || o->nLevels > 19) { delete o; return fail(VT_ERR_FORMAT, "bad octree header: %s", path); }
    o->levels.resize(o->nLevels + 1);
    for (int l = o->nLevels; l >= 0; l--) {
        int n = 0;
        f.read((char*)&n, 4);
        if (!f || n < 0 || (n & 1)) { delete o; return fail(VT_ERR_FORMAT, "bad level %d size in %s", l, path); }
        o->levels[l].resize(n);
        if (n) f.read((char*)o->levels[l].data(), (std::streamsize)n * 8);
        if (!f) { delete o; return fail(VT_ERR_FORMAT, "truncated octree %s", path); }
    }
    *out = o;
    return VT_OK;
}

extern "C" void vt_octree_free(vt_octree* o) { delete o; }

extern "C" vt_status vt_octree_info(const vt_octree* o, float* iso, int* dimension, int realDim[3], int* nLevels) {
    clear_error();
    if (!o) return fail(VT_ERR_INVALID, "null octree");
    if (iso) *iso = o->iso;
    if (dimension) *dimension = o->dimension;
    if (realDim) memcpy(realDim, o->realDim, 12);
    if (nLevels) *nLevels = o->nLevels;
    return VT_OK;
}

extern "C" vt_status vt_octree_level(const vt_octree* o, int level, int64_t* n, uint64_t* words) {
    clear_error();
    if (!o || level < 0 || level > o->nLevels) return fail(VT_ERR_INVALID, "bad octree level %d", level);
    if (n) *n = (int64_t)o->levels[level].size();
    if (words && !o->levels[level].empty()) memcpy(words, o->levels[level].data(), o->levels[level].size() * 8);
    return VT_OK;
}
