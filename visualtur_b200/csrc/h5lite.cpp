/*
 * h5lite.cpp -- HDF5 container support for volume files, written from the
 * published HDF5 file-format specification (libhdf5 is not linked).
 *
 * The reference reads its volume with libhdf5: one 3-D dataset, hyperslab
 * reads converted to H5T_IEEE_F32LE (src/FileManager.cu:13-167), and
 * writes one with FileManager::CreateFile (:169-243).  libvt memory-maps the
 * file and needs the dataset's raw bytes in one piece, so the reader here
 * accepts:
 *   - superblock versions 0-3, at offset 0 or after a user block (512,
 *     1024, ... bytes, as MATLAB v7.3 files have);
 *   - groups stored as a symbol table (v1 B-tree + local heap) or as compact
 *     link messages; a dataset path may name nested groups;
 *   - object headers version 1 and 2, with continuation chunks;
 *   - dataspace versions 1-2, datatype classes fixed-point and IEEE float,
 *     layout versions 1-4, contiguous or compact storage.
 * Chunked or filtered storage, external files, dense (fractal-heap) groups
 * and big-endian data are reported as unsupported.
 *
 * The writer produces the layout libhdf5 itself writes with its default
 * ("earliest") format: superblock 0, root group with a symbol table, the
 * dataset's object header version 1 with dataspace, datatype, fill value and
 * contiguous layout messages, and the voxels at a 512-byte aligned offset.
 */
#include <stdio.h>
#include <string.h>

#include <functional>
#include <string>
#include <vector>

#include "vt_runtime.h"

namespace vtrt {
namespace {

const uint64_t kUndef = ~0ull;
const unsigned char kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

struct Reader {
    const unsigned char* p;
    size_t len;
    uint64_t base = 0;      /* addresses are relative to the base address */
    int so = 8, sl = 8;     /* sizes of offsets and lengths */
    std::string* why;

    bool fail(const char* msg) const { *why = msg; return false; }
    bool in(uint64_t off, uint64_t n) const { return off <= len && n <= len - off; }
    uint64_t u(uint64_t off, int n) const {
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)p[off + i] << (8 * i);
        return v;
    }
    bool undef(uint64_t a) const { return so == 8 ? a == kUndef : a == ((1ull << (8 * so)) - 1); }
    /* file offset of address a */
    uint64_t at(uint64_t a) const { return a + base; }
};

/* Calls fn(type, data offset, data size) for every message of the object
 * header at `addr`; fn returns false to stop early (then true is returned). */
bool for_messages(Reader& r, uint64_t addr, const std::function<bool(int, uint64_t, uint64_t)>& fn) {
    uint64_t a = r.at(addr);
    struct Chunk { uint64_t off, len; bool v2; };
    std::vector<Chunk> chunks;
    int version;
    int creationOrder = 0;
    if (r.in(a, 4) && memcmp(r.p + a, "OHDR", 4) == 0) {
        if (!r.in(a, 16)) return r.fail("truncated object header");
        version = r.p[a + 4];
        if (version != 2) return r.fail("unknown object header version");
        int flags = r.p[a + 5];
        uint64_t q = a + 6;
        if (flags & 0x20) q += 16;
        if (flags & 0x10) q += 4;
        int w = 1 << (flags & 3);
        if (!r.in(q, (uint64_t)w)) return r.fail("truncated object header");
        uint64_t size0 = r.u(q, w);
        q += (uint64_t)w;
        creationOrder = (flags & 0x04) ? 2 : 0;
        chunks.push_back({q, size0, true});
    } else {
        if (!r.in(a, 16)) return r.fail("truncated object header");
        version = r.p[a];
        if (version != 1) return r.fail("unknown object header version");
        chunks.push_back({a + 16, r.u(a + 8, 4), false});
    }
    for (size_t c = 0; c < chunks.size() && c < 4096; c++) {
        Chunk ch = chunks[c];
        if (!r.in(ch.off, ch.len)) return r.fail("object header chunk outside the file");
        uint64_t q = ch.off, end = ch.off + ch.len;
        const uint64_t hdr = ch.v2 ? 4u + creationOrder : 8u;
        while (q + hdr <= end) {
            int type;
            uint64_t size;
            if (ch.v2) { type = r.p[q]; size = r.u(q + 1, 2); }
            else { type = (int)r.u(q, 2); size = r.u(q + 2, 2); }
            uint64_t d = q + hdr;
            if (d + size > end) return r.fail("object header message overruns its chunk");
            if (type == 0x10) {   /* continuation: address, length */
                if (size < (uint64_t)(r.so + r.sl)) return r.fail("bad continuation message");
                uint64_t ca = r.u(d, r.so), cl = r.u(d + r.so, r.sl);
                uint64_t co = r.at(ca);
                if (ch.v2) {
                    if (cl < 8 || !r.in(co, 8) || memcmp(r.p + co, "OCHK", 4) != 0) return r.fail("bad continuation chunk");
                    chunks.push_back({co + 4, cl - 8, true});
                } else {
                    chunks.push_back({co, cl, false});
                }
            } else if (!fn(type, d, size)) {
                return true;
            }
            q = d + size;
        }
    }
    return true;
}

/* v1 B-tree (group nodes) under `node`: looks `name` up in the symbol table
 * nodes, names stored in the local heap data segment at `heap`. */
bool btree_lookup(Reader& r, uint64_t node, uint64_t heap, uint64_t heapSize, const std::string& name,
                  uint64_t* obj, int depth) {
    if (depth > 32) return r.fail("group B-tree too deep");
    uint64_t a = r.at(node);
    if (!r.in(a, 8 + 2 * (uint64_t)r.so) || memcmp(r.p + a, "TREE", 4) != 0) return r.fail("bad group B-tree node");
    if (r.p[a + 4] != 0) return r.fail("not a group B-tree");
    int level = r.p[a + 5];
    uint64_t used = r.u(a + 6, 2);
    uint64_t q = a + 8 + 2 * (uint64_t)r.so;   /* key0 */
    for (uint64_t i = 0; i < used; i++) {
        uint64_t childPos = q + (uint64_t)r.sl + i * (uint64_t)(r.sl + r.so);
        if (!r.in(childPos, (uint64_t)r.so)) return r.fail("truncated group B-tree node");
        uint64_t child = r.u(childPos, r.so);
        if (level > 0) {
            if (btree_lookup(r, child, heap, heapSize, name, obj, depth + 1)) return true;
            if (r.why->size()) return false;
            continue;
        }
        uint64_t s = r.at(child);
        if (!r.in(s, 8) || memcmp(r.p + s, "SNOD", 4) != 0) return r.fail("bad symbol table node");
        uint64_t nsym = r.u(s + 6, 2);
        uint64_t esz = 2 * (uint64_t)r.so + 24;
        if (!r.in(s + 8, nsym * esz)) return r.fail("truncated symbol table node");
        for (uint64_t k = 0; k < nsym; k++) {
            uint64_t e = s + 8 + k * esz;
            uint64_t nameOff = r.u(e, r.so);
            if (nameOff >= heapSize) return r.fail("symbol name outside the local heap");
            const char* nm = (const char*)r.p + heap + nameOff;
            size_t maxn = (size_t)(heapSize - nameOff);
            if (strnlen(nm, maxn) == name.size() && memcmp(nm, name.data(), name.size()) == 0) {
                *obj = r.u(e + r.so, r.so);
                return true;
            }
        }
    }
    return false;
}

/* Object header address of the member `name` of the group at `grp`. */
bool group_member(Reader& r, uint64_t grp, const std::string& name, uint64_t* obj) {
    bool found = false, symtab = false, dense = false;
    uint64_t bt = 0, hp = 0;
    bool ok = for_messages(r, grp, [&](int type, uint64_t d, uint64_t size) {
        if (type == 0x11 && size >= 2 * (uint64_t)r.so) {          /* symbol table */
            symtab = true; bt = r.u(d, r.so); hp = r.u(d + r.so, r.so);
        } else if (type == 0x02 && size >= 2 + 8 + 2 * (uint64_t)r.so) { /* link info */
            int flags = r.p[d + 1];
            uint64_t fh = r.u(d + 2 + ((flags & 1) ? 8 : 0), r.so);
            if (!r.undef(fh)) dense = true;
        } else if (type == 0x06 && size >= 3) {                   /* link */
            int flags = r.p[d + 1];
            uint64_t q = d + 2;
            int ltype = 0;
            if (flags & 0x08) ltype = r.p[q++];
            if (flags & 0x04) q += 8;
            if (flags & 0x10) q++;
            int w = 1 << (flags & 3);
            if (q + (uint64_t)w > d + size) return true;
            uint64_t nlen = r.u(q, w);
            q += (uint64_t)w;
            if (q + nlen + (uint64_t)r.so > d + size) return true;
            if (ltype == 0 && nlen == name.size() && memcmp(r.p + q, name.data(), nlen) == 0) {
                *obj = r.u(q + nlen, r.so);
                found = true;
                return false;
            }
        }
        return true;
    });
    if (!ok) return false;
    if (found) return true;
    if (symtab) {
        uint64_t h = r.at(hp);
        if (!r.in(h, 8 + 2 * (uint64_t)r.sl + r.so) || memcmp(r.p + h, "HEAP", 4) != 0) return r.fail("bad local heap");
        uint64_t hsize = r.u(h + 8, r.sl);
        uint64_t hdata = r.at(r.u(h + 8 + 2 * (uint64_t)r.sl, r.so));
        if (!r.in(hdata, hsize)) return r.fail("local heap outside the file");
        r.why->clear();
        if (btree_lookup(r, bt, hdata, hsize, name, obj, 0)) return true;
        if (!r.why->empty()) return false;
    }
    if (dense) return r.fail("groups with dense (fractal heap) link storage are not supported");
    std::string m = "no member \"" + name + "\" in the group";
    *r.why = m;
    return false;
}

}  // namespace

bool h5_describe(const unsigned char* file, size_t len, const char* path, H5Dataset* ds, std::string* why) {
    why->clear();
    Reader r{file, len};
    r.why = why;
    /* superblock: offset 0, then 512, 1024, 2048, ... */
    uint64_t sb = kUndef;
    for (uint64_t o = 0; o + 8 <= len; o = o ? o * 2 : 512)
        if (memcmp(file + o, kSig, 8) == 0) { sb = o; break; }
    if (sb == kUndef) return r.fail("no HDF5 signature");
    if (!r.in(sb, 48)) return r.fail("truncated superblock");
    int sv = file[sb + 8];
    uint64_t root;
    if (sv == 0 || sv == 1) {
        r.so = file[sb + 13]; r.sl = file[sb + 14];
        uint64_t q = sb + 24 + (sv == 1 ? 4 : 0);
        if ((r.so != 4 && r.so != 8) || (r.sl != 4 && r.sl != 8)) return r.fail("unsupported offset/length size");
        if (!r.in(q, 4 * (uint64_t)r.so + 2 * (uint64_t)r.so + 8)) return r.fail("truncated superblock");
        r.base = r.u(q, r.so);
        root = r.u(q + 4 * (uint64_t)r.so + r.so, r.so);   /* root entry: name offset, header address */
    } else if (sv == 2 || sv == 3) {
        r.so = file[sb + 9]; r.sl = file[sb + 10];
        if ((r.so != 4 && r.so != 8) || (r.sl != 4 && r.sl != 8)) return r.fail("unsupported offset/length size");
        uint64_t q = sb + 12;
        if (!r.in(q, 4 * (uint64_t)r.so)) return r.fail("truncated superblock");
        r.base = r.u(q, r.so);
        root = r.u(q + 3 * (uint64_t)r.so, r.so);
    } else {
        return r.fail("unknown superblock version");
    }
    /* walk the path from the root group */
    std::string p = path ? path : "";
    uint64_t obj = root;
    size_t i = 0;
    while (i < p.size()) {
        size_t j = p.find('/', i);
        if (j == std::string::npos) j = p.size();
        if (j > i && !group_member(r, obj, p.substr(i, j - i), &obj)) return false;
        i = j + 1;
    }
    /* dataset messages */
    bool haveSpace = false, haveType = false, haveLayout = false, filtered = false, external = false;
    ds->rank = 0; ds->offset = kUndef; ds->bytes = 0;
    int layoutClass = -1;
    bool ok = for_messages(r, obj, [&](int type, uint64_t d, uint64_t size) {
        if (type == 0x01 && size >= 4) {                 /* dataspace */
            int v = file[d], rank = file[d + 1];
            uint64_t q = v == 1 ? d + 8 : d + 4;
            if (rank > 32 || q + (uint64_t)rank * r.sl > d + size) return true;
            ds->rank = rank;
            for (int k = 0; k < rank; k++) ds->dims[k] = (int64_t)r.u(q + (uint64_t)k * r.sl, r.sl);
            haveSpace = true;
        } else if (type == 0x03 && size >= 8) {          /* datatype */
            ds->type_class = file[d] & 0x0f;
            ds->type_size = (int)r.u(d + 4, 4);
            int b0 = file[d + 1];
            ds->big_endian = (b0 & 1) != 0 || (ds->type_class == 1 && (b0 & 0x40));
            ds->is_signed = ds->type_class == 0 ? (b0 & 0x08) != 0 : true;
            haveType = true;
        } else if (type == 0x08 && size >= 4) {          /* layout */
            int v = file[d];
            if (v == 3 || v == 4) {
                layoutClass = file[d + 1];
                if (layoutClass == 1 && size >= 2 + (uint64_t)(r.so + r.sl)) {
                    ds->offset = r.u(d + 2, r.so); ds->bytes = r.u(d + 2 + r.so, r.sl); ds->offset_is_addr = true;
                } else if (layoutClass == 0) {
                    ds->bytes = r.u(d + 2, 2); ds->offset = d + 4; ds->offset_is_addr = false;
                    if (4 + ds->bytes > size) return true;
                }
            } else if (v == 1 || v == 2) {
                int nd = file[d + 1];
                layoutClass = file[d + 2];
                if (layoutClass == 1 && size >= 8 + r.so + 4 * (uint64_t)nd) {
                    ds->offset = r.u(d + 8, r.so); ds->offset_is_addr = true;
                    uint64_t n = 1;   /* the last dimension is the element size */
                    for (int k = 0; k < nd; k++) n *= r.u(d + 8 + r.so + 4 * (uint64_t)k, 4);
                    ds->bytes = n;
                } else if (layoutClass == 0 && size >= 12 + 4 * (uint64_t)nd) {
                    uint64_t q = d + 8 + 4 * (uint64_t)nd;
                    ds->bytes = r.u(q, 4); ds->offset = q + 4; ds->offset_is_addr = false;
                    if (12 + 4 * (uint64_t)nd + ds->bytes > size) return true;
                }
            }
            haveLayout = true;
        } else if (type == 0x0b) {
            filtered = true;
        } else if (type == 0x07) {
            external = true;
        }
        return true;
    });
    if (!ok) return false;
    if (!haveSpace || !haveType || !haveLayout) return r.fail("object is not a dataset");
    if (external) return r.fail("datasets in external files are not supported");
    if (filtered || layoutClass == 2) return r.fail("chunked or filtered datasets are not supported");
    if (layoutClass != 0 && layoutClass != 1) return r.fail("unsupported dataset layout");
    if (ds->offset_is_addr) {
        if (r.undef(ds->offset)) return r.fail("dataset storage was never allocated");
        ds->offset = r.at(ds->offset);
        ds->offset_is_addr = false;
    }
    uint64_t n = 1;
    for (int k = 0; k < ds->rank; k++) n *= (uint64_t)ds->dims[k];
    if (n * (uint64_t)ds->type_size > ds->bytes || !r.in(ds->offset, n * (uint64_t)ds->type_size))
        return r.fail("dataset storage is truncated");
    return true;
}

namespace {
struct Writer {
    std::vector<unsigned char> b;
    void put(uint64_t v, int n) { for (int i = 0; i < n; i++) b.push_back((unsigned char)(v >> (8 * i))); }
    void bytes(const void* s, size_t n) { b.insert(b.end(), (const unsigned char*)s, (const unsigned char*)s + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad_to(size_t n) { if (b.size() < n) zeros(n - b.size()); }
    void set(size_t at, uint64_t v, int n) { for (int i = 0; i < n; i++) b[at + i] = (unsigned char)(v >> (8 * i)); }
    /* object header message, version 1 framing: data padded to 8 bytes */
    void msg(int type, int flags, const std::vector<unsigned char>& data) {
        size_t sz = (data.size() + 7) & ~(size_t)7;
        put((uint64_t)type, 2); put(sz, 2); put((uint64_t)flags, 1); zeros(3);
        bytes(data.data(), data.size());
        zeros(sz - data.size());
    }
};
std::vector<unsigned char> le(std::initializer_list<std::pair<uint64_t, int> > f) {
    std::vector<unsigned char> v;
    for (auto& x : f) for (int i = 0; i < x.second; i++) v.push_back((unsigned char)(x.first >> (8 * i)));
    return v;
}
}  // namespace

bool h5_write(const char* path, const char* dataset, const void* data, int vtype, const int64_t dims[3],
              std::string* why) {
    std::string name = dataset ? dataset : "value";
    while (!name.empty() && name[0] == '/') name.erase(0, 1);
    if (name.empty() || name.find('/') != std::string::npos) { *why = "dataset name must be one path component"; return false; }
    const int es = vtype == VT_U8 ? 1 : 4;
    const uint64_t nbytes = (uint64_t)dims[0] * dims[1] * dims[2] * es;
    Writer w;
    /* superblock 0 (96 bytes), patched below */
    const size_t A_ROOT = 96, A_BT = 136, A_HEAP = 680, A_HEAPDATA = 712;
    const size_t nameOff = 8, nameLen = (name.size() + 1 + 7) & ~(size_t)7;
    const size_t freeOff = nameOff + nameLen, heapSize = freeOff + 16;
    const size_t A_SNOD = A_HEAPDATA + heapSize;
    const size_t A_DSET = A_SNOD + 8 + 8 * 40;
    w.bytes(kSig, 8);
    w.put(0, 1); w.put(0, 1); w.put(0, 1); w.put(0, 1); w.put(0, 1);  /* versions, reserved */
    w.put(8, 1); w.put(8, 1); w.put(0, 1);                              /* offset/length sizes */
    w.put(4, 2); w.put(16, 2);                                          /* group leaf K, internal K */
    w.put(0, 4);                                                        /* consistency flags */
    w.put(0, 8); w.put(kUndef, 8);                                      /* base, free-space info */
    const size_t eofAt = w.b.size();
    w.put(0, 8); w.put(kUndef, 8);                                      /* EOF (patched), driver info */
    /* root group symbol table entry: cached B-tree and heap addresses */
    w.put(0, 8); w.put(A_ROOT, 8); w.put(1, 4); w.put(0, 4); w.put(A_BT, 8); w.put(A_HEAP, 8);
    /* root group object header: symbol table message */
    w.pad_to(A_ROOT);
    w.put(1, 1); w.put(0, 1); w.put(1, 2); w.put(1, 4); w.put(24, 4); w.zeros(4);
    w.msg(0x11, 1, le({{A_BT, 8}, {A_HEAP, 8}}));
    /* group B-tree: one leaf entry pointing at the symbol table node; room
     * for 2K = 32 children as the internal-node K above implies */
    w.pad_to(A_BT);
    w.bytes("TREE", 4); w.put(0, 1); w.put(0, 1); w.put(1, 2); w.put(kUndef, 8); w.put(kUndef, 8);
    w.put(0, 8); w.put(A_SNOD, 8); w.put(nameOff, 8);
    w.pad_to(A_BT + 24 + 32 * 8 + 33 * 8);
    /* local heap: "" at 0, the dataset name, then one free block whose
     * next-block offset 1 ends the free list */
    w.pad_to(A_HEAP);
    w.bytes("HEAP", 4); w.put(0, 1); w.zeros(3); w.put(heapSize, 8); w.put(freeOff, 8); w.put(A_HEAPDATA, 8);
    w.zeros(nameOff);
    w.bytes(name.data(), name.size()); w.zeros(nameLen - name.size());
    w.put(1, 8); w.put(16, 8);
    /* symbol table node: one entry (2K = 8 slots for leaf K 4) */
    w.pad_to(A_SNOD);
    w.bytes("SNOD", 4); w.put(1, 1); w.put(0, 1); w.put(1, 2);
    w.put(nameOff, 8); w.put(A_DSET, 8); w.put(0, 4); w.put(0, 4); w.zeros(16);
    w.pad_to(A_DSET);
    /* dataset object header */
    std::vector<unsigned char> space = le({{1, 1}, {3, 1}, {0, 1}, {0, 1}, {0, 4},
                                           {(uint64_t)dims[0], 8}, {(uint64_t)dims[1], 8}, {(uint64_t)dims[2], 8}});
    std::vector<unsigned char> dtype;
    if (vtype == VT_U8)   /* fixed point, unsigned, little-endian, 8 bits */
        dtype = le({{0x10, 1}, {0, 1}, {0, 1}, {0, 1}, {1, 4}, {0, 2}, {8, 2}});
    else                  /* IEEE single, little-endian, implied mantissa MSB */
        dtype = le({{0x11, 1}, {0x20, 1}, {31, 1}, {0, 1}, {4, 4}, {0, 2}, {32, 2}, {23, 1}, {8, 1}, {0, 1},
                    {23, 1}, {127, 4}});
    std::vector<unsigned char> fill = le({{2, 1}, {2, 1}, {2, 1}, {0, 1}});   /* v2, late, if set, undefined */
    const size_t msgBytes = (8 + 32) + (8 + ((dtype.size() + 7) & ~(size_t)7)) + (8 + 8) + (8 + 24);
    const size_t A_DATA = (A_DSET + 16 + msgBytes + 511) & ~(size_t)511;
    std::vector<unsigned char> layout = le({{3, 1}, {1, 1}, {A_DATA, 8}, {nbytes, 8}});
    w.put(1, 1); w.put(0, 1); w.put(4, 2); w.put(1, 4); w.put(msgBytes, 4); w.zeros(4);
    w.msg(0x01, 0, space);
    w.msg(0x03, 1, dtype);
    w.msg(0x05, 1, fill);
    w.msg(0x08, 0, layout);
    if (w.b.size() != A_DSET + 16 + msgBytes) { *why = "internal layout error"; return false; }
    w.pad_to(A_DATA);
    w.set(eofAt, A_DATA + nbytes, 8);
    FILE* f = fopen(path, "wb");
    if (!f) { *why = "cannot create the file"; return false; }
    bool ok = fwrite(w.b.data(), 1, w.b.size(), f) == w.b.size();
    const unsigned char* src = (const unsigned char*)data;
    for (uint64_t o = 0; ok && o < nbytes; o += (1u << 26)) {
        size_t n = (size_t)std::min<uint64_t>(1u << 26, nbytes - o);
        ok = fwrite(src + o, 1, n, f) == n;
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) *why = "write failed";
    return ok;
}

}  // namespace vtrt
