/*
 * cache.cu -- two-tier brick cache (see cache.h).
 *
 * Semantics kept from lruCache (src/lruCache.cu:168-313): a brick is the
 * zero-padded box [min - inc, min + edge + inc) of the volume, its id is
 * the candidate id shifted to the brick level (:177), the device tier is
 * filled from the host tier, the host tier from the volume, both evict the
 * least recently used entry, and admission per pass is capped by the tier
 * sizes (rays over the cap retry in the next pass, as NOCACHED rays do).
 * Unlike the reference, a slot handed out in a pass is never evicted within
 * that pass (the reference can, src/lruCache.cu:184,:256).
 */
#include <string.h>

#include <algorithm>
#include <chrono>
#include <numeric>

#include <omp.h>

#include "cache.h"
#include "vt_math.cuh"

namespace vtrt {

#define CKC(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(VT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

/* Warp-cooperative copy of n bytes through this warp's shared buffer
 * (kCopyBuf bytes): the source is read in aligned 16-byte words whatever
 * its alignment (loads from mapped host memory cross PCIe, so they must be
 * wide), four words in flight per lane; the destination is written in
 * 4-byte words assembled with byte permutes, bytes at its unaligned ends.
 * The aligned words may reach up to 15 bytes before and after the range:
 * every caller copies within a 16-byte aligned slot. */
constexpr int kCopyBuf = 2048;
__device__ __forceinline__ void warp_copy(unsigned char* dst, const unsigned char* src, size_t n, int lane,
                                          unsigned int* buf) {
    const int sa = (int)((size_t)src & 15);
    const uint4* s16 = (const uint4*)(src - sa);
    const size_t piece = kCopyBuf - 16;
    const unsigned char* sb = (const unsigned char*)buf;
    for (size_t b0 = 0; b0 < n; b0 += piece) {
        const int len = (int)min(piece, n - b0);
        const int words = (sa + len + 15) >> 4;
        const uint4* sw = s16 + (b0 >> 4);
        for (int i = lane; i < words; i += 128) {
            uint4 v0 = sw[i], v1, v2, v3;
            if (i + 32 < words) v1 = sw[i + 32];
            if (i + 64 < words) v2 = sw[i + 64];
            if (i + 96 < words) v3 = sw[i + 96];
            ((uint4*)buf)[i] = v0;
            if (i + 32 < words) ((uint4*)buf)[i + 32] = v1;
            if (i + 64 < words) ((uint4*)buf)[i + 64] = v2;
            if (i + 96 < words) ((uint4*)buf)[i + 96] = v3;
        }
        __syncwarp();
        unsigned char* d = dst + b0;
        const int head = min((int)((4 - ((size_t)d & 3)) & 3), len);
        if (lane < head) d[lane] = sb[sa + lane];
        const int nw = (len - head) >> 2;
        unsigned int* dw = (unsigned int*)(d + head);
        for (int j = lane; j < nw; j += 32) {
            const int p = sa + head + 4 * j;
            dw[j] = __byte_perm(buf[p >> 2], buf[(p >> 2) + 1], 0x3210 + 0x1111 * (p & 3));
        }
        const int t = head + 4 * nw;
        if (lane < len - t) d[t + lane] = sb[sa + t + lane];
        __syncwarp();
    }
}

/* Brick loads, one CTA per brick, in up to three launches on one stream:
 * phase 1 copies the parts the brick takes from the host tier (mapped
 * memory, packed by part) into its slot; phase 2 the y aprons from the y
 * neighbours' middles; phase 3 the x aprons from the x neighbours' planes,
 * which by then hold their own y aprons. */
__global__ void k_fill_split(const unsigned char* __restrict__ tier, const unsigned char* __restrict__ stage,
                             unsigned char* __restrict__ slab, TierGeo g, const SplitItem* __restrict__ items,
                             int phase) {
    __shared__ __align__(16) unsigned int cbuf[8][kCopyBuf / 4];
    const SplitItem it = items[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    unsigned int* const buf = cbuf[warp];
    const int e = g.e, inc = g.inc;
    unsigned char* dst = slab + (size_t)it.slot * g.slotBytes;
    const size_t row = (size_t)g.D * g.es, plane = (size_t)g.D * row;
    if (phase == 1) {
        const unsigned char* src = (it.staged ? stage : tier) + (size_t)it.hs * g.tierBytes;
        /* one chunk per plane of a part: [0, e) M, then inc X- planes, inc
         * X+ planes, e Y- and e Y+ plane pieces */
        for (int c = warp; c < 3 * e + 2 * inc; c += nwarps) {
            int b, q;
            size_t soff, doff, len;
            if (c < e) {
                b = 0; q = c;
                soff = g.off[0] + (size_t)q * e * row; doff = (size_t)(inc + q) * plane + (size_t)inc * row;
                len = (size_t)e * row;
            } else if (c < e + 2 * inc) {
                const bool lo = c < e + inc;
                b = lo ? 1 : 2; q = lo ? c - e : c - e - inc;
                soff = g.off[b] + (size_t)q * plane; doff = (size_t)(lo ? q : inc + e + q) * plane; len = plane;
            } else {
                const bool lo = c < 2 * e + 2 * inc;
                b = lo ? 3 : 4; q = lo ? c - e - 2 * inc : c - 2 * e - 2 * inc;
                soff = g.off[b] + (size_t)q * inc * row;
                doff = (size_t)(inc + q) * plane + (lo ? 0 : (size_t)(inc + e) * row);
                len = (size_t)inc * row;
            }
            if (it.parts & (1 << b)) warp_copy(dst + doff, src + soff, len, lane, buf);
        }
    } else if (phase == 2) {
        /* Y-: rows [0, inc) = the (y-1) neighbour's rows [e, e+inc); Y+: rows
         * [inc+e, D) = the (y+1) neighbour's rows [inc, 2 inc) */
        for (int c = warp; c < 2 * e; c += nwarps) {
            const bool lo = c < e;
            const int nb = it.nb[lo ? 2 : 3];
            if (nb < 0) continue;
            const int p = lo ? c : c - e;
            const size_t doff = (size_t)(inc + p) * plane + (lo ? 0 : (size_t)(inc + e) * row);
            const size_t soff = lo ? doff + (size_t)e * row : doff - (size_t)e * row;
            warp_copy(dst + doff, slab + (size_t)nb * g.slotBytes + soff, (size_t)inc * row, lane, buf);
        }
    } else {
        /* X-: planes [0, inc) = the (x-1) neighbour's planes [e, e+inc); X+:
         * planes [inc+e, D) = the (x+1) neighbour's planes [inc, 2 inc) */
        for (int c = warp; c < 2 * inc; c += nwarps) {
            const bool lo = c < inc;
            const int nb = it.nb[lo ? 0 : 1];
            if (nb < 0) continue;
            const int q = lo ? c : c - inc;
            const size_t doff = (size_t)(lo ? q : inc + e + q) * plane;
            const size_t soff = (size_t)(lo ? e + q : inc + q) * plane;
            warp_copy(dst + doff, slab + (size_t)nb * g.slotBytes + soff, plane, lane, buf);
        }
    }
}

/* page-table / stamp updates: x = page index, y = value; slot stamps for
 * loaded bricks */
__global__ void k_page_update(int* page, const int2* upd, int n, unsigned int* stamp, unsigned int stampValue) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int2 u = upd[i];
    page[u.x] = u.y;
    if (u.y >= 0) stamp[u.y] = stampValue;
}

/* requested pages (-2, -3) back to absent */
__global__ void k_cancel_requests(int* page, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (page[i] < -1) page[i] = -1;
}

BrickCache::~BrickCache() {
    if (specStream_) cudaStreamSynchronize(specStream_);
    for (SpecChunk& C : chunks_) {
        if (C.ev) cudaEventDestroy(C.ev);
        if (C.hi) cudaFreeHost(C.hi);
        if (C.hu) cudaFreeHost(C.hu);
        cudaFree(C.di); cudaFree(C.du);
    }
    if (specStream_) cudaStreamDestroy(specStream_);
    if (svcEv_) cudaEventDestroy(svcEv_);
    cudaFree(d_page_); cudaFree(d_slab_); cudaFree(d_stamp_); cudaFree(d_stage_);
    if (h_tier_) cudaFreeHost(h_tier_);
    for (Xfer& X : xf_) {
        if (X.ev) cudaEventSynchronize(X.ev), cudaEventDestroy(X.ev);
        if (X.hu) cudaFreeHost(X.hu);
        if (X.hi) cudaFreeHost(X.hi);
        cudaFree(X.du); cudaFree(X.di);
    }
    if (svcItemsH_) cudaFreeHost(svcItemsH_);
    if (svcUpdH_) cudaFreeHost(svcUpdH_);
    cudaFree(svcItemsD_); cudaFree(svcUpdD_);
    if (h_req_) cudaFreeHost(h_req_);

}

vt_status BrickCache::init(const CacheConfig& c) {
    cfg_ = c;
    if (c.deviceSlots < 1) return fail(VT_ERR_INVALID, "maxElementsCache must be >= 1");
    if (c.hostSlots < 1) return fail(VT_ERR_INVALID, "maxElementsCache_CPU must be >= 1");
    esize_ = (int)c.vol->esize();
    D_ = c.edge + 2 * c.inc;
    slotBytes_ = ((size_t)D_ * D_ * D_ * esize_ + 15) & ~(size_t)15;
    brickVol_ = slotBytes_ / esize_;
    {
        TierGeo& g = geo_;
        g.D = D_; g.e = c.edge; g.inc = c.inc; g.es = esize_;
        const size_t row = (size_t)D_ * esize_;
        g.len[0] = (size_t)c.edge * c.edge * row;                        /* M */
        g.len[1] = g.len[2] = (size_t)c.inc * D_ * row;                  /* X-, X+ */
        g.len[3] = g.len[4] = (size_t)c.edge * c.inc * row;              /* Y-, Y+ */
        size_t o = 0;
        for (int b = 0; b < 5; b++) { g.off[b] = o; o = (o + g.len[b] + 63) & ~(size_t)63; }
        g.tierBytes = tierBytes_ = o;
        g.slotBytes = slotBytes_;
        /* rows of every part mask, in the volume's (plane, row) order, with
         * their packed offsets */
        if (tierBytes_ > 0xFFFFFFFFull) return fail(VT_ERR_INVALID, "brick too large");
        const int D = D_, e = c.edge, inc = c.inc;
        const long long NY = c.vol->dims[1], NZ = c.vol->dims[2];
        for (int parts = 0; parts < 32; parts++) {
            std::vector<TierRow>& L = rowList_[parts];
            L.clear();
            for (int x = 0; x < D; x++) {
                if (x < inc || x >= inc + e) {
                    const bool lo = x < inc;
                    if (!(parts & (lo ? kPartXm : kPartXp))) continue;
                    const size_t base = g.off[lo ? 1 : 2] + (size_t)(lo ? x : x - inc - e) * D * row;
                    for (int y = 0; y < D; y++)
                        L.push_back({x, y, (unsigned int)(base + (size_t)y * row), ((long long)x * NY + y) * NZ});
                    continue;
                }
                const int p = x - inc;
                for (int y = 0; y < D; y++) {
                    size_t o2;
                    if (y < inc) {
                        if (!(parts & kPartYm)) continue;
                        o2 = g.off[3] + ((size_t)p * inc + y) * row;
                    } else if (y >= inc + e) {
                        if (!(parts & kPartYp)) continue;
                        o2 = g.off[4] + ((size_t)p * inc + (y - inc - e)) * row;
                    } else {
                        if (!(parts & kPartM)) continue;
                        o2 = g.off[0] + ((size_t)p * e + (y - inc)) * row;
                    }
                    L.push_back({x, y, (unsigned int)o2, ((long long)x * NY + y) * NZ});
                }
            }
        }
    }
    pageBase_ = 0;                     /* keys are page indices (bx << 2Lc | by << Lc | bz) */
    pageN_ = (size_t)1 << (3 * c.Lc);
    nSlots_ = c.deviceSlots;
    nHost_ = c.hostSlots;
    CKC(cudaMalloc(&d_page_, pageN_ * 4));
    CKC(cudaMemset(d_page_, 0xFF, pageN_ * 4));
    CKC(cudaMalloc(&d_slab_, slotBytes_ * (size_t)nSlots_));
    stageCap_ = std::min<size_t>(4096, (size_t)nSlots_);
    CKC(cudaMalloc(&d_stage_, stageCap_ * tierBytes_));
    CKC(cudaMalloc(&d_stamp_, (size_t)nSlots_ * 4));
    CKC(cudaMemset(d_stamp_, 0, (size_t)nSlots_ * 4));
    CKC(cudaHostAlloc((void**)&h_tier_, tierBytes_ * (size_t)nHost_, cudaHostAllocMapped | cudaHostAllocPortable));
    CKC(cudaHostGetDevicePointer(&d_tier_, h_tier_, 0));
    slotBrick_.assign(nSlots_, kEmpty);
    mark_.assign(nSlots_, 0);
    freeSlots_.resize(nSlots_);
    for (int i = 0; i < nSlots_; i++) freeSlots_[i] = nSlots_ - 1 - i;   /* slot 0 is handed out first */
    stampHost_.assign(nSlots_, 0);
    pageMirror_.assign(pageN_, -1);
    hostIndex_.assign(pageN_, -1);
    hostBrick_.assign(nHost_, kEmpty);
    freeHost_.resize(nHost_);
    for (int i = 0; i < nHost_; i++) freeHost_[i] = nHost_ - 1 - i;
    hostTick_.assign(nHost_, 0);
    hostMask_.assign(nHost_, 0);
    sharedAprons_ = c.sharedAprons;
    demandBatch_ = c.demandBatch > 0 ? c.demandBatch : 0;
    CKC(cudaEventCreateWithFlags(&svcEv_, cudaEventDisableTiming));
    slotBusy_.assign(nSlots_, 0);
    hostBusy_.assign(nHost_, 0);
    asyncSpec_ = c.asyncSpec;
    {
        specMark_.assign(pageN_, 0);
        specChunkOf_.assign(pageN_, -1);
        CKC(cudaStreamCreateWithFlags(&specStream_, cudaStreamNonBlocking));
        chunks_.resize(kSpecChunks);
        for (int i = 0; i < kSpecChunks; i++) {
            SpecChunk& C = chunks_[i];
            C.cap = kSpecChunk;
            CKC(cudaEventCreateWithFlags(&C.ev, cudaEventDisableTiming));
            CKC(cudaHostAlloc((void**)&C.hi, C.cap * sizeof(SplitItem), cudaHostAllocDefault));
            CKC(cudaHostAlloc((void**)&C.hu, C.cap * sizeof(int2), cudaHostAllocDefault));
            CKC(cudaMalloc(&C.di, C.cap * sizeof(SplitItem)));
            CKC(cudaMalloc(&C.du, C.cap * sizeof(int2)));
            chunkFree_.push_back(kSpecChunks - 1 - i);
        }
    }
    return VT_OK;
}

void BrickCache::fill_args(DevBricks& b) const {
    b.page = d_page_; b.pageBase = pageBase_; b.slab = d_slab_; b.D = D_; b.brickVol = (long long)brickVol_;
    b.inc = cfg_.inc; b.vtype = cfg_.vol->vtype; b.stamp = d_stamp_; b.pass = pass_;
}

double BrickCache::part_bytes(int parts) const {
    double n = 0;
    for (int b = 0; b < 5; b++)
        if (parts & (1 << b)) n += (double)geo_.len[b];
    return n;
}

bool BrickCache::read_part(uint64_t page, int part, unsigned char* img) const {
    const int Lc = cfg_.Lc, sh = cfg_.nLevels - cfg_.Lc, inc = cfg_.inc, e = cfg_.edge, D = D_;
    const uint64_t msk = (1ull << Lc) - 1;
    const int o[3] = {(int)((page >> (2 * Lc)) << sh) - inc, (int)(((page >> Lc) & msk) << sh) - inc,
                      (int)((page & msk) << sh) - inc};
    /* the part's planes [x0, x1) and rows [y0, y1) of the slot, every z:
     * read as a box, it is the part's packed block as it stands */
    int x0 = inc, x1 = inc + e, y0 = inc, y1 = inc + e, b = 0;
    if (part == kPartXm) { x0 = 0; x1 = inc; y0 = 0; y1 = D; b = 1; }
    else if (part == kPartXp) { x0 = inc + e; x1 = D; y0 = 0; y1 = D; b = 2; }
    else if (part == kPartYm) { y0 = 0; y1 = inc; b = 3; }
    else if (part == kPartYp) { y0 = inc + e; y1 = D; b = 4; }
    const int s[3] = {o[0] + x0, o[1] + y0, o[2]}, en[3] = {o[0] + x1, o[1] + y1, o[2] + D};
    return volume_read_native(cfg_.vol, s, en, img + geo_.off[b]);
}

void BrickCache::read_rows(uint64_t page, int parts, unsigned char* img) const {
    const vt_volume* v = cfg_.vol;
    const int Lc = cfg_.Lc, sh = cfg_.nLevels - cfg_.Lc, inc = cfg_.inc, D = D_;
    const uint64_t msk = (1ull << Lc) - 1;
    const int64_t o[3] = {(int64_t)((page >> (2 * Lc)) << sh) - inc, (int64_t)(((page >> Lc) & msk) << sh) - inc,
                          (int64_t)((page & msk) << sh) - inc};
    const size_t es = (size_t)esize_, row = (size_t)D * es;
    /* z overlap of every row with the volume */
    const int64_t z0 = std::max<int64_t>(0, o[2]), z1 = std::min<int64_t>(v->dims[2], o[2] + D);
    const size_t zb = z1 > z0 ? (size_t)(z1 - z0) * es : 0;
    const TierRow* const rows = rowList_[parts & kPartAll].data();
    const size_t nr = rowList_[parts & kPartAll].size();
    const int64_t X0 = o[0], Y0 = o[1], NX = v->dims[0], NY = v->dims[1], NZ = v->dims[2];
    const unsigned char* const base = v->data;
    /* the row's first voxel in the volume, or NULL outside it */
    auto src_row = [=](const TierRow& r) -> const unsigned char* {
        const int64_t X = X0 + r.x, Y = Y0 + r.y;
        if (X < 0 || X >= NX || Y < 0 || Y >= NY || zb == 0) return nullptr;
        return base + (size_t)((X * NY + Y) * NZ + z0) * es;
    };
    /* rows are short and far apart: prefetch PF rows ahead */
    const size_t PF = row < 64 ? 32 : 8;
    if (X0 >= 0 && Y0 >= 0 && o[2] >= 0 && X0 + D <= NX && Y0 + D <= NY && o[2] + D <= NZ) {
        /* the slot lies inside the volume: every row is whole */
        const unsigned char* const first = base + (size_t)((X0 * NY + Y0) * NZ + o[2]) * es;
        for (size_t i = 0; i < PF && i < nr; i++) {
            const unsigned char* q = first + rows[i].src * (long long)es;
            for (size_t c = 0; c < row; c += 64) __builtin_prefetch(q + c);
            __builtin_prefetch(q + row - 1);
        }
        for (size_t i = 0; i < nr; i++) {
            if (i + PF < nr) {
                const unsigned char* q = first + rows[i + PF].src * (long long)es;
                for (size_t c = 0; c < row; c += 64) __builtin_prefetch(q + c);
                __builtin_prefetch(q + row - 1);
            }
            memcpy(img + rows[i].off, first + rows[i].src * (long long)es, row);
        }
        return;
    }
    for (size_t i = 0; i < PF && i < nr; i++) {
        const unsigned char* q = src_row(rows[i]);
        if (!q) continue;
        for (size_t c = 0; c < zb; c += 64) __builtin_prefetch(q + c);
        __builtin_prefetch(q + zb - 1);
    }
    for (size_t i = 0; i < nr; i++) {
        if (i + PF < nr) {
            const unsigned char* q = src_row(rows[i + PF]);
            if (q) {
                for (size_t c = 0; c < zb; c += 64) __builtin_prefetch(q + c);
                __builtin_prefetch(q + zb - 1);
            }
        }
        unsigned char* d = img + rows[i].off;
        const unsigned char* q = src_row(rows[i]);
        if (!q) { memset(d, 0, row); continue; }
        if (z0 > o[2]) memset(d, 0, (size_t)(z0 - o[2]) * es);
        memcpy(d + (size_t)(z0 - o[2]) * es, q, zb);
        if (z1 < o[2] + D) memset(d + (size_t)(z1 - o[2]) * es, 0, (size_t)(o[2] + D - z1) * es);
    }
}

int BrickCache::host_threads() const { return cfg_.hostThreads > 0 ? cfg_.hostThreads : omp_get_max_threads(); }

vt_status BrickCache::ensure_host(const std::vector<uint64_t>& bricks, std::vector<int>& hslot, int64_t* diskLoads,
                                  uint64_t protectTick, const std::vector<unsigned char>* need) {
    const size_t n = bricks.size();
    hslot.assign(n, -1);
    const uint64_t callStart = protectTick ? protectTick : tick_ + 1;
    std::vector<size_t> miss;
    /* reads: (brick index, parts to read); hits that lack a needed part
     * read just that part */
    std::vector<std::pair<size_t, unsigned char>> reads;
    for (size_t i = 0; i < n; i++) {
        const unsigned char want = need ? (unsigned char)((*need)[i] | kPartM) : (unsigned char)kPartAll;
        int hs = hostIndex_[bricks[i] - pageBase_];
        if (hs >= 0) {
            hslot[i] = hs; hostTick_[hs] = ++tick_; hostHits_++;
            const unsigned char lack = want & (unsigned char)~hostMask_[hs];
            if (lack) reads.emplace_back(i, lack);
        } else {
            miss.push_back(i);
        }
    }
    const size_t nfill = reads.size();
    /* victims: never-filled host slots first, then a sweep over the filled
     * ones skipping every slot touched in this call */
    size_t want = miss.size();
    if (want > (size_t)nHost_) return fail(VT_ERR_STATE, "host tier smaller than one request batch");
    std::vector<int> order;
    order.reserve(want);
    while (order.size() < want && !freeHost_.empty()) { order.push_back(freeHost_.back()); freeHost_.pop_back(); }
    for (int scanned = 0; scanned < nHost_ && order.size() < want; scanned++) {
        const int hs = hostClock_;
        hostClock_ = hostClock_ + 1 == nHost_ ? 0 : hostClock_ + 1;
        if (hostBrick_[hs] != kEmpty && hostTick_[hs] < callStart && !hostBusy_[hs]) order.push_back(hs);
    }
    if (order.size() < want) return fail(VT_ERR_STATE, "host tier exhausted");
    for (size_t k = 0; k < want; k++) {
        int hs = order[k];
        if (hostBrick_[hs] != kEmpty) hostIndex_[hostBrick_[hs] - pageBase_] = -1;
        uint64_t b = bricks[miss[k]];
        hostBrick_[hs] = b;
        hostIndex_[b - pageBase_] = hs;
        hostTick_[hs] = ++tick_;
        hostMask_[hs] = 0;
        hslot[miss[k]] = hs;
        reads.emplace_back(miss[k], need ? (unsigned char)((*need)[miss[k]] | kPartM) : (unsigned char)kPartAll);
    }
    if (reads.empty()) return VT_OK;
    const size_t nread = reads.size();
    const auto tr = std::chrono::steady_clock::now();
    /* each brick (or part) is gathered in a per-thread buffer that stays in
     * cache, then streamed to its tier slot: the tier's lines are written
     * without being read first, and do not displace the volume rows other
     * reads share */
    /* a few hundred bricks (a steady-state pass) still spread over every
     * thread */
    const int nth = host_threads();
    const int grain = (int)std::max<size_t>(1, std::min<size_t>(8, nread / ((size_t)nth * 4)));
    std::vector<unsigned char> bad(nread, 0);
    int nbad = 0;
#pragma omp parallel num_threads(nth) reduction(+ : nbad)
    {
        static thread_local std::vector<unsigned char> stage;
        if (stage.size() < tierBytes_) stage.resize(tierBytes_);
        unsigned char* const img = stage.data();
#pragma omp for schedule(dynamic, grain)
        for (long long k = 0; k < (long long)nread; k++) {
            const size_t i = reads[k].first;
            const unsigned char parts = reads[k].second;
            unsigned char* slot = h_tier_ + (size_t)hslot[i] * tierBytes_;
            /* the parts' rows into a packed image in a per-thread buffer
             * that stays in cache, then streamed to the tier slot block by
             * block: whole aligned lines, written without being read first,
             * not displacing the volume rows other reads share */
            if (!cfg_.vol->reader) {
                read_rows(bricks[i], parts, img);
            } else {
                bool ok = true;
                for (int q = 0; q < 5 && ok; q++)
                    if (parts & (1 << q)) ok = read_part(bricks[i], 1 << q, img);
                if (!ok) { bad[k] = 1; nbad++; continue; }
            }
            if (parts == kPartAll) {
                stream_copy(slot, img, tierBytes_);
            } else {
                for (int q = 0; q < 5; q++)
                    if (parts & (1 << q))
                        stream_copy(slot + geo_.off[q], img + geo_.off[q], (geo_.len[q] + 63) & ~(size_t)63);
            }
        }
        stream_fence();
    }
    msHostRead_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tr).count();
    for (size_t k = 0; k < nread; k++)
        if (!bad[k]) hostMask_[hslot[reads[k].first]] |= reads[k].second;
    if (nbad) {
        /* a failed read leaves its tier slot empty again: nothing refers to
         * the brick, and the next request reads it anew */
        uint64_t first = kEmpty;
        for (size_t k = 0; k < nread; k++) {
            if (!bad[k]) continue;
            const size_t i = reads[k].first;
            const int hs = hslot[i];
            if (first == kEmpty) first = bricks[i];
            hostIndex_[bricks[i] - pageBase_] = -1;
            hostBrick_[hs] = kEmpty;
            hostTick_[hs] = 0;
            hostMask_[hs] = 0;
            freeHost_.push_back(hs);
            hslot[i] = -1;
        }
        int missBad = 0;
        for (size_t k = nfill; k < nread; k++) missBad += bad[k];
        hostMisses_ += (int64_t)(want - missBad);
        *diskLoads += (int64_t)(want - missBad);
        return fail(VT_ERR_IO, "reading %d brick(s) from the volume failed (first: page %llu)", nbad,
                    (unsigned long long)first);
    }
    hostMisses_ += (int64_t)want;
    *diskLoads += (int64_t)want;
    return VT_OK;
}

vt_status BrickCache::refresh_stamps(cudaStream_t s) {
    if (stampsFresh_) return VT_OK;
    CKC(cudaMemcpyAsync(stampHost_.data(), d_stamp_, (size_t)nSlots_ * 4, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    stampsFresh_ = true;
    return VT_OK;
}

vt_status BrickCache::launch_loads(const SplitItem* d_items, size_t n, int phase, cudaStream_t s) {
    /* grid.x stays far below its limit: a launch loads at most one item per
     * device slot */
    launches_++;
    k_fill_split<<<(unsigned int)n, 256, 0, s>>>((const unsigned char*)d_tier_, d_stage_, (unsigned char*)d_slab_, geo_,
                                                 d_items, phase);
    CKC(cudaGetLastError());
    return VT_OK;
}

vt_status BrickCache::stage_runs(SplitItem* items, size_t n, cudaStream_t s, double* bytes) {
    /* the copy engine outruns SM loads from mapped memory over PCIe (55
     * against 49 GB/s), but moves whole slots only: runs of >= 16 whole
     * bricks in consecutive tier slots (a cold start hands tier slots out
     * in order) go by it, into staging slots reused by the next call (a
     * later copy on the same stream waits for this call's fill kernel) */
    const size_t kMinRun = 16;
    size_t used = 0;
    for (size_t k = 0; k < n;) {
        size_t e = k + 1;
        if (items[k].parts == kPartAll)
            while (e < n && items[e].parts == kPartAll && items[e].hs == items[e - 1].hs + 1) e++;
        const size_t len = e - k;
        if (items[k].parts == kPartAll && len >= kMinRun && used + len <= stageCap_) {
            CKC(cudaMemcpyAsync(d_stage_ + used * tierBytes_, h_tier_ + (size_t)items[k].hs * tierBytes_,
                                len * tierBytes_, cudaMemcpyHostToDevice, s));
            for (size_t j = k; j < e; j++) { items[j].hs = (int)(used + (j - k)); items[j].staged = 1; }
            used += len;
            *bytes += (double)len * tierBytes_;
        }
        k = e;
    }
    return VT_OK;
}

vt_status BrickCache::pick_slots(size_t m, unsigned int protectFrom, cudaStream_t s, std::vector<int>& order) {
    /* never-filled slots first; then a sweep over the filled slots with the
     * kernels' stamps, first taking slots not used since the frame began,
     * then any stamped before protectFrom (slots a kernel of the current
     * pass used always have a newer stamp) */
    order.clear();
    order.reserve(m);
    while (order.size() < m && !freeSlots_.empty()) { order.push_back(freeSlots_.back()); freeSlots_.pop_back(); }
    if (order.size() < m) {
        vt_status st = refresh_stamps(s);
        if (st != VT_OK) return st;
        ++epoch_;
        for (int round = 0; round < 2 && order.size() < m; round++) {
            const unsigned int lim = round == 0 ? std::min(frameStart_, protectFrom) : protectFrom;
            for (int scanned = 0; scanned < nSlots_ && order.size() < m; scanned++) {
                const int slot = clock_;
                clock_ = clock_ + 1 == nSlots_ ? 0 : clock_ + 1;
                if (slotBrick_[slot] != kEmpty && stampHost_[slot] < lim && mark_[slot] != epoch_ && !slotBusy_[slot]) {
                    mark_[slot] = epoch_;
                    order.push_back(slot);
                }
            }
        }
    }
    return VT_OK;
}

vt_status BrickCache::assign_device(const std::vector<uint64_t>& bricks, const std::vector<int>& hslot, cudaStream_t s,
                                    unsigned int protectFrom, double* h2d, int64_t* loaded, bool sync) {
    const size_t n = bricks.size();
    if (n == 0) return VT_OK;
    Xfer& X = xf_[xfNext_];
    xfNext_ ^= 1;
    if (X.pending) {
        const auto tw = std::chrono::steady_clock::now();
        CKC(cudaEventSynchronize(X.ev));
        X.pending = false;
        msFillWait_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
    }
    /* bricks with a host-tier copy, at most one per device slot */
    size_t m = 0;
    while (m < n && m < (size_t)nSlots_ && hslot[m] >= 0) m++;
    std::vector<int> order;
    vt_status pst = pick_slots(m, protectFrom, s, order);
    if (pst != VT_OK) return pst;
    size_t need = n * 2 + 2;
    if (need > X.ucap) {
        if (X.hu) cudaFreeHost(X.hu);
        cudaFree(X.du);
        X.ucap = need * 2;
        CKC(cudaHostAlloc((void**)&X.hu, X.ucap * sizeof(int2), cudaHostAllocDefault));
        CKC(cudaMalloc(&X.du, X.ucap * sizeof(int2)));
    }
    if (n > X.icap) {
        if (X.hi) cudaFreeHost(X.hi);
        cudaFree(X.di);
        X.icap = n * 2;
        CKC(cudaHostAlloc((void**)&X.hi, X.icap * sizeof(SplitItem), cudaHostAllocDefault));
        CKC(cudaMalloc(&X.di, X.icap * sizeof(SplitItem)));
    }
    int2* const h_upd_ = X.hu;
    SplitItem* const items = X.hi;
    size_t nu = 0, np = 0;
    for (size_t k = 0; k < order.size(); k++) {
        int slot = order[k];
        if (slotBrick_[slot] != kEmpty) {
            uint64_t old = slotBrick_[slot];
            pageMirror_[old - pageBase_] = -1;
            h_upd_[nu++] = make_int2((int)(old - pageBase_), -1);
        }
        uint64_t b = bricks[np];
        slotBrick_[slot] = b;
        pageMirror_[b - pageBase_] = slot;
        stampHost_[slot] = pass_ + 1;
        h_upd_[nu++] = make_int2((int)(b - pageBase_), slot);
        SplitItem& it = items[np];
        it.hs = hslot[np]; it.slot = slot; it.parts = kPartAll; it.staged = 0;
        it.nb[0] = it.nb[1] = it.nb[2] = it.nb[3] = -1;
        np++;
    }
    /* requests that got no slot go back to absent (retried next pass) */
    for (size_t k = np; k < n; k++)
        if (pageMirror_[bricks[k] - pageBase_] < 0) h_upd_[nu++] = make_int2((int)(bricks[k] - pageBase_), -1);
    double bytes = 0;
    if (np) {
        vt_status lst = stage_runs(items, np, s, &bytes);
        if (lst != VT_OK) return lst;
        for (size_t k = 0; k < np; k++)
            if (!items[k].staged) bytes += part_bytes(kPartAll);
        CKC(cudaMemcpyAsync(X.di, items, np * sizeof(SplitItem), cudaMemcpyHostToDevice, s));
        if ((lst = launch_loads(X.di, np, 1, s)) != VT_OK) return lst;
    }
    if (nu) {
        launches_++;
        CKC(cudaMemcpyAsync(X.du, h_upd_, nu * sizeof(int2), cudaMemcpyHostToDevice, s));
        k_page_update<<<(unsigned int)((nu + 255) / 256), 256, 0, s>>>(d_page_, X.du, (int)nu, d_stamp_, pass_ + 1);
        CKC(cudaGetLastError());
    }
    /* the pinned lists are reused by the call after next */
    if (!X.ev) CKC(cudaEventCreateWithFlags(&X.ev, cudaEventDisableTiming));
    CKC(cudaEventRecord(X.ev, s));
    X.pending = true;
    if (sync) {
        const auto tw = std::chrono::steady_clock::now();
        CKC(cudaStreamSynchronize(s));
        xf_[0].pending = xf_[1].pending = false;
        msFillWait_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
    }
    *h2d += bytes;
    *loaded += (int64_t)np;
    return VT_OK;
}

vt_status BrickCache::load_demand(const std::vector<uint64_t>& demand, size_t cap, size_t chunk, cudaStream_t s,
                                  uint64_t svcStart, double* h2d, int64_t* loaded, int64_t* disk) {
    const size_t n = demand.size();
    if (n == 0) return VT_OK;
    /* transfers of earlier calls (lookahead, prefetch) end first: their
     * pinned lists are not shared with this one, but their slots are */
    for (Xfer& X : xf_)
        if (X.pending) {
            const auto tw = std::chrono::steady_clock::now();
            CKC(cudaEventSynchronize(X.ev));
            X.pending = false;
            msFillWait_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
        }
    std::vector<int> order;
    vt_status st = pick_slots(std::min(cap, (size_t)nSlots_), 0xFFFFFFFFu, s, order);
    if (st != VT_OK) return st;
    const size_t np = order.size();
    if (np > svcItemsCap_) {
        if (svcItemsH_) cudaFreeHost(svcItemsH_);
        cudaFree(svcItemsD_);
        svcItemsCap_ = np * 2;
        CKC(cudaHostAlloc((void**)&svcItemsH_, svcItemsCap_ * sizeof(SplitItem), cudaHostAllocDefault));
        CKC(cudaMalloc(&svcItemsD_, svcItemsCap_ * sizeof(SplitItem)));
    }
    if (n + np + 2 > svcUpdCap_) {
        if (svcUpdH_) cudaFreeHost(svcUpdH_);
        cudaFree(svcUpdD_);
        svcUpdCap_ = (n + np + 2) * 2;
        CKC(cudaHostAlloc((void**)&svcUpdH_, svcUpdCap_ * sizeof(int2), cudaHostAllocDefault));
        CKC(cudaMalloc(&svcUpdD_, svcUpdCap_ * sizeof(int2)));
    }
    int2* const upd = svcUpdH_;
    size_t nu = 0;
    /* placement first (evictions included): a neighbour counts as a source
     * of aprons only if its slot holds it when the copies run */
    for (size_t k = 0; k < np; k++) {
        const int slot = order[k];
        if (slotBrick_[slot] != kEmpty) {
            const uint64_t old = slotBrick_[slot];
            pageMirror_[old - pageBase_] = -1;
            upd[nu++] = make_int2((int)(old - pageBase_), -1);
        }
        slotBrick_[slot] = demand[k];
        pageMirror_[demand[k] - pageBase_] = slot;
        stampHost_[slot] = pass_ + 1;
    }
    /* requests that got no slot go back to absent (retried next pass) */
    for (size_t k = np; k < n; k++)
        if (pageMirror_[demand[k] - pageBase_] < 0) upd[nu++] = make_int2((int)(demand[k] - pageBase_), -1);
    /* x/y aprons: from a neighbour resident now (not one still in flight
     * on the side stream) or placed in this service, else from the tier */
    const int Lc = cfg_.Lc;
    const uint64_t grid = 1ull << Lc, msk = grid - 1;
    const bool share = sharedAprons_ && cfg_.inc <= cfg_.edge;
    std::vector<unsigned char> need(np, (unsigned char)kPartAll);
    SplitItem* const items = svcItemsH_;
    bool anyX = false, anyY = false;
    for (size_t k = 0; k < np; k++) {
        SplitItem& it = items[k];
        it.hs = -1; it.slot = order[k]; it.parts = kPartAll; it.staged = 0;
        it.nb[0] = it.nb[1] = it.nb[2] = it.nb[3] = -1;
        if (!share) continue;
        const uint64_t p = demand[k] - pageBase_;
        const uint64_t bx = p >> (2 * Lc), by = (p >> Lc) & msk;
        const bool inGrid[4] = {bx > 0, bx + 1 < grid, by > 0, by + 1 < grid};
        const uint64_t nbPage[4] = {p - (1ull << (2 * Lc)), p + (1ull << (2 * Lc)), p - (1ull << Lc), p + (1ull << Lc)};
        const unsigned char bit[4] = {kPartXm, kPartXp, kPartYm, kPartYp};
        unsigned char parts = kPartM;
        for (int d = 0; d < 4; d++) {
            const int sl = inGrid[d] ? pageMirror_[nbPage[d]] : -1;
            if (sl >= 0 && specMark_[nbPage[d]] != 2) it.nb[d] = sl;
            else parts |= bit[d];
        }
        anyX = anyX || it.nb[0] >= 0 || it.nb[1] >= 0;
        anyY = anyY || it.nb[2] >= 0 || it.nb[3] >= 0;
        need[k] = it.parts = parts;
    }
    /* host reads and tier-to-slot transfers in chunks: the reads of one
     * chunk overlap the transfer of the one before */
    size_t ramp = std::max<size_t>(64, chunk / 8);
    double bytes = 0;
    for (size_t c0 = 0, c1; c0 < np && st == VT_OK; c0 = c1) {
        /* chunks ramp up from chunk/8 (the first chunk's reads overlap
         * nothing) and halve over the last 2 chunks' worth of bricks (the
         * last chunk's transfer overlaps nothing either) */
        const size_t rem = np - c0;
        size_t len = std::min(ramp, rem);
        if (rem <= 2 * chunk) len = std::min(len, std::max(std::min(rem, std::max<size_t>(64, chunk / 16)), rem / 2));
        ramp = std::min(chunk, ramp * 2);
        c1 = c0 + len;
        std::vector<uint64_t> head(demand.begin() + c0, demand.begin() + c1);
        std::vector<unsigned char> hneed(need.begin() + c0, need.begin() + c1);
        std::vector<int> hs;
        st = ensure_host(head, hs, disk, svcStart, &hneed);
        if (st != VT_OK) break;
        for (size_t j = 0; j < len; j++) items[c0 + j].hs = hs[j];
        if ((st = stage_runs(items + c0, len, s, &bytes)) != VT_OK) break;
        for (size_t j = 0; j < len; j++)
            if (!items[c0 + j].staged) bytes += part_bytes(need[c0 + j]);
        CKC(cudaMemcpyAsync(svcItemsD_ + c0, items + c0, len * sizeof(SplitItem), cudaMemcpyHostToDevice, s));
        if ((st = launch_loads(svcItemsD_ + c0, len, 1, s)) != VT_OK) break;
    }
    if (st == VT_OK) {
        if (anyY && (st = launch_loads(svcItemsD_, np, 2, s)) != VT_OK) return st;
        if (anyX && (st = launch_loads(svcItemsD_, np, 3, s)) != VT_OK) return st;
        for (size_t k = 0; k < np; k++) upd[nu++] = make_int2((int)(demand[k] - pageBase_), order[k]);
    } else {
        /* nothing of this service loads (a neighbour may count on a brick
         * whose read failed): its slots are free again, its pages absent;
         * the evictions stand */
        for (size_t k = 0; k < np; k++) {
            slotBrick_[order[k]] = kEmpty;
            pageMirror_[demand[k] - pageBase_] = -1;
            freeSlots_.push_back(order[k]);
            upd[nu++] = make_int2((int)(demand[k] - pageBase_), -1);
        }
    }
    if (nu) {
        launches_++;
        CKC(cudaMemcpyAsync(svcUpdD_, upd, nu * sizeof(int2), cudaMemcpyHostToDevice, s));
        k_page_update<<<(unsigned int)((nu + 255) / 256), 256, 0, s>>>(d_page_, svcUpdD_, (int)nu, d_stamp_, pass_ + 1);
        CKC(cudaGetLastError());
    }
    /* the loads end before the next use of the service lists (and before
     * any freed slot is handed out again) */
    const auto tw = std::chrono::steady_clock::now();
    CKC(cudaStreamSynchronize(s));
    msFillWait_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
    if (st != VT_OK) return st;
    *h2d += bytes;
    *loaded += (int64_t)np;
    return VT_OK;
}

vt_status BrickCache::service(const unsigned long long* d_req, unsigned int nReq, cudaStream_t s, double* h2dBytes) {
    if (nReq == 0) return VT_OK;
    if (nReq > reqCap_) {
        if (h_req_) cudaFreeHost(h_req_);
        reqCap_ = (size_t)nReq * 2;
        CKC(cudaHostAlloc((void**)&h_req_, reqCap_ * 8, cudaHostAllocDefault));
    }
    CKC(cudaMemcpyAsync(h_req_, d_req, (size_t)nReq * 8, cudaMemcpyDeviceToHost, s));
    /* the pass's slot stamps come with the request list, so victim choice
     * never waits for a fill in flight -- unless never-filled slots can take
     * every request (a cold start), when no victim is chosen and speculative
     * requests only join the side stream's queue */
    const bool needStamps = !(asyncSpec_ && (size_t)nReq <= freeSlots_.size());
    if (!stampsFresh_ && needStamps)
        CKC(cudaMemcpyAsync(stampHost_.data(), d_stamp_, (size_t)nSlots_ * 4, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    if (needStamps) stampsFresh_ = true;
    requested_ += nReq;
    std::vector<uint64_t> demand, spec;
    demand.reserve(nReq);
    for (unsigned int i = 0; i < nReq; i++) {
        const uint64_t r = h_req_[i];
        if (r & VT_REQ_SPECULATIVE) spec.push_back(r & ~VT_REQ_SPECULATIVE);
        else demand.push_back(r);
    }
    speculative_ += (int64_t)spec.size();
    if (asyncSpec_) {
        /* speculative requests join the side stream's queue; a demand request
         * for a queued brick takes it out (it loads now), one for a brick in
         * flight waits for its chunk, one for a brick that landed meanwhile
         * needs nothing */
        spec_poll(false);
        std::vector<int> waitFor;
        size_t keep = 0;
        for (size_t i = 0; i < demand.size(); i++) {
            const uint64_t p = demand[i] - pageBase_;
            if (specMark_[p] == 2) { waitFor.push_back(specChunkOf_[p]); continue; }
            if (specMark_[p] == 1) { specMark_[p] = 0; specQueued_--; }
            if (pageMirror_[p] >= 0) continue;
            demand[keep++] = demand[i];
        }
        demand.resize(keep);
        std::sort(waitFor.begin(), waitFor.end());
        waitFor.erase(std::unique(waitFor.begin(), waitFor.end()), waitFor.end());
        for (int c : waitFor) CKC(cudaStreamWaitEvent(s, chunks_[c].ev, 0));
        std::sort(spec.begin(), spec.end());
        for (uint64_t q : spec) {
            const uint64_t p = q - pageBase_;
            if (pageMirror_[p] >= 0 || specMark_[p] != 0 || specQueued_ >= (size_t)nSlots_) continue;
            specMark_[p] = 1;
            specQ_.push_back(q);
            specQueued_++;
        }
        spec.clear();
    }
    /* in page order (z fastest): neighbouring bricks share the volume rows
     * of their aprons, so reading them one after another hits the cache */
    std::sort(demand.begin(), demand.end());
    std::sort(spec.begin(), spec.end());
    int64_t disk = 0, loaded = 0;
    vt_status st;
    /* a cold start's large demand list: the first demandBatch_ bricks load
     * now, the rest go back to "requested speculatively" and to the front of
     * the side stream's queue -- they load into never-filled slots while the
     * next pass runs, and a ray that still finds one absent requests it
     * again (then it loads with the demand) */
    std::vector<uint64_t> deferred;
    if (asyncSpec_ && demandBatch_ > 0 && demand.size() > (size_t)demandBatch_ &&
        freeSlots_.size() >= demand.size() && specQueued_ + demand.size() <= (size_t)nSlots_) {
        deferred.assign(demand.begin() + demandBatch_, demand.end());
        demand.resize(demandBatch_);
    }
    /* chunk size: large services in chunks of 4 096 bricks (the first
     * chunk's reads and the last one's transfer are not overlapped: 8 192
     * left 6 ms of transfer waiting at the end of the c2 cold start, 4 096
     * leaves 3.5); small ones (a
     * steady-state pass) still in four, so the reads of one overlap the
     * transfer of the one before */
    const size_t kChunk = std::min<size_t>(4096, std::max<size_t>(64, ((size_t)nReq + 3) / 4));
    /* host slots touched in this service stay put until it returns: fills of
     * earlier chunks may still be reading them */
    const uint64_t svcStart = tick_ + 1;
    /* demand requests first: no kernel runs, so any slot may be reused;
     * bricks over the admission cap are re-requested next pass
     * (assign_device loads the first `cap` and resets the rest) */
    if (!demand.empty()) {
        /* in chunks: the host-tier reads of one chunk overlap the device fill
         * of the one before */
        const size_t cap = std::min<size_t>({demand.size(), (size_t)nSlots_, (size_t)nHost_});
        if ((st = load_demand(demand, cap, kChunk, s, svcStart, h2dBytes, &loaded, &disk)) != VT_OK) return st;
    }
    if (!deferred.empty()) {
        const size_t nd = deferred.size();
        if (nd + 2 > svcUpdCap_) {
            if (svcUpdH_) cudaFreeHost(svcUpdH_);
            cudaFree(svcUpdD_);
            svcUpdCap_ = (nd + 2) * 2;
            CKC(cudaHostAlloc((void**)&svcUpdH_, svcUpdCap_ * sizeof(int2), cudaHostAllocDefault));
            CKC(cudaMalloc(&svcUpdD_, svcUpdCap_ * sizeof(int2)));
        }
        for (size_t k = 0; k < nd; k++) {
            const uint64_t p = deferred[k] - pageBase_;
            svcUpdH_[k] = make_int2((int)p, VT_PAGE_SPECULATIVE);
            specMark_[p] = 1;
            hintQ_.push_back(deferred[k]);
            specQueued_++;
        }
        deferred_ += (int64_t)nd;
        launches_++;
        CKC(cudaMemcpyAsync(svcUpdD_, svcUpdH_, nd * sizeof(int2), cudaMemcpyHostToDevice, s));
        k_page_update<<<(unsigned int)((nd + 255) / 256), 256, 0, s>>>(d_page_, svcUpdD_, (int)nd, d_stamp_, pass_ + 1);
        CKC(cudaGetLastError());
        CKC(cudaEventRecord(svcEv_, s));
        /* the list's pinned copy is reused by the next service: the copy must
         * have left it */
        CKC(cudaStreamSynchronize(s));
    }
    /* speculative requests (lookahead): only into free slots or slots this
     * frame has not used, so they never evict what its rays still need;
     * the rest go back to absent */
    if (!spec.empty()) {
        std::vector<uint64_t> want;
        want.reserve(spec.size());
        for (uint64_t p : spec)
            if (pageMirror_[p - pageBase_] < 0) want.push_back(p);   /* not loaded as a demand request */
        if (!want.empty()) {
            /* admit only as many as there are slots they may take, so no
             * host-tier read is spent on a brick that finds no slot */
            size_t avail = 0;
            for (int i = 0; i < nSlots_; i++) avail += slotBrick_[i] == kEmpty || stampHost_[i] < frameStart_;
            const size_t hostFree = (size_t)nHost_ - std::min<size_t>((size_t)nHost_, (size_t)(tick_ + 1 - svcStart));
            const size_t cap = std::min<size_t>({want.size(), avail, hostFree});
            /* chunked like the demand requests; slots filled by one chunk
             * carry the current pass's stamp, so later chunks skip them */
            for (size_t c0 = 0; c0 < cap || c0 == 0; c0 += kChunk) {
                const size_t c1 = std::min(cap, c0 + kChunk);
                const bool last = c1 == cap;
                std::vector<uint64_t> head(want.begin() + c0, want.begin() + c1);
                std::vector<int> hs;
                if ((st = ensure_host(head, hs, &disk, svcStart)) != VT_OK) return st;
                if (last) head.insert(head.end(), want.begin() + cap, want.end());   /* reset to absent */
                hs.resize(head.size(), -1);
                if ((st = assign_device(head, hs, s, frameStart_, h2dBytes, &loaded, false)) != VT_OK) return st;
                if (last) break;
            }
        }
    }
    /* fills end before the service returns (their time is a stall) */
    if (xf_[0].pending || xf_[1].pending) {
        const auto tw = std::chrono::steady_clock::now();
        CKC(cudaStreamSynchronize(s));
        xf_[0].pending = xf_[1].pending = false;
        msFillWait_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
    }
    return VT_OK;
}

vt_status BrickCache::prefetch_stage(const std::vector<uint64_t>& bricks, std::vector<uint64_t>& staged,
                                      std::vector<int>& hslot, bool append, uint64_t protectTick) {
    if (!append) { staged.clear(); hslot.clear(); }
    const size_t cap = (size_t)std::min(nSlots_, nHost_);
    hinted_ += (int64_t)bricks.size();
    std::vector<uint64_t> part;
    for (uint64_t b : bricks) {
        if (staged.size() + part.size() >= cap) break;
        if (pageMirror_[b - pageBase_] < 0) part.push_back(b);
    }
    staged_ += (int64_t)part.size();
    if (part.empty()) return VT_OK;
    int64_t disk = 0;
    std::vector<int> hs;
    vt_status st = ensure_host(part, hs, &disk, protectTick);
    if (st != VT_OK) return st;
    staged.insert(staged.end(), part.begin(), part.end());
    hslot.insert(hslot.end(), hs.begin(), hs.end());
    return VT_OK;
}

vt_status BrickCache::prefetch_commit(const std::vector<uint64_t>& staged, const std::vector<int>& hslot,
                                      cudaStream_t s, int64_t* loaded) {
    std::vector<uint64_t> b;
    std::vector<int> hs;
    for (size_t i = 0; i < staged.size(); i++) {
        /* skip bricks demand paging loaded meanwhile, or whose host copy was evicted */
        if (pageMirror_[staged[i] - pageBase_] >= 0 || hslot[i] < 0) continue;
        if (hostIndex_[staged[i] - pageBase_] != hslot[i]) continue;
        b.push_back(staged[i]);
        hs.push_back(hslot[i]);
    }
    if (b.empty()) return VT_OK;
    double h2d = 0;
    int64_t got = 0;
    /* never evict a slot used since the frame began */
    vt_status st = assign_device(b, hs, s, frameStart_, &h2d, &got);
    prefetched_ += got;
    if (loaded) *loaded += got;
    return st;
}

vt_status BrickCache::prefetch(const std::vector<uint64_t>& bricks, cudaStream_t s, int64_t* loaded) {
    std::vector<uint64_t> staged;
    std::vector<int> hs;
    vt_status st = prefetch_stage(bricks, staged, hs);
    if (st != VT_OK) return st;
    return prefetch_commit(staged, hs, s, loaded);
}

vt_status BrickCache::preload(const std::vector<uint64_t>& bricks) {
    size_t batch = (size_t)std::min(nHost_, nSlots_);
    int64_t loaded = 0;
    double h2d = 0;
    for (size_t i = 0; i < bricks.size(); i += batch) {
        std::vector<uint64_t> b(bricks.begin() + i, bricks.begin() + std::min(bricks.size(), i + batch));
        std::vector<int> hs;
        int64_t disk = 0;
        vt_status st = ensure_host(b, hs, &disk);
        if (st != VT_OK) return st;
        st = assign_device(b, hs, 0, 0xFFFFFFFFu, &h2d, &loaded);
        if (st != VT_OK) return st;
    }
    allResident_ = (size_t)loaded == bricks.size() && bricks.size() <= (size_t)nSlots_;
    return VT_OK;
}

void BrickCache::fold_stats(vt_stats& st) {
    st.host_hits = hostHits_; st.host_misses = hostMisses_;
    st.bricks_requested = requested_; st.bricks_loaded_disk = hostMisses_;
    st.bricks_loaded_host = hostHits_; st.bricks_prefetched = prefetched_;
    st.bricks_hinted = hinted_; st.bricks_staged = staged_; st.bricks_speculative = speculative_;
    st.bricks_spec_loaded = specLoaded_;
    st.ms_host_read_total = msHostRead_; st.ms_fill_wait_total = msFillWait_;
    st.launches += launches_ - launchesFolded_;
    launchesFolded_ = launches_;
}
vt_status BrickCache::drop() {
    CKC(cudaDeviceSynchronize());
    spec_poll(true);
    if (!specMark_.empty()) std::fill(specMark_.begin(), specMark_.end(), 0);
    if (!specChunkOf_.empty()) std::fill(specChunkOf_.begin(), specChunkOf_.end(), -1);
    specQ_.clear(); specHead_ = 0; specQueued_ = 0;
    hintQ_.clear(); hintHead_ = 0;
    CKC(cudaMemset(d_page_, 0xFF, pageN_ * 4));
    CKC(cudaMemset(d_stamp_, 0, (size_t)nSlots_ * 4));
    std::fill(slotBrick_.begin(), slotBrick_.end(), kEmpty);
    freeSlots_.resize(nSlots_);
    for (int i = 0; i < nSlots_; i++) freeSlots_[i] = nSlots_ - 1 - i;
    clock_ = 0;
    std::fill(stampHost_.begin(), stampHost_.end(), 0);
    stampsFresh_ = false;
    std::fill(pageMirror_.begin(), pageMirror_.end(), -1);
    std::fill(hostIndex_.begin(), hostIndex_.end(), -1);
    std::fill(hostBrick_.begin(), hostBrick_.end(), kEmpty);
    freeHost_.resize(nHost_);
    for (int i = 0; i < nHost_; i++) freeHost_[i] = nHost_ - 1 - i;
    hostClock_ = 0;
    std::fill(hostTick_.begin(), hostTick_.end(), 0);
    std::fill(hostMask_.begin(), hostMask_.end(), 0);
    allResident_ = false;
    return VT_OK;
}

void BrickCache::spec_poll(bool wait) {
    size_t done = 0;
    for (; done < chunkLive_.size(); done++) {
        SpecChunk& C = chunks_[chunkLive_[done]];
        if (wait && done == 0) cudaEventSynchronize(C.ev);   /* the oldest; later ones as they are */
        else if (cudaEventQuery(C.ev) == cudaErrorNotReady) { cudaGetLastError(); break; }
        for (size_t i = 0; i < C.pages.size(); i++) {
            const uint64_t p = C.pages[i] - pageBase_;
            if (specMark_[p] == 2 && specChunkOf_[p] == chunkLive_[done]) { specMark_[p] = 0; specChunkOf_[p] = -1; }
            slotBusy_[C.slots[i]]--;
            hostBusy_[C.hslots[i]] = 0;
        }
        for (int sl : C.sources) slotBusy_[sl]--;
        C.sources.clear();
        chunkFree_.push_back(chunkLive_[done]);
    }
    chunkLive_.erase(chunkLive_.begin(), chunkLive_.begin() + done);
}

vt_status BrickCache::spec_issue(const std::vector<uint64_t>& pages, int64_t* loaded) {
    const int c = chunkFree_.back();
    chunkFree_.pop_back();
    SpecChunk& C = chunks_[c];
    const size_t n = pages.size();
    /* placement first (never-filled slots), so the chunk's own bricks count
     * as apron sources for one another */
    C.pages = pages;
    C.slots.resize(n);
    C.sources.clear();
    for (size_t i = 0; i < n; i++) {
        const int slot = freeSlots_.back();
        freeSlots_.pop_back();
        const uint64_t p = pages[i] - pageBase_;
        slotBrick_[slot] = pages[i];
        pageMirror_[p] = slot;
        stampHost_[slot] = pass_;
        slotBusy_[slot]++;
        specMark_[p] = 2;
        specChunkOf_[p] = c;
        C.slots[i] = slot;
    }
    /* x/y aprons from neighbours resident now (not loading in another chunk)
     * or placed in this chunk; a resident source stays busy -- no service
     * evicts it -- until the chunk has landed */
    const int Lc = cfg_.Lc;
    const uint64_t grid = 1ull << Lc, msk = grid - 1;
    const bool share = sharedAprons_ && cfg_.inc <= cfg_.edge;
    std::vector<unsigned char> need(n, (unsigned char)kPartAll);
    bool anyX = false, anyY = false;
    for (size_t i = 0; i < n; i++) {
        SplitItem& it = C.hi[i];
        it.slot = C.slots[i]; it.parts = kPartAll; it.staged = 0;
        it.nb[0] = it.nb[1] = it.nb[2] = it.nb[3] = -1;
        if (!share) continue;
        const uint64_t p = pages[i] - pageBase_;
        const uint64_t bx = p >> (2 * Lc), by = (p >> Lc) & msk;
        const bool inGrid[4] = {bx > 0, bx + 1 < grid, by > 0, by + 1 < grid};
        const uint64_t nbPage[4] = {p - (1ull << (2 * Lc)), p + (1ull << (2 * Lc)), p - (1ull << Lc), p + (1ull << Lc)};
        const unsigned char bit[4] = {kPartXm, kPartXp, kPartYm, kPartYp};
        unsigned char parts = kPartM;
        for (int d = 0; d < 4; d++) {
            const int sl = inGrid[d] ? pageMirror_[nbPage[d]] : -1;
            const bool ours = sl >= 0 && specMark_[nbPage[d]] == 2 && specChunkOf_[nbPage[d]] == c;
            if (sl >= 0 && (ours || specMark_[nbPage[d]] != 2)) {
                it.nb[d] = sl;
                if (!ours) { slotBusy_[sl]++; C.sources.push_back(sl); }
            } else {
                parts |= bit[d];
            }
        }
        anyX = anyX || it.nb[0] >= 0 || it.nb[1] >= 0;
        anyY = anyY || it.nb[2] >= 0 || it.nb[3] >= 0;
        need[i] = it.parts = parts;
    }
    std::vector<int> hs;
    int64_t disk = 0;
    vt_status st = ensure_host(pages, hs, &disk, 0, &need);
    if (st != VT_OK) {
        /* nothing of the chunk loads: its slots are never-filled again */
        for (size_t i = 0; i < n; i++) {
            const uint64_t p = pages[i] - pageBase_;
            slotBrick_[C.slots[i]] = kEmpty;
            pageMirror_[p] = -1;
            slotBusy_[C.slots[i]]--;
            specMark_[p] = 0;
            specChunkOf_[p] = -1;
            freeSlots_.push_back(C.slots[i]);
        }
        for (int sl : C.sources) slotBusy_[sl]--;
        C.sources.clear();
        chunkFree_.push_back(c);
        return st;
    }
    C.hslots = hs;
    for (size_t i = 0; i < n; i++) {
        hostBusy_[hs[i]] = 1;
        C.hi[i].hs = hs[i];
        C.hu[i] = make_int2((int)(pages[i] - pageBase_), C.slots[i]);
    }
    /* the bricks, then the page entries, after the data -- and after any
     * page reset of the last service (deferred demand bricks) */
    CKC(cudaStreamWaitEvent(specStream_, svcEv_, 0));
    CKC(cudaMemcpyAsync(C.di, C.hi, n * sizeof(SplitItem), cudaMemcpyHostToDevice, specStream_));
    if ((st = launch_loads(C.di, n, 1, specStream_)) != VT_OK) return st;
    if (anyY && (st = launch_loads(C.di, n, 2, specStream_)) != VT_OK) return st;
    if (anyX && (st = launch_loads(C.di, n, 3, specStream_)) != VT_OK) return st;
    launches_++;
    CKC(cudaMemcpyAsync(C.du, C.hu, n * sizeof(int2), cudaMemcpyHostToDevice, specStream_));
    k_page_update<<<(unsigned int)((n + 255) / 256), 256, 0, specStream_>>>(d_page_, C.du, (int)n, d_stamp_, pass_);
    CKC(cudaGetLastError());
    CKC(cudaEventRecord(C.ev, specStream_));
    chunkLive_.push_back(c);
    specLoaded_ += (int64_t)n;
    if (loaded) *loaded += (int64_t)n;
    return VT_OK;
}

void BrickCache::spec_hint(const unsigned int* pages, size_t n) {
    hinted_ += (int64_t)n;
    for (size_t i = 0; i < n; i++) {
        const uint64_t q = pageBase_ + pages[i];
        const uint64_t p = pages[i];
        if (p >= pageN_ || pageMirror_[p] >= 0 || specMark_[p] == 2) continue;
        if (specMark_[p] == 0) { specMark_[p] = 1; specQueued_++; }
        hintQ_.push_back(q);
        staged_++;
    }
}

void BrickCache::set_async_spec(bool on) {
    if (on == asyncSpec_) return;
    if (!on) {
        /* the queue is dropped (its pages stay requested speculatively, so a
         * ray that needs one asks for it on demand); chunks in flight land */
        for (size_t i = specHead_; i < specQ_.size(); i++)
            if (specMark_[specQ_[i] - pageBase_] == 1) specMark_[specQ_[i] - pageBase_] = 0;
        for (size_t i = hintHead_; i < hintQ_.size(); i++)
            if (specMark_[hintQ_[i] - pageBase_] == 1) specMark_[hintQ_[i] - pageBase_] = 0;
        specQ_.clear(); specHead_ = 0; specQueued_ = 0;
        hintQ_.clear(); hintHead_ = 0;
    }
    asyncSpec_ = on;
}

vt_status BrickCache::spec_work(cudaEvent_t passDone, int64_t* loaded) {
    if (!asyncSpec_) return VT_OK;
    for (;;) {
        spec_poll(false);
        if (specQueued_ == 0 || freeSlots_.empty()) break;
        if (cudaEventQuery(passDone) != cudaErrorNotReady) break;
        cudaGetLastError();   /* the query's answer, not a fault */
        if (chunkFree_.empty()) spec_poll(true);
        /* next chunk from the queue: entries loaded as demand meanwhile are
         * gone (mark 0); a never-filled device slot each */
        std::vector<uint64_t> pages;
        const size_t want = std::min<size_t>(kSpecChunk, freeSlots_.size());
        while (hintHead_ < hintQ_.size() && pages.size() < want) {
            const uint64_t q = hintQ_[hintHead_++];
            const uint64_t p = q - pageBase_;
            if (specMark_[p] != 1) continue;
            specMark_[p] = 0;
            specQueued_--;
            if (pageMirror_[p] < 0) pages.push_back(q);
        }
        if (hintHead_ == hintQ_.size()) { hintQ_.clear(); hintHead_ = 0; }
        while (specHead_ < specQ_.size() && pages.size() < want) {
            const uint64_t q = specQ_[specHead_++];
            const uint64_t p = q - pageBase_;
            if (specMark_[p] != 1) continue;
            specMark_[p] = 0;
            specQueued_--;
            if (pageMirror_[p] < 0) pages.push_back(q);
        }
        if (specHead_ == specQ_.size()) { specQ_.clear(); specHead_ = 0; }
        if (pages.empty()) continue;
        /* in page order: neighbouring bricks share the volume rows of their aprons */
        std::sort(pages.begin(), pages.end());
        if (spec_issue(pages, loaded) != VT_OK) {
            /* speculation never fails a frame: the bricks stay requested
             * speculatively, and a ray that needs one loads it on demand
             * (where a failed read is reported) */
            clear_error();
            break;
        }
    }
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    return VT_OK;
}

vt_status BrickCache::cancel_requests(cudaStream_t s) {
    const unsigned int blocks = (unsigned int)std::min<size_t>(4096, (pageN_ + 255) / 256);
    launches_++;
    k_cancel_requests<<<blocks, 256, 0, s>>>(d_page_, pageN_);
    CKC(cudaGetLastError());
    /* queued speculative bricks are forgotten with their pages; those in
     * flight land as usual */
    for (size_t i = specHead_; i < specQ_.size(); i++)
        if (specMark_[specQ_[i] - pageBase_] == 1) specMark_[specQ_[i] - pageBase_] = 0;
    for (size_t i = hintHead_; i < hintQ_.size(); i++)
        if (specMark_[hintQ_[i] - pageBase_] == 1) specMark_[hintQ_[i] - pageBase_] = 0;
    specQ_.clear(); specHead_ = 0; specQueued_ = 0;
    hintQ_.clear(); hintHead_ = 0;
    CKC(cudaStreamSynchronize(s));
    xf_[0].pending = xf_[1].pending = false;
    return VT_OK;
}

vt_status BrickCache::copy_slot(uint64_t page, void* host, int* resident) {
    *resident = 0;
    if (page - pageBase_ >= pageN_) return fail(VT_ERR_INVALID, "brick outside the brick grid");
    const int slot = pageMirror_[page - pageBase_];
    if (slot < 0) return VT_OK;
    CKC(cudaDeviceSynchronize());
    CKC(cudaMemcpy(host, (unsigned char*)d_slab_ + (size_t)slot * slotBytes_, (size_t)D_ * D_ * D_ * esize_,
                   cudaMemcpyDeviceToHost));
    *resident = 1;
    return VT_OK;
}

void BrickCache::reset_stats() {
    hostHits_ = hostMisses_ = diskLoads_ = requested_ = prefetched_ = hinted_ = staged_ = speculative_ = specLoaded_ = 0;
    msHostRead_ = msFillWait_ = 0;
}

}  // namespace vtrt
