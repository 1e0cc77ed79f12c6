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

/* one CTA per brick: 16-byte copies from mapped host memory */
__global__ void k_fill_bricks(const unsigned char* __restrict__ tier, size_t slotBytes, const int2* __restrict__ pairs,
                              unsigned char* __restrict__ slab) {
    int2 p = pairs[blockIdx.x];
    const uint4* src = (const uint4*)(tier + (size_t)p.x * slotBytes);
    uint4* dst = (uint4*)(slab + (size_t)p.y * slotBytes);
    size_t n = slotBytes / 16;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
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
        if (C.hp) cudaFreeHost(C.hp);
        if (C.hu) cudaFreeHost(C.hu);
        cudaFree(C.dp); cudaFree(C.du);
    }
    if (specStream_) cudaStreamDestroy(specStream_);
    cudaFree(d_page_); cudaFree(d_slab_); cudaFree(d_stamp_);
    if (h_tier_) cudaFreeHost(h_tier_);
    for (Xfer& X : xf_) {
        if (X.ev) cudaEventSynchronize(X.ev), cudaEventDestroy(X.ev);
        if (X.hp) cudaFreeHost(X.hp);
        if (X.hu) cudaFreeHost(X.hu);
        cudaFree(X.dp); cudaFree(X.du);
    }
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
    pageBase_ = 0;                     /* keys are page indices (bx << 2Lc | by << Lc | bz) */
    pageN_ = (size_t)1 << (3 * c.Lc);
    nSlots_ = c.deviceSlots;
    nHost_ = c.hostSlots;
    CKC(cudaMalloc(&d_page_, pageN_ * 4));
    CKC(cudaMemset(d_page_, 0xFF, pageN_ * 4));
    CKC(cudaMalloc(&d_slab_, slotBytes_ * (size_t)nSlots_));
    CKC(cudaMalloc(&d_stamp_, (size_t)nSlots_ * 4));
    CKC(cudaMemset(d_stamp_, 0, (size_t)nSlots_ * 4));
    CKC(cudaHostAlloc((void**)&h_tier_, slotBytes_ * (size_t)nHost_, cudaHostAllocMapped | cudaHostAllocPortable));
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
            CKC(cudaHostAlloc((void**)&C.hp, C.cap * sizeof(int2), cudaHostAllocDefault));
            CKC(cudaHostAlloc((void**)&C.hu, C.cap * sizeof(int2), cudaHostAllocDefault));
            CKC(cudaMalloc(&C.dp, C.cap * sizeof(int2)));
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

bool BrickCache::read_brick(uint64_t page, void* dst) const {
    const int Lc = cfg_.Lc, sh = cfg_.nLevels - cfg_.Lc;
    const uint64_t msk = (1ull << Lc) - 1;
    int3 m = make_int3((int)((page >> (2 * Lc)) << sh), (int)(((page >> Lc) & msk) << sh), (int)((page & msk) << sh));
    int s[3] = {m.x - cfg_.inc, m.y - cfg_.inc, m.z - cfg_.inc};
    int e[3] = {s[0] + D_, s[1] + D_, s[2] + D_};
    return volume_read_native(cfg_.vol, s, e, dst);
}

int BrickCache::host_threads() const { return cfg_.hostThreads > 0 ? cfg_.hostThreads : omp_get_max_threads(); }

vt_status BrickCache::ensure_host(const std::vector<uint64_t>& bricks, std::vector<int>& hslot, int64_t* diskLoads,
                                  uint64_t protectTick) {
    const size_t n = bricks.size();
    hslot.assign(n, -1);
    const uint64_t callStart = protectTick ? protectTick : tick_ + 1;
    std::vector<size_t> miss;
    for (size_t i = 0; i < n; i++) {
        int hs = hostIndex_[bricks[i] - pageBase_];
        if (hs >= 0) { hslot[i] = hs; hostTick_[hs] = ++tick_; hostHits_++; }
        else miss.push_back(i);
    }
    if (miss.empty()) return VT_OK;
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
        hslot[miss[k]] = hs;
    }
    const auto tr = std::chrono::steady_clock::now();
    /* each brick is gathered in a per-thread buffer that stays in cache, then
     * streamed to its tier slot: the tier's lines are written without being
     * read first, and do not displace the volume rows other reads share */
    /* a few hundred bricks (a steady-state pass) still spread over every
     * thread */
    const int nth = host_threads();
    const int grain = (int)std::max<size_t>(1, std::min<size_t>(8, want / ((size_t)nth * 4)));
    std::vector<unsigned char> bad(want, 0);
    int nbad = 0;
#pragma omp parallel num_threads(nth) reduction(+ : nbad)
    {
        static thread_local std::vector<unsigned char> stage;
        if (stage.size() < slotBytes_) stage.resize(slotBytes_);
#pragma omp for schedule(dynamic, grain)
        for (long long k = 0; k < (long long)want; k++) {
            size_t i = miss[k];
            if (!read_brick(bricks[i], stage.data())) { bad[k] = 1; nbad++; continue; }
            stream_copy(h_tier_ + (size_t)hslot[i] * slotBytes_, stage.data(), slotBytes_);
        }
        stream_fence();
    }
    msHostRead_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tr).count();
    if (nbad) {
        /* a failed read leaves its tier slot empty again: nothing refers to
         * the brick, and the next request reads it anew */
        uint64_t first = kEmpty;
        for (size_t k = 0; k < want; k++) {
            if (!bad[k]) continue;
            const size_t i = miss[k];
            const int hs = hslot[i];
            if (first == kEmpty) first = bricks[i];
            hostIndex_[bricks[i] - pageBase_] = -1;
            hostBrick_[hs] = kEmpty;
            hostTick_[hs] = 0;
            freeHost_.push_back(hs);
            hslot[i] = -1;
        }
        hostMisses_ += (int64_t)(want - nbad);
        *diskLoads += (int64_t)(want - nbad);
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
    /* slots: never-filled ones first; then a sweep over the filled slots
     * with the kernels' stamps, first taking slots not used since the frame
     * began, then any stamped before protectFrom (slots a kernel of the
     * current pass used always have a newer stamp) */
    std::vector<int> order;
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
    size_t need = n * 2 + 2;
    if (need > X.ucap) {
        if (X.hu) cudaFreeHost(X.hu);
        cudaFree(X.du);
        X.ucap = need * 2;
        CKC(cudaHostAlloc((void**)&X.hu, X.ucap * sizeof(int2), cudaHostAllocDefault));
        CKC(cudaMalloc(&X.du, X.ucap * sizeof(int2)));
    }
    if (n > X.pcap) {
        if (X.hp) cudaFreeHost(X.hp);
        cudaFree(X.dp);
        X.pcap = n * 2;
        CKC(cudaHostAlloc((void**)&X.hp, X.pcap * sizeof(int2), cudaHostAllocDefault));
        CKC(cudaMalloc(&X.dp, X.pcap * sizeof(int2)));
    }
    int2* const h_upd_ = X.hu;
    int2* const h_pairs_ = X.hp;
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
        h_pairs_[np] = make_int2(hslot[np], slot);
        np++;
    }
    /* requests that got no slot go back to absent (retried next pass) */
    for (size_t k = np; k < n; k++)
        if (pageMirror_[bricks[k] - pageBase_] < 0) h_upd_[nu++] = make_int2((int)(bricks[k] - pageBase_), -1);
    /* runs of consecutive host slots going to consecutive device slots (a
     * cold start hands out both in order) move by the copy engine, which
     * outruns SM loads from mapped memory over PCIe; the rest by the kernel */
    const size_t kMinRun = 16;
    size_t nk = 0;
    for (size_t k = 0; k < np;) {
        size_t e = k + 1;
        while (e < np && h_pairs_[e].x == h_pairs_[e - 1].x + 1 && h_pairs_[e].y == h_pairs_[e - 1].y + 1) e++;
        if (e - k >= kMinRun) {
            CKC(cudaMemcpyAsync((unsigned char*)d_slab_ + (size_t)h_pairs_[k].y * slotBytes_, h_tier_ + (size_t)h_pairs_[k].x * slotBytes_,
                                (e - k) * slotBytes_, cudaMemcpyHostToDevice, s));
        } else {
            for (size_t j = k; j < e; j++) h_pairs_[nk++] = h_pairs_[j];
        }
        k = e;
    }
    if (nk) {
        launches_++;
        CKC(cudaMemcpyAsync(X.dp, h_pairs_, nk * sizeof(int2), cudaMemcpyHostToDevice, s));
        k_fill_bricks<<<(unsigned int)nk, 256, 0, s>>>((const unsigned char*)d_tier_, slotBytes_, X.dp,
                                                       (unsigned char*)d_slab_);
        CKC(cudaGetLastError());
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
    *h2d += (double)np * (double)slotBytes_;
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
        for (size_t c0 = 0; c0 < cap; c0 += kChunk) {
            const size_t c1 = std::min(cap, c0 + kChunk);
            const bool last = c1 == cap;
            std::vector<uint64_t> head(demand.begin() + c0, demand.begin() + c1);
            std::vector<int> hs;
            if ((st = ensure_host(head, hs, &disk, svcStart)) != VT_OK) return st;
            if (last) head.insert(head.end(), demand.begin() + cap, demand.end());   /* reset to absent */
            hs.resize(head.size(), -1);
            if ((st = assign_device(head, hs, s, 0xFFFFFFFFu, h2dBytes, &loaded, false)) != VT_OK) return st;
        }
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
            slotBusy_[C.slots[i]] = 0;
            hostBusy_[C.hslots[i]] = 0;
        }
        chunkFree_.push_back(chunkLive_[done]);
    }
    chunkLive_.erase(chunkLive_.begin(), chunkLive_.begin() + done);
}

vt_status BrickCache::spec_issue(const std::vector<uint64_t>& pages, int64_t* loaded) {
    const int c = chunkFree_.back();
    chunkFree_.pop_back();
    SpecChunk& C = chunks_[c];
    const size_t n = pages.size();
    std::vector<int> hs;
    int64_t disk = 0;
    vt_status st = ensure_host(pages, hs, &disk);
    if (st != VT_OK) { chunkFree_.push_back(c); return st; }
    C.pages = pages;
    C.slots.resize(n);
    C.hslots = hs;
    for (size_t i = 0; i < n; i++) {
        const int slot = freeSlots_.back();
        freeSlots_.pop_back();
        const uint64_t p = pages[i] - pageBase_;
        slotBrick_[slot] = pages[i];
        pageMirror_[p] = slot;
        stampHost_[slot] = pass_;
        slotBusy_[slot] = 1;
        hostBusy_[hs[i]] = 1;
        specMark_[p] = 2;
        specChunkOf_[p] = c;
        C.slots[i] = slot;
        C.hp[i] = make_int2(hs[i], slot);
        C.hu[i] = make_int2((int)p, slot);
    }
    /* runs of consecutive host and device slots by the copy engine, the rest
     * by the fill kernel; then the page entries, after the data */
    size_t nk = 0;
    for (size_t k = 0; k < n;) {
        size_t e = k + 1;
        while (e < n && C.hp[e].x == C.hp[e - 1].x + 1 && C.hp[e].y == C.hp[e - 1].y + 1) e++;
        if (e - k >= 16) {
            CKC(cudaMemcpyAsync((unsigned char*)d_slab_ + (size_t)C.hp[k].y * slotBytes_,
                                h_tier_ + (size_t)C.hp[k].x * slotBytes_, (e - k) * slotBytes_, cudaMemcpyHostToDevice,
                                specStream_));
        } else {
            for (size_t j = k; j < e; j++) C.hp[nk++] = C.hp[j];
        }
        k = e;
    }
    if (nk) {
        launches_++;
        CKC(cudaMemcpyAsync(C.dp, C.hp, nk * sizeof(int2), cudaMemcpyHostToDevice, specStream_));
        k_fill_bricks<<<(unsigned int)nk, 256, 0, specStream_>>>((const unsigned char*)d_tier_, slotBytes_, C.dp,
                                                                  (unsigned char*)d_slab_);
        CKC(cudaGetLastError());
    }
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
