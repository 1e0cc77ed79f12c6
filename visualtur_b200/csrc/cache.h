/*
 * cache.h -- two-tier brick cache of libvt.so (replaces class lruCache,
 * inc/lruCache.hpp:16-97, src/lruCache.cu).
 *
 * Device tier: a slab of `deviceSlots` bricks of (edge + 2*inc)^3 voxels and
 * a direct-mapped page table indexed by brick Morton code (8^levelCubes
 * entries indexed bx << 2Lc | by << Lc | bz: slot >= 0, -1 absent, -2
 * requested this pass, -3 requested by a lookahead).  Bricks are keyed by
 * that page index throughout.  Kernels look bricks up with one load and
 * request absent ones with one atomicCAS; each use stamps the slot with the
 * pass number, and eviction between passes takes the least recently used
 * slots.
 * Host tier: `hostSlots` bricks in pinned, device-mapped memory with the
 * same LRU rule; misses read the brick zero-padded from the volume source
 * (FileManager::readHDF5_Voxel_Array semantics) on host threads.  A fill
 * kernel reading the mapped tier moves bricks to their device slots.
 *
 * Shared aprons (demand loads): a slot is five parts -- the middle M
 * (planes [inc, inc+e) x rows [inc, inc+e), every z) and the x and y
 * aprons X-, X+ (planes [0, inc), [inc+e, D)) and Y-, Y+ (planes
 * [inc, inc+e), rows [0, inc), [inc+e, D)).  An x or y apron is the same
 * voxels as planes or rows of the neighbouring brick's middle, so when
 * that neighbour is resident (or loads in the same chunk) the apron is
 * copied from its slot on the device, and only the rest is read from the
 * volume, written to the host tier and crosses PCIe (the tier stores a
 * brick packed by part, TierGeo).  Host-tier slots remember which parts
 * they hold; a later load that needs another part reads just that part.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "vt_kernels.h"
#include "vt_runtime.h"

namespace vtrt {

struct CacheConfig {
    const vt_volume* vol = nullptr;
    int nLevels = 0, Lc = 0, inc = 3, edge = 0;
    int deviceSlots = 0, hostSlots = 0, hostThreads = 0;
    bool asyncSpec = true;   /* lookahead bricks load on a side stream while passes run */
    bool sharedAprons = true;   /* demand loads copy x/y aprons from resident neighbours */
    /* with side-stream loads: a service loads at most this many demand
     * bricks itself while never-filled slots can take them all, and queues
     * the rest on the side stream, which loads them while the next pass runs
     * (0: no bound) */
    int demandBatch = 0;
};

/* parts of a slot (bit masks; see above) */
enum { kPartM = 1, kPartXm = 2, kPartXp = 4, kPartYm = 8, kPartYp = 16, kPartAll = 31 };

/* one brick load: host-tier slot, device slot, the parts it takes from
 * the host tier, and the device slots of the X-, X+, Y-, Y+ neighbours
 * whose middles supply its other x/y aprons (-1: none) */
struct SplitItem {
    int hs, slot, parts, staged;   /* staged: hs indexes the device staging area, not the tier */
    int nb[4];
};

/* Slot geometry.  A device slot is the D^3 box (x slowest).  A host-tier
 * slot holds the same voxels packed by part -- M, X-, X+, Y-, Y+, each a
 * block starting on a 64-byte line, rows in (plane, row) order -- so a
 * load that needs some parts reads, writes and transfers only their
 * lines. */
struct TierGeo {
    int D, e, inc, es;
    unsigned long long slotBytes, tierBytes;
    unsigned long long off[5], len[5];
};

/* a row of a slot (plane x, row y), its offset in a packed tier slot and,
 * for an in-memory volume, the offset of its first voxel from the slot's
 * first voxel in the volume (in voxels) */
struct TierRow {
    int x, y;
    unsigned int off;
    long long src;
};

class BrickCache {
public:
    ~BrickCache();
    vt_status init(const CacheConfig& c);
    /* loads `bricks` (sorted codes) into device slots before any frame */
    vt_status preload(const std::vector<uint64_t>& bricks);
    bool all_resident() const { return allResident_; }
    void fill_args(DevBricks& b) const;
    /* a kernel pass is about to stamp slots: the host's stamp copy is stale */
    unsigned int next_pass() { stampsFresh_ = false; return ++pass_; }
    void begin_frame() { frameStart_ = pass_ + 1; }
    /* services the nReq brick requests of the last pass (d_req, device) */
    vt_status service(const unsigned long long* d_req, unsigned int nReq, cudaStream_t s, double* h2dBytes);
    /* loads bricks ahead of demand (prefetch); never evicts slots stamped
     * in the current frame */
    vt_status prefetch(const std::vector<uint64_t>& bricks, cudaStream_t s, int64_t* loaded);
    /* the two halves of prefetch: host-tier loads (no device work, may run
     * while a frame's kernels are in flight) and the device fill */
    vt_status prefetch_stage(const std::vector<uint64_t>& bricks, std::vector<uint64_t>& staged,
                             std::vector<int>& hslot, bool append = false, uint64_t protectTick = 0);
    /* threads for host-tier reads (0 in the config: all hardware threads) */
    int host_threads() const;
    /* host-tier clock, for protecting slots staged over several calls */
    uint64_t host_tick() const { return tick_; }
    vt_status prefetch_commit(const std::vector<uint64_t>& staged, const std::vector<int>& hslot, cudaStream_t s,
                              int64_t* loaded);
    void fold_stats(vt_stats& st);
    /* empties both tiers (cold cache); no kernel may be in flight */
    vt_status drop();
    /* pages left requested (-2, -3) by a pass whose requests will not be
     * serviced (a frame that ended in an error) go back to absent */
    vt_status cancel_requests(cudaStream_t s);
    /* Speculative (lookahead) bricks, asynchronous mode: service() queues
     * them instead of loading them; spec_work() loads queued bricks in
     * chunks on a side stream into never-filled device slots while the
     * kernel pass behind `passDone` runs, and returns once that pass has
     * ended (or nothing is left to do).  A demand request for a queued
     * brick loads it at once; one for a brick in flight makes `s` wait for
     * its chunk. */
    vt_status spec_work(cudaEvent_t passDone, int64_t* loaded);
    void set_async_spec(bool on);
    void set_shared_aprons(bool on) { sharedAprons_ = on; }
    void set_demand_batch(int n) { demandBatch_ = n > 0 ? n : 0; }
    /* pages predicted for the coming frames (already marked requested
     * speculatively on the device): queued ahead of the lookahead queue */
    void spec_hint(const unsigned int* pages, size_t n);
    bool async_spec() const { return asyncSpec_; }
    size_t spec_queued() const { return specQueued_; }
    void reset_stats();
    int device_slots() const { return nSlots_; }
    /* host copy of a brick's device slot (D^3 voxels); *resident = 0 if none */
    vt_status copy_slot(uint64_t page, void* host, int* resident);
    size_t slot_bytes() const { return slotBytes_; }

private:
    /* protectTick: host slots touched at or after this tick are not evicted
     * (0: those touched in this call); need: the parts each brick needs in
     * the tier (NULL: all; the middle always) */
    vt_status ensure_host(const std::vector<uint64_t>& bricks, std::vector<int>& hslot, int64_t* diskLoads,
                          uint64_t protectTick = 0, const std::vector<unsigned char>* need = nullptr);
    /* device slots for up to m bricks: never-filled slots first, then the
     * clock sweep over slots not used since the frame began, then any
     * stamped before protectFrom */
    vt_status pick_slots(size_t m, unsigned int protectFrom, cudaStream_t s, std::vector<int>& order);
    /* the demand loads of one service: demand[0, cap) load (as many as get
     * a device slot), the rest go back to absent.  Every brick is placed
     * first, so a neighbour loading in the same service counts as a source
     * of aprons; host reads and transfers then run in chunks (the reads of
     * one overlapping the transfer of the one before), the neighbour
     * copies once at the end. */
    vt_status load_demand(const std::vector<uint64_t>& demand, size_t cap, size_t chunk, cudaStream_t s,
                          uint64_t svcStart, double* h2d, int64_t* loaded, int64_t* disk);
    /* reads `part` of a brick from the volume (caller's read function) into
     * a packed tier image */
    bool read_part(uint64_t page, int part, unsigned char* img) const;
    /* reads the rows of `parts` of a brick of an in-memory volume into a
     * packed tier image, in one pass */
    void read_rows(uint64_t page, int parts, unsigned char* img) const;
    /* host-tier bytes of `parts` */
    double part_bytes(int parts) const;
    /* loads whole bricks (with a host-tier copy, hslot >= 0) into device
     * slots; sync = false leaves the fill running (the transfer lists are
     * double buffered, so the next call overlaps it) */
    vt_status assign_device(const std::vector<uint64_t>& bricks, const std::vector<int>& hslot, cudaStream_t s,
                            unsigned int protectFrom, double* h2d, int64_t* loaded, bool sync = true);
    static constexpr int kSpecChunks = 8;      /* chunks in flight on the side stream */
    static constexpr size_t kSpecChunk = 512;  /* bricks per chunk: the host reads of one
                                                  outlast a pass's end by ~0.4 ms at most */

    CacheConfig cfg_;
    int D_ = 0, esize_ = 4;
    size_t brickVol_ = 0, slotBytes_ = 0, tierBytes_ = 0;
    TierGeo geo_{};
    std::vector<TierRow> rowList_[32];       /* the rows of each part mask, in (plane, row) order */
    uint64_t pageBase_ = 0; size_t pageN_ = 0;
    int* d_page_ = nullptr;
    void* d_slab_ = nullptr;
    unsigned int* d_stamp_ = nullptr;
    int nSlots_ = 0;
    static constexpr uint64_t kEmpty = ~0ull;  /* slot holds no brick (page 0 is a brick) */
    std::vector<uint64_t> slotBrick_;        /* device slot -> brick page (kEmpty: free) */
    std::vector<int> freeSlots_;             /* device slots never filled since init / drop */
    int clock_ = 0;                          /* victim sweep position over device slots */
    std::vector<unsigned int> mark_;         /* slot picked in the current call (== epoch_) */
    unsigned int epoch_ = 0;
    std::vector<int> pageMirror_;            /* host copy of page (>= 0 or -1) */
    std::vector<unsigned int> stampHost_;
    /* stampHost_ equals the device stamps: no kernel pass ran since the copy
     * (assign_device mirrors its own stamp writes) */
    bool stampsFresh_ = false;
    vt_status refresh_stamps(cudaStream_t s);
    /* host tier */
    unsigned char* h_tier_ = nullptr; void* d_tier_ = nullptr; int nHost_ = 0;
    std::vector<int> hostIndex_;             /* brick -> host slot or -1 */
    std::vector<uint64_t> hostBrick_;        /* host slot -> brick page (kEmpty: free) */
    std::vector<int> freeHost_;              /* host slots never filled since init / drop */
    int hostClock_ = 0;                      /* victim sweep position over host slots */
    std::vector<uint64_t> hostTick_;
    std::vector<unsigned char> hostMask_;    /* host slot -> parts it holds */
    bool sharedAprons_ = true;
    int demandBatch_ = 0;
    /* recorded on the service stream after deferred demand pages were set
     * to "requested speculatively"; side-stream page updates wait for it */
    cudaEvent_t svcEv_ = nullptr;
    int64_t deferred_ = 0;
    uint64_t tick_ = 0;
    /* transfer lists */
    struct Xfer {
        int2* hu = nullptr; int2* du = nullptr; size_t ucap = 0;   /* (page, slot) updates */
        SplitItem* hi = nullptr; SplitItem* di = nullptr; size_t icap = 0;   /* loads */
        cudaEvent_t ev = nullptr; bool pending = false;            /* last use still on the GPU */
    } xf_[2];
    /* a service's demand loads (all on the device until it returns) */
    SplitItem* svcItemsH_ = nullptr; SplitItem* svcItemsD_ = nullptr; size_t svcItemsCap_ = 0;
    int2* svcUpdH_ = nullptr; int2* svcUpdD_ = nullptr; size_t svcUpdCap_ = 0;
    vt_status launch_loads(const SplitItem* d_items, size_t n, int phase, cudaStream_t s);
    /* whole bricks in runs of consecutive host-tier slots cross PCIe by the
     * copy engine into a device staging area (the fill kernel then reads
     * them there); marks those items (pad = 1, hs = staging index) */
    vt_status stage_runs(SplitItem* items, size_t n, cudaStream_t s, double* bytes);
    unsigned char* d_stage_ = nullptr;     /* staging area: stageCap_ packed tier slots */
    size_t stageCap_ = 0;
    int xfNext_ = 0;
    unsigned long long* h_req_ = nullptr; size_t reqCap_ = 0;
    /* asynchronous speculative loads */
    struct SpecChunk {
        cudaEvent_t ev = nullptr;
        std::vector<uint64_t> pages;
        std::vector<int> slots, hslots;
        std::vector<int> sources;                 /* other slots the chunk's apron copies read */
        SplitItem* hi = nullptr; SplitItem* di = nullptr;   /* loads */
        int2* hu = nullptr; int2* du = nullptr;   /* page updates */
        size_t cap = 0;
    };
    vt_status spec_issue(const std::vector<uint64_t>& pages, int64_t* loaded);
    void spec_poll(bool wait);
    cudaStream_t specStream_ = nullptr;
    bool asyncSpec_ = true;
    std::vector<uint64_t> specQ_;            /* queued pages (FIFO from specHead_) */
    size_t specHead_ = 0, specQueued_ = 0;
    std::vector<uint64_t> hintQ_;            /* predicted pages, loaded before specQ_ */
    size_t hintHead_ = 0;
    std::vector<unsigned char> specMark_;    /* per page: 0, 1 queued, 2 in flight */
    std::vector<int> specChunkOf_;           /* page in flight -> chunk index */
    std::vector<SpecChunk> chunks_;          /* ring of chunks (index = issue order % size) */
    std::vector<int> chunkFree_;             /* chunks not in flight */
    std::vector<int> chunkLive_;             /* chunks in flight, issue order */
    std::vector<unsigned short> slotBusy_;   /* device slot: side-stream chunks in flight that write or read it */
    std::vector<unsigned char> hostBusy_;    /* host slot read by a side-stream chunk in flight */
    unsigned int pass_ = 0, frameStart_ = 1;
    bool allResident_ = false;
    /* stats */
    int64_t hostHits_ = 0, hostMisses_ = 0, diskLoads_ = 0, requested_ = 0, prefetched_ = 0, hinted_ = 0, staged_ = 0,
            speculative_ = 0, specLoaded_ = 0;
    int64_t launches_ = 0, launchesFolded_ = 0;
    double msHostRead_ = 0, msFillWait_ = 0;
};

}  // namespace vtrt
