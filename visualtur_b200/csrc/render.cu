/*
 * render.cu -- ray-casting kernels of libvt.so (sm_100a).
 *
 * k_trace fuses the reference's three per-iteration phases -- octree
 * traversal (cuda_getFirtsVoxel, src/Octree.cu:620-739), cache lookup
 * (lruCache::updateCube, src/lruCache.cu:168-296) and march + shade
 * (cuda_rayCaster, src/rayCaster.cu:139-265) -- into one kernel: each ray
 * walks its DFS, marches every candidate node whose brick is resident, and
 * either finishes or suspends with its stack saved when a brick is absent.
 * The result equals the reference's iterate-until-PAINTED loop: candidates
 * are marched in the same DFS order and the first hit is shaded.  The
 * instantiations with SKIP = true let a ray set absent-brick candidates
 * aside and march later ones in the same pass (see run_ray); the first hit
 * in DFS order still decides the pixel.
 *
 * Octree: a flattened node array with 8-bit child masks holding the result
 * of the reference's range search (computed once per octree load), so a
 * traversal step is 8 slab tests and a popcount instead of binary searches.
 */
#include "vt_kernels.h"
#include "vt_math.cuh"

namespace vt {

/* ---- samplers: voxel at brick-relative integer coordinates ------------- */
template <int VTYPE, bool SHM = false>
__device__ __forceinline__ float ldv(const void* p, long long i) {
    if (SHM) {   /* a brick staged in shared memory */
        if (VTYPE == 0) return ((const float*)p)[i];
        return (float)((const unsigned char*)p)[i];
    }
    if (VTYPE == 0) return __ldg((const float*)p + i);
    return (float)__ldg((const unsigned char*)p + i);
}

/* Trilinear sampler over one brick (slab mode) or the padded volume
 * (dense mode).  ox,oy,oz: integer origin of the index space (the
 * reference's minBox = brick min corner - cubeInc); lo/hi: clamp range of
 * the first tap so both taps stay inside the buffer (never active for
 * finite positions with cubeInc >= 3). */
struct Samp {
    const void* base; long long sx, sy; int ox, oy, oz; int hx, hy, hz;
};

/* getElementInterpolate (src/rayCaster.cu:86-106). */
template <int VTYPE, bool SLAB = false, bool SHM = false>
__device__ __forceinline__ float interp(const Samp& s, float3 p) {
    float rx, ry, rz;
    float px = modff(p.x, &rx), py = modff(p.y, &ry), pz = modff(p.z, &rz);
    int x0 = f2i(rx - (float)s.ox), y0 = f2i(ry - (float)s.oy), z0 = f2i(rz - (float)s.oz);
    x0 = min(max(x0, 0), s.hx); y0 = min(max(y0, 0), s.hy); z0 = min(max(z0, 0), s.hz);
    float v000, v001, v010, v011, v100, v101, v110, v111;
    if (SLAB) {
        /* a brick holds < 2^31 voxels: 32-bit index arithmetic */
        const int sx = (int)s.sx, sy = (int)s.sy;
        const int b = x0 * sx + y0 * sy + z0;
        v000 = ldv<VTYPE, SHM>(s.base, b); v001 = ldv<VTYPE, SHM>(s.base, b + 1);
        v010 = ldv<VTYPE, SHM>(s.base, b + sy); v011 = ldv<VTYPE, SHM>(s.base, b + sy + 1);
        v100 = ldv<VTYPE, SHM>(s.base, b + sx); v101 = ldv<VTYPE, SHM>(s.base, b + sx + 1);
        v110 = ldv<VTYPE, SHM>(s.base, b + sx + sy); v111 = ldv<VTYPE, SHM>(s.base, b + sx + sy + 1);
    } else {
        const long long b = (long long)x0 * s.sx + (long long)y0 * s.sy + z0;
        v000 = ldv<VTYPE>(s.base, b); v001 = ldv<VTYPE>(s.base, b + 1);
        v010 = ldv<VTYPE>(s.base, b + s.sy); v011 = ldv<VTYPE>(s.base, b + s.sy + 1);
        v100 = ldv<VTYPE>(s.base, b + s.sx); v101 = ldv<VTYPE>(s.base, b + s.sx + 1);
        v110 = ldv<VTYPE>(s.base, b + s.sx + s.sy); v111 = ldv<VTYPE>(s.base, b + s.sx + s.sy + 1);
    }
    float qx = 1.0f - px, qy = 1.0f - py, qz = 1.0f - pz;
    float c00 = v000 * qx + v100 * px;
    float c01 = v001 * qx + v101 * px;
    float c10 = v010 * qx + v110 * px;
    float c11 = v011 * qx + v111 * px;
    float c0 = c00 * qy + c10 * py;
    float c1 = c01 * qy + c11 * py;
    return c0 * qz + c1 * pz;
}

/* getNormal (src/rayCaster.cu:131-137). */
template <int VTYPE, bool SLAB, bool SHM = false>
__device__ __forceinline__ float3 normal_at(const Samp& s, float3 p) {
    /* six taps through one call site: shading runs once per hit ray, and
     * the smaller kernel keeps the traversal loop in the instruction cache */
    float v[6];
#pragma unroll 1
    for (int t = 0; t < 6; t++) {
        const float d = (t & 1) ? 1.0f : -1.0f;
        float3 q = p;
        if (t < 2) q.x = p.x + d;
        else if (t < 4) q.y = p.y + d;
        else q.z = p.z + d;
        v[t] = interp<VTYPE, SLAB, SHM>(s, q);
    }
    return normalize(f3((v[0] - v[1]) / 2.0f, (v[2] - v[3]) / 2.0f, (v[4] - v[5]) / 2.0f));
}

/* The march of cuda_rayCaster (src/rayCaster.cu:166-237): samples at
 * Xnear, Xnear += 0.5*dir, for steps 0..maxStep; the first sign change of
 * iso - value (equality counts) is refined once linearly.  U samples are
 * fetched per round: their positions accumulate in the reference's order,
 * their taps are issued together, and the crossing test then runs sample
 * by sample -- fetches past the hit are discarded (indices stay clamped to
 * the brick) and are not counted.
 *
 * refine > 0 bisects the bracketing pair [previous, current sample] that
 * many times before the linear step: the midpoint replaces the end whose
 * iso - value has the same strict sign as its own (the crossing test's
 * "no crossing" condition), so the pair keeps bracketing the crossing.
 * Each midpoint is one more trilinear sample. */
template <int VTYPE, bool SLAB, int U, bool SHM = false>
__device__ __forceinline__ bool march(const Samp& s, float3 origin, float3 ray, float tnear,
                                      int maxStep, float iso, int refine, float3* Xhit, unsigned int* nsamp) {
    float3 Xnear = add(origin, mul(ray, tnear));
    float3 Xfar = Xnear;
    float3 vStep = mul(ray, 0.5f);
    if (maxStep < 0) return false;
    float ant = interp<VTYPE, SLAB, SHM>(s, Xnear);
    unsigned int ns = 1;
    bool hit = false;
    for (int steps = 1; steps <= maxStep && !hit; steps += U) {
        float3 X[U];
        float v[U];
#pragma unroll
        for (int u = 0; u < U; u++) X[u] = add(u == 0 ? Xnear : X[u - 1], vStep);
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = interp<VTYPE, SLAB, SHM>(s, X[u]);
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (hit || steps + u > maxStep) break;
            float sig = v[u];
            ns++;
            if ((((iso - ant) < 0.0f) && ((iso - sig) < 0.0f)) ||
                (((iso - ant) > 0.0f) && ((iso - sig) > 0.0f))) {
                ant = sig;
                Xfar = X[u];
            } else {
                float3 P = Xfar, Q = X[u];
                for (int k = 0; k < refine; k++) {
                    float3 M = mul(add(P, Q), 0.5f);
                    float vm = interp<VTYPE, SLAB, SHM>(s, M);
                    ns++;
                    if ((((iso - ant) < 0.0f) && ((iso - vm) < 0.0f)) ||
                        (((iso - ant) > 0.0f) && ((iso - vm) > 0.0f))) {
                        P = M; ant = vm;
                    } else {
                        Q = M; sig = vm;
                    }
                }
                float a = (iso - ant) / (sig - ant);
                *Xhit = add(mul(P, 1.0f - a), mul(Q, a));
                hit = true;
            }
        }
        Xnear = X[U - 1];
    }
    *nsamp += ns;
    return hit;
}

/* Stack entry: (node index in its level << code_bits) | Morton code. */
struct Stk {
    unsigned long long e[VT_STACK];
    unsigned long long sk[VT_SKIP_MAX];   /* passed-over candidates, DFS order */
};

/* stack entry helpers (layout in vt_kernels.h) */
__device__ __forceinline__ unsigned long long make_entry(unsigned int idx, int level, unsigned int x, unsigned int y,
                                                         unsigned int z) {
    return ((unsigned long long)idx << VT_E_INDEX_SHIFT) | ((unsigned long long)level << VT_E_LEVEL_SHIFT) |
           ((unsigned long long)x << (2 * VT_E_COORD_BITS)) | ((unsigned long long)y << VT_E_COORD_BITS) | z;
}
__device__ __forceinline__ int e_level(unsigned long long e) { return (int)((e >> VT_E_LEVEL_SHIFT) & 15u); }
__device__ __forceinline__ unsigned int e_index(unsigned long long e) { return (unsigned int)(e >> VT_E_INDEX_SHIFT); }
__device__ __forceinline__ unsigned int e_x(unsigned long long e) { return (unsigned int)(e >> (2 * VT_E_COORD_BITS)) & 0x7FFu; }
__device__ __forceinline__ unsigned int e_y(unsigned long long e) { return (unsigned int)(e >> VT_E_COORD_BITS) & 0x7FFu; }
__device__ __forceinline__ unsigned int e_z(unsigned long long e) { return (unsigned int)e & 0x7FFu; }

/* sampler for the brick at brick coordinates (bx,by,bz) */
template <int VTYPE, bool SLAB>
__device__ __forceinline__ void setup_sampler(const TraceArgs& A, unsigned int bx, unsigned int by, unsigned int bz,
                                              unsigned int pidx, Samp& s, int* slot) {
    const DevBricks& B = A.br;
    if (SLAB) {
        const int sh = A.oct.nLevels - A.oct.Lc;
        s.ox = (int)(bx << sh) - B.inc; s.oy = (int)(by << sh) - B.inc; s.oz = (int)(bz << sh) - B.inc;
        int sl = B.page[pidx];
        *slot = sl;
        if (sl < 0) return;
        s.base = (const char*)B.slab + (size_t)sl * (size_t)B.brickVol * (VTYPE == 0 ? 4 : 1);
        s.sx = (long long)B.D * B.D; s.sy = B.D;
        s.hx = s.hy = s.hz = B.D - 2;
    } else {
        /* dense: index space = the padded volume, global voxel g at g + P.
         * Equals the brick-relative index of the reference whenever every
         * tap lies inside the brick and its apron (cubeInc >= 3). */
        *slot = 0;
        s.ox = s.oy = s.oz = -B.P;
        s.base = B.vol;
        s.sx = B.vsx; s.sy = B.vsy;
        s.hx = s.hy = s.hz = B.ve - 2;
    }
}

/* One ray in flight. */
struct Ray {
    RayInv r;
    int lastSlot;          /* slot whose stamp this ray wrote last */
    float3 dir;
    int top;
    int view, i, j;
    unsigned int g;        /* padded global ray index */
    float4 rgba;
    unsigned long long node, brick;
    float t;
    float3 n;
    bool hit;
    int nskip;             /* candidates passed over (brick absent), in st.sk */
    bool tent;             /* the pixel holds a hit found past them */
    bool resumeSkips;      /* the passed-over candidates come first (a resumed ray) */
};

/* RAY_TENTATIVE: a hit past passed-over candidates (the pixel is written,
 * the ray suspends until they are decided); RAY_DONE_WRITTEN: they all
 * missed, the pixel written earlier stands. */
enum { RAY_RUNNING = 0, RAY_DONE = 1, RAY_SUSPENDED = 2, RAY_TENTATIVE = 3, RAY_DONE_WRITTEN = 4 };
enum { CAND_MISSING = 0, CAND_EMPTY = 1, CAND_HIT = 2 };

/* Requests page `pidx` once per pass.  A demand request (a ray waits on
 * the brick) moves the page from absent (-1) or speculatively requested
 * (-3) to -2; a speculative one (lookahead) from -1 to -3 and is tagged in
 * the list, so the host loads it only into a slot this frame has not used.
 * Past the list's capacity the page goes back to absent and the request
 * waits for the next pass (the rays that need it suspend and ask again),
 * as the reference's per-pass admission cap defers NOCACHED rays
 * (src/lruCache.cu:184-192). */
__device__ __forceinline__ void request_brick(const TraceArgs& A, unsigned int pidx, bool spec = false) {
    const int mark = spec ? VT_PAGE_SPECULATIVE : VT_PAGE_REQUESTED;
    int old = atomicCAS(&A.br.page[pidx], -1, mark);
    if (old == VT_PAGE_SPECULATIVE && !spec)
        old = atomicCAS(&A.br.page[pidx], VT_PAGE_SPECULATIVE, VT_PAGE_REQUESTED) == VT_PAGE_SPECULATIVE ? -1 : old;
    if (old == -1) {
        unsigned int q = atomicAdd(A.ctl.n_req, 1u);
        if (q < A.ctl.req_cap) {
            A.ctl.req[q] = pidx | (spec ? VT_REQ_SPECULATIVE : 0ull);
        } else {
            atomicCAS(&A.br.page[pidx], mark, -1);
            atomicAdd(&A.ctl.counters[VT_C_REQDEFER], 1ull);
        }
    }
}

/* Expands the inner node `ent` (_cuda_searchChildrenValidAndHit2,
 * src/Octree.cu:375-532, with membership from the flattened child mask):
 * children hit by the ray with tfar >= 0 are sorted by (tnear, tfar)
 * (src/Octree.cu:665-706) and pushed far to near. */
__device__ __forceinline__ bool expand(const TraceArgs& A, const RayInv& r, Stk& st, int& top,
                                       unsigned long long ent, unsigned int* cnt, bool sortChildren) {
    const DevOctree& O = A.oct;
    const int nLevels = O.nLevels, Lo = O.Lo;
    const int level = e_level(ent);
    const unsigned int px_ = e_x(ent), py_ = e_y(ent), pz_ = e_z(ent);
    const uint2 nd = O.nodes[e_index(ent)];
    const int cl = level + 1;
    const int cd = 1 << (nLevels - cl);
    const int mx = (int)(px_ << (nLevels - level)), my = (int)(py_ << (nLevels - level)), mz = (int)(pz_ << (nLevels - level));
    /* the children's faces lie on 3 planes per axis: the slab products of
     * all 8 children are these 9 values (the same float operations the
     * reference performs per child, src/Octree.cu:258-330) */
    const float x0 = ((float)mx - r.o.x) * r.dx, x1 = ((float)(mx + cd) - r.o.x) * r.dx,
                x2 = ((float)(mx + 2 * cd) - r.o.x) * r.dx;
    const float y0 = ((float)my - r.o.y) * r.dy, y1 = ((float)(my + cd) - r.o.y) * r.dy,
                y2 = ((float)(my + 2 * cd) - r.o.y) * r.dy;
    const float z0 = ((float)mz - r.o.z) * r.dz, z1 = ((float)(mz + cd) - r.o.z) * r.dz,
                z2 = ((float)(mz + 2 * cd) - r.o.z) * r.dz;
    /* entry / exit parameter of the low (0) and high (1) half on each axis,
     * ordered by the direction's sign as the reference's slab test orders
     * them (src/Octree.cu:268-300) */
    const bool sx = r.dx >= 0, sy = r.dy >= 0, sz = r.dz >= 0;
    const float ex0 = sx ? x0 : x1, fx0 = sx ? x1 : x0, ex1 = sx ? x1 : x2, fx1 = sx ? x2 : x1;
    const float ey0 = sy ? y0 : y1, fy0 = sy ? y1 : y0, ey1 = sy ? y1 : y2, fy1 = sy ? y2 : y1;
    const float ez0 = sz ? z0 : z1, fz0 = sz ? z1 : z0, ez1 = sz ? z1 : z2, fz1 = sz ? z2 : z1;
    const unsigned int m = nd.y;
    /* Fast path (parametric traversal).  Inside the node the ray's
     * parameter runs from T0 to T1 and changes half on axis a where it
     * crosses the mid-plane, at t = a1.  When T0, T1, the three crossings
     * and 0 are finite and pairwise distinct, the children the slab tests
     * accept are exactly the segments between consecutive events whose end
     * is >= 0; their tnear values are the segment starts, distinct after
     * the clamp to 0, so (tnear, tfar) order is segment order.  The
     * segments, filtered by membership, are pushed directly; any
     * coincidence, infinity or NaN takes the literal path below. */
    if (sortChildren) {
        const float T0 = fmaxf(fmaxf(sx ? x0 : x2, sy ? y0 : y2), sz ? z0 : z2);
        const float T1 = fminf(fminf(sx ? x2 : x0, sy ? y2 : y0), sz ? z2 : z0);
        bool ok = isfinite(x0) && isfinite(x1) && isfinite(x2) && isfinite(y0) && isfinite(y1) && isfinite(y2) &&
                  isfinite(z0) && isfinite(z1) && isfinite(z2) && T0 < T1;
        ok = ok && T0 != x1 && T0 != y1 && T0 != z1 && T0 != 0.0f && T1 != x1 && T1 != y1 && T1 != z1 &&
             T1 != 0.0f && x1 != y1 && x1 != z1 && y1 != z1 && x1 != 0.0f && y1 != 0.0f && z1 != 0.0f;
        if (ok) {
            /* half of each axis at entry: the sign-ordered first half while
             * the crossing lies ahead */
            const int kx = (x1 > T0) ? (sx ? 0 : 1) : (sx ? 1 : 0);
            const int ky = (y1 > T0) ? (sy ? 0 : 1) : (sy ? 1 : 0);
            const int kz = (z1 > T0) ? (sz ? 0 : 1) : (sz ? 1 : 0);
            /* crossings inside (T0, T1), sorted with the child-index bit each flips */
            const float INF = __int_as_float(0x7f800000);
            float c0 = (x1 > T0 && x1 < T1) ? x1 : INF, c1 = (y1 > T0 && y1 < T1) ? y1 : INF,
                  c2 = (z1 > T0 && z1 < T1) ? z1 : INF;
            int b0 = 4, b1 = 2, b2 = 1;
            if (c1 < c0) { float t = c0; c0 = c1; c1 = t; int b = b0; b0 = b1; b1 = b; }
            if (c2 < c1) { float t = c1; c1 = c2; c2 = t; int b = b1; b1 = b2; b2 = b; }
            if (c1 < c0) { float t = c0; c0 = c1; c1 = t; int b = b0; b0 = b1; b1 = b; }
            const int n1 = c0 < INF, n2 = c1 < INF, n3 = c2 < INF;
            const int ch0 = (kx << 2) | (ky << 1) | kz, ch1 = ch0 ^ b0, ch2 = ch1 ^ b1, ch3 = ch2 ^ b2;
            const bool a0 = (n1 ? c0 : T1) >= 0.0f && ((m >> ch0) & 1u);
            const bool a1 = n1 && (n2 ? c1 : T1) >= 0.0f && ((m >> ch1) & 1u);
            const bool a2 = n2 && (n3 ? c2 : T1) >= 0.0f && ((m >> ch2) & 1u);
            const bool a3 = n3 && T1 >= 0.0f && ((m >> ch3) & 1u);
            const int nvf = (int)a0 + (int)a1 + (int)a2 + (int)a3;
            if (top + nvf >= VT_STACK) {
                atomicOr(A.ctl.err, VT_KERR_STACK);
                top = -1;
                return false;
            }
            /* near to far: the first accepted segment ends on top */
            int q = top + nvf;
            const int chs[4] = {ch0, ch1, ch2, ch3};
            const bool acc[4] = {a0, a1, a2, a3};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if (acc[i]) {
                    const int k = chs[i];
                    const unsigned int cidx = cl < Lo ? nd.x + __popc(m & ((1u << k) - 1u)) : 0u;
                    st.e[q--] = make_entry(cidx, cl, (px_ << 1) | ((k >> 2) & 1), (py_ << 1) | ((k >> 1) & 1),
                                           (pz_ << 1) | (k & 1));
                }
            }
            top += nvf;
            if ((unsigned int)(top + 1) > cnt[VT_C_MAXSTACK]) cnt[VT_C_MAXSTACK] = top + 1;
            return true;
        }
    }
    unsigned long long cent[8];
    float ctn[8], ctf[8];
    int nv = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if ((m >> k) & 1u) {
            const int kx = (k >> 2) & 1, ky = (k >> 1) & 1, kz = k & 1;
            float a, b;
            if (slab_t(kx ? ex1 : ex0, kx ? fx1 : fx0, ky ? ey1 : ey0, ky ? fy1 : fy0, kz ? ez1 : ez0, kz ? fz1 : fz0,
                       &a, &b) &&
                b >= 0.0f) {
                unsigned int cidx = cl < Lo ? nd.x + __popc(m & ((1u << k) - 1u)) : 0u;
                cent[nv] = make_entry(cidx, cl, (px_ << 1) | kx, (py_ << 1) | ky, (pz_ << 1) | kz);
                ctn[nv] = a; ctf[nv] = b;
                nv++;
            }
        }
    }
    if (sortChildren) {
        if (nv == 2) {
            /* one pass of the bubble sort decides two children */
            if (ctn[0] > ctn[1] || (ctn[0] == ctn[1] && ctf[0] > ctf[1])) {
                unsigned long long te = cent[0]; cent[0] = cent[1]; cent[1] = te;
            }
        } else if (nv > 2) {
            int n = nv;
            while (n != 0) {
                int newn = 0;
                for (int q = 1; q < nv; q++) {
                    if (ctn[q - 1] > ctn[q] || (ctn[q - 1] == ctn[q] && ctf[q - 1] > ctf[q])) {
                        unsigned long long te = cent[q]; cent[q] = cent[q - 1]; cent[q - 1] = te;
                        float tt = ctn[q]; ctn[q] = ctn[q - 1]; ctn[q - 1] = tt;
                        tt = ctf[q]; ctf[q] = ctf[q - 1]; ctf[q - 1] = tt;
                        newn = q;
                    }
                }
                n = newn;
            }
        }
    }
    if (top + nv >= VT_STACK) {
        if (sortChildren) atomicOr(A.ctl.err, VT_KERR_STACK);   /* lookahead walks only stop */
        top = -1;
        return false;
    }
    for (int q = nv - 1; q >= 0; q--) st.e[++top] = cent[q];
    if ((unsigned int)(top + 1) > cnt[VT_C_MAXSTACK]) cnt[VT_C_MAXSTACK] = top + 1;
    return true;
}

/* Shading of a hit at X (src/rayCaster.cu:238-250): the normal from
 * central differences, |n . l| against the light, the colour ramp over y;
 * the ray's hit fields for the pixel and the diagnostics. */
template <int VTYPE, bool SLAB, bool SHM>
__device__ __forceinline__ void shade_hit(const TraceArgs& A, Ray& R, const Samp& s, float3 X, unsigned int x,
                                          unsigned int y, unsigned int z, unsigned int bx, unsigned int by,
                                          unsigned int bz, unsigned int* cnt) {
    float3 n = normal_at<VTYPE, SLAB, SHM>(s, X);
    cnt[VT_C_NSAMPLES] += 6;
    float3 l = normalize(sub(X, A.light));
    float dif = fabsf(n.x * l.x + n.y * l.y + n.z * l.z);
    float a = X.y / 256.0f;
    R.rgba = make_float4((1 - a) * dif, a * dif, 0.0f * dif, 1.0f);
    R.hit = true; R.node = node_code(x, y, z, A.oct.Lo); R.brick = node_code(bx, by, bz, A.oct.Lc); R.n = n;
    R.t = dot(sub(X, R.r.o), R.dir);
}

/* Candidate `ent` (a node at octreeLevel): brick lookup
 * (lruCache::updateCube, src/lruCache.cu:177-291), then march and shade
 * (src/rayCaster.cu:139-265).  CAND_MISSING when the brick is absent (it is
 * requested), CAND_HIT with R's hit fields set, else CAND_EMPTY. */
template <int VTYPE, bool SLAB, int U>
__device__ __forceinline__ int candidate(const TraceArgs& A, Ray& R, unsigned long long ent, unsigned int* cnt) {
    const DevOctree& O = A.oct;
    const int nLevels = O.nLevels, Lo = O.Lo, Lc = O.Lc;
    const int dimO = 1 << (nLevels - Lo);
    const unsigned int x = e_x(ent), y = e_y(ent), z = e_z(ent);
    const unsigned int bx = x >> (Lo - Lc), by = y >> (Lo - Lc), bz = z >> (Lo - Lc);
    const unsigned int pidx = (bx << (2 * Lc)) | (by << Lc) | bz;
    Samp s; int slot;
    setup_sampler<VTYPE, SLAB>(A, bx, by, bz, pidx, s, &slot);
    if (SLAB && slot < 0) {
        if (slot == -1 || slot == VT_PAGE_SPECULATIVE) request_brick(A, pidx);
        cnt[VT_C_DEVMISSES]++;
        return CAND_MISSING;
    }
    cnt[VT_C_CANDIDATES]++;
    if (SLAB) {
        cnt[VT_C_DEVHITS]++;
        if (slot != R.lastSlot) { A.br.stamp[slot] = A.br.pass; R.lastSlot = slot; }   /* once per brick run */
    }
    if (A.ctl.touched) {
        const int d = A.ctl.touch_shift / 3;   /* Lo - trace level */
        unsigned long long tn = (spread3(x >> d) << 2) | (spread3(y >> d) << 1) | spread3(z >> d);
        atomicOr(&A.ctl.touched[tn >> 5], 1u << (tn & 31));
    }
    const int mbx = (int)(x << (nLevels - Lo)), mby = (int)(y << (nLevels - Lo)), mbz = (int)(z << (nLevels - Lo));
    float tn, tf;
    if (!slab(R.r, mbx, mby, mbz, mbx + dimO, mby + dimO, mbz + dimO, &tn, &tf)) return CAND_EMPTY;
    float3 X;
    unsigned int ns = 0;
    bool h = march<VTYPE, SLAB, U>(s, R.r.o, R.dir, tn, max_steps(tn, tf), A.iso, A.refine, &X, &ns);
    cnt[VT_C_SAMPLES] += ns;
    if (!h) return CAND_EMPTY;
    shade_hit<VTYPE, SLAB, false>(A, R, s, X, x, y, z, bx, by, bz, cnt);
    return CAND_HIT;
}

/* Advances one ray's DFS by at most `budget` steps (src/Octree.cu:620-720
 * interleaved with src/rayCaster.cu:139-265): inner nodes are expanded
 * until a candidate is on top, then the candidate is marched.  Returns
 * RAY_DONE when the ray is shaded or exhausted, RAY_SUSPENDED when it must
 * wait for absent bricks, RAY_RUNNING when the budget ran out.
 *
 * Passing over absent bricks (A.ctl.skip > 0): a candidate whose brick is
 * absent is requested and set aside, and the DFS goes on to later
 * candidates, up to A.ctl.skip of them a pass.  The first hit still wins in
 * DFS order: a hit found past set-aside candidates is tentative (written,
 * RAY_TENTATIVE), the rest of the DFS is dropped, and the next pass marches
 * the set-aside candidates first, in order; the first of them that hits
 * replaces it, and if none does it stands.  So a ray whose candidates lie
 * in several absent bricks asks for all of them in one pass instead of one
 * per pass, and the image is the one of the in-order traversal. */
template <int VTYPE, bool SLAB, int U, bool SKIP>
__device__ int run_ray(const TraceArgs& A, Ray& R, Stk& st, unsigned int* cnt, int budget) {
    const int Lo = A.oct.Lo;
    if (SKIP) {
        while (R.resumeSkips) {
            if (R.nskip == 0) {
                R.resumeSkips = false;
                if (R.tent) return RAY_DONE_WRITTEN;
                break;
            }
            if (budget-- == 0) return RAY_RUNNING;
            const int c = candidate<VTYPE, SLAB, U>(A, R, st.sk[0], cnt);
            if (c == CAND_MISSING) return RAY_SUSPENDED;
            for (int k = 1; k < R.nskip; k++) st.sk[k - 1] = st.sk[k];
            R.nskip--;
            if (c == CAND_HIT) { R.nskip = 0; R.resumeSkips = false; return RAY_DONE; }
        }
    }
    const int K = SKIP ? A.ctl.skip : 0;
    for (;;) {
        unsigned long long ent;
        for (;;) {
            if (R.top < 0) return (SKIP && R.nskip > 0) ? RAY_SUSPENDED : RAY_DONE;   /* exhausted: background */
            ent = st.e[R.top];
            if (e_level(ent) == Lo) break;
            if (budget-- == 0) return RAY_RUNNING;
            R.top--;
            cnt[VT_C_EXPANSIONS]++;
            if (!expand(A, R.r, st, R.top, ent, cnt, true)) return RAY_DONE;
        }
        if (budget-- == 0) return RAY_RUNNING;
        const int c = candidate<VTYPE, SLAB, U>(A, R, ent, cnt);
        if (c == CAND_MISSING) {
            if (SKIP && R.nskip < K) { st.sk[R.nskip++] = ent; R.top--; continue; }
            return RAY_SUSPENDED;   /* the candidate stays on the stack */
        }
        R.top--;
        if (c == CAND_HIT) {
            if (!SKIP || R.nskip == 0) return RAY_DONE;
            R.top = -1;             /* later candidates cannot matter */
            R.tent = true;
            return RAY_TENTATIVE;
        }
    }
}

/* Speculative requests: walks a copy of a suspended ray's DFS (without
 * marching) and requests up to `lookahead` further absent bricks. */
template <int VTYPE>
__device__ void lookahead_requests(const TraceArgs& A, Ray R, Stk& st, unsigned int* cnt) {
    const DevOctree& O = A.oct;
    const int Lo = O.Lo, Lc = O.Lc;
    int want = A.ctl.lookahead, pops = 0;
    unsigned int last = 0xFFFFFFFFu;
    while (R.top >= 0 && want > 0 && pops++ < 256) {
        unsigned long long ent = st.e[R.top--];
        if (e_level(ent) == Lo) {
            const unsigned int pidx = ((e_x(ent) >> (Lo - Lc)) << (2 * Lc)) | ((e_y(ent) >> (Lo - Lc)) << Lc) |
                                      (e_z(ent) >> (Lo - Lc));
            if (pidx != last && A.br.page[pidx] == -1) { request_brick(A, pidx, true); want--; }
            last = pidx;
            continue;
        }
        unsigned int scratch[VT_C_COUNT];
        scratch[VT_C_MAXSTACK] = cnt[VT_C_MAXSTACK];
        if (!expand(A, R.r, st, R.top, ent, scratch, false)) break;   /* order only affects which bricks get asked */
    }
}

/* padded global ray index -> view and pixel (tile order) */
__device__ __forceinline__ bool decode_ray(const DevView* sv, int nv, int tw, int th, unsigned int g, int& v, int& i,
                                           int& j) {
    v = 0;
    for (int k = 1; k < nv; k++) if (sv[k].rayBase <= g) v = k;
    unsigned int local = g - sv[v].rayBase;
    unsigned int tile = local / (unsigned)(tw * th), lt = local % (unsigned)(tw * th);
    unsigned int ti = tile / sv[v].tilesX, tj = tile % sv[v].tilesX;
    i = (int)(ti * th + lt / tw);
    j = (int)(tj * tw + lt % tw);
    return i < sv[v].cam.H && j < sv[v].cam.W;
}

/* Sets up work item w (pass 0: padded ray index; later passes: suspended
 * record).  Returns RAY_RUNNING when the ray has traversal to do, RAY_DONE
 * when it is background already (root miss), -1 for tile padding. */
template <int VTYPE, bool SKIP>
__device__ int start_ray(const TraceArgs& A, const DevView* sv, unsigned int w, Ray& R, Stk& st,
                          unsigned int* cnt) {
    unsigned int depth = 0;
    unsigned long long off = 0;
    bool resume = A.ctl.in != nullptr;
    if (resume) {
        SuspRec rec = A.ctl.in[w];
        R.g = rec.ray; depth = rec.depth; off = rec.off;
    } else {
        R.g = w;
    }
    if (!decode_ray(sv, A.views.n, A.tile_w, A.tile_h, R.g, R.view, R.i, R.j)) return -1;
    const DevCamera& C = sv[R.view].cam;
    R.dir = ray_dir(C.look, C.up, C.right, C.dist, C.h, C.w, C.H, C.W, R.i, R.j);
    R.r.o = C.pos; R.r.dx = 1 / R.dir.x; R.r.dy = 1 / R.dir.y; R.r.dz = 1 / R.dir.z;
    R.rgba = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    R.hit = false; R.node = 0; R.brick = 0; R.t = -1.0f; R.n = f3(0, 0, 0);
    R.top = -1;
    R.lastSlot = -1;
    R.nskip = 0; R.tent = false; R.resumeSkips = false;
    if (resume && depth > 0) {
        int nsk = 0;
        if (SKIP) {
            nsk = (int)((depth >> 8) & 7u);
            R.nskip = nsk;
            R.tent = (depth >> 11) & 1u;
            R.resumeSkips = nsk > 0 || R.tent;
            for (int e = 0; e < nsk; e++) st.sk[e] = A.ctl.pool_in[off + e];
        }
        R.top = (int)(depth & 255u) - 1;
        for (int e = 0; e <= R.top; e++) st.e[e] = A.ctl.pool_in[off + nsk + e];
        return RAY_RUNNING;
    }
    if (!resume) cnt[VT_C_RAYS]++;
    const int N = 1 << A.oct.nLevels;
    float tn, tf;
    /* root test (src/Octree.cu:729) */
    if (A.oct.rootValid && slab(R.r, 0, 0, 0, N, N, N, &tn, &tf)) { R.top = 0; st.e[0] = make_entry(0, 0, 0, 0, 0); return RAY_RUNNING; }
    return RAY_DONE;   /* background */
}

/* count = false: a tentative hit (past set-aside candidates) is written
 * uncounted; the hit is counted once, when the pixel is final */
__device__ __forceinline__ void write_ray(const TraceArgs& A, const DevView* sv, const Ray& R, unsigned int* cnt,
                                          bool count = true) {
    const DevView& V = sv[R.view];
    const size_t id = (size_t)R.i * V.cam.W + R.j;
    if (R.hit && count) cnt[VT_C_HITS]++;
    if (V.rgba) V.rgba[id] = R.rgba;
    if (V.rgb8) {
        V.rgb8[3 * id] = to_u8(R.rgba.x);
        V.rgb8[3 * id + 1] = to_u8(R.rgba.y);
        V.rgb8[3 * id + 2] = to_u8(R.rgba.z);
    }
    if (R.view == 0) {
        if (A.out.node) A.out.node[id] = R.node;
        if (A.out.brick) A.out.brick[id] = R.brick;
        if (A.out.t) A.out.t[id] = R.t;
        if (A.out.n) { A.out.n[3 * id] = R.n.x; A.out.n[3 * id + 1] = R.n.y; A.out.n[3 * id + 2] = R.n.z; }
    }
}

template <int VTYPE, bool SLAB, bool SKIP>
__device__ __forceinline__ void suspend_ray(const TraceArgs& A, Ray& R, Stk& st, unsigned int* cnt) {
    cnt[VT_C_SUSPENDED]++;
    unsigned int q = atomicAdd(A.ctl.n_out, 1u);
    if (q >= A.ctl.out_cap) { atomicOr(A.ctl.err, VT_KERR_SUSPEND_FULL); return; }
    const unsigned int depth = (unsigned int)(R.top + 1), nsk = SKIP ? (unsigned int)R.nskip : 0u;
    unsigned long long off = atomicAdd(A.ctl.pool_used, (unsigned long long)(depth + nsk));
    SuspRec rec;
    rec.ray = R.g;
    if (off + depth + nsk <= A.ctl.pool_cap) {
        for (unsigned int e = 0; e < nsk; e++) A.ctl.pool_out[off + e] = st.sk[e];
        for (unsigned int e = 0; e < depth; e++) A.ctl.pool_out[off + nsk + e] = st.e[e];
        rec.depth = depth | (nsk << 8) | ((SKIP && R.tent ? 1u : 0u) << 11); rec.off = off;
    } else {
        /* pool full: the ray restarts from the root and finds the same first
         * hit; a tentative pixel is rewritten then, and counted once */
        rec.depth = 0; rec.off = 0;
    }
    A.ctl.out[q] = rec;
    if (SLAB && A.ctl.lookahead > 0) lookahead_requests<VTYPE>(A, R, st, cnt);
}

__device__ __forceinline__ void flush_counters(const TraceArgs& A, unsigned int* cnt) {
#pragma unroll
    for (int c = 0; c < VT_C_COUNT; c++) {
        unsigned int v = cnt[c];
        if (c == VT_C_MAXSTACK) {
            for (int off = 16; off; off >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
            if ((threadIdx.x & 31) == 0 && v) atomicMax(&A.ctl.counters[c], (unsigned long long)v);
        } else {
            for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31) == 0 && v) atomicAdd(&A.ctl.counters[c], (unsigned long long)v);
        }
    }
}

/* One ray per thread (PERSIST = false) or a persistent ray queue: each warp
 * keeps its 32 lanes busy, and after every `pops` traversal steps the lanes
 * whose ray finished or suspended take new work items -- a ballot of the
 * idle lanes, one atomicAdd by the leader, and a popcount rank per lane.
 * Eight 128-thread CTAs per SM (64 registers a thread): the traversal is
 * latency-bound, and the extra resident warps hide more of it than the
 * few spilled registers cost. */
template <int VTYPE, bool SLAB, bool PERSIST, int U, bool SKIP>
__global__ void __launch_bounds__(128, 8) k_trace(TraceArgs A) {
    __shared__ DevView sv[VT_MAX_VIEWS];
    for (int k = threadIdx.x; k < A.views.n; k += blockDim.x) sv[k] = A.views.v[k];
    __syncthreads();
    unsigned int cnt[VT_C_COUNT];
#pragma unroll
    for (int c = 0; c < VT_C_COUNT; c++) cnt[c] = 0;
    const unsigned int nItems =
        A.ctl.in ? (A.ctl.n_in_dev ? min(*A.ctl.n_in_dev, A.ctl.n_in) : A.ctl.n_in) : A.views.totalRays;
    Stk st;
    Ray R;
    if (!PERSIST) {
        unsigned int w = blockIdx.x * blockDim.x + threadIdx.x;
        if (w < nItems) {
            int s = start_ray<VTYPE, SKIP>(A, sv, w, R, st, cnt);
            if (s == RAY_RUNNING) s = run_ray<VTYPE, SLAB, U, SKIP>(A, R, st, cnt, -1);
            if (s == RAY_DONE) write_ray(A, sv, R, cnt);
            else if (SKIP && s == RAY_TENTATIVE) {
                write_ray(A, sv, R, cnt, false);
                suspend_ray<VTYPE, SLAB, SKIP>(A, R, st, cnt);
            } else if (s == RAY_SUSPENDED) suspend_ray<VTYPE, SLAB, SKIP>(A, R, st, cnt);
            else if (SKIP && s == RAY_DONE_WRITTEN) cnt[VT_C_HITS]++;   /* the tentative hit stands */
        }
    } else {
        const unsigned int lane = threadIdx.x & 31;
        bool has = false;
        for (;;) {
            unsigned int need = __ballot_sync(0xffffffffu, !has);
            if (need) {
                unsigned int base = 0;
                int leader = __ffs(need) - 1;
                if ((int)lane == leader) base = atomicAdd(A.ctl.work, (unsigned int)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base >= nItems && need == 0xffffffffu) break;   /* queue drained, warp idle */
                if (!has) {
                    unsigned int w = base + __popc(need & ((1u << lane) - 1u));
                    if (w < nItems) {
                        int s = start_ray<VTYPE, SKIP>(A, sv, w, R, st, cnt);
                        has = s == RAY_RUNNING;
                        if (s == RAY_DONE) write_ray(A, sv, R, cnt);
                    }
                }
            }
            if (has) {
                int s = run_ray<VTYPE, SLAB, U, SKIP>(A, R, st, cnt, A.pops);
                if (s == RAY_DONE) { write_ray(A, sv, R, cnt); has = false; }
                else if (SKIP && s == RAY_TENTATIVE) {
                    write_ray(A, sv, R, cnt, false);
                    suspend_ray<VTYPE, SLAB, SKIP>(A, R, st, cnt);
                    has = false;
                } else if (s == RAY_SUSPENDED) { suspend_ray<VTYPE, SLAB, SKIP>(A, R, st, cnt); has = false; }
                else if (SKIP && s == RAY_DONE_WRITTEN) { cnt[VT_C_HITS]++; has = false; }   /* the tentative hit stands */
            }
        }
    }
    flush_counters(A, cnt);
}

/* ---- wavefront passes ------------------------------------------------- */
/* Traversal round: each input ray (a fresh ray of the pass, a ray resumed
 * from the last pass, or a ray whose candidate missed in the last round)
 * walks its DFS (the same expansions as run_ray) to its next candidate.  An
 * absent brick suspends the ray as in the one-kernel pass; a resident one
 * pops the candidate, saves the ray's remaining stack as a wait record and
 * queues a march item, counted into its slot's bin (the first item of a
 * slot lists the slot as touched).  Where the wait pool is full the ray
 * marches the candidate itself, as the one-kernel pass does. */
template <int VTYPE>
__global__ void __launch_bounds__(128, 8) k_wf_traverse(TraceArgs A, WaveRound W) {
    __shared__ DevView sv[VT_MAX_VIEWS];
    for (int k = threadIdx.x; k < A.views.n; k += blockDim.x) sv[k] = A.views.v[k];
    __syncthreads();
    unsigned int cnt[VT_C_COUNT];
#pragma unroll
    for (int c = 0; c < VT_C_COUNT; c++) cnt[c] = 0;
    const unsigned int nItems =
        A.ctl.in ? (A.ctl.n_in_dev ? min(*A.ctl.n_in_dev, A.ctl.n_in) : A.ctl.n_in) : A.views.totalRays;
    const DevOctree& O = A.oct;
    const int Lo = O.Lo, Lc = O.Lc, nLevels = O.nLevels, dimO = 1 << (nLevels - Lo);
    Stk st;
    Ray R;
    for (unsigned int w = blockIdx.x * blockDim.x + threadIdx.x; w < nItems; w += gridDim.x * blockDim.x) {
        const int s0 = start_ray<VTYPE, false>(A, sv, w, R, st, cnt);
        if (s0 < 0) continue;
        if (s0 == RAY_DONE) { write_ray(A, sv, R, cnt); continue; }
        for (;;) {
            bool stop = false;
            for (;;) {   /* expand until a candidate is on top */
                if (R.top < 0) { stop = true; break; }
                const unsigned long long e = st.e[R.top];
                if (e_level(e) == Lo) break;
                R.top--;
                cnt[VT_C_EXPANSIONS]++;
                if (!expand(A, R.r, st, R.top, e, cnt, true)) { stop = true; break; }
            }
            if (stop) { write_ray(A, sv, R, cnt); break; }   /* exhausted (or stack overflow, flagged) */
            const unsigned long long ent = st.e[R.top];
            const unsigned int x = e_x(ent), y = e_y(ent), z = e_z(ent);
            const unsigned int bx = x >> (Lo - Lc), by = y >> (Lo - Lc), bz = z >> (Lo - Lc);
            const unsigned int pidx = (bx << (2 * Lc)) | (by << Lc) | bz;
            const int slot = A.br.page[pidx];
            if (slot < 0) {
                if (slot == -1 || slot == VT_PAGE_SPECULATIVE) request_brick(A, pidx);
                cnt[VT_C_DEVMISSES]++;
                suspend_ray<VTYPE, true, false>(A, R, st, cnt);   /* the candidate stays on the stack */
                break;
            }
            cnt[VT_C_CANDIDATES]++;
            cnt[VT_C_DEVHITS]++;
            if (slot != R.lastSlot) { A.br.stamp[slot] = A.br.pass; R.lastSlot = slot; }
            const int mbx = (int)(x << (nLevels - Lo)), mby = (int)(y << (nLevels - Lo)), mbz = (int)(z << (nLevels - Lo));
            float tn, tf;
            R.top--;
            if (!slab(R.r, mbx, mby, mbz, mbx + dimO, mby + dimO, mbz + dimO, &tn, &tf)) continue;   /* empty */
            const unsigned int depth = (unsigned int)(R.top + 1);
            const unsigned int q = atomicAdd(W.n_wait, 1u);
            const unsigned long long off = atomicAdd(W.pool_wait_used, (unsigned long long)depth);
            if (q < W.wait_cap && off + depth <= W.pool_wait_cap) {
                for (unsigned int e = 0; e < depth; e++) W.pool_wait[off + e] = st.e[e];
                SuspRec rec;
                rec.ray = R.g; rec.depth = depth; rec.off = off;
                W.wait[q] = rec;
                const unsigned int i = atomicAdd(W.n_items, 1u);
                if (i >= W.items_cap) { atomicOr(A.ctl.err, VT_KERR_WAVE); break; }   /* cannot happen: one item a ray */
                const unsigned int rank = atomicAdd(&W.binCount[slot], 1u);
                if (rank == 0) W.touched[atomicAdd(W.n_touched, 1u)] = (unsigned int)slot;
                MarchItem it;
                it.entry = ent; it.rec = q; it.slot = slot; it.tn = tn; it.maxStep = max_steps(tn, tf);
                it.g = R.g; it.rank = rank; it.dx = R.dir.x; it.dy = R.dir.y; it.dz = R.dir.z; it.pad = 0;
                W.items[i] = it;
                break;
            }
            /* no room to wait: march here */
            Samp sm;
            int sl;
            setup_sampler<VTYPE, true>(A, bx, by, bz, pidx, sm, &sl);
            float3 X;
            unsigned int ns = 0;
            const bool h = march<VTYPE, true, 1>(sm, R.r.o, R.dir, tn, max_steps(tn, tf), A.iso, A.refine, &X, &ns);
            cnt[VT_C_SAMPLES] += ns;
            if (h) {
                shade_hit<VTYPE, true, false>(A, R, sm, X, x, y, z, bx, by, bz, cnt);
                write_ray(A, sv, R, cnt);
                break;
            }
        }
    }
    flush_counters(A, cnt);
}

/* Bin offsets: an exclusive prefix sum of the touched slots' counts (one
 * CTA; a few tens of thousands of slots per round). */
__global__ void __launch_bounds__(1024) k_wf_scan(WaveRound W) {
    __shared__ unsigned int part[1024];
    const unsigned int nT = *W.n_touched;
    const unsigned int per = (nT + 1023u) / 1024u;
    const unsigned int b = threadIdx.x * per, e = min(nT, b + per);
    unsigned int sum = 0;
    for (unsigned int i = b; i < e; i++) sum += W.binCount[W.touched[i]];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const unsigned int v = (int)threadIdx.x >= o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned int base = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (unsigned int i = b; i < e; i++) {
        const unsigned int sl = W.touched[i];
        W.binStart[sl] = base;
        base += W.binCount[sl];
    }
}

/* Items into slot order. */
__global__ void k_wf_scatter(WaveRound W) {
    const unsigned int n = min(*W.n_items, W.items_cap);
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MarchItem it = W.items[i];
        const unsigned int d = W.binStart[it.slot] + it.rank;
        if (d < W.items_cap) W.sorted[d] = it;
    }
}

/* March round: one touched slot at a time per CTA.  One thread stages the
 * slot's brick (edge + 2 inc voxels a side, contiguous) into shared memory
 * with a single bulk copy (cp.async.bulk, the tensor memory accelerator's
 * non-tensor form) completing on an mbarrier; every thread then marches
 * items of that slot from shared memory (src/rayCaster.cu:166-250, the same
 * arithmetic as the one-kernel pass).  A hit shades and writes the pixel; a
 * miss sends the ray's wait record on to the next traversal round, or, with
 * nothing left on its stack, writes the background.  Waits are bounded: past
 * the limit the CTA flags VT_KERR_STAGE and stops. */
template <int VTYPE>
__global__ void __launch_bounds__(128) k_wf_march(TraceArgs A, WaveRound W, unsigned int slotBytes) {
    __shared__ DevView sv[VT_MAX_VIEWS];
    __shared__ __align__(8) unsigned long long mbar;
    extern __shared__ __align__(128) unsigned char wf_brick[];
    for (int k = threadIdx.x; k < A.views.n; k += blockDim.x) sv[k] = A.views.v[k];
    const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mb), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    unsigned int cnt[VT_C_COUNT];
#pragma unroll
    for (int c = 0; c < VT_C_COUNT; c++) cnt[c] = 0;
    const DevOctree& O = A.oct;
    const int Lo = O.Lo, Lc = O.Lc, sh = O.nLevels - O.Lc;
    const DevBricks& B = A.br;
    const unsigned int nT = *W.n_touched;
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(wf_brick);
    uint32_t phase = 0;
    for (unsigned int t = blockIdx.x; t < nT; t += gridDim.x) {
        const unsigned int slot = W.touched[t];
        const unsigned int count = W.binCount[slot], start = W.binStart[slot];
        if (threadIdx.x == 0) {
            /* the last slot's reads (generic proxy) before this copy's writes (async proxy) */
            asm volatile("fence.proxy.async.shared::cta;");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mb), "r"(slotBytes) : "memory");
            const char* src = (const char*)B.slab + (size_t)slot * slotBytes;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(dst), "l"(src), "r"(slotBytes), "r"(mb) : "memory");
        }
        uint32_t done = 0;
        for (long long it = 0; it < (1ll << 22) && !done; it++) {
            asm volatile("{\n\t.reg .pred P1;\n\t"
                         "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                         "selp.b32 %0, 1, 0, P1;\n\t}"
                         : "=r"(done) : "r"(mb), "r"(phase) : "memory");
        }
        phase ^= 1u;
        if (__syncthreads_or(!done)) {
            if (threadIdx.x == 0) atomicOr(A.ctl.err, VT_KERR_STAGE);
            break;
        }
        for (unsigned int k = threadIdx.x; k < count && start + k < W.items_cap; k += blockDim.x) {
            const MarchItem it = W.sorted[start + k];
            Ray R;
            decode_ray(sv, A.views.n, A.tile_w, A.tile_h, it.g, R.view, R.i, R.j);
            R.g = it.g;
            R.dir = f3(it.dx, it.dy, it.dz);
            R.r.o = sv[R.view].cam.pos;
            R.hit = false;
            const unsigned int x = e_x(it.entry), y = e_y(it.entry), z = e_z(it.entry);
            const unsigned int bx = x >> (Lo - Lc), by = y >> (Lo - Lc), bz = z >> (Lo - Lc);
            Samp sm;
            sm.base = wf_brick;
            sm.sx = (long long)B.D * B.D; sm.sy = B.D;
            sm.ox = (int)(bx << sh) - B.inc; sm.oy = (int)(by << sh) - B.inc; sm.oz = (int)(bz << sh) - B.inc;
            sm.hx = sm.hy = sm.hz = B.D - 2;
            float3 X;
            unsigned int ns = 0;
            const bool h = march<VTYPE, true, 1, true>(sm, R.r.o, R.dir, it.tn, it.maxStep, A.iso, A.refine, &X, &ns);
            cnt[VT_C_SAMPLES] += ns;
            if (h) {
                shade_hit<VTYPE, true, true>(A, R, sm, X, x, y, z, bx, by, bz, cnt);
                write_ray(A, sv, R, cnt);
            } else {
                const SuspRec rec = W.wait[it.rec];
                if (rec.depth == 0) {   /* nothing left on its stack: background */
                    R.rgba = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                    R.node = 0; R.brick = 0; R.t = -1.0f; R.n = f3(0, 0, 0);
                    write_ray(A, sv, R, cnt);
                } else {
                    W.next[atomicAdd(W.n_next, 1u)] = rec;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) W.binCount[slot] = 0;   /* the bins start empty next round */
    }
    flush_counters(A, cnt);
}

/* cuda_updateRays (src/Camera.cu:39-74) */
__global__ void k_rays(DevCamera C, float* dirs) {
    long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)C.W * C.H) return;
    int i = (int)(id / C.W), j = (int)(id % C.W);
    float3 d = ray_dir(C.look, C.up, C.right, C.dist, C.h, C.w, C.H, C.W, i, j);
    dirs[3 * id] = d.x; dirs[3 * id + 1] = d.y; dirs[3 * id + 2] = d.z;
}

/* cuda_rayCasterCube (src/rayCaster.cu:267-357) */
__device__ __forceinline__ float cube_get(const float* c, int D, long long total, int x, int y, int z) {
    long long i = (long long)z + (long long)y * D + (long long)x * D * D;
    if (i < 0 || i >= total) return 0.0f;   /* outside the allocation */
    return __ldg(c + i);
}
__device__ __forceinline__ float cube_interp(const float* c, int D, long long total, int3 mb, float3 p) {
    float rx, ry, rz;
    float px = modff(p.x, &rx), py = modff(p.y, &ry), pz = modff(p.z, &rz);
    int x0 = f2i(rx - (float)mb.x), y0 = f2i(ry - (float)mb.y), z0 = f2i(rz - (float)mb.z);
    int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    float c00 = cube_get(c, D, total, x0, y0, z0) * (1.0f - px) + cube_get(c, D, total, x1, y0, z0) * px;
    float c01 = cube_get(c, D, total, x0, y0, z1) * (1.0f - px) + cube_get(c, D, total, x1, y0, z1) * px;
    float c10 = cube_get(c, D, total, x0, y1, z0) * (1.0f - px) + cube_get(c, D, total, x1, y1, z0) * px;
    float c11 = cube_get(c, D, total, x0, y1, z1) * (1.0f - px) + cube_get(c, D, total, x1, y1, z1) * px;
    float c0 = c00 * (1.0f - py) + c10 * py;
    float c1 = c01 * (1.0f - py) + c11 * py;
    return c0 * (1.0f - pz) + c1 * pz;
}
__global__ void k_cube(DevCamera C, const float* cube, int3 pmin, int3 cdim, int3 cinc, float iso,
                       float3 light, float4* rgba) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)C.W * C.H) return;
    int i = (int)(tid / C.W), j = (int)(tid % C.W);
    float3 ray = ray_dir(C.look, C.up, C.right, C.dist, C.h, C.w, C.H, C.W, i, j);
    RayInv r; r.o = C.pos; r.dx = 1 / ray.x; r.dy = 1 / ray.y; r.dz = 1 / ray.z;
    int3 mb = pmin;
    const int D = cdim.x + 2 * cinc.x;
    const long long total = (long long)(cdim.x + 2 * cinc.x) * (cdim.y + 2 * cinc.y) * (cdim.z + 2 * cinc.z);
    float tn, tf;
    bool hit = false;
    float3 Xnew = f3(0, 0, 0);
    if (slab(r, mb.x, mb.y, mb.z, mb.x + cdim.x, mb.y + cdim.y, mb.z + cdim.z, &tn, &tf)) {
        mb.x -= cinc.x; mb.y -= cinc.y; mb.z -= cinc.z;
        float3 Xnear = add(C.pos, mul(ray, tn));
        float3 Xfar = Xnear;
        Xnew = Xnear;
        bool primera = true;
        float ant = 0.0f, sig = 0.0f;
        float steps = 0;
        float3 vStep = mul(ray, 0.5f);
        float maxStep = (tf - tn) * 2.0f;   /* (tfar-tnear)/0.5, an exact doubling */
        while (steps <= maxStep) {
            if (primera) {
                primera = false;
                ant = cube_interp(cube, D, total, mb, Xnear);
                Xfar = Xnear;
            } else {
                sig = cube_interp(cube, D, total, mb, Xnear);
                if ((((iso - ant) < 0.0f) && ((iso - sig) < 0.0f)) ||
                    (((iso - ant) > 0.0f) && ((iso - sig) > 0.0f))) {
                    ant = sig;
                    Xfar = Xnear;
                } else {
                    float a = (iso - ant) / (sig - ant);
                    Xnew = add(mul(Xfar, 1.0f - a), mul(Xnear, a));
                    hit = true;
                    steps = maxStep;
                }
            }
            Xnear = add(Xnear, vStep);
            steps++;
        }
    }
    float4 out = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    if (hit) {
        float gx = (cube_interp(cube, D, total, mb, f3(Xnew.x - 1.0f, Xnew.y, Xnew.z)) -
                    cube_interp(cube, D, total, mb, f3(Xnew.x + 1.0f, Xnew.y, Xnew.z))) / 2.0f;
        float gy = (cube_interp(cube, D, total, mb, f3(Xnew.x, Xnew.y - 1.0f, Xnew.z)) -
                    cube_interp(cube, D, total, mb, f3(Xnew.x, Xnew.y + 1.0f, Xnew.z))) / 2.0f;
        float gz = (cube_interp(cube, D, total, mb, f3(Xnew.x, Xnew.y, Xnew.z - 1.0f)) -
                    cube_interp(cube, D, total, mb, f3(Xnew.x, Xnew.y, Xnew.z + 1.0f))) / 2.0f;
        float3 n = normalize(f3(gx, gy, gz));
        float3 l = normalize(sub(Xnew, light));
        float dif = fabsf(dot(n, l));
        float a = Xnew.y / (float)cdim.y;
        out = make_float4((1 - a) * dif, a * dif, 0.0f * dif, 1.0f);
    }
    rgba[tid] = out;
}

/* Copies a host-visible (mapped) volume into the zero-padded device copy. */
template <int VTYPE>
__global__ void k_fill_dense(void* dst, const void* src, long long nx, long long ny, long long nz, int P,
                             long long ey, long long ez) {
    long long row = blockIdx.x;   /* one (x,y) row per block */
    long long x = row / ny, y = row % ny;
    long long dbase = ((x + P) * ey + (y + P)) * ez + P;
    long long sbase = (x * ny + y) * nz;
    for (long long z = threadIdx.x; z < nz; z += blockDim.x) {
        if (VTYPE == 0) ((float*)dst)[dbase + z] = ((const float*)src)[sbase + z];
        else ((unsigned char*)dst)[dbase + z] = ((const unsigned char*)src)[sbase + z];
    }
}

/* Learned prefetch: one thread per leaf brick (page index); its coarse
 * node at `level` is the brick's coordinates shifted by levelCubes - level,
 * Morton-ordered like the trace log's bits.  Absent pages of predicted
 * nodes go to -3 (requested speculatively) and into the list; past the
 * list's capacity a page goes back to absent. */
__global__ void k_predict_requests(int* page, const unsigned int* leafPages, int nLeaf, const float* probs, int ncams,
                                   int level, int Lc, float thr, unsigned int* list, unsigned int* count,
                                   unsigned int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nLeaf) return;
    const unsigned int p = leafPages[i];
    const unsigned int m = (1u << Lc) - 1u, sh = (unsigned int)(Lc - level);
    const unsigned int bx = p >> (2 * Lc), by = (p >> Lc) & m, bz = p & m;
    const unsigned long long node = (spread3(bx >> sh) << 2) | (spread3(by >> sh) << 1) | spread3(bz >> sh);
    const long long nodes = 1ll << (3 * level);
    float pm = 0.0f;
    for (int c = 0; c < ncams; c++) pm = fmaxf(pm, __ldg(probs + (long long)c * nodes + (long long)node));
    if (!(pm > thr) || page[p] != -1) return;
    if (atomicCAS(&page[p], -1, VT_PAGE_SPECULATIVE) != -1) return;
    const unsigned int q = atomicAdd(count, 1u);
    if (q < cap) list[q] = p;
    else atomicCAS(&page[p], VT_PAGE_SPECULATIVE, -1);
}

}  // namespace vt

using namespace vt;

cudaError_t vt_launch_predict_requests(int* page, const unsigned int* leafPages, int nLeaf, const float* probs,
                                       int ncams, int level, int Lc, float thr, unsigned int* list,
                                       unsigned int* count, unsigned int cap, cudaStream_t s) {
    if (nLeaf <= 0) return cudaSuccess;
    k_predict_requests<<<(nLeaf + 255) / 256, 256, 0, s>>>(page, leafPages, nLeaf, probs, ncams, level, Lc, thr, list,
                                                          count, cap);
    return cudaGetLastError();
}

cudaError_t vt_launch_trace(const TraceArgs& a, bool slabMode, bool persistent, int blocksPerSM, cudaStream_t s) {
    const int threads = 128;
    unsigned int items = a.ctl.in ? a.ctl.n_in : a.views.totalRays;
    if (items == 0) return cudaSuccess;
    if (a.views.n < 1 || a.views.n > VT_MAX_VIEWS) return cudaErrorInvalidValue;
    unsigned int blocks;
    if (persistent) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        unsigned int want = (items + threads - 1) / threads;
        blocks = (unsigned int)(sms * (blocksPerSM > 0 ? blocksPerSM : 8));
        if (blocks > want) blocks = want;
    } else {
        blocks = (items + threads - 1) / threads;
    }
    /* setting absent bricks aside is compiled into its own kernels, so the
     * in-order traversal keeps its registers; it needs bricks (slab mode)
     * and is off while a trace is logged */
    const bool skip = slabMode && a.ctl.skip > 0 && !a.ctl.touched;
#define VT_LAUNCH_U(V, S, P, K)                                            \
    switch (a.unroll) {                                                    \
        case 2: k_trace<V, S, P, 2, K><<<blocks, threads, 0, s>>>(a); break; \
        case 4: k_trace<V, S, P, 4, K><<<blocks, threads, 0, s>>>(a); break; \
        case 8: k_trace<V, S, P, 8, K><<<blocks, threads, 0, s>>>(a); break; \
        default: k_trace<V, S, P, 1, K><<<blocks, threads, 0, s>>>(a); break; \
    }
#define VT_LAUNCH(V, S, P) { if (S && skip) VT_LAUNCH_U(V, S, P, S) else VT_LAUNCH_U(V, S, P, false) }
    if (a.br.vtype == 0) {
        if (slabMode) { if (persistent) VT_LAUNCH(0, true, true) else VT_LAUNCH(0, true, false) }
        else { if (persistent) VT_LAUNCH(0, false, true) else VT_LAUNCH(0, false, false) }
    } else {
        if (slabMode) { if (persistent) VT_LAUNCH(1, true, true) else VT_LAUNCH(1, true, false) }
        else { if (persistent) VT_LAUNCH(1, false, true) else VT_LAUNCH(1, false, false) }
    }
#undef VT_LAUNCH_U
#undef VT_LAUNCH
    return cudaGetLastError();
}

cudaError_t vt_launch_wave_round(const TraceArgs& a, const WaveRound& w, int blocksPerSM, size_t slotBytes,
                                 cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned int grid = (unsigned int)(sms * (blocksPerSM > 0 ? blocksPerSM : 8));
    if (slotBytes % 16 != 0 || slotBytes > 200 * 1024) return cudaErrorInvalidValue;
    /* per launch (a cheap host call): the attribute belongs to the current device */
    const int v = a.br.vtype == 0 ? 0 : 1;
    cudaError_t e = v == 0 ? cudaFuncSetAttribute(k_wf_march<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)
                           : cudaFuncSetAttribute(k_wf_march<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    if (v == 0) k_wf_traverse<0><<<grid, 128, 0, s>>>(a, w);
    else k_wf_traverse<1><<<grid, 128, 0, s>>>(a, w);
    k_wf_scan<<<1, 1024, 0, s>>>(w);
    k_wf_scatter<<<(unsigned int)(sms * 4), 256, 0, s>>>(w);
    if (v == 0) k_wf_march<0><<<(unsigned int)(sms * 4), 128, slotBytes, s>>>(a, w, (unsigned int)slotBytes);
    else k_wf_march<1><<<(unsigned int)(sms * 4), 128, slotBytes, s>>>(a, w, (unsigned int)slotBytes);
    return cudaGetLastError();
}

cudaError_t vt_launch_rays(const DevCamera& c, float* dirs, cudaStream_t s) {
    long long n = (long long)c.W * c.H;
    if (n == 0) return cudaSuccess;
    k_rays<<<(unsigned int)((n + 255) / 256), 256, 0, s>>>(c, dirs);
    return cudaGetLastError();
}

cudaError_t vt_launch_cube(const DevCamera& c, const float* cube, int3 minBox, int3 cubeDim,
                           int3 cubeInc, float iso, float3 light, float4* rgba, cudaStream_t s) {
    long long n = (long long)c.W * c.H;
    if (n == 0) return cudaSuccess;
    k_cube<<<(unsigned int)((n + 127) / 128), 128, 0, s>>>(c, cube, minBox, cubeDim, cubeInc, iso, light, rgba);
    return cudaGetLastError();
}

cudaError_t vt_launch_fill_dense(void* dst, int vtype, const void* src, long long nx, long long ny,
                                 long long nz, int P, long long ey, long long ez, cudaStream_t s) {
    long long rows = nx * ny;
    if (rows == 0) return cudaSuccess;
    if (rows > 2147483647LL) return cudaErrorInvalidValue;
    if (vtype == 0) k_fill_dense<0><<<(unsigned int)rows, 256, 0, s>>>(dst, src, nx, ny, nz, P, ey, ez);
    else k_fill_dense<1><<<(unsigned int)rows, 256, 0, s>>>(dst, src, nx, ny, nz, P, ey, ez);
    return cudaGetLastError();
}
