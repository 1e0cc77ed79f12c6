/*
 * mlp.cu -- the brick-prefetch network of libvt.so (no reference
 * counterpart): pose features (12) -> 512 -> 512 -> 4096 sigmoid, one
 * output per coarse octree node, trained with binary cross-entropy on
 * traces of the nodes each frame marched.
 *
 * Weights are stored in BF16 with FP32 master copies updated by Adam.  The
 * forward and backward GEMMs run on the tensor cores (tcgen05.mma, BF16 x
 * BF16 -> FP32 in tensor memory): activations and gradients are kept in
 * FP32 and rounded to BF16 as they are staged for the MMA.  A register-tiled
 * SIMT kernel (FP32 activations x BF16 weights, FMA) does the same
 * contraction where vt_mlp_use_tensor_cores switches the tensor cores off.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <cmath>
#include <vector>

#include "../../include/vt.h"
#include "vt_runtime.h"

namespace vtm {

#define CKM(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return vtrt::fail(VT_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <class T> __device__ __forceinline__ float ld(const T* p, long long i);
template <> __device__ __forceinline__ float ld<float>(const float* p, long long i) { return p[i]; }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, long long i) {
    return __bfloat162float(p[i]);
}

enum { ACT_NONE = 0, ACT_RELU = 1, ACT_SIGMOID = 2 };

/* C[m,n] = act(sum_k A[m,k] B[k,n] + bias[n]) (+ C if accumulate), with
 * element (m,k) of A at A[m*am + k*ak] and (k,n) of B at B[k*bk + n*bn], so
 * transposed operands are just other strides.  64x64 tile per 256-thread
 * CTA, 4x4 outputs per thread, K staged through shared memory in 16s. */
template <class TA, class TB>
__global__ void __launch_bounds__(256) k_gemm(const TA* A, long long am, long long ak, const TB* B, long long bk,
                                              long long bn, float* C, long long cm, int M, int N, int K,
                                              const float* bias, int act, int accumulate) {
    __shared__ float As[16][64 + 1];
    __shared__ float Bs[16][64 + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            int kk = e / 64, mm = e % 64;
            int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? ld<TA>(A, (long long)m * am + (long long)k * ak) : 0.0f;
            int n = n0 + mm;
            Bs[kk][mm] = (n < N && k < K) ? ld<TB>(B, (long long)k * bk + (long long)n * bn) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) { a[i] = As[kk][ty * 4 + i]; b[i] = Bs[kk][tx * 4 + i]; }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j] + (bias ? bias[n] : 0.0f);
            if (accumulate) v += C[(long long)m * cm + n];
            if (act == ACT_RELU) v = fmaxf(v, 0.0f);
            else if (act == ACT_SIGMOID) v = 1.0f / (1.0f + expf(-v));
            C[(long long)m * cm + n] = v;
        }
    }
}

/* dZ = (p - y) / batch for sigmoid + BCE; loss partial sums */
__global__ void k_bce_grad(const float* P, const float* Y, float* dZ, long long n, float invB, float* loss) {
    float l = 0.0f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float p = P[i], y = Y[i];
        dZ[i] = (p - y) * invB;
        float pc = fminf(fmaxf(p, 1e-7f), 1.0f - 1e-7f);
        l -= y * logf(pc) + (1.0f - y) * logf(1.0f - pc);
    }
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * invB);
}
/* dX *= (X > 0) for ReLU layers (X = post-activation values) */
__global__ void k_relu_mask(float* d, const float* a, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (a[i] <= 0.0f) d[i] = 0.0f;
}
/* db[n] = sum_m dZ[m,n] */
__global__ void k_colsum(const float* dZ, int M, int N, float* db) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; m++) s += dZ[(long long)m * N + n];
    db[n] = s;
}
/* Adam on FP32 masters, refresh the BF16 copy */
__global__ void k_adam(float* w, __nv_bfloat16* wb, const float* g, float* m, float* v, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi; v[i] = vi;
        float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}
__global__ void k_to_bf16(const float* w, __nv_bfloat16* wb, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

/* ------------------------------------------------------------------------ */
/* Tensor-core GEMM (tcgen05, sm_100a)                                       */
/* ------------------------------------------------------------------------ */
/* The same contraction as k_gemm on the 5th-generation tensor cores: one
 * 128-thread CTA per 128 x 128 output tile.  Per 64-wide K step the CTA
 * converts its A and B tiles to BF16 and stores them in shared memory in
 * the tensor core's K-major, unswizzled layout (core matrices of 8 rows x
 * 16 bytes; the two 8-element halves of each 16-deep MMA step LBO bytes
 * apart, successive 8-row groups SBO bytes apart); one thread issues four
 * tcgen05.mma (M 128, N 128, K 16, BF16 x BF16 -> FP32) into a 128-column
 * tensor-memory accumulator and commits them to an mbarrier that every
 * thread waits on before the tiles are overwritten.  The epilogue reads the
 * accumulator back with tcgen05.ld (warp w owns rows 32w..32w+31), adds the
 * bias and applies the activation.  Waits are bounded: past the limit the
 * kernel records VT_MMA_TIMEOUT, frees its tensor memory and returns. */
#define TC_M 128
#define TC_N 128
#define TC_K 64
#define TC_SMEM (72 * 1024)   /* tiles use 32 KB; 72 KB keeps <= 3 CTAs (384 TMEM columns) per SM */

__device__ unsigned int g_mma_err;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

/* tensor-core shared-memory matrix descriptor: K-major, no swizzle */
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

/* element (row r, k) of a TC_K-deep tile with R rows, in core-matrix order */
__device__ __forceinline__ int tc_idx(int r, int k, int R) { return (((k >> 3) * (R >> 3) + (r >> 3)) << 6) + ((r & 7) << 3) + (k & 7); }

template <class T> __device__ __forceinline__ __nv_bfloat16 to_bf(T v);
template <> __device__ __forceinline__ __nv_bfloat16 to_bf<float>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_bf<__nv_bfloat16>(__nv_bfloat16 v) { return v; }

template <class TA, class TB>
__global__ void __launch_bounds__(128, 1) k_gemm_tc(const TA* A, long long am, long long ak, const TB* B, long long bk,
                                                    long long bn, float* C, long long cm, int M, int N, int K,
                                                    const float* bias, int act, int accumulate) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __nv_bfloat16* sA = (__nv_bfloat16*)tc_smem;                      /* TC_M x TC_K */
    __nv_bfloat16* sB = (__nv_bfloat16*)(tc_smem + TC_M * TC_K * 2);   /* TC_N x TC_K */
    unsigned long long* mbar = (unsigned long long*)(tc_smem + (TC_M + TC_N) * TC_K * 2);
    uint32_t* tslot = (uint32_t*)(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tslot)), "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    /* kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
     * K-major, N / 8 and M / 16 */
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);
    const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K && ok; k0 += TC_K) {
        /* stage the tiles (zero outside the matrices), walking the operand's
         * unit-stride dimension across the threads */
        for (int e = tid; e < TC_M * TC_K; e += 128) {
            int r, k;
            if (ak == 1) { r = e / TC_K; k = e % TC_K; } else { k = e / TC_M; r = e % TC_M; }
            const int m = m0 + r, kk = k0 + k;
            sA[tc_idx(r, k, TC_M)] = (m < M && kk < K) ? to_bf<TA>(A[(long long)m * am + (long long)kk * ak])
                                                       : __float2bfloat16_rn(0.0f);
        }
        for (int e = tid; e < TC_N * TC_K; e += 128) {
            int r, k;
            if (bn == 1) { k = e / TC_N; r = e % TC_N; } else { r = e / TC_K; k = e % TC_K; }
            const int n = n0 + r, kk = k0 + k;
            sB[tc_idx(r, k, TC_N)] = (n < N && kk < K) ? to_bf<TB>(B[(long long)kk * bk + (long long)n * bn])
                                                       : __float2bfloat16_rn(0.0f);
        }
        /* the tensor core reads shared memory through the async proxy */
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int j = 0; j < TC_K / 16; j++) {
                const uint64_t da = tc_desc(aBase + j * 2 * (TC_M / 8) * 128, (TC_M / 8) * 128, 128);
                const uint64_t db = tc_desc(bBase + j * 2 * (TC_N / 8) * 128, (TC_N / 8) * 128, 128);
                const uint32_t accum = (k0 > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(0), "r"(0), "r"(0), "r"(0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(mbar)));
        }
        /* every thread waits for the MMAs: the tiles are reused next step */
        uint32_t done = 0;
        for (long long it = 0; it < (1ll << 22) && !done; it++) {
            asm volatile("{\n\t.reg .pred P1;\n\t"
                         "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                         "selp.b32 %0, 1, 0, P1;\n\t}"
                         : "=r"(done) : "r"(smem_u32(mbar)), "r"(phase) : "memory");
        }
        if (!done) { atomicOr(&g_mma_err, 1u); ok = false; }
        phase ^= 1u;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < TC_N; c0 += 32) {
            uint32_t v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const int n = n0 + c0 + j;
                    if (n >= N) continue;
                    float x = __uint_as_float(v[j]) + (bias ? bias[n] : 0.0f);
                    if (accumulate) x += C[(long long)row * cm + n];
                    if (act == ACT_RELU) x = fmaxf(x, 0.0f);
                    else if (act == ACT_SIGMOID) x = 1.0f / (1.0f + expf(-x));
                    C[(long long)row * cm + n] = x;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TC_N));
}

static unsigned int g1(long long n) { long long b = (n + 255) / 256; return (unsigned int)(b > 4096 ? 4096 : (b < 1 ? 1 : b)); }

template <class TA, class TB>
static cudaError_t gemm(bool tc, const TA* A, long long am, long long ak, const TB* B, long long bk, long long bn,
                        float* C, long long cm, int M, int N, int K, const float* bias, int act, int acc, cudaStream_t s) {
    if (tc) {
        /* per launch (a cheap host call): the attribute belongs to the current device */
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
        if (e != cudaSuccess) return e;
        dim3 grid((N + TC_N - 1) / TC_N, (M + TC_M - 1) / TC_M);
        k_gemm_tc<TA, TB><<<grid, 128, TC_SMEM, s>>>(A, am, ak, B, bk, bn, C, cm, M, N, K, bias, act, acc);
        return cudaGetLastError();
    }
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_gemm<TA, TB><<<grid, 256, 0, s>>>(A, am, ak, B, bk, bn, C, cm, M, N, K, bias, act, acc);
    return cudaGetLastError();
}

}  // namespace vtm

using namespace vtm;

struct vt_mlp {
    int L = 3;
    int dims[4];                          /* in, h1, h2, out */
    float* w[3] = {}; __nv_bfloat16* wb[3] = {}; float* b[3] = {};       /* w[l]: dims[l] x dims[l+1] */
    float* gw[3] = {}; float* gb[3] = {};
    float* mw[3] = {}; float* vw[3] = {}; float* mb[3] = {}; float* vb[3] = {};
    float* act[4] = {};                   /* activations per layer (act[0] = input copy) */
    float* dact[4] = {};
    float* target = nullptr; float* loss = nullptr;
    int cap = 0;                          /* batch capacity of the activation buffers */
    long long step = 0;
    bool tc = true;                       /* GEMMs on the tensor cores (tcgen05); false: SIMT FMA */
};

/* a bounded tensor-core wait gave up (reported by the synchronising calls) */
static vt_status mma_status() {
    unsigned int e = 0;
    if (cudaMemcpyFromSymbol(&e, g_mma_err, sizeof(e)) != cudaSuccess) return vtrt::fail(VT_ERR_CUDA, "MLP status read");
    if (e) {
        e = 0;
        cudaMemcpyToSymbol(g_mma_err, &e, sizeof(e));
        return vtrt::fail(VT_ERR_TIMEOUT, "a tensor-core GEMM did not complete within its wait bound");
    }
    return VT_OK;
}

static vt_status mlp_buffers(vt_mlp* m, int batch) {
    if (batch <= m->cap) return VT_OK;
    for (int l = 0; l < 4; l++) { cudaFree(m->act[l]); cudaFree(m->dact[l]); m->act[l] = m->dact[l] = nullptr; }
    cudaFree(m->target);
    for (int l = 0; l < 4; l++) {
        CKM(cudaMalloc(&m->act[l], (size_t)batch * m->dims[l] * 4));
        CKM(cudaMalloc(&m->dact[l], (size_t)batch * m->dims[l] * 4));
    }
    CKM(cudaMalloc(&m->target, (size_t)batch * m->dims[3] * 4));
    m->cap = batch;
    return VT_OK;
}

extern "C" vt_status vt_mlp_create(int in, int h1, int h2, int out, uint64_t seed, vt_mlp** res) {
    vtrt::clear_error();
    if (!res || in <= 0 || h1 <= 0 || h2 <= 0 || out <= 0) return vtrt::fail(VT_ERR_INVALID, "bad MLP shape");
    vt_mlp* m = new vt_mlp();
    int d[4] = {in, h1, h2, out};
    memcpy(m->dims, d, sizeof(d));
    /* He initialisation (normal, std sqrt(2/fan_in)) from splitmix64 + Box-Muller; biases 0 */
    uint64_t k = vtrt::splitmix64(seed ^ 0x4D4C50ull);
    for (int l = 0; l < 3; l++) {
        long long n = (long long)d[l] * d[l + 1];
        std::vector<float> w(n);
        float sd = sqrtf(2.0f / (float)d[l]);
        for (long long i = 0; i < n; i++) {
            double u1 = ((vtrt::splitmix64(k++) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
            double u2 = (vtrt::splitmix64(k++) >> 11) * (1.0 / 9007199254740992.0);
            w[i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
        vt_status st = VT_OK;
        cudaError_t e = cudaSuccess;
        size_t nb = (size_t)d[l + 1] * 4;
        if ((e = cudaMalloc(&m->w[l], n * 4)) != cudaSuccess || (e = cudaMalloc(&m->wb[l], n * 2)) != cudaSuccess ||
            (e = cudaMalloc(&m->b[l], nb)) != cudaSuccess || (e = cudaMalloc(&m->gw[l], n * 4)) != cudaSuccess ||
            (e = cudaMalloc(&m->gb[l], nb)) != cudaSuccess || (e = cudaMalloc(&m->mw[l], n * 4)) != cudaSuccess ||
            (e = cudaMalloc(&m->vw[l], n * 4)) != cudaSuccess || (e = cudaMalloc(&m->mb[l], nb)) != cudaSuccess ||
            (e = cudaMalloc(&m->vb[l], nb)) != cudaSuccess) {
            st = vtrt::fail(VT_ERR_NOMEM, "MLP alloc: %s", cudaGetErrorString(e));
        }
        if (st == VT_OK) {
            cudaMemcpy(m->w[l], w.data(), n * 4, cudaMemcpyHostToDevice);
            cudaMemset(m->b[l], 0, nb);
            cudaMemset(m->mw[l], 0, n * 4); cudaMemset(m->vw[l], 0, n * 4);
            cudaMemset(m->mb[l], 0, nb); cudaMemset(m->vb[l], 0, nb);
            k_to_bf16<<<g1(n), 256>>>(m->w[l], m->wb[l], n);
            if ((e = cudaDeviceSynchronize()) != cudaSuccess) st = vtrt::fail(VT_ERR_CUDA, "MLP init: %s", cudaGetErrorString(e));
        }
        if (st != VT_OK) { vt_mlp_free(m); return st; }
    }
    if (cudaMalloc(&m->loss, 4) != cudaSuccess) { vt_mlp_free(m); return vtrt::fail(VT_ERR_NOMEM, "MLP loss"); }
    *res = m;
    return VT_OK;
}

extern "C" void vt_mlp_free(vt_mlp* m) {
    if (!m) return;
    for (int l = 0; l < 3; l++) {
        cudaFree(m->w[l]); cudaFree(m->wb[l]); cudaFree(m->b[l]); cudaFree(m->gw[l]); cudaFree(m->gb[l]);
        cudaFree(m->mw[l]); cudaFree(m->vw[l]); cudaFree(m->mb[l]); cudaFree(m->vb[l]);
    }
    for (int l = 0; l < 4; l++) { cudaFree(m->act[l]); cudaFree(m->dact[l]); }
    cudaFree(m->target); cudaFree(m->loss);
    delete m;
}

/* forward pass for `batch` rows of dev_x (batch x in, FP32); output probabilities */
static vt_status forward(vt_mlp* m, const float* x, int batch, cudaStream_t s) {
    vt_status st = mlp_buffers(m, batch);
    if (st != VT_OK) return st;
    const int* d = m->dims;
    CKM(cudaMemcpyAsync(m->act[0], x, (size_t)batch * d[0] * 4, cudaMemcpyDeviceToDevice, s));
    for (int l = 0; l < 3; l++)
        CKM((gemm<float, __nv_bfloat16>(m->tc, m->act[l], d[l], 1, m->wb[l], d[l + 1], 1, m->act[l + 1], d[l + 1], batch,
                                       d[l + 1], d[l], m->b[l], l < 2 ? ACT_RELU : ACT_SIGMOID, 0, s)));
    return VT_OK;
}

extern "C" vt_status vt_mlp_forward(vt_mlp* m, const float* dev_x, int batch, float* dev_p, void* stream) {
    vtrt::clear_error();
    if (!m || !dev_x || !dev_p || batch <= 0) return vtrt::fail(VT_ERR_INVALID, "vt_mlp_forward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    vt_status st = forward(m, dev_x, batch, s);
    if (st != VT_OK) return st;
    CKM(cudaMemcpyAsync(dev_p, m->act[3], (size_t)batch * m->dims[3] * 4, cudaMemcpyDeviceToDevice, s));
    return VT_OK;
}

/* gradients of the mean BCE over the batch into gw/gb; loss into m->loss */
static vt_status backward(vt_mlp* m, const float* y, int batch, cudaStream_t s) {
    const int* d = m->dims;
    long long no = (long long)batch * d[3];
    CKM(cudaMemsetAsync(m->loss, 0, 4, s));
    k_bce_grad<<<g1(no), 256, 0, s>>>(m->act[3], y, m->dact[3], no, 1.0f / batch, m->loss);
    for (int l = 2; l >= 0; l--) {
        /* gW[l] = act[l]^T dact[l+1]   (d[l] x d[l+1]) */
        CKM((gemm<float, float>(m->tc, m->act[l], 1, d[l], m->dact[l + 1], d[l + 1], 1, m->gw[l], d[l + 1], d[l], d[l + 1],
                               batch, nullptr, ACT_NONE, 0, s)));
        k_colsum<<<(d[l + 1] + 255) / 256, 256, 0, s>>>(m->dact[l + 1], batch, d[l + 1], m->gb[l]);
        if (l > 0) {
            /* dact[l] = dact[l+1] W[l]^T, masked by ReLU */
            CKM((gemm<float, __nv_bfloat16>(m->tc, m->dact[l + 1], d[l + 1], 1, m->wb[l], 1, d[l + 1], m->dact[l], d[l], batch,
                                           d[l], d[l + 1], nullptr, ACT_NONE, 0, s)));
            k_relu_mask<<<g1((long long)batch * d[l]), 256, 0, s>>>(m->dact[l], m->act[l], (long long)batch * d[l]);
        }
    }
    CKM(cudaGetLastError());
    return VT_OK;
}

extern "C" vt_status vt_mlp_train_step(vt_mlp* m, const float* dev_x, const float* dev_y, int batch, float lr,
                                       float* loss, void* stream) {
    vtrt::clear_error();
    if (!m || !dev_x || !dev_y || batch <= 0) return vtrt::fail(VT_ERR_INVALID, "vt_mlp_train_step: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    vt_status st = forward(m, dev_x, batch, s);
    if (st != VT_OK) return st;
    if ((st = backward(m, dev_y, batch, s)) != VT_OK) return st;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
    for (int l = 0; l < 3; l++) {
        long long n = (long long)m->dims[l] * m->dims[l + 1];
        k_adam<<<g1(n), 256, 0, s>>>(m->w[l], m->wb[l], m->gw[l], m->mw[l], m->vw[l], n, lr, b1, b2, 1e-8f, c1, c2);
        k_adam<<<g1(m->dims[l + 1]), 256, 0, s>>>(m->b[l], nullptr, m->gb[l], m->mb[l], m->vb[l], m->dims[l + 1], lr,
                                                  b1, b2, 1e-8f, c1, c2);
    }
    CKM(cudaGetLastError());
    if (loss) {
        CKM(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, s));
        CKM(cudaStreamSynchronize(s));
        return mma_status();
    }
    return VT_OK;
}

/* gradients only (no update), for checking against a CPU implementation:
 * host buffers laid out as the weights (layer by layer: W then b) */
extern "C" vt_status vt_mlp_gradients(vt_mlp* m, const float* dev_x, const float* dev_y, int batch, float* host_grads,
                                      float* loss) {
    vtrt::clear_error();
    if (!m || !dev_x || !dev_y || !host_grads || batch <= 0) return vtrt::fail(VT_ERR_INVALID, "bad arguments");
    vt_status st = forward(m, dev_x, batch, 0);
    if (st != VT_OK) return st;
    if ((st = backward(m, dev_y, batch, 0)) != VT_OK) return st;
    CKM(cudaDeviceSynchronize());
    size_t o = 0;
    for (int l = 0; l < 3; l++) {
        size_t n = (size_t)m->dims[l] * m->dims[l + 1];
        CKM(cudaMemcpy(host_grads + o, m->gw[l], n * 4, cudaMemcpyDeviceToHost)); o += n;
        CKM(cudaMemcpy(host_grads + o, m->gb[l], (size_t)m->dims[l + 1] * 4, cudaMemcpyDeviceToHost)); o += m->dims[l + 1];
    }
    if (loss) CKM(cudaMemcpy(loss, m->loss, 4, cudaMemcpyDeviceToHost));
    return mma_status();
}

extern "C" vt_status vt_mlp_use_tensor_cores(vt_mlp* m, int on) {
    vtrt::clear_error();
    if (!m) return vtrt::fail(VT_ERR_INVALID, "null argument");
    m->tc = on != 0;
    return VT_OK;
}

extern "C" vt_status vt_mlp_info(const vt_mlp* m, int dims[4]) {
    vtrt::clear_error();
    if (!m || !dims) return vtrt::fail(VT_ERR_INVALID, "null argument");
    memcpy(dims, m->dims, sizeof(m->dims));
    return VT_OK;
}

/* FP32 master weights (layer by layer: W [in x out] then b [out]) */
extern "C" vt_status vt_mlp_get_weights(vt_mlp* m, float* host, int64_t* n) {
    vtrt::clear_error();
    if (!m || !n) return vtrt::fail(VT_ERR_INVALID, "null argument");
    int64_t total = 0;
    for (int l = 0; l < 3; l++) total += (int64_t)m->dims[l] * m->dims[l + 1] + m->dims[l + 1];
    int64_t cap = *n;
    *n = total;
    if (!host) return VT_OK;
    if (cap < total) return vtrt::fail(VT_ERR_INVALID, "need %lld floats", (long long)total);
    CKM(cudaDeviceSynchronize());
    size_t o = 0;
    for (int l = 0; l < 3; l++) {
        size_t nw = (size_t)m->dims[l] * m->dims[l + 1];
        CKM(cudaMemcpy(host + o, m->w[l], nw * 4, cudaMemcpyDeviceToHost)); o += nw;
        CKM(cudaMemcpy(host + o, m->b[l], (size_t)m->dims[l + 1] * 4, cudaMemcpyDeviceToHost)); o += m->dims[l + 1];
    }
    return VT_OK;
}

extern "C" vt_status vt_mlp_set_weights(vt_mlp* m, const float* host, int64_t n) {
    vtrt::clear_error();
    if (!m || !host) return vtrt::fail(VT_ERR_INVALID, "null argument");
    int64_t total = 0;
    for (int l = 0; l < 3; l++) total += (int64_t)m->dims[l] * m->dims[l + 1] + m->dims[l + 1];
    if (n != total) return vtrt::fail(VT_ERR_INVALID, "expected %lld floats", (long long)total);
    size_t o = 0;
    for (int l = 0; l < 3; l++) {
        size_t nw = (size_t)m->dims[l] * m->dims[l + 1];
        CKM(cudaMemcpy(m->w[l], host + o, nw * 4, cudaMemcpyHostToDevice)); o += nw;
        CKM(cudaMemcpy(m->b[l], host + o, (size_t)m->dims[l + 1] * 4, cudaMemcpyHostToDevice)); o += m->dims[l + 1];
        k_to_bf16<<<g1((long long)nw), 256>>>(m->w[l], m->wb[l], (long long)nw);
    }
    CKM(cudaDeviceSynchronize());
    return VT_OK;
}

/* ------------------------------------------------------------------------ */
/* Allocation-free inference                                                */
/* ------------------------------------------------------------------------ */
/* Some callers cannot allocate GPU memory at the point where they run the
 * prefetch network: a render loop inside a host application that owns the
 * device's memory (its own pool, a fixed budget), or a frame thread that
 * must not call cudaMalloc because it synchronises the device and can stall
 * the frame.  vt_mlp_forward_noalloc serves them: its two hidden-layer
 * activations live in this fixed, file-scope device array instead of the
 * handle's lazily allocated buffers.  Every GPU that loads libvt.so holds
 * the array (1 MiB) until the process exits. */
#define VT_MLP_NOALLOC_FLOATS (1 << 18)
static __device__ __align__(256) float g_mlp_noalloc_scratch[VT_MLP_NOALLOC_FLOATS];

#include <mutex>
static std::mutex g_noalloc_mu;
static float* g_noalloc_dev[256];   /* per device: address of the array, looked up once */

extern "C" vt_status vt_mlp_forward_noalloc(vt_mlp* m, const float* dev_x, int batch, float* dev_p, void* stream) {
    vtrt::clear_error();
    if (!m || !dev_x || !dev_p || batch <= 0) return vtrt::fail(VT_ERR_INVALID, "vt_mlp_forward_noalloc: bad arguments");
    const int* d = m->dims;
    long long need = (long long)batch * (d[1] + d[2]);
    if (need > VT_MLP_NOALLOC_FLOATS)
        return vtrt::fail(VT_ERR_INVALID,
                          "vt_mlp_forward_noalloc: batch %d x (%d + %d) hidden units = %lld floats exceeds the "
                          "static scratch of %d floats", batch, d[1], d[2], need, VT_MLP_NOALLOC_FLOATS);
    int dev = 0;
    CKM(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return vtrt::fail(VT_ERR_UNSUPPORTED, "device ordinal %d", dev);
    float* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (g_noalloc_dev[dev]) {
            /* an address looked up before a cudaDeviceReset belongs to the
             * destroyed context: the runtime no longer knows it as device
             * memory of this device, so it is looked up again (a host query,
             * no allocation) */
            cudaPointerAttributes pa;
            if (cudaPointerGetAttributes(&pa, g_noalloc_dev[dev]) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
                pa.device != dev) {
                cudaGetLastError();
                g_noalloc_dev[dev] = nullptr;
            }
        }
        if (!g_noalloc_dev[dev]) {
            /* host code only sees a stand-in for the array: its device address
             * comes from the runtime, once per device (and context), with
             * that device current */
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_mlp_noalloc_scratch);
            if (e != cudaSuccess)
                return vtrt::fail(VT_ERR_CUDA, "cudaGetSymbolAddress(g_mlp_noalloc_scratch): %s", cudaGetErrorString(e));
            g_noalloc_dev[dev] = (float*)p;
        }
        scratch = g_noalloc_dev[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    float* h1 = scratch;
    float* h2 = scratch + (size_t)batch * d[1];
    /* every activation element is written before it is read, so the array's
     * leftovers from the previous call need no clearing */
    CKM((gemm<float, __nv_bfloat16>(m->tc, dev_x, d[0], 1, m->wb[0], d[1], 1, h1, d[1], batch, d[1], d[0], m->b[0],
                                    ACT_RELU, 0, s)));
    CKM((gemm<float, __nv_bfloat16>(m->tc, h1, d[1], 1, m->wb[1], d[2], 1, h2, d[2], batch, d[2], d[1], m->b[1],
                                    ACT_RELU, 0, s)));
    CKM((gemm<float, __nv_bfloat16>(m->tc, h2, d[2], 1, m->wb[2], d[3], 1, dev_p, d[3], batch, d[3], d[2], m->b[2],
                                    ACT_SIGMOID, 0, s)));
    return VT_OK;
}
