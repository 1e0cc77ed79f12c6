/*
 * mlp.cu -- the brick-prefetch network of libvt.so (no reference
 * counterpart): pose features (12) -> 512 -> 512 -> 4096 sigmoid, one
 * output per coarse octree node, trained with binary cross-entropy on
 * traces of the nodes each frame marched.
 *
 * Weights are stored in BF16 (what the forward and backward GEMMs read) with
 * FP32 master copies updated by Adam; every GEMM accumulates in FP32.
 * Activations are FP32.  The network is tiny (4.73 MFLOP per pose), so the
 * GEMMs are register-tiled SIMT kernels: inference of one pose per frame is
 * latency-bound and training 20k poses takes well under a second.
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

static unsigned int g1(long long n) { long long b = (n + 255) / 256; return (unsigned int)(b > 4096 ? 4096 : (b < 1 ? 1 : b)); }

template <class TA, class TB>
static cudaError_t gemm(const TA* A, long long am, long long ak, const TB* B, long long bk, long long bn, float* C,
                        long long cm, int M, int N, int K, const float* bias, int act, int acc, cudaStream_t s) {
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
};

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
        CKM((gemm<float, __nv_bfloat16>(m->act[l], d[l], 1, m->wb[l], d[l + 1], 1, m->act[l + 1], d[l + 1], batch,
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
        CKM((gemm<float, float>(m->act[l], 1, d[l], m->dact[l + 1], d[l + 1], 1, m->gw[l], d[l + 1], d[l], d[l + 1],
                               batch, nullptr, ACT_NONE, 0, s)));
        k_colsum<<<(d[l + 1] + 255) / 256, 256, 0, s>>>(m->dact[l + 1], batch, d[l + 1], m->gb[l]);
        if (l > 0) {
            /* dact[l] = dact[l+1] W[l]^T, masked by ReLU */
            CKM((gemm<float, __nv_bfloat16>(m->dact[l + 1], d[l + 1], 1, m->wb[l], 1, d[l + 1], m->dact[l], d[l], batch,
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
    CKM((gemm<float, __nv_bfloat16>(dev_x, d[0], 1, m->wb[0], d[1], 1, h1, d[1], batch, d[1], d[0], m->b[0],
                                    ACT_RELU, 0, s)));
    CKM((gemm<float, __nv_bfloat16>(h1, d[1], 1, m->wb[1], d[2], 1, h2, d[2], batch, d[2], d[1], m->b[1],
                                    ACT_RELU, 0, s)));
    CKM((gemm<float, __nv_bfloat16>(h2, d[2], 1, m->wb[2], d[3], 1, dev_p, d[3], batch, d[3], d[2], m->b[2],
                                    ACT_SIGMOID, 0, s)));
    return VT_OK;
}
