/*
 * gen.cu -- seeded synthetic volumes, on the device (full size, into HBM)
 * and on the host (test sizes).  No reference counterpart: the reference
 * renders external HDF5 data.
 *
 *   sphere  : |x-c| + sigma*g, g a 4-term Irwin-Hall normal from splitmix64
 *             counters; bit-identical host/device (no contraction, exact
 *             integer sum, correctly rounded sqrt).
 *   blobs   : sum of anisotropic Gaussian blobs + 4-octave value noise.
 *   fractal : 6-octave value noise quantised to 0..255 plus spheres of a
 *             constant value (uint8).
 * Blob/fractal values use expf, so host and device agree to a few ulp only;
 * full-size volumes are always generated on the device.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/vt.h"
#include "vt_runtime.h"

#define HD __host__ __device__ __forceinline__

namespace vtgen {

HD uint64_t sm64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
HD float u01(uint64_t h) { return (float)(h >> 40) * 5.9604644775390625e-08f; }   /* [0,1) */

HD float sphere_voxel(uint64_t seed, long long x, long long y, long long z, long long dy, long long dz,
                      float cx, float cy, float cz, float sigma) {
    float dxv = (float)x - cx, dyv = (float)y - cy, dzv = (float)z - cz;
    float r = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv);
    uint64_t k = (uint64_t)((x * dy + y) * dz + z);
    uint64_t r0 = sm64(seed + 2 * k), r1 = sm64(seed + 2 * k + 1);
    uint32_t S = (uint32_t)(r0 >> 40) + (uint32_t)((r0 >> 16) & 0xFFFFFFu) + (uint32_t)(r1 >> 40) +
                 (uint32_t)((r1 >> 16) & 0xFFFFFFu);
    float g = ((float)S * 5.9604644775390625e-08f - 2.0f) * 1.7320508075688772f;
    return r + sigma * g;
}

/* value noise: lattice values in [-1,1) at integer lattice points of cell
 * size `cell`, smoothstep-weighted trilinear interpolation */
HD float lattice(uint64_t seed, long long ix, long long iy, long long iz, int oct) {
    uint64_t key = ((((uint64_t)ix * 1048583ull) + (uint64_t)iy) * 1048589ull + (uint64_t)iz) * 16ull + (uint64_t)oct;
    return u01(sm64(seed ^ 0x5bd1e9955bd1e995ull) ^ sm64(key)) * 2.0f - 1.0f;
}
HD float smooth(float t) { return t * t * (3.0f - 2.0f * t); }
HD float value_noise(uint64_t seed, float x, float y, float z, float cell, int oct) {
    float fx = x / cell, fy = y / cell, fz = z / cell;
    float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
    long long ix = (long long)flx, iy = (long long)fly, iz = (long long)flz;
    float tx = smooth(fx - flx), ty = smooth(fy - fly), tz = smooth(fz - flz);
    float v000 = lattice(seed, ix, iy, iz, oct), v001 = lattice(seed, ix, iy, iz + 1, oct);
    float v010 = lattice(seed, ix, iy + 1, iz, oct), v011 = lattice(seed, ix, iy + 1, iz + 1, oct);
    float v100 = lattice(seed, ix + 1, iy, iz, oct), v101 = lattice(seed, ix + 1, iy, iz + 1, oct);
    float v110 = lattice(seed, ix + 1, iy + 1, iz, oct), v111 = lattice(seed, ix + 1, iy + 1, iz + 1, oct);
    float a00 = v000 + (v100 - v000) * tx, a01 = v001 + (v101 - v001) * tx;
    float a10 = v010 + (v110 - v010) * tx, a11 = v011 + (v111 - v011) * tx;
    float b0 = a00 + (a10 - a00) * ty, b1 = a01 + (a11 - a01) * ty;
    return b0 + (b1 - b0) * tz;
}
HD float fractal(uint64_t seed, float x, float y, float z, float cell, int octaves) {
    float sum = 0.0f, amp = 1.0f, norm = 0.0f;
    for (int o = 0; o < octaves; o++) {
        sum += amp * value_noise(seed, x, y, z, cell, o);
        norm += amp;
        amp *= 0.5f;
        cell *= 0.5f;
    }
    return sum / norm;
}

struct Blob { float cx, cy, cz, ix2, iy2, iz2, amp; };   /* ixx2 = 0.5/sigma^2 */
#define VT_MAX_BLOBS 1024
#define VT_MAX_SPHERES 256

HD float blobs_voxel(const Blob* b, int nb, uint64_t seed, float noiseAmp, float x, float y, float z) {
    float v = 0.0f;
    for (int i = 0; i < nb; i++) {
        float dx = x - b[i].cx, dy = y - b[i].cy, dz = z - b[i].cz;
        float e = dx * dx * b[i].ix2 + dy * dy * b[i].iy2 + dz * dz * b[i].iz2;
        if (e < 40.0f) v += b[i].amp * expf(-e);
    }
    return v + noiseAmp * fractal(seed, x, y, z, 128.0f, 4);
}

struct Sph { float cx, cy, cz, r2; };
HD uint8_t fractal_voxel(const Sph* s, int ns, uint8_t sval, uint64_t seed, float x, float y, float z) {
    for (int i = 0; i < ns; i++) {
        float dx = x - s[i].cx, dy = y - s[i].cy, dz = z - s[i].cz;
        if (dx * dx + dy * dy + dz * dz < s[i].r2) return sval;
    }
    float f = fractal(seed, x, y, z, 256.0f, 6);        /* [-1,1] */
    float u = 0.5f + 0.5f * f;
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    return (uint8_t)(u * 255.0f + 0.5f);
}

/* blob / sphere parameters drawn from the seed (host) */
static int make_blobs(uint64_t seed, const int64_t dims[3], const float* prm, int np, std::vector<Blob>& out,
                      float* noiseAmp) {
    int nb = np > 0 ? (int)prm[0] : 256;
    float smin = np > 1 ? prm[1] : 20.0f, smax = np > 2 ? prm[2] : 120.0f;
    float amin = np > 3 ? prm[3] : 0.5f, amax = np > 4 ? prm[4] : 1.5f;
    *noiseAmp = np > 5 ? prm[5] : 0.05f;
    if (nb < 0 || nb > VT_MAX_BLOBS) return -1;
    out.resize(nb);
    uint64_t k = sm64(seed ^ 0xB10B5ull);
    for (int i = 0; i < nb; i++) {
        float u[7];
        for (int j = 0; j < 7; j++) u[j] = u01(sm64(k + (uint64_t)(i * 7 + j)));
        Blob& b = out[i];
        b.cx = u[0] * (float)dims[0]; b.cy = u[1] * (float)dims[1]; b.cz = u[2] * (float)dims[2];
        float sx = smin + (smax - smin) * u[3], sy = smin + (smax - smin) * u[4], sz = smin + (smax - smin) * u[5];
        b.ix2 = 0.5f / (sx * sx); b.iy2 = 0.5f / (sy * sy); b.iz2 = 0.5f / (sz * sz);
        b.amp = amin + (amax - amin) * u[6];
    }
    return 0;
}
static int make_spheres(uint64_t seed, const int64_t dims[3], const float* prm, int np, std::vector<Sph>& out,
                        uint8_t* sval) {
    int ns = np > 0 ? (int)prm[0] : 32;
    float rmin = np > 1 ? prm[1] : 50.0f, rmax = np > 2 ? prm[2] : 400.0f;
    *sval = (uint8_t)(np > 3 ? prm[3] : 200.0f);
    if (ns < 0 || ns > VT_MAX_SPHERES) return -1;
    out.resize(ns);
    uint64_t k = sm64(seed ^ 0x5FE4Eull);
    for (int i = 0; i < ns; i++) {
        float u[4];
        for (int j = 0; j < 4; j++) u[j] = u01(sm64(k + (uint64_t)(i * 4 + j)));
        float r = rmin + (rmax - rmin) * u[3];
        out[i].cx = u[0] * (float)dims[0]; out[i].cy = u[1] * (float)dims[1]; out[i].cz = u[2] * (float)dims[2];
        out[i].r2 = r * r;
    }
    return 0;
}

__constant__ Blob c_blobs[VT_MAX_BLOBS];
__constant__ Sph c_sph[VT_MAX_SPHERES];

__global__ void k_sphere(float* out, uint64_t seed, long long nx, long long ny, long long nz, float cx, float cy,
                         float cz, float sigma) {
    long long n = nx * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long z = i % nz, t = i / nz, y = t % ny, x = t / ny;
        out[i] = sphere_voxel(seed, x, y, z, ny, nz, cx, cy, cz, sigma);
    }
}
__global__ void k_blobs(float* out, int nb, uint64_t seed, float noiseAmp, long long nx, long long ny, long long nz) {
    long long n = nx * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long z = i % nz, t = i / nz, y = t % ny, x = t / ny;
        out[i] = blobs_voxel(c_blobs, nb, seed, noiseAmp, (float)x, (float)y, (float)z);
    }
}
__global__ void k_fractal(uint8_t* out, int ns, uint8_t sval, uint64_t seed, long long nx, long long ny, long long nz) {
    long long n = nx * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long z = i % nz, t = i / nz, y = t % ny, x = t / ny;
        out[i] = fractal_voxel(c_sph, ns, sval, seed, (float)x, (float)y, (float)z);
    }
}

}  // namespace vtgen

using namespace vtgen;

extern "C" vt_status vt_generate_volume(int kind, uint64_t seed, const int64_t dims[3], const float* params,
                                        int nparams, void* out) {
    vtrt::clear_error();
    if (!dims || !out) return vtrt::fail(VT_ERR_INVALID, "vt_generate_volume: null argument");
    const long long nx = dims[0], ny = dims[1], nz = dims[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return vtrt::fail(VT_ERR_INVALID, "bad dims");
    if (kind == VT_GEN_SPHERE) {
        float c[4] = {(float)(nx - 1) * 0.5f, (float)(ny - 1) * 0.5f, (float)(nz - 1) * 0.5f, 0.25f};
        for (int i = 0; i < nparams && i < 4; i++) c[i] = params[i];
        float* o = (float*)out;
#pragma omp parallel for schedule(static)
        for (long long x = 0; x < nx; x++)
            for (long long y = 0; y < ny; y++)
                for (long long z = 0; z < nz; z++)
                    o[(x * ny + y) * nz + z] = sphere_voxel(seed, x, y, z, ny, nz, c[0], c[1], c[2], c[3]);
        return VT_OK;
    }
    if (kind == VT_GEN_BLOBS) {
        std::vector<Blob> b;
        float na;
        if (make_blobs(seed, dims, params, nparams, b, &na) != 0) return vtrt::fail(VT_ERR_INVALID, "bad blob parameters");
        float* o = (float*)out;
#pragma omp parallel for schedule(static)
        for (long long x = 0; x < nx; x++)
            for (long long y = 0; y < ny; y++)
                for (long long z = 0; z < nz; z++)
                    o[(x * ny + y) * nz + z] = blobs_voxel(b.data(), (int)b.size(), seed, na, (float)x, (float)y, (float)z);
        return VT_OK;
    }
    if (kind == VT_GEN_FRACTAL_U8) {
        std::vector<Sph> sp;
        uint8_t sv;
        if (make_spheres(seed, dims, params, nparams, sp, &sv) != 0) return vtrt::fail(VT_ERR_INVALID, "bad sphere parameters");
        uint8_t* o = (uint8_t*)out;
#pragma omp parallel for schedule(static)
        for (long long x = 0; x < nx; x++)
            for (long long y = 0; y < ny; y++)
                for (long long z = 0; z < nz; z++)
                    o[(x * ny + y) * nz + z] = fractal_voxel(sp.data(), (int)sp.size(), sv, seed, (float)x, (float)y, (float)z);
        return VT_OK;
    }
    return vtrt::fail(VT_ERR_INVALID, "unknown generator %d", kind);
}

extern "C" vt_status vt_generate_volume_device(int kind, uint64_t seed, const int64_t dims[3], const float* params,
                                               int nparams, void* dev_out, void* stream) {
    vtrt::clear_error();
    if (!dims || !dev_out) return vtrt::fail(VT_ERR_INVALID, "vt_generate_volume_device: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned int blocks = 148 * 16, threads = 256;
    cudaError_t e;
    if (kind == VT_GEN_SPHERE) {
        float c[4] = {(float)(dims[0] - 1) * 0.5f, (float)(dims[1] - 1) * 0.5f, (float)(dims[2] - 1) * 0.5f, 0.25f};
        for (int i = 0; i < nparams && i < 4; i++) c[i] = params[i];
        k_sphere<<<blocks, threads, 0, s>>>((float*)dev_out, seed, dims[0], dims[1], dims[2], c[0], c[1], c[2], c[3]);
    } else if (kind == VT_GEN_BLOBS) {
        std::vector<Blob> b;
        float na;
        if (make_blobs(seed, dims, params, nparams, b, &na) != 0) return vtrt::fail(VT_ERR_INVALID, "bad blob parameters");
        if (!b.empty() && (e = cudaMemcpyToSymbolAsync(c_blobs, b.data(), b.size() * sizeof(Blob), 0,
                                                       cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return vtrt::fail(VT_ERR_CUDA, "blob upload: %s", cudaGetErrorString(e));
        k_blobs<<<blocks, threads, 0, s>>>((float*)dev_out, (int)b.size(), seed, na, dims[0], dims[1], dims[2]);
        /* the constant bank is reused by the next call: finish before returning */
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return vtrt::fail(VT_ERR_CUDA, "blobs: %s", cudaGetErrorString(e));
    } else if (kind == VT_GEN_FRACTAL_U8) {
        std::vector<Sph> sp;
        uint8_t sv;
        if (make_spheres(seed, dims, params, nparams, sp, &sv) != 0) return vtrt::fail(VT_ERR_INVALID, "bad sphere parameters");
        if (!sp.empty() && (e = cudaMemcpyToSymbolAsync(c_sph, sp.data(), sp.size() * sizeof(Sph), 0,
                                                        cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return vtrt::fail(VT_ERR_CUDA, "sphere upload: %s", cudaGetErrorString(e));
        k_fractal<<<blocks, threads, 0, s>>>((uint8_t*)dev_out, (int)sp.size(), sv, seed, dims[0], dims[1], dims[2]);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return vtrt::fail(VT_ERR_CUDA, "fractal: %s", cudaGetErrorString(e));
    } else {
        return vtrt::fail(VT_ERR_INVALID, "unknown generator %d", kind);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return vtrt::fail(VT_ERR_CUDA, "generator launch: %s", cudaGetErrorString(e));
    return VT_OK;
}
