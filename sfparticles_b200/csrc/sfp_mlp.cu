// sfp_mlp.cu -- the learned photon-energy sampler of the optical-depth method
// (no counterpart in the reference).  An MLP (log10 chi, u) -> delta stands in
// for the inverse-CDF table sampler _bisect_interp
// (qed/optical_depth_tables.py:59-102) when it is selected.  This file holds
// the batched table sampler the MLP is trained on and judged against, the
// training kernels and the tensor-core inference kernel.
//
// Network: features x = (log10 chi / 3, logit(u) / 8) -> 64 -> 64 -> 64 -> 1
// with SiLU on the hidden layers; output y, delta = 10^(3 (y - 1)) clamped to
// [1e-6, 1] (training target y = log10(delta) / 3 + 1).  The logit feature
// log(u / (1 - u)) is linear in both ends of the inverse CDF: delta ~ u^3 as
// u -> 0 and an exponential tail as u -> 1.
//
// Parameters, 8577 float32:
//   W0[64][2] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[64] b3
// Row j of W holds the weights of output unit j.
//
// Inference (sfp_mlp.cuh): weights in BF16, FP32 accumulation; the two
// 64x64 layers run on the tensor cores (mma.sync m16n8k16).
//
// Training: FP32 master weights.  The forward pass uses the weights rounded to
// BF16, as inference does, and FP32 activations; the gradient is taken with
// respect to those rounded weights and applied to the master weights.  Each
// block runs fused forward + backward passes over 64-sample tiles; an Adam
// step follows.
#include <cuda_runtime.h>

#include <string>

#include "sfp.h"
#include "sfp_device.cuh"
#include "sfp_internal.h"
#include "sfp_mlp.cuh"

namespace {

using sfp_mlp::H;
using sfp_mlp::NP;
using sfp_mlp::OB0;
using sfp_mlp::OB1;
using sfp_mlp::OB2;
using sfp_mlp::OB3;
using sfp_mlp::OW0;
using sfp_mlp::OW1;
using sfp_mlp::OW2;
using sfp_mlp::OW3;
using sfp_mlp::bf16r;
using sfp_mlp::feat_chi;
using sfp_mlp::feat_u;
static_assert(H == SFP_MLP_HIDDEN && NP == SFP_MLP_NPARAM, "parameter count");

#define MLP_CUDA(call)                                                                                         \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return sfp_set_error(SFP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int sm_count_here() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
}


// training activation: SiLU with its exact derivative
__device__ __forceinline__ void silu_train(float z, float& a, float& d) {
    const float s = 1.0f / (1.0f + expf(-z));
    a = z * s;
    d = s * (1.0f + z * (1.0f - s));
}

// ------------------------------------------------------------------ tables
__global__ void k_od_inverse_cdf(sfp_od_table t, const double* __restrict__ lc, const double* __restrict__ u,
                                 double* __restrict__ d, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = sfp::od_bisect(pow(10.0, lc[i]), u[i], t);
}

// training samples: Philox purpose 3, counter step = chunk.  log10 chi is
// uniform; u is uniform for three samples in four and drawn from the tail
// (1 - u log-uniform in [1e-8, 1e-1], the hardest photons) for the fourth,
// so that the fit resolves the tail that high spectral moments and pair
// creation depend on.
__global__ void k_mlp_samples(sfp_od_table t, unsigned long long seed, unsigned int chunk, double lo, double hi,
                              long long n, float* __restrict__ feat, float* __restrict__ target) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double r1, r2, r3, r4;
        sfp::uniform2(seed, 0u, chunk, 3u, i, r1, r2);
        sfp::uniform2(seed, 1u, chunk, 3u, i, r3, r4);
        if (r3 < 0.25) r2 = 1.0 - exp10(-1.0 - 7.0 * r4);
        const double a = lo + (hi - lo) * r1;
        const double d = sfp::od_bisect(pow(10.0, a), r2, t);
        feat[2 * i] = feat_chi(a);
        feat[2 * i + 1] = feat_u(r2);
        target[i] = (float)(log10(d) / 3.0 + 1.0);
    }
}

// ---------------------------------------------------------------- training
// One block of 256 threads per SM; 64-sample tiles.  Thread (ty, tx) =
// (tid / 16, tid % 16) owns samples ty + 16 a and units tx + 16 b
// (a, b = 0..3) of every 64 x 64 tile product, and the weight-gradient
// entries (j = tx + 16 b, i = ty + 16 a) of W1 and W2.
constexpr int TS = 64;   // samples per tile
constexpr int LD = H + 1;  // padded row stride of the smem matrices

struct TrainSmem {
    float W1[H][LD], W2[H][LD];   // BF16-rounded forward weights
    float A1[TS][LD], A2[TS][LD], A3[TS][LD];
    float D1[TS][LD], D2[TS][LD], D3[TS][LD];  // silu'(z), then dL/dz in place
    float W0[H][2], b0[H], b1[H], b2[H], W3[H];
    float x[TS][2], y[TS], dy[TS];
    float gW0[H][2], gb0[H], gb1[H], gb2[H], gW3[H];
    float gb3, b3;
    double loss;
};

// out[s][j] = sum_i W[j][i] in[s][i] + b[j]  ->  A = silu, D = silu'
__device__ __forceinline__ void dense_fwd(const float (*W)[LD], const float* b, const float (*in)[LD],
                                          float (*A)[LD], float (*D)[LD], int ty, int tx) {
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = b[tx + 16 * q];
#pragma unroll 4
    for (int i = 0; i < H; ++i) {
        float xi[4], wi[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) xi[a] = in[ty + 16 * a][i];
#pragma unroll
        for (int q = 0; q < 4; ++q) wi[q] = W[tx + 16 * q][i];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] = fmaf(wi[q], xi[a], acc[a][q]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) silu_train(acc[a][q], A[ty + 16 * a][tx + 16 * q], D[ty + 16 * a][tx + 16 * q]);
}

// backward through a 64 -> 64 layer: dZ (in Dout, per sample and output unit),
// input activations Ain; accumulates gW (registers) and gb (smem); writes
// dL/dz of the layer below into Din (Din *= W^T dZ).
__device__ __forceinline__ void dense_bwd(const float (*W)[LD], const float (*Dout)[LD], const float (*Ain)[LD],
                                          float (*Din)[LD], float (&gW)[4][4], float* gb, int ty, int tx, int tid,
                                          bool below) {
    // weight gradient: gW[j][i] += sum_s dZ[s][j] Ain[s][i]   (j = tx + 16 q, i = ty + 16 a)
#pragma unroll 4
    for (int s = 0; s < TS; ++s) {
        float dz[4], ai[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) dz[q] = Dout[s][tx + 16 * q];
#pragma unroll
        for (int a = 0; a < 4; ++a) ai[a] = Ain[s][ty + 16 * a];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int a = 0; a < 4; ++a) gW[q][a] = fmaf(dz[q], ai[a], gW[q][a]);
    }
    if (tid < H) {
        float g = 0.0f;
        for (int s = 0; s < TS; ++s) g += Dout[s][tid];
        gb[tid] += g;
    }
    if (!below) return;
    // dA_in[s][i] = sum_j W[j][i] dZ[s][j];  Din[s][i] = silu'(z_in) * dA_in   (s = ty + 16 a, i = tx + 16 q)
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.0f;
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
        float dz[4], wj[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) dz[a] = Dout[ty + 16 * a][j];
#pragma unroll
        for (int q = 0; q < 4; ++q) wj[q] = W[j][tx + 16 * q];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] = fmaf(wj[q], dz[a], acc[a][q]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) Din[ty + 16 * a][tx + 16 * q] *= acc[a][q];
}

__global__ void __launch_bounds__(256, 1) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ feat,
                                                     const float* __restrict__ target, long long n,
                                                     float* __restrict__ grad, double* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    for (int k = tid; k < H * H; k += blockDim.x) {
        S.W1[k / H][k % H] = bf16r(P[OW1 + k]);
        S.W2[k / H][k % H] = bf16r(P[OW2 + k]);
    }
    for (int k = tid; k < H; k += blockDim.x) {
        S.W0[k][0] = bf16r(P[OW0 + 2 * k]);
        S.W0[k][1] = bf16r(P[OW0 + 2 * k + 1]);
        S.b0[k] = P[OB0 + k];
        S.b1[k] = P[OB1 + k];
        S.b2[k] = P[OB2 + k];
        S.W3[k] = bf16r(P[OW3 + k]);
        S.gW0[k][0] = S.gW0[k][1] = 0.0f;
        S.gb0[k] = S.gb1[k] = S.gb2[k] = S.gW3[k] = 0.0f;
    }
    if (tid == 0) {
        S.b3 = P[OB3];
        S.gb3 = 0.0f;
        S.loss = 0.0;
    }
    float gW1[4][4], gW2[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int a = 0; a < 4; ++a) gW1[q][a] = gW2[q][a] = 0.0f;
    __syncthreads();
    const long long ntiles = (n + TS - 1) / TS;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long s0 = tile * TS;
        if (tid < TS) {
            const long long i = s0 + tid;
            const bool ok = i < n;
            S.x[tid][0] = ok ? feat[2 * i] : 0.0f;
            S.x[tid][1] = ok ? feat[2 * i + 1] : 0.0f;
            S.dy[tid] = ok ? target[i] : 0.0f;  // target, replaced by dL/dy below
        }
        __syncthreads();
        // layer 0 (2 -> 64)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = ty + 16 * a, j = tx + 16 * q;
                const float z = fmaf(S.W0[j][0], S.x[s][0], fmaf(S.W0[j][1], S.x[s][1], S.b0[j]));
                silu_train(z, S.A1[s][j], S.D1[s][j]);
            }
        __syncthreads();
        dense_fwd(S.W1, S.b1, S.A1, S.A2, S.D2, ty, tx);
        __syncthreads();
        dense_fwd(S.W2, S.b2, S.A2, S.A3, S.D3, ty, tx);
        __syncthreads();
        // layer 3 (64 -> 1): four threads per sample; loss sum (y - t)^2
        {
            const int s = tid >> 2, part = tid & 3;
            float y = 0.0f;
            for (int j = part * 16; j < part * 16 + 16; ++j) y = fmaf(S.W3[j], S.A3[s][j], y);
            y += __shfl_xor_sync(0xffffffffu, y, 1);
            y += __shfl_xor_sync(0xffffffffu, y, 2);
            __syncwarp();
            if (part == 0) {
                y += S.b3;
                const bool ok = s0 + s < n;
                const float e = ok ? y - S.dy[s] : 0.0f;
                S.y[s] = y;
                S.dy[s] = 2.0f * e;
                atomicAdd(&S.loss, (double)e * (double)e);
            }
        }
        __syncthreads();
        // layer 3 backward: gW3, gb3, dz3 = W3 dy silu'(z3)
        if (tid < H) {
            float g = 0.0f;
            for (int s = 0; s < TS; ++s) g = fmaf(S.dy[s], S.A3[s][tid], g);
            S.gW3[tid] += g;
        }
        if (tid == 0) {
            float g = 0.0f;
            for (int s = 0; s < TS; ++s) g += S.dy[s];
            S.gb3 += g;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = ty + 16 * a, j = tx + 16 * q;
                S.D3[s][j] *= S.W3[j] * S.dy[s];
            }
        __syncthreads();
        dense_bwd(S.W2, S.D3, S.A2, S.D2, gW2, S.gb2, ty, tx, tid, true);
        __syncthreads();
        dense_bwd(S.W1, S.D2, S.A1, S.D1, gW1, S.gb1, ty, tx, tid, true);
        __syncthreads();
        // layer 0 backward
        if (tid < H) {
            float g0 = 0.0f, g1 = 0.0f, gb = 0.0f;
            for (int s = 0; s < TS; ++s) {
                const float dz = S.D1[s][tid];
                g0 = fmaf(dz, S.x[s][0], g0);
                g1 = fmaf(dz, S.x[s][1], g1);
                gb += dz;
            }
            S.gW0[tid][0] += g0;
            S.gW0[tid][1] += g1;
            S.gb0[tid] += gb;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int j = tx + 16 * q, i = ty + 16 * a;
            atomicAdd(&grad[OW1 + j * H + i], gW1[q][a]);
            atomicAdd(&grad[OW2 + j * H + i], gW2[q][a]);
        }
    for (int k = tid; k < H; k += blockDim.x) {
        atomicAdd(&grad[OW0 + 2 * k], S.gW0[k][0]);
        atomicAdd(&grad[OW0 + 2 * k + 1], S.gW0[k][1]);
        atomicAdd(&grad[OB0 + k], S.gb0[k]);
        atomicAdd(&grad[OB1 + k], S.gb1[k]);
        atomicAdd(&grad[OB2 + k], S.gb2[k]);
        atomicAdd(&grad[OW3 + k], S.gW3[k]);
    }
    if (tid == 0) {
        atomicAdd(&grad[OB3], S.gb3);
        atomicAdd(loss, S.loss);
    }
}

__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float scale, float bc1,
                           float bc2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= NP) return;
    const float gk = g[k] * scale;
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk * bc1) / (sqrtf(vk * bc2) + eps);
}

// --------------------------------------------------------------- inference
// one warp per 16-sample tile (sfp_mlp.cuh), strided over the grid.  (Two
// tiles per warp share the B-fragment reads but need ~120 registers; the
// lower occupancy made them slower on this latency-bound kernel.)
__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ P, const double* __restrict__ lc,
                                                   const double* __restrict__ u, double* __restrict__ out,
                                                   long long n) {
    __shared__ __align__(16) sfp_mlp::Smem S;
    sfp_mlp::stage(S, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = wid * 16; base < n; base += nw * 16) {
        float x0[2], x1[2], y[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const long long i = base + g + 8 * h;
            x0[h] = i < n ? sfp_mlp::feat_chi(lc[i]) : 0.0f;
            x1[h] = i < n ? sfp_mlp::feat_u(u[i]) : 0.0f;
        }
        sfp_mlp::tile16(S, x0, x1, y);
        if (t == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long i = base + g + 8 * h;
                if (i < n) out[i] = sfp_mlp::delta_of(y[h]);
            }
        }
    }
}

}  // namespace

extern "C" {

int sfp_od_inverse_cdf(const sfp_od_table* table, const double* log_chi, const double* u, double* delta, int64_t N,
                       void* stream) {
    if (!table || (N > 0 && (!log_chi || !u || !delta))) return sfp_set_error(SFP_EINVAL, "sfp_od_inverse_cdf: NULL argument");
    if (N <= 0) return SFP_OK;
    const long long grid = (N + 255) / 256 < (long long)sm_count_here() * 16 ? (N + 255) / 256 : sm_count_here() * 16;
    k_od_inverse_cdf<<<(unsigned)grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*table, log_chi, u, delta, N);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

int sfp_mlp_make_samples(const sfp_od_table* table, uint64_t seed, uint32_t chunk, double log_chi_lo,
                         double log_chi_hi, int64_t N, float* features, float* targets, void* stream) {
    if (!table || (N > 0 && (!features || !targets)))
        return sfp_set_error(SFP_EINVAL, "sfp_mlp_make_samples: NULL argument");
    if (!(log_chi_lo < log_chi_hi)) return sfp_set_error(SFP_EINVAL, "sfp_mlp_make_samples: empty log10 chi range");
    if (N <= 0) return SFP_OK;
    const long long grid = (N + 255) / 256 < (long long)sm_count_here() * 16 ? (N + 255) / 256 : sm_count_here() * 16;
    k_mlp_samples<<<(unsigned)grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*table, seed, chunk, log_chi_lo,
                                                                                      log_chi_hi, N, features, targets);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

int sfp_mlp_grad(const float* params, const float* features, const float* targets, int64_t N, float* grad,
                 double* loss, void* stream) {
    if (!params || !grad || !loss || (N > 0 && (!features || !targets)))
        return sfp_set_error(SFP_EINVAL, "sfp_mlp_grad: NULL argument");
    if (N <= 0) return SFP_OK;
    static bool attr_set = false;
    const int smem = (int)sizeof(TrainSmem);
    if (!attr_set) {
        MLP_CUDA(cudaFuncSetAttribute((const void*)k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_set = true;
    }
    const long long tiles = (N + TS - 1) / TS;
    const int grid = (int)(tiles < sm_count_here() ? tiles : sm_count_here());
    k_mlp_grad<<<grid, 256, smem, reinterpret_cast<cudaStream_t>(stream)>>>(params, features, targets, N, grad, loss);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

int sfp_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t step, float lr, float beta1,
                 float beta2, float eps, float grad_scale, void* stream) {
    if (!params || !grad || !m || !v) return sfp_set_error(SFP_EINVAL, "sfp_mlp_adam: NULL argument");
    if (step < 1) return sfp_set_error(SFP_EINVAL, "sfp_mlp_adam: step counts from 1");
    const float bc1 = (float)(1.0 / (1.0 - pow((double)beta1, (double)step)));
    const float bc2 = (float)(1.0 / (1.0 - pow((double)beta2, (double)step)));
    k_mlp_adam<<<(NP + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(params, grad, m, v, lr, beta1,
                                                                                      beta2, eps, grad_scale, bc1, bc2);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

int sfp_mlp_infer(const float* params, const double* log_chi, const double* u, double* delta, int64_t N,
                  void* stream) {
    if (!params || (N > 0 && (!log_chi || !u || !delta))) return sfp_set_error(SFP_EINVAL, "sfp_mlp_infer: NULL argument");
    if (N <= 0) return SFP_OK;
    const long long warps = (N + 15) / 16;
    long long grid = (warps + 3) / 4;
    const long long cap = (long long)sm_count_here() * 16;
    if (grid > cap) grid = cap;
    k_mlp_infer<<<(unsigned)grid, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(params, log_chi, u, delta, N);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

}  // extern "C"
