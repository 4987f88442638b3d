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
// Inference: weights in BF16, FP32 accumulation.  The batched sampler
// (sfp_mlp_infer) runs every layer but the output dot product as tcgen05.mma
// chains with the accumulators in tensor memory (k_mlp_infer_tc below); the
// in-step sampler, a warp's few events at a time, uses warp-level mma.sync
// tiles (sfp_mlp.cuh), also reachable batched as sfp_mlp_infer_warp.
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

// ------------------------------------------------ inference on tcgen05 / TMEM
// One CTA of 128 threads takes tiles of 128 queries, one query per thread
// (row = thread).  Each layer is one tcgen05.mma chain issued by thread 0:
// A (the tile's inputs or activations, BF16) and B (the layer's weights,
// BF16) in shared memory, D (128 x 64 FP32) in tensor memory.  The input
// layer and the biases are folded into the MMAs:
//   layer 0: A = [x0_hi, x0_lo, x1_hi, x1_lo, 1, 1, 0 ...] (K = 16),
//            B row n = [W0[n][0], W0[n][0], W0[n][1], W0[n][1], b0_hi, b0_lo, 0 ...];
//   layers 1, 2: A = [h (64), 1, 1, 0 ...] (K = 80), B row n = [W[n][:], b_hi, b_lo, 0 ...];
// with v_hi = bf16(v), v_lo = bf16(v - v_hi), so features and biases keep
// ~16 bits where one BF16 would keep 8.  Each thread reads its row of D with
// tcgen05.ld (the warp's 32-lane quarter of tensor memory), applies SiLU
// (one packed half-precision tanh per two activations) and writes the next
// layer's A row; the output layer is an FP32 dot product on the CUDA cores.
// Shared-memory operands use the K-major layout without swizzle: 8 x 8 BF16
// core matrices of 128 B, element (r, k) at (r/8) (K/8) 128 + (k/8) 128 +
// (r%8) 16 + (k%8) 2 (leading-dimension byte offset 128, stride-dimension
// byte offset (K/8) 128).  Every wait on the MMA barrier is bounded (one
// second); on timeout the block sets g_mlp_tc_error, stops, and still frees
// its tensor memory.  `withhold` (a test of that path) issues no MMA and no
// commit, so the first wait runs out.
namespace tc {

constexpr int TM = 128;  // queries per tile (the MMA's M)
constexpr int K0 = 16;   // input layer K
constexpr int KH = 80;   // hidden layers K
constexpr int CM = 128;  // bytes of one core matrix
constexpr unsigned TMEM_COLS = 64;
// kind::f16 instruction descriptor: FP32 accumulator (bits 4-5 = 1), BF16 A
// (bits 7-9 = 1) and B (bits 10-12 = 1), both K-major, N = 64 (bits 17-22 =
// N/8), M = 128 (bits 24-28 = M/16)
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
// bound of every wait on the MMA barrier: one second, far above the
// microseconds an MMA group takes
constexpr unsigned long long WAIT_NS = 1000000000ull;
constexpr long long WAIT_TRIES = 1ll << 30;

struct Smem {
    alignas(128) unsigned char B0[64 * K0 * 2];
    alignas(128) unsigned char B1[64 * KH * 2];
    alignas(128) unsigned char B2[64 * KH * 2];
    alignas(128) unsigned char A0[TM * K0 * 2];
    alignas(128) unsigned char A1[TM * KH * 2];
    float W3[64];
    float b3;
    unsigned tmem;
    alignas(8) unsigned long long mbar;
};

__device__ __forceinline__ unsigned cm_off(int r, int k, int K) {
    return (unsigned)((r >> 3) * (K / 8) * CM + (k >> 3) * CM + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (K-major, no swizzle) of a K-column operand
__device__ __forceinline__ unsigned long long desc(const void* base, int K) {
    const unsigned long long lbo = CM >> 4, sbo = (unsigned long long)((K / 8) * CM) >> 4;
    return (unsigned long long)((smem_u32(base) >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(unsigned d_tmem, unsigned long long a, unsigned long long b, unsigned acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc), "r"(0u));
}
__device__ __forceinline__ void commit(unsigned mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// true once the barrier has completed the given phase; false after WAIT_NS
// nanoseconds (or WAIT_TRIES polls, whichever comes first)
__device__ __forceinline__ bool wait_phase(unsigned mbar, unsigned phase) {
    const unsigned long long t0 = now_ns();
    for (long long i = 0; i < WAIT_TRIES; ++i) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (ok) return true;
        if (now_ns() - t0 > WAIT_NS) return false;
    }
    return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes of shared memory become visible to the tensor cores
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's row of D
__device__ __forceinline__ void ld16(unsigned taddr, float (&v)[16]) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// SiLU of two pre-activations through one packed half-precision tanh:
// z sigma(z) = h (1 + tanh h), h = z / 2
__device__ __forceinline__ void silu2(float za, float zb, float& a, float& b) {
    const float ha = 0.5f * za, hb = 0.5f * zb;
    unsigned hh, th;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(hh) : "f"(hb), "f"(ha));
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(th) : "r"(hh));
    float ta, tb;
    asm("{\n\t.reg .f16 l, h;\n\tmov.b32 {l, h}, %2;\n\tcvt.f32.f16 %0, l;\n\tcvt.f32.f16 %1, h;\n\t}"
        : "=f"(ta), "=f"(tb)
        : "r"(th));
    a = fmaf(ha, ta, ha);
    b = fmaf(hb, tb, hb);
}

__device__ __forceinline__ unsigned short bf(float f) { return (unsigned short)sfp_mlp::f2bf(f); }
__device__ __forceinline__ void hi_lo(float v, unsigned short& h, unsigned short& l) {
    h = bf(v);
    l = bf(v - sfp_mlp::bf2f(h));
}

}  // namespace tc

__device__ int g_mlp_tc_error;

__global__ void __launch_bounds__(128, 4) k_mlp_infer_tc(const float* __restrict__ P, const double* __restrict__ lc,
                                                         const double* __restrict__ u, double* __restrict__ out,
                                                         long long n, int withhold) {
    using namespace tc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights as B operands (BF16, core-matrix layout), the output layer in FP32
    for (int k = tid; k < 64 * K0; k += blockDim.x) {
        const int r = k / K0, c = k % K0;
        float w = 0.0f;
        unsigned short h, l;
        if (c < 4) w = sfp_mlp::bf16r(P[OW0 + 2 * r + (c >> 1)]);
        *reinterpret_cast<unsigned short*>(S.B0 + cm_off(r, c, K0)) = bf(w);
        if (c == 4 || c == 5) {
            hi_lo(P[OB0 + r], h, l);
            *reinterpret_cast<unsigned short*>(S.B0 + cm_off(r, c, K0)) = c == 4 ? h : l;
        }
    }
    for (int k = tid; k < 64 * KH; k += blockDim.x) {
        const int r = k / KH, c = k % KH;
        unsigned short v1 = 0, v2 = 0, h, l;
        if (c < 64) {
            v1 = bf(P[OW1 + r * 64 + c]);
            v2 = bf(P[OW2 + r * 64 + c]);
        } else if (c < 66) {
            hi_lo(P[OB1 + r], h, l);
            v1 = c == 64 ? h : l;
            hi_lo(P[OB2 + r], h, l);
            v2 = c == 64 ? h : l;
        }
        *reinterpret_cast<unsigned short*>(S.B1 + cm_off(r, c, KH)) = v1;
        *reinterpret_cast<unsigned short*>(S.B2 + cm_off(r, c, KH)) = v2;
    }
    for (int k = tid; k < 64; k += blockDim.x) S.W3[k] = sfp_mlp::bf16r(P[OW3 + k]);
    if (tid == 0) S.b3 = P[OB3];
    // the constant columns of this thread's A rows: A0 chunk 1 (zeros), A1
    // chunk 8 (the two bias ones) and chunk 9 (zeros)
    {
        const uint4 z{0u, 0u, 0u, 0u};
        const unsigned one2 = 0x3F803F80u;  // two BF16 ones
        *reinterpret_cast<uint4*>(S.A0 + cm_off(tid, 8, K0)) = z;
        *reinterpret_cast<uint4*>(S.A1 + cm_off(tid, 64, KH)) = uint4{one2, 0u, 0u, 0u};
        *reinterpret_cast<uint4*>(S.A1 + cm_off(tid, 72, KH)) = z;
    }
    const unsigned mbar = smem_u32(&S.mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // 64 columns of tensor memory: the 128 x 64 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const unsigned tmem = S.tmem;
    const unsigned trow = tmem + ((unsigned)(32 * warp) << 16);  // this warp's lane quarter
    const unsigned long long dA0 = desc(S.A0, K0), dA1 = desc(S.A1, KH);
    const unsigned long long dB0 = desc(S.B0, K0), dB1 = desc(S.B1, KH), dB2 = desc(S.B2, KH);
    unsigned phase = 0;
    bool ok = true;
    const long long n_tiles = (n + TM - 1) / TM;
    // this thread's inputs of the next tile are loaded while the current one
    // runs its layers, so their latency is hidden behind the MMAs and SiLU
    double lc_next = 0.0, u_next = 0.0;
    {
        const long long q0 = (long long)blockIdx.x * TM + tid;
        if (blockIdx.x < n_tiles && q0 < n) {
            lc_next = lc[q0];
            u_next = u[q0];
        }
    }
    for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const long long q = tile * TM + tid;
        const double lc_q = lc_next, u_q = u_next;
        {
            const long long qn = q + (long long)gridDim.x * TM;
            lc_next = 0.0;
            u_next = 0.0;
            if (qn < n) {
                lc_next = lc[qn];
                u_next = u[qn];
            }
        }
        // layer 0 inputs: the features split into BF16 hi / lo parts
        {
            float x0 = 0.0f, x1 = 0.0f;
            if (q < n) {
                x0 = sfp_mlp::feat_chi(lc_q);
                x1 = sfp_mlp::feat_u(u_q);
            }
            unsigned short a, b, c, d;
            hi_lo(x0, a, b);
            hi_lo(x1, c, d);
            *reinterpret_cast<uint4*>(S.A0 + cm_off(tid, 0, K0)) =
                uint4{(unsigned)a | ((unsigned)b << 16), (unsigned)c | ((unsigned)d << 16), 0x3F803F80u, 0u};
        }
        float y = 0.0f;
        for (int layer = 0; layer < 3 && ok; ++layer) {
            fence_smem_async();
            fence_before();
            __syncthreads();  // A written, D of the previous layer read
            if (tid == 0 && !withhold) {
                fence_after();
                if (layer == 0) {
                    mma(tmem, dA0, dB0, 0u);
                } else {
                    const unsigned long long dB = layer == 1 ? dB1 : dB2;
#pragma unroll
                    for (int kk = 0; kk < KH / 16; ++kk)  // K-steps of 16: start address + 256 B
                        mma(tmem, dA1 + (unsigned long long)(16 * kk), dB + (unsigned long long)(16 * kk),
                            kk ? 1u : 0u);
                }
                commit(mbar);
            }
            ok = __syncthreads_and(wait_phase(mbar, phase)) != 0;
            if (!ok) break;  // phase stays the one of the commit still outstanding
            phase ^= 1u;
            fence_after();
            float v[64];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float w[16];
                ld16(trow + 16u * c, w);
#pragma unroll
                for (int i = 0; i < 16; ++i) v[16 * c + i] = w[i];
            }
            ld_wait();
            if (layer < 2) {  // next layer's A row, 8 columns (one core-matrix row) per store
#pragma unroll
                for (int ch = 0; ch < 8; ++ch) {
                    unsigned p[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        float a, b;
                        silu2(v[8 * ch + 2 * j], v[8 * ch + 2 * j + 1], a, b);
                        p[j] = sfp_mlp::pack(a, b);
                    }
                    *reinterpret_cast<uint4*>(S.A1 + cm_off(tid, 8 * ch, KH)) = uint4{p[0], p[1], p[2], p[3]};
                }
            } else {  // output layer on the CUDA cores, FP32
                y = S.b3;
#pragma unroll
                for (int k = 0; k < 64; k += 2) {
                    float a, b;
                    silu2(v[k], v[k + 1], a, b);
                    y = fmaf(S.W3[k], a, y);
                    y = fmaf(S.W3[k + 1], b, y);
                }
            }
        }
        if (!ok) break;
        if (q < n) out[q] = sfp_mlp::delta_of(y);
    }
    if (!ok && tid == 0) {
        atomicExch(&g_mlp_tc_error, 1);
        tc::wait_phase(mbar, phase);  // the MMAs in flight, again bounded
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
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

}  // extern "C"

namespace {

int mlp_infer_tc(const char* name, const float* params, const double* log_chi, const double* u, double* delta,
                 int64_t N, void* stream, int withhold) {
    if (!params || (N > 0 && (!log_chi || !u || !delta)))
        return sfp_set_error(SFP_EINVAL, std::string(name) + ": NULL argument");
    if (N <= 0) return SFP_OK;
    static int attr_dev = -1;
    int dev = 0;
    MLP_CUDA(cudaGetDevice(&dev));
    const int smem = (int)sizeof(tc::Smem);
    if (attr_dev != dev) {
        MLP_CUDA(cudaFuncSetAttribute((const void*)k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_dev = dev;
    }
    const long long tiles = (N + tc::TM - 1) / tc::TM;
    const long long cap = (long long)sm_count_here() * 4;  // four CTAs (4 x 64 tensor-memory columns) per SM
    const long long grid = tiles < cap ? tiles : cap;
    k_mlp_infer_tc<<<(unsigned)grid, 128, smem, reinterpret_cast<cudaStream_t>(stream)>>>(params, log_chi, u, delta,
                                                                                        N, withhold);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

}  // namespace

extern "C" {

int sfp_mlp_infer(const float* params, const double* log_chi, const double* u, double* delta, int64_t N,
                  void* stream) {
    return mlp_infer_tc("sfp_mlp_infer", params, log_chi, u, delta, N, stream, 0);
}

int sfp_mlp_infer_withheld(const float* params, const double* log_chi, const double* u, double* delta, int64_t N,
                           void* stream) {
    return mlp_infer_tc("sfp_mlp_infer_withheld", params, log_chi, u, delta, N, stream, 1);
}

int sfp_mlp_infer_warp(const float* params, const double* log_chi, const double* u, double* delta, int64_t N,
                       void* stream) {
    if (!params || (N > 0 && (!log_chi || !u || !delta)))
        return sfp_set_error(SFP_EINVAL, "sfp_mlp_infer_warp: NULL argument");
    if (N <= 0) return SFP_OK;
    const long long warps = (N + 15) / 16;
    long long grid = (warps + 3) / 4;
    const long long cap = (long long)sm_count_here() * 16;
    if (grid > cap) grid = cap;
    k_mlp_infer<<<(unsigned)grid, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(params, log_chi, u, delta, N);
    MLP_CUDA(cudaGetLastError());
    return SFP_OK;
}

int sfp_mlp_device_error(int* code) {
    if (!code) return sfp_set_error(SFP_EINVAL, "sfp_mlp_device_error: NULL argument");
    int v = 0;
    MLP_CUDA(cudaDeviceSynchronize());
    MLP_CUDA(cudaMemcpyFromSymbol(&v, g_mlp_tc_error, sizeof(int)));
    if (v) {
        const int zero = 0;
        MLP_CUDA(cudaMemcpyToSymbol(g_mlp_tc_error, &zero, sizeof(int)));
    }
    *code = v;
    return SFP_OK;
}

}  // extern "C"
