// sfp_mlp.cuh -- inference of the learned photon-energy sampler, shared by
// libsfp.so (batched kernel, sfp_mlp.cu) and the NVRTC step modules
// (in-step sampling).
//
// Network: features (log10 chi / 3, logit(u) / 8) -> 64 -> 64 -> 64 -> 1,
// SiLU on the hidden layers; output y, delta = 10^(3 (y - 1)) clamped to
// [1e-6, 1].  Parameters, 8577 float32:
//   W0[64][2] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[64] b3
// (row j of W = the weights of output unit j).
//
// A warp evaluates 16 or 32 samples at a time.  The two 64x64 layers run on the
// tensor cores (mma.sync m16n8k16, BF16 in, FP32 accumulate), and the
// accumulators of one layer become the A fragments of the next in
// registers.  Thread (g, t) = (lane / 4, lane % 4) holds rows g and g + 8,
// and columns 2t, 2t + 1 of every 8-column tile.
#pragma once

#ifndef SFP_DEVICE_INLINE
#define SFP_DEVICE_INLINE __device__ __forceinline__
#endif

namespace sfp_mlp {

constexpr int H = 64;
constexpr int OW0 = 0, OB0 = OW0 + 2 * H, OW1 = OB0 + H, OB1 = OW1 + H * H, OW2 = OB1 + H, OB2 = OW2 + H * H,
              OW3 = OB2 + H, OB3 = OW3 + H, NP = OB3 + 1;
constexpr int WLD = H + 8;  // padded BF16 row stride: conflict-free B-fragment loads

// weights as the tensor cores read them (BF16 bits), the rest in float32
struct Smem {
    unsigned short W1[H][WLD], W2[H][WLD];
    float W0[H][2], b0[H], b1[H], b2[H], W3[H];
    float b3;
};

// float32 -> BF16 bits, round to nearest, ties to even (finite inputs)
SFP_DEVICE_INLINE unsigned f2bf(float f) {
    const unsigned u = __float_as_uint(f);
    return (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
}
SFP_DEVICE_INLINE float bf2f(unsigned h) { return __uint_as_float(h << 16); }
SFP_DEVICE_INLINE float bf16r(float f) { return bf2f(f2bf(f)); }
// two floats -> packed BF16 pair (lo in the low half), round to nearest even
SFP_DEVICE_INLINE unsigned pack(float lo, float hi) {
    unsigned d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// all threads of the block; a __syncthreads must follow
SFP_DEVICE_INLINE void stage(Smem& S, const float* __restrict__ P) {
    for (int k = threadIdx.x; k < H * H; k += blockDim.x) {
        S.W1[k / H][k % H] = (unsigned short)f2bf(P[OW1 + k]);
        S.W2[k / H][k % H] = (unsigned short)f2bf(P[OW2 + k]);
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        S.W0[k][0] = bf16r(P[OW0 + 2 * k]);
        S.W0[k][1] = bf16r(P[OW0 + 2 * k + 1]);
        S.b0[k] = P[OB0 + k];
        S.b1[k] = P[OB1 + k];
        S.b2[k] = P[OB2 + k];
        S.W3[k] = bf16r(P[OW3 + k]);
    }
    if (threadIdx.x == 0) S.b3 = P[OB3];
}

SFP_DEVICE_INLINE float feat_chi(double log_chi) { return (float)(log_chi / 3.0); }
// logit(u) / 8 in float32: u is kept inside [2^-53, 1 - 2^-53] so that the
// logit stays finite, and 1 - u is formed in float64 first so that the tail
// (u near 1) keeps its relative precision
SFP_DEVICE_INLINE float feat_u(double u) {
    u = fmin(fmax(u, 0x1p-53), 1.0 - 0x1p-53);
    return (logf((float)u) - logf((float)(1.0 - u))) * 0.125f;
}
// delta = 10^(3 (y - 1)) in float32, clamped to [1e-6, 1]
SFP_DEVICE_INLINE double delta_of(float y) {
    const float d = exp2f((y - 1.0f) * (3.0f * 3.32192809488736234787f));  // 3 log2(10)
    return d < 1e-6f ? 1e-6 : (d > 1.0f ? 1.0 : (double)d);
}

// SiLU through one hardware tanh: z sigma(z) = z (1 + tanh(z / 2)) / 2
SFP_DEVICE_INLINE float silu_fast(float z) {
    float th;
    asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(0.5f * z));
    return 0.5f * z * (1.0f + th);
}

SFP_DEVICE_INLINE void mma(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C[m][nt] = A[m] x W^T for one 64 -> 64 layer, MT row tiles of 16 (each
// A[m]: four k16 fragments); every B fragment read serves all MT tiles
template <int MT>
SFP_DEVICE_INLINE void layer(const unsigned short (*W)[WLD], const unsigned (&A)[MT][4][4], float (&C)[MT][8][4],
                             int g, int t) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
        for (int m = 0; m < MT; ++m) C[m][nt][0] = C[m][nt][1] = C[m][nt][2] = C[m][nt][3] = 0.0f;
        const unsigned short* row = W[8 * nt + g];
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            const unsigned b0 = *reinterpret_cast<const unsigned*>(row + 16 * kc + 2 * t);
            const unsigned b1 = *reinterpret_cast<const unsigned*>(row + 16 * kc + 8 + 2 * t);
#pragma unroll
            for (int m = 0; m < MT; ++m) mma(C[m][nt], A[m][kc], b0, b1);
        }
    }
}

// bias + SiLU on the accumulators, packed as the next layer's A fragments
SFP_DEVICE_INLINE void to_fragments(const float (&C)[8][4], const float* b, unsigned (&A)[4][4], int t) {
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
        const int c0 = 16 * kc + 2 * t, c1 = c0 + 8;
        A[kc][0] = pack(silu_fast(C[2 * kc][0] + b[c0]), silu_fast(C[2 * kc][1] + b[c0 + 1]));
        A[kc][1] = pack(silu_fast(C[2 * kc][2] + b[c0]), silu_fast(C[2 * kc][3] + b[c0 + 1]));
        A[kc][2] = pack(silu_fast(C[2 * kc + 1][0] + b[c1]), silu_fast(C[2 * kc + 1][1] + b[c1 + 1]));
        A[kc][3] = pack(silu_fast(C[2 * kc + 1][2] + b[c1]), silu_fast(C[2 * kc + 1][3] + b[c1 + 1]));
    }
}

// MT tiles of 16 rows, called by all 32 lanes: x0[m][h], x1[m][h] are the
// features of row g + 8 h of tile m; returns the outputs y[m][h] of those
// rows (in every lane of the group of four).
template <int MT>
SFP_DEVICE_INLINE void tiles(const Smem& S, const float (&x0)[MT][2], const float (&x1)[MT][2], float (&y)[MT][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    unsigned A[MT][4][4];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int h = r & 1, c = 16 * kc + 2 * t + ((r >> 1) ? 8 : 0);
                const float z0 = fmaf(S.W0[c][0], x0[m][h], fmaf(S.W0[c][1], x1[m][h], S.b0[c]));
                const float z1 = fmaf(S.W0[c + 1][0], x0[m][h], fmaf(S.W0[c + 1][1], x1[m][h], S.b0[c + 1]));
                A[m][kc][r] = pack(silu_fast(z0), silu_fast(z1));
            }
        }
    float C[MT][8][4];
    layer<MT>(S.W1, A, C, g, t);
#pragma unroll
    for (int m = 0; m < MT; ++m) to_fragments(C[m], S.b1, A[m], t);
    layer<MT>(S.W2, A, C, g, t);
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        y[m][0] = y[m][1] = 0.0f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int c = 8 * nt + 2 * t;
            y[m][0] = fmaf(S.W3[c], silu_fast(C[m][nt][0] + S.b2[c]), y[m][0]);
            y[m][0] = fmaf(S.W3[c + 1], silu_fast(C[m][nt][1] + S.b2[c + 1]), y[m][0]);
            y[m][1] = fmaf(S.W3[c], silu_fast(C[m][nt][2] + S.b2[c]), y[m][1]);
            y[m][1] = fmaf(S.W3[c + 1], silu_fast(C[m][nt][3] + S.b2[c + 1]), y[m][1]);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            y[m][h] += __shfl_xor_sync(0xffffffffu, y[m][h], 1);
            y[m][h] += __shfl_xor_sync(0xffffffffu, y[m][h], 2);
            y[m][h] += S.b3;
        }
    }
}

// one 16-row tile (the in-step sampler: a warp's few events)
SFP_DEVICE_INLINE void tile16(const Smem& S, const float (&x0)[2], const float (&x1)[2], float (&y)[2]) {
    const float a0[1][2] = {{x0[0], x0[1]}}, a1[1][2] = {{x1[0], x1[1]}};
    float r[1][2];
    tiles<1>(S, a0, a1, r);
    y[0] = r[0][0];
    y[1] = r[0][1];
}

}  // namespace sfp_mlp
