// sfp_step.cuh -- the fused particle step (one launch per kernel advances
// every species of every instance by one step) plus its bookkeeping kernel.
//
// Compiled by NVRTC together with a generated field program that defines
//     SFP_DEVICE_INLINE void sfp_field_program(double x, double y, double z,
//                                              double t, const double* P, double F[6]);
// so the field expression is inlined into the push.
//
// Semantics follow simulation.py:102-144 exactly:
//   1. fields at t for pushed species (particles.py:299-323),
//   2. chi + pair events for photon species (QED at t),
//   3. chi + photon events + hard-photon filter for e+- species,
//   4. photons appended (e- species first, in buffer order), recoil,
//   5. pairs appended, converted photons pruned,
//   6. every pushed particle -- children included -- pushed from t to t+dt:
//      half position, fields at t+dt/2, Boris / Boris-TBMT (+LL/CLL), half position.
// After the bookkeeping kernel a step is:
//   massive -- 3; a particle with an event is marked and left as it was at t
//              (its delta stored), every other one takes 6;
//   photon  -- 2; a converted photon is marked (its delta stored), every
//              other one takes 6;
//   scan    -- the children's slots: per-tile event counts scanned in the
//              reference's order;
//   appends -- 4 (child from the parent's state at t, then the parent's
//              recoil and 6) and 5 (children pushed, 6), at those slots.
// The massive and photon kernels touch disjoint memory: each writes only
// below the start-of-step counts of its own group's buffers.  Appends are
// ordered: a child gets the slot that the reference's find_event_index +
// create_* would give it, so Philox streams keyed by slot are reproducible.
// No kernel waits on another block.
#pragma once
#include "sfp_device.cuh"
#include "sfp_device32.cuh"
#include "sfp_mlp.cuh"
#include "sfp_run.cuh"

// threads per block of the group kernels (8 warps, each on its own tiles)
#ifndef SFP_TILE
#define SFP_TILE 256
#endif
// tiles per super-tile of the event scan
#define SFP_SUPER_TILE 64
// pruned-flag value of a particle whose event of this step awaits its children
#define SFP_MARK 2

namespace sfp {

SFP_DEVICE_INLINE unsigned int u4_get(const uint4& v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}
SFP_DEVICE_INLINE uint4 u4_one(int c, unsigned int n) {
    uint4 v{0u, 0u, 0u, 0u};
    if (c == 0) v.x = n;
    else if (c == 1) v.y = n;
    else if (c == 2) v.z = n;
    else v.w = n;
    return v;
}
SFP_DEVICE_INLINE uint4 u4_add(uint4 a, uint4 b) { return uint4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }

// Asynchronous 16-byte global -> shared copies (cp.async, one per thread,
// L2 only); `src_bytes` < 16 zero-fills the rest and reads only that many.
// Issue and commit carry no "memory" clobber, so values the compiler holds in
// registers survive them; the destination's earlier readers are ordered by
// the caller's __syncwarp() before the issue (volatile asm is not moved across
// it), and the data is read only after cp_async_wait, which is a clobber.
SFP_DEVICE_INLINE void cp_async16(void* smem_dst, const void* gsrc, unsigned int src_bytes) {
    const unsigned int d = (unsigned int)__cvta_generic_to_shared(smem_dst);
    const unsigned long long g = (unsigned long long)__cvta_generic_to_global(gsrc);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(g), "r"(src_bytes));
}
SFP_DEVICE_INLINE void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
SFP_DEVICE_INLINE void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// inclusive / exclusive warp sums
SFP_DEVICE_INLINE unsigned int warp_incl_scan(unsigned int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}
SFP_DEVICE_INLINE unsigned int warp_sum(unsigned int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// bit b set where byte b of the 16 bytes v equals SFP_MARK
SFP_DEVICE_INLINE unsigned int marks16(uint4 v) {
    const unsigned int k = SFP_MARK * 0x01010101u;
    const unsigned int w[4] = {__vcmpeq4(v.x, k), __vcmpeq4(v.y, k), __vcmpeq4(v.z, k), __vcmpeq4(v.w, k)};
    unsigned int m = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
        m |= (((w[q] >> 7) & 1u) | ((w[q] >> 14) & 2u) | ((w[q] >> 21) & 4u) | ((w[q] >> 28) & 8u)) << (4 * q);
    return m;
}

// Push of one massive particle from t to t+dt (simulation.py:128-137 with
// particles.py:244-296 / 575-604).  x, u (and s) in/out.
SFP_DEVICE_INLINE void push_massive(double& x, double& y, double& z, double& ux, double& uy, double& uz, double& sx,
                                    double& sy, double& sz, const sfp_segment& S, const double* __restrict__ P,
                                    double t, double dt) {
    double ig = inv_gamma_massive(ux, uy, uz);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
    double F[6];
    sfp_field_program(x, y, z, t + 0.5 * dt, P, F);
    if (S.spin)
        ig = boris_tbmt(ux, uy, uz, sx, sy, sz, F, S.q, S.ae, dt);
    else
        ig = boris(ux, uy, uz, F, S.q, dt);
    if (S.rr == SFP_RR_LL || (S.rr == SFP_RR_CLL && !S.spin)) {
        const double chi = chi_of(F, ux, uy, uz, ig);
        ig = ll_push(ux, uy, uz, ig, chi, dt, S.rr == SFP_RR_CLL);
    }
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
}

SFP_DEVICE_INLINE void push_photon(double& x, double& y, double& z, double ux, double uy, double uz, double dt) {
    const double ig = inv_gamma_photon(ux, uy, uz);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
}

// float32 form of push_massive: float32 increments, float64 accumulation.
// The float32 push's per-(segment, step) constants, formed once per tile
// rather than once per particle (the same expressions, so the same values)
struct sfp_pc32 {
    double th;  // t + dt/2, the time of the push's field
    float hc;   // c dt / 2
    float eps;  // q dt / (2 m c)
    float bq;   // q dt / (2 m)
    float ll;   // the LL / CLL prefactor
};

SFP_DEVICE_INLINE sfp_pc32 push_consts32(const sfp_segment& S, double t, double dt) {
    sfp_pc32 K;
    K.th = t + 0.5 * dt;
    K.hc = (float)(0.5 * kC * dt);
    K.eps = (float)((S.q * dt) / ((2.0 * kMe) * kC));
    K.bq = (float)((S.q * dt) / (2.0 * kMe));
    K.ll = (float)ll_factor(dt);
    return K;
}

SFP_DEVICE_INLINE void push_massive32(double& x, double& y, double& z, double& ux, double& uy, double& uz,
                                      double& sx, double& sy, double& sz, const sfp_segment& S,
                                      const double* __restrict__ P, const sfp_pc32& K) {
    const float hc = K.hc;
    float g = sfp32::gamma_of(ux, uy, uz, false);
    float fx = sfp32::d2f(ux), fy = sfp32::d2f(uy), fz = sfp32::d2f(uz);
    float a = __fdividef(hc, g);
    x += (double)(a * fx);
    y += (double)(a * fy);
    z += (double)(a * fz);
    float F[6];
    sfp_field_program32(x, y, z, K.th, P, F);
    const float eps = K.eps;
    const float bq = K.bq;
    const float ex = eps * F[0], ey = eps * F[1], ez = eps * F[2];
    const float umx = fx + ex, umy = fy + ey, umz = fz + ez;
    float gm;
    if (g < (float)sfp32::kGammaSplit) {
        gm = sqrtf(1.0f + umx * umx + umy * umy + umz * umz);
    } else {
        const double dx = ux + (double)ex, dy = uy + (double)ey, dz = uz + (double)ez;
        gm = sfp32::d2f(sqrt(((1.0 + dx * dx) + dy * dy) + dz * dz));
    }
    const float igm = __fdividef(1.0f, gm);
    if (S.spin) {  // inline.py:39-70: spin rotation with B_eff(u-), as an increment
        const float ae = sfp32::d2f(S.ae);
        const float uB = umx * F[3] + umy * F[4] + umz * F[5];
        const float a1 = ae + igm, a2 = __fdividef(ae * gm, gm + 1.0f), a3 = ae + __fdividef(1.0f, gm + 1.0f);
        const float bex = a1 * F[3] - a2 * uB * umx - a3 * (umy * F[2] - umz * F[1]);
        const float bey = a1 * F[4] - a2 * uB * umy - a3 * (umz * F[0] - umx * F[2]);
        const float bez = a1 * F[5] - a2 * uB * umz - a3 * (umx * F[1] - umy * F[0]);
        const float Tx = bq * bex, Ty = bq * bey, Tz = bq * bez;
        const float f2 = __fdividef(2.0f, 1.0f + Tx * Tx + Ty * Ty + Tz * Tz);
        const float s0x = sfp32::d2f(sx), s0y = sfp32::d2f(sy), s0z = sfp32::d2f(sz);
        const float spx = s0x + (s0y * Tz - s0z * Ty), spy = s0y + (s0z * Tx - s0x * Tz), spz = s0z + (s0x * Ty - s0y * Tx);
        sx += (double)(f2 * (spy * Tz - spz * Ty));
        sy += (double)(f2 * (spz * Tx - spx * Tz));
        sz += (double)(f2 * (spx * Ty - spy * Tx));
    }
    // Boris (inline.py:4-36) as u += 2 eps E + u' x S
    const float Tx = bq * F[3] * igm, Ty = bq * F[4] * igm, Tz = bq * F[5] * igm;
    const float upx = umx + (umy * Tz - umz * Ty), upy = umy + (umz * Tx - umx * Tz), upz = umz + (umx * Ty - umy * Tx);
    const float f2 = __fdividef(2.0f, 1.0f + Tx * Tx + Ty * Ty + Tz * Tz);
    ux += (double)(2.0f * ex + f2 * (upy * Tz - upz * Ty));
    uy += (double)(2.0f * ey + f2 * (upz * Tx - upx * Tz));
    uz += (double)(2.0f * ez + f2 * (upx * Ty - upy * Tx));
    g = sfp32::gamma_of(ux, uy, uz, false);
    if (S.rr == SFP_RR_LL || (S.rr == SFP_RR_CLL && !S.spin)) {  // inline.py:104-123
        fx = sfp32::d2f(ux); fy = sfp32::d2f(uy); fz = sfp32::d2f(uz);
        const float chi = sfp32::chi_of(F, fx, fy, fz, g);
        float factor = K.ll;
        if (S.rr == SFP_RR_CLL) {
            const float q = 1.0f + 4.8f * (1.0f + chi) * __logf(1.0f + 1.7f * chi) + 2.44f * chi * chi;
            factor *= exp2f(-0.66666667f * __log2f(q));
        }
        const float c = __fdividef(factor * chi * chi, g);
        ux += (double)(c * fx);
        uy += (double)(c * fy);
        uz += (double)(c * fz);
        g = sfp32::gamma_of(ux, uy, uz, false);
    }
    a = __fdividef(hc, g);
    x += (double)(a * sfp32::d2f(ux));
    y += (double)(a * sfp32::d2f(uy));
    z += (double)(a * sfp32::d2f(uz));
}

SFP_DEVICE_INLINE void push_photon32(double& x, double& y, double& z, double ux, double uy, double uz, double dt) {
    const float fx = sfp32::d2f(ux), fy = sfp32::d2f(uy), fz = sfp32::d2f(uz);
    const float a = sfp32::d2f(kC * dt) * rsqrtf(fx * fx + fy * fy + fz * fz);
    x += (double)(a * fx);
    y += (double)(a * fy);
    z += (double)(a * fz);
}

// n steps of the photon push at once (n may be negative): a photon's
// momentum does not change while it flies, so n pushes add n times the same
// displacement.  float64: each push adds ((c dt/2) / |u|) u twice (cpu.py:
// 5-19 with dt/2, push_photon); float32: (c dt / |u|) u as one float32
// increment (push_photon32).  Equal to n successive pushes up to the
// rounding of the float64 sum.
template <int FORM>
SFP_DEVICE_INLINE void photon_shift(double& x, double& y, double& z, double ux, double uy, double uz, double dt,
                                    double n) {
    if (FORM == SFP_FORM_FP64) {
        const double k = ((kC * (0.5 * dt)) * inv_gamma_photon(ux, uy, uz)) * (2.0 * n);
        x += k * ux;
        y += k * uy;
        z += k * uz;
    } else {
        const float fx = sfp32::d2f(ux), fy = sfp32::d2f(uy), fz = sfp32::d2f(uz);
        const float a = sfp32::d2f(kC * dt) * rsqrtf(fx * fx + fy * fy + fz * fz);
        x += n * (double)(a * fx);
        y += n * (double)(a * fy);
        z += n * (double)(a * fz);
    }
}

}  // namespace sfp

#if defined(SFP_WANT_STEP)

// ---------------------------------------------------------------------------
// Field parameters.  A module built for runs of one instance (a Simulation)
// defines SFP_CONST_FIELD_N, the length of its field's parameter block, and
// reads the block from this module's constant bank: the field program's
// reads are at compile-time offsets, so they become constant operands of
// the arithmetic instead of loads.  The host copies the run's block into
// sfp_cfield on the run's stream before each launch sequence (sfp_capi.cu,
// runs sharing a module are ordered).  Modules for several instances read
// each instance's block from global memory.
// ---------------------------------------------------------------------------
#if defined(SFP_CONST_FIELD_N)
// (a variable at global scope: its name is not mangled)
__constant__ __align__(16) double sfp_cfield[SFP_CONST_FIELD_N];
#endif

SFP_DEVICE_INLINE const double* sfp_field_params(const sfp_instance& I) {
#if defined(SFP_CONST_FIELD_N)
    (void)I;
    return sfp_cfield;
#else
    return I.field_params;
#endif
}

// The step's rejection-sampling draws: Philox-4x32-10 keyed by the instance
// seed (sfp::uniform2 / sfp32::uniform2f).  A one-instance module takes the
// ten rounds' keys (the seed's key schedule, k0 and k1 per round) from its
// constant bank, copied by the host with the field parameters, instead of
// forming them with two additions per round: the same numbers.
#if defined(SFP_CONST_FIELD_N)
__constant__ unsigned int sfp_ckeys[20];
#endif

SFP_DEVICE_INLINE sfp::U4 sfp_step_philox(sfp::U4 c, unsigned long long seed) {
#if defined(SFP_CONST_FIELD_N)
    (void)seed;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned int lo0 = 0xD2511F53u * c.x;
        const unsigned int hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned int lo1 = 0xCD9E8D57u * c.z;
        const unsigned int hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = sfp::U4{hi1 ^ c.y ^ sfp_ckeys[2 * r], lo1, hi0 ^ c.w ^ sfp_ckeys[2 * r + 1], lo0};
    }
    return c;
#else
    return sfp::philox4x32_10(c, (unsigned int)seed, (unsigned int)(seed >> 32));
#endif
}

SFP_DEVICE_INLINE void sfp_step_uniform2(unsigned long long seed, unsigned int stream, unsigned int step,
                                         unsigned int purpose, long long slot, double& r1, double& r2) {
    const sfp::U4 o = sfp_step_philox(sfp::philox_counter(stream, step, purpose, slot), seed);
    r1 = sfp::u01(o.x, o.y);
    r2 = sfp::u01(o.z, o.w);
}

SFP_DEVICE_INLINE void sfp_step_uniform2f(unsigned long long seed, unsigned int stream, unsigned int step,
                                          unsigned int purpose, long long slot, float& r1, float& r2) {
    sfp32::uniform2f_of(sfp_step_philox(sfp::philox_counter(stream, step, purpose, slot), seed), r1, r2);
}

// ---------------------------------------------------------------------------
// QED tables staged in shared memory (float64, or float32 copies for FP32)
// ---------------------------------------------------------------------------
struct sfp_qed_smem {
    const double* iAt;
    const double* dAt;
    const float* iAf;
    const float* dAf;
    const double* od_ph;
    const double* od_pa;
    int zN;
    double zmax;
    float inv_dzf;
    float base_maxf;
    double chi_pair_min;  // below: no pair event is possible (z_min > z_max)
    double od_chi_min_ph, od_chi_min_pa;  // optical depth: 10^log_chi_min of each table
    const float* od_phf;  // float32 form, optical depth: the total-rate tables as float32
    const float* od_paf;
};

template <int FORM, int QED>
__device__ __forceinline__ sfp_qed_smem sfp_stage_tables(const sfp_run_dev* __restrict__ R, double* s_tab) {
    sfp_qed_smem T;
    T.iAt = T.dAt = s_tab;
    T.iAf = T.dAf = reinterpret_cast<const float*>(s_tab);
    T.od_ph = T.od_pa = s_tab;
    T.od_phf = T.od_paf = reinterpret_cast<const float*>(s_tab);
    T.zN = 0;
    T.zmax = 0.0;
    if (QED == SFP_QED_REJECTION) {
        T.zN = R->rs.z_N;
        T.zmax = R->rs.z_max;
        if (FORM == SFP_FORM_FP64) {
            for (int i = threadIdx.x; i < T.zN; i += blockDim.x) {
                s_tab[i] = R->rs.int_Ai[i];
                s_tab[T.zN + i] = R->rs.Aip[i];
            }
            T.dAt = s_tab + T.zN;
        } else {
            float* f = reinterpret_cast<float*>(s_tab);
            for (int i = threadIdx.x; i < T.zN; i += blockDim.x) {
                f[i] = (float)R->rs.int_Ai[i];
                f[T.zN + i] = (float)R->rs.Aip[i];
            }
            T.dAf = f + T.zN;
        }
    } else {
        const int n1 = R->od_photon.chi_N, n2 = R->od_pair.chi_N;
        if (FORM == SFP_FORM_FP64) {
            for (int i = threadIdx.x; i < n1; i += blockDim.x) s_tab[i] = R->od_photon.rate_total[i];
            for (int i = threadIdx.x; i < n2; i += blockDim.x) s_tab[n1 + i] = R->od_pair.rate_total[i];
            T.od_pa = s_tab + n1;
        } else {
            float* f = reinterpret_cast<float*>(s_tab);
            for (int i = threadIdx.x; i < n1; i += blockDim.x) f[i] = (float)R->od_photon.rate_total[i];
            for (int i = threadIdx.x; i < n2; i += blockDim.x) f[n1 + i] = (float)R->od_pair.rate_total[i];
            T.od_paf = f + n1;
        }
    }
    T.inv_dzf = (float)((double)(T.zN - 1) / T.zmax);
    T.base_maxf = (float)(T.zmax * sqrt(T.zmax));
    // pair creation needs z_min = (4/chi)^(2/3) <= z_max: exact cut with margin
    T.chi_pair_min = QED == SFP_QED_REJECTION ? 4.0 / (T.zmax * sqrt(T.zmax)) * (1.0 - 1e-6) : 0.0;
    T.od_chi_min_ph = QED == SFP_QED_OPTICAL_DEPTH ? pow(10.0, R->od_photon.log_chi_min) : 0.0;
    T.od_chi_min_pa = QED == SFP_QED_OPTICAL_DEPTH ? pow(10.0, R->od_pair.log_chi_min) : 0.0;
    return T;
}

// photon emission by a massive particle at t (qed/rejection_sampling.py:73-89,
// optical_depth.py:15-62, hard-photon filter cpu.py:226-231).  With the
// learned sampler (optical depth, R->mlp_params) an event returns, instead of
// delta, the uniform u its energy is drawn from, with log10 chi and the
// hard-photon scale hs (1/gamma in float64, gamma in float32); the warp then
// samples delta with the network and applies the cut (sfp_mlp_events).
template <int FORM, int QED>
__device__ __forceinline__ bool sfp_photon_event(const sfp_run_dev* __restrict__ R, const sfp_qed_smem& T,
                                                 const sfp_segment& S, const sfp_instance& I,
                                                 const double* __restrict__ P, double x, double y, double z, double ux,
                                                 double uy, double uz, double t, unsigned int step, long long i,
                                                 double& tau, double& delta, double& hs, double& lchi) {
    using namespace sfp;
    const double dt = R->dt;
    bool ev = false;
    double d = 0.0;
    if (FORM == SFP_FORM_FP64) {
        double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (S.push) sfp_field_program(x, y, z, t, P, F);
        const double ig = inv_gamma_massive(ux, uy, uz);
        const double chi = chi_of(F, ux, uy, uz, ig);
        if (QED == SFP_QED_REJECTION) {
            if (chi != 0.0) {
                double r1, r2;
                sfp_step_uniform2(I.seed, S.stream, step, 0u, i, r1, r2);
                ev = photon_event_rs(chi, ig, dt, r1, r2, T.iAt, T.dAt, T.zN, T.zmax, d);
            }
        } else if (R->mlp_params) {
            ev = od_event_u(chi, ig, dt, tau, R->od_photon, T.od_ph, T.od_chi_min_ph, I.seed, S.stream, step, i, d);
            hs = ig;
            lchi = ev ? log10(chi) : 0.0;
        } else {
            ev = od_event(chi, ig, dt, tau, R->od_photon, T.od_ph, T.od_chi_min_ph, I.seed, S.stream, step, i, d);
        }
        if (ev && !(QED == SFP_QED_OPTICAL_DEPTH && R->mlp_params) && d / ig < R->photon_threshold) ev = false;
    } else {
        float F[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (S.push) sfp_field_program32(x, y, z, t, P, F);
        const float g = sfp32::gamma_of(ux, uy, uz, false);
        const float chi = sfp32::chi_of(F, sfp32::d2f(ux), sfp32::d2f(uy), sfp32::d2f(uz), g);
        if (QED == SFP_QED_REJECTION) {
            // straight-line: the draw and the rate for every lane, the
            // conditions combined at the end (chi = 0 gives W = 0)
            float r1, r2;
            sfp_step_uniform2f(I.seed, S.stream, step, 0u, i, r1, r2);
            const float kRate = (float)((kAlpha * kMe) * (kC * kC) / kHbar);
            const float dl = r1 * r1 * r1;
            const float base = __fdividef(dl, (1.0f - dl) * chi);
            const float W = -kRate * sfp32::rate_core(dl * chi, base, T.iAf, T.dAf, T.inv_dzf, T.zN, T.base_maxf, 1.0f);
            ev = (chi > 0.0f) & (r2 < 3.0f * r1 * r1 * W * __fdividef(sfp32::d2f(dt), g)) &
                 !(dl * g < sfp32::d2f(R->photon_threshold));
            d = (double)dl;
        } else {
            // float32 rate lookup, float64 optical depth
            double u = 0.0;
            ev = !((double)chi < T.od_chi_min_ph) &&
                 od_tau_step((double)sfp32::od_rate(chi, R->od_photon, T.od_phf), (double)__fdividef(1.0f, g), dt, tau, I.seed,
                             S.stream, step, i, u);
            if (R->mlp_params) {
                d = u;
                hs = (double)g;
                lchi = ev ? log10((double)chi) : 0.0;
            } else {
                d = ev ? od_bisect((double)chi, u, R->od_photon) : 0.0;
                if (ev && d * (double)g < R->photon_threshold) ev = false;
            }
        }
        if (!ev) d = 0.0;
    }
    delta = d;
    return ev;
}

// pair creation by a photon at t (qed/rejection_sampling.py:92-107,
// optical_depth.py:64-111)
template <int FORM, int QED>
__device__ __forceinline__ bool sfp_pair_event(const sfp_run_dev* __restrict__ R, const sfp_qed_smem& T,
                                               const sfp_segment& S, const sfp_instance& I,
                                               const double* __restrict__ P, double x, double y, double z, double ux,
                                               double uy, double uz, double t, unsigned int step, long long i,
                                               double& tau, double& delta) {
    using namespace sfp;
    const double dt = R->dt;
    bool ev = false;
    double d = 0.0;
    if (FORM == SFP_FORM_FP64) {
        double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (S.push) sfp_field_program(x, y, z, t, P, F);
        const double ig = inv_gamma_photon(ux, uy, uz);
        const double chi = chi_of(F, ux, uy, uz, ig);
        if (QED == SFP_QED_REJECTION) {
            if (chi != 0.0 && !(chi < T.chi_pair_min)) {
                double r1, r2;
                sfp_step_uniform2(I.seed, S.stream, step, 0u, i, r1, r2);
                ev = pair_event_rs(chi, ig, dt, r1, r2, T.iAt, T.dAt, T.zN, T.zmax, d);
            }
        } else {
            ev = od_event(chi, ig, dt, tau, R->od_pair, T.od_pa, T.od_chi_min_pa, I.seed, S.stream, step, i, d);
        }
    } else {
        float F[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (S.push) sfp_field_program32(x, y, z, t, P, F);
        // in a zero field (outside every pulse: the far-field cut) chi is
        // exactly 0, so neither method can create a pair or change tau
        const bool field = F[0] != 0.f || F[1] != 0.f || F[2] != 0.f || F[3] != 0.f || F[4] != 0.f || F[5] != 0.f;
        if (field) {
            const float g = sfp32::gamma_of(ux, uy, uz, true);
            const float chi = sfp32::chi_of(F, sfp32::d2f(ux), sfp32::d2f(uy), sfp32::d2f(uz), g);
            if (QED == SFP_QED_REJECTION) {
                if (chi > 0.0f && !((double)chi < T.chi_pair_min)) {
                    float r1, r2;
                    sfp_step_uniform2f(I.seed, S.stream, step, 0u, i, r1, r2);
                    const float kRate = (float)((kAlpha * kMe) * (kC * kC) / kHbar);
                    const float base = __fdividef(1.0f, (r1 * (1.0f - r1)) * chi);
                    const float W =
                        kRate * sfp32::rate_core(chi, base, T.iAf, T.dAf, T.inv_dzf, T.zN, T.base_maxf, -1.0f);
                    ev = r2 < W * __fdividef(sfp32::d2f(dt), g);
                    d = (double)r1;
                }
            } else {
                // float32 rate lookup, float64 optical depth
                double u = 0.0;
                ev = !((double)chi < T.od_chi_min_pa) &&
                     od_tau_step((double)sfp32::od_rate(chi, R->od_pair, T.od_paf), (double)__fdividef(1.0f, g), dt, tau, I.seed,
                                 S.stream, step, i, u);
                d = ev ? od_bisect((double)chi, u, R->od_pair) : 0.0;
            }
        }
        if (!ev) d = 0.0;
    }
    delta = d;
    return ev;
}

// Energies of this warp's emission events from the learned sampler: the
// events are packed into per-warp rows, run through the network 16 rows per
// tensor-core tile (sfp_mlp.cuh), and the hard-photon cut is applied.  On
// entry delta[k] holds each event's uniform u, on exit its delta (0 if cut).
template <int FORM, int ITEMS>
__device__ __forceinline__ void sfp_mlp_events(const sfp_run_dev* __restrict__ R, const sfp_mlp::Smem& M,
                                               bool (&ev)[ITEMS], double (&delta)[ITEMS], const double (&hs)[ITEMS],
                                               const double (&lchi)[ITEMS]) {
    constexpr int NW = SFP_TILE / 32;
    __shared__ float s_x[NW][32 * ITEMS][2];
    __shared__ float s_y[NW][32 * ITEMS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const unsigned int lt = (1u << lane) - 1u;
    int rk[ITEMS];
    int ne = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const unsigned int bal = __ballot_sync(0xffffffffu, ev[k]);
        rk[k] = ne + __popc(bal & lt);
        if (ev[k]) {
            s_x[warp][rk[k]][0] = sfp_mlp::feat_chi(lchi[k]);
            s_x[warp][rk[k]][1] = sfp_mlp::feat_u(delta[k]);
        }
        ne += __popc(bal);
    }
    if (ne == 0) return;
    __syncwarp();
    for (int r0 = 0; r0 < ne; r0 += 16) {
        float x0[2], x1[2], y[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = r0 + g + 8 * h;
            x0[h] = r < ne ? s_x[warp][r][0] : 0.0f;
            x1[h] = r < ne ? s_x[warp][r][1] : 0.0f;
        }
        sfp_mlp::tile16(M, x0, x1, y);
        if (t == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + g + 8 * h;
                if (r < ne) s_y[warp][r] = y[h];
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (!ev[k]) continue;
        const double d = sfp_mlp::delta_of(s_y[warp][rk[k]]);
        const bool cut = FORM == SFP_FORM_FP64 ? d / hs[k] < R->photon_threshold : d * hs[k] < R->photon_threshold;
        ev[k] = !cut;
        delta[k] = cut ? 0.0 : d;
    }
    __syncwarp();
}

// largest j with start[j] <= tk (binary search over a group's tile starts)
__device__ __forceinline__ int sfp_find_group_pos(const long long* __restrict__ start, int n, long long tk) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= tk) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Bookkeeping: fold the appends of the step that ran, advance t; then
// (prepare, bit 0) each group's tile length and tile map, tickets,
// super-tile counts.  Bits 1 and 2 of `prepare`: the step's massive /
// photon launch is the long-tile kernel, so that group's tiles must be
// SFP_TILE_MAX long.  One block of 256 threads.
// ---------------------------------------------------------------------------
SFP_DEVICE_INLINE long long sfp_group_map(const sfp_run_dev* __restrict__ R, const sfp_group_dev& G, int tile) {
    long long acc = 0;
    for (int j = 0; j < G.n_seg; ++j) {
        acc = (acc + SFP_SUPER_TILE - 1) / SFP_SUPER_TILE * SFP_SUPER_TILE;
        G.tile_start[j] = acc;
        acc += (R->n_buffered[G.seg[j]] + tile - 1) / tile;
    }
    G.tile_start[G.n_seg] = acc;
    return acc;
}

// the group's tile of this step (SFP_TILE_MIN..SFP_TILE_MAX, a power of two)
// and its tile map; a map too long for the counters takes a longer tile
SFP_DEVICE_INLINE long long sfp_group_plan(const sfp_run_dev* __restrict__ R, const sfp_group_dev& G, int& tile) {
    long long n = 0;
    for (int j = 0; j < G.n_seg; ++j) n += R->n_buffered[G.seg[j]];
    tile = SFP_TILE_MIN;
    while (tile < SFP_TILE_MAX && (long long)tile * SFP_TILE_TARGET < n) tile <<= 1;
    long long tiles = sfp_group_map(R, G, tile);
    while (tiles > G.max_tiles && tile < SFP_TILE_MAX) {
        tile <<= 1;
        tiles = sfp_group_map(R, G, tile);
    }
    return tiles;
}

extern "C" __global__ void __launch_bounds__(256) sfp_book_kernel(const sfp_run_dev* __restrict__ R, int prepare) {
    __shared__ long long s_nsuper_m, s_nsuper_p;
    sfp_step_state* st = R->st;
    const int n = R->n_seg;
    // a step that stopped before writing its children is folded only once resumed
    if (st->pending && !st->append_wait) {
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            R->n_buffered[s] += (long long)R->appended[s];
            R->appended[s] = 0ull;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            st->t = st->t + R->dt;
            st->step += 1;
            st->pending = 0;
        }
    }
    __syncthreads();
    if (!prepare) return;
    if (st->halted || st->error || st->append_wait) {
        if (threadIdx.x == 0) st->skip = 1;
        return;
    }
    if (threadIdx.x == 0) {
        s_nsuper_m = s_nsuper_p = 0;
        long long ps = 0;
        for (int s = 0; s < n; ++s) {
            R->n_buf_step[s] = R->n_buffered[s];
            ps += R->n_buffered[s];
        }
        // each segment's tiles start at a multiple of SFP_SUPER_TILE tiles
        int mt = SFP_TILE_MAX, pt = SFP_TILE_MAX;
        const long long m_tiles = sfp_group_plan(R, R->mg, mt);
        const long long p_tiles = sfp_group_plan(R, R->pg, pt);
        if (m_tiles > R->mg.max_tiles || p_tiles > R->pg.max_tiles) {
            st->error = SFP_DEV_CAPACITY;
            st->skip = 1;
        } else if (((prepare & 2) && mt != SFP_TILE_MAX) || ((prepare & 4) && pt != SFP_TILE_MAX)) {
            st->error = SFP_DEV_TILE;  // the long-tile kernels launched for a step with shorter tiles
            st->skip = 1;
        } else {
            st->n_mtiles = m_tiles;
            st->n_ptiles = p_tiles;
            st->mtile = mt;
            st->ptile = pt;
            st->mticket = 0;
            st->pticket = 0;
            st->skip = 0;
            st->pending = 1;
            st->particle_steps += ps;
            s_nsuper_m = (m_tiles + SFP_SUPER_TILE - 1) / SFP_SUPER_TILE;
            s_nsuper_p = (p_tiles + SFP_SUPER_TILE - 1) / SFP_SUPER_TILE;
        }
    }
    __syncthreads();
    // the group kernels add into the super-tile counts: start them at zero
    for (long long k = threadIdx.x; k < s_nsuper_m; k += blockDim.x) R->mg.super_cnt[k] = 0u;
    for (long long k = threadIdx.x; k < s_nsuper_p; k += blockDim.x) R->pg.super_cnt[k] = 0u;
}

// ---------------------------------------------------------------------------
// The copy ring of both group kernels.  A warp streams its tile (32 to 1024
// particles) 32 at a time through STAGES shared-memory stages
// filled with cp.async, so the state of the next sub-steps is in flight
// while the current one computes.  The copies and the stores address the
// tile through a per-warp descriptor in shared memory, written once per
// tile: slots 0..NC-1 the staged float64 arrays (x, y, z, ux, uy, uz, then
// tau under optical depth, then sx, sy, sz for spin), slot NC the pruned
// flags, slot NC+1 the delta array; each offset to the tile's first
// particle (NULL where the segment has no such array).
// ---------------------------------------------------------------------------
template <int NC>
struct sfp_ring {
    static constexpr int STAGE_BYTES = NC * 32 * 8 + 32;  // NC components + 32 flags
};

template <int QED, bool SPIN>
SFP_DEVICE_INLINE char* sfp_desc_slot(const sfp_segment& S, int c, long long base) {
    constexpr int OD = QED == SFP_QED_OPTICAL_DEPTH ? 1 : 0;
    constexpr int NC = 6 + OD + (SPIN ? 3 : 0);
    double* p = nullptr;
    switch (c) {
        case 0: p = S.x; break;
        case 1: p = S.y; break;
        case 2: p = S.z; break;
        case 3: p = S.ux; break;
        case 4: p = S.uy; break;
        case 5: p = S.uz; break;
        default: break;
    }
    if (OD && c == 6) p = S.tau;
    if (SPIN && c == 6 + OD) p = S.sx;
    if (SPIN && c == 7 + OD) p = S.sy;
    if (SPIN && c == 8 + OD) p = S.sz;
    if (c == NC) return reinterpret_cast<char*>(S.pruned + base);
    if (c == NC + 1) p = S.delta;
    return p ? reinterpret_cast<char*>(p + base) : nullptr;
}

// copies of sub-step `sub` (tile particles 32 sub .. + 31) into one stage:
// copy c is component c/16 of particles 2(c%16), +1 (c < 16 NC) or 16
// flags, always to dst + 16 c, so components land at dst + 256 comp and the
// flags at dst + 256 NC.  `left` = particles of the segment from the tile's
// first on; entries past them are zero-filled and not read.  One commit group.
// Every segment has components 0-5 (x .. uz) and, in the spin variant, the
// spin components; only component 6 under optical depth (tau) can be absent,
// so only copies that can read it test for a NULL array (at compile time
// for the others: copy c = lane + 32 k reads components 2k and 2k + 1).
template <int NC, int OD>
__device__ __forceinline__ void sfp_ring_issue(char* const* D, int sub, long long left, unsigned char* dst,
                                               int lane) {
    constexpr int NCOPY = NC * 16 + 2;
    const bool full = left >= (long long)(sub + 1) * 32;  // warp-uniform: no copy is short
#pragma unroll
    for (int k = 0; k < (NCOPY + 31) / 32; ++k) {
        const int c = lane + 32 * k;
        if (c < NC * 16) {
            const int e = sub * 32 + 2 * (c & 15);
            const char* src = D[c >> 4];
            unsigned int nb = 16u;
            if (!full) nb = left - e >= 2 ? 16u : (left - e == 1 ? 8u : 0u);
            if (OD && 2 * k <= 6 && 6 <= 2 * k + 1 && !src) nb = 0u;  // the segment has no tau array
            sfp::cp_async16(dst + c * 16, nb ? (const void*)(src + (size_t)e * 8) : (const void*)D[NC], nb);
        } else if (c < NCOPY) {
            const int e = sub * 32 + 16 * (c - NC * 16);
            const char* src = D[NC];
            unsigned int nb = 16u;
            if (!full) nb = left - e >= 16 ? 16u : (left - e > 0 ? (unsigned int)(left - e) : 0u);
            sfp::cp_async16(dst + c * 16, nb ? (const void*)(src + e) : (const void*)src, nb);
        }
    }
    sfp::cp_async_commit();
}

// The copies of a full tile (no copy is short): copy c = lane + 32 k of
// sub-step `sub` reads component c / 16 at byte offset 256 sub + 16 (c % 16)
// of the tile (or the flags at 32 sub + 16 (c - 16 NC)), straight from the
// descriptor, with none of the general issue's bounds arithmetic; a
// component the segment lacks is zero-filled.
template <int NC, int OD>
__device__ __forceinline__ void sfp_ring_issue_full(char* const* D, int sub, unsigned char* dst, int lane) {
    constexpr int NCOPY = NC * 16 + 2;
    const unsigned int off = (unsigned int)sub * 256u + 16u * (unsigned int)(lane & 15);
#pragma unroll
    for (int k = 0; k < (NCOPY + 31) / 32; ++k) {
        const int c = lane + 32 * k;
        if (c < NC * 16) {
            const char* p = D[c >> 4];
            const bool has = !(OD && 2 * k <= 6 && 6 <= 2 * k + 1) || p != nullptr;  // see sfp_ring_issue
            sfp::cp_async16(dst + c * 16, has ? (const void*)(p + off) : (const void*)D[NC], has ? 16u : 0u);
        } else if (c < NCOPY) {
            sfp::cp_async16(dst + c * 16, D[NC] + sub * 32 + 16 * (c - NC * 16), 16u);
        }
    }
    sfp::cp_async_commit();
}

// ---------------------------------------------------------------------------
// Massive group.  Each warp takes tiles of the step's length by ticket
// (the next ticket in flight while the tile computes) and streams them
// through the copy ring; after the tables are staged no block barrier is
// taken.  Per particle: the photon event at t (rejection sampling or optical
// depth, hard-photon cut); an emitter is marked (pruned = SFP_MARK) with its
// delta stored and keeps its state at t for the appends kernel; every other
// alive particle is pushed to t+dt (Boris / Boris-TBMT, LL/CLL) and stored.
// The warp's event count goes to its tile's counter and its super-tile's.
// ---------------------------------------------------------------------------
template <int FORM, int QED, int STAGES, bool SPIN, bool LONG>
__device__ __forceinline__ unsigned int sfp_massive_tile(const sfp_run_dev* __restrict__ R, const sfp_qed_smem& T,
                                                         const sfp_mlp::Smem& M, const sfp_segment& S, char** desc,
                                                         unsigned char* ring, int SB, int PT, long long base,
                                                         long long left, double t, double dt, unsigned int step) {
    using namespace sfp;
    constexpr int OD = QED == SFP_QED_OPTICAL_DEPTH ? 1 : 0;
    constexpr int NC = 6 + OD + (SPIN ? 3 : 0);
    const int lane = threadIdx.x & 31;
    const sfp_instance& I = R->inst[S.instance];
    const double* __restrict__ P = sfp_field_params(I);
    const bool rad = S.radiating != 0, push = S.push != 0;
    const sfp_pc32 K32 = push_consts32(S, t, dt);  // float32 form's push constants of this segment
    __syncwarp();  // the previous tile's lanes are done with the descriptor and the stages
    if (lane < NC + 2) desc[lane] = sfp_desc_slot<QED, SPIN>(S, lane, base);
    __syncwarp();
    char* const* D = desc;
    unsigned int cnt = 0;
    // LONG: a tile of SFP_TILE_MAX particles, 32 sub-steps of 32 with
    // compile-time bounds; else the step's shorter tile, sub-steps up to its
    // last particle (`len`, the tile length or fewer at a segment's end)
    const int len = LONG ? SFP_TILE_MAX : (int)min(left, (long long)PT);
    const bool full = LONG ? left >= (long long)SFP_TILE_MAX : len == PT;
    auto issue = [&](int sb, unsigned char* dst) {
        if (full) sfp_ring_issue_full<NC, OD>(D, sb, dst, lane);
        else sfp_ring_issue<NC, OD>(D, sb, LONG ? left : (long long)len, dst, lane);
    };
#pragma unroll
    for (int k = 0; k < STAGES - 1; ++k) {
        if (LONG || 32 * k < len) issue(k, ring + k * SB);
        else cp_async_commit();  // a short tile: nothing to fetch, the group count stays
    }
#pragma unroll 1
    // rd: the stage of `sub` (sub % STAGES); the stage refilled, that of
    // sub + STAGES - 1, is the one before it
    for (int sub = 0, rd = 0; LONG ? sub < SFP_TILE_MAX / 32 : 32 * sub < len;
         ++sub, rd = rd == STAGES - 1 ? 0 : rd + 1) {
        __syncwarp();  // every lane has read the stage about to be refilled
        const int nsub = sub + STAGES - 1;
        if (LONG ? nsub < SFP_TILE_MAX / 32 : 32 * nsub < len)
            issue(nsub, ring + (rd == 0 ? STAGES - 1 : rd - 1) * SB);
        else
            cp_async_commit();
        cp_async_wait<STAGES - 1>();
        __syncwarp();  // the stage of `sub` is complete for the whole warp
        const unsigned char* stg = ring + rd * SB;
        const double* sd = reinterpret_cast<const double*>(stg);
        const int e = sub * 32 + lane;  // particle index from the tile's first
        const long long i = base + e;
        const bool alive = (LONG ? e < left : e < len) && stg[NC * 256 + lane] == 0;
        double x = sd[lane], y = sd[32 + lane], z = sd[64 + lane];
        double ux = sd[96 + lane], uy = sd[128 + lane], uz = sd[160 + lane];
        double tau = OD ? sd[192 + lane] : 0.0;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        if (SPIN) {
            sx = sd[(6 + OD) * 32 + lane];
            sy = sd[(7 + OD) * 32 + lane];
            sz = sd[(8 + OD) * 32 + lane];
        }
        // every lane runs the event test and the push (dead lanes on their
        // zero-filled stage entries); marks and stores are conditional
        bool ev = false;
        double delta = 0.0, hs = 0.0, lchi = 0.0;
        if (rad) {
            const bool e1 = sfp_photon_event<FORM, QED>(R, T, S, I, P, x, y, z, ux, uy, uz, t, step, i, tau, delta, hs,
                                                        lchi);
            ev = alive & e1;
        }
        if (OD && R->mlp_params) {  // warp-uniform: the learned sampler draws the events' energies
            bool e1[1] = {ev};
            double d1[1] = {delta};
            const double h1[1] = {hs}, l1[1] = {lchi};
            sfp_mlp_events<FORM, 1>(R, M, e1, d1, h1, l1);
            ev = e1[0];
            delta = d1[0];
        }
        if (ev) {
            // the appends kernel writes the photon and pushes the parent
            reinterpret_cast<unsigned char*>(D[NC])[e] = SFP_MARK;
            reinterpret_cast<double*>(D[NC + 1])[e] = delta;
        }
        if (FORM == SFP_FORM_FP64) push_massive(x, y, z, ux, uy, uz, sx, sy, sz, S, P, t, dt);
        else push_massive32(x, y, z, ux, uy, uz, sx, sy, sz, S, P, K32);
        if (!ev && alive && push) {
            reinterpret_cast<double*>(D[0])[e] = x;
            reinterpret_cast<double*>(D[1])[e] = y;
            reinterpret_cast<double*>(D[2])[e] = z;
            reinterpret_cast<double*>(D[3])[e] = ux;
            reinterpret_cast<double*>(D[4])[e] = uy;
            reinterpret_cast<double*>(D[5])[e] = uz;
            if (SPIN) {
                reinterpret_cast<double*>(D[6 + OD])[e] = sx;
                reinterpret_cast<double*>(D[7 + OD])[e] = sy;
                reinterpret_cast<double*>(D[8 + OD])[e] = sz;
            }
        }
        if (OD && alive && rad && D[6]) reinterpret_cast<double*>(D[6])[e] = tau;
        cnt += __popc(__ballot_sync(0xffffffffu, ev));
    }
    return cnt;
}

// LONG: the kernel of steps whose tiles are all SFP_TILE_MAX long (the host
// launches it while the group's population guarantees that, and the
// bookkeeping kernel refuses a step planned otherwise with SFP_DEV_TILE).
template <int FORM, int QED, int STAGES, bool LONG>
__device__ __forceinline__ void sfp_massive_body(const sfp_run_dev* __restrict__ R) {
    using namespace sfp;
    constexpr int OD = QED == SFP_QED_OPTICAL_DEPTH ? 1 : 0;
    extern __shared__ __align__(16) double s_tab[];
    __shared__ char* s_desc[SFP_TILE / 32][6 + OD + 3 + 2];
    sfp_step_state* st = R->st;
    if (st->skip || st->n_mtiles == 0) return;
    const long long n_tiles = st->n_mtiles;
    const int PT = LONG ? SFP_TILE_MAX : st->mtile;
    const double t = st->t;
    const double dt = R->dt;
    const unsigned int step = (unsigned int)st->step;
    const sfp_qed_smem T = sfp_stage_tables<FORM, QED>(R, s_tab);
    // learned photon-energy sampler: weights after the tables
    sfp_mlp::Smem& M = *reinterpret_cast<sfp_mlp::Smem*>(reinterpret_cast<unsigned char*>(s_tab) + R->mlp_off);
    if (OD && R->mlp_params) sfp_mlp::stage(M, R->mlp_params);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int SB = R->m_stage_bytes;
    unsigned char* ring = reinterpret_cast<unsigned char*>(s_tab) + R->m_ring_off + (size_t)warp * STAGES * SB;

    int tk = 0;
    if (lane == 0) tk = atomicAdd(&st->mticket, 1);
    long long tile = __shfl_sync(0xffffffffu, tk, 0);
    while (tile < n_tiles) {
        if (lane == 0) tk = atomicAdd(&st->mticket, 1);  // next ticket, in flight during this tile
        const int pos = sfp_find_group_pos(R->mg.tile_start, R->mg.n_seg, tile);
        const sfp_segment& S = R->seg[R->mg.seg[pos]];
        const long long N = R->n_buf_step[R->mg.seg[pos]];
        const long long base = (tile - R->mg.tile_start[pos]) * (long long)PT;
        unsigned int cnt = 0;
        if (base < N) {  // else: alignment padding between segments
            if (S.spin)
                cnt = sfp_massive_tile<FORM, QED, STAGES, true, LONG>(R, T, M, S, s_desc[warp], ring, SB, PT, base,
                                                                      N - base, t, dt, step);
            else
                cnt = sfp_massive_tile<FORM, QED, STAGES, false, LONG>(R, T, M, S, s_desc[warp], ring, SB, PT, base,
                                                                       N - base, t, dt, step);
        }
        if (lane == 0) {
            R->mg.tile_cnt[tile] = cnt;
            if (cnt) atomicAdd(&R->mg.super_cnt[tile / SFP_SUPER_TILE], cnt);
        }
        tile = __shfl_sync(0xffffffffu, tk, 0);
    }
}

// ---------------------------------------------------------------------------
// Photon group.  Same tiles, tickets and ring.  Per photon: the position at
// t (stored position + (step - pos_epoch) pushes, photon_shift), the pair
// event at t; a converted photon is marked (pruned = SFP_MARK, not pushed)
// and its delta stored for the appends kernel.  A photon that does not
// convert writes nothing: its push is the epoch's advance, so the kernel
// reads 49 bytes per photon (state and flag) and writes only events.
//
// Rejection sampling: an event needs r2 < W(r1) dt / gamma, and r2 is never
// below 2^-33 (float32 draws) or 2^-53 (float64 draws).  The pair-rate bound
// of the photon's chi bin (R->pair_bound) times dt / gamma below that means
// no draw passes: the photon is done at once, with no draw and no rate.
// Before any field is evaluated, a photon's energy alone bounds its chi
// (chi <= gamma (|E| + c|B|)_max / E_s, sfp_pair_reachable): most photons
// of a cascade are too soft for any draw to pass anywhere in the pulse and
// are done after reading their momentum.  The others go, with their stored
// state, to a 32-entry per-warp queue in shared memory; full queues get the
// position at t, the field, chi and the bound above, and the few photons
// kept (a few percent) the draws and the rate, so this work is paid by full
// warps instead of by every warp that holds one such photon.  Results are
// those of testing every photon.  Optical depth updates every photon's tau
// and tests each.
// ---------------------------------------------------------------------------
template <int FORM>
__device__ __forceinline__ bool sfp_pair_possible(const sfp_run_dev* __restrict__ R, const sfp_qed_smem& T,
                                                  const float* __restrict__ pb, const sfp_segment& S,
                                                  const double* __restrict__ P, double x, double y, double z,
                                                  double ux, double uy, double uz, double t) {
    using namespace sfp;
    if (FORM == SFP_FORM_FP64) {
        double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (S.push) sfp_field_program(x, y, z, t, P, F);
        const double ig = inv_gamma_photon(ux, uy, uz);
        const double chi = chi_of(F, ux, uy, uz, ig);
        if (chi == 0.0 || chi < T.chi_pair_min) return false;
        return !((double)pb[sfp_pair_bin(__double2float_ru(chi))] * (R->dt * ig) < 0x1p-53);
    } else {
        // straight-line: every condition is combined at the end (no early exit)
        float F[6];
        sfp_field_program32(x, y, z, t, P, F);
        const bool field = S.push && (F[0] != 0.f || F[1] != 0.f || F[2] != 0.f || F[3] != 0.f || F[4] != 0.f ||
                                      F[5] != 0.f);
        const float g = sfp32::gamma_of(ux, uy, uz, true);
        const float chi = sfp32::chi_of(F, sfp32::d2f(ux), sfp32::d2f(uy), sfp32::d2f(uz), g);
        const bool some = chi > 0.0f && !((double)chi < T.chi_pair_min);
        return field & some & !(pb[sfp_pair_bin(chi)] * __fdividef(sfp32::d2f(R->dt), g) < 0x1p-33f);
    }
}

// chi per unit of gamma that no photon can exceed in this instance's field:
// chi <= gamma (|E| + c|B|) / E_s, with sfp_field_bound(P) >= |E| + c|B| over
// all space and time (generated with the field program), rounded up with a
// margin for the rounding of the computed chi; +inf when the field has no
// bound (a focused pulse, a user callable)
SFP_DEVICE_INLINE float sfp_chi_per_gamma(const double* __restrict__ P) {
    const double b = sfp_field_bound(P);
    if (!(b < 1e299)) return __int_as_float(0x7f800000);
    return __double2float_ru(b * (1.0 / sfp32::kEs) * (1.0 + 0x1p-10));
}

// Whether a photon's pair test can pass anywhere in the field, from its
// energy alone: its chi is at most gamma cpg, and pbmax (the prefix maximum
// of the pair-rate bound table, nondecreasing in chi) at that chi bounds the
// rate.  False implies that sfp_pair_possible is false for this photon (the
// same gamma and dt / gamma, a larger chi bin, a larger bound), so such a
// photon skips the field evaluation: results are those of testing it.
template <int FORM>
__device__ __forceinline__ bool sfp_pair_reachable(float cpg, const float* __restrict__ pbmax, double ux, double uy,
                                                   double uz, double dt) {
    using namespace sfp;
    if (FORM == SFP_FORM_FP64) {
        const double ig = inv_gamma_photon(ux, uy, uz);
        const float chimax = __double2float_ru((double)cpg / ig);
        return !((double)pbmax[sfp_pair_bin(chimax)] * (dt * ig) < 0x1p-53);
    } else {
        const float g = sfp32::gamma_of(ux, uy, uz, true);
        return !(pbmax[sfp_pair_bin(g * cpg)] * __fdividef(sfp32::d2f(dt), g) < 0x1p-33f);
    }
}

// a warp's queue of photons whose pair test can pass: tile index and, with STATE, the stored state
// (the float32 form: no second read of their rows); without it the batch
// reads the rows again (the float64 form, whose kernel has no registers to
// spare for the state held across a batch)
template <bool STATE>
struct sfp_pair_queue {
    unsigned short e[32];
};
template <>
struct sfp_pair_queue<true> {
    double x[32], y[32], z[32], ux[32], uy[32], uz[32];
    unsigned short e[32];
};

// the n queued photons (n <= 32), one per lane: their positions at t, the
// field filter (sfp_pair_possible), then the full pair test of those it
// keeps; a converted photon is marked and its delta stored; returns the
// events.  Every lane runs the filter (lanes past n on zeros, masked), as
// the field program votes across the warp.
template <int FORM, bool STATE>
__device__ __forceinline__ unsigned int sfp_pair_batch(const sfp_run_dev* __restrict__ R, const sfp_qed_smem& T,
                                                       const float* __restrict__ pb, const sfp_segment& S,
                                                       const sfp_instance& I, const double* __restrict__ P,
                                                       char* const* D, const sfp_pair_queue<STATE>& q,
                                                       unsigned int n, long long base, double t, double dt,
                                                       unsigned int step, double lag) {
    using namespace sfp;
    const int lane = threadIdx.x & 31;
    const bool in = (unsigned int)lane < n;
    const int e = in ? (int)q.e[lane] : 0;
    double x = 0.0, y = 0.0, z = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
    if (in) {
        if constexpr (STATE) {
            x = q.x[lane], y = q.y[lane], z = q.z[lane];
            ux = q.ux[lane], uy = q.uy[lane], uz = q.uz[lane];
        } else {  // the row again (indices only in the float64 form's queue)
            x = reinterpret_cast<const double*>(D[0])[e], y = reinterpret_cast<const double*>(D[1])[e];
            z = reinterpret_cast<const double*>(D[2])[e], ux = reinterpret_cast<const double*>(D[3])[e];
            uy = reinterpret_cast<const double*>(D[4])[e], uz = reinterpret_cast<const double*>(D[5])[e];
        }
    }
    if (S.push) photon_shift<FORM>(x, y, z, ux, uy, uz, dt, lag);  // the stored position advanced to t
    const bool keep = in & sfp_pair_possible<FORM>(R, T, pb, S, P, x, y, z, ux, uy, uz, t);
    bool ev = false;
    if (__any_sync(0xffffffffu, keep)) {
        if (keep) {
            double tau = 0.0, delta = 0.0;
            ev = sfp_pair_event<FORM, SFP_QED_REJECTION>(R, T, S, I, P, x, y, z, ux, uy, uz, t, step, base + e, tau,
                                                         delta);
            if (ev) {
                reinterpret_cast<unsigned char*>(D[6])[e] = SFP_MARK;
                reinterpret_cast<double*>(D[7])[e] = delta;
            }
        }
    }
    return __popc(__ballot_sync(0xffffffffu, ev));
}

template <bool STATE>
__device__ __forceinline__ void sfp_pair_enqueue(sfp_pair_queue<STATE>& q, unsigned int k, int e, double x, double y,
                                                 double z, double ux, double uy, double uz) {
    q.e[k] = (unsigned short)e;
    if constexpr (STATE) {
        q.x[k] = x;
        q.y[k] = y;
        q.z[k] = z;
        q.ux[k] = ux;
        q.uy[k] = uy;
        q.uz[k] = uz;
    }
}

template <int FORM, int QED, int STAGES, bool LONG>
__device__ __forceinline__ void sfp_photon_body(const sfp_run_dev* __restrict__ R) {
    using namespace sfp;
    constexpr int OD = QED == SFP_QED_OPTICAL_DEPTH ? 1 : 0;
    constexpr bool QUEUE = QED == SFP_QED_REJECTION;
    constexpr int NC = 6 + OD;
    constexpr int SB = sfp_ring<NC>::STAGE_BYTES;
    extern __shared__ __align__(16) double s_tab[];
    __shared__ char* s_desc[SFP_TILE / 32][NC + 2];
    constexpr bool QSTATE = FORM == SFP_FORM_FP32;  // the queue holds the kept photons' state
    __shared__ sfp_pair_queue<QSTATE> s_q[QUEUE ? SFP_TILE / 32 : 1];  // per-warp queue of kept photons
    __shared__ float s_pb[QUEUE ? SFP_PAIR_BOUND_BINS : 1];
    __shared__ float s_pbmax[QUEUE ? SFP_PAIR_BOUND_BINS : 1];  // its prefix maximum
    sfp_step_state* st = R->st;
    if (st->skip || st->n_ptiles == 0) return;
    const long long n_tiles = st->n_ptiles;
    const int PT = LONG ? SFP_TILE_MAX : st->ptile;
    const double t = st->t;
    const double dt = R->dt;
    const unsigned int step = (unsigned int)st->step;
    const double lag = (double)(st->step - st->pos_epoch);  // steps since the stored positions
    const sfp_qed_smem T = sfp_stage_tables<FORM, QED>(R, s_tab);
    if (QUEUE)
        for (int k = threadIdx.x; k < SFP_PAIR_BOUND_BINS; k += blockDim.x) s_pb[k] = R->pair_bound[k];
    __syncthreads();
    if (QUEUE && threadIdx.x == 0) {
        float m = 0.0f;
        for (int k = 0; k < SFP_PAIR_BOUND_BINS; ++k) {
            m = fmaxf(m, s_pb[k]);
            s_pbmax[k] = m;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* ring = reinterpret_cast<unsigned char*>(s_tab) + R->ring_off + (size_t)warp * STAGES * SB;
    char* const* D = s_desc[warp];
    sfp_pair_queue<QSTATE>& q = s_q[QUEUE ? warp : 0];

    int tk = 0;
    if (lane == 0) tk = atomicAdd(&st->pticket, 1);
    long long tile = __shfl_sync(0xffffffffu, tk, 0);
    while (tile < n_tiles) {
        if (lane == 0) tk = atomicAdd(&st->pticket, 1);  // next ticket, in flight during this tile
        const int pos = sfp_find_group_pos(R->pg.tile_start, R->pg.n_seg, tile);
        const int si = R->pg.seg[pos];
        const sfp_segment& S = R->seg[si];
        const sfp_instance& I = R->inst[S.instance];
        const double* __restrict__ P = sfp_field_params(I);
        const float cpg = QUEUE ? sfp_chi_per_gamma(P) : 0.0f;  // chi per gamma no photon exceeds here
        const long long N = R->n_buf_step[si];
        const long long base = (tile - R->pg.tile_start[pos]) * (long long)PT;
        if (base >= N) {  // alignment padding between segments: no photons
            if (lane == 0) R->pg.tile_cnt[tile] = 0u;
            tile = __shfl_sync(0xffffffffu, tk, 0);
            continue;
        }
        // LONG: 32 sub-steps of 32 with compile-time bounds; else sub-steps up
        // to the tile's last photon (`len`: the tile length or fewer at a
        // segment's end)
        const long long left = N - base;
        const int len = LONG ? SFP_TILE_MAX : (int)min(left, (long long)PT);
        const bool bw = S.bw != 0, push = S.push != 0;
        __syncwarp();  // the previous tile's lanes are done with its descriptor, stages and queue
        if (lane < NC + 2) s_desc[warp][lane] = sfp_desc_slot<QED, false>(S, lane, base);
        __syncwarp();
        unsigned int cnt = 0, qn = 0;
        const bool full = LONG ? left >= (long long)SFP_TILE_MAX : len == PT;
        // full long tiles of the float32 form without optical depth: each
        // lane's three component copies (components 2k + lane/16, k = 0..2)
        // read from per-tile pointers held in registers, lanes 0-1 copy the
        // flags; no descriptor reads per stage.  (The float64 form and the
        // any-tile kernel have no registers to spare for them.)
        constexpr bool REGPTR = FORM == SFP_FORM_FP32 && !OD && LONG;
        const char* q0 = nullptr;
        const char* q1 = nullptr;
        const char* q2 = nullptr;
        if (REGPTR && full) {
            const int h = lane >> 4, o = 16 * (lane & 15);
            q0 = D[h] + o;
            q1 = D[2 + h] + o;
            q2 = D[4 + h] + o;
        }
        auto issue = [&](int sb, unsigned char* dst) {
            if (REGPTR && full) {
                const unsigned int off = (unsigned int)sb * 256u;
                sfp::cp_async16(dst + lane * 16, q0 + off, 16u);
                sfp::cp_async16(dst + (lane + 32) * 16, q1 + off, 16u);
                sfp::cp_async16(dst + (lane + 64) * 16, q2 + off, 16u);
                if (lane < 2) sfp::cp_async16(dst + (lane + 96) * 16, D[NC] + sb * 32 + 16 * lane, 16u);
                sfp::cp_async_commit();
            } else if (full) {
                sfp_ring_issue_full<NC, OD>(D, sb, dst, lane);
            } else {
                sfp_ring_issue<NC, OD>(D, sb, LONG ? left : (long long)len, dst, lane);
            }
        };
#pragma unroll
        for (int k = 0; k < STAGES - 1; ++k) {
            if (LONG || 32 * k < len) issue(k, ring + k * SB);
            else cp_async_commit();  // a short tile: nothing to fetch, the group count stays
        }
#pragma unroll 1
        for (int sub = 0; LONG ? sub < SFP_TILE_MAX / 32 : 32 * sub < len; ++sub) {
            __syncwarp();  // every lane has read the stage about to be refilled
            const int nsub = sub + STAGES - 1;
            if (LONG ? nsub < SFP_TILE_MAX / 32 : 32 * nsub < len) issue(nsub, ring + (nsub % STAGES) * SB);
            else cp_async_commit();
            cp_async_wait<STAGES - 1>();
            __syncwarp();  // the stage of `sub` is complete for the whole warp
            const unsigned char* stg = ring + (sub % STAGES) * SB;
            const double* sd = reinterpret_cast<const double*>(stg);
            const int e = sub * 32 + lane;  // photon index from the tile's first
            const long long i = base + e;
            const bool alive = (LONG ? e < left : e < len) && stg[NC * 256 + lane] == 0;
            double x = sd[lane], y = sd[32 + lane], z = sd[64 + lane];
            double ux = sd[96 + lane], uy = sd[128 + lane], uz = sd[160 + lane];
            // the step's push is carried by the epoch (pos_epoch), so a photon
            // that does not convert stores nothing
            if (QUEUE) {
                // from its energy alone, whether a photon's pair test can pass
                // anywhere in the field; those that can go, with their stored
                // state, to the queue, where the position at t, the field and
                // the rate bound are evaluated for full warps
                const bool keep = alive & bw & push & sfp_pair_reachable<FORM>(cpg, s_pbmax, ux, uy, uz, dt);
                // kept photons fill the queue; a full queue is tested at once and
                // the sub-step's remaining kept photons start the next one
                const unsigned int kb = __ballot_sync(0xffffffffu, keep);
                const unsigned int slot = qn + __popc(kb & ((1u << lane) - 1u)), nk = __popc(kb);
                if (keep && slot < 32u) sfp_pair_enqueue(q, slot, e, x, y, z, ux, uy, uz);
                if (qn + nk >= 32u) {
                    __syncwarp();  // the queue entries are written
                    cnt += sfp_pair_batch<FORM, QSTATE>(R, T, s_pb, S, I, P, D, q, 32u, base, t, dt, step, lag);
                    __syncwarp();  // every lane has read its entry
                    if (keep && slot >= 32u) sfp_pair_enqueue(q, slot - 32u, e, x, y, z, ux, uy, uz);
                    qn = qn + nk - 32u;
                } else {
                    qn += nk;
                }
            } else {
                double tau = OD ? sd[192 + lane] : 0.0;
                bool ev = false;
                double delta = 0.0;
                if (push) photon_shift<FORM>(x, y, z, ux, uy, uz, dt, lag);  // the position at t
                if (alive && bw)
                    ev = sfp_pair_event<FORM, QED>(R, T, S, I, P, x, y, z, ux, uy, uz, t, step, i, tau, delta);
                if (ev) {
                    // converted photons are pruned, not pushed (cpu.py:190); marked until their pairs are written
                    reinterpret_cast<unsigned char*>(D[NC])[e] = SFP_MARK;
                    reinterpret_cast<double*>(D[NC + 1])[e] = delta;
                }
                if (OD && alive && bw && D[6]) reinterpret_cast<double*>(D[6])[e] = tau;
                cnt += __popc(__ballot_sync(0xffffffffu, ev));
            }
        }
        if (QUEUE && qn) {  // the tile's last kept photons
            __syncwarp();
            cnt += sfp_pair_batch<FORM, QSTATE>(R, T, s_pb, S, I, P, D, q, qn, base, t, dt, step, lag);
        }
        if (lane == 0) {
            R->pg.tile_cnt[tile] = cnt;
            if (cnt) atomicAdd(&R->pg.super_cnt[tile / SFP_SUPER_TILE], cnt);
        }
        tile = __shfl_sync(0xffffffffu, tk, 0);
    }
}

// ---------------------------------------------------------------------------
// Scan: one block.  For each group, an exclusive scan of the super-tile
// event counts in tile order, restarted at each instance and kept per
// append channel, so super_pre[s] is the number of children that the same
// instance's earlier segments and tiles with the same destinations append
// before super-tile s.  Adds every segment's events to its destinations'
// append counts, then checks that every destination holds this step's
// children; if one does not, the step waits for the host (append_wait).
// ---------------------------------------------------------------------------
// segment of super-tile s of group G and whether s starts a chain (the first
// super-tile of its instance's tiles in that group)
SFP_DEVICE_INLINE void sfp_super_info(const sfp_run_dev* __restrict__ R, const sfp_group_dev& G, long long s, int& si,
                                      bool& head) {
    const long long tile = s * SFP_SUPER_TILE;
    si = G.seg[sfp_find_group_pos(G.tile_start, G.n_seg, tile)];
    if (s == 0) {
        head = true;
        return;
    }
    const int prev = G.seg[sfp_find_group_pos(G.tile_start, G.n_seg, tile - SFP_SUPER_TILE)];
    head = R->seg[prev].instance != R->seg[si].instance;
}

SFP_DEVICE_INLINE uint4 shfl_up_u4(uint4 v, int o) {
    return uint4{__shfl_up_sync(0xffffffffu, v.x, o), __shfl_up_sync(0xffffffffu, v.y, o),
                 __shfl_up_sync(0xffffffffu, v.z, o), __shfl_up_sync(0xffffffffu, v.w, o)};
}

// inclusive warp scan of (head, value) pairs: a head restarts the sum
SFP_DEVICE_INLINE void seg_scan_warp(unsigned int& h, uint4& v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int oh = __shfl_up_sync(0xffffffffu, h, o);
        const uint4 ov = shfl_up_u4(v, o);
        if (lane >= o) {
            if (!h) v = sfp::u4_add(ov, v);
            h |= oh;
        }
    }
}

// a segment's events become appends of its destinations: photons (massive
// group) or one electron and one positron each (photon group)
template <bool MASSIVE>
SFP_DEVICE_INLINE void sfp_add_appends(const sfp_run_dev* __restrict__ R, int si, unsigned long long n) {
    if (!n) return;
    const sfp_segment& S = R->seg[si];
    if (MASSIVE) {
        atomicAdd(&R->appended[S.photon_dest], n);
    } else {
        atomicAdd(&R->appended[S.ele_dest], n);
        atomicAdd(&R->appended[S.pos_dest], n);
    }
}

// block-wide: every thread calls it (n_tiles is uniform)
template <bool MASSIVE>
__device__ __forceinline__ void sfp_scan_group(const sfp_run_dev* __restrict__ R, const sfp_group_dev& G,
                                               long long n_tiles, unsigned int* s_wh, uint4* s_wv) {
    const long long n_super = (n_tiles + SFP_SUPER_TILE - 1) / SFP_SUPER_TILE;
    if (n_super == 0) return;
    const long long per = (n_super + blockDim.x - 1) / blockDim.x;
    const long long s0 = min(n_super, (long long)threadIdx.x * per), s1 = min(n_super, s0 + per);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // this thread's run of super-tiles as one scan element
    unsigned int h = 0;
    uint4 v{0u, 0u, 0u, 0u};
    for (long long s = s0; s < s1; ++s) {
        int si;
        bool hd;
        sfp_super_info(R, G, s, si, hd);
        if (hd) {
            h = 1;
            v = uint4{0u, 0u, 0u, 0u};
        }
        v = sfp::u4_add(v, sfp::u4_one(R->seg[si].channel, G.super_cnt[s]));
    }
    seg_scan_warp(h, v);
    __syncthreads();  // the previous user of s_wh / s_wv is done
    if (lane == 31) {
        s_wh[warp] = h;
        s_wv[warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        unsigned int wh = lane < nw ? s_wh[lane] : 0u;
        uint4 wv = lane < nw ? s_wv[lane] : uint4{0u, 0u, 0u, 0u};
        seg_scan_warp(wh, wv);
        unsigned int eh = __shfl_up_sync(0xffffffffu, wh, 1);
        uint4 ev = shfl_up_u4(wv, 1);
        if (lane == 0) {
            eh = 0u;
            ev = uint4{0u, 0u, 0u, 0u};
        }
        if (lane < nw) {
            s_wh[lane] = eh;
            s_wv[lane] = ev;
        }
    }
    __syncthreads();
    // exclusive value of this thread: earlier warps, then earlier lanes of this warp
    unsigned int lh = __shfl_up_sync(0xffffffffu, h, 1);
    uint4 lv = shfl_up_u4(v, 1);
    if (lane == 0) {
        lh = 0u;
        lv = uint4{0u, 0u, 0u, 0u};
    }
    uint4 run = lh ? lv : sfp::u4_add(s_wv[warp], lv);
    int cur = -1;
    unsigned long long acc = 0ull;
    for (long long s = s0; s < s1; ++s) {
        int si;
        bool hd;
        sfp_super_info(R, G, s, si, hd);
        if (hd) run = uint4{0u, 0u, 0u, 0u};
        const int ch = R->seg[si].channel;
        G.super_pre[s] = (long long)sfp::u4_get(run, ch);
        const unsigned int c = G.super_cnt[s];
        run = sfp::u4_add(run, sfp::u4_one(ch, c));
        if (si != cur) {
            if (cur >= 0) sfp_add_appends<MASSIVE>(R, cur, acc);
            cur = si;
            acc = 0ull;
        }
        acc += c;
    }
    if (cur >= 0) sfp_add_appends<MASSIVE>(R, cur, acc);
}

extern "C" __global__ void __launch_bounds__(1024) sfp_scan_kernel(const sfp_run_dev* __restrict__ R) {
    __shared__ unsigned int s_wh[32];
    __shared__ uint4 s_wv[32];
    __shared__ int s_short;
    const sfp_step_state* st = R->st;
    if (st->skip) return;
    if (R->any_rad) sfp_scan_group<true>(R, R->mg, st->n_mtiles, s_wh, s_wv);
    if (R->any_bw) sfp_scan_group<false>(R, R->pg, st->n_ptiles, s_wh, s_wv);
    if (threadIdx.x == 0) s_short = 0;
    __syncthreads();  // every append count is in
    // exact room check: the appends kernel writes nothing unless every
    // destination holds its children; otherwise the step waits for the host
    for (int c = threadIdx.x; c < R->n_dseg; c += blockDim.x) {
        const int d = R->dseg[c];
        if (R->n_buf_step[d] + (long long)R->appended[d] > R->seg[d].capacity) atomicExch(&s_short, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_short) {
        R->st->append_wait = 1;
        R->st->halted = 1;
    }
}

// ---------------------------------------------------------------------------
// Appends.  The massive group's tile counters and then the photon group's
// are dealt to the warps by stride (warp w: tiles w, w + nw, ...), read 32
// at a time, one per lane; for a tile with events the warp adds the counts of
// the earlier tiles of its super-tile to the super-tile's prefix, gathers
// the tile's marked particles in index order into shared memory (16 flags
// per lane per pass) and then handles 32 of them at a time, so every lane
// works: the k-th marked particle's children go to slot
// n_buffered(start of step) + prefix + k.
//   massive: the photon (cpu.py:89-116) from the parent's state at t,
//            pushed; the parent's recoil (cpu.py:76-87) and push; unmarked;
//   photon:  e- with delta u and e+ with (1 - delta) u (cpu.py:119-189),
//            both pushed; the photon pruned.
// ---------------------------------------------------------------------------
template <int FORM>
__device__ __forceinline__ void sfp_write_pair_child(const sfp_segment& D, long long slot, const double* __restrict__ P,
                                                     double x, double y, double z, double ux, double uy, double uz,
                                                     double t, double dt) {
    using namespace sfp;
    if (D.push) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        if (FORM == SFP_FORM_FP64) push_massive(x, y, z, ux, uy, uz, sx, sy, sz, D, P, t, dt);
        else push_massive32(x, y, z, ux, uy, uz, sx, sy, sz, D, P, push_consts32(D, t, dt));
    }
    D.x[slot] = x;
    D.y[slot] = y;
    D.z[slot] = z;
    D.ux[slot] = ux;
    D.uy[slot] = uy;
    D.uz[slot] = uz;
    if (D.spin) {
        D.sx[slot] = 0.0;
        D.sy[slot] = 0.0;
        D.sz[slot] = 0.0;
    }
    if (D.tau) D.tau[slot] = 0.0;
    D.pruned[slot] = 0;
}

template <int FORM>
__device__ __forceinline__ void sfp_write_photon(const sfp_run_dev* __restrict__ R, const sfp_segment& S, long long i,
                                                 long long rank, long long pre, const double* __restrict__ P, double t,
                                                 double dt, double lag) {
    using namespace sfp;
    const sfp_segment& D = R->seg[S.photon_dest];
    const long long slot = R->n_buf_step[S.photon_dest] + pre + rank;
    double x = S.x[i], y = S.y[i], z = S.z[i];
    double ux = S.ux[i], uy = S.uy[i], uz = S.uz[i];
    const double d = S.delta[i];
    double cx = x, cy = y, cz = z;
    const double cux = d * ux, cuy = d * uy, cuz = d * uz;
    // the child is pushed in its creation step (simulation.py:117-121): at
    // the next step it is at x + one push, so it is stored `lag` pushes
    // behind x, as of pos_epoch like every photon of its segment
    if (D.push) photon_shift<FORM>(cx, cy, cz, cux, cuy, cuz, dt, -lag);
    D.x[slot] = cx;
    D.y[slot] = cy;
    D.z[slot] = cz;
    D.ux[slot] = cux;
    D.uy[slot] = cuy;
    D.uz[slot] = cuz;
    if (D.tau) D.tau[slot] = 0.0;
    D.pruned[slot] = 0;
    if (S.rr == SFP_RR_PHOTON) {
        const double f = 1.0 - d;
        ux = ux * f;
        uy = uy * f;
        uz = uz * f;
    }
    if (S.push) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        if (S.spin) {
            sx = S.sx[i];
            sy = S.sy[i];
            sz = S.sz[i];
        }
        if (FORM == SFP_FORM_FP64) push_massive(x, y, z, ux, uy, uz, sx, sy, sz, S, P, t, dt);
        else push_massive32(x, y, z, ux, uy, uz, sx, sy, sz, S, P, push_consts32(S, t, dt));
        S.x[i] = x;
        S.y[i] = y;
        S.z[i] = z;
        if (S.spin) {
            S.sx[i] = sx;
            S.sy[i] = sy;
            S.sz[i] = sz;
        }
    }
    if (S.push || S.rr == SFP_RR_PHOTON) {
        S.ux[i] = ux;
        S.uy[i] = uy;
        S.uz[i] = uz;
    }
    S.pruned[i] = 0;
}

template <int FORM>
__device__ __forceinline__ void sfp_write_pair(const sfp_run_dev* __restrict__ R, const sfp_segment& S, long long i,
                                               long long rank, long long pre, const double* __restrict__ P, double t,
                                               double dt, double lag) {
    const double d = S.delta[i];
    double px = S.x[i], py = S.y[i], pz = S.z[i];
    const double pux = S.ux[i], puy = S.uy[i], puz = S.uz[i];
    // the converted photon at t, written out: it is pruned, and pruned
    // photons keep their stored position (no later advance)
    if (S.push) {
        sfp::photon_shift<FORM>(px, py, pz, pux, puy, puz, dt, lag);
        S.x[i] = px;
        S.y[i] = py;
        S.z[i] = pz;
    }
    S.pruned[i] = 1;
    const long long be = R->n_buf_step[S.ele_dest] + pre + rank;
    const long long bp = R->n_buf_step[S.pos_dest] + pre + rank;
    sfp_write_pair_child<FORM>(R->seg[S.ele_dest], be, P, px, py, pz, d * pux, d * puy, d * puz, t, dt);
    const double d2 = 1.0 - d;
    sfp_write_pair_child<FORM>(R->seg[S.pos_dest], bp, P, px, py, pz, d2 * pux, d2 * puy, d2 * puz, t, dt);
}

template <int FORM, bool MASSIVE>
__device__ __forceinline__ void sfp_append_tile(const sfp_run_dev* __restrict__ R, const sfp_group_dev& G, int PT,
                                                long long tile, unsigned int c, unsigned short* list, double t,
                                                double dt, double lag) {
    using namespace sfp;
    const int lane = threadIdx.x & 31;
    const long long s = tile / SFP_SUPER_TILE;
    unsigned int part = 0u;
    for (long long k = s * SFP_SUPER_TILE + lane; k < tile; k += 32) part += G.tile_cnt[k];
    const long long pre = G.super_pre[s] + (long long)warp_sum(part);
    const int pos = sfp_find_group_pos(G.tile_start, G.n_seg, tile);
    const sfp_segment& S = R->seg[G.seg[pos]];
    const double* __restrict__ P = sfp_field_params(R->inst[S.instance]);
    const long long N = R->n_buf_step[G.seg[pos]];
    const long long base = (tile - G.tile_start[pos]) * (long long)PT;
    const int len = (int)min(N - base, (long long)PT);  // the tile's particles
    // the tile's marked particles, in index order: lane q covers 16 flags per pass
    unsigned int n = 0u;
    for (int q0 = 0; q0 < len && n < c; q0 += 512) {
        const int e0 = q0 + 16 * lane;
        const unsigned char* f = S.pruned + base + e0;
        unsigned int m = 0u;
        if (e0 + 16 <= len) {
            m = marks16(*reinterpret_cast<const uint4*>(f));
        } else {
            for (int b = 0; b < 16; ++b)
                if (e0 + b < len && f[b] == SFP_MARK) m |= 1u << b;
        }
        const unsigned int k = __popc(m);
        const unsigned int inc = warp_incl_scan(k);
        unsigned int w = n + inc - k;
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1u;
            if (w < (unsigned int)len) list[w] = (unsigned short)(e0 + b);
            ++w;
        }
        n += __shfl_sync(0xffffffffu, inc, 31);
    }
    __syncwarp();
    // never more children than the scan counted and made room for
    n = min(min(n, c), (unsigned int)len);
    for (unsigned int j0 = 0; j0 < n; j0 += 32) {
        const unsigned int j = j0 + lane;
        if (j < n) {
            const long long i = base + list[j];
            if (MASSIVE) sfp_write_photon<FORM>(R, S, i, j, pre, P, t, dt, lag);
            else sfp_write_pair<FORM>(R, S, i, j, pre, P, t, dt, lag);
        }
    }
    __syncwarp();  // the list is read before the next tile rewrites it
}

template <int FORM>
__device__ __forceinline__ void sfp_appends_body(const sfp_run_dev* __restrict__ R) {
    __shared__ unsigned short s_list[SFP_TILE / 32][SFP_TILE_MAX];
    const sfp_step_state* st = R->st;
    if (st->skip || st->append_wait) return;
    const long long nm = R->any_rad ? st->n_mtiles : 0, np = R->any_bw ? st->n_ptiles : 0;
    const int mt = st->mtile, pt = st->ptile;
    const long long n_all = nm + np;
    const double t = st->t;
    const double dt = R->dt;
    const double lag = (double)(st->step - st->pos_epoch);  // photon positions: steps since stored
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    // warp gw owns tiles gw, gw + nw, gw + 2 nw, ...: tiles with events
    // (every massive tile in a cascade, a few photon tiles) spread over all
    // warps instead of queueing behind one warp per 32 neighbours
    for (long long j0 = 0; gw + j0 * nw < n_all; j0 += 32) {
        const long long mine = gw + (j0 + lane) * nw;
        unsigned int mc = 0u;
        if (mine < nm) mc = R->mg.tile_cnt[mine];
        else if (mine < n_all) mc = R->pg.tile_cnt[mine - nm];
        unsigned int busy = __ballot_sync(0xffffffffu, mc != 0u);
        while (busy) {
            const int b = __ffs(busy) - 1;
            busy &= busy - 1u;
            const long long tg = gw + (j0 + b) * nw;
            const unsigned int c = __shfl_sync(0xffffffffu, mc, b);
            if (tg < nm) sfp_append_tile<FORM, true>(R, R->mg, mt, tg, c, s_list[warp], t, dt, lag);
            else sfp_append_tile<FORM, false>(R, R->pg, pt, tg - nm, c, s_list[warp], t, dt, lag);
        }
    }
}

// kernels: sfp_massive_<form>_<qed>_s<stages>_b<blocks>,
// sfp_photon_<form>_<qed>_s<stages>_b<blocks>, sfp_scan_kernel, sfp_appends_<form>
// (long-tile kernels) and sfp_massive_<form>_<qed>_s<stages>_b<blocks>_t,
// sfp_photon_..._t (any tile length: the steps of small populations)
#define SFP_MASSIVE_KERNEL(FORM_S, QED_S, FORM, QED, STAGES, MINB)                                             \
    extern "C" __global__ void __launch_bounds__(SFP_TILE, MINB)                                              \
        sfp_massive_##FORM_S##_##QED_S##_s##STAGES##_b##MINB(const sfp_run_dev* __restrict__ R) {             \
        sfp_massive_body<FORM, QED, STAGES, true>(R);                                                        \
    }
#define SFP_PHOTON_KERNEL(FORM_S, QED_S, FORM, QED, STAGES, MINB)                                              \
    extern "C" __global__ void __launch_bounds__(SFP_TILE, MINB)                                              \
        sfp_photon_##FORM_S##_##QED_S##_s##STAGES##_b##MINB(const sfp_run_dev* __restrict__ R) {              \
        sfp_photon_body<FORM, QED, STAGES, true>(R);                                                         \
    }
#define SFP_MASSIVE_KERNEL_T(FORM_S, QED_S, FORM, QED, STAGES, MINB)                                           \
    extern "C" __global__ void __launch_bounds__(SFP_TILE, MINB)                                              \
        sfp_massive_##FORM_S##_##QED_S##_s##STAGES##_b##MINB##_t(const sfp_run_dev* __restrict__ R) {         \
        sfp_massive_body<FORM, QED, STAGES, false>(R);                                                       \
    }
#define SFP_PHOTON_KERNEL_T(FORM_S, QED_S, FORM, QED, STAGES, MINB)                                            \
    extern "C" __global__ void __launch_bounds__(SFP_TILE, MINB)                                              \
        sfp_photon_##FORM_S##_##QED_S##_s##STAGES##_b##MINB##_t(const sfp_run_dev* __restrict__ R) {          \
        sfp_photon_body<FORM, QED, STAGES, false>(R);                                                        \
    }

// ---------------------------------------------------------------------------
// Photon positions written out (sfp_run_sync_positions): every photon of a
// pushed photon segment that is not pruned (alive, or marked inside a step
// that stopped for room) advances by the steps since pos_epoch; pruned
// photons keep the position they were pruned at.  sfp_epoch_kernel, launched
// after it, then moves pos_epoch to the current step (a second launch, so
// that every block of the first has read the old epoch).
// ---------------------------------------------------------------------------
template <int FORM>
__device__ __forceinline__ void sfp_sync_positions_body(const sfp_run_dev* __restrict__ R) {
    const sfp_step_state* st = R->st;
    const double lag = (double)(st->step - st->pos_epoch);
    if (lag == 0.0) return;
    const double dt = R->dt;
    const long long first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int k = 0; k < R->pg.n_seg; ++k) {
        const int si = R->pg.seg[k];
        const sfp_segment& S = R->seg[si];
        if (!S.push) continue;
        const long long N = R->n_buffered[si];
        for (long long i = first; i < N; i += stride) {
            if (S.pruned[i] == 1) continue;
            double x = S.x[i], y = S.y[i], z = S.z[i];
            sfp::photon_shift<FORM>(x, y, z, S.ux[i], S.uy[i], S.uz[i], dt, lag);
            S.x[i] = x;
            S.y[i] = y;
            S.z[i] = z;
        }
    }
}

extern "C" __global__ void __launch_bounds__(32) sfp_epoch_kernel(const sfp_run_dev* __restrict__ R) {
    if (threadIdx.x == 0) R->st->pos_epoch = R->st->step;
}

#if defined(SFP_STEP_FORM_FP64)
extern "C" __global__ void __launch_bounds__(SFP_TILE, 2) sfp_appends_fp64(const sfp_run_dev* __restrict__ R) {
    sfp_appends_body<SFP_FORM_FP64>(R);
}
extern "C" __global__ void __launch_bounds__(256) sfp_sync_positions_fp64(const sfp_run_dev* __restrict__ R) {
    sfp_sync_positions_body<SFP_FORM_FP64>(R);
}
#if defined(SFP_STEP_QED_RS)
SFP_MASSIVE_KERNEL(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 2, 2)
SFP_MASSIVE_KERNEL(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 3, 2)
SFP_PHOTON_KERNEL(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 2, 3)
SFP_PHOTON_KERNEL(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 3, 3)
SFP_PHOTON_KERNEL(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 3, 2)
SFP_MASSIVE_KERNEL_T(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 2, 2)
SFP_PHOTON_KERNEL_T(fp64, rs, SFP_FORM_FP64, SFP_QED_REJECTION, 3, 3)
#else
SFP_MASSIVE_KERNEL(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 2, 2)
SFP_MASSIVE_KERNEL(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 3, 2)
SFP_PHOTON_KERNEL(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 2, 3)
SFP_PHOTON_KERNEL(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 3, 3)
SFP_MASSIVE_KERNEL_T(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 2, 2)
SFP_PHOTON_KERNEL_T(fp64, od, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 3, 3)
#endif
#endif
#if defined(SFP_STEP_FORM_FP32)
extern "C" __global__ void __launch_bounds__(SFP_TILE, 3) sfp_appends_fp32(const sfp_run_dev* __restrict__ R) {
    sfp_appends_body<SFP_FORM_FP32>(R);
}
extern "C" __global__ void __launch_bounds__(256) sfp_sync_positions_fp32(const sfp_run_dev* __restrict__ R) {
    sfp_sync_positions_body<SFP_FORM_FP32>(R);
}
#if defined(SFP_STEP_QED_RS)
SFP_MASSIVE_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 3)
SFP_MASSIVE_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 3, 3)
SFP_MASSIVE_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 3, 2)
SFP_MASSIVE_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 4, 2)
SFP_MASSIVE_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 4)
SFP_PHOTON_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 4)
SFP_PHOTON_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 3, 4)
SFP_PHOTON_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 3, 3)
SFP_PHOTON_KERNEL(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 4, 3)
SFP_MASSIVE_KERNEL_T(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 3)
SFP_PHOTON_KERNEL_T(fp32, rs, SFP_FORM_FP32, SFP_QED_REJECTION, 3, 3)
#else
SFP_MASSIVE_KERNEL(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 2, 3)
SFP_MASSIVE_KERNEL(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 3, 2)
SFP_PHOTON_KERNEL(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 3, 4)
SFP_PHOTON_KERNEL(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 3, 3)
SFP_MASSIVE_KERNEL_T(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 2, 3)
SFP_PHOTON_KERNEL_T(fp32, od, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 3, 3)
#endif
#endif
#endif  // SFP_WANT_STEP

#if defined(SFP_WANT_FIELD_EVAL)

// Field evaluation of the program at particle positions (Fields.field_func,
// fields.py:31-46): the per-op boundary kernel of the NVRTC module.
extern "C" __global__ void __launch_bounds__(256)
    sfp_field_eval_kernel(const double* __restrict__ P, const double* __restrict__ x, const double* __restrict__ y,
                          const double* __restrict__ z, double t, long long N, const unsigned char* __restrict__ pruned,
                          double* __restrict__ Ex, double* __restrict__ Ey, double* __restrict__ Ez,
                          double* __restrict__ Bx, double* __restrict__ By, double* __restrict__ Bz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        if (pruned[i]) continue;
        double F[6];
        sfp_field_program(x[i], y[i], z[i], t, P, F);
        Ex[i] = F[0]; Ey[i] = F[1]; Ez[i] = F[2];
        Bx[i] = F[3]; By[i] = F[4]; Bz[i] = F[5];
    }
}
#endif  // SFP_WANT_FIELD_EVAL
