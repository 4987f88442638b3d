// sfp_device32.cuh -- float32 arithmetic of the fused step's FP32 form.
//
// The particle state stays float64 in HBM.  Fields, chi, the QED samplers
// and the Boris / Thomas-BMT / Landau-Lifshitz updates are evaluated in
// float32 (MUFU transcendentals after explicit range reduction, divisions
// as __fdividef: a reciprocal and a product, within 2 ulp), and every
// update is applied as a float32 INCREMENT to the float64 state:
//   x += dx,  u += du,  s += ds          (float64 accumulation of float32 steps)
// so rounding errors scale with the step, not with |x|, |u| (the role Kahan
// compensation plays for float32 storage).  gamma = sqrt(1 + u^2) is taken in
// float64 when gamma > 1e4, where 1 + u^2 is below float32 resolution.
// The phase argument x - x0 - dir c t of the pulses is formed in float64.
#pragma once
#include "sfp_device.cuh"

namespace sfp32 {

constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr float kCf = 299792458.0f;
// Schwinger field E_s = m^2 c^3 / (e hbar); chi is formed in units of E_s
constexpr double kEs = (sfp::kMe * sfp::kMe) * (sfp::kC * (sfp::kC * sfp::kC)) / (sfp::kE * sfp::kHbar);
constexpr float kInvEs = (float)(1.0 / kEs);
constexpr float kCOverEs = (float)(sfp::kC / kEs);
constexpr double kGammaSplit = 1.0e4;

// float64 -> float32, rounded to nearest, as one conversion instruction.
// The float32 form is compiled with float32 denormals flushed (-ftz=true),
// under which a plain (float) cast of a double must also flush a denormal
// result and takes two more instructions per conversion.  The values
// converted here (positions, momenta, phases, parameters) are either 0 or
// far above the float32 denormal range; a denormal result would in any case
// be flushed by the float32 arithmetic it enters.
SFP_DEVICE_INLINE float d2f(double v) {
    float r;
    asm("cvt.rn.f32.f64 %0, %1;" : "=f"(r) : "d"(v));
    return r;
}

// cos / sin of a float32 phase of any size: reduce to [-pi, pi], then MUFU
SFP_DEVICE_INLINE float cos_r(float a) {
    const float k = rintf(a * kInvTwoPi);
    return __cosf(fmaf(-k, kTwoPi, a));
}
SFP_DEVICE_INLINE float sin_r(float a) {
    const float k = rintf(a * kInvTwoPi);
    return __sinf(fmaf(-k, kTwoPi, a));
}

// uniforms of 24 bits (r1) and 32-bit resolution near 0 (r2), in (0, 1).
// They are taken from the same Philox words as the float64 draws
// (sfp::uniform2: r1 <- word 0, r2 <- word 2), so both forms see the same
// random numbers to float32 precision and make the same event decisions
// except within float32 rounding of the acceptance threshold.
SFP_DEVICE_INLINE void uniform2f_of(sfp::U4 o, float& r1, float& r2) {
    r1 = ((float)(o.x >> 8) + 0.5f) * 0x1p-24f;
    r2 = __uint2float_rn(o.z) * 0x1p-32f + 0x1p-33f;
}
SFP_DEVICE_INLINE void uniform2f(unsigned long long seed, unsigned int stream, unsigned int step,
                                 unsigned int purpose, long long slot, float& r1, float& r2) {
    uniform2f_of(sfp::philox4x32_10(sfp::philox_counter(stream, step, purpose, slot), (unsigned int)seed,
                                    (unsigned int)(seed >> 32)),
                 r1, r2);
}

// atan of a float32, branch-free: t = min(|a|, 1/|a|), atan(t) = t P(t^2)
// with P of degree 8 fitted here by weighted least squares to atan(t)/t on
// [0, 1] (max error 1.9 ulp in float32 there), and
// atan(|a|) = pi/2 - atan(1/|a|) for |a| > 1; the sign of a is restored
SFP_DEVICE_INLINE float atan_r(float a) {
    const float ax = fabsf(a);
    const bool big = ax > 1.0f;
    const float t = big ? __frcp_rn(ax) : ax;
    const float u = t * t;
    float p = 0.002849900396540761f;
    p = fmaf(p, u, -0.016068672761321068f);
    p = fmaf(p, u, 0.04269159212708473f);
    p = fmaf(p, u, -0.07504300773143768f);
    p = fmaf(p, u, 0.10640937089920044f);
    p = fmaf(p, u, -0.14203645288944244f);
    p = fmaf(p, u, 0.1999261975288391f);
    p = fmaf(p, u, -0.3333307206630707f);
    p = fmaf(p, u, 1.0f);
    float r = t * p;
    if (big) r = 1.57079632679489662f - r;
    return copysignf(r, a);
}

// ---- field presets (same parameter blocks as the float64 forms) ----------
// gaussian_laser_pulse (fields.py:152-168); the curvature term k0 r^2 / (2 Rx)
// is written as k0 r^2 x / (2 (x^2 + zR^2)) = (k0 / (2 zR^2)) r^2 x / q with
// q = 1 + (x/zR)^2, finite at x = 0, and r^2 / w(x)^2 as (1/w0^2) r^2 / q.
// Slots 10-15 of the block hold float32 constants in pairs (fields.py,
// _pack_float32): E0, k0, 1/zR, k0/(2 zR^2), 1/w0^2, 1/kc^2, direction/c,
// cep, cos(pol), sin(pol), k0/(4 zR), kc = k0 ctau.  1/q is rsqrt(q)^2.
// |phi| / kc beyond which a Gaussian envelope exp(-(phi/kc)^2) is exactly 0
// in float32, denormals included: sqrt(110), with exp(-104) already below
// half the smallest denormal
constexpr float kFieldCut32 = 10.5f;

// The longitudinal focusing factors of a Gaussian term at a point:
// 1/sqrt(q), 1/q and the Gouy phase atan(x/zR), q = 1 + (x/zR)^2.  They
// depend on the point's x and on 1/zR only, so the terms of a sum with the
// same zR (the polarisations and directions of one beam geometry) share
// them: the first such term the warp evaluates (one not skipped by the
// far-field cut) forms them, the others reuse them (`have`), with bitwise
// the same results.
struct GaussXY {
    float inv_zR;  // the 1/zR they were formed with
    float rs, rq, gouy;
};

// one term, sharing G (see GaussXY); F receives the term's field
SFP_DEVICE_INLINE void field_gaussian_g(const double* __restrict__ P, double x, double y, double z, double t,
                                        GaussXY& G, bool& have, float F[6]) {
    // three 16-byte loads (a term's block starts 16-byte aligned: 16 doubles
    // per term, and the run requires an aligned parameter array)
    const float4 g0 = *reinterpret_cast<const float4*>(P + 10);
    const float4 g1 = *reinterpret_cast<const float4*>(P + 12);
    const float4 g2 = *reinterpret_cast<const float4*>(P + 14);
    const float E0 = g0.x, k0 = g0.y, inv_zR = g0.z, cq = g0.w, inv_w02 = g1.x, inv_kc2 = g1.y, dirc = g1.z;
    const float cep = g1.w, cp = g2.x, sp = g2.y, cut_r = g2.z, kc = g2.w;
    const double dir = P[5], x0 = P[6];
    const float xf = d2f(x), yf = d2f(y), zf = d2f(z);
    const float xr = d2f((x - x0) - (dir * sfp::kC) * t);
    const float r2 = yf * yf + zf * zf;
    // |phi| >= k0 |xr| - k0 r2 / (4 zR) - pi/2 (as in the float64 form):
    // beyond kFieldCut32 kc the envelope is exactly 0, and so is the field.
    // The work is skipped when every active lane is past the cut; a lane
    // past it among others computes and takes exact zeros (no divergence)
    const bool cut = k0 * fabsf(xr) - cut_r * r2 - 1.5708f > kFieldCut32 * kc;
    if (__all_sync(__activemask(), cut)) {
        for (int k = 0; k < 6; ++k) F[k] = 0.0f;
        return;
    }
    if (!have || G.inv_zR != inv_zR) {
        const float xz = xf * inv_zR;
        const float q = fmaf(xz, xz, 1.0f);
        G.inv_zR = inv_zR;
        G.rs = rsqrtf(q);
        G.rq = G.rs * G.rs;
        G.gouy = atan_r(xz);
        have = true;
    }
    const float curv = (cq * r2) * (xf * G.rq);  // (k0 / (2 zR^2)) r^2 x / q
    const float tenv = (r2 * inv_w02) * G.rq;    // r^2 / w(x)^2
    const float phi = fmaf(k0, xr, curv) - G.gouy;
    const float env = __expf(-fmaf(phi * phi, inv_kc2, tenv));
    const float E = E0 * cos_r(phi + cep) * G.rs * env;
    const float Ey = E * cp, Ez = E * sp;
    F[0] = 0.0f;
    F[1] = cut ? 0.0f : Ey;
    F[2] = cut ? 0.0f : Ez;
    F[3] = 0.0f;
    F[4] = cut ? 0.0f : -Ez * dirc;
    F[5] = cut ? 0.0f : Ey * dirc;
}

SFP_DEVICE_INLINE void field_gaussian(const double* __restrict__ P, double x, double y, double z, double t,
                                      float F[6]) {
    GaussXY G;
    bool have = false;
    field_gaussian_g(P, x, y, z, t, G, have, F);
}

// simple_laser_pulse (fields.py:102-116)
SFP_DEVICE_INLINE void field_simple(const double* __restrict__ P, double x, double y, double z, double t, float F[6]) {
    const float E0 = d2f(P[0]), k0 = d2f(P[1]), w0 = d2f(P[2]), ctau = d2f(P[3]);
    const double dir = P[4], x0 = P[5];
    const float cep = d2f(P[6]), cp = d2f(P[7]), sp = d2f(P[8]);
    const int tord = (int)P[9];
    const float yf = d2f(y), zf = d2f(z);
    const float phi = k0 * d2f((dir * x - dir * x0) - sfp::kC * t);
    const float r2 = yf * yf + zf * zf;
    float num, den;
    const float kc = k0 * ctau;
    // far outside the pulse the envelope is exactly 0 in float32 (see kFieldCut32)
    if (P[10] != 0.0 && tord == 2 && fabsf(phi) > kFieldCut32 * kc) {
        for (int k = 0; k < 6; ++k) F[k] = 0.0f;
        return;
    }
    if (P[10] != 0.0 && tord == 2) {
        num = phi * phi;
        den = kc * kc;
    } else {
        num = powf(phi, d2f(P[9]));
        den = powf(kc, d2f(P[9]));
    }
    const float E = E0 * cos_r(phi + cep) * __expf(-(r2 / (w0 * w0)) - num / den);
    const float Ey = E * cp, Ez = E * sp;
    const float d = d2f(dir);
    F[0] = 0.0f;
    F[1] = Ey;
    F[2] = Ez;
    F[3] = 0.0f;
    F[4] = -Ez * (d / kCf);
    F[5] = Ey * (d / kCf);
}

SFP_DEVICE_INLINE void field_static(const double* __restrict__ P, float F[6]) {
#pragma unroll
    for (int i = 0; i < 6; ++i) F[i] = d2f(P[i]);
}

// focused_gaussian_laser_pulse: evaluated in float64 (its eps^5 expansion
// cancels), returned as float32
SFP_DEVICE_INLINE void field_focused(const double* __restrict__ P, double x, double y, double z, double t, float F[6]) {
    double D[6];
    sfp::field_focused(P, x, y, z, t, D);
#pragma unroll
    for (int i = 0; i < 6; ++i) F[i] = d2f(D[i]);
}

// ---- chi (inline.py:126-134) in Schwinger units ----------------------------
SFP_DEVICE_INLINE float chi_of(const float F[6], float ux, float uy, float uz, float gamma) {
    const float Ex = F[0] * kInvEs, Ey = F[1] * kInvEs, Ez = F[2] * kInvEs;
    const float Bx = F[3] * kCOverEs, By = F[4] * kCOverEs, Bz = F[5] * kCOverEs;
    const float a = gamma * Ex + (uy * Bz - uz * By);
    const float b = gamma * Ey + (uz * Bx - ux * Bz);
    const float c = gamma * Ez + (ux * By - uy * Bx);
    const float s = ux * Ex + uy * Ey + uz * Ez;
    const float rad = a * a + b * b + c * c - s * s;
    return rad > 0.0f ? sqrtf(rad) : 0.0f;
}

// gamma of u (float64 state), float64 above the split
SFP_DEVICE_INLINE float gamma_of(double ux, double uy, double uz, bool massless) {
    const float fx = d2f(ux), fy = d2f(uy), fz = d2f(uz);
    const float u2 = fx * fx + fy * fy + fz * fz;
    if (massless) return sqrtf(u2);
    if (u2 < (float)(kGammaSplit * kGammaSplit)) return sqrtf(1.0f + u2);
    return d2f(sqrt(((1.0 + ux * ux) + uy * uy) + uz * uz));
}

// ---- rejection sampling (qed/rejection_sampling*.py) -----------------------
SFP_DEVICE_INLINE float ai_lerp(const float* __restrict__ tab, float z, float inv_dz, int zN) {
    const float fi = z * inv_dz;
    int i = (int)fi;
    if (i > zN - 2) i = zN - 2;
    const float w = fi - (float)i;
    return fmaf(w, tab[i + 1] - tab[i], tab[i]);
}

// dW/ddelta up to the common factor alpha m c^2 / hbar; sign s = +1 photon
// emission (2/z + chi_g sqrt z), -1 pair creation (2/z - chi_g sqrt z)
SFP_DEVICE_INLINE float rate_core(float chi_g, float base, const float* __restrict__ iAt, const float* __restrict__ dAt,
                                  float inv_dz, int zN, float base_max, float sgn) {
    // z = base^(2/3) > z_max  <=>  base > z_max^(3/2) = base_max
    if (!(base <= base_max)) return 0.0f;
    const float z = exp2f(0.66666667f * __log2f(base));
    const float iA = ai_lerp(iAt, z, inv_dz, zN);
    const float dA = ai_lerp(dAt, z, inv_dz, zN);
    return iA + (__fdividef(2.0f, z) + sgn * chi_g * sqrtf(z)) * dA;
}

// _linear_interp1d (qed/optical_depth_tables.py:56-66) in float32: the float32
// form's total-rate lookup (rate: the table staged as float32).  The optical
// depth it is subtracted from stays float64.
SFP_DEVICE_INLINE float od_rate(float chi, const sfp_od_table& t, const float* __restrict__ rate) {
    const float lmin = d2f(t.log_chi_min), ldel = d2f(t.log_chi_delta), lmax = d2f(t.log_chi_max);
    float lc = __log10f(chi);  // the fast log10: within 2^-21.4 absolute near 1, 3 ulp elsewhere
    if (lc < lmin) return 0.0f;
    if (lc > lmax) lc = lmax;
    int idx = (int)floorf((lc - lmin) / ldel);
    if (idx > t.chi_N - 2) idx = t.chi_N - 2;
    if (idx < 0) idx = 0;
    const float left = lmin + (float)idx * ldel;
    return rate[idx] + (rate[idx + 1] - rate[idx]) * ((lc - left) / ldel);
}

}  // namespace sfp32
