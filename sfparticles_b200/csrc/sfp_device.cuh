// sfp_device.cuh -- per-particle device math of the sfparticles step.
//
// Compiled twice: by nvcc into libsfp.so (the per-op kernels that replace the
// reference's 12 Numba kernels one for one) and by NVRTC into the
// field-specialised fused step modules.  Nothing here allocates or launches.
//
// Each routine restates a reference routine (cited) in float64 with the same
// operation order; nvcc/NVRTC may contract a*b+c into one FMA, which moves
// results by <= 1 ulp per operation relative to the reference.
#pragma once
#include "sfp_types.h"

#ifndef SFP_DEVICE_INLINE
#define SFP_DEVICE_INLINE __device__ __forceinline__
#endif

namespace sfp {

// scipy.constants (CODATA 2022), the values the reference binds at import
// (particles.py:5, inline.py:1, qed table modules).
constexpr double kC = 299792458.0;
constexpr double kMe = 0x1.279dcc922bcd9p-100;  // 9.1093837139e-31 kg
constexpr double kE = 0x1.7a4da290c1653p-63;    // 1.602176634e-19 C
constexpr double kHbar = 0x1.185a7057c690dp-113; // 1.0545718176461565e-34 J s
constexpr double kEps0 = 0x1.37876f1591150p-37;  // 8.8541878188e-12 F/m
constexpr double kPi = 0x1.921fb54442d18p+1;
constexpr double kAlpha = 0x1.de3d429c6dc9dp-8;  // 0.0072973525643

// x**n for an integer literal n, unrolled as Numba lowers it
// (numba/cpython/numbers.py static_power_impl): res*=val on set bits,
// val*=val every round.
template <int N>
SFP_DEVICE_INLINE double ipow(double val) {
    double res = 1.0;
    int e = N;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (e == 0) break;
        if (e & 1) res = res * val;
        e >>= 1;
        val = val * val;
    }
    return res;
}
// Python's float modulo (result takes the sign of the divisor)
SFP_DEVICE_INLINE double py_mod(double a, double b) {
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}
SFP_DEVICE_INLINE double ipow_rt(double val, int n) {
    double res = 1.0;
    int e = n < 0 ? -n : n;
    while (e != 0) {
        if (e & 1) res = res * val;
        e >>= 1;
        val = val * val;
    }
    return n < 0 ? 1.0 / res : res;
}

// ---------------------------------------------------------------------------
// Counter-based RNG: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
// counter = (slot lo, slot hi | purpose<<24, step, stream), key = seed.
// ---------------------------------------------------------------------------
struct U4 {
    unsigned int x, y, z, w;
};

SFP_DEVICE_INLINE U4 philox4x32_10(U4 c, unsigned int k0, unsigned int k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned int lo0 = 0xD2511F53u * c.x;
        const unsigned int hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned int lo1 = 0xCD9E8D57u * c.z;
        const unsigned int hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// 52 random bits -> (k + 0.5) * 2^-52: exact, strictly inside (0, 1)
SFP_DEVICE_INLINE double u01(unsigned int a, unsigned int b) {
    unsigned long long k = ((unsigned long long)a << 20) ^ (unsigned long long)(b >> 12);
    k &= (1ull << 52) - 1ull;
    return ((double)k + 0.5) * 0x1p-52;
}

// the counter of a particle's draw: (slot lo, slot hi | purpose << 24, step, species stream)
SFP_DEVICE_INLINE U4 philox_counter(unsigned int stream, unsigned int step, unsigned int purpose, long long slot) {
    const unsigned long long s = (unsigned long long)slot;
    return U4{(unsigned int)s, ((unsigned int)(s >> 32) & 0x00FFFFFFu) | (purpose << 24), step, stream};
}

SFP_DEVICE_INLINE void uniform2(unsigned long long seed, unsigned int stream, unsigned int step,
                                unsigned int purpose, long long slot, double& r1, double& r2) {
    U4 o = philox4x32_10(philox_counter(stream, step, purpose, slot), (unsigned int)seed, (unsigned int)(seed >> 32));
    r1 = u01(o.x, o.y);
    r2 = u01(o.z, o.w);
}

// ---------------------------------------------------------------------------
// Field presets (fields.py).  P points at SFP_FIELD_PARAMS doubles whose
// layout is written by sfparticles_b200/fields.py.
// ---------------------------------------------------------------------------

// static_field, fields.py:268-271.  P = Ex,Ey,Ez,Bx,By,Bz
SFP_DEVICE_INLINE void field_static(const double* __restrict__ P, double F[6]) {
#pragma unroll
    for (int i = 0; i < 6; ++i) F[i] = P[i];
}

// |phi| / kc beyond which a Gaussian envelope exp(-(phi/kc)^2) is exactly 0
// in float64: sqrt(800), with exp(-745.2) already below half the smallest
// denormal
constexpr double kFieldCut64 = 28.2843;

// simple_laser_pulse, fields.py:102-116.
// P = E0, k0, w0, ctau, direction, x0, cep, cos(pol), sin(pol), t_order, t_order_is_int
SFP_DEVICE_INLINE void field_simple(const double* __restrict__ P, double x, double y, double z, double t,
                                    double F[6]) {
    const double E0 = P[0], k0 = P[1], w0 = P[2], ctau = P[3], dir = P[4], x0 = P[5];
    const double cep = P[6], cp = P[7], sp = P[8], tord = P[9];
    x = dir * x;
    const double r2 = y * y + z * z;
    const double phi = k0 * ((x - dir * x0) - kC * t);
    // far outside the pulse the envelope exp(-(phi/kc)^2) is exactly 0 in
    // float64 ((phi/kc)^2 > 745.2); past (phi/kc)^2 = 800 the field is 0
    // without evaluating cos and exp (the formula gives +-0 there)
    if (P[10] != 0.0 && tord == 2.0 && fabs(phi) > kFieldCut64 * (k0 * ctau)) {
        for (int k = 0; k < 6; ++k) F[k] = 0.0;
        return;
    }
    double num, den;
    if (P[10] != 0.0) {
        if (tord == 2.0) {
            num = ipow<2>(phi);
            den = ipow<2>(k0 * ctau);
        } else {
            num = ipow_rt(phi, (int)tord);
            den = ipow_rt(k0 * ctau, (int)tord);
        }
    } else {
        num = pow(phi, tord);
        den = pow(k0 * ctau, tord);
    }
    const double E = ((E0 * cos(phi + cep)) * exp((-r2) / (w0 * w0))) * exp((-num) / den);
    const double Ey = E * cp, Ez = E * sp;
    F[0] = 0.0;
    F[1] = Ey;
    F[2] = Ez;
    F[3] = 0.0;
    F[4] = ((-Ez) / kC) * dir;
    F[5] = (Ey / kC) * dir;
}

// gaussian_laser_pulse, fields.py:152-168.
// P = E0, k0, zR, w0, ctau, direction, x0, cep, cos(pol), sin(pol)
SFP_DEVICE_INLINE void field_gaussian(const double* __restrict__ P, double x, double y, double z, double t,
                                      double F[6]) {
    const double E0 = P[0], k0 = P[1], zR = P[2], w0 = P[3], ctau = P[4], dir = P[5], x0 = P[6];
    const double cep = P[7], cp = P[8], sp = P[9];
    const double r2 = y * y + z * z;
    // Far outside the pulse the envelope exp(-(phi/kc)^2) is exactly 0 in
    // float64 ((phi/kc)^2 > 745.2).  |phi| >= |k0 xr| - k0 r2 / (4 zR) - pi/2,
    // because |x| / (x^2 + zR^2) <= 1 / (2 zR) and |atan| < pi/2; once that
    // bound exceeds sqrt(800) kc the field is 0 without evaluating atan, cos
    // and the divisions (the formula gives +-0 there).  Multiplied by 4 zR > 0.
    if (4.0 * zR * fabs(k0 * ((x - x0) - (dir * kC) * t)) - k0 * r2 - 6.2832 * zR >
        4.0 * zR * kFieldCut64 * (k0 * ctau)) {
        for (int k = 0; k < 6; ++k) F[k] = 0.0;
        return;
    }
    const double xz = x / zR;
    const double wx = w0 * sqrt(1.0 + xz * xz);
    const double zx = zR / x;
    const double Rx = x * (1.0 + zx * zx);
    const double gouy = atan(x / zR);
    const double phi = ((k0 * ((x - x0) - (dir * kC) * t)) + (((k0 * r2) / 2.0) / Rx)) - gouy;
    const double kc = k0 * ctau;
    const double E = ((((E0 * cos(phi + cep)) * w0) / wx) * exp((-r2) / (wx * wx))) * exp((-(phi * phi)) / (kc * kc));
    const double Ey = E * cp, Ez = E * sp;
    F[0] = 0.0;
    F[1] = Ey;
    F[2] = Ez;
    F[3] = 0.0;
    F[4] = ((-Ez) / kC) * dir;
    F[5] = (Ey / kC) * dir;
}

// focused_gaussian_laser_pulse, fields.py:211-263 (Salamin-type expansion
// to eps^5).  P = E0, k0, zR, w0, ctau, direction, xfoc, x0, cep, cos(pol), sin(pol), eps
SFP_DEVICE_INLINE void field_focused(const double* __restrict__ P, double x, double y, double z, double t,
                                     double F[6]) {
    const double E0 = P[0], k0 = P[1], zR = P[2], w0 = P[3], ctau = P[4], dir = P[5];
    const double xfoc = P[6], x0 = P[7], cep = P[8], cp = P[9], sp = P[10], ep = P[11];
    x = dir * (x - xfoc);
    const double r2 = y * y + z * z;
    const double xz = x / zR;
    const double wx = w0 * sqrt(1.0 + xz * xz);
    const double psiG = atan(x / zR);
    const double psiR = (((k0 * x) * r2) / 2.0) / ((x * x) + (zR * zR));
    const double psiP = k0 * ((x - dir * x0) - kC * t);
    const double psi = ((psiG + psiR) + psiP) + cep;
    const double rho = sqrt(r2) / w0;
    const double xi = y / w0;
    const double nu = z / w0;
    const double eta = 1.0 / sqrt(1.0 + xz * xz);
    const double rho2 = ipow<2>(rho), rho4 = ipow<4>(rho), rho6 = ipow<6>(rho), rho8 = ipow<8>(rho);
    const double kc = k0 * ctau;
    const double pc = psi - cep;
    const double E = (((E0 * w0) / wx) * exp((-r2) / (wx * wx))) * exp((-(pc * pc)) / (kc * kc));
    const double S0 = sin(psi);
    const double S2 = ipow<2>(eta) * sin(psi + 2.0 * psiG);
    const double S3 = ipow<3>(eta) * sin(psi + 3.0 * psiG);
    const double S4 = ipow<4>(eta) * sin(psi + 4.0 * psiG);
    const double S5 = ipow<5>(eta) * sin(psi + 5.0 * psiG);
    const double S6 = ipow<6>(eta) * sin(psi + 6.0 * psiG);
    const double C1 = ipow<1>(eta) * cos(psi + 1.0 * psiG);
    const double C2 = ipow<2>(eta) * cos(psi + 2.0 * psiG);
    const double C3 = ipow<3>(eta) * cos(psi + 3.0 * psiG);
    const double C4 = ipow<4>(eta) * cos(psi + 4.0 * psiG);
    const double C5 = ipow<5>(eta) * cos(psi + 5.0 * psiG);
    const double C6 = ipow<6>(eta) * cos(psi + 6.0 * psiG);
    const double C7 = ipow<7>(eta) * cos(psi + 7.0 * psiG);
    const double e2 = ipow<2>(ep), e3 = ipow<3>(ep), e4 = ipow<4>(ep), e5 = ipow<5>(ep);
    const double xi2 = ipow<2>(xi);
    const double exA = (((-C2) / 2.0) + rho2 * C3) - (rho4 * C4) / 4.0;
    const double exB =
        ((((-0.375 * C3) - (0.375 * rho2) * C4) + (1.0625 * rho4) * C5) - (0.375 * rho6) * C6) + (rho8 * C7) / 32.0;
    const double Ex_ = (E * xi) * (((ep * C1) + e3 * exA) + e5 * exB);
    const double eyA = (xi2 * S2) - (rho4 * S3) / 4.0;
    const double eyB = ((((S2 / 8.0) - (rho2 * S3) / 4.0) - ((rho2 * (rho2 - 16.0 * xi2)) * S4) / 16.0) -
                        ((rho4 * (rho2 + 2.0 * xi2)) * S5) / 8.0) +
                       (rho8 * S6) / 32.0;
    const double Ey_ = E * ((S0 + e2 * eyA) + e4 * eyB);
    const double Ez_ = ((E * xi) * nu) * ((e2 * S2) + e4 * ((rho2 * S4) - (rho4 * S5) / 4.0));
    const double bxA = ((C2 / 2.0) + (rho2 * C3) / 2.0) - (rho4 * C4) / 4.0;
    const double bxB =
        ((((0.375 * C3) + (0.375 * rho2) * C4) + (0.1875 * rho4) * C5) - (rho6 * C6) / 4.0) + (rho8 * C7) / 32.0;
    const double Bx_ = ((E / kC) * nu) * (((ep * C1) + e3 * bxA) + e5 * bxB);
    const double bzA = ((rho2 * S2) / 2.0) - (rho4 * S3) / 4.0;
    const double bzB =
        (((((-S2) / 8.0) + (rho2 * S3) / 4.0) + (0.3125 * rho4) * S4) - (rho6 * S5) / 4.0) + (rho8 * S6) / 32.0;
    const double Bz_ = (E / kC) * ((S0 + e2 * bzA) + e4 * bzB);
    const double By_ = 0.0;
    F[0] = Ex_;
    F[1] = Ey_ * cp - Ez_ * sp;
    F[2] = Ey_ * sp + Ez_ * cp;
    F[3] = Bx_;
    F[4] = (By_ * cp - Bz_ * sp) * dir;
    F[5] = (By_ * sp + Bz_ * cp) * dir;
}

// ---------------------------------------------------------------------------
// Pushers (inline.py, cpu.py)
// ---------------------------------------------------------------------------

// 1/gamma of a massive particle / 1/|u| of a photon, as the reference stores
// it (particles.py:119,122; cpu.py:86,114,187)
SFP_DEVICE_INLINE double inv_gamma_massive(double ux, double uy, double uz) {
    return 1.0 / sqrt(((1.0 + ux * ux) + uy * uy) + uz * uz);
}
SFP_DEVICE_INLINE double inv_gamma_photon(double ux, double uy, double uz) {
    return 1.0 / sqrt((ux * ux + uy * uy) + uz * uz);
}

// cpu.py:5-19, one particle
SFP_DEVICE_INLINE void push_position(double& x, double& y, double& z, double ux, double uy, double uz, double ig,
                                     double dt) {
    const double cdt = kC * dt;
    x += (cdt * ig) * ux;
    y += (cdt * ig) * uy;
    z += (cdt * ig) * uz;
}

// inline.py:4-36.  Returns the new 1/gamma.
SFP_DEVICE_INLINE double boris(double& ux, double& uy, double& uz, const double F[6], double q, double dt) {
    const double efactor = (q * dt) / ((2.0 * kMe) * kC);
    const double bfactor = (q * dt) / (2.0 * kMe);
    const double uxm = ux + efactor * F[0];
    const double uym = uy + efactor * F[1];
    const double uzm = uz + efactor * F[2];
    const double igm = 1.0 / sqrt(((1.0 + uxm * uxm) + uym * uym) + uzm * uzm);
    const double Tx = (bfactor * F[3]) * igm;
    const double Ty = (bfactor * F[4]) * igm;
    const double Tz = (bfactor * F[5]) * igm;
    const double uxp = (uxm + uym * Tz) - uzm * Ty;
    const double uyp = (uym + uzm * Tx) - uxm * Tz;
    const double uzp = (uzm + uxm * Ty) - uym * Tx;
    const double Tf = 2.0 / (((1.0 + Tx * Tx) + Ty * Ty) + Tz * Tz);
    const double Sx = Tf * Tx, Sy = Tf * Ty, Sz = Tf * Tz;
    const double uxl = (uxm + uyp * Sz) - uzp * Sy;
    const double uyl = (uym + uzp * Sx) - uxp * Sz;
    const double uzl = (uzm + uxp * Sy) - uyp * Sx;
    ux = uxl + efactor * F[0];
    uy = uyl + efactor * F[1];
    uz = uzl + efactor * F[2];
    return inv_gamma_massive(ux, uy, uz);
}

// inline.py:39-100: spin rotated with B_eff built from u-, then the momentum.
SFP_DEVICE_INLINE double boris_tbmt(double& ux, double& uy, double& uz, double& sx, double& sy, double& sz,
                                    const double F[6], double q, double ae, double dt) {
    const double Ex = F[0], Ey = F[1], Ez = F[2], Bx = F[3], By = F[4], Bz = F[5];
    const double efactor = (q * dt) / ((2.0 * kMe) * kC);
    const double bfactor = (q * dt) / (2.0 * kMe);
    const double uxm = ux + efactor * Ex;
    const double uym = uy + efactor * Ey;
    const double uzm = uz + efactor * Ez;
    const double uB = (uxm * Bx + uym * By) + uzm * Bz;
    const double gm = sqrt(((1.0 + uxm * uxm) + uym * uym) + uzm * uzm);
    const double igm = 1.0 / gm;
    const double a1 = ae + igm;
    const double a2 = (ae * gm) / (gm + 1.0);
    const double a3 = ae + 1.0 / (gm + 1.0);
    const double Bxe = (a1 * Bx - (a2 * uB) * uxm) - a3 * (uym * Ez - uzm * Ey);
    const double Bye = (a1 * By - (a2 * uB) * uym) - a3 * (uzm * Ex - uxm * Ez);
    const double Bze = (a1 * Bz - (a2 * uB) * uzm) - a3 * (uxm * Ey - uym * Ex);
    double Tx = bfactor * Bxe, Ty = bfactor * Bye, Tz = bfactor * Bze;
    const double T2 = (Tx * Tx + Ty * Ty) + Tz * Tz;
    double Sx = (2.0 * Tx) / (1.0 + T2);
    double Sy = (2.0 * Ty) / (1.0 + T2);
    double Sz = (2.0 * Tz) / (1.0 + T2);
    const double s0x = sx, s0y = sy, s0z = sz;
    const double sxp = (s0x + s0y * Tz) - s0z * Ty;
    const double syp = (s0y + s0z * Tx) - s0x * Tz;
    const double szp = (s0z + s0x * Ty) - s0y * Tx;
    sx = (s0x + syp * Sz) - szp * Sy;
    sy = (s0y + szp * Sx) - sxp * Sz;
    sz = (s0z + sxp * Sy) - syp * Sx;
    Tx = (bfactor * Bx) * igm;
    Ty = (bfactor * By) * igm;
    Tz = (bfactor * Bz) * igm;
    const double uxp = (uxm + uym * Tz) - uzm * Ty;
    const double uyp = (uym + uzm * Tx) - uxm * Tz;
    const double uzp = (uzm + uxm * Ty) - uym * Tx;
    const double Tf = 2.0 / (((1.0 + Tx * Tx) + Ty * Ty) + Tz * Tz);
    Sx = Tf * Tx;
    Sy = Tf * Ty;
    Sz = Tf * Tz;
    const double uxl = (uxm + uyp * Sz) - uzp * Sy;
    const double uyl = (uym + uzp * Sx) - uxp * Sz;
    const double uzl = (uzm + uxp * Sy) - uyp * Sx;
    ux = uxl + efactor * Ex;
    uy = uyl + efactor * Ey;
    uz = uzl + efactor * Ez;
    return inv_gamma_massive(ux, uy, uz);
}

// LL prefactor, inline.py:105: -2/3 / (4 pi eps0) * e**2 * m_e * c / hbar**2 * dt
SFP_DEVICE_INLINE double ll_factor(double dt) {
    return ((((((-2.0 / 3.0) / ((4.0 * kPi) * kEps0)) * (kE * kE)) * kMe) * kC) / (kHbar * kHbar)) * dt;
}

// inline.py:104-123 (quantum = CLL g(chi) correction).  Returns new 1/gamma.
SFP_DEVICE_INLINE double ll_push(double& ux, double& uy, double& uz, double ig, double chi, double dt, bool quantum) {
    double factor = ll_factor(dt);
    if (quantum) {
        const double g = pow((1.0 + (4.8 * (1.0 + chi)) * log(1.0 + 1.7 * chi)) + 2.44 * (chi * chi), -2.0 / 3.0);
        factor = factor * g;
    }
    const double c2 = chi * chi;
    ux = ux + ((factor * c2) * ux) * ig;
    uy = uy + ((factor * c2) * uy) * ig;
    uz = uz + ((factor * c2) * uz) * ig;
    return inv_gamma_massive(ux, uy, uz);
}

// inline.py:126-134.  A non-positive radicand (rounding) gives chi = 0.
SFP_DEVICE_INLINE double chi_of(const double F[6], double ux, double uy, double uz, double ig) {
    const double factor = (kE * kHbar) / ((kMe * kMe) * (kC * (kC * kC)));
    const double gamma = 1.0 / ig;
    const double a = gamma * F[0] + (uy * F[5] - uz * F[4]) * kC;
    const double b = gamma * F[1] + (uz * F[3] - ux * F[5]) * kC;
    const double c = gamma * F[2] + (ux * F[4] - uy * F[3]) * kC;
    const double s = (ux * F[0] + uy * F[1]) + uz * F[2];
    double rad = ((a * a + b * b) + c * c) - s * s;
    if (!(rad > 0.0)) rad = 0.0;
    return factor * sqrt(rad);
}

// ---------------------------------------------------------------------------
// Rejection sampling (qed/rejection_sampling*.py).  T points at
// [int_Ai[z_N] | Aip[z_N]] (shared memory in the fused kernel).
// ---------------------------------------------------------------------------
SFP_DEVICE_INLINE void ai_interp(double z, const double* __restrict__ iAt, const double* __restrict__ dAt, int zN,
                                 double zmax, double& iA, double& dA) {
    const double dz = (zmax - 0.0) / (double)(zN - 1);
    long long idx = (long long)((z - 0.0) / dz);
    if (idx > zN - 2) idx = zN - 2;
    const double zl = 0.0 + (double)idx * dz;
    double k = (iAt[idx + 1] - iAt[idx]) / dz;
    iA = iAt[idx] + k * (z - zl);
    k = (dAt[idx + 1] - dAt[idx]) / dz;
    dA = dAt[idx] + k * (z - zl);
}

// qed/rejection_sampling_tables.py:32-53; z beyond the table -> 0
SFP_DEVICE_INLINE double photon_rate(double chi_e, double delta, const double* iAt, const double* dAt, int zN,
                                     double zmax) {
    const double chi_gamma = delta * chi_e;
    const double chi_ep = chi_e - chi_gamma;
    const double z = pow((chi_gamma / chi_e) / chi_ep, 2.0 / 3.0);
    const double factor = (((-kAlpha) * kMe) * (kC * kC)) / kHbar;
    if (!(z <= zmax)) return 0.0;
    double iA, dA;
    ai_interp(z, iAt, dAt, zN, zmax, iA, dA);
    return factor * (iA + (2.0 / z + chi_gamma * sqrt(z)) * dA);
}

// qed/rejection_sampling_tables.py:56-78
SFP_DEVICE_INLINE double pair_rate(double chi_gamma, double delta, const double* iAt, const double* dAt, int zN,
                                   double zmax) {
    const double chi_e = delta * chi_gamma;
    const double chi_ep = chi_gamma - chi_e;
    const double z = pow((chi_gamma / chi_e) / chi_ep, 2.0 / 3.0);
    const double factor = ((kAlpha * kMe) * (kC * kC)) / kHbar;
    if (!(z <= zmax)) return 0.0;
    double iA, dA;
    ai_interp(z, iAt, dAt, zN, zmax, iA, dA);
    return factor * (iA + (2.0 / z - chi_gamma * sqrt(z)) * dA);
}

// qed/rejection_sampling.py:73-89 with draws (r1, r2): returns event, sets delta
SFP_DEVICE_INLINE bool photon_event_rs(double chi, double ig, double dt, double r1, double r2, const double* iAt,
                                       const double* dAt, int zN, double zmax, double& delta) {
    const double dtau = dt * ig;
    const double d = r1 * (r1 * r1);
    const double prob = ((3.0 * (r1 * r1)) * photon_rate(chi, d, iAt, dAt, zN, zmax)) * dtau;
    if (r2 < prob) {
        delta = d;
        return true;
    }
    delta = 0.0;
    return false;
}

// qed/rejection_sampling.py:92-107
SFP_DEVICE_INLINE bool pair_event_rs(double chi, double ig, double dt, double r1, double r2, const double* iAt,
                                     const double* dAt, int zN, double zmax, double& delta) {
    const double dtau = dt * ig;
    const double prob = pair_rate(chi, r1, iAt, dAt, zN, zmax) * dtau;
    if (r2 < prob) {
        delta = r1;
        return true;
    }
    delta = 0.0;
    return false;
}

// ---------------------------------------------------------------------------
// Optical depth (qed/optical_depth*.py)
// ---------------------------------------------------------------------------
SFP_DEVICE_INLINE double od_row(double log_chi, const sfp_od_table& t) {
    if (log_chi > t.log_chi_max) log_chi = t.log_chi_max;
    double idx = (log_chi - t.log_chi_min) / t.log_chi_delta;
    if (idx > (double)(t.chi_N - 1)) idx = (double)(t.chi_N - 1);
    return idx;
}

// _linear_interp1d, qed/optical_depth_tables.py:56-66 (rate may be in smem)
SFP_DEVICE_INLINE double od_interp1d(double chi, const sfp_od_table& t, const double* __restrict__ rate) {
    double log_chi = log10(chi);
    if (log_chi < t.log_chi_min) return 0.0;
    long long idx = (long long)floor(od_row(log_chi, t));
    if (idx > t.chi_N - 2) idx = t.chi_N - 2;
    if (log_chi > t.log_chi_max) log_chi = t.log_chi_max;
    const double left = t.log_chi_min + (double)idx * t.log_chi_delta;
    const double k = (rate[idx + 1] - rate[idx]) / t.log_chi_delta;
    return rate[idx] + k * (log_chi - left);
}

// _bisect_interp, qed/optical_depth_tables.py:69-112 (rows blended linearly in
// chi, bisection over delta columns, inverse linear interpolation); equality
// with r moves `high` down (the reference has no branch for it).
SFP_DEVICE_INLINE double od_bisect(double chi, double r_uniform, const sfp_od_table& t) {
    const int n = t.delta_N;
    const double log_chi = log10(chi);
    long long lo_i = (long long)floor(od_row(log_chi, t));
    if (lo_i > t.chi_N - 2) lo_i = t.chi_N - 2;
    if (lo_i < 0) lo_i = 0;
    const long long hi_i = lo_i + 1;
    const double chi_top = pow(10.0, t.log_chi_max);
    if (chi > chi_top) chi = chi_top;
    const double chi_low = pow(10.0, t.log_chi_min + (double)lo_i * t.log_chi_delta);
    const double chi_high = pow(10.0, t.log_chi_min + (double)hi_i * t.log_chi_delta);
    const double* __restrict__ TL = t.cumulative + (size_t)lo_i * n;
    const double* __restrict__ TH = t.cumulative + (size_t)hi_i * n;
    const double w = chi - chi_low;
    const double span = chi_high - chi_low;
#define SFP_ROWVAL(j) (__ldg(TL + (j)) + ((__ldg(TH + (j)) - __ldg(TL + (j))) / span) * w)
    const double ymin = SFP_ROWVAL(0);
    const double ymax = SFP_ROWVAL(n - 1);
    const double r = r_uniform * (ymax - ymin) + ymin;
    int low = 0, high = n - 1;
    while (low <= high) {
        const int mid = (low + high) / 2;
        const double md = SFP_ROWVAL(mid);
        if (md < r)
            low = mid + 1;
        else
            high = mid - 1;
    }
    int di = high;
    if (di < 0) di = 0;
    if (di > n - 2) di = n - 2;
    const double y1 = SFP_ROWVAL(di);
    const double y2 = SFP_ROWVAL(di + 1);
#undef SFP_ROWVAL
    const double dl = pow(10.0, t.log_delta_min + (double)di * t.log_delta_delta);
    const double dr = pow(10.0, t.log_delta_min + (double)(di + 1) * t.log_delta_delta);
    const double k = (dr - dl) / (y2 - y1);
    return dl + k * (r - y1);
}

// update_tau_e / update_tau_gamma body for one particle (optical_depth.py:42-62)
// up to the energy draw: true on an event, with `u` the uniform that the
// inverse CDF maps to delta.  chi_min = 10^log_chi_min, computed once by the
// caller (the reference's module constant _chi_min, optical_depth.py:14).
// od_tau_step is the part after the total-rate lookup (optical_depth.py:47-62).
// Draws, taken only when needed as in the reference (counter-based, so
// identical to drawing always): purpose 1 -> (tau reset, tau after event),
// purpose 2 -> inverse-CDF u.
SFP_DEVICE_INLINE bool od_tau_step(double rtot, double ig, double dt, double& tau, unsigned long long seed,
                                   unsigned int stream, unsigned int step, long long slot, double& u) {
    const double dtau = dt * ig;
    double ra = 0.0, rb = 0.0;
    bool drawn = false;
    if (tau == 0.0) {
        uniform2(seed, stream, step, 1u, slot, ra, rb);
        drawn = true;
        tau = -log(1.0 - ra);
    }
    tau -= rtot * dtau;
    if (tau < 0.0) {
        if (!drawn) uniform2(seed, stream, step, 1u, slot, ra, rb);
        double rc, rd;
        uniform2(seed, stream, step, 2u, slot, rc, rd);
        tau = -log(1.0 - rb);
        u = rc;
        return true;
    }
    u = 0.0;
    return false;
}

SFP_DEVICE_INLINE bool od_event_u(double chi, double ig, double dt, double& tau, const sfp_od_table& t,
                                  const double* rate, double chi_min, unsigned long long seed, unsigned int stream,
                                  unsigned int step, long long slot, double& u) {
    if (chi < chi_min) {
        u = 0.0;
        return false;
    }
    return od_tau_step(od_interp1d(chi, t, rate), ig, dt, tau, seed, stream, step, slot, u);
}

// the whole update with the table's inverse CDF for delta
SFP_DEVICE_INLINE bool od_event(double chi, double ig, double dt, double& tau, const sfp_od_table& t,
                                const double* rate, double chi_min, unsigned long long seed, unsigned int stream,
                                unsigned int step, long long slot, double& delta) {
    double u;
    const bool ev = od_event_u(chi, ig, dt, tau, t, rate, chi_min, seed, stream, step, slot, u);
    delta = ev ? od_bisect(chi, u, t) : 0.0;
    return ev;
}

}  // namespace sfp
