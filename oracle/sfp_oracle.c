/*
 * sfp_oracle.c -- CPU oracle for the sfparticles per-particle step.
 *
 * TEST INFRASTRUCTURE ONLY (see sfp_oracle.h).  Restates the reference's
 * Numba kernels in C with the same floating-point operation order.  Build
 * with -O2 -fopenmp -ffp-contract=off and without -ffast-math (oracle/Makefile),
 * so that no multiply-add is fused and no expression is reassociated, as in
 * Numba's default (non-fastmath) LLVM lowering.
 *
 * x**n with an integer literal n is restated as Numba lowers it
 * (numba/cpython/numbers.py static_power_impl: exponentiation by
 * squaring, res = res*val on set bits, val = val*val every round).
 */
#include "sfp_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* scipy.constants (CODATA 2022, scipy 1.18) -- same values the reference
 * binds at import in particles.py:5 and the qed table modules. */
static const double C_LIGHT = 299792458.0;
static const double M_E = 0x1.279dcc922bcd9p-100;   /* 9.1093837139e-31 */
static const double E_CHARGE = 0x1.7a4da290c1653p-63; /* 1.602176634e-19 */
static const double HBAR = 0x1.185a7057c690dp-113;  /* 1.0545718176461565e-34 */
static const double EPS0 = 0x1.37876f1591150p-37;   /* 8.8541878188e-12 */
static const double PI_ = 0x1.921fb54442d18p+1;
static const double ALPHA = 0x1.de3d429c6dc9dp-8;   /* 0.0072973525643 */

/* integer power as Numba's static_power_impl unrolls it */
static inline double ipow(double val, int n) {
    double res = 1.0;
    int e = n < 0 ? -n : n;
    while (e != 0) {
        if (e & 1) res = res * val;
        e >>= 1;
        val = val * val;
    }
    return n < 0 ? 1.0 / res : res;
}

/* ======================================================================== */
/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), restated from the   */
/* paper: two 32x32->64 multiplies per round, Weyl key schedule.           */
/* ======================================================================== */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 52 random bits -> (k + 0.5) * 2^-52, exactly representable, in (0,1) */
static inline double u01(uint32_t a, uint32_t b) {
    uint64_t k = ((uint64_t)a << 20) ^ (uint64_t)(b >> 12);
    k &= ((uint64_t)1 << 52) - 1;
    return ((double)k + 0.5) * 0x1p-52;
}

/* counter = (slot lo, slot hi | purpose<<24, step, stream); key = seed */
void orc_uniform2(uint64_t seed, uint32_t stream, uint32_t step, uint32_t purpose,
                  int64_t slot, double out[2]) {
    uint32_t ctr[4], key[2], r[4];
    uint64_t s = (uint64_t)slot;
    ctr[0] = (uint32_t)s;
    ctr[1] = ((uint32_t)(s >> 32) & 0x00FFFFFFu) | (purpose << 24);
    ctr[2] = step;
    ctr[3] = stream;
    key[0] = (uint32_t)seed;
    key[1] = (uint32_t)(seed >> 32);
    orc_philox4x32_10(ctr, key, r);
    out[0] = u01(r[0], r[1]);
    out[1] = u01(r[2], r[3]);
}

void orc_uniform2_batch(uint64_t seed, uint32_t stream, uint32_t step, uint32_t purpose,
                        const int64_t *slots, int64_t n, double *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) orc_uniform2(seed, stream, step, purpose, slots[i], out + 2 * i);
}

/* ======================================================================== */
/* Field presets (fields.py)                                                 */
/* ======================================================================== */

/* static_field, fields.py:268-271.  p = Ex,Ey,Ez,Bx,By,Bz */
static void field_static(const double *p, double F[6]) {
    for (int i = 0; i < 6; ++i) F[i] = p[i];
}

/* simple_laser_pulse._laser_pulse, fields.py:102-116.
 * p = E0, k0, w0, ctau, direction, x0, cep, cos(pol), sin(pol), t_order, t_order_is_int */
static void field_simple(const double *p, double x, double y, double z, double t, double F[6]) {
    const double E0 = p[0], k0 = p[1], w0 = p[2], ctau = p[3], dir = p[4], x0 = p[5];
    const double cep = p[6], cp = p[7], sp = p[8], tord = p[9];
    const int tord_int = p[10] != 0.0;
    x = dir * x;
    double r2 = y * y + z * z;
    double phi = k0 * ((x - dir * x0) - C_LIGHT * t);
    double num, den;
    if (tord_int) {
        num = ipow(phi, (int)tord);
        den = ipow(k0 * ctau, (int)tord);
    } else {
        num = pow(phi, tord);
        den = pow(k0 * ctau, tord);
    }
    double E = ((E0 * cos(phi + cep)) * exp((-r2) / (w0 * w0))) * exp((-num) / den);
    double Ey = E * cp, Ez = E * sp;
    F[0] = 0.0; F[1] = Ey; F[2] = Ez;
    F[3] = 0.0; F[4] = ((-Ez) / C_LIGHT) * dir; F[5] = (Ey / C_LIGHT) * dir;
}

/* gaussian_laser_pulse._gaussian_pulse, fields.py:152-168.
 * p = E0, k0, zR, w0, ctau, direction, x0, cep, cos(pol), sin(pol) */
static void field_gaussian(const double *p, double x, double y, double z, double t, double F[6]) {
    const double E0 = p[0], k0 = p[1], zR = p[2], w0 = p[3], ctau = p[4], dir = p[5], x0 = p[6];
    const double cep = p[7], cp = p[8], sp = p[9];
    double r2 = y * y + z * z;
    double xz = x / zR;
    double wx = w0 * sqrt(1.0 + xz * xz);
    double zx = zR / x;
    double Rx = x * (1.0 + zx * zx);
    double gouy = atan(x / zR);
    double phi = ((k0 * ((x - x0) - (dir * C_LIGHT) * t)) + (((k0 * r2) / 2.0) / Rx)) - gouy;
    double kc = k0 * ctau;
    double E = ((((E0 * cos(phi + cep)) * w0) / wx) * exp((-r2) / (wx * wx))) *
               exp((-(phi * phi)) / (kc * kc));
    double Ey = E * cp, Ez = E * sp;
    F[0] = 0.0; F[1] = Ey; F[2] = Ez;
    F[3] = 0.0; F[4] = ((-Ez) / C_LIGHT) * dir; F[5] = (Ey / C_LIGHT) * dir;
}

/* focused_gaussian_laser_pulse._gaussian_pulse, fields.py:211-263.
 * p = E0, k0, zR, w0, ctau, direction, xfoc, x0, cep, cos(pol), sin(pol), eps */
static void field_focused(const double *p, double x, double y, double z, double t, double F[6]) {
    const double E0 = p[0], k0 = p[1], zR = p[2], w0 = p[3], ctau = p[4], dir = p[5];
    const double xfoc = p[6], x0 = p[7], cep = p[8], cp = p[9], sp = p[10], ep = p[11];
    x = dir * (x - xfoc);
    double r2 = y * y + z * z;
    double xz = x / zR;
    double wx = w0 * sqrt(1.0 + xz * xz);
    double psiG = atan(x / zR);
    double psiR = (((k0 * x) * r2) / 2.0) / ((x * x) + (zR * zR));
    double psiP = k0 * ((x - dir * x0) - C_LIGHT * t);
    double psi = ((psiG + psiR) + psiP) + cep;
    double rho = sqrt(r2) / w0;
    double xi = y / w0;
    double nu = z / w0;
    double eta = 1.0 / sqrt(1.0 + xz * xz);
    double rho2 = ipow(rho, 2), rho4 = ipow(rho, 4), rho6 = ipow(rho, 6), rho8 = ipow(rho, 8);
    double kc = k0 * ctau;
    double pc = psi - cep;
    double E = (((E0 * w0) / wx) * exp((-r2) / (wx * wx))) * exp((-(pc * pc)) / (kc * kc));

    double S0 = sin(psi);
    double S2 = ipow(eta, 2) * sin(psi + 2.0 * psiG);
    double S3 = ipow(eta, 3) * sin(psi + 3.0 * psiG);
    double S4 = ipow(eta, 4) * sin(psi + 4.0 * psiG);
    double S5 = ipow(eta, 5) * sin(psi + 5.0 * psiG);
    double S6 = ipow(eta, 6) * sin(psi + 6.0 * psiG);
    double C1 = ipow(eta, 1) * cos(psi + 1.0 * psiG);
    double C2 = ipow(eta, 2) * cos(psi + 2.0 * psiG);
    double C3 = ipow(eta, 3) * cos(psi + 3.0 * psiG);
    double C4 = ipow(eta, 4) * cos(psi + 4.0 * psiG);
    double C5 = ipow(eta, 5) * cos(psi + 5.0 * psiG);
    double C6 = ipow(eta, 6) * cos(psi + 6.0 * psiG);
    double C7 = ipow(eta, 7) * cos(psi + 7.0 * psiG);
    double e2 = ipow(ep, 2), e3 = ipow(ep, 3), e4 = ipow(ep, 4), e5 = ipow(ep, 5);
    double xi2 = ipow(xi, 2);

    double exA = (((-C2) / 2.0) + rho2 * C3) - (rho4 * C4) / 4.0;
    double exB = ((((-0.375 * C3) - (0.375 * rho2) * C4) + (1.0625 * rho4) * C5) -
                  (0.375 * rho6) * C6) + (rho8 * C7) / 32.0;
    double Ex_ = (E * xi) * (((ep * C1) + e3 * exA) + e5 * exB);

    double eyA = (xi2 * S2) - (rho4 * S3) / 4.0;
    double eyB = ((((S2 / 8.0) - (rho2 * S3) / 4.0) - ((rho2 * (rho2 - 16.0 * xi2)) * S4) / 16.0) -
                  ((rho4 * (rho2 + 2.0 * xi2)) * S5) / 8.0) + (rho8 * S6) / 32.0;
    double Ey_ = E * ((S0 + e2 * eyA) + e4 * eyB);

    double Ez_ = ((E * xi) * nu) * ((e2 * S2) + e4 * ((rho2 * S4) - (rho4 * S5) / 4.0));

    double bxA = ((C2 / 2.0) + (rho2 * C3) / 2.0) - (rho4 * C4) / 4.0;
    double bxB = ((((0.375 * C3) + (0.375 * rho2) * C4) + (0.1875 * rho4) * C5) - (rho6 * C6) / 4.0) +
                 (rho8 * C7) / 32.0;
    double Bx_ = ((E / C_LIGHT) * nu) * (((ep * C1) + e3 * bxA) + e5 * bxB);

    double bzA = ((rho2 * S2) / 2.0) - (rho4 * S3) / 4.0;
    double bzB = (((((-S2) / 8.0) + (rho2 * S3) / 4.0) + (0.3125 * rho4) * S4) - (rho6 * S5) / 4.0) +
                 (rho8 * S6) / 32.0;
    double Bz_ = (E / C_LIGHT) * ((S0 + e2 * bzA) + e4 * bzB);
    double By_ = 0.0;

    F[0] = Ex_;
    F[1] = Ey_ * cp - Ez_ * sp;
    F[2] = Ey_ * sp + Ez_ * cp;
    F[3] = Bx_;
    F[4] = (By_ * cp - Bz_ * sp) * dir;
    F[5] = (By_ * sp + Bz_ * cp) * dir;
}

static void field_term(int kind, const double *p, double x, double y, double z, double t, double F[6]) {
    switch (kind) {
    case ORC_FIELD_STATIC: field_static(p, F); break;
    case ORC_FIELD_SIMPLE: field_simple(p, x, y, z, t, F); break;
    case ORC_FIELD_GAUSSIAN: field_gaussian(p, x, y, z, t, F); break;
    case ORC_FIELD_FOCUSED: field_focused(p, x, y, z, t, F); break;
    default: for (int i = 0; i < 6; ++i) F[i] = NAN;
    }
}

/* Fields.__add__ (fields.py:52-61) sums componentwise in tree order; the
 * tree is given in postfix form. */
#define ORC_MAX_STACK 32
static void field_program(const int32_t *ops, int32_t n_ops, const int32_t *kinds, const double *params,
                          double x, double y, double z, double t, double out[6]) {
    double st[ORC_MAX_STACK][6];
    int sp = 0;
    for (int i = 0; i < n_ops; ++i) {
        int op = ops[i];
        if (op >= 0) {
            field_term(kinds[op], params + (size_t)op * ORC_TERM_PARAMS, x, y, z, t, st[sp]);
            ++sp;
        } else {
            --sp;
            for (int k = 0; k < 6; ++k) st[sp - 1][k] = st[sp - 1][k] + st[sp][k];
        }
    }
    for (int k = 0; k < 6; ++k) out[k] = st[0][k];
}

/* Fields.field_func CPU launcher, fields.py:41-46 */
void orc_field_eval(const int32_t *ops, int32_t n_ops, const int32_t *kinds, const double *params,
                    const double *x, const double *y, const double *z, double t,
                    int64_t N, const uint8_t *to_be_pruned,
                    double *Ex, double *Ey, double *Ez, double *Bx, double *By, double *Bz) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        double F[6];
        field_program(ops, n_ops, kinds, params, x[ip], y[ip], z[ip], t, F);
        Ex[ip] = F[0]; Ey[ip] = F[1]; Ez[ip] = F[2];
        Bx[ip] = F[3]; By[ip] = F[4]; Bz[ip] = F[5];
    }
}

/* ======================================================================== */
/* Pushers                                                                   */
/* ======================================================================== */

/* cpu.py:5-19 */
void orc_push_position(double *x, double *y, double *z, const double *ux, const double *uy,
                       const double *uz, const double *inv_gamma, int64_t N,
                       const uint8_t *to_be_pruned, double dt) {
    const double cdt = C_LIGHT * dt;
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        x[ip] += (cdt * inv_gamma[ip]) * ux[ip];
        y[ip] += (cdt * inv_gamma[ip]) * uy[ip];
        z[ip] += (cdt * inv_gamma[ip]) * uz[ip];
    }
}

/* inline.py:4-36 */
static void boris_one(double *ux, double *uy, double *uz, double *ig,
                      double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                      double q, double dt) {
    double efactor = (q * dt) / ((2.0 * M_E) * C_LIGHT);
    double bfactor = (q * dt) / (2.0 * M_E);
    double uxm = *ux + efactor * Ex;
    double uym = *uy + efactor * Ey;
    double uzm = *uz + efactor * Ez;
    double igm = 1.0 / sqrt(((1.0 + uxm * uxm) + uym * uym) + uzm * uzm);
    double Tx = (bfactor * Bx) * igm;
    double Ty = (bfactor * By) * igm;
    double Tz = (bfactor * Bz) * igm;
    double uxp = (uxm + uym * Tz) - uzm * Ty;
    double uyp = (uym + uzm * Tx) - uxm * Tz;
    double uzp = (uzm + uxm * Ty) - uym * Tx;
    double Tf = 2.0 / (((1.0 + Tx * Tx) + Ty * Ty) + Tz * Tz);
    double Sx = Tf * Tx, Sy = Tf * Ty, Sz = Tf * Tz;
    double uxl = (uxm + uyp * Sz) - uzp * Sy;
    double uyl = (uym + uzp * Sx) - uxp * Sz;
    double uzl = (uzm + uxp * Sy) - uyp * Sx;
    double uxn = uxl + efactor * Ex;
    double uyn = uyl + efactor * Ey;
    double uzn = uzl + efactor * Ez;
    *ux = uxn; *uy = uyn; *uz = uzn;
    *ig = 1.0 / sqrt(((1.0 + uxn * uxn) + uyn * uyn) + uzn * uzn);
}

/* cpu.py:22-31 */
void orc_boris(double *ux, double *uy, double *uz, double *inv_gamma,
               const double *Ex, const double *Ey, const double *Ez,
               const double *Bx, const double *By, const double *Bz,
               double q, int64_t N, const uint8_t *to_be_pruned, double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        boris_one(ux + ip, uy + ip, uz + ip, inv_gamma + ip, Ex[ip], Ey[ip], Ez[ip],
                  Bx[ip], By[ip], Bz[ip], q, dt);
    }
}

/* inline.py:39-100 (spin first with B_eff from u-, then the Boris momentum) */
static void boris_tbmt_one(double *ux, double *uy, double *uz, double *ig,
                           double *sx, double *sy, double *sz,
                           double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                           double q, double ae, double dt) {
    double efactor = (q * dt) / ((2.0 * M_E) * C_LIGHT);
    double bfactor = (q * dt) / (2.0 * M_E);
    double uxm = *ux + efactor * Ex;
    double uym = *uy + efactor * Ey;
    double uzm = *uz + efactor * Ez;
    double uB = (uxm * Bx + uym * By) + uzm * Bz;
    double gm = sqrt(((1.0 + uxm * uxm) + uym * uym) + uzm * uzm);
    double igm = 1.0 / gm;
    double a1 = ae + igm;
    double a2 = (ae * gm) / (gm + 1.0);
    double a3 = ae + 1.0 / (gm + 1.0);
    double Bxe = (a1 * Bx - (a2 * uB) * uxm) - a3 * (uym * Ez - uzm * Ey);
    double Bye = (a1 * By - (a2 * uB) * uym) - a3 * (uzm * Ex - uxm * Ez);
    double Bze = (a1 * Bz - (a2 * uB) * uzm) - a3 * (uxm * Ey - uym * Ex);
    double Tx = bfactor * Bxe, Ty = bfactor * Bye, Tz = bfactor * Bze;
    double T2 = (Tx * Tx + Ty * Ty) + Tz * Tz;
    double Sx = (2.0 * Tx) / (1.0 + T2);
    double Sy = (2.0 * Ty) / (1.0 + T2);
    double Sz = (2.0 * Tz) / (1.0 + T2);
    double s0x = *sx, s0y = *sy, s0z = *sz;
    double sxp = (s0x + s0y * Tz) - s0z * Ty;
    double syp = (s0y + s0z * Tx) - s0x * Tz;
    double szp = (s0z + s0x * Ty) - s0y * Tx;
    *sx = (s0x + syp * Sz) - szp * Sy;
    *sy = (s0y + szp * Sx) - sxp * Sz;
    *sz = (s0z + sxp * Sy) - syp * Sx;

    Tx = (bfactor * Bx) * igm;
    Ty = (bfactor * By) * igm;
    Tz = (bfactor * Bz) * igm;
    double uxp = (uxm + uym * Tz) - uzm * Ty;
    double uyp = (uym + uzm * Tx) - uxm * Tz;
    double uzp = (uzm + uxm * Ty) - uym * Tx;
    double Tf = 2.0 / (((1.0 + Tx * Tx) + Ty * Ty) + Tz * Tz);
    Sx = Tf * Tx; Sy = Tf * Ty; Sz = Tf * Tz;
    double uxl = (uxm + uyp * Sz) - uzp * Sy;
    double uyl = (uym + uzp * Sx) - uxp * Sz;
    double uzl = (uzm + uxp * Sy) - uyp * Sx;
    double uxn = uxl + efactor * Ex;
    double uyn = uyl + efactor * Ey;
    double uzn = uzl + efactor * Ez;
    *ux = uxn; *uy = uyn; *uz = uzn;
    *ig = 1.0 / sqrt(((1.0 + uxn * uxn) + uyn * uyn) + uzn * uzn);
}

/* cpu.py:33-42 */
void orc_boris_tbmt(double *ux, double *uy, double *uz, double *inv_gamma,
                    double *sx, double *sy, double *sz,
                    const double *Ex, const double *Ey, const double *Ez,
                    const double *Bx, const double *By, const double *Bz,
                    double q, double ae, int64_t N, const uint8_t *to_be_pruned, double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        boris_tbmt_one(ux + ip, uy + ip, uz + ip, inv_gamma + ip, sx + ip, sy + ip, sz + ip,
                       Ex[ip], Ey[ip], Ez[ip], Bx[ip], By[ip], Bz[ip], q, ae, dt);
    }
}

/* LL prefactor, inline.py:105: -2/3 / (4 pi eps0) * e**2 * m_e * c / hbar**2 * dt */
static inline double ll_factor(double dt) {
    return ((((((-2.0 / 3.0) / ((4.0 * PI_) * EPS0)) * (E_CHARGE * E_CHARGE)) * M_E) * C_LIGHT) /
            (HBAR * HBAR)) * dt;
}

/* inline.py:104-111 (g = 1) and 114-123 (quantum correction g(chi)) */
static void ll_one(double *ux, double *uy, double *uz, double *ig, double chi, double dt, int quantum) {
    double factor = ll_factor(dt);
    if (quantum) {
        double g = pow((1.0 + (4.8 * (1.0 + chi)) * log(1.0 + 1.7 * chi)) + 2.44 * (chi * chi),
                       -2.0 / 3.0);
        factor = factor * g;
    }
    double c2 = chi * chi;
    double uxn = *ux + ((factor * c2) * (*ux)) * (*ig);
    double uyn = *uy + ((factor * c2) * (*uy)) * (*ig);
    double uzn = *uz + ((factor * c2) * (*uz)) * (*ig);
    *ux = uxn; *uy = uyn; *uz = uzn;
    *ig = 1.0 / sqrt(((1.0 + uxn * uxn) + uyn * uyn) + uzn * uzn);
}

/* cpu.py:44-51 */
void orc_LL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi,
                 int64_t N, const uint8_t *to_be_pruned, double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        ll_one(ux + ip, uy + ip, uz + ip, inv_gamma + ip, chi[ip], dt, 0);
    }
}

/* cpu.py:53-60 */
void orc_CLL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi,
                  int64_t N, const uint8_t *to_be_pruned, double dt) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        ll_one(ux + ip, uy + ip, uz + ip, inv_gamma + ip, chi[ip], dt, 1);
    }
}

/* inline.py:126-134.  A negative radicand (rounding, |E| ~ c|B| along u)
 * gives chi = 0 here; the reference yields NaN, which also never fires. */
static inline double chi_one(double Ex, double Ey, double Ez, double Bx, double By, double Bz,
                             double ux, double uy, double uz, double ig) {
    const double factor = (E_CHARGE * HBAR) / ((M_E * M_E) * (C_LIGHT * (C_LIGHT * C_LIGHT)));
    double gamma = 1.0 / ig;
    double a = gamma * Ex + (uy * Bz - uz * By) * C_LIGHT;
    double b = gamma * Ey + (uz * Bx - ux * Bz) * C_LIGHT;
    double c = gamma * Ez + (ux * By - uy * Bx) * C_LIGHT;
    double s = (ux * Ex + uy * Ey) + uz * Ez;
    double rad = ((a * a + b * b) + c * c) - s * s;
    if (!(rad > 0.0)) rad = 0.0;
    return factor * sqrt(rad);
}

/* cpu.py:62-74 */
void orc_update_chi(const double *Ex, const double *Ey, const double *Ez,
                    const double *Bx, const double *By, const double *Bz,
                    const double *ux, const double *uy, const double *uz,
                    const double *inv_gamma, double *chi, int64_t N, const uint8_t *to_be_pruned) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        chi[ip] = chi_one(Ex[ip], Ey[ip], Ez[ip], Bx[ip], By[ip], Bz[ip], ux[ip], uy[ip], uz[ip],
                          inv_gamma[ip]);
    }
}

/* ======================================================================== */
/* Events and appends                                                        */
/* ======================================================================== */

/* cpu.py:76-87 */
void orc_photon_recoil(double *ux, double *uy, double *uz, double *inv_gamma,
                       const uint8_t *event, const double *delta, int64_t N,
                       const uint8_t *to_be_pruned) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip]) continue;
        if (event[ip]) {
            double f = 1.0 - delta[ip];
            ux[ip] = ux[ip] * f;
            uy[ip] = uy[ip] * f;
            uz[ip] = uz[ip] * f;
            inv_gamma[ip] = 1.0 / sqrt(((1.0 + ux[ip] * ux[ip]) + uy[ip] * uy[ip]) + uz[ip] * uz[ip]);
        }
    }
}

/* cpu.py:226-231 */
void orc_pick_hard_photon(uint8_t *event, const double *delta, const double *inv_gamma,
                          double threshold, int64_t N) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (event[ip]) {
            if (delta[ip] / inv_gamma[ip] < threshold) event[ip] = 0;
        }
    }
}

/* cpu.py:217-224 */
int64_t orc_bool_sum(const uint8_t *event, int64_t N) {
    int64_t n = 0;
#pragma omp parallel for reduction(+ : n) schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) n += event[ip] ? 1 : 0;
    return n;
}

/* cpu.py:192-215 (serial compaction, ascending index order) */
void orc_find_event_index(const uint8_t *event, int64_t N_event, int64_t N, int64_t *index) {
    int64_t idx = 0;
    for (int64_t i = 0; i < N && idx < N_event; ++i)
        if (event[i]) index[idx++] = i;
}

/* cpu.py:89-116 */
void orc_create_photon(const double *x_src, const double *y_src, const double *z_src,
                       const double *ux_src, const double *uy_src, const double *uz_src,
                       double *x_dst, double *y_dst, double *z_dst,
                       double *ux_dst, double *uy_dst, double *uz_dst,
                       double *inv_gamma_dst, uint8_t *photon_to_be_pruned,
                       const int64_t *event_index, const double *photon_delta,
                       int64_t N_buffered, int64_t N_photon) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N_photon; ++ip) {
        int64_t s = event_index[ip], d = N_buffered + ip;
        x_dst[d] = x_src[s];
        y_dst[d] = y_src[s];
        z_dst[d] = z_src[s];
        ux_dst[d] = photon_delta[s] * ux_src[s];
        uy_dst[d] = photon_delta[s] * uy_src[s];
        uz_dst[d] = photon_delta[s] * uz_src[s];
        inv_gamma_dst[d] = 1.0 / sqrt((ux_dst[d] * ux_dst[d] + uy_dst[d] * uy_dst[d]) + uz_dst[d] * uz_dst[d]);
        photon_to_be_pruned[d] = 0;
    }
}

/* cpu.py:119-189 */
void orc_create_pair(const double *x_src, const double *y_src, const double *z_src,
                     const double *ux_src, const double *uy_src, const double *uz_src,
                     uint8_t *photon_to_be_pruned,
                     double *x_dst, double *y_dst, double *z_dst,
                     double *ux_dst, double *uy_dst, double *uz_dst,
                     double *inv_gamma_dst, uint8_t *pair_to_be_pruned,
                     const int64_t *event_index, const double *pair_delta,
                     int64_t N_buffered, int64_t N_pair, int32_t inverse_delta) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N_pair; ++ip) {
        int64_t s = event_index[ip], d = N_buffered + ip;
        x_dst[d] = x_src[s];
        y_dst[d] = y_src[s];
        z_dst[d] = z_src[s];
        double delta = pair_delta[s];
        if (inverse_delta) delta = 1.0 - delta;
        ux_dst[d] = delta * ux_src[s];
        uy_dst[d] = delta * uy_src[s];
        uz_dst[d] = delta * uz_src[s];
        inv_gamma_dst[d] =
            1.0 / sqrt(((1.0 + ux_dst[d] * ux_dst[d]) + uy_dst[d] * uy_dst[d]) + uz_dst[d] * uz_dst[d]);
        pair_to_be_pruned[d] = 0;
        photon_to_be_pruned[s] = 1;
    }
}

/* ======================================================================== */
/* Rejection sampling                                                        */
/* ======================================================================== */

/* linear interpolation on the uniform z grid z = i * z_max/(z_N-1).
 * The reference indexes table[idx+1] with idx = int(z/dz); for z == z_max
 * that can be z_N-1 (one past the end), so idx is capped at z_N-2 here, which
 * gives the same interpolant value. */
static inline void ai_interp(double z, const double *int_Ai, const double *Aip, int32_t z_N,
                             double z_max, double *iA, double *dA) {
    const double dz = (z_max - 0.0) / (double)(z_N - 1);
    int64_t idx = (int64_t)((z - 0.0) / dz);
    if (idx > z_N - 2) idx = z_N - 2;
    double zl = 0.0 + (double)idx * dz;
    double k = (int_Ai[idx + 1] - int_Ai[idx]) / dz;
    *iA = int_Ai[idx] + k * (z - zl);
    k = (Aip[idx + 1] - Aip[idx]) / dz;
    *dA = Aip[idx] + k * (z - zl);
}

/* qed/rejection_sampling_tables.py:32-53.  z > z_max -> 0 (the reference
 * reads one element past the table there; its measured behaviour is 0). */
double orc_photon_prob_rate_from_table(double chi_e, double delta, const double *int_Ai,
                                       const double *Aip, int32_t z_N, double z_max) {
    double chi_gamma = delta * chi_e;
    double chi_ep = chi_e - chi_gamma;
    double z = pow((chi_gamma / chi_e) / chi_ep, 2.0 / 3.0);
    const double factor = (((-ALPHA) * M_E) * (C_LIGHT * C_LIGHT)) / HBAR;
    if (!(z <= z_max)) return 0.0;
    double iA, dA;
    ai_interp(z, int_Ai, Aip, z_N, z_max, &iA, &dA);
    return factor * (iA + (2.0 / z + chi_gamma * sqrt(z)) * dA);
}

/* qed/rejection_sampling_tables.py:56-78 */
double orc_pair_prob_rate_from_table(double chi_gamma, double delta, const double *int_Ai,
                                     const double *Aip, int32_t z_N, double z_max) {
    double chi_e = delta * chi_gamma;
    double chi_ep = chi_gamma - chi_e;
    double z = pow((chi_gamma / chi_e) / chi_ep, 2.0 / 3.0);
    const double factor = ((ALPHA * M_E) * (C_LIGHT * C_LIGHT)) / HBAR;
    if (!(z <= z_max)) return 0.0;
    double iA, dA;
    ai_interp(z, int_Ai, Aip, z_N, z_max, &iA, &dA);
    return factor * (iA + (2.0 / z - chi_gamma * sqrt(z)) * dA);
}

/* qed/rejection_sampling.py:73-89 (Gonoskov et al. 2015 modified event
 * generator: delta = r1**3, accept if r2 < 3 r1**2 W(chi, delta) dt/gamma) */
void orc_photon_from_rejection_sampling(const double *inv_gamma, const double *chi_e, double dt,
                                        int64_t N, const uint8_t *to_be_pruned,
                                        uint8_t *event, double *delta,
                                        const double *int_Ai, const double *Aip, int32_t z_N,
                                        double z_max, uint64_t seed, uint32_t stream,
                                        uint32_t step) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip] || chi_e[ip] == 0.0) {
            event[ip] = 0;
            continue;
        }
        double r[2];
        orc_uniform2(seed, stream, step, 0, ip, r);
        double r1 = r[0], r2 = r[1];
        double dtau = dt * inv_gamma[ip];
        double d = r1 * (r1 * r1);
        double prob = ((3.0 * (r1 * r1)) * orc_photon_prob_rate_from_table(chi_e[ip], d, int_Ai, Aip, z_N, z_max)) * dtau;
        if (r2 < prob) {
            delta[ip] = d;
            event[ip] = 1;
        } else {
            delta[ip] = 0.0;
            event[ip] = 0;
        }
    }
}

/* qed/rejection_sampling.py:92-107 (delta = r1, accept if r2 < W dt/gamma) */
void orc_pair_from_rejection_sampling(const double *inv_gamma, const double *chi_gamma, double dt,
                                      int64_t N, const uint8_t *to_be_pruned,
                                      uint8_t *event, double *delta,
                                      const double *int_Ai, const double *Aip, int32_t z_N,
                                      double z_max, uint64_t seed, uint32_t stream,
                                      uint32_t step) {
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip] || chi_gamma[ip] == 0.0) {
            event[ip] = 0;
            continue;
        }
        double r[2];
        orc_uniform2(seed, stream, step, 0, ip, r);
        double r1 = r[0], r2 = r[1];
        double dtau = dt * inv_gamma[ip];
        double prob = orc_pair_prob_rate_from_table(chi_gamma[ip], r1, int_Ai, Aip, z_N, z_max) * dtau;
        if (r2 < prob) {
            delta[ip] = r1;
            event[ip] = 1;
        } else {
            delta[ip] = 0.0;
            event[ip] = 0;
        }
    }
}

/* ======================================================================== */
/* Optical depth                                                             */
/* ======================================================================== */

/* fractional row index of qed/optical_depth_tables.py:44-53 (_get_chi_idx),
 * clamped to the last row above the table (the reference reads past it) */
static inline double od_row(double log_chi, const orc_od_table *t) {
    if (log_chi > t->log_chi_max) log_chi = t->log_chi_max;
    double idx = (log_chi - t->log_chi_min) / t->log_chi_delta;
    if (idx > (double)(t->chi_N - 1)) idx = (double)(t->chi_N - 1);
    return idx;
}

/* _linear_interp1d, qed/optical_depth_tables.py:56-66 */
double orc_od_interp1d(double chi, const orc_od_table *t) {
    double log_chi = log10(chi);
    if (log_chi < t->log_chi_min) return 0.0;
    double fidx = od_row(log_chi, t);
    int64_t idx = (int64_t)floor(fidx);
    if (idx > t->chi_N - 2) idx = t->chi_N - 2;
    if (log_chi > t->log_chi_max) log_chi = t->log_chi_max;
    double left = t->log_chi_min + (double)idx * t->log_chi_delta;
    double k = (t->rate_total[idx + 1] - t->rate_total[idx]) / t->log_chi_delta;
    return t->rate_total[idx] + k * (log_chi - left);
}

/* _bisect_interp, qed/optical_depth_tables.py:69-112: rows blended linearly
 * in chi, bisection over the delta columns, linear inverse interpolation.
 * Equality mid == r (no exit branch in the reference) moves `high` down. */
double orc_od_bisect(double chi, double r_uniform, const orc_od_table *t) {
    const int32_t n = t->delta_N;
    double log_chi = log10(chi);
    double fidx = od_row(log_chi, t);
    int64_t lo_i = (int64_t)floor(fidx);
    if (lo_i > t->chi_N - 2) lo_i = t->chi_N - 2;
    if (lo_i < 0) lo_i = 0;
    int64_t hi_i = lo_i + 1;
    if (chi > pow(10.0, t->log_chi_max)) chi = pow(10.0, t->log_chi_max);
    double chi_low = pow(10.0, t->log_chi_min + (double)lo_i * t->log_chi_delta);
    double chi_high = pow(10.0, t->log_chi_min + (double)hi_i * t->log_chi_delta);
    const double *TL = t->cumulative + (size_t)lo_i * n;
    const double *TH = t->cumulative + (size_t)hi_i * n;
#define ROWVAL(j) (TL[(j)] + ((TH[(j)] - TL[(j)]) / (chi_high - chi_low)) * (chi - chi_low))
    double ymin = ROWVAL(0);
    double ymax = ROWVAL(n - 1);
    double r = r_uniform * (ymax - ymin) + ymin;
    int64_t low = 0, high = n - 1;
    while (low <= high) {
        int64_t mid = (low + high) / 2;
        double md = ROWVAL(mid);
        if (md < r) low = mid + 1;
        else high = mid - 1;
    }
    int64_t di = high;
    if (di < 0) di = 0;
    if (di > n - 2) di = n - 2;
    double y1 = ROWVAL(di);
    double y2 = ROWVAL(di + 1);
#undef ROWVAL
    double dl = pow(10.0, t->log_delta_min + (double)di * t->log_delta_delta);
    double dr = pow(10.0, t->log_delta_min + (double)(di + 1) * t->log_delta_delta);
    double k = (dr - dl) / (y2 - y1);
    return dl + k * (r - y1);
}

/* _bisect_interp over a batch of (log10 chi, u) queries, OpenMP: the CPU
 * counterpart of the batched table sampler (optical_depth_tables.py:59-102) */
void orc_od_bisect_batch(const double *log_chi, const double *u, int64_t n, const orc_od_table *t, double *delta) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) delta[i] = orc_od_bisect(pow(10.0, log_chi[i]), u[i], t);
}

/* update_tau_e / update_tau_gamma, qed/optical_depth.py:15-111.
 * Draws: purpose 1 -> (tau reset, tau after event); purpose 2 -> (inverse-CDF r, unused) */
void orc_update_tau(double *tau, const double *inv_gamma, const double *chi, double dt,
                    int64_t N, const uint8_t *to_be_pruned, uint8_t *event, double *delta,
                    const orc_od_table *t, uint64_t seed, uint32_t stream, uint32_t step) {
    const double chi_min = pow(10.0, t->log_chi_min);
#pragma omp parallel for schedule(static)
    for (int64_t ip = 0; ip < N; ++ip) {
        if (to_be_pruned[ip] || chi[ip] < chi_min) {
            event[ip] = 0;
            delta[ip] = 0.0;
            continue;
        }
        double rate = orc_od_interp1d(chi[ip], t);
        double dtau = dt * inv_gamma[ip];
        double ra[2];
        orc_uniform2(seed, stream, step, 1, ip, ra);
        if (tau[ip] == 0.0) tau[ip] = -log(1.0 - ra[0]);
        tau[ip] -= rate * dtau;
        if (tau[ip] < 0.0) {
            double rb[2];
            orc_uniform2(seed, stream, step, 2, ip, rb);
            tau[ip] = -log(1.0 - ra[1]);
            event[ip] = 1;
            delta[ip] = orc_od_bisect(chi[ip], rb[0], t);
        } else {
            event[ip] = 0;
            delta[ip] = 0.0;
        }
    }
}
