// sfp_airy.h -- Ai(z) and Ai'(z) for z >= 0 in float64, host and device.
//
// Used by the QED table generator (sfp_tables.cu), which restates the
// reference's table generators (qed/rejection_sampling_tables.py:80-112,
// qed/optical_depth_tables.py:126-230); the reference takes these values
// from scipy.special.airy.  Written from the mathematics:
//   * 0 <= z <= 2: the Maclaurin series (DLMF 9.4.1-9.4.2)
//       Ai(z) = c1 f(z) - c2 g(z),  Ai'(z) = c1 f'(z) - c2 g'(z),
//       f = sum_k 3^k (1/3)_k z^(3k) / (3k)!,  g = sum_k 3^k (2/3)_k z^(3k+1) / (3k+1)!,
//       c1 = Ai(0) = 3^(-2/3) / Gamma(2/3),  c2 = -Ai'(0) = 3^(-1/3) / Gamma(1/3);
//     at z = 2 the two terms cancel to 1/30 of their size, so about 1.5
//     digits are lost;
//   * z > 2: through the modified Bessel function of the third kind
//     (DLMF 9.6.1, 9.6.2), zeta = (2/3) z^(3/2) > 1.88,
//       Ai(z) = sqrt(z / 3) K_{1/3}(zeta) / pi,  Ai'(z) = -z K_{2/3}(zeta) / (pi sqrt 3),
//     with K_{1/3} and K_{2/3} from Steed's continued fraction for
//     K_mu(x), K_{mu+1}(x) at mu = -1/3 (Temme, J. Comput. Phys. 19 (1975)
//     324; Thompson and Barnett, J. Comput. Phys. 64 (1986) 490), using
//     K_{-1/3} = K_{1/3}.
// Both are exactly 0 from z = 108 on, where their float64 values are 0
// (exp(-(2/3) 108^1.5) = 1e-325).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SFP_HD __host__ __device__ inline
#else
#define SFP_HD inline
#endif

namespace sfp_airy {

constexpr double kAiryZero = 108.0;
constexpr double kC1 = 0.35502805388781723926;  // Ai(0)
constexpr double kC2 = 0.25881940379280679840;  // -Ai'(0)
constexpr double kPi = 3.14159265358979323846;

// Maclaurin series, 0 <= z <= 2
SFP_HD void series(double z, double& ai, double& aip) {
    const double z3 = z * z * z;
    double f = 1.0, g = z, fp = 0.0, gp = 1.0;
    double tf = 1.0, tg = z;  // current terms of f and g
    for (int k = 1; k < 60; ++k) {
        const double k3 = 3.0 * k;
        tf *= z3 / ((k3 - 1.0) * k3);
        tg *= z3 / (k3 * (k3 + 1.0));
        f += tf;
        g += tg;
        // d/dz z^(3k) = 3k z^(3k-1), d/dz z^(3k+1) = (3k+1) z^(3k)
        if (z > 0.0) {
            fp += k3 * tf / z;
            gp += (k3 + 1.0) * tg / z;
        }
        if (tf < 1e-18 * f && tg < 1e-18 * fabs(g) + 1e-300) break;
    }
    ai = kC1 * f - kC2 * g;
    aip = kC1 * fp - kC2 * gp;
}

// Steed's continued fraction (CF2): K_mu(x) and K_{mu+1}(x), |mu| <= 1/2, x > 0
SFP_HD void bessel_k_cf2(double mu, double x, double& kmu, double& kmu1) {
    double b = 2.0 * (1.0 + x), d = 1.0 / b, h = d, delh = d;
    double q1 = 0.0, q2 = 1.0;
    const double a1 = 0.25 - mu * mu;
    double q = a1, c = a1, a = -a1, s = 1.0 + q * delh;
    for (int i = 2; i < 20000; ++i) {
        a -= 2.0 * (i - 1);
        c = -a * c / i;
        const double qnew = (q1 - b * q2) / a;
        q1 = q2;
        q2 = qnew;
        q += c * qnew;
        b += 2.0;
        d = 1.0 / (b + a * d);
        delh = (b * d - 1.0) * delh;
        h += delh;
        const double dels = q * delh;
        s += dels;
        if (fabs(dels / s) < 1e-17) break;
    }
    h = a1 * h;
    kmu = sqrt(kPi / (2.0 * x)) * exp(-x) / s;
    kmu1 = kmu * (mu + x + 0.5 - h) / x;
}

// Ai(z), Ai'(z) for z >= 0
SFP_HD void airy(double z, double& ai, double& aip) {
    if (z >= kAiryZero) {
        ai = 0.0;
        aip = 0.0;
    } else if (z <= 2.0) {
        series(z, ai, aip);
    } else {
        const double zeta = (2.0 / 3.0) * z * sqrt(z);
        double k13, k23;
        bessel_k_cf2(-1.0 / 3.0, zeta, k13, k23);  // K_{-1/3} = K_{1/3}, K_{2/3}
        ai = sqrt(z / 3.0) * k13 / kPi;
        aip = -z * k23 / (kPi * sqrt(3.0));
    }
}

SFP_HD double Ai(double z) {
    double a, d;
    airy(z, a, d);
    return a;
}

}  // namespace sfp_airy
