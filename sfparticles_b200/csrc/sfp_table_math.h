// sfp_table_math.h -- the differential rates of the QED tables, host and
// device (sfp_tables.cu runs them on the GPU; the CPU tests compile the
// same code for the host).
//
// rejection sampling (qed/rejection_sampling_tables.py:80-88): int_Ai(z) =
// quad(Ai, z, inf) and Ai'(z); optical depth
// (qed/optical_depth_tables.py:136-160):
//   photon: P(delta) = factor (int_Ai(z) + (2/z + chi_g sqrt z) Ai'(z)),
//           chi_g = delta chi_e, z = (chi_g / chi_e / (chi_e - chi_g))^(2/3);
//   pair:   P(delta) = factor (int_Ai(z) + (2/z - chi_g sqrt z) Ai'(z)),
//           chi_e = delta chi_g, z = (chi_g / chi_e / (chi_g - chi_e))^(2/3);
// P(1) = 0.  int_Ai and Ai' are exactly 0 from z = 108 on, where their
// float64 values are 0 (the reference's scipy returns NaN at z ~ 1e8 and
// leaves its low-chi pair rows NaN).
#pragma once
#include "sfp_quadpack.h"

namespace sfp_tab {

struct AiFn {
    SFP_HD double operator()(double x) const { return sfp_airy::Ai(x); }
};

// int_Ai and Ai' at z
SFP_HD void airy_terms(double z, double& ia, double& aip) {
    if (z >= sfp_airy::kAiryZero) {
        ia = 0.0;
        aip = 0.0;
        return;
    }
    double ai;
    sfp_airy::airy(z, ai, aip);
    ia = sfp_quad::quad_inf(AiFn{}, z);
}

// the differential rate of one chi row (kind 0: photon emission, 1: pair creation)
struct RateFn {
    double chi, factor;
    int kind;
    SFP_HD double operator()(double delta) const {
        if (delta == 1.0) return 0.0;
        const double chi_part = delta * chi;  // chi_gamma (photon) or chi_e (pair)
        const double chi_rest = chi - chi_part;
        double z;
        if (kind == 0) z = pow(chi_part / chi / chi_rest, 2.0 / 3.0);
        else z = pow(chi / chi_part / chi_rest, 2.0 / 3.0);
        double ia, aip;
        airy_terms(z, ia, aip);
        const double chi_g = kind == 0 ? chi_part : chi;
        const double s = kind == 0 ? 2.0 / z + chi_g * sqrt(z) : 2.0 / z - chi_g * sqrt(z);
        return factor * (ia + s * aip);
    }
};

}  // namespace sfp_tab
