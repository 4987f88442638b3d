// sfp_tables.cu -- the QED rate tables generated on the GPU (no counterpart
// kernel in the reference, which builds them with scipy on the CPU).
//
// Restates the reference's generators with their own algorithm, so that the
// tables reproduce its entries:
//   * rejection sampling (qed/rejection_sampling_tables.py:80-112): on a z
//     grid, int_Ai(z) = quad(Ai, z, inf) and Ai'(z);
//   * optical depth (qed/optical_depth_tables.py:136-198): per chi row the
//     total rate quad(P, 0, 1) and the cumulative row
//       integ[0] = quad(P, 0, delta_0),
//       integ[i] = integ[i-1] + P(delta_i) (delta_i - delta_{i-1}),
//     with the differential rate
//       photon: P(delta) = factor (int_Ai(z) + (2/z + chi_g sqrt z) Ai'(z)),
//               chi_g = delta chi_e, z = (chi_g / chi_e / (chi_e - chi_g))^(2/3);
//       pair:   P(delta) = factor (int_Ai(z) + (2/z - chi_g sqrt z) Ai'(z)),
//               chi_e = delta chi_g, z = (chi_g / chi_e / (chi_g - chi_e))^(2/3);
//     P(1) = 0, and int_Ai = Ai' = 0 from z = 108 on (the product's tables'
//     convention: their float64 values there are 0; the reference's scipy
//     returns NaN at z ~ 1e8, which leaves its low-chi pair rows NaN).
// quad is QUADPACK's QAGS / QAGI as scipy runs it (sfp_quadpack.h) and Ai,
// Ai' come from sfp_airy.h.  The grids (z, chi rows, log-spaced delta) and
// the rate prefactor are computed by the caller exactly as the reference
// computes them (numpy linspace / logspace, -alpha m c^2 / hbar) and passed
// in.  One thread per z point, per chi row, or per (chi row, delta column).
#include <cuda_runtime.h>

#include <string>

#include "sfp.h"
#include "sfp_internal.h"
#include "sfp_table_math.h"

namespace {

using sfp_tab::RateFn;
using sfp_tab::airy_terms;

__global__ void k_rs_table(const double* __restrict__ z, long long n, double* __restrict__ int_ai,
                           double* __restrict__ aip) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double ia, d;
        airy_terms(z[i], ia, d);
        int_ai[i] = ia;
        aip[i] = d;
    }
}

// per chi row: the total rate and the first cumulative entry
__global__ void k_od_totals(int kind, double factor, const double* __restrict__ chi, long long n_chi,
                            const double* __restrict__ delta, double* __restrict__ total, double* __restrict__ first) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n_chi;
         r += (long long)gridDim.x * blockDim.x) {
        const RateFn P{chi[r], factor, kind};
        total[r] = sfp_quad::quad(P, 0.0, 1.0);
        first[r] = sfp_quad::quad(P, 0.0, delta[0]);
    }
}

// P(delta_i) on every (row, column >= 1)
__global__ void k_od_rates(int kind, double factor, const double* __restrict__ chi, long long n_chi,
                           const double* __restrict__ delta, long long n_delta, double* __restrict__ rate) {
    const long long n = n_chi * n_delta;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long r = k / n_delta, i = k % n_delta;
        rate[k] = i == 0 ? 0.0 : RateFn{chi[r], factor, kind}(delta[i]);
    }
}

// the left-Riemann accumulation of each row, in the reference's order and
// rounding (product rounded, then added)
__global__ void k_od_accumulate(const double* __restrict__ first, const double* __restrict__ delta, long long n_delta,
                                long long n_chi, double* __restrict__ cum) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n_chi;
         r += (long long)gridDim.x * blockDim.x) {
        double* row = cum + r * n_delta;  // holds P(delta_i) on entry
        double acc = first[r];
        row[0] = acc;
        for (long long i = 1; i < n_delta; ++i) {
            acc = __dadd_rn(acc, __dmul_rn(row[i], __dsub_rn(delta[i], delta[i - 1])));
            row[i] = acc;
        }
    }
}

unsigned grid_of(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 65535) g = 65535;
    return (unsigned)g;
}

}  // namespace

extern "C" {

int sfp_table_rs(const double* z, int64_t n, double* int_ai, double* aip, void* stream) {
    if (n > 0 && (!z || !int_ai || !aip)) return sfp_set_error(SFP_EINVAL, "sfp_table_rs: NULL argument");
    if (n <= 0) return SFP_OK;
    k_rs_table<<<grid_of(n, 64), 64, 0, reinterpret_cast<cudaStream_t>(stream)>>>(z, n, int_ai, aip);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sfp_set_error(SFP_ECUDA, std::string("sfp_table_rs: ") + cudaGetErrorString(e));
    return SFP_OK;
}

int sfp_table_od(int kind, double factor, const double* chi, int64_t n_chi, const double* delta, int64_t n_delta,
                 double* total, double* cumulative, double* first, void* stream) {
    if (kind != 0 && kind != 1) return sfp_set_error(SFP_EINVAL, "sfp_table_od: kind is 0 (photon) or 1 (pair)");
    if (n_chi > 0 && (!chi || !delta || !total || !cumulative || !first || n_delta < 1))
        return sfp_set_error(SFP_EINVAL, "sfp_table_od: NULL argument or empty delta grid");
    if (n_chi <= 0) return SFP_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // deep quadrature recursion per thread: small blocks, one chi row per thread
    k_od_totals<<<grid_of(n_chi, 32), 32, 0, s>>>(kind, factor, chi, n_chi, delta, total, first);
    k_od_rates<<<grid_of(n_chi * n_delta, 64), 64, 0, s>>>(kind, factor, chi, n_chi, delta, n_delta, cumulative);
    k_od_accumulate<<<grid_of(n_chi, 32), 32, 0, s>>>(first, delta, n_delta, n_chi, cumulative);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return sfp_set_error(SFP_ECUDA, std::string("sfp_table_od: ") + cudaGetErrorString(e));
    return SFP_OK;
}

}  // extern "C"
