/*
 * sfp_oracle.h -- CPU oracle for the sfparticles per-particle step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * path is compared against; the product (sfparticles_b200) never links,
 * loads or calls it.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline legs of bench.py use it.
 *
 * Every function restates one routine of the reference package
 * (xsgeng/sfparticles v0.4.12, pure Python + Numba) in plain C with the
 * same operation order, so that with glibc libm and -ffp-contract=off the
 * results agree bit-for-bit with the Numba CPU kernels.  The random draws
 * are NOT the reference's (Numba's per-thread MT19937 cannot be matched);
 * they come from a keyed Philox-4x32-10 stream shared with the CUDA path,
 * so GPU and oracle agree particle by particle.
 *
 * Array arguments are float64 / uint8 (bool) SoA vectors, exactly the
 * reference's attribute arrays; N is the buffered particle count.
 */
#ifndef SFP_ORACLE_H
#define SFP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- RNG ---------------------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* two uniforms in (0,1) for (seed, stream, step, purpose, slot) */
void orc_uniform2(uint64_t seed, uint32_t stream, uint32_t step, uint32_t purpose,
                  int64_t slot, double out[2]);
void orc_uniform2_batch(uint64_t seed, uint32_t stream, uint32_t step, uint32_t purpose,
                        const int64_t *slots, int64_t n, double *out);

/* ---- fields ------------------------------------------------------------- */
/* term kinds; parameter layouts are documented in oracle.py (FieldProgram) */
enum { ORC_FIELD_STATIC = 0, ORC_FIELD_SIMPLE = 1, ORC_FIELD_GAUSSIAN = 2, ORC_FIELD_FOCUSED = 3 };
#define ORC_TERM_PARAMS 16
/* ops: value >= 0 pushes term #value, -1 adds the two top entries */
void orc_field_eval(const int32_t *ops, int32_t n_ops, const int32_t *kinds, const double *params,
                    const double *x, const double *y, const double *z, double t,
                    int64_t N, const uint8_t *to_be_pruned,
                    double *Ex, double *Ey, double *Ez, double *Bx, double *By, double *Bz);

/* ---- pushers (cpu.py / inline.py) -------------------------------------- */
void orc_push_position(double *x, double *y, double *z, const double *ux, const double *uy,
                       const double *uz, const double *inv_gamma, int64_t N,
                       const uint8_t *to_be_pruned, double dt);
void orc_boris(double *ux, double *uy, double *uz, double *inv_gamma,
               const double *Ex, const double *Ey, const double *Ez,
               const double *Bx, const double *By, const double *Bz,
               double q, int64_t N, const uint8_t *to_be_pruned, double dt);
void orc_boris_tbmt(double *ux, double *uy, double *uz, double *inv_gamma,
                    double *sx, double *sy, double *sz,
                    const double *Ex, const double *Ey, const double *Ez,
                    const double *Bx, const double *By, const double *Bz,
                    double q, double ae, int64_t N, const uint8_t *to_be_pruned, double dt);
void orc_LL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi,
                 int64_t N, const uint8_t *to_be_pruned, double dt);
void orc_CLL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi,
                  int64_t N, const uint8_t *to_be_pruned, double dt);
void orc_update_chi(const double *Ex, const double *Ey, const double *Ez,
                    const double *Bx, const double *By, const double *Bz,
                    const double *ux, const double *uy, const double *uz,
                    const double *inv_gamma, double *chi, int64_t N, const uint8_t *to_be_pruned);

/* ---- events and appends ------------------------------------------------- */
void orc_photon_recoil(double *ux, double *uy, double *uz, double *inv_gamma,
                       const uint8_t *event, const double *delta, int64_t N,
                       const uint8_t *to_be_pruned);
void orc_pick_hard_photon(uint8_t *event, const double *delta, const double *inv_gamma,
                          double threshold, int64_t N);
int64_t orc_bool_sum(const uint8_t *event, int64_t N);
void orc_find_event_index(const uint8_t *event, int64_t N_event, int64_t N, int64_t *index);
void orc_create_photon(const double *x_src, const double *y_src, const double *z_src,
                       const double *ux_src, const double *uy_src, const double *uz_src,
                       double *x_dst, double *y_dst, double *z_dst,
                       double *ux_dst, double *uy_dst, double *uz_dst,
                       double *inv_gamma_dst, uint8_t *photon_to_be_pruned,
                       const int64_t *event_index, const double *photon_delta,
                       int64_t N_buffered, int64_t N_photon);
void orc_create_pair(const double *x_src, const double *y_src, const double *z_src,
                     const double *ux_src, const double *uy_src, const double *uz_src,
                     uint8_t *photon_to_be_pruned,
                     double *x_dst, double *y_dst, double *z_dst,
                     double *ux_dst, double *uy_dst, double *uz_dst,
                     double *inv_gamma_dst, uint8_t *pair_to_be_pruned,
                     const int64_t *event_index, const double *pair_delta,
                     int64_t N_buffered, int64_t N_pair, int32_t inverse_delta);

/* ---- QED: rejection sampling (qed/rejection_sampling*.py) ------------------ */
double orc_photon_prob_rate_from_table(double chi_e, double delta, const double *int_Ai,
                                       const double *Aip, int32_t z_N, double z_max);
double orc_pair_prob_rate_from_table(double chi_gamma, double delta, const double *int_Ai,
                                     const double *Aip, int32_t z_N, double z_max);
/* draws: orc_uniform2(seed, stream, step, purpose 0, slot) -> (r1, r2) */
void orc_photon_from_rejection_sampling(const double *inv_gamma, const double *chi_e, double dt,
                                        int64_t N, const uint8_t *to_be_pruned,
                                        uint8_t *event, double *delta,
                                        const double *int_Ai, const double *Aip, int32_t z_N,
                                        double z_max, uint64_t seed, uint32_t stream,
                                        uint32_t step);
void orc_pair_from_rejection_sampling(const double *inv_gamma, const double *chi_gamma, double dt,
                                      int64_t N, const uint8_t *to_be_pruned,
                                      uint8_t *event, double *delta,
                                      const double *int_Ai, const double *Aip, int32_t z_N,
                                      double z_max, uint64_t seed, uint32_t stream,
                                      uint32_t step);

/* ---- QED: optical depth (qed/optical_depth*.py) ---------------------------- */
typedef struct {
    int32_t chi_N;          /* rows of the tables                        */
    int32_t delta_N;        /* columns of the cumulative tables          */
    double log_chi_min;     /* log10 chi of row 0                        */
    double log_chi_delta;   /* row spacing in log10 chi                  */
    double log_delta_min;   /* log10 delta of column 0                   */
    double log_delta_delta; /* column spacing in log10 delta             */
    double log_chi_max;     /* log10 chi of the last row (clamp above)    */
    const double *rate_total;  /* [chi_N]                                */
    const double *cumulative;  /* [chi_N][delta_N]                       */
} orc_od_table;

double orc_od_interp1d(double chi, const orc_od_table *tab);
double orc_od_bisect(double chi, double r_uniform, const orc_od_table *tab);
void orc_od_bisect_batch(const double *log_chi, const double *u, int64_t n, const orc_od_table *tab, double *delta);
void orc_update_tau(double *tau, const double *inv_gamma, const double *chi, double dt,
                    int64_t N, const uint8_t *to_be_pruned, uint8_t *event, double *delta,
                    const orc_od_table *tab, uint64_t seed, uint32_t stream, uint32_t step);

#ifdef __cplusplus
}
#endif
#endif
