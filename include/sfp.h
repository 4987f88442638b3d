/*
 * sfp.h -- C-ABI of libsfp.so, the B200 implementation of the sfparticles
 * per-particle step.
 *
 * Conventions
 *   - every entry point returns 0 on success or a negative SFP_E* code; the
 *     message of the last failure on the calling thread is sfp_last_error();
 *   - array arguments are DEVICE pointers (float64 / uint8 bool / int64);
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default);
 *   - no entry point synchronises the device unless it says so.
 *
 * Reference interfaces replaced (paths inside xsgeng/sfparticles v0.4.12):
 * the 12 kernels bound at sfparticles/particles.py:14-25 (from cpu.py /
 * gpu.py), the QED samplers bound at particles.py:8-12, the field launcher
 * Fields.field_func (fields.py:26-49, called at particles.py:310-323) and the
 * step loop Simulation.start (simulation.py:74-160).
 */
#ifndef SFP_H
#define SFP_H
#include <stddef.h>
#include <stdint.h>

#include "sfp_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SFP_OK 0
#define SFP_EINVAL (-1)   /* bad argument                                  */
#define SFP_ECUDA (-2)    /* CUDA runtime error                            */
#define SFP_ENVRTC (-3)   /* NVRTC compilation failed (log returned)       */
#define SFP_ENOMEM (-4)   /* device allocation failed                      */
#define SFP_EDEVICE (-5)  /* device-side error word set (see sfp_run_state) */
#define SFP_ENOKERNEL (-6) /* kernel not found in a module                  */

/* ---- library ------------------------------------------------------------- */
const char *sfp_version(void);
const char *sfp_last_error(void);
int sfp_device_count(int *count);
/* free a buffer returned by this library (NVRTC image / log) */
void sfp_free(void *p);

/* ---- field programs (NVRTC) ------------------------------------------------
 * Replaces Fields.__init__'s jitting of a user/preset callable
 * (fields.py:26-50): `src` is CUDA C++ defining sfp_field_program() followed
 * by the step source.  Compiles for sm_100a to a cubin image; needs no GPU. */
int sfp_nvrtc_compile(const char *src, const char *name, const char *const *opts, int n_opts, void **image,
                      size_t *image_size, char **log);
typedef struct sfp_module sfp_module;
int sfp_module_load(const void *image, size_t image_size, sfp_module **out);
int sfp_module_unload(sfp_module *m);

/* Fields.field_func[bpg, tpb](x, y, z, t, N, to_be_pruned, Ex..Bz)
 * (fields.py:31-35 / 41-46, particles.py:310-323).  params: the program's
 * term parameters (device). */
int sfp_field_eval(sfp_module *m, const double *params, const double *x, const double *y, const double *z, double t,
                   int64_t N, const uint8_t *to_be_pruned, double *Ex, double *Ey, double *Ez, double *Bx, double *By,
                   double *Bz, void *stream);

/* ---- per-op kernels: the reference's plugin boundary ----------------------- */
/* push_position, cpu.py:5-19 */
int sfp_push_position(double *x, double *y, double *z, const double *ux, const double *uy, const double *uz,
                      const double *inv_gamma, int64_t N, const uint8_t *to_be_pruned, double dt, void *stream);
/* boris, cpu.py:22-31 (inline.py:4-36) */
int sfp_boris(double *ux, double *uy, double *uz, double *inv_gamma, const double *Ex, const double *Ey,
              const double *Ez, const double *Bx, const double *By, const double *Bz, double q, int64_t N,
              const uint8_t *to_be_pruned, double dt, void *stream);
/* boris_tbmt, cpu.py:33-42 (inline.py:39-100) */
int sfp_boris_tbmt(double *ux, double *uy, double *uz, double *inv_gamma, double *sx, double *sy, double *sz,
                   const double *Ex, const double *Ey, const double *Ez, const double *Bx, const double *By,
                   const double *Bz, double q, double ae, int64_t N, const uint8_t *to_be_pruned, double dt,
                   void *stream);
/* LL_push / CLL_push, cpu.py:44-60 (inline.py:104-123) */
int sfp_LL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi, int64_t N,
                const uint8_t *to_be_pruned, double dt, void *stream);
int sfp_CLL_push(double *ux, double *uy, double *uz, double *inv_gamma, const double *chi, int64_t N,
                 const uint8_t *to_be_pruned, double dt, void *stream);
/* update_chi, cpu.py:62-74 (inline.py:126-134) */
int sfp_update_chi(const double *Ex, const double *Ey, const double *Ez, const double *Bx, const double *By,
                   const double *Bz, const double *ux, const double *uy, const double *uz, const double *inv_gamma,
                   double *chi, int64_t N, const uint8_t *to_be_pruned, void *stream);
/* photon_recoil, cpu.py:76-87 */
int sfp_photon_recoil(double *ux, double *uy, double *uz, double *inv_gamma, const uint8_t *event,
                      const double *photon_delta, int64_t N, const uint8_t *to_be_pruned, void *stream);
/* pick_hard_photon, cpu.py:226-231 */
int sfp_pick_hard_photon(uint8_t *event, const double *delta, const double *inv_gamma, double threshold, int64_t N,
                         void *stream);
/* bool_sum, cpu.py:217-224: count written to *count (device int64) */
int sfp_bool_sum(const uint8_t *event, int64_t N, int64_t *count, void *stream);
/* find_event_index, cpu.py:192-215: ascending indices of the N_event set
 * entries of event[0:N], into index (device int64[N_event]).  workspace:
 * caller-provided device scratch of sfp_find_event_index_workspace(N) bytes. */
size_t sfp_find_event_index_workspace(int64_t N);
int sfp_find_event_index(const uint8_t *event, int64_t N_event, int64_t N, int64_t *index, void *workspace,
                         size_t workspace_bytes, void *stream);
/* find_event_index without a workspace and without any allocation.  No
 * counterpart in the reference: for callers that cannot allocate device
 * memory on demand (memory owned by a pool or caching allocator sized at
 * start-up; code that must not stall, as cudaMalloc / cudaFree synchronise
 * the device).  Same result as sfp_find_event_index.  Its scratch is a fixed
 * 512 KiB array in the library's device image, held on every GPU that loads
 * the library until exit, so N <= SFP_FEI_NOALLOC_MAX_N (2^28); larger N is
 * rejected with SFP_EINVAL.  The first call with a device current looks up
 * that device's scratch address (a call with N = 0 does only this); make it
 * before any stream capture.  The address is kept for the life of the
 * process: after cudaDeviceReset (or any end of the device's primary
 * context) this entry point must not be called on that device again.
 * Calls in flight at once on one device (other streams or threads) share
 * the scratch and race. */
#define SFP_FEI_NOALLOC_MAX_N (1LL << 28)
int sfp_find_event_index_noalloc(const uint8_t *event, int64_t N_event, int64_t N, int64_t *index, void *stream);
/* create_photon, cpu.py:89-116 */
int sfp_create_photon(const double *x_src, const double *y_src, const double *z_src, const double *ux_src,
                      const double *uy_src, const double *uz_src, double *x_dst, double *y_dst, double *z_dst,
                      double *ux_dst, double *uy_dst, double *uz_dst, double *inv_gamma_dst,
                      uint8_t *photon_to_be_pruned, const int64_t *event_index, const double *photon_delta,
                      int64_t N_buffered, int64_t N_photon, void *stream);
/* create_pair, cpu.py:119-189 */
int sfp_create_pair(const double *x_src, const double *y_src, const double *z_src, const double *ux_src,
                    const double *uy_src, const double *uz_src, uint8_t *photon_to_be_pruned, double *x_dst,
                    double *y_dst, double *z_dst, double *ux_dst, double *uy_dst, double *uz_dst,
                    double *inv_gamma_dst, uint8_t *pair_to_be_pruned, const int64_t *event_index,
                    const double *pair_delta, int64_t N_buffered, int64_t N_pair, int inverse_delta, void *stream);
/* photon_from_rejection_sampling / pair_from_rejection_sampling,
 * qed/rejection_sampling.py:73-107.  The reference draws from Numba's
 * per-thread generator; here draws are Philox-4x32-10 keyed by
 * (seed, rng_stream, step, slot). */
int sfp_photon_from_rejection_sampling(const double *inv_gamma, const double *chi_e, double dt, int64_t N,
                                       const uint8_t *to_be_pruned, uint8_t *event, double *delta,
                                       const sfp_rs_table *table, uint64_t seed, uint32_t rng_stream, uint32_t step,
                                       void *stream);
int sfp_pair_from_rejection_sampling(const double *inv_gamma, const double *chi_gamma, double dt, int64_t N,
                                     const uint8_t *to_be_pruned, uint8_t *event, double *delta,
                                     const sfp_rs_table *table, uint64_t seed, uint32_t rng_stream, uint32_t step,
                                     void *stream);
/* update_tau_e / update_tau_gamma, qed/optical_depth.py:15-111 */
int sfp_update_tau(double *tau, const double *inv_gamma, const double *chi, double dt, int64_t N,
                   const uint8_t *to_be_pruned, uint8_t *event, double *delta, const sfp_od_table *table,
                   uint64_t seed, uint32_t rng_stream, uint32_t step, void *stream);
/* inv_gamma from u for a whole buffer (particles.py:119 / 122), used to
 * refresh the stored 1/gamma after fused steps, which keep only x and u. */
int sfp_inv_gamma(const double *ux, const double *uy, const double *uz, double *inv_gamma, int64_t N, int massless,
                  void *stream);

/* ---- fused step: Simulation.start (simulation.py:74-160) -------------------
 * A run owns the device bookkeeping of one or more instances whose species
 * buffers are described by segments (device pointers owned by the caller). */
typedef struct sfp_run sfp_run;
typedef struct sfp_run_config {
    double dt;
    double photon_threshold; /* Simulation(photon_threshold=...), units of m_e c^2 */
    double t0;
    int64_t step0;           /* steps already taken (Philox step key)     */
    int32_t qed;             /* SFP_QED_*                                  */
    int32_t form;            /* SFP_FORM_*                                 */
    int32_t m_stages;        /* massive kernel: depth of the copy ring, 2..4 (0 = default)  */
    int32_t min_blocks;      /* massive kernel: min resident blocks per SM (0 = default)    */
    int32_t p_stages;        /* photon kernel: depth of the copy ring, 2..4 (0 = default)   */
    int32_t p_min_blocks;    /* photon kernel: min resident blocks per SM (0 = default)     */
    const float *mlp_params; /* optical depth: the learned photon-energy sampler's 8577
                                parameters (device), or NULL for the table sampler      */
    sfp_rs_table rs;
    sfp_od_table od_photon;
    sfp_od_table od_pair;
} sfp_run_config;

/* A step module compiled with SFP_CONST_FIELD_N (a module for runs of one
 * instance) holds the field parameters in its constant bank: a run on it
 * must have n_inst == 1, and each sfp_run_steps / sfp_run_steps_timed /
 * sfp_run_resume call first copies inst[0].field_params (SFP_CONST_FIELD_N
 * doubles), and the Philox round keys of inst[0].seed, there on the run's
 * stream, after the launches of the previous
 * call made on the same module by any run.  Calls on one module from
 * several host threads are serialised.  Other modules read each instance's
 * parameters from global memory. */
int sfp_run_create(sfp_module *m, const sfp_run_config *cfg, int n_inst, const sfp_instance *inst, int n_seg,
                   const sfp_segment *seg, const int64_t *n_buffered, sfp_run **out);
/* after buffers were regrown / moved: new segment table and counts
 * (n_buffered NULL keeps the device's counts) */
int sfp_run_update(sfp_run *r, int n_seg, const sfp_segment *seg, const int64_t *n_buffered);
/* advance up to nsteps steps; graph_chunk > 0 replays CUDA graphs of that
 * many steps.  Asynchronous on `stream`.  The run stops early with halted=1
 * inside a step, once its photon and pair events are counted, when a
 * destination lacks room for that step's children (appends_pending=1): grow
 * every segment to sfp_run_pending_need (the reference's _extend rule),
 * sfp_run_update with NULL counts, then sfp_run_resume to finish that step.
 * The steps queued behind it do nothing. */
int sfp_run_steps(sfp_run *r, int64_t nsteps, int graph_chunk, void *stream);
/* like sfp_run_steps without graphs, with CUDA events recorded around the
 * kernels of every step on the run's stream; synchronous.
 * kernel_ms[3*i + k] is the duration of step i's massive (k=0) and photon
 * (k=1) kernels and of its scan + appends kernels (k=2); 0 for kernels the
 * run does not launch (3*nsteps entries). */
int sfp_run_steps_timed(sfp_run *r, int64_t nsteps, float *kernel_ms, void *stream);
/* Photon positions are stored as of the run's position epoch: the step
 * kernels advance a photon's position in registers (photons fly straight,
 * one push per step) and store nothing for a photon that does not convert.
 * This writes every photon segment's positions out as of the current step
 * (alive photons, and photons marked inside a step stopped for room) and
 * moves the epoch there; asynchronous on `stream`.  Call it before reading
 * photon x, y, z from the device, and before sfp_run_destroy when the
 * arrays live on.  Momenta, flags, tau and every massive species are always
 * current.  No counterpart in the reference, whose photon push
 * (cpu.py:5-19) writes every step. */
int sfp_run_sync_positions(sfp_run *r, void *stream);
/* synchronous: state and per-segment buffered counts (n_seg entries) */
int sfp_run_read_state(sfp_run *r, sfp_run_state *state, int64_t *n_buffered, void *stream);
/* clear a halted flag that no stopped step holds */
int sfp_run_clear_halt(sfp_run *r, void *stream);
/* synchronous: while appends_pending, the buffer size each segment needs to
 * finish the stopped step (n_seg entries); otherwise its buffered count */
int sfp_run_pending_need(sfp_run *r, int64_t *need);
/* finish a step stopped with appends_pending: write and push its children,
 * fold its appends and advance t / step.  Asynchronous on the run's stream. */
int sfp_run_resume(sfp_run *r, void *stream);
int sfp_run_destroy(sfp_run *r);

/* ---- learned photon-energy sampler (no counterpart in the reference) ------
 * An MLP (log10 chi, u) -> delta, 2 -> 64 -> 64 -> 64 -> 1 with SiLU, that can
 * stand in for the optical-depth method's inverse-CDF table sampler
 * (_bisect_interp, qed/optical_depth_tables.py:59-102).  Parameters: 8577
 * float32, W0[64][2] b0[64] W1[64][64] b1[64] W2[64][64] b2[64] W3[64] b3.
 * Features (log10 chi / 3, log(u / (1 - u)) / 8); output y, delta =
 * 10^(3 (y - 1)) clamped to [1e-6, 1]. */
#define SFP_MLP_HIDDEN 64
#define SFP_MLP_NPARAM 8577
/* the table sampler, batched: delta[i] = _bisect_interp at chi = 10^log_chi[i], u[i] */
int sfp_od_inverse_cdf(const sfp_od_table *table, const double *log_chi, const double *u, double *delta, int64_t N,
                       void *stream);
/* N training samples: log10 chi ~ U[lo, hi]; u ~ U(0,1) for 3 in 4 samples and
 * 1 - u log-uniform in [1e-8, 0.1] for the rest (Philox(seed, chunk));
 * features[2i], features[2i+1] as above, targets[i] = log10(table delta) / 3 + 1 */
int sfp_mlp_make_samples(const sfp_od_table *table, uint64_t seed, uint32_t chunk, double log_chi_lo,
                         double log_chi_hi, int64_t N, float *features, float *targets, void *stream);
/* adds to grad (8577 floats) the gradient of sum_i (y_i - targets_i)^2 with
 * respect to the BF16-rounded weights, and that sum to *loss (device double) */
int sfp_mlp_grad(const float *params, const float *features, const float *targets, int64_t N, float *grad,
                 double *loss, void *stream);
/* one Adam step (step counts from 1) with gradient grad * grad_scale */
int sfp_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t step, float lr, float beta1,
                 float beta2, float eps, float grad_scale, void *stream);
/* batched inference on the tensor cores (BF16 weights, FP32 accumulation):
 * tcgen05.mma chains on 128-query tiles with the accumulators in tensor
 * memory.  A wait on the tensor cores that gives up sets a device error
 * flag (sfp_mlp_device_error) and leaves the rest of the batch unwritten. */
int sfp_mlp_infer(const float *params, const double *log_chi, const double *u, double *delta, int64_t N,
                  void *stream);
/* the same network on warp-level mma.sync tiles of 16 queries, the form the
 * fused step uses for a warp's few emission events */
int sfp_mlp_infer_warp(const float *params, const double *log_chi, const double *u, double *delta, int64_t N,
                       void *stream);
/* synchronous: 1 if an sfp_mlp_infer launch on the current device gave up
 * waiting for its tensor cores since the last call, else 0; clears it */
int sfp_mlp_device_error(int *code);
/* test hook of that failure path: sfp_mlp_infer with every MMA and commit
 * withheld, so each block's first wait runs out (after one second), sets the
 * flag, frees its tensor memory and returns; delta is left unwritten */
int sfp_mlp_infer_withheld(const float *params, const double *log_chi, const double *u, double *delta, int64_t N,
                           void *stream);

/* The per-chi-bin upper bound of the rejection-sampling pair rate
 * (qed/rejection_sampling_tables.py:56-78) over every delta, that the fused
 * step's photon kernel uses to skip pair tests no draw can pass: out[k] for
 * the chi of bin k (SFP_PAIR_BOUND_BINS = 256 bins: the float's exponent and
 * 3 mantissa bits from chi = 2^-16; bin 0 takes every smaller chi, the last
 * bin every larger one and is +inf), 4 times the tables' interval maxima
 * from (4/chi)^(2/3) on.  No counterpart in the reference: exposed so that
 * tests and tools can check the bound.  out: 256 floats on the device. */
int sfp_pair_rate_bound(const double *int_ai, const double *aip, int z_n, double z_max, float *out, void *stream);

/* ---- QED rate tables generated on the GPU --------------------------------
 * The reference's table generators (qed/rejection_sampling_tables.py:80-112,
 * qed/optical_depth_tables.py:136-198, scipy airy + quad) restated with the
 * same quadrature algorithm (QUADPACK QAGS / QAGI as scipy.integrate.quad
 * runs them, its default tolerances) so the entries agree with the
 * reference's.  Grids and the rate prefactor (-alpha m c^2 / hbar for
 * photons, +alpha m c^2 / hbar for pairs) are the caller's, on the device.
 * rejection sampling: int_ai[i] = integral_{z_i}^inf Ai, aip[i] = Ai'(z_i) */
int sfp_table_rs(const double *z, int64_t n, double *int_ai, double *aip, void *stream);
/* optical depth, kind 0 photon emission / 1 pair creation: per chi row the
 * total rate and the cumulative row over the delta grid (n_chi x n_delta,
 * row-major); first: n_chi doubles of device scratch (the rows' first
 * entries) */
int sfp_table_od(int kind, double factor, const double *chi, int64_t n_chi, const double *delta, int64_t n_delta,
                 double *total, double *cumulative, double *first, void *stream);

#ifdef __cplusplus
}
#endif
#endif
