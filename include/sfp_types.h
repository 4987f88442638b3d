/*
 * sfp_types.h -- plain-C data layouts shared by the host C-ABI (libsfp.so),
 * its callers (ctypes), and the device code (nvcc- and NVRTC-compiled).
 *
 * No includes: integer widths are spelled with C99 names when <stdint.h> is
 * available and with builtin types under NVRTC.
 */
#ifndef SFP_TYPES_H
#define SFP_TYPES_H

#if defined(__CUDACC_RTC__)
typedef long long sfp_i64;
typedef unsigned long long sfp_u64;
typedef int sfp_i32;
typedef unsigned int sfp_u32;
typedef unsigned char sfp_u8;
#else
#include <stdint.h>
typedef int64_t sfp_i64;
typedef uint64_t sfp_u64;
typedef int32_t sfp_i32;
typedef uint32_t sfp_u32;
typedef uint8_t sfp_u8;
#endif

/* radiation reaction types, values of the reference's RadiationReactionType
 * enum (particles.py:27-40: NONE=1, PHOTON=2, LL=3, CLL=4) */
#define SFP_RR_NONE 1
#define SFP_RR_PHOTON 2
#define SFP_RR_LL 3
#define SFP_RR_CLL 4

/* QED event generators */
#define SFP_QED_REJECTION 0    /* qed/rejection_sampling.py (default)  */
#define SFP_QED_OPTICAL_DEPTH 1 /* qed/optical_depth.py                  */

/* arithmetic forms of the fused step */
#define SFP_FORM_FP64 0  /* plain float64, the reference's arithmetic        */
#define SFP_FORM_FP32 1  /* float32 arithmetic on float64 state: float32
                            increments accumulated in float64, float64
                            gamma when gamma>1e4, float64 optical depth      */

#define SFP_MAX_CHANNELS 4  /* distinct append destinations per instance */
#define SFP_FIELD_PARAMS 16 /* doubles per preset term; each preset's layout
                               is written by sfparticles_b200/fields.py (the
                               Gaussian pulse: slots 0-9 its float64
                               parameters, 10-15 float32 constants for the
                               float32 form, two per slot)                    */

/* One particle species of one collision instance: the reference's Particles
 * attribute arrays (particles.py:87-146) as device pointers. */
typedef struct sfp_segment {
    double *x, *y, *z, *ux, *uy, *uz;
    double *sx, *sy, *sz; /* NULL unless spin (SpinParticles)              */
    double *tau;          /* NULL unless the optical-depth method is used  */
    double *delta;        /* the delta of this step's events: photon_delta
                             of a radiating species, pair_delta of a
                             pair-creating one (NULL otherwise)             */
    sfp_u8 *pruned;       /* _to_be_pruned                                 */
    sfp_i64 capacity;     /* buffer_size                                   */
    double q;             /* charge [C]                                    */
    double ae;            /* anomalous magnetic moment (spin only)         */
    sfp_i32 massless;     /* photon species                                */
    sfp_i32 push;         /* member of Simulation.particles_push           */
    sfp_i32 rr;           /* SFP_RR_*                                      */
    sfp_i32 spin;
    sfp_i32 radiating;    /* emits photons into photon_dest                */
    sfp_i32 bw;           /* creates pairs into ele_dest / pos_dest        */
    sfp_i32 photon_dest;  /* segment index, or -1                          */
    sfp_i32 ele_dest;
    sfp_i32 pos_dest;
    sfp_i32 channel;      /* append channel its children use (0..3)        */
    sfp_i32 instance;     /* owning instance                               */
    sfp_u32 stream;       /* Philox stream id (species index in the run)   */
} sfp_segment;

/* One collision instance: its own RNG key and field parameters. */
typedef struct sfp_instance {
    sfp_u64 seed;
    const double *field_params; /* [n_terms * SFP_FIELD_PARAMS], 16-byte aligned */
    sfp_i32 first_seg;
    sfp_i32 n_seg;
} sfp_instance;

/* Optical-depth tables (qed/optical_depth_tables.py layout). */
typedef struct sfp_od_table {
    const double *rate_total; /* [chi_N]            */
    const double *cumulative; /* [chi_N][delta_N]   */
    sfp_i32 chi_N;
    sfp_i32 delta_N;
    double log_chi_min;
    double log_chi_delta;
    double log_chi_max;
    double log_delta_min;
    double log_delta_delta;
} sfp_od_table;

/* Rejection-sampling tables (qed/rejection_sampling_tables.py layout). */
typedef struct sfp_rs_table {
    const double *int_Ai; /* [z_N] integral of Ai from z to infinity */
    const double *Aip;    /* [z_N] Ai'(z)                             */
    sfp_i32 z_N;
    sfp_i32 pad;
    double z_max;
} sfp_rs_table;

/* Host-visible snapshot of a run (sfp_run_read_state); per-segment buffered
 * counts are returned through a separate array. */
typedef struct sfp_run_state {
    double t;               /* time of the next step                        */
    sfp_i64 step;           /* steps completed                              */
    sfp_i32 halted;         /* 1: the run stopped for lack of capacity      */
    sfp_i32 error;          /* device error code (0 = none)                 */
    sfp_i64 particle_steps; /* sum over executed steps of all N_buffered    */
    sfp_i32 appends_pending; /* 1: a step stopped before writing its
                               children (photons or pairs) for lack of room:
                               grow to sfp_run_pending_need, then
                               sfp_run_resume                               */
    sfp_i32 pad;
} sfp_run_state;

#define SFP_MAX_SEGMENTS 4096

/* device error codes */
#define SFP_DEV_OK 0
#define SFP_DEV_CAPACITY 2 /* more tiles than the run's counters hold */
#define SFP_DEV_TILE 3     /* a long-tile kernel met a step planned with shorter tiles */

#endif
