// sfp_run.cuh -- device-side layout of a fused-step run, shared by the host
// C-ABI (nvcc) and the NVRTC-compiled step modules.
#pragma once
#include "sfp_types.h"

struct sfp_step_state {
    double t;            // time of the prepared / running step
    long long step;      // steps completed
    long long n_tiles;   // tiles of the prepared step
    int ticket;          // next tile to hand out
    int skip;            // 1: the prepared step must not run
    int halted;          // sticky: capacity guard tripped (host regrows, resets)
    int error;           // sticky device error (SFP_DEV_*)
    unsigned int epoch;  // look-back flag epoch of the prepared step
    int pending;         // a prepared step awaits folding
    long long particle_steps;  // sum over executed steps of all N_buffered
};

struct sfp_run_dev {
    const sfp_segment* seg;
    const sfp_instance* inst;
    int n_seg;
    int n_inst;
    double dt;
    double photon_threshold;
    int qed;              // SFP_QED_*
    int tile;             // particles per tile (= block size)
    int any_appends;      // some segment radiates or creates pairs
    int pad;
    sfp_rs_table rs;
    sfp_od_table od_photon;
    sfp_od_table od_pair;
    long long* n_buffered;        // [n_seg] authoritative buffered counts
    unsigned long long* appended; // [n_seg] children appended by the running step
    long long* n_buf_step;        // [n_seg] counts at the start of the running step
    long long* tile_start;        // [n_seg + 1]
    long long max_tiles;
    unsigned int* tile_flag;      // [max_tiles] (epoch << 2) | status
    uint4* tile_agg;              // [max_tiles] per-channel tile counts
    uint4* tile_incl;             // [max_tiles] per-channel inclusive prefixes
    sfp_step_state* st;
};
