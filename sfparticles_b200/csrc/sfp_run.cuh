// sfp_run.cuh -- device-side layout of a fused-step run, shared by the host
// C-ABI (nvcc) and the NVRTC-compiled step modules.
//
// A step runs four kernels after the bookkeeping kernel:
//   massive   -- block tiles over the e+- (massive) segments: QED photon
//                emission, recoil, Boris push, photon children (ordered by
//                a decoupled look-back over the tiles);
//   photon    -- warp tiles over the photon segments: pair creation (the
//                converted photon is marked and its delta stored), photon
//                push; per-tile event counts, summed per super-tile of 64;
//   pair scan -- one block: exclusive scan of the super-tile counts;
//   pairs     -- e-/e+ children of the marked photons, in index order, pushed.
// Photon-segment tile ranges start at multiples of 64 tiles, so a
// super-tile never spans two segments.
#pragma once
#include "sfp_types.h"

struct sfp_step_state {
    double t;                   // time of the prepared / running step
    long long step;             // steps completed
    long long n_mtiles;         // massive-group tiles of the prepared step
    long long n_ptiles;         // photon-group tiles
    int mticket;                // next massive tile to hand out
    int pticket;                // next photon tile to hand out
    int skip;                   // 1: the prepared step must not run
    int halted;                 // sticky: capacity guard tripped (host regrows, resets)
    int error;                  // sticky device error (SFP_DEV_*)
    unsigned int epoch;         // look-back flag epoch of the prepared step
    int pending;                // a prepared step awaits folding
    int pair_wait;              // the prepared step stopped before writing its pairs (no room)
    long long particle_steps;   // sum over executed steps of all N_buffered
};

struct sfp_run_dev {
    const sfp_segment* seg;
    const sfp_instance* inst;
    int n_seg;
    int n_inst;
    double dt;
    double photon_threshold;
    int qed;                    // SFP_QED_*
    int mtile;                  // particles per massive tile (256 * items)
    int ptile;                  // photons per photon (warp) tile
    int any_appends;            // some massive segment radiates (the massive look-back runs)
    int n_mseg;                 // massive segments (instance order)
    int n_pseg;                 // photon segments
    int n_cseg;                 // segments receiving pair children
    int pad;
    const int* mseg;            // [n_mseg] segment indices
    const int* pseg;            // [n_pseg]
    const int* cseg;            // [n_cseg]
    sfp_rs_table rs;
    sfp_od_table od_photon;
    sfp_od_table od_pair;
    long long* n_buffered;        // [n_seg] authoritative buffered counts
    unsigned long long* appended; // [n_seg] children appended by the running step
    long long* n_buf_step;        // [n_seg] counts at the start of the running step
    long long* mtile_start;       // [n_mseg + 1]
    long long* ptile_start;       // [n_pseg + 1]
    long long* chain_first;       // [n_seg] first massive tile of the segment's chain
    long long max_ptiles;
    unsigned int* ptile_cnt;      // [max_ptiles] pair events per photon tile
    unsigned int* psuper_cnt;     // [max_ptiles / 64 + 1] pair events per super-tile
    long long* psuper_pre;        // [max_ptiles / 64 + 1] exclusive prefix in its chain
    int ring_off;                 // photon kernel: byte offset of the copy ring in dynamic smem
    int mlp_off;                  // massive kernel: byte offset of the network weights in dynamic smem
    const float* mlp_params;      // learned photon-energy sampler (optical depth), or NULL: the table
    long long max_tiles;
    unsigned int* tile_flag;      // [max_tiles] (epoch << 2) | status
    uint4* tile_agg;              // [max_tiles] per-channel tile counts
    uint4* tile_incl;             // [max_tiles] per-channel inclusive prefixes
    sfp_step_state* st;
};
