// sfp_run.cuh -- device-side layout of a fused-step run, shared by the host
// C-ABI (nvcc) and the NVRTC-compiled step modules.
//
// A step runs four kernels after the bookkeeping kernel:
//   massive -- warp tiles over the e+- (massive) segments, streamed through
//              a ring of asynchronous copies: QED photon emission at t; an
//              emitter is marked (pruned = 2) with its delta stored and is
//              left unpushed, every other particle is pushed to t+dt;
//              per-tile emission counts, summed per super-tile of 64;
//   photon  -- warp tiles over the photon segments: pair creation (the
//              converted photon is marked and its delta stored), photon
//              push; per-tile event counts, summed per super-tile;
//   scan    -- one block: exclusive scans of both groups' super-tile counts
//              (segmented by instance, per append channel), the step's
//              append counts, and the exact room check of every destination;
//   appends -- photon children of the marked emitters (then their recoil
//              and push) and e-/e+ children of the marked photons (pushed),
//              each written at the slot the reference's find_event_index +
//              create_* gives it.
// Both groups' segments start at multiples of 64 tiles, so a super-tile
// never spans two segments.  No kernel waits on another block: there is no
// spin-wait anywhere in a step.
#pragma once
#include "sfp_types.h"

// Tile length.  Each step the bookkeeping kernel gives each group the
// shortest power-of-two tile from SFP_TILE_MIN to SFP_TILE_MAX particles
// that cuts its population into at most SFP_TILE_TARGET tiles: a large
// population keeps 1024-particle tiles (32 sub-steps of the copy ring per
// ticket), a small one is spread over every warp of the grid instead of
// running a few long tiles serially.  Results do not depend on the tile:
// draws are keyed by particle index and children are written in index
// order.  The tile counters hold SFP_TILE_TARGET tiles plus the segments'
// padding at least, so the rule always fits.
#define SFP_TILE_MIN 32
#define SFP_TILE_MAX 1024
#define SFP_TILE_TARGET 4096

struct sfp_step_state {
    double t;                   // time of the prepared / running step
    long long step;             // steps completed
    long long n_mtiles;         // massive-group tiles of the prepared step
    long long n_ptiles;         // photon-group tiles
    int mticket;                // next massive tile to hand out
    int pticket;                // next photon tile to hand out
    int skip;                   // 1: the prepared step must not run
    int halted;                 // sticky: a destination lacked room (host regrows, resumes)
    int error;                  // sticky device error (SFP_DEV_*)
    int mtile;                  // particles per massive-group tile of the prepared step
    int pending;                // a prepared step awaits folding
    int append_wait;            // the prepared step stopped before writing its children (no room)
    int ptile;                  // particles per photon-group tile of the prepared step
    int pad0;
    long long particle_steps;   // sum over executed steps of all N_buffered
    // Photons fly straight: a photon segment stores each position as of the
    // start of step pos_epoch, and the photon at the start of step `step`
    // is at stored + (step - pos_epoch) * (its one-step displacement).  The
    // step kernels advance positions in registers only; sfp_sync_positions
    // writes them out and moves pos_epoch to step.
    long long pos_epoch;
};

// one group of tiles (massive or photon): the tile map of its segments and
// its per-tile / per-super-tile event counts
struct sfp_group_dev {
    const int* seg;             // [n_seg] segment indices, in segment order
    long long* tile_start;      // [n_seg + 1] first tile of each segment (multiples of 64)
    unsigned int* tile_cnt;     // [max_tiles] events per tile
    unsigned int* super_cnt;    // [max_tiles / 64 + 2] events per super-tile
    long long* super_pre;       // [max_tiles / 64 + 2] exclusive prefix in its instance, per channel
    long long max_tiles;
    int n_seg;
    int pad;
};

struct sfp_run_dev {
    const sfp_segment* seg;
    const sfp_instance* inst;
    int n_seg;
    int n_inst;
    double dt;
    double photon_threshold;
    int qed;                    // SFP_QED_*
    int pad_tile;
    int any_rad;                // some massive segment radiates
    int any_bw;                 // some photon segment creates pairs
    int n_dseg;                 // segments receiving children (photons or pairs)
    int m_ring_off;             // massive kernel: byte offset of its copy ring in dynamic smem
    int m_stage_bytes;          // massive kernel: bytes per ring stage (the run's widest segment layout)
    int ring_off;               // photon kernel: byte offset of its copy ring in dynamic smem
    int mlp_off;                // massive kernel: byte offset of the network weights in dynamic smem
    int pad1;
    const int* dseg;            // [n_dseg]
    sfp_group_dev mg;           // massive group
    sfp_group_dev pg;           // photon group
    sfp_rs_table rs;
    sfp_od_table od_photon;
    sfp_od_table od_pair;
    long long* n_buffered;        // [n_seg] authoritative buffered counts
    unsigned long long* appended; // [n_seg] children appended by the running step
    long long* n_buf_step;        // [n_seg] counts at the start of the running step
    const float* mlp_params;      // learned photon-energy sampler (optical depth), or NULL: the table
    sfp_step_state* st;
    // rejection sampling: per chi bin an upper bound of the pair rate over
    // every delta (SFP_PAIR_BOUND_BINS floats, the bins of sfp_pair_bin), so
    // photons whose pair test no draw can pass skip the draw
    const float* pair_bound;
};

// chi bins of the pair-rate bound: the float's exponent and 3 mantissa bits
// from chi = 2^-16 up; bin 0 also holds every smaller chi, the last bin
// (bound +inf) every larger one
#define SFP_PAIR_BOUND_BINS 256
#define SFP_PAIR_BOUND_BASE ((127 - 16) << 3)
SFP_DEVICE_INLINE int sfp_pair_bin(float chi) {
    int k = (int)(__float_as_uint(chi) >> 20) - SFP_PAIR_BOUND_BASE;
    return k < 0 ? 0 : (k > SFP_PAIR_BOUND_BINS - 1 ? SFP_PAIR_BOUND_BINS - 1 : k);
}
