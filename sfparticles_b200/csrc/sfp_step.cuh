// sfp_step.cuh -- the fused particle step (one launch advances every species
// of every instance by one step) plus its bookkeeping kernel.
//
// Compiled by NVRTC together with a generated field program that defines
//     SFP_DEVICE_INLINE void sfp_field_program(double x, double y, double z,
//                                              double t, const double* P, double F[6]);
// so the field expression is inlined into the push.
//
// Semantics follow simulation.py:102-144 exactly:
//   1. fields at t for pushed species (particles.py:299-323),
//   2. chi + pair events for photon species (QED at t),
//   3. chi + photon events + hard-photon filter for e+- species,
//   4. photons appended (e- species first, in buffer order), recoil,
//   5. pairs appended, converted photons pruned,
//   6. every pushed particle -- children included -- pushed from t to t+dt:
//      half position, fields at t+dt/2, Boris / Boris-TBMT (+LL/CLL), half position.
// Appends are ordered: a block-wide scan plus a decoupled look-back across
// tiles gives each child the slot the reference's find_event_index + create_*
// would give it, so Philox streams keyed by slot are reproducible.
#pragma once
#include "sfp_device.cuh"
#include "sfp_device32.cuh"
#include "sfp_run.cuh"

#ifndef SFP_TILE
#define SFP_TILE 256
#endif
#define SFP_LOOKBACK_SPIN_LIMIT (1u << 24)

#define SFP_FLAG_AGG 1u
#define SFP_FLAG_INCL 2u

namespace sfp {

SFP_DEVICE_INLINE void st_release_u32(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
SFP_DEVICE_INLINE unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
SFP_DEVICE_INLINE uint4 ld_cg_u4(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}
SFP_DEVICE_INLINE void st_cg_u4(uint4* p, uint4 v) {
    asm volatile("st.global.cg.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}
SFP_DEVICE_INLINE unsigned int u4_get(const uint4& v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}
SFP_DEVICE_INLINE uint4 u4_one(int c, unsigned int n) {
    uint4 v{0u, 0u, 0u, 0u};
    if (c == 0) v.x = n;
    else if (c == 1) v.y = n;
    else if (c == 2) v.z = n;
    else v.w = n;
    return v;
}
SFP_DEVICE_INLINE uint4 u4_add(uint4 a, uint4 b) { return uint4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
SFP_DEVICE_INLINE uint4 warp_sum_u4(uint4 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
        v.w += __shfl_xor_sync(0xffffffffu, v.w, o);
    }
    return v;
}

// Decoupled look-back (Merrill & Garland, 2016) over the tiles of one
// instance, run by warp 0.  A tile publishes its aggregate (AGG) as soon as
// its events are known and its inclusive prefix (INCL) once the exclusive
// prefix is known; look-backs sum predecessors' AGGs until an INCL.
SFP_DEVICE_INLINE void publish(const sfp_run_dev* R, long long tile, uint4 v, unsigned int epoch, bool incl) {
    if ((threadIdx.x & 31) == 0) {
        st_cg_u4((incl ? R->tile_incl : R->tile_agg) + tile, v);
        st_release_u32(R->tile_flag + tile, (epoch << 2) | (incl ? SFP_FLAG_INCL : SFP_FLAG_AGG));
    }
}

// one window of 32 predecessors without waiting: true (and the exclusive
// prefix) when an INCL is reached through ready tiles only
SFP_DEVICE_INLINE bool lookback_try(const sfp_run_dev* R, long long tile, long long first_tile, unsigned int epoch,
                                    uint4& excl) {
    const int lane = threadIdx.x & 31;
    const long long p = tile - 1 - lane;
    const bool valid = p >= first_tile;
    unsigned int status = 0;
    if (valid) {
        const unsigned int f = ld_acquire_u32(R->tile_flag + p);
        if ((f >> 2) == epoch) status = f & 3u;
    }
    const unsigned int incl_mask = __ballot_sync(0xffffffffu, valid && status == SFP_FLAG_INCL);
    const unsigned int ready_mask = __ballot_sync(0xffffffffu, valid && status != 0u);
    if (!incl_mask) return false;
    const int k = __ffs(incl_mask) - 1;
    const unsigned int need = (k == 31) ? 0xffffffffu : ((1u << (k + 1)) - 1u);
    if ((ready_mask & need) != need) return false;
    uint4 v{0u, 0u, 0u, 0u};
    if (lane < k) v = ld_cg_u4(R->tile_agg + p);
    else if (lane == k) v = ld_cg_u4(R->tile_incl + p);
    excl = warp_sum_u4(v);
    return true;
}

// blocking look-back; every wait is bounded, and on timeout the run's error
// word is set and the tile still publishes so that no successor waits on it
SFP_DEVICE_INLINE uint4 lookback_wait(const sfp_run_dev* R, long long tile, long long first_tile, unsigned int epoch) {
    const int lane = threadIdx.x & 31;
    uint4 excl{0u, 0u, 0u, 0u};
    long long base = tile - 1;
    bool failed = false;
    while (base >= first_tile) {
        const long long p = base - lane;
        const bool valid = p >= first_tile;
        unsigned int status = 0;
        if (valid) {
            unsigned int spins = 0;
            while (true) {
                const unsigned int f = ld_acquire_u32(R->tile_flag + p);
                if ((f >> 2) == epoch && (f & 3u) != 0u) {
                    status = f & 3u;
                    break;
                }
                if (++spins > SFP_LOOKBACK_SPIN_LIMIT ||
                    ((spins & 255u) == 0u && *(volatile int*)&R->st->error != 0)) {
                    failed = true;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (__any_sync(0xffffffffu, failed)) {
            if (lane == 0) atomicExch(&R->st->error, SFP_DEV_LOOKBACK_TIMEOUT);
            return uint4{0u, 0u, 0u, 0u};
        }
        const unsigned int incl_mask = __ballot_sync(0xffffffffu, valid && status == SFP_FLAG_INCL);
        uint4 v{0u, 0u, 0u, 0u};
        if (incl_mask) {
            const int k = __ffs(incl_mask) - 1;
            if (lane < k) v = ld_cg_u4(R->tile_agg + p);
            else if (lane == k) v = ld_cg_u4(R->tile_incl + p);
            excl = u4_add(excl, warp_sum_u4(v));
            break;
        }
        if (valid) v = ld_cg_u4(R->tile_agg + p);
        excl = u4_add(excl, warp_sum_u4(v));
        base -= 32;
    }
    return excl;
}

// Push of one massive particle from t to t+dt (simulation.py:128-137 with
// particles.py:244-296 / 575-604).  x, u (and s) in/out.
SFP_DEVICE_INLINE void push_massive(double& x, double& y, double& z, double& ux, double& uy, double& uz, double& sx,
                                    double& sy, double& sz, const sfp_segment& S, const double* __restrict__ P,
                                    double t, double dt) {
    double ig = inv_gamma_massive(ux, uy, uz);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
    double F[6];
    sfp_field_program(x, y, z, t + 0.5 * dt, P, F);
    if (S.spin)
        ig = boris_tbmt(ux, uy, uz, sx, sy, sz, F, S.q, S.ae, dt);
    else
        ig = boris(ux, uy, uz, F, S.q, dt);
    if (S.rr == SFP_RR_LL || (S.rr == SFP_RR_CLL && !S.spin)) {
        const double chi = chi_of(F, ux, uy, uz, ig);
        ig = ll_push(ux, uy, uz, ig, chi, dt, S.rr == SFP_RR_CLL);
    }
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
}

SFP_DEVICE_INLINE void push_photon(double& x, double& y, double& z, double ux, double uy, double uz, double dt) {
    const double ig = inv_gamma_photon(ux, uy, uz);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
    push_position(x, y, z, ux, uy, uz, ig, 0.5 * dt);
}

// float32 form of push_massive: float32 increments, float64 accumulation.
SFP_DEVICE_INLINE void push_massive32(double& x, double& y, double& z, double& ux, double& uy, double& uz,
                                      double& sx, double& sy, double& sz, const sfp_segment& S,
                                      const double* __restrict__ P, double t, double dt) {
    const float hc = (float)(0.5 * kC * dt);
    float g = sfp32::gamma_of(ux, uy, uz, false);
    float fx = (float)ux, fy = (float)uy, fz = (float)uz;
    float a = hc / g;
    x += (double)(a * fx);
    y += (double)(a * fy);
    z += (double)(a * fz);
    float F[6];
    sfp_field_program32(x, y, z, t + 0.5 * dt, P, F);
    const float eps = (float)((S.q * dt) / ((2.0 * kMe) * kC));
    const float bq = (float)((S.q * dt) / (2.0 * kMe));
    const float ex = eps * F[0], ey = eps * F[1], ez = eps * F[2];
    const float umx = fx + ex, umy = fy + ey, umz = fz + ez;
    float gm;
    if (g < (float)sfp32::kGammaSplit) {
        gm = sqrtf(1.0f + umx * umx + umy * umy + umz * umz);
    } else {
        const double dx = ux + (double)ex, dy = uy + (double)ey, dz = uz + (double)ez;
        gm = (float)sqrt(((1.0 + dx * dx) + dy * dy) + dz * dz);
    }
    const float igm = 1.0f / gm;
    if (S.spin) {  // inline.py:39-70: spin rotation with B_eff(u-), as an increment
        const float ae = (float)S.ae;
        const float uB = umx * F[3] + umy * F[4] + umz * F[5];
        const float a1 = ae + igm, a2 = ae * gm / (gm + 1.0f), a3 = ae + 1.0f / (gm + 1.0f);
        const float bex = a1 * F[3] - a2 * uB * umx - a3 * (umy * F[2] - umz * F[1]);
        const float bey = a1 * F[4] - a2 * uB * umy - a3 * (umz * F[0] - umx * F[2]);
        const float bez = a1 * F[5] - a2 * uB * umz - a3 * (umx * F[1] - umy * F[0]);
        const float Tx = bq * bex, Ty = bq * bey, Tz = bq * bez;
        const float f2 = 2.0f / (1.0f + Tx * Tx + Ty * Ty + Tz * Tz);
        const float s0x = (float)sx, s0y = (float)sy, s0z = (float)sz;
        const float spx = s0x + (s0y * Tz - s0z * Ty), spy = s0y + (s0z * Tx - s0x * Tz), spz = s0z + (s0x * Ty - s0y * Tx);
        sx += (double)(f2 * (spy * Tz - spz * Ty));
        sy += (double)(f2 * (spz * Tx - spx * Tz));
        sz += (double)(f2 * (spx * Ty - spy * Tx));
    }
    // Boris (inline.py:4-36) as u += 2 eps E + u' x S
    const float Tx = bq * F[3] * igm, Ty = bq * F[4] * igm, Tz = bq * F[5] * igm;
    const float upx = umx + (umy * Tz - umz * Ty), upy = umy + (umz * Tx - umx * Tz), upz = umz + (umx * Ty - umy * Tx);
    const float f2 = 2.0f / (1.0f + Tx * Tx + Ty * Ty + Tz * Tz);
    ux += (double)(2.0f * ex + f2 * (upy * Tz - upz * Ty));
    uy += (double)(2.0f * ey + f2 * (upz * Tx - upx * Tz));
    uz += (double)(2.0f * ez + f2 * (upx * Ty - upy * Tx));
    g = sfp32::gamma_of(ux, uy, uz, false);
    if (S.rr == SFP_RR_LL || (S.rr == SFP_RR_CLL && !S.spin)) {  // inline.py:104-123
        fx = (float)ux; fy = (float)uy; fz = (float)uz;
        const float chi = sfp32::chi_of(F, fx, fy, fz, g);
        float factor = (float)ll_factor(dt);
        if (S.rr == SFP_RR_CLL) {
            const float q = 1.0f + 4.8f * (1.0f + chi) * __logf(1.0f + 1.7f * chi) + 2.44f * chi * chi;
            factor *= exp2f(-0.66666667f * __log2f(q));
        }
        const float c = factor * chi * chi / g;
        ux += (double)(c * fx);
        uy += (double)(c * fy);
        uz += (double)(c * fz);
        g = sfp32::gamma_of(ux, uy, uz, false);
    }
    a = hc / g;
    x += (double)(a * (float)ux);
    y += (double)(a * (float)uy);
    z += (double)(a * (float)uz);
}

SFP_DEVICE_INLINE void push_photon32(double& x, double& y, double& z, double ux, double uy, double uz, double dt) {
    const float fx = (float)ux, fy = (float)uy, fz = (float)uz;
    const float a = (float)(kC * dt) * rsqrtf(fx * fx + fy * fy + fz * fz);
    x += (double)(a * fx);
    y += (double)(a * fy);
    z += (double)(a * fz);
}

}  // namespace sfp

#if defined(SFP_WANT_STEP)
// ---------------------------------------------------------------------------
// Bookkeeping: fold the appends of the step that ran, advance t, then (mode 1)
// prepare the next step: capacity guard, tile map, ticket, epoch.
// One block of 256 threads.
// ---------------------------------------------------------------------------
extern "C" __global__ void __launch_bounds__(256) sfp_book_kernel(const sfp_run_dev* __restrict__ R, int prepare) {
    __shared__ int s_bad;
    sfp_step_state* st = R->st;
    const int n = R->n_seg;
    if (st->pending) {
        for (int s = threadIdx.x; s < n; s += blockDim.x) {
            R->n_buffered[s] += (long long)R->appended[s];
            R->appended[s] = 0ull;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            st->t = st->t + R->dt;
            st->step += 1;
            st->pending = 0;
        }
    }
    __syncthreads();
    if (!prepare) return;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    if (st->halted || st->error) {
        if (threadIdx.x == 0) st->skip = 1;
        return;
    }
    // worst case appends per destination: every emitter emits, every photon converts
    for (int d = threadIdx.x; d < n; d += blockDim.x) {
        long long need = 0;
        const int inst = R->seg[d].instance;
        const int f = R->inst[inst].first_seg, l = f + R->inst[inst].n_seg;
        for (int s = f; s < l; ++s) {
            const sfp_segment& S = R->seg[s];
            if (S.radiating && S.photon_dest == d) need += R->n_buffered[s];
            if (S.bw && (S.ele_dest == d || S.pos_dest == d)) need += R->n_buffered[s];
        }
        if (R->n_buffered[d] + need > R->seg[d].capacity) atomicExch(&s_bad, 1);
    }
    __syncthreads();
    if (s_bad) {
        if (threadIdx.x == 0) {
            st->halted = 1;
            st->skip = 1;
        }
        return;
    }
    if (threadIdx.x == 0) {
        long long acc = 0, ps = 0;
        const long long T = R->tile;
        for (int s = 0; s < n; ++s) {
            R->tile_start[s] = acc;
            R->n_buf_step[s] = R->n_buffered[s];
            acc += (R->n_buffered[s] + T - 1) / T;
            ps += R->n_buffered[s];
        }
        R->tile_start[n] = acc;
        if (acc > R->max_tiles) {
            st->error = SFP_DEV_CAPACITY;
            st->skip = 1;
            return;
        }
        st->n_tiles = acc;
        st->ticket = 0;
        st->epoch = (unsigned int)((st->step + 1) & 0x3FFFFFFFll);
        if (st->epoch == 0u) st->epoch = 1u;
        st->skip = 0;
        st->pending = 1;
        st->particle_steps += ps;
    }
}

// ---------------------------------------------------------------------------
// The fused step.  Persistent grid; tiles of SFP_TILE * ITEMS particles are
// handed out in order; item k of thread j covers particle k*SFP_TILE + j of
// the tile, so the ordered append scans items k-major.
//
// Per tile:  load -> QED events -> publish the tile's append count (and try
// a non-blocking look-back) -> recoil + push every parent (registers) ->
// finish the look-back -> write children (from the parent's stored,
// not yet overwritten state) -> store the parents.  The look-back wait is
// thus taken after the expensive push, when the predecessors are done.
// ---------------------------------------------------------------------------
template <int FORM, int QED, int ITEMS>
__device__ __forceinline__ void sfp_step_body(const sfp_run_dev* __restrict__ R) {
    using namespace sfp;
    extern __shared__ double s_tab[];
    __shared__ long long s_tile;
    __shared__ int s_seg;
    __shared__ unsigned int s_warp[ITEMS][SFP_TILE / 32];
    __shared__ uint4 s_excl;

    sfp_step_state* st = R->st;
    if (st->skip) return;
    const long long n_tiles = st->n_tiles;
    const double t = st->t;
    const double dt = R->dt;
    const unsigned int step = (unsigned int)st->step;
    const unsigned int epoch = st->epoch;

    // QED tables into shared memory (float64 or float32 copies)
    const double* iAt = s_tab;
    const double* dAt = s_tab;
    const float* iAf = reinterpret_cast<const float*>(s_tab);
    const float* dAf = iAf;
    const double* od_rate_ph = s_tab;
    const double* od_rate_pa = s_tab;
    int zN = 0;
    double zmax = 0.0;
    if (QED == SFP_QED_REJECTION) {
        zN = R->rs.z_N;
        zmax = R->rs.z_max;
        if (FORM == SFP_FORM_FP64) {
            for (int i = threadIdx.x; i < zN; i += blockDim.x) {
                s_tab[i] = R->rs.int_Ai[i];
                s_tab[zN + i] = R->rs.Aip[i];
            }
            dAt = s_tab + zN;
        } else {
            float* f = reinterpret_cast<float*>(s_tab);
            for (int i = threadIdx.x; i < zN; i += blockDim.x) {
                f[i] = (float)R->rs.int_Ai[i];
                f[zN + i] = (float)R->rs.Aip[i];
            }
            dAf = f + zN;
        }
    } else {
        const int n1 = R->od_photon.chi_N, n2 = R->od_pair.chi_N;
        for (int i = threadIdx.x; i < n1; i += blockDim.x) s_tab[i] = R->od_photon.rate_total[i];
        for (int i = threadIdx.x; i < n2; i += blockDim.x) s_tab[n1 + i] = R->od_pair.rate_total[i];
        od_rate_pa = s_tab + n1;
    }
    const float inv_dzf = (float)((double)(zN - 1) / zmax);
    const float base_maxf = (float)(zmax * sqrt(zmax));
    // pair creation needs z_min = (4/chi)^(2/3) <= z_max (the rate is 0 above
    // the table): below this chi no pair event can happen, exactly
    const double chi_pair_min = QED == SFP_QED_REJECTION ? 4.0 / (zmax * sqrt(zmax)) * (1.0 - 1e-6) : 0.0;
    const float kRate = (float)((kAlpha * kMe) * (kC * kC) / kHbar);  // alpha m c^2 / hbar
    const float thrf = (float)R->photon_threshold;
    const bool any_appends = R->any_appends != 0;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long tk = (long long)atomicAdd(&st->ticket, 1);
            s_tile = tk;
            int s = 0;
            if (tk < n_tiles) {  // largest s with tile_start[s] <= tk
                int lo = 0, hi = R->n_seg - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (R->tile_start[mid] <= tk) lo = mid;
                    else hi = mid - 1;
                }
                s = lo;
            }
            s_seg = s;
        }
        __syncthreads();
        const long long tile = s_tile;
        if (tile >= n_tiles) break;
        const int si = s_seg;
        const sfp_segment& S = R->seg[si];
        const sfp_instance& I = R->inst[S.instance];
        const double* __restrict__ P = I.field_params;
        const long long N = R->n_buf_step[si];
        const long long first_tile = R->tile_start[I.first_seg];
        const long long i0 = (tile - R->tile_start[si]) * (long long)(SFP_TILE * ITEMS) + threadIdx.x;
        const bool qed_seg = S.radiating || S.bw;

        bool alive[ITEMS], ev[ITEMS];
        double x[ITEMS], y[ITEMS], z[ITEMS], ux[ITEMS], uy[ITEMS], uz[ITEMS], tau[ITEMS], delta[ITEMS];
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const long long i = i0 + (long long)k * SFP_TILE;
            alive[k] = (i < N) && (S.pruned[i] == 0);
            ev[k] = false;
            delta[k] = 0.0;
            x[k] = y[k] = z[k] = ux[k] = uy[k] = uz[k] = tau[k] = 0.0;
            if (alive[k]) {
                x[k] = S.x[i]; y[k] = S.y[i]; z[k] = S.z[i];
                ux[k] = S.ux[i]; uy[k] = S.uy[i]; uz[k] = S.uz[i];
                if (QED == SFP_QED_OPTICAL_DEPTH && S.tau) tau[k] = S.tau[i];
            }
        }

        // --- QED events at t (fields at t only for pushed species) ---------
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            if (!(alive[k] && qed_seg)) continue;
            const long long i = i0 + (long long)k * SFP_TILE;
            if (FORM == SFP_FORM_FP64) {
                double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (S.push) sfp_field_program(x[k], y[k], z[k], t, P, F);
                const double ig = S.massless ? inv_gamma_photon(ux[k], uy[k], uz[k])
                                             : inv_gamma_massive(ux[k], uy[k], uz[k]);
                const double chi = chi_of(F, ux[k], uy[k], uz[k], ig);
                double d = 0.0;
                if (QED == SFP_QED_REJECTION) {
                    if (chi != 0.0 && !(S.bw && chi < chi_pair_min)) {
                        double r1, r2;
                        uniform2(I.seed, S.stream, step, 0u, i, r1, r2);
                        ev[k] = S.bw ? pair_event_rs(chi, ig, dt, r1, r2, iAt, dAt, zN, zmax, d)
                                     : photon_event_rs(chi, ig, dt, r1, r2, iAt, dAt, zN, zmax, d);
                    }
                } else {
                    ev[k] = S.bw ? od_event(chi, ig, dt, tau[k], R->od_pair, od_rate_pa, I.seed, S.stream, step, i, d)
                                 : od_event(chi, ig, dt, tau[k], R->od_photon, od_rate_ph, I.seed, S.stream, step, i, d);
                }
                if (ev[k] && S.radiating && d / ig < R->photon_threshold) ev[k] = false;  // cpu.py:226-231
                delta[k] = d;
            } else {
                float F[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (S.push) sfp_field_program32(x[k], y[k], z[k], t, P, F);
                const float g = sfp32::gamma_of(ux[k], uy[k], uz[k], S.massless != 0);
                const float chi = sfp32::chi_of(F, (float)ux[k], (float)uy[k], (float)uz[k], g);
                double d = 0.0;
                if (QED == SFP_QED_REJECTION) {
                    if (chi > 0.0f && !(S.bw && (double)chi < chi_pair_min)) {
                        float r1, r2;
                        sfp32::uniform2f(I.seed, S.stream, step, 0u, i, r1, r2);
                        const float dtau = (float)dt / g;
                        if (S.bw) {  // qed/rejection_sampling.py:92-107, delta = r1
                            const float base = 1.0f / ((r1 * (1.0f - r1)) * chi);
                            const float W = kRate * sfp32::rate_core(chi, base, iAf, dAf, inv_dzf, zN, base_maxf, -1.0f);
                            ev[k] = r2 < W * dtau;
                            d = (double)r1;
                        } else {  // qed/rejection_sampling.py:73-89, delta = r1^3
                            const float dl = r1 * r1 * r1;
                            const float base = dl / ((1.0f - dl) * chi);
                            const float W = -kRate * sfp32::rate_core(dl * chi, base, iAf, dAf, inv_dzf, zN, base_maxf, 1.0f);
                            ev[k] = r2 < 3.0f * r1 * r1 * W * dtau;
                            d = (double)dl;
                            if (ev[k] && dl * g < thrf) ev[k] = false;
                        }
                    }
                } else {
                    const double igd = 1.0 / (double)g;
                    ev[k] = S.bw ? od_event((double)chi, igd, dt, tau[k], R->od_pair, od_rate_pa, I.seed, S.stream, step,
                                            i, d)
                                 : od_event((double)chi, igd, dt, tau[k], R->od_photon, od_rate_ph, I.seed, S.stream,
                                            step, i, d);
                    if (ev[k] && S.radiating && d * (double)g < R->photon_threshold) ev[k] = false;
                }
                if (!ev[k]) d = 0.0;
                delta[k] = d;
            }
        }

        // --- tile count: block scan (k-major); publish, try the look-back ---
        unsigned int wpre[ITEMS];
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const unsigned int bal = __ballot_sync(0xffffffffu, ev[k]);
            wpre[k] = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0) s_warp[k][warp] = __popc(bal);
        }
        __syncthreads();
        uint4 agg{0u, 0u, 0u, 0u};
        bool have_excl = true;
        if (warp == 0 && any_appends) {
            constexpr int NW = SFP_TILE / 32;
            const unsigned int v = (lane < ITEMS * NW) ? s_warp[lane / NW][lane % NW] : 0u;
            unsigned int inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int n2 = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += n2;
            }
            const unsigned int total = __shfl_sync(0xffffffffu, inc, 31);
            if (lane < ITEMS * NW) s_warp[lane / NW][lane % NW] = inc - v;
            if (qed_seg) agg = u4_one(S.channel, total);
            if (lane == 0 && total) {
                if (S.radiating) atomicAdd(&R->appended[S.photon_dest], (unsigned long long)total);
                if (S.bw) {
                    atomicAdd(&R->appended[S.ele_dest], (unsigned long long)total);
                    atomicAdd(&R->appended[S.pos_dest], (unsigned long long)total);
                }
            }
            uint4 ex{0u, 0u, 0u, 0u};
            if (tile == first_tile) {
                publish(R, tile, agg, epoch, true);
            } else {
                publish(R, tile, agg, epoch, false);
                have_excl = lookback_try(R, tile, first_tile, epoch, ex);
                if (have_excl) publish(R, tile, u4_add(ex, agg), epoch, true);
            }
            if (lane == 0) s_excl = ex;
        }

        // --- recoil and push of every parent, in registers ------------------
        bool conv[ITEMS];
        double sx[ITEMS], sy[ITEMS], sz[ITEMS];
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const long long i = i0 + (long long)k * SFP_TILE;
            conv[k] = ev[k] && S.bw;  // converted photons are pruned, not pushed (cpu.py:190)
            sx[k] = sy[k] = sz[k] = 0.0;
            if (ev[k] && S.radiating && S.rr == SFP_RR_PHOTON) {  // recoil, cpu.py:76-87
                const double f = 1.0 - delta[k];
                ux[k] = ux[k] * f; uy[k] = uy[k] * f; uz[k] = uz[k] * f;
            }
            if (!(alive[k] && !conv[k] && S.push)) continue;
            if (S.massless) {
                if (FORM == SFP_FORM_FP64) push_photon(x[k], y[k], z[k], ux[k], uy[k], uz[k], dt);
                else push_photon32(x[k], y[k], z[k], ux[k], uy[k], uz[k], dt);
            } else {
                if (S.spin) { sx[k] = S.sx[i]; sy[k] = S.sy[i]; sz[k] = S.sz[i]; }
                if (FORM == SFP_FORM_FP64) push_massive(x[k], y[k], z[k], ux[k], uy[k], uz[k], sx[k], sy[k], sz[k], S, P, t, dt);
                else push_massive32(x[k], y[k], z[k], ux[k], uy[k], uz[k], sx[k], sy[k], sz[k], S, P, t, dt);
            }
        }

        // --- finish the look-back -------------------------------------------
        if (warp == 0 && any_appends && !__all_sync(0xffffffffu, have_excl)) {
            const uint4 ex = lookback_wait(R, tile, first_tile, epoch);
            publish(R, tile, u4_add(ex, agg), epoch, true);
            if (lane == 0) s_excl = ex;
        }
        __syncthreads();
        const long long ch_base = any_appends ? (long long)u4_get(s_excl, S.channel) : 0ll;

        // --- children, then the parents' state ------------------------------
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const long long i = i0 + (long long)k * SFP_TILE;
            if (ev[k]) {
                const long long off = ch_base + s_warp[k][warp] + wpre[k];
                if (S.radiating) {  // photon at the parent's pre-push position, u = delta * u (cpu.py:89-116)
                    const sfp_segment& D = R->seg[S.photon_dest];
                    const long long slot = R->n_buf_step[S.photon_dest] + off;
                    double cx = S.x[i], cy = S.y[i], cz = S.z[i];
                    const double cux = delta[k] * S.ux[i], cuy = delta[k] * S.uy[i], cuz = delta[k] * S.uz[i];
                    if (D.push) {
                        if (FORM == SFP_FORM_FP64) push_photon(cx, cy, cz, cux, cuy, cuz, dt);
                        else push_photon32(cx, cy, cz, cux, cuy, cuz, dt);
                    }
                    D.x[slot] = cx; D.y[slot] = cy; D.z[slot] = cz;
                    D.ux[slot] = cux; D.uy[slot] = cuy; D.uz[slot] = cuz;
                    if (D.tau) D.tau[slot] = 0.0;
                    D.pruned[slot] = 0;
                } else {  // e- and e+ from the (unpushed) photon (cpu.py:119-189)
                    for (int w = 0; w < 2; ++w) {
                        const int di = (w == 0) ? S.ele_dest : S.pos_dest;
                        const sfp_segment& D = R->seg[di];
                        const double d = (w == 0) ? delta[k] : 1.0 - delta[k];
                        double cx = x[k], cy = y[k], cz = z[k], cux = d * ux[k], cuy = d * uy[k], cuz = d * uz[k];
                        double csx = 0.0, csy = 0.0, csz = 0.0;
                        if (D.push) {
                            if (FORM == SFP_FORM_FP64) push_massive(cx, cy, cz, cux, cuy, cuz, csx, csy, csz, D, P, t, dt);
                            else push_massive32(cx, cy, cz, cux, cuy, cuz, csx, csy, csz, D, P, t, dt);
                        }
                        const long long slot = R->n_buf_step[di] + off;
                        D.x[slot] = cx; D.y[slot] = cy; D.z[slot] = cz;
                        D.ux[slot] = cux; D.uy[slot] = cuy; D.uz[slot] = cuz;
                        if (D.spin) { D.sx[slot] = csx; D.sy[slot] = csy; D.sz[slot] = csz; }
                        if (D.tau) D.tau[slot] = 0.0;
                        D.pruned[slot] = 0;
                    }
                    S.pruned[i] = 1;
                }
            }
            if (alive[k] && !conv[k]) {
                if (S.push) { S.x[i] = x[k]; S.y[i] = y[k]; S.z[i] = z[k]; }
                if (!S.massless && (S.push || (ev[k] && S.rr == SFP_RR_PHOTON))) {
                    S.ux[i] = ux[k]; S.uy[i] = uy[k]; S.uz[i] = uz[k];
                }
                if (S.spin && S.push && !S.massless) { S.sx[i] = sx[k]; S.sy[i] = sy[k]; S.sz[i] = sz[k]; }
            }
            if (QED == SFP_QED_OPTICAL_DEPTH && alive[k] && S.tau && qed_seg) S.tau[i] = tau[k];
        }
    }
}

// kernels: <form>_<qed>_i<items per thread>_b<min resident blocks per SM>
#define SFP_STEP_KERNEL(NAME, FORM, QED, ITEMS, MINB)                                                      \
    extern "C" __global__ void __launch_bounds__(SFP_TILE, MINB) NAME(const sfp_run_dev* __restrict__ R) { \
        sfp_step_body<FORM, QED, ITEMS>(R);                                                                \
    }

#if defined(SFP_STEP_FORM_FP64) && defined(SFP_STEP_QED_RS)
SFP_STEP_KERNEL(sfp_step_fp64_rs_i1_b2, SFP_FORM_FP64, SFP_QED_REJECTION, 1, 2)
SFP_STEP_KERNEL(sfp_step_fp64_rs_i1_b3, SFP_FORM_FP64, SFP_QED_REJECTION, 1, 3)
SFP_STEP_KERNEL(sfp_step_fp64_rs_i2_b2, SFP_FORM_FP64, SFP_QED_REJECTION, 2, 2)
#endif
#if defined(SFP_STEP_FORM_FP64) && defined(SFP_STEP_QED_OD)
SFP_STEP_KERNEL(sfp_step_fp64_od_i1_b2, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 1, 2)
SFP_STEP_KERNEL(sfp_step_fp64_od_i2_b2, SFP_FORM_FP64, SFP_QED_OPTICAL_DEPTH, 2, 2)
#endif
#if defined(SFP_STEP_FORM_FP32) && defined(SFP_STEP_QED_RS)
SFP_STEP_KERNEL(sfp_step_fp32_rs_i1_b2, SFP_FORM_FP32, SFP_QED_REJECTION, 1, 2)
SFP_STEP_KERNEL(sfp_step_fp32_rs_i1_b3, SFP_FORM_FP32, SFP_QED_REJECTION, 1, 3)
SFP_STEP_KERNEL(sfp_step_fp32_rs_i1_b4, SFP_FORM_FP32, SFP_QED_REJECTION, 1, 4)
SFP_STEP_KERNEL(sfp_step_fp32_rs_i2_b2, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 2)
SFP_STEP_KERNEL(sfp_step_fp32_rs_i2_b3, SFP_FORM_FP32, SFP_QED_REJECTION, 2, 3)
#endif
#if defined(SFP_STEP_FORM_FP32) && defined(SFP_STEP_QED_OD)
SFP_STEP_KERNEL(sfp_step_fp32_od_i1_b3, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 1, 3)
SFP_STEP_KERNEL(sfp_step_fp32_od_i2_b2, SFP_FORM_FP32, SFP_QED_OPTICAL_DEPTH, 2, 2)
#endif
#endif  // SFP_WANT_STEP

#if defined(SFP_WANT_FIELD_EVAL)

// Field evaluation of the program at particle positions (Fields.field_func,
// fields.py:31-46): the per-op boundary kernel of the NVRTC module.
extern "C" __global__ void __launch_bounds__(256)
    sfp_field_eval_kernel(const double* __restrict__ P, const double* __restrict__ x, const double* __restrict__ y,
                          const double* __restrict__ z, double t, long long N, const unsigned char* __restrict__ pruned,
                          double* __restrict__ Ex, double* __restrict__ Ey, double* __restrict__ Ez,
                          double* __restrict__ Bx, double* __restrict__ By, double* __restrict__ Bz) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        if (pruned[i]) continue;
        double F[6];
        sfp_field_program(x[i], y[i], z[i], t, P, F);
        Ex[i] = F[0]; Ey[i] = F[1]; Ez[i] = F[2];
        Bx[i] = F[3]; By[i] = F[4]; Bz[i] = F[5];
    }
}
#endif  // SFP_WANT_FIELD_EVAL
