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
// instance, run by warp 0.  Returns the exclusive per-channel prefix.
// Every wait is bounded; on timeout the run's error word is set.
SFP_DEVICE_INLINE uint4 lookback(const sfp_run_dev* R, long long tile, long long first_tile, uint4 agg,
                                 unsigned int epoch) {
    const int lane = threadIdx.x & 31;
    uint4 excl{0u, 0u, 0u, 0u};
    if (tile == first_tile) {
        if (lane == 0) {
            st_cg_u4(R->tile_incl + tile, agg);
            st_release_u32(R->tile_flag + tile, (epoch << 2) | SFP_FLAG_INCL);
        }
        return excl;
    }
    if (lane == 0) {
        st_cg_u4(R->tile_agg + tile, agg);
        st_release_u32(R->tile_flag + tile, (epoch << 2) | SFP_FLAG_AGG);
    }
    long long base = tile - 1;
    bool failed = false;
    while (true) {
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
            // give up: flag the run and still publish, so no successor waits on this tile
            if (lane == 0) {
                atomicExch(&R->st->error, SFP_DEV_LOOKBACK_TIMEOUT);
                st_cg_u4(R->tile_incl + tile, agg);
                st_release_u32(R->tile_flag + tile, (epoch << 2) | SFP_FLAG_INCL);
            }
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
        if (base < first_tile) break;  // unreachable: the first tile publishes INCL
    }
    if (lane == 0) {
        st_cg_u4(R->tile_incl + tile, u4_add(excl, agg));
        st_release_u32(R->tile_flag + tile, (epoch << 2) | SFP_FLAG_INCL);
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
// The fused step, float64 form.  Persistent grid; tiles handed out in order.
// ---------------------------------------------------------------------------
template <int QED>
__device__ __forceinline__ void sfp_step_fp64(const sfp_run_dev* __restrict__ R) {
    using namespace sfp;
    extern __shared__ double s_tab[];
    __shared__ long long s_tile;
    __shared__ int s_seg;
    __shared__ unsigned int s_warp[SFP_TILE / 32];
    __shared__ uint4 s_excl;

    sfp_step_state* st = R->st;
    if (st->skip) return;
    const long long n_tiles = st->n_tiles;
    const double t = st->t;
    const double dt = R->dt;
    const unsigned int step = (unsigned int)st->step;
    const unsigned int epoch = st->epoch;

    // tables into shared memory
    const double* iAt = s_tab;
    const double* dAt = s_tab;
    const double* od_rate_ph = s_tab;
    const double* od_rate_pa = s_tab;
    int zN = 0;
    double zmax = 0.0;
    if (QED == SFP_QED_REJECTION) {
        zN = R->rs.z_N;
        zmax = R->rs.z_max;
        for (int i = threadIdx.x; i < zN; i += blockDim.x) {
            s_tab[i] = R->rs.int_Ai[i];
            s_tab[zN + i] = R->rs.Aip[i];
        }
        dAt = s_tab + zN;
    } else {
        const int n1 = R->od_photon.chi_N, n2 = R->od_pair.chi_N;
        for (int i = threadIdx.x; i < n1; i += blockDim.x) s_tab[i] = R->od_photon.rate_total[i];
        for (int i = threadIdx.x; i < n2; i += blockDim.x) s_tab[n1 + i] = R->od_pair.rate_total[i];
        od_rate_pa = s_tab + n1;
    }

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long tk = (long long)atomicAdd(&st->ticket, 1);
            s_tile = tk;
            int s = 0;
            if (tk < n_tiles) {  // largest s with tile_start[s] <= tk < tile_start[s+1]
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
        const long long i = (tile - R->tile_start[si]) * (long long)SFP_TILE + threadIdx.x;

        const bool alive = (i < N) && (S.pruned[i] == 0);
        double x = 0, y = 0, z = 0, ux = 0, uy = 0, uz = 0, sx = 0, sy = 0, sz = 0, tau = 0;
        if (alive) {
            x = S.x[i]; y = S.y[i]; z = S.z[i];
            ux = S.ux[i]; uy = S.uy[i]; uz = S.uz[i];
            if (S.spin) { sx = S.sx[i]; sy = S.sy[i]; sz = S.sz[i]; }
            if (QED == SFP_QED_OPTICAL_DEPTH && S.tau) tau = S.tau[i];
        }

        // --- QED events at t (fields at t only for pushed species) ---------
        bool ev = false;
        double delta = 0.0;
        if (alive && (S.radiating || S.bw)) {
            double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (S.push) sfp_field_program(x, y, z, t, P, F);
            const double ig = S.massless ? inv_gamma_photon(ux, uy, uz) : inv_gamma_massive(ux, uy, uz);
            const double chi = chi_of(F, ux, uy, uz, ig);
            if (QED == SFP_QED_REJECTION) {
                if (chi != 0.0) {
                    double r1, r2;
                    uniform2(I.seed, S.stream, step, 0u, i, r1, r2);
                    if (S.bw)
                        ev = pair_event_rs(chi, ig, dt, r1, r2, iAt, dAt, zN, zmax, delta);
                    else
                        ev = photon_event_rs(chi, ig, dt, r1, r2, iAt, dAt, zN, zmax, delta);
                }
            } else {
                if (S.bw)
                    ev = od_event(chi, ig, dt, tau, R->od_pair, od_rate_pa, I.seed, S.stream, step, i, delta);
                else
                    ev = od_event(chi, ig, dt, tau, R->od_photon, od_rate_ph, I.seed, S.stream, step, i, delta);
            }
            if (ev && S.radiating && delta / ig < R->photon_threshold) ev = false;  // cpu.py:226-231
        }

        // --- ordered slots: block scan + look-back -------------------------
        const unsigned int bal = __ballot_sync(0xffffffffu, ev);
        const unsigned int wpre = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) s_warp[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0 && R->any_appends) {
            unsigned int v = (lane < SFP_TILE / 32) ? s_warp[lane] : 0u;
            unsigned int inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int n2 = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += n2;
            }
            const unsigned int total = __shfl_sync(0xffffffffu, inc, 31);
            if (lane < SFP_TILE / 32) s_warp[lane] = inc - v;
            const bool appends = S.radiating || S.bw;
            uint4 ex{0u, 0u, 0u, 0u};
            if (appends) {
                ex = lookback(R, tile, first_tile, u4_one(S.channel, total), epoch);
                if (lane == 0 && total) {
                    if (S.radiating) atomicAdd(&R->appended[S.photon_dest], (unsigned long long)total);
                    if (S.bw) {
                        atomicAdd(&R->appended[S.ele_dest], (unsigned long long)total);
                        atomicAdd(&R->appended[S.pos_dest], (unsigned long long)total);
                    }
                }
            } else {
                ex = lookback(R, tile, first_tile, uint4{0u, 0u, 0u, 0u}, epoch);
            }
            if (lane == 0) s_excl = ex;
        }
        __syncthreads();
        const long long off =
            R->any_appends ? (long long)u4_get(s_excl, S.channel) + s_warp[warp] + wpre : 0ll;

        // --- appends, recoil and pushes -------------------------------------
        bool converted = false;
        int n_items = 0;
        if (ev && S.radiating) {
            const sfp_segment& D = R->seg[S.photon_dest];
            const long long slot = R->n_buf_step[S.photon_dest] + off;
            double cx = x, cy = y, cz = z;
            const double cux = delta * ux, cuy = delta * uy, cuz = delta * uz;
            if (D.push) push_photon(cx, cy, cz, cux, cuy, cuz, dt);
            D.x[slot] = cx; D.y[slot] = cy; D.z[slot] = cz;
            D.ux[slot] = cux; D.uy[slot] = cuy; D.uz[slot] = cuz;
            if (D.tau) D.tau[slot] = 0.0;
            D.pruned[slot] = 0;
            if (S.rr == SFP_RR_PHOTON) {  // cpu.py:76-87
                const double f = 1.0 - delta;
                ux = ux * f; uy = uy * f; uz = uz * f;
            }
        }
        if (ev && S.bw) {
            converted = true;
            S.pruned[i] = 1;
            n_items = 2;
        }
        const bool parent_massive = alive && !converted && S.push && !S.massless;
        if (parent_massive) n_items = 1;

        // massive pushes: the parent (e+- species) or the two pair children
        for (int w = 0; w < 2; ++w) {
            if (w >= n_items) break;
            if (parent_massive) {
                push_massive(x, y, z, ux, uy, uz, sx, sy, sz, S, P, t, dt);
            } else {
                const int di = (w == 0) ? S.ele_dest : S.pos_dest;
                const sfp_segment& D = R->seg[di];
                const double d = (w == 0) ? delta : 1.0 - delta;  // cpu.py:175-182
                double cx = x, cy = y, cz = z, cux = d * ux, cuy = d * uy, cuz = d * uz;
                double csx = 0.0, csy = 0.0, csz = 0.0;
                if (D.push) push_massive(cx, cy, cz, cux, cuy, cuz, csx, csy, csz, D, P, t, dt);
                const long long slot = R->n_buf_step[di] + off;
                D.x[slot] = cx; D.y[slot] = cy; D.z[slot] = cz;
                D.ux[slot] = cux; D.uy[slot] = cuy; D.uz[slot] = cuz;
                if (D.spin) { D.sx[slot] = csx; D.sy[slot] = csy; D.sz[slot] = csz; }
                if (D.tau) D.tau[slot] = 0.0;
                D.pruned[slot] = 0;
            }
        }
        if (alive && !converted && S.push && S.massless) push_photon(x, y, z, ux, uy, uz, dt);

        if (alive && !converted) {
            if (S.push) { S.x[i] = x; S.y[i] = y; S.z[i] = z; }
            if (!S.massless && (S.push || (ev && S.rr == SFP_RR_PHOTON))) {
                S.ux[i] = ux; S.uy[i] = uy; S.uz[i] = uz;
            }
            if (S.spin && S.push) { S.sx[i] = sx; S.sy[i] = sy; S.sz[i] = sz; }
        }
        if (QED == SFP_QED_OPTICAL_DEPTH && alive && S.tau && (S.radiating || S.bw)) S.tau[i] = tau;
    }
}

#if defined(SFP_STEP_FORM_FP64) && defined(SFP_STEP_QED_RS)
extern "C" __global__ void __launch_bounds__(SFP_TILE) sfp_step_fp64_rs(const sfp_run_dev* __restrict__ R) {
    sfp_step_fp64<SFP_QED_REJECTION>(R);
}
#endif
#if defined(SFP_STEP_FORM_FP64) && defined(SFP_STEP_QED_OD)
extern "C" __global__ void __launch_bounds__(SFP_TILE) sfp_step_fp64_od(const sfp_run_dev* __restrict__ R) {
    sfp_step_fp64<SFP_QED_OPTICAL_DEPTH>(R);
}
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
