// sfp_capi.cu -- libsfp.so: the C-ABI of the B200 sfparticles step.
//
//   * per-op kernels that replace the reference's Numba kernels one for one
//     (the plugin boundary, sfparticles/particles.py:14-25);
//   * NVRTC compilation / loading of field-specialised step modules;
//   * step runs: device bookkeeping, persistent launches of the massive /
//     photon / scan / appends kernels, CUDA graphs.
//
// Device memory of particle buffers belongs to the caller; a run allocates
// only its own bookkeeping (segment tables, tile maps, event counters).
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <algorithm>
#include <unordered_map>
#include <vector>

#include "sfp.h"
#include "sfp_device.cuh"
#include "sfp_internal.h"
#include "sfp_mlp.cuh"
#include "sfp_run.cuh"

#define SFP_VERSION_STRING "sfparticles_b200 0.1.0 (sm_100a)"
// threads per block of the fused step's group kernels; the NVRTC modules are built with SFP_TILE equal to it
#define SFP_TILE_HOST 256

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define SFP_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(SFP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SFP_CHECK_LAUNCH() SFP_CUDA(cudaGetLastError())

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

constexpr int kBlock = 256;

inline unsigned int grid_for(long long n) {
    if (n <= 0) return 1;
    long long b = (n + kBlock - 1) / kBlock;
    long long cap = (long long)sm_count() * 16;
    return (unsigned int)(b < cap ? b : cap);
}

#define GRID_STRIDE(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// ------------------------------- per-op kernels ------------------------------

__global__ void k_push_position(double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                                const double* __restrict__ ux, const double* __restrict__ uy,
                                const double* __restrict__ uz, const double* __restrict__ ig, long long N,
                                const unsigned char* __restrict__ pr, double dt) {
    GRID_STRIDE(i, N) {
        if (pr[i]) continue;
        double a = x[i], b = y[i], c = z[i];
        sfp::push_position(a, b, c, ux[i], uy[i], uz[i], ig[i], dt);
        x[i] = a; y[i] = b; z[i] = c;
    }
}

__global__ void k_boris(double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                        double* __restrict__ ig, const double* __restrict__ Ex, const double* __restrict__ Ey,
                        const double* __restrict__ Ez, const double* __restrict__ Bx, const double* __restrict__ By,
                        const double* __restrict__ Bz, double q, long long N, const unsigned char* __restrict__ pr,
                        double dt) {
    GRID_STRIDE(i, N) {
        if (pr[i]) continue;
        const double F[6] = {Ex[i], Ey[i], Ez[i], Bx[i], By[i], Bz[i]};
        double a = ux[i], b = uy[i], c = uz[i];
        ig[i] = sfp::boris(a, b, c, F, q, dt);
        ux[i] = a; uy[i] = b; uz[i] = c;
    }
}

__global__ void k_boris_tbmt(double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                             double* __restrict__ ig, double* __restrict__ sx, double* __restrict__ sy,
                             double* __restrict__ sz, const double* __restrict__ Ex, const double* __restrict__ Ey,
                             const double* __restrict__ Ez, const double* __restrict__ Bx,
                             const double* __restrict__ By, const double* __restrict__ Bz, double q, double ae,
                             long long N, const unsigned char* __restrict__ pr, double dt) {
    GRID_STRIDE(i, N) {
        if (pr[i]) continue;
        const double F[6] = {Ex[i], Ey[i], Ez[i], Bx[i], By[i], Bz[i]};
        double a = ux[i], b = uy[i], c = uz[i], s1 = sx[i], s2 = sy[i], s3 = sz[i];
        ig[i] = sfp::boris_tbmt(a, b, c, s1, s2, s3, F, q, ae, dt);
        ux[i] = a; uy[i] = b; uz[i] = c;
        sx[i] = s1; sy[i] = s2; sz[i] = s3;
    }
}

__global__ void k_ll(double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                     double* __restrict__ ig, const double* __restrict__ chi, long long N,
                     const unsigned char* __restrict__ pr, double dt, int quantum) {
    GRID_STRIDE(i, N) {
        if (pr[i]) continue;
        double a = ux[i], b = uy[i], c = uz[i];
        ig[i] = sfp::ll_push(a, b, c, ig[i], chi[i], dt, quantum != 0);
        ux[i] = a; uy[i] = b; uz[i] = c;
    }
}

__global__ void k_update_chi(const double* __restrict__ Ex, const double* __restrict__ Ey,
                             const double* __restrict__ Ez, const double* __restrict__ Bx,
                             const double* __restrict__ By, const double* __restrict__ Bz,
                             const double* __restrict__ ux, const double* __restrict__ uy,
                             const double* __restrict__ uz, const double* __restrict__ ig, double* __restrict__ chi,
                             long long N, const unsigned char* __restrict__ pr) {
    GRID_STRIDE(i, N) {
        if (pr[i]) continue;
        const double F[6] = {Ex[i], Ey[i], Ez[i], Bx[i], By[i], Bz[i]};
        chi[i] = sfp::chi_of(F, ux[i], uy[i], uz[i], ig[i]);
    }
}

__global__ void k_photon_recoil(double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                                double* __restrict__ ig, const unsigned char* __restrict__ ev,
                                const double* __restrict__ delta, long long N, const unsigned char* __restrict__ pr) {
    GRID_STRIDE(i, N) {
        if (pr[i] || !ev[i]) continue;
        const double f = 1.0 - delta[i];
        const double a = ux[i] * f, b = uy[i] * f, c = uz[i] * f;
        ux[i] = a; uy[i] = b; uz[i] = c;
        ig[i] = sfp::inv_gamma_massive(a, b, c);
    }
}

__global__ void k_pick_hard(unsigned char* __restrict__ ev, const double* __restrict__ delta,
                            const double* __restrict__ ig, double thr, long long N) {
    GRID_STRIDE(i, N) {
        if (ev[i] && delta[i] / ig[i] < thr) ev[i] = 0;
    }
}

__global__ void k_bool_sum(const unsigned char* __restrict__ ev, long long N, unsigned long long* __restrict__ out) {
    unsigned long long n = 0;
    GRID_STRIDE(i, N) n += ev[i] ? 1ull : 0ull;
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    __shared__ unsigned long long s[kBlock / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x < 32) {
        n = threadIdx.x < kBlock / 32 ? s[threadIdx.x] : 0ull;
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
        if (threadIdx.x == 0 && n) atomicAdd(out, n);
    }
}

// ordered compaction (find_event_index): 16 items per thread, 4096 per block
constexpr int kItems = 16;
constexpr long long kChunk = (long long)kBlock * kItems;

__global__ void k_fei_count(const unsigned char* __restrict__ ev, long long N, long long* __restrict__ counts) {
    const long long base = blockIdx.x * kChunk;
    unsigned int n = 0;
    for (int k = 0; k < kItems; ++k) {
        const long long i = base + (long long)k * kBlock + threadIdx.x;
        if (i < N && ev[i]) ++n;
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    __shared__ unsigned int s[kBlock / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += s[w];
        counts[blockIdx.x] = t;
    }
}

// single-block exclusive scan of n counts (in place)
__global__ void k_fei_scan(long long* __restrict__ counts, long long n) {
    __shared__ long long s_carry;
    __shared__ long long s_w[32];
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (long long base = 0; base < n; base += blockDim.x) {
        const long long i = base + threadIdx.x;
        const long long v = i < n ? counts[i] : 0;
        long long inc = v;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            long long w = lane < nw ? s_w[lane] : 0;
            long long wi = w;
            for (int o = 1; o < 32; o <<= 1) {
                const long long u = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += u;
            }
            if (lane < nw) s_w[lane] = wi - w;
        }
        __syncthreads();
        const long long excl = s_carry + s_w[warp] + inc - v;
        if (i < n) counts[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = excl + v;
        __syncthreads();
    }
}

__global__ void k_fei_scatter(const unsigned char* __restrict__ ev, long long N, const long long* __restrict__ offs,
                              long long* __restrict__ index, long long N_event) {
    const long long base = blockIdx.x * kChunk;
    // each thread owns kItems consecutive elements so the output stays ordered
    const long long first = base + (long long)threadIdx.x * kItems;
    unsigned int mask = 0;
    for (int k = 0; k < kItems; ++k) {
        const long long i = first + k;
        if (i < N && ev[i]) mask |= 1u << k;
    }
    const unsigned int n = __popc(mask);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int inc = n;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    __shared__ unsigned int s_w[kBlock / 32];
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        unsigned int w = lane < kBlock / 32 ? s_w[lane] : 0u;
        unsigned int wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < kBlock / 32) s_w[lane] = wi - w;
    }
    __syncthreads();
    long long pos = offs[blockIdx.x] + s_w[warp] + (inc - n);
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        if (pos < N_event) index[pos] = first + k;
        ++pos;
    }
}

__global__ void k_create_photon(const double* __restrict__ xs, const double* __restrict__ ys,
                                const double* __restrict__ zs, const double* __restrict__ uxs,
                                const double* __restrict__ uys, const double* __restrict__ uzs, double* __restrict__ xd,
                                double* __restrict__ yd, double* __restrict__ zd, double* __restrict__ uxd,
                                double* __restrict__ uyd, double* __restrict__ uzd, double* __restrict__ igd,
                                unsigned char* __restrict__ prd, const long long* __restrict__ idx,
                                const double* __restrict__ delta, long long Nb, long long Np) {
    GRID_STRIDE(k, Np) {
        const long long s = idx[k], d = Nb + k;
        xd[d] = xs[s]; yd[d] = ys[s]; zd[d] = zs[s];
        const double dl = delta[s];
        const double a = dl * uxs[s], b = dl * uys[s], c = dl * uzs[s];
        uxd[d] = a; uyd[d] = b; uzd[d] = c;
        igd[d] = sfp::inv_gamma_photon(a, b, c);
        prd[d] = 0;
    }
}

__global__ void k_create_pair(const double* __restrict__ xs, const double* __restrict__ ys,
                              const double* __restrict__ zs, const double* __restrict__ uxs,
                              const double* __restrict__ uys, const double* __restrict__ uzs,
                              unsigned char* __restrict__ prs, double* __restrict__ xd, double* __restrict__ yd,
                              double* __restrict__ zd, double* __restrict__ uxd, double* __restrict__ uyd,
                              double* __restrict__ uzd, double* __restrict__ igd, unsigned char* __restrict__ prd,
                              const long long* __restrict__ idx, const double* __restrict__ delta, long long Nb,
                              long long Np, int inverse) {
    GRID_STRIDE(k, Np) {
        const long long s = idx[k], d = Nb + k;
        xd[d] = xs[s]; yd[d] = ys[s]; zd[d] = zs[s];
        double dl = delta[s];
        if (inverse) dl = 1.0 - dl;
        const double a = dl * uxs[s], b = dl * uys[s], c = dl * uzs[s];
        uxd[d] = a; uyd[d] = b; uzd[d] = c;
        igd[d] = sfp::inv_gamma_massive(a, b, c);
        prd[d] = 0;
        prs[s] = 1;
    }
}

__global__ void k_rs(const double* __restrict__ ig, const double* __restrict__ chi, double dt, long long N,
                     const unsigned char* __restrict__ pr, unsigned char* __restrict__ ev, double* __restrict__ delta,
                     sfp_rs_table tab, unsigned long long seed, unsigned int stream, unsigned int step, int pair) {
    GRID_STRIDE(i, N) {
        const double c = chi[i];
        if (pr[i] || c == 0.0) {
            ev[i] = 0;
            continue;
        }
        double r1, r2, d;
        sfp::uniform2(seed, stream, step, 0u, i, r1, r2);
        const bool e = pair ? sfp::pair_event_rs(c, ig[i], dt, r1, r2, tab.int_Ai, tab.Aip, tab.z_N, tab.z_max, d)
                            : sfp::photon_event_rs(c, ig[i], dt, r1, r2, tab.int_Ai, tab.Aip, tab.z_N, tab.z_max, d);
        ev[i] = e ? 1 : 0;
        delta[i] = d;
    }
}

__global__ void k_update_tau(double* __restrict__ tau, const double* __restrict__ ig, const double* __restrict__ chi,
                             double dt, long long N, const unsigned char* __restrict__ pr, unsigned char* __restrict__ ev,
                             double* __restrict__ delta, sfp_od_table tab, unsigned long long seed,
                             unsigned int stream, unsigned int step) {
    const double chi_min = pow(10.0, tab.log_chi_min);  // _chi_min, optical_depth.py:14
    GRID_STRIDE(i, N) {
        if (pr[i]) {
            ev[i] = 0;
            delta[i] = 0.0;
            continue;
        }
        double tv = tau[i], d = 0.0;
        const bool e = sfp::od_event(chi[i], ig[i], dt, tv, tab, tab.rate_total, chi_min, seed, stream, step, i, d);
        tau[i] = tv;
        ev[i] = e ? 1 : 0;
        delta[i] = d;
    }
}

__global__ void k_inv_gamma(const double* __restrict__ ux, const double* __restrict__ uy,
                            const double* __restrict__ uz, double* __restrict__ ig, long long N, int massless) {
    GRID_STRIDE(i, N) {
        ig[i] = massless ? sfp::inv_gamma_photon(ux[i], uy[i], uz[i]) : sfp::inv_gamma_massive(ux[i], uy[i], uz[i]);
    }
}

// Per chi bin (sfp_pair_bin) an upper bound of the rejection-sampling pair
// rate over every delta, for the photon kernel's skip of pair tests that no
// draw can pass.  The rate is factor (iA + (2/z - chi sqrt z) dA) with
// z = (delta (1 - delta) chi)^(-2/3) >= z_min = (4/chi)^(2/3) and iA, dA
// linear between the table's grid points.  From the grid interval below
// z_min on, each interval contributes its largest iA, its largest positive
// dA times 2/z and chi sqrt(z at its right end) times its largest |dA|;
// chi is the bin's upper edge (the bound grows with chi), z_min is taken an
// interval early for the rounding of z, and the result is multiplied by 4
// for the rounding of the device's float32 and float64 rate arithmetic.
// The last bin, and any run without rejection-sampling tables, never skips.
__global__ void k_pair_bound(const double* __restrict__ iA, const double* __restrict__ dA, int zN, double zmax,
                             float* __restrict__ out) {
    const int k = threadIdx.x;
    if (k >= SFP_PAIR_BOUND_BINS) return;
    if (zN < 2 || !iA || !dA || k == SFP_PAIR_BOUND_BINS - 1) {
        out[k] = __int_as_float(0x7f800000);
        return;
    }
    const double chi = (double)__uint_as_float((unsigned int)(k + SFP_PAIR_BOUND_BASE + 1) << 20);
    const double zmin = pow(4.0 / chi, 2.0 / 3.0);
    if (zmin * (1.0 - 1e-4) > zmax) {  // every z is beyond the table: rate 0
        out[k] = 0.0f;
        return;
    }
    const double dz = zmax / (double)(zN - 1);
    long long j0 = (long long)floor(zmin / dz) - 1;
    if (j0 < 0) j0 = 0;
    double b = 0.0;
    for (long long j = j0; j < zN - 1; ++j) {
        const double zl = fmax((double)j * dz, zmin * (1.0 - 1e-4)), zr = (double)(j + 1) * dz;
        const double ia = fmax(iA[j], iA[j + 1]);
        const double dpos = fmax(fmax(dA[j], dA[j + 1]), 0.0);
        const double dabs = fmax(fabs(dA[j]), fabs(dA[j + 1]));
        b = fmax(b, ia + (dpos > 0.0 ? 2.0 / zl * dpos : 0.0) + chi * sqrt(zr) * dabs);
    }
    const double factor = ((sfp::kAlpha * sfp::kMe) * (sfp::kC * sfp::kC)) / sfp::kHbar;
    out[k] = __double2float_ru(4.0 * factor * b);
}

}  // namespace

int sfp_set_error(int code, const std::string& msg) { return fail(code, msg); }

extern "C" int sfp_pair_rate_bound(const double* int_ai, const double* aip, int z_n, double z_max, float* out,
                                   void* stream) {
    if (!out || (z_n >= 2 && (!int_ai || !aip))) return fail(SFP_EINVAL, "sfp_pair_rate_bound: NULL argument");
    k_pair_bound<<<1, SFP_PAIR_BOUND_BINS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(int_ai, aip, z_n, z_max, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SFP_ECUDA, std::string("sfp_pair_rate_bound: ") + cudaGetErrorString(e));
    return SFP_OK;
}

// ============== find_event_index without allocation (scratch) ===============
//
// sfp_find_event_index needs a scratch array of one count per 4096-entry
// chunk of the event mask, and asks its caller for it.  Some callers cannot
// provide device memory on demand: their device memory belongs to a pool or
// a caching allocator sized at start-up (cudaMalloc beside it fails or
// fragments the pool), or they must not stall, and cudaMalloc / cudaFree
// synchronise the whole device.  For them the scratch is a fixed array in
// the library's own device image instead: 65536 chunk counts (512 KiB), so
// at most 65536 * 4096 = 2^28 entries per call.  Every GPU on which this
// library's device code is loaded holds the 512 KiB until the process exits.
#define SFP_FEI_NOALLOC_CHUNKS 65536
static_assert((long long)SFP_FEI_NOALLOC_CHUNKS * kChunk == SFP_FEI_NOALLOC_MAX_N,
              "scratch size and the declared maximum disagree");
static __device__ __align__(256) long long g_fei_noalloc_scratch[SFP_FEI_NOALLOC_CHUNKS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_fei_noalloc_mu;
long long* g_fei_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device.  Looked up once per
// device, by the first call made with that device current; later calls on
// that device reuse the cached address.  The address belongs to the
// device's primary context: a cudaDeviceReset ends it, and the entry point
// is not to be used on that device afterwards (declared in sfp.h).
int fei_noalloc_scratch(long long** out) {
    int dev = -1;
    SFP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(SFP_EINVAL, "sfp_find_event_index_noalloc: device index " + std::to_string(dev) +
                                    " beyond the supported 64 devices");
    std::lock_guard<std::mutex> g(g_fei_noalloc_mu);
    if (!g_fei_noalloc_ptr[dev]) {
        long long* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_fei_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(SFP_ECUDA, std::string("sfp_find_event_index_noalloc: cudaGetSymbolAddress of the scratch "
                                               "failed: ") + cudaGetErrorString(e));
        g_fei_noalloc_ptr[dev] = ptr;
    }
    *out = g_fei_noalloc_ptr[dev];
    return SFP_OK;
}

}  // namespace

// ================================ C-ABI ======================================

struct sfp_module {
    cudaLibrary_t lib = nullptr;
    std::mutex mu;
    std::unordered_map<std::string, cudaKernel_t> kernels;
    // a module for runs of one instance holds that instance's field
    // parameters in its constant bank (sfp_cfield); every run on the module
    // copies its own block there before launching, after the launches of
    // the run that used the module last (cf_done), under cf_mu
    std::mutex cf_mu;
    cudaEvent_t cf_done = nullptr;
};

static int module_kernel(sfp_module* m, const char* name, cudaKernel_t* out) {
    std::lock_guard<std::mutex> g(m->mu);
    auto it = m->kernels.find(name);
    if (it != m->kernels.end()) {
        *out = it->second;
        return SFP_OK;
    }
    cudaKernel_t k = nullptr;
    cudaError_t e = cudaLibraryGetKernel(&k, m->lib, name);
    if (e != cudaSuccess) return fail(SFP_ENOKERNEL, std::string("kernel not in module: ") + name + " (" + cudaGetErrorString(e) + ")");
    m->kernels[name] = k;
    *out = k;
    return SFP_OK;
}

extern "C" {

const char* sfp_version(void) { return SFP_VERSION_STRING; }
const char* sfp_last_error(void) { return g_err.c_str(); }
void sfp_free(void* p) { std::free(p); }

int sfp_device_count(int* count) {
    if (!count) return fail(SFP_EINVAL, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(SFP_ECUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    *count = n;
    return SFP_OK;
}

int sfp_nvrtc_compile(const char* src, const char* name, const char* const* opts, int n_opts, void** image,
                      size_t* image_size, char** log) {
    if (!src || !image || !image_size) return fail(SFP_EINVAL, "sfp_nvrtc_compile: NULL argument");
    *image = nullptr;
    *image_size = 0;
    if (log) *log = nullptr;
    nvrtcProgram prog;
    nvrtcResult r = nvrtcCreateProgram(&prog, src, name ? name : "sfp_module.cu", 0, nullptr, nullptr);
    if (r != NVRTC_SUCCESS) return fail(SFP_ENVRTC, std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r));
    r = nvrtcCompileProgram(prog, n_opts, opts);
    size_t ls = 0;
    nvrtcGetProgramLogSize(prog, &ls);
    std::string lg(ls, '\0');
    if (ls) nvrtcGetProgramLog(prog, &lg[0]);
    if (log && ls) {
        *log = static_cast<char*>(std::malloc(ls + 1));
        std::memcpy(*log, lg.data(), ls);
        (*log)[ls] = 0;
    }
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return fail(SFP_ENVRTC, std::string("nvrtcCompileProgram: ") + nvrtcGetErrorString(r) + "\n" + lg);
    }
    size_t n = 0;
    r = nvrtcGetCUBINSize(prog, &n);
    if (r != NVRTC_SUCCESS || n == 0) {
        nvrtcDestroyProgram(&prog);
        return fail(SFP_ENVRTC, "nvrtcGetCUBINSize failed (compile with -arch=sm_100a)");
    }
    void* buf = std::malloc(n);
    r = nvrtcGetCUBIN(prog, static_cast<char*>(buf));
    nvrtcDestroyProgram(&prog);
    if (r != NVRTC_SUCCESS) {
        std::free(buf);
        return fail(SFP_ENVRTC, std::string("nvrtcGetCUBIN: ") + nvrtcGetErrorString(r));
    }
    *image = buf;
    *image_size = n;
    return SFP_OK;
}

int sfp_module_load(const void* image, size_t image_size, sfp_module** out) {
    if (!image || !out) return fail(SFP_EINVAL, "sfp_module_load: NULL argument");
    (void)image_size;
    auto* m = new sfp_module();
    cudaError_t e = cudaLibraryLoadData(&m->lib, image, nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) {
        delete m;
        return fail(SFP_ECUDA, std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e));
    }
    *out = m;
    return SFP_OK;
}

int sfp_module_unload(sfp_module* m) {
    if (!m) return SFP_OK;
    if (m->cf_done) cudaEventDestroy(m->cf_done);
    cudaError_t e = cudaLibraryUnload(m->lib);
    delete m;
    if (e != cudaSuccess) return fail(SFP_ECUDA, std::string("cudaLibraryUnload: ") + cudaGetErrorString(e));
    return SFP_OK;
}

int sfp_field_eval(sfp_module* m, const double* params, const double* x, const double* y, const double* z, double t,
                   int64_t N, const uint8_t* pr, double* Ex, double* Ey, double* Ez, double* Bx, double* By,
                   double* Bz, void* stream) {
    if (!m) return fail(SFP_EINVAL, "sfp_field_eval: NULL module");
    if (N <= 0) return SFP_OK;
    cudaKernel_t k;
    int rc = module_kernel(m, "sfp_field_eval_kernel", &k);
    if (rc) return rc;
    long long n = N;
    void* args[] = {&params, &x, &y, &z, &t, &n, &pr, &Ex, &Ey, &Ez, &Bx, &By, &Bz};
    SFP_CUDA(cudaLaunchKernel((const void*)k, dim3(grid_for(N)), dim3(kBlock), args, 0, as_stream(stream)));
    return SFP_OK;
}

#define RETURN_IF_EMPTY(n) \
    if ((n) <= 0) return SFP_OK

int sfp_push_position(double* x, double* y, double* z, const double* ux, const double* uy, const double* uz,
                      const double* ig, int64_t N, const uint8_t* pr, double dt, void* stream) {
    RETURN_IF_EMPTY(N);
    k_push_position<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(x, y, z, ux, uy, uz, ig, N, pr, dt);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_boris(double* ux, double* uy, double* uz, double* ig, const double* Ex, const double* Ey, const double* Ez,
              const double* Bx, const double* By, const double* Bz, double q, int64_t N, const uint8_t* pr, double dt,
              void* stream) {
    RETURN_IF_EMPTY(N);
    k_boris<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, Ex, Ey, Ez, Bx, By, Bz, q, N, pr, dt);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_boris_tbmt(double* ux, double* uy, double* uz, double* ig, double* sx, double* sy, double* sz,
                   const double* Ex, const double* Ey, const double* Ez, const double* Bx, const double* By,
                   const double* Bz, double q, double ae, int64_t N, const uint8_t* pr, double dt, void* stream) {
    RETURN_IF_EMPTY(N);
    k_boris_tbmt<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, sx, sy, sz, Ex, Ey, Ez, Bx, By, Bz, q,
                                                                 ae, N, pr, dt);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_LL_push(double* ux, double* uy, double* uz, double* ig, const double* chi, int64_t N, const uint8_t* pr,
                double dt, void* stream) {
    RETURN_IF_EMPTY(N);
    k_ll<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, chi, N, pr, dt, 0);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_CLL_push(double* ux, double* uy, double* uz, double* ig, const double* chi, int64_t N, const uint8_t* pr,
                 double dt, void* stream) {
    RETURN_IF_EMPTY(N);
    k_ll<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, chi, N, pr, dt, 1);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_update_chi(const double* Ex, const double* Ey, const double* Ez, const double* Bx, const double* By,
                   const double* Bz, const double* ux, const double* uy, const double* uz, const double* ig,
                   double* chi, int64_t N, const uint8_t* pr, void* stream) {
    RETURN_IF_EMPTY(N);
    k_update_chi<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(Ex, Ey, Ez, Bx, By, Bz, ux, uy, uz, ig, chi, N, pr);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_photon_recoil(double* ux, double* uy, double* uz, double* ig, const uint8_t* ev, const double* delta,
                      int64_t N, const uint8_t* pr, void* stream) {
    RETURN_IF_EMPTY(N);
    k_photon_recoil<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, ev, delta, N, pr);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_pick_hard_photon(uint8_t* ev, const double* delta, const double* ig, double thr, int64_t N, void* stream) {
    RETURN_IF_EMPTY(N);
    k_pick_hard<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ev, delta, ig, thr, N);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_bool_sum(const uint8_t* ev, int64_t N, int64_t* count, void* stream) {
    if (!count) return fail(SFP_EINVAL, "sfp_bool_sum: count is NULL");
    SFP_CUDA(cudaMemsetAsync(count, 0, sizeof(int64_t), as_stream(stream)));
    RETURN_IF_EMPTY(N);
    k_bool_sum<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ev, N, reinterpret_cast<unsigned long long*>(count));
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

size_t sfp_find_event_index_workspace(int64_t N) {
    const long long nb = N <= 0 ? 1 : (N + kChunk - 1) / kChunk;
    return (size_t)nb * sizeof(long long);
}

int sfp_find_event_index(const uint8_t* ev, int64_t N_event, int64_t N, int64_t* index, void* ws, size_t ws_bytes,
                         void* stream) {
    if (N <= 0 || N_event <= 0) return SFP_OK;
    const long long nb = (N + kChunk - 1) / kChunk;
    if (!ws || ws_bytes < (size_t)nb * sizeof(long long))
        return fail(SFP_EINVAL, "sfp_find_event_index: workspace too small");
    long long* counts = static_cast<long long*>(ws);
    cudaStream_t s = as_stream(stream);
    k_fei_count<<<(unsigned int)nb, kBlock, 0, s>>>(ev, N, counts);
    SFP_CHECK_LAUNCH();
    k_fei_scan<<<1, 1024, 0, s>>>(counts, nb);
    SFP_CHECK_LAUNCH();
    k_fei_scatter<<<(unsigned int)nb, kBlock, 0, s>>>(ev, N, counts, reinterpret_cast<long long*>(index), N_event);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

// Same three kernels as sfp_find_event_index, with the file-scope scratch in
// place of the caller's workspace.  Allocates nothing.  Nothing in the
// scratch has to start at zero: k_fei_count writes every chunk count that
// k_fei_scan and k_fei_scatter then read.  The scratch is shared by all
// calls on a device, so two calls in flight at once on one device (on
// different streams, or from different host threads) race; calls queued on
// one stream run one after the other and do not.
int sfp_find_event_index_noalloc(const uint8_t* ev, int64_t N_event, int64_t N, int64_t* index, void* stream) {
    if (N > SFP_FEI_NOALLOC_MAX_N)
        return fail(SFP_EINVAL, "sfp_find_event_index_noalloc: N = " + std::to_string((long long)N) +
                                    " exceeds the maximum of 268435456 (2^28) entries; use sfp_find_event_index "
                                    "with a caller workspace");
    // set-up first, so that a call with N = 0 performs only the set-up
    long long* counts = nullptr;
    const int rc = fei_noalloc_scratch(&counts);
    if (rc) return rc;
    if (N <= 0 || N_event <= 0) return SFP_OK;
    const long long nb = (N + kChunk - 1) / kChunk;
    cudaStream_t s = as_stream(stream);
    k_fei_count<<<(unsigned int)nb, kBlock, 0, s>>>(ev, N, counts);
    SFP_CHECK_LAUNCH();
    k_fei_scan<<<1, 1024, 0, s>>>(counts, nb);
    SFP_CHECK_LAUNCH();
    k_fei_scatter<<<(unsigned int)nb, kBlock, 0, s>>>(ev, N, counts, reinterpret_cast<long long*>(index), N_event);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_create_photon(const double* xs, const double* ys, const double* zs, const double* uxs, const double* uys,
                      const double* uzs, double* xd, double* yd, double* zd, double* uxd, double* uyd, double* uzd,
                      double* igd, uint8_t* prd, const int64_t* idx, const double* delta, int64_t Nb, int64_t Np,
                      void* stream) {
    RETURN_IF_EMPTY(Np);
    k_create_photon<<<grid_for(Np), kBlock, 0, as_stream(stream)>>>(xs, ys, zs, uxs, uys, uzs, xd, yd, zd, uxd, uyd,
                                                                     uzd, igd, prd,
                                                                     reinterpret_cast<const long long*>(idx), delta,
                                                                     Nb, Np);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_create_pair(const double* xs, const double* ys, const double* zs, const double* uxs, const double* uys,
                    const double* uzs, uint8_t* prs, double* xd, double* yd, double* zd, double* uxd, double* uyd,
                    double* uzd, double* igd, uint8_t* prd, const int64_t* idx, const double* delta, int64_t Nb,
                    int64_t Np, int inverse, void* stream) {
    RETURN_IF_EMPTY(Np);
    k_create_pair<<<grid_for(Np), kBlock, 0, as_stream(stream)>>>(xs, ys, zs, uxs, uys, uzs, prs, xd, yd, zd, uxd, uyd,
                                                                   uzd, igd, prd,
                                                                   reinterpret_cast<const long long*>(idx), delta, Nb,
                                                                   Np, inverse);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_photon_from_rejection_sampling(const double* ig, const double* chi, double dt, int64_t N, const uint8_t* pr,
                                       uint8_t* ev, double* delta, const sfp_rs_table* tab, uint64_t seed,
                                       uint32_t rng_stream, uint32_t step, void* stream) {
    if (!tab) return fail(SFP_EINVAL, "rate table is NULL");
    RETURN_IF_EMPTY(N);
    k_rs<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ig, chi, dt, N, pr, ev, delta, *tab, seed, rng_stream, step, 0);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_pair_from_rejection_sampling(const double* ig, const double* chi, double dt, int64_t N, const uint8_t* pr,
                                     uint8_t* ev, double* delta, const sfp_rs_table* tab, uint64_t seed,
                                     uint32_t rng_stream, uint32_t step, void* stream) {
    if (!tab) return fail(SFP_EINVAL, "rate table is NULL");
    RETURN_IF_EMPTY(N);
    k_rs<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ig, chi, dt, N, pr, ev, delta, *tab, seed, rng_stream, step, 1);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_update_tau(double* tau, const double* ig, const double* chi, double dt, int64_t N, const uint8_t* pr,
                   uint8_t* ev, double* delta, const sfp_od_table* tab, uint64_t seed, uint32_t rng_stream,
                   uint32_t step, void* stream) {
    if (!tab) return fail(SFP_EINVAL, "optical-depth table is NULL");
    RETURN_IF_EMPTY(N);
    k_update_tau<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(tau, ig, chi, dt, N, pr, ev, delta, *tab, seed,
                                                                 rng_stream, step);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

int sfp_inv_gamma(const double* ux, const double* uy, const double* uz, double* ig, int64_t N, int massless,
                  void* stream) {
    RETURN_IF_EMPTY(N);
    k_inv_gamma<<<grid_for(N), kBlock, 0, as_stream(stream)>>>(ux, uy, uz, ig, N, massless);
    SFP_CHECK_LAUNCH();
    return SFP_OK;
}

}  // extern "C"

// ================================ runs =======================================
//
// One step = book(prepare) + massive + photon [+ scan + appends] launches on
// the run's stream.  The massive and photon kernels are persistent grids that
// take warp tiles by ticket; the scan is one block; the appends kernel is a
// grid over both groups' tile counters.

#define SFP_SUPER_TILE_HOST 64
// the any-tile kernels (..._t) of each form: ring stages and blocks per SM
#define SFP_T_M_STAGES 2
#define SFP_T_P_STAGES 3
#define SFP_T_P_MINB 3
// a group of more particles than this has SFP_TILE_MAX-long tiles at every
// step (the tile rule), so the long-tile kernels may run it
#define SFP_LONG_TILE_POP ((long long)(SFP_TILE_MAX / 2) * SFP_TILE_TARGET)

struct sfp_group_host {
    std::vector<int> seg;
    int* d_seg = nullptr;
    long long* d_start = nullptr;
};

struct sfp_run {
    sfp_module* mod = nullptr;
    void* cfield = nullptr;  // the module's sfp_cfield (runs of one instance), or NULL
    size_t cfield_bytes = 0;
    void* ckeys = nullptr;           // the module's sfp_ckeys: the instance seed's Philox round keys
    unsigned int* d_keys = nullptr;  // those keys, formed at creation (20 words, device)
    cudaKernel_t k_massive = nullptr, k_photon = nullptr, k_scan = nullptr, k_appends = nullptr, k_book = nullptr;
    cudaKernel_t k_massive_t = nullptr, k_photon_t = nullptr;  // any tile length
    cudaKernel_t k_sync = nullptr, k_epoch = nullptr;           // photon positions written out
    int grid_m = 0, grid_p = 0, grid_a = 0, grid_mt = 0, grid_pt = 0;
    size_t smem_m = 0, smem_p = 0, smem_mt = 0, smem_pt = 0;
    std::vector<long long> nb_lo;  // lower bounds of the device's n_buffered (it only grows between reads)
    cudaStream_t s = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int n_seg = 0, n_inst = 0;
    sfp_run_dev h{};
    sfp_run_dev* d = nullptr;
    std::map<int, cudaGraphExec_t> graphs;
    std::vector<sfp_segment> segs;
    std::vector<sfp_instance> insts;
    sfp_group_host mg, pg;
    std::vector<int> dseg;
};

// tile counters a group needs at full capacity: each segment's longest
// tiles plus the padding up to the next multiple of a super-tile, and at
// least what the shorter tiles of a small population take (at most
// SFP_TILE_TARGET tiles plus one partial tile and the padding per segment)
static long long tiles_for(const sfp_run* r, const std::vector<int>& segs) {
    long long t = 0;
    for (int s : segs) t += (r->segs[s].capacity + SFP_TILE_MAX - 1) / SFP_TILE_MAX + SFP_SUPER_TILE_HOST;
    const long long small = SFP_TILE_TARGET + (long long)segs.size() * (SFP_SUPER_TILE_HOST + 1);
    return (t > small ? t : small) + 1;
}

// (re)allocate a group's tile counters for the current capacities; a step
// stopped for room keeps its counters through a reallocation
static int group_alloc(sfp_run* r, sfp_group_dev& G, long long need) {
    if (need <= G.max_tiles) return SFP_OK;
    const long long n = need + need / 4 + 64;
    const long long ns = n / SFP_SUPER_TILE_HOST + 2;
    const long long n_old = G.max_tiles, ns_old = n_old ? n_old / SFP_SUPER_TILE_HOST + 2 : 0;
    unsigned int *cnt = nullptr, *scnt = nullptr;
    long long* spre = nullptr;
    if (cudaMalloc(&cnt, n * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&scnt, ns * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&spre, ns * sizeof(long long)) != cudaSuccess) {
        cudaFree(cnt);
        cudaFree(scnt);
        cudaFree(spre);
        return fail(SFP_ENOMEM, "cudaMalloc of the tile counters");
    }
    if (n_old) {
        SFP_CUDA(cudaMemcpyAsync(cnt, G.tile_cnt, n_old * sizeof(unsigned int), cudaMemcpyDeviceToDevice, r->s));
        SFP_CUDA(cudaMemcpyAsync(scnt, G.super_cnt, ns_old * sizeof(unsigned int), cudaMemcpyDeviceToDevice, r->s));
        SFP_CUDA(cudaMemcpyAsync(spre, G.super_pre, ns_old * sizeof(long long), cudaMemcpyDeviceToDevice, r->s));
        SFP_CUDA(cudaStreamSynchronize(r->s));
    }
    cudaFree(G.tile_cnt);
    cudaFree(G.super_cnt);
    cudaFree(G.super_pre);
    G.tile_cnt = cnt;
    G.super_cnt = scnt;
    G.super_pre = spre;
    G.max_tiles = n;
    return SFP_OK;
}

static int run_alloc_tiles(sfp_run* r) {
    int rc = group_alloc(r, r->h.mg, tiles_for(r, r->mg.seg));
    if (rc) return rc;
    return group_alloc(r, r->h.pg, tiles_for(r, r->pg.seg));
}

static int validate_segments(int n_inst, const sfp_instance* inst, int n_seg, const sfp_segment* seg) {
    if (n_seg <= 0 || n_seg > SFP_MAX_SEGMENTS) return fail(SFP_EINVAL, "segment count out of range");
    if (n_inst <= 0) return fail(SFP_EINVAL, "instance count must be positive");
    int expect = 0;
    for (int i = 0; i < n_inst; ++i) {
        if (inst[i].first_seg != expect || inst[i].n_seg <= 0)
            return fail(SFP_EINVAL, "instances must cover the segments contiguously in order");
        // the step's float32 field presets read their constants 16 bytes at a time
        if (reinterpret_cast<uintptr_t>(inst[i].field_params) % 16 != 0)
            return fail(SFP_EINVAL, "instance field parameters must be 16-byte aligned");
        expect += inst[i].n_seg;
    }
    if (expect != n_seg) return fail(SFP_EINVAL, "instances do not cover all segments");
    for (int s = 0; s < n_seg; ++s) {
        const sfp_segment& S = seg[s];
        const std::string name = "segment " + std::to_string(s);
        if (S.capacity < 0) return fail(SFP_EINVAL, name + ": negative capacity");
        // an empty buffer (capacity 0) may have NULL arrays: nothing reads or writes it
        if (S.capacity > 0 && (!S.x || !S.y || !S.z || !S.ux || !S.uy || !S.uz || !S.pruned))
            return fail(SFP_EINVAL, name + ": NULL state pointer");
        if (S.capacity > 0 && S.spin && (!S.sx || !S.sy || !S.sz))
            return fail(SFP_EINVAL, "spin segment without spin arrays");
        if (S.channel < 0 || S.channel >= SFP_MAX_CHANNELS) return fail(SFP_EINVAL, "append channel out of range");
        // both group kernels stream the state with 16-byte asynchronous copies,
        // and the appends kernel reads the flags 16 at a time
        if (S.capacity > 0) {
            const void* a[] = {S.x, S.y, S.z, S.ux, S.uy, S.uz, S.pruned, S.tau, S.sx, S.sy, S.sz};
            for (const void* p : a)
                if (p && (reinterpret_cast<uintptr_t>(p) & 15u))
                    return fail(SFP_EINVAL, name + ": state arrays must be 16-byte aligned");
            if ((S.bw || S.radiating) && !S.delta)
                return fail(SFP_EINVAL, name + ": a segment with events needs a delta array");
        }
        // the massive kernel handles emission, the photon kernel pair creation
        if (S.massless && S.radiating) return fail(SFP_EINVAL, name + ": a photon cannot radiate");
        if (!S.massless && S.bw) return fail(SFP_EINVAL, name + ": only photons create pairs");
        const sfp_instance& I = inst[S.instance];
        auto in_inst = [&](int d) { return d >= I.first_seg && d < I.first_seg + I.n_seg; };
        if (S.radiating && (!in_inst(S.photon_dest) || !seg[S.photon_dest].massless))
            return fail(SFP_EINVAL, "radiating segment needs a photon destination in its instance");
        if (S.bw && (!in_inst(S.ele_dest) || !in_inst(S.pos_dest) || seg[S.ele_dest].massless ||
                     seg[S.pos_dest].massless))
            return fail(SFP_EINVAL, "pair-creating segment needs massive destinations in its instance");
        if (S.bw && S.ele_dest == S.pos_dest)
            return fail(SFP_EINVAL, "pair-creating segment: electron and positron destinations must differ");
    }
    return SFP_OK;
}

// the counts last uploaded or read back: a lower bound of every later step's
static void note_counts(sfp_run* r, const long long* nb) {
    r->nb_lo.assign(nb, nb + r->n_seg);
}

// whether every step from here on gives the group SFP_TILE_MAX-long tiles
static bool long_tiles(const sfp_run* r, const std::vector<int>& segs) {
    long long n = 0;
    for (int s : segs) n += r->nb_lo.empty() ? 0 : r->nb_lo[s];
    return n > SFP_LONG_TILE_POP;
}

static int run_upload(sfp_run* r, const sfp_instance* inst, const int64_t* n_buffered) {
    if (inst) SFP_CUDA(cudaMemcpyAsync((void*)r->h.inst, inst, r->n_inst * sizeof(sfp_instance), cudaMemcpyHostToDevice, r->s));
    SFP_CUDA(cudaMemcpyAsync((void*)r->h.seg, r->segs.data(), r->n_seg * sizeof(sfp_segment), cudaMemcpyHostToDevice, r->s));
    if (n_buffered) {
        SFP_CUDA(cudaMemcpyAsync(r->h.n_buffered, n_buffered, r->n_seg * sizeof(long long), cudaMemcpyHostToDevice, r->s));
        note_counts(r, reinterpret_cast<const long long*>(n_buffered));
    }
    SFP_CUDA(cudaMemcpyAsync(r->d, &r->h, sizeof(sfp_run_dev), cudaMemcpyHostToDevice, r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    return SFP_OK;
}

// the kernel's dynamic shared memory limit, raised to at least `need` bytes
static cudaError_t raise_dynamic_smem(const void* k, size_t need) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= need) return cudaSuccess;
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
}

// persistent grid of one kernel: resident blocks per SM x SMs
static int persistent_grid(cudaKernel_t k, size_t smem, int fallback_per_sm) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, SFP_TILE_HOST, smem) != cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = fallback_per_sm;
    }
    return sm_count() * per_sm;
}

extern "C" {

int sfp_run_create(sfp_module* m, const sfp_run_config* cfg, int n_inst, const sfp_instance* inst, int n_seg,
                   const sfp_segment* seg, const int64_t* n_buffered, sfp_run** out) {
    if (!cfg || !inst || !seg || !n_buffered || !out) return fail(SFP_EINVAL, "sfp_run_create: NULL argument");
    int rc = validate_segments(n_inst, inst, n_seg, seg);
    if (rc) return rc;
    if (!m) return fail(SFP_EINVAL, "sfp_run_create: NULL module");
    if (cfg->qed != SFP_QED_REJECTION && cfg->qed != SFP_QED_OPTICAL_DEPTH) return fail(SFP_EINVAL, "unknown QED method");
    if (cfg->form != SFP_FORM_FP64 && cfg->form != SFP_FORM_FP32) return fail(SFP_EINVAL, "unknown arithmetic form");
    if (cfg->mlp_params && cfg->qed != SFP_QED_OPTICAL_DEPTH)
        return fail(SFP_EINVAL, "the learned photon-energy sampler serves the optical-depth method only");
    const bool f64 = cfg->form == SFP_FORM_FP64;
    const int mstages = cfg->m_stages > 0 ? cfg->m_stages : (f64 ? 2 : 3);
    const int minb = cfg->min_blocks > 0 ? cfg->min_blocks : (f64 ? 2 : 3);
    const int stages = cfg->p_stages > 0 ? cfg->p_stages : 3;
    const int pminb = cfg->p_min_blocks > 0 ? cfg->p_min_blocks : (f64 ? 3 : 4);
    if (mstages < 2 || mstages > 4 || minb < 1 || minb > 8 || stages < 2 || stages > 4 || pminb < 1 || pminb > 8)
        return fail(SFP_EINVAL, "kernel variant out of range");
    auto* r = new sfp_run();
    r->mod = m;
    r->n_seg = n_seg;
    r->n_inst = n_inst;
    r->segs.assign(seg, seg + n_seg);
    r->insts.assign(inst, inst + n_inst);
    bool any_spin = false;
    for (int s = 0; s < n_seg; ++s) {
        (seg[s].massless ? r->pg.seg : r->mg.seg).push_back(s);
        if (!seg[s].massless && seg[s].spin) any_spin = true;
        bool dest = false;
        for (int q = 0; q < n_seg; ++q)
            if ((seg[q].bw && (seg[q].ele_dest == s || seg[q].pos_dest == s)) ||
                (seg[q].radiating && seg[q].photon_dest == s))
                dest = true;
        if (dest) r->dseg.push_back(s);
    }
    const std::string fq = std::string(f64 ? "fp64_" : "fp32_") + (cfg->qed == SFP_QED_REJECTION ? "rs" : "od");
    const std::string km = "sfp_massive_" + fq + "_s" + std::to_string(mstages) + "_b" + std::to_string(minb);
    const std::string kp = "sfp_photon_" + fq + "_s" + std::to_string(stages) + "_b" + std::to_string(pminb);
    const std::string ka = f64 ? "sfp_appends_fp64" : "sfp_appends_fp32";
    const std::string ksy = f64 ? "sfp_sync_positions_fp64" : "sfp_sync_positions_fp32";
    const int t_minb = f64 ? 2 : 3;
    const std::string kmt = "sfp_massive_" + fq + "_s" + std::to_string(SFP_T_M_STAGES) + "_b" +
                            std::to_string(t_minb) + "_t";
    const std::string kpt = "sfp_photon_" + fq + "_s" + std::to_string(SFP_T_P_STAGES) + "_b" +
                            std::to_string(SFP_T_P_MINB) + "_t";
    if ((rc = module_kernel(m, km.c_str(), &r->k_massive)) || (rc = module_kernel(m, kp.c_str(), &r->k_photon)) ||
        (rc = module_kernel(m, kmt.c_str(), &r->k_massive_t)) || (rc = module_kernel(m, kpt.c_str(), &r->k_photon_t)) ||
        (rc = module_kernel(m, ka.c_str(), &r->k_appends)) ||
        (rc = module_kernel(m, "sfp_scan_kernel", &r->k_scan)) ||
        (rc = module_kernel(m, ksy.c_str(), &r->k_sync)) || (rc = module_kernel(m, "sfp_epoch_kernel", &r->k_epoch)) ||
        (rc = module_kernel(m, "sfp_book_kernel", &r->k_book))) {
        delete r;
        return rc;
    }
    {
        // a module built for runs of one instance reads the field parameters
        // from its constant bank
        void* cf = nullptr;
        size_t cb = 0;
        if (cudaLibraryGetGlobal(&cf, &cb, m->lib, "sfp_cfield") == cudaSuccess && cf) {
            if (n_inst != 1) {
                delete r;
                return fail(SFP_EINVAL, "sfp_run_create: this step module serves runs of one instance (its field "
                                        "parameters sit in its constant bank); compile it without that option for " +
                                            std::to_string(n_inst) + " instances");
            }
            r->cfield = cf;
            r->cfield_bytes = cb;
            void* ck = nullptr;
            size_t kb = 0;
            if (cudaLibraryGetGlobal(&ck, &kb, m->lib, "sfp_ckeys") != cudaSuccess || !ck || kb != 20 * sizeof(unsigned)) {
                delete r;
                return fail(SFP_EINVAL, "sfp_run_create: a one-instance step module without its Philox key array");
            }
            // the key schedule of Philox-4x32-10 for the instance seed: round r
            // uses k0 + r 0x9E3779B9 and k1 + r 0xBB67AE85 (sfp::philox4x32_10)
            unsigned int keys[20];
            unsigned int k0 = (unsigned int)inst[0].seed, k1 = (unsigned int)(inst[0].seed >> 32);
            for (int q = 0; q < 10; ++q) {
                keys[2 * q] = k0;
                keys[2 * q + 1] = k1;
                k0 += 0x9E3779B9u;
                k1 += 0xBB67AE85u;
            }
            if (cudaMalloc(&r->d_keys, sizeof(keys)) != cudaSuccess ||
                cudaMemcpy(r->d_keys, keys, sizeof(keys), cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaFree(r->d_keys);
                delete r;
                return fail(SFP_ENOMEM, "sfp_run_create: Philox key array");
            }
            r->ckeys = ck;
        } else {
            cudaGetLastError();  // no such symbol: parameters are read from global memory
        }
    }
    auto cleanup = [&](int code) {
        sfp_run_destroy(r);
        return code;
    };
    if (cudaStreamCreateWithFlags(&r->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r->ev_out, cudaEventDisableTiming) != cudaSuccess)
        return cleanup(fail(SFP_ECUDA, "stream/event creation failed"));
    sfp_run_dev& h = r->h;
    h.n_seg = n_seg;
    h.n_inst = n_inst;
    h.dt = cfg->dt;
    h.photon_threshold = cfg->photon_threshold;
    h.qed = cfg->qed;
    h.any_rad = h.any_bw = 0;
    for (int s = 0; s < n_seg; ++s) {
        h.any_rad |= seg[s].radiating ? 1 : 0;
        h.any_bw |= seg[s].bw ? 1 : 0;
    }
    h.n_dseg = (int)r->dseg.size();
    h.mg.n_seg = (int)r->mg.seg.size();
    h.pg.n_seg = (int)r->pg.seg.size();
    h.rs = cfg->rs;
    h.od_photon = cfg->od_photon;
    h.od_pair = cfg->od_pair;
#define ALLOC(ptr, bytes) \
    if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) return cleanup(fail(SFP_ENOMEM, "cudaMalloc " #ptr))
    sfp_segment* dseg;
    sfp_instance* dinst;
    int* dd;
    ALLOC(dseg, n_seg * sizeof(sfp_segment));
    ALLOC(dinst, n_inst * sizeof(sfp_instance));
    h.seg = dseg;
    h.inst = dinst;
    ALLOC(r->mg.d_seg, (r->mg.seg.size() + 1) * sizeof(int));
    ALLOC(r->pg.d_seg, (r->pg.seg.size() + 1) * sizeof(int));
    ALLOC(dd, (r->dseg.size() + 1) * sizeof(int));
    ALLOC(r->mg.d_start, (r->mg.seg.size() + 1) * sizeof(long long));
    ALLOC(r->pg.d_start, (r->pg.seg.size() + 1) * sizeof(long long));
    h.mg.seg = r->mg.d_seg;
    h.pg.seg = r->pg.d_seg;
    h.mg.tile_start = r->mg.d_start;
    h.pg.tile_start = r->pg.d_start;
    h.dseg = dd;
    ALLOC(h.n_buffered, n_seg * sizeof(long long));
    ALLOC(h.appended, n_seg * sizeof(unsigned long long));
    ALLOC(h.n_buf_step, n_seg * sizeof(long long));
    ALLOC(h.st, sizeof(sfp_step_state));
    ALLOC(r->d, sizeof(sfp_run_dev));
    float* pb;
    ALLOC(pb, SFP_PAIR_BOUND_BINS * sizeof(float));
    h.pair_bound = pb;
#undef ALLOC
    k_pair_bound<<<1, SFP_PAIR_BOUND_BINS, 0, r->s>>>(cfg->qed == SFP_QED_REJECTION ? cfg->rs.int_Ai : nullptr,
                                                      cfg->rs.Aip, cfg->rs.z_N, cfg->rs.z_max, pb);
    if (cudaGetLastError() != cudaSuccess) return cleanup(fail(SFP_ECUDA, "pair-rate bound table"));
    if ((!r->mg.seg.empty() && cudaMemcpyAsync(r->mg.d_seg, r->mg.seg.data(), r->mg.seg.size() * sizeof(int),
                                               cudaMemcpyHostToDevice, r->s) != cudaSuccess) ||
        (!r->pg.seg.empty() && cudaMemcpyAsync(r->pg.d_seg, r->pg.seg.data(), r->pg.seg.size() * sizeof(int),
                                               cudaMemcpyHostToDevice, r->s) != cudaSuccess) ||
        (!r->dseg.empty() &&
         cudaMemcpyAsync(dd, r->dseg.data(), r->dseg.size() * sizeof(int), cudaMemcpyHostToDevice, r->s) != cudaSuccess) ||
        cudaMemsetAsync(r->mg.d_start, 0, (r->mg.seg.size() + 1) * sizeof(long long), r->s) != cudaSuccess ||
        cudaMemsetAsync(r->pg.d_start, 0, (r->pg.seg.size() + 1) * sizeof(long long), r->s) != cudaSuccess ||
        cudaMemsetAsync(h.appended, 0, n_seg * sizeof(unsigned long long), r->s) != cudaSuccess)
        return cleanup(fail(SFP_ECUDA, "segment lists upload"));
    sfp_step_state st0{};
    st0.t = cfg->t0;
    st0.step = cfg->step0;
    st0.pos_epoch = cfg->step0;  // the photon positions handed in are those at the start of step0
    st0.skip = 1;
    if (cudaMemcpyAsync(h.st, &st0, sizeof(st0), cudaMemcpyHostToDevice, r->s) != cudaSuccess)
        return cleanup(fail(SFP_ECUDA, "state upload"));
    // shared memory: the QED tables (both kernels); the massive kernel then
    // the learned sampler's weights (when used) and its copy ring, the photon
    // kernel its copy ring; rings of `stages` stages per warp
    size_t tab;
    if (cfg->qed == SFP_QED_REJECTION)
        tab = 2 * (size_t)cfg->rs.z_N * (f64 ? sizeof(double) : sizeof(float));
    else
        tab = ((size_t)cfg->od_photon.chi_N + (size_t)cfg->od_pair.chi_N) * sizeof(double);
    const int od = cfg->qed == SFP_QED_OPTICAL_DEPTH ? 1 : 0;
    const size_t warps = SFP_TILE_HOST / 32;
    h.mlp_params = cfg->mlp_params;
    h.mlp_off = (int)((tab + 127) / 128 * 128);
    const size_t m_head = cfg->mlp_params ? (size_t)h.mlp_off + sizeof(sfp_mlp::Smem) : tab;
    h.m_stage_bytes = (6 + od + (any_spin ? 3 : 0)) * 256 + 32;
    h.m_ring_off = (int)((m_head + 127) / 128 * 128);
    r->smem_m = (size_t)h.m_ring_off + warps * mstages * (size_t)h.m_stage_bytes;
    h.ring_off = (int)((tab + 127) / 128 * 128);
    r->smem_p = (size_t)h.ring_off + warps * stages * ((6 + od) * 256 + 32);
    r->smem_mt = (size_t)h.m_ring_off + warps * SFP_T_M_STAGES * (size_t)h.m_stage_bytes;
    r->smem_pt = (size_t)h.ring_off + warps * SFP_T_P_STAGES * ((6 + od) * 256 + 32);
    if ((rc = run_alloc_tiles(r))) return cleanup(rc);
    if ((rc = run_upload(r, inst, n_buffered))) return cleanup(rc);
    const size_t cap = 200 * 1024;
    if (r->smem_m > cap || r->smem_p > cap || r->smem_mt > cap || r->smem_pt > cap)
        return cleanup(fail(SFP_EINVAL, "QED tables and copy rings too large for shared memory"));
    // always raised, never lowered: the kernels' static shared memory counts
    // toward the 48 KB a launch gets without it, and runs that share a module
    // need different amounts
    if (raise_dynamic_smem((const void*)r->k_massive, r->smem_m) != cudaSuccess ||
        raise_dynamic_smem((const void*)r->k_photon, r->smem_p) != cudaSuccess ||
        raise_dynamic_smem((const void*)r->k_massive_t, r->smem_mt) != cudaSuccess ||
        raise_dynamic_smem((const void*)r->k_photon_t, r->smem_pt) != cudaSuccess)
        return cleanup(fail(SFP_ECUDA, "cannot raise dynamic shared memory"));
    r->grid_m = persistent_grid(r->k_massive, r->smem_m, minb);
    r->grid_p = persistent_grid(r->k_photon, r->smem_p, pminb);
    r->grid_mt = persistent_grid(r->k_massive_t, r->smem_mt, t_minb);
    r->grid_pt = persistent_grid(r->k_photon_t, r->smem_pt, SFP_T_P_MINB);
    r->grid_a = persistent_grid(r->k_appends, 0, 2);
    *out = r;
    return SFP_OK;
}

int sfp_run_update(sfp_run* r, int n_seg, const sfp_segment* seg, const int64_t* n_buffered) {
    if (!r || !seg) return fail(SFP_EINVAL, "sfp_run_update: NULL argument");
    if (n_seg != r->n_seg) return fail(SFP_EINVAL, "sfp_run_update: segment count changed");
    for (int s = 0; s < n_seg; ++s)
        if (seg[s].massless != r->segs[s].massless || seg[s].radiating != r->segs[s].radiating ||
            seg[s].bw != r->segs[s].bw || seg[s].ele_dest != r->segs[s].ele_dest ||
            seg[s].pos_dest != r->segs[s].pos_dest || seg[s].photon_dest != r->segs[s].photon_dest ||
            (!seg[s].massless && seg[s].spin != r->segs[s].spin))
            return fail(SFP_EINVAL, "sfp_run_update: segment roles changed");
    int rc = validate_segments(r->n_inst, r->insts.data(), n_seg, seg);
    if (rc) return rc;
    r->segs.assign(seg, seg + n_seg);
    rc = run_alloc_tiles(r);
    if (rc) return rc;
    return run_upload(r, nullptr, n_buffered);
}

// Runs of one instance: their field parameters into the module's constant
// bank on the run's stream, after the launches of every earlier call on the
// same module (which read the bank).  The guard holds the module's lock
// until the call has recorded its own launches (`done`).
struct cfield_guard {
    sfp_run* r;
    std::unique_lock<std::mutex> lk;
    explicit cfield_guard(sfp_run* run) : r(run) {
        if (r->cfield) lk = std::unique_lock<std::mutex>(r->mod->cf_mu);
    }
    int put() {
        if (!r->cfield) return SFP_OK;
        sfp_module* m = r->mod;
        if (!m->cf_done) SFP_CUDA(cudaEventCreateWithFlags(&m->cf_done, cudaEventDisableTiming));
        else SFP_CUDA(cudaStreamWaitEvent(r->s, m->cf_done, 0));
        SFP_CUDA(cudaMemcpyAsync(r->cfield, r->insts[0].field_params, r->cfield_bytes, cudaMemcpyDeviceToDevice, r->s));
        SFP_CUDA(cudaMemcpyAsync(r->ckeys, r->d_keys, 20 * sizeof(unsigned int), cudaMemcpyDeviceToDevice, r->s));
        return SFP_OK;
    }
    int done() {
        if (!r->cfield) return SFP_OK;
        SFP_CUDA(cudaEventRecord(r->mod->cf_done, r->s));
        return SFP_OK;
    }
};

// one step: book(prepare), massive, photon, scan + appends; ev (6 events)
// brackets the massive, the photon and the scan + appends kernels when given.
// mlong / plong: the group's steps all have SFP_TILE_MAX-long tiles, run by
// the autotuned long-tile kernel; else by the any-tile kernel
static int launch_unit(sfp_run* r, cudaStream_t s, cudaEvent_t* ev, bool mlong, bool plong) {
    int prep = 1 | (mlong ? 2 : 0) | (plong ? 4 : 0);  // the book kernel checks the tiles the launches assume
    void* a_book[] = {&r->d, &prep};
    void* a[] = {&r->d};
    SFP_CUDA(cudaLaunchKernel((const void*)r->k_book, dim3(1), dim3(256), a_book, 0, s));
    if (ev) SFP_CUDA(cudaEventRecord(ev[0], s));
    if (!r->mg.seg.empty()) {
        if (mlong)
            SFP_CUDA(cudaLaunchKernel((const void*)r->k_massive, dim3(r->grid_m), dim3(SFP_TILE_HOST), a, r->smem_m, s));
        else
            SFP_CUDA(cudaLaunchKernel((const void*)r->k_massive_t, dim3(r->grid_mt), dim3(SFP_TILE_HOST), a,
                                      r->smem_mt, s));
    }
    if (ev) SFP_CUDA(cudaEventRecord(ev[1], s));
    if (ev) SFP_CUDA(cudaEventRecord(ev[2], s));
    if (!r->pg.seg.empty()) {
        if (plong)
            SFP_CUDA(cudaLaunchKernel((const void*)r->k_photon, dim3(r->grid_p), dim3(SFP_TILE_HOST), a, r->smem_p, s));
        else
            SFP_CUDA(cudaLaunchKernel((const void*)r->k_photon_t, dim3(r->grid_pt), dim3(SFP_TILE_HOST), a,
                                      r->smem_pt, s));
    }
    if (ev) SFP_CUDA(cudaEventRecord(ev[3], s));
    if (ev) SFP_CUDA(cudaEventRecord(ev[4], s));
    if (!r->dseg.empty()) {
        SFP_CUDA(cudaLaunchKernel((const void*)r->k_scan, dim3(1), dim3(1024), a, 0, s));
        SFP_CUDA(cudaLaunchKernel((const void*)r->k_appends, dim3(r->grid_a), dim3(SFP_TILE_HOST), a, 0, s));
    }
    if (ev) SFP_CUDA(cudaEventRecord(ev[5], s));
    return SFP_OK;
}

static int launch_fold(sfp_run* r) {
    int prep = 0;
    void* a_book[] = {&r->d, &prep};
    SFP_CUDA(cudaLaunchKernel((const void*)r->k_book, dim3(1), dim3(256), a_book, 0, r->s));
    return SFP_OK;
}

int sfp_run_steps(sfp_run* r, int64_t nsteps, int graph_chunk, void* stream) {
    if (!r) return fail(SFP_EINVAL, "sfp_run_steps: NULL run");
    if (nsteps <= 0) return SFP_OK;
    cudaStream_t cs = as_stream(stream);
    SFP_CUDA(cudaEventRecord(r->ev_in, cs));
    SFP_CUDA(cudaStreamWaitEvent(r->s, r->ev_in, 0));
    cfield_guard cg(r);
    if (const int rc0 = cg.put()) return rc0;
    int64_t done = 0;
    const bool ml = long_tiles(r, r->mg.seg), pl = long_tiles(r, r->pg.seg);
    if (graph_chunk > 0 && nsteps >= graph_chunk) {
        const int key = graph_chunk * 4 + (ml ? 2 : 0) + (pl ? 1 : 0);
        auto it = r->graphs.find(key);
        if (it == r->graphs.end()) {
            cudaGraph_t g;
            SFP_CUDA(cudaStreamBeginCapture(r->s, cudaStreamCaptureModeThreadLocal));
            int rc = SFP_OK;
            for (int k = 0; k < graph_chunk && rc == SFP_OK; ++k) rc = launch_unit(r, r->s, nullptr, ml, pl);
            cudaError_t e = cudaStreamEndCapture(r->s, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return fail(SFP_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            cudaGraphExec_t ge;
            e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(SFP_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            it = r->graphs.emplace(key, ge).first;
        }
        for (; done + graph_chunk <= nsteps; done += graph_chunk) SFP_CUDA(cudaGraphLaunch(it->second, r->s));
    }
    for (; done < nsteps; ++done) {
        int rc = launch_unit(r, r->s, nullptr, ml, pl);
        if (rc) return rc;
    }
    int rc = launch_fold(r);
    if (rc) return rc;
    if ((rc = cg.done())) return rc;
    SFP_CUDA(cudaEventRecord(r->ev_out, r->s));
    SFP_CUDA(cudaStreamWaitEvent(cs, r->ev_out, 0));
    return SFP_OK;
}

int sfp_run_steps_timed(sfp_run* r, int64_t nsteps, float* kernel_ms, void* stream) {
    if (!r || !kernel_ms) return fail(SFP_EINVAL, "sfp_run_steps_timed: NULL argument");
    if (nsteps <= 0) return SFP_OK;
    cudaStream_t cs = as_stream(stream);
    SFP_CUDA(cudaEventRecord(r->ev_in, cs));
    SFP_CUDA(cudaStreamWaitEvent(r->s, r->ev_in, 0));
    cfield_guard cg(r);
    if (const int rc0 = cg.put()) return rc0;
    std::vector<cudaEvent_t> ev(6 * nsteps, nullptr);
    int rc = SFP_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = fail(SFP_ECUDA, "cudaEventCreate");
    const bool ml = long_tiles(r, r->mg.seg), pl = long_tiles(r, r->pg.seg);
    for (int64_t k = 0; k < nsteps && rc == SFP_OK; ++k) rc = launch_unit(r, r->s, &ev[6 * k], ml, pl);
    if (rc == SFP_OK) rc = launch_fold(r);
    if (rc == SFP_OK) rc = cg.done();
    if (rc == SFP_OK && cudaStreamSynchronize(r->s) != cudaSuccess) rc = fail(SFP_ECUDA, "synchronize");
    const bool has[3] = {!r->mg.seg.empty(), !r->pg.seg.empty(), !r->dseg.empty()};
    for (int64_t k = 0; k < nsteps && rc == SFP_OK; ++k)
        for (int j = 0; j < 3 && rc == SFP_OK; ++j) {
            kernel_ms[3 * k + j] = 0.0f;
            if (has[j] && cudaEventElapsedTime(&kernel_ms[3 * k + j], ev[6 * k + 2 * j], ev[6 * k + 2 * j + 1]) !=
                              cudaSuccess)
                rc = fail(SFP_ECUDA, "elapsed");
        }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (rc) return rc;
    SFP_CUDA(cudaEventRecord(r->ev_out, r->s));
    SFP_CUDA(cudaStreamWaitEvent(cs, r->ev_out, 0));
    return SFP_OK;
}

int sfp_run_sync_positions(sfp_run* r, void* stream) {
    if (!r) return fail(SFP_EINVAL, "sfp_run_sync_positions: NULL run");
    if (r->pg.seg.empty()) return SFP_OK;
    cudaStream_t cs = as_stream(stream);
    SFP_CUDA(cudaEventRecord(r->ev_in, cs));
    SFP_CUDA(cudaStreamWaitEvent(r->s, r->ev_in, 0));
    void* a[] = {&r->d};
    SFP_CUDA(cudaLaunchKernel((const void*)r->k_sync, dim3(4 * sm_count()), dim3(256), a, 0, r->s));
    SFP_CUDA(cudaLaunchKernel((const void*)r->k_epoch, dim3(1), dim3(32), a, 0, r->s));
    SFP_CUDA(cudaEventRecord(r->ev_out, r->s));
    SFP_CUDA(cudaStreamWaitEvent(cs, r->ev_out, 0));
    return SFP_OK;
}

int sfp_run_read_state(sfp_run* r, sfp_run_state* state, int64_t* n_buffered, void* stream) {
    if (!r || !state) return fail(SFP_EINVAL, "sfp_run_read_state: NULL argument");
    (void)stream;
    sfp_step_state st;
    std::vector<long long> nb(r->n_seg);
    SFP_CUDA(cudaMemcpyAsync(&st, r->h.st, sizeof(st), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(nb.data(), r->h.n_buffered, r->n_seg * sizeof(long long), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    note_counts(r, nb.data());
    if (n_buffered) std::copy(nb.begin(), nb.end(), n_buffered);
    state->t = st.t;
    state->step = st.step;
    state->halted = st.halted;
    state->error = st.error;
    state->particle_steps = st.particle_steps;
    state->appends_pending = st.append_wait;
    state->pad = 0;
    return SFP_OK;
}

int sfp_run_clear_halt(sfp_run* r, void* stream) {
    if (!r) return fail(SFP_EINVAL, "NULL run");
    (void)stream;
    sfp_step_state st;
    SFP_CUDA(cudaMemcpyAsync(&st, r->h.st, sizeof(st), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    if (st.append_wait)
        return fail(SFP_EINVAL, "sfp_run_clear_halt: a step waits for room for its children; finish it with "
                                "sfp_run_resume");
    st.halted = 0;
    st.skip = 1;
    SFP_CUDA(cudaMemcpyAsync(r->h.st, &st, sizeof(st), cudaMemcpyHostToDevice, r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    return SFP_OK;
}

int sfp_run_pending_need(sfp_run* r, int64_t* need) {
    if (!r || !need) return fail(SFP_EINVAL, "sfp_run_pending_need: NULL argument");
    sfp_step_state st;
    std::vector<long long> nb(r->n_seg), ns(r->n_seg);
    std::vector<unsigned long long> ap(r->n_seg);
    SFP_CUDA(cudaMemcpyAsync(&st, r->h.st, sizeof(st), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(nb.data(), r->h.n_buffered, r->n_seg * sizeof(long long), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(ns.data(), r->h.n_buf_step, r->n_seg * sizeof(long long), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(ap.data(), r->h.appended, r->n_seg * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    for (int s = 0; s < r->n_seg; ++s) need[s] = st.append_wait ? ns[s] + (long long)ap[s] : nb[s];
    return SFP_OK;
}

int sfp_run_resume(sfp_run* r, void* stream) {
    if (!r) return fail(SFP_EINVAL, "sfp_run_resume: NULL run");
    sfp_step_state st;
    std::vector<long long> ns(r->n_seg);
    std::vector<unsigned long long> ap(r->n_seg);
    SFP_CUDA(cudaMemcpyAsync(&st, r->h.st, sizeof(st), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(ns.data(), r->h.n_buf_step, r->n_seg * sizeof(long long), cudaMemcpyDeviceToHost, r->s));
    SFP_CUDA(cudaMemcpyAsync(ap.data(), r->h.appended, r->n_seg * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    if (!st.append_wait) return SFP_OK;
    // the appends kernel runs only when every destination holds its children
    for (int c : r->dseg)
        if (ns[c] + (long long)ap[c] > r->segs[c].capacity)
            return fail(SFP_EINVAL, "sfp_run_resume: segment " + std::to_string(c) +
                                        " still lacks room for the children of the stopped step");
    st.append_wait = 0;
    st.halted = 0;
    st.skip = 0;
    cudaStream_t cs = as_stream(stream);
    SFP_CUDA(cudaEventRecord(r->ev_in, cs));
    SFP_CUDA(cudaStreamWaitEvent(r->s, r->ev_in, 0));
    SFP_CUDA(cudaMemcpyAsync(r->h.st, &st, sizeof(st), cudaMemcpyHostToDevice, r->s));
    SFP_CUDA(cudaStreamSynchronize(r->s));
    cfield_guard cg(r);
    if (const int rc0 = cg.put()) return rc0;
    void* a[] = {&r->d};
    SFP_CUDA(cudaLaunchKernel((const void*)r->k_appends, dim3(r->grid_a), dim3(SFP_TILE_HOST), a, 0, r->s));
    int rc = launch_fold(r);
    if (rc) return rc;
    if ((rc = cg.done())) return rc;
    SFP_CUDA(cudaEventRecord(r->ev_out, r->s));
    SFP_CUDA(cudaStreamWaitEvent(cs, r->ev_out, 0));
    return SFP_OK;
}

int sfp_run_destroy(sfp_run* r) {
    if (!r) return SFP_OK;
    if (r->s) cudaStreamSynchronize(r->s);
    for (auto& kv : r->graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(r->d_keys);
    cudaFree((void*)r->h.seg);
    cudaFree((void*)r->h.inst);
    cudaFree(r->mg.d_seg);
    cudaFree(r->pg.d_seg);
    cudaFree(r->mg.d_start);
    cudaFree(r->pg.d_start);
    cudaFree((void*)r->h.dseg);
    cudaFree(r->h.n_buffered);
    cudaFree(r->h.appended);
    cudaFree(r->h.n_buf_step);
    for (sfp_group_dev* G : {&r->h.mg, &r->h.pg}) {
        cudaFree(G->tile_cnt);
        cudaFree(G->super_cnt);
        cudaFree(G->super_pre);
    }
    cudaFree(r->h.st);
    cudaFree((void*)r->h.pair_bound);
    cudaFree(r->d);
    if (r->ev_in) cudaEventDestroy(r->ev_in);
    if (r->ev_out) cudaEventDestroy(r->ev_out);
    if (r->s) cudaStreamDestroy(r->s);
    delete r;
    return SFP_OK;
}

}  // extern "C"
