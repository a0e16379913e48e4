// bh_variant.cuh -- the kernels and their launch sequences, compiled once
// per arithmetic variant: the including file defines BH_VARIANT (the
// namespace) and is compiled with the variant's flags (bh_fp64.cu with
// --fmad=false, the reference's separate roundings; bh_fp64fma.cu with
// FMA contraction; bh_mixed.cu with BH_REAL = float).  bh_abi.cu dispatches the C ABI to one of them.
//
// One thread per cell / face / edge; patches are the unit of parallel work
// (blockIdx.y walks a patch list, blockIdx.x the items of one patch), so a
// CTA never straddles two patches and all per-patch arrays are read with
// unit stride along the reference's fastest index k.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cstring>
#include "bhgpu.h"
#include "bh_items.cuh"
#include "bh_init.cuh"
#include "bh_tc.cuh"
#include "bh_api.h"

#ifndef BH_VARIANT
#error "define BH_VARIANT before including bh_variant.cuh"
#endif
// arithmetic type of reconstruction, face fluxes and sources (FP64 unless
// the including file asks for the mixed variant)
#ifndef BH_REAL
#define BH_REAL double
#endif

namespace BH_VARIANT {
using namespace bh;

namespace {

constexpr int TPB = 128;
// minimum resident CTAs per SM requested from ptxas for the heavy kernels
// (caps their registers per thread); tuned on B200
// (sweeps on the 128^3 box: con2prim and floors run fastest at 6 CTAs of
// 128 threads per SM, the FP64 flux kernel at 4 -- the FP32 one of the
// mixed variant at 6, set in bh_mixed.cu -- and the update at 4)
#ifndef BH_MINB_PRIMS
#define BH_MINB_PRIMS 6
#endif
#ifndef BH_MINB_GHOST
#define BH_MINB_GHOST 6
#endif
#ifndef BH_MINB_FLUX
#define BH_MINB_FLUX 4
#endif
#ifndef BH_MINB_FLOORS
#define BH_MINB_FLOORS 6
#endif
#ifndef BH_MINB_UPDATE
#define BH_MINB_UPDATE 4
#endif

// ---- thin kernels: thread index -> item --------------------------------
#define ITEM(n) int e = blockIdx.x * blockDim.x + threadIdx.x; if (e >= (n)) return
#define BATCH int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; if (q >= n) return

__global__ void k_geometry(Pool P, const int32_t* list) { ITEM(NC); geometry_item(P, list[blockIdx.y], e); }

__global__ void k_metric(KP k, const double* r, const double* th, int64_t n, double* out) { BATCH; metric_item(k, r, th, q, out); }
__global__ void k_ptoc(KP k, const double* W, const double* r, const double* th, int64_t n, double* U, double* Wd) {
    BATCH; ptoc_item(k, W, r, th, n, q, U, Wd, nullptr);
}
__global__ void k_ctop(KP k, const double* U, const double* r, const double* th, int64_t n, double* W, double* Wd,
                       int32_t* st, int32_t* it, int32_t* pa) {
    BATCH; ctop_item(k, U, r, th, n, q, W, Wd, st, it, pa);
}
__global__ void k_ctop_guess(KP k, const double* U, const double* r, const double* th, int64_t n, const double* xi0,
                             double* W, double* Wd, int32_t* st, int32_t* it, int32_t* pa) {
    BATCH; ctop_guess_item(k, U, r, th, n, q, xi0, W, Wd, st, it, pa);
}
__global__ void k_ctop_pre(KP k, const double* U, const double* r, const double* th, int64_t n, double* pre) {
    BATCH; ctop_pre_item(k, U, r, th, n, q, pre);
}
// the learned con2prim start for every cell, the network on the tensor
// cores (bh_tc.cuh): one tile of 128 cells per pass, the CTAs persistent
// over the tiles (grid = the resident CTAs, at most 8 per SM so that their
// tensor memory always fits).  Per cell: the metric, con2prim's preamble
// (conserved.cpp:135-150), the features and the network; xi0 = D exp(y0),
// NaN where a feature is not finite.  The work per cell is nearly uniform,
// so the CTA-wide steps of the network cost little; con2prim's own
// iterations, whose count varies from cell to cell, run afterwards in
// k_ctop_guess (one thread per cell, no barriers).
__global__ void __launch_bounds__(bh_tc::ROWS, 4)
    k_guess_tc(KP k, const __nv_bfloat16* wb, const float* norm, const double* U, const double* r,
               const double* th, int64_t n, double* xi0_out, int32_t* err) {
    __shared__ bh_tc::Smem s;
    const int t = threadIdx.x;
    bh_tc::stage_weights(s, wb, norm);
    if (t == 0) bh_tc::mbar_init(&s.mbar);
    if (t < 32) bh_tc::tmem_alloc(&s.tmem);
    bh_tc::fence_before();
    __syncthreads();
    bh_tc::fence_after();
    const uint32_t tmem = s.tmem;
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntile = (n + bh_tc::ROWS - 1) / bh_tc::ROWS;
    for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int64_t q = tile * bh_tc::ROWS + t;
        const bool in = q < n;
        double p5[5] = {NAN, NAN, NAN, NAN, NAN};
        float xn[bh_tc::NI];
        bool valid = false;
        if (in) {
            Cons c;
            c.D = U[q]; c.tau = U[4 * n + q];
            for (int d = 0; d < 3; d++) { c.S[d] = U[(1 + d) * n + q]; c.B[d] = U[(5 + d) * n + q]; }
            Met mc;
            met_comp(k.tree, r[q], th[q], mc);
            Prim w0;
            bool dom0 = false;
            ctop(k.gamma, 0, k.tol, mc, c, w0, dom0, nullptr, NAN, p5);   // the preamble only
            float x[bh_tc::NI];
            bh_tc::features(p5, r[q], x);
            valid = true;
            for (int i = 0; i < bh_tc::NI; i++) {
                valid &= isfinite(x[i]);
                xn[i] = (x[i] - s.norm[i]) * s.norm[bh_tc::NI + i];
            }
        }
        float y0 = 0.0f;
        if (!bh_tc::network(s, tmem, phase, xn, valid, y0)) { ok = false; break; }
        if (in) xi0_out[q] = valid ? p5[0] * exp((double)y0) : NAN;
    }
    if (!ok) {
        // an MMA did not complete in time: record it, give it one more bounded
        // wait, then release the tensor memory all the same
        bh_tc::mbar_wait(&s.mbar, phase ^ 1u);
        if (t == 0) atomicOr(err, BH_ERR_TIMEOUT);
    }
    bh_tc::fence_before();
    __syncthreads();
    bh_tc::fence_after();
    if (t < 32) bh_tc::tmem_free(tmem);
}
__global__ void k_hlld(KP k, const double* WL, const double* WR, const double* UL, const double* UR, const double* r,
                       const double* th, int dim, int64_t n, double* F, double* cts) {
    BATCH; hlld_item(k, WL, WR, UL, UR, r, th, dim, n, q, F, cts);
}
__global__ void k_reconfp(KP kp, Pool P, int dim, int lim, int64_t n, double* Lo, double* Ro) {
    ITEM(NFACE); reconfp_item<BH_REAL>(kp, P, blockIdx.y, dim, e, lim, n, Lo, Ro);
}
// patch::fluxcomp: one face per thread, direction blockIdx.z; with the
// per-cell scratch, k_aux first fills it for every cell of every patch
__global__ void __launch_bounds__(TPB, BH_MINB_FLUX) k_flux(KP kp, Pool P, const int32_t* list) {
    ITEM(NFACE); flux_item<BH_REAL>(kp, P, list[blockIdx.y], blockIdx.z, e);
}
__global__ void k_aux(KP kp, Pool P, const int32_t* list) { ITEM(NC); aux_item<BH_REAL>(kp, P, list[blockIdx.y], e); }
// the kernels the autotuner sets: one instantiation per candidate number
// of resident CTAs per SM (MB), which caps their registers per thread
template <int MB>
__global__ void __launch_bounds__(TPB, MB) k_flux_aux(KP kp, Pool P, const int32_t* list) {
    ITEM(NFACE); flux_item<BH_REAL, true>(kp, P, list[blockIdx.y], blockIdx.z, e);
}
__global__ void k_emf(Pool P, const int32_t* list) { ITEM(N_EDGE); emf_item(P, list[blockIdx.y], e); }
__global__ void k_bfupdate(Pool P, const int32_t* list, const double* dtp) {
    ITEM(N_BUP); bfupdate_item(P, list[blockIdx.y], e, *dtp);
}
__global__ void k_f2cb(KP kp, Pool P, const int32_t* list) { ITEM(N_F2C); f2cb_item(kp, P, list[blockIdx.y], e); }
__global__ void k_div_source(KP kp, Pool P, const int32_t* list, double* dv, double* sv) {
    ITEM(N_INT); div_source_item<BH_REAL>(kp, P, list[blockIdx.y], e, dv, sv);
}
// f2cB + RK update: CTAs [0, UPD_INT) take the interior cells, the others
// the shell cells, so no warp mixes the two
constexpr int UPD_INT = N_INT / TPB;
constexpr int UPD_BLOCKS = UPD_INT + (N_SHELL + TPB - 1) / TPB;
template <int MB>
__global__ void __launch_bounds__(TPB, MB) k_update(KP kp, Pool P, const int32_t* list, const double* dtp, int stage) {
    int p = list[blockIdx.y];
    if ((int)blockIdx.x < UPD_INT) {
        update_interior_item<BH_REAL>(kp, P, p, blockIdx.x * TPB + threadIdx.x, *dtp, stage);
    } else {
        int e = (blockIdx.x - UPD_INT) * TPB + threadIdx.x;
        if (e < N_SHELL) update_shell_item(kp, P, p, e);
    }
}
// amrtree::ghosts strip fill: one copied double per thread, then the
// prolonged cells (CTAs whose slot has another neighbour kind exit at once)
__global__ void k_ghost_copy(Pool P, const int32_t* list) { ITEM(2 * N_COPY); ghost_copy_item(P, list[blockIdx.y], e); }
__global__ void k_ghost_prolong(KP kp, Pool P, const int32_t* list) {
    ITEM(N_STRIP); ghost_prolong_item(kp, P, list[blockIdx.y], e);
}
__global__ void k_ghost_ctop(KP kp, Pool P, const int32_t* list) { ITEM(NC); ghost_ctop_item(kp, P, list[blockIdx.y], e); }
__global__ void __launch_bounds__(TPB, BH_MINB_PRIMS) k_prims(KP kp, Pool P, const int32_t* list, int ghost_first) {
    ITEM(NC); prims_item(kp, P, list[blockIdx.y], e, ghost_first);
}
template <int MB>
__global__ void __launch_bounds__(TPB, MB) k_prims_interior(KP kp, Pool P, const int32_t* list) {
    ITEM(N_INT); prims_interior_item(kp, P, list[blockIdx.y], e);
}
template <int MB>
__global__ void __launch_bounds__(TPB, MB) k_prims_ghost(KP kp, Pool P, const int32_t* list) {
    ITEM(N_GHOST); prims_ghost_item(kp, P, list[blockIdx.y], e);
}
template <int MB>
__global__ void __launch_bounds__(TPB, MB) k_floors(KP kp, Pool P, const int32_t* list) {
    ITEM(N_INT); floors_item(kp, P, list[blockIdx.y], e);
}

// ---- AMR regrid: flags (one CTA per leaf patch, OR-reduced over its
// cells), refine and ccrstr (one thread per new cell; plan rows are
// parent + 8 children), B_init (one thread per face) -----------------------
__global__ void k_regrid_flags(Pool P, const int32_t* list, const int32_t* lvl, uint8_t* flags) {
    int p = list[blockIdx.x];
    int L = lvl[p];
    bool ref = false, nf = false;
    for (int c = threadIdx.x; c < N_INT; c += blockDim.x) regrid_cell(P, p, L, c, ref, nf);
    int any_ref = __syncthreads_or(ref);
    int any_nf = __syncthreads_or(nf);
    if (threadIdx.x == 0) flags[p] = regrid_patch_flags(L, any_ref != 0, any_nf != 0);
}
__global__ void __launch_bounds__(TPB, BH_MINB_PRIMS) k_refine(KP kp, Pool P, const int32_t* plan) {
    ITEM(N_INT);
    const int32_t* row = plan + (blockIdx.y / 8) * 9;
    int h = blockIdx.y % 8;
    refine_item(kp, P, row[0], row[1 + h], h, e);
}
__global__ void __launch_bounds__(TPB, BH_MINB_PRIMS) k_ccrstr(KP kp, Pool P, const int32_t* plan) {
    ITEM(N_INT);
    const int32_t* row = plan + blockIdx.y * 9;
    ccrstr_item(kp, P, row[0], row + 1, e);
}
__global__ void k_b_init(Pool P, const int32_t* list) { ITEM(3 * NF); b_init_item(P, list[blockIdx.y], e); }
// B_init of the patches in columns [col0, col0 + ncol) of the plan rows
__global__ void k_b_init_rows(Pool P, const int32_t* plan, int col0, int ncol) {
    ITEM(3 * NF);
    b_init_item(P, plan[(blockIdx.y / ncol) * 9 + col0 + blockIdx.y % ncol], e);
}

// ---- analysis::analyser: one CTA per leaf patch sums its cells (each
// thread a fixed stride of cells, then the warps in order), a second kernel
// sums the patches in order: a fixed summation order, so reruns agree
constexpr int ANL_TPB = 256;
__global__ void __launch_bounds__(ANL_TPB) k_analysis(KP kp, Pool P, const int32_t* leaves, AParams A,
                                                     double* partial) {
    int p = leaves[blockIdx.x];
    double acc[BH_NQ];
    for (int q = 0; q < BH_NQ; q++) acc[q] = 0.0;
    for (int c = threadIdx.x; c < N_INT; c += ANL_TPB) analysis_cell(kp, P, p, c, A, acc);
    __shared__ double red[BH_NQ][ANL_TPB / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < BH_NQ; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < BH_NQ) {
        double s = 0.0;
        for (int w = 0; w < ANL_TPB / 32; w++) s += red[threadIdx.x][w];
        partial[(size_t)blockIdx.x * BH_NQ + threadIdx.x] = s;
    }
}
__global__ void k_analysis_sum(const double* partial, int n, double* out) {
    int q = threadIdx.x;
    if (q >= BH_NQ) return;
    double s = 0.0;
    for (int i = 0; i < n; i++) s += partial[(size_t)i * BH_NQ + q];
    out[q] = s;
}

// ---- torus initial data: max-reductions on the bit patterns of
// non-negative doubles (they order like the values), so they are exact ----
__device__ inline void atomic_max_nonneg(unsigned long long* m, double v) {
    if (v >= 0.0) atomicMax(m, (unsigned long long)__double_as_longlong(v));
}
__global__ void k_floor_all(KP kp, Pool P, const int32_t* list) { ITEM(NC); floor_cell(kp, P, list[blockIdx.y], e); }
__global__ void k_fm_scalars(KP kp, double r_max, double r_in, TorusScalars* out) {
    *out = fm_scalars(kp.tree, kp.gamma, r_max, r_in);
}
__global__ void k_fm_rho_max(KP kp, Pool P, const int32_t* list, const TorusScalars* s, unsigned long long* m) {
    ITEM(N_INT);
    atomic_max_nonneg(m, fm_cell_rho(kp, P, list[blockIdx.y], e, *s));
}
__global__ void k_fm_prims(KP kp, Pool P, const int32_t* list, const TorusScalars* s, const unsigned long long* m) {
    ITEM(N_INT);
    fm_cell_prims(kp, P, list[blockIdx.y], e, *s, 1.0 / __longlong_as_double((long long)*m));
}
__global__ void k_interior_rho_max(Pool P, const int32_t* list, unsigned long long* m) {
    ITEM(N_INT);
    int p = list[blockIdx.y];
    atomic_max_nonneg(m, Wv(P, p, 0)[lindx(e / 256, (e / 16) % 16, e % 16)]);
}
__global__ void k_bpot(Pool P, const int32_t* list, const unsigned long long* m) {
    ITEM(N_F2C);
    bpot_item(P, list[blockIdx.y], e, __longlong_as_double((long long)*m));
}
__global__ void k_ptoc_interior(KP kp, Pool P, const int32_t* list) {
    ITEM(N_INT); ptoc_interior_item(kp, P, list[blockIdx.y], e);
}

// constrans::maxdivB: one CTA per patch, max-reduction in shared memory
__global__ void k_maxdivb(Pool P, double* out) {
    int p = blockIdx.x;
    double m = 0.0;
    for (int e = threadIdx.x; e < N_BUP; e += blockDim.x) m = smax(m, maxdivb_item(P, p, e));
    __shared__ double red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = smax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[p] = red[0];
}

// rk2integrator::dtcomp: per-cell candidates, warp and block minimum, then
// one atomicMin per block on the 64-bit pattern (positive doubles order
// like their bit patterns, and min is exact, so the result is deterministic)
__global__ void k_dt_init(double* dt) { *dt = DBL_BIG; }
__global__ void k_dtcomp(KP kp, Pool P, const int32_t* list, double cfl, double* dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double best = c < N_INT ? dt_item(kp, P, list[blockIdx.y], c, cfl) : DBL_BIG;
    unsigned long long b = __double_as_longlong(best);
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        b = x < b ? x : b;
    }
    __shared__ unsigned long long red[TPB / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = red[w] < b ? red[w] : b;
        b = red[0] < b ? red[0] : b;
        atomicMin((unsigned long long*)dt, b);
    }
}

// ==========================================================================
// host helpers
// ==========================================================================
inline cudaStream_t S(void* s) { return (cudaStream_t)s; }
inline int launched() { return cudaGetLastError() == cudaSuccess ? BH_OK : BH_ECUDA; }
inline bool bad_pool(const bh_pool* p) {
    return !p || p->npatch <= 0 || !p->all || p->nall < 0 || p->nall > p->npatch || p->nleaf < 0 ||
           p->nleaf > p->npatch;
}
// entries of pool->all: the patches the flux/CT/update/floors kernels visit
inline int nall(const bh_pool* p) { return p->nall > 0 ? p->nall : p->npatch; }
inline dim3 grid2(int items, int npatch, int z = 1) { return dim3((items + TPB - 1) / TPB, npatch, z); }

// ---- launch bounds chosen by the autotuner --------------------------------
// The current choice per tuned kernel (resident 128-thread CTAs per SM asked
// of ptxas), per process and per variant, initially the compiled-in
// default; launches made after bh_tune_set (and graphs captured after it)
// use the new choice.  The candidate lists are bh_tune_cands (bh_api.h);
// each switch below instantiates exactly those.
int g_minb[BH_TUNE_NKERNEL] = {BH_MINB_FLUX, BH_MINB_UPDATE, BH_MINB_PRIMS, BH_MINB_GHOST, BH_MINB_FLOORS};

#define BH_TUNED_CASE(K, MB, GRID, ST, ...) \
    case MB: K<MB><<<GRID, TPB, 0, ST>>>(__VA_ARGS__); break;
// flux and update: 3, 4, 5, 6; con2prim (interior, ghost) and floors: 4, 6, 8
#define BH_LAUNCH_3456(K, WHICH, GRID, ST, ...)                                                            \
    switch (g_minb[WHICH]) {                                                                             \
        BH_TUNED_CASE(K, 3, GRID, ST, __VA_ARGS__) BH_TUNED_CASE(K, 4, GRID, ST, __VA_ARGS__)            \
        BH_TUNED_CASE(K, 5, GRID, ST, __VA_ARGS__) BH_TUNED_CASE(K, 6, GRID, ST, __VA_ARGS__)            \
        default: return BH_EINVAL;                                                                       \
    }
#define BH_LAUNCH_468(K, WHICH, GRID, ST, ...)                                                             \
    switch (g_minb[WHICH]) {                                                                             \
        BH_TUNED_CASE(K, 4, GRID, ST, __VA_ARGS__) BH_TUNED_CASE(K, 6, GRID, ST, __VA_ARGS__)            \
        BH_TUNED_CASE(K, 8, GRID, ST, __VA_ARGS__)                                                       \
        default: return BH_EINVAL;                                                                       \
    }

}  // namespace

int tune_set(int32_t kernel, int32_t ctas) {
    if (!bh_tune_valid(kernel, ctas)) return BH_EINVAL;
    g_minb[kernel] = ctas;
    return BH_OK;
}
int tune_get(int32_t kernel, int32_t* ctas) {
    if (kernel < 0 || kernel >= BH_TUNE_NKERNEL || !ctas) return BH_EINVAL;
    *ctas = g_minb[kernel];
    return BH_OK;
}

int metric_comp(const bh_params* P, const double* r, const double* th, int64_t n, double* out, void* stream) {
    if (!P || n < 0) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_metric<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), r, th, n, out);
    return launched();
}
int ptoc(const bh_params* P, const double* W, const double* r, const double* th, int64_t n, double* U, double* Wd,
            void* stream) {
    if (!P || n < 0) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_ptoc<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), W, r, th, n, U, Wd);
    return launched();
}
int ctop(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, double* W, double* Wd,
            int32_t* status, int32_t* iters, int32_t* path, void* stream) {
    if (!P || n < 0 || (n > 0 && !status)) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_ctop<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), U, r, th, n, W, Wd, status, iters, path);
    return launched();
}
int hlld(const bh_params* P, const double* WL, const double* WR, const double* UL, const double* UR,
            const double* r, const double* th, int32_t dim, int64_t n, double* F, double* ctspeed, void* stream) {
    if (!P || n < 0 || dim < 0 || dim > 2) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_hlld<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), WL, WR, UL, UR, r, th, dim, n, F,
                                                                    ctspeed);
    return launched();
}

int geometry(const bh_pool* pool, void* stream) {
    if (bad_pool(pool)) return BH_EINVAL;
    k_geometry<<<grid2(NC, nall(pool)), TPB, 0, S(stream)>>>(pool_of(pool), pool->all);
    return launched();
}
int reconfp(const bh_params* P, const bh_pool* pool, int32_t dim, int32_t limiter, double* L, double* R,
               void* stream) {
    if (!P || bad_pool(pool) || dim < 0 || dim > 2) return BH_EINVAL;
    int64_t n = (int64_t)pool->npatch * NFACE;
    k_reconfp<<<grid2(NFACE, pool->npatch), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), dim, limiter, n, L, R);
    return launched();
}
int fluxcomp(const bh_params* P, const bh_pool* pool, void* stream) {
    if (!P || bad_pool(pool)) return BH_EINVAL;
    if (pool->aux) {
        k_aux<<<grid2(NC, nall(pool)), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->all);
        BH_LAUNCH_3456(k_flux_aux, BH_TUNE_FLUX, grid2(NFACE, nall(pool), 3), S(stream), kp_of(P), pool_of(pool),
                       pool->all)
    } else {
        k_flux<<<grid2(NFACE, nall(pool), 3), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->all);
    }
    return launched();
}
int emfcomp(const bh_pool* pool, void* stream) {
    if (bad_pool(pool)) return BH_EINVAL;
    k_emf<<<grid2(N_EDGE, nall(pool)), TPB, 0, S(stream)>>>(pool_of(pool), pool->all);
    return launched();
}
int bfupdate(const bh_pool* pool, const double* dt_dev, void* stream) {
    if (bad_pool(pool) || !dt_dev) return BH_EINVAL;
    k_bfupdate<<<grid2(N_BUP, nall(pool)), TPB, 0, S(stream)>>>(pool_of(pool), pool->all, dt_dev);
    return launched();
}
int f2cb(const bh_params* P, const bh_pool* pool, void* stream) {
    if (!P || bad_pool(pool)) return BH_EINVAL;
    k_f2cb<<<grid2(N_F2C, nall(pool)), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->all);
    return launched();
}
int maxdivb(const bh_pool* pool, double* out, void* stream) {
    if (bad_pool(pool) || !out) return BH_EINVAL;
    k_maxdivb<<<pool->npatch, 256, 0, S(stream)>>>(pool_of(pool), out);
    return launched();
}
int div_source(const bh_params* P, const bh_pool* pool, double* div, double* src, void* stream) {
    if (!P || bad_pool(pool) || !div || !src) return BH_EINVAL;
    k_div_source<<<grid2(N_INT, nall(pool)), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->all, div,
                                                                               src);
    return launched();
}
int ghosts(const bh_params* P, const bh_pool* pool, const int32_t* patches, int32_t n, void* stream) {
    if (!P || bad_pool(pool) || n < 0 || (n > 0 && !patches)) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_ghost_copy<<<grid2(2 * N_COPY, n), TPB, 0, S(stream)>>>(pool_of(pool), patches);
    k_ghost_prolong<<<grid2(N_STRIP, n), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), patches);
    k_ghost_ctop<<<grid2(NC, n), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), patches);
    return launched();
}
int prims(const bh_params* P, const bh_pool* pool, void* stream) {
    if (!P || bad_pool(pool)) return BH_EINVAL;
    if (pool->nleaf == 0) return BH_OK;
    k_prims<<<grid2(NC, pool->nleaf), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->leaves, 0);
    return launched();
}
// the fused ghost fill + reconstruction; status (may be null) is the
// per-cell scratch of the interior-first variant
int ghosts_prims_status(const bh_params* P, const bh_pool* pool, uint8_t* status, void* stream) {
    if (!P || bad_pool(pool)) return BH_EINVAL;
    if (pool->nleaf == 0) return BH_OK;
    Pool pv = pool_of(pool);
    pv.status = status;
    k_ghost_copy<<<grid2(2 * N_COPY, pool->nleaf), TPB, 0, S(stream)>>>(pv, pool->leaves);
    k_ghost_prolong<<<grid2(N_STRIP, pool->nleaf), TPB, 0, S(stream)>>>(kp_of(P), pv, pool->leaves);
    if (status && pool->leafmask) {
        BH_LAUNCH_468(k_prims_interior, BH_TUNE_PRIMS_INTERIOR, grid2(N_INT, pool->nleaf), S(stream), kp_of(P), pv,
                      pool->leaves)
        BH_LAUNCH_468(k_prims_ghost, BH_TUNE_PRIMS_GHOST, grid2(N_GHOST, pool->nleaf), S(stream), kp_of(P), pv,
                      pool->leaves)
    } else {
        k_prims<<<grid2(NC, pool->nleaf), TPB, 0, S(stream)>>>(kp_of(P), pv, pool->leaves, 1);
    }
    return launched();
}
int ghosts_prims(const bh_params* P, const bh_pool* pool, void* stream) {
    return ghosts_prims_status(P, pool, pool ? pool->status : nullptr, stream);
}
int update(const bh_params* P, const bh_pool* pool, const double* dt_dev, int32_t stage, void* stream) {
    if (!P || bad_pool(pool) || !dt_dev || (stage != 0 && stage != 1)) return BH_EINVAL;
    BH_LAUNCH_3456(k_update, BH_TUNE_UPDATE, dim3(UPD_BLOCKS, nall(pool)), S(stream), kp_of(P), pool_of(pool),
                   pool->all, dt_dev, stage)
    return launched();
}
int floors(const bh_params* P, const bh_pool* pool, void* stream) {
    if (!P || bad_pool(pool)) return BH_EINVAL;
    BH_LAUNCH_468(k_floors, BH_TUNE_FLOORS, grid2(N_INT, nall(pool)), S(stream), kp_of(P), pool_of(pool), pool->all)
    return launched();
}
int ctop_guess(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, const double* xi0,
               double* W, double* Wd, int32_t* status, int32_t* iters, int32_t* path, void* stream) {
    if (!P || n < 0 || (n > 0 && (!U || !r || !th || !xi0 || !W || !status))) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_ctop_guess<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), U, r, th, n, xi0, W, Wd, status,
                                                                      iters, path);
    return launched();
}
int ctop_learned(const bh_params* P, const bh_mlp* m, const double* U, const double* r, const double* th,
                 int64_t n, double* xi0, double* W, double* Wd, int32_t* status, int32_t* iters, int32_t* path,
                 int32_t* err, void* stream) {
    if (!P || !m || !m->w || !m->wb || !err || n < 0 ||
        (n > 0 && (!U || !r || !th || !xi0 || !W || !status)))
        return BH_EINVAL;
    if (n == 0) return BH_OK;
    int dev = 0, nsm = 0;
    // 44 KB of static shared memory per CTA: ask for the largest carveout
    if (cudaFuncSetAttribute(k_guess_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
        cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BH_ECUDA;
    // CTAs per SM: the launch bounds (128 threads, 4 CTAs) cap the registers
    // so that 4 fit, 4 x 45 KB of shared memory fit, and 4 x 64 tensor-memory
    // columns fit in 512, so no CTA ever waits in tcgen05.alloc.  (The
    // occupancy calculator answered 1 for this kernel on B200, which left 3
    // of 4 slots idle; CTAs beyond the resident ones would only queue.)
    const int occ = 4;
    static_assert(4 <= bh_tc::MAX_CTAS_PER_SM, "tensor memory of the resident CTAs");
    const int64_t ntile = (n + bh_tc::ROWS - 1) / bh_tc::ROWS;
    const int64_t grid = ntile < (int64_t)nsm * occ ? ntile : (int64_t)nsm * occ;
    k_guess_tc<<<(unsigned)grid, bh_tc::ROWS, 0, S(stream)>>>(kp_of(P), (const __nv_bfloat16*)m->wb,
                                                            m->w + BH_MLP_NPARAM, U, r, th, n, xi0, err);
    if (cudaGetLastError() != cudaSuccess) return BH_ECUDA;
    k_ctop_guess<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), U, r, th, n, xi0, W, Wd, status,
                                                                      iters, path);
    return launched();
}
int ctop_pre(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, double* pre,
             void* stream) {
    if (!P || n < 0 || (n > 0 && (!U || !r || !th || !pre))) return BH_EINVAL;
    if (n == 0) return BH_OK;
    k_ctop_pre<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, S(stream)>>>(kp_of(P), U, r, th, n, pre);
    return launched();
}
int regrid_flags(const bh_params* P, const bh_pool* pool, const int32_t* lvl, uint8_t* flags, void* stream) {
    if (!P || bad_pool(pool) || !lvl || !flags) return BH_EINVAL;
    if (pool->nleaf == 0) return BH_OK;
    k_regrid_flags<<<pool->nleaf, 256, 0, S(stream)>>>(pool_of(pool), pool->leaves, lvl, flags);
    return launched();
}
int refine(const bh_params* P, const bh_pool* pool, const int32_t* plan, int32_t n, void* stream) {
    if (!P || bad_pool(pool) || n < 0 || (n > 0 && !plan)) return BH_EINVAL;
    if (n == 0) return BH_OK;
    if (n > 65535 / 8) return BH_ERANGE;
    k_refine<<<dim3(N_INT / TPB, n * 8), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), plan);
    k_b_init_rows<<<dim3((3 * NF + TPB - 1) / TPB, n * 8), TPB, 0, S(stream)>>>(pool_of(pool), plan, 1, 8);
    return launched();
}
int ccrstr(const bh_params* P, const bh_pool* pool, const int32_t* plan, int32_t n, void* stream) {
    if (!P || bad_pool(pool) || n < 0 || (n > 0 && !plan)) return BH_EINVAL;
    if (n == 0) return BH_OK;
    if (n > 65535) return BH_ERANGE;
    k_ccrstr<<<dim3(N_INT / TPB, n), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), plan);
    k_b_init_rows<<<dim3((3 * NF + TPB - 1) / TPB, n), TPB, 0, S(stream)>>>(pool_of(pool), plan, 0, 1);
    return launched();
}
int b_init(const bh_params* P, const bh_pool* pool, const int32_t* patches, int32_t n, void* stream) {
    if (!P || bad_pool(pool) || n < 0 || (n > 0 && !patches)) return BH_EINVAL;
    if (n == 0) return BH_OK;
    if (n > 65535) return BH_ERANGE;
    k_b_init<<<grid2(3 * NF, n), TPB, 0, S(stream)>>>(pool_of(pool), patches);
    return launched();
}
int analysis(const bh_params* P, const bh_pool* pool, const bh_analysis_params* A, double* partial, double* out,
             void* stream) {
    if (!P || bad_pool(pool) || !A || !partial || !out || !pool->Wd) return BH_EINVAL;
    if (pool->nleaf == 0) return BH_OK;
    AParams ap{A->hrz, A->rs, A->rho_min_full, A->rho_min_bundle};
    k_analysis<<<pool->nleaf, ANL_TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->leaves, ap, partial);
    k_analysis_sum<<<1, 32, 0, S(stream)>>>(partial, pool->nleaf, out);
    return launched();
}
// the initial-data sequence of main() (main.cpp:89-160) on every listed patch:
// out[5] (host) = l0, W_in, ln h at r_max, the torus' rho_max before
// normalisation, the global interior rho_max after fm_init
int torus_init(const bh_params* P, const bh_pool* pool, double r_max, double r_in, double* out, void* stream) {
    if (!P || bad_pool(pool) || !out) return BH_EINVAL;
    cudaStream_t st = S(stream);
    KP kp = kp_of(P);
    Pool pv = pool_of(pool);
    int n = nall(pool);
    TorusScalars* ds = nullptr;
    unsigned long long* dm = nullptr;
    if (cudaMallocAsync((void**)&ds, sizeof(TorusScalars), st) != cudaSuccess) return BH_ECUDA;
    if (cudaMallocAsync((void**)&dm, 2 * sizeof(unsigned long long), st) != cudaSuccess) {
        cudaFreeAsync(ds, st);
        return BH_ECUDA;
    }
    cudaMemsetAsync(dm, 0, 2 * sizeof(unsigned long long), st);
    k_floor_all<<<grid2(NC, n), TPB, 0, st>>>(kp, pv, pool->all);          // amrtree::amrtree, grid.cpp:191-205
    k_fm_scalars<<<1, 1, 0, st>>>(kp, r_max, r_in, ds);
    TorusScalars hs;
    cudaMemcpyAsync(&hs, ds, sizeof(hs), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    out[0] = hs.l0; out[1] = hs.W_in; out[2] = hs.lnh_max;
    double rho_fm = 0.0;
    if (hs.lnh_max > 0.0) {                                                   // initconds.cpp:425-429
        k_fm_rho_max<<<grid2(N_INT, n), TPB, 0, st>>>(kp, pv, pool->all, ds, dm);
        unsigned long long bits = 0;
        cudaMemcpyAsync(&bits, dm, sizeof(bits), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        memcpy(&rho_fm, &bits, sizeof(double));
        if (rho_fm >= 1e-14)                                                  // :481-484
            k_fm_prims<<<grid2(N_INT, n), TPB, 0, st>>>(kp, pv, pool->all, ds, dm);
    }
    out[3] = rho_fm;
    k_interior_rho_max<<<grid2(N_INT, n), TPB, 0, st>>>(pv, pool->all, dm + 1);   // main.cpp:99-108
    unsigned long long gbits = 0;
    cudaMemcpyAsync(&gbits, dm + 1, sizeof(gbits), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    double glmx;
    memcpy(&glmx, &gbits, sizeof(double));
    out[4] = glmx;
    int rc = BH_OK;
    if (glmx < 1e-14) {
        rc = BH_ERANGE;                                                       // main.cpp:109-112
    } else {
        if (glmx > 1e-10) {                                                   // B_pot_init :598
            k_bpot<<<grid2(N_F2C, n), TPB, 0, st>>>(pv, pool->all, dm + 1);
            k_f2cb<<<grid2(N_F2C, n), TPB, 0, st>>>(kp, pv, pool->all);
        }
        k_ptoc_interior<<<grid2(N_INT, n), TPB, 0, st>>>(kp, pv, pool->all);
    }
    cudaFreeAsync(ds, st);
    cudaFreeAsync(dm, st);
    int lr = launched();
    return lr ? lr : rc;
}
int dtcomp(const bh_params* P, const bh_pool* pool, double cfl, double* dt_dev, void* stream) {
    if (!P || bad_pool(pool) || !dt_dev) return BH_EINVAL;
    k_dt_init<<<1, 1, 0, S(stream)>>>(dt_dev);
    if (pool->nleaf > 0)
        k_dtcomp<<<grid2(N_INT, pool->nleaf), TPB, 0, S(stream)>>>(kp_of(P), pool_of(pool), pool->leaves,
                                                                             cfl, dt_dev);
    return launched();
}
int rkstg(const bh_params* P, const bh_pool* pool, const double* dt_dev, int32_t stage, const int32_t* waves,
             const int32_t* wave_off, int32_t nwave, void* stream) {
    if (!P || bad_pool(pool) || !dt_dev || nwave < 0 || (nwave > 1 && (!waves || !wave_off))) return BH_EINVAL;
    int rc;
    if (nwave <= 1) {
        rc = ghosts_prims(P, pool, stream);
    } else {
        for (int w = 0; w < nwave; w++) {
            rc = ghosts(P, pool, waves + wave_off[w], wave_off[w + 1] - wave_off[w], stream);
            if (rc) return rc;
        }
        rc = prims(P, pool, stream);
    }
    if (rc) return rc;
    if ((rc = fluxcomp(P, pool, stream))) return rc;
    if ((rc = emfcomp(pool, stream))) return rc;
    if ((rc = bfupdate(pool, dt_dev, stream))) return rc;
    return update(P, pool, dt_dev, stage, stream);
}
int step(const bh_params* P, const bh_pool* pool, double cfl, double* dt_dev, const int32_t* waves,
            const int32_t* wave_off, int32_t nwave, void* stream) {
    int rc;
    if ((rc = dtcomp(P, pool, cfl, dt_dev, stream))) return rc;
    if ((rc = rkstg(P, pool, dt_dev, 0, waves, wave_off, nwave, stream))) return rc;
    if ((rc = rkstg(P, pool, dt_dev, 1, waves, wave_off, nwave, stream))) return rc;
    return floors(P, pool, stream);
}

}  // namespace BH_VARIANT

// the corrected scheme's kernels, compiled in this variant's arithmetic
#include "bh_fixed.cuh"
