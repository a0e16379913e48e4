// bh_abi.cu -- the C ABI (include/bhgpu.h): argument checks and dispatch
// to the arithmetic variant bh_params.precision selects.
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include <new>
#include "bhgpu.h"
#include "bh_api.h"
#include "bh_phys.cuh"

namespace {
inline cudaStream_t S(void* s) { return (cudaStream_t)s; }
inline bool bad_pool(const bh_pool* p) { return !p || p->npatch <= 0 || !p->all; }
constexpr int NC_ = bh::NC;
// ---- library-owned scratch for bh_ghosts_prims_static ---------------------
// The con2prim outcome of every interior cell, BH_STATIC_MAX_PATCHES x 8000
// bytes, held by every GPU that loads the library until the process exits.
// Host code cannot use the array's name as a device address: the current
// device's address is looked up (cudaGetSymbolAddress) and handed to the
// kernels.  The lookup is repeated on every call made while the stream is
// not being captured, so the address follows the module when a device reset
// (cudaDeviceReset) or a new primary context reloads it; a call made during
// a capture cannot look it up and takes the address the last uncaptured
// call on that device found.
__device__ __align__(256) uint8_t g_static_status[(size_t)BH_STATIC_MAX_PATCHES * NC_];
constexpr int kMaxDevices = 64;
void* g_static_status_ptr[kMaxDevices] = {nullptr};
std::mutex g_static_status_mu;

int static_status_ptr(cudaStream_t st, uint8_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BH_ECUDA;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return BH_ECUDA;
    std::lock_guard<std::mutex> lock(g_static_status_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_status) != cudaSuccess || !p) return BH_ECUDA;
        g_static_status_ptr[dev] = p;
    } else if (!g_static_status_ptr[dev]) {
        return BH_ECUDA;   // no uncaptured call has looked the address up on this device
    }
    *out = (uint8_t*)g_static_status_ptr[dev];
    return BH_OK;
}

}  // namespace

#define BH_DISPATCH(P, call)                                 \
    switch ((P) ? (P)->precision : -1) {                     \
    case BH_FP64: return vfp64::call;                        \
    case BH_FP64_FMA: return vfma::call;                     \
    case BH_MIXED: return vmixed::call;                      \
    default: return BH_EINVAL;                               \
    }

extern "C" {

int bh_abi_version(void) { return BHGPU_ABI_VERSION; }

int bh_read_error(const bh_pool* pool, int32_t* out, void* stream) {
    if (!pool || !pool->err || !out) return BH_EINVAL;
    if (cudaMemcpyAsync(out, pool->err, sizeof(int32_t), cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess) return BH_ECUDA;
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? BH_OK : BH_ECUDA;
}
int bh_clear_error(const bh_pool* pool, void* stream) {
    if (!pool || !pool->err) return BH_EINVAL;
    return cudaMemsetAsync(pool->err, 0, sizeof(int32_t), S(stream)) == cudaSuccess ? BH_OK : BH_ECUDA;
}
int bh_metric_comp(const bh_params* P, const double* r, const double* th, int64_t n, double* out, void* stream) {
    BH_DISPATCH(P, metric_comp(P, r, th, n, out, stream));
}
int bh_ptoc(const bh_params* P, const double* W, const double* r, const double* th, int64_t n, double* U, double* Wd,
            void* stream) {
    BH_DISPATCH(P, ptoc(P, W, r, th, n, U, Wd, stream));
}
int bh_ctop(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, double* W, double* Wd,
            int32_t* status, int32_t* iters, int32_t* path, void* stream) {
    BH_DISPATCH(P, ctop(P, U, r, th, n, W, Wd, status, iters, path, stream));
}
int bh_hlld(const bh_params* P, const double* WL, const double* WR, const double* UL, const double* UR,
            const double* r, const double* th, int32_t dim, int64_t n, double* F, double* ctspeed, void* stream) {
    BH_DISPATCH(P, hlld(P, WL, WR, UL, UR, r, th, dim, n, F, ctspeed, stream));
}
int bh_geometry(const bh_pool* pool, void* stream) { return vfp64::geometry(pool, stream); }
int bh_reconfp(const bh_params* P, const bh_pool* pool, int32_t dim, int32_t limiter, double* L, double* R,
               void* stream) {
    BH_DISPATCH(P, reconfp(P, pool, dim, limiter, L, R, stream));
}
int bh_fluxcomp(const bh_params* P, const bh_pool* pool, void* stream) { BH_DISPATCH(P, fluxcomp(P, pool, stream)); }
int bh_emfcomp(const bh_pool* pool, void* stream) { return vfp64::emfcomp(pool, stream); }
int bh_bfupdate(const bh_pool* pool, const double* dt_dev, void* stream) { return vfp64::bfupdate(pool, dt_dev, stream); }
int bh_f2cb(const bh_params* P, const bh_pool* pool, void* stream) { BH_DISPATCH(P, f2cb(P, pool, stream)); }
int bh_maxdivb(const bh_pool* pool, double* out, void* stream) { return vfp64::maxdivb(pool, out, stream); }
int bh_div_source(const bh_params* P, const bh_pool* pool, double* div, double* src, void* stream) {
    BH_DISPATCH(P, div_source(P, pool, div, src, stream));
}
int bh_ghosts(const bh_params* P, const bh_pool* pool, const int32_t* patches, int32_t n, void* stream) {
    BH_DISPATCH(P, ghosts(P, pool, patches, n, stream));
}
int bh_prims(const bh_params* P, const bh_pool* pool, void* stream) { BH_DISPATCH(P, prims(P, pool, stream)); }
int bh_ghosts_prims(const bh_params* P, const bh_pool* pool, void* stream) {
    BH_DISPATCH(P, ghosts_prims(P, pool, stream));
}
int bh_ghosts_prims_static(const bh_params* P, const bh_pool* pool, void* stream) {
    if (!P || bad_pool(pool) || !pool->leafmask) return BH_EINVAL;
    if (pool->npatch > BH_STATIC_MAX_PATCHES) return BH_ERANGE;
    if (pool->nleaf == 0) return BH_OK;
    uint8_t* status = nullptr;
    int rc = static_status_ptr(S(stream), &status);
    if (rc) return rc;
    // every entry read is written by the interior pass of the same call first
    BH_DISPATCH(P, ghosts_prims_status(P, pool, status, stream));
}
int bh_update(const bh_params* P, const bh_pool* pool, const double* dt_dev, int32_t stage, void* stream) {
    BH_DISPATCH(P, update(P, pool, dt_dev, stage, stream));
}
int bh_floors(const bh_params* P, const bh_pool* pool, void* stream) { BH_DISPATCH(P, floors(P, pool, stream)); }
int bh_regrid_flags(const bh_params* P, const bh_pool* pool, const int32_t* lvl, uint8_t* flags, void* stream) {
    BH_DISPATCH(P, regrid_flags(P, pool, lvl, flags, stream));
}
int bh_refine(const bh_params* P, const bh_pool* pool, const int32_t* plan, int32_t n, void* stream) {
    BH_DISPATCH(P, refine(P, pool, plan, n, stream));
}
int bh_ccrstr(const bh_params* P, const bh_pool* pool, const int32_t* plan, int32_t n, void* stream) {
    BH_DISPATCH(P, ccrstr(P, pool, plan, n, stream));
}
int bh_b_init(const bh_params* P, const bh_pool* pool, const int32_t* patches, int32_t n, void* stream) {
    BH_DISPATCH(P, b_init(P, pool, patches, n, stream));
}
int bh_analysis(const bh_params* P, const bh_pool* pool, const bh_analysis_params* A, double* partial,
                double* out, void* stream) {
    BH_DISPATCH(P, analysis(P, pool, A, partial, out, stream));
}
int bh_torus_init(const bh_params* P, const bh_pool* pool, double r_max, double r_in, double* out, void* stream) {
    BH_DISPATCH(P, torus_init(P, pool, r_max, r_in, out, stream));
}
int bh_ctop_guess(const bh_params* P, const double* U, const double* r, const double* th, int64_t n,
                  const double* xi0, double* W, double* Wd, int32_t* status, int32_t* iters, int32_t* path,
                  void* stream) {
    BH_DISPATCH(P, ctop_guess(P, U, r, th, n, xi0, W, Wd, status, iters, path, stream));
}
int bh_ctop_pre(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, double* pre,
                void* stream) {
    BH_DISPATCH(P, ctop_pre(P, U, r, th, n, pre, stream));
}
int bh_tune_candidates(int32_t kernel, int32_t* out, int32_t max) {
    if (kernel < 0 || kernel >= BH_TUNE_NKERNEL || (max > 0 && !out) || max < 0) return BH_EINVAL;
    int n = 0;
    while (n < 5 && bh_tune_cands[kernel][n]) n++;
    for (int i = 0; i < n && i < max; i++) out[i] = bh_tune_cands[kernel][i];
    return n;
}
int bh_tune_set(int32_t precision, int32_t kernel, int32_t ctas) {
    bh_params P = {};
    P.precision = precision;
    BH_DISPATCH(&P, tune_set(kernel, ctas));
}
int bh_tune_get(int32_t precision, int32_t kernel, int32_t* ctas) {
    bh_params P = {};
    P.precision = precision;
    BH_DISPATCH(&P, tune_get(kernel, ctas));
}
int bh_ctop_learned(const bh_params* P, const bh_mlp* m, const double* U, const double* r, const double* th,
                    int64_t n, double* xi0, double* W, double* Wd, int32_t* status, int32_t* iters, int32_t* path,
                    int32_t* err, void* stream) {
    BH_DISPATCH(P, ctop_learned(P, m, U, r, th, n, xi0, W, Wd, status, iters, path, err, stream));
}
int bh_dtcomp(const bh_params* P, const bh_pool* pool, double cfl, double* dt_dev, void* stream) {
    BH_DISPATCH(P, dtcomp(P, pool, cfl, dt_dev, stream));
}
int bh_rkstg(const bh_params* P, const bh_pool* pool, const double* dt_dev, int32_t stage, const int32_t* waves,
             const int32_t* wave_off, int32_t nwave, void* stream) {
    BH_DISPATCH(P, rkstg(P, pool, dt_dev, stage, waves, wave_off, nwave, stream));
}
int bh_step(const bh_params* P, const bh_pool* pool, double cfl, double* dt_dev, const int32_t* waves,
            const int32_t* wave_off, int32_t nwave, void* stream) {
    BH_DISPATCH(P, step(P, pool, cfl, dt_dev, waves, wave_off, nwave, stream));
}

// ---- the corrected scheme ----------------------------------------------
namespace {
int fx_bad(const bh_fx_params* P, const bh_fx_grid* g) {
    if (!P || !g || g->nblock <= 0 || !g->blocks || !g->nbr || !g->U || !g->U1 || !g->W || !g->Bf || !g->Bf1 ||
        !g->F || !g->dt || !g->count || g->ncell <= 0)
        return 1;
    if ((g->nitem_cell > 0 && !g->items_cell) || (g->nitem_pos > 0 && !g->items_pos) ||
        (g->nitem_ghost > 0 && !g->items_ghost) || g->nitem_cell < 0 || g->nitem_pos < 0 || g->nitem_ghost < 0)
        return 1;
    if (P->precision < BH_FP64 || P->precision > BH_MIXED || P->maxiter <= 0 || !(P->gamma > 1.0)) return 1;
    if (g->maxlevel < 0 || g->maxlevel > 8 || (g->maxlevel > 0 && !g->E)) return 1;
    if (P->limiter < BH_MINMOD || P->limiter > BH_PPM || (g->ghost_depth != 0 && g->ghost_depth != 2 && g->ghost_depth != 3) ||
        (P->limiter == BH_PPM && g->ghost_depth != 3) || (g->nitem_flux > 0 && !g->items_flux))
        return 1;
    return 0;
}
}  // namespace
#define FX_DISPATCH(P, call)                                 \
    switch ((P)->precision) {                                \
    case BH_FP64: return vfp64::call;                        \
    case BH_FP64_FMA: return vfma::call;                     \
    case BH_MIXED: return vmixed::call;                      \
    default: return BH_EINVAL;                               \
    }

int bh_fx_step(const bh_fx_params* P, const bh_fx_grid* g, void* stream) {
    if (fx_bad(P, g)) return BH_EINVAL;
    FX_DISPATCH(P, fx_step(P, g, stream));
}
int bh_fx_prims(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, int32_t with_dt, void* stream) {
    if (fx_bad(P, g) || stage < 0 || stage > 1) return BH_EINVAL;
    FX_DISPATCH(P, fx_prims(P, g, stage, with_dt, stream));
}
int bh_fx_ghost_pass(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, int32_t pass, void* stream) {
    if (fx_bad(P, g) || stage < 0 || stage > 1 || pass < 0 || pass > g->maxlevel) return BH_EINVAL;
    FX_DISPATCH(P, fx_ghost_pass(P, g, stage, pass, stream));
}
int bh_fx_ghosts(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* stream) {
    if (fx_bad(P, g) || stage < 0 || stage > 1) return BH_EINVAL;
    FX_DISPATCH(P, fx_ghosts(P, g, stage, stream));
}
int bh_fx_fluxes(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* stream) {
    if (fx_bad(P, g) || stage < 0 || stage > 1) return BH_EINVAL;
    FX_DISPATCH(P, fx_fluxes(P, g, stage, stream));
}
int bh_fx_update(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* stream) {
    if (fx_bad(P, g) || stage < 0 || stage > 1) return BH_EINVAL;
    FX_DISPATCH(P, fx_update(P, g, stage, stream));
}
int bh_fx_emf(const bh_fx_params* P, const bh_fx_grid* g, void* stream) {
    if (fx_bad(P, g) || !g->E) return BH_EINVAL;
    FX_DISPATCH(P, fx_update_parts(P, g, 0, 1, stream));
}
int bh_fx_update_from_emf(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* stream) {
    if (fx_bad(P, g) || !g->E || stage < 0 || stage > 1) return BH_EINVAL;
    FX_DISPATCH(P, fx_update_parts(P, g, stage, 2, stream));
}
int bh_fx_tune_set(int32_t precision, int32_t kernel, int32_t ctas) {
    switch (precision) {
    case BH_FP64: return vfp64::fx_tune_set(kernel, ctas);
    case BH_FP64_FMA: return vfma::fx_tune_set(kernel, ctas);
    case BH_MIXED: return vmixed::fx_tune_set(kernel, ctas);
    default: return BH_EINVAL;
    }
}
int bh_fx_tune_get(int32_t precision, int32_t kernel, int32_t* ctas) {
    switch (precision) {
    case BH_FP64: return vfp64::fx_tune_get(kernel, ctas);
    case BH_FP64_FMA: return vfma::fx_tune_get(kernel, ctas);
    case BH_MIXED: return vmixed::fx_tune_get(kernel, ctas);
    default: return BH_EINVAL;
    }
}
int bh_fx_pack_state(const bh_fx_params* P, const bh_fx_grid* g, const int64_t* face_off, void* packed, int32_t dir,
                     void* stream) {
    if (fx_bad(P, g) || !face_off || !packed || (dir != 0 && dir != 1)) return BH_EINVAL;
    FX_DISPATCH(P, fx_pack_state(g, face_off, packed, dir, stream));
}
int bh_fx_divb(const bh_fx_grid* g, double* out, void* stream) {
    if (!g || g->nblock <= 0 || !g->blocks || !g->Bf || !out || (g->nitem_cell > 0 && !g->items_cell)) return BH_EINVAL;
    return vfp64::fx_divb(g, out, stream);
}
int bh_fx_torus_init(const bh_fx_params* P, const bh_fx_grid* g, const bh_fx_torus* T, double* scratch, double* out,
                     void* stream) {
    if (fx_bad(P, g) || !T || !scratch || !(T->r_max > T->r_in) || !(T->r_in > 0.0) || !(T->kappa > 0.0)) return BH_EINVAL;
    FX_DISPATCH(P, fx_torus_init(P, g, T, scratch, out, stream));
}

struct bh_step_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

extern "C++" {
namespace {
// capture fn(stream) on stream into an instantiated graph
template <typename Fn>
int capture_graph(void* stream, bh_step_graph** out, Fn fn);
}  // namespace
}

int bh_step_graph_create(const bh_params* P, const bh_pool* pool, double cfl, double* dt_dev,
                         const int32_t* waves, const int32_t* wave_off, int32_t nwave, void* stream,
                         bh_step_graph** out) {
    if (!P || !out || !stream) return BH_EINVAL;
    return capture_graph(stream, out, [&](void* s) { return bh_step(P, pool, cfl, dt_dev, waves, wave_off, nwave, s); });
}
int bh_fx_graph_create(const bh_fx_params* P, const bh_fx_grid* g, void* stream, bh_step_graph** out) {
    if (!P || !out || !stream) return BH_EINVAL;
    if (fx_bad(P, g)) return BH_EINVAL;
    return capture_graph(stream, out, [&](void* s) { return bh_fx_step(P, g, s); });
}

extern "C++" {
namespace {
template <typename Fn>
int capture_graph(void* stream, bh_step_graph** out, Fn fn) {
    *out = nullptr;
    cudaStream_t st = S(stream);
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return BH_ECUDA;
    int rc = fn(stream);
    cudaGraph_t graph = nullptr;
    // the capture is always ended, also when the step refused its arguments
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc != BH_OK || e != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        return rc != BH_OK ? rc : BH_ECUDA;
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return BH_ECUDA;
    }
    bh_step_graph* g = new (std::nothrow) bh_step_graph{graph, exec};
    if (!g) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return BH_ECUDA;
    }
    *out = g;
    return BH_OK;
}
}  // namespace
}

int bh_step_graph_replay(bh_step_graph* g, void* stream) {
    if (!g) return BH_EINVAL;
    return cudaGraphLaunch(g->exec, S(stream)) == cudaSuccess ? BH_OK : BH_ECUDA;
}
int bh_step_graph_destroy(bh_step_graph* g) {
    if (!g) return BH_EINVAL;
    cudaError_t a = cudaGraphExecDestroy(g->exec), b = cudaGraphDestroy(g->graph);
    delete g;
    return a == cudaSuccess && b == cudaSuccess ? BH_OK : BH_ECUDA;
}

}  // extern "C"
