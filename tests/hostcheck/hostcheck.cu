// hostcheck.cu -- runs the kernels' per-item functions (csrc/bh_items.cuh)
// on the CPU, launch by launch in the order the C ABI issues them, on host
// copies of the pool.  Built with nvcc as host code, the math functions
// are the host libm's, so a bit-exact match with the oracle shows the
// kernel logic is the reference's; GPU-vs-oracle tests then only see the
// last-bit differences of the device math library.  Test code only.
#include <stdint.h>
#include "bhgpu.h"
#include "bh_items.cuh"
#include "bh_init.cuh"
#include "bh_fixed_phys.cuh"

using namespace bh;

// entries of pool->all, as the launchers count them
static inline int NALL(const bh_pool* p) { return p->nall > 0 ? p->nall : p->npatch; }

extern "C" {

void hc_metric(const bh_params* P, const double* r, const double* th, int64_t n, double* out) {
    KP k = kp_of(P);
    for (int64_t q = 0; q < n; q++) metric_item(k, r, th, q, out);
}
void hc_ptoc(const bh_params* P, const double* W, const double* r, const double* th, int64_t n, double* U, double* Wd) {
    KP k = kp_of(P);
    for (int64_t q = 0; q < n; q++) ptoc_item(k, W, r, th, n, q, U, Wd, nullptr);
}
void hc_ctop(const bh_params* P, const double* U, const double* r, const double* th, int64_t n, double* W, double* Wd,
             int32_t* st, int32_t* it, int32_t* pa) {
    KP k = kp_of(P);
    for (int64_t q = 0; q < n; q++) ctop_item(k, U, r, th, n, q, W, Wd, st, it, pa);
}
void hc_hlld(const bh_params* P, const double* WL, const double* WR, const double* UL, const double* UR, const double* r,
             const double* th, int dim, int64_t n, double* F, double* cts) {
    KP k = kp_of(P);
    for (int64_t q = 0; q < n; q++) hlld_item(k, WL, WR, UL, UR, r, th, dim, n, q, F, cts);
}
void hc_geometry(const bh_pool* pool) {
    Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int l = 0; l < NC; l++) geometry_item(P, pool->all[i], l);
}
void hc_reconfp(const bh_params* Pp, const bh_pool* pool, int dim, int lim, double* L, double* R) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    int64_t n = (int64_t)pool->npatch * NFACE;
    for (int p = 0; p < pool->npatch; p++)
        for (int f = 0; f < NFACE; f++) reconfp_item<double>(k, P, p, dim, f, lim, n, L, R);
}
void hc_fluxcomp(const bh_params* Pp, const bh_pool* pool) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    if (pool->aux) {
        for (int i = 0; i < NALL(pool); i++)
            for (int l = 0; l < NC; l++) aux_item<double>(k, P, pool->all[i], l);
        for (int i = 0; i < NALL(pool); i++)
            for (int dim = 0; dim < 3; dim++)
                for (int f = 0; f < NFACE; f++) flux_item<double, true>(k, P, pool->all[i], dim, f);
        return;
    }
    for (int i = 0; i < NALL(pool); i++)
        for (int dim = 0; dim < 3; dim++)
            for (int f = 0; f < NFACE; f++) flux_item<double>(k, P, pool->all[i], dim, f);
}
void hc_emfcomp(const bh_pool* pool) {
    Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int e = 0; e < N_EDGE; e++) emf_item(P, pool->all[i], e);
}
void hc_bfupdate(const bh_pool* pool, double dt) {
    Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int e = 0; e < N_BUP; e++) bfupdate_item(P, pool->all[i], e, dt);
}
void hc_f2cb(const bh_params* Pp, const bh_pool* pool) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int e = 0; e < N_F2C; e++) f2cb_item(k, P, pool->all[i], e);
}
void hc_maxdivb(const bh_pool* pool, double* out) {
    Pool P = pool_of(pool);
    for (int p = 0; p < pool->npatch; p++) {
        double m = 0.0;
        for (int e = 0; e < N_BUP; e++) m = smax(m, maxdivb_item(P, p, e));
        out[p] = m;
    }
}
void hc_div_source(const bh_params* Pp, const bh_pool* pool, double* dv, double* sv) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int c = 0; c < N_INT; c++) div_source_item<double>(k, P, pool->all[i], c, dv, sv);
}
void hc_ghosts(const bh_params* Pp, const bh_pool* pool, const int32_t* list, int n) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < n; i++)
        for (int e = 0; e < 2 * N_COPY; e++) ghost_copy_item(P, list[i], e);
    for (int i = 0; i < n; i++)
        for (int e = 0; e < N_STRIP; e++) ghost_prolong_item(k, P, list[i], e);
    for (int i = 0; i < n; i++)
        for (int l = 0; l < NC; l++) ghost_ctop_item(k, P, list[i], l);
}
void hc_prims(const bh_params* Pp, const bh_pool* pool, int ghost_first) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < pool->nleaf; i++)
        for (int l = 0; l < NC; l++) prims_item(k, P, pool->leaves[i], l, ghost_first);
}
void hc_ghosts_prims(const bh_params* Pp, const bh_pool* pool) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < pool->nleaf; i++)
        for (int e = 0; e < 2 * N_COPY; e++) ghost_copy_item(P, pool->leaves[i], e);
    for (int i = 0; i < pool->nleaf; i++)
        for (int e = 0; e < N_STRIP; e++) ghost_prolong_item(k, P, pool->leaves[i], e);
    if (pool->status && pool->leafmask) {
        for (int i = 0; i < pool->nleaf; i++)
            for (int c = 0; c < N_INT; c++) prims_interior_item(k, P, pool->leaves[i], c);
        for (int i = 0; i < pool->nleaf; i++)
            for (int e = 0; e < N_GHOST; e++) prims_ghost_item(k, P, pool->leaves[i], e);
    } else {
        hc_prims(Pp, pool, 1);
    }
}
void hc_update(const bh_params* Pp, const bh_pool* pool, double dt, int stage) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int c = 0; c < N_INT; c++) update_interior_item<double>(k, P, pool->all[i], c, dt, stage);
    for (int i = 0; i < NALL(pool); i++)
        for (int e = 0; e < N_SHELL; e++) update_shell_item(k, P, pool->all[i], e);
}
void hc_floors(const bh_params* Pp, const bh_pool* pool) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int i = 0; i < NALL(pool); i++)
        for (int c = 0; c < N_INT; c++) floors_item(k, P, pool->all[i], c);
}
// AMR regrid pieces, in the launch order of bh_regrid_flags / bh_refine /
// bh_ccrstr (flags of the leaf patches; plan rows parent + 8 children)
void hc_regrid_flags(const bh_params* Pp, const bh_pool* pool, const int32_t* lvl, uint8_t* flags) {
    (void)Pp;
    Pool P = pool_of(pool);
    for (int i = 0; i < pool->nleaf; i++) {
        int p = pool->leaves[i];
        bool ref = false, nf = false;
        for (int c = 0; c < N_INT; c++) regrid_cell(P, p, lvl[p], c, ref, nf);
        flags[p] = regrid_patch_flags(lvl[p], ref, nf);
    }
}
void hc_refine(const bh_params* Pp, const bh_pool* pool, const int32_t* plan, int n) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int r = 0; r < n; r++)
        for (int h = 0; h < 8; h++)
            for (int c = 0; c < N_INT; c++) refine_item(k, P, plan[r * 9], plan[r * 9 + 1 + h], h, c);
    for (int r = 0; r < n; r++)
        for (int h = 0; h < 8; h++)
            for (int e = 0; e < 3 * NF; e++) b_init_item(P, plan[r * 9 + 1 + h], e);
}
void hc_ccrstr(const bh_params* Pp, const bh_pool* pool, const int32_t* plan, int n) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    for (int r = 0; r < n; r++)
        for (int c = 0; c < N_INT; c++) ccrstr_item(k, P, plan[r * 9], plan + r * 9 + 1, c);
    for (int r = 0; r < n; r++)
        for (int e = 0; e < 3 * NF; e++) b_init_item(P, plan[r * 9], e);
}
// analysis integrals with the cells visited and added in the reference's
// serial order (quilt order, then i, j, k), so the sums equal the oracle's
void hc_analysis(const bh_params* Pp, const bh_pool* pool, const bh_analysis_params* A, double* out) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    AParams ap{A->hrz, A->rs, A->rho_min_full, A->rho_min_bundle};
    for (int q = 0; q < BH_NQ; q++) out[q] = 0.0;
    for (int i = 0; i < pool->nleaf; i++)
        for (int c = 0; c < N_INT; c++) analysis_cell(k, P, pool->leaves[i], c, ap, out);
}
// the initial-data sequence of bh_torus_init, serially; out[5] as there
int hc_torus_init(const bh_params* Pp, const bh_pool* pool, double r_max, double r_in, double* out) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    int n = NALL(pool);
    for (int i = 0; i < n; i++)
        for (int l = 0; l < NC; l++) floor_cell(k, P, pool->all[i], l);
    TorusScalars s = fm_scalars(k.tree, k.gamma, r_max, r_in);
    out[0] = s.l0; out[1] = s.W_in; out[2] = s.lnh_max;
    double rho_fm = 0.0;
    if (s.lnh_max > 0.0) {
        for (int i = 0; i < n; i++)
            for (int c = 0; c < N_INT; c++) rho_fm = smax(rho_fm, fm_cell_rho(k, P, pool->all[i], c, s));
        if (rho_fm >= 1e-14)
            for (int i = 0; i < n; i++)
                for (int c = 0; c < N_INT; c++) fm_cell_prims(k, P, pool->all[i], c, s, 1.0 / rho_fm);
    }
    out[3] = rho_fm;
    double glmx = 0.0;
    for (int i = 0; i < n; i++)
        for (int c = 0; c < N_INT; c++) glmx = smax(glmx, Wv(P, pool->all[i], 0)[lindx(c / 256, (c / 16) % 16, c % 16)]);
    out[4] = glmx;
    if (glmx < 1e-14) return BH_ERANGE;
    if (glmx > 1e-10)
        for (int i = 0; i < n; i++) {
            for (int e = 0; e < N_F2C; e++) bpot_item(P, pool->all[i], e, glmx);
            for (int e = 0; e < N_F2C; e++) f2cb_item(k, P, pool->all[i], e);
        }
    for (int i = 0; i < n; i++)
        for (int c = 0; c < N_INT; c++) ptoc_interior_item(k, P, pool->all[i], c);
    return BH_OK;
}
double hc_dtcomp(const bh_params* Pp, const bh_pool* pool, double cfl) {
    KP k = kp_of(Pp); Pool P = pool_of(pool);
    double best = DBL_BIG;
    for (int i = 0; i < pool->nleaf; i++)
        for (int c = 0; c < N_INT; c++) best = smin(best, dt_item(k, P, pool->leaves[i], c, cfl));
    return best;
}
// bh_rkstg / bh_step in the order the ABI launches them
void hc_rkstg(const bh_params* Pp, const bh_pool* pool, double dt, int stage, const int32_t* waves,
              const int32_t* off, int nwave) {
    if (nwave <= 1) hc_ghosts_prims(Pp, pool);
    else {
        for (int w = 0; w < nwave; w++) hc_ghosts(Pp, pool, waves + off[w], off[w + 1] - off[w]);
        hc_prims(Pp, pool, 0);
    }
    hc_fluxcomp(Pp, pool);
    hc_emfcomp(pool);
    hc_bfupdate(pool, dt);
    hc_update(Pp, pool, dt, stage);
}
double hc_step(const bh_params* Pp, const bh_pool* pool, double cfl, const int32_t* waves, const int32_t* off,
               int nwave) {
    double dt = hc_dtcomp(Pp, pool, cfl);
    hc_rkstg(Pp, pool, dt, 0, waves, off, nwave);
    hc_rkstg(Pp, pool, dt, 1, waves, off, nwave);
    hc_floors(Pp, pool);
    return dt;
}

// the corrected scheme's PLM face value (bhfx::plm_value) of cell w0 toward
// wn, wf its other neighbour, in double and in float (the inputs rounded)
void hc_fx_plm(const double* wf, const double* w0, const double* wn, int lim, int64_t n, double* o64, float* o32) {
    for (int64_t q = 0; q < n; q++) {
        o64[q] = bhfx::plm_value<double>(wf[q], w0[q], wn[q], lim);
        o32[q] = bhfx::plm_value<float>(float(wf[q]), float(w0[q]), float(wn[q]), lim);
    }
}

// the corrected scheme's prim2cons (derive + prim2cons) at Kerr-Schild
// points x, y, z in double and in float (metric and primitives rounded):
// u64[8][n], u32[8][n]
void hc_fx_prim2cons(const bhfx::FxPar* P, const double* x, const double* y, const double* z, const double* w,
                     int64_t n, double* u64, float* u32) {
    for (int64_t q = 0; q < n; q++) {
        double wd[8];
        float wf[8];
        for (int v = 0; v < 8; v++) { wd[v] = w[v * n + q]; wf[v] = float(wd[v]); }
        bhfx::KS mk;
        bhfx::ks_metric(*P, x[q], y[q], z[q], mk);
        bhfx::KSm<double> md;
        bhfx::ks_cast(mk, md);
        bhfx::Derived<double> dd;
        bhfx::derive(md, P->gg, wd, dd);
        double ud[8];
        bhfx::prim2cons(md, P->gamma, wd, dd, ud);
        bhfx::KSb<float> mf;
        bhfx::ks_metric<float>(*P, float(x[q]), float(y[q]), float(z[q]), mf);
        bhfx::KSm<float> mm;
        bhfx::ks_cast(mf, mm);
        bhfx::Derived<float> df;
        bhfx::derive(mm, float(P->gg), wf, df);
        float uf[8];
        bhfx::prim2cons(mm, float(P->gamma), wf, df, uf);
        for (int v = 0; v < 8; v++) { u64[v * n + q] = ud[v]; u32[v * n + q] = uf[v]; }
    }
}

}  // extern "C"
