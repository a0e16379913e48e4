/*
 * bhgpu.h -- C ABI of the B200 (sm_100a) GRMHD block update.
 *
 * A drop-in for the fluid hot path of Fjoerde/black-hole-simulator
 * (src/fluid): the reference's C++ entry points (file:line below, paths
 * relative to src/fluid) map one to one onto these functions.  Every
 * function takes plain device pointers and sizes, launches on the caller's
 * CUDA stream (`stream`, a cudaStream_t passed as void*, NULL = legacy
 * default stream) and returns without synchronising.
 *
 * Ownership: the caller allocates every device buffer (the reference's
 * patch members, grid.hpp:27-105) and describes them in a bh_pool; the
 * library allocates nothing unless a function says so.
 *
 * Errors: nothing throws.  Functions return BH_OK or a negative BH_E*
 * code for bad arguments or a CUDA launch error.  Conditions the reference
 * reports by throwing std::domain_error from its EOS (thermo.cpp:11-31)
 * are detected on the device and recorded in *pool->err (bit BH_ERR_DOMAIN);
 * the caller reads that word (bh_read_error) once the stream has drained.
 *
 * Layout (reference per-patch linear indices, grid.cpp:51-89): a pool
 * holds npatch patches of 16^3 interior cells + 2 ghost layers (20^3
 * cells), structure of arrays per patch:
 *   U, W, dU  [npatch][8][8000]    conserved D,S0,S1,S2,tau,B0,B1,B2 /
 *                                  primitive rho,eps,v0,v1,v2,B0,B1,B2
 *   F         [npatch][3][8][8400] face fluxes Fx, Fy, Fz (cons order)
 *   Bf        [npatch][3][8400]    face B: Bfx, Bfy, Bfz
 *   EMF       [npatch][3][8820]    edge EMFs: EMFx, EMFy, EMFz
 *   rth       [npatch][2][8000]    cell-centre r, theta
 */
#ifndef BHGPU_H
#define BHGPU_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BHGPU_ABI_VERSION 1

enum {
    BH_OK = 0,
    BH_EINVAL = -1,   /* bad argument                          */
    BH_ECUDA = -2,    /* a CUDA call or kernel launch failed   */
    BH_ERANGE = -3    /* size above a documented maximum       */
};
/* bits of the device error word */
enum {
    BH_ERR_DOMAIN = 1,  /* density <= 0 reached the EOS (reference throws) */
    BH_ERR_TIMEOUT = 2  /* a bounded on-device wait ran out (bh_ctop_learned) */
};

/* arithmetic variant (bh_params.precision) */
enum {
    BH_FP64 = 0,      /* FP64 with the reference's separate multiply/add roundings */
    BH_FP64_FMA = 1,  /* FP64 with fused multiply-add contraction                  */
    BH_MIXED = 2      /* reconstruction, face fluxes (ptoc + HLLD) and the geometric
                         source in FP32; metric, constrained transport, flux
                         divergence, RK combine, con2prim, floors and dt in FP64  */
};
/* reconstruction limiter (recon.hpp:36); BH_PPM (the corrected scheme only):
 * the piecewise-parabolic method of Colella & Woodward (1984) */
enum { BH_MINMOD = 0, BH_VANLEER = 1, BH_MC = 2, BH_PPM = 3 };
/* neighbour kinds of the ghost fill (grid.cpp:528-534) */
enum { BH_NB_BNDY = 0, BH_NB_COPY = 1, BH_NB_PROLONG = 2 };

typedef struct bh_params {
    double M, a, Q;      /* tree metric, metric(M,a,Q)          metric.hpp:31       */
    double gamma;        /* adiabatic index, state(gm)          state.hpp:11        */
    int32_t limiter;     /* BH_MINMOD / BH_VANLEER / BH_MC      recon.hpp:41        */
    int32_t maxiter;     /* con2prim Newton cap (500)           cons.hpp:75         */
    double tol;          /* con2prim tolerance (1e-10)          cons.hpp:75         */
    double cM, ca, cQ;   /* metric carried by every cell: the default metric()
                            = (1, 0, 0) in the reference       cell.hpp:25, metric.hpp:30 */
    int32_t precision;   /* BH_FP64 (reference-faithful), BH_FP64_FMA or BH_MIXED    */
    int32_t reserved;
} bh_params;

typedef struct bh_pool {
    int32_t npatch;
    double *U, *W, *dU;  /* [np][8][8000]                                        */
    double *F;           /* [np][3][8][8400]                                     */
    double *Bf;          /* [np][3][8400]                                        */
    double *EMF;         /* [np][3][8820]                                        */
    double *rth;         /* [np][2][8000]   written by bh_geometry               */
    const double *pgeo;  /* [np][6]  xedge[0], yedge[0], zedge[0], dx, dy, dz    */
    const int32_t *nbr;  /* [np][6][2] (neighbour, kind), slot dim*2 + (side>0)  */
    const int32_t *all;  /* [nall] patch indices the flux/CT/update/floors kernels
                            visit (normally 0..npatch-1)                       */
    const int32_t *leaves; int32_t nleaf;  /* leaf patch indices (ghosts, prims, dt) */
    int32_t *err;        /* device error word (BH_ERR_* bits)                    */
    const uint8_t *leafmask; /* [npatch] 1 for leaf patches                       */
    uint8_t *status;     /* [np][8000] scratch: con2prim outcome of the interior
                            cells in the current stage; NULL disables the reuse
                            of those outcomes by the ghost cells copied from them */
    double *aux;         /* [np][6][8000] scratch of bh_fluxcomp: log rho, log eps
                            and the cell-metric entries of the causality check,
                            computed once per cell instead of once per face that
                            reads the cell; NULL computes them per face.  Either
                            way the fluxes are the same bit for bit. */
    double *Wd;          /* [np][4][8000] lor, p, h, b2 of the primitives as floors,
                            refine and ccrstr leave them (the derived fields of the
                            reference's prim, prim.hpp:21-25; read by bh_analysis);
                            NULL: not kept */
    int32_t nall;        /* entries of `all` (0: npatch); a subset of the patches,
                            e.g. those one rank owns when a domain is sharded */
} bh_pool;

/* ---- library --------------------------------------------------------------- */
int bh_abi_version(void);
/* copy the device error word to *out (synchronises the stream) */
int bh_read_error(const bh_pool *pool, int32_t *out, void *stream);
int bh_clear_error(const bh_pool *pool, void *stream);

/* ---- L0/L1 physics, batched over n independent items (SoA [k][n]) ---------- */
/* metric::comp (physics/spacetime.cpp:122-134): out [n][120] in the member
 * order of struct metriccomp (metric.hpp:11-21) */
int bh_metric_comp(const bh_params *P, const double *r, const double *th, int64_t n,
                   double *out, void *stream);
/* conserved::ptoc (physics/conserved.cpp:17-73): W [8][n] -> U [8][n];
 * Wd [4][n] (may be NULL) receives lor, p, h, b2 -- the fields ptoc mutates */
int bh_ptoc(const bh_params *P, const double *W, const double *r, const double *th, int64_t n,
            double *U, double *Wd, void *stream);
/* conserved::ctop (physics/conserved.cpp:135-285): U [8][n] -> W [8][n];
 * Wd [5][n] = p, T, h, lor, b2 (may be NULL); status[n] = 1 ok, 0 failed,
 * -1 domain error; iters/path (may be NULL) = Newton iterations and the
 * route taken (0 Newton, 1 Newton cap, 2 Brent root, 3 Brent failed) */
int bh_ctop(const bh_params *P, const double *U, const double *r, const double *th, int64_t n,
            double *W, double *Wd, int32_t *status, int32_t *iters, int32_t *path, void *stream);
/* hlld (solver/hlld.cpp:230-312): per item L/R primitive and conserved
 * states at face coordinates (r, th); F [8][n], ctspeed [n] */
int bh_hlld(const bh_params *P, const double *WL, const double *WR, const double *UL,
            const double *UR, const double *r, const double *th, int32_t dim, int64_t n,
            double *F, double *ctspeed, void *stream);

/* ---- L1/L2 over a patch pool -------------------------------------------- */
/* patch::cell_init geometry (grid/grid.cpp:149-175): fills pool->rth */
int bh_geometry(const bh_pool *pool, void *stream);
/* reconfp (grid/reconstruction.cpp:40-97) at every flux face of direction
 * dim of every patch, in the loop order of patch::fluxcomp; L, R [8][np*4352] */
int bh_reconfp(const bh_params *P, const bh_pool *pool, int32_t dim, int32_t limiter,
               double *L, double *R, void *stream);
/* patch::fluxcomp (grid/grid.cpp:255-329) on every patch */
int bh_fluxcomp(const bh_params *P, const bh_pool *pool, void *stream);
/* constrans::emfcomp / Bfupdate / f2cB (grid/transport.cpp:11-75), every patch;
 * dt is read from device memory */
int bh_emfcomp(const bh_pool *pool, void *stream);
int bh_bfupdate(const bh_pool *pool, const double *dt_dev, void *stream);
int bh_f2cb(const bh_params *P, const bh_pool *pool, void *stream);
/* constrans::maxdivB (grid/transport.cpp:77-89): out [npatch] */
int bh_maxdivb(const bh_pool *pool, double *out, void *stream);
/* rk2integrator::div_flux and ::source (solver/integrator.cpp:18-153) at
 * every interior cell: div, src [np][8][8000] (ghost entries untouched) */
int bh_div_source(const bh_params *P, const bh_pool *pool, double *div, double *src, void *stream);
/* amrtree::ghosts (grid/grid.cpp:524-571) for the leaf patches listed in
 * `patches` (one ghost-fill wave; waves must run in order) */
int bh_ghosts(const bh_params *P, const bh_pool *pool, const int32_t *patches, int32_t n,
              void *stream);
/* reconstruction loop of rk2integrator::rkstg (solver/integrator.cpp:288-310) */
int bh_prims(const bh_params *P, const bh_pool *pool, void *stream);
/* ghosts + reconstruction loop fused, valid when every leaf patch is in a
 * single ghost-fill wave (no prolongation dependencies).  With
 * pool->status set, interior cells are recovered first, and a ghost cell
 * copied from a leaf cell at the same (r, theta) takes that cell's con2prim
 * outcome: its primitives where con2prim succeeded (the reference's two
 * con2prim calls on the identical U and position return exactly them), the
 * failure where it failed, so that the ghost cell starts at its fallback
 * (grid.cpp:538-570, integrator.cpp:288-310). */
int bh_ghosts_prims(const bh_params *P, const bh_pool *pool, void *stream);
/* No counterpart in the reference (it allocates nothing on a GPU): the
 * ghost fill and reconstruction of bh_ghosts_prims for callers that cannot
 * allocate device memory -- e.g. one whose memory arena owns every device
 * byte and lends libraries none.
 * The per-cell con2prim outcome that bh_ghosts_prims keeps in the caller's
 * pool->status is kept instead in a scratch array inside this library,
 * BH_STATIC_MAX_PATCHES x 8000 bytes (8 MB), which every GPU that loads
 * the library holds until the process exits; pool->status is ignored.
 * Nothing is allocated or freed; pools of more than BH_STATIC_MAX_PATCHES
 * patches are rejected with BH_ERANGE before anything is launched.
 * A call whose stream is not capturing looks up the array's device address
 * on the current device (cudaGetSymbolAddress), so the address stays right
 * after a device reset; a call whose stream is capturing takes the address
 * the last such lookup found on that device (BH_ECUDA if there was none).
 * Every call uses the same array and leaves its
 * contents behind; each call writes every entry it later reads, so nothing
 * needs clearing, but calls that overlap on the GPU (concurrent streams)
 * race on the array.  Results equal bh_ghosts_prims bit for bit. */
#define BH_STATIC_MAX_PATCHES 1024
int bh_ghosts_prims_static(const bh_params *P, const bh_pool *pool, void *stream);
/* conserved update loop of rkstg (solver/integrator.cpp:325-347) */
int bh_update(const bh_params *P, const bh_pool *pool, const double *dt_dev, int32_t stage,
              void *stream);
/* patch::floors (grid/grid.cpp:331-358) on every patch */
int bh_floors(const bh_params *P, const bh_pool *pool, void *stream);

/* ---- L2 AMR regrid (grid/grid.cpp:573-835) ------------------------------ */
/* The data operations of amrtree::regrid; the quilt bookkeeping (which
 * patches refine or flatten, the order of the new quilt) is the caller's,
 * from the flags below.  Plans are device arrays of rows
 * (parent, child0 .. child7), children in octant order (grid.cpp:596-599). */
/* the cell loop of amrtree::regrid (:763-820) on every leaf patch: flags[p]
 * bit 0 = patch->refine, bit 1 = patch->erase; lvl[npatch] = patch levels.
 * Entries of non-leaf patches are not written. */
int bh_regrid_flags(const bh_params *P, const bh_pool *pool, const int32_t *lvl, uint8_t *flags,
                    void *stream);
/* the cell data of amrtree::refine (:603-648) for n refined patches: the
 * children (already in the pool with zeroed arrays and geometry from
 * bh_geometry) take the parent's prolonged U, con2prim with its fallback,
 * and patch::B_init (:207-250).  n <= 8191 per call. */
int bh_refine(const bh_params *P, const bh_pool *pool, const int32_t *plan, int32_t n, void *stream);
/* amrtree::ccrstr (:651-712) + B_init for n flattened patches: each parent
 * cell takes the volume-weighted mean of its octant child's cells and
 * con2prim with its fallback.  n <= 65535 per call. */
int bh_ccrstr(const bh_params *P, const bh_pool *pool, const int32_t *plan, int32_t n, void *stream);
/* patch::B_init (:207-250) on the n listed patches */
int bh_b_init(const bh_params *P, const bh_pool *pool, const int32_t *patches, int32_t n, void *stream);

/* ---- L3 analysis (data/quantitatives.cpp) ------------------------------- */
/* Raw integrals of analysis::analyser over the leaf patches' interior cells:
 * vol_int (:44-59) and surf_int (:61-79, cells within one cell diagonal of
 * the radius) of each integrand times the cell volume, on the state a step
 * (floors) or a regrid left -- the derived fields come from pool->Wd.  The
 * sums run in a fixed order on the device (per patch, then over patches), not
 * the reference's serial order.  out[BH_NQ] in this order: */
enum { BH_Q_MASS, BH_Q_ENERGY, BH_Q_LPOL, BH_Q_MDOT, BH_Q_EDOT, BH_Q_LDOT, BH_Q_PHIB, BH_Q_MAGE,
       BH_Q_THERME, BH_Q_LBZ, BH_Q_PNUM, BH_Q_PDEN, BH_Q_ASTRESS, BH_Q_APRESS, BH_Q_ASTRESS_B,
       BH_Q_APRESS_B, BH_Q_MAXW, BH_Q_REYN, BH_Q_HNUM, BH_Q_HDEN, BH_NQ };
typedef struct bh_analysis_params {
    double hrz;             /* surface radius of the accretion integrals (r_horizon, :19-22) */
    double rs;              /* surface radius of Hscal (batch_: 10 M)                   */
    double rho_min_full;    /* density cut of alpha_ss / maxreyn in batch_ (0.01)        */
    double rho_min_bundle;  /* density cut of alpha_ss in bundle_ (0.005)                */
} bh_analysis_params;
/* partial: device scratch [nleaf][BH_NQ]; out: device [BH_NQ]; needs pool->Wd */
int bh_analysis(const bh_params *P, const bh_pool *pool, const bh_analysis_params *A, double *partial,
                double *out, void *stream);

/* ---- initial data (solver/initconds.cpp, main.cpp:89-160) --------------- */
/* The initial-data sequence of the reference's main() on the patches of
 * pool->all: the floor state of every cell (amrtree::amrtree, grid.cpp:
 * 191-205); init::fm_init (:228-591), a Fishbone-Moncrief torus with pressure
 * maximum at r_max and inner edge r_in (the reference: 12 M and 4.5 M),
 * polytrope K = 0.001 M^(Gamma-1), normalised to rho_max = 1, in the
 * interior cells; init::B_pot_init (:594-667) on every patch, face B from the
 * curl of A_phi = max(rho / rho_max - 0.2, 0) sampled at cell edges, then
 * f2cB; U = ptoc(W) in the interior cells.  Synchronises the stream and
 * allocates (stream-ordered, freed before it returns) 64 bytes of scratch.
 * out[5] (host): l0, W_in, ln h at r_max, the torus density maximum before
 * normalisation (0 where fm_init gives up and leaves the floor state), the
 * interior density maximum after it.  Returns BH_ERANGE where main() stops
 * (that maximum below 1e-14; no field, no ptoc). */
int bh_torus_init(const bh_params *P, const bh_pool *pool, double r_max, double r_in, double *out,
                  void *stream);

/* ---- learned con2prim initial guess ------------------------------------- */
/* No counterpart in the reference (its Newton iteration starts at the bracket
 * midpoint, conserved.cpp:170): a 6 -> 64 -> 64 -> 2 network (tanh) maps
 * features of a cell's conserved state to log(xi / D) and log W; con2prim
 * then starts Newton there (inside the bracket; else at the midpoint) and
 * keeps the reference's Newton, Brent fallback and acceptance tests.
 * Parameters (FP32, flat): W1 [64][6], b1 [64], W2 [64][64], b2 [64],
 * W3 [2][64], b3 [2], then 12 floats of feature normalisation (mean[6],
 * 1/std[6]); inference reads their BF16 copy and accumulates in FP32. */
#define BH_MLP_NPARAM 4738
typedef struct bh_mlp {
    float *w;                /* [BH_MLP_NPARAM + 12] device                 */
    void *wb;                /* [BH_MLP_NPARAM] device, bf16                 */
    float *adam_m, *adam_v;  /* [BH_MLP_NPARAM] device, training only        */
    int64_t step;            /* Adam steps taken (host)                      */
} bh_mlp;
/* the preamble of conserved::ctop (conserved.cpp:135-168): pre [5][n] =
 * D, tau, Ssq, Bsq, SB (with the reference's assignment loop, A2) */
int bh_ctop_pre(const bh_params *P, const double *U, const double *r, const double *th, int64_t n, double *pre,
                void *stream);
/* bh_ctop with Newton started from xi0[n] where it lies strictly inside the
 * bracket (NaN or outside: the reference's midpoint) */
int bh_ctop_guess(const bh_params *P, const double *U, const double *r, const double *th, int64_t n,
                  const double *xi0, double *W, double *Wd, int32_t *status, int32_t *iters, int32_t *path,
                  void *stream);
/* bh_ctop_guess started from the network's guess, the network on the
 * tensor cores (tcgen05, BF16 weights, FP32 accumulation in tensor memory;
 * activations as BF16 hi + lo halves): one kernel computes per cell the
 * metric, the preamble, the features and the network and writes the
 * starting points to xi0 [n] (caller's buffer, required); a second runs the
 * reference's Newton / Brent from them.  *err (device word) gets
 * BH_ERR_TIMEOUT if a tensor-core wait ran out.  Replaces the sequence
 * bh_ctop_pre, bh_mlp_guess, bh_ctop_guess. */
int bh_ctop_learned(const bh_params *P, const bh_mlp *m, const double *U, const double *r, const double *th,
                    int64_t n, double *xi0, double *W, double *Wd, int32_t *status, int32_t *iters, int32_t *path,
                    int32_t *err, void *stream);
/* xi0[n] = D exp(y0) of the network (NaN where a feature is not finite) */
int bh_mlp_guess(const bh_mlp *m, const double *pre, const double *r, int64_t n, double *xi0, void *stream);
/* one Adam step (lr > 0; lr = 0 only computes) on the mean squared error of
 * y against target [2][n]; scratch: (4 * 64 + 9) * n + BH_MLP_NPARAM floats,
 * whose last BH_MLP_NPARAM hold the gradient; loss_out (device, may be NULL)
 * receives the summed squared error */
int bh_mlp_train_step(bh_mlp *m, const double *pre, const double *r, const float *target, int64_t n, float lr,
                      float *scratch, float *loss_out, void *stream);
/* refresh the BF16 copy from the FP32 weights */
int bh_mlp_sync_bf16(bh_mlp *m, void *stream);
/* failure-detection self test (no counterpart in the reference): one CTA
 * waits, with the bounded wait of bh_ctop_learned, on an mbarrier that nothing
 * arrives on; after about a second it gives up and sets BH_ERR_TIMEOUT in
 * *err (device word) */
int bh_wait_selftest(int32_t *err, void *stream);

/* ---- launch-bound autotuning (no counterpart in the reference) ----------
 * The heaviest kernels are compiled for several numbers of resident
 * 128-thread CTAs per SM (which caps their registers per thread); which one
 * runs is chosen per process and per arithmetic variant, initially the
 * compiled-in default.  bhgpu.tune.autotune times the candidates on a
 * caller's pool and sets the fastest.  Launches made after bh_tune_set, and
 * CUDA graphs captured after it, use the new choice. */
enum {
    BH_TUNE_FLUX = 0,            /* fluxcomp face kernel (3, 4, 5, 6)          */
    BH_TUNE_UPDATE = 1,          /* f2cB + RK update (3, 4, 5, 6)              */
    BH_TUNE_PRIMS_INTERIOR = 2,  /* con2prim of interior cells (4, 6, 8)       */
    BH_TUNE_PRIMS_GHOST = 3,     /* con2prim of ghost cells (4, 6, 8)          */
    BH_TUNE_FLOORS = 4,          /* patch::floors (4, 6, 8)                    */
    BH_TUNE_NKERNEL = 5
};
/* the candidates of `kernel` into out[max]; returns their number, or BH_EINVAL */
int bh_tune_candidates(int32_t kernel, int32_t *out, int32_t max);
/* the CTAs per SM `kernel` of variant `precision` launches with */
int bh_tune_set(int32_t precision, int32_t kernel, int32_t ctas_per_sm);
int bh_tune_get(int32_t precision, int32_t kernel, int32_t *ctas_per_sm);

/* ---- L3 integrator ------------------------------------------------------ */
/* rk2integrator::dtcomp (solver/integrator.cpp:156-189): *dt_dev = CFL step */
int bh_dtcomp(const bh_params *P, const bh_pool *pool, double cfl, double *dt_dev, void *stream);
/* rk2integrator::rkstg (solver/integrator.cpp:191-260): one RK2 stage.
 * waves/nwave: ghost-fill waves (concatenated patch lists, wave_off[nwave+1]);
 * nwave == 1 uses the fused ghost+reconstruction kernel */
int bh_rkstg(const bh_params *P, const bh_pool *pool, const double *dt_dev, int32_t stage,
             const int32_t *waves, const int32_t *wave_off_host, int32_t nwave, void *stream);
/* rk2integrator::step (solver/integrator.cpp:262-275): dtcomp, two stages,
 * floors; dt stays on the device in *dt_dev */
int bh_step(const bh_params *P, const bh_pool *pool, double cfl, double *dt_dev,
            const int32_t *waves, const int32_t *wave_off_host, int32_t nwave, void *stream);

/* rk2integrator::step recorded once as a CUDA graph and replayed: the step
 * never synchronises with the host (dt stays in *dt_dev), so its launches
 * form one graph.  bh_step_graph_create captures bh_step with these
 * arguments on `stream` (required, not the legacy default stream) and
 * instantiates it; the pool's arrays, dt_dev and waves must stay valid and
 * at the same addresses while the graph lives.  The graph keeps the launch
 * bounds chosen when it was captured (bh_tune_set).  The CUDA graph objects
 * are host-side handles the CUDA runtime allocates; no device memory is
 * allocated.  (The reference has no counterpart: its step is a host loop.) */
typedef struct bh_step_graph bh_step_graph;
int bh_step_graph_create(const bh_params *P, const bh_pool *pool, double cfl, double *dt_dev,
                         const int32_t *waves, const int32_t *wave_off_host, int32_t nwave, void *stream,
                         bh_step_graph **out);
/* one step: a replay of the captured graph on `stream` (NULL: the legacy
 * default stream) */
int bh_step_graph_replay(bh_step_graph *g, void *stream);
int bh_step_graph_destroy(bh_step_graph *g);

/* ==========================================================================
 * The corrected scheme ("fixed" physics mode).  No counterpart in the
 * reference: its own scheme stops in the first step of a Kerr torus
 * (physics/thermo.cpp:10-11 reached from conserved.cpp:205) and has several
 * defects listed in csrc/bh_fixed_phys.cuh.  This is textbook Valencia GRMHD
 * in Cartesian Kerr-Schild coordinates (M, a) with the reference's structure:
 * PLM face states, two-wave HLL fluxes in each face's own normal direction,
 * geometric sources from the analytic metric derivatives, constrained
 * transport with a Heun-averaged face field, an exact-derivative Newton
 * con2prim started from the previous primitives, floors
 * (rho >= rho_floor r^-3/2, p/(Gamma-1) >= u_floor r^-5/2, b^2/rho <=
 * sigma_max, W <= W_max) and excision (cells with r < r_exc are reset to
 * the floor state at rest every stage).
 *
 * Layout: a list of cubic blocks of n^3 interior cells (n even, at least 4)
 * with three ghost layers (the fill covers two, or three with BH_PPM).  Blocks are equal cubes of space; a block of level
 * l holds twice the cells per axis of level l-1 (the 27-neighbour table
 * links equal cubes, whose levels differ by one at most): ghost cells of a
 * coarser or finer neighbour are prolonged or restricted, and the edge EMFs
 * of a coarse block along a finer one take the finer block's values; every
 * array stores each block as a (n+7)^3 box (cells -3 .. n+3 per axis) at
 * offset blocks[b].off, index ((i+3) S + (j+3)) S + (k+3), S = n + 7 (i
 * slowest, k fastest, as the reference's patches).  The x-face (i-1/2, j, k), y-face (i, j-1/2, k) and
 * z-face (i, j, k-1/2) share the index of cell (i, j, k).
 *   U, U1  [8][ncell] conserved D, S_x, S_y, S_z, tau, B^x, B^y, B^z
 *                     densitised by sqrt(gamma) (U1: the RK stage state)
 *   W      [8][ncell] primitives rho, p, ut^x, ut^y, ut^z (ut = W v, the
 *                     Eulerian velocity times its Lorentz factor), B^x, B^y,
 *                     B^z; double, or float when precision is BH_MIXED
 *   Bf, Bf1 [3][ncell] face field sqrt(gamma) B^d (Bf1: the stage's)
 *   F      [3][8][ncell] face fluxes (double, or float for BH_MIXED)
 * Work lists: items_* are device arrays of int32 pairs (block, first index)
 * of BH_FX_CHUNK consecutive indices of the block's index space: interior
 * cells (n^3, index (i n + j) n + k), flux positions ((n+2)^3, positions
 * -1 .. n per axis) and ghost cells ((n+2g)^3 - n^3, the shell of the g =
 * ghost_depth layers the fill covers).
 * ========================================================================== */
#define BH_FX_CHUNK 128
typedef struct bh_fx_params {
    double M, a, gamma;
    double cfl;
    double rho_floor, u_floor;   /* floor coefficients                             */
    double sigma_max, W_max;     /* magnetisation and Lorentz-factor ceilings       */
    double r_exc;                /* excision radius                                 */
    double tol;                  /* con2prim: stop when |dZ| <= tol Z (1e-12)       */
    int32_t maxiter;             /* con2prim Newton cap (30)                        */
    int32_t limiter;             /* BH_MINMOD / BH_VANLEER / BH_MC / BH_PPM         */
    int32_t precision;           /* BH_FP64 / BH_FP64_FMA / BH_MIXED                */
    int32_t flags;               /* BH_FX_C2P_FP64: in BH_MIXED, every cell's
                                    con2prim ends with FP64 Newton iterations (by
                                    default a cell whose FP32 iterations converge
                                    on a well-conditioned residual keeps the FP32
                                    root; the others end in FP64)                  */
} bh_fx_params;
#define BH_FX_C2P_FP64 1

typedef struct bh_fx_block {
    int32_t n, level;
    int64_t off;                 /* offset of the block's box in every array        */
    double x0[3];                /* lower corner of the interior                    */
    double dx;                   /* cell size                                       */
} bh_fx_block;

typedef struct bh_fx_grid {
    int32_t nblock;
    const bh_fx_block *blocks;   /* device [nblock]                                  */
    const int32_t *nbr;          /* device [nblock][27]: the block at offset
                                    (ox, oy, oz) in {-1,0,1}^3, index
                                    (ox+1)*9 + (oy+1)*3 + (oz+1); -1 = outside the
                                    domain (outflow)                               */
    const int32_t *items_cell; int32_t nitem_cell;
    const int32_t *items_pos;  int32_t nitem_pos;
    const int32_t *items_ghost; int32_t nitem_ghost;
    int64_t ncell;               /* entries per array (sum of (n+7)^3)               */
    double *U, *U1;
    void *W;
    double *Bf, *Bf1;
    void *F;
    double *dt;                  /* device [2]: dt[0] min over cells of dx / |signal
                                    speed|, dt[1] the step's time step cfl dt[0]    */
    int32_t *count;              /* device [4]: con2prim failures, floored cells,
                                    cells the mixed variant's FP32 con2prim handed
                                    to FP64 (away from the hole), unused            */
    int32_t *err;                /* device error word                                */
    double *E;                   /* [3][ncell] edge EMFs, or NULL: computed on the fly
                                    (allowed only when every block has one level)  */
    int32_t maxlevel;            /* highest block level (0: one level)               */
    int32_t queue_ctas;          /* CTAs of a persistent launch (0: the SMs times the
                                    CTAs the kernel keeps resident per SM)          */
    int32_t *queue;              /* device [2 * BH_FX_QSLOTS], zeroed once before the
                                    first launch, or NULL.  Set: every step kernel is
                                    launched persistent, its CTAs taking work items
                                    from a counter in this array (the counters reset
                                    themselves at the end of each launch).  NULL: one
                                    CTA per work item.  Both give the same results. */
    const int32_t *items_flux;   /* device [nitem_flux][2] (block, e), or NULL/0: the work
                                    of the staged flux kernel.  e >= 0: tile e of the
                                    block's position box [-1, n]^3, tiles of 4 x 4 x 8
                                    positions (i, j, k), tile index (ti * nj + tj) * nk
                                    + tk with nj = ceil((n+2)/4), nk = ceil((n+2)/8);
                                    e < 0: the 128 positions from -(e+1) on, as in
                                    items_pos (bhgrid.blocks.flux_items builds it)  */
    int32_t nitem_flux;
    int32_t ghost_depth;         /* ghost layers the fill covers (and items_ghost
                                    lists): 2 (0 reads as 2), or 3, which BH_PPM
                                    requires                                        */
} bh_fx_grid;
#define BH_FX_QSLOTS 7

/* Launch bounds of the scheme's three heavy kernels (no counterpart in the
 * reference): each is compiled for 1 (no register cap) and 3 to 8
 * resident 128-thread CTAs per SM; the choice is per process and variant,
 * initially 1.  BH_FX_TUNE_STAGE (0 or 1, initially 0) selects the flux
 * kernel: 1 = the stencil staged in shared memory per tile (items_flux; grids
 * without items_flux keep the unstaged kernel), with the launch bounds of
 * BH_FX_TUNE_FLUX.  BH_FX_TUNE_SPLIT (0 or 1, initially 0): 1 = the update
 * as two kernels, the conserved state (launch bounds of BH_FX_TUNE_UPDATE)
 * and the face field.  bhgpu.fixed.autotune times the candidates on a grid and
 * sets the fastest.  Launches (and graphs captured) after the call use it. */
enum { BH_FX_TUNE_C2P = 0, BH_FX_TUNE_FLUX = 1, BH_FX_TUNE_UPDATE = 2, BH_FX_TUNE_STAGE = 3, BH_FX_TUNE_SPLIT = 4,
       BH_FX_TUNE_N = 5 };
int bh_fx_tune_set(int32_t precision, int32_t kernel, int32_t ctas_per_sm);
int bh_fx_tune_get(int32_t precision, int32_t kernel, int32_t *ctas_per_sm);

/* one RK2 step: con2prim (+ CFL reduction), ghost fill, fluxes, update, twice */
int bh_fx_step(const bh_fx_params *P, const bh_fx_grid *g, void *stream);
/* bh_fx_step recorded once as a CUDA graph (9 launches; dt stays on the
 * device): replay and release it with bh_step_graph_replay / _destroy.
 * stream is required (not the legacy default stream); the grid's arrays
 * must stay valid at the same addresses while the graph lives. */
int bh_fx_graph_create(const bh_fx_params *P, const bh_fx_grid *g, void *stream, bh_step_graph **out);
/* the pieces of a stage (stage 0 works on U/Bf, stage 1 on U1/Bf1) */
int bh_fx_prims(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, int32_t with_dt, void *stream);
int bh_fx_ghosts(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, void *stream);
/* one pass of bh_fx_ghosts (pass 0: copies and restrictions; pass l in
 * 1..maxlevel: prolongations into level-l blocks), for a grid whose blocks
 * are shared with other processes: the neighbours' boxes are exchanged
 * between passes (bhgpu.fxshard) */
int bh_fx_ghost_pass(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, int32_t pass, void *stream);
int bh_fx_fluxes(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, void *stream);
int bh_fx_update(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, void *stream);
/* bh_fx_update in two parts, for a grid whose blocks are shared with other
 * processes (bhgpu.fxshard): bh_fx_emf writes the edge EMFs of the grid's own
 * blocks (the work lists) into E; bh_fx_update_from_emf applies the
 * level-change correction, which reads E of finer neighbours (their EMFs
 * copied in beforehand where another process owns them), and the update.
 * Both require E. */
int bh_fx_emf(const bh_fx_params *P, const bh_fx_grid *g, void *stream);
int bh_fx_update_from_emf(const bh_fx_params *P, const bh_fx_grid *g, int32_t stage, void *stream);
/* The state a step reads -- rows 0-4 of U (conserved fluid) and of W (the
 * previous primitives, con2prim's start) and the blocks' own face field --
 * between the grid's boxes and a compact device buffer (dir 0: pack, 1:
 * unpack; the cell-centred field rows 5-7 are recomputed by the step's
 * con2prim).  Layout, Q = nitem_cell * BH_FX_CHUNK slots, slot q = item *
 * BH_FX_CHUNK + lane of items_cell: double U[5][Q]; W[5][Q] (float for
 * BH_MIXED, else double); double Bf[3][Q] (each cell's three lower faces);
 * then per block b from face_off[b] (device, doubles) its upper boundary
 * faces, 3 n^2: x-faces at i = n in (j, k) order, y at j = n in (i, k), z at
 * k = n in (i, j).  Slots past a block's last cell are not touched. */
int bh_fx_pack_state(const bh_fx_params *P, const bh_fx_grid *g, const int64_t *face_off, void *packed,
                     int32_t dir, void *stream);
/* max over each block's interior cells of |div B~| / max |B~| of the cell's
 * faces (a relative divergence, 0 up to roundoff under CT): out [nblock]
 * device, cleared by the call */
int bh_fx_divb(const bh_fx_grid *g, double *out, void *stream);

/* Fishbone-Moncrief torus (pressure maximum at r_max, inner edge r_in,
 * polytrope p = kappa rho^Gamma normalised to rho_max = 1) in the atmosphere
 * of the floors, pressure perturbed by (1 + noise (2 u - 1)) with u uniform
 * from a hash of the seed and the cell's global integer coordinates (the
 * same for any cutting of the grid into blocks), and a single field loop from
 * A_phi = max(rho / rho_max - 0.2, 0) scaled so that max p_gas / max p_mag
 * = beta over the interior cells.  Fills W, U (every cell of every box), Bf.
 * scratch: device [4] doubles.  out (host, may be NULL) [4]: the torus's
 * specific angular momentum u^t u_phi, the density maximum before
 * normalisation, the field scale applied, max p_gas / max p_mag after it. */
typedef struct bh_fx_torus {
    double r_in, r_max, kappa, beta, noise;
    uint64_t seed;
} bh_fx_torus;
int bh_fx_torus_init(const bh_fx_params *P, const bh_fx_grid *g, const bh_fx_torus *T, double *scratch,
                     double *out, void *stream);

/* ---- FMA throughput (no counterpart in the reference) -------------------
 * n threads each run `iters` rounds of independent multiply-add chains in
 * FP64 (precision BH_FP64, 8 chains) or FP32 (BH_MIXED, 16 chains) and
 * write one value to out[n] (device, caller-allocated); *flops receives the
 * floating-point operations issued (2 per multiply-add).  Timed by the
 * caller, it gives the pipe peaks that bound the compute-heavy kernels. */
int bh_peak_fma(int32_t precision, int32_t iters, void *out, int64_t n, int64_t *flops, void *stream);

#ifdef __cplusplus
}
#endif
#endif
