/*
 * bh_oracle.h -- CPU restatement of the reference GRMHD block update.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation: tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product library never does.
 *
 * Every function restates one function of the reference fluid solver
 * (Fjoerde/black-hole-simulator, src/fluid) in plain C, keeping the
 * reference's floating-point operation order so that a build with
 * -ffp-contract=off reproduces the compiled reference bit for bit.
 * Deliberate deviations from the reference are limited to:
 *   - conserved.cpp:144-150 reads B[j], S[j] for j>i before they are
 *     assigned (undefined behaviour).  With a zeroed stack the compiled
 *     reference behaves as if those reads return 0; this restatement
 *     implements exactly that.
 *   - std::domain_error (thermo.cpp:11-31) becomes the return code
 *     ORC_EDOMAIN, which the callers propagate like the exception.
 *
 * Data layout (shared with the CUDA library and the harness around the
 * compiled reference): one "pool" of patches of 16^3 interior cells plus
 * 2 ghost layers, structure-of-arrays per patch, using the reference's
 * per-patch linear indices (grid.cpp:51-89).
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_BLOCK = 16, ORC_GHOST = 2, ORC_CPN = 20,
    ORC_NC = 8000,  /* cells per patch, cpn^3                          */
    ORC_NF = 8400,  /* faces per direction, (cpn+1)*cpn*cpn             */
    ORC_NE = 8820,  /* edges per direction, cpn*(cpn+1)*(cpn+1)         */
    ORC_NMC = 120   /* doubles in the metriccomp struct (metric.hpp:11) */
};

/* conserved order (cons.hpp:14-18) and primitive order (prim.hpp:14-18) */
enum { ORC_D = 0, ORC_S0 = 1, ORC_S1 = 2, ORC_S2 = 3, ORC_TAU = 4, ORC_B0 = 5 };
enum { ORC_RHO = 0, ORC_EPS = 1, ORC_V0 = 2 };

/* neighbour kinds for the ghost fill (grid.cpp:524-536) */
enum { ORC_NB_BNDY = 0, ORC_NB_COPY = 1, ORC_NB_PROLONG = 2 };

/* return codes */
enum { ORC_OK = 0, ORC_EDOMAIN = -1 };

typedef struct orc_params {
    double M, a, Q;   /* metric(M,a,Q)             metric.hpp:28-32 */
    double gamma;     /* state(gm)                 state.hpp:11     */
    int32_t limiter;  /* 0 minmod, 1 vanleer, 2 mc recon.hpp:36     */
    int32_t maxiter;  /* ctop default 500          cons.hpp:75      */
    double tol;       /* ctop default 1e-10        cons.hpp:75      */
    /* metric held by every cell (cell.hpp:25, `const metric mtr;`): it is
     * default-constructed, i.e. metric() = (M=1, a=0, Q=0) (metric.hpp:30),
     * whatever the tree's metric is.  Used by reconfp's causality check,
     * div_flux, source, dtcomp, f2cB and the RK update. */
    double cM, ca, cQ;
} orc_params;

typedef struct orc_pool {
    int32_t npatch;
    double *U;      /* [np][8][NC]  conserved, all 20^3 cells            */
    double *W;      /* [np][8][NC]  primitives rho,eps,v[3],B[3]         */
    double *dU;     /* [np][8][NC]  RK accumulator (interior used)       */
    double *F;      /* [np][3][8][NF] face fluxes Fx,Fy,Fz               */
    double *Bf;     /* [np][3][NF]  face-centred B: Bfx,Bfy,Bfz          */
    double *EMF;    /* [np][3][NE]  edge EMFs: EMFx,EMFy,EMFz            */
    double *rth;    /* [np][2][NC]  cell-centre r, theta                 */
    double *pgeo;   /* [np][6]      xedge[0], yedge[0], zedge[0], dx,dy,dz */
    int32_t *nbr;   /* [np][6][2]   (neighbour index, kind), slot dim*2+(side>0) */
    uint8_t *leaf;  /* [np]                                              */
    int32_t *lvl;   /* [np]                                              */
    int32_t *ijk;   /* [np][3]                                           */
    double *Wd;     /* [np][4][NC] lor, p, h, b2 of the primitives that
                       floors and regrid set (NULL: not kept)           */
} orc_pool;

/* ---- L0 physics ------------------------------------------------------ */
void orc_metric_comp(const orc_params *P, double r, double th, double mc[ORC_NMC]);
/* ptoc: W[8] in, U[8] out, Wd[4] = lor,p,h,b2 (the fields ptoc mutates) */
int orc_ptoc(const orc_params *P, const double W[8], double r, double th,
             double U[8], double Wd[4]);
/* ctop: returns 1 ok, 0 failed, ORC_EDOMAIN on a thrown domain_error.
 * Wd[5] = p,T,h,lor,b2.  iters = Newton iterations taken,
 * path = 0 Newton converged, 1 Newton ran out of iterations,
 *        2 Brent root, 3 Brent failed.                              */
int orc_ctop(const orc_params *P, const double U[8], double r, double th,
             double W[8], double Wd[5], int32_t *iters, int32_t *path);
int orc_hlld(const orc_params *P, const double WL[8], const double WR[8],
             const double UL[8], const double UR[8], double r, double th,
             int dim, double F[8], double *ctspeed);
void orc_pvfs(const orc_params *P, double r, double W[8]);

/* ---- L1/L2 per patch --------------------------------------------------- */
void orc_geometry(orc_pool *pool);
void orc_reconfp(const orc_params *P, const orc_pool *pool, int p, int i, int j,
                 int k, int dim, int lim, double L[8], double R[8]);
int  orc_fluxcomp(const orc_params *P, orc_pool *pool, int p);
void orc_emfcomp(orc_pool *pool, int p);
void orc_bfupdate(orc_pool *pool, int p, double dt);
void orc_f2cb(const orc_params *P, orc_pool *pool, int p);
double orc_maxdivb(const orc_pool *pool, int p);
void orc_div_flux(const orc_params *P, const orc_pool *pool, int p, int i, int j,
                  int k, double out[8]);
int  orc_source(const orc_params *P, const orc_pool *pool, int p, int i, int j,
                int k, double out[8]);
int  orc_ghosts(const orc_params *P, orc_pool *pool, int p);
int  orc_floors(const orc_params *P, orc_pool *pool, int p);

/* ---- L2 AMR regrid (grid.cpp:573-835) ---------------------------------- */
int  orc_regrid_flags(const orc_pool *pool, int p, int lvl);   /* bit 0 refine, bit 1 erase */
void orc_b_init(orc_pool *pool, int p);
int  orc_refine_data(const orc_params *P, orc_pool *pool, int p, const int32_t child[8]);
int  orc_ccrstr(const orc_params *P, orc_pool *pool, int p, const int32_t child[8]);

/* ---- L3 analysis (data/quantitatives.cpp) ----------------------------- */
/* the raw integrals of analysis::analyser over the leaf patches' interior
 * cells, each summed in the reference's order; out[ORC_NQ] (ORC_Q_* below).
 * hrz = horizon radius of surf_int, rs = Hscal's radius, rho_min_full and
 * rho_min_bundle = the density cuts of batch_ (0.01) and bundle_ (0.005) */
enum { ORC_Q_MASS, ORC_Q_ENERGY, ORC_Q_LPOL, ORC_Q_MDOT, ORC_Q_EDOT, ORC_Q_LDOT, ORC_Q_PHIB,
       ORC_Q_MAGE, ORC_Q_THERME, ORC_Q_LBZ, ORC_Q_PNUM, ORC_Q_PDEN, ORC_Q_ASTRESS, ORC_Q_APRESS,
       ORC_Q_ASTRESS_B, ORC_Q_APRESS_B, ORC_Q_MAXW, ORC_Q_REYN, ORC_Q_HNUM, ORC_Q_HDEN, ORC_NQ };
void orc_analysis(const orc_params *P, const orc_pool *pool, double hrz, double rs, double rho_min_full,
                  double rho_min_bundle, double out[ORC_NQ], double out_abs[ORC_NQ]);   /* out_abs: sum |f vol|, may be NULL */

/* ---- L3 integrator ------------------------------------------------------ */
int orc_dtcomp(const orc_params *P, const orc_pool *pool, double cfl, double *dt);
int orc_prims(const orc_params *P, orc_pool *pool);          /* integrator.cpp:288-310 */
int orc_update(const orc_params *P, orc_pool *pool, double dt, int stage); /* :325-347 */
int orc_rkstg(const orc_params *P, orc_pool *pool, double dt, int stage);
int orc_step(const orc_params *P, orc_pool *pool, double cfl, double *dt);

/* ctop with a learned Newton start (xi0 NaN: the reference's midpoint) */
void orc_ctop_guess_batch(const orc_params *P, const double *U, const double *r, const double *th, int64_t n,
                          const double *xi0, double *W, double *Wd, int32_t *status, int32_t *iters,
                          int32_t *path, double *pre);

/* batch helpers used by the tests (vectorised over n items, SoA [8][n]) */
void orc_metric_batch(const orc_params *P, const double *r, const double *th,
                      int64_t n, double *mc);
int  orc_ptoc_batch(const orc_params *P, const double *W, const double *r,
                    const double *th, int64_t n, double *U, double *Wd);
void orc_ctop_batch(const orc_params *P, const double *U, const double *r,
                    const double *th, int64_t n, double *W, double *Wd,
                    int32_t *status, int32_t *iters, int32_t *path);
void orc_hlld_batch(const orc_params *P, const double *WL, const double *WR,
                    const double *UL, const double *UR, const double *r,
                    const double *th, int dim, int64_t n, double *F,
                    double *cts, int32_t *status);
void orc_reconfp_all(const orc_params *P, const orc_pool *pool, int dim, int lim,
                     double *L, double *R);
int  orc_fluxcomp_all(const orc_params *P, orc_pool *pool);
void orc_ct_all(const orc_params *P, orc_pool *pool, double dt);
void orc_div_source_all(const orc_params *P, const orc_pool *pool, double *div,
                        double *src);
int  orc_ghosts_all(const orc_params *P, orc_pool *pool);
int  orc_floors_all(const orc_params *P, orc_pool *pool);
void orc_maxdivb_all(const orc_pool *pool, double *out);

#ifdef __cplusplus
}
#endif
#endif
