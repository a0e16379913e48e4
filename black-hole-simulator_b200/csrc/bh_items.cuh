// bh_items.cuh -- the per-item work of every kernel (one cell, face, edge
// or ghost cell), written once as __host__ __device__ functions.
//
// The __global__ kernels in bh_variant.cuh map their thread index to an
// item and call these; the CPU check of the kernel logic
// (tests/hostcheck) compiles the same functions for the host and runs
// them in loops.  Items of one launch never depend on each other.
#pragma once
#include "bh_phys.cuh"

namespace bh {

struct KP {                 // kernel-side copy of bh_params
    MP tree, cell;
    double gamma, tol;
    int limiter, maxiter;
};
inline KP kp_of(const bh_params* P) {
    KP k;
    k.tree = MP{P->M, P->a, P->Q};
    k.cell = MP{P->cM, P->ca, P->cQ};
    k.gamma = P->gamma; k.tol = P->tol; k.limiter = P->limiter; k.maxiter = P->maxiter;
    return k;
}

struct Pool {               // kernel-side view of bh_pool
    double *U, *W, *dU, *F, *Bf, *EMF, *rth;
    const double* pgeo;
    const int32_t* nbr;
    int32_t* err;
    const uint8_t* leafmask;
    uint8_t* status;
    double* aux;
    double* Wd;
};
inline Pool pool_of(const bh_pool* p) {
    return Pool{p->U, p->W, p->dU, p->F, p->Bf, p->EMF, p->rth, p->pgeo, p->nbr, p->err, p->leafmask, p->status,
                p->aux, p->Wd};
}
// the derived fields lor, p, h, b2 of a cell's primitives (pool->Wd)
BH_HD inline void store_derived(const Pool& P, int p, int l, double lor, double pr, double h, double b2) {
    double* d = P.Wd + (size_t)p * 4 * NC;
    d[l] = lor; d[NC + l] = pr; d[2 * NC + l] = h; d[3 * NC + l] = b2;
}

BH_HD inline double* Uv(const Pool& P, int p, int v) { return P.U + ((size_t)p * 8 + v) * NC; }
BH_HD inline double* Wv(const Pool& P, int p, int v) { return P.W + ((size_t)p * 8 + v) * NC; }
BH_HD inline double* dUv(const Pool& P, int p, int v) { return P.dU + ((size_t)p * 8 + v) * NC; }
BH_HD inline double* Fv(const Pool& P, int p, int d, int v) { return P.F + (((size_t)p * 3 + d) * 8 + v) * NF; }
BH_HD inline double* Bfv(const Pool& P, int p, int d) { return P.Bf + ((size_t)p * 3 + d) * NF; }
BH_HD inline double* Ev(const Pool& P, int p, int d) { return P.EMF + ((size_t)p * 3 + d) * NE; }
BH_HD inline double rr(const Pool& P, int p, int l) { return P.rth[(size_t)p * 2 * NC + l]; }
BH_HD inline double tt(const Pool& P, int p, int l) { return P.rth[((size_t)p * 2 + 1) * NC + l]; }

BH_HD inline void load_prim(const Pool& P, int p, int l, Prim& w) {
    w.rho = Wv(P, p, 0)[l]; w.eps = Wv(P, p, 1)[l];
    for (int d = 0; d < 3; d++) { w.v[d] = Wv(P, p, 2 + d)[l]; w.B[d] = Wv(P, p, 5 + d)[l]; }
}
BH_HD inline void store_prim(const Pool& P, int p, int l, const Prim& w) {
    Wv(P, p, 0)[l] = w.rho; Wv(P, p, 1)[l] = w.eps;
    for (int d = 0; d < 3; d++) { Wv(P, p, 2 + d)[l] = w.v[d]; Wv(P, p, 5 + d)[l] = w.B[d]; }
}
BH_HD inline void load_cons(const Pool& P, int p, int l, Cons& c) {
    c.D = Uv(P, p, 0)[l]; c.tau = Uv(P, p, 4)[l];
    for (int d = 0; d < 3; d++) { c.S[d] = Uv(P, p, 1 + d)[l]; c.B[d] = Uv(P, p, 5 + d)[l]; }
}
BH_HD inline void store_cons(const Pool& P, int p, int l, const Cons& c) {
    Uv(P, p, 0)[l] = c.D; Uv(P, p, 4)[l] = c.tau;
    for (int d = 0; d < 3; d++) { Uv(P, p, 1 + d)[l] = c.S[d]; Uv(P, p, 5 + d)[l] = c.B[d]; }
}
BH_HD inline void lin_ijk(int l, int& i, int& j, int& k) {
    i = l / (CPN * CPN) - GH; j = (l / CPN) % CPN - GH; k = l % CPN - GH;
}
BH_HD inline bool is_ghost(int i, int j, int k) {
    return i < 0 || i >= BLK || j < 0 || j >= BLK || k < 0 || k >= BLK;
}

// item counts per patch
constexpr int N_INT = BLK * BLK * BLK;   // interior cells
constexpr int N_EDGE = 19 * 19 * 19;     // emfcomp, i,j,k in [-2,17)
constexpr int N_BUP = 18 * 18 * 18;      // Bfupdate / maxdivB, i,j,k in [-1,17)
constexpr int N_F2C = 19 * 19 * 19;      // f2cB, i,j,k in [-1,18)
constexpr int N_STRIP = 6 * 2 * BLK * BLK;  // ghost strip cells
constexpr int N_GHOST = NC - N_INT;         // all ghost cells
constexpr int N_EDGEC = N_GHOST - N_STRIP;  // edge and corner ghost cells (832)

// linear indices of the edge and corner ghost cells (two or three of
// i, j, k outside [0,16)), in lindx order
struct EdgeCells {
    short l[N_EDGEC];
    constexpr EdgeCells() : l() {
        int n = 0;
        for (int i = -GH; i < BLK + GH; i++)
            for (int j = -GH; j < BLK + GH; j++)
                for (int k = -GH; k < BLK + GH; k++) {
                    int out = (i < 0 || i >= BLK) + (j < 0 || j >= BLK) + (k < 0 || k >= BLK);
                    if (out >= 2) l[n++] = (short)((i + GH) * CPN * CPN + (j + GH) * CPN + (k + GH));
                }
    }
};
static __constant__ EdgeCells kEdgeCells = EdgeCells();   // device copy (one per translation unit)
static constexpr EdgeCells hEdgeCells = EdgeCells();      // host copy
#ifdef __CUDA_ARCH__
#define BH_EDGE_CELLS kEdgeCells
#else
#define BH_EDGE_CELLS hEdgeCells
#endif

// W = pvfs(r) with the cell's B kept; U = ptoc(W) (integrator.cpp:211-218,
// grid.cpp:484-487, grid.cpp:349-353)
BH_HD inline void floor_reset(const KP& k, const Pool& P, int p, int l, Prim& w, Cons& u, PtocOut* po = nullptr) {
    double r = rr(P, p, l), th = tt(P, p, l);
    pvfs(r, w.rho, w.eps);
    w.v[0] = w.v[1] = w.v[2] = 0.0;
    Met mc;
    met_comp(k.tree, r, th, mc);
    if (!ptoc(k.gamma, mc, w, u, po)) flag(P.err, BH_ERR_DOMAIN);
}

// ctop with the fallback of refine and ccrstr (grid.cpp:636-645, 694-703),
// recording the derived fields of the primitives it leaves in pool->Wd
BH_HD inline void recover_keep_derived(const KP& k, const Pool& P, int p, int l, Prim& w, Cons& u) {
    Met mc;
    met_comp(k.tree, rr(P, p, l), tt(P, p, l), mc);
    Prim pv;
    bool dom = false;
    CtopOut co;
    int ok = ctop(k.gamma, k.maxiter, k.tol, mc, u, pv, dom, P.Wd ? &co : nullptr);
    if (dom) flag(P.err, BH_ERR_DOMAIN);
    if (ok) {
        w = pv;
        if (P.Wd) store_derived(P, p, l, co.lor, co.p, co.h, co.b2);
        return;
    }
    PtocOut po;
    floor_reset(k, P, p, l, w, u, &po);
    if (P.Wd) store_derived(P, p, l, po.lor, po.p, po.h, po.b2);
}

// ctop of one cell with the tree metric, rkstg's fallback on failure
BH_HD inline void recover_cell(const KP& k, const Pool& P, int p, int l, Prim& w, Cons& u, bool& dirty) {
    Met mc;
    met_comp(k.tree, rr(P, p, l), tt(P, p, l), mc);
    Prim pv;
    bool dom = false;
    int ok = ctop(k.gamma, k.maxiter, k.tol, mc, u, pv, dom);
    if (dom) flag(P.err, BH_ERR_DOMAIN);
    if (ok) w = pv;
    else { floor_reset(k, P, p, l, w, u); dirty = true; }
}

// ctop of one ghost cell as amrtree::ghosts does it (grid.cpp:538-570): on
// failure only rho and eps take the floor values, v and B stay, U = ptoc(W)
BH_HD inline void ghost_recover(const KP& kp, const Pool& P, int p, int l, Prim& w, Cons& u, bool& dirty) {
    double r = rr(P, p, l), th = tt(P, p, l);
    Met mc;
    met_comp(kp.tree, r, th, mc);
    Prim pv;
    bool dom = false;
    int ok = ctop(kp.gamma, kp.maxiter, kp.tol, mc, u, pv, dom);
    if (dom) flag(P.err, BH_ERR_DOMAIN);
    if (ok) { w = pv; return; }
    pvfs(r, w.rho, w.eps);
    if (!ptoc(kp.gamma, mc, w, u)) flag(P.err, BH_ERR_DOMAIN);
    dirty = true;
}

// ---- geometry: patch::cell_init (grid.cpp:149-175) ---------------------
BH_HD inline void geometry_item(const Pool& P, int p, int l) {
    int i, j, k;
    lin_ijk(l, i, j, k);
    const double* g = P.pgeo + 6 * p;
    double xc = g[0] + (i + 0.5) * g[3];
    double yc = g[1] + (j + 0.5) * g[4];
    double zc = g[2] + (k + 0.5) * g[5];
    double r = sqrt(xc * xc + yc * yc + zc * zc);
    if (r < 1e-10) r = 1e-10;
    double th = acos(smax(-1.0, smin(1.0, zc / r)));
    P.rth[(size_t)p * 2 * NC + l] = r;
    P.rth[((size_t)p * 2 + 1) * NC + l] = th;
}

// ---- face index of patch::fluxcomp's loops (grid.cpp:258-328) ------------
BH_HD inline void face_ijk(int dim, int f, int& i, int& j, int& k) {
    if (dim == 0) { i = f / 256 - 1; j = (f / 16) % 16; k = f % 16; }
    else if (dim == 1) { i = f / (17 * 16); j = (f / 16) % 17 - 1; k = f % 16; }
    else { i = f / (16 * 17); j = (f / 17) % 16; k = f % 17 - 1; }
}

// per-cell inputs of reconfp, computed once per cell ahead of the face loop
// (each cell is read by up to 12 faces): log rho and log eps, in RT and
// stored widened to FP64, and the entries of the cell's spatial metric that
// causalv reads -- gam00, gam02 (= gam20), gam11, gam22; the other entries
// are metric::comp's structural zeros
constexpr int NAUX = 6;
template <typename RT>
BH_HD inline void aux_item(const KP& kp, const Pool& P, int p, int l) {
    double* a = P.aux + (size_t)p * NAUX * NC;
    a[l] = double(log(RT(Wv(P, p, 0)[l])));
    a[NC + l] = double(log(RT(Wv(P, p, 1)[l])));
    Met m;
    met_comp(kp.cell, rr(P, p, l), tt(P, p, l), m);
    a[2 * NC + l] = m.gam[0][0];
    a[3 * NC + l] = m.gam[0][2];
    a[4 * NC + l] = m.gam[1][1];
    a[5 * NC + l] = m.gam[2][2];
}
template <typename RT>
BH_HD inline void aux_gam(const Pool& P, int p, int l, RT g[3][3]) {
    const double* a = P.aux + (size_t)p * NAUX * NC + 2 * NC;
    g[0][0] = RT(a[l]);          g[0][1] = RT(0.0);           g[0][2] = RT(a[NC + l]);
    g[1][0] = RT(0.0);           g[1][1] = RT(a[2 * NC + l]); g[1][2] = RT(0.0);
    g[2][0] = RT(a[NC + l]);     g[2][1] = RT(0.0);           g[2][2] = RT(a[3 * NC + l]);
}

// reconfp (reconstruction.cpp:40-97) for the face between cells (i,j,k)
// and (i,j,k)+e_dim of patch p, computed in RT (the stored primitives and
// the cell metric are FP64 and rounded to RT).  AUX reads the logarithms and
// the cell metric from the per-cell scratch (aux_item) instead of computing
// them here; the values are the same.
template <typename RT, bool AUX = false>
BH_HD inline void reconfp(const KP& kp, const Pool& P, int p, int i, int j, int k, int dim, int lim, PrimT<RT>& L,
                          PrimT<RT>& R) {
    int di = dim == 0, dj = dim == 1, dk = dim == 2;
    int lm = lindx(i - di, j - dj, k - dk), lc = lindx(i, j, k);
    int lp = lindx(i + di, j + dj, k + dk), lpp = lindx(i + 2 * di, j + 2 * dj, k + 2 * dk);
    if (AUX) {
        const double* lr = P.aux + (size_t)p * NAUX * NC;
        const double* le = lr + NC;
        recon_scal(RT(lr[lm]), RT(lr[lc]), RT(lr[lp]), RT(lr[lpp]), lim, L.rho, R.rho);
        L.rho = exp(L.rho); R.rho = exp(R.rho);
        recon_scal(RT(le[lm]), RT(le[lc]), RT(le[lp]), RT(le[lpp]), lim, L.eps, R.eps);
        L.eps = exp(L.eps); R.eps = exp(R.eps);
    } else {
        const double* Wr = Wv(P, p, 0);
        recon_scal(log(RT(Wr[lm])), log(RT(Wr[lc])), log(RT(Wr[lp])), log(RT(Wr[lpp])), lim, L.rho, R.rho);
        L.rho = exp(L.rho); R.rho = exp(R.rho);
        const double* We = Wv(P, p, 1);
        recon_scal(log(RT(We[lm])), log(RT(We[lc])), log(RT(We[lp])), log(RT(We[lpp])), lim, L.eps, R.eps);
        L.eps = exp(L.eps); R.eps = exp(R.eps);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double* x = Wv(P, p, 2 + d);
        recon_scal(RT(x[lm]), RT(x[lc]), RT(x[lp]), RT(x[lpp]), lim, L.v[d], R.v[d]);
    }
    if (AUX) {
        RT gL[3][3], gR[3][3];
        aux_gam(P, p, lc, gL);
        aux_gam(P, p, lp, gR);
        causalv_gam(L.v, gL);
        causalv_gam(R.v, gR);
    } else {
        Met mL, mR;
        met_comp(kp.cell, rr(P, p, lc), tt(P, p, lc), mL);
        met_comp(kp.cell, rr(P, p, lp), tt(P, p, lp), mR);
        causalv(L.v, met_cast<RT>(mL));
        causalv(R.v, met_cast<RT>(mR));
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double* x = Wv(P, p, 5 + d);
        if (d == dim) { L.B[d] = RT(x[lc]); R.B[d] = RT(x[lp]); }
        else recon_scal(RT(x[lm]), RT(x[lc]), RT(x[lp]), RT(x[lpp]), lim, L.B[d], R.B[d]);
    }
}

template <typename RT>
BH_HD inline void reconfp_item(const KP& kp, const Pool& P, int p, int dim, int f, int lim, int64_t n, double* Lo,
                               double* Ro) {
    int i, j, k;
    face_ijk(dim, f, i, j, k);
    PrimT<RT> L, R;
    reconfp<RT>(kp, P, p, i, j, k, dim, lim, L, R);
    int64_t q = (int64_t)p * NFACE + f;
    Lo[q] = L.rho; Lo[n + q] = L.eps; Ro[q] = R.rho; Ro[n + q] = R.eps;
    for (int d = 0; d < 3; d++) {
        Lo[(2 + d) * n + q] = L.v[d]; Lo[(5 + d) * n + q] = L.B[d];
        Ro[(2 + d) * n + q] = R.v[d]; Ro[(5 + d) * n + q] = R.B[d];
    }
}

// one face of patch::fluxcomp (grid.cpp:255-329): reconstruction, face
// ptoc and HLLD in RT; face metric evaluated in FP64; flux stored in FP64
template <typename RT, bool AUX = false>
BH_HD inline void flux_item(const KP& kp, const Pool& P, int p, int dim, int f) {
    int i, j, k;
    face_ijk(dim, f, i, j, k);
    PrimT<RT> L, R;
    reconfp<RT, AUX>(kp, P, p, i, j, k, dim, kp.limiter, L, R);
    double bn;
    int fi;
    if (dim == 0) { bn = Bfv(P, p, 0)[xfc(i + 1, j, k)]; fi = xfc(i, j, k); }
    else if (dim == 1) { bn = Bfv(P, p, 1)[yfc(i, j + 1, k)]; fi = yfc(i, j, k); }
    else { bn = Bfv(P, p, 2)[zfc(i, j, k + 1)]; fi = zfc(i, j, k); }
    // constant indices keep L and R in registers (dim is a launch index)
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (d == dim) { L.B[d] = RT(bn); R.B[d] = RT(bn); }
    int lL = lindx(i, j, k), lR = lindx(i + (dim == 0), j + (dim == 1), k + (dim == 2));
    double rf = (rr(P, p, lL) + rr(P, p, lR)) / 2;
    double thf = (tt(P, p, lL) + tt(P, p, lR)) / 2;
    Met md;
    met_comp(kp.tree, rf, thf, md);
    MetT<RT> mc = met_cast<RT>(md);
    ConsT<RT> UL, UR;
    RT g = RT(kp.gamma);
    bool ok = ptoc(g, mc, L, UL);
    ok &= ptoc(g, mc, R, UR);
    RT F[8], cts;
    ok &= hlld(g, mc, L, R, UL, UR, 0 /* every call site passes dim 0 */, F, cts);
    if (!ok) flag(P.err, BH_ERR_DOMAIN);
    for (int v = 0; v < 8; v++) Fv(P, p, dim, v)[fi] = F[v];
}

// ---- constrained transport (transport.cpp) ----------------------------
BH_HD inline void emf_item(const Pool& P, int p, int e) {                // emfcomp :11-36
    int i = e / 361 - 2, j = (e / 19) % 19 - 2, k = e % 19 - 2;
    const double *FxB1 = Fv(P, p, 0, 6), *FxB2 = Fv(P, p, 0, 7);
    const double *FyB0 = Fv(P, p, 1, 5), *FyB2 = Fv(P, p, 1, 7);
    const double *FzB0 = Fv(P, p, 2, 5), *FzB1 = Fv(P, p, 2, 6);
    Ev(P, p, 0)[exi(i, j, k)] = (FyB2[yfc(i, j, k)] + FyB2[yfc(i, j, k + 1)] - FzB1[zfc(i, j, k)] - FzB1[zfc(i, j + 1, k)]) / 4;
    Ev(P, p, 1)[eyi(i, j, k)] = (FzB0[zfc(i, j, k)] + FzB0[zfc(i + 1, j, k)] - FxB2[xfc(i, j, k)] - FxB2[xfc(i, j, k + 1)]) / 4;
    Ev(P, p, 2)[ezi(i, j, k)] = (FxB1[xfc(i, j, k)] + FxB1[xfc(i, j + 1, k)] - FyB0[yfc(i, j, k)] - FyB0[yfc(i + 1, j, k)]) / 4;
}

BH_HD inline void bfupdate_item(const Pool& P, int p, int e, double dt) {  // Bfupdate :38-58
    int i = e / 324 - 1, j = (e / 18) % 18 - 1, k = e % 18 - 1;
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double *Ex = Ev(P, p, 0), *Ey = Ev(P, p, 1), *Ez = Ev(P, p, 2);
    double dEz_dy = (Ez[ezi(i, j, k)] - Ez[ezi(i, j - 1, k)]) / dy;
    double dEy_dz = (Ey[eyi(i, j, k)] - Ey[eyi(i, j, k - 1)]) / dz;
    Bfv(P, p, 0)[xfc(i, j, k)] += dt * (dEz_dy - dEy_dz);
    double dEz_dx = (Ez[ezi(i, j, k)] - Ez[ezi(i - 1, j, k)]) / dx;
    double dEx_dz = (Ex[exi(i, j, k)] - Ex[exi(i, j, k - 1)]) / dz;
    Bfv(P, p, 1)[yfc(i, j, k)] += dt * (dEx_dz - dEz_dx);
    double dEy_dx = (Ey[eyi(i, j, k)] - Ey[eyi(i - 1, j, k)]) / dx;
    double dEx_dy = (Ex[exi(i, j, k)] - Ex[exi(i, j - 1, k)]) / dy;
    Bfv(P, p, 2)[zfc(i, j, k)] += dt * (dEy_dx - dEx_dy);
}

BH_HD inline double maxdivb_item(const Pool& P, int p, int e) {        // maxdivB :77-89
    int i = e / 324 - 1, j = (e / 18) % 18 - 1, k = e % 18 - 1;
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double *Bx = Bfv(P, p, 0), *By = Bfv(P, p, 1), *Bz = Bfv(P, p, 2);
    double divB = (Bx[xfc(i, j, k)] - Bx[xfc(i - 1, j, k)]) / dx + (By[yfc(i, j, k)] - By[yfc(i, j - 1, k)]) / dy +
                  (Bz[zfc(i, j, k)] - Bz[zfc(i, j, k - 1)]) / dz;
    return fabs(divB);
}

// f2cB (:60-75) for one cell: the face-averaged B and the cell's sqrt(-g)
BH_HD inline void face_avg_B(const Pool& P, int p, int i, int j, int k, double B[3]);
BH_HD inline void f2cb_cell(const KP& kp, const Pool& P, int p, int i, int j, int k, double B[3], double& sg) {
    face_avg_B(P, p, i, j, k, B);
    int l = lindx(i, j, k);
    Met mc;
    met_comp(kp.cell, rr(P, p, l), tt(P, p, l), mc);
    sg = mc.sqrtdetg;
}

BH_HD inline void f2cb_item(const KP& kp, const Pool& P, int p, int e) {
    int i = e / 361 - 1, j = (e / 19) % 19 - 1, k = e % 19 - 1;
    double B[3], sg;
    f2cb_cell(kp, P, p, i, j, k, B, sg);
    int l = lindx(i, j, k);
    for (int d = 0; d < 3; d++) { Wv(P, p, 5 + d)[l] = B[d]; Uv(P, p, 5 + d)[l] = sg * B[d]; }
}

// ---- div_flux + source (integrator.cpp:18-153) -------------------------
BH_HD inline void div_flux(const Pool& P, int p, int i, int j, int k, double sg, double out[8]) {
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    int xr = xfc(i, j, k), xl = xfc(i - 1, j, k);
    int yr = yfc(i, j, k), yl = yfc(i, j - 1, k);
    int zr = zfc(i, j, k), zl = zfc(i, j, k - 1);
    double idx = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz, isg = 1.0 / sg;
#pragma unroll
    for (int v = 0; v < 5; v++) {
        const double *Fx = Fv(P, p, 0, v), *Fy = Fv(P, p, 1, v), *Fz = Fv(P, p, 2, v);
        out[v] = -quo(quo(Fx[xr] - Fx[xl], dx, idx) + quo(Fy[yr] - Fy[yl], dy, idy) + quo(Fz[zr] - Fz[zl], dz, idz),
                      sg, isg);
    }
    out[5] = out[6] = out[7] = 0.0;
}

// geometric source (:41-153) with the cell metric (evaluated in FP64) and
// arithmetic in RT; false where the EOS throws.  The contraction
// src[m] = sum_n sum_q T[n][q] (sum_s g[m][s] Gamma[s][n][q]) runs with
// (n, q) outermost so that each Christoffel symbol is formed once and used
// for all four m; every accumulator still adds its terms in the order
// (n, q) of the reference, so the roundings are the reference's.
template <typename RT>
BH_HD inline bool source(const KP& kp, const MetSrc& mc, const Prim& Wd, RT out[8]) {
    PrimT<RT> W;
    W.rho = RT(Wd.rho); W.eps = RT(Wd.eps);
    for (int d = 0; d < 3; d++) { W.v[d] = RT(Wd.v[d]); W.B[d] = RT(Wd.B[d]); }
    RT gam[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) gam[i][j] = RT(mc.g[i + 1][j + 1]);
    RT v2 = RT(0.0), vlow[3] = {RT(0), RT(0), RT(0)}, Blow[3] = {RT(0), RT(0), RT(0)};
    for (int m = 0; m < 3; m++) {
        for (int n = 0; n < 3; n++) {
            vlow[m] += gam[m][n] * W.v[n];
            Blow[m] += gam[m][n] * W.B[n];
        }
        v2 += vlow[m] * W.v[m];
    }
    v2 = smin(v2, RT(1) - RT(1e-10));
    RT om = RT(1.0) - v2;                 // 1 / ltz2 within an ulp
    RT ltz2 = RT(1.0) / om;
    RT ltz = sqrt(ltz2);
    RT Bv = RT(0.0), Bsq = RT(0.0);
    for (int m = 0; m < 3; m++) { Bv += Blow[m] * W.v[m]; Bsq += Blow[m] * W.B[m]; }
    RT b2 = Bv * Bv + quo(Bsq, ltz2, om);
    bool ok = eos_ok(W.rho);
    RT g = RT(kp.gamma);
    RT px = press(g, W.rho, W.eps);
    RT h = enth(g, W.eps);
    RT alpha = RT(mc.alpha), ialpha = RT(1.0) / alpha, iltz = RT(1.0) / ltz;
    RT u4[4], b4[4];
    u4[0] = quo(ltz, alpha, ialpha);
    for (int m = 0; m < 3; m++) u4[m + 1] = ltz * (W.v[m] - quo(RT(mc.beta[m]), alpha, ialpha));
    b4[0] = quo(ltz * Bv, alpha, ialpha);
    for (int m = 0; m < 3; m++) b4[m + 1] = quo(W.B[m] + alpha * b4[0] * u4[m + 1], ltz, iltz);
    RT T44[4][4];
    RT rhohb2 = W.rho * h + b2;
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) T44[m][n] = rhohb2 * u4[m] * u4[n] + px * RT(mc.gi[m][n]) - b4[m] * b4[n];
    RT acc[4] = {RT(0.0), RT(0.0), RT(0.0), RT(0.0)};
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            RT Gs[4];
#pragma unroll
            for (int s = 0; s < 4; s++) Gs[s] = RT(christoffel(mc, s, n, q));
#pragma unroll
            for (int m = 0; m < 4; m++) {
                RT G_ = RT(0.0);   // lowered Christoffel g[m][s] Gamma[s][n][q], summed over s
#pragma unroll
                for (int s = 0; s < 4; s++) G_ += RT(mc.g[m][s]) * Gs[s];
                acc[m] += T44[n][q] * G_;
            }
        }
    RT src[4];
    for (int m = 0; m < 4; m++) src[m] = acc[m] * RT(mc.sqrtdetg);
    out[0] = RT(0.0);
    out[4] = src[0];
    out[1] = src[1]; out[2] = src[2]; out[3] = src[3];
    out[5] = out[6] = out[7] = RT(0.0);
    return ok;
}

template <typename RT>
BH_HD inline void div_source_item(const KP& kp, const Pool& P, int p, int c, double* dv, double* sv) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int l = lindx(i, j, k);
    MetSrc mf;
    met_src(kp.cell, rr(P, p, l), tt(P, p, l), mf);
    double d8[8];
    RT s8[8];
    div_flux(P, p, i, j, k, mf.sqrtdetg, d8);
    Prim w;
    load_prim(P, p, l, w);
    if (!source(kp, mf, w, s8)) flag(P.err, BH_ERR_DOMAIN);
    for (int v = 0; v < 8; v++) {
        dv[((size_t)p * 8 + v) * NC + l] = d8[v];
        sv[((size_t)p * 8 + v) * NC + l] = s8[v];
    }
}

// f2cB + the conserved update of rkstg (integrator.cpp:325-347), fused.
// Cells in [-1,18)^3 take the face-averaged B; interior cells then add
// dt * (div_flux + source) and refresh U.B = sqrt(-g) W.B.  The two kinds
// of cells are separate items so that a warp holds one kind only:
// update_interior_item for the 16^3 interior cells, update_shell_item for
// the 2763 cells of [-1,18)^3 outside it (f2cB alone).
BH_HD inline void face_avg_B(const Pool& P, int p, int i, int j, int k, double B[3]) {
    const double *Bx = Bfv(P, p, 0), *By = Bfv(P, p, 1), *Bz = Bfv(P, p, 2);
    B[0] = (Bx[xfc(i, j, k)] + Bx[xfc(i - 1, j, k)]) / 2;
    B[1] = (By[yfc(i, j, k)] + By[yfc(i, j - 1, k)]) / 2;
    B[2] = (Bz[zfc(i, j, k)] + Bz[zfc(i, j, k - 1)]) / 2;
}

template <typename RT>
BH_HD inline void update_interior_item(const KP& kp, const Pool& P, int p, int c, double dt, int stage) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int l = lindx(i, j, k);
    double B[3];
    face_avg_B(P, p, i, j, k, B);
    for (int d = 0; d < 3; d++) Wv(P, p, 5 + d)[l] = B[d];
    // the cell metric's sqrt(-g): f2cB's metric::comp and the source's
    // metric share the expression, hence the value
    MetSrc mf;
    met_src(kp.cell, rr(P, p, l), tt(P, p, l), mf);
    double d8[8];
    RT s8[8];
    div_flux(P, p, i, j, k, mf.sqrtdetg, d8);
    Prim w;
    w.rho = Wv(P, p, 0)[l]; w.eps = Wv(P, p, 1)[l];
    for (int d = 0; d < 3; d++) { w.v[d] = Wv(P, p, 2 + d)[l]; w.B[d] = B[d]; }
    if (!source(kp, mf, w, s8)) flag(P.err, BH_ERR_DOMAIN);
    for (int v = 0; v < 5; v++) {
        double dU = d8[v] + double(s8[v]);
        double u = Uv(P, p, v)[l];
        if (stage == 0) {
            dUv(P, p, v)[l] = u;
            Uv(P, p, v)[l] = u + dU * dt;
        } else {
            Uv(P, p, v)[l] = (dUv(P, p, v)[l] + u + dU * dt) * 0.5;
        }
    }
    if (stage == 0)   // c.dU = c.U after f2cB has set U.B = sqrt(-g) W.B
        for (int d = 0; d < 3; d++) dUv(P, p, 5 + d)[l] = mf.sqrtdetg * B[d];
    for (int d = 0; d < 3; d++) Uv(P, p, 5 + d)[l] = mf.sqrtdetg * B[d];
}

constexpr int N_SHELL = N_F2C - N_INT;   // 2763
// shell cell e in [0, N_SHELL): the planes i = -1, 16, 17 (19 x 19 each),
// then j = -1, 16, 17 for i in [0,16) (19 each), then k = -1, 16, 17
BH_HD inline void shell_ijk(int e, int& i, int& j, int& k) {
    if (e < 1083) {
        int ii = e / 361;
        i = ii == 0 ? -1 : 15 + ii; j = (e / 19) % 19 - 1; k = e % 19 - 1;
    } else if (e < 1995) {
        e -= 1083;
        int jj = (e / 19) % 3;
        i = e / 57; j = jj == 0 ? -1 : 15 + jj; k = e % 19 - 1;
    } else {
        e -= 1995;
        int kk = e % 3;
        i = e / 48; j = (e / 3) % 16; k = kk == 0 ? -1 : 15 + kk;
    }
}

BH_HD inline void update_shell_item(const KP& kp, const Pool& P, int p, int e) {
    int i, j, k;
    shell_ijk(e, i, j, k);
    double B[3], sg;
    f2cb_cell(kp, P, p, i, j, k, B, sg);
    int l = lindx(i, j, k);
    for (int d = 0; d < 3; d++) { Wv(P, p, 5 + d)[l] = B[d]; Uv(P, p, 5 + d)[l] = sg * B[d]; }
}

// ---- ghost fill: amrtree::ghosts (grid.cpp:390-571) ---------------------
// strip cell e of patch p: face slot s = dim*2 + (side>0), layer gg,
// transverse t1, t2 in [0,16) (edges and corners are never filled, :418)
BH_HD inline void strip_ijk(int dim, int pos, int t1, int t2, int& i, int& j, int& k) {
    if (dim == 0) { i = pos; j = t1; k = t2; }
    else if (dim == 1) { i = t1; j = pos; k = t2; }
    else { i = t1; j = t2; k = pos; }
}

// ghost-strip copy (gh_copy :390-425, gh_bndy :494-522) of two cells' state
// vectors: item e of patch p copies U (a = 0) or W (a = 1), a = e / N_COPY,
// of the strip-cell pair e % N_COPY.  A pair is two cells adjacent in k --
// the same row for the x- and y-strips, the two layers of a k-strip -- so
// the eight variables move as eight aligned 16-byte loads and stores (the
// per-patch linear index of an even k is even, grid.cpp:51-53).  Pairs are
// ordered so that neighbouring items are neighbours in memory.  The 128
// items of a CTA share one array and one slot, so the neighbour kind is
// uniform.
constexpr int N_COPY = N_STRIP / 2;
BH_HD inline void ghost_copy_item(const Pool& P, int p, int e) {
    int a = e / N_COPY, c = e % N_COPY;
    int s = c / 256, rem = c % 256;
    int dim = s / 2, side = (s & 1) ? 1 : -1;
    int nb = P.nbr[(p * 6 + s) * 2], kind = P.nbr[(p * 6 + s) * 2 + 1];
    if (kind != BH_NB_COPY && kind != BH_NB_BNDY) return;
    // the first cell of the pair: ghost (gi, gj, gk), source (ai, aj, ak);
    // the second is k + 1 in both, except an outflow k-strip on the +k side,
    // whose layers mirror the interior (ghost 16, 17 <- 15, 14)
    int gi, gj, gk, ai, aj, ak, src_p, row_end = 0;
    bool swap = false;
    if (dim == 2) {
        int t1 = rem >> 4, t2 = rem & 15;
        strip_ijk(2, side == 1 ? BLK : -GH, t1, t2, gi, gj, gk);
        if (kind == BH_NB_COPY) {
            src_p = nb;
            strip_ijk(2, side == 1 ? 0 : BLK - GH, t1, t2, ai, aj, ak);
        } else {
            src_p = p;
            strip_ijk(2, side == 1 ? BLK - 2 : 0, t1, t2, ai, aj, ak);
            swap = side == 1;
        }
    } else {
        int gg = rem >> 7, t1 = (rem >> 3) & 15, t2 = (rem & 7) * 2;
        row_end = t2 == 0 ? -1 : (t2 == BLK - 2 ? 1 : 0);
        strip_ijk(dim, (side == 1 ? BLK : -GH) + gg, t1, t2, gi, gj, gk);
        if (kind == BH_NB_COPY) {
            src_p = nb;
            strip_ijk(dim, (side == 1 ? 0 : BLK - GH) + gg, t1, t2, ai, aj, ak);
        } else {
            src_p = p;
            strip_ijk(dim, side == 1 ? BLK - 1 - gg : gg, t1, t2, ai, aj, ak);
        }
    }
    double* dst = a == 0 ? Uv(P, p, 0) : Wv(P, p, 0);
    const double* src = a == 0 ? Uv(P, src_p, 0) : Wv(P, src_p, 0);
    int lg = lindx(gi, gj, gk), la = lindx(ai, aj, ak);
    double2 x[8];
#pragma unroll
    for (int v = 0; v < 8; v++) x[v] = *reinterpret_cast<const double2*>(src + (size_t)v * NC + la);
    if (row_end != 0) {
        // The first and last pair of an x- or y-strip row share their
        // 32-byte sector with the row's two cells beyond the strip (k = -2,
        // -1 or 16, 17: edge cells, which no strip fills): written back with
        // the pair, every store of the row is a whole sector.
        const int edge = row_end < 0 ? lg - 2 : lg + 2;
        double2 own[8];
#pragma unroll
        for (int v = 0; v < 8; v++) own[v] = *reinterpret_cast<const double2*>(dst + (size_t)v * NC + edge);
#pragma unroll
        for (int v = 0; v < 8; v++) {
            double2* row = reinterpret_cast<double2*>(dst + (size_t)v * NC + (row_end < 0 ? edge : lg));
            row[0] = row_end < 0 ? own[v] : x[v];
            row[1] = row_end < 0 ? x[v] : own[v];
        }
        return;
    }
    if (dim == 2) {
        // A k-strip pair is half of a 32-byte sector (rows of CPN = 20
        // doubles start on sector boundaries); the other half is the row's
        // own two interior cells next to it, which this kernel never changes.
        // Writing them back with the pair makes every store a whole sector
        // (no partial-sector read-modify-write below L2).
        const int lo = side == 1 ? lg - 2 : lg + 2;   // the interior pair of the sector
        double2 own[8];
#pragma unroll
        for (int v = 0; v < 8; v++) own[v] = *reinterpret_cast<const double2*>(dst + (size_t)v * NC + lo);
#pragma unroll
        for (int v = 0; v < 8; v++) {
            double2 y = swap ? make_double2(x[v].y, x[v].x) : x[v];
            double2* row = reinterpret_cast<double2*>(dst + (size_t)v * NC + (side == 1 ? lo : lg));
            row[0] = side == 1 ? own[v] : y;
            row[1] = side == 1 ? y : own[v];
        }
        return;
    }
#pragma unroll
    for (int v = 0; v < 8; v++) {
        double2 y = swap ? make_double2(x[v].y, x[v].x) : x[v];
        *reinterpret_cast<double2*>(dst + (size_t)v * NC + lg) = y;
    }
}

// ghost-strip prolongation from a coarser neighbour, strip cell e of patch p
// in [0, N_STRIP) (cells of other neighbour kinds are left to ghost_copy_item)
BH_HD inline void ghost_prolong_item(const KP& kp, const Pool& P, int p, int e) {
    int s = e / 512, rem = e % 512;
    int nb = P.nbr[(p * 6 + s) * 2], kind = P.nbr[(p * 6 + s) * 2 + 1];
    if (kind != BH_NB_PROLONG) return;
    int gg = rem / 256, t1 = (rem / 16) % 16, t2 = rem % 16;
    int dim = s / 2, side = (s & 1) ? 1 : -1;
    int gi, gj, gk;
    strip_ijk(dim, (side == 1 ? BLK : -GH) + gg, t1, t2, gi, gj, gk);
    int lg = lindx(gi, gj, gk);
    // gh_prolong (:427-492): minmod-limited interpolation from the coarse patch
    int ci = (dim == 0) ? gg / 2 : t1 / 2;
    int cj = (dim == 1) ? gg / 2 : (dim == 0 ? t1 / 2 : t2 / 2);
    int ck = (dim == 2) ? gg / 2 : t2 / 2;
    double offg = (gg % 2 == 0) ? -0.25 : 0.25;
    double offt1 = (t1 % 2 == 0) ? -0.25 : 0.25;
    double offt2 = (t2 % 2 == 0) ? -0.25 : 0.25;
    double on, ot1, ot2;
    if (dim == 0) { on = offg; ot1 = offt1; ot2 = offt2; }
    else if (dim == 1) { on = offt1; ot1 = offg; ot2 = offt2; }
    else { on = offt1; ot1 = offt2; ot2 = offg; }
    int lc = lindx(ci, cj, ck);
    int lxm = lindx(ci - 1, cj, ck), lxp = lindx(ci + 1, cj, ck);
    int lym = lindx(ci, cj - 1, ck), lyp = lindx(ci, cj + 1, ck);
    int lzm = lindx(ci, cj, ck - 1), lzp = lindx(ci, cj, ck + 1);
    double u8[8];
    for (int v = 0; v < 8; v++) {
        const double* c = Uv(P, nb, v);
        double vc = c[lc];
        double sn = minmod(vc - c[lxm], c[lxp] - vc);
        double st1 = minmod(vc - c[lym], c[lyp] - vc);
        double st2 = minmod(vc - c[lzm], c[lzp] - vc);
        u8[v] = vc + sn * on + st1 * ot1 + st2 * ot2;
    }
    Cons u;
    u.D = u8[0]; u.tau = u8[4];
    for (int d = 0; d < 3; d++) { u.S[d] = u8[1 + d]; u.B[d] = u8[5 + d]; }
    Prim w;
    load_prim(P, p, lg, w);
    bool dirty = false;
    recover_cell(kp, P, p, lg, w, u, dirty);
    store_cons(P, p, lg, u);
    store_prim(P, p, lg, w);
}

// ghost ctop of amrtree::ghosts for one cell of a patch of one wave
BH_HD inline void ghost_ctop_item(const KP& kp, const Pool& P, int p, int l) {
    int i, j, k;
    lin_ijk(l, i, j, k);
    if (!is_ghost(i, j, k)) return;
    Prim w; Cons u;
    load_prim(P, p, l, w);
    load_cons(P, p, l, u);
    bool dirty = false;
    ghost_recover(kp, P, p, l, w, u, dirty);
    store_prim(P, p, l, w);
    if (dirty) store_cons(P, p, l, u);
}

// reconstruction loop of rkstg (integrator.cpp:288-310) for one cell of a
// leaf patch.  With ghost_first, ghost cells first take amrtree::ghosts'
// ctop (grid.cpp:538-570); a second ctop on an unchanged U reproduces the
// first, so it only runs after a fallback changed U.  One ctop call site
// serves both passes, so ghost and interior cells of a warp do not diverge.
BH_HD inline void prims_item(const KP& kp, const Pool& P, int p, int l, int ghost_first) {
    int i, j, k;
    lin_ijk(l, i, j, k);
    Cons u;
    load_cons(P, p, l, u);
    bool g = ghost_first && is_ghost(i, j, k);
    Prim w;
    if (g) {
        load_prim(P, p, l, w);
    } else {
        w.rho = w.eps = 0.0;
        w.v[0] = w.v[1] = w.v[2] = 0.0;
        for (int d = 0; d < 3; d++) w.B[d] = Wv(P, p, 5 + d)[l];
    }
    double r = rr(P, p, l), th = tt(P, p, l);
    Met mc;
    met_comp(kp.tree, r, th, mc);
    bool dirty = false;
    for (int pass = g ? 0 : 1; pass < 2; pass++) {
        Prim pv;
        bool dom = false;
        int ok = ctop(kp.gamma, kp.maxiter, kp.tol, mc, u, pv, dom);
        if (dom) flag(P.err, BH_ERR_DOMAIN);
        if (ok) { w = pv; break; }
        // pass 0 (ghosts): floor rho, eps, keep v and B; pass 1 (rkstg):
        // floor state with the cell's B; then U = ptoc(W) either way
        pvfs(r, w.rho, w.eps);
        if (pass == 1) w.v[0] = w.v[1] = w.v[2] = 0.0;
        if (!ptoc(kp.gamma, mc, w, u)) flag(P.err, BH_ERR_DOMAIN);
        dirty = true;
    }
    store_prim(P, p, l, w);
    if (dirty) store_cons(P, p, l, u);
}

// ---- reconstruction with reuse of interior outcomes ----------------------
// interior cell c of a leaf patch: rkstg's ctop and fallback; records the
// outcome (1 recovered, 0 floored) in the status scratch
BH_HD inline void prims_interior_item(const KP& kp, const Pool& P, int p, int c) {
    int l = lindx(c / 256, (c / 16) % 16, c % 16);
    Cons u;
    load_cons(P, p, l, u);
    Prim w;
    w.rho = w.eps = 0.0;
    w.v[0] = w.v[1] = w.v[2] = 0.0;
    for (int d = 0; d < 3; d++) w.B[d] = Wv(P, p, 5 + d)[l];
    bool dirty = false;
    recover_cell(kp, P, p, l, w, u, dirty);
    store_prim(P, p, l, w);
    if (dirty) store_cons(P, p, l, u);
    P.status[(size_t)p * NC + l] = dirty ? 0 : 1;
}

// the two con2prim passes of a ghost cell: amrtree::ghosts' ctop with its
// fallback, then (only if that changed U) rkstg's ctop with its fallback.
// first_fails: the first ctop is known to fail (it already failed on the
// same U at the same position), so the cell starts at its fallback.
BH_HD inline void ghost_two_pass(const KP& kp, const Pool& P, int p, int l, bool first_fails = false) {
    Cons u;
    load_cons(P, p, l, u);
    Prim w;
    load_prim(P, p, l, w);
    double r = rr(P, p, l), th = tt(P, p, l);
    Met mc;
    met_comp(kp.tree, r, th, mc);
    bool dirty = false;
    for (int pass = 0; pass < 2; pass++) {
        Prim pv;
        bool dom = false;
        int ok = (pass == 0 && first_fails) ? 0 : ctop(kp.gamma, kp.maxiter, kp.tol, mc, u, pv, dom);
        if (dom) flag(P.err, BH_ERR_DOMAIN);
        if (ok) { w = pv; break; }
        pvfs(r, w.rho, w.eps);
        if (pass == 1) w.v[0] = w.v[1] = w.v[2] = 0.0;
        if (!ptoc(kp.gamma, mc, w, u)) flag(P.err, BH_ERR_DOMAIN);
        dirty = true;
    }
    store_prim(P, p, l, w);
    if (dirty) store_cons(P, p, l, u);
}

// ghost cell e of a leaf patch after the interior pass: items [0, 3072)
// are the face strips in the order of ghost_fill_item, items [3072, 3904)
// the edge and corner cells
BH_HD inline void prims_ghost_item(const KP& kp, const Pool& P, int p, int e) {
    if (e >= N_STRIP) {
        ghost_two_pass(kp, P, p, BH_EDGE_CELLS.l[e - N_STRIP]);
        return;
    }
    int s = e / 512, rem = e % 512;
    int gg = rem / 256, t1 = (rem / 16) % 16, t2 = rem % 16;
    int dim = s / 2, side = (s & 1) ? 1 : -1;
    int nb = P.nbr[(p * 6 + s) * 2], kind = P.nbr[(p * 6 + s) * 2 + 1];
    int gi, gj, gk;
    strip_ijk(dim, (side == 1 ? BLK : -GH) + gg, t1, t2, gi, gj, gk);
    int lg = lindx(gi, gj, gk);
    if (kind == BH_NB_COPY || kind == BH_NB_BNDY) {
        int src_p = kind == BH_NB_COPY ? nb : p;
        int ai, aj, ak;
        if (kind == BH_NB_COPY) strip_ijk(dim, (side == 1 ? 0 : BLK - GH) + gg, t1, t2, ai, aj, ak);
        else strip_ijk(dim, side == 1 ? BLK - 1 - gg : gg, t1, t2, ai, aj, ak);
        int la = lindx(ai, aj, ak);
        // same U and the same (r, theta) bit for bit as the source (not so
        // across a periodic wrap or an outflow copy, where the ghost sits
        // elsewhere): ctop is a function of U and the position, so the
        // ghost's first ctop has the source's outcome.  Success: the same
        // primitives.  Failure: the ghost goes straight to its fallback.
        if (P.leafmask[src_p] && rr(P, p, lg) == rr(P, src_p, la) && tt(P, p, lg) == tt(P, src_p, la)) {
            uint8_t st = P.status[(size_t)src_p * NC + la];
            if (st == 1) {
                for (int v = 0; v < 8; v++) Wv(P, p, v)[lg] = Wv(P, src_p, v)[la];
                return;
            }
            if (st == 0) {
                ghost_two_pass(kp, P, p, lg, true);
                return;
            }
        }
    }
    ghost_two_pass(kp, P, p, lg);
}

// ---- floors: patch::floors (grid.cpp:331-358) ---------------------------
BH_HD inline void floors_item(const KP& kp, const Pool& P, int p, int c) {
    int l = lindx(c / 256, (c / 16) % 16, c % 16);
    Cons u;
    load_cons(P, p, l, u);
    double r = rr(P, p, l), th = tt(P, p, l);
    bool bhl = !isfinite(u.D) || !isfinite(u.tau) || u.D <= 0.0 || u.tau <= 0.0;
    Prim w;
    load_prim(P, p, l, w);
    bool wrote = false;
    double d4[4];           // derived fields of the primitives written (pool->Wd)
    if (!bhl) {
        Met mc;
        met_comp(kp.tree, r, th, mc);
        Prim pv;
        bool dom = false;
        CtopOut co;
        int ok = ctop(kp.gamma, kp.maxiter, kp.tol, mc, u, pv, dom, P.Wd ? &co : nullptr);
        if (dom) flag(P.err, BH_ERR_DOMAIN);
        bhl = !ok;
        if (!bhl && !(pv.rho <= 0.0 || pv.eps <= 0.0)) {
            w = pv; wrote = true;
            d4[0] = co.lor; d4[1] = co.p; d4[2] = co.h; d4[3] = co.b2;
        }
    }
    double frho, feps;
    pvfs(r, frho, feps);
    if (bhl || w.rho <= frho) {
        PtocOut po;
        floor_reset(kp, P, p, l, w, u, P.Wd ? &po : nullptr);
        store_cons(P, p, l, u);
        wrote = true;
        d4[0] = po.lor; d4[1] = po.p; d4[2] = po.h; d4[3] = po.b2;
    }
    if (wrote) {
        store_prim(P, p, l, w);
        if (P.Wd) store_derived(P, p, l, d4[0], d4[1], d4[2], d4[3]);
    }
}

// ---- AMR regrid (grid.cpp:573-835) ---------------------------------------
// One interior cell of amrtree::regrid's refinement test (:771-818): ref =
// the cell asks for refinement, noflat = it forbids flattening its patch.
constexpr int REGRID_MAX_LVL = 4;
BH_HD inline void regrid_cell(const Pool& P, int p, int lvl, int c, bool& ref, bool& noflat) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int l = lindx(i, j, k);
    if (rr(P, p, l) < 3.0 && lvl < REGRID_MAX_LVL) { ref = true; noflat = true; return; }
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double* rho = Wv(P, p, 0);
    double chro = rho[l];
    if (chro > 0.0) {
        double drho_dx = fabs(rho[lindx(i + 1, j, k)] - rho[lindx(i - 1, j, k)]) / (2 * dx);
        double drho_dy = fabs(rho[lindx(i, j + 1, k)] - rho[lindx(i, j - 1, k)]) / (2 * dy);
        double drho_dz = fabs(rho[lindx(i, j, k + 1)] - rho[lindx(i, j, k - 1)]) / (2 * dz);
        double drho = sqrt(drho_dx * drho_dx + drho_dy * drho_dy + drho_dz * drho_dz);
        double rgrh = drho * dx / chro;
        if (rgrh > 0.5 && lvl < REGRID_MAX_LVL) { ref = true; noflat = true; }
        if (rgrh > 0.1) noflat = true;
    }
    const double *B0 = Wv(P, p, 5), *B1 = Wv(P, p, 6), *B2 = Wv(P, p, 7);
    double Bmag = sqrt(B0[l] * B0[l] + B1[l] * B1[l] + B2[l] * B2[l]);
    if (Bmag > 1e-14) {
        double dB_dx = fabs(B0[lindx(i + 1, j, k)] - B0[lindx(i - 1, j, k)]) / (2 * dx);
        double dB_dy = fabs(B1[lindx(i, j + 1, k)] - B1[lindx(i, j - 1, k)]) / (2 * dy);
        double dB_dz = fabs(B2[lindx(i, j, k + 1)] - B2[lindx(i, j, k - 1)]) / (2 * dz);
        double rdB = (dB_dx * dx + dB_dy * dy + dB_dz * dz) / Bmag;
        if (rdB > 0.5 && lvl < REGRID_MAX_LVL) { ref = true; noflat = true; }
    }
}
// the patch's flags from the OR of its cells: bit 0 patch->refine, bit 1 patch->erase
BH_HD inline uint8_t regrid_patch_flags(int lvl, bool anyref, bool anynoflat) {
    return (uint8_t)(((anyref && lvl < REGRID_MAX_LVL) ? 1 : 0) | ((!anynoflat && lvl > 0) ? 2 : 0));
}

// patch::B_init (grid.cpp:207-250), face e of 3 x 8400: face B from the
// cells' W.B.  The z-face branch tests i (not k) against -ghost; its cell
// indices k = -3 and k = 18 are taken as the reference's linear index
// computes them, i.e. neighbouring cells in memory order (all within the
// patch's 8000 cells).
BH_HD inline void b_init_item(const Pool& P, int p, int e) {
    int d = e / NF, f = e % NF;
    const double* Bc = Wv(P, p, 5 + d);
    double v;
    if (d == 0) {
        int i = f / (CPN * CPN) - GH, j = (f / CPN) % CPN - GH, k = f % CPN - GH;
        if (i > -GH && i < BLK + GH) v = (Bc[lindx(i - 1, j, k)] + Bc[lindx(i, j, k)]) / 2;
        else if (i == -GH) v = Bc[lindx(i, j, k)];
        else v = Bc[lindx(i - 1, j, k)];
    } else if (d == 1) {
        int i = f / ((CPN + 1) * CPN) - GH, j = (f / CPN) % (CPN + 1) - GH, k = f % CPN - GH;
        if (j > -GH && j < BLK + GH) v = (Bc[lindx(i, j - 1, k)] + Bc[lindx(i, j, k)]) / 2;
        else if (j == -GH) v = Bc[lindx(i, j, k)];
        else v = Bc[lindx(i, j - 1, k)];
    } else {
        int i = f / (CPN * (CPN + 1)) - GH, j = (f / (CPN + 1)) % CPN - GH, k = f % (CPN + 1) - GH;
        if (k > -GH && k < BLK + GH) v = (Bc[lindx(i, j, k - 1)] + Bc[lindx(i, j, k)]) / 2;
        else if (i == -GH) v = Bc[lindx(i, j, k)];
        else v = Bc[lindx(i, j, k - 1)];
    }
    Bfv(P, p, d)[f] = v;
}

// the cell data of amrtree::refine (:603-648) for interior cell c of child h
// (patch `child`) of patch `parent`: a minmod-limited interpolation of the
// parent's conserved variables, then ctop with its fallback (W = pvfs with
// v = 0 and the cell's current B, zero in a new child; U = ptoc(W)).  The
// reference's prolong lambda is declared (vc, vmx, vpx, ...) but called
// with the +x neighbour first, so each slope is minmod(vc - v[+1], v[-1] - vc).
BH_HD inline void refine_item(const KP& kp, const Pool& P, int parent, int child, int h, int c) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int ix = (h >> 2) & 1, iy = (h >> 1) & 1, iz = h & 1;
    int pi = (i + ix * BLK) / 2, pj = (j + iy * BLK) / 2, pk = (k + iz * BLK) / 2;
    double ox = (i % 2 == 0) ? -0.25 : 0.25;
    double oy = (j % 2 == 0) ? -0.25 : 0.25;
    double oz = (k % 2 == 0) ? -0.25 : 0.25;
    int lc = lindx(pi, pj, pk);
    int lpx = lindx(pi + 1, pj, pk), lmx = lindx(pi - 1, pj, pk);
    int lpy = lindx(pi, pj + 1, pk), lmy = lindx(pi, pj - 1, pk);
    int lpz = lindx(pi, pj, pk + 1), lmz = lindx(pi, pj, pk - 1);
    double u8[8];
    for (int v = 0; v < 8; v++) {
        const double* u = Uv(P, parent, v);
        double vc = u[lc];
        double sx = minmod(vc - u[lpx], u[lmx] - vc);
        double sy = minmod(vc - u[lpy], u[lmy] - vc);
        double sz = minmod(vc - u[lpz], u[lmz] - vc);
        u8[v] = vc + sx * ox + sy * oy + sz * oz;
    }
    Cons cu;
    cu.D = u8[0]; cu.tau = u8[4];
    for (int d = 0; d < 3; d++) { cu.S[d] = u8[1 + d]; cu.B[d] = u8[5 + d]; }
    int lf = lindx(i, j, k);
    Prim w;
    load_prim(P, child, lf, w);
    recover_keep_derived(kp, P, child, lf, w, cu);
    store_cons(P, child, lf, cu);
    store_prim(P, child, lf, w);
}

// amrtree::ccrstr (:651-712) for interior cell c of `parent`: the
// volume-weighted mean of the eight cells of its octant child (cons() +
// vol * U, in the child-cell order di, dj, dk; the reference also visits
// the other children, none of whose cells lies in range), then ctop with
// the fallback keeping the parent cell's B
BH_HD inline void ccrstr_item(const KP& kp, const Pool& P, int parent, const int32_t* kids, int c) {
    int pi = c / 256, pj = (c / 16) % 16, pk = c % 16;
    int ix = pi >= BLK / 2, iy = pj >= BLK / 2, iz = pk >= BLK / 2;
    int ch = kids[ix * 4 + iy * 2 + iz];
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double volt = 0.0;
    if (ch >= 0) {
        const double* g = P.pgeo + 6 * ch;
        double vol = g[3] * g[4] * g[5];
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++) {
                    int lf = lindx(2 * (pi - ix * (BLK / 2)) + di, 2 * (pj - iy * (BLK / 2)) + dj,
                                   2 * (pk - iz * (BLK / 2)) + dk);
                    volt += vol;
                    for (int v = 0; v < 8; v++) acc[v] += vol * Uv(P, ch, v)[lf];
                }
    }
    if (volt > 0.0) {
        double inv = 1.0 / volt;
        for (int v = 0; v < 8; v++) acc[v] *= inv;
    }
    Cons cu;
    cu.D = acc[0]; cu.tau = acc[4];
    for (int d = 0; d < 3; d++) { cu.S[d] = acc[1 + d]; cu.B[d] = acc[5 + d]; }
    int l = lindx(pi, pj, pk);
    Prim w;
    load_prim(P, parent, l, w);
    recover_keep_derived(kp, P, parent, l, w, cu);
    store_cons(P, parent, l, cu);
    store_prim(P, parent, l, w);
}

// ---- analysis::analyser (data/quantitatives.cpp:17-199) -------------------
// The integrands of the diagnostics at interior cell c of leaf patch p,
// times the cell volume, added to acc[BH_NQ]; surface integrals take the
// cells within one cell diagonal of their radius (surf_int, :61-79).  The
// cell's metric (the cell metric, cell.hpp:25) gives sqrt(-g), lapse, shift,
// g_0mu and gamma_i2.
struct AParams { double hrz, rs, rho_min_full, rho_min_bundle; };
BH_HD inline void analysis_cell(const KP& kp, const Pool& P, int p, int c, const AParams& A, double acc[BH_NQ]) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int l = lindx(i, j, k);
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    double xc = g[0] + (i + 0.5) * g[3], yc = g[1] + (j + 0.5) * g[4], zc = g[2] + (k + 0.5) * g[5];
    double vol = dx * dy * dz;
    double r = rr(P, p, l), th = tt(P, p, l);
    Prim w;
    load_prim(P, p, l, w);
    const double* d = P.Wd + (size_t)p * 4 * NC;
    double lor = d[l], pr = d[NC + l], h = d[2 * NC + l], b2 = d[3 * NC + l];
    double D = Uv(P, p, 0)[l], tau = Uv(P, p, 4)[l], S0 = Uv(P, p, 1)[l], S1 = Uv(P, p, 2)[l];
    MetSrc m;
    met_src(kp.cell, r, th, m);
    double sg = m.sqrtdetg;
    double R = sqrt(xc * xc + yc * yc);
    double vr = (xc * w.v[0] + yc * w.v[1] + zc * w.v[2]) / r;                    // val_vr :24-26
    double vphi = (R < 1e-10) ? 0.0 : (xc * w.v[1] - yc * w.v[0]) / (R * R);     // val_vphi :27-31
    double Br = (xc * w.B[0] + yc * w.B[1] + zc * w.B[2]) / r;                    // val_Br :33-35
    double Bphi = (R < 1e-10) ? 0.0 : (xc * w.B[1] - yc * w.B[0]) / (R * R);     // val_Bphi :36-40
    double shell = sqrt(dx * dx + dy * dy + dz * dz);
    bool on_h = !(fabs(r - A.hrz) > shell), on_s = !(fabs(r - A.rs) > shell);
    acc[BH_Q_MASS] += D * vol;
    acc[BH_Q_ENERGY] += (tau + D) * vol;
    acc[BH_Q_LPOL] += (xc * S1 - yc * S0) * vol;
    if (on_h) {
        acc[BH_Q_MDOT] += (-w.rho * lor * vr * sg) * vol;
        acc[BH_Q_EDOT] += (-((tau + D) * (m.alpha * vr - (m.beta[0] * xc + m.beta[1] * yc + m.beta[2] * zc) / r))) * vol;
        double wh = w.rho * h + b2;
        acc[BH_Q_LDOT] += ((wh * lor * lor * vr * vphi - Br - Bphi) * sg) * vol;
        acc[BH_Q_PHIB] += (fabs(Br) * sg) * vol;
        // L_BZ (:135-155): Blow[i] is assigned inside the j loop, so gamma_i2 B_2 survives
        double Blow[3] = {m.g[1][3] * w.B[2], m.g[2][3] * w.B[2], m.g[3][3] * w.B[2]};
        double Bv = 0.0;
        for (int a = 0; a < 3; a++) Bv += Blow[a] * w.v[a];
        double bt = lor * Bv / m.alpha;
        double br = (Br + m.alpha * bt * lor * vr) / lor;
        double bt_ = m.g[0][0] * bt + m.g[0][1] * br + m.g[0][3] * (Bphi * lor);
        double ur = lor * vr;
        double ut_ = -m.alpha * lor;
        acc[BH_Q_LBZ] += (-(b2 * ur * ut_ - br * bt_) * sg) * vol;
    }
    acc[BH_Q_MAGE] += (0.5 * b2 * sg) * vol;
    acc[BH_Q_THERME] += (w.rho * w.eps * sg) * vol;
    acc[BH_Q_PNUM] += (pr * sg) * vol;
    acc[BH_Q_PDEN] += (0.5 * b2 * sg) * vol;
    double stress = (w.rho * h * vr * vphi - Br * Bphi) * sg;
    double ptot = (pr + 0.5 * b2) * sg;
    acc[BH_Q_ASTRESS] += (w.rho < A.rho_min_full ? 0.0 : stress) * vol;
    acc[BH_Q_APRESS] += (w.rho < A.rho_min_full ? 0.0 : ptot) * vol;
    acc[BH_Q_ASTRESS_B] += (w.rho < A.rho_min_bundle ? 0.0 : stress) * vol;
    acc[BH_Q_APRESS_B] += (w.rho < A.rho_min_bundle ? 0.0 : ptot) * vol;
    acc[BH_Q_MAXW] += (w.rho < A.rho_min_full ? 0.0 : -Br * Bphi * sg) * vol;
    acc[BH_Q_REYN] += (w.rho < A.rho_min_full ? 0.0 : w.rho * h * lor * lor * vr * vphi * sg) * vol;
    if (on_s) {
        acc[BH_Q_HNUM] += (fabs(zc) * w.rho * sg) * vol;
        acc[BH_Q_HDEN] += (w.rho * sg) * vol;
    }
}

// ---- dtcomp (integrator.cpp:156-189): one cell's CFL candidate -----------
constexpr double DBL_BIG = 1.7976931348623157e308;   // std::numeric_limits<double>::max()
BH_HD inline double dt_item(const KP& kp, const Pool& P, int p, int c, double cfl) {
    double best = DBL_BIG;
    int l = lindx(c / 256, (c / 16) % 16, c % 16);
    double rho = Wv(P, p, 0)[l], eps = Wv(P, p, 1)[l];
    if (!eos_ok(rho)) flag(P.err, BH_ERR_DOMAIN);
    double cs = sqrt(cs2f(kp.gamma, rho, eps));
    Met mc;
    met_comp(kp.cell, rr(P, p, l), tt(P, p, l), mc);
    const double* g = P.pgeo + 6 * p;
    for (int d = 0; d < 3; d++) {
        double v = Wv(P, p, 2 + d)[l];
        double ld_p = fabs(mc.alpha * (v + cs) - mc.beta[d]);
        double ld_m = fabs(mc.alpha * (v - cs) - mc.beta[d]);
        double vmax = smax(ld_p, ld_m);
        if (vmax > 1e-14) best = smin(best, cfl * g[3 + d] / vmax);
    }
    return best;
}

// ---- batched physics items ----------------------------------------------
BH_HD inline void metric_item(const KP& k, const double* r, const double* th, int64_t q, double* out) {
    MetFull f;
    met_full(k.tree, r[q], th[q], f);
    Met m;
    met_comp(k.tree, r[q], th[q], m);
    double* o = out + q * 120;
    // struct metriccomp member order (metric.hpp:11-21)
    for (int i = 0; i < 16; i++) o[i] = f.g[i / 4][i % 4];
    for (int i = 0; i < 16; i++) o[16 + i] = f.gi[i / 4][i % 4];
    for (int i = 0; i < 64; i++) o[32 + i] = f.G[i / 16][(i / 4) % 4][i % 4];
    o[96] = m.sqrtdetg;
    for (int i = 0; i < 9; i++) o[97 + i] = m.gam[i / 3][i % 3];
    for (int i = 0; i < 9; i++) o[106 + i] = m.gam_inv[i / 3][i % 3];
    o[115] = m.sqrtdetgam;
    o[116] = m.alpha;
    for (int i = 0; i < 3; i++) o[117 + i] = m.beta[i];
}

BH_HD inline void ptoc_item(const KP& k, const double* W, const double* r, const double* th, int64_t n, int64_t q,
                            double* U, double* Wd, int32_t* err) {
    Prim w;
    w.rho = W[q]; w.eps = W[n + q];
    for (int d = 0; d < 3; d++) { w.v[d] = W[(2 + d) * n + q]; w.B[d] = W[(5 + d) * n + q]; }
    Met mc;
    met_comp(k.tree, r[q], th[q], mc);
    Cons c;
    PtocOut po;
    if (!ptoc(k.gamma, mc, w, c, &po)) flag(err, BH_ERR_DOMAIN);
    U[q] = c.D; U[4 * n + q] = c.tau;
    for (int d = 0; d < 3; d++) { U[(1 + d) * n + q] = c.S[d]; U[(5 + d) * n + q] = c.B[d]; }
    if (Wd) { Wd[q] = po.lor; Wd[n + q] = po.p; Wd[2 * n + q] = po.h; Wd[3 * n + q] = po.b2; }
}

BH_HD inline void ctop_item(const KP& k, const double* U, const double* r, const double* th, int64_t n, int64_t q,
                            double* W, double* Wd, int32_t* status, int32_t* iters, int32_t* path) {
    Cons c;
    c.D = U[q]; c.tau = U[4 * n + q];
    for (int d = 0; d < 3; d++) { c.S[d] = U[(1 + d) * n + q]; c.B[d] = U[(5 + d) * n + q]; }
    Met mc;
    met_comp(k.tree, r[q], th[q], mc);
    Prim w = {0, 0, {0, 0, 0}, {0, 0, 0}};
    CtopOut co = {0, 0, 0, 0, 0, 0, 0};
    bool dom = false;
    int ok = ctop(k.gamma, k.maxiter, k.tol, mc, c, w, dom, &co);
    W[q] = w.rho; W[n + q] = w.eps;
    for (int d = 0; d < 3; d++) { W[(2 + d) * n + q] = w.v[d]; W[(5 + d) * n + q] = w.B[d]; }
    if (Wd) { Wd[q] = co.p; Wd[n + q] = co.T; Wd[2 * n + q] = co.h; Wd[3 * n + q] = co.lor; Wd[4 * n + q] = co.b2; }
    status[q] = dom ? -1 : ok;
    if (iters) iters[q] = co.iters;
    if (path) path[q] = co.path;
}

// ctop with Newton started from xi0[q] (bh_ctop_guess); the outputs of ctop_item
BH_HD inline void ctop_guess_item(const KP& k, const double* U, const double* r, const double* th, int64_t n,
                                  int64_t q, const double* xi0, double* W, double* Wd, int32_t* status, int32_t* iters,
                                  int32_t* path) {
    Cons c;
    c.D = U[q]; c.tau = U[4 * n + q];
    for (int d = 0; d < 3; d++) { c.S[d] = U[(1 + d) * n + q]; c.B[d] = U[(5 + d) * n + q]; }
    Met mc;
    met_comp(k.tree, r[q], th[q], mc);
    Prim w = {0, 0, {0, 0, 0}, {0, 0, 0}};
    CtopOut co = {0, 0, 0, 0, 0, 0, 0};
    bool dom = false;
    int ok = ctop(k.gamma, k.maxiter, k.tol, mc, c, w, dom, &co, xi0[q]);
    W[q] = w.rho; W[n + q] = w.eps;
    for (int d = 0; d < 3; d++) { W[(2 + d) * n + q] = w.v[d]; W[(5 + d) * n + q] = w.B[d]; }
    if (Wd) { Wd[q] = co.p; Wd[n + q] = co.T; Wd[2 * n + q] = co.h; Wd[3 * n + q] = co.lor; Wd[4 * n + q] = co.b2; }
    status[q] = dom ? -1 : ok;
    if (iters) iters[q] = co.iters;
    if (path) path[q] = co.path;
}
// the preamble quantities of ctop (D, tau, Ssq, Bsq, SB) of cell q, pre [5][n]
BH_HD inline void ctop_pre_item(const KP& k, const double* U, const double* r, const double* th, int64_t n, int64_t q,
                                double* pre) {
    Cons c;
    c.D = U[q]; c.tau = U[4 * n + q];
    for (int d = 0; d < 3; d++) { c.S[d] = U[(1 + d) * n + q]; c.B[d] = U[(5 + d) * n + q]; }
    Met mc;
    met_comp(k.tree, r[q], th[q], mc);
    Prim w;
    bool dom = false;
    double p5[5];
    ctop(k.gamma, 0, k.tol, mc, c, w, dom, nullptr, NAN, p5);   // no Newton step: only the preamble is wanted
    for (int i = 0; i < 5; i++) pre[i * n + q] = p5[i];
}

BH_HD inline void hlld_item(const KP& k, const double* WL, const double* WR, const double* UL, const double* UR,
                            const double* r, const double* th, int dim, int64_t n, int64_t q, double* F,
                            double* cts) {
    Prim l, rw;
    Cons ul, ur;
    l.rho = WL[q]; l.eps = WL[n + q]; rw.rho = WR[q]; rw.eps = WR[n + q];
    ul.D = UL[q]; ul.tau = UL[4 * n + q]; ur.D = UR[q]; ur.tau = UR[4 * n + q];
    for (int d = 0; d < 3; d++) {
        l.v[d] = WL[(2 + d) * n + q]; l.B[d] = WL[(5 + d) * n + q];
        rw.v[d] = WR[(2 + d) * n + q]; rw.B[d] = WR[(5 + d) * n + q];
        ul.S[d] = UL[(1 + d) * n + q]; ul.B[d] = UL[(5 + d) * n + q];
        ur.S[d] = UR[(1 + d) * n + q]; ur.B[d] = UR[(5 + d) * n + q];
    }
    Met mc;
    met_comp(k.tree, r[q], th[q], mc);
    double f[8], c = 0;
    hlld(k.gamma, mc, l, rw, ul, ur, dim, f, c);
    for (int v = 0; v < 8; v++) F[v * n + q] = f[v];
    cts[q] = c;
}

}  // namespace bh
