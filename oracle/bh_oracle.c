/*
 * bh_oracle.c -- CPU restatement of the reference GRMHD block update.
 *
 * TEST INFRASTRUCTURE ONLY (see bh_oracle.h).  Each function cites the
 * reference function it restates (paths relative to src/fluid of
 * Fjoerde/black-hole-simulator).  Expression trees follow the reference's
 * left-to-right evaluation so that, compiled with -ffp-contract=off and
 * the same libm, results agree with the compiled reference bit for bit.
 */
#include "bh_oracle.h"
#include <math.h>
#include <string.h>

#ifdef ORC_NOISE
/* Built with -DORC_NOISE (liboracle_noise.so): every libm result on the
 * path (sin, cos, acos, log, exp, pow) is moved by at most one ulp, as a
 * deterministic function of its bits -- the same algorithm on a different
 * but equally accurate math library.  Its divergence from the plain build
 * measures how far the reference's own result is defined. */
static uint64_t orc_noise_seed = 0;
void orc_set_noise_seed(uint64_t s) { orc_noise_seed = s; }
static inline double orc_noise(double y) {
    if (!isfinite(y) || y == 0.0) return y;
    uint64_t b;
    memcpy(&b, &y, sizeof b);
    uint64_t h = (b ^ (orc_noise_seed * 0xD6E8FEB86659FD93ull)) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
    switch (h % 3) {
    case 0: return nextafter(y, -INFINITY);
    case 1: return y;
    default: return nextafter(y, INFINITY);
    }
}
#define sin(x) orc_noise(sin(x))
#define cos(x) orc_noise(cos(x))
#define acos(x) orc_noise(acos(x))
#define log(x) orc_noise(log(x))
#define exp(x) orc_noise(exp(x))
#define pow(x, y) orc_noise(pow(x, y))
#endif

#define BLK ORC_BLOCK
#define GH ORC_GHOST
#define CPN ORC_CPN
#define NC ORC_NC
#define NF ORC_NF
#define NE ORC_NE

/* std::min / std::max / std::abs semantics (NaN handling included) */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double sabs(double a) { return fabs(a); }

/* metriccomp, metric.hpp:11-21 (120 doubles, same member order) */
typedef struct {
    double g[4][4];
    double g_inv[4][4];
    double Gamma[4][4][4];
    double sqrtdetg;
    double gam[3][3];
    double gam_inv[3][3];
    double sqrtdetgam;
    double alpha;
    double beta[3];
} mcomp;

/* ======================================================================
 * L0: metric (physics/spacetime.cpp)
 * ==================================================================== */
/* black-hole parameters of one `metric` object (metric.hpp:25-32) */
typedef struct { double M, a, Q; } mpar;
static double Sigma_(const mpar *P, double r, double th) {          /* :12-14 */
    return r * r + P->a * P->a * pow(cos(th), 2);
}
static double H_(const mpar *P, double r, double th) {              /* :15-17 */
    return (2 * P->M * r - P->Q * P->Q) * pow(Sigma_(P, r, th), -1);
}
static void gcova(const mpar *P, double r, double th, double g[4][4]) { /* :20-34 */
    const double a = P->a;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) g[i][j] = 0.0;
    g[0][0] = -1 + H_(P, r, th);
    g[0][1] = g[1][0] = H_(P, r, th);
    g[1][1] = 1 + H_(P, r, th);
    g[2][2] = Sigma_(P, r, th);
    g[0][3] = g[1][3] = g[3][0] = g[3][1] = -H_(P, r, th) * a * pow(sin(th), 2);
    g[3][3] = (r * r + a * a + H_(P, r, th) * a * a * pow(sin(th), 2)) * pow(sin(th), 2);
}
static void gcntr(const mpar *P, double r, double th, double gi[4][4]) { /* :35-49 */
    const double a = P->a;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) gi[i][j] = 0.0;
    gi[0][0] = -1 - H_(P, r, th);
    gi[0][1] = gi[1][0] = H_(P, r, th);
    gi[1][1] = 1 - H_(P, r, th);
    gi[2][2] = pow(Sigma_(P, r, th), -1);
    gi[1][3] = gi[3][1] = a * pow(Sigma_(P, r, th), -1);
    gi[3][3] = pow(Sigma_(P, r, th) * sin(th) * sin(th), -1);
}
static void christ(const mpar *P, double r, double th, double gi[4][4],
                   double G[4][4][4]) {                              /* :57-90 */
    const double M = P->M, a = P->a, Q = P->Q;
    double d[4][4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) d[i][j][k] = 0;
    /* the eight distinct metric derivatives d[l][m][n] = d_l g_mn */
    d[1][0][0] = d[1][0][1] = d[1][1][0] = d[1][1][1] =
        -2 * (M * r * r - Q * Q * r - M * a * a * pow(cos(th), 2)) *
        pow(r * r + a * a * pow(cos(th), 2), -2);
    d[2][0][0] = d[2][0][1] = d[2][1][0] = d[2][1][1] =
        2 * a * a * (2 * M * r - Q * Q) * cos(th) * sin(th) *
        pow(r * r + a * a * pow(cos(th), 2), -1);
    d[1][2][2] = 2 * r;
    d[2][2][2] = -a * a * cos(th) * sin(th);
    d[1][0][3] = d[1][3][0] = d[1][1][3] = d[1][3][1] =
        2 * a * a * pow(sin(th), 2) * (M * r * r - Q * Q * r - M * a * a * pow(cos(th), 2)) *
        pow(r * r + a * a * pow(cos(th), 2), -2);
    d[2][0][3] = d[2][3][0] = d[2][1][3] = d[2][3][1] =
        2 * a * cos(th) * sin(th) * (2 * M * r - Q * Q) * (r * r + a * a) *
        pow(r * r + a * a * pow(cos(th), 2), -2);
    d[1][3][3] = pow(sin(th), 2) *
        (((2 * M * a * a * pow(sin(th), 2)) * pow(r * r + a * a * pow(cos(th), 2), -1)) +
         ((2 * r * a * a * pow(sin(th), 2) * (2 * M * r - Q * Q)) *
          pow(r * r + a * a * pow(cos(th), 2), -2)) +
         2 * r);
    d[2][3][3] = pow(sin(th), 2) *
        (((2 * pow(a, 4) * (2 * M * r - Q * Q) * cos(th) * pow(sin(th), 3)) *
          pow(r * r + a * a * pow(cos(th), 2), -2)) +
         ((2 * a * a * (2 * M * r - Q * Q) * cos(th) * sin(th)) *
          pow(r * r + a * a * pow(cos(th), 2), -1))) +
        cos(th) * sin(th) *
        (((a * a * pow(sin(th), 2) * (2 * M * r - Q * Q)) *
          pow(r * r + a * a * pow(cos(th), 2), -1)) +
         r * r + a * a);
    for (int l = 0; l < 4; l++)
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++)
                G[l][m][n] = 0.5 * (gi[l][0] * (d[m][0][n] + d[n][0][m] - d[0][m][n]) +
                                    gi[l][1] * (d[m][1][n] + d[n][1][m] - d[1][m][n]) +
                                    gi[l][2] * (d[m][2][n] + d[n][2][m] - d[2][m][n]) +
                                    gi[l][3] * (d[m][3][n] + d[n][3][m] - d[3][m][n]));
}
static void mcomp_m(const mpar *P, double r, double th, mcomp *mc) { /* :122-134 */
    gcova(P, r, th, mc->g);
    gcntr(P, r, th, mc->g_inv);
    mc->sqrtdetg = (r * r + P->a * P->a * pow(sin(th), 2)) * sin(th);   /* gdet :52-54 */
    christ(P, r, th, mc->g_inv, mc->Gamma);
    mc->alpha = pow(1 + H_(P, r, th), -1.0 / 2.0);                       /* lapse :93-95 */
    for (int i = 0; i < 3; i++) mc->beta[i] = -mc->g_inv[0][i + 1] / mc->g_inv[0][0]; /* :96-100 */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            mc->gam[i][j] = mc->g[i + 1][j + 1];                          /* :103-109 */
            mc->gam_inv[i][j] = mc->g_inv[i + 1][j + 1];                  /* :110-116 */
        }
    mc->sqrtdetgam = mc->alpha * mc->sqrtdetg;                            /* :117-119 */
}
/* the tree's metric (amrtree::mtr, used by conserved and hlld) */
static void mcomp_fill(const orc_params *P, double r, double th, mcomp *mc) {
    mpar m = {P->M, P->a, P->Q};
    mcomp_m(&m, r, th, mc);
}
/* the metric every cell carries (cell.hpp:25) */
static void mcomp_cell(const orc_params *P, double r, double th, mcomp *mc) {
    mpar m = {P->cM, P->ca, P->cQ};
    mcomp_m(&m, r, th, mc);
}
void orc_metric_comp(const orc_params *P, double r, double th, double out[ORC_NMC]) {
    mcomp mc;
    mcomp_fill(P, r, th, &mc);
    memcpy(out, &mc, sizeof(mc));
}

/* ======================================================================
 * L0: ideal-gas EOS (physics/thermo.cpp:10-35); rho<=0 -> domain_error
 * ==================================================================== */
#define EOS_CHECK(rho) do { if ((rho) <= 0.0) return ORC_EDOMAIN; } while (0)
static int press(const orc_params *P, double rho, double eps, double *out) {
    EOS_CHECK(rho); *out = (P->gamma - 1.0) * rho * eps; return 0;
}
static int enth(const orc_params *P, double rho, double eps, double *out) {
    EOS_CHECK(rho); *out = 1.0 + P->gamma * eps; return 0;
}
static int temp(double rho, double p, double *out) {
    EOS_CHECK(rho); *out = p / rho; return 0;
}
static int cs2f(const orc_params *P, double rho, double eps, double *out) {
    double p, h;
    EOS_CHECK(rho);
    press(P, rho, eps, &p);
    enth(P, rho, eps, &h);
    *out = (P->gamma * p) / (rho * h);
    return 0;
}

/* prim struct (prim.hpp:14-27) */
typedef struct { double rho, eps, v[3], B[3], p, T, h, lor, b2; } prim;
/* cons struct (cons.hpp:14-18) */
typedef struct { double D, S[3], tau, B[3]; } cons;

static void prim_from(const double W[8], prim *pv) {
    memset(pv, 0, sizeof(*pv));
    pv->rho = W[0]; pv->eps = W[1];
    for (int i = 0; i < 3; i++) { pv->v[i] = W[2 + i]; pv->B[i] = W[5 + i]; }
}
static void prim_to(const prim *pv, double W[8]) {
    W[0] = pv->rho; W[1] = pv->eps;
    for (int i = 0; i < 3; i++) { W[2 + i] = pv->v[i]; W[5 + i] = pv->B[i]; }
}
static void cons_from(const double U[8], cons *c) {
    c->D = U[0]; c->tau = U[4];
    for (int i = 0; i < 3; i++) { c->S[i] = U[1 + i]; c->B[i] = U[5 + i]; }
}
static void cons_to(const cons *c, double U[8]) {
    U[0] = c->D; U[4] = c->tau;
    for (int i = 0; i < 3; i++) { U[1 + i] = c->S[i]; U[5 + i] = c->B[i]; }
}

/* ======================================================================
 * L1: prim -> cons (physics/conserved.cpp:17-73); mutates lor,p,h,b2
 * ==================================================================== */
static int ptoc_(const orc_params *P, prim *pv, double r, double th, cons *CV) {
    mcomp mc;
    mcomp_fill(P, r, th, &mc);
    double sg = mc.sqrtdetgam;
    double v2 = 0.0, vlow[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) vlow[i] += mc.gam[i][j] * pv->v[j];
        v2 += vlow[i] * pv->v[i];
    }
    v2 = smin(v2, 1.0 - 1e-10);
    pv->lor = 1.0 / sqrt(1.0 - v2);
    if (press(P, pv->rho, pv->eps, &pv->p)) return ORC_EDOMAIN;
    if (enth(P, pv->rho, pv->eps, &pv->h)) return ORC_EDOMAIN;
    double Blow[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Blow[i] += mc.gam[i][j] * pv->B[j];
    double Bv = 0.0;
    for (int i = 0; i < 3; i++) Bv += Blow[i] * pv->v[i];
    double Bsq = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Bsq += Blow[i] * mc.gam[i][j] * pv->B[j];
    pv->b2 = (Bv * Bv + Bsq) / (pv->lor);
    double bt = pv->lor * Bv / mc.alpha;
    double pstar = pv->p + pv->b2 / 2;
    double w = pv->rho * pv->h + pv->b2;
    CV->D = sg * pv->rho * pv->lor;
    CV->tau = sg * (w * pv->lor * pv->lor - pstar - bt * bt) - CV->D;
    for (int i = 0; i < 3; i++) {
        double bi = (Blow[i] + mc.alpha * bt * pv->lor * vlow[i]) / pv->lor;
        CV->S[i] = sg * (w * pv->lor * pv->lor * vlow[i] - mc.alpha * bt * bi);
        CV->B[i] = sg * pv->B[i];
    }
    return 0;
}
int orc_ptoc(const orc_params *P, const double W[8], double r, double th, double U[8],
             double Wd[4]) {
    prim pv; cons c;
    prim_from(W, &pv);
    int rc = ptoc_(P, &pv, r, th, &c);
    if (rc) return rc;
    cons_to(&c, U);
    if (Wd) { Wd[0] = pv.lor; Wd[1] = pv.p; Wd[2] = pv.h; Wd[3] = pv.b2; }
    return 0;
}

/* ======================================================================
 * L1: cons -> prim (physics/conserved.cpp:80-285)
 * ==================================================================== */
static double f_df(const orc_params *P, double xi, double Ssq, double Bsq, double SB,
                   double Dn, double taun, double *df) {            /* :80-124 */
    double Yi = SB * SB;
    double K = Bsq;
    double X = xi * xi;
    double xipK = xi + K;
    double vsq = (Ssq * X + Yi * (2.0 * xi + K)) / (X + xipK * xipK);
    if (vsq >= 1.0) { *df = 0.0; return 1e30; }
    double ltz2 = 1.0 / (1.0 - vsq);
    double ltz = sqrt(ltz2);
    double rho = Dn / ltz;
    double G = P->gamma - 1.0;
    double p = (G / P->gamma) * (xi / ltz2 - Dn / ltz);
    double pstar = p + K / (2 * ltz2) + Yi / (2 * X);
    if (p < 0.0 || rho < 0.0) { *df = 0.0; return 1e32; }
    double f = xi - taun - Dn - pstar;
    double N = Ssq * X + Yi * (2.0 * xi + K);
    double Mq = X * xipK * xipK;
    double dN = 2.0 * Ssq * xi + 2.0 * Yi;
    double dM = 2.0 * xi * xipK * xipK + 2.0 * X * X;
    double dvv = (dN * Mq - dM * N) / (Mq * Mq);
    double dltz2 = ltz2 * ltz2 * dvv;
    double dltz = dltz2 / (2.0 * ltz);
    double dp = (G / P->gamma) * ((1.0 / ltz2) - (xi * dltz2) / (ltz2 * ltz2) + Dn * dltz / ltz2);
    double dpstar = dp - (K * dltz2) / (2.0 * ltz2 * ltz2) - Yi / (xi * X);
    *df = 1 - dpstar;
    return f;
}
static double fres(const orc_params *P, double xi, double Ssq, double Bsq, double SB,
                   double Dn, double taun) {                       /* :125-128 */
    double dum;
    return f_df(P, xi, Ssq, Bsq, SB, Dn, taun, &dum);
}
#define SWAPD(x, y) do { double t_ = (x); (x) = (y); (y) = t_; } while (0)
static int cp_bd(const orc_params *P, double xa, double xb, double Ssq, double Bsq,
                 double SB, double D, double tau, double *root, double tol) { /* :232-285 */
    double fa = fres(P, xa, Ssq, Bsq, SB, D, tau);
    double fb = fres(P, xb, Ssq, Bsq, SB, D, tau);
    if (fa * fb > 0.0) return 0;
    if (sabs(fa) < sabs(fb)) { SWAPD(xa, xb); SWAPD(fa, fb); }
    double xc = xa, fc = fa;
    int mflag = 1;
    double s = 0.0, d = 0.0;
    for (int i = 0; i < 100; i++) {
        if (sabs(xb - xa) < tol) { *root = xb; return 1; }
        if (fa != fc && fb != fc)
            s = (xa * fb * fc) / ((fa - fb) - (fa - fc)) + (xb * fa * fc) / ((fb - fa) - (fb - fc)) +
                (xc * fa * fb) / ((fc - fa) - (fc - fb));
        else
            s = xb - fb * (xb - xa) / (fb - fa);
        int c1 = !((3 * xa + 4) / 4 < s && s < xb);
        int c2 = mflag && sabs(s - xb) >= sabs(xb - xc) / 2;
        int c3 = !mflag && sabs(s - xb) >= sabs(xc - d) / 2;
        if (c1 || c2 || c3) { s = (xa + xb) / 2; mflag = 1; }
        else mflag = 0;
        double fs = fres(P, s, Ssq, Bsq, SB, D, tau);
        d = xc; xc = xb; fc = fb;
        if (fa * fs < 0.0) xb = s;
        else xa = s;
        if (sabs(fa) < sabs(fb)) { SWAPD(xa, xb); SWAPD(fa, fb); }
    }
    return 0;
}
/* ctop (:135-230).  Returns 1 / 0 like the reference's bool, or ORC_EDOMAIN
 * where the reference throws from the EOS. */
/* ctop with Newton started from xi0 when xi0 lies strictly inside the bracket
 * (the learned initial guess; NaN: the reference's bracket midpoint), and the
 * preamble's quantities D, tau, Ssq, Bsq, SB, xi_l, xi_h in pre[7] (may be NULL) */
static int ctop_g(const orc_params *P, const cons *cv, double r, double th, prim *pv,
                  int maxiter, double tol, int32_t *iters, int32_t *path, double xi0, double *pre);
static int ctop_(const orc_params *P, const cons *cv, double r, double th, prim *pv,
                 int maxiter, double tol, int32_t *iters, int32_t *path) {
    return ctop_g(P, cv, r, th, pv, maxiter, tol, iters, path, NAN, 0);
}
static int ctop_g(const orc_params *P, const cons *cv, double r, double th, prim *pv,
                  int maxiter, double tol, int32_t *iters, int32_t *path, double xi0, double *pre) {
    mcomp mc;
    mcomp_fill(P, r, th, &mc);
    double sg = mc.sqrtdetgam;
    double D = cv->D / sg;
    double tau = cv->tau / sg;
    double B[3] = {0.0, 0.0, 0.0}, S[3] = {0.0, 0.0, 0.0}; /* unassigned reads see 0 */
    double Bsq = 0.0, Ssq = 0.0, SB = 0.0;
    double Bu[3], Su[3];
    for (int i = 0; i < 3; i++) {
        B[i] = cv->B[i] / sg;
        S[i] = cv->S[i] / sg;
        for (int j = 0; j < 3; j++) {        /* assignment, not accumulation */
            Bu[i] = mc.gam_inv[i][j] * B[j];
            Su[i] = mc.gam_inv[i][j] * S[j];
        }
        Ssq += S[i] * Su[i];
        Bsq += B[i] * Bu[i];
        SB += S[i] * Bu[i];
    }
    double xi = tau + D;
    double xi_l = D;
    double xi_h = tau + D + Bsq / 2.0 + 1e3;
    double fl = fres(P, xi_l, Ssq, Bsq, SB, D, tau);
    double fh = fres(P, xi_h, Ssq, Bsq, SB, D, tau);
    while (fl * fh > 0.0 && xi_h < 1e8 * D) {
        xi_h *= 2.0;
        fl = fres(P, xi_h, Ssq, Bsq, SB, D, tau);
    }
    xi = (xi_l + xi_h) / 2.0;
    if (pre) { pre[0] = D; pre[1] = tau; pre[2] = Ssq; pre[3] = Bsq; pre[4] = SB; pre[5] = xi_l; pre[6] = xi_h; }
    if (isfinite(xi0) && xi0 > xi_l && xi0 < xi_h) xi = xi0;
    int nr_ok = 1, it = 0, converged = 0;
    for (int i = 0; i < maxiter; i++) {
        double dF;
        double F = f_df(P, xi, Ssq, Bsq, SB, D, tau, &dF);
        it = i + 1;
        if (sabs(F) < tol) { converged = 1; break; }
        if (sabs(dF) < 1e-30) { nr_ok = 0; break; }
        double xin = xi - F / dF;
        if (xin < xi_l || xin > xi_h) { nr_ok = 0; break; }
        xi = xin;
    }
    if (iters) *iters = it;
    if (path) *path = converged ? 0 : 1;
    if (!nr_ok) {
        double xib;
        if (!cp_bd(P, xi_l, xi_h, Ssq, Bsq, SB, D, tau, &xib, tol)) {
            if (path) *path = 3;
            return 0;
        }
        if (path) *path = 2;
        xi = xib;
    }
    double xpQ = xi + Bsq;
    double sdb2 = SB * SB;
    double vsq = (Ssq * xpQ * xpQ + sdb2 * (2.0 * xi + Bsq)) / (xpQ * xpQ * xi * xi);
    vsq = smin(vsq, 1.0 - 1e-10);
    double ltz2 = 1.0 / (1.0 - vsq);
    double ltz = sqrt(ltz2);
    pv->lor = ltz;
    pv->rho = D / ltz;
    double h = xi / (pv->rho * ltz2);
    pv->eps = (h - 1.0) / (P->gamma);
    if (press(P, pv->rho, pv->eps, &pv->p)) return ORC_EDOMAIN;
    if (enth(P, pv->rho, pv->eps, &pv->h)) return ORC_EDOMAIN;
    if (temp(pv->rho, pv->p, &pv->T)) return ORC_EDOMAIN;
    for (int i = 0; i < 3; i++) {
        pv->v[i] = (Su[i] + (SB / xi) * Bu[i]) / xpQ;
        pv->B[i] = B[i];
    }
    double Blow[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Blow[i] += mc.gam[i][j] * B[j];
    double Bv = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Bv += Blow[i] * mc.gam[i][j] * pv->v[j];
    pv->b2 = (Bv * Bv + Bsq) / ltz2;
    if (pv->rho <= 0.0 || pv->eps <= 0.0 || pv->p <= 0.0) return 0;
    return 1;
}
/* batched ctop with a per-cell Newton start xi0[n] (NaN: the midpoint) and
 * the preamble quantities pre [7][n] (may be NULL) */
void orc_ctop_guess_batch(const orc_params *P, const double *U, const double *r, const double *th, int64_t n,
                          const double *xi0, double *W, double *Wd, int32_t *status, int32_t *iters,
                          int32_t *path, double *pre) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t q = 0; q < n; q++) {
        cons c; prim pv;
        c.D = U[q]; c.tau = U[4 * n + q];
        for (int d = 0; d < 3; d++) { c.S[d] = U[(1 + d) * n + q]; c.B[d] = U[(5 + d) * n + q]; }
        memset(&pv, 0, sizeof(pv));
        double pr[7];
        int32_t it = 0, pa = 0;
        int ok = ctop_g(P, &c, r[q], th[q], &pv, P->maxiter, P->tol, &it, &pa, xi0 ? xi0[q] : NAN, pr);
        W[q] = pv.rho; W[n + q] = pv.eps;
        for (int d = 0; d < 3; d++) { W[(2 + d) * n + q] = pv.v[d]; W[(5 + d) * n + q] = pv.B[d]; }
        if (Wd) { Wd[q] = pv.p; Wd[n + q] = pv.T; Wd[2 * n + q] = pv.h; Wd[3 * n + q] = pv.lor; Wd[4 * n + q] = pv.b2; }
        status[q] = ok;
        if (iters) iters[q] = it;
        if (path) path[q] = pa;
        if (pre) for (int k = 0; k < 7; k++) pre[k * n + q] = pr[k];
    }
}
int orc_ctop(const orc_params *P, const double U[8], double r, double th, double W[8],
             double Wd[5], int32_t *iters, int32_t *path) {
    cons c; prim pv;
    memset(&pv, 0, sizeof(pv));
    cons_from(U, &c);
    int rc = ctop_(P, &c, r, th, &pv, P->maxiter, P->tol, iters, path);
    prim_to(&pv, W);
    if (Wd) { Wd[0] = pv.p; Wd[1] = pv.T; Wd[2] = pv.h; Wd[3] = pv.lor; Wd[4] = pv.b2; }
    return rc;
}

/* floor state (grid.cpp:133-146, constants grid.hpp:140-143) */
static void pvfs_(const orc_params *P, double r, prim *W) {
    memset(W, 0, sizeof(*W));
    double rfscal = 1.0 / pow(sqrt(smax(r, 1e-10) / 1.0), 3.0);
    W->rho = 1e-7 * rfscal;
    W->eps = 1e-5 * rfscal;
    press(P, W->rho, W->eps, &W->p);
    enth(P, W->rho, W->eps, &W->h);
    W->T = 1e-12;
}
void orc_pvfs(const orc_params *P, double r, double W[8]) {
    prim pv;
    pvfs_(P, r, &pv);
    prim_to(&pv, W);
}

/* ======================================================================
 * L1: HLLD (solver/hlld.cpp)
 * ==================================================================== */
typedef struct {
    double rho, eps, p, h, vn, vt1, vt2, Bn, Bt1, Bt2, v2, ltz, ltz2, b2, pt, cf, D, tau,
        Sn, St1, St2, Bc, E;
} side;
typedef struct { double D, Sn, St1, St2, tau, Bn, Bt1, Bt2; } cstt;

static double fastspeed(double rho, double h, double b2, double cs2) { /* :34-39 */
    double va2 = b2 / (rho * h + b2);
    double cf2 = cs2 + va2 * (1 - cs2);
    cf2 = smin(cf2, 1 - 1e-10);
    return sqrt(cf2);
}
static void magcomp(const prim *W, const mcomp *mc, int dim, side *s) { /* :41-71 */
    int t1 = (dim + 1) % 3, t2 = (dim + 2) % 3;
    double v2 = 0.0, vlow[3] = {0, 0, 0}, Blow[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            vlow[i] += mc->gam[i][j] * W->v[j];
            Blow[i] += mc->gam[i][j] * W->B[j];
        }
        v2 += vlow[i] * W->v[i];
    }
    v2 = smin(v2, 1 - 1e-10);
    s->v2 = v2;
    s->ltz2 = 1.0 / (1.0 - v2);
    s->ltz = sqrt(s->ltz2);
    double Bv = 0.0;
    for (int i = 0; i < 3; i++) Bv += Blow[i] * W->v[i];
    double Bsq = 0.0;
    for (int i = 0; i < 3; i++) Bsq += Blow[i] * W->B[i];
    s->b2 = Bv * Bv + Bsq / s->ltz2;
    s->vn = W->v[dim]; s->vt1 = W->v[t1]; s->vt2 = W->v[t2];
    s->Bn = W->B[dim]; s->Bt1 = W->B[t1]; s->Bt2 = W->B[t2];
}
static int side_(const orc_params *P, const prim *W, const cons *U, const mcomp *mc,
                 double sqrtg, int dim, side *s) {                  /* :73-94 */
    int t1 = (dim + 1) % 3, t2 = (dim + 2) % 3;
    s->rho = W->rho; s->eps = W->eps;
    if (press(P, W->rho, W->eps, &s->p)) return ORC_EDOMAIN;
    if (enth(P, W->rho, W->eps, &s->h)) return ORC_EDOMAIN;
    magcomp(W, mc, dim, s);
    s->pt = s->p + s->b2 / 2;
    double cs2;
    if (cs2f(P, W->rho, W->eps, &cs2)) return ORC_EDOMAIN;
    s->cf = fastspeed(s->rho, s->h, s->b2, cs2);
    s->D = U->D / sqrtg; s->tau = U->tau / sqrtg;
    s->Sn = U->S[dim] / sqrtg; s->St1 = U->S[t1] / sqrtg; s->St2 = U->S[t2] / sqrtg;
    s->Bc = U->B[dim] / sqrtg;
    s->E = s->tau + s->D;
    return 0;
}
static cstt physflux(const side *s, const mcomp *mc, int dim) {      /* :97-122 */
    cstt F;
    double vn = s->vn;
    F.D = s->D * vn;
    F.tau = (s->E + s->pt) * vn - s->Bn * (s->Bn * vn + s->Bt1 * s->vt1 + s->Bt2 * s->vt2) / s->ltz2;
    F.Sn = s->Sn * vn - s->Bn * s->Bn / s->ltz2 + s->pt;
    F.St1 = s->St1 * vn - s->Bt1 * s->Bn / s->ltz2;
    F.St2 = s->St2 * vn - s->Bt2 * s->Bn / s->ltz2;
    F.Bn = 0.0;
    F.Bt1 = s->Bt1 * vn - s->Bn * s->vt1;
    F.Bt2 = s->Bt2 * vn - s->Bn * s->vt2;
    double a = mc->alpha, btn = mc->beta[dim];
    F.D = a * F.D - btn * s->D;
    F.tau = a * F.tau - btn * s->tau;
    F.Sn = a * F.Sn - btn * s->Sn;
    F.St1 = a * F.St1 - btn * s->St1;
    F.St2 = a * F.St2 - btn * s->St2;
    F.Bn = a * F.Bn - btn * s->Bn;
    F.Bt1 = a * F.Bt1 - btn * s->Bt1;
    F.Bt2 = a * F.Bt2 - btn * s->Bt2;
    return F;
}
static cstt hll_flux(const side *L, const side *R, const cstt *FL, const cstt *FR,
                     double SL, double SR) {                        /* :124-137 */
    double dS = SR - SL;
    cstt F;
    F.D = (SR * FL->D - SL * FR->D + SL * SR * (R->D - L->D)) / dS;
    F.tau = (SR * FL->tau - SL * FR->tau + SL * SR * (R->tau - L->tau)) / dS;
    F.Sn = (SR * FL->Sn - SL * FR->Sn + SL * SR * (R->Sn - L->Sn)) / dS;
    F.St1 = (SR * FL->St1 - SL * FR->St1 + SL * SR * (R->St1 - L->St1)) / dS;
    F.St2 = (SR * FL->St2 - SL * FR->St2 + SL * SR * (R->St2 - L->St2)) / dS;
    F.Bn = (SR * FL->Bn - SL * FR->Bn + SL * SR * (R->Bn - L->Bn)) / dS;
    F.Bt1 = (SR * FL->Bt1 - SL * FR->Bt1 + SL * SR * (R->Bt1 - L->Bt1)) / dS;
    F.Bt2 = (SR * FL->Bt2 - SL * FR->Bt2 + SL * SR * (R->Bt2 - L->Bt2)) / dS;
    return F;
}
static cstt star_stt(const side *s, double SK, double SM, double pt_x) { /* :140-159 */
    cstt Ux;
    Ux.D = s->D * (SK - s->vn) / (SK - SM);
    Ux.tau = (s->E * (SK - s->vn) - s->pt * s->vn + pt_x * SM) / (SK - SM) - Ux.D;
    Ux.Sn = (s->Sn * (SK - s->vn) - s->pt + pt_x) / (SK - SM);
    Ux.St1 = s->St1 * (SK - s->vn) / (SK - SM);
    Ux.St2 = s->St2 * (SK - s->vn) / (SK - SM);
    Ux.Bn = s->Bc;
    double den = s->D * (SK - s->vn) * (SK - SM) - s->Bn * s->Bn;
    if (sabs(den) > 1e-14) {
        double k = s->Bn * (SM - s->vn) / den;
        Ux.Bt1 = s->Bt1 - s->Bn * (s->vt1 * (SK - s->vn) + s->Bn * s->Bt1 / s->D) * k;
        Ux.Bt2 = s->Bt2 - s->Bn * (s->vt2 * (SK - s->vn) + s->Bn * s->Bt2 / s->D) * k;
    } else {
        Ux.Bt1 = s->Bt1; Ux.Bt2 = s->Bt2;
    }
    return Ux;
}
/* alfstar_stt (:161-201); the degenerate branch at :171-173 is overwritten
 * by the assignments that follow it, so it has no effect. */
static void alfstar_stt(const cstt *UxL, const cstt *UxR, const side *L, double SM,
                        cstt *UxxL, cstt *UxxR) {
    UxxL->D = UxL->D; UxxL->tau = UxL->tau;
    UxxR->D = UxR->D; UxxR->tau = UxR->tau;
    UxxL->Bn = UxL->Bn; UxxR->Bn = UxR->Bn;
    double sq_DL = sqrt(sabs(UxL->D));
    double sq_DR = sqrt(sabs(UxR->D));
    double Bn = L->Bn;
    double den = sq_DL + sq_DR;
    double sgnBn = (Bn >= 0.0) ? 1.0 : -1.0;
    double vt1xx = (sq_DL * UxL->St1 / UxL->D + sq_DR * UxR->St1 / UxR->D + sgnBn * (UxR->Bt1 - UxL->Bt1)) / den;
    double vt2xx = (sq_DL * UxL->St2 / UxL->D + sq_DR * UxR->St2 / UxR->D + sgnBn * (UxR->Bt2 - UxL->Bt2)) / den;
    double Bt1xx = (sq_DL * UxL->Bt1 / UxL->D + sq_DR * UxR->Bt1 / UxR->D +
                    sgnBn * sq_DL * sq_DR * (UxR->St1 / UxR->D - UxL->St1 / UxL->D)) / den;
    double Bt2xx = (sq_DL * UxL->Bt2 / UxL->D + sq_DR * UxR->Bt2 / UxR->D +
                    sgnBn * sq_DL * sq_DR * (UxR->St2 / UxR->D - UxL->St2 / UxL->D)) / den;
    UxxL->St1 = UxL->D * vt1xx; UxxR->St1 = UxR->D * vt1xx;
    UxxL->St2 = UxL->D * vt2xx; UxxR->St2 = UxR->D * vt2xx;
    UxxL->Bt1 = Bt1xx; UxxR->Bt1 = Bt1xx;
    UxxL->Bt2 = Bt2xx; UxxR->Bt2 = Bt2xx;
    UxxL->Sn = UxL->D * SM; UxxR->Sn = UxR->D * SM;
    const double vt1xL = UxL->St1 / UxL->D;
    const double vt2xL = UxL->St2 / UxL->D;
    const double vt1xR = UxR->St1 / UxR->D;
    const double vt2xR = UxR->St2 / UxR->D;
    double dE_L = sq_DL * sgnBn * (vt1xx * Bt1xx + vt2xx * Bt2xx - vt1xL * UxL->Bt1 - vt2xL * UxL->Bt2);
    double dE_R = sq_DR * sgnBn * (vt1xx * Bt1xx + vt2xx * Bt2xx - vt1xR * UxR->Bt1 - vt2xR * UxR->Bt2);
    UxxL->tau = UxL->tau - dE_L;
    UxxR->tau = UxR->tau + dE_R;
}
static cstt interflux(const cstt *FK, double SK, const cstt *Ux, const side *s) { /* :203-216 */
    cstt F;
    F.D = FK->D + SK * (Ux->D - s->D);
    F.tau = FK->tau + SK * (Ux->tau - (s->E - s->D));
    F.Sn = FK->Sn + SK * (Ux->Sn - s->Sn);
    F.St1 = FK->St1 + SK * (Ux->St1 - s->St1);
    F.St2 = FK->St2 + SK * (Ux->St2 - s->St2);
    F.Bn = FK->Bn + SK * (Ux->Bn - s->Bc);
    F.Bt1 = FK->Bt1 + SK * (Ux->Bt1 - s->Bt1);
    F.Bt2 = FK->Bt2 + SK * (Ux->Bt2 - s->Bt2);
    return F;
}
static void flux_out(const cstt *F, double sg, int dim, cons *c) {  /* :218-227 */
    int t1 = (dim + 1) % 3, t2 = (dim + 2) % 3;
    c->D = sg * F->D; c->tau = sg * F->tau;
    c->B[dim] = sg * F->Bn; c->B[t1] = sg * F->Bt1; c->B[t2] = sg * F->Bt2;
    c->S[dim] = sg * F->Sn; c->S[t1] = sg * F->St1; c->S[t2] = sg * F->St2;
}
static int hlld_(const orc_params *P, const prim *WL, const prim *WR, const cons *UL,
                 const cons *UR, double r, double th, int dim, cons *Fout,
                 double *ctspeed) {                                  /* :230-312 */
    mcomp mc;
    mcomp_fill(P, r, th, &mc);
    double sg = mc.sqrtdetg;
    side L, R;
    if (side_(P, WL, UL, &mc, sg, dim, &L)) return ORC_EDOMAIN;
    if (side_(P, WR, UR, &mc, sg, dim, &R)) return ORC_EDOMAIN;
    double SL = smin(mc.alpha * (L.vn - L.cf) - mc.beta[dim], mc.alpha * (R.vn - R.cf) - mc.beta[dim]);
    double SR = smax(mc.alpha * (L.vn + L.cf) - mc.beta[dim], mc.alpha * (R.vn + R.cf) - mc.beta[dim]);
    cstt FL = physflux(&L, &mc, dim), FR = physflux(&R, &mc, dim);
    double cts = smax(sabs(SL), sabs(SR));
    cstt Fs;
    /* :244-246 computes an HLL flux that every later path overwrites */
    if (SL >= 0.0) { flux_out(&FL, sg, dim, Fout); *ctspeed = cts; return 0; }
    if (SR <= 0.0) { flux_out(&FR, sg, dim, Fout); *ctspeed = cts; return 0; }
    double pt_x = (SR * L.pt - SL * R.pt + SL * SR * (R.Sn - L.Sn)) / (SR - SL);
    double SM_u = SR * L.E - SL * R.E - FR.tau - FR.D + FL.tau + FL.D;
    double SM_d = SR * L.D - SL * R.D - FR.D + FL.D;
    if (sabs(SM_d) < 1e-12) {
        Fs = hll_flux(&L, &R, &FL, &FR, SL, SR);
        flux_out(&Fs, sg, dim, Fout); *ctspeed = cts; return 0;
    }
    double SM = SM_u / SM_d;
    cstt UxL = star_stt(&L, SL, SM, pt_x);
    cstt UxR = star_stt(&R, SR, SM, pt_x);
    double SLx = SM - sabs(L.Bn) / sqrt(sabs(UxL.D));
    double SRx = SM + sabs(R.Bn) / sqrt(sabs(UxR.D));
    if (UxL.D <= 0.0 || UxR.D <= 0.0) {
        Fs = hll_flux(&L, &R, &FL, &FR, SL, SR);
        flux_out(&Fs, sg, dim, Fout); *ctspeed = cts; return 0;
    }
    cons F;
    if (SM >= 0.0) {
        if (SLx >= 0.0) {
            Fs = interflux(&FL, SL, &UxL, &L);
        } else {
            cstt UxxL, UxxR;
            alfstar_stt(&UxL, &UxR, &L, SM, &UxxL, &UxxR);
            cstt FLx = interflux(&FL, SL, &UxL, &L);
            Fs = interflux(&FLx, SLx, &UxxL, &L);
        }
    } else {
        if (SRx >= 0.0) {
            Fs = interflux(&FR, SR, &UxR, &R);
        } else {
            cstt UxxL, UxxR;
            alfstar_stt(&UxL, &UxR, &L, SM, &UxxL, &UxxR);
            cstt FRx = interflux(&FR, SR, &UxR, &R);
            Fs = interflux(&FRx, SRx, &UxxR, &R);
        }
    }
    flux_out(&Fs, sg, dim, &F);
    if (!isfinite(F.D) || !isfinite(F.tau) || !isfinite(F.S[dim % 3]) ||
        !isfinite(F.S[(dim + 1) % 3]) || !isfinite(F.S[(dim + 2) % 3]) ||
        !isfinite(F.B[dim % 3]) || !isfinite(F.B[(dim + 1) % 3]) || !isfinite(F.B[(dim + 2) % 3])) {
        Fs = hll_flux(&L, &R, &FL, &FR, SL, SR);
        flux_out(&Fs, sg, dim, &F);
    }
    if (cts > 1.0) {
        Fs = hll_flux(&L, &R, &FL, &FR, SL, SR);
        flux_out(&Fs, sg, dim, &F);
        cts = smin(cts, 1.0);
    }
    *Fout = F;
    *ctspeed = cts;
    return 0;
}
int orc_hlld(const orc_params *P, const double WL[8], const double WR[8], const double UL[8],
             const double UR[8], double r, double th, int dim, double F[8], double *ctspeed) {
    prim L, R; cons cl, cr, f;
    prim_from(WL, &L); prim_from(WR, &R);
    cons_from(UL, &cl); cons_from(UR, &cr);
    memset(&f, 0, sizeof(f));
    double cts = 0.0;
    int rc = hlld_(P, &L, &R, &cl, &cr, r, th, dim, &f, &cts);
    cons_to(&f, F);
    if (ctspeed) *ctspeed = cts;
    return rc;
}

/* ======================================================================
 * patch storage and indexing (grid.hpp:19-21, grid.cpp:51-89)
 * ==================================================================== */
static inline int lindx(int i, int j, int k) { return (i + GH) * CPN * CPN + (j + GH) * CPN + (k + GH); }
static inline int xfc(int i, int j, int k) { return (i + GH) * CPN * CPN + (j + GH) * CPN + (k + GH); }
static inline int yfc(int i, int j, int k) { return (i + GH) * (CPN + 1) * CPN + (j + GH) * CPN + (k + GH); }
static inline int zfc(int i, int j, int k) { return (i + GH) * CPN * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
static inline int exi(int i, int j, int k) { return (i + GH) * (CPN + 1) * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
static inline int eyi(int i, int j, int k) { return (i + GH) * CPN * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
static inline int ezi(int i, int j, int k) { return (i + GH) * (CPN + 1) * CPN + (j + GH) * CPN + (k + GH); }

#define UP(pool, p, v) ((pool)->U + ((size_t)(p) * 8 + (v)) * NC)
#define WP(pool, p, v) ((pool)->W + ((size_t)(p) * 8 + (v)) * NC)
#define DUP(pool, p, v) ((pool)->dU + ((size_t)(p) * 8 + (v)) * NC)
#define FP(pool, p, d, v) ((pool)->F + (((size_t)(p) * 3 + (d)) * 8 + (v)) * NF)
#define BFP(pool, p, d) ((pool)->Bf + ((size_t)(p) * 3 + (d)) * NF)
#define EMP(pool, p, d) ((pool)->EMF + ((size_t)(p) * 3 + (d)) * NE)
#define RP(pool, p) ((pool)->rth + (size_t)(p) * 2 * NC)
#define TP(pool, p) ((pool)->rth + ((size_t)(p) * 2 + 1) * NC)

static void get_prim(const orc_pool *pool, int p, int l, prim *pv) {
    memset(pv, 0, sizeof(*pv));
    pv->rho = WP(pool, p, 0)[l]; pv->eps = WP(pool, p, 1)[l];
    for (int d = 0; d < 3; d++) { pv->v[d] = WP(pool, p, 2 + d)[l]; pv->B[d] = WP(pool, p, 5 + d)[l]; }
}
static void put_prim(orc_pool *pool, int p, int l, const prim *pv) {
    WP(pool, p, 0)[l] = pv->rho; WP(pool, p, 1)[l] = pv->eps;
    for (int d = 0; d < 3; d++) { WP(pool, p, 2 + d)[l] = pv->v[d]; WP(pool, p, 5 + d)[l] = pv->B[d]; }
}
static void get_cons(const orc_pool *pool, int p, int l, cons *c) {
    c->D = UP(pool, p, 0)[l]; c->tau = UP(pool, p, 4)[l];
    for (int d = 0; d < 3; d++) { c->S[d] = UP(pool, p, 1 + d)[l]; c->B[d] = UP(pool, p, 5 + d)[l]; }
}
static void put_cons(orc_pool *pool, int p, int l, const cons *c) {
    UP(pool, p, 0)[l] = c->D; UP(pool, p, 4)[l] = c->tau;
    for (int d = 0; d < 3; d++) { UP(pool, p, 1 + d)[l] = c->S[d]; UP(pool, p, 5 + d)[l] = c->B[d]; }
}

/* cell geometry, patch::cell_init (grid.cpp:149-175) */
void orc_geometry(orc_pool *pool) {
    for (int p = 0; p < pool->npatch; p++) {
        const double *g = pool->pgeo + 6 * p;
        for (int i = -GH; i < BLK + GH; i++)
            for (int j = -GH; j < BLK + GH; j++)
                for (int k = -GH; k < BLK + GH; k++) {
                    double xc = g[0] + (i + 0.5) * g[3];
                    double yc = g[1] + (j + 0.5) * g[4];
                    double zc = g[2] + (k + 0.5) * g[5];
                    double r = sqrt(xc * xc + yc * yc + zc * zc);
                    if (r < 1e-10) r = 1e-10;
                    double th = acos(smax(-1.0, smin(1.0, zc / r)));
                    int l = lindx(i, j, k);
                    RP(pool, p)[l] = r;
                    TP(pool, p)[l] = th;
                }
    }
}

/* ======================================================================
 * L1: PLM reconstruction (recon.hpp:16-41, grid/reconstruction.cpp)
 * ==================================================================== */
static double minmod(double a, double b) { if (a * b <= 0.0) return 0.0; return (sabs(a) < sabs(b)) ? a : b; }
static double min3mod(double a, double b, double c) { return minmod(a, minmod(b, c)); }
static double vanleer(double a, double b) { if (a * b <= 0.0) return 0.0; return 2.0 * a * b / (a + b); }
static double mclim(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    double c = (a + b) / 2;
    double s = (a > 0.0) ? 1.0 : -1.0;
    return s * min3mod(sabs(2 * a), sabs(2 * b), sabs(c));
}
static double lim_(double dl, double dr, int lim) {
    switch (lim) {
    case 0: return minmod(dl, dr);
    case 1: return vanleer(dl, dr);
    case 2: return mclim(dl, dr);
    default: return minmod(dl, dr);
    }
}
static void recon_scal(double Wm, double Wc, double Wp, double Wpp, int lim, double *fL, double *fR) {
    double dLc = Wc - Wm, dRc = Wp - Wc;
    double cslop = lim_(dLc, dRc, lim);
    *fL = Wc + cslop / 2.0;
    double dLp = Wp - Wc, dRp = Wpp - Wp;
    double pslop = lim_(dLp, dRp, lim);
    *fR = Wp - pslop / 2.0;
}
static void causalv(const orc_params *P, prim *W, double r, double th) {
    double v2 = 0.0;
    mcomp mc;
    mcomp_cell(P, r, th, &mc);
    for (int m = 0; m < 3; m++)
        for (int n = 0; n < 3; n++) v2 += mc.gam[m][n] * W->v[m] * W->v[n];
    if (v2 >= 1.0) {
        double s = (1 - 1e-10) / sqrt(v2);
        for (int a = 0; a < 3; a++) W->v[a] *= s;
    }
}
static void reconfp_(const orc_params *P, const orc_pool *pool, int p, int i, int j, int k,
                     int dim, int lim, prim *L, prim *R) {
    int di = (dim == 0), dj = (dim == 1), dk = (dim == 2);
    prim Wm, Wc, Wp, Wpp;
    get_prim(pool, p, lindx(i - di, j - dj, k - dk), &Wm);
    get_prim(pool, p, lindx(i, j, k), &Wc);
    get_prim(pool, p, lindx(i + di, j + dj, k + dk), &Wp);
    get_prim(pool, p, lindx(i + 2 * di, j + 2 * dj, k + 2 * dk), &Wpp);
    memset(L, 0, sizeof(*L));
    memset(R, 0, sizeof(*R));
    double fl, fr;
    recon_scal(log(Wm.rho), log(Wc.rho), log(Wp.rho), log(Wpp.rho), lim, &fl, &fr);
    L->rho = exp(fl); R->rho = exp(fr);
    recon_scal(log(Wm.eps), log(Wc.eps), log(Wp.eps), log(Wpp.eps), lim, &fl, &fr);
    L->eps = exp(fl); R->eps = exp(fr);
    for (int d = 0; d < 3; d++) {
        recon_scal(Wm.v[d], Wc.v[d], Wp.v[d], Wpp.v[d], lim, &fl, &fr);
        L->v[d] = fl; R->v[d] = fr;
    }
    int lc = lindx(i, j, k), lp = lindx(i + di, j + dj, k + dk);
    causalv(P, L, RP(pool, p)[lc], TP(pool, p)[lc]);
    causalv(P, R, RP(pool, p)[lp], TP(pool, p)[lp]);
    for (int d = 0; d < 3; d++) {
        if (d == dim) {
            L->B[d] = Wc.B[d]; R->B[d] = Wp.B[d];
        } else {
            recon_scal(Wm.B[d], Wc.B[d], Wp.B[d], Wpp.B[d], lim, &fl, &fr);
            L->B[d] = fl; R->B[d] = fr;
        }
    }
}
void orc_reconfp(const orc_params *P, const orc_pool *pool, int p, int i, int j, int k, int dim,
                 int lim, double L[8], double R[8]) {
    prim l, r;
    reconfp_(P, pool, p, i, j, k, dim, lim, &l, &r);
    prim_to(&l, L);
    prim_to(&r, R);
}

/* ======================================================================
 * L2: face fluxes, patch::fluxcomp (grid.cpp:255-329)
 * ==================================================================== */
static int face_flux(const orc_params *P, orc_pool *pool, int p, int i, int j, int k, int dim) {
    int di = (dim == 0), dj = (dim == 1), dk = (dim == 2);
    prim L, R;
    reconfp_(P, pool, p, i, j, k, dim, P->limiter, &L, &R);
    double bn;
    if (dim == 0) bn = BFP(pool, p, 0)[xfc(i + 1, j, k)];
    else if (dim == 1) bn = BFP(pool, p, 1)[yfc(i, j + 1, k)];
    else bn = BFP(pool, p, 2)[zfc(i, j, k + 1)];
    L.B[dim] = bn; R.B[dim] = bn;
    int lL = lindx(i, j, k), lR = lindx(i + di, j + dj, k + dk);
    double rf = (RP(pool, p)[lL] + RP(pool, p)[lR]) / 2;
    double thf = (TP(pool, p)[lL] + TP(pool, p)[lR]) / 2;
    cons UL, UR, F;
    if (ptoc_(P, &L, rf, thf, &UL)) return ORC_EDOMAIN;
    if (ptoc_(P, &R, rf, thf, &UR)) return ORC_EDOMAIN;
    double cts;
    memset(&F, 0, sizeof(F));
    if (hlld_(P, &L, &R, &UL, &UR, rf, thf, 0 /* every call site passes 0 */, &F, &cts))
        return ORC_EDOMAIN;
    int fi = dim == 0 ? xfc(i, j, k) : dim == 1 ? yfc(i, j, k) : zfc(i, j, k);
    double U8[8];
    cons_to(&F, U8);
    for (int v = 0; v < 8; v++) FP(pool, p, dim, v)[fi] = U8[v];
    return 0;
}
int orc_fluxcomp(const orc_params *P, orc_pool *pool, int p) {
    for (int i = -1; i < BLK; i++)
        for (int j = 0; j < BLK; j++)
            for (int k = 0; k < BLK; k++)
                if (face_flux(P, pool, p, i, j, k, 0)) return ORC_EDOMAIN;
    for (int i = 0; i < BLK; i++)
        for (int j = -1; j < BLK; j++)
            for (int k = 0; k < BLK; k++)
                if (face_flux(P, pool, p, i, j, k, 1)) return ORC_EDOMAIN;
    for (int i = 0; i < BLK; i++)
        for (int j = 0; j < BLK; j++)
            for (int k = -1; k < BLK; k++)
                if (face_flux(P, pool, p, i, j, k, 2)) return ORC_EDOMAIN;
    return 0;
}

/* ======================================================================
 * L2: constrained transport (grid/transport.cpp)
 * ==================================================================== */
void orc_emfcomp(orc_pool *pool, int p) {                            /* :11-36 */
    const double *FxB0 = FP(pool, p, 0, 5), *FxB1 = FP(pool, p, 0, 6), *FxB2 = FP(pool, p, 0, 7);
    const double *FyB0 = FP(pool, p, 1, 5), *FyB2 = FP(pool, p, 1, 7);
    const double *FzB0 = FP(pool, p, 2, 5), *FzB1 = FP(pool, p, 2, 6);
    double *Ex = EMP(pool, p, 0), *Ey = EMP(pool, p, 1), *Ez = EMP(pool, p, 2);
    (void)FxB0;
    for (int i = -GH; i < BLK + GH - 1; i++)
        for (int j = -GH; j < BLK + GH - 1; j++)
            for (int k = -GH; k < BLK + GH - 1; k++) {
                double a = FyB2[yfc(i, j, k)], b = FyB2[yfc(i, j, k + 1)];
                double c = FzB1[zfc(i, j, k)], d = FzB1[zfc(i, j + 1, k)];
                Ex[exi(i, j, k)] = (a + b - c - d) / 4;
                double e = FxB2[xfc(i, j, k)], f = FxB2[xfc(i, j, k + 1)];
                double g = FzB0[zfc(i, j, k)], h = FzB0[zfc(i + 1, j, k)];
                Ey[eyi(i, j, k)] = (g + h - e - f) / 4;
                double m = FxB1[xfc(i, j, k)], n = FxB1[xfc(i, j + 1, k)];
                double o = FyB0[yfc(i, j, k)], q = FyB0[yfc(i + 1, j, k)];
                Ez[ezi(i, j, k)] = (m + n - o - q) / 4;
            }
}
void orc_bfupdate(orc_pool *pool, int p, double dt) {                /* :38-58 */
    const double *g = pool->pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double *Ex = EMP(pool, p, 0), *Ey = EMP(pool, p, 1), *Ez = EMP(pool, p, 2);
    double *Bx = BFP(pool, p, 0), *By = BFP(pool, p, 1), *Bz = BFP(pool, p, 2);
    for (int i = -GH + 1; i < BLK + GH - 1; i++)
        for (int j = -GH + 1; j < BLK + GH - 1; j++)
            for (int k = -GH + 1; k < BLK + GH - 1; k++) {
                double dEz_dy = (Ez[ezi(i, j, k)] - Ez[ezi(i, j - 1, k)]) / dy;
                double dEy_dz = (Ey[eyi(i, j, k)] - Ey[eyi(i, j, k - 1)]) / dz;
                Bx[xfc(i, j, k)] += dt * (dEz_dy - dEy_dz);
                double dEz_dx = (Ez[ezi(i, j, k)] - Ez[ezi(i - 1, j, k)]) / dx;
                double dEx_dz = (Ex[exi(i, j, k)] - Ex[exi(i, j, k - 1)]) / dz;
                By[yfc(i, j, k)] += dt * (dEx_dz - dEz_dx);
                double dEy_dx = (Ey[eyi(i, j, k)] - Ey[eyi(i - 1, j, k)]) / dx;
                double dEx_dy = (Ex[exi(i, j, k)] - Ex[exi(i, j - 1, k)]) / dy;
                Bz[zfc(i, j, k)] += dt * (dEy_dx - dEx_dy);
            }
}
void orc_f2cb(const orc_params *P, orc_pool *pool, int p) {         /* :60-75 */
    const double *Bx = BFP(pool, p, 0), *By = BFP(pool, p, 1), *Bz = BFP(pool, p, 2);
    for (int i = -GH + 1; i < BLK + GH; i++)
        for (int j = -GH + 1; j < BLK + GH; j++)
            for (int k = -GH + 1; k < BLK + GH; k++) {
                int l = lindx(i, j, k);
                double b0 = (Bx[xfc(i, j, k)] + Bx[xfc(i - 1, j, k)]) / 2;
                double b1 = (By[yfc(i, j, k)] + By[yfc(i, j - 1, k)]) / 2;
                double b2 = (Bz[zfc(i, j, k)] + Bz[zfc(i, j, k - 1)]) / 2;
                WP(pool, p, 5)[l] = b0; WP(pool, p, 6)[l] = b1; WP(pool, p, 7)[l] = b2;
                mcomp mc;
                mcomp_cell(P, RP(pool, p)[l], TP(pool, p)[l], &mc);
                double sg = mc.sqrtdetg;
                UP(pool, p, 5)[l] = sg * b0; UP(pool, p, 6)[l] = sg * b1; UP(pool, p, 7)[l] = sg * b2;
            }
}
double orc_maxdivb(const orc_pool *pool, int p) {                   /* :77-89 */
    const double *g = pool->pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double *Bx = BFP(pool, p, 0), *By = BFP(pool, p, 1), *Bz = BFP(pool, p, 2);
    double maxdiv = 0;
    for (int i = -GH + 1; i < BLK + GH - 1; i++)
        for (int j = -GH + 1; j < BLK + GH - 1; j++)
            for (int k = -GH + 1; k < BLK + GH - 1; k++) {
                double divB = (Bx[xfc(i, j, k)] - Bx[xfc(i - 1, j, k)]) / dx +
                              (By[yfc(i, j, k)] - By[yfc(i, j - 1, k)]) / dy +
                              (Bz[zfc(i, j, k)] - Bz[zfc(i, j, k - 1)]) / dz;
                maxdiv = smax(maxdiv, sabs(divB));
            }
    return maxdiv;
}

/* ======================================================================
 * L3: flux divergence and geometric source (solver/integrator.cpp:18-153)
 * ==================================================================== */
void orc_div_flux(const orc_params *P, const orc_pool *pool, int p, int i, int j, int k,
                  double out[8]) {
    const double *g = pool->pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    int l = lindx(i, j, k);
    mcomp mc;
    mcomp_cell(P, RP(pool, p)[l], TP(pool, p)[l], &mc);
    double sg = mc.sqrtdetg;
    int xr = xfc(i, j, k), xl = xfc(i - 1, j, k);
    int yr = yfc(i, j, k), yl = yfc(i, j - 1, k);
    int zr = zfc(i, j, k), zl = zfc(i, j, k - 1);
    for (int v = 0; v < 5; v++) {
        const double *Fx = FP(pool, p, 0, v), *Fy = FP(pool, p, 1, v), *Fz = FP(pool, p, 2, v);
        out[v] = -((Fx[xr] - Fx[xl]) / dx + (Fy[yr] - Fy[yl]) / dy + (Fz[zr] - Fz[zl]) / dz) / sg;
    }
    out[5] = out[6] = out[7] = 0.0;
}
int orc_source(const orc_params *P, const orc_pool *pool, int p, int i, int j, int k,
               double out[8]) {
    int l = lindx(i, j, k);
    double r = RP(pool, p)[l], th = TP(pool, p)[l];
    prim W;
    get_prim(pool, p, l, &W);
    mcomp mc;
    mcomp_cell(P, r, th, &mc);
    double v2 = 0.0, vlow[3] = {0, 0, 0}, Blow[3] = {0, 0, 0};
    for (int m = 0; m < 3; m++) {
        for (int n = 0; n < 3; n++) {
            vlow[m] += mc.gam[m][n] * W.v[n];
            Blow[m] += mc.gam[m][n] * W.B[n];
        }
        v2 += vlow[m] * W.v[m];
    }
    v2 = smin(v2, 1 - 1e-10);
    double ltz2 = 1.0 / (1.0 - v2);
    double ltz = sqrt(ltz2);
    double Bv = 0.0, Bsq = 0.0;
    for (int m = 0; m < 3; m++) {
        Bv += Blow[m] * W.v[m];
        Bsq += Blow[m] * W.B[m];
    }
    double b2 = Bv * Bv + Bsq / ltz2;
    double px, h;
    if (press(P, W.rho, W.eps, &px)) return ORC_EDOMAIN;
    if (enth(P, W.rho, W.eps, &h)) return ORC_EDOMAIN;
    double u4[4], u_4[4] = {0, 0, 0, 0};
    u4[0] = ltz / mc.alpha;
    for (int m = 0; m < 3; m++) u4[m + 1] = ltz * (W.v[m] - mc.beta[m] / mc.alpha);
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) u_4[m] += mc.g[m][n] * u4[n];
    double b4[4], b_4[4] = {0, 0, 0, 0};
    b4[0] = ltz * Bv / mc.alpha;
    for (int m = 0; m < 3; m++) b4[m + 1] = (W.B[m] + mc.alpha * b4[0] * u4[m + 1]) / ltz;
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) b_4[m] += mc.g[m][n] * b4[n];
    (void)u_4; (void)b_4;
    double T44[4][4];
    double rhohb2 = W.rho * h + b2;
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
            T44[m][n] = rhohb2 * u4[m] * u4[n] + px * mc.g_inv[m][n] - b4[m] * b4[n];
    double Gam_[4][4][4];
    memset(Gam_, 0, sizeof(Gam_));
    for (int n = 0; n < 4; n++)
        for (int z = 0; z < 4; z++)
            for (int q = 0; q < 4; q++)
                for (int s = 0; s < 4; s++) Gam_[n][z][q] += mc.g[n][s] * mc.Gamma[s][z][q];
    double src[4] = {0, 0, 0, 0};
    for (int m = 0; m < 4; m++) {
        for (int n = 0; n < 4; n++)
            for (int q = 0; q < 4; q++) src[m] += T44[n][q] * Gam_[m][n][q];
        src[m] *= mc.sqrtdetg;
    }
    out[0] = 0.0;
    out[4] = src[0];
    out[1] = src[1]; out[2] = src[2]; out[3] = src[3];
    out[5] = out[6] = out[7] = 0.0;
    return 0;
}

/* ======================================================================
 * L2: ghost fill, amrtree::ghosts (grid.cpp:361-571), neighbour from table
 * ==================================================================== */
static void copy_cell(orc_pool *pool, int pd, int ld, int ps, int ls) {
    for (int v = 0; v < 8; v++) {
        UP(pool, pd, v)[ld] = UP(pool, ps, v)[ls];
        WP(pool, pd, v)[ld] = WP(pool, ps, v)[ls];
    }
}
static void gh_copy(orc_pool *pool, int p, int nb, int dim, int side) { /* :390-425 */
    int pstart = (side == 1) ? BLK : -GH;
    int nbstart = (side == 1) ? 0 : BLK - GH;
    for (int g = 0; g < GH; g++)
        for (int t1 = 0; t1 < BLK; t1++)
            for (int t2 = 0; t2 < BLK; t2++) {
                int pi, pj, pk, ni, nj, nk;
                if (dim == 0) { pi = pstart + g; pj = t1; pk = t2; ni = nbstart + g; nj = t1; nk = t2; }
                else if (dim == 1) { pi = t1; pj = pstart + g; pk = t2; ni = t1; nj = nbstart + g; nk = t2; }
                else { pi = t1; pj = t2; pk = pstart + g; ni = t1; nj = t2; nk = nbstart + g; }
                copy_cell(pool, p, lindx(pi, pj, pk), nb, lindx(ni, nj, nk));
            }
}
static void gh_bndy(orc_pool *pool, int p, int dim, int side) {      /* :494-522 */
    int pstart = (side == 1) ? BLK : -GH;
    for (int g = 0; g < GH; g++)
        for (int t1 = 0; t1 < BLK; t1++)
            for (int t2 = 0; t2 < BLK; t2++) {
                int gi, gj, gk, ai, aj, ak;
                int a = (side == 1) ? BLK - 1 - g : g;
                if (dim == 0) { gi = pstart + g; gj = t1; gk = t2; ai = a; aj = t1; ak = t2; }
                else if (dim == 1) { gi = t1; gj = pstart + g; gk = t2; ai = t1; aj = a; ak = t2; }
                else { gi = t1; gj = t2; gk = pstart + g; ai = t1; aj = t2; ak = a; }
                copy_cell(pool, p, lindx(gi, gj, gk), p, lindx(ai, aj, ak));
            }
}
/* floor fallback used after a failed ctop in refine/prolong/rkstg:
 * W = pvfs with the cell's B kept, U = ptoc(W) */
static int floor_reset_out(const orc_params *P, orc_pool *pool, int p, int l, prim *out) {
    double r = RP(pool, p)[l], th = TP(pool, p)[l];
    prim fl, cur;
    get_prim(pool, p, l, &cur);
    pvfs_(P, r, &fl);
    for (int d = 0; d < 3; d++) fl.B[d] = cur.B[d];
    put_prim(pool, p, l, &fl);
    cons U;
    if (ptoc_(P, &fl, r, th, &U)) return ORC_EDOMAIN;   /* ptoc sets fl's lor, p, h, b2 */
    put_cons(pool, p, l, &U);
    if (out) *out = fl;
    return 0;
}
static int floor_reset(const orc_params *P, orc_pool *pool, int p, int l) {
    return floor_reset_out(P, pool, p, l, 0);
}
/* the derived primitive fields a cell's W carries (prim.hpp:21-25) */
static void put_derived(orc_pool *pool, int p, int l, const prim *pv) {
    if (!pool->Wd) return;
    double *d = pool->Wd + (size_t)p * 4 * NC;
    d[l] = pv->lor; d[NC + l] = pv->p; d[2 * NC + l] = pv->h; d[3 * NC + l] = pv->b2;
}
static int gh_prolong(const orc_params *P, orc_pool *pool, int p, int nb, int dim, int side) { /* :427-492 */
    int pstart = (side == 1) ? BLK : -GH;
    for (int g = 0; g < GH; g++)
        for (int t1 = 0; t1 < BLK; t1++)
            for (int t2 = 0; t2 < BLK; t2++) {
                int fi, fj, fk;
                if (dim == 0) { fi = pstart + g; fj = t1; fk = t2; }
                else if (dim == 1) { fi = t1; fj = pstart + g; fk = t2; }
                else { fi = t1; fj = t2; fk = pstart + g; }
                int ci = (dim == 0) ? g / 2 : t1 / 2;
                int cj = (dim == 1) ? g / 2 : (dim == 0 ? t1 / 2 : t2 / 2);
                int ck = (dim == 2) ? g / 2 : t2 / 2;
                double offg = (g % 2 == 0) ? -0.25 : 0.25;
                double offt1 = (t1 % 2 == 0) ? -0.25 : 0.25;
                double offt2 = (t2 % 2 == 0) ? -0.25 : 0.25;
                double on, ot1, ot2;
                if (dim == 0) { on = offg; ot1 = offt1; ot2 = offt2; }
                else if (dim == 1) { on = offt1; ot1 = offg; ot2 = offt2; }
                else { on = offt1; ot1 = offt2; ot2 = offg; }
                int lf = lindx(fi, fj, fk);
                int lc = lindx(ci, cj, ck);
                int lxm = lindx(ci - 1, cj, ck), lxp = lindx(ci + 1, cj, ck);
                int lym = lindx(ci, cj - 1, ck), lyp = lindx(ci, cj + 1, ck);
                int lzm = lindx(ci, cj, ck - 1), lzp = lindx(ci, cj, ck + 1);
                static const int order[8] = {0, 4, 5, 1, 6, 2, 7, 3}; /* D, tau, B0,S0, B1,S1, B2,S2 */
                for (int q = 0; q < 8; q++) {
                    int v = order[q];
                    const double *c = UP(pool, nb, v);
                    double vm = c[lxm], vc = c[lc], vp = c[lxp];
                    double vm1 = c[lym], vp1 = c[lyp], vm2 = c[lzm], vp2 = c[lzp];
                    double sn = minmod(vc - vm, vp - vc);
                    double st1 = minmod(vc - vm1, vp1 - vc);
                    double st2 = minmod(vc - vm2, vp2 - vc);
                    UP(pool, p, v)[lf] = vc + sn * on + st1 * ot1 + st2 * ot2;
                }
                cons U; prim pv;
                get_cons(pool, p, lf, &U);
                memset(&pv, 0, sizeof(pv));
                int ok = ctop_(P, &U, RP(pool, p)[lf], TP(pool, p)[lf], &pv, P->maxiter, P->tol, 0, 0);
                if (ok < 0) return ORC_EDOMAIN;
                if (ok) put_prim(pool, p, lf, &pv);
                else if (floor_reset(P, pool, p, lf)) return ORC_EDOMAIN;
            }
    return 0;
}
int orc_ghosts(const orc_params *P, orc_pool *pool, int p) {          /* :524-571 */
    for (int dim = 0; dim < 3; dim++)
        for (int s = 0; s < 2; s++) {
            int side = s ? 1 : -1;
            int nb = pool->nbr[(p * 6 + dim * 2 + s) * 2 + 0];
            int kind = pool->nbr[(p * 6 + dim * 2 + s) * 2 + 1];
            if (kind == ORC_NB_COPY) gh_copy(pool, p, nb, dim, side);
            else if (kind == ORC_NB_PROLONG) { if (gh_prolong(P, pool, p, nb, dim, side)) return ORC_EDOMAIN; }
            else gh_bndy(pool, p, dim, side);
        }
    for (int i = -GH; i < BLK + GH; i++)
        for (int j = -GH; j < BLK + GH; j++)
            for (int k = -GH; k < BLK + GH; k++) {
                if (!(i < 0 || i >= BLK || j < 0 || j >= BLK || k < 0 || k >= BLK)) continue;
                int l = lindx(i, j, k);
                cons U; prim pv;
                get_cons(pool, p, l, &U);
                memset(&pv, 0, sizeof(pv));
                int ok = ctop_(P, &U, RP(pool, p)[l], TP(pool, p)[l], &pv, P->maxiter, P->tol, 0, 0);
                if (ok < 0) return ORC_EDOMAIN;
                if (ok) {
                    put_prim(pool, p, l, &pv);
                } else {
                    /* :560-565 -- only rho and eps take the floor values;
                     * v and B keep the cell's previous primitives */
                    prim fl, cur;
                    pvfs_(P, RP(pool, p)[l], &fl);
                    get_prim(pool, p, l, &cur);
                    cur.rho = fl.rho; cur.eps = fl.eps;
                    put_prim(pool, p, l, &cur);
                    cons Un;
                    if (ptoc_(P, &cur, RP(pool, p)[l], TP(pool, p)[l], &Un)) return ORC_EDOMAIN;
                    put_cons(pool, p, l, &Un);
                }
            }
    return 0;
}

/* ======================================================================
 * L2: AMR regrid (grid/grid.cpp:573-835)
 * ==================================================================== */

/* refinement / flattening flags of leaf patch p at level lvl, from the cell
 * loop of amrtree::regrid (:763-820): bit 0 = some cell asks for refinement
 * (patch->refine), bit 1 = every cell allows flattening (patch->erase) */
int orc_regrid_flags(const orc_pool *pool, int p, int lvl) {
    const double lim_refine = 0.5, lim_flatten = 0.1, r0 = 3.0;   /* :765-768 */
    const int max_lvl = 4;
    const double *g = pool->pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    const double *rho = WP(pool, p, 0);
    const double *B0 = WP(pool, p, 5), *B1 = WP(pool, p, 6), *B2 = WP(pool, p, 7);
    int anyref = 0, allflt = 1;
    for (int i = 0; i < BLK; i++)
        for (int j = 0; j < BLK; j++)
            for (int k = 0; k < BLK; k++) {
                int l = lindx(i, j, k);
                if (RP(pool, p)[l] < r0 && lvl < max_lvl) { anyref = 1; allflt = 0; continue; }
                double chro = rho[l];
                if (chro > 0.0) {
                    double drho_dx = fabs(rho[lindx(i + 1, j, k)] - rho[lindx(i - 1, j, k)]) / (2 * dx);
                    double drho_dy = fabs(rho[lindx(i, j + 1, k)] - rho[lindx(i, j - 1, k)]) / (2 * dy);
                    double drho_dz = fabs(rho[lindx(i, j, k + 1)] - rho[lindx(i, j, k - 1)]) / (2 * dz);
                    double drho = sqrt(drho_dx * drho_dx + drho_dy * drho_dy + drho_dz * drho_dz);
                    double rgrh = drho * dx / chro;
                    if (rgrh > lim_refine && lvl < max_lvl) { anyref = 1; allflt = 0; }
                    if (rgrh > lim_flatten) allflt = 0;
                }
                double Bmag = sqrt(B0[l] * B0[l] + B1[l] * B1[l] + B2[l] * B2[l]);
                if (Bmag > 1e-14) {
                    double dB_dx = fabs(B0[lindx(i + 1, j, k)] - B0[lindx(i - 1, j, k)]) / (2 * dx);
                    double dB_dy = fabs(B1[lindx(i, j + 1, k)] - B1[lindx(i, j - 1, k)]) / (2 * dy);
                    double dB_dz = fabs(B2[lindx(i, j, k + 1)] - B2[lindx(i, j, k - 1)]) / (2 * dz);
                    double rdB = (dB_dx * dx + dB_dy * dy + dB_dz * dz) / Bmag;
                    if (rdB > lim_refine && lvl < max_lvl) { anyref = 1; allflt = 0; }
                }
            }
    return ((anyref && lvl < max_lvl) ? 1 : 0) | ((allflt && lvl > 0) ? 2 : 0);
}

/* patch::B_init (:207-250): face B from the cells' W.B over all 20^3 cells.
 * The z-face branch tests i (not k) against -ghost (quirk A19); its
 * out-of-range cell indices k = -3 and k = 18 are used as the reference's
 * linear index computes them (neighbouring cells in memory order). */
void orc_b_init(orc_pool *pool, int p) {
    const double *B0 = WP(pool, p, 5), *B1 = WP(pool, p, 6), *B2 = WP(pool, p, 7);
    double *Bx = BFP(pool, p, 0), *By = BFP(pool, p, 1), *Bz = BFP(pool, p, 2);
    for (int i = -GH; i < BLK + GH + 1; i++)
        for (int j = -GH; j < BLK + GH; j++)
            for (int k = -GH; k < BLK + GH; k++) {
                if (i > -GH && i < BLK + GH) Bx[xfc(i, j, k)] = (B0[lindx(i - 1, j, k)] + B0[lindx(i, j, k)]) / 2;
                else if (i == -GH) Bx[xfc(i, j, k)] = B0[lindx(i, j, k)];
                else Bx[xfc(i, j, k)] = B0[lindx(i - 1, j, k)];
            }
    for (int i = -GH; i < BLK + GH; i++)
        for (int j = -GH; j < BLK + GH + 1; j++)
            for (int k = -GH; k < BLK + GH; k++) {
                if (j > -GH && j < BLK + GH) By[yfc(i, j, k)] = (B1[lindx(i, j - 1, k)] + B1[lindx(i, j, k)]) / 2;
                else if (j == -GH) By[yfc(i, j, k)] = B1[lindx(i, j, k)];
                else By[yfc(i, j, k)] = B1[lindx(i, j - 1, k)];
            }
    for (int i = -GH; i < BLK + GH; i++)
        for (int j = -GH; j < BLK + GH; j++)
            for (int k = -GH; k < BLK + GH + 1; k++) {
                if (k > -GH && k < BLK + GH) Bz[zfc(i, j, k)] = (B2[lindx(i, j, k - 1)] + B2[lindx(i, j, k)]) / 2;
                else if (i == -GH) Bz[zfc(i, j, k)] = B2[lindx(i, j, k)];
                else Bz[zfc(i, j, k)] = B2[lindx(i, j, k - 1)];
            }
}

/* ctop of a regridded cell with the fallback of refine/ccrstr (:636-645,
 * :694-703): on failure W = pvfs(r) with B = the cell's current W.B (zero
 * in a newly created child), U = ptoc(W) */
static int regrid_recover(const orc_params *P, orc_pool *pool, int p, int l) {
    cons U; prim pv;
    get_cons(pool, p, l, &U);
    memset(&pv, 0, sizeof(pv));
    int ok = ctop_(P, &U, RP(pool, p)[l], TP(pool, p)[l], &pv, P->maxiter, P->tol, 0, 0);
    if (ok < 0) return ORC_EDOMAIN;
    if (ok) { put_prim(pool, p, l, &pv); put_derived(pool, p, l, &pv); return 0; }
    prim fl;
    if (floor_reset_out(P, pool, p, l, &fl)) return ORC_EDOMAIN;
    put_derived(pool, p, l, &fl);
    return 0;
}

/* the cell data of amrtree::refine (:603-648): child h of parent p takes a
 * minmod-limited interpolation of the parent's conserved variables.  The
 * reference's prolong lambda is declared (vc, vmx, vpx, ...) but called
 * with the +x neighbour first, so each slope is minmod(vc - v[+1], v[-1] - vc).
 * Then ctop with its fallback, and B_init of the child. */
int orc_refine_data(const orc_params *P, orc_pool *pool, int p, const int32_t child[8]) {
    for (int h = 0; h < 8; h++) {
        int c = child[h];
        int ix = (h >> 2) & 1, iy = (h >> 1) & 1, iz = h & 1;
        for (int i = 0; i < BLK; i++)
            for (int j = 0; j < BLK; j++)
                for (int k = 0; k < BLK; k++) {
                    int pi = (i + ix * BLK) / 2, pj = (j + iy * BLK) / 2, pk = (k + iz * BLK) / 2;
                    double ox = (i % 2 == 0) ? -0.25 : 0.25;
                    double oy = (j % 2 == 0) ? -0.25 : 0.25;
                    double oz = (k % 2 == 0) ? -0.25 : 0.25;
                    int lc = lindx(pi, pj, pk);
                    int lpx = lindx(pi + 1, pj, pk), lmx = lindx(pi - 1, pj, pk);
                    int lpy = lindx(pi, pj + 1, pk), lmy = lindx(pi, pj - 1, pk);
                    int lpz = lindx(pi, pj, pk + 1), lmz = lindx(pi, pj, pk - 1);
                    int lf = lindx(i, j, k);
                    for (int v = 0; v < 8; v++) {
                        const double *u = UP(pool, p, v);
                        double vc = u[lc];
                        double sx = minmod(vc - u[lpx], u[lmx] - vc);
                        double sy = minmod(vc - u[lpy], u[lmy] - vc);
                        double sz = minmod(vc - u[lpz], u[lmz] - vc);
                        UP(pool, c, v)[lf] = vc + sx * ox + sy * oy + sz * oz;
                    }
                    if (regrid_recover(P, pool, c, lf)) return ORC_EDOMAIN;
                }
        orc_b_init(pool, c);
    }
    return 0;
}

/* amrtree::ccrstr (:651-712): each parent cell takes the volume-weighted
 * mean of the eight child cells of its octant (cons() + vol * U, in the
 * child-cell order di, dj, dk), then ctop with its fallback; then B_init */
int orc_ccrstr(const orc_params *P, orc_pool *pool, int p, const int32_t child[8]) {
    for (int pi = 0; pi < BLK; pi++)
        for (int pj = 0; pj < BLK; pj++)
            for (int pk = 0; pk < BLK; pk++) {
                double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, volt = 0.0;
                for (int h = 0; h < 8; h++) {
                    int c = child[h];
                    if (c < 0) continue;
                    int ix = (h >> 2) & 1, iy = (h >> 1) & 1, iz = h & 1;
                    const double *g = pool->pgeo + 6 * c;
                    double vol = g[3] * g[4] * g[5];
                    for (int di = 0; di < 2; di++)
                        for (int dj = 0; dj < 2; dj++)
                            for (int dk = 0; dk < 2; dk++) {
                                int fi = 2 * (pi - ix * (BLK / 2)) + di;
                                int fj = 2 * (pj - iy * (BLK / 2)) + dj;
                                int fk = 2 * (pk - iz * (BLK / 2)) + dk;
                                if (fi < 0 || fi >= BLK || fj < 0 || fj >= BLK || fk < 0 || fk >= BLK) continue;
                                int lf = lindx(fi, fj, fk);
                                volt += vol;
                                for (int v = 0; v < 8; v++) acc[v] += vol * UP(pool, c, v)[lf];
                            }
                }
                int l = lindx(pi, pj, pk);
                if (volt > 0.0) {
                    double inv = 1.0 / volt;
                    for (int v = 0; v < 8; v++) acc[v] *= inv;
                }
                for (int v = 0; v < 8; v++) UP(pool, p, v)[l] = acc[v];
                if (regrid_recover(P, pool, p, l)) return ORC_EDOMAIN;
            }
    orc_b_init(pool, p);
    return 0;
}

/* ======================================================================
 * L2: floors, patch::floors (grid.cpp:331-358)
 * ==================================================================== */
int orc_floors(const orc_params *P, orc_pool *pool, int p) {
    for (int i = 0; i < BLK; i++)
        for (int j = 0; j < BLK; j++)
            for (int k = 0; k < BLK; k++) {
                int l = lindx(i, j, k);
                double r = RP(pool, p)[l], th = TP(pool, p)[l];
                double D = UP(pool, p, 0)[l], tau = UP(pool, p, 4)[l];
                int bhl = !isfinite(D) || !isfinite(tau) || D <= 0.0 || tau <= 0.0;
                if (!bhl) {
                    cons U; prim pv;
                    get_cons(pool, p, l, &U);
                    memset(&pv, 0, sizeof(pv));
                    int ok = ctop_(P, &U, r, th, &pv, P->maxiter, P->tol, 0, 0);
                    if (ok < 0) return ORC_EDOMAIN;
                    bhl = !ok;
                    if (!bhl) {
                        int hl = !(pv.rho <= 0.0 || pv.eps <= 0.0);
                        if (hl) { put_prim(pool, p, l, &pv); put_derived(pool, p, l, &pv); }
                    }
                }
                prim fl;
                pvfs_(P, r, &fl);
                if (bhl || WP(pool, p, 0)[l] <= fl.rho) {
                    prim fo;
                    if (floor_reset_out(P, pool, p, l, &fo)) return ORC_EDOMAIN;
                    put_derived(pool, p, l, &fo);
                }
            }
    return 0;
}

/* ======================================================================
 * L3: analysis (data/quantitatives.cpp:17-247)
 * ==================================================================== */
typedef struct { double xc, yc, zc, r, th, dx, dy, dz, vol; prim W; cons U; } acell;
static void acell_get(const orc_pool *pool, int p, int i, int j, int k, acell *c) {
    const double *g = pool->pgeo + 6 * p;
    int l = lindx(i, j, k);
    c->dx = g[3]; c->dy = g[4]; c->dz = g[5];                 /* patch::cell_init, grid.cpp:154-157 */
    c->xc = g[0] + (i + 0.5) * g[3]; c->yc = g[1] + (j + 0.5) * g[4]; c->zc = g[2] + (k + 0.5) * g[5];
    c->vol = c->dx * c->dy * c->dz;
    c->r = RP(pool, p)[l]; c->th = TP(pool, p)[l];
    get_prim(pool, p, l, &c->W);
    const double *d = pool->Wd + (size_t)p * 4 * NC;
    c->W.lor = d[l]; c->W.p = d[NC + l]; c->W.h = d[2 * NC + l]; c->W.b2 = d[3 * NC + l];
    get_cons(pool, p, l, &c->U);
}
static double val_vr(const acell *c) { return (c->xc * c->W.v[0] + c->yc * c->W.v[1] + c->zc * c->W.v[2]) / c->r; }
static double val_vphi(const acell *c) {
    double R = sqrt(c->xc * c->xc + c->yc * c->yc);
    if (R < 1e-10) return 0.0;
    return (c->xc * c->W.v[1] - c->yc * c->W.v[0]) / (R * R);
}
static double val_Br(const acell *c) { return (c->xc * c->W.B[0] + c->yc * c->W.B[1] + c->zc * c->W.B[2]) / c->r; }
static double val_Bphi(const acell *c) {
    double R = sqrt(c->xc * c->xc + c->yc * c->yc);
    if (R < 1e-10) return 0.0;
    return (c->xc * c->W.B[1] - c->yc * c->W.B[0]) / (R * R);
}
/* the integrand of quantity q at cell c, sg = sqrt(-g) of the cell's metric */
static double aterm(int q, const acell *c, const mcomp *mc, double sg, double rho_min) {
    switch (q) {
    case ORC_Q_MASS: return c->U.D;                                               /* :83-87 */
    case ORC_Q_ENERGY: return c->U.tau + c->U.D;                                  /* :88-92 */
    case ORC_Q_LPOL: return c->xc * c->U.S[1] - c->yc * c->U.S[0];                /* :93-97 */
    case ORC_Q_MDOT: return -c->W.rho * c->W.lor * val_vr(c) * sg;                /* :99-103 */
    case ORC_Q_EDOT:                                                              /* :104-108 */
        return -((c->U.tau + c->U.D) * (mc->alpha * val_vr(c) -
                                        (mc->beta[0] * c->xc + mc->beta[1] * c->yc + mc->beta[2] * c->zc) / c->r));
    case ORC_Q_LDOT: {                                                            /* :109-114 */
        double w = c->W.rho * c->W.h + c->W.b2;
        return (w * c->W.lor * c->W.lor * val_vr(c) * val_vphi(c) - val_Br(c) - val_Bphi(c)) * sg;
    }
    case ORC_Q_PHIB: return fabs(val_Br(c)) * sg;                                 /* :115-119 */
    case ORC_Q_MAGE: return 0.5 * c->W.b2 * sg;                                   /* :125-129 */
    case ORC_Q_THERME: return c->W.rho * c->W.eps * sg;                           /* :130-134 */
    case ORC_Q_LBZ: {                                                             /* :135-155 */
        double Blow[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Blow[i] = mc->gam[i][j] * c->W.B[j];   /* assignment: j = 2 survives */
        double Bv = 0.0;
        for (int i = 0; i < 3; i++) Bv += Blow[i] * c->W.v[i];
        double bt = c->W.lor * Bv / mc->alpha;
        double br = (val_Br(c) + mc->alpha * bt * c->W.lor * val_vr(c)) / c->W.lor;
        double bt_ = mc->g[0][0] * bt + mc->g[0][1] * br + mc->g[0][3] * (val_Bphi(c) * c->W.lor);
        double ur = c->W.lor * val_vr(c);
        double ut_ = -mc->alpha * c->W.lor;
        return -(c->W.b2 * ur * ut_ - br * bt_) * sg;
    }
    case ORC_Q_PNUM: return c->W.p * sg;                                          /* :163-168 */
    case ORC_Q_PDEN: return 0.5 * c->W.b2 * sg;
    case ORC_Q_ASTRESS: case ORC_Q_ASTRESS_B:                                     /* :171-176 */
        if (c->W.rho < rho_min) return 0.0;
        return (c->W.rho * c->W.h * val_vr(c) * val_vphi(c) - val_Br(c) * val_Bphi(c)) * sg;
    case ORC_Q_APRESS: case ORC_Q_APRESS_B:                                       /* :177-180 */
        if (c->W.rho < rho_min) return 0.0;
        return (c->W.p + 0.5 * c->W.b2) * sg;
    case ORC_Q_MAXW:                                                              /* :184-187 */
        if (c->W.rho < rho_min) return 0.0;
        return -val_Br(c) * val_Bphi(c) * sg;
    case ORC_Q_REYN:                                                              /* :188-191 */
        if (c->W.rho < rho_min) return 0.0;
        return c->W.rho * c->W.h * c->W.lor * c->W.lor * val_vr(c) * val_vphi(c) * sg;
    case ORC_Q_HNUM: return fabs(c->zc) * c->W.rho * sg;                          /* :195-197 */
    case ORC_Q_HDEN: return c->W.rho * sg;
    default: return 0.0;
    }
}
/* analyser::vol_int (:44-59) and surf_int (:61-79, r_surf >= 0): the sum of
 * f * vol over the leaf patches' interior cells in quilt and i, j, k order */
static double aint(const orc_params *P, const orc_pool *pool, int q, double r_surf, double rho_min,
                   double *absint) {
    double integral = 0.0, a = 0.0;
    for (int p = 0; p < pool->npatch; p++) {
        if (!pool->leaf[p]) continue;
        for (int i = 0; i < BLK; i++)
            for (int j = 0; j < BLK; j++)
                for (int k = 0; k < BLK; k++) {
                    acell c;
                    acell_get(pool, p, i, j, k, &c);
                    if (r_surf >= 0.0) {
                        double shell = sqrt(c.dx * c.dx + c.dy * c.dy + c.dz * c.dz);
                        if (fabs(c.r - r_surf) > shell) continue;
                    }
                    mcomp mc;
                    mcomp_cell(P, c.r, c.th, &mc);
                    double f = aterm(q, &c, &mc, mc.sqrtdetg, rho_min) * c.vol;
                    integral += f;
                    a += fabs(f);
                }
    }
    if (absint) *absint = a;
    return integral;
}
void orc_analysis(const orc_params *P, const orc_pool *pool, double hrz, double rs, double rho_min_full,
                  double rho_min_bundle, double out[ORC_NQ], double out_abs[ORC_NQ]) {
    for (int q = 0; q < ORC_NQ; q++) {
        int surf = q == ORC_Q_MDOT || q == ORC_Q_EDOT || q == ORC_Q_LDOT || q == ORC_Q_PHIB || q == ORC_Q_LBZ ||
                   q == ORC_Q_HNUM || q == ORC_Q_HDEN;
        double rsurf = (q == ORC_Q_HNUM || q == ORC_Q_HDEN) ? rs : hrz;
        double rmin = (q == ORC_Q_ASTRESS_B || q == ORC_Q_APRESS_B) ? rho_min_bundle : rho_min_full;
        out[q] = aint(P, pool, q, surf ? rsurf : -1.0, rmin, out_abs ? out_abs + q : 0);
    }
}

/* ======================================================================
 * L3: integrator (solver/integrator.cpp)
 * ==================================================================== */
int orc_dtcomp(const orc_params *P, const orc_pool *pool, double cfl, double *dt) { /* :156-189 */
    double dt_min = 1.7976931348623157e308;
    int err = 0;
    for (int p = 0; p < pool->npatch; p++) {
        if (!pool->leaf[p]) continue;
        const double *g = pool->pgeo + 6 * p;
        const double ds[3] = {g[3], g[4], g[5]};
        for (int m = 0; m < BLK; m++)
            for (int n = 0; n < BLK; n++)
                for (int q = 0; q < BLK; q++) {
                    int l = lindx(m, n, q);
                    double cs2;
                    if (cs2f(P, WP(pool, p, 0)[l], WP(pool, p, 1)[l], &cs2)) { err = 1; continue; }
                    double cs = sqrt(cs2);
                    mcomp mc;
                    mcomp_cell(P, RP(pool, p)[l], TP(pool, p)[l], &mc);
                    for (int d = 0; d < 3; d++) {
                        double v = WP(pool, p, 2 + d)[l];
                        double ld_p = sabs(mc.alpha * (v + cs) - mc.beta[d]);
                        double ld_m = sabs(mc.alpha * (v - cs) - mc.beta[d]);
                        double vmax = smax(ld_p, ld_m);
                        if (vmax > 1e-14) dt_min = smin(dt_min, cfl * ds[d] / vmax);
                    }
                }
    }
    *dt = dt_min;
    return err ? ORC_EDOMAIN : 0;
}
int orc_prims(const orc_params *P, orc_pool *pool) {                 /* :288-310 */
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int p = 0; p < pool->npatch; p++) {
        if (!pool->leaf[p]) continue;
        for (int l = 0; l < NC; l++) {
            cons U; prim pv;
            get_cons(pool, p, l, &U);
            memset(&pv, 0, sizeof(pv));
            int ok = ctop_(P, &U, RP(pool, p)[l], TP(pool, p)[l], &pv, P->maxiter, P->tol, 0, 0);
            if (ok < 0) { err = 1; continue; }
            if (ok) put_prim(pool, p, l, &pv);
            else if (floor_reset(P, pool, p, l)) err = 1;
        }
    }
    return err ? ORC_EDOMAIN : 0;
}
int orc_update(const orc_params *P, orc_pool *pool, double dt, int stage) { /* :325-347 */
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int p = 0; p < pool->npatch; p++) {
        for (int i = 0; i < BLK; i++)
            for (int j = 0; j < BLK; j++)
                for (int k = 0; k < BLK; k++) {
                    int l = lindx(i, j, k);
                    double dv[8], sv[8], dU[8];
                    orc_div_flux(P, pool, p, i, j, k, dv);
                    if (orc_source(P, pool, p, i, j, k, sv)) { err = 1; continue; }
                    for (int v = 0; v < 8; v++) dU[v] = dv[v] + sv[v];
                    for (int v = 0; v < 8; v++) {
                        double u = UP(pool, p, v)[l];
                        if (stage == 0) {
                            DUP(pool, p, v)[l] = u;
                            UP(pool, p, v)[l] = u + dU[v] * dt;
                        } else {
                            UP(pool, p, v)[l] = (DUP(pool, p, v)[l] + u + dU[v] * dt) * 0.5;
                        }
                    }
                    mcomp mc;
                    mcomp_cell(P, RP(pool, p)[l], TP(pool, p)[l], &mc);
                    for (int d = 0; d < 3; d++) UP(pool, p, 5 + d)[l] = mc.sqrtdetg * WP(pool, p, 5 + d)[l];
                }
    }
    return err ? ORC_EDOMAIN : 0;
}
int orc_ghosts_all(const orc_params *P, orc_pool *pool) {
    for (int p = 0; p < pool->npatch; p++) {
        if (!pool->leaf[p]) continue;
        if (orc_ghosts(P, pool, p)) return ORC_EDOMAIN;
    }
    return 0;
}
int orc_fluxcomp_all(const orc_params *P, orc_pool *pool) {
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int p = 0; p < pool->npatch; p++)
        if (orc_fluxcomp(P, pool, p)) err = 1;
    return err ? ORC_EDOMAIN : 0;
}
void orc_ct_all(const orc_params *P, orc_pool *pool, double dt) {
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < pool->npatch; p++) {
        orc_emfcomp(pool, p);
        orc_bfupdate(pool, p, dt);
        orc_f2cb(P, pool, p);
    }
}
int orc_rkstg(const orc_params *P, orc_pool *pool, double dt, int stage) { /* :191-260 */
    if (orc_ghosts_all(P, pool)) return ORC_EDOMAIN;
    if (orc_prims(P, pool)) return ORC_EDOMAIN;
    if (orc_fluxcomp_all(P, pool)) return ORC_EDOMAIN;
    orc_ct_all(P, pool, dt);
    return orc_update(P, pool, dt, stage);
}
int orc_floors_all(const orc_params *P, orc_pool *pool) {
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int p = 0; p < pool->npatch; p++)
        if (orc_floors(P, pool, p)) err = 1;
    return err ? ORC_EDOMAIN : 0;
}
int orc_step(const orc_params *P, orc_pool *pool, double cfl, double *dt) { /* :262-275 */
    if (orc_dtcomp(P, pool, cfl, dt)) return ORC_EDOMAIN;
    if (orc_rkstg(P, pool, *dt, 0)) return ORC_EDOMAIN;
    if (orc_rkstg(P, pool, *dt, 1)) return ORC_EDOMAIN;
    return orc_floors_all(P, pool);
}

/* ======================================================================
 * batch helpers for the tests
 * ==================================================================== */
void orc_metric_batch(const orc_params *P, const double *r, const double *th, int64_t n,
                      double *mc) {
    for (int64_t q = 0; q < n; q++) orc_metric_comp(P, r[q], th[q], mc + q * ORC_NMC);
}
int orc_ptoc_batch(const orc_params *P, const double *W, const double *r, const double *th,
                   int64_t n, double *U, double *Wd) {
    int err = 0;
    for (int64_t q = 0; q < n; q++) {
        double w[8], u[8], wd[4];
        for (int v = 0; v < 8; v++) w[v] = W[v * n + q];
        if (orc_ptoc(P, w, r[q], th[q], u, wd)) { err = 1; continue; }
        for (int v = 0; v < 8; v++) U[v * n + q] = u[v];
        if (Wd) for (int v = 0; v < 4; v++) Wd[v * n + q] = wd[v];
    }
    return err ? ORC_EDOMAIN : 0;
}
void orc_ctop_batch(const orc_params *P, const double *U, const double *r, const double *th,
                    int64_t n, double *W, double *Wd, int32_t *status, int32_t *iters,
                    int32_t *path) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t q = 0; q < n; q++) {
        double u[8], w[8], wd[5];
        int32_t it = 0, pa = 0;
        for (int v = 0; v < 8; v++) u[v] = U[v * n + q];
        int rc = orc_ctop(P, u, r[q], th[q], w, wd, &it, &pa);
        for (int v = 0; v < 8; v++) W[v * n + q] = w[v];
        if (Wd) for (int v = 0; v < 5; v++) Wd[v * n + q] = wd[v];
        status[q] = rc;
        if (iters) iters[q] = it;
        if (path) path[q] = pa;
    }
}
void orc_hlld_batch(const orc_params *P, const double *WL, const double *WR, const double *UL,
                    const double *UR, const double *r, const double *th, int dim, int64_t n,
                    double *F, double *cts, int32_t *status) {
    for (int64_t q = 0; q < n; q++) {
        double wl[8], wr[8], ul[8], ur[8], f[8], c = 0;
        for (int v = 0; v < 8; v++) {
            wl[v] = WL[v * n + q]; wr[v] = WR[v * n + q];
            ul[v] = UL[v * n + q]; ur[v] = UR[v * n + q];
        }
        status[q] = orc_hlld(P, wl, wr, ul, ur, r[q], th[q], dim, f, &c);
        for (int v = 0; v < 8; v++) F[v * n + q] = f[v];
        cts[q] = c;
    }
}
/* face states of every flux face of every patch, [8][np*(17*16*16)] in the
 * loop order of patch::fluxcomp */
void orc_reconfp_all(const orc_params *P, const orc_pool *pool, int dim, int lim, double *L,
                     double *R) {
    const int64_t nfp = 17 * 16 * 16, n = nfp * pool->npatch;
    for (int p = 0; p < pool->npatch; p++) {
        int64_t q = (int64_t)p * nfp;
        int i0 = dim == 0 ? -1 : 0, j0 = dim == 1 ? -1 : 0, k0 = dim == 2 ? -1 : 0;
        for (int i = i0; i < BLK; i++)
            for (int j = j0; j < BLK; j++)
                for (int k = k0; k < BLK; k++, q++) {
                    double l8[8], r8[8];
                    orc_reconfp(P, pool, p, i, j, k, dim, lim, l8, r8);
                    for (int v = 0; v < 8; v++) { L[v * n + q] = l8[v]; R[v * n + q] = r8[v]; }
                }
    }
}
void orc_div_source_all(const orc_params *P, const orc_pool *pool, double *div, double *src) {
    for (int p = 0; p < pool->npatch; p++)
        for (int i = 0; i < BLK; i++)
            for (int j = 0; j < BLK; j++)
                for (int k = 0; k < BLK; k++) {
                    int l = lindx(i, j, k);
                    double d8[8], s8[8];
                    orc_div_flux(P, pool, p, i, j, k, d8);
                    if (orc_source(P, pool, p, i, j, k, s8)) for (int v = 0; v < 8; v++) s8[v] = NAN;
                    for (int v = 0; v < 8; v++) {
                        div[((size_t)p * 8 + v) * NC + l] = d8[v];
                        src[((size_t)p * 8 + v) * NC + l] = s8[v];
                    }
                }
}
void orc_maxdivb_all(const orc_pool *pool, double *out) {
    for (int p = 0; p < pool->npatch; p++) out[p] = orc_maxdivb(pool, p);
}
