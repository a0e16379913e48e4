/*
 * bh_fixed.c -- CPU oracle of the corrected ("fixed") scheme.  TEST
 * INFRASTRUCTURE ONLY: the tests, the smoke check and the bench's CPU leg
 * call it to check the CUDA kernels; nothing in the product path links it.
 *
 * A plain, sequential C restatement of textbook Valencia GRMHD in Cartesian
 * Kerr-Schild coordinates on the block layout of include/bhgpu.h
 * (bh_fx_grid): the step the reference's rk2integrator::step performs
 * (solver/integrator.cpp:191-275 of Fjoerde/black-hole-simulator,
 * src/fluid) with its defects corrected:
 *   - metric: g = eta + 2 H l (x) l, H = M r^3 / (r^4 + a^2 z^2), null
 *     covector l = (1, (r x + a y)/(r^2+a^2), (r y - a x)/(r^2+a^2), z/r)
 *     (in place of the (t,r,theta,phi) components on Cartesian vectors of
 *     physics/spacetime.cpp:20-54);
 *   - con2prim: Newton on Z = rho h W^2 with the exact derivative
 *     (Noble et al. 2006) (conserved.cpp:80-230 uses a wrong derivative);
 *   - fluxes: Valencia fluxes in each face's normal direction, HLL with
 *     fast magnetosonic speed bounds (grid.cpp:298,322 pass dim = 0);
 *   - sources: 1/2 T^{mu nu} d_j g_{mu nu} and
 *     alpha (T^{mu 0} d_mu ln alpha - T^{mu nu} Gamma^0_{mu nu});
 *   - CT: Heun-averaged face field (transport.cpp:38-58 takes dt twice).
 * Parity is "unpinned" against the reference by construction (the reference
 * has no such scheme); the restatement is pinned by the tests in
 * tests/test_fixed_oracle.py against physical identities computed
 * independently in numpy (T^{mu nu} projections, finite differences of the
 * metric, con2prim round trips, the Fishbone-Moncrief equilibrium).
 *
 * Only +, -, *, / and sqrt are used in the step, in the order of the device
 * code, so the device's FP64 build without contraction must equal this file
 * bit for bit (compiled with -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    double M, a, gamma, cfl, rho_floor, u_floor, sigma_max, W_max, r_exc, tol;
    int32_t maxiter, limiter, precision, reserved;
} fxo_params;

typedef struct {
    int32_t n, level;
    int64_t off;
    double x0[3];
    double dx;
} fxo_block;

enum { RHO = 0, PRS = 1, UT = 2, BB = 5 };
enum { CD = 0, CS = 1, CTAU = 4, CB = 5 };

static double dmin(double a, double b) { return b < a ? b : a; }
static double dmax(double a, double b) { return a < b ? b : a; }
static double dabs(double a) { return a < 0.0 ? -a : a; }

/* ---------------------------------------------------------------- metric */
typedef struct {
    double H, l[3], alpha, sqrtgam, beta[3], g[6], gi[6], r;
} ksm;

static int sy(int i, int j) {
    int a = i < j ? i : j, b = i < j ? j : i;
    return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

static double r2_of(double a, double x, double y, double z) {
    double a2 = a * a;
    double d = x * x + y * y + z * z - a2;
    return 0.5 * (d + sqrt(d * d + 4.0 * a2 * z * z));
}

static void metric(const fxo_params* P, double x, double y, double z, ksm* m) {
    double a = P->a, a2 = a * a;
    double r2 = r2_of(a, x, y, z);
    double r = sqrt(r2);
    double q = r2 * r2 + a2 * z * z;
    double H = q > 0.0 ? P->M * r * r2 / q : 0.0;
    double ir2a = 1.0 / (r2 + a2);
    m->r = r;
    m->H = H;
    m->l[0] = (r * x + a * y) * ir2a;
    m->l[1] = (r * y - a * x) * ir2a;
    m->l[2] = r > 0.0 ? z / r : 0.0;
    double h2 = 2.0 * H, f = 1.0 + h2;
    m->sqrtgam = sqrt(f);
    m->alpha = 1.0 / m->sqrtgam;
    double hf = h2 / f;
    for (int i = 0; i < 3; i++) m->beta[i] = hf * m->l[i];
    for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++) {
            double ll = m->l[i] * m->l[j];
            m->g[sy(i, j)] = (i == j ? 1.0 : 0.0) + h2 * ll;
            m->gi[sy(i, j)] = (i == j ? 1.0 : 0.0) - hf * ll;
        }
}

typedef struct {
    double dH[3], dl[3][3];
} ksd;

static void deriv(const fxo_params* P, double x, double y, double z, const ksm* m, ksd* d) {
    double a = P->a, a2 = a * a, r = m->r, r2 = r * r;
    double q = r2 * r2 + a2 * z * z;
    if (!(q > 0.0) || !(r > 0.0)) {
        memset(d, 0, sizeof *d);
        return;
    }
    double iq = 1.0 / q, r3 = r2 * r;
    double dr[3] = {x * r3 * iq, y * r3 * iq, z * r * (r2 + a2) * iq};
    double ir2a = 1.0 / (r2 + a2);
    for (int k = 0; k < 3; k++) {
        double dq = 4.0 * r3 * dr[k] + (k == 2 ? 2.0 * a2 * z : 0.0);
        d->dH[k] = P->M * (3.0 * r2 * dr[k] * q - r3 * dq) * iq * iq;
        double t = 2.0 * r * dr[k];
        d->dl[k][0] = (dr[k] * x + (k == 0 ? r : 0.0) + (k == 1 ? a : 0.0) - m->l[0] * t) * ir2a;
        d->dl[k][1] = (dr[k] * y + (k == 1 ? r : 0.0) - (k == 0 ? a : 0.0) - m->l[1] * t) * ir2a;
        d->dl[k][2] = ((k == 2 ? 1.0 : 0.0) - m->l[2] * dr[k]) / r;
    }
}

static void lower3(const double* g, const double* v, double* o) {
    o[0] = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
    o[1] = g[1] * v[0] + g[3] * v[1] + g[4] * v[2];
    o[2] = g[2] * v[0] + g[4] * v[1] + g[5] * v[2];
}

/* ------------------------------------------------------- prim -> cons */
typedef struct {
    double W, iW, rhoh, v[3], vl[3], Bl[3], B2, Bv, b2, rhohW2, ptot;
} drv;

static void derive(const ksm* m, double gamma, const double* w, drv* d) {
    double ut[3] = {w[UT], w[UT + 1], w[UT + 2]};
    double B[3] = {w[BB], w[BB + 1], w[BB + 2]};
    double utl[3];
    lower3(m->g, ut, utl);
    double u2 = utl[0] * ut[0] + utl[1] * ut[1] + utl[2] * ut[2];
    d->W = sqrt(1.0 + u2);
    double iW = 1.0 / d->W;
    d->iW = iW;
    for (int i = 0; i < 3; i++) {
        d->v[i] = ut[i] * iW;
        d->vl[i] = utl[i] * iW;
    }
    lower3(m->g, B, d->Bl);
    d->B2 = d->Bl[0] * B[0] + d->Bl[1] * B[1] + d->Bl[2] * B[2];
    d->Bv = d->Bl[0] * d->v[0] + d->Bl[1] * d->v[1] + d->Bl[2] * d->v[2];
    d->b2 = d->B2 * iW * iW + d->Bv * d->Bv;
    double rhoh = w[RHO] + gamma / (gamma - 1.0) * w[PRS];
    d->rhoh = rhoh;
    d->rhohW2 = rhoh * d->W * d->W;
    d->ptot = w[PRS] + 0.5 * d->b2;
}

static void p2c(const ksm* m, const double* w, const drv* d, double* u) {
    double sg = m->sqrtgam;
    double v2 = 1.0 - d->iW * d->iW;
    u[CD] = sg * w[RHO] * d->W;
    double e = d->rhohW2 + d->B2;
    for (int i = 0; i < 3; i++) u[CS + i] = sg * (e * d->vl[i] - d->Bv * d->Bl[i]);
    double E = d->rhohW2 - w[PRS] + 0.5 * d->B2 * (1.0 + v2) - 0.5 * d->Bv * d->Bv;
    u[CTAU] = sg * E - u[CD];
    for (int i = 0; i < 3; i++) u[CB + i] = sg * w[BB + i];
}

static void pflux(const ksm* m, int dd, const double* w, const drv* d, const double* u, double* F) {
    double vt = m->alpha * d->v[dd] - m->beta[dd];
    double ag = m->alpha * m->sqrtgam;
    double iW2 = d->iW * d->iW;
    double Bd = w[BB + dd];
    F[CD] = u[CD] * vt;
    for (int j = 0; j < 3; j++) {
        double bjB = (d->Bl[j] * iW2 + d->Bv * d->vl[j]) * Bd;
        F[CS + j] = u[CS + j] * vt + ag * ((j == dd ? d->ptot : 0.0) - bjB);
    }
    F[CTAU] = u[CTAU] * vt + ag * (d->ptot * d->v[dd] - d->Bv * Bd);
    for (int k = 0; k < 3; k++) {
        double vtk = m->alpha * d->v[k] - m->beta[k];
        F[CB + k] = k == dd ? 0.0 : m->sqrtgam * (w[BB + k] * vt - Bd * vtk);
    }
}

static void speeds(const ksm* m, double gamma, int dd, const double* w, const drv* d, double* lm, double* lp) {
    double rhoh = d->rhoh;
    double c2 = (gamma * w[PRS] + d->b2) / (rhoh + d->b2);
    c2 = dmin(dmax(c2, 0.0), 1.0);
    double v2 = 1.0 - d->iW * d->iW;
    double vd = d->v[dd];
    double gdd = m->gi[dd == 0 ? 0 : (dd == 1 ? 3 : 5)];
    double den = 1.0 / (1.0 - v2 * c2);
    double disc = (1.0 - v2) * (gdd * (1.0 - v2 * c2) - vd * vd * (1.0 - c2));
    double rt = sqrt(dmax(c2 * disc, 0.0));
    double base = vd * (1.0 - c2);
    *lm = m->alpha * (base - rt) * den - m->beta[dd];
    *lp = m->alpha * (base + rt) * den - m->beta[dd];
}

/* ------------------------------------------------------------------ PLM */
enum { LIM_MINMOD = 0, LIM_VANLEER = 1, LIM_MC = 2, LIM_PPM = 3 };
/* The face value of cell w0 toward its neighbour wn across the face, wf
 * its other neighbour: w0 + sigma/2 with sigma the limited slope of
 * (w0 - wf, wn - w0) (minmod, van Leer, MC; zero at an extremum).  At MC's
 * bound sigma = 2 (wn - w0) the value is wn itself, and van Leer's with
 * |wn - w0| < |w0 - wf| is formed from wn, so no difference of the two
 * cells cancels against w0 (the device kernels' plm_value, same
 * operations). */
static double face_value(double wf, double w0, double wn, int lim) {
    double df = w0 - wf, dn = wn - w0;
    if (df * dn <= 0.0) return w0;
    double af = dabs(df), an = dabs(dn);
    if (lim == LIM_VANLEER) {
        double q = df + dn;
        return an < af ? wn - dn * dn / q : w0 + df * dn / q;
    }
    if (lim == LIM_MC) { /* sigma/2 = s min((af + an)/4, af, an) */
        double t = dmin(0.25 * (af + an), af);
        if (an < t) return wn;
        return w0 + (dn > 0.0 ? t : -t);
    }
    double t = 0.5 * dmin(af, an);
    return w0 + (dn > 0.0 ? t : -t);
}

/* PPM (Colella & Woodward 1984, J. Comput. Phys. 54, 174: eqs. 1.6-1.8 and
 * 1.10, without contact steepening or flattening): the face between cells
 * a[2] and a[3] of a[0..5] (cells p-3 .. p+2 for the face p-1/2).  Limited
 * slopes of cells p-2 .. p+1, the fourth-order interface values a_{p-3/2},
 * a_{p-1/2}, a_{p+1/2}, and the monotonised parabolas of cells p-1 (its
 * right value is L) and p (its left value is R). */
static double ppm_dm(double am, double a0, double ap) {
    double dl = a0 - am, dr = ap - a0;
    if (dl * dr <= 0.0) return 0.0;
    double da = 0.5 * (ap - am);
    double m = dmin(dabs(da), 2.0 * dmin(dabs(dl), dabs(dr)));
    return da > 0.0 ? m : -m;
}
static void ppm_parabola(double a, double* aL, double* aR) {
    double l = *aL, r = *aR;
    if ((r - a) * (a - l) <= 0.0) {
        l = a;
        r = a;
    } else {
        double d = r - l, c = a - 0.5 * (l + r), d2 = d * d * (1.0 / 6.0);
        if (d * c > d2)
            l = 3.0 * a - 2.0 * r;
        else if (-d2 > d * c)
            r = 3.0 * a - 2.0 * l;
    }
    *aL = l;
    *aR = r;
}
static void ppm_face(const double* a, double* L, double* R) {
    double dm[4];
    for (int q = 0; q < 4; q++) dm[q] = ppm_dm(a[q], a[q + 1], a[q + 2]);   /* cells p-2 .. p+1 */
    double f[3];   /* a_{p-3/2}, a_{p-1/2}, a_{p+1/2} */
    for (int q = 0; q < 3; q++) f[q] = a[q + 1] + 0.5 * (a[q + 2] - a[q + 1]) - (1.0 / 6.0) * (dm[q + 1] - dm[q]);
    double lL = f[0], lR = f[1], rL = f[1], rR = f[2];
    ppm_parabola(a[2], &lL, &lR);
    ppm_parabola(a[3], &rL, &rR);
    *L = lR;
    *R = rL;
}

static double hll(const ksm* m, double gamma, int dd, const double* wL, const double* wR, double* F) {
    drv dL, dR;
    derive(m, gamma, wL, &dL);
    derive(m, gamma, wR, &dR);
    double uL[8], uR[8], FL[8], FR[8];
    p2c(m, wL, &dL, uL);
    p2c(m, wR, &dR, uR);
    pflux(m, dd, wL, &dL, uL, FL);
    pflux(m, dd, wR, &dR, uR, FR);
    double lmL, lpL, lmR, lpR;
    speeds(m, gamma, dd, wL, &dL, &lmL, &lpL);
    speeds(m, gamma, dd, wR, &dR, &lmR, &lpR);
    double sl = dmin(dmin(lmL, lmR), 0.0);
    double sr = dmax(dmax(lpL, lpR), 0.0);
    double ds = sr - sl;
    if (ds > 0.0) {
        double ids = 1.0 / ds, ss = sr * sl;
        for (int v = 0; v < 8; v++) F[v] = (sr * FL[v] - sl * FR[v] + ss * (uR[v] - uL[v])) * ids;
    } else {
        for (int v = 0; v < 8; v++) F[v] = 0.5 * (FL[v] + FR[v]);
    }
    F[CB + dd] = 0.0;
    return dmax(sr, -sl);
}

/* --------------------------------------------------------------- source */
static void source(const ksm* m, const ksd* dk, double gamma, const double* w, double* S) {
    drv d;
    derive(m, gamma, w, &d);
    double H = m->H;
    double l[4] = {1.0, m->l[0], m->l[1], m->l[2]};
    double ia = 1.0 / m->alpha;
    double u[4], b[4];
    u[0] = d.W * ia;
    for (int i = 0; i < 3; i++) u[1 + i] = w[UT + i] - u[0] * m->beta[i];
    b[0] = d.W * d.Bv * ia;
    double iW = 1.0 / d.W;
    for (int i = 0; i < 3; i++) b[1 + i] = (w[BB + i] + m->alpha * b[0] * u[1 + i]) * iW;
    double e = d.rhoh + d.b2;
    double lu[4] = {-1.0, l[1], l[2], l[3]};
    double T[4][4];
    for (int mu = 0; mu < 4; mu++)
        for (int nu = mu; nu < 4; nu++) {
            double eta = mu == nu ? (mu == 0 ? -1.0 : 1.0) : 0.0;
            double gi = eta - 2.0 * H * lu[mu] * lu[nu];
            T[mu][nu] = e * u[mu] * u[nu] + d.ptot * gi - b[mu] * b[nu];
            T[nu][mu] = T[mu][nu];
        }
    double Tl[4];
    for (int mu = 0; mu < 4; mu++) Tl[mu] = T[mu][0] * l[0] + T[mu][1] * l[1] + T[mu][2] * l[2] + T[mu][3] * l[3];
    double Tll = Tl[0] * l[0] + Tl[1] * l[1] + Tl[2] * l[2] + Tl[3] * l[3];
    double s[3];
    for (int j = 0; j < 3; j++)
        s[j] = dk->dH[j] * Tll + 2.0 * H * (Tl[1] * dk->dl[j][0] + Tl[2] * dk->dl[j][1] + Tl[3] * dk->dl[j][2]);
    double A = Tl[1] * dk->dH[0] + Tl[2] * dk->dH[1] + Tl[3] * dk->dH[2];
    double lB = 0.0, Cc = 0.0;
    for (int i = 0; i < 3; i++) {
        double Bi = Tl[1] * dk->dl[0][i] + Tl[2] * dk->dl[1][i] + Tl[3] * dk->dl[2][i];
        lB += l[1 + i] * Bi;
        Cc += T[1][1 + i] * dk->dl[0][i] + T[2][1 + i] * dk->dl[1][i] + T[3][1 + i] * dk->dl[2][i];
    }
    double ls = l[1] * s[0] + l[2] * s[1] + l[3] * s[2];
    double TG = -2.0 * A + 4.0 * H * H * lB - 2.0 * H * Cc - 2.0 * H * ls;
    double a2 = m->alpha * m->alpha;
    double T0dH = T[0][1] * dk->dH[0] + T[0][2] * dk->dH[1] + T[0][3] * dk->dH[2];
    double ag = m->alpha * m->sqrtgam;
    S[CD] = 0.0;
    for (int j = 0; j < 3; j++) S[CS + j] = ag * s[j];
    S[CTAU] = ag * m->alpha * (-a2 * T0dH - TG);
    for (int k = 0; k < 3; k++) S[CB + k] = 0.0;
}

/* ------------------------------------------------- floors and con2prim */
static void floor_state(const fxo_params* P, double r, double* rho, double* p) {
    double re = r > 1.0 ? r : 1.0;
    double s = sqrt(re);
    double ir = 1.0 / (re * re * s); /* r^-5/2 */
    *rho = P->rho_floor * re * ir;
    *p = (P->gamma - 1.0) * P->u_floor * ir;
}

typedef struct {
    double D, S2, B2, SB2, B4, E, gf, v2max;
} c2pq;

static void c2p_eval(const c2pq* q, double Z, double* f, double* df, double* v2, int* clamped) {
    double iZ = 1.0 / Z, ZB = Z + q->B2, iZB = 1.0 / ZB;
    double iZB2 = iZB * iZB, iZ2 = iZ * iZ;
    *v2 = q->S2 * iZB2 + q->SB2 * (q->B2 + 2.0 * Z) * iZ2 * iZB2;
    *clamped = *v2 > q->v2max;
    if (*clamped) *v2 = q->v2max;
    double W2i = 1.0 - *v2, Wi = sqrt(W2i);
    double p = q->gf * (Z * W2i - q->D * Wi);
    *f = Z - p + 0.5 * (1.0 + *v2) * q->B2 - 0.5 * q->SB2 * iZ2 - q->E;
    double dv2 = *clamped ? 0.0
                          : -2.0 * q->S2 * iZB2 * iZB -
                                2.0 * q->SB2 * (3.0 * Z * Z + 3.0 * Z * q->B2 + q->B4) * iZ2 * iZ * iZB2 * iZB;
    double dp = q->gf * (W2i - Z * dv2 + 0.5 * q->D * dv2 / Wi);
    *df = 1.0 - dp + 0.5 * q->B2 * dv2 + q->SB2 * iZ2 * iZ;
}

/* Newton on Z = rho h W^2 from the previous primitives (phase 1); where it
 * reaches the Lorentz-factor ceiling or leaves Z > 0, a bracket [0, Z_hi]
 * narrowed by safeguarded Newton / bisection (phase 2) */
static int c2p(const fxo_params* P, const ksm* m, const double* U, const double* B, const double* wo, double* w,
               int* iters) {
    double gm = P->gamma;
    double isg = 1.0 / m->sqrtgam;
    c2pq q;
    q.gf = (gm - 1.0) / gm;
    q.D = U[CD] * isg;
    double tau = U[CTAU] * isg;
    double S[3] = {U[CS] * isg, U[CS + 1] * isg, U[CS + 2] * isg};
    double Su[3];
    lower3(m->gi, S, Su);
    double Bl[3];
    lower3(m->g, B, Bl);
    q.S2 = Su[0] * S[0] + Su[1] * S[1] + Su[2] * S[2];
    q.B2 = Bl[0] * B[0] + Bl[1] * B[1] + Bl[2] * B[2];
    double SB = S[0] * B[0] + S[1] * B[1] + S[2] * B[2];
    q.SB2 = SB * SB;
    q.B4 = q.B2 * q.B2;
    q.E = tau + q.D;
    q.v2max = 1.0 - 1.0 / (P->W_max * P->W_max);
    double uto[3] = {wo[UT], wo[UT + 1], wo[UT + 2]}, utl[3];
    lower3(m->g, uto, utl);
    double W2o = 1.0 + utl[0] * uto[0] + utl[1] * uto[1] + utl[2] * uto[2];
    double Z = (wo[RHO] + gm / (gm - 1.0) * wo[PRS]) * W2o;
    if (!(Z > 0.0) || !(Z < 1e300)) Z = q.E > q.D ? q.E : q.D;
    int it = 0, ok = 0;
    double f = 0.0, df = 0.0, v2 = 0.0;
    int clamped = 0;
    /* a step of at most sqrt(tol) Z is the last: Newton's quadratic
     * convergence leaves an error of order tol Z after it */
    double qtol = sqrt(P->tol);
    for (; it < P->maxiter; it++) {
        c2p_eval(&q, Z, &f, &df, &v2, &clamped);
        if (clamped || !(df != 0.0)) break;
        double Zn = Z - f / df;
        if (!(Zn > 0.0)) break;
        double err = dabs(Zn - Z);
        Z = Zn;
        if (err <= qtol * Z) {
            ok = 1;
            it++;
            break;
        }
    }
    if (!ok) {
        double lo = 0.0, hi = Z > q.E ? Z : q.E;
        if (!(hi > 0.0)) hi = 1.0;
        int k = 0;
        for (; k < 64; k++) {
            c2p_eval(&q, hi, &f, &df, &v2, &clamped);
            it++;
            if (f > 0.0) break;
            lo = hi;
            hi = 2.0 * hi;
        }
        if (f > 0.0 && hi < 1e300) {
            Z = hi;
            for (k = 0; k < 2 * P->maxiter + 60; k++) {
                double Zn = (df > 0.0) ? Z - f / df : 0.5 * (lo + hi);
                if (!(Zn > lo && Zn < hi)) Zn = 0.5 * (lo + hi);
                double err = dabs(Zn - Z);
                Z = Zn;
                if (err <= P->tol * Z) {
                    ok = 1;
                    break;
                }
                c2p_eval(&q, Z, &f, &df, &v2, &clamped);
                it++;
                if (f > 0.0) hi = Z; else lo = Z;
            }
        }
    }
    *iters = it;
    if (!ok) return 1;
    double iZ = 1.0 / Z, ZB = Z + q.B2, iZB = 1.0 / ZB;
    v2 = q.S2 * iZB * iZB + q.SB2 * (q.B2 + 2.0 * Z) * iZ * iZ * iZB * iZB;
    if (!(v2 < q.v2max)) v2 = q.v2max;
    double W2i = 1.0 - v2, Wi = sqrt(W2i);
    double Wl = 1.0 / Wi;
    double rho = q.D * Wi;
    double p = q.gf * (Z * W2i - rho);
    double vl[3], vu[3];
    for (int i = 0; i < 3; i++) vl[i] = (S[i] + SB * iZ * Bl[i]) * iZB;
    lower3(m->gi, vl, vu);
    w[RHO] = rho;
    w[PRS] = p;
    for (int i = 0; i < 3; i++) {
        w[UT + i] = Wl * vu[i];
        w[BB + i] = B[i];
    }
    if (!(rho > 0.0) || !(p == p) || !(Wl == Wl)) return 2;
    return 0;
}

static int floors(const fxo_params* P, const ksm* m, double* w) {
    double rf, pf;
    floor_state(P, m->r, &rf, &pf);
    int changed = 0;
    if (m->r < P->r_exc) {
        w[RHO] = rf;
        w[PRS] = pf;
        w[UT] = w[UT + 1] = w[UT + 2] = 0.0;
        return 1;
    }
    double ut[3] = {w[UT], w[UT + 1], w[UT + 2]}, utl[3];
    lower3(m->g, ut, utl);
    double u2 = utl[0] * ut[0] + utl[1] * ut[1] + utl[2] * ut[2];
    double umax2 = P->W_max * P->W_max - 1.0;
    if (u2 > umax2) {
        double s = sqrt(umax2 / u2);
        for (int i = 0; i < 3; i++) w[UT + i] = ut[i] * s;
        u2 = umax2;
        changed = 1;
    }
    double W2 = 1.0 + u2, iW2 = 1.0 / W2;
    double B[3] = {w[BB], w[BB + 1], w[BB + 2]}, Bl[3];
    lower3(m->g, B, Bl);
    double B2 = Bl[0] * B[0] + Bl[1] * B[1] + Bl[2] * B[2];
    double Bu2 = Bl[0] * w[UT] + Bl[1] * w[UT + 1] + Bl[2] * w[UT + 2]; /* W (B.v) */
    double b2 = (B2 + Bu2 * Bu2) * iW2;
    double rs = b2 * (1.0 / P->sigma_max);
    if (rs > rf) rf = rs;
    if (!(w[RHO] >= rf)) {
        w[RHO] = rf;
        changed = 1;
    }
    if (!(w[PRS] >= pf)) {
        w[PRS] = pf;
        changed = 1;
    }
    return changed;
}

static double cell_dt(const fxo_params* P, const ksm* m, const double* w, double dx) {
    drv d;
    derive(m, P->gamma, w, &d);
    double best = 1e300;
    for (int dd = 0; dd < 3; dd++) {
        double lm, lp;
        speeds(m, P->gamma, dd, w, &d, &lm, &lp);
        double c = dmax(dabs(lm), dabs(lp));
        if (c > 0.0) best = dmin(best, dx / c);
    }
    return best;
}

/* ---------------------------------------------------------------- grid */
typedef struct {
    const fxo_params* P;
    int32_t nblock;
    const fxo_block* blk;
    const int32_t* nbr;
    int64_t N;
    double *U, *U1, *W, *Bf, *Bf1, *F, *dt;
    int32_t* count;
} fxo_grid;

/* every block is stored as a box of GB ghost layers (and one more cell per
 * axis above) per array: index ((i+GB) S + (j+GB)) S + (k+GB), S = n+2GB+1 */
#define GB 3
#define SP(n) ((n) + 2 * GB + 1)
static int64_t bx(const fxo_block* b, int i, int j, int k) {
    int64_t S = SP(b->n);
    return b->off + ((int64_t)(i + GB) * S + (j + GB)) * S + (k + GB);
}
static void centre(const fxo_block* b, int i, int j, int k, double* x) {
    x[0] = b->x0[0] + (i + 0.5) * b->dx;
    x[1] = b->x0[1] + (j + 0.5) * b->dx;
    x[2] = b->x0[2] + (k + 0.5) * b->dx;
}

static void prims_cell(const fxo_grid* G, const fxo_block* B, int i, int j, int k, int stage, double* dtmin,
                       int with_dt) {
    const fxo_params* P = G->P;
    int64_t N = G->N, c = bx(B, i, j, k);
    int si = SP(B->n) * SP(B->n), sj = SP(B->n);
    double* U = stage ? G->U1 : G->U;
    const double* Bf = stage ? G->Bf1 : G->Bf;
    double x[3];
    centre(B, i, j, k, x);
    ksm m;
    metric(P, x[0], x[1], x[2], &m);
    double Bt[3] = {0.5 * (Bf[c] + Bf[c + si]), 0.5 * (Bf[N + c] + Bf[N + c + sj]),
                    0.5 * (Bf[2 * N + c] + Bf[2 * N + c + 1])};
    double isg = 1.0 / m.sqrtgam;
    double Bc[3] = {Bt[0] * isg, Bt[1] * isg, Bt[2] * isg};
    double u[8], wo[8], w[8];
    for (int v = 0; v < 5; v++) u[v] = U[v * N + c];
    for (int v = 0; v < 5; v++) wo[v] = G->W[v * N + c];
    int iters = 0;
    int st = c2p(P, &m, u, Bc, wo, w, &iters);
    int rewrite = 0;
    if (st != 0) {
        for (int v = 0; v < 5; v++) w[v] = wo[v];
        for (int d = 0; d < 3; d++) w[BB + d] = Bc[d];
        G->count[0]++;
        rewrite = 1;
    }
    if (floors(P, &m, w)) {
        rewrite = 1;
        G->count[1]++;
    }
    if (rewrite) {
        drv d;
        derive(&m, P->gamma, w, &d);
        p2c(&m, w, &d, u);
        for (int v = 0; v < 5; v++) U[v * N + c] = u[v];
    }
    for (int d = 0; d < 3; d++) U[(5 + d) * N + c] = Bt[d];
    for (int v = 0; v < 8; v++) G->W[v * N + c] = w[v];
    if (with_dt) {
        double t = cell_dt(P, &m, w, B->dx);
        if (t < *dtmin) *dtmin = t;
    }
}

void fxo_prims(const fxo_params* P, int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, double* U,
               double* U1, double* W, double* Bf, double* Bf1, double* F, double* dt, int32_t* count, int stage,
               int with_dt) {
    double dtmin = INFINITY;
    int32_t c0 = 0, c1 = 0;
    for (int b = 0; b < nblock; b++) {
        int n = blk[b].n;
#pragma omp parallel for schedule(static) reduction(min : dtmin) reduction(+ : c0, c1)
        for (int i = 0; i < n; i++) {
            int32_t cnt[4] = {0, 0, 0, 0};
            fxo_grid G = {P, nblock, blk, nbr, N, U, U1, W, Bf, Bf1, F, dt, cnt};
            double tmin = INFINITY;
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) prims_cell(&G, &blk[b], i, j, k, stage, &tmin, with_dt);
            if (tmin < dtmin) dtmin = tmin;
            c0 += cnt[0];
            c1 += cnt[1];
        }
    }
    count[0] += c0;
    count[1] += c1;
    if (with_dt) dt[0] = dtmin;
}

/* ghost fill: the source of ghost position c[] (cell: fdim = -1) */
static int gsrc(const int32_t* nbr, int b, int n, int fdim, int* c) {
    int o[3];
    const int32_t* nb = nbr + (int64_t)b * 27;
    for (int d = 0; d < 3; d++) {
        int hi = d == fdim ? n : n - 1;
        o[d] = c[d] < 0 ? -1 : (c[d] > hi ? 1 : 0);
        if (o[d] != 0) {
            int face_nb = nb[d == 0 ? (o[d] + 1) * 9 + 4 : d == 1 ? 9 + (o[d] + 1) * 3 + 1 : 12 + o[d] + 1];
            if (face_nb < 0) {
                c[d] = c[d] < 0 ? 0 : hi;
                o[d] = 0;
            }
        }
    }
    int s = nb[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)];
    if (s < 0) s = b;
    for (int d = 0; d < 3; d++) c[d] -= o[d] * n;
    return s;
}

/* minmod of the two differences around b */
static double mm_slope(double a, double b, double c) {
    double l = b - a, r = c - b;
    if (l * r <= 0.0) return 0.0;
    return dabs(l) < dabs(r) ? l : r;
}

/* Ghost fill over blocks of several levels (equal cubes, levels one apart
 * at most): a same-level image is copied, a finer one averaged (8 cells or
 * 4 faces), a coarser one interpolated (the covering cell plus a quarter of
 * its minmod slope per direction; a face takes the coarse face it lies on
 * or the mean of the two it lies between).  Pass 0: copies and
 * restrictions; pass l: prolongations into level-l blocks. */
void fxo_ghost_pass(int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, double* W, double* Bf,
                    double* Bf1, int stage, int pass, int depth) {
    double* F = stage ? Bf1 : Bf;
    {
        for (int b = 0; b < nblock; b++) {
            int n = blk[b].n;
            if (pass > 0 && blk[b].level != pass) continue;
#pragma omp parallel for schedule(static)
            for (int i = -depth; i < n + depth; i++)
                for (int j = -depth; j < n + depth; j++)
                    for (int k = -depth; k < n + depth; k++) {
                        if (i >= 0 && i < n && j >= 0 && j < n && k >= 0 && k < n) continue;
                        int64_t c = bx(&blk[b], i, j, k);
                        int q[3] = {i, j, k};
                        int s = gsrc(nbr, b, n, -1, q);
                        const fxo_block* S = &blk[s];
                        int kind = S->n == n ? 0 : (S->n > n ? 1 : 2);
                        if ((kind == 2) == (pass > 0)) {
                            if (kind == 0) {
                                int64_t sc = bx(S, q[0], q[1], q[2]);
                                for (int v = 0; v < 8; v++) W[v * N + c] = W[v * N + sc];
                            } else if (kind == 1) {
                                for (int v = 0; v < 8; v++) {
                                    double sum = 0.0;
                                    for (int a = 0; a < 2; a++)
                                        for (int e = 0; e < 2; e++)
                                            for (int r = 0; r < 2; r++)
                                                sum += W[v * N + bx(S, 2 * q[0] + a, 2 * q[1] + e, 2 * q[2] + r)];
                                    W[v * N + c] = 0.125 * sum;
                                }
                            } else {
                                int ic = q[0] >> 1, jc = q[1] >> 1, kc = q[2] >> 1;
                                double gx = (q[0] & 1) ? 0.25 : -0.25, gy = (q[1] & 1) ? 0.25 : -0.25,
                                       gz = (q[2] & 1) ? 0.25 : -0.25;
                                for (int v = 0; v < 8; v++) {
                                    const double* Wv = W + v * N;
                                    double w0 = Wv[bx(S, ic, jc, kc)];
                                    double sx = mm_slope(Wv[bx(S, ic - 1, jc, kc)], w0, Wv[bx(S, ic + 1, jc, kc)]);
                                    double sy = mm_slope(Wv[bx(S, ic, jc - 1, kc)], w0, Wv[bx(S, ic, jc + 1, kc)]);
                                    double sz = mm_slope(Wv[bx(S, ic, jc, kc - 1)], w0, Wv[bx(S, ic, jc, kc + 1)]);
                                    W[v * N + c] = w0 + gx * sx + gy * sy + gz * sz;
                                }
                            }
                        }
                        for (int d = 0; d < 3; d++) {
                            int cc[3] = {i, j, k};
                            if (cc[d] < 0 || cc[d] > n) continue;
                            int need = 1;
                            for (int e = 0; e < 3; e++)
                                if (e != d && (cc[e] < -1 || cc[e] > n)) need = 0;
                            if (!need) continue;
                            int t[3] = {i, j, k};
                            int fs = gsrc(nbr, b, n, d, t);
                            const fxo_block* T = &blk[fs];
                            int fk = T->n == n ? 0 : (T->n > n ? 1 : 2);
                            if ((fk == 2) != (pass > 0)) continue;
                            const double* Bd = F + d * N;
                            double v;
                            if (fk == 0) {
                                v = Bd[bx(T, t[0], t[1], t[2])];
                            } else if (fk == 1) {
                                int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                                double sum = 0.0;
                                for (int a = 0; a < 2; a++)
                                    for (int e = 0; e < 2; e++) {
                                        int g[3] = {2 * t[0], 2 * t[1], 2 * t[2]};
                                        g[t1] += a;
                                        g[t2] += e;
                                        sum += Bd[bx(T, g[0], g[1], g[2])];
                                    }
                                v = 0.25 * sum;
                            } else {
                                int g[3] = {t[0] >> 1, t[1] >> 1, t[2] >> 1};
                                if (t[d] & 1) {
                                    int h[3] = {g[0], g[1], g[2]};
                                    h[d] += 1;
                                    v = 0.5 * (Bd[bx(T, g[0], g[1], g[2])] + Bd[bx(T, h[0], h[1], h[2])]);
                                } else {
                                    v = Bd[bx(T, g[0], g[1], g[2])];
                                }
                            }
                            F[d * N + c] = v;
                        }
                    }
        }
    }
}

void fxo_ghosts(int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, double* W, double* Bf,
                double* Bf1, int stage, int maxlevel, int depth) {
    for (int pass = 0; pass <= maxlevel; pass++) fxo_ghost_pass(nblock, blk, nbr, N, W, Bf, Bf1, stage, pass, depth);
}

static void face(const fxo_params* P, const fxo_block* B, int64_t N, const double* W, const double* Bfs, double* F,
                 int i, int j, int k, int d) {
    int64_t c = bx(B, i, j, k);
    int st = d == 0 ? SP(B->n) * SP(B->n) : (d == 1 ? SP(B->n) : 1);
    double x[3];
    centre(B, i, j, k, x);
    x[d] -= 0.5 * B->dx;
    ksm m;
    metric(P, x[0], x[1], x[2], &m);
    double wL[8], wR[8];
    for (int v = 0; v < 8; v++) {
        if (v == BB + d) continue;
        if (P->limiter == LIM_PPM) {
            double a6[6];
            for (int o = 0; o < 6; o++) a6[o] = W[v * N + c + (o - 3) * st];
            ppm_face(a6, &wL[v], &wR[v]);
            continue;
        }
        double a = W[v * N + c - 2 * st], b = W[v * N + c - st], cc = W[v * N + c], dd = W[v * N + c + st];
        wL[v] = face_value(a, b, cc, P->limiter);
        wR[v] = face_value(dd, cc, b, P->limiter);
    }
    double Bn = Bfs[d * N + c] * m.alpha; /* alpha = 1 / sqrt(gamma) */
    wL[BB + d] = Bn;
    wR[BB + d] = Bn;
    double Fo[8];
    hll(&m, P->gamma, d, wL, wR, Fo);
    for (int v = 0; v < 8; v++) F[((int64_t)d * 8 + v) * N + c] = Fo[v];
}

void fxo_fluxes(const fxo_params* P, int32_t nblock, const fxo_block* blk, int64_t N, const double* W,
                const double* Bf, const double* Bf1, double* F, int stage) {
    const double* Bfs = stage ? Bf1 : Bf;
    for (int b = 0; b < nblock; b++) {
        int n = blk[b].n;
#pragma omp parallel for schedule(static)
        for (int i = -1; i <= n; i++)
            for (int j = -1; j <= n; j++)
                for (int k = -1; k <= n; k++) {
                    if (i >= 0) face(P, &blk[b], N, W, Bfs, F, i, j, k, 0);
                    if (j >= 0) face(P, &blk[b], N, W, Bfs, F, i, j, k, 1);
                    if (k >= 0) face(P, &blk[b], N, W, Bfs, F, i, j, k, 2);
                }
    }
}

#define FG(d, v, c) F[((int64_t)(d) * 8 + (v)) * N + (c)]
static double ex_(const double* F, int64_t N, int64_t c, int sj, int sk) {
    return 0.25 * (FG(2, CB + 1, c) + FG(2, CB + 1, c - sj) - FG(1, CB + 2, c) - FG(1, CB + 2, c - sk));
}
static double ey_(const double* F, int64_t N, int64_t c, int si, int sk) {
    return 0.25 * (FG(0, CB + 2, c) + FG(0, CB + 2, c - sk) - FG(2, CB + 0, c) - FG(2, CB + 0, c - si));
}
static double ez_(const double* F, int64_t N, int64_t c, int si, int sj) {
    return 0.25 * (FG(1, CB + 0, c) + FG(1, CB + 0, c - si) - FG(0, CB + 1, c) - FG(0, CB + 1, c - sj));
}
/* edge EMFs of every block (E_x at i in [0,n), j, k in [0,n], alike for y,
 * z) from the face fluxes; then, where a finer block touches a boundary
 * edge, the mean of its two EMFs along that edge */
void fxo_emf_raw(int32_t nblock, const fxo_block* blk, int64_t N, const double* F, double* E) {
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n, si = SP(n) * SP(n), sj = SP(n), sk = 1;
#pragma omp parallel for schedule(static)
        for (int i = 0; i <= n; i++)
            for (int j = 0; j <= n; j++)
                for (int k = 0; k <= n; k++) {
                    int64_t c = bx(B, i, j, k);
                    if (i < n) E[c] = ex_(F, N, c, sj, sk);
                    if (j < n) E[N + c] = ey_(F, N, c, si, sk);
                    if (k < n) E[2 * N + c] = ez_(F, N, c, si, sj);
                }
    }
}
void fxo_emf_fix(int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, double* E) {
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n;
        const int32_t* nb = nbr + (int64_t)b * 27;
        for (int i = 0; i <= n; i++)
            for (int j = 0; j <= n; j++)
                for (int k = 0; k <= n; k++) {
                    int p[3] = {i, j, k};
                    for (int d = 0; d < 3; d++) {
                        if (p[d] >= n) continue;
                        int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                        int o1 = p[t1] == 0 ? -1 : (p[t1] == n ? 1 : 0);
                        int o2 = p[t2] == 0 ? -1 : (p[t2] == n ? 1 : 0);
                        if (o1 == 0 && o2 == 0) continue;
                        int done = 0;
                        for (int a1 = 0; a1 <= (o1 != 0) && !done; a1++)
                            for (int a2 = 0; a2 <= (o2 != 0) && !done; a2++) {
                                if (!a1 && !a2) continue;
                                int o[3] = {0, 0, 0};
                                o[t1] = a1 * o1;
                                o[t2] = a2 * o2;
                                int s = nb[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)];
                                if (s < 0) continue;
                                const fxo_block* S = &blk[s];
                                if (S->n != 2 * n) continue;
                                int f[3] = {2 * (p[0] - o[0] * n), 2 * (p[1] - o[1] * n), 2 * (p[2] - o[2] * n)};
                                int g[3] = {f[0], f[1], f[2]};
                                g[d] += 1;
                                const double* Es = E + d * N;
                                E[d * N + bx(B, p[0], p[1], p[2])] =
                                    0.5 * (Es[bx(S, f[0], f[1], f[2])] + Es[bx(S, g[0], g[1], g[2])]);
                                done = 1;
                            }
                    }
                }
    }
}

void fxo_emf(int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, const double* F, double* E,
             int maxlevel) {
    fxo_emf_raw(nblock, blk, N, F, E);
    if (maxlevel > 0) fxo_emf_fix(nblock, blk, nbr, N, E);
}

static void fupd(const double* E, int64_t N, double* Bf, double* Bf1, int d, int64_t c, int si, int sj, int sk,
                 double idx, double dt, int stage) {
    const double *Ex = E, *Ey = E + N, *Ez = E + 2 * N;
    double curl;
    if (d == 0)
        curl = (Ez[c + sj] - Ez[c]) * idx - (Ey[c + sk] - Ey[c]) * idx;
    else if (d == 1)
        curl = (Ex[c + sk] - Ex[c]) * idx - (Ez[c + si] - Ez[c]) * idx;
    else
        curl = (Ey[c + si] - Ey[c]) * idx - (Ex[c + sj] - Ex[c]) * idx;
    if (stage == 0)
        Bf1[d * N + c] = Bf[d * N + c] - dt * curl;
    else
        Bf[d * N + c] = 0.5 * (Bf[d * N + c] + Bf1[d * N + c] - dt * curl);
}

void fxo_update(const fxo_params* P, int32_t nblock, const fxo_block* blk, int64_t N, double* U, double* U1,
                const double* W, double* Bf, double* Bf1, const double* F, const double* E, double* dt, int stage) {
    double dtv = P->cfl * dt[0];
    if (stage == 0) dt[1] = dtv;
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n, si = SP(n) * SP(n), sj = SP(n), sk = 1;
        double idx = 1.0 / B->dx;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double x[3];
                    centre(B, i, j, k, x);
                    ksm m;
                    metric(P, x[0], x[1], x[2], &m);
                    ksd dk;
                    deriv(P, x[0], x[1], x[2], &m, &dk);
                    double w[8], S[8];
                    for (int v = 0; v < 8; v++) w[v] = W[v * N + c];
                    source(&m, &dk, P->gamma, w, S);
                    for (int v = 0; v < 5; v++) {
                        double div = (FG(0, v, c + si) - FG(0, v, c)) * idx + (FG(1, v, c + sj) - FG(1, v, c)) * idx +
                                     (FG(2, v, c + sk) - FG(2, v, c)) * idx;
                        double L = S[v] - div;
                        if (stage == 0)
                            U1[v * N + c] = U[v * N + c] + dtv * L;
                        else
                            U[v * N + c] = 0.5 * (U[v * N + c] + U1[v * N + c] + dtv * L);
                    }
                    fupd(E, N, Bf, Bf1, 0, c, si, sj, sk, idx, dtv, stage);
                    fupd(E, N, Bf, Bf1, 1, c, si, sj, sk, idx, dtv, stage);
                    fupd(E, N, Bf, Bf1, 2, c, si, sj, sk, idx, dtv, stage);
                    if (i == n - 1) fupd(E, N, Bf, Bf1, 0, c + si, si, sj, sk, idx, dtv, stage);
                    if (j == n - 1) fupd(E, N, Bf, Bf1, 1, c + sj, si, sj, sk, idx, dtv, stage);
                    if (k == n - 1) fupd(E, N, Bf, Bf1, 2, c + sk, si, sj, sk, idx, dtv, stage);
                }
    }
}

void fxo_step(const fxo_params* P, int32_t nblock, const fxo_block* blk, const int32_t* nbr, int64_t N, double* U,
              double* U1, double* W, double* Bf, double* Bf1, double* F, double* E, double* dt, int32_t* count,
              int maxlevel) {
    for (int stage = 0; stage < 2; stage++) {
        fxo_prims(P, nblock, blk, nbr, N, U, U1, W, Bf, Bf1, F, dt, count, stage, stage == 0);
        fxo_ghosts(nblock, blk, nbr, N, W, Bf, Bf1, stage, maxlevel, P->limiter == LIM_PPM ? 3 : 2);
        fxo_fluxes(P, nblock, blk, N, W, Bf, Bf1, F, stage);
        fxo_emf(nblock, blk, nbr, N, F, E, maxlevel);
        fxo_update(P, nblock, blk, N, U, U1, W, Bf, Bf1, F, E, dt, stage);
    }
}

/* |div B~| / max |B~| per block (interior cells) */
void fxo_divb(int32_t nblock, const fxo_block* blk, int64_t N, const double* Bf, double* out) {
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n, si = SP(n) * SP(n), sj = SP(n);
        double mx = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double f[6] = {Bf[c], Bf[c + si], Bf[N + c], Bf[N + c + sj], Bf[2 * N + c], Bf[2 * N + c + 1]};
                    double div = (f[1] - f[0]) + (f[3] - f[2]) + (f[5] - f[4]);
                    double m = 0.0;
                    for (int q = 0; q < 6; q++) m = dmax(m, dabs(f[q]));
                    double v = m > 0.0 ? dabs(div) / m : 0.0;
                    if (v > mx) mx = v;
                }
        out[b] = mx;
    }
}

/* ---------------------------------------------- batch physics (tests) */
/* face states of n faces from a[6][n] (cells p-3 .. p+2 of each face) */
void fxo_ppm_batch(int64_t n, const double* a, double* L, double* R) {
    for (int64_t t = 0; t < n; t++) {
        double c[6];
        for (int q = 0; q < 6; q++) c[q] = a[q * n + t];
        ppm_face(c, &L[t], &R[t]);
    }
}

void fxo_metric_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z,
                      double* out /* [n][22]: H, l[3], alpha, sqrtgam, beta[3], g[6], gi[6], r */) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        metric(P, x[q], y[q], z[q], &m);
        double* o = out + q * 22;
        o[0] = m.H;
        for (int i = 0; i < 3; i++) o[1 + i] = m.l[i];
        o[4] = m.alpha;
        o[5] = m.sqrtgam;
        for (int i = 0; i < 3; i++) o[6 + i] = m.beta[i];
        for (int i = 0; i < 6; i++) {
            o[9 + i] = m.g[i];
            o[15 + i] = m.gi[i];
        }
        o[21] = m.r;
    }
}
void fxo_deriv_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z,
                     double* out /* [n][12]: dH[3], dl[3][3] */) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        ksd d;
        metric(P, x[q], y[q], z[q], &m);
        deriv(P, x[q], y[q], z[q], &m, &d);
        double* o = out + q * 12;
        for (int k = 0; k < 3; k++) {
            o[k] = d.dH[k];
            for (int i = 0; i < 3; i++) o[3 + 3 * k + i] = d.dl[k][i];
        }
    }
}
/* w, u, F: [8][n] */
void fxo_cons_flux_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z, int dd,
                         const double* w, double* u, double* F, double* lm, double* lp) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        metric(P, x[q], y[q], z[q], &m);
        double wq[8], uq[8], Fq[8];
        for (int v = 0; v < 8; v++) wq[v] = w[v * n + q];
        drv d;
        derive(&m, P->gamma, wq, &d);
        p2c(&m, wq, &d, uq);
        pflux(&m, dd, wq, &d, uq, Fq);
        speeds(&m, P->gamma, dd, wq, &d, &lm[q], &lp[q]);
        for (int v = 0; v < 8; v++) {
            u[v * n + q] = uq[v];
            F[v * n + q] = Fq[v];
        }
    }
}
void fxo_hll_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z, int dd,
                   const double* wL, const double* wR, double* F) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        metric(P, x[q], y[q], z[q], &m);
        double a[8], b[8], Fq[8];
        for (int v = 0; v < 8; v++) {
            a[v] = wL[v * n + q];
            b[v] = wR[v * n + q];
        }
        hll(&m, P->gamma, dd, a, b, Fq);
        for (int v = 0; v < 8; v++) F[v * n + q] = Fq[v];
    }
}
void fxo_source_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z,
                      const double* w, double* S) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        ksd dk;
        metric(P, x[q], y[q], z[q], &m);
        deriv(P, x[q], y[q], z[q], &m, &dk);
        double wq[8], Sq[8];
        for (int v = 0; v < 8; v++) wq[v] = w[v * n + q];
        source(&m, &dk, P->gamma, wq, Sq);
        for (int v = 0; v < 8; v++) S[v * n + q] = Sq[v];
    }
}
/* U: [8][n] densitised conserved (B slots ignored), B: [3][n] Eulerian field,
 * wo: [8][n] previous primitives; w: [8][n]; st, it: [n] */
void fxo_c2p_batch(const fxo_params* P, int64_t n, const double* x, const double* y, const double* z, const double* U,
                   const double* B, const double* wo, double* w, int32_t* st, int32_t* it) {
    for (int64_t q = 0; q < n; q++) {
        ksm m;
        metric(P, x[q], y[q], z[q], &m);
        double u[8], b[3], o[8], wq[8];
        for (int v = 0; v < 8; v++) {
            u[v] = U[v * n + q];
            o[v] = wo[v * n + q];
        }
        for (int v = 0; v < 3; v++) b[v] = B[v * n + q];
        int its = 0;
        st[q] = c2p(P, &m, u, b, o, wq, &its);
        it[q] = its;
        for (int v = 0; v < 8; v++) w[v * n + q] = wq[v];
    }
}

/* ------------------------------------------------------ initial data */
/* Fishbone & Moncrief (1976) torus: conserved u^t u_phi of the circular
 * equatorial orbit at r_max; enthalpy potential; velocity in the locally
 * non-rotating frame; Cartesian Kerr-Schild four-velocity */
static double fm_ell(double a, double r) {
    double sr = sqrt(r), r32 = r * sr;
    return (r * r - 2.0 * a * sr + a * a) * (r32 + a) / (r32 * (r32 - 3.0 * sr + 2.0 * a));
}
static void fm_pt(double a, double r, double s2, double c2, double* Sig, double* Del, double* A, double* e2) {
    *Sig = r * r + a * a * c2;
    *Del = r * r - 2.0 * r + a * a;
    double ra = r * r + a * a;
    *A = ra * ra - *Del * a * a * s2;
    *e2 = *Sig * *Sig * *Del / (*A * *A * s2);
}
static double fm_pot(double a, double ell, double r, double s2, double c2) {
    double Sig, Del, A, e2;
    fm_pt(a, r, s2, c2, &Sig, &Del, &A, &e2);
    double X = sqrt(1.0 + 4.0 * ell * ell * e2);
    return 0.5 * log((1.0 + X) * A / (Sig * Del)) - 0.5 * X - 2.0 * a * r * ell / A;
}
typedef struct {
    double a, gamma, kappa, r_in, ell, w_in;
} fmt;
static double fm_rho(const fmt* t, double x, double y, double z, double* lnh_out) {
    double r = sqrt(r2_of(t->a, x, y, z));
    if (!(r >= t->r_in)) return 0.0;
    double c = z / r, c2 = c * c, s2 = 1.0 - c2;
    if (!(s2 > 0.0)) return 0.0;
    double lnh = fm_pot(t->a, t->ell, r, s2, c2) - t->w_in;
    if (lnh_out) *lnh_out = lnh;
    if (!(lnh > 0.0)) return 0.0;
    double h = exp(lnh);
    return pow((h - 1.0) * (t->gamma - 1.0) / (t->kappa * t->gamma), 1.0 / (t->gamma - 1.0));
}
static void fm_vel(const fmt* t, double x, double y, double z, double* ut, double* ux, double* uy) {
    double a = t->a;
    double r = sqrt(r2_of(a, x, y, z));
    double c = z / r, c2 = c * c, s2 = 1.0 - c2;
    double Sig, Del, A, e2;
    fm_pt(a, r, s2, c2, &Sig, &Del, &A, &e2);
    double U = sqrt(0.5 * (-1.0 + sqrt(1.0 + 4.0 * t->ell * t->ell * e2)));
    *ut = sqrt((1.0 + U * U) * A / (Sig * Del));
    double uphi = 2.0 * a * r * *ut / A + U * sqrt(Sig / (A * s2));
    *ux = -y * uphi;
    *uy = x * uphi;
}
static uint64_t cell_key(const double* x0, double dx, int i, int j, int k) {
    const int64_t off = 1 << 20;
    int64_t g0 = llround(x0[0] / dx) + i + off, g1 = llround(x0[1] / dx) + j + off, g2 = llround(x0[2] / dx) + k + off;
    return ((uint64_t)g0 << 42) | ((uint64_t)g1 << 21) | (uint64_t)g2;
}
static double hash_u(uint64_t seed, uint64_t id) {
    uint64_t z = seed * 0x100000001B3ULL + id + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
/* batch of the FM functions at points: out [n][6] = rho (unnormalised),
 * ln h, u^t, u^x, u^y, and the constant ell */
void fxo_fm_batch(double a, double gamma, double kappa, double r_in, double r_max, int64_t n, const double* x,
                  const double* y, const double* z, double* out) {
    fmt t = {a, gamma, kappa, r_in, fm_ell(a, r_max), 0.0};
    t.w_in = fm_pot(a, t.ell, r_in, 1.0, 0.0);
    for (int64_t q = 0; q < n; q++) {
        double lnh = -1.0, ut = 0.0, ux = 0.0, uy = 0.0;
        double rho = fm_rho(&t, x[q], y[q], z[q], &lnh);
        double r = sqrt(r2_of(a, x[q], y[q], z[q]));
        if (r >= r_in) fm_vel(&t, x[q], y[q], z[q], &ut, &ux, &uy);
        double* o = out + q * 6;
        o[0] = rho; o[1] = lnh; o[2] = ut; o[3] = ux; o[4] = uy; o[5] = t.ell;
    }
}
double fxo_fm_potential(double a, double ell, double r, double s2, double c2) { return fm_pot(a, ell, r, s2, c2); }
double fxo_fm_ell(double a, double r) { return fm_ell(a, r); }

static void apot(const fmt* t, double rmax, double x, double y, double z, double* ax, double* ay) {
    double rho = fm_rho(t, x, y, z, 0);
    double A = rho / rmax - 0.2;
    *ax = *ay = 0.0;
    if (A > 0.0) {
        double iw = 1.0 / (x * x + y * y);
        *ax = -A * y * iw;
        *ay = A * x * iw;
    }
}

/* A along an edge: the mean over its K finest-level sub-edge midpoints */
static void apot_edge(const fmt* t, double rmax, double x, double y, double z, int d, double h, int K, double* ax,
                      double* ay) {
    double sx = 0.0, sy = 0.0, p[3] = {x, y, z};
    double hk = h / K;
    for (int q = 0; q < K; q++) {
        double r[3] = {p[0], p[1], p[2]};
        r[d] = p[d] + (q + 0.5) * hk;
        double a, b;
        apot(t, rmax, r[0], r[1], r[2], &a, &b);
        sx += a;
        sy += b;
    }
    *ax = sx / K;
    *ay = sy / K;
}

/* the torus initial data of bh_fx_torus_init; out[4] as there */
void fxo_torus_init(const fxo_params* P, int32_t nblock, const fxo_block* blk, int64_t N, double* U, double* W,
                    double* Bf, double r_in, double r_max, double kappa, double beta, double noise, uint64_t seed,
                    double* out, int maxlevel) {
    fmt t = {P->a, P->gamma, kappa, r_in, fm_ell(P->a, r_max), 0.0};
    t.w_in = fm_pot(P->a, t.ell, r_in, 1.0, 0.0);
    memset(Bf, 0, sizeof(double) * 3 * N);
    double rmax = 0.0, pgmax = 0.0, pmmax = 0.0;
    for (int b = 0; b < nblock; b++) {
        int n = blk[b].n;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    double x[3];
                    centre(&blk[b], i, j, k, x);
                    double r = fm_rho(&t, x[0], x[1], x[2], 0);
                    if (r > rmax) rmax = r;
                }
    }
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double x[3];
                    centre(B, i, j, k, x);
                    ksm m;
                    metric(P, x[0], x[1], x[2], &m);
                    double rho = fm_rho(&t, x[0], x[1], x[2], 0);
                    double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    if (rho > 0.0 && rmax > 0.0) {
                        double p = t.kappa * pow(rho, t.gamma) / rmax;
                        double u = hash_u(seed, cell_key(B->x0, B->dx, i, j, k));
                        p = p * (1.0 + noise * (2.0 * u - 1.0));
                        double ut, ux, uy;
                        fm_vel(&t, x[0], x[1], x[2], &ut, &ux, &uy);
                        w[RHO] = rho / rmax;
                        w[PRS] = p;
                        w[UT] = ux + ut * m.beta[0];
                        w[UT + 1] = uy + ut * m.beta[1];
                        w[UT + 2] = ut * m.beta[2];
                    } else {
                        floor_state(P, m.r, &w[RHO], &w[PRS]);
                    }
                    floors(P, &m, w);
                    if (rho > 0.0 && rmax > 0.0 && w[PRS] > pgmax) pgmax = w[PRS];
                    for (int v = 0; v < 8; v++) W[v * N + c] = w[v];
                }
    }
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n;
        double h = B->dx, X = B->x0[0], Y = B->x0[1], Z = B->x0[2];
        int K = 1 << (maxlevel - B->level);
        for (int i = -1; i <= n; i++)
            for (int j = -1; j <= n; j++)
                for (int k = -1; k <= n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double ax0, ay0, ax1, ay1, d0, d1;
                    if (i >= 0) {
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + k * h, 1, h, K, &d0, &ay0);
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + (k + 1) * h, 1, h, K, &d1, &ay1);
                        Bf[c] = -(ay1 - ay0) / h;
                    }
                    if (j >= 0) {
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + k * h, 0, h, K, &ax0, &d0);
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + (k + 1) * h, 0, h, K, &ax1, &d1);
                        Bf[N + c] = (ax1 - ax0) / h;
                    }
                    if (k >= 0) {
                        double ayl, ayr, axl, axr;
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + k * h, 1, h, K, &d0, &ayl);
                        apot_edge(&t, rmax, X + (i + 1) * h, Y + j * h, Z + k * h, 1, h, K, &d1, &ayr);
                        apot_edge(&t, rmax, X + i * h, Y + j * h, Z + k * h, 0, h, K, &axl, &d0);
                        apot_edge(&t, rmax, X + i * h, Y + (j + 1) * h, Z + k * h, 0, h, K, &axr, &d1);
                        Bf[2 * N + c] = (ayr - ayl) / h - (axr - axl) / h;
                    }
                }
    }
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n, si = SP(n) * SP(n), sj = SP(n);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double x[3];
                    centre(B, i, j, k, x);
                    ksm m;
                    metric(P, x[0], x[1], x[2], &m);
                    double isg = 1.0 / m.sqrtgam;
                    double w[8];
                    for (int v = 0; v < 5; v++) w[v] = W[v * N + c];
                    w[BB] = 0.5 * (Bf[c] + Bf[c + si]) * isg;
                    w[BB + 1] = 0.5 * (Bf[N + c] + Bf[N + c + sj]) * isg;
                    w[BB + 2] = 0.5 * (Bf[2 * N + c] + Bf[2 * N + c + 1]) * isg;
                    drv d;
                    derive(&m, P->gamma, w, &d);
                    double pm = 0.5 * d.b2;
                    if (pm > pmmax) pmmax = pm;
                }
    }
    double s = (pmmax > 0.0 && beta > 0.0) ? sqrt(pgmax / (beta * pmmax)) : 0.0;
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n;
        for (int i = -1; i <= n; i++)
            for (int j = -1; j <= n; j++)
                for (int k = -1; k <= n; k++) {
                    int64_t c = bx(B, i, j, k);
                    if (i >= 0) Bf[c] *= s;
                    if (j >= 0) Bf[N + c] *= s;
                    if (k >= 0) Bf[2 * N + c] *= s;
                }
    }
    for (int b = 0; b < nblock; b++) {
        const fxo_block* B = &blk[b];
        int n = B->n, si = SP(n) * SP(n), sj = SP(n);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    int64_t c = bx(B, i, j, k);
                    double x[3];
                    centre(B, i, j, k, x);
                    ksm m;
                    metric(P, x[0], x[1], x[2], &m);
                    double Bt[3] = {0.5 * (Bf[c] + Bf[c + si]), 0.5 * (Bf[N + c] + Bf[N + c + sj]),
                                    0.5 * (Bf[2 * N + c] + Bf[2 * N + c + 1])};
                    double isg = 1.0 / m.sqrtgam;
                    double w[8], u[8];
                    for (int v = 0; v < 5; v++) w[v] = W[v * N + c];
                    for (int d = 0; d < 3; d++) w[BB + d] = Bt[d] * isg;
                    drv d;
                    derive(&m, P->gamma, w, &d);
                    p2c(&m, w, &d, u);
                    for (int v = 0; v < 5; v++) U[v * N + c] = u[v];
                    for (int q = 0; q < 3; q++) U[(5 + q) * N + c] = Bt[q];
                    for (int v = 5; v < 8; v++) W[v * N + c] = w[v];
                }
    }
    if (out) {
        out[0] = t.ell;
        out[1] = rmax;
        out[2] = s;
        out[3] = s > 0.0 ? pgmax / (s * s * pmmax) : 0.0;
    }
}
