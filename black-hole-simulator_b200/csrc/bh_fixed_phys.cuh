// bh_fixed_phys.cuh -- device physics of the corrected ("fixed") scheme:
// textbook Valencia GRMHD in Cartesian Kerr-Schild coordinates.
//
// The reference's scheme (src/fluid) cannot carry a Kerr torus through one
// step: its EOS throws in the first stage (physics/thermo.cpp:10-11 reached
// from conserved.cpp:205), its Newton derivative is wrong
// (conserved.cpp:114), its Brent fallback never updates fa/fb
// (conserved.cpp:261,272-282), its y and z faces call hlld(..., dim = 0)
// (grid.cpp:298,322), its metric is the (t,r,theta,phi) form applied to
// Cartesian vectors (spacetime.cpp:20-54), and its face field takes the full
// dt in both RK stages (transport.cpp:38-58, integrator.cpp:233-234).  This
// header keeps the reference's structure -- metric at cell and face centres,
// ptoc, a Newton con2prim, PLM face states, a two-wave HLL flux (the
// reference's own fallback, hlld.cpp:124-137), edge EMFs averaged from face
// fluxes (transport.cpp:11-36), the RK2 combine (integrator.cpp:238-259) --
// with each of those defects corrected:
//
//   metric    Kerr-Schild in Cartesian form, g = eta + 2 H l (x) l with
//             H = M r^3 / (r^4 + a^2 z^2) and the null covector
//             l = (1, (r x + a y)/(r^2+a^2), (r y - a x)/(r^2+a^2), z/r):
//             alpha = (1+2H)^-1/2, beta^i = 2H l_i/(1+2H),
//             gamma_ij = delta_ij + 2H l_i l_j, sqrt(gamma) = (1+2H)^1/2,
//             sqrt(-g) = 1; its first derivatives are analytic.
//   con2prim  Newton on Z = rho h W^2 with the exact derivative of the
//             energy residual (Noble et al. 2006, the "1D" scheme), raised
//             indices with the full inverse spatial metric.
//   fluxes    Valencia fluxes in the face's own normal direction; wave
//             speeds from the fast magnetosonic estimate in the GR
//             eigenvalue formula (Banyuls et al. 1997); HLL (Harten, Lax,
//             van Leer; Einfeldt's speed bounds).
//   sources   S(S_j) = 1/2 T^{mu nu} d_j g_{mu nu} and
//             S(tau) = alpha (T^{mu 0} d_mu ln alpha - T^{mu nu} Gamma^0_{mu nu}),
//             both evaluated from the analytic metric derivatives.
//   CT        face B advanced by a Heun average of the two stages' EMFs.
//
// Every operation of the time step is +, -, *, / or sqrt, so a build with
// --fmad=false and IEEE division equals a C restatement with the same
// operation order bit for bit.  RT is the arithmetic type of the face work
// (reconstruction, fluxes, sources): double, or float in the mixed variant;
// the metric is always evaluated in double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#ifndef BH_HD
#define BH_HD __host__ __device__
#endif
// every function of the scheme is inlined into its kernel: an outlined call
// would pass the small state arrays (face states, metric) through local
// memory and lose the constant face direction
#define BH_FI BH_HD __forceinline__

namespace bhfx {

// primitive slots: rho, p, ut^x, ut^y, ut^z (ut^i = W v^i, the spatial
// velocity of the fluid measured by normal observers times its Lorentz
// factor), B^x, B^y, B^z (Eulerian field, not densitised)
enum { P_RHO = 0, P_PRS = 1, P_UT = 2, P_B = 5 };
// conserved slots (the reference's cons order, cons.hpp:14-60), densitised
// by sqrt(gamma): D, S_x, S_y, S_z, tau, B^x, B^y, B^z
enum { C_D = 0, C_S = 1, C_TAU = 4, C_B = 5 };

struct FxPar {
    double M, a, gamma;
    double rho_fl, u_fl;      // floors rho >= rho_fl r^-3/2, u = p/(Gamma-1) >= u_fl r^-5/2
    double sigma_max, W_max;  // b^2/rho <= sigma_max, Lorentz factor <= W_max
    double r_exc;             // cells with r < r_exc are reset to the floor state
    double tol;               // con2prim: |dZ| <= tol Z
    int maxiter, limiter;
    // derived once per launch: Gamma/(Gamma-1), (Gamma-1)/Gamma, the v^2 of W_max
    double gg, gf, v2max;
    int flags;                // BH_FX_C2P_FP64
};

template <typename T>
BH_FI T fmin_(T a, T b) { return b < a ? b : a; }
template <typename T>
BH_FI T fmax_(T a, T b) { return a < b ? b : a; }
template <typename T>
BH_FI T fabs_(T a) { return a < T(0) ? -a : a; }
BH_FI double sqrt_(double x) { return sqrt(x); }
BH_FI float sqrt_(float x) { return sqrtf(x); }

// ======================================================================
// metric
// ======================================================================
// Kerr-Schild radius of a Cartesian point: the positive root of
// r^4 - (R^2 - a^2) r^2 - a^2 z^2 = 0
template <typename T>
BH_FI T ks_r2(T a, T x, T y, T z) {
    T a2 = a * a;
    T d = x * x + y * y + z * z - a2;
    return T(0.5) * (d + sqrt_(d * d + T(4) * a2 * z * z));
}

// The metric at a point, in the arithmetic type T (double everywhere but in
// the mixed variant's face and source work away from the horizon)
template <typename T>
struct KSb {
    T H, l[3];              // H and the spatial part of l_mu (l_0 = 1)
    T alpha, sqrtgam;       // lapse, sqrt(det gamma)
    T beta[3];              // shift beta^i
    T g[6], gi[6];          // gamma_ij and gamma^ij: xx, xy, xz, yy, yz, zz
    T r;
};
using KS = KSb<double>;
BH_FI int sym(int i, int j) {   // index into the 6-entry symmetric storage
    int a = i < j ? i : j, b = i < j ? j : i;
    return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

template <typename T>
BH_FI void ks_metric(const FxPar& P, T x, T y, T z, KSb<T>& m) {
    const T a = T(P.a), a2 = a * a;
    T r2 = ks_r2(a, x, y, z);
    T r = sqrt_(r2);
    T q = r2 * r2 + a2 * z * z;
    // on the disc z = 0, x^2 + y^2 <= a^2 (r = 0) the metric is flat
    T H = q > T(0) ? T(P.M) * r * r2 / q : T(0);
    T ir2a = T(1) / (r2 + a2);
    m.r = r;
    m.H = H;
    m.l[0] = (r * x + a * y) * ir2a;
    m.l[1] = (r * y - a * x) * ir2a;
    m.l[2] = r > T(0) ? z / r : T(0);
    T h2 = T(2) * H, f = T(1) + h2;
    m.sqrtgam = sqrt_(f);
    m.alpha = T(1) / m.sqrtgam;
    T hf = h2 / f;
    for (int i = 0; i < 3; i++) m.beta[i] = hf * m.l[i];
    for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++) {
            T ll = m.l[i] * m.l[j];
            m.g[sym(i, j)] = (i == j ? T(1) : T(0)) + h2 * ll;
            m.gi[sym(i, j)] = (i == j ? T(1) : T(0)) - hf * ll;
        }
}

// first derivatives: dH[k] = d_k H, dl[k][i] = d_k l_i (d_k l_0 = 0)
template <typename T>
struct KSDb {
    T dH[3], dl[3][3];
};
using KSD = KSDb<double>;
template <typename T>
BH_FI void ks_deriv(const FxPar& P, T x, T y, T z, const KSb<T>& m, KSDb<T>& d) {
    const T a = T(P.a), a2 = a * a, r = m.r, r2 = r * r;
    T q = r2 * r2 + a2 * z * z;
    if (!(q > T(0)) || !(r > T(0))) {
        for (int k = 0; k < 3; k++) {
            d.dH[k] = T(0);
            for (int i = 0; i < 3; i++) d.dl[k][i] = T(0);
        }
        return;
    }
    T iq = T(1) / q, r3 = r2 * r;
    T dr[3] = {x * r3 * iq, y * r3 * iq, z * r * (r2 + a2) * iq};
    T ir2a = T(1) / (r2 + a2);
    for (int k = 0; k < 3; k++) {
        T dq = T(4) * r3 * dr[k] + (k == 2 ? T(2) * a2 * z : T(0));
        d.dH[k] = T(P.M) * (T(3) * r2 * dr[k] * q - r3 * dq) * iq * iq;
        T t = T(2) * r * dr[k];
        d.dl[k][0] = (dr[k] * x + (k == 0 ? r : T(0)) + (k == 1 ? a : T(0)) - m.l[0] * t) * ir2a;
        d.dl[k][1] = (dr[k] * y + (k == 1 ? r : T(0)) - (k == 0 ? a : T(0)) - m.l[1] * t) * ir2a;
        d.dl[k][2] = ((k == 2 ? T(1) : T(0)) - m.l[2] * dr[k]) / r;
    }
}

// the spatial metric at the arithmetic type of the face work
template <typename RT>
struct KSm {
    RT alpha, sqrtgam, beta[3], g[6], gi[6];
};
template <typename RT, typename T>
BH_FI void ks_cast(const KSb<T>& m, KSm<RT>& o) {
    o.alpha = RT(m.alpha); o.sqrtgam = RT(m.sqrtgam);
    for (int i = 0; i < 3; i++) o.beta[i] = RT(m.beta[i]);
    for (int i = 0; i < 6; i++) { o.g[i] = RT(m.g[i]); o.gi[i] = RT(m.gi[i]); }
}
template <typename RT>
BH_FI void lower(const RT* g, const RT* v, RT* o) {
    o[0] = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
    o[1] = g[1] * v[0] + g[3] * v[1] + g[4] * v[2];
    o[2] = g[2] * v[0] + g[4] * v[1] + g[5] * v[2];
}

// ======================================================================
// primitive -> conserved (the role of conserved::ptoc, conserved.cpp:17-73)
// ======================================================================
// Derived quantities of a primitive state at a point.
template <typename RT>
struct Derived {
    RT W, iW, rhoh, v[3], vl[3], Bl[3], B2, Bv, b2, rhohW2, ptot;
    RT u2, ggp;   // W^2 - 1 = u_i u^i, and Gamma/(Gamma-1) p
};
template <typename RT>
// gg = Gamma / (Gamma - 1)
BH_FI void derive(const KSm<RT>& m, RT gg, const RT* w, Derived<RT>& d) {
    RT ut[3] = {w[P_UT], w[P_UT + 1], w[P_UT + 2]};
    RT B[3] = {w[P_B], w[P_B + 1], w[P_B + 2]};
    RT utl[3];
    lower(m.g, ut, utl);
    RT u2 = utl[0] * ut[0] + utl[1] * ut[1] + utl[2] * ut[2];
    d.u2 = u2;
    d.W = sqrt_(RT(1) + u2);
    RT iW = RT(1) / d.W;
    d.iW = iW;
    for (int i = 0; i < 3; i++) { d.v[i] = ut[i] * iW; d.vl[i] = utl[i] * iW; }
    lower(m.g, B, d.Bl);
    d.B2 = d.Bl[0] * B[0] + d.Bl[1] * B[1] + d.Bl[2] * B[2];
    d.Bv = d.Bl[0] * d.v[0] + d.Bl[1] * d.v[1] + d.Bl[2] * d.v[2];
    d.b2 = d.B2 * iW * iW + d.Bv * d.Bv;
    d.ggp = gg * w[P_PRS];
    RT rhoh = w[P_RHO] + d.ggp;
    d.rhoh = rhoh;
    d.rhohW2 = rhoh * d.W * d.W;
    d.ptot = w[P_PRS] + RT(0.5) * d.b2;
}
// densitised conserved state of primitives w (B slots: sqrt(gamma) B)
template <typename RT>
BH_FI void prim2cons(const KSm<RT>& m, RT gamma, const RT* w, const Derived<RT>& d, RT* u) {
    const RT sg = m.sqrtgam;
    RT v2 = RT(1) - d.iW * d.iW;
    u[C_D] = sg * w[P_RHO] * d.W;
    RT e = d.rhohW2 + d.B2;
    for (int i = 0; i < 3; i++) u[C_S + i] = sg * (e * d.vl[i] - d.Bv * d.Bl[i]);
    if (sizeof(RT) < sizeof(double)) {
        // tau = sqrt(gamma) (E - rho W) from its non-negative parts, with
        // W - 1 = u^2 / (1 + W): formed as sqrt(gamma) E - D it would carry
        // an error of eps E, which for slow, cold gas (tau << E) is large
        // relative to tau in FP32
        RT e = w[P_RHO] * d.W * (d.u2 / (RT(1) + d.W)) + (d.ggp * d.W * d.W - w[P_PRS]) +
               RT(0.5) * d.B2 * (RT(1) + v2) - RT(0.5) * d.Bv * d.Bv;
        u[C_TAU] = sg * e;
    } else {
        RT E = d.rhohW2 - w[P_PRS] + RT(0.5) * d.B2 * (RT(1) + v2) - RT(0.5) * d.Bv * d.Bv;
        u[C_TAU] = sg * E - u[C_D];
    }
    for (int i = 0; i < 3; i++) u[C_B + i] = sg * w[P_B + i];
}

// ======================================================================
// fluxes in direction dd (Valencia, densitised: sqrt(-g) F^dd with
// sqrt(-g) = alpha sqrt(gamma))
// ======================================================================
template <typename RT>
BH_FI void phys_flux(const KSm<RT>& m, int dd, const RT* w, const Derived<RT>& d, const RT* u, RT* F) {
    RT vt = m.alpha * d.v[dd] - m.beta[dd];       // coordinate transport velocity
    RT ag = m.alpha * m.sqrtgam;
    RT iW2 = d.iW * d.iW;
    RT Bd = w[P_B + dd];
    F[C_D] = u[C_D] * vt;
    for (int j = 0; j < 3; j++) {
        RT bjB = (d.Bl[j] * iW2 + d.Bv * d.vl[j]) * Bd;   // b_j B^dd / W
        F[C_S + j] = u[C_S + j] * vt + ag * ((j == dd ? d.ptot : RT(0)) - bjB);
    }
    F[C_TAU] = u[C_TAU] * vt + ag * (d.ptot * d.v[dd] - d.Bv * Bd);
    for (int k = 0; k < 3; k++) {
        RT vtk = m.alpha * d.v[k] - m.beta[k];
        F[C_B + k] = k == dd ? RT(0) : m.sqrtgam * (w[P_B + k] * vt - Bd * vtk);
    }
}

// fast magnetosonic signal speeds lambda-, lambda+ in direction dd
template <typename RT>
BH_FI void signal_speeds(const KSm<RT>& m, RT gamma, int dd, const RT* w, const Derived<RT>& d, RT& lm,
                                RT& lp) {
    RT rhoh = d.rhoh;
    // c_s^2 + v_A^2 - c_s^2 v_A^2 with c_s^2 = Gamma p / (rho h), v_A^2 = b^2 / (rho h + b^2)
    RT c2 = (gamma * w[P_PRS] + d.b2) / (rhoh + d.b2);
    c2 = fmin_(fmax_(c2, RT(0)), RT(1));
    RT v2 = RT(1) - d.iW * d.iW;
    RT vd = d.v[dd];
    RT gdd = m.gi[dd == 0 ? 0 : (dd == 1 ? 3 : 5)];
    RT den = RT(1) / (RT(1) - v2 * c2);
    RT disc = (RT(1) - v2) * (gdd * (RT(1) - v2 * c2) - vd * vd * (RT(1) - c2));
    RT rt = sqrt_(fmax_(c2 * disc, RT(0)));
    RT base = vd * (RT(1) - c2);
    lm = m.alpha * (base - rt) * den - m.beta[dd];
    lp = m.alpha * (base + rt) * den - m.beta[dd];
}

// ======================================================================
// PLM (reconfp's role, reconstruction.cpp:40-97): limited slopes
// ======================================================================
enum { FX_MINMOD = 0, FX_VANLEER = 1, FX_MC = 2, FX_PPM = 3 };
// The face value of cell w0 toward its neighbour wn across the face (wf:
// its neighbour on the other side): w0 + sigma/2, sigma the limited slope
// of (df, dn) = (w0 - wf, wn - w0) -- zero at an extremum, else, with
// s = sign(dn),
//   minmod    s min(|df|, |dn|)
//   van Leer  2 df dn / (df + dn)
//   MC        s min((|df| + |dn|)/2, 2 min(|df|, |dn|)).
// Where the extrapolation reaches the neighbour's value (MC's bound
// sigma = 2 dn) or comes within half the near difference of it (van Leer
// with |dn| < |df|), the value is formed from wn: w0 + sigma/2 would cancel
// dn against w0, and at a jump from the torus to the floor atmosphere
// (density ratio ~1e6 between neighbours) that leaves the face's density
// and pressure ~1e-2 relative accuracy in FP32.  sigma/2 is formed
// directly (MC: s min((|df| + |dn|)/4, |df|, |dn|)); the halvings are
// exact, so every other value rounds as w0 + (sigma)/2 does.
template <typename RT>
BH_FI RT plm_value(RT wf, RT w0, RT wn, int lim) {
    RT df = w0 - wf, dn = wn - w0;
    if (df * dn <= RT(0)) return w0;
    RT af = fabs_(df), an = fabs_(dn);
    if (lim == FX_VANLEER) {
        RT q = df + dn;
        return an < af ? wn - dn * dn / q : w0 + df * dn / q;
    }
    if (lim == FX_MC) {
        RT t = fmin_(RT(0.25) * (af + an), af);
        if (an < t) return wn;   // sigma = 2 dn: w0 + sigma/2 = wn
        return w0 + (dn > RT(0) ? t : -t);
    }
    RT t = RT(0.5) * fmin_(af, an);
    return w0 + (dn > RT(0) ? t : -t);
}
// face values at i-1/2 from cells i-2, i-1 (left) and i-1, i (right)
template <typename RT>
BH_FI void plm_face(RT wmm, RT wm, RT wp, RT wpp, int lim, RT& L, RT& R) {
    L = plm_value(wmm, wm, wp, lim);
    R = plm_value(wpp, wp, wm, lim);
}

// ======================================================================
// PPM (Colella & Woodward 1984, J. Comput. Phys. 54, 174, eqs. 1.6-1.8 and
// 1.10; no contact steepening, no flattening).  The face p-1/2 from the
// cells a[0..5] = p-3 .. p+2: limited slopes of cells p-2 .. p+1, the
// fourth-order interface values a_{p-3/2}, a_{p-1/2}, a_{p+1/2}, and the
// monotonised parabolas of cells p-1 (its right value is L) and p (its left
// value is R).  Every interface value lies between its two cells' values,
// so face densities and pressures stay positive as with PLM.
// ======================================================================
template <typename RT>
BH_FI RT ppm_dm(RT am, RT a0, RT ap) {
    RT dl = a0 - am, dr = ap - a0;
    if (dl * dr <= RT(0)) return RT(0);
    RT da = RT(0.5) * (ap - am);
    RT m = fmin_(fabs_(da), RT(2) * fmin_(fabs_(dl), fabs_(dr)));
    return da > RT(0) ? m : -m;
}
template <typename RT>
BH_FI void ppm_parabola(RT a, RT& l, RT& r) {
    if ((r - a) * (a - l) <= RT(0)) {
        l = a;
        r = a;
    } else {
        RT d = r - l, c = a - RT(0.5) * (l + r), d2 = d * d * (RT(1) / RT(6));
        if (d * c > d2)
            l = RT(3) * a - RT(2) * r;
        else if (-d2 > d * c)
            r = RT(3) * a - RT(2) * l;
    }
}
template <typename RT>
BH_FI void ppm_face(const RT* a, RT& L, RT& R) {
    RT dm[4];
    for (int q = 0; q < 4; q++) dm[q] = ppm_dm(a[q], a[q + 1], a[q + 2]);
    RT f[3];
    for (int q = 0; q < 3; q++)
        f[q] = a[q + 1] + RT(0.5) * (a[q + 2] - a[q + 1]) - (RT(1) / RT(6)) * (dm[q + 1] - dm[q]);
    RT lL = f[0], lR = f[1], rL = f[1], rR = f[2];
    ppm_parabola(a[2], lL, lR);
    ppm_parabola(a[3], rL, rR);
    L = lR;
    R = rL;
}

// ======================================================================
// HLL flux at a face from reconstructed left/right primitives.  The normal
// field comes from the face (wL[P_B+dd] = wR[P_B+dd]).  Returns the larger
// signal speed magnitude.
// ======================================================================
template <typename RT>
BH_FI RT hll_face(const KSm<RT>& m, RT gamma, RT gg, int dd, const RT* wL, const RT* wR, RT* F) {
    Derived<RT> dL, dR;
    derive(m, gg, wL, dL);
    derive(m, gg, wR, dR);
    RT uL[8], uR[8], FL[8], FR[8];
    prim2cons(m, gamma, wL, dL, uL);
    prim2cons(m, gamma, wR, dR, uR);
    phys_flux(m, dd, wL, dL, uL, FL);
    phys_flux(m, dd, wR, dR, uR, FR);
    RT lmL, lpL, lmR, lpR;
    signal_speeds(m, gamma, dd, wL, dL, lmL, lpL);
    signal_speeds(m, gamma, dd, wR, dR, lmR, lpR);
    RT sl = fmin_(fmin_(lmL, lmR), RT(0));
    RT sr = fmax_(fmax_(lpL, lpR), RT(0));
    RT ds = sr - sl;
    if (ds > RT(0)) {
        RT ids = RT(1) / ds, ss = sr * sl;
        for (int v = 0; v < 8; v++) F[v] = (sr * FL[v] - sl * FR[v] + ss * (uR[v] - uL[v])) * ids;
    } else {
        for (int v = 0; v < 8; v++) F[v] = RT(0.5) * (FL[v] + FR[v]);
    }
    F[C_B + dd] = RT(0);
    return fmax_(sr, -sl);
}

// ======================================================================
// geometric source of a cell (densitised: sqrt(-g) S = S here)
// ======================================================================
template <typename RT, typename MT>
BH_FI void source(const KSb<MT>& mk, const KSDb<MT>& dk, RT gg, const RT* w, RT* S) {
    KSm<RT> m;
    ks_cast(mk, m);
    Derived<RT> d;
    derive(m, gg, w, d);
    const RT H = RT(mk.H);
    RT l[4] = {RT(1), RT(mk.l[0]), RT(mk.l[1]), RT(mk.l[2])};
    // four-velocity and magnetic four-vector
    RT ia = RT(1) / m.alpha;
    RT u[4], b[4];
    u[0] = d.W * ia;
    for (int i = 0; i < 3; i++) u[1 + i] = w[P_UT + i] - u[0] * m.beta[i];
    b[0] = d.W * d.Bv * ia;
    RT iW = RT(1) / d.W;
    for (int i = 0; i < 3; i++) b[1 + i] = (w[P_B + i] + m.alpha * b[0] * u[1 + i]) * iW;
    RT e = d.rhoh + d.b2;
    // inverse four-metric g^{mu nu} = eta^{mu nu} - 2H l^mu l^nu, l^mu = (-1, l_i)
    RT lu[4] = {RT(-1), l[1], l[2], l[3]};
    RT T[4][4];
    for (int mu = 0; mu < 4; mu++)
        for (int nu = mu; nu < 4; nu++) {
            RT eta = mu == nu ? (mu == 0 ? RT(-1) : RT(1)) : RT(0);
            RT gi = eta - RT(2) * H * lu[mu] * lu[nu];
            T[mu][nu] = e * u[mu] * u[nu] + d.ptot * gi - b[mu] * b[nu];
            T[nu][mu] = T[mu][nu];
        }
    // Tl^mu = T^{mu nu} l_nu
    RT Tl[4];
    for (int mu = 0; mu < 4; mu++) Tl[mu] = T[mu][0] * l[0] + T[mu][1] * l[1] + T[mu][2] * l[2] + T[mu][3] * l[3];
    RT Tll = Tl[0] * l[0] + Tl[1] * l[1] + Tl[2] * l[2] + Tl[3] * l[3];
    RT dH[3], dl[3][3];
    for (int k = 0; k < 3; k++) {
        dH[k] = RT(dk.dH[k]);
        for (int i = 0; i < 3; i++) dl[k][i] = RT(dk.dl[k][i]);
    }
    // S(S_j) = 1/2 T^{mu nu} d_j g_{mu nu} = dH_j Tl.l + 2H Tl^i d_j l_i
    RT s[3];
    for (int j = 0; j < 3; j++)
        s[j] = dH[j] * Tll + RT(2) * H * (Tl[1] * dl[j][0] + Tl[2] * dl[j][1] + Tl[3] * dl[j][2]);
    // T^{mu nu} Gamma^0_{mu nu} = -2A + 4H^2 (l.Bv) - 2H C - 2H (l.s) with
    // A = Tl^k d_k H, Bv_i = Tl^k d_k l_i, C = T^{kj} d_k l_j
    RT A = Tl[1] * dH[0] + Tl[2] * dH[1] + Tl[3] * dH[2];
    RT lB = RT(0), Cc = RT(0);
    for (int i = 0; i < 3; i++) {
        RT Bi = Tl[1] * dl[0][i] + Tl[2] * dl[1][i] + Tl[3] * dl[2][i];
        lB += l[1 + i] * Bi;
        Cc += T[1][1 + i] * dl[0][i] + T[2][1 + i] * dl[1][i] + T[3][1 + i] * dl[2][i];
    }
    RT ls = l[1] * s[0] + l[2] * s[1] + l[3] * s[2];
    RT TG = RT(-2) * A + RT(4) * H * H * lB - RT(2) * H * Cc - RT(2) * H * ls;
    // d_i ln alpha = -alpha^2 d_i H
    RT a2 = m.alpha * m.alpha;
    RT T0dH = T[0][1] * dH[0] + T[0][2] * dH[1] + T[0][3] * dH[2];
    RT ag = m.alpha * m.sqrtgam;
    S[C_D] = RT(0);
    for (int j = 0; j < 3; j++) S[C_S + j] = ag * s[j];
    S[C_TAU] = ag * m.alpha * (-a2 * T0dH - TG);
    for (int k = 0; k < 3; k++) S[C_B + k] = RT(0);
}

// ======================================================================
// floors (the atmosphere of amrtree::pvfs, grid.cpp:133-146, as the
// configuration asks: rho_fl r^-3/2, u_fl r^-5/2), evaluated at max(r, 1)
// ======================================================================
template <typename T>
BH_FI void floor_state(const FxPar& P, T r, T& rho, T& p) {
    T re = r > T(1) ? r : T(1);
    T s = sqrt_(re);
    T ir = T(1) / (re * re * s);          // r^-5/2
    rho = T(P.rho_fl) * re * ir;
    p = (T(P.gamma) - T(1)) * T(P.u_fl) * ir;
}

// ======================================================================
// con2prim: Newton on Z = rho h W^2 (FP64).  U densitised, B^i the cell's
// Eulerian field (not densitised), wo the previous primitives (initial
// guess).  Returns 0 on success (w filled), 1 if the root was not found,
// 2 if the recovered state is unphysical; iters receives the residual
// evaluations.
//
// Phase 1: Newton from the previous primitives' Z (a step's change of the
// state is small, so this converges in two or three iterations).  It stops
// at the first iterate where v^2(Z) reaches the Lorentz-factor ceiling (the
// derivative is not that of the clamped residual there).  Phase 2: the
// residual is negative as Z -> 0 and positive for large Z; a bracket
// [0, Z_hi] (Z_hi doubled until f > 0) is narrowed by safeguarded Newton
// steps, each replaced by bisection when it would leave the bracket.
// ======================================================================
template <typename T>
struct C2Pb {
    T D, S2, B2, SB2, B4, E, gf, v2max;
};
using C2P = C2Pb<double>;
// residual f(Z) and its derivative; v2 is clamped to v2max (clamped = 1)
template <typename T>
BH_FI void c2p_eval(const C2Pb<T>& q, T Z, T& f, T& df, T& v2, int& clamped) {
    T iZ = T(1) / Z, ZB = Z + q.B2, iZB = T(1) / ZB;
    T iZB2 = iZB * iZB, iZ2 = iZ * iZ;
    v2 = q.S2 * iZB2 + q.SB2 * (q.B2 + T(2) * Z) * iZ2 * iZB2;
    clamped = v2 > q.v2max;
    if (clamped) v2 = q.v2max;
    T W2i = T(1) - v2, Wi = sqrt_(W2i);
    T p = q.gf * (Z * W2i - q.D * Wi);
    f = Z - p + T(0.5) * (T(1) + v2) * q.B2 - T(0.5) * q.SB2 * iZ2 - q.E;
    T dv2 = clamped ? T(0)
                    : T(-2) * q.S2 * iZB2 * iZB -
                          T(2) * q.SB2 * (T(3) * Z * Z + T(3) * Z * q.B2 + q.B4) * iZ2 * iZ * iZB2 * iZB;
    T dp = q.gf * (W2i - Z * dv2 + T(0.5) * q.D * dv2 / Wi);
    df = T(1) - dp + T(0.5) * q.B2 * dv2 + q.SB2 * iZ2 * iZ;
}

// PRE32 (the mixed variant): up to four FP32 Newton iterations from the
// previous primitives' Z.  Where they converge on a well-conditioned
// residual the FP32 root is the result; elsewhere the FP64 iterations start
// from it and alone decide convergence.
// The solver in three parts -- setup (the metric's invariants into q),
// solve (q and Z alone), finish (raise v with gamma^ij) -- so that a caller
// can let the metric go while it iterates.
template <typename T>
struct C2PSb {
    C2Pb<T> q;
    T S[3], Bl[3], SB, Z;
};
using C2PS = C2PSb<double>;
template <typename T>
BH_FI void c2p_setup(const FxPar& P, const KSb<T>& m, const T* U, const T* B, const T* wo, C2PSb<T>& s) {
    const T isg = m.alpha;   // 1 / sqrt(gamma)
    C2Pb<T>& q = s.q;
    q.gf = T(P.gf);
    q.D = U[C_D] * isg;
    T tau = U[C_TAU] * isg;
    for (int i = 0; i < 3; i++) s.S[i] = U[C_S + i] * isg;
    T Su[3];
    lower(m.gi, s.S, Su);   // S^i = gamma^ij S_j
    lower(m.g, B, s.Bl);
    q.S2 = Su[0] * s.S[0] + Su[1] * s.S[1] + Su[2] * s.S[2];
    q.B2 = s.Bl[0] * B[0] + s.Bl[1] * B[1] + s.Bl[2] * B[2];
    s.SB = s.S[0] * B[0] + s.S[1] * B[1] + s.S[2] * B[2];
    q.SB2 = s.SB * s.SB;
    q.B4 = q.B2 * q.B2;
    q.E = tau + q.D;
    q.v2max = T(P.v2max);
    // initial guess from the previous primitives
    T uto[3] = {wo[P_UT], wo[P_UT + 1], wo[P_UT + 2]}, utl[3];
    lower(m.g, uto, utl);
    T W2o = T(1) + utl[0] * uto[0] + utl[1] * uto[1] + utl[2] * uto[2];
    T Z = (wo[P_RHO] + T(P.gg) * wo[P_PRS]) * W2o;
    if (!(Z > T(0)) || !(Z < T(sizeof(T) < sizeof(double) ? 1e30 : 1e300))) Z = q.E > q.D ? q.E : q.D;
    s.Z = Z;
}
// FP32 con2prim (the mixed variant away from the hole): up to six Newton
// iterations on the FP32 residual.  Returns 0 when they converge (|dZ| <=
// 1e-6 Z) on a well-conditioned residual -- its rounding error, 2^-24 times
// its largest term (E, B^2, (S.B)^2 / Z^2), moves the root by at most
// 2^-24 * 16 Z / f'(Z), f' >= 1/2 -- else 1 (the caller solves in FP64).
BH_FI int c2p_solve32(C2PSb<float>& s, int& iters) {
    const C2Pb<float>& q = s.q;
    float Z = s.Z, f, df, v2;
    int cl = 0;
    for (int it = 0; it < 6; it++) {
        c2p_eval(q, Z, f, df, v2, cl);
        if (cl || !(df >= 0.5f)) { iters = it + 1; return 1; }
        float Zn = Z - f / df;
        if (!(Zn > 0.0f)) { iters = it + 1; return 1; }
        float e = fabs_(Zn - Z);
        Z = Zn;
        if (e <= 1e-6f * Z) {
            iters = it + 1;
            s.Z = Z;
            float iz = 1.0f / Z;
            return q.E + q.B2 + q.SB2 * iz * iz <= 16.0f * Z ? 0 : 1;
        }
    }
    iters = 6;
    return 1;
}
// returns 0 with s.Z the root, 1 if it was not found
template <bool PRE32 = false>
BH_FI int c2p_solve(const FxPar& P, C2PS& s, int& iters) {
    const C2P& q = s.q;
    double Z = s.Z;
    int it = 0, ok = 0, it32 = 0;
    double f, df, v2;
    int clamped;
    if (PRE32) {
        C2Pb<float> qf;
        qf.D = float(q.D); qf.S2 = float(q.S2); qf.B2 = float(q.B2); qf.SB2 = float(q.SB2);
        qf.B4 = float(q.B4); qf.E = float(q.E); qf.gf = float(q.gf); qf.v2max = float(q.v2max);
        float Zf = float(Z), ff, dff, v2f;
        int cl, conv = 0;
        for (; it32 < 4; it32++) {
            c2p_eval(qf, Zf, ff, dff, v2f, cl);
            if (cl || !(dff != 0.0f)) break;
            float Zn = Zf - ff / dff;
            if (!(Zn > 0.0f)) break;
            float e = fabs_(Zn - Zf);
            Zf = Zn;
            if (e <= 1e-6f * Zf) { it32++; conv = 1; break; }
        }
        if (Zf > 0.0f && Zf < 1e30f) {
            Z = double(Zf);
            // The FP32 root is kept (the primitives it gives are stored in
            // FP32) where the residual is well conditioned: its rounding
            // error, 2^-24 times its largest term (E, B^2, (S.B)^2 / Z^2),
            // moves the root by at most 2^-24 * 16 Z / f'(Z), f' >= 1/2 here
            if (conv && dff >= 0.5f) {
                float iz = 1.0f / Zf;
                float big = qf.E + qf.B2 + qf.SB2 * iz * iz;
                if (big <= 16.0f * Zf) {
                    iters = it32;
                    s.Z = Z;
                    return 0;
                }
            }
        }
    }
    // phase 1; a step of at most sqrt(tol) Z is accepted as the last one:
    // Newton's quadratic convergence leaves an error of order tol Z after it
    const double qtol = sqrt(P.tol);
    for (; it < P.maxiter; it++) {
        c2p_eval(q, Z, f, df, v2, clamped);
        if (clamped || !(df != 0.0)) break;
        double Zn = Z - f / df;
        if (!(Zn > 0.0)) break;
        double err = fabs_(Zn - Z);
        Z = Zn;
        if (err <= qtol * Z) { ok = 1; it++; break; }
    }
    // phase 2
    if (!ok) {
        double lo = 0.0, hi = Z > q.E ? Z : q.E;
        if (!(hi > 0.0)) hi = 1.0;
        int k = 0;
        for (; k < 64; k++) {
            c2p_eval(q, hi, f, df, v2, clamped);
            it++;
            if (f > 0.0) break;
            lo = hi;
            hi = 2.0 * hi;
        }
        if (f > 0.0 && hi < 1e300) {
            Z = hi;
            for (k = 0; k < 2 * P.maxiter + 60; k++) {
                double Zn = (df > 0.0) ? Z - f / df : 0.5 * (lo + hi);
                if (!(Zn > lo && Zn < hi)) Zn = 0.5 * (lo + hi);
                double err = fabs_(Zn - Z);
                Z = Zn;
                if (err <= P.tol * Z) { ok = 1; break; }
                c2p_eval(q, Z, f, df, v2, clamped);
                it++;
                if (f > 0.0) hi = Z; else lo = Z;
            }
        }
    }
    iters = it + it32;
    s.Z = Z;
    return ok ? 0 : 1;
}
// the primitives at the root; returns 0, or 2 if the state is unphysical
template <typename T>
BH_FI int c2p_finish(const T* gi, const C2PSb<T>& s, const T* B, T* w) {
    const C2Pb<T>& q = s.q;
    const T Z = s.Z;
    T iZ = T(1) / Z, ZB = Z + q.B2, iZB = T(1) / ZB;
    T v2 = q.S2 * iZB * iZB + q.SB2 * (q.B2 + T(2) * Z) * iZ * iZ * iZB * iZB;
    if (!(v2 < q.v2max)) v2 = q.v2max;
    T W2i = T(1) - v2, Wi = sqrt_(W2i);
    T Wl = T(1) / Wi;
    T rho = q.D * Wi;
    T p = q.gf * (Z * W2i - rho);
    // v_i = (S_i + (S.B / Z) B_i) / (Z + B^2), raised with gamma^ij
    T vl[3], vu[3];
    for (int i = 0; i < 3; i++) vl[i] = (s.S[i] + s.SB * iZ * s.Bl[i]) * iZB;
    lower(gi, vl, vu);
    w[P_RHO] = rho;
    w[P_PRS] = p;
    for (int i = 0; i < 3; i++) { w[P_UT + i] = Wl * vu[i]; w[P_B + i] = B[i]; }
    if (!(rho > T(0)) || !(p == p) || !(Wl == Wl)) return 2;
    return 0;
}
template <bool PRE32 = false>
BH_FI int con2prim(const FxPar& P, const KS& m, const double* U, const double* B, const double* wo,
                          double* w, int& iters) {
    C2PS s;
    c2p_setup(P, m, U, B, wo, s);
    if (c2p_solve<PRE32>(P, s, iters)) return 1;
    return c2p_finish(m.gi, s, B, w);
}

// ======================================================================
// floors and excision on a recovered state: returns 1 if w was changed
// (the caller then rewrites U = prim2cons(w))
// ======================================================================
template <typename T>
BH_FI int apply_floors(const FxPar& P, const KSb<T>& m, T* w) {
    T rf, pf;
    floor_state(P, m.r, rf, pf);
    int changed = 0;
    if (m.r < T(P.r_exc)) {
        w[P_RHO] = rf; w[P_PRS] = pf;
        w[P_UT] = w[P_UT + 1] = w[P_UT + 2] = T(0);
        return 1;
    }
    // Lorentz factor ceiling
    T ut[3] = {w[P_UT], w[P_UT + 1], w[P_UT + 2]}, utl[3];
    lower(m.g, ut, utl);
    T u2 = utl[0] * ut[0] + utl[1] * ut[1] + utl[2] * ut[2];
    T umax2 = T(P.W_max) * T(P.W_max) - T(1);
    if (u2 > umax2) {
        T sc = sqrt_(umax2 / u2);
        for (int i = 0; i < 3; i++) w[P_UT + i] = ut[i] * sc;
        u2 = umax2;
        changed = 1;
    }
    // magnetisation ceiling b^2 / rho <= sigma_max
    T W2 = T(1) + u2, iW2 = T(1) / W2;
    T B[3] = {w[P_B], w[P_B + 1], w[P_B + 2]}, Bl[3];
    lower(m.g, B, Bl);
    T B2 = Bl[0] * B[0] + Bl[1] * B[1] + Bl[2] * B[2];
    T Bu2 = Bl[0] * w[P_UT] + Bl[1] * w[P_UT + 1] + Bl[2] * w[P_UT + 2];   // W (B.v)
    T b2 = (B2 + Bu2 * Bu2) * iW2;
    T rs = b2 * (T(1) / T(P.sigma_max));
    if (rs > rf) rf = rs;
    if (!(w[P_RHO] >= rf)) { w[P_RHO] = rf; changed = 1; }
    if (!(w[P_PRS] >= pf)) { w[P_PRS] = pf; changed = 1; }
    return changed;
}

// ======================================================================
// CFL limit of a cell: the smallest dx_d / max|lambda_d|
// ======================================================================
template <typename A, typename B>
BH_FI void copy_metric(const KSb<A>& m, KSb<B>& mo) {
    mo.H = B(m.H); mo.alpha = B(m.alpha); mo.sqrtgam = B(m.sqrtgam); mo.r = B(m.r);
    for (int i = 0; i < 3; i++) { mo.l[i] = B(m.l[i]); mo.beta[i] = B(m.beta[i]); }
    for (int i = 0; i < 6; i++) { mo.g[i] = B(m.g[i]); mo.gi[i] = B(m.gi[i]); }
}
template <typename A, typename B>
BH_FI void copy_geometry(const KSb<A>& m, const KSDb<A>& d, KSb<B>& mo, KSDb<B>& dout) {
    mo.H = B(m.H); mo.alpha = B(m.alpha); mo.sqrtgam = B(m.sqrtgam); mo.r = B(m.r);
    for (int i = 0; i < 3; i++) { mo.l[i] = B(m.l[i]); mo.beta[i] = B(m.beta[i]); dout.dH[i] = B(d.dH[i]); }
    for (int i = 0; i < 6; i++) { mo.g[i] = B(m.g[i]); mo.gi[i] = B(m.gi[i]); }
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++) dout.dl[k][i] = B(d.dl[k][i]);
}

template <typename RT = double, typename MT = double, typename WT = double>
BH_FI double cell_dt(const FxPar& P, const KSb<MT>& mk, const WT* w64, const double* dx) {
    KSm<RT> m;
    ks_cast(mk, m);
    RT w[8];
    for (int v = 0; v < 8; v++) w[v] = RT(w64[v]);
    Derived<RT> d;
    derive(m, RT(P.gg), w, d);
    double best = 1e300;
    for (int dd = 0; dd < 3; dd++) {
        RT lm, lp;
        signal_speeds(m, RT(P.gamma), dd, w, d, lm, lp);
        double c = fmax_(fabs_(double(lm)), fabs_(double(lp)));
        if (c > 0.0) best = fmin_(best, dx[dd] / c);
    }
    return best;
}

// ======================================================================
// geometry for the face and source work.  FP64 everywhere in the FP64
// variants; in the mixed variant (RT = float) the metric and its
// derivatives are evaluated in FP32 beyond r ~ FX_R_FP64 (Euclidean
// radius), and in FP64 and rounded inside it, where the horizon's steep
// gradients are.
// ======================================================================
constexpr double FX_R_FP64 = 4.0;
template <typename RT>
BH_FI bool fp32_geometry(const double* x) {
    if (sizeof(RT) == sizeof(double)) return false;
    return x[0] * x[0] + x[1] * x[1] + x[2] * x[2] > FX_R_FP64 * FX_R_FP64;
}
// spatial metric at a face centre
template <typename RT>
BH_FI void face_geometry(const FxPar& P, const double* x, KSm<RT>& m) {
    if (fp32_geometry<RT>(x)) {
        KSb<float> mf;
        ks_metric<float>(P, float(x[0]), float(x[1]), float(x[2]), mf);
        ks_cast(mf, m);
    } else {
        KS mk;
        ks_metric(P, x[0], x[1], x[2], mk);
        ks_cast(mk, m);
    }
}
// metric and derivatives at a cell centre, in RT
template <typename RT>
BH_FI void cell_geometry(const FxPar& P, const double* x, KSb<RT>& m, KSDb<RT>& d) {
    if (fp32_geometry<RT>(x)) {
        KSb<float> mf;
        KSDb<float> df;
        ks_metric<float>(P, float(x[0]), float(x[1]), float(x[2]), mf);
        ks_deriv<float>(P, float(x[0]), float(x[1]), float(x[2]), mf, df);
        copy_geometry(mf, df, m, d);
    } else {
        KS mk;
        KSD dk;
        ks_metric(P, x[0], x[1], x[2], mk);
        ks_deriv(P, x[0], x[1], x[2], mk, dk);
        copy_geometry(mk, dk, m, d);
    }
}

// ======================================================================
// initial data: Fishbone & Moncrief (1976) torus in Boyer-Lindquist form,
// carried to Cartesian Kerr-Schild (the role of init::fm_init,
// initconds.cpp:228-591, with the configuration's parameters)
// ======================================================================
// u^t u_phi of the prograde circular equatorial orbit at r (M = 1 units):
// the torus's conserved angular momentum when its pressure peaks at r
BH_FI double fm_ell(double a, double r) {
    double sr = sqrt(r), r32 = r * sr;
    return (r * r - 2.0 * a * sr + a * a) * (r32 + a) / (r32 * (r32 - 3.0 * sr + 2.0 * a));
}
struct FMPoint {
    double Sig, Del, A, e2;   // Sigma, Delta, A and e^{2 nu - 2 psi} = Sigma^2 Delta / (A^2 sin^2)
};
BH_FI FMPoint fm_point(double a, double r, double s2, double c2) {
    FMPoint f;
    f.Sig = r * r + a * a * c2;
    f.Del = r * r - 2.0 * r + a * a;
    double ra = r * r + a * a;
    f.A = ra * ra - f.Del * a * a * s2;
    f.e2 = f.Sig * f.Sig * f.Del / (f.A * f.A * s2);
    return f;
}
// the FM enthalpy potential W(r, theta); ln h = W(r, theta) - W(r_in, pi/2)
BH_FI double fm_potential(double a, double ell, double r, double s2, double c2) {
    FMPoint f = fm_point(a, r, s2, c2);
    double X = sqrt(1.0 + 4.0 * ell * ell * f.e2);
    return 0.5 * log((1.0 + X) * f.A / (f.Sig * f.Del)) - 0.5 * X - 2.0 * a * r * ell / f.A;
}
struct FMTorus {
    double a, gamma, kappa, r_in, ell, w_in;
};
BH_FI FMTorus fm_torus(double a, double gamma, double kappa, double r_in, double r_max) {
    FMTorus t;
    t.a = a; t.gamma = gamma; t.kappa = kappa; t.r_in = r_in;
    t.ell = fm_ell(a, r_max);
    t.w_in = fm_potential(a, t.ell, r_in, 1.0, 0.0);
    return t;
}
// density (before normalisation) at a Cartesian KS point; 0 outside the torus
BH_FI double fm_rho(const FMTorus& t, double x, double y, double z, double* lnh_out) {
    double r = sqrt(ks_r2(t.a, x, y, z));
    if (!(r >= t.r_in)) return 0.0;
    double c = z / r, c2 = c * c, s2 = 1.0 - c2;
    if (!(s2 > 0.0)) return 0.0;
    double lnh = fm_potential(t.a, t.ell, r, s2, c2) - t.w_in;
    if (lnh_out) *lnh_out = lnh;
    if (!(lnh > 0.0)) return 0.0;
    double h = exp(lnh);
    return pow((h - 1.0) * (t.gamma - 1.0) / (t.kappa * t.gamma), 1.0 / (t.gamma - 1.0));
}
// four-velocity of the torus at a Cartesian KS point inside it:
// u^t and the Cartesian u^x, u^y (u^r = u^theta = 0, u^z = 0)
BH_FI void fm_velocity(const FMTorus& t, double x, double y, double z, double& ut, double& ux, double& uy) {
    const double a = t.a;
    double r = sqrt(ks_r2(a, x, y, z));
    double c = z / r, c2 = c * c, s2 = 1.0 - c2;
    FMPoint f = fm_point(a, r, s2, c2);
    // velocity in the locally non-rotating frame, u_(phi)^2 (1 + u_(phi)^2) = ell^2 e2
    double U = sqrt(0.5 * (-1.0 + sqrt(1.0 + 4.0 * t.ell * t.ell * f.e2)));
    ut = sqrt((1.0 + U * U) * f.A / (f.Sig * f.Del));
    double uphi = 2.0 * a * r * ut / f.A + U * sqrt(f.Sig / (f.A * s2));
    // x + i y = (r + i a) e^{i phi} sin(theta): d x / d phi = -y, d y / d phi = x
    ux = -y * uphi;
    uy = x * uphi;
}
// key of a cell from its global integer coordinates (x / dx - 1/2 rounded),
// so that the seeded perturbation does not depend on how the grid is cut
// into blocks; 21 bits per axis
BH_FI uint64_t cell_key(const double* x0, double dx, int i, int j, int k) {
    const int64_t off = 1 << 20;
    int64_t g0 = llround(x0[0] / dx) + i + off, g1 = llround(x0[1] / dx) + j + off, g2 = llround(x0[2] / dx) + k + off;
    return ((uint64_t)g0 << 42) | ((uint64_t)g1 << 21) | (uint64_t)g2;
}
// uniform deviate in [0, 1) from a 64-bit counter hash (SplitMix64 finaliser)
BH_FI double hash_uniform(uint64_t seed, uint64_t id) {
    uint64_t z = seed * 0x100000001B3ULL + id + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace bhfx
