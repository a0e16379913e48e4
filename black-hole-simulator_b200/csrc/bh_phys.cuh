// bh_phys.cuh -- device physics of the GRMHD block update (FP64).
//
// Each function restates one function of the reference fluid solver
// (Fjoerde/black-hole-simulator, src/fluid; paths below are relative to
// it).  Floating-point expressions keep the reference's left-to-right
// evaluation and its explicit zero metric entries, so that with
// --fmad=false results differ from the reference only through the last
// bits of sin/cos/acos/log/exp/pow.  Conditions where the reference throws
// std::domain_error (thermo.cpp:11-31) set BH_ERR_DOMAIN in *err and the
// computation continues.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "bhgpu.h"

#ifndef BH_HD
#define BH_HD __host__ __device__
#endif

namespace bh {

// ---- powers the reference takes from libm pow() ------------------------
// On the GPU they are plain multiplies/divides; a host build of this header
// (the bit-exact CPU check of the kernel logic) calls pow() like the
// reference does.
#ifdef __CUDA_ARCH__
BH_HD inline double pow_m1(double x) { return 1.0 / x; }
BH_HD inline double pow_m2(double x) { return 1.0 / (x * x); }
BH_HD inline double pow_mhalf(double x) { return 1.0 / sqrt(x); }
BH_HD inline double pow_3(double x) { return x * x * x; }
BH_HD inline double pow_4(double x) { return x * x * x * x; }
#else
BH_HD inline double pow_m1(double x) { return pow(x, -1); }
BH_HD inline double pow_m2(double x) { return pow(x, -2); }
BH_HD inline double pow_mhalf(double x) { return pow(x, -1.0 / 2.0); }
BH_HD inline double pow_3(double x) { return pow(x, 3.0); }
BH_HD inline double pow_4(double x) { return pow(x, 4); }
#endif

// ---- quotients ---------------------------------------------------------
// quo(a, b, rb) is the reference's a / b.  Variants compiled with BH_RCP
// (the FMA-contracted FP64 one and the mixed one) multiply by rb, a
// reciprocal of b the caller forms once for several quotients with the same
// divisor: each quotient moves by an ulp or two, as a contracted multiply-add
// does, and a multiply replaces the multi-instruction IEEE division.  In the
// reference-faithful build rb is never read and its computation is dead.
template <typename T>
BH_HD inline T quo(T a, T b, T rb) {
#ifdef BH_RCP
    (void)b;
    return a * rb;
#else
    (void)rb;
    return a / b;
#endif
}

constexpr int BLK = 16, GH = 2, CPN = 20;
constexpr int NC = CPN * CPN * CPN;                 // 8000 cells / patch
constexpr int NF = (CPN + 1) * CPN * CPN;           // 8400 faces / direction
constexpr int NE = CPN * (CPN + 1) * (CPN + 1);     // 8820 edges / direction
constexpr int NFACE = (BLK + 1) * BLK * BLK;        // 4352 flux faces / direction

// ---- std::min / std::max semantics (NaN included) ----------------------
template <typename T>
BH_HD inline T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T>
BH_HD inline T smax(T a, T b) { return (a < b) ? b : a; }

BH_HD inline void flag(int32_t* err, int bit) {
#ifdef __CUDA_ARCH__
    if (err) atomicOr(err, bit);
#else
    if (err) __atomic_fetch_or(err, bit, __ATOMIC_RELAXED);
#endif
}

// ---- indices (grid.cpp:51-89) -------------------------------------------
BH_HD inline int lindx(int i, int j, int k) { return (i + GH) * CPN * CPN + (j + GH) * CPN + (k + GH); }
BH_HD inline int xfc(int i, int j, int k) { return (i + GH) * CPN * CPN + (j + GH) * CPN + (k + GH); }
BH_HD inline int yfc(int i, int j, int k) { return (i + GH) * (CPN + 1) * CPN + (j + GH) * CPN + (k + GH); }
BH_HD inline int zfc(int i, int j, int k) { return (i + GH) * CPN * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
BH_HD inline int exi(int i, int j, int k) { return (i + GH) * (CPN + 1) * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
BH_HD inline int eyi(int i, int j, int k) { return (i + GH) * CPN * (CPN + 1) + (j + GH) * (CPN + 1) + (k + GH); }
BH_HD inline int ezi(int i, int j, int k) { return (i + GH) * (CPN + 1) * CPN + (j + GH) * CPN + (k + GH); }

// ======================================================================
// metric (physics/spacetime.cpp)
// ======================================================================
struct MP { double M, a, Q; };

// Spatial 3+1 part of metric::comp: gam = g[i+1][j+1], gam_inv =
// g_inv[i+1][j+1] (dense, with the reference's structural zeros), lapse,
// shift, sqrt(-g), sqrt(gamma).
template <typename RT>
struct MetT {
    RT gam[3][3], gam_inv[3][3];
    RT alpha, beta[3], sqrtdetg, sqrtdetgam;
    RT ialpha;   // 1 / alpha, for the reciprocal variants' quo
};
using Met = MetT<double>;
// the spatial metric at reduced precision (values computed in FP64)
template <typename RT>
BH_HD inline MetT<RT> met_cast(const Met& m) {
    MetT<RT> o;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { o.gam[i][j] = RT(m.gam[i][j]); o.gam_inv[i][j] = RT(m.gam_inv[i][j]); }
    o.alpha = RT(m.alpha); o.sqrtdetg = RT(m.sqrtdetg); o.sqrtdetgam = RT(m.sqrtdetgam); o.ialpha = RT(m.ialpha);
    for (int i = 0; i < 3; i++) o.beta[i] = RT(m.beta[i]);
    return o;
}

struct Trig { double c, s; };
BH_HD inline Trig trig(double th) {
    Trig t;
#ifdef __CUDA_ARCH__
    sincos(th, &t.s, &t.c);
#else
    t.s = sin(th); t.c = cos(th);
#endif
    return t;
}

BH_HD inline double Sigma_(const MP& m, double r, const Trig& t) {   // :12-14
    return r * r + m.a * m.a * (t.c * t.c);
}
BH_HD inline double H_(const MP& m, double r, double Sig) {           // :15-17
    return (2 * m.M * r - m.Q * m.Q) * pow_m1(Sig);
}

BH_HD inline void met_comp(const MP& m, double r, double th, Met& o) {
    Trig t = trig(th);
    const double a = m.a;
    double Sig = Sigma_(m, r, t);
    double H = H_(m, r, Sig);
    double s2 = t.s * t.s;
    // gcova (:20-34), spatial block
    double g11 = 1 + H, g13 = -H * a * s2, g22 = Sig;
    double g33 = (r * r + a * a + H * a * a * s2) * s2;
    // gcntr (:35-49)
    double gi00 = -1 - H, gi01 = H, gi11 = 1 - H, gi22 = pow_m1(Sig), gi13 = a * pow_m1(Sig);
    double gi33 = pow_m1(Sig * t.s * t.s);
    o.gam[0][0] = g11; o.gam[0][1] = 0.0; o.gam[0][2] = g13;
    o.gam[1][0] = 0.0; o.gam[1][1] = g22; o.gam[1][2] = 0.0;
    o.gam[2][0] = g13; o.gam[2][1] = 0.0; o.gam[2][2] = g33;
    o.gam_inv[0][0] = gi11; o.gam_inv[0][1] = 0.0; o.gam_inv[0][2] = gi13;
    o.gam_inv[1][0] = 0.0;  o.gam_inv[1][1] = gi22; o.gam_inv[1][2] = 0.0;
    o.gam_inv[2][0] = gi13; o.gam_inv[2][1] = 0.0; o.gam_inv[2][2] = gi33;
    o.sqrtdetg = (r * r + a * a * s2) * t.s;                // gdet :52-54
#if defined(BH_RCP) && defined(__CUDA_ARCH__)
    // the reciprocal variants on the device: the lapse from the hardware
    // reciprocal square root (within an ulp), its inverse without a division
    o.alpha = rsqrt(1 + H);                                 // lapse :93-95
    o.ialpha = (1 + H) * o.alpha;
#else
    o.alpha = pow_mhalf(1 + H);                             // lapse :93-95
    o.ialpha = 1.0 / o.alpha;
#endif
    // shift :96-100, three quotients by g^00 (one reciprocal in the
    // reciprocal variants; the sign of -0.0 / g^00 is kept by the product)
    double igi00 = 1.0 / gi00;
    o.beta[0] = quo(-gi01, gi00, igi00);
    o.beta[1] = quo(-0.0, gi00, igi00);
    o.beta[2] = quo(-0.0, gi00, igi00);
    o.sqrtdetgam = o.alpha * o.sqrtdetg;                    // :117-119
}

// Metric for the geometric source: g, g_inv, lapse, shift, sqrt(-g) and the
// metric derivatives d[l][m][n] = d_l g_mn (christ, :57-90) from which
// each Christoffel symbol is formed on demand (christoffel below), so that
// a caller never holds all 64 of them at once.
struct MetSrc {
    double g[4][4], gi[4][4], d[4][4][4];
    double alpha, beta[3], sqrtdetg;
};
BH_HD inline void met_src(const MP& m, double r, double th, MetSrc& o) {
    Trig t = trig(th);
    const double M = m.M, a = m.a, Q = m.Q;
    double Sig = Sigma_(m, r, t);
    double H = H_(m, r, Sig);
    double s2 = t.s * t.s, c2 = t.c * t.c;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) { o.g[i][j] = 0.0; o.gi[i][j] = 0.0; }
    o.g[0][0] = -1 + H;
    o.g[0][1] = o.g[1][0] = H;
    o.g[1][1] = 1 + H;
    o.g[2][2] = Sig;
    o.g[0][3] = o.g[1][3] = o.g[3][0] = o.g[3][1] = -H * a * s2;
    o.g[3][3] = (r * r + a * a + H * a * a * s2) * s2;
    o.gi[0][0] = -1 - H;
    o.gi[0][1] = o.gi[1][0] = H;
    o.gi[1][1] = 1 - H;
    o.gi[2][2] = pow_m1(Sig);
    o.gi[1][3] = o.gi[3][1] = a * pow_m1(Sig);
    o.gi[3][3] = pow_m1(Sig * t.s * t.s);
    o.sqrtdetg = (r * r + a * a * s2) * t.s;
#if defined(BH_RCP) && defined(__CUDA_ARCH__)
    // the same lapse as met_comp's in the reciprocal variants, so that the
    // face/ptoc metric and the source metric of a cell agree to the bit
    o.alpha = rsqrt(1 + H);
#else
    o.alpha = pow_mhalf(1 + H);
#endif
    double igi00 = 1.0 / o.gi[0][0];
    for (int i = 0; i < 3; i++) o.beta[i] = quo(-o.gi[0][i + 1], o.gi[0][0], igi00);
    // metric derivatives (:72-80)
    double sig = r * r + a * a * c2;
    double isig = pow_m1(sig), isig2 = pow_m2(sig);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) o.d[i][j][k] = 0;
    double A1 = -2 * (M * r * r - Q * Q * r - M * a * a * c2) * isig2;
    double A2 = 2 * a * a * (2 * M * r - Q * Q) * t.c * t.s * isig;
    double A3 = 2 * a * a * s2 * (M * r * r - Q * Q * r - M * a * a * c2) * isig2;
    double A4 = 2 * a * t.c * t.s * (2 * M * r - Q * Q) * (r * r + a * a) * isig2;
    double A5 = s2 * (((2 * M * a * a * s2) * isig) + ((2 * r * a * a * s2 * (2 * M * r - Q * Q)) * isig2) + 2 * r);
    double A6 = s2 * (((2 * pow_4(a) * (2 * M * r - Q * Q) * t.c * pow_3(t.s)) * isig2) +
                      ((2 * a * a * (2 * M * r - Q * Q) * t.c * t.s) * isig)) +
                t.c * t.s * (((a * a * s2 * (2 * M * r - Q * Q)) * isig) + r * r + a * a);
    o.d[1][0][0] = o.d[1][0][1] = o.d[1][1][0] = o.d[1][1][1] = A1;
    o.d[2][0][0] = o.d[2][0][1] = o.d[2][1][0] = o.d[2][1][1] = A2;
    o.d[1][2][2] = 2 * r;
    o.d[2][2][2] = -a * a * t.c * t.s;
    o.d[1][0][3] = o.d[1][3][0] = o.d[1][1][3] = o.d[1][3][1] = A3;
    o.d[2][0][3] = o.d[2][3][0] = o.d[2][1][3] = o.d[2][3][1] = A4;
    o.d[1][3][3] = A5;
    o.d[2][3][3] = A6;
}
// Christoffel symbol Gamma^l_{mm n} (christ, :81-90)
BH_HD inline double christoffel(const MetSrc& o, int l, int mm, int n) {
    return 0.5 * (o.gi[l][0] * (o.d[mm][0][n] + o.d[n][0][mm] - o.d[0][mm][n]) +
                  o.gi[l][1] * (o.d[mm][1][n] + o.d[n][1][mm] - o.d[1][mm][n]) +
                  o.gi[l][2] * (o.d[mm][2][n] + o.d[n][2][mm] - o.d[2][mm][n]) +
                  o.gi[l][3] * (o.d[mm][3][n] + o.d[n][3][mm] - o.d[3][mm][n]));
}

// Full metric with every Christoffel symbol (the batched metric::comp)
struct MetFull {
    double g[4][4], gi[4][4], G[4][4][4];
    double alpha, beta[3], sqrtdetg;
};
BH_HD inline void met_full(const MP& m, double r, double th, MetFull& o) {
    MetSrc s;
    met_src(m, r, th, s);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) { o.g[i][j] = s.g[i][j]; o.gi[i][j] = s.gi[i][j]; }
    o.alpha = s.alpha; o.sqrtdetg = s.sqrtdetg;
    for (int i = 0; i < 3; i++) o.beta[i] = s.beta[i];
#pragma unroll
    for (int l = 0; l < 4; l++)
#pragma unroll
        for (int mm = 0; mm < 4; mm++)
#pragma unroll
            for (int n = 0; n < 4; n++) o.G[l][mm][n] = christoffel(s, l, mm, n);
}

// ======================================================================
// EOS (physics/thermo.cpp:10-35)
// ======================================================================
template <typename RT>
BH_HD inline bool eos_ok(RT rho) { return !(rho <= RT(0.0)); }
template <typename RT>
BH_HD inline RT press(RT g, RT rho, RT eps) { return (g - RT(1.0)) * rho * eps; }
template <typename RT>
BH_HD inline RT enth(RT g, RT eps) { return RT(1.0) + g * eps; }
template <typename RT>
BH_HD inline RT cs2f(RT g, RT rho, RT eps) {
    RT p = press(g, rho, eps), h = enth(g, eps);
    return (g * p) / (rho * h);
}

// primitive / conserved vectors in the reference member order
template <typename RT> struct PrimT { RT rho, eps, v[3], B[3]; };
template <typename RT> struct ConsT { RT D, S[3], tau, B[3]; };

// ======================================================================
// prim -> cons, conserved::ptoc (physics/conserved.cpp:17-73)
// returns false where the reference throws (rho <= 0)
// ======================================================================
template <typename RT> struct PtocOutT { RT lor, p, h, b2; };
template <typename RT>
BH_HD inline bool ptoc(RT gamma, const MetT<RT>& mc, const PrimT<RT>& pv, ConsT<RT>& CV, PtocOutT<RT>* po = nullptr) {
    RT sg = mc.sqrtdetgam;
    RT v2 = RT(0.0), vlow[3] = {RT(0.0), RT(0.0), RT(0.0)};
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) vlow[i] += mc.gam[i][j] * pv.v[j];
        v2 += vlow[i] * pv.v[i];
    }
    v2 = smin(v2, RT(1.0) - RT(1e-10));
    RT sq1v = sqrt(RT(1.0) - v2);
    RT lor = RT(1.0) / sq1v;              // 1 / lor = sq1v within an ulp
    bool ok = eos_ok(pv.rho);
    RT p = press(gamma, pv.rho, pv.eps);
    RT h = enth(gamma, pv.eps);
    RT Blow[3] = {RT(0.0), RT(0.0), RT(0.0)};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) Blow[i] += mc.gam[i][j] * pv.B[j];
    RT Bv = RT(0.0);
#pragma unroll
    for (int i = 0; i < 3; i++) Bv += Blow[i] * pv.v[i];
    RT Bsq = RT(0.0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) Bsq += Blow[i] * mc.gam[i][j] * pv.B[j];
    RT b2 = quo(Bv * Bv + Bsq, lor, sq1v);
    RT bt = quo(lor * Bv, mc.alpha, mc.ialpha);
    RT pstar = p + b2 / 2;
    RT w = pv.rho * h + b2;
    CV.D = sg * pv.rho * lor;
    CV.tau = sg * (w * lor * lor - pstar - bt * bt) - CV.D;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        RT bi = quo(Blow[i] + mc.alpha * bt * lor * vlow[i], lor, sq1v);
        CV.S[i] = sg * (w * lor * lor * vlow[i] - mc.alpha * bt * bi);
        CV.B[i] = sg * pv.B[i];
    }
    if (po) { po->lor = lor; po->p = p; po->h = h; po->b2 = b2; }
    return ok;
}

using Prim = PrimT<double>;
using Cons = ConsT<double>;
using PtocOut = PtocOutT<double>;

// ======================================================================
// cons -> prim, conserved::ctop + f_df + cp_bd (physics/conserved.cpp:80-285)
// ======================================================================
BH_HD inline double f_df(double gamma, double xi, double Ssq, double Bsq, double SB,
                                       double Dn, double taun, double& df) {
    double Yi = SB * SB;
    double K = Bsq;
    double X = xi * xi;
    double xipK = xi + K;
#ifdef BH_RCP
    // one division for the divisors of the residual, X + (xi + K)^2 and X,
    // and of its derivative, X (xi + K)^2: their reciprocals from that of
    // the product (an ulp or two each)
    double xipK2 = xipK * xipK;
    double Dv = X + xipK2;
    double r3 = 1.0 / (X * Dv * xipK2);
    double rXD = xipK2 * r3;
    double vsq = (Ssq * X + Yi * (2.0 * xi + K)) * (X * rXD);
    double iX = Dv * rXD;
#else
    double vsq = (Ssq * X + Yi * (2.0 * xi + K)) / (X + xipK * xipK);
#endif
    if (vsq >= 1.0) { df = 0.0; return 1e30; }
    double om = 1.0 - vsq;                // 1 / ltz2 within an ulp
    double ltz2 = 1.0 / om;
    double ltz = sqrt(ltz2);
    // reciprocals for quo: 1 / ltz = sqrt(om) within two ulps; with them the
    // residual alone (fres) needs neither ltz2 nor ltz
#ifdef BH_RCP
    double il = sqrt(om);
#else
    double il = sqrt(om), iX = 1.0 / X;   // read only by the reciprocal variants' quo
#endif
    double rho = quo(Dn, ltz, il);
    double G = gamma - 1.0;
    double p = (G / gamma) * (quo(xi, ltz2, om) - quo(Dn, ltz, il));
    double pstar = p + quo(K, 2 * ltz2, 0.5 * om) + quo(Yi, 2 * X, 0.5 * iX);
    if (p < 0.0 || rho < 0.0) { df = 0.0; return 1e32; }
    double f = xi - taun - Dn - pstar;
    double N = Ssq * X + Yi * (2.0 * xi + K);
    double Mq = X * xipK * xipK;
    double dN = 2.0 * Ssq * xi + 2.0 * Yi;
    double dM = 2.0 * xi * xipK * xipK + 2.0 * X * X;
#ifdef BH_RCP
    double iMq = Dv * r3;
#else
    double iMq = 1.0 / Mq;               // read only by the reciprocal variants' quo
#endif
    double dvv = quo(dN * Mq - dM * N, Mq * Mq, iMq * iMq);
    double dltz2 = ltz2 * ltz2 * dvv;
    double dltz = quo(dltz2, 2.0 * ltz, 0.5 * il);
    double dp = (G / gamma) * (quo(1.0, ltz2, om) - quo(xi * dltz2, ltz2 * ltz2, om * om) + quo(Dn * dltz, ltz2, om));
    double dpstar = dp - quo(K * dltz2, 2.0 * ltz2 * ltz2, 0.5 * om * om) - quo(Yi, xi * X, xi * iX * iX);
    df = 1 - dpstar;
    return f;
}
BH_HD inline double fres(double gamma, double xi, double Ssq, double Bsq, double SB, double Dn,
                                       double taun) {
    double d;
    return f_df(gamma, xi, Ssq, Bsq, SB, Dn, taun, d);
}
BH_HD inline bool cp_bd(double gamma, double xa, double xb, double Ssq, double Bsq, double SB, double D,
                             double tau, double& root, double tol) {
    double fa = fres(gamma, xa, Ssq, Bsq, SB, D, tau);
    double fb = fres(gamma, xb, Ssq, Bsq, SB, D, tau);
    if (fa * fb > 0.0) return false;
    if (fabs(fa) < fabs(fb)) { double t = xa; xa = xb; xb = t; t = fa; fa = fb; fb = t; }
    double xc = xa, fc = fa;
    bool mflag = true;
    double s = 0.0, d = 0.0;
    // fa and fb change only by the swap at the end of an iteration (A7: they
    // are never updated from fs), so fb - fa is loop-invariant until a swap;
    // its reciprocal is formed here and again after a swap (used by the
    // variants that multiply by reciprocals; the faithful one divides)
    double idfba = 1.0 / (fb - fa);
    for (int i = 0; i < 100; i++) {
        if (fabs(xb - xa) < tol) { root = xb; return true; }
        if (fa != fc && fb != fc)
            s = (xa * fb * fc) / ((fa - fb) - (fa - fc)) + (xb * fa * fc) / ((fb - fa) - (fb - fc)) +
                (xc * fa * fb) / ((fc - fa) - (fc - fb));
        else
            s = xb - quo(fb * (xb - xa), fb - fa, idfba);
        bool c1 = !((3 * xa + 4) / 4 < s && s < xb);
        bool c2 = mflag && fabs(s - xb) >= fabs(xb - xc) / 2;
        bool c3 = !mflag && fabs(s - xb) >= fabs(xc - d) / 2;
        if (c1 || c2 || c3) { s = (xa + xb) / 2; mflag = true; }
        else mflag = false;
        double fs = fres(gamma, s, Ssq, Bsq, SB, D, tau);
        d = xc; xc = xb; fc = fb;
        if (fa * fs < 0.0) xb = s;
        else xa = s;
        if (fabs(fa) < fabs(fb)) {
            double t = xa; xa = xb; xb = t; t = fa; fa = fb; fb = t;
            idfba = 1.0 / (fb - fa);
        }
    }
    return false;
}

struct CtopOut { double p, T, h, lor, b2; int iters, path; };
// returns 1 ok / 0 failed; *domain set where the reference throws
// xi0: Newton's start where it lies strictly inside the bracket (the learned
// guess; NaN, the default, keeps the reference's midpoint); pre[5] (may be
// null) receives D, tau, Ssq, Bsq, SB of the preamble, and with maxiter = 0
// ctop returns right after it (pv and co are then not written)
BH_HD inline int ctop(double gamma, int maxiter, double tol, const Met& mc, const Cons& cv, Prim& pv,
                           bool& domain, CtopOut* co = nullptr, double xi0 = NAN, double* pre = nullptr) {
    double sg = mc.sqrtdetgam, isg = 1.0 / sg;
    double D = quo(cv.D, sg, isg);
    double tau = quo(cv.tau, sg, isg);
    // conserved.cpp:144-150 reads B[j], S[j] for j > i before they are
    // assigned; those reads are zero here (the reference's value on a clean stack)
    double B[3] = {0.0, 0.0, 0.0}, S[3] = {0.0, 0.0, 0.0};
    double Bu[3], Su[3];
    double Bsq = 0.0, Ssq = 0.0, SB = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        B[i] = quo(cv.B[i], sg, isg);
        S[i] = quo(cv.S[i], sg, isg);
        Bu[i] = mc.gam_inv[i][2] * B[2];     // the inner j-loop assigns; j = 2 survives
        Su[i] = mc.gam_inv[i][2] * S[2];
        Ssq += S[i] * Su[i];
        Bsq += B[i] * Bu[i];
        SB += S[i] * Bu[i];
    }
    if (pre) {
        pre[0] = D; pre[1] = tau; pre[2] = Ssq; pre[3] = Bsq; pre[4] = SB;
        if (maxiter == 0) return 0;   // only the preamble was asked for
    }
    double xi_l = D;
    double xi_h = tau + D + Bsq / 2.0 + 1e3;
    double fl = fres(gamma, xi_l, Ssq, Bsq, SB, D, tau);
    double fh = fres(gamma, xi_h, Ssq, Bsq, SB, D, tau);
    while (fl * fh > 0.0 && xi_h < 1e8 * D) {
        xi_h *= 2.0;
        fl = fres(gamma, xi_h, Ssq, Bsq, SB, D, tau);
    }
    double xi = (xi_l + xi_h) / 2.0;
    if (isfinite(xi0) && xi0 > xi_l && xi0 < xi_h) xi = xi0;
    bool nr_ok = true, conv = false;
    int it = 0;
    for (int i = 0; i < maxiter; i++) {
        double dF;
        double F = f_df(gamma, xi, Ssq, Bsq, SB, D, tau, dF);
        it = i + 1;
        if (fabs(F) < tol) { conv = true; break; }
        if (fabs(dF) < 1e-30) { nr_ok = false; break; }
        double xin = xi - F / dF;
        if (xin < xi_l || xin > xi_h) { nr_ok = false; break; }
        xi = xin;
    }
    int path = conv ? 0 : 1;
    if (!nr_ok) {
        double xib;
        if (!cp_bd(gamma, xi_l, xi_h, Ssq, Bsq, SB, D, tau, xib, tol)) {
            if (co) { co->iters = it; co->path = 3; }
            return 0;
        }
        path = 2;
        xi = xib;
    }
    double xpQ = xi + Bsq;
    double sdb2 = SB * SB;
    double vsq = (Ssq * xpQ * xpQ + sdb2 * (2.0 * xi + Bsq)) / (xpQ * xpQ * xi * xi);
    vsq = smin(vsq, 1.0 - 1e-10);
    double ltz2 = 1.0 / (1.0 - vsq);
    double ltz = sqrt(ltz2);
    pv.rho = D / ltz;
    double h = xi / (pv.rho * ltz2);
    pv.eps = (h - 1.0) / (gamma);
    if (!eos_ok(pv.rho)) domain = true;
    double p = press(gamma, pv.rho, pv.eps);
    double hh = enth(gamma, pv.eps);
    double T = p / pv.rho;
    double ixpQ = 1.0 / xpQ;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        pv.v[i] = quo(Su[i] + (SB / xi) * Bu[i], xpQ, ixpQ);
        pv.B[i] = B[i];
    }
    if (co) {
        double Blow[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) Blow[i] += mc.gam[i][j] * B[j];
        double Bv = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) Bv += Blow[i] * mc.gam[i][j] * pv.v[j];
        co->b2 = (Bv * Bv + Bsq) / ltz2;
        co->p = p; co->h = hh; co->T = T; co->lor = ltz; co->iters = it; co->path = path;
    }
    if (pv.rho <= 0.0 || pv.eps <= 0.0 || p <= 0.0) return 0;
    return 1;
}

// floor state amrtree::pvfs (grid.cpp:133-146; constants grid.hpp:140-143)
BH_HD inline void pvfs(double r, double& rho, double& eps) {
    double rfscal = 1.0 / pow_3(sqrt(smax(r, 1e-10) / 1.0));
    rho = 1e-7 * rfscal;
    eps = 1e-5 * rfscal;
}

// ======================================================================
// HLLD (solver/hlld.cpp)
// ======================================================================
template <typename RT> struct SideT {
    RT rho, eps, p, h, vn, vt1, vt2, Bn, Bt1, Bt2, ltz2, iltz2, b2, pt, cf, D, tau, Sn, St1, St2, Bc, E;
};
template <typename RT> struct CstT { RT D, Sn, St1, St2, tau, Bn, Bt1, Bt2; };

template <typename RT>
BH_HD inline RT fastspeed(RT rho, RT h, RT b2, RT cs2) {  // :34-39
    RT va2 = b2 / (rho * h + b2);
    RT cf2 = cs2 + va2 * (1 - cs2);
    cf2 = smin(cf2, 1 - RT(1e-10));
    return sqrt(cf2);
}
template <typename RT>
BH_HD inline bool side_(RT gamma, const PrimT<RT>& W, const ConsT<RT>& U, const MetT<RT>& mc, RT sqrtg, int dim,
                             SideT<RT>& s) {                                         // :41-94
    int t1 = (dim + 1) % 3, t2 = (dim + 2) % 3;
    s.rho = W.rho; s.eps = W.eps;
    bool ok = eos_ok(W.rho);
    s.p = press(gamma, W.rho, W.eps);
    s.h = enth(gamma, W.eps);
    RT v2 = RT(0.0), vlow[3] = {0, 0, 0}, Blow[3] = {0, 0, 0};
    RT isg = RT(1.0) / sqrtg;
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            vlow[i] += mc.gam[i][j] * W.v[j];
            Blow[i] += mc.gam[i][j] * W.B[j];
        }
        v2 += vlow[i] * W.v[i];
    }
    v2 = smin(v2, 1 - RT(1e-10));
    s.iltz2 = RT(1.0) - v2;               // 1 / ltz2 within an ulp
    s.ltz2 = RT(1.0) / s.iltz2;
    RT Bv = RT(0.0);
#pragma unroll
    for (int i = 0; i < 3; i++) Bv += Blow[i] * W.v[i];
    RT Bsq = RT(0.0);
#pragma unroll
    for (int i = 0; i < 3; i++) Bsq += Blow[i] * W.B[i];
    s.b2 = Bv * Bv + quo(Bsq, s.ltz2, s.iltz2);
    s.vn = W.v[dim]; s.vt1 = W.v[t1]; s.vt2 = W.v[t2];
    s.Bn = W.B[dim]; s.Bt1 = W.B[t1]; s.Bt2 = W.B[t2];
    s.pt = s.p + s.b2 / 2;
    RT cs2 = cs2f(gamma, W.rho, W.eps);
    s.cf = fastspeed(s.rho, s.h, s.b2, cs2);
    s.D = quo(U.D, sqrtg, isg); s.tau = quo(U.tau, sqrtg, isg);
    s.Sn = quo(U.S[dim], sqrtg, isg); s.St1 = quo(U.S[t1], sqrtg, isg); s.St2 = quo(U.S[t2], sqrtg, isg);
    s.Bc = quo(U.B[dim], sqrtg, isg);
    s.E = s.tau + s.D;
    return ok;
}
template <typename RT>
BH_HD inline CstT<RT> physflux(const SideT<RT>& s, RT a, RT btn) {     // :97-122
    CstT<RT> F;
    RT vn = s.vn;
    F.D = s.D * vn;
    F.tau = (s.E + s.pt) * vn - quo(s.Bn * (s.Bn * vn + s.Bt1 * s.vt1 + s.Bt2 * s.vt2), s.ltz2, s.iltz2);
    F.Sn = s.Sn * vn - quo(s.Bn * s.Bn, s.ltz2, s.iltz2) + s.pt;
    F.St1 = s.St1 * vn - quo(s.Bt1 * s.Bn, s.ltz2, s.iltz2);
    F.St2 = s.St2 * vn - quo(s.Bt2 * s.Bn, s.ltz2, s.iltz2);
    F.Bn = RT(0.0);
    F.Bt1 = s.Bt1 * vn - s.Bn * s.vt1;
    F.Bt2 = s.Bt2 * vn - s.Bn * s.vt2;
    F.D = a * F.D - btn * s.D;
    F.tau = a * F.tau - btn * s.tau;
    F.Sn = a * F.Sn - btn * s.Sn;
    F.St1 = a * F.St1 - btn * s.St1;
    F.St2 = a * F.St2 - btn * s.St2;
    F.Bn = a * F.Bn - btn * s.Bn;
    F.Bt1 = a * F.Bt1 - btn * s.Bt1;
    F.Bt2 = a * F.Bt2 - btn * s.Bt2;
    return F;
}
template <typename RT>
BH_HD inline CstT<RT> hll_flux(const SideT<RT>& L, const SideT<RT>& R, const CstT<RT>& FL, const CstT<RT>& FR, RT SL,
                                        RT SR) {                            // :124-137
    RT dS = SR - SL, idS = RT(1.0) / dS;
    CstT<RT> F;
    F.D = quo(SR * FL.D - SL * FR.D + SL * SR * (R.D - L.D), dS, idS);
    F.tau = quo(SR * FL.tau - SL * FR.tau + SL * SR * (R.tau - L.tau), dS, idS);
    F.Sn = quo(SR * FL.Sn - SL * FR.Sn + SL * SR * (R.Sn - L.Sn), dS, idS);
    F.St1 = quo(SR * FL.St1 - SL * FR.St1 + SL * SR * (R.St1 - L.St1), dS, idS);
    F.St2 = quo(SR * FL.St2 - SL * FR.St2 + SL * SR * (R.St2 - L.St2), dS, idS);
    F.Bn = quo(SR * FL.Bn - SL * FR.Bn + SL * SR * (R.Bn - L.Bn), dS, idS);
    F.Bt1 = quo(SR * FL.Bt1 - SL * FR.Bt1 + SL * SR * (R.Bt1 - L.Bt1), dS, idS);
    F.Bt2 = quo(SR * FL.Bt2 - SL * FR.Bt2 + SL * SR * (R.Bt2 - L.Bt2), dS, idS);
    return F;
}
template <typename RT>
BH_HD inline CstT<RT> star_stt(const SideT<RT>& s, RT SK, RT SM, RT pt_x) {  // :140-159
    CstT<RT> Ux;
    RT dK = SK - SM, idK = RT(1.0) / dK;
    Ux.D = quo(s.D * (SK - s.vn), dK, idK);
    Ux.tau = quo(s.E * (SK - s.vn) - s.pt * s.vn + pt_x * SM, dK, idK) - Ux.D;
    Ux.Sn = quo(s.Sn * (SK - s.vn) - s.pt + pt_x, dK, idK);
    Ux.St1 = quo(s.St1 * (SK - s.vn), dK, idK);
    Ux.St2 = quo(s.St2 * (SK - s.vn), dK, idK);
    Ux.Bn = s.Bc;
    RT den = s.D * (SK - s.vn) * (SK - SM) - s.Bn * s.Bn;
    if (fabs(den) > RT(1e-14)) {
        RT k = s.Bn * (SM - s.vn) / den;
        RT iD = RT(1.0) / s.D;
        Ux.Bt1 = s.Bt1 - s.Bn * (s.vt1 * (SK - s.vn) + quo(s.Bn * s.Bt1, s.D, iD)) * k;
        Ux.Bt2 = s.Bt2 - s.Bn * (s.vt2 * (SK - s.vn) + quo(s.Bn * s.Bt2, s.D, iD)) * k;
    } else {
        Ux.Bt1 = s.Bt1; Ux.Bt2 = s.Bt2;
    }
    return Ux;
}
// alfstar_stt (:161-201); its degenerate branch (:171-173) is overwritten
// by the assignments after it and has no effect
template <typename RT>
BH_HD inline void alfstar_stt(const CstT<RT>& UxL, const CstT<RT>& UxR, RT Bn, RT SM, CstT<RT>& UxxL,
                                            CstT<RT>& UxxR) {
    UxxL.D = UxL.D; UxxL.tau = UxL.tau;
    UxxR.D = UxR.D; UxxR.tau = UxR.tau;
    UxxL.Bn = UxL.Bn; UxxR.Bn = UxR.Bn;
    RT sq_DL = sqrt(fabs(UxL.D));
    RT sq_DR = sqrt(fabs(UxR.D));
    RT den = sq_DL + sq_DR;
    RT iden = RT(1.0) / den, iDL = RT(1.0) / UxL.D, iDR = RT(1.0) / UxR.D;
    RT sgnBn = (Bn >= RT(0.0)) ? RT(1.0) : -RT(1.0);
    RT vt1xx = quo(quo(sq_DL * UxL.St1, UxL.D, iDL) + quo(sq_DR * UxR.St1, UxR.D, iDR) + sgnBn * (UxR.Bt1 - UxL.Bt1),
                   den, iden);
    RT vt2xx = quo(quo(sq_DL * UxL.St2, UxL.D, iDL) + quo(sq_DR * UxR.St2, UxR.D, iDR) + sgnBn * (UxR.Bt2 - UxL.Bt2),
                   den, iden);
    RT Bt1xx = quo(quo(sq_DL * UxL.Bt1, UxL.D, iDL) + quo(sq_DR * UxR.Bt1, UxR.D, iDR) +
                       sgnBn * sq_DL * sq_DR * (quo(UxR.St1, UxR.D, iDR) - quo(UxL.St1, UxL.D, iDL)),
                   den, iden);
    RT Bt2xx = quo(quo(sq_DL * UxL.Bt2, UxL.D, iDL) + quo(sq_DR * UxR.Bt2, UxR.D, iDR) +
                       sgnBn * sq_DL * sq_DR * (quo(UxR.St2, UxR.D, iDR) - quo(UxL.St2, UxL.D, iDL)),
                   den, iden);
    UxxL.St1 = UxL.D * vt1xx; UxxR.St1 = UxR.D * vt1xx;
    UxxL.St2 = UxL.D * vt2xx; UxxR.St2 = UxR.D * vt2xx;
    UxxL.Bt1 = Bt1xx; UxxR.Bt1 = Bt1xx;
    UxxL.Bt2 = Bt2xx; UxxR.Bt2 = Bt2xx;
    UxxL.Sn = UxL.D * SM; UxxR.Sn = UxR.D * SM;
    const RT vt1xL = quo(UxL.St1, UxL.D, iDL), vt2xL = quo(UxL.St2, UxL.D, iDL);
    const RT vt1xR = quo(UxR.St1, UxR.D, iDR), vt2xR = quo(UxR.St2, UxR.D, iDR);
    RT dE_L = sq_DL * sgnBn * (vt1xx * Bt1xx + vt2xx * Bt2xx - vt1xL * UxL.Bt1 - vt2xL * UxL.Bt2);
    RT dE_R = sq_DR * sgnBn * (vt1xx * Bt1xx + vt2xx * Bt2xx - vt1xR * UxR.Bt1 - vt2xR * UxR.Bt2);
    UxxL.tau = UxL.tau - dE_L;
    UxxR.tau = UxR.tau + dE_R;
}
template <typename RT>
BH_HD inline CstT<RT> interflux(const CstT<RT>& FK, RT SK, const CstT<RT>& Ux, const SideT<RT>& s) {  // :203-216
    CstT<RT> F;
    F.D = FK.D + SK * (Ux.D - s.D);
    F.tau = FK.tau + SK * (Ux.tau - (s.E - s.D));
    F.Sn = FK.Sn + SK * (Ux.Sn - s.Sn);
    F.St1 = FK.St1 + SK * (Ux.St1 - s.St1);
    F.St2 = FK.St2 + SK * (Ux.St2 - s.St2);
    F.Bn = FK.Bn + SK * (Ux.Bn - s.Bc);
    F.Bt1 = FK.Bt1 + SK * (Ux.Bt1 - s.Bt1);
    F.Bt2 = FK.Bt2 + SK * (Ux.Bt2 - s.Bt2);
    return F;
}
// flux (:218-227): out in cons order D,S0,S1,S2,tau,B0,B1,B2, times sqrt(-g)
template <typename RT>
BH_HD inline void flux_out(const CstT<RT>& F, RT sg, int dim, RT o[8]) {
    int t1 = (dim + 1) % 3, t2 = (dim + 2) % 3;
    o[0] = sg * F.D; o[4] = sg * F.tau;
    o[5 + dim] = sg * F.Bn; o[5 + t1] = sg * F.Bt1; o[5 + t2] = sg * F.Bt2;
    o[1 + dim] = sg * F.Sn; o[1 + t1] = sg * F.St1; o[1 + t2] = sg * F.St2;
}
// hlld (:230-312); returns false where the reference throws
template <typename RT>
BH_HD inline bool hlld(RT gamma, const MetT<RT>& mc, const PrimT<RT>& WL, const PrimT<RT>& WR, const ConsT<RT>& UL,
                            const ConsT<RT>& UR, int dim, RT Fo[8], RT& ctspeed) {
    RT sg = mc.sqrtdetg;
    SideT<RT> L, R;
    bool ok = side_(gamma, WL, UL, mc, sg, dim, L);
    ok &= side_(gamma, WR, UR, mc, sg, dim, R);
    RT a = mc.alpha, bd = mc.beta[dim];
    RT SL = smin(a * (L.vn - L.cf) - bd, a * (R.vn - R.cf) - bd);
    RT SR = smax(a * (L.vn + L.cf) - bd, a * (R.vn + R.cf) - bd);
    CstT<RT> FL = physflux(L, a, bd), FR = physflux(R, a, bd);
    RT cts = smax(fabs(SL), fabs(SR));
    ctspeed = cts;
    // :244-246 computes an HLL flux that every later path overwrites
    if (SL >= RT(0.0)) { flux_out(FL, sg, dim, Fo); return ok; }
    if (SR <= RT(0.0)) { flux_out(FR, sg, dim, Fo); return ok; }
    RT pt_x = (SR * L.pt - SL * R.pt + SL * SR * (R.Sn - L.Sn)) / (SR - SL);
    RT SM_u = SR * L.E - SL * R.E - FR.tau - FR.D + FL.tau + FL.D;
    RT SM_d = SR * L.D - SL * R.D - FR.D + FL.D;
    if (fabs(SM_d) < RT(1e-12)) { flux_out(hll_flux(L, R, FL, FR, SL, SR), sg, dim, Fo); return ok; }
    RT SM = SM_u / SM_d;
    CstT<RT> UxL = star_stt(L, SL, SM, pt_x);
    CstT<RT> UxR = star_stt(R, SR, SM, pt_x);
    RT SLx = SM - fabs(L.Bn) / sqrt(fabs(UxL.D));
    RT SRx = SM + fabs(R.Bn) / sqrt(fabs(UxR.D));
    if (UxL.D <= RT(0.0) || UxR.D <= RT(0.0)) { flux_out(hll_flux(L, R, FL, FR, SL, SR), sg, dim, Fo); return ok; }
    CstT<RT> Fs;
    if (SM >= RT(0.0)) {
        if (SLx >= RT(0.0)) {
            Fs = interflux(FL, SL, UxL, L);
        } else {
            CstT<RT> UxxL, UxxR;
            alfstar_stt(UxL, UxR, L.Bn, SM, UxxL, UxxR);
            CstT<RT> FLx = interflux(FL, SL, UxL, L);
            Fs = interflux(FLx, SLx, UxxL, L);
        }
    } else {
        if (SRx >= RT(0.0)) {
            Fs = interflux(FR, SR, UxR, R);
        } else {
            CstT<RT> UxxL, UxxR;
            alfstar_stt(UxL, UxR, L.Bn, SM, UxxL, UxxR);
            CstT<RT> FRx = interflux(FR, SR, UxR, R);
            Fs = interflux(FRx, SRx, UxxR, R);
        }
    }
    RT F[8];
    flux_out(Fs, sg, dim, F);
    bool fin = true;
#pragma unroll
    for (int q = 0; q < 8; q++) fin &= isfinite(F[q]);
    if (!fin || cts > RT(1.0)) {
        flux_out(hll_flux(L, R, FL, FR, SL, SR), sg, dim, F);
        if (cts > RT(1.0)) ctspeed = smin(cts, RT(1.0));
    }
#pragma unroll
    for (int q = 0; q < 8; q++) Fo[q] = F[q];
    return ok;
}

// ======================================================================
// PLM reconstruction (recon.hpp:16-41, grid/reconstruction.cpp:28-97)
// ======================================================================
template <typename RT>
BH_HD inline RT minmod(RT a, RT b) {
    if (a * b <= RT(0.0)) return RT(0.0);
    return (fabs(a) < fabs(b)) ? a : b;
}
template <typename RT>
BH_HD inline RT vanleer(RT a, RT b) {
    if (a * b <= RT(0.0)) return RT(0.0);
    return RT(2.0) * a * b / (a + b);
}
template <typename RT>
BH_HD inline RT mclim(RT a, RT b) {
    if (a * b <= RT(0.0)) return RT(0.0);
    RT c = (a + b) / 2;
    RT s = (a > RT(0.0)) ? RT(1.0) : -RT(1.0);
    return s * minmod(fabs(2 * a), minmod(fabs(2 * b), fabs(c)));
}
template <typename RT>
BH_HD inline RT limit(RT dl, RT dr, int lim) {
    return lim == BH_VANLEER ? vanleer(dl, dr) : lim == BH_MC ? mclim(dl, dr) : minmod(dl, dr);
}
template <typename RT>
BH_HD inline void recon_scal(RT Wm, RT Wc, RT Wp, RT Wpp, int lim, RT& fL,
                                           RT& fR) {
    fL = Wc + limit(Wc - Wm, Wp - Wc, lim) / RT(2.0);
    fR = Wp - limit(Wp - Wc, Wpp - Wp, lim) / RT(2.0);
}
// causality rescale of reconfp (:69-83) with the cell's metric
template <typename RT>
BH_HD inline void causalv_gam(RT v[3], const RT gam[3][3]) {
    RT v2 = RT(0.0);
#pragma unroll
    for (int m = 0; m < 3; m++)
#pragma unroll
        for (int n = 0; n < 3; n++) v2 += gam[m][n] * v[m] * v[n];
    if (v2 >= RT(1.0)) {
        RT s = (1 - RT(1e-10)) / sqrt(v2);
#pragma unroll
        for (int a = 0; a < 3; a++) v[a] *= s;
    }
}
template <typename RT>
BH_HD inline void causalv(RT v[3], const MetT<RT>& mc) { causalv_gam(v, mc.gam); }

}  // namespace bh
