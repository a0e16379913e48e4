// bh_init.cuh -- per-item work of the Fishbone-Moncrief torus initial data
// (solver/initconds.cpp:17-668) in the order main() applies it
// (main.cpp:89-160): the floor state of every cell, the torus primitives of
// the interior cells, the face field from the curl of A_phi with its cell
// average, and the interior cells' conserved variables.
//
// Like bh_items.cuh, written once as __host__ __device__ functions; the host
// build (tests/hostcheck) equals the reference bit for bit.
#pragma once
#include "bh_items.cuh"

namespace bh {

#ifdef __CUDA_ARCH__
BH_HD inline double pow_2(double x) { return x * x; }
#else
BH_HD inline double pow_2(double x) { return pow(x, 2); }
#endif

constexpr double HALF_PI = 3.14159265358979323846 / 2.0;   // M_PI/2.0

// scalars fm_init derives before it touches a cell
struct TorusScalars {
    double l0, W_in, lnh_max, r_H, K, gamma;
};

// L0_comp (:121-141): angular momentum of the circular orbit at r_max from
// central differences of the metric at the equator; NaN where the reference
// throws (|B| < 1e-14)
BH_HD inline double fm_L0(const MP& m, double r_max, double M) {
    const double dr = 1e-4 * M;
    MetSrc mc0, mcp, mcm;
    met_src(m, r_max, HALF_PI, mc0);
    met_src(m, r_max + dr, HALF_PI, mcp);
    met_src(m, r_max - dr, HALF_PI, mcm);
    double gtt = mc0.g[0][0], gtp = mc0.g[0][3], gpp = mc0.g[3][3];
    const double dgtt = (mcp.g[0][0] - mcm.g[0][0]) / (2.0 * dr);
    const double dgtp = (mcp.g[0][3] - mcm.g[0][3]) / (2.0 * dr);
    const double dgpp = (mcp.g[3][3] - mcm.g[3][3]) / (2.0 * dr);
    double A = -gtp * (gpp * (dgtt * dgpp + 2 * dgtp * dgtp) + gtt * dgpp * dgpp) +
               sqrt((dgtp * dgtp - dgtt * dgpp) *
                    pow_2((gpp * (gpp * dgtt - gtt * dgpp) + 2 * gtp * gtp * dgpp - 2 * gtp * gpp * dgtp))) +
               gpp * gpp * dgtt * dgtp + gtt * gpp * dgtp * dgpp + 2 * gtp * gtp * dgtp * dgpp;
    double B = dgtt * (gpp * gpp * dgtt + 4 * gtp * gtp * dgpp - 4 * gtp * gpp * dgtp) -
               2 * gtt * (gpp * (dgtt * dgpp - 2 * dgtp * dgtp) + 2 * gtp * dgtp * dgpp) + gtt * gtt * dgpp * dgpp;
    if (fabs(B) < 1e-14) return NAN;
    return A / B;
}

// locally non-rotating frame (:151-171)
struct Lnrf { double e2nu, e2psi, enu, epsi, omega; };
BH_HD inline Lnrf lnrf_of(const MetSrc& mc) {
    const double gtt = mc.g[0][0], gtp = mc.g[0][3], gpp = mc.g[3][3];
    Lnrf lp;
    lp.e2nu = gtp * gtp / gpp - gtt;
    lp.e2psi = gpp;
    lp.enu = sqrt(lp.e2nu);
    lp.epsi = sqrt(lp.e2psi);
    lp.omega = -gtp / gpp;
    return lp;
}
// torus potentials (:173-185)
BH_HD inline double lnh_pot(const MetSrc& mc, double l, double W_in) {
    const Lnrf lp = lnrf_of(mc);
    if (lp.e2nu <= 0.0) return -1e30;
    return -0.5 * sqrt((4 * l * l * lp.e2nu) / lp.e2psi + 1) +
           0.5 * log((sqrt((4 * l * l * lp.e2nu) / lp.e2psi + 1) + 1) / lp.e2nu) - l * lp.omega + W_in;
}
BH_HD inline double W_in_of(const MetSrc& mc, double l) {
    const Lnrf lp = lnrf_of(mc);
    if (lp.e2nu <= 0.0) return -1e30;
    return 0.5 * sqrt((4 * l * l * lp.e2nu) / lp.e2psi + 1) -
           0.5 * log((sqrt((4 * l * l * lp.e2nu) / lp.e2psi + 1) + 1) / lp.e2nu) + l * lp.omega;
}
// disctherm (:187-204): polytrope rho, p, eps from ln h
BH_HD inline void disctherm(double lnH, double Gamma, double K, double& rho, double& p, double& eps) {
    if (lnH <= 0.0) { rho = p = eps = 0.0; return; }
    const double H = exp(lnH);
    const double arg = (Gamma - 1) * (H - 1) / (Gamma * K);
    if (arg <= 0.0) { rho = p = eps = 0.0; return; }
    rho = pow(arg, 1.0 / (Gamma - 1.0));
    p = K * pow(arg, Gamma / (Gamma - 1.0));
    eps = p / ((Gamma - 1.0) * rho);
}
// velcomp (:206-226): Cartesian 3-velocity of the circular flow
BH_HD inline void velcomp(const MetSrc& mc, const Lnrf& lp, double l, double xc, double yc, double v[3]) {
    v[0] = v[1] = v[2] = 0.0;
    const double u_phi = sqrt(0.5 * (sqrt(1.0 + 4.0 * l * l * lp.e2nu / lp.e2psi) - 1.0));
    const double uphi = u_phi / lp.epsi + (lp.omega / lp.enu) * sqrt(1.0 + u_phi * u_phi);
    const double gtt = mc.g[0][0], gtp = mc.g[0][3], gpp = mc.g[3][3];
    const double B = 2.0 * gtp * uphi;
    const double C = gpp * uphi * uphi + 1.0;
    const double D = B * B - 4.0 * gtt * C;
    if (D < 0.0) return;
    const double ut = (-B - sqrt(D)) / (2.0 * gtt);
    const double Omega = uphi / ut;
    const double vphi = Omega - mc.beta[2] / mc.alpha;
    const double rcyl = sqrt(xc * xc + yc * yc);
    if (rcyl < 1e-10) return;
    v[0] = -vphi * yc; v[1] = vphi * xc; v[2] = 0.0;
}

// the scalars of fm_init (:228-420): l0, W_in at r_in, ln h at r_max
BH_HD inline TorusScalars fm_scalars(const MP& m, double gamma, double r_max, double r_in) {
    TorusScalars s;
    const double M = m.M, a = m.a, Q = m.Q;
    s.r_H = M + sqrt(M * M - a * a - Q * Q);
    s.K = 0.001 * pow(M, gamma - 1.0);
    s.gamma = gamma;
    s.l0 = fm_L0(m, r_max, M);
    MetSrc mc_in, mc_max;
    met_src(m, r_in, HALF_PI, mc_in);
    s.W_in = W_in_of(mc_in, s.l0);
    met_src(m, r_max, HALF_PI, mc_max);
    s.lnh_max = lnh_pot(mc_max, s.l0, s.W_in);
    return s;
}

// the cell tests of fm_init's loops (:459-464, 519-527)
BH_HD inline bool fm_skip(double r, double th, double r_H) {
    return !isfinite(r) || !isfinite(th) || r <= 1.05 * r_H || fabs(sin(th)) < 0.01;
}

// rho of interior cell c of patch p before normalisation (:455-479), or
// -1 where the cell does not count
BH_HD inline double fm_cell_rho(const KP& kp, const Pool& P, int p, int c, const TorusScalars& s) {
    int l = lindx(c / 256, (c / 16) % 16, c % 16);
    double r = rr(P, p, l), th = tt(P, p, l);
    if (fm_skip(r, th, s.r_H)) return -1.0;
    MetSrc mc;
    met_src(kp.tree, r, th, mc);
    const double lnH = lnh_pot(mc, s.l0, s.W_in);
    if (lnH <= 0.0 || !isfinite(lnH)) return -1.0;
    double rho, pr, eps;
    disctherm(lnH, s.gamma, s.K, rho, pr, eps);
    return isfinite(rho) ? rho : -1.0;
}

// the primitives fm_init gives interior cell c (:512-585): the floor state
// (pvfs, already in W) outside the torus, else the scaled polytrope with
// the circular velocity
BH_HD inline void fm_cell_prims(const KP& kp, const Pool& P, int p, int c, const TorusScalars& s, double rho_scal) {
    int i = c / 256, j = (c / 16) % 16, k = c % 16;
    int l = lindx(i, j, k);
    double r = rr(P, p, l), th = tt(P, p, l);
    double fr, fe;
    pvfs(r, fr, fe);
    double rho = fr, eps = fe, v[3] = {0.0, 0.0, 0.0};
    if (!fm_skip(r, th, s.r_H)) {
        MetSrc mc;
        met_src(kp.tree, r, th, mc);
        const double lnH = lnh_pot(mc, s.l0, s.W_in);
        if (!(lnH <= 0.0 || !isfinite(lnH))) {
            double trho, tp, te;
            disctherm(lnH, s.gamma, s.K, trho, tp, te);
            rho = rho_scal * trho;
            double pr = s.K * pow(rho, s.gamma);
            eps = pr / ((s.gamma - 1.0) * rho);
            const double* g = P.pgeo + 6 * p;
            double xc = g[0] + (i + 0.5) * g[3], yc = g[1] + (j + 0.5) * g[4];
            velcomp(mc, lnrf_of(mc), s.l0, xc, yc, v);
        }
    }
    Wv(P, p, 0)[l] = rho; Wv(P, p, 1)[l] = eps;
    for (int d = 0; d < 3; d++) { Wv(P, p, 2 + d)[l] = v[d]; Wv(P, p, 5 + d)[l] = 0.0; }
}

// the floor state of the amrtree constructor for cell l (grid.cpp:191-205):
// W = pvfs(r), U = ptoc(W)
BH_HD inline void floor_cell(const KP& kp, const Pool& P, int p, int l) {
    Prim w;
    pvfs(rr(P, p, l), w.rho, w.eps);
    w.v[0] = w.v[1] = w.v[2] = 0.0;
    w.B[0] = w.B[1] = w.B[2] = 0.0;
    Met mc;
    met_comp(kp.tree, rr(P, p, l), tt(P, p, l), mc);
    Cons u;
    if (!ptoc(kp.gamma, mc, w, u)) flag(P.err, BH_ERR_DOMAIN);
    store_prim(P, p, l, w);
    store_cons(P, p, l, u);
}

// interior cell c: U = ptoc(W) (main.cpp:147-157)
BH_HD inline void ptoc_interior_item(const KP& kp, const Pool& P, int p, int c) {
    int l = lindx(c / 256, (c / 16) % 16, c % 16);
    Prim w;
    load_prim(P, p, l, w);
    Met mc;
    met_comp(kp.tree, rr(P, p, l), tt(P, p, l), mc);
    Cons u;
    if (!ptoc(kp.gamma, mc, w, u)) flag(P.err, BH_ERR_DOMAIN);
    store_cons(P, p, l, u);
}

// ---- B_pot_init (:594-667): face B = curl of A_phi sampled at cell edges ---
BH_HD inline void A_vpot(double x, double y, double z, double rho, double rho_max, double A[3]) {   // :17-23
    double Ap = smax(rho / rho_max - 0.2, 0.0);
    double phi = atan2(y, x);
    double theta = acos(z / sqrt(x * x + y * y + z * z));
    A[0] = -Ap * sin(phi) * sin(theta);
    A[1] = Ap * cos(phi) * sin(theta);
    A[2] = 0.0;
}
BH_HD inline int clampc(int i) { return i < BLK + GH - 1 ? i : BLK + GH - 1; }   // std::min(i, block+ghost-1)
BH_HD inline double edge_rho(const Pool& P, int p, int axis, int i, int j, int k) {       // :25-40
    const double* rho = Wv(P, p, 0);
    if (axis == 0) {
        int j1 = clampc(j + 1), k1 = clampc(k + 1);
        return (rho[lindx(i, j, k)] + rho[lindx(i, j1, k)] + rho[lindx(i, j, k1)] + rho[lindx(i, j1, k1)]) / 4;
    }
    if (axis == 1) {
        int i1 = clampc(i + 1), k1 = clampc(k + 1);
        return (rho[lindx(i, j, k)] + rho[lindx(i1, j, k)] + rho[lindx(i, j, k1)] + rho[lindx(i1, j, k1)]) / 4;
    }
    int i1 = clampc(i + 1), j1 = clampc(j + 1);
    return (rho[lindx(i, j, k)] + rho[lindx(i1, j, k)] + rho[lindx(i, j1, k)] + rho[lindx(i1, j1, k)]) / 4;
}
// A component `comp` at the edge of direction `axis` of cell (i, j, k) (:41-52)
BH_HD inline double A_edge(const Pool& P, int p, int axis, int i, int j, int k, double rho_max, int comp) {
    const double* g = P.pgeo + 6 * p;
    double xc = g[0] + (i + 0.5) * g[3], yc = g[1] + (j + 0.5) * g[4], zc = g[2] + (k + 0.5) * g[5];
    double x = xc, y = yc, z = zc;
    if (axis == 0) { y = yc + g[4] / 2.0; z = zc + g[5] / 2.0; }
    else if (axis == 1) { x = xc + g[3] / 2.0; z = zc + g[5] / 2.0; }
    else { x = xc + g[3] / 2.0; y = yc + g[4] / 2.0; }
    double A[3];
    A_vpot(x, y, z, edge_rho(P, p, axis, i, j, k), rho_max, A);
    return A[comp];
}
// the three faces of item e = (i, j, k) in [-1, 18)^3 (:603-664)
BH_HD inline void bpot_item(const Pool& P, int p, int e, double rho_max) {
    int i = e / 361 - 1, j = (e / 19) % 19 - 1, k = e % 19 - 1;
    const double* g = P.pgeo + 6 * p;
    double dx = g[3], dy = g[4], dz = g[5];
    // Bfx: y edges (k, k-1) and z edges (j, j-1)
    double Ay_kp = A_edge(P, p, 1, i, j, k, rho_max, 1), Ay_km = A_edge(P, p, 1, i, j, k - 1, rho_max, 1);
    double Az_jp = A_edge(P, p, 2, i, j, k, rho_max, 2), Az_jm = A_edge(P, p, 2, i, j - 1, k, rho_max, 2);
    Bfv(P, p, 0)[xfc(i, j, k)] = (Az_jp - Az_jm) / dy - (Ay_kp - Ay_km) / dz;
    // Bfy: x edges (k, k-1) and z edges (i, i-1)
    double Ax_kp = A_edge(P, p, 0, i, j, k, rho_max, 0), Ax_km = A_edge(P, p, 0, i, j, k - 1, rho_max, 0);
    double Az_ip = A_edge(P, p, 2, i, j, k, rho_max, 2), Az_im = A_edge(P, p, 2, i - 1, j, k, rho_max, 2);
    Bfv(P, p, 1)[yfc(i, j, k)] = (Ax_kp - Ax_km) / dz - (Az_ip - Az_im) / dx;
    // Bfz: x edges (i, i-1) and y edges (j, j-1) -- the reference names them
    // the other way round but samples exactly these
    double Ay_ip = A_edge(P, p, 0, i, j, k, rho_max, 1), Ay_im = A_edge(P, p, 0, i - 1, j, k, rho_max, 1);
    double Ax_jp = A_edge(P, p, 1, i, j, k, rho_max, 0), Ax_jm = A_edge(P, p, 1, i, j - 1, k, rho_max, 0);
    Bfv(P, p, 2)[zfc(i, j, k)] = (Ay_ip - Ay_im) / dx - (Ax_jp - Ax_jm) / dy;
}

}  // namespace bh
