// bh_fixed.cuh -- kernels and launch sequences of the corrected ("fixed")
// scheme (bh_fixed_phys.cuh), compiled once per arithmetic variant inside
// the variant's namespace (bh_variant.cuh includes this file):
//   RT  arithmetic type of reconstruction, face fluxes and sources
//       (double; float in the mixed variant)
//   WT  storage type of the primitives (the face work's input) and FT of
//       the face fluxes: RT as well, so the mixed variant moves half the
//       bytes of the face work
// Conserved state, face field, con2prim, the CT update and dt stay FP64.
//
// Data: a list of cubic blocks, each n^3 interior cells with FX_GB = 3
// ghost layers, stored per array as a (n+7)^3 box (cells -3..n+3 per axis;
// the extra layer holds the upper faces): index ((i+3) S + (j+3)) S + (k+3)
// with S = n + 7 -- the reference's per-patch order (grid.cpp:51-53: i
// slowest, k fastest).  The ghost fill covers the two layers PLM reads, or
// all three for PPM (Grid::gdepth).  The x-face (i-1/2, j, k), the y-face
// (i, j-1/2, k) and the z-face (i, j, k-1/2) share the index of cell
// (i, j, k); so do the edges
// E_x (i, j-1/2, k-1/2), E_y (i-1/2, j, k-1/2) and E_z (i-1/2, j-1/2, k).
//
// Work: every kernel walks a list of items (block, first index); item t of
// a launch is CTA t, and its threads take consecutive indices of that
// block's index space (interior cells, flux positions or ghost cells), so
// blocks of different sizes share one launch with equal work per CTA.
#pragma once
#include "bh_fixed_phys.cuh"

namespace fx {
namespace {   // internal linkage: every arithmetic variant compiles its own copy
using namespace bhfx;

constexpr int FX_TPB = BH_FX_CHUNK;

struct Grid {
    const bh_fx_block* blk;
    const int32_t* nbr;
    double *U, *U1, *Bf, *Bf1;
    void *W, *F;
    int64_t ncell;
    double* dt;
    int32_t* count;
    int32_t* err;
    double* E;
    int gdepth;   // ghost layers filled: 2, or 3 (PPM)
};
inline Grid grid_of(const bh_fx_grid* g) {
    return Grid{g->blocks, g->nbr, g->U,     g->U1,  g->Bf, g->Bf1, g->W, g->F, g->ncell, g->dt, g->count, g->err,
                g->E,      g->ghost_depth > 2 ? 3 : 2};
}
inline FxPar par_of(const bh_fx_params* p) {
    FxPar q;
    q.M = p->M; q.a = p->a; q.gamma = p->gamma;
    q.rho_fl = p->rho_floor; q.u_fl = p->u_floor; q.sigma_max = p->sigma_max; q.W_max = p->W_max;
    q.r_exc = p->r_exc; q.tol = p->tol; q.maxiter = p->maxiter; q.limiter = p->limiter;
    q.gg = p->gamma / (p->gamma - 1.0);
    q.gf = (p->gamma - 1.0) / p->gamma;
    q.v2max = 1.0 - 1.0 / (p->W_max * p->W_max);
    q.flags = p->flags;
    return q;
}

constexpr int FX_GB = 3;
__device__ inline int64_t bidx(const bh_fx_block& b, int i, int j, int k) {
    const int S = b.n + 2 * FX_GB + 1;
    return b.off + ((int64_t)(i + FX_GB) * S + (j + FX_GB)) * S + (k + FX_GB);
}
__device__ inline int bstride_i(const bh_fx_block& b) { return (b.n + 2 * FX_GB + 1) * (b.n + 2 * FX_GB + 1); }
__device__ inline int bstride_j(const bh_fx_block& b) { return b.n + 2 * FX_GB + 1; }

// ---- positions ---------------------------------------------------------
__device__ inline void cell_centre(const bh_fx_block& b, int i, int j, int k, double* x) {
    x[0] = b.x0[0] + (i + 0.5) * b.dx;
    x[1] = b.x0[1] + (j + 0.5) * b.dx;
    x[2] = b.x0[2] + (k + 0.5) * b.dx;
}

template <typename T>
__device__ inline T* arr(void* base, int64_t ncell, int v) { return (T*)base + (int64_t)v * ncell; }

// ======================================================================
// CFL reduction on the bit patterns of non-negative doubles
// ======================================================================
__device__ inline void atomic_min_pos(double* slot, double v) {
    atomicMin((unsigned long long*)slot, (unsigned long long)__double_as_longlong(v));
}
__device__ inline void atomic_max_pos(double* slot, double v) {
    atomicMax((unsigned long long*)slot, (unsigned long long)__double_as_longlong(v));
}
// ======================================================================
// the item loop.  Without a queue, CTA t takes item t of the launch's work
// list.  With one (the persistent form: a grid of resident CTAs), each CTA
// takes items from a device counter until none is left; the last CTA to
// finish resets the counter for the next launch of the slot, so a step
// needs no extra launch or memset and records into a CUDA graph as is.
// ======================================================================
struct Queue {
    int32_t* head;   // next item (NULL: one CTA per item)
    int32_t* done;   // CTAs finished
    int32_t nitem;
};
// the item bodies are inlined into the kernel: an outlined body would take
// the kernel's parameter structs by address and copy them to local memory
#define FX_INLINE __attribute__((always_inline))
template <typename Body>
__device__ __forceinline__ void for_items(const Queue& q, Body body) {
    if (!q.head) {
        body((int)blockIdx.x);
        return;
    }
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(q.head, 1);
        __syncthreads();
        const int t = s_item;
        __syncthreads();
        if (t >= q.nitem) break;
        body(t);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(q.done, 1) == (int)gridDim.x - 1) {
            *q.head = 0;
            *q.done = 0;
            __threadfence();
        }
    }
}

__global__ void k_fx_dt_init(double* dt) {
    dt[0] = __longlong_as_double(0x7FF0000000000000LL);   // +inf
}

// ======================================================================
// con2prim + floors + excision on every interior cell of the stage buffer
// (U, Bf for stage 0; U1, Bf1 for stage 1); stage 0 also reduces the CFL
// limit into dt[0]
// ======================================================================
// FP64 con2prim of cell c (metric m, cell field Bc) started from its previous
// primitives; where it fails, the previous primitives with the new field
// (counted).  Returns 1 if the conserved state must be rewritten.
template <bool PRE32, typename WT>
__device__ inline int c2p_cell64(const FxPar& P, const Grid& G, const KS& m, const double* U, const WT* W,
                                 int64_t N, int64_t c, const double* Bc, double* w) {
    C2PS cs;
    double wo[5];
    {
        double u[5];
        for (int v = 0; v < 5; v++) u[v] = U[v * N + c];
        for (int v = 0; v < 5; v++) wo[v] = (double)W[v * N + c];
        c2p_setup(P, m, u, Bc, wo, cs);
    }
    int iters = 0;
    int st = c2p_solve<PRE32>(P, cs, iters);
    if (st == 0) st = c2p_finish(m.gi, cs, Bc, w);
    if (st == 0) return 0;
    for (int v = 0; v < 5; v++) w[v] = wo[v];
    for (int d = 0; d < 3; d++) w[P_B + d] = Bc[d];
    atomicAdd(&G.count[0], 1);
    return 1;
}

// the whole FP64 path of a cell: metric, con2prim, floors, excision, the
// rewrite of U where the primitives changed, W and the cell field; returns
// the cell's CFL limit (with_dt)
template <typename RT, typename WT>
__device__ inline double c2p_cell_fp64(const FxPar& P, const Grid& G, const bh_fx_block& B, int64_t c,
                                       const double* x, const double* Bt, double* U, int with_dt) {
    const int64_t N = G.ncell;
    WT* W = (WT*)G.W;
    KS m;
    if (fp32_geometry<RT>(x)) {   // the mixed variant away from the hole: the FP32 metric
        KSb<float> mf;
        ks_metric<float>(P, float(x[0]), float(x[1]), float(x[2]), mf);
        copy_metric(mf, m);
    } else {
        ks_metric(P, x[0], x[1], x[2], m);
    }
    const double Bc[3] = {Bt[0] * m.alpha, Bt[1] * m.alpha, Bt[2] * m.alpha};   // B~ / sqrt(gamma)
    double w[8];
    // (the mixed variant: up to four FP32 Newton iterations start the FP64 ones)
    int rewrite = c2p_cell64<(sizeof(RT) < sizeof(double))>(P, G, m, U, W, N, c, Bc, w);
    if (apply_floors(P, m, w)) {
        rewrite = 1;
        atomicAdd(&G.count[1], 1);
    }
    if (rewrite) {
        KSm<double> mm;
        ks_cast(m, mm);
        Derived<double> d;
        double u[8];
        derive(mm, P.gg, w, d);
        prim2cons(mm, P.gamma, w, d, u);
        for (int v = 0; v < 5; v++) U[v * N + c] = u[v];
    }
    for (int d = 0; d < 3; d++) U[(5 + d) * N + c] = Bt[d];
    for (int v = 0; v < 8; v++) W[v * N + c] = (WT)w[v];
    if (!with_dt) return 1e300;
    const double dx[3] = {B.dx, B.dx, B.dx};
    return cell_dt<RT>(P, m, w, dx);
}

// the mixed variant's FP32 path of a cell (away from the hole): returns 0
// and the cell's CFL limit in dtc when the FP32 con2prim succeeded (W, U
// written), 1 when the cell needs the FP64 path (nothing written)
__device__ inline int c2p_cell_fp32(const FxPar& P, const Grid& G, const bh_fx_block& B, int64_t c, const double* x,
                                    const double* Bt, double* U, int with_dt, double& dtc) {
    const int64_t N = G.ncell;
    float* W = (float*)G.W;
    KSb<float> mf;
    ks_metric<float>(P, float(x[0]), float(x[1]), float(x[2]), mf);
    const float Bcf[3] = {float(Bt[0]) * mf.alpha, float(Bt[1]) * mf.alpha, float(Bt[2]) * mf.alpha};
    float wf[8];
    {
        float u[5], wo[5];
        for (int v = 0; v < 5; v++) u[v] = float(U[v * N + c]);
        for (int v = 0; v < 5; v++) wo[v] = W[v * N + c];
        C2PSb<float> cf;
        c2p_setup(P, mf, u, Bcf, wo, cf);
        int iters = 0;
        if (c2p_solve32(cf, iters) || c2p_finish(mf.gi, cf, Bcf, wf)) return 1;
    }
    if (apply_floors(P, mf, wf)) {
        atomicAdd(&G.count[1], 1);
        KSm<float> mm;
        ks_cast(mf, mm);
        Derived<float> d;
        float uf[8];
        derive(mm, float(P.gg), wf, d);
        prim2cons(mm, float(P.gamma), wf, d, uf);
        for (int v = 0; v < 5; v++) U[v * N + c] = (double)uf[v];
    }
    for (int d = 0; d < 3; d++) U[(5 + d) * N + c] = Bt[d];
    for (int v = 0; v < 8; v++) W[v * N + c] = wf[v];
    if (with_dt) {
        const double dx[3] = {B.dx, B.dx, B.dx};
        dtc = cell_dt<float>(P, mf, wf, dx);
    }
    return 0;
}

// a cell's centre and face-averaged field (the role of f2cB, transport.cpp:60-75)
__device__ inline void c2p_inputs(const Grid& G, const bh_fx_block& B, int i, int j, int k, int stage, double* x,
                                  double* Bt) {
    const int64_t N = G.ncell, c = bidx(B, i, j, k);
    const double* Bf = stage ? G.Bf1 : G.Bf;
    const int si = bstride_i(B), sj = bstride_j(B);
    cell_centre(B, i, j, k, x);
    Bt[0] = 0.5 * (Bf[c] + Bf[c + si]);
    Bt[1] = 0.5 * (Bf[N + c] + Bf[N + c + sj]);
    Bt[2] = 0.5 * (Bf[2 * N + c] + Bf[2 * N + c + 1]);
}

// con2prim + floors + excision on every interior cell.  The mixed variant
// solves in FP32 beyond r ~ FX_R_FP64 where the FP32 residual is well
// conditioned; the other cells take the FP64 path.  (Handing those cells
// to a second kernel through a list, which leaves this one the FP32 path's
// registers, measured slower: the extra launch costs more than the
// registers save.)
template <typename RT, typename WT, int MINB>
__global__ void __launch_bounds__(FX_TPB, MINB) k_fx_c2p(FxPar P, Grid G, const int32_t* items, int stage,
                                                       int with_dt, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n;
        const int e = items[2 * t + 1] + threadIdx.x;
        double dtc = 1e300;
        if (e < n * n * n) {
            const int i = e / (n * n), j = (e / n) % n, k = e % n;
            const int64_t c = bidx(B, i, j, k);
            double* U = stage ? G.U1 : G.U;
            double x[3], Bt[3];
            c2p_inputs(G, B, i, j, k, stage, x, Bt);
            constexpr bool MIXED = sizeof(RT) < sizeof(double);
            int full = 1;
            if (MIXED && fp32_geometry<RT>(x) && !(P.flags & BH_FX_C2P_FP64)) {
                full = c2p_cell_fp32(P, G, B, c, x, Bt, U, with_dt, dtc);
                if (full) atomicAdd(&G.count[2], 1);
            }
            if (full) dtc = c2p_cell_fp64<RT, WT>(P, G, B, c, x, Bt, U, with_dt);
        }
        if (with_dt) {
            for (int o = 16; o > 0; o >>= 1) dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
            if ((threadIdx.x & 31) == 0 && dtc < 1e300) atomic_min_pos(G.dt, dtc);
        }
    });
}

// ======================================================================
// ghost fill: cells of the g ghost layers (edges and corners included)
// take the primitives of the cell they image -- in a neighbour block
// (same size and level) or, across the outer boundary, the nearest
// interior cell (outflow: copy, the role of gh_bndy, grid.cpp:494-522) --
// and the face field of their faces outside the block's own range.
// ======================================================================
// ghost cell e of the g layers around n^3 cells: i in the 2g ghost planes
// first (all j, k), then j (interior i), then k (interior i, j)
__device__ inline int shell_decode(int n, int g, int e, int& i, int& j, int& k) {
    const int m = n + 2 * g, h = 2 * g;
    const int s1 = h * m * m, s2 = h * n * m, s3 = h * n * n;
    if (e < s1) {   // i in {-g..-1, n..n+g-1}, j, k in [-g, n+g)
        int q = e / (m * m), r = e % (m * m);
        i = q < g ? q - g : n + q - g; j = r / m - g; k = r % m - g;
        return 1;
    }
    e -= s1;
    if (e < s2) {   // i in [0,n), j in the ghost planes, k in [-g, n+g)
        int q = e / (n * m), r = e % (n * m);
        i = r / m; k = r % m - g;
        j = q < g ? q - g : n + q - g;
        return 1;
    }
    e -= s2;
    if (e < s3) {   // i, j in [0,n), k in the ghost planes
        int q = e / (n * n), r = e % (n * n);
        i = r / n; j = r % n;
        k = q < g ? q - g : n + q - g;
        return 1;
    }
    return 0;
}

// the source of ghost position (i, j, k) (cell, or face of normal fdim
// when fdim >= 0): block and in-block coordinates
__device__ inline int ghost_source(const Grid& G, int b, int n, int fdim, int& i, int& j, int& k) {
    int c[3] = {i, j, k};
    int o[3];
    const int32_t* nb = G.nbr + (int64_t)b * 27;
    for (int d = 0; d < 3; d++) {
        int hi = (d == fdim) ? n : n - 1;   // a face's normal index runs to n
        o[d] = c[d] < 0 ? -1 : (c[d] > hi ? 1 : 0);
        if (o[d] != 0) {
            int face_nb = nb[(d == 0 ? (o[d] + 1) * 9 + 4 : d == 1 ? 9 + (o[d] + 1) * 3 + 1 : 12 + o[d] + 1)];
            if (face_nb < 0) {   // outer boundary: outflow
                c[d] = c[d] < 0 ? 0 : hi;
                o[d] = 0;
            }
        }
    }
    int src = nb[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)];
    if (src < 0) src = b;
    i = c[0] - o[0] * n; j = c[1] - o[1] * n; k = c[2] - o[2] * n;
    return src;
}

// Where the image lies in a block of another level (blocks are equal cubes,
// one level apart at most): a finer source is averaged (restriction, the 8
// cells or 4 faces that cover the ghost), a coarser one is interpolated
// (prolongation: the covering coarse cell plus a quarter of its
// minmod-limited slope towards the ghost cell in each direction; a face
// takes the coarse face it lies on, or the mean of the two it lies between).
// Pass 0 fills the copies and restrictions; pass l > 0 the prolongations
// into the blocks of level l, whose coarse sources' ghosts earlier passes
// have filled.
__device__ inline double mm_slope(double a, double b, double c) {   // minmod of the two differences
    double l = b - a, r = c - b;
    if (l * r <= 0.0) return 0.0;
    return fabs(l) < fabs(r) ? l : r;
}
template <typename WT>
__global__ void __launch_bounds__(FX_TPB) k_fx_ghost(Grid G, const int32_t* items, int stage, int pass, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        if (pass > 0 && B.level != pass) return;
        const int n = B.n;
        const int e = items[2 * t + 1] + threadIdx.x;
        int i, j, k;
        if (!shell_decode(n, G.gdepth, e, i, j, k)) return;
        const int64_t N = G.ncell;
        WT* W = (WT*)G.W;
        double* Bf = stage ? G.Bf1 : G.Bf;
        const int64_t c = bidx(B, i, j, k);
        {
            int si = i, sj = j, sk = k;
            int s = ghost_source(G, b, n, -1, si, sj, sk);
            const bh_fx_block S = G.blk[s];
            const int kind = S.n == n ? 0 : (S.n > n ? 1 : 2);   // copy, restrict, prolong
            if ((kind == 2) == (pass > 0)) {
                if (kind == 0) {
                    const int64_t sc = bidx(S, si, sj, sk);
                    for (int v = 0; v < 8; v++) W[v * N + c] = W[v * N + sc];
                } else if (kind == 1) {
                    for (int v = 0; v < 8; v++) {
                        double sum = 0.0;
                        for (int a = 0; a < 2; a++)
                            for (int q = 0; q < 2; q++)
                                for (int r = 0; r < 2; r++)
                                    sum += (double)W[v * N + bidx(S, 2 * si + a, 2 * sj + q, 2 * sk + r)];
                        W[v * N + c] = (WT)(0.125 * sum);
                    }
                } else {
                    const int ic = si >> 1, jc = sj >> 1, kc = sk >> 1;
                    const double gx = (si & 1) ? 0.25 : -0.25, gy = (sj & 1) ? 0.25 : -0.25, gz = (sk & 1) ? 0.25 : -0.25;
                    for (int v = 0; v < 8; v++) {
                        const WT* Wv = W + v * N;
                        double w0 = (double)Wv[bidx(S, ic, jc, kc)];
                        double sx = mm_slope((double)Wv[bidx(S, ic - 1, jc, kc)], w0, (double)Wv[bidx(S, ic + 1, jc, kc)]);
                        double sy = mm_slope((double)Wv[bidx(S, ic, jc - 1, kc)], w0, (double)Wv[bidx(S, ic, jc + 1, kc)]);
                        double sz = mm_slope((double)Wv[bidx(S, ic, jc, kc - 1)], w0, (double)Wv[bidx(S, ic, jc, kc + 1)]);
                        W[v * N + c] = (WT)(w0 + gx * sx + gy * sy + gz * sz);
                    }
                }
            }
        }
        // the lower faces of this ghost cell that the flux kernel reads: normal
        // index 0..n, transverse index -1..n, outside the block's own faces
        // (transverse 0..n-1)
        for (int d = 0; d < 3; d++) {
            int cc[3] = {i, j, k};
            if (cc[d] < 0 || cc[d] > n) continue;
            bool need = true;
            for (int q = 0; q < 3; q++)
                if (q != d && (cc[q] < -1 || cc[q] > n)) need = false;
            if (!need) continue;
            int t[3] = {i, j, k};
            int s = ghost_source(G, b, n, d, t[0], t[1], t[2]);
            const bh_fx_block S = G.blk[s];
            const int kind = S.n == n ? 0 : (S.n > n ? 1 : 2);
            if ((kind == 2) != (pass > 0)) continue;
            const double* Bd = Bf + d * N;
            double v;
            if (kind == 0) {
                v = Bd[bidx(S, t[0], t[1], t[2])];
            } else if (kind == 1) {
                // the 4 fine faces on this coarse face
                int f[3] = {2 * t[0], 2 * t[1], 2 * t[2]};
                const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                double sum = 0.0;
                for (int a = 0; a < 2; a++)
                    for (int q = 0; q < 2; q++) {
                        int g[3] = {f[0], f[1], f[2]};
                        g[t1] += a;
                        g[t2] += q;
                        sum += Bd[bidx(S, g[0], g[1], g[2])];
                    }
                v = 0.25 * sum;
            } else {
                int g[3] = {t[0] >> 1, t[1] >> 1, t[2] >> 1};
                if (t[d] & 1) {   // between two coarse faces
                    int h[3] = {g[0], g[1], g[2]};
                    h[d] += 1;
                    v = 0.5 * (Bd[bidx(S, g[0], g[1], g[2])] + Bd[bidx(S, h[0], h[1], h[2])]);
                } else {
                    v = Bd[bidx(S, g[0], g[1], g[2])];
                }
            }
            Bf[d * N + c] = v;
        }
    });
}

// ======================================================================
// face fluxes: one thread per position (i, j, k) in [-1, n]^3 computes the
// HLL flux at the lower x-, y- and z-face of that position where the face
// is needed: normal index 0..n and transverse index -1..n (the transverse
// layer feeds the EMFs of the block's boundary edges)
// ======================================================================
// the face computation; sten(v, o) is variable v of the cell o = -2..1
// (PLM) or -3..2 (PPM, where PPM6) steps along d from (i, j, k) (the face
// lies between o = -1 and o = 0)
template <typename RT, typename FT, bool PPM6, typename Sten>
__device__ __forceinline__ void face_flux_at(const FxPar& P, const Grid& G, const bh_fx_block& B, int i, int j, int k,
                                             int d, const double* Bfs, const Sten& sten) {
    const int64_t N = G.ncell;
    const int64_t c = bidx(B, i, j, k);
    KSm<RT> m;
    if (sizeof(RT) < sizeof(double)) {
        // the face centre in FP32 (exact on these grids: binary spacings),
        // FP64 only where the metric is evaluated in FP64
        const float h = float(B.dx);
        float xf[3] = {float(B.x0[0]) + (float(i) + 0.5f) * h, float(B.x0[1]) + (float(j) + 0.5f) * h,
                       float(B.x0[2]) + (float(k) + 0.5f) * h};
        xf[d] -= 0.5f * h;
        if (xf[0] * xf[0] + xf[1] * xf[1] + xf[2] * xf[2] > float(FX_R_FP64 * FX_R_FP64)) {
            KSb<float> mf;
            ks_metric<float>(P, xf[0], xf[1], xf[2], mf);
            ks_cast(mf, m);
        } else {
            double x[3];
            cell_centre(B, i, j, k, x);
            x[d] -= 0.5 * B.dx;
            KS mk;
            ks_metric(P, x[0], x[1], x[2], mk);
            ks_cast(mk, m);
        }
    } else {
        double x[3];
        cell_centre(B, i, j, k, x);
        x[d] -= 0.5 * B.dx;
        face_geometry<RT>(P, x, m);
    }
    RT wL[8], wR[8];
#pragma unroll   // (wL, wR stay in registers only if every index is a constant)
    for (int v = 0; v < 8; v++) {
        if (v == P_B + d) continue;
        if (PPM6 && P.limiter == FX_PPM) {
            const RT a[6] = {sten(v, -3), sten(v, -2), sten(v, -1), sten(v, 0), sten(v, 1), sten(v, 2)};
            ppm_face(a, wL[v], wR[v]);
        } else {
            plm_face(sten(v, -2), sten(v, -1), sten(v, 0), sten(v, 1), P.limiter, wL[v], wR[v]);
        }
    }
    // (the limiters keep every face value between its two cells' values, so
    // face densities and pressures stay positive)
    RT Bn = RT(Bfs[d * N + c]) * m.alpha;   // alpha = 1 / sqrt(gamma)
    wL[P_B + d] = Bn;
    wR[P_B + d] = Bn;
    RT F[8];
    hll_face(m, RT(P.gamma), RT(P.gg), d, wL, wR, F);
    FT* Fo = (FT*)G.F;
    for (int v = 0; v < 8; v++) Fo[((int64_t)d * 8 + v) * N + c] = (FT)F[v];
}

// the stencil read from the primitives in global memory
template <typename RT, typename WT, typename FT>
__device__ inline void face_flux(const FxPar& P, const Grid& G, const bh_fx_block& B, int i, int j, int k, int d,
                                 const double* Bfs) {
    const int64_t N = G.ncell;
    const WT* Wc = (const WT*)G.W + bidx(B, i, j, k);
    const int st = d == 0 ? bstride_i(B) : (d == 1 ? bstride_j(B) : 1);
    face_flux_at<RT, FT, true>(P, G, B, i, j, k, d, Bfs, [&](int v, int o) { return RT(Wc[v * N + o * st]); });
}

template <typename RT, typename WT, typename FT, int MINB>
__global__ void __launch_bounds__(FX_TPB, MINB) k_fx_flux(FxPar P, Grid G, const int32_t* items, int stage, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n, m = n + 2;
        const int e = items[2 * t + 1] + threadIdx.x;
        if (e >= m * m * m) return;
        const int i = e / (m * m) - 1, j = (e / m) % m - 1, k = e % m - 1;
        const double* Bfs = stage ? G.Bf1 : G.Bf;
        if (i >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 0, Bfs);
        if (j >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 1, Bfs);
        if (k >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 2, Bfs);
    });
}

// ----------------------------------------------------------------------
// face fluxes with the stencil staged in shared memory.  A tile of
// FX_TI x FX_TJ x FX_TK positions (i, j, k; 128 threads) first loads the
// primitives its faces read -- the tile's cells and the cross-shaped halo
// of two cells below and one above along each axis (the stencil of PLM) --
// into shared memory with coalesced loads along k, then computes the
// x-, y- and z-faces of every position from there: each primitive is read
// from L2 once per tile instead of once per face that uses it.  The work
// items (block, e) are tiles (e >= 0, tile e of the block's position box
// [-1, n]^3) or, for blocks too small to tile well, chunks of 128
// positions starting at -(e + 1) as in k_fx_flux.  The arithmetic is that
// of k_fx_flux: the same bits.
// ----------------------------------------------------------------------
constexpr int FX_TI = 4, FX_TJ = 4, FX_TK = 8;
constexpr int FX_HI = FX_TI + 3, FX_HJ = FX_TJ + 3, FX_HK = FX_TK + 3;   // -2 .. T per axis
// row pitch of the staged box: 12 rather than FX_HK = 11 entries, so that a
// warp's 4 rows of 8 cells fall on fewer shared banks at once
constexpr int FX_HKP = FX_HK + 1;
constexpr int FX_HBOX = FX_HI * FX_HJ * FX_HKP;
constexpr int FX_NX = FX_HI * FX_TJ * FX_TK;   // the tile and its x-halo
constexpr int FX_NY = FX_TI * 3 * FX_TK;       // y-halo: j = -2, -1, TJ
constexpr int FX_NZ = FX_TI * FX_TJ * 3;       // z-halo: k = -2, -1, TK
constexpr int FX_NCROSS = FX_NX + FX_NY + FX_NZ;
static_assert(FX_TI * FX_TJ * FX_TK == FX_TPB, "one thread per tile position");

// offsets (a, b, c) in [-2, T] of the q-th cell of the cross-shaped halo
__device__ inline void cross_cell(int q, int& a, int& b, int& c) {
    if (q < FX_NX) {
        a = q / (FX_TJ * FX_TK) - 2; b = (q / FX_TK) % FX_TJ; c = q % FX_TK;
    } else if ((q -= FX_NX) < FX_NY) {
        const int h = (q / FX_TK) % 3;
        a = q / (3 * FX_TK); b = h < 2 ? h - 2 : FX_TJ; c = q % FX_TK;
    } else {
        q -= FX_NY;
        const int h = q % 3;
        a = q / (FX_TJ * 3); b = (q / 3) % FX_TJ; c = h < 2 ? h - 2 : FX_TK;
    }
}
__device__ inline int box_at(int a, int b, int c) { return ((a + 2) * FX_HJ + (b + 2)) * FX_HKP + (c + 2); }

template <typename RT, typename WT, typename FT, int MINB>
__global__ void __launch_bounds__(FX_TPB, MINB) k_fx_flux_tile(FxPar P, Grid G, const int32_t* items, int stage,
                                                             Queue Q) {
    __shared__ WT sW[8][FX_HBOX];
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n, m = n + 2;
        const double* Bfs = stage ? G.Bf1 : G.Bf;
        const int32_t e0 = items[2 * t + 1];
        if (e0 < 0) {   // a chunk of positions, as in k_fx_flux
            const int e = -(e0 + 1) + threadIdx.x;
            if (e >= m * m * m) return;
            const int i = e / (m * m) - 1, j = (e / m) % m - 1, k = e % m - 1;
            if (i >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 0, Bfs);
            if (j >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 1, Bfs);
            if (k >= 0) face_flux<RT, WT, FT>(P, G, B, i, j, k, 2, Bfs);
            return;
        }
        const int nj = (m + FX_TJ - 1) / FX_TJ, nk = (m + FX_TK - 1) / FX_TK;
        const int i0 = -1 + (e0 / (nj * nk)) * FX_TI, j0 = -1 + ((e0 / nk) % nj) * FX_TJ,
                  k0 = -1 + (e0 % nk) * FX_TK;
        const int64_t N = G.ncell;
        const WT* W = (const WT*)G.W;
        __syncthreads();   // the previous tile's reads of sW are done
        for (int q = threadIdx.x; q < FX_NCROSS; q += FX_TPB) {
            int a, bb, c;
            cross_cell(q, a, bb, c);
            const int i = i0 + a, j = j0 + bb, k = k0 + c;
            // cells of the box -2 .. n+2 only (those outside feed no face)
            if (i < -2 || i > n + 2 || j < -2 || j > n + 2 || k < -2 || k > n + 2) continue;
            const WT* Wc = W + bidx(B, i, j, k);
            const int o = box_at(a, bb, c);
#pragma unroll
            for (int v = 0; v < 8; v++) sW[v][o] = Wc[v * N];
        }
        __syncthreads();
        const int a = threadIdx.x / (FX_TJ * FX_TK), bb = (threadIdx.x / FX_TK) % FX_TJ, c = threadIdx.x % FX_TK;
        const int i = i0 + a, j = j0 + bb, k = k0 + c;
        if (i > n || j > n || k > n) return;
        const int o = box_at(a, bb, c);
        // (PLM only: the launch keeps PPM's wider stencil on k_fx_flux)
        if (i >= 0)
            face_flux_at<RT, FT, false>(P, G, B, i, j, k, 0, Bfs,
                                        [&](int v, int s) { return RT(sW[v][o + s * (FX_HJ * FX_HKP)]); });
        if (j >= 0)
            face_flux_at<RT, FT, false>(P, G, B, i, j, k, 1, Bfs,
                                        [&](int v, int s) { return RT(sW[v][o + s * FX_HKP]); });
        if (k >= 0)
            face_flux_at<RT, FT, false>(P, G, B, i, j, k, 2, Bfs, [&](int v, int s) { return RT(sW[v][o + s]); });
    });
}

// ======================================================================
// update: flux divergence + geometric source + RK2 (Heun) combine of the
// conserved state; constrained transport of the face field with edge EMFs
// averaged from the face fluxes (emfcomp's stencil, transport.cpp:11-36)
// and the Heun average of the two stages (stage 0: U1 = U + dt L(U),
// Bf1 = Bf - dt curl E; stage 1: U = (U + U1 + dt L(U1)) / 2, Bf = (Bf +
// Bf1 - dt curl E) / 2)
// ======================================================================
template <typename FT>
__device__ inline FT fget(const Grid& G, int d, int v, int64_t c) {
    return __ldg((const FT*)G.F + ((int64_t)d * 8 + v) * G.ncell + c);   // read-only in the update
}
// EMF components at the edges indexed like cell c, averaged in the flux
// type (FP32 in the mixed variant: one conversion per edge, and every face
// sharing the edge sees the same value, so div B stays at roundoff)
template <typename FT>
__device__ inline double emf_x(const Grid& G, int64_t c, int sj, int sk) {   // (i, j-1/2, k-1/2)
    return (double)(FT(0.25) * (fget<FT>(G, 2, C_B + 1, c) + fget<FT>(G, 2, C_B + 1, c - sj) -
                                fget<FT>(G, 1, C_B + 2, c) - fget<FT>(G, 1, C_B + 2, c - sk)));
}
template <typename FT>
__device__ inline double emf_y(const Grid& G, int64_t c, int si, int sk) {   // (i-1/2, j, k-1/2)
    return (double)(FT(0.25) * (fget<FT>(G, 0, C_B + 2, c) + fget<FT>(G, 0, C_B + 2, c - sk) -
                                fget<FT>(G, 2, C_B + 0, c) - fget<FT>(G, 2, C_B + 0, c - si)));
}
template <typename FT>
__device__ inline double emf_z(const Grid& G, int64_t c, int si, int sj) {   // (i-1/2, j-1/2, k)
    return (double)(FT(0.25) * (fget<FT>(G, 1, C_B + 0, c) + fget<FT>(G, 1, C_B + 0, c - si) -
                                fget<FT>(G, 0, C_B + 1, c) - fget<FT>(G, 0, C_B + 1, c - sj)));
}
template <typename FT>
__device__ inline void face_update(const Grid& G, int d, int64_t c, int si, int sj, int sk, double idx, double dt,
                                   int stage) {
    const int64_t N = G.ncell;
    double curl;
    if (G.E) {   // the edge EMFs of the grid (corrected at level changes)
        const double *Ex = G.E, *Ey = G.E + N, *Ez = G.E + 2 * N;
        if (d == 0)
            curl = (Ez[c + sj] - Ez[c]) * idx - (Ey[c + sk] - Ey[c]) * idx;
        else if (d == 1)
            curl = (Ex[c + sk] - Ex[c]) * idx - (Ez[c + si] - Ez[c]) * idx;
        else
            curl = (Ey[c + si] - Ey[c]) * idx - (Ex[c + sj] - Ex[c]) * idx;
    } else if (d == 0)
        curl = (emf_z<FT>(G, c + sj, si, sj) - emf_z<FT>(G, c, si, sj)) * idx -
               (emf_y<FT>(G, c + sk, si, sk) - emf_y<FT>(G, c, si, sk)) * idx;
    else if (d == 1)
        curl = (emf_x<FT>(G, c + sk, sj, sk) - emf_x<FT>(G, c, sj, sk)) * idx -
               (emf_z<FT>(G, c + si, si, sj) - emf_z<FT>(G, c, si, sj)) * idx;
    else
        curl = (emf_y<FT>(G, c + si, si, sk) - emf_y<FT>(G, c, si, sk)) * idx -
               (emf_x<FT>(G, c + sj, sj, sk) - emf_x<FT>(G, c, sj, sk)) * idx;
    if (stage == 0)
        G.Bf1[d * N + c] = G.Bf[d * N + c] - dt * curl;
    else
        G.Bf[d * N + c] = 0.5 * (G.Bf[d * N + c] + G.Bf1[d * N + c] - dt * curl);
}

// edge EMFs of every block (the edges its face updates read: E_x at
// i in [0,n), j, k in [0,n], and alike), from the face fluxes
template <typename FT>
__global__ void __launch_bounds__(FX_TPB) k_fx_emf(Grid G, const int32_t* items, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n, m = n + 2;
        const int e = items[2 * t + 1] + threadIdx.x;
        if (e >= m * m * m) return;
        const int i = e / (m * m) - 1, j = (e / m) % m - 1, k = e % m - 1;
        if (i < 0 || j < 0 || k < 0) return;
        const int64_t N = G.ncell, c = bidx(B, i, j, k);
        const int si = bstride_i(B), sj = bstride_j(B), sk = 1;
        if (i < n) G.E[c] = emf_x<FT>(G, c, sj, sk);
        if (j < n) G.E[N + c] = emf_y<FT>(G, c, si, sk);
        if (k < n) G.E[2 * N + c] = emf_z<FT>(G, c, si, sj);
    });
}

// EMF correction at level changes: an edge on a block's boundary that a
// finer block also touches takes the mean of that block's two EMFs along it,
// so every copy of a shared face sees the same circulation and the face
// field of the coarse side stays the mean of the fine faces (div B at
// roundoff).  Levels differ by one at most, so one pass suffices.
__global__ void __launch_bounds__(FX_TPB) k_fx_emf_fix(Grid G, const int32_t* items, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n, m = n + 2;
        const int e = items[2 * t + 1] + threadIdx.x;
        if (e >= m * m * m) return;
        const int p[3] = {e / (m * m) - 1, (e / m) % m - 1, e % m - 1};
        if (p[0] < 0 || p[1] < 0 || p[2] < 0) return;
        const int64_t N = G.ncell;
        const int32_t* nb = G.nbr + (int64_t)b * 27;
        for (int d = 0; d < 3; d++) {          // edge direction
            if (p[d] >= n) continue;
            const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
            const int o1 = p[t1] == 0 ? -1 : (p[t1] == n ? 1 : 0);
            const int o2 = p[t2] == 0 ? -1 : (p[t2] == n ? 1 : 0);
            if (o1 == 0 && o2 == 0) continue;  // not on the boundary
            // the cubes sharing the edge: offsets (a1 o1, a2 o2), (a1, a2) != (0, 0)
            for (int a1 = 0; a1 <= (o1 != 0); a1++)
                for (int a2 = 0; a2 <= (o2 != 0); a2++) {
                    if (!a1 && !a2) continue;
                    int o[3] = {0, 0, 0};
                    o[t1] = a1 * o1;
                    o[t2] = a2 * o2;
                    const int s = nb[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)];
                    if (s < 0) continue;
                    const bh_fx_block S = G.blk[s];
                    if (S.n != 2 * n) continue;
                    // the two fine edges along this one, in the finer block's frame
                    int f[3] = {2 * (p[0] - o[0] * n), 2 * (p[1] - o[1] * n), 2 * (p[2] - o[2] * n)};
                    int g[3] = {f[0], f[1], f[2]};
                    g[d] += 1;
                    const double* Es = G.E + d * N;
                    G.E[d * N + bidx(B, p[0], p[1], p[2])] = 0.5 * (Es[bidx(S, f[0], f[1], f[2])] + Es[bidx(S, g[0], g[1], g[2])]);
                    a1 = 2;   // done with this edge
                    break;
                }
        }
    });
}

// PART 3: the whole update; 1: the conserved state (source, divergence,
// RK); 2: the face field (EMFs, CT) -- the two halves read disjoint flux
// components, so as two kernels (BH_FX_TUNE_SPLIT) each keeps fewer
// registers than the whole
template <typename RT, typename WT, typename FT, int MINB, int PART>
__global__ void __launch_bounds__(FX_TPB, MINB) k_fx_update(FxPar P, Grid G, const int32_t* items, int stage,
                                                      double cfl, Queue Q) {
    for_items(Q, [&](int t) FX_INLINE {
        const int32_t b = items[2 * t];
        const bh_fx_block B = G.blk[b];
        const int n = B.n;
        const int e = items[2 * t + 1] + threadIdx.x;
        if (e >= n * n * n) return;
        const int i = e / (n * n), j = (e / n) % n, k = e % n;
        const int64_t N = G.ncell;
        const int64_t c = bidx(B, i, j, k);
        const int si = bstride_i(B), sj = bstride_j(B), sk = 1;
        const double dt = cfl * G.dt[0];
        if ((PART & 1) && stage == 0 && t == 0 && threadIdx.x == 0) G.dt[1] = dt;
        const double idx = 1.0 / B.dx;
        if (PART & 1) {
        // source at the cell centre from the stage's primitives
        double x[3];
        cell_centre(B, i, j, k, x);
        KSb<RT> mk;
        KSDb<RT> dk;
        cell_geometry<RT>(P, x, mk, dk);
        const WT* W = (const WT*)G.W;
        RT w[8];
        for (int v = 0; v < 8; v++) w[v] = RT(W[v * N + c]);
        RT S[8];
        source<RT>(mk, dk, RT(P.gg), w, S);
        // the flux divergence in the flux type (the differences of
        // neighbouring faces' values are exact in FP32 where they are within
        // a factor of two of each other)
        const FT idf = FT(idx);
        for (int v = 0; v < 5; v++) {
            FT div = (fget<FT>(G, 0, v, c + si) - fget<FT>(G, 0, v, c)) * idf +
                     (fget<FT>(G, 1, v, c + sj) - fget<FT>(G, 1, v, c)) * idf +
                     (fget<FT>(G, 2, v, c + sk) - fget<FT>(G, 2, v, c)) * idf;
            double L = (double)S[v] - (double)div;
            if (stage == 0)
                G.U1[v * N + c] = G.U[v * N + c] + dt * L;
            else
                G.U[v * N + c] = 0.5 * (G.U[v * N + c] + G.U1[v * N + c] + dt * L);
        }
        }
        if (!(PART & 2)) return;
        // the nine distinct edge EMFs of the cell's three lower faces: ex at
        // the edges of c, c+sj, c+sk; ey at c, c+si, c+sk; ez at c, c+si, c+sj
        double ex[3], ey[3], ez[3];
        if (G.E) {   // the edge EMFs of the grid (corrected at level changes)
            const double *Ex = G.E, *Ey = G.E + N, *Ez = G.E + 2 * N;
            ex[0] = Ex[c]; ex[1] = Ex[c + sj]; ex[2] = Ex[c + sk];
            ey[0] = Ey[c]; ey[1] = Ey[c + si]; ey[2] = Ey[c + sk];
            ez[0] = Ez[c]; ez[1] = Ez[c + si]; ez[2] = Ez[c + sj];
        } else {
            ex[0] = emf_x<FT>(G, c, sj, sk); ex[1] = emf_x<FT>(G, c + sj, sj, sk); ex[2] = emf_x<FT>(G, c + sk, sj, sk);
            ey[0] = emf_y<FT>(G, c, si, sk); ey[1] = emf_y<FT>(G, c + si, si, sk); ey[2] = emf_y<FT>(G, c + sk, si, sk);
            ez[0] = emf_z<FT>(G, c, si, sj); ez[1] = emf_z<FT>(G, c + si, si, sj); ez[2] = emf_z<FT>(G, c + sj, si, sj);
        }
        // face field: this cell's three lower faces (curl E as in face_update),
        // and the upper boundary faces
        const double curl[3] = {(ez[2] - ez[0]) * idx - (ey[2] - ey[0]) * idx,
                                (ex[2] - ex[0]) * idx - (ez[1] - ez[0]) * idx,
                                (ey[1] - ey[0]) * idx - (ex[1] - ex[0]) * idx};
        for (int d = 0; d < 3; d++) {
            if (stage == 0)
                G.Bf1[d * N + c] = G.Bf[d * N + c] - dt * curl[d];
            else
                G.Bf[d * N + c] = 0.5 * (G.Bf[d * N + c] + G.Bf1[d * N + c] - dt * curl[d]);
        }
        if (i == n - 1) face_update<FT>(G, 0, c + si, si, sj, sk, idx, dt, stage);
        if (j == n - 1) face_update<FT>(G, 1, c + sj, si, sj, sk, idx, dt, stage);
        if (k == n - 1) face_update<FT>(G, 2, c + sk, si, sj, sk, idx, dt, stage);
    });
}

// ======================================================================
// the state a step reads, between the grid's boxes and a compact buffer
// (dir 0: pack, 1: unpack): per interior-cell slot q = item * 128 + lane
// (Q = nitem_cell * 128 slots) rows 0-4 of U (double [5][Q]) and of W
// (WT [5][Q]) and the cell's three lower faces (double [3][Q]); then the
// blocks' upper boundary faces, 3 n^2 doubles per block from face_off[b]
// (x-faces at i = n by (j, k), y at j = n by (i, k), z at k = n by (i, j)).
// Slots past a block's last cell are left alone.
// ======================================================================
template <typename WT>
__global__ void __launch_bounds__(FX_TPB) k_fx_pack(Grid G, const int32_t* items, int nitem, const int64_t* face_off,
                                                    char* packed, int dir) {
    const int t = blockIdx.x;
    const int32_t b = items[2 * t];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * t + 1] + threadIdx.x;
    if (e >= n * n * n) return;
    const int i = e / (n * n), j = (e / n) % n, k = e % n;
    const int64_t N = G.ncell, c = bidx(B, i, j, k), Q = (int64_t)nitem * FX_TPB, q = (int64_t)t * FX_TPB + threadIdx.x;
    double* pu = (double*)packed;
    WT* pw = (WT*)(pu + 5 * Q);
    double* pb = (double*)(pw + 5 * Q);
    double* pf = pb + 3 * Q + face_off[b];
    WT* W = (WT*)G.W;
    const int si = bstride_i(B), sj = bstride_j(B);
    if (dir == 0) {
        for (int v = 0; v < 5; v++) pu[v * Q + q] = G.U[v * N + c];
        for (int v = 0; v < 5; v++) pw[v * Q + q] = W[v * N + c];
        for (int d = 0; d < 3; d++) pb[d * Q + q] = G.Bf[d * N + c];
        if (i == n - 1) pf[j * n + k] = G.Bf[c + si];
        if (j == n - 1) pf[n * n + i * n + k] = G.Bf[N + c + sj];
        if (k == n - 1) pf[2 * n * n + i * n + j] = G.Bf[2 * N + c + 1];
    } else {
        for (int v = 0; v < 5; v++) G.U[v * N + c] = pu[v * Q + q];
        for (int v = 0; v < 5; v++) W[v * N + c] = pw[v * Q + q];
        for (int d = 0; d < 3; d++) G.Bf[d * N + c] = pb[d * Q + q];
        if (i == n - 1) G.Bf[c + si] = pf[j * n + k];
        if (j == n - 1) G.Bf[N + c + sj] = pf[n * n + i * n + k];
        if (k == n - 1) G.Bf[2 * N + c + 1] = pf[2 * n * n + i * n + j];
    }
}

// ======================================================================
// divergence of the face field: per interior cell |div B| dx / max(|B~|)
// of its six faces; max over each block into out[b] (non-negative doubles)
// ======================================================================
__global__ void __launch_bounds__(FX_TPB) k_fx_divb(Grid G, const int32_t* items, double* out) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    double v = 0.0;
    if (e < n * n * n) {
        const int i = e / (n * n), j = (e / n) % n, k = e % n;
        const int64_t N = G.ncell, c = bidx(B, i, j, k);
        const int si = bstride_i(B), sj = bstride_j(B);
        double f[6] = {G.Bf[c], G.Bf[c + si], G.Bf[N + c], G.Bf[N + c + sj], G.Bf[2 * N + c], G.Bf[2 * N + c + 1]};
        double div = (f[1] - f[0]) + (f[3] - f[2]) + (f[5] - f[4]);
        double mx = 0.0;
        for (int q = 0; q < 6; q++) mx = fmax(mx, fabs(f[q]));
        v = mx > 0.0 ? fabs(div) / mx : 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomic_max_pos(out + b, v);
}


// ======================================================================
// initial data (bh_fx_torus_init)
// ======================================================================
struct TorusK {
    FMTorus t;
    double noise;
    uint64_t seed;
};
__global__ void __launch_bounds__(FX_TPB) k_fxi_rho(Grid G, const int32_t* items, TorusK T, double* scratch) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    double rho = 0.0;
    if (e < n * n * n) {
        const int i = e / (n * n), j = (e / n) % n, k = e % n;
        double x[3];
        cell_centre(B, i, j, k, x);
        rho = fm_rho(T.t, x[0], x[1], x[2], nullptr);
    }
    for (int o = 16; o > 0; o >>= 1) rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
    if ((threadIdx.x & 31) == 0 && rho > 0.0) atomic_max_pos(scratch, rho);
}
// primitives of the interior cells (no field yet); max p_gas of the torus
template <typename WT>
__global__ void __launch_bounds__(FX_TPB) k_fxi_prims(FxPar P, Grid G, const int32_t* items, TorusK T,
                                                      double* scratch) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    double pg = 0.0;
    if (e < n * n * n) {
        const int i = e / (n * n), j = (e / n) % n, k = e % n;
        const int64_t N = G.ncell, c = bidx(B, i, j, k);
        double x[3];
        cell_centre(B, i, j, k, x);
        KS m;
        ks_metric(P, x[0], x[1], x[2], m);
        const double rmax = scratch[0];
        double rho = fm_rho(T.t, x[0], x[1], x[2], nullptr);
        double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (rho > 0.0 && rmax > 0.0) {
            double p = T.t.kappa * pow(rho, T.t.gamma) / rmax;
            double u = hash_uniform(T.seed, cell_key(B.x0, B.dx, i, j, k));
            p = p * (1.0 + T.noise * (2.0 * u - 1.0));
            double ut, ux, uy;
            fm_velocity(T.t, x[0], x[1], x[2], ut, ux, uy);
            // ut^i = u^i + u^t beta^i
            w[P_RHO] = rho / rmax;
            w[P_PRS] = p;
            w[P_UT] = ux + ut * m.beta[0];
            w[P_UT + 1] = uy + ut * m.beta[1];
            w[P_UT + 2] = ut * m.beta[2];
        } else {
            floor_state(P, m.r, w[P_RHO], w[P_PRS]);
        }
        apply_floors(P, m, w);
        if (rho > 0.0 && rmax > 0.0) pg = w[P_PRS];
        WT* W = (WT*)G.W;
        for (int v = 0; v < 8; v++) W[v * N + c] = (WT)w[v];
    }
    for (int o = 16; o > 0; o >>= 1) pg = fmax(pg, __shfl_xor_sync(0xffffffffu, pg, o));
    if ((threadIdx.x & 31) == 0 && pg > 0.0) atomic_max_pos(scratch + 1, pg);
}
// A_phi = max(rho / rho_max - 0.2, 0) at a point, as Cartesian (A_x, A_y)
__device__ inline void apot(const TorusK& T, double rmax, double x, double y, double z, double& ax, double& ay) {
    double rho = fm_rho(T.t, x, y, z, nullptr);
    double A = rho / rmax - 0.2;
    ax = ay = 0.0;
    if (A > 0.0) {
        double iw = 1.0 / (x * x + y * y);
        ax = -A * y * iw;
        ay = A * x * iw;
    }
}
// face field = curl of the edge potential (A_z = 0), unscaled.  An edge's
// A is the mean of A at the midpoints of its sub-edges at the finest level
// of the grid (2^(maxlevel - level) of them), so that a coarse face's
// circulation equals the mean of the finer faces that cover it.
__device__ inline void apot_edge(const TorusK& T, double rmax, double x, double y, double z, int d, double h, int K,
                                 double& ax, double& ay) {
    double sx = 0.0, sy = 0.0, p[3] = {x, y, z};
    const double hk = h / K;
    for (int q = 0; q < K; q++) {
        double r[3] = {p[0], p[1], p[2]};
        r[d] = p[d] + (q + 0.5) * hk;
        double a, b;
        apot(T, rmax, r[0], r[1], r[2], a, b);
        sx += a;
        sy += b;
    }
    ax = sx / K;
    ay = sy / K;
}
__global__ void __launch_bounds__(FX_TPB) k_fxi_faces(Grid G, const int32_t* items, TorusK T, double* scratch,
                                                      int maxlevel) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n, m = n + 2;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    if (e >= m * m * m) return;
    const int i = e / (m * m) - 1, j = (e / m) % m - 1, k = e % m - 1;
    const int64_t N = G.ncell, c = bidx(B, i, j, k);
    const double rmax = scratch[0], h = B.dx;
    const double X = B.x0[0], Y = B.x0[1], Z = B.x0[2];
    const int K = 1 << (maxlevel - B.level);
    double ax0, ay0, ax1, ay1, d0, d1;
    if (i >= 0) {   // x-face (i-1/2, j, k): -(A_y(k+1/2) - A_y(k-1/2)) / dz, y-edges at (i-1/2, j, k -+ 1/2)
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + k * h, 1, h, K, d0, ay0);
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + (k + 1) * h, 1, h, K, d1, ay1);
        G.Bf[c] = -(ay1 - ay0) / h;
    }
    if (j >= 0) {   // y-face (i, j-1/2, k): (A_x(k+1/2) - A_x(k-1/2)) / dz, x-edges at (i, j-1/2, k -+ 1/2)
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + k * h, 0, h, K, ax0, d0);
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + (k + 1) * h, 0, h, K, ax1, d1);
        G.Bf[N + c] = (ax1 - ax0) / h;
    }
    if (k >= 0) {   // z-face (i, j, k-1/2): dA_y/dx - dA_x/dy
        double ayl, ayr, axl, axr;
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + k * h, 1, h, K, d0, ayl);
        apot_edge(T, rmax, X + (i + 1) * h, Y + j * h, Z + k * h, 1, h, K, d1, ayr);
        apot_edge(T, rmax, X + i * h, Y + j * h, Z + k * h, 0, h, K, axl, d0);
        apot_edge(T, rmax, X + i * h, Y + (j + 1) * h, Z + k * h, 0, h, K, axr, d1);
        G.Bf[2 * N + c] = (ayr - ayl) / h - (axr - axl) / h;
    }
}
// max b^2 / 2 of the interior cells with the unscaled field
template <typename WT>
__global__ void __launch_bounds__(FX_TPB) k_fxi_pmag(FxPar P, Grid G, const int32_t* items, double* scratch) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    double pm = 0.0;
    if (e < n * n * n) {
        const int i = e / (n * n), j = (e / n) % n, k = e % n;
        const int64_t N = G.ncell, c = bidx(B, i, j, k);
        const int si = bstride_i(B), sj = bstride_j(B);
        double x[3];
        cell_centre(B, i, j, k, x);
        KS mk;
        ks_metric(P, x[0], x[1], x[2], mk);
        double isg = 1.0 / mk.sqrtgam;
        const WT* W = (const WT*)G.W;
        double w[8];
        for (int v = 0; v < 5; v++) w[v] = (double)W[v * N + c];
        w[P_B] = 0.5 * (G.Bf[c] + G.Bf[c + si]) * isg;
        w[P_B + 1] = 0.5 * (G.Bf[N + c] + G.Bf[N + c + sj]) * isg;
        w[P_B + 2] = 0.5 * (G.Bf[2 * N + c] + G.Bf[2 * N + c + 1]) * isg;
        KSm<double> m;
        ks_cast(mk, m);
        Derived<double> d;
        derive(m, P.gg, w, d);
        pm = 0.5 * d.b2;
    }
    for (int o = 16; o > 0; o >>= 1) pm = fmax(pm, __shfl_xor_sync(0xffffffffu, pm, o));
    if ((threadIdx.x & 31) == 0 && pm > 0.0) atomic_max_pos(scratch + 2, pm);
}
__device__ inline double field_scale(const double* scratch, double beta) {
    return (scratch[2] > 0.0 && beta > 0.0) ? sqrt(scratch[1] / (beta * scratch[2])) : 0.0;
}
__global__ void __launch_bounds__(FX_TPB) k_fxi_scale(Grid G, const int32_t* items, double beta, double* scratch) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n, m = n + 2;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    const double s = field_scale(scratch, beta);
    if (blockIdx.x == 0 && threadIdx.x == 0) scratch[3] = s;
    if (e >= m * m * m) return;
    const int i = e / (m * m) - 1, j = (e / m) % m - 1, k = e % m - 1;
    const int64_t N = G.ncell, c = bidx(B, i, j, k);
    if (i >= 0) G.Bf[c] *= s;
    if (j >= 0) G.Bf[N + c] *= s;
    if (k >= 0) G.Bf[2 * N + c] *= s;
}
// cell field and conserved state of the interior cells
template <typename WT>
__global__ void __launch_bounds__(FX_TPB) k_fxi_cons(FxPar P, Grid G, const int32_t* items) {
    const int32_t b = items[2 * blockIdx.x];
    const bh_fx_block B = G.blk[b];
    const int n = B.n;
    const int e = items[2 * blockIdx.x + 1] + threadIdx.x;
    if (e >= n * n * n) return;
    const int i = e / (n * n), j = (e / n) % n, k = e % n;
    const int64_t N = G.ncell, c = bidx(B, i, j, k);
    const int si = bstride_i(B), sj = bstride_j(B);
    double x[3];
    cell_centre(B, i, j, k, x);
    KS mk;
    ks_metric(P, x[0], x[1], x[2], mk);
    double Bt[3] = {0.5 * (G.Bf[c] + G.Bf[c + si]), 0.5 * (G.Bf[N + c] + G.Bf[N + c + sj]),
                    0.5 * (G.Bf[2 * N + c] + G.Bf[2 * N + c + 1])};
    double isg = 1.0 / mk.sqrtgam;
    WT* W = (WT*)G.W;
    double w[8], u[8];
    for (int v = 0; v < 5; v++) w[v] = (double)W[v * N + c];
    for (int d = 0; d < 3; d++) w[P_B + d] = Bt[d] * isg;
    KSm<double> m;
    ks_cast(mk, m);
    Derived<double> d;
    derive(m, P.gg, w, d);
    prim2cons(m, P.gamma, w, d, u);
    for (int v = 0; v < 5; v++) G.U[v * N + c] = u[v];
    for (int q = 0; q < 3; q++) G.U[(5 + q) * N + c] = Bt[q];
    for (int v = 5; v < 8; v++) W[v * N + c] = (WT)w[v];
}

}  // namespace
}  // namespace fx

// ---- launch sequences of this variant (bh_api.h) -------------------------
namespace BH_VARIANT {
namespace {
using FRT = BH_REAL;
inline cudaStream_t fxs(void* s) { return (cudaStream_t)s; }
inline int fx_launched() { return cudaGetLastError() == cudaSuccess ? BH_OK : BH_ECUDA; }
// work-queue slots of the step kernels
enum { QS_C2P = 0, QS_GHOST = 1, QS_FLUX = 2, QS_EMF = 3, QS_EMF_FIX = 4, QS_UPDATE = 5, QS_UPDATE_B = 6 };
static_assert(QS_UPDATE_B + 1 == BH_FX_QSLOTS, "queue slots");
inline fx::Queue fx_q(const bh_fx_grid* g, int slot, int nitem) {
    if (!g->queue) return fx::Queue{nullptr, nullptr, nitem};
    return fx::Queue{g->queue + 2 * slot, g->queue + 2 * slot + 1, nitem};
}
inline int fx_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
    }
    return sms;
}
// CTAs of a launch: one per item, or (persistent) the resident CTAs of the
// kernel on this device, from the occupancy calculator (cached per kernel)
inline int fx_grid(const void* fn, int nitem, const bh_fx_grid* g) {
    if (!g->queue) return nitem;
    int ctas = g->queue_ctas;
    if (ctas <= 0) {
        static const void* keys[96];
        static int vals[96];
        static int nkeys = 0;
        int occ = 0;
        for (int i = 0; i < nkeys; i++)
            if (keys[i] == fn) occ = vals[i];
        if (!occ) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, fx::FX_TPB, 0) != cudaSuccess || occ < 1) occ = 1;
            if (nkeys < 96) { keys[nkeys] = fn; vals[nkeys] = occ; nkeys++; }
        }
        ctas = fx_sms() * occ;
    }
    return nitem < ctas ? nitem : ctas;
}
}  // namespace

// launch bounds of the heavy kernels: resident 128-thread CTAs per SM asked
// of ptxas (which caps registers per thread); 1 leaves the choice to ptxas.
// Chosen per process and variant (bh_fx_tune_set), initially 1.
int fx_tune_tab[BH_FX_TUNE_N] = {1, 1, 1, 0, 0};
#define FX_TUNED(kernel, LAUNCH)                                                  \
    switch (fx_tune_tab[kernel]) {                                                \
    case 3: LAUNCH(3); break;                                                     \
    case 4: LAUNCH(4); break;                                                     \
    case 5: LAUNCH(5); break;                                                     \
    case 6: LAUNCH(6); break;                                                     \
    case 7: LAUNCH(7); break;                                                     \
    case 8: LAUNCH(8); break;                                                     \
    default: LAUNCH(1); break;                                                    \
    }

int fx_tune_set(int32_t kernel, int32_t ctas) {
    if (kernel == BH_FX_TUNE_STAGE || kernel == BH_FX_TUNE_SPLIT) {
        if (ctas != 0 && ctas != 1) return BH_EINVAL;
    } else if (kernel < 0 || kernel >= BH_FX_TUNE_N || !(ctas == 1 || (ctas >= 3 && ctas <= 8))) {
        return BH_EINVAL;
    }
    fx_tune_tab[kernel] = ctas;
    return BH_OK;
}
int fx_tune_get(int32_t kernel, int32_t* ctas) {
    if (kernel < 0 || kernel >= BH_FX_TUNE_N || !ctas) return BH_EINVAL;
    *ctas = fx_tune_tab[kernel];
    return BH_OK;
}

int fx_prims(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, int32_t with_dt, void* s) {
    fx::FxPar p = fx::par_of(P);
    fx::Grid G = fx::grid_of(g);
    if (with_dt) fx::k_fx_dt_init<<<1, 1, 0, fxs(s)>>>(g->dt);
    if (g->nitem_cell) {
#define L_(M) fx::k_fx_c2p<FRT, FRT, M><<<fx_grid((const void*)fx::k_fx_c2p<FRT, FRT, M>, g->nitem_cell, g), fx::FX_TPB, 0, fxs(s)>>>(p, G, g->items_cell, stage, with_dt, fx_q(g, QS_C2P, g->nitem_cell))
        FX_TUNED(BH_FX_TUNE_C2P, L_)
#undef L_
    }
    return fx_launched();
}
int fx_ghost_pass(const bh_fx_params*, const bh_fx_grid* g, int32_t stage, int32_t pass, void* s) {
    fx::Grid G = fx::grid_of(g);
    if (g->nitem_ghost)
        fx::k_fx_ghost<FRT><<<fx_grid((const void*)fx::k_fx_ghost<FRT>, g->nitem_ghost, g), fx::FX_TPB, 0, fxs(s)>>>(
            G, g->items_ghost, stage, pass, fx_q(g, QS_GHOST, g->nitem_ghost));
    return fx_launched();
}
int fx_ghosts(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* s) {
    // pass 0: copies and restrictions; pass l: prolongations into level l
    int rc = BH_OK;
    for (int pass = 0; pass <= g->maxlevel && rc == BH_OK; pass++) rc = fx_ghost_pass(P, g, stage, pass, s);
    return rc;
}
int fx_fluxes(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* s) {
    fx::FxPar p = fx::par_of(P);
    fx::Grid G = fx::grid_of(g);
    if (fx_tune_tab[BH_FX_TUNE_STAGE] && g->nitem_flux && P->limiter != fx::FX_PPM) {
#define L_(M) fx::k_fx_flux_tile<FRT, FRT, FRT, M><<<fx_grid((const void*)fx::k_fx_flux_tile<FRT, FRT, FRT, M>, g->nitem_flux, g), fx::FX_TPB, 0, fxs(s)>>>(p, G, g->items_flux, stage, fx_q(g, QS_FLUX, g->nitem_flux))
        FX_TUNED(BH_FX_TUNE_FLUX, L_)
#undef L_
    } else if (g->nitem_pos) {
#define L_(M) fx::k_fx_flux<FRT, FRT, FRT, M><<<fx_grid((const void*)fx::k_fx_flux<FRT, FRT, FRT, M>, g->nitem_pos, g), fx::FX_TPB, 0, fxs(s)>>>(p, G, g->items_pos, stage, fx_q(g, QS_FLUX, g->nitem_pos))
        FX_TUNED(BH_FX_TUNE_FLUX, L_)
#undef L_
    }
    return fx_launched();
}
// parts: 1 = the edge EMFs into E, 2 = their level-change correction and
// the update (3 = both: the update of a stage)
int fx_update_parts(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, int32_t parts, void* s) {
    fx::FxPar p = fx::par_of(P);
    fx::Grid G = fx::grid_of(g);
    if (g->E && g->nitem_pos && (parts & 1))
        fx::k_fx_emf<FRT><<<fx_grid((const void*)fx::k_fx_emf<FRT>, g->nitem_pos, g), fx::FX_TPB, 0, fxs(s)>>>(
            G, g->items_pos, fx_q(g, QS_EMF, g->nitem_pos));
    if (!(parts & 2)) return fx_launched();
    if (g->E && g->nitem_pos && g->maxlevel > 0)
        fx::k_fx_emf_fix<<<fx_grid((const void*)fx::k_fx_emf_fix, g->nitem_pos, g), fx::FX_TPB, 0, fxs(s)>>>(
            G, g->items_pos, fx_q(g, QS_EMF_FIX, g->nitem_pos));
    if (g->nitem_cell && fx_tune_tab[BH_FX_TUNE_SPLIT]) {
#define L_(M) fx::k_fx_update<FRT, FRT, FRT, M, 1><<<fx_grid((const void*)fx::k_fx_update<FRT, FRT, FRT, M, 1>, g->nitem_cell, g), fx::FX_TPB, 0, fxs(s)>>>(p, G, g->items_cell, stage, P->cfl, fx_q(g, QS_UPDATE, g->nitem_cell))
        FX_TUNED(BH_FX_TUNE_UPDATE, L_)
#undef L_
        fx::k_fx_update<FRT, FRT, FRT, 8, 2><<<fx_grid((const void*)fx::k_fx_update<FRT, FRT, FRT, 8, 2>, g->nitem_cell, g), fx::FX_TPB, 0, fxs(s)>>>(
            p, G, g->items_cell, stage, P->cfl, fx_q(g, QS_UPDATE_B, g->nitem_cell));
    } else if (g->nitem_cell) {
#define L_(M) fx::k_fx_update<FRT, FRT, FRT, M, 3><<<fx_grid((const void*)fx::k_fx_update<FRT, FRT, FRT, M, 3>, g->nitem_cell, g), fx::FX_TPB, 0, fxs(s)>>>(p, G, g->items_cell, stage, P->cfl, fx_q(g, QS_UPDATE, g->nitem_cell))
        FX_TUNED(BH_FX_TUNE_UPDATE, L_)
#undef L_
    }
    return fx_launched();
}
int fx_update(const bh_fx_params* P, const bh_fx_grid* g, int32_t stage, void* s) {
    return fx_update_parts(P, g, stage, 3, s);
}
int fx_step(const bh_fx_params* P, const bh_fx_grid* g, void* s) {
    for (int stage = 0; stage < 2; stage++) {
        int rc = fx_prims(P, g, stage, stage == 0, s);
        if (!rc) rc = fx_ghosts(P, g, stage, s);
        if (!rc) rc = fx_fluxes(P, g, stage, s);
        if (!rc) rc = fx_update(P, g, stage, s);
        if (rc) return rc;
    }
    return BH_OK;
}
int fx_pack_state(const bh_fx_grid* g, const int64_t* face_off, void* packed, int32_t dir, void* s) {
    fx::Grid G = fx::grid_of(g);
    if (g->nitem_cell)
        fx::k_fx_pack<FRT><<<g->nitem_cell, fx::FX_TPB, 0, fxs(s)>>>(G, g->items_cell, g->nitem_cell, face_off,
                                                                     (char*)packed, dir);
    return fx_launched();
}
int fx_divb(const bh_fx_grid* g, double* out, void* s) {
    fx::Grid G = fx::grid_of(g);
    if (cudaMemsetAsync(out, 0, sizeof(double) * g->nblock, fxs(s)) != cudaSuccess) return BH_ECUDA;
    if (g->nitem_cell) fx::k_fx_divb<<<g->nitem_cell, fx::FX_TPB, 0, fxs(s)>>>(G, g->items_cell, out);
    return fx_launched();
}
int fx_torus_init(const bh_fx_params* P, const bh_fx_grid* g, const bh_fx_torus* T, double* scratch, double* out,
                  void* s) {
    fx::FxPar p = fx::par_of(P);
    fx::Grid G = fx::grid_of(g);
    fx::TorusK tk;
    tk.t = bhfx::fm_torus(P->a, P->gamma, T->kappa, T->r_in, T->r_max);
    tk.noise = T->noise;
    tk.seed = T->seed;
    cudaStream_t st = fxs(s);
    if (cudaMemsetAsync(scratch, 0, 4 * sizeof(double), st) != cudaSuccess) return BH_ECUDA;
    if (cudaMemsetAsync(g->Bf, 0, 3 * sizeof(double) * g->ncell, st) != cudaSuccess) return BH_ECUDA;
    fx::k_fxi_rho<<<g->nitem_cell, fx::FX_TPB, 0, st>>>(G, g->items_cell, tk, scratch);
    fx::k_fxi_prims<FRT><<<g->nitem_cell, fx::FX_TPB, 0, st>>>(p, G, g->items_cell, tk, scratch);
    fx::k_fxi_faces<<<g->nitem_pos, fx::FX_TPB, 0, st>>>(G, g->items_pos, tk, scratch, g->maxlevel);
    fx::k_fxi_pmag<FRT><<<g->nitem_cell, fx::FX_TPB, 0, st>>>(p, G, g->items_cell, scratch);
    fx::k_fxi_scale<<<g->nitem_pos, fx::FX_TPB, 0, st>>>(G, g->items_pos, T->beta, scratch);
    fx::k_fxi_cons<FRT><<<g->nitem_cell, fx::FX_TPB, 0, st>>>(p, G, g->items_cell);
    int rc = fx_launched();
    if (rc) return rc;
    if (out) {
        double h[4];
        if (cudaMemcpyAsync(h, scratch, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess) return BH_ECUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return BH_ECUDA;
        out[0] = tk.t.ell;
        out[1] = h[0];
        out[2] = h[3];
        out[3] = h[3] > 0.0 ? h[1] / (h[3] * h[3] * h[2]) : 0.0;
    }
    return BH_OK;
}
}  // namespace BH_VARIANT
