#!/usr/bin/env python
"""Benchmark of the GPU GRMHD update (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the torus configuration the metric is quoted on): a Kerr black
hole (M = 1, a = 0.9375) on a uniform Cartesian 128^3 grid over
[-40, 40]^3, excision inside r = 1.2 r_H; a Fishbone-Moncrief torus with
r_in = 6, r_max = 12, Gamma = 4/3, atmosphere rho = 1e-6 r^-3/2, a seeded 4 %
pressure perturbation and a single field loop from A_phi ~ max(rho/rho_max -
0.2, 0) normalised to plasma beta = 100 -- stepped with RK2 at CFL 0.4 by the
corrected Valencia scheme (bhgpu.fixed: PLM with the MC limiter, HLL fluxes in each
face's normal, analytic Kerr-Schild sources, constrained transport, Newton
con2prim).  The reference's own scheme cannot run this configuration: it
throws std::domain_error in its first stage (src/fluid/physics/thermo.cpp:11).
Synthetic seeded data.

value : zone-updates/s of the mixed-precision form (reconstruction, fluxes
        and sources in FP32; conserved state, constrained transport,
        con2prim and dt in FP64), the step replayed as one CUDA graph;
        after the warm-up replays the torus is initialised again, so the K
        timed steps are steps 1..K of the run; device-timed with CUDA events,
        max over ranks; N > 1 runs one independent torus per GPU (weak
        scaling, no data-path collective).  The plain FP64 form (and the
        FMA-contracted FP64 form) are timed the same way beside it, and the
        mixed form's relative L1/Linf error against plain FP64 after 100
        steps from the same initial data is reported per conserved field
        with the face field's divergence.
e2e   : the same metric through the public API with host buffers
        (bhgpu.fixed.FxHostPipeline.submit_packed): per step the state a
        step reads (the interior cells' conserved fluid variables and
        previous primitives, the blocks' own face field), packed, goes up
        from pinned host memory, is unpacked, stepped and packed on the
        device, and comes back down; three device grids overlap the copies of
        neighbouring steps.
roofline : the kernel with the largest share of the step, its algorithmic
        bytes per launch over its CUDA-event duration, against the measured
        HBM copy bandwidth (MEASURED_PEAKS.json; fallback 6650 GB/s); the
        FP64/FP32 pipe peaks measured here by bh_peak_fma are reported beside
        it, since these kernels are instruction-bound.
cpu_baseline : the CPU port of the same scheme (oracle/bh_fixed.c,
        OpenMP over all host cores) on the same 128^3 torus.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "black-hole-simulator_b200"))
sys.path.insert(0, REPO)

METRIC = "zone-updates/s"
GAMMA = 4.0 / 3.0
CFL = 0.4
LO, HI = -40.0, 40.0
TORUS = dict(r_in=6.0, r_max=12.0, kappa=1e-3, beta=100.0, noise=0.04, seed=1)
STEP_BYTES = 296          # algorithmic HBM bytes per zone-update of an RK2 step
LAUNCHES_PER_STEP = 9     # dt init, then con2prim, ghosts, fluxes, update per stage (+1 per stage: split update)
# DRAM bytes (read + write) per launch of the mixed variant's step kernels at
# 128^3, from the ncu capture summarised in profiles/kernels_torus_128cube.md
# (the update as its two kernels, cells + faces: the autotuner's choice there)
PROFILED_TRAFFIC = {"fluxes": 155.20e6 + 173.36e6, "update": (381.83e6 + 108.76e6) + (70.69e6 + 29.07e6),
                    "prims": 190.98e6 + 145.83e6}
E2E_DEPTH = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--block", type=int, default=128, help="cells per block edge (the grid is one block by default)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=2, help="steps of the CPU port in cpu_baseline")
    ap.add_argument("--faithful", type=int, default=1, help="also time the reference-faithful FP64 path")
    ap.add_argument("--con2prim-batch", type=int, default=1, help="also measure the 2^24-cell con2prim batch")
    ap.add_argument("--amr", type=int, default=1, help="also measure the block-AMR configurations 3 and 5")
    ap.add_argument("--autotune", type=int, default=1,
                    help="choose the launch bounds of the heavy kernels on the torus first (bhgpu.fixed.autotune)")
    return ap.parse_args()


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons (every 50 ms);
    summary() keeps the samples time-stamped inside a host-time window."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_uuid: str | None):
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "50"]
        if gpu_uuid:
            cmd += ["-i", gpu_uuid]
        try:
            self.p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception as e:
            self.p, self.err = None, str(e)

    def stop(self, t0=None, t1=None):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvidia-smi unavailable: {self.err}"]}
        time.sleep(0.1)
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        rows = []
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                ts = time.mktime(time.strptime(f[0].split(".")[0], "%Y/%m/%d %H:%M:%S")) + float(
                    "0." + f[0].split(".")[1]) if "." in f[0] else 0.0
                rows.append((ts, float(f[1]), float(f[2]), f[4:8]))
            except ValueError:
                continue
        inside = [r for r in rows if t0 is not None and t0 - 0.05 <= r[0] <= t1 + 0.05]
        window = "timed region" if inside else "whole sampling span (no sample inside the timed region)"
        use = inside or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in use for n, v in zip(names, r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median([r[1] for r in use]) if use else None,
                "sm_max_mhz": max(r[2] for r in use) if use else None, "reasons": reasons,
                "samples": len(use), "window": window}


def gpu_uuid(dev):
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def l2_note(grid):
    """the mixed step's working set against the 126 MB L2: per cell of a
    block box U, U1 (FP64 x8), W (FP32 x8), face field and its stage copy
    (FP64 x3 each), fluxes (FP32 x24) = 304 bytes"""
    ws = (grid + 7) ** 3 * 304
    rel = "exceeds" if ws > 126e6 else "fits in"
    return f"working set {ws / 1e6:.0f} MB {rel} the 126 MB L2 (state, primitives, fluxes)"


def arm_config(args, world):
    return {"workload": f"Kerr-Schild torus {args.grid}^3 (configuration 2): a=0.9375 over [-40,40]^3, "
                        "Fishbone-Moncrief r_in=6 r_max=12, Gamma=4/3, beta=100 single loop, 4% pressure noise, "
                        "excision r<1.2 r_H; corrected Valencia scheme, PLM MC + HLL + CT, RK2 CFL 0.4",
            "grid": f"{args.grid}^3", "blocks": (args.grid // args.block) ** 3,
            "block": f"{args.block}^3 + 3 ghost layers (2 filled for PLM)", "parallelism": f"replicas x{world}",
            "l2": l2_note(args.grid),
            "run": "steps 1..K from the torus initial data (re-initialised after the warm-up replays; "
                   "every step continues the last)"}


# ---------------------------------------------------------------------------
def torus_grid(args, precision, limiter="mc", **kw):
    from bhgpu.fixed import FxGrid, FxParams
    g = FxGrid.uniform(LO, HI, args.grid, args.block, FxParams(precision=precision, limiter=limiter, **kw))
    info = g.torus_init(**TORUS)
    return g, info


def restart_torus(g):
    """the torus initial data again (into the same buffers, so a captured
    step graph stays valid) and the counters zeroed"""
    def restart():
        g.torus_init(**TORUS)
        g.reset_counters()
    return restart


def timed_steps(g, K, W, dist, clocks_uuid=False, restart=None):
    """ms per step of K graph replays after W warm-up replays (max over
    ranks); with clocks_uuid the SM clocks are sampled during the K steps.
    restart (the grid's initial data again) runs after the warm-up replays,
    so that the timed steps are steps 1..K of the run."""
    import torch
    g.capture()
    ck = Clocks(clocks_uuid or None) if clocks_uuid is not False else None
    for _ in range(W):
        g.replay()
    if ck is not None:       # let the sampler come up while the GPU keeps stepping
        torch.cuda.synchronize()
        t_w = time.time()
        while time.time() - t_w < 0.4:
            g.replay()
            torch.cuda.synchronize()
    if restart is not None:
        restart()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    a.record()
    for _ in range(K):
        g.replay()
    b.record()
    torch.cuda.synchronize()
    t1 = time.time()
    clocks = ck.stop(t0, t1) if ck else None
    t = torch.tensor([a.elapsed_time(b)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    g.release_graph()
    return float(t.item()) / K, clocks


def piece_ms(g, reps=5):
    """CUDA-event ms of each launch of a stage (stage 0 and 1 averaged)."""
    import torch
    out = {}
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name in ("prims", "ghosts", "fluxes", "update"):
        ts = []
        for stage in (0, 1):
            fn = {"prims": lambda: g.prims(stage, stage == 0), "ghosts": lambda: g.ghosts(stage),
                  "fluxes": lambda: g.fluxes(stage), "update": lambda: g.update(stage)}[name]
            fn()
            torch.cuda.synchronize()
            a.record()
            for _ in range(reps):
                fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) / reps)
        out[name] = sum(ts) / 2
    return out


def alg_bytes(piece, n, wb):
    """Algorithmic HBM bytes of one launch over one n^3 block (each value the
    launch must read or write, once); wb = bytes per primitive/flux value:
      prims:  U (5) and the face field (3) in, the previous primitives (5)
              in, primitives (8) and the cell field of U (3) out
      ghosts: 8 primitives and 3 face values per ghost cell, in and out
      fluxes: primitives of the (n+4)^3 stencil box; per face of the
              3 (n+1)(n+2)^2 the normal face field in and 8 flux components out
      update: 24 flux components, 8 primitives, U (and U1 at stage 1: 7.5
              values on average) in, 5 conserved out; 3 face values in and
              out"""
    cells, ghost = n ** 3, (n + 4) ** 3 - n ** 3
    faces = 3 * (n + 1) * (n + 2) ** 2
    if piece == "prims":
        return cells * ((5 + 3 + 3) * 8 + (5 + 8) * wb)
    if piece == "ghosts":
        return ghost * 2 * (8 * wb + 3 * 8)
    if piece == "fluxes":
        return (n + 4) ** 3 * 8 * wb + faces * (8 + 8 * wb)
    if piece == "update":
        return cells * (24 * wb + 8 * wb + 7.5 * 8 + 5 * 8 + 6 * 8)
    raise KeyError(piece)


def accuracy(args, steps, **kw):
    """plain FP64 and mixed from the same initial data, `steps` steps each"""
    import numpy as np
    import torch
    from bhgpu.fixed import FxGrid, FxParams
    ref, _ = torus_grid(args, "fp64")
    mix = FxGrid(ref.blocks_np, ref.nbr_np, FxParams(precision="mixed", **kw))
    mix.copy_state_from(ref)
    ref.capture()
    mix.capture()
    for _ in range(steps):
        ref.replay()
        mix.replay()
    torch.cuda.synchronize()
    ref.release_graph()
    mix.release_graph()
    a, b = mix.interior(mix.U), ref.interior(ref.U)
    fields = {"D": [0], "S": [1, 2, 3], "tau": [4], "B": [5, 6, 7]}
    out = {"steps": steps, "finite": bool(np.isfinite(a).all() and np.isfinite(b).all()),
           "rel_l1": {k: float(np.abs(a[c] - b[c]).sum() / np.abs(b[c]).sum()) for k, c in fields.items()},
           "rel_linf": {k: float(np.abs(a[c] - b[c]).max() / np.abs(b[c]).max()) for k, c in fields.items()},
           "div_B_rel": {"fp64": ref.divb(), "mixed": mix.divb()},
           "c2p_failures": {"fp64": ref.counters()["c2p_failures"], "mixed": mix.counters()["c2p_failures"]},
           "torus_rho_max": float(ref.interior(ref.W)[0].max())}
    out["max_rel_l1"] = max(out["rel_l1"].values())
    out["within_1e-5"] = out["max_rel_l1"] <= 1e-5
    del ref, mix
    torch.cuda.empty_cache()
    return out


def e2e_measure(args, g0, dist):
    import torch
    from bhgpu.fixed import FxGrid, FxHostPipeline
    # the state a step reads, packed: the interior cells' rows 0-4 of U and W
    # (the cell-centred field rows are recomputed from the face field on the
    # device) and the blocks' own faces
    nbytes = g0.state_nbytes()
    dbuf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    g0.pack_state(dbuf)
    torch.cuda.synchronize()
    hin = dbuf.cpu().pin_memory()
    del dbuf
    grids = [g0] + [FxGrid(g0.blocks_np, g0.nbr_np, g0.params) for _ in range(E2E_DEPTH - 1)]
    outs = [torch.empty_like(hin).pin_memory() for _ in range(E2E_DEPTH)]

    def run(pipe, nstep):
        for i in range(len(pipe.grids)):
            pipe.submit_packed(hin, outs[i])
        pipe.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(pipe.s_in)
        for i in range(nstep):
            pipe.submit_packed(hin, outs[i % len(pipe.grids)])
        b.record(pipe.s_out)
        torch.cuda.synchronize()
        t = torch.tensor([a.elapsed_time(b)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()) / nstep

    ms = run(FxHostPipeline(grids), args.e2e_steps)
    ms_serial = run(FxHostPipeline(grids[:1]), max(3, args.e2e_steps // 3))
    del grids
    return ms, ms_serial, nbytes


def cpu_port_sample(args, threads, steps):
    """The CPU port of the scheme (oracle/bh_fixed.c, OpenMP) on the same
    torus: zone-updates/s over `steps` steps after one warm-up step."""
    import oracle
    from oracle import fixed as ofx
    from bhgrid.blocks import uniform_blocks
    os.environ["OMP_NUM_THREADS"] = str(threads)
    oracle.build(ref=False)

    class _P:
        M, a, gamma, cfl, rho_floor, u_floor, sigma_max, W_max = 1.0, 0.9375, GAMMA, CFL, 1e-6, 1e-8, 100.0, 50.0
        r_exc, tol, maxiter, limiter = None, 1e-12, 30, "mc"
    blocks, nbr = uniform_blocks(LO, HI, args.grid, args.block)
    h = ofx.FxHost(blocks, nbr, ofx.params(_P))
    h.torus_init(**TORUS)
    h.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        h.step()
    t = time.perf_counter() - t0
    return args.grid ** 3 * steps / t, t / steps


def reference_scheme_cpu(threads):
    """The reference's own rk2integrator::step (oracle/_ref, its OpenMP
    loops) on the 64^3 magnetised box it can run (outflow, van Leer)."""
    import oracle
    from bhgrid import configs
    from bhgrid.mesh import Quilt
    if not oracle.ref_available():
        return {"unavailable": "the reference harness (oracle/_ref) is not built on this host"}
    os.environ["OMP_NUM_THREADS"] = str(threads)
    q = Quilt([10.0] * 3, [12.0] * 3, 4, periodic=False)
    W, Bf = configs.magnetised_box(q, seed=1, gamma=GAMMA)
    orc = oracle.Oracle(0.0, 0.0, 0.0, GAMMA, limiter=1)
    hp = oracle.HostPool(q.tables())
    orc.geometry(hp)
    hp.W[:] = W
    hp.Bf[:] = Bf
    for p in range(hp.npatch):
        hp.U[p] = orc.ptoc(W[p], hp.rth[p, 0], hp.rth[p, 1])[0]
    ref = oracle.RefSolver([10.0] * 3, [12.0] * 3, 4, 0.0, 0.0, 0.0, GAMMA)
    times = []
    for _ in range(3):
        ref.put(hp)
        t0 = time.perf_counter()
        ref.step_native(CFL)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": 64 ** 3 / t, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": "the reference's own rk2integrator::step on the 64^3 magnetised box it can run "
                      f"(outflow, van Leer), median of 3 steps from the initial state, {t:.2f} s/step"}


def faithful_gpu(steps=20):
    """The reference-faithful FP64 path (bhgpu.RK2Integrator, the reference's
    own arithmetic) on the 128^3 magnetised box, each step restarted."""
    import torch
    import bhgpu
    from bhgrid import configs
    from bhgrid.mesh import Quilt
    q = Quilt([10.0] * 3, [12.0] * 3, 8, periodic=True)
    tree = bhgpu.AmrTree(q.dom_l, q.dom_h, 8, M=0.0, a=0.0, Q=0.0, gm=GAMMA, periodic=True, limiter="minmod",
                         quilt=q, init_floor=False, precision="fp64")
    W, Bf = configs.magnetised_box(q, seed=1, gamma=GAMMA)
    tree.load(W=W, Bf=Bf)
    tree.prim_to_cons()
    U0, W0, B0 = tree.U.clone(), tree.W.clone(), tree.Bf.clone()
    rk = bhgpu.RK2Integrator(CFL)

    def one():
        tree.U.copy_(U0)
        tree.W.copy_(W0)
        tree.Bf.copy_(B0)
        rk.step(tree, sync=False, check_domain=False)
    for _ in range(3):
        one()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        one()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    tree.clear_error()
    return {"workload": "magnetised box 128^3 (flat, periodic, PLM minmod + the reference's HLLD + CT), "
                        "reference-faithful FP64 (the reference's roundings), each step restarted",
            "ms_per_step": ms, "zone_updates_per_s": 128 ** 3 / (ms / 1e3)}


# ---------------------------------------------------------------------------
# con2prim stress batch: 2^24 independent Kerr cells (a = 0.9375)
C2P_ALG_BYTES = 8 * 8 + 2 * 8 + 5 * 8 + 4   # U + (r, theta) in; rho, eps, v out; iterations


def con2prim_batch(n_cells=1 << 24, reps=3):
    import numpy as np
    import torch
    import bhgpu
    from bhgrid import configs
    W, r, th = configs.con2prim_batch(n_cells, seed=4, gamma=GAMMA, a=0.9375)
    mtr, stt = bhgpu.Metric(1.0, 0.9375, 0.0), bhgpu.State(GAMMA)
    cn = bhgpu.Conserved(mtr, stt)
    U, _ = cn.ptoc(W, r, th, check_domain=False)
    rd, thd = torch.as_tensor(r, device="cuda"), torch.as_tensor(th, device="cuda")
    cn.ctop(U, rd, thd, check_domain=False)      # warm-up
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
    # each call's outputs are dropped before the next call allocates its own,
    # so that the caching allocator reuses the same blocks (no cudaMalloc in
    # the timed loop, whatever the cache held before)
    res = None
    a.record()
    for _ in range(reps):
        res = None
        res = cn.ctop(U, rd, thd, check_domain=False)
    b.record(); torch.cuda.synchronize()
    Wg, _, st, it, pa = res
    ms = a.elapsed_time(b) / reps
    st, it, pa = st.cpu().numpy(), it.cpu().numpy(), pa.cpu().numpy()
    Wg0 = Wg.cpu().numpy()
    out = {"workload": f"con2prim stress batch: {n_cells} independent Kerr-Schild cells (a=0.9375, Gamma=4/3), "
                       "log-uniform rho, W in [1,20], log-uniform sigma, isotropic v and B, r in [1.5,50]",
           "cells": n_cells, "ms": ms, "cells_per_s": n_cells / (ms / 1e3),
           "recovered_frac": float(np.mean(st == 1)), "failed_frac": float(np.mean(st == 0)),
           "domain_error_frac": float(np.mean(st < 0)),
           "routes": {"newton": float(np.mean(pa == 0)), "newton_cap": float(np.mean(pa == 1)),
                      "brent": float(np.mean(pa == 2)), "brent_failed": float(np.mean(pa == 3))},
           "mean_newton_iters": float(it.mean()),
           "alg_bytes_per_cell": C2P_ALG_BYTES,
           "achieved_GBs": n_cells * C2P_ALG_BYTES / (ms / 1e3) / 1e9}
    # the learned initial guess: trained on this batch's first 2^16 cells,
    # timed (preamble + network + con2prim) on the whole batch
    try:
        g = bhgpu.C2PGuess(cn, seed=0)
        t0 = time.perf_counter()
        g.train(U[:, :1 << 16].contiguous(), rd[:1 << 16].contiguous(), thd[:1 << 16].contiguous(), steps=1500)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        g.ctop(U, rd, thd)
        torch.cuda.synchronize()
        res = None
        a.record()
        for _ in range(reps):
            res = None
            res = g.ctop(U, rd, thd)
        b.record(); torch.cuda.synchronize()
        Wg, Wdg, stg, itg, pag = res
        msg = a.elapsed_time(b) / reps
        stg_, itg_ = stg.cpu().numpy(), itg.cpu().numpy()
        both = (st == 1) & (stg_ == 1)
        out["mlp_guess"] = {"network": "6-64-64-2 tanh, BF16 weights, FP32 math, trained on the GPU on 2^16 "
                                       "solver-generated pairs (1500 Adam steps)",
                            "train_s": t_train, "ms": msg, "cells_per_s": n_cells / (msg / 1e3),
                            "mean_newton_iters_where_both_recover": {"plain": float(it[both].mean()),
                                                                     "guess": float(itg_[both].mean())},
                            "failed_frac": {"plain": float(np.mean(st != 1)), "guess": float(np.mean(stg_ != 1))},
                            "other_root_frac": float(np.mean(np.abs(Wg[0].cpu().numpy()[both] - Wg0[0][both]) >
                                                             1e-6 * np.abs(Wg0[0][both])))}
        # the same with the network on the tensor cores (bh_ctop_learned)
        g.ctop_learned(U, rd, thd)
        torch.cuda.synchronize()
        err_t = torch.zeros(1, dtype=torch.int32, device="cuda")   # checked after the loop: no sync per call
        res = None
        a.record()
        for _ in range(reps):
            res = None
            res = g.ctop_learned(U, rd, thd, err=err_t)
        b.record(); torch.cuda.synchronize()
        Wt, Wdt, stt_, itt, pat = res
        mst = a.elapsed_time(b) / reps
        if int(err_t.item()) != 0:
            raise RuntimeError(f"bh_ctop_learned: device error word {int(err_t.item())} in the timed loop")
        # its second kernel alone (Newton / Brent from the same starting points)
        xi0t = g.ctop_learned(U, rd, thd, want_xi0=True)[5]
        torch.cuda.synchronize()
        res = None
        a.record()
        for _ in range(reps):
            res = None
            res = g.ctop_from(U, rd, thd, xi0t)
        b.record(); torch.cuda.synchronize()
        res = None
        ms_newton = a.elapsed_time(b) / reps
        stt_, itt = stt_.cpu().numpy(), itt.cpu().numpy()
        both_t = (st == 1) & (stt_ == 1)
        fail_t = (st != 1) & (stt_ != 1)
        out["mlp_guess"]["tensor_core"] = {
            "kernels": "k_guess_tc (metric, preamble, network as tcgen05.mma BF16 -> FP32 in TMEM, 128-cell "
                       "tiles, persistent CTAs) + k_ctop_guess (Newton / Brent, one thread per cell)",
            "ms": mst, "guess_kernel_ms": mst - ms_newton, "newton_kernel_ms": ms_newton,
            "cells_per_s": n_cells / (mst / 1e3), "speedup_vs_plain": ms / mst,
            "mean_newton_iters_where_both_recover": {"plain": float(it[both_t].mean()),
                                                     "guess": float(itt[both_t].mean())},
            "mean_newton_iters_all_cells": {"plain": float(it.mean()), "guess": float(itt.mean())},
            "mean_newton_iters_where_both_fail": {"plain": float(it[fail_t].mean()),
                                                  "guess": float(itt[fail_t].mean())},
            "failed_frac": float(np.mean(stt_ != 1)),
            "status_equal_to_three_kernel_form": float(np.mean(stt_ == stg_))}
    except Exception as e:      # informational
        out["mlp_guess"] = {"error": str(e)}
    # the reference's own conserved::ctop on a sample, all host threads
    try:
        import oracle
        if oracle.ref_available():
            ns = 1 << 16
            ref = oracle.RefSolver([10.0] * 3, [12.0] * 3, 1, 1.0, 0.9375, 0.0, GAMMA)
            Us = U[:, :ns].cpu().numpy()
            t0 = time.perf_counter()
            ref.ctop(Us, r[:ns], th[:ns])
            t = time.perf_counter() - t0
            out["cpu_reference"] = {"cells_per_s": ns / t, "cores": os.cpu_count() or 1,
                                    "sample": f"reference conserved::ctop on the first {ns} cells"}
    except Exception as e:      # the CPU figure is informational
        out["cpu_reference"] = {"error": str(e)}
    return out

# ---------------------------------------------------------------------------
# block AMR: equal cubes (8 per axis over [-40, 40]^3) at several levels, all
# blocks of all sizes in one launch per kernel (persistent CTAs fed by the
# device work queue), the step replayed as a CUDA graph
AMR_CONFIGS = {
    "config3": {"n0": 8, "r_fine": (14.0, 26.0), "seed": 3, "accuracy_steps": 100,
                "what": "3 levels: blocks of 8^3, 16^3 and 32^3 cells (+3 ghost layers), seeded uneven mix "
                        "concentrated near the hole"},
    "config5": {"n0": 4, "r_fine": (10.0, 18.0, 28.0), "seed": 5, "accuracy_steps": 200,
                "what": "4 levels: blocks of 4^3 to 32^3 cells, effective 256^3 at the finest level"},
}


def amr_bench(warm, steps, autotuned=None):
    import numpy as np
    import torch
    from bhgpu.fixed import FxGrid, FxParams
    from bhgrid.blocks import torus_levels
    peak, _ = measured_peaks()
    out = {}
    for name, c in AMR_CONFIGS.items():
        lv = torus_levels(nb=8, r_fine=c["r_fine"], seed=c["seed"])
        n_of = {l: c["n0"] << l for l in range(int(lv.max()) + 1)}
        zones = int(sum((n_of[int(l)] ** 3) for l in lv.ravel()))
        res = {"workload": f"Kerr-Schild torus on 512 equal cubes over [-40,40]^3, {c['what']}",
               "blocks_per_size": {f"{n_of[l]}^3": int((lv == l).sum()) for l in n_of},
               "zones": zones, "torus": dict(TORUS)}
        for prec, persistent in (("mixed", True), ("mixed", False), ("fp64", True)):
            g = FxGrid.leveled(LO, HI, lv, c["n0"], FxParams(precision=prec), persistent=persistent)
            g.torus_init(**TORUS)
            ms, _ = timed_steps(g, steps, warm, None, restart=restart_torus(g))
            key = f"{prec}{'' if persistent else '_one_cta_per_item'}"
            res[key] = {"ms_per_step": ms, "zone_updates_per_s": zones / (ms / 1e3),
                        "hbm_frac_296B": zones / (ms / 1e3) * STEP_BYTES / (peak * 1e9)}
            del g
            torch.cuda.empty_cache()
        res["mixed_vs_plain_fp64_speedup"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
        # accuracy after the configuration's step count
        ref = FxGrid.leveled(LO, HI, lv, c["n0"], FxParams(precision="fp64"), persistent=True)
        ref.torus_init(**TORUS)
        mix = FxGrid(ref.blocks_np, ref.nbr_np, FxParams(precision="mixed"), persistent=True)
        mix.copy_state_from(ref)
        ref.capture()
        mix.capture()
        for _ in range(c["accuracy_steps"]):
            ref.replay()
            mix.replay()
        torch.cuda.synchronize()
        ref.release_graph()
        mix.release_graph()
        a, b = mix.U.cpu().numpy(), ref.U.cpu().numpy()
        fields = {"D": [0], "S": [1, 2, 3], "tau": [4], "B": [5, 6, 7]}
        res["accuracy"] = {"steps": c["accuracy_steps"], "finite": bool(np.isfinite(a).all()),
                           "rel_l1": {k: float(np.abs(a[f] - b[f]).sum() / np.abs(b[f]).sum()) for k, f in fields.items()},
                           "div_B_rel": {"fp64": ref.divb(), "mixed": mix.divb()},
                           "c2p_failures": {"fp64": ref.counters()["c2p_failures"],
                                            "mixed": mix.counters()["c2p_failures"]}}
        del ref, mix
        torch.cuda.empty_cache()
        out[name] = res
    return out


# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference arm: the same torus on the host cores.  The reference's
    own scheme cannot step it (std::domain_error in its first stage), so the
    timed implementation is the CPU port of the scheme this repository runs
    on the GPU (oracle/bh_fixed.c), OpenMP over all host threads."""
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    nsteps = max(1, min(args.steps, 10))
    value, s_per_step = cpu_port_sample(args, threads, nsteps)
    sample = (f"each step: one RK2 step of the {args.grid}^3 torus by the CPU port of the corrected scheme "
              f"(oracle/bh_fixed.c, {threads} OpenMP threads); {nsteps} of the {args.steps} steps timed "
              f"after 1 warm-up step, {s_per_step:.2f} s/step")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * s_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": arm_config(args, world),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's own rk2integrator::step cannot run this configuration (its EOS throws "
                    "std::domain_error in the first stage, src/fluid/physics/thermo.cpp:11); "
                    "reference_scheme times it on the box it can run",
            "reference_scheme": reference_scheme_cpu(threads)}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    from bhgpu import peaks
    warm = max(args.warmup, 3)
    uuid = gpu_uuid(local_rank)

    from bhgpu.fixed import autotune
    tuning = {}
    # the headline: the mixed form
    g, info = torus_grid(args, "mixed")
    if args.autotune:
        tuning["mixed"] = autotune(g)
    ms_mixed, clocks = timed_steps(g, args.steps, warm, dist, clocks_uuid=uuid or "", restart=restart_torus(g))
    counters = g.counters()
    divb_after = g.divb()
    pieces = {"mixed": piece_ms(g)}
    ms_e2e, ms_e2e_serial, nbytes = e2e_measure(args, g, dist)
    del g
    torch.cuda.empty_cache()
    variants = {}
    for prec in ("fp64", "fp64-fma"):
        gv, _ = torus_grid(args, prec)
        if args.autotune:
            tuning[prec] = autotune(gv)
        ms_v, _ = timed_steps(gv, args.steps, warm, dist, restart=restart_torus(gv))
        variants[prec] = {"ms_per_step": ms_v, "zone_updates_per_s": world * args.grid ** 3 / (ms_v / 1e3)}
        if prec == "fp64":
            pieces["fp64"] = piece_ms(gv)
        del gv
        torch.cuda.empty_cache()
    # PPM reconstruction (three ghost layers, unstaged flux kernel) beside it
    ppm = {}
    for prec in ("mixed", "fp64"):
        gv, _ = torus_grid(args, prec, "ppm")
        ms_v, _ = timed_steps(gv, args.steps, warm, dist, restart=restart_torus(gv))
        ppm[prec] = {"ms_per_step": ms_v, "zone_updates_per_s": world * args.grid ** 3 / (ms_v / 1e3)}
        del gv
        torch.cuda.empty_cache()
    ppm["mixed_vs_plain_fp64"] = ppm["fp64"]["ms_per_step"] / ppm["mixed"]["ms_per_step"]
    # the mixed variant with every cell's con2prim ending in FP64 Newton iterations
    gv, _ = torus_grid(args, "mixed", c2p_fp64=True)
    ms_v, _ = timed_steps(gv, args.steps, warm, dist, restart=restart_torus(gv))
    del gv
    torch.cuda.empty_cache()
    strict = {"ms_per_step": ms_v, "zone_updates_per_s": world * args.grid ** 3 / (ms_v / 1e3),
              "speedup_vs_plain_fp64": variants["fp64"]["ms_per_step"] / ms_v,
              "accuracy_after_steps": accuracy(args, args.accuracy_steps, c2p_fp64=True)}
    acc = accuracy(args, args.accuracy_steps)
    if dist:
        dist.barrier()

    if rank == 0:
        zones = args.grid ** 3
        value = world * zones / (ms_mixed / 1e3)
        peak, peak_kind = measured_peaks()
        fp64_tf, fp32_tf = peaks.fma_peak("fp64"), peaks.fma_peak("fp32")
        nblk = (args.grid // args.block) ** 3
        share = {k: v * 2 / ms_mixed for k, v in pieces["mixed"].items()}
        top = max(pieces["mixed"], key=lambda k: pieces["mixed"][k])
        top_ms = pieces["mixed"][top]
        byts = alg_bytes(top, args.block, 4) * nblk
        achieved = byts / (top_ms * 1e-3) / 1e9
        from bhgpu.fixed import tune_get
        flux_k = "k_fx_flux_tile" if tune_get("mixed", "stage") else "k_fx_flux"
        kname = {"prims": "k_fx_c2p<float>", "ghosts": "k_fx_ghost<float>", "fluxes": f"{flux_k}<float,float,float>",
                 "update": "k_fx_update<float,float,float>"}[top]
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "precision": "mixed (reconstruction, fluxes, sources FP32; state, CT, con2prim, dt FP64)",
            "config": arm_config(args, world),
            "mixed_vs_plain_fp64": {"speedup": variants["fp64"]["ms_per_step"] / ms_mixed,
                                    "speedup_vs_fp64_fma": variants["fp64-fma"]["ms_per_step"] / ms_mixed,
                                    "accuracy_after_steps": acc},
            "variants": variants,
            "ppm": ppm,
            "mixed_c2p_fp64": strict,
            "torus": {"ell": info["ell"], "field_scale": info["field_scale"], "beta": info["beta"],
                      "div_B_rel_after_timed_steps": divb_after, "counters_after_timed_steps": counters},
            "e2e": {"value": world * zones / (ms_e2e / 1e3), "unit": METRIC, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "ms_per_step": ms_e2e,
                    "api": f"bhgpu.fixed.FxHostPipeline.submit_packed, {E2E_DEPTH} device grids, the packed state "
                           "(interior cells' U and W rows 0-4, the blocks' own faces) from pinned host memory in and "
                           "out every step, unpacked and packed on the device",
                    "serial_value": world * zones / (ms_e2e_serial / 1e3), "serial_ms_per_step": ms_e2e_serial},
            "gpu_launches": (LAUNCHES_PER_STEP + (2 if tune_get("mixed", "split") else 0)) * args.steps,
            "roofline": {"bound": "hbm", "kernel": f"{kname} ({top})", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": PROFILED_TRAFFIC.get(top) if args.grid == 128 else None,
                         "traffic_source": "ncu capture of the same kernel at 128^3 "
                                           "(profiles/kernels_torus_128cube.md)", "peak_source": peak_kind,
                         "ms_per_launch": top_ms, "alg_bytes_per_launch": byts,
                         "launch_ms": {k: {p: round(v, 5) for p, v in d.items()} for k, d in pieces.items()},
                         "step_share": {k: round(v, 4) for k, v in share.items()},
                         "step_frac": value / world * STEP_BYTES / (peak * 1e9),
                         "fp_pipe_peaks_tflops": {"fp64": fp64_tf, "fp32": fp32_tf,
                                                  "source": "bh_peak_fma on this GPU"}},
            "clocks": clocks,
            "autotune": ({p: {"choice_ctas_per_sm": t["choice"],
                              "step_ms_per_candidate": {k: {str(c): round(m, 4) for c, m in v.items()}
                                                        for k, v in t["ms"].items()}}
                          for p, t in tuning.items()} if tuning else "off (ptxas's own register choice)"),
        }
        if world == 1:
            threads = os.cpu_count() or 1
            v, s_per = cpu_port_sample(args, threads, args.cpu_steps)
            line["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                                    "sample": f"{args.cpu_steps} RK2 steps of the same {args.grid}^3 torus by the "
                                              f"CPU port of the scheme (oracle/bh_fixed.c, OpenMP), "
                                              f"{s_per:.2f} s/step"}
            line["reference_scheme_cpu"] = reference_scheme_cpu(threads)
            if args.amr:
                line["block_amr"] = amr_bench(warm, min(args.steps, 20))
            if args.faithful:
                line["reference_faithful_gpu"] = faithful_gpu()
            if args.con2prim_batch:
                line["con2prim_batch"] = con2prim_batch()
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
