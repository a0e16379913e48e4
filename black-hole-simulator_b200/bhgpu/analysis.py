"""analysis::analyser (src/fluid/analysis.hpp:52-80, data/quantitatives.cpp)
on the device.

The integrals -- vol_int (:44-59) and surf_int (:61-79) of each integrand
times the cell volume over the leaf patches' interior cells -- run on the GPU
(bh_analysis); the quantities the reference builds from them (Phi_B, MAD,
eta_BZ, Pbeta, alpha_ss, maxreyn, Hscal) are composed here with the
reference's arithmetic.  The integrands read the derived primitive fields
(Lorentz factor, pressure, enthalpy, b^2) that floors and regrid record, so
the analyser is meant for the state right after RK2Integrator.step or
AmrTree.regrid -- where the reference's main() calls it (main.cpp:172-186).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from ._lib import BH_NQ, BhAnalysisParams, check, lib
from .solver import AmrTree, _p, _stream

# order of the raw integrals (include/bhgpu.h, BH_Q_*)
Q = ("mass", "energy", "L_pol", "Mdot", "Edot", "Ldot", "Phi_B_int", "magE", "thermE", "L_BZ", "p_int",
     "pmag_int", "stress", "ptot", "stress_bundle", "ptot_bundle", "maxwell", "reynolds", "H_num", "H_den")
QI = {k: i for i, k in enumerate(Q)}

BATCH_FIELDS = ("t", "mass", "energy", "L_pol", "Mdot", "Edot", "Ldot", "Phi_B", "MAD", "magE", "thermE",
                "L_BZ", "eta_BZ", "Pbeta", "alpha_ss", "maxreyn", "Hscal")    # struct batch, analysis.hpp:15-38
BUNDLE_FIELDS = ("t", "mass", "Mdot", "MAD", "L_BZ", "alpha_ss")               # struct bundle, :39-47


def r_horizon(M: float, a: float, Q_: float) -> float:
    """quantitatives.cpp:19-22 (NaN where std::sqrt would be)"""
    d = M * M - a * a - Q_ * Q_
    return M + (math.sqrt(d) if d >= 0 else math.nan)


def compose_batch(q, t: float, M: float, a: float, Q_: float) -> dict:
    """analyser::batch_ (:222-247) from the raw integrals."""
    Mdot = q[QI["Mdot"]]
    Phi_B = 0.5 * q[QI["Phi_B_int"]]
    L_BZ = q[QI["L_BZ"]]
    md = abs(Mdot)
    den, reyn, hden = q[QI["pmag_int"]], q[QI["reynolds"]], q[QI["H_den"]]
    press = q[QI["ptot"]]
    rs = 10.0 * M
    return {
        "t": t, "mass": q[QI["mass"]], "energy": q[QI["energy"]], "L_pol": q[QI["L_pol"]],
        "Mdot": Mdot, "Edot": q[QI["Edot"]], "Ldot": q[QI["Ldot"]], "Phi_B": Phi_B,
        "MAD": 0.0 if abs(Mdot) < 1e-30 else Phi_B / Mdot,
        "magE": q[QI["magE"]], "thermE": q[QI["thermE"]], "L_BZ": L_BZ,
        "eta_BZ": L_BZ / md if md > 1e-25 else 0.0,
        "Pbeta": q[QI["p_int"]] / den if den > 1e-20 else 1e30,
        "alpha_ss": q[QI["stress"]] / press if press > 1e-25 else 0.0,
        "maxreyn": q[QI["maxwell"]] / reyn if abs(reyn) > 1e-30 else 0.0,
        "Hscal": (q[QI["H_num"]] / hden) / rs if hden > 1e-20 else 0.0,
    }


def compose_bundle(q, t: float) -> dict:
    """analyser::bundle_ (:205-220) from the raw integrals."""
    Mdot = q[QI["Mdot"]]
    Phi_B = 0.5 * q[QI["Phi_B_int"]]
    press = q[QI["ptot_bundle"]]
    return {"t": t, "mass": q[QI["mass"]], "Mdot": Mdot,
            "MAD": 0.0 if abs(Mdot) < 1e-30 else Phi_B / Mdot, "L_BZ": q[QI["L_BZ"]],
            "alpha_ss": q[QI["stress_bundle"]] / press if press > 1e-25 else 0.0}


class Analyser:
    """analysis::analyser: batch_ and bundle_ of an AmrTree's state."""

    def integrals(self, tree: AmrTree, hrz: float, rs: float, rho_min_full: float = 0.01,
                  rho_min_bundle: float = 0.005) -> np.ndarray:
        partial = torch.empty((max(int(tree.leaves.numel()), 1), BH_NQ), dtype=torch.float64, device=tree.device)
        out = torch.zeros(BH_NQ, dtype=torch.float64, device=tree.device)
        A = BhAnalysisParams(hrz, rs, rho_min_full, rho_min_bundle)
        P = tree.params()
        check(lib.bh_analysis(C.byref(P), C.byref(tree.pool), C.byref(A), _p(partial), _p(out), _stream()),
              "analysis::analyser")
        return out.cpu().numpy()

    def _params(self, tree):
        m = tree.mtr
        return m.M, m.a, m.Q

    def batch_(self, tree: AmrTree, t: float) -> dict:
        M, a, Q_ = self._params(tree)
        q = self.integrals(tree, r_horizon(M, a, Q_), 10.0 * M)
        return compose_batch(q, t, M, a, Q_)

    def bundle_(self, tree: AmrTree, t: float) -> dict:
        M, a, Q_ = self._params(tree)
        q = self.integrals(tree, r_horizon(M, a, Q_), 10.0 * M)
        return compose_bundle(q, t)
