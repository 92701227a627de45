"""Loads the golden fixtures written by make_golden.py into host.Problem
objects (the arrays exactly as the reference handed them to its device
layer) plus the reference's final state."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

from esdgsem_mpiocca_b200 import host

HERE = os.path.dirname(os.path.abspath(__file__))


def names():
    """Solver fixtures (state after a reference run)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "*.npz"))
                  if not os.path.basename(p).startswith("okada"))


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    p = host.Params(**meta["params"])
    if meta.get("reference_h_zero") is not None:  # the h_0 the reference's analysis kernels measured from
        p.h_0 = float(meta["reference_h_zero"])
    N = p.N
    n2 = (N + 1) ** 2
    K = z["Jinv"].size // n2
    F = z["EdgeReversed"].size
    mesh = host.MeshArrays(N, K, F, z["x"], z["y"], z["x_xi"], z["x_eta"], z["y_xi"], z["y_eta"], z["Jinv"],
                           z["nx"], z["ny"], z["scal"], z["b"], z["EdgeData"].astype(np.int32),
                           z["EdgeReversed"].astype(np.int32), z["ElemToEdge"].astype(np.int32),
                           z["MasterSlave"].astype(np.int32), z["Orientation"].astype(np.int32))
    basis = host.Basis.build(N, p.FluxDifferencing)
    # the matrices the reference used (identical to basis' -- checked by tests)
    basis.D, basis.Dstrong, basis.Dhat, basis.VdmInv = z["D"], z["Dstrong"], z["Dhat"], z["VdmInv"]
    if "DcFD" in z.files:  # copyPartialDryData's matrices (partial-dry runs)
        basis.fd_mats = (z["DcFD"], z["DfFD"], z["DbFD"])
    EleSizes = z["EleSizes"]
    minEle = float(np.sqrt(EleSizes.min()))
    prob = host.Problem(p, basis, mesh, z["b"], z["Bx"], z["By"], z["q"], EleSizes, minEle, z["rkA"], z["rkB"],
                        z["rkC"], meta)
    return prob, z["q_final"], z
