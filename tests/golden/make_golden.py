"""Generates the golden fixtures in tests/golden/*.npz from runs of the
reference program itself (oracle/_ref/esdg_ref: the reference's main.cpp and
src/*.cpp compiled unmodified against the OCCA-v0 shim, kernels from its own
okl/ files).  Run in a container that has the reference tree:

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py CASE ...   # selected cases

Each fixture holds every array the reference handed to copyDeviceVariables
(its own set-up, or the injected initial state / bathymetry), the time-loop
parameters, and q after its DGtimeloop (o_q.copyTo at main.cpp:1051).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from esdgsem_mpiocca_b200 import host, problems  # noqa: E402
from oracle import run_ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def gaussian_state(x, y, seed, depth=1.0, ripple=0.02, nb=3):
    rng = np.random.default_rng(seed)
    lx, ly = x.max() - x.min(), y.max() - y.min()
    b = np.zeros_like(x)
    for _ in range(nb):
        a = rng.uniform(0.05, 0.2)
        w = rng.uniform(0.1, 0.25) * min(lx, ly)
        cx = rng.uniform(x.min(), x.max())
        cy = rng.uniform(y.min(), y.max())
        b += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / w ** 2)
    cx, cy = x.min() + 0.4 * lx, y.min() + 0.55 * ly
    h = depth - b + ripple * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (0.15 * min(lx, ly)) ** 2)
    return b, h


def pack_q(h, hu=None, hv=None, n2=None):
    K = h.size // n2
    q = np.zeros((K, 3, n2))
    q[:, 0] = h.reshape(K, n2)
    if hu is not None:
        q[:, 1] = hu.reshape(K, n2)
    if hv is not None:
        q[:, 2] = hv.reshape(K, n2)
    return q.reshape(-1)


def bottom_derivs(ref_setup, N, b):
    """Bx, By of b on the reference's own geometry (its CalcBDerivatives is
    bypassed by injection, so they are recomputed here on its arrays)."""
    K = ref_setup["Jinv"].size // (N + 1) ** 2
    mesh = host.MeshArrays(N, K, ref_setup["EdgeReversed"].size, ref_setup["x"], ref_setup["y"], ref_setup["x_xi"],
                           ref_setup["x_eta"], ref_setup["y_xi"], ref_setup["y_eta"], ref_setup["Jinv"],
                           ref_setup["nx"], ref_setup["ny"], ref_setup["scal"], b, ref_setup["EdgeData"],
                           ref_setup["EdgeReversed"], ref_setup["ElemToEdge"], ref_setup["MasterSlave"],
                           ref_setup["Orientation"])
    return host.bottom_derivatives(mesh, host.Basis.build(N), b)


def save(name, params, out, meta):
    arrays = {k: v for k, v in out.items() if isinstance(v, np.ndarray)}
    rk = host.rk_coefficients(params.rkOrder, params.rkSSP)
    arrays["rkA"], arrays["rkB"], arrays["rkC"] = rk
    p = {k: getattr(params, k) for k in vars(params)}
    meta = dict(meta)
    meta["params"] = p
    meta["reference_stdout_tail"] = out["stdout"][-400:]
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrays)
    print(f"{name}: K={out['Jinv'].size // (params.N + 1) ** 2} wall={out['wall']:.2f}s")


def case_periodic(numflux, name):
    pr = problems.periodic_bump(NumFlux=numflux, steps=0)
    pr.params.T = 0.1
    out = run_ref.run(name, pr.params, cartesian=(0.0, 2.0, 0.0, 2.0, 16, 16, 1, 1),
                      inject={"q": pr.q0, "b": pr.b, "Bx": pr.Bx, "By": pr.By})
    save(name, pr.params, out, {"mesh": "Cartesian periodic 16x16 on [0,2]^2", "state": "periodic_bump"})


def case_mapped_rotated(name="mapped_rot_N4", N=4):
    """Curved 8x8 mesh with rotated element corners, written as ISM-V2 by the
    engine's writer and read by the reference's Mesh::ReadMesh."""
    params = host.Params(N=N, CFL=0.4, T=0.02, NumFlux=0, rkOrder=4, rkSSP=0)
    rd = os.path.join(ROOT, "oracle", "_ref", "meshes")
    os.makedirs(rd, exist_ok=True)
    path = os.path.join(rd, "mapped_rot.mesh")
    m = host.mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, 8, 8, amp=0.03, curve_order=5, rotate_seed=7, write_path=path)
    b, h = gaussian_state(m.x, m.y, seed=11)
    setup = run_ref.run(name + "_setup", params, mesh_file=path)
    Bx, By = bottom_derivs(setup, N, b)
    out = run_ref.run(name, params, mesh_file=path, inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx,
                                                            "By": By})
    save(name, params, out, {"mesh": "engine-written ISM-V2: curved 8x8, rotated corners, order 5", "walls": True})


def case_circle(name, N=3, AV=0, T=0.01, state="lake"):
    params = host.Params(N=N, CFL=0.4, DFL=0.1, T=T, NumFlux=0, rkOrder=4, rkSSP=0, ArtificialViscosity=AV,
                         epsilon_0=0.02, sigma_min=-6.0, sigma_max=-2.0)
    mf = "meshFiles/CircleInCircle.mesh"
    setup = run_ref.run(name + "_setup", params, mesh_file=mf)
    x, y = setup["x"], setup["y"]
    if state == "lake":
        b, h = gaussian_state(x, y, seed=5)
    else:  # circular dam on a flat bottom
        b = np.zeros_like(x)
        cx, cy = np.median(x), np.median(y)
        r = 0.3 * (x.max() - x.min())
        h = np.where((x - cx) ** 2 + (y - cy) ** 2 < r * r, 2.0, 1.0)
    Bx, By = bottom_derivs(setup, N, b)
    out = run_ref.run(name, params, mesh_file=mf, inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx,
                                                          "By": By})
    save(name, params, out, {"mesh": "reference meshFiles/CircleInCircle.mesh (curved order 6, 83 reversed faces)",
                             "state": state})


def case_positivity(name="periodic_pp_N3"):
    pr = problems.periodic_bump(NumFlux=0, steps=0)
    pr.params.PositivityPreserving = 1
    pr.params.PosPresTOL = 1e-3
    pr.params.T = 0.01
    q = pr.q0.reshape(pr.K, 3, -1).copy()
    xi = np.tile(np.linspace(-1.0, 1.0, pr.ngl), pr.ngl)
    for e in (3, 77, 150):
        q[e, 0] = 0.01
        q[e, 1] = 0.01 * 5.0 * xi
    out = run_ref.run(name, pr.params, cartesian=(0.0, 2.0, 0.0, 2.0, 16, 16, 1, 1),
                      inject={"q": q.reshape(-1), "b": pr.b, "Bx": pr.Bx, "By": pr.By})
    save(name, pr.params, out, {"mesh": "Cartesian periodic 16x16", "state": "draining shallow elements"})


def case_ssp_walls(name="walls_ssp3_N2"):
    N = 2
    params = host.Params(N=N, CFL=0.3, T=0.05, NumFlux=3, rkOrder=3, rkSSP=1)
    m = host.mesh_cartesian(N, -1.0, 1.0, 0.0, 1.0, 10, 8)
    b, h = gaussian_state(m.x, m.y, seed=9)
    basis = host.Basis.build(N)
    Bx, By = host.bottom_derivatives(m, basis, b)
    out = run_ref.run(name, params, cartesian=(-1.0, 1.0, 0.0, 1.0, 10, 8, 0, 0),
                      inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx, "By": By})
    save(name, params, out, {"mesh": "Cartesian walls 10x8 on [-1,1]x[0,1]", "rk": "SSP-RK3"})



def case_island_pd(name="island_pd_N3"):
    """Lake with an island that rises above the surface (h = 0 on the dry
    top) and a ripple on the water: partial-dry treatment and the
    positivity limiter on, walls."""
    N = 3
    params = host.Params(N=N, CFL=0.3, T=0.01, NumFlux=0, rkOrder=4, rkSSP=0, PositivityPreserving=1,
                         PosPresTOL=1e-3, PartialDryTreatment=1)
    m = host.mesh_cartesian(N, 0.0, 1.0, 0.0, 1.0, 12, 12)
    x, y = m.x, m.y
    b = 1.4 * np.exp(-((x - 0.47) ** 2 + (y - 0.52) ** 2) / 0.18 ** 2)
    wet = np.maximum(0.0, 1.0 - b)
    h = np.where(wet > 0, wet + 0.02 * np.exp(-((x - 0.8) ** 2 + (y - 0.25) ** 2) / 0.1 ** 2), 0.0)
    basis = host.Basis.build(N)
    Bx, By = host.bottom_derivatives(m, basis, b)
    out = run_ref.run(name, params, cartesian=(0.0, 1.0, 0.0, 1.0, 12, 12, 0, 0),
                      inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx, "By": By})
    save(name, params, out, {"mesh": "Cartesian walls 12x12 on [0,1]^2", "state": "island above the surface",
                             "partial_dry": True})



def case_conv_tc1(name="conv_tc1_N3"):
    """The reference's own convergence test (Testcase 1): manufactured
    solution, Dirichlet boundary states from the exact solution, its source
    term; initial state and bathymetry from the reference's set-up."""
    N = 3
    params = host.Params(N=N, CFL=0.4, T=0.1, NumFlux=0, rkOrder=4, rkSSP=0, Testcase=1)
    out = run_ref.run(name, params, cartesian=(0.0, 2.0, 0.0, 2.0, 8, 8, 0, 0))
    save(name, params, out, {"mesh": "Cartesian 8x8 on [0,2]^2, Dirichlet (exact) boundaries",
                             "state": "Testcase 1 manufactured solution"})


def case_shipped_mesh(name, mesh, N, state, T):
    """A run on one of the reference's own meshes (meshFiles/), read by its
    reader: a circular dam break on a flat bottom, or a lake at rest over
    Gaussian bumps with a ripple; plain path, walls."""
    params = host.Params(N=N, CFL=0.4, T=T, NumFlux=0, rkOrder=4, rkSSP=0)
    mf = f"meshFiles/{mesh}"
    setup = run_ref.run(name + "_setup", params, mesh_file=mf)
    x, y = setup["x"], setup["y"]
    if state == "dam":
        b = np.zeros_like(x)
        cx, cy = 0.5 * (x.min() + x.max()), 0.5 * (y.min() + y.max())
        r = 0.25 * (x.max() - x.min())
        h = np.where((x - cx) ** 2 + (y - cy) ** 2 < r * r, 1.5, 1.0)
    else:
        b, h = gaussian_state(x, y, seed=13)
    Bx, By = bottom_derivs(setup, N, b)
    out = run_ref.run(name, params, mesh_file=mf, inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx,
                                                          "By": By})
    save(name, params, out, {"mesh": f"reference meshFiles/{mesh}", "state": state})


def case_analysis(name="walls_analysis_N3"):
    """Arrival times and maximum elevation (okl/Analysis/*): a ripple on a
    lake whose still-water level is 0 (b = -depth), walls.  The reference
    measures both from its h_0, which main.cpp sets only when it reads a
    bottom file (main.cpp:370,515); otherwise the value is whatever the
    stack held, recorded here from the compiled kernel's define (a
    subnormal in the runs seen, i.e. 0 for these results)."""
    import glob
    import re
    N = 3
    params = host.Params(N=N, CFL=0.4, T=0.08, NumFlux=0, rkOrder=4, rkSSP=0, ArrivalTimings=1,
                         maximumElevation=1)
    m = host.mesh_cartesian(N, 0.0, 1.0, 0.0, 1.0, 12, 12)
    x, y = m.x, m.y
    b = -1.0 + 0.3 * np.exp(-((x - 0.6) ** 2 + (y - 0.55) ** 2) / 0.2 ** 2)
    h = -b + 0.01 * np.exp(-((x - 0.25) ** 2 + (y - 0.3) ** 2) / 0.06 ** 2)
    basis = host.Basis.build(N)
    Bx, By = host.bottom_derivatives(m, basis, b)
    out = run_ref.run(name, params, cartesian=(0.0, 1.0, 0.0, 1.0, 12, 12, 0, 0),
                      inject={"q": pack_q(h, n2=(N + 1) ** 2), "b": b, "Bx": Bx, "By": By})
    kc = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "kcache", "*.cpp")), key=os.path.getmtime)
    hz = [re.findall(r"#define h_zero \((.*)\)", open(f).read()) for f in kc
          if "Arrivaltimes" in open(f).read()]
    save(name, params, out, {"mesh": "Cartesian walls 12x12 on [0,1]^2", "state": "ripple, still water at 0",
                             "reference_h_zero": hz[-1][0] if hz and hz[-1] else None})


CASES = {
    "periodic_nf0_N3": lambda: case_periodic(0, "periodic_nf0_N3"),
    "periodic_nf3_N3": lambda: case_periodic(3, "periodic_nf3_N3"),
    "mapped_rot_N4": lambda: case_mapped_rotated(),
    "circle_lake_N3": lambda: case_circle("circle_lake_N3", N=3, T=0.01, state="lake"),
    "circle_dam_av_N3": lambda: case_circle("circle_dam_av_N3", N=3, AV=1, T=0.005, state="dam"),
    "periodic_pp_N3": lambda: case_positivity(),
    "walls_ssp3_N2": lambda: case_ssp_walls(),
    "island_pd_N3": lambda: case_island_pd(),
    "conv_tc1_N3": lambda: case_conv_tc1(),
    "walls_analysis_N3": lambda: case_analysis(),
    "curvedam_N3": lambda: case_shipped_mesh("curvedam_N3", "CurveDamN3.mesh", 3, "dam", 0.05),
    "pxy4_lake_N4": lambda: case_shipped_mesh("pxy4_lake_N4", "PeriodicXandY4.mesh", 4, "lake", 0.05),
}



# ---------------------------------------------------------------------------
# Printed diagnostics of the reference's own driver on a native test case,
# for the drop-in test (the reference's main.cpp linked against the engine).
DROPIN_CASES = {
    # Testcase 20: Cartesian dam break (h = 10 | 5), b = 0, solid walls
    "dropin_tc20_nf0": dict(N=3, T=0.02, NumFlux=0, Testcase=20, cart=(-5.0, 5.0, -5.0, 5.0, 20, 20, 0, 0)),
    "dropin_tc20_nf3_ssp": dict(N=4, T=0.02, NumFlux=3, Testcase=20, rkOrder=3, rkSSP=1,
                                cart=(-5.0, 5.0, -5.0, 5.0, 12, 10, 0, 0)),
    # Testcase 1: manufactured solution; its errors against the exact
    # solution are compared to a relative 1e-6 (sin/cos of two math libraries)
    "dropin_tc1_conv": dict(N=3, T=0.1, NumFlux=0, Testcase=1, cart=(0.0, 2.0, 0.0, 2.0, 8, 8, 0, 0), rtol=1e-6),
    # Testcase 5: dry lake + lake at rest (h = max(0, 0.4 - b)), with the
    # partial-dry treatment and the positivity limiter, solid walls
    "dropin_tc5_pd": dict(N=3, T=0.05, NumFlux=0, Testcase=5, cart=(0.0, 1.0, 0.0, 1.0, 8, 8, 0, 0),
                          PositivityPreserving=1, PosPresTOL=1e-3, PartialDryTreatment=1),
    # the reference's lake-at-rest cases on solid walls: a bump on nine
    # elements of a 20x20 grid (Testcase 2), a smooth bottom (4), no bottom (7)
    "dropin_tc2_wb": dict(N=3, T=0.05, NumFlux=0, Testcase=2, cart=(0.0, 20.0, 0.0, 20.0, 20, 20, 0, 0)),
    "dropin_tc4_wb_nf3": dict(N=4, T=0.05, NumFlux=3, Testcase=4, cart=(0.0, 6.0, 0.0, 6.0, 8, 8, 0, 0)),
    "dropin_tc7_ssp": dict(N=2, T=0.05, NumFlux=0, Testcase=7, rkOrder=3, rkSSP=1,
                           cart=(0.0, 1.0, 0.0, 1.0, 6, 6, 0, 0)),
    # dam break with the shock sensor and artificial viscosity (its log10 / sin
    # come from different math libraries: relative 1e-9)
    "dropin_tc20_av": dict(N=3, T=0.02, NumFlux=0, Testcase=20, cart=(-5.0, 5.0, -5.0, 5.0, 16, 16, 0, 0),
                           ArtificialViscosity=1, epsilon_0=0.5, sigma_min=-6.0, sigma_max=-2.0, rtol=1e-9,
                           atol=1e-10),
}


def dropin_params(spec):
    p = host.Params(N=spec["N"], CFL=0.4, T=spec["T"], NumFlux=spec["NumFlux"], Testcase=spec["Testcase"],
                    rkOrder=spec.get("rkOrder", 4), rkSSP=spec.get("rkSSP", 0),
                    PositivityPreserving=spec.get("PositivityPreserving", 0),
                    PosPresTOL=spec.get("PosPresTOL", 1e-4), PartialDryTreatment=spec.get("PartialDryTreatment", 0),
                    ArtificialViscosity=spec.get("ArtificialViscosity", 0), epsilon_0=spec.get("epsilon_0", 0.1),
                    sigma_min=spec.get("sigma_min", -16.0), sigma_max=spec.get("sigma_max", -12.0))
    return p


def diag_lines(stdout):
    keys = ("Entropydifference is", "relative Entropydifference", "Mass difference is", "relative mass difference",
            "L2Error[", "LinfError[")
    return [ln.strip() for ln in stdout.splitlines() if ln.strip().startswith(keys)]


def make_dropin(name):
    spec = DROPIN_CASES[name]
    p = dropin_params(spec)
    out = run_ref.run(name, p, cartesian=spec["cart"])
    rec = {"spec": spec, "params": {k: getattr(p, k) for k in vars(p)}, "diagnostics": diag_lines(out["stdout"]),
           "input_dat": open(os.path.join(ROOT, "oracle", "_ref", "runs", name, "input.dat")).read(),
           "cartesian_dat": open(os.path.join(ROOT, "oracle", "_ref", "runs", name, "Cartesian.dat")).read()}
    with open(os.path.join(OUT, f"{name}.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(name, rec["diagnostics"])


for _n in DROPIN_CASES:
    CASES[_n] = (lambda n: (lambda: make_dropin(n)))(_n)


# The time loop's outputs (src/deviceclass.cpp:797-838, 1143-1309 and
# src/Plots.cpp): plot checkpoints with the solution (PlotVar 1), total
# entropy and mass over time (EntropyPlot), written by the reference program
# into movie/; the drop-in driver must write the same files.
DROPIN_OUTPUT_CASES = {
    "dropin_outputs_tc20": dict(N=2, T=0.03, NumFlux=0, Testcase=20, cart=(-5.0, 5.0, -5.0, 5.0, 6, 6, 0, 0),
                                NumPlots=4, EntropyPlot=1, PlotVar=1),
}


def make_dropin_outputs(name):
    import shutil
    import subprocess
    spec = DROPIN_OUTPUT_CASES[name]
    p = dropin_params(spec)
    rd = os.path.join(ROOT, "oracle", "_ref", "runs", name)
    if os.path.isdir(rd):
        shutil.rmtree(rd)
    os.makedirs(os.path.join(rd, "movie"))
    for d in ("okl", "meshFiles", "data"):
        os.symlink(os.path.join(run_ref.REF, d), os.path.join(rd, d))
    run_ref.write_input(os.path.join(rd, "input.dat"), p, "none", 1)
    run_ref.write_cartesian(os.path.join(rd, "Cartesian.dat"), *spec["cart"])
    txt = open(os.path.join(rd, "input.dat")).read()
    for k in ("NumPlots", "EntropyPlot", "PlotVar"):
        txt = txt.replace(f"{k}={'2' if k == 'PlotVar' else '0'}\n", f"{k}={spec[k]}\n")
    open(os.path.join(rd, "input.dat"), "w").write(txt)
    env = dict(os.environ, ESDG_REF_KCACHE=os.path.join(ROOT, "oracle", "_ref", "kcache"))
    out = subprocess.run(["bash", "-c", f"ulimit -s unlimited; exec {run_ref.EXE} Serial"], cwd=rd, env=env,
                         capture_output=True, text=True, timeout=600, check=True)
    files = {f: open(os.path.join(rd, "movie", f)).read() for f in sorted(os.listdir(os.path.join(rd, "movie")))}
    rec = {"spec": spec, "input_dat": txt, "cartesian_dat": open(os.path.join(rd, "Cartesian.dat")).read(),
           "diagnostics": diag_lines(out.stdout), "movie": files}
    with open(os.path.join(OUT, f"{name}.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(name, sorted(files))


for _n in DROPIN_OUTPUT_CASES:
    CASES[_n] = (lambda n: (lambda: make_dropin_outputs(n)))(_n)


# ---------------------------------------------------------------------------
# The reference's Okada routine (src/okada.cpp) on a lon/lat grid around the
# epicentre of its shipped fault file data/indianOceanFault1.txt.
def make_okada(name="okada_fault1"):
    import subprocess
    import tempfile
    R = 6.378e6
    lon = np.linspace(94.57 - 2.5, 94.57 + 2.5, 121)
    lat = np.linspace(3.83 - 1.5, 3.83 + 1.5, 73)
    LO, LA = np.meshgrid(lon, lat)
    x = (LO * R * np.pi / 180 / 1000).ravel()
    y = (R * np.arcsinh(np.tan(LA * np.pi / 180)) / 1000).ravel()
    d = tempfile.mkdtemp()
    os.symlink(os.path.join(run_ref.REF, "data"), os.path.join(d, "data"))
    np.concatenate([[x.size], x, y]).astype(np.float64).tofile(os.path.join(d, "pts.bin"))
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "okada_driver"), "pts.bin", "out.bin"], cwd=d, check=True)
    uplift = np.fromfile(os.path.join(d, "out.bin"))
    fault = [float(v) for v in open(os.path.join(run_ref.REF, "data", "indianOceanFault1.txt")).read().split()]
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), x_km=x, y_km=y, uplift_km=uplift, fault=np.array(fault))
    print(name, "points", x.size, "nonzero", int((uplift != 0).sum()))


CASES["okada_fault1"] = make_okada

if __name__ == "__main__":
    if not run_ref.available():
        sys.exit("the reference tree is not available here")
    run_ref.build()
    for c in (sys.argv[1:] or list(CASES)):
        CASES[c]()
