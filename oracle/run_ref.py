"""ORACLE test infrastructure: run the reference program (oracle/_ref/esdg_ref,
built by oracle/build_ref.sh from the reference's own sources) on a chosen
problem and collect what it hands to its device layer and what it returns.

The reference reads input.dat / Cartesian.dat / .okl files relative to its
working directory; each run gets a fresh directory under oracle/_ref/runs/
with those files and links to the reference's okl/ and meshFiles/.  The
OCCA shim's ESDG_REF_INJECT hook replaces the testcase's initial state and
bathymetry by the problem's (copyDeviceVariables arguments 7-9 and 16), its
ESDG_REF_DUMP hook records every copyDeviceVariables argument and the final
o_q.copyTo(q) of main.cpp:1051.

`run` generates and checks fixtures and needs the reference tree.
`run_timed` runs the program once without dumps and returns its own timing
of DGtimeloop; it also runs where the reference tree is absent, as long as
every kernel the run needs was built before (`warm_kernels` builds them, the
shim finds them in _ref/kcache by its index).
"""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference source tree: $ESDG_REFERENCE, else a checkout named
# `reference` beside this repository.
REF = os.environ.get("ESDG_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
EXE = os.path.join(HERE, "_ref", "esdg_ref")

# copyDeviceVariables argument order (src/deviceclass.cpp:576-626) as seen by
# the shim's copyFrom sequence numbers; GLw is copied only when PP=1.
SEQ_BEFORE_GLW = ["nx", "ny", "scal", "y_xi", "y_eta", "x_xi", "x_eta", "b", "Bx", "By", "D", "Dstrong", "Dhat",
                  "Jinv", "x", "y", "q", "EleSizes", "gRK", "Qt", "VdmInv"]
SEQ_AFTER_GLW = ["MasterSlave", "Orientation", "ElemToEdge", "EdgeData", "EdgeReversed"]
INT_ARRAYS = set(SEQ_AFTER_GLW)

INPUT_KEYS = ["meshFile", "N", "CFL", "DFL", "T", "g_const", "ArtificialViscosity", "PositivityPreserving",
              "PosPresTOL", "epsilon_0", "sigma_min", "sigma_max", "PlotVar", "EntropyPlot", "NumPlots",
              "NumTimeChecks", "Testcase", "ES", "NumFlux", "FluxDifferencing", "Cartesian", "rkOrder", "rkSSP",
              "NEpad", "NEsurfpad", "Nedgepad", "NavgPad", "KernelVersionFD", "KernelVersionSTD", "DiscBottom",
              "ReadInBottom", "PartialDryTreatment", "FrictionTerms", "ConvertToKM", "ArrivalTimings",
              "createTimeSeries", "maximumElevation"]


def available() -> bool:
    return os.path.isdir(os.path.join(REF, "okl")) and os.path.exists(os.path.join(REF, "main.cpp"))


def build():
    subprocess.run(["sh", os.path.join(HERE, "build_ref.sh")], check=True, stdout=subprocess.DEVNULL)
    return EXE


def seq_names(pp: int, pd: int = 0, at: int = 0, me: int = 0):
    # initDeviceVariables first fills the arrival-time and maximum-elevation
    # buffers (src/deviceclass.cpp:324-341); copyPartialDryData
    # (main.cpp:938-941) follows copyDeviceVariables
    return ((["ArrivalTimings0"] if at else []) + (["MaximumElevation0"] if me else []) + SEQ_BEFORE_GLW +
            (["GLw"] if pp else []) + SEQ_AFTER_GLW + (["DcFD", "DfFD", "DbFD"] if pd else []))


def write_input(path, params, mesh_file="none", cartesian=1):
    vals = {"meshFile": mesh_file, "N": params.N, "CFL": repr(params.CFL), "DFL": repr(params.DFL),
            "T": repr(params.T), "g_const": repr(params.g_const), "ArtificialViscosity": params.ArtificialViscosity,
            "PositivityPreserving": params.PositivityPreserving, "PosPresTOL": repr(params.PosPresTOL),
            "epsilon_0": repr(params.epsilon_0), "sigma_min": repr(params.sigma_min),
            "sigma_max": repr(params.sigma_max), "PlotVar": 2, "EntropyPlot": 0, "NumPlots": 0, "NumTimeChecks": 0,
            "Testcase": params.Testcase, "ES": params.ES, "NumFlux": params.NumFlux,
            "FluxDifferencing": params.FluxDifferencing, "Cartesian": cartesian, "rkOrder": params.rkOrder,
            "rkSSP": params.rkSSP, "NEpad": params.NEpad, "NEsurfpad": params.NEsurfpad, "Nedgepad": params.Nedgepad,
            "NavgPad": params.NavgPad, "KernelVersionFD": 99, "KernelVersionSTD": 99, "DiscBottom": 0,
            "ReadInBottom": 0, "PartialDryTreatment": 0, "FrictionTerms": 0, "ConvertToKM": 0, "ArrivalTimings": 0,
            "createTimeSeries": 0, "maximumElevation": 0}
    for k in ("PartialDryTreatment", "ArrivalTimings", "maximumElevation"):
        vals[k] = int(getattr(params, k, 0))
    with open(path, "w") as f:
        for k in INPUT_KEYS:
            f.write(f"{k}={vals[k]}\n")


def write_cartesian(path, xL, xR, yL, yR, NX, NY, per_rows, per_cols):
    with open(path, "w") as f:
        for k, v in (("xL", repr(xL)), ("xR", repr(xR)), ("yL", repr(yL)), ("yR", repr(yR)), ("NelemX", NX),
                     ("NelemY", NY), ("PeriodicBD_X", int(per_rows)), ("PeriodicBD_Y", int(per_cols))):
            f.write(f"{k}={v}\n")


def run(tag, params, cartesian=None, mesh_file=None, inject=None, mode="Serial", threads=None, timeout=3600):
    """Runs the reference once.  cartesian=(xL,xR,yL,yR,NX,NY,per_rows,per_cols)
    or mesh_file (path relative to the reference tree).  inject: dict with
    any of q, b, Bx, By (arrays in the reference layout).  Returns a dict of
    the copyDeviceVariables arrays (as dumped), 'q_final', the stdout text and
    the wall time of the run."""
    if not os.path.exists(EXE):
        build()
    rd = os.path.join(HERE, "_ref", "runs", tag)
    if os.path.isdir(rd):
        shutil.rmtree(rd)
    os.makedirs(os.path.join(rd, "dump"))
    os.makedirs(os.path.join(rd, "inject"))
    for d in ("okl", "meshFiles", "data"):
        os.symlink(os.path.join(REF, d), os.path.join(rd, d))
    if cartesian is not None:
        write_input(os.path.join(rd, "input.dat"), params, "none", 1)
        write_cartesian(os.path.join(rd, "Cartesian.dat"), *cartesian)
    else:
        write_input(os.path.join(rd, "input.dat"), params, mesh_file, 0)
    names = seq_names(params.PositivityPreserving, int(getattr(params, "PartialDryTreatment", 0)),
                      int(getattr(params, "ArrivalTimings", 0)), int(getattr(params, "maximumElevation", 0)))
    for k, v in (inject or {}).items():
        np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(rd, "inject", f"from_{names.index(k):03d}.bin"))
    env = dict(os.environ)
    env["ESDG_REF_DUMP"] = os.path.join(rd, "dump")
    env["ESDG_REF_INJECT"] = os.path.join(rd, "inject")
    env["ESDG_REF_KCACHE"] = os.path.join(HERE, "_ref", "kcache")
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    import time
    t0 = time.perf_counter()
    p = subprocess.run(["bash", "-c", f"ulimit -s unlimited; exec {EXE} {mode}"], cwd=rd, env=env,
                       capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"reference run failed ({p.returncode}):\n{p.stdout[-3000:]}\n{p.stderr[-3000:]}")
    out = {"stdout": p.stdout, "wall": wall}
    mem_of_seq = {}
    with open(os.path.join(rd, "dump", "manifest.txt")) as f:
        for line in f:
            w = line.split()
            if w[0] == "from":
                mem_of_seq[int(w[1])] = int(w[3])
    for i, nm in enumerate(names):
        fn = os.path.join(rd, "dump", f"from_{i:03d}.bin")
        out[nm] = np.fromfile(fn, dtype=np.int32 if nm in INT_ARRAYS else np.float64)
    qmem = mem_of_seq[names.index("q")]
    out["q_final"] = np.fromfile(os.path.join(rd, "dump", f"to_{qmem:03d}.bin"), dtype=np.float64)
    # the analysis buffers as DGtimeloop reads them back at its end
    # (src/deviceclass.cpp:1296-1309)
    for nm in ("ArrivalTimings", "MaximumElevation"):
        if nm + "0" in names:
            mem = mem_of_seq[names.index(nm + "0")]
            out[nm] = np.fromfile(os.path.join(rd, "dump", f"to_{mem:03d}.bin"), dtype=np.float64)
    return out


def _prepare(rd, params, mesh_file, inject, cartesian=None):
    if cartesian is not None:
        write_input(os.path.join(rd, "input.dat"), params, "none", 1)
        write_cartesian(os.path.join(rd, "Cartesian.dat"), *cartesian)
    else:
        write_input(os.path.join(rd, "input.dat"), params, mesh_file, 0)
    names = seq_names(params.PositivityPreserving, int(getattr(params, "PartialDryTreatment", 0)),
                      int(getattr(params, "ArrivalTimings", 0)), int(getattr(params, "maximumElevation", 0)))
    os.makedirs(os.path.join(rd, "inject"), exist_ok=True)
    for k, v in (inject or {}).items():
        np.ascontiguousarray(v, dtype=np.float64).tofile(os.path.join(rd, "inject", f"from_{names.index(k):03d}.bin"))
    if available():
        for d in ("okl", "meshFiles", "data"):
            os.symlink(os.path.join(REF, d), os.path.join(rd, d))


def run_timed(params, mesh_file, inject=None, threads=None, mode="OpenMP", timeout=900, want_q=False,
              extra_env=None):
    """One run of the reference program on an absolute mesh path, state and
    bathymetry injected as in `run` (extra_env: further environment, e.g.
    ESDG_REF_CASE for the case hook of oracle/ref_shim/bench_case.cpp).  Returns (seconds, stdout, q_final):
    the time its own timer reports around DGtimeloop (main.cpp:1009-1072,
    printed as "time taken in seconds"), and with want_q the final state
    (o_q.copyTo at main.cpp:1051, through the dump hook; None otherwise)."""
    import re
    import tempfile
    if not os.path.exists(EXE):
        raise FileNotFoundError(f"reference program not built: {EXE}")
    rd = tempfile.mkdtemp(prefix="esdg_ref_")
    q_final = None
    try:
        _prepare(rd, params, mesh_file, inject)
        env = dict(os.environ)
        env.pop("ESDG_REF_DUMP", None)
        if want_q:
            os.makedirs(os.path.join(rd, "dump"))
            env["ESDG_REF_DUMP"] = os.path.join(rd, "dump")
        env["ESDG_REF_INJECT"] = os.path.join(rd, "inject")
        env["ESDG_REF_KCACHE"] = os.path.join(HERE, "_ref", "kcache")
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        env.update(extra_env or {})
        p = subprocess.run(["bash", "-c", f"ulimit -s unlimited; exec {EXE} {mode}"], cwd=rd, env=env,
                           capture_output=True, text=True, timeout=timeout)
        if want_q and p.returncode == 0:
            names = seq_names(params.PositivityPreserving, int(getattr(params, "PartialDryTreatment", 0)),
                              int(getattr(params, "ArrivalTimings", 0)), int(getattr(params, "maximumElevation", 0)))
            with open(os.path.join(rd, "dump", "manifest.txt")) as f:
                mem = {int(w[1]): int(w[3]) for w in (ln.split() for ln in f) if w[0] == "from"}
            q_final = np.fromfile(os.path.join(rd, "dump", f"to_{mem[names.index('q')]:03d}.bin"), dtype=np.float64)
    finally:
        shutil.rmtree(rd, ignore_errors=True)
    m = re.search(r"time taken in seconds = ([0-9.eE+-]+)", p.stdout)
    if p.returncode != 0 or not m:
        raise RuntimeError(f"reference run failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    return float(m.group(1)), p.stdout, q_final


def warm_kernels(params, mesh_file, mode="OpenMP"):
    """Builds (here, from the reference tree) every kernel a run with these
    parameters loads, so that `run_timed` with the same parameters needs no
    .okl sources.  The kernels depend on the parameters, not on the mesh:
    a small mesh does."""
    if not available():
        return False
    if not os.path.exists(EXE):
        build()
    run_timed(params, mesh_file, None, threads=2, mode=mode, timeout=600)
    return True


def kernel_calls(stdout):
    """Kernel call counts the OCCA stand-in prints at exit with ESDG_REF_COUNT=1."""
    import re
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"\[occa shim\] calls (\S+) (\d+)", stdout)}
