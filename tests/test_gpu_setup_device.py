"""Set-up computed on the device against the host set-up (GPU).

* Geometry (esdg_geometry_device): the transfinite map of the element
  curves, collocation metric terms, Jacobian and side normals must equal the
  host set-up's arrays (which reproduce the reference's own set-up bit for
  bit, tests/test_golden_cpu.py) bit for bit -- on mapped meshes with
  rotated corner numbering at N = 3 and 4, and on an ISM-V2 file read back
  whose elements mix curved, straight and partly straight sides (the
  transfinite and the bilinear branches).
* Okada uplift (esdg_okada_uplift): the same dislocation formulas in CUDA
  against the host restatement on the tsunami members' meshes (Cartesian
  geometry) and against the reference routine's own output on its shipped
  fault (Mercator geometry, tests/golden/okada_fault1.npz); the math
  library differs (CUDA vs glibc/NumPy log, atan, sqrt), so within 1e-12 of
  the largest uplift.
"""
import ctypes
import os

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import geometry, host, lib, okada, problems
from oracle import ref_inputs

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _compare(N, mesh, make):
    import torch
    torch.cuda.set_device(0)
    m, corners, curved, curves = geometry.element_curves(make, N)
    g = {k: v.cpu().numpy() for k, v in geometry.device_geometry(N, m, corners, curved, curves).items()}
    torch.cuda.synchronize()
    for k in ("x", "y", "x_xi", "x_eta", "y_xi", "y_eta"):
        np.testing.assert_array_equal(g[k], getattr(mesh, k), err_msg=k)
    np.testing.assert_array_equal(1.0 / g["J"], mesh.Jinv)
    for k, side in (("nx", "nx_side"), ("ny", "ny_side"), ("scal", "scal_side")):
        np.testing.assert_array_equal(geometry.face_normals(g[side], mesh.EdgeData, N), getattr(mesh, k), err_msg=k)


@pytest.mark.parametrize("N,nel,rot", [(3, 12, 7), (4, 10, 5), (4, 9, 0)])
def test_device_geometry_matches_host_mapped(N, nel, rot):
    mesh = host.mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, nel, nel, amp=0.03, rotate_seed=rot)
    _compare(N, mesh, lambda out: lib().esdg_mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, nel, nel, 0.03, max(N, 4), rot, out))


def _write_mixed(path, nel, m=4):
    """The mapped mesh as ISM-V2 with every third element's sides straight
    and the bottom side of every fifth element straight."""
    M = ref_inputs.mapped_mesh(nel, m=m)
    K, F, corners, edges, curves = M["K"], M["F"], M["corners"], M["edges"], M["curves"]
    with open(path, "w") as f:
        f.write("ISM-V2\n%d %d %d %d\n" % (len(M["nodes_x"]), F, K, m))
        for x, y in zip(M["nodes_x"].tolist(), M["nodes_y"].tolist()):
            f.write("%.17g %.17g\n" % (x, y))
        for r in edges.tolist():
            sr = 0 if r[3] < 0 else (r[5] + 1 if r[6] == 1 else -(r[5] + 1))
            f.write("%d %d %d %d %d %d\n" % (r[0] + 1, r[1] + 1, r[2] + 1, r[3] + 1, r[4] + 1, sr))
        for e in range(K):
            flags = [0, 0, 0, 0] if e % 3 == 0 else ([0, 1, 1, 1] if e % 5 == 0 else [1, 1, 1, 1])
            c = corners[e]
            f.write("%d %d %d %d\n" % (c[0] + 1, c[1] + 1, c[2] + 1, c[3] + 1))
            f.write("%d %d %d %d\n" % tuple(flags))
            for s in range(4):
                if flags[s]:
                    for k in range(m + 1):
                        f.write("%.17g %.17g\n" % (curves[e, s, k, 0], curves[e, s, k, 1]))
            f.write("wall wall wall wall\n")


@pytest.mark.parametrize("N", [3, 4])
def test_device_geometry_matches_host_read_mixed_sides(tmp_path, N):
    path = str(tmp_path / "mixed.mesh")
    _write_mixed(path, 8)
    mesh = host.mesh_read(N, path)
    _compare(N, mesh, lambda out: lib().esdg_mesh_read_ism2(N, path.encode(), 0, 0, out))


@pytest.mark.parametrize("seed", [0, 3, 17, 40])
def test_device_okada_matches_host_cartesian(seed):
    import torch
    torch.cuda.set_device(0)
    pr = problems.tsunami_member(seed, sizes=(64,), steps=0)
    f = okada.Fault(**pr.meta["fault"])
    x, y = pr.mesh.x, pr.mesh.y
    ref = okada.uplift_cartesian(x, y, f)
    got = okada.uplift_device(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), f).cpu().numpy()
    assert np.abs(ref).max() > 0
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    # add mode: on top of a given field
    base = torch.full((x.size,), 2.5, dtype=torch.float64, device="cuda")
    okada.uplift_device(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), f, out=base, add=True)
    assert np.abs(base.cpu().numpy() - 2.5 - ref).max() <= 1e-12 * np.abs(ref).max()


def test_device_okada_matches_reference_routine():
    import torch
    torch.cuda.set_device(0)
    z = np.load(os.path.join(GOLDEN, "okada_fault1.npz"))
    lon, lat, depth, length, width, strike, rake, dip, slip = z["fault"][:9]
    f = okada.Fault(lon, lat, depth, length, width, strike, rake, dip, slip)
    got = okada.uplift_device(torch.from_numpy(z["x_km"]).cuda(), torch.from_numpy(z["y_km"]).cuda(), f,
                              mercator=True).cpu().numpy()
    ref = z["uplift_km"]
    assert np.abs(ref).max() > 0
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
