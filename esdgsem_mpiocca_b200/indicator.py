"""Learned troubled-cell indicator: parameters, device training and
inference through the engine's MLP kernels (libesdg_b200.so,
esdg_mlp_* entry points).  No counterpart in the reference.

The network maps an element's features (normalised nodal h+b, hu, hv and
their log energy fractions) to the modal shock sensor's
sigma = log10(energy ratio) (okl/ShockCapturing/ShockCapturing.okl:131-204):
sigma_hat = y + s_eta.  In the solver it replaces the sensor only where it
is confident: sigma_hat below sigma_min - margin (no viscosity) or above
sigma_max + margin (full viscosity); every other element, every element
failing the positivity check and every element near the sensor's absolute
energy threshold gets the modal sensor itself.

PyTorch is used here only to hold device buffers and order work on its
current stream; every computation is one of the library's kernels.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass, field

import numpy as np

H = 32
S_MIN = -12.0
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


def _lib():
    from . import lib
    return lib()


def layout(ngl: int) -> dict:
    out = (ctypes.c_int * 8)()
    rc = _lib().esdg_mlp_layout(ngl, out)
    if rc != 0:
        raise ValueError(f"no indicator layout for ngl={ngl}")
    return dict(zip(("kp", "w1", "b1", "w2", "b2", "w3", "b3", "total"), list(out)))


def nin(ngl: int) -> int:
    return 3 * ngl * ngl + 3


def init_params(ngl: int, seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases; padding columns of W1 stay zero."""
    rng = np.random.default_rng(seed)
    L = layout(ngl)
    P = np.zeros(L["total"], dtype=np.float32)
    W1 = np.zeros((H, L["kp"]), dtype=np.float32)
    a1 = np.sqrt(6.0 / nin(ngl))
    W1[:, :nin(ngl)] = rng.uniform(-a1, a1, size=(H, nin(ngl)))
    P[L["w1"]:L["b1"]] = W1.ravel()
    P[L["w2"]:L["b2"]] = rng.uniform(-np.sqrt(6.0 / H), np.sqrt(6.0 / H), size=H * H)
    P[L["w3"]:L["b3"]] = rng.uniform(-np.sqrt(3.0 / H), np.sqrt(3.0 / H), size=H)
    return P


def energy_bounds(VdmInv: np.ndarray) -> tuple[float, float]:
    """Smallest and largest ratio n1 / sum(m^2) of the sensor's modal energy
    n1 = |V m V^T|_F^2 to the nodal energy, for V = VdmInv (products of the
    extreme eigenvalues of V^T V)."""
    V = np.asarray(VdmInv, dtype=np.float64)
    n = int(round(np.sqrt(V.size)))
    ev = np.linalg.eigvalsh(V.reshape(n, n).T @ V.reshape(n, n))
    return float(ev.min() ** 2), float(ev.max() ** 2)


@dataclass
class IndicatorNet:
    """Parameters of one trained network (one polynomial degree)."""
    ngl: int
    P: np.ndarray
    margin: float = 0.5
    meta: dict = field(default_factory=dict)

    @classmethod
    def fresh(cls, ngl: int, seed: int = 0) -> "IndicatorNet":
        return cls(ngl, init_params(ngl, seed))

    @classmethod
    def load(cls, path: str) -> "IndicatorNet":
        z = np.load(path)
        meta = json.loads(bytes(z["meta"]).decode())
        return cls(int(z["ngl"]), z["P"].astype(np.float32), float(z["margin"]), meta)

    @classmethod
    def default(cls, N: int) -> "IndicatorNet":
        """The committed network for polynomial degree N (N = 3 or 4)."""
        return cls.load(os.path.join(WEIGHTS_DIR, f"indicator_N{N}.npz"))

    def save(self, path: str):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, P=self.P.astype(np.float32), ngl=np.int32(self.ngl), margin=np.float64(self.margin),
                 meta=np.frombuffer(json.dumps(self.meta).encode(), dtype=np.uint8))


class DeviceMLP:
    """FP32 master weights, BF16 copy and Adam moments on the GPU; training
    and inference calls on torch's current stream of `device`."""

    def __init__(self, net: IndicatorNet, device: int = 0, blocks: int = 296):
        import torch
        self.torch = torch
        self.net = net
        self.ngl = net.ngl
        self.L = layout(net.ngl)
        self.dev = torch.device("cuda", device)
        self.P = torch.tensor(net.P, dtype=torch.float32, device=self.dev)
        self.Pb = torch.empty(self.L["total"], dtype=torch.bfloat16, device=self.dev)
        self.m = torch.zeros_like(self.P)
        self.v = torch.zeros_like(self.P)
        self.G = torch.zeros_like(self.P)
        self.blocks = blocks
        self.partial = torch.zeros(blocks * 4 * self.L["total"], dtype=torch.float32, device=self.dev)
        self.step_count = 0
        self._ok(_lib().esdg_mlp_cast(self.ngl, self._p(self.P), self._p(self.Pb), self._s()))

    # -- helpers --
    def _s(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    @staticmethod
    def _ok(rc):
        if rc != 0:
            msg = _lib().esdg_last_error(None)
            raise RuntimeError(f"indicator kernel failed ({rc}): {msg.decode() if msg else ''}")

    # -- kernels --
    def features(self, q_ptr: int, b_ptr: int, V_ptr: int, K: int, target: bool = True, ZeroTOL: float = 1e-5):
        """X [K][kp] (bf16), target t [K] or None, s_eta [K] from device
        arrays q [K][3][ngl^2], b [K][ngl^2], VdmInv."""
        torch = self.torch
        X = torch.empty((K, self.L["kp"]), dtype=torch.bfloat16, device=self.dev)
        t = torch.empty(K, dtype=torch.float32, device=self.dev) if target else None
        s = torch.empty(K, dtype=torch.float32, device=self.dev)
        self._ok(_lib().esdg_mlp_features(self.ngl, K, ctypes.c_void_p(q_ptr), ctypes.c_void_p(b_ptr),
                                          ctypes.c_void_p(V_ptr), ZeroTOL, self._p(X), self._p(t), self._p(s),
                                          self._s()))
        return X, t, s

    def forward(self, X):
        y = self.torch.empty(X.shape[0], dtype=self.torch.float32, device=self.dev)
        self._ok(_lib().esdg_mlp_forward(self.ngl, X.shape[0], self._p(X), self._p(self.P), self._p(self.Pb),
                                         self._p(y), self.blocks, self._s()))
        return y

    def gradient(self, X, t):
        """Loss gradient G (device, float32) and the summed squared error
        (device scalar) without updating the weights."""
        self._ok(_lib().esdg_mlp_backward(self.ngl, X.shape[0], self._p(X), self._p(t), self._p(self.P),
                                          self._p(self.Pb), self._p(self.partial), self.blocks, self._s()))
        rows = self.partial.view(self.blocks * 4, self.L["total"])
        return rows.sum(0), rows[:, self.L["b3"] + 1].sum()

    def train_step(self, X, t, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam step on the minibatch; returns the device scalar sum of
        squared errors (before the step)."""
        self.step_count += 1
        self._ok(_lib().esdg_mlp_backward(self.ngl, X.shape[0], self._p(X), self._p(t), self._p(self.P),
                                          self._p(self.Pb), self._p(self.partial), self.blocks, self._s()))
        self._ok(_lib().esdg_mlp_adam(self.ngl, self.blocks * 4, self._p(self.partial), self._p(self.G),
                                      self._p(self.P), self._p(self.Pb), self._p(self.m), self._p(self.v),
                                      lr, beta1, beta2, eps, self.step_count, self._s()))
        return self.G[self.L["b3"] + 1]

    def to_net(self, **meta) -> IndicatorNet:
        net = IndicatorNet(self.ngl, self.P.detach().cpu().numpy().astype(np.float32), self.net.margin,
                           dict(self.net.meta, **meta))
        return net
