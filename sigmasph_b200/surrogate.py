"""The Johnson-Cook return-map surrogate: sample collection from the plain solver,
training and inference on the GPU through libsph_b200's sph_mlp_* kernels.

There is no counterpart in the reference, whose Johnson-Cook return is an exact
bracketed Newton-bisection (MAT002_johnson_cook.py:251-354, called from
SOLID.py:2889-2913).  The network (4 -> 64 -> 64 -> 64 -> 1, SiLU) maps the features of a
yielding return to u = 10 (1 - d / d_hi), the hardening share of the overstress, from
which the plastic increment d follows (d_hi is the increment's upper bracket); in the
solver it only proposes: the exact residual decides, and the Newton runs wherever the
proposal misses the yield surface by more than `tol` (|g| / sigma_y).

    sur = JCSurrogate()
    X, T = collect_returns(scene, steps=..., capacity=...)   # plain solver, exact returns
    sur.fit(X, T)                                             # T = exact d / d_hi
    solver.enable_jc_surrogate(sur, tol=1e-3)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from .config import SimConfig
from .particle_system import ParticleSystem

FEATURES = ("vm / sigma_y0 - 1", "eps_p", "ln(max(eps_dot_eq / eps0_dot, 1)) / 10",
            "ln(max(d_hi / (dt eps0_dot), 1)) / 10")
LOG_COLUMNS = FEATURES + ("d / d_hi", "d_hi", "vm", "sigma_y0")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class JCSurrogate:
    """Float32 master parameters on the GPU; BF16 tensor-core inference."""

    def __init__(self, weights=None, device="cuda", seed=20260101):
        self.L = abi.lib()
        self.n_params = self.L.sph_mlp_param_count()
        self.device = torch.device(device)
        if weights is None:
            g = torch.Generator().manual_seed(seed)
            w = torch.zeros(self.n_params, dtype=torch.float32)
            h, o = 64, 0
            for fan_in, fan_out in ((4, h), (h, h), (h, h)):
                w[o:o + fan_in * fan_out] = torch.randn(fan_in * fan_out, generator=g) * (2.0 / fan_in) ** 0.5
                o += fan_in * fan_out + fan_out
            w[o:o + h] = torch.randn(h, generator=g) * (1.0 / h) ** 0.5
            w[o + h] = 1.0          # u is O(1)
            weights = w
        self.W = torch.as_tensor(weights, dtype=torch.float32).to(self.device).contiguous()
        if self.W.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {self.W.numel()}")
        self.packed = torch.empty(int(self.L.sph_mlp_packed_bytes()), dtype=torch.uint8,
                                  device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)

    # ------------------------------------------------------------------ inference
    def _rows(self, X):
        X = torch.as_tensor(X, dtype=torch.float32, device=self.device).reshape(-1, 4).contiguous()
        return X, torch.empty(X.shape[0], dtype=torch.float32, device=self.device)

    def predict_f32(self, X):
        """Float32 forward on CUDA cores (the training reference)."""
        X, Y = self._rows(X)
        abi.check(self.L.sph_mlp_forward(_ptr(self.W), _ptr(X), X.shape[0], _ptr(Y), _stream()),
                  "sph_mlp_forward")
        return Y

    @staticmethod
    def target(fraction):
        """The network's output for a plastic increment d = fraction * d_hi."""
        return 10.0 * (1.0 - fraction)

    def predict_fraction(self, X):
        """d / d_hi from the tensor-core forward."""
        return 1.0 - 0.1 * self.predict(X)

    def predict(self, X):
        """BF16 tensor-core forward with FP32 accumulation (what the solver runs)."""
        X, Y = self._rows(X)
        abi.check(self.L.sph_mlp_pack(_ptr(self.W), _ptr(self.packed), _stream()), "sph_mlp_pack")
        self.err.zero_()
        abi.check(self.L.sph_mlp_infer_tc(_ptr(self.W), _ptr(self.packed), _ptr(X), X.shape[0],
                                          _ptr(Y), _ptr(self.err), _stream()), "sph_mlp_infer_tc")
        if int(self.err.item()) != 0:
            raise RuntimeError("tensor-core surrogate pass timed out waiting for its MMAs")
        return Y

    # ------------------------------------------------------------------ training
    def loss_and_grad(self, X, T):
        X = torch.as_tensor(X, dtype=torch.float32, device=self.device).reshape(-1, 4).contiguous()
        T = torch.as_tensor(T, dtype=torch.float32, device=self.device).reshape(-1).contiguous()
        G = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        abi.check(self.L.sph_mlp_grad(_ptr(self.W), _ptr(X), _ptr(T), X.shape[0], _ptr(G),
                                      _ptr(loss), _stream()), "sph_mlp_grad")
        return loss, G

    def fit(self, X, F, steps=3000, batch=8192, lr=2e-3, lr_final=1e-4, seed=7, log_every=0):
        """Adam on minibatches of (X, target(F)) -- F the exact d / d_hi of each return --
        with a cosine-decayed rate; returns the loss history (one value per `log_every`
        steps, or the last loss)."""
        X = torch.as_tensor(X, dtype=torch.float32, device=self.device).reshape(-1, 4).contiguous()
        F = torch.as_tensor(F, dtype=torch.float32, device=self.device).reshape(-1)
        T = self.target(F).contiguous()
        n = X.shape[0]
        M = torch.zeros_like(self.W)
        V = torch.zeros_like(self.W)
        G = torch.empty_like(self.W)
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        gen = torch.Generator(device=self.device).manual_seed(seed)
        hist = []
        st = _stream()
        for k in range(1, steps + 1):
            idx = torch.randint(0, n, (min(batch, n),), device=self.device, generator=gen)
            xb, tb = X[idx].contiguous(), T[idx].contiguous()
            abi.check(self.L.sph_mlp_grad(_ptr(self.W), _ptr(xb), _ptr(tb), xb.shape[0], _ptr(G),
                                          _ptr(loss), st), "sph_mlp_grad")
            rate = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * (k - 1) / max(steps - 1, 1)))
            abi.check(self.L.sph_mlp_adam(_ptr(self.W), _ptr(G), _ptr(M), _ptr(V), k,
                                          C.c_float(rate), st), "sph_mlp_adam")
            if log_every and k % log_every == 0:
                hist.append(float(loss.item()))
        if not hist:
            hist.append(float(loss.item()))
        return hist

    # ------------------------------------------------------------------ persistence
    def save(self, path):
        np.save(path, self.W.detach().cpu().numpy())

    @classmethod
    def load(cls, path, device="cuda"):
        return cls(np.load(path), device=device)


def collect_returns(scene, steps, capacity, perturb=None, device="cuda"):
    """Exact Johnson-Cook returns of the plain solver on `scene` over `steps` steps:
    (X [m][4] features, T [m] d / d_hi, all 8 logged columns), m <= capacity."""
    ps = ParticleSystem(SimConfig(scene), device=device)
    if perturb is not None:
        perturb(ps)
    sv = ps.build_solver()
    rows = torch.zeros((capacity, 8), dtype=torch.float32, device=device)
    count = torch.zeros(1, dtype=torch.int64, device=device)
    sv.attach_jc_log(rows, count)
    sv.initialize()
    sv.step_many(steps)
    torch.cuda.synchronize()
    m = min(int(count.item()), capacity)
    sv.attach_jc_log(None, None)
    data = rows[:m].clone()
    return data[:, :4].contiguous(), data[:, 4].contiguous(), data
