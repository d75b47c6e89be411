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

FEATURES = ("ln(max(vm / sigma_y0 - 1, 1e-8)) / 10", "eps_p", "ln(max(eps_dot_eq / eps0_dot, 1)) / 10",
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


def config0_samples(total=5_000_000, rates=None, seed=20260101, dx=0.1, C=0.02, eps0_dot=1.0,
                    chunk=2000, max_steps=200_000, device="cuda"):
    """Exact returns logged from the axisymmetric parallel-gauge bar (scenes.tensile_axi_gauge)
    pulled at grip speeds drawn log-uniformly from [0.1, 10] m/s, an equal quota per run.
    Returns (X, F, speeds)."""
    from .scenes import tensile_axi_gauge
    rng = np.random.default_rng(seed)
    if rates is None:
        rates = np.exp(rng.uniform(np.log(0.1), np.log(10.0), 8))
    quota = int(total // len(rates))
    Xs, Fs = [], []
    for v in rates:
        ps = ParticleSystem(SimConfig(tensile_axi_gauge(dx=dx, speed=float(v), C=C, eps0_dot=eps0_dot)),
                            device=device)
        sv = ps.build_solver()
        rows = torch.zeros((quota, 8), dtype=torch.float32, device=device)
        count = torch.zeros(1, dtype=torch.int64, device=device)
        sv.attach_jc_log(rows, count)
        sv.initialize()
        done = 0
        while done < max_steps:
            sv.step_many(chunk)
            done += chunk
            if int(count.item()) >= quota:
                break
        sv.attach_jc_log(None, None)
        m = min(int(count.item()), quota)
        Xs.append(rows[:m, :4].clone())
        Fs.append(rows[:m, 4].clone())
        del sv, ps
    return torch.cat(Xs), torch.cat(Fs), list(map(float, rates))


def force_displacement(scene, surrogate=None, tol=1e-3, record_every=50, t_end=None, device="cuda"):
    """Runs a solid scene to t_end (default: its load ramp) recording the right grip's
    force and displacement along the pull axis every `record_every` steps; returns
    (disp, force, ms_per_step, stats)."""
    ps = ParticleSystem(SimConfig(scene), device=device)
    sv = ps.build_solver()
    if surrogate is not None:
        sv.enable_jc_surrogate(surrogate, tol=tol)
    sv.initialize()
    t_end = t_end if t_end is not None else float(ps.cfg.get_cfg("rampTime"))
    axis = int(np.argmax(np.abs(np.array(ps.cfg.get_constraints()[-1]["displacement"]))))
    sv.jc_stats(reset=True)
    disp, force = [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = 0
    e0.record()
    while sv.sim_time < t_end:
        sv.step_many(record_every)
        steps += record_every
        d = sv.get_constraint_data()[-1]
        disp.append(float(d["displacement"][axis]))
        force.append(float(d["force"][axis]))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(steps, 1)
    return np.array(disp), np.array(force), ms, sv.jc_stats()


def compare_bar(surrogate, dx=0.4, tol=1e-3, record_every=50, device="cuda"):
    """Plain vs surrogate on the Johnson-Cook 3D round bar (scenes.tensile_bar3d, grips
    +-1 mm over 1 ms): peak-force error and L2 error of the force-displacement curve."""
    from .scenes import tensile_bar3d
    sc = tensile_bar3d(dx=dx, plasticity="jc", hourglass_subcycle=True)
    dp, fp, msp, sp = force_displacement(sc, None, tol, record_every, device=device)
    ds, fs, mss, ss = force_displacement(sc, surrogate, tol, record_every, device=device)
    m = min(len(fp), len(fs))
    peak_p, peak_s = float(np.max(np.abs(fp))), float(np.max(np.abs(fs)))
    return {"dx_mm": dx, "records": m,
            "peak_force_plain": peak_p, "peak_force_surrogate": peak_s,
            "peak_force_rel_err": abs(peak_s - peak_p) / peak_p,
            "curve_l2_rel_err": float(np.linalg.norm(fs[:m] - fp[:m]) / np.linalg.norm(fp[:m])),
            "ms_per_step_plain": msp, "ms_per_step_surrogate": mss,
            "stats_plain": sp, "stats_surrogate": ss,
            "curve_plain": [[float(a), float(b)] for a, b in zip(dp[:m], fp[:m])],
            "curve_surrogate": [[float(a), float(b)] for a, b in zip(ds[:m], fs[:m])]}


def step_cost(surrogate, dx=0.113, tol=1e-3, seed=3, s_amp=0.35, ep_max=0.2, device="cuda"):
    """Per-kernel cost of one eager step of the Johnson-Cook 3D round bar from a synthetic
    plastic state (seeded random trace-free deviators of amplitude s_amp, plastic strains
    uniform in [0, ep_max]), plain and with the surrogate: {mode: {step_ms, kernels, stats}}."""
    from .scenes import tensile_bar3d
    out = {}
    for mode, sur in (("plain", None), ("surrogate", surrogate)):
        ps = ParticleSystem(SimConfig(tensile_bar3d(dx=dx, plasticity="jc")), device=device)
        rng = np.random.default_rng(seed)
        n = ps.particle_max_num
        sd = rng.normal(0.0, s_amp, (n, 3, 3))
        sd = 0.5 * (sd + sd.transpose(0, 2, 1))
        sd -= (np.trace(sd, axis1=1, axis2=2) / 3.0)[:, None, None] * np.eye(3)[None]
        ps.sigma_dev.from_numpy(sd.astype(np.float32))
        ps.eps_plastic.from_numpy(rng.uniform(0.0, ep_max, n).astype(np.float32))
        sv = ps.build_solver()
        if sur is not None:
            sv.enable_jc_surrogate(sur, tol=tol)
        sv.initialize()
        sv.jc_stats(reset=True)
        sv.profile(True)
        sv.profile_read()
        sv.step()
        torch.cuda.synchronize()
        prof = sv.profile_read()
        sv.profile(False)
        out[mode] = {"particles": n, "step_ms": sum(v[0] for v in prof.values()),
                     "kernels": {k: v[0] for k, v in prof.items()
                                 if k in ("k_solid_b", "k_mlp_tc", "k_jc_finish")},
                     "stats": sv.jc_stats(), "error_word": sv.error_word()}
        del sv, ps
        torch.cuda.empty_cache()
    return out


def main(argv=None):
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="Train / evaluate the Johnson-Cook return-map surrogate")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="log config-0 returns, train, save the parameters")
    t.add_argument("--out", required=True)
    t.add_argument("--samples", type=int, default=5_000_000)
    t.add_argument("--steps", type=int, default=20000)
    t.add_argument("--batch", type=int, default=8192)
    c = sub.add_parser("compare", help="plain vs surrogate force-displacement on the 3D JC bar")
    c.add_argument("--weights", required=True)
    c.add_argument("--dx", type=float, default=0.4)
    c.add_argument("--out", default=None)
    k = sub.add_parser("cost", help="per-kernel cost of one step from a synthetic plastic state")
    k.add_argument("--weights", required=True)
    k.add_argument("--dx", type=float, default=0.113)
    a = ap.parse_args(argv)
    if a.cmd == "cost":
        print(json.dumps(step_cost(JCSurrogate.load(a.weights), dx=a.dx)))
        return 0
    if a.cmd == "train":
        t0 = time.time()
        X, F, rates = config0_samples(total=a.samples)
        t1 = time.time()
        sur = JCSurrogate()
        hist = sur.fit(X, F, steps=a.steps, batch=a.batch, lr=3e-3, lr_final=3e-5,
                       log_every=max(a.steps // 10, 1))
        t2 = time.time()
        sur.save(a.out)
        u = sur.predict(X[:200000])
        err = (u - JCSurrogate.target(F[:200000])).abs()
        print(json.dumps({"samples": int(X.shape[0]), "speeds_mps": rates, "loss": hist,
                          "collect_s": t1 - t0, "train_s": t2 - t1,
                          "abs_err_u_tc_p50": float(err.median()),
                          "abs_err_u_tc_p99": float(err.quantile(0.99))}))
    else:
        res = compare_bar(JCSurrogate.load(a.weights), dx=a.dx)
        line = {k: v for k, v in res.items() if not k.startswith("curve")}
        print(json.dumps(line))
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
