"""The Johnson-Cook return-map surrogate on the GPU: the training kernels against the
float64 oracle (oracle/mlp.py), the BF16 tensor-core inference against the float32
forward, and the trained network inside the solver, where every proposal is checked by
the exact residual (|g| / sigma_y <= tol) and the Newton runs otherwise.

Tolerances: gradient and loss within 1e-4 of float64 (float32 sums over 8k parameters);
tensor-core output within 2e-2 of max |y| of the float32 forward (BF16 operands: 8-bit
mantissa activations through two 64-wide layers); solver fields with the surrogate within
the acceptance tolerance of the plain path (eps_p and s within 1e-3 relative)."""
import numpy as np
import pytest
import torch

from oracle import mlp
from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import scene_path
from sigmasph_b200.surrogate import JCSurrogate, collect_returns
from tests.test_solid_gpu import perturb_solid, solid_gpu_fields

pytestmark = pytest.mark.gpu


def _rand_problem(rows, seed=1):
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, 0.25, mlp.N_PARAMS)
    X = rng.uniform(0.0, 1.0, (rows, 4))
    T = rng.uniform(0.6, 1.0, rows)
    return w, X, T


def test_training_gradient_matches_oracle(cuda):
    w, X, T = _rand_problem(1000)          # not a multiple of the 128-thread blocks
    sur = JCSurrogate(w.astype(np.float32))
    loss, G = sur.loss_and_grad(X.astype(np.float32), T.astype(np.float32))
    l_ref, g_ref = mlp.loss_and_grad(w.astype(np.float32).astype(np.float64),
                                     X.astype(np.float32), T.astype(np.float32))
    g = G.cpu().numpy().astype(np.float64)
    assert float(loss.item()) == pytest.approx(l_ref, rel=1e-4)
    assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


def test_adam_step_matches_formula(cuda):
    w, X, T = _rand_problem(256, seed=2)
    sur = JCSurrogate(w.astype(np.float32))
    w0 = sur.W.clone()
    sur.fit(X.astype(np.float32), T.astype(np.float32), steps=1, batch=256, lr=1e-3, lr_final=1e-3)
    # first Adam step with bias correction: w - lr * g / (|g| + eps), sign descent
    _, g = mlp.loss_and_grad(w0.cpu().numpy().astype(np.float64), X.astype(np.float32),
                             JCSurrogate.target(T.astype(np.float32)))
    # the batch is a resampling of the 256 rows with replacement: compare only the sign
    # and the size of the step, which do not depend on the draw for a first step
    step = (w0 - sur.W).cpu().numpy()
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    assert np.all(np.abs(np.abs(step[big]) - 1e-3) <= 2e-5)


@pytest.mark.parametrize("rows", [1, 127, 129, 5000])
def test_tensor_core_inference_matches_f32(cuda, rows):
    rng = np.random.default_rng(rows)
    w = rng.normal(0.0, 0.2, mlp.N_PARAMS).astype(np.float32)
    X = rng.uniform(0.0, 1.0, (rows, 4)).astype(np.float32)
    sur = JCSurrogate(w)
    y32 = sur.predict_f32(X).cpu().numpy().astype(np.float64)
    ytc = sur.predict(X).cpu().numpy().astype(np.float64)
    y64, _ = mlp.forward(w.astype(np.float64), X)
    assert np.abs(y32 - y64).max() <= 1e-5 * max(np.abs(y64).max(), 1e-6)
    assert np.abs(ytc - y32).max() <= 2e-2 * max(np.abs(y32).max(), 1e-6)


def _dogbone_state(seed):
    return lambda ps: perturb_solid(ps, seed=seed, s_amp=0.3, ep_max=0.1)


@pytest.fixture(scope="module")
def trained():
    """Trained on exact returns of the plain solver on the shipped Johnson-Cook dogbone,
    from three perturbed plastic states."""
    deck = scene_path("tensile_axi_dogbone_dx0.1.json")
    Xs, Ts = [], []
    for seed in (101, 102, 103):
        X, T, _ = collect_returns(deck, steps=6, capacity=200000, perturb=_dogbone_state(seed))
        Xs.append(X)
        Ts.append(T)
    X, T = torch.cat(Xs), torch.cat(Ts)
    sur = JCSurrogate()
    hist = sur.fit(X, T, steps=8000, batch=8192, lr=3e-3, lr_final=3e-5, log_every=1000)
    return sur, X, T, hist


def test_logged_returns_are_exact_fractions(cuda, trained):
    _, X, T, _ = trained
    assert X.shape[0] > 5000
    t = T.cpu().numpy()
    assert np.all(t > 0.0) and np.all(t <= 1.0 + 1e-6)
    assert np.all(np.isfinite(X.cpu().numpy()))


def test_surrogate_in_solver_matches_plain_and_saves_newton(cuda, trained):
    sur, X, T, hist = trained
    assert hist[-1] < 0.2 * hist[0]
    deck = scene_path("tensile_axi_dogbone_dx0.1.json")
    runs = {}
    for mode in ("plain", "surrogate"):
        ps = ParticleSystem(SimConfig(deck), device="cuda")
        _dogbone_state(777)(ps)              # a state the network has not seen
        sv = ps.build_solver()
        if mode == "surrogate":
            sv.enable_jc_surrogate(sur, tol=1e-3)
        sv.initialize()
        sv.jc_stats(reset=True)
        sv.step_many(3)
        runs[mode] = (solid_gpu_fields(ps), sv.jc_stats(), sv.error_word())
    (gp, sp, ep_), (gs, ss, es) = runs["plain"], runs["surrogate"]
    assert ep_ & ~abi.EW_HASHED_GRID == 0 and es & ~abi.EW_HASHED_GRID == 0
    # every yielding return went through the network, and a large share of the proposals
    # was kept: 50-54% in the runs so far (the in-test training sees returns whose float32
    # rounding moves with the solver's own arithmetic), so the bar is 40%
    assert ss["proposals"] >= 0.9 * sp["newton_solves"] and ss["proposals"] > 1000
    assert ss["accepted"] >= 0.4 * ss["proposals"]
    # the gain: exact Newton solves and iterations avoided on the same steps
    assert ss["newton_solves"] <= 0.6 * sp["newton_solves"]
    assert ss["newton_iterations"] <= 0.6 * sp["newton_iterations"]
    for k in ("eps_p", "sdev"):
        scale = np.abs(gp[k]).max()
        assert np.abs(gs[k] - gp[k]).max() <= 1e-3 * scale, k
