"""The CPU oracle against the reference's known-answer values and against numpy
(no GPU).  These pin the restatement before it is trusted as the checker."""
import numpy as np
import pytest

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import dambreak3d, dx_for_particles
from sigmasph_b200.solver import build_params
from oracle.oracle import Oracle, state_from_sets, sym_eig3, spd_inverse3


def _oracle(scene, fp64=True):
    ps = ParticleSystem(SimConfig(scene), device="cpu")
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=fp64)
    o.set_state(state_from_sets(ps.state_numpy()), 1e-4)
    o.stage(abi.STAGE_SORT)
    return ps, o


def plane_strain_block(dx=0.1):
    sc = dambreak3d(dx=dx, column=(3.0, 2.0, dx), tank=(5, 5, 1))
    sc["Domain"]["planeStrain"] = True
    sc["Domain"]["supportRadiusFactor"] = 6.0
    sc["Domain"]["boundary"] = "open"
    b = sc["FluidBlocks"][0]
    b["start"] = [1.0, 1.0, 0.0]
    b["end"] = [3.95, 2.95, 0.5 * dx]
    return sc


def test_lambda_plateau_known_answers():
    """SOLID.py:350-359: at support 3 dx0 in plane strain lambda is 0.997 in the
    interior, 0.499 on a flat free edge and 0.254 at a convex corner."""
    dx = 0.1
    ps, o = _oracle(plane_strain_block(dx))
    o.stage(abi.STAGE_LAM)
    s = o.get_state()
    x, lam = s["x"], s["lam"]
    xmin, xmax, ymin, ymax = x[:, 0].min(), x[:, 0].max(), x[:, 1].min(), x[:, 1].max()
    inner = ((x[:, 0] > xmin + 3.5 * dx) & (x[:, 0] < xmax - 3.5 * dx) &
             (x[:, 1] > ymin + 3.5 * dx) & (x[:, 1] < ymax - 3.5 * dx))
    edge = (np.abs(x[:, 1] - ymin) < 1e-6) & (x[:, 0] > xmin + 3.5 * dx) & (x[:, 0] < xmax - 3.5 * dx)
    corner = (np.abs(x[:, 1] - ymin) < 1e-6) & (np.abs(x[:, 0] - xmin) < 1e-6)
    assert np.allclose(lam[inner], 0.997, atol=1e-3)
    assert np.allclose(lam[edge], 0.499, atol=1e-3)
    assert np.allclose(lam[corner], 0.254, atol=1e-3)


def test_lattice_neighbour_counts():
    """Strict-< lattice counts: 80 at 2.6 dx in 3D (lattice rounding may admit the
    exact-distance ties at 3 dx, so the 3 dx counts lie in [24, 28] and [92, 122])."""
    ps, o = _oracle(dambreak3d(dx=dx_for_particles(6000)))
    pi, _, _ = o.pairs()
    cnt = np.bincount(pi, minlength=ps.particle_max_num)
    assert cnt.max() == 80
    ps, o = _oracle(plane_strain_block())
    pi, _, _ = o.pairs()
    cnt = np.bincount(pi, minlength=ps.particle_max_num)
    assert 24 <= np.median(cnt) <= 28


def test_pair_relation_is_symmetric():
    ps, o = _oracle(dambreak3d(dx=dx_for_particles(4000)))
    pi, pj, _ = o.pairs()
    n = ps.particle_max_num
    a = np.sort(pi.astype(np.int64) * n + pj)
    b = np.sort(pj.astype(np.int64) * n + pi)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("seed", range(6))
def test_jacobi_eigensolver_matches_numpy(seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(3, 3))
    A = A + A.T
    if seed == 0:
        A = np.eye(3) * 0.97
    if seed == 1:
        A = np.diag([1.0, 1.0, 1e-7])
    ev, Q = sym_eig3(A)
    ref = np.linalg.eigvalsh(A)
    assert np.allclose(np.sort(ev), ref, atol=1e-12 * max(1.0, np.abs(ref).max()))
    assert np.allclose(Q.T @ Q, np.eye(3), atol=1e-12)
    assert np.allclose(Q @ np.diag(ev) @ Q.T, A, atol=1e-11 * max(1.0, np.abs(A).max()))
    ev32, Q32 = sym_eig3(A, f32=True)
    assert np.allclose(np.sort(ev32), ref, atol=2e-6 * max(1.0, np.abs(ref).max()))


def test_regularised_inverse_properties():
    """spd_inverse.py: full inverse where every eigenvalue >= 2 tol, the identity where
    all are <= tol, symmetric and basis independent."""
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    E = Q @ np.diag([0.9, 0.5, 0.3]) @ Q.T
    assert np.allclose(spd_inverse3(E, 0.1), np.linalg.inv(E), atol=1e-12)
    E = Q @ np.diag([0.05, 0.01, 0.0]) @ Q.T
    assert np.allclose(spd_inverse3(E, 0.1), np.eye(3), atol=1e-12)
    E = Q @ np.diag([0.9, 0.15, 0.15]) @ Q.T
    L = spd_inverse3(E, 0.1)
    assert np.allclose(L, L.T)
    u = (0.15 - 0.1) / 0.1
    beta = u * u * (3 - 2 * u)
    w = beta / 0.15 + 1 - beta
    assert np.allclose(L, Q @ np.diag([1 / 0.9, w, w]) @ Q.T, atol=1e-12)


def test_fp32_oracle_tracks_fp64_oracle():
    sc = dambreak3d(dx=dx_for_particles(3000))
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    st = state_from_sets(ps.state_numpy())
    res = []
    for fp64 in (False, True):
        o = Oracle(build_params(ps), ps.particle_max_num, fp64=fp64)
        o.set_state(st, 4e-4)
        o.stage(abi.STAGE_SORT)
        o.step(5)
        s = o.get_state()
        res.append(s["x"][np.argsort(s["pid"])])
    assert np.abs(res[0] - res[1]).max() < 1e-6 * ps.particle_diameter * 100


# ------------------------------------------------------------------ analytic identities
# The oracle's pair sums restate the reference's kernel bodies; these identities pin them
# to the physics they discretise, independently of the restatement: on a lattice interior
# the kernel's first moment sum_j V_j (x_j - x_i) (x) grad W_ij is lambda I (lambda: the
# lambda pass's value there, 0.979 at 2.6 dx in 3D), so a linear field's SPH derivative
# is lambda times the exact one.

def _linear_field_oracle(n=8000):
    sc = dambreak3d(dx=dx_for_particles(n), pst=False, viscosity=0.0)
    sc["Load"]["gravitation"] = [0.0, 0.0, 0.0]
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    st = state_from_sets(ps.state_numpy())
    x = st["x"].astype(np.float64)
    h = float(ps.support_radius)
    box = (x.min(0) + h, x.max(0) - h)
    return ps, build_params(ps), st, x, box


def _interior(x, box):
    return np.all((x > box[0]) & (x < box[1]), axis=1)


def test_continuity_of_a_linear_velocity_field():
    """v = A x: the continuity pass's volumetric strain rate sum_j V_j (v_i - v_j) . grad W
    (DSPH.py:1208-1338) is -lambda tr(A) in the interior (dV/dt = -V times it: a field
    that spreads grows the volume)."""
    ps, p, st, x, box = _linear_field_oracle()
    A = np.random.default_rng(3).normal(size=(3, 3)) * 0.1
    st["v"] = x @ A.T
    o = Oracle(p, ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-4)
    for s in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY):
        o.stage(s)
    g = o.get_state()
    inn = _interior(g["x"], box)
    assert inn.sum() > 2000
    want = -g["lam"][inn] * np.trace(A)
    assert np.abs(g["divergence"][inn] - want).max() <= 1e-4 * np.abs(want).max()
    V0 = dict(zip(st["pid"], st["V"]))
    V_before = np.array([V0[k] for k in g["pid"][inn]])
    assert np.all(np.sign(g["V"][inn] - V_before) == np.sign(np.trace(A)))


def test_pressure_acceleration_of_a_linear_pressure_field():
    """p = p0 + G . x (set through the volumes, the Tait EOS inverted): the symmetric
    pressure force -sum_j w_i w_j (p_i + p_j) grad W / mw_i (DSPH.py:1523-1560) is
    -lambda G / rho in the interior.  The volumes' 1e-4 spread leaves a p_i sum_j V_j grad W
    of ~6e-4 of the result."""
    ps, p, st, x, box = _linear_field_oracle()
    G = np.array([300.0, -200.0, 150.0])
    pt = 20.0 - (x @ G).min() + x @ G
    S, gam, rho0 = float(p.stiffness), float(p.exponent), float(p.density0)
    st["V"] = st["m"] / (rho0 * (1.0 + pt / S) ** (1.0 / gam))
    o = Oracle(p, ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-7)
    for s in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY, abi.STAGE_FORCES):
        o.stage(s)
    g = o.get_state()
    inn = _interior(g["x"], box)
    want = -(g["lam"][:, None] * G[None, :]) / (g["m"] / g["V"])[:, None]
    assert np.abs(g["acc"][inn] - want[inn]).max() <= 2e-3 * np.abs(want[inn]).max()


def test_kernel_corrected_velocity_gradient_is_exact_for_linear_fields():
    """Solver.kernelCorrection: grad v = sum_j V_j (v_j - v_i) (x) grad W times the FP64
    regularised inverse of the moment (SOLID.py:1757-1771, spd_inverse.py:45-101) is
    exact for v = A x at every particle, the free surface included (where the moment is
    far from lambda I)."""
    from tests.test_solid_gpu import bar3d_kc_deck
    ps = ParticleSystem(SimConfig(bar3d_kc_deck()), device="cpu")
    st = state_from_sets(ps.state_numpy())
    A = np.random.default_rng(5).normal(size=(3, 3)) * 1e-3
    st["v"] = st["x"].astype(np.float64) @ A.T
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-6)
    o.stage(abi.STAGE_SORT)
    o.stage(abi.STAGE_LAM)
    g = o.get_state()
    assert g["lam"].min() < 0.3            # the surface and its edges are in the sample
    G = g["grad_v"].reshape(-1, 3, 3)
    assert np.abs(G - A[None]).max() <= 1e-12 * np.abs(A).max()


def test_morris_viscosity_vanishes_for_a_linear_velocity_field():
    """The Morris viscous term 2 (dim + 2) nu sum_j w_j (v_ij . r_ij) / (|r_ij|^2 + eta^2)
    grad W_ij (DSPH.py:1560-1600) discretises nu lap(v); lap(A x) = 0, and on a lattice
    interior each pair's even (v_ij . r) against the odd grad W cancels with its mirror
    neighbour: the interior acceleration vanishes (to 1e-3 of nu |A| / dx, a single pair
    term's scale; the float32 lattice positions are symmetric to ~1e-7)."""
    sc = dambreak3d(dx=dx_for_particles(8000), pst=False, viscosity=1e-3)
    sc["Load"]["gravitation"] = [0.0, 0.0, 0.0]
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    p = build_params(ps)
    st = state_from_sets(ps.state_numpy())
    x = st["x"].astype(np.float64)
    h, dx = float(ps.support_radius), float(ps.particle_diameter)
    box = (x.min(0) + h, x.max(0) - h)
    A = np.random.default_rng(3).normal(size=(3, 3)) * 0.1
    st["v"] = x @ A.T
    o = Oracle(p, ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-7)
    for s in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY, abi.STAGE_FORCES):
        o.stage(s)
    g = o.get_state()
    inn = _interior(g["x"], box)
    assert np.abs(g["acc"][inn]).max() <= 1e-3 * float(p.viscosity) * np.abs(A).max() / dx


def test_delta_diffusion_of_linear_and_quadratic_densities():
    """delta-SPH density diffusion delta h c0 sum_j V_j psi_ij . grad W / rho_i with
    psi_ij = 2 (rho_j - rho_i)(-r_ij) / (|r_ij|^2 + eta^2) (DSPH.py:1269-1300, Molteni &
    Colagrossi) discretises delta h c0 lap(rho) / rho: at rest it is the whole continuity
    rate.  A linear density has no Laplacian and the interior rate vanishes (to 1e-3 of a
    single pair term's scale delta h c0 |grad rho| / (rho dx)); a quadratic one,
    rho = rho0 + a (y - y_mid)^2, gives a positive rate within 10% of delta h c0 2a / rho
    (the lattice and the eta^2 regularisation take ~6%)."""
    ps, p, st, x, box = _linear_field_oracle()
    hdc = float(p.delta_sph) * float(ps.support_radius) * float(p.c0)
    G = np.array([1.0, -0.5, 0.7])
    for name, rho in (("linear", 1000.0 + x @ G),
                      ("quadratic", 1000.0 + 50.0 * (x[:, 1] - x[:, 1].mean()) ** 2)):
        s = dict(st)
        s["V"] = st["m"] / rho
        o = Oracle(p, ps.particle_max_num, fp64=True)
        o.set_state(s, 1e-7)
        for k in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY):
            o.stage(k)
        g = o.get_state()
        inn = _interior(g["x"], box)
        rate = g["divergence"][inn]
        if name == "linear":
            scale = hdc * np.abs(G).max() / 1000.0 / float(ps.particle_diameter)
            assert np.abs(rate).max() <= 1e-3 * scale
        else:
            want = hdc * 100.0 / (g["m"][inn] / g["V"][inn])
            assert np.all(rate > 0.9 * want) and np.all(rate < 1.0 * want)


def test_shift_vanishes_on_an_undisturbed_lattice():
    """The particle shift (Sun form, DSPH.py:712-1049) is driven by the kernel-weighted
    disorder sum sum_j (1 + R (W / W(dx0))^n) m_j / rho_ij grad W, which the symmetric
    lattice cancels: after one step of the column at rest without gravity, the interior
    shift is zero (1e-12 of the spacing)."""
    sc = dambreak3d(dx=dx_for_particles(8000), viscosity=0.0)
    sc["Load"]["gravitation"] = [0.0, 0.0, 0.0]
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    st = state_from_sets(ps.state_numpy())
    x = st["x"].astype(np.float64)
    h = float(ps.support_radius)
    box = (x.min(0) + h, x.max(0) - h)
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-4)
    for k in range(8):
        o.stage(k)
    g = o.get_state()
    inn = _interior(g["x"], box)
    assert inn.sum() > 2000
    assert np.abs(g["pst_shift"][inn]).max() <= 1e-12 * float(ps.particle_diameter)


def test_pressure_force_conserves_momentum():
    """The symmetric pressure force w_i w_j (p_i + p_j) grad W_ij / mw_i (DSPH.py:1523-1560)
    is antisymmetric in the pair once multiplied by m_i = mw_i: for any pressure field
    (random densities here, at rest, no gravity, no viscosity or shift) the accelerations
    carry no net momentum, sum_i m_i a_i = 0 (to 1e-12 of sum_i m_i |a_i|)."""
    ps, p, st, x, box = _linear_field_oracle()
    rng = np.random.default_rng(4)
    S, gam, rho0 = float(p.stiffness), float(p.exponent), float(p.density0)
    pt = rng.uniform(10.0, 500.0, len(x))
    st["V"] = st["m"] / (rho0 * (1.0 + pt / S) ** (1.0 / gam))
    o = Oracle(p, ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-7)
    for k in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY, abi.STAGE_FORCES):
        o.stage(k)
    g = o.get_state()
    ma = g["m"][:, None] * g["acc"]
    gross = np.abs(ma).sum()
    assert gross > 0.0
    assert np.abs(ma.sum(axis=0)).max() <= 1e-12 * gross
