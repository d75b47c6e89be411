"""Synthetic scenes in the reference's card format.

`dambreak3d(dx)` is the 3D delta+-SPH dam break: a water column 0.6 (x, length) x 0.6
(y, height) x 0.3 (z, width) m at the corner of a 1.6 x 1.0 x 0.6 m tank, gravity along
-y, Tait EOS gamma = 7 with c0 = 10 sqrt(2 g H), H = 0.6 m, Wendland support 2.6 dx
(smoothing length 1.3 dx), delta = 0.1, Sun particle shifting.  The tank walls are the
reference's reflecting domain walls, which sit one support radius inside the domain box,
so the domain is the tank grown by that radius.  dx = 4.762 mm gives 126 x 126 x 63 =
1,000,188 particles; dx = 9.449 mm about 128k.

`dambreak3d_1M.json` is the dx = 4.762 mm deck written out.

`tensile_bar3d(dx, plasticity)` is the 3D round-bar tensile test: a parallel-gauge
dogbone revolved about y (gauge diameter 6 mm x 30 mm, heads 10 mm x 15 mm, 3 mm
fillets), steel (rho 7.9e-6 kg/mm^3, E 200 GPa, nu 0.3, linear EOS) with J2 linear
hardening (sigma_y 0.3 GPa, H 1 GPa) or Johnson-Cook hardening (A 0.31, B 1.0 GPa,
n 0.65, C 0.02, reference rate 1/ms), hourglass damper alpha 4, Colle shifting with a
fixed Mach 0.05 and ALE transport, delta 0.1, viscosity 0.02.  The grips are the
outer 10 mm of each head, pulled apart by 1 mm each over a 1 ms smoothstep ramp
(1 m/s on average).  Units mm, GPa, ms.  dx = 0.113 mm lays about 2.3M particles.

`tensile_axi_gauge(dx, speed)` is the same bar as an axisymmetric (x axial, y = r from
dx/2) half-section: about 26k particles at dx = 0.1 mm, Johnson-Cook steel (A 0.31,
B 1.0 GPa, n 0.65; C and the reference rate selectable), hourglass damper sub-cycled,
the outer 10 mm of each head pulled apart by 1 mm over a smoothstep ramp lasting
1 mm / speed (speed in m/s = mm/ms).
"""
from __future__ import annotations

import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

G = 9.81
H_COLUMN = 0.6


def dambreak3d(dx=0.004762, support_factor_dx=2.6, cfl=0.25, column=(0.6, 0.6, 0.3),
               tank=(1.6, 1.0, 0.6), pst=True, viscosity=1.0e-6, delta=0.1):
    r = 0.5 * dx
    h = support_factor_dx * dx
    c0 = 10.0 * math.sqrt(2.0 * G * H_COLUMN)
    nx = [int(round(column[k] / dx)) for k in range(3)]
    start = [h + 0.5 * dx] * 3
    # end half a spacing short of the last site so np.arange lays exactly nx sites
    end = [start[k] + (nx[k] - 0.5) * dx for k in range(3)]
    return {
        "Domain": {"particleRadius": r, "supportRadiusFactor": support_factor_dx * 2.0,
                   "start": [0.0, 0.0, 0.0],
                   "end": [tank[k] + 2.0 * h for k in range(3)],
                   "boundary": "reflect", "restitution": 0.5},
        "Time": {"CFL": cfl, "duration": 2.0},
        "Solver": {"type": "deltaPlusSPH", "viscosity": viscosity,
                   "allowNegativePressure": False},
        "Materials": [{"name": "water", "density0": 1000.0,
                       "eos": {"type": "tait", "c0": c0, "exponent": 7.0}}],
        "Load": {"gravitation": [0.0, -G, 0.0]},
        "Diffusion": {"delta": delta},
        "Shifting": {"enabled": bool(pst), "mode": "sun", "maMode": "local"},
        "FluidBlocks": [{"objectId": 0, "start": start, "end": end,
                         "translation": [0.0, 0.0, 0.0], "scale": [1, 1, 1],
                         "velocity": [0.0, 0.0, 0.0], "density": 1000.0,
                         "color": [50, 100, 200], "material": "water"}],
    }


def dx_for_particles(n, column=(0.6, 0.6, 0.3)):
    """The lattice spacing that lays about n particles in the column."""
    return (column[0] * column[1] * column[2] / float(n)) ** (1.0 / 3.0)


def tensile_bar3d(dx=0.113, plasticity="j2", hourglass_subcycle=False, cfl=0.3):
    gauge_d, gauge_l, head_d, head_l, fillet = 6.0, 30.0, 10.0, 15.0, 3.0
    red = 0.5 * (head_d - gauge_d)
    shoulder = math.sqrt(red * (2.0 * fillet - red))
    half = 0.5 * gauge_l + shoulder + head_l
    grip = half - 10.0
    r = 0.5 * head_d
    if plasticity == "j2":
        plast = {"model": "linear", "yieldStress": 0.3, "hardeningModulus": 1.0}
    elif plasticity == "jc":
        plast = {"model": "johnson_cook", "A": 0.31, "B": 1.0, "n": 0.65, "C": 0.02,
                 "eps0_dot": 1.0, "T0": 293.0, "Tm": 0.0}
    else:
        raise ValueError("plasticity must be 'j2' or 'jc'")
    hg = {"alpha": 4.0}
    if hourglass_subcycle:
        hg["superTimeStepping"] = {"mode": "subcycle"}
    # lattice sites span [start, end) from start + dx/2: the box is the bar's bounding box
    return {
        "Domain": {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "boundary": "open"},
        "Time": {"CFL": cfl},
        "Solver": {"type": "hypoElastic", "viscosity": 0.02, "allowNegativePressure": True},
        "Materials": [{"name": "steel", "density0": 7.9e-6, "eos": {"type": "linear"},
                       "strength": {"type": "hypoElastic", "youngsModulus": 200.0,
                                    "poissonRatio": 0.3, "plasticity": plast}}],
        "Load": {"gravitation": [0.0, 0.0, 0.0], "rampTime": 1.0},
        "Diffusion": {"delta": 0.1},
        "Shifting": {"enabled": True, "mode": "colle", "maMode": "fixed", "maFixed": 0.05,
                     "aleMomentum": True, "aleHistory": True},
        "Hourglass": hg,
        "SolidBlocks": [{"objectId": 0, "start": [-r, -half, -r], "end": [r, half, r],
                         "translation": [0, 0, 0], "scale": [1, 1, 1], "velocity": [0, 0, 0],
                         "density": 7.9e-6, "color": [200, 120, 60], "material": "steel",
                         "shape": {"type": "gaugedogbone3d", "tabWidth": head_d,
                                   "tabHeight": head_l, "gaugeWidth": gauge_d,
                                   "radius": fillet, "gaugeLength": gauge_l,
                                   "center": [0.0, 0.0, 0.0]}}],
        "Constraints": [
            {"name": "low", "region": [[-r - 1, -half - 1, -r - 1], [r + 1, -grip, r + 1]],
             "components": "xyz", "displacement": [0.0, -1.0, 0.0]},
            {"name": "high", "region": [[-r - 1, grip, -r - 1], [r + 1, half + 1, r + 1]],
             "components": "xyz", "displacement": [0.0, 1.0, 0.0]}],
    }


def tensile_axi_gauge(dx=0.1, speed=1.0, C=0.0, eps0_dot=1.0, cfl=0.3, disp=1.0):
    gauge_d, gauge_l, head_d, head_l, fillet = 6.0, 30.0, 10.0, 15.0, 3.0
    red = 0.5 * (head_d - gauge_d)
    shoulder = math.sqrt(red * (2.0 * fillet - red))
    half = 0.5 * gauge_l + shoulder + head_l
    grip = half - 10.0
    r = 0.5 * head_d
    return {
        "Domain": {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "axisymmetric": True,
                   "boundary": "open"},
        "Time": {"CFL": cfl},
        "Solver": {"type": "hypoElastic", "viscosity": 0.02, "allowNegativePressure": True},
        "Materials": [{"name": "steel", "density0": 7.9e-6, "eos": {"type": "linear"},
                       "strength": {"type": "hypoElastic", "youngsModulus": 200.0,
                                    "poissonRatio": 0.3,
                                    "plasticity": {"model": "johnson_cook", "A": 0.31, "B": 1.0,
                                                   "n": 0.65, "C": C, "eps0_dot": eps0_dot,
                                                   "T0": 293.0, "Tm": 0.0}}}],
        "Load": {"gravitation": [0.0, 0.0, 0.0], "rampTime": disp / speed},
        "Diffusion": {"delta": 0.1},
        "Shifting": {"enabled": True, "mode": "colle", "maMode": "fixed", "maFixed": 0.05,
                     "aleMomentum": True, "aleHistory": True},
        "Hourglass": {"alpha": 4.0, "superTimeStepping": {"mode": "subcycle"}},
        "SolidBlocks": [{"objectId": 0, "start": [-half, 0.5 * dx, 0.0], "end": [half, r, 0.5 * dx],
                         "translation": [0, 0, 0], "scale": [1, 1, 1], "velocity": [0, 0, 0],
                         "density": 7.9e-6, "color": [200, 120, 60], "material": "steel",
                         "shape": {"type": "gaugedogboneaxi", "tabWidth": head_d,
                                   "tabHeight": head_l, "gaugeWidth": gauge_d,
                                   "radius": fillet, "gaugeLength": gauge_l,
                                   "center": [0.0, 0.0, 0.0]}}],
        "Constraints": [
            {"name": "left", "region": [[-half - 1, -1, -1], [-grip, r + 1, 1]],
             "components": "xy", "displacement": [-disp, 0.0, 0.0]},
            {"name": "right", "region": [[grip, -1, -1], [half + 1, r + 1, 1]],
             "components": "xy", "displacement": [disp, 0.0, 0.0]}],
    }


def scene_path(name):
    return os.path.join(HERE, name)
