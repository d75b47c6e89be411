"""Synthetic scenes in the reference's card format.

`dambreak3d(dx)` is the 3D delta+-SPH dam break: a water column 0.6 (x, length) x 0.6
(y, height) x 0.3 (z, width) m at the corner of a 1.6 x 1.0 x 0.6 m tank, gravity along
-y, Tait EOS gamma = 7 with c0 = 10 sqrt(2 g H), H = 0.6 m, Wendland support 2.6 dx
(smoothing length 1.3 dx), delta = 0.1, Sun particle shifting.  The tank walls are the
reference's reflecting domain walls, which sit one support radius inside the domain box,
so the domain is the tank grown by that radius.  dx = 4.762 mm gives 126 x 126 x 63 =
1,000,188 particles; dx = 9.449 mm about 128k.

`dambreak3d_1M.json` is the dx = 4.762 mm deck written out.
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


def scene_path(name):
    return os.path.join(HERE, name)
