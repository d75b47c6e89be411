"""Grip force / displacement recorder (the reference's constraint_recorder.py:25-138).

Writes the reference's two CSV layouts, column for column, so existing plotting scripts
read them unchanged:

* `<scene>_constraints.csv`: step, time, load_s, then per constraint k named N the eight
  columns c{k}_{N}_ux, _uy, _uz, _umag, _Fx, _Fy, _Fz, _Fmag; with exactly two
  constraints also u_rel_mag (|u_1 - u_0|) and F_axial_avg ((|F_0x| + |F_1x|) / 2);
* `<scene>_constraint_{N}.csv` per constraint (N keeps a leading "constraint_"):
  step, time, load_s, u_x, u_y, u_z, u_mag, F_x, F_y, F_z, F_mag.

Numbers are written with 9 significant digits (%.8e), load_s with 7 (%.6e).  The solver
is anything with num_constraints, constraints_list, load_s[None] and
get_constraint_data() (HypoElasticSolver); each record() reads the grips once (one
device synchronisation).
"""
from __future__ import annotations

import os

import numpy as np


def _e8(x):
    return f"{float(x):.8e}"


class ConstraintRecorder:
    def __init__(self, scene_name, solver, interval=1, output_dir="."):
        self.scene_name = scene_name
        self.solver = solver
        self.interval = max(1, int(interval))
        self.output_dir = output_dir
        self.num_constraints = int(getattr(solver, "num_constraints", 0))
        self.enabled = self.num_constraints > 0
        self.wide_file = None
        self.indiv_files = []
        self.indiv_paths = []
        self._last_step = None
        if not self.enabled:
            return
        self.constraints_list = list(getattr(solver, "constraints_list", []))
        os.makedirs(output_dir, exist_ok=True)
        names = [c.get("name", f"constraint_{k}") for k, c in enumerate(self.constraints_list)]
        self.wide_path = os.path.join(output_dir, f"{scene_name}_constraints.csv")
        head = ["step", "time", "load_s"]
        for k, nm in enumerate(names):
            pre = f"c{k}_{nm}"
            head += [pre + s for s in ("_ux", "_uy", "_uz", "_umag", "_Fx", "_Fy", "_Fz", "_Fmag")]
        if self.num_constraints == 2:
            head += ["u_rel_mag", "F_axial_avg"]
        self.wide_file = open(self.wide_path, "w", buffering=65536)
        self.wide_file.write(",".join(head) + "\n")
        for nm in names:
            tag = nm if nm.startswith("constraint_") else f"constraint_{nm}"
            path = os.path.join(output_dir, f"{scene_name}_{tag}.csv")
            f = open(path, "w", buffering=65536)
            f.write("step,time,load_s,u_x,u_y,u_z,u_mag,F_x,F_y,F_z,F_mag\n")
            self.indiv_files.append(f)
            self.indiv_paths.append(path)

    def record(self, step, time):
        """Append the grips' state at `step` if it is on the interval and not yet written."""
        if not self.enabled or step % self.interval != 0 or step == self._last_step:
            return
        data = self.solver.get_constraint_data()
        if not data:
            return
        self._last_step = step
        s = float(self.solver.load_s[None])
        lead = [str(step), _e8(time), f"{s:.6e}"]
        wide = list(lead)
        us, fs = [], []
        for k, d in enumerate(data):
            u = np.asarray(d["displacement"], dtype=np.float64)
            f = np.asarray(d["force"], dtype=np.float64)
            us.append(u)
            fs.append(f)
            cols = [_e8(u[0]), _e8(u[1]), _e8(u[2]), _e8(np.linalg.norm(u)),
                    _e8(f[0]), _e8(f[1]), _e8(f[2]), _e8(np.linalg.norm(f))]
            wide += cols
            if k < len(self.indiv_files):
                self.indiv_files[k].write(",".join(lead + cols) + "\n")
        if self.num_constraints == 2 and len(us) == 2:
            wide += [_e8(np.linalg.norm(us[1] - us[0])), _e8(0.5 * (abs(fs[0][0]) + abs(fs[1][0])))]
        self.wide_file.write(",".join(wide) + "\n")

    def close(self):
        if not self.enabled:
            return
        for f in [self.wide_file] + self.indiv_files:
            if f:
                f.flush()
                f.close()
        self.wide_file = None
        self.indiv_files = []
