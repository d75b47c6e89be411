"""The grip recorder writes the reference's CSV layouts (constraint_recorder.py:47-125):
file names, headers, number formats, the two-grip summary columns."""
import numpy as np

from sigmasph_b200.constraint_recorder import ConstraintRecorder


class _FakeSolver:
    num_constraints = 2
    constraints_list = [{"name": "left"}, {"name": "right"}]

    def __init__(self):
        self.k = 0
        self.load_s = {None: 0.25}

    def get_constraint_data(self):
        self.k += 1
        return [{"index": 0, "name": "left", "displacement": np.array([-0.1 * self.k, 0.0, 0.0]),
                 "force": np.array([3.0 * self.k, 0.5, 0.0])},
                {"index": 1, "name": "right", "displacement": np.array([0.1 * self.k, 0.0, 0.0]),
                 "force": np.array([-2.0 * self.k, -0.5, 0.0])}]


def test_recorder_layout(tmp_path):
    rec = ConstraintRecorder("deck", _FakeSolver(), interval=2, output_dir=str(tmp_path))
    for step in range(5):
        rec.record(step, 1e-3 * step)
    rec.record(4, 4e-3)                      # a repeated step is not written twice
    rec.close()
    wide = (tmp_path / "deck_constraints.csv").read_text().splitlines()
    head = wide[0].split(",")
    assert head[:3] == ["step", "time", "load_s"]
    assert head[3:11] == ["c0_left_ux", "c0_left_uy", "c0_left_uz", "c0_left_umag",
                          "c0_left_Fx", "c0_left_Fy", "c0_left_Fz", "c0_left_Fmag"]
    assert head[-2:] == ["u_rel_mag", "F_axial_avg"] and len(head) == 3 + 16 + 2
    assert [r.split(",")[0] for r in wide[1:]] == ["0", "2", "4"]
    row = wide[2].split(",")                  # step 2, second read: k = 2
    assert row[1] == "2.00000000e-03" and row[2] == "2.500000e-01"
    assert float(row[-2]) == np.float64(0.4) and float(row[-1]) == 0.5 * (6.0 + 4.0)
    indiv = (tmp_path / "deck_constraint_right.csv").read_text().splitlines()
    assert indiv[0] == "step,time,load_s,u_x,u_y,u_z,u_mag,F_x,F_y,F_z,F_mag"
    r = indiv[2].split(",")
    assert float(r[3]) == 0.2 and float(r[7]) == -4.0
    assert abs(float(r[10]) - np.hypot(4.0, 0.5)) < 1e-7
