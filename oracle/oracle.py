"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (liboracle_sph.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker
or the timed CPU baseline; never by the sigmasph_b200 product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle_sph.so")


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("sph_oracle.cpp", "sph_oracle_common.hpp", "Makefile")]
    srcs.append(os.path.join(os.path.dirname(HERE), "include", "sph_b200.h"))
    if not force and os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB)
                                                 for s in srcs):
        return LIB
    r = subprocess.run(["make", "-C", HERE, "-B" if force else "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


class _State(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "x0", "u", "v", "acc", "V", "V_lo", "m",
                                          "pressure", "pst_shift", "pid")]


class _Out(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "x0", "u", "v", "acc", "V", "V_lo", "m",
                                          "pressure", "pst_shift", "pid", "lam", "L_sym",
                                          "lam_grad", "divergence", "de_visc")]


_L = None


def lib():
    global _L
    if _L is None:
        build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, C.c_int64, C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_state.argtypes = [vp, C.POINTER(_State)]
        L.orc_get_state.argtypes = [vp, C.POINTER(_Out)]
        L.orc_set_dt.argtypes = [vp, C.c_double]
        L.orc_get_scalars.argtypes = [vp, C.POINTER(C.c_double)]
        L.orc_step.argtypes = [vp, C.c_int]
        L.orc_stage.argtypes = [vp, C.c_int]
        L.orc_pairs.restype = C.c_int64
        L.orc_pairs.argtypes = [vp, vp, vp, vp, C.c_int64]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_sym_eig3.argtypes = [vp, vp, vp]
        L.orc_sym_eig3_f32.argtypes = [vp, vp, vp]
        L.orc_spd_inverse3.argtypes = [vp, C.c_double, vp]
        _L = L
    return _L


SCALARS = ("dt", "max_c_sq", "max_accel", "max_v", "off_grid_num", "off_grid_mass",
           "wall_work", "visc_work", "diff_work", "leftover_work")


class Oracle:
    """The reference's step restated on the CPU (float32 or float64 arithmetic)."""

    def __init__(self, params, n, fp64=False):
        self.L = lib()
        self.n = int(n)
        self.fp64 = bool(fp64)
        self._params = params
        self.h = self.L.orc_create(C.addressof(params), self.n, int(fp64))

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    @staticmethod
    def threads(nt=None):
        L = lib()
        if nt:
            L.orc_set_threads(int(nt))
        return L.orc_max_threads()

    def set_state(self, st, dt):
        """st: dict with x, x0, u, v, V, V_lo, m, pressure, pst_shift, pid (reference layout)."""
        keep = {}
        s = _State()
        for k in ("x", "x0", "u", "v", "V", "V_lo", "m", "pressure", "pst_shift"):
            a = np.ascontiguousarray(st[k], dtype=np.float64)
            keep[k] = a
            setattr(s, k, a.ctypes.data)
        if st.get("acc") is not None:
            a = np.ascontiguousarray(st["acc"], dtype=np.float64)
            keep["acc"] = a
            s.acc = a.ctypes.data
        p = np.ascontiguousarray(st["pid"], dtype=np.int32)
        keep["pid"] = p
        s.pid = p.ctypes.data
        self.L.orc_set_state(self.h, C.byref(s))
        self.L.orc_set_dt(self.h, float(dt))

    def get_state(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "x0", "u", "v", "acc", "pst_shift", "lam_grad")}
        out.update({k: np.zeros(n) for k in ("V", "V_lo", "m", "pressure", "lam", "divergence",
                                             "de_visc")})
        out["L_sym"] = np.zeros((n, 6))
        out["pid"] = np.zeros(n, dtype=np.int32)
        o = _Out()
        for k, a in out.items():
            setattr(o, k, a.ctypes.data)
        self.L.orc_get_state(self.h, C.byref(o))
        return out

    def scalars(self):
        a = (C.c_double * len(SCALARS))()
        self.L.orc_get_scalars(self.h, a)
        return dict(zip(SCALARS, list(a)))

    def step(self, k=1):
        self.L.orc_step(self.h, int(k))

    def stage(self, s):
        self.L.orc_stage(self.h, int(s))

    def pairs(self):
        cnt = self.L.orc_pairs(self.h, None, None, None, 0)
        pi = np.zeros(cnt, dtype=np.int32)
        pj = np.zeros(cnt, dtype=np.int32)
        pm = np.zeros(cnt, dtype=np.int32)
        self.L.orc_pairs(self.h, pi.ctypes.data, pj.ctypes.data, pm.ctypes.data, cnt)
        return pi, pj, pm


def state_from_sets(sets_np):
    """Reference-layout state from one buffer set of sigmasph_b200 (numpy copies)."""
    s = sets_np
    return {"x": s["pos"][:, :3], "V": s["pos"][:, 3], "v": s["vel"][:, :3], "m": s["vel"][:, 3],
            "x0": s["x0"][:, :3], "V_lo": s["x0"][:, 3], "u": s["disp"][:, :3],
            "pressure": s["disp"][:, 3], "pst_shift": s["shift"][:, :3], "pid": s["pid"]}


def sym_eig3(A, f32=False):
    L = lib()
    if f32:
        a = np.ascontiguousarray(A, dtype=np.float32)
        ev = np.zeros(3, dtype=np.float32)
        Q = np.zeros((3, 3), dtype=np.float32)
        L.orc_sym_eig3_f32(a.ctypes.data, ev.ctypes.data, Q.ctypes.data)
    else:
        a = np.ascontiguousarray(A, dtype=np.float64)
        ev = np.zeros(3)
        Q = np.zeros((3, 3))
        L.orc_sym_eig3(a.ctypes.data, ev.ctypes.data, Q.ctypes.data)
    return ev, Q


def spd_inverse3(E, tol):
    L = lib()
    a = np.ascontiguousarray(E, dtype=np.float64)
    out = np.zeros((3, 3))
    L.orc_spd_inverse3(a.ctypes.data, float(tol), out.ctypes.data)
    return out
