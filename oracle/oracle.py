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


STATE_KEYS = ("x", "x0", "u", "v", "acc", "V", "V_lo", "m", "pressure", "pst_shift", "pid",
              "sdev", "eps_p", "e_int", "temperature", "de_int", "bc_flag", "bc_id", "bc_disp",
              "eos_id")
INT_KEYS = ("pid", "bc_flag", "bc_id", "eos_id")


class _State(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in STATE_KEYS]


class _Out(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("x", "x0", "u", "v", "acc", "V", "V_lo", "m",
                                          "pressure", "pst_shift", "pid", "lam", "L_sym",
                                          "lam_grad", "divergence", "de_visc", "sdev", "eps_p",
                                          "e_int", "temperature", "de_int", "bc_flag",
                                          "grad_v")]


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
        L.orc_j2_return.restype = C.c_double
        L.orc_j2_return.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, vp]
        L.orc_jc_return.restype = C.c_double
        L.orc_jc_return.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, vp, vp]
        _L = L
    return _L


SCALARS = ("dt", "max_c_sq", "max_accel", "max_v", "off_grid_num", "off_grid_mass",
           "wall_work", "visc_work", "diff_work", "leftover_work", "sim_time", "plastic_work",
           "hg_work", "load_s", "load_sdot", "sts_stages")
N_SCALAR_SLOTS = 64


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
        for k in STATE_KEYS:
            if st.get(k) is None:
                continue
            a = np.ascontiguousarray(st[k], dtype=np.int32 if k in INT_KEYS else np.float64)
            keep[k] = a
            setattr(s, k, a.ctypes.data)
        self.L.orc_set_state(self.h, C.byref(s))
        self.L.orc_set_dt(self.h, float(dt))

    def get_state(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "x0", "u", "v", "acc", "pst_shift", "lam_grad")}
        out.update({k: np.zeros(n) for k in ("V", "V_lo", "m", "pressure", "lam", "divergence",
                                             "de_visc")})
        out["L_sym"] = np.zeros((n, 6))
        out["pid"] = np.zeros(n, dtype=np.int32)
        if self._params.is_solid:
            out.update({k: np.zeros(n) for k in ("eps_p", "e_int", "temperature", "de_int")})
            out["sdev"] = np.zeros((n, 6))
            out["grad_v"] = np.zeros((n, 9))
            out["bc_flag"] = np.zeros(n, dtype=np.int32)
        o = _Out()
        for k, a in out.items():
            setattr(o, k, a.ctypes.data)
        self.L.orc_get_state(self.h, C.byref(o))
        return out

    def scalars(self):
        a = (C.c_double * N_SCALAR_SLOTS)()
        self.L.orc_get_scalars(self.h, a)
        out = dict(zip(SCALARS, list(a)))
        out["constraint_force"] = np.array(a[16:40]).reshape(8, 3)
        out["constraint_disp"] = np.array(a[40:64]).reshape(8, 3)
        return out

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
    out = {"x": s["pos"][:, :3], "V": s["pos"][:, 3], "v": s["vel"][:, :3], "m": s["vel"][:, 3],
           "x0": s["x0"][:, :3], "V_lo": s["x0"][:, 3], "u": s["disp"][:, :3],
           "pressure": s["disp"][:, 3], "pst_shift": s["shift"][:, :3], "pid": s["pid"]}
    if "sdev" in s:
        out.update({"sdev": s["sdev"][:, :6], "eps_p": s["sdev"][:, 6],
                    "temperature": s["sdev"][:, 7], "e_int": s["shift"][:, 3],
                    "bc_flag": s["bc"][:, 0], "bc_id": s["bc"][:, 1],
                    "bc_disp": s["bcdisp"][:, :3],
                    "eos_id": np.rint(s["bcdisp"][:, 3]).astype(np.int32),
                    "acc": s["acc"][:, :3], "de_int": s["acc"][:, 3]})
    return out


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


def j2_return(s, G, sy0, H, eps_p):
    """Linear-hardening radial return of one deviator: (s_new, d_eps_p)."""
    a = np.ascontiguousarray(s, dtype=np.float64).reshape(9)
    out = np.zeros(9)
    d = lib().orc_j2_return(a.ctypes.data, float(G), float(sy0), float(H), float(eps_p),
                            out.ctypes.data)
    return out.reshape(3, 3), d


def jc_return(s, G, A, B, n, C_rate, eps0_dot, T0, Tm, m, eps_p, temp, dt):
    """Johnson-Cook radial return of one deviator: (s_new, d_eps_p, iterations)."""
    a = np.ascontiguousarray(s, dtype=np.float64).reshape(9)
    k = np.array([G, A, B, n, C_rate, eps0_dot, T0, Tm, m], dtype=np.float64)
    out = np.zeros(9)
    it = C.c_int(0)
    d = lib().orc_jc_return(a.ctypes.data, k.ctypes.data, float(eps_p), float(temp), float(dt),
                            out.ctypes.data, C.byref(it))
    return out.reshape(3, 3), d, it.value
