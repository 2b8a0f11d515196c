"""ctypes view of the f64 oracle library (oracle/_build/liboracle.so).

Test infrastructure: tests/, the smoke check and bench.py's CPU-baseline leg use it as the checker. It builds the
library with `make -C oracle` when the shared object is missing or older than its sources.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE, "_build", "liboracle.so")
CLI = os.path.join(ORACLE, "_build", "oracle")
P = ctypes.c_void_p
_lib = None


def build():
    sources = [os.path.join(ORACLE, f) for f in os.listdir(ORACLE) if f.endswith((".h", ".cpp"))]
    newest = max(os.path.getmtime(s) for s in sources)
    if not (os.path.exists(LIB) and os.path.exists(CLI)) or min(os.path.getmtime(LIB), os.path.getmtime(CLI)) < newest:
        subprocess.run(["make", "-s", "-C", ORACLE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        lib.oracle_last_error.restype = ctypes.c_char_p
        lib.oracle_unit_test_name.restype = ctypes.c_char_p
        lib.oracle_unit_test_message.restype = ctypes.c_char_p
        lib.oracle_scene_create.restype = P
        lib.oracle_scene_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_uint64,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        lib.oracle_scene_free.argtypes = [P]
        lib.oracle_energy_change.restype = ctypes.c_double
        lib.oracle_energy_change.argtypes = [P, P, P, ctypes.c_double, P, ctypes.c_double]
        lib.oracle_max_step.restype = ctypes.c_double
        lib.oracle_max_step.argtypes = [P, P, P]
        lib.oracle_static_energy.restype = ctypes.c_double
        lib.oracle_static_energy.argtypes = [P, P]
        lib.oracle_assemble.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_int, P, P]
        lib.oracle_ptc.argtypes = [P, P, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double, P, P]
        lib.oracle_time_step.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, P, P, P]
        lib.oracle_pcg.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_int, P, P]
        _lib = lib
    return _lib


def ptr(a):
    return a.ctypes.data_as(P)


class Scene:
    """One oracle drape: kind 'reference' (edit), 'sheet' (seed, radius, young, plane) or 'pinned'."""

    def __init__(self, kind="sheet", columns=33, edit="base", seed=0, radius=0.25, young=5e5, plane=False,
                 projected=False):
        self.lib = load()
        k = {"reference": 0, "sheet": 1, "pinned": 2}[kind]
        self.h = self.lib.oracle_scene_create(k, columns, edit.encode(), seed, radius, young, int(plane),
                                              int(projected))
        if not self.h:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        sz = np.zeros(6, np.int64)
        self.lib.oracle_scene_sizes(P(self.h), ptr(sz))
        self.V, self.T, self.H, self.R, self.B, self.colliders = (int(v) for v in sz)
        sc = np.zeros(7)
        self.lib.oracle_scene_scalars(P(self.h), ptr(sc))
        self.dhat, self.kappa, self.g, self.gravity_load = sc[:4]
        self.gravity = sc[4:7].copy()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_scene_free(P(self.h))

    def start(self):
        x = np.zeros(3 * self.V)
        self.lib.oracle_scene_start(P(self.h), ptr(x))
        return x

    def mass(self):
        m = np.zeros(self.V)
        self.lib.oracle_scene_mass(P(self.h), ptr(m))
        return m

    def pattern(self):
        rp = np.zeros(self.R + 1, np.int32)
        ci = np.zeros(self.B, np.int32)
        self.lib.oracle_scene_pattern(P(self.h), ptr(rp), ptr(ci))
        return rp, ci

    def kernel_state(self):
        x = np.zeros(3 * self.V)
        self.lib.oracle_kernel_state(P(self.h), ptr(x))
        return x

    def contact_state(self):
        x = np.zeros(3 * self.V)
        self.lib.oracle_contact_state(P(self.h), ptr(x))
        return x

    def assemble(self, x, x_hat, h, mu=0.0, curvature=True):
        g = np.zeros(3 * self.R)
        v = np.zeros(9 * self.B)
        if self.lib.oracle_assemble(P(self.h), ptr(x), ptr(x_hat), h, mu, int(curvature), ptr(g), ptr(v)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return g, v

    def energy_change(self, x, x_hat, h, d, alpha):
        return self.lib.oracle_energy_change(P(self.h), ptr(x), ptr(x_hat), h, ptr(d), alpha)

    def max_step(self, x, d):
        return self.lib.oracle_max_step(P(self.h), ptr(x), ptr(d))

    def static_gradient(self, x):
        g = np.zeros(3 * self.R)
        self.lib.oracle_static_gradient(P(self.h), ptr(x), ptr(g))
        return g

    def static_energy(self, x):
        return self.lib.oracle_static_energy(P(self.h), ptr(x))

    def time_step(self, x, v, h, tolerance=1e-10, max_iterations=30, pcg=False, rtol=1e-6, maxit=2000):
        """One backward-Euler step (drape.rs:410-417) from (x, v): (x_new, v_new, stats dict)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        x_out, v_out, st = np.zeros(3 * self.V), np.zeros(3 * self.V), np.zeros(5)
        if self.lib.oracle_time_step(P(self.h), ptr(x), None if v is None else ptr(v), h, tolerance, max_iterations,
                                     int(pcg), rtol, maxit, ptr(x_out), ptr(v_out), ptr(st)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return x_out, v_out, dict(zip(["iterations", "status", "final_relative_residual", "scale", "max_mu"],
                                      st.tolist()))

    def ptc(self, start=None, h0=1e-3, doubling=True, equilibrium=0.0, absolute=1e-6, floor=False,
            max_steps=1000, pcg=True, rtol=1e-6, maxit=2000, progress=False, predicted_start=False, budget_s=0.0):
        x = np.zeros(3 * self.V)
        stats = np.zeros(9)
        s = None if start is None else ptr(np.ascontiguousarray(start, dtype=np.float64))
        if self.lib.oracle_ptc(P(self.h), s, h0, int(doubling), equilibrium, absolute, int(floor), max_steps,
                               int(pcg), rtol, maxit, int(progress), int(predicted_start), budget_s, ptr(x),
                               ptr(stats)):
            raise RuntimeError(self.lib.oracle_last_error().decode())
        keys = ["steps", "newton", "rejected", "pcg", "final_residual", "final_h", "seconds", "converged", "reason"]
        return x, dict(zip(keys, stats.tolist()))


def pcg(row_ptr, col_idx, vals, rhs, tol, maxit, replace_every=0, replace_above=0.0, single=False,
        detect_breakdown=False):
    lib = load()
    rows = len(row_ptr) - 1
    x = np.zeros(3 * rows)
    info = np.zeros(4)
    lib.oracle_pcg(rows, ptr(np.ascontiguousarray(row_ptr, np.int32)), ptr(np.ascontiguousarray(col_idx, np.int32)),
                   ptr(np.ascontiguousarray(vals, np.float64)), ptr(np.ascontiguousarray(rhs, np.float64)), tol,
                   maxit, replace_every, replace_above, int(single), int(detect_breakdown), ptr(x), ptr(info))
    return x, {"iterations": int(info[0]), "converged": bool(info[1]), "breakdown": bool(info[2]),
               "relative": float(info[3])}


def linear_case(kind, columns):
    lib = load()
    k = {"tension": 0, "slack": 1, "dynamic": 2}[kind]
    sz = np.zeros(2, np.int64)
    lib.oracle_case_sizes(k, columns, ptr(sz))
    R, B = int(sz[0]), int(sz[1])
    rp, ci = np.zeros(R + 1, np.int32), np.zeros(B, np.int32)
    vals, rhs = np.zeros(9 * B), np.zeros(3 * R)
    lib.oracle_case_build(k, columns, ptr(rp), ptr(ci), ptr(vals), ptr(rhs))
    return rp, ci, vals, rhs


def bandwidth(row_ptr, col_idx):
    return load().oracle_band_bandwidth(len(row_ptr) - 1, ptr(row_ptr), ptr(col_idx))
