"""Python view of libdrape_b200.so (the C ABI in include/drape_b200.h) through ctypes.

The names follow the reference's GPU stage: ``solve_equilibrium`` (drape-e7.ts:156-180), the kernel checks
(run-e7.ts:140-145), ``pcg`` (solver.ts:179-191). The product path is the CUDA library only: importing this module
raises when the shared object is missing, and there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libdrape_b200.so")
P = ctypes.c_void_p
_lib = None

STATUS = {0: "ok", 1: "invalid argument", 2: "cuda error", 3: "diverged", 4: "timeout", 5: "io error", 6: "bad state"}
REASON = {0: "tolerance", 1: "cap", 2: "stalled", 3: "time_budget"}
PCG_STATUS = {0: "running", 1: "converged", 2: "iteration_limit", 3: "breakdown", 4: "timeout"}


class DrapeError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [
        ("controller", ctypes.c_int32), ("h0", ctypes.c_double), ("h_max", ctypes.c_double),
        ("h_min_factor", ctypes.c_double), ("growth", ctypes.c_double), ("shrink", ctypes.c_double),
        ("inner_tolerance", ctypes.c_double), ("inner_max", ctypes.c_int32), ("max_rejections", ctypes.c_int32),
        ("max_steps", ctypes.c_int32), ("equilibrium_relative", ctypes.c_double),
        ("equilibrium_absolute", ctypes.c_double), ("pcg_rtol", ctypes.c_double),
        ("pcg_max_iterations", ctypes.c_int32), ("forcing", ctypes.c_int32), ("replace_every", ctypes.c_int32),
        ("replace_above", ctypes.c_double), ("refine", ctypes.c_int32), ("refine_rtol", ctypes.c_double),
        ("curvature", ctypes.c_int32), ("preconditioner", ctypes.c_int32), ("armijo", ctypes.c_double),
        ("max_halvings", ctypes.c_int32), ("time_budget_s", ctypes.c_double), ("pcg_grid", ctypes.c_int32),
        ("pcg_threads", ctypes.c_int32), ("pcg_lanes", ctypes.c_int32), ("progress", ctypes.c_int32),
        ("newton_start", ctypes.c_int32), ("tangent", ctypes.c_int32), ("smoother_omega", ctypes.c_double),
        ("prolongation", ctypes.c_int32), ("pcg_single_reduction", ctypes.c_int32),
    ]


class RunLog(ctypes.Structure):
    _fields_ = [
        ("ptc_steps", ctypes.c_int32), ("newton_iterations", ctypes.c_int32), ("pcg_iterations", ctypes.c_int32),
        ("rejected_attempts", ctypes.c_int32), ("mu_retries", ctypes.c_int32), ("reason", ctypes.c_int32),
        ("final_residual", ctypes.c_double), ("final_relative_residual", ctypes.c_double),
        ("final_h", ctypes.c_double), ("gravity_load", ctypes.c_double), ("static_energy", ctypes.c_double),
        ("seconds", ctypes.c_double), ("ms_assembly", ctypes.c_double), ("ms_pcg", ctypes.c_double),
        ("ms_line_search", ctypes.c_double), ("ms_ccd", ctypes.c_double), ("ms_other", ctypes.c_double),
        ("pcg_launches", ctypes.c_int32), ("pcg_grid", ctypes.c_int32), ("device_seconds", ctypes.c_double),
        ("kernel_launches", ctypes.c_int32), ("fallbacks", ctypes.c_int32), ("mg_levels", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["reason"] = REASON.get(self.reason, str(self.reason))
        return d


class ProblemView(ctypes.Structure):
    _fields_ = [
        ("columns", ctypes.c_int32), ("vertices", ctypes.c_int32), ("triangles", ctypes.c_int32),
        ("hinges", ctypes.c_int32), ("rows", ctypes.c_int32), ("blocks", ctypes.c_int32),
        ("start_xyz", P), ("elem_vertices", P), ("elem_geom", P), ("hinge_vertices", P), ("hinge_stiffness", P),
        ("row_vertex", P), ("row_unit_mass", P), ("row_ptr", P), ("col_idx", P),
        ("wale", ctypes.c_double), ("course", ctypes.c_double), ("coupling", ctypes.c_double),
        ("shear", ctypes.c_double), ("gravity", ctypes.c_double * 3), ("colliders", ctypes.c_int32),
        ("collider_data", P), ("dhat", ctypes.c_double), ("kappa", ctypes.c_double),
    ]


class TimeStepLog(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("status", ctypes.c_int32), ("pcg_iterations", ctypes.c_int32),
                ("mu_retries", ctypes.c_int32), ("scale", ctypes.c_double), ("final_relative_residual", ctypes.c_double),
                ("max_mu", ctypes.c_double), ("seconds", ctypes.c_double)]


STEP_STATUS = {1: "converged", 2: "iteration_limit", 3: "line_search_failed", 5: "regularization_cap", 6: "non_finite"}


class StepRecord(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int32), ("inner", ctypes.c_int32), ("rejected", ctypes.c_int32),
                ("pcg_iterations", ctypes.c_int32), ("h", ctypes.c_double), ("residual", ctypes.c_double),
                ("min_distance", ctypes.c_double), ("seconds", ctypes.c_double)]


class NewtonRecord(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("step", "iteration", "pcg_iterations", "pcg_status", "halvings",
                                              "status", "retries", "pad")] + \
               [(k, ctypes.c_double) for k in ("relative_residual", "linear_residual", "step_length", "eta", "mu",
                                               "alpha_max", "delta_sum", "slope", "norm_squared", "resolution")]


class AttemptRecord(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("step", "attempt", "reason", "record_start", "record_end", "pad")] + \
               [("h", ctypes.c_double)]


def load():
    """Loads the CUDA library (raises if it has not been built: `python -m drape_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m drape_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    lib.drape_version.restype = ctypes.c_char_p
    lib.drape_last_error.restype = ctypes.c_char_p
    lib.drape_last_error.argtypes = [P]
    lib.drape_default_options.argtypes = [ctypes.POINTER(Options)]
    lib.drape_create_sheet.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, ctypes.POINTER(Options), ctypes.c_int32, ctypes.POINTER(P)]
    lib.drape_create_reference.argtypes = [ctypes.c_int32, ctypes.c_char_p, ctypes.POINTER(Options), ctypes.c_int32,
                                           ctypes.POINTER(P)]
    lib.drape_create_from_files.argtypes = [ctypes.c_char_p, ctypes.POINTER(Options), ctypes.c_int32, ctypes.POINTER(P)]
    lib.drape_destroy.argtypes = [P]
    lib.drape_sizes.argtypes = [P, P]
    lib.drape_set_options.argtypes = [P, ctypes.POINTER(Options)]
    lib.drape_set_state.argtypes = [P, P]
    lib.drape_get_state.argtypes = [P, P, P]
    lib.drape_solve_equilibrium.argtypes = [P, P, ctypes.c_double, ctypes.POINTER(RunLog)]
    lib.drape_step_records.argtypes = [P, P, ctypes.c_int32, P]
    lib.drape_assemble.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, P, P]
    lib.drape_pcg.argtypes = [P, P, P, ctypes.c_double, ctypes.c_int32, P, P, P]
    lib.drape_precondition.argtypes = [P, P, P, P]
    lib.drape_network_create.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(P)]
    lib.drape_network_destroy.argtypes = [P]
    lib.drape_network_load.argtypes = [P, ctypes.c_char_p]
    lib.drape_network_save.argtypes = [P, ctypes.c_char_p]
    lib.drape_network_parameters.argtypes = [P, P, P]
    lib.drape_set_network.argtypes = [P, P]
    lib.drape_network_gradient.argtypes = [P, P, P, P, P, P, P, P]
    lib.drape_network_train.argtypes = [P, P, ctypes.c_int32, P, P, P, ctypes.c_int32, ctypes.c_double, P]
    lib.drape_multilevel_view.argtypes = [P, ctypes.c_int32, P, P, P, P]
    lib.drape_time_step.argtypes = [P, ctypes.c_double, P, ctypes.c_double, ctypes.c_int32, P, P]
    lib.drape_energy_change.argtypes = [P, P, P, ctypes.c_double, P, ctypes.c_double, ctypes.c_int32, P]
    lib.drape_max_step.argtypes = [P, P, P, P]
    lib.drape_static_residual.argtypes = [P, P, P]
    lib.drape_static_energy.argtypes = [P, P, P]
    lib.drape_time_spmv.argtypes = [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P]
    lib.drape_time_assembly.argtypes = [P, ctypes.c_int32, P]
    lib.drape_pcg_profile.argtypes = [P, P, ctypes.c_int32]
    lib.drape_create.argtypes = [ctypes.POINTER(ProblemView), ctypes.POINTER(Options), ctypes.c_int32, ctypes.POINTER(P)]
    lib.drape_write_sheet_problem.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int32, ctypes.c_char_p]
    lib.drape_write_reference_problem.argtypes = [ctypes.c_int32, ctypes.c_char_p, ctypes.c_char_p]
    lib.drape_inspect_problem.argtypes = [ctypes.c_char_p, P]
    _lib = lib
    return lib


def default_options(**overrides):
    o = Options()
    load().drape_default_options(ctypes.byref(o))
    for k, v in overrides.items():
        if not hasattr(o, k):
            raise AttributeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def _ptr(a):
    return a.ctypes.data_as(P) if a is not None else None


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Drape:
    """One drape context on one GPU (``drape_ctx``)."""

    def __init__(self, handle):
        self.lib = load()
        self.h = handle
        sz = np.zeros(6, np.int64)
        self._check(self.lib.drape_sizes(self.h, _ptr(sz)))
        self.V, self.T, self.H, self.R, self.B, self.colliders = (int(v) for v in sz)

    @classmethod
    def _create(cls, fn, *args, options=None, device=0):
        lib = load()
        h = P()
        st = fn(*args, ctypes.byref(options) if options is not None else None, device, ctypes.byref(h))
        if st != 0:
            raise DrapeError(st, lib.drape_last_error(None).decode())
        return cls(h)

    @classmethod
    def sheet(cls, columns, seed=0, radius=0.25, young=5e5, plane=False, options=None, device=0):
        return cls._create(load().drape_create_sheet, columns, seed, radius, young, int(plane), options=options,
                           device=device)

    @classmethod
    def reference(cls, columns, edit="base", options=None, device=0):
        return cls._create(load().drape_create_reference, columns, edit.encode(), options=options, device=device)

    @classmethod
    def from_files(cls, directory, options=None, device=0):
        return cls._create(load().drape_create_from_files, os.fsencode(directory), options=options, device=device)

    @classmethod
    def from_arrays(cls, start, row_vertex, unit_mass, row_ptr, col_idx, tri=None, geom=None, hinge=None,
                    hinge_k=None, material=(0.0, 0.0, 0.0, 0.0), gravity=(0.0, 0.0, -9.81), colliders=None,
                    dhat=0.0, kappa=0.0, columns=0, options=None, device=0):
        """A context over caller-owned arrays (the drape_problem_view of the C ABI)."""
        keep = {
            "start": _f64(start), "row_vertex": np.ascontiguousarray(row_vertex, np.uint32),
            "mass": _f64(unit_mass), "row_ptr": np.ascontiguousarray(row_ptr, np.uint32),
            "col_idx": np.ascontiguousarray(col_idx, np.uint32),
            "tri": np.ascontiguousarray(tri if tri is not None else np.zeros(0), np.uint32),
            "geom": _f64(geom if geom is not None else np.zeros(0)),
            "hinge": np.ascontiguousarray(hinge if hinge is not None else np.zeros(0), np.uint32),
            "hinge_k": _f64(hinge_k if hinge_k is not None else np.zeros(0)),
            "colliders": _f64(colliders if colliders is not None else np.zeros(0)),
        }
        v = ProblemView()
        v.columns = columns
        v.vertices = len(keep["start"]) // 3
        v.triangles = len(keep["tri"]) // 3
        v.hinges = len(keep["hinge"]) // 4
        v.rows = len(keep["row_vertex"])
        v.blocks = len(keep["col_idx"])
        v.start_xyz, v.row_vertex, v.row_unit_mass = _ptr(keep["start"]), _ptr(keep["row_vertex"]), _ptr(keep["mass"])
        v.row_ptr, v.col_idx = _ptr(keep["row_ptr"]), _ptr(keep["col_idx"])
        v.elem_vertices, v.elem_geom = _ptr(keep["tri"]), _ptr(keep["geom"])
        v.hinge_vertices, v.hinge_stiffness = _ptr(keep["hinge"]), _ptr(keep["hinge_k"])
        v.wale, v.course, v.coupling, v.shear = material
        v.gravity[:] = list(gravity)
        v.colliders = len(keep["colliders"]) // 8
        v.collider_data = _ptr(keep["colliders"])
        v.dhat, v.kappa = dhat, kappa
        return cls._create(load().drape_create, ctypes.byref(v), options=options, device=device)

    def close(self):
        if self.h:
            self.lib.drape_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st):
        if st != 0:
            raise DrapeError(st, self.lib.drape_last_error(self.h).decode())

    def set_options(self, options):
        self._check(self.lib.drape_set_options(self.h, ctypes.byref(options)))

    @property
    def state(self):
        x = np.zeros(3 * self.V)
        self._check(self.lib.drape_get_state(self.h, _ptr(x), None))
        return x

    @state.setter
    def state(self, xyz):
        self._check(self.lib.drape_set_state(self.h, _ptr(_f64(xyz))))

    def final_h(self):
        h = ctypes.c_double()
        self._check(self.lib.drape_get_state(self.h, None, ctypes.byref(h)))
        return h.value

    def solve_equilibrium(self, start=None, h0=0.0, check=True):
        log = RunLog()
        st = self.lib.drape_solve_equilibrium(self.h, _ptr(_f64(start)), h0, ctypes.byref(log))
        if check:
            self._check(st)
        out = log.as_dict()
        out["status"] = st
        return out

    def time_step(self, h, velocity=None, tolerance=1e-8, max_iterations=30):
        """One backward-Euler step (drape_time_step) from the current state with `velocity` (3V, None: at rest):
        returns (new velocity, log dict); the context's state advances."""
        v_out = np.zeros(3 * self.V)
        log = TimeStepLog()
        v = _f64(velocity)
        self._check(self.lib.drape_time_step(self.h, ctypes.c_double(h), _ptr(v), ctypes.c_double(tolerance),
                                             max_iterations, _ptr(v_out), ctypes.byref(log)))
        d = {k: getattr(log, k) for k, _ in TimeStepLog._fields_}
        d["status_name"] = STEP_STATUS.get(d["status"], "unknown")
        return v_out, d

    def step_records(self):
        n = ctypes.c_int32()
        self._check(self.lib.drape_step_records(self.h, None, 0, ctypes.byref(n)))
        recs = (StepRecord * max(n.value, 1))()
        self._check(self.lib.drape_step_records(self.h, recs, n.value, ctypes.byref(n)))
        return [{k: getattr(r, k) for k, _ in StepRecord._fields_} for r in recs[: n.value]]

    def _records(self, fn, cls):
        fn.argtypes = [P, P, ctypes.c_int32, P]
        n = ctypes.c_int32()
        self._check(fn(self.h, None, 0, ctypes.byref(n)))
        recs = (cls * max(n.value, 1))()
        self._check(fn(self.h, recs, n.value, ctypes.byref(n)))
        return [{k: getattr(r, k) for k, _ in cls._fields_ if k != "pad"} for r in recs[: n.value]]

    def newton_records(self):
        """The last solve's Newton iterates (drape_newton_records; gpu-iterations.bin / gpu-robust.bin rows)."""
        return self._records(self.lib.drape_newton_records, NewtonRecord)

    def attempt_records(self):
        """The last solve's attempts (drape_attempt_records; gpu-attempts.bin rows)."""
        return self._records(self.lib.drape_attempt_records, AttemptRecord)

    def keep_states(self, keep=True):
        """Later solves keep every accepted state (drape_keep_states); step_states() returns them, [steps, 3V] f32."""
        self.lib.drape_keep_states.argtypes = [P, ctypes.c_int32]
        self._check(self.lib.drape_keep_states(self.h, int(keep)))

    def step_states(self):
        fn = self.lib.drape_step_states
        fn.argtypes = [P, P, ctypes.c_int64, P]
        n = ctypes.c_int64()
        self._check(fn(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._check(fn(self.h, _ptr(out), n.value, ctypes.byref(n)))
        return out.reshape(-1, 3 * self.V)

    def probe(self, probes):
        """PTC probes (drape_probe_begin / drape_probe_step): one logged Newton attempt per (step, h, positions).
        Returns (Newton records, iterates [n, 3V] f32, direction pairs [m, 2, 3V] f32, trials [k, 8] f64)."""
        lib = self.lib
        lib.drape_probe_begin.argtypes = [P]
        lib.drape_probe_step.argtypes = [P, P, ctypes.c_double, ctypes.c_int32]
        lib.drape_probe_logs.argtypes = [P, P, ctypes.c_int64, P, P, ctypes.c_int64, P, P, ctypes.c_int64, P]
        self._check(lib.drape_probe_begin(self.h))
        for step, h, x in probes:
            self._check(lib.drape_probe_step(self.h, _ptr(_f64(x)), h, int(step)))
        ni, nd, nt = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(lib.drape_probe_logs(self.h, None, 0, ctypes.byref(ni), None, 0, ctypes.byref(nd), None, 0,
                                         ctypes.byref(nt)))
        it, dr, tr = np.zeros(ni.value, np.float32), np.zeros(nd.value, np.float32), np.zeros(nt.value)
        self._check(lib.drape_probe_logs(self.h, _ptr(it), ni.value, ctypes.byref(ni), _ptr(dr), nd.value,
                                         ctypes.byref(nd), _ptr(tr), nt.value, ctypes.byref(nt)))
        return (self.newton_records(), it.reshape(-1, 3 * self.V), dr.reshape(-1, 2, 3 * self.V),
                tr.reshape(-1, 8))

    def assemble(self, x, x_hat=None, h=0.0, mu=0.0, mode=0, curvature=False, blocks=True):
        g = np.zeros(3 * self.R)
        b = np.zeros(9 * self.B, np.float32) if blocks else None
        self._check(self.lib.drape_assemble(self.h, _ptr(_f64(x)), _ptr(_f64(x_hat)), h, mu, mode, int(curvature),
                                            _ptr(g), _ptr(b)))
        return g, b

    def pcg(self, rhs, rtol, max_iterations, blocks=None):
        sol = np.zeros(3 * self.R)
        info = np.zeros(3, np.int32)
        rel = ctypes.c_double()
        blk = None if blocks is None else np.ascontiguousarray(blocks, np.float32)
        self._check(self.lib.drape_pcg(self.h, _ptr(blk), _ptr(_f64(rhs)), rtol, max_iterations, _ptr(sol), _ptr(info),
                                       ctypes.byref(rel)))
        return sol, {"iterations": int(info[0]), "status": PCG_STATUS.get(int(info[1]), int(info[1])),
                     "replacements": int(info[2]), "relative": rel.value}

    def set_network(self, network):
        """Attach the network preconditioner 2 uses (kept alive by this object)."""
        self._network = network
        self._check(self.lib.drape_set_network(self.h, network.h if network is not None else None))

    def precondition(self, r, blocks=None):
        """One multilevel V-cycle z = M r (the preconditioner of options.preconditioner 1 and 2)."""
        z = np.zeros(3 * self.R)
        blk = None if blocks is None else np.ascontiguousarray(blocks, np.float32)
        self._check(self.lib.drape_precondition(self.h, _ptr(blk), _ptr(_f64(r)), _ptr(z)))
        return z

    def multilevel_view(self, level, operator=True, width=False):
        """(columns, f64 stencil [w^2 * 9][rows] or None, f32 smoother [9][rows]) of one hierarchy level, w its
        stencil width (5, or 7 for level 1 under the smoothed prolongation); with width=True also w."""
        cols, w = ctypes.c_int32(), ctypes.c_int32()
        self._check(self.lib.drape_multilevel_view(self.h, level, ctypes.byref(cols), ctypes.byref(w), None, None))
        n = cols.value
        op = np.zeros((w.value * w.value * 9, n * n)) if operator and level > 0 else None
        sm = np.zeros((9, n * n), np.float32)
        self._check(self.lib.drape_multilevel_view(self.h, level, ctypes.byref(cols), ctypes.byref(w), _ptr(op),
                                                   _ptr(sm)))
        return (n, op, sm, w.value) if width else (n, op, sm)

    def energy_change(self, x, d, alpha, x_hat=None, h=0.0, mode=0):
        out = ctypes.c_double()
        self._check(self.lib.drape_energy_change(self.h, _ptr(_f64(x)), _ptr(_f64(x_hat)), h, _ptr(_f64(d)), alpha,
                                                 mode, ctypes.byref(out)))
        return out.value

    def max_step(self, x, d):
        out = ctypes.c_double()
        self._check(self.lib.drape_max_step(self.h, _ptr(_f64(x)), _ptr(_f64(d)), ctypes.byref(out)))
        return out.value

    def element_terms(self, x, exact=True):
        """(grad [9T + 12H], hess [81T + 144H]) f32 element terms at x in the reference's per-element layout."""
        fn = self.lib.drape_element_terms
        fn.argtypes = [P, P, ctypes.c_int32, P, P]
        g = np.zeros(9 * self.T + 12 * self.H, np.float32)
        hs = np.zeros(81 * self.T + 144 * self.H, np.float32)
        self._check(fn(self.h, _ptr(_f64(x)), int(exact), _ptr(g), _ptr(hs)))
        return g, hs

    def row_terms(self, x, x_hat, row_mass=None, mu=0.0, contact=False, curvature=True):
        """(grad [3R], hess [9R]) f32 per-row inertia (row_mass: mass over h^2 per row) and barrier terms."""
        fn = self.lib.drape_row_terms
        fn.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, P, P]
        g = np.zeros(3 * self.R, np.float32)
        hs = np.zeros(9 * self.R, np.float32)
        self._check(fn(self.h, _ptr(_f64(x)), _ptr(_f64(x_hat)), _ptr(_f64(row_mass)), mu, int(contact), int(curvature),
                       _ptr(g), _ptr(hs)))
        return g, hs

    def static_residual(self, x=None):
        out = ctypes.c_double()
        self._check(self.lib.drape_static_residual(self.h, _ptr(_f64(x)), ctypes.byref(out)))
        return out.value

    def static_energy(self, x=None):
        out = ctypes.c_double()
        self._check(self.lib.drape_static_energy(self.h, _ptr(_f64(x)), ctypes.byref(out)))
        return out.value

    def time_spmv(self, launches=100, lanes_per_row=8, threads=256):
        ms = ctypes.c_float()
        self._check(self.lib.drape_time_spmv(self.h, launches, lanes_per_row, threads, ctypes.byref(ms)))
        return ms.value

    def pcg_profile(self, clear=False):
        """CTA 0's SM cycles per PCG phase: phase A, sum A, barrier A, phase B, sum B, barrier B, iterations."""
        out = np.zeros(7, np.int64)
        self._check(self.lib.drape_pcg_profile(self.h, _ptr(out), int(clear)))
        keys = ["phase_a", "sum_a", "barrier_a", "phase_b", "sum_b", "barrier_b", "iterations"]
        return dict(zip(keys, out.tolist()))

    def time_assembly(self, launches=50):
        ms = ctypes.c_float()
        self._check(self.lib.drape_time_assembly(self.h, launches, ctypes.byref(ms)))
        return ms.value


def version():
    return load().drape_version().decode()


def _host_call(st):
    if st != 0:
        raise DrapeError(st, load().drape_last_error(None).decode())


def spmv_benchmark(row_ptr, col_idx, values, x, launches=20, lanes_per_row=8, threads=256, device=0, result=False):
    """Device ms per launch of the BSR(3x3) SpMV on the given matrix (and y = A x if `result`)."""
    lib = load()
    lib.drape_spmv_benchmark.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, P, P, P, P, ctypes.c_int32,
                                         ctypes.c_int32, ctypes.c_int32, P, P]
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    vals = np.ascontiguousarray(values, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    y = np.zeros(3 * (len(rp) - 1), np.float32) if result else None
    ms = ctypes.c_float()
    st = lib.drape_spmv_benchmark(device, len(rp) - 1, len(ci), _ptr(rp), _ptr(ci), _ptr(vals), _ptr(xx), launches,
                                  lanes_per_row, threads, _ptr(y), ctypes.byref(ms))
    if st != 0:
        raise DrapeError(st, lib.drape_last_error(None).decode())
    return (ms.value, y) if result else ms.value


def solve_batch(drapes, workers=16, check=True):
    """Solves the drapes (distinct `Drape` objects) concurrently from their current states (drape_solve_batch):
    `workers` host threads, each solving one drape at a time on that drape's own stream. Returns (logs, seconds,
    total_seconds): one run-log dict per drape (with its "status"), each drape's host solve time, and the batch's."""
    lib = load()
    lib.drape_solve_batch.argtypes = [P, ctypes.c_int32, ctypes.c_int32, P, P, P, P]
    n = len(drapes)
    handles = (P * n)(*[d.h for d in drapes])
    logs = (RunLog * n)()
    status = np.zeros(n, np.int32)
    seconds = np.zeros(n, np.float64)
    total = ctypes.c_double()
    st = lib.drape_solve_batch(handles, n, workers, logs, _ptr(status), _ptr(seconds), ctypes.byref(total))
    if check and st != 0:
        raise DrapeError(st, lib.drape_last_error(None).decode())
    out = []
    for i in range(n):
        d = logs[i].as_dict()
        d["status"] = int(status[i])
        out.append(d)
    return out, seconds, total.value


NETWORK_PARAMETERS = 34177
NETWORK_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "preconditioner_network.bin")


class Network:
    """The preconditioner network (options.preconditioner = 2): a 4-layer mesh message-passing network that scales
    the multilevel preconditioner's fine Jacobi smoother per row. `Network.trained()` loads the shipped weights."""

    def __init__(self, seed=0, device=0, path=None):
        self.lib = load()
        h = P()
        if self.lib.drape_network_create(device, seed, ctypes.byref(h)) != 0:
            raise DrapeError(2, self.lib.drape_last_error(None).decode())
        self.h = h
        if path:
            self.load(path)

    @classmethod
    def trained(cls, device=0):
        return cls(device=device, path=NETWORK_FILE)

    def close(self):
        if getattr(self, "h", None):
            self.lib.drape_network_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, st, ctx=None):
        if st != 0:
            raise DrapeError(st, self.lib.drape_last_error(ctx).decode())

    def load(self, path):
        self._check(self.lib.drape_network_load(self.h, os.fsencode(path)))

    def save(self, path):
        self._check(self.lib.drape_network_save(self.h, os.fsencode(path)))

    @property
    def parameters(self):
        p = np.zeros(NETWORK_PARAMETERS, np.float32)
        self._check(self.lib.drape_network_parameters(self.h, _ptr(p), None))
        return p

    @parameters.setter
    def parameters(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == NETWORK_PARAMETERS
        self._check(self.lib.drape_network_parameters(self.h, None, _ptr(p)))

    def gradient(self, drape, blocks, rhs, solution):
        """(loss, gradient, factors) of one (blocks, rhs, solution) tuple on the drape's pattern."""
        grad = np.zeros(NETWORK_PARAMETERS, np.float32)
        fac = np.zeros(drape.R, np.float32)
        loss = ctypes.c_double()
        blk = np.ascontiguousarray(blocks, np.float32)
        self._check(self.lib.drape_network_gradient(drape.h, self.h, _ptr(blk), _ptr(_f64(rhs)), _ptr(_f64(solution)),
                                                    ctypes.byref(loss), _ptr(grad), _ptr(fac)), drape.h)
        return loss.value, grad, fac

    def train(self, drape, tuples, steps, lr=1e-3):
        """Adam over [(blocks, rhs, solution), ...] of the drape's pattern; returns the per-step losses."""
        keep = [(np.ascontiguousarray(b, np.float32), _f64(r), _f64(x)) for b, r, x in tuples]
        n = len(keep)
        B = (P * n)(*[_ptr(k[0]) for k in keep])
        Rr = (P * n)(*[_ptr(k[1]) for k in keep])
        X = (P * n)(*[_ptr(k[2]) for k in keep])
        losses = np.zeros(steps)
        self._check(self.lib.drape_network_train(drape.h, self.h, n, B, Rr, X, steps, lr, _ptr(losses)), drape.h)
        return losses


def write_sheet_problem(directory, columns, seed=0, radius=0.25, young=5e5, plane=False):
    """problem.json / problem.bin of the sheet over a sphere (host only)."""
    _host_call(load().drape_write_sheet_problem(columns, seed, radius, young, int(plane), os.fsencode(directory)))


def write_reference_problem(directory, columns, edit="base"):
    """problem.json / problem.bin of the reference's sphere-on-floor scene (host only)."""
    _host_call(load().drape_write_reference_problem(columns, edit.encode(), os.fsencode(directory)))


def inspect_problem(directory):
    """Reads and validates a problem pair (host only): (V, T, H, R, B, colliders)."""
    sz = np.zeros(6, np.int64)
    _host_call(load().drape_inspect_problem(os.fsencode(directory), _ptr(sz)))
    return tuple(int(v) for v in sz)


def read_problem_arrays(directory):
    """The arrays of a problem.bin as numpy arrays, keyed by manifest name."""
    import json

    meta = json.load(open(os.path.join(directory, "problem.json")))
    raw = open(os.path.join(directory, "problem.bin"), "rb").read()
    out = {}
    for a in meta["arrays"]:
        dt = {"f32": np.float32, "f64": np.float64, "u32": np.uint32}[a["dtype"]]
        out[a["name"]] = np.frombuffer(raw, dt, a["length"], a["offset"]).copy()
    return meta, out
