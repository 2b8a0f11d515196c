"""The reference comparer's replays of a GPU run's record tables, restated in Python (test checker only): the
Eisenstat-Walker forcing replay (engine/oracle/src/e4_compare.rs:87-95 with e4_rules.rs:8-30), the PTC step-size
controller replay (e7_compare.rs:111-121), the rejection replay (e7_compare.rs:128-136) and the probe replays:
alpha_max (e5_compare.rs:70-101), resolution (e5_compare.rs:103-110) and line-search acceptance
(e6_compare.rs:40-62). The tables are the
gpu-<mode>/ files the `drape` command writes (gpu-iterations.bin, gpu-robust.bin by the names in gpu-result.json's
"robust_fields", gpu-attempts.bin, gpu-ptc.bin)."""
import json
import os

import numpy as np

ETA_START = 1e-2
CONTROLLER_TOLERANCE = 1e-12


def next_forcing(previous, ratio):
    """e4_rules.rs:8-20: 0.9 (|g_k| / |g_k-1|)^2, safeguarded by 0.9 eta_k-1^2 when that exceeds 0.1, in [1e-7, 1e-2]."""
    eta = 0.9 * ratio * ratio
    safeguard = 0.9 * previous * previous
    guarded = max(eta, safeguard) if safeguard > 0.1 else eta
    return min(max(guarded, 1e-7), 1e-2)


def forcing_sequence(norms):
    out, eta = [], ETA_START
    for k, norm in enumerate(norms):
        if k > 0:
            eta = next_forcing(eta, norm / norms[k - 1])
        out.append(eta)
    return out


def read_run(out_dir):
    res = json.load(open(os.path.join(out_dir, "gpu-result.json")))
    fields = res["robust_fields"]
    it = np.fromfile(os.path.join(out_dir, "gpu-iterations.bin"), np.float64).reshape(-1, 9)
    rb = np.fromfile(os.path.join(out_dir, "gpu-robust.bin"), np.float64).reshape(-1, len(fields))
    at = np.fromfile(os.path.join(out_dir, "gpu-attempts.bin"), np.float64).reshape(-1, 6)
    ptc = np.fromfile(os.path.join(out_dir, "gpu-ptc.bin"), np.float64).reshape(-1, 7)
    return res, fields, it, rb, at, ptc


def forcing_replay(it, rb, fields, at):
    """Largest relative gap between each attempt's recorded eta and the rule replayed on its recorded residuals."""
    eta_col = fields.index("eta")
    worst = 0.0
    for a in at:
        seg = slice(int(a[4]), int(a[5]))
        updates = np.isfinite(it[seg, 3])
        norms = it[seg, 2][updates]
        etas = rb[seg, eta_col][updates]
        for got, want in zip(etas, forcing_sequence(list(norms))):
            worst = max(worst, abs((got - want) / want))
    return worst


def controller_replay(problem, ptc):
    """h_k+1 = clamp(h_k x growth (inner below the cap) or x shrink) x shrink^rejections of step k+1, floored."""
    p = problem["ptc"]
    growth, shrink, cap = p["growth"], p["shrink"], p["inner_max_iterations"]
    floor, top = p["h0"] * p["h_min_factor"], p["h_max"]
    for prev, row in zip(ptc[:-1], ptc[1:]):
        factor = growth if prev[3] < cap else shrink
        base = min(max(prev[1] * factor, floor), top)
        expected = max(base * shrink ** int(row[4]), floor)
        if abs((row[1] - expected) / expected) > CONTROLLER_TOLERANCE:
            return False
    return True


def rejection_replay(it, at):
    """A rejected attempt made no update and ended on the mu cap (reason 1, status 5) or a failed line search
    (reason 2, status 3); reasons 3 (non-finite) and 4 (curvature retry) need nothing more."""
    for a in at[at[:, 3] != 0]:
        seg = it[int(a[4]):int(a[5])]
        updates = int(((seg[:, 8] == 0) & np.isfinite(seg[:, 3])).sum())
        last = seg[-1, 8] if len(seg) else np.nan
        ok = a[3] in (3, 4) or (updates == 0 and ((a[3] == 1 and last == 5) or (a[3] == 2 and last == 3)))
        if not ok:
            return False
    return True


def f32_spacing(max_abs):
    """e4_rules.rs:35-39: 2^(exponent of max_abs as f32 - 23)."""
    bits = int(np.array([max_abs], np.float32).view(np.uint32)[0])
    return 2.0 ** (((bits >> 23) & 0xFF) - 127 - 23)


def resolution_replay(it, rb, fields, iterates, free_rows):
    """Every probe update's recorded resolution equals f32_spacing(max |x_i|) over the free vertices' coordinates."""
    col = fields.index("resolution")
    for k, x in enumerate(iterates):
        if not np.isfinite(it[k, 3]):
            continue
        largest = np.abs(x.reshape(-1, 3)[free_rows]).max()
        if f32_spacing(float(largest)) != rb[k, col]:
            return False
    return True


def alpha_errors(it, rb, fields, directions, max_step):
    """Relative errors of the recorded alpha_max against the f64 CCD rule `max_step(x, d)` at each update's recorded
    f32 (x, d) pair (the reference's tolerance is max(1e-5, 8 eps32 cond) with cond the limiting sphere's |q|/d0)."""
    col = fields.index("alphaMax")
    updates = np.flatnonzero(np.isfinite(it[:, 3]))
    assert len(updates) == len(directions), (len(updates), len(directions))
    return [abs(max_step(pair[0].astype(np.float64), pair[1].astype(np.float64)) - rb[k, col]) / rb[k, col]
            for k, pair in zip(updates, directions)]


def acceptance_replay(trials, armijo):
    """Each trial's accept decision replayed from its recorded numbers: plain Armijo sum <= f32(c alpha g.d) (the
    noise term needs the absolute change sum, which this solver does not record)."""
    plain = (armijo * trials[:, 3] * trials[:, 6]).astype(np.float32).astype(np.float64)
    return bool(np.all((trials[:, 4] <= plain) == (trials[:, 7] == 1.0)))
