"""The reference comparer's replays of a GPU run's record tables, restated in Python (test checker only): the
Eisenstat-Walker forcing replay (engine/oracle/src/e4_compare.rs:87-95 with e4_rules.rs:8-30), the PTC step-size
controller replay (e7_compare.rs:111-121) and the rejection replay (e7_compare.rs:128-136). The tables are the
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
