"""The restated comparer replays (tests/e7_replays.py) on small hand-made record tables: tables that follow the
reference's rules pass, and each planted rule violation is caught."""
import numpy as np

from tests import e7_replays as rp

FIELDS = ["eta", "mu", "updateInf", "stepInf", "retries", "resolution", "alphaMax", "limitingVertex", "minDistance",
          "deltaSum", "deltaAbs", "noiseOnly", "slope", "slopeExact", "normSquared", "normSquaredExact"]
PROBLEM = {"ptc": {"growth": 2.0, "shrink": 0.5, "inner_max_iterations": 10, "h0": 1e-3, "h_min_factor": 1e-6,
                   "h_max": 1e6}}


def _tables():
    """Two accepted steps (3 updates then converged; 1 update then converged) and one rejected attempt (a failed
    line search before any update) between them."""
    rel = [1.0, 0.1, 0.02, 1e-4, 1.0, 3e-4, 1.0, 1e-3, 1e-9]
    rows = [(1, 0, 0), (1, 1, 0), (1, 2, 0), (1, 3, 1),  # step 1: updates, then converged
            (2, 0, 3),                                  # step 2, attempt 0: line search failed, no update
            (2, 0, 0), (2, 1, 1)]                       # step 2, attempt 1
    it = np.full((len(rows), 9), np.nan)
    rb = np.full((len(rows), 16), np.nan)
    for k, (step, i, status) in enumerate(rows):
        it[k, 0], it[k, 1], it[k, 2], it[k, 8] = step, i, rel[k], status
        solved = status != 1
        if solved:
            it[k, 3] = 10
    at = np.array([[1, 0, 1e-3, 0, 0, 4], [2, 0, 2e-3, 2, 4, 5], [2, 1, 1e-3, 0, 5, 7]], float)
    for a in at:
        seg = slice(int(a[4]), int(a[5]))
        solved = np.isfinite(it[seg, 3])
        idx = np.arange(int(a[4]), int(a[5]))[solved]
        for k, eta in zip(idx, rp.forcing_sequence(list(it[idx, 2]))):
            rb[k, 0] = eta
    # gpu-ptc rows: step, h, residual, inner, rejected, pcg, min distance; h_2 = 2 h_1 x shrink^1
    ptc = np.array([[1, 1e-3, 1.0, 3, 0, 30, 0.01], [2, 1e-3, 0.5, 1, 1, 20, 0.01]])
    return it, rb, at, ptc


def test_tables_that_follow_the_rules_pass():
    it, rb, at, ptc = _tables()
    assert rp.forcing_replay(it, rb, FIELDS, at) <= 1e-12
    assert rp.controller_replay(PROBLEM, ptc)
    assert rp.rejection_replay(it, at)


def test_planted_violations_are_caught():
    it, rb, at, ptc = _tables()
    bad = rb.copy()
    bad[1, 0] *= 1.001
    assert rp.forcing_replay(it, bad, FIELDS, at) > 1e-5
    ptc_bad = ptc.copy()
    ptc_bad[1, 1] *= 2
    assert not rp.controller_replay(PROBLEM, ptc_bad)
    it_bad = it.copy()
    it_bad[4, 8] = 5  # a "line search failed" attempt whose last record is the mu cap
    assert not rp.rejection_replay(it_bad, at)


def test_forcing_rule_bounds():
    assert rp.next_forcing(1e-2, 1.0) == 1e-2  # capped above
    assert rp.next_forcing(1e-2, 1e-6) == 1e-7  # floored
    assert abs(rp.next_forcing(1e-2, 0.1) - 0.9 * 0.01) < 1e-18  # 0.9 ratio^2, no safeguard below 0.1
    assert rp.next_forcing(0.4, 1e-3) == 1e-2  # the safeguard 0.9 x 0.16 > 0.1 keeps eta up, then the cap


def test_probe_replays_on_made_up_records():
    """The probe replays (alpha, resolution, acceptance) pass on consistent made-up logs and catch planted errors."""
    V = 2
    x0 = np.array([0.1, 0.2, -0.3, 1.5, 0.0, 0.25], np.float32)
    x1 = np.array([0.1, 0.2, -0.3, 0.7, 0.0, 0.25], np.float32)
    d = np.full(6, 0.01, np.float32)
    it = np.full((3, 9), np.nan)
    it[:, 0] = 4
    it[:, 1] = [0, 1, 2]
    it[:2, 3] = 7  # two updates, the last iterate takes no solve
    fields = FIELDS
    rb = np.full((3, 16), np.nan)
    rb[0, 5] = rp.f32_spacing(1.5)
    rb[1, 5] = rp.f32_spacing(0.7)
    rb[:2, 6] = [0.5, 0.25]
    iterates = np.stack([x0, x1, x1])
    pairs = np.stack([np.stack([x0, d]), np.stack([x1, d])])
    free = np.arange(V)
    assert rp.f32_spacing(1.5) == 2.0 ** -23 and rp.f32_spacing(0.7) == 2.0 ** -24
    assert rp.resolution_replay(it, rb, fields, iterates, free)
    bad = rb.copy()
    bad[1, 5] *= 2
    assert not rp.resolution_replay(it, bad, fields, iterates, free)
    # alpha: the rule replayed exactly gives 0 error; a recorded alpha 1 % off is caught
    rule = {0: 0.5, 1: 0.25}
    calls = iter(range(2))
    errors = rp.alpha_errors(it, rb, fields, pairs, lambda x, dd: rule[next(calls)])
    assert max(errors) == 0.0
    calls = iter(range(2))
    off = rb.copy()
    off[1, 6] *= 1.01
    assert max(rp.alpha_errors(it, off, fields, pairs, lambda x, dd: rule[next(calls)])) > 1e-3
    # acceptance: sum <= f32(c alpha slope) decides; a flipped decision is caught
    trials = np.array([[4, 0, 0, 0.5, -1e-3, np.nan, -1.0, 1.0],
                       [4, 1, 0, 0.25, 1e-3, np.nan, -1.0, 0.0]])
    assert rp.acceptance_replay(trials, 1e-4)
    flipped = trials.copy()
    flipped[1, 7] = 1.0
    assert not rp.acceptance_replay(flipped, 1e-4)
