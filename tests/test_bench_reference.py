"""The reference arm's arithmetic in bench.py, on the CPU with a stand-in oracle: a bounded sample is scaled by the
oracle's own whole solve of the workload (its whole-solve seconds over its seconds to the sample's last step, from
the FULL_SOLVE record), never by a GPU solve's counts; with no record the whole solve is run and timed. The record
itself is parsed from the oracle's progress lines."""
import argparse
import json

import pytest

import bench
from tests import oracle_py


class FakeScene:
    budgets = []

    def __init__(self, *a, **k):
        pass

    def ptc(self, budget_s=0.0, **k):
        FakeScene.budgets.append(budget_s)
        if budget_s == 0.0:
            return None, {"steps": 400, "newton": 3000, "seconds": 3600.0, "converged": 1.0}
        return None, {"steps": 8, "newton": 16, "seconds": 20.0, "converged": 0.0}


RECORD = {"seconds": 4000.0, "steps": 410, "newton": 3300, "seconds_to_1e-6": 3800.0, "host": "a test host",
          "seconds_at_step": [1.0 * k for k in range(1, 21)]}


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(oracle_py, "Scene", FakeScene)
    monkeypatch.setattr(bench, "FULL_SOLVE", {(129, 1, 0, 1e-7): RECORD})
    FakeScene.budgets = []
    return argparse.Namespace(n=129, plane=1, seed=0, cpu_budget=20.0, absolute=1e-7)


def test_sample_is_scaled_by_the_oracle_whole_solve(fake):
    r = bench.cpu_baseline(fake)
    # 8 sampled steps took 20 s here; the recorded whole solve took 4000 s, 8 s of it to its 8th step.
    assert r["value"] == pytest.approx(20.0 * 4000.0 / 8.0)
    assert FakeScene.budgets == [20.0] and r["extrapolated"]
    assert r["whole_solve_measured"]["seconds"] == 4000.0 and "3300 Newton" in r["sample"]


def test_whole_solve_when_a_small_workload_has_no_record(fake):
    fake.seed, fake.n = 5, 33
    r = bench.cpu_baseline(fake)
    assert FakeScene.budgets == [0.0]
    assert r["value"] == 3600.0 and r["newton_iterations"] == 3000 and r["converged"]


def test_the_reference_arm_reports_the_scaled_sample(fake, capsys):
    fake.impl, fake.warmup, fake.steps, fake.full_solve = "reference", 0, 1, False
    bench.run_reference(fake)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] == pytest.approx(20.0 * 4000.0 / 8.0)
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["extrapolated"] and line["config"]["tolerance_N"] == 1e-7


def test_progress_lines_give_the_record():
    lines = ["ptc step 1 h=1e-3 ...",
             "state after 0 steps: residual 1.0e-02 N at 0.500 s, 0 Newton iterations",
             "state after 1 steps: residual 5.0e-03 N at 1.500 s, 3 Newton iterations",
             "state after 2 steps: residual 9.0e-07 N at 2.500 s, 5 Newton iterations",
             "state after 3 steps: residual 8.0e-08 N at 3.250 s, 6 Newton iterations"]
    rec = bench.parse_progress(lines, "host")
    assert rec["seconds_at_step"] == [1.5, 2.5, 3.25]
    assert rec["seconds"] == 3.25 and rec["steps"] == 3 and rec["newton"] == 6 and rec["seconds_to_1e-6"] == 2.5


def test_tolerance_crossing_reads_the_step_records():
    recs = [{"residual": 1e-2, "seconds": 1.0, "inner": 3, "pcg_iterations": 30},
            {"residual": 5e-6, "seconds": 2.0, "inner": 2, "pcg_iterations": 20},
            {"residual": 8e-7, "seconds": 2.5, "inner": 1, "pcg_iterations": 10}]
    c = bench.tolerance_crossing(recs, 1e-6)
    # the third step starts below 1e-6 N: a solve stopped at 1e-6 N ends after the second step
    assert c == {"tolerance_N": 1e-6, "seconds": 2.0, "ptc_steps": 2, "newton_iterations": 5, "pcg_iterations": 50}
    assert bench.tolerance_crossing(recs, 1e-9) is None


def test_a_large_workload_without_record_reports_the_bare_sample(fake):
    fake.seed = 5
    fake.n = 129
    r = bench.cpu_baseline(fake)
    assert FakeScene.budgets == [20.0] and r["sample_only"] and r["value"] == 20.0


def test_the_committed_whole_solve_records_are_consistent():
    """Each committed record of the oracle's whole solve: cumulative step times that grow, end no later than the
    whole solve, and a 1e-6 N crossing inside it; the n129 ones cover the bench's default stop."""
    assert (129, 1, 0, 5e-08) in bench.FULL_SOLVE
    for key, r in bench.FULL_SOLVE.items():
        t = r["seconds_at_step"]
        assert t and all(a <= b for a, b in zip(t, t[1:])), key
        assert t[-1] <= r["seconds"] and len(t) <= r["steps"] and r["seconds_to_1e-6"] <= r["seconds"], key
        assert r["newton"] >= r["steps"], key
