"""The reference arm's arithmetic in bench.py, on the CPU with a stand-in oracle: a bounded sample is scaled by the
Newton iterations of the whole solve (the counted whole solve of the workload first, else this run's GPU solve),
and with neither count the whole solve is run and timed."""
import argparse

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


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(oracle_py, "Scene", FakeScene)
    monkeypatch.setattr(bench, "FULL_SOLVE_NEWTON", {(129, 1, 0): (3200, "the oracle's own full solve")})
    FakeScene.budgets = []
    return argparse.Namespace(n=129, plane=1, seed=0, cpu_budget=20.0)


def test_sample_is_scaled_by_the_oracle_full_solve_count(fake):
    r = bench.cpu_baseline(fake, {"newton_iterations": 3040})
    assert r["value"] == pytest.approx(20.0 / 16 * 3200)  # the counted whole solve wins over this run's GPU count
    assert FakeScene.budgets == [20.0] and "oracle's own full solve" in r["sample"]


def test_gpu_count_when_the_workload_has_no_oracle_count(fake):
    fake.seed = 5
    r = bench.cpu_baseline(fake, {"newton_iterations": 3040})
    assert r["value"] == pytest.approx(20.0 / 16 * 3040) and "GPU solve" in r["sample"]


def test_whole_solve_when_no_count_is_known(fake):
    fake.seed = 5
    r = bench.cpu_baseline(fake, None)
    assert FakeScene.budgets == [0.0]
    assert r["value"] == 3600.0 and r["newton_iterations"] == 3000 and r["converged"]


def test_the_reference_arm_never_reports_the_bare_sample(fake, capsys):
    import json

    fake.impl, fake.warmup, fake.steps, fake.full_solve = "reference", 0, 1, False
    bench.run_reference(fake)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] == pytest.approx(20.0 / 16 * 3200)
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["value"] == line["value"]
