"""The E1 gate checkers (tests/e1_gates.py) on the CPU: each gate passes on a clean case and fails on the case that
plants its failure, and the growth and bandwidth arithmetic follows the reference's definitions."""
import pytest

from tests import e1_gates as g

CLEAN = dict(status="converged", iterations=151, true_relative_residual=1e-7, f64_iterations=149,
             emulated_iterations=151, difference_vs_cpu_f32=1e-7, relative_error=1e-6, deterministic=True,
             cpu_f64_seconds=0.5, gpu_solve_ms=10.0)


def test_clean_case_passes_every_gate():
    assert all(g.verdict(**CLEAN).values())


@pytest.mark.parametrize("change, gate", [
    ({"status": "iteration_limit"}, "converged"),
    ({"true_relative_residual": 2e-2}, "forcing_term_ok"),
    ({"iterations": 230, "emulated_iterations": 230}, "f32_iterations_ok"),
    ({"iterations": 162}, "faithful_to_cpu_f32_emulation"),       # more than 2 + 5 % off the emulation's 151
    ({"difference_vs_cpu_f32": 3e-6}, "faithful_to_cpu_f32_emulation"),
    ({"deterministic": False}, "deterministic"),
    ({"gpu_solve_ms": 60.0}, "speedup_ok"),                         # 500 ms / 60 ms < 10
])
def test_each_planted_failure_trips_its_gate(change, gate):
    v = g.verdict(**dict(CLEAN, **change))
    assert not v[gate]
    assert all(ok for k, ok in v.items() if k != gate)


def test_growth_and_bandwidth():
    ratios = g.growth([(3 * 4225, 303), (3 * 1089, 151), (3 * 16641, 631)])
    assert [round(r, 3) for r, _ in ratios] == [round(303 / 151, 3), round(631 / 303, 3)]
    assert all(ok for _, ok in ratios)
    assert not g.growth([(1, 100), (2, 300)])[0][1]
    assert g.effective_bandwidth_gbs(1000, 100, 10, 1.0) == pytest.approx((40 * 1000 + 196 * 100) * 10 / 1e6)
