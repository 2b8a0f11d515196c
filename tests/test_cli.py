"""The `drape` command (drape_b200/drape): usage and error paths on the host (no GPU needed)."""
import os
import subprocess
import tempfile

import pytest

from drape_b200 import api
from drape_b200.build import CLI


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        pytest.skip("the drape command is not built (python -m drape_b200.build)")
    return CLI


def test_usage_errors_exit_2(cli):
    for args in ([], ["--case"], ["--case", "/x", "--mode", "sideways"], ["--case", "/x", "--mode", "warm"],
                 ["--case", "/x", "--preconditioner", "magic"], ["--bogus"]):
        p = subprocess.run([cli] + args, capture_output=True, text=True)
        assert p.returncode == 2, (args, p.stderr)
        assert "usage: drape" in p.stderr


def test_missing_problem_exits_1(cli):
    with tempfile.TemporaryDirectory() as t:
        p = subprocess.run([cli, "--case", t], capture_output=True, text=True)
        assert p.returncode == 1 and "problem.json" in p.stderr


def test_missing_start_state_exits_1(cli):
    with tempfile.TemporaryDirectory() as t:
        api.write_reference_problem(t, 17, "base")
        p = subprocess.run([cli, "--case", t, "--mode", "warm", "--start", os.path.join(t, "nothing")],
                           capture_output=True, text=True)
        assert p.returncode == 1 and "nothing" in p.stderr
