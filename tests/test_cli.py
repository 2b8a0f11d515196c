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


def test_prolong_writes_the_oracle_prolongation(cli):
    """`drape prolong` (host arithmetic, no GPU) from the oracle's own n17 equilibrium of the reference's base case
    to its n33 case writes, bit for bit, the start state `oracle e7-prolong` writes (e7_prolong.rs:52-64): the
    four-corner average and the projection of vertices within d_hat of a collider."""
    import numpy as np

    from tests import oracle_py

    oracle_py.build()
    with tempfile.TemporaryDirectory() as t:
        c17, c33 = os.path.join(t, "n17"), os.path.join(t, "n33")
        for n, c in ((17, c17), (33, c33)):
            subprocess.run([oracle_py.CLI, "e7-generate", "--n", str(n), "--edit", "base", "--out", c], check=True,
                           capture_output=True)
        subprocess.run([oracle_py.CLI, "e7-solve", "--dir", c17, "--mode", "cold"], check=True, capture_output=True)
        eq = os.path.join(c17, "equilibrium-cold")
        mine, ref = os.path.join(t, "mine"), os.path.join(t, "ref")
        p = subprocess.run([cli, "prolong", "--coarse", eq, "--coarse-n", "17", "--fine-dir", c33, "--out", mine],
                           capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        subprocess.run([oracle_py.CLI, "e7-prolong", "--coarse", eq, "--coarse-n", "17", "--fine-dir", c33, "--out",
                        ref], check=True, capture_output=True)
        a, b = np.fromfile(mine + ".bin"), np.fromfile(ref + ".bin")
        assert a.size == 3 * 33 * 33 and np.array_equal(a, b)
        # a grid that does not prolong to the case's is refused
        p = subprocess.run([cli, "prolong", "--coarse", eq, "--coarse-n", "9", "--fine-dir", c33, "--out", mine],
                           capture_output=True, text=True)
        assert p.returncode == 1 and "vertices" in p.stderr
        p = subprocess.run([cli, "prolong", "--coarse", eq], capture_output=True, text=True)
        assert p.returncode == 2
