"""PTC probes of `drape --checks` (runPtcProbes, drape-e7.ts:190-200; run-e7.ts:146-152) and the reference comparer's
probe replays on the files they write (needs a B200): alpha_max against the f64 CCD rule at each recorded (x, d)
pair, the recorded f32 resolution against the iterate's, and every line-search decision against its numbers."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from drape_b200 import api
from drape_b200.build import CLI
from tests import e7_replays, oracle_py
from tests.test_gpu_checks import H_STEP, KERNEL_MU, N, _add_arrays

pytestmark = pytest.mark.gpu


def _write_probes(directory, probes):
    """probes.json / probes.bin in the problem-file layout: probe_steps u32, probe_h f32, probe_positions f32."""
    steps = np.array([p[0] for p in probes], np.uint32)
    hs = np.array([p[1] for p in probes], np.float32)
    pos = np.concatenate([np.asarray(p[2], np.float32) for p in probes])
    raw, arrays = bytearray(), []
    for name, dtype, values in (("probe_steps", "u32", steps), ("probe_h", "f32", hs), ("probe_positions", "f32", pos)):
        while len(raw) % 8:
            raw.append(0)
        arrays.append({"name": name, "dtype": dtype, "length": int(values.size), "offset": len(raw)})
        raw += values.tobytes()
    open(os.path.join(directory, "probes.bin"), "wb").write(bytes(raw))
    open(os.path.join(directory, "probes.json"), "w").write(json.dumps({"arrays": arrays}, separators=(",", ":")))


def test_probe_files_pass_the_probe_replays():
    with tempfile.TemporaryDirectory() as t:
        api.write_sheet_problem(t, N, seed=0, plane=True)
        oracle = oracle_py.Scene("sheet", N, seed=0, plane=True)
        _add_arrays(t, {"kernel_state": oracle.kernel_state(), "contact_state": oracle.contact_state(),
                        "row_mass": oracle.mass() / H_STEP ** 2}, {"kernel_mu": KERNEL_MU})
        _, arr = api.read_problem_arrays(t)
        # probed states: the starts of the two steps of a 40-step GPU solve of the same problem that took the most
        # Newton updates (early steps of the falling sheet converge at the prediction, with no update to log)
        d = api.Drape.from_files(t, options=api.default_options(max_steps=40))
        d.keep_states()
        d.solve_equilibrium(check=False)
        recs, states = d.step_records(), d.step_states()
        d.close()
        busiest = sorted(range(1, len(recs)), key=lambda k: (-recs[k]["inner"], k))[:2]
        assert all(recs[k]["inner"] > 0 for k in busiest)
        probes = [(recs[k]["step"], recs[k]["h"], states[k - 1]) for k in sorted(busiest)]
        _write_probes(t, probes)
        p = subprocess.run([CLI, "--case", t, "--mode", "cold", "--checks"], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stderr
        out = os.path.join(t, "gpu-cold")
        res = json.load(open(os.path.join(out, "gpu-result.json")))
        fields = res["robust_fields"]
        V = arr["rest_positions"].size // 3
        it = np.fromfile(os.path.join(out, "gpu-probe-iterations.bin"), np.float64).reshape(-1, 9)
        rb = np.fromfile(os.path.join(out, "gpu-probe-robust.bin"), np.float64).reshape(-1, len(fields))
        iterates = np.fromfile(os.path.join(out, "gpu-probe-iterates.bin"), np.float32).reshape(-1, 3 * V)
        pairs = np.fromfile(os.path.join(out, "gpu-probe-directions.bin"), np.float32).reshape(-1, 2, 3 * V)
        trials = np.fromfile(os.path.join(out, "gpu-probe-search.bin"), np.float64).reshape(-1, 8)
        assert len(it) == len(rb) == len(iterates) > 0
        assert set(it[:, 0].astype(int)) == {p[0] for p in probes}
        updates = np.isfinite(it[:, 3])
        assert len(pairs) == int(updates.sum()) > 0 and len(trials) >= len(pairs)
        assert np.isfinite(iterates).all() and np.isfinite(pairs).all()
        free = arr["row_vertex"].astype(int)
        assert e7_replays.resolution_replay(it, rb, fields, iterates, free)
        errors = e7_replays.alpha_errors(it, rb, fields, pairs, oracle.max_step)
        assert max(errors) <= 1e-4, max(errors)
        assert e7_replays.acceptance_replay(trials, api.default_options().armijo)
        # the checks and probes leave the cold solve alone: the same equilibrium as a run without --checks
        with tempfile.TemporaryDirectory() as t2:
            for name in ("problem.json", "problem.bin"):
                open(os.path.join(t2, name), "wb").write(open(os.path.join(t, name), "rb").read())
            p2 = subprocess.run([CLI, "--case", t2, "--mode", "cold"], capture_output=True, text=True, timeout=600)
            assert p2.returncode == 0, p2.stderr
            eq1 = np.fromfile(os.path.join(out, "gpu-equilibrium.bin"), np.float32)
            eq2 = np.fromfile(os.path.join(t2, "gpu-cold", "gpu-equilibrium.bin"), np.float32)
            assert np.array_equal(eq1, eq2)
