"""The kernel checks of `drape --checks` (run-e7.ts:140-145) against the f64 oracle (needs a B200).

The element terms are written per element in the reference's layout (membrane_element.wgsl, hinge_element.wgsl)
and the row terms per row (inertia.wgsl). Scattered into rows and added to the row terms they must give the
oracle's assembled gradient and tangent at the same state: exact element terms with the barrier's curvature term
against the exact-tangent oracle, projected ones without it against the projected oracle. Tolerance: every entry
is an f64 value rounded to f32 once and a row sums about a dozen of them, so 2e-6 of the largest term.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from drape_b200 import api
from drape_b200.build import CLI
from tests import oracle_py

pytestmark = pytest.mark.gpu

N, H_STEP, KERNEL_MU = 17, 1e-2, 0.25


def _add_arrays(directory, arrays, robust):
    """Appends f32 arrays to problem.bin and their manifest entries (and a robust block) to problem.json."""
    meta = json.load(open(os.path.join(directory, "problem.json")))
    raw = bytearray(open(os.path.join(directory, "problem.bin"), "rb").read())
    for name, values in arrays.items():
        while len(raw) % 8:
            raw.append(0)
        data = np.asarray(values, np.float32).tobytes()
        meta["arrays"].append({"name": name, "dtype": "f32", "length": len(values), "offset": len(raw)})
        raw += data
    meta["robust"] = robust
    open(os.path.join(directory, "problem.bin"), "wb").write(bytes(raw))
    open(os.path.join(directory, "problem.json"), "w").write(json.dumps(meta, separators=(",", ":")))


def _scatter(d, tri, hinge, eg, eh):
    """Element terms summed into the row gradient [3R] and a dense tangent [3R, 3R] (rows = vertices here)."""
    R = d.R
    g = np.zeros(3 * R)
    K = np.zeros((3 * R, 3 * R))
    for e in range(d.T):
        v = tri[3 * e:3 * e + 3]
        blocks = eh[81 * e:81 * e + 81].astype(np.float64).reshape(3, 3, 3, 3)
        for k in range(3):
            g[3 * v[k]:3 * v[k] + 3] += eg[9 * e + 3 * k:9 * e + 3 * k + 3]
            for l in range(3):
                K[3 * v[k]:3 * v[k] + 3, 3 * v[l]:3 * v[l] + 3] += blocks[k, l]
    g0, h0 = 9 * d.T, 81 * d.T
    for hh in range(d.H):
        v = hinge[4 * hh:4 * hh + 4]
        blocks = eh[h0 + 144 * hh:h0 + 144 * hh + 144].astype(np.float64).reshape(4, 4, 3, 3)
        for k in range(4):
            g[3 * v[k]:3 * v[k] + 3] += eg[g0 + 12 * hh + 3 * k:g0 + 12 * hh + 3 * k + 3]
            for l in range(4):
                K[3 * v[k]:3 * v[k] + 3, 3 * v[l]:3 * v[l] + 3] += blocks[k, l]
    return g, K


def _dense(rp, ci, vals, R):
    K = np.zeros((3 * R, 3 * R))
    b = vals.reshape(-1, 3, 3)
    for r in range(R):
        for k in range(rp[r], rp[r + 1]):
            K[3 * r:3 * r + 3, 3 * ci[k]:3 * ci[k] + 3] = b[k]
    return K


def _rows_dense(rh, R):
    K = np.zeros((3 * R, 3 * R))
    b = rh.astype(np.float64).reshape(-1, 3, 3)
    for r in range(R):
        K[3 * r:3 * r + 3, 3 * r:3 * r + 3] = b[r]
    return K


@pytest.fixture(scope="module")
def case():
    with tempfile.TemporaryDirectory() as t:
        api.write_sheet_problem(t, N, seed=0, plane=True)
        oracle = oracle_py.Scene("sheet", N, seed=0, plane=True)
        ks, cs = oracle.kernel_state(), oracle.contact_state()
        _add_arrays(t, {"kernel_state": ks, "contact_state": cs, "row_mass": oracle.mass() / H_STEP ** 2},
                    {"kernel_mu": KERNEL_MU})
        p = subprocess.run([CLI, "--case", t, "--mode", "cold", "--checks"], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stderr
        out = os.path.join(t, "gpu-cold")
        files = {name: np.fromfile(os.path.join(out, f"gpu-{name}.bin"), np.float32)
                 for name in ("kernel", "contact-kernel", "inertia-h")}
        _, arr = api.read_problem_arrays(t)
        d = api.Drape.from_files(t)
        yield d, oracle, files, arr
        d.close()


def test_file_sizes(case):
    d, _, f, _ = case
    ng, nh = 9 * d.T + 12 * d.H, 81 * d.T + 144 * d.H
    assert f["kernel"].size == 2 * (ng + nh) + 12 * d.R
    assert f["contact-kernel"].size == 12 * d.R
    assert f["inertia-h"].size == 3 * 12 * d.R


@pytest.mark.parametrize("state", ["kernel_state", "contact_state"])
@pytest.mark.parametrize("exact", [True, False])
def test_element_and_row_terms_assemble_to_the_oracle(case, state, exact):
    d, _, _, arr = case
    oracle = oracle_py.Scene("sheet", N, seed=0, plane=True, projected=not exact)
    x = arr[state].astype(np.float64)
    eg, eh = d.element_terms(x, exact=exact)
    m = oracle.mass() / H_STEP ** 2
    rg, rh = d.row_terms(x, x, row_mass=m, mu=0.0, contact=True, curvature=exact)
    g, K = _scatter(d, arr["elem_vertices"].astype(int), arr["hinge_vertices"].astype(int), eg, eh)
    g += rg
    K += _rows_dense(rh, d.R)
    g_o, v_o = oracle.assemble(x, x, H_STEP, mu=0.0, curvature=exact)
    rp, ci = oracle.pattern()
    K_o = _dense(rp, ci, v_o, d.R)
    # each row sums a dozen f32-rounded terms: bound the error by the largest term, not the (cancelled) sum
    assert np.abs(g - g_o).max() <= 2e-6 * max(np.abs(eg).max(), np.abs(rg).max())
    assert np.abs(K - K_o).max() <= 2e-6 * max(np.abs(eh).max(), np.abs(rh).max())


def test_check_files_hold_the_reference_passes(case):
    d, _, f, arr = case
    ks, cs, rest = (arr[k].astype(np.float64) for k in ("kernel_state", "contact_state", "rest_positions"))
    ng, nh = 9 * d.T + 12 * d.H, 81 * d.T + 144 * d.H
    k = f["kernel"]
    for i, exact in enumerate((True, False)):
        eg, eh = d.element_terms(ks, exact=exact)
        assert np.array_equal(k[i * (ng + nh):i * (ng + nh) + ng], eg)
        assert np.array_equal(k[i * (ng + nh) + ng:(i + 1) * (ng + nh)], eh)
    # inertia at x = kernel_state, x_hat = rest, mu = kernel_mu: (M/h^2)(x - x_hat) and (1 + mu) M/h^2 I
    rows = k[2 * (ng + nh):]
    row_mass = arr["row_mass"].astype(np.float64)
    want_g = (row_mass[:, None] * (ks - rest).reshape(-1, 3)).reshape(-1)
    assert np.allclose(rows[:3 * d.R], want_g, rtol=2e-6, atol=2e-6 * np.abs(want_g).max())
    diag = rows[3 * d.R:].reshape(-1, 3, 3)
    assert np.allclose(diag, (1 + KERNEL_MU) * row_mass[:, None, None] * np.eye(3), rtol=2e-6)
    # contact: the barrier rows alone at contact_state equal the API's
    cg, ch = d.row_terms(cs, cs, contact=True, curvature=True)
    assert np.array_equal(f["contact-kernel"], np.concatenate([cg, ch]))
    assert np.abs(cg).max() > 0  # contact_state touches a collider
    # inertia at h = 1/240, 0.1, 1 s
    unit = arr["row_unit_mass_f64"] if "row_unit_mass_f64" in arr else arr["row_unit_mass"].astype(np.float64)
    for j, size in enumerate((1 / 240, 0.1, 1.0)):
        part = f["inertia-h"][12 * d.R * j:12 * d.R * (j + 1)]
        mass = (unit / size ** 2).astype(np.float32).astype(np.float64)
        want = (mass[:, None] * (ks - rest).reshape(-1, 3)).reshape(-1)
        assert np.allclose(part[:3 * d.R], want, rtol=2e-6, atol=2e-6 * np.abs(want).max())
