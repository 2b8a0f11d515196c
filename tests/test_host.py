"""Host-side checks of libdrape_b200.so that need no GPU: the C ABI exports, the product's scene builders
against the oracle's scenes, and the problem-file reader on files in the reference's format."""
import os
import re
import subprocess

import numpy as np
import pytest

from drape_b200 import api
from tests import oracle_py

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from drape_b200 import build

    build.build()
    return api.load()


def declared_functions():
    text = open(os.path.join(ROOT, "include", "drape_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(drape_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (drape_[a-z0-9_]+)$", out, flags=re.M))
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)


def test_options_struct_matches_the_header(lib):
    o = api.default_options()
    assert o.controller == 0 and o.newton_start == 0 and o.h0 == 1e-3 and o.equilibrium_absolute == 1e-6
    assert o.pcg_rtol == 1e-6 and o.pcg_max_iterations == 2000 and o.inner_max == 10 and o.max_halvings == 30


def _oracle_topology(scene):
    tris = np.zeros(3 * scene.T, np.int32)
    hinges = np.zeros(4 * scene.H, np.int32)
    k = np.zeros(scene.H)
    scene.lib.oracle_scene_topology(oracle_py.P(scene.h), oracle_py.ptr(tris), oracle_py.ptr(hinges), oracle_py.ptr(k))
    return tris, hinges, k


def _compare(tmp_path, arrays, meta, scene):
    tris, hinges, k = _oracle_topology(scene)
    assert np.array_equal(arrays["elem_vertices"].astype(np.int32), tris)
    assert np.array_equal(arrays["hinge_vertices"].astype(np.int32), hinges)
    assert np.allclose(arrays["hinge_stiffness_f64"], k, rtol=1e-14, atol=0)
    rp, ci = scene.pattern()
    assert np.array_equal(arrays["row_ptr"].astype(np.int32), rp)
    assert np.array_equal(arrays["col_idx"].astype(np.int32), ci)
    assert np.allclose(arrays["row_unit_mass_f64"], scene.mass(), rtol=1e-14, atol=0)
    assert np.array_equal(arrays["rest_positions_f64"], scene.start())
    assert meta["contact"]["dhat_m"] == scene.dhat
    assert abs(meta["contact"]["kappa"] - scene.kappa) <= 1e-15 * scene.kappa
    assert np.allclose(meta["gravity_vector"], scene.gravity)


@pytest.mark.parametrize("n,seed,plane", [(9, 0, False), (17, 3, True), (33, 0, True)])
def test_sheet_builder_matches_the_oracle(lib, tmp_path, n, seed, plane):
    d = str(tmp_path / "sheet")
    api.write_sheet_problem(d, n, seed=seed, radius=0.2, young=8e5, plane=plane)
    meta, arrays = api.read_problem_arrays(d)
    scene = oracle_py.Scene("sheet", n, seed=seed, radius=0.2, young=8e5, plane=plane)
    _compare(tmp_path, arrays, meta, scene)
    assert api.inspect_problem(d) == (scene.V, scene.T, scene.H, scene.R, scene.B, scene.colliders)


@pytest.mark.parametrize("edit", ["base", "w1", "w2", "w3"])
def test_reference_builder_matches_the_oracle(lib, tmp_path, edit):
    d = str(tmp_path / edit)
    api.write_reference_problem(d, 17, edit)
    meta, arrays = api.read_problem_arrays(d)
    _compare(tmp_path, arrays, meta, oracle_py.Scene("reference", 17, edit=edit))


def test_reads_problem_files_in_the_reference_format(lib, tmp_path):
    """`oracle e7-generate` writes the reference's problem.json / problem.bin layout (e3_generate.rs:84-229); the
    GPU stage's reader accepts it."""
    oracle_py.build()
    d = str(tmp_path / "n17")
    subprocess.run([oracle_py.CLI, "e7-generate", "--n", "17", "--edit", "base", "--out", d], check=True)
    s = oracle_py.Scene("reference", 17, edit="base")
    assert api.inspect_problem(d) == (s.V, s.T, s.H, s.R, s.B, 2)


def test_problem_reader_rejects_bad_input(lib, tmp_path):
    with pytest.raises(api.DrapeError) as e:
        api.inspect_problem(str(tmp_path / "missing"))
    assert e.value.status == 5
    d = str(tmp_path / "trunc")
    api.write_sheet_problem(d, 9)
    raw = open(os.path.join(d, "problem.bin"), "rb").read()
    open(os.path.join(d, "problem.bin"), "wb").write(raw[: len(raw) // 2])
    with pytest.raises(api.DrapeError):
        api.inspect_problem(d)
    with pytest.raises(api.DrapeError) as e:
        api.write_sheet_problem(str(tmp_path / "x"), 2)
    assert e.value.status == 1


def test_creating_a_context_without_a_device_fails_loudly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.DrapeError):
        api.Drape.sheet(9)


def test_batch_solve_rejects_an_empty_batch(lib):
    # argument checks of drape_solve_batch happen on the host, before any context or thread is touched
    with pytest.raises(api.DrapeError) as e:
        api.solve_batch([])
    assert e.value.status == 1
    assert "count or workers" in str(e.value)


def test_record_structs_match_the_header(tmp_path):
    """The ctypes views of the record structs have the C layout (sizes from the header, compiled here)."""
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "drape_b200.h"\nint main(void) { printf("%zu %zu %zu %zu %zu\\n", '
                   'sizeof(drape_newton_record), sizeof(drape_attempt_record), sizeof(drape_step_record), '
                   'sizeof(drape_options), sizeof(drape_run_log)); return 0; }\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    import ctypes
    assert sizes == [ctypes.sizeof(api.NewtonRecord), ctypes.sizeof(api.AttemptRecord),
                     ctypes.sizeof(api.StepRecord), ctypes.sizeof(api.Options), ctypes.sizeof(api.RunLog)]


def test_named_array_reader_reads_probe_files(tmp_path):
    """read_named_array (problem.cpp, compiled here with the host compiler) reads a probes.json / probes.bin pair in
    the problem-file layout (u32 and f32 arrays at 8-byte-aligned offsets) and returns nothing for an absent name."""
    import json

    steps = np.array([3, 17], np.uint32)
    h = np.array([1e-3, 0.25], np.float32)
    pos = np.arange(12, dtype=np.float32) * 0.5
    raw, arrays = bytearray(), []
    for name, dtype, values in (("probe_steps", "u32", steps), ("probe_h", "f32", h), ("probe_positions", "f32", pos)):
        while len(raw) % 8:
            raw.append(0)
        arrays.append({"name": name, "dtype": dtype, "length": int(values.size), "offset": len(raw)})
        raw += values.tobytes()
    (tmp_path / "probes.bin").write_bytes(bytes(raw))
    (tmp_path / "probes.json").write_text(json.dumps({"arrays": arrays}, separators=(",", ":")))
    src = tmp_path / "read.cpp"
    src.write_text('#include <cstdio>\n#include "problem.h"\nint main(int, char** argv) {\n'
                   '  for (const char* name : {"probe_steps", "probe_h", "probe_positions", "missing"}) {\n'
                   '    auto v = drape::read_named_array(std::string(argv[1]) + "/probes.json", std::string(argv[1]) +'
                   ' "/probes.bin", name);\n    std::printf("%s %zu", name, v.size());\n'
                   '    for (double x : v) std::printf(" %.17g", x);\n    std::printf("\\n");\n  }\n}\n')
    exe = tmp_path / "read"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "drape_b200", "csrc"), str(src),
                    os.path.join(ROOT, "drape_b200", "csrc", "problem.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, check=True).stdout.splitlines()
    got = {line.split()[0]: [float(v) for v in line.split()[2:]] for line in out}
    assert got["probe_steps"] == [3.0, 17.0]
    assert np.allclose(got["probe_h"], h.astype(np.float64), rtol=0, atol=0)
    assert np.array_equal(got["probe_positions"], pos.astype(np.float64))
    assert got["missing"] == []
