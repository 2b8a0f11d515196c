"""Extract the reference's stored known answers for the drape path into tests/golden/reference_values.json.

Run once where the reference tree is checked out, with its path as the one argument
(`python tests/golden/make_golden.py <reference checkout>`); the JSON it writes is committed so the test suite never
reads the reference tree.

Sources (paths inside the reference project):
  experiments/cases/<kind>-n<N>/reference.json   E1 block-Jacobi PCG iteration counts, f64 and f32, the
                                                 recursive-residual history, band Cholesky bandwidth
  experiments/cases/<kind>-n<N>/problem.json     rows / blocks of the E1 matrices
  experiments/drape7/drape-n<N>/<edit>/problem.json           rows, blocks, kappa, release height, gravity load
  experiments/drape7/drape-n<N>/<edit>/reference-<mode>.json  converged f64 static energy, PTC/Newton counts
"""
import glob
import json
import os
import sys


def main(root: str) -> None:
    out = {"e1": {}, "drape7": {}}
    for ref in sorted(glob.glob(os.path.join(root, "experiments/cases/*/reference.json"))):
        case = os.path.basename(os.path.dirname(ref))
        r = json.load(open(ref))
        p = json.load(open(os.path.join(os.path.dirname(ref), "problem.json")))
        entry = {"rows": p["rows"], "blocks": p["blocks"], "bandwidth": r["cholesky_f64"]["bandwidth"],
                 "replace_every": p.get("replace_every", 0), "replace_above": p.get("replace_above", 0.0)}
        for key in ("pcg_f64_cpu", "pcg_f32_cpu"):
            s = r[key]
            # The residual history is kept for converged solves only (non-converged f32 runs are 20000 noisy
            # iterations whose history pins nothing).
            entry[key] = {"iterations": s["iterations"], "converged": s["converged"],
                          "recursive_relative_residual": s["recursive_relative_residual"],
                          "history": s.get("history", []) if s["converged"] else []}
        out["e1"][case] = entry
    for prob in sorted(glob.glob(os.path.join(root, "experiments/drape7/drape-n*/*/problem.json"))):
        edit = os.path.basename(os.path.dirname(prob))
        case = os.path.basename(os.path.dirname(os.path.dirname(prob)))
        p = json.load(open(prob))
        entry = {"columns": p["grid_columns"], "vertices": p["vertices"], "triangles": p["triangles"],
                 "hinges": p["hinges"], "rows": p["rows"], "blocks": p["blocks"],
                 "kappa": p["contact"]["kappa"], "dhat": p["contact"]["dhat_m"],
                 "release_height": p["contact"]["release_height_m"], "gravity_load": p["ptc"]["gravity_load"],
                 "references": {}}
        for ref in sorted(glob.glob(os.path.join(os.path.dirname(prob), "reference-*.json"))):
            mode = os.path.basename(ref)[len("reference-"):-len(".json")]
            r = json.load(open(ref))
            entry["references"][mode] = {k: r[k] for k in (
                "converged", "reason", "ptc_steps", "newton_iterations", "final_relative_residual",
                "static_energy", "gravity_load", "representation_floor", "final_h") if k in r}
        out["drape7"][f"{case}/{edit}"] = entry
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_values.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote {path}: {len(out['e1'])} E1 cases, {len(out['drape7'])} drape7 cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
