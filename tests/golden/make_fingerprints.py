"""Writes tests/golden/fingerprints.json: a SHA-256 prefix of all six fields and the probe series
of the CUDA stepper after a few steps, per case, storage form, rounding and kernel path.

Every rounding of the update is explicit, so these bits depend only on the arithmetic, not on
launch shapes, staging or vector widths; tests/test_gpu_fingerprints.py recomputes them and
fails on any change, which a change of the kernels' arithmetic must explain (and regenerate
with this script, on a B200).  Run from the repository root: python tests/golden/make_fingerprints.py
"""
import hashlib
import importlib
import json
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
GOLDEN = ROOT / "tests" / "golden"
CASES = [("step_g1_gain", 60), ("step_g2_planewave", 60), ("step_g3_pec", 60),
         ("c0_dipole_sphere", 120), ("c1_gain_slab", 40), ("b256_gain_slab", 20)]
# (precision, rounding): FP64, FP32, FP16, BF16 nearest, BF16 stochastic
FORMS = [(1, 0), (0, 0), (2, 0), (3, 0), (3, 1)]


def case_path(pkg, name):
    p = GOLDEN / "cases" / (name + ".params")
    return p if p.exists() else pkg.config_path(name + ".params")


def fingerprint(pkg, name, steps, precision, rounding, path):
    """Seeded fields (small cases) or the case's own source (the 280^3 workload), `steps` steps."""
    s = pkg.Setup.from_file(case_path(pkg, name))
    v = pkg.SetupV1.from_buffer_copy(s.view)
    v.rounding = rounding
    sol = pkg.Solver(s, precision=precision, view=v, kernel_path=path)
    if not name.startswith("b256"):
        rng = np.random.default_rng(7)
        for c in ("Ex", "Ey", "Ez"):
            sol.set_field(c, rng.normal(0, 1e-2, sol.shape))
    sol.run(steps)
    h = hashlib.sha256()
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        h.update(sol.field(c).tobytes())
    h.update(sol.probe_series().tobytes())
    sol.close()
    return h.hexdigest()[:16]


def keys():
    for name, steps in CASES:
        for prec, rnd in FORMS:
            for path in (1, 2):
                if path == 2 and name.startswith("b256"):
                    continue
                yield name, steps, prec, rnd, path


def key_name(name, prec, rnd, path):
    return f"{name}/p{prec}r{rnd}/k{path}"


def main():
    sys.path.insert(0, str(ROOT))
    pkg = importlib.import_module("3d_fdtd_version008_b200")
    out = {key_name(n, p, r, k): fingerprint(pkg, n, st, p, r, k) for n, st, p, r, k in keys()}
    (GOLDEN / "fingerprints.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(len(out), "fingerprints")


if __name__ == "__main__":
    main()
