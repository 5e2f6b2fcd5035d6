"""Regenerates the golden fixtures in tests/golden/ from the reference solver itself.

Runs oracle/_ref/ref_harness (the reference headers compiled where they lie; build it
with ``make -C oracle ref``) on every parameter file in tests/golden/cases/ and on the
shipped configs, and stores what it produced:

  mesh_*.npz   mesh lines (x/y/z_bounds) of the reference auto-mesher: the scenarios of
               the reference's tests/test_auto_mesh.cpp and tests/verify_mesh_override.cpp
  step_*.npz   setup arrays (mesh lines, CPML profiles, gain map; SHA-256 digests of the
               bE arrays and of the seeded initial fields), and the reference's state and
               probe series after N_STEPS steps
  det_*.npz    every file the reference's detectors wrote (frames/<RUN_TAG>/..., as bytes
               keyed by relative path) over N_STEPS steps
  configs.json mesh lines and SHA-256 digests of the material arrays of the shipped
               configs (their full arrays are too large to commit)

Usage: python tests/golden/make_golden.py [case stem ...]   (needs the reference checkout;
the GPU box only reads the .npz/.json files this writes; with stems, only those cases)
"""
from __future__ import annotations

import hashlib
import json
import os
import pathlib
import shutil
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
NOISE_SEED = {"step_g1_gain": 7}
NOISE_AMPLITUDE = 1e-3


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def mesh_case(path: pathlib.Path) -> None:
    r = oracle.run_harness(path, 0, "--mesh-only")
    np.savez_compressed(HERE / (path.stem + ".npz"), **{k: r[k] for k in ("x_bounds", "y_bounds", "z_bounds")})
    print(path.stem, [len(r[k]) - 1 for k in ("x_bounds", "y_bounds", "z_bounds")])


def initial_noise(stem: str, n: int):
    """Seeded initial E noise of a step case (tests regenerate it from the same seed)."""
    rng = np.random.default_rng(NOISE_SEED[stem])
    return {c: (rng.normal(0.0, NOISE_AMPLITUDE, n) if c[0] == "E" else np.zeros(n)) for c in FIELDS}


def step_case(path: pathlib.Path) -> None:
    probe = oracle.run_harness(path, 0, "--mesh-only")
    shape = tuple(probe["meta"][k] for k in ("NxT", "NyT", "NzT"))
    n = int(np.prod(shape))
    init_dir = None
    init = {}
    if path.stem in NOISE_SEED:
        (oracle.ORACLE_DIR / "_ref" / "runs").mkdir(parents=True, exist_ok=True)
        init_dir = tempfile.mkdtemp(prefix="golden_init_", dir=str(oracle.ORACLE_DIR / "_ref" / "runs"))
        for c, v in initial_noise(path.stem, n).items():
            init["init_" + c] = v
            v.tofile(os.path.join(init_dir, c + ".f64"))
    text = path.read_text()
    steps = int([ln.split("=")[1] for ln in text.splitlines() if ln.strip().startswith("N_STEPS")][0])
    r = oracle.run_harness(path, steps, "--dump-materials", init_dir=init_dir)
    if init_dir:
        shutil.rmtree(init_dir, ignore_errors=True)
    keep = {k: r[k] for k in ("x_bounds", "y_bounds", "z_bounds", "probe_series") + FIELDS}
    digests = {"sha256_" + k: sha(r[k]) for k in ("bEx", "bEy", "bEz", "n_grid")}
    for k in list(r):
        if isinstance(k, str) and k.startswith("cpml_"):
            keep[k] = r[k]
    if "tls_region_map" in r:
        keep["tls_region_map"] = r["tls_region_map"].astype(np.int8)
    for k in ("Pz", "Pz_prev", "Nu", "Ng"):
        if k in r:
            keep[k] = r[k]
    for k, v in init.items():
        digests["sha256_" + k] = sha(v)
    meta = dict(r["meta"], noise_seed=NOISE_SEED.get(path.stem), noise_amplitude=NOISE_AMPLITUDE, **digests)
    keep["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / (path.stem + ".npz"), **keep)
    print(path.stem, shape, steps, "steps")


def detector_case(path: pathlib.Path) -> None:
    text = path.read_text()
    steps = int([ln.split("=")[1] for ln in text.splitlines() if ln.strip().startswith("N_STEPS")][0])
    r = oracle.run_harness(path, steps, "--detectors", "--no-fields")
    # the reference's TLSGlobalHistory also drops a plotting script; it is not an output format
    files = {k: np.frombuffer(v, dtype=np.uint8) for k, v in r["frames"].items() if not k.endswith(".py")}
    np.savez_compressed(HERE / (path.stem + ".npz"), **files)
    print(path.stem, len(files), "files")


def configs() -> None:
    out = {}
    cfg_dir = ROOT / "3d_fdtd_version008_b200" / "configs"
    for path in sorted(cfg_dir.glob("*.params")):
        r = oracle.run_harness(path, 0, "--dump-materials", "--no-fields")
        entry = {"shape": [r["meta"][k] for k in ("NxT", "NyT", "NzT")], "dt": r["meta"]["dt"]}
        for k in ("x_bounds", "y_bounds", "z_bounds"):
            entry[k] = r[k].tolist()
        for k in ("bEx", "bEy", "bEz", "bHx", "n_grid") + tuple(f"cpml_{a}{x}" for a in ("k", "bE", "cE", "bH", "cH")
                                                              for x in "xyz"):
            entry["sha256_" + k] = sha(r[k])
        if "tls_region_map" in r:
            entry["sha256_tls_region_map"] = sha(r["tls_region_map"].astype(np.float64))
        entry["sources"] = r["meta"]["sources"]
        entry["tls_regions"] = r["meta"]["tls_regions"]
        entry["probes"] = r["meta"]["probes"]
        out[path.name] = entry
        print(path.name, entry["shape"])
    (HERE / "configs.json").write_text(json.dumps(out, indent=1))


def main(only=()) -> None:
    oracle.build(ref=True)
    for path in sorted((HERE / "cases").glob("mesh_*.params")):
        if not only or path.stem in only:
            mesh_case(path)
    for path in sorted((HERE / "cases").glob("step_*.params")):
        if not only or path.stem in only:
            step_case(path)
    for path in sorted((HERE / "cases").glob("det_*.params")):
        if not only or path.stem in only:
            detector_case(path)
    if not only:
        configs()


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
