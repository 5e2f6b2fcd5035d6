"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import importlib
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product stepper")


@pytest.fixture(scope="session")
def pkg():
    mod = importlib.import_module("3d_fdtd_version008_b200")
    if not mod.library_path().exists():
        mod.build_library()
    return mod


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    if not o.ORACLE_LIB.exists():
        o.build(ref=False)
    return o


@pytest.fixture
def outdir():
    """A scratch directory inside the repository's build area, removed afterwards."""
    import shutil
    import tempfile
    base = ROOT / "_build" / "test_out"
    base.mkdir(parents=True, exist_ok=True)
    d = pathlib.Path(tempfile.mkdtemp(dir=str(base)))
    yield d
    shutil.rmtree(d, ignore_errors=True)


def golden(name: str):
    d = np.load(GOLDEN / (name + ".npz"))
    out = {k: d[k] for k in d.files}
    if "meta_json" in out:
        import json
        out["meta"] = json.loads(bytes(out.pop("meta_json")).decode())
    return out


def field_rel_l2(mine: dict, ref: dict, kind: str) -> float:
    """Relative L2 of the stacked (x, y, z) components of E or H."""
    num = sum(float(np.sum((np.asarray(mine[kind + c]).ravel() - np.asarray(ref[kind + c]).ravel()) ** 2)) for c in "xyz")
    den = sum(float(np.sum(np.asarray(ref[kind + c]).ravel() ** 2)) for c in "xyz")
    return (num / den) ** 0.5 if den > 0 else num ** 0.5
