"""The reference's output files: the run directory written by make_context and the files of
its detectors (MeshDetector, FieldMovie2D, PointFieldDetector), against what the reference
itself wrote for tests/golden/cases/det_d0_outputs.params (tests/golden/det_d0_outputs.npz).

Setup-time files are compared byte for byte.  mesh_info.json is the one exception: the
reference fills its source_* and structures entries from its compiled-in UserConfig lists,
which a parameter file cannot change, so those lines are checked against this setup's own
dipole and structures instead."""
import json
import pathlib

import numpy as np
import pytest

from conftest import GOLDEN, golden

CASE = GOLDEN / "cases" / "det_d0_outputs.params"
TAG = "det_case"


def ref_files():
    return {k: bytes(v) for k, v in golden("det_d0_outputs").items()}


def is_frame(name: str) -> bool:
    return name.endswith(".raw") and "refractive_index" not in name


def is_run_time(name: str) -> bool:
    """Written while the solve steps (or at its end), not at setup."""
    return is_frame(name) or name.endswith(("_ts.bin", "populations_Nu.bin", "populations_Ng.bin", ".csv",
                                            "metadata_populations.json"))


def csv_rows(data: bytes):
    lines = data.decode().splitlines()
    return lines[0], np.array([[float(x) for x in ln.split(",")] for ln in lines[1:]])


def config_line(line: str) -> bool:
    t = line.strip()
    return t.startswith('"source_') or t.startswith('"num_structures') or t.startswith('"structures') or \
        t.startswith('{"type"') or t in ("]", "],")


def test_setup_outputs_match_reference(pkg, outdir):
    s = pkg.Setup.from_file(CASE)
    s.write_outputs(outdir)
    ref = ref_files()
    root = pathlib.Path(outdir) / "frames"
    mine = {str(f.relative_to(root)): f.read_bytes() for f in root.rglob("*") if f.is_file()}
    setup_time = {k for k in ref if not is_run_time(k)}
    assert setup_time <= set(mine), sorted(setup_time - set(mine))
    assert {k for k in mine if k.endswith("_ts.bin")} == {k for k in ref if k.endswith("_ts.bin")}
    for k in ref:  # the two-level CSVs start with the reference's header line
        if k.endswith(".csv"):
            assert mine[k] == ref[k].split(b"\n")[0] + b"\n", k
        if k.endswith(("populations_Nu.bin", "populations_Ng.bin")):
            assert mine[k] == b""
    for k in sorted(setup_time):
        if k.endswith("mesh_info.json"):
            a = [ln for ln in mine[k].decode().splitlines() if not config_line(ln)]
            b = [ln for ln in ref[k].decode().splitlines() if not config_line(ln)]
            assert a == b
        else:
            assert mine[k] == ref[k], k
    for k in mine:
        if k.endswith("_ts.bin"):
            assert mine[k] == b""
    assert not any(k.endswith("metadata_populations.json") for k in mine)


def test_mesh_info_uses_this_setups_dipole_and_structures(pkg, outdir):
    s = pkg.Setup.from_file(CASE)
    s.write_outputs(outdir)
    info = json.loads((pathlib.Path(outdir) / "frames" / TAG / "mesh_info.json").read_text())
    d = s.view.dipoles[0]
    assert (info["source_i"], info["source_j"], info["source_k"]) == (d.i, d.j, d.k)
    assert abs(info["source_x_target_nm"] - 160.0) < 1e-9 and abs(info["source_z_target_nm"] - 140.0) < 1e-9
    assert info["num_structures"] == 2
    assert info["structures"][1] == {"type": "box", "n": 3.4, "params_nm": [104, 216, 104, 174, 128, 152]}


def test_output_plan_errors(pkg, outdir):
    text = CASE.read_text()
    bad_pattern = text.replace('"sx_%04d.raw"', '"sx_%s.raw"')
    with pytest.raises(pkg.FdtdError):
        pkg.Setup.from_text(bad_pattern).write_outputs(outdir)
    with pytest.raises(pkg.FdtdError):
        pkg.Setup.from_text(text.replace("RUN_TAG = det_case", "RUN_TAG = ../escape")).write_outputs(outdir)
    with pytest.raises(pkg.FdtdError):
        pkg.Setup.from_text(text.replace("true, Ex_xy,", "true, ../Ex_xy,")).write_outputs(outdir)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 2e-5)])
def test_streamed_outputs_match_reference(pkg, outdir, precision, tol):
    """Movie frames captured on the device and point time series, written while the solve
    runs (in two run() calls), against the reference's files."""
    s = pkg.Setup.from_file(CASE)
    sol = pkg.Solver(s, precision=precision)
    sol.attach_outputs(outdir)
    sol.run(17)
    sol.run(13)
    sol.close_outputs()
    ref = ref_files()
    root = pathlib.Path(outdir) / "frames"
    mine = {str(f.relative_to(root)): f.read_bytes() for f in root.rglob("*") if f.is_file()}
    assert set(mine) == set(ref), sorted(set(mine) ^ set(ref))
    for k in sorted(ref):
        if k.endswith(".csv"):
            h1, a = csv_rows(mine[k])
            h2, b = csv_rows(ref[k])
            assert h1 == h2 and a.shape == b.shape, k
            scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
            # tls_global_history.csv prints 6-12 significant digits: its own rounding dominates
            ctol = max(tol, 2e-8) if "tls_global" in k else tol
            assert np.all(np.abs(a - b) <= ctol * scale + 1e-300), (k, np.abs(a - b).max(axis=0) / scale)
            if "tls_global" in k:
                assert np.array_equal(a[:, 0], b[:, 0])
        elif k.endswith(("populations_Nu.bin", "populations_Ng.bin")):
            a = np.frombuffer(mine[k], dtype=np.float64)
            b = np.frombuffer(ref[k], dtype=np.float64)
            assert a.shape == b.shape and np.linalg.norm(a - b) <= max(tol, 1e-6) * np.linalg.norm(b), k
        elif is_frame(k) or k.endswith("_ts.bin"):
            a = np.frombuffer(mine[k], dtype=np.float64)
            b = np.frombuffer(ref[k], dtype=np.float64)
            assert a.shape == b.shape, k
            movie = pathlib.PurePath(k).parent
            scale = max(np.linalg.norm(np.frombuffer(ref[j], dtype=np.float64))
                        for j in ref if pathlib.PurePath(j).parent == movie and (is_frame(j) or j.endswith("_ts.bin")))
            assert np.linalg.norm(a - b) <= tol * max(scale, 1e-300), k
        elif not k.endswith("mesh_info.json"):
            assert mine[k] == ref[k], k
    assert sol.kernel_launches > 0
    sol.close()


def _run_files(pkg, s, outdir, precision, shards, sub):
    sol = pkg.Solver(s, precision=precision, shards=shards)
    d = pathlib.Path(outdir) / sub
    sol.attach_outputs(d)
    sol.run(17)
    sol.run(13)
    sol.close_outputs()
    sol.close()
    root = d / "frames"
    return {str(f.relative_to(root)): f.read_bytes() for f in root.rglob("*") if f.is_file()}


@pytest.mark.gpu
@pytest.mark.parametrize("precision,shards", [(1, 2), (1, 3), (0, 3), (3, 3), (2, 2)])
def test_sharded_outputs_match_whole_solve(pkg, outdir, precision, shards):
    """A solve split into z shards writes the whole solve's files: movie frames joined from the
    shards' owned planes (XY slices from the shard that holds the plane, XZ / YZ slices from
    every shard), point series from the shard that holds the probe, population frames gathered,
    the two-level sums added over the shards.  The fields are bit-identical, so are the frames,
    series and population frames; the CSV sums differ only by FP64 summation order.  FP64, FP32,
    BF16 and FP16 storage."""
    s = pkg.Setup.from_file(CASE)
    whole = _run_files(pkg, s, outdir, precision, 1, "whole")
    split = _run_files(pkg, s, outdir, precision, shards, "split")
    assert set(split) == set(whole), sorted(set(split) ^ set(whole))
    for k in sorted(whole):
        if k.endswith(".csv"):
            h1, a = csv_rows(split[k])
            h2, b = csv_rows(whole[k])
            assert h1 == h2 and a.shape == b.shape, k
            scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
            assert np.all(np.abs(a - b) <= 1e-12 * scale), (k, np.abs(a - b).max(axis=0) / scale)
        elif not k.endswith("mesh_info.json"):
            assert split[k] == whole[k], k
    # the reference's file set (the whole solve's files are checked against the reference's
    # values in test_streamed_outputs_match_reference)
    assert set(split) == set(ref_files())


@pytest.mark.gpu
def test_float32_outputs(pkg, outdir):
    s = pkg.Setup.from_text(CASE.read_text() + "\nWRITE_FLOAT64 = false\n")
    sol = pkg.Solver(s, precision=1)
    sol.attach_outputs(outdir)
    sol.run(30)
    sol.flush_outputs()
    ref = ref_files()
    d = pathlib.Path(outdir) / "frames" / TAG
    a = np.fromfile(d / "Ex_xy" / "ex_0003.raw", dtype=np.float32)
    b = np.frombuffer(ref[f"{TAG}/Ex_xy/ex_0003.raw"], dtype=np.float64)
    assert a.shape == b.shape and np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b))
    ts = np.fromfile(d / "probe_c" / "S_mag_ts.bin", dtype=np.float32)
    assert ts.shape == (6,)
    assert json.loads((d / "probe_c" / "metadata.json").read_text())["dtype"] == "float32"
    with pytest.raises(pkg.FdtdError):
        sol.attach_outputs(outdir)  # once, and before the first step
    sol.close()
