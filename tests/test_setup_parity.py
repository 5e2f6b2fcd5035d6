"""Host setup API vs the reference setup: mesh lines, dt, CPML profiles, materials and
gain map bit-identical (golden fixtures made by the reference itself), plus the
reference's own mesher assertions (tests/test_auto_mesh.cpp, tests/verify_mesh_override.cpp)
restated on this library's meshes."""
import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, golden

MESH_CASES = sorted(p.stem for p in (GOLDEN / "cases").glob("mesh_*.params"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits_equal(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("case", MESH_CASES)
def test_mesh_lines_bit_identical(pkg, case):
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"), mesh_only=True)
    g = golden(case)
    for a in "xyz":
        assert bits_equal(s.array(a + "_bounds"), g[a + "_bounds"]), (case, a)


def grading(dx):
    return float(np.max(np.maximum(dx[1:] / dx[:-1], dx[:-1] / dx[1:]))) if len(dx) > 1 else 1.0


def spacing_at(bounds, pos):
    dx = np.diff(bounds)
    for i in range(len(bounds) - 1):
        if bounds[i] <= pos < bounds[i + 1]:
            return dx[i]
    return dx[-1]


def lines(pkg, case):
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"), mesh_only=True)
    return s, {a: s.array(a + "_bounds") for a in "xyz"}


def on_grid(b, pos, tol=1e-12):
    return bool(np.any(np.abs(b - pos) < tol))


def test_reference_mesher_assertions_interface(pkg):
    # tests/test_auto_mesh.cpp:80-135
    _, b = lines(pkg, "mesh_t1_interface")
    x = b["x"]
    assert on_grid(x, 400e-9) and on_grid(x, 600e-9)
    assert spacing_at(x, 500e-9) <= spacing_at(x, 100e-9) * 1.2
    assert grading(np.diff(x)) <= np.sqrt(2.0) * 1.05


def test_reference_mesher_assertions_override(pkg):
    # tests/test_auto_mesh.cpp:138-228
    _, b = lines(pkg, "mesh_t2_override")
    x = b["x"]
    assert on_grid(x, 300e-9) and on_grid(x, 700e-9)
    dx = np.diff(x)
    centers = 0.5 * (x[1:] + x[:-1])
    inside = dx[(centers > 300e-9) & (centers < 700e-9)]
    assert len(inside) and (inside.max() - inside.min()) / inside.min() < 0.01
    assert abs(inside.mean() - 10e-9) / 10e-9 < 0.05
    assert grading(dx) <= np.sqrt(2.0) * 1.1


def test_reference_mesher_assertions_grading_and_monotonic(pkg):
    # tests/test_auto_mesh.cpp:307-367
    _, b = lines(pkg, "mesh_t4_grading")
    for a in "xyz":
        assert np.all(np.diff(b[a]) > 0)
        assert grading(np.diff(b[a])) <= np.sqrt(2.0) * 1.1


def test_reference_mesher_ppw_mapping(pkg):
    # tests/test_auto_mesh.cpp:370-432: accuracy -> ppw 6/10/14/18/22/34, and more cells at higher accuracy
    base = (GOLDEN / "cases" / "mesh_t5_ppw_low.params").read_text()
    for acc, ppw in [(1, 6), (2, 10), (3, 14), (4, 18), (5, 22), (8, 34)]:
        text = base.replace("AUTO_MESH_ACCURACY = 1", f"AUTO_MESH_ACCURACY = {acc}").replace("AUTO_MESH_DX_MAX = 200e-9", "AUTO_MESH_DX_MAX = 1e-6")
        s = pkg.Setup.from_text(text, mesh_only=True)
        dx = np.diff(s.array("x_bounds"))
        # air-only domain: uniform cells near lambda / ppw after rounding to the domain
        assert abs(np.median(dx) - 500e-9 / ppw) / (500e-9 / ppw) < 0.15, (acc, np.median(dx))
    _, lo = lines(pkg, "mesh_t5_ppw_low")
    _, hi = lines(pkg, "mesh_t5_ppw_high")
    assert len(hi["x"]) > len(lo["x"])


def test_reference_mesher_pml_extension_and_override_alignment(pkg):
    # tests/test_auto_mesh.cpp:531-701 and tests/verify_mesh_override.cpp:163-267
    s, b = lines(pkg, "mesh_t7_pml_override")
    npml = 8
    x = b["x"]
    phys0 = x[npml]
    phys = x - phys0
    assert abs(x[len(x) - 1 - npml] - phys0 - 1000e-9) < 1e-12
    assert on_grid(phys, 50e-9, 1e-9) and on_grid(phys, 350e-9, 1e-9)
    dx = np.diff(x)
    c = 0.5 * (phys[1:] + phys[:-1])
    inside = dx[(c > 50e-9) & (c < 350e-9)]
    assert (inside.max() - inside.min()) / inside.mean() < 0.01
    assert abs(inside.mean() - 5e-9) < 0.5e-9
    # fine mesh (< 10 nm) confined to the override box within 50 nm, and not reaching 400 nm
    fine = [(phys[i], phys[i + 1]) for i in range(npml, len(dx) - npml) if dx[i] < 10e-9]
    assert fine and fine[0][0] >= 50e-9 - 50e-9 and fine[-1][1] <= 350e-9 + 50e-9 and fine[-1][1] < 400e-9
    assert np.allclose(dx[:npml], dx[npml]) and np.allclose(dx[-npml:], dx[-npml - 1])


@pytest.mark.xfail(strict=True, reason="reference behaviour: build_segmented_grid_1d takes the first override "
                                       "containing a segment midpoint, so the coarser 20 nm region wins "
                                       "(src/auto_mesh_generator.hpp:447-455); the reference's own test fails too")
def test_reference_mesher_finer_override_wins(pkg):
    # tests/test_auto_mesh.cpp:231-304 ("Finer mesh wins in overlap") -- fails on the unmodified reference
    _, b = lines(pkg, "mesh_t3_nested_overrides")
    x = b["x"]
    assert abs(spacing_at(x, 500e-9) - 5e-9) / 5e-9 < 0.2


@pytest.mark.parametrize("cfg", ["c0_dipole_sphere.params", "c1_gain_slab.params"])
def test_shipped_configs_match_reference_setup(pkg, cfg):
    ref = json.loads((GOLDEN / "configs.json").read_text())[cfg]
    s = pkg.Setup.from_file(pkg.config_path(cfg))
    assert list(s.shape) == ref["shape"]
    assert s.dt == ref["dt"]
    for a in "xyz":
        assert bits_equal(s.array(a + "_bounds"), ref[a + "_bounds"])
    for k, v in ref.items():
        if k.startswith("sha256_"):
            name = k[len("sha256_"):]
            assert sha(s.array(name)) == v, name
    v = s.view
    for q, src in enumerate(ref["sources"]):
        d = v.dipoles[q]
        assert (d.i, d.j, d.k) == (src["i"], src["j"], src["k"])
        for f in ("cell_area", "I0", "f0", "tau", "t0", "t_shift"):
            assert getattr(d, f) == src[f], f
    for q, r in enumerate(ref["tls_regions"]):
        t = v.tls_regions[q]
        for f in ("kapa_coeff", "pa2", "pa3", "inv_dt", "tau", "hbar", "omega_a"):
            assert getattr(t, f) == r[f], f
        assert t.N0 == r["N0"]
    for q, p in enumerate(ref["probes"]):
        assert (v.probes[q].i, v.probes[q].j, v.probes[q].k) == (p["i"], p["j"], p["k"])


@pytest.mark.parametrize("case", ["step_g0_sphere", "step_g1_gain", "step_g2_planewave", "step_g3_pec"])
def test_step_case_setup_matches_reference(pkg, case):
    g = golden(case)
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"))
    for a in "xyz":
        assert bits_equal(s.array(a + "_bounds"), g[a + "_bounds"])
    for k in g:
        if k.startswith("cpml_"):
            assert bits_equal(s.array(k), g[k]), k
    for k, v in g["meta"].items():
        if k.startswith("sha256_") and not k.startswith("sha256_init"):
            assert sha(s.array(k[len("sha256_"):])) == v, k
    if "tls_region_map" in g:
        assert np.array_equal(s.array("tls_region_map").astype(np.int8), g["tls_region_map"])


def test_live_reference_harness_setup(pkg, oracle):
    """When the reference checkout is here, compare against it directly (not only fixtures)."""
    if not oracle.REF_HARNESS.exists():
        pytest.skip("reference harness not built (no reference checkout on this machine)")
    p = pkg.config_path("c1_gain_slab.params")
    r = oracle.run_harness(p, 0, "--dump-materials", "--no-fields")
    s = pkg.Setup.from_file(p)
    for k in ("x_bounds", "dz", "inv_dy", "bEx", "bEz", "cpml_cHz", "n_grid"):
        assert bits_equal(s.array(k), r[k]), k
    assert np.array_equal(s.array("tls_region_map"), r["tls_region_map"].astype(np.float64))


def test_plane_wave_sheet_geometry(pkg):
    """make_plane_wave_source's plane clamp and compute_bounds, and the component rule of
    inject_*_plane: an Ez plane wave along z drives nothing and is dropped."""
    text = (GOLDEN / "cases" / "step_g2_planewave.params").read_text()
    s = pkg.Setup.from_text(text)
    v = s.view
    assert v.n_sheets == 2
    a, b = v.sheets[0], v.sheets[1]
    # +Z / Ex over the whole non-PML plane; z = 80 nm -> core index 3 + npml
    assert (a.axis, a.comp, a.sign, a.plane) == (2, 0, 1.0, 6)
    assert (a.lo0, a.hi0, a.lo1, a.hi1) == (3, 14, 3, 12)
    assert abs(a.d - 25e-9) < 1e-20 and a.E0 == 1.0
    # -Y / Ez over x 50..200 nm, z 100..250 nm (in-plane axes x, z)
    assert (b.axis, b.comp, b.sign, b.plane) == (1, 2, -1.0, 9)
    assert (b.lo0, b.hi0, b.lo1, b.hi1) == (5, 11, 7, 13)
    ez_along_z = text + "\nPLANE_WAVE_SOURCES += true, 80e-9, 1.0, 193.4e12, 0, 2e-15, 0, 1.0, 1, 5, 2, 0, 0, 0, 0, 0, 0"
    s2 = pkg.Setup.from_text(ez_along_z)
    assert s2.view.n_sheets == 2
    with pytest.raises(pkg.FdtdError):
        pkg.Setup.from_text(ez_along_z.replace(", 1, 5, 2, 0, 0,", ", 1, 5, 1, 0, 0,"))  # a third sheet


def test_pec_grid_is_the_padded_mesh_origin(pkg):
    """PECBoundary's context: the field grid is the core size, taken from the start of the
    padded mesh, with no PML layer; the mesh arrays keep their padded length."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g3_pec.params")
    v = s.view
    g = golden("step_g3_pec")
    assert v.pec_boundary == 1 and v.npml == 0
    assert (v.NxT, v.NyT, v.NzT) == tuple(g["meta"][k] for k in ("NxT", "NyT", "NzT"))
    assert len(s.array("dx")) == v.NxT + 2 * 3 and len(s.array("x_bounds")) == v.NxT + 2 * 3 + 1
    c = pkg.Setup.from_text((GOLDEN / "cases" / "step_g3_pec.params").read_text().replace("BOUNDARY_TYPE = 0",
                                                                                            "BOUNDARY_TYPE = 1"))
    assert c.view.pec_boundary == 0 and c.view.npml == 3 and c.view.NxT == v.NxT + 6
