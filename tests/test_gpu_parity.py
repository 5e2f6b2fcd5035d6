"""GPU parity: the CUDA stepper (called through the C ABI) against the reference's golden
state and against the oracle on the shipped configs.

Tolerances: FP64 mode <= 1e-12 relative L2 (the accuracy reference).  FP32 mode <= 1e-5
relative L2 while the field is active; where the pulse has left the domain the bound is
3x the drift of the oracle's FP32 twin (same formulas, FP32 storage): the floor any FP32
storage reaches, since the decayed field is small against the rounding of its peak."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, field_rel_l2, golden

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def fields(obj):
    return {c: obj.field(c) for c in FIELDS}


def ref_fields(g, shape):
    return {c: g[c].reshape(shape) for c in FIELDS}


def rel(a, b):
    d = float(np.linalg.norm(np.ravel(b)))
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b))) / (d if d else 1.0)


def golden_solver(pkg, case, precision):
    g = golden(case)
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"))
    sol = pkg.Solver(s, precision=precision)
    seed = g["meta"].get("noise_seed")
    if seed is not None:
        sys.path.insert(0, str(GOLDEN))
        from make_golden import initial_noise
        for c, v in initial_noise(case, int(np.prod(sol.shape))).items():
            sol.set_field(c, v.reshape(sol.shape))
    return g, s, sol


@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_sphere_case_matches_reference(pkg, precision, tol):
    g, s, sol = golden_solver(pkg, "step_g0_sphere", precision)
    sol.run(g["meta"]["steps"])
    ref = ref_fields(g, sol.shape)
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= tol
    assert field_rel_l2(mine, ref, "H") <= tol
    series = sol.probe_series()
    assert series.shape == (g["meta"]["steps"], 4)
    assert rel(series, g["probe_series"].reshape(series.shape)) <= tol


@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_gain_case_matches_reference(pkg, precision, tol):
    g, s, sol = golden_solver(pkg, "step_g1_gain", precision)
    sol.run(g["meta"]["steps"])
    ref = ref_fields(g, sol.shape)
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= tol
    assert field_rel_l2(mine, ref, "H") <= tol
    gain = g["tls_region_map"].reshape(sol.shape) >= 0
    for c in ("Pz", "Pz_prev"):
        assert rel(sol.tls_state(c)[gain], g[c].reshape(sol.shape)[gain]) <= max(tol, 1e-5 if precision == 0 else tol), c
    for c in ("Nu", "Ng"):
        assert rel(sol.tls_state(c)[gain], g[c].reshape(sol.shape)[gain]) <= (1e-12 if precision == 1 else 1e-6), c
    series = sol.probe_series()
    assert rel(series, g["probe_series"].reshape(series.shape)) <= tol


@pytest.mark.parametrize("path", [1, 2])
@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_plane_wave_case_matches_reference(pkg, precision, tol, path):
    """Two plane-wave soft sources (a full +Z / Ex plane and a -Y / Ez sub-rectangle) and a
    dipole, against the reference's own fields and probe series."""
    g, s, _ = golden_solver(pkg, "step_g2_planewave", precision)
    assert s.view.n_sheets == 2
    sol = pkg.Solver(s, precision=precision, kernel_path=path)
    sol.run(g["meta"]["steps"])
    ref = ref_fields(g, sol.shape)
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= tol and field_rel_l2(mine, ref, "H") <= tol
    series = sol.probe_series()
    assert rel(series, g["probe_series"].reshape(series.shape)) <= tol


@pytest.mark.parametrize("path", [1, 2])
@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_pec_case_matches_reference(pkg, precision, tol, path):
    """PECBoundary (E zeroed on the six faces after every E update, no CPML) with a gain core,
    a dipole and a plane-wave sheet that reaches the faces, against the reference's state."""
    g, s, _ = golden_solver(pkg, "step_g3_pec", precision)
    assert s.view.pec_boundary == 1
    sol = pkg.Solver(s, precision=precision, kernel_path=path)
    sol.run(g["meta"]["steps"])
    ref = ref_fields(g, sol.shape)
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= tol and field_rel_l2(mine, ref, "H") <= tol
    for c in ("Ex", "Ey", "Ez"):
        f = mine[c]
        assert not (f[0].any() or f[-1].any() or f[:, 0].any() or f[:, -1].any() or f[:, :, 0].any() or f[:, :, -1].any())
    gain = g["tls_region_map"].reshape(sol.shape) >= 0
    for c in ("Pz", "Nu", "Ng"):
        assert rel(sol.tls_state(c)[gain], g[c].reshape(sol.shape)[gain]) <= max(tol, 1e-6), c
    series = sol.probe_series()
    assert rel(series, g["probe_series"].reshape(series.shape)) <= tol


def test_pec_refuses_path_0_and_packed_engine(pkg):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g3_pec.params")
    sol = pkg.Solver(s)
    with pytest.raises(pkg.FdtdError) as e:
        sol.set_kernel_path(0)
    assert e.value.code == 7
    sol.close()
    b = pkg.Batch(budget_bytes=1 << 30)
    with pytest.raises(pkg.FdtdError) as e:
        b.submit(s, 10)
    assert e.value.code == 7
    b.close()


PLANE_WAVE_PAIRS = [
    # (+X / Ey full plane, -Z / Ex sub-rectangle), (+Y / Ez, -X / Ez), (-Y / Ex, +Z / Ey)
    ("true, 400e-9, 1.0, 193.4e12, 0, 2e-15, 0, 1.0, 1, 0, 1, 0, 0, 0, 0, 0, 0",
     "true, 700e-9, 0.7, 0, 1400e-9, 0, 30e12, 1.2, 2, 5, 0, 300e-9, 1200e-9, 100e-9, 800e-9, 0, 0"),
    ("true, 300e-9, 1.0, 193.4e12, 0, 2e-15, 0, 1.0, 1, 2, 2, 0, 0, 0, 0, 0, 0",
     "true, 1300e-9, 2.0, 193.4e12, 0, 3e-15, 0, 1.0, 0, 1, 5, 0, 0, 200e-9, 500e-9, 400e-9, 900e-9"),
    ("true, 500e-9, 1.0, 193.4e12, 0, 2e-15, 0, 1.0, 1, 3, 0, 0, 0, 0, 0, 0, 0",
     "true, 600e-9, 1.0, 193.4e12, 0, 2e-15, 0, 1.0, 1, 4, 4, 0, 0, 0, 0, 0, 0"),
]


@pytest.mark.parametrize("pair", range(len(PLANE_WAVE_PAIRS)))
def test_plane_waves_on_odd_grid(pkg, oracle, pair):
    """Sheets along every axis and both signs, full planes and sub-rectangles, on a grid that
    is not a multiple of any tile or slab; both kernel paths against the oracle."""
    text = (GOLDEN / "cases" / "step_g0_sphere.params").read_text()
    text = text.replace("NX = 10", "NX = 71").replace("NY = 9", "NY = 37").replace("NZ = 8", "NZ = 45")
    text = text.replace("DOMAIN_X_MAX = 250e-9", "DOMAIN_X_MAX = 1775e-9").replace("DOMAIN_Y_MAX = 225e-9", "DOMAIN_Y_MAX = 925e-9")
    text = text.replace("DOMAIN_Z_MAX = 200e-9", "DOMAIN_Z_MAX = 1125e-9")
    text = "\n".join(ln for ln in text.splitlines() if not ln.startswith("DIPOLE_SOURCES"))
    for w in PLANE_WAVE_PAIRS[pair]:
        text += "\nPLANE_WAVE_SOURCES += " + w
    s = pkg.Setup.from_text(text)
    assert s.view.n_sheets == 2 and s.view.n_dipoles == 0
    o = oracle.OracleSolve(s, 0)
    o.run(70)
    ref = {c: o.field(c) for c in FIELDS}
    for path in (1, 2):
        for precision, tol in ((1, 1e-12), (0, 1e-5)):
            sol = pkg.Solver(s, precision=precision, kernel_path=path)
            sol.run(70)
            mine = fields(sol)
            assert field_rel_l2(mine, ref, "E") <= tol, (path, precision)
            assert field_rel_l2(mine, ref, "H") <= tol, (path, precision)
            sol.close()


def test_c0_fp32_active_field_within_1e5(pkg, oracle):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    o = oracle.OracleSolve(s, 0)
    o.run(600)
    sol = pkg.Solver(s, precision=0)
    sol.run(600)
    ref = {c: o.field(c) for c in FIELDS}
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= 1e-5
    assert field_rel_l2(mine, ref, "H") <= 1e-5


def test_c0_full_run_probe_dft_and_fp32_floor(pkg, oracle):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    steps = 2000
    o64 = oracle.OracleSolve(s, 0)
    p64 = o64.run(steps)[:, 0]
    o32 = oracle.OracleSolve(s, 1)
    p32 = o32.run(steps)[:, 0]
    sol = pkg.Solver(s, precision=0)
    sol.run(steps)
    pg = sol.probe_series()[:, 0]
    ref = {c: o64.field(c) for c in FIELDS}
    twin = {c: o32.field(c) for c in FIELDS}
    mine = fields(sol)
    for kind in "EH":
        floor = field_rel_l2(twin, ref, kind)
        assert field_rel_l2(mine, ref, kind) <= max(1e-5, 3.0 * floor), kind
    assert rel(pg, p64) <= max(1e-5, 3.0 * rel(p32, p64))
    freqs = s.array("dft_freqs")
    d_ref = oracle.dft(p64, s.dt, freqs)
    d_gpu = sol.dft(0)
    assert rel(d_gpu, d_ref) <= 1e-5


def test_c0_fp64_matches_oracle(pkg, oracle):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    o = oracle.OracleSolve(s, 0)
    p = o.run(400)[:, 0]
    sol = pkg.Solver(s, precision=1)
    sol.run(400)
    ref = {c: o.field(c) for c in FIELDS}
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= 1e-12
    assert field_rel_l2(mine, ref, "H") <= 1e-12
    assert rel(sol.probe_series()[:, 0], p) <= 1e-12
    assert rel(sol.dft(0), oracle.dft(p, s.dt, s.array("dft_freqs"))) <= 1e-12


@pytest.mark.parametrize("pump", ["0", "1e9"])
def test_c1_gain_slab_vs_oracle(pkg, oracle, pump):
    s = pkg.Setup.from_file(pkg.config_path("c1_gain_slab.params"), overrides={"PUMP_RATE": pump})
    rng = np.random.default_rng(1)
    o = oracle.OracleSolve(s, 0)
    init = {c: rng.normal(0.0, 1e-6, o.E[0].size) for c in ("Ex", "Ey", "Ez")}
    for c, v in init.items():
        o.E["xyz".index(c[1])][:] = v
    steps = 120
    o.run(steps)
    for precision, tol in ((1, 1e-12), (0, 1e-5)):
        sol = pkg.Solver(s, precision=precision)
        for c, v in init.items():
            sol.set_field(c, v.reshape(sol.shape))
        sol.run(steps)
        ref = {c: o.field(c) for c in FIELDS}
        mine = fields(sol)
        assert field_rel_l2(mine, ref, "E") <= tol, precision
        assert field_rel_l2(mine, ref, "H") <= tol, precision
        gain = s.array("tls_region_map").reshape(sol.shape) >= 0
        assert rel(sol.tls_state("Pz")[gain], o.Pz.reshape(sol.shape)[gain]) <= max(tol, 1e-5)
        assert rel(sol.tls_state("Nu")[gain], o.Nu.reshape(sol.shape)[gain]) <= (1e-12 if precision else 1e-5)
        sol.close()


def test_split_runs_equal_one_run(pkg):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params")
    a = pkg.Solver(s, precision=0)
    a.run(37)
    b = pkg.Solver(s, precision=0)
    b.run(17)
    b.run(20)
    assert a.steps_done == b.steps_done == 37
    for c in FIELDS:
        assert np.array_equal(a.field(c), b.field(c)), c
    for c in ("Pz", "Pz_prev", "Nu", "Ng"):
        assert np.array_equal(a.tls_state(c), b.tls_state(c)), c
    assert np.array_equal(a.probe_series(), b.probe_series())


@pytest.mark.parametrize("precision", [0, 1])
def test_field_and_state_round_trip(pkg, precision):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params")
    sol = pkg.Solver(s, precision=precision)
    rng = np.random.default_rng(5)
    for c in FIELDS:
        v = rng.normal(size=sol.shape)
        sol.set_field(c, v)
        got = sol.field(c)
        want = v if precision == 1 else v.astype(np.float32).astype(np.float64)
        assert np.array_equal(got, want), c
    gain = s.array("tls_region_map").reshape(sol.shape) >= 0
    v = rng.normal(size=sol.shape)
    sol.set_tls_state("Nu", v)
    got = sol.tls_state("Nu")
    want = v if precision == 1 else v.astype(np.float32).astype(np.float64)
    assert np.array_equal(got[gain], want[gain]) and np.all(got[~gain] == 0)


def test_monitor_stops_on_nan(pkg):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    sol = pkg.Solver(s, precision=0)
    ez = np.zeros(sol.shape)
    ez[40, 40, 40] = np.nan
    sol.set_field("Ez", ez)
    with pytest.raises(pkg.FdtdError) as e:
        sol.run(50)
    assert e.value.code == pkg.FDTD_ERR_UNSTABLE
    d = sol.diagnostics()
    assert d["stable"] == 0 and d["step"] == 0 and (d["nan_flags"] & 1)
    assert sol.steps_done == 1
    with pytest.raises(pkg.FdtdError):
        sol.run(5)  # the handle stays stopped, like the reference's early return


def test_monitor_counts_threshold_warnings(pkg):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"),
                            overrides={"STABILITY_MAX_E": "1e-300", "STABILITY_MONITOR_INTERVAL": "10"})
    sol = pkg.Solver(s, precision=0)
    with pytest.raises(pkg.FdtdError) as e:
        sol.run(300)
    assert e.value.code == pkg.FDTD_ERR_UNSTABLE
    d = sol.diagnostics()
    # > 10 warnings: the 11th monitor step (n = 100) is fatal in StabilityMonitor::check_stability
    assert d["instability_count"] == 11 and d["step"] == 100 and sol.steps_done == 101


def test_diagnostics_match_oracle_integrals(pkg, oracle):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params",
                            overrides={"STABILITY_MONITOR_INTERVAL": "10"})
    o = oracle.OracleSolve(s, 0)
    o.run(31)  # last monitor step of a 40-step run is n = 30
    sol = pkg.Solver(s, precision=1)
    sol.run(40)
    d = sol.diagnostics()
    assert d["step"] == 30 and d["stable"] == 1
    shape = sol.shape
    dV = (s.array("dx")[:, None, None] * s.array("dy")[None, :, None] * s.array("dz")[None, None, :]).ravel()
    gain = s.array("tls_region_map") >= 0
    assert abs(d["integrated_Nu"] - np.sum(o.Nu[gain] * dV[gain])) <= 1e-10 * abs(np.sum(o.Nu[gain] * dV[gain]))
    assert abs(d["integrated_Ng"] - np.sum(o.Ng[gain] * dV[gain])) <= 1e-10 * abs(np.sum(o.Ng[gain] * dV[gain]))
    pe = np.sum(-0.5 * o.Pz[gain] * o.E[2][gain] * dV[gain])
    assert abs(d["polarization_energy"] - pe) <= 1e-9 * abs(pe)
    maxE = max(np.abs(o.E[q]).max() for q in range(3))
    assert abs(d["max_E"] - maxE) <= 1e-12 * maxE
    N0 = np.where(gain, 1e24, 0.0)
    cons = abs(np.sum((o.Nu + o.Ng)[gain]) - np.sum(N0[gain])) / np.sum(N0[gain])
    assert abs(d["conservation_err"] - cons) <= 1e-9 + 1e-6 * cons
    assert sol.kernel_launches > 0 and sol.device_bytes > 0
    del shape


@pytest.mark.parametrize("precision", [0, 1, 3])
def test_kernel_paths_agree(pkg, precision):
    """The slab-ordered step (path 2) and the separate sweeps (path 1) run the same block code
    with explicitly rounded arithmetic: fields, gain state and probe series are bit-identical."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params", overrides={"PUMP_RATE": "1e11"})
    out = []
    for path in (1, 2):
        sol = pkg.Solver(s, precision=precision, kernel_path=path)
        rng = np.random.default_rng(11)
        for c in ("Ex", "Ey", "Ez"):
            sol.set_field(c, rng.normal(0, 1e-3, sol.shape))
        sol.run(33)
        out.append((fields(sol), {c: sol.tls_state(c) for c in ("Pz", "Nu", "Ng")}, sol.probe_series()))
        sol.close()
    (f1, g1, p1), (f2, g2, p2) = out
    for c in FIELDS:
        assert np.array_equal(f1[c], f2[c]), c
    for c in g1:
        assert np.array_equal(g1[c], g2[c]), c
    assert np.array_equal(p1, p2)


@pytest.mark.parametrize("path", [1, 2])
@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_sweep_paths_match_reference(pkg, precision, tol, path):
    g, s, _ = golden_solver(pkg, "step_g0_sphere", precision)
    sol = pkg.Solver(s, precision=precision, kernel_path=path)
    sol.run(g["meta"]["steps"])
    ref = ref_fields(g, sol.shape)
    mine = fields(sol)
    assert field_rel_l2(mine, ref, "E") <= tol and field_rel_l2(mine, ref, "H") <= tol


def test_kernel_path_fixed_after_first_step(pkg):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g0_sphere.params")
    sol = pkg.Solver(s)
    sol.run(1)
    with pytest.raises(pkg.FdtdError):
        sol.set_kernel_path(1)


@pytest.mark.parametrize("path,planes", [(1, ""), (2, "1"), (2, "3"), (2, "4")])
def test_tile_edges_on_odd_grid(pkg, oracle, path, planes, monkeypatch):
    """A grid that is not a multiple of the sweeps' row segments or of the slab-ordered step's
    slab in any axis, CPML on every face; the slab-ordered step with 1, 3 and 4 planes per slab."""
    if planes:
        monkeypatch.setenv("FDTD_B200_SLAB_PLANES", planes)
    text = (GOLDEN / "cases" / "step_g0_sphere.params").read_text()
    text = text.replace("NX = 10", "NX = 71").replace("NY = 9", "NY = 37").replace("NZ = 8", "NZ = 45")
    text = text.replace("DOMAIN_X_MAX = 250e-9", "DOMAIN_X_MAX = 1775e-9").replace("DOMAIN_Y_MAX = 225e-9", "DOMAIN_Y_MAX = 925e-9")
    text = text.replace("DOMAIN_Z_MAX = 200e-9", "DOMAIN_Z_MAX = 1125e-9")
    s = pkg.Setup.from_text(text)
    o = oracle.OracleSolve(s, 0)
    o.run(80)
    for precision, tol in ((1, 1e-12), (0, 1e-5)):
        sol = pkg.Solver(s, precision=precision, kernel_path=path)
        sol.run(80)
        ref = {c: o.field(c) for c in FIELDS}
        mine = fields(sol)
        assert field_rel_l2(mine, ref, "E") <= tol, precision
        assert field_rel_l2(mine, ref, "H") <= tol, precision


# Measured against the FP64 solve (one B200): on the 64^3 sphere case FP16 storage keeps the
# DFT within 5e-4 and BF16 within 3e-3, on the gain slab within 2e-2 and 3e-3; the late-time
# fields are not close (a static residual of the near field's rounding, about 1e-3 of the
# pulse peak, against a field that has decayed 5000-fold).
@pytest.mark.parametrize("precision,cfg,tol", [(2, "c0_dipole_sphere.params", 2e-3), (3, "c0_dipole_sphere.params", 6e-3),
                                               (2, "c1_gain_slab.params", 5e-2), (3, "c1_gain_slab.params", 1e-2)])
def test_16bit_storage_spectrum(pkg, precision, cfg, tol):
    overrides = {"PUMP_RATE": "0"} if cfg.startswith("c1") else {}
    s = pkg.Setup.from_file(pkg.config_path(cfg), overrides=overrides)
    out = []
    for prec in (1, precision):
        sol = pkg.Solver(s, precision=prec)
        sol.run(2000)
        out.append((sol.dft(0), sol.probe_series()[:, 0], sol.diagnostics()))
        sol.close()
    (d64, p64, g64), (d16, p16, g16) = out
    assert g16["nan_flags"] == 0 and g16["stable"] == 1
    assert np.all(np.isfinite(p16))
    assert np.argmax(np.abs(d16)) == np.argmax(np.abs(d64))
    assert rel(d16, d64) <= tol


@pytest.mark.parametrize("precision", [0, 2])
def test_kernel_path_0_is_refused(pkg, precision):
    """Path 0 (one fused H+E launch per step) is reserved: it measured slower than the sweeps and
    is not built."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g0_sphere.params")
    sol = pkg.Solver(s, precision=precision)
    with pytest.raises(pkg.FdtdError) as e:
        sol.set_kernel_path(0)
    assert e.value.code == 7


@pytest.mark.parametrize("precision,path", [(0, 1), (1, 1), (3, 1), (0, 2), (1, 2)])
def test_material_index_matches_arrays(pkg, precision, path, monkeypatch):
    """The indexed material (a uint16 row number per cell and a table of distinct rows), as the
    setup view brings it or as the stepper derives it from the arrays, gives bit-identical
    fields to the three bE arrays: the same values reach the same arithmetic."""
    monkeypatch.setenv("FDTD_B200_E_PIPE", "0")
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g2_planewave.params")
    assert s.view.n_bE_rows > 0
    bare = pkg.SetupV1.from_buffer_copy(s.view)
    bare.n_bE_rows = 0
    bare.bE_rows = None
    bare.bE_index = None
    out = []
    for mode, view in (("1", None), ("1", bare), ("0", None)):
        monkeypatch.setenv("FDTD_B200_MATERIAL_INDEX", mode)
        sol = pkg.Solver(s, precision=precision, kernel_path=path, view=view)
        assert (sol.material_rows == s.view.n_bE_rows) == (mode == "1")
        sol.run(45)
        out.append(fields(sol))
        sol.close()
    for c in FIELDS:
        assert np.array_equal(out[0][c], out[2][c]) and np.array_equal(out[1][c], out[2][c]), c


@pytest.mark.parametrize("precision", [1, 0, 2, 3])
@pytest.mark.parametrize("case", ["step_g2_planewave", "step_g1_gain", "step_g3_pec"])
def test_staged_sweeps_match_direct_loads(pkg, precision, case, monkeypatch):
    """The sweeps whose interior columns stage their planes in shared memory (cp.async, two
    stages for 32/64-bit storage, four for 16-bit) against the same sweeps loading straight
    from global memory: the same explicitly rounded update, so bit-identical fields."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"))
    out = []
    for mode in ("1", "0"):
        monkeypatch.setenv("FDTD_B200_E_PIPE", mode)
        monkeypatch.setenv("FDTD_B200_H_PIPE", mode)
        sol = pkg.Solver(s, precision=precision, kernel_path=1)
        rng = np.random.default_rng(5)
        for c in ("Ex", "Ey", "Ez"):
            sol.set_field(c, rng.normal(0, 1e-3, sol.shape))
        sol.run(40)
        out.append(fields(sol))
        sol.close()
    for c in FIELDS:
        assert np.array_equal(out[0][c], out[1][c]), c


@pytest.mark.parametrize("precision,path", [(1, 1), (0, 1), (2, 1), (3, 1), (1, 2), (0, 2)])
@pytest.mark.parametrize("case", ["step_g2_planewave", "step_g1_gain", "step_g3_pec", "c0_dipole_sphere"])
def test_interior_lane_widths_give_identical_bits(pkg, precision, path, case, monkeypatch):
    """Interior warps of 32-lane rows, two 16-lane rows or four 8-lane rows (FDTD_B200_LANES):
    the same cells get the same explicitly rounded update, x-neighbours come from the shuffle
    inside a row segment or from memory at its ends, rows past the grid edge ride along as
    inactive lanes -- bit-identical fields.  The small cases have 2-3 interior vectors per row and
    odd row counts (rows of a warp beyond the grid); c0 has 16 or 32 per row."""
    src = GOLDEN / "cases" / (case + ".params") if case.startswith("step") else pkg.config_path(case + ".params")
    s = pkg.Setup.from_file(src)
    steps = 60 if case.startswith("step") else 150
    out = []
    for lanes in ("32", "16", "8"):
        monkeypatch.setenv("FDTD_B200_LANES", lanes)
        sol = pkg.Solver(s, precision=precision, kernel_path=path)
        rng = np.random.default_rng(11)
        for c in ("Ex", "Ey", "Ez"):
            sol.set_field(c, rng.normal(0, 1e-3, sol.shape))
        sol.run(steps)
        out.append((fields(sol), sol.probe_series()))
        sol.close()
    for k in (1, 2):
        for c in FIELDS:
            assert np.array_equal(out[k][0][c], out[0][0][c]), (k, c)
        assert np.array_equal(out[k][1], out[0][1]), k


def test_lane_width_setting_is_checked(pkg, monkeypatch):
    monkeypatch.setenv("FDTD_B200_LANES", "12")
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g3_pec.params")
    with pytest.raises(pkg.FdtdError):
        pkg.Solver(s, precision=0)


def _bf16_run(pkg, s, rounding, steps, path=1):
    v = pkg.SetupV1.from_buffer_copy(s.view)
    v.rounding = rounding
    sol = pkg.Solver(s, precision=3, view=v, kernel_path=path)
    sol.run(steps)
    out = (fields(sol), sol.dft(0), sol.diagnostics())
    sol.close()
    return out


def test_bf16_stochastic_rounding_is_deterministic_and_active(pkg):
    """ROUNDING = stochastic: the same solve twice gives the same fields (the random bits are a
    hash of cell, array and step); the fields differ from round-to-nearest; the kernel paths
    (two sweeps, slab-ordered step) give the same bits."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params")
    a = _bf16_run(pkg, s, 1, 60)
    b = _bf16_run(pkg, s, 1, 60)
    c = _bf16_run(pkg, s, 0, 60)
    d = _bf16_run(pkg, s, 1, 60, path=2)
    for k in FIELDS:
        assert np.array_equal(a[0][k], b[0][k]), k
    assert any(not np.array_equal(a[0][k], c[0][k]) for k in FIELDS)
    assert field_rel_l2(a[0], c[0], "E") <= 2e-2
    for k in FIELDS:
        assert np.array_equal(a[0][k], d[0][k]), k


# Measured (one B200): on the 80^3 sphere and the gain slab stochastic rounding keeps the DFT
# within the round-to-nearest bars of test_16bit_storage_spectrum.
@pytest.mark.parametrize("cfg,tol", [("c0_dipole_sphere.params", 6e-3), ("c1_gain_slab.params", 1e-2)])
def test_bf16_stochastic_rounding_spectrum(pkg, cfg, tol):
    overrides = {"PUMP_RATE": "0"} if cfg.startswith("c1") else {}
    s = pkg.Setup.from_file(pkg.config_path(cfg), overrides=overrides)
    sol = pkg.Solver(s, precision=1)
    sol.run(2000)
    d64 = sol.dft(0)
    sol.close()
    _, d16, g16 = _bf16_run(pkg, s, 1, 2000)
    assert g16["nan_flags"] == 0 and g16["stable"] == 1
    assert np.argmax(np.abs(d16)) == np.argmax(np.abs(d64))
    assert rel(d16, d64) <= tol


def test_bounded_device_wait_expires_with_timeout_status(pkg, monkeypatch):
    """The slab-ordered step's dependency waits are bounded.  With the hold word left set (every
    E tile then waits on a word that nothing clears) and a 20 us bound, fdtd_run returns
    FDTD_ERR_TIMEOUT instead of hanging, the handle refuses further steps, it is destroyed
    cleanly, and a new handle on the same device steps normally.  No GPU fault is involved:
    the kernel gives up, flags the status word and returns."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g0_sphere.params")
    monkeypatch.setenv("FDTD_B200_WAIT_NS", "20000")
    monkeypatch.setenv("FDTD_B200_SLAB_HOLD", "1")
    sol = pkg.Solver(s, precision=0, kernel_path=2)
    with pytest.raises(pkg.FdtdError) as e:
        sol.run(3)
    assert e.value.code == pkg.FDTD_ERR_TIMEOUT and "wait" in str(e.value)
    with pytest.raises(pkg.FdtdError) as e:
        sol.run(1)
    assert e.value.code == pkg.FDTD_ERR_TIMEOUT
    sol.close()
    monkeypatch.delenv("FDTD_B200_SLAB_HOLD")
    monkeypatch.delenv("FDTD_B200_WAIT_NS")
    g = golden("step_g0_sphere")
    sol = pkg.Solver(s, precision=0, kernel_path=2)
    sol.run(g["meta"]["steps"])
    assert field_rel_l2(fields(sol), ref_fields(g, sol.shape), "E") <= 1e-5
    sol.close()


def _lockstep(pkg, s, precisions, marks, init=None):
    """Solves of one setup in several storage forms, stepped together; at each step count of
    `marks` yields (step, {precision: (fields, probe series, DFT)})."""
    sols = {p: pkg.Solver(s, precision=p) for p in precisions}
    if init:
        for sol in sols.values():
            for c, v in init.items():
                sol.set_field(c, v.reshape(sol.shape))
    done = 0
    try:
        for m in marks:
            for sol in sols.values():
                sol.run(m - done)
            done = m
            yield m, {p: (fields(sol), sol.probe_series(), sol.dft(0)) for p, sol in sols.items()}
    finally:
        for sol in sols.values():
            sol.close()


# The timed workload's physics on its profiling-size grid (280^3: 256^3 core, 12-cell CPML, slab
# with a pumped gain layer).  FP32 against the FP64 mode, measured on a B200: 1000 steps 7.0e-6 /
# 3.4e-6 / 4.4e-6 / 3.9e-6 (E, H, probe, DFT); 2000 steps 1.2e-4 / 7.8e-5 / 3.0e-5 / 3.2e-5, when
# the pulse has left the grid and the rounding residual of its peak dominates the small field.
def test_timed_workload_fp32_against_fp64_2000_steps(pkg):
    s = pkg.Setup.from_file(pkg.config_path("b256_gain_slab.params"))
    for m, r in _lockstep(pkg, s, (1, 0), (1000, 2000)):
        (f64, p64, d64), (f32, p32, d32) = r[1], r[0]
        eE, eH, ep, ed = field_rel_l2(f32, f64, "E"), field_rel_l2(f32, f64, "H"), rel(p32, p64), rel(d32, d64)
        if m == 1000:
            assert max(eE, eH, ep, ed) <= 1e-5, (m, eE, eH, ep, ed)
        else:
            assert eE <= 3e-4 and eH <= 2e-4 and ep <= 1e-4 and ed <= 1e-4, (m, eE, eH, ep, ed)
        assert np.argmax(np.abs(d32)) == np.argmax(np.abs(d64))


@pytest.mark.xfail(strict=True, reason="FP32 storage floor: after 2000 steps the decayed field is small against the "
                                       "rounding of its peak (C0 E 3.6e-4, timed workload E 1.2e-4 against FP64); the "
                                       "oracle's FP32 twin shows the same, so the FP32 parity bar of 1e-5 field L2 holds "
                                       "only while the pulse is in the grid")
@pytest.mark.parametrize("cfg", ["c0_dipole_sphere.params", "b256_gain_slab.params"])
def test_fp32_fields_within_1e5_after_2000_steps(pkg, cfg):
    s = pkg.Setup.from_file(pkg.config_path(cfg))
    for _, r in _lockstep(pkg, s, (1, 0), (2000,)):
        assert field_rel_l2(r[0][0], r[1][0], "E") <= 1e-5 and field_rel_l2(r[0][0], r[1][0], "H") <= 1e-5


def test_c1_gain_slab_2000_steps_vs_oracle(pkg, oracle):
    """Config C1 (graded mesh, pumped gain layer, seeded field noise) for 2000 steps against the
    oracle: FP64 within 1e-12 on fields, polarization and populations; FP32 within 2e-5 on the
    fields (measured 9e-6 against the FP64 mode) and 1e-5 on the probe series and DFT."""
    import os
    s = pkg.Setup.from_file(pkg.config_path("c1_gain_slab.params"), overrides={"PUMP_RATE": "1e9"})
    rng = np.random.default_rng(1)
    o = oracle.OracleSolve(s, 0)
    init = {c: rng.normal(0.0, 1e-6, o.E[0].size) for c in ("Ex", "Ey", "Ez")}
    for c, v in init.items():
        o.E["xyz".index(c[1])][:] = v
    steps = 2000
    p_ref = o.run(steps, threads=os.cpu_count() or 1)
    ref = {c: o.field(c) for c in FIELDS}
    gain = s.array("tls_region_map").reshape(s.shape) >= 0
    d_ref = oracle.dft(p_ref[:, 0], s.dt, s.array("dft_freqs"))
    for m, r in _lockstep(pkg, s, (1, 0), (steps,), init=init):
        (f64, p64, d64), (f32, p32, d32) = r[1], r[0]
        assert field_rel_l2(f64, ref, "E") <= 1e-12 and field_rel_l2(f64, ref, "H") <= 1e-12
        assert rel(p64, p_ref.reshape(p64.shape)) <= 1e-12 and rel(d64, d_ref) <= 1e-12
        assert field_rel_l2(f32, ref, "E") <= 2e-5 and field_rel_l2(f32, ref, "H") <= 2e-5
        assert rel(p32, p_ref.reshape(p32.shape)) <= 1e-5 and rel(d32, d_ref) <= 1e-5
    sol = pkg.Solver(s, precision=1)
    for c, v in init.items():
        sol.set_field(c, v.reshape(sol.shape))
    sol.run(steps)
    assert rel(sol.tls_state("Pz")[gain], o.Pz.reshape(s.shape)[gain]) <= 1e-12
    assert rel(sol.tls_state("Nu")[gain], o.Nu.reshape(s.shape)[gain]) <= 1e-12
    assert rel(sol.tls_state("Ng")[gain], o.Ng.reshape(s.shape)[gain]) <= 1e-12
    sol.close()


# 16-bit storage against the FP64 mode while the pulse is in the grid (C0, 600 steps; measured on a
# B200: FP16 E 1.7e-3, H 2.1e-2, probe 1.3e-2, DFT 2.4e-3; BF16 E 1.2e-2, H 0.16, probe 2.3e-2, DFT
# 4.1e-3).  The 1e-3 field bar set for 16-bit storage is met by neither form (next test).
@pytest.mark.parametrize("precision,bars", [(2, (4e-3, 5e-2, 3e-2, 6e-3)), (3, (3e-2, 0.35, 5e-2, 1e-2))])
def test_16bit_fields_against_fp64_in_the_active_window(pkg, precision, bars):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    for _, r in _lockstep(pkg, s, (1, precision), (600,)):
        (f64, p64, d64), (f16, p16, d16) = r[1], r[precision]
        got = (field_rel_l2(f16, f64, "E"), field_rel_l2(f16, f64, "H"), rel(p16, p64), rel(d16, d64))
        assert all(g <= b for g, b in zip(got, bars)), got
        assert np.argmax(np.abs(d16)) == np.argmax(np.abs(d64))


@pytest.mark.xfail(strict=True, reason="16-bit storage rounds every stored E and H value to 11 (FP16) or 8 (BF16) "
                                       "significant bits: the field L2 against FP64 is 2e-3 to 0.2 even in the active "
                                       "window, above the 1e-3 bar set for 16-bit storage")
@pytest.mark.parametrize("precision", [2, 3])
def test_16bit_fields_within_1e3_in_the_active_window(pkg, precision):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    for _, r in _lockstep(pkg, s, (1, precision), (600,)):
        assert field_rel_l2(r[precision][0], r[1][0], "E") <= 1e-3 and field_rel_l2(r[precision][0], r[1][0], "H") <= 1e-3
