"""Packed multi-solve engine (fdtd_batch_*): solves of different grids, step counts and
physics resident together on one GPU, each result the same alone and in the mix."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = [  # (setup source, overrides, steps)
    (GOLDEN / "cases" / "step_g0_sphere.params", {}, 150),
    (GOLDEN / "cases" / "step_g1_gain.params", {"PUMP_RATE": "1e11"}, 120),
    (GOLDEN / "cases" / "step_g2_planewave.params", {}, 100),
    ("c0_dipole_sphere.params", {}, 300),
    ("c1_gain_slab.params", {"PUMP_RATE": "1e9"}, 210),
]


def _setup(pkg, src, ov):
    path = src if not isinstance(src, str) else pkg.config_path(src)
    return pkg.Setup.from_file(path, overrides=ov)


def _single(pkg, s, n):
    sol = pkg.Solver(s, precision=0, kernel_path=1)
    sol.run(n)
    out = (sol.probe_series(), sol.dft(0), sol.diagnostics())
    sol.close()
    return out


def _drain(pkg, b, tickets, rounds=400):
    for _ in range(rounds):
        if all(b.state(t)[0] in (pkg.JOB_DONE, pkg.JOB_FAILED) for t in tickets):
            return
        b.run(64)
    raise AssertionError("batch did not finish")


def _batch_results(pkg, setups):
    b = pkg.Batch(budget_bytes=8 << 30)
    tickets = [b.submit(s, n) for s, n in setups]
    r, q = b.run(1)
    assert r == len(setups) and q == 0  # all resident at once
    _drain(pkg, b, tickets)
    out = []
    for t, (s, n) in zip(tickets, setups):
        st, done = b.state(t)
        assert st == pkg.JOB_DONE and done == n
        out.append((b.probe_series(t), b.dft(t), b.diagnostics(t)))
        b.release(t)
    b.close()
    return out


def test_batch_result_is_the_same_alone_and_in_the_mix(pkg):
    """Bit for bit: a job's blocks run the same code whatever else is resident."""
    setups = [(_setup(pkg, src, ov), n) for src, ov, n in CASES]
    mixed = _batch_results(pkg, setups)
    for k, sn in enumerate(setups):
        (series, dft, diag), = _batch_results(pkg, [sn])
        assert np.array_equal(mixed[k][0], series) and np.array_equal(mixed[k][1], dft)
        assert mixed[k][2]["max_E"] == diag["max_E"]


def test_batch_matches_single_solves(pkg):
    """Against fdtd_create + fdtd_run, bit for bit: the packed kernels run the same block code
    with explicitly rounded arithmetic (every product, difference and fused multiply-add is an
    intrinsic, so no instantiation contracts differently), the same probe/DFT code, and the
    monitor's max |E| does not depend on the reduction order.  The monitor's FP64 integrals
    are sums in a different block order: 1e-12 relative."""
    setups = [(_setup(pkg, src, ov), n) for src, ov, n in CASES]
    got = _batch_results(pkg, setups)
    for (s, n), (series, dft, diag) in zip(setups, got):
        ref = _single(pkg, s, n)
        assert np.array_equal(series, ref[0]) and np.array_equal(dft, ref[1])
        assert diag["max_E"] == ref[2]["max_E"]
        for k in ("integrated_Nu", "integrated_Ng", "polarization_energy"):
            assert abs(diag[k] - ref[2][k]) <= 1e-12 * abs(ref[2][k]), k
        assert diag["step"] == ref[2]["step"] and diag["steps_done"] == n


@pytest.mark.parametrize("case", ["step_g0_sphere", "step_g2_planewave"])
def test_batch_matches_reference_golden(pkg, case):
    """Packed FP32 solves against the reference's own FP64 probe series (golden state of the
    dielectric-sphere and plane-wave cases, src/3D_FDTD_version008.cpp:269-328 replayed by the
    reference harness): within the single-solve FP32 bar, 1e-5 relative."""
    from conftest import golden
    g = golden(case)
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"))
    steps = g["meta"]["steps"]
    (series, dft, diag), = _batch_results(pkg, [(s, steps)])
    assert _rel(series, g["probe_series"].reshape(series.shape)) <= 1e-5
    assert diag["stable"] == 1


def test_batch_c0_matches_oracle(pkg, oracle):
    """A packed FP32 solve of the 80^3 sphere config against the oracle (the C restatement of
    the reference loop, FP64): probe series and DFT within 1e-5 relative."""
    s = _setup(pkg, "c0_dipole_sphere.params", {})
    ref = oracle.OracleSolve(s, 0).run(300)
    (series, dft, _), = _batch_results(pkg, [(s, 300)])
    assert _rel(series, ref.reshape(series.shape)) <= 1e-5
    assert _rel(dft, oracle.dft(ref[:, 0], s.dt, s.array("dft_freqs"))) <= 1e-5


def test_batch_gain_matches_oracle_at_fp32_storage_floor(pkg, oracle):
    """A packed FP32 solve with gain (pump 1e11, zero initial field) against the FP64 oracle.
    Here FP32 storage itself cannot reach 1e-5: the oracle's FP32 twin (the same formulas with
    FP32 storage) is 3.4e-5 from FP64 on the probe series.  The packed solve must be within
    1.5x of that floor (and below 5e-5), the DFT within 1e-5."""
    s = _setup(pkg, GOLDEN / "cases" / "step_g1_gain.params", {"PUMP_RATE": "1e11"})
    ref = oracle.OracleSolve(s, 0).run(120)
    twin = oracle.OracleSolve(s, 1).run(120)
    floor = _rel(twin, ref)
    (series, dft, _), = _batch_results(pkg, [(s, 120)])
    err = _rel(series, ref.reshape(series.shape))
    assert err <= min(5e-5, 1.5 * floor), (err, floor)


def test_batch_admits_by_memory_budget(pkg):
    s = _setup(pkg, "c0_dipole_sphere.params", {})
    single = _single(pkg, s, 100)
    b = pkg.Batch(budget_bytes=40 << 20)  # room for one 80^3 solve at a time
    tickets = [b.submit(s, 100) for _ in range(3)]
    r, q = b.run(1)
    assert (r, q) == (1, 2)
    assert [b.state(t)[0] for t in tickets] == [pkg.JOB_RESIDENT, pkg.JOB_QUEUED, pkg.JOB_QUEUED]
    _drain(pkg, b, tickets)
    first = b.probe_series(tickets[0])
    assert np.array_equal(first, single[0])
    for t in tickets[1:]:
        assert np.array_equal(b.probe_series(t), first)
    with pytest.raises(pkg.FdtdError) as e:
        b.submit(_setup(pkg, "c1_gain_slab.params", {}), 10)  # larger than the whole budget
    assert e.value.code == 2
    b.close()


def test_batch_unstable_job_fails_alone(pkg):
    good = _setup(pkg, "c0_dipole_sphere.params", {})
    bad = _setup(pkg, GOLDEN / "cases" / "step_g0_sphere.params", {"STABILITY_MAX_E": "1e-30"})
    ref = _single(pkg, good, 250)
    b = pkg.Batch(budget_bytes=8 << 30)
    tg, tb = b.submit(good, 250), b.submit(bad, 400)
    _drain(pkg, b, [tg, tb])
    st, done = b.state(tb)
    assert st == pkg.JOB_FAILED and done == 101  # 11th threshold warning at monitor step 100
    assert b.state(tg)[0] == pkg.JOB_DONE
    assert np.array_equal(b.probe_series(tg), ref[0])
    b.close()


def test_batch_rejects_fp64(pkg):
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g0_sphere.params", overrides={"PRECISION": "fp64"})
    b = pkg.Batch()
    with pytest.raises(pkg.FdtdError) as e:
        b.submit(s, 10)
    assert e.value.code == 7
    b.close()


def test_one_batch_per_device(pkg):
    """The per-solve records live in the device's constant memory: a second engine on the
    same device is refused while the first one lives, and allowed once it is closed."""
    b = pkg.Batch()
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Batch()
    assert e.value.code == 1
    b.close()
    pkg.Batch().close()


def _with_precision(s, precision):
    v = type(s.view).from_buffer_copy(s.view)
    v.precision = precision
    return v


def _batch_views(pkg, jobs):
    """jobs: (setup, view, steps); all resident at once; returns (series, dft, diagnostics)."""
    b = pkg.Batch(budget_bytes=8 << 30)
    tickets = [b.submit(s, n, view=v) for s, v, n in jobs]
    r, q = b.run(1)
    assert r == len(jobs) and q == 0
    _drain(pkg, b, tickets, rounds=4000)
    out = []
    for t, (s, v, n) in zip(tickets, jobs):
        st, done = b.state(t)
        assert st == pkg.JOB_DONE and done == n
        out.append((b.probe_series(t), b.dft(t), b.diagnostics(t)))
    b.close()
    return out


MIXED = [  # (setup source, overrides, steps, precision): all three storage forms and E kinds
    (GOLDEN / "cases" / "step_g0_sphere.params", {}, 150, 3),
    (GOLDEN / "cases" / "step_g1_gain.params", {"PUMP_RATE": "1e11"}, 120, 2),
    (GOLDEN / "cases" / "step_g2_planewave.params", {}, 100, 3),
    (GOLDEN / "cases" / "step_g2_planewave.params", {}, 90, 2),
    ("c0_dipole_sphere.params", {}, 300, 0),
    ("c1_gain_slab.params", {"PUMP_RATE": "1e9"}, 210, 3),
    ("c1_gain_slab.params", {"PUMP_RATE": "1e9", "ROUNDING": "stochastic"}, 200, 3),
]


@pytest.mark.parametrize("shape", [{}, {"FDTD_B200_BATCH_KCHUNK": "16", "FDTD_B200_BATCH_H_PIPE": "0",
                                      "FDTD_B200_BATCH_E_PIPE": "0"}])
def test_batch_mixed_storage_alone_and_in_the_mix(pkg, shape, monkeypatch):
    """FP32, FP16 and BF16 solves resident together: each storage form's blocks run in their
    own launch, and each job's results are bit-identical alone and in the mix (default launch
    shape: each solve's own z-chunks and staged sweeps; and 16-plane chunks, direct loads)."""
    for k, v in shape.items():
        monkeypatch.setenv(k, v)
    jobs = []
    for src, ov, n, prec in MIXED:
        s = _setup(pkg, src, ov)
        jobs.append((s, _with_precision(s, prec), n))
    mixed = _batch_views(pkg, jobs)
    for k, job in enumerate(jobs):
        (series, dft, diag), = _batch_views(pkg, [job])
        assert np.array_equal(mixed[k][0], series) and np.array_equal(mixed[k][1], dft), k
        assert mixed[k][2]["max_E"] == diag["max_E"] and diag["nan_flags"] == 0


def test_batch_lane_widths_give_identical_bits(pkg, monkeypatch):
    """The packed sweeps run each solve's blocks with its own interior row width: the mix with
    every solve on 32-lane rows and with the width each solve picks (8 or 16 lanes for these
    narrow interiors) gives the same bits."""
    jobs = []
    for src, ov, n, prec in MIXED:
        s = _setup(pkg, src, ov)
        jobs.append((s, _with_precision(s, prec), n))
    monkeypatch.setenv("FDTD_B200_LANES", "32")
    wide = _batch_views(pkg, jobs)
    monkeypatch.delenv("FDTD_B200_LANES")
    auto = _batch_views(pkg, jobs)
    for k in range(len(jobs)):
        assert np.array_equal(wide[k][0], auto[k][0]) and np.array_equal(wide[k][1], auto[k][1]), k
        assert wide[k][2]["max_E"] == auto[k][2]["max_E"], k


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


# The bars of test_16bit_storage_spectrum (the single-solve 16-bit forms against FP64):
# the packed 16-bit solves meet the same bars.
@pytest.mark.parametrize("precision,cfg,tol", [(3, "c0_dipole_sphere.params", 6e-3), (2, "c0_dipole_sphere.params", 2e-3),
                                               (3, "c1_gain_slab.params", 1e-2)])
def test_batch_16bit_spectrum_against_fp64(pkg, precision, cfg, tol):
    overrides = {"PUMP_RATE": "0"} if cfg.startswith("c1") else {}
    s = _setup(pkg, cfg, overrides)
    sol = pkg.Solver(s, precision=1)
    sol.run(2000)
    d64 = sol.dft(0)
    sol.close()
    (series, d16, diag), = _batch_views(pkg, [(s, _with_precision(s, precision), 2000)])
    assert diag["nan_flags"] == 0 and diag["stable"] == 1 and np.all(np.isfinite(series))
    assert np.argmax(np.abs(d16)) == np.argmax(np.abs(d64))
    assert _rel(d16, d64) <= tol


@pytest.mark.parametrize("precision", [3, 2])
def test_batch_16bit_matches_single_16bit_solve(pkg, precision):
    """Against fdtd_create + fdtd_run of the same BF16 / FP16 solve: the same explicitly rounded
    block code, so the probe series, DFT and max |E| are bit-identical."""
    s = _setup(pkg, "c1_gain_slab.params", {"PUMP_RATE": "1e9"})
    sol = pkg.Solver(s, precision=precision, kernel_path=1)
    sol.run(300)
    ref = (sol.probe_series(), sol.dft(0), sol.diagnostics())
    sol.close()
    (series, dft, diag), = _batch_views(pkg, [(s, _with_precision(s, precision), 300)])
    assert np.array_equal(series, ref[0]) and np.array_equal(dft, ref[1])
    assert diag["max_E"] == ref[2]["max_E"]
    assert diag["steps_done"] == 300


def test_batch_job_submitted_while_others_step_is_bit_identical(pkg):
    """Continuous batching: jobs submitted while others are resident and stepping are prepared
    by the admission thread (device state built on their own streams) and spliced into the
    packed step; each result is bit-identical to the same job run alone."""
    first = [(_setup(pkg, src, ov), n) for src, ov, n in CASES[:2]]
    late = [(_setup(pkg, src, ov), n) for src, ov, n in CASES[2:]]
    b = pkg.Batch(budget_bytes=8 << 30)
    t_first = [b.submit(s, n) for s, n in first]
    b.run(24)
    states = [b.state(t) for t in t_first]
    assert all(st == pkg.JOB_RESIDENT and 0 < done < n for (st, done), (_, n) in zip(states, first))
    t_late = [b.submit(s, n) for s, n in late]  # the first jobs are mid-run
    _drain(pkg, b, t_first + t_late)
    got = {}
    for t, (s, n) in zip(t_first + t_late, first + late):
        st, done = b.state(t)
        assert st == pkg.JOB_DONE and done == n
        got[t] = (b.probe_series(t), b.dft(t), b.diagnostics(t))
        b.release(t)
    b.close()
    for t, sn in zip(t_first + t_late, first + late):
        (series, dft, diag), = _batch_results(pkg, [sn])
        assert np.array_equal(got[t][0], series) and np.array_equal(got[t][1], dft)
        assert got[t][2]["max_E"] == diag["max_E"]


def test_batch_run_waits_for_the_prepared_jobs(pkg):
    """With nothing resident, fdtd_batch_run waits for the admission thread to prepare what can
    be admitted instead of returning without stepping; n_queued counts jobs queued or in
    preparation."""
    s = _setup(pkg, "c0_dipole_sphere.params", {})
    b = pkg.Batch(budget_bytes=8 << 30)
    t = b.submit(s, 40)
    r, q = b.run(8)
    assert r == 1 and q == 0
    st, done = b.state(t)
    assert st == pkg.JOB_RESIDENT and done == 8
    _drain(pkg, b, [t])
    assert b.state(t) == (pkg.JOB_DONE, 40)
    b.close()


def test_batch_lone_job_steps_the_same_solo_or_packed(pkg, monkeypatch):
    """A lone resident job is stepped with the single-solve launches (the tail of a stream);
    with FDTD_B200_BATCH_SOLO=0 it stays in the packed kernels: the same bits either way, and a
    job that the monitor stops fails at the same step."""
    good = _setup(pkg, "c0_dipole_sphere.params", {})
    bad = _setup(pkg, GOLDEN / "cases" / "step_g0_sphere.params", {"STABILITY_MAX_E": "1e-30"})
    out = []
    for mode in ("1", "0"):
        monkeypatch.setenv("FDTD_B200_BATCH_SOLO", mode)
        (series, dft, diag), = _batch_results(pkg, [(good, 250)])
        b = pkg.Batch(budget_bytes=8 << 30)
        tb = b.submit(bad, 400)
        _drain(pkg, b, [tb])
        out.append((series, dft, diag["max_E"], b.state(tb)))
        b.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
    assert out[0][3] == out[1][3] == (pkg.JOB_FAILED, 101)
