"""Pins the oracle (plain-C restatement in oracle/fdtd_oracle.c) to the reference: its
FP64 time loop must reproduce the reference's golden state bit for bit, and (when the
reference checkout is here) the live reference harness as well."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def run_oracle(pkg, oracle, case, precision=0, overrides=None):
    g = golden(case)
    s = pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"), overrides=overrides)
    o = oracle.OracleSolve(s, precision=precision)
    seed = g["meta"].get("noise_seed")
    if seed is not None:
        sys.path.insert(0, str(GOLDEN))
        from make_golden import initial_noise
        init = initial_noise(case, int(np.prod(o.shape)))
        for c, v in init.items():
            assert oracle_sha(v) == g["meta"]["sha256_init_" + c]
            (o.E if c[0] == "E" else o.H)["xyz".index(c[1])][:] = v
    steps = g["meta"]["steps"]
    series = o.run(steps)
    return g, o, series


def oracle_sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", ["step_g0_sphere", "step_g1_gain", "step_g2_planewave", "step_g3_pec"])
def test_oracle_reproduces_reference_bit_for_bit(pkg, oracle, case):
    g, o, series = run_oracle(pkg, oracle, case)
    for c in FIELDS:
        assert np.array_equal(o.field(c).ravel(), g[c]), c
    assert np.array_equal(series.ravel(), g["probe_series"])
    if o.gain:
        for c in ("Pz", "Pz_prev", "Nu", "Ng"):
            assert np.array_equal(getattr(o, c), g[c]), c


def test_oracle_fp32_twin_drift_is_small(pkg, oracle):
    from conftest import field_rel_l2
    g, o, _ = run_oracle(pkg, oracle, "step_g0_sphere", precision=1)
    mine = {c: o.field(c) for c in FIELDS}
    assert field_rel_l2(mine, g, "E") < 1e-5
    assert field_rel_l2(mine, g, "H") < 1e-5


def test_oracle_pump_extension(pkg, oracle):
    """W_p > 0 (this library's extension) moves population upward at dt*W_p*Ng per step."""
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params", overrides={"PUMP_RATE": "1e12"})
    o = oracle.OracleSolve(s)
    nu0 = o.Nu.copy()
    o.run(3)
    gain = s.array("tls_region_map") >= 0
    assert np.all(o.Nu[gain] > nu0[gain])


def test_dft_helper_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    v = rng.normal(size=257)
    dt, f = 1e-17, np.array([1.9e14, 2.0e14])
    t = (np.arange(257) + 1) * dt
    ref = (v[None, :] * np.exp(-2j * np.pi * f[:, None] * t[None, :])).sum(axis=1) * dt
    assert np.allclose(oracle.dft(v, dt, f), ref, rtol=1e-12, atol=0)


def test_oracle_against_live_reference(pkg, oracle):
    if not oracle.REF_HARNESS.exists():
        pytest.skip("reference harness not built (no reference checkout on this machine)")
    p = pkg.config_path("c0_dipole_sphere.params")
    r = oracle.run_harness(p, 60)
    o = oracle.OracleSolve(pkg.Setup.from_file(p))
    series = o.run(60)
    for c in FIELDS:
        assert np.array_equal(o.field(c).ravel(), r[c]), c
    assert np.array_equal(series.ravel(), r["probe_series"])
