"""A solve split along z into shards (fdtd_create_sharded) against the same solve whole: the
shards run the same kernels with their global z offset and exchange one E and one H plane per
step, so fields, gain state, probe series and DFT must match bit for bit, and the monitor's
reductions (summed in another order) to rounding.  Here every shard is on device 0; on a
multi-GPU node the same code places shard r on devices[r] and the halo copies cross NVLink."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def setup_for(pkg, case):
    if case.endswith(".params") and not case.startswith("step_"):
        return pkg.Setup.from_file(pkg.config_path(case))
    return pkg.Setup.from_file(GOLDEN / "cases" / (case + ".params"))


def run(pkg, s, precision, shards, steps):
    sol = pkg.Solver(s, precision=precision, shards=shards)
    rng = np.random.default_rng(3)
    for c in ("Ex", "Ey", "Ez"):
        sol.set_field(c, rng.normal(0, 1e-3, sol.shape))
    sol.run(steps // 2)
    sol.run(steps - steps // 2)
    out = {c: sol.field(c) for c in FIELDS}
    if s.view.n_tls_regions:
        out.update({c: sol.tls_state(c) for c in ("Pz", "Pz_prev", "Nu", "Ng")})
    out["series"] = sol.probe_series()
    out["dft"] = sol.dft(0) if s.view.n_dft_freqs and s.view.n_probes else None
    out["diag"] = sol.diagnostics()
    out["steps"] = sol.steps_done
    sol.close()
    return out


@pytest.mark.parametrize("case,shards", [("step_g1_gain", 2), ("step_g1_gain", 3), ("step_g2_planewave", 2),
                                         ("step_g2_planewave", 4), ("c0_dipole_sphere.params", 3), ("step_g3_pec", 2),
                                         ("step_g3_pec", 3)])
@pytest.mark.parametrize("precision", [1, 0, 3])
def test_sharded_matches_whole_solve(pkg, case, shards, precision):
    s = setup_for(pkg, case)
    whole = run(pkg, s, precision, 1, 40)
    split = run(pkg, s, precision, shards, 40)
    for c in FIELDS + ("Pz", "Pz_prev", "Nu", "Ng"):
        if c in whole:
            assert np.array_equal(whole[c], split[c]), c
    assert np.array_equal(whole["series"], split["series"])
    if whole["dft"] is not None:
        assert np.array_equal(whole["dft"], split["dft"])
    assert split["steps"] == whole["steps"] == 40
    dw, ds = whole["diag"], split["diag"]
    assert dw["step"] == ds["step"] and dw["max_E"] == ds["max_E"] and dw["nan_flags"] == ds["nan_flags"]
    for k in ("integrated_Nu", "integrated_Ng"):
        assert abs(dw[k] - ds[k]) <= 1e-12 * max(abs(dw[k]), 1e-300) + 1e-300, k
    # a relative difference of two sums, itself at rounding level: compare absolutely
    assert abs(dw["conservation_err"] - ds["conservation_err"]) <= 1e-12


@pytest.mark.parametrize("precision,tol", [(1, 1e-12), (0, 1e-5)])
def test_sharded_pec_matches_reference(pkg, precision, tol):
    """PECBoundary split over 3 shards (each zeroes the faces of the planes it owns; the z faces
    belong to the end shards) against the reference's own golden state."""
    from conftest import field_rel_l2, golden
    g = golden("step_g3_pec")
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g3_pec.params")
    sol = pkg.Solver(s, precision=precision, shards=3)
    sol.run(g["meta"]["steps"])
    mine = {c: sol.field(c) for c in FIELDS}
    ref = {c: g[c].reshape(sol.shape) for c in FIELDS}
    assert field_rel_l2(mine, ref, "E") <= tol and field_rel_l2(mine, ref, "H") <= tol
    for c in ("Ex", "Ey", "Ez"):
        f = mine[c]
        assert not (f[0].any() or f[-1].any() or f[:, 0].any() or f[:, -1].any() or f[:, :, 0].any() or f[:, :, -1].any())
    sol.close()


def test_sharded_refusals(pkg):
    s = setup_for(pkg, "step_g1_gain")
    sol = pkg.Solver(s, shards=2)
    with pytest.raises(pkg.FdtdError):
        sol.set_kernel_path(0)
    sol.close()
    with pytest.raises(pkg.FdtdError):
        pkg.Solver(s, shards=40)  # fewer than 3 planes per shard


@pytest.mark.parametrize("case,shards", [("step_g1_gain", 3), ("c0_dipole_sphere.params", 2)])
def test_sharded_bf16_stochastic_rounding_matches_whole_solve(pkg, case, shards):
    """BF16 storage with stochastic rounding: the rounding is keyed by the global cell, so the
    shards round every value as the whole solve does -- bit-identical fields and results."""
    s = setup_for(pkg, case)
    v = pkg.SetupV1.from_buffer_copy(s.view)
    v.rounding = 1
    out = []
    for n in (1, shards):
        sol = pkg.Solver(s, precision=3, shards=n, view=v)
        sol.run(30)
        out.append({c: sol.field(c) for c in FIELDS})
        sol.close()
    for c in FIELDS:
        assert np.array_equal(out[0][c], out[1][c]), c
