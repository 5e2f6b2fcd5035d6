"""The GPU subpixel bake (BAKE = gpu) against the host bake, which is itself bit-identical to
the reference's StructureScene::bake (tests/test_setup_parity.py): the bE arrays must match
bit for bit, and a solve stepped from either must give the same fields."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def random_scene() -> str:
    """Overlapping spheres, boxes and z-cylinders of several indices on a graded auto mesh."""
    rng = np.random.default_rng(21)
    lines = ["MESH_MODE = 1", "DOMAIN_X_MIN = 0", "DOMAIN_X_MAX = 900e-9", "DOMAIN_Y_MIN = 0", "DOMAIN_Y_MAX = 800e-9",
             "DOMAIN_Z_MIN = 0", "DOMAIN_Z_MAX = 700e-9", "LAMBDA0 = 1550e-9", "AUTO_MESH_DX_MAX = 40e-9",
             "AUTO_MESH_DX_MIN = 8e-9", "AUTO_MESH_MAX_GRADING_RATIO = 1.3", "MESH_OVERRIDE_ENABLED = false",
             "CPML_NPML = 4", "TLS_ENABLED = false", "N_STEPS = 30", "SAVE_EVERY = 5",
             "DIPOLE_SOURCES += true, 450e-9, 400e-9, 350e-9, 1e-7, 193.4e12, 0, 2e-15, 0, 1.0, 1, 2"]
    for q in range(120):
        n = float(rng.choice([1.5, 2.0, 2.5, 3.5]))
        kind = q % 3
        if kind == 0:
            c = rng.uniform([0, 0, 0], [900e-9, 800e-9, 700e-9])
            lines.append(f"STRUCTURES += sphere, {n}, {c[0]:.6e}, {c[1]:.6e}, {c[2]:.6e}, {rng.uniform(20e-9, 120e-9):.6e}, 0, 0, \"\"")
        elif kind == 1:
            lo = rng.uniform([0, 0, 0], [800e-9, 700e-9, 600e-9])
            hi = lo + rng.uniform(20e-9, 200e-9, 3)
            lines.append(f"STRUCTURES += box, {n}, {lo[0]:.6e}, {hi[0]:.6e}, {lo[1]:.6e}, {hi[1]:.6e}, {lo[2]:.6e}, {hi[2]:.6e}, \"\"")
        else:
            c = rng.uniform([0, 0], [900e-9, 800e-9])
            z0 = rng.uniform(0, 500e-9)
            lines.append(f"STRUCTURES += cylinder, {n}, {c[0]:.6e}, {c[1]:.6e}, {rng.uniform(20e-9, 100e-9):.6e}, {z0:.6e}, {z0 + rng.uniform(50e-9, 200e-9):.6e}, 0, \"\"")
    return "\n".join(lines) + "\n"


def case_text(case: str, pkg) -> str:
    if case == "random":
        return random_scene()
    if case.startswith("c0"):
        return pkg.config_path(case).read_text()
    return (GOLDEN / "cases" / (case + ".params")).read_text()


@pytest.mark.parametrize("case", ["step_g0_sphere", "step_g1_gain", "step_g2_planewave", "step_g3_pec",
                                  "c0_dipole_sphere.params", "random"])
def test_gpu_bake_is_bit_identical(pkg, case):
    text = case_text(case, pkg)
    host = pkg.Setup.from_text(text)
    gpu = pkg.Setup.from_text(text + "\nBAKE = gpu\n")
    for c in ("bEx", "bEy", "bEz"):
        a, b = host.array(c), gpu.array(c)
        assert a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64)), c
    assert host.view.bH_uniform == gpu.view.bH_uniform
    assert host.view.n_bE_rows == gpu.view.n_bE_rows
    assert not gpu.view.aE[0] and not gpu.view.bH[0]  # uniform: passed as NULL


def test_gpu_baked_solve_matches(pkg):
    text = random_scene()
    out = []
    for extra in ("", "\nBAKE = gpu\n"):
        sol = pkg.Solver(pkg.Setup.from_text(text + extra), precision=1)
        sol.run(30)
        out.append({c: sol.field(c) for c in FIELDS})
        sol.close()
    for c in FIELDS:
        assert np.array_equal(out[0][c], out[1][c]), c
