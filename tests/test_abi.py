"""The C-ABI library loads without a GPU, exports every symbol of include/fdtd_b200.h,
reports setup errors the way the header documents, and refuses to step without a device
(no CPU fallback)."""
import ctypes
import re

import pytest

from conftest import ROOT


def header_symbols():
    text = (ROOT / "include" / "fdtd_b200.h").read_text()
    return sorted(set(re.findall(r"\b(fdtd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_header_symbol(pkg):
    lib = ctypes.CDLL(str(pkg.library_path()))
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(pkg.EXPORTED_SYMBOLS) == syms


def test_parse_error_reports_message(pkg):
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Setup.from_text("MESH_MODE = 0\nNX = abc\n")
    assert e.value.code == 6 and "NX" in str(e.value)
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Setup.from_text("this line has no equals sign\n")
    assert e.value.code == 6
    with pytest.raises(pkg.FdtdError):
        pkg.Setup.from_text("MESH_MODE = 0\nSTRUCTURES += prism, 2.0, 0, 1, 0, 1, 0, 1\n")
    with pytest.raises(pkg.FdtdError) as e:  # PEC: the field grid ends 2 npml cells before the mesh
        pkg.Setup.from_text("MESH_MODE = 0\nNX = 20\nNY = 20\nNZ = 20\nBOUNDARY_TYPE = 0\n"
                            "DIPOLE_SOURCES += true, 210e-9, 50e-9, 50e-9, 1e-7, 193.4e12, 0, 2e-15, 0, 1.0, 1, 2\n")
    assert "outside the field grid" in str(e.value)


def test_rounding_key(pkg):
    """ROUNDING (build-only key): nearest (default) or stochastic, carried by the setup view."""
    text = "MESH_MODE = 0\nNX = 12\nNY = 12\nNZ = 12\nCPML_NPML = 2\nPRECISION = bf16\n"
    assert pkg.Setup.from_text(text).view.rounding == 0
    assert pkg.Setup.from_text(text + "ROUNDING = stochastic\n").view.rounding == 1
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Setup.from_text(text + "ROUNDING = up\n")
    assert e.value.code == 6 and "ROUNDING" in str(e.value)
    # fdtd_create checks the view before it looks for a device
    s = pkg.Setup.from_text(text)
    v = pkg.SetupV1.from_buffer_copy(s.view)
    v.rounding = 2
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Solver(s, view=v)
    assert e.value.code == 1 and "rounding" in str(e.value)


def test_unknown_setup_array_is_an_error(pkg):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"), mesh_only=True)
    with pytest.raises(pkg.FdtdError):
        s.array("no_such_array")


def test_create_without_device_fails_loudly(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"))
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Solver(s)
    assert e.value.code == pkg.FDTD_ERR_NO_DEVICE


def test_create_validates_view(pkg):
    s = pkg.Setup.from_file(pkg.config_path("c0_dipole_sphere.params"), mesh_only=True)
    v = pkg.SetupV1.from_buffer_copy(s.view)
    v.struct_size = 4
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Solver(s, view=v)
    assert e.value.code == 1
    v = pkg.SetupV1.from_buffer_copy(s.view)  # mesh-only setup has no bE arrays
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Solver(s, view=v)
    assert e.value.code == 1


def test_gpu_bake_fails_loudly_without_a_device(pkg):
    """BAKE = gpu bakes on a CUDA device or reports that it cannot; it never falls back silently."""
    text = (pkg.config_path("c0_dipole_sphere.params")).read_text() + "\nBAKE = gpu\n"
    try:
        s = pkg.Setup.from_text(text)
    except pkg.FdtdError as e:
        assert "CUDA device" in str(e)
    else:
        assert s.view.n_bE_rows > 0


def test_noalloc_scan_refusals_need_no_device(pkg):
    """fdtd_field_scan_noalloc checks its arguments before it touches a device: a precision
    other than FP32/FP64, a null pointer, an empty scan and a scan beyond the fixed scratch
    (FDTD_FIELD_SCAN_MAX_CELLS = 16384 x 16384 cells) are refused with FDTD_ERR_INVALID."""
    limit = 16384 * 16384
    cases = [(2, [1] * 6, 10, "precision"), (3, [1] * 6, 10, "precision"), (1, [1, 1, 0, 1, 1, 1], 10, "null"),
             (0, [1] * 6, 0, "empty"), (1, [1] * 6, limit + 1, "limit")]
    for precision, ptrs, n, word in cases:
        with pytest.raises(pkg.FdtdError) as e:
            pkg.field_scan_noalloc(precision, ptrs, n, 1)
        assert e.value.code == pkg.FDTD_ERR_INVALID and word in str(e.value), (precision, n)
    with pytest.raises(pkg.FdtdError) as e:
        pkg.field_scan_noalloc(1, [1] * 6, 10, 0)
    assert e.value.code == pkg.FDTD_ERR_INVALID
