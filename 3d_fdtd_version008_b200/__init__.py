"""Python binding of libfdtd_b200.so, the B200 Yee FDTD stepper.

The library replaces the time loop of XiaofengYuChina/3D_FDTD_version008
(src/3D_FDTD_version008.cpp:231-381) behind the C ABI declared in
include/fdtd_b200.h.  This module is a thin ctypes mirror of that ABI:

    setup = Setup.from_file("configs/c0_dipole_sphere.params")   # host C++ setup API
    solver = Solver(setup)                                        # resident state on cuda:0
    solver.run(2000)                                              # GPU stepping
    ez = solver.field("Ez")                                       # reference idx3 layout, FP64

Nothing here computes physics; every call goes through the compiled library, and
the stepper entry points fail with FdtdError when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
from typing import Dict, Optional, Sequence

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libfdtd_b200.so"
CONFIG_DIR = PKG_DIR / "configs"

FDTD_OK = 0
STATUS_NAMES = {
    0: "FDTD_OK", 1: "FDTD_ERR_INVALID", 2: "FDTD_ERR_OOM", 3: "FDTD_ERR_CUDA",
    4: "FDTD_ERR_UNSTABLE", 5: "FDTD_ERR_TIMEOUT", 6: "FDTD_ERR_PARSE",
    7: "FDTD_ERR_UNSUPPORTED", 8: "FDTD_ERR_NO_DEVICE", 9: "FDTD_ERR_IO",
}
FDTD_ERR_INVALID = 1
FDTD_ERR_UNSTABLE = 4
FDTD_ERR_TIMEOUT = 5
FDTD_ERR_UNSUPPORTED = 7
FDTD_ERR_NO_DEVICE = 8
PREC_FP32, PREC_FP64, PREC_FP16, PREC_BF16 = 0, 1, 2, 3
TIMING_OFF, TIMING_RUN, TIMING_KERNELS = 0, 1, 2
COMPONENTS = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5,
              "E_mag": 6, "H_mag": 7, "Sx": 8, "Sy": 9, "Sz": 10, "S_mag": 11}
TLS_STATE = {"Pz": 0, "Pz_prev": 1, "Nu": 2, "Ng": 3}

# Every exported symbol of include/fdtd_b200.h.
EXPORTED_SYMBOLS = (
    "fdtd_setup_parse", "fdtd_setup_view", "fdtd_setup_array_len", "fdtd_setup_array",
    "fdtd_setup_destroy", "fdtd_setup_write_outputs", "fdtd_create", "fdtd_set_field", "fdtd_get_field",
    "fdtd_set_tls_state", "fdtd_get_tls_state", "fdtd_run", "fdtd_steps_done",
    "fdtd_get_probe_series", "fdtd_get_dft", "fdtd_get_diagnostics", "fdtd_device_bytes",
    "fdtd_kernel_launches", "fdtd_set_timing", "fdtd_get_timing", "fdtd_set_kernel_path", "fdtd_synchronize", "fdtd_last_error",
    "fdtd_destroy", "fdtd_field_scan_noalloc", "fdtd_attach_outputs", "fdtd_flush_outputs", "fdtd_material_rows",
    "fdtd_create_sharded",
    "fdtd_close_outputs",
    "fdtd_batch_create", "fdtd_batch_submit", "fdtd_batch_run", "fdtd_batch_job_state",
    "fdtd_batch_probe_series", "fdtd_batch_dft", "fdtd_batch_diagnostics", "fdtd_batch_release",
    "fdtd_batch_last_error", "fdtd_batch_destroy",
)
JOB_QUEUED, JOB_RESIDENT, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class FdtdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_dptr = C.POINTER(C.c_double)


class DipoleV1(C.Structure):
    _fields_ = [("i", C.c_uint64), ("j", C.c_uint64), ("k", C.c_uint64), ("polarization", C.c_int32),
                ("waveform", C.c_int32), ("cell_area", C.c_double), ("I0", C.c_double), ("f0", C.c_double),
                ("tau", C.c_double), ("t0", C.c_double), ("t_shift", C.c_double)]


class TlsRegionV1(C.Structure):
    _fields_ = [("kapa_coeff", C.c_double), ("pa2", C.c_double), ("pa3", C.c_double), ("inv_dt", C.c_double),
                ("tau", C.c_double), ("hbar", C.c_double), ("omega_a", C.c_double), ("N0", C.c_double),
                ("pump_rate", C.c_double), ("enable_population_clamp", C.c_int32), ("reserved", C.c_int32)]


class ProbeV1(C.Structure):
    _fields_ = [("i", C.c_uint64), ("j", C.c_uint64), ("k", C.c_uint64), ("component", C.c_int32),
                ("reserved", C.c_int32)]


class SheetV1(C.Structure):
    _fields_ = [("axis", C.c_int32), ("comp", C.c_int32), ("plane", C.c_uint64), ("lo0", C.c_uint64),
                ("hi0", C.c_uint64), ("lo1", C.c_uint64), ("hi1", C.c_uint64), ("d", C.c_double),
                ("sign", C.c_double), ("waveform", C.c_int32), ("reserved", C.c_int32), ("E0", C.c_double),
                ("f0", C.c_double), ("tau", C.c_double), ("t0", C.c_double), ("t_shift", C.c_double)]


class SetupV1(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("precision", C.c_int32),
        ("NxT", C.c_uint64), ("NyT", C.c_uint64), ("NzT", C.c_uint64),
        ("npml", C.c_uint32), ("save_every", C.c_uint32), ("dt", C.c_double),
        ("dx", _dptr), ("dy", _dptr), ("dz", _dptr),
        ("inv_dx", _dptr), ("inv_dy", _dptr), ("inv_dz", _dptr),
        ("cpml_kappa", _dptr * 3), ("cpml_bE", _dptr * 3), ("cpml_cE", _dptr * 3),
        ("cpml_bH", _dptr * 3), ("cpml_cH", _dptr * 3),
        ("bE", _dptr * 3), ("aE", _dptr * 3), ("aH", _dptr * 3), ("bH", _dptr * 3),
        ("bH_uniform", C.c_double),
        ("n_dipoles", C.c_uint32), ("dipoles", C.POINTER(DipoleV1)),
        ("n_tls_regions", C.c_uint32), ("tls_regions", C.POINTER(TlsRegionV1)),
        ("tls_region_map", C.POINTER(C.c_int32)), ("tls_Nu", _dptr), ("tls_Ng", _dptr),
        ("n_probes", C.c_uint32), ("probes", C.POINTER(ProbeV1)),
        ("n_dft_freqs", C.c_uint32), ("dft_freqs", _dptr),
        ("monitor_interval", C.c_uint32), ("max_E", C.c_double), ("max_P", C.c_double),
        ("conservation_err", C.c_double), ("growth_rate", C.c_double),
        ("field_scale", C.c_double),
        ("n_sheets", C.c_uint32), ("sheets", C.POINTER(SheetV1)),
        ("pec_boundary", C.c_uint32), ("n_bE_rows", C.c_uint32),
        ("bE_rows", C.POINTER(C.c_double)), ("bE_index", C.POINTER(C.c_uint16)),
        ("rounding", C.c_uint32),
    ]


class DiagnosticsV1(C.Structure):
    _fields_ = [("step", C.c_uint64), ("steps_done", C.c_uint64), ("max_E", C.c_double), ("max_P", C.c_double),
                ("conservation_err", C.c_double), ("integrated_Nu", C.c_double), ("integrated_Ng", C.c_double),
                ("polarization_energy", C.c_double), ("nan_flags", C.c_uint32), ("instability_count", C.c_uint32),
                ("stable", C.c_int32), ("reserved", C.c_int32)]


class FieldScanV1(C.Structure):
    _fields_ = [("max_E", C.c_double), ("nan_flags", C.c_uint32), ("reserved", C.c_uint32)]


class TimingV1(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("run_ms", C.c_double), ("h_ms", C.c_double), ("e_ms", C.c_double),
                ("aux_ms", C.c_double)]


_lib: Optional[C.CDLL] = None


def library_path() -> pathlib.Path:
    return pathlib.Path(os.environ.get("FDTD_B200_LIB", str(LIB_PATH)))


def load_library() -> C.CDLL:
    """Load libfdtd_b200.so (built by build_library()); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing: run __graft_entry__.build() (make -C csrc)")
    lib = C.CDLL(str(path))
    vp = C.c_void_p
    sig = {
        "fdtd_setup_parse": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(vp), C.c_char_p, C.c_size_t]),
        "fdtd_setup_view": (C.c_int, [vp, C.POINTER(SetupV1)]),
        "fdtd_setup_array_len": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_uint64)]),
        "fdtd_setup_array": (C.c_int, [vp, C.c_char_p, _dptr, C.c_uint64]),
        "fdtd_setup_destroy": (None, [vp]),
        "fdtd_setup_write_outputs": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_size_t]),
        "fdtd_attach_outputs": (C.c_int, [vp, vp, C.c_char_p]),
        "fdtd_flush_outputs": (C.c_int, [vp]),
        "fdtd_material_rows": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fdtd_create_sharded": (C.c_int, [C.POINTER(SetupV1), C.c_int, C.POINTER(C.c_int), C.POINTER(vp)]),
        "fdtd_close_outputs": (C.c_int, [vp]),
        "fdtd_create": (C.c_int, [C.POINTER(SetupV1), C.c_int, C.POINTER(vp)]),
        "fdtd_set_field": (C.c_int, [vp, C.c_int, _dptr]),
        "fdtd_get_field": (C.c_int, [vp, C.c_int, _dptr]),
        "fdtd_set_tls_state": (C.c_int, [vp, C.c_int, _dptr]),
        "fdtd_get_tls_state": (C.c_int, [vp, C.c_int, _dptr]),
        "fdtd_run": (C.c_int, [vp, C.c_uint64]),
        "fdtd_steps_done": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fdtd_get_probe_series": (C.c_int, [vp, _dptr, C.c_uint64, C.POINTER(C.c_uint64)]),
        "fdtd_get_dft": (C.c_int, [vp, C.c_uint32, _dptr, _dptr]),
        "fdtd_get_diagnostics": (C.c_int, [vp, C.POINTER(DiagnosticsV1)]),
        "fdtd_device_bytes": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fdtd_kernel_launches": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
        "fdtd_set_timing": (C.c_int, [vp, C.c_int]),
        "fdtd_get_timing": (C.c_int, [vp, C.POINTER(TimingV1)]),
        "fdtd_set_kernel_path": (C.c_int, [vp, C.c_int]),
        "fdtd_synchronize": (C.c_int, [vp]),
        "fdtd_last_error": (C.c_char_p, [vp]),
        "fdtd_destroy": (None, [vp]),
        "fdtd_field_scan_noalloc": (C.c_int, [C.c_int, vp, vp, vp, vp, vp, vp, C.c_uint64, vp, vp]),
        "fdtd_batch_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(vp)]),
        "fdtd_batch_submit": (C.c_int, [vp, C.POINTER(SetupV1), C.c_uint64, C.POINTER(C.c_uint64)]),
        "fdtd_batch_run": (C.c_int, [vp, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
        "fdtd_batch_job_state": (C.c_int, [vp, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]),
        "fdtd_batch_probe_series": (C.c_int, [vp, C.c_uint64, _dptr, C.c_uint64, C.POINTER(C.c_uint64)]),
        "fdtd_batch_dft": (C.c_int, [vp, C.c_uint64, C.c_uint32, _dptr, _dptr]),
        "fdtd_batch_diagnostics": (C.c_int, [vp, C.c_uint64, C.POINTER(DiagnosticsV1)]),
        "fdtd_batch_release": (C.c_int, [vp, C.c_uint64]),
        "fdtd_batch_last_error": (C.c_char_p, [vp]),
        "fdtd_batch_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _as_dptr(a: np.ndarray):
    return a.ctypes.data_as(_dptr)


class Setup:
    """Host setup built by the library's C++ setup API from a runtime parameter file."""

    def __init__(self, handle: int, text: str):
        self._h = C.c_void_p(handle)
        self.text = text
        self.view = SetupV1()
        lib = load_library()
        rc = lib.fdtd_setup_view(self._h, C.byref(self.view))
        if rc != FDTD_OK:
            raise FdtdError(rc, "fdtd_setup_view failed")

    @classmethod
    def from_text(cls, text: str, mesh_only: bool = False) -> "Setup":
        lib = load_library()
        h = C.c_void_p()
        err = C.create_string_buffer(1024)
        rc = lib.fdtd_setup_parse(text.encode(), int(mesh_only), C.byref(h), err, len(err))
        if rc != FDTD_OK:
            raise FdtdError(rc, err.value.decode())
        return cls(h.value, text)

    @classmethod
    def from_file(cls, path, mesh_only: bool = False, overrides: Optional[Dict[str, str]] = None) -> "Setup":
        text = pathlib.Path(path).read_text()
        if overrides:
            text += "\n" + "\n".join(f"{k} = {v}" for k, v in overrides.items()) + "\n"
        return cls.from_text(text, mesh_only)

    @property
    def shape(self):
        return int(self.view.NxT), int(self.view.NyT), int(self.view.NzT)

    @property
    def dt(self) -> float:
        return float(self.view.dt)

    def array(self, name: str) -> np.ndarray:
        lib = load_library()
        n = C.c_uint64()
        rc = lib.fdtd_setup_array_len(self._h, name.encode(), C.byref(n))
        if rc != FDTD_OK:
            raise FdtdError(rc, f"unknown setup array {name!r}")
        out = np.empty(n.value, dtype=np.float64)
        rc = lib.fdtd_setup_array(self._h, name.encode(), _as_dptr(out), n.value)
        if rc != FDTD_OK:
            raise FdtdError(rc, f"fdtd_setup_array({name!r}) failed")
        return out

    def array3(self, name: str) -> np.ndarray:
        return self.array(name).reshape(self.shape)

    def write_outputs(self, out_dir) -> pathlib.Path:
        """The files the reference writes before its time loop, under out_dir/frames/<RUN_TAG>/."""
        err = C.create_string_buffer(1024)
        rc = load_library().fdtd_setup_write_outputs(self._h, str(out_dir).encode(), err, len(err))
        if rc != FDTD_OK:
            raise FdtdError(rc, err.value.decode())
        return pathlib.Path(out_dir)

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value and _lib is not None:
            _lib.fdtd_setup_destroy(self._h)
            self._h = None


class Solver:
    """One resident solve on one GPU (fdtd_create ... fdtd_destroy)."""

    def __init__(self, setup: Setup, device: int = 0, precision: Optional[int] = None,
                 view: Optional[SetupV1] = None, kernel_path: Optional[int] = None, shards: int = 1,
                 devices=None):
        """shards > 1: the solve split along z (fdtd_create_sharded), shard r on devices[r]
        (default: all on `device`)."""
        lib = load_library()
        v = view if view is not None else setup.view
        if precision is not None:
            v = SetupV1.from_buffer_copy(v)
            v.precision = int(precision)
        self.setup = setup
        self.view = v
        h = C.c_void_p()
        if shards > 1:
            devs = (C.c_int * shards)(*(devices if devices is not None else [device] * shards))
            rc = lib.fdtd_create_sharded(C.byref(v), int(shards), devs, C.byref(h))
        else:
            rc = lib.fdtd_create(C.byref(v), int(device), C.byref(h))
        if rc != FDTD_OK:
            raise FdtdError(rc, lib.fdtd_last_error(None).decode())
        self._h = h
        self.shape = (int(v.NxT), int(v.NyT), int(v.NzT))
        if kernel_path is not None:
            self.set_kernel_path(kernel_path)
        self.n_probes = int(v.n_probes)
        self.n_freqs = int(v.n_dft_freqs)

    def _check(self, rc: int, what: str):
        if rc != FDTD_OK:
            raise FdtdError(rc, f"{what}: {load_library().fdtd_last_error(self._h).decode()}")

    def run(self, n_steps: int) -> None:
        self._check(load_library().fdtd_run(self._h, int(n_steps)), "fdtd_run")

    @property
    def steps_done(self) -> int:
        n = C.c_uint64()
        self._check(load_library().fdtd_steps_done(self._h, C.byref(n)), "fdtd_steps_done")
        return n.value

    def field(self, comp) -> np.ndarray:
        c = COMPONENTS[comp] if isinstance(comp, str) else int(comp)
        out = np.empty(self.shape, dtype=np.float64)
        self._check(load_library().fdtd_get_field(self._h, c, _as_dptr(out)), "fdtd_get_field")
        return out

    def set_field(self, comp, values: np.ndarray) -> None:
        c = COMPONENTS[comp] if isinstance(comp, str) else int(comp)
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.shape)
        self._check(load_library().fdtd_set_field(self._h, c, _as_dptr(a)), "fdtd_set_field")

    def tls_state(self, which: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(load_library().fdtd_get_tls_state(self._h, TLS_STATE[which], _as_dptr(out)), "fdtd_get_tls_state")
        return out

    def set_tls_state(self, which: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.shape)
        self._check(load_library().fdtd_set_tls_state(self._h, TLS_STATE[which], _as_dptr(a)), "fdtd_set_tls_state")

    def probe_series(self) -> np.ndarray:
        lib = load_library()
        n = C.c_uint64()
        self._check(lib.fdtd_get_probe_series(self._h, None, 0, C.byref(n)), "fdtd_get_probe_series")
        out = np.empty((n.value, max(self.n_probes, 1)), dtype=np.float64)
        if n.value:
            self._check(lib.fdtd_get_probe_series(self._h, _as_dptr(out), n.value, C.byref(n)),
                        "fdtd_get_probe_series")
        return out[:, : self.n_probes]

    def dft(self, probe: int = 0) -> np.ndarray:
        re = np.empty(self.n_freqs, dtype=np.float64)
        im = np.empty(self.n_freqs, dtype=np.float64)
        self._check(load_library().fdtd_get_dft(self._h, probe, _as_dptr(re), _as_dptr(im)), "fdtd_get_dft")
        return re + 1j * im

    def diagnostics(self) -> Dict[str, float]:
        d = DiagnosticsV1()
        self._check(load_library().fdtd_get_diagnostics(self._h, C.byref(d)), "fdtd_get_diagnostics")
        return {name: getattr(d, name) for name, _ in DiagnosticsV1._fields_ if name != "reserved"}

    @property
    def device_bytes(self) -> int:
        n = C.c_uint64()
        self._check(load_library().fdtd_device_bytes(self._h, C.byref(n)), "fdtd_device_bytes")
        return n.value

    @property
    def material_rows(self) -> int:
        """Distinct bE rows when the material is held as a row index per cell, else 0."""
        n = C.c_uint64()
        self._check(load_library().fdtd_material_rows(self._h, C.byref(n)), "fdtd_material_rows")
        return n.value

    @property
    def kernel_launches(self) -> int:
        n = C.c_uint64()
        self._check(load_library().fdtd_kernel_launches(self._h, C.byref(n)), "fdtd_kernel_launches")
        return n.value

    def set_timing(self, mode: int) -> None:
        """0 off, 1 one event pair per run() call, 2 per-kernel events every step."""
        self._check(load_library().fdtd_set_timing(self._h, int(mode)), "fdtd_set_timing")

    def timing(self) -> Dict[str, float]:
        t = TimingV1()
        self._check(load_library().fdtd_get_timing(self._h, C.byref(t)), "fdtd_get_timing")
        return {"steps": t.steps, "run_ms": t.run_ms, "h_ms": t.h_ms, "e_ms": t.e_ms, "aux_ms": t.aux_ms}

    def set_kernel_path(self, path: int) -> None:
        """1 = separate H and E sweeps (default), 2 = slab-ordered step; before the first step (0 is refused)."""
        self._check(load_library().fdtd_set_kernel_path(self._h, int(path)), "fdtd_set_kernel_path")

    def synchronize(self) -> None:
        self._check(load_library().fdtd_synchronize(self._h), "fdtd_synchronize")

    def attach_outputs(self, out_dir, setup: Optional[Setup] = None) -> None:
        """Stream the reference's detector files (movie frames, point time series) to
        out_dir/frames/<RUN_TAG>/ while the solve steps; before the first step."""
        s = setup if setup is not None else self.setup
        self._check(load_library().fdtd_attach_outputs(self._h, s._h, str(out_dir).encode()), "fdtd_attach_outputs")

    def flush_outputs(self) -> None:
        self._check(load_library().fdtd_flush_outputs(self._h), "fdtd_flush_outputs")

    def close_outputs(self) -> None:
        """End-of-run files (last population frame, its metadata), then detach."""
        self._check(load_library().fdtd_close_outputs(self._h), "fdtd_close_outputs")

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().fdtd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Packed multi-solve engine (fdtd_batch_*): FP32, FP16 and BF16 solves queued on one GPU,
    admitted by device footprint under `budget_bytes`, stepped together with one launch per
    sweep and storage form.  One engine per device at a time in a process."""

    def __init__(self, device: int = 0, budget_bytes: int = 150 << 30):
        self._h = C.c_void_p()
        self._keep = {}  # ticket -> (Setup, view): must outlive the job
        rc = load_library().fdtd_batch_create(int(device), C.c_uint64(int(budget_bytes)), C.byref(self._h))
        if rc != FDTD_OK:
            raise FdtdError(rc, f"fdtd_batch_create: {load_library().fdtd_batch_last_error(None).decode()}")

    def _check(self, rc: int, what: str):
        if rc != FDTD_OK:
            raise FdtdError(rc, f"{what}: {load_library().fdtd_batch_last_error(self._h).decode()}")

    def submit(self, setup: Setup, n_steps: int, view: Optional[SetupV1] = None) -> int:
        v = SetupV1.from_buffer_copy(view if view is not None else setup.view)
        t = C.c_uint64()
        self._check(load_library().fdtd_batch_submit(self._h, C.byref(v), C.c_uint64(int(n_steps)), C.byref(t)),
                    "fdtd_batch_submit")
        self._keep[t.value] = (setup, v)
        return t.value

    def run(self, max_steps: int):
        r, q = C.c_uint32(), C.c_uint32()
        self._check(load_library().fdtd_batch_run(self._h, C.c_uint64(int(max_steps)), C.byref(r), C.byref(q)),
                    "fdtd_batch_run")
        return r.value, q.value

    def state(self, ticket: int):
        st, n = C.c_int(), C.c_uint64()
        self._check(load_library().fdtd_batch_job_state(self._h, C.c_uint64(ticket), C.byref(st), C.byref(n)),
                    "fdtd_batch_job_state")
        return st.value, n.value

    def probe_series(self, ticket: int) -> np.ndarray:
        n = C.c_uint64()
        self._check(load_library().fdtd_batch_probe_series(self._h, C.c_uint64(ticket), None, 0, C.byref(n)),
                    "fdtd_batch_probe_series")
        npr = int(self._keep[ticket][1].n_probes)
        out = np.zeros((n.value, max(npr, 1)))
        self._check(load_library().fdtd_batch_probe_series(self._h, C.c_uint64(ticket), _as_dptr(out), n.value,
                                                           C.byref(n)), "fdtd_batch_probe_series")
        return out

    def dft(self, ticket: int, probe: int = 0) -> np.ndarray:
        nf = int(self._keep[ticket][1].n_dft_freqs)
        re, im = np.zeros(nf), np.zeros(nf)
        self._check(load_library().fdtd_batch_dft(self._h, C.c_uint64(ticket), probe, _as_dptr(re), _as_dptr(im)),
                    "fdtd_batch_dft")
        return re + 1j * im

    def diagnostics(self, ticket: int) -> Dict[str, float]:
        d = DiagnosticsV1()
        self._check(load_library().fdtd_batch_diagnostics(self._h, C.c_uint64(ticket), C.byref(d)),
                    "fdtd_batch_diagnostics")
        return {name: getattr(d, name) for name, _ in DiagnosticsV1._fields_ if name != "reserved"}

    def release(self, ticket: int) -> None:
        self._check(load_library().fdtd_batch_release(self._h, C.c_uint64(ticket)), "fdtd_batch_release")
        self._keep.pop(ticket, None)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            load_library().fdtd_batch_destroy(self._h)
            self._h = C.c_void_p()

    # `with Batch(...) as b:` releases the device's engine even when the block raises
    def __enter__(self) -> "Batch":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
        self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def field_scan_noalloc(precision: int, fields, n: int, out_ptr: int, stream: int = 0) -> None:
    """fdtd_field_scan_noalloc: the monitor's field scan (max |E|, non-finite flags) over n
    cells of six caller-owned device arrays `fields` = (Ex, Ey, Ez, Hx, Hy, Hz) given as
    device addresses, into the 16-byte device record at out_ptr, on `stream`; allocates no
    device memory (for callers that cannot allocate).  Overlapping calls race."""
    ptrs = [C.c_void_p(int(p)) for p in fields]
    rc = load_library().fdtd_field_scan_noalloc(int(precision), *ptrs, C.c_uint64(int(n)), C.c_void_p(int(out_ptr)),
                                                C.c_void_p(int(stream)))
    if rc != 0:
        raise FdtdError(rc, (load_library().fdtd_last_error(None) or b"").decode())


def config_path(name: str) -> pathlib.Path:
    return CONFIG_DIR / name


def build_library(verbose: bool = False) -> pathlib.Path:
    """Compile csrc/ into lib/libfdtd_b200.so (nvcc for sm_100a, g++ for the host API)."""
    import subprocess
    out = subprocess.run(["make", "-C", str(PKG_DIR / "csrc"), "-j8"], capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"library build failed:\n{out.stdout}\n{out.stderr}")
    return LIB_PATH
