"""TEST INFRASTRUCTURE ONLY -- Python access to the oracle.

Two checkers live under oracle/:
  * libfdtd_oracle.so -- the plain-C restatement of the reference time loop
    (fdtd_oracle.c), built by ``make -C oracle oracle`` (gcc only, no reference needed);
  * _ref/ref_harness -- the reference solver itself (its headers compiled where they
    lie), built by ``make -C oracle ref`` when the reference checkout is present.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs use
this module, and only as the checker or the timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import pathlib
import shutil
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

ORACLE_DIR = pathlib.Path(__file__).resolve().parent
ORACLE_LIB = ORACLE_DIR / "lib" / "libfdtd_oracle.so"
REF_HARNESS = ORACLE_DIR / "_ref" / "ref_harness"
REF_HARNESS_NATIVE = ORACLE_DIR / "_ref" / "ref_harness_native"
REF_HARNESS_NATIVE_V4 = ORACLE_DIR / "_ref" / "ref_harness_native_v4"


def host_has_avx512() -> bool:
    """True when this host's CPU runs x86-64-v4 code (AVX-512 F, BW, CD, DQ, VL)."""
    try:
        flags = next(ln for ln in open("/proc/cpuinfo") if ln.startswith("flags")).split()
    except (OSError, StopIteration):
        return False
    return all(f in flags for f in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))


def native_harness() -> pathlib.Path:
    """The timed build of the reference harness for this host: x86-64-v4 where the CPU has
    AVX-512, else x86-64-v3."""
    if REF_HARNESS_NATIVE_V4.exists() and host_has_avx512():
        return REF_HARNESS_NATIVE_V4
    return REF_HARNESS_NATIVE
# Where the reference's headers lie (only in the build container; the GPU hosts use the
# prebuilt harness): FDTD_REFERENCE_SRC, else the checkout's default location.
REF_SRC = pathlib.Path(os.environ.get("FDTD_REFERENCE_SRC", "/root/reference/3D_FDTD_version008/src"))

_dp = C.POINTER(C.c_double)


class OSource(C.Structure):
    _fields_ = [("i", C.c_uint64), ("j", C.c_uint64), ("k", C.c_uint64), ("comp", C.c_int32),
                ("waveform", C.c_int32), ("cell_area", C.c_double), ("I0", C.c_double), ("f0", C.c_double),
                ("tau", C.c_double), ("t0", C.c_double), ("t_shift", C.c_double)]


class OSheet(C.Structure):
    _fields_ = [("axis", C.c_int32), ("comp", C.c_int32), ("plane", C.c_uint64), ("lo0", C.c_uint64),
                ("hi0", C.c_uint64), ("lo1", C.c_uint64), ("hi1", C.c_uint64), ("d", C.c_double),
                ("sign", C.c_double), ("waveform", C.c_int32), ("reserved", C.c_int32), ("E0", C.c_double),
                ("f0", C.c_double), ("tau", C.c_double), ("t0", C.c_double), ("t_shift", C.c_double)]


class ORegion(C.Structure):
    _fields_ = [("kapa_coeff", C.c_double), ("pa2", C.c_double), ("pa3", C.c_double), ("inv_dt", C.c_double),
                ("tau", C.c_double), ("hbar", C.c_double), ("omega_a", C.c_double), ("N0", C.c_double),
                ("pump_rate", C.c_double), ("clamp", C.c_int32), ("reserved", C.c_int32)]


class OCase(C.Structure):
    _fields_ = [("NxT", C.c_uint64), ("NyT", C.c_uint64), ("NzT", C.c_uint64),
                ("npml", C.c_int32), ("n_src", C.c_int32), ("n_regions", C.c_int32), ("n_probes", C.c_int32),
                ("dt", C.c_double), ("bH", C.c_double),
                ("inv_dx", _dp), ("inv_dy", _dp), ("inv_dz", _dp), ("dx", _dp), ("dy", _dp), ("dz", _dp),
                ("kappa", _dp * 3), ("bEp", _dp * 3), ("cEp", _dp * 3), ("bHp", _dp * 3), ("cHp", _dp * 3),
                ("bE", _dp * 3), ("src", OSource * 8), ("regions", ORegion * 16),
                ("region_map", C.POINTER(C.c_int32)), ("probe_idx", C.c_uint64 * 16),
                ("probe_comp", C.c_int32 * 16), ("save_every", C.c_uint32), ("n_sheets", C.c_int32),
                ("sheets", OSheet * 2), ("pec", C.c_int32)]


class OState(C.Structure):
    _fields_ = [("E", _dp * 3), ("H", _dp * 3), ("Pz", _dp), ("Pz_prev", _dp), ("Nu", _dp), ("Ng", _dp)]


_lib = None


def build(ref: bool = True) -> None:
    """Build the C restatement, and the reference harness when the reference is present."""
    targets = ["oracle"] + (["ref"] if ref and REF_SRC.exists() else [])
    subprocess.run(["make", "-C", str(ORACLE_DIR), f"REF_SRC={REF_SRC}", *targets], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build(ref=False)
        _lib = C.CDLL(str(ORACLE_LIB))
        _lib.oracle_run.restype = C.c_int64
        _lib.oracle_run.argtypes = [C.POINTER(OCase), C.POINTER(OState), C.c_uint64, C.c_uint64, _dp, C.c_int,
                                    C.c_int]
        _lib.oracle_dft.restype = None
        _lib.oracle_dft.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_double, _dp, C.c_int,
                                    _dp, _dp]
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class OracleSolve:
    """A case plus its FP64 state arrays (idx3), built from a product setup view.

    ``setup`` is the product's Setup (its arrays are bit-identical to the reference's,
    which tests/test_setup_parity.py checks); the oracle only reads them."""

    def __init__(self, setup, precision: int = 0):
        v = setup.view
        self.shape = (int(v.NxT), int(v.NyT), int(v.NzT))
        N = int(np.prod(self.shape))
        self.precision = precision
        self.keep = []
        c = OCase()
        c.NxT, c.NyT, c.NzT = self.shape
        c.npml = int(v.npml)
        c.dt = float(v.dt)
        c.bH = float(setup.array("bHx")[0]) if v.bH[0] else float(v.bH_uniform)
        arrays = {}
        for n in ("inv_dx", "inv_dy", "inv_dz", "dx", "dy", "dz"):
            arrays[n] = np.ascontiguousarray(setup.array(n))
            setattr(c, n, _ptr(arrays[n]))
        for a, ax in enumerate("xyz"):
            for fld, nm in (("kappa", "cpml_k"), ("bEp", "cpml_bE"), ("cEp", "cpml_cE"), ("bHp", "cpml_bH"),
                            ("cHp", "cpml_cH")):
                arr = np.ascontiguousarray(setup.array(nm + ax))
                arrays[nm + ax] = arr
                getattr(c, fld)[a] = _ptr(arr)
            arr = np.ascontiguousarray(setup.array("bE" + ax))
            arrays["bE" + ax] = arr
            c.bE[a] = _ptr(arr)
        c.n_src = int(v.n_dipoles)
        for q in range(c.n_src):
            d = v.dipoles[q]
            c.src[q] = OSource(d.i, d.j, d.k, d.polarization % 3, d.waveform, d.cell_area, d.I0, d.f0, d.tau, d.t0,
                               d.t_shift)
        c.pec = int(v.pec_boundary)
        c.n_sheets = int(v.n_sheets)
        for q in range(c.n_sheets):
            w = v.sheets[q]
            c.sheets[q] = OSheet(w.axis, w.comp, w.plane, w.lo0, w.hi0, w.lo1, w.hi1, w.d, w.sign, w.waveform, 0,
                                 w.E0, w.f0, w.tau, w.t0, w.t_shift)
        c.n_regions = int(v.n_tls_regions)
        for q in range(c.n_regions):
            r = v.tls_regions[q]
            c.regions[q] = ORegion(r.kapa_coeff, r.pa2, r.pa3, r.inv_dt, r.tau, r.hbar, r.omega_a, r.N0, r.pump_rate,
                                   r.enable_population_clamp, 0)
        if c.n_regions:
            rm = np.ascontiguousarray(setup.array("tls_region_map").astype(np.int32))
            arrays["region_map"] = rm
            c.region_map = rm.ctypes.data_as(C.POINTER(C.c_int32))
        c.n_probes = int(v.n_probes)
        NyT, NzT = self.shape[1], self.shape[2]
        for q in range(c.n_probes):
            p = v.probes[q]
            c.probe_idx[q] = (p.i * NyT + p.j) * NzT + p.k
            c.probe_comp[q] = p.component
        c.save_every = max(1, int(v.save_every))
        self.case = c
        self.arrays = arrays
        self.E = [np.zeros(N) for _ in range(3)]
        self.H = [np.zeros(N) for _ in range(3)]
        self.gain = c.n_regions > 0
        self.Pz = np.zeros(N) if self.gain else None
        self.Pz_prev = np.zeros(N) if self.gain else None
        self.Nu = np.ascontiguousarray(setup.array("tls_Nu")) if self.gain else None
        self.Ng = np.ascontiguousarray(setup.array("tls_Ng")) if self.gain else None
        self.steps = 0
        self.freqs = np.ascontiguousarray(setup.array("dft_freqs"))

    def _state(self) -> OState:
        s = OState()
        for q in range(3):
            s.E[q] = _ptr(self.E[q])
            s.H[q] = _ptr(self.H[q])
        if self.gain:
            s.Pz, s.Pz_prev, s.Nu, s.Ng = _ptr(self.Pz), _ptr(self.Pz_prev), _ptr(self.Nu), _ptr(self.Ng)
        return s

    def run(self, nsteps: int, threads: int = 0) -> np.ndarray:
        """One call per run (CPML psi is not carried between calls).  Returns probe samples."""
        nprobe = max(1, self.case.n_probes)
        every = self.case.save_every
        nsamp = (self.steps + nsteps + every - 1) // every - (self.steps + every - 1) // every
        out = np.zeros((max(nsamp, 1), nprobe))
        st = self._state()
        got = lib().oracle_run(C.byref(self.case), C.byref(st), self.steps, nsteps, _ptr(out), self.precision,
                               threads)
        self.steps += nsteps
        return out[:got, : self.case.n_probes]

    def field(self, comp: str) -> np.ndarray:
        q = "xyz".index(comp[1])
        return (self.E if comp[0] == "E" else self.H)[q].reshape(self.shape)


def dft(series: np.ndarray, dt: float, freqs: np.ndarray, n0: int = 0, every: int = 1) -> np.ndarray:
    s = np.ascontiguousarray(series, dtype=np.float64)
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    re = np.zeros(len(f))
    im = np.zeros(len(f))
    lib().oracle_dft(_ptr(s), len(s), 1, n0, every, dt, _ptr(f), len(f), _ptr(re), _ptr(im))
    return re + 1j * im


def run_harness(params_path, steps: int, *flags: str, native: bool = False, init_dir: Optional[str] = None,
                outdir: Optional[str] = None, env: Optional[Dict[str, str]] = None) -> Dict[str, object]:
    """Run the reference harness; returns meta plus every array it wrote (name -> ndarray)
    and, under "frames", every file of its frames/ directory (relative path -> bytes).
    Without outdir it runs in a scratch directory under oracle/_ref/runs that is removed
    afterwards."""
    exe = native_harness() if native else REF_HARNESS
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is missing: build it with make -C oracle ref")
    scratch = outdir is None
    if scratch:
        (ORACLE_DIR / "_ref" / "runs").mkdir(parents=True, exist_ok=True)
    out = outdir or tempfile.mkdtemp(prefix="refh_", dir=str(ORACLE_DIR / "_ref" / "runs"))
    cmd = [str(exe), str(params_path), out, "--steps", str(steps), *flags]
    if init_dir:
        cmd += ["--init", init_dir]
    e = dict(os.environ)
    if env:
        e.update(env)
    subprocess.run(cmd, check=True, capture_output=True, env=e, cwd=out)
    meta = json.load(open(os.path.join(out, "meta.json")))
    res: Dict[str, object] = {"meta": meta, "dir": out}
    for f in os.listdir(out):
        if f.endswith(".f64"):
            res[f[:-4]] = np.fromfile(os.path.join(out, f), dtype=np.float64)
        elif f.endswith(".i32"):
            res[f[:-4]] = np.fromfile(os.path.join(out, f), dtype=np.int32)
    frames = pathlib.Path(out) / "frames"
    res["frames"] = {str(f.relative_to(frames)): f.read_bytes() for f in sorted(frames.rglob("*")) if f.is_file()}
    if scratch:
        shutil.rmtree(out, ignore_errors=True)
        del res["dir"]
    return res


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.linalg.norm(b.ravel()))
    return float(np.linalg.norm((a - b).ravel())) / (den if den > 0 else 1.0)
