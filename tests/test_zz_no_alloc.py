"""fdtd_field_scan_noalloc: the stability monitor's field scan for callers that cannot
allocate device memory (an application running the stepper inside its own device pool or
arena, a callback under its allocator's lock, code whose watchdog treats an allocation as a
fault).  It must agree with the scan the stepper itself runs (fdtd_get_diagnostics after a
monitor step) on two calls in a row, with its scratch shared between the calls.

This file is named so that pytest collects it last."""
import numpy as np
import pytest

from conftest import GOLDEN

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _scan(pkg, torch, precision, arrays):
    dt = torch.float32 if precision == pkg.PREC_FP32 else torch.float64
    dev = [torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda:0", dtype=dt) for a in arrays]
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")  # 16-byte result record
    stream = torch.cuda.current_stream().cuda_stream
    pkg.field_scan_noalloc(precision, [t.data_ptr() for t in dev], dev[0].numel(), out.data_ptr(), stream)
    torch.cuda.synchronize()
    rec = out.cpu().numpy()
    return float(rec[0]), int(rec[1:].view(np.uint32)[0])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_scan_matches_monitor_on_two_calls(pkg, precision):
    import torch
    s = pkg.Setup.from_file(GOLDEN / "cases" / "step_g1_gain.params", overrides={"PUMP_RATE": "1e11"})
    sol = pkg.Solver(s, precision=precision)
    rng = np.random.default_rng(5)
    for c in ("Ex", "Ey", "Ez"):
        sol.set_field(c, rng.normal(0, 1e-3, sol.shape))
    for steps in (11, 21):  # the monitor runs after steps 0, 10, 20 (interval 10)
        sol.run(steps - sol.steps_done)
        d = sol.diagnostics()
        assert d["step"] == steps - 1
        got_max, got_flags = _scan(pkg, torch, precision, [sol.field(c) for c in FIELDS])
        assert got_max > 0.0
        assert abs(got_max - d["max_E"]) <= 1e-12 * d["max_E"], (steps, got_max, d["max_E"])
        assert got_flags == (d["nan_flags"] & 3) == 0
    sol.close()


@pytest.mark.gpu
def test_noalloc_scan_leaves_free_memory_unchanged(pkg):
    """The property the entry point exists for: once the inputs and the result record are on
    the device and a first call has loaded the kernels and looked up the scratch address,
    further calls change the device's free memory by nothing."""
    import torch
    rng = np.random.default_rng(3)
    n = 5 * 16384 + 11
    dev = [torch.from_numpy(rng.normal(0, 1.0, n)).to("cuda:0") for _ in FIELDS]
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    ptrs = [t.data_ptr() for t in dev]
    pkg.field_scan_noalloc(1, ptrs, n, out.data_ptr(), stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        pkg.field_scan_noalloc(1, ptrs, n, out.data_ptr(), stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert float(out[0].item()) == max(float(t.abs().max().item()) for t in dev[:3])


@pytest.mark.gpu
def test_noalloc_scan_flags_and_limit(pkg):
    import torch
    rng = np.random.default_rng(9)
    n = 3 * 16384 + 77  # several scratch records, ragged last block
    arrays = [rng.normal(0, 1.0, n) for _ in FIELDS]
    arrays[1][n - 5] = np.inf   # Ey: E flag, cell left out of max |E|
    arrays[4][123] = np.nan     # Hy: H flag
    keep = np.isfinite(arrays[0]) & np.isfinite(arrays[1]) & np.isfinite(arrays[2])
    want = max(np.abs(a[keep]).max() for a in arrays[:3])
    for _ in range(2):
        got_max, got_flags = _scan(pkg, torch, 1, arrays)
        assert got_max == want and got_flags == 3
    clean = [np.where(np.isfinite(a), a, 0.0) for a in arrays]
    got_max, got_flags = _scan(pkg, torch, 1, clean)
    assert got_flags == 0 and got_max == max(np.abs(a).max() for a in clean[:3])
    with pytest.raises(pkg.FdtdError) as e:  # beyond the scratch limit: refused before any launch
        pkg.field_scan_noalloc(1, [1] * 6, 16384 * 16384 + 1, 1)
    assert e.value.code == pkg.FDTD_ERR_INVALID and "limit" in str(e.value)
