"""The ring-down analysis of bench.py --sweep-check (emission peak, growth rate, Q) on
synthetic probe series with known answers: a damped or growing sinusoid sampled at the
sweep cavities' time step, with the static offset, slow drift and noise that 16-bit storage
leaves in a probe series added."""
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402

DT = 3.8e-17  # the 96x96x64 cavities' time step at 20 nm cells, S = 0.99
N = 20000


@pytest.mark.parametrize("f,g", [(221.1e12, -4.0e12), (193.4e12, -2.0e12), (205.0e12, 0.5e12)])
@pytest.mark.parametrize("dirty", [False, True])
def test_ringdown_recovers_frequency_rate_and_q(f, g, dirty):
    t = np.arange(N) * DT
    x = np.exp(g * t) * np.sin(2 * np.pi * f * t + 0.3)
    if dirty:  # static residual, drift and noise, well below the ringing over the window
        rng = np.random.default_rng(1)
        x = x + 0.02 + 0.01 * t / t[-1] + 1e-3 * rng.standard_normal(N) * np.exp(g * t)
    f_est, g_est, q_est = bench.ringdown(x, DT, 4000 * DT)
    assert abs(f_est - f) <= 2e-4 * f
    assert abs(g_est - g) <= 0.02 * abs(g)
    if g < 0:
        assert q_est == pytest.approx(np.pi * f / -g, rel=0.02)
    else:
        assert q_est is None  # a growing field has no ring-down Q


def test_raw_rms_fit_would_be_fooled_by_a_static_residual():
    """Why the estimator band-passes: a static residual comparable to the late ringing (as
    16-bit storage leaves near the source) flattens a fit of the raw series' RMS; the
    band-passed fit ignores it."""
    t = np.arange(N) * DT
    f, g = 221.1e12, -4.0e12
    x = np.exp(g * t) * np.sin(2 * np.pi * f * t) + 3.0 * np.exp(g * t[-1])
    seg = x[4000:]
    per = int(round(1 / (f * DT)))
    nw = len(seg) // per
    rms = np.sqrt(np.mean(seg[:nw * per].reshape(nw, per) ** 2, axis=1))
    tw = (np.arange(nw) + 0.5) * per * DT
    g_raw = np.polyfit(tw, np.log(rms), 1)[0]
    _, g_est, _ = bench.ringdown(x, DT, 4000 * DT)
    assert abs(g_est - g) <= 0.02 * abs(g) and abs(g_raw - g) > 0.2 * abs(g)


def test_ringdown_ignores_a_noise_floor_and_lines_outside_the_band():
    """A low-Q ring-down (Q 46, as on the graded-mesh cavities) that decays into a white noise
    floor, with a strong rounding-noise line at 3000 THz: the peak comes from the source band
    and the rate from the part of the window above the floor."""
    dt = 2.19e-17
    n = 20000
    t = np.arange(n) * dt
    f, g = 194.7e12, -13.4e12
    rng = np.random.default_rng(7)
    x = np.exp(g * t) * np.sin(2 * np.pi * f * t) + 3e-4 * rng.standard_normal(n)
    x += 2e-3 * np.sin(2 * np.pi * 3000e12 * t)
    f_est, g_est, q_est = bench.ringdown(x, dt, 4000 * dt)
    assert abs(f_est - f) <= 2e-3 * f
    assert abs(g_est - g) <= 0.05 * abs(g)
    assert q_est == pytest.approx(np.pi * f / -g, rel=0.05)
