// waveform.hpp -- source current waveforms, shared by the host setup and the stepper.
//
// compute_waveform (src/sources/isource.hpp:41-68) with the reference's FP64 operation
// order, so the per-step current density J(n) = I((n + 1/2) dt) / cell_area that the
// stepper passes to its E kernel is bit-identical to DipoleSource::inject_half_step
// (src/sources/dipole_source.hpp:60-85).
#pragma once

#include <cmath>
#include <numbers>

namespace fdtd {

// w: 0 Ricker, 1 GaussianModulatedSine, 2 RickerLikeGaussian2nd, 3 ContinuousWave.
inline double waveform_value(int w, double t, double I0, double f0, double tau, double t0, double t_shift) {
    const double pi = std::numbers::pi;
    switch (w) {
        case 0: {
            const double a = pi * f0 * (t - t0);
            const double a2 = a * a;
            return I0 * (1 - 2 * a2) * std::exp(-a2);
        }
        case 1: {
            const double x = (t - t0);
            return I0 * std::sin(2 * pi * f0 * (t - t_shift)) * std::exp(-(x * x) / (tau * tau));
        }
        case 2: {
            const double x = (t - t0) / tau;
            const double x2 = x * x;
            return I0 * (1 - 2 * x2) * std::exp(-x2);
        }
        case 3: {
            const double env = (t < tau) ? (0.5 * (1 - std::cos(pi * t / tau))) : 1.0;
            return I0 * env * std::sin(2 * pi * f0 * t);
        }
    }
    return 0;
}

// J(n): the value inject_half_step adds to J at step n.
inline double current_density(int w, std::size_t n, double dt, double I0, double f0, double tau, double t0,
                              double t_shift, double cell_area) {
    const double t_half = (static_cast<double>(n) + 0.5) * dt;
    return waveform_value(w, t_half, I0, f0, tau, t0, t_shift) / cell_area;
}

}  // namespace fdtd
