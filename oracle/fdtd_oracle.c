/* fdtd_oracle.c -- TEST INFRASTRUCTURE ONLY: plain-C restatement of the reference time
 * loop (see fdtd_oracle.h).  Each routine cites the reference function it restates and
 * keeps its loop bounds, branches and FP64 operation order.  Compiled with
 * -ffp-contract=off so that, in FP64, it matches the reference built the same way
 * bit for bit (checked by tests/test_oracle.py against oracle/_ref/ref_harness).
 */
#include "fdtd_oracle.h"

#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdlib.h>
#include <string.h>

#define IDX3(i, j, k, NyT, NzT) (((size_t)(i) * (NyT) + (size_t)(j)) * (NzT) + (size_t)(k))

/* compute_waveform (src/sources/isource.hpp:41-68) */
static double waveform_value(int w, double t, double I0, double f0, double tau, double t0, double t_shift) {
    const double pi = 3.141592653589793238462643383279502884;
    switch (w) {
        case 0: {
            const double a = pi * f0 * (t - t0);
            const double a2 = a * a;
            return I0 * (1 - 2 * a2) * exp(-a2);
        }
        case 1: {
            const double x = (t - t0);
            return I0 * sin(2 * pi * f0 * (t - t_shift)) * exp(-(x * x) / (tau * tau));
        }
        case 2: {
            const double x = (t - t0) / tau;
            const double x2 = x * x;
            return I0 * (1 - 2 * x2) * exp(-x2);
        }
        case 3: {
            const double env = (t < tau) ? (0.5 * (1 - cos(pi * t / tau))) : 1.0;
            return I0 * env * sin(2 * pi * f0 * t);
        }
    }
    return 0;
}

/* get_field_value (src/detectors/idetector.hpp:79-109) */
#define PROBE_VALUE(REAL, comp, id, E, H)                                                                     \
    ((comp) == 0   ? (double)E[0][id]                                                                          \
     : (comp) == 1 ? (double)E[1][id]                                                                          \
     : (comp) == 2 ? (double)E[2][id]                                                                          \
     : (comp) == 3 ? (double)H[0][id]                                                                          \
     : (comp) == 4 ? (double)H[1][id]                                                                          \
     : (comp) == 5 ? (double)H[2][id]                                                                          \
     : (comp) == 6 ? sqrt((double)E[0][id] * E[0][id] + (double)E[1][id] * E[1][id] + (double)E[2][id] * E[2][id]) \
     : (comp) == 7 ? sqrt((double)H[0][id] * H[0][id] + (double)H[1][id] * H[1][id] + (double)H[2][id] * H[2][id]) \
     : (comp) == 8 ? (double)E[1][id] * H[2][id] - (double)E[2][id] * H[1][id]                                \
     : (comp) == 9 ? (double)E[2][id] * H[0][id] - (double)E[0][id] * H[2][id]                                \
     : (comp) == 10 ? (double)E[0][id] * H[1][id] - (double)E[1][id] * H[0][id]                               \
                    : PROBE_SMAG(id, E, H))

#define PROBE_SMAG(id, E, H)                                                                     \
    sqrt(((double)E[1][id] * H[2][id] - (double)E[2][id] * H[1][id]) *                           \
             ((double)E[1][id] * H[2][id] - (double)E[2][id] * H[1][id]) +                       \
         ((double)E[2][id] * H[0][id] - (double)E[0][id] * H[2][id]) *                           \
             ((double)E[2][id] * H[0][id] - (double)E[0][id] * H[2][id]) +                       \
         ((double)E[0][id] * H[1][id] - (double)E[1][id] * H[0][id]) *                           \
             ((double)E[0][id] * H[1][id] - (double)E[1][id] * H[0][id]))

#define REAL double
#define SUFFIX _f64
#define ORACLE_IS_F64 1
#include "fdtd_oracle_impl.h"
#undef ORACLE_IS_F64
#undef REAL
#undef SUFFIX

#define REAL float
#define SUFFIX _f32
#define ORACLE_IS_F64 0
#include "fdtd_oracle_impl.h"
#undef ORACLE_IS_F64
#undef REAL
#undef SUFFIX

int64_t oracle_run(const oracle_case *c, oracle_state *s, uint64_t n0, uint64_t nsteps, double *probe_out,
                   int precision, int threads) {
    if (precision == 1) return oracle_run_f32(c, s, n0, nsteps, probe_out, threads);
    return oracle_run_f64(c, s, n0, nsteps, probe_out, threads);
}

void oracle_dft(const double *series, uint64_t n, uint64_t stride, uint64_t n0, uint64_t every, double dt,
                const double *freqs, int nf, double *re, double *im) {
    const double pi = 3.141592653589793238462643383279502884;
    for (int m = 0; m < nf; ++m) {
        double xr = 0.0, xi = 0.0;
        for (uint64_t q = 0; q < n; ++q) {
            const double t = (double)(n0 + q * every + 1) * dt;
            const double ph = 2.0 * pi * freqs[m] * t;
            xr += series[q * stride] * cos(ph) * dt;
            xi -= series[q * stride] * sin(ph) * dt;
        }
        re[m] = xr;
        im[m] = xi;
    }
}
