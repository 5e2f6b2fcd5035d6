/* fdtd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's time-stepping loop
 * (XiaofengYuChina/3D_FDTD_version008, src/3D_FDTD_version008.cpp:269-328) used as the
 * checker for the CUDA stepper.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it.  Pinned against the reference itself: the test suite
 * compares it with oracle/_ref/ref_harness (the reference headers compiled as they
 * are) and with the golden vectors in tests/golden/.
 *
 * Arrays use the reference's idx3 layout (i*NyT + j)*NzT + k; fields are full-grid,
 * psi is the reference's 12 full-grid arrays.  REAL = double reproduces the reference
 * operation for operation; the float twin stores everything in FP32 (same formulas)
 * to measure single-precision drift.
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#define ORACLE_MAX_SRC 8
#define ORACLE_MAX_REGIONS 16

typedef struct oracle_source {
    uint64_t i, j, k;
    int32_t comp; /* 0,1,2 -> Jx,Jy,Jz */
    int32_t waveform;
    double cell_area, I0, f0, tau, t0, t_shift;
} oracle_source;

/* A plane-wave soft source (src/sources/plane_wave_source.hpp:77-98): every step adds
 * J = 2 E(t_half) / (eta0 d) * sign to component comp over the cells lo0..hi0 x lo1..hi1
 * (inclusive) of the plane index `plane` along `axis`; the in-plane axes are (x, y) for a
 * z plane, (y, z) for an x plane and (x, z) for a y plane. */
typedef struct oracle_sheet {
    int32_t axis, comp;
    uint64_t plane, lo0, hi0, lo1, hi1;
    double d, sign;
    int32_t waveform, reserved;
    double E0, f0, tau, t0, t_shift;
} oracle_sheet;

typedef struct oracle_region {
    double kapa_coeff, pa2, pa3, inv_dt, tau, hbar, omega_a, N0, pump_rate;
    int32_t clamp, reserved;
} oracle_region;

/* Read-only description of a case (FP64 setup arrays, as the reference setup makes them). */
typedef struct oracle_case {
    uint64_t NxT, NyT, NzT;
    int32_t npml, n_src, n_regions, n_probes;
    double dt, bH; /* bH = dt/mu0 (aH = 1, aE = 1) */
    const double *inv_dx, *inv_dy, *inv_dz, *dx, *dy, *dz;
    const double *kappa[3], *bEp[3], *cEp[3], *bHp[3], *cHp[3];
    const double *bE[3];
    oracle_source src[ORACLE_MAX_SRC];
    oracle_region regions[ORACLE_MAX_REGIONS];
    const int32_t *region_map; /* idx3, -1 = none (NULL without gain) */
    uint64_t probe_idx[16];    /* idx3 offsets */
    int32_t probe_comp[16];
    uint32_t save_every;
    int32_t n_sheets;
    oracle_sheet sheets[2];
    int32_t pec; /* PECBoundary instead of CPML (npml = 0) */
} oracle_case;

/* Mutable state (FP64 caller-owned arrays, idx3).  Gain arrays may be NULL without gain. */
typedef struct oracle_state {
    double *E[3], *H[3];
    double *Pz, *Pz_prev, *Nu, *Ng;
} oracle_state;

/* Runs steps n0 .. n0+nsteps-1.  CPML psi starts from zero in every call, so a run is
 * one call (the fields and gain state carry over between calls, psi does not).  probe_out (may be NULL) receives one value per probe per
 * sampled step (n % save_every == 0), probe-major per sample; returns the sample count.
 * precision 0 = FP64 (operation-for-operation reference), 1 = FP32 storage and arithmetic.
 * threads = OpenMP threads (0 = default). */
int64_t oracle_run(const oracle_case *c, oracle_state *s, uint64_t n0, uint64_t nsteps, double *probe_out,
                   int precision, int threads);

/* FP64 DFT of a sampled series: X_m = sum_n v_n exp(-i 2 pi f_m t_n) dt, t_n = (n0 + n*every + 1) dt. */
void oracle_dft(const double *series, uint64_t n, uint64_t stride, uint64_t n0, uint64_t every, double dt,
                const double *freqs, int nf, double *re, double *im);

#endif
