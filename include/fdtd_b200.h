/* fdtd_b200.h -- C ABI of the B200 Yee FDTD stepper (libfdtd_b200.so).
 *
 * Drop-in for the time-stepping loop of XiaofengYuChina/3D_FDTD_version008
 * (src/3D_FDTD_version008.cpp:231-381).  That loop calls, per step:
 *   ISource::inject_half_step            src/sources/isource.hpp:28-31, dipole_source.hpp:60-85
 *   update_polarization_multi_region     src/two_level_system.hpp:574-609
 *   fdtd_update_H                        src/fdtd_stepper.hpp:8-47
 *   IBoundary::apply_after_H (CPML)      src/boundary.hpp:150-225
 *   fdtd_update_E / _with_gain           src/fdtd_stepper.hpp:49-89, src/two_level_system.hpp:299-342
 *   IBoundary::apply_after_E (CPML)      src/boundary.hpp:227-300
 *   Runtime::after_E detectors           src/params.hpp:793-810, point_field_detector.hpp:111-124
 *   update_populations_multi_region      src/two_level_system.hpp:612-666
 *   StabilityMonitor::check_stability    src/stability_monitor.hpp:42-144 (every interval steps)
 * fdtd_run() performs all of them on the GPU, in that order, for n steps.
 *
 * Conventions: plain C types only; every function returns an fdtd status code
 * (0 = FDTD_OK) unless stated; host arrays are caller-owned and are copied in or out
 * during the call; device memory is owned by the handle.  3-D host arrays use the
 * reference's idx3 layout: index (i*NyT + j)*NzT + k (z fastest, FP64).  A handle is
 * not thread-safe: calls on one handle must be serialised by the caller; distinct
 * handles are independent.  No entry point ever falls back to a CPU implementation:
 * without a usable CUDA device fdtd_create returns FDTD_ERR_NO_DEVICE.
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_B200_ABI_VERSION 1

/* ------------------------------------------------------------ status codes */
enum {
    FDTD_OK = 0,
    FDTD_ERR_INVALID = 1,     /* bad argument or inconsistent setup */
    FDTD_ERR_OOM = 2,         /* device allocation failed */
    FDTD_ERR_CUDA = 3,        /* a CUDA call failed (message in fdtd_last_error) */
    FDTD_ERR_UNSTABLE = 4,    /* stability monitor stopped the run (NaN/Inf or >10 warnings) */
    FDTD_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    FDTD_ERR_PARSE = 6,       /* parameter file could not be parsed / set up */
    FDTD_ERR_UNSUPPORTED = 7, /* valid for the reference, not handled by this stepper */
    FDTD_ERR_NO_DEVICE = 8,   /* no CUDA device available */
    FDTD_ERR_IO = 9           /* an output file could not be written */
};

/* ------------------------------------------------------------ enums */
typedef enum {
    FDTD_PREC_FP32 = 0, /* fields, CPML psi and gain state stored and updated in FP32 */
    FDTD_PREC_FP64 = 1, /* everything in FP64: the accuracy reference */
    FDTD_PREC_FP16 = 2, /* E, H, CPML psi stored in FP16 as E / sE, H / sH (sH = sE / eta0),
                           arithmetic, material, gain state in FP32 */
    FDTD_PREC_BF16 = 3  /* the same with BF16 storage */
} fdtd_precision;

/* Field / detector components: Detectors::FieldComponent (src/detectors/idetector.hpp:19-29). */
enum {
    FDTD_EX = 0, FDTD_EY = 1, FDTD_EZ = 2, FDTD_HX = 3, FDTD_HY = 4, FDTD_HZ = 5,
    FDTD_E_MAG = 6, FDTD_H_MAG = 7, FDTD_SX = 8, FDTD_SY = 9, FDTD_SZ = 10, FDTD_S_MAG = 11
};

/* Two-level gain state arrays for fdtd_get_tls_state / fdtd_set_tls_state. */
enum { FDTD_TLS_PZ = 0, FDTD_TLS_PZ_PREV = 1, FDTD_TLS_NU = 2, FDTD_TLS_NG = 3 };

/* ------------------------------------------------------------ plain-data setup view */
/* One point current source: the public members of Sources::DipoleSource
 * (src/sources/dipole_source.hpp:12-22).  The stepper evaluates compute_waveform
 * (src/sources/isource.hpp:41-68) in FP64 on the host, J(n) = I((n+1/2)dt)/cell_area. */
typedef struct fdtd_dipole_v1 {
    uint64_t i, j, k;      /* cell (total-grid indices) */
    int32_t polarization;  /* Sources::Polarization 0..5; 3..5 drive Jx..Jz like 0..2 */
    int32_t waveform;      /* Sources::Waveform 0 Ricker, 1 GaussianModulatedSine,
                              2 RickerLikeGaussian2nd, 3 ContinuousWave */
    double cell_area, I0, f0, tau, t0, t_shift;
} fdtd_dipole_v1;

/* One plane-wave soft source: PlaneWaveSource after make_plane_wave_source
 * (src/sources/plane_wave_source.hpp:19-312).  Each step it adds
 * J = 2 E(t) / (eta0 d) * sign, t = (n + 1/2) dt, E(t) = compute_waveform(waveform, t, E0, f0,
 * tau, t0, t_shift), to J component `comp` of the cells of plane `plane` (normal to `axis`)
 * whose in-plane indices lie in [lo0, hi0] x [lo1, hi1] (axis 2: i, j; axis 0: j, k;
 * axis 1: i, k), d = the spacing along `axis` at `plane`. */
typedef struct fdtd_sheet_v1 {
    int32_t axis;      /* 0 x, 1 y, 2 z: the propagation axis */
    int32_t comp;      /* 0 Jx, 1 Jy, 2 Jz */
    uint64_t plane, lo0, hi0, lo1, hi1;
    double d, sign;    /* spacing at the plane; +1 / -1 for + / - propagation */
    int32_t waveform;  /* Sources::Waveform */
    int32_t reserved;
    double E0, f0, tau, t0, t_shift;
} fdtd_sheet_v1;

/* One gain region: TwoLevelParams after finalize()/finalize_with_dt()
 * (src/two_level_system.hpp:17-110). */
typedef struct fdtd_tls_region_v1 {
    double kapa_coeff, pa2, pa3, inv_dt; /* three-point recursion */
    double tau, hbar, omega_a;           /* population rate equation */
    double N0;                           /* Ndip = Ng0 of the region's cells */
    double pump_rate;                    /* W_p (1/s); 0 reproduces the reference */
    int32_t enable_population_clamp;     /* TLS_ENABLE_CLAMP */
    int32_t reserved;
} fdtd_tls_region_v1;

/* One point probe: PointFieldDetector (src/detectors/point_field_detector.hpp:150-255),
 * indices already clamped to [1, N-2].  Every probe also feeds the DFT monitor. */
typedef struct fdtd_probe_v1 {
    uint64_t i, j, k;
    int32_t component; /* FDTD_EX..FDTD_S_MAG */
    int32_t reserved;
} fdtd_probe_v1;

/* Everything one solve needs, as the reference's setup leaves it.  Pointers are only
 * read during fdtd_create.  Optional arrays may be NULL as noted. */
typedef struct fdtd_setup_v1 {
    uint32_t struct_size; /* sizeof(fdtd_setup_v1) */
    int32_t precision;    /* fdtd_precision */
    uint64_t NxT, NyT, NzT;
    uint32_t npml;        /* CPML thickness in cells (CPMLBoundary::npml_) */
    uint32_t save_every;  /* probe sampling period (SAVE_EVERY) */
    double dt;
    /* GridSpacing (src/global_function.hpp:92-105): spacings and inverses, lengths N*T */
    const double *dx, *dy, *dz;
    const double *inv_dx, *inv_dy, *inv_dz;
    /* CPMLBoundary 1-D profiles (src/boundary.hpp:87-91): kappa (kx_,ky_,kz_) and the
     * E-side / H-side recursion coefficients (bEx_,cEx_ ... bHz_,cHz_), index 0/1/2 = x/y/z */
    const double *cpml_kappa[3];
    const double *cpml_bE[3], *cpml_cE[3];
    const double *cpml_bH[3], *cpml_cH[3];
    /* MaterialGrids (src/global_function.hpp:70-90), idx3.  bE is required.  aE/aH may be
     * NULL (all 1); bH may be NULL (uniform bH_uniform).  Non-NULL aE/aH must be all 1 and
     * non-NULL bH must be uniform (sigma = 0, mu_r = 1, as make_nk gives), else
     * FDTD_ERR_UNSUPPORTED. */
    const double *bE[3];
    const double *aE[3];
    const double *aH[3];
    const double *bH[3];
    double bH_uniform;
    /* sources */
    uint32_t n_dipoles;
    const fdtd_dipole_v1 *dipoles;
    /* gain: regions + TLSRegionManager::cell_region_map (idx3, -1 = none) + initial
     * Nu/Ng (idx3).  n_tls_regions = 0 disables gain. */
    uint32_t n_tls_regions;
    const fdtd_tls_region_v1 *tls_regions;
    const int32_t *tls_region_map;
    const double *tls_Nu, *tls_Ng;
    /* detectors */
    uint32_t n_probes;
    const fdtd_probe_v1 *probes;
    uint32_t n_dft_freqs; /* DFT monitor frequencies (Hz), accumulated every step in FP64 */
    const double *dft_freqs;
    /* StabilityMonitor thresholds (src/user_config.hpp:156-160); interval 0 disables */
    uint32_t monitor_interval;
    double max_E, max_P, conservation_err, growth_rate;
    /* FP16 / BF16 storage: the E field scale sE (stored E' = E / sE); 0 = automatic (FP16: the
     * dipoles' tau |I0| / (eps0 cell_area) rounded up to a power of two; BF16: 1) */
    double field_scale;
    /* plane-wave soft sources (at most 2) */
    uint32_t n_sheets;
    const fdtd_sheet_v1 *sheets;
    /* 1: PECBoundary (src/boundary.hpp:51-79): npml must be 0, and after every E update
     * Ex, Ey, Ez are zeroed on the six outer faces.  0: CPML. */
    uint32_t pec_boundary;
    /* Optional compact material: n_bE_rows distinct (bEx, bEy, bEz) rows (bE_rows, row-major,
     * FP64) and each cell's row number (bE_index, idx3).  When given (n_bE_rows <= 65535) the
     * stepper uploads these instead of reading bE[0..2]; fdtd_setup_view fills them.  NULL / 0:
     * the stepper derives them from bE[0..2] itself.  No counterpart in the reference, whose
     * material is the three arrays. */
    uint32_t n_bE_rows;
    const double *bE_rows;
    const uint16_t *bE_index;
    /* Rounding of the E and H stores with BF16 storage: FDTD_ROUND_NEAREST (0, the default) or
     * FDTD_ROUND_STOCHASTIC (1: up or down at random, with probability given by the distance
     * to the two neighbouring BF16 values, so the rounding error is zero on average; keyed by
     * cell, array and step, so a solve's result does not depend on its launch shape, sharding
     * or packing).  Other storage forms round to nearest whatever this holds.  No counterpart
     * in the reference, which stores FP64. */
    uint32_t rounding;
} fdtd_setup_v1;
enum { FDTD_ROUND_NEAREST = 0, FDTD_ROUND_STOCHASTIC = 1 };

/* Diagnostics of the most recent monitor step, FP64 device reductions
 * (StabilityMonitor + compute_integrated_* + PolarizationDiagnostics). */
typedef struct fdtd_diagnostics_v1 {
    uint64_t step;            /* step index n of the last monitor evaluation */
    uint64_t steps_done;      /* total steps completed by the handle */
    double max_E;             /* max |Ex|,|Ey|,|Ez| */
    double max_P;             /* max |Pz| (0 without gain) */
    double conservation_err;  /* |sum(Nu+Ng) - sum(Ng0)| / sum(Ng0) over Ndip > 1e10 */
    double integrated_Nu;     /* sum Nu dV over gain cells */
    double integrated_Ng;     /* sum Ng dV */
    double polarization_energy; /* -1/2 sum Pz Ez dV */
    uint32_t nan_flags;       /* bit0 E, bit1 H, bit2 P, bit3 populations */
    uint32_t instability_count;
    int32_t stable;           /* 0 once the monitor declared the run unstable */
    int32_t reserved;
} fdtd_diagnostics_v1;

/* Device time measured with CUDA events on the handle's stream (fdtd_set_timing).
 * FDTD_TIMING_RUN brackets each fdtd_run call with one event pair (no extra
 * synchronisation); FDTD_TIMING_KERNELS brackets every kernel group of every step
 * (synchronises once per step). */
enum { FDTD_TIMING_OFF = 0, FDTD_TIMING_RUN = 1, FDTD_TIMING_KERNELS = 2 };
typedef struct fdtd_timing_v1 {
    uint64_t steps;      /* steps run with timing enabled */
    double run_ms;       /* FDTD_TIMING_RUN: total device time of the fdtd_run calls */
    double h_ms;         /* FDTD_TIMING_KERNELS: k_update_H total */
    double e_ms;         /* FDTD_TIMING_KERNELS: k_update_E total */
    double aux_ms;       /* FDTD_TIMING_KERNELS: probe/DFT and monitor kernels total */
} fdtd_timing_v1;

typedef struct fdtd_setup fdtd_setup;   /* host setup built by this library */
typedef struct fdtd_handle fdtd_handle; /* one resident solve on one GPU */

/* ------------------------------------------------------------ host setup API */
/* Runs the reference setup sequence (Config::make_context, bake_and_bind, sources,
 * TLS regions, detectors: src/3D_FDTD_version008.cpp:37-172, src/params.hpp:180-868)
 * on a runtime parameter file whose keys are the UserConfig names
 * (src/user_config.hpp:11-211).  mesh_only != 0 stops after mesh, dt and CPML
 * profiles.  On failure returns FDTD_ERR_PARSE and writes a message into err. */
int fdtd_setup_parse(const char *params_text, int mesh_only, fdtd_setup **out, char *err, size_t errlen);
/* Fills a view whose pointers stay valid until fdtd_setup_destroy. */
int fdtd_setup_view(const fdtd_setup *s, fdtd_setup_v1 *out);
/* Named host arrays of the setup ("x_bounds", "dx", "inv_dx", "cpml_kx", "cpml_bEx",
 * "bEx", "aHz", "n_grid", "tls_region_map", ...): length query, then copy as FP64. */
int fdtd_setup_array_len(const fdtd_setup *s, const char *name, uint64_t *len);
int fdtd_setup_array(const fdtd_setup *s, const char *name, double *out, uint64_t len);

/* Writes the files the reference writes before its time loop, under
 * out_dir/frames/<RUN_TAG>/ (out_dir plays the reference's working directory):
 * grid_spacing.txt, coordinate_mapping.txt, mesh_info.json (make_context,
 * src/params.hpp:296-505), the MESH_DETECTORS' files (MeshDetector,
 * src/detectors/mesh_detector.hpp), the metadata.json of every FIELD_MOVIE_2D_DETECTORS
 * and POINT_FIELD_DETECTORS entry and their empty <component>_ts.bin files.  Needs a baked
 * setup (mesh_only = 0).  FDTD_ERR_IO when a file cannot be written. */
int fdtd_setup_write_outputs(const fdtd_setup *s, const char *out_dir, char *err, size_t errlen);
void fdtd_setup_destroy(fdtd_setup *s);

/* ------------------------------------------------------------ stepper */
/* Allocates the resident device state on CUDA device `device` and uploads the setup. */
int fdtd_create(const fdtd_setup_v1 *setup, int device, fdtd_handle **out);
/* Overwrite / read one field component (FDTD_EX..FDTD_HZ), idx3 FP64 host array. */
int fdtd_set_field(fdtd_handle *h, int component, const double *idx3);
int fdtd_get_field(fdtd_handle *h, int component, double *idx3);
/* Gain state (FDTD_TLS_*), idx3 FP64; cells outside the gain regions read as 0. */
int fdtd_set_tls_state(fdtd_handle *h, int which, const double *idx3);
int fdtd_get_tls_state(fdtd_handle *h, int which, double *idx3);
/* Advance n steps (steps n0 .. n0+n-1 of the reference loop).  Returns
 * FDTD_ERR_UNSTABLE if the stability monitor stopped the solve; fields then hold the
 * state of the monitor step that failed, as when the reference's main() returns 1. */
int fdtd_run(fdtd_handle *h, uint64_t n_steps);
int fdtd_steps_done(const fdtd_handle *h, uint64_t *n);
/* Probe samples recorded so far (every save_every steps, probe-major per sample:
 * sample s, probe p at out[s*n_probes + p]).  *n_samples receives the count. */
int fdtd_get_probe_series(fdtd_handle *h, double *out, uint64_t max_samples, uint64_t *n_samples);
/* DFT of probe p: X(f_m) = sum_n v(t_{n+1}) exp(-i 2 pi f_m t_{n+1}) dt, FP64. */
int fdtd_get_dft(fdtd_handle *h, uint32_t probe, double *re, double *im);
int fdtd_get_diagnostics(fdtd_handle *h, fdtd_diagnostics_v1 *out);
/* Device memory held by the handle, bytes. */
int fdtd_device_bytes(const fdtd_handle *h, uint64_t *bytes);
/* Number of CUDA kernel launches issued by the handle since creation. */
int fdtd_kernel_launches(const fdtd_handle *h, uint64_t *n);
/* How the handle holds bE: *rows = the number of distinct (bEx, bEy, bEz) rows when it keeps a
 * 2-byte row index per cell and a table of the rows (at most 65535 rows), 0 when it keeps the
 * three arrays.  Results are the same either way. */
int fdtd_material_rows(const fdtd_handle *h, uint64_t *rows);
/* Select FDTD_TIMING_OFF / _RUN / _KERNELS; any call resets the totals. */
int fdtd_set_timing(fdtd_handle *h, int mode);
int fdtd_get_timing(fdtd_handle *h, fdtd_timing_v1 *out);
/* Kernel path, before the first step only: 1 = separate H and E sweeps (default), 2 = one
 * persistent launch that runs the H and E sweeps slab by slab in dependency order (its
 * device waits are bounded; an expired wait makes fdtd_run return FDTD_ERR_TIMEOUT).  Both
 * paths give bit-identical results.  0 (one fused H+E launch per step) is reserved and
 * refused with FDTD_ERR_UNSUPPORTED. */
int fdtd_set_kernel_path(fdtd_handle *h, int path);
/* Streams the reference's detector files of the parsed setup `s` -- the one whose view
 * created h -- while the handle steps (FieldMovie2D and PointFieldDetector,
 * src/detectors/field_movie_2d.hpp, point_field_detector.hpp): first writes everything
 * fdtd_setup_write_outputs writes, then every SAVE_EVERY-th step each
 * FIELD_MOVIE_2D_DETECTORS slice is captured on the device, copied out and written as its
 * own frame file by a background thread, and after every fdtd_run call the new point
 * samples are appended to the <component>_ts.bin files.  With gain, the two-level
 * detectors of main() (src/two_level_detectors.hpp) record at the same steps:
 * populations/inversion_time.csv, polarization/polarization_time.csv and
 * tls_global_history.csv from device reductions, and the first Nu/Ng frame.  Before the
 * first step only. */
int fdtd_attach_outputs(fdtd_handle *h, const fdtd_setup *s, const char *out_dir);
/* Waits until every frame and sample captured so far is on disk; FDTD_ERR_IO if a write
 * failed.  fdtd_destroy also waits. */
int fdtd_flush_outputs(fdtd_handle *h);
/* Ends the outputs as the reference ends its run (PopulationTimeSeriesDetector::finalize:
 * the last Nu/Ng frame and metadata_populations.json), waits for every write and detaches;
 * later steps write nothing. */
int fdtd_close_outputs(fdtd_handle *h);
/* One solve split along z into nshards slabs, shard r on devices[r] (NULL: all on device 0),
 * each stepped by the same kernels with its global z offset; neighbouring shards exchange one
 * plane of E and one of H per step by device-to-device (peer) copies, and the stability
 * monitor is evaluated once for the whole solve.  The handle answers the same calls as a
 * whole solve (fields, gain state, probes, DFT, diagnostics) with identical values; CPML or
 * PEC boundary (each shard zeroes the PEC faces of the planes it owns); kernel path 1 only,
 * whole-run timing only.  Detector files (fdtd_attach_outputs) are the whole solve's: each
 * shard captures the part of every movie slice in the planes it owns and its two-level sums,
 * and one writer thread joins them into the reference's files.  No counterpart in the reference's
 * time loop; its slab-parallel variant (src/parallel_domain.hpp) splits one process's loop. */
int fdtd_create_sharded(const fdtd_setup_v1 *setup, int nshards, const int *devices, fdtd_handle **out);
/* Block until all device work of the handle is complete. */
int fdtd_synchronize(fdtd_handle *h);
/* Message of the last failing call on h (or of the last global failure when h is NULL). */
const char *fdtd_last_error(const fdtd_handle *h);
void fdtd_destroy(fdtd_handle *h);

/* ------------------------------------------------------------ packed multi-solve engine */
/* The serving form of the stepper: a queue of FP32, FP16 and BF16 solves (mixed freely; FP64
 * and PEC solves are refused with FDTD_ERR_UNSUPPORTED) on one GPU.  fdtd_batch_submit
 * queues a solve and returns at once (the setup view and the arrays it points to must stay
 * valid until the job has finished).  An admission thread inside the batch takes queued jobs
 * in order while their device footprint fits budget_bytes and fewer than 64 are resident or
 * being prepared, and builds each one's device state (allocation, set-up uploads) on the
 * job's own stream while the resident solves keep stepping.  fdtd_batch_run splices the
 * prepared jobs in, then advances every resident solve by up to max_steps steps, each step
 * of all of them issued as one packed H and one packed E launch per storage form present
 * (E: per kind of solve) and one probe launch (plus one monitor pair on monitor steps); a
 * lone resident solve is stepped with fdtd_run's own launches instead, 64 steps at a time
 * (environment FDTD_B200_BATCH_SOLO=0 keeps it packed); every
 * 16 steps, and whenever a solve reaches its step count, it retires finished solves (and any
 * the stability monitor stopped) and splices in newly prepared ones.  With nothing resident it
 * first waits until every job that can be admitted is prepared, so a batch starts with all
 * that fit.  n_queued counts jobs queued or being prepared.  The
 * per-cell arithmetic is fdtd_run's, with every rounding explicit, so a job's probe series,
 * DFT and max |E| are bit-identical to fdtd_create + fdtd_run on the same setup, alone or in
 * any mix.  No counterpart in the reference (it runs one solve per process); it replaces
 * running the reference once per design point.
 * A batch is driven from one host thread.  One batch per device at a time in a process (its
 * per-solve records live in the device's constant memory): fdtd_batch_create on a device
 * that has one returns FDTD_ERR_INVALID. */
typedef struct fdtd_batch fdtd_batch;
enum { FDTD_JOB_QUEUED = 0, FDTD_JOB_RESIDENT = 1, FDTD_JOB_DONE = 2, FDTD_JOB_FAILED = 3 };
int fdtd_batch_create(int device, uint64_t budget_bytes, fdtd_batch **out);
int fdtd_batch_submit(fdtd_batch *b, const fdtd_setup_v1 *setup, uint64_t n_steps, uint64_t *ticket);
int fdtd_batch_run(fdtd_batch *b, uint64_t max_steps, uint32_t *n_resident, uint32_t *n_queued);
int fdtd_batch_job_state(fdtd_batch *b, uint64_t ticket, int *state, uint64_t *steps_done);
/* Results of a finished job (FDTD_JOB_DONE, or FDTD_JOB_FAILED up to the failing step). */
int fdtd_batch_probe_series(fdtd_batch *b, uint64_t ticket, double *out, uint64_t max_samples, uint64_t *n_samples);
int fdtd_batch_dft(fdtd_batch *b, uint64_t ticket, uint32_t probe, double *re, double *im);
int fdtd_batch_diagnostics(fdtd_batch *b, uint64_t ticket, fdtd_diagnostics_v1 *out);
/* Forget a finished job's results. */
int fdtd_batch_release(fdtd_batch *b, uint64_t ticket);
const char *fdtd_batch_last_error(const fdtd_batch *b);
void fdtd_batch_destroy(fdtd_batch *b);

/* ---- Field scan without device allocation.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc when they need the scan -- an application that
 * runs the stepper inside its own device memory pool or arena (which owns all device
 * memory and forbids side allocations), a callback running under its allocator's lock, or
 * code whose watchdog treats any device allocation as a fault.  It computes what the
 * stepper's stability monitor computes over the fields (max |E| over cells whose three E
 * values are finite; bit0 = some E value non-finite, bit1 = some H value non-finite) over n
 * cells of six caller-owned device arrays (any common layout), and writes the result into
 * a caller-owned device record, on `stream` (a cudaStream_t; NULL = the default stream).
 * Nothing is allocated: the scratch is a fixed 256 KiB device array inside the library,
 * held on every GPU that loads the library until the process exits, which bounds n by
 * FDTD_FIELD_SCAN_MAX_CELLS (larger n: FDTD_ERR_INVALID with a message; scan in pieces).
 * Only FP32 and FP64 fields (precision FDTD_PREC_FP32 / FDTD_PREC_FP64) are accepted.
 * The first call on each device (with that device current) looks up the array's device
 * address and keeps it for the life of the process; make that first call before any stream
 * capture, and do not use the entry point across a cudaDeviceReset.  A CUDA error already
 * pending when the call starts is refused with FDTD_ERR_CUDA and left pending.  All calls share the one
 * scratch array: calls that overlap on the GPU race and give wrong results -- serialise
 * them (one stream per device, or events).  Errors: fdtd_last_error(NULL). */
#define FDTD_FIELD_SCAN_MAX_CELLS (16384ull * 16384ull)
typedef struct fdtd_field_scan_v1 {
    double max_E;       /* max |Ex|,|Ey|,|Ez| over cells whose three E values are finite */
    uint32_t nan_flags; /* bit0 E, bit1 H */
    uint32_t reserved;
} fdtd_field_scan_v1;
int fdtd_field_scan_noalloc(int precision, const void *ex, const void *ey, const void *ez, const void *hx,
                            const void *hy, const void *hz, uint64_t n, fdtd_field_scan_v1 *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_B200_H */
