// solver.cu -- resident device state of one FDTD solve and the stepper C ABI.
//
// One fdtd_handle owns, on one GPU: the six field arrays (x-fastest, padded rows), the
// three bE coefficient arrays, the 1-D spacing/CPML profiles, psi only inside the PML
// slabs, the gain block (bounding box of the gain cells: region id, P ping-pong, Nu,
// Ng), probe series / DFT accumulators and the stability-monitor state.  fdtd_run()
// issues, per step, k_update_H, k_update_E, the probe/DFT kernel and on monitor steps
// the FP64 diagnostic reduction, on the handle's stream.  All device memory comes from
// cudaMalloc at create time (staging for layout transposes on first use).
#include "../../include/fdtd_b200.h"
#include "host/outputs.hpp"
#include "host/waveform.hpp"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <condition_variable>
#include <map>
#include <mutex>
#include <deque>
#include <type_traits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <string>
#include <future>
#include <optional>
#include <thread>
#include <vector>

namespace fdtdk {

// ================================================================ small kernels
// idx3 (z fastest, FP64) <-> device layout (x fastest, padded), 32x32 tiles over (k, i)
// for each j.
// dst = scale * src (the storage's field scale), converted to the storage type D.
template <typename D>
__global__ void k_from_idx3(const double* __restrict__ src, D* __restrict__ dst, int NxT, int NyT, int NzT,
                            int NxP, double scale) {
    __shared__ double tile[32][33];
    const int j = blockIdx.z;
    const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < NxT && k < NzT) ? src[(size_t(i) * NyT + j) * NzT + k] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        if (i < NxT && k < NzT) dst[(size_t(k) * NyT + j) * NxP + i] = from_d<D>(tile[threadIdx.x][r] * scale);
    }
}

// The per-cell material index, idx3 (uint16) -> device layout, 32x32 tiles over (k, i).
__global__ void k_index_from_idx3(const uint16_t* __restrict__ src, uint16_t* __restrict__ dst, int NxT, int NyT,
                                  int NzT, int NxP) {
    __shared__ uint16_t tile[32][33];
    const int j = blockIdx.z;
    const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < NxT && k < NzT) ? src[(size_t(i) * NyT + j) * NzT + k] : uint16_t(0);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        if (i < NxT && k < NzT) dst[(size_t(k) * NyT + j) * NxP + i] = tile[threadIdx.x][r];
    }
}

// PECBoundary::apply_after_E (src/boundary.hpp:55-74): Ex = Ey = Ez = 0 on the six outer
// faces, after the E update.  One thread per face cell, the z faces first, then y, then x,
// so that consecutive threads write consecutive i where the layout allows.  The x and y faces
// are zeroed on the planes [k0, k1) this grid owns; the z faces are the local planes zlo and
// zhi, -1 where the face belongs to another shard (a whole solve: k0 = 0, k1 = NzT, zlo = 0,
// zhi = NzT - 1).
template <typename D>
__global__ void k_pec_faces(D* __restrict__ Ex, D* __restrict__ Ey, D* __restrict__ Ez, int NxT, int NyT, int NxP,
                            int k0, int k1, int zlo, int zhi) {
    const int nzp = k1 - k0;
    const long long nz = (long long)NxT * NyT, ny = (long long)NxT * nzp, nx = (long long)NyT * nzp;
    const long long total = 2 * (nx + ny + nz);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        long long u = t;
        int i, j, k;
        if (u < 2 * nz) {
            const int side = int(u / nz);
            u -= side * nz;
            i = int(u % NxT); j = int(u / NxT); k = side ? zhi : zlo;
            if (k < 0) continue;
        } else if ((u -= 2 * nz) < 2 * ny) {
            const int side = int(u / ny);
            u -= side * ny;
            i = int(u % NxT); k = k0 + int(u / NxT); j = side ? NyT - 1 : 0;
        } else {
            u -= 2 * ny;
            const int side = int(u / nx);
            u -= side * nx;
            j = int(u % NyT); k = k0 + int(u / NyT); i = side ? NxT - 1 : 0;
        }
        const size_t q = (size_t(k) * NyT + j) * NxP + i;
        Ex[q] = from_d<D>(0.0);
        Ey[q] = from_d<D>(0.0);
        Ez[q] = from_d<D>(0.0);
    }
}

template <typename D>
__global__ void k_to_idx3(const D* __restrict__ src, double* __restrict__ dst, int NxT, int NyT, int NzT, int NxP,
                          double scale) {
    __shared__ double tile[32][33];
    const int j = blockIdx.z;
    const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        tile[threadIdx.x][r] = (i < NxT && k < NzT) ? double(to_c(src[(size_t(k) * NyT + j) * NxP + i])) * scale : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        if (i < NxT && k < NzT) dst[(size_t(i) * NyT + j) * NzT + k] = tile[r][threadIdx.x];
    }
}

// Gather (to_dev = 0) or scatter (to_dev = 1) the gain block from / to an idx3 array.
template <typename T>
__global__ void k_gain_block(double* __restrict__ full, T* __restrict__ blk, const int8_t* __restrict__ reg, int gi0,
                             int gj0, int gk0, int gX, int gY, int gZ, int NyT, int NzT, int to_dev) {
    const size_t n = size_t(gX) * gY * gZ;
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < n; t += size_t(gridDim.x) * blockDim.x) {
        const int i = int(t % gX) + gi0;
        const int j = int((t / gX) % gY) + gj0;
        const int k = int(t / (size_t(gX) * gY)) + gk0;
        const size_t id = (size_t(i) * NyT + j) * NzT + k;
        if (to_dev) blk[t] = reg[t] >= 0 ? T(full[id]) : T(0);
        else if (reg[t] >= 0) full[id] = double(blk[t]);
    }
}

struct ProbeDev {
    long long off;  // device-layout offset of the probe cell
    int comp;
};

// Probe value in physical units: stored E and H times their field scales es, hs.
// get_field_value (src/detectors/idetector.hpp:79-110) on one cell's six FP64 values, with
// every product and sum rounded on its own (no contraction), as the reference computes it.
__device__ __forceinline__ double component_value(int comp, double ex, double ey, double ez, double hx, double hy,
                                                  double hz) {
    auto cross = [](double a, double b, double c, double d) { return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d)); };
    auto norm = [](double x, double y, double z) {
        return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    };
    switch (comp) {
        case 0: return ex;
        case 1: return ey;
        case 2: return ez;
        case 3: return hx;
        case 4: return hy;
        case 5: return hz;
        case 6: return norm(ex, ey, ez);
        case 7: return norm(hx, hy, hz);
        case 8: return cross(ey, hz, ez, hy);
        case 9: return cross(ez, hx, ex, hz);
        case 10: return cross(ex, hy, ey, hx);
        case 11: return norm(cross(ey, hz, ez, hy), cross(ez, hx, ex, hz), cross(ex, hy, ey, hx));
    }
    return 0.0;
}

// FieldMovie2D::record_after_E (src/detectors/field_movie_2d.hpp:107-148): one component on
// one slice plane, in the reference's order -- XY: (i, j), XZ: (i, k), YZ: (j, k), the
// second index fastest -- as FP64 or FP32.  One thread per output value.
template <typename S>
__global__ void k_slice(const S* __restrict__ Ex, const S* __restrict__ Ey, const S* __restrict__ Ez,
                        const S* __restrict__ Hx, const S* __restrict__ Hy, const S* __restrict__ Hz, int NyT, int NxP,
                        int plane, int index, int comp, long long d2, long long count, double es, double hs,
                        void* __restrict__ out, int f64) {
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < count;
         o += (long long)gridDim.x * blockDim.x) {
        const int a = int(o / d2), b = int(o - (o / d2) * d2);
        const int i = plane == 2 ? index : a;
        const int j = plane == 0 ? b : plane == 1 ? index : a;
        const int k = plane == 0 ? index : b;
        const size_t q = (size_t(k) * NyT + j) * NxP + i;
        const double v = component_value(comp, double(to_c(Ex[q])) * es, double(to_c(Ey[q])) * es,
                                         double(to_c(Ez[q])) * es, double(to_c(Hx[q])) * hs, double(to_c(Hy[q])) * hs,
                                         double(to_c(Hz[q])) * hs);
        if (f64) static_cast<double*>(out)[o] = v;
        else static_cast<float*>(out)[o] = float(v);
    }
}

template <typename S, typename T>
__device__ double probe_value(const StepArgs<S, T>& a, const ProbeDev& p, double es, double hs) {
    const size_t o = size_t(p.off);
    return component_value(p.comp, double(to_c(a.Ex[o])) * es, double(to_c(a.Ey[o])) * es, double(to_c(a.Ez[o])) * es,
                           double(to_c(a.Hx[o])) * hs, double(to_c(a.Hy[o])) * hs, double(to_c(a.Hz[o])) * hs);
}

// Point probes after the E update of step n: sample (every save_every steps) and the
// FP64 DFT accumulation X_m += v * exp(-i 2 pi f_m t) * dt at t = (n+1) dt.
// One thread per (probe, frequency).
template <typename S, typename T>
__device__ void probe_dft_thread(const StepArgs<S, T>& a, const ProbeDev* __restrict__ probes, int nprobes,
                                 const double* __restrict__ freqs, int nf, double* __restrict__ dft,
                                 double* __restrict__ series, long long sample, double t, double dt, double es,
                                 double hs, int tid) {
    const int per = nf > 0 ? nf : 1;
    if (tid >= nprobes * per) return;
    const int p = tid / per, m = tid % per;
    const double v = probe_value(a, probes[p], es, hs);
    if (m == 0 && sample >= 0) series[size_t(sample) * nprobes + p] = v;
    if (nf > 0) {
        double s, c;
        sincospi(2.0 * freqs[m] * t, &s, &c);
        double* acc = dft + 2 * (size_t(p) * nf + m);
        acc[0] = __dadd_rn(acc[0], __dmul_rn(__dmul_rn(v, c), dt));
        acc[1] = __dsub_rn(acc[1], __dmul_rn(__dmul_rn(v, s), dt));
    }
}

template <typename S, typename T>
__global__ void k_probe_dft(const StepArgs<S, T> a, const ProbeDev* __restrict__ probes, int nprobes,
                            const double* __restrict__ freqs, int nf, double* __restrict__ dft,
                            double* __restrict__ series, long long sample, double t, double dt, double es, double hs) {
    if (*a.status) return;
    probe_dft_thread(a, probes, nprobes, freqs, nf, dft, series, sample, t, dt, es, hs,
                     int(blockIdx.x * blockDim.x + threadIdx.x));
}

struct DiagAccum {
    unsigned long long maxE, maxP;  // bit patterns of non-negative doubles
    unsigned flags;                 // bit0 E, bit1 H, bit2 P, bit3 populations non-finite
    unsigned pad;
    double sum_pop, sum_N0, int_Nu, int_Ng, p_energy;
};

struct MonitorState {
    double prev_max_E;
    unsigned instability_count;
    int stable;
    // last evaluation
    unsigned long long step;
    double max_E, max_P, cons, int_Nu, int_Ng, p_energy;
    unsigned flags;
    int has_gain;
    // thresholds
    double thr_E, thr_P, thr_cons, thr_growth;
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// Block-wide reduction of 7 quantities into the accumulator (one atomic each per block).
__device__ void block_commit(DiagAccum* acc, double mE, double mP, unsigned fl, double s0, double s1, double s2,
                             double s3, double s4) {
    __shared__ double sh[8][32];
    __shared__ unsigned shf;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) shf = 0;
    __syncthreads();
    mE = warp_max(mE); mP = warp_max(mP);
    s0 = warp_sum(s0); s1 = warp_sum(s1); s2 = warp_sum(s2); s3 = warp_sum(s3); s4 = warp_sum(s4);
    if (fl) atomicOr(&shf, fl);
    if (lane == 0) {
        sh[0][wid] = mE; sh[1][wid] = mP; sh[2][wid] = s0; sh[3][wid] = s1;
        sh[4][wid] = s2; sh[5][wid] = s3; sh[6][wid] = s4;
    }
    __syncthreads();
    if (wid == 0) {
        double v[7];
        for (int q = 0; q < 7; ++q) v[q] = lane < nw ? sh[q][lane] : 0.0;
        v[0] = warp_max(v[0]); v[1] = warp_max(v[1]);
        for (int q = 2; q < 7; ++q) v[q] = warp_sum(v[q]);
        if (lane == 0) {
            atomicMax(&acc->maxE, (unsigned long long)__double_as_longlong(v[0]));
            atomicMax(&acc->maxP, (unsigned long long)__double_as_longlong(v[1]));
            if (shf) atomicOr(&acc->flags, shf);
            if (v[2] != 0.0) atomicAdd(&acc->sum_pop, v[2]);
            if (v[3] != 0.0) atomicAdd(&acc->sum_N0, v[3]);
            if (v[4] != 0.0) atomicAdd(&acc->int_Nu, v[4]);
            if (v[5] != 0.0) atomicAdd(&acc->int_Ng, v[5]);
            if (v[6] != 0.0) atomicAdd(&acc->p_energy, v[6]);
        }
    }
}

// FP64 scans of StabilityMonitor::check_stability (src/stability_monitor.hpp:42-135),
// calculate_conservation_error (:155-170), compute_integrated_Nu/Ng and
// compute_polarization_energy (src/two_level_system.hpp:344-418) over the fields after
// the step.  Field arrays are scanned as flat padded arrays (padding holds zeros).
template <typename S, typename T, bool FIELDS = true>
__device__ void monitor_reduce_blocks(const StepArgs<S, T>& a, size_t f0, size_t nflat, const double* __restrict__ dxs,
                                      const double* __restrict__ dys, const double* __restrict__ dzs, int parity_next,
                                      DiagAccum* acc, double es, unsigned bid, unsigned nblk) {
    if (*a.status) return;
    double mE = 0.0, mP = 0.0, s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    unsigned fl = 0;
    const size_t stride = size_t(nblk) * blockDim.x;
    // 16-byte vectors: nflat is a multiple of the padded row, itself a multiple of W
    constexpr int W = Vec<T>::W;
    for (size_t v = f0 / W + bid * size_t(blockDim.x) + threadIdx.x; FIELDS && v < nflat / W; v += stride) {
        const size_t t = v * W;
        T ex[W], ey[W], ez[W], hx[W], hy[W], hz[W];
        Fld<S, T>::ldg(a.Ex + t, ex); Fld<S, T>::ldg(a.Ey + t, ey); Fld<S, T>::ldg(a.Ez + t, ez);
        Fld<S, T>::ldg(a.Hx + t, hx); Fld<S, T>::ldg(a.Hy + t, hy); Fld<S, T>::ldg(a.Hz + t, hz);
#pragma unroll
        for (int e = 0; e < W; ++e) {
            const double x = double(ex[e]) * es, y = double(ey[e]) * es, z = double(ez[e]) * es;
            if (!isfinite(x) || !isfinite(y) || !isfinite(z)) fl |= 1u;
            else mE = fmax(mE, fmax(fabs(x), fmax(fabs(y), fabs(z))));
            if (!isfinite(double(hx[e])) || !isfinite(double(hy[e])) || !isfinite(double(hz[e]))) fl |= 2u;
        }
    }
    if (a.gain) {
        const T* Pn = parity_next ? a.P1 : a.P0;
        const T* Po = parity_next ? a.P0 : a.P1;
        const size_t ng = size_t(a.gX) * a.gY * a.gZ;
        for (size_t t = bid * size_t(blockDim.x) + threadIdx.x; t < ng; t += stride) {
            const int r = a.greg[t];
            if (r < 0 || !a.gcoef[r].active) continue;
            const int i = int(t % a.gX) + a.gi0;
            const int j = int((t / a.gX) % a.gY) + a.gj0;
            const int k = int(t / (size_t(a.gX) * a.gY)) + a.gk0;
            const double P = double(Pn[t]), Pp = double(Po[t]);
            const double Nu = double(a.Nu[t]), Ng = double(a.Ng[t]);
            if (!isfinite(P) || !isfinite(Pp)) fl |= 4u;
            else mP = fmax(mP, fabs(P));
            if (!isfinite(Nu) || !isfinite(Ng)) fl |= 8u;
            const double N0 = double(a.gcoef[r].N0);
            if (N0 > 1e10) { s0 += Nu + Ng; s1 += N0; }
            const double dV = dxs[i] * dys[j] * dzs[k];
            s2 += Nu * dV;
            s3 += Ng * dV;
            const double ez = double(to_c(a.Ez[(size_t(k) * a.NyT + j) * a.NxP + i])) * es;
            s4 += -0.5 * P * ez * dV;
        }
    }
    block_commit(acc, mE, mP, fl, s0, s1, s2, s3, s4);
}

// The two-level detectors' record at one step: the gain integrals (as the monitor computes
// them, without the field scan) and, at the PolarizationDiagnostics cell (gain-box offset
// mon_t, or -1), Pz^{n+1} and dPz/dt = (Pz^{n+1} - Pz^n) inv_dt (src/two_level_system.hpp:600-604).
struct TlsRecord {
    DiagAccum acc;
    double P_center, dP_dt;
};

template <typename S, typename T>
__global__ void k_tls_reduce(const StepArgs<S, T> a, const double* __restrict__ dxs, const double* __restrict__ dys,
                             const double* __restrict__ dzs, int parity_next, double es, TlsRecord* rec,
                             long long mon_t) {
    monitor_reduce_blocks<S, T, false>(a, 0, 0, dxs, dys, dzs, parity_next, &rec->acc, es, blockIdx.x, gridDim.x);
    if (blockIdx.x == 0 && threadIdx.x == 0 && mon_t >= 0) {
        const int r = a.greg[mon_t];
        if (r >= 0 && a.gcoef[r].active) {
            const T* Pn = parity_next ? a.P1 : a.P0;
            const T* Po = parity_next ? a.P0 : a.P1;
            const double pn = double(Pn[mon_t]), po = double(Po[mon_t]);
            rec->P_center = pn;
            rec->dP_dt = __dmul_rn(__dsub_rn(pn, po), double(a.gcoef[r].inv_dt));
        }
    }
}

// One thread: the StabilityMonitor decision for monitor step `step`; sets the abort
// word when the reference would terminate (NaN/Inf anywhere, or > 10 threshold warnings).
template <typename S, typename T>
__global__ void k_monitor_reduce(const StepArgs<S, T> a, size_t f0, size_t nflat, const double* __restrict__ dxs,
                                 const double* __restrict__ dys, const double* __restrict__ dzs, int parity_next,
                                 DiagAccum* acc, double es) {
    monitor_reduce_blocks(a, f0, nflat, dxs, dys, dzs, parity_next, acc, es, blockIdx.x, gridDim.x);
}

__device__ void monitor_eval(DiagAccum* acc, MonitorState* ms, unsigned* status, unsigned long long step) {
    if (*status) return;
    const double max_E = __longlong_as_double((long long)acc->maxE);
    const double max_P = __longlong_as_double((long long)acc->maxP);
    const unsigned fl = acc->flags;
    double cons = 0.0;
    if (ms->has_gain && acc->sum_N0 >= 1e-30) cons = fabs(acc->sum_pop - acc->sum_N0) / acc->sum_N0;
    ms->step = step;
    ms->max_E = max_E;
    ms->max_P = ms->has_gain ? max_P : 0.0;
    ms->cons = cons;
    ms->int_Nu = acc->int_Nu;
    ms->int_Ng = acc->int_Ng;
    ms->p_energy = acc->p_energy;
    ms->flags = fl;
    bool fatal = (fl & 3u) != 0 || (ms->has_gain && (fl & 12u) != 0);
    if (!fatal) {
        if (max_E > ms->thr_E) ms->instability_count++;
        if (ms->has_gain && max_P > ms->thr_P) ms->instability_count++;
        if (step > 0 && step % 100 == 0 && ms->prev_max_E > 1e-20) ms->prev_max_E = max_E;
        else if (step == 0 || ms->prev_max_E < 1e-20) ms->prev_max_E = fmax(max_E, 1e-20);
        if (ms->instability_count > 10) fatal = true;
    }
    if (fatal) {
        ms->stable = 0;
        *status = 1u;
    }
    acc->maxE = 0; acc->maxP = 0; acc->flags = 0;
    acc->sum_pop = acc->sum_N0 = acc->int_Nu = acc->int_Ng = acc->p_energy = 0.0;
}

__global__ void k_monitor_eval(DiagAccum* acc, MonitorState* ms, unsigned* status, unsigned long long step) {
    monitor_eval(acc, ms, status, step);
}

// The monitor of a sharded solve: the other shards' accumulators, copied next to shard 0's,
// folded into it (max, or, sums) before the one evaluation.
__global__ void k_acc_combine(DiagAccum* dst, const DiagAccum* parts, int n) {
    for (int r = 0; r < n; ++r) {
        const DiagAccum& p = parts[r];
        dst->maxE = dst->maxE > p.maxE ? dst->maxE : p.maxE;
        dst->maxP = dst->maxP > p.maxP ? dst->maxP : p.maxP;
        dst->flags |= p.flags;
        dst->sum_pop += p.sum_pop;
        dst->sum_N0 += p.sum_N0;
        dst->int_Nu += p.int_Nu;
        dst->int_Ng += p.int_Ng;
        dst->p_energy += p.p_energy;
    }
}

// ================================================================ packed multi-solve step
// Up to kMaxBatch resident solves (FP32, or FP16/BF16 storage with FP32 arithmetic) advance
// together: every sweep is one launch per storage form present, whose blocks are listed in a
// table (solve, bx, by, bz), each block running the same block code as the single-solve
// kernels on its solve's arguments, read from constant memory with a block-uniform index.
// Per-solve step data (sources, probe sample, monitor flag) is rewritten in constant memory
// before every step.
constexpr int kMaxBatch = 64;
constexpr int kMonBlocks = 64;  // monitor blocks per solve

struct BatchSolve {
    SweepGeom g;
    int kchunkH, kchunkE;
    int storage;    // 0 FP32, 1 FP16, 2 BF16 (fills the gap before the pointers)
    const ProbeDev* probes;
    int nprobes, nf;
    const double* freqs;
    double *dft, *series;
    const double *dx, *dy, *dz;
    DiagAccum* acc;
    MonitorState* ms;
    unsigned* status;
    unsigned long long nflat;
    double dt;
    double sE, sH;  // stored fields are E / sE and H / sH (1 for FP32)
};

struct BatchTick {
    ESrc src;
    long long sample;         // probe sample index of this step, or -1
    double t;                 // (n + 1) dt
    unsigned long long step;  // n
    int monitor;              // the stability monitor runs after this step
    int pad;
};

// A resident solve's sweep arguments, whichever its storage form (the three forms differ
// only in the element type of the field and psi pointers).
union BatchArgs {
    StepArgs<float, float> f32;
    StepArgs<__half, float> f16;
    StepArgs<__nv_bfloat16, float> bf16;
};
static_assert(sizeof(StepArgs<float, float>) == sizeof(StepArgs<__nv_bfloat16, float>) &&
                  sizeof(StepArgs<float, float>) == sizeof(StepArgs<__half, float>),
              "storage forms share one argument layout");

__constant__ BatchArgs c_bargs[kMaxBatch];
__constant__ BatchSolve c_bsolve[kMaxBatch];
__constant__ BatchTick c_btick[kMaxBatch];
// The 64 KB constant bank also holds the monitor's and DFT kernels' few constants.
static_assert((sizeof(BatchArgs) + sizeof(BatchSolve) + sizeof(BatchTick)) * kMaxBatch <= 60 * 1024,
              "per-solve constant records exceed the constant bank");

template <typename S>
__device__ __forceinline__ const StepArgs<S, float>& bargs(int r) {
    if constexpr (std::is_same_v<S, float>) return c_bargs[r].f32;
    else if constexpr (std::is_same_v<S, __half>) return c_bargs[r].f16;
    else return c_bargs[r].bf16;
}

// The blocks of the solves stored as S.  PIPE: interior columns stage their planes in shared
// memory (HPipe<S>::bytes() / EPipe<S>::bytes() dynamic), as in the single-solve sweeps.
template <typename S, bool PIPE, int SRM>
__global__ void __launch_bounds__(32 * kBlockY, 2) k_update_H_multi(const int4* __restrict__ tab) {
    const int4 e = tab[blockIdx.x];
    update_H_block<S, float, PIPE, SRM>(bargs<S>(e.x), c_bsolve[e.x].kchunkH, c_bsolve[e.x].g, e.y, e.z, e.w,
                                   c_btick[e.x].src.step);
}

// SH / MAT: the blocks of solves with plane-wave sheets / an indexed material; the table lists
// each (storage, SH, MAT) kind in a separate run, so a solve runs the same code whatever else
// is resident.
template <typename S, bool SH, bool MAT, bool PIPE, int SRM>
__global__ void __launch_bounds__(32 * kBlockY, 2) k_update_E_multi(const int4* __restrict__ tab) {
    const int4 e = tab[blockIdx.x];
    update_E_block<S, float, false, SH, MAT, PIPE, SRM>(bargs<S>(e.x), c_bsolve[e.x].kchunkE, c_btick[e.x].src,
                                                   c_bsolve[e.x].g, e.y, e.z, e.w);
}

template <typename S>
__device__ __forceinline__ void probe_multi_block(int r) {
    const StepArgs<S, float>& a = bargs<S>(r);
    const BatchSolve& b = c_bsolve[r];
    const BatchTick& tk = c_btick[r];
    if (*a.status || b.nprobes == 0) return;
    const int n = b.nprobes * (b.nf > 0 ? b.nf : 1);
    for (int tid = threadIdx.x; tid < n; tid += blockDim.x)
        probe_dft_thread(a, b.probes, b.nprobes, b.freqs, b.nf, b.dft, b.series, tk.sample, tk.t, b.dt, b.sE, b.sH, tid);
}

// one block per solve
__global__ void k_probe_multi() {
    const int r = blockIdx.x;
    const int st = c_bsolve[r].storage;
    if (st == 0) probe_multi_block<float>(r);
    else if (st == 1) probe_multi_block<__half>(r);
    else probe_multi_block<__nv_bfloat16>(r);
}

template <typename S>
__device__ __forceinline__ void monitor_multi_block(int r) {
    const BatchSolve& b = c_bsolve[r];
    monitor_reduce_blocks(bargs<S>(r), 0, size_t(b.nflat), b.dx, b.dy, b.dz, int((c_btick[r].step + 1) & 1), b.acc,
                          b.sE, blockIdx.x % kMonBlocks, kMonBlocks);
}

// kMonBlocks blocks per solve; solves without a monitor step this step return at once
__global__ void k_monitor_reduce_multi() {
    const int r = blockIdx.x / kMonBlocks;
    if (!c_btick[r].monitor) return;
    const int st = c_bsolve[r].storage;
    if (st == 0) monitor_multi_block<float>(r);
    else if (st == 1) monitor_multi_block<__half>(r);
    else monitor_multi_block<__nv_bfloat16>(r);
}

// The status words of the n resident solves, gathered for one copy to the host.
__global__ void k_status_multi(int n, unsigned* __restrict__ out) {
    const int r = threadIdx.x;
    if (r < n) out[r] = *c_bsolve[r].status;
}

__global__ void k_monitor_eval_multi(int nres) {
    const int r = threadIdx.x;
    if (r >= nres || !c_btick[r].monitor) return;
    monitor_eval(c_bsolve[r].acc, c_bsolve[r].ms, c_bsolve[r].status, c_btick[r].step);
}

}  // namespace fdtdk

// ==================================================================== host side
namespace {

using namespace fdtdk;

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int code = (e == cudaErrorMemoryAllocation) ? FDTD_ERR_OOM : FDTD_ERR_CUDA;
    throw Failure(code, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

// The E field scale of 16-bit storage (see the Solver constructor).
double field_scale_of(const fdtd_setup_v1& s, bool fp16) {
    double sE = s.field_scale;
    if (!(sE > 0.0)) {
        sE = 1.0;
        if (fp16) {
            double est = 0.0;
            for (uint32_t q = 0; q < s.n_dipoles; ++q) {
                const fdtd_dipole_v1& d = s.dipoles[q];
                if (d.cell_area > 0) est = std::max(est, d.tau * std::fabs(d.I0) / (8.8541878128e-12 * d.cell_area));
            }
            for (uint32_t q = 0; q < s.n_sheets; ++q) est = std::max(est, 64.0 * std::fabs(s.sheets[q].E0));
            if (est > 0) sE = std::exp2(std::round(std::log2(est / 4096.0)));
        }
    }
    return sE;
}

// One z shard of a solve: the shard's grid holds global planes [kz0, kz0 + NzT) of NzG, of
// which it updates (owns) the local planes [own0, own1); the planes around them are halo copies
// of the neighbours' planes.  A whole solve: kz0 = 0, NzG = NzT, own = [0, NzT).
struct ShardSpec {
    int kz0 = 0, NzG = 0, own0 = 0, own1 = 0;
    double psi_dx = 0;  // 16-bit storage: the whole solve's smallest cell edge (0: this grid's)
};

class SolverBase {
public:
    virtual ~SolverBase() = default;
    virtual void run(uint64_t n) = 0;
    virtual void set_field(int comp, const double* h) = 0;
    virtual void get_field(int comp, double* h) = 0;
    virtual void set_tls(int which, const double* h) = 0;
    virtual void get_tls(int which, double* h) = 0;
    virtual void probe_series(double* out, uint64_t max, uint64_t* n) = 0;
    virtual void dft(uint32_t p, double* re, double* im) = 0;
    virtual void diagnostics(fdtd_diagnostics_v1* d) = 0;
    virtual void sync() = 0;
    virtual void set_timing(int mode) = 0;
    virtual void set_path(int path) = 0;
    virtual void timing(fdtd_timing_v1* t) = 0;
    virtual void attach_outputs(const fdtd::SimSetup& setup, const std::string& root) = 0;
    virtual void flush_outputs() = 0;
    virtual void close_outputs() = 0;
    uint64_t steps = 0, launches = 0, dev_bytes = 0, material_rows = 0;
    int device = 0;
};

// Fields and CPML psi stored as S, arithmetic in T (S = T for FP32 / FP64; S = __half or
// __nv_bfloat16 with T = float for the 16-bit storage forms, whose stored values are
// E' = E / sE and H' = H / sH).
class Batch;
template <typename S, typename T>
class Sharded;

template <typename S, typename T>
class Solver final : public SolverBase {
    friend class Batch;
    friend class Sharded<S, T>;

public:
    // Device memory comes from the device's stream-ordered pool (pooled_, the default), or from
    // cudaMalloc / cudaFree when the environment sets FDTD_B200_ALLOC=malloc for a solve that is
    // not a packed-engine job (pooled = true: its retirement must not stall the resident solves).
    explicit Solver(const fdtd_setup_v1& s, int dev, const ShardSpec* shard = nullptr, bool pooled = false);
    ~Solver() override;
    void run(uint64_t n) override;
    void set_field(int comp, const double* h) override;
    void get_field(int comp, double* h) override;
    void set_tls(int which, const double* h) override;
    void get_tls(int which, double* h) override;
    void probe_series(double* out, uint64_t max, uint64_t* n) override;
    void dft(uint32_t p, double* re, double* im) override;
    void diagnostics(fdtd_diagnostics_v1* d) override;
    void sync() override { ck(cudaStreamSynchronize(st_), "cudaStreamSynchronize"); }
    void set_timing(int mode) override;
    void set_path(int path) override {
        if (path < 0 || path > 2)
            throw Failure(FDTD_ERR_INVALID, "kernel path must be 1 (two sweeps) or 2 (slab-ordered step)");
        if (path == 0)
            throw Failure(FDTD_ERR_UNSUPPORTED,
                          "kernel path 0 (one fused H+E launch per step) is not built: it measured slower than the two sweeps");
        if (steps != 0) throw Failure(FDTD_ERR_INVALID, "the kernel path can only change before the first step");
        path_ = path;
    }
    void timing(fdtd_timing_v1* t) override { *t = tm_; }

private:
    template <typename U> U* alloc(size_t n, bool zero = true) {
        void* p = nullptr;
        dev_alloc(&p, std::max<size_t>(n, 1) * sizeof(U));
        ptrs_.push_back(p);
        dev_bytes += std::max<size_t>(n, 1) * sizeof(U);
        if (zero) ck(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(U), st_), "cudaMemsetAsync");
        return static_cast<U*>(p);
    }
    template <typename U> U* upload(const std::vector<U>& v) {
        U* d = alloc<U>(v.size(), false);
        ck(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(U), cudaMemcpyHostToDevice, st_), "cudaMemcpyAsync");
        return d;
    }
    // A solve's own arrays.  The stream-ordered pool (kept memory, see keep_pool_memory) makes
    // retiring a packed job free for the resident ones and a repeated solve cheap to create and
    // destroy.  Measured on one B200: growing the pool by 9 GB costs 53 ms against 5 ms for
    // cudaMalloc, but create + destroy of a small solve cost 1-2 ms through the pool against
    // 7-8 ms through cudaMalloc, and the FP64 sweeps ran 0.7 % slower on cudaMalloc'd fields.
    bool pooled_ = true;
    void dev_alloc(void** p, size_t bytes) {
        if (pooled_) ck(cudaMallocAsync(p, bytes, st_), "cudaMallocAsync");
        else ck(cudaMalloc(p, bytes), "cudaMalloc");
    }
    void dev_free(void* p) {
        if (pooled_) cudaFreeAsync(p, st_);
        else cudaFree(p);
    }
    double* staging();
    void attach_outputs(const fdtd::SimSetup& setup, const std::string& root) override;
    void flush_outputs() override;
    void capture_movies();
    void write_point_samples();
    void capture_tls(uint64_t s);
    void phase_H(uint64_t s);
    void phase_E(uint64_t s, ESrc& src, bool monitor);
    void write_population_frame();
    void close_outputs() override;
    // Host <-> device copies of FP64 arrays through the device's two pinned chunks
    // (pinned_chunks): the host-side copy of one chunk (OpenMP) overlaps the DMA of the other.
    static constexpr size_t kPinBytes = size_t(32) << 20;
    void h2d(const double* h, double* d, size_t n);
    void d2h(const double* d, double* h, size_t n);
    void upload_gain_box(const double* idx3, const std::vector<int8_t>& reg, T* dst);
    template <typename D> void to_device(const double* host_idx3, D* dst, double scale = 1.0);
    template <typename D> void from_device(const D* src, double* host_idx3, double scale = 1.0);
    void ensure_series(uint64_t samples);

    cudaStream_t st_ = nullptr;
    std::vector<void*> ptrs_;
    StepArgs<S, T> a_{};
    double sE_ = 1.0, sH_ = 1.0;  // stored fields are E / sE_ and H / sH_
    int NxT_, NyT_, NzT_, NxP_, np_;
    size_t plane_, nflat_;
    int kchunkH_ = 1, kchunkE_ = 1;
    SweepGeom geom_{};
    // path 2: k_step_slabs (persistent, slab-ordered H + E in one launch)
    SlabPlan plan_{};
    unsigned* d_ctr_ = nullptr;
    bool slab_hold_ = false;  // FDTD_B200_SLAB_HOLD: E tiles wait on a hold word that nothing clears
    dim3 gridS_;
    void setup_slabs();
    dim3 gridH_, gridE_;
    double dt_;
    // sources
    std::vector<fdtd_dipole_v1> dip_;
    std::vector<fdtd_sheet_v1> sheets_;
    // Point sources and sheet geometry of the per-step source record, then this step's J.
    void src_static(ESrc& src) const {
        src.n = int(dip_.size());
        for (int q = 0; q < src.n; ++q) {
            src.si[q] = int(dip_[q].i); src.sj[q] = int(dip_[q].j); src.sk[q] = int(dip_[q].k);
            src.sc[q] = dip_[q].polarization % 3;
        }
        src.ns = int(sheets_.size());
        for (int q = 0; q < src.ns; ++q) {
            const fdtd_sheet_v1& w = sheets_[q];
            src.ax[q] = w.axis; src.pc[q] = w.comp; src.pl[q] = int(w.plane);
            src.lo0[q] = int(w.lo0); src.hi0[q] = int(w.hi0); src.lo1[q] = int(w.lo1); src.hi1[q] = int(w.hi1);
        }
    }
    void src_step(ESrc& src, uint64_t s) const {
        src.parity = int(s & 1);
        src.step = unsigned(s);
        for (int q = 0; q < src.n; ++q) {
            const fdtd_dipole_v1& d = dip_[q];
            src.J[q] = fdtd::current_density(d.waveform, s, dt_, d.I0, d.f0, d.tau, d.t0, d.t_shift, d.cell_area) *
                       (1.0 / sH_);
        }
        const double t_half = (double(s) + 0.5) * dt_;
        for (int q = 0; q < src.ns; ++q) {  // PlaneWaveSource::inject_*_plane
            const fdtd_sheet_v1& w = sheets_[q];
            const double Et = fdtd::waveform_value(w.waveform, t_half, w.E0, w.f0, w.tau, w.t0, w.t_shift);
            src.sJ[q] = 2.0 * Et / (376.730313668 * w.d) * w.sign * (1.0 / sH_);
        }
    }
    // detectors
    uint32_t save_every_ = 1, nprobes_ = 0, nf_ = 0;

    // The reference's detector files (fdtd_attach_outputs): movie slices are captured into
    // one of kOutSlots device buffers, copied to the matching pinned buffer on the stream,
    // and written by the writer thread once the copy's event has completed; a slot is
    // reused after the writer has finished with it.  Point samples are appended to their
    // _ts.bin files after every run() call.
    static constexpr int kOutSlots = 4;
    std::unique_ptr<fdtd::OutputWriter> writer_;
    fdtd::OutputPlan oplan_;
    std::string oroot_;
    std::vector<size_t> mov_off_, mov_bytes_;
    size_t oslot_bytes_ = 0;
    char* d_oslot_[kOutSlots] = {};
    char* h_oslot_[kOutSlots] = {};
    cudaEvent_t oslot_ev_[kOutSlots] = {};
    std::mutex oslot_mu_;
    std::condition_variable oslot_cv_;
    int oslot_busy_[kOutSlots] = {};
    uint64_t oframe_ = 0, ots_written_ = 0;
    // two-level detector records: kTlsSlots device records and pinned copies, same reuse rule
    static constexpr int kTlsSlots = 16;
    TlsRecord* d_trec_ = nullptr;
    TlsRecord* h_trec_ = nullptr;
    cudaEvent_t trec_ev_[kTlsSlots] = {};
    int trec_busy_[kTlsSlots] = {};
    uint64_t tls_count_ = 0;
    long long mon_t_ = -1;
    bool pop_first_done_ = false;
    ProbeDev* d_probes_ = nullptr;
    double *d_freqs_ = nullptr, *d_dft_ = nullptr, *d_series_ = nullptr;
    uint64_t series_cap_ = 0, series_count_ = 0;
    // monitor
    uint32_t interval_ = 0;
    double *d_dx_ = nullptr, *d_dy_ = nullptr, *d_dz_ = nullptr;
    DiagAccum* d_acc_ = nullptr;
    MonitorState* d_ms_ = nullptr;
    unsigned* d_status_ = nullptr;
    double* d_stage_ = nullptr;
    bool has_gain_ = false;
    bool pec_ = false;  // PECBoundary: zero E on the outer faces after every E update
    size_t mat_rows_ = 0;  // > 0: indexed material (a_.bidx / a_.btab)
    ShardSpec shard_{};
    // The sweeps' interior columns stage their planes in shared memory through cp.async
    // (FDTD_B200_E_PIPE / FDTD_B200_H_PIPE = 0 / 1 override the defaults set in the constructor).
    bool pipe_ = false, hpipe_ = false;
    // BF16 stores with stochastic rounding: the sweeps are compiled per rounding mode (SRM 0 / 1),
    // so that the common round-to-nearest kernel carries no stochastic-rounding code.
    int srm_ = 0;
    template <int SRM>
    static void e_kernels(void (*(&k)[8])(const StepArgs<S, T>, const int, const ESrc, const SweepGeom)) {
        // the staged form exists for the indexed material only (pipe_ implies a_.bidx)
        k[0] = k_update_E<S, T, false, false, false, SRM>; k[1] = k_update_E<S, T, false, false, false, SRM>;
        k[2] = k_update_E<S, T, false, true, false, SRM>;  k[3] = k_update_E<S, T, false, true, true, SRM>;
        k[4] = k_update_E<S, T, true, false, false, SRM>;  k[5] = k_update_E<S, T, true, false, false, SRM>;
        k[6] = k_update_E<S, T, true, true, false, SRM>;   k[7] = k_update_E<S, T, true, true, true, SRM>;
    }
    using EKernel = void (*)(const StepArgs<S, T>, const int, const ESrc, const SweepGeom);
    EKernel e_kernel(bool sheets) const {
        EKernel k[8];
        if constexpr (std::is_same_v<S, __nv_bfloat16>) {
            if (srm_) e_kernels<1>(k);
            else e_kernels<0>(k);
        } else {
            e_kernels<0>(k);
        }
        return k[4 * int(sheets) + 2 * int(a_.bidx != nullptr) + int(pipe_)];
    }
    using HKernel = void (*)(const StepArgs<S, T>, const int, const SweepGeom, const unsigned);
    HKernel h_kernel() const {
        if constexpr (std::is_same_v<S, __nv_bfloat16>)
            if (srm_) return hpipe_ ? k_update_H<S, T, true, 1> : k_update_H<S, T, false, 1>;
        return hpipe_ ? k_update_H<S, T, true, 0> : k_update_H<S, T, false, 0>;
    }
    // event timing: ev_[0..3] bracket H, E and the auxiliary kernels of one step
    // kernel path 1 (default): k_update_H + k_update_E in place; path 2: k_step_slabs.
    int path_ = 1;
    S* fld_[6] = {};
    int xoff_ = 0;  // the field arrays start xoff_ elements into their allocation
    S* psiH_[6] = {};
    size_t psi_sz_[6] = {};
    void point_args_at();
    void pec_faces();  // PECBoundary after the E sweep: the faces of the planes this grid owns
    int timing_ = FDTD_TIMING_OFF;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    fdtd_timing_v1 tm_{};
};

// The device's default memory pool (which cudaMallocAsync draws from) keeps what solves give
// back instead of returning it to the driver at the next synchronisation: a retired solve's
// memory is then reused by the next one without new mappings, and retiring does not unmap
// gigabytes.  Set once per device.
void keep_pool_memory(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> l(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    ck(cudaDeviceGetDefaultMemPool(&pool, dev), "cudaDeviceGetDefaultMemPool");
    uint64_t keep = ~uint64_t(0);
    ck(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    done.push_back(dev);
}

// The setup's full-grid checks that need no device: the material index's range and the gain
// cells' bounding box and placement.  A large solve runs them on a helper thread while it
// allocates its device arrays (for a 536^3 first solve both take tens of milliseconds: growing
// the device pool, scanning the region map).
struct GridScan {
    bool bad_index = false;  // a bE_index entry >= n_bE_rows
    int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
    long long out_of_range = 0, on_boundary = 0;
};

GridScan scan_grid(const fdtd_setup_v1& s, bool pec) {
    GridScan g;
    const int NxT = int(s.NxT), NyT = int(s.NyT), NzT = int(s.NzT);
    const size_t N = size_t(NxT) * NyT * NzT;
    if (s.bE_index && s.n_bE_rows > 0 && s.n_bE_rows <= 65535) {
        const uint16_t* hidx = s.bE_index;
        const uint32_t nr = s.n_bE_rows;
        uint16_t bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
        for (long long q = 0; q < (long long)N; ++q) bad |= uint16_t(hidx[q] >= nr);
        g.bad_index = bad != 0;
    }
    if (s.n_tls_regions > 0 && s.tls_region_map) {
        int lo0 = NxT, lo1 = NyT, lo2 = NzT, hi0 = -1, hi1 = -1, hi2 = -1;
        long long out_of_range = 0, on_boundary = 0;
        const int nreg = int(s.n_tls_regions);
#pragma omp parallel for reduction(min : lo0, lo1, lo2) reduction(max : hi0, hi1, hi2) \
    reduction(+ : out_of_range, on_boundary) schedule(static)
        for (int i = 0; i < NxT; ++i)
            for (int j = 0; j < NyT; ++j)
                for (int k = 0; k < NzT; ++k) {
                    const int32_t r = s.tls_region_map[(size_t(i) * NyT + j) * NzT + k];
                    if (r < 0) continue;
                    out_of_range += r >= nreg;
                    on_boundary += (i == 0 || j == 0 || k == 0) ||
                                   (pec && (i == NxT - 1 || j == NyT - 1 || k == NzT - 1));
                    lo0 = std::min(lo0, i); hi0 = std::max(hi0, i);
                    lo1 = std::min(lo1, j); hi1 = std::max(hi1, j);
                    lo2 = std::min(lo2, k); hi2 = std::max(hi2, k);
                }
        g.lo[0] = lo0; g.lo[1] = lo1; g.lo[2] = lo2;
        g.hi[0] = hi0; g.hi[1] = hi1; g.hi[2] = hi2;
        g.out_of_range = out_of_range;
        g.on_boundary = on_boundary;
    }
    return g;
}

struct PinnedChunks;
PinnedChunks& pinned_chunks(int dev, size_t bytes);

template <typename S, typename T>
Solver<S, T>::Solver(const fdtd_setup_v1& s, int dev, const ShardSpec* shard, bool pooled) {
    device = dev;
    pooled_ = true;
    if (const char* e = std::getenv("FDTD_B200_ALLOC")) pooled_ = pooled || std::string(e) != "malloc";
    ck(cudaSetDevice(dev), "cudaSetDevice");
    if (pooled_) keep_pool_memory(dev);
    ck(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
    constexpr int W = Vec<T>::W;
    NxT_ = int(s.NxT); NyT_ = int(s.NyT); NzT_ = int(s.NzT);
    np_ = int(s.npml);
    pec_ = s.pec_boundary != 0;
    if (pec_ && np_ != 0) throw Failure(FDTD_ERR_INVALID, "a PEC boundary has no CPML layer: npml must be 0");
    // A grid of 2^25 cells or more is scanned on a helper thread (the task reads only the
    // caller's view; an exception below waits for it in the future's destructor); a smaller one
    // in this thread when the result is first needed, where a thread and its OpenMP team would
    // cost more than the scan.
    const bool big = uint64_t(s.NxT) * s.NyT * s.NzT >= (uint64_t(1) << 25);
    std::future<GridScan> scan_task =
        std::async(big ? std::launch::async : std::launch::deferred, scan_grid, std::cref(s), pec_);
    std::optional<GridScan> scanned;
    auto scan = [&]() -> const GridScan& {
        if (!scanned) scanned = scan_task.get();
        return *scanned;
    };
    pinned_chunks(dev, kPinBytes);  // the process's first solve makes the staging chunks
    NxP_ = int(round_up(size_t(NxT_), 128 / sizeof(S)));
    if constexpr (!std::is_same_v<S, T>) {
        // 16-bit storage: E' = E / sE, H' = H / sH with sH = sE / eta0 so that E' and H' have
        // the same magnitude.  FP16's range ends at 65504 and its normal numbers at 6e-5, and sE
        // is fixed for the run, so it must leave the stored peak well below the top while the
        // weak early field (the pulse building up) stays above the bottom: the estimate
        // tau |I0| / (eps0 cell_area) -- the field a dipole's current would build in its cell
        // over one pulse width without radiating -- overshoots the peak by one to two decades,
        // and sE is that over 4096, as a power of two, which puts the stored peak near 40-400.
        // (Over 64, the earlier choice, left the first 250 steps of the 536^3 workload below
        // FP16's normal range: probe series error 1.0 against FP64, 0.084 now; DFT error after
        // 1000 steps 1.7e-3, 5.3e-4 now.)  A plane-wave soft source launches a wave of its own
        // amplitude E0: it counts as 64 |E0|.  BF16 has FP32's range: sE = 1.
        const double sE = field_scale_of(s, std::is_same_v<S, __half>);
        sE_ = sE;
        sH_ = sE / 376.730313668;
    }
    plane_ = size_t(NxP_) * NyT_;
    nflat_ = plane_ * NzT_;
    dt_ = s.dt;
    const size_t N = size_t(NxT_) * NyT_ * NzT_;

    StepArgs<S, T>& a = a_;
    a.NxT = NxT_; a.NyT = NyT_; a.NzT = NzT_; a.NxP = NxP_; a.np = np_;
    a.plane = (long long)plane_;
    // plane ranges: H is updated for global k < NzG - 1, E for global k >= 1, each on the owned planes
    shard_ = shard ? *shard : ShardSpec{0, NzT_, 0, NzT_};
    a.kz0 = shard_.kz0;
    a.NzG = shard_.NzG;
    a.kH0 = shard_.own0;
    a.kH1 = std::min(shard_.own1, shard_.NzG - 1 - shard_.kz0);
    a.kE0 = std::max(shard_.own0, 1 - shard_.kz0);
    a.kE1 = shard_.own1;
    // 16-bit storage: the H sweep's 8-cell interior vectors start at xi0 = np rounded up to 4
    // cells; the field arrays are offset by xoff_ elements so that xi0 (and every interior
    // vector) falls on a 16-byte boundary.  Every kernel addresses them from the offset pointer.
    xoff_ = 0;
    if constexpr (sizeof(S) == 2) xoff_ = int((8 - round_up(size_t(np_), size_t(W)) % 8) % 8);
    for (int c = 0; c < 6; ++c) fld_[c] = alloc<S>(nflat_ + 8) + xoff_;
    point_args_at();

    // bH must be uniform and aE = aH = 1 (sigma = 0, mu_r = 1).
    double bH = s.bH_uniform;
    if (s.bH[0]) bH = s.bH[0][0];
    auto all_equal = [N](const double* v, double x) {  // OpenMP scan of a full-grid array
        long long bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
        for (long long q = 0; q < (long long)N; ++q) bad += v[q] != x;
        return bad == 0;
    };
    for (int c = 0; c < 3; ++c) {
        if (s.aE[c] && !all_equal(s.aE[c], 1.0)) throw Failure(FDTD_ERR_UNSUPPORTED, "aE != 1 (lossy material) is not supported");
        if (s.aH[c] && !all_equal(s.aH[c], 1.0)) throw Failure(FDTD_ERR_UNSUPPORTED, "aH != 1 (magnetic loss) is not supported");
        if (s.bH[c] && !all_equal(s.bH[c], bH)) throw Failure(FDTD_ERR_UNSUPPORTED, "non-uniform bH (mu_r != 1) is not supported");
    }
    a.bH = T(bH * (sE_ / sH_));
    // Material: a uint16 row index per cell and a table of the distinct rows when the solve
    // has at most 65535 of them (2 bytes per cell per step instead of 3 words), else the
    // three arrays.  FDTD_B200_MATERIAL_INDEX=0 forces the arrays.
    // The setup view may bring the rows and the index (fdtd_setup_parse makes them); else they
    // are made here from the arrays.
    std::vector<std::array<double, 3>> rows;
    std::vector<uint16_t> rid;
    const uint16_t* hidx = nullptr;  // the host index (the view's, or rid)
    const char* mi = std::getenv("FDTD_B200_MATERIAL_INDEX");
    const bool want_index = !(mi && std::string(mi) == "0");
    bool have_index = false;
    if (want_index && s.bE_index && s.bE_rows && s.n_bE_rows > 0 && s.n_bE_rows <= 65535) {
        rows.resize(s.n_bE_rows);
        for (uint32_t r = 0; r < s.n_bE_rows; ++r)
            for (int c = 0; c < 3; ++c) rows[r][c] = s.bE_rows[3 * size_t(r) + c];
        hidx = s.bE_index;
        if (scan().bad_index) throw Failure(FDTD_ERR_INVALID, "bE_index holds a row number >= n_bE_rows");
        have_index = true;
    } else if (want_index) {
        have_index = fdtd::distinct_rows(s.bE, N, rows, rid);
        hidx = rid.data();
    }
    if (have_index) {
        std::vector<T> tab(4 * rows.size(), T(0));
        for (size_t r = 0; r < rows.size(); ++r)
            for (int c = 0; c < 3; ++c) tab[4 * r + c] = T(rows[r][c] * (sH_ / sE_));
        a.btab = upload(tab);
        uint16_t* d_idx = alloc<uint16_t>(nflat_);
        // the host index straight to the staging buffer as whole doubles, then the last N % 4
        // values through a padded double
        double* sbuf = staging();
        const size_t whole = N / 4;
        if (whole) h2d(reinterpret_cast<const double*>(hidx), sbuf, whole);
        if (N % 4) {
            uint16_t tail[4] = {0, 0, 0, 0};
            std::memcpy(tail, hidx + 4 * whole, (N % 4) * sizeof(uint16_t));
            ck(cudaMemcpyAsync(sbuf + whole, tail, sizeof(tail), cudaMemcpyHostToDevice, st_), "H2D");
            ck(cudaStreamSynchronize(st_), "H2D");
        }
        dim3 g((NzT_ + 31) / 32, (NxT_ + 31) / 32, NyT_), b(32, 8);
        k_index_from_idx3<<<g, b, 0, st_>>>(reinterpret_cast<const uint16_t*>(sbuf), d_idx, NxT_, NyT_, NzT_, NxP_);
        ++launches;
        ck(cudaGetLastError(), "k_index_from_idx3");
        ck(cudaStreamSynchronize(st_), "material index upload");
        a.bidx = d_idx;
        mat_rows_ = rows.size();
        material_rows = rows.size();
    } else {
        T* be[3];
        for (int c = 0; c < 3; ++c) {
            be[c] = alloc<T>(nflat_);
            to_device(s.bE[c], be[c], sH_ / sE_);
        }
        a.bEx = be[0]; a.bEy = be[1]; a.bEz = be[2];
    }
    // Where the staging pays (536^3 slab case, one B200): the E sweep with the row-indexed
    // material in FP32 (-2 %), FP64 (-3 %) and 16-bit storage (-10 %); the H sweep with 16-bit
    // storage only (-8 %; FP32 and FP64 +4 %).  With the three bE arrays the E staging takes 96 KB of shared
    // memory per block, leaves L1 too small for the neighbour rows, and is 15 % slower.
    pipe_ = a.bidx != nullptr;
    hpipe_ = sizeof(S) == 2;
    if (const char* e = std::getenv("FDTD_B200_H_PIPE")) hpipe_ = std::string(e) != "0";
    if (const char* e = std::getenv("FDTD_B200_E_PIPE")) pipe_ = a.bidx != nullptr && std::string(e) != "0";
    srm_ = std::is_same_v<S, __nv_bfloat16> && s.rounding == FDTD_ROUND_STOCHASTIC ? 1 : 0;
    if (hpipe_)
        ck(cudaFuncSetAttribute(h_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, int(HPipe<S>::bytes())),
           "cudaFuncSetAttribute");
    if (pipe_) {
        const int smem = int(EPipe<S>::bytes());
        for (bool sh : {false, true})
            ck(cudaFuncSetAttribute(e_kernel(sh), cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
               "cudaFuncSetAttribute");
    }

    // 1-D arrays
    std::vector<T> idx(NxP_, T(0)), idy(NyT_), idz(NzT_);
    for (int i = 0; i < NxT_; ++i) idx[i] = T(s.inv_dx[i]);
    for (int j = 0; j < NyT_; ++j) idy[j] = T(s.inv_dy[j]);
    for (int k = 0; k < NzT_; ++k) idz[k] = T(s.inv_dz[k]);
    a.idx = upload(idx); a.idy = upload(idy); a.idz = upload(idz);
    // 16-bit storage keeps psi * dx_min (psi is a field derivative); full precision keeps psi
    double psi_dx = 1.0;
    if constexpr (!std::is_same_v<S, T>) {
        psi_dx = *std::min_element(s.dx, s.dx + NxT_);
        psi_dx = std::min(psi_dx, *std::min_element(s.dy, s.dy + NyT_));
        psi_dx = std::min(psi_dx, *std::min_element(s.dz, s.dz + NzT_));
        if (shard_.psi_dx > 0) psi_dx = shard_.psi_dx;  // a shard scales psi as the whole solve
    }
    a.psc = T(1.0 / psi_dx);
    a.sr = std::is_same_v<S, __nv_bfloat16> && s.rounding == FDTD_ROUND_STOCHASTIC;
    const int Ns[3] = {NxT_, NyT_, NzT_};
    for (int ax = 0; ax < 3; ++ax) {
        const int n = Ns[ax];
        const int len = ax == 0 ? NxP_ : n;
        std::vector<T> ik(len, T(1)), bE(len, T(1)), cE(len, T(0)), bHp(len, T(1)), cH(len, T(0));
        for (int q = 0; q < n; ++q) {
            ik[q] = T(1.0 / s.cpml_kappa[ax][q]);
            bE[q] = T(s.cpml_bE[ax][q]); cE[q] = T(s.cpml_cE[ax][q] * psi_dx);
            bHp[q] = T(s.cpml_bH[ax][q]); cH[q] = T(s.cpml_cH[ax][q] * psi_dx);
        }
        a.ik[ax] = upload(ik);
        a.pbE[ax] = upload(bE); a.pcE[ax] = upload(cE);
        a.pbH[ax] = upload(bHp); a.pcH[ax] = upload(cH);
    }
    // psi slabs
    const size_t np2 = size_t(2 * np_);
    for (int q = 0; q < 6; ++q) { a.psiH[q] = nullptr; a.psiE[q] = nullptr; }
    if (np_ > 0) {
        const size_t xs = size_t(NzT_) * NyT_ * np2, ys = size_t(NzT_) * np2 * NxP_, zs = np2 * NyT_ * NxP_;
        // 0 *_y, 1 *_z, 2 *_z, 3 *_x, 4 *_x, 5 *_y
        const size_t sz[6] = {ys, zs, zs, xs, xs, ys};
        for (int q = 0; q < 6; ++q) {
            psi_sz_[q] = sz[q];
            psiH_[q] = alloc<S>(sz[q]);
            a.psiE[q] = alloc<S>(sz[q]);
            a.psiH[q] = psiH_[q];
        }
    }

    // gain block
    a.gain = 0;
    a.greg = nullptr; a.P0 = a.P1 = a.Nu = a.Ng = nullptr; a.gcoef = nullptr;
    a.gi0 = a.gj0 = a.gk0 = 0; a.gX = a.gY = a.gZ = 0;
    if (s.n_tls_regions > 0) {
        if (!s.tls_region_map || !s.tls_regions) throw Failure(FDTD_ERR_INVALID, "gain regions without region map");
        if (s.n_tls_regions > 127) throw Failure(FDTD_ERR_UNSUPPORTED, "more than 127 gain regions");
        const GridScan& gs = scan();
        if (gs.out_of_range) throw Failure(FDTD_ERR_INVALID, "region map entry out of range");
        if (gs.on_boundary)
            throw Failure(FDTD_ERR_UNSUPPORTED, pec_ ? "gain cells on the outer faces of a PEC grid"
                                                     : "gain cells on the i=0/j=0/k=0 boundary planes");
        const int* lo = gs.lo;
        const int* hi = gs.hi;
        if (hi[0] >= 0) {
            has_gain_ = true;
            a.gain = 1;
            a.gi0 = lo[0]; a.gj0 = lo[1]; a.gk0 = lo[2];
            a.gX = hi[0] - lo[0] + 1; a.gY = hi[1] - lo[1] + 1; a.gZ = hi[2] - lo[2] + 1;
            const size_t ng = size_t(a.gX) * a.gY * a.gZ;
            std::vector<int8_t> reg(ng);
#pragma omp parallel for schedule(static)
            for (int k = 0; k < a.gZ; ++k)
                for (int j = 0; j < a.gY; ++j)
                    for (int i = 0; i < a.gX; ++i)
                        reg[(size_t(k) * a.gY + j) * a.gX + i] = int8_t(
                            s.tls_region_map[(size_t(i + a.gi0) * NyT_ + (j + a.gj0)) * NzT_ + (k + a.gk0)]);
            a.greg = upload(reg);
            a.P0 = alloc<T>(ng); a.P1 = alloc<T>(ng); a.Nu = alloc<T>(ng); a.Ng = alloc<T>(ng);
            std::vector<GainCoef<T>> gc(s.n_tls_regions);
            for (uint32_t r = 0; r < s.n_tls_regions; ++r) {
                const fdtd_tls_region_v1& R = s.tls_regions[r];
                GainCoef<T>& g = gc[r];
                g.kapaN0 = T(R.kapa_coeff * R.N0 * sE_);
                g.pa2 = T(R.pa2); g.pa3 = T(R.pa3); g.inv_dt = T(R.inv_dt);
                g.inv_N0 = T(R.N0 > 0 ? 1.0 / R.N0 : 0.0);
                g.N0 = T(R.N0);
                g.dt = T(s.dt);
                g.inv_tau = T(1.0 / R.tau);
                g.inv_hbar_omega = T(sE_ / (R.hbar * R.omega_a));
                g.dp_scale = T(1.0 / sH_);
                g.pump = T(R.pump_rate);
                g.clamp = R.enable_population_clamp;
                g.active = R.N0 > 0 ? 1 : 0;
            }
            a.gcoef = upload(gc);
            if (s.tls_Nu) upload_gain_box(s.tls_Nu, reg, a.Nu);
            if (s.tls_Ng) upload_gain_box(s.tls_Ng, reg, a.Ng);
        }
    }

    // sources
    if (s.n_dipoles > uint32_t(kMaxSources)) throw Failure(FDTD_ERR_UNSUPPORTED, "more than 8 point sources");
    for (uint32_t q = 0; q < s.n_dipoles; ++q) {
        const fdtd_dipole_v1& d = s.dipoles[q];
        if (d.i >= s.NxT || d.j >= s.NyT || d.k >= s.NzT) throw Failure(FDTD_ERR_INVALID, "source cell outside the grid");
        if (d.polarization < 0 || d.polarization > 5) throw Failure(FDTD_ERR_INVALID, "source polarization must be 0..5");
        dip_.push_back(d);
    }


    if (s.n_sheets > uint32_t(kMaxSheets)) throw Failure(FDTD_ERR_UNSUPPORTED, "more than 2 plane-wave sources");
    for (uint32_t q = 0; q < s.n_sheets; ++q) {
        const fdtd_sheet_v1& w = s.sheets[q];
        const uint64_t N[3] = {s.NxT, s.NyT, s.NzT};
        if (w.axis < 0 || w.axis > 2 || w.comp < 0 || w.comp > 2 || w.comp == w.axis || w.plane >= N[w.axis] ||
            !(w.d > 0))
            throw Failure(FDTD_ERR_INVALID, "bad plane-wave source");
        sheets_.push_back(w);
    }

    // probes / DFT
    save_every_ = std::max<uint32_t>(1, s.save_every);
    nprobes_ = s.n_probes;
    nf_ = s.n_dft_freqs;
    if (nprobes_) {
        std::vector<ProbeDev> pd(nprobes_);
        for (uint32_t q = 0; q < nprobes_; ++q) {
            const fdtd_probe_v1& p = s.probes[q];
            if (p.i >= s.NxT || p.j >= s.NyT || p.k >= s.NzT || p.component < 0 || p.component > 11)
                throw Failure(FDTD_ERR_INVALID, "probe outside the grid or bad component");
            pd[q].off = (long long)((size_t(p.k) * NyT_ + p.j) * NxP_ + p.i);
            pd[q].comp = p.component;
        }
        d_probes_ = upload(pd);
        if (nf_) {
            d_freqs_ = upload(std::vector<double>(s.dft_freqs, s.dft_freqs + nf_));
            d_dft_ = alloc<double>(size_t(2) * nprobes_ * nf_);
        }
    }

    // monitor
    interval_ = s.monitor_interval;
    d_dx_ = upload(std::vector<double>(s.dx, s.dx + NxT_));
    d_dy_ = upload(std::vector<double>(s.dy, s.dy + NyT_));
    d_dz_ = upload(std::vector<double>(s.dz, s.dz + NzT_));
    d_acc_ = alloc<DiagAccum>(1);
    MonitorState ms{};
    ms.stable = 1;
    ms.has_gain = has_gain_ ? 1 : 0;
    ms.thr_E = s.max_E; ms.thr_P = s.max_P; ms.thr_cons = s.conservation_err; ms.thr_growth = s.growth_rate;
    d_ms_ = upload(std::vector<MonitorState>{ms});
    d_status_ = alloc<unsigned>(1);
    a.status = d_status_;

    // x split: W-aligned interior without x-slab cells, and the edge vectors around it
    SweepGeom& g = geom_;
    // interior vectors of WI cells (16-bit storage: 8 in the H sweep, one 16-byte word per
    // array; its E sweep covers the same interior with 4-cell vectors, gxi_E), edge vectors of W
    constexpr int WI = sizeof(S) == 2 ? 8 : W;
    g.xi0 = int(round_up(size_t(np_), size_t(W)));
    g.xi1 = std::max(g.xi0, g.xi0 + (NxT_ - np_ - g.xi0) / WI * WI);
    // Interior row segments of 32, 16 or 8 lanes.  A narrow interior (at most two 32-lane
    // segments) takes the width that leaves the fewest lanes idle in the last block column,
    // ties to the wider segment (its warps load one x-neighbour per plane, not one per row);
    // a wide one keeps 32-lane rows.  Measured on one B200, FP32 sweeps: a 156-cell-wide
    // cavity (35 interior vectors) runs at 23.1 Gcell/s on 32-lane rows, 25.7 on 8-lane rows;
    // the 536^3 grid (130 vectors, 81 % of 32-lane rows busy) at 74.2 on 32-lane rows, 71.6 on
    // 16 and 68.9 on 8 -- with enough blocks to keep HBM busy the extra row ends cost more than
    // the idle lanes.  FDTD_B200_LANES=32|16|8 sets the width (results do not depend on it).
    const int nvec = (g.xi1 - g.xi0) / WI;
    g.lanes = 32;
    if (nvec <= 64)
        for (int L : {16, 8})
            if ((nvec + L - 1) / L * L < (nvec + g.lanes - 1) / g.lanes * g.lanes) g.lanes = L;
    if (const char* e = std::getenv("FDTD_B200_LANES")) {
        const int L = std::atoi(e);
        if (L != 32 && L != 16 && L != 8) throw Failure(FDTD_ERR_INVALID, "FDTD_B200_LANES must be 32, 16 or 8");
        g.lanes = L;
    }
    const int rows_blk = kBlockY * (32 / g.lanes);  // rows of an interior block
    g.gxi = (nvec + g.lanes - 1) / g.lanes;
    g.nl = g.xi0 / W;
    g.ne = g.nl + std::max(0, (NxT_ - g.xi1 + W - 1) / W);
    if (g.ne > 32 * kBlockY) throw Failure(FDTD_ERR_UNSUPPORTED, "CPML too thick for the sweep launch shape");
    g.er = g.ne ? (32 * kBlockY) / g.ne : 1;
    const int gxH = g.gxi + (g.ne ? 1 : 0), gxE = gxi_E<S>(g) + (g.ne ? 1 : 0);
    const int gyE = std::max((NyT_ + rows_blk - 1) / rows_blk, g.ne ? (NyT_ + g.er - 1) / g.er : 0);
    // launch shapes: z-chunks of at most 16 planes, and enough of them that the grid holds
    // several waves of blocks.  Measured on the 536^3 CPML + gain workload (one B200): chunks
    // of 67 -> 34 -> 16 planes take the E sweep from 1.258 to 1.159 to 1.107 ms (FP32) and from
    // 1.006 to 0.900 to 0.868 ms (BF16), the H sweep from 1.025 to 0.972 ms (FP32); 12 and 8
    // planes are no faster.  Short chunks balance the blocks' work (a chunk of an edge column
    // or a CPML row runs longer than an interior one) and shorten the last wave.
    auto chunk = [&](int rows, int planes, int gx) {
        const int bxy = std::max(1, gx * ((rows + rows_blk - 1) / rows_blk));
        const int want = std::max(1, (148 * 16 + bxy - 1) / bxy);
        const int zc = std::max({1, std::min(want, std::max(1, planes / 8)), (planes + 15) / 16});
        return std::max(1, (planes + zc - 1) / zc);
    };
    kchunkH_ = chunk(NyT_ - 1, NzT_ - 1, gxH);
    kchunkE_ = chunk(NyT_, NzT_, gxE);
    if (const char* e = std::getenv("FDTD_B200_KCHUNK")) kchunkH_ = kchunkE_ = std::max(1, std::atoi(e));
    if (gyE > 65535) throw Failure(FDTD_ERR_INVALID, "grid too large for the sweep launch shape (NyT)");
    gridH_ = dim3(gxH, gyE, std::max(1, (a.kH1 + kchunkH_ - 1) / kchunkH_));
    gridE_ = dim3(gxE, gyE, std::max(1, (a.kE1 + kchunkE_ - 1) / kchunkE_));
    if (const char* p = std::getenv("FDTD_B200_KERNEL_PATH")) set_path(std::atoi(p));
    ck(cudaStreamSynchronize(st_), "setup upload");
}

template <typename S, typename T>
void Solver<S, T>::setup_slabs() {
    int P = 4;
    if (const char* e = std::getenv("FDTD_B200_SLAB_PLANES")) P = std::max(1, std::atoi(e));
    plan_.P = P;
    plan_.nslab = (NzT_ + P - 1) / P;
    plan_.gxH = int(gridH_.x);
    plan_.nH = int(gridH_.x * gridH_.y);
    plan_.gxE = int(gridE_.x);
    plan_.nE = int(gridE_.x * gridE_.y);
    if ((long long)plan_.nslab * (plan_.nH + plan_.nE) > 0x7fffffffLL) throw Failure(FDTD_ERR_INVALID, "grid too large for the slab-ordered step");
    // Bound on one dependency wait of an E tile: FDTD_B200_WAIT_NS nanoseconds (at least 1000),
    // else 2 s.  FDTD_B200_SLAB_HOLD=1 leaves the hold word set, so that every E tile's wait
    // runs out and the step ends with FDTD_ERR_TIMEOUT (how the bounded wait is tested).
    plan_.wait_ns = kWaitNs;
    if (const char* e = std::getenv("FDTD_B200_WAIT_NS")) plan_.wait_ns = std::max(1000ull, std::strtoull(e, nullptr, 10));
    if (const char* e = std::getenv("FDTD_B200_SLAB_HOLD")) slab_hold_ = std::string(e) == "1";
    d_ctr_ = alloc<unsigned>(size_t(plan_.nslab) + 2);
    int sms = 148, per = 0;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    const auto slabs_fn = sheets_.empty() ? (a_.bidx ? k_step_slabs<S, T, false, true> : k_step_slabs<S, T, false, false>)
                                          : (a_.bidx ? k_step_slabs<S, T, true, true> : k_step_slabs<S, T, true, false>);
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, slabs_fn, 32 * kBlockY, 0),
       "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per < 1) throw Failure(FDTD_ERR_CUDA, "slab-ordered step kernel does not fit on an SM");
    gridS_ = dim3(unsigned(sms * per));
}

template <typename S, typename T>
void Solver<S, T>::pec_faces() {
    const int k0 = shard_.own0, k1 = shard_.own1;
    const int zlo = shard_.kz0 + k0 == 0 ? k0 : -1;                 // global plane 0 is ours
    const int zhi = shard_.kz0 + k1 == shard_.NzG ? k1 - 1 : -1;    // global plane NzG - 1 is ours
    const long long faces = 2ll * ((long long)NxT_ * NyT_ + (long long)NxT_ * (k1 - k0) + (long long)NyT_ * (k1 - k0));
    const unsigned nb = unsigned(std::min<long long>((faces + 255) / 256, 148 * 8));
    k_pec_faces<S><<<nb, 256, 0, st_>>>(a_.Ex, a_.Ey, a_.Ez, NxT_, NyT_, NxP_, k0, k1, zlo, zhi);
    ++launches;
}

template <typename S, typename T>
void Solver<S, T>::point_args_at() {
    a_.Ex = fld_[0]; a_.Ey = fld_[1]; a_.Ez = fld_[2];
    a_.Hx = fld_[3]; a_.Hy = fld_[4]; a_.Hz = fld_[5];
}

template <typename S, typename T>
void Solver<S, T>::set_timing(int mode) {
    if (mode < FDTD_TIMING_OFF || mode > FDTD_TIMING_KERNELS) throw Failure(FDTD_ERR_INVALID, "bad timing mode");
    ck(cudaSetDevice(device), "cudaSetDevice");
    if (mode != FDTD_TIMING_OFF && !ev_[0])
        for (auto& e : ev_) ck(cudaEventCreate(&e), "cudaEventCreate");
    timing_ = mode;
    tm_ = fdtd_timing_v1{};
}

template <typename S, typename T>
Solver<S, T>::~Solver() {
    cudaSetDevice(device);
    if (st_) cudaStreamSynchronize(st_);
    if (writer_) {
        try {
            writer_->drain();
        } catch (const std::exception&) {
        }
        writer_.reset();
    }
    for (int q = 0; q < kOutSlots; ++q) {
        if (h_oslot_[q]) cudaFreeHost(h_oslot_[q]);
        if (oslot_ev_[q]) cudaEventDestroy(oslot_ev_[q]);
    }
    if (h_trec_) cudaFreeHost(h_trec_);
    for (int q = 0; q < kTlsSlots; ++q)
        if (trec_ev_[q]) cudaEventDestroy(trec_ev_[q]);
    for (auto& e : ev_) if (e) cudaEventDestroy(e);
    for (void* p : ptrs_) dev_free(p);
    if (d_stage_) dev_free(d_stage_);
    if (d_series_) dev_free(d_series_);
    if (st_) cudaStreamDestroy(st_);
}

template <typename S, typename T>
double* Solver<S, T>::staging() {
    if (!d_stage_) {
        dev_alloc(reinterpret_cast<void**>(&d_stage_), size_t(NxT_) * NyT_ * NzT_ * sizeof(double));
        dev_bytes += size_t(NxT_) * NyT_ * NzT_ * sizeof(double);
    }
    return d_stage_;
}

// Two pinned staging chunks per device, shared by every solve of the process: made at the
// first large copy on the device and kept for the life of the process, so that creating and
// destroying a solve neither pins nor unpins host memory.  A copy holds them (mu) throughout.
struct PinnedChunks {
    std::mutex mu;
    void* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

PinnedChunks& pinned_chunks(int dev, size_t bytes) {
    static std::mutex m;
    static std::map<int, PinnedChunks*> all;  // never freed: released with the process
    PinnedChunks* p;
    {
        std::lock_guard<std::mutex> l(m);
        PinnedChunks*& q = all[dev];
        if (!q) q = new PinnedChunks;
        p = q;
    }
    std::lock_guard<std::mutex> l(p->mu);
    for (int b = 0; b < 2; ++b) {
        if (!p->buf[b]) ck(cudaHostAlloc(&p->buf[b], bytes, cudaHostAllocDefault), "cudaHostAlloc");
        if (!p->ev[b]) ck(cudaEventCreateWithFlags(&p->ev[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    return *p;
}

// memcpy split over the host threads (the pageable side of a chunk copy)
static void par_copy(void* dst, const void* src, size_t bytes) {
    const size_t piece = size_t(1) << 20;
    const long long n = (long long)((bytes + piece - 1) / piece);
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < n; ++q) {
        const size_t o = size_t(q) * piece;
        std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, std::min(piece, bytes - o));
    }
}

template <typename S, typename T>
void Solver<S, T>::h2d(const double* h, double* d, size_t n) {
    if (n * sizeof(double) <= kPinBytes) {  // small grids: one copy, no pinned buffers to set up
        ck(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, st_), "H2D");
        ck(cudaStreamSynchronize(st_), "H2D");
        return;
    }
    PinnedChunks& pc = pinned_chunks(device, kPinBytes);
    std::lock_guard<std::mutex> l(pc.mu);
    const size_t chunk = kPinBytes / sizeof(double);
    for (size_t off = 0, it = 0; off < n; off += chunk, ++it) {
        const int b = int(it & 1);
        const size_t m = std::min(chunk, n - off);
        ck(cudaEventSynchronize(pc.ev[b]), "pinned buffer");  // its previous DMA is done
        par_copy(pc.buf[b], h + off, m * sizeof(double));
        ck(cudaMemcpyAsync(d + off, pc.buf[b], m * sizeof(double), cudaMemcpyHostToDevice, st_), "H2D");
        ck(cudaEventRecord(pc.ev[b], st_), "cudaEventRecord");
    }
    ck(cudaStreamSynchronize(st_), "H2D");  // the chunks are free for the next copy
}

template <typename S, typename T>
void Solver<S, T>::d2h(const double* d, double* h, size_t n) {
    if (n * sizeof(double) <= kPinBytes) {
        ck(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st_), "D2H");
        ck(cudaStreamSynchronize(st_), "D2H");
        return;
    }
    PinnedChunks& pc = pinned_chunks(device, kPinBytes);
    std::lock_guard<std::mutex> l(pc.mu);
    const size_t chunk = kPinBytes / sizeof(double);
    const size_t nch = (n + chunk - 1) / chunk;
    auto issue = [&](size_t it) {
        const size_t off = it * chunk, m = std::min(chunk, n - off);
        ck(cudaMemcpyAsync(pc.buf[it & 1], d + off, m * sizeof(double), cudaMemcpyDeviceToHost, st_), "D2H");
        ck(cudaEventRecord(pc.ev[it & 1], st_), "cudaEventRecord");
    };
    if (nch) issue(0);
    for (size_t it = 0; it < nch; ++it) {
        if (it + 1 < nch) issue(it + 1);  // the other buffer was drained in the previous iteration
        const size_t off = it * chunk, m = std::min(chunk, n - off);
        ck(cudaEventSynchronize(pc.ev[it & 1]), "D2H chunk");
        par_copy(h + off, pc.buf[it & 1], m * sizeof(double));
    }
}

// Initial gain state: the bounding box is cut out of the idx3 array on the host (cells
// outside the gain regions hold 0, as k_gain_block stores them) and only the box is copied.
template <typename S, typename T>
void Solver<S, T>::upload_gain_box(const double* h, const std::vector<int8_t>& reg, T* dst) {
    const int gX = a_.gX, gY = a_.gY, gZ = a_.gZ;
    std::vector<T> box(size_t(gX) * gY * gZ);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < gZ; ++k)
        for (int j = 0; j < gY; ++j)
            for (int i = 0; i < gX; ++i) {
                const size_t t = (size_t(k) * gY + j) * gX + i;
                const size_t id = (size_t(i + a_.gi0) * NyT_ + (j + a_.gj0)) * NzT_ + (k + a_.gk0);
                box[t] = reg[t] >= 0 ? T(h[id]) : T(0);
            }
    ck(cudaMemcpyAsync(dst, box.data(), box.size() * sizeof(T), cudaMemcpyHostToDevice, st_), "gain box");
    ck(cudaStreamSynchronize(st_), "gain box");
}

template <typename S, typename T>
template <typename D>
void Solver<S, T>::to_device(const double* h, D* dst, double scale) {
    if (!h) throw Failure(FDTD_ERR_INVALID, "null host array");
    double* sbuf = staging();
    h2d(h, sbuf, size_t(NxT_) * NyT_ * NzT_);
    dim3 g((NzT_ + 31) / 32, (NxT_ + 31) / 32, NyT_), b(32, 8);
    k_from_idx3<D><<<g, b, 0, st_>>>(sbuf, dst, NxT_, NyT_, NzT_, NxP_, scale);
    ++launches;
    ck(cudaGetLastError(), "k_from_idx3");
    ck(cudaStreamSynchronize(st_), "to_device");
}

template <typename S, typename T>
template <typename D>
void Solver<S, T>::from_device(const D* src, double* h, double scale) {
    if (!h) throw Failure(FDTD_ERR_INVALID, "null host array");
    double* sbuf = staging();
    dim3 g((NzT_ + 31) / 32, (NxT_ + 31) / 32, NyT_), b(32, 8);
    k_to_idx3<D><<<g, b, 0, st_>>>(src, sbuf, NxT_, NyT_, NzT_, NxP_, scale);
    ++launches;
    ck(cudaGetLastError(), "k_to_idx3");
    d2h(sbuf, h, size_t(NxT_) * NyT_ * NzT_);
    ck(cudaStreamSynchronize(st_), "from_device");
}

template <typename S, typename T>
void Solver<S, T>::set_field(int comp, const double* h) {
    if (comp < 0 || comp > 5) throw Failure(FDTD_ERR_INVALID, "component must be 0..5");
    to_device(h, fld_[comp], 1.0 / (comp < 3 ? sE_ : sH_));
    ck(cudaStreamSynchronize(st_), "set_field");
}

template <typename S, typename T>
void Solver<S, T>::get_field(int comp, double* h) {
    if (comp < 0 || comp > 5) throw Failure(FDTD_ERR_INVALID, "component must be 0..5");
    from_device(fld_[comp], h, comp < 3 ? sE_ : sH_);
}

template <typename S, typename T>
void Solver<S, T>::set_tls(int which, const double* h) {
    if (which < 0 || which > 3) throw Failure(FDTD_ERR_INVALID, "which must be FDTD_TLS_*");
    if (!has_gain_) throw Failure(FDTD_ERR_INVALID, "solve has no gain region");
    T* dst = which == FDTD_TLS_PZ ? ((steps & 1) ? a_.P1 : a_.P0)
           : which == FDTD_TLS_PZ_PREV ? ((steps & 1) ? a_.P0 : a_.P1)
           : which == FDTD_TLS_NU ? a_.Nu : a_.Ng;
    double* sbuf = staging();
    h2d(h, sbuf, size_t(NxT_) * NyT_ * NzT_);
    k_gain_block<T><<<592, 256, 0, st_>>>(sbuf, dst, a_.greg, a_.gi0, a_.gj0, a_.gk0, a_.gX, a_.gY, a_.gZ, NyT_, NzT_, 1);
    ++launches;
    ck(cudaGetLastError(), "k_gain_block");
    ck(cudaStreamSynchronize(st_), "set_tls");
}

template <typename S, typename T>
void Solver<S, T>::get_tls(int which, double* h) {
    if (which < 0 || which > 3) throw Failure(FDTD_ERR_INVALID, "which must be FDTD_TLS_*");
    const size_t N = size_t(NxT_) * NyT_ * NzT_;
    std::memset(h, 0, N * sizeof(double));
    if (!has_gain_) return;
    T* src = which == FDTD_TLS_PZ ? ((steps & 1) ? a_.P1 : a_.P0)
           : which == FDTD_TLS_PZ_PREV ? ((steps & 1) ? a_.P0 : a_.P1)
           : which == FDTD_TLS_NU ? a_.Nu : a_.Ng;
    double* sbuf = staging();
    ck(cudaMemsetAsync(sbuf, 0, N * sizeof(double), st_), "memset");
    k_gain_block<T><<<592, 256, 0, st_>>>(sbuf, src, a_.greg, a_.gi0, a_.gj0, a_.gk0, a_.gX, a_.gY, a_.gZ, NyT_, NzT_, 0);
    ++launches;
    ck(cudaGetLastError(), "k_gain_block");
    d2h(sbuf, h, N);
    ck(cudaStreamSynchronize(st_), "get_tls");
}

template <typename S, typename T>
void Solver<S, T>::ensure_series(uint64_t samples) {
    if (nprobes_ == 0 || samples <= series_cap_) return;
    uint64_t cap = std::max<uint64_t>(samples, series_cap_ * 2);
    double* d = nullptr;
    dev_alloc(reinterpret_cast<void**>(&d), cap * nprobes_ * sizeof(double));
    if (d_series_) {
        ck(cudaMemcpyAsync(d, d_series_, series_count_ * nprobes_ * sizeof(double), cudaMemcpyDeviceToDevice, st_), "series copy");
        ck(cudaStreamSynchronize(st_), "series copy");
        dev_free(d_series_);
        dev_bytes -= series_cap_ * nprobes_ * sizeof(double);
    }
    d_series_ = d;
    dev_bytes += cap * nprobes_ * sizeof(double);
    series_cap_ = cap;
}

template <typename S, typename T>
void Solver<S, T>::run(uint64_t n) {
    ck(cudaSetDevice(device), "cudaSetDevice");
    if (path_ == 2 && !d_ctr_) setup_slabs();
    const uint64_t n0 = steps;
    const uint64_t last = n0 + n;  // exclusive
    ensure_series((last + save_every_ - 1) / save_every_);
    const dim3 blk(32, kBlockY);
    ESrc src{};
    src_static(src);
    const int pthreads = int(nprobes_ * std::max<uint32_t>(nf_, 1));
    const bool per_kernel = timing_ == FDTD_TIMING_KERNELS;
    if (timing_ == FDTD_TIMING_RUN) ck(cudaEventRecord(ev_[0], st_), "cudaEventRecord");
    for (uint64_t s = n0; s < last; ++s) {
        src_step(src, s);
        if (per_kernel) ck(cudaEventRecord(ev_[0], st_), "cudaEventRecord");
        if (path_ == 2) {
            ck(cudaMemsetAsync(d_ctr_, 0, (size_t(plan_.nslab) + 2) * sizeof(unsigned), st_), "cudaMemsetAsync");
            if (slab_hold_)
                ck(cudaMemsetAsync(d_ctr_ + plan_.nslab + 1, 0xff, sizeof(unsigned), st_), "cudaMemsetAsync");
            if (per_kernel) ck(cudaEventRecord(ev_[0], st_), "cudaEventRecord");
            const auto slabs = src.ns ? (a_.bidx ? k_step_slabs<S, T, true, true> : k_step_slabs<S, T, true, false>)
                                      : (a_.bidx ? k_step_slabs<S, T, false, true> : k_step_slabs<S, T, false, false>);
            slabs<<<gridS_, blk, 0, st_>>>(a_, src, geom_, plan_, d_ctr_, d_status_);
            if (per_kernel) ck(cudaEventRecord(ev_[1], st_), "cudaEventRecord");
            launches += 1;
        } else {
            h_kernel()<<<gridH_, blk, hpipe_ ? HPipe<S>::bytes() : 0, st_>>>(a_, kchunkH_, geom_, src.step);
            if (per_kernel) ck(cudaEventRecord(ev_[1], st_), "cudaEventRecord");
            const size_t smem = pipe_ ? EPipe<S>::bytes() : 0;
            e_kernel(src.ns != 0)<<<gridE_, blk, smem, st_>>>(a_, kchunkE_, src, geom_);
            launches += 2;
        }
        if (pec_) pec_faces();
        if (per_kernel) ck(cudaEventRecord(ev_[2], st_), "cudaEventRecord");
        if (nprobes_) {
            const long long sample = (s % save_every_ == 0) ? (long long)(s / save_every_) : -1;
            k_probe_dft<S, T><<<(pthreads + 127) / 128, 128, 0, st_>>>(a_, d_probes_, int(nprobes_), d_freqs_, int(nf_),
                                                                         d_dft_, d_series_, sample, double(s + 1) * dt_, dt_,
                                                                         sE_, sH_);
            ++launches;
            if (sample >= 0) series_count_ = uint64_t(sample) + 1;
        }
        if (writer_ && !oplan_.movies.empty() && s % save_every_ == 0) capture_movies();
        if (writer_ && oplan_.tls && s % save_every_ == 0) capture_tls(s);
        if (interval_ && s % interval_ == 0) {
            k_monitor_reduce<S, T><<<8 * 148, 256, 0, st_>>>(a_, size_t(shard_.own0) * plane_, size_t(shard_.own1) * plane_,
                                                             d_dx_, d_dy_, d_dz_, int((s + 1) & 1), d_acc_, sE_);
            k_monitor_eval<<<1, 1, 0, st_>>>(d_acc_, d_ms_, d_status_, s);
            launches += 2;
        }
        if (per_kernel) {
            ck(cudaEventRecord(ev_[3], st_), "cudaEventRecord");
            ck(cudaEventSynchronize(ev_[3]), "cudaEventSynchronize");
            float a = 0, b = 0, c = 0;
            ck(cudaEventElapsedTime(&a, ev_[0], ev_[1]), "cudaEventElapsedTime");
            ck(cudaEventElapsedTime(&b, ev_[1], ev_[2]), "cudaEventElapsedTime");
            ck(cudaEventElapsedTime(&c, ev_[2], ev_[3]), "cudaEventElapsedTime");
            tm_.h_ms += a; tm_.e_ms += b; tm_.aux_ms += c;
            tm_.steps += 1;
        }
    }
    if (timing_ == FDTD_TIMING_RUN) ck(cudaEventRecord(ev_[3], st_), "cudaEventRecord");
    ck(cudaGetLastError(), "step kernels");
    unsigned status = 0;
    ck(cudaMemcpyAsync(&status, d_status_, sizeof(unsigned), cudaMemcpyDeviceToHost, st_), "status");
    ck(cudaStreamSynchronize(st_), "run");
    if (timing_ == FDTD_TIMING_RUN) {
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, ev_[0], ev_[3]), "cudaEventElapsedTime");
        tm_.run_ms += ms;
        tm_.steps += n;
    }
    if (status & kStatusTimeout)
        throw Failure(FDTD_ERR_TIMEOUT, "a bounded device wait expired; the state is invalid and the handle stays stopped");
    if (status) {
        MonitorState ms{};
        ck(cudaMemcpy(&ms, d_ms_, sizeof(ms), cudaMemcpyDeviceToHost), "monitor state");
        steps = ms.step + 1;
        series_count_ = std::min<uint64_t>(series_count_, (steps + save_every_ - 1) / save_every_);
        if (writer_) write_point_samples();
        throw Failure(FDTD_ERR_UNSTABLE, "stability monitor stopped the solve at step " + std::to_string(ms.step));
    }
    steps = last;
    if (writer_) write_point_samples();
}

// ---- the phases of one step, for the sharded stepper (run() keeps its own loop)
template <typename S, typename T>
void Solver<S, T>::phase_H(uint64_t s) {
    const dim3 blk(32, kBlockY);
    h_kernel()<<<gridH_, blk, hpipe_ ? HPipe<S>::bytes() : 0, st_>>>(a_, kchunkH_, geom_, unsigned(s));
    ++launches;
}

// E sweep, probes / DFT and, on monitor steps, this shard's part of the monitor reduction
// (the evaluation is made once, on the combined accumulators).
template <typename S, typename T>
void Solver<S, T>::phase_E(uint64_t s, ESrc& src, bool monitor) {
    const dim3 blk(32, kBlockY);
    src_step(src, s);
    const size_t smem = pipe_ ? EPipe<S>::bytes() : 0;
    e_kernel(src.ns != 0)<<<gridE_, blk, smem, st_>>>(a_, kchunkE_, src, geom_);
    ++launches;
    if (pec_) pec_faces();
    if (nprobes_) {
        const int pthreads = int(nprobes_ * std::max<uint32_t>(nf_, 1));
        const long long sample = (s % save_every_ == 0) ? (long long)(s / save_every_) : -1;
        k_probe_dft<S, T><<<(pthreads + 127) / 128, 128, 0, st_>>>(a_, d_probes_, int(nprobes_), d_freqs_, int(nf_),
                                                                     d_dft_, d_series_, sample, double(s + 1) * dt_, dt_,
                                                                     sE_, sH_);
        ++launches;
        if (sample >= 0) series_count_ = uint64_t(sample) + 1;
    }
    if (monitor) {
        k_monitor_reduce<S, T><<<8 * 148, 256, 0, st_>>>(a_, size_t(shard_.own0) * plane_, size_t(shard_.own1) * plane_,
                                                         d_dx_, d_dy_, d_dz_, int((s + 1) & 1), d_acc_, sE_);
        ++launches;
    }
}

template <typename S, typename T>
void Solver<S, T>::attach_outputs(const fdtd::SimSetup& Sp, const std::string& root) {
    if (writer_) throw Failure(FDTD_ERR_INVALID, "outputs are already attached");
    if (steps != 0) throw Failure(FDTD_ERR_INVALID, "outputs can only be attached before the first step");
    if (Sp.NxT != size_t(NxT_) || Sp.NyT != size_t(NyT_) || Sp.NzT != size_t(NzT_) || Sp.save_every != save_every_)
        throw Failure(FDTD_ERR_INVALID, "the setup does not match the handle (grid or SAVE_EVERY)");
    fdtd::OutputPlan plan;
    try {
        plan = fdtd::make_output_plan(Sp);
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_INVALID, e.what());
    }
    size_t comps = 0;
    for (const auto& p : plan.points) comps += p.components.size();
    if (comps != nprobes_) throw Failure(FDTD_ERR_INVALID, "the setup's point detectors do not match the handle's probes");
    try {
        fdtd::write_setup_outputs(Sp, plan, root);
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_IO, e.what());
    }
    ck(cudaSetDevice(device), "cudaSetDevice");
    const size_t word = plan.float64 ? sizeof(double) : sizeof(float);
    oslot_bytes_ = 0;
    for (const auto& m : plan.movies) {
        mov_off_.push_back(oslot_bytes_);
        mov_bytes_.push_back(m.dim1 * m.dim2 * word);
        oslot_bytes_ += round_up(m.dim1 * m.dim2 * word, 256);
    }
    if (oslot_bytes_) {
        for (int q = 0; q < kOutSlots; ++q) {
            d_oslot_[q] = alloc<char>(oslot_bytes_, false);
            ck(cudaHostAlloc(reinterpret_cast<void**>(&h_oslot_[q]), oslot_bytes_, cudaHostAllocDefault), "cudaHostAlloc");
            ck(cudaEventCreateWithFlags(&oslot_ev_[q], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
    if (plan.tls) {
        d_trec_ = alloc<TlsRecord>(kTlsSlots);
        ck(cudaHostAlloc(reinterpret_cast<void**>(&h_trec_), kTlsSlots * sizeof(TlsRecord), cudaHostAllocDefault),
           "cudaHostAlloc");
        for (int q = 0; q < kTlsSlots; ++q)
            ck(cudaEventCreateWithFlags(&trec_ev_[q], cudaEventDisableTiming), "cudaEventCreate");
        const StepArgs<S, T>& a = a_;
        if (has_gain_ && plan.mon_valid) {
            const long long i = (long long)plan.mon_i - a.gi0, j = (long long)plan.mon_j - a.gj0,
                            k = (long long)plan.mon_k - a.gk0;
            if (i >= 0 && i < a.gX && j >= 0 && j < a.gY && k >= 0 && k < a.gZ) mon_t_ = (k * a.gY + j) * a.gX + i;
        }
    }
    oplan_ = std::move(plan);
    oroot_ = root;
    writer_ = std::make_unique<fdtd::OutputWriter>();
}

template <typename S, typename T>
void Solver<S, T>::write_population_frame() {
    // PopulationTimeSeriesDetector::write_binary_frame: the full-grid Nu and Ng, FP64, idx3.
    const size_t N = size_t(NxT_) * NyT_ * NzT_;
    const std::string dir = fdtd::run_dir(oplan_, oroot_) + "/populations/";
    for (int w : {int(FDTD_TLS_NU), int(FDTD_TLS_NG)}) {
        auto buf = std::make_shared<std::vector<double>>(N);
        get_tls(w, buf->data());
        fdtd::OutputWriter::Job j;
        j.path = dir + (w == FDTD_TLS_NU ? "populations_Nu.bin" : "populations_Ng.bin");
        j.data = buf->data();
        j.bytes = N * sizeof(double);
        j.append = true;
        j.done = [buf] {};
        writer_->submit(std::move(j));
    }
}

template <typename S, typename T>
void Solver<S, T>::capture_tls(uint64_t s) {
    if (!pop_first_done_) {
        write_population_frame();
        pop_first_done_ = true;
    }
    const int sl = int(tls_count_++ % kTlsSlots);
    {
        std::unique_lock<std::mutex> l(oslot_mu_);
        oslot_cv_.wait(l, [&] { return trec_busy_[sl] == 0; });
        trec_busy_[sl] = 3;
    }
    ck(cudaMemsetAsync(d_trec_ + sl, 0, sizeof(TlsRecord), st_), "cudaMemsetAsync");
    if (has_gain_) {
        const size_t ng = size_t(a_.gX) * a_.gY * a_.gZ;
        const unsigned nb = unsigned(std::max<size_t>(1, std::min<size_t>((ng + 255) / 256, 148 * 4)));
        k_tls_reduce<S, T><<<nb, 256, 0, st_>>>(a_, d_dx_, d_dy_, d_dz_, int((s + 1) & 1), sE_, d_trec_ + sl, mon_t_);
        ++launches;
    }
    ck(cudaMemcpyAsync(h_trec_ + sl, d_trec_ + sl, sizeof(TlsRecord), cudaMemcpyDeviceToHost, st_), "TLS record D2H");
    ck(cudaEventRecord(trec_ev_[sl], st_), "cudaEventRecord");
    const cudaEvent_t ev = trec_ev_[sl];
    const int dev = device;
    const TlsRecord* r = h_trec_ + sl;
    const double dt = dt_;
    const std::string dir = fdtd::run_dir(oplan_, oroot_);
    auto release = [this, sl] {
        {
            std::lock_guard<std::mutex> l(oslot_mu_);
            --trec_busy_[sl];
        }
        oslot_cv_.notify_all();
    };
    fdtd::OutputWriter::Job a, b, c;
    a.wait = [ev, dev] {
        cudaSetDevice(dev);
        if (cudaEventSynchronize(ev) != cudaSuccess) throw std::runtime_error("two-level record copy failed");
    };
    a.text = [r, s, dt] { return fdtd::inversion_line(s, dt, r->acc.int_Nu, r->acc.int_Ng); };
    a.path = dir + "/populations/inversion_time.csv";
    b.text = [r, s, dt] { return fdtd::polarization_line(s, dt, r->P_center, r->dP_dt, r->acc.p_energy); };
    b.path = dir + "/polarization/polarization_time.csv";
    c.text = [r, s, dt] { return fdtd::global_history_line(s, dt, r->acc.int_Nu, r->acc.int_Ng); };
    c.path = dir + "/tls_global_history.csv";
    for (fdtd::OutputWriter::Job* j : {&a, &b, &c}) {
        j->append = true;
        j->done = release;
        writer_->submit(std::move(*j));
    }
}

template <typename S, typename T>
void Solver<S, T>::close_outputs() {
    if (!writer_) return;
    ck(cudaSetDevice(device), "cudaSetDevice");
    if (oplan_.tls) {  // PopulationTimeSeriesDetector::finalize: the last frame and the metadata
        write_population_frame();
        try {
            fdtd::write_population_metadata(oplan_, oroot_);
        } catch (const std::exception& e) {
            throw Failure(FDTD_ERR_IO, e.what());
        }
    }
    flush_outputs();
    writer_.reset();
}

template <typename S, typename T>
void Solver<S, T>::capture_movies() {
    const int sl = int(oframe_ % kOutSlots);
    {
        std::unique_lock<std::mutex> l(oslot_mu_);
        oslot_cv_.wait(l, [&] { return oslot_busy_[sl] == 0; });
        oslot_busy_[sl] = int(oplan_.movies.size());
    }
    for (size_t m = 0; m < oplan_.movies.size(); ++m) {
        const fdtd::MoviePlan& v = oplan_.movies[m];
        const long long count = (long long)(v.dim1 * v.dim2);
        const unsigned nb = unsigned(std::min<long long>((count + 255) / 256, 148 * 4));
        k_slice<S><<<nb, 256, 0, st_>>>(a_.Ex, a_.Ey, a_.Ez, a_.Hx, a_.Hy, a_.Hz, NyT_, NxP_, v.plane, int(v.index),
                                        v.component, (long long)v.dim2, count, sE_, sH_, d_oslot_[sl] + mov_off_[m],
                                        oplan_.float64 ? 1 : 0);
        ++launches;
    }
    ck(cudaMemcpyAsync(h_oslot_[sl], d_oslot_[sl], oslot_bytes_, cudaMemcpyDeviceToHost, st_), "movie frame D2H");
    ck(cudaEventRecord(oslot_ev_[sl], st_), "cudaEventRecord");
    const cudaEvent_t ev = oslot_ev_[sl];
    const int dev = device;
    for (size_t m = 0; m < oplan_.movies.size(); ++m) {
        fdtd::OutputWriter::Job j;
        if (m == 0)
            j.wait = [ev, dev] {
                cudaSetDevice(dev);
                if (cudaEventSynchronize(ev) != cudaSuccess) throw std::runtime_error("movie frame copy failed");
            };
        j.done = [this, sl] {
            {
                std::lock_guard<std::mutex> l(oslot_mu_);
                --oslot_busy_[sl];
            }
            oslot_cv_.notify_all();
        };
        j.path = fdtd::frame_path(oplan_, oroot_, m, oframe_);
        j.data = h_oslot_[sl] + mov_off_[m];
        j.bytes = mov_bytes_[m];
        writer_->submit(std::move(j));
    }
    ++oframe_;
}

template <typename S, typename T>
void Solver<S, T>::write_point_samples() {
    if (oplan_.points.empty() || series_count_ <= ots_written_) return;
    const uint64_t n0 = ots_written_, n = series_count_ - ots_written_;
    std::vector<double> v(size_t(n) * nprobes_);
    ck(cudaMemcpy(v.data(), d_series_ + size_t(n0) * nprobes_, v.size() * sizeof(double), cudaMemcpyDeviceToHost),
       "probe samples D2H");
    const std::string dir = fdtd::run_dir(oplan_, oroot_);
    size_t col = 0;
    for (const auto& p : oplan_.points) {
        for (int c : p.components) {
            auto buf = std::make_shared<std::vector<char>>();
            if (oplan_.float64) {
                buf->resize(n * sizeof(double));
                for (uint64_t t = 0; t < n; ++t) std::memcpy(buf->data() + t * 8, &v[t * nprobes_ + col], 8);
            } else {
                buf->resize(n * sizeof(float));
                for (uint64_t t = 0; t < n; ++t) {
                    const float f = float(v[t * nprobes_ + col]);
                    std::memcpy(buf->data() + t * 4, &f, 4);
                }
            }
            fdtd::OutputWriter::Job j;
            j.path = dir + "/" + p.name + "/" + fdtd::component_name(c) + "_ts.bin";
            j.data = buf->data();
            j.bytes = buf->size();
            j.append = true;
            j.done = [buf] {};
            writer_->submit(std::move(j));
            ++col;
        }
    }
    ots_written_ = series_count_;
}

template <typename S, typename T>
void Solver<S, T>::flush_outputs() {
    if (!writer_) return;
    try {
        writer_->drain();
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_IO, e.what());
    }
}

template <typename S, typename T>
void Solver<S, T>::probe_series(double* out, uint64_t max, uint64_t* n) {
    const uint64_t cnt = std::min<uint64_t>(series_count_, max);
    if (n) *n = series_count_;
    if (cnt && nprobes_ && out)
        ck(cudaMemcpy(out, d_series_, cnt * nprobes_ * sizeof(double), cudaMemcpyDeviceToHost), "series D2H");
}

template <typename S, typename T>
void Solver<S, T>::dft(uint32_t p, double* re, double* im) {
    if (p >= nprobes_ || nf_ == 0) throw Failure(FDTD_ERR_INVALID, "no DFT for this probe");
    std::vector<double> buf(2 * size_t(nf_));
    ck(cudaMemcpy(buf.data(), d_dft_ + 2 * size_t(p) * nf_, buf.size() * sizeof(double), cudaMemcpyDeviceToHost), "dft D2H");
    for (uint32_t m = 0; m < nf_; ++m) { re[m] = buf[2 * m]; im[m] = buf[2 * m + 1]; }
}

template <typename S, typename T>
void Solver<S, T>::diagnostics(fdtd_diagnostics_v1* d) {
    MonitorState ms{};
    ck(cudaMemcpy(&ms, d_ms_, sizeof(ms), cudaMemcpyDeviceToHost), "monitor state");
    std::memset(d, 0, sizeof(*d));
    d->step = ms.step;
    d->steps_done = steps;
    d->max_E = ms.max_E;
    d->max_P = ms.max_P;
    d->conservation_err = ms.cons;
    d->integrated_Nu = ms.int_Nu;
    d->integrated_Ng = ms.int_Ng;
    d->polarization_energy = ms.p_energy;
    d->nan_flags = ms.flags;
    d->instability_count = ms.instability_count;
    d->stable = ms.stable;
}

}  // namespace


namespace {
// ==================================================================== packed multi-solve engine
// A queue of solves (FP32, FP16 or BF16 storage, mixed) served by one GPU: jobs wait until
// their device footprint fits the budget and a slot is free, then stay resident (fields, CPML
// psi, gain state, probes in HBM) until their last step, while every step of every resident
// solve is issued as one packed H launch per storage form, one packed E launch per kind, one
// probe launch and (on monitor steps) one monitor pair.
// The per-cell arithmetic is the single-solve kernels' own, so a solve's result does not
// depend on what it shares the GPU with.
class Batch {
public:
    enum { QUEUED = 0, RESIDENT = 1, DONE = 2, FAILED = 3 };
    // A resident solve: one of the three storage forms (storage = BatchSolve::storage).
    struct Job {
        const fdtd_setup_v1* setup = nullptr;
        uint64_t target = 0;
        int state = QUEUED;
        int storage = 0;
        uint64_t bytes = 0;
        std::unique_ptr<Solver<float, float>> f32;
        std::unique_ptr<Solver<__half, float>> f16;
        std::unique_ptr<Solver<__nv_bfloat16, float>> bf16;
        std::vector<double> series, dft;
        uint64_t samples = 0;
        uint32_t nprobes = 0, nf = 0;
        fdtd_diagnostics_v1 diag{};
        std::string err;
        uint64_t steps() const { return f32 ? f32->steps : f16 ? f16->steps : bf16 ? bf16->steps : 0; }
        bool live() const { return f32 || f16 || bf16; }
        void drop() { f32.reset(); f16.reset(); bf16.reset(); }
    };
    // f(solver) on the job's solver, whatever its storage form.
    template <typename F>
    static void with(Job& j, F&& f) {
        if (j.f32) f(*j.f32);
        else if (j.f16) f(*j.f16);
        else f(*j.bf16);
    }

    Batch(int dev, uint64_t budget) : device_(dev), budget_(budget) {
        ck(cudaSetDevice(dev), "cudaSetDevice");
        claim(dev, true);
        try {
            keep_pool_memory(dev);
            ck(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaHostAlloc(reinterpret_cast<void**>(&ticks_), sizeof(BatchTick) * kMaxBatch * kRing,
                             cudaHostAllocDefault),
               "cudaHostAlloc");
            for (auto& e : ring_ev_) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaHostAlloc(reinterpret_cast<void**>(&h_status_), sizeof(unsigned) * kMaxBatch, cudaHostAllocDefault),
               "cudaHostAlloc");
            ck(cudaMalloc(&d_status_, sizeof(unsigned) * kMaxBatch), "cudaMalloc");
            ck(cudaMalloc(&d_poll_, sizeof(unsigned) * kMaxBatch), "cudaMalloc");
            ck(cudaHostAlloc(reinterpret_cast<void**>(&h_poll_), sizeof(unsigned) * kMaxBatch, cudaHostAllocDefault),
               "cudaHostAlloc");
            ck(cudaEventCreateWithFlags(&poll_ev_, cudaEventDisableTiming), "cudaEventCreate");
            if (const char* e = std::getenv("FDTD_B200_BATCH_H_PIPE")) hpipe_ = std::string(e) != "0";
            if (const char* e = std::getenv("FDTD_B200_BATCH_E_PIPE")) epipe_ = std::string(e) != "0";
            if (const char* e = std::getenv("FDTD_B200_BATCH_KCHUNK")) kchunk_ = std::max(0, std::atoi(e));
            if (const char* e = std::getenv("FDTD_B200_BATCH_SOLO")) solo_ = std::string(e) != "0";
            for (int f = 0; f < kForms; ++f) {
                ck(cudaFuncSetAttribute(hkernel(f, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(hsmem(storage_of(f)))),
                   "cudaFuncSetAttribute");
                for (int sh = 0; sh < 2; ++sh)
                    ck(cudaFuncSetAttribute(ekernel(4 * f + 2 * sh + 1, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(esmem(storage_of(f)))),
                       "cudaFuncSetAttribute");
            }
            worker_ = std::thread([this] { prepare_loop(); });
        } catch (...) {
            release_all();
            throw;
        }
    }
    ~Batch() {
        stop_worker();
        release_all();
    }

    uint64_t submit(const fdtd_setup_v1& s, uint64_t nsteps) {
        int storage = 0;
        if (s.precision == FDTD_PREC_FP32) storage = 0;
        else if (s.precision == FDTD_PREC_FP16) storage = 1;
        else if (s.precision == FDTD_PREC_BF16) storage = 2;
        else throw Failure(FDTD_ERR_UNSUPPORTED, "the packed engine steps FP32, FP16 and BF16 solves");
        if (s.pec_boundary) throw Failure(FDTD_ERR_UNSUPPORTED, "the packed engine steps CPML solves");
        if (nsteps == 0) throw Failure(FDTD_ERR_INVALID, "a job needs at least one step");
        Job j;
        j.setup = &s;
        j.target = nsteps;
        j.storage = storage;
        j.bytes = footprint(s);
        if (j.bytes > budget_) throw Failure(FDTD_ERR_OOM, "job footprint exceeds the batch memory budget");
        std::lock_guard<std::mutex> l(mu_);
        const uint64_t t = next_++;
        jobs_.emplace(t, std::move(j));
        queue_.push_back(t);
        cv_work_.notify_one();
        return t;
    }

    // Splices in the solves the admission worker has made ready, then advances the resident
    // solves by up to max_steps steps each, retiring solves as they reach their target and
    // splicing in newly ready ones at every check.  With nothing resident it first waits for
    // the worker to prepare every job that can be admitted (or returns when there is none).
    void run(uint64_t max_steps) {
        ck(cudaSetDevice(device_), "cudaSetDevice");
        splice(true);
        for (uint64_t t = 0; t < max_steps && !res_.empty();) {
            if (res_.size() == 1 && solo_) {
                // One resident solve (the tail of a stream, or a lone request): step it with the
                // single-solve launches (launch parameters instead of per-block argument records,
                // no packed bookkeeping; measured 13-15 % faster per step than packed alone).  The
                // block code and its explicit rounding are the same, so are the bits.  In chunks,
                // so that arrivals are spliced in and the packed step resumes.
                Job& j = jobs_.at(res_[0]);
                const uint64_t n = std::min<uint64_t>({j.target - j.steps(), max_steps - t, uint64_t(kSoloChunk)});
                ck(cudaStreamSynchronize(st_), "batch solo");  // its packed steps are done
                bool stopped = false;
                with(j, [&](auto& v) {
                    try {
                        v.run(n);
                    } catch (const Failure& f) {
                        if (f.code != FDTD_ERR_UNSTABLE) throw;
                        stopped = true;  // the monitor stopped it: retired as failed below
                    }
                });
                t += n;
                if (stopped || j.steps() >= j.target) {
                    check_and_retire();
                    splice(res_.empty());
                } else {
                    splice(false);
                }
                continue;
            }
            step();
            ++t;
            bool finished = false;
            for (uint64_t r : res_) finished |= jobs_.at(r).steps() >= jobs_.at(r).target;
            if (finished) {
                check_and_retire();
                splice(res_.empty());
            } else if (++since_check_ >= kCheckEvery) {
                poll();
                splice(false);
            }
        }
        ck(cudaStreamSynchronize(st_), "batch run");
    }

    // A finished job's record (DONE or FAILED); the caller reads it without the worker
    // touching it again.
    Job& finished_job(uint64_t t) {
        std::lock_guard<std::mutex> l(mu_);
        Job& j = job_locked(t);
        if (j.state != DONE && j.state != FAILED) throw Failure(FDTD_ERR_INVALID, "job has not finished");
        return j;
    }
    // API state and steps done of any job.
    void state_of(uint64_t t, int* state, uint64_t* steps_done) {
        std::lock_guard<std::mutex> l(mu_);
        Job& j = job_locked(t);
        *state = j.state;
        if (steps_done) *steps_done = j.state == RESIDENT ? j.steps() : j.state == QUEUED ? 0 : j.diag.steps_done;
    }
    void release(uint64_t t) {
        std::lock_guard<std::mutex> l(mu_);
        Job& j = job_locked(t);
        if (j.state != DONE && j.state != FAILED) throw Failure(FDTD_ERR_INVALID, "job has not finished");
        jobs_.erase(t);
    }
    uint32_t resident() const { return uint32_t(res_.size()); }
    uint32_t queued() const {
        std::lock_guard<std::mutex> l(mu_);
        return uint32_t(queue_.size() + preparing_ + ready_.size());
    }

private:
    static constexpr int kRing = 64;        // pinned per-step records in flight
    static constexpr int kCheckEvery = 16;  // steps between status checks
    static constexpr int kSoloChunk = 64;   // steps per single-solve run of a lone resident solve
    // Sweep forms: 0 FP32, 1 FP16, 2 BF16 rounded to nearest, 3 BF16 rounded stochastically (the
    // packed sweeps are compiled per rounding mode, as the single-solve ones).  E kernel kinds:
    // form (4) x plane-wave sheets x indexed material.
    static constexpr int kForms = 4;
    static constexpr int kEKinds = 16;
    static int storage_of(int form) { return form == 3 ? 2 : form; }
    using K = void (*)(const int4*);
    static K hkernel(int form, bool pipe) {
        static constexpr K k[2 * kForms] = {
            k_update_H_multi<float, false, 0>,         k_update_H_multi<float, true, 0>,
            k_update_H_multi<__half, false, 0>,        k_update_H_multi<__half, true, 0>,
            k_update_H_multi<__nv_bfloat16, false, 0>, k_update_H_multi<__nv_bfloat16, true, 0>,
            k_update_H_multi<__nv_bfloat16, false, 1>, k_update_H_multi<__nv_bfloat16, true, 1>};
        return k[2 * form + int(pipe)];
    }
    // dynamic shared memory of the staged sweeps of storage form st (0 FP32, 1 FP16, 2 BF16)
    static size_t hsmem(int st) { return st == 0 ? HPipe<float>::bytes() : st == 1 ? HPipe<__half>::bytes() : HPipe<__nv_bfloat16>::bytes(); }
    static size_t esmem(int st) { return st == 0 ? EPipe<float>::bytes() : st == 1 ? EPipe<__half>::bytes() : EPipe<__nv_bfloat16>::bytes(); }
    // kind = 4 form + 2 SH + MAT; the staged form exists for the indexed material only
    static K ekernel(int kind, bool pipe) {
        static constexpr K k[kEKinds] = {
            k_update_E_multi<float, false, false, false, 0>,         k_update_E_multi<float, false, true, false, 0>,
            k_update_E_multi<float, true, false, false, 0>,          k_update_E_multi<float, true, true, false, 0>,
            k_update_E_multi<__half, false, false, false, 0>,        k_update_E_multi<__half, false, true, false, 0>,
            k_update_E_multi<__half, true, false, false, 0>,         k_update_E_multi<__half, true, true, false, 0>,
            k_update_E_multi<__nv_bfloat16, false, false, false, 0>, k_update_E_multi<__nv_bfloat16, false, true, false, 0>,
            k_update_E_multi<__nv_bfloat16, true, false, false, 0>,  k_update_E_multi<__nv_bfloat16, true, true, false, 0>,
            k_update_E_multi<__nv_bfloat16, false, false, false, 1>, k_update_E_multi<__nv_bfloat16, false, true, false, 1>,
            k_update_E_multi<__nv_bfloat16, true, false, false, 1>,  k_update_E_multi<__nv_bfloat16, true, true, false, 1>};
        static constexpr K kp[kEKinds] = {
            nullptr, k_update_E_multi<float, false, true, true, 0>,         nullptr, k_update_E_multi<float, true, true, true, 0>,
            nullptr, k_update_E_multi<__half, false, true, true, 0>,        nullptr, k_update_E_multi<__half, true, true, true, 0>,
            nullptr, k_update_E_multi<__nv_bfloat16, false, true, true, 0>, nullptr, k_update_E_multi<__nv_bfloat16, true, true, true, 0>,
            nullptr, k_update_E_multi<__nv_bfloat16, false, true, true, 1>, nullptr, k_update_E_multi<__nv_bfloat16, true, true, true, 1>};
        return pipe && kp[kind] ? kp[kind] : k[kind];
    }

    // The per-solve records live in the module's constant memory, one set per device: a
    // second engine on the same device would overwrite the first one's, so it is refused.
    static void claim(int dev, bool take) {
        static std::mutex mu;
        static std::vector<int> owned;
        std::lock_guard<std::mutex> l(mu);
        auto it = std::find(owned.begin(), owned.end(), dev);
        if (!take) {
            if (it != owned.end()) owned.erase(it);
            return;
        }
        if (it != owned.end())
            throw Failure(FDTD_ERR_INVALID, "device " + std::to_string(dev) + " already has a packed engine in this process");
        owned.push_back(dev);
    }
    Job& job_locked(uint64_t t) {
        auto it = jobs_.find(t);
        if (it == jobs_.end()) throw Failure(FDTD_ERR_INVALID, "unknown ticket");
        return it->second;
    }
    void stop_worker() {
        {
            std::lock_guard<std::mutex> l(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        if (worker_.joinable()) worker_.join();
    }
    void release_all() {
        cudaSetDevice(device_);
        if (st_) cudaStreamSynchronize(st_);
        jobs_.clear();
        if (d_tab_) cudaFree(d_tab_);
        if (ticks_) cudaFreeHost(ticks_);
        if (d_status_) cudaFree(d_status_);
        if (h_status_) cudaFreeHost(h_status_);
        d_status_ = nullptr; h_status_ = nullptr;
        if (d_poll_) cudaFree(d_poll_);
        if (h_poll_) cudaFreeHost(h_poll_);
        if (poll_ev_) cudaEventDestroy(poll_ev_);
        d_poll_ = nullptr; h_poll_ = nullptr; poll_ev_ = nullptr;
        for (auto& e : ring_ev_) if (e) cudaEventDestroy(e);
        if (st_) cudaStreamDestroy(st_);
        d_tab_ = nullptr; ticks_ = nullptr; st_ = nullptr;
        for (auto& e : ring_ev_) e = nullptr;
        claim(device_, false);
    }

    // Device bytes a solve will hold: fields, bE, psi slabs, gain box (upper bound; the FP32
    // figure bounds the 16-bit forms too).
    static uint64_t footprint(const fdtd_setup_v1& s) {
        const uint64_t NxP = (s.NxT + 31) / 32 * 32, NyT = s.NyT, NzT = s.NzT, np2 = 2ull * s.npml;
        uint64_t b = 9ull * NxP * NyT * NzT * 4;
        b += 2ull * 4 * (NzT * NyT * np2 + NzT * np2 * NxP + np2 * NyT * NxP) * 3;  // 12 psi arrays
        if (s.n_tls_regions) b += 17ull * s.NxT * NyT * NzT / 4;  // gain box, worst case the grid
        return b + (64ull << 10) + 3ull * (s.NxT + NyT + NzT) * 8 * 8;
    }

    // Admission worker: takes queued jobs first come, first served while their footprint fits
    // the budget (counting resident, ready and in-preparation solves) and fewer than kMaxBatch
    // are resident or on the way, and builds each one's Solver -- device allocation, set-up
    // uploads, its probe series buffer -- on the solve's own stream, while the stepping thread
    // keeps launching packed steps.  Ready solves wait in ready_ until the stepping thread
    // splices them in (splice), so admission never stalls the packed step.
    void prepare_loop() {
        std::unique_lock<std::mutex> l(mu_);
        for (;;) {
            cv_work_.wait(l, [&] {
                if (stop_) return true;
                if (queue_.empty()) return false;
                const Job& j = jobs_.at(queue_.front());
                return used_ + j.bytes <= budget_ && nres_ + preparing_ + ready_.size() < size_t(kMaxBatch);
            });
            if (stop_) return;
            const uint64_t t = queue_.front();
            queue_.pop_front();
            Job& j = jobs_.at(t);
            used_ += j.bytes;
            ++preparing_;
            l.unlock();
            std::string err;
            try {
                if (j.storage == 0) j.f32 = std::make_unique<Solver<float, float>>(*j.setup, device_, nullptr, true);
                else if (j.storage == 1) j.f16 = std::make_unique<Solver<__half, float>>(*j.setup, device_, nullptr, true);
                else j.bf16 = std::make_unique<Solver<__nv_bfloat16, float>>(*j.setup, device_, nullptr, true);
                with(j, [&](auto& v) {
                    v.ensure_series((j.target + v.save_every_ - 1) / v.save_every_);
                    ck(cudaStreamSynchronize(v.st_), "admit");
                });
            } catch (const std::exception& e) {
                err = e.what();
                j.drop();
            }
            l.lock();
            --preparing_;
            if (err.empty()) {
                ready_.push_back(t);
            } else {
                j.state = FAILED;
                j.err = err;
                used_ -= j.bytes;
            }
            cv_ready_.notify_all();
        }
    }

    // Moves the ready solves into the resident set (admission order) and rebuilds the packed
    // tables.  wait (nothing resident, so the GPU is idle): first wait until the worker has
    // prepared every job that can be admitted now, so a batch starts with all that fit.
    void splice(bool wait) {
        std::vector<uint64_t> add;
        {
            std::unique_lock<std::mutex> l(mu_);
            auto admissible = [&] {
                return !queue_.empty() && used_ + jobs_.at(queue_.front()).bytes <= budget_ &&
                       nres_ + preparing_ + ready_.size() < size_t(kMaxBatch);
            };
            if (wait) cv_ready_.wait(l, [&] { return stop_ || (preparing_ == 0 && !admissible()); });
            add.swap(ready_);
            for (uint64_t t : add) jobs_.at(t).state = RESIDENT;
            nres_ = res_.size() + add.size();
        }
        if (add.empty()) return;
        res_.insert(res_.end(), add.begin(), add.end());
        rebuild();
    }

    // Per-solve constants and the packed block tables.
    void rebuild() {
        const int n = int(res_.size());
        std::vector<BatchArgs> args(n);
        std::vector<BatchSolve> bs(n);
        std::vector<int4> tab;
        std::vector<int> ekind(n), form(n);
        for (int r = 0; r < n; ++r) {
            Job& j = jobs_.at(res_[r]);
            BatchSolve& b = bs[r];
            std::memset(&args[r], 0, sizeof(BatchArgs));
            if (j.f32) args[r].f32 = j.f32->a_;
            else if (j.f16) args[r].f16 = j.f16->a_;
            else args[r].bf16 = j.bf16->a_;
            with(j, [&](auto& v) {
                b.g = v.geom_;
                b.kchunkH = kchunk_ ? kchunk_ : v.kchunkH_;
                b.kchunkE = kchunk_ ? kchunk_ : v.kchunkE_;
                b.probes = v.d_probes_;
                b.nprobes = int(v.nprobes_);
                b.nf = int(v.nf_);
                b.freqs = v.d_freqs_;
                b.dft = v.d_dft_;
                b.series = v.d_series_;
                b.dx = v.d_dx_; b.dy = v.d_dy_; b.dz = v.d_dz_;
                b.acc = v.d_acc_;
                b.ms = v.d_ms_;
                b.status = v.d_status_;
                b.nflat = v.nflat_;
                b.dt = v.dt_;
                b.sE = v.sE_;
                b.sH = v.sH_;
                b.storage = j.storage;
                form[r] = j.storage == 2 && v.a_.sr ? 3 : j.storage;
                ekind[r] = 4 * form[r] + 2 * int(!v.sheets_.empty()) + int(v.a_.bidx != nullptr);
            });
        }
        // the solve's launch shape with z-chunks of kc planes over planes [0, k1)
        auto zchunks = [](dim3 g, int k1, int kc) { return dim3(g.x, g.y, unsigned(std::max(1, (k1 + kc - 1) / kc))); };
        auto add_blocks = [&](int r, dim3 g) {
            for (unsigned z = 0; z < g.z; ++z)
                for (unsigned y = 0; y < g.y; ++y)
                    for (unsigned x = 0; x < g.x; ++x) tab.push_back(make_int4(r, int(x), int(y), int(z)));
        };
        nHk_[0] = 0;
        for (int f = 0; f < kForms; ++f) {  // H blocks by sweep form, then E blocks by kind
            for (int r = 0; r < n; ++r) {
                Job& j = jobs_.at(res_[r]);
                if (form[r] == f) with(j, [&](auto& v) { add_blocks(r, zchunks(v.gridH_, v.a_.kH1, bs[r].kchunkH)); });
            }
            nHk_[f + 1] = tab.size();
        }
        nH_ = tab.size();
        nEk_[0] = 0;
        for (int kind = 0; kind < kEKinds; ++kind) {
            for (int r = 0; r < n; ++r)
                if (ekind[r] == kind)
                    with(jobs_.at(res_[r]), [&](auto& v) { add_blocks(r, zchunks(v.gridE_, v.a_.kE1, bs[r].kchunkE)); });
            nEk_[kind + 1] = tab.size() - nH_;
        }
        ck(cudaStreamSynchronize(st_), "rebuild");  // no step may read the old tables
        if (tab.size() > tab_cap_) {
            if (d_tab_) ck(cudaFree(d_tab_), "cudaFree");
            d_tab_ = nullptr;
            tab_cap_ = std::max<size_t>(tab.size(), 2 * tab_cap_);
            ck(cudaMalloc(&d_tab_, tab_cap_ * sizeof(int4)), "cudaMalloc block table");
        }
        if (!tab.empty()) ck(cudaMemcpy(d_tab_, tab.data(), tab.size() * sizeof(int4), cudaMemcpyHostToDevice), "block table");
        if (n) {
            ck(cudaMemcpyToSymbol(c_bargs, args.data(), n * sizeof(BatchArgs)), "cudaMemcpyToSymbol");
            ck(cudaMemcpyToSymbol(c_bsolve, bs.data(), n * sizeof(BatchSolve)), "cudaMemcpyToSymbol");
        }
    }

    void step() {
        const int n = int(res_.size());
        const int slot = ring_++ % kRing;
        ck(cudaEventSynchronize(ring_ev_[slot]), "tick ring");  // its previous copy has been read
        BatchTick* tk = ticks_ + size_t(slot) * kMaxBatch;
        bool monitor = false;
        for (int r = 0; r < n; ++r) {
            with(jobs_.at(res_[r]), [&](auto& v) {
                const uint64_t s = v.steps;
                BatchTick& k = tk[r];
                k = BatchTick{};
                v.src_static(k.src);
                v.src_step(k.src, s);
                k.sample = (s % v.save_every_ == 0) ? (long long)(s / v.save_every_) : -1;
                if (k.sample >= 0) v.series_count_ = uint64_t(k.sample) + 1;
                k.t = double(s + 1) * v.dt_;
                k.step = s;
                k.monitor = (v.interval_ && s % v.interval_ == 0) ? 1 : 0;
                monitor |= k.monitor != 0;
                v.steps = s + 1;
            });
        }
        ck(cudaMemcpyToSymbolAsync(c_btick, tk, n * sizeof(BatchTick), 0, cudaMemcpyHostToDevice, st_), "step records");
        ck(cudaEventRecord(ring_ev_[slot], st_), "cudaEventRecord");
        const dim3 blk(32, kBlockY);
        for (int q = 0; q < kForms; ++q)
            if (nHk_[q + 1] > nHk_[q]) {
                const bool pipe = hpipe_ && q != 0;
                hkernel(q, pipe)<<<unsigned(nHk_[q + 1] - nHk_[q]), blk, pipe ? hsmem(storage_of(q)) : 0, st_>>>(
                    d_tab_ + nHk_[q]);
            }
        for (int q = 0; q < kEKinds; ++q)
            if (nEk_[q + 1] > nEk_[q]) {
                const bool pipe = epipe_ && (q & 1);
                ekernel(q, pipe)<<<unsigned(nEk_[q + 1] - nEk_[q]), blk, pipe ? esmem(storage_of(q / 4)) : 0, st_>>>(
                    d_tab_ + nH_ + nEk_[q]);
            }
        k_probe_multi<<<n, 128, 0, st_>>>();
        if (monitor) {
            k_monitor_reduce_multi<<<n * kMonBlocks, 256, 0, st_>>>();
            k_monitor_eval_multi<<<1, kMaxBatch, 0, st_>>>(n);
        }
        ck(cudaGetLastError(), "packed step");
    }

    // Reads every resident solve's status word; retires finished and failed solves.
    // Periodic status check that does not drain the stream: the resident solves' status words
    // are gathered and copied to the host behind the queued steps, and read at the next poll
    // once that copy has landed.  A stopped solve (rare) is then retired by the synchronous
    // check.  Finished solves are known on the host from their step counts.
    void poll() {
        since_check_ = 0;
        if (poll_pending_) {
            const cudaError_t q = cudaEventQuery(poll_ev_);
            if (q == cudaErrorNotReady) return;  // still behind queued work: look next time
            ck(q, "status poll");
            poll_pending_ = false;
            bool stopped = false;
            for (int r = 0; r < poll_n_; ++r) stopped |= h_poll_[r] != 0;
            if (stopped) {
                check_and_retire();
                return;
            }
        }
        const int n = int(res_.size());
        if (!n) return;
        k_status_multi<<<1, kMaxBatch, 0, st_>>>(n, d_poll_);
        ck(cudaGetLastError(), "k_status_multi");
        ck(cudaMemcpyAsync(h_poll_, d_poll_, n * sizeof(unsigned), cudaMemcpyDeviceToHost, st_), "status poll");
        ck(cudaEventRecord(poll_ev_, st_), "cudaEventRecord");
        poll_pending_ = true;
        poll_n_ = n;
    }

    void check_and_retire() {
        since_check_ = 0;
        poll_pending_ = false;  // the synchronous check below sees every status
        const int n = int(res_.size());
        if (n) {
            k_status_multi<<<1, kMaxBatch, 0, st_>>>(n, d_status_);
            ck(cudaGetLastError(), "k_status_multi");
            ck(cudaMemcpyAsync(h_status_, d_status_, n * sizeof(unsigned), cudaMemcpyDeviceToHost, st_), "status");
        }
        ck(cudaStreamSynchronize(st_), "batch check");
        std::vector<uint64_t> keep;
        for (int r = 0; r < n; ++r) {
            const uint64_t t = res_[r];
            Job& j = jobs_.at(t);
            bool stay = false;
            with(j, [&](auto& v) {
                const unsigned status = h_status_[r];
                if (status == 0 && v.steps < j.target) { stay = true; return; }
                if (status) {
                    MonitorState ms{};
                    ck(cudaMemcpy(&ms, v.d_ms_, sizeof(ms), cudaMemcpyDeviceToHost), "monitor state");
                    j.err = "stability monitor stopped the solve at step " + std::to_string(ms.step);
                    v.steps = ms.step + 1;
                    v.series_count_ = std::min<uint64_t>(v.series_count_, (v.steps + v.save_every_ - 1) / v.save_every_);
                }
                j.nprobes = v.nprobes_;
                j.nf = v.nf_;
                j.series.assign(size_t(v.series_count_) * v.nprobes_, 0.0);
                uint64_t got = 0;
                if (v.nprobes_) v.probe_series(j.series.data(), v.series_count_, &got);
                j.samples = got;
                j.dft.assign(size_t(2) * v.nprobes_ * v.nf_, 0.0);
                if (v.nprobes_ && v.nf_)
                    ck(cudaMemcpy(j.dft.data(), v.d_dft_, j.dft.size() * sizeof(double), cudaMemcpyDeviceToHost), "dft");
                v.diagnostics(&j.diag);
            });
            if (stay) { keep.push_back(t); continue; }
            j.drop();
            std::lock_guard<std::mutex> l(mu_);
            j.state = h_status_[r] ? FAILED : DONE;
            j.setup = nullptr;
            used_ -= j.bytes;
        }
        const bool changed = keep.size() != res_.size();
        res_.swap(keep);
        {
            std::lock_guard<std::mutex> l(mu_);
            nres_ = res_.size();
        }
        cv_work_.notify_one();  // retired footprint and slots free up
        if (changed) rebuild();
    }

    int device_;
    uint64_t budget_, used_ = 0, next_ = 1;  // used_: resident, ready and in-preparation footprints
    cudaStream_t st_ = nullptr;
    // mu_ guards jobs_' structure, queue_, ready_, preparing_, nres_, used_ and the job states;
    // a job's Solver belongs to the worker while it is being prepared and to the stepping
    // thread from the splice on.
    mutable std::mutex mu_;
    std::condition_variable cv_work_, cv_ready_;
    std::thread worker_;
    bool stop_ = false;
    size_t preparing_ = 0, nres_ = 0;
    std::vector<uint64_t> ready_;
    std::map<uint64_t, Job> jobs_;
    std::deque<uint64_t> queue_;
    std::vector<uint64_t> res_;  // resident tickets in slot order
    int4* d_tab_ = nullptr;
    size_t tab_cap_ = 0, nH_ = 0;
    size_t nHk_[kForms + 1] = {};  // H blocks of sweep form q are table entries [nHk_[q], nHk_[q + 1])
    size_t nEk_[kEKinds + 1] = {};  // E blocks of kind q are entries [nEk_[q], nEk_[q + 1]) after the H ones
    BatchTick* ticks_ = nullptr;
    cudaEvent_t ring_ev_[kRing] = {};
    uint64_t ring_ = 0;
    int since_check_ = 0;
    unsigned* d_status_ = nullptr;  // gathered status words
    unsigned* d_poll_ = nullptr;    // the same, for the non-blocking poll
    unsigned* h_poll_ = nullptr;
    cudaEvent_t poll_ev_ = nullptr;
    bool poll_pending_ = false;
    int poll_n_ = 0;
    unsigned* h_status_ = nullptr;
    // Launch shape: staged sweeps (the E sweep for every storage form, the H sweep for 16-bit
    // storage, as for a single solve: staging the FP32 H sweep costs 4 %) and each solve's own
    // z-chunks (at most 16 planes, shorter on small grids so that a lone solve still fills the
    // GPU; 16-plane chunks for every solve had measured 1.19 -> 1.12 ms per packed step of 64
    // BF16 cavities of 96x96x64 against each solve's chunks of the time, which were up to 64
    // planes).  FDTD_B200_BATCH_KCHUNK (planes, 0 = each solve's own) / _H_PIPE / _E_PIPE
    // override them.
    bool hpipe_ = true, epipe_ = true;
    int kchunk_ = 0;
    // A lone resident solve steps with the single-solve launches (FDTD_B200_BATCH_SOLO=0: packed).
    bool solo_ = true;
};

// ==================================================================== sharded solve
// One solve split into z slabs, one Solver per shard (on one device or several).  A shard's
// grid is its owned planes plus one halo plane on each side that has a neighbour; every step
// the neighbours exchange one plane of E (Ex, Ey: the H sweep reads E at k+1) and one plane of
// H (Hx, Hy: the E sweep reads H at k-1), as device-to-device (peer) copies ordered by events
// between the shards' streams; no kernel waits on another GPU.  The kernels take the shard's
// global z offset for the z CPML and the global plane ranges they update, so a sharded solve
// computes the same values, cell for cell, as the whole solve.  The stability monitor reduces
// each shard's owned planes and is evaluated once, on shard 0, which then hands its status
// word to the others.  Kernel path 1 only, CPML or PEC boundary, no detector files.
template <typename S, typename T>
class Sharded final : public SolverBase {
public:
    Sharded(const fdtd_setup_v1& s, int n, const int* devices);
    ~Sharded() override;
    void run(uint64_t n) override;
    void set_field(int comp, const double* h) override { scatter(h, [&](Solver<S, T>& p, const double* l) { p.set_field(comp, l); }); }
    void get_field(int comp, double* h) override { gather(h, [&](Solver<S, T>& p, double* l) { p.get_field(comp, l); }); }
    void set_tls(int which, const double* h) override { scatter(h, [&](Solver<S, T>& p, const double* l) { p.set_tls(which, l); }); }
    void get_tls(int which, double* h) override {
        // the P slots by parity of the shard's own step count, which run() keeps in step
        gather(h, [&](Solver<S, T>& p, double* l) { p.get_tls(which, l); });
    }
    void probe_series(double* out, uint64_t max, uint64_t* n) override;
    void dft(uint32_t p, double* re, double* im) override;
    void diagnostics(fdtd_diagnostics_v1* d) override {
        part_[0]->diagnostics(d);
        d->steps_done = steps;
    }
    void sync() override {
        for (auto& p : part_) p->sync();
    }
    // FDTD_TIMING_RUN: one event pair per run() on shard 0's stream, the other shards' work
    // fenced between them; per-kernel timing is a whole solve's mode.
    void set_timing(int mode) override {
        if (mode == FDTD_TIMING_KERNELS) throw Failure(FDTD_ERR_UNSUPPORTED, "a sharded solve times whole runs only");
        if (mode != FDTD_TIMING_OFF && mode != FDTD_TIMING_RUN) throw Failure(FDTD_ERR_INVALID, "bad timing mode");
        timing_ = mode;
        run_ms_ = 0;
        tsteps_ = 0;
        if (mode == FDTD_TIMING_RUN && !tev_[0]) {
            ck(cudaSetDevice(part_[0]->device), "cudaSetDevice");
            for (auto& e : tev_) ck(cudaEventCreate(&e), "cudaEventCreate");
        }
    }
    void set_path(int path) override {
        if (path != 1) throw Failure(FDTD_ERR_UNSUPPORTED, "a sharded solve steps with kernel path 1");
    }
    void timing(fdtd_timing_v1* t) override {
        std::memset(t, 0, sizeof(*t));
        t->steps = tsteps_;
        t->run_ms = run_ms_;
    }
    void attach_outputs(const fdtd::SimSetup& setup, const std::string& root) override;
    void flush_outputs() override;
    void close_outputs() override;

private:
    // A shard's slice of the setup view: the arrays it needs, copied out of the whole view.
    struct Slice {
        fdtd_setup_v1 v{};
        std::vector<double> dz, inv_dz, kz[5], bE[3], freqs;
        std::unique_ptr<double[]> Nu, Ng;  // valid in the gain cells' columns only
        std::vector<uint16_t> bidx;
        std::vector<int32_t> reg;
        std::vector<fdtd_dipole_v1> dip;
        std::vector<fdtd_probe_v1> probes;
        std::vector<fdtd_sheet_v1> sheets;
    };
    template <typename F> void scatter(const double* h, F&& f);
    template <typename F> void gather(double* h, F&& f);
    void copy_planes(int dst, int dst_plane, int src, int src_plane, int c0, int c1);

    std::vector<std::unique_ptr<Slice>> slice_;
    std::vector<std::unique_ptr<Solver<S, T>>> part_;
    std::vector<int> z0_, z1_, lo_;   // owned global planes [z0, z1); local plane 0 is global lo
    std::vector<std::pair<int, int>> probe_at_;  // global probe -> (shard, local probe)
    uint64_t NxT_, NyT_, NzT_;
    uint32_t interval_ = 0;
    std::vector<cudaEvent_t> evE_, evH_, evCpE_, evCpH_, evMon_;
    DiagAccum* d_parts_ = nullptr;  // shard 0's device: the other shards' accumulators
    int timing_ = FDTD_TIMING_OFF;
    cudaEvent_t tev_[2] = {};
    double run_ms_ = 0;
    uint64_t tsteps_ = 0;

    // Detector files (fdtd_attach_outputs): the whole solve's plan and one writer thread.  At a
    // save step every shard captures, on its own stream, the part of each movie slice that lies
    // in the planes it holds and its two-level sums; the writer joins the parts once every
    // shard's copy has completed.  A ring slot is reused after the writer is done with it.
    static constexpr int kOutSlots = 4, kTlsSlots = 16;
    static constexpr size_t kNoPart = ~size_t(0);
    struct OutPart {
        std::vector<size_t> off;    // per movie: byte offset of this shard's part in a slot, or kNoPart
        std::vector<int> index;     // per movie: the slice index in the shard's local grid
        std::vector<long long> d2;  // per movie: the part's second dimension
        size_t slot_bytes = 0;
        char* d_slot[kOutSlots] = {};
        char* h_slot[kOutSlots] = {};
        cudaEvent_t ev[kOutSlots] = {};
        TlsRecord* d_trec = nullptr;
        TlsRecord* h_trec = nullptr;
        cudaEvent_t trec_ev[kTlsSlots] = {};
        long long mon_t = -1;  // the PolarizationDiagnostics cell in this shard's gain box, or -1
    };
    std::unique_ptr<fdtd::OutputWriter> writer_;
    fdtd::OutputPlan oplan_;
    std::string oroot_;
    std::vector<OutPart> out_;
    std::mutex oslot_mu_;
    std::condition_variable oslot_cv_;
    int oslot_busy_[kOutSlots] = {}, trec_busy_[kTlsSlots] = {};
    uint64_t oframe_ = 0, tls_count_ = 0, ots_written_ = 0;
    bool pop_first_done_ = false;
    void capture_movies();
    void capture_tls(uint64_t s);
    void write_point_samples();
    void write_population_frame();
    void free_outputs();
};

template <typename S, typename T>
Sharded<S, T>::Sharded(const fdtd_setup_v1& s, int n, const int* devices) {
    NxT_ = s.NxT; NyT_ = s.NyT; NzT_ = s.NzT;
    if (n < 2) throw Failure(FDTD_ERR_INVALID, "a sharded solve needs at least 2 shards");
    for (int c = 0; c < 3; ++c)
        if (s.aE[c] || s.aH[c] || s.bH[c])
            throw Failure(FDTD_ERR_UNSUPPORTED, "a sharded solve takes uniform aE/aH/bH (passed as NULL)");
    if (int64_t(NzT_) < 3 * n) throw Failure(FDTD_ERR_INVALID, "fewer than 3 z planes per shard");
    const size_t N = NxT_ * NyT_ * NzT_;
    device = devices ? devices[0] : 0;
    const bool fp16 = std::is_same_v<S, __half>;
    const double sE = field_scale_of(s, fp16);  // one scale for all shards
    // and one psi scale (16-bit storage): the smallest cell edge of the whole grid
    double psi_dx = *std::min_element(s.dx, s.dx + NxT_);
    psi_dx = std::min(psi_dx, *std::min_element(s.dy, s.dy + NyT_));
    psi_dx = std::min(psi_dx, *std::min_element(s.dz, s.dz + NzT_));
    interval_ = s.monitor_interval;
    probe_at_.assign(s.n_probes, {-1, -1});
    for (int r = 0; r < n; ++r) {
        const int z0 = int(NzT_ * uint64_t(r) / uint64_t(n)), z1 = int(NzT_ * uint64_t(r + 1) / uint64_t(n));
        const int lo = std::max(0, z0 - 1), hi = std::min(int(NzT_), z1 + 1), nz = hi - lo;
        z0_.push_back(z0); z1_.push_back(z1); lo_.push_back(lo);
        auto sl = std::make_unique<Slice>();
        fdtd_setup_v1& v = sl->v;
        v = s;
        v.NzT = uint64_t(nz);
        v.field_scale = sE;
        auto cut1 = [&](const double* a, std::vector<double>& out) -> const double* {
            if (!a) return nullptr;
            out.assign(a + lo, a + hi);
            return out.data();
        };
        auto cut3 = [&](auto* a, auto& out) {
            using E = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
            if (!a) return (const E*)nullptr;
            out.resize(NxT_ * NyT_ * size_t(nz));
#pragma omp parallel for schedule(static)
            for (long long ij = 0; ij < (long long)(NxT_ * NyT_); ++ij)
                std::memcpy(out.data() + size_t(ij) * nz, a + size_t(ij) * NzT_ + lo, size_t(nz) * sizeof(E));
            return (const E*)out.data();
        };
        v.dz = cut1(s.dz, sl->dz);
        v.inv_dz = cut1(s.inv_dz, sl->inv_dz);
        v.cpml_kappa[2] = cut1(s.cpml_kappa[2], sl->kz[0]);
        v.cpml_bE[2] = cut1(s.cpml_bE[2], sl->kz[1]);
        v.cpml_cE[2] = cut1(s.cpml_cE[2], sl->kz[2]);
        v.cpml_bH[2] = cut1(s.cpml_bH[2], sl->kz[3]);
        v.cpml_cH[2] = cut1(s.cpml_cH[2], sl->kz[4]);
        const char* mi = std::getenv("FDTD_B200_MATERIAL_INDEX");
        const bool use_index = s.bE_index && s.n_bE_rows && !(mi && std::string(mi) == "0");
        if (use_index) {  // the shard reads the row index; the arrays are not copied
            v.bE_index = cut3(s.bE_index, sl->bidx);
            for (int c = 0; c < 3; ++c) v.bE[c] = nullptr;
        } else {
            v.bE_index = nullptr;
            v.n_bE_rows = 0;
            for (int c = 0; c < 3; ++c) v.bE[c] = cut3(s.bE[c], sl->bE[c]);
        }
        if (s.tls_region_map) {
            v.tls_region_map = cut3(s.tls_region_map, sl->reg);
            // gain cells only where this shard updates E: none in the halo planes
            for (size_t ij = 0; ij < NxT_ * NyT_; ++ij)
                for (int k = 0; k < nz; ++k)
                    if (lo + k < z0 || lo + k >= z1) sl->reg[ij * nz + k] = -1;
        }
        // initial Nu, Ng: the stepper reads them at gain cells only, so only the (i, j) columns
        // that hold one are copied (the rest of the buffer is never read)
        v.tls_Nu = v.tls_Ng = nullptr;
        if (s.tls_Nu || s.tls_Ng) {
            const size_t nl = NxT_ * NyT_ * size_t(nz);
            if (s.tls_Nu) sl->Nu.reset(new double[nl]);
            if (s.tls_Ng) sl->Ng.reset(new double[nl]);
#pragma omp parallel for schedule(static)
            for (long long ij = 0; ij < (long long)(NxT_ * NyT_); ++ij) {
                bool any = false;
                for (int k = 0; k < nz && v.tls_region_map; ++k) any |= sl->reg[size_t(ij) * nz + k] >= 0;
                if (!any) continue;
                if (s.tls_Nu) std::memcpy(sl->Nu.get() + size_t(ij) * nz, s.tls_Nu + size_t(ij) * NzT_ + lo, size_t(nz) * 8);
                if (s.tls_Ng) std::memcpy(sl->Ng.get() + size_t(ij) * nz, s.tls_Ng + size_t(ij) * NzT_ + lo, size_t(nz) * 8);
            }
            v.tls_Nu = sl->Nu.get();
            v.tls_Ng = sl->Ng.get();
        }
        for (uint32_t q = 0; q < s.n_dipoles; ++q) {
            fdtd_dipole_v1 d = s.dipoles[q];
            if (int(d.k) < z0 || int(d.k) >= z1) continue;
            d.k -= uint64_t(lo);
            sl->dip.push_back(d);
        }
        v.n_dipoles = uint32_t(sl->dip.size());
        v.dipoles = sl->dip.data();
        for (uint32_t q = 0; q < s.n_sheets; ++q) {
            fdtd_sheet_v1 w = s.sheets[q];
            if (w.axis == 2) {
                if (int(w.plane) < z0 || int(w.plane) >= z1) continue;
                w.plane -= uint64_t(lo);
            } else {  // z is the second in-plane axis
                const int a = std::max(int(w.lo1), z0), b = std::min(int(w.hi1), z1 - 1);
                if (a > b) continue;
                w.lo1 = uint64_t(a - lo);
                w.hi1 = uint64_t(b - lo);
            }
            sl->sheets.push_back(w);
        }
        v.n_sheets = uint32_t(sl->sheets.size());
        v.sheets = sl->sheets.data();
        for (uint32_t q = 0; q < s.n_probes; ++q) {
            fdtd_probe_v1 pr = s.probes[q];
            if (int(pr.k) < z0 || int(pr.k) >= z1) continue;
            probe_at_[q] = {r, int(sl->probes.size())};
            pr.k -= uint64_t(lo);
            sl->probes.push_back(pr);
        }
        v.n_probes = uint32_t(sl->probes.size());
        v.probes = sl->probes.data();
        ShardSpec spec{lo, int(NzT_), z0 - lo, z1 - lo, psi_dx};
        part_.push_back(std::make_unique<Solver<S, T>>(v, devices ? devices[r] : 0, &spec));
        slice_.push_back(std::move(sl));
    }
    (void)N;
    // the monitor is evaluated on shard 0 for the whole solve
    bool gain = false;
    for (auto& p : part_) gain |= p->has_gain_;
    {
        Solver<S, T>& p0 = *part_[0];
        ck(cudaSetDevice(p0.device), "cudaSetDevice");
        MonitorState ms{};
        ck(cudaMemcpy(&ms, p0.d_ms_, sizeof(ms), cudaMemcpyDeviceToHost), "monitor state");
        ms.has_gain = gain ? 1 : 0;
        ck(cudaMemcpy(p0.d_ms_, &ms, sizeof(ms), cudaMemcpyHostToDevice), "monitor state");
        ck(cudaMalloc(&d_parts_, std::max<size_t>(1, part_.size()) * sizeof(DiagAccum)), "cudaMalloc");
    }
    for (auto* evs : {&evE_, &evH_, &evCpE_, &evCpH_, &evMon_}) {
        evs->resize(part_.size());
        for (size_t r = 0; r < part_.size(); ++r) {
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            ck(cudaEventCreateWithFlags(&(*evs)[r], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
    for (auto& p : part_) dev_bytes += p->dev_bytes;
    material_rows = part_[0]->material_rows;
    // neighbours on different GPUs copy their halo planes directly over NVLink
    for (size_t r = 0; r + 1 < part_.size(); ++r) {
        const int a = part_[r]->device, b = part_[r + 1]->device;
        if (a == b) continue;
        for (auto [x, y] : {std::pair<int, int>{a, b}, std::pair<int, int>{b, a}}) {
            int can = 0;
            ck(cudaDeviceCanAccessPeer(&can, x, y), "cudaDeviceCanAccessPeer");
            if (!can) continue;
            ck(cudaSetDevice(x), "cudaSetDevice");
            const cudaError_t e = cudaDeviceEnablePeerAccess(y, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            else ck(e, "cudaDeviceEnablePeerAccess");
        }
    }
}

template <typename S, typename T>
Sharded<S, T>::~Sharded() {
    for (auto& p : part_) p->sync();
    if (writer_) {
        try {
            writer_->drain();
        } catch (const std::exception&) {
        }
        writer_.reset();
    }
    free_outputs();
    for (auto* evs : {&evE_, &evH_, &evCpE_, &evCpH_, &evMon_})
        for (cudaEvent_t e : *evs) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : tev_) if (e) cudaEventDestroy(e);
    if (d_parts_) {
        cudaSetDevice(part_[0]->device);
        cudaFree(d_parts_);
    }
}

// Planes [c0, c1) components of one local plane of shard src into a local plane of shard dst,
// on dst's stream (components 0-2 E, 3-5 H).
template <typename S, typename T>
void Sharded<S, T>::copy_planes(int dst, int dst_plane, int src, int src_plane, int c0, int c1) {
    Solver<S, T>& a = *part_[dst];
    const Solver<S, T>& b = *part_[src];
    S* const da[6] = {a.a_.Ex, a.a_.Ey, a.a_.Ez, a.a_.Hx, a.a_.Hy, a.a_.Hz};
    const S* const sb[6] = {b.a_.Ex, b.a_.Ey, b.a_.Ez, b.a_.Hx, b.a_.Hy, b.a_.Hz};
    for (int c = c0; c < c1; ++c)
        ck(cudaMemcpyPeerAsync(da[c] + size_t(dst_plane) * a.plane_, a.device, sb[c] + size_t(src_plane) * b.plane_,
                               b.device, a.plane_ * sizeof(S), a.st_),
           "halo copy");
}

template <typename S, typename T>
void Sharded<S, T>::run(uint64_t n) {
    const int R = int(part_.size());
    const uint64_t n0 = steps, last = n0 + n;
    std::vector<ESrc> src(R);
    for (int r = 0; r < R; ++r) {
        ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
        part_[r]->ensure_series((last + part_[r]->save_every_ - 1) / part_[r]->save_every_);
        src[r] = ESrc{};
        part_[r]->src_static(src[r]);
    }
    auto loc = [&](int r, int g) { return g - lo_[r]; };  // global plane -> shard r's local plane
    const bool timed = timing_ == FDTD_TIMING_RUN;
    if (timed) {  // every shard starts after the start event
        ck(cudaSetDevice(part_[0]->device), "cudaSetDevice");
        ck(cudaEventRecord(tev_[0], part_[0]->st_), "cudaEventRecord");
        for (int r = 1; r < R; ++r) {
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            ck(cudaStreamWaitEvent(part_[r]->st_, tev_[0], 0), "cudaStreamWaitEvent");
        }
    }
    for (uint64_t s = n0; s < last; ++s) {
        // E of shard r+1's first plane -> shard r's top halo, after r+1's last E sweep
        for (int r = 0; r + 1 < R; ++r) {
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            ck(cudaStreamWaitEvent(part_[r]->st_, evE_[r + 1], 0), "cudaStreamWaitEvent");
            copy_planes(r, loc(r, z1_[r]), r + 1, loc(r + 1, z0_[r + 1]), 0, 2);
            ck(cudaEventRecord(evCpE_[r], part_[r]->st_), "cudaEventRecord");
        }
        for (int r = 0; r < R; ++r) {  // H, once shard r-1 has read r's H plane of the last step
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            if (r + 1 < R) ck(cudaStreamWaitEvent(part_[r]->st_, evCpH_[r], 0), "cudaStreamWaitEvent");
            ck(cudaStreamWaitEvent(part_[r]->st_, evMon_[r], 0), "cudaStreamWaitEvent");
            part_[r]->phase_H(s);
            ck(cudaEventRecord(evH_[r], part_[r]->st_), "cudaEventRecord");
        }
        // H of shard r's last plane -> shard r+1's bottom halo
        for (int r = 0; r + 1 < R; ++r) {
            ck(cudaSetDevice(part_[r + 1]->device), "cudaSetDevice");
            ck(cudaStreamWaitEvent(part_[r + 1]->st_, evH_[r], 0), "cudaStreamWaitEvent");
            copy_planes(r + 1, loc(r + 1, z0_[r + 1] - 1), r, loc(r, z1_[r] - 1), 3, 5);
            ck(cudaEventRecord(evCpH_[r], part_[r + 1]->st_), "cudaEventRecord");
        }
        const bool mon = interval_ && s % interval_ == 0;
        for (int r = 0; r < R; ++r) {  // E, once shard r-1 has read r's E plane
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            if (r > 0) ck(cudaStreamWaitEvent(part_[r]->st_, evCpE_[r - 1], 0), "cudaStreamWaitEvent");
            part_[r]->phase_E(s, src[r], mon);
            ck(cudaEventRecord(evE_[r], part_[r]->st_), "cudaEventRecord");
        }
        if (writer_ && s % part_[0]->save_every_ == 0) {  // each shard after its own E sweep
            if (!oplan_.movies.empty()) capture_movies();
            if (oplan_.tls) capture_tls(s);
        }
        if (mon) {
            Solver<S, T>& p0 = *part_[0];
            ck(cudaSetDevice(p0.device), "cudaSetDevice");
            for (int r = 1; r < R; ++r) {
                ck(cudaStreamWaitEvent(p0.st_, evE_[r], 0), "cudaStreamWaitEvent");
                ck(cudaMemcpyPeerAsync(d_parts_ + (r - 1), p0.device, part_[r]->d_acc_, part_[r]->device,
                                       sizeof(DiagAccum), p0.st_),
                   "monitor copy");
            }
            k_acc_combine<<<1, 1, 0, p0.st_>>>(p0.d_acc_, d_parts_, R - 1);
            k_monitor_eval<<<1, 1, 0, p0.st_>>>(p0.d_acc_, p0.d_ms_, p0.d_status_, s);
            p0.launches += 2;
            for (int r = 1; r < R; ++r)
                ck(cudaMemcpyPeerAsync(part_[r]->d_status_, part_[r]->device, p0.d_status_, p0.device,
                                       sizeof(unsigned), p0.st_),
                   "status copy");
            ck(cudaEventRecord(evMon_[0], p0.st_), "cudaEventRecord");
            for (int r = 1; r < R; ++r) {  // the shard's accumulator restarts once it was read
                ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
                ck(cudaStreamWaitEvent(part_[r]->st_, evMon_[0], 0), "cudaStreamWaitEvent");
                ck(cudaMemsetAsync(part_[r]->d_acc_, 0, sizeof(DiagAccum), part_[r]->st_), "cudaMemsetAsync");
                ck(cudaEventRecord(evMon_[r], part_[r]->st_), "cudaEventRecord");
            }
        }
    }
    if (timed) {  // the end event after every shard's last work
        for (int r = 1; r < R; ++r) {
            ck(cudaSetDevice(part_[r]->device), "cudaSetDevice");
            ck(cudaEventRecord(evE_[r], part_[r]->st_), "cudaEventRecord");
        }
        ck(cudaSetDevice(part_[0]->device), "cudaSetDevice");
        for (int r = 1; r < R; ++r) ck(cudaStreamWaitEvent(part_[0]->st_, evE_[r], 0), "cudaStreamWaitEvent");
        ck(cudaEventRecord(tev_[1], part_[0]->st_), "cudaEventRecord");
    }
    unsigned status = 0;
    for (auto& p : part_) {
        ck(cudaSetDevice(p->device), "cudaSetDevice");
        ck(cudaStreamSynchronize(p->st_), "run");
        ck(cudaGetLastError(), "step kernels");
    }
    if (timed) {
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, tev_[0], tev_[1]), "cudaEventElapsedTime");
        run_ms_ += ms;
        tsteps_ += n;
    }
    Solver<S, T>& p0 = *part_[0];
    ck(cudaSetDevice(p0.device), "cudaSetDevice");
    ck(cudaMemcpy(&status, p0.d_status_, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
    uint64_t done = last;
    if (status) {
        MonitorState ms{};
        ck(cudaMemcpy(&ms, p0.d_ms_, sizeof(ms), cudaMemcpyDeviceToHost), "monitor state");
        done = ms.step + 1;
    }
    launches = 0;
    for (auto& p : part_) {
        p->steps = done;
        p->series_count_ = std::min<uint64_t>(p->series_count_, (done + p->save_every_ - 1) / p->save_every_);
        launches += p->launches;
    }
    steps = done;
    if (writer_) write_point_samples();
    if (status) throw Failure(FDTD_ERR_UNSTABLE, "stability monitor stopped the solve at step " + std::to_string(done - 1));
}

// Whole-grid idx3 array -> each shard's planes (halos included), and back (owned planes).
template <typename S, typename T>
template <typename F>
void Sharded<S, T>::scatter(const double* h, F&& f) {
    if (!h) throw Failure(FDTD_ERR_INVALID, "null host array");
    for (size_t r = 0; r < part_.size(); ++r) {
        const int nz = int(slice_[r]->v.NzT), lo = lo_[r];
        std::vector<double> l(NxT_ * NyT_ * size_t(nz));
#pragma omp parallel for schedule(static)
        for (long long ij = 0; ij < (long long)(NxT_ * NyT_); ++ij)
            std::memcpy(l.data() + size_t(ij) * nz, h + size_t(ij) * NzT_ + lo, size_t(nz) * sizeof(double));
        f(*part_[r], l.data());
    }
}

template <typename S, typename T>
template <typename F>
void Sharded<S, T>::gather(double* h, F&& f) {
    if (!h) throw Failure(FDTD_ERR_INVALID, "null host array");
    for (size_t r = 0; r < part_.size(); ++r) {
        const int nz = int(slice_[r]->v.NzT), lo = lo_[r], z0 = z0_[r], z1 = z1_[r];
        std::vector<double> l(NxT_ * NyT_ * size_t(nz));
        f(*part_[r], l.data());
#pragma omp parallel for schedule(static)
        for (long long ij = 0; ij < (long long)(NxT_ * NyT_); ++ij)
            std::memcpy(h + size_t(ij) * NzT_ + z0, l.data() + size_t(ij) * nz + (z0 - lo), size_t(z1 - z0) * sizeof(double));
    }
}

template <typename S, typename T>
void Sharded<S, T>::probe_series(double* out, uint64_t max, uint64_t* n) {
    const size_t np = probe_at_.size();
    uint64_t count = 0;
    std::vector<std::vector<double>> col(part_.size());
    for (size_t r = 0; r < part_.size(); ++r) {
        Solver<S, T>& p = *part_[r];
        if (!p.nprobes_) continue;
        count = std::max(count, p.series_count_);
        col[r].resize(p.series_count_ * p.nprobes_);
        if (!col[r].empty()) p.probe_series(col[r].data(), p.series_count_, nullptr);
    }
    if (n) *n = count;
    if (!out || !np) return;
    const uint64_t cnt = std::min(count, max);
    for (size_t q = 0; q < np; ++q) {
        const auto [r, lq] = probe_at_[q];
        const uint32_t pn = part_[r]->nprobes_;
        for (uint64_t t = 0; t < cnt; ++t) out[t * np + q] = col[r][t * pn + size_t(lq)];
    }
}

template <typename S, typename T>
void Sharded<S, T>::dft(uint32_t p, double* re, double* im) {
    if (p >= probe_at_.size()) throw Failure(FDTD_ERR_INVALID, "no DFT for this probe");
    part_[probe_at_[p].first]->dft(uint32_t(probe_at_[p].second), re, im);
}

// ---- detector files of a sharded solve
template <typename S, typename T>
void Sharded<S, T>::attach_outputs(const fdtd::SimSetup& Sp, const std::string& root) {
    if (writer_) throw Failure(FDTD_ERR_INVALID, "outputs are already attached");
    if (steps != 0) throw Failure(FDTD_ERR_INVALID, "outputs can only be attached before the first step");
    if (Sp.NxT != NxT_ || Sp.NyT != NyT_ || Sp.NzT != NzT_ || Sp.save_every != part_[0]->save_every_)
        throw Failure(FDTD_ERR_INVALID, "the setup does not match the handle (grid or SAVE_EVERY)");
    fdtd::OutputPlan plan;
    try {
        plan = fdtd::make_output_plan(Sp);
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_INVALID, e.what());
    }
    size_t comps = 0;
    for (const auto& p : plan.points) comps += p.components.size();
    if (comps != probe_at_.size()) throw Failure(FDTD_ERR_INVALID, "the setup's point detectors do not match the handle's probes");
    try {
        fdtd::write_setup_outputs(Sp, plan, root);
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_IO, e.what());
    }
    const size_t word = plan.float64 ? sizeof(double) : sizeof(float);
    out_.assign(part_.size(), OutPart{});
    try {
        for (size_t r = 0; r < part_.size(); ++r) {
            Solver<S, T>& p = *part_[r];
            OutPart& o = out_[r];
            const int nz = int(slice_[r]->v.NzT), lo = lo_[r];
            for (const auto& m : plan.movies) {
                // XY at plane k: the owner's local plane; XZ / YZ: the shard's whole local z
                // extent, of which the writer keeps the owned planes
                size_t bytes = 0;
                int idx = int(m.index);
                long long d2 = (long long)m.dim2;
                if (m.plane == 0) {
                    if (idx >= z0_[r] && idx < z1_[r]) {
                        idx -= lo;
                        bytes = m.dim1 * m.dim2 * word;
                    }
                } else {
                    d2 = nz;
                    bytes = m.dim1 * size_t(nz) * word;
                }
                o.off.push_back(bytes ? o.slot_bytes : kNoPart);
                o.index.push_back(idx);
                o.d2.push_back(d2);
                o.slot_bytes += round_up(bytes, 256);
            }
            ck(cudaSetDevice(p.device), "cudaSetDevice");
            if (o.slot_bytes)
                for (int q = 0; q < kOutSlots; ++q) {
                    ck(cudaMalloc(reinterpret_cast<void**>(&o.d_slot[q]), o.slot_bytes), "cudaMalloc");
                    ck(cudaHostAlloc(reinterpret_cast<void**>(&o.h_slot[q]), o.slot_bytes, cudaHostAllocDefault), "cudaHostAlloc");
                    ck(cudaEventCreateWithFlags(&o.ev[q], cudaEventDisableTiming), "cudaEventCreate");
                }
            if (plan.tls) {
                ck(cudaMalloc(reinterpret_cast<void**>(&o.d_trec), kTlsSlots * sizeof(TlsRecord)), "cudaMalloc");
                ck(cudaHostAlloc(reinterpret_cast<void**>(&o.h_trec), kTlsSlots * sizeof(TlsRecord), cudaHostAllocDefault),
                   "cudaHostAlloc");
                for (int q = 0; q < kTlsSlots; ++q)
                    ck(cudaEventCreateWithFlags(&o.trec_ev[q], cudaEventDisableTiming), "cudaEventCreate");
                const StepArgs<S, T>& a = p.a_;
                const long long mk = (long long)plan.mon_k;
                if (p.has_gain_ && plan.mon_valid && mk >= z0_[r] && mk < z1_[r]) {
                    const long long i = (long long)plan.mon_i - a.gi0, j = (long long)plan.mon_j - a.gj0, k = mk - lo - a.gk0;
                    if (i >= 0 && i < a.gX && j >= 0 && j < a.gY && k >= 0 && k < a.gZ) o.mon_t = (k * a.gY + j) * a.gX + i;
                }
            }
        }
    } catch (...) {
        free_outputs();
        throw;
    }
    oplan_ = std::move(plan);
    oroot_ = root;
    writer_ = std::make_unique<fdtd::OutputWriter>();
}

template <typename S, typename T>
void Sharded<S, T>::free_outputs() {
    for (size_t r = 0; r < out_.size(); ++r) {
        OutPart& o = out_[r];
        cudaSetDevice(part_[r]->device);
        for (int q = 0; q < kOutSlots; ++q) {
            if (o.d_slot[q]) cudaFree(o.d_slot[q]);
            if (o.h_slot[q]) cudaFreeHost(o.h_slot[q]);
            if (o.ev[q]) cudaEventDestroy(o.ev[q]);
        }
        if (o.d_trec) cudaFree(o.d_trec);
        if (o.h_trec) cudaFreeHost(o.h_trec);
        for (int q = 0; q < kTlsSlots; ++q)
            if (o.trec_ev[q]) cudaEventDestroy(o.trec_ev[q]);
    }
    out_.clear();
}

template <typename S, typename T>
void Sharded<S, T>::capture_movies() {
    const int sl = int(oframe_ % kOutSlots);
    const size_t nm = oplan_.movies.size();
    {
        std::unique_lock<std::mutex> l(oslot_mu_);
        oslot_cv_.wait(l, [&] { return oslot_busy_[sl] == 0; });
        oslot_busy_[sl] = int(nm);
    }
    const int f64 = oplan_.float64 ? 1 : 0;
    const size_t word = f64 ? sizeof(double) : sizeof(float);
    for (size_t r = 0; r < part_.size(); ++r) {
        Solver<S, T>& p = *part_[r];
        OutPart& o = out_[r];
        if (!o.slot_bytes) continue;
        ck(cudaSetDevice(p.device), "cudaSetDevice");
        for (size_t m = 0; m < nm; ++m) {
            if (o.off[m] == kNoPart) continue;
            const fdtd::MoviePlan& v = oplan_.movies[m];
            const long long count = (long long)v.dim1 * o.d2[m];
            const unsigned nb = unsigned(std::min<long long>((count + 255) / 256, 148 * 4));
            k_slice<S><<<nb, 256, 0, p.st_>>>(p.a_.Ex, p.a_.Ey, p.a_.Ez, p.a_.Hx, p.a_.Hy, p.a_.Hz, int(NyT_), p.NxP_,
                                               v.plane, o.index[m], v.component, o.d2[m], count, p.sE_, p.sH_,
                                               o.d_slot[sl] + o.off[m], f64);
            ++p.launches;
        }
        ck(cudaMemcpyAsync(o.h_slot[sl], o.d_slot[sl], o.slot_bytes, cudaMemcpyDeviceToHost, p.st_), "movie part D2H");
        ck(cudaEventRecord(o.ev[sl], p.st_), "cudaEventRecord");
    }
    for (size_t m = 0; m < nm; ++m) {
        const fdtd::MoviePlan& v = oplan_.movies[m];
        auto frame = std::make_shared<std::vector<char>>(v.dim1 * v.dim2 * word);
        fdtd::OutputWriter::Job j;
        // join the shards' parts once their copies are complete (on the writer thread)
        j.wait = [this, sl, m, frame, word] {
            const fdtd::MoviePlan& v = oplan_.movies[m];
            for (size_t r = 0; r < part_.size(); ++r) {
                const OutPart& o = out_[r];
                if (o.off[m] == kNoPart) continue;
                cudaSetDevice(part_[r]->device);
                if (cudaEventSynchronize(o.ev[sl]) != cudaSuccess) throw std::runtime_error("movie frame copy failed");
                const char* part = o.h_slot[sl] + o.off[m];
                if (v.plane == 0) {
                    std::memcpy(frame->data(), part, frame->size());
                    continue;
                }
                const size_t nz = size_t(o.d2[m]), own = size_t(z1_[r] - z0_[r]), skip = size_t(z0_[r] - lo_[r]);
                for (size_t a = 0; a < v.dim1; ++a)
                    std::memcpy(frame->data() + (a * v.dim2 + size_t(z0_[r])) * word, part + (a * nz + skip) * word,
                                own * word);
            }
        };
        j.done = [this, sl, frame] {
            {
                std::lock_guard<std::mutex> l(oslot_mu_);
                --oslot_busy_[sl];
            }
            oslot_cv_.notify_all();
        };
        j.path = fdtd::frame_path(oplan_, oroot_, m, oframe_);
        j.data = frame->data();
        j.bytes = frame->size();
        writer_->submit(std::move(j));
    }
    ++oframe_;
}

template <typename S, typename T>
void Sharded<S, T>::capture_tls(uint64_t s) {
    if (!pop_first_done_) {
        write_population_frame();
        pop_first_done_ = true;
    }
    const int sl = int(tls_count_++ % kTlsSlots);
    {
        std::unique_lock<std::mutex> l(oslot_mu_);
        oslot_cv_.wait(l, [&] { return trec_busy_[sl] == 0; });
        trec_busy_[sl] = 3;
    }
    for (size_t r = 0; r < part_.size(); ++r) {
        Solver<S, T>& p = *part_[r];
        OutPart& o = out_[r];
        ck(cudaSetDevice(p.device), "cudaSetDevice");
        ck(cudaMemsetAsync(o.d_trec + sl, 0, sizeof(TlsRecord), p.st_), "cudaMemsetAsync");
        if (p.has_gain_) {
            const size_t ng = size_t(p.a_.gX) * p.a_.gY * p.a_.gZ;
            const unsigned nb = unsigned(std::max<size_t>(1, std::min<size_t>((ng + 255) / 256, 148 * 4)));
            k_tls_reduce<S, T><<<nb, 256, 0, p.st_>>>(p.a_, p.d_dx_, p.d_dy_, p.d_dz_, int((s + 1) & 1), p.sE_,
                                                        o.d_trec + sl, o.mon_t);
            ++p.launches;
        }
        ck(cudaMemcpyAsync(o.h_trec + sl, o.d_trec + sl, sizeof(TlsRecord), cudaMemcpyDeviceToHost, p.st_), "TLS record D2H");
        ck(cudaEventRecord(o.trec_ev[sl], p.st_), "cudaEventRecord");
    }
    // the whole solve's record: the shards' sums added in shard order; Pz and dPz/dt from the
    // shard that holds the cell (the others leave them 0)
    auto sum = std::make_shared<TlsRecord>();
    const double dt = part_[0]->dt_;
    const std::string dir = fdtd::run_dir(oplan_, oroot_);
    auto release = [this, sl] {
        {
            std::lock_guard<std::mutex> l(oslot_mu_);
            --trec_busy_[sl];
        }
        oslot_cv_.notify_all();
    };
    fdtd::OutputWriter::Job a, b, c;
    a.wait = [this, sl, sum] {
        std::memset(sum.get(), 0, sizeof(TlsRecord));
        for (size_t r = 0; r < part_.size(); ++r) {
            cudaSetDevice(part_[r]->device);
            if (cudaEventSynchronize(out_[r].trec_ev[sl]) != cudaSuccess) throw std::runtime_error("two-level record copy failed");
            const TlsRecord& x = out_[r].h_trec[sl];
            sum->acc.int_Nu += x.acc.int_Nu;
            sum->acc.int_Ng += x.acc.int_Ng;
            sum->acc.p_energy += x.acc.p_energy;
            if (out_[r].mon_t >= 0) {
                sum->P_center = x.P_center;
                sum->dP_dt = x.dP_dt;
            }
        }
    };
    a.text = [sum, s, dt] { return fdtd::inversion_line(s, dt, sum->acc.int_Nu, sum->acc.int_Ng); };
    a.path = dir + "/populations/inversion_time.csv";
    b.text = [sum, s, dt] { return fdtd::polarization_line(s, dt, sum->P_center, sum->dP_dt, sum->acc.p_energy); };
    b.path = dir + "/polarization/polarization_time.csv";
    c.text = [sum, s, dt] { return fdtd::global_history_line(s, dt, sum->acc.int_Nu, sum->acc.int_Ng); };
    c.path = dir + "/tls_global_history.csv";
    for (fdtd::OutputWriter::Job* j : {&a, &b, &c}) {
        j->append = true;
        j->done = release;
        writer_->submit(std::move(*j));
    }
}

template <typename S, typename T>
void Sharded<S, T>::write_population_frame() {
    // PopulationTimeSeriesDetector::write_binary_frame: the full-grid Nu and Ng, FP64, idx3,
    // gathered from the shards' owned planes
    const size_t N = size_t(NxT_) * NyT_ * NzT_;
    const std::string dir = fdtd::run_dir(oplan_, oroot_) + "/populations/";
    for (int w : {int(FDTD_TLS_NU), int(FDTD_TLS_NG)}) {
        auto buf = std::make_shared<std::vector<double>>(N);
        get_tls(w, buf->data());
        fdtd::OutputWriter::Job j;
        j.path = dir + (w == FDTD_TLS_NU ? "populations_Nu.bin" : "populations_Ng.bin");
        j.data = buf->data();
        j.bytes = N * sizeof(double);
        j.append = true;
        j.done = [buf] {};
        writer_->submit(std::move(j));
    }
}

template <typename S, typename T>
void Sharded<S, T>::write_point_samples() {
    const size_t np = probe_at_.size();
    if (oplan_.points.empty() || !np) return;
    uint64_t count = 0;  // every shard samples the same steps
    for (auto& p : part_)
        if (p->nprobes_) count = std::max(count, p->series_count_);
    if (count <= ots_written_) return;
    const uint64_t n0 = ots_written_, n = count - ots_written_;
    // only the samples not yet written, from each shard that holds probes
    std::vector<std::vector<double>> col(part_.size());
    for (size_t r = 0; r < part_.size(); ++r) {
        Solver<S, T>& p = *part_[r];
        if (!p.nprobes_) continue;
        col[r].resize(size_t(n) * p.nprobes_);
        ck(cudaSetDevice(p.device), "cudaSetDevice");
        ck(cudaMemcpy(col[r].data(), p.d_series_ + size_t(n0) * p.nprobes_, col[r].size() * sizeof(double),
                      cudaMemcpyDeviceToHost),
           "probe samples D2H");
    }
    const std::string dir = fdtd::run_dir(oplan_, oroot_);
    size_t q = 0;  // global probe index, in the plan's order
    for (const auto& pt : oplan_.points) {
        for (int c : pt.components) {
            const auto [r, lq] = probe_at_[q];
            const uint32_t pn = part_[r]->nprobes_;
            auto value = [&](uint64_t t) { return col[r][size_t(t) * pn + size_t(lq)]; };
            auto buf = std::make_shared<std::vector<char>>();
            if (oplan_.float64) {
                buf->resize(n * sizeof(double));
                for (uint64_t t = 0; t < n; ++t) {
                    const double d = value(t);
                    std::memcpy(buf->data() + t * 8, &d, 8);
                }
            } else {
                buf->resize(n * sizeof(float));
                for (uint64_t t = 0; t < n; ++t) {
                    const float f = float(value(t));
                    std::memcpy(buf->data() + t * 4, &f, 4);
                }
            }
            fdtd::OutputWriter::Job j;
            j.path = dir + "/" + pt.name + "/" + fdtd::component_name(c) + "_ts.bin";
            j.data = buf->data();
            j.bytes = buf->size();
            j.append = true;
            j.done = [buf] {};
            writer_->submit(std::move(j));
            ++q;
        }
    }
    ots_written_ = count;
}

template <typename S, typename T>
void Sharded<S, T>::flush_outputs() {
    if (!writer_) return;
    try {
        writer_->drain();
    } catch (const std::exception& e) {
        throw Failure(FDTD_ERR_IO, e.what());
    }
}

template <typename S, typename T>
void Sharded<S, T>::close_outputs() {
    if (!writer_) return;
    if (oplan_.tls) {  // PopulationTimeSeriesDetector::finalize: the last frame and the metadata
        write_population_frame();
        try {
            fdtd::write_population_metadata(oplan_, oroot_);
        } catch (const std::exception& e) {
            throw Failure(FDTD_ERR_IO, e.what());
        }
    }
    flush_outputs();
    writer_.reset();
}
}  // namespace

// ==================================================================== C ABI
struct fdtd_handle {
    std::unique_ptr<SolverBase> s;
    std::string err;
};

namespace {
thread_local std::string g_err;

template <typename F>
int guarded(fdtd_handle* h, F&& f) {
    try {
        f();
        return FDTD_OK;
    } catch (const Failure& e) {
        (h ? h->err : g_err) = e.what();
        return e.code;
    } catch (const std::exception& e) {
        (h ? h->err : g_err) = e.what();
        return FDTD_ERR_INVALID;
    }
}
}  // namespace

namespace {
// Why a setup view cannot be stepped, or nullptr.
const char* setup_problem(const fdtd_setup_v1* s) {
    if (s->struct_size != sizeof(fdtd_setup_v1)) return "fdtd_setup_v1.struct_size mismatch";
    if (s->rounding > FDTD_ROUND_STOCHASTIC) return "fdtd_setup_v1.rounding must be 0 (nearest) or 1 (stochastic)";
    // NyT is a grid dimension (z) of the layout-transpose kernels: at most 65535.
    if (s->NxT < 3 || s->NyT < 3 || s->NzT < 3 || s->NxT > (1u << 30) || s->NyT > 65535 || s->NzT > (1u << 30))
        return "grid dimensions out of range";
    if (2 * uint64_t(s->npml) >= s->NxT || 2 * uint64_t(s->npml) >= s->NyT || 2 * uint64_t(s->npml) >= s->NzT)
        return "npml too large for the grid";
    if (!s->bE[0] || !s->bE[1] || !s->bE[2] || !s->inv_dx || !s->inv_dy || !s->inv_dz || !s->dx || !s->dy || !s->dz)
        return "missing required setup arrays";
    for (int a = 0; a < 3; ++a)
        if (!s->cpml_kappa[a] || !s->cpml_bE[a] || !s->cpml_cE[a] || !s->cpml_bH[a] || !s->cpml_cH[a])
            return "missing CPML profile arrays";
    return nullptr;
}
}  // namespace

const fdtd::SimSetup* fdtd_internal_setup(const fdtd_setup* s);  // capi_setup.cpp

extern "C" {

int fdtd_create(const fdtd_setup_v1* s, int device, fdtd_handle** out) {
    if (!s || !out) { g_err = "null argument"; return FDTD_ERR_INVALID; }
    *out = nullptr;
    if (const char* why = setup_problem(s)) { g_err = why; return FDTD_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_err = "no CUDA device available";
        return FDTD_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) { g_err = "device index out of range"; return FDTD_ERR_INVALID; }
    auto* h = new fdtd_handle();
    const int rc = guarded(nullptr, [&] {
        if (s->precision == FDTD_PREC_FP64) h->s = std::make_unique<Solver<double, double>>(*s, device);
        else if (s->precision == FDTD_PREC_FP32) h->s = std::make_unique<Solver<float, float>>(*s, device);
        else if (s->precision == FDTD_PREC_FP16) h->s = std::make_unique<Solver<__half, float>>(*s, device);
        else if (s->precision == FDTD_PREC_BF16) h->s = std::make_unique<Solver<__nv_bfloat16, float>>(*s, device);
        else throw Failure(FDTD_ERR_UNSUPPORTED, "precision must be FDTD_PREC_FP32, _FP64, _FP16 or _BF16");
    });
    if (rc != FDTD_OK) { delete h; return rc; }
    *out = h;
    return FDTD_OK;
}

int fdtd_create_sharded(const fdtd_setup_v1* s, int nshards, const int* devices, fdtd_handle** out) {
    if (!s || !out) { g_err = "null argument"; return FDTD_ERR_INVALID; }
    *out = nullptr;
    if (const char* why = setup_problem(s)) { g_err = why; return FDTD_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_err = "no CUDA device available";
        return FDTD_ERR_NO_DEVICE;
    }
    if (nshards < 2 || nshards > 64) { g_err = "nshards must be 2..64"; return FDTD_ERR_INVALID; }
    for (int r = 0; devices && r < nshards; ++r)
        if (devices[r] < 0 || devices[r] >= ndev) { g_err = "device index out of range"; return FDTD_ERR_INVALID; }
    auto* h = new fdtd_handle();
    const int rc = guarded(nullptr, [&] {
        if (s->precision == FDTD_PREC_FP64) h->s = std::make_unique<Sharded<double, double>>(*s, nshards, devices);
        else if (s->precision == FDTD_PREC_FP32) h->s = std::make_unique<Sharded<float, float>>(*s, nshards, devices);
        else if (s->precision == FDTD_PREC_FP16) h->s = std::make_unique<Sharded<__half, float>>(*s, nshards, devices);
        else if (s->precision == FDTD_PREC_BF16) h->s = std::make_unique<Sharded<__nv_bfloat16, float>>(*s, nshards, devices);
        else throw Failure(FDTD_ERR_UNSUPPORTED, "precision must be FDTD_PREC_FP32, _FP64, _FP16 or _BF16");
    });
    if (rc != FDTD_OK) { delete h; return rc; }
    *out = h;
    return FDTD_OK;
}

int fdtd_set_field(fdtd_handle* h, int c, const double* a) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->set_field(c, a); }); }
int fdtd_get_field(fdtd_handle* h, int c, double* a) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->get_field(c, a); }); }
int fdtd_set_tls_state(fdtd_handle* h, int w, const double* a) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->set_tls(w, a); }); }
int fdtd_get_tls_state(fdtd_handle* h, int w, double* a) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->get_tls(w, a); }); }
int fdtd_run(fdtd_handle* h, uint64_t n) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->run(n); }); }
int fdtd_steps_done(const fdtd_handle* h, uint64_t* n) { if (!h || !n) return FDTD_ERR_INVALID; *n = h->s->steps; return FDTD_OK; }
int fdtd_get_probe_series(fdtd_handle* h, double* out, uint64_t max, uint64_t* n) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->probe_series(out, max, n); }); }
int fdtd_get_dft(fdtd_handle* h, uint32_t p, double* re, double* im) { if (!h || !re || !im) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->dft(p, re, im); }); }
int fdtd_get_diagnostics(fdtd_handle* h, fdtd_diagnostics_v1* d) { if (!h || !d) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->diagnostics(d); }); }
int fdtd_device_bytes(const fdtd_handle* h, uint64_t* b) { if (!h || !b) return FDTD_ERR_INVALID; *b = h->s->dev_bytes; return FDTD_OK; }
int fdtd_kernel_launches(const fdtd_handle* h, uint64_t* n) { if (!h || !n) return FDTD_ERR_INVALID; *n = h->s->launches; return FDTD_OK; }
int fdtd_material_rows(const fdtd_handle* h, uint64_t* rows) { if (!h || !rows) return FDTD_ERR_INVALID; *rows = h->s->material_rows; return FDTD_OK; }
int fdtd_set_timing(fdtd_handle* h, int mode) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->set_timing(mode); }); }
int fdtd_get_timing(fdtd_handle* h, fdtd_timing_v1* t) { if (!h || !t) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->timing(t); }); }
int fdtd_set_kernel_path(fdtd_handle* h, int path) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->set_path(path); }); }
int fdtd_attach_outputs(fdtd_handle* h, const fdtd_setup* s, const char* out_dir) {
    if (!h || !s || !out_dir) return FDTD_ERR_INVALID;
    return guarded(h, [&] { h->s->attach_outputs(*fdtd_internal_setup(s), out_dir); });
}
int fdtd_flush_outputs(fdtd_handle* h) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->flush_outputs(); }); }
int fdtd_close_outputs(fdtd_handle* h) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->close_outputs(); }); }
int fdtd_synchronize(fdtd_handle* h) { if (!h) return FDTD_ERR_INVALID; return guarded(h, [&] { h->s->sync(); }); }
const char* fdtd_last_error(const fdtd_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }
void fdtd_destroy(fdtd_handle* h) { delete h; }

}  // extern "C"


// ---- packed multi-solve engine
struct fdtd_batch {
    std::unique_ptr<Batch> b;
    std::string err;
};

namespace {
template <typename F>
int bguard(fdtd_batch* b, F&& f) {
    try {
        f();
        return FDTD_OK;
    } catch (const Failure& e) {
        (b ? b->err : g_err) = e.what();
        return e.code;
    } catch (const std::exception& e) {
        (b ? b->err : g_err) = e.what();
        return FDTD_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

int fdtd_batch_create(int device, uint64_t budget_bytes, fdtd_batch** out) {
    if (!out) { g_err = "null argument"; return FDTD_ERR_INVALID; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_err = "no CUDA device available";
        return FDTD_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) { g_err = "device index out of range"; return FDTD_ERR_INVALID; }
    auto* b = new fdtd_batch();
    const int rc = bguard(nullptr, [&] { b->b = std::make_unique<Batch>(device, budget_bytes); });
    if (rc != FDTD_OK) { delete b; return rc; }
    *out = b;
    return FDTD_OK;
}

int fdtd_batch_submit(fdtd_batch* b, const fdtd_setup_v1* s, uint64_t n_steps, uint64_t* ticket) {
    if (!b || !s || !ticket) return FDTD_ERR_INVALID;
    if (const char* why = setup_problem(s)) { b->err = why; return FDTD_ERR_INVALID; }
    return bguard(b, [&] { *ticket = b->b->submit(*s, n_steps); });
}

int fdtd_batch_run(fdtd_batch* b, uint64_t max_steps, uint32_t* n_resident, uint32_t* n_queued) {
    if (!b) return FDTD_ERR_INVALID;
    return bguard(b, [&] {
        b->b->run(max_steps);
        if (n_resident) *n_resident = b->b->resident();
        if (n_queued) *n_queued = b->b->queued();
    });
}

int fdtd_batch_job_state(fdtd_batch* b, uint64_t ticket, int* state, uint64_t* steps_done) {
    if (!b || !state) return FDTD_ERR_INVALID;
    return bguard(b, [&] { b->b->state_of(ticket, state, steps_done); });
}

int fdtd_batch_probe_series(fdtd_batch* b, uint64_t ticket, double* out, uint64_t max_samples, uint64_t* n_samples) {
    if (!b || !n_samples) return FDTD_ERR_INVALID;
    return bguard(b, [&] {
        Batch::Job& j = b->b->finished_job(ticket);
        const uint64_t n = std::min<uint64_t>(max_samples, j.samples);
        if (out && n) std::memcpy(out, j.series.data(), n * j.nprobes * sizeof(double));
        *n_samples = j.samples;
    });
}

int fdtd_batch_dft(fdtd_batch* b, uint64_t ticket, uint32_t probe, double* re, double* im) {
    if (!b || !re || !im) return FDTD_ERR_INVALID;
    return bguard(b, [&] {
        Batch::Job& j = b->b->finished_job(ticket);
        if (probe >= j.nprobes) throw Failure(FDTD_ERR_INVALID, "probe index out of range");
        for (uint32_t m = 0; m < j.nf; ++m) {
            re[m] = j.dft[2 * (size_t(probe) * j.nf + m)];
            im[m] = j.dft[2 * (size_t(probe) * j.nf + m) + 1];
        }
    });
}

int fdtd_batch_diagnostics(fdtd_batch* b, uint64_t ticket, fdtd_diagnostics_v1* out) {
    if (!b || !out) return FDTD_ERR_INVALID;
    return bguard(b, [&] {
        Batch::Job& j = b->b->finished_job(ticket);
        *out = j.diag;
    });
}

int fdtd_batch_release(fdtd_batch* b, uint64_t ticket) {
    if (!b) return FDTD_ERR_INVALID;
    return bguard(b, [&] { b->b->release(ticket); });
}

const char* fdtd_batch_last_error(const fdtd_batch* b) { return b ? b->err.c_str() : g_err.c_str(); }

void fdtd_batch_destroy(fdtd_batch* b) { delete b; }

}  // extern "C"

// Lets other translation units of the library report through fdtd_last_error(NULL).
namespace fdtd_internal {
__attribute__((visibility("hidden"))) void set_global_error(const std::string& msg) { g_err = msg; }
}
