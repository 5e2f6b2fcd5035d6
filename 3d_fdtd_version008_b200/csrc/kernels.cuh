// kernels.cuh -- sm_100a stepping kernels of the Yee FDTD loop.
//
// Device layout: every 3-D array is stored x-fastest, (k, j, i) -> (k*NyT + j)*NxP + i,
// rows padded to NxP (a multiple of 128 bytes).  A thread owns W = 16/sizeof(T)
// consecutive x cells (one 128-bit load per array; 16-bit storage: 4 cells, and 8 in the
// H sweep's interior), a warp owns one row segment of 32, 16 or 8 vectors, and each
// thread marches in +z through a chunk of planes carrying the z-neighbour plane in
// registers (2.5D blocking).  x-neighbours come from the adjacent lane by warp shuffle
// (one scalar load at the segment edge), y-neighbours from the adjacent row through L1.
//
// Physics per step n (reference order, src/3D_FDTD_version008.cpp:269-328):
//   k_update_H : H -= bH * curl E with the CPML psi_H recursion fused in
//                (fdtd_update_H src/fdtd_stepper.hpp:8-47 + apply_after_H src/boundary.hpp:150-225)
//   k_update_E : polarization P^{n+1} (src/two_level_system.hpp:574-609), E += bE*(curl H - J - dP/dt)
//                with psi_E fused (src/fdtd_stepper.hpp:49-89, src/two_level_system.hpp:299-342,
//                src/boundary.hpp:227-300), then the population update with E^{n+1}
//                (src/two_level_system.hpp:612-666), all in one pass over the cell.
// CPML psi lives only in the PML slabs: x-slab [k][j][2np], y-slab [k][2np][NxP],
// z-slab [2np][j][NxP], index 0 for the low side, np.. for the high side.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace fdtdk {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned kStatusTimeout = 2u;                // status bit: a bounded device wait expired
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s bound on any device-side wait

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr int kBlockY = 8;    // rows (warps) per block
constexpr int kMaxSources = 8;

template <typename T> struct Vec;
template <> struct Vec<float> {
    static constexpr int W = 4;
    __device__ __forceinline__ static void ld(const float* p, float (&a)[4]) {
        float4 t = *reinterpret_cast<const float4*>(p);
        a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
    }
    __device__ __forceinline__ static void ldg(const float* p, float (&a)[4]) {
        float4 t = __ldg(reinterpret_cast<const float4*>(p));
        a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
    }
    __device__ __forceinline__ static void st(float* p, const float (&a)[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
    }
    __device__ __forceinline__ static void ldcg(const float* p, float (&a)[4]) {
        float4 t = __ldcg(reinterpret_cast<const float4*>(p));
        a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
    }
};
template <> struct Vec<double> {
    static constexpr int W = 2;
    __device__ __forceinline__ static void ld(const double* p, double (&a)[2]) {
        double2 t = *reinterpret_cast<const double2*>(p);
        a[0] = t.x; a[1] = t.y;
    }
    __device__ __forceinline__ static void ldg(const double* p, double (&a)[2]) {
        double2 t = __ldg(reinterpret_cast<const double2*>(p));
        a[0] = t.x; a[1] = t.y;
    }
    __device__ __forceinline__ static void st(double* p, const double (&a)[2]) {
        *reinterpret_cast<double2*>(p) = make_double2(a[0], a[1]);
    }
    __device__ __forceinline__ static void ldcg(const double* p, double (&a)[2]) {
        double2 t = __ldcg(reinterpret_cast<const double2*>(p));
        a[0] = t.x; a[1] = t.y;
    }
};

// Field / psi storage.  S is the type held in memory, T the type the update computes in;
// a thread moves W = Vec<T>::W consecutive cells per array (16 bytes of T, 8 bytes of a
// 16-bit S).
template <typename S, typename T> struct Fld;
template <typename T> struct Fld<T, T> {
    __device__ __forceinline__ static void ld(const T* p, T (&a)[Vec<T>::W]) { Vec<T>::ld(p, a); }
    __device__ __forceinline__ static void ldg(const T* p, T (&a)[Vec<T>::W]) { Vec<T>::ldg(p, a); }
    __device__ __forceinline__ static void st(T* p, const T (&a)[Vec<T>::W]) { Vec<T>::st(p, a); }
    __device__ __forceinline__ static void ldcg(const T* p, T (&a)[Vec<T>::W]) { Vec<T>::ldcg(p, a); }
};
template <> struct Fld<__half, float> {
    __device__ __forceinline__ static void ld(const __half* p, float (&a)[4]) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void ldcg(const __half* p, float (&a)[4]) {
        const uint2 u = __ldcg(reinterpret_cast<const uint2*>(p));
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void ldg(const __half* p, float (&a)[4]) {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void st(__half* p, const float (&a)[4]) {
        const __half2 lo = __floats2half2_rn(a[0], a[1]), hi = __floats2half2_rn(a[2], a[3]);
        uint2 u;
        u.x = *reinterpret_cast<const unsigned*>(&lo);
        u.y = *reinterpret_cast<const unsigned*>(&hi);
        *reinterpret_cast<uint2*>(p) = u;
    }
};
template <> struct Fld<__nv_bfloat16, float> {
    __device__ __forceinline__ static void ld(const __nv_bfloat16* p, float (&a)[4]) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void ldcg(const __nv_bfloat16* p, float (&a)[4]) {
        const uint2 u = __ldcg(reinterpret_cast<const uint2*>(p));
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void ldg(const __nv_bfloat16* p, float (&a)[4]) {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
    __device__ __forceinline__ static void st(__nv_bfloat16* p, const float (&a)[4]) {
        const __nv_bfloat162 lo = __floats2bfloat162_rn(a[0], a[1]), hi = __floats2bfloat162_rn(a[2], a[3]);
        uint2 u;
        u.x = *reinterpret_cast<const unsigned*>(&lo);
        u.y = *reinterpret_cast<const unsigned*>(&hi);
        *reinterpret_cast<uint2*>(p) = u;
    }
};

// 32-bit integer mixer (the finaliser of Austin Appleby's MurmurHash3, public domain).
__device__ __forceinline__ unsigned mix32(unsigned x) {
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

// FP32 -> BF16 with stochastic rounding: r's low 16 bits (uniform) are added to the 16 bits
// that the conversion drops, then the value is truncated, so it rounds away from zero with
// probability (dropped bits) / 2^16 and the rounding error is zero on average.  Inf and NaN
// pass unchanged.
__device__ __forceinline__ unsigned short bf16_stochastic(float f, unsigned r) {
    unsigned b = __float_as_uint(f);
    if ((b & 0x7f800000u) != 0x7f800000u) b += r & 0xffffu;
    return static_cast<unsigned short>(b >> 16);
}

// Scalar load through L2 only (no L1): values another SM wrote during this launch.
__device__ __forceinline__ float ldcg1(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg1(const double* p) { return __ldcg(p); }
__device__ __forceinline__ __half ldcg1(const __half* p) {
    const unsigned short u = __ldcg(reinterpret_cast<const unsigned short*>(p));
    return *reinterpret_cast<const __half*>(&u);
}
__device__ __forceinline__ __nv_bfloat16 ldcg1(const __nv_bfloat16* p) {
    const unsigned short u = __ldcg(reinterpret_cast<const unsigned short*>(p));
    return *reinterpret_cast<const __nv_bfloat16*>(&u);
}

// Scalar conversions between the storage and compute types.
__device__ __forceinline__ float to_c(float v) { return v; }
__device__ __forceinline__ double to_c(double v) { return v; }
__device__ __forceinline__ float to_c(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_c(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ void put(float& d, float v) { d = v; }
__device__ __forceinline__ void put(double& d, double v) { d = v; }
__device__ __forceinline__ void put(__half& d, float v) { d = __float2half_rn(v); }
__device__ __forceinline__ void put(__nv_bfloat16& d, float v) { d = __float2bfloat16_rn(v); }
// FP64 host value -> storage type (set-up and field writes)
template <typename S> __device__ __forceinline__ S from_d(double v);
template <> __device__ __forceinline__ float from_d<float>(double v) { return float(v); }
template <> __device__ __forceinline__ double from_d<double>(double v) { return v; }
template <> __device__ __forceinline__ __half from_d<__half>(double v) { return __double2half(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v) { return __double2bfloat16(v); }

// 16-bit storage, interior columns: a thread holds 8 cells of an array as one 16-byte word
// (uint4) and updates them as two 4-cell halves; half h is cells 4h .. 4h+3, the word's
// (x, y) or (z, w).
template <typename S>
__device__ __forceinline__ void unpack4(const uint2 u, float (&a)[4]) {
    if constexpr (std::is_same_v<S, __half>) {
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    } else {
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
        a[0] = lo.x; a[1] = lo.y; a[2] = hi.x; a[3] = hi.y;
    }
}
__device__ __forceinline__ uint2 half_of(const uint4& v, int h) { return h ? make_uint2(v.z, v.w) : make_uint2(v.x, v.y); }
// cell 0 and cell 7 of a word, as FP32
template <typename S>
__device__ __forceinline__ float first_of(const uint4& v) {
    const unsigned short b = (unsigned short)(v.x & 0xffffu);
    return to_c(*reinterpret_cast<const S*>(&b));
}
template <typename S>
__device__ __forceinline__ float last_of(const uint4& v) {
    const unsigned short b = (unsigned short)(v.w >> 16);
    return to_c(*reinterpret_cast<const S*>(&b));
}

// Explicitly rounded arithmetic of the update formulas.  Every product, difference and
// fused multiply-add of an update goes through one of these, so the compiler can neither
// contract nor reassociate them: every instantiation of one update (the single-solve sweeps,
// the packed engine, staged or direct loads, the slab-ordered step, any launch shape) gives
// the same bits.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// One-sided difference quotient (b - a) * inv_d.
template <typename T>
__device__ __forceinline__ T dq(T b, T a, T inv_d) { return mul_rn(sub_rn(b, a), inv_d); }

// CPML recursion psi = b * psi + c * d.
template <typename T>
__device__ __forceinline__ T psi_rec(T b, T psi, T c, T d) { return fma_rn(b, psi, mul_rn(c, d)); }

// CPML: d_eff = d / kappa + psi.  With 16-bit storage psi is kept as psi * dx_min (the host
// folds dx_min into the recursion's c coefficient) so it stays in the storage's range, and
// is scaled back here by psc = 1 / dx_min; with S = T psi is stored as is.
template <typename S, typename T>
__device__ __forceinline__ T psi_eff(T d, T ik, T psi, T psc) {
    if constexpr (sizeof(S) == sizeof(T)) return fma_rn(d, ik, psi);
    else return fma_rn(d, ik, mul_rn(psi, psc));
}

// Per gain region constants (TwoLevelParams after finalize_with_dt), in compute type T.
// With scaled field storage (E = sE * E', H = sH * H') kapaN0 and inv_hbar_omega carry
// the factor sE and dp_scale = 1 / sH; unscaled storage has sE = sH = 1.
template <typename T>
struct GainCoef {
    T kapaN0;          // kapa_coeff * Ndip
    T pa2, pa3, inv_dt;
    T inv_N0;          // 1 / Ng0
    T N0;
    T dt, inv_tau, inv_hbar_omega, pump;
    T dp_scale;        // 1 / sH: dP/dt enters the scaled Ez update as dP * dp_scale
    int clamp;         // TLS_ENABLE_CLAMP renormalisation
    int active;        // Ndip > 0
};

// Fields and CPML psi are stored as S, everything else as T.
template <typename S, typename T = S>
struct StepArgs {
    int NxT, NyT, NzT, NxP, np;
    long long plane;  // NxP * NyT
    // z sharding: local plane k is global plane k + kz0 of NzG; the H sweep updates local planes
    // [kH0, kH1), the E sweep [kE0, kE1).  A whole solve: kz0 = 0, NzG = NzT, [0, NzT-1), [1, NzT).
    int kz0, NzG, kH0, kH1, kE0, kE1;
    S *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    const T *bEx, *bEy, *bEz;
    // Indexed material (the E kernels' MAT instantiation): per cell a uint16 index into a table
    // of distinct (bEx, bEy, bEz, 0) rows; bEx/bEy/bEz are then unused.
    const uint16_t* bidx;
    const T* btab;
    T bH;
    const T *idx, *idy, *idz;         // 1/dx (padded to NxP), 1/dy, 1/dz
    const T *ik[3];                   // 1/kappa per axis
    const T *pbE[3], *pcE[3], *pbH[3], *pcH[3];
    // psi_H: 0 Hx_y, 1 Hx_z, 2 Hy_z, 3 Hy_x, 4 Hz_x, 5 Hz_y ; psi_E likewise for E
    S *psiH[6], *psiE[6];
    // gain block: bounding box of the gain cells, x-fastest with row length gX
    int gain, gi0, gj0, gk0, gX, gY, gZ;
    const int8_t* greg;               // region id per bbox cell, -1 = none
    T *P0, *P1;                       // polarization ping-pong: P^n lives in slot (n & 1)
    T *Nu, *Ng;
    const GainCoef<T>* gcoef;
    const unsigned* status;           // nonzero: a monitor step failed, skip all work
    T psc;                            // psi scale (16-bit storage: 1 / dx_min; else 1)
    int sr;                           // BF16 storage: E and H stores rounded stochastically
};

// W values of field array `arr` (Ex..Hz = 0..5) at local offset c.  With stochastic rounding
// (BF16 storage) they are rounded stochastically, keyed by (global cell, array, step), so a
// cell's rounding is the same whatever the launch shape, sharding or packing; else rounded to
// nearest.  SRM: 0 nearest, 1 stochastic (the single-solve sweeps, compiled per mode so that
// the default kernel carries no stochastic-rounding code), 2 as a.sr says (the packed and
// slab-ordered kernels, whose launches serve both).
template <int SRM = 2, typename S, typename T>
__device__ __forceinline__ void st_field(const StepArgs<S, T>& a, S* p, size_t c, const T (&v)[Vec<T>::W], unsigned arr,
                                         unsigned step) {
    if constexpr (std::is_same_v<S, __nv_bfloat16> && SRM != 0) {
        if (SRM == 1 || a.sr) {
            const unsigned cell = unsigned(c + size_t(a.kz0) * size_t(a.plane));
            const unsigned salt = mix32(step * 0x9e3779b9u + arr);
            unsigned short h[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) h[e] = bf16_stochastic(v[e], mix32((cell + e) ^ salt));
            uint2 u;
            u.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
            u.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
            *reinterpret_cast<uint2*>(p + c) = u;
            return;
        }
    }
    Fld<S, T>::st(p + c, v);
}

constexpr int kMaxSheets = 2;

// Per-step arguments of the E kernel.
struct ESrc {
    int n;                 // number of point sources
    int parity;            // step & 1
    int si[kMaxSources], sj[kMaxSources], sk[kMaxSources], sc[kMaxSources];
    double J[kMaxSources]; // I((n+1/2)dt)/cell_area
    // plane-wave sheets: J added on plane `pl` normal to `ax` over [lo0, hi0] x [lo1, hi1]
    // (in-plane axes in x, y, z order), component `pc`
    int ns;
    int ax[kMaxSheets], pc[kMaxSheets], pl[kMaxSheets];
    int lo0[kMaxSheets], hi0[kMaxSheets], lo1[kMaxSheets], hi1[kMaxSheets];
    unsigned step;         // n (low 32 bits): the stochastic rounding key of step n's stores
    double sJ[kMaxSheets];
};

__device__ __forceinline__ bool in_pml(int n, int N, int np) { return n < np || n >= N - np; }
__device__ __forceinline__ int slab_index(int n, int N, int np) { return n < np ? n : n - (N - 2 * np); }

// x-slab psi ([k][j][2 np]) of one W-cell vector.  Both arrays are read before any psi
// store is issued: the compiler may not move a load of one psi array above a store to the
// other, and a read-after-store chain per cell would cost one memory round trip each.
template <typename S, typename T>
__device__ __forceinline__ void xpsi_load(const S* p3, const S* p4, const StepArgs<S, T>& a, int k, int j, int i0,
                                          T (&x3)[Vec<T>::W], T (&x4)[Vec<T>::W]) {
    const size_t row = (size_t(k) * a.NyT + j) * (2 * a.np);
#pragma unroll
    for (int e = 0; e < Vec<T>::W; ++e) {
        const int i = i0 + e;
        const bool in = i < a.NxT && in_pml(i, a.NxT, a.np);
        const size_t q = row + (in ? slab_index(i, a.NxT, a.np) : 0);
        x3[e] = in ? T(to_c(p3[q])) : T(0);
        x4[e] = in ? T(to_c(p4[q])) : T(0);
    }
}

// Writes back the x-slab psi of the cells ilo <= i < ihi of the vector.
template <typename S, typename T>
__device__ __forceinline__ void xpsi_store(S* p3, S* p4, const StepArgs<S, T>& a, int k, int j, int i0, int ilo, int ihi,
                                           const T (&x3)[Vec<T>::W], const T (&x4)[Vec<T>::W]) {
    const size_t row = (size_t(k) * a.NyT + j) * (2 * a.np);
#pragma unroll
    for (int e = 0; e < Vec<T>::W; ++e) {
        const int i = i0 + e;
        if (i >= ilo && i < ihi && in_pml(i, a.NxT, a.np)) {
            const size_t q = row + slab_index(i, a.NxT, a.np);
            put(p3[q], x3[e]);
            put(p4[q], x4[e]);
        }
    }
}

// One row (bEx, bEy, bEz) of the indexed material's table.
template <typename T>
__device__ __forceinline__ void table_row(const T* tab, unsigned id, T& x, T& y, T& z) {
    if constexpr (sizeof(T) == 4) {
        const float4 r = __ldg(reinterpret_cast<const float4*>(tab) + id);
        x = r.x; y = r.y; z = r.z;
    } else {
        const double2 r0 = __ldg(reinterpret_cast<const double2*>(tab) + 2 * id);
        x = r0.x; y = r0.y;
        z = __ldg(tab + 4 * size_t(id) + 2);
    }
}

// The W row numbers at p, packed two per word (W = 4: 8 bytes, W = 2: 4 bytes).
template <int W>
struct RowIds {
    unsigned w[W / 2];
    __device__ __forceinline__ void load(const uint16_t* p) {
        if constexpr (W == 4) {
            const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
            w[0] = v.x; w[1] = v.y;
        } else {
            w[0] = __ldg(reinterpret_cast<const unsigned*>(p));
        }
    }
    __device__ __forceinline__ unsigned operator[](int e) const { return (w[e >> 1] >> (16 * (e & 1))) & 0xffffu; }
};

// bEx, bEy, bEz of the W cells at offset c: from the three arrays, or (MAT) the table rows of
// the ids the caller loaded one plane ahead (so the table reads, which hit L1, do not wait
// for an HBM load of the same iteration).
template <bool MAT, typename S, typename T>
__device__ __forceinline__ void load_bE(const StepArgs<S, T>& a, size_t c, const RowIds<Vec<T>::W>& ids,
                                        T (&bx)[Vec<T>::W], T (&by)[Vec<T>::W], T (&bz)[Vec<T>::W]) {
    constexpr int W = Vec<T>::W;
    if constexpr (MAT) {
#pragma unroll
        for (int e = 0; e < W; ++e) table_row(a.btab, ids[e], bx[e], by[e], bz[e]);
    } else {
        Vec<T>::ldg(a.bEx + c, bx);
        Vec<T>::ldg(a.bEy + c, by);
        Vec<T>::ldg(a.bEz + c, bz);
    }
}

// ---------------------------------------------------------------------------------
// Asynchronous copies into shared memory (cp.async): the loads of the next plane are in
// flight while the current one is computed, without registers held for them.
// L1: keep the line in L1 (data another warp of the block reads too: H, whose row j is the
// next warp's row j-1); else 16-byte copies go through L2 only.
template <int BYTES, bool L1 = true>
__device__ __forceinline__ void cp_async(void* smem, const void* g) {
    const unsigned s = unsigned(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16 && !L1) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(g) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(g), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared-memory staging of the sweeps' interior columns.  A slot holds one field vector of
// one thread (SB bytes), slots are slot-major so a warp's slots are consecutive, and kStages
// planes of slots form a ring: the thread copies plane k + kStages - 1 while it computes
// plane k.  A 16-byte slot holds 4 FP32 or 2 FP64 cells, or the 8 cells of an H-sweep vector
// of 16-bit storage; the E sweep's 4-cell 16-bit vectors fill 8-byte slots and run four stages
// (three planes in flight) in the shared memory the others spend on two.
template <int SB_, int STAGES>
struct PipeShape {
    static constexpr int SB = SB_;
    static constexpr int kStages = STAGES;
};

// E sweep slots: 0-2 E, 3-5 H, 6 Hz(j-1), 7 Hx(j-1), 8 the material row ids, last: Hz and
// Hy at i0-1 for the warp's first lane (at byte 0 and SB/2 of the slot).  Staging is used with
// the row-indexed material only.
template <typename S>
struct EPipe : PipeShape<sizeof(S) == 2 ? 8 : 16, sizeof(S) == 2 ? 4 : 2> {
    static constexpr int kSlots = 10;
    static constexpr int kX = kSlots - 1;
    static constexpr size_t bytes() { return size_t(EPipe::kStages) * kSlots * (32 * kBlockY) * EPipe::SB; }
};

// True when a point source or (SH) a plane-wave sheet touches one of the W cells (i0.., j, k).
template <bool SH>
__device__ __forceinline__ bool src_in_vector(const ESrc& src, int i0, int j, int k, int W) {
    bool hit = false;
    for (int s = 0; s < src.n; ++s)
        hit |= src.sj[s] == j && src.sk[s] == k && src.si[s] >= i0 && src.si[s] < i0 + W;
    if constexpr (SH) for (int s = 0; s < src.ns; ++s) {
        if (src.ax[s] == 2)
            hit |= k == src.pl[s] && j >= src.lo1[s] && j <= src.hi1[s] && i0 + W > src.lo0[s] && i0 <= src.hi0[s];
        else if (src.ax[s] == 1)
            hit |= j == src.pl[s] && k >= src.lo1[s] && k <= src.hi1[s] && i0 + W > src.lo0[s] && i0 <= src.hi0[s];
        else
            hit |= src.pl[s] >= i0 && src.pl[s] < i0 + W && j >= src.lo0[s] && j <= src.hi0[s] && k >= src.lo1[s] &&
                   k <= src.hi1[s];
    }
    return hit;
}

// J of the plane-wave sheets at cell (i, j, k), added after the point sources (the
// reference's source registration order).
template <typename T>
__device__ __forceinline__ void sheet_J(const ESrc& src, int i, int j, int k, T& Jx, T& Jy, T& Jz) {
    for (int s = 0; s < src.ns; ++s) {
        bool in;
        if (src.ax[s] == 2) in = k == src.pl[s] && i >= src.lo0[s] && i <= src.hi0[s] && j >= src.lo1[s] && j <= src.hi1[s];
        else if (src.ax[s] == 1) in = j == src.pl[s] && i >= src.lo0[s] && i <= src.hi0[s] && k >= src.lo1[s] && k <= src.hi1[s];
        else in = i == src.pl[s] && j >= src.lo0[s] && j <= src.hi0[s] && k >= src.lo1[s] && k <= src.hi1[s];
        if (in) {
            const T v = T(src.sJ[s]);
            if (src.pc[s] == 0) Jx = add_rn(Jx, v);
            else if (src.pc[s] == 1) Jy = add_rn(Jy, v);
            else Jz = add_rn(Jz, v);
        }
    }
}

// Plain-vector updates: no CPML slab, gain cell or source in the W cells, every cell
// updated.  Same operations in the same order as the general update with psi, J and dP/dt
// absent; the general path carries per-cell tests that cost more issue slots than the
// arithmetic itself, and about 85 % of the cells of a CPML-bounded grid are plain.
template <typename S, typename T, int SRM = 2>
__device__ __forceinline__ void h_plain(const StepArgs<S, T>& a, const size_t c, const T (&ex0)[Vec<T>::W],
                                        const T (&ex1)[Vec<T>::W], const T (&ey0)[Vec<T>::W],
                                        const T (&ey1)[Vec<T>::W], const T (&ez)[Vec<T>::W],
                                        const T (&exj)[Vec<T>::W], const T (&ezj)[Vec<T>::W], const T eyn,
                                        const T ezn, T (&hx)[Vec<T>::W], T (&hy)[Vec<T>::W], T (&hz)[Vec<T>::W],
                                        const T (&idx)[Vec<T>::W], const T idy, const T idz, const unsigned step) {
    constexpr int W = Vec<T>::W;
    const T nbH = -a.bH;
#pragma unroll
    for (int e = 0; e < W; ++e) {
        const T eyx = (e < W - 1) ? ey0[e + 1] : eyn;
        const T ezx = (e < W - 1) ? ez[e + 1] : ezn;
        const T dEz_dy = dq(ezj[e], ez[e], idy);
        const T dEy_dz = dq(ey1[e], ey0[e], idz);
        const T dEx_dz = dq(ex1[e], ex0[e], idz);
        const T dEz_dx = dq(ezx, ez[e], idx[e]);
        const T dEy_dx = dq(eyx, ey0[e], idx[e]);
        const T dEx_dy = dq(exj[e], ex0[e], idy);
        hx[e] = fma_rn(nbH, sub_rn(dEz_dy, dEy_dz), hx[e]);
        hy[e] = fma_rn(nbH, sub_rn(dEx_dz, dEz_dx), hy[e]);
        hz[e] = fma_rn(nbH, sub_rn(dEy_dx, dEx_dy), hz[e]);
    }
    st_field<SRM>(a, a.Hx, c, hx, 3, step);
    st_field<SRM>(a, a.Hy, c, hy, 4, step);
    st_field<SRM>(a, a.Hz, c, hz, 5, step);
}

template <typename S, typename T, int SRM = 2>
__device__ __forceinline__ void e_plain(const StepArgs<S, T>& a, const size_t c, T (&ex)[Vec<T>::W], T (&ey)[Vec<T>::W],
                                        T (&ez)[Vec<T>::W], const T (&bx)[Vec<T>::W], const T (&by)[Vec<T>::W],
                                        const T (&bz)[Vec<T>::W], const T (&hx)[Vec<T>::W],
                                        const T (&hy)[Vec<T>::W], const T (&hz)[Vec<T>::W],
                                        const T (&hzj)[Vec<T>::W], const T (&hxj)[Vec<T>::W],
                                        const T (&hxm)[Vec<T>::W], const T (&hym)[Vec<T>::W], const T hzp,
                                        const T hyp, const T (&idx)[Vec<T>::W], const T idy, const T idz,
                                        const unsigned step) {
    constexpr int W = Vec<T>::W;
#pragma unroll
    for (int e = 0; e < W; ++e) {
        const T hzx = (e > 0) ? hz[e - 1] : hzp;
        const T hyx = (e > 0) ? hy[e - 1] : hyp;
        const T dHz_dy = dq(hz[e], hzj[e], idy);
        const T dHy_dz = dq(hy[e], hym[e], idz);
        const T dHx_dz = dq(hx[e], hxm[e], idz);
        const T dHz_dx = dq(hz[e], hzx, idx[e]);
        const T dHy_dx = dq(hy[e], hyx, idx[e]);
        const T dHx_dy = dq(hx[e], hxj[e], idy);
        // (curl - J) with J = 0 is the curl itself, bit for bit: the general path's result
        ex[e] = fma_rn(bx[e], sub_rn(dHz_dy, dHy_dz), ex[e]);
        ey[e] = fma_rn(by[e], sub_rn(dHx_dz, dHz_dx), ey[e]);
        ez[e] = fma_rn(bz[e], sub_rn(dHy_dx, dHx_dy), ez[e]);
    }
    st_field<SRM>(a, a.Ex, c, ex, 0, step);
    st_field<SRM>(a, a.Ey, c, ey, 1, step);
    st_field<SRM>(a, a.Ez, c, ez, 2, step);
}

// ---------------------------------------------------------------------------------
// Launch geometry of the sweeps.  The x range of a row is split into the interior
// [xi0, xi1) -- vectors with no x-slab cell, of W cells (8 for 16-bit storage, whose field
// arrays are offset so that xi0 falls on a 16-byte boundary) -- covered by gxi block columns of
// `lanes`-vector row segments, and the edge vectors outside it (nl on the left, ne in total),
// which one extra block column packs er rows at a time, one thread per edge vector.
// Interior warps therefore never diverge on the x slab, and edge threads all take the
// general path together.  An interior warp holds 32 / lanes adjacent rows of one block
// column (lanes = 32, 16 or 8), so that a narrow interior does not leave most lanes idle:
// a 100-vector interior fills 100 of 128 lanes in 32-lane rows, 100 of 104 in 8-lane rows.
struct SweepGeom {
    int xi0, xi1;  // interior x range (cells)
    int gxi;       // interior block columns
    int nl, ne;    // edge vectors per row: on the left, in total
    int er;        // rows per edge block
    int lanes;     // lanes per interior row segment (32, 16 or 8)
};

// Interior block columns of the E sweep: gxi, except for 16-bit storage, whose E sweep runs
// 4-cell vectors over the interior that the H sweep covers with 8-cell ones (H measured 10-12 %
// faster with 8-cell vectors, E 0-11 % slower, on the 536^3 workload).
template <typename S>
__host__ __device__ __forceinline__ int gxi_E(const SweepGeom& g) {
    if constexpr (sizeof(S) == 2) return ((g.xi1 - g.xi0) / 4 + g.lanes - 1) / g.lanes;
    else return g.gxi;
}

// Row and first vector of an interior thread: warp w of block row `by` holds rows
// (by * kBlockY + w) * R .. + R - 1 (R = 32 / lanes), segment `lane / lanes` of the warp one row.
struct InteriorLane {
    int j;   // row (may lie outside the grid: the caller masks it)
    int li;  // lane within the row segment
};
__device__ __forceinline__ InteriorLane interior_lane(const SweepGeom& g, const int by, const int lane) {
    const int R = 32 / g.lanes;
    const int seg = lane / g.lanes;
    return {(by * kBlockY + int(threadIdx.y)) * R + seg, lane - seg * g.lanes};
}

// One thread's column of W-cell vectors (i0.., j, kb..ke-1), marching in +z.
// Every load of an iteration (the vectors, the x-neighbour at the warp or interior edge,
// 1/dz, the CPML psi of the vector) is issued before the first use of any of them, so a
// vector costs one memory round trip per plane whatever slab it lies in.  EDGE columns
// read the x-neighbour from memory (lanes hold other rows); interior columns shuffle it.
// H sweep slots (as EPipe): 0-1 Ex, Ey at k+1, 2 Ez, 3 Ex(j+1), 4 Ez(j+1), 5-7 H, 8 Ey and Ez
// at i0+W for the lanes that load it (at byte 0 and SB/2 of the slot).
template <typename S>
struct HPipe : PipeShape<16, 2> {
    static constexpr int kSlots = 9;
    static constexpr size_t bytes() { return size_t(HPipe::kStages) * kSlots * (32 * kBlockY) * HPipe::SB; }
};

// li: the thread's lane within its row segment of g.lanes lanes (interior columns).
template <typename S, typename T, bool EDGE, bool PIPE = false, int SRM = 2>
__device__ __forceinline__ void h_column(const StepArgs<S, T>& a, const SweepGeom& g, const int j, const int i0,
                                         const bool act, const int kb, const int ke, const int li,
                                         const unsigned step) {
    constexpr int W = Vec<T>::W;
    const int np = a.np, np2 = 2 * np;
    const T nbH = -a.bH;

    T idx[W];
#pragma unroll
    for (int e = 0; e < W; ++e) idx[e] = act ? __ldg(a.idx + i0 + e) : T(0);
    const T idy = __ldg(a.idy + j);
    const bool ypml = in_pml(j, a.NyT, np);
    const int jy = ypml ? slab_index(j, a.NyT, np) : 0;
    T yb = 1, yc = 0, yik = 1;
    if (ypml) { yb = __ldg(a.pbH[1] + j); yc = __ldg(a.pcH[1] + j); yik = __ldg(a.ik[1] + j); }
    const bool xpml = EDGE && act && (i0 < np || i0 + W > a.NxT - np);
    const bool plain_row = act && !ypml && !xpml && i0 + W <= a.NxT - 1;
    // Ey, Ez at i0+W come from memory at the end of the row segment, at the end of the
    // interior (the next lane then holds no interior vector) and for every edge column
    const bool nload = EDGE || li == g.lanes - 1 || i0 + W >= g.xi1;

    const size_t row = size_t(j) * a.NxP + i0;
    T ex0[W], ey0[W];
    if (act) {
        Fld<S, T>::ldg(a.Ex + size_t(kb) * a.plane + row, ex0);
        Fld<S, T>::ldg(a.Ey + size_t(kb) * a.plane + row, ey0);
    } else {
#pragma unroll
        for (int e = 0; e < W; ++e) ex0[e] = ey0[e] = T(0);
    }

    // PIPE (interior columns of k_update_H): this thread's planes come from shared memory,
    // filled by cp.async one plane ahead.
    extern __shared__ uint4 pipe_smem[];
    constexpr int NT = 32 * kBlockY, NV = HPipe<S>::kSlots, SB = HPipe<S>::SB, NS = HPipe<S>::kStages;
    constexpr int VB = W * int(sizeof(S));
    static_assert(VB <= SB, "a field vector fills at most one slot");
    constexpr int NB = sizeof(S) < 4 ? 4 : int(sizeof(S));
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const bool xn = nload && i0 + W < a.NxT;
    char* const pipe = reinterpret_cast<char*>(pipe_smem);
    auto slot = [&](int stg, int q) { return pipe + ((size_t(stg) * NV + q) * NT + tid) * SB; };
    auto issue = [&](int kk, int stg) {
        const size_t cc = size_t(kk) * a.plane + row;
        cp_async<VB>(slot(stg, 0), a.Ex + cc + a.plane);
        cp_async<VB>(slot(stg, 1), a.Ey + cc + a.plane);
        cp_async<VB>(slot(stg, 2), a.Ez + cc);
        cp_async<VB>(slot(stg, 3), a.Ex + cc + a.NxP);
        cp_async<VB>(slot(stg, 4), a.Ez + cc + a.NxP);
        cp_async<VB, false>(slot(stg, 5), a.Hx + cc);
        cp_async<VB, false>(slot(stg, 6), a.Hy + cc);
        cp_async<VB, false>(slot(stg, 7), a.Hz + cc);
        if (xn) {
            cp_async<NB>(slot(stg, 8), a.Ey + cc + W);
            cp_async<NB>(slot(stg, 8) + SB / 2, a.Ez + cc + W);
        }
    };
    if constexpr (PIPE) {
        // planes kb .. kb + NS - 2 in flight before the loop
#pragma unroll
        for (int q = 0; q < NS - 1; ++q) {
            if (act && kb + q < ke) issue(kb + q, q);
            cp_async_commit();
        }
    }

    for (int k = kb; k < ke; ++k) {
        const size_t c = size_t(k) * a.plane + row;
        T ex1[W], ey1[W], ez[W], exj[W], ezj[W], hx[W], hy[W], hz[W];
        T eye = T(0), eze = T(0);
        if (PIPE && act) {
            // plane k + NS - 1 into the stage read last iteration, then wait for plane k
            if (k + NS - 1 < ke) issue(k + NS - 1, (k + NS - 1 - kb) & (NS - 1));
            cp_async_commit();
            cp_async_wait<NS - 1>();
            const int stg = (k - kb) & (NS - 1);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 0)), ex1);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 1)), ey1);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 2)), ez);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 3)), exj);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 4)), ezj);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 5)), hx);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 6)), hy);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 7)), hz);
            if (xn) {
                const char* xs = slot(stg, 8);
                eye = T(to_c(reinterpret_cast<const S*>(xs)[0]));
                eze = T(to_c(reinterpret_cast<const S*>(xs + SB / 2)[0]));
            }
        } else if (act) {
            Fld<S, T>::ldg(a.Ex + c + a.plane, ex1);
            Fld<S, T>::ldg(a.Ey + c + a.plane, ey1);
            Fld<S, T>::ldg(a.Ez + c, ez);
            Fld<S, T>::ldg(a.Ex + c + a.NxP, exj);
            Fld<S, T>::ldg(a.Ez + c + a.NxP, ezj);
            Fld<S, T>::ld(a.Hx + c, hx);
            Fld<S, T>::ld(a.Hy + c, hy);
            Fld<S, T>::ld(a.Hz + c, hz);
        } else {
#pragma unroll
            for (int e = 0; e < W; ++e) ex1[e] = ey1[e] = ez[e] = exj[e] = ezj[e] = hx[e] = hy[e] = hz[e] = T(0);
        }
        if (!PIPE && xn && act) { eye = to_c(a.Ey[c + W]); eze = to_c(a.Ez[c + W]); }
        const T idz = __ldg(a.idz + k);
        const bool zpml = in_pml(k + a.kz0, a.NzG, np);
        T zb = 1, zc = 0, zik = 1;
        size_t zs = 0, ys = 0;
        T pxy[W], pzy[W], pxz[W], pyz[W];  // psi Hx_y, Hz_y, Hx_z, Hy_z
        if (zpml) {
            zb = __ldg(a.pbH[2] + k); zc = __ldg(a.pcH[2] + k); zik = __ldg(a.ik[2] + k);
            zs = (size_t(slab_index(k + a.kz0, a.NzG, np)) * a.NyT + j) * a.NxP + i0;
            if (act) { Fld<S, T>::ld(a.psiH[1] + zs, pxz); Fld<S, T>::ld(a.psiH[2] + zs, pyz); }
        }
        if (ypml) {
            ys = (size_t(k) * np2 + jy) * a.NxP + i0;
            if (act) { Fld<S, T>::ld(a.psiH[0] + ys, pxy); Fld<S, T>::ld(a.psiH[5] + ys, pzy); }
        }
        T x3[W], x4[W];  // psi Hy_x, Hz_x
        if (xpml) xpsi_load<S, T>(a.psiH[3], a.psiH[4], a, k, j, i0, x3, x4);
        // x-neighbour at i0+W: the next lane's first cell, or the loaded one
        T eyn = eye, ezn = eze;
        if (!EDGE) {
            const T sy = __shfl_down_sync(kFull, ey0[0], 1, g.lanes);
            const T sz = __shfl_down_sync(kFull, ez[0], 1, g.lanes);
            if (!nload) { eyn = sy; ezn = sz; }
        }
        if (plain_row && !zpml) {
            h_plain<S, T, SRM>(a, c, ex0, ex1, ey0, ey1, ez, exj, ezj, eyn, ezn, hx, hy, hz, idx, idy, idz, step);
#pragma unroll
            for (int e = 0; e < W; ++e) { ex0[e] = ex1[e]; ey0[e] = ey1[e]; }
            continue;
        }
#pragma unroll
        for (int e = 0; e < W; ++e) {
            const int i = i0 + e;
            if (i >= a.NxT - 1) continue;  // last x plane (and padding) never updated
            const T eyx = (e < W - 1) ? ey0[e + 1] : eyn;
            const T ezx = (e < W - 1) ? ez[e + 1] : ezn;
            T dEz_dy = dq(ezj[e], ez[e], idy);
            T dEy_dz = dq(ey1[e], ey0[e], idz);
            T dEx_dz = dq(ex1[e], ex0[e], idz);
            T dEz_dx = dq(ezx, ez[e], idx[e]);
            T dEy_dx = dq(eyx, ey0[e], idx[e]);
            T dEx_dy = dq(exj[e], ex0[e], idy);
            if (ypml) {
                pxy[e] = psi_rec(yb, pxy[e], yc, dEz_dy); dEz_dy = psi_eff<S, T>(dEz_dy, yik, pxy[e], a.psc);
                pzy[e] = psi_rec(yb, pzy[e], yc, dEx_dy); dEx_dy = psi_eff<S, T>(dEx_dy, yik, pzy[e], a.psc);
            }
            if (zpml) {
                pxz[e] = psi_rec(zb, pxz[e], zc, dEy_dz); dEy_dz = psi_eff<S, T>(dEy_dz, zik, pxz[e], a.psc);
                pyz[e] = psi_rec(zb, pyz[e], zc, dEx_dz); dEx_dz = psi_eff<S, T>(dEx_dz, zik, pyz[e], a.psc);
            }
            if (xpml && in_pml(i, a.NxT, np)) {
                const T b = __ldg(a.pbH[0] + i), cc = __ldg(a.pcH[0] + i), ik = __ldg(a.ik[0] + i);
                x3[e] = psi_rec(b, x3[e], cc, dEz_dx);
                dEz_dx = psi_eff<S, T>(dEz_dx, ik, x3[e], a.psc);
                x4[e] = psi_rec(b, x4[e], cc, dEy_dx);
                dEy_dx = psi_eff<S, T>(dEy_dx, ik, x4[e], a.psc);
            }
            hx[e] = fma_rn(nbH, sub_rn(dEz_dy, dEy_dz), hx[e]);
            hy[e] = fma_rn(nbH, sub_rn(dEx_dz, dEz_dx), hy[e]);
            hz[e] = fma_rn(nbH, sub_rn(dEy_dx, dEx_dy), hz[e]);
        }
        if (act) {
            st_field<SRM>(a, a.Hx, c, hx, 3, step);
            st_field<SRM>(a, a.Hy, c, hy, 4, step);
            st_field<SRM>(a, a.Hz, c, hz, 5, step);
            if (zpml) { Fld<S, T>::st(a.psiH[1] + zs, pxz); Fld<S, T>::st(a.psiH[2] + zs, pyz); }
            if (ypml) { Fld<S, T>::st(a.psiH[0] + ys, pxy); Fld<S, T>::st(a.psiH[5] + ys, pzy); }
            if (xpml) xpsi_store<S, T>(a.psiH[3], a.psiH[4], a, k, j, i0, 0, a.NxT - 1, x3, x4);
        }
#pragma unroll
        for (int e = 0; e < W; ++e) { ex0[e] = ex1[e]; ey0[e] = ey1[e]; }
    }
}

// 16-bit storage, interior column: the thread's 8 cells (i0 .. i0+7, i0 16-byte aligned) of
// every array come as one 16-byte word per plane (PIPE: one 16-byte cp.async each), and the
// two 4-cell halves take h_column's update in the same order: the same bits.  Ey, Ez at
// i0+8 come from the next lane's first cell or, at the end of the row segment or of the
// interior, from memory.
template <typename S, bool PIPE, int SRM = 2>
__device__ __forceinline__ void h_column8(const StepArgs<S, float>& a, const SweepGeom& g, const int j, const int i0,
                                          const bool act, const int kb, const int ke, const int li,
                                          const unsigned step) {
    using T = float;
    constexpr int W = 4;
    const int np = a.np, np2 = 2 * np;
    const T nbH = -a.bH;

    T idx[2][W];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int e = 0; e < W; ++e) idx[h][e] = act ? __ldg(a.idx + i0 + 4 * h + e) : T(0);
    const T idy = __ldg(a.idy + j);
    const bool ypml = in_pml(j, a.NyT, np);
    const int jy = ypml ? slab_index(j, a.NyT, np) : 0;
    T yb = 1, yc = 0, yik = 1;
    if (ypml) { yb = __ldg(a.pbH[1] + j); yc = __ldg(a.pcH[1] + j); yik = __ldg(a.ik[1] + j); }
    const bool nload = li == g.lanes - 1 || i0 + 8 >= g.xi1;
    const bool xn = nload && i0 + 8 < a.NxT;

    const size_t row = size_t(j) * a.NxP + i0;
    auto ld16 = [](const S* p) { return __ldg(reinterpret_cast<const uint4*>(p)); };
    uint4 ex0 = make_uint4(0, 0, 0, 0), ey0 = make_uint4(0, 0, 0, 0);
    if (act) {
        ex0 = ld16(a.Ex + size_t(kb) * a.plane + row);
        ey0 = ld16(a.Ey + size_t(kb) * a.plane + row);
    }

    extern __shared__ uint4 pipe_smem[];
    constexpr int NT = 32 * kBlockY, NV = HPipe<S>::kSlots, NS = HPipe<S>::kStages;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    char* const pipe = reinterpret_cast<char*>(pipe_smem);
    auto slot = [&](int stg, int q) { return pipe + ((size_t(stg) * NV + q) * NT + tid) * 16; };
    auto issue = [&](int kk, int stg) {
        const size_t cc = size_t(kk) * a.plane + row;
        cp_async<16>(slot(stg, 0), a.Ex + cc + a.plane);
        cp_async<16>(slot(stg, 1), a.Ey + cc + a.plane);
        cp_async<16>(slot(stg, 2), a.Ez + cc);
        cp_async<16>(slot(stg, 3), a.Ex + cc + a.NxP);
        cp_async<16>(slot(stg, 4), a.Ez + cc + a.NxP);
        cp_async<16, false>(slot(stg, 5), a.Hx + cc);
        cp_async<16, false>(slot(stg, 6), a.Hy + cc);
        cp_async<16, false>(slot(stg, 7), a.Hz + cc);
        if (xn) {
            cp_async<4>(slot(stg, 8), a.Ey + cc + 8);
            cp_async<4>(slot(stg, 8) + 8, a.Ez + cc + 8);
        }
    };
    if constexpr (PIPE) {
#pragma unroll
        for (int q = 0; q < NS - 1; ++q) {
            if (act && kb + q < ke) issue(kb + q, q);
            cp_async_commit();
        }
    }

    for (int k = kb; k < ke; ++k) {
        const size_t c = size_t(k) * a.plane + row;
        uint4 ex1, ey1, ez, exj, ezj, hx, hy, hz;
        T eye = T(0), eze = T(0);
        if (PIPE && act) {
            if (k + NS - 1 < ke) issue(k + NS - 1, (k + NS - 1 - kb) & (NS - 1));
            cp_async_commit();
            cp_async_wait<NS - 1>();
            const int stg = (k - kb) & (NS - 1);
            ex1 = *reinterpret_cast<const uint4*>(slot(stg, 0));
            ey1 = *reinterpret_cast<const uint4*>(slot(stg, 1));
            ez = *reinterpret_cast<const uint4*>(slot(stg, 2));
            exj = *reinterpret_cast<const uint4*>(slot(stg, 3));
            ezj = *reinterpret_cast<const uint4*>(slot(stg, 4));
            hx = *reinterpret_cast<const uint4*>(slot(stg, 5));
            hy = *reinterpret_cast<const uint4*>(slot(stg, 6));
            hz = *reinterpret_cast<const uint4*>(slot(stg, 7));
            if (xn) {
                const char* xs = slot(stg, 8);
                eye = T(to_c(reinterpret_cast<const S*>(xs)[0]));
                eze = T(to_c(reinterpret_cast<const S*>(xs + 8)[0]));
            }
        } else if (act) {
            ex1 = ld16(a.Ex + c + a.plane);
            ey1 = ld16(a.Ey + c + a.plane);
            ez = ld16(a.Ez + c);
            exj = ld16(a.Ex + c + a.NxP);
            ezj = ld16(a.Ez + c + a.NxP);
            hx = *reinterpret_cast<const uint4*>(a.Hx + c);
            hy = *reinterpret_cast<const uint4*>(a.Hy + c);
            hz = *reinterpret_cast<const uint4*>(a.Hz + c);
            if (xn) { eye = to_c(a.Ey[c + 8]); eze = to_c(a.Ez[c + 8]); }
        } else {
            ex1 = ey1 = ez = exj = ezj = hx = hy = hz = make_uint4(0, 0, 0, 0);
        }
        const T idz = __ldg(a.idz + k);
        const bool zpml = in_pml(k + a.kz0, a.NzG, np);
        T zb = 1, zc = 0, zik = 1;
        if (zpml) { zb = __ldg(a.pbH[2] + k); zc = __ldg(a.pcH[2] + k); zik = __ldg(a.ik[2] + k); }
        // Ey, Ez at i0+8: the next lane's first cell, or the loaded one
        const T sy = __shfl_down_sync(kFull, first_of<S>(ey0), 1, g.lanes);
        const T sz = __shfl_down_sync(kFull, first_of<S>(ez), 1, g.lanes);
        const T eyn8 = nload ? eye : sy, ezn8 = nload ? eze : sz;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ih = i0 + 4 * h;
            const size_t ch = c + 4 * h;
            T vex0[W], vex1[W], vey0[W], vey1[W], vez[W], vexj[W], vezj[W], vhx[W], vhy[W], vhz[W];
            unpack4<S>(half_of(ex0, h), vex0); unpack4<S>(half_of(ex1, h), vex1);
            unpack4<S>(half_of(ey0, h), vey0); unpack4<S>(half_of(ey1, h), vey1);
            unpack4<S>(half_of(ez, h), vez);
            unpack4<S>(half_of(exj, h), vexj); unpack4<S>(half_of(ezj, h), vezj);
            unpack4<S>(half_of(hx, h), vhx); unpack4<S>(half_of(hy, h), vhy); unpack4<S>(half_of(hz, h), vhz);
            // x-neighbour of the half's last cell: the other half's first cell, or i0+8
            T eyn = eyn8, ezn = ezn8;
            if (h == 0) {
                T t[W];
                unpack4<S>(half_of(ey0, 1), t); eyn = t[0];
                unpack4<S>(half_of(ez, 1), t); ezn = t[0];
            }
            const bool plain = act && !ypml && ih + W <= a.NxT - 1;
            if (plain && !zpml) {
                h_plain<S, T, SRM>(a, ch, vex0, vex1, vey0, vey1, vez, vexj, vezj, eyn, ezn, vhx, vhy, vhz, idx[h], idy, idz, step);
                continue;
            }
            size_t zs = 0, ys = 0;
            T pxy[W], pzy[W], pxz[W], pyz[W];  // psi Hx_y, Hz_y, Hx_z, Hy_z
            if (zpml) {
                zs = (size_t(slab_index(k + a.kz0, a.NzG, np)) * a.NyT + j) * a.NxP + ih;
                if (act) { Fld<S, T>::ld(a.psiH[1] + zs, pxz); Fld<S, T>::ld(a.psiH[2] + zs, pyz); }
            }
            if (ypml) {
                ys = (size_t(k) * np2 + jy) * a.NxP + ih;
                if (act) { Fld<S, T>::ld(a.psiH[0] + ys, pxy); Fld<S, T>::ld(a.psiH[5] + ys, pzy); }
            }
#pragma unroll
            for (int e = 0; e < W; ++e) {
                const int i = ih + e;
                if (i >= a.NxT - 1) continue;  // last x plane (and padding) never updated
                const T eyx = (e < W - 1) ? vey0[e + 1] : eyn;
                const T ezx = (e < W - 1) ? vez[e + 1] : ezn;
                T dEz_dy = dq(vezj[e], vez[e], idy);
                T dEy_dz = dq(vey1[e], vey0[e], idz);
                T dEx_dz = dq(vex1[e], vex0[e], idz);
                T dEz_dx = dq(ezx, vez[e], idx[h][e]);
                T dEy_dx = dq(eyx, vey0[e], idx[h][e]);
                T dEx_dy = dq(vexj[e], vex0[e], idy);
                if (ypml) {
                    pxy[e] = psi_rec(yb, pxy[e], yc, dEz_dy); dEz_dy = psi_eff<S, T>(dEz_dy, yik, pxy[e], a.psc);
                    pzy[e] = psi_rec(yb, pzy[e], yc, dEx_dy); dEx_dy = psi_eff<S, T>(dEx_dy, yik, pzy[e], a.psc);
                }
                if (zpml) {
                    pxz[e] = psi_rec(zb, pxz[e], zc, dEy_dz); dEy_dz = psi_eff<S, T>(dEy_dz, zik, pxz[e], a.psc);
                    pyz[e] = psi_rec(zb, pyz[e], zc, dEx_dz); dEx_dz = psi_eff<S, T>(dEx_dz, zik, pyz[e], a.psc);
                }
                vhx[e] = fma_rn(nbH, sub_rn(dEz_dy, dEy_dz), vhx[e]);
                vhy[e] = fma_rn(nbH, sub_rn(dEx_dz, dEz_dx), vhy[e]);
                vhz[e] = fma_rn(nbH, sub_rn(dEy_dx, dEx_dy), vhz[e]);
            }
            if (act) {
                st_field<SRM>(a, a.Hx, ch, vhx, 3, step);
                st_field<SRM>(a, a.Hy, ch, vhy, 4, step);
                st_field<SRM>(a, a.Hz, ch, vhz, 5, step);
                if (zpml) { Fld<S, T>::st(a.psiH[1] + zs, pxz); Fld<S, T>::st(a.psiH[2] + zs, pyz); }
                if (ypml) { Fld<S, T>::st(a.psiH[0] + ys, pxy); Fld<S, T>::st(a.psiH[5] + ys, pzy); }
            }
        }
        ex0 = ex1;
        ey0 = ey1;
    }
}

// One block of the H sweep: block (bx, by, bz) of the solve's launch grid.
template <typename S, typename T, bool PIPE = false, int SRM = 2>
__device__ __forceinline__ void update_H_block(const StepArgs<S, T>& a, const int kchunk, const SweepGeom& g,
                                               const int bx, const int by, const int bz, const unsigned step) {
    constexpr int W = Vec<T>::W;
    if (*a.status) return;
    const int lane = threadIdx.x;
    const int kb = max(bz * kchunk, a.kH0);
    const int ke = min(bz * kchunk + kchunk, a.kH1);
    if (kb >= ke) return;
    if (bx < g.gxi) {
        // H is updated for rows j < NyT - 1.  A warp with no such row leaves as a whole; in a
        // warp that has one, a row beyond it stays in the loop (the shuffles need every lane)
        // as inactive lanes on a valid row index, which load and store nothing.
        const InteriorLane il = interior_lane(g, by, lane);
        const int jlast = a.NyT - 2;
        if ((by * kBlockY + int(threadIdx.y)) * (32 / g.lanes) > jlast) return;
        const bool row_ok = il.j <= jlast;
        if constexpr (sizeof(S) == 2) {  // 8-cell interior vectors
            const int i0 = g.xi0 + (bx * g.lanes + il.li) * 8;
            h_column8<S, PIPE, SRM>(a, g, row_ok ? il.j : jlast, i0, row_ok && i0 < g.xi1, kb, ke, il.li, step);
        } else {
            const int i0 = g.xi0 + (bx * g.lanes + il.li) * W;
            h_column<S, T, false, PIPE, SRM>(a, g, row_ok ? il.j : jlast, i0, row_ok && i0 < g.xi1, kb, ke, il.li, step);
        }
    } else {
        const int t = threadIdx.y * 32 + lane;
        const int rr = t / g.ne, v = t - rr * g.ne;
        const int j = by * g.er + rr;
        if (rr >= g.er || j >= a.NyT - 1) return;
        const int i0 = v < g.nl ? v * W : g.xi1 + (v - g.nl) * W;
        if (i0 >= a.NxT) return;
        h_column<S, T, true, false, SRM>(a, g, j, i0, true, kb, ke, 0, step);
    }
}

// Two resident blocks per SM (at most 128 registers; a third block would spill).
// PIPE: interior columns stage their planes in shared memory (HPipe<S>::bytes() dynamic).
template <typename S, typename T, bool PIPE = false, int SRM = 2>
__global__ void __launch_bounds__(32 * kBlockY, 2)
k_update_H(const StepArgs<S, T> a, const int kchunk, const SweepGeom g, const unsigned step) {
    update_H_block<S, T, PIPE, SRM>(a, kchunk, g, blockIdx.x, blockIdx.y, blockIdx.z, step);
}

// ---------------------------------------------------------------------------------
// CG: H is read through L2 only -- the slab-ordered step (k_step_slabs) reads H that other
// SMs wrote in the same launch, which a stale L1 line could hide.  SH: the step has
// plane-wave sheets (a separate instantiation keeps the sheet tests out of the common case).
// li: the thread's lane within its row segment of g.lanes lanes (interior columns).
template <typename S, typename T, bool EDGE, bool CG = false, bool SH = false, bool MAT = false, bool PIPE = false,
          int SRM = 2>
__device__ __forceinline__ void e_column(const StepArgs<S, T>& a, const SweepGeom& g, const ESrc& src, const int j,
                                         const int i0, const bool act, const int kb, const int ke, const int li) {
    auto ldH = [](const S* p, T (&v)[Vec<T>::W]) {
        if constexpr (CG) Fld<S, T>::ldcg(p, v);
        else Fld<S, T>::ldg(p, v);
    };
    auto ldH1 = [](const S* p) -> T {
        if constexpr (CG) return T(to_c(ldcg1(p)));
        else return T(to_c(*p));
    };
    constexpr int W = Vec<T>::W;
    const int np = a.np, np2 = 2 * np;

    T idx[W];
#pragma unroll
    for (int e = 0; e < W; ++e) idx[e] = act ? __ldg(a.idx + i0 + e) : T(0);
    const T idy = __ldg(a.idy + j);
    const bool ypml = in_pml(j, a.NyT, np);
    const int jy = ypml ? slab_index(j, a.NyT, np) : 0;
    T yb = 1, yc = 0, yik = 1;
    if (ypml) { yb = __ldg(a.pbE[1] + j); yc = __ldg(a.pcE[1] + j); yik = __ldg(a.ik[1] + j); }
    const bool xpml = EDGE && act && (i0 < np || i0 + W > a.NxT - np);
    // (the gain state is written outside the act-guarded stores: inactive lanes never enter it)
    const bool grow = act && a.gain && j >= a.gj0 && j < a.gj0 + a.gY && i0 + W > a.gi0 && i0 < a.gi0 + a.gX;
    const bool plain_row = act && !ypml && !xpml && i0 >= 1 && i0 + W <= a.NxT;
    // Hz, Hy at i0-1 come from memory at the start of the row segment (whose lane also holds
    // the first interior vector) and for every edge column
    const bool pload = EDGE || li == 0;
    T* const Pcur = src.parity ? a.P1 : a.P0;
    T* const Pold = src.parity ? a.P0 : a.P1;  // holds P^{n-1}, receives P^{n+1}

    const size_t row = size_t(j) * a.NxP + i0;
    T hxm[W], hym[W];  // Hx, Hy at k-1
    RowIds<W> ids{};   // (MAT) material rows of the current plane, loaded one plane ahead
    if (act) {
        ldH(a.Hx + size_t(kb - 1) * a.plane + row, hxm);
        ldH(a.Hy + size_t(kb - 1) * a.plane + row, hym);
        if constexpr (MAT && !PIPE) ids.load(a.bidx + size_t(kb) * a.plane + row);
    } else {
#pragma unroll
        for (int e = 0; e < W; ++e) hxm[e] = hym[e] = T(0);
    }

    // PIPE (interior columns of k_update_E): the plane's vectors come from this thread's
    // shared-memory slots, filled by cp.async one plane ahead.
    extern __shared__ uint4 pipe_smem[];
    constexpr int NT = 32 * kBlockY, NV = EPipe<S>::kSlots, XS = EPipe<S>::kX, SB = EPipe<S>::SB;
    constexpr int NS = EPipe<S>::kStages;
    constexpr int VB = W * int(sizeof(S));                 // bytes of one field vector
    static_assert(VB <= SB && 2 * W <= SB, "a field vector and the row ids fill at most one slot");
    static_assert(!PIPE || MAT, "the staged E sweep takes the row-indexed material");
    constexpr int NB = sizeof(S) < 4 ? 4 : int(sizeof(S));  // x-neighbour copy (>= 4 bytes)
    constexpr int NE = NB / int(sizeof(S));                 // elements in it; the neighbour is the last
    const int tid = threadIdx.y * 32 + threadIdx.x;
    char* const pipe = reinterpret_cast<char*>(pipe_smem);
    auto slot = [&](int stg, int q) { return pipe + ((size_t(stg) * NV + q) * NT + tid) * SB; };
    auto issue = [&](int kk, int stg) {
        const size_t cc = size_t(kk) * a.plane + row;
        cp_async<VB, false>(slot(stg, 0), a.Ex + cc);
        cp_async<VB, false>(slot(stg, 1), a.Ey + cc);
        cp_async<VB, false>(slot(stg, 2), a.Ez + cc);
        cp_async<VB>(slot(stg, 3), a.Hx + cc);
        cp_async<VB>(slot(stg, 4), a.Hy + cc);
        cp_async<VB>(slot(stg, 5), a.Hz + cc);
        cp_async<VB>(slot(stg, 6), a.Hz + cc - a.NxP);
        cp_async<VB>(slot(stg, 7), a.Hx + cc - a.NxP);
        cp_async<2 * W>(slot(stg, 8), a.bidx + cc);
        if (pload && i0 > 0) {
            cp_async<NB>(slot(stg, XS), a.Hz + cc - NE);
            cp_async<NB>(slot(stg, XS) + SB / 2, a.Hy + cc - NE);
        }
    };
    if constexpr (PIPE) {
        // planes kb .. kb + NS - 2 in flight before the loop
#pragma unroll
        for (int q = 0; q < NS - 1; ++q) {
            if (act && kb + q < ke) issue(kb + q, q);
            cp_async_commit();
        }
    }

    for (int k = kb; k < ke; ++k) {
        const size_t c = size_t(k) * a.plane + row;
        T ex[W], ey[W], ez[W], bx[W], by[W], bz[W], hx[W], hy[W], hz[W], hzj[W], hxj[W];
        T hze = T(0), hye = T(0);
        if (PIPE && act) {
            // plane k + NS - 1 into the stage read last iteration (its contents are used), then
            // wait for this plane's copies
            if (k + NS - 1 < ke) issue(k + NS - 1, (k + NS - 1 - kb) & (NS - 1));
            cp_async_commit();
            cp_async_wait<NS - 1>();
            const int stg = (k - kb) & (NS - 1);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 0)), ex);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 1)), ey);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 2)), ez);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 3)), hx);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 4)), hy);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 5)), hz);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 6)), hzj);
            Fld<S, T>::ld(reinterpret_cast<const S*>(slot(stg, 7)), hxj);
            if constexpr (MAT) {
                RowIds<W> idk;
                const unsigned* w = reinterpret_cast<const unsigned*>(slot(stg, 8));
#pragma unroll
                for (int q = 0; q < W / 2; ++q) idk.w[q] = w[q];
                load_bE<MAT>(a, c, idk, bx, by, bz);
            }
            if (pload && i0 > 0) {
                const char* xs = slot(stg, XS);
                hze = T(to_c(reinterpret_cast<const S*>(xs)[NE - 1]));
                hye = T(to_c(reinterpret_cast<const S*>(xs + SB / 2)[NE - 1]));
            }
        } else if (act) {
            Fld<S, T>::ld(a.Ex + c, ex);
            Fld<S, T>::ld(a.Ey + c, ey);
            Fld<S, T>::ld(a.Ez + c, ez);
            load_bE<MAT>(a, c, ids, bx, by, bz);
            if constexpr (MAT) {
                if (k + 1 < ke) ids.load(a.bidx + c + a.plane);
            }
            ldH(a.Hx + c, hx);
            ldH(a.Hy + c, hy);
            ldH(a.Hz + c, hz);
            ldH(a.Hz + c - a.NxP, hzj);
            ldH(a.Hx + c - a.NxP, hxj);
            if (pload && i0 > 0) { hze = ldH1(a.Hz + c - 1); hye = ldH1(a.Hy + c - 1); }
        } else {
#pragma unroll
            for (int e = 0; e < W; ++e)
                ex[e] = ey[e] = ez[e] = bx[e] = by[e] = bz[e] = hx[e] = hy[e] = hz[e] = hzj[e] = hxj[e] = T(0);
        }
        const T idz = __ldg(a.idz + k);
        const bool zpml = in_pml(k + a.kz0, a.NzG, np);
        T zb = 1, zc = 0, zik = 1;
        size_t zs = 0, ys = 0;
        T pxy[W], pzy[W], pxz[W], pyz[W];  // psi Ex_y, Ez_y, Ex_z, Ey_z
        if (zpml) {
            zb = __ldg(a.pbE[2] + k); zc = __ldg(a.pcE[2] + k); zik = __ldg(a.ik[2] + k);
            zs = (size_t(slab_index(k + a.kz0, a.NzG, np)) * a.NyT + j) * a.NxP + i0;
            if (act) { Fld<S, T>::ld(a.psiE[1] + zs, pxz); Fld<S, T>::ld(a.psiE[2] + zs, pyz); }
        }
        if (ypml) {
            ys = (size_t(k) * np2 + jy) * a.NxP + i0;
            if (act) { Fld<S, T>::ld(a.psiE[0] + ys, pxy); Fld<S, T>::ld(a.psiE[5] + ys, pzy); }
        }
        T x3[W], x4[W];  // psi Ey_x, Ez_x
        if (xpml) xpsi_load<S, T>(a.psiE[3], a.psiE[4], a, k, j, i0, x3, x4);
        // x-neighbour at i0-1: the previous lane's last cell, or the loaded one
        T hzp = hze, hyp = hye;
        if (!EDGE) {
            const T sz = __shfl_up_sync(kFull, hz[W - 1], 1, g.lanes);
            const T sy = __shfl_up_sync(kFull, hy[W - 1], 1, g.lanes);
            if (!pload) { hzp = sz; hyp = sy; }
        }
        const bool gplane = grow && k >= a.gk0 && k < a.gk0 + a.gZ;
        if (plain_row && !zpml && !gplane && !src_in_vector<SH>(src, i0, j, k, W)) {
            e_plain<S, T, SRM>(a, c, ex, ey, ez, bx, by, bz, hx, hy, hz, hzj, hxj, hxm, hym, hzp, hyp, idx, idy, idz, src.step);
#pragma unroll
            for (int e = 0; e < W; ++e) { hxm[e] = hx[e]; hym[e] = hy[e]; }
            continue;
        }
#pragma unroll
        for (int e = 0; e < W; ++e) {
            const int i = i0 + e;
            if (i < 1 || i >= a.NxT) continue;  // x = 0 plane and padding never updated
            const T hzx = (e > 0) ? hz[e - 1] : hzp;
            const T hyx = (e > 0) ? hy[e - 1] : hyp;
            T dHz_dy = dq(hz[e], hzj[e], idy);
            T dHy_dz = dq(hy[e], hym[e], idz);
            T dHx_dz = dq(hx[e], hxm[e], idz);
            T dHz_dx = dq(hz[e], hzx, idx[e]);
            T dHy_dx = dq(hy[e], hyx, idx[e]);
            T dHx_dy = dq(hx[e], hxj[e], idy);
            if (ypml) {
                pxy[e] = psi_rec(yb, pxy[e], yc, dHz_dy); dHz_dy = psi_eff<S, T>(dHz_dy, yik, pxy[e], a.psc);
                pzy[e] = psi_rec(yb, pzy[e], yc, dHx_dy); dHx_dy = psi_eff<S, T>(dHx_dy, yik, pzy[e], a.psc);
            }
            if (zpml) {
                pxz[e] = psi_rec(zb, pxz[e], zc, dHy_dz); dHy_dz = psi_eff<S, T>(dHy_dz, zik, pxz[e], a.psc);
                pyz[e] = psi_rec(zb, pyz[e], zc, dHx_dz); dHx_dz = psi_eff<S, T>(dHx_dz, zik, pyz[e], a.psc);
            }
            if (xpml && in_pml(i, a.NxT, np)) {
                const T b = __ldg(a.pbE[0] + i), cc = __ldg(a.pcE[0] + i), ik = __ldg(a.ik[0] + i);
                x3[e] = psi_rec(b, x3[e], cc, dHz_dx);
                dHz_dx = psi_eff<S, T>(dHz_dx, ik, x3[e], a.psc);
                x4[e] = psi_rec(b, x4[e], cc, dHy_dx);
                dHy_dx = psi_eff<S, T>(dHy_dx, ik, x4[e], a.psc);
            }
            T Jx = 0, Jy = 0, Jz = 0;
            for (int s = 0; s < src.n; ++s) {
                if (src.si[s] == i && src.sj[s] == j && src.sk[s] == k) {
                    const T v = T(src.J[s]);
                    if (src.sc[s] == 0) Jx = add_rn(Jx, v);
                    else if (src.sc[s] == 1) Jy = add_rn(Jy, v);
                    else Jz = add_rn(Jz, v);
                }
            }
            if constexpr (SH) sheet_J(src, i, j, k, Jx, Jy, Jz);
            ex[e] = fma_rn(bx[e], sub_rn(sub_rn(dHz_dy, dHy_dz), Jx), ex[e]);
            ey[e] = fma_rn(by[e], sub_rn(sub_rn(dHx_dz, dHz_dx), Jy), ey[e]);
            // Two-level gain: polarization with E^n, E update with -dP/dt, populations with E^{n+1}.
            int r = -1;
            size_t gidx = 0;
            if (gplane && i >= a.gi0 && i < a.gi0 + a.gX) {
                gidx = (size_t(k - a.gk0) * a.gY + (j - a.gj0)) * a.gX + (i - a.gi0);
                r = a.greg[gidx];
            }
            if (r >= 0 && a.gcoef[r].active) {
                const GainCoef<T> g = a.gcoef[r];
                const T ez_old = ez[e];
                const T P = Pcur[gidx], Pp = Pold[gidx];
                T Nu = a.Nu[gidx], Ng = a.Ng[gidx];
                const T ng_frac = mul_rn(sub_rn(Ng, Nu), g.inv_N0);
                const T Pn = fma_rn(g.pa3, Pp, fma_rn(g.pa2, P, mul_rn(g.kapaN0, mul_rn(ng_frac, ez_old))));
                const T dPn = sub_rn(Pn, P);
                const T dP = mul_rn(dPn, g.inv_dt);
                ez[e] = fma_rn(bz[e], sub_rn(sub_rn(sub_rn(dHy_dx, dHx_dy), Jz), mul_rn(dP, g.dp_scale)), ez[e]);
                const T e_avg = mul_rn(T(0.5), add_rn(ez[e], ez_old));
                const T stim = mul_rn(mul_rn(mul_rn(e_avg, dPn), g.inv_dt), g.inv_hbar_omega);
                T dNu = fma_rn(-g.inv_tau, Nu, stim);
                T dNg = fma_rn(g.inv_tau, Nu, -stim);
                if (g.pump != T(0)) { dNu = fma_rn(g.pump, Ng, dNu); dNg = fma_rn(-g.pump, Ng, dNg); }
                Nu = fma_rn(g.dt, dNu, Nu);
                Ng = fma_rn(g.dt, dNg, Ng);
                Nu = fmax(T(0), Nu);
                Ng = fmax(T(0), Ng);
                if (g.clamp) {
                    const T tot = add_rn(Nu, Ng);
                    if (tot > T(1e-30)) { const T sc = div_rn(g.N0, tot); Nu = mul_rn(Nu, sc); Ng = mul_rn(Ng, sc); }
                    Nu = fmin(Nu, g.N0);
                    Ng = sub_rn(g.N0, Nu);
                }
                Pold[gidx] = Pn;
                a.Nu[gidx] = Nu;
                a.Ng[gidx] = Ng;
            } else {
                ez[e] = fma_rn(bz[e], sub_rn(sub_rn(dHy_dx, dHx_dy), Jz), ez[e]);
            }
        }
        if (act) {
            st_field<SRM>(a, a.Ex, c, ex, 0, src.step);
            st_field<SRM>(a, a.Ey, c, ey, 1, src.step);
            st_field<SRM>(a, a.Ez, c, ez, 2, src.step);
            if (zpml) { Fld<S, T>::st(a.psiE[1] + zs, pxz); Fld<S, T>::st(a.psiE[2] + zs, pyz); }
            if (ypml) { Fld<S, T>::st(a.psiE[0] + ys, pxy); Fld<S, T>::st(a.psiE[5] + ys, pzy); }
            if (xpml) xpsi_store<S, T>(a.psiE[3], a.psiE[4], a, k, j, i0, 1, a.NxT, x3, x4);
        }
#pragma unroll
        for (int e = 0; e < W; ++e) { hxm[e] = hx[e]; hym[e] = hy[e]; }
    }
}

template <typename S, typename T, bool CG = false, bool SH = false, bool MAT = false, bool PIPE = false, int SRM = 2>
__device__ __forceinline__ void update_E_block(const StepArgs<S, T>& a, const int kchunk, const ESrc& src,
                                               const SweepGeom& g, const int bx, const int by, const int bz) {
    constexpr int W = Vec<T>::W;
    if (*a.status) return;
    const int lane = threadIdx.x;
    const int kb = max(bz * kchunk, a.kE0);
    const int ke = min(bz * kchunk + kchunk, a.kE1);
    if (kb >= ke) return;
    if (bx < gxi_E<S>(g)) {
        // E is updated for rows 1 <= j < NyT.  A warp with no such row leaves as a whole; in a
        // warp that has one, the other rows stay in the loop as inactive lanes on row 1.
        const InteriorLane il = interior_lane(g, by, lane);
        const int R = 32 / g.lanes;
        const int w0 = (by * kBlockY + int(threadIdx.y)) * R;
        if (w0 + R - 1 < 1 || w0 >= a.NyT) return;
        const bool row_ok = il.j >= 1 && il.j < a.NyT;
        const int i0 = g.xi0 + (bx * g.lanes + il.li) * W;
        e_column<S, T, false, CG, SH, MAT, PIPE, SRM>(a, g, src, row_ok ? il.j : 1, i0, row_ok && i0 < g.xi1, kb, ke, il.li);
    } else {
        const int t = threadIdx.y * 32 + lane;
        const int rr = t / g.ne, v = t - rr * g.ne;
        const int j = by * g.er + rr;
        if (rr >= g.er || j < 1 || j >= a.NyT) return;
        const int i0 = v < g.nl ? v * W : g.xi1 + (v - g.nl) * W;
        if (i0 >= a.NxT) return;
        e_column<S, T, true, CG, SH, MAT, false, SRM>(a, g, src, j, i0, true, kb, ke, 0);
    }
}

// PIPE: interior columns stage their planes in shared memory (EPipe<S>::bytes() dynamic).
template <typename S, typename T, bool SH = false, bool MAT = false, bool PIPE = false, int SRM = 2>
__global__ void __launch_bounds__(32 * kBlockY, 2)
k_update_E(const StepArgs<S, T> a, const int kchunk, const ESrc src, const SweepGeom g) {
    update_E_block<S, T, false, SH, MAT, PIPE, SRM>(a, kchunk, src, g, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------------
// Slab-ordered step: one persistent launch does the whole H + E step in slabs of P planes,
// in the order H(0), H(1), E(0), H(2), E(1), ..., E(n-1), handed out through a global work
// counter.  The schedule is a valid order for the Yee step: H(k) reads E(k), E(k+1) (not yet
// updated: E of a slab is written only after H of that slab and of the slab below are done),
// E(k) reads H(k), H(k-1) (done: E(s) waits for H(s) and H(s-1)).  E(s) runs about one slab
// after H(s), while the E and H planes it reads are still in L2, so a cell costs DRAM bytes
// for E, H and bE once each instead of E and H twice.  Blocks wait only on work handed out
// before theirs (already running), so the waits always end; each is bounded all the same
// (wait_ns of %globaltimer, 2 s by default), after which the block flags the status word and
// leaves.  An E tile also waits while the hold word (the counter after the per-slab counts)
// is nonzero; the host clears it before every launch, and sets it only to make the waits
// run out on purpose (the bounded-wait test).
struct SlabPlan {
    int P;          // planes per slab
    int nslab;
    int gxH, nH;    // H tiles per slab: gxH columns x (nH / gxH) row groups
    int gxE, nE;
    unsigned long long wait_ns;  // bound on one dependency wait
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// One resident block per SM: the H and E block code together need more than 128 registers.
template <typename S, typename T, bool SH = false, bool MAT = false>
__global__ void __launch_bounds__(32 * kBlockY, 1)
k_step_slabs(const StepArgs<S, T> a, const ESrc src, const SweepGeom g, const SlabPlan p, unsigned* ctr,
             unsigned* status_w) {
    __shared__ int item_s;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const long long total = (long long)p.nslab * (p.nH + p.nE);
    unsigned* const hdone = ctr + 1;
    const unsigned* const hold = ctr + 1 + p.nslab;
    for (;;) {
        if (tid == 0) item_s = int(atomicAdd(ctr, 1u));
        __syncthreads();
        const long long it = item_s;
        __syncthreads();
        if (it >= total) return;
        // order: H(0) | H(1) E(0) | H(2) E(1) | ... | E(n-1)
        int slab, r;
        bool isH;
        if (it < p.nH) { isH = true; slab = 0; r = int(it); }
        else {
            const long long q = it - p.nH;
            const int pair = int(q / (p.nH + p.nE)), r2 = int(q % (p.nH + p.nE));
            if (pair < p.nslab - 1 && r2 < p.nH) { isH = true; slab = pair + 1; r = r2; }
            else { isH = false; slab = pair; r = pair < p.nslab - 1 ? r2 - p.nH : r2; }
        }
        if (isH) {
            update_H_block<S, T>(a, p.P, g, r % p.gxH, r / p.gxH, slab, src.step);
            __threadfence();  // this thread's H stores, before the block signals
            __syncthreads();
            if (tid == 0) atomicAdd(hdone + slab, 1u);
        } else {
            bool ok = true;
            if (tid == 0) {
                const unsigned long long t0 = global_ns();
                while (ld_acquire(hdone + slab) < unsigned(p.nH) ||
                       (slab > 0 && ld_acquire(hdone + slab - 1) < unsigned(p.nH)) || ld_acquire(hold) != 0u) {
                    if (global_ns() - t0 > p.wait_ns) { ok = false; break; }
                }
            }
            if (!__syncthreads_and(ok)) {
                if (tid == 0) atomicOr(status_w, kStatusTimeout);
                return;
            }
            update_E_block<S, T, true, SH, MAT>(a, p.P, src, g, r % p.gxE, r / p.gxE, slab);
            __syncthreads();
        }
    }
}

}  // namespace fdtdk
