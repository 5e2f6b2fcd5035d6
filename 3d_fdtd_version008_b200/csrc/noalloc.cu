// noalloc.cu -- field scan that allocates no device memory (fdtd_field_scan_noalloc).
//
// The stability monitor of the stepper (k_monitor_reduce, solver.cu) scans the E and H
// fields for max |E| and non-finite values into an accumulator that the handle obtains
// from cudaMalloc.  Some callers of this code cannot allocate device memory at the time
// they want such a scan: a host application that embeds the stepper inside its own memory
// pool or arena (which owns every byte of the device and forbids side allocations), a
// callback that runs while the caller holds its allocator's lock, or code running under a
// watchdog that treats any cudaMalloc/cudaFree as a fault.  This file gives them the same
// scan with its scratch in a fixed, file-scope device array: the caller passes the field
// arrays and a 16-byte device output, nothing is allocated.
//
// Scratch: one partial record per block of kScanTile cells, kScanMaxBlocks records
// (256 KiB), so at most kScanMaxBlocks * kScanTile = 268,435,456 cells per call; larger
// scans are refused with FDTD_ERR_INVALID.  Every GPU that loads the library keeps the
// array until the process exits.  Each call writes every record that it later reads, so
// nothing needs clearing between calls; all calls share the one array, so calls that
// overlap on the GPU (different streams, or different host threads on one device) race.
//
// The scratch address of a device is looked up once, at the first call on that device, and
// kept for the life of the process; a caller that resets the device (cudaDeviceReset)
// reloads the module, which may move the array, so the entry point must not be used across a
// device reset.  Only FP32 and FP64 fields are scanned (16-bit storage keeps a field scale
// that this entry point does not take).
#include "../../include/fdtd_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

namespace fdtd_internal {
void set_global_error(const std::string& msg);  // solver.cu: message of fdtd_last_error(NULL)
}

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 64;
constexpr long long kScanTile = (long long)kScanThreads * kScanPerThread;  // cells per block
constexpr int kScanMaxBlocks = 16384;
constexpr int kMaxDevices = 64;

struct ScanPartial {
    double max_e;    // max |Ex|,|Ey|,|Ez| over the block's cells whose three E values are finite
    unsigned flags;  // bit0: non-finite E, bit1: non-finite H
    unsigned pad;
};

// The scan's scratch.  Host code must not pass this name to a kernel (it is a host-side
// stand-in); the host uses the address from cudaGetSymbolAddress below.
static __device__ __align__(256) ScanPartial g_scan_scratch[kScanMaxBlocks];

__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned warp_or(unsigned v) {
    for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block reduction of (max, flags); thread 0 returns the block's values.
__device__ void block_reduce(double& m, unsigned& fl) {
    __shared__ double sm[kScanThreads / 32];
    __shared__ unsigned sf[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    m = warp_max_d(m);
    fl = warp_or(fl);
    if (lane == 0) { sm[wid] = m; sf[wid] = fl; }
    __syncthreads();
    if (wid == 0) {
        m = lane < kScanThreads / 32 ? sm[lane] : 0.0;
        fl = lane < kScanThreads / 32 ? sf[lane] : 0u;
        m = warp_max_d(m);
        fl = warp_or(fl);
    }
}

// Same per-cell test as the stepper's monitor scan: a cell contributes to max |E| only
// when its three E values are finite; any non-finite E or H value sets its flag.
template <typename T>
__global__ void __launch_bounds__(kScanThreads)
k_field_scan_partial(const T* __restrict__ ex, const T* __restrict__ ey, const T* __restrict__ ez,
                     const T* __restrict__ hx, const T* __restrict__ hy, const T* __restrict__ hz, long long n,
                     ScanPartial* __restrict__ part) {
    const long long b0 = (long long)blockIdx.x * kScanTile;
    const long long b1 = b0 + kScanTile < n ? b0 + kScanTile : n;
    double m = 0.0;
    unsigned fl = 0;
    for (long long t = b0 + threadIdx.x; t < b1; t += kScanThreads) {
        const double vx = double(ex[t]), vy = double(ey[t]), vz = double(ez[t]);
        if (!isfinite(vx) || !isfinite(vy) || !isfinite(vz)) fl |= 1u;
        else m = fmax(m, fmax(fabs(vx), fmax(fabs(vy), fabs(vz))));
        if (!isfinite(double(hx[t])) || !isfinite(double(hy[t])) || !isfinite(double(hz[t]))) fl |= 2u;
    }
    block_reduce(m, fl);
    if (threadIdx.x == 0) {
        part[blockIdx.x].max_e = m;
        part[blockIdx.x].flags = fl;
        part[blockIdx.x].pad = 0u;
    }
}

__global__ void __launch_bounds__(kScanThreads)
k_field_scan_finish(const ScanPartial* __restrict__ part, int nblocks, fdtd_field_scan_v1* __restrict__ out) {
    double m = 0.0;
    unsigned fl = 0;
    for (int b = threadIdx.x; b < nblocks; b += kScanThreads) {
        m = fmax(m, part[b].max_e);
        fl |= part[b].flags;
    }
    block_reduce(m, fl);
    if (threadIdx.x == 0) {
        out->max_E = m;
        out->nan_flags = fl;
        out->reserved = 0u;
    }
}

// Device address of the scratch, looked up once per device with that device current.
std::mutex g_scan_mu;
void* g_scan_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
    fdtd_internal::set_global_error(msg);
    return code;
}

}  // namespace

extern "C" int fdtd_field_scan_noalloc(int precision, const void* ex, const void* ey, const void* ez, const void* hx,
                                       const void* hy, const void* hz, uint64_t n, fdtd_field_scan_v1* out,
                                       void* stream) {
    if (precision != FDTD_PREC_FP32 && precision != FDTD_PREC_FP64)
        return fail(FDTD_ERR_INVALID, "fdtd_field_scan_noalloc: precision must be FDTD_PREC_FP32 or FDTD_PREC_FP64");
    if (!ex || !ey || !ez || !hx || !hy || !hz || !out)
        return fail(FDTD_ERR_INVALID, "fdtd_field_scan_noalloc: null field or output pointer");
    if (n == 0) return fail(FDTD_ERR_INVALID, "fdtd_field_scan_noalloc: empty scan (n = 0)");
    if (n > FDTD_FIELD_SCAN_MAX_CELLS)
        return fail(FDTD_ERR_INVALID, "fdtd_field_scan_noalloc: " + std::to_string(n) +
                                          " cells exceed the scratch limit of " +
                                          std::to_string((unsigned long long)FDTD_FIELD_SCAN_MAX_CELLS) +
                                          " cells per call; scan in pieces");
    // An error left pending by earlier work of the caller is reported as such, not as a
    // failure of this scan, and is left in place for the caller.
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return fail(FDTD_ERR_CUDA, std::string("fdtd_field_scan_noalloc: a CUDA error was already pending before the "
                                               "call (nothing launched): ") + cudaGetErrorString(e));
    int dev = -1;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(FDTD_ERR_NO_DEVICE, std::string("fdtd_field_scan_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(FDTD_ERR_UNSUPPORTED, "fdtd_field_scan_noalloc: device ordinal out of range");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scan_mu);
        if (!g_scan_addr[dev]) {
            // first call on this device: resolve the scratch array's device address
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_scan_scratch);
            if (e != cudaSuccess || !p)
                return fail(FDTD_ERR_CUDA, std::string("fdtd_field_scan_noalloc: cudaGetSymbolAddress: ") +
                                               cudaGetErrorString(e));
            g_scan_addr[dev] = p;
        }
        scratch = g_scan_addr[dev];
    }
    const int nblocks = int((n + kScanTile - 1) / kScanTile);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    if (precision == FDTD_PREC_FP32)
        k_field_scan_partial<float><<<nblocks, kScanThreads, 0, st>>>(
            static_cast<const float*>(ex), static_cast<const float*>(ey), static_cast<const float*>(ez),
            static_cast<const float*>(hx), static_cast<const float*>(hy), static_cast<const float*>(hz),
            (long long)n, part);
    else
        k_field_scan_partial<double><<<nblocks, kScanThreads, 0, st>>>(
            static_cast<const double*>(ex), static_cast<const double*>(ey), static_cast<const double*>(ez),
            static_cast<const double*>(hx), static_cast<const double*>(hy), static_cast<const double*>(hz),
            (long long)n, part);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(FDTD_ERR_CUDA, std::string("fdtd_field_scan_noalloc: launch of the partial scan: ") + cudaGetErrorString(e));
    k_field_scan_finish<<<1, kScanThreads, 0, st>>>(part, nblocks, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(FDTD_ERR_CUDA, std::string("fdtd_field_scan_noalloc: launch of the final reduction: ") + cudaGetErrorString(e));
    return FDTD_OK;
}
