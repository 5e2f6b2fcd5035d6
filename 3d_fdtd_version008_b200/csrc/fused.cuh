// fused.cuh -- one-launch-per-step Yee update (H then E) with TMA-staged planes.
//
// Each block owns a TX x TY tile of the (x, y) plane and marches in +z through a chunk of
// planes.  Per plane it needs E^n(k), E^n(k+1), H^{n-1/2}(k) and bE(k): one elected thread
// streams the E and H planes (tile + halo) and the bE tile into a shared-memory ring with
// cp.async.bulk.tensor (TMA) DEPTH planes ahead of the compute, completion tracked by
// mbarriers.  From shared memory the block
//   1. computes H^{n+1/2}(k) on the tile plus a ring at x0-W..x0-1 and y0-1 (the ring is
//      recomputed here instead of exchanged, so E needs no data from other blocks),
//   2. computes E^{n+1}(k-1) on the tile from H^{n+1/2}(k-1) and H^{n+1/2}(k-2), kept in
//      shared memory, with the CPML psi recursion, two-level gain (P, populations) and the
//      point sources as in k_update_E.
// The z loop is skewed (H on plane kh, E on plane kh-1 in the same iteration) so that one
// block-wide barrier per plane suffices.  Threads are register-blocked: each owns a group
// of W = 16 / sizeof(T) consecutive x cells and moves them with 128-bit shared-memory and
// global accesses; only the x-neighbour across a group edge is a scalar load.
//
// Fields are double-buffered (read set src, write set dst, swapped every step), and so is
// psi_H, because ring cells are computed from values that their owning block overwrites in
// the same launch.  Cells that the reference never updates are written back unchanged.
// Every mbarrier wait is bounded (2 s of %globaltimer): on expiry the block records a
// timeout in the status word, waits (bounded again) for the copies it still has in flight
// and exits.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.cuh"

namespace fdtdk {

// Tile / pipeline shape: TX x TY cells per block (TX a multiple of 16 / sizeof(T)),
// THREADS threads, DEPTH stages in flight ahead of the one being consumed.
template <typename T, int TX_, int TY_, int THREADS_, int DEPTH_, int MINB_>
struct FusedShape {
    static constexpr int TX = TX_, TY = TY_, THREADS = THREADS_, DEPTH = DEPTH_, MINB = MINB_;
    static constexpr int W = 16 / int(sizeof(T));  // cells per thread group; also the x halo
    static constexpr int GX = TX / W;              // groups per tile row
    static_assert(TX % W == 0, "tile width must be a whole number of groups");
};

struct FusedMaps {
    CUtensorMap E[3];  // source E (x,y,z), box (TX + 2W) x (TY + 2) x 1 at (x0 - W, y0 - 1)
    CUtensorMap H[3];  // source H, same box
    CUtensorMap B[3];  // bE, box TX x TY x 1 at (x0, y0)
};

template <typename T>
struct FusedArgs {
    StepArgs<T> a;          // geometry, coefficients, psi_E, gain (field pointers unused)
    T *dE[3], *dH[3];       // destination fields
    const T *psiHs[6];      // psi_H read set
    T *psiHd[6];            // psi_H write set
    unsigned* status_w;     // writable status word (timeout flag)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}


// Bounded wait: false once kWaitNs of wall time have passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int q = 0; q < 64; ++q)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Shared-memory layout of one block.  Every TMA destination box starts on a 128-byte
// boundary; rows of every array are multiples of 16 bytes so group accesses are 128-bit.
// Iteration t reads E planes kh-1..kh+1, H_old(kh), bE(kh-1), H_new(kh-1), H_new(kh-2) and
// writes H_new(kh) (kh = ks + t).
template <typename T, typename Shape>
struct FusedSmem {
    static constexpr int TX = Shape::TX, TY = Shape::TY, W = Shape::W, D = Shape::DEPTH;
    static constexpr int PX = TX + 2 * W;    // E/H box row (x0-W .. x0+TX+W-1)
    static constexpr int PY = TY + 2;        // E/H box rows (y0-1 .. y0+TY)
    static constexpr int HX = TX + W;        // H_new row (x0-W .. x0+TX-1)
    static constexpr int HY = TY + 1;        // H_new rows (y0-1 .. y0+TY-1)
    static constexpr int NE = 3 + D;         // E planes kh-1, kh, kh+1 in use + D in flight
    static constexpr int NH = 1 + D;         // H_old(kh) + D in flight
    static constexpr int NB = 2 + D;         // bE(kh-1), bE(kh) + D in flight; also the barrier ring
    static constexpr int BOX = int(((PX * PY * sizeof(T) + 127) / 128) * 128 / sizeof(T));
    static constexpr int BBOX = int(((TX * TY * sizeof(T) + 127) / 128) * 128 / sizeof(T));
    alignas(128) T E[NE][3][BOX];
    alignas(128) T H[NH][3][BOX];
    alignas(128) T B[NB][3][BBOX];
    alignas(128) T Hn[3][3][HY * HX];
    alignas(8) uint64_t full[NB];
    alignas(8) uint64_t pre;  // first E plane of the chunk
    static constexpr unsigned kEBox = 3u * PY * PX * sizeof(T);
    static constexpr unsigned kStageBytes = 2u * kEBox + 3u * TY * TX * sizeof(T);
};

template <typename T, typename Shape>
__global__ void __launch_bounds__(Shape::THREADS, Shape::MINB)
k_step_fused(const __grid_constant__ FusedMaps maps, const FusedArgs<T> f, const int kchunk, const ESrc src) {
    using S = FusedSmem<T, Shape>;
    using V = Vec<T>;
    constexpr int TX = S::TX, TY = S::TY, W = S::W, PX = S::PX, HX = S::HX;
    constexpr int NE = S::NE, NH = S::NH, NB = S::NB, D = S::D;
    constexpr int GX = Shape::GX;
    constexpr int HT = (GX + 1) * (TY + 1);  // H tasks: groups -1..GX-1, rows y0-1..y0+TY-1
    constexpr int ET = GX * TY;              // E tasks: groups 0..GX-1, rows y0..y0+TY-1
    static_assert(HT <= Shape::THREADS && ET <= Shape::THREADS, "one task of each kind per thread");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);
    const StepArgs<T>& a = f.a;
    if (*a.status) return;
    // TMA destinations need a 128-byte aligned base; refuse (never copy) if it is not.
    if (smem_u32(smem_raw) & 127u) {
        if (threadIdx.x == 0) atomicOr(f.status_w, kStatusTimeout);
        return;
    }

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int k0 = blockIdx.z * kchunk;
    const int k1 = min(k0 + kchunk, a.NzT);
    const int ks = max(k0 - 1, 0);  // first H plane (k0-1 is recomputed, not stored)
    const int nit = k1 - ks;        // H planes ks..k1-1
    const int np = a.np, np2 = 2 * np;

    // ---- this thread's H task (group hg, row hr) and E task (group eg, row er)
    const bool has_h = tid < HT, has_e = tid < ET;
    const int hg = tid % (GX + 1) - 1, hr = tid / (GX + 1);
    const int hi0 = x0 + W * hg, hj = y0 - 1 + hr;
    const int eg = tid % GX, er = tid / GX;
    const int ei0 = x0 + W * eg, ej = y0 + er;
    const bool h_row = has_h && hj >= 0 && hj < a.NyT - 1;         // H updated on this row
    // stored by this block: own rows/groups inside the padded array (the last x tile can
    // extend past the padded row length NxP; those groups are never stored)
    const bool h_own = has_h && hg >= 0 && hr >= 1 && hj < a.NyT && x0 + W * hg < a.NxP;
    const bool e_row = has_e && ej >= 1 && ej < a.NyT;              // E updated on this row
    const bool e_own = has_e && ej < a.NyT && x0 + W * eg < a.NxP;
    T h_idx[W], e_idx[W];
#pragma unroll
    for (int e = 0; e < W; ++e) {
        const int ih = hi0 + e, ie = ei0 + e;
        h_idx[e] = (h_row && ih >= 0 && ih < a.NxT) ? __ldg(a.idx + ih) : T(0);
        e_idx[e] = (e_row && ie < a.NxT) ? __ldg(a.idx + ie) : T(0);
    }
    const T h_idy = h_row ? __ldg(a.idy + hj) : T(0);
    const T e_idy = e_row ? __ldg(a.idy + ej) : T(0);
    const bool h_ypml = h_row && in_pml(hj, a.NyT, np);
    const bool e_ypml = e_row && in_pml(ej, a.NyT, np);
    const bool h_xpml = h_row && (hi0 < np || hi0 + W > a.NxT - np);
    const bool e_xpml = e_row && (ei0 < np || ei0 + W > a.NxT - np);
    const bool e_grow = e_row && a.gain && ej >= a.gj0 && ej < a.gj0 + a.gY && ei0 + W > a.gi0 && ei0 < a.gi0 + a.gX;
    bool e_src = false;
    for (int q = 0; q < src.n; ++q)
        e_src |= (src.sj[q] == ej && src.si[q] >= ei0 && src.si[q] < ei0 + W);
    e_src = e_src && e_row;

    if (tid == 0) {
        for (int q = 0; q < NB; ++q) mbar_init(&sm.full[q], 1);
        mbar_init(&sm.pre, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // Stage t: E(ks+t+1) -> E slot (t+1)%NE, H(ks+t) -> H slot t%NH, bE(ks+t) -> B slot t%NB.
    auto issue_stage = [&](int t) {
        const int k = ks + t;
        uint64_t* bar = &sm.full[t % NB];
        fence_proxy_async();
        mbar_expect_tx(bar, S::kStageBytes);
        for (int c = 0; c < 3; ++c) {
            tma_load_3d(&sm.E[(t + 1) % NE][c][0], &maps.E[c], x0 - W, y0 - 1, k + 1, bar);
            tma_load_3d(&sm.H[t % NH][c][0], &maps.H[c], x0 - W, y0 - 1, k, bar);
            tma_load_3d(&sm.B[t % NB][c][0], &maps.B[c], x0, y0, k, bar);
        }
    };
    bool ok = true;
    if (tid == 0) {
        fence_proxy_async();
        mbar_expect_tx(&sm.pre, S::kEBox);
        for (int c = 0; c < 3; ++c) tma_load_3d(&sm.E[0][c][0], &maps.E[c], x0 - W, y0 - 1, ks, &sm.pre);
        for (int t = 0; t < D && t < nit; ++t) issue_stage(t);
        ok = mbar_wait(&sm.pre, 0);
    }
    ok = __syncthreads_and(ok);
    if (ok) mbar_try_wait(&sm.pre, 0);  // acquire: the first E plane is visible to this thread
    int consumed = 0;                   // stages waited on

    const T bH = a.bH;
    const T* Pcur = src.parity ? a.P1 : a.P0;
    T* Pold = src.parity ? a.P0 : a.P1;
    for (int t = 0; t <= nit; ++t) {
        // One barrier per iteration: stage t has landed (thread 0 polls, the barrier
        // broadcasts a block-uniform verdict) and every thread is done with iteration t-1,
        // whose buffers the next copies may reuse (ring sizes: E D+3, H D+1, bE D+2).
        bool got = true;
        if (tid == 0 && t < nit) got = mbar_wait(&sm.full[t % NB], unsigned((t / NB) & 1));
        ok = __syncthreads_and(ok && got);
        if (!ok) break;
        if (t < nit) {
            mbar_try_wait(&sm.full[t % NB], unsigned((t / NB) & 1));  // acquire for this thread
            consumed = t + 1;
        }
        if (tid == 0 && t + D < nit) issue_stage(t + D);
        const int kh = ks + t;

        // ---------------- H^{n+1/2} on plane kh: group hg of row hj
        if (t < nit && has_h) {
            const int e0 = t % NE, e1 = (t + 1) % NE, hs = t % NH;
            const int o = hr * PX + W + W * hg;  // box offset of the group's first cell
            T hx[W], hy[W], hz[W];
            V::ld(&sm.H[hs][0][o], hx);
            V::ld(&sm.H[hs][1][o], hy);
            V::ld(&sm.H[hs][2][o], hz);
            if (h_row && kh < a.NzT - 1) {
                T ex[W], ey[W], ez[W], exj[W], ezj[W], ex1[W], ey1[W];
                V::ld(&sm.E[e0][0][o], ex);
                V::ld(&sm.E[e0][1][o], ey);
                V::ld(&sm.E[e0][2][o], ez);
                V::ld(&sm.E[e0][0][o + PX], exj);
                V::ld(&sm.E[e0][2][o + PX], ezj);
                V::ld(&sm.E[e1][0][o], ex1);
                V::ld(&sm.E[e1][1][o], ey1);
                const T eyn = sm.E[e0][1][o + W], ezn = sm.E[e0][2][o + W];
                const T idz = __ldg(a.idz + kh);
                const bool zpml = in_pml(kh, a.NzT, np);
                const bool own = h_own && kh >= k0;
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    const int i = hi0 + e;
                    if (i < 0 || i >= a.NxT - 1) continue;
                    const T eyx = e < W - 1 ? ey[e + 1] : eyn;
                    const T ezx = e < W - 1 ? ez[e + 1] : ezn;
                    T dEz_dy = (ezj[e] - ez[e]) * h_idy;
                    T dEy_dz = (ey1[e] - ey[e]) * idz;
                    T dEx_dz = (ex1[e] - ex[e]) * idz;
                    T dEz_dx = (ezx - ez[e]) * h_idx[e];
                    T dEy_dx = (eyx - ey[e]) * h_idx[e];
                    T dEx_dy = (exj[e] - ex[e]) * h_idy;
                    if (h_ypml) {
                        const size_t ys = (size_t(kh) * np2 + slab_index(hj, a.NyT, np)) * a.NxP + i;
                        const T b = __ldg(a.pbH[1] + hj), cc = __ldg(a.pcH[1] + hj), ik = __ldg(a.ik[1] + hj);
                        const T p0 = b * f.psiHs[0][ys] + cc * dEz_dy;
                        const T p5 = b * f.psiHs[5][ys] + cc * dEx_dy;
                        if (own) { f.psiHd[0][ys] = p0; f.psiHd[5][ys] = p5; }
                        dEz_dy = dEz_dy * ik + p0;
                        dEx_dy = dEx_dy * ik + p5;
                    }
                    if (zpml) {
                        const size_t zs = (size_t(slab_index(kh, a.NzT, np)) * a.NyT + hj) * a.NxP + i;
                        const T b = __ldg(a.pbH[2] + kh), cc = __ldg(a.pcH[2] + kh), ik = __ldg(a.ik[2] + kh);
                        const T p1 = b * f.psiHs[1][zs] + cc * dEy_dz;
                        const T p2 = b * f.psiHs[2][zs] + cc * dEx_dz;
                        if (own) { f.psiHd[1][zs] = p1; f.psiHd[2][zs] = p2; }
                        dEy_dz = dEy_dz * ik + p1;
                        dEx_dz = dEx_dz * ik + p2;
                    }
                    if (h_xpml && in_pml(i, a.NxT, np)) {
                        const size_t xs = (size_t(kh) * a.NyT + hj) * np2 + slab_index(i, a.NxT, np);
                        const T b = __ldg(a.pbH[0] + i), cc = __ldg(a.pcH[0] + i), ik = __ldg(a.ik[0] + i);
                        const T p3 = b * f.psiHs[3][xs] + cc * dEz_dx;
                        const T p4 = b * f.psiHs[4][xs] + cc * dEy_dx;
                        if (own) { f.psiHd[3][xs] = p3; f.psiHd[4][xs] = p4; }
                        dEz_dx = dEz_dx * ik + p3;
                        dEy_dx = dEy_dx * ik + p4;
                    }
                    hx[e] = hx[e] - bH * (dEz_dy - dEy_dz);
                    hy[e] = hy[e] - bH * (dEx_dz - dEz_dx);
                    hz[e] = hz[e] - bH * (dEy_dx - dEx_dy);
                }
            }
            const int on = hr * HX + W * (hg + 1);
            V::st(&sm.Hn[kh % 3][0][on], hx);
            V::st(&sm.Hn[kh % 3][1][on], hy);
            V::st(&sm.Hn[kh % 3][2][on], hz);
            if (h_own && kh >= k0) {
                const size_t g = size_t(kh) * a.plane + size_t(hj) * a.NxP + hi0;
                V::st(f.dH[0] + g, hx);
                V::st(f.dH[1] + g, hy);
                V::st(f.dH[2] + g, hz);
            }
        }

        // ---------------- E^{n+1} on plane ke = kh - 1: group eg of row ej
        const int ke = kh - 1;
        if (t >= 1 && ke >= k0 && e_own) {
            const int ee = (t - 1) % NE, bs = (t - 1) % NB, hn = ke % 3, hp = (ke + 2) % 3;
            const int oe = (er + 1) * PX + W + W * eg;     // E box offset of the group
            const int on = (er + 1) * HX + W * (eg + 1);   // H_new offset of the group
            const int ob = er * TX + W * eg;               // bE box offset
            T ex[W], ey[W], ez[W];
            V::ld(&sm.E[ee][0][oe], ex);
            V::ld(&sm.E[ee][1][oe], ey);
            V::ld(&sm.E[ee][2][oe], ez);
            if (e_row && ke >= 1) {
                T Hx[W], Hy[W], Hz[W], Hzj[W], Hxj[W], Hxk[W], Hyk[W], bx[W], by[W], bz[W];
                V::ld(&sm.Hn[hn][0][on], Hx);
                V::ld(&sm.Hn[hn][1][on], Hy);
                V::ld(&sm.Hn[hn][2][on], Hz);
                V::ld(&sm.Hn[hn][2][on - HX], Hzj);
                V::ld(&sm.Hn[hn][0][on - HX], Hxj);
                V::ld(&sm.Hn[hp][0][on], Hxk);
                V::ld(&sm.Hn[hp][1][on], Hyk);
                V::ld(&sm.B[bs][0][ob], bx);
                V::ld(&sm.B[bs][1][ob], by);
                V::ld(&sm.B[bs][2][ob], bz);
                const T Hzp = sm.Hn[hn][2][on - 1], Hyp = sm.Hn[hn][1][on - 1];
                const T idz = __ldg(a.idz + ke);
                const bool zpml = in_pml(ke, a.NzT, np);
                const bool gplane = e_grow && ke >= a.gk0 && ke < a.gk0 + a.gZ;
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    const int i = ei0 + e;
                    if (i < 1 || i >= a.NxT) continue;
                    const T Hzx = e > 0 ? Hz[e - 1] : Hzp;
                    const T Hyx = e > 0 ? Hy[e - 1] : Hyp;
                    T dHz_dy = (Hz[e] - Hzj[e]) * e_idy;
                    T dHy_dz = (Hy[e] - Hyk[e]) * idz;
                    T dHx_dz = (Hx[e] - Hxk[e]) * idz;
                    T dHz_dx = (Hz[e] - Hzx) * e_idx[e];
                    T dHy_dx = (Hy[e] - Hyx) * e_idx[e];
                    T dHx_dy = (Hx[e] - Hxj[e]) * e_idy;
                    if (e_ypml) {
                        const size_t ys = (size_t(ke) * np2 + slab_index(ej, a.NyT, np)) * a.NxP + i;
                        const T b = __ldg(a.pbE[1] + ej), cc = __ldg(a.pcE[1] + ej), ik = __ldg(a.ik[1] + ej);
                        T p = b * a.psiE[0][ys] + cc * dHz_dy; a.psiE[0][ys] = p; dHz_dy = dHz_dy * ik + p;
                        p = b * a.psiE[5][ys] + cc * dHx_dy; a.psiE[5][ys] = p; dHx_dy = dHx_dy * ik + p;
                    }
                    if (zpml) {
                        const size_t zs = (size_t(slab_index(ke, a.NzT, np)) * a.NyT + ej) * a.NxP + i;
                        const T b = __ldg(a.pbE[2] + ke), cc = __ldg(a.pcE[2] + ke), ik = __ldg(a.ik[2] + ke);
                        T p = b * a.psiE[1][zs] + cc * dHy_dz; a.psiE[1][zs] = p; dHy_dz = dHy_dz * ik + p;
                        p = b * a.psiE[2][zs] + cc * dHx_dz; a.psiE[2][zs] = p; dHx_dz = dHx_dz * ik + p;
                    }
                    if (e_xpml && in_pml(i, a.NxT, np)) {
                        const size_t xs = (size_t(ke) * a.NyT + ej) * np2 + slab_index(i, a.NxT, np);
                        const T b = __ldg(a.pbE[0] + i), cc = __ldg(a.pcE[0] + i), ik = __ldg(a.ik[0] + i);
                        T p = b * a.psiE[3][xs] + cc * dHz_dx; a.psiE[3][xs] = p; dHz_dx = dHz_dx * ik + p;
                        p = b * a.psiE[4][xs] + cc * dHy_dx; a.psiE[4][xs] = p; dHy_dx = dHy_dx * ik + p;
                    }
                    T Jx = 0, Jy = 0, Jz = 0;
                    if (e_src) {
                        for (int q = 0; q < src.n; ++q) {
                            if (src.si[q] == i && src.sj[q] == ej && src.sk[q] == ke) {
                                const T v = T(src.J[q]);
                                if (src.sc[q] == 0) Jx += v;
                                else if (src.sc[q] == 1) Jy += v;
                                else Jz += v;
                            }
                        }
                    }
                    if (src.ns) sheet_J(src, i, ej, ke, Jx, Jy, Jz);
                    ex[e] = ex[e] + bx[e] * ((dHz_dy - dHy_dz) - Jx);
                    ey[e] = ey[e] + by[e] * ((dHx_dz - dHz_dx) - Jy);
                    int r = -1;
                    size_t gidx = 0;
                    if (gplane && i >= a.gi0 && i < a.gi0 + a.gX) {
                        gidx = (size_t(ke - a.gk0) * a.gY + (ej - a.gj0)) * a.gX + (i - a.gi0);
                        r = a.greg[gidx];
                    }
                    if (r >= 0 && a.gcoef[r].active) {
                        const GainCoef<T> gc = a.gcoef[r];
                        const T ez_old = ez[e];
                        const T P = Pcur[gidx], Pp = Pold[gidx];
                        T Nu = a.Nu[gidx], Ng = a.Ng[gidx];
                        const T ng_frac = (Ng - Nu) * gc.inv_N0;
                        const T Pn = gc.kapaN0 * (ng_frac * ez_old) + gc.pa2 * P + gc.pa3 * Pp;
                        const T dP = (Pn - P) * gc.inv_dt;
                        ez[e] = ez[e] + bz[e] * (((dHy_dx - dHx_dy) - Jz) - dP);
                        const T e_avg = T(0.5) * (ez[e] + ez_old);
                        const T stim = e_avg * (Pn - P) * gc.inv_dt * gc.inv_hbar_omega;
                        T dNu = -gc.inv_tau * Nu + stim;
                        T dNg = gc.inv_tau * Nu - stim;
                        if (gc.pump != T(0)) { dNu += gc.pump * Ng; dNg -= gc.pump * Ng; }
                        Nu = Nu + gc.dt * dNu;
                        Ng = Ng + gc.dt * dNg;
                        Nu = fmax(T(0), Nu);
                        Ng = fmax(T(0), Ng);
                        if (gc.clamp) {
                            const T tot = Nu + Ng;
                            if (tot > T(1e-30)) { const T sc = gc.N0 / tot; Nu *= sc; Ng *= sc; }
                            Nu = fmin(Nu, gc.N0);
                            Ng = gc.N0 - Nu;
                        }
                        Pold[gidx] = Pn;
                        a.Nu[gidx] = Nu;
                        a.Ng[gidx] = Ng;
                    } else {
                        ez[e] = ez[e] + bz[e] * ((dHy_dx - dHx_dy) - Jz);
                    }
                }
            }
            const size_t g = size_t(ke) * a.plane + size_t(ej) * a.NxP + ei0;
            V::st(f.dE[0] + g, ex);
            V::st(f.dE[1] + g, ey);
            V::st(f.dE[2] + g, ez);
        }
    }
    if (!ok && tid == 0) {
        // A copy never arrived: record it, wait (bounded) for the stages this block issued
        // but did not consume, then leave.
        atomicOr(f.status_w, kStatusTimeout);
        const int issued = min(nit, consumed + D);
        for (int t = consumed; t < issued; ++t) mbar_wait(&sm.full[t % NB], unsigned((t / NB) & 1));
    }
}

// Tile shapes (TX, TY, threads, stages in flight, blocks per SM), shared memory in FP32:
// shape 0 = 64x16 cells (32x16 in FP64), 320 threads, 2 stages ahead, 1 block (212 KB);
// shape 1 = 64x12 (32x12), 224 threads, 3 stages ahead, 1 block (196 KB);
// shape 2 = 64x8 (32x8), 160 threads, 1 stage ahead, 2 blocks (91 KB each).
template <typename T> struct ShapeSet;
template <> struct ShapeSet<float> {
    using S0 = FusedShape<float, 64, 16, 320, 2, 1>;
    using S1 = FusedShape<float, 64, 12, 224, 3, 1>;
    using S2 = FusedShape<float, 64, 8, 160, 1, 2>;
};
template <> struct ShapeSet<double> {
    using S0 = FusedShape<double, 32, 16, 320, 2, 1>;
    using S1 = FusedShape<double, 32, 12, 224, 3, 1>;
    using S2 = FusedShape<double, 32, 8, 160, 1, 2>;
};

template <typename T, typename Shape>
void launch_fused(dim3 grid, int threads, size_t smem, cudaStream_t st, const FusedMaps& maps,
                  const FusedArgs<T>& fa, int kchunk, const ESrc& src) {
    k_step_fused<T, Shape><<<grid, threads, smem, st>>>(maps, fa, kchunk, src);
}

}  // namespace fdtdk
