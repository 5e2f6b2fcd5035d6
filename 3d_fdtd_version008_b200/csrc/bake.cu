// bake.cu -- the subpixel material bake on the GPU (StructureScene::bake,
// src/structure_material.hpp:211-288, for the three E components).
//
// Per cell and E component: the relative permittivity of the last-defined item containing
// each of the 2x2x2 samples at the Yee offset, eps = sum(eps_r * eps0) / 8, bE = (dt/eps)/(1+c1)
// with c1 = sigma*dt/(2 eps) = 0.  The host bake (Scene::bake, compiled without contraction) is
// reproduced operation for operation: every product, sum and quotient below is rounded on its
// own (__dmul_rn / __dadd_rn / __ddiv_rn), in the host's order, so the arrays are bit-identical.
// The item lists come from the same spatial bins as the host's (make_item_bins).
#include "host/setup.hpp"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct BakeItem {
    int type;  // 0 box, 1 sphere, 2 z-cylinder (ShapeType)
    int pad;
    double a[6];
    double eps_r;
};

struct BinGeom {
    double lo[3], w[3];
    unsigned long long nb[3];
};

__device__ __forceinline__ unsigned long long bin_of(const BinGeom& g, int a, double v) {
    const double t = __ddiv_rn(__dsub_rn(v, g.lo[a]), g.w[a]);
    if (!(t > 0)) return 0;
    const unsigned long long b = __double2ull_rz(t);
    return b >= g.nb[a] ? g.nb[a] - 1 : b;
}

// Shape::contains (src/structure_material.hpp:53-80)
__device__ __forceinline__ bool contains(const BakeItem& it, double x, double y, double z) {
    if (it.type == 0)
        return x >= it.a[0] && x < it.a[1] && y >= it.a[2] && y < it.a[3] && z >= it.a[4] && z < it.a[5];
    if (it.type == 1) {
        const double dx = __dsub_rn(x, it.a[0]), dy = __dsub_rn(y, it.a[1]), dz = __dsub_rn(z, it.a[2]);
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        return r2 <= __dmul_rn(it.a[3], it.a[3]);
    }
    if (z < it.a[3] || z >= it.a[4]) return false;
    const double dx = __dsub_rn(x, it.a[0]), dy = __dsub_rn(y, it.a[1]);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= __dmul_rn(it.a[2], it.a[2]);
}

// One thread per cell (idx3 order, z fastest, so the FP64 outputs are written coalesced).
__global__ void k_bake_E(const BakeItem* __restrict__ items, const unsigned* __restrict__ start,
                         const unsigned* __restrict__ ids, BinGeom bg, const double* __restrict__ xb,
                         const double* __restrict__ yb, const double* __restrict__ zb, const double* __restrict__ dxs,
                         const double* __restrict__ dys, const double* __restrict__ dzs, long long NxT, long long NyT,
                         long long NzT, double eps0, double bg_eps_r, double dt, double* __restrict__ bEx,
                         double* __restrict__ bEy, double* __restrict__ bEz) {
    const long long N = NxT * NyT * NzT;
    // Yee offsets of Ex, Ey, Ez (src/structure_material.hpp:226-231) and the sample
    // fractions (a + 0.5) / 2
    const double off[3][3] = {{0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0}};
    const double rs[2] = {0.25, 0.75};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
        const long long i = q / (NyT * NzT), j = (q / NzT) % NyT, k = q % NzT;
        const double x0 = xb[i], y0 = yb[j], z0 = zb[k], dxl = dxs[i], dyl = dys[j], dzl = dzs[k];
        double out[3];
        for (int comp = 0; comp < 3; ++comp) {
            double eps_sum = 0.0;
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b)
                    for (int c = 0; c < 2; ++c) {
                        const double xs = __dadd_rn(x0, __dmul_rn(__dadd_rn(off[comp][0], rs[a]), dxl));
                        const double ys = __dadd_rn(y0, __dmul_rn(__dadd_rn(off[comp][1], rs[b]), dyl));
                        const double zs = __dadd_rn(z0, __dmul_rn(__dadd_rn(off[comp][2], rs[c]), dzl));
                        const unsigned long long bin =
                            (bin_of(bg, 0, xs) * bg.nb[1] + bin_of(bg, 1, ys)) * bg.nb[2] + bin_of(bg, 2, zs);
                        double er = bg_eps_r;
                        for (unsigned t = start[bin]; t < start[bin + 1]; ++t) {
                            const BakeItem& it = items[ids[t]];
                            if (contains(it, xs, ys, zs)) { er = it.eps_r; break; }
                        }
                        eps_sum = __dadd_rn(eps_sum, __dmul_rn(er, eps0));
                    }
            const double eps = __ddiv_rn(eps_sum, 8.0);
            const double c1 = __ddiv_rn(__dmul_rn(0.0, dt), __dmul_rn(2.0, eps));  // sigma = 0
            out[comp] = __ddiv_rn(__ddiv_rn(dt, eps), __dadd_rn(1.0, c1));
        }
        bEx[q] = out[0];
        bEy[q] = out[1];
        bEz[q] = out[2];
    }
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("GPU bake: ") + what + ": " + cudaGetErrorString(e));
}

template <typename T>
T* to_dev(const std::vector<T>& v, std::vector<void*>& owned) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    if (!v.empty()) check(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    return static_cast<T*>(p);
}

}  // namespace

namespace fdtd {

bool gpu_bake(const Scene& sc, MaterialGrids& mg, real dt, real eps0, real mu0) {
    auto plain = [](const Material& m) { return m.sigma == 0.0 && m.sigma_m == 0.0 && m.mu_r == 1.0; };
    if (!plain(sc.bg)) return false;
    for (const auto& it : sc.items)
        if (!plain(it.mat)) return false;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw std::runtime_error("BAKE = gpu needs a CUDA device");
    }
    const ItemBins B = make_item_bins(sc.items, sc.grid);
    std::vector<BakeItem> items(sc.items.size());
    for (size_t q = 0; q < items.size(); ++q) {
        const Shape& sh = sc.items[q].shape;
        items[q].type = sh.type == ShapeType::Box ? 0 : sh.type == ShapeType::Sphere ? 1 : 2;
        items[q].pad = 0;
        for (int c = 0; c < 6; ++c) items[q].a[c] = sh.a[c];
        items[q].eps_r = sc.items[q].mat.eps_r;
    }
    BinGeom bg{};
    for (int a = 0; a < 3; ++a) {
        bg.lo[a] = B.lo[a];
        bg.w[a] = B.w[a];
        bg.nb[a] = B.nb[a];
    }
    const size_t N = sc.NxT * sc.NyT * sc.NzT;
    std::vector<void*> owned;
    try {
        const BakeItem* d_items = to_dev(items, owned);
        const unsigned* d_start = to_dev(B.start, owned);
        const unsigned* d_ids = to_dev(B.ids, owned);
        const double* d_b[3] = {to_dev(sc.grid.x_bounds, owned), to_dev(sc.grid.y_bounds, owned),
                                to_dev(sc.grid.z_bounds, owned)};
        const double* d_d[3] = {to_dev(sc.grid.dx, owned), to_dev(sc.grid.dy, owned), to_dev(sc.grid.dz, owned)};
        double* d_out[3];
        for (int c = 0; c < 3; ++c) {
            void* p = nullptr;
            check(cudaMalloc(&p, N * sizeof(double)), "cudaMalloc");
            owned.push_back(p);
            d_out[c] = static_cast<double*>(p);
        }
        k_bake_E<<<148 * 16, 256>>>(d_items, d_start, d_ids, bg, d_b[0], d_b[1], d_b[2], d_d[0], d_d[1], d_d[2],
                                    (long long)sc.NxT, (long long)sc.NyT, (long long)sc.NzT, eps0, sc.bg.eps_r, dt,
                                    d_out[0], d_out[1], d_out[2]);
        check(cudaGetLastError(), "k_bake_E");
        mg.NxT = sc.NxT; mg.NyT = sc.NyT; mg.NzT = sc.NzT;
        for (int c = 0; c < 3; ++c) {
            mg.bE[c].resize(N);
            check(cudaMemcpy(mg.bE[c].data(), d_out[c], N * sizeof(double), cudaMemcpyDeviceToHost), "bE read-back");
            mg.aE[c].clear(); mg.aH[c].clear(); mg.bH[c].clear();
        }
    } catch (...) {
        for (void* p : owned) cudaFree(p);
        throw;
    }
    for (void* p : owned) cudaFree(p);
    // The H components with mu_r = 1 and sigma_m = 0, as Scene::bake computes them: the same
    // value in every cell.
    real mu_sum = 0;
    for (int q = 0; q < 8; ++q) mu_sum += 1.0 * mu0;
    const real mu = mu_sum / 8;
    const real c2 = 0.0 * dt / (2 * mu);
    mg.uniform_ah = true;
    mg.bH_value = (dt / mu) / (1 + c2);
    return true;
}

}  // namespace fdtd
