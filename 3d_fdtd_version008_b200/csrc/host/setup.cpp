// setup.cpp -- host setup API: parameter file, grid spacing, CPML profiles, scene
// bake, sources, two-level gain regions and the make_context sequence.
//
// Each routine keeps the reference's double-precision operation order (cited per
// function) because the setup arrays are part of the parity contract: mesh lines,
// bE coefficients, CPML profiles and the gain-cell map must be bit-identical.
#include "setup.hpp"
#include "waveform.hpp"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numbers>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace fdtd {

// ================================================================ parameter file
namespace {

std::string trim(const std::string& s) {
    std::size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    std::size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::vector<std::string> split_fields(const std::string& s) {
    std::vector<std::string> out;
    std::string cur;
    bool quoted = false;
    for (char c : s) {
        if (c == '"') { quoted = !quoted; continue; }
        if (c == ',' && !quoted) { out.push_back(trim(cur)); cur.clear(); continue; }
        cur.push_back(c);
    }
    out.push_back(trim(cur));
    return out;
}

bool parse_bool(const std::string& v) {
    if (v == "1" || v == "true" || v == "TRUE" || v == "True") return true;
    if (v == "0" || v == "false" || v == "FALSE" || v == "False" || v.empty()) return false;
    throw std::runtime_error("not a boolean: '" + v + "'");
}

double parse_num(const std::string& v) {
    if (v.empty()) return 0.0;
    char* end = nullptr;
    double x = std::strtod(v.c_str(), &end);
    if (end == v.c_str() || trim(std::string(end)).size() != 0)
        throw std::runtime_error("not a number: '" + v + "'");
    return x;
}

double field(const std::vector<std::string>& f, std::size_t i) { return i < f.size() ? parse_num(f[i]) : 0.0; }

}  // namespace

ParamFile ParamFile::parse(const std::string& text) {
    ParamFile pf;
    std::istringstream in(text);
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        auto hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        auto pe = line.find("+=");
        if (pe != std::string::npos) {
            std::string key = trim(line.substr(0, pe));
            if (key.empty()) throw std::runtime_error("line " + std::to_string(lineno) + ": missing key");
            pf.lists[key].push_back(split_fields(line.substr(pe + 2)));
            continue;
        }
        auto eq = line.find('=');
        if (eq == std::string::npos)
            throw std::runtime_error("line " + std::to_string(lineno) + ": expected KEY = value or KEY += fields");
        std::string key = trim(line.substr(0, eq));
        if (key.empty()) throw std::runtime_error("line " + std::to_string(lineno) + ": missing key");
        pf.scalars[key] = trim(line.substr(eq + 1));
    }
    return pf;
}

double ParamFile::num(const std::string& key, double dflt) const {
    auto it = scalars.find(key);
    if (it == scalars.end()) return dflt;
    try {
        return parse_num(it->second);
    } catch (const std::exception& e) {
        throw std::runtime_error(key + ": " + e.what());
    }
}

bool ParamFile::flag(const std::string& key, bool dflt) const {
    auto it = scalars.find(key);
    if (it == scalars.end()) return dflt;
    try {
        return parse_bool(it->second);
    } catch (const std::exception& e) {
        throw std::runtime_error(key + ": " + e.what());
    }
}

std::string ParamFile::str(const std::string& key, const std::string& dflt) const {
    auto it = scalars.find(key);
    return it == scalars.end() ? dflt : it->second;
}

const std::vector<std::vector<std::string>>& ParamFile::list(const std::string& key) const {
    static const std::vector<std::vector<std::string>> empty;
    auto it = lists.find(key);
    return it == lists.end() ? empty : it->second;
}

// ================================================================ grid spacing
void GridSpacing::compute_inverses() {  // src/global_function.hpp:98-105
    inv_dx.resize(dx.size());
    inv_dy.resize(dy.size());
    inv_dz.resize(dz.size());
    for (std::size_t i = 0; i < dx.size(); ++i) inv_dx[i] = 1.0 / dx[i];
    for (std::size_t j = 0; j < dy.size(); ++j) inv_dy[j] = 1.0 / dy[j];
    for (std::size_t k = 0; k < dz.size(); ++k) inv_dz[k] = 1.0 / dz[k];
}

real GridSpacing::pml_offset(int axis) const {  // src/global_function.hpp:111-113
    const auto& b = bounds(axis);
    return (npml < b.size()) ? b[npml] : 0.0;
}

std::size_t GridSpacing::physical_to_index(int axis, real phys) const {  // :137-157
    const auto& b = bounds(axis);
    real total = phys + pml_offset(axis);
    if (total <= b.front()) return 0;
    if (total >= b.back()) return b.size() - 2;
    auto it = std::upper_bound(b.begin(), b.end(), total);
    return std::size_t(it - b.begin()) - 1;
}

real GridSpacing::cell_center_physical(int axis, std::size_t i) const {  // :123-134
    const auto& b = bounds(axis);
    if (i + 1 >= b.size()) return b.back() - pml_offset(axis);
    return 0.5 * (b[i] + b[i + 1]) - pml_offset(axis);
}

void build_cumulative_bounds(const std::vector<real>& spacing, std::vector<real>& bounds) {  // :160-167
    std::size_t N = spacing.size();
    bounds.resize(N + 1);
    bounds[0] = 0.0;
    for (std::size_t i = 0; i < N; ++i) bounds[i + 1] = bounds[i] + spacing[i];
}

// ================================================================ CPML profiles
// CPMLBoundary::build_profiles_and_coeffs (src/boundary.hpp:303-373), including the
// reference's grading sigma = sigma_max * kappa * r^m and its H-side normalisation
// of sigma by mu0 (not eps0), both part of the parity contract.
CpmlProfiles build_cpml_profiles(const GridSpacing& g, const CpmlConfig& cfg, real dt) {
    CpmlProfiles p;
    p.npml = cfg.npml;
    const int npml = cfg.npml;
    const real eps0 = phys::EPS0, mu0 = phys::MU0, c0 = phys::C0;

    auto avg_spacing = [&](const std::vector<real>& s, int N) {
        real sum = 0;
        int count = 0;
        for (int i = 0; i < npml; ++i) {
            sum += s[i] + s[N - 1 - i];
            count += 2;
        }
        return sum / count;
    };
    auto sigma_max = [&](real ds) -> real {
        real d = npml * ds;
        return ((cfg.m + 1.0) * std::log(1.0 / cfg.Rerr) * eps0 * c0) / (2.0 * d);
    };
    for (int a = 0; a < 3; ++a) {
        const auto& sp = g.spacing(a);
        const int N = int(sp.size());
        const real smax = sigma_max(avg_spacing(sp, N));
        p.kappa[a].assign(N, 1.0);
        p.sigma[a].assign(N, 0.0);
        p.alpha[a].assign(N, 0.0);
        for (int n = 0; n < N; ++n) {
            int d = std::min(n, N - 1 - n);
            if (d >= npml) continue;
            real r = real(npml - (d + 0.5)) / real(npml);
            real rm = std::pow(r, cfg.m);
            real kap = 1.0 + (cfg.kappa_max - 1.0) * rm;
            real sig = smax * kap * rm;
            real ds = sp[n];
            real alf = cfg.alpha_linear ? (cfg.alpha0 * (c0 / ds) * (1.0 - r))
                                        : (cfg.alpha0 * (c0 / ds) * std::pow(1.0 - r, cfg.m));
            p.sigma[a][n] = sig;
            p.kappa[a][n] = kap;
            p.alpha[a][n] = alf;
        }
        auto coeffs = [&](real norm, std::vector<real>& b, std::vector<real>& c) {
            b.assign(N, 1.0);
            c.assign(N, 0.0);
            for (int n = 0; n < N; ++n) {
                real sn = p.sigma[a][n] / norm;
                real kap = p.kappa[a][n];
                real alf = p.alpha[a][n];
                real be = std::exp(-(sn / kap + alf) * dt);
                be = std::max<real>(be, 1e-30);
                real ce = 0.0;
                if (std::abs(sn) > 1e-30 || std::abs(alf) > 1e-30) ce = (sn * (be - 1.0)) / (kap * (sn + kap * alf));
                b[n] = be;
                c[n] = ce;
            }
        };
        coeffs(eps0, p.bE[a], p.cE[a]);
        coeffs(mu0, p.bH[a], p.cH[a]);
    }
    return p;
}

// ================================================================ scene / bake
Material make_nk(real n) {  // src/structure_material.hpp:24-30 (k ignored, sigma = 0)
    Material m;
    m.eps_r = n * n;
    m.mu_r = 1.0;
    m.sigma = 0.0;
    return m;
}

bool Shape::contains(real x, real y, real z) const {  // src/structure_material.hpp:53-80
    switch (type) {
        case ShapeType::Box:
            return (x >= a[0] && x < a[1] && y >= a[2] && y < a[3] && z >= a[4] && z < a[5]);
        case ShapeType::Sphere: {
            real dx = x - a[0], dy = y - a[1], dz = z - a[2];
            return (dx * dx + dy * dy + dz * dz) <= a[3] * a[3];
        }
        case ShapeType::CylinderZ: {
            if (z < a[3] || z >= a[4]) return false;
            real dx = x - a[0], dy = y - a[1];
            return (dx * dx + dy * dy) <= a[2] * a[2];
        }
    }
    return false;
}

void Shape::bounding_box(real bb[6]) const {
    switch (type) {
        case ShapeType::Box:
            for (int i = 0; i < 6; ++i) bb[i] = a[i];
            break;
        case ShapeType::Sphere:
            bb[0] = a[0] - a[3]; bb[1] = a[0] + a[3];
            bb[2] = a[1] - a[3]; bb[3] = a[1] + a[3];
            bb[4] = a[2] - a[3]; bb[5] = a[2] + a[3];
            break;
        case ShapeType::CylinderZ:
            bb[0] = a[0] - a[2]; bb[1] = a[0] + a[2];
            bb[2] = a[1] - a[2]; bb[3] = a[1] + a[2];
            bb[4] = a[3]; bb[5] = a[4];
            break;
    }
}

// Spatial bins over the scene items so that "the last item containing the point wins"
// (src/structure_material.hpp:214-220) is answered by scanning, newest first, only the
// items whose bounding box overlaps the point's bin.  Same winner as the full scan.
ItemBins make_item_bins(const std::vector<StructureItem>& items, const GridSpacing& g) {
    ItemBins B;
    for (int a = 0; a < 3; ++a) {
        const auto& b = g.bounds(a);
        B.lo[a] = b.front();
        const real hi = b.back();
        B.nb[a] = std::max<std::size_t>(1, std::min<std::size_t>(64, (b.size() + 7) / 8));
        B.w[a] = (hi - B.lo[a]) / real(B.nb[a]);
        if (!(B.w[a] > 0)) B.w[a] = 1.0;
    }
    std::vector<std::vector<uint32_t>> bins(B.nb[0] * B.nb[1] * B.nb[2]);
    for (std::size_t it = items.size(); it-- > 0;) {
        real bb[6];
        items[it].shape.bounding_box(bb);
        std::size_t b0[3], b1[3];
        for (int a = 0; a < 3; ++a) {
            b0[a] = B.bin(a, bb[2 * a]);
            b1[a] = B.bin(a, bb[2 * a + 1]);
        }
        for (std::size_t x = b0[0]; x <= b1[0]; ++x)
            for (std::size_t y = b0[1]; y <= b1[1]; ++y)
                for (std::size_t z = b0[2]; z <= b1[2]; ++z)
                    bins[(x * B.nb[1] + y) * B.nb[2] + z].push_back(uint32_t(it));
    }
    B.start.push_back(0);
    for (const auto& l : bins) {
        B.ids.insert(B.ids.end(), l.begin(), l.end());
        B.start.push_back(uint32_t(B.ids.size()));
    }
    return B;
}

namespace {

class ItemIndex {
public:
    ItemIndex(const std::vector<StructureItem>& items, const GridSpacing& g)
        : items_(items), B_(make_item_bins(items, g)) {}

    const Material& sample(real x, real y, real z, const Material& bg) const {
        const std::size_t b = (B_.bin(0, x) * B_.nb[1] + B_.bin(1, y)) * B_.nb[2] + B_.bin(2, z);
        for (uint32_t q = B_.start[b]; q < B_.start[b + 1]; ++q)
            if (items_[B_.ids[q]].shape.contains(x, y, z)) return items_[B_.ids[q]].mat;
        return bg;
    }

private:
    const std::vector<StructureItem>& items_;
    ItemBins B_;
};

}  // namespace

// StructureScene::bake (src/structure_material.hpp:211-288): 2x2x2 (s^3) samples per
// Yee component at the staggered offsets, eps/mu/sigma averaged in sample order.
void Scene::bake(MaterialGrids& mg, real dt, real eps0_arg, real mu0_arg, int subpixel_samples) const {
    mg.NxT = NxT; mg.NyT = NyT; mg.NzT = NzT;
    const std::size_t N = NxT * NyT * NzT;
    for (int c = 0; c < 3; ++c) {
        mg.aE[c].assign(N, 1); mg.bE[c].assign(N, 0);
        mg.aH[c].assign(N, 1); mg.bH[c].assign(N, 0);
    }
    int s = int(std::round(std::cbrt((double)subpixel_samples)));
    if (s < 1) s = 1;
    const ItemIndex index(items, grid);
    static const real off[6][3] = {{0.0, 0.5, 0.5}, {0.5, 0.0, 0.5}, {0.5, 0.5, 0.0},
                                   {0.5, 0.0, 0.0}, {0.0, 0.5, 0.0}, {0.0, 0.0, 0.5}};
#pragma omp parallel for schedule(dynamic, 1)
    for (long long ii = 0; ii < (long long)NxT; ++ii) {
        const std::size_t i = std::size_t(ii);
        for (std::size_t j = 0; j < NyT; ++j)
            for (std::size_t k = 0; k < NzT; ++k) {
                const std::size_t id = idx3(i, j, k, NyT, NzT);
                const real dxl = grid.dx[i], dyl = grid.dy[j], dzl = grid.dz[k];
                const real x0 = grid.x_bounds[i], y0 = grid.y_bounds[j], z0 = grid.z_bounds[k];
                for (int comp = 0; comp < 6; ++comp) {
                    const real ux = off[comp][0], uy = off[comp][1], uz = off[comp][2];
                    real eps_sum = 0, mu_sum = 0, sg_sum = 0, sgm_sum = 0;
                    int cnt = 0;
                    for (int a = 0; a < s; ++a)
                        for (int b = 0; b < s; ++b)
                            for (int c = 0; c < s; ++c) {
                                real rx = (a + 0.5) / s, ry = (b + 0.5) / s, rz = (c + 0.5) / s;
                                real xs = x0 + (ux + rx) * dxl;
                                real ys = y0 + (uy + ry) * dyl;
                                real zs = z0 + (uz + rz) * dzl;
                                const Material& m = index.sample(xs, ys, zs, bg);
                                eps_sum += m.eps_r * eps0_arg;
                                mu_sum += m.mu_r * mu0_arg;
                                sg_sum += m.sigma;
                                sgm_sum += m.sigma_m;
                                ++cnt;
                            }
                    const real eps = eps_sum / cnt, mu = mu_sum / cnt, sigma = sg_sum / cnt, sigm = sgm_sum / cnt;
                    if (comp < 3) {
                        real c1 = sigma * dt / (2 * eps);
                        mg.aE[comp][id] = (1 - c1) / (1 + c1);
                        mg.bE[comp][id] = (dt / eps) / (1 + c1);
                    } else {
                        real c2 = sigm * dt / (2 * mu);
                        mg.aH[comp - 3][id] = (1 - c2) / (1 + c2);
                        mg.bH[comp - 3][id] = (dt / mu) / (1 + c2);
                    }
                }
            }
    }
}

void Scene::n_grid(std::vector<real>& out) const {  // make_n_grid_from_scene (:291-310)
    out.assign(NxT * NyT * NzT, 1.0);
    const ItemIndex index(items, grid);
#pragma omp parallel for
    for (long long ii = 0; ii < (long long)NxT; ++ii) {
        const std::size_t i = std::size_t(ii);
        for (std::size_t j = 0; j < NyT; ++j)
            for (std::size_t k = 0; k < NzT; ++k) {
                real x = 0.5 * (grid.x_bounds[i] + grid.x_bounds[i + 1]);
                real y = 0.5 * (grid.y_bounds[j] + grid.y_bounds[j + 1]);
                real z = 0.5 * (grid.z_bounds[k] + grid.z_bounds[k + 1]);
                const Material& m = index.sample(x, y, z, bg);
                out[idx3(i, j, k, NyT, NzT)] = std::sqrt(m.eps_r * m.mu_r);
            }
    }
}

// ================================================================ sources
real compute_waveform(Waveform w, real t, real I0, real f0, real tau, real t0, real t_shift) {
    return waveform_value(int(w), t, I0, f0, tau, t0, t_shift);
}

real DipoleSource::current_density(std::size_t n, real dt) const {  // inject_half_step, :60-85
    return fdtd::current_density(int(waveform), n, dt, I0, f0, tau, t0, t_shift, cell_area);
}

// ================================================================ two-level gain
void TlsParams::finalize(real c0, real eps0, real hbar_in) {  // src/two_level_system.hpp:37-52
    hbar = hbar_in;
    omega_a = 2.0 * std::numbers::pi * c0 / lambda0;
    real numerator = 3.0 * std::numbers::pi * eps0 * hbar * c0 * c0 * c0;
    real denominator = omega_a * omega_a * omega_a * tau;
    mu_z = std::sqrt(numerator / denominator);
}

void TlsParams::finalize_with_dt(real dt) {  // src/two_level_system.hpp:70-87
    if (omega_a <= 0.0) return;
    const real dt2 = dt * dt;
    const real omega_sq = omega_a * omega_a;
    const real beta = 2.0 + gamma * dt;
    const real two_omega_over_hbar = 2.0 * omega_a / hbar;
    const real mu_z_sq = mu_z * mu_z;
    kapa_coeff = (2.0 * dt2 / beta) * two_omega_over_hbar * mu_z_sq;
    pa2 = 2.0 * (2.0 - omega_sq * dt2) / beta;
    pa3 = (gamma * dt - 2.0) / beta;
    inv_dt = 1.0 / dt;
    coefficients_initialized = true;
}

bool TlsRegion::contains(std::size_t i, std::size_t j, std::size_t k, const GridSpacing& g) const {  // :431-443
    if (!(i >= i0 && i < i1 && j >= j0 && j < j1 && k >= k0 && k < k1)) return false;
    real x = 0.5 * (g.x_bounds[i] + g.x_bounds[i + 1]);
    real y = 0.5 * (g.y_bounds[j] + g.y_bounds[j + 1]);
    real z = 0.5 * (g.z_bounds[k] + g.z_bounds[k + 1]);
    return shape.contains(x, y, z);
}

// ================================================================ make_context
namespace {

int to_polarization(int p) { return (p >= 0 && p <= 5) ? p : 2; }

Waveform to_waveform(int w) {
    switch (w) {
        case 1: return Waveform::GaussianModulatedSine;
        case 2: return Waveform::RickerLikeGaussian2nd;
        case 3: return Waveform::ContinuousWave;
        default: return Waveform::Ricker;
    }
}

void require(bool ok, const std::string& msg) {
    if (!ok) throw std::runtime_error(msg);
}

}  // namespace

SimSetup SimSetup::from_params(const ParamFile& pf, bool bake) {
    SimSetup S;
    S.params = pf;
    // Defaults are the reference's UserConfig values (src/user_config.hpp).
    S.auto_mesh = int(pf.num("MESH_MODE", 1)) != 0;
    const real dxu = pf.num("DX_UNIFORM", 10e-9), dyu = pf.num("DY_UNIFORM", 10e-9), dzu = pf.num("DZ_UNIFORM", 10e-9);
    std::size_t Nx = std::size_t(pf.num("NX", 100)), Ny = std::size_t(pf.num("NY", 100)), Nz = std::size_t(pf.num("NZ", 100));
    const real lambda0 = pf.num("LAMBDA0", 1500e-9);
    S.domain_min[0] = pf.num("DOMAIN_X_MIN", 0.0); S.domain_max[0] = pf.num("DOMAIN_X_MAX", 4000e-9);
    S.domain_min[1] = pf.num("DOMAIN_Y_MIN", 0.0); S.domain_max[1] = pf.num("DOMAIN_Y_MAX", 4000e-9);
    S.domain_min[2] = pf.num("DOMAIN_Z_MIN", 0.0); S.domain_max[2] = pf.num("DOMAIN_Z_MAX", 1000e-9);
    S.S = pf.num("CFL_FACTOR", 0.99);
    S.n_steps = std::size_t(pf.num("N_STEPS", 100000));
    S.save_every = std::size_t(pf.num("SAVE_EVERY", 10));
    require(S.save_every >= 1, "SAVE_EVERY must be >= 1");
    S.boundary_pec = int(pf.num("BOUNDARY_TYPE", 1)) == 0;
    S.cpml_cfg.npml = int(pf.num("CPML_NPML", 8));
    S.cpml_cfg.m = pf.num("CPML_M", 3.0);
    S.cpml_cfg.Rerr = pf.num("CPML_RERR", 1e-8);
    S.cpml_cfg.alpha0 = pf.num("CPML_ALPHA0", 0.2);
    S.cpml_cfg.kappa_max = pf.num("CPML_KAPPA_MAX", 10.0);
    S.cpml_cfg.alpha_linear = pf.flag("CPML_ALPHA_LINEAR", true);
    require(S.cpml_cfg.npml >= 0, "CPML_NPML must be >= 0");
    const bool tls_enabled_cfg = pf.flag("TLS_ENABLED", true);
    const bool tls_clamp = pf.flag("TLS_ENABLE_CLAMP", false);
    const real background_n = pf.num("BACKGROUND_N", 1.0);
    const bool override_enabled = pf.flag("MESH_OVERRIDE_ENABLED", true);
    S.stability_interval = std::size_t(pf.num("STABILITY_MONITOR_INTERVAL", 10));
    S.stability_max_E = pf.num("STABILITY_MAX_E", 1e10);
    S.stability_max_P = pf.num("STABILITY_MAX_P", 1e5);
    S.stability_conservation = pf.num("STABILITY_CONSERVATION_ERR", 0.01);
    S.stability_growth = pf.num("STABILITY_GROWTH_RATE", 10.0);
    S.precision = pf.str("PRECISION", "fp32");
    if (S.precision != "fp32" && S.precision != "fp64" && S.precision != "fp16" && S.precision != "bf16")
        throw std::runtime_error("PRECISION must be fp32, fp64, fp16 or bf16");
    S.field_scale = pf.num("FIELD_SCALE", 0.0);
    const std::string rounding = pf.str("ROUNDING", "nearest");
    if (rounding != "nearest" && rounding != "stochastic") throw std::runtime_error("ROUNDING must be nearest or stochastic");
    S.stochastic_rounding = rounding == "stochastic";
    S.noise_amplitude = pf.num("NOISE_AMPLITUDE", 0.0);
    S.seed = uint64_t(pf.num("SEED", 1));
    const real pump = pf.num("PUMP_RATE", 0.0);
    if (pf.scalars.count("DFT_FREQS")) {
        auto f = split_fields(pf.scalars.at("DFT_FREQS"));
        require(f.size() == 3, "DFT_FREQS expects: start, stop, count");
        const real f0 = parse_num(f[0]), f1 = parse_num(f[1]);
        const int nf = int(parse_num(f[2]));
        require(nf >= 1 && nf <= 1024, "DFT_FREQS count must be in [1, 1024]");
        for (int m = 0; m < nf; ++m) S.dft_freqs.push_back(nf == 1 ? f0 : f0 + (f1 - f0) * m / (nf - 1));
    }

    AutoMeshConfig amc;
    amc.lambda_min = lambda0;
    amc.mesh_accuracy = int(pf.num("AUTO_MESH_ACCURACY", 2));
    amc.ppw_override = pf.num("AUTO_MESH_PPW_OVERRIDE", 20.0);
    amc.dx_min = pf.num("AUTO_MESH_DX_MIN", 2e-9);
    amc.dx_max = pf.num("AUTO_MESH_DX_MAX", 100e-9);
    amc.max_grading_ratio = pf.num("AUTO_MESH_MAX_GRADING_RATIO", 1.41421356237);
    amc.mesh_override_enabled = override_enabled;

    // Structure definitions (StructureDef{type, n, params[6], tls_material}).
    struct Def { std::string type; real n; real p[6]; std::string tls; };
    std::vector<Def> defs;
    for (const auto& s : pf.list("STRUCTURES")) {
        require(s.size() >= 8, "STRUCTURES entry needs: type, n, p0..p5[, tls_material]");
        Def d{s[0], field(s, 1), {field(s, 2), field(s, 3), field(s, 4), field(s, 5), field(s, 6), field(s, 7)},
              s.size() > 8 ? s[8] : std::string()};
        require(d.type == "box" || d.type == "sphere" || d.type == "cylinder",
                "STRUCTURES type must be box, sphere or cylinder (got '" + d.type + "')");
        defs.push_back(d);
    }
    std::vector<TlsMaterialDef> library;
    for (const auto& e : pf.list("TLS_MATERIALS")) {
        require(e.size() >= 6, "TLS_MATERIALS entry needs: name, lambda0, gamma, tau, N0, inversion_fraction");
        library.push_back({e[0], field(e, 1), field(e, 2), field(e, 3), field(e, 4), field(e, 5)});
    }

    // register_structure_bounds_for_auto_mesh + register_mesh_override_regions
    // (src/params.hpp:518-555).
    std::vector<StructureBounds> sb;
    if (S.auto_mesh) {
        for (const auto& d : defs) {
            if (d.type == "box") sb.push_back({d.p[0], d.p[1], d.p[2], d.p[3], d.p[4], d.p[5], d.n});
            else if (d.type == "sphere")
                sb.push_back({d.p[0] - d.p[3], d.p[0] + d.p[3], d.p[1] - d.p[3], d.p[1] + d.p[3], d.p[2] - d.p[3],
                              d.p[2] + d.p[3], d.n});
            else
                sb.push_back({d.p[0] - d.p[2], d.p[0] + d.p[2], d.p[1] - d.p[2], d.p[1] + d.p[2], d.p[3], d.p[4], d.n});
        }
        amc.override_regions.clear();
        if (override_enabled) {
            for (const auto& r : pf.list("MESH_OVERRIDE_REGIONS")) {
                require(r.size() >= 10, "MESH_OVERRIDE_REGIONS entry needs: enabled, x0, x1, y0, y1, z0, z1, dx, dy, dz");
                if (!parse_bool(r[0])) continue;
                MeshOverrideRegion o;
                o.enabled = true;
                o.x0 = field(r, 1); o.x1 = field(r, 2); o.y0 = field(r, 3);
                o.y1 = field(r, 4); o.z0 = field(r, 5); o.z1 = field(r, 6);
                o.dx = field(r, 7); o.dy = field(r, 8); o.dz = field(r, 9);
                o.priority = 0;
                amc.override_regions.push_back(o);
            }
        }
    }

    // make_context (src/params.hpp:180-510)
    const std::size_t npml = std::size_t(S.cpml_cfg.npml);
    if (S.auto_mesh) {
        amc.lambda_min = lambda0;
        if (amc.dx_min <= 0) amc.dx_min = lambda0 / 100.0;
        if (amc.dx_max <= 0) amc.dx_max = lambda0 / 4.0;
        real dom[3];
        const real du[3] = {dxu, dyu, dzu};
        const std::size_t Nc[3] = {Nx, Ny, Nz};
        for (int a = 0; a < 3; ++a) {
            dom[a] = S.domain_max[a] - S.domain_min[a];
            if (dom[a] <= 0) dom[a] = Nc[a] * du[a];
        }
        S.grid = automesh_generate(amc, dom[0], dom[1], dom[2], npml, sb, 1.0);
    } else {
        require(Nx >= 1 && Ny >= 1 && Nz >= 1, "NX, NY, NZ must be >= 1");
        S.grid.dx.assign(Nx + 2 * npml, dxu);
        S.grid.dy.assign(Ny + 2 * npml, dyu);
        S.grid.dz.assign(Nz + 2 * npml, dzu);
        build_cumulative_bounds(S.grid.dx, S.grid.x_bounds);
        build_cumulative_bounds(S.grid.dy, S.grid.y_bounds);
        build_cumulative_bounds(S.grid.dz, S.grid.z_bounds);
    }
    S.grid.compute_inverses();
    S.NxT = S.grid.dx.size();
    S.NyT = S.grid.dy.size();
    S.NzT = S.grid.dz.size();
    require(S.NxT >= 3 && S.NyT >= 3 && S.NzT >= 3, "grid must have at least 3 cells per axis");
    require(S.NxT > 2 * npml && S.NyT > 2 * npml && S.NzT > 2 * npml, "grid smaller than the two CPML layers");
    const real dx_min = *std::min_element(S.grid.dx.begin(), S.grid.dx.end());
    const real dy_min = *std::min_element(S.grid.dy.begin(), S.grid.dy.end());
    const real dz_min = *std::min_element(S.grid.dz.begin(), S.grid.dz.end());
    const real sum_inv2 = (1.0 / (dx_min * dx_min)) + (1.0 / (dy_min * dy_min)) + (1.0 / (dz_min * dz_min));
    S.dt = S.S / (phys::C0 * std::sqrt(sum_inv2));
    S.Nx_core = S.NxT - 2 * npml;
    S.Ny_core = S.NyT - 2 * npml;
    S.Nz_core = S.NzT - 2 * npml;
    S.npml = npml;
    if (S.boundary_pec) {
        // PECBoundary(NxCore, NyCore, NzCore) reports the core sizes as the totals and no PML
        // layer (src/boundary.hpp:51-79, src/params.hpp:271-294): the fields cover the first
        // Nx_core cells of the padded mesh, whose arrays keep their padded length, and every
        // position is taken from the mesh origin.
        S.NxT = S.Nx_core; S.NyT = S.Ny_core; S.NzT = S.Nz_core;
        S.npml = 0;
        require(S.NxT >= 3 && S.NyT >= 3 && S.NzT >= 3, "PEC grid must have at least 3 core cells per axis");
    }
    S.grid.npml = S.npml;
    CpmlConfig cc = S.cpml_cfg;
    cc.npml = int(S.npml);
    S.cpml = build_cpml_profiles(S.grid, cc, S.dt);
    if (!bake) return S;

    // apply_structure_packages (register_default_structures, src/params.hpp:557-592)
    Scene& sc = S.scene;
    sc.NxT = S.NxT; sc.NyT = S.NyT; sc.NzT = S.NzT; sc.npml_cells = S.npml;
    sc.grid = S.grid;
    sc.bg = make_nk(background_n);
    const std::size_t np0 = S.npml;
    const real pml_x = S.grid.x_bounds[np0], pml_y = S.grid.y_bounds[np0], pml_z = S.grid.z_bounds[np0];
    for (const auto& d : defs) {
        StructureItem it;
        it.mat = make_nk(d.n);
        const TlsMaterialDef* tm = nullptr;
        if (!d.tls.empty())
            for (const auto& m : library)
                if (m.name == d.tls) { tm = &m; break; }
        require(d.tls.empty() || tm, "TLS material '" + d.tls + "' is not defined in TLS_MATERIALS");
        if (tm && tls_enabled_cfg) {
            it.tls_enabled = true;
            it.tls = *tm;
        }
        if (d.type == "box") {
            it.shape.type = ShapeType::Box;
            real v[6] = {pml_x + d.p[0], pml_x + d.p[1], pml_y + d.p[2], pml_y + d.p[3], pml_z + d.p[4], pml_z + d.p[5]};
            std::copy(v, v + 6, it.shape.a);
        } else if (d.type == "sphere") {
            it.shape.type = ShapeType::Sphere;
            real v[6] = {pml_x + d.p[0], pml_y + d.p[1], pml_z + d.p[2], d.p[3], 0, 0};
            std::copy(v, v + 6, it.shape.a);
        } else {
            it.shape.type = ShapeType::CylinderZ;
            real v[6] = {pml_x + d.p[0], pml_y + d.p[1], d.p[2], pml_z + d.p[3], pml_z + d.p[4], 0};
            std::copy(v, v + 6, it.shape.a);
        }
        sc.items.push_back(it);
    }
    // bake_and_bind (src/params.hpp:512-516), 8 subpixel samples as main() passes.  BAKE = gpu
    // (a build-only key) bakes bE on the CUDA device instead, bit-identical, when the items
    // allow it.
    const std::string bake_on = pf.str("BAKE", "host");
    require(bake_on == "host" || bake_on == "gpu", "BAKE must be host or gpu");
    if (!(bake_on == "gpu" && gpu_bake(sc, S.mats, S.dt, phys::EPS0, phys::MU0)))
        sc.bake(S.mats, S.dt, phys::EPS0, phys::MU0, 8);

    // Dipole sources (register_default_sources / make_dipole_source,
    // src/params.hpp:594-647, src/sources/dipole_source.hpp:90-153).
    for (const auto& s : pf.list("DIPOLE_SOURCES")) {
        require(s.size() >= 12, "DIPOLE_SOURCES entry needs 12 fields (DipoleSourceDef order)");
        if (!parse_bool(s[0])) continue;
        const real x = field(s, 1), y = field(s, 2), z = field(s, 3);
        const real amplitude = field(s, 4), frequency = field(s, 5), wavelength = field(s, 6);
        const real tau = field(s, 7), df = field(s, 8), t0f = field(s, 9);
        DipoleSource src;
        src.waveform = to_waveform(int(field(s, 10)));
        src.polarization = to_polarization(int(field(s, 11)));
        src.i = S.grid.physical_to_index(0, x - S.domain_min[0]);
        src.j = S.grid.physical_to_index(1, y - S.domain_min[1]);
        src.k = S.grid.physical_to_index(2, z - S.domain_min[2]);
        // Only reachable with PEC, whose field grid is shorter than the mesh: the reference
        // would write past its J arrays.
        require(src.i < S.NxT && src.j < S.NyT && src.k < S.NzT, "dipole source lies outside the field grid");
        const real c0 = 299792458.0;
        real f = frequency > 0.0 ? frequency : (wavelength > 0.0 ? c0 / wavelength : c0 / 500e-9);
        real tau_eff = tau > 0.0 ? tau
                                 : (df > 0.0 ? 2.0 * std::sqrt(std::log(2.0)) / (std::numbers::pi * df) : 20.0 * S.dt);
        real t0 = t0f > 0.0 ? t0f * tau_eff : 3.0 / f;
        src.I0 = amplitude;
        src.f0 = f;
        src.tau = tau_eff;
        src.t0 = t0;
        src.t_shift = t0;
        switch (src.j_component()) {
            case 0: src.cell_area = S.grid.dy[src.j] * S.grid.dz[src.k]; break;
            case 1: src.cell_area = S.grid.dx[src.i] * S.grid.dz[src.k]; break;
            default: src.cell_area = S.grid.dx[src.i] * S.grid.dy[src.j]; break;
        }
        S.sources.push_back(src);
    }
    // Plane-wave soft sources (make_plane_wave_source, src/sources/plane_wave_source.hpp:201-290,
    // registered after the dipoles at src/params.hpp:643-679).
    for (const auto& s : pf.list("PLANE_WAVE_SOURCES")) {
        require(s.size() >= 17, "PLANE_WAVE_SOURCES entry needs 17 fields (PlaneWaveSourceDef order)");
        if (!parse_bool(s[0])) continue;
        const real pos = field(s, 1), amplitude = field(s, 2), frequency = field(s, 3), wavelength = field(s, 4);
        const real tau = field(s, 5), df = field(s, 6), t0f = field(s, 7);
        PlaneWave w;
        w.waveform = to_waveform(int(field(s, 8)));
        const int dir = int(field(s, 9));  // 0 +X, 1 -X, 2 +Y, 3 -Y, 4 +Z, 5 -Z, otherwise +Z
        const int pol = to_polarization(int(field(s, 10)));
        w.axis = (dir == 0 || dir == 1) ? 0 : (dir == 2 || dir == 3) ? 1 : 2;
        w.sign = (dir == 1 || dir == 3 || dir == 5) ? -1.0 : 1.0;
        const real c0 = 299792458.0;
        w.f0 = frequency > 0.0 ? frequency : (wavelength > 0.0 ? c0 / wavelength : c0 / 500e-9);
        w.tau = tau > 0.0 ? tau : (df > 0.0 ? 2.0 * std::sqrt(std::log(2.0)) / (std::numbers::pi * df) : 20.0 * S.dt);
        w.t0 = t0f > 0.0 ? t0f * w.tau : 3.0 / w.f0;
        w.t_shift = w.t0;
        w.E0 = amplitude;
        const std::size_t Nax[3] = {S.NxT, S.NyT, S.NzT}, np = S.npml;
        std::size_t pi = S.grid.physical_to_index(w.axis, pos - S.domain_min[w.axis]);
        pi = std::max(np + 1, std::min(pi, Nax[w.axis] - np - 2));
        w.plane = pi;
        const real mins[3] = {field(s, 11), field(s, 13), field(s, 15)}, maxs[3] = {field(s, 12), field(s, 14), field(s, 16)};
        std::size_t lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {  // compute_bounds, on the domain-shifted coordinates
            const real mn = mins[a] - S.domain_min[a], mx = maxs[a] - S.domain_min[a];
            if (mn == 0.0 && mx == 0.0) { lo[a] = np; hi[a] = Nax[a] - np - 1; }
            else {
                lo[a] = std::max(np, S.grid.physical_to_index(a, mn));
                hi[a] = std::min(Nax[a] - np - 1, S.grid.physical_to_index(a, mx));
            }
        }
        const int u = w.axis == 0 ? 1 : 0, v = w.axis == 2 ? 1 : 2;  // in-plane axes
        w.lo0 = lo[u]; w.hi0 = hi[u]; w.lo1 = lo[v]; w.hi1 = hi[v];
        const std::vector<real>& dd = w.axis == 0 ? S.grid.dx : w.axis == 1 ? S.grid.dy : S.grid.dz;
        w.d = dd[pi];
        const int pc = pol % 3;  // Ex/Hx, Ey/Hy, Ez/Hz; only the two in-plane components are driven
        w.comp = pc == w.axis ? -1 : pc;
        if (w.comp >= 0) S.plane_waves.push_back(w);
    }
    require(S.plane_waves.size() <= 2, "at most 2 plane-wave sources");

    // Two-level gain regions (src/3D_FDTD_version008.cpp:100-164,
    // TLSRegionManager::add_region_from_structure / initialize, src/two_level_system.hpp:503-546).
    TlsSetup& T = S.tls;
    if (tls_enabled_cfg) {
        for (const auto& it : sc.items) {
            if (!it.tls_enabled) continue;
            real bb[6];
            it.shape.bounding_box(bb);
            TlsRegion r;
            r.params.lambda0 = it.tls.lambda0;
            r.params.gamma = it.tls.gamma;
            r.params.tau = it.tls.tau;
            r.params.N0_total = it.tls.N0;
            r.params.enable_population_clamp = tls_clamp;
            r.params.pump_rate = pump;
            r.i0 = S.grid.physical_to_index(0, bb[0] - pml_x);
            r.i1 = S.grid.physical_to_index(0, bb[1] - pml_x) + 1;
            r.j0 = S.grid.physical_to_index(1, bb[2] - pml_y);
            r.j1 = S.grid.physical_to_index(1, bb[3] - pml_y) + 1;
            r.k0 = S.grid.physical_to_index(2, bb[4] - pml_z);
            r.k1 = S.grid.physical_to_index(2, bb[5] - pml_z) + 1;
            r.inversion_fraction = it.tls.inversion_fraction;
            r.shape = it.shape;
            T.regions.push_back(r);
        }
    }
    if (T.enabled()) {
        const std::size_t N = S.NxT * S.NyT * S.NzT;
        T.cell_region_map.assign(N, -1);
        T.Nu.assign(N, 0.0);
        T.Ng.assign(N, 0.0);
        T.Ndip.assign(N, 0.0);
        for (std::size_t r = 0; r < T.regions.size(); ++r) {
            TlsRegion& rg = T.regions[r];
            rg.params.finalize();
            const real N0 = rg.params.N0_total;
            for (std::size_t i = rg.i0; i < rg.i1; ++i)
                for (std::size_t j = rg.j0; j < rg.j1; ++j)
                    for (std::size_t k = rg.k0; k < rg.k1; ++k) {
                        if (i >= S.NxT || j >= S.NyT || k >= S.NzT) continue;
                        if (!rg.contains(i, j, k, S.grid)) continue;
                        const std::size_t id = idx3(i, j, k, S.NyT, S.NzT);
                        T.Ndip[id] = N0;
                        T.Nu[id] = rg.inversion_fraction * N0;
                        T.Ng[id] = (1.0 - rg.inversion_fraction) * N0;
                        T.cell_region_map[id] = int32_t(r);
                    }
        }
        for (auto& rg : T.regions) rg.params.finalize_with_dt(S.dt);
        T.gain_i0 = T.regions[0].i0; T.gain_i1 = T.regions[0].i1;
        T.gain_j0 = T.regions[0].j0; T.gain_j1 = T.regions[0].j1;
        T.gain_k0 = T.regions[0].k0; T.gain_k1 = T.regions[0].k1;
        for (std::size_t r = 1; r < T.regions.size(); ++r) {
            const auto& rg = T.regions[r];
            T.gain_i0 = std::min(T.gain_i0, rg.i0); T.gain_i1 = std::max(T.gain_i1, rg.i1);
            T.gain_j0 = std::min(T.gain_j0, rg.j0); T.gain_j1 = std::max(T.gain_j1, rg.j1);
            T.gain_k0 = std::min(T.gain_k0, rg.k0); T.gain_k1 = std::max(T.gain_k1, rg.k1);
        }
    }

    // Point probes (PointFieldDetector::initialize, src/detectors/point_field_detector.hpp:191-205).
    for (const auto& p : pf.list("POINT_FIELD_DETECTORS")) {
        require(p.size() >= 6, "POINT_FIELD_DETECTORS entry needs: enabled, name, x, y, z, component...");
        if (!parse_bool(p[0])) continue;
        PointProbe pr;
        pr.name = p[1];
        std::size_t ijk[3];
        for (int a = 0; a < 3; ++a) {
            std::size_t v = S.grid.physical_to_index(a, field(p, 2 + a) - S.domain_min[a]);
            const std::size_t N = a == 0 ? S.NxT : a == 1 ? S.NyT : S.NzT;
            ijk[a] = std::max(std::size_t(1), std::min(v, N - 2));
        }
        pr.i = ijk[0]; pr.j = ijk[1]; pr.k = ijk[2];
        for (std::size_t c = 5; c < p.size(); ++c) {
            int comp = int(parse_num(p[c]));
            require(comp >= 0 && comp <= 11, "POINT_FIELD_DETECTORS component must be 0..11");
            pr.components.push_back(comp);
        }
        S.probes.push_back(pr);
    }
    return S;
}

// ================================================================ material rows
// Each thread numbers the rows of its chunk (a cell equal to the previous one costs one
// compare, which is nearly every cell: materials are piecewise constant), then the chunk
// tables are merged in chunk order.
namespace {
struct RowKey {
    uint64_t b[3];
    bool operator==(const RowKey& o) const { return b[0] == o.b[0] && b[1] == o.b[1] && b[2] == o.b[2]; }
};
struct RowHash {
    size_t operator()(const RowKey& k) const {
        uint64_t h = k.b[0] * 0x9E3779B97F4A7C15ull;
        h ^= (k.b[1] + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full;
        h ^= (k.b[2] + 0x165667B19E3779F9ull) * 0x85EBCA77C2B2AE63ull;
        return size_t(h ^ (h >> 29));
    }
};

}  // namespace

bool distinct_rows(const double* const bE[3], size_t N, std::vector<std::array<double, 3>>& rows,
                    std::vector<uint16_t>& idx) {
    constexpr size_t kMaxRows = 65535;
    const int P = std::max(1, omp_get_max_threads());
    idx.resize(N);
    std::vector<std::vector<RowKey>> local(P);
    int over = 0, used = 1;
#pragma omp parallel num_threads(P) reduction(| : over)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        if (t == 0) used = nt;
        const size_t lo = N * size_t(t) / size_t(nt), hi = N * size_t(t + 1) / size_t(nt);
        std::unordered_map<RowKey, uint16_t, RowHash> map;
        RowKey prev{};
        unsigned prev_id = ~0u;
        for (size_t q = lo; q < hi; ++q) {
            RowKey k;
            std::memcpy(&k.b[0], bE[0] + q, 8);
            std::memcpy(&k.b[1], bE[1] + q, 8);
            std::memcpy(&k.b[2], bE[2] + q, 8);
            if (prev_id != ~0u && k == prev) { idx[q] = uint16_t(prev_id); continue; }
            auto it = map.find(k);
            unsigned id;
            if (it == map.end()) {
                if (local[t].size() >= kMaxRows) { over = 1; break; }
                id = unsigned(local[t].size());
                map.emplace(k, uint16_t(id));
                local[t].push_back(k);
            } else {
                id = it->second;
            }
            idx[q] = uint16_t(id);
            prev = k;
            prev_id = id;
        }
    }
    if (over) return false;
    std::unordered_map<RowKey, uint16_t, RowHash> global;
    std::vector<std::vector<uint16_t>> remap(P);
    rows.clear();
    for (int t = 0; t < P; ++t) {
        for (const RowKey& k : local[t]) {
            auto it = global.find(k);
            if (it == global.end()) {
                if (rows.size() >= kMaxRows) return false;
                it = global.emplace(k, uint16_t(rows.size())).first;
                std::array<double, 3> r;
                std::memcpy(r.data(), k.b, 24);
                rows.push_back(r);
            }
            remap[t].push_back(it->second);
        }
    }
#pragma omp parallel for schedule(static)
    for (int t = 0; t < used; ++t) {  // the chunks of the first pass
        const size_t lo = N * size_t(t) / size_t(used), hi = N * size_t(t + 1) / size_t(used);
        for (size_t q = lo; q < hi; ++q) idx[q] = remap[t][idx[q]];
    }
    return true;
}


}  // namespace fdtd
