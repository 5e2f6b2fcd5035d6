// setup.hpp -- host-side setup API of the B200 FDTD stepper.
//
// This is the part of the reference solver that stays on the host: the runtime
// parameter file (the reference's compile-time UserConfig, src/user_config.hpp:11-211),
// the non-uniform auto-mesher (src/auto_mesh_generator.hpp), the structure scene and
// its 2x2x2 subpixel bake (src/structure_material.hpp), the CPML 1-D profiles
// (src/boundary.hpp:303-373), the dipole source (src/sources/*.hpp) and the two-level
// gain regions (src/two_level_system.hpp:17-110,421-571).  Every routine reproduces
// the reference's double-precision arithmetic step for step, so mesh lines, material
// coefficients and gain masks come out bit-identical; the CUDA stepper consumes the
// result through the plain-data fdtd_setup_v1 view declared in include/fdtd_b200.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <array>
#include <string>
#include <vector>

namespace fdtd {

using real = double;

// Physical constants exactly as the reference defines them (src/global_function.hpp:12-19).
namespace phys {
inline constexpr real PI = 3.141592653589793238462643383279502884;
inline constexpr real C0 = 299792458.0;
inline constexpr real EPS0 = 8.854187817e-12;
inline constexpr real MU0 = 4.0 * PI * 1e-7;
inline constexpr real HBAR = 1.054571817e-34;
}  // namespace phys

inline std::size_t idx3(std::size_t i, std::size_t j, std::size_t k, std::size_t Ny, std::size_t Nz) {
    return (i * Ny + j) * Nz + k;
}

// ---------------------------------------------------------------- parameter file
// Scalars keyed by the UserConfig names; list entries ("KEY += a, b, ...") keyed by the
// name of the UserConfig vector they extend, fields in that struct's declaration order.
struct ParamFile {
    std::map<std::string, std::string> scalars;
    std::map<std::string, std::vector<std::vector<std::string>>> lists;

    static ParamFile parse(const std::string& text);  // throws std::runtime_error
    double num(const std::string& key, double dflt) const;
    bool flag(const std::string& key, bool dflt) const;
    std::string str(const std::string& key, const std::string& dflt) const;
    const std::vector<std::vector<std::string>>& list(const std::string& key) const;
};

// ---------------------------------------------------------------- grid spacing
// Mirror of GridSpacing (src/global_function.hpp:92-158).
struct GridSpacing {
    std::vector<real> dx, dy, dz;
    std::vector<real> inv_dx, inv_dy, inv_dz;
    std::vector<real> x_bounds, y_bounds, z_bounds;
    std::size_t npml = 0;

    void compute_inverses();
    real pml_offset(int axis) const;
    std::size_t physical_to_index(int axis, real phys) const;
    real cell_center_physical(int axis, std::size_t i) const;
    const std::vector<real>& bounds(int axis) const { return axis == 0 ? x_bounds : axis == 1 ? y_bounds : z_bounds; }
    const std::vector<real>& spacing(int axis) const { return axis == 0 ? dx : axis == 1 ? dy : dz; }
};

void build_cumulative_bounds(const std::vector<real>& spacing, std::vector<real>& bounds);

// The distinct (bEx, bEy, bEz) rows of N cells and each cell's row number (idx3 order), rows
// compared bit for bit; false when there are more than 65535 rows.
bool distinct_rows(const double* const bE[3], std::size_t N, std::vector<std::array<double, 3>>& rows,
                   std::vector<uint16_t>& idx);

// ---------------------------------------------------------------- auto mesher
// Mirrors of MeshOverrideRegion / AutoMeshConfig / AutoMeshStructureBounds
// (src/auto_mesh_generator.hpp:52-116,118-126).
struct MeshOverrideRegion {
    bool enabled = false;
    real x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
    real dx = 10e-9, dy = 10e-9, dz = 10e-9;
    int priority = 0;
};

enum class PmlStrategy { UNIFORM, GRADED };

struct AutoMeshConfig {
    real lambda_min = 300e-9;
    real f_max = 0;
    int mesh_accuracy = 2;
    real ppw_override = 0;
    real dx_min = 1e-9;
    real dx_max = 100e-9;
    real max_grading_ratio = 1.41421356237;
    std::size_t npml = 0;
    PmlStrategy pml_strategy = PmlStrategy::UNIFORM;
    bool mesh_override_enabled = false;
    std::vector<MeshOverrideRegion> override_regions;

    real ppw_target() const;
    real lambda_min_eff() const;
};

struct StructureBounds {
    real x_min, x_max, y_min, y_max, z_min, z_max;
    real n_material;
};

// AutoMeshGenerator::generate (src/auto_mesh_generator.hpp:156-253).
GridSpacing automesh_generate(const AutoMeshConfig& cfg, real domain_x, real domain_y, real domain_z,
                              std::size_t npml, const std::vector<StructureBounds>& structures,
                              real background_n);

// ---------------------------------------------------------------- CPML profiles
// CPMLConfig (src/boundary.hpp:18-25) and the 1-D coefficient arrays that
// CPMLBoundary::build_profiles_and_coeffs (src/boundary.hpp:303-373) produces.
struct CpmlConfig {
    int npml = 8;
    real m = 3.0;
    real Rerr = 1e-10;
    real alpha0 = 0.05;
    real kappa_max = 8.0;
    bool alpha_linear = true;
};

struct CpmlProfiles {
    int npml = 0;
    // index 0/1/2 = x/y/z axis, each of length N_axis
    std::vector<real> kappa[3], sigma[3], alpha[3];
    std::vector<real> bE[3], cE[3], bH[3], cH[3];
};

CpmlProfiles build_cpml_profiles(const GridSpacing& g, const CpmlConfig& cfg, real dt);

// ---------------------------------------------------------------- scene / bake
struct Material {  // src/structure_material.hpp:16-30
    real eps_r = 1.0, mu_r = 1.0, sigma = 0.0, sigma_m = 0.0;
};
Material make_nk(real n);

enum class ShapeType { Box, Sphere, CylinderZ };

struct Shape {  // Box / Sphere / CylinderZ (src/structure_material.hpp:50-85)
    ShapeType type = ShapeType::Box;
    real a[6] = {0, 0, 0, 0, 0, 0};  // box: x0,x1,y0,y1,z0,z1; sphere: cx,cy,cz,r; cyl: cx,cy,r,z0,z1
    bool contains(real x, real y, real z) const;
    void bounding_box(real bb[6]) const;
};

struct TlsMaterialDef {  // TLSMaterials::TLSMaterial (src/tls_materials.hpp:11-18)
    std::string name;
    real lambda0 = 1500e-9, gamma = 7e12, tau = 1e-12, N0 = 1e25, inversion_fraction = 1.0;
};

struct StructureItem {
    Shape shape;
    Material mat;
    bool tls_enabled = false;
    TlsMaterialDef tls;
};

// MaterialGrids (src/global_function.hpp:70-90), idx3 layout.
struct MaterialGrids {
    std::size_t NxT = 0, NyT = 0, NzT = 0;
    std::vector<real> aE[3], bE[3], aH[3], bH[3];
    // Set by the GPU bake, which only makes bE: aE = aH = 1 everywhere and bH = bH_value
    // everywhere (the aE/aH/bH arrays are then left empty).
    bool uniform_ah = false;
    real bH_value = 0;
};

// Spatial bins over the scene items (CSR): the items whose bounding box overlaps a bin,
// newest first, so the first one containing a point is the last-defined one.
struct ItemBins {
    real lo[3], w[3];
    std::size_t nb[3];
    std::vector<uint32_t> start, ids;  // bin b holds ids[start[b] .. start[b+1])
    std::size_t bin(int a, real v) const {
        const real t = (v - lo[a]) / w[a];
        if (!(t > 0)) return 0;  // also catches NaN
        const std::size_t b = std::size_t(t);
        return b >= nb[a] ? nb[a] - 1 : b;
    }
};

struct Scene {
    std::size_t NxT = 0, NyT = 0, NzT = 0, npml_cells = 0;
    GridSpacing grid;
    Material bg;
    std::vector<StructureItem> items;

    // StructureScene::bake (src/structure_material.hpp:211-288); threads over cells,
    // bit-identical to the serial reference loop.
    void bake(MaterialGrids& mg, real dt, real eps0, real mu0, int subpixel_samples) const;
    void n_grid(std::vector<real>& out) const;  // make_n_grid_from_scene (:291-310)
};

ItemBins make_item_bins(const std::vector<StructureItem>& items, const GridSpacing& g);

// The same bake for bE on the current CUDA device, bit-identical to Scene::bake with 8
// samples (every product and sum rounded on its own, in the same order).  Only for
// lossless, non-magnetic items (sigma = sigma_m = 0, mu_r = 1, what make_nk gives): returns
// false otherwise, and the caller bakes on the host.  Throws std::runtime_error when no
// CUDA device can be used.
bool gpu_bake(const Scene& sc, MaterialGrids& mg, real dt, real eps0, real mu0);

// ---------------------------------------------------------------- sources
enum class Waveform { Ricker = 0, GaussianModulatedSine = 1, RickerLikeGaussian2nd = 2, ContinuousWave = 3 };

// compute_waveform (src/sources/isource.hpp:41-68)
real compute_waveform(Waveform w, real t, real I0, real f0, real tau, real t0, real t_shift);

struct DipoleSource {  // src/sources/dipole_source.hpp:11-85
    std::size_t i = 0, j = 0, k = 0;
    int polarization = 2;  // 0..5 = Ex,Ey,Ez,Hx,Hy,Hz; Hx/Hy/Hz drive Jx/Jy/Jz
    real cell_area = 1.0;
    real I0 = 0, f0 = 0, tau = 0, t0 = 0, t_shift = 0;
    Waveform waveform = Waveform::Ricker;
    int j_component() const { return polarization % 3; }
    // Jval(n) = I((n + 1/2) dt) / cell_area, the value inject_half_step adds.
    real current_density(std::size_t n, real dt) const;
};

struct PlaneWave {  // PlaneWaveSource (src/sources/plane_wave_source.hpp:19-72,201-290)
    int axis = 2, comp = 0;     // propagation axis; J component driven (-1: none)
    std::size_t plane = 0, lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0;
    real d = 1, sign = 1;
    Waveform waveform = Waveform::GaussianModulatedSine;
    real E0 = 0, f0 = 0, tau = 0, t0 = 0, t_shift = 0;
};

// ---------------------------------------------------------------- two-level gain
struct TlsParams {  // TwoLevelParams (src/two_level_system.hpp:17-110)
    real lambda0 = 1500e-9, omega_a = 0, gamma = 7e12, tau = 1e-12, mu_z = 0, N0_total = 1e25;
    real hbar = phys::HBAR;
    bool enable_population_clamp = false;
    real kapa_coeff = 0, pa2 = 0, pa3 = 0, inv_dt = 0;
    bool coefficients_initialized = false;
    real pump_rate = 0;  // build extension: W_p (1/s), adds W_p*Ng to dNu/dt; 0 = reference physics
    void finalize(real c0 = 299792458.0, real eps0 = 8.854187817e-12, real hbar_in = 1.054571817e-34);
    void finalize_with_dt(real dt);
};

struct TlsRegion {  // TLSRegion (src/two_level_system.hpp:421-497)
    std::size_t i0 = 0, i1 = 0, j0 = 0, j1 = 0, k0 = 0, k1 = 0;
    TlsParams params;
    real inversion_fraction = 1.0;
    Shape shape;
    bool contains(std::size_t i, std::size_t j, std::size_t k, const GridSpacing& g) const;
};

struct TlsSetup {
    std::vector<TlsRegion> regions;
    std::vector<int32_t> cell_region_map;  // idx3, -1 = no gain
    // initial per-cell state of the gain cells (idx3; zero elsewhere)
    std::vector<real> Nu, Ng, Ndip;
    std::size_t gain_i0 = 0, gain_i1 = 0, gain_j0 = 0, gain_j1 = 0, gain_k0 = 0, gain_k1 = 0;
    bool enabled() const { return !regions.empty(); }
};

// ---------------------------------------------------------------- detectors
struct PointProbe {  // PointFieldDetector (src/detectors/point_field_detector.hpp:150-255)
    std::string name;
    std::size_t i = 0, j = 0, k = 0;  // clamped to [1, N-2] like the reference
    std::vector<int> components;      // FieldComponent codes 0..11
};

// ---------------------------------------------------------------- whole setup
struct SimSetup {
    ParamFile params;
    bool auto_mesh = false;
    std::size_t NxT = 0, NyT = 0, NzT = 0, npml = 0;
    std::size_t Nx_core = 0, Ny_core = 0, Nz_core = 0;
    real dt = 0, S = 0.99;
    std::size_t n_steps = 0, save_every = 1;
    real domain_min[3] = {0, 0, 0}, domain_max[3] = {0, 0, 0};
    GridSpacing grid;
    CpmlConfig cpml_cfg;
    CpmlProfiles cpml;
    bool boundary_pec = false;
    Scene scene;
    MaterialGrids mats;
    std::vector<DipoleSource> sources;
    std::vector<PlaneWave> plane_waves;
    TlsSetup tls;
    std::vector<PointProbe> probes;
    // build-only keys
    std::vector<real> dft_freqs;
    std::string precision = "fp32";  // fp32 | fp64 | fp16 | bf16
    bool stochastic_rounding = false;  // ROUNDING = stochastic (build-only key; BF16 storage)
    real field_scale = 0;            // FP16/BF16 storage scale sE (0 = automatic)
    real noise_amplitude = 0;
    uint64_t seed = 1;
    std::size_t stability_interval = 10;
    real stability_max_E = 1e10, stability_max_P = 1e5, stability_conservation = 0.01, stability_growth = 10.0;

    // Runs the reference setup sequence (src/3D_FDTD_version008.cpp:37-172) on a parameter
    // file; bake=false stops after the mesh, CPML and dt (mesh-only use).  Throws
    // std::runtime_error with a message on invalid input.
    static SimSetup from_params(const ParamFile& pf, bool bake = true);
};

}  // namespace fdtd
