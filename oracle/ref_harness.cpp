// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle side).
//
// Drives the reference solver XiaofengYuChina/3D_FDTD_version008 itself: this file
// #includes the reference headers where they lie (include path set by oracle/Makefile)
// and replays the reference's own setup and serial time loop on a runtime parameter
// file, then dumps every array the GPU path is checked against.  Nothing here is
// linked into the product; only tests/, bench.py's reference arm and the golden
// fixture generator run the binary this file builds (oracle/_ref/ref_harness).
//
// Mirrors:
//   setup         src/3D_FDTD_version008.cpp:37-172 (P.finalize, packages,
//                 make_context, bake_and_bind(…, 8), sources, TLS regions)
//   packages      src/params.hpp:518-678 (structure bounds / override regions /
//                 structures / dipole sources), with the lists taken from the
//                 parameter file instead of the compile-time UserConfig vectors
//   time loop     src/3D_FDTD_version008.cpp:269-328 (serial / OpenMP path)
//   point probe   src/detectors/point_field_detector.hpp:195-201,242-255
//
// Usage: ref_harness PARAMS OUTDIR [--steps N] [--mesh-only] [--dump-materials]
//                    [--init DIR] [--no-fields]
// OUTDIR receives <name>.f64 / <name>.i32 raw little-endian arrays and meta.json.

#include "params.hpp"
#include "fdtd_stepper.hpp"
#include "boundary.hpp"
#include "structure_material.hpp"
#include "two_level_system.hpp"
#include "stability_monitor.hpp"
#include "two_level_detectors.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::vector<std::string> split_csv(const std::string& s) {
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

bool to_bool(const std::string& v) {
    return v == "1" || v == "true" || v == "TRUE" || v == "True";
}

// Parsed parameter file: scalars by UserConfig name, list entries by vector name.
struct ParamFile {
    std::map<std::string, std::string> scalars;
    std::map<std::string, std::vector<std::vector<std::string>>> lists;

    double num(const std::string& k, double dflt) const {
        auto it = scalars.find(k);
        return it == scalars.end() ? dflt : std::strtod(it->second.c_str(), nullptr);
    }
    bool flag(const std::string& k, bool dflt) const {
        auto it = scalars.find(k);
        return it == scalars.end() ? dflt : to_bool(it->second);
    }
    const std::vector<std::vector<std::string>>& list(const std::string& k) const {
        static const std::vector<std::vector<std::string>> empty;
        auto it = lists.find(k);
        return it == lists.end() ? empty : it->second;
    }
};

ParamFile parse_params(const std::string& path) {
    ParamFile pf;
    std::ifstream f(path);
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
    std::string line;
    while (std::getline(f, line)) {
        auto hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        auto pluseq = line.find("+=");
        if (pluseq != std::string::npos) {
            pf.lists[trim(line.substr(0, pluseq))].push_back(split_csv(line.substr(pluseq + 2)));
            continue;
        }
        auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        pf.scalars[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    return pf;
}

double d(const std::vector<std::string>& v, size_t i) {
    return i < v.size() ? std::strtod(v[i].c_str(), nullptr) : 0.0;
}

struct TLSMat { std::string name; double lambda0, gamma, tau, N0, inv; };

void write_f64(const std::string& dir, const std::string& name, const std::vector<double>& v) {
    std::ofstream o(dir + "/" + name + ".f64", std::ios::binary);
    o.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
}
void write_i32(const std::string& dir, const std::string& name, const std::vector<int>& v) {
    std::ofstream o(dir + "/" + name + ".i32", std::ios::binary);
    o.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(int)));
}
bool read_f64(const std::string& path, std::vector<double>& v) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.read(reinterpret_cast<char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
    return bool(f);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s PARAMS OUTDIR [--steps N] [--warmup W] [--mesh-only] [--dump-materials] [--init DIR] [--no-fields] [--detectors]\n", argv[0]);
        return 2;
    }
    const std::string params_path = fs::absolute(argv[1]).string();
    const std::string outdir = fs::absolute(argv[2]).string();
    long long steps_override = -1, warmup = 0;
    bool mesh_only = false, dump_materials = false, dump_fields = true, with_detectors = false;
    std::string init_dir;
    for (int a = 3; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--steps" && a + 1 < argc) steps_override = std::atoll(argv[++a]);
        else if (s == "--warmup" && a + 1 < argc) warmup = std::max(0LL, std::atoll(argv[++a]));
        else if (s == "--mesh-only") mesh_only = true;
        else if (s == "--dump-materials") dump_materials = true;
        else if (s == "--no-fields") dump_fields = false;
        else if (s == "--detectors") with_detectors = true;
        else if (s == "--init" && a + 1 < argc) init_dir = fs::absolute(argv[++a]).string();
    }
    fs::create_directories(outdir);
    const ParamFile pf = parse_params(params_path);

    // ---- Config::sim equivalent (src/params.hpp:823-868), values from the file ----
    Config::SimulationParams P;
    P.mesh_mode = (int(pf.num("MESH_MODE", UserConfig::MESH_MODE)) == 0) ? Config::MeshMode::UNIFORM
                                                                         : Config::MeshMode::AUTO_NONUNIFORM;
    P.dx_uniform = pf.num("DX_UNIFORM", UserConfig::DX_UNIFORM);
    P.dy_uniform = pf.num("DY_UNIFORM", UserConfig::DY_UNIFORM);
    P.dz_uniform = pf.num("DZ_UNIFORM", UserConfig::DZ_UNIFORM);
    P.Nx = size_t(pf.num("NX", double(UserConfig::NX)));
    P.Ny = size_t(pf.num("NY", double(UserConfig::NY)));
    P.Nz = size_t(pf.num("NZ", double(UserConfig::NZ)));
    P.lambda0 = pf.num("LAMBDA0", UserConfig::LAMBDA0);
    P.domain_x_min = pf.num("DOMAIN_X_MIN", UserConfig::DOMAIN_X_MIN);
    P.domain_x_max = pf.num("DOMAIN_X_MAX", UserConfig::DOMAIN_X_MAX);
    P.domain_y_min = pf.num("DOMAIN_Y_MIN", UserConfig::DOMAIN_Y_MIN);
    P.domain_y_max = pf.num("DOMAIN_Y_MAX", UserConfig::DOMAIN_Y_MAX);
    P.domain_z_min = pf.num("DOMAIN_Z_MIN", UserConfig::DOMAIN_Z_MIN);
    P.domain_z_max = pf.num("DOMAIN_Z_MAX", UserConfig::DOMAIN_Z_MAX);
    P.S = pf.num("CFL_FACTOR", UserConfig::CFL_FACTOR);
    P.nSteps = size_t(pf.num("N_STEPS", double(UserConfig::N_STEPS)));
    P.saveEvery = size_t(pf.num("SAVE_EVERY", double(UserConfig::SAVE_EVERY)));
    P.probe_x = pf.num("PROBE_X", UserConfig::PROBE_X);
    P.probe_y = pf.num("PROBE_Y", UserConfig::PROBE_Y);
    P.probe_z = pf.num("PROBE_Z", UserConfig::PROBE_Z);
    P.bp.type = (int(pf.num("BOUNDARY_TYPE", UserConfig::BOUNDARY_TYPE)) == 0) ? BcType::PEC : BcType::CPML_RC;
    if (pf.scalars.count("RUN_TAG")) P.run_tag = pf.scalars.at("RUN_TAG");
    P.writeFloat64 = pf.flag("WRITE_FLOAT64", UserConfig::WRITE_FLOAT64);
    P.bp.cpml.npml = int(pf.num("CPML_NPML", UserConfig::CPML_NPML));
    P.bp.cpml.m = pf.num("CPML_M", UserConfig::CPML_M);
    P.bp.cpml.Rerr = pf.num("CPML_RERR", UserConfig::CPML_RERR);
    P.bp.cpml.alpha0 = pf.num("CPML_ALPHA0", UserConfig::CPML_ALPHA0);
    P.bp.cpml.kappa_max = pf.num("CPML_KAPPA_MAX", UserConfig::CPML_KAPPA_MAX);
    P.bp.cpml.alpha_linear = pf.flag("CPML_ALPHA_LINEAR", UserConfig::CPML_ALPHA_LINEAR);
    P.auto_mesh_config.lambda_min = P.lambda0;
    P.auto_mesh_config.mesh_accuracy = int(pf.num("AUTO_MESH_ACCURACY", UserConfig::AUTO_MESH_ACCURACY));
    P.auto_mesh_config.ppw_override = pf.num("AUTO_MESH_PPW_OVERRIDE", UserConfig::AUTO_MESH_PPW_OVERRIDE);
    P.auto_mesh_config.dx_min = pf.num("AUTO_MESH_DX_MIN", UserConfig::AUTO_MESH_DX_MIN);
    P.auto_mesh_config.dx_max = pf.num("AUTO_MESH_DX_MAX", UserConfig::AUTO_MESH_DX_MAX);
    P.auto_mesh_config.max_grading_ratio = pf.num("AUTO_MESH_MAX_GRADING_RATIO", UserConfig::AUTO_MESH_MAX_GRADING_RATIO);
    const bool override_enabled = pf.flag("MESH_OVERRIDE_ENABLED", UserConfig::MESH_OVERRIDE_ENABLED);
    P.auto_mesh_config.mesh_override_enabled = override_enabled;
    const bool tls_enabled_cfg = pf.flag("TLS_ENABLED", UserConfig::TLS_ENABLED);
    const bool tls_clamp = pf.flag("TLS_ENABLE_CLAMP", UserConfig::TLS_ENABLE_CLAMP);
    const double background_n = pf.num("BACKGROUND_N", UserConfig::BACKGROUND_N);

    std::vector<TLSMat> tls_library;
    for (const auto& e : pf.list("TLS_MATERIALS"))
        tls_library.push_back({e.at(0), d(e, 1), d(e, 2), d(e, 3), d(e, 4), d(e, 5)});
    auto find_tls = [&](const std::string& name) -> const TLSMat* {
        if (name.empty()) return nullptr;
        for (const auto& m : tls_library) if (m.name == name) return &m;
        return nullptr;
    };

    P.finalize();

    // ---- register_structure_bounds_for_auto_mesh / register_mesh_override_regions ----
    if (P.mesh_mode == Config::MeshMode::AUTO_NONUNIFORM) {
        Config::clear_structure_bounds();
        for (const auto& s : pf.list("STRUCTURES")) {
            const std::string& type = s.at(0);
            const double n = d(s, 1);
            if (type == "box") {
                Config::register_structure_bounds(d(s, 2), d(s, 3), d(s, 4), d(s, 5), d(s, 6), d(s, 7), n);
            } else if (type == "sphere") {
                double cx = d(s, 2), cy = d(s, 3), cz = d(s, 4), r = d(s, 5);
                Config::register_structure_bounds(cx - r, cx + r, cy - r, cy + r, cz - r, cz + r, n);
            } else if (type == "cylinder") {
                double cx = d(s, 2), cy = d(s, 3), r = d(s, 4), z0 = d(s, 5), z1 = d(s, 6);
                Config::register_structure_bounds(cx - r, cx + r, cy - r, cy + r, z0, z1, n);
            }
        }
        P.auto_mesh_config.override_regions.clear();
        if (!override_enabled) {
            P.auto_mesh_config.mesh_override_enabled = false;
        } else {
            P.auto_mesh_config.mesh_override_enabled = true;
            for (const auto& r : pf.list("MESH_OVERRIDE_REGIONS")) {
                if (!to_bool(r.at(0))) continue;
                MeshOverrideRegion region;
                region.enabled = true;
                region.x0 = d(r, 1); region.x1 = d(r, 2);
                region.y0 = d(r, 3); region.y1 = d(r, 4);
                region.z0 = d(r, 5); region.z1 = d(r, 6);
                region.dx = d(r, 7); region.dy = d(r, 8); region.dz = d(r, 9);
                region.priority = 0;
                P.auto_mesh_config.override_regions.push_back(region);
            }
        }
    }

    // ---- structure package (register_default_structures, src/params.hpp:557-592) ----
    Config::g_structure_pkgs.clear();
    Config::g_structure_pkgs.push_back([&](StructureScene& scene) {
        scene.bg = make_nk(background_n);
        real pml_x = scene.grid_spacing.x_bounds[scene.npml_cells];
        real pml_y = scene.grid_spacing.y_bounds[scene.npml_cells];
        real pml_z = scene.grid_spacing.z_bounds[scene.npml_cells];
        for (const auto& s : pf.list("STRUCTURES")) {
            Material mat = make_nk(d(s, 1));
            StructureTLSConfig tls_cfg;
            const TLSMat* tm = find_tls(s.size() > 8 ? s[8] : std::string());
            if (tm && tls_enabled_cfg) {
                tls_cfg.enabled = true;
                tls_cfg.lambda0 = tm->lambda0;
                tls_cfg.gamma = tm->gamma;
                tls_cfg.tau = tm->tau;
                tls_cfg.N0 = tm->N0;
                tls_cfg.inversion_fraction = tm->inv;
            }
            const std::string& type = s.at(0);
            if (type == "box") {
                scene.add_box(AABB{pml_x + d(s, 2), pml_x + d(s, 3), pml_y + d(s, 4), pml_y + d(s, 5),
                                   pml_z + d(s, 6), pml_z + d(s, 7)}, mat, tls_cfg);
            } else if (type == "sphere") {
                scene.add_sphere(pml_x + d(s, 2), pml_y + d(s, 3), pml_z + d(s, 4), d(s, 5), mat, tls_cfg);
            } else if (type == "cylinder") {
                scene.add_cylinder_z(pml_x + d(s, 2), pml_y + d(s, 3), d(s, 4), pml_z + d(s, 5), pml_z + d(s, 6),
                                     mat, tls_cfg);
            }
        }
    });

    // make_context writes frames/<run_tag>/ files relative to the working directory.
    fs::current_path(outdir);
    Config::SimContext ctx = Config::make_context(P);

    const size_t NxT = ctx.NxT, NyT = ctx.NyT, NzT = ctx.NzT;
    std::ostringstream meta;
    meta.precision(17);
    meta << "{\n  \"NxT\": " << NxT << ", \"NyT\": " << NyT << ", \"NzT\": " << NzT
         << ", \"npml\": " << ctx.npml << ",\n  \"dt\": " << ctx.dt << ",\n";

    const std::string od = ".";
    write_f64(od, "x_bounds", ctx.grid_spacing.x_bounds);
    write_f64(od, "y_bounds", ctx.grid_spacing.y_bounds);
    write_f64(od, "z_bounds", ctx.grid_spacing.z_bounds);
    write_f64(od, "dx", ctx.grid_spacing.dx);
    write_f64(od, "dy", ctx.grid_spacing.dy);
    write_f64(od, "dz", ctx.grid_spacing.dz);
    write_f64(od, "inv_dx", ctx.grid_spacing.inv_dx);
    write_f64(od, "inv_dy", ctx.grid_spacing.inv_dy);
    write_f64(od, "inv_dz", ctx.grid_spacing.inv_dz);
    if (mesh_only) {
        meta << "  \"mesh_only\": true\n}\n";
        std::ofstream("meta.json") << meta.str();
        return 0;
    }

    if (auto* cp = dynamic_cast<CPMLBoundary*>(ctx.bc.get())) {
        write_f64(od, "cpml_kx", cp->kx_); write_f64(od, "cpml_ky", cp->ky_); write_f64(od, "cpml_kz", cp->kz_);
        write_f64(od, "cpml_bEx", cp->bEx_); write_f64(od, "cpml_cEx", cp->cEx_);
        write_f64(od, "cpml_bEy", cp->bEy_); write_f64(od, "cpml_cEy", cp->cEy_);
        write_f64(od, "cpml_bEz", cp->bEz_); write_f64(od, "cpml_cEz", cp->cEz_);
        write_f64(od, "cpml_bHx", cp->bHx_); write_f64(od, "cpml_cHx", cp->cHx_);
        write_f64(od, "cpml_bHy", cp->bHy_); write_f64(od, "cpml_cHy", cp->cHy_);
        write_f64(od, "cpml_bHz", cp->bHz_); write_f64(od, "cpml_cHz", cp->cHz_);
    }

    Config::apply_structure_packages(ctx);
    Config::bake_and_bind(ctx, P, /*subpixel_samples=*/8);

    if (dump_materials) {
        write_f64(od, "bEx", ctx.mats.bEx); write_f64(od, "bEy", ctx.mats.bEy); write_f64(od, "bEz", ctx.mats.bEz);
        write_f64(od, "aEx", ctx.mats.aEx); write_f64(od, "aEy", ctx.mats.aEy); write_f64(od, "aEz", ctx.mats.aEz);
        write_f64(od, "bHx", ctx.mats.bHx); write_f64(od, "bHy", ctx.mats.bHy); write_f64(od, "bHz", ctx.mats.bHz);
        write_f64(od, "aHx", ctx.mats.aHx); write_f64(od, "aHy", ctx.mats.aHy); write_f64(od, "aHz", ctx.mats.aHz);
        std::vector<real> n_grid;
        make_n_grid_from_scene(ctx.scene, n_grid);
        write_f64(od, "n_grid", n_grid);
    }

    // ---- sources (register_default_sources, src/params.hpp:594-678: dipoles, then plane waves) ----
    Config::Runtime rt;
    meta << "  \"sources\": [";
    bool first_src = true;
    for (const auto& s : pf.list("DIPOLE_SOURCES")) {
        if (!to_bool(s.at(0))) continue;
        Sources::SourceConfig cfg;
        cfg.x = d(s, 1); cfg.y = d(s, 2); cfg.z = d(s, 3);
        cfg.amplitude = d(s, 4); cfg.frequency = d(s, 5); cfg.wavelength = d(s, 6);
        cfg.tau = d(s, 7); cfg.df_fwhm = d(s, 8); cfg.t0_factor = d(s, 9);
        switch (int(d(s, 10))) {
            case 1: cfg.waveform = Sources::Waveform::GaussianModulatedSine; break;
            case 2: cfg.waveform = Sources::Waveform::RickerLikeGaussian2nd; break;
            case 3: cfg.waveform = Sources::Waveform::ContinuousWave; break;
            default: cfg.waveform = Sources::Waveform::Ricker; break;
        }
        const int pol = int(d(s, 11));
        cfg.polarization = static_cast<Sources::Polarization>((pol >= 0 && pol <= 5) ? pol : 2);
        auto src = Sources::make_dipole_source(cfg, ctx.grid_spacing, ctx.NyT, ctx.NzT, ctx.dt,
                                               P.domain_x_min, P.domain_y_min, P.domain_z_min);
        auto* dp = static_cast<Sources::DipoleSource*>(src.get());
        meta << (first_src ? "" : ", ") << "{\"i\": " << dp->i << ", \"j\": " << dp->j << ", \"k\": " << dp->k
             << ", \"cell_area\": " << dp->cell_area << ", \"I0\": " << dp->I0 << ", \"f0\": " << dp->f0
             << ", \"tau\": " << dp->tau << ", \"t0\": " << dp->t0 << ", \"t_shift\": " << dp->t_shift
             << ", \"waveform\": " << int(dp->waveform) << ", \"polarization\": " << int(dp->polarization) << "}";
        first_src = false;
        rt.sources.push_back(std::move(src));
    }
    meta << "],\n";
    for (const auto& s : pf.list("PLANE_WAVE_SOURCES")) {  // src/params.hpp:643-679
        if (!to_bool(s.at(0))) continue;
        Sources::PlaneWaveConfig cfg;
        cfg.injection_position = d(s, 1);
        cfg.amplitude = d(s, 2); cfg.frequency = d(s, 3); cfg.wavelength = d(s, 4);
        cfg.tau = d(s, 5); cfg.df_fwhm = d(s, 6); cfg.t0_factor = d(s, 7);
        switch (int(d(s, 8))) {
            case 1: cfg.waveform = Sources::Waveform::GaussianModulatedSine; break;
            case 2: cfg.waveform = Sources::Waveform::RickerLikeGaussian2nd; break;
            case 3: cfg.waveform = Sources::Waveform::ContinuousWave; break;
            default: cfg.waveform = Sources::Waveform::Ricker; break;
        }
        const int dir = int(d(s, 9));
        cfg.direction = static_cast<Sources::PlaneWaveDirection>((dir >= 0 && dir <= 5) ? dir : 4);
        const int pol = int(d(s, 10));
        cfg.polarization = static_cast<Sources::Polarization>((pol >= 0 && pol <= 5) ? pol : 2);
        cfg.x_min = d(s, 11); cfg.x_max = d(s, 12); cfg.y_min = d(s, 13);
        cfg.y_max = d(s, 14); cfg.z_min = d(s, 15); cfg.z_max = d(s, 16);
        rt.sources.push_back(Sources::make_plane_wave_source(cfg, ctx.grid_spacing, ctx.NxT, ctx.NyT, ctx.NzT,
                                                             ctx.npml, ctx.dt, P.domain_x_min, P.domain_y_min,
                                                             P.domain_z_min));
    }

    std::vector<real> Ex(NxT * NyT * NzT, 0), Ey(Ex), Ez(Ex), Hx(Ex), Hy(Ex), Hz(Ex), Jx(Ex), Jy(Ex), Jz(Ex);
    if (!init_dir.empty()) {
        read_f64(init_dir + "/Ex.f64", Ex); read_f64(init_dir + "/Ey.f64", Ey); read_f64(init_dir + "/Ez.f64", Ez);
        read_f64(init_dir + "/Hx.f64", Hx); read_f64(init_dir + "/Hy.f64", Hy); read_f64(init_dir + "/Hz.f64", Hz);
    }

    // ---- TLS (src/3D_FDTD_version008.cpp:100-172) ----
    TwoLevelState tls_state;
    TLSRegionManager tls_manager;
    const bool any_tls = tls_enabled_cfg && ctx.scene.has_any_tls();
    if (any_tls) {
        tls_state.allocate(NxT, NyT, NzT);
        auto tls_structures = ctx.scene.get_tls_structures();
        for (size_t idx = 0; idx < tls_structures.size(); ++idx) {
            const auto* item = tls_structures[idx];
            const auto& tc = item->tls_config;
            AABB bb = item->shape->bounding_box();
            real pml_x = ctx.grid_spacing.x_bounds[ctx.npml];
            real pml_y = ctx.grid_spacing.y_bounds[ctx.npml];
            real pml_z = ctx.grid_spacing.z_bounds[ctx.npml];
            TwoLevelParams rp;
            rp.lambda0 = tc.lambda0; rp.gamma = tc.gamma; rp.tau = tc.tau; rp.N0_total = tc.N0;
            rp.enable_population_clamp = tls_clamp;
            tls_manager.add_region_from_structure(ctx.grid_spacing, bb.x0 - pml_x, bb.x1 - pml_x, bb.y0 - pml_y,
                                                  bb.y1 - pml_y, bb.z0 - pml_z, bb.z1 - pml_z, rp,
                                                  tc.inversion_fraction, item->shape.get(),
                                                  "structure_" + std::to_string(idx));
        }
        tls_manager.initialize(tls_state, ctx.grid_spacing);
        tls_manager.finalize_with_dt(ctx.dt);
        if (tls_manager.num_regions() > 0) {  // gain bounding box (src/3D_FDTD_version008.cpp:146-163)
            const auto& r0 = tls_manager.regions[0];
            tls_state.gain_i0 = r0.i0; tls_state.gain_i1 = r0.i1;
            tls_state.gain_j0 = r0.j0; tls_state.gain_j1 = r0.j1;
            tls_state.gain_k0 = r0.k0; tls_state.gain_k1 = r0.k1;
            for (size_t r = 1; r < tls_manager.num_regions(); ++r) {
                const auto& rg = tls_manager.regions[r];
                tls_state.gain_i0 = std::min(tls_state.gain_i0, rg.i0); tls_state.gain_i1 = std::max(tls_state.gain_i1, rg.i1);
                tls_state.gain_j0 = std::min(tls_state.gain_j0, rg.j0); tls_state.gain_j1 = std::max(tls_state.gain_j1, rg.j1);
                tls_state.gain_k0 = std::min(tls_state.gain_k0, rg.k0); tls_state.gain_k1 = std::max(tls_state.gain_k1, rg.k1);
            }
        }
        write_i32(od, "tls_region_map", tls_manager.cell_region_map);
        write_f64(od, "tls_Ndip", tls_state.Ndip);
        if (!init_dir.empty()) {
            std::vector<double> tmp(NxT * NyT * NzT);
            if (read_f64(init_dir + "/Pz.f64", tmp)) tls_state.Pz = tmp;
            if (read_f64(init_dir + "/Pz_prev.f64", tmp)) tls_state.Pz_prev = tmp;
            if (read_f64(init_dir + "/Nu.f64", tmp)) tls_state.Nu = tmp;
            if (read_f64(init_dir + "/Ng.f64", tmp)) tls_state.Ng = tmp;
        }
    }
    meta << "  \"tls_regions\": [";
    for (size_t r = 0; r < tls_manager.regions.size(); ++r) {
        const auto& rg = tls_manager.regions[r];
        const auto& pr = rg.params;
        meta << (r ? ", " : "") << "{\"i0\": " << rg.i0 << ", \"i1\": " << rg.i1 << ", \"j0\": " << rg.j0
             << ", \"j1\": " << rg.j1 << ", \"k0\": " << rg.k0 << ", \"k1\": " << rg.k1
             << ", \"kapa_coeff\": " << pr.kapa_coeff << ", \"pa2\": " << pr.pa2 << ", \"pa3\": " << pr.pa3
             << ", \"inv_dt\": " << pr.inv_dt << ", \"tau\": " << pr.tau << ", \"hbar\": " << pr.hbar
             << ", \"omega_a\": " << pr.omega_a << ", \"mu_z\": " << pr.mu_z << ", \"N0\": " << pr.N0_total
             << ", \"inversion_fraction\": " << rg.inversion_fraction << "}";
    }
    meta << "],\n";

    // ---- point probes (PointFieldDetector::initialize index clamp) ----
    struct Probe { size_t id; std::vector<int> comps; };
    std::vector<Probe> probes;
    meta << "  \"probes\": [";
    for (const auto& p : pf.list("POINT_FIELD_DETECTORS")) {
        if (!to_bool(p.at(0))) continue;
        size_t i0 = ctx.grid_spacing.physical_to_index_x(d(p, 2) - P.domain_x_min);
        size_t j0 = ctx.grid_spacing.physical_to_index_y(d(p, 3) - P.domain_y_min);
        size_t k0 = ctx.grid_spacing.physical_to_index_z(d(p, 4) - P.domain_z_min);
        i0 = std::max(size_t(1), std::min(i0, NxT - 2));
        j0 = std::max(size_t(1), std::min(j0, NyT - 2));
        k0 = std::max(size_t(1), std::min(k0, NzT - 2));
        Probe pr{idx3(i0, j0, k0, NyT, NzT), {}};
        for (size_t c = 5; c < p.size(); ++c) pr.comps.push_back(int(d(p, c)));
        meta << (probes.empty() ? "" : ", ") << "{\"i\": " << i0 << ", \"j\": " << j0 << ", \"k\": " << k0
             << ", \"ncomp\": " << pr.comps.size() << "}";
        probes.push_back(pr);
    }
    meta << "],\n";

    // ---- detectors (register_default_detectors, src/params.hpp:681-790, lists from the file) ----
    std::vector<std::unique_ptr<Detectors::IDetector>> dets;
    if (with_detectors) {
        const fs::path out_root = fs::path("frames") / P.run_tag;
        std::vector<real> n_grid;
        make_n_grid_from_scene(ctx.scene, n_grid);
        auto comp = [](int fc) {
            return (fc >= 0 && fc <= 11) ? static_cast<Detectors::FieldComponent>(fc) : Detectors::FieldComponent::Ez;
        };
        for (const auto& m : pf.list("MESH_DETECTORS")) {
            if (!to_bool(m.at(0))) continue;
            Detectors::MeshDetectorConfig cfg;
            cfg.name = m.at(1); cfg.slice_position = d(m, 2); cfg.slice_plane = int(d(m, 3));
            cfg.export_mesh_lines = to_bool(m.at(4)); cfg.export_spacing_arrays = to_bool(m.at(5));
            auto det = Detectors::make_mesh_detector(out_root, cfg, NxT, NyT, NzT, ctx.Nx_core, ctx.Ny_core,
                                                     ctx.Nz_core, ctx.npml, ctx.grid_spacing, P.domain_size_x(),
                                                     P.domain_size_y(), P.domain_size_z(), P.domain_x_min,
                                                     P.domain_y_min, P.domain_z_min);
            det->save_index_slice(n_grid);
            det->save_mesh_info();
            dets.push_back(std::move(det));
        }
        for (const auto& m : pf.list("FIELD_MOVIE_2D_DETECTORS")) {
            if (!to_bool(m.at(0))) continue;
            Detectors::FieldMovie2DConfig cfg;
            cfg.name = m.at(1); cfg.component = comp(int(d(m, 2))); cfg.slice_plane = int(d(m, 3));
            cfg.slice_position = d(m, 4); cfg.frame_pattern = m.at(5);
            cfg.save_every = P.saveEvery; cfg.n_steps = P.nSteps; cfg.write_float64 = P.writeFloat64;
            dets.push_back(Detectors::make_field_movie_2d(out_root, cfg, NxT, NyT, NzT, ctx.Nx_core, ctx.Ny_core,
                                                          ctx.Nz_core, ctx.npml, ctx.grid_spacing, P.domain_size_x(),
                                                          P.domain_size_y(), P.domain_size_z(), P.domain_x_min,
                                                          P.domain_y_min, P.domain_z_min));
        }
        for (const auto& m : pf.list("POINT_FIELD_DETECTORS")) {
            if (!to_bool(m.at(0))) continue;
            Detectors::PointFieldDetectorConfig cfg;
            cfg.name = m.at(1); cfg.x = d(m, 2); cfg.y = d(m, 3); cfg.z = d(m, 4);
            cfg.save_every = P.saveEvery; cfg.n_steps = P.nSteps; cfg.write_float64 = P.writeFloat64;
            cfg.components.clear();
            for (size_t c = 5; c < m.size(); ++c) cfg.components.push_back(comp(int(d(m, c))));
            dets.push_back(Detectors::make_point_field_detector(out_root, cfg, NxT, NyT, NzT, ctx.npml,
                                                                ctx.grid_spacing, ctx.dt, P.domain_x_min,
                                                                P.domain_y_min, P.domain_z_min));
        }
    }

    // ---- two-level detectors (src/3D_FDTD_version008.cpp:174-198), with the gain ----
    std::unique_ptr<PopulationTimeSeriesDetector> pop_detector;
    std::unique_ptr<PolarizationDiagnostics> pol_diagnostics;
    std::unique_ptr<TLSGlobalHistory> tls_global_history;
    if (with_detectors && any_tls) {
        const fs::path out_root = fs::path("frames") / P.run_tag;
        const size_t ic = ctx.grid_spacing.physical_to_index_x(P.probe_x - P.domain_x_min);
        const size_t jc = ctx.grid_spacing.physical_to_index_y(P.probe_y - P.domain_y_min);
        const size_t kc = ctx.grid_spacing.physical_to_index_z(P.probe_z - P.domain_z_min);
        pop_detector = std::make_unique<PopulationTimeSeriesDetector>(out_root, "populations", NxT, NyT, NzT,
                                                                      P.saveEvery, P.nSteps, P.dt, ctx.grid_spacing);
        pol_diagnostics = std::make_unique<PolarizationDiagnostics>(out_root, "polarization", NxT, NyT, NzT, ic, jc,
                                                                    kc, P.saveEvery, P.dt);
        tls_global_history = std::make_unique<TLSGlobalHistory>(out_root, tls_state, ctx.grid_spacing, P.saveEvery,
                                                                P.dt, false);
    }

    // ---- time loop (src/3D_FDTD_version008.cpp:269-328, serial path) ----
    const size_t nsteps = steps_override >= 0 ? size_t(steps_override) : P.nSteps;
    std::vector<double> probe_series;
    // the first `warmup` steps run untimed; loop_seconds covers the remaining steps, and
    // step_seconds lists each timed step
    const size_t warm = std::min<size_t>(size_t(warmup), nsteps);
    std::vector<double> step_s;
    auto t_begin = std::chrono::steady_clock::now();
    auto t_step = t_begin;
    for (size_t n = 0; n < nsteps; ++n) {
        if (n == warm) t_begin = t_step = std::chrono::steady_clock::now();
        std::fill(Jx.begin(), Jx.end(), 0.0);
        std::fill(Jy.begin(), Jy.end(), 0.0);
        std::fill(Jz.begin(), Jz.end(), 0.0);
        for (auto& src : rt.sources) src->inject_half_step(n, ctx.dt, Jx, Jy, Jz);
        if (any_tls) update_polarization_multi_region(NxT, NyT, NzT, tls_manager, Ez, tls_state);
        fdtd_update_H(NxT, NyT, NzT, ctx.grid_spacing.dx.data(), ctx.grid_spacing.dy.data(),
                      ctx.grid_spacing.dz.data(), ctx.grid_spacing.inv_dx.data(), ctx.grid_spacing.inv_dy.data(),
                      ctx.grid_spacing.inv_dz.data(), ctx.mats.aHx.data(), ctx.mats.bHx.data(), ctx.mats.aHy.data(),
                      ctx.mats.bHy.data(), ctx.mats.aHz.data(), ctx.mats.bHz.data(), Ex.data(), Ey.data(),
                      Ez.data(), Hx.data(), Hy.data(), Hz.data());
        ctx.bc->apply_after_H(Ex, Ey, Ez, Hx, Hy, Hz);
        if (any_tls) {
            fdtd_update_E_with_gain(NxT, NyT, NzT, ctx.grid_spacing.dx.data(), ctx.grid_spacing.dy.data(),
                                    ctx.grid_spacing.dz.data(), ctx.grid_spacing.inv_dx.data(),
                                    ctx.grid_spacing.inv_dy.data(), ctx.grid_spacing.inv_dz.data(),
                                    ctx.mats.aEx.data(), ctx.mats.bEx.data(), ctx.mats.aEy.data(),
                                    ctx.mats.bEy.data(), ctx.mats.aEz.data(), ctx.mats.bEz.data(), Ex.data(),
                                    Ey.data(), Ez.data(), Hx.data(), Hy.data(), Hz.data(), Jx.data(), Jy.data(),
                                    Jz.data(), tls_state);
        } else {
            fdtd_update_E(NxT, NyT, NzT, ctx.grid_spacing.dx.data(), ctx.grid_spacing.dy.data(),
                          ctx.grid_spacing.dz.data(), ctx.grid_spacing.inv_dx.data(), ctx.grid_spacing.inv_dy.data(),
                          ctx.grid_spacing.inv_dz.data(), ctx.mats.aEx.data(), ctx.mats.bEx.data(),
                          ctx.mats.aEy.data(), ctx.mats.bEy.data(), ctx.mats.aEz.data(), ctx.mats.bEz.data(),
                          Ex.data(), Ey.data(), Ez.data(), Hx.data(), Hy.data(), Hz.data(), Jx.data(), Jy.data(),
                          Jz.data());
        }
        ctx.bc->apply_after_E(Ex, Ey, Ez, Hx, Hy, Hz);
        for (auto& det : dets) det->record_after_E(n, ctx.dt, Ex, Ey, Ez, Hx, Hy, Hz);
        if (n % P.saveEvery == 0) {
            for (const auto& pr : probes)
                for (int c : pr.comps)
                    probe_series.push_back(Detectors::get_field_value(static_cast<Detectors::FieldComponent>(c),
                                                                      pr.id, Ex, Ey, Ez, Hx, Hy, Hz));
        }
        if (any_tls) update_populations_multi_region(NxT, NyT, NzT, ctx.dt, tls_manager, Ez, tls_state);
        if (pop_detector) pop_detector->record(n, tls_state);
        if (pol_diagnostics) pol_diagnostics->record(n, tls_state, Ez, ctx.grid_spacing);
        if (tls_global_history) tls_global_history->record(n, tls_state);
        if (n >= warm) {
            const auto now = std::chrono::steady_clock::now();
            step_s.push_back(std::chrono::duration<double>(now - t_step).count());
            t_step = now;
        }
    }
    if (warm == nsteps) t_begin = std::chrono::steady_clock::now();
    if (pop_detector) pop_detector->finalize(tls_state);
    if (tls_global_history) tls_global_history->finalize();
    auto t_end = std::chrono::steady_clock::now();
    for (auto& det : dets) det->finalize();
    const double loop_s = std::chrono::duration<double>(t_end - t_begin).count();
    meta << "  \"steps\": " << nsteps << ", \"warmup_steps\": " << warm << ", \"loop_seconds\": " << loop_s
         << ", \"threads\": " << omp_get_max_threads() << ", \"step_seconds\": [";
    for (size_t q = 0; q < step_s.size(); ++q) meta << (q ? ", " : "") << step_s[q];
    meta << "],\n";

    // Diagnostics at the final state (src/stability_monitor.hpp:155-178,
    // src/two_level_system.hpp:344-418).
    StabilityMonitor sm(1e300, 1e300, 1e300, 1e300);
    meta << "  \"max_E\": " << sm.get_max_E(Ex, Ey, Ez);
    if (any_tls) {
        meta << ", \"conservation_error\": " << sm.calculate_conservation_error(tls_state)
             << ", \"integrated_Nu\": " << compute_integrated_Nu(tls_state, ctx.grid_spacing)
             << ", \"integrated_Ng\": " << compute_integrated_Ng(tls_state, ctx.grid_spacing)
             << ", \"polarization_energy\": " << compute_polarization_energy(tls_state, Ez, ctx.grid_spacing)
             << ", \"max_P\": " << NumericUtils::max_abs(tls_state.Pz);
    }
    meta << ",\n  \"any_tls\": " << (any_tls ? "true" : "false") << "\n}\n";

    write_f64(od, "probe_series", probe_series);
    if (dump_fields) {
        write_f64(od, "Ex", Ex); write_f64(od, "Ey", Ey); write_f64(od, "Ez", Ez);
        write_f64(od, "Hx", Hx); write_f64(od, "Hy", Hy); write_f64(od, "Hz", Hz);
        if (any_tls) {
            write_f64(od, "Pz", tls_state.Pz); write_f64(od, "Pz_prev", tls_state.Pz_prev);
            write_f64(od, "Nu", tls_state.Nu); write_f64(od, "Ng", tls_state.Ng);
        }
    }
    std::ofstream("meta.json") << meta.str();
    return 0;
}
