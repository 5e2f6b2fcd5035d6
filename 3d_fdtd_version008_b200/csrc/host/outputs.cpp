// outputs.cpp -- the reference's run-directory and detector files (see outputs.hpp).
//
// Every text file is written with the same stream settings as the reference's writer
// (default 6 significant digits for grid_spacing.txt / coordinate_mapping.txt,
// setprecision(15) for the JSON and mesh-line files, setprecision(18) for a point
// detector's dt), so the files are byte-identical to the reference's for the same setup.
#include "outputs.hpp"

#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace fdtd {
namespace fs = std::filesystem;

namespace {

std::string unquote(std::string s) {
    if (s.size() >= 2 && s.front() == '"' && s.back() == '"') s = s.substr(1, s.size() - 2);
    return s;
}

bool as_bool(const std::string& v, const char* what) {
    if (v == "1" || v == "true" || v == "TRUE" || v == "True") return true;
    if (v == "0" || v == "false" || v == "FALSE" || v == "False") return false;
    throw std::runtime_error(std::string(what) + ": not a boolean: '" + v + "'");
}

double as_num(const std::vector<std::string>& f, std::size_t i, const char* what) {
    if (i >= f.size() || f[i].empty()) return 0.0;
    char* end = nullptr;
    const double x = std::strtod(f[i].c_str(), &end);
    if (end == f[i].c_str() || *end != '\0') throw std::runtime_error(std::string(what) + ": not a number: '" + f[i] + "'");
    return x;
}

// A frame pattern may hold one integer conversion (%d with flags and a width) and %%; the
// reference hands it to snprintf as the format.
void check_pattern(const std::string& p) {
    int conversions = 0;
    for (std::size_t q = 0; q < p.size(); ++q) {
        if (p[q] != '%') continue;
        if (q + 1 < p.size() && p[q + 1] == '%') { ++q; continue; }
        std::size_t r = q + 1;
        while (r < p.size() && std::string("-+ 0#").find(p[r]) != std::string::npos) ++r;
        while (r < p.size() && p[r] >= '0' && p[r] <= '9') ++r;
        if (r >= p.size() || p[r] != 'd') throw std::runtime_error("frame pattern '" + p + "': only %d conversions are allowed");
        ++conversions;
        q = r;
    }
    if (conversions > 1) throw std::runtime_error("frame pattern '" + p + "' has more than one conversion");
}

// Detector names become directory names under the run directory.
void check_name(const std::string& n, const char* what) {
    if (n.empty() || n == "." || n == ".." || n.find('/') != std::string::npos || n.find('\\') != std::string::npos)
        throw std::runtime_error(std::string(what) + " name '" + n + "' is not a plain directory name");
}

const char* plane_name(int p) { return p == 0 ? "XY" : p == 1 ? "XZ" : p == 2 ? "YZ" : "Unknown"; }

// Slice index of a plane at a physical position (the three initialize() functions).
void slice_of(const SimSetup& S, int plane, real pos, std::size_t& index, real& coord) {
    const int axis = plane == 0 ? 2 : plane == 1 ? 1 : 0;
    const std::size_t N = axis == 0 ? S.NxT : axis == 1 ? S.NyT : S.NzT;
    std::size_t i = S.grid.physical_to_index(axis, pos - S.domain_min[axis]);
    index = std::max(std::size_t(1), std::min(i, N - 2));
    coord = S.grid.cell_center_physical(axis, index);
}

std::ofstream open_text(const fs::path& p) {
    std::ofstream f(p);
    if (!f) throw std::runtime_error("cannot write " + p.string());
    return f;
}

void write_values(std::ofstream& f, const std::vector<double>& v, bool f64) {
    if (f64) {
        f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
    } else {
        std::vector<float> w(v.begin(), v.end());
        f.write(reinterpret_cast<const char*>(w.data()), std::streamsize(w.size() * sizeof(float)));
    }
}

void slice_dims(const SimSetup& S, int plane, std::size_t& d1, std::size_t& d2) {
    d1 = plane == 2 ? S.NyT : S.NxT;
    d2 = plane == 0 ? S.NyT : S.NzT;
}

}  // namespace

const char* component_name(int c) {  // field_component_name (src/detectors/idetector.hpp:31-50)
    static const char* names[] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "E_mag", "H_mag", "Sx", "Sy", "Sz", "S_mag"};
    return (c >= 0 && c < 12) ? names[c] : "Unknown";
}

OutputPlan make_output_plan(const SimSetup& S) {
    const ParamFile& pf = S.params;
    OutputPlan plan;
    plan.run_tag = unquote(pf.str("RUN_TAG", plan.run_tag));
    if (plan.run_tag.empty() || plan.run_tag.find("..") != std::string::npos || plan.run_tag.front() == '/')
        throw std::runtime_error("RUN_TAG must be a relative directory name");
    plan.float64 = pf.flag("WRITE_FLOAT64", true);
    auto comp = [](double c) { return (c >= 0 && c <= 11) ? int(c) : 2; };  // to_field_component's default: Ez
    for (const auto& m : pf.list("MESH_DETECTORS")) {  // MeshDetectorDef order (src/user_config.hpp:104-111)
        if (m.size() < 6) throw std::runtime_error("MESH_DETECTORS entry needs: enabled, name, position, plane, lines, spacing");
        if (!as_bool(m[0], "MESH_DETECTORS")) continue;
        MeshDetectorPlan d;
        d.name = m[1];
        check_name(d.name, "MESH_DETECTORS");
        d.plane = int(as_num(m, 3, "MESH_DETECTORS"));
        if (d.plane < 0 || d.plane > 2) throw std::runtime_error("MESH_DETECTORS slice plane must be 0, 1 or 2");
        slice_of(S, d.plane, as_num(m, 2, "MESH_DETECTORS"), d.index, d.coord);
        d.mesh_lines = as_bool(m[4], "MESH_DETECTORS");
        d.spacing = as_bool(m[5], "MESH_DETECTORS");
        plan.meshes.push_back(d);
    }
    for (const auto& m : pf.list("FIELD_MOVIE_2D_DETECTORS")) {  // FieldMovie2DDef (src/user_config.hpp:118-125)
        if (m.size() < 6)
            throw std::runtime_error("FIELD_MOVIE_2D_DETECTORS entry needs: enabled, name, component, plane, position, pattern");
        if (!as_bool(m[0], "FIELD_MOVIE_2D_DETECTORS")) continue;
        MoviePlan v;
        v.name = m[1];
        check_name(v.name, "FIELD_MOVIE_2D_DETECTORS");
        v.component = comp(as_num(m, 2, "FIELD_MOVIE_2D_DETECTORS"));
        v.plane = int(as_num(m, 3, "FIELD_MOVIE_2D_DETECTORS"));
        if (v.plane < 0 || v.plane > 2) throw std::runtime_error("FIELD_MOVIE_2D_DETECTORS slice plane must be 0, 1 or 2");
        slice_of(S, v.plane, as_num(m, 4, "FIELD_MOVIE_2D_DETECTORS"), v.index, v.coord);
        v.pattern = m[5];
        check_pattern(v.pattern);
        slice_dims(S, v.plane, v.dim1, v.dim2);
        plan.movies.push_back(v);
    }
    for (const auto& p : S.probes) {
        PointPlan q;
        q.name = p.name;
        check_name(q.name, "POINT_FIELD_DETECTORS");
        q.i = p.i; q.j = p.j; q.k = p.k;
        q.components = p.components;
        q.px = S.grid.cell_center_physical(0, p.i);
        q.py = S.grid.cell_center_physical(1, p.j);
        q.pz = S.grid.cell_center_physical(2, p.k);
        plan.points.push_back(q);
    }
    plan.NxT = S.NxT; plan.NyT = S.NyT; plan.NzT = S.NzT;
    plan.save_every = S.save_every; plan.n_steps = S.n_steps; plan.dt = S.dt;
    plan.tls = S.tls.enabled();
    if (plan.tls) {  // src/3D_FDTD_version008.cpp:175-180 (P.probe_* from PROBE_X/Y/Z)
        const real pr[3] = {pf.num("PROBE_X", 2000e-9), pf.num("PROBE_Y", 2000e-9), pf.num("PROBE_Z", 500e-9)};
        std::size_t ix[3];
        for (int a = 0; a < 3; ++a) ix[a] = S.grid.physical_to_index(a, pr[a] - S.domain_min[a]);
        plan.mon_i = ix[0]; plan.mon_j = ix[1]; plan.mon_k = ix[2];
        plan.mon_valid = ix[0] < S.NxT && ix[1] < S.NyT && ix[2] < S.NzT;
    }
    return plan;
}

std::string inversion_line(uint64_t n, double dt, double total_Nu, double total_Ng) {
    const double inversion = total_Nu - total_Ng, denom = total_Nu + total_Ng;
    const double inv_fraction = (denom > 1e-30) ? (inversion / denom) : 0.0;
    const real t = real(n) * dt;
    std::ostringstream o;
    o << std::setprecision(18) << t << "," << total_Nu << "," << total_Ng << "," << inversion << "," << inv_fraction
      << "\n";
    return o.str();
}

std::string polarization_line(uint64_t n, double dt, double Pz_center, double dPz_dt_center, double P_energy) {
    const real t = real(n) * dt;
    std::ostringstream o;
    o << std::setprecision(18) << t << "," << Pz_center << "," << dPz_dt_center << "," << P_energy << "\n";
    return o.str();
}

std::string global_history_line(uint64_t n, double dt, double Nu_total, double Ng_total) {
    const double Ntotal = Nu_total + Ng_total, inversion_total = Nu_total - Ng_total;
    double Nu_percent = 0.0, Ng_percent = 0.0, inv_norm = 0.5;
    if (Ntotal > 1e-30) {
        Nu_percent = Nu_total / Ntotal;
        Ng_percent = Ng_total / Ntotal;
        inv_norm = (inversion_total / Ntotal + 1.0) / 2.0;
    }
    const double t_fs = double(n) * dt * 1e15;
    std::ostringstream o;
    o << n << "," << std::setprecision(6) << std::fixed << t_fs << "," << std::setprecision(12) << std::scientific
      << Nu_total << "," << Ng_total << "," << inversion_total << "," << std::setprecision(8) << std::fixed
      << Nu_percent << "," << Ng_percent << "," << inv_norm << "\n";
    return o.str();
}

void write_population_metadata(const OutputPlan& S, const std::string& root) {
    const OutputPlan& plan = S;
    const fs::path p = fs::path(run_dir(plan, root)) / "populations" / "metadata_populations.json";
    std::ofstream meta(p);
    if (!meta) throw std::runtime_error("cannot write " + p.string());
    meta << "{\n"
         << "  \"NxT\": " << S.NxT << ",\n"
         << "  \"NyT\": " << S.NyT << ",\n"
         << "  \"NzT\": " << S.NzT << ",\n"
         << "  \"saveEvery\": " << S.save_every << ",\n"
         << "  \"nSteps\": " << S.n_steps << ",\n"
         << "  \"dt\": " << std::setprecision(18) << S.dt << ",\n"
         << "  \"dtype\": \"float64\",\n"
         << "  \"binary_frames\": 2,\n"
         << "  \"binary_mode\": \"first_and_last\",\n"
         << "  \"binary_data_units\": \"m^-3 (density)\",\n"
         << "  \"csv_total_units\": \"atoms (integrated)\",\n"
         << "  \"what\": \"population_densities_Nu_and_Ng_vs_time\"\n"
         << "}\n";
}

std::string run_dir(const OutputPlan& plan, const std::string& root) {
    return (fs::path(root) / "frames" / plan.run_tag).string();
}

std::string frame_path(const OutputPlan& plan, const std::string& root, std::size_t m, uint64_t frame) {
    char fname[128];  // the reference's buffer: longer names are cut at 127 characters
    std::snprintf(fname, sizeof(fname), plan.movies[m].pattern.c_str(), int(frame));
    return (fs::path(run_dir(plan, root)) / plan.movies[m].name / fname).string();
}

void write_setup_outputs(const SimSetup& S, const OutputPlan& plan, const std::string& root) {
    const fs::path dir = run_dir(plan, root);
    std::error_code ec;
    fs::create_directories(dir, ec);
    if (ec) throw std::runtime_error("cannot create " + dir.string() + ": " + ec.message());
    const GridSpacing& g = S.grid;
    const std::size_t np = S.npml;
    const char* mode = S.auto_mesh ? "AUTO_NONUNIFORM" : "UNIFORM";

    {  // grid_spacing.txt (src/params.hpp:297-308)
        auto f = open_text(dir / "grid_spacing.txt");
        f << "# Mode: " << mode << "\n";
        f << "# dx\n"; for (auto v : g.dx) f << v << "\n";
        f << "# dy\n"; for (auto v : g.dy) f << v << "\n";
        f << "# dz\n"; for (auto v : g.dz) f << v << "\n";
        f << "# x_bounds\n"; for (auto v : g.x_bounds) f << v << "\n";
        f << "# y_bounds\n"; for (auto v : g.y_bounds) f << v << "\n";
        f << "# z_bounds\n"; for (auto v : g.z_bounds) f << v << "\n";
    }
    const real core_min[3] = {g.x_bounds[np], g.y_bounds[np], g.z_bounds[np]};
    const real core_max[3] = {g.x_bounds[S.NxT - np], g.y_bounds[S.NyT - np], g.z_bounds[S.NzT - np]};
    {  // coordinate_mapping.txt (src/params.hpp:310-393)
        auto f = open_text(dir / "coordinate_mapping.txt");
        const std::size_t NT[3] = {S.NxT, S.NyT, S.NzT};
        const char* ax = "xyz";
        f << "# Coordinate System Mapping Diagnostics\n";
        f << "# =====================================\n\n";
        f << "# Total Domain (includes PML)\n";
        for (int a = 0; a < 3; ++a) {
            f << "total_" << ax[a] << "_min_nm = " << g.bounds(a).front() * 1e9 << "\n";
            f << "total_" << ax[a] << "_max_nm = " << g.bounds(a).back() * 1e9 << "\n";
        }
        f << "\n# Core Region indices\n";
        for (int a = 0; a < 3; ++a) {
            const char c = "ijk"[a];
            f << c << "_core_start = " << np << "\n";
            f << c << "_core_end = " << (NT[a] - np) << "\n";
        }
        f << "\n# Core Region in total coordinates (nm)\n";
        for (int a = 0; a < 3; ++a) {
            f << "core_" << ax[a] << "_min_total_nm = " << core_min[a] * 1e9 << "\n";
            f << "core_" << ax[a] << "_max_total_nm = " << core_max[a] * 1e9 << "\n";
        }
        f << "\n# PML Offsets (nm)\n";
        for (int a = 0; a < 3; ++a) f << "pml_offset_" << ax[a] << "_nm = " << g.pml_offset(a) * 1e9 << "\n";
        f << "\n# Physical domain size (nm)\n";
        for (int a = 0; a < 3; ++a) f << "phys_size_" << ax[a] << "_nm = " << (core_max[a] - core_min[a]) * 1e9 << "\n";
    }
    {  // mesh_info.json (src/params.hpp:395-505)
        const real phys[3] = {core_max[0] - core_min[0], core_max[1] - core_min[1], core_max[2] - core_min[2]};
        real target[3] = {phys[0] / 2.0, phys[1] / 2.0, phys[2] / 2.0};  // first enabled dipole, else the centre
        for (const auto& d : S.params.list("DIPOLE_SOURCES")) {
            if (d.empty() || !as_bool(d[0], "DIPOLE_SOURCES")) continue;
            for (int a = 0; a < 3; ++a) target[a] = as_num(d, 1 + a, "DIPOLE_SOURCES") - S.domain_min[a];
            break;
        }
        std::size_t si[3];
        real actual[3];
        for (int a = 0; a < 3; ++a) {
            si[a] = g.physical_to_index(a, target[a]);
            actual[a] = g.cell_center_physical(a, si[a]);
        }
        auto mm = [](const std::vector<real>& v) { return std::minmax_element(v.begin(), v.end()); };
        const auto ex = mm(g.dx), ey = mm(g.dy), ez = mm(g.dz);
        const auto& structs = S.params.list("STRUCTURES");
        auto f = open_text(dir / "mesh_info.json");
        f << std::setprecision(15);
        f << "{\n";
        f << "  \"mode\": \"" << mode << "\",\n";
        f << "  \"NxT\": " << S.NxT << ",\n";
        f << "  \"NyT\": " << S.NyT << ",\n";
        f << "  \"NzT\": " << S.NzT << ",\n";
        f << "  \"npml\": " << np << ",\n";
        f << "  \"dx_min_nm\": " << *ex.first * 1e9 << ",\n";
        f << "  \"dx_max_nm\": " << *ex.second * 1e9 << ",\n";
        f << "  \"dy_min_nm\": " << *ey.first * 1e9 << ",\n";
        f << "  \"dy_max_nm\": " << *ey.second * 1e9 << ",\n";
        f << "  \"dz_min_nm\": " << *ez.first * 1e9 << ",\n";
        f << "  \"dz_max_nm\": " << *ez.second * 1e9 << ",\n";
        f << "  \"domain_x_nm\": " << g.x_bounds.back() * 1e9 << ",\n";
        f << "  \"domain_y_nm\": " << g.y_bounds.back() * 1e9 << ",\n";
        f << "  \"domain_z_nm\": " << g.z_bounds.back() * 1e9 << ",\n";
        f << "  \"dt_fs\": " << S.dt * 1e15 << ",\n";
        f << "  \"lambda0_nm\": " << S.params.num("LAMBDA0", 1500e-9) * 1e9 << ",\n";
        f << "  \"source_x_target_nm\": " << target[0] * 1e9 << ",\n";
        f << "  \"source_y_target_nm\": " << target[1] * 1e9 << ",\n";
        f << "  \"source_z_target_nm\": " << target[2] * 1e9 << ",\n";
        f << "  \"source_i\": " << si[0] << ",\n";
        f << "  \"source_j\": " << si[1] << ",\n";
        f << "  \"source_k\": " << si[2] << ",\n";
        f << "  \"source_x_actual_nm\": " << actual[0] * 1e9 << ",\n";
        f << "  \"source_y_actual_nm\": " << actual[1] * 1e9 << ",\n";
        f << "  \"source_z_actual_nm\": " << actual[2] * 1e9 << ",\n";
        for (int a = 0; a < 3; ++a) {
            f << "  \"phys_domain_" << "xyz"[a] << "_min_nm\": 0.0,\n";
            f << "  \"phys_domain_" << "xyz"[a] << "_max_nm\": " << phys[a] * 1e9 << ",\n";
        }
        f << "  \"grid_type\": \"bounds\",\n";
        f << "  \"grid_x_count\": " << g.x_bounds.size() << ",\n";
        f << "  \"grid_y_count\": " << g.y_bounds.size() << ",\n";
        f << "  \"grid_z_count\": " << g.z_bounds.size() << ",\n";
        f << "  \"num_structures\": " << structs.size();
        if (!structs.empty()) {
            f << ",\n  \"structures\": [\n";
            for (std::size_t i = 0; i < structs.size(); ++i) {
                const auto& s = structs[i];
                f << "    {\"type\": \"" << s[0] << "\", \"n\": " << as_num(s, 1, "STRUCTURES") << ", \"params_nm\": [";
                for (int j = 0; j < 6; ++j) {
                    f << as_num(s, 2 + j, "STRUCTURES") * 1e9;
                    if (j < 5) f << ", ";
                }
                f << "]}";
                if (i < structs.size() - 1) f << ",";
                f << "\n";
            }
            f << "  ]\n";
        } else {
            f << ",\n  \"structures\": []\n";
        }
        f << "}\n";
    }

    const real L[3] = {S.domain_max[0] - S.domain_min[0], S.domain_max[1] - S.domain_min[1],
                       S.domain_max[2] - S.domain_min[2]};
    // Common header of the mesh detector's and the movie's metadata.json.
    auto grid_block = [&](std::ofstream& f) {
        f << "  \"NxT\": " << S.NxT << ",\n";
        f << "  \"NyT\": " << S.NyT << ",\n";
        f << "  \"NzT\": " << S.NzT << ",\n";
        f << "  \"Nx_phys\": " << S.Nx_core << ",\n";
        f << "  \"Ny_phys\": " << S.Ny_core << ",\n";
        f << "  \"Nz_phys\": " << S.Nz_core << ",\n";
        f << "  \"npml\": " << np << ",\n";
    };
    auto offsets_block = [&](std::ofstream& f) {
        f << "  \"pml_offset_x_m\": " << g.pml_offset(0) << ",\n";
        f << "  \"pml_offset_y_m\": " << g.pml_offset(1) << ",\n";
        f << "  \"pml_offset_z_m\": " << g.pml_offset(2) << ",\n";
        f << "  \"Lx_phys_m\": " << L[0] << ",\n";
        f << "  \"Ly_phys_m\": " << L[1] << ",\n";
        f << "  \"Lz_phys_m\": " << L[2] << ",\n";
    };
    auto dims_block = [&](std::ofstream& f, int plane) {
        static const char* lab1[] = {"x", "x", "y"};
        static const char* lab2[] = {"y", "z", "z"};
        std::size_t d1, d2;
        slice_dims(S, plane, d1, d2);
        f << "  \"slice_dim1\": " << d1 << ",\n";
        f << "  \"slice_dim2\": " << d2 << ",\n";
        f << "  \"dim1_label\": \"" << lab1[plane] << "\",\n";
        f << "  \"dim2_label\": \"" << lab2[plane] << "\",\n";
        f << "  \"note\": \"row-major storage, dim1 varies fastest\"\n";
        f << "}\n";
    };

    if (!plan.meshes.empty()) {  // MeshDetector (src/detectors/mesh_detector.hpp:97-270)
        std::vector<real> n;
        S.scene.n_grid(n);
        if (n.size() != S.NxT * S.NyT * S.NzT) throw std::runtime_error("mesh detectors need a baked setup");
        for (const auto& d : plan.meshes) {
            const fs::path dd = dir / d.name;
            fs::create_directories(dd, ec);
            if (ec) throw std::runtime_error("cannot create " + dd.string());
            {
                std::vector<double> v;
                for (std::size_t a = 0; a < (d.plane == 2 ? S.NyT : S.NxT); ++a)
                    for (std::size_t b = 0; b < (d.plane == 0 ? S.NyT : S.NzT); ++b) {
                        const std::size_t i = d.plane == 2 ? d.index : a, j = d.plane == 0 ? b : d.plane == 1 ? d.index : a,
                                          k = d.plane == 0 ? d.index : b;
                        v.push_back(n[(i * S.NyT + j) * S.NzT + k]);
                    }
                std::ofstream f(dd / "refractive_index.raw", std::ios::binary);
                if (!f) throw std::runtime_error("cannot write " + (dd / "refractive_index.raw").string());
                write_values(f, v, true);  // MeshDetectorConfig::write_float64 stays true
            }
            {
                auto f = open_text(dd / "metadata.json");
                f << std::setprecision(15);
                f << "{\n";
                f << "  \"detector_type\": \"MeshDetector\",\n";
                f << "  \"slice_plane\": \"" << plane_name(d.plane) << "\",\n";
                f << "  \"slice_index\": " << d.index << ",\n";
                f << "  \"slice_physical_m\": " << d.coord << ",\n";
                f << "  \"slice_physical_nm\": " << d.coord * 1e9 << ",\n";
                grid_block(f);
                offsets_block(f);
                f << "  \"dtype\": \"float64\",\n";
                dims_block(f, d.plane);
            }
            if (d.mesh_lines) {
                static const char* up = "XYZ";
                for (int a = 0; a < 3; ++a) {
                    auto f = open_text(dd / (std::string(1, "xyz"[a]) + "_bounds.txt"));
                    f << std::setprecision(15);
                    f << "# " << up[a] << " cell boundaries (meters)\n";
                    for (auto v : g.bounds(a)) f << v << "\n";
                }
            }
            if (d.spacing) {
                for (int a = 0; a < 3; ++a) {
                    const std::string nm = std::string("d") + "xyz"[a];
                    auto f = open_text(dd / (nm + "_array.txt"));
                    f << std::setprecision(15);
                    f << "# " << nm << " spacing array (meters)\n";
                    for (auto v : g.spacing(a)) f << v << "\n";
                }
            }
        }
    }

    for (const auto& m : plan.movies) {  // FieldMovie2D::write_metadata (field_movie_2d.hpp:150-205)
        const fs::path dd = dir / m.name;
        fs::create_directories(dd, ec);
        if (ec) throw std::runtime_error("cannot create " + dd.string());
        auto f = open_text(dd / "metadata.json");
        f << std::setprecision(15);
        f << "{\n";
        f << "  \"detector_type\": \"FieldMovie2D\",\n";
        f << "  \"field_component\": \"" << component_name(m.component) << "\",\n";
        f << "  \"slice_plane\": \"" << plane_name(m.plane) << "\",\n";
        f << "  \"slice_index\": " << m.index << ",\n";
        f << "  \"slice_physical_m\": " << m.coord << ",\n";
        f << "  \"slice_physical_nm\": " << m.coord * 1e9 << ",\n";
        grid_block(f);
        f << "  \"save_every\": " << S.save_every << ",\n";
        f << "  \"n_steps\": " << S.n_steps << ",\n";
        f << "  \"frame_pattern\": \"" << m.pattern << "\",\n";
        offsets_block(f);
        f << "  \"dtype\": \"" << (plan.float64 ? "float64" : "float32") << "\",\n";
        dims_block(f, m.plane);
    }

    for (const auto& p : plan.points) {  // PointFieldDetector::write_metadata (point_field_detector.hpp:131-180)
        const fs::path dd = dir / p.name;
        fs::create_directories(dd, ec);
        if (ec) throw std::runtime_error("cannot create " + dd.string());
        for (int c : p.components) {
            std::ofstream t(dd / (std::string(component_name(c)) + "_ts.bin"), std::ios::binary | std::ios::trunc);
            if (!t) throw std::runtime_error("cannot write " + (dd / (std::string(component_name(c)) + "_ts.bin")).string());
        }
        auto f = open_text(dd / "metadata.json");
        f << std::setprecision(15);
        f << "{\n";
        f << "  \"detector_type\": \"PointFieldDetector\",\n";
        f << "  \"NxT\": " << S.NxT << ",\n";
        f << "  \"NyT\": " << S.NyT << ",\n";
        f << "  \"NzT\": " << S.NzT << ",\n";
        f << "  \"i0\": " << p.i << ",\n";
        f << "  \"j0\": " << p.j << ",\n";
        f << "  \"k0\": " << p.k << ",\n";
        f << "  \"probe_x_physical_m\": " << p.px << ",\n";
        f << "  \"probe_y_physical_m\": " << p.py << ",\n";
        f << "  \"probe_z_physical_m\": " << p.pz << ",\n";
        f << "  \"probe_x_physical_nm\": " << p.px * 1e9 << ",\n";
        f << "  \"probe_y_physical_nm\": " << p.py * 1e9 << ",\n";
        f << "  \"probe_z_physical_nm\": " << p.pz * 1e9 << ",\n";
        f << "  \"pml_offset_x_m\": " << g.pml_offset(0) << ",\n";
        f << "  \"pml_offset_y_m\": " << g.pml_offset(1) << ",\n";
        f << "  \"pml_offset_z_m\": " << g.pml_offset(2) << ",\n";
        f << "  \"save_every\": " << S.save_every << ",\n";
        f << "  \"n_steps\": " << S.n_steps << ",\n";
        f << "  \"dt\": " << std::setprecision(18) << S.dt << ",\n";
        f << "  \"dtype\": \"" << (plan.float64 ? "float64" : "float32") << "\",\n";
        f << "  \"components\": [";
        for (std::size_t c = 0; c < p.components.size(); ++c)
            f << (c ? ", " : "") << "\"" << component_name(p.components[c]) << "\"";
        f << "],\n";
        f << "  \"files\": [";
        for (std::size_t c = 0; c < p.components.size(); ++c)
            f << (c ? ", " : "") << "\"" << component_name(p.components[c]) << "_ts.bin\"";
        f << "],\n";
        f << "  \"note\": \"time series of field components at single point\"\n";
        f << "}\n";
    }

    if (plan.tls) {  // the constructors of the two-level detectors (src/two_level_detectors.hpp)
        const fs::path pop = dir / "populations", pol = dir / "polarization";
        for (const fs::path& d : {pop, pol}) {
            fs::create_directories(d, ec);
            if (ec) throw std::runtime_error("cannot create " + d.string());
        }
        for (const char* b : {"populations_Nu.bin", "populations_Ng.bin"}) {
            std::ofstream t(pop / b, std::ios::binary | std::ios::trunc);
            if (!t) throw std::runtime_error("cannot write " + (pop / b).string());
        }
        open_text(pop / "inversion_time.csv") << "t, total_Nu, total_Ng, inversion, inv_fraction\n";
        open_text(pol / "polarization_time.csv") << "t, Pz_center, dPz_dt_center, total_P_energy\n";
        open_text(dir / "tls_global_history.csv")
            << "step,t_fs,Nu_total,Ng_total,inversion_total,Nu_percent,Ng_percent,inv_norm\n";
    }
}

// ---------------------------------------------------------------- writer thread
OutputWriter::OutputWriter() : th_([this] { loop(); }) {}

OutputWriter::~OutputWriter() {
    {
        std::lock_guard<std::mutex> l(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    th_.join();
}

void OutputWriter::submit(Job j) {
    {
        std::lock_guard<std::mutex> l(mu_);
        q_.push_back(std::move(j));
    }
    cv_.notify_all();
}

void OutputWriter::drain() {
    std::unique_lock<std::mutex> l(mu_);
    idle_.wait(l, [this] { return q_.empty() && !busy_; });
    if (!error_.empty()) {
        std::string e;
        e.swap(error_);
        throw std::runtime_error(e);
    }
}

void OutputWriter::loop() {
    for (;;) {
        Job j;
        {
            std::unique_lock<std::mutex> l(mu_);
            cv_.wait(l, [this] { return stop_ || !q_.empty(); });
            if (q_.empty()) return;  // stop requested and nothing left
            j = std::move(q_.front());
            q_.pop_front();
            busy_ = true;
        }
        std::string err;
        try {
            if (j.wait) j.wait();
            std::ofstream f(j.path, std::ios::binary | (j.append ? std::ios::app : std::ios::trunc));
            if (!f) throw std::runtime_error("cannot write " + j.path);
            if (j.text) {
                const std::string t = j.text();
                f.write(t.data(), std::streamsize(t.size()));
            } else {
                f.write(static_cast<const char*>(j.data), std::streamsize(j.bytes));
            }
            if (!f) throw std::runtime_error("write failed: " + j.path);
        } catch (const std::exception& e) {
            err = e.what();
        }
        if (j.done) j.done();
        {
            std::lock_guard<std::mutex> l(mu_);
            if (!err.empty() && error_.empty()) error_ = err;
            busy_ = false;
        }
        idle_.notify_all();
    }
}

}  // namespace fdtd
