// capi_setup.cpp -- extern "C" entry points of the host setup API (include/fdtd_b200.h).
#include "../../../include/fdtd_b200.h"
#include "outputs.hpp"
#include "setup.hpp"

#include <cstring>
#include <exception>
#include <string>
#include <vector>

struct fdtd_setup {
    fdtd::SimSetup S;
    // Storage backing the plain-data view.
    std::vector<fdtd_dipole_v1> dipoles;
    std::vector<fdtd_tls_region_v1> regions;
    std::vector<fdtd_probe_v1> probes;
    std::vector<fdtd_sheet_v1> sheets;
    std::vector<double> uniform_kappa[3], unit_b[3], zero_c[3];
    // aE = aH = 1 and bH uniform everywhere (lossless, mu_r = 1 -- what make_nk gives): the
    // view then passes those arrays as NULL and the stepper skips scanning them
    bool uniform_ah = false;
    // distinct bE rows and each cell's row number (empty when there are more than 65535)
    std::vector<double> bE_rows;
    std::vector<uint16_t> bE_index;
};

namespace {
bool all_equal(const std::vector<double>& v, double x) {
    long long bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(static)
    for (long long q = 0; q < (long long)v.size(); ++q) bad += v[q] != x;
    return bad == 0;
}
}  // namespace

namespace {

void write_err(char* err, std::size_t errlen, const std::string& msg) {
    if (!err || errlen == 0) return;
    std::size_t n = std::min(errlen - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

// Returns a pointer to the named array and its length, or nullptr.
const std::vector<double>* find_array(const fdtd_setup* s, const std::string& name, std::vector<double>& scratch) {
    const fdtd::SimSetup& S = s->S;
    static const char* axes = "xyz";
    for (int a = 0; a < 3; ++a) {
        const std::string ax(1, axes[a]);
        if (name == ax + "_bounds") return &S.grid.bounds(a);
        if (name == "d" + ax) return &S.grid.spacing(a);
        if (name == "inv_d" + ax) return a == 0 ? &S.grid.inv_dx : a == 1 ? &S.grid.inv_dy : &S.grid.inv_dz;
        if (name == "cpml_k" + ax) return &S.cpml.kappa[a];
        if (name == "cpml_s" + ax) return &S.cpml.sigma[a];
        if (name == "cpml_a" + ax) return &S.cpml.alpha[a];
        if (name == "cpml_bE" + ax) return &S.cpml.bE[a];
        if (name == "cpml_cE" + ax) return &S.cpml.cE[a];
        if (name == "cpml_bH" + ax) return &S.cpml.bH[a];
        if (name == "cpml_cH" + ax) return &S.cpml.cH[a];
        if (name == "bE" + ax) return &S.mats.bE[a];
        if (name == "aE" + ax) return &S.mats.aE[a];
        if (name == "bH" + ax) return &S.mats.bH[a];
        if (name == "aH" + ax) return &S.mats.aH[a];
    }
    if (name == "n_grid") {
        if (S.scene.NxT == 0) return nullptr;
        S.scene.n_grid(scratch);
        return &scratch;
    }
    if (name == "tls_region_map") {
        scratch.assign(S.tls.cell_region_map.begin(), S.tls.cell_region_map.end());
        return &scratch;
    }
    if (name == "tls_Nu") return &S.tls.Nu;
    if (name == "tls_Ng") return &S.tls.Ng;
    if (name == "tls_Ndip") return &S.tls.Ndip;
    if (name == "dft_freqs") return &S.dft_freqs;
    if (name == "source_J") {  // J(n) for n < N_STEPS of the first dipole
        scratch.clear();
        if (!S.sources.empty())
            for (std::size_t n = 0; n < S.n_steps; ++n) scratch.push_back(S.sources[0].current_density(n, S.dt));
        return &scratch;
    }
    return nullptr;
}

}  // namespace

// The parsed setup behind a handle, for the stepper's output attachment (solver.cu).
const fdtd::SimSetup* fdtd_internal_setup(const fdtd_setup* s) { return s ? &s->S : nullptr; }

extern "C" {

int fdtd_setup_parse(const char* params_text, int mesh_only, fdtd_setup** out, char* err, size_t errlen) {
    if (!params_text || !out) {
        write_err(err, errlen, "null argument");
        return FDTD_ERR_INVALID;
    }
    *out = nullptr;
    try {
        auto* s = new fdtd_setup();
        s->S = fdtd::SimSetup::from_params(fdtd::ParamFile::parse(params_text), mesh_only == 0);
        const fdtd::SimSetup& S = s->S;
        for (const auto& d : S.sources)
            s->dipoles.push_back({d.i, d.j, d.k, d.polarization, int32_t(d.waveform), d.cell_area, d.I0, d.f0,
                                  d.tau, d.t0, d.t_shift});
        for (const auto& r : S.tls.regions)
            s->regions.push_back({r.params.kapa_coeff, r.params.pa2, r.params.pa3, r.params.inv_dt, r.params.tau,
                                  r.params.hbar, r.params.omega_a, r.params.N0_total, r.params.pump_rate,
                                  r.params.enable_population_clamp ? 1 : 0, 0});
        for (const auto& p : S.probes)
            for (int c : p.components) s->probes.push_back({p.i, p.j, p.k, c, 0});
        for (const auto& w : S.plane_waves)
            s->sheets.push_back({w.axis, w.comp, w.plane, w.lo0, w.hi0, w.lo1, w.hi1, w.d, w.sign, int32_t(w.waveform), 0,
                                 w.E0, w.f0, w.tau, w.t0, w.t_shift});
        bool u = S.mats.uniform_ah || !S.mats.bH[0].empty();
        for (int a = 0; a < 3 && u && !S.mats.uniform_ah; ++a)
            u = !S.mats.aE[a].empty() && !S.mats.aH[a].empty() && !S.mats.bH[a].empty() && all_equal(S.mats.aE[a], 1.0) &&
                all_equal(S.mats.aH[a], 1.0) && all_equal(S.mats.bH[a], S.mats.bH[0][0]);
        s->uniform_ah = u;
        if (!S.mats.bE[0].empty()) {
            const double* bE[3] = {S.mats.bE[0].data(), S.mats.bE[1].data(), S.mats.bE[2].data()};
            std::vector<std::array<double, 3>> rows;
            if (fdtd::distinct_rows(bE, S.mats.bE[0].size(), rows, s->bE_index)) {
                for (const auto& r : rows) s->bE_rows.insert(s->bE_rows.end(), r.begin(), r.end());
            } else {
                s->bE_index.clear();
            }
        }
        *out = s;
        return FDTD_OK;
    } catch (const std::exception& e) {
        write_err(err, errlen, e.what());
        return FDTD_ERR_PARSE;
    }
}

int fdtd_setup_view(const fdtd_setup* s, fdtd_setup_v1* v) {
    if (!s || !v) return FDTD_ERR_INVALID;
    const fdtd::SimSetup& S = s->S;
    std::memset(v, 0, sizeof(*v));
    v->struct_size = sizeof(fdtd_setup_v1);
    v->precision = S.precision == "fp64" ? FDTD_PREC_FP64
                 : S.precision == "fp16" ? FDTD_PREC_FP16
                 : S.precision == "bf16" ? FDTD_PREC_BF16 : FDTD_PREC_FP32;
    v->field_scale = S.field_scale;
    v->NxT = S.NxT; v->NyT = S.NyT; v->NzT = S.NzT;
    v->npml = uint32_t(S.npml);
    v->save_every = uint32_t(S.save_every);
    v->dt = S.dt;
    v->dx = S.grid.dx.data(); v->dy = S.grid.dy.data(); v->dz = S.grid.dz.data();
    v->inv_dx = S.grid.inv_dx.data(); v->inv_dy = S.grid.inv_dy.data(); v->inv_dz = S.grid.inv_dz.data();
    for (int a = 0; a < 3; ++a) {
        v->cpml_kappa[a] = S.cpml.kappa[a].data();
        v->cpml_bE[a] = S.cpml.bE[a].data(); v->cpml_cE[a] = S.cpml.cE[a].data();
        v->cpml_bH[a] = S.cpml.bH[a].data(); v->cpml_cH[a] = S.cpml.cH[a].data();
        v->bE[a] = S.mats.bE[a].empty() ? nullptr : S.mats.bE[a].data();
        v->aE[a] = (s->uniform_ah || S.mats.aE[a].empty()) ? nullptr : S.mats.aE[a].data();
        v->aH[a] = (s->uniform_ah || S.mats.aH[a].empty()) ? nullptr : S.mats.aH[a].data();
        v->bH[a] = (s->uniform_ah || S.mats.bH[a].empty()) ? nullptr : S.mats.bH[a].data();
    }
    v->bH_uniform = S.mats.uniform_ah ? S.mats.bH_value : s->uniform_ah ? S.mats.bH[0][0] : S.dt / fdtd::phys::MU0;
    v->n_sheets = uint32_t(s->sheets.size());
    v->sheets = s->sheets.data();
    v->pec_boundary = S.boundary_pec ? 1 : 0;
    v->rounding = S.stochastic_rounding ? FDTD_ROUND_STOCHASTIC : FDTD_ROUND_NEAREST;
    if (!s->bE_index.empty()) {
        v->n_bE_rows = uint32_t(s->bE_rows.size() / 3);
        v->bE_rows = s->bE_rows.data();
        v->bE_index = s->bE_index.data();
    }
    v->n_dipoles = uint32_t(s->dipoles.size());
    v->dipoles = s->dipoles.data();
    v->n_tls_regions = uint32_t(s->regions.size());
    v->tls_regions = s->regions.data();
    v->tls_region_map = S.tls.cell_region_map.empty() ? nullptr : S.tls.cell_region_map.data();
    v->tls_Nu = S.tls.Nu.empty() ? nullptr : S.tls.Nu.data();
    v->tls_Ng = S.tls.Ng.empty() ? nullptr : S.tls.Ng.data();
    v->n_probes = uint32_t(s->probes.size());
    v->probes = s->probes.data();
    v->n_dft_freqs = uint32_t(S.dft_freqs.size());
    v->dft_freqs = S.dft_freqs.data();
    v->monitor_interval = uint32_t(S.stability_interval);
    v->max_E = S.stability_max_E;
    v->max_P = S.stability_max_P;
    v->conservation_err = S.stability_conservation;
    v->growth_rate = S.stability_growth;
    return FDTD_OK;
}

int fdtd_setup_array_len(const fdtd_setup* s, const char* name, uint64_t* len) {
    if (!s || !name || !len) return FDTD_ERR_INVALID;
    std::vector<double> scratch;
    const std::vector<double>* a = find_array(s, name, scratch);
    if (!a) return FDTD_ERR_INVALID;
    *len = a->size();
    return FDTD_OK;
}

int fdtd_setup_array(const fdtd_setup* s, const char* name, double* out, uint64_t len) {
    if (!s || !name || !out) return FDTD_ERR_INVALID;
    std::vector<double> scratch;
    const std::vector<double>* a = find_array(s, name, scratch);
    if (!a || a->size() != len) return FDTD_ERR_INVALID;
    std::memcpy(out, a->data(), len * sizeof(double));
    return FDTD_OK;
}

int fdtd_setup_write_outputs(const fdtd_setup* s, const char* out_dir, char* err, size_t errlen) {
    if (!s || !out_dir) {
        write_err(err, errlen, "null argument");
        return FDTD_ERR_INVALID;
    }
    fdtd::OutputPlan plan;
    try {
        plan = fdtd::make_output_plan(s->S);
    } catch (const std::exception& e) {
        write_err(err, errlen, e.what());
        return FDTD_ERR_INVALID;
    }
    try {
        fdtd::write_setup_outputs(s->S, plan, out_dir);
    } catch (const std::exception& e) {
        write_err(err, errlen, e.what());
        return FDTD_ERR_IO;
    }
    return FDTD_OK;
}

void fdtd_setup_destroy(fdtd_setup* s) { delete s; }

}  // extern "C"
