// automesh.cpp -- non-uniform auto-mesher of the host setup API.
//
// Produces the same mesh lines as the reference's AutoMeshGenerator
// (src/auto_mesh_generator.hpp): physical-domain mesh per axis first
// (build_segmented_grid_1d, :386-856), grading repair by subdivision (:859-898),
// duplicate removal, then the uniform PML extension (extend_with_pml_1d, :280-377).
// The reference's meshes are part of the parity contract (mesh lines bit-identical),
// so every branch, clamp and floating-point operation below keeps the reference's
// order; only the code organisation is this library's own.  The reference's
// diagnostics-only passes (constraint collection, validation, statistics printing)
// have no effect on the lines and are not repeated.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <set>

namespace fdtd {

real AutoMeshConfig::ppw_target() const {  // get_ppw_target, :100-107
    if (ppw_override > 0) return ppw_override;
    if (mesh_accuracy <= 1) return 6.0;
    if (mesh_accuracy == 2) return 10.0;
    return 14.0 + (mesh_accuracy - 3) * 4.0;
}

real AutoMeshConfig::lambda_min_eff() const {  // get_lambda_min, :110-115
    if (f_max > 0) return phys::C0 / f_max;
    return lambda_min;
}

namespace {

struct OverrideSpan {  // OverrideSegment1D
    real start, end, dx;
    int priority;
};

struct Segment {  // the Region list of build_segmented_grid_1d
    real start, end, target_dx;
    bool is_override;
};

void axis_extent(const StructureBounds& s, int axis, real& lo, real& hi) {
    switch (axis) {
        case 0: lo = s.x_min; hi = s.x_max; break;
        case 1: lo = s.y_min; hi = s.y_max; break;
        default: lo = s.z_min; hi = s.z_max; break;
    }
}

// sample_n_at_position (:1011-1031): first structure whose [min, max) holds pos.
real refractive_index_at(const std::vector<StructureBounds>& structures, int axis, real pos, real bg) {
    for (const auto& s : structures) {
        real lo, hi;
        axis_extent(s, axis, lo, hi);
        if (pos >= lo && pos < hi) return s.n_material;
    }
    return bg;
}

// collect_override_segments_1d (:986-1012)
std::vector<OverrideSpan> override_spans(const AutoMeshConfig& cfg, int axis, real domain) {
    std::vector<OverrideSpan> out;
    if (!cfg.mesh_override_enabled) return out;
    for (const auto& r : cfg.override_regions) {
        if (!r.enabled) continue;
        real lo, hi, d;
        switch (axis) {
            case 0: lo = r.x0; hi = r.x1; d = r.dx; break;
            case 1: lo = r.y0; hi = r.y1; d = r.dy; break;
            default: lo = r.z0; hi = r.z1; d = r.dz; break;
        }
        lo = std::max(0.0, std::min(lo, domain));
        hi = std::max(0.0, std::min(hi, domain));
        if (lo < hi) {
            d = std::clamp(d, cfg.dx_min, cfg.dx_max);
            out.push_back({lo, hi, d, r.priority});
        }
    }
    return out;
}

// fix_grading_by_subdivision (:859-898): split the larger cell of the worst pair.
std::vector<real> repair_grading(std::vector<real> lines, real g, real dx_min) {
    const int max_iter = 300;
    const real tol = dx_min * 0.01;
    for (int iter = 0; iter < max_iter; ++iter) {
        real worst = 1.0;
        std::size_t at = 0;
        for (std::size_t i = 0; i + 2 < lines.size(); ++i) {
            real a = lines[i + 1] - lines[i];
            real b = lines[i + 2] - lines[i + 1];
            if (a < tol || b < tol) continue;
            real ratio = std::max(a / b, b / a);
            if (ratio > worst) { worst = ratio; at = i; }
        }
        if (worst <= g * 1.005) break;
        real a = lines[at + 1] - lines[at];
        real b = lines[at + 2] - lines[at + 1];
        std::size_t split = (a > b) ? at : at + 1;
        real w = lines[split + 1] - lines[split];
        if (w < dx_min * 1.5) break;
        real mid = 0.5 * (lines[split] + lines[split + 1]);
        lines.insert(lines.begin() + std::ptrdiff_t(split + 1), mid);
    }
    return lines;
}

// Appends n equal cells from `from` to `to`, the last line snapped to `to`.
real fill_uniform(std::vector<real>& lines, real from, real to, std::size_t n, real cell) {
    for (std::size_t i = 1; i <= n; ++i) {
        real p = from + i * cell;
        if (i == n) p = to;
        lines.push_back(p);
    }
    return cell;
}

// Appends n cells of width w by repeated addition from pos (the reference's end-fill loops).
void fill_repeated(std::vector<real>& lines, real& pos, int n, real w) {
    for (int j = 0; j < n; ++j) {
        pos += w;
        lines.push_back(pos);
    }
}

class AxisMesher {
public:
    AxisMesher(const AutoMeshConfig& cfg, const std::vector<StructureBounds>& st, int axis, real domain, real bg)
        : cfg_(cfg), st_(st), axis_(axis), domain_(domain), bg_(bg), g_(cfg.max_grading_ratio) {}

    std::vector<real> run() {
        const auto overrides = override_spans(cfg_, axis_, domain_);
        build_segments(overrides);

        lines_.clear();
        lines_.push_back(0.0);
        prev_dx_ = segs_[0].target_dx;
        for (std::size_t ri = 0; ri < segs_.size(); ++ri) {
            if (segs_[ri].is_override) mesh_override(segs_[ri]);
            else mesh_free(ri);
        }
        lines_.back() = domain_;
        std::vector<real> repaired = repair_grading(lines_, g_, cfg_.dx_min);

        std::vector<real> clean;
        clean.push_back(repaired[0]);
        for (std::size_t i = 1; i < repaired.size(); ++i)
            if (repaired[i] > clean.back() + cfg_.dx_min * 0.001) clean.push_back(repaired[i]);
        return clean;
    }

private:
    const AutoMeshConfig& cfg_;
    const std::vector<StructureBounds>& st_;
    int axis_;
    real domain_, bg_, g_;
    std::vector<Segment> segs_;
    std::vector<real> lines_;
    real prev_dx_ = 0;

    real auto_dx(real pos) const {
        real n_local = refractive_index_at(st_, axis_, pos, bg_);
        real lambda_eff = cfg_.lambda_min_eff() / n_local;
        real d = lambda_eff / cfg_.ppw_target();
        return std::clamp(d, cfg_.dx_min, cfg_.dx_max);
    }

    real clamp_size(real d) const { return std::clamp(d, cfg_.dx_min, cfg_.dx_max); }

    void build_segments(const std::vector<OverrideSpan>& overrides) {
        std::set<real> cuts;
        cuts.insert(0.0);
        cuts.insert(domain_);
        for (const auto& ov : overrides) {
            cuts.insert(std::max(0.0, std::min(ov.start, domain_)));
            cuts.insert(std::max(0.0, std::min(ov.end, domain_)));
        }
        for (const auto& s : st_) {
            real lo, hi;
            axis_extent(s, axis_, lo, hi);
            if (lo > 0 && lo < domain_) cuts.insert(lo);
            if (hi > 0 && hi < domain_) cuts.insert(hi);
        }
        std::vector<real> c(cuts.begin(), cuts.end());
        segs_.clear();
        for (std::size_t i = 0; i + 1 < c.size(); ++i) {
            real a = c[i], b = c[i + 1];
            real mid = (a + b) / 2;
            bool ov_hit = false;
            real ov_dx = 0;
            for (const auto& ov : overrides) {
                if (mid >= ov.start && mid <= ov.end) { ov_hit = true; ov_dx = ov.dx; break; }
            }
            segs_.push_back({a, b, ov_hit ? ov_dx : auto_dx(mid), ov_hit});
        }
    }

    // Override segment: strictly uniform cells (:462-478).
    void mesh_override(const Segment& s) {
        real len = s.end - s.start;
        std::size_t n = std::max(std::size_t(1), (std::size_t)std::round(len / s.target_dx));
        real cell = len / n;
        prev_dx_ = fill_uniform(lines_, s.start, s.end, n, cell);
    }

    void mesh_free(std::size_t ri) {
        const Segment& s = segs_[ri];
        const bool prev_ov = (ri > 0 && segs_[ri - 1].is_override);
        const bool next_ov = (ri + 1 < segs_.size() && segs_[ri + 1].is_override);
        const real len = s.end - s.start;
        const real want = s.target_dx;

        if (prev_ov && next_ov) {
            between_overrides(ri, len, want);
            return;
        }
        const real air_dx = cfg_.lambda_min_eff() / bg_ / cfg_.ppw_target();
        const bool material_segment = (want < air_dx * 0.6) && (want > cfg_.dx_min * 2);
        if (material_segment && !next_ov) {
            material_fill(s, len, want);
            return;
        }
        graded_fill(ri, len, want, next_ov);
    }

    // CASE 1 (:490-567): gap between two override segments.
    void between_overrides(std::size_t ri, real len, real want) {
        const Segment& s = segs_[ri];
        const real start_dx = prev_dx_;
        const real end_dx = segs_[ri + 1].target_dx;

        real half = len / 2;
        real peak = start_dx;
        real run = 0;
        while (run < half && peak < want) {
            peak *= g_;
            run += peak;
        }
        peak = std::min(peak, want);

        std::vector<real> up, down;
        real t = start_dx;
        while (t < peak * 0.95) {
            t = std::min(t * g_, peak);
            up.push_back(t);
        }
        t = peak;
        while (t > end_dx * 1.05) {
            t = std::max(t / g_, end_dx);
            down.push_back(t);
        }
        real graded = 0;
        for (real v : up) graded += v;
        for (real v : down) graded += v;

        if (graded > 0 && graded <= len * 1.3) {
            real scale = len / graded;
            std::vector<real> seq(up);
            seq.insert(seq.end(), down.begin(), down.end());
            real p = s.start;
            for (std::size_t i = 0; i < seq.size(); ++i) {
                p += seq[i] * scale;
                if (i == seq.size() - 1) p = s.end;
                lines_.push_back(p);
            }
            prev_dx_ = seq.back() * scale;
            return;
        }
        real fine = std::min(start_dx, end_dx);
        std::size_t n = std::max(std::size_t(1), (std::size_t)std::round(len / fine));
        prev_dx_ = fill_uniform(lines_, s.start, s.end, n, len / n);
    }

    // CASE 2 (:569-639): material segment not followed by an override.
    void material_fill(const Segment& s, real len, real want) {
        real pos = lines_.back();
        if (prev_dx_ < want * 0.7) {
            std::vector<real> ramp;
            real t = prev_dx_;
            while (t < want * 0.95) {
                t *= g_;
                if (t > want) t = want;
                ramp.push_back(t);
            }
            real ramp_len = 0;
            for (real v : ramp) ramp_len += v;
            if (ramp_len < len) {
                for (real v : ramp) {
                    pos += v;
                    if (pos > s.end - cfg_.dx_min) break;
                    lines_.push_back(pos);
                    prev_dx_ = v;
                }
            }
        }
        real left = s.end - pos;
        if (left > cfg_.dx_min) {
            real use = want;
            if (use / prev_dx_ > g_) use = prev_dx_ * g_;
            if (prev_dx_ / use > g_) use = prev_dx_ / g_;
            std::size_t n = std::max(std::size_t(1), (std::size_t)std::round(left / use));
            real cell = left / n;
            if (cell / prev_dx_ > g_ || prev_dx_ / cell > g_) {
                if (prev_dx_ < cell) cell = std::min(cell, prev_dx_ * g_);
                else cell = std::max(cell, prev_dx_ / g_);
                n = std::max(std::size_t(1), (std::size_t)std::round(left / cell));
                cell = left / n;
            }
            prev_dx_ = fill_uniform(lines_, pos, s.end, n, cell);
        }
    }

    // Closing fill used by both exit branches of CASE 3 (:774-794, :808-826).
    void close_out(real& pos, real remaining, real next_dx, real current_dx) {
        int n = std::max(1, (int)std::round(remaining / next_dx));
        real w = remaining / n;
        if (w / current_dx > g_ || current_dx / w > g_) {
            n = std::max(2, (int)std::ceil(remaining / (current_dx * g_)));
            w = remaining / n;
        }
        fill_repeated(lines_, pos, n, w);
        prev_dx_ = w;
    }

    // CASE 3 (:641-851): air segment or transition into an override.
    void graded_fill(std::size_t ri, real len, real want, bool next_ov) {
        const Segment& s = segs_[ri];
        real pos = lines_.back();
        const real target = s.end;
        const real entry_dx = prev_dx_;
        real exit_dx = s.target_dx;
        bool need_exit = false;
        if (next_ov) {
            exit_dx = segs_[ri + 1].target_dx;
            need_exit = true;
        } else if (ri + 1 < segs_.size()) {
            real nt = segs_[ri + 1].target_dx;
            if (nt < want) { exit_dx = nt; need_exit = true; }
        }

        std::vector<real> entry, exit;
        if (entry_dx < want * 0.99) {
            real t = entry_dx;
            while (t < want * 0.99) {
                t = std::min(t * g_, want);
                t = clamp_size(t);
                entry.push_back(t);
            }
        }
        if (need_exit && exit_dx < want * 0.99) {
            real t = want;
            while (t > exit_dx * 1.01) {
                t = std::max(t / g_, exit_dx);
                t = clamp_size(t);
                exit.push_back(t);
            }
            if (exit.empty() || exit.back() > exit_dx * 1.2) exit.push_back(exit_dx);
        }
        real entry_len = 0;
        for (real v : entry) entry_len += v;
        real exit_len = 0;
        for (real v : exit) exit_len += v;
        real stable_len = len - entry_len - exit_len;
        if (stable_len < 0) {
            real total = entry_len + exit_len;
            real scale = len / total * 0.95;
            for (real& v : entry) v *= scale;
            for (real& v : exit) v *= scale;
            entry_len *= scale;
            exit_len *= scale;
            stable_len = len - entry_len - exit_len;
        }
        const real stable_dx = clamp_size(want);
        real cur = entry_dx;

        for (real v : entry) {  // phase 1: entry ramp
            real nd = std::clamp(v, cur / g_, cur * g_);
            nd = clamp_size(nd);
            if (pos + nd > target - cfg_.dx_min) break;
            pos += nd;
            lines_.push_back(pos);
            cur = nd;
            prev_dx_ = nd;
        }

        if (stable_len > stable_dx * 0.5 && pos < target - exit_len - cfg_.dx_min) {  // phase 2
            real stable_end = target - exit_len;
            real rem = stable_end - pos;
            if (rem > 0) {
                real use = stable_dx;
                if (use / cur > g_) use = cur * g_;
                if (cur / use > g_) use = cur / g_;
                use = clamp_size(use);
                std::size_t n = std::max(std::size_t(1), (std::size_t)std::round(rem / use));
                real cell = rem / n;
                fill_uniform(lines_, pos, stable_end, n, cell);
                pos = stable_end;
                cur = cell;
                prev_dx_ = cell;
            }
        }

        if (!exit.empty() && pos < target - cfg_.dx_min * 0.5) {  // phase 3: exit ramp
            for (std::size_t i = 0; i < exit.size(); ++i) {
                real nd = std::clamp(exit[i], cur / g_, cur * g_);
                nd = clamp_size(nd);
                real rem = target - pos;
                if (rem < nd * 0.5) break;
                if (i == exit.size() - 1 || rem < nd * 1.5) {
                    close_out(pos, rem, nd, cur);
                    break;
                }
                pos += nd;
                lines_.push_back(pos);
                cur = nd;
                prev_dx_ = nd;
            }
        } else if (exit.empty() && pos < target - cfg_.dx_min * 0.5) {
            while (pos < target - cfg_.dx_min * 0.5) {
                real rem = target - pos;
                real nd = stable_dx;
                nd = std::clamp(nd, cur / g_, cur * g_);
                nd = clamp_size(nd);
                if (rem < nd * 1.5) {
                    close_out(pos, rem, nd, cur);
                    break;
                }
                pos += nd;
                lines_.push_back(pos);
                cur = nd;
                prev_dx_ = nd;
            }
        }

        if (std::abs(lines_.back() - target) > cfg_.dx_min * 0.1 && lines_.back() < target) {
            lines_.push_back(target);
            prev_dx_ = target - lines_[lines_.size() - 2];
        }
    }
};

// extend_with_pml_1d (:280-377)
std::vector<real> add_pml_cells(const std::vector<real>& phys, std::size_t npml, const AutoMeshConfig& cfg) {
    if (npml == 0 || phys.size() < 2) return phys;
    const real dl = phys[1] - phys[0];
    const real dr = phys.back() - phys[phys.size() - 2];
    std::vector<real> left, right;
    if (cfg.pml_strategy == PmlStrategy::UNIFORM) {
        real thick = npml * dl;
        for (std::size_t i = 0; i < npml; ++i) left.push_back(-thick + i * dl);
        real end = phys.back();
        for (std::size_t i = 1; i <= npml; ++i) right.push_back(end + i * dr);
    } else {
        const real g = cfg.max_grading_ratio;
        real w = dl, p = 0;
        std::vector<real> tmp;
        for (std::size_t i = 0; i < npml; ++i) {
            p -= w;
            tmp.push_back(p);
            w = std::min(w * g, cfg.dx_max);
        }
        left.assign(tmp.rbegin(), tmp.rend());
        w = dr;
        p = phys.back();
        for (std::size_t i = 0; i < npml; ++i) {
            p += w;
            right.push_back(p);
            w = std::min(w * g, cfg.dx_max);
        }
    }
    std::vector<real> all;
    all.reserve(left.size() + phys.size() + right.size());
    all.insert(all.end(), left.begin(), left.end());
    all.insert(all.end(), phys.begin(), phys.end());
    all.insert(all.end(), right.begin(), right.end());
    real off = -all[0];
    for (real& x : all) x += off;
    return all;
}

}  // namespace

GridSpacing automesh_generate(const AutoMeshConfig& cfg_in, real domain_x, real domain_y, real domain_z,
                              std::size_t npml, const std::vector<StructureBounds>& structures,
                              real background_n) {
    AutoMeshConfig cfg = cfg_in;
    cfg.npml = npml;
    const real dom[3] = {domain_x, domain_y, domain_z};
    GridSpacing g;
    std::vector<real>* bounds[3] = {&g.x_bounds, &g.y_bounds, &g.z_bounds};
    std::vector<real>* widths[3] = {&g.dx, &g.dy, &g.dz};
    for (int axis = 0; axis < 3; ++axis) {
        std::vector<real> phys = AxisMesher(cfg, structures, axis, dom[axis], background_n).run();
        *bounds[axis] = add_pml_cells(phys, npml, cfg);
        const auto& b = *bounds[axis];
        widths[axis]->resize(b.size() - 1);
        for (std::size_t i = 0; i + 1 < b.size(); ++i) (*widths[axis])[i] = b[i + 1] - b[i];
    }
    g.npml = npml;
    return g;
}

}  // namespace fdtd
