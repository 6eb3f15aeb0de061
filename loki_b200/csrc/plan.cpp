// Host-side search plan: the configuration checks and per-level grid
// geometry of the reference's PulsarSearchConfig and FFAPlan. The formulas
// must produce the same integers and doubles as the reference (they fix the
// coordinate grids every kernel indexes), so each one keeps the reference's
// operation order; the citations name the lines restated.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

#include "lk_internal.hpp"

namespace lk {

namespace {

bool is_pow2(uint64_t x) { return x != 0 && (x & (x - 1)) == 0; }

// math::factorial<double>(n) = std::tgamma(n + 1) (lib/loki/math.hpp:35-44).
double factorial_d(double n) { return std::tgamma(n + 1.0); }

// psr_utils::poly_taylor_step_f (lib/psr_utils.cpp:14-29).
std::vector<double> poly_taylor_step_f(uint32_t nparams, double tobs, uint64_t fold_bins,
                                       double tol_bins, double t_ref) {
    const double dphi = tol_bins / static_cast<double>(fold_bins);
    const double dt = tobs - t_ref;
    std::vector<double> out(nparams);
    for (uint32_t i = 0; i < nparams; ++i) {
        const double orth_factor = std::pow(2.0, static_cast<double>(i));
        out[nparams - 1 - i] = dphi * orth_factor * factorial_d(static_cast<double>(i + 1)) /
                               std::pow(dt, static_cast<double>(i + 1));
    }
    return out;
}

// psr_utils::poly_taylor_step_d_f (lib/psr_utils.cpp:31-45): the derivative
// steps are converted to velocity-like units with c / f_max.
std::vector<double> poly_taylor_step_d_f(uint32_t nparams, double tobs, uint64_t fold_bins,
                                         double tol_bins, double f_max, double t_ref) {
    auto f = poly_taylor_step_f(nparams, tobs, fold_bins, tol_bins, t_ref);
    for (uint32_t i = 0; i + 1 < nparams; ++i) {
        f[i] = f[i] * kCval / f_max;
    }
    return f;
}

// psr_utils::range_param_count (lib/loki/psr_utils.hpp:235-242).
uint64_t range_param_count(double vmin, double vmax, double dv) {
    require(vmax > vmin, "vmax must be greater than vmin");
    require(dv > 0, "dv must be positive");
    if (dv >= (vmax - vmin)) {
        return 1;
    }
    return static_cast<uint64_t>(std::ceil((vmax - vmin) / dv));
}

}  // namespace

std::vector<double> range_param(double vmin, double vmax, double dv) {
    require(vmax > vmin, "vmax must be greater than vmin");
    require(dv > 0, "dv must be positive");
    if (dv >= (vmax - vmin)) {
        return {(vmax + vmin) / 2.0};
    }
    const auto npoints = static_cast<uint64_t>(std::ceil((vmax - vmin) / dv));
    const double dv_actual = (vmax - vmin) / static_cast<double>(npoints);
    const double start = vmin + (0.5 * dv_actual);
    std::vector<double> out(npoints);
    for (uint64_t i = 0; i < npoints; ++i) {
        out[i] = start + (dv_actual * static_cast<double>(i));
    }
    return out;
}

// detection::generate_box_width_trials (lib/score.cpp:390-405).
std::vector<uint32_t> box_width_trials(uint64_t nbins, double ducy_max, double wtsp) {
    const auto wmax =
        static_cast<uint64_t>(std::max(1.0, ducy_max * static_cast<double>(nbins)));
    std::vector<uint32_t> w = {1};
    while (w.back() < wmax) {
        const auto next = std::max(static_cast<uint64_t>(w.back() + 1),
                                   static_cast<uint64_t>(wtsp * static_cast<double>(w.back())));
        if (next > wmax) {
            break;
        }
        w.push_back(static_cast<uint32_t>(next));
    }
    return w;
}

std::vector<double> Plan::param_grid(uint32_t level, uint32_t iparam) const {
    return range_param(lim_min(iparam), lim_max(iparam), dparams[level][iparam]);
}

// core::generate_bp_poly_taylor (lib/taylor.cpp:1643-1741): the average
// branching factor of each pruning level for a run seeded at ref_seg,
// weighted over the final level's frequency grid.
std::vector<double> Plan::branching_pattern(uint64_t ref_seg, bool conservative) const {
    require(nparams >= 2 && nparams <= 4, "branching pattern needs 2 <= nparams <= 4");
    const uint32_t L = n_levels - 1;
    const uint64_t nseg = nsegments[L];
    require(ref_seg < nseg, "ref_idx must be less than nsegments.");
    const double tseg = tsegments[L];
    const uint32_t np = nparams;
    const std::vector<double> f0 = param_grid(L, np - 1);
    const uint64_t nf = f0.size();
    // MiddleOutScheme order and coordinates (lib/loki/psr_utils.hpp:331-448)
    std::vector<uint64_t> order{ref_seg};
    for (uint64_t d = 1; order.size() < nseg; ++d) {
        if (d <= ref_seg) {
            order.push_back(ref_seg - d);
        }
        if (ref_seg + d < nseg && order.size() < nseg) {
            order.push_back(ref_seg + d);
        }
    }
    auto coord = [&](uint64_t level) {
        uint64_t mn = order[0], mx = order[0];
        for (uint64_t i = 1; i <= level; ++i) {
            mn = std::min(mn, order[i]);
            mx = std::max(mx, order[i]);
        }
        const double ref_val = (static_cast<double>(mn) + static_cast<double>(mx) + 1.0) / 2.0;
        const double scale_val = ref_val - static_cast<double>(mn);
        return std::pair<double, double>{ref_val * tseg, scale_val * tseg};
    };
    std::vector<double> weights(nf, 1.0), bp(nseg - 1, 0.0);
    std::vector<double> cur(nf * np), nxt(nf * np, 0.0), dnew(nf * np, 0.0), shift(nf * np, 0.0);
    std::vector<double> nbr(nf, 1.0), dvec(nf * (np + 1), 0.0);
    for (uint64_t i = 0; i < nf; ++i) {
        for (uint32_t j = 0; j < np; ++j) {
            cur[i * np + j] = dparams_actual[L][j];
        }
        cur[i * np + np - 1] = cur[i * np + np - 1] * (kCval / f0[i]);
    }
    const double nbins_d = static_cast<double>(cfg.nbins);
    for (uint64_t level = 1; level < nseg; ++level) {
        const auto cn = coord(level);
        const auto cc = std::pair<double, double>{coord(level - 1).first, coord(level).second};
        const double tobs = cc.second;
        // psr_utils::poly_taylor_step_d_vec with t_ref = 0 (lib/psr_utils.cpp:62-80)
        const std::vector<double> df = poly_taylor_step_f(np, tobs, cfg.nbins, cfg.eta, 0.0);
        for (uint64_t i = 0; i < nf; ++i) {
            const double factor = kCval / f0[i];
            for (uint32_t j = 0; j < np; ++j) {
                dnew[i * np + j] = df[j] * factor;
            }
        }
        // psr_utils::poly_taylor_shift_d_vec (lib/psr_utils.cpp:116-154)
        std::vector<double> dtp(np), fac(np);
        double dtpow = tobs;
        for (uint32_t i = 0; i < np; ++i) {
            dtp[i] = dtpow;
            fac[i] = factorial_d(static_cast<double>(i + 1));
            dtpow *= tobs;
        }
        for (uint32_t i = 0; i < np; ++i) {
            const uint32_t k = np - 1 - i;
            const double factor_base = dtp[k] * nbins_d / fac[k];
            const double factor_opt = factor_base / std::pow(2.0, k);
            const double scale = factor_opt / kCval;
            for (uint64_t b = 0; b < nf; ++b) {
                const uint64_t idx = b * np + i;
                shift[idx] = std::abs(cur[idx] - dnew[idx]) * scale * f0[b];
            }
        }
        std::fill(nbr.begin(), nbr.end(), 1.0);
        for (uint64_t i = 0; i < nf; ++i) {
            for (uint32_t j = 0; j < np; ++j) {
                const uint64_t idx = i * np + j;
                if (shift[idx] < (cfg.eta - kFloatEps)) {
                    nxt[idx] = cur[idx];
                    continue;
                }
                const double ratio = cur[idx] / dnew[idx];
                const double c = std::ceil(ratio - kFloatEps);
                const uint64_t num = c < 1.0 ? 1 : static_cast<uint64_t>(c);
                nbr[i] *= static_cast<double>(num);
                nxt[idx] = cur[idx] / static_cast<double>(num);
            }
        }
        double children = 0.0, parents = 0.0;
        for (uint64_t i = 0; i < nf; ++i) {
            children += weights[i] * nbr[i];
            parents += weights[i];
            weights[i] *= nbr[i];
        }
        bp[level - 1] = children / parents;
        // transforms::shift_taylor_errors_batch (lib/transforms.cpp:55-98)
        const double delta_t = cn.first - cc.first;
        const uint32_t npd = np + 1;
        for (uint64_t i = 0; i < nf; ++i) {
            for (uint32_t j = 0; j < np; ++j) {
                dvec[i * npd + j] = nxt[i * np + j];
            }
        }
        if (!conservative) {
            for (uint64_t i = 0; i < nf; ++i) {
                for (uint32_t j = 0; j < np; ++j) {
                    cur[i * np + j] = dvec[i * npd + j];
                }
            }
        } else {
            std::vector<double> tsq(npd * npd, 0.0);
            for (uint32_t i = 0; i < npd; ++i) {
                for (uint32_t j = 0; j <= i; ++j) {
                    const uint32_t k = i - j;
                    const double t = std::pow(delta_t, k) / factorial_d(static_cast<double>(k));
                    tsq[i * npd + j] = t * t;
                }
            }
            for (uint64_t b = 0; b < nf; ++b) {
                for (uint32_t i = 0; i < np; ++i) {
                    double sum = 0.0;
                    for (uint32_t j = 0; j <= i; ++j) {
                        const double e = dvec[b * npd + j];
                        sum += e * e * tsq[i * npd + j];
                    }
                    cur[b * np + i] = std::sqrt(sum);
                }
            }
        }
    }
    return bp;
}

// generate_bp_poly_chebyshev (lib/chebyshev.cpp:1796-1890): the branching
// pattern of a pruning run in the Chebyshev basis, with the errors converted by
// transforms::taylor_to_cheby_errors_batch and rescaled between coordinates by
// shift_cheb_errors_batch (lib/transforms.cpp:164-235), steps and shifts from
// poly_cheb_step_vec / poly_cheb_shift_vec (lib/psr_utils.cpp:157-194).
std::vector<double> Plan::branching_pattern_cheby(uint64_t ref_seg) const {
    require(nparams >= 2 && nparams <= 4, "branching pattern needs 2 <= nparams <= 4");
    const uint32_t L = n_levels - 1;
    const uint64_t nseg = nsegments[L];
    require(ref_seg < nseg, "ref_idx must be less than nsegments.");
    const double tseg = tsegments[L];
    const uint32_t np = nparams;
    const std::vector<double> f0 = param_grid(L, np - 1);
    const uint64_t nf = f0.size();
    std::vector<uint64_t> order{ref_seg};
    for (uint64_t d = 1; order.size() < nseg; ++d) {
        if (d <= ref_seg) {
            order.push_back(ref_seg - d);
        }
        if (ref_seg + d < nseg && order.size() < nseg) {
            order.push_back(ref_seg + d);
        }
    }
    auto coord = [&](uint64_t level) {
        uint64_t mn = order[0], mx = order[0];
        for (uint64_t i = 1; i <= level; ++i) {
            mn = std::min(mn, order[i]);
            mx = std::max(mx, order[i]);
        }
        const double ref_val = (static_cast<double>(mn) + static_cast<double>(mx) + 1.0) / 2.0;
        const double scale_val = ref_val - static_cast<double>(mn);
        return std::pair<double, double>{ref_val * tseg, scale_val * tseg};
    };
    std::vector<double> weights(nf, 1.0), bp(nseg - 1, 0.0);
    std::vector<double> cur(nf * np), nxt(nf * np, 0.0), dnew(nf * np, 0.0), shift(nf * np, 0.0);
    std::vector<double> nbr(nf, 1.0);
    for (uint64_t i = 0; i < nf; ++i) {
        for (uint32_t j = 0; j < np; ++j) {
            cur[i * np + j] = dparams_actual[L][j];
        }
        cur[i * np + np - 1] = cur[i * np + np - 1] * (kCval / f0[i]);
    }
    {  // taylor_to_cheby_errors_batch at coord_init's scale
        const double ts = coord(0).second;
        const double ts2 = ts * ts;
        const double ts3 = ts2 * ts;
        const double ts4 = ts3 * ts;
        const double w2_2 = (ts2 / 2.0) * 0.5;
        const double w4_4 = (ts4 / 24.0) * 0.125;
        const double w3_3 = (ts3 / 6.0) * 0.25;
        const double w4_2 = (ts4 / 24.0) * 0.5;
        const double w3_1 = (ts3 / 6.0) * 0.75;
        for (uint64_t i = 0; i < nf; ++i) {
            double* e = cur.data() + i * np;
            if (np == 2) {
                const double d2 = e[0], d1 = e[1];
                e[0] = d2 * w2_2;
                e[1] = d1 * ts;
            } else if (np == 3) {
                const double d3 = e[0], d2 = e[1], d1 = e[2];
                const double e3_1 = d3 * w3_1;
                const double e1_ts = d1 * ts;
                e[0] = d3 * w3_3;
                e[1] = d2 * w2_2;
                e[2] = std::sqrt((e1_ts * e1_ts) + (e3_1 * e3_1));
            } else {
                const double d4 = e[0], d3 = e[1], d2 = e[2], d1 = e[3];
                const double e4_2 = d4 * w4_2;
                const double e2_2 = d2 * w2_2;
                const double e3_1 = d3 * w3_1;
                const double e1_ts = d1 * ts;
                e[0] = d4 * w4_4;
                e[1] = d3 * w3_3;
                e[2] = std::sqrt((e2_2 * e2_2) + (e4_2 * e4_2));
                e[3] = std::sqrt((e1_ts * e1_ts) + (e3_1 * e3_1));
            }
        }
    }
    // shift_cheb_errors_batch: error j scaled by (scale_next / scale_cur)^(np - j)
    auto rescale = [&](std::vector<double>& v, double scale_next, double scale_cur) {
        const double p = scale_next / scale_cur;
        for (uint64_t i = 0; i < nf; ++i) {
            for (uint32_t j = 0; j < np; ++j) {
                v[i * np + j] = v[i * np + j] * std::pow(p, static_cast<double>(np - j));
            }
        }
    };
    const double nbins_d = static_cast<double>(cfg.nbins);
    const double dphi = cfg.eta / nbins_d;
    for (uint64_t level = 1; level < nseg; ++level) {
        const auto cp = coord(level - 1);
        const auto cn = coord(level);
        const auto cc = std::pair<double, double>{cp.first, cn.second};
        rescale(cur, cc.second, cp.second);
        for (uint64_t i = 0; i < nf; ++i) {
            const double factor = kCval / f0[i];
            for (uint32_t j = 0; j < np; ++j) {
                dnew[i * np + j] = dphi * factor;
            }
        }
        const double scale_factor = nbins_d / kCval;
        for (uint32_t j = 0; j < np; ++j) {
            for (uint64_t b = 0; b < nf; ++b) {
                const uint64_t idx = b * np + j;
                const double diff = std::abs(cur[idx] - dnew[idx]);
                shift[idx] = diff * scale_factor * f0[b];
            }
        }
        std::fill(nbr.begin(), nbr.end(), 1.0);
        for (uint64_t i = 0; i < nf; ++i) {
            for (uint32_t j = 0; j < np; ++j) {
                const uint64_t idx = i * np + j;
                if (shift[idx] < (cfg.eta - kFloatEps)) {
                    nxt[idx] = cur[idx];
                    continue;
                }
                const double ratio = cur[idx] / dnew[idx];
                const double c = std::ceil(ratio - kFloatEps);
                const uint64_t num = c < 1.0 ? 1 : static_cast<uint64_t>(c);
                nbr[i] *= static_cast<double>(num);
                nxt[idx] = cur[idx] / static_cast<double>(num);
            }
        }
        double children = 0.0, parents = 0.0;
        for (uint64_t i = 0; i < nf; ++i) {
            children += weights[i] * nbr[i];
            parents += weights[i];
            weights[i] *= nbr[i];
        }
        bp[level - 1] = children / parents;
        rescale(nxt, cn.second, cc.second);
        cur = nxt;
    }
    return bp;
}

// EPMultiPass's branch_max (lib/prune.cpp:648-651): the pattern of ref_seg 0,
// in the run's basis (1: Chebyshev).
uint64_t Plan::prune_branch_max(bool conservative, int basis) const {
    const std::vector<double> bp =
        basis == 1 ? branching_pattern_cheby(0) : branching_pattern(0, conservative);
    double mx = bp.empty() ? 0.0 : bp[0];
    for (double v : bp) {
        mx = std::max(mx, v);
    }
    return std::max<uint64_t>(static_cast<uint64_t>(std::ceil(mx * 2)), 32);
}

// PulsarSearchConfig::get_dparams / get_dparams_f / get_dparams_actual
// (lib/configs.cpp:152-174).
std::vector<double> Plan::dparams_at(double tseg_cur, int kind) const {
    const double t_ref = (nparams == 1) ? 0.0 : tseg_cur / 2.0;
    if (kind == 1) {
        return poly_taylor_step_f(nparams, tseg_cur, cfg.nbins, cfg.eta, t_ref);
    }
    auto d = poly_taylor_step_d_f(nparams, tseg_cur, cfg.nbins, cfg.eta,
                                  lim_max(nparams - 1), t_ref);
    if (kind == 2) {
        for (uint32_t i = 0; i < nparams; ++i) {
            const uint64_t c = range_param_count(lim_min(i), lim_max(i), d[i]);
            d[i] = (lim_max(i) - lim_min(i)) / static_cast<double>(c);
        }
    }
    return d;
}

Plan make_plan(const lk_config& cfg, bool sizes_only) {
    Plan p;
    p.cfg = cfg;
    const uint32_t np = cfg.nparams;
    require(np >= 1 && np <= LK_MAX_PARAMS, "nparams must be in [1, 5]");
    p.nparams = np;
    const double f_min = p.lim_min(np - 1);
    const double f_max = p.lim_max(np - 1);

    // PulsarSearchConfig::Impl ctor + validate (lib/configs.cpp:64-95,262-302).
    require(cfg.nsamps > 0, "nsamps must be positive");
    require(is_pow2(cfg.nsamps), "nsamps must be a power of 2");
    require(cfg.tsamp > 0, "tsamp must be positive");
    require(cfg.eta > 0, "eta (tolerance bins) must be positive");
    require(cfg.nbins >= 1, "nbins must be positive");
    if (cfg.bseg_brute != 0) {
        p.bseg_brute = cfg.bseg_brute;
    } else {
        // get_bseg_brute_default (lib/configs.cpp:295-300).
        const uint64_t init_levels = (np == 1) ? 1 : 2;
        const auto levels = static_cast<uint64_t>(
            std::log2(static_cast<double>(cfg.nsamps) * cfg.tsamp * f_min));
        require(levels >= init_levels,
                "observation too short for f_min: cannot derive the default bseg_brute");
        p.bseg_brute = cfg.nsamps / (uint64_t{1} << (levels - init_levels));
    }
    p.bseg_ffa = cfg.bseg_ffa != 0 ? cfg.bseg_ffa : cfg.nsamps;
    require(is_pow2(p.bseg_brute), "bseg_brute must be a power of 2");
    require(is_pow2(p.bseg_ffa), "bseg_ffa must be a power of 2");
    require(p.bseg_brute < cfg.nsamps, "bseg_brute must be less than nsamps");
    require(p.bseg_ffa <= cfg.nsamps, "bseg_ffa must be less than or equal to nsamps");
    require(p.bseg_ffa >= p.bseg_brute, "bseg_ffa must be greater than or equal to bseg_brute");
    for (uint32_t i = 0; i < np; ++i) {
        require(p.lim_max(i) >= p.lim_min(i),
                "param_limits[" + std::to_string(i) + "] must be increasing");
    }
    p.tseg_brute = static_cast<double>(p.bseg_brute) * cfg.tsamp;
    p.tseg_ffa = static_cast<double>(p.bseg_ffa) * cfg.tsamp;
    const auto niters = static_cast<uint64_t>(
        std::log2(static_cast<double>(p.bseg_ffa) / static_cast<double>(p.bseg_brute)));
    require(niters + 1 <= LK_MAX_LEVELS, "too many FFA levels");
    p.n_levels = static_cast<uint32_t>(niters + 1);

    if (cfg.n_score_widths == 0) {
        p.widths = box_width_trials(cfg.nbins, cfg.ducy_max, cfg.wtsp);
    } else {
        require(cfg.n_score_widths <= LK_MAX_WIDTHS, "too many score widths");
        p.widths.assign(cfg.score_widths, cfg.score_widths + cfg.n_score_widths);
    }
    require(!p.widths.empty() && p.widths.size() <= LK_MAX_WIDTHS, "bad score widths");
    for (auto w : p.widths) {
        require(w >= 1 && w < cfg.nbins, "score widths must lie in [1, nbins)");
    }

    // FFAPlanBase::Impl::configure_plan (lib/plans.cpp:264-320).
    const uint32_t L = p.n_levels;
    p.segment_lens.resize(L);
    p.nsegments.resize(L);
    p.tsegments.resize(L);
    p.ncoords.resize(L);
    p.ncoords_offsets.resize(L + 1);
    p.param_counts.assign(L, std::vector<uint64_t>(np));
    p.dparams.assign(L, std::vector<double>(np));
    p.dparams_actual.assign(L, std::vector<double>(np));
    uint64_t offset = 0;
    for (uint32_t l = 0; l < L; ++l) {
        const uint64_t segment_len = p.bseg_brute * (uint64_t{1} << l);
        const double tsegment = static_cast<double>(segment_len) * cfg.tsamp;
        p.segment_lens[l] = segment_len;
        p.nsegments[l] = cfg.nsamps / segment_len;
        p.tsegments[l] = tsegment;
        // PulsarSearchConfig::get_dparams (lib/configs.cpp:158-162).
        const double t_ref = (np == 1) ? 0.0 : tsegment / 2.0;
        p.dparams[l] = poly_taylor_step_d_f(np, tsegment, cfg.nbins, cfg.eta, f_max, t_ref);
        uint64_t nc = 1;
        for (uint32_t i = 0; i < np; ++i) {
            const uint64_t c = range_param_count(p.lim_min(i), p.lim_max(i), p.dparams[l][i]);
            p.param_counts[l][i] = c;
            // get_dparams_actual (lib/configs.cpp:164-174).
            p.dparams_actual[l][i] = (p.lim_max(i) - p.lim_min(i)) / static_cast<double>(c);
            nc *= c;
        }
        p.ncoords[l] = nc;
        // The level offsets are 32-bit (as the reference's). A plan made for
        // its sizes only (a configuration, the sweep planner's probes) may
        // exceed that; executors and coordinate resolution refuse it.
        if (offset + nc > 0xffffffffULL) {
            require(sizes_only, "coordinate offsets exceed 32 bits");
            p.offsets_overflow = true;
        }
        p.ncoords_offsets[l] = static_cast<uint32_t>(offset);
        offset += nc;
        p.buffer_size = std::max(p.buffer_size, p.fold_size(l));
    }
    p.ncoords_offsets[L] = static_cast<uint32_t>(offset);
    p.coord_size = offset;
    // FFAPlanBase::Impl::validate_plan (lib/plans.cpp:322-333).
    for (uint32_t i = 0; i + 1 < np; ++i) {
        require(p.param_counts[0][i] == 1,
                "FFAPlan::validate_plan: Only one parameter for higher order derivatives is "
                "supported for the initialization for the first level");
    }
    // Final coordinates index the fold with 32-bit values (sizes-only plans
    // are flagged instead, like the offsets).
    if (p.ncoords[L - 1] > 0xffffffffULL) {
        require(sizes_only, "too many final coordinates");
        p.offsets_overflow = true;
    }
    return p;
}

}  // namespace lk
