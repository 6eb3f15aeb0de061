/* Test infrastructure only: C restatement of the reference's time-domain
 * FFA / boxcar-score path. See loki_oracle.h for the contract. Reference
 * citations are paths inside the reference project. */
#include "loki_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* utils::kCval, kInvCval, kFloatEps (lib/loki/utils.hpp:11-15). */
static const double kCval = 299792458.0;
static const double kInvCval = 3.3356409519815204e-09;
static const double kFloatEps = 1e-6;

static _Thread_local char g_err[512];

const char* lko_last_error(void) { return g_err; }

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return 1;
}

static int is_pow2(uint64_t x) { return x != 0 && (x & (x - 1)) == 0; }

/* math::factorial for floating types is std::tgamma(n + 1)
 * (lib/loki/math.hpp:35-44). */
static double factorial_d(double n) { return tgamma(n + 1.0); }

/* psr_utils::poly_taylor_step_f (lib/psr_utils.cpp:14-29). */
static void poly_taylor_step_f(uint32_t nparams, double tobs, uint64_t fold_bins,
                               double tol_bins, double t_ref, double* out) {
    const double dphi = tol_bins / (double)fold_bins;
    const double dt = tobs - t_ref;
    for (uint32_t i = 0; i < nparams; ++i) {
        const double orth_factor = pow(2.0, (double)i);
        out[nparams - 1 - i] =
            dphi * orth_factor * factorial_d((double)(i + 1)) / pow(dt, (double)(i + 1));
    }
}

/* psr_utils::poly_taylor_step_d_f (lib/psr_utils.cpp:31-45). */
static void poly_taylor_step_d_f(uint32_t nparams, double tobs, uint64_t fold_bins,
                                 double tol_bins, double f_max, double t_ref, double* out) {
    double f[LKO_MAX_PARAMS];
    poly_taylor_step_f(nparams, tobs, fold_bins, tol_bins, t_ref, f);
    for (uint32_t i = 0; i + 1 < nparams; ++i) {
        out[i] = f[i] * kCval / f_max;
    }
    out[nparams - 1] = f[nparams - 1];
}

/* psr_utils::range_param_count (lib/loki/psr_utils.hpp:235-242); the
 * reference throws when vmax <= vmin or dv <= 0, signalled here by 0. */
uint64_t lko_range_param_count(double vmin, double vmax, double dv) {
    if (!(vmax > vmin) || !(dv > 0)) {
        return 0;
    }
    if (dv >= (vmax - vmin)) {
        return 1;
    }
    return (uint64_t)ceil((vmax - vmin) / dv);
}

uint64_t lko_range_param(double vmin, double vmax, double dv, double* out, uint64_t max_out) {
    if (!(vmax > vmin) || !(dv > 0)) {
        return 0;
    }
    if (dv >= (vmax - vmin)) {
        if (max_out >= 1) {
            out[0] = (vmax + vmin) / 2.0;
        }
        return 1;
    }
    const uint64_t npoints = (uint64_t)ceil((vmax - vmin) / dv);
    const double dv_actual = (vmax - vmin) / (double)npoints;
    const double start = vmin + (0.5 * dv_actual);
    for (uint64_t i = 0; i < npoints && i < max_out; ++i) {
        out[i] = start + (dv_actual * (double)i);
    }
    return npoints;
}

/* detection::generate_box_width_trials (lib/score.cpp:390-405). */
uint64_t lko_box_widths(uint64_t nbins, double ducy_max, double wtsp, uint64_t* out,
                        uint64_t max_out) {
    double m = ducy_max * (double)nbins;
    if (m < 1.0) {
        m = 1.0;
    }
    const uint64_t wmax = (uint64_t)m;
    uint64_t n = 0;
    out[n++] = 1;
    while (out[n - 1] < wmax) {
        const uint64_t a = out[n - 1] + 1;
        const uint64_t b = (uint64_t)(wtsp * (double)out[n - 1]);
        const uint64_t next = a > b ? a : b;
        if (next > wmax || n >= max_out) {
            break;
        }
        out[n++] = next;
    }
    return n;
}

/* PulsarSearchConfig::Impl (lib/configs.cpp:16-95, 152-184, 262-302) and
 * FFAPlanBase::Impl::configure_plan / validate_plan (lib/plans.cpp:264-333),
 * FFAPlan::get_buffer_size (lib/plans.cpp:463-470). */
int lko_plan_create(const lko_cfg* cfg, lko_plan* p) {
    memset(p, 0, sizeof(*p));
    const uint32_t np = cfg->nparams;
    if (np < 1 || np > LKO_MAX_PARAMS) {
        return fail("nparams must be in [1, %d]", LKO_MAX_PARAMS);
    }
    p->nparams = np;
    p->nsamps = cfg->nsamps;
    p->nbins = cfg->nbins;
    p->tsamp = cfg->tsamp;
    p->eta = cfg->eta;
    memcpy(p->limits, cfg->limits, sizeof(p->limits));
    const double f_min = cfg->limits[2 * (np - 1)];
    const double f_max = cfg->limits[2 * (np - 1) + 1];
    if (cfg->bseg_brute != 0) {
        p->bseg_brute = cfg->bseg_brute;
    } else {
        const uint64_t init_levels = (np == 1) ? 1 : 2;
        const uint64_t levels = (uint64_t)log2((double)cfg->nsamps * cfg->tsamp * f_min);
        p->bseg_brute = cfg->nsamps / (uint64_t)(1U << (unsigned)(levels - init_levels));
    }
    p->bseg_ffa = cfg->bseg_ffa != 0 ? cfg->bseg_ffa : cfg->nsamps;
    if (cfg->nsamps == 0 || !is_pow2(cfg->nsamps)) {
        return fail("nsamps must be a positive power of 2");
    }
    if (!(cfg->tsamp > 0)) {
        return fail("tsamp must be positive");
    }
    if (!(cfg->eta > 0)) {
        return fail("eta (tolerance bins) must be positive");
    }
    if (!is_pow2(p->bseg_brute) || !is_pow2(p->bseg_ffa)) {
        return fail("bseg_brute and bseg_ffa must be powers of 2");
    }
    if (!(p->bseg_brute < cfg->nsamps)) {
        return fail("bseg_brute must be less than nsamps");
    }
    if (!(p->bseg_ffa <= cfg->nsamps) || !(p->bseg_ffa >= p->bseg_brute)) {
        return fail("bseg_ffa must lie in [bseg_brute, nsamps]");
    }
    for (uint32_t i = 0; i < np; ++i) {
        if (!(cfg->limits[2 * i + 1] >= cfg->limits[2 * i])) {
            return fail("param_limits[%u] must be increasing", i);
        }
    }
    p->tseg_brute = (double)p->bseg_brute * cfg->tsamp;
    const uint64_t niters = (uint64_t)log2((double)p->bseg_ffa / (double)p->bseg_brute);
    if (niters + 1 > LKO_MAX_LEVELS) {
        return fail("too many levels");
    }
    p->n_levels = (uint32_t)(niters + 1);
    p->n_widths = (uint32_t)lko_box_widths(cfg->nbins, cfg->ducy_max, cfg->wtsp, p->widths,
                                           LKO_MAX_WIDTHS);
    uint64_t offset = 0;
    uint64_t buffer = 0;
    for (uint32_t l = 0; l < p->n_levels; ++l) {
        const uint64_t segment_len = p->bseg_brute * (uint64_t)(1U << l);
        const double tsegment = (double)segment_len * cfg->tsamp;
        p->segment_lens[l] = segment_len;
        p->nsegments[l] = cfg->nsamps / segment_len;
        p->tsegments[l] = tsegment;
        const double t_ref = (np == 1) ? 0.0 : tsegment / 2.0;
        poly_taylor_step_d_f(np, tsegment, cfg->nbins, cfg->eta, f_max, t_ref, p->dparams[l]);
        uint64_t nc = 1;
        for (uint32_t i = 0; i < np; ++i) {
            const uint64_t c =
                lko_range_param_count(cfg->limits[2 * i], cfg->limits[2 * i + 1], p->dparams[l][i]);
            if (c == 0) {
                return fail("vmax must be greater than vmin (param %u)", i);
            }
            p->param_counts[l][i] = c;
            nc *= c;
        }
        p->ncoords[l] = nc;
        p->ncoords_offsets[l] = (uint32_t)offset;
        offset += nc;
        const uint64_t fs = p->nsegments[l] * nc * 2 * cfg->nbins;
        if (fs > buffer) {
            buffer = fs;
        }
    }
    p->ncoords_offsets[p->n_levels] = (uint32_t)offset;
    p->coord_size = offset;
    p->buffer_size = buffer;
    for (uint32_t i = 0; i + 1 < np; ++i) {
        if (p->param_counts[0][i] != 1) {
            return fail("FFAPlan::validate_plan: Only one parameter for higher order derivatives "
                        "is supported for the initialization for the first level");
        }
    }
    (void)f_min;
    return 0;
}

/* psr_utils::get_phase_idx (lib/loki/psr_utils.hpp:32-49). */
float lko_phase_idx(double proper_time, double freq, uint64_t nbins, double delay) {
    const double total_phase = (proper_time - delay) * freq;
    const double norm_phase = total_phase - floor(total_phase);
    double iphase = norm_phase * (double)nbins;
    if (iphase >= (double)nbins) {
        iphase = 0.0;
    }
    return (float)iphase;
}

/* psr_utils::get_phase_idx_uint (lib/loki/psr_utils.hpp:53-63). */
uint32_t lko_phase_idx_uint(double proper_time, double freq, uint64_t nbins, double delay) {
    const float iphase = lko_phase_idx(proper_time, freq, nbins, delay);
    uint32_t iphase_int = (uint32_t)(iphase + 0.5F);
    if (iphase_int == nbins) {
        iphase_int = 0;
    }
    return iphase_int;
}

/* psr_utils::get_param_val_at_idx (lib/loki/psr_utils.hpp:283-293). */
double lko_param_val_at_idx(double vmin, double vmax, uint64_t count, uint64_t i) {
    if (count <= 1) {
        return (vmax + vmin) / 2.0;
    }
    const double dv_actual = (vmax - vmin) / (double)count;
    return vmin + (dv_actual * ((double)i + 0.5));
}

/* psr_utils::get_nearest_idx_analytical (lib/loki/psr_utils.hpp:304-320). */
uint64_t lko_nearest_idx(double val, double vmin, double vmax, uint64_t count) {
    if (count <= 1) {
        return 0;
    }
    const double raw_idx = (double)count * (val - vmin) / (vmax - vmin);
    const int idx = (int)(raw_idx + kFloatEps);
    if (idx < 0) {
        return 0;
    }
    if (idx >= (int)count) {
        return count - 1;
    }
    return (uint64_t)idx;
}

/* core::ffa_taylor_resolve_freq_batch (lib/taylor_ffa.cpp:249-271). */
int lko_resolve_freq(const lko_plan* p, lko_coord_freq* out) {
    if (p->nparams != 1) {
        return fail("resolve_coordinates_freq() only supports nparams=1");
    }
    memset(out, 0, sizeof(lko_coord_freq) * p->coord_size);
    const double fmin = p->limits[0];
    const double fmax = p->limits[1];
    for (uint32_t l = 1; l < p->n_levels; ++l) {
        const uint64_t n_cur = p->param_counts[l][0];
        const uint64_t n_prev = p->param_counts[l - 1][0];
        const double delta_t = ldexp(p->tseg_brute, (int)(l - 1));
        lko_coord_freq* c = out + p->ncoords_offsets[l];
        for (uint64_t i = 0; i < n_cur; ++i) {
            const double f_cur = lko_param_val_at_idx(fmin, fmax, n_cur, i);
            c[i].idx = (uint32_t)lko_nearest_idx(f_cur, fmin, fmax, n_prev);
            c[i].shift = lko_phase_idx(delta_t, f_cur, p->nbins, 0.0);
        }
    }
    return 0;
}

/* ffa_taylor_resolve_accel_batch<LATTER> (lib/taylor_ffa.cpp:19-86). */
static void resolve_accel(const lko_plan* p, uint32_t l, int latter, lko_coord* c) {
    const uint64_t n_accel_cur = p->param_counts[l][0];
    const uint64_t n_freq_cur = p->param_counts[l][1];
    const uint64_t n_accel_prev = p->param_counts[l - 1][0];
    const uint64_t n_freq_prev = p->param_counts[l - 1][1];
    const double amin = p->limits[0], amax = p->limits[1];
    const double fmin = p->limits[2], fmax = p->limits[3];
    const double tsegment = ldexp(p->tseg_brute, (int)(l - 1));
    const double delta_t = ((double)latter - 0.5) * tsegment;
    const double half_delta_t_sq = 0.5 * delta_t * delta_t;
    for (uint64_t ia = 0; ia < n_accel_cur; ++ia) {
        const double a_cur = lko_param_val_at_idx(amin, amax, n_accel_cur, ia);
        const double v_new = a_cur * delta_t;
        const double d_new = a_cur * half_delta_t_sq;
        const uint64_t idx_a = lko_nearest_idx(a_cur, amin, amax, n_accel_prev);
        for (uint64_t jf = 0; jf < n_freq_cur; ++jf) {
            const double f_cur = lko_param_val_at_idx(fmin, fmax, n_freq_cur, jf);
            const double f_new = f_cur * (1.0 - (v_new * kInvCval));
            const double delay_rel = d_new * kInvCval;
            const float phase = lko_phase_idx(delta_t, f_cur, p->nbins, delay_rel);
            const uint64_t idx_f = lko_nearest_idx(f_new, fmin, fmax, n_freq_prev);
            const uint32_t final_idx = (uint32_t)(idx_a * n_freq_prev + idx_f);
            lko_coord* d = &c[ia * n_freq_cur + jf];
            if (latter == 0) {
                d->i_tail = final_idx;
                d->shift_tail = phase;
            } else {
                d->i_head = final_idx;
                d->shift_head = phase;
            }
        }
    }
}

/* ffa_taylor_resolve_jerk_batch<LATTER> (lib/taylor_ffa.cpp:88-188), nparams=3. */
static void resolve_jerk(const lko_plan* p, uint32_t l, int latter, lko_coord* c) {
    const uint64_t n_jerk_cur = p->param_counts[l][0];
    const uint64_t n_accel_cur = p->param_counts[l][1];
    const uint64_t n_freq_cur = p->param_counts[l][2];
    const uint64_t n_jerk_prev = p->param_counts[l - 1][0];
    const uint64_t n_accel_prev = p->param_counts[l - 1][1];
    const uint64_t n_freq_prev = p->param_counts[l - 1][2];
    const double jmin = p->limits[0], jmax = p->limits[1];
    const double amin = p->limits[2], amax = p->limits[3];
    const double fmin = p->limits[4], fmax = p->limits[5];
    const double tsegment = ldexp(p->tseg_brute, (int)(l - 1));
    const double delta_t = ((double)latter - 0.5) * tsegment;
    const double delta_t_sq = delta_t * delta_t;
    const double delta_t_cubed = delta_t_sq * delta_t;
    const double half_delta_t_sq = 0.5 * delta_t_sq;
    const double sixth_delta_t_cubed = delta_t_cubed / 6.0;
    for (uint64_t ij = 0; ij < n_jerk_cur; ++ij) {
        const double j_cur = lko_param_val_at_idx(jmin, jmax, n_jerk_cur, ij);
        const double j_delta_t = j_cur * delta_t;
        const double half_j_delta_t_sq = 0.5 * j_cur * delta_t_sq;
        const double j_sixth_delta_t_cubed = j_cur * sixth_delta_t_cubed;
        const uint64_t idx_j = lko_nearest_idx(j_cur, jmin, jmax, n_jerk_prev);
        const uint64_t coord_j_offset = ij * n_accel_cur * n_freq_cur;
        const uint64_t idx_j_offset = idx_j * n_accel_prev * n_freq_prev;
        for (uint64_t ia = 0; ia < n_accel_cur; ++ia) {
            const double a_cur = lko_param_val_at_idx(amin, amax, n_accel_cur, ia);
            const double a_new = a_cur + j_delta_t;
            const double v_new = (a_cur * delta_t) + half_j_delta_t_sq;
            const double d_new = (a_cur * half_delta_t_sq) + j_sixth_delta_t_cubed;
            const uint64_t idx_a = lko_nearest_idx(a_new, amin, amax, n_accel_prev);
            const uint64_t coord_a_offset = coord_j_offset + (ia * n_freq_cur);
            const uint64_t idx_a_offset = idx_j_offset + (idx_a * n_freq_prev);
            for (uint64_t jf = 0; jf < n_freq_cur; ++jf) {
                const double f_cur = lko_param_val_at_idx(fmin, fmax, n_freq_cur, jf);
                const double f_new = f_cur * (1.0 - (v_new * kInvCval));
                const double delay_rel = d_new * kInvCval;
                const float phase = lko_phase_idx(delta_t, f_cur, p->nbins, delay_rel);
                const uint64_t idx_f = lko_nearest_idx(f_new, fmin, fmax, n_freq_prev);
                const uint32_t final_idx = (uint32_t)(idx_a_offset + idx_f);
                lko_coord* d = &c[coord_a_offset + jf];
                if (latter == 0) {
                    d->i_tail = final_idx;
                    d->shift_tail = phase;
                } else {
                    d->i_head = final_idx;
                    d->shift_head = phase;
                }
            }
        }
    }
}

/* FFAPlanBase::Impl::resolve_coordinates (lib/plans.cpp:64-94). The dispatch
 * in lib/taylor_ffa.cpp:288-310 maps its `latter` argument to the template
 * inverted, but both halves are always computed, so the tables are: tail
 * with delta_t = -tseg/2, head with delta_t = +tseg/2. */
int lko_resolve_taylor(const lko_plan* p, lko_coord* out) {
    if (p->nparams != 2 && p->nparams != 3) {
        return fail("resolve_coordinates: the oracle supports nparams in {2, 3}");
    }
    memset(out, 0, sizeof(lko_coord) * p->coord_size);
    for (uint32_t l = 1; l < p->n_levels; ++l) {
        lko_coord* c = out + p->ncoords_offsets[l];
        for (int latter = 0; latter <= 1; ++latter) {
            if (p->nparams == 2) {
                resolve_accel(p, l, latter, c);
            } else {
                resolve_jerk(p, l, latter, c);
            }
        }
    }
    return 0;
}

/* BruteFold<float>::Impl::compute_phase_time_domain, phase part
 * (lib/fold.cpp:113-127). */
void lko_phase_map(const double* freqs, uint64_t nfreqs, uint64_t segment_len, uint64_t nbins,
                   double tsamp, double t_ref, uint32_t* out) {
    for (uint64_t f = 0; f < nfreqs; ++f) {
        for (uint64_t i = 0; i < segment_len; ++i) {
            const double proper_time = ((double)i * tsamp) - t_ref;
            out[f * segment_len + i] = lko_phase_idx_uint(proper_time, freqs[f], nbins, 0.0);
        }
    }
}

/* Brute fold: every bucket (freq, bin) sums its samples in increasing
 * sample order, starting from 0.0f (lib/kernels.cpp:550-580), for every
 * segment (lib/kernels.cpp:1132-1154). Equivalent to one in-order pass over
 * the samples adding each to its bucket. */
int lko_brute_fold(const float* ts_e, const float* ts_v, uint64_t nsamps, const double* freqs,
                   uint64_t nfreqs, uint64_t segment_len, uint64_t nbins, double tsamp,
                   double t_ref, float* out) {
    if (nfreqs == 0) {
        return fail("BruteFold::Impl: Frequency array is empty");
    }
    if (segment_len == 0 || nsamps % segment_len != 0) {
        return fail("BruteFold::Impl: Number of samples is not a multiple of segment length");
    }
    const uint64_t nseg = nsamps / segment_len;
    uint32_t* map = (uint32_t*)malloc(sizeof(uint32_t) * nfreqs * segment_len);
    if (map == NULL) {
        return fail("out of memory");
    }
    lko_phase_map(freqs, nfreqs, segment_len, nbins, tsamp, t_ref, map);
    memset(out, 0, sizeof(float) * nseg * nfreqs * 2 * nbins);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < (int64_t)nseg; ++s) {
        const float* e = ts_e + (uint64_t)s * segment_len;
        const float* v = ts_v + (uint64_t)s * segment_len;
        for (uint64_t f = 0; f < nfreqs; ++f) {
            float* fe = out + (((uint64_t)s * nfreqs) + f) * 2 * nbins;
            float* fv = fe + nbins;
            const uint32_t* m = map + f * segment_len;
            for (uint64_t i = 0; i < segment_len; ++i) {
                fe[m[i]] += e[i];
                fv[m[i]] += v[i];
            }
        }
    }
    free(map);
    return 0;
}

static uint64_t shift_bins(float phase, uint64_t nbins) {
    uint64_t s = (uint64_t)(phase + 0.5F);
    if (s == nbins) {
        s = 0;
    }
    return s;
}

/* kernels::ffa_iter_freq -> shift_add_linear_with_buffer
 * (lib/kernels.cpp:118-146, 722-827): tail unshifted, head rotated right. */
void lko_merge_freq(const float* in, float* out, const lko_coord_freq* coords,
                    uint64_t ncur, uint64_t nprev, uint64_t nseg, uint64_t nbins) {
    const uint64_t fs = 2 * nbins;
    for (uint64_t s = 0; s < nseg; ++s) {
        for (uint64_t c = 0; c < ncur; ++c) {
            const float* tail = in + ((2 * s) * nprev + coords[c].idx) * fs;
            const float* head = in + ((2 * s + 1) * nprev + coords[c].idx) * fs;
            float* o = out + (s * ncur + c) * fs;
            const uint64_t sh = shift_bins(coords[c].shift, nbins);
            for (uint64_t r = 0; r < 2; ++r) {
                for (uint64_t j = 0; j < nbins; ++j) {
                    const uint64_t jh = (j + nbins - sh) % nbins;
                    o[r * nbins + j] = tail[r * nbins + j] + head[r * nbins + jh];
                }
            }
        }
    }
}

/* kernels::ffa_iter -> shift_add_binary_with_buffer
 * (lib/kernels.cpp:71-112, 829-940): both halves rotated right, summed
 * tail + head. */
void lko_merge_taylor(const float* in, float* out, const lko_coord* coords, uint64_t ncur,
                      uint64_t nprev, uint64_t nseg, uint64_t nbins) {
    const uint64_t fs = 2 * nbins;
    for (uint64_t s = 0; s < nseg; ++s) {
        for (uint64_t c = 0; c < ncur; ++c) {
            const float* tail = in + ((2 * s) * nprev + coords[c].i_tail) * fs;
            const float* head = in + ((2 * s + 1) * nprev + coords[c].i_head) * fs;
            float* o = out + (s * ncur + c) * fs;
            const uint64_t st = shift_bins(coords[c].shift_tail, nbins);
            const uint64_t sh = shift_bins(coords[c].shift_head, nbins);
            for (uint64_t r = 0; r < 2; ++r) {
                for (uint64_t j = 0; j < nbins; ++j) {
                    const uint64_t jt = (j + nbins - st) % nbins;
                    const uint64_t jh = (j + nbins - sh) % nbins;
                    o[r * nbins + j] = tail[r * nbins + jt] + head[r * nbins + jh];
                }
            }
        }
    }
}

/* FFA<float>::Impl::initialize_brute_fold + execute_unified
 * (lib/ffa.cpp:174-198, 242-310). */
int lko_ffa(const lko_plan* p, const float* ts_e, const float* ts_v, uint32_t level_out,
            float* fold_out) {
    if (p->n_levels < 2) {
        return fail("FFA::execute_unified: levels must be greater than or equal to 2");
    }
    if (level_out >= p->n_levels) {
        return fail("level_out out of range");
    }
    const uint32_t np = p->nparams;
    const double fmin = p->limits[2 * (np - 1)];
    const double fmax = p->limits[2 * (np - 1) + 1];
    const uint64_t nfreq0 = p->param_counts[0][np - 1];
    double* freqs = (double*)malloc(sizeof(double) * nfreq0);
    float* a = (float*)malloc(sizeof(float) * p->buffer_size);
    float* b = (float*)malloc(sizeof(float) * p->buffer_size);
    void* coords = malloc((np == 1 ? sizeof(lko_coord_freq) : sizeof(lko_coord)) * p->coord_size);
    int rc = 0;
    if (freqs == NULL || a == NULL || b == NULL || coords == NULL) {
        rc = fail("out of memory");
        goto done;
    }
    lko_range_param(fmin, fmax, p->dparams[0][np - 1], freqs, nfreq0);
    const double t_ref = (np == 1) ? 0.0 : p->tsegments[0] / 2.0;
    rc = (np == 1) ? lko_resolve_freq(p, (lko_coord_freq*)coords)
                   : lko_resolve_taylor(p, (lko_coord*)coords);
    if (rc != 0) {
        goto done;
    }
    rc = lko_brute_fold(ts_e, ts_v, p->nsamps, freqs, nfreq0, p->segment_lens[0], p->nbins,
                        p->tsamp, t_ref, a);
    if (rc != 0) {
        goto done;
    }
    for (uint32_t l = 1; l <= level_out; ++l) {
        if (np == 1) {
            lko_merge_freq(a, b, (const lko_coord_freq*)coords + p->ncoords_offsets[l],
                           p->ncoords[l], p->ncoords[l - 1], p->nsegments[l], p->nbins);
        } else {
            lko_merge_taylor(a, b, (const lko_coord*)coords + p->ncoords_offsets[l],
                             p->ncoords[l], p->ncoords[l - 1], p->nsegments[l], p->nbins);
        }
        float* t = a;
        a = b;
        b = t;
    }
    memcpy(fold_out, a,
           sizeof(float) * p->nsegments[level_out] * p->ncoords[level_out] * 2 * p->nbins);
done:
    free(freqs);
    free(a);
    free(b);
    free(coords);
    return rc;
}

/* utils::circular_prefix_sum (lib/utils.cpp:33-67). */
void lko_circular_prefix_sum(const float* x, float* out, uint64_t nbins, uint64_t nsum) {
    if (nbins == 0 || nsum == 0) {
        return;
    }
    out[0] = x[0];
    for (uint64_t i = 1; i < nbins; ++i) {
        out[i] = out[i - 1] + x[i];
    }
    if (nsum <= nbins) {
        return;
    }
    const float last_sum = out[nbins - 1];
    const uint64_t first_wrap_end = (2 * nbins < nsum) ? 2 * nbins : nsum;
    for (uint64_t i = nbins; i < first_wrap_end; ++i) {
        out[i] = out[i - nbins] + last_sum;
    }
    for (uint64_t i = 2 * nbins; i < nsum; ++i) {
        const uint64_t wrap_count = i / nbins;
        const uint64_t pos = i % nbins;
        out[i] = out[pos] + ((float)wrap_count * last_sum);
    }
}

/* utils::diff_max (lib/utils.cpp:22-31). */
static float diff_max(const float* x, const float* y, uint64_t size) {
    float m = -FLT_MAX;
    for (uint64_t i = 0; i < size; ++i) {
        const float d = x[i] - y[i];
        m = (m < d) ? d : m; /* std::max(m, d): m unless m < d */
    }
    return m;
}

/* snr_boxcar_impl<Is3D, FindMax> (lib/score.cpp:95-172). */
static void snr_boxcar(int is3d, int find_max, const float* folds, uint64_t nprof,
                       uint64_t nbins, const uint64_t* widths, uint64_t nw, float stdnoise,
                       float* scores) {
    uint64_t wmax = 0;
    for (uint64_t i = 0; i < nw; ++i) {
        wmax = widths[i] > wmax ? widths[i] : wmax;
    }
    float h[LKO_MAX_WIDTHS], b[LKO_MAX_WIDTHS];
    for (uint64_t i = 0; i < nw; ++i) {
        const uint64_t w = widths[i];
        h[i] = sqrtf((float)(nbins - w) / (float)(nbins * w));
        b[i] = (float)w * h[i] / (float)(nbins - w);
    }
    const float inv_stdnoise = is3d ? 1.0F : (1.0F / stdnoise);
#pragma omp parallel
    {
        float* work = (float*)malloc(sizeof(float) * nbins);
        float* psum = (float*)calloc(nbins + wmax, sizeof(float));
#pragma omp for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)nprof; ++ii) {
            const uint64_t i = (uint64_t)ii;
            const float* fp;
            if (is3d) {
                const float* e = folds + i * 2 * nbins;
                const float* v = e + nbins;
                for (uint64_t j = 0; j < nbins; ++j) {
                    const float inv_sqrt_v = 1.0F / sqrtf(v[j]);
                    work[j] = e[j] * inv_sqrt_v;
                }
                fp = work;
            } else {
                fp = folds + i * nbins;
            }
            lko_circular_prefix_sum(fp, psum, nbins, nbins + wmax);
            const float sum = psum[nbins - 1];
            float max_snr = -FLT_MAX;
            for (uint64_t iw = 0; iw < nw; ++iw) {
                const float dmax = diff_max(psum + widths[iw], psum, nbins);
                const float snr_base = ((h[iw] + b[iw]) * dmax) - (b[iw] * sum);
                const float snr = snr_base * inv_stdnoise;
                if (find_max) {
                    max_snr = (max_snr < snr) ? snr : max_snr;
                } else {
                    scores[i * nw + iw] = snr;
                }
            }
            if (find_max) {
                scores[i] = max_snr;
            }
        }
        free(work);
        free(psum);
    }
}

void lko_snr_boxcar_3d(const float* folds, uint64_t nprof, uint64_t nbins, const uint64_t* widths,
                       uint64_t nw, float* scores) {
    snr_boxcar(1, 0, folds, nprof, nbins, widths, nw, 1.0F, scores);
}

void lko_snr_boxcar_3d_max(const float* folds, uint64_t nprof, uint64_t nbins,
                           const uint64_t* widths, uint64_t nw, float* scores) {
    snr_boxcar(1, 1, folds, nprof, nbins, widths, nw, 1.0F, scores);
}

void lko_snr_boxcar_2d_max(const float* folds, uint64_t nprof, uint64_t nbins,
                           const uint64_t* widths, uint64_t nw, float stdnoise, float* scores) {
    snr_boxcar(0, 1, folds, nprof, nbins, widths, nw, stdnoise, scores);
}

uint64_t lko_compact(const float* scores, uint64_t n, float snr_min, uint32_t* idx_out,
                     float* score_out) {
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (scores[i] >= snr_min) {
            idx_out[k] = (uint32_t)i;
            score_out[k] = scores[i];
            ++k;
        }
    }
    return k;
}
