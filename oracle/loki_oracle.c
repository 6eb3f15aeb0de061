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
    /* every output row is independent: rows are split over threads */
#pragma omp parallel for schedule(static)
    for (int64_t sc = 0; sc < (int64_t)(nseg * ncur); ++sc) {
        const uint64_t s = (uint64_t)sc / ncur, c = (uint64_t)sc % ncur;
        {
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
#pragma omp parallel for schedule(static)
    for (int64_t sc = 0; sc < (int64_t)(nseg * ncur); ++sc) {
        const uint64_t s = (uint64_t)sc / ncur, c = (uint64_t)sc % ncur;
        {
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

/* ======================================================================== */
/* FP64 statement of the FFA + boxcar S/N (the error reference of the FP32    */
/* and BF16-stored device paths): the same algorithm with every sum in        */
/* double -- the FP32 path's phase map and coordinate tables (so the same    */
/* samples land in the same bins and the same rows are merged with the same  */
/* shifts), brute fold and merges as lko_brute_fold / lko_merge_*, scores as */
/* snr_boxcar (lib/score.cpp:95-172) with double prefix sums and constants.  */
/* ======================================================================== */

static void merge64(const double* in, double* out, const void* coords, int taylor, uint64_t ncur,
                    uint64_t nprev, uint64_t nseg, uint64_t nbins) {
    const uint64_t fs = 2 * nbins;
#pragma omp parallel for schedule(static)
    for (int64_t sc = 0; sc < (int64_t)(nseg * ncur); ++sc) {
        const uint64_t s = (uint64_t)sc / ncur, c = (uint64_t)sc % ncur;
        uint64_t it, ih, st, sh;
        if (taylor) {
            const lko_coord* cc = (const lko_coord*)coords + c;
            it = cc->i_tail;
            ih = cc->i_head;
            st = shift_bins(cc->shift_tail, nbins);
            sh = shift_bins(cc->shift_head, nbins);
        } else {
            const lko_coord_freq* cc = (const lko_coord_freq*)coords + c;
            it = ih = cc->idx;
            st = 0;
            sh = shift_bins(cc->shift, nbins);
        }
        const double* tail = in + ((2 * s) * nprev + it) * fs;
        const double* head = in + ((2 * s + 1) * nprev + ih) * fs;
        double* o = out + (s * ncur + c) * fs;
        for (uint64_t r = 0; r < 2; ++r) {
            for (uint64_t j = 0; j < nbins; ++j) {
                o[r * nbins + j] =
                    tail[r * nbins + (j + nbins - st) % nbins] + head[r * nbins + (j + nbins - sh) % nbins];
            }
        }
    }
}

/* snr_boxcar_impl<Is3D=true> (lib/score.cpp:95-172) in double: per profile
 * x_j = E_j / sqrt(V_j), circular prefix sums, the largest window sum of
 * each width and (h + b) * dmax - b * sum(x). folds [nc][2][nbins]. */
static void score64(const double* a, uint64_t nc, uint64_t nbins, const uint64_t* widths,
                    uint64_t nw, double* scores) {
    uint64_t wmax = 0;
    double hb[LKO_MAX_WIDTHS], bb[LKO_MAX_WIDTHS];
    for (uint64_t k = 0; k < nw; ++k) {
        const double w = (double)widths[k];
        const double h = sqrt(((double)nbins - w) / ((double)nbins * w));
        bb[k] = w * h / ((double)nbins - w);
        hb[k] = h + bb[k];
        wmax = widths[k] > wmax ? widths[k] : wmax;
    }
#pragma omp parallel
    {
        double* ps = (double*)malloc(sizeof(double) * (nbins + wmax));
#pragma omp for schedule(static)
        for (int64_t ci = 0; ci < (int64_t)nc; ++ci) {
            const double* e = a + (uint64_t)ci * 2 * nbins;
            const double* v = e + nbins;
            double acc = 0.0;
            for (uint64_t j = 0; j < nbins; ++j) {
                acc += e[j] / sqrt(v[j]);
                ps[j] = acc;
            }
            for (uint64_t k = 0; k < wmax; ++k) {
                ps[nbins + k] = ps[k] + acc;
            }
            for (uint64_t k = 0; k < nw; ++k) {
                double dm = -DBL_MAX;
                for (uint64_t j = 0; j < nbins; ++j) {
                    const double d = ps[j + widths[k]] - ps[j];
                    dm = d > dm ? d : dm;
                }
                scores[(uint64_t)ci * nw + k] = hb[k] * dm - bb[k] * acc;
            }
        }
        free(ps);
    }
}

int lko_ffa_scores64(const lko_plan* p, const float* ts_e, const float* ts_v,
                     const uint64_t* widths, uint64_t nw, double* scores) {
    if (p->n_levels < 2 || p->nsegments[p->n_levels - 1] != 1) {
        return fail("lko_ffa_scores64: the final level must have one segment");
    }
    if (nw == 0 || nw > LKO_MAX_WIDTHS) {
        return fail("lko_ffa_scores64: number of widths out of range");
    }
    const uint32_t np = p->nparams;
    const uint64_t nbins = p->nbins;
    const uint64_t nfreq0 = p->param_counts[0][np - 1];
    const uint64_t seglen = p->segment_lens[0];
    const uint64_t nseg0 = p->nsegments[0];
    double* freqs = (double*)malloc(sizeof(double) * nfreq0);
    uint32_t* map = (uint32_t*)malloc(sizeof(uint32_t) * nfreq0 * seglen);
    double* a = (double*)malloc(sizeof(double) * p->buffer_size);
    double* b = (double*)malloc(sizeof(double) * p->buffer_size);
    void* coords = malloc((np == 1 ? sizeof(lko_coord_freq) : sizeof(lko_coord)) * p->coord_size);
    int rc = 0;
    if (freqs == NULL || map == NULL || a == NULL || b == NULL || coords == NULL) {
        rc = fail("out of memory");
        goto done;
    }
    lko_range_param(p->limits[2 * (np - 1)], p->limits[2 * (np - 1) + 1], p->dparams[0][np - 1], freqs,
                    nfreq0);
    rc = (np == 1) ? lko_resolve_freq(p, (lko_coord_freq*)coords)
                   : lko_resolve_taylor(p, (lko_coord*)coords);
    if (rc != 0) {
        goto done;
    }
    lko_phase_map(freqs, nfreq0, seglen, nbins, p->tsamp, (np == 1) ? 0.0 : p->tsegments[0] / 2.0, map);
    memset(a, 0, sizeof(double) * nseg0 * nfreq0 * 2 * nbins);
#pragma omp parallel for schedule(static)
    for (int64_t sf = 0; sf < (int64_t)(nseg0 * nfreq0); ++sf) {
        const uint64_t s = (uint64_t)sf / nfreq0, f = (uint64_t)sf % nfreq0;
        const float* e = ts_e + s * seglen;
        const float* v = ts_v + s * seglen;
        double* fe = a + (s * nfreq0 + f) * 2 * nbins;
        double* fv = fe + nbins;
        const uint32_t* m = map + f * seglen;
        for (uint64_t i = 0; i < seglen; ++i) {
            fe[m[i]] += (double)e[i];
            fv[m[i]] += (double)v[i];
        }
    }
    for (uint32_t l = 1; l < p->n_levels; ++l) {
        const void* cl = (np == 1) ? (const void*)((const lko_coord_freq*)coords + p->ncoords_offsets[l])
                                   : (const void*)((const lko_coord*)coords + p->ncoords_offsets[l]);
        merge64(a, b, cl, np > 1, p->ncoords[l], p->ncoords[l - 1], p->nsegments[l], nbins);
        double* t = a;
        a = b;
        b = t;
    }
    score64(a, p->ncoords[p->n_levels - 1], nbins, widths, nw, scores);
done:
    free(freqs);
    free(map);
    free(a);
    free(b);
    free(coords);
    return rc;
}

/* ======================================================================== */
/* Pruning leaf step (Taylor basis).                                         */
/* ======================================================================== */

/* utils::kZeroEps (lib/loki/utils.hpp:15). */
static const double kZeroEps = 1e-12;

/* MiddleOutScheme order: np.argsort(|arange(nseg) - ref|, kind="stable")
 * (lib/loki/psr_utils.hpp:331-347): ref, then ref-1, ref+1, ref-2, ... with
 * the lower index first on equal distance. */
static void middle_out_order(uint64_t nseg, uint64_t ref, uint64_t* order) {
    uint64_t k = 0;
    order[k++] = ref;
    for (uint64_t d = 1; k < nseg; ++d) {
        if (d <= ref) {
            order[k++] = ref - d;
        }
        if (ref + d < nseg && k < nseg) {
            order[k++] = ref + d;
        }
    }
}

/* get_coord (lib/loki/psr_utils.hpp:378-393). */
static void mo_coord(const uint64_t* order, uint64_t level, double tseg, double* ref,
                     double* scale) {
    uint64_t mn = order[0], mx = order[0];
    for (uint64_t i = 1; i <= level; ++i) {
        mn = order[i] < mn ? order[i] : mn;
        mx = order[i] > mx ? order[i] : mx;
    }
    const double min_val = (double)mn;
    const double max_val = (double)mx;
    const double ref_val = (min_val + max_val + 1.0) / 2.0;
    const double scale_val = ref_val - min_val;
    *ref = ref_val * tseg;
    *scale = scale_val * tseg;
}

/* get_current_coord (lib/loki/psr_utils.hpp:440-448). */
static void mo_current_coord(const uint64_t* order, uint64_t level, double tseg, double* ref,
                             double* scale) {
    if (level == 0) {
        mo_coord(order, 0, tseg, ref, scale);
        return;
    }
    double pr, ps, cr, cs;
    mo_coord(order, level - 1, tseg, &pr, &ps);
    mo_coord(order, level, tseg, &cr, &cs);
    *ref = pr;
    *scale = cs;
}

/* get_segment_coord (lib/loki/psr_utils.hpp:402-408). */
static void mo_segment_coord(const uint64_t* order, uint64_t level, double tseg, double* ref,
                             double* scale) {
    const double idx = (double)order[level];
    *ref = (idx + 0.5) * tseg;
    *scale = 0.5 * tseg;
}

int lko_middle_out(uint64_t nseg, uint64_t ref_idx, double tseg, uint64_t level, double* out) {
    if (nseg == 0 || ref_idx >= nseg || level >= nseg) {
        return fail("MiddleOutScheme: invalid nsegments / ref_idx / level");
    }
    uint64_t* order = (uint64_t*)malloc(sizeof(uint64_t) * nseg);
    middle_out_order(nseg, ref_idx, order);
    out[0] = (double)order[level];
    mo_coord(order, level, tseg, &out[1], &out[2]);
    mo_current_coord(order, level, tseg, &out[3], &out[4]);
    mo_segment_coord(order, level, tseg, &out[5], &out[6]);
    free(order);
    return 0;
}

/* FFAPlan::get_dparams_actual of a level (lib/configs.cpp:164-174). */
static double dparam_actual(const lko_plan* p, uint32_t l, uint32_t i) {
    return (p->limits[2 * i + 1] - p->limits[2 * i]) / (double)p->param_counts[l][i];
}

/* core::poly_taylor_seed (lib/taylor.cpp:1197-1257). */
uint64_t lko_taylor_seed(const lko_plan* p, double* leaves) {
    const uint32_t np = p->nparams;
    const uint32_t L = p->n_levels - 1;
    if (np < 2 || np > 3) {
        fail("pruning supports nparams 2 or 3");
        return 0;
    }
    const uint64_t stride = (np + 2) * 2;
    const uint64_t n_accel = p->param_counts[L][np - 2];
    const uint64_t n_freq = p->param_counts[L][np - 1];
    if (p->ncoords[L] != n_accel * n_freq) {
        fail("n_leaves mismatch");
        return 0;
    }
    const double a_min = p->limits[2 * (np - 2)], a_max = p->limits[2 * (np - 2) + 1];
    const double f_min = p->limits[2 * (np - 1)], f_max = p->limits[2 * (np - 1) + 1];
    const double d_freq_cur = dparam_actual(p, L, np - 1);
    uint64_t leaf = 0;
    for (uint64_t ia = 0; ia < n_accel; ++ia) {
        const double accel_cur = lko_param_val_at_idx(a_min, a_max, n_accel, ia);
        for (uint64_t jf = 0; jf < n_freq; ++jf) {
            const double freq_cur = lko_param_val_at_idx(f_min, f_max, n_freq, jf);
            double* o = leaves + leaf * stride;
            for (uint32_t j = 0; j + 1 < np; ++j) {
                o[j * 2 + 0] = 0;
                o[j * 2 + 1] = dparam_actual(p, L, j);
            }
            o[(np - 2) * 2 + 0] = accel_cur;
            o[(np - 1) * 2 + 0] = 0;
            o[(np - 1) * 2 + 1] = d_freq_cur * (kCval / freq_cur);
            o[np * 2 + 0] = 0;
            o[np * 2 + 1] = 0;
            o[(np + 1) * 2 + 0] = freq_cur;
            o[(np + 1) * 2 + 1] = 0;
            ++leaf;
        }
    }
    return leaf;
}

/* Steps and shifts of one parent (lib/taylor.cpp:64-85 accel, 199-227 jerk):
 * param p holds derivative order k = np - p; K = 1, 4, 24 for k = 1, 2, 3. */
static void branch_steps(const double* lf, uint32_t np, double dt, double nbins_d, double dphi,
                         double* sig_new, double* shift) {
    const double dt2 = dt * dt;
    const double inv_dt = 1.0 / dt;
    const double inv_dt2 = inv_dt * inv_dt;
    const double f0 = lf[(np + 1) * 2];
    const double dfactor = kCval / f0;
    if (np == 2) {
        const double d2_sig_cur = lf[1], d1_sig_cur = lf[3];
        sig_new[0] = dphi * dfactor * 4.0 * inv_dt2;
        sig_new[1] = dphi * dfactor * 1.0 * inv_dt;
        shift[0] = fabs(d2_sig_cur - sig_new[0]) * dt2 * nbins_d / (4.0 * dfactor);
        shift[1] = fabs(d1_sig_cur - sig_new[1]) * dt * nbins_d / (1.0 * dfactor);
    } else {
        const double dt3 = dt2 * dt;
        const double inv_dt3 = inv_dt2 * inv_dt;
        const double d3_sig_cur = lf[1], d2_sig_cur = lf[3], d1_sig_cur = lf[5];
        sig_new[0] = dphi * dfactor * 24.0 * inv_dt3;
        sig_new[1] = dphi * dfactor * 4.0 * inv_dt2;
        sig_new[2] = dphi * dfactor * 1.0 * inv_dt;
        shift[0] = fabs(d3_sig_cur - sig_new[0]) * dt3 * nbins_d / (24.0 * dfactor);
        shift[1] = fabs(d2_sig_cur - sig_new[1]) * dt2 * nbins_d / (4.0 * dfactor);
        shift[2] = fabs(d1_sig_cur - sig_new[2]) * dt * nbins_d / (1.0 * dfactor);
    }
}

/* psr_utils::branch_one_param_padded + branch_param_padded
 * (lib/loki/psr_utils.hpp:189-211, lib/psr_utils.cpp:226-259): the count of
 * child values of one parameter, and (when vals != NULL) the values. */
static int branch_one(double cur, double sig_cur, double sig_new, double shift, double eta,
                      uint64_t branch_max, double* vals, double* dparam, uint64_t* count) {
    if (!(shift >= (eta - kFloatEps))) {
        if (vals != NULL) {
            vals[0] = cur;
        }
        *dparam = sig_cur;
        *count = 1;
        return 0;
    }
    if (sig_cur <= kZeroEps || sig_new <= kZeroEps) {
        return fail("Both dparam_cur and dparam_new must be positive (got %g, %g)", sig_cur,
                    sig_new);
    }
    const double ratio = sig_cur / sig_new;
    const double c = ceil(ratio - kFloatEps);
    const uint64_t num = c < 1.0 ? 1 : (uint64_t)c;
    if (num > branch_max) {
        return fail("num_points must be less than or equal to branch_max");
    }
    const double act = sig_cur / (double)num;
    const double parent_min = cur - (sig_cur / 2.0);
    const double first = parent_min + (act / 2.0);
    if (vals != NULL) {
        for (uint64_t i = 0; i < num; ++i) {
            vals[i] = first + ((double)i * act);
        }
    }
    *dparam = act;
    *count = num;
    return 0;
}

int lko_taylor_branch(const double* leaves, uint64_t n, uint32_t np, double t_cur,
                      double scale_cur, uint64_t nbins, double eta, uint64_t branch_max,
                      double* out, uint64_t* origins, uint64_t cap_out, uint64_t* n_out) {
    (void)t_cur;
    if (np < 2 || np > 3) {
        return fail("pruning supports nparams 2 or 3");
    }
    const uint64_t stride = (np + 2) * 2;
    const double dt = scale_cur; /* t_obs_minus_t_ref */
    const double nbins_d = (double)nbins;
    const double dphi = eta / nbins_d;
    /* Pass 1: children counts. */
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const double* lf = leaves + i * stride;
        double sig_new[3], shift[3], dp;
        branch_steps(lf, np, dt, nbins_d, dphi, sig_new, shift);
        uint64_t prod = 1;
        for (uint32_t k = 0; k < np; ++k) {
            uint64_t cnt;
            if (branch_one(lf[2 * k], lf[2 * k + 1], sig_new[k], shift[k], eta, branch_max, NULL,
                           &dp, &cnt) != 0) {
                return 1;
            }
            prod *= cnt;
        }
        total += prod;
    }
    *n_out = total;
    if (total > cap_out) {
        return 2;
    }
    /* Pass 2: Cartesian product, highest derivative outermost. */
    double* vals = (double*)malloc(sizeof(double) * 3 * (branch_max > 0 ? branch_max : 1));
    uint64_t o = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const double* lf = leaves + i * stride;
        double sig_new[3], shift[3], dp[3];
        uint64_t cnt[3] = {1, 1, 1};
        branch_steps(lf, np, dt, nbins_d, dphi, sig_new, shift);
        for (uint32_t k = 0; k < np; ++k) {
            branch_one(lf[2 * k], lf[2 * k + 1], sig_new[k], shift[k], eta, branch_max,
                       vals + k * branch_max, &dp[k], &cnt[k]);
        }
        for (uint64_t a = 0; a < cnt[0]; ++a) {
            for (uint64_t b = 0; b < cnt[1]; ++b) {
                for (uint64_t c = 0; c < (np == 3 ? cnt[2] : 1); ++c) {
                    double* d = out + o * stride;
                    d[0] = vals[a];
                    d[1] = dp[0];
                    d[2] = vals[branch_max + b];
                    d[3] = dp[1];
                    if (np == 3) {
                        d[4] = vals[2 * branch_max + c];
                        d[5] = dp[2];
                    }
                    memcpy(d + 2 * np, lf + 2 * np, 4 * sizeof(double));
                    origins[o] = i;
                    ++o;
                }
            }
        }
    }
    free(vals);
    return 0;
}

/* poly_taylor_resolve_accel_batch / _jerk_batch (lib/taylor.cpp:492-619). */
void lko_taylor_resolve(const lko_plan* p, const double* leaves, uint64_t n, const double* co,
                        uint64_t* param_idx, float* phase_shift) {
    const uint32_t np = p->nparams;
    const uint32_t L = p->n_levels - 1;
    const uint64_t stride = (np + 2) * 2;
    const uint64_t n_accel = p->param_counts[L][np - 2];
    const uint64_t n_freq = p->param_counts[L][np - 1];
    const double a_min = p->limits[2 * (np - 2)], a_max = p->limits[2 * (np - 2) + 1];
    const double f_min = p->limits[2 * (np - 1)], f_max = p->limits[2 * (np - 1) + 1];
    const double t0_add = co[0], t0_cur = co[2], t0_init = co[4];
    const double dt_add = t0_add - t0_cur;
    const double dt_init = t0_init - t0_cur;
    if (np == 2) {
        const double dt = dt_add - dt_init;
        const double half_dt2 = 0.5 * ((dt_add * dt_add) - (dt_init * dt_init));
        for (uint64_t i = 0; i < n; ++i) {
            const double* lf = leaves + i * stride;
            const double a_cur = lf[0], v_cur = lf[2], f0 = lf[6];
            const double a_new = a_cur;
            const double delta_v = a_cur * dt;
            const double delta_d = (v_cur * dt) + (a_cur * half_dt2);
            const double f_new = f0 * (1.0 - (delta_v * kInvCval));
            const double delay_rel = delta_d * kInvCval;
            const uint64_t ia = lko_nearest_idx(a_new, a_min, a_max, n_accel);
            const uint64_t jf = lko_nearest_idx(f_new, f_min, f_max, n_freq);
            param_idx[i] = (ia * n_freq) + jf;
            phase_shift[i] = lko_phase_idx(dt, f0, p->nbins, delay_rel);
        }
    } else {
        const double half_dt2_add = 0.5 * (dt_add * dt_add);
        const double half_dt2_init = 0.5 * (dt_init * dt_init);
        const double dt = dt_add - dt_init;
        const double half_dt2 = half_dt2_add - half_dt2_init;
        const double sixth_dt3 = ((half_dt2_add * dt_add) - (half_dt2_init * dt_init)) / 3.0;
        for (uint64_t i = 0; i < n; ++i) {
            const double* lf = leaves + i * stride;
            const double j_cur = lf[0], a_cur = lf[2], v_cur = lf[4], f0 = lf[8];
            const double a_new = a_cur + (j_cur * dt_add);
            const double delta_v = (a_cur * dt) + (j_cur * half_dt2);
            const double delta_d = (v_cur * dt) + (a_cur * half_dt2) + (j_cur * sixth_dt3);
            const double f_new = f0 * (1.0 - (delta_v * kInvCval));
            const double delay_rel = delta_d * kInvCval;
            phase_shift[i] = lko_phase_idx(dt, f0, p->nbins, delay_rel);
            const uint64_t ia = lko_nearest_idx(a_new, a_min, a_max, n_accel);
            const uint64_t jf = lko_nearest_idx(f_new, f_min, f_max, n_freq);
            param_idx[i] = (ia * n_freq) + jf;
        }
    }
}

/* poly_taylor_transform_{accel,jerk}_batch (lib/taylor.cpp:881-1005). */
void lko_taylor_transform(double* leaves, const uint64_t* indices, uint64_t n, uint32_t np,
                          double t_next, double t_cur, int conservative) {
    const uint64_t stride = (np + 2) * 2;
    const double dt = t_next - t_cur;
    if (np == 2) {
        const double half_dt2 = 0.5 * (dt * dt);
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + indices[i] * stride;
            const double d2v = lf[0], d2e = lf[1], d1v = lf[2], d1e = lf[3], d0v = lf[4],
                         d0e = lf[5];
            const double d2v_j = d2v;
            const double d1v_j = d1v + (d2v * dt);
            const double d0v_j = d0v + (d1v * dt) + (d2v * half_dt2);
            double d2e_j, d1e_j;
            if (conservative) {
                d2e_j = d2e;
                d1e_j = sqrt((d1e * d1e) + (d2e * d2e * dt * dt));
            } else {
                d2e_j = d2e;
                d1e_j = d1e;
            }
            lf[0] = d2v_j;
            lf[1] = d2e_j;
            lf[2] = d1v_j;
            lf[3] = d1e_j;
            lf[4] = d0v_j;
            lf[5] = d0e;
        }
    } else {
        const double dt2 = dt * dt;
        const double half_dt2 = 0.5 * (dt2);
        const double sixth_dt3 = dt2 * dt / 6.0;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + indices[i] * stride;
            const double d3v = lf[0], d3e = lf[1], d2v = lf[2], d2e = lf[3], d1v = lf[4],
                         d1e = lf[5], d0v = lf[6], d0e = lf[7];
            const double d3v_j = d3v;
            const double d2v_j = d2v + (d3v * dt);
            const double d1v_j = d1v + (d2v * dt) + (d3v * half_dt2);
            const double d0v_j = d0v + (d1v * dt) + (d2v * half_dt2) + (d3v * sixth_dt3);
            double d3e_j, d2e_j, d1e_j;
            if (conservative) {
                d3e_j = d3e;
                d2e_j = sqrt((d2e * d2e) + (d3e * d3e * dt2));
                d1e_j = sqrt((d1e * d1e) + (d2e * d2e * dt2) +
                             (d3e * d3e * half_dt2 * half_dt2));
            } else {
                d3e_j = d3e;
                d2e_j = d2e;
                d1e_j = d1e;
            }
            lf[0] = d3v_j;
            lf[1] = d3e_j;
            lf[2] = d2v_j;
            lf[3] = d2e_j;
            lf[4] = d1v_j;
            lf[5] = d1e_j;
            lf[6] = d0v_j;
            lf[7] = d0e;
        }
    }
}

/* ======================================================================== */
/* Chebyshev basis of the pruning leaf step (lib/chebyshev.cpp).            */
/* Leaves keep the Taylor layout [np + 2][value, error]: rows 0 .. np-1 the  */
/* Chebyshev coefficients alpha_np .. alpha_1, row np alpha_0, row np+1 f0.  */
/* ======================================================================== */

/* poly_taylor_to_cheby_{accel,jerk}_batch (lib/chebyshev.cpp:58-93,145-189),
 * ts = coord_init.second. */
void lko_taylor_to_cheby(double* leaves, uint64_t n, uint32_t np, double ts) {
    const uint64_t stride = (np + 2) * 2;
    const double ts2 = ts * ts;
    if (np == 2) {
        const double w2_2 = (ts2 / 2.0) * 0.5;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + i * stride;
            const double d2v = lf[0], d2e = lf[1], d1v = lf[2], d1e = lf[3], d0v = lf[4],
                         d0e = lf[5];
            lf[0] = d2v * w2_2;
            lf[2] = d1v * ts;
            lf[4] = d0v + (d2v * w2_2);
            const double e2 = d2e * w2_2;
            const double e1_ts = d1e * ts;
            lf[1] = e2;
            lf[3] = e1_ts;
            lf[5] = sqrt((d0e * d0e) + (e2 * e2));
        }
    } else {
        const double ts3 = ts2 * ts;
        const double w3_3 = (ts3 / 6.0) * 0.25;
        const double w2_2 = (ts2 / 2.0) * 0.5;
        const double w3_1 = (ts3 / 6.0) * 0.75;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + i * stride;
            const double d3v = lf[0], d3e = lf[1], d2v = lf[2], d2e = lf[3], d1v = lf[4],
                         d1e = lf[5], d0v = lf[6], d0e = lf[7];
            lf[0] = d3v * w3_3;
            lf[2] = d2v * w2_2;
            lf[4] = (d1v * ts) + (d3v * w3_1);
            lf[6] = d0v + (d2v * w2_2);
            const double e3_3 = d3e * w3_3;
            const double e2_2 = d2e * w2_2;
            const double e3_1 = d3e * w3_1;
            const double e1_ts = d1e * ts;
            lf[1] = e3_3;
            lf[3] = e2_2;
            lf[5] = sqrt((e1_ts * e1_ts) + (e3_1 * e3_1));
            lf[7] = sqrt((d0e * d0e) + (e2_2 * e2_2));
        }
    }
}

/* poly_cheby_to_taylor_{accel,jerk}_batch (lib/chebyshev.cpp:21-56,95-143),
 * ts = coord_report.second. */
void lko_cheby_to_taylor(double* leaves, uint64_t n, uint32_t np, double ts) {
    const uint64_t stride = (np + 2) * 2;
    const double inv_ts = 1.0 / ts;
    const double inv_ts2 = inv_ts * inv_ts;
    if (np == 2) {
        const double w2_2 = 4.0 * inv_ts2;
        const double w1_1 = inv_ts;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + i * stride;
            const double a2v = lf[0], a2e = lf[1], a1v = lf[2], a1e = lf[3], a0v = lf[4],
                         a0e = lf[5];
            lf[0] = a2v * w2_2;
            lf[2] = a1v * w1_1;
            lf[4] = a0v - a2v;
            lf[1] = a2e * w2_2;
            lf[3] = a1e * w1_1;
            lf[5] = sqrt((a0e * a0e) + (a2e * a2e));
        }
    } else {
        const double inv_ts3 = inv_ts2 * inv_ts;
        const double w3_3 = 24.0 * inv_ts3;
        const double w2_2 = 4.0 * inv_ts2;
        const double w1_1 = inv_ts;
        const double w3_1 = 3.0 * inv_ts;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + i * stride;
            const double a3v = lf[0], a3e = lf[1], a2v = lf[2], a2e = lf[3], a1v = lf[4],
                         a1e = lf[5], a0v = lf[6], a0e = lf[7];
            lf[0] = a3v * w3_3;
            lf[2] = a2v * w2_2;
            lf[4] = (a1v * w1_1) - (a3v * w3_1);
            lf[6] = a0v - a2v;
            const double e3_3 = a3e * w3_3;
            const double e2_2 = a2e * w2_2;
            const double e1_1 = a1e * w1_1;
            const double e3_1 = a3e * w3_1;
            lf[1] = e3_3;
            lf[3] = e2_2;
            lf[5] = sqrt((e1_1 * e1_1) + (e3_1 * e3_1));
            lf[7] = sqrt((a0e * a0e) + (a2e * a2e));
        }
    }
}

/* poly_chebyshev_transform_{accel,jerk}_batch (lib/chebyshev.cpp:316-409):
 * re-centre from coord_cur (t_cur, s_cur) to coord_next (t_next, s_next);
 * errors scaled by the diagonal (non-conservative). */
void lko_cheby_transform(double* leaves, const uint64_t* indices, uint64_t n, uint32_t np,
                         double t_next, double s_next, double t_cur, double s_cur) {
    const uint64_t stride = (np + 2) * 2;
    const double dt = t_next - t_cur;
    const double p = s_next / s_cur;
    const double q = dt / s_cur;
    const double p2 = p * p;
    const double q2 = q * q;
    if (np == 2) {
        const double pq = p * q;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + indices[i] * stride;
            const double a2v = lf[0], a2e = lf[1], a1v = lf[2], a1e = lf[3], a0v = lf[4];
            lf[0] = p2 * a2v;
            lf[2] = (p * a1v) + (4.0 * pq * a2v);
            lf[4] = a0v + (q * a1v) + ((p2 + (2.0 * q2) - 1.0) * a2v);
            lf[1] = p2 * a2e;
            lf[3] = p * a1e;
        }
    } else {
        const double p3 = p2 * p;
        for (uint64_t i = 0; i < n; ++i) {
            double* lf = leaves + indices[i] * stride;
            const double a3v = lf[0], a3e = lf[1], a2v = lf[2], a2e = lf[3], a1v = lf[4],
                         a1e = lf[5], a0v = lf[6];
            lf[0] = p3 * a3v;
            lf[2] = (6.0 * p2 * q * a3v) + (p2 * a2v);
            lf[4] = (3.0 * p * (p2 + (4.0 * q2) - 1.0) * a3v) + (4.0 * p * q * a2v) + (p * a1v);
            lf[6] = (q * ((6.0 * p2) + (4.0 * q2) - 3.0) * a3v) + ((p2 + (2.0 * q2) - 1.0) * a2v) +
                    (q * a1v) + a0v;
            lf[1] = p3 * a3e;
            lf[3] = p2 * a2e;
            lf[5] = p * a1e;
        }
    }
}

/* Steps and shifts of one (transformed) parent in the Chebyshev basis
 * (lib/chebyshev.cpp:530-551, 677-702): one step dphi C / f0 for every
 * coefficient, shift |sigma_cur - step| nbins / (C / f0). */
static void cheby_steps(const double* lf, uint32_t np, double nbins_d, double dphi,
                        double* sig_new, double* shift) {
    const double f0 = lf[(np + 1) * 2];
    const double dfactor = kCval / f0;
    const double base_step = dphi * dfactor;
    const double inv_base = nbins_d / dfactor;
    for (uint32_t k = 0; k < np; ++k) {
        sig_new[k] = base_step;
        shift[k] = fabs(lf[2 * k + 1] - base_step) * inv_base;
    }
}

/* poly_chebyshev_branch_{accel,jerk}_batch (lib/chebyshev.cpp:475-779): the
 * parents are first transformed in place from coord_prev to coord_cur, then
 * branched as in the Taylor basis (branch_one_param_padded, Cartesian
 * product with the highest coefficient outermost, alpha_0 and f0 copied). */
int lko_cheby_branch(double* leaves, uint64_t n, uint32_t np, double t_cur, double s_cur,
                     double t_prev, double s_prev, uint64_t nbins, double eta,
                     uint64_t branch_max, double* out, uint64_t* origins, uint64_t cap_out,
                     uint64_t* n_out) {
    if (np < 2 || np > 3) {
        return fail("pruning supports nparams 2 or 3");
    }
    const uint64_t stride = (np + 2) * 2;
    const double nbins_d = (double)nbins;
    const double dphi = eta / nbins_d;
    {
        uint64_t* ident = (uint64_t*)malloc(sizeof(uint64_t) * (n > 0 ? n : 1));
        for (uint64_t i = 0; i < n; ++i) {
            ident[i] = i;
        }
        lko_cheby_transform(leaves, ident, n, np, t_cur, s_cur, t_prev, s_prev);
        free(ident);
    }
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const double* lf = leaves + i * stride;
        double sig_new[3], shift[3], dp;
        cheby_steps(lf, np, nbins_d, dphi, sig_new, shift);
        uint64_t prod = 1;
        for (uint32_t k = 0; k < np; ++k) {
            uint64_t cnt;
            if (branch_one(lf[2 * k], lf[2 * k + 1], sig_new[k], shift[k], eta, branch_max, NULL,
                           &dp, &cnt) != 0) {
                return 1;
            }
            prod *= cnt;
        }
        total += prod;
    }
    *n_out = total;
    if (total > cap_out) {
        return 2;
    }
    double* vals = (double*)malloc(sizeof(double) * 3 * (branch_max > 0 ? branch_max : 1));
    uint64_t o = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const double* lf = leaves + i * stride;
        double sig_new[3], shift[3], dp[3];
        uint64_t cnt[3] = {1, 1, 1};
        cheby_steps(lf, np, nbins_d, dphi, sig_new, shift);
        for (uint32_t k = 0; k < np; ++k) {
            branch_one(lf[2 * k], lf[2 * k + 1], sig_new[k], shift[k], eta, branch_max,
                       vals + k * branch_max, &dp[k], &cnt[k]);
        }
        for (uint64_t a = 0; a < cnt[0]; ++a) {
            for (uint64_t b = 0; b < cnt[1]; ++b) {
                for (uint64_t c = 0; c < (np == 3 ? cnt[2] : 1); ++c) {
                    double* d = out + o * stride;
                    d[0] = vals[a];
                    d[1] = dp[0];
                    d[2] = vals[branch_max + b];
                    d[3] = dp[1];
                    if (np == 3) {
                        d[4] = vals[2 * branch_max + c];
                        d[5] = dp[2];
                    }
                    memcpy(d + 2 * np, lf + 2 * np, 4 * sizeof(double));
                    origins[o] = i;
                    ++o;
                }
            }
        }
    }
    free(vals);
    return 0;
}

/* poly_chebyshev_resolve_{accel,jerk}_batch (lib/chebyshev.cpp:961-1097);
 * co = {t_add, s_add, t_cur, s_cur, t_init, s_init}. */
void lko_cheby_resolve(const lko_plan* p, const double* leaves, uint64_t n, const double* co,
                       uint64_t* param_idx, float* phase_shift) {
    const uint32_t np = p->nparams;
    const uint32_t L = p->n_levels - 1;
    const uint64_t stride = (np + 2) * 2;
    const uint64_t n_accel = p->param_counts[L][np - 2];
    const uint64_t n_freq = p->param_counts[L][np - 1];
    const double a_min = p->limits[2 * (np - 2)], a_max = p->limits[2 * (np - 2) + 1];
    const double f_min = p->limits[2 * (np - 1)], f_max = p->limits[2 * (np - 1) + 1];
    const double t0_add = co[0], t0_cur = co[2], scale_cur = co[3], t0_init = co[4];
    const double dt_add = t0_add - t0_cur;
    const double dt_init = t0_init - t0_cur;
    const double inv_ts = 1.0 / scale_cur;
    const double inv_ts2 = inv_ts * inv_ts;
    if (np == 2) {
        const double dt = dt_add - dt_init;
        const double dt2 = ((dt_add * dt_add) - (dt_init * dt_init));
        for (uint64_t i = 0; i < n; ++i) {
            const double* lf = leaves + i * stride;
            const double alpha_2 = lf[0], alpha_1 = lf[2], f0 = lf[6];
            const double a_new = 4.0 * alpha_2 * inv_ts2;
            const double delta_v = 4.0 * alpha_2 * inv_ts2 * dt;
            const double delta_d = (alpha_1 * inv_ts * dt) + (2.0 * alpha_2 * inv_ts2 * dt2);
            const double f_new = f0 * (1.0 - (delta_v * kInvCval));
            const double delay_rel = delta_d * kInvCval;
            const uint64_t ia = lko_nearest_idx(a_new, a_min, a_max, n_accel);
            const uint64_t jf = lko_nearest_idx(f_new, f_min, f_max, n_freq);
            param_idx[i] = (ia * n_freq) + jf;
            phase_shift[i] = lko_phase_idx(dt, f0, p->nbins, delay_rel);
        }
    } else {
        const double dt2_add = dt_add * dt_add;
        const double dt2_init = dt_init * dt_init;
        const double dt = dt_add - dt_init;
        const double dt2 = dt2_add - dt2_init;
        const double dt3 = (dt2_add * dt_add) - (dt2_init * dt_init);
        const double inv_ts3 = inv_ts2 * inv_ts;
        for (uint64_t i = 0; i < n; ++i) {
            const double* lf = leaves + i * stride;
            const double alpha_3 = lf[0], alpha_2 = lf[2], alpha_1 = lf[4], f0 = lf[8];
            const double a_new = (4.0 * alpha_2 * inv_ts2) + (24.0 * alpha_3 * dt_add * inv_ts3);
            const double delta_v =
                ((4.0 * alpha_2 * inv_ts2) * dt) + ((12.0 * alpha_3 * inv_ts3) * dt2);
            const double delta_d = ((alpha_1 - (3.0 * alpha_3)) * inv_ts * dt) +
                                   ((2.0 * alpha_2 * inv_ts2) * dt2) +
                                   ((4.0 * alpha_3 * inv_ts3) * dt3);
            const double f_new = f0 * (1.0 - (delta_v * kInvCval));
            const double delay_rel = delta_d * kInvCval;
            phase_shift[i] = lko_phase_idx(dt, f0, p->nbins, delay_rel);
            const uint64_t ia = lko_nearest_idx(a_new, a_min, a_max, n_accel);
            const uint64_t jf = lko_nearest_idx(f_new, f_min, f_max, n_freq);
            param_idx[i] = (ia * n_freq) + jf;
        }
    }
}

/* kernels::shift_add_linear_batch + shift_add_linear_with_buffer
 * (lib/kernels.cpp:118-146,1328-1355): tree fold unshifted, FFA fold rotated
 * right by round(shift). The tree index is formed in 32 bits as there. */
void lko_shift_add_batch(const float* folds_tree, const uint64_t* indices_tree,
                         const float* folds_ffa, const uint64_t* indices_ffa,
                         const float* phase_shift, float* folds_out, uint64_t nbins,
                         uint64_t n_leaves, uint64_t physical_start_idx, uint64_t capacity) {
    const uint64_t fs = 2 * nbins;
    for (uint64_t i = 0; i < n_leaves; ++i) {
        const uint32_t logical = (uint32_t)(indices_tree[i] + physical_start_idx);
        const uint32_t phys = logical < capacity ? logical : (uint32_t)(logical - capacity);
        const float* tail = folds_tree + (uint64_t)phys * fs;
        const float* head = folds_ffa + indices_ffa[i] * fs;
        float* o = folds_out + i * fs;
        const uint64_t s = shift_bins(phase_shift[i], nbins);
        for (uint64_t r = 0; r < 2; ++r) {
            for (uint64_t j = 0; j < nbins; ++j) {
                const uint64_t src = (j + nbins - s) % nbins;
                o[r * nbins + j] = tail[r * nbins + j] + head[r * nbins + src];
            }
        }
    }
}

uint64_t lko_score_filter(const float* folds, uint64_t n, uint64_t nbins, const uint64_t* widths,
                          uint64_t nwidths, float threshold, float* scores, uint64_t* indices) {
    snr_boxcar(1, 1, folds, n, nbins, widths, nwidths, 1.0F, scores);
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (scores[i] >= threshold) {
            indices[k++] = i;
        }
    }
    return k;
}

/* ---- WorldTree (lib/world_tree.cpp) ----------------------------------------- */

typedef struct wtree {
    uint64_t cap, ls, fs, max_batch;
    double* leaves;
    float* folds;
    float* scores;
    float* scratch;    /* cap + max_batch */
    uint64_t* pending; /* max_batch */
    uint64_t head, size, size_old, write_head, write_start, read_consumed;
    int updating;
} wtree;

static uint64_t wt_circ(uint64_t logical, uint64_t start, uint64_t cap) {
    return (start + logical) % cap;
}

static uint64_t wt_space_left(const wtree* t) {
    const int64_t remaining_old = (int64_t)t->size_old - (int64_t)t->read_consumed;
    const int64_t space = (int64_t)t->cap - (remaining_old + (int64_t)t->size);
    return space < 0 ? 0 : (uint64_t)space;
}

static uint64_t wt_start(const wtree* t) { return t->updating ? t->write_start : t->head; }

/* prepare_in_place_update / finalize_in_place_update / consume_read
 * (lib/world_tree.cpp:237-274). */
static void wt_prepare(wtree* t) {
    t->size_old = t->size;
    t->write_start = wt_circ(t->size, t->head, t->cap);
    t->write_head = t->write_start;
    t->size = 0;
    t->updating = 1;
    t->read_consumed = 0;
}

static void wt_finalize(wtree* t) {
    t->head = t->write_start;
    t->size_old = 0;
    t->updating = 0;
    t->read_consumed = 0;
    t->write_head = 0;
    t->write_start = 0;
}

/* scatter_to_circular_copy (lib/world_tree.cpp:503-525). */
static void wt_scatter(wtree* t, const double* lv, const float* fo, const float* sc,
                       const uint64_t* idx, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t s = idx[i], d = t->write_head;
        memcpy(t->leaves + d * t->ls, lv + s * t->ls, t->ls * sizeof(double));
        memcpy(t->folds + d * t->fs, fo + s * t->fs, t->fs * sizeof(float));
        t->scores[d] = sc[s];
        if (++t->write_head == t->cap) {
            t->write_head = 0;
        }
    }
    t->size += n;
}

static int cmp_desc(const void* a, const void* b) {
    const float x = *(const float*)a, y = *(const float*)b;
    return (x < y) - (x > y);
}

/* get_prune_threshold (lib/world_tree.cpp:570-618). With D the candidates
 * sorted in descending order, N of them and K = size + space_left: the
 * top-k value is D[K-1]; the second nth_element runs on the top K (or the
 * remaining N-K) in ascending order, which selects D[K-1-N/2] when
 * N/2 <= K-1 and D[N-1-N/2+K] otherwise. */
static float wt_prune_threshold(wtree* t, const float* sc, const uint64_t* idx, uint64_t n,
                                float cur) {
    if (n == 0) {
        return cur;
    }
    const uint64_t space = wt_space_left(t);
    const uint64_t N = t->size + n;
    const uint64_t K = t->size + space;
    if (N <= K) {
        return cur;
    }
    const uint64_t start = wt_start(t);
    for (uint64_t i = 0; i < t->size; ++i) {
        t->scratch[i] = t->scores[wt_circ(i, start, t->cap)];
    }
    for (uint64_t i = 0; i < n; ++i) {
        t->scratch[t->size + i] = sc[idx[i]];
    }
    qsort(t->scratch, N, sizeof(float), cmp_desc);
    const float topk = nextafterf(t->scratch[K - 1], FLT_MAX);
    const uint64_t m = N / 2;
    const float medv = (m <= K - 1) ? t->scratch[K - 1 - m] : t->scratch[N - 1 - m + K];
    const float med = nextafterf(medv, FLT_MAX);
    float eff = cur;
    eff = (eff < topk) ? topk : eff;
    eff = (eff < med) ? med : eff;
    return eff;
}

/* prune_on_overload (lib/world_tree.cpp:620-669): keep score > threshold. */
static void wt_prune_on_overload(wtree* t, float thr) {
    if (t->size == 0) {
        return;
    }
    uint64_t r = wt_start(t), w = r, kept = 0;
    for (uint64_t i = 0; i < t->size; ++i) {
        if (t->scores[r] > thr) {
            if (r != w) {
                memcpy(t->leaves + w * t->ls, t->leaves + r * t->ls, t->ls * sizeof(double));
                memcpy(t->folds + w * t->fs, t->folds + r * t->fs, t->fs * sizeof(float));
                t->scores[w] = t->scores[r];
            }
            ++kept;
            if (++w == t->cap) {
                w = 0;
            }
        }
        if (++r == t->cap) {
            r = 0;
        }
    }
    t->size = kept;
    t->write_head = w;
}

/* add_batch_scattered (lib/world_tree.cpp:361-422). */
static float wt_add_batch(wtree* t, const double* lv, const float* fo, const float* sc,
                          const uint64_t* idx, float cur, uint64_t n) {
    if (n == 0) {
        return cur;
    }
    uint64_t space = wt_space_left(t);
    if (n <= space) {
        wt_scatter(t, lv, fo, sc, idx, n);
        return cur;
    }
    const float eff = wt_prune_threshold(t, sc, idx, n, cur);
    wt_prune_on_overload(t, eff);
    uint64_t pending = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (sc[idx[i]] >= eff) {
            t->pending[pending++] = idx[i];
        }
    }
    space = wt_space_left(t);
    const uint64_t n_add = pending < space ? pending : space;
    if (n_add == 0) {
        return eff;
    }
    wt_scatter(t, lv, fo, sc, t->pending, n_add);
    return eff;
}

/* PruneImpl::initialize + execute_iteration_batched (lib/prune.cpp:181-226,
 * 429-620) for the Taylor basis, where validate is the identity
 * (lib/dynamic.cpp:70-77). */
/* Ascend resolve for one segment (poly_taylor_ascend_resolve_{accel,jerk}_batch,
 * lib/taylor.cpp:693-813; poly_chebyshev_ascend_resolve_{accel,jerk}_batch,
 * lib/chebyshev.cpp:1181-1312): the leaf's parameters carried from coord_cur
 * to the segment's centre t0_seg, nearest final-level grid cell and phase
 * shift. */
static void ascend_resolve_one(const lko_plan* p, int basis, const double* lf, double t0_seg,
                               double t0_cur, double scale_cur, uint64_t* pidx, float* shift) {
    const uint32_t np = p->nparams;
    const uint32_t L = p->n_levels - 1;
    const uint64_t n_accel = p->param_counts[L][np - 2];
    const uint64_t n_freq = p->param_counts[L][np - 1];
    const double a_min = p->limits[2 * (np - 2)], a_max = p->limits[2 * (np - 2) + 1];
    const double f_min = p->limits[2 * (np - 1)], f_max = p->limits[2 * (np - 1) + 1];
    const double dt = t0_seg - t0_cur;
    double a_new, v_new, d_new, f0;
    if (basis == 0 && np == 2) {
        const double half_dt2 = 0.5 * (dt * dt);
        const double a_cur = lf[0], v_cur = lf[2], d_cur = lf[4];
        f0 = lf[6];
        a_new = a_cur;
        v_new = v_cur + (a_cur * dt);
        d_new = d_cur + (v_cur * dt) + (a_cur * half_dt2);
    } else if (basis == 0) {
        const double half_dt2 = 0.5 * (dt * dt);
        const double sixth_dt3 = (half_dt2 * dt) / 3.0;
        const double j_cur = lf[0], a_cur = lf[2], v_cur = lf[4], d_cur = lf[6];
        f0 = lf[8];
        a_new = a_cur + (j_cur * dt);
        v_new = v_cur + (a_cur * dt) + (j_cur * half_dt2);
        d_new = d_cur + (v_cur * dt) + (a_cur * half_dt2) + (j_cur * sixth_dt3);
    } else if (np == 2) {
        const double dt2 = dt * dt;
        const double inv_ts = 1.0 / scale_cur;
        const double inv_ts2 = inv_ts * inv_ts;
        const double alpha_2 = lf[0], alpha_1 = lf[2], alpha_0 = lf[4];
        f0 = lf[6];
        a_new = 4.0 * alpha_2 * inv_ts2;
        v_new = (alpha_1 * inv_ts) + (4.0 * alpha_2 * inv_ts2 * dt);
        d_new = (alpha_0 - alpha_2) + (alpha_1 * inv_ts * dt) + (2.0 * alpha_2 * inv_ts2 * dt2);
    } else {
        const double dt2 = dt * dt;
        const double dt3 = dt2 * dt;
        const double inv_ts = 1.0 / scale_cur;
        const double inv_ts2 = inv_ts * inv_ts;
        const double inv_ts3 = inv_ts2 * inv_ts;
        const double alpha_3 = lf[0], alpha_2 = lf[2], alpha_1 = lf[4], alpha_0 = lf[6];
        f0 = lf[8];
        a_new = (4.0 * alpha_2 * inv_ts2) + (24.0 * alpha_3 * dt * inv_ts3);
        v_new = ((alpha_1 - (3.0 * alpha_3)) * inv_ts) + (4.0 * alpha_2 * inv_ts2 * dt) +
                (12.0 * alpha_3 * inv_ts3 * dt2);
        d_new = (alpha_0 - alpha_2) + ((alpha_1 - (3.0 * alpha_3)) * dt * inv_ts) +
                (2.0 * alpha_2 * inv_ts2 * dt2) + (4.0 * alpha_3 * inv_ts3 * dt3);
    }
    const double f_new = f0 * (1.0 - (v_new * kInvCval));
    const double delay_rel = d_new * kInvCval;
    *shift = lko_phase_idx(dt, f0, p->nbins, delay_rel);
    const uint64_t ia = lko_nearest_idx(a_new, a_min, a_max, n_accel);
    const uint64_t jf = lko_nearest_idx(f_new, f_min, f_max, n_freq);
    *pidx = (ia * n_freq) + jf;
}

/* poly_taylor_report_batch (lib/taylor.cpp:1529-1564): gauge transform of
 * the leaf to the observer frame with first-order error propagation. */
static void taylor_report_one(double* lf, uint32_t np) {
    const double v_final = lf[(np - 1) * 2 + 0];
    const double dv_final = lf[(np - 1) * 2 + 1];
    const double f0_batch = lf[(np + 1) * 2 + 0];
    const double s_factor = 1.0 - (v_final * kInvCval);
    for (uint32_t j = 0; j + 1 < np; ++j) {
        const double val = lf[j * 2 + 0];
        const double err = lf[j * 2 + 1];
        lf[j * 2 + 0] = val / s_factor;
        lf[j * 2 + 1] = sqrt(((err / s_factor) * (err / s_factor)) +
                             ((val * kInvCval / (s_factor * s_factor)) *
                              (val * kInvCval / (s_factor * s_factor)) * (dv_final * dv_final)));
    }
    lf[(np - 1) * 2 + 0] = f0_batch * s_factor;
    lf[(np - 1) * 2 + 1] = f0_batch * dv_final * kInvCval;
}

int lko_prune_finalize(const lko_plan* p, int basis, const float* ffa_fold, uint64_t ref_seg,
                       uint64_t prune_level, double* leaves, float* folds, float* scores,
                       float* scores_ep, uint64_t n) {
    const uint32_t np = p->nparams;
    if (np < 2 || np > 3) {
        return fail("pruning supports nparams 2 or 3");
    }
    const uint32_t L = p->n_levels - 1;
    const uint64_t nseg = p->nsegments[L];
    const double tseg = p->tsegments[L];
    const uint64_t nbins = p->nbins;
    const uint64_t ncoords = p->ncoords[L];
    const uint64_t ls = (np + 2) * 2, fs = 2 * nbins;
    if (ref_seg >= nseg || prune_level >= nseg) {
        return fail("MiddleOutScheme: invalid ref_idx / level");
    }
    uint64_t* order = (uint64_t*)malloc(sizeof(uint64_t) * nseg);
    middle_out_order(nseg, ref_seg, order);
    double t0_mid, s_mid;
    mo_coord(order, prune_level, tseg, &t0_mid, &s_mid);
    for (uint64_t i = 0; i < n; ++i) {
        double* lf = leaves + i * ls;
        float* out = folds + i * fs;
        /* shift_add_ascend_linear_batch (lib/kernels.cpp:1390-1416): zero,
         * then every segment so far, in middle-out order, rotated right by
         * round(shift) and added (shift_add_linear_with_buffer_inplace,
         * lib/kernels.cpp:149-176). */
        for (uint64_t j = 0; j < fs; ++j) {
            out[j] = 0.0F;
        }
        for (uint64_t k = 0; k <= prune_level; ++k) {
            double t_seg, s_seg;
            mo_segment_coord(order, k, tseg, &t_seg, &s_seg);
            uint64_t pidx;
            float ph;
            ascend_resolve_one(p, basis, lf, t_seg, t0_mid, s_mid, &pidx, &ph);
            uint64_t sh = (uint64_t)(ph + 0.5F);
            if (sh == nbins) {
                sh = 0;
            }
            const float* src = ffa_fold + (order[k] * ncoords + pidx) * fs;
            for (uint64_t j = 0; j < nbins; ++j) {
                const uint64_t jj = (j + nbins - sh) % nbins;
                out[j] += src[jj];
                out[nbins + j] += src[nbins + jj];
            }
        }
        scores_ep[i] = scores[i];
    }
    lko_snr_boxcar_3d_max(folds, n, nbins, p->widths, p->n_widths, scores);
    /* report: Chebyshev leaves to Taylor at coord_mid first
     * (PrunePolyChebyshevDPFuncts::report, lib/dynamic.cpp:510-519). */
    if (basis == 1) {
        lko_cheby_to_taylor(leaves, n, np, s_mid);
    }
    for (uint64_t i = 0; i < n; ++i) {
        taylor_report_one(leaves + i * ls, np);
    }
    free(order);
    return 0;
}

int lko_prune_run(const lko_plan* p, int conservative, const float* ffa_fold,
                  const float* thresholds, uint64_t n_thresholds, uint64_t ref_seg,
                  uint64_t max_sugg, uint64_t batch_size, uint64_t branch_max, uint64_t n_iters,
                  lko_prune_stats* stats, uint64_t* n_stats, double* leaves_out,
                  float* folds_out, float* scores_out, uint64_t cap_out, uint64_t* n_out) {
    return lko_prune_run_basis(p, 0, conservative, ffa_fold, thresholds, n_thresholds, ref_seg,
                               max_sugg, batch_size, branch_max, n_iters, stats, n_stats,
                               leaves_out, folds_out, scores_out, cap_out, n_out);
}

/* basis 0: Taylor (lib/dynamic.cpp:155-310); basis 1: Chebyshev
 * (BaseChebyshevPruneDPFuncts / PrunePolyChebyshevDPFuncts,
 * lib/dynamic.cpp:203-240,381-450): seeds converted to the Chebyshev basis,
 * the branch transforms the parents from coord_prev to coord_cur, and the
 * conservative tile is rejected. */
int lko_prune_run_basis(const lko_plan* p, int basis, int conservative, const float* ffa_fold,
                        const float* thresholds, uint64_t n_thresholds, uint64_t ref_seg,
                        uint64_t max_sugg, uint64_t batch_size, uint64_t branch_max,
                        uint64_t n_iters, lko_prune_stats* stats, uint64_t* n_stats,
                        double* leaves_out, float* folds_out, float* scores_out, uint64_t cap_out,
                        uint64_t* n_out) {
    const uint32_t np = p->nparams;
    if (np < 2 || np > 3) {
        return fail("pruning supports nparams 2 or 3");
    }
    if (basis == 1 && conservative) {
        return fail("Conservative tile not implemented for Chebyshev basis");
    }
    const uint32_t L = p->n_levels - 1;
    const uint64_t nseg = p->nsegments[L];
    const double tseg = p->tsegments[L];
    const uint64_t nbins = p->nbins;
    const uint64_t ncoords = p->ncoords[L];
    const uint64_t ls = (np + 2) * 2, fs = 2 * nbins;
    const uint64_t max_branched = batch_size * branch_max;
    if (ref_seg >= nseg) {
        return fail("ref_idx must be less than nsegments.");
    }
    if (ncoords > max_sugg) {
        return fail("WorldTree: Suggestions too large to add.");
    }
    wtree t;
    memset(&t, 0, sizeof(t));
    t.cap = max_sugg;
    t.ls = ls;
    t.fs = fs;
    t.max_batch = max_branched;
    t.leaves = (double*)calloc(max_sugg * ls, sizeof(double));
    t.folds = (float*)calloc(max_sugg * fs, sizeof(float));
    t.scores = (float*)calloc(max_sugg, sizeof(float));
    t.scratch = (float*)calloc(max_sugg + max_branched, sizeof(float));
    t.pending = (uint64_t*)calloc(max_branched, sizeof(uint64_t));
    uint64_t* order = (uint64_t*)malloc(sizeof(uint64_t) * nseg);
    double* b_leaves = (double*)malloc(sizeof(double) * max_branched * ls);
    uint64_t* b_org = (uint64_t*)malloc(sizeof(uint64_t) * max_branched);
    uint64_t* b_pidx = (uint64_t*)malloc(sizeof(uint64_t) * max_branched);
    float* b_shift = (float*)malloc(sizeof(float) * max_branched);
    float* b_folds = (float*)malloc(sizeof(float) * max_branched * fs);
    float* b_scores = (float*)malloc(sizeof(float) * max_branched);
    uint64_t* b_idx = (uint64_t*)malloc(sizeof(uint64_t) * max_branched);
    int rc = 0;
    middle_out_order(nseg, ref_seg, order);

    /* initialize: seed leaves, seed scores, add_initial */
    const float* seg0 = ffa_fold + order[0] * ncoords * fs;
    if (lko_taylor_seed(p, t.leaves) != ncoords) {
        rc = 1;
        goto done;
    }
    if (basis == 1) {
        double ci0, cs0;
        mo_coord(order, 0, tseg, &ci0, &cs0);
        lko_taylor_to_cheby(t.leaves, ncoords, np, cs0);
    }
    memcpy(t.folds, seg0, ncoords * fs * sizeof(float));
    lko_snr_boxcar_3d_max(seg0, ncoords, nbins, p->widths, p->n_widths, t.scores);
    t.size = ncoords;
    uint64_t ns = 0;
    {
        float mn = t.scores[0], mx = t.scores[0];
        for (uint64_t i = 1; i < ncoords; ++i) {
            mn = (t.scores[i] < mn) ? t.scores[i] : mn;
            mx = (mx < t.scores[i]) ? t.scores[i] : mx;
        }
        if (ncoords == 0) {
            mn = mx = 0.0F;
        }
        lko_prune_stats s0 = {0, order[0], ncoords, ncoords, ncoords, ncoords, 0.0F, mn, mx, 0};
        stats[ns++] = s0;
    }

    const uint64_t levels = (nseg - 1) < n_iters ? (nseg - 1) : n_iters;
    for (uint64_t level = 1; level <= levels; ++level) {
        if (level > n_thresholds) {
            rc = fail("Pruning complete - exceeded threshold scheme length");
            goto done;
        }
        wt_prepare(&t);
        const uint64_t seg_idx = order[level];
        const float threshold = thresholds[level - 1];
        const uint64_t n_branches = t.size_old;
        uint64_t n_leaves = 0, n_phy = 0;
        float smin = FLT_MAX, smax = -FLT_MAX;
        double ci[2], cn[2], cc[2], ca[2], cp[2];
        mo_coord(order, 0, tseg, &ci[0], &ci[1]);
        mo_coord(order, level - 1, tseg, &cp[0], &cp[1]);
        mo_coord(order, level, tseg, &cn[0], &cn[1]);
        mo_current_coord(order, level, tseg, &cc[0], &cc[1]);
        mo_segment_coord(order, level, tseg, &ca[0], &ca[1]);
        const double coords[6] = {ca[0], ca[1], cc[0], cc[1], ci[0], ci[1]};
        const float* seg = ffa_fold + seg_idx * ncoords * fs;
        float cur_thr = threshold;
        uint64_t bsize = batch_size < n_branches ? batch_size : n_branches;
        bsize = bsize < 1 ? 1 : bsize;
        uint64_t processed = 0;
        while (processed < n_branches) {
            const uint64_t remaining = n_branches - processed;
            const uint64_t want = bsize < remaining ? bsize : remaining;
            /* get_leaves_span (lib/world_tree.cpp:148-163) */
            const uint64_t pstart = wt_circ(t.read_consumed, t.head, t.cap);
            const uint64_t nb = want < (t.cap - pstart) ? want : (t.cap - pstart);
            if (nb == 0) {
                rc = fail("Loaded batch size is 0");
                goto done;
            }
            processed += nb;
            uint64_t nl = 0;
            const int brc =
                basis == 1 ? lko_cheby_branch(t.leaves + pstart * ls, nb, np, cc[0], cc[1], cp[0],
                                              cp[1], nbins, p->eta, branch_max, b_leaves, b_org,
                                              max_branched, &nl)
                           : lko_taylor_branch(t.leaves + pstart * ls, nb, np, cc[0], cc[1],
                                               nbins, p->eta, branch_max, b_leaves, b_org,
                                               max_branched, &nl);
            if (brc == 2) {
                rc = fail("Branch factor exceeded workspace size:n_leaves_batch <= "
                          "max_branched_leaves");
                goto done;
            }
            if (brc != 0) {
                rc = 1;
                goto done;
            }
            n_leaves += nl;
            n_phy += nl;
            if (nl == 0) {
                t.read_consumed += nb;
                continue;
            }
            if (basis == 1) {
                lko_cheby_resolve(p, b_leaves, nl, coords, b_pidx, b_shift);
            } else {
                lko_taylor_resolve(p, b_leaves, nl, coords, b_pidx, b_shift);
            }
            lko_shift_add_batch(t.folds, b_org, seg, b_pidx, b_shift, b_folds, nbins, nl, pstart,
                                t.cap);
            const uint64_t npass =
                lko_score_filter(b_folds, nl, nbins, p->widths, p->n_widths, cur_thr, b_scores, b_idx);
            for (uint64_t i = 0; i < nl; ++i) {
                smin = (b_scores[i] < smin) ? b_scores[i] : smin;
                smax = (smax < b_scores[i]) ? b_scores[i] : smax;
            }
            if (npass == 0) {
                t.read_consumed += nb;
                continue;
            }
            if (basis == 1) {
                lko_cheby_transform(b_leaves, b_idx, npass, np, cn[0], cn[1], cc[0], cc[1]);
            } else {
                lko_taylor_transform(b_leaves, b_idx, npass, np, cn[0], cc[0], conservative);
            }
            cur_thr = wt_add_batch(&t, b_leaves, b_folds, b_scores, b_idx, cur_thr, npass);
            t.read_consumed += nb;
        }
        wt_finalize(&t);
        lko_prune_stats sl = {level, seg_idx, n_branches, n_leaves, n_phy, t.size,
                              threshold, smin, smax, 0};
        stats[ns++] = sl;
        if (t.size == 0) {
            break;
        }
    }
    *n_stats = ns;
    *n_out = t.size;
    if (t.size <= cap_out) {
        for (uint64_t i = 0; i < t.size; ++i) {
            const uint64_t ph = wt_circ(i, t.head, t.cap);
            memcpy(leaves_out + i * ls, t.leaves + ph * ls, ls * sizeof(double));
            memcpy(folds_out + i * fs, t.folds + ph * fs, fs * sizeof(float));
            scores_out[i] = t.scores[ph];
        }
    }
done:
    free(t.leaves);
    free(t.folds);
    free(t.scores);
    free(t.scratch);
    free(t.pending);
    free(order);
    free(b_leaves);
    free(b_org);
    free(b_pidx);
    free(b_shift);
    free(b_folds);
    free(b_scores);
    free(b_idx);
    return rc;
}

/* ======================================================================== */
/* Monte-Carlo threshold stage.                                              */
/* ======================================================================== */

/* detection::snr_boxcar_threshold_with_cache (lib/score.cpp:434-462): the
 * largest boxcar S/N of one 2-D profile, each width's S/N divided by
 * stdnoise; the reference returns (any S/N > threshold), which equals
 * (this maximum > threshold). */
float lko_snr_max_div(const float* prof, uint64_t nbins, const uint64_t* widths, uint64_t nw,
                      float stdnoise) {
    uint64_t wmax = 0;
    for (uint64_t i = 0; i < nw; ++i) {
        wmax = widths[i] > wmax ? widths[i] : wmax;
    }
    float* psum = (float*)malloc(sizeof(float) * (nbins + wmax));
    lko_circular_prefix_sum(prof, psum, nbins, nbins + wmax);
    const float sum = psum[nbins - 1];
    float best = -FLT_MAX;
    for (uint64_t iw = 0; iw < nw; ++iw) {
        const uint64_t w = widths[iw];
        const float h = sqrtf((float)(nbins - w) / (float)(nbins * w));
        const float b = (float)w * h / (float)(nbins - w);
        const float dmax = diff_max(psum + w, psum, nbins);
        const float snr = (((h + b) * dmax) - (b * sum)) / stdnoise;
        best = (best < snr) ? snr : best;
    }
    free(psum);
    return best;
}

/* simulate_score_prune_fused (lib/thresholds.cpp:358-431): out_i =
 * (in[src_i] + noise_i) + signal, stdnoise = sqrt(var_in + var_add), keep
 * trials whose S/N exceeds the threshold, compacted in trial order.
 * src == NULL: src_i = i (the reference draws src_i at random only for
 * i >= ntrials_in). Noise row of trial i: rowmap[i] (NULL: i); signal:
 * [nbins] shared, or per trial (row rowmap[i]) when signal_per_trial, times
 * signal_scale (a power of two keeps it exact). ids_out receives the noise
 * row of each kept trial. With cls (a flag per noise row), counts[n_thr + k]
 * counts the flagged trials above thr[k].
 * counts[k] (n_thr entries, may be NULL) = trials with maximum S/N > thr[k].
 * Returns the number kept. */
uint64_t lko_mc_stage(const float* folds_in, const uint32_t* src, uint64_t ntrials,
                      uint64_t nbins, const float* noise, const float* signal,
                      int signal_per_trial, float signal_scale, const uint32_t* rowmap,
                      float var_in, float var_add, const uint64_t* widths, uint64_t nw,
                      float threshold, const float* thr, uint64_t n_thr, const uint8_t* cls,
                      float* folds_out, uint32_t* ids_out, uint64_t* counts, float* max_snr) {
    const float stdnoise = sqrtf(var_in + var_add);
    float* row = (float*)malloc(sizeof(float) * nbins);
    for (uint64_t k = 0; k < (cls != NULL ? 2 : 1) * n_thr; ++k) {
        counts[k] = 0;
    }
    uint64_t kept = 0;
    for (uint64_t i = 0; i < ntrials; ++i) {
        const uint64_t s = src != NULL ? src[i] : i;
        const uint64_t rw = rowmap != NULL ? rowmap[i] : i;
        const float* in = folds_in + s * nbins;
        const float* nz = noise + rw * nbins;
        const float* sg = signal + (signal_per_trial ? rw * nbins : 0);
        for (uint64_t j = 0; j < nbins; ++j) {
            row[j] = (in[j] + nz[j]) + (sg[j] * signal_scale);
        }
        const float m = lko_snr_max_div(row, nbins, widths, nw, stdnoise);
        if (max_snr != NULL) {
            max_snr[i] = m;
        }
        for (uint64_t k = 0; k < n_thr; ++k) {
            counts[k] += (m > thr[k]) ? 1 : 0;
            if (cls != NULL && cls[rw] != 0) {
                counts[n_thr + k] += (m > thr[k]) ? 1 : 0;
            }
        }
        if (m > threshold) {
            memcpy(folds_out + kept * nbins, row, nbins * sizeof(float));
            if (ids_out != NULL) {
                ids_out[kept] = (uint32_t)rw;
            }
            ++kept;
        }
    }
    free(row);
    return kept;
}

/* ======================================================================== */
/* DynamicThresholdScheme beam search (lib/thresholds.cpp:560-907): host     */
/* set-up (lib/scheme.cpp, lib/simulation.cpp:12-50, lib/utils.cpp:138-185), */
/* State::gen_next (include/loki/detection/thresholds.hpp:32-58) and the      */
/* stage loop, sequential in the reference's order. The noise is the          */
/* reference's table method (lib/loki/math.hpp:363-390: a 32-bit uniform     */
/* through a 2^17 + 1 entry normal quantile table, fmaf interpolation) and    */
/* its Lemire resampling (math.hpp:267-285), fed by Philox4x32-10 words of    */
/* the counter (trial, bin / 4, transition * 2 + hypothesis, stage + 1) --    */
/* the reference's thread-local PCG32 streams seeded from random_device       */
/* cannot be reproduced.                                                      */
/* ======================================================================== */

#define LKO_DTS_LUT ((1u << 17) + 1u)

/* Acklam's inverse normal CDF (2003) with one Halley step on erfc. */
double lko_normal_quantile(double p) {
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02,
                                -2.759285104469687e+02, 1.383577518672690e+02,
                                -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02,
                                -1.556989798598866e+02, 6.680131188771972e+01,
                                -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01,
                                -2.400758277161838e+00, -2.549732539343734e+00,
                                4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01,
                                2.445134137142996e+00, 3.754408661907416e+00};
    const double p_low = 0.02425;
    double x;
    if (p < p_low) {
        const double q = sqrt(-2.0 * log(p));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else if (p <= 1.0 - p_low) {
        const double q = p - 0.5;
        const double r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    } else {
        const double q = sqrt(-2.0 * log(1.0 - p));
        x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    const double e = 0.5 * erfc(-x / sqrt(2.0)) - p;
    const double u = e * sqrt(2.0 * 3.14159265358979323846) * exp(x * x / 2.0);
    return x - u / (1.0 + x * u / 2.0);
}

/* ThreadLocalNormalRNG::init_lut (lib/loki/math.hpp:304-312). */
void lko_dts_normal_lut(float* out) {
    const double n = (double)(LKO_DTS_LUT - 1);
    for (uint32_t i = 0; i < LKO_DTS_LUT; ++i) {
        double p = (double)i / n;
        p = p < 1e-9 ? 1e-9 : (p > 1.0 - 1e-9 ? 1.0 - 1e-9 : p);
        out[i] = (float)lko_normal_quantile(p);
    }
}

/* detail::compute_thresholds (lib/scheme.cpp:16-25). */
void lko_dts_thresholds(float snr_start, float snr_final, uint32_t n, float* out) {
    const float step = (snr_final - snr_start) / (float)(n - 1);
    for (uint32_t i = 0; i < n; ++i) {
        out[i] = ((float)i * step) + snr_start;
    }
}

/* detail::compute_probs (lib/scheme.cpp:27-40). */
void lko_dts_probs(uint32_t n, float prob_min, float* out) {
    const float lpm = log10f(prob_min);
    const float step = (0.0F - lpm) / (float)(n - 1);
    for (uint32_t i = 0; i < n; ++i) {
        out[i] = powf(10.0F, lpm + (step * (float)i));
    }
}

/* simulation::generate_folded_profile (lib/simulation.cpp:12-50). */
void lko_dts_profile(uint32_t nbins, float ducy, float center, float* out) {
    const float step = 1.0F / (float)nbins;
    const float ln10 = 2.302585092994045684017991454684364208F;
    const float sigma = ducy / (2.0F * sqrtf(2.0F * ln10));
    float mx = -FLT_MAX;
    for (uint32_t i = 0; i < nbins; ++i) {
        const float p = (float)i * step;
        const float w = fmodf(p - center + 0.5F, 1.0F) - 0.5F;
        out[i] = expf(-(w * w) / (2.0F * sigma * sigma));
        mx = out[i] > mx ? out[i] : mx;
    }
    float ss = 0.0F;
    for (uint32_t i = 0; i < nbins; ++i) {
        out[i] = out[i] / mx;
    }
    for (uint32_t i = 0; i < nbins; ++i) {
        ss = ss + out[i] * out[i];
    }
    const float norm = sqrtf(ss);
    for (uint32_t i = 0; i < nbins; ++i) {
        out[i] = out[i] / norm;
    }
}

/* detail::guess_scheme = min(bound_scheme, trials_scheme) (lib/scheme.cpp:56-96),
 * norm_isf(p) = -quantile(p). */
void lko_dts_guess(uint32_t nstages, float snr_bound, const float* branching, uint32_t trials_start,
                   float min_trials, float* out) {
    const uint32_t nseg = nstages + 1;
    float l2 = log2f((float)trials_start);
    for (uint32_t i = 0; i < nstages; ++i) {
        const float bound = sqrtf((float)(i + 2) * snr_bound * snr_bound / (float)nseg);
        l2 += log2f(branching[i]);
        const float trials = exp2f(l2);
        const float eff = trials > min_trials ? trials : min_trials;
        const float thr = (float)(-lko_normal_quantile((double)(1 / eff)));
        out[i] = bound < thr ? bound : thr;
    }
}

/* utils::find_neighbouring_indices (lib/utils.cpp:138-163). */
uint32_t lko_dts_neighbours(const uint32_t* idx, uint32_t n, uint32_t target, uint32_t num,
                            uint32_t* out) {
    uint32_t pos = 0;
    while (pos < n && idx[pos] < target) {
        ++pos;
    }
    const uint32_t half = num / 2;
    uint32_t left = pos > half ? pos - half : 0;
    const uint32_t right = (left + num < n) ? left + num : n;
    if (right - left < num && right == n) {
        left = right > num ? right - num : 0;
    }
    for (uint32_t k = left; k < right; ++k) {
        out[k - left] = idx[k];
    }
    return right - left;
}

/* utils::find_lower_bin_index (lib/utils.cpp:181-185). */
int64_t lko_dts_lower_bin(const float* range, uint32_t n, float v) {
    uint32_t k = 0;
    while (k < n && !(v < range[k])) {
        ++k;
    }
    return (int64_t)k - 1;
}

static lko_dts_state dts_empty(void) {
    lko_dts_state s;
    memset(&s, 0, sizeof(s));
    s.complexity_cumul = FLT_MAX;
    s.threshold = -1.0F;
    s.cost = FLT_MAX;
    s.threshold_prev = -1.0F;
    s.is_empty = 1;
    return s;
}

/* State::gen_next (include/loki/detection/thresholds.hpp:32-58). */
lko_dts_state lko_dts_gen_next(const lko_dts_state* s, float threshold, float s0, float s1,
                               float nbranches) {
    const float nleaves_next = s->complexity * nbranches;
    const float nleaves_surv = nleaves_next * s0;
    const float cc = s->complexity_cumul + nleaves_next;
    const float h1 = s->success_h1_cumul * s1;
    lko_dts_state n = dts_empty();
    n.success_h0 = s0;
    n.success_h1 = s1;
    n.complexity = nleaves_surv;
    n.complexity_cumul = cc;
    n.success_h1_cumul = h1;
    n.nbranches = nbranches;
    n.threshold = threshold;
    n.cost = cc / h1;
    n.is_empty = 0;
    n.threshold_prev = s->threshold;
    n.success_h1_cumul_prev = s->success_h1_cumul;
    return n;
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011). */
void lko_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* ThreadLocalNormalRNG::generate_impl for one uniform word, mean 0, stddev 1. */
float lko_dts_normal(uint32_t r, const float* lut) {
    const float inv_u32 = 1.0F / 4294967296.0F;
    const float max_idx = (float)(LKO_DTS_LUT - 2);
    const float u = ((float)r * inv_u32) * max_idx;
    const uint32_t idx = (uint32_t)u;
    const float frac = u - (float)idx;
    const float z = fmaf(frac, lut[idx + 1] - lut[idx], lut[idx]);
    return fmaf(z, 1.0F, 0.0F);
}

/* uniform_index(range - 1): Lemire's bounded draw with rejection on the words
 * of counters (i, 0xffffffff - call, tid2, stage_code). */
uint32_t lko_dts_resample(uint32_t range, uint32_t i, uint32_t tid2, uint32_t stage_code, uint32_t k0,
                          uint32_t k1) {
    const uint64_t t = (1ull << 32) % range;
    uint64_t m = 0;
    for (uint32_t call = 0; call < 2; ++call) {
        const uint32_t ctr[4] = {i, 0xFFFFFFFFu - call, tid2, stage_code};
        uint32_t w[4];
        lko_philox4x32_10(ctr, k0, k1, w);
        for (int q = 0; q < 4; ++q) {
            m = (uint64_t)w[q] * range;
            if ((uint32_t)m >= range || (uint32_t)m >= t) {
                return (uint32_t)(m >> 32);
            }
        }
    }
    return (uint32_t)(m >> 32);
}

/* Trial fold i of one (transition, hypothesis): (in[src] + noise) + prof. */
static void dts_fold(const float* in, uint32_t n_in, const float* prof, uint32_t nbins, uint32_t i,
                     uint32_t tid2, uint32_t stage_code, uint32_t k0, uint32_t k1, const float* lut,
                     float* out) {
    const uint32_t src = i < n_in ? i : lko_dts_resample(n_in, i, tid2, stage_code, k0, k1);
    const float* ir = in + (uint64_t)src * nbins;
    for (uint32_t q = 0; q * 4 < nbins; ++q) {
        const uint32_t ctr[4] = {i, q, tid2, stage_code};
        uint32_t w[4];
        lko_philox4x32_10(ctr, k0, k1, w);
        for (uint32_t k = 0; k < 4 && 4 * q + k < nbins; ++k) {
            const uint32_t j = 4 * q + k;
            out[j] = (ir[j] + lko_dts_normal(w[k], lut)) + prof[j];
        }
    }
}

/* simulate_score_prune_fused on one hypothesis: survivors in trial order. */
static uint32_t dts_sim(const float* in, uint32_t n_in, const float* prof, const lko_dts_config* c,
                        uint32_t tid2, uint32_t stage_code, float thr, float stdnoise, const uint64_t* w,
                        uint64_t nw, const float* lut, float* out) {
    uint32_t n = 0;
    const uint32_t k0 = (uint32_t)c->seed, k1 = (uint32_t)(c->seed >> 32);
    for (uint32_t i = 0; i < c->ntrials; ++i) {
        float* row = out + (uint64_t)n * c->nbins;
        dts_fold(in, n_in, prof, c->nbins, i, tid2, stage_code, k0, k1, lut, row);
        if (lko_snr_max_div(row, c->nbins, w, nw, stdnoise) > thr) {
            ++n;
        }
    }
    return n;
}

int lko_dts_run(const lko_dts_config* c, uint32_t thres_neigh, uint32_t stages_run, lko_dts_state* states) {
    const uint32_t S = c->nstages, NT = c->nthresholds, NP = c->nprobs, NB = c->nbins, NTR = c->ntrials;
    const uint64_t ncell = (uint64_t)NT * NP;
    const uint64_t fold_f = (uint64_t)NTR * NB;
    float* lut = (float*)malloc(sizeof(float) * LKO_DTS_LUT);
    float* prof = (float*)malloc(sizeof(float) * 2 * NB);
    float* thr = (float*)malloc(sizeof(float) * NT);
    float* probs = (float*)malloc(sizeof(float) * NP);
    float* guess = (float*)malloc(sizeof(float) * S);
    float* pool[2] = {(float*)malloc(sizeof(float) * ncell * 2 * fold_f),
                      (float*)malloc(sizeof(float) * ncell * 2 * fold_f)};
    uint32_t* cnt[2] = {(uint32_t*)calloc(ncell * 2, sizeof(uint32_t)),
                        (uint32_t*)calloc(ncell * 2, sizeof(uint32_t))};
    float* init = (float*)malloc(sizeof(float) * 2 * fold_f);
    float* tmp[2] = {(float*)malloc(sizeof(float) * fold_f), (float*)malloc(sizeof(float) * fold_f)};
    uint32_t* beam_prev = (uint32_t*)malloc(sizeof(uint32_t) * NT);
    uint32_t* beam_cur = (uint32_t*)malloc(sizeof(uint32_t) * NT);
    uint32_t* neigh = (uint32_t*)malloc(sizeof(uint32_t) * (thres_neigh + 1));
    uint64_t w[LKO_MAX_WIDTHS];
    int rc = 0;
    if (!lut || !prof || !thr || !probs || !guess || !pool[0] || !pool[1] || !cnt[0] || !cnt[1] ||
        !init || !tmp[0] || !tmp[1] || !beam_prev || !beam_cur || !neigh) {
        rc = fail("out of memory");
        goto done;
    }
    {
        const uint32_t k0 = (uint32_t)c->seed, k1 = (uint32_t)(c->seed >> 32);
        const uint64_t nw = lko_box_widths(NB, c->ducy_max, c->wtsp, w, LKO_MAX_WIDTHS);
        float* p1 = (float*)malloc(sizeof(float) * NB);
        lko_dts_normal_lut(lut);
        lko_dts_profile(NB, c->ref_ducy, 0.5F, p1);
        const float bias = c->snr_final / (float)sqrt((double)(S + 1));
        for (uint32_t j = 0; j < NB; ++j) {
            prof[j] = p1[j] * 0.0F;
            prof[NB + j] = p1[j] * bias;
        }
        free(p1);
        lko_dts_thresholds(0.1F, c->snr_final, NT, thr);
        lko_dts_probs(NP, c->prob_min, probs);
        lko_dts_guess(S, c->snr_final, c->branching_pattern, c->trials_start, 1E10F, guess);
        for (uint64_t k = 0; k < (uint64_t)S * ncell; ++k) {
            states[k] = dts_empty();
        }
        /* initial folds: simulate_folds from zero folds (no scoring) */
        float* zeros = (float*)calloc(fold_f, sizeof(float));
        for (uint32_t h = 0; h < 2; ++h) {
            for (uint32_t i = 0; i < NTR; ++i) {
                dts_fold(zeros, NTR, prof + h * NB, NB, i, h, 0u, k0, k1, lut,
                         init + (uint64_t)h * fold_f + (uint64_t)i * NB);
            }
        }
        free(zeros);
        const lko_dts_state initial = {0.0F, 0.0F, 1.0F, 1.0F, 1.0F, 0.0F, -1.0F, FLT_MAX, -1.0F, 0.0F, 0, {0, 0, 0}};
        float var_in = 1.0F;
        uint32_t nprev = 0;
        const uint32_t S_run = (stages_run == 0 || stages_run > S) ? S : stages_run;
        for (uint32_t st = 0; st < S_run; ++st) {
            const int cur = (int)(st % 2);
            const float var_new = var_in + 1.0F;
            const float stdnoise = sqrtf(var_new);
            /* beam of this stage (get_current_thresholds_idx) */
            uint32_t ncur = 0;
            {
                const float lo = guess[st] - c->beam_width > 0.0F ? guess[st] - c->beam_width : 0.0F;
                const float hi = guess[st] + c->beam_width < thr[NT - 1] ? guess[st] + c->beam_width : thr[NT - 1];
                for (uint32_t i = 0; i < NT; ++i) {
                    if (thr[i] >= lo && thr[i] <= hi) {
                        beam_cur[ncur++] = i;
                    }
                }
            }
            memset(cnt[cur], 0, sizeof(uint32_t) * ncell * 2);
            lko_dts_state* sc = states + (uint64_t)st * ncell;
            for (uint32_t b = 0; b < ncur; ++b) {
                const uint32_t ithres = beam_cur[b];
                const uint32_t nn = st == 0 ? 1 : lko_dts_neighbours(beam_prev, nprev, ithres, thres_neigh, neigh);
                for (uint32_t jn = 0; jn < nn; ++jn) {
                    for (uint32_t k = 0; k < (st == 0 ? 1u : NP); ++k) {
                        const lko_dts_state* ps;
                        const float* in0;
                        const float* in1;
                        uint32_t n0, n1, tid;
                        if (st == 0) {
                            ps = &initial;
                            in0 = init;
                            in1 = init + fold_f;
                            n0 = n1 = NTR;
                            tid = ithres;
                        } else {
                            const uint32_t pc = neigh[jn] * NP + k;
                            ps = states + (uint64_t)(st - 1) * ncell + pc;
                            in0 = pool[1 - cur] + (uint64_t)pc * 2 * fold_f;
                            in1 = in0 + fold_f;
                            n0 = cnt[1 - cur][2 * pc];
                            n1 = cnt[1 - cur][2 * pc + 1];
                            tid = (ithres * NT + neigh[jn]) * NP + k;
                        }
                        if (ps->is_empty || n0 == 0 || n1 == 0) {
                            continue;
                        }
                        const uint32_t m0 = dts_sim(in0, n0, prof, c, 2 * tid, st + 1, thr[ithres], stdnoise, w,
                                                    nw, lut, tmp[0]);
                        const uint32_t m1 = dts_sim(in1, n1, prof + NB, c, 2 * tid + 1, st + 1, thr[ithres],
                                                    stdnoise, w, nw, lut, tmp[1]);
                        const lko_dts_state ns = lko_dts_gen_next(ps, thr[ithres], (float)m0 / (float)NTR,
                                                                  (float)m1 / (float)NTR, c->branching_pattern[st]);
                        const int64_t ip = lko_dts_lower_bin(probs, NP, ns.success_h1_cumul);
                        if (ip < 0) {
                            continue;
                        }
                        const uint64_t cell = (uint64_t)ithres * NP + (uint64_t)ip;
                        if (sc[cell].is_empty || ns.complexity_cumul < sc[cell].complexity_cumul) {
                            sc[cell] = ns;
                            float* dst = pool[cur] + cell * 2 * fold_f;
                            memcpy(dst, tmp[0], sizeof(float) * (uint64_t)m0 * NB);
                            memcpy(dst + fold_f, tmp[1], sizeof(float) * (uint64_t)m1 * NB);
                            cnt[cur][2 * cell] = m0;
                            cnt[cur][2 * cell + 1] = m1;
                        }
                    }
                }
            }
            memcpy(beam_prev, beam_cur, sizeof(uint32_t) * ncur);
            nprev = ncur;
            var_in = var_new;
        }
    }
done:
    free(lut);
    free(prof);
    free(thr);
    free(probs);
    free(guess);
    free(pool[0]);
    free(pool[1]);
    free(cnt[0]);
    free(cnt[1]);
    free(init);
    free(tmp[0]);
    free(tmp[1]);
    free(beam_prev);
    free(beam_cur);
    free(neigh);
    return rc;
}

/* ======================================================================== */
/* Fourier-domain FFA (FFA<ComplexType>, lib/ffa.cpp:99-135,170-240), every  */
/* sum and phasor in double. Complex folds are [nseg][ncoords][2][nbins_f]   */
/* with nbins_f = nbins / 2 + 1, stored as interleaved (re, im) doubles.      */
/* ======================================================================== */

static const double kTwoPi = 6.283185307179586476925286766559;

/* exp(-2 pi i * cycles), the angle taken modulo one cycle first. */
static void unit_phasor(double cycles, double* re, double* im) {
    const double fr = cycles - floor(cycles);
    *re = cos(kTwoPi * fr);
    *im = -sin(kTwoPi * fr);
}

/* kernels::brute_fold_ts_complex (lib/kernels.cpp:1156-1242) with
 * brute_fold_segment_complex (:582-720): harmonic m of segment s at
 * frequency f is sum_k x[s * L + k] * exp(-2 pi i m f t_k) with
 * t_k = k * tsamp - t_ref (the DC term m = 0 is the plain sum). The
 * reference forms the phasor in float and raises it to the m-th power by a
 * recurrence; here the phase is reduced modulo one cycle in double and the
 * powers are taken in double. */
int lko_fourier_brute_fold(const float* ts_e, const float* ts_v, uint64_t nsamps,
                           const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                           uint64_t nbins, double tsamp, double t_ref, double* out) {
    if (segment_len == 0 || nbins < 2 || nfreqs == 0) {
        return fail("lko_fourier_brute_fold: empty segment, frequency list or nbins < 2");
    }
    const uint64_t nbf = nbins / 2 + 1;
    const uint64_t nseg = nsamps / segment_len;
#pragma omp parallel
    {
        double* acc = (double*)malloc(sizeof(double) * 4 * nbf);
#pragma omp for schedule(dynamic, 4)
        for (int64_t sf = 0; sf < (int64_t)(nseg * nfreqs); ++sf) {
            const uint64_t s = (uint64_t)sf / nfreqs, f = (uint64_t)sf % nfreqs;
            memset(acc, 0, sizeof(double) * 4 * nbf);
            const float* e = ts_e + s * segment_len;
            const float* v = ts_v + s * segment_len;
            for (uint64_t k = 0; k < segment_len; ++k) {
                const double t = (double)k * tsamp - t_ref;
                double zr, zi;
                unit_phasor(freqs[f] * t, &zr, &zi);
                const double xe = (double)e[k], xv = (double)v[k];
                double pr = 1.0, pi = 0.0;
                for (uint64_t m = 0; m < nbf; ++m) {
                    acc[4 * m + 0] += xe * pr;
                    acc[4 * m + 1] += xe * pi;
                    acc[4 * m + 2] += xv * pr;
                    acc[4 * m + 3] += xv * pi;
                    const double nr = pr * zr - pi * zi;
                    pi = pr * zi + pi * zr;
                    pr = nr;
                }
            }
            double* oe = out + (s * nfreqs + f) * 4 * nbf;
            double* ov = oe + 2 * nbf;
            for (uint64_t m = 0; m < nbf; ++m) {
                oe[2 * m] = acc[4 * m + 0];
                oe[2 * m + 1] = acc[4 * m + 1];
                ov[2 * m] = acc[4 * m + 2];
                ov[2 * m + 1] = acc[4 * m + 3];
            }
        }
        free(acc);
    }
    return 0;
}

/* kernels::ffa_complex_iter / ffa_complex_iter_freq (lib/kernels.cpp:
 * 942-1130, 1283-1326) with shift_add_complex_recurrence_binary / _linear
 * (:241-453): out[k] = tail[k] * exp(-2 pi i k shift_tail / nbins)
 * + head[k] * exp(-2 pi i k shift_head / nbins) for E and V, the shifts
 * fractional (the frequency-only table has no tail shift). */
void lko_fourier_merge(const double* in, double* out, const void* coords, int taylor,
                       uint64_t ncur, uint64_t nprev, uint64_t nseg, uint64_t nbins) {
    const uint64_t nbf = nbins / 2 + 1;
    const uint64_t fs = 4 * nbf; /* doubles per (E, V) row pair */
#pragma omp parallel for schedule(static)
    for (int64_t sc = 0; sc < (int64_t)(nseg * ncur); ++sc) {
        const uint64_t s = (uint64_t)sc / ncur, c = (uint64_t)sc % ncur;
        uint64_t it, ih;
        double st, sh;
        if (taylor) {
            const lko_coord* cc = (const lko_coord*)coords + c;
            it = cc->i_tail;
            ih = cc->i_head;
            st = (double)cc->shift_tail;
            sh = (double)cc->shift_head;
        } else {
            const lko_coord_freq* cc = (const lko_coord_freq*)coords + c;
            it = ih = cc->idx;
            st = 0.0;
            sh = (double)cc->shift;
        }
        const double* tail = in + ((2 * s) * nprev + it) * fs;
        const double* head = in + ((2 * s + 1) * nprev + ih) * fs;
        double* o = out + (s * ncur + c) * fs;
        for (uint64_t k = 0; k < nbf; ++k) {
            double tr, ti, hr, hi;
            unit_phasor((double)k * st / (double)nbins, &tr, &ti);
            unit_phasor((double)k * sh / (double)nbins, &hr, &hi);
            for (uint64_t r = 0; r < 2; ++r) {
                const double* a = tail + r * 2 * nbf + 2 * k;
                const double* b = head + r * 2 * nbf + 2 * k;
                double* d = o + r * 2 * nbf + 2 * k;
                d[0] = (a[0] * tr - a[1] * ti) + (b[0] * hr - b[1] * hi);
                d[1] = (a[0] * ti + a[1] * tr) + (b[0] * hi + b[1] * hr);
            }
        }
    }
}

/* math::irfft_batch (lib/fft.cpp:503-552): FFTW's c2r transform of size n
 * (the imaginary parts of the DC and, for even n, the Nyquist term are not
 * used) scaled by 1 / n. in [nprof][n/2 + 1] complex, out [nprof][n]. */
void lko_irfft(const double* in, double* out, uint64_t nprof, uint64_t n) {
    const uint64_t nbf = n / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)nprof; ++p) {
        const double* x = in + (uint64_t)p * 2 * nbf;
        double* y = out + (uint64_t)p * n;
        for (uint64_t j = 0; j < n; ++j) {
            double acc = x[0];
            for (uint64_t m = 1; m < nbf; ++m) {
                double c, s;
                unit_phasor((double)((m * j) % n) / (double)n, &c, &s);
                /* Re(X_m exp(+2 pi i m j / n)) = Re X c + Im X s  (s = -sin) */
                const double re = x[2 * m] * c + x[2 * m + 1] * s;
                acc += (2 * m == n) ? re : 2.0 * re;
            }
            y[j] = acc / (double)n;
        }
    }
}

/* math::rfft_batch (lib/fft.cpp:375-415): FFTW's r2c transform of size n,
 * unscaled. in [nprof][n], out [nprof][n/2 + 1] complex. */
void lko_rfft(const double* in, double* out, uint64_t nprof, uint64_t n) {
    const uint64_t nbf = n / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)nprof; ++p) {
        const double* x = in + (uint64_t)p * n;
        double* y = out + (uint64_t)p * 2 * nbf;
        for (uint64_t m = 0; m < nbf; ++m) {
            double re = 0.0, im = 0.0;
            for (uint64_t j = 0; j < n; ++j) {
                double c, s;
                unit_phasor((double)((m * j) % n) / (double)n, &c, &s);
                re += x[j] * c;
                im += x[j] * s;
            }
            y[2 * m] = re;
            y[2 * m + 1] = im;
        }
    }
}

/* FFA<ComplexType>::execute (lib/ffa.cpp:75-97, 242-310): level-0 fold by
 * the direct transform, or for nbins > nbins_min_lossy by the time-domain
 * brute fold (float sums, as lko_brute_fold) and a real transform
 * (initialize, :201-240); then every merge level up to level_out. out holds
 * the level's complex fold. */
int lko_ffa_fourier(const lko_plan* p, const float* ts_e, const float* ts_v, uint32_t level_out,
                    uint64_t nbins_min_lossy, double* fold_out) {
    if (p->n_levels < 2) {
        return fail("FFA::execute_unified: levels must be greater than or equal to 2");
    }
    if (level_out >= p->n_levels) {
        return fail("level_out out of range");
    }
    const uint32_t np = p->nparams;
    const uint64_t nbins = p->nbins;
    const uint64_t nbf = nbins / 2 + 1;
    const uint64_t nfreq0 = p->param_counts[0][np - 1];
    uint64_t cmax = 0;
    for (uint32_t l = 0; l < p->n_levels; ++l) {
        const uint64_t c = p->nsegments[l] * p->ncoords[l] * 4 * nbf;
        cmax = c > cmax ? c : cmax;
    }
    double* freqs = (double*)malloc(sizeof(double) * nfreq0);
    double* a = (double*)malloc(sizeof(double) * cmax);
    double* b = (double*)malloc(sizeof(double) * cmax);
    void* coords = malloc((np == 1 ? sizeof(lko_coord_freq) : sizeof(lko_coord)) * p->coord_size);
    float* tfold = NULL;
    double* tfold64 = NULL;
    int rc = 0;
    if (freqs == NULL || a == NULL || b == NULL || coords == NULL) {
        rc = fail("out of memory");
        goto done;
    }
    lko_range_param(p->limits[2 * (np - 1)], p->limits[2 * (np - 1) + 1], p->dparams[0][np - 1], freqs,
                    nfreq0);
    const double t_ref = (np == 1) ? 0.0 : p->tsegments[0] / 2.0;
    rc = (np == 1) ? lko_resolve_freq(p, (lko_coord_freq*)coords)
                   : lko_resolve_taylor(p, (lko_coord*)coords);
    if (rc != 0) {
        goto done;
    }
    if (nbins > nbins_min_lossy) {
        const uint64_t nprof = p->nsegments[0] * nfreq0 * 2;
        tfold = (float*)malloc(sizeof(float) * nprof * nbins);
        tfold64 = (double*)malloc(sizeof(double) * nprof * nbins);
        if (tfold == NULL || tfold64 == NULL) {
            rc = fail("out of memory");
            goto done;
        }
        rc = lko_brute_fold(ts_e, ts_v, p->nsamps, freqs, nfreq0, p->segment_lens[0], nbins, p->tsamp,
                            t_ref, tfold);
        if (rc != 0) {
            goto done;
        }
        for (uint64_t i = 0; i < nprof * nbins; ++i) {
            tfold64[i] = (double)tfold[i];
        }
        lko_rfft(tfold64, a, nprof, nbins);
    } else {
        rc = lko_fourier_brute_fold(ts_e, ts_v, p->nsamps, freqs, nfreq0, p->segment_lens[0], nbins,
                                    p->tsamp, t_ref, a);
        if (rc != 0) {
            goto done;
        }
    }
    for (uint32_t l = 1; l <= level_out; ++l) {
        const void* cl = (np == 1) ? (const void*)((const lko_coord_freq*)coords + p->ncoords_offsets[l])
                                   : (const void*)((const lko_coord*)coords + p->ncoords_offsets[l]);
        lko_fourier_merge(a, b, cl, np > 1, p->ncoords[l], p->ncoords[l - 1], p->nsegments[l], nbins);
        double* t = a;
        a = b;
        b = t;
    }
    memcpy(fold_out, a, sizeof(double) * p->nsegments[level_out] * p->ncoords[level_out] * 4 * nbf);
done:
    free(freqs);
    free(a);
    free(b);
    free(coords);
    free(tfold);
    free(tfold64);
    return rc;
}

/* compute_ffa_scores with use_fourier (lib/ffa.cpp:425-466): the final
 * complex fold, back to time by the inverse real transform, and the boxcar
 * S/N of every final cell and width, all in double. scores [ncoords][nw]. */
int lko_ffa_fourier_scores64(const lko_plan* p, const float* ts_e, const float* ts_v,
                             uint64_t nbins_min_lossy, const uint64_t* widths, uint64_t nw,
                             double* scores) {
    if (p->n_levels < 2 || p->nsegments[p->n_levels - 1] != 1) {
        return fail("compute_ffa_scores: nsegments must be 1 for scores");
    }
    if (nw == 0 || nw > LKO_MAX_WIDTHS) {
        return fail("lko_ffa_fourier_scores64: number of widths out of range");
    }
    const uint64_t nbins = p->nbins;
    const uint64_t nbf = nbins / 2 + 1;
    const uint64_t nc = p->ncoords[p->n_levels - 1];
    double* cf = (double*)malloc(sizeof(double) * nc * 4 * nbf);
    double* tf = (double*)malloc(sizeof(double) * nc * 2 * nbins);
    int rc = 0;
    if (cf == NULL || tf == NULL) {
        rc = fail("out of memory");
    } else {
        rc = lko_ffa_fourier(p, ts_e, ts_v, p->n_levels - 1, nbins_min_lossy, cf);
        if (rc == 0) {
            lko_irfft(cf, tf, nc * 2, nbins);
            score64(tf, nc, nbins, widths, nw, scores);
        }
    }
    free(cf);
    free(tf);
    return rc;
}
