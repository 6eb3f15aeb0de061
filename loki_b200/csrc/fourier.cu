// Fourier-domain FFA on the GPU: the level-0 direct transform of segments,
// phase-rotation merges, batched real transforms, and the executor's level
// loop (FFACUDA<ComplexTypeCUDA>).
//
// Reference: FFA<ComplexType> (lib/ffa.cpp:75-135,170-310) and its CUDA twin
// (lib/ffa_cuda.cu); kernels in lib/kernels.cpp: brute_fold_ts_complex /
// brute_fold_segment_complex (:1156-1242, :582-720), ffa_complex_iter[_freq]
// (:942-1130, :1283-1326) with shift_add_complex_recurrence_binary / _linear
// (:241-453); transforms math::rfft_batch / irfft_batch (lib/fft.cpp:375-552).
//
// Numerics. Every sum is FP32 (the reference's type); where the reference
// forms phasors in float from unreduced angles (its CUDA kernels call
// __sincosf on angles of thousands of radians), phases here are reduced
// modulo one cycle in double and the sine and cosine taken by sincospif.
// The level-0 transform steps each harmonic's phasor by one complex multiply
// per sample and re-anchors it every kDftChunk samples; merges evaluate each
// harmonic's rotation directly. Results match an FP64 statement of the same
// algorithm to about 1e-6 of the fold's scale.
#include <algorithm>
#include <cmath>
#include <memory>

#include "lk_fourier.hpp"
#include "lk_merge.cuh"
#include "lk_score.cuh"

namespace lk {
namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kDftH = 4;          // harmonics per thread
constexpr uint32_t kDftChunk = 256;    // samples per shared-memory chunk (re-anchor interval)
static_assert(kDftChunk == kThreads, "one sample per thread per chunk");

// exp(-2 pi i u), u in cycles, reduced to [0, 1) in double first.
__device__ __forceinline__ float2 unit_phasor(double u) {
    u -= floor(u);
    float s, c;
    sincospif(-2.0f * static_cast<float>(u), &s, &c);
    return make_float2(c, s);
}

// x * p (complex).
__device__ __forceinline__ float2 cmul(float2 x, float2 p) {
    return make_float2(fmaf(x.x, p.x, -(x.y * p.y)), fmaf(x.x, p.y, x.y * p.x));
}

// acc + a * b on both lanes in one sm_100a instruction (two fused
// multiply-adds, each rounded once).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 acc) {
    uint64_t ra, rb, rc, rd;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rc) : "f"(acc.x), "f"(acc.y));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(rc));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rd));
    return r;
}

struct DftArgs {
    const float* ts_e;
    const float* ts_v;
    const double* freqs;
    float2* out;
    uint64_t seglen;
    double tsamp;
    double t_ref;
    uint32_t nfreq;
    uint32_t nbf;
    uint32_t groups;  // harmonic groups of kDftH per frequency
    uint32_t fpb;     // frequencies per block
};

// Block (segment, frequency group); thread (frequency, harmonic group).
// Harmonic m of frequency f: sum_k x_k exp(-2 pi i m f t_k), t_k = k tsamp -
// t_ref, for E and V; m = 0 is the segment sum.
__global__ void __launch_bounds__(kThreads) fourier_dft_kernel(DftArgs a) {
    __shared__ float4 xs[kDftChunk];  // (e, e, v, v)
    __shared__ float2 part[kThreads / 32];
    const uint64_t seg = blockIdx.x;
    const uint32_t fl = threadIdx.x / a.groups;
    const uint32_t g = threadIdx.x - fl * a.groups;
    const uint32_t f = blockIdx.y * a.fpb + fl;
    const bool active = fl < a.fpb && f < a.nfreq;
    const double freq = active ? a.freqs[f] : 0.0;

    uint32_t mh[kDftH];
    float2 w[kDftH], p[kDftH], ae[kDftH], av[kDftH];
    double ustep = freq * a.tsamp;
    ustep -= floor(ustep);
#pragma unroll
    for (uint32_t j = 0; j < kDftH; ++j) {
        mh[j] = 1 + g * kDftH + j;
        w[j] = unit_phasor(static_cast<double>(mh[j]) * ustep);
        ae[j] = make_float2(0.0f, 0.0f);
        av[j] = make_float2(0.0f, 0.0f);
    }
    const float* e = a.ts_e + seg * a.seglen;
    const float* v = a.ts_v + seg * a.seglen;
    float2 dc = make_float2(0.0f, 0.0f);
    for (uint64_t k0 = 0; k0 < a.seglen; k0 += kDftChunk) {
        __syncthreads();  // the previous chunk is consumed
        {
            const uint64_t k = k0 + threadIdx.x;
            float xe = 0.0f, xv = 0.0f;
            if (k < a.seglen) {
                xe = __ldg(e + k);
                xv = __ldg(v + k);
            }
            dc.x += xe;
            dc.y += xv;
            xs[threadIdx.x] = make_float4(xe, xe, xv, xv);
        }
        __syncthreads();
        double u0 = freq * (static_cast<double>(k0) * a.tsamp - a.t_ref);
        u0 -= floor(u0);
#pragma unroll
        for (uint32_t j = 0; j < kDftH; ++j) {
            p[j] = unit_phasor(static_cast<double>(mh[j]) * u0);
        }
        const uint64_t left = a.seglen - k0;
        const uint32_t n = left < kDftChunk ? static_cast<uint32_t>(left) : kDftChunk;
#pragma unroll 4
        for (uint32_t k = 0; k < n; ++k) {
            const float4 x = xs[k];
            const float2 xe = make_float2(x.x, x.y), xv = make_float2(x.z, x.w);
#pragma unroll
            for (uint32_t j = 0; j < kDftH; ++j) {
                ae[j] = fma2(xe, p[j], ae[j]);
                av[j] = fma2(xv, p[j], av[j]);
                p[j] = cmul(p[j], w[j]);
            }
        }
    }
    // segment sums (DC): warp, then block
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1) {
        dc.x += __shfl_xor_sync(0xffffffffu, dc.x, o);
        dc.y += __shfl_xor_sync(0xffffffffu, dc.y, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = dc;
    }
    __syncthreads();
    if (!active) {
        return;
    }
    float2* row = a.out + ((seg * a.nfreq + f) * 2) * a.nbf;
    if (g == 0) {
        float2 t = part[0];
        for (uint32_t i = 1; i < kThreads / 32; ++i) {
            t.x += part[i].x;
            t.y += part[i].y;
        }
        row[0] = make_float2(t.x, 0.0f);
        row[a.nbf] = make_float2(t.y, 0.0f);
    }
#pragma unroll
    for (uint32_t j = 0; j < kDftH; ++j) {
        if (mh[j] < a.nbf) {
            row[mh[j]] = ae[j];
            row[a.nbf + mh[j]] = av[j];
        }
    }
}

// One output harmonic k of one (segment, coordinate) row, E and V:
// out = tail * exp(-2 pi i k st / nbins) + head * exp(-2 pi i k sh / nbins).
template <bool TAYLOR, class Idx>
__global__ void __launch_bounds__(kThreads)
fourier_merge_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                     const void* __restrict__ coords, Idx ncur, Idx nprev, Idx total,
                     uint32_t nbf, uint32_t nbins) {
    const double inv_nbins = 1.0 / static_cast<double>(nbins);
    for (Idx t = static_cast<Idx>(blockIdx.x) * kThreads + threadIdx.x; t < total;
         t += static_cast<Idx>(gridDim.x) * kThreads) {
        const Idx rowi = t / nbf;
        const uint32_t k = static_cast<uint32_t>(t - rowi * nbf);
        const Idx s = rowi / ncur;
        const Idx c = rowi - s * ncur;
        uint32_t it, ih;
        float st = 0.0f, sh;
        if constexpr (TAYLOR) {
            const CoordTaylor cc = reinterpret_cast<const CoordTaylor*>(coords)[c];
            it = cc.i_tail;
            ih = cc.i_head;
            st = cc.shift_tail;
            sh = cc.shift_head;
        } else {
            const CoordFreq cc = reinterpret_cast<const CoordFreq*>(coords)[c];
            it = ih = cc.idx;
            sh = cc.shift;
        }
        const uint64_t rs = 2ull * nbf;
        const float2* tail = in + ((2ull * s) * nprev + it) * rs + k;
        const float2* head = in + ((2ull * s + 1) * nprev + ih) * rs + k;
        float2* o = out + static_cast<uint64_t>(rowi) * rs + k;
        const float2 ph = unit_phasor(static_cast<double>(k) * static_cast<double>(sh) * inv_nbins);
        const float2 te = __ldg(tail), tv = __ldg(tail + nbf);
        const float2 he = cmul(__ldg(head), ph), hv = cmul(__ldg(head + nbf), ph);
        if constexpr (TAYLOR) {
            const float2 pt =
                unit_phasor(static_cast<double>(k) * static_cast<double>(st) * inv_nbins);
            const float2 re = cmul(te, pt), rv = cmul(tv, pt);
            o[0] = make_float2(re.x + he.x, re.y + he.y);
            o[nbf] = make_float2(rv.x + hv.x, rv.y + hv.y);
        } else {
            o[0] = make_float2(te.x + he.x, te.y + he.y);
            o[nbf] = make_float2(tv.x + hv.x, tv.y + hv.y);
        }
    }
}

// Twiddles (cos, sin)(2 pi t / n) for t in [0, n) into shared memory.
__device__ __forceinline__ void fill_twiddles(float2* tw, uint32_t n) {
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        float s, c;
        sincospif(2.0f * static_cast<float>(t) / static_cast<float>(n), &s, &c);
        tw[t] = make_float2(c, s);
    }
}

// c2r of size n, scaled by `scale`: x_j = scale (Re X_0 + sum_{0<m<n/2}
// 2 Re(X_m e^{2 pi i m j / n}) + [n even] Re X_{n/2} (-1)^j). Block: ppb
// profiles; shared memory: n twiddles, then ppb * nbf coefficients.
__global__ void __launch_bounds__(kThreads)
irfft_kernel(const float2* __restrict__ in, float* __restrict__ out, uint64_t nprof, uint32_t n,
             uint32_t nbf, uint32_t ppb, float scale) {
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* xs = sm + n;
    fill_twiddles(tw, n);
    for (uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * ppb; p0 < nprof;
         p0 += static_cast<uint64_t>(gridDim.x) * ppb) {
        const uint64_t left = nprof - p0;
        const uint32_t np = left < ppb ? static_cast<uint32_t>(left) : ppb;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < np * nbf; i += blockDim.x) {
            xs[i] = in[p0 * nbf + i];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < np * n; i += blockDim.x) {
            const uint32_t pl = i / n;
            const uint32_t j = i - pl * n;
            const float2* x = xs + pl * nbf;
            float acc = x[0].x;
            uint32_t t = 0;
            for (uint32_t m = 1; m < nbf; ++m) {
                t += j;
                t = t >= n ? t - n : t;
                const float re = fmaf(x[m].x, tw[t].x, -(x[m].y * tw[t].y));
                acc += (2 * m == n) ? re : 2.0f * re;
            }
            out[(p0 + pl) * n + j] = acc * scale;
        }
    }
}

// r2c of size n, unscaled: X_m = sum_j x_j e^{-2 pi i m j / n}, m < nbf.
__global__ void __launch_bounds__(kThreads)
rfft_kernel(const float* __restrict__ in, float2* __restrict__ out, uint64_t nprof, uint32_t n,
            uint32_t nbf, uint32_t ppb) {
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float* xs = reinterpret_cast<float*>(sm + n);
    fill_twiddles(tw, n);
    for (uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * ppb; p0 < nprof;
         p0 += static_cast<uint64_t>(gridDim.x) * ppb) {
        const uint64_t left = nprof - p0;
        const uint32_t np = left < ppb ? static_cast<uint32_t>(left) : ppb;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < np * n; i += blockDim.x) {
            xs[i] = in[p0 * n + i];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < np * nbf; i += blockDim.x) {
            const uint32_t pl = i / nbf;
            const uint32_t m = i - pl * nbf;
            const float* x = xs + pl * n;
            float re = 0.0f, im = 0.0f;
            uint32_t t = 0;
            for (uint32_t j = 0; j < n; ++j) {
                re = fmaf(x[j], tw[t].x, re);
                im = fmaf(-x[j], tw[t].y, im);
                t += m;
                t = t >= n ? t - n : t;
            }
            out[(p0 + pl) * nbf + m] = make_float2(re, im);
        }
    }
}

// ---- fused final level: merge + inverse real transform + boxcar S/N ----
//
// One block of kFinCells final cells (nbins <= 64, one final segment).
// Phase 1, all threads: the merged harmonics of the block's cells (tail and
// head rows of the previous level rotated and added, as fourier_merge_kernel;
// consecutive threads take consecutive harmonics of a row) into shared memory
// as [harmonic][cell] (E re, E im, V re, V im), rows padded by one entry.
// Phase 2, a thread per cell: its harmonics into registers, then the inverse
// transform by sums over the harmonics with the folding symmetries of the c2r
// kernel (x_j and x_{n-j} from one cosine and one sine sum; for n divisible
// by 4 also x_{n/2-j} and x_{n/2+j} from the even and odd harmonics apart),
// each output normalised E / sqrt(V) into the cell's row, which reuses the
// harmonic tile. Phase 3: the boxcar scorer on the row. The twiddle table
// holds (c_m / n) (cos, sin)(2 pi m j / n) for the j a thread evaluates
// (c_m = 1 for the DC and Nyquist terms, else 2), so the scale of the c2r
// transform and the unused imaginary parts of the DC and Nyquist terms come
// out of the table.
constexpr uint32_t kFinCells = 64;
constexpr uint32_t kFinPitch = kFinCells + 1;  // float4 entries per harmonic row

struct FinalArgs {
    const float2* in;       // level L-2 complex fold [2 segments][nprev][2][nbf]
    const void* coords;     // level L-1 coordinates
    const float2* tw;       // [jcount][nbf] scaled twiddles
    float* scores;          // [ncur][nwidths]
    uint64_t ncur, nprev;
    uint32_t nbins, nbf, jcount, rs;
    ScoreParams sp;
    MaskScoreParams mp;     // the masked scorer's widths (NB > 0)
};

// NB > 0: nbins NB (32 or 64) with the widths in mp, scored by the masked
// scorer (rows of NB + WM + 2 floats; FM its compile-time mask or 0); NB = 0:
// any nbins, scored by score_row.
template <bool TAYLOR, int NW, int NBF, int NB, int WM, uint64_t FM>
__global__ void __launch_bounds__(kFinCells)
fourier_final_kernel(FinalArgs a) {
    extern __shared__ float4 fsm[];
    float2* tw = reinterpret_cast<float2*>(fsm);                       // [jcount][nbf]
    float4* coef = fsm + (a.jcount * a.nbf + 1) / 2;                   // [nbf][kFinPitch]
    float* rows = reinterpret_cast<float*>(coef);                      // [kFinCells][rs], after phase 2 loads
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kFinCells;
    const uint64_t left = a.ncur - c0;
    const uint32_t ncells = left < kFinCells ? static_cast<uint32_t>(left) : kFinCells;
    for (uint32_t i = threadIdx.x; i < a.jcount * a.nbf; i += blockDim.x) {
        tw[i] = a.tw[i];
    }
    const double inv_nbins = 1.0 / static_cast<double>(a.nbins);
    const uint64_t rs2 = 2ull * a.nbf;
    // the block's coordinates, staged once: the row loads below then depend
    // on shared memory only
    __shared__ uint32_t c_it[kFinCells], c_ih[kFinCells];
    __shared__ float c_st[kFinCells], c_sh[kFinCells];
    if (threadIdx.x < ncells) {
        const uint64_t c = c0 + threadIdx.x;
        if constexpr (TAYLOR) {
            const CoordTaylor cc = reinterpret_cast<const CoordTaylor*>(a.coords)[c];
            c_it[threadIdx.x] = cc.i_tail;
            c_ih[threadIdx.x] = cc.i_head;
            c_st[threadIdx.x] = cc.shift_tail;
            c_sh[threadIdx.x] = cc.shift_head;
        } else {
            const CoordFreq cc = reinterpret_cast<const CoordFreq*>(a.coords)[c];
            c_it[threadIdx.x] = c_ih[threadIdx.x] = cc.idx;
            c_st[threadIdx.x] = 0.0f;
            c_sh[threadIdx.x] = cc.shift;
        }
    }
    __syncthreads();
    // four items per thread in flight: all their row loads first
    constexpr uint32_t kU = 4;
    const uint32_t total = ncells * a.nbf;
    for (uint32_t base = threadIdx.x; base < total; base += kU * blockDim.x) {
        float2 te[kU], tv[kU], he[kU], hv[kU];
        uint32_t kk[kU], cls[kU];
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            const uint32_t i = base + u * blockDim.x;
            const uint32_t ii = i < total ? i : base;
            cls[u] = ii / a.nbf;
            kk[u] = ii - cls[u] * a.nbf;
            const float2* tail = a.in + static_cast<uint64_t>(c_it[cls[u]]) * rs2 + kk[u];
            const float2* head = a.in + (a.nprev + c_ih[cls[u]]) * rs2 + kk[u];
            te[u] = __ldg(tail);
            tv[u] = __ldg(tail + a.nbf);
            he[u] = __ldg(head);
            hv[u] = __ldg(head + a.nbf);
        }
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            if (base + u * blockDim.x >= total) {
                break;
            }
            const double k = static_cast<double>(kk[u]);
            const float2 ph = unit_phasor(k * static_cast<double>(c_sh[cls[u]]) * inv_nbins);
            float2 e0 = te[u], v0 = tv[u];
            if constexpr (TAYLOR) {
                const float2 pt = unit_phasor(k * static_cast<double>(c_st[cls[u]]) * inv_nbins);
                e0 = cmul(e0, pt);
                v0 = cmul(v0, pt);
            }
            const float2 e1 = cmul(he[u], ph), v1 = cmul(hv[u], ph);
            coef[kk[u] * kFinPitch + cls[u]] = make_float4(e0.x + e1.x, e0.y + e1.y, v0.x + v1.x, v0.y + v1.y);
        }
    }
    __syncthreads();
    const uint32_t t = threadIdx.x;
    float4 x[NBF];
#pragma unroll
    for (int m = 0; m < NBF; ++m) {
        x[m] = (t < ncells && m < static_cast<int>(a.nbf)) ? coef[m * kFinPitch + t]
                                                          : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();  // the harmonic tile becomes the rows
    if (t >= ncells) {
        return;
    }
    float* r = rows + t * a.rs;
    const uint32_t n = a.nbins;
    const bool quad = (n % 4) == 0;
    for (uint32_t j = 0; j < a.jcount; ++j) {
        float ce0 = 0.0f, ce1 = 0.0f, se0 = 0.0f, se1 = 0.0f;  // E: even / odd harmonics
        float cv0 = 0.0f, cv1 = 0.0f, sv0 = 0.0f, sv1 = 0.0f;  // V
        const float2* twj = tw + j * a.nbf;
#pragma unroll
        for (int m = 0; m < NBF; ++m) {
            if (m < static_cast<int>(a.nbf)) {
                const float2 w = twj[m];
                if (m % 2 == 0) {
                    ce0 = fmaf(x[m].x, w.x, ce0);
                    se0 = fmaf(x[m].y, w.y, se0);
                    cv0 = fmaf(x[m].z, w.x, cv0);
                    sv0 = fmaf(x[m].w, w.y, sv0);
                } else {
                    ce1 = fmaf(x[m].x, w.x, ce1);
                    se1 = fmaf(x[m].y, w.y, se1);
                    cv1 = fmaf(x[m].z, w.x, cv1);
                    sv1 = fmaf(x[m].w, w.y, sv1);
                }
            }
        }
        const float ce = ce0 + ce1, se = se0 + se1, cv = cv0 + cv1, sv = sv0 + sv1;
        r[j] = (ce - se) * rsqrtf(cv - sv);
        if (j > 0) {
            r[n - j] = (ce + se) * rsqrtf(cv + sv);
        }
        if (quad) {
            const float de = ce0 - ce1, he = se0 - se1, dv = cv0 - cv1, hv = sv0 - sv1;
            r[n / 2 - j] = (de + he) * rsqrtf(dv + hv);
            r[n / 2 + j] = (de - he) * rsqrtf(dv - hv);
        }
    }
    float* out = a.scores + (c0 + t) * a.sp.nwidths;
    if constexpr (NB > 0) {
        sc::max_snr_div_wm<NB, WM, FM>(r, a.mp, 1.0f, out);
    } else {
        sc::score_row<NW>(r, n, 1.0f, a.sp, LK_SCORE_PER_WIDTH, out);
    }
}

uint32_t grid_for(uint64_t work, uint32_t per_block) {
    const uint64_t b = (work + per_block - 1) / per_block;
    return static_cast<uint32_t>(std::clamp<uint64_t>(b, 1, 148ull * 64));
}

// Profiles per block of the transforms and their shared-memory bytes.
uint32_t transform_ppb(uint32_t n) { return std::max<uint32_t>(1, 1024 / std::max<uint32_t>(n, 1)); }

}  // namespace

void fourier_dft_fold(const float* d_ts_e, const float* d_ts_v, const double* d_freqs,
                      uint32_t nfreq, uint64_t seglen, uint64_t nseg, uint32_t nbins, double tsamp,
                      double t_ref, float2* d_out, cudaStream_t s) {
    require(nbins >= 2 && nbins <= 2 * kDftH * kThreads, "direct transform: nbins out of range");
    require(nseg >= 1 && nseg <= 0x7fffffffULL && seglen >= 1, "direct transform: bad segments");
    DftArgs a{};
    a.ts_e = d_ts_e;
    a.ts_v = d_ts_v;
    a.freqs = d_freqs;
    a.out = d_out;
    a.seglen = seglen;
    a.tsamp = tsamp;
    a.t_ref = t_ref;
    a.nfreq = nfreq;
    a.nbf = nbins / 2 + 1;
    a.groups = std::max<uint32_t>(1, (a.nbf - 1 + kDftH - 1) / kDftH);
    a.fpb = std::max<uint32_t>(1, kThreads / a.groups);
    const uint64_t gy = (static_cast<uint64_t>(nfreq) + a.fpb - 1) / a.fpb;
    require(gy <= 65535, "direct transform: too many frequencies");
    fourier_dft_kernel<<<dim3(static_cast<uint32_t>(nseg), static_cast<uint32_t>(gy)), kThreads, 0,
                         s>>>(a);
    LK_CUDA(cudaGetLastError());
}

void fourier_merge_level(const float2* d_in, float2* d_out, const void* d_coords, bool taylor,
                         uint64_t ncur, uint64_t nprev, uint64_t nseg, uint32_t nbins,
                         cudaStream_t s) {
    const uint32_t nbf = nbins / 2 + 1;
    const uint64_t total = nseg * ncur * nbf;
    const uint32_t grid = grid_for(total, kThreads * 4);
    if (total < (1ull << 32)) {
        const auto t32 = static_cast<uint32_t>(total);
        const auto c32 = static_cast<uint32_t>(ncur);
        const auto p32 = static_cast<uint32_t>(nprev);
        if (taylor) {
            fourier_merge_kernel<true, uint32_t>
                <<<grid, kThreads, 0, s>>>(d_in, d_out, d_coords, c32, p32, t32, nbf, nbins);
        } else {
            fourier_merge_kernel<false, uint32_t>
                <<<grid, kThreads, 0, s>>>(d_in, d_out, d_coords, c32, p32, t32, nbf, nbins);
        }
    } else if (taylor) {
        fourier_merge_kernel<true, uint64_t>
            <<<grid, kThreads, 0, s>>>(d_in, d_out, d_coords, ncur, nprev, total, nbf, nbins);
    } else {
        fourier_merge_kernel<false, uint64_t>
            <<<grid, kThreads, 0, s>>>(d_in, d_out, d_coords, ncur, nprev, total, nbf, nbins);
    }
    LK_CUDA(cudaGetLastError());
}

void rfft_profiles(const float* d_in, float2* d_out, uint64_t nprof, uint32_t nbins,
                   cudaStream_t s) {
    const uint32_t nbf = nbins / 2 + 1;
    const uint32_t ppb = transform_ppb(nbins);
    const size_t smem = sizeof(float2) * nbins + sizeof(float) * ppb * nbins;
    require(smem <= 48 * 1024, "real transform: nbins too large");
    rfft_kernel<<<grid_for(nprof, ppb), kThreads, smem, s>>>(d_in, d_out, nprof, nbins, nbf, ppb);
    LK_CUDA(cudaGetLastError());
}

void irfft_profiles(const float2* d_in, float* d_out, uint64_t nprof, uint32_t nbins,
                    cudaStream_t s) {
    const uint32_t nbf = nbins / 2 + 1;
    const uint32_t ppb = transform_ppb(nbins);
    const size_t smem = sizeof(float2) * (nbins + static_cast<size_t>(ppb) * nbf);
    require(smem <= 48 * 1024, "inverse real transform: nbins too large");
    irfft_kernel<<<grid_for(nprof, ppb), kThreads, smem, s>>>(d_in, d_out, nprof, nbins, nbf, ppb,
                                                              1.0f / static_cast<float>(nbins));
    LK_CUDA(cudaGetLastError());
}

bool fourier_final_supported(uint32_t nbins) { return nbins >= 2 && nbins <= 64; }

uint32_t fourier_final_jcount(uint32_t nbins) {
    // outputs a thread evaluates directly: j in [0, n/4] with the four-fold
    // symmetry (n divisible by 4), else j in [0, n/2]
    return (nbins % 4 == 0) ? nbins / 4 + 1 : nbins / 2 + 1;
}

std::vector<float2> fourier_final_twiddles(uint32_t nbins) {
    const uint32_t nbf = nbins / 2 + 1;
    const uint32_t jc = fourier_final_jcount(nbins);
    std::vector<float2> tw(static_cast<size_t>(jc) * nbf);
    const double two_pi = 6.283185307179586476925286766559;
    for (uint32_t j = 0; j < jc; ++j) {
        for (uint32_t m = 0; m < nbf; ++m) {
            const bool edge = m == 0 || 2 * m == nbins;
            const double cm = edge ? 1.0 : 2.0;
            const double th = two_pi * static_cast<double>((static_cast<uint64_t>(m) * j) % nbins) /
                              static_cast<double>(nbins);
            const double sn = edge ? 0.0 : std::sin(th);
            tw[static_cast<size_t>(j) * nbf + m] = make_float2(static_cast<float>(cm * std::cos(th) / nbins),
                                                               static_cast<float>(cm * sn / nbins));
        }
    }
    return tw;
}

void fourier_final_score(const float2* d_in, const void* d_coords, bool taylor, uint64_t ncur,
                         uint64_t nprev, uint32_t nbins, const ScoreParams& sp, const float2* d_tw,
                         float* d_scores, cudaStream_t s) {
    require(fourier_final_supported(nbins), "fused Fourier final level: nbins must lie in [2, 64]");
    FinalArgs a{};
    a.in = d_in;
    a.coords = d_coords;
    a.tw = d_tw;
    a.scores = d_scores;
    a.ncur = ncur;
    a.nprev = nprev;
    a.nbins = nbins;
    a.nbf = nbins / 2 + 1;
    a.jcount = fourier_final_jcount(nbins);
    a.rs = sc::row_stride(nbins, sp.wmax);
    a.sp = sp;
    MaskScoreParams mp{};
    const bool masked = (nbins == 32 || nbins == 64) && make_mask_score_params(sp, nbins, &mp);
    uint32_t wm = 0;
    if (masked) {
        wm = mp.wmax <= 8 ? 8u : (mp.wmax <= 16 ? 16u : 32u);
        a.rs = nbins + wm + 2;  // even: rows start on 8 bytes
        a.mp = mp;
    }
    const size_t tile = std::max(sizeof(float4) * a.nbf * kFinPitch, sizeof(float) * kFinCells * a.rs);
    const size_t smem = sizeof(float4) * ((a.jcount * a.nbf + 1) / 2) + tile;
    const uint64_t blocks = (ncur + kFinCells - 1) / kFinCells;
    require(blocks <= 0x7fffffffULL, "fused Fourier final level: too many cells");
    auto launch = [&](auto kern) {
        sc::set_smem(kern, smem);
        kern<<<static_cast<uint32_t>(blocks), kFinCells, smem, s>>>(a);
    };
    auto by_nbf = [&](auto tay, auto nw) {
        constexpr bool T = decltype(tay)::value;
        constexpr int NW = decltype(nw)::value;
        if (masked) {
            auto by_wm = [&](auto nbf, auto nbc) {
                constexpr int NBF = decltype(nbf)::value;
                constexpr int NB = decltype(nbc)::value;
                if (wm == 8) {
                    launch(fourier_final_kernel<T, NW, NBF, NB, 8, 0>);
                } else if (wm == 16) {
                    if (mp.wmask == sc::kFixedMask16 && mp.wmax == 16) {
                        launch(fourier_final_kernel<T, NW, NBF, NB, 16, sc::kFixedMask16>);
                    } else {
                        launch(fourier_final_kernel<T, NW, NBF, NB, 16, 0>);
                    }
                } else {
                    launch(fourier_final_kernel<T, NW, NBF, NB, 32, 0>);
                }
            };
            if (nbins == 32) {
                by_wm(std::integral_constant<int, 17>{}, std::integral_constant<int, 32>{});
            } else {
                by_wm(std::integral_constant<int, 33>{}, std::integral_constant<int, 64>{});
            }
        } else if (a.nbf <= 9) {
            launch(fourier_final_kernel<T, NW, 9, 0, 0, 0>);
        } else if (a.nbf <= 17) {
            launch(fourier_final_kernel<T, NW, 17, 0, 0, 0>);
        } else {
            launch(fourier_final_kernel<T, NW, 33, 0, 0, 0>);
        }
    };
    auto by_nw = [&](auto tay) {
        if (sp.nwidths <= 8) {
            by_nbf(tay, std::integral_constant<int, 8>{});
        } else if (sp.nwidths <= 16) {
            by_nbf(tay, std::integral_constant<int, 16>{});
        } else {
            by_nbf(tay, std::integral_constant<int, 32>{});
        }
    };
    if (taylor) {
        by_nw(std::true_type{});
    } else {
        by_nw(std::false_type{});
    }
    LK_CUDA(cudaGetLastError());
}

// ---- executor -------------------------------------------------------------

FourierExec::FourierExec(const Plan& p, int device_, uint64_t nbins_min_lossy)
    : plan(p), device(device_) {
    require(!plan.offsets_overflow, "coordinate offsets exceed 32 bits");
    require(plan.nparams <= 3, "the FFA executor supports nparams <= 3");
    require(plan.n_levels >= 2, "FFA::execute_unified: levels must be greater than or equal to 2");
    require(plan.cfg.nbins >= 2 && plan.cfg.nbins <= 4096, "Fourier FFA: nbins must lie in [2, 4096]");
    if (nbins_min_lossy == 0) {
        nbins_min_lossy = kNbinsMinLossy;
    }
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    nbf = nbins / 2 + 1;
    lossy = plan.cfg.nbins > nbins_min_lossy;
    require(lossy || nbins <= 2 * kDftH * kThreads, "Fourier FFA: direct transform needs nbins <= 2048");
    DeviceGuard g(device);
    status.alloc(sizeof(uint32_t));
    LK_CUDA(cudaMemset(status.ptr, 0, sizeof(uint32_t)));
    const size_t elem = plan.nparams == 1 ? 8 : 16;
    coords.alloc(elem * plan.coord_size);
    resolve_coords_device(plan, coords.ptr, nullptr);
    const uint32_t np = plan.nparams;
    const std::vector<double> f0 = plan.param_grid(0, np - 1);
    require(f0.size() == plan.ncoords[0], "internal: level-0 frequency grid");
    freqs0.alloc(sizeof(double) * f0.size());
    LK_CUDA(cudaMemcpy(freqs0.ptr, f0.data(), sizeof(double) * f0.size(), cudaMemcpyHostToDevice));
    if (lossy) {
        bf = std::make_unique<BruteFoldDevice>(f0, plan.segment_lens[0], plan.cfg.nbins,
                                               plan.cfg.nsamps, plan.cfg.tsamp, plan.t_ref0(),
                                               status.as<uint32_t>());
        tfold.alloc(sizeof(float) * plan.fold_size(0));
    }
    if (!lossy && fourier_mma_supported(plan.segment_lens[0], plan.nsegments[0], nbins)) {
        mma = std::make_unique<FourierMma>(plan.segment_lens[0], plan.nsegments[0], nbins,
                                           static_cast<uint32_t>(plan.ncoords[0]));
    }
    uint64_t inter = 0;
    for (uint32_t l = 0; l < plan.n_levels; ++l) {
        inter = std::max(inter, fold_size(l));
    }
    buf[0].alloc(sizeof(float2) * inter);
    buf[1].alloc(sizeof(float2) * inter);
    sp = make_score_params(plan.widths.data(), static_cast<uint32_t>(plan.widths.size()), nbins);
    if (fourier_final_supported(nbins) && plan.nsegments[plan.n_levels - 1] == 1) {
        const std::vector<float2> tw = fourier_final_twiddles(nbins);
        final_tw.alloc(sizeof(float2) * tw.size());
        LK_CUDA(cudaMemcpy(final_tw.ptr, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice));
    }
    LK_CUDA(cudaDeviceSynchronize());
}

uint64_t FourierExec::device_bytes() const {
    return status.bytes + coords.bytes + freqs0.bytes + buf[0].bytes + buf[1].bytes + tfold.bytes +
           tfinal.bytes + scores_tmp.bytes + compact_scratch.bytes + (bf ? bf->device_bytes() : 0) +
           (mma ? mma->device_bytes() : 0) + final_tw.bytes;
}

const void* FourierExec::level_coords(uint32_t l) const {
    const size_t elem = plan.nparams == 1 ? 8 : 16;
    return static_cast<const char*>(coords.ptr) + elem * plan.ncoords_offsets[l];
}

const float2* FourierExec::run_levels(const float* ts_e, const float* ts_v, float2* final_out,
                                      cudaStream_t s, int last_level) {
    const uint32_t L = last_level < 0 ? plan.n_levels : static_cast<uint32_t>(last_level) + 1;
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    const bool taylor = plan.nparams > 1;
    // Level l lands in buf[l % 2], the final one in final_out when given.
    auto dst = [&](uint32_t l) -> float2* {
        return (l == plan.n_levels - 1 && final_out != nullptr) ? final_out : buf[l % 2].as<float2>();
    };
    const uint64_t series_bytes = 8 * plan.cfg.nsamps;
    float2* in = dst(0);
    if (lossy) {
        bf->bind_inputs(ts_e, ts_v, s);
        prof.begin(LK_STAGE_BRUTE_FOLD, 0, bf->interleaves() ? 2 : 1,
                   series_bytes + 4 * plan.fold_size(0), s);
        bf->fold(tfold.as<float>(), s);
        prof.end(s);
        prof.begin(LK_STAGE_TRANSFORM, 0, 1, 4 * plan.fold_size(0) + 8 * fold_size(0), s);
        rfft_profiles(tfold.as<float>(), in, plan.fold_size(0) / nbins, nbins, s);
        prof.end(s);
    } else if (uses_mma()) {
        // series in, FP16 staging out and in again (hi + lo), fold out
        prof.begin(LK_STAGE_BRUTE_FOLD, 0, 4, 2 * series_bytes + 16 * plan.cfg.nsamps + 8 * fold_size(0),
                   s);
        mma->run(ts_e, ts_v, freqs0.as<double>(), plan.cfg.tsamp, plan.t_ref0(), in,
                 status.as<uint32_t>(), s);
        prof.end(s);
    } else {
        prof.begin(LK_STAGE_BRUTE_FOLD, 0, 1, series_bytes + 8 * fold_size(0), s);
        fourier_dft_fold(ts_e, ts_v, freqs0.as<double>(), static_cast<uint32_t>(plan.ncoords[0]),
                         plan.segment_lens[0], plan.nsegments[0], nbins, plan.cfg.tsamp,
                         plan.t_ref0(), in, s);
        prof.end(s);
    }
    for (uint32_t l = 1; l < L; ++l) {
        float2* out = dst(l);
        prof.begin(LK_STAGE_MERGE, static_cast<int>(l), 1,
                   8 * (fold_size(l - 1) + fold_size(l)) +
                       plan.ncoords[l] * (plan.nparams == 1 ? 8 : 16),
                   s);
        fourier_merge_level(in, out, level_coords(l), taylor, plan.ncoords[l], plan.ncoords[l - 1],
                            plan.nsegments[l], nbins, s);
        prof.end(s);
        in = out;
    }
    return in;
}

void FourierExec::execute(const float* ts_e, const float* ts_v, float2* fold, uint64_t len_complex,
                          cudaStream_t s) {
    require(len_complex >= fold_size(plan.n_levels - 1), "fold must hold fold_size complex values");
    DeviceGuard g(device);
    prof.reset();
    run_levels(ts_e, ts_v, fold, s);
}

void FourierExec::execute_time(const float* ts_e, const float* ts_v, float* fold, uint64_t len,
                               cudaStream_t s) {
    const uint32_t L = plan.n_levels;
    require(len >= fold_size_time(L - 1), "fold must hold fold_size_time floats");
    DeviceGuard g(device);
    prof.reset();
    const float2* fin = run_levels(ts_e, ts_v, nullptr, s);
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    prof.begin(LK_STAGE_TRANSFORM, static_cast<int>(L - 1), 1,
               8 * fold_size(L - 1) + 4 * fold_size_time(L - 1), s);
    irfft_profiles(fin, fold, fold_size(L - 1) / nbf, nbins, s);
    prof.end(s);
}

void FourierExec::scores_into(const float* ts_e, const float* ts_v, float* d_scores,
                              cudaStream_t s) {
    const uint32_t L = plan.n_levels;
    const uint64_t nc = plan.ncoords[L - 1];
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    if (final_tw.ptr != nullptr) {
        // levels 0 .. L-2, then the final merge fused with the transform and scorer
        run_levels(ts_e, ts_v, nullptr, s, static_cast<int>(L) - 2);
        const float2* in = buf[(L - 2) % 2].as<float2>();
        prof.begin(LK_STAGE_MERGE_SCORE, static_cast<int>(L - 1), 1,
                   8 * fold_size(L - 2) + 4 * nc * plan.widths.size() +
                       plan.ncoords[L - 1] * (plan.nparams == 1 ? 8 : 16),
                   s);
        fourier_final_score(in, level_coords(L - 1), plan.nparams > 1, nc, plan.ncoords[L - 2], nbins, sp,
                            final_tw.as<float2>(), d_scores, s);
        prof.end(s);
        return;
    }
    if (tfinal.bytes < sizeof(float) * fold_size_time(L - 1)) {
        tfinal.alloc(sizeof(float) * fold_size_time(L - 1));
    }
    const float2* fin = run_levels(ts_e, ts_v, nullptr, s);
    prof.begin(LK_STAGE_TRANSFORM, static_cast<int>(L - 1), 1,
               8 * fold_size(L - 1) + 4 * fold_size_time(L - 1), s);
    irfft_profiles(fin, tfinal.as<float>(), fold_size(L - 1) / nbf, nbins, s);
    prof.end(s);
    prof.begin(LK_STAGE_SCORE, static_cast<int>(L - 1), 1,
               4 * fold_size_time(L - 1) + 4 * nc * plan.widths.size(), s);
    score_folds(tfinal.as<float>(), nc, nbins, true, 1.0f, sp, LK_SCORE_PER_WIDTH, d_scores, s);
    prof.end(s);
}

void FourierExec::scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                         cudaStream_t s) {
    const uint32_t L = plan.n_levels;
    require(plan.nsegments[L - 1] == 1, "compute_ffa_scores: nsegments must be 1 for scores");
    require(len >= plan.ncoords[L - 1] * plan.widths.size(),
            "scores must hold ncoords * n_widths floats");
    DeviceGuard g(device);
    prof.reset();
    scores_into(ts_e, ts_v, d_scores, s);
}

void FourierExec::search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx,
                         float* d_snr, uint64_t max_cands, uint64_t* d_count, cudaStream_t s) {
    const uint32_t L = plan.n_levels;
    require(plan.nsegments[L - 1] == 1, "compute_ffa_scores: nsegments must be 1 for scores");
    const uint64_t n = plan.ncoords[L - 1] * plan.widths.size();
    DeviceGuard g(device);
    if (scores_tmp.bytes < n * sizeof(float)) {
        scores_tmp.alloc(n * sizeof(float));
        compact_scratch.alloc(compact_scratch_bytes(n));
    }
    prof.reset();
    scores_into(ts_e, ts_v, scores_tmp.as<float>(), s);
    prof.begin(LK_STAGE_COMPACT, -1, 3, 8 * n, s);
    compact_ge(scores_tmp.as<float>(), n, snr_min, d_idx, d_snr, max_cands, d_count,
               compact_scratch.ptr, s);
    prof.end(s);
}

void FourierExec::set_level0(int mode) {
    require(mode == LK_FOURIER_L0_AUTO || mode == LK_FOURIER_L0_CUDA_CORES ||
                mode == LK_FOURIER_L0_TENSOR_CORES,
            "level-0 mode must be LK_FOURIER_L0_AUTO, _CUDA_CORES or _TENSOR_CORES");
    if (mode == LK_FOURIER_L0_TENSOR_CORES && mma == nullptr) {
        fail(LK_ERR_UNSUPPORTED, lossy ? "the level-0 fold of nbins > nbins_min_lossy_bf is the lossy one"
                                       : "tensor-core level 0 needs nbins / 2 <= 64 and segment lengths "
                                         "that are multiples of 8");
    }
    level0 = mode;
}

float FourierExec::tune_level0(const float* ts_e, const float* ts_v, uint32_t reps, cudaStream_t s) {
    require(reps >= 1 && reps <= 100, "reps must lie in [1, 100]");
    DeviceGuard g(device);
    if (!mma) {
        return 0.0f;
    }
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    const uint32_t nfreq = static_cast<uint32_t>(plan.ncoords[0]);
    cudaEvent_t e0, e1;
    LK_CUDA(cudaEventCreate(&e0));
    LK_CUDA(cudaEventCreate(&e1));
    float best = 0.0f;
    std::unique_ptr<FourierMma> keep;
    for (uint32_t sub : {2u, 1u}) {
        for (uint32_t pc : {64u, 128u, 256u}) {
            auto cand = std::make_unique<FourierMma>(plan.segment_lens[0], plan.nsegments[0], nbins, nfreq,
                                                     sub, pc);
            auto run = [&] {
                cand->run(ts_e, ts_v, freqs0.as<double>(), plan.cfg.tsamp, plan.t_ref0(),
                          buf[0].as<float2>(), status.as<uint32_t>(), s);
            };
            run();  // warm-up
            LK_CUDA(cudaEventRecord(e0, s));
            for (uint32_t r = 0; r < reps; ++r) {
                run();
            }
            LK_CUDA(cudaEventRecord(e1, s));
            LK_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            LK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= static_cast<float>(reps);
            if (!keep || ms < best) {
                best = ms;
                keep = std::move(cand);
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    mma = std::move(keep);
    return best;
}

uint32_t FourierExec::read_status(cudaStream_t s) {
    DeviceGuard g(device);
    LK_CUDA(cudaStreamSynchronize(s));
    uint32_t st = 0;
    LK_CUDA(cudaMemcpy(&st, status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return st;
}

std::vector<lk_stage_time> FourierExec::profile(cudaStream_t s) {
    DeviceGuard g(device);
    LK_CUDA(cudaStreamSynchronize(s));
    std::vector<lk_stage_time> out;
    for (size_t i = 0; i < prof.used; ++i) {
        const auto& st = prof.stages[i];
        lk_stage_time t{};
        t.kind = st.kind;
        t.level = st.level;
        t.launches = st.launches;
        t.bytes = st.bytes;
        LK_CUDA(cudaEventElapsedTime(&t.ms, st.start, st.stop));
        out.push_back(t);
    }
    return out;
}

}  // namespace lk
