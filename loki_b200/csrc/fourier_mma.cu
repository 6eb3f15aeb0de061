// Level-0 direct transform of the Fourier-domain FFA on the tensor cores.
//
// The transform of every level-0 segment at every frequency and harmonic
// (kernels::brute_fold_ts_complex, lib/kernels.cpp:1156-1242) is one matrix
// product per frequency tile, shared by all segments:
//
//   D[r, n] = sum_k A[r, k] B[n, k]
//   r = (frequency, harmonic m >= 1, re / im): A = Re / Im exp(-2 pi i m f t_k)
//   n = (row E or V, segment s):               B = x[s * L + k]
//   k < L (segment length), t_k = k tsamp - t_ref
//
// A is generated on the fly into shared memory by four warps (a phasor
// recurrence per (frequency, harmonic), re-anchored every 256 samples from
// phases reduced in FP64); B is the series, staged once by a pre-pass as FP16
// hi / lo halves scaled by a power of two (x 2^q = hi + lo to 2^-22) and
// loaded by TMA. Each product is three FP16 tcgen05.mma passes with FP32
// accumulation in tensor memory (A_hi B_hi + A_hi B_lo + A_lo B_hi), which
// keeps about 22 bits of the operands: the same accuracy class as FP32 sums.
//
// Block: warp 0 issues the TMA loads of B, warp 1 allocates tensor memory and
// issues the MMAs, warps 2-5 generate A and, after the last K chunk, read the
// accumulators (each warp its 32-lane quadrant) and write the complex fold.
// Two stages of (A, B) in shared memory; every wait is bounded.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "lk_fourier.hpp"
#include "lk_ptx.cuh"

namespace lk {
namespace {

constexpr uint32_t kRows = 128;       // MMA M: rows (frequency, harmonic, re/im) per tile
constexpr uint32_t kKc = 32;          // samples per stage (64 bytes of FP16 per row)
constexpr uint32_t kStages = 2;
constexpr uint32_t kMaxN = 256;       // MMA N per instruction
constexpr uint32_t kThreads = 192;    // 6 warps
constexpr uint32_t kGenThreads = 128; // warps 2-5
constexpr uint32_t kAnchor = 8;       // stages between exact phasor anchors (256 samples)
constexpr uint32_t kMaxParts = 8;     // K parts at most
constexpr uint32_t kRowBytes = kKc * 2;               // 64
constexpr uint32_t kATileBytes = kRows * kRowBytes;   // 8 KB per (hi | lo)

// status bits of this kernel's bounded waits
constexpr uint32_t kStMmaWaitA = 1u << 8;
constexpr uint32_t kStMmaWaitB = 1u << 9;
constexpr uint32_t kStProdWait = 1u << 10;
constexpr uint32_t kStGenWait = 1u << 11;
constexpr uint32_t kStEpiWait = 1u << 12;

struct MmaArgs {
    const double* freqs;
    const float* dc;      // [2 * nseg] row sums (E rows, then V rows)
    const int* qexp;      // [2] power-of-two exponents of the FP16 staging (E, V)
    float* out;           // [nseg][nfreq][2][nbf] complex as interleaved floats
    uint32_t* status;
    uint64_t seglen;
    double tsamp;
    double t_ref;
    uint32_t nfreq;
    uint32_t nseg;
    uint32_t nbf;
    uint32_t H;           // harmonics m = 1 .. H per frequency
    uint32_t fpt;         // frequencies per tile
    uint32_t ntile;       // MMA N (columns per subtile)
    uint32_t nsub;        // subtiles per block (1 or 2)
    uint32_t nk;          // K chunks of the segment
    uint32_t cpp;         // K chunks per part (a multiple of kAnchor); part z = blockIdx.z
    uint64_t part_stride; // floats between the parts' partial folds (0: one part)
    uint32_t tmem_cols;
};

__device__ __forceinline__ float2 unit_phasor(double u) {
    u -= floor(u);
    float s, c;
    sincospif(-2.0f * static_cast<float>(u), &s, &c);
    return make_float2(c, s);
}

__device__ __forceinline__ float2 cmul(float2 x, float2 p) {
    return make_float2(fmaf(x.x, p.x, -(x.y * p.y)), fmaf(x.x, p.y, x.y * p.x));
}

// Byte offset of 16-byte chunk c (0..3) of row r in a K-major tile of 64-byte
// rows with the 64-byte swizzle (8-row atoms of 512 bytes; chunk index XOR
// bits 1-2 of the row within the atom), the layout TMA writes for
// CU_TENSOR_MAP_SWIZZLE_64B and the MMA reads for layout type SWIZZLE_64B.
__device__ __forceinline__ uint32_t swz64(uint32_t r, uint32_t c) {
    return (r >> 3) * 512u + (r & 7u) * 64u + ((c ^ ((r & 7u) >> 1)) << 4);
}

// Shared-memory matrix descriptor (tcgen05): K-major, 64-byte swizzle,
// 512 bytes between 8-row groups.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(1u) << 16;              // leading byte offset (unused here)
    d |= static_cast<uint64_t>(512u >> 4) << 32;       // stride byte offset
    d |= static_cast<uint64_t>(1u) << 46;              // descriptor version (sm_100)
    d |= static_cast<uint64_t>(4u) << 61;              // SWIZZLE_64B
    return d;
}

// Instruction descriptor: FP16 A and B, FP32 D, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t n) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((n >> 3) << 17) | ((kRows >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     ptx::smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

// FP16 hi / lo halves of two floats packed as half2 pairs.
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

__global__ void __launch_bounds__(kThreads, 1)
fourier_dft_mma_kernel(const __grid_constant__ CUtensorMap map_hi,
                       const __grid_constant__ CUtensorMap map_lo, MmaArgs a) {
    extern __shared__ uint8_t smem_raw[];
    // base 1024-byte aligned in the shared window: stages of [A_hi | A_lo | B_hi | B_lo]
    uint8_t* base = smem_raw + ((1024u - (ptx::smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t bbytes = a.nsub * a.ntile * kRowBytes;  // one of B_hi / B_lo
    const uint32_t stage_bytes = 2 * kATileBytes + 2 * bbytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * stage_bytes);
    uint64_t* full_a = bars;                 // [kStages]
    uint64_t* full_b = bars + kStages;       // [kStages]
    uint64_t* empty = bars + 2 * kStages;    // [kStages]
    uint64_t* done = bars + 3 * kStages;     // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * kStages + 1);

    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;
    auto a_hi = [&](uint32_t s) { return base + s * stage_bytes; };
    auto a_lo = [&](uint32_t s) { return base + s * stage_bytes + kATileBytes; };
    auto b_hi = [&](uint32_t s) { return base + s * stage_bytes + 2 * kATileBytes; };
    auto b_lo = [&](uint32_t s) { return base + s * stage_bytes + 2 * kATileBytes + bbytes; };

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kStages; ++s) {
            ptx::mbar_init(&full_a[s], kGenThreads);
            ptx::mbar_init(&full_b[s], 1);
            ptx::mbar_init(&empty[s], 1);
        }
        ptx::mbar_init(done, 1);
        ptx::fence_barrier_init();
        ptx::prefetch_tensormap(&map_hi);
        ptx::prefetch_tensormap(&map_lo);
    }
    if (warp == 1) {
        ptx::tmem_alloc(tmem_slot, a.tmem_cols);
        ptx::tmem_relinquish();
    }
    ptx::tmem_fence_before_sync();
    __syncthreads();
    ptx::tmem_fence_after_sync();
    const uint32_t tbase = *tmem_slot;

    const uint32_t mt = blockIdx.x;                      // frequency tile
    const uint32_t col0 = blockIdx.y * a.nsub * a.ntile; // first B row of this block
    // K part of this block: chunks [it0, it0 + nloc); each part sums into its
    // own partial fold, so no accumulator sums more than cpp chunks
    const uint32_t it0 = blockIdx.z * a.cpp;
    const uint32_t nloc = min(a.cpp, a.nk - it0);
    float* const out = a.out + blockIdx.z * a.part_stride;

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            const uint32_t tx = 2 * bbytes;
            uint32_t issued = 0;
            for (uint32_t li = 0; li < nloc; ++li) {
                const uint32_t it = it0 + li;
                const uint32_t s = li % kStages;
                if (li >= kStages &&
                    !ptx::mbar_wait_bounded(&empty[s], ((li / kStages) - 1) & 1, a.status, kStProdWait)) {
                    break;
                }
                ptx::mbar_arrive_expect_tx(&full_b[s], tx);
                for (uint32_t sub = 0; sub < a.nsub; ++sub) {
                    const int x = static_cast<int>(it * kKc);
                    const int y = static_cast<int>(col0 + sub * a.ntile);
                    ptx::tma_load_2d(b_hi(s) + sub * a.ntile * kRowBytes, &map_hi, &full_b[s], x, y);
                    ptx::tma_load_2d(b_lo(s) + sub * a.ntile * kRowBytes, &map_lo, &full_b[s], x, y);
                }
                issued = li + 1;
            }
            // the copies of the last stages land before the block can exit
            for (uint32_t li = (issued > kStages ? issued - kStages : 0); li < issued; ++li) {
                ptx::mbar_wait_bounded(&full_b[li % kStages], (li / kStages) & 1, a.status, kStProdWait);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = idesc_f16(a.ntile);
            for (uint32_t li = 0; li < nloc; ++li) {
                const uint32_t s = li % kStages;
                const uint32_t par = (li / kStages) & 1;
                if (!ptx::mbar_wait_bounded(&full_a[s], par, a.status, kStMmaWaitA) ||
                    !ptx::mbar_wait_bounded(&full_b[s], par, a.status, kStMmaWaitB)) {
                    break;
                }
                ptx::tmem_fence_after_sync();
                const uint32_t ah = ptx::smem_u32(a_hi(s)), al = ptx::smem_u32(a_lo(s));
                const uint32_t bh = ptx::smem_u32(b_hi(s)), bl = ptx::smem_u32(b_lo(s));
                for (uint32_t sub = 0; sub < a.nsub; ++sub) {
                    const uint32_t d = tbase + sub * a.ntile;
                    const uint32_t boff = sub * a.ntile * kRowBytes;
#pragma unroll
                    for (uint32_t kk = 0; kk < kKc / 16; ++kk) {
                        const uint32_t acc = (li > 0 || kk > 0) ? 1u : 0u;
                        mma_f16(d, sdesc(ah + 32 * kk), sdesc(bh + boff + 32 * kk), idesc, acc);
                        mma_f16(d, sdesc(ah + 32 * kk), sdesc(bl + boff + 32 * kk), idesc, 1u);
                        mma_f16(d, sdesc(al + 32 * kk), sdesc(bh + boff + 32 * kk), idesc, 1u);
                    }
                }
                mma_commit(&empty[s]);
            }
            mma_commit(done);
        }
    } else {
        // ---- A generation (warps 2-5), then the epilogue ----
        const uint32_t g = threadIdx.x - 64;
        const uint32_t p = g >> 1;        // (frequency, harmonic) pair: rows 2p (re), 2p + 1 (im)
        const uint32_t h = g & 1;         // samples 16h .. 16h + 15 of each chunk
        const uint32_t fi = p / a.H;
        const uint32_t m = 1 + p % a.H;
        const uint32_t f = mt * a.fpt + fi;
        const bool valid = fi < a.fpt && f < a.nfreq;
        const double freq = valid ? a.freqs[f] : 0.0;
        double ustep = freq * a.tsamp;
        ustep -= floor(ustep);
        const float2 w1 = unit_phasor(static_cast<double>(m) * ustep);
        const float2 w32 = unit_phasor(static_cast<double>(m) * ustep * static_cast<double>(kKc));
        float2 start = make_float2(1.0f, 0.0f);
        for (uint32_t li = 0; li < nloc; ++li) {
            const uint32_t it = it0 + li;
            const uint32_t s = li % kStages;
            if (li >= kStages &&
                !ptx::mbar_wait_bounded(&empty[s], ((li / kStages) - 1) & 1, a.status, kStGenWait)) {
                break;
            }
            const uint64_t k0 = static_cast<uint64_t>(it) * kKc + 16 * h;
            if (it % kAnchor == 0) {
                double u = freq * (static_cast<double>(k0) * a.tsamp - a.t_ref);
                u -= floor(u);
                start = unit_phasor(static_cast<double>(m) * u);
            } else {
                start = cmul(start, w32);
            }
            uint32_t re_hi[8], re_lo[8], im_hi[8], im_lo[8];
            float2 ph = start;
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                const float2 p0 = ph;
                const float2 p1 = cmul(p0, w1);
                ph = cmul(p1, w1);
                if (valid) {
                    split2(p0.x, p1.x, re_hi[j], re_lo[j]);
                    split2(p0.y, p1.y, im_hi[j], im_lo[j]);
                } else {
                    re_hi[j] = re_lo[j] = im_hi[j] = im_lo[j] = 0u;
                }
            }
            const uint32_t rre = 2 * p, rim = 2 * p + 1;
#pragma unroll
            for (uint32_t c = 0; c < 2; ++c) {
                const uint32_t ch = 2 * h + c;
                *reinterpret_cast<uint4*>(a_hi(s) + swz64(rre, ch)) =
                    make_uint4(re_hi[4 * c], re_hi[4 * c + 1], re_hi[4 * c + 2], re_hi[4 * c + 3]);
                *reinterpret_cast<uint4*>(a_lo(s) + swz64(rre, ch)) =
                    make_uint4(re_lo[4 * c], re_lo[4 * c + 1], re_lo[4 * c + 2], re_lo[4 * c + 3]);
                *reinterpret_cast<uint4*>(a_hi(s) + swz64(rim, ch)) =
                    make_uint4(im_hi[4 * c], im_hi[4 * c + 1], im_hi[4 * c + 2], im_hi[4 * c + 3]);
                *reinterpret_cast<uint4*>(a_lo(s) + swz64(rim, ch)) =
                    make_uint4(im_lo[4 * c], im_lo[4 * c + 1], im_lo[4 * c + 2], im_lo[4 * c + 3]);
            }
            fence_proxy_async_smem();
            ptx::mbar_arrive(&full_a[s]);
        }
        // ---- epilogue: tensor memory -> complex fold ----
        const bool got = ptx::mbar_wait_bounded(done, 0, a.status, kStEpiWait);
        ptx::tmem_fence_after_sync();
        if (got) {
            const uint32_t q = warp & 3;              // TMEM lane quadrant of this warp
            const uint32_t r = 32 * q + lane;         // tile row
            const uint32_t efi = r / (2 * a.H);
            const uint32_t within = r - efi * 2 * a.H;
            const uint32_t em = 1 + within / 2;
            const uint32_t ec = within & 1;
            const uint32_t ef = mt * a.fpt + efi;
            const bool evalid = efi < a.fpt && ef < a.nfreq;
            const float scale_e = __int_as_float((127 - a.qexp[0]) << 23);
            const float scale_v = __int_as_float((127 - a.qexp[1]) << 23);
            const uint32_t nrows = 2 * a.nseg;
            for (uint32_t sub = 0; sub < a.nsub; ++sub) {
                for (uint32_t cb = 0; cb < a.ntile; cb += 32) {
                    float v[32];
                    tmem_ld32(tbase + ((32 * q) << 16) + sub * a.ntile + cb, v);
                    if (!evalid) {
                        continue;
                    }
#pragma unroll
                    for (uint32_t j = 0; j < 32; ++j) {
                        const uint32_t n = col0 + sub * a.ntile + cb + j;
                        if (n < nrows) {
                            const uint32_t ev = n >= a.nseg ? 1u : 0u;
                            const uint64_t sg = n - ev * a.nseg;
                            const uint64_t row = ((sg * a.nfreq + ef) * 2 + ev) * a.nbf;
                            out[(row + em) * 2 + ec] = v[j] * (ev ? scale_v : scale_e);
                            if (em == 1 && ec == 0) {
                                out[row * 2] = blockIdx.z == 0 ? a.dc[n] : 0.0f;
                                out[row * 2 + 1] = 0.0f;
                            }
                        }
                    }
                }
            }
        }
    }
    ptx::tmem_fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        ptx::tmem_dealloc(tbase, a.tmem_cols);
    }
}

// Largest |x| of E and V over the folded samples, as float bits (non-negative
// floats order as unsigned integers).
__global__ void absmax_kernel(const float* __restrict__ e, const float* __restrict__ v, uint64_t n,
                              uint32_t* __restrict__ out) {
    float me = 0.0f, mv = 0.0f;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        me = fmaxf(me, fabsf(__ldg(e + i)));
        mv = fmaxf(mv, fabsf(__ldg(v + i)));
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1) {
        me = fmaxf(me, __shfl_xor_sync(0xffffffffu, me, o));
        mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, __float_as_uint(me));
        atomicMax(out + 1, __float_as_uint(mv));
    }
}

// Exponent q with max |x| 2^q in [2^13, 2^14): the FP16 halves keep their
// range with room to spare.
__device__ __forceinline__ int stage_exponent(uint32_t maxbits) {
    const float mx = __uint_as_float(maxbits);
    if (!(mx > 0.0f) || !isfinite(mx)) {
        return 0;
    }
    int e = 0;
    frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1)
    return min(max(14 - e, -100), 100);
}

// Row b of [2 nseg][L] (E rows then V rows): FP16 hi / lo of x 2^q, and the
// row's FP32 sum. One block per row.
__global__ void __launch_bounds__(256)
stage_rows_kernel(const float* __restrict__ e, const float* __restrict__ v, uint64_t seglen,
                  uint32_t nseg, const uint32_t* __restrict__ maxbits, __half* __restrict__ hi,
                  __half* __restrict__ lo, float* __restrict__ dc, int* __restrict__ qexp) {
    __shared__ float part[8];
    const uint32_t row = blockIdx.x;
    const uint32_t ev = row >= nseg ? 1 : 0;
    const uint64_t s = row - ev * nseg;
    const float* x = (ev ? v : e) + s * seglen;
    const int q = stage_exponent(maxbits[ev]);
    if (blockIdx.x == 0 && threadIdx.x < 2) {
        qexp[threadIdx.x] = stage_exponent(maxbits[threadIdx.x]);
    }
    const float sc = ldexpf(1.0f, q);
    float sum = 0.0f;
    __half* oh = hi + static_cast<uint64_t>(row) * seglen;
    __half* ol = lo + static_cast<uint64_t>(row) * seglen;
    for (uint64_t k = threadIdx.x; k < seglen; k += blockDim.x) {
        const float xv = __ldg(x + k);
        sum += xv;
        const float xs = xv * sc;
        const __half h = __float2half_rn(xs);
        oh[k] = h;
        ol[k] = __float2half_rn(xs - __half2float(h));
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (uint32_t i = 0; i < blockDim.x / 32; ++i) {
            t += part[i];
        }
        dc[row] = t;
    }
}

// out[i] = sum over the parts of part[p][i], in part order (FP32).
__global__ void sum_parts_kernel(const float4* __restrict__ parts, uint64_t n4, uint32_t nparts,
                                 float4* __restrict__ out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float4 acc = __ldg(parts + i);
        for (uint32_t p = 1; p < nparts; ++p) {
            const float4 x = __ldg(parts + p * n4 + i);
            acc.x += x.x;
            acc.y += x.y;
            acc.z += x.z;
            acc.w += x.w;
        }
        out[i] = acc;
    }
}

}  // namespace

bool fourier_mma_supported(uint64_t seglen, uint64_t nseg, uint32_t nbins) {
    const uint32_t H = (nbins / 2 + 1) - 1;
    return H >= 1 && 2 * H <= kRows && seglen % 8 == 0 && seglen >= kKc && nseg >= 1 &&
           2 * nseg < (1ull << 31) && seglen < (1ull << 31);
}

FourierMma::FourierMma(uint64_t seglen_, uint64_t nseg_, uint32_t nbins_, uint32_t nfreq_,
                       uint32_t max_sub, uint32_t part_chunks)
    : seglen(seglen_), nseg(nseg_), nbins(nbins_), nfreq(nfreq_) {
    require(fourier_mma_supported(seglen, nseg, nbins), "tensor-core transform: unsupported shape");
    require(max_sub == 1 || max_sub == 2, "tensor-core transform: subtiles per block must be 1 or 2");
    require(part_chunks >= kAnchor && part_chunks % kAnchor == 0,
            "tensor-core transform: K part length must be a multiple of 256 samples");
    const uint64_t rows = 2 * nseg;
    hi.alloc(sizeof(__half) * rows * seglen);
    lo.alloc(sizeof(__half) * rows * seglen);
    dc.alloc(sizeof(float) * rows);
    aux.alloc(16);  // [0, 2): max bits, [2, 4): exponents
    if (rows <= kMaxN) {
        nsub = 1;
        ntile = static_cast<uint32_t>((rows + 15) / 16 * 16);
    } else {
        nsub = max_sub;
        ntile = kMaxN;
    }
    ngroups = static_cast<uint32_t>((rows + nsub * ntile - 1) / (nsub * ntile));
    require(ngroups <= 65535, "tensor-core transform: too many segments");
    tmem_cols = 32;
    while (tmem_cols < nsub * ntile) {
        tmem_cols *= 2;
    }
    // K parts of at most kPartChunks chunks each (anchored starts): shorter
    // accumulation chains in tensor memory, and more blocks per wave
    const uint32_t nk = static_cast<uint32_t>((seglen + kKc - 1) / kKc);
    const uint32_t want = std::min<uint32_t>(kMaxParts, (nk + part_chunks - 1) / part_chunks);
    cpp = (nk + want - 1) / want;
    cpp = (cpp + kAnchor - 1) / kAnchor * kAnchor;
    nparts = (nk + cpp - 1) / cpp;
    if (nparts > 1) {
        const uint64_t elems = 2 * nseg * nfreq * 2 * static_cast<uint64_t>(nbins / 2 + 1);  // floats
        parts.alloc(sizeof(float) * elems * nparts);
    }
    auto encode = [&](CUtensorMap* map, void* ptr) {
        cuuint64_t dims[2] = {seglen, rows};
        cuuint64_t strides[1] = {seglen * sizeof(__half)};
        cuuint32_t box[2] = {kKc, ntile};
        cuuint32_t estr[2] = {1, 1};
        const CUresult r = tensor_map_encoder()(
            map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, ptr, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled failed for the staged series");
        }
    };
    encode(&map_hi, hi.ptr);
    encode(&map_lo, lo.ptr);
    smem_bytes = kStages * (2 * kATileBytes + 2 * nsub * ntile * kRowBytes) + 1024 + 128;
    require(smem_bytes <= 227 * 1024, "tensor-core transform: shared memory");
}

uint64_t FourierMma::device_bytes() const {
    return hi.bytes + lo.bytes + dc.bytes + aux.bytes + parts.bytes;
}

void FourierMma::run(const float* d_ts_e, const float* d_ts_v, const double* d_freqs, double tsamp,
                     double t_ref, float2* d_out, uint32_t* d_status, cudaStream_t s) {
    const uint64_t nused = nseg * seglen;
    uint32_t* maxbits = aux.as<uint32_t>();
    int* qexp = reinterpret_cast<int*>(aux.as<uint32_t>() + 2);
    LK_CUDA(cudaMemsetAsync(maxbits, 0, 2 * sizeof(uint32_t), s));
    absmax_kernel<<<std::min<uint64_t>((nused + 255) / 256, 148 * 8), 256, 0, s>>>(d_ts_e, d_ts_v, nused,
                                                                                 maxbits);
    LK_CUDA(cudaGetLastError());
    stage_rows_kernel<<<static_cast<uint32_t>(2 * nseg), 256, 0, s>>>(
        d_ts_e, d_ts_v, seglen, static_cast<uint32_t>(nseg), maxbits, hi.as<__half>(), lo.as<__half>(),
        dc.as<float>(), qexp);
    LK_CUDA(cudaGetLastError());
    MmaArgs a{};
    const uint64_t elems = 2 * nseg * static_cast<uint64_t>(nfreq) * 2 * (nbins / 2 + 1);  // floats
    a.freqs = d_freqs;
    a.dc = dc.as<float>();
    a.qexp = qexp;
    a.out = nparts > 1 ? parts.as<float>() : reinterpret_cast<float*>(d_out);
    a.part_stride = nparts > 1 ? elems : 0;
    a.status = d_status;
    a.seglen = seglen;
    a.tsamp = tsamp;
    a.t_ref = t_ref;
    a.nfreq = nfreq;
    a.nseg = static_cast<uint32_t>(nseg);
    a.nbf = nbins / 2 + 1;
    a.H = a.nbf - 1;
    a.fpt = kRows / (2 * a.H);
    a.ntile = ntile;
    a.nsub = nsub;
    a.nk = static_cast<uint32_t>((seglen + kKc - 1) / kKc);
    a.cpp = cpp;
    a.tmem_cols = tmem_cols;
    const uint32_t mtiles = (nfreq + a.fpt - 1) / a.fpt;
    // the kernel's shared-memory limit is per function, and executors of
    // other shapes set it too: set it for this launch
    LK_CUDA(cudaFuncSetAttribute(fourier_dft_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_bytes)));
    fourier_dft_mma_kernel<<<dim3(mtiles, ngroups, nparts), kThreads, smem_bytes, s>>>(map_hi, map_lo, a);
    LK_CUDA(cudaGetLastError());
    if (nparts > 1) {
        const uint64_t n4 = elems / 4;  // elems = 4 * (...) floats
        sum_parts_kernel<<<static_cast<uint32_t>(std::min<uint64_t>((n4 + 255) / 256, 148 * 16)), 256, 0, s>>>(
            parts.as<float4>(), n4, nparts, reinterpret_cast<float4*>(d_out));
        LK_CUDA(cudaGetLastError());
    }
}

}  // namespace lk
