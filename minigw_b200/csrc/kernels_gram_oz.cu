// kernels_gram_oz.cu -- the refined mixed form's FP64 Gram term y^T V y = ||C^T y||^2 on the int8
// tensor cores (tcgen05 kind::i8), exact integer products of digit slices.
//
// V = C C^T (pivoted Cholesky, kernels_refine.cu) with C^T r x n.  For every frequency f and right-
// hand side j the correction needs t3 = sum_k (C^T y_j)_k^2 to FP64 accuracy: a GEMM G = C^T Y
// (r x m per frequency, K = n) reduced by squares over k.  Here the operands are cut into balanced
// digits in [-64, 64] (each the nearest integer to the scaled remainder) with one power-of-two scale
// 2^{e} > 2 max|row| per row:
//     C^T[k][i] = 2^{e_k} sum_{s=1..7} A_s[k][i] 2^{-7s} + (|.| <= 2^{e_k - 50})
//     y_j[i]    = 2^{e_j} sum_{t=1..4} B_t[j][i] 2^{-7t}          (y rounded to 28 bits)
// so that G[k][j] = 2^{e_k + e_j} sum_{l=2..9} 2^{-7l} S_l[k][j],  S_l = sum_{s+t=l} A_s . B_t,
// dropping only s + t > 9 (products below 2^{-58} of the row scales, of either sign).  Each S_l is an
// exact int32 sum over the whole K (at most four (s, t) pairs per level: |S_l| <= 4 * 64^2 * nk <
// 2^31 for nk <= 65536, the K extent this path accepts), accumulated by 25 int8 tensor-core
// products per 32-deep K step in 8 TMEM accumulators of 64 columns (the whole 512).
//
// G sums n products of partly cancelling terms, so its error is set by the digits' error relative
// to the row scale: truncated digits (a one-sided error of up to 2^-49) left the forms 1e-12 away
// from the FP64 Gram on n = 336 and n = 500 (1.6e-10 Ha in Sigma_c on n = 2000); rounded digits and
// the ninth level bring them to the FP64 product's own rounding level.
//
// Rounding y is nearly free: the refined form evaluates the energy functional F(z) = 2 b^T z -
// z^T eps z, which is stationary at the solution, so a perturbation dz changes F by dz^T eps dz
// only; what matters is that t1 = x^T y, t2 = z^T z and t3 = y^T V y all use the same rounded y
// (k_refine_prep_oz computes t1 and t2 from the values it slices).  The rounding is absolute
// (2^{e_j - 29} per element) and z = y / D^1/2 magnifies it where D is small: 3 digits (21 bits)
// left 1e-11 relative in the forms, 4 digits are at the FP64 level.
//
// k_gram_oz: one CTA per (frequency, 128-row tile of C^T, 64 right-hand sides); warp 0 streams
// the B slices of a 128-deep K chunk (4 x 8 KB, double-buffered) and the A slices (16 KB each)
// through an 8-stage ring with bulk copies; warp 1 allocates TMEM (512 columns) and its lane 0
// issues the MMAs; warps 2-5 read the 8 levels of their 32-row quadrant (warp % 4), form G in FP64, square,
// and sum each column over the rows (fixed shuffle tree, then the four quadrants in order): one
// partial sum per (frequency, row tile, j), summed over row tiles by k_refine_finish.  Every
// mbarrier wait is bounded (tc_common.cuh: expiry -> pivot 0 -> GWB200_DEVICE_TIMEOUT).
#include "internal.cuh"
#include "tc_common.cuh"

namespace gwb200 {
namespace {

using namespace tc;

constexpr int kGM = 128;                      // C^T rows per tile (TMEM lanes)
constexpr int kGN = 64;                       // right-hand sides per tile (accumulator columns per level)
constexpr int kASl = 7, kBSl = 4, kLevels = 8;  // levels l = 2 .. kLevels + 1
constexpr int64_t kMaxNk = 65536;                 // 4 pairs * 64^2 * kMaxNk = 2^30
constexpr int kKc = 128;                      // K bytes per chunk (one 128-byte swizzled row)
constexpr int kSliceA = kGM * kKc;            // 16 KB
constexpr int kSliceB = kGN * kKc;            // 8 KB
constexpr int kAStages = 8;
constexpr int kHdr = 1024;
constexpr int kGramSmem = kHdr + 1024 + 2 * kBSl * kSliceB + kAStages * kSliceA + 4 * kGN * 8;
constexpr int kGramThreads = 32 * 6;

constexpr int kOffAF = 0, kOffAE = kOffAF + 8 * kAStages, kOffBF = kOffAE + 8 * kAStages, kOffBE = kOffBF + 16,
              kOffTF = kOffBE + 16, kOffDrain = kOffTF + 8, kOffTmem = kOffDrain + 8, kOffAbort = kOffTmem + 4;
static_assert(kOffAbort + 4 <= kHdr, "header");
static_assert(kGramSmem <= 227 * 1024, "shared memory");
static_assert(kLevels * kGN <= 512, "TMEM columns");

// kind::i8: D S32, A and B signed 8-bit, K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kGN >> 3) << 17) | ((uint32_t)(kGM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ double pow2i(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// Byte offset of element (row, k) of a 128-byte-swizzled K-major slice of one 128-deep K chunk.
__device__ __forceinline__ size_t swz(int64_t row, int k) {
    const int chunk = k >> 4, in = k & 15;
    return (size_t)row * kKc + (size_t)(((chunk ^ (int)(row & 7)) << 4) + in);
}

// Next balanced digit of v (|v| <= 1/2 in units of the current digit): rint(128 v) in [-64, 64],
// v <- 128 v - digit, again |v| <= 1/2.  Exact in FP64.
__device__ __forceinline__ int next_digit(double& v) {
    const double t = v * 128.0;
    const double d = rint(t);
    v = t - d;
    return (int)d;
}

// C^T (r x n_pad FP64, row stride n_pad) into 7 digit slices over nk = n_pad rounded up to 128 (zero
// beyond n_pad and from row r), layout [kc][s][row < r128][128 B], one exponent e per row with
// max|row| < 2^{e-1}.  One warp per row.
__global__ void __launch_bounds__(256) k_slice_ct(const double* __restrict__ ct, int64_t r, int64_t n_pad, int64_t nk,
                                                  int64_t r128, uint8_t* __restrict__ out, int32_t* __restrict__ exps) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * 8 + warp;
    if (row >= r128) return;
    const double* src = ct + (size_t)row * n_pad;
    double m = 0.0;
    if (row < r)
        for (int64_t i = lane; i < n_pad; i += 32) m = fmax(m, fabs(src[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    if (m > 0.0) frexp(m, &e);  // |x| < 2^e
    ++e;                        // |x| < 2^{e-1}
    const double inv = pow2i(-e);
    const int64_t nkc = nk / kKc;
    for (int64_t kc = 0; kc < nkc; ++kc) {
        const int k0 = lane * 4;  // four consecutive K bytes per lane
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t i = kc * kKc + k0 + q;
            v[q] = (row < r && i < n_pad) ? src[i] * inv : 0.0;  // |v| < 1/2, exact
        }
#pragma unroll
        for (int s = 0; s < kASl; ++s) {
            uint32_t word = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) word |= ((uint32_t)next_digit(v[q]) & 0xFFu) << (8 * q);
            *reinterpret_cast<uint32_t*>(out + ((size_t)(kc * kASl + s) * r128) * kKc + swz(row, k0)) = word;
        }
    }
    if (lane == 0) exps[row] = e;
}

// One CTA per right-hand side j of one frequency (k_refine_prep's inputs): y_j = dvec * z_j in FP64,
// rounded to kBSl balanced digits below its row scale; the digits into B slices [kc][t][j][128 B] of
// the frequency, the exponent into yexp; t1 = x_j . y^ and t2 = z^ . z^ (z^ = y^ / dvec) from the
// rounded values (fixed-order sums).  The grid's x index is the frequency, so that the CTAs in flight
// together share j and its row of xt (read from DRAM once, not once per frequency).
constexpr int64_t kPrepMaxNpad = 25600;  // y staged in shared memory: 8 n_pad bytes <= 200 KB
constexpr int kPrepThreads = 256;        // 8 warps: the block reductions keep one value per warp

__global__ void __launch_bounds__(kPrepThreads) k_refine_prep_oz(const float* __restrict__ a, int64_t ld, int64_t stride,
                                                        int64_t row0, int64_t na, int64_t n, int64_t n_pad, int64_t nk,
                                                        int64_t m, int64_t m_pad, const double* __restrict__ xt,
                                                        const double* __restrict__ dvec, uint8_t* __restrict__ yslices,
                                                        size_t fbytes, int32_t* __restrict__ yexp,
                                                        double* __restrict__ t12) {
    extern __shared__ double yrow[];  // n_pad
    __shared__ double r1[kPrepThreads / 32], r2[kPrepThreads / 32], rm[kPrepThreads / 32];  // one value per warp
    const int f = blockIdx.x;
    const int64_t j = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float* row = a + (size_t)f * stride + (size_t)(row0 + j) * ld;
    const double* d = dvec + (size_t)f * n_pad;
    const bool live = j < m;
    double mx = 0.0;
    for (int64_t i = threadIdx.x; i < n_pad; i += blockDim.x) {
        const double yi = (live && i < n) ? d[i] * (double)row[na - 1 - i] : 0.0;
        yrow[i] = yi;
        mx = fmax(mx, fabs(yi));
    }
    // block maximum: shuffle tree per warp, then the 8 warp values (two barriers)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) rm[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = rm[0];
        for (int w = 1; w < kPrepThreads / 32; ++w) v = fmax(v, rm[w]);
        rm[0] = v;
    }
    __syncthreads();
    int e = 0;
    if (rm[0] > 0.0) frexp(rm[0], &e);
    ++e;  // |y| < 2^{e-1}
    const double inv = pow2i(-e), scale = pow2i(e);
    uint8_t* out = yslices + (size_t)f * fbytes;
    double s1 = 0.0, s2 = 0.0;
    for (int64_t w4 = threadIdx.x; w4 < nk / 4; w4 += blockDim.x) {  // 4 consecutive elements per word
        const int64_t i0 = w4 * 4, kc = i0 / kKc;
        const int kb = (int)(i0 % kKc);
        uint32_t word[kBSl] = {};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t i = i0 + q;
            double v = i < n_pad ? yrow[i] * inv : 0.0;  // |v| < 1/2, exact
            double rec = 0.0;          // the rounded value, in units of the last digit
#pragma unroll
            for (int t = 0; t < kBSl; ++t) {
                const int dg = next_digit(v);
                rec = fma(rec, 128.0, (double)dg);  // exact: |rec| < 2^{7 kBSl}
                word[t] |= ((uint32_t)dg & 0xFFu) << (8 * q);
            }
            if (live && i < n) {
                const double yh = rec * pow2i(-7 * kBSl) * scale;  // exact
                const double zh = yh / d[i];
                s1 = fma(xt[j * n + i], yh, s1);
                s2 = fma(zh, zh, s2);
            }
        }
#pragma unroll
        for (int t = 0; t < kBSl; ++t)
            *reinterpret_cast<uint32_t*>(out + ((size_t)(kc * kBSl + t) * m_pad) * kKc + swz(j, kb)) = word[t];
    }
    // block sums in a fixed order: shuffle tree per warp, then the 8 warp sums in warp order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        r1[warp] = s1;
        r2[warp] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double u1 = r1[0], u2 = r2[0];
        for (int w = 1; w < kPrepThreads / 32; ++w) {
            u1 += r1[w];
            u2 += r2[w];
        }
        t12[((size_t)f * m_pad + j) * 2] = u1;
        t12[((size_t)f * m_pad + j) * 2 + 1] = u2;
        yexp[(size_t)f * m_pad + j] = e;
    }
}

// part[f][it][jt*64 + c] = sum over the tile's 128 rows k of G[k][j]^2.
__global__ void __launch_bounds__(kGramThreads, 1)
    k_gram_oz(const uint8_t* __restrict__ aslices, const int32_t* __restrict__ aexp, int64_t r128,
              const uint8_t* __restrict__ yslices, size_t fbytes, const int32_t* __restrict__ yexp, int64_t m_pad,
              int64_t nkc, double* __restrict__ part, unsigned long long* err) {
    extern __shared__ __align__(1024) uint8_t gsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t jt = blockIdx.x, it = blockIdx.y, f = blockIdx.z;
    const uint32_t base = smem_u32(gsm);
    const uint32_t bbuf = (base + kHdr + 1023u) & ~1023u;   // 2 x kBSl B slices
    const uint32_t aring = bbuf + 2 * kBSl * kSliceB;        // A stages
    double* red = reinterpret_cast<double*>(gsm + (aring - base) + kAStages * kSliceA);  // 4 x 64
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(gsm + kOffAbort);
    auto af = [&](int s) { return base + kOffAF + 8 * s; };
    auto ae = [&](int s) { return base + kOffAE + 8 * s; };
    auto bf = [&](int b) { return base + kOffBF + 8 * b; };
    auto be = [&](int b) { return base + kOffBE + 8 * b; };
    const uint32_t tfull = base + kOffTF, drain = base + kOffDrain;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kAStages; ++s) {
            mbar_init(af(s), 1);
            mbar_init(ae(s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(bf(b), 1);
            mbar_init(be(b), 1);
        }
        mbar_init(tfull, 1);
        mbar_init(drain, 1);
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kOffTmem), "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(gsm + kOffTmem);
    const uint8_t* ysl = yslices + (size_t)f * fbytes;

    if (warp == 0) {
        // ---- producer ----
        if (lane == 0) {
            int sa = 0;
            uint32_t pa = 0;
            bool ok = true;
            uint32_t filled_a = 0, par_a = 0, filled_b = 0, par_b = 0;
            for (int64_t kc = 0; ok && kc < nkc; ++kc) {
                const int b = (int)(kc & 1);
                const uint32_t pb = (uint32_t)((kc >> 1) & 1);
                if (!mbar_wait(be(b), pb ^ 1u, abort_flag, err)) break;
                mbar_expect_tx(bf(b), (uint32_t)(kBSl * kSliceB));
                for (int t = 0; t < kBSl; ++t)
                    bulk_g2s(bbuf + (uint32_t)((b * kBSl + t) * kSliceB),
                             ysl + ((size_t)(kc * kBSl + t) * m_pad + (size_t)jt * kGN) * kKc, kSliceB, bf(b));
                filled_b |= 1u << b;
                par_b = (par_b & ~(1u << b)) | (pb << b);
                for (int s = 0; s < kASl; ++s) {
                    if (!mbar_wait(ae(sa), pa ^ 1u, abort_flag, err)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(af(sa), (uint32_t)kSliceA);
                    bulk_g2s(aring + (uint32_t)(sa * kSliceA),
                             aslices + ((size_t)(kc * kASl + s) * r128 + (size_t)it * kGM) * kKc, kSliceA, af(sa));
                    filled_a |= 1u << sa;
                    par_a = (par_a & ~(1u << sa)) | (pa << sa);
                    if (++sa == kAStages) {
                        sa = 0;
                        pa ^= 1u;
                    }
                }
            }
            // drain this thread's copies before exit (bounded)
            for (int q = 0; q < kAStages; ++q)
                if (filled_a & (1u << q)) mbar_drain(af(q), (par_a >> q) & 1u);
            for (int q = 0; q < 2; ++q)
                if (filled_b & (1u << q)) mbar_drain(bf(q), (par_b >> q) & 1u);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            int sa = 0;
            uint32_t pa = 0, started = 0;
            bool ok = true, issued = false;
            const uint64_t da0 = smem_desc_sw128(aring), db0 = smem_desc_sw128(bbuf);
            for (int64_t kc = 0; ok && kc < nkc; ++kc) {
                const int b = (int)(kc & 1);
                const uint32_t pb = (uint32_t)((kc >> 1) & 1);
                if (!mbar_wait_fast(bf(b), pb, abort_flag, err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int s = 0; s < kASl; ++s) {  // A slice s+1 against B slices 1 .. min(kBSl, kLevels - s)
                    if (!mbar_wait_fast(af(sa), pa, abort_flag, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t da = da0 + (uint64_t)((uint32_t)(sa * kSliceA) >> 4);
                    for (int t = 0; t < kBSl && s + t <= kLevels - 1; ++t) {
                        const int lvl = s + t;  // level l = (s+1) + (t+1), accumulator l - 2
                        const uint32_t d = tmem + (uint32_t)(lvl * kGN);
                        const uint64_t db = db0 + (uint64_t)((uint32_t)((b * kBSl + t) * kSliceB) >> 4);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            const uint32_t acc = ((started >> lvl) & 1u) ? 1u : 0u;
                            mma_i8(d, da + (uint64_t)(2 * kk), db + (uint64_t)(2 * kk), acc);
                            started |= 1u << lvl;
                        }
                        issued = true;
                    }
                    mma_commit(ae(sa));
                    if (++sa == kAStages) {
                        sa = 0;
                        pa ^= 1u;
                    }
                }
                if (ok) mma_commit(be(b));
            }
            if (ok) mma_commit(tfull);
            if (issued) {
                mma_commit(drain);
                mbar_drain(drain, 0);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: warps 2-5; a warp reads the TMEM lane quadrant warp % 4 ----
        const int q = warp & 3;
        bool ok = true;
        if (lane == 0) ok = mbar_wait(tfull, 0, abort_flag, err);
        ok = __shfl_sync(0xffffffffu, ok ? 1u : 0u, 0) != 0u;
        if (ok) {
            tc_fence_after();
            const int64_t krow = it * kGM + q * 32 + lane;
            const int ek = aexp[krow];
            constexpr int kHalf = kLevels / 2;
            for (int c16 = 0; c16 < kGN / 16; ++c16) {
                double g[16];  // sum_l S_l 2^{-7l}, smallest level first (each term exact)
                uint32_t v[kHalf][16];
#pragma unroll
                for (int h = 1; h >= 0; --h) {  // levels kHalf.. (the small ones), then 0..kHalf-1
#pragma unroll
                    for (int L = 0; L < kHalf; ++L)
                        tmem_ld16_nowait(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((h * kHalf + L) * kGN + 16 * c16),
                                         v[L]);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < 16; ++c) {
                        if (h == 1) g[c] = 0.0;
#pragma unroll
                        for (int L = kHalf - 1; L >= 0; --L)
                            g[c] += (double)(int32_t)v[L][c] * pow2i(-7 * (h * kHalf + L + 2));
                    }
                }
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int64_t jj = jt * kGN + 16 * c16 + c;
                    const int ej = yexp[(size_t)f * m_pad + jj];
                    const double gg = g[c] * pow2i(ek + ej);
                    double sq = gg * gg;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
                    if (lane == 0) red[q * kGN + 16 * c16 + c] = sq;
                }
            }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");  // the four epilogue warps
        if (q == 0) {
            for (int c = lane; c < kGN; c += 32) {
                const double s = (red[c] + red[kGN + c]) + (red[2 * kGN + c] + red[3 * kGN + c]);
                part[((size_t)f * (r128 / kGM) + it) * m_pad + jt * kGN + c] = ok ? s : 0.0;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

} // namespace

int64_t gram_oz_rows(int64_t r) { return std::max<int64_t>(kGM, round_up(r, kGM)); }

bool gram_oz_fits(int64_t n_pad) { return round_up(n_pad, kKc) <= kMaxNk && n_pad <= kPrepMaxNpad; }

size_t gram_oz_system_bytes(int64_t n_pad, int64_t r) {
    const int64_t r128 = gram_oz_rows(r), nk = round_up(n_pad, kKc);
    return (size_t)kASl * r128 * nk + sizeof(int32_t) * (size_t)r128;
}

void launch_slice_ct(const double* ct, int64_t r, int64_t n_pad, void* out, cudaStream_t s) {
    const int64_t r128 = gram_oz_rows(r), nk = round_up(n_pad, kKc);
    uint8_t* sl = static_cast<uint8_t*>(out);
    int32_t* ex = reinterpret_cast<int32_t*>(sl + (size_t)kASl * r128 * nk);
    k_slice_ct<<<(unsigned)(r128 / 8), 256, 0, s>>>(ct, r, n_pad, nk, r128, sl, ex);
    GWB_LAUNCH("k_slice_ct");
}

int launch_refine_terms_oz(const TallGeometry& ga, int64_t nf, const float* a, const TallGeometry& gm,
                           const double* xt, const double* dvec, const void* ct_slices, int64_t r, void* work,
                           unsigned long long* err, cudaStream_t s, double** t12_out, double** part_out,
                           int64_t* nkt_out) {
    const int64_t r128 = gram_oz_rows(r), n_pad = gm.n_pad, m_pad = gm.m_pad, nk = round_up(n_pad, kKc);
    const size_t fbytes = ((size_t)kBSl * m_pad * nk + 1023) / 1024 * 1024;
    uint8_t* ysl = static_cast<uint8_t*>(work);
    int32_t* yexp = reinterpret_cast<int32_t*>(ysl + fbytes * (size_t)nf);
    double* t12 = reinterpret_cast<double*>(yexp + ((size_t)nf * m_pad + 1) / 2 * 2);
    double* part = t12 + (size_t)nf * 2 * m_pad;
    const size_t prep_smem = sizeof(double) * (size_t)n_pad;
    GWB_CUDA(cudaFuncSetAttribute(k_refine_prep_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)prep_smem));
    if (m_pad > 65535) fail(GWB200_BAD_SHAPE, "refined form: more than 65535 right-hand sides per frequency");
    k_refine_prep_oz<<<dim3((unsigned)nf, (unsigned)m_pad), kPrepThreads, prep_smem, s>>>(
        a, ga.ld, ga.stride, ga.n_pad, gm.n_pad, gm.n, n_pad, nk, gm.m, m_pad, xt, dvec, ysl, fbytes, yexp, t12);
    GWB_LAUNCH("k_refine_prep_oz");
    const uint8_t* asl = static_cast<const uint8_t*>(ct_slices);
    const int32_t* aex = reinterpret_cast<const int32_t*>(asl + (size_t)kASl * r128 * nk);
    GWB_CUDA(cudaFuncSetAttribute(k_gram_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, kGramSmem));
    k_gram_oz<<<dim3((unsigned)(m_pad / kGN), (unsigned)(r128 / kGM), (unsigned)nf), kGramThreads, kGramSmem, s>>>(
        asl, aex, r128, ysl, fbytes, yexp, m_pad, nk / kKc, part, err);
    GWB_LAUNCH("k_gram_oz");
    *nkt_out = r128 / kGM;
    *t12_out = t12;
    *part_out = part;
    return 2;
}

size_t refine_oz_bytes_per_freq(const TallGeometry& g, int64_t r) {
    const size_t fbytes = ((size_t)kBSl * g.m_pad * round_up(g.n_pad, kKc) + 1023) / 1024 * 1024;
    return fbytes + sizeof(int32_t) * (size_t)g.m_pad + sizeof(double) * (2 * (size_t)g.m_pad +
                                                                          (size_t)(gram_oz_rows(r) / kGM) * g.m_pad) + 16;
}

} // namespace gwb200
