// kernels_oz.cu -- FP64 trailing update emulated on the int8 tensor cores (tcgen05 kind::i8).
//
// The plain form's dominant work is C -= P_r . P_c over the trailing lower part after each outer
// block of K = 128 columns (FP64; kernels_fp64.cu runs it on the FP64 DMMA pipe, 37 TFLOP/s
// peak).  Here each panel row P_r (128 values) is written as
//     P_r[k] = 2^e_r * sum_{s=1..6} D_s[r][k] 2^{-7 s} + (remainder of at most 2^{e_r - 43}),
// with 2^{e_r - 1} the smallest power of two above max_k |P_r[k]| and D_s balanced 7-bit digits
// (round to nearest of the scaled remainder, |D_s| <= 64, so each digit and each remainder is
// exact and the dropped remainder is centred on zero).  The product of two rows is then
//     P_r . P_c ~= 2^{e_r + e_c} sum_{l=2..8} 2^{-7 l} S_l,   S_l = sum_{s+t=l} D_s[r] . D_t[c],
// dropping only the terms with s + t > 8 (below 2^{-58} relative to the row maxima).  Each S_l is
// an exact int32 sum of int8 products (|S_l| <= 6 * 64^2 * 128 < 2^22), accumulated by 26
// int8 tensor-core products per 32-deep K step; the levels are combined exactly in 64-bit
// integers into two parts, converted, joined with one FP64 rounding and scaled by exact powers
// of two.  The error per element is at the level of an FP64
// dot product of the same rows (measured: screened forms within ~1e-13 relative of the FP64 DMMA
// path); this is the Ozaki splitting scheme restated for power-of-two row scaling.  (Six balanced
// digits with levels <= 8 match seven truncated ones with levels <= 8 in accuracy -- the
// remainder, not the level cut, dominates either way -- at 26 products instead of 28.)
//
// Two launches per update:
//   k_slice_panel64  one warp per panel row: e_r, and the 6 digit slices of the row's 128 values,
//                    each slice a 128-byte row in the 128-byte-swizzled K-major layout
//                    ([slice][row][128 bytes]) the tensor core reads;
//   k_update64_oz    persistent, warp-specialised, one CTA per SM (10 warps, 222 KB of shared
//                    memory, 512 TMEM columns):
//                      warp 0     producer: units from a global counter handed on through a
//                                 4-slot mbarrier ring; loads the unit's A slices 3-6 (128 rows,
//                                 64 KB, resident for the unit) and streams the B slices (64
//                                 rows, 8 KB each) through a 15-stage ring;
//                      warp 1     TMEM allocation; lane 0 issues tcgen05.mma kind::i8 (M = 128,
//                                 N = 64, K = 32 per instruction; A slices 1-2, which take part
//                                 in 12 of the 26 products, from TMEM (columns 448-511), the
//                                 others and B from shared memory) into 7 int32 accumulators,
//                                 one per level l (columns 64 (l - 2));
//                      warps 2-9  epilogue: at each unit start, write A slices 1-2 into TMEM;
//                                 per tile, warp w reads lane quadrant w % 4, 32 columns (16
//                                 columns per tcgen05.wait::ld), combines the levels, scales by
//                                 2^{e_r + e_c}, stages -value per row (128 bytes per half) and
//                                 adds it to C with a bulk reduction (cp.reduce.async.bulk
//                                 .add.f64) per row and half.
// The accumulators are drained in two level groups so that the tensor core does not wait for the
// whole drain: per tile the MMAs of group X (levels 4-8, 23 of the 26 products) run first and are
// committed, then those of group Y (levels 2-3, 3 products).  The epilogue reads group X (keeping
// S4 2^7 + S5 and the exact low part (S6 2^14 + S7 2^7 + S8) per element) and releases it while
// group Y runs; the next tile's group X then runs while the epilogue reads group Y and finishes
// the tile.  (At N = 64 a tcgen05.mma kind::i8 costs ~48 cycles whatever its operands, so these
// are the tile's 112 instructions back to back; 7 levels x 64 columns leave no room for a second
// accumulator buffer.)
// A work unit is (frequency, 128-row tile i, up to kOzSeg column tiles of 64); column tile c of
// row tile i has work iff c < 2 (i + 1); rows are written from the column tile's first column
// (the diagonal 64 x 64 blocks in full, as the other update kernels do).  Every mbarrier wait is
// bounded as in kernels_tc.cu (expiry -> pivot 0 -> GWB200_DEVICE_TIMEOUT).
#include "internal.cuh"
#include "tc_common.cuh"

#include <cstdlib>

namespace gwb200 {
namespace {

using namespace tc;

constexpr int kOzM = 128;                    // accumulator rows = TMEM lanes
constexpr int kOzN = 64;                     // accumulator columns per level
constexpr int kOzSlices = 6;                 // digit slices per value
constexpr int kOzLevels = 7;                 // levels s + t = 2..8, one accumulator each
constexpr int kOzMaxSum = kOzLevels - 1;     // 0-based slice indices: products with sa + t <= 6
constexpr int kOzSeg = 32;                   // column tiles per work unit
constexpr int kOzStages = 15;                // B ring depth (one slice per stage): a tile's 6, the 2 held
                                             // for group Y, and 7 ahead
constexpr int kOzTmemSlices = 2;             // A slices 1-2 (12 of the 26 products) read from TMEM
constexpr int kSchedSlots = 4;
constexpr int kSliceA = kOzM * 128;          // one slice of 128 rows: 16 KB
constexpr int kSliceB = kOzN * 128;          // of 64 rows: 8 KB
constexpr int kEpiWarps = 8;                 // 4 lane quadrants x 2 column halves of 32
constexpr int kOzThreads = 32 * (2 + kEpiWarps);
constexpr int kTmemCols = 512;               // 7 levels x 64 columns, then A slices 1-2 (32 each)
constexpr int kTmemA = kOzLevels * kOzN;     // first column of the A slices held in TMEM
static_assert(kTmemA + 32 * kOzTmemSlices <= kTmemCols, "TMEM columns");
constexpr int kStgRow = 128 + 16;            // staging row stride: 16 doubles + 16 bytes (banks)
constexpr int kStgBytes = 32 * kStgRow;      // per epilogue warp
constexpr int kHeader = 1024;
constexpr int kOzSmem = kHeader + 1024 + (kOzSlices - kOzTmemSlices) * kSliceA + kOzStages * kSliceB + kEpiWarps * kStgBytes;

constexpr int kOffFull = 0;
constexpr int kOffEmpty = kOffFull + 8 * kOzStages;
constexpr int kOffTFull = kOffEmpty + 8 * kOzStages;    // level group g (0 = X, 1 = Y) ready (tcgen05.commit)
constexpr int kOffTEmpty = kOffTFull + 16;              // group g drained (kEpiWarps arrivals)
constexpr int kOffAFull = kOffTEmpty + 16;              // A slices 3-7 of the unit in smem (tx bytes)
constexpr int kOffAEmpty = kOffAFull + 8;               // MMAs of the unit complete
constexpr int kOffATmem = kOffAEmpty + 8;               // A slices 1-2 in TMEM (kEpiWarps arrivals)
constexpr int kOffDrain = kOffATmem + 8;
constexpr int kOffUFull = kOffDrain + 8;
constexpr int kOffUEmpty = kOffUFull + 8 * kSchedSlots;
constexpr int kOffUnit = kOffUEmpty + 8 * kSchedSlots;
constexpr int kOffTmem = kOffUnit + 8 * kSchedSlots;
constexpr int kOffAbort = kOffTmem + 4;
static_assert(kOffAbort + 4 <= kHeader, "header overflow");
static_assert(kOzSmem <= 227 * 1024, "shared memory");

// Instruction descriptor, kind::i8: D S32 (bits 4-5 = 2), A and B signed 8-bit (bits 7-9,
// 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzN >> 3) << 17) |
                              ((uint32_t)(kOzM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdescI8), "r"(accumulate)
        : "memory");
}

// A from TMEM (lane = row, 4 consecutive K bytes per 32-bit column), B from shared memory.
__device__ __forceinline__ void mma_i8_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(db), "r"(kIdescI8), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tmem_st32u(uint32_t taddr, const uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]),
        "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
        "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
}

__device__ __forceinline__ double pow2(int k) {  // 2^k for -1022 <= k <= 1023, exact
    return __longlong_as_double((long long)(k + 1023) << 52);
}

// Per frequency: 6 slices of rp rows x 128 bytes, then rp int32 exponents.
__host__ __device__ constexpr size_t oz_freq_bytes(int64_t rp) {
    return ((size_t)kOzSlices * rp * 128 + (size_t)rp * 4 + 1023) / 1024 * 1024;
}

__global__ void __launch_bounds__(256) k_slice_panel64(const double* __restrict__ a, int64_t ld, int64_t stride,
                                                       int64_t kb0, int64_t c_begin, int64_t rows, int64_t rp,
                                                       uint8_t* __restrict__ buf) {
    const int f = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t rr = (int64_t)blockIdx.x * 8 + warp;  // panel row
    if (rr >= rp) return;
    const int64_t r = c_begin + rr;
    uint8_t* slices = buf + (size_t)f * oz_freq_bytes(rp);
    int32_t* exps = reinterpret_cast<int32_t*>(slices + (size_t)kOzSlices * rp * 128);
    double x[4] = {0.0, 0.0, 0.0, 0.0};
    if (r < rows) {
        const double* row = a + (size_t)f * stride + (size_t)r * ld + kb0 + 4 * lane;
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = row[j];
    }
    double m = fmax(fmax(fabs(x[0]), fabs(x[1])), fmax(fabs(x[2]), fabs(x[3])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    if (m > 0.0) frexp(m, &e);  // m = frac * 2^e, frac in [0.5, 1): |x| < 2^e
    ++e;                        // the row scale: |x| < 2^{e - 1}
    const double inv = pow2(-e);
    double v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = x[j] * inv;  // |v| < 1/2, exact
    const uint32_t chunk = (uint32_t)(lane >> 2), in_chunk = (uint32_t)(lane & 3) * 4;
    const size_t pos = (size_t)((chunk ^ (uint32_t)(rr & 7)) * 16 + in_chunk);
#pragma unroll
    for (int s = 0; s < kOzSlices; ++s) {
        uint32_t word = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double t = v[j] * 128.0;  // exact, |t| <= 64
            const double d = rint(t);        // |d| <= 64
            v[j] = t - d;                    // exact, |v| <= 1/2
            word |= ((uint32_t)(int)d & 0xFFu) << (8 * j);
        }
        *reinterpret_cast<uint32_t*>(slices + ((size_t)s * rp + rr) * 128 + pos) = word;
    }
    if (lane == 0) exps[rr] = e;
}

struct UnitSpace {
    int64_t T, NI, NS, per_f, total;
};

// unit -> (frequency, row tile i, column tiles [c0, c1)); the longest row tiles first
__device__ __forceinline__ bool decode_unit(const UnitSpace& us, int64_t u, int& f, int64_t& i, int64_t& c0,
                                            int64_t& c1) {
    f = (int)(u / us.per_f);
    const int64_t rem = u - (int64_t)f * us.per_f;
    const int64_t q = rem / us.NS;
    i = us.NI - 1 - q;
    c0 = (rem - q * us.NS) * kOzSeg;
    c1 = min(c0 + kOzSeg, min(us.T, 2 * i + 2));
    return c0 < c1;
}

__global__ void __launch_bounds__(kOzThreads, 1)
    k_update64_oz(double* __restrict__ a, int64_t ld, int64_t stride, int64_t c_begin, int64_t rows,
                  const uint8_t* __restrict__ buf, int64_t rp, UnitSpace us, unsigned long long* __restrict__ sched,
                  unsigned long long* err, int withhold_first_stage) {
    extern __shared__ __align__(1024) uint8_t osm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = smem_u32(osm);
    const uint32_t abuf = (base + kHeader + 1023u) & ~1023u;  // A slices 3-6, 1024-aligned
    const uint32_t ring = abuf + (kOzSlices - kOzTmemSlices) * kSliceA;  // B stages (A slices 3-6 before)
    const uint32_t stg0 = ring + kOzStages * kSliceB;          // epilogue staging rows
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(osm + kOffAbort);
    volatile int64_t* uslot = reinterpret_cast<volatile int64_t*>(osm + kOffUnit);
    auto full = [&](int s) { return base + kOffFull + 8 * s; };
    auto empty = [&](int s) { return base + kOffEmpty + 8 * s; };
    auto ufull = [&](int j) { return base + kOffUFull + 8 * j; };
    auto uempty = [&](int j) { return base + kOffUEmpty + 8 * j; };
    auto tfull = [&](int g) { return base + kOffTFull + 8 * g; };
    auto tempty = [&](int g) { return base + kOffTEmpty + 8 * g; };
    const uint32_t afull = base + kOffAFull, aempty = base + kOffAEmpty, drain = base + kOffDrain;
    const uint32_t atmem = base + kOffATmem;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kOzStages; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int j = 0; j < kSchedSlots; ++j) {
            mbar_init(ufull(j), 1);
            mbar_init(uempty(j), 1 + kEpiWarps);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(tfull(g), 1);
            mbar_init(tempty(g), kEpiWarps);
        }
        mbar_init(afull, 1);
        mbar_init(atmem, kEpiWarps);
        mbar_init(aempty, 1);
        mbar_init(drain, 1);
        *abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kOffTmem),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(osm + kOffTmem);
    const size_t fbytes = oz_freq_bytes(rp);

    if (warp == 0) {
        // ---- producer ----
        int s = 0, js = 0;
        uint32_t ph = 0, aph = 0, jph = 0;
        uint32_t filled = 0, fill_par = 0;
        bool a_filled = false;
        for (;;) {
            int f = 0;
            int64_t i = 0, c0 = 0, c1 = 0, u = 0;
            if (lane == 0) {
                do {
                    u = (int64_t)atomicAdd(sched, 1ull);
                } while (u < us.total && !decode_unit(us, u, f, i, c0, c1));
                if (u > us.total) u = us.total;
            }
            u = __shfl_sync(0xffffffffu, u, 0);
            uint32_t got = 1;
            if (lane == 0) {
                got = mbar_wait(uempty(js), jph ^ 1u, abort_flag, err) ? 1u : 0u;
                if (got) {
                    uslot[js] = u;
                    mbar_arrive(ufull(js));
                }
            }
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) break;
            if (++js == kSchedSlots) {
                js = 0;
                jph ^= 1u;
            }
            if (u >= us.total) break;
            decode_unit(us, u, f, i, c0, c1);
            const uint8_t* slices = buf + (size_t)f * fbytes;
            if (lane == 0) got = mbar_wait(aempty, aph ^ 1u, abort_flag, err) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) break;
            if (lane == 0) mbar_expect_tx(afull, (uint32_t)((kOzSlices - kOzTmemSlices) * kSliceA));
            __syncwarp();
            if (lane < kOzSlices - kOzTmemSlices)  // one 16 KB copy per smem slice (slices 3-6)
                bulk_g2s(abuf + lane * kSliceA, slices + ((size_t)(lane + kOzTmemSlices) * rp + i * kOzM) * 128, kSliceA,
                         afull);
            a_filled = true;
            aph ^= 1u;
            bool ok = true;
            for (int64_t c = c0; ok && c < c1; ++c) {
                for (int t = 0; t < kOzSlices; ++t) {
                    if (lane == 0) got = mbar_wait(empty(s), ph ^ 1u, abort_flag, err) ? 1u : 0u;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (!got) {
                        ok = false;
                        break;
                    }
                    if (withhold_first_stage && blockIdx.x == 0 && filled == 0) {
                        withhold_first_stage = 0;  // test of the bounded waits (see kernels_tc.cu)
                    } else {
                        if (lane == 0) {
                            mbar_expect_tx(full(s), (uint32_t)kSliceB);
                            bulk_g2s(ring + s * kSliceB, slices + ((size_t)t * rp + c * kOzN) * 128, kSliceB, full(s));
                        }
                        filled |= 1u << s;
                        fill_par = (fill_par & ~(1u << s)) | (ph << s);
                    }
                    __syncwarp();
                    if (++s == kOzStages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) break;
        }
        if (lane == 0) {
            for (int q = 0; q < kOzStages; ++q)
                if (filled & (1u << q)) mbar_drain(full(q), (fill_par >> q) & 1u);
            if (a_filled) mbar_drain(afull, aph ^ 1u);
        }
        __syncwarp();
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        const uint64_t desc_a0 = smem_desc_sw128(abuf), desc_b0 = smem_desc_sw128(ring);
        int s = 0, js = 0;
        uint32_t ph = 0, acc_ph = 0, aph = 0, jph = 0;
        bool issued = false, ok = true;
        for (;;) {
            const int64_t u = take_unit(ufull(js), uempty(js), uslot + js, jph, abort_flag, err);
            if (++js == kSchedSlots) {
                js = 0;
                jph ^= 1u;
            }
            if (u < 0 || u >= us.total) break;
            int f;
            int64_t i, c0, c1;
            decode_unit(us, u, f, i, c0, c1);
            if (!mbar_wait(afull, aph, abort_flag, err)) break;
            if (!mbar_wait(atmem, aph, abort_flag, err)) break;
            tc_fence_after();
            aph ^= 1u;
            // A slice sa+1 against B slice t+1 (in stage st) into level sa + t + 2.  Products are
            // issued with t ascending, so the first product of level sa + t has the smallest t
            // the level allows, t0 = max(0, sa + t - (kOzSlices - 1)); it starts the accumulator
            // at kk = 0 (level 8 has no t = 0 product: it starts at sa = 6, t = 2, 1-based)
            auto pair = [&](int sa, int t, int st) {
                // descriptors differ from the stage / A bases only in the address field (bytes >>
                // 4, below 2^14 for shared memory): constant offsets, no carries
                const uint64_t db0 = desc_b0 + (uint64_t)((uint32_t)(st * kSliceB) >> 4);
                const uint32_t d = tmem + (uint32_t)((sa + t) * kOzN);
                const bool starts = t == (sa + t > kOzSlices - 1 ? sa + t - (kOzSlices - 1) : 0);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const uint32_t acc = (!starts || kk > 0) ? 1u : 0u;
                    if (sa < kOzTmemSlices)  // A slice from TMEM: 32 bytes of K = 8 columns
                        mma_i8_ts(d, tmem + (uint32_t)(kTmemA + 32 * sa + 8 * kk), db0 + (uint64_t)(2 * kk), acc);
                    else
                        mma_i8(d, desc_a0 + (uint64_t)(((sa - kOzTmemSlices) * kSliceA + 32 * kk) >> 4),
                               db0 + (uint64_t)(2 * kk), acc);
                }
            };
            for (int64_t c = c0; ok && c < c1; ++c) {
                // group X (levels 4-8, sa + t >= 2) once the epilogue has read the previous tile's
                if (!mbar_wait_fast(tempty(0), acc_ph ^ 1u, abort_flag, err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                int st01[2] = {0, 0};  // stages of B slices 1-2, held for group Y
#pragma unroll
                for (int t = 0; t < kOzSlices; ++t) {
                    if (!mbar_wait_fast(full(s), ph, abort_flag, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
#pragma unroll
                    for (int sa = 0; sa < kOzSlices; ++sa)
                        if (sa + t >= 2 && sa + t <= kOzMaxSum) pair(sa, t, s);
                    if (t < 2)
                        st01[t] = s;
                    else
                        mma_commit(empty(s));
                    issued = true;
                    if (++s == kOzStages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(tfull(0));
                // group Y (levels 2-3) once the epilogue has read the previous tile's
                if (!mbar_wait_fast(tempty(1), acc_ph ^ 1u, abort_flag, err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                pair(0, 0, st01[0]);
                pair(1, 0, st01[0]);
                pair(0, 1, st01[1]);
                mma_commit(empty(st01[0]));
                mma_commit(empty(st01[1]));
                mma_commit(tfull(1));
                acc_ph ^= 1u;
            }
            if (!ok) break;
            mma_commit(aempty);
        }
        if (issued) {
            mma_commit(drain);
            mbar_drain(drain, 0);
        }
    } else if (warp >= 2) {
        // ---- epilogue ----
        const int q = warp & 3, half = (warp - 2) >> 2;
        const uint32_t stg = stg0 + (uint32_t)(warp - 2) * kStgBytes + (uint32_t)lane * kStgRow;
        int js = 0;
        uint32_t acc_ph = 0, jph = 0, aph = 0;
        bool ok = true, reduced = false;
        while (ok) {
            int64_t u = 0;
            if (lane == 0) u = take_unit(ufull(js), uempty(js), uslot + js, jph, abort_flag, err);
            u = __shfl_sync(0xffffffffu, u, 0);
            if (++js == kSchedSlots) {
                js = 0;
                jph ^= 1u;
            }
            if (u < 0 || u >= us.total) break;
            int f;
            int64_t i, c0, c1;
            decode_unit(us, u, f, i, c0, c1);
            const uint8_t* slices = buf + (size_t)f * fbytes;
            const int32_t* exps = reinterpret_cast<const int32_t*>(slices + (size_t)kOzSlices * rp * 128);
            const int64_t rr = i * kOzM + q * 32 + lane;  // panel row of this lane
            {   // A slices 1-2 of the unit into TMEM (warp half h writes slice h + 1 of its lane
                // quadrant) once the previous unit's MMAs are done with them
                uint32_t got = 1;
                if (lane == 0) got = mbar_wait(aempty, aph ^ 1u, abort_flag, err) ? 1u : 0u;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) break;
                aph ^= 1u;
                tc_fence_after();
                const uint4* row = reinterpret_cast<const uint4*>(slices + ((size_t)half * rp + rr) * 128);
                uint32_t w[32];
#pragma unroll
                for (int c = 0; c < 8; ++c) {  // undo the 128-byte swizzle of the slice row
                    const uint4 x = row[c ^ (int)(rr & 7)];
                    w[4 * c] = x.x;
                    w[4 * c + 1] = x.y;
                    w[4 * c + 2] = x.z;
                    w[4 * c + 3] = x.w;
                }
                tmem_st32u(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kTmemA + 32 * half), w);
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(atmem);
            }
            const int64_t r = c_begin + rr;
            const int er = exps[rr];
            for (int64_t c = c0; c < c1; ++c) {
                const int64_t cj = c_begin + c * kOzN + half * 32;  // this warp's first column
                const bool valid = r < rows && r >= c_begin + c * kOzN;
                const int ec_lane = exps[c * kOzN + half * 32 + lane];  // exponent of column cj + lane
                // Levels combined exactly: adjacent pairs in int32 (|S_l| <= 6 64^2 128 < 2^22, so
                // S2 2^7 + S3, S4 2^7 + S5, S6 2^7 + S7 < 2^30), then hi = (S2 2^7 + S3) 2^14 +
                // S4 2^7 + S5 < 2^44 and lo = (S6 2^7 + S7) 2^7 + S8 < 2^37 in int64 (held as an
                // exact double between the groups); value = hi 2^-35 + lo 2^-56 with one rounding,
                // scaled by 2^{e_r + e_c}.
                const uint32_t lanes = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(half * 32);
                auto wait_group = [&](int g) {
                    uint32_t got = 1;
                    if (lane == 0) got = mbar_wait(tfull(g), acc_ph, abort_flag, err) ? 1u : 0u;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (got) tc_fence_after();
                    return got != 0u;
                };
                auto release_group = [&](int g) {  // the group's levels are in registers
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty(g));
                };
                if (!wait_group(0)) {
                    ok = false;
                    break;
                }
                // group X leaves m = (S4 2^7 + S5) 2^21 + lo (|m| < 2^51: exact as a double), and
                // value = p23 2^-21 + m 2^-56 = hi 2^-35 + lo 2^-56, the same sum rounded once
                double m_d[32];
#pragma unroll
                for (int h16 = 0; h16 < 2; ++h16) {  // group X: levels 4-8, 16 columns per wait
                    uint32_t v[kOzLevels - 2][16];
#pragma unroll
                    for (int L = 2; L < kOzLevels; ++L) tmem_ld16_nowait(lanes + (uint32_t)(L * kOzN + 16 * h16), v[L - 2]);
                    tmem_wait_ld();
                    if (h16 == 1) release_group(0);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int32_t p45 = (int32_t)v[0][j] * 128 + (int32_t)v[1][j];
                        const int32_t p67 = (int32_t)v[2][j] * 128 + (int32_t)v[3][j];
                        const long long lo = (long long)p67 * 128 + (int32_t)v[4][j];
                        m_d[16 * h16 + j] = (double)((long long)p45 * (1LL << 21) + lo);  // exact
                    }
                }
                if (!wait_group(1)) {
                    ok = false;
                    break;
                }
                acc_ph ^= 1u;
#pragma unroll
                for (int h16 = 0; h16 < 2; ++h16) {  // group Y: levels 2-3, then the half's 16 columns to C
                    uint32_t v[2][16];
                    tmem_ld16_nowait(lanes + (uint32_t)(16 * h16), v[0]);
                    tmem_ld16_nowait(lanes + (uint32_t)(kOzN + 16 * h16), v[1]);
                    tmem_wait_ld();
                    if (h16 == 1) release_group(1);
                    double val[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int32_t p23 = (int32_t)v[0][j] * 128 + (int32_t)v[1][j];
                        const int ej = __shfl_sync(0xffffffffu, ec_lane, 16 * h16 + j);
                        // (p23 2^35 + m) rounded once is 2^56 times the value rounded once: the
                        // 2^-56 joins the exact power-of-two scale (one FP64 multiply less; the
                        // epilogue's FP64 work is on this kernel's critical path)
                        val[j] = -fma((double)p23, 0x1p35, m_d[16 * h16 + j]) * pow2(er + ej - 56);
                    }
                    if (valid) {  // stage the half row (128 bytes), then one bulk reduction
                        if (reduced) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
#pragma unroll
                        for (int j = 0; j < 16; j += 2)
                            asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(stg + 8u * j), "d"(val[j]),
                                         "d"(val[j + 1])
                                         : "memory");
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    if (valid) {
                        double* dst = a + (size_t)f * stride + (size_t)r * ld + cj + 16 * h16;
                        asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], 128;" ::"l"(
                                         dst),
                                     "r"(stg)
                                     : "memory");
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                        reduced = true;
                    }
                }
            }
        }
        if (reduced) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // this lane's reductions done
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

} // namespace

size_t oz_slice_bytes_per_freq(const TallGeometry& g) { return oz_freq_bytes((g.rows + kOzM - 1) / kOzM * kOzM); }

int launch_update64_oz(const TallGeometry& g, int64_t nf, double* a, int64_t kb0, int64_t c_begin, void* slices,
                       unsigned long long* sched, unsigned long long* err, cudaStream_t s, int max_ctas) {
    const int64_t T = (g.n_pad - c_begin) / kOzN;
    if (T <= 0 || nf <= 0) return 0;
    const int64_t H = g.rows - c_begin;
    const int64_t NI = (H + kOzM - 1) / kOzM, rp = NI * kOzM;
    uint8_t* buf = static_cast<uint8_t*>(slices);
    k_slice_panel64<<<dim3((unsigned)(rp / 8), (unsigned)nf), 256, 0, s>>>(a, g.ld, g.stride, kb0, c_begin, g.rows, rp,
                                                                          buf);
    GWB_LAUNCH("k_slice_panel64");
    GWB_CUDA(cudaFuncSetAttribute(k_update64_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem));
    UnitSpace us;
    us.T = T;
    us.NI = NI;
    us.NS = (T + kOzSeg - 1) / kOzSeg;
    us.per_f = NI * us.NS;
    us.total = nf * us.per_f;
    GWB_CUDA(cudaMemsetAsync(sched, 0, sizeof(unsigned long long), s));
    const char* expire = std::getenv("GWB200_TEST_EXPIRE_WAIT");
    const int withhold = (expire && expire[0] == '1') ? 1 : 0;
    const unsigned grid = (unsigned)std::min<int64_t>(us.total, max_ctas > 0 ? std::min(max_ctas, sm_count()) : sm_count());
    k_update64_oz<<<grid, kOzThreads, kOzSmem, s>>>(a, g.ld, g.stride, c_begin, g.rows, buf, rp, us, sched, err,
                                                     withhold);
    GWB_LAUNCH("k_update64_oz");
    return 2;
}

} // namespace gwb200
