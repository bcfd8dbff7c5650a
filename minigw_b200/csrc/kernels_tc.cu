// kernels_tc.cu -- the mixed form's trailing update on the 5th-generation tensor cores (tcgen05).
//
// After an outer block of K = 64 or 128 columns [kb0, kb0+K) has been factored, every element of
// the trailing lower part C = A[r][c] (c_begin <= c < n_pad, c <= r < rows) takes
// C -= P_r . P_c with P the FP32 panel A[:, kb0:kb0+K).  The products use the 3xTF32 split
// (x = hi + lo, hi = rna_tf32(x), lo = rna_tf32(x - hi); x.y ~ lo.hi + hi.lo + hi.hi, in that
// order per 8-deep K step) accumulated in FP32: the same arithmetic, in the same order, as the
// mma.sync update of kernels_f32.cu.
//
// Two launches per update:
//   k_split_panel32  writes hi and lo of the panel rows [c_begin, rows) in the 128-byte-swizzled
//                    K-major layout the tensor core reads ([K slice of 32 floats][row][128 bytes],
//                    rows padded with zeros to a multiple of 128), so that every operand slice of a
//                    tile is one contiguous 16 KB block (one cp.async.bulk);
//   k_update32_tc    a persistent, warp-specialised kernel, one CTA per SM (18 warps, 226 KB of
//                    shared memory, all 512 TMEM columns):
//                      warp 0     producer: takes work units from a global counter and hands them
//                                 to the other roles through a 4-slot mbarrier ring; streams B
//                                 (128 rows x 32 of K, hi and lo) through a 6-stage ring,
//                                 and prefetches the unit's A rows into L2;
//                      warp 1     allocates TMEM; lane 0 issues tcgen05.mma kind::tf32 (M = 128,
//                                 N = 128, K = 8 per instruction) with A from TMEM (the unit's 128
//                                 rows, hi and lo, K = 128: columns 256-511) and B from shared
//                                 memory (K-major SW128)
//                                 into a double-buffered FP32 accumulator (columns 0-255), and
//                                 commits stage releases, accumulator-ready and A-release;
//                      warps 2-9  epilogue: warp w reads TMEM lane quadrant w % 4, 64 columns
//                                 as two 32 x 32 boxes; tcgen05.ld, releases the accumulator,
//                                 stages -acc 128B-swizzled in shared memory and adds it to C with
//                                 a TMA tensor reduce (cp.reduce.async.bulk.tensor .add, whole
//                                 128-byte lines; the read-modify-write happens in L2);
//                      warps 10-17 A loaders: fill the unit's A into TMEM (tcgen05.st) as soon as
//                                 the previous unit's MMAs release it.
// A work unit is (frequency, 128-row tile i, up to 48 column tiles of 128); column tile c of row
// tile i has work iff c <= i, and units of the longest row tiles are handed out first.  Writes are
// limited to the lower part at 64-column-block granularity (the diagonal 64 x 64 blocks in full,
// as the other update kernels do).
//
// Every mbarrier wait is bounded (kWaitNs of %globaltimer); on expiry the CTA raises a shared
// abort flag, records 0 in the pivot word (read back by the host as GWB200_DEVICE_TIMEOUT), waits
// (bounded) for its own bulk copies and MMAs, frees its TMEM and returns.
#include "internal.cuh"
#include "tc_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <mutex>

namespace gwb200 {
namespace {

using namespace tc;

constexpr int kTcM = 128;                   // accumulator rows = TMEM lanes = A rows per unit
constexpr int kTcN = 128;                   // accumulator columns per tile
constexpr int kTcKc = 32;                   // floats of K per B pipeline stage
constexpr int kTcStages = 6;                // B ring depth
constexpr int kTcSeg = 48;                  // column tiles per work unit (A is loaded once per unit, and
                                            // the MMAs wait for it: 16 -> 48 took config 3's mixed
                                            // solve from 127.8 to 124.2 ms)
constexpr int kSchedSlots = 4;              // unit-index ring from the producer to the other roles
constexpr int kRowBytes = kTcKc * 4;        // one row of a K slice: 128 bytes = one swizzle atom row
constexpr int kSliceB = kTcN * kRowBytes;   // 16384 bytes
constexpr int kStageBytes = 2 * kSliceB;    // B stage: hi + lo slice, two copies
constexpr int kEpiWarps = 8;                // epilogue: 4 lane quadrants x 2 column halves of 64
constexpr int kLoadWarps = 8;               // A into TMEM: 4 lane quadrants x (hi | lo)
constexpr int kTcThreads = 32 * (2 + kEpiWarps + kLoadWarps);
constexpr int kTmemCols = 512;       // accumulators [0, 256), A hi [256, 384), A lo [384, 512)
constexpr int kTmemAHi = 2 * kTcN, kTmemALo = kTmemAHi + 128;
constexpr int kHeader = 1024;        // mbarriers, unit ring, TMEM address, abort flag
// + 1024: the operand region starts at the first 1024-byte boundary after the header (the
// 128-byte swizzle is applied to shared-memory address bits, so every slice is 1024-aligned)
constexpr int kStgBytes = 32 * 32 * 4;       // per epilogue warp: 32 rows x 32 floats, 128B-swizzled
constexpr int kTcSmem = kHeader + 1024 + kTcStages * kStageBytes + kEpiWarps * kStgBytes;

// header layout (byte offsets)
constexpr int kOffFull = 0;                              // kTcStages: B stage filled (tx bytes)
constexpr int kOffEmpty = kOffFull + 8 * kTcStages;      // kTcStages: B stage consumed (tcgen05.commit)
constexpr int kOffTFull = kOffEmpty + 8 * kTcStages;     // 2: accumulator ready (tcgen05.commit)
constexpr int kOffTEmpty = kOffTFull + 16;               // 2: accumulator drained (kEpiWarps arrivals)
constexpr int kOffAFull = kOffTEmpty + 16;               // 1: A of the unit in TMEM (kLoadWarps arrivals)
constexpr int kOffAEmpty = kOffAFull + 8;                // 1: all MMAs reading A of the unit complete
constexpr int kOffDrain = kOffAEmpty + 8;                // 1: all MMAs of this CTA complete
constexpr int kOffUFull = kOffDrain + 8;                 // kSchedSlots: unit index written
constexpr int kOffUEmpty = kOffUFull + 8 * kSchedSlots;  // kSchedSlots: read by MMA + epilogue warps
constexpr int kOffUnit = kOffUEmpty + 8 * kSchedSlots;   // kSchedSlots x i64 unit indices
constexpr int kOffTmem = kOffUnit + 8 * kSchedSlots;     // u32 TMEM base address
constexpr int kOffAbort = kOffTmem + 4;                  // u32 abort flag

static_assert(kOffAbort + 4 <= kHeader, "header overflow");
static_assert(kTcSmem <= 227 * 1024, "shared memory");

// Instruction descriptor, kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdescTf32 =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

// A from TMEM (lane = row, one 32-bit column per K element), B from shared memory.
__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(db), "r"(kIdescTf32), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
        "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]), "f"(v[17]), "f"(v[18]),
        "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]),
        "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}
// C[f][y .. y+32)[x .. x+32) += staging tile (FP32 add performed by the TMA unit / L2, whole
// 128-byte lines), tracked in this thread's bulk async-group.
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* map, uint32_t src, int x, int y, int z) {
    asm volatile("cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(src), "r"(x), "r"(y), "r"(z)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ float rna_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi/lo of panel rows [c_begin, rows) x columns [kb0, kb0 + 32 nkc) in the 128-byte-swizzled
// K-major layout: [K slice of 32 floats][row][128 bytes], the 16-byte chunk c of row rr stored at
// chunk position c ^ (rr % 8); rows [rows - c_begin, rp) are zero.  Per frequency: hi at
// panel + f*2*nkc*rp*32, lo nkc*rp*32 floats later.  One thread per 16-byte chunk.
__global__ void k_split_panel32(const float* __restrict__ a, int64_t ld, int64_t stride, int64_t kb0, int nkc,
                                int64_t c_begin, int64_t rows, int64_t rp, float* __restrict__ panel) {
    const int f = blockIdx.y;
    const float* A = a + (size_t)f * stride;
    float4* hi = reinterpret_cast<float4*>(panel + (size_t)f * 2 * nkc * rp * 32);
    float4* lo = hi + (size_t)nkc * rp * 8;
    const int64_t total = (int64_t)nkc * rp * 8;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t srow = idx >> 3;  // kb * rp + rr
        const int c = (int)(idx & 7);
        const int64_t kb = srow / rp, rr = srow - kb * rp;
        const int64_t r = c_begin + rr;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (r < rows) x = *reinterpret_cast<const float4*>(A + (size_t)r * ld + kb0 + 32 * kb + 4 * c);
        float4 h, l;
        h.x = rna_tf32(x.x);
        h.y = rna_tf32(x.y);
        h.z = rna_tf32(x.z);
        h.w = rna_tf32(x.w);
        l.x = rna_tf32(x.x - h.x);
        l.y = rna_tf32(x.y - h.y);
        l.z = rna_tf32(x.z - h.z);
        l.w = rna_tf32(x.w - h.w);
        const int64_t dst = srow * 8 + (c ^ (int)(rr & 7));
        hi[dst] = h;
        lo[dst] = l;
    }
}

// Work units: (frequency, 128-row tile i, segment of kTcSeg column tiles of 128).  Column tile c
// of row tile i holds something to write iff c <= i; a unit covers column tiles
// [seg*kTcSeg, min((seg+1)*kTcSeg, T, i+1)).  Within a frequency the units of the longest row
// tiles (largest i) come first; CTAs take units in that order from a global counter.
struct UnitSpace {
    int64_t T, NI, NS, per_f, total;
};

__device__ __forceinline__ bool decode_unit(const UnitSpace& us, int64_t u, int& f, int64_t& i, int64_t& c0,
                                            int64_t& c1) {
    f = (int)(u / us.per_f);
    const int64_t rem = u - (int64_t)f * us.per_f;
    const int64_t q = rem / us.NS;
    i = us.NI - 1 - q;
    c0 = (rem - q * us.NS) * kTcSeg;
    c1 = min(c0 + kTcSeg, min(us.T, i + 1));
    return c0 < c1;
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_update32_tc(float* __restrict__ a, int64_t ld, int64_t stride, int64_t c_begin, int64_t rows, int64_t n_pad,
                  int64_t row_min, int nkc, const float* __restrict__ panel, int64_t rp, UnitSpace us,
                  unsigned long long* __restrict__ sched, unsigned long long* err, int withhold_first_stage,
                  const __grid_constant__ CUtensorMap cmap) {
    extern __shared__ __align__(1024) uint8_t tsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = smem_u32(tsm);
    const uint32_t ring = (base + kHeader + 1023u) & ~1023u;  // B stages, 1024-aligned
    const uint32_t stg0 = ring + kTcStages * kStageBytes;     // epilogue staging tiles, 1024-aligned
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(tsm + kOffAbort);
    volatile int64_t* uslot = reinterpret_cast<volatile int64_t*>(tsm + kOffUnit);
    auto full = [&](int s) { return base + kOffFull + 8 * s; };
    auto empty = [&](int s) { return base + kOffEmpty + 8 * s; };
    auto tfull = [&](int b) { return base + kOffTFull + 8 * b; };
    auto tempty = [&](int b) { return base + kOffTEmpty + 8 * b; };
    auto ufull = [&](int j) { return base + kOffUFull + 8 * j; };
    auto uempty = [&](int j) { return base + kOffUEmpty + 8 * j; };
    const uint32_t afull = base + kOffAFull, aempty = base + kOffAEmpty, drain = base + kOffDrain;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull(b), 1);
            mbar_init(tempty(b), kEpiWarps);
        }
        for (int j = 0; j < kSchedSlots; ++j) {
            mbar_init(ufull(j), 1);
            mbar_init(uempty(j), 1 + kEpiWarps + kLoadWarps);
        }
        mbar_init(afull, kLoadWarps);
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
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tsm + kOffTmem);

    const size_t half_floats = (size_t)nkc * rp * 32;  // hi (or lo) of one frequency

    if (warp == 0) {
        // ---- producer: takes units from the global counter, hands them on, streams B ----
        int s = 0, js = 0;
        uint32_t ph = 0, jph = 0;
        uint32_t filled = 0, fill_par = 0;  // per B stage: ever filled, parity of its last fill
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
            const float* hi = panel + (size_t)f * 2 * half_floats;
            const float* lo = hi + half_floats;
            // the unit's A rows (read once, by the epilogue warps into TMEM when the unit starts):
            // bring them into L2 now, about a tile ahead of their use
            if (lane < 2 * nkc) {
                const int which = lane / nkc, kb = lane - which * nkc;
                const float* src = (which == 0 ? hi : lo) + (size_t)((int64_t)kb * rp + i * kTcM) * 32;
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(kTcM * kRowBytes) : "memory");
            }
            bool ok = true;
            for (int64_t c = c0; ok && c < c1; ++c) {
                for (int kb = 0; kb < nkc; ++kb) {
                    if (lane == 0) got = mbar_wait(empty(s), ph ^ 1u, abort_flag, err) ? 1u : 0u;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (!got) {
                        ok = false;
                        break;
                    }
                    if (withhold_first_stage && blockIdx.x == 0 && filled == 0) {
                        // test of the bounded waits: this stage is never filled, so the MMA
                        // thread's wait for it can only end by expiry (GWB200_DEVICE_TIMEOUT)
                        withhold_first_stage = 0;
                    } else {
                        if (lane == 0) mbar_expect_tx(full(s), kStageBytes);
                        __syncwarp();
                        if (lane < 2) {  // one 16 KB copy each of hi and lo
                            const float* src = (lane == 0 ? hi : lo) + (size_t)((int64_t)kb * rp + c * kTcN) * 32;
                            bulk_g2s(ring + s * kStageBytes + lane * kSliceB, src, kSliceB, full(s));
                        }
                        filled |= 1u << s;
                    }
                    fill_par = (fill_par & ~(1u << s)) | (ph << s);
                    if (++s == kTcStages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) break;
        }
        // every issued copy has landed before the CTA may exit (normally already consumed)
        if (lane == 0) {
            for (int q = 0; q < kTcStages; ++q)
                if (filled & (1u << q)) mbar_drain(full(q), (fill_par >> q) & 1u);
        }
        __syncwarp();
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer: one thread waits, issues and commits ----
        int s = 0, ab = 0, js = 0;
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
            if (!mbar_wait(afull, aph, abort_flag, err)) break;  // A of the unit is in TMEM
            tc_fence_after();
            aph ^= 1u;
            for (int64_t c = c0; ok && c < c1; ++c) {
                if (!mbar_wait_fast(tempty(ab), acc_ph ^ 1u, abort_flag, err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(ab * kTcN);
                for (int kb = 0; kb < nkc; ++kb) {
                    if (!mbar_wait_fast(full(s), ph, abort_flag, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = ring + s * kStageBytes;
#pragma unroll
                    for (int kk = 0; kk < kTcKc / 8; ++kk) {
                        const uint32_t acol = (uint32_t)(kb * kTcKc + 8 * kk);
                        const uint64_t bhi = smem_desc_sw128(st + 32u * kk);
                        const uint64_t blo = smem_desc_sw128(st + kSliceB + 32u * kk);
                        mma_tf32_ts(d, tmem + kTmemALo + acol, bhi, (kb > 0 || kk > 0) ? 1u : 0u);
                        mma_tf32_ts(d, tmem + kTmemAHi + acol, blo, 1u);
                        mma_tf32_ts(d, tmem + kTmemAHi + acol, bhi, 1u);
                    }
                    mma_commit(empty(s));
                    issued = true;
                    if (++s == kTcStages) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(tfull(ab));
                if (++ab == 2) {
                    ab = 0;
                    acc_ph ^= 1u;
                }
            }
            if (!ok) break;
            mma_commit(aempty);
        }
        // all MMAs of this CTA complete before TMEM is released
        if (issued) {
            mma_commit(drain);
            mbar_drain(drain, 0);
        }
    } else if (warp >= 2 && warp < 2 + kEpiWarps) {
        // ---- epilogue: warp -> TMEM lane quadrant (warp % 4) and 64-column half, two 32x32 boxes ----
        const int q = warp & 3, half = (warp - 2) >> 2;
        const uint32_t stg = stg0 + (uint32_t)(warp - 2) * kStgBytes;
        int ab = 0, js = 0;
        uint32_t acc_ph = 0, jph = 0;
        bool ok = true;
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
            const int64_t rs = c_begin + i * kTcM + q * 32;  // first row of this warp's 32-row boxes
            for (int64_t c = c0; c < c1; ++c) {
                uint32_t got = 1;
                if (lane == 0) got = mbar_wait(tfull(ab), acc_ph, abort_flag, err) ? 1u : 0u;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int b = 0; b < 2; ++b) {
                    const int64_t cj = c_begin + c * kTcN + half * 64 + b * 32;  // first column of the box
                    // lower part at 64-column-block granularity (the diagonal 64x64 blocks in full): a
                    // 32-row box starting at a multiple of 32 is wholly in or wholly out; rows past
                    // `rows` are clipped by the tensor map
                    const bool box = cj < n_pad && rs < rows && rs >= (cj & ~(int64_t)63) && rs >= row_min;
                    float acc[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * kTcN + half * 64 + b * 32), acc);
                    if (b == 1) {  // both halves read: the accumulator is free
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(tempty(ab));
                    }
                    if (box) {
                        // C += (-acc): the box staged 128B-swizzled (row `lane`, 16-byte chunk j at
                        // chunk j ^ (lane % 8): conflict-free), then one TMA reduce-add; the staging
                        // buffer is rewritten only after the previous reduce has read it
                        if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                        __syncwarp();
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const uint32_t dst = stg + (uint32_t)lane * 128u + (uint32_t)((j ^ (lane & 7)) * 16);
                            asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(dst), "f"(-acc[4 * j]),
                                         "f"(-acc[4 * j + 1]), "f"(-acc[4 * j + 2]), "f"(-acc[4 * j + 3])
                                         : "memory");
                        }
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        __syncwarp();
                        if (lane == 0) tma_reduce_add_3d(&cmap, stg, (int)cj, (int)rs, f);
                    }
                }
                if (++ab == 2) {
                    ab = 0;
                    acc_ph ^= 1u;
                }
            }
        }
    } else if (warp >= 2 + kEpiWarps) {
        // ---- A loaders: warp -> TMEM lane quadrant (warp % 4), hi (first four warps) or lo; each
        // fills the unit's A as soon as the previous unit's MMAs release it, the first K slice
        // loaded before that and the next one in flight while the current one is stored ----
        const int q = warp & 3, which = (warp - 2 - kEpiWarps) >> 2;
        int js = 0;
        uint32_t jph = 0, aph = 0;
        for (;;) {
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
            const int64_t rr = i * kTcM + q * 32 + lane;  // panel row (< rp)
            const float* src = panel + (size_t)f * 2 * half_floats + (size_t)which * half_floats;
            auto load_slice = [&](int kb, float (&v)[32]) {
                const float4* row = reinterpret_cast<const float4*>(src + ((size_t)kb * rp + rr) * 32);
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const float4 x = row[c ^ (int)(rr & 7)];
                    v[4 * c] = x.x;
                    v[4 * c + 1] = x.y;
                    v[4 * c + 2] = x.z;
                    v[4 * c + 3] = x.w;
                }
            };
            float v[32];
            load_slice(0, v);
            uint32_t got = 1;
            if (lane == 0) got = mbar_wait(aempty, aph ^ 1u, abort_flag, err) ? 1u : 0u;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) break;
            aph ^= 1u;
            tc_fence_after();
            for (int kb = 0; kb < nkc; ++kb) {
                float nv[32];
                if (kb + 1 < nkc) load_slice(kb + 1, nv);
                tmem_st32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kTmemAHi + 128 * which + 32 * kb), v);
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = nv[j];
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(afull);
        }
    }
    if (warp >= 2 && warp < 2 + kEpiWarps && lane == 0)
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // this warp's reduces are complete
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

} // namespace

size_t tc_panel_bytes_per_freq(const TallGeometry& g) {
    const int64_t rp = (g.rows + kTcM - 1) / kTcM * kTcM;
    return (size_t)2 * (128 / 4) * (size_t)rp * 16;
}

int launch_update32_tc(const TallGeometry& g, int64_t nf, float* a, int64_t kb0, int kdim, int64_t c_begin,
                       float* panel, unsigned long long* sched, unsigned long long* err, cudaStream_t s, int max_ctas,
                       int64_t row_min) {
    if (kdim <= 0 || kdim > 128 || kdim % kTcKc != 0)
        fail(GWB200_BAD_SHAPE, "tcgen05 update: K must be 32, 64, 96 or 128");
    const int64_t T = (g.n_pad - c_begin + kTcN - 1) / kTcN;  // the last column tile may be 64 wide
    if (T <= 0 || nf <= 0) return 0;
    const int64_t H = g.rows - c_begin;
    const int64_t NI = (H + kTcM - 1) / kTcM, rp = NI * kTcM;
    const int nkc = kdim / kTcKc;
    {
        const int64_t total = (int64_t)nkc * rp * 8;
        const unsigned gx = (unsigned)std::min<int64_t>((total + 255) / 256, 4096);
        k_split_panel32<<<dim3(gx, (unsigned)nf), 256, 0, s>>>(a, g.ld, g.stride, kb0, nkc, c_begin, g.rows, rp, panel);
        GWB_LAUNCH("k_split_panel32");
    }
    GWB_CUDA(cudaFuncSetAttribute(k_update32_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    // C of the chunk as a 3-D FP32 tensor (columns, rows, frequencies), 32 x 32 boxes, 128B swizzle
    CUtensorMap cmap;
    {
        static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
        static std::once_flag once;
        std::call_once(once, [] {
            void* fn = nullptr;
            cudaDriverEntryPointQueryResult q{};
            if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess)
                encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        });
        if (!encode) fail(GWB200_CUDA_ERROR, "cuTensorMapEncodeTiled is not available from the driver");
        const cuuint64_t dims[3] = {(cuuint64_t)g.n_pad, (cuuint64_t)g.rows, (cuuint64_t)nf};
        const cuuint64_t strides[2] = {(cuuint64_t)g.ld * 4, (cuuint64_t)g.stride * 4};
        const cuuint32_t box[3] = {32, 32, 1}, estr[3] = {1, 1, 1};
        const CUresult r = encode(&cmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, a, dims, strides, box, estr,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                  CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) fail(GWB200_CUDA_ERROR, "cuTensorMapEncodeTiled failed for the tall matrices");
    }
    UnitSpace us;
    us.T = T;
    us.NI = NI;
    us.NS = (T + kTcSeg - 1) / kTcSeg;
    // row_min > c_begin (the solve-only pass): only the row tiles that reach row_min have work
    const int64_t i0 = std::max<int64_t>(0, (row_min - c_begin) / kTcM);
    us.per_f = (NI - i0) * us.NS;
    us.total = nf * us.per_f;
    GWB_CUDA(cudaMemsetAsync(sched, 0, sizeof(unsigned long long), s));
    const unsigned grid = (unsigned)std::min<int64_t>(us.total, max_ctas > 0 ? std::min(max_ctas, sm_count()) : sm_count());
    // GWB200_TEST_EXPIRE_WAIT=1 (tests only): one CTA withholds its first operand stage, so a
    // device wait expires and the call reports GWB200_DEVICE_TIMEOUT with the context intact.
    const char* expire = std::getenv("GWB200_TEST_EXPIRE_WAIT");
    const int withhold = (expire && expire[0] == '1') ? 1 : 0;
    k_update32_tc<<<grid, kTcThreads, kTcSmem, s>>>(a, g.ld, g.stride, c_begin, g.rows, g.n_pad, row_min, nkc, panel, rp,
                                                     us, sched, err, withhold, cmap);
    GWB_LAUNCH("k_update32_tc");
    return 2;
}

} // namespace gwb200
