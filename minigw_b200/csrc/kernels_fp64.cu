// kernels_fp64.cu -- plain-form (FP64) screening kernels for sm_100a.
//
// Per frequency f the reference builds eps_left = I - diag(Pi0) V and forms
// W_c = eps_left^{-1} diag(Pi0) with a complex LU (src/workspace/screening_workspace.cpp:21-66,
// src/workspace/device_screening_workspace.cu:337-374), then evaluates x^T W_c x per panel
// (src/workspace/screening_workspace.cpp:69-102).  At eta = 0, Pi0 = -D with
// D = 4 delta / (w^2 + delta^2) > 0, and
//     x^T W_c x = -|| L^{-1} D^1/2 x ||^2,   L L^T = eps = I + D^1/2 V D^1/2  (SPD, eigenvalues >= 1).
// The kernels below factor the tall matrix [eps ; (D^1/2 X)^T] with one right-looking
// blocked Cholesky: its lower rows become (L^{-1} D^1/2 X)^T, whose row norms are the
// quadratic forms.  All arithmetic is FP64; the O(n^3) and O(n^2 m) work runs on FP64
// tensor cores (mma.sync m8n8k4 f64, DMMA).
#include "internal.cuh"

#include <array>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include <cmath>
#include <cstdlib>

namespace gwb200 {
namespace {

// ---------------------------------------------------------------------------
// Gathers (bit-exact copies).

// The device keeps only the (pq|o.) block of the ERI: pqo[(p*nmo + q)*nocc + i][s] = eri[p,q,i,s]
// for i < nocc (every element the path reads except the exchange diagonal), uploaded by one 2D
// copy whose rows are nocc*nmo contiguous doubles.

// V[jb, ia] = eri[j, b, i, a]  (src/gw/sigma.cpp:56-71), row-major n x n.
// blockIdx.y strides over rows jb; threads over ia: for fixed (jb, i) the source run
// pqo[(j,b,i)][nocc:nmo] is contiguous, so loads coalesce in runs of nvir.
__global__ void k_gather_vph(const double* __restrict__ pqo, int nmo, int nocc, int n, double* __restrict__ v) {
    const int nvir = nmo - nocc;
    for (int jb = blockIdx.y; jb < n; jb += gridDim.y) {
        const int j = jb / nvir, b = nocc + jb % nvir;
        const size_t base = ((size_t)j * nmo + b) * (size_t)nocc * nmo;
        for (int ia = blockIdx.x * blockDim.x + threadIdx.x; ia < n; ia += gridDim.x * blockDim.x) {
            const int i = ia / nvir, a = nocc + ia % nvir;
            v[(size_t)jb * n + ia] = pqo[base + (size_t)i * nmo + a];
        }
    }
}

// Xt[s*nmo + k, ia] = eri[p_s, k, i, a]  (src/workspace/pq_ph_panel.cpp:25-47, transposed so
// that every right-hand side is a contiguous row), row-major m x n.
__global__ void k_gather_panel(const double* __restrict__ pqo, int nmo, int nocc, int n,
                               const int64_t* __restrict__ states, int m, double* __restrict__ xt) {
    const int nvir = nmo - nocc;
    for (int row = blockIdx.y; row < m; row += gridDim.y) {
        const int s = row / nmo, k = row % nmo;
        const size_t p = (size_t)states[s];
        const size_t base = (p * nmo + k) * (size_t)nocc * nmo;
        for (int ia = blockIdx.x * blockDim.x + threadIdx.x; ia < n; ia += gridDim.x * blockDim.x) {
            const int i = ia / nvir, a = nocc + ia % nvir;
            xt[(size_t)row * n + ia] = pqo[base + (size_t)i * nmo + a];
        }
    }
}

// Sigma_x[p,p] = -sum_{i<nocc} eri[p,i,p,i] in the reference's order (src/gw/sigma.cpp:29-36);
// xdiag[p*nocc + i] = eri[p,i,p,i] (uploaded element by element).
__global__ void k_sigma_x_diag(const double* __restrict__ xdiag, int nmo, int nocc, double* __restrict__ out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nmo) return;
    double value = 0.0;
    for (int i = 0; i < nocc; ++i) value = __dsub_rn(value, xdiag[(size_t)p * nocc + i]);
    out[p] = value;
}

// delta[ph] = e_a - e_i with ph = i*nvir + a_vir (include/gw/particle_hole.hpp:22-35).
__global__ void k_delta(const double* __restrict__ mo, int nmo, int nocc, double* __restrict__ delta,
                        int* __restrict__ bad_gap) {
    const int nvir = nmo - nocc, n = nocc * nvir;
    const int ph = blockIdx.x * blockDim.x + threadIdx.x;
    if (ph >= n) return;
    const int i = ph / nvir, a = nocc + ph % nvir;
    const double d = __dsub_rn(mo[a], mo[i]);
    delta[ph] = d;
    if (!(d > 0.0)) atomicExch(bad_gap, 1);
}

// dvec[f, c] = sqrt(D_f[c]) with D = -Pi0(i w_f) = 4 delta / (w^2 + delta^2); zero padding.
__global__ void k_scale_vectors(const double* __restrict__ delta, int n, int n_pad, const double* __restrict__ omega,
                                int nf, double* __restrict__ dvec) {
    const int f = blockIdx.y;
    const double w = omega[f];
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_pad; c += gridDim.x * blockDim.x) {
        double val = 0.0;
        if (c < n) {
            const double d = delta[c];
            val = sqrt(4.0 * d / (w * w + d * d));
        }
        dvec[(size_t)f * n_pad + c] = val;
    }
}

// Build the tall matrices of nf frequencies.  Thread (r, c): rows r < n_pad hold the lower
// triangle of eps (c <= r), rows r >= n_pad hold d_c * Xt[r - n_pad, c].  V and Xt are read
// once per chunk; the loop over frequencies reuses the value from registers.
__global__ void k_build_tall(int64_t n, int64_t m, int64_t n_pad, int64_t ld, int64_t stride,
                             const double* __restrict__ v, const double* __restrict__ xt,
                             const double* __restrict__ dvec, int nf, double* __restrict__ a) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_pad) return;
    const int64_t rows = n_pad + ((m + kNb - 1) / kNb) * kNb;
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
    if (r < n_pad) {
        if (c > r) continue;
        const bool inside = (r < n) && (c < n);
        const double vrc = inside ? v[r * n + c] : 0.0;
        const double diag = (r == c) ? 1.0 : 0.0;
        for (int f = 0; f < nf; ++f) {
            const double* d = dvec + (size_t)f * n_pad;
            a[(size_t)f * stride + r * ld + c] = fma(d[r] * vrc, d[c], diag);
        }
    } else {
        const int64_t j = r - n_pad;
        const double x = (j < m && c < n) ? xt[j * n + c] : 0.0;
        for (int f = 0; f < nf; ++f) {
            a[(size_t)f * stride + r * ld + c] = dvec[(size_t)f * n_pad + c] * x;
        }
    }
    }
}

// ---------------------------------------------------------------------------
// DMMA 64x64x64 tile product:  acc += sgn * As(64x64) * Bs(64x64)^T, both in shared memory,
// row-major with stride kLds.  8 warps; warp w owns rows 16*(w/2)..+15, cols 32*(w%2)..+31,
// i.e. 2 x 4 fragments of the m8n8k4 f64 MMA.  Fragment layout (PTX ISA, mma.m8n8k4 .f64):
// A: a = A[lane/4][lane%4]; B: b = B[lane%4][lane/4]; C: {C[lane/4][2*(lane%4)], +1}.
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <int LD, int KD>
__device__ __forceinline__ void tile_mma(const double* __restrict__ As, const double* __restrict__ Bs,
                                         double (&acc)[2][4][2], double sgn) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 16 * (w >> 1), c0 = 32 * (w & 1);
#pragma unroll 4
    for (int kk = 0; kk < KD; kk += 4) {
        double af[2], bf[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) af[i] = sgn * As[(r0 + 8 * i + g) * LD + kk + t];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = Bs[(c0 + 8 * j + g) * LD + kk + t];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], af[i], bf[j]);
    }
}

__device__ __forceinline__ void tile_mma_64(const double* __restrict__ As, const double* __restrict__ Bs,
                                            double (&acc)[2][4][2], double sgn) {
    tile_mma<kLds, kNb>(As, Bs, acc, sgn);
}

// Copy a 64x64 tile (global row stride ld) into shared memory (stride kLds), 16-byte loads.
__device__ __forceinline__ void load_tile_64(double* __restrict__ s, const double* __restrict__ gsrc, int64_t ld) {
    for (int idx = threadIdx.x; idx < 64 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c2 = idx & 31;
        const double2 v = *reinterpret_cast<const double2*>(gsrc + (size_t)r * ld + 2 * c2);
        *reinterpret_cast<double2*>(s + r * kLds + 2 * c2) = v;
    }
}

// ---------------------------------------------------------------------------
// Step 1: factor the diagonal block A[k:k+64, k:k+64] of each frequency in shared memory,
// write L back and its inverse to linv (64x64 row-major, zero above the diagonal).
// A pivot that is not > 0 (or NaN) records the 1-based global pivot row in *err_pivot
// (minimum over all frequencies) and is replaced by 1 so the factorisation stays finite.
__global__ void __launch_bounds__(256) k_potrf_diag(double* __restrict__ a, int64_t ld, int64_t stride, int64_t k,
                                                    double* __restrict__ linv, unsigned long long* err_pivot) {
    extern __shared__ double smem[];
    constexpr int L = kNb + 1;
    double* T = smem;            // 64 x 65: the block, then L
    double* Y = smem + kNb * L;  // 64 x 65: L^{-1}
    double* A = a + (size_t)blockIdx.x * stride + k * ld + k;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int i = idx / kNb, j = idx % kNb;
        T[i * L + j] = (j <= i) ? A[(size_t)i * ld + j] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kNb; ++j) {
        if (tid == 0) {
            double piv = T[j * L + j];
            if (!(piv > 0.0)) {
                atomicMin(err_pivot, (unsigned long long)(k + j + 1));
                piv = 1.0;
            }
            T[j * L + j] = sqrt(piv);
        }
        __syncthreads();
        const double rjj = 1.0 / T[j * L + j];
        for (int i = j + 1 + tid; i < kNb; i += blockDim.x) T[i * L + j] *= rjj;
        __syncthreads();
        // rank-1 update of the trailing lower triangle on a 16 x 16 thread grid (no index division)
        for (int i = j + 1 + (tid >> 4); i < kNb; i += 16) {
            const double lij = T[i * L + j];
            for (int l = j + 1 + (tid & 15); l <= i; l += 16) T[i * L + l] -= lij * T[l * L + j];
        }
        __syncthreads();
    }
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int i = idx / kNb, j = idx % kNb;
        if (j <= i) A[(size_t)i * ld + j] = T[i * L + j];
    }
    // Inverse of the lower-triangular block by forward substitution: column `col` is owned by the
    // four lanes 4*col..4*col+3 of one warp (all 256 threads busy), which split each dot product
    // and combine it with two xor-shuffles.
    {
        const int col = tid >> 2, part = tid & 3;
        for (int i = 0; i < kNb; ++i) {
            double sum = 0.0;
            if (i > col)
                for (int l = col + part; l < i; l += 4) sum = fma(T[i * L + l], Y[l * L + col], sum);
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 2);
            if (part == 0) {
                double y;
                if (i < col) y = 0.0;
                else if (i == col) y = 1.0 / T[i * L + i];
                else y = -sum / T[i * L + i];
                Y[i * L + col] = y;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    double* out = linv + (size_t)blockIdx.x * kNb * kNb;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) out[idx] = Y[(idx / kNb) * L + idx % kNb];
}

// Step 2: panel solve.  Rows [k+64, rows) of block column k: P = A[:, k:k+64] * Linv^T, in place.
// Rows in the right-hand-side block also add their squared norms to qacc (one thread per row,
// fixed order, so the accumulation is deterministic).
__global__ void __launch_bounds__(256) k_trsm_panel(double* __restrict__ a, int64_t ld, int64_t stride, int64_t k,
                                                    int64_t n_pad, int64_t rows, const double* __restrict__ linv,
                                                    double* __restrict__ qacc, int64_t ldq) {
    extern __shared__ double smem[];
    double* Ps = smem;              // 64 x kLds
    double* Ls = smem + 64 * kLds;  // 64 x kLds
    const int f = blockIdx.y;
    const int64_t r0 = k + kNb + (int64_t)blockIdx.x * kNb;
    if (r0 >= rows) return;
    double* A = a + (size_t)f * stride;
    load_tile_64(Ps, A + r0 * ld + k, ld);
    load_tile_64(Ls, linv + (size_t)f * kNb * kNb, kNb);
    __syncthreads();
    double acc[2][4][2] = {};
    tile_mma_64(Ps, Ls, acc, 1.0);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rr = 16 * (w >> 1), cc = 32 * (w & 1);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Ps[(rr + 8 * i + g) * kLds + cc + 8 * j + 2 * t] = acc[i][j][0];
            Ps[(rr + 8 * i + g) * kLds + cc + 8 * j + 2 * t + 1] = acc[i][j][1];
        }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 64 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c2 = idx & 31;
        *reinterpret_cast<double2*>(A + (size_t)(r0 + r) * ld + k + 2 * c2) =
            *reinterpret_cast<const double2*>(Ps + r * kLds + 2 * c2);
    }
    if (r0 >= n_pad && threadIdx.x < kNb) {
        const int r = threadIdx.x;
        double s = 0.0;
        for (int j = 0; j < kNb; ++j) s = fma(Ps[r * kLds + j], Ps[r * kLds + j], s);
        qacc[(size_t)f * ldq + (r0 - n_pad + r)] += s;
    }
}

// Step 3: update C -= sum_chunks P_i P_j^T of the output column tiles [tc0, tc0+T) (64-wide,
// absolute tile indices): every tile on or below the diagonal in the square block, then every
// tile of the right-hand-side rows.  The contraction runs over nk 64-wide column chunks of the
// factored panels starting at column kb0, one chunk in shared memory at a time (cp.async), so
// K = 64*nk costs one read and one write of C: the outer-block trailing update uses nk = 2
// (16 flop per byte of C traffic), the narrow look-left update of an inner block nk = 1..q-1.
// C is loaded into registers before the chunk loop and added in the epilogue, so its latency
// overlaps the MMAs.
__device__ __forceinline__ void cp_async_16(double* smem_dst, const double* gsrc) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}
// Update kernel family: 64x64 output tile per CTA, warp tile (8*WM) x (8*WN) of m8n8k4 DMMA
// fragments, K streamed in KC-wide slices through a STAGES-deep cp.async pipeline.
template <int KC>
__device__ __forceinline__ void load_slice_async(double* __restrict__ s, const double* __restrict__ gsrc, int64_t ld,
                                                 int nthreads) {
    constexpr int LD = KC + 4;  // (KC+4)*8 bytes per row: the 8 rows of one fragment load hit distinct banks
    for (int idx = threadIdx.x; idx < 64 * (KC / 2); idx += nthreads) {
        const int r = idx / (KC / 2), c2 = idx % (KC / 2);
        cp_async_16(s + r * LD + 2 * c2, gsrc + (size_t)r * ld + 2 * c2);
    }
}

template <int WM, int WN, int LD, int KD>
__device__ __forceinline__ void warp_mma(const double* __restrict__ As, const double* __restrict__ Bs,
                                         double (&acc)[WM][WN][2], int r0, int c0) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int kk = 0; kk < KD; kk += 4) {
        double af[WM], bf[WN];
#pragma unroll
        for (int i = 0; i < WM; ++i) af[i] = -As[(r0 + 8 * i + g) * LD + kk + t];
#pragma unroll
        for (int j = 0; j < WN; ++j) bf[j] = Bs[(c0 + 8 * j + g) * LD + kk + t];
#pragma unroll
        for (int i = 0; i < WM; ++i)
#pragma unroll
            for (int j = 0; j < WN; ++j) dmma_8x8x4(acc[i][j], af[i], bf[j]);
    }
}

template <int WM, int WN, int KC, int STAGES>
struct UpdateCfg {
    static constexpr int kWarpsM = 64 / (8 * WM), kWarpsN = 64 / (8 * WN);
    static constexpr int kThreads = 32 * kWarpsM * kWarpsN;
    static constexpr int kLd = KC + 4;
    static constexpr size_t kSmem = (size_t)STAGES * 2 * 64 * kLd * sizeof(double);
    static constexpr int kMinBlocks = (227 * 1024) / (int)kSmem < 4 ? (227 * 1024) / (int)kSmem : 4;
};

template <int WM, int WN, int KC, int STAGES>
__global__ void __launch_bounds__(UpdateCfg<WM, WN, KC, STAGES>::kThreads, UpdateCfg<WM, WN, KC, STAGES>::kMinBlocks)
    k_update(double* __restrict__ a, int64_t ld, int64_t stride, int64_t kb0, int nk, int64_t tc0, int64_t T,
             int64_t nsq) {
    using Cfg = UpdateCfg<WM, WN, KC, STAGES>;
    constexpr int LD = Cfg::kLd;
    extern __shared__ double smem[];
    auto stage = [&](int st, int which) { return smem + (2 * st + which) * 64 * LD; };
    const int f = blockIdx.y;
    const int64_t x = blockIdx.x;
    const int64_t L = nsq - tc0;                     // square row tiles of the first column tile
    const int64_t n_square = T * L - T * (T - 1) / 2;
    int64_t c, tr;
    if (x < n_square) {
        // column offset c: largest c with cum(c) = c*L - c(c-1)/2 <= x
        const double b = 2.0 * (double)L + 1.0;
        c = (int64_t)((b - sqrt(fmax(b * b - 8.0 * (double)x, 0.0))) * 0.5);
        auto cum = [L](int64_t cc) { return cc * L - cc * (cc - 1) / 2; };
        while (c > 0 && cum(c) > x) --c;
        while (c + 1 < T && cum(c + 1) <= x) ++c;
        tr = tc0 + c + (x - cum(c));
    } else {
        const int64_t y = x - n_square;
        c = y % T;
        tr = nsq + y / T;
    }
    const int64_t ri = tr * kNb, cj = (tc0 + c) * kNb;
    double* A = a + (size_t)f * stride;
    const int nsub = nk * (kNb / KC);
    // prologue: STAGES-1 slices in flight
#pragma unroll
    for (int p = 0; p < STAGES - 1; ++p) {
        if (p < nsub) {
            const int64_t kc = kb0 + (int64_t)p * KC;
            load_slice_async<KC>(stage(p, 0), A + ri * ld + kc, ld, Cfg::kThreads);
            load_slice_async<KC>(stage(p, 1), A + cj * ld + kc, ld, Cfg::kThreads);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    }
    const int w = threadIdx.x >> 5;
    const int r0 = 8 * WM * (w / Cfg::kWarpsN), c0 = 8 * WN * (w % Cfg::kWarpsN);
    double acc[WM][WN][2] = {};
    for (int sc = 0; sc < nsub; ++sc) {
        const int pf = sc + STAGES - 1;  // slice to prefetch into the stage freed last iteration
        if (pf < nsub) {
            const int64_t kc = kb0 + (int64_t)pf * KC;
            load_slice_async<KC>(stage(pf % STAGES, 0), A + ri * ld + kc, ld, Cfg::kThreads);
            load_slice_async<KC>(stage(pf % STAGES, 1), A + cj * ld + kc, ld, Cfg::kThreads);
        }
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 1));
        __syncthreads();
        warp_mma<WM, WN, LD, KC>(stage(sc % STAGES, 0), stage(sc % STAGES, 1), acc, r0, c0);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int i = 0; i < WM; ++i)
#pragma unroll
        for (int j = 0; j < WN; ++j) {
            double2* pc = reinterpret_cast<double2*>(A + (size_t)(ri + r0 + 8 * i + g) * ld + cj + c0 + 8 * j + 2 * t);
            double2 v = *pc;
            v.x += acc[i][j][0];
            v.y += acc[i][j][1];
            *pc = v;
        }
}

// Variant table of the update kernel (selected by GWB200_UPDATE_VARIANT, default kDefaultUpdateVariant).
struct UpdateVariant {
    void (*fn)(double*, int64_t, int64_t, int64_t, int, int64_t, int64_t, int64_t);
    int threads;
    size_t smem;
    const char* name;
};
template <int WM, int WN, int KC, int ST>
UpdateVariant make_variant(const char* name) {
    using Cfg = UpdateCfg<WM, WN, KC, ST>;
    return {k_update<WM, WN, KC, ST>, Cfg::kThreads, Cfg::kSmem, name};
}
const UpdateVariant kVariants[] = {
    make_variant<2, 4, 32, 2>("w16x32_k32_s2"),
    make_variant<4, 4, 32, 2>("w32x32_k32_s2"),
    make_variant<4, 4, 16, 3>("w32x32_k16_s3"),
    make_variant<2, 4, 32, 3>("w16x32_k32_s3"),
    make_variant<4, 8, 32, 2>("w32x64_k32_s2"),
    make_variant<4, 4, 32, 3>("w32x32_k32_s3"),
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

}  // namespace

int fp64_update_mode() {  // GWB200_FP64_UPDATE: 1 = dmma (FP64 pipe only), 2 = ozaki (int8 emulation), 0 = tuned
    const char* env = std::getenv("GWB200_FP64_UPDATE");
    if (env && std::strcmp(env, "dmma") == 0) return 1;
    if (env && std::strcmp(env, "ozaki") == 0) return 2;
    return 0;
}

namespace {

int env_update_variant() {  // GWB200_UPDATE_VARIANT forces a variant; -1 if unset or out of range
    if (const char* env = std::getenv("GWB200_UPDATE_VARIANT")) {
        const int e = std::atoi(env);
        if (e >= 0 && e < kNumVariants) return e;
    }
    return -1;
}

void launch_variant(int v, const TallGeometry& g, int64_t nf, double* a, int64_t kb0, int nk, int64_t tc0, int64_t T,
                    cudaStream_t s) {
    const UpdateVariant& uv = kVariants[v];
    const int64_t nsq = g.n_pad / kNb, nrt = g.rows / kNb;
    const int64_t L = nsq - tc0;
    const int64_t tiles = T * L - T * (T - 1) / 2 + T * (nrt - nsq);
    if (tiles <= 0) return;
    uv.fn<<<dim3((unsigned)tiles, (unsigned)nf), uv.threads, uv.smem, s>>>(a, g.ld, g.stride, kb0, nk, tc0, T, nsq);
    GWB_LAUNCH("k_update");
}

std::mutex g_tune_mu;
std::map<std::array<int64_t, 6>, int> g_tuned;  // (device, n_pad, rows, nf, int8 candidate, all) -> variant

// q_out[f, j] = -qacc[f, j]  (x^T W_c x = -||L^{-1} D^1/2 x||^2).
__global__ void k_negate_copy(const double* __restrict__ qacc, int nf, int m, int64_t ldq_in, double* __restrict__ q,
                              int64_t ldq_out) {
    const int f = blockIdx.y;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        q[(size_t)f * ldq_out + j] = -qacc[(size_t)f * ldq_in + j];
}

} // namespace

int launch_gather_vph(const double* pqo, int64_t nmo, int64_t nocc, double* v, cudaStream_t s) {
    const int n = (int)(nocc * (nmo - nocc));
    dim3 grid((unsigned)std::min<int64_t>((n + 255) / 256, 64), (unsigned)std::min(n, 65535));
    k_gather_vph<<<grid, 256, 0, s>>>(pqo, (int)nmo, (int)nocc, n, v);
    GWB_LAUNCH("k_gather_vph");
    return 1;
}

int launch_gather_panel(const double* pqo, int64_t nmo, int64_t nocc, const int64_t* states, int64_t nstates,
                        double* xt, cudaStream_t s) {
    const int n = (int)(nocc * (nmo - nocc));
    const int m = (int)(nstates * nmo);
    dim3 grid((unsigned)std::min<int64_t>((n + 255) / 256, 64), (unsigned)std::min(m, 65535));
    k_gather_panel<<<grid, 256, 0, s>>>(pqo, (int)nmo, (int)nocc, n, states, m, xt);
    GWB_LAUNCH("k_gather_panel");
    return 1;
}

int launch_sigma_x_diag(const double* xdiag, int64_t nmo, int64_t nocc, double* out, cudaStream_t s) {
    k_sigma_x_diag<<<(unsigned)((nmo + 127) / 128), 128, 0, s>>>(xdiag, (int)nmo, (int)nocc, out);
    GWB_LAUNCH("k_sigma_x_diag");
    return 1;
}

int launch_delta(const double* mo, int64_t nmo, int64_t nocc, double* delta, int* bad_gap, cudaStream_t s) {
    const int64_t n = nocc * (nmo - nocc);
    k_delta<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mo, (int)nmo, (int)nocc, delta, bad_gap);
    GWB_LAUNCH("k_delta");
    return 1;
}

int launch_scale_vectors(const double* delta, int64_t n, int64_t n_pad, const double* omega, int64_t nf,
                         double* dvec, cudaStream_t s) {
    dim3 grid((unsigned)((n_pad + 255) / 256), (unsigned)nf);
    k_scale_vectors<<<grid, 256, 0, s>>>(delta, (int)n, (int)n_pad, omega, (int)nf, dvec);
    GWB_LAUNCH("k_scale_vectors");
    return 1;
}

int launch_build_tall(const TallGeometry& g, const double* v, const double* xt, const double* dvec, int64_t nf,
                      double* a, cudaStream_t s) {
    dim3 grid((unsigned)((g.n_pad + 255) / 256), (unsigned)std::min<int64_t>(g.rows, 65535));
    k_build_tall<<<grid, 256, 0, s>>>(g.n, g.m, g.n_pad, g.ld, g.stride, v, xt, dvec, (int)nf, a);
    GWB_LAUNCH("k_build_tall");
    return 1;
}

// Algorithmic flops of one update: 2 * K_true * (true lower elements of the output columns
// [c0, c1) intersected with [0, n) + m per output column).
static double update_flops(const TallGeometry& g, int64_t kb0, int nk, int64_t c0, int64_t c1) {
    const int64_t kt = std::max<int64_t>(0, std::min<int64_t>(kb0 + (int64_t)nk * kNb, g.n) - kb0);
    const int64_t a0 = std::min(c0, g.n), a1 = std::min(c1, g.n);
    const double cols = (double)(a1 - a0);
    const double lower = cols * (double)g.n - 0.5 * (double)(a0 + a1 - 1) * cols;  // sum_{c} (n - c)
    return 2.0 * (double)kt * (lower + (double)g.m * cols);
}

int tune_update_variant(const TallGeometry& g, int64_t nf, double* a, cudaStream_t s, void* oz,
                        unsigned long long* sched, unsigned long long* err_pivot, bool timed) {
    const int forced = env_update_variant();
    if (forced >= 0) return forced;
    const int64_t nsq = g.n_pad / kNb;
    if (nsq <= 2) return kDefaultUpdateVariant;  // no outer trailing update to tune on
    if (oz && fp64_update_mode() == 2) return kUpdateOzaki;
    if (fp64_update_mode() == 1) oz = nullptr;  // the FP64 pipe only
    // Untimed (memory-capped handles: the serving loop's slots, whose requests run side by side):
    // the non-persistent DMMA kernel, which leaves SMs to the other slots' kernels (the persistent
    // int8 kernel holds one CTA on every SM it gets); GWB200_FP64_UPDATE=ozaki still forces it.
    if (!timed) return kDefaultUpdateVariant;
    const char* all_env = std::getenv("GWB200_TUNE_ALL");
    const bool all = all_env && all_env[0] == '1';  // every DMMA variant, not only the default
    int dev = 0;
    GWB_CUDA(cudaGetDevice(&dev));
    const std::array<int64_t, 6> key = {dev, g.n_pad, g.rows, nf, oz ? 1 : 0, all ? 1 : 0};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return it->second;
    // Time the candidates on the largest trailing update of this geometry (K = 128 from column 0
    // onto columns [128, n_pad) and all RHS rows), in the workspace before the tall matrix is built
    // there: the values are irrelevant to the timing and are overwritten afterwards.
    cudaEvent_t e0, e1;
    GWB_CUDA(cudaEventCreate(&e0));
    GWB_CUDA(cudaEventCreate(&e1));
    float times[kNumVariants + 1] = {};
    auto time_it = [&](auto&& launch) {
        launch();  // warm-up
        GWB_CUDA(cudaEventRecord(e0, s));
        launch();
        GWB_CUDA(cudaEventRecord(e1, s));
        GWB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GWB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    };
    float best_ms = 0.f, def_ms = 0.f;
    int best = -1;
    for (int v = 0; v < kNumVariants; ++v) {
        if (!all && v != kDefaultUpdateVariant) continue;
        GWB_CUDA(cudaFuncSetAttribute(kVariants[v].fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kVariants[v].smem));
        const float ms = time_it([&] { launch_variant(v, g, nf, a, 0, 2, 2, nsq - 2, s); });
        times[v] = ms;
        if (v == kDefaultUpdateVariant) def_ms = ms;
        if (best < 0 || ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    if (oz) {  // the int8 emulation of the outer update (kernels_oz.cu), slicing included
        const float ms = time_it([&] { launch_update64_oz(g, nf, a, 0, 2 * kNb, oz, sched, err_pivot, s); });
        times[kUpdateOzaki] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = kUpdateOzaki;
        }
        // a wait that expired during the timing would have recorded pivot 0: start clean
        GWB_CUDA(cudaMemsetAsync(err_pivot, 0xFF, sizeof(unsigned long long), s));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (def_ms <= 1.03f * best_ms) best = kDefaultUpdateVariant;  // keep the default unless clearly beaten
    g_tuned[key] = best;
    if (const char* verbose = std::getenv("GWB200_VERBOSE"); verbose && verbose[0] == '1') {
        std::fprintf(stderr, "gwb200: update kernel for n_pad=%lld rows=%lld nf=%lld:", (long long)g.n_pad,
                     (long long)g.rows, (long long)nf);
        for (int v = 0; v < kNumVariants; ++v)
            if (all || v == kDefaultUpdateVariant) std::fprintf(stderr, " %s %.3f ms", kVariants[v].name, times[v]);
        if (oz) std::fprintf(stderr, " int8_emulation %.3f ms", times[kUpdateOzaki]);
        std::fprintf(stderr, " -> %s\n", update_variant_name(best));
    }
    return best;
}

const char* update_variant_name(int v) {
    if (v == kUpdateOzaki) return "int8_emulation";
    return (v >= 0 && v < kNumVariants) ? kVariants[v].name : "?";
}

int launch_factor_chunk(const TallGeometry& g, int64_t nf, double* a, double* linv, double* qacc,
                        unsigned long long* err_pivot, cudaStream_t s, UpdateProfiler* prof, int variant, void* oz,
                        unsigned long long* sched, int max_ctas) {
    const size_t smem = 2 * 64 * kLds * sizeof(double);
    const size_t smem_potrf = 2 * kNb * (kNb + 1) * sizeof(double);
    GWB_CUDA(cudaFuncSetAttribute(k_trsm_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const bool use_oz = oz && variant == kUpdateOzaki;  // outer updates emulated; look-left on DMMA
    if (variant < 0 || variant >= kNumVariants)  // untuned caller: GWB200_UPDATE_VARIANT, else the default
        variant = env_update_variant() >= 0 ? env_update_variant() : kDefaultUpdateVariant;
    const UpdateVariant& uv = kVariants[variant];
    GWB_CUDA(cudaFuncSetAttribute(uv.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)uv.smem));
    GWB_CUDA(cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
    const int64_t nsq = g.n_pad / kNb;   // square tile rows/cols
    const int64_t nrt = g.rows / kNb;    // all tile rows
    constexpr int64_t kInner = 2;        // 64-wide inner blocks per outer block
    int launches = 0;
    // with the int8-emulated outer updates, the profiler times those alone (the look-left updates
    // that stay on DMMA are a few percent of the flops)
    UpdateProfiler* lprof = use_oz ? nullptr : prof;
    auto update = [&](int64_t kb0, int nk, int64_t tc0, int64_t T) {
        const int64_t L = nsq - tc0;
        const int64_t tiles = T * L - T * (T - 1) / 2 + T * (nrt - nsq);
        if (tiles <= 0) return;
        dim3 grid((unsigned)tiles, (unsigned)nf);
        if (lprof) lprof->begin();
        uv.fn<<<grid, uv.threads, uv.smem, s>>>(a, g.ld, g.stride, kb0, nk, tc0, T, nsq);
        GWB_LAUNCH("k_update");
        if (lprof) lprof->end((double)nf * update_flops(g, kb0, nk, tc0 * kNb, (tc0 + T) * kNb));
        ++launches;
    };
    for (int64_t ob = 0; ob < nsq; ob += kInner) {
        const int64_t q = std::min(kInner, nsq - ob);
        for (int64_t j = 0; j < q; ++j) {
            const int64_t kt = ob + j;
            const int64_t k = kt * kNb;
            if (j > 0) update(ob * kNb, (int)j, kt, 1);  // look-left: earlier inner blocks onto this column
            k_potrf_diag<<<(unsigned)nf, 256, smem_potrf, s>>>(a, g.ld, g.stride, k, linv, err_pivot);
            GWB_LAUNCH("k_potrf_diag");
            ++launches;
            const int64_t below = g.rows - (k + kNb);
            if (below > 0) {
                dim3 grid((unsigned)(below / kNb), (unsigned)nf);
                k_trsm_panel<<<grid, 256, smem, s>>>(a, g.ld, g.stride, k, g.n_pad, g.rows, linv, qacc, g.m_pad);
                GWB_LAUNCH("k_trsm_panel");
                ++launches;
            }
        }
        const int64_t tc0 = ob + q;
        if (tc0 < nsq) {  // outer-block trailing update, K = 64*q (= 128 whenever columns remain)
            if (use_oz && q == kInner) {
                if (prof) prof->begin();
                launches += launch_update64_oz(g, nf, a, ob * kNb, tc0 * kNb, oz, sched, err_pivot, s, max_ctas);
                if (prof) prof->end((double)nf * update_flops(g, ob * kNb, (int)q, tc0 * kNb, nsq * kNb));
            } else {
                update(ob * kNb, (int)q, tc0, nsq - tc0);
            }
        }
    }
    return launches;
}

int launch_negate_copy(const double* qacc, int64_t nf, int64_t m, int64_t ldq_in, double* q_out, int64_t ldq_out,
                       cudaStream_t s) {
    dim3 grid((unsigned)std::min<int64_t>((m + 255) / 256, 64), (unsigned)nf);
    k_negate_copy<<<grid, 256, 0, s>>>(qacc, (int)nf, (int)m, ldq_in, q_out, ldq_out);
    GWB_LAUNCH("k_negate_copy");
    return 1;
}

} // namespace gwb200
