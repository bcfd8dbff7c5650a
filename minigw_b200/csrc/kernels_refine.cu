// kernels_refine.cu -- FP64 accuracy for the mixed form: one energy-functional correction.
//
// The mixed form factors eps = I + D^1/2 V D^1/2 in FP32 (kernels_f32.cu / kernels_tc.cu): the
// tall matrix ends as L~ (FP32, eps ~ L~ L~^T) and the rows w_j^T = (L~^{-1} b_j)^T with
// b_j = D^1/2 x_j, whose squared norms carry FP32-level error (~1e-7 relative).  For z_j close to
// eps^{-1} b_j the functional
//     F(z) = 2 b^T z - z^T eps z
// is stationary at z* = eps^{-1} b with F(z*) = b^T eps^{-1} b = -q, and F(z) = F(z*) - e^T eps e for
// e = z - z*: its error is quadratic in the solve error.  With z_j = L~^{-T} w_j (FP32, relative error
// ~ cond(eps) * 1e-7) and F evaluated in FP64,
//     q~_j = -F(z_j) = -(2 t1 - t2 - t3),  t1 = x_j^T y_j,  t2 = z_j^T z_j,  t3 = y_j^T V y_j,
// with y_j = D^1/2 z_j (FP64), is within ~1e-14 relative of the FP64 forms (the error is
// ||e||_eps^2 >= 0, so q~ >= q).
//
// Steps per frequency chunk (after the mixed factorisation of the chunk):
//   k_flip_tiles32 + k_reverse_rows32  turn L~ into P L~^T P (P the index reversal of [0, n_pad)),
//                 which is lower triangular, and reverse every RHS row: the backward solve
//                 L~^T z = w becomes the forward solve (P L~^T P)(P z) = P w, which the mixed
//                 factorisation's kernels run in their solve-only mode (the RHS rows alone against
//                 the finished factor) -> the RHS rows end as (P z_j)^T;
//   k_refine_prep   y_j = D^1/2 z_j into an FP64 buffer, t1 and t2 per row (FP64, fixed-order sums);
//   k_gram_sq       t3 = || C^T y_j ||^2 with V = C C^T the pivoted Cholesky factor of V (below), on
//                   the FP64 tensor pipe (DMMA): per 64-row tile of C^T a partial sum;
//   k_refine_finish qacc_j = 2 t1 - t2 - t3 (the partials summed in a fixed order); the caller's
//                   negate-copy turns it into q~.
//
// V = C C^T: a pivoted Cholesky of V (FP64, once per loaded system, k_pchol_step), stopped when the
// largest remaining diagonal drops below 1e-13 of the largest diagonal of V.  C has as many columns r
// as the numerical rank of V: r = n for a full-rank V (then t3 costs 2 n^2 m flops per frequency, as
// the product V y would), fewer when V is rank deficient (2 r n m).  The truncated remainder R is
// positive semidefinite with diagonal below the threshold, so the term it leaves out, y^T R y, is
// at most 1e-13 max(diag V) ||y||_1^2.
//
// Everything here is deterministic: sums run in a fixed order, no floating-point atomics.
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace gwb200 {
namespace {

constexpr int kT = 64;      // tile edge
constexpr int kKs = 32;     // K slice of the DMMA GEMM (doubles)
constexpr int kLdk = kKs + 4;

// ---------------------------------------------------------------------------------------------
// In place: A <- P A^T P on the lower triangle of the top n_pad x n_pad block of each tall matrix,
// i.e. element (r, c) moves to (n_pad-1-c, n_pad-1-r).  64x64 tile (I, J) maps to tile
// (nb-1-J, nb-1-I) with local (ii, jj) -> (63-jj, 63-ii); lower tiles map to lower tiles and the
// upper part of a diagonal tile to the upper part, so whole tiles are exchanged.  One CTA per pair
// of tiles (I, J), J <= I, I + J <= nb - 1 (the pairs with I + J == nb - 1 map to themselves).
__global__ void __launch_bounds__(256) k_flip_tiles32(float* __restrict__ a, int64_t ld, int64_t stride, int nb) {
    __shared__ float sx[kT][kT + 1];
    __shared__ float sy[kT][kT + 1];
    const int I = blockIdx.y, J = blockIdx.x;
    if (J > I || I + J > nb - 1) return;
    const int Ip = nb - 1 - J, Jp = nb - 1 - I;  // partner tile
    float* A = a + (size_t)blockIdx.z * stride;
    float* X = A + (size_t)I * kT * ld + (size_t)J * kT;
    float* Y = A + (size_t)Ip * kT * ld + (size_t)Jp * kT;
    const bool self = (Ip == I);
    for (int idx = threadIdx.x; idx < kT * kT; idx += blockDim.x) {
        const int r = idx / kT, c = idx % kT;
        sx[r][c] = X[(size_t)r * ld + c];
        if (!self) sy[r][c] = Y[(size_t)r * ld + c];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kT * kT; idx += blockDim.x) {
        const int r = idx / kT, c = idx % kT;
        Y[(size_t)r * ld + c] = sx[kT - 1 - c][kT - 1 - r];
        if (!self) X[(size_t)r * ld + c] = sy[kT - 1 - c][kT - 1 - r];
    }
}

// Reverse [0, width) of every right-hand-side row (rows row0 .. row0 + m_pad - 1).
__global__ void k_reverse_rows32(float* __restrict__ a, int64_t ld, int64_t stride, int64_t row0, int64_t width,
                                 int64_t m_pad) {
    for (int64_t j = blockIdx.y; j < m_pad; j += gridDim.y) {
        float* row = a + (size_t)blockIdx.z * stride + (size_t)(row0 + j) * ld;
        for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < width / 2;
             c += (int64_t)gridDim.x * blockDim.x) {
            const float t = row[c];
            row[c] = row[width - 1 - c];
            row[width - 1 - c] = t;
        }
    }
}

// One CTA per right-hand side j (row row0 + j of the tall matrix) of one frequency: z_j[i] =
// row[na-1-i] (the solve ran on indices reversed within na, the molecule's own n_pad; a batched
// molecule sits in the top-left corner of a bucket's larger matrix), y_j = dvec * z_j (FP64) into Y
// (m_pad x n_pad of the molecule, zero past n and past m), t1 = x_j . y_j and t2 = z_j . z_j
// (per-thread partial sums over a fixed stride, then a fixed tree).
__global__ void __launch_bounds__(256) k_refine_prep(const float* __restrict__ a, int64_t ld, int64_t stride,
                                                     int64_t row0, int64_t na, int64_t n, int64_t n_pad, int64_t m,
                                                     int64_t m_pad, const double* __restrict__ xt,
                                                     const double* __restrict__ dvec, double* __restrict__ y,
                                                     double* __restrict__ t12) {
    const int f = blockIdx.y;
    const int64_t j = blockIdx.x;
    const float* row = a + (size_t)f * stride + (size_t)(row0 + j) * ld;
    const double* d = dvec + (size_t)f * n_pad;
    double* yrow = y + ((size_t)f * m_pad + j) * n_pad;
    double s1 = 0.0, s2 = 0.0;
    const bool live = j < m;
    for (int64_t i = threadIdx.x; i < n_pad; i += blockDim.x) {
        double yi = 0.0;
        if (live && i < n) {
            const double zi = (double)row[na - 1 - i];
            yi = d[i] * zi;
            s1 = fma(xt[j * n + i], yi, s1);
            s2 = fma(zi, zi, s2);
        }
        yrow[i] = yi;
    }
    __shared__ double r1[256], r2[256];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            r1[threadIdx.x] += r1[threadIdx.x + w];
            r2[threadIdx.x] += r2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        t12[((size_t)f * m_pad + j) * 2] = r1[0];
        t12[((size_t)f * m_pad + j) * 2 + 1] = r2[0];
    }
}

// ---------------------------------------------------------------------------------------------
// DMMA m8n8k4 f64 (PTX ISA, mma.m8n8k4 .f64): A a = A[lane/4][lane%4]; B b = B[lane%4][lane/4];
// C {C[lane/4][2*(lane%4)], +1}.
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp16(double* sdst, const double* gsrc) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gsrc));
}

// 64 rows x kKs doubles of global (row stride ld) into shared memory (row stride kLdk).
__device__ __forceinline__ void load_slice(double* __restrict__ s, const double* __restrict__ g, int64_t ld) {
    for (int idx = threadIdx.x; idx < kT * (kKs / 2); idx += blockDim.x) {
        const int r = idx / (kKs / 2), c2 = idx % (kKs / 2);
        cp16(s + r * kLdk + 2 * c2, g + (size_t)r * ld + 2 * c2);
    }
}

// part[f][kt][j] = sum over the 64 rows k of C^T tile kt of (C^T[k, :] . Y_f[j, :])^2, K = n_pad.
// Grid (m_pad/64 column tiles j, r_pad/64 row tiles k, frequencies).  8 warps as 4 (rows) x 2
// (columns), warp tile 16 x 32; two-stage cp.async ring of 32-deep K slices.
__global__ void __launch_bounds__(256, 3) k_gram_sq(const double* __restrict__ ct, const double* __restrict__ y,
                                                    int64_t n_pad, int64_t m_pad, int64_t r_pad,
                                                    double* __restrict__ part) {
    extern __shared__ double gsm[];
    auto stage = [&](int st, int which) { return gsm + (2 * st + which) * kT * kLdk; };
    const int f = blockIdx.z;
    const int64_t kt = blockIdx.y, jt = blockIdx.x;
    const double* A = ct + (size_t)kt * kT * n_pad;
    const double* B = y + ((size_t)f * m_pad + (size_t)jt * kT) * n_pad;
    const int nsl = (int)(n_pad / kKs);
    load_slice(stage(0, 0), A, n_pad);
    load_slice(stage(0, 1), B, n_pad);
    asm volatile("cp.async.commit_group;\n" ::);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 16 * (w >> 1), c0 = 32 * (w & 1);
    double acc[2][4][2] = {};
    for (int sc = 0; sc < nsl; ++sc) {
        if (sc + 1 < nsl) {
            load_slice(stage((sc + 1) & 1, 0), A + (size_t)(sc + 1) * kKs, n_pad);
            load_slice(stage((sc + 1) & 1, 1), B + (size_t)(sc + 1) * kKs, n_pad);
            asm volatile("cp.async.commit_group;\n" ::);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        const double* As = stage(sc & 1, 0);
        const double* Bs = stage(sc & 1, 1);
#pragma unroll
        for (int kk = 0; kk < kKs; kk += 4) {
            double af[2], bf[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) af[i] = As[(r0 + 8 * i + g) * kLdk + kk + t];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) bf[jj] = Bs[(c0 + 8 * jj + g) * kLdk + kk + t];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) dmma(acc[i][jj], af[i], bf[jj]);
        }
        __syncthreads();
    }
    // column sums of squares: thread rows g, g+8 (of its warp's 16), columns c0 + 8 jj + 2 t + {0, 1};
    // over g by shuffles (fixed tree), over the four row warps through shared memory (fixed order)
    double cs[4][2];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double v = fma(acc[0][jj][h], acc[0][jj][h], acc[1][jj][h] * acc[1][jj][h]);
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            v += __shfl_xor_sync(0xffffffffu, v, 8);
            v += __shfl_xor_sync(0xffffffffu, v, 16);
            cs[jj][h] = v;
        }
    double* red = gsm;  // 4 x 64 after the main loop (the ring is no longer read)
    if (g == 0) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
#pragma unroll
            for (int h = 0; h < 2; ++h) red[(w >> 1) * kT + c0 + 8 * jj + 2 * t + h] = cs[jj][h];
    }
    __syncthreads();
    if (threadIdx.x < kT) {
        const int c = threadIdx.x;
        const double v = (red[c] + red[kT + c]) + (red[2 * kT + c] + red[3 * kT + c]);
        part[((size_t)f * (r_pad / kT) + kt) * m_pad + jt * kT + c] = v;
    }
}

// qacc[f][j] = 2 t1 - t2 - t3, t3 = sum over the row tiles of C^T in order.
__global__ void k_refine_finish(const double* __restrict__ t12, const double* __restrict__ part, int64_t m_pad,
                                int64_t nkt, int64_t m, double* __restrict__ qacc, int64_t ldq) {
    const int f = blockIdx.y;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    double t3 = 0.0;
    for (int64_t k = 0; k < nkt; ++k) t3 += part[((size_t)f * nkt + k) * m_pad + j];
    const double t1 = t12[((size_t)f * m_pad + j) * 2], t2 = t12[((size_t)f * m_pad + j) * 2 + 1];
    qacc[(size_t)f * ldq + j] = (2.0 * t1 - t2) - t3;
}

// ---------------------------------------------------------------------------------------------
// Pivoted Cholesky V = C C^T (FP64).  L is n x ldl row-major (L[i][k] = C[i][k], original row
// order); d[i] the remaining diagonal (d < 0 marks a pivoted row); cand[2][ncta] the per-CTA
// (value, index) maxima of the remaining diagonal, ping-pong between steps; state[0] = rank so far,
// state[1] = done.  Step k: every CTA reduces the previous step's candidates to the pivot p (the
// largest remaining diagonal, ties to the smallest index); if it is at most tau the factor is
// complete (rank k).  Else column k: L[i][k] = (V[p][i] - L[i][:k] . L[p][:k]) / sqrt(d_p) for the
// rows not yet pivoted (V is symmetric, so row p is read), L[p][k] = sqrt(d_p), 0 for pivoted rows;
// d[i] -= L[i][k]^2.  One warp per row.
struct Cand {
    double v;
    int64_t i;
};
__device__ __forceinline__ bool better(const Cand& a, const Cand& b) { return a.v > b.v || (a.v == b.v && a.i < b.i); }

__global__ void __launch_bounds__(256) k_pchol_init(const double* __restrict__ v, int64_t n, double* __restrict__ d,
                                                    Cand* __restrict__ cand0, long long* __restrict__ state) {
    __shared__ Cand sc[256];
    Cand best{-1.0, n};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double di = v[i * n + i];
        d[i] = di;
        const Cand c{di, i};
        if (better(c, best)) best = c;
    }
    sc[threadIdx.x] = best;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w && better(sc[threadIdx.x + w], sc[threadIdx.x])) sc[threadIdx.x] = sc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) cand0[blockIdx.x] = sc[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        state[0] = 0;
        state[1] = 0;
    }
}

__global__ void __launch_bounds__(256) k_pchol_step(const double* __restrict__ v, int64_t n, double* __restrict__ L,
                                                    int64_t ldl, double* __restrict__ d, const Cand* __restrict__ cin,
                                                    Cand* __restrict__ cout, int ncta, int64_t k, double tau,
                                                    long long* __restrict__ state) {
    __shared__ Cand sc[256];
    __shared__ Cand piv;
    if (state[1]) return;  // complete at an earlier step
    {
        Cand best{-1.0, n};
        for (int q = threadIdx.x; q < ncta; q += blockDim.x)
            if (better(cin[q], best)) best = cin[q];
        sc[threadIdx.x] = best;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w && better(sc[threadIdx.x + w], sc[threadIdx.x])) sc[threadIdx.x] = sc[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) piv = sc[0];
        __syncthreads();
    }
    const Cand p = piv;
    if (!(p.v > tau) || p.i >= n) {  // nothing left above the threshold (NaN included): rank k
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            state[0] = k;
            state[1] = 1;
        }
        return;
    }
    const double sp = sqrt(p.v), inv = 1.0 / sp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* Lp = L + (size_t)p.i * ldl;
    Cand best{-1.0, n};
    for (int64_t i = (int64_t)blockIdx.x * 8 + warp; i < n; i += (int64_t)gridDim.x * 8) {
        const double di = d[i];
        double lik = 0.0;
        if (i == p.i) {
            lik = sp;
        } else if (di >= 0.0) {  // not pivoted
            double dot = 0.0;
            const double* Li = L + (size_t)i * ldl;
            for (int64_t q = lane; q < k; q += 32) dot = fma(Li[q], Lp[q], dot);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
            lik = (v[p.i * n + i] - dot) * inv;
        }
        if (lane == 0) {
            L[(size_t)i * ldl + k] = lik;
            double nd = -1.0;  // pivoted rows (earlier ones and p) leave the candidate set
            if (i != p.i && di >= 0.0) nd = fmax(di - lik * lik, 0.0);
            d[i] = nd;
            const Cand c{nd, i};
            if (better(c, best)) best = c;
        }
    }
    if (lane == 0) sc[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        Cand b = sc[0];
        for (int w = 1; w < 8; ++w)
            if (better(sc[w], b)) b = sc[w];
        cout[blockIdx.x] = b;
    }
}

// C^T (r_pad x n_pad, zero padded) from L (n x ldl, first r columns).
__global__ void k_pchol_transpose(const double* __restrict__ L, int64_t n, int64_t ldl, int64_t r, int64_t n_pad,
                                  int64_t r_pad, double* __restrict__ ct) {
    __shared__ double tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.x * 32, k0 = (int64_t)blockIdx.y * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const int64_t i = i0 + yy, k = k0 + threadIdx.x;
        tile[yy][threadIdx.x] = (i < n && k < r) ? L[(size_t)i * ldl + k] : 0.0;
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const int64_t k = k0 + yy, i = i0 + threadIdx.x;
        if (k < r_pad && i < n_pad) ct[(size_t)k * n_pad + i] = tile[threadIdx.x][yy];
    }
}

constexpr int kPcholCtas = 128;

} // namespace

size_t refine_bytes_per_freq(const TallGeometry& g, int64_t r_pad) {  // either Gram path's workspace
    return std::max(sizeof(double) * ((size_t)g.m_pad * g.n_pad + 2 * (size_t)g.m_pad + (size_t)(r_pad / kT) * g.m_pad),
                    refine_oz_bytes_per_freq(g, r_pad));
}

size_t pchol_bytes(int64_t n) {
    const int64_t n_pad = round_up(n, kT);
    return sizeof(double) * ((size_t)n * n_pad + (size_t)n_pad * n_pad + (size_t)n) + 2 * kPcholCtas * sizeof(Cand) +
           2 * sizeof(long long);
}

int64_t launch_pchol(const double* v, int64_t n, void* work, double** ct_out, cudaStream_t s) {
    const int64_t n_pad = round_up(n, kT);
    double* L = static_cast<double*>(work);
    double* ct = L + (size_t)n * n_pad;
    double* d = ct + (size_t)n_pad * n_pad;
    Cand* cand = reinterpret_cast<Cand*>(d + n);
    long long* state = reinterpret_cast<long long*>(cand + 2 * kPcholCtas);
    k_pchol_init<<<kPcholCtas, 256, 0, s>>>(v, n, d, cand, state);
    GWB_LAUNCH("k_pchol_init");
    // threshold: 1e-13 of the largest diagonal element (read back once)
    double dmax = 0.0;
    {
        Cand host[kPcholCtas];
        GWB_CUDA(cudaMemcpyAsync(host, cand, sizeof(host), cudaMemcpyDeviceToHost, s));
        GWB_CUDA(cudaStreamSynchronize(s));
        for (const Cand& c : host) dmax = std::fmax(dmax, c.v);
    }
    const double tau = 1e-13 * dmax;
    long long st[2] = {0, 0};
    constexpr int64_t kBlockSteps = 64;  // steps between host checks of completion
    for (int64_t k0 = 0; k0 < n && !st[1]; k0 += kBlockSteps) {
        for (int64_t k = k0; k < std::min(n, k0 + kBlockSteps); ++k) {
            k_pchol_step<<<kPcholCtas, 256, 0, s>>>(v, n, L, n_pad, d, cand + (k & 1) * kPcholCtas,
                                                    cand + ((k + 1) & 1) * kPcholCtas, kPcholCtas, k, tau, state);
            GWB_LAUNCH("k_pchol_step");
        }
        GWB_CUDA(cudaMemcpyAsync(st, state, sizeof(st), cudaMemcpyDeviceToHost, s));
        GWB_CUDA(cudaStreamSynchronize(s));
    }
    const int64_t r = st[1] ? (int64_t)st[0] : n;
    const int64_t r_pad = std::max<int64_t>(kT, round_up(r, kT));
    k_pchol_transpose<<<dim3((unsigned)(n_pad / 32), (unsigned)(r_pad / 32)), dim3(32, 8), 0, s>>>(L, n, n_pad, r, n_pad,
                                                                                                  r_pad, ct);
    GWB_LAUNCH("k_pchol_transpose");
    *ct_out = ct;
    return r;
}

int launch_refine_flip(const TallGeometry& ga, int64_t nf, float* a, int64_t n_flip, cudaStream_t s) {
    const int nb = (int)(n_flip / kT);
    k_flip_tiles32<<<dim3((unsigned)nb, (unsigned)nb, (unsigned)nf), 256, 0, s>>>(a, ga.ld, ga.stride, nb);
    GWB_LAUNCH("k_flip_tiles32");
    k_reverse_rows32<<<dim3((unsigned)std::max<int64_t>(1, n_flip / 512), (unsigned)std::min<int64_t>(ga.m_pad, 65535),
                            (unsigned)nf),
                       256, 0, s>>>(a, ga.ld, ga.stride, ga.n_pad, n_flip, ga.m_pad);
    GWB_LAUNCH("k_reverse_rows32");
    return 2;
}

int launch_refine_solve(const TallGeometry& g, int64_t nf, float* a, float* linv, unsigned long long* err_pivot,
                        cudaStream_t s, float* panel, unsigned long long* sched, int max_ctas, bool flip) {
    int launches = flip ? launch_refine_flip(g, nf, a, g.n_pad, s) : 0;
    launches += launch_factor_chunk32(g, nf, a, linv, nullptr, err_pivot, s, nullptr, panel, sched, max_ctas,
                                      /*solve_only=*/true);
    return launches;
}

int launch_refine_terms(const TallGeometry& ga, int64_t nf, const float* a, const TallGeometry& gm, const double* xt,
                        const double* dvec, const RefineFactor& fac, void* work, double* qacc, int64_t ldq,
                        unsigned long long* err, cudaStream_t s) {
    double* t12;
    double* part;
    int64_t nkt;
    int launches;
    if (refine_gram_on_int8(gm.n_pad)) {  // y^T V y from exact int8 products of digit slices (kernels_gram_oz.cu)
        launches = launch_refine_terms_oz(ga, nf, a, gm, xt, dvec, fac.ct_slices, fac.rank, work, err, s, &t12, &part,
                                          &nkt);
    } else {  // on the FP64 tensor pipe (DMMA)
        const int64_t r_pad = fac.r_pad;
        double* y = static_cast<double*>(work);
        t12 = y + (size_t)nf * gm.m_pad * gm.n_pad;
        part = t12 + (size_t)nf * 2 * gm.m_pad;
        // the solve ran on indices reversed within the molecule's own n_pad (launch_refine_flip), in
        // the chunk's matrices (row stride ga.ld, right-hand sides from row ga.n_pad)
        k_refine_prep<<<dim3((unsigned)gm.m_pad, (unsigned)nf), 256, 0, s>>>(a, ga.ld, ga.stride, ga.n_pad, gm.n_pad,
                                                                            gm.n, gm.n_pad, gm.m, gm.m_pad, xt, dvec, y,
                                                                            t12);
        GWB_LAUNCH("k_refine_prep");
        const size_t smem = 4 * kT * kLdk * sizeof(double);
        GWB_CUDA(cudaFuncSetAttribute(k_gram_sq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_gram_sq<<<dim3((unsigned)(gm.m_pad / kT), (unsigned)(r_pad / kT), (unsigned)nf), 256, smem, s>>>(
            fac.ct, y, gm.n_pad, gm.m_pad, r_pad, part);
        GWB_LAUNCH("k_gram_sq");
        nkt = r_pad / kT;
        launches = 2;
    }
    k_refine_finish<<<dim3((unsigned)((gm.m + 255) / 256), (unsigned)nf), 256, 0, s>>>(t12, part, gm.m_pad, nkt, gm.m,
                                                                                      qacc, ldq);
    GWB_LAUNCH("k_refine_finish");
    return launches + 1;
}

int launch_refine_chunk(const TallGeometry& g, int64_t nf, float* a, float* linv, const double* xt,
                        const double* dvec, const RefineFactor& fac, void* work, double* qacc,
                        unsigned long long* err_pivot, cudaStream_t s, float* panel, unsigned long long* sched,
                        int max_ctas) {
    return launch_refine_solve(g, nf, a, linv, err_pivot, s, panel, sched, max_ctas, /*flip=*/true) +
           launch_refine_terms(g, nf, a, g, xt, dvec, fac, work, qacc, g.m_pad, err_pivot, s);
}

bool refine_gram_on_int8(int64_t n_pad) {
    const char* e = std::getenv("GWB200_REFINE_GRAM");
    return !(e && std::strcmp(e, "dmma") == 0) && gram_oz_fits(n_pad);
}

} // namespace gwb200
