// kernels_f32.cu -- the mixed-precision form of the screening (GWB200_MIXED, eta == 0).
//
// Same algorithm as kernels_fp64.cu (tall matrix [eps ; (D^1/2 X)^T], right-looking blocked
// Cholesky, squared row norms), with:
//   * the tall matrices stored in FP32 (eps has eigenvalues >= 1, entries O(1..100)), halving HBM
//     footprint and traffic;
//   * each 64x64 diagonal block factored and inverted in FP64 in shared memory, stored as FP32;
//   * the panel solve and the trailing updates on the tensor cores through mma.sync m16n8k8 TF32
//     with the 3xTF32 split (a = a_hi + a_lo, each a TF32 value; a*b ~ a_hi b_hi + a_hi b_lo +
//     a_lo b_hi, accumulated in FP32), about 21 significant bits per product;
//   * the squared norms, the G0 frequency contraction, Pade and QP in FP64.
// There is no FP64 refinement: the result carries FP32-level error (stated, not hidden, by
// bench.py and the tests).
#include "internal.cuh"

#include <cmath>

namespace gwb200 {
namespace {

constexpr int kLdf = 68;  // padded shared row stride (floats) of a 64-wide FP32 tile
constexpr int kKcf = 32;  // K slice of the pipelined FP32 update
constexpr int kLdkf = kKcf + 4;

__device__ __forceinline__ unsigned to_tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc += sgn * As(64 x KD) * Bs(64 x KD)^T, FP32 tiles in shared memory with row stride LD.
// 8 warps as 4 (rows) x 2 (cols): warp tile 16 x 32 = one m16 tile by four n8 tiles.
// Fragments (PTX ISA, mma.m16n8k8 .tf32): A a0..a3 = (g,t) (g+8,t) (g,t+4) (g+8,t+4);
// B b0,b1 = (k=t, n=g) (k=t+4, n=g); C c0..c3 = (g,2t) (g,2t+1) (g+8,2t) (g+8,2t+1).
template <int LD, int KD>
__device__ __forceinline__ void tile_mma_3xtf32(const float* __restrict__ As, const float* __restrict__ Bs,
                                                float (&acc)[4][4], float sgn) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 16 * (w >> 1), c0 = 32 * (w & 1);
#pragma unroll 2
    for (int kk = 0; kk < KD; kk += 8) {
        unsigned ah[4], al[4];
        split_tf32(sgn * As[(r0 + g) * LD + kk + t], ah[0], al[0]);
        split_tf32(sgn * As[(r0 + g + 8) * LD + kk + t], ah[1], al[1]);
        split_tf32(sgn * As[(r0 + g) * LD + kk + t + 4], ah[2], al[2]);
        split_tf32(sgn * As[(r0 + g + 8) * LD + kk + t + 4], ah[3], al[3]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            unsigned bh0, bl0, bh1, bl1;
            split_tf32(Bs[(c0 + 8 * j + g) * LD + kk + t], bh0, bl0);
            split_tf32(Bs[(c0 + 8 * j + g) * LD + kk + t + 4], bh1, bl1);
            mma_tf32(acc[j], al, bh0, bh1);
            mma_tf32(acc[j], ah, bl0, bl1);
            mma_tf32(acc[j], ah, bh0, bh1);
        }
    }
}

__device__ __forceinline__ void cp_async_16f(float* smem_dst, const float* gsrc) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gsrc));
}

// 64 x W floats of global (row stride ld) into shared memory (row stride LD), 16-byte pieces.
template <int W, int LD>
__device__ __forceinline__ void load_f32_async(float* __restrict__ s, const float* __restrict__ gsrc, int64_t ld) {
    for (int idx = threadIdx.x; idx < 64 * (W / 4); idx += blockDim.x) {
        const int r = idx / (W / 4), c4 = idx % (W / 4);
        cp_async_16f(s + r * LD + 4 * c4, gsrc + (size_t)r * ld + 4 * c4);
    }
}

// Tall FP32 matrices: eps lower triangle (computed in FP64, rounded) and (D^1/2 X)^T rows.
__global__ void k_build_tall32(int64_t n, int64_t m, int64_t n_pad, int64_t ld, int64_t stride, int64_t rows,
                               const double* __restrict__ v, const double* __restrict__ xt,
                               const double* __restrict__ dvec, int nf, float* __restrict__ a) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_pad) return;
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
        if (r < n_pad) {
            if (c > r) continue;
            const double vrc = (r < n && c < n) ? v[r * n + c] : 0.0;
            const double diag = (r == c) ? 1.0 : 0.0;
            for (int f = 0; f < nf; ++f) {
                const double* d = dvec + (size_t)f * n_pad;
                a[(size_t)f * stride + r * ld + c] = (float)fma(d[r] * vrc, d[c], diag);
            }
        } else {
            const int64_t j = r - n_pad;
            const double x = (j < m && c < n) ? xt[j * n + c] : 0.0;
            for (int f = 0; f < nf; ++f) a[(size_t)f * stride + r * ld + c] = (float)(dvec[(size_t)f * n_pad + c] * x);
        }
    }
}

// Diagonal block in FP64 (from the FP32 tall matrix), written back as FP32 L and FP32 L^{-1}.
// One 64 x 65 FP64 tile: L in the lower triangle, Y = L^{-1} (lower too) transposed into the
// upper triangle (Y[l][c] at T[c][l], l > c) with its diagonal in Yd, so 6 CTAs fit an SM.
// invert_only: the block already holds a Cholesky factor (the solve-only pass of the mixed form's
// refinement); only its inverse is formed and the block is left as it is.
__global__ void __launch_bounds__(256) k_potrf_diag32(float* __restrict__ a, int64_t ld, int64_t stride, int64_t k,
                                                      float* __restrict__ linv, unsigned long long* err_pivot,
                                                      int invert_only) {
    extern __shared__ double smem[];
    constexpr int L = kNb + 1;
    double* T = smem;
    double* Yd = smem + kNb * L;
    float* A = a + (size_t)blockIdx.x * stride + k * ld + k;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int i = idx / kNb, j = idx % kNb;
        T[i * L + j] = (j <= i) ? (double)A[(size_t)i * ld + j] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kNb && !invert_only; ++j) {
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
    if (!invert_only)
        for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
            const int i = idx / kNb, j = idx % kNb;
            if (j <= i) A[(size_t)i * ld + j] = (float)T[i * L + j];
        }
    {
        const int col = tid >> 2, part = tid & 3;
        for (int i = 0; i < kNb; ++i) {
            double sum = 0.0;
            if (i > col)
                for (int l = col + part; l < i; l += 4) sum = fma(T[i * L + l], l == col ? Yd[col] : T[col * L + l], sum);
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 2);
            if (part == 0) {
                if (i == col) Yd[col] = 1.0 / T[i * L + i];
                else if (i > col) T[col * L + i] = -sum / T[i * L + i];
            }
            __syncwarp();
        }
    }
    __syncthreads();
    float* out = linv + (size_t)blockIdx.x * kNb * kNb;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int r = idx / kNb, c = idx % kNb;
        out[idx] = r > c ? (float)T[c * L + r] : (r == c ? (float)Yd[r] : 0.0f);
    }
}

// Panel solve P <- P Linv^T on the tensor cores (3xTF32) for the 64-row blocks from row0 on; RHS
// rows add their squared norms (FP64) to qacc unless it is null.
__global__ void __launch_bounds__(256) k_trsm_panel32(float* __restrict__ a, int64_t ld, int64_t stride, int64_t k,
                                                      int64_t row0, int64_t n_pad, const float* __restrict__ linv,
                                                      double* __restrict__ qacc, int64_t ldq) {
    extern __shared__ float fsm[];
    float* Ps = fsm;
    float* Ls = fsm + 64 * kLdf;
    const int f = blockIdx.y;
    const int64_t r0 = row0 + (int64_t)blockIdx.x * kNb;
    float* A = a + (size_t)f * stride;
    load_f32_async<64, kLdf>(Ps, A + r0 * ld + k, ld);
    load_f32_async<64, kLdf>(Ls, linv + (size_t)f * kNb * kNb, kNb);
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    float acc[4][4] = {};
    tile_mma_3xtf32<kLdf, 64>(Ps, Ls, acc, 1.0f);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rr = 16 * (w >> 1), cc = 32 * (w & 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        Ps[(rr + g) * kLdf + cc + 8 * j + 2 * t] = acc[j][0];
        Ps[(rr + g) * kLdf + cc + 8 * j + 2 * t + 1] = acc[j][1];
        Ps[(rr + g + 8) * kLdf + cc + 8 * j + 2 * t] = acc[j][2];
        Ps[(rr + g + 8) * kLdf + cc + 8 * j + 2 * t + 1] = acc[j][3];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 64 * 16; idx += blockDim.x) {
        const int r = idx >> 4, c4 = idx & 15;
        *reinterpret_cast<float4*>(A + (size_t)(r0 + r) * ld + k + 4 * c4) =
            *reinterpret_cast<const float4*>(Ps + r * kLdf + 4 * c4);
    }
    if (qacc && r0 >= n_pad && threadIdx.x < kNb) {
        const int r = threadIdx.x;
        double s = 0.0;
        for (int j = 0; j < kNb; ++j) {
            const double y = (double)Ps[r * kLdf + j];
            s = fma(y, y, s);
        }
        qacc[(size_t)f * ldq + (r0 - n_pad + r)] += s;
    }
}

// Trailing / look-left update on FP32 tiles (3xTF32), same tile enumeration and K chunking as the
// FP64 k_update: output column tiles [tc0, tc0+T), lower square tiles then all RHS tiles
// (rhs_only: the RHS tiles alone, for the solve-only pass against a finished factor).
__global__ void __launch_bounds__(256, 3) k_update32(float* __restrict__ a, int64_t ld, int64_t stride, int64_t kb0,
                                                     int nk, int64_t tc0, int64_t T, int64_t nsq, int rhs_only) {
    extern __shared__ float fsm[];
    auto stage = [&](int st, int which) { return fsm + (2 * st + which) * 64 * kLdkf; };
    const int f = blockIdx.y;
    const int64_t Lr = nsq - tc0;
    const int64_t n_square = rhs_only ? 0 : T * Lr - T * (T - 1) / 2;
    const int64_t x = blockIdx.x;
    int64_t c, tr;
    if (x < n_square) {
        const double b = 2.0 * (double)Lr + 1.0;
        c = (int64_t)((b - sqrt(fmax(b * b - 8.0 * (double)x, 0.0))) * 0.5);
        auto cum = [Lr](int64_t cc) { return cc * Lr - cc * (cc - 1) / 2; };
        while (c > 0 && cum(c) > x) --c;
        while (c + 1 < T && cum(c + 1) <= x) ++c;
        tr = tc0 + c + (x - cum(c));
    } else {
        const int64_t y = x - n_square;
        c = y % T;
        tr = nsq + y / T;
    }
    const int64_t ri = tr * kNb, cj = (tc0 + c) * kNb;
    float* A = a + (size_t)f * stride;
    const int nsub = nk * (kNb / kKcf);
    load_f32_async<kKcf, kLdkf>(stage(0, 0), A + ri * ld + kb0, ld);
    load_f32_async<kKcf, kLdkf>(stage(0, 1), A + cj * ld + kb0, ld);
    asm volatile("cp.async.commit_group;\n" ::);
    float acc[4][4] = {};
    for (int sc = 0; sc < nsub; ++sc) {
        if (sc + 1 < nsub) {
            const int64_t kc = kb0 + (int64_t)(sc + 1) * kKcf;
            load_f32_async<kKcf, kLdkf>(stage((sc + 1) & 1, 0), A + ri * ld + kc, ld);
            load_f32_async<kKcf, kLdkf>(stage((sc + 1) & 1, 1), A + cj * ld + kc, ld);
            asm volatile("cp.async.commit_group;\n" ::);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        tile_mma_3xtf32<kLdkf, kKcf>(stage(sc & 1, 0), stage(sc & 1, 1), acc, -1.0f);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rr = 16 * (w >> 1), cc = 32 * (w & 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float2* pc = reinterpret_cast<float2*>(A + (size_t)(ri + rr + g + 8 * h) * ld + cj + cc + 8 * j + 2 * t);
            float2 v = *pc;
            v.x += acc[j][2 * h];
            v.y += acc[j][2 * h + 1];
            *pc = v;
        }
    }
}

double update_flops32(const TallGeometry& g, int64_t kb0, int nk, int64_t c0, int64_t c1) {
    const int64_t kt = std::max<int64_t>(0, std::min<int64_t>(kb0 + (int64_t)nk * kNb, g.n) - kb0);
    const int64_t a0 = std::min(c0, g.n), a1 = std::min(c1, g.n);
    const double cols = (double)(a1 - a0);
    const double lower = cols * (double)g.n - 0.5 * (double)(a0 + a1 - 1) * cols;
    return 2.0 * (double)kt * (lower + (double)g.m * cols);
}

} // namespace

int launch_build_tall32(const TallGeometry& g, const double* v, const double* xt, const double* dvec, int64_t nf,
                        float* a, cudaStream_t s) {
    dim3 grid((unsigned)((g.n_pad + 255) / 256), (unsigned)std::min<int64_t>(g.rows, 65535));
    k_build_tall32<<<grid, 256, 0, s>>>(g.n, g.m, g.n_pad, g.ld, g.stride, g.rows, v, xt, dvec, (int)nf, a);
    GWB_LAUNCH("k_build_tall32");
    return 1;
}

int launch_factor_chunk32(const TallGeometry& g, int64_t nf, float* a, float* linv, double* qacc,
                          unsigned long long* err_pivot, cudaStream_t s, UpdateProfiler* prof, float* panel,
                          unsigned long long* sched, int max_ctas, bool solve_only) {
    const size_t smem_tile = 2 * 64 * kLdf * sizeof(float);
    const size_t smem_update = 4 * 64 * kLdkf * sizeof(float);
    const size_t smem_potrf = (kNb * (kNb + 1) + kNb) * sizeof(double);
    GWB_CUDA(cudaFuncSetAttribute(k_trsm_panel32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tile));
    GWB_CUDA(cudaFuncSetAttribute(k_update32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_update));
    GWB_CUDA(cudaFuncSetAttribute(k_potrf_diag32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
    const int64_t nsq = g.n_pad / kNb, nrt = g.rows / kNb;
    constexpr int64_t kInner = 2;
    int launches = 0;
    // with the tcgen05 outer updates, the profiler times those alone (the look-left updates that
    // stay on mma.sync are a few percent of the flops)
    UpdateProfiler* lprof = panel ? nullptr : prof;
    auto update = [&](int64_t kb0, int nk, int64_t tc0, int64_t T) {
        const int64_t L = nsq - tc0;
        const int64_t tiles = (solve_only ? 0 : T * L - T * (T - 1) / 2) + T * (nrt - nsq);
        if (tiles <= 0) return;
        if (lprof) lprof->begin();
        k_update32<<<dim3((unsigned)tiles, (unsigned)nf), 256, smem_update, s>>>(a, g.ld, g.stride, kb0, nk, tc0, T, nsq,
                                                                                  solve_only ? 1 : 0);
        GWB_LAUNCH("k_update32");
        if (lprof) lprof->end((double)nf * update_flops32(g, kb0, nk, tc0 * kNb, (tc0 + T) * kNb));
        ++launches;
    };
    for (int64_t ob = 0; ob < nsq; ob += kInner) {
        const int64_t q = std::min(kInner, nsq - ob);
        for (int64_t j = 0; j < q; ++j) {
            const int64_t kt = ob + j, k = kt * kNb;
            if (j > 0) update(ob * kNb, (int)j, kt, 1);
            k_potrf_diag32<<<(unsigned)nf, 256, smem_potrf, s>>>(a, g.ld, g.stride, k, linv, err_pivot,
                                                                 solve_only ? 1 : 0);
            GWB_LAUNCH("k_potrf_diag32");
            ++launches;
            // the panel rows below the block: all of them while factoring, the RHS rows alone when
            // solving against a finished factor
            const int64_t row0 = solve_only ? g.n_pad : k + kNb;
            const int64_t below = g.rows - row0;
            if (below > 0) {
                k_trsm_panel32<<<dim3((unsigned)(below / kNb), (unsigned)nf), 256, smem_tile, s>>>(
                    a, g.ld, g.stride, k, row0, g.n_pad, linv, solve_only ? nullptr : qacc, g.m_pad);
                GWB_LAUNCH("k_trsm_panel32");
                ++launches;
            }
        }
        const int64_t tc0 = ob + q;
        if (tc0 < nsq) {
            if (panel) {  // outer trailing update on tcgen05
                if (prof) prof->begin();
                launches += launch_update32_tc(g, nf, a, ob * kNb, (int)(q * kNb), tc0 * kNb, panel, sched, err_pivot, s,
                                                max_ctas, solve_only ? g.n_pad : 0);
                if (prof) prof->end((double)nf * update_flops32(g, ob * kNb, (int)q, tc0 * kNb, nsq * kNb));
            } else {
                update(ob * kNb, (int)q, tc0, nsq - tc0);
            }
        }
    }
    return launches;
}

} // namespace gwb200
