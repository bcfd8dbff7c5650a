// kernels_c64.cu -- screening for eta != 0 (complex FP64).
//
// With broadening eta the reference's Pi0 = 2[1/(w - d + i eta) - 1/(w + d - i eta)]
// (src/gw/sigma.cpp:41-54, w = i omega) is complex and eps_left = I - diag(Pi0) V is no longer
// SPD.  With S = diag(Pi0)^1/2 (any branch: only S*S = diag(Pi0) matters)
//     W_c = (I - diag(Pi0) V)^{-1} diag(Pi0) = S M^{-1} S,   M = I - S V S  (complex symmetric)
//     x^T W_c x = (S x)^T M^{-1} (S x) = sum_j (L^{-1} S x)_j^2,   M = L L^T  (no conjugation)
// so the same tall-matrix right-looking Cholesky runs in complex arithmetic without pivoting
// (M is a small perturbation of the SPD eta = 0 matrix).  A pivot of modulus < 1e-300 or a
// non-finite one is reported like the real path's non-positive pivot.  Every complex tile product
// is four FP64 DMMA tile products on separate real and imaginary planes.  At eta = 0 this path
// gives the real path's numbers (S = i D^1/2); the real path is used there.
#include "internal.cuh"

#include <cmath>

namespace gwb200 {
namespace {

__device__ __forceinline__ void dmma_8x8x4c(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// acc += sgn * As(64x64) * Bs(64x64)^T from shared memory (stride kLds); same warp layout as the
// real path: warp w owns rows 16*(w/2)..+15, cols 32*(w%2)..+31.
__device__ __forceinline__ void tile_mma_c(const double* __restrict__ As, const double* __restrict__ Bs,
                                           double (&acc)[2][4][2], double sgn) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 16 * (w >> 1), c0 = 32 * (w & 1);
#pragma unroll 4
    for (int kk = 0; kk < kNb; kk += 4) {
        double af[2], bf[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) af[i] = sgn * As[(r0 + 8 * i + g) * kLds + kk + t];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = Bs[(c0 + 8 * j + g) * kLds + kk + t];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma_8x8x4c(acc[i][j], af[i], bf[j]);
    }
}

__device__ __forceinline__ void load_tile_c(double* __restrict__ s, const double* __restrict__ gsrc, int64_t ld) {
    for (int idx = threadIdx.x; idx < 64 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c2 = idx & 31;
        *reinterpret_cast<double2*>(s + r * kLds + 2 * c2) = *reinterpret_cast<const double2*>(gsrc + (size_t)r * ld + 2 * c2);
    }
}

// principal square root of x + i y
__device__ __forceinline__ void csqrt_dev(double x, double y, double& sr, double& si) {
    const double r = hypot(x, y);
    if (r == 0.0) {
        sr = si = 0.0;
        return;
    }
    const double t = sqrt(0.5 * (fabs(x) + r));
    if (x >= 0.0) {
        sr = t;
        si = y / (2.0 * t);
    } else {
        sr = fabs(y) / (2.0 * t);
        si = copysign(t, y);
    }
}

// S_f[c] = sqrt(Pi0(i w_f)[c]) for eta != 0, as two planes (re, im) of n_pad each; zero padding.
__global__ void k_scale_vectors_c(const double* __restrict__ delta, int n, int n_pad, const double* __restrict__ omega,
                                  double eta, double* __restrict__ svec) {
    const int f = blockIdx.y;
    const double w = omega[f];
    double* sr_out = svec + (size_t)f * 2 * n_pad;
    double* si_out = sr_out + n_pad;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_pad; c += gridDim.x * blockDim.x) {
        double sr = 0.0, si = 0.0;
        if (c < n) {
            const double d = delta[c];
            // 1/(i w - d + i eta) = 1/(-d + i(w + eta)); 1/(i w + d - i eta) = 1/(d + i(w - eta))
            const double a1r = -d, a1i = w + eta, n1 = a1r * a1r + a1i * a1i;
            const double a2r = d, a2i = w - eta, n2 = a2r * a2r + a2i * a2i;
            const double pr = 2.0 * (a1r / n1 - a2r / n2);
            const double pi = 2.0 * (-a1i / n1 + a2i / n2);
            csqrt_dev(pr, pi, sr, si);
        }
        sr_out[c] = sr;
        si_out[c] = si;
    }
}

// Tall complex matrices: rows r < n_pad hold the lower triangle of M = I - S V S, rows >= n_pad
// hold (S x_j)^T.  Planes: a_re, a_im with the real geometry g.
__global__ void k_build_tall_c(int64_t n, int64_t m, int64_t n_pad, int64_t ld, int64_t stride, int64_t rows,
                               const double* __restrict__ v, const double* __restrict__ xt,
                               const double* __restrict__ svec, int nf, double* __restrict__ a_re,
                               double* __restrict__ a_im) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_pad) return;
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
        if (r < n_pad) {
            if (c > r) continue;
            const double vrc = (r < n && c < n) ? v[r * n + c] : 0.0;
            const double diag = (r == c) ? 1.0 : 0.0;
            for (int f = 0; f < nf; ++f) {
                const double* sr = svec + (size_t)f * 2 * n_pad;
                const double* si = sr + n_pad;
                // s_r * s_c
                const double pr = sr[r] * sr[c] - si[r] * si[c], pi = sr[r] * si[c] + si[r] * sr[c];
                a_re[(size_t)f * stride + r * ld + c] = diag - pr * vrc;
                a_im[(size_t)f * stride + r * ld + c] = -pi * vrc;
            }
        } else {
            const int64_t j = r - n_pad;
            const double x = (j < m && c < n) ? xt[j * n + c] : 0.0;
            for (int f = 0; f < nf; ++f) {
                const double* sr = svec + (size_t)f * 2 * n_pad;
                a_re[(size_t)f * stride + r * ld + c] = sr[c] * x;
                a_im[(size_t)f * stride + r * ld + c] = sr[n_pad + c] * x;
            }
        }
    }
}

// Complex 64x64 diagonal block: L L^T (no conjugation) in shared memory, then L^{-1}.
__global__ void __launch_bounds__(256) k_potrf_diag_c(double* __restrict__ a_re, double* __restrict__ a_im, int64_t ld,
                                                      int64_t stride, int64_t k, double* __restrict__ linv,
                                                      unsigned long long* err_pivot) {
    extern __shared__ double smem[];
    constexpr int L = kNb + 1;
    double* Tr = smem;
    double* Ti = Tr + kNb * L;
    double* Yr = Ti + kNb * L;
    double* Yi = Yr + kNb * L;
    double* Ar = a_re + (size_t)blockIdx.x * stride + k * ld + k;
    double* Ai = a_im + (size_t)blockIdx.x * stride + k * ld + k;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int i = idx / kNb, j = idx % kNb;
        Tr[i * L + j] = (j <= i) ? Ar[(size_t)i * ld + j] : 0.0;
        Ti[i * L + j] = (j <= i) ? Ai[(size_t)i * ld + j] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kNb; ++j) {
        if (tid == 0) {
            double xr = Tr[j * L + j], xi = Ti[j * L + j];
            const double mod = hypot(xr, xi);
            if (!(mod > 1e-300) || !isfinite(mod)) {
                atomicMin(err_pivot, (unsigned long long)(k + j + 1));
                xr = 1.0;
                xi = 0.0;
            }
            double sr, si;
            csqrt_dev(xr, xi, sr, si);
            Tr[j * L + j] = sr;
            Ti[j * L + j] = si;
        }
        __syncthreads();
        const double dr = Tr[j * L + j], di = Ti[j * L + j];
        const double dn = dr * dr + di * di;
        for (int i = j + 1 + tid; i < kNb; i += blockDim.x) {  // a_ij / d
            const double xr = Tr[i * L + j], xi = Ti[i * L + j];
            Tr[i * L + j] = (xr * dr + xi * di) / dn;
            Ti[i * L + j] = (xi * dr - xr * di) / dn;
        }
        __syncthreads();
        const int rem = kNb - 1 - j;
        for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
            const int i = j + 1 + idx / rem, l = j + 1 + idx % rem;
            if (l <= i) {
                const double ar = Tr[i * L + j], ai = Ti[i * L + j], br = Tr[l * L + j], bi = Ti[l * L + j];
                Tr[i * L + l] -= ar * br - ai * bi;
                Ti[i * L + l] -= ar * bi + ai * br;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        const int i = idx / kNb, j = idx % kNb;
        if (j <= i) {
            Ar[(size_t)i * ld + j] = Tr[i * L + j];
            Ai[(size_t)i * ld + j] = Ti[i * L + j];
        }
    }
    if (tid < kNb) {  // forward substitution, one column of L^{-1} per thread
        const int col = tid;
        for (int i = 0; i < kNb; ++i) {
            double yr, yi;
            if (i < col) {
                yr = yi = 0.0;
            } else {
                double sr = (i == col) ? 1.0 : 0.0, si = 0.0;
                for (int l = col; l < i; ++l) {
                    sr -= Tr[i * L + l] * Yr[l * L + col] - Ti[i * L + l] * Yi[l * L + col];
                    si -= Tr[i * L + l] * Yi[l * L + col] + Ti[i * L + l] * Yr[l * L + col];
                }
                const double dr = Tr[i * L + i], di = Ti[i * L + i], dn = dr * dr + di * di;
                yr = (sr * dr + si * di) / dn;
                yi = (si * dr - sr * di) / dn;
            }
            Yr[i * L + col] = yr;
            Yi[i * L + col] = yi;
        }
    }
    __syncthreads();
    double* out = linv + (size_t)blockIdx.x * 2 * kNb * kNb;
    for (int idx = tid; idx < kNb * kNb; idx += blockDim.x) {
        out[idx] = Yr[(idx / kNb) * L + idx % kNb];
        out[kNb * kNb + idx] = Yi[(idx / kNb) * L + idx % kNb];
    }
}

// Panel solve: P <- P * Linv^T (complex) for rows below the block; RHS rows add sum_j y_j^2 to q.
__global__ void __launch_bounds__(256) k_trsm_panel_c(double* __restrict__ a_re, double* __restrict__ a_im, int64_t ld,
                                                      int64_t stride, int64_t k, int64_t n_pad,
                                                      const double* __restrict__ linv, double* __restrict__ qacc,
                                                      int64_t ldq) {
    extern __shared__ double smem[];
    double* Pr = smem;
    double* Pi = Pr + 64 * kLds;
    double* Lr = Pi + 64 * kLds;
    double* Li = Lr + 64 * kLds;
    const int f = blockIdx.y;
    const int64_t r0 = k + kNb + (int64_t)blockIdx.x * kNb;
    double* Ar = a_re + (size_t)f * stride;
    double* Ai = a_im + (size_t)f * stride;
    load_tile_c(Pr, Ar + r0 * ld + k, ld);
    load_tile_c(Pi, Ai + r0 * ld + k, ld);
    const double* lv = linv + (size_t)f * 2 * kNb * kNb;
    load_tile_c(Lr, lv, kNb);
    load_tile_c(Li, lv + kNb * kNb, kNb);
    __syncthreads();
    double accr[2][4][2] = {}, acci[2][4][2] = {};
    tile_mma_c(Pr, Lr, accr, 1.0);
    tile_mma_c(Pi, Li, accr, -1.0);
    tile_mma_c(Pr, Li, acci, 1.0);
    tile_mma_c(Pi, Lr, acci, 1.0);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rr = 16 * (w >> 1), cc = 32 * (w & 1);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                Pr[(rr + 8 * i + g) * kLds + cc + 8 * j + 2 * t + e] = accr[i][j][e];
                Pi[(rr + 8 * i + g) * kLds + cc + 8 * j + 2 * t + e] = acci[i][j][e];
            }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 64 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c2 = idx & 31;
        *reinterpret_cast<double2*>(Ar + (size_t)(r0 + r) * ld + k + 2 * c2) =
            *reinterpret_cast<const double2*>(Pr + r * kLds + 2 * c2);
        *reinterpret_cast<double2*>(Ai + (size_t)(r0 + r) * ld + k + 2 * c2) =
            *reinterpret_cast<const double2*>(Pi + r * kLds + 2 * c2);
    }
    if (r0 >= n_pad && threadIdx.x < kNb) {
        const int r = threadIdx.x;
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < kNb; ++j) {
            const double yr = Pr[r * kLds + j], yi = Pi[r * kLds + j];
            sr += yr * yr - yi * yi;
            si += 2.0 * yr * yi;
        }
        qacc[(size_t)f * 2 * ldq + (r0 - n_pad + r)] += sr;
        qacc[(size_t)f * 2 * ldq + ldq + (r0 - n_pad + r)] += si;
    }
}

// Trailing update C -= P_i P_j^T (complex, K = 64) over lower square tiles and all RHS tiles.
__global__ void __launch_bounds__(256) k_update_c(double* __restrict__ a_re, double* __restrict__ a_im, int64_t ld,
                                                  int64_t stride, int64_t k, int64_t t_sq, int64_t t_rhs) {
    extern __shared__ double smem[];
    double* Pir = smem;
    double* Pii = Pir + 64 * kLds;
    double* Pjr = Pii + 64 * kLds;
    double* Pji = Pjr + 64 * kLds;
    const int f = blockIdx.y;
    const int64_t x = blockIdx.x;
    const int64_t n_sq = t_sq * (t_sq + 1) / 2;
    int64_t ti, tj;
    if (x < n_sq) {
        ti = (int64_t)((sqrt(8.0 * (double)x + 1.0) - 1.0) * 0.5);
        while (ti * (ti + 1) / 2 > x) --ti;
        while ((ti + 1) * (ti + 2) / 2 <= x) ++ti;
        tj = x - ti * (ti + 1) / 2;
    } else {
        const int64_t y = x - n_sq;
        ti = t_sq + y / t_sq;
        tj = y % t_sq;
        if (ti >= t_sq + t_rhs) return;
    }
    const int64_t base = k + kNb;
    const int64_t ri = base + ti * kNb, cj = base + tj * kNb;
    double* Ar = a_re + (size_t)f * stride;
    double* Ai = a_im + (size_t)f * stride;
    load_tile_c(Pir, Ar + ri * ld + k, ld);
    load_tile_c(Pii, Ai + ri * ld + k, ld);
    load_tile_c(Pjr, Ar + cj * ld + k, ld);
    load_tile_c(Pji, Ai + cj * ld + k, ld);
    __syncthreads();
    double accr[2][4][2] = {}, acci[2][4][2] = {};
    tile_mma_c(Pir, Pjr, accr, -1.0);
    tile_mma_c(Pii, Pji, accr, 1.0);
    tile_mma_c(Pir, Pji, acci, -1.0);
    tile_mma_c(Pii, Pjr, acci, -1.0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int rr = 16 * (w >> 1), cc = 32 * (w & 1);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const size_t off = (size_t)(ri + rr + 8 * i + g) * ld + cj + cc + 8 * j + 2 * t;
            double2 vr = *reinterpret_cast<double2*>(Ar + off), vi = *reinterpret_cast<double2*>(Ai + off);
            vr.x += accr[i][j][0];
            vr.y += accr[i][j][1];
            vi.x += acci[i][j][0];
            vi.y += acci[i][j][1];
            *reinterpret_cast<double2*>(Ar + off) = vr;
            *reinterpret_cast<double2*>(Ai + off) = vi;
        }
}

// q_out[f] (complex, interleaved) = qacc (planes re, im).
__global__ void k_forms_out_c(const double* __restrict__ qacc, int m, int64_t ldq, double* __restrict__ q,
                              int64_t ldq_out) {
    const int f = blockIdx.y;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        q[(size_t)f * 2 * ldq_out + 2 * j] = qacc[(size_t)f * 2 * ldq + j];
        q[(size_t)f * 2 * ldq_out + 2 * j + 1] = qacc[(size_t)f * 2 * ldq + ldq + j];
    }
}

// Sigma contraction with complex forms (interleaved [f][2*ldq]):
// Sigma_c(p_s, i w_n) = -(1/pi) sum_{f', k} w_{f'} g(k, n, f') q[f', s, k].
__global__ void __launch_bounds__(256) k_sigma_contract_c(const double* __restrict__ qall, int nf_int, int nmo,
                                                          int64_t ldq, const int64_t* __restrict__ states,
                                                          const double* __restrict__ mo, double fermi,
                                                          const double* __restrict__ omega_int,
                                                          const double* __restrict__ weight_int,
                                                          const double* __restrict__ omega_out, int nf_out,
                                                          double* __restrict__ sigma) {
    const int fn = blockIdx.x, s = blockIdx.y;
    const double wn = omega_out[fn];
    double sr = 0.0, si = 0.0;
    const int total = nf_int * nmo;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int fp = idx / nmo, k = idx % nmo;
        const size_t qi = (size_t)fp * 2 * ldq + 2 * ((size_t)s * nmo + k);
        const double qr = qall[qi], qim = qall[qi + 1];
        const double ar = fermi - mo[k], ai = wn;
        const double wp = omega_int[fp];
        const double dr = ar * ar - ai * ai + wp * wp, di = 2.0 * ar * ai;
        const double inv = 1.0 / (dr * dr + di * di);
        const double gr = (ar * dr + ai * di) * inv, gi = (ai * dr - ar * di) * inv;
        const double wgt = -weight_int[fp];
        sr += wgt * (gr * qr - gi * qim);
        si += wgt * (gr * qim + gi * qr);
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = sr;
    red[1][threadIdx.x] = si;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            red[0][threadIdx.x] += red[0][threadIdx.x + off];
            red[1][threadIdx.x] += red[1][threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const size_t p = (size_t)states[s];
        const double inv_pi = 1.0 / 3.141592653589793238462643383279502884;
        sigma[2 * (p * nf_out + fn)] = red[0][0] * inv_pi;
        sigma[2 * (p * nf_out + fn) + 1] = red[1][0] * inv_pi;
    }
}

} // namespace

int launch_factor_chunk_c(const TallGeometry& g, int64_t nf, const double* delta, const double* omega, double eta,
                          const double* v, const double* xt, double* a_re, double* a_im, double* svec, double* linv,
                          double* qacc, unsigned long long* err_pivot, cudaStream_t s) {
    const size_t smem4 = 4 * 64 * kLds * sizeof(double);
    const size_t smem_potrf = 4 * kNb * (kNb + 1) * sizeof(double);
    GWB_CUDA(cudaFuncSetAttribute(k_potrf_diag_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
    GWB_CUDA(cudaFuncSetAttribute(k_trsm_panel_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem4));
    GWB_CUDA(cudaFuncSetAttribute(k_update_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem4));
    int launches = 0;
    k_scale_vectors_c<<<dim3((unsigned)((g.n_pad + 255) / 256), (unsigned)nf), 256, 0, s>>>(delta, (int)g.n, (int)g.n_pad,
                                                                                          omega, eta, svec);
    GWB_LAUNCH("k_scale_vectors_c");
    k_build_tall_c<<<dim3((unsigned)((g.n_pad + 255) / 256), (unsigned)std::min<int64_t>(g.rows, 65535)), 256, 0, s>>>(
        g.n, g.m, g.n_pad, g.ld, g.stride, g.rows, v, xt, svec, (int)nf, a_re, a_im);
    GWB_LAUNCH("k_build_tall_c");
    GWB_CUDA(cudaMemsetAsync(qacc, 0, sizeof(double) * 2 * (size_t)nf * g.m_pad, s));
    launches += 2;
    for (int64_t k = 0; k < g.n_pad; k += kNb) {
        k_potrf_diag_c<<<(unsigned)nf, 256, smem_potrf, s>>>(a_re, a_im, g.ld, g.stride, k, linv, err_pivot);
        GWB_LAUNCH("k_potrf_diag_c");
        ++launches;
        const int64_t below = g.rows - (k + kNb);
        if (below > 0) {
            k_trsm_panel_c<<<dim3((unsigned)(below / kNb), (unsigned)nf), 256, smem4, s>>>(a_re, a_im, g.ld, g.stride, k,
                                                                                      g.n_pad, linv, qacc, g.m_pad);
            GWB_LAUNCH("k_trsm_panel_c");
            ++launches;
        }
        const int64_t t_sq = (g.n_pad - (k + kNb)) / kNb;
        if (t_sq > 0) {
            const int64_t t_rhs = g.m_pad / kNb;
            const int64_t tiles = t_sq * (t_sq + 1) / 2 + t_rhs * t_sq;
            k_update_c<<<dim3((unsigned)tiles, (unsigned)nf), 256, smem4, s>>>(a_re, a_im, g.ld, g.stride, k, t_sq, t_rhs);
            GWB_LAUNCH("k_update_c");
            ++launches;
        }
    }
    return launches;
}

int launch_forms_out_c(const double* qacc, int64_t nf, int64_t m, int64_t ldq, double* q_out, int64_t ldq_out,
                       cudaStream_t s) {
    k_forms_out_c<<<dim3((unsigned)std::min<int64_t>((m + 255) / 256, 64), (unsigned)nf), 256, 0, s>>>(
        qacc, (int)m, ldq, q_out, ldq_out);
    GWB_LAUNCH("k_forms_out_c");
    return 1;
}

int launch_sigma_contract_c(const double* qall, int64_t nf_int, int64_t nstates, int64_t nmo, int64_t ldq,
                            const int64_t* states, const double* mo, double fermi, const double* omega_int,
                            const double* weight_int, const double* omega_out, int64_t nf_out, double* sigma,
                            cudaStream_t s) {
    k_sigma_contract_c<<<dim3((unsigned)nf_out, (unsigned)nstates), 256, 0, s>>>(
        qall, (int)nf_int, (int)nmo, ldq, states, mo, fermi, omega_int, weight_int, omega_out, (int)nf_out, sigma);
    GWB_LAUNCH("k_sigma_contract_c");
    return 1;
}

} // namespace gwb200
