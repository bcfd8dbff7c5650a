// kernels_small.cu -- FP64 device kernels after the screening: the G0-weighted frequency
// contraction into Sigma_c(iw), the Pade continued fraction, the quasiparticle fixed point
// and the E_c.out sweep, plus the FP64 DMMA peak probe.
//
// The Pade / QP kernels reproduce the reference's std::complex<double> arithmetic operation
// by operation (src/gw/pade.cpp:10-101, src/gw/qp_solver.cpp:10-47): products are
// (ac - bd, ad + bc) with no fused multiply-add (explicit __dmul_rn / __dadd_rn), and
// quotients use Smith's algorithm (R. L. Smith, "Algorithm 116: Complex division",
// CACM 5(8), 1962), the method GCC's runtime applies for std::complex<double> division in
// the normal exponent range.  Given identical Sigma_c input the device quasiparticle
// energies therefore match a host build of the reference bit for bit.
#include "internal.cuh"

#include <cmath>

namespace gwb200 {
namespace {

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx c_add(cplx a, cplx b) { return {__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }
__device__ __forceinline__ cplx c_sub(cplx a, cplx b) { return {__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)}; }
__device__ __forceinline__ cplx c_mul(cplx a, cplx b) {
    const double ac = __dmul_rn(a.re, b.re), bd = __dmul_rn(a.im, b.im);
    const double ad = __dmul_rn(a.re, b.im), bc = __dmul_rn(a.im, b.re);
    return {__dsub_rn(ac, bd), __dadd_rn(ad, bc)};
}
// Smith's algorithm, evaluated without contraction.
__device__ __forceinline__ cplx c_div(cplx x, cplx y) {
    const double a = x.re, b = x.im, c = y.re, d = y.im;
    if (fabs(c) < fabs(d)) {
        const double ratio = __ddiv_rn(c, d);
        const double denom = __dadd_rn(__dmul_rn(c, ratio), d);
        return {__ddiv_rn(__dadd_rn(__dmul_rn(a, ratio), b), denom),
                __ddiv_rn(__dsub_rn(__dmul_rn(b, ratio), a), denom)};
    }
    const double ratio = __ddiv_rn(d, c);
    const double denom = __dadd_rn(__dmul_rn(d, ratio), c);
    return {__ddiv_rn(__dadd_rn(__dmul_rn(b, ratio), a), denom),
            __ddiv_rn(__dsub_rn(b, __dmul_rn(a, ratio)), denom)};
}
__device__ __forceinline__ double c_abs(cplx a) { return hypot(a.re, a.im); }

constexpr int kMaxPade = 128;

// Thiele continued-fraction coefficients (src/gw/pade.cpp:10-63).  Only the previous column
// of the reference's table g is live, so it is kept as one vector `col` updated in place:
// after column ip, col[ip] = g(ip, ip) = coeffs[ip].
__device__ int pade_coeffs(const cplx* __restrict__ x, const cplx* __restrict__ y, int n, int npar, cplx* coeffs,
                           cplx* xs) {
    const int na = npar < n ? npar : n;
    if (na == 1) {
        coeffs[0] = y[0];
        xs[0] = x[0];
        return 1;
    }
    cplx col[kMaxPade];
    const int step = n / (na - 1);
    if (step == 0) {
        for (int i = 0; i < na; ++i) {
            xs[i] = x[i];
            col[i] = y[i];
        }
    } else {
        int idat = 0;
        for (int ip = 0; ip < na - 1; ++ip) {
            xs[ip] = x[idat];
            col[ip] = y[idat];
            idat += step;
        }
        xs[na - 1] = x[n - 1];
        col[na - 1] = y[n - 1];
    }
    coeffs[0] = col[0];
    for (int ip = 1; ip < na; ++ip) {
        const cplx pivot = col[ip - 1];
        for (int id = ip; id < na; ++id) {
            const cplx num = c_sub(pivot, col[id]);
            const cplx den = c_mul(c_sub(xs[id], xs[ip - 1]), col[id]);
            col[id] = (c_abs(den) < 1e-20) ? c_div(num, cplx{1e-20, 0.0}) : c_div(num, den);
        }
        coeffs[ip] = col[ip];
    }
    return na;
}

// Backward evaluation at real z (src/gw/pade.cpp:65-101).
__device__ cplx pade_eval(const cplx* coeffs, int npar, double z, const cplx* xs) {
    if (npar == 0) return {0.0, 0.0};
    if (npar == 1) return coeffs[0];
    const cplx zt{z, 0.0};
    cplx val{1.0, 0.0};
    for (int kr = npar - 1; kr > 0; --kr) {
        const int k = kr - 1;
        const cplx num = c_mul(coeffs[k + 1], c_sub(zt, xs[k]));
        if (c_abs(val) < 1e-20) val = cplx{1e-20, 0.0};
        val = c_add(cplx{1.0, 0.0}, c_div(num, val));
    }
    if (c_abs(val) < 1e-20) return c_div(coeffs[0], cplx{1e-20, 0.0});
    return c_div(coeffs[0], val);
}

// One thread per requested state: Pade fit of Sigma_c(p, iw) and the fixed-point QP update
// (src/gw/qp_solver.cpp:18-43), <= 200 iterations, tolerance 1e-6.
__global__ void k_qp(const double* __restrict__ sigma, const double* __restrict__ omega, int nfreq, int nmo,
                     const int64_t* __restrict__ states, int nstates, int npade, const double* __restrict__ mo,
                     double fermi, const double* __restrict__ sigx, const double* __restrict__ vxc_diag,
                     double* __restrict__ qp, cplx* __restrict__ scratch) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nstates) return;
    const int p = (int)states[s];
    cplx* x = scratch + (size_t)s * 2 * nfreq;
    cplx* y = x + nfreq;
    for (int f = 0; f < nfreq; ++f) {
        x[f] = {0.0, omega[f]};
        y[f] = {sigma[2 * ((size_t)p * nfreq + f)], sigma[2 * ((size_t)p * nfreq + f) + 1]};
    }
    cplx coeffs[kMaxPade], xs[kMaxPade];
    const int na = pade_coeffs(x, y, nfreq, npade, coeffs, xs);
    const double e = mo[p];
    double cur = e;
    for (int it = 0; it < 200; ++it) {
        const double target = __dsub_rn(cur, fermi);
        const cplx sc = pade_eval(coeffs, na, target, xs);
        const double nq = __dsub_rn(__dadd_rn(__dadd_rn(e, sc.re), sigx[p]), vxc_diag[p]);
        if (fabs(__dsub_rn(nq, cur)) < 1e-6) {
            cur = nq;
            break;
        }
        cur = nq;
    }
    qp[p] = cur;
}

// E_c.out sweep (src/io.cpp:94-108): coefficients once per block, one point per thread.
__global__ void k_pade_sweep(const double* __restrict__ sigma_row, const double* __restrict__ omega, int nfreq,
                             int npade, int npts, double fermi, double x_start, double interval,
                             double* __restrict__ out, cplx* __restrict__ scratch) {
    __shared__ cplx coeffs_s[kMaxPade], xs_s[kMaxPade];
    __shared__ int na_s;
    if (threadIdx.x == 0) {
        cplx* x = scratch + (size_t)blockIdx.x * 2 * nfreq;
        cplx* y = x + nfreq;
        for (int f = 0; f < nfreq; ++f) {
            x[f] = {0.0, omega[f]};
            y[f] = {sigma_row[2 * f], sigma_row[2 * f + 1]};
        }
        cplx coeffs[kMaxPade], xs[kMaxPade];
        const int na = pade_coeffs(x, y, nfreq, npade, coeffs, xs);
        for (int i = 0; i < na; ++i) {
            coeffs_s[i] = coeffs[i];
            xs_s[i] = xs[i];
        }
        na_s = na;
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
        const double e = __dsub_rn(__dadd_rn(x_start, __dmul_rn((double)i, interval)), fermi);
        const cplx v = pade_eval(coeffs_s, na_s, e, xs_s);
        out[3 * (size_t)i + 0] = __dmul_rn(__dadd_rn(e, fermi), 27.211386245988);
        out[3 * (size_t)i + 1] = v.re;
        out[3 * (size_t)i + 2] = v.im;
    }
}

// Sigma_c(p_s, i w_n) = -(1/pi) sum_{f', k} w_{f'} g(k, n, f') q[f', s, k], with
// g = a / (a^2 + w_{f'}^2), a = i w_n + E_F - e_k, and q = x^T W_c x <= 0 the screened forms
// (the reference's accumulation, src/gw/sigma_c_driver.cpp:154-168, with W_c hoisted out of
// the loop over w_n).  The integration frequencies f' (omega_int, weight_int, rows of qall) may be
// a shard of the output grid (omega_out): the shards' results then add up to the full sum.
// One block per (n, s); fixed-shape tree reduction (deterministic).
__global__ void __launch_bounds__(256) k_sigma_contract(const double* __restrict__ qall, int nf_int, int nmo,
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
        const double q = qall[(size_t)fp * ldq + (size_t)s * nmo + k];
        const double ar = fermi - mo[k], ai = wn;
        const double wp = omega_int[fp];
        const double dr = ar * ar - ai * ai + wp * wp, di = 2.0 * ar * ai;
        const double inv = 1.0 / (dr * dr + di * di);
        const double gr = (ar * dr + ai * di) * inv, gi = (ai * dr - ar * di) * inv;
        const double scale = -weight_int[fp] * q;
        sr = fma(gr, scale, sr);
        si = fma(gi, scale, si);
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

__global__ void k_fill(double* __restrict__ p, double v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

// Short FP64 DMMA throughput probe (8 warps/block, 4 independent accumulators per warp).
__global__ void k_dmma_probe(double* out, int iters) {
    double a = threadIdx.x * 1e-3, b = 1.0 - threadIdx.x * 1e-4;
    double c[4][2] = {};
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(c[j][0]), "+d"(c[j][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
    for (int j = 0; j < 4; ++j) s += c[j][0] + c[j][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

} // namespace

int launch_sigma_contract(const double* qall, int64_t nf_int, int64_t nstates, int64_t nmo, int64_t ldq,
                          const int64_t* states, const double* mo, double fermi, const double* omega_int,
                          const double* weight_int, const double* omega_out, int64_t nf_out, double* sigma,
                          cudaStream_t s) {
    dim3 grid((unsigned)nf_out, (unsigned)nstates);
    k_sigma_contract<<<grid, 256, 0, s>>>(qall, (int)nf_int, (int)nmo, ldq, states, mo, fermi, omega_int, weight_int,
                                          omega_out, (int)nf_out, sigma);
    GWB_LAUNCH("k_sigma_contract");
    return 1;
}

int launch_fill(double* p, double v, int64_t n, cudaStream_t s) {
    k_fill<<<(unsigned)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, s>>>(p, v, n);
    GWB_LAUNCH("k_fill");
    return 1;
}

size_t qp_scratch_bytes(int64_t nfreq, int64_t nstates) { return 2 * sizeof(cplx) * (size_t)nfreq * (size_t)nstates; }

int launch_qp(const double* sigma, const double* omega, int64_t nfreq, int64_t nmo, const int64_t* states,
              int64_t nstates, int64_t npade, const double* mo, double fermi, const double* sigx,
              const double* vxc_diag, double* qp, void* scratch, cudaStream_t s) {
    if (npade > kMaxPade) fail(GWB200_BAD_SHAPE, "npade exceeds the device Pade limit of 128");
    k_qp<<<(unsigned)((nstates + 63) / 64), 64, 0, s>>>(sigma, omega, (int)nfreq, (int)nmo, states, (int)nstates,
                                                         (int)npade, mo, fermi, sigx, vxc_diag, qp,
                                                         static_cast<cplx*>(scratch));
    GWB_LAUNCH("k_qp");
    return 1;
}

int pade_sweep_blocks(int64_t npts) { return (int)std::min<int64_t>((npts + 255) / 256, 148); }

int launch_pade_sweep(const double* sigma_row, const double* omega, int64_t nfreq, int64_t npade, int64_t npts,
                      double fermi, double x_start, double interval, double* out, void* scratch, cudaStream_t s) {
    if (npade > kMaxPade) fail(GWB200_BAD_SHAPE, "npade exceeds the device Pade limit of 128");
    k_pade_sweep<<<(unsigned)pade_sweep_blocks(npts), 256, 0, s>>>(sigma_row, omega, (int)nfreq, (int)npade,
                                                                   (int)npts, fermi, x_start, interval, out,
                                                                   static_cast<cplx*>(scratch));
    GWB_LAUNCH("k_pade_sweep");
    return 1;
}

double measure_fp64_peak_tflops(cudaStream_t s) {
    int dev = 0, sms = 0;
    GWB_CUDA(cudaGetDevice(&dev));
    GWB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double* d = nullptr;
    GWB_CUDA(cudaMalloc(&d, sizeof(double) * blocks * threads));
    cudaEvent_t e0, e1;
    GWB_CUDA(cudaEventCreate(&e0));
    GWB_CUDA(cudaEventCreate(&e1));
    k_dmma_probe<<<blocks, threads, 0, s>>>(d, 64);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        GWB_CUDA(cudaEventRecord(e0, s));
        k_dmma_probe<<<blocks, threads, 0, s>>>(d, iters);
        GWB_CUDA(cudaEventRecord(e1, s));
        GWB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GWB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    GWB_LAUNCH("k_dmma_probe");
    GWB_CUDA(cudaFree(d));
    GWB_CUDA(cudaEventDestroy(e0));
    GWB_CUDA(cudaEventDestroy(e1));
    const double flops = 2.0 * (blocks * threads / 32) * (double)iters * 4 * (8 * 8 * 4);
    return flops / (best * 1e-3) / 1e12;
}

} // namespace gwb200
