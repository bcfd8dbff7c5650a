// kernels_offdiag.cu -- the correlation self-energy between the requested states, Sigma_c(p_s, p_t; i w):
// an extension beside the reference, which computes the diagonal only (docs/formulation.md:186).
//
// The plain form factors the tall matrix [eps ; (D^1/2 X)^T] per frequency; its lower block ends as
// the solved rows w_{s,k} = L^{-1} D^1/2 x_{p_s k} (tall row n_pad + s nmo + k), whose squared norms
// are the diagonal forms.  The same rows give every cross form at the cost of dot products:
//     q[f, k, s, t] = x_{p_s k}^T W_c(i w_f) x_{p_t k} = -w_{s,k} . w_{t,k}
// and the G0-weighted contraction of the diagonal (kernels_small.cu, src/gw/sigma_c_driver.cpp:
// 119-169) applies unchanged, the Green's function depending on k only:
//     Sigma_c(p_s, p_t; i w_n) = -(1/pi) sum_{f,k} w_f g_{n f k} q[f, k, s, t],
//     g_{n f k} = a / (a^2 + w_f^2),  a = i w_n + E_F - e_k.
//   k_cross_forms          one CTA per (k, frequency): the nstates rows staged in shared memory in
//                          chunks of the row length, each thread the running dot products of its
//                          (s <= t) pairs in a fixed order;
//   k_sigma_contract_pairs one CTA per (output frequency, pair s <= t): the contraction, a fixed
//                          reduction tree; both triangles written.
#include "internal.cuh"

namespace gwb200 {
namespace {

constexpr int kXThreads = 256;
constexpr int kXSmem = 48 * 1024;  // default dynamic shared memory, no opt-in needed

// (s, t) with s <= t of upper-triangle index p (row-major: row s holds t = s .. ns-1).
__device__ __forceinline__ void pair_of(int p, int ns, int& s, int& t) {
    s = 0;
    while (p >= ns - s) {
        p -= ns - s;
        ++s;
    }
    t = s + p;
}

__global__ void __launch_bounds__(kXThreads) k_cross_forms(const double* __restrict__ a, int64_t ld, int64_t stride,
                                                           int64_t n, int64_t n_pad, int nmo, int ns, int ch,
                                                           double* __restrict__ qx) {
    extern __shared__ double xsm[];
    const int k = blockIdx.x, f = blockIdx.y;
    const int npair = ns * (ns + 1) / 2;
    const int ldr = ch + 1;  // odd row stride: the pair loop's reads spread over the banks
    double* rows = xsm;
    double* acc = xsm + (size_t)ns * ldr;
    for (int p = threadIdx.x; p < npair; p += kXThreads) acc[p] = 0.0;
    const double* A = a + (size_t)f * stride;
    for (int64_t i0 = 0; i0 < n; i0 += ch) {
        const int len = (int)min((int64_t)ch, n - i0);
        __syncthreads();  // the previous chunk's reads are done
        for (int idx = threadIdx.x; idx < ns * ch; idx += kXThreads) {
            const int s = idx / ch, c = idx - s * ch;
            rows[s * ldr + c] = c < len ? A[(size_t)(n_pad + (int64_t)s * nmo + k) * ld + i0 + c] : 0.0;
        }
        __syncthreads();
        for (int p = threadIdx.x; p < npair; p += kXThreads) {
            int s, t;
            pair_of(p, ns, s, t);
            const double* rs = rows + s * ldr;
            const double* rt = rows + t * ldr;
            double sum = acc[p];
            for (int c = 0; c < len; ++c) sum = fma(rs[c], rt[c], sum);
            acc[p] = sum;
        }
    }
    __syncthreads();
    double* out = qx + ((size_t)f * nmo + k) * ns * ns;
    for (int p = threadIdx.x; p < npair; p += kXThreads) {
        int s, t;
        pair_of(p, ns, s, t);
        out[s * ns + t] = -acc[p];
        out[t * ns + s] = -acc[p];
    }
}

__global__ void __launch_bounds__(256) k_sigma_contract_pairs(const double* __restrict__ qx, int nf_int, int nmo,
                                                              int ns, const double* __restrict__ mo, double fermi,
                                                              const double* __restrict__ omega_int,
                                                              const double* __restrict__ weight_int,
                                                              const double* __restrict__ omega_out, int nf_out,
                                                              double* __restrict__ sigma) {
    const int fn = blockIdx.x;
    int s, t;
    pair_of(blockIdx.y, ns, s, t);
    const double wn = omega_out[fn];
    double sr = 0.0, si = 0.0;
    const int total = nf_int * nmo;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int fp = idx / nmo, k = idx - fp * nmo;
        const double q = qx[((size_t)fp * nmo + k) * ns * ns + (size_t)s * ns + t];
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
        if ((int)threadIdx.x < off) {
            red[0][threadIdx.x] += red[0][threadIdx.x + off];
            red[1][threadIdx.x] += red[1][threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double inv_pi = 1.0 / 3.141592653589793238462643383279502884;
        for (int e = 0; e < (s == t ? 1 : 2); ++e) {
            const size_t pos = (size_t)(e == 0 ? s * ns + t : t * ns + s) * nf_out + fn;
            sigma[2 * pos] = red[0][0] * inv_pi;
            sigma[2 * pos + 1] = red[1][0] * inv_pi;
        }
    }
}

} // namespace

int launch_cross_forms(const TallGeometry& g, int64_t nf, const double* a, int64_t nmo, int64_t nstates, double* qx,
                       cudaStream_t s) {
    const int ns = (int)nstates;
    const int npair = ns * (ns + 1) / 2;
    // rows chunk: ns rows of (ch + 1) doubles and the pair accumulators in 48 KB, ch a multiple of 32
    int ch = (int)(((size_t)kXSmem / sizeof(double) - (size_t)npair) / (size_t)ns) - 1;
    ch = std::max(32, ch / 32 * 32);
    const size_t smem = sizeof(double) * ((size_t)ns * (ch + 1) + npair);
    if (smem > (size_t)kXSmem) fail(GWB200_BAD_SHAPE, "too many states for the cross forms");
    k_cross_forms<<<dim3((unsigned)nmo, (unsigned)nf), kXThreads, smem, s>>>(a, g.ld, g.stride, g.n, g.n_pad, (int)nmo,
                                                                              ns, ch, qx);
    GWB_LAUNCH("k_cross_forms");
    return 1;
}

int launch_sigma_contract_pairs(const double* qx, int64_t nf_int, int64_t nmo, int64_t nstates, const double* mo,
                                double fermi, const double* omega_int, const double* weight_int,
                                const double* omega_out, int64_t nf_out, double* sigma, cudaStream_t s) {
    const int64_t npair = nstates * (nstates + 1) / 2;
    k_sigma_contract_pairs<<<dim3((unsigned)nf_out, (unsigned)npair), 256, 0, s>>>(
        qx, (int)nf_int, (int)nmo, (int)nstates, mo, fermi, omega_int, weight_int, omega_out, (int)nf_out, sigma);
    GWB_LAUNCH("k_sigma_contract_pairs");
    return 1;
}

} // namespace gwb200
