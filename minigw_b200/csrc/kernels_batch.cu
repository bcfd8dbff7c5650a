// kernels_batch.cu -- many molecules of uneven size factored by shared launches
// (gwb200_run_g0w0_batch).
//
// Molecules are sorted by size and grouped into buckets.  A bucket's tall matrices all take the
// bucket's largest geometry (n_pad, m_pad): a smaller molecule's eps is padded with identity rows
// and columns and its right-hand sides with zero rows, so its Cholesky factor is blockdiag(L, I), the
// padded right-hand sides stay exactly zero, and every real element sees the same arithmetic in the
// same order as in the molecule's own solve (padding only adds exact zeros).  The bucket's
// (molecule, frequency) matrices then go through the same launches as the frequencies of one
// molecule (launch_factor_chunk / launch_factor_chunk32), so a bucket of 20 molecules x 64
// frequencies costs one launch sequence instead of 20.
//
// The bucket boundaries trade launch latency (each bucket runs n_pad/64 dependent block steps)
// against padded work (a molecule computes at its bucket's size): plan_buckets minimises a cost
// model over contiguous groups of the sorted molecules; gwb200_run_g0w0_batch times the plans of a
// few latency weights on first use and keeps the fastest per batch signature.
//
// No counterpart in the reference (it runs one molecule per process).
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace gwb200 {
namespace {

// Tall matrices of a batched chunk.  Block (x, y, z): columns 256x.., rows y, y + gridDim.y, ..,
// group z (one molecule's run of frequencies).  Same formulas as k_build_tall / k_build_tall32;
// rows/columns past the molecule's n are the identity, right-hand-side rows past its m are zero.
template <class T>
__global__ void k_build_tall_batch(const BatchGroup* __restrict__ groups, int64_t n_pad, int64_t ld, int64_t stride,
                                   int64_t rows, T* __restrict__ a) {
    const BatchGroup gr = groups[blockIdx.z];
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_pad) return;
    const int64_t n = gr.n, m = gr.m, npi = gr.n_pad;
    T* base = a + (size_t)gr.mat0 * stride;
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
        if (r < n_pad) {
            if (c > r) continue;
            const bool inside = (r < n) && (c < n);
            const double vrc = inside ? gr.v[r * n + c] : 0.0;
            const double diag = (r == c) ? 1.0 : 0.0;
            for (int64_t f = 0; f < gr.nf; ++f) {
                const double* d = gr.dvec + (size_t)f * npi;
                const double dr = r < npi ? d[r] : 0.0, dc = c < npi ? d[c] : 0.0;
                base[(size_t)f * stride + r * ld + c] = (T)fma(dr * vrc, dc, diag);
            }
        } else {
            const int64_t j = r - n_pad;
            const double x = (j < m && c < n) ? gr.xt[j * n + c] : 0.0;
            for (int64_t f = 0; f < gr.nf; ++f) {
                const double dc = c < npi ? gr.dvec[(size_t)f * npi + c] : 0.0;
                base[(size_t)f * stride + r * ld + c] = (T)(dc * x);
            }
        }
    }
}

// Each group's forms: q_out[f, j] = -qacc[mat0 + f, j] for j < m (block y = group).
__global__ void k_forms_scatter(const BatchGroup* __restrict__ groups, const double* __restrict__ qacc, int64_t ldq) {
    const BatchGroup gr = groups[blockIdx.y];
    const int64_t total = gr.nf * gr.m;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = idx / gr.m, j = idx % gr.m;
        gr.q_out[f * gr.ldq_out + j] = -qacc[(size_t)(gr.mat0 + f) * ldq + j];
    }
}

} // namespace

int launch_build_tall_batch(const TallGeometry& g, const BatchGroup* groups, int64_t ngroups, bool fp32, void* a,
                            cudaStream_t s) {
    if (ngroups <= 0) return 0;
    const unsigned gy = (unsigned)std::min<int64_t>({g.rows, 65535, std::max<int64_t>(1, 65536 / ngroups)});
    dim3 grid((unsigned)((g.n_pad + 255) / 256), std::max(1u, gy), (unsigned)ngroups);
    if (fp32)
        k_build_tall_batch<float><<<grid, 256, 0, s>>>(groups, g.n_pad, g.ld, g.stride, g.rows, static_cast<float*>(a));
    else
        k_build_tall_batch<double><<<grid, 256, 0, s>>>(groups, g.n_pad, g.ld, g.stride, g.rows, static_cast<double*>(a));
    GWB_LAUNCH("k_build_tall_batch");
    return 1;
}

int launch_forms_scatter(const BatchGroup* groups, int64_t ngroups, const double* qacc, int64_t ldq, cudaStream_t s) {
    if (ngroups <= 0) return 0;
    k_forms_scatter<<<dim3(8, (unsigned)ngroups), 256, 0, s>>>(groups, qacc, ldq);
    GWB_LAUNCH("k_forms_scatter");
    return 1;
}

size_t batch_bytes_per_matrix(const TallGeometry& g, bool mixed, bool fp64_oz, bool refine) {
    if (mixed)  // refined: the correction's workspace at the bucket's geometry (rank <= n_pad)
        return sizeof(float) * ((size_t)g.stride + kNb * kNb) + sizeof(double) * (g.n_pad + g.m_pad) +
               tc_panel_bytes_per_freq(g) + (refine ? refine_bytes_per_freq(g, g.n_pad) : 0);
    return sizeof(double) * ((size_t)g.stride + g.n_pad + kNb * kNb + g.m_pad) + (fp64_oz ? oz_slice_bytes_per_freq(g) : 0);
}

// Contiguous groups of the molecules sorted by (n, m) that minimise
//   sum over buckets of  chunks * (n_pad / 64) * step_us  +  padded flops / rate,
// chunks = the bucket's matrices (its molecules' frequency counts f_sorted, summed) over what
// fits `budget` bytes at once, padded flops = matrices * (N^3/3 + N^2 M) at the bucket's padded
// N, M.  Dynamic programming over the end of
// the last bucket, O(nsys^2).  Returns the bucket sizes in sorted order.
std::vector<int64_t> plan_buckets(const std::vector<int64_t>& n_sorted, const std::vector<int64_t>& m_sorted,
                                  const std::vector<int64_t>& f_sorted, bool mixed, size_t budget, double step_us,
                                  double tflops) {
    const int64_t ns = (int64_t)n_sorted.size();
    std::vector<double> best((size_t)ns + 1, std::numeric_limits<double>::infinity());
    std::vector<int64_t> from((size_t)ns + 1, 0);
    std::vector<double> fsum((size_t)ns + 1, 0.0);  // prefix sums of the frequency counts
    for (int64_t i = 0; i < ns; ++i) fsum[(size_t)i + 1] = fsum[(size_t)i] + (double)f_sorted[(size_t)i];
    best[0] = 0.0;
    const double rate = std::max(tflops, 1e-3) * 1e12;
    for (int64_t k = 1; k <= ns; ++k) {
        int64_t mmax = 0;
        for (int64_t j = k; j >= 1; --j) {  // bucket = sorted molecules j-1 .. k-1
            mmax = std::max(mmax, m_sorted[(size_t)j - 1]);
            const TallGeometry g = make_geometry(n_sorted[(size_t)k - 1], mmax);
            const double nmat = fsum[(size_t)k] - fsum[(size_t)j - 1];
            const double per = (double)batch_bytes_per_matrix(g, mixed, false);
            const double fit = std::max(1.0, std::floor((double)budget / per));
            const double chunks = std::ceil(nmat / fit);
            const double N = (double)g.n_pad, M = (double)g.m_pad;
            const double cost = chunks * (double)(g.n_pad / kNb) * step_us * 1e-6 + nmat * (N * N * N / 3.0 + N * N * M) / rate;
            if (best[(size_t)j - 1] + cost < best[(size_t)k]) {
                best[(size_t)k] = best[(size_t)j - 1] + cost;
                from[(size_t)k] = j - 1;
            }
        }
    }
    std::vector<int64_t> sizes;
    for (int64_t k = ns; k > 0; k = from[(size_t)k]) sizes.push_back(k - from[(size_t)k]);
    std::reverse(sizes.begin(), sizes.end());
    return sizes;
}

} // namespace gwb200
