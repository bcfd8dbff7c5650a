// internal.cuh -- shared declarations of libgwb200 (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gwb200.h"

// Sets the calling thread's gwb200_last_error() message and returns `code` (gwb200_abi.cu).
int gwb200_fail_status(int code, const char* message);
// Exact-size buffers of a memory-limited handle come from `pool` (gwb200_abi.cu; used by the server).
void gwb200_attach_pool(gwb200_handle* h, cudaMemPool_t pool);
// A handle that shares the GPU with `ways` concurrent streams caps its persistent kernels'
// grids at SMs / ways, so that the other streams' kernels keep running beside them.
void gwb200_share_sms(gwb200_handle* h, int ways);

namespace gwb200 {

// Error carrying a gwb200_status across the host code; converted to a return code
// at the C-ABI boundary.
struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Failure(code, msg); }

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? GWB200_OOM : GWB200_CUDA_ERROR;
        fail(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" + std::to_string(line) + ")");
    }
}
#define GWB_CUDA(x) ::gwb200::cuda_check((x), #x, __FILE__, __LINE__)
#define GWB_LAUNCH(what) ::gwb200::cuda_check(cudaGetLastError(), what, __FILE__, __LINE__)

// Block size of the right-looking Cholesky (rows/cols of one diagonal block) and
// the square tile edge of every DMMA tile kernel.
constexpr int kNb = 64;
// Padded shared-memory row stride (doubles) of a 64-wide tile: 68*8 B rows put the
// 8 rows touched by one m8n8k4 fragment load on distinct banks.
constexpr int kLds = 68;
// Default variant of the trailing-update kernel (index into the table in kernels_fp64.cu).
constexpr int kDefaultUpdateVariant = 0;

// Geometry of one frequency chunk of the tall screening matrices
//   A_f = [ eps_f (n_pad x n_pad, lower) ; B_f^T (m_pad x n_pad) ],  row-major, ld = n_pad.
struct TallGeometry {
    int64_t n;      // nph
    int64_t m;      // nstates * nmo (right-hand sides)
    int64_t n_pad;  // n rounded up to kNb
    int64_t m_pad;  // m rounded up to kNb
    int64_t rows;   // n_pad + m_pad
    int64_t ld;     // n_pad
    int64_t stride; // rows * ld (elements per frequency)
};

inline int64_t round_up(int64_t x, int64_t r) { return (x + r - 1) / r * r; }

inline TallGeometry make_geometry(int64_t n, int64_t m) {
    TallGeometry g{};
    g.n = n;
    g.m = m;
    g.n_pad = round_up(n, kNb);
    g.m_pad = round_up(m, kNb);
    g.rows = g.n_pad + g.m_pad;
    g.ld = g.n_pad;
    g.stride = g.rows * g.ld;
    return g;
}

// Optional event timing of every trailing-update launch (the dominant kernel).
struct UpdateProfiler {
    bool enabled;
    cudaStream_t stream;
    std::vector<cudaEvent_t> events;  // pairs (start, stop)
    double flops = 0.0;
    UpdateProfiler(bool on, cudaStream_t s) : enabled(on), stream(s) {}
    ~UpdateProfiler() {
        for (auto e : events) cudaEventDestroy(e);
    }
    void begin() {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate", __FILE__, __LINE__);
        cuda_check(cudaEventRecord(e, stream), "cudaEventRecord", __FILE__, __LINE__);
        events.push_back(e);
    }
    void end(double launch_flops) {
        begin();
        flops += launch_flops;
    }
    void collect(gwb200_stats* st) {
        cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize", __FILE__, __LINE__);
        double ms = 0.0;
        for (size_t i = 0; i + 1 < events.size(); i += 2) {
            float t = 0.f;
            cuda_check(cudaEventElapsedTime(&t, events[i], events[i + 1]), "cudaEventElapsedTime", __FILE__, __LINE__);
            ms += t;
        }
        st->device_ms_update = ms;
        st->update_launches = (int64_t)(events.size() / 2);
        st->flops_update = flops;
    }
};

// ---- kernel launchers (kernels_fp64.cu, kernels_small.cu) ----
// pqo: the device-resident (pq|o.) block, pqo[(p*nmo + q)*nocc + i][s] = eri[p,q,i,s], i < nocc.
int launch_gather_vph(const double* pqo, int64_t nmo, int64_t nocc, double* v, cudaStream_t s);
int launch_gather_panel(const double* pqo, int64_t nmo, int64_t nocc, const int64_t* states, int64_t nstates,
                        double* xt, cudaStream_t s);
// xdiag[p*nocc + i] = eri[p,i,p,i]
int launch_sigma_x_diag(const double* xdiag, int64_t nmo, int64_t nocc, double* out, cudaStream_t s);
int launch_delta(const double* mo, int64_t nmo, int64_t nocc, double* delta, int* bad_gap, cudaStream_t s);
int launch_scale_vectors(const double* delta, int64_t n, int64_t n_pad, const double* omega, int64_t nf,
                         double* dvec, cudaStream_t s);
int launch_build_tall(const TallGeometry& g, const double* v, const double* xt, const double* dvec, int64_t nf,
                      double* a, cudaStream_t s);
// Blocked Cholesky of the tall matrices of nf frequencies (outer blocks of two 64-wide inner
// blocks); returns launches issued.
// `variant`: index into the FP64 update kernel table (tune_update_variant); -1: GWB200_UPDATE_VARIANT
// if set, else the default; kUpdateOzaki: the outer trailing updates run as the int8 emulation of
// kernels_oz.cu with `oz` as its slice workspace (oz_slice_bytes_per_freq(g) per frequency) and
// `sched` as its work counter (look-left updates on the default DMMA kernel).
int launch_factor_chunk(const TallGeometry& g, int64_t nf, double* a, double* linv, double* qacc,
                        unsigned long long* err_pivot, cudaStream_t s, UpdateProfiler* prof, int variant,
                        void* oz = nullptr, unsigned long long* sched = nullptr, int max_ctas = 0);
// kernels_oz.cu: FP64 trailing update C -= P P^T (K = 128 from kb0, columns [c_begin, n_pad), rows
// [c_begin, rows)) from exact int8 products of 6-digit row slices (tcgen05 kind::i8).  Two launches.
size_t oz_slice_bytes_per_freq(const TallGeometry& g);
// max_ctas > 0 caps the persistent grid (a handle that shares the GPU with other streams).
int launch_update64_oz(const TallGeometry& g, int64_t nf, double* a, int64_t kb0, int64_t c_begin, void* slices,
                       unsigned long long* sched, unsigned long long* err_pivot, cudaStream_t s, int max_ctas = 0);
// Autotuner of the FP64 trailing-update kernel: GWB200_UPDATE_VARIANT if set, else the fastest
// candidate on this geometry's largest trailing update, timed once per (device, n_pad, rows, nf)
// per process in the workspace `a` (nf tall matrices) BEFORE the matrices are built there (the
// timing overwrites it).  The default is kept unless another candidate is more than 3% faster.
// oz != NULL adds the int8 emulation of the outer updates (kernels_oz.cu) as a candidate
// (kUpdateOzaki), timed with the slicing; GWB200_FP64_UPDATE=dmma / =ozaki force either side.
// Timed candidates: the default DMMA kernel and the int8 emulation (all six DMMA variants with
// GWB200_TUNE_ALL=1).  timed == false (memory-capped handles, whose requests run side by side and
// rarely repeat a geometry): no timing, the default DMMA kernel.
constexpr int kUpdateOzaki = 6;
int fp64_update_mode();
int tune_update_variant(const TallGeometry& g, int64_t nf, double* a, cudaStream_t s, void* oz = nullptr,
                        unsigned long long* sched = nullptr, unsigned long long* err_pivot = nullptr,
                        bool timed = true);
const char* update_variant_name(int v);
// kernels_offdiag.cu: the cross forms q[f][k][s][t] = -w_{s,k} . w_{t,k} of a factored chunk of
// nf tall matrices (nstates <= 64), and their contraction into Sigma_c(p_s, p_t; i w_n) (layout
// [s][t][n] complex interleaved), the diagonal's G0 weighting.
int launch_cross_forms(const TallGeometry& g, int64_t nf, const double* a, int64_t nmo, int64_t nstates, double* qx,
                       cudaStream_t s);
int launch_sigma_contract_pairs(const double* qx, int64_t nf_int, int64_t nmo, int64_t nstates, const double* mo,
                                double fermi, const double* omega_int, const double* weight_int,
                                const double* omega_out, int64_t nf_out, double* sigma, cudaStream_t s);
// Contraction of the screened forms of nf_int integration frequencies onto nf_out output
// frequencies (the full grid; a shard of integration frequencies gives a partial sum).
int launch_sigma_contract(const double* qall, int64_t nf_int, int64_t nstates, int64_t nmo, int64_t ldq,
                          const int64_t* states, const double* mo, double fermi, const double* omega_int,
                          const double* weight_int, const double* omega_out, int64_t nf_out, double* sigma,
                          cudaStream_t s);
int launch_fill(double* p, double v, int64_t n, cudaStream_t s);
// scratch: qp_scratch_bytes(nfreq, nstates) bytes of device memory
size_t qp_scratch_bytes(int64_t nfreq, int64_t nstates);
int launch_qp(const double* sigma, const double* omega, int64_t nfreq, int64_t nmo, const int64_t* states,
              int64_t nstates, int64_t npade, const double* mo, double fermi, const double* sigx,
              const double* vxc_diag, double* qp, void* scratch, cudaStream_t s);
// scratch: qp_scratch_bytes(nfreq, pade_sweep_blocks(npts)) bytes of device memory
int pade_sweep_blocks(int64_t npts);
int launch_pade_sweep(const double* sigma_row, const double* omega, int64_t nfreq, int64_t npade, int64_t npts,
                      double fermi, double x_start, double interval, double* out, void* scratch, cudaStream_t s);
int launch_negate_copy(const double* qacc, int64_t nf, int64_t m, int64_t ldq_in, double* q_out, int64_t ldq_out,
                       cudaStream_t s);
double measure_fp64_peak_tflops(cudaStream_t s);
// kernels_f32.cu: the mixed-precision form (FP32 tall matrices, 3xTF32 tensor-core updates).
int launch_build_tall32(const TallGeometry& g, const double* v, const double* xt, const double* dvec, int64_t nf,
                        float* a, cudaStream_t s);
// panel != NULL: the outer trailing updates run on tcgen05 (kernels_tc.cu) with `panel` as the
// split-panel workspace (tc_panel_bytes_per_freq(g) bytes per frequency); NULL: mma.sync.
int launch_factor_chunk32(const TallGeometry& g, int64_t nf, float* a, float* linv, double* qacc,
                          unsigned long long* err_pivot, cudaStream_t s, UpdateProfiler* prof, float* panel,
                          unsigned long long* sched, int max_ctas = 0, bool solve_only = false);
// kernels_refine.cu: FP64 energy-functional correction of the mixed form.  launch_pchol factors
// V = C C^T (pivoted, FP64; `work` of pchol_bytes(n)), returns the rank r and C^T (r_pad x n_pad,
// r_pad = max(64, r rounded up to 64)) in *ct_out (inside `work`).  launch_refine_chunk runs after
// launch_factor_chunk32 on the same chunk: the backward solve against the FP32 factor (solve-only
// pass), then qacc[f][j] = 2 x^T y - z^T z - y^T V y (`work`: refine_bytes_per_freq(g, r_pad) * nf).
// The factor of V a correction uses: C^T (r_pad x n_pad FP64, r_pad = r rounded up to 64) for the
// DMMA Gram product, and its digit slices (gram_oz_system_bytes, launch_slice_ct) for the int8 one.
struct RefineFactor {
    const double* ct;
    int64_t r_pad;
    const void* ct_slices;
    int64_t rank;
};
size_t refine_bytes_per_freq(const TallGeometry& g, int64_t r_pad);
size_t pchol_bytes(int64_t n);
int64_t launch_pchol(const double* v, int64_t n, void* work, double** ct_out, cudaStream_t s);
int launch_refine_chunk(const TallGeometry& g, int64_t nf, float* a, float* linv, const double* xt,
                        const double* dvec, const RefineFactor& fac, void* work, double* qacc,
                        unsigned long long* err_pivot, cudaStream_t s, float* panel, unsigned long long* sched,
                        int max_ctas);
// GWB200_REFINE_GRAM=dmma runs y^T V y on the FP64 pipe; by default on the int8 tensor cores
// (when gram_oz_fits).
bool refine_gram_on_int8(int64_t n_pad);
// kernels_gram_oz.cu: y^T V y = ||C^T y||^2 from int8 digit slices (tcgen05 kind::i8).
int64_t gram_oz_rows(int64_t r);
// the int8 path (exact int32 sums, y of a right-hand side in shared memory) takes n_pad up to 25600; beyond, DMMA
bool gram_oz_fits(int64_t n_pad);
size_t refine_oz_bytes_per_freq(const TallGeometry& g, int64_t r);
size_t gram_oz_system_bytes(int64_t n_pad, int64_t r);
void launch_slice_ct(const double* ct, int64_t r, int64_t n_pad, void* out, cudaStream_t s);
int launch_refine_terms_oz(const TallGeometry& ga, int64_t nf, const float* a, const TallGeometry& gm,
                           const double* xt, const double* dvec, const void* ct_slices, int64_t r, void* work,
                           unsigned long long* err, cudaStream_t s, double** t12_out, double** part_out,
                           int64_t* nkt_out);
// The parts of launch_refine_chunk, for batches: the in-place reversal-transpose of the factor and
// the reversal of the right-hand sides within the first n_flip indices (a molecule's own n_pad: it
// sits in the top-left corner of the chunk's matrices, identity-padded, so its blocks keep the
// positions they have in its own solve); the backward solve of a chunk of geometry g (flip: first
// the reversal over g.n_pad); the correction terms of one molecule (own geometry gm) for its nf
// matrices from `a`, into qacc (row stride ldq).
int launch_refine_flip(const TallGeometry& ga, int64_t nf, float* a, int64_t n_flip, cudaStream_t s);
int launch_refine_solve(const TallGeometry& g, int64_t nf, float* a, float* linv, unsigned long long* err_pivot,
                        cudaStream_t s, float* panel, unsigned long long* sched, int max_ctas, bool flip);
int launch_refine_terms(const TallGeometry& ga, int64_t nf, const float* a, const TallGeometry& gm, const double* xt,
                        const double* dvec, const RefineFactor& fac, void* work, double* qacc, int64_t ldq,
                        unsigned long long* err, cudaStream_t s);
// kernels_tc.cu: tcgen05 3xTF32 trailing update C -= P P^T of the mixed form (K = kdim columns from
// kb0, output columns [c_begin, n_pad), rows [c_begin, rows)).  Two launches; `sched` is one
// device word the kernel's work counter lives in.  A device wait that expires records pivot 0 in
// err_pivot.
size_t tc_panel_bytes_per_freq(const TallGeometry& g);
int launch_update32_tc(const TallGeometry& g, int64_t nf, float* a, int64_t kb0, int kdim, int64_t c_begin,
                       float* panel, unsigned long long* sched, unsigned long long* err_pivot, cudaStream_t s,
                       int max_ctas = 0, int64_t row_min = 0);
// kernels_c64.cu: eta != 0 (complex symmetric M = I - S V S, S = diag(Pi0)^1/2).  Planes a_re/a_im
// of geometry g; svec 2*n_pad, linv 2*64*64, qacc 2*m_pad doubles per frequency.
int launch_factor_chunk_c(const TallGeometry& g, int64_t nf, const double* delta, const double* omega, double eta,
                          const double* v, const double* xt, double* a_re, double* a_im, double* svec, double* linv,
                          double* qacc, unsigned long long* err_pivot, cudaStream_t s);
int launch_forms_out_c(const double* qacc, int64_t nf, int64_t m, int64_t ldq, double* q_out, int64_t ldq_out,
                       cudaStream_t s);
int launch_sigma_contract_c(const double* qall, int64_t nf_int, int64_t nstates, int64_t nmo, int64_t ldq,
                            const int64_t* states, const double* mo, double fermi, const double* omega_int,
                            const double* weight_int, const double* omega_out, int64_t nf_out, double* sigma,
                            cudaStream_t s);
// kernels_batch.cu: one molecule's run of consecutive matrices in a batched chunk (device table).
struct BatchGroup {
    const double* v;     // V_ph, n x n
    const double* xt;    // (D-independent) panel rows, m x n
    const double* dvec;  // scale vectors of the group's first frequency, then one per frequency (n_pad apart)
    double* q_out;       // forms of the group's first frequency, ldq_out apart
    int64_t n, m, n_pad, ldq_out;
    int64_t mat0, nf;    // first matrix of the chunk this group fills, and how many (frequencies)
    RefineFactor fac;    // refined mixed form: the molecule's pivoted Cholesky factor of V
};
int launch_build_tall_batch(const TallGeometry& g, const BatchGroup* groups, int64_t ngroups, bool fp32, void* a,
                            cudaStream_t s);
int launch_forms_scatter(const BatchGroup* groups, int64_t ngroups, const double* qacc, int64_t ldq, cudaStream_t s);
// device bytes of one batched matrix (tall matrix, 64x64 inverse, scale vector, norm accumulators,
// tcgen05 / int8 operand workspace)
size_t batch_bytes_per_matrix(const TallGeometry& g, bool mixed, bool fp64_oz, bool refine = false);
// bucket sizes over the molecules sorted by (n, m): minimises block-step latency + padded work
std::vector<int64_t> plan_buckets(const std::vector<int64_t>& n_sorted, const std::vector<int64_t>& m_sorted,
                                  const std::vector<int64_t>& f_sorted, bool mixed, size_t budget, double step_us,
                                  double tflops);

// noalloc.cu
size_t noalloc_scratch_bytes();
void screened_forms_noalloc(int64_t n, int64_t m, const double* d_v, const double* d_xt, const double* d_delta,
                            const double* d_omega, int64_t nfreq, double* d_q_out, cudaStream_t s);

// ---- host helpers (host_grid.cpp, host_h5.cpp) ----
void transformed_legendre_grid(int64_t n, double* omega, double* weight);
void read_gw_input_h5(const std::string& path, int64_t* nmo, int64_t* nocc, double* fermi, double* mo, double* eri,
                      double* vxc);
void read_gw_input_h5_slices(const std::string& path, const int64_t* states, int64_t nstates, int64_t* nmo,
                             int64_t* nocc, double* fermi, double* mo, double* vph, double* panel, double* xdiag,
                             double* vxc_diag);

} // namespace gwb200
