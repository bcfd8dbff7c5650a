/*
 * gwb200.h -- C ABI of the B200-native G0W0 screening / self-energy backend.
 *
 * One library (libgwb200.so) with plain pointers and sizes.  Host buffers are
 * borrowed for the duration of a call; device memory belongs to the handle.
 * One host thread per handle.  No exception crosses this boundary: every entry
 * point returns a gwb200_status and gwb200_last_error() gives a thread-local
 * message.  There is no CPU fallback: when the CUDA device or the sm_100a code
 * is unavailable the calls fail with GWB200_CUDA_ERROR.
 *
 * Layout contract (the reference's, include/types.hpp:15-192): every matrix is
 * row-major (C order); complex numbers are interleaved (re, im) doubles, i.e.
 * std::complex<double> / double _Complex; eri is eri_mo[p,q,r,s] in C order
 * (include/gw/integrals.hpp:28-32); states are 0-based MO indices.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * scnlong/miniGW).
 */
#ifndef GWB200_H
#define GWB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gwb200_status {
    GWB200_OK = 0,
    GWB200_BAD_SHAPE = 1,        /* nmo/nocc/nfreq/state out of range (reference: std::runtime_error) */
    GWB200_ETA_NONZERO = 2,      /* eta != 0 where only the real (eta == 0) form exists (real forms, no-alloc entry) */
    GWB200_NOT_SPD = 3,          /* Cholesky pivot <= 0 (eta == 0) or ~0 (eta != 0); stats.info = 1-based row */
    GWB200_OOM = 4,              /* device allocation failed */
    GWB200_DEVICE_TIMEOUT = 5,   /* a bounded device wait gave up */
    GWB200_CUDA_ERROR = 6,       /* CUDA runtime error, or no usable sm_100 device */
    GWB200_BAD_ARGUMENT = 7,     /* null pointer, unknown precision, bad handle */
    GWB200_NO_SYSTEM = 8,        /* sigma/qp requested before gwb200_load_system */
    GWB200_IO_ERROR = 9,         /* gw_input.h5 missing, malformed or unsupported */
    GWB200_NONPOSITIVE_GAP = 10  /* some e_a - e_i <= 0: chi0(iw) is not negative definite */
} gwb200_status;

typedef enum gwb200_precision {
    GWB200_FP64 = 0,             /* plain form: FP64 throughout (the drop-in) */
    GWB200_MIXED = 1,            /* mixed form (eta == 0): FP32 tall matrices, FP64 diagonal blocks, 3xTF32
                                  * tensor-core panel solves and updates, FP64 norms / contraction / Pade /
                                  * QP; FP32-level error (~1e-7 relative), no FP64 refinement */
    GWB200_MIXED_REFINED = 2     /* the mixed factorisation brought to FP64 accuracy (eta == 0): a backward
                                  * solve against the FP32 factor gives z ~ eps^{-1} D^1/2 x, and the forms
                                  * are the energy functional -(2 x^T D^1/2 z - z^T eps z) evaluated in FP64
                                  * (error quadratic in the FP32 solve error, ~1e-14 relative); y^T V y
                                  * through a pivoted Cholesky factor of V computed once per loaded system.
                                  * Every screening entry point and gwb200_run_g0w0_batch; not the
                                  * no-allocation entry */
} gwb200_precision;

typedef struct gwb200_stats {
    double device_ms_total;      /* CUDA-event time of the whole call */
    double device_ms_gather;     /* V_ph / panel gathers */
    double device_ms_screening;  /* eps build + Cholesky + panel solve (all frequency chunks) */
    double device_ms_contract;   /* G0-weighted frequency contraction */
    double flops_screening;      /* algorithmic flops n^3/3 + n^2 m + 3 n m per frequency, summed */
    int64_t frequency_chunks;    /* frequency chunks the screening was split into (HBM budget) */
    int64_t kernel_launches;     /* kernels this call launched */
    int64_t info;                /* NOT_SPD: 1-based failing pivot; else 0 */
    int64_t nph;                 /* n = nocc * nvir */
    int64_t ncols;               /* m = nstates * nmo */
    /* Filled only when the environment sets GWB200_PROFILE=1: CUDA-event time summed over the
     * launches of the trailing-update kernel (the dominant kernel), their count, and their
     * algorithmic flops (lower-triangle and right-hand-side tiles of the true n, m). */
    double device_ms_update;
    int64_t update_launches;
    double flops_update;
} gwb200_stats;

typedef struct gwb200_handle gwb200_handle;

/* Thread-local description of the last failure on this thread ("" if none). */
const char* gwb200_last_error(void);

/* Library / build information, e.g. "gwb200 sm_100a fp64-dmma". */
const char* gwb200_version(void);

/* Create a handle bound to CUDA device `device` (it owns a stream and device buffers).
 * Replaces: gw::workspace::DeviceScreeningWorkspace construction and the device
 * selection gw::linalg::set_cuda_device_for_local_rank
 * (include/workspace/device_screening_workspace.hpp:27-59, src/linalg/linalg_cublas.cu:393-405). */
int gwb200_create(int device, gwb200_handle** out);

/* Release every device buffer of the handle.  Safe on NULL. */
int gwb200_destroy(gwb200_handle* h);

/* Issue the handle's work on the caller's CUDA stream (a cudaStream_t passed as void*; NULL
 * restores the handle's own stream), so a caller can order and time it with its own events.
 * No reference counterpart: the reference's device workspace owns its implicit stream
 * (src/workspace/device_screening_workspace.cu:288-310). */
int gwb200_set_stream(gwb200_handle* h, void* stream);

/* Cap the device memory this handle may hold (resident system + workspaces); the frequency chunk is
 * sized to fit.  0 = no cap beyond the device's free memory.  No reference counterpart (the
 * reference sizes nothing: it allocates per call). */
int gwb200_set_memory_limit(gwb200_handle* h, int64_t bytes);

/* Upload one molecular system and build its resident device state: the occupied-virtual
 * index map, the V_ph=(jb|ia) gather and the exchange diagonal.  eri (nmo^4), mo_energy
 * (nmo) and vxc (nmo^2) are borrowed for the call.
 * Replaces: gw::OrbitalSpace / gw::ParticleHoleBasis (include/gw/orbital_space.hpp:10-70,
 * include/gw/particle_hole.hpp:18-59), gw::calculate_v_ph_matrix (src/gw/sigma.cpp:56-71),
 * gw::workspace::DeviceScreeningWorkspace(v_ph) (src/workspace/device_screening_workspace.cu:288-310)
 * and gw::workspace::DevicePqPhPanelView (src/workspace/device_pq_ph_panel.cu:168-237). */
int gwb200_load_system(gwb200_handle* h, int64_t nmo, int64_t nocc, const double* mo_energy,
                       const double* eri, const double* vxc, double fermi_energy);

/* gwb200_load_system for a known state list: only V_ph = (ia|jb) (n^2 doubles), the panel rows
 * (p k|i a) of the given states (nstates * nmo * n doubles) and the exchange diagonal are copied
 * from eri (3D copies of contiguous runs of nvir doubles), instead of the (pq|o.) block
 * (nmo^3 * nocc doubles): 0.29 GB instead of 1.92 GB at nmo = 200, nocc = 30, 10 states.  Later
 * calls on the handle must pass this same state list (same order); results are bit-identical
 * to gwb200_load_system's.  Replaces the same reference code as gwb200_load_system, with the
 * (p k|ov) slices of gw::workspace::DevicePqPhPanelView::fill_panel
 * (src/workspace/device_pq_ph_panel.cu:141-166) taken once per state. */
int gwb200_load_system_states(gwb200_handle* h, int64_t nmo, int64_t nocc, const double* mo_energy,
                              const double* eri, const double* vxc, double fermi_energy,
                              const int64_t* states, int64_t nstates);

/* gwb200_load_system_states from inputs the caller has already sliced, for callers that never hold
 * the nmo^4 ERI (34 GB at nmo = 256): vph (n x n) V_ph[jb, ia] = (jb|ia); panel (nstates*nmo x n),
 * row t*nmo + k = (states[t] k|ia); xdiag (nmo x nocc) = (p i|p i); vxc_diag (nmo) the diagonal of
 * vxc_mo; all host memory, row-major, with n = nocc * (nmo - nocc) and ia = i*nvir + (a - nocc).
 * Contiguous copies; later calls use `states` as after gwb200_load_system_states, and the results
 * are bit-identical to loading the full ERI these slices were cut from.  Replaces the same
 * reference code as gwb200_load_system_states, with the hyperslab reads of the input the reference
 * does with its HDF5 reader (src/hdf5_input.cpp:192-212) moved to the caller. */
int gwb200_load_system_slices(gwb200_handle* h, int64_t nmo, int64_t nocc, const double* mo_energy,
                              const double* vph, const double* panel, const double* xdiag,
                              const double* vxc_diag, double fermi_energy, const int64_t* states,
                              int64_t nstates);

/* Correlation self-energy Sigma_c(i w_n) on the imaginary grid for the requested states.
 * sigma_out is nmo x nfreq complex, row-major (gw::MatrixComplex); rows of states not
 * requested are set to zero.  eta == 0: real SPD Cholesky of eps = I + D^1/2 V D^1/2;
 * eta != 0: complex symmetric L L^T of I - S V S with S = diag(Pi0)^1/2 (no pivoting).
 * Replaces: gw::compute_sigma_c_with_backend (src/gw/sigma_c_driver.cpp:451-592) with the
 * device branch (:471-514): compute_w_c (src/workspace/device_screening_workspace.cu:337-374),
 * fill_panel (src/workspace/device_pq_ph_panel.cu:284), quadratic_forms_panel (:376-417) and the
 * Sigma accumulation (src/gw/sigma_c_driver.cpp:186-222). */
int gwb200_sigma_c(gwb200_handle* h, const double* omega, const double* weight, int64_t nfreq,
                   const int64_t* states, int64_t nstates, double eta, int precision,
                   double* sigma_out, gwb200_stats* stats);

/* Correlation self-energy between the requested states, Sigma_c(p_s, p_t; i w_n), plain FP64 form,
 * eta = 0, 1 <= nstates <= 64: sigma_out is nstates x nstates x nfreq complex (element (s, t, n) at
 * 2 * ((s * nstates + t) * nfreq + n)), symmetric in (s, t); its diagonal is gwb200_sigma_c's rows
 * of the states to rounding.  The cross forms x_{p_s k}^T W_c x_{p_t k} come from the solved
 * right-hand-side rows of the same factorisation, and the frequency contraction is the diagonal's.
 * No counterpart in the reference: it computes the diagonal only (docs/formulation.md:186); this
 * is the data an off-diagonal QP Hamiltonian would start from. */
int gwb200_sigma_c_matrix(gwb200_handle* h, const double* omega, const double* weight, int64_t nfreq,
                          const int64_t* states, int64_t nstates, double* sigma_out, gwb200_stats* stats);

/* The contribution of the integration frequencies f' in [f_begin, f_end) of the grid to Sigma_c at
 * every output frequency of the grid: sigma_partial_out is nmo x nfreq complex.  The partial sums of
 * a partition of [0, nfreq) add up to gwb200_sigma_c's result (up to summation order); ranks that
 * each solve one shard of one system reduce them with one all-reduce of nmo x nfreq complex.
 * Replaces: the MPI frequency distribution of compute_sigma_c_serial_or_mpi + mpi_allreduce_sum_in_place
 * (src/gw/sigma_c_driver.cpp:368-401, 507-512; src/mpi_context.cpp:45-64), split here over the
 * integration frequency f' (each W_c solved once) instead of the output frequency f_n. */
int gwb200_sigma_c_shard(gwb200_handle* h, const double* omega, const double* weight, int64_t nfreq,
                         int64_t f_begin, int64_t f_end, const int64_t* states, int64_t nstates, double eta,
                         int precision, double* sigma_partial_out, gwb200_stats* stats);

/* One whole G0W0 solve on the device for the loaded system: the transformed Gauss-Legendre grid,
 * Sigma_c(iw) for the requested states, the exchange diagonal and the QP energies, with Sigma_c
 * staying on the device between the screening and the Pade/QP step (one host synchronisation).
 * Outputs are optional (NULL skips): omega_out/weight_out nfreq, sigma_out nmo x nfreq complex,
 * sigma_x_out nmo, qp_out nmo (NaN where not requested).
 * Replaces: gw::run_g0w0 (src/gw/gw.cpp:125-191) past input loading: grid (:138),
 * calculate_exchange (:149), compute_sigma_c_with_backend (:163-172), solve_qp_energies (:180-186). */
int gwb200_run_g0w0(gwb200_handle* h, int64_t nfreq, int64_t npade, const int64_t* states, int64_t nstates,
                    double eta, int precision, double* omega_out, double* weight_out, double* sigma_out,
                    double* sigma_x_out, double* qp_out, gwb200_stats* stats);

/* Copies of the resident screening inputs, for checking the gathers bit for bit.  vph_out (n x n,
 * row-major): V_ph[jb, ia] = (jb|ia), as gw::calculate_v_ph_matrix builds it (src/gw/sigma.cpp:56-71).
 * panel_out (nstates*nmo x n, row-major): row s*nmo + k = (p_s k|ia), i.e. the columns of the panels
 * gw::workspace::PqPhPanelView::fill_panel fills (src/workspace/pq_ph_panel.cpp:25-47) for state p_s.
 * Either output may be NULL.  After gwb200_load_system the panel rows are gathered from the resident
 * (pq|o.) block by the kernel the screening calls use; after gwb200_load_system_states `states` must be
 * the bound list (the rows are the resident ones).  Exported for checking; it replaces nothing. */
int gwb200_read_resident(gwb200_handle* h, const int64_t* states, int64_t nstates, double* vph_out,
                         double* panel_out);

/* Screened quadratic forms Q[f, s, k] = x_{p_s k}^T W_c(i w_f) x_{p_s k} (real, <= 0) at eta == 0
 * (GWB200_ETA_NONZERO otherwise), layout [nfreq][nstates][nmo].  The per-frequency quantity the reference computes as
 * quadratic_forms_panel (src/workspace/screening_workspace.cpp:69-102); exported for checking. */
int gwb200_screened_forms(gwb200_handle* h, const double* omega, int64_t nfreq, const int64_t* states,
                          int64_t nstates, double eta, int precision, double* q_out, gwb200_stats* stats);

/* Screened quadratic forms for any eta as complex numbers (layout [nfreq][nstates][nmo], interleaved
 * re/im): x^T W_c x of the reference's quadratic_forms_panel (src/workspace/screening_workspace.cpp:69-102).
 * At eta == 0 the imaginary parts are zero. */
int gwb200_screened_forms_complex(gwb200_handle* h, const double* omega, int64_t nfreq, const int64_t* states,
                                  int64_t nstates, double eta, double* q_out, gwb200_stats* stats);

/* Diagonal of the exchange self-energy, Sigma_x[p,p] = -sum_{i<nocc} (p i | p i), out[nmo].
 * Replaces: gw::calculate_exchange (src/gw/sigma.cpp:22-39) (only its diagonal is consumed,
 * src/gw/qp_solver.cpp:36 and src/io.cpp:110-126). */
int gwb200_sigma_x_diag(gwb200_handle* h, double* out);

/* Quasiparticle energies by Pade continuation of Sigma_c and the fixed-point update, on the
 * device in FP64.  sigma is nmo x nfreq complex (as returned by gwb200_sigma_c), qp_out[nmo]
 * is NaN for states not requested.
 * Replaces: gw::solve_qp_energies (src/gw/qp_solver.cpp:10-47) with
 * get_pade_coefficients_continued_fraction / evaluate_pade_continued_fraction (src/gw/pade.cpp:10-101). */
int gwb200_qp(gwb200_handle* h, const double* omega, int64_t nfreq, const double* sigma, int64_t npade,
              const int64_t* states, int64_t nstates, double* qp_out);

/* Pade continuation of one state's Sigma_c(iw) (sigma_row: nfreq complex) evaluated on the real
 * axis at e_i = x_start + i*interval - fermi, i < npts; out is npts x 3: (e_i+fermi)*Ha->eV, Re, Im.
 * Replaces: gw::output_self_energy_after_pade's sweep (src/io.cpp:94-108). */
int gwb200_pade_sweep(gwb200_handle* h, const double* omega, int64_t nfreq, const double* sigma_row,
                      int64_t npade, int64_t npts, double fermi, double x_start, double interval,
                      double* out);

/* Transformed Gauss-Legendre grid (host, FP64, same arithmetic as the reference).
 * Replaces: gw::generate_transformed_legendre_grid (src/gw/frequency_grids.cpp:62-93). */
int gwb200_grid(int64_t nfreq, double* omega, double* weight);

/* Minimal reader for gw_input.h5 (HDF5 superblock v0/v1, v1 object headers, symbol-table groups,
 * contiguous or compact float64 datasets, scalar attributes).  Call with eri/mo/vxc NULL to query
 * nmo, nocc and fermi; then with buffers of nmo^4, nmo and nmo^2 doubles.
 * Replaces: gw::read_gw_input_hdf5 (src/hdf5_input.cpp:192-212). */
int gwb200_read_input_h5(const char* path, int64_t* nmo, int64_t* nocc, double* fermi_energy,
                         double* mo_energy, double* eri, double* vxc);

/* gw_input.h5 read for a known state list without the nmo^4 ERI tensor in memory: only the slices
 * gwb200_load_system_slices takes are read from /eri_mo (one contiguous run of nocc*nmo doubles
 * per row of V_ph and of the panel, single elements for the exchange diagonal), with the layouts
 *   vph       n x n              vph[(j*nvir + b)*n + i*nvir + a]  = eri[j, nocc+b, i, nocc+a]
 *   panel     (nstates*nmo) x n  panel[(t*nmo + k)*n + i*nvir + a] = eri[states[t], k, i, nocc+a]
 *   xdiag     nmo x nocc         xdiag[p*nocc + i] = eri[p, i, p, i]
 *   vxc_diag  nmo                vxc_mo[p, p]
 * (n = nocc*nvir), plus mo_energy (nmo).  Call with all five output arrays NULL to query nmo, nocc
 * and fermi (states may then be NULL); otherwise every array must be given and every state be in
 * [0, nmo) (GWB200_BAD_SHAPE).  Config 3 (nmo = 200, 10 states): 0.29 GB read instead of 12.8 GB.
 * No counterpart in the reference, which reads the whole tensor (src/hdf5_input.cpp:192-212). */
int gwb200_read_input_h5_slices(const char* path, const int64_t* states, int64_t nstates, int64_t* nmo,
                                int64_t* nocc, double* fermi_energy, double* mo_energy, double* vph,
                                double* panel, double* xdiag, double* vxc_diag);

/* Screened quadratic forms with NO device allocation, for callers that cannot call cudaMalloc
 * (a framework whose caching allocator owns the device memory, a serving loop that cannot take
 * the device-wide synchronisation of cudaMalloc/cudaFree, a process admitted under a fixed memory
 * budget).  Same result as gwb200_screened_forms, from caller-owned DEVICE buffers:
 *   d_v      n x n   V_ph[jb, ia] = (jb|ia), row-major
 *   d_xt     m x n   the right-hand sides, row j = x_j[ia] (e.g. (p_s k|ia) for j = s*nmo + k)
 *   d_delta  n       e_a - e_i, all > 0
 *   d_omega  nfreq   imaginary frequencies
 *   d_q_out  nfreq x m  x_j^T W_c(i w_f) x_j (<= 0), row-major
 * on `stream` (a cudaStream_t as void*, NULL = the legacy default stream) of the CURRENT device.
 * Every intermediate lives in one file-scope device array of 4 MiB that each GPU loading the
 * library holds until exit; one frequency must fit: (n64 + m64) * n64 + n64 + 4096 + m64 doubles
 * <= 524256 (n64, m64 = n, m rounded up to 64), e.g. n = m = 320, else GWB200_BAD_SHAPE.  Every
 * buffer must be device (or managed) memory of the current device, else GWB200_BAD_ARGUMENT.  Each
 * call looks up that array's device address (cudaGetSymbolAddress; the first call on a device
 * loads the library's device code there).  The call reads the factorisation's pivot flag back and
 * synchronises `stream` before it returns, so it cannot be captured into a CUDA graph.
 * All calls share the array and it keeps the last call's contents: calls that overlap on the GPU
 * race and must be serialised by the caller.
 * No counterpart in the reference (an addition of this library). */
int gwb200_screened_forms_noalloc(int64_t n, int64_t m, const double* d_v, const double* d_xt,
                                  const double* d_delta, const double* d_omega, int64_t nfreq,
                                  double* d_q_out, void* stream);

/* ---- Serving: a continuous-batching request loop (no reference counterpart) ----
 * One request = one G0W0 solve.  All pointers are host memory owned by the caller and must stay
 * valid until gwb200_server_wait returns for the request's ticket.  Outputs (may be NULL) are
 * filled when the request completes: omega/weight nfreq, sigma nmo x nfreq complex, sigma_x and
 * qp nmo. */
typedef struct gwb200_request {
    int64_t nmo, nocc;
    const double* mo_energy;  /* nmo */
    const double* eri;        /* nmo^4, C order */
    const double* vxc;        /* nmo^2 */
    double fermi_energy;
    int64_t nfreq, npade;
    const int64_t* states;
    int64_t nstates;
    double eta;
    int precision;
    double* omega_out;
    double* weight_out;
    double* sigma_out;
    double* sigma_x_out;
    double* qp_out;
} gwb200_request;

typedef struct gwb200_server gwb200_server;

/* Start `slots` workers on `device`, each with its own handle and stream and a device-memory cap
 * of hbm_budget_bytes / slots.  Requests are admitted FIFO as workers free up; requests in
 * different slots overlap on the GPU.  Results do not depend on which requests ran alongside. */
int gwb200_server_create(int device, int slots, int64_t hbm_budget_bytes, gwb200_server** out);

/* Queue one request (non-blocking).  GWB200_OOM if it cannot fit one slot's budget. */
int gwb200_server_submit(gwb200_server* s, const gwb200_request* req, int64_t* ticket);

/* The system of a request as pre-cut slices (gwb200_load_system_slices' inputs, host memory owned
 * by the caller until the request completes). */
typedef struct gwb200_request_slices {
    const double* vph;       /* n x n */
    const double* panel;     /* nstates*nmo x n */
    const double* xdiag;     /* nmo x nocc */
    const double* vxc_diag;  /* nmo */
} gwb200_request_slices;

/* gwb200_server_submit for a request whose system comes as slices: req->eri and req->vxc are not
 * read (may be NULL), the worker loads with gwb200_load_system_slices. */
int gwb200_server_submit_slices(gwb200_server* s, const gwb200_request* req, const gwb200_request_slices* slices,
                                int64_t* ticket);

/* Block until the request completes; its status is returned (and in *status), with the time it
 * waited for a slot, its service time (host, from admission to results) and its device time. */
int gwb200_server_wait(gwb200_server* s, int64_t ticket, int* status, double* queue_ms, double* service_ms,
                       double* device_ms);

/* Finish every queued request, stop the workers, release their handles. */
int gwb200_server_destroy(gwb200_server* s);

/* Continuous batching across requests: a worker that frees up takes, besides the oldest request,
 * further waiting requests that can share launches with it (eta == 0, the same precision, at most
 * 1536 particle-hole pairs: larger requests fill the GPU alone; their
 * resident data plus one frequency of the largest tall matrix within 80% of the slot's budget), up
 * to max_requests in all and to a fair share of the waiting requests per worker, and solves them
 * together with gwb200_run_g0w0_batch, each on a handle of its own.  Results are bit-identical to
 * the requests' own solves.  1 turns merging off; the default is 8. */
int gwb200_server_set_merge(gwb200_server* s, int max_requests);

/* Batches of two or more requests solved so far, and the requests in them. */
int gwb200_server_counters(gwb200_server* s, int64_t* merged_batches, int64_t* merged_requests);

/* ---- Batched solves: many molecules of uneven size in shared launches (no reference counterpart;
 * the reference runs one molecule per process, src/main.cpp:68-103) ----
 * systems[i] holds molecule i (gwb200_load_system or gwb200_load_system_states), all on one device,
 * no handle twice, at most 65535.  Molecule i is solved as gwb200_run_g0w0(systems[i], nfreq[i],
 * npade[i], states[i], nstates[i], 0, precision, ...) would solve it (eta = 0, any precision; frequency and Pade
 * counts may differ between molecules).  The molecules are sorted by size and grouped into
 * buckets; a bucket's matrices (every member x every one of its frequencies) take the bucket's
 * largest geometry (identity / zero padding, exact) and are factored by shared launches on up to 4
 * streams.  Bucket boundaries: a cost model (block-step latency against padded work) gives
 * candidate plans, timed on the first call of a batch signature (sorted sizes and frequency
 * counts, precision); the fastest is kept for later calls in the process
 * (GWB200_BATCH_PLAN=model|each|single skips the timing).  A repeated call with one plan replays
 * a CUDA graph of the whole sequence while no buffer has moved.  All work runs on systems[0]'s
 * stream with systems[0]'s workspaces.  Outputs (either array, or any entry, may be NULL):
 * sigma_out[i] nmo_i x nfreq[i] complex row-major, qp_out[i] nmo_i (NaN where not requested).
 * *nbuckets_out: the buckets used.  stats: totals of the call (flops at the true sizes, device
 * times, launches).  Each result is bit-identical to the molecule's own gwb200_run_g0w0. */
int gwb200_run_g0w0_batch(gwb200_handle* const* systems, int64_t nsys, const int64_t* nfreq,
                          const int64_t* npade, const int64_t* const* states, const int64_t* nstates,
                          int precision, double* const* sigma_out, double* const* qp_out,
                          int64_t* nbuckets_out, gwb200_stats* stats);

/* The cost model's bucket plan alone (host only, no device): bucket_of[i] in 0..*nbuckets-1 for
 * molecules of nph[i] x ncols[i] (buckets in ascending size), budget_bytes of device memory for the
 * batched matrices, step_us / tflops the model's block-step latency and padded-work rate
 * (<= 0: the defaults). */
int gwb200_plan_buckets(int64_t nsys, const int64_t* nph, const int64_t* ncols, int64_t nfreq, int precision,
                        int64_t budget_bytes, double step_us, double tflops, int64_t* bucket_of,
                        int64_t* nbuckets);

/* Measured FP64 tensor (DMMA) throughput of this device in TFLOP/s, from a short
 * microbenchmark of mma.sync f64 (used as the roofline denominator of the plain form). */
int gwb200_fp64_peak_tflops(gwb200_handle* h, double* tflops);

/* The trailing-update kernel the last screening call on this handle used (no counterpart in the
 * reference; for rooflines and diagnostics): 0-5 one of the FP64 DMMA variants, 6 the int8
 * tensor-core emulation of the FP64 update, 7 the mixed form's tcgen05 3xTF32 update, 8 the mixed
 * form's mma.sync update, -1 none (no outer trailing update, eta != 0, or no call yet). */
int gwb200_update_kernel(gwb200_handle* h, int64_t* kernel);

/* Device time of the memory-bound kernels, for their HBM rooflines (no counterpart in the
 * reference).  While the environment sets GWB200_PROFILE=1 each launch of these kernels on the
 * handle is bracketed by CUDA events on its stream; this call synchronises the stream and returns,
 * summed since the previous call (then reset), per kind k: ms_out[k] the event time, bytes_out[k]
 * the algorithmic bytes, launches_out[k] the launches.  Kinds: 0 k_gather_vph (V_ph gather, 16 n^2
 * bytes; gwb200_load_system), 1 k_gather_panel (panel rows, 16 n m; screening calls after
 * gwb200_load_system), 2 k_build_tall / k_build_tall32 (eps and right-hand sides of a frequency chunk:
 * 8 (n^2 + n m) read + (n64 (n64 + 1) / 2 + m64 n64) elements of 8 or 4 bytes written per frequency),
 * 3 k_sigma_contract (8 F m + 16 nmo F).  Launches captured into a CUDA graph are not timed. */
int gwb200_kernel_profile(gwb200_handle* h, double* ms_out, double* bytes_out, int64_t* launches_out);

#ifdef __cplusplus
}
#endif

#endif /* GWB200_H */
