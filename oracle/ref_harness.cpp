// ref_harness.cpp -- TEST INFRASTRUCTURE: a C-ABI driver around the reference's
// own compiled sources (oracle/_ref/libgwref.so, built by oracle/Makefile from the
// reference's src/ tree where it lies; no reference source is copied here).
//
// It lets tests/ pin the oracle restatement (oracle/gw_oracle.c) against the real
// reference, and lets bench.py time the reference's own CPU path (the
// "reference" arm and cpu_baseline).  Only tests/, __graft_entry__.smoke() and
// bench.py load it.
//
// Entry points:
//   ref_g0w0        -- the sequence of gw::run_g0w0 (src/gw/gw.cpp:125-191) with an
//                      explicit state list, driven through the public
//                      compute_sigma_c_with_backend (src/gw/sigma_c_driver.cpp:451)
//                      and solve_qp_energies (src/gw/qp_solver.cpp:10).
//   ref_run_g0w0    -- gw::run_g0w0 itself (single selected state or all states).
//   ref_forms       -- q[f,s,k] = x^T W_c(iw_f) x via HostScreeningWorkspace
//                      (src/workspace/screening_workspace.cpp:21-102).
//   ref_resident    -- V_ph (calculate_v_ph_matrix) and the panel columns of the
//                      requested states (PqPhPanelView::make_panel), for bit-exact
//                      checks of the device gathers.
//   ref_pair_seconds-- wall time of the body of the reference's per-(f_n, f') loop
//                      (src/gw/sigma_c_driver.cpp:133-164) over `npairs` pairs,
//                      run on `threads` OpenMP threads like the reference's OpenMP
//                      frequency mode (src/gw/sigma_c_driver.cpp:403-447).
//   ref_grid / ref_pade_coeffs / ref_pade_eval / ref_write_ec -- thin wrappers.
#include "gw/frequency_grids.hpp"
#include "gw/gw.hpp"
#include "gw/pade.hpp"
#include "gw/qp_solver.hpp"
#include "gw/sigma.hpp"
#include "gw/sigma_c_driver.hpp"
#include "io.hpp"
#include "linalg/linalg_blas_lapack.hpp"
#include "workspace/pq_ph_panel.hpp"
#include "workspace/screening_workspace.hpp"

#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using i64 = std::int64_t;

namespace {

thread_local std::string g_last_error;

std::shared_ptr<const gw::linalg::Backend> pick_backend(int backend) {
    if (backend == 1) return gw::linalg::make_blas_lapack_backend();
    return gw::linalg::make_reference_backend();
}

gw::GwInput make_input(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc) {
    gw::GwInput in;
    const auto n = static_cast<std::size_t>(nmo);
    in.mo_energy.assign(mo, mo + n);
    in.vxc_mo = gw::MatrixReal(n, n, std::vector<double>(vxc, vxc + n * n));
    in.eri_mo = gw::Tensor4Real(n, n, n, n, std::vector<double>(eri, eri + n * n * n * n));
    in.nocc = static_cast<std::size_t>(nocc);
    in.fermi_energy = fermi;
    return in;
}

struct SilenceCout {
    std::streambuf* old;
    std::ostringstream sink;
    SilenceCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~SilenceCout() { std::cout.rdbuf(old); }
};

} // namespace

extern "C" {

const char* ref_last_error() { return g_last_error.c_str(); }

int ref_g0w0(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc,
             i64 nfreq, i64 npade, const i64* states, i64 nstates, double eta, int backend, int openmp_freq,
             double* sigma_out, double* qp_out, double* sigx_out, double* omegas_out, double* weights_out,
             double* wall_seconds) {
    try {
        SilenceCout quiet;
        const auto t0 = std::chrono::steady_clock::now();
        gw::GwInput in = make_input(nmo, nocc, fermi, mo, eri, vxc);
        gw::OrbitalSpace orbitals(in.mo_energy, in.nocc, in.fermi_energy);
        gw::MolecularIntegrals integrals(std::move(in.eri_mo), std::move(in.vxc_mo));
        const gw::ParticleHoleBasis ph(orbitals);
        gw::GwSettings settings;
        settings.num_freq_points_total = static_cast<std::size_t>(nfreq);
        settings.num_pade_params = static_cast<std::size_t>(npade);
        settings.eta = eta;
        settings.linalg_backend = pick_backend(backend);
        if (openmp_freq) {
            settings.execution.frequency_parallel_mode = gw::FrequencyParallelMode::OpenMP;
            settings.execution.openmp_frequency_parallel = true;
            settings.execution.openmp_kernel_loops = false;
        }
        auto [omegas, weights] = gw::generate_transformed_legendre_grid(settings.num_freq_points_total);
        const gw::MatrixReal sigma_x = gw::calculate_exchange(orbitals, integrals);
        std::vector<gw::Complex> omega_im(omegas.size());
        for (std::size_t i = 0; i < omegas.size(); ++i) omega_im[i] = gw::Complex{0.0, omegas[i]};
        gw::MatrixComplex sigma(orbitals.nmo(), settings.num_freq_points_total, gw::Complex{0.0, 0.0});
        std::vector<std::size_t> st(static_cast<std::size_t>(nstates));
        for (i64 s = 0; s < nstates; ++s) st[static_cast<std::size_t>(s)] = static_cast<std::size_t>(states[s]);
        gw::GwTimings timings;
        gw::compute_sigma_c_with_backend(orbitals, integrals, ph, omega_im, weights, st, settings,
                                         *settings.linalg_backend, sigma, timings);
        const std::vector<double> qp =
            gw::solve_qp_energies(orbitals, integrals, sigma_x, sigma, omega_im, st, settings);
        const auto t1 = std::chrono::steady_clock::now();
        std::memcpy(sigma_out, sigma.data().data(), sizeof(gw::Complex) * sigma.size());
        std::memcpy(qp_out, qp.data(), sizeof(double) * qp.size());
        std::memcpy(sigx_out, sigma_x.data().data(), sizeof(double) * sigma_x.size());
        std::memcpy(omegas_out, omegas.data(), sizeof(double) * omegas.size());
        std::memcpy(weights_out, weights.data(), sizeof(double) * weights.size());
        if (wall_seconds) *wall_seconds = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int ref_run_g0w0(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc,
                 i64 nfreq, i64 npade, i64 state0, int backend, double* sigma_out, double* qp_out,
                 double* sigx_out) {
    try {
        SilenceCout quiet;
        gw::GwInput in = make_input(nmo, nocc, fermi, mo, eri, vxc);
        gw::GwSettings settings;
        settings.num_freq_points_total = static_cast<std::size_t>(nfreq);
        settings.num_pade_params = static_cast<std::size_t>(npade);
        if (state0 >= 0) settings.selected_state_0based = static_cast<std::size_t>(state0);
        else settings.selected_state_0based.reset();
        settings.linalg_backend = pick_backend(backend);
        const gw::GwResult r = gw::run_g0w0(in, settings);
        std::memcpy(sigma_out, r.sigma_c_im_points.data().data(), sizeof(gw::Complex) * r.sigma_c_im_points.size());
        std::memcpy(qp_out, r.qp_energy.data(), sizeof(double) * r.qp_energy.size());
        std::memcpy(sigx_out, r.sigma_x.data().data(), sizeof(double) * r.sigma_x.size());
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int ref_forms(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc,
              i64 nf, const double* omegas, const i64* states, i64 nstates, double eta, int backend,
              i64 panel, double* q_out) {
    try {
        gw::GwInput in = make_input(nmo, nocc, fermi, mo, eri, vxc);
        gw::OrbitalSpace orbitals(in.mo_energy, in.nocc, in.fermi_energy);
        gw::MolecularIntegrals integrals(std::move(in.eri_mo), std::move(in.vxc_mo));
        const gw::ParticleHoleBasis ph(orbitals);
        const auto be = pick_backend(backend);
        gw::workspace::HostScreeningWorkspace screening(gw::calculate_v_ph_matrix(integrals, ph), *be);
        const gw::workspace::PqPhPanelView view(integrals, ph);
        auto* q = reinterpret_cast<gw::Complex*>(q_out);
        const auto unmo = static_cast<std::size_t>(nmo);
        const auto upanel = static_cast<std::size_t>(panel > 0 ? panel : 32);
        for (i64 f = 0; f < nf; ++f) {
            const auto pi0 = gw::calculate_pi0_ph_diag(gw::Complex{0.0, omegas[f]}, ph, eta);
            const gw::MatrixComplex w = screening.compute_w_c(pi0);
            for (i64 s = 0; s < nstates; ++s) {
                for (std::size_t k0 = 0; k0 < unmo; k0 += upanel) {
                    const std::size_t width = std::min(upanel, unmo - k0);
                    const gw::MatrixReal x = view.make_panel(static_cast<std::size_t>(states[s]), k0, width);
                    const auto vals = screening.quadratic_forms_panel(w, x);
                    for (std::size_t kk = 0; kk < width; ++kk)
                        q[(static_cast<std::size_t>(f * nstates + s)) * unmo + k0 + kk] = vals[kk];
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// The reference's V_ph (gw::calculate_v_ph_matrix, src/gw/sigma.cpp:56-71) into vph_out (n x n, may be
// NULL) and, for each state, the panel columns k = 0..nmo-1 of PqPhPanelView::make_panel
// (src/workspace/pq_ph_panel.cpp:18-47) transposed into panel_out rows s*nmo + k (may be NULL).
int ref_resident(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc,
                 const i64* states, i64 nstates, double* vph_out, double* panel_out) {
    try {
        gw::GwInput in = make_input(nmo, nocc, fermi, mo, eri, vxc);
        gw::OrbitalSpace orbitals(in.mo_energy, in.nocc, in.fermi_energy);
        gw::MolecularIntegrals integrals(std::move(in.eri_mo), std::move(in.vxc_mo));
        const gw::ParticleHoleBasis ph(orbitals);
        const std::size_t n = ph.size(), unmo = static_cast<std::size_t>(nmo);
        if (vph_out) {
            const gw::MatrixReal v = gw::calculate_v_ph_matrix(integrals, ph);
            std::memcpy(vph_out, v.data().data(), sizeof(double) * v.size());
        }
        if (panel_out) {
            const gw::workspace::PqPhPanelView view(integrals, ph);
            for (i64 s = 0; s < nstates; ++s) {
                const gw::MatrixReal x = view.make_panel(static_cast<std::size_t>(states[s]), 0, unmo);
                double* dst = panel_out + static_cast<std::size_t>(s) * unmo * n;
                for (std::size_t r = 0; r < n; ++r)
                    for (std::size_t k = 0; k < unmo; ++k) dst[k * n + r] = x(r, k);
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int ref_pair_seconds(i64 nmo, i64 nocc, double fermi, const double* mo, const double* eri, const double* vxc,
                     i64 npairs, const double* omegas_fp, double omega_n, const double* weights_fp,
                     const i64* states, i64 nstates, int backend, int threads, double* seconds,
                     double* checksum) {
    try {
        gw::GwInput in = make_input(nmo, nocc, fermi, mo, eri, vxc);
        gw::OrbitalSpace orbitals(in.mo_energy, in.nocc, in.fermi_energy);
        gw::MolecularIntegrals integrals(std::move(in.eri_mo), std::move(in.vxc_mo));
        const gw::ParticleHoleBasis ph(orbitals);
        const auto be = pick_backend(backend);
        gw::workspace::HostScreeningWorkspace screening(gw::calculate_v_ph_matrix(integrals, ph), *be);
        const gw::workspace::PqPhPanelView view(integrals, ph);
        const std::size_t unmo = orbitals.nmo();
        const std::size_t panel_size = 32;
        std::vector<gw::Complex> acc(static_cast<std::size_t>(npairs), gw::Complex{0.0, 0.0});
        const gw::Complex omega_n_im{0.0, omega_n};
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
        for (i64 pr = 0; pr < npairs; ++pr) {
            // body of src/gw/sigma_c_driver.cpp:133-164 for one f'
            const gw::Complex omega_prime_im{0.0, omegas_fp[pr]};
            const auto pi0 = gw::calculate_pi0_ph_diag(omega_prime_im, ph, 0.0);
            const gw::MatrixComplex w_c = screening.compute_w_c(pi0);
            gw::Complex cur{0.0, 0.0};
            for (i64 s = 0; s < nstates; ++s) {
                for (std::size_t k0 = 0; k0 < unmo; k0 += panel_size) {
                    const std::size_t width = std::min(panel_size, unmo - k0);
                    const gw::MatrixReal x = view.make_panel(static_cast<std::size_t>(states[s]), k0, width);
                    const auto vals = screening.quadratic_forms_panel(w_c, x);
                    for (std::size_t kk = 0; kk < width; ++kk) {
                        const gw::Complex den = omega_n_im + orbitals.fermi_energy() - orbitals.energy(k0 + kk);
                        const gw::Complex g0 = den / (den * den - omega_prime_im * omega_prime_im);
                        cur -= g0 * vals[kk] * weights_fp[pr];
                    }
                }
            }
            acc[static_cast<std::size_t>(pr)] = cur;
        }
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
        gw::Complex sum{0.0, 0.0};
        for (const auto& a : acc) sum += a;
        checksum[0] = sum.real();
        checksum[1] = sum.imag();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int ref_grid(i64 n, double* omegas, double* weights) {
    try {
        auto [o, w] = gw::generate_transformed_legendre_grid(static_cast<std::size_t>(n));
        std::memcpy(omegas, o.data(), sizeof(double) * o.size());
        std::memcpy(weights, w.data(), sizeof(double) * w.size());
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

i64 ref_pade_coeffs(i64 n, const double* x, const double* y, i64 npar, double* coeffs, double* xs) {
    try {
        const auto* xc = reinterpret_cast<const gw::Complex*>(x);
        const auto* yc = reinterpret_cast<const gw::Complex*>(y);
        std::vector<gw::Complex> xv(xc, xc + n), yv(yc, yc + n);
        auto [c, s] = gw::get_pade_coefficients_continued_fraction(xv, yv, static_cast<std::size_t>(npar));
        std::memcpy(coeffs, c.data(), sizeof(gw::Complex) * c.size());
        std::memcpy(xs, s.data(), sizeof(gw::Complex) * s.size());
        return static_cast<i64>(c.size());
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

void ref_pade_eval(i64 npar, const double* coeffs, double z, const double* xs, double* out) {
    const auto* cc = reinterpret_cast<const gw::Complex*>(coeffs);
    const auto* xc = reinterpret_cast<const gw::Complex*>(xs);
    std::vector<gw::Complex> cv(cc, cc + npar), xv(xc, xc + npar);
    const gw::Complex v = gw::evaluate_pade_continued_fraction(cv, z, xv);
    out[0] = v.real();
    out[1] = v.imag();
}

int ref_write_ec(const char* path, i64 nfreq, const double* sigma_row, const double* omegas, i64 npar,
                 i64 npts, double fermi) {
    try {
        const auto* sc = reinterpret_cast<const gw::Complex*>(sigma_row);
        std::vector<gw::Complex> st(sc, sc + nfreq);
        std::vector<double> om(omegas, omegas + nfreq);
        gw::output_self_energy_after_pade(path, st, om, static_cast<std::size_t>(npar),
                                          static_cast<std::size_t>(npts), fermi);
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

} // extern "C"
