/*
 * gw_oracle.c -- CPU ORACLE for the per-frequency G0W0 screening and self-energy path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the reference
 * miniGW algorithm (scnlong/miniGW) used as the checker in tests/, in
 * __graft_entry__.smoke() and in bench.py's cpu_baseline leg.  The product path
 * (minigw_b200/, libgwb200.so) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement against the
 * reference's committed H2O golden vectors (regression_tests/h2o_serial/
 * E_c_before_Pade.out, E_c.out, gw.out) and, where oracle/_ref was built from
 * the reference's own sources, against the reference itself on synthetic inputs.
 *
 * Every function cites the reference file:line it restates.  Arithmetic follows
 * the reference's operation order (complex double, C99 _Complex semantics match
 * std::complex<double> under GCC), so on x86-64 without FMA contraction the
 * results match the reference bit for bit.  Build with -ffp-contract=off.
 *
 * One deliberate reorganisation: the reference rebuilds W_c(f') inside the loop
 * over output frequencies f_n (src/gw/sigma_c_driver.cpp:119-169), i.e. nfreq^2
 * times.  W_c(f') does not depend on f_n and the reference's arithmetic is
 * deterministic, so this oracle computes the screened quadratic forms
 * q[f', p, k] once per f' and replays the reference's accumulation loop over
 * (f_n, f', p, k) in the reference's order.  The result is identical.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex zc;
typedef int64_t i64;

static const double kPi = 3.141592653589793238462643383279502884;

/* ------------------------------------------------------------------------- */
/* Orbital space / particle-hole map.
 * include/gw/orbital_space.hpp:48-64 (occ = 0..nocc-1, vir = nocc..nmo-1),
 * include/gw/particle_hole.hpp:22-35 (ph = i_occ*nvir + a_vir, delta = e_a - e_i). */
int gwo_ph_map(i64 nmo, i64 nocc, const double* mo, i64* i_occ, i64* a_mo, double* delta) {
    if (nmo <= 0 || nocc <= 0 || nocc >= nmo) return -1;
    const i64 nvir = nmo - nocc;
    for (i64 i = 0; i < nocc; ++i) {
        for (i64 a = 0; a < nvir; ++a) {
            const i64 ph = i * nvir + a;
            i_occ[ph] = i;
            a_mo[ph] = nocc + a;
            delta[ph] = mo[nocc + a] - mo[i];
        }
    }
    return 0;
}

static inline double eri_at(const double* eri, i64 nmo, i64 p, i64 q, i64 r, i64 s) {
    /* include/gw/integrals.hpp:28-32: exact C-order payload eri_mo[p,q,r,s]. */
    return eri[((p * nmo + q) * nmo + r) * nmo + s];
}

/* src/gw/sigma.cpp:56-71: V_ph[jb, ia] = eri(j, b, i, a), row-major n x n. */
void gwo_vph(i64 nmo, i64 nocc, const double* eri, double* v) {
    const i64 nvir = nmo - nocc, n = nocc * nvir;
    for (i64 ia = 0; ia < n; ++ia) {
        const i64 i = ia / nvir, a = nocc + ia % nvir;
        for (i64 jb = 0; jb < n; ++jb) {
            const i64 j = jb / nvir, b = nocc + jb % nvir;
            v[jb * n + ia] = eri_at(eri, nmo, j, b, i, a);
        }
    }
}

/* src/gw/sigma.cpp:22-39: Sigma_x[p,q] = -sum_{k<nocc} eri(p,k,q,k), nmo x nmo row-major. */
void gwo_exchange(i64 nmo, i64 nocc, const double* eri, double* sx) {
    for (i64 q = 0; q < nmo; ++q) {
        for (i64 p = 0; p < nmo; ++p) {
            double value = 0.0;
            for (i64 k = 0; k < nocc; ++k) value -= eri_at(eri, nmo, p, k, q, k);
            sx[p * nmo + q] = value;
        }
    }
}

/* src/gw/sigma.cpp:41-54: Pi0[ph] = 2 * (1/(w - d + i eta) - 1/(w + d - i eta)), w complex. */
void gwo_pi0(double omega_re, double omega_im, i64 n, const double* delta, double eta, double* out_c) {
    const zc omega = CMPLX(omega_re, omega_im);
    const zc ieta = CMPLX(0.0, eta);
    zc* out = (zc*)out_c;
    for (i64 ph = 0; ph < n; ++ph) {
        const zc term = CMPLX(1.0, 0.0) / (omega - delta[ph] + ieta) - CMPLX(1.0, 0.0) / (omega + delta[ph] - ieta);
        out[ph] = 2.0 * term;
    }
}

/* src/linalg/linalg.cpp:44-91: Gauss-Jordan inverse with partial pivoting (row-major).
 * Returns 0, or -1 on a near-singular pivot (|pivot| < 1e-14), like the reference's throw. */
int gwo_inverse(i64 n, double* a_c, double* inv_c) {
    zc* a = (zc*)a_c;
    zc* inv = (zc*)inv_c;
    for (i64 i = 0; i < n * n; ++i) inv[i] = 0.0;
    for (i64 i = 0; i < n; ++i) inv[i * n + i] = 1.0;
    for (i64 col = 0; col < n; ++col) {
        i64 pivot = col;
        double pivot_abs = cabs(a[col * n + col]);
        for (i64 row = col + 1; row < n; ++row) {
            const double cand = cabs(a[row * n + col]);
            if (cand > pivot_abs) { pivot_abs = cand; pivot = row; }
        }
        if (pivot_abs < 1e-14) return -1;
        if (pivot != col) {
            for (i64 j = 0; j < n; ++j) {
                zc t = a[col * n + j]; a[col * n + j] = a[pivot * n + j]; a[pivot * n + j] = t;
                t = inv[col * n + j]; inv[col * n + j] = inv[pivot * n + j]; inv[pivot * n + j] = t;
            }
        }
        const zc diag = a[col * n + col];
        for (i64 j = 0; j < n; ++j) { a[col * n + j] /= diag; inv[col * n + j] /= diag; }
        for (i64 row = 0; row < n; ++row) {
            if (row == col) continue;
            const zc factor = a[row * n + col];
            if (cabs(factor) == 0.0) continue;
            for (i64 j = 0; j < n; ++j) {
                a[row * n + j] -= factor * a[col * n + j];
                inv[row * n + j] -= factor * inv[col * n + j];
            }
        }
    }
    return 0;
}

/* src/workspace/screening_workspace.cpp:21-66:
 * eps_left = I - diag(Pi0) V, W_c = eps_left^{-1}, then W_c[:,k] *= Pi0[k]. */
int gwo_w_c(i64 n, const double* v, const double* pi0_c, double* w_c) {
    const zc* pi0 = (const zc*)pi0_c;
    zc* w = (zc*)w_c;
    zc* eps = (zc*)malloc(sizeof(zc) * (size_t)(n * n));
    if (!eps) return -2;
    for (i64 i = 0; i < n; ++i)
        for (i64 k = 0; k < n; ++k) eps[i * n + k] = -pi0[i] * CMPLX(v[i * n + k], 0.0);
    for (i64 i = 0; i < n; ++i) eps[i * n + i] += CMPLX(1.0, 0.0);
    const int rc = gwo_inverse(n, (double*)eps, (double*)w);
    free(eps);
    if (rc) return rc;
    for (i64 i = 0; i < n; ++i)
        for (i64 k = 0; k < n; ++k) w[i * n + k] *= pi0[k];
    return 0;
}

/* src/workspace/pq_ph_panel.cpp:25-47: X(ph, kk) = eri(p, k0+kk, i, a), row-major n x width. */
void gwo_panel(i64 nmo, i64 nocc, const double* eri, i64 p, i64 k0, i64 width, double* x) {
    const i64 nvir = nmo - nocc, n = nocc * nvir;
    for (i64 ph = 0; ph < n; ++ph) {
        const i64 i = ph / nvir, a = nocc + ph % nvir;
        for (i64 kk = 0; kk < width; ++kk) x[ph * width + kk] = eri_at(eri, nmo, p, k0 + kk, i, a);
    }
}

/* src/workspace/screening_workspace.cpp:69-102 with the reference backend's naive
 * gemm (src/linalg/linalg.cpp:93-116): Y = W_c * X, q_j = sum_i x_ij * y_ij. */
void gwo_qforms(i64 n, const double* w_c, const double* x, i64 nvec, double* out_c) {
    const zc* w = (const zc*)w_c;
    zc* out = (zc*)out_c;
    zc* y = (zc*)malloc(sizeof(zc) * (size_t)(n * nvec));
    for (i64 i = 0; i < n; ++i) {
        for (i64 j = 0; j < nvec; ++j) {
            zc sum = 0.0;
            for (i64 k = 0; k < n; ++k) sum += w[i * n + k] * CMPLX(x[k * nvec + j], 0.0);
            y[i * nvec + j] = sum;
        }
    }
    for (i64 j = 0; j < nvec; ++j) {
        zc sum = 0.0;
        for (i64 i = 0; i < n; ++i) sum += x[i * nvec + j] * y[i * nvec + j];
        out[j] = sum;
    }
    free(y);
}

/* Screened quadratic forms q[f, s, k] = x_{p_s k}^T W_c(i w_f) x_{p_s k} for the
 * frequencies in `freq_index` (complex, layout [nf][nstates][nmo]).  The panel loop
 * (panel width `panel`) is the reference's (src/gw/sigma_c_driver.cpp:140-150). */
int gwo_screened_forms(i64 nmo, i64 nocc, const double* mo, const double* eri,
                       i64 nf, const double* omegas, const i64* states, i64 nstates,
                       double eta, i64 panel, double* q_c) {
    const i64 nvir = nmo - nocc, n = nocc * nvir;
    zc* q = (zc*)q_c;
    i64* io = (i64*)malloc(sizeof(i64) * (size_t)n);
    i64* am = (i64*)malloc(sizeof(i64) * (size_t)n);
    double* delta = (double*)malloc(sizeof(double) * (size_t)n);
    double* v = (double*)malloc(sizeof(double) * (size_t)(n * n));
    zc* pi0 = (zc*)malloc(sizeof(zc) * (size_t)n);
    zc* w = (zc*)malloc(sizeof(zc) * (size_t)(n * n));
    double* x = (double*)malloc(sizeof(double) * (size_t)(n * panel));
    zc* vals = (zc*)malloc(sizeof(zc) * (size_t)panel);
    int rc = 0;
    if (panel <= 0) panel = 32;
    gwo_ph_map(nmo, nocc, mo, io, am, delta);
    gwo_vph(nmo, nocc, eri, v);
    for (i64 f = 0; f < nf && rc == 0; ++f) {
        gwo_pi0(0.0, omegas[f], n, delta, eta, (double*)pi0);
        rc = gwo_w_c(n, v, (const double*)pi0, (double*)w);
        if (rc) break;
        for (i64 s = 0; s < nstates; ++s) {
            for (i64 k0 = 0; k0 < nmo; k0 += panel) {
                const i64 width = (panel < nmo - k0) ? panel : nmo - k0;
                gwo_panel(nmo, nocc, eri, states[s], k0, width, x);
                gwo_qforms(n, (const double*)w, x, width, (double*)vals);
                for (i64 kk = 0; kk < width; ++kk) q[(f * nstates + s) * nmo + k0 + kk] = vals[kk];
            }
        }
    }
    free(io); free(am); free(delta); free(v); free(pi0); free(w); free(x); free(vals);
    return rc;
}

/* src/gw/sigma_c_driver.cpp:119-169 accumulation, replayed from cached forms
 * q[f', s, k] (see the header).  sigma_out is nmo x nfreq complex row-major
 * (MatrixComplex), rows of unrequested states left at zero (src/gw/gw.cpp:156). */
void gwo_sigma_from_forms(i64 nmo, const double* mo, double fermi, i64 nfreq,
                          const double* omegas, const double* weights,
                          const i64* states, i64 nstates, i64 panel,
                          const double* q_c, double* sigma_c) {
    const zc* q = (const zc*)q_c;
    zc* sigma = (zc*)sigma_c;
    zc* current = (zc*)malloc(sizeof(zc) * (size_t)nmo);
    if (panel <= 0) panel = 32;
    for (i64 i = 0; i < nmo * nfreq; ++i) sigma[i] = 0.0;
    for (i64 fn = 0; fn < nfreq; ++fn) {
        const zc omega_n = CMPLX(0.0, omegas[fn]);
        for (i64 p = 0; p < nmo; ++p) current[p] = 0.0;
        for (i64 fp = 0; fp < nfreq; ++fp) {
            const zc omega_p = CMPLX(0.0, omegas[fp]);
            for (i64 s = 0; s < nstates; ++s) {
                const i64 p = states[s];
                for (i64 k0 = 0; k0 < nmo; k0 += panel) {
                    const i64 width = (panel < nmo - k0) ? panel : nmo - k0;
                    for (i64 kk = 0; kk < width; ++kk) {
                        const i64 k = k0 + kk;
                        const zc g0_den = omega_n + fermi - mo[k];
                        const zc g0_term = g0_den / (g0_den * g0_den - omega_p * omega_p);
                        current[p] -= g0_term * q[(fp * nstates + s) * nmo + k] * weights[fp];
                    }
                }
            }
        }
        for (i64 s = 0; s < nstates; ++s) {
            const i64 p = states[s];
            sigma[p * nfreq + fn] = current[p] / kPi;
        }
    }
    free(current);
}

/* Full Sigma_c(i w) of the reference (forms + accumulation). */
int gwo_sigma_c(i64 nmo, i64 nocc, const double* mo, const double* eri, double fermi,
                i64 nfreq, const double* omegas, const double* weights,
                const i64* states, i64 nstates, double eta, i64 panel, double* sigma_c) {
    double* q = (double*)malloc(sizeof(zc) * (size_t)(nfreq * nstates * nmo));
    const int rc = gwo_screened_forms(nmo, nocc, mo, eri, nfreq, omegas, states, nstates, eta, panel, q);
    if (rc == 0) gwo_sigma_from_forms(nmo, mo, fermi, nfreq, omegas, weights, states, nstates, panel, q, sigma_c);
    free(q);
    return rc;
}

/* src/gw/frequency_grids.cpp:12-44: Gauss-Legendre nodes/weights on [x1,x2] by Newton. */
static void gauleg(double x1, double x2, i64 n, double* x, double* w) {
    const double eps = 3e-14;
    const i64 m = (n + 1) / 2;
    const double xm = 0.5 * (x2 + x1);
    const double xl = 0.5 * (x2 - x1);
    for (i64 i = 0; i < n; ++i) { x[i] = 0.0; w[i] = 0.0; }
    for (i64 i = 0; i < m; ++i) {
        double z = cos(kPi * ((double)(i + 1) - 0.25) / ((double)n + 0.5));
        double pp = 0.0;
        for (int iter = 0; iter < 100; ++iter) {
            double p1 = 1.0, p2 = 0.0;
            for (i64 j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * (double)j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
            }
            pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
            const double z_old = z;
            z = z_old - p1 / pp;
            if (fabs(z - z_old) <= eps) break;
        }
        x[i] = xm - xl * z;
        x[n - 1 - i] = xm + xl * z;
        w[i] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
        w[n - 1 - i] = w[i];
    }
}

/* src/gw/frequency_grids.cpp:62-93: w = (1+y)/(2(1-y)), weight = w_y/(1-y)^2,
 * stable ascending sort (ties impossible for distinct nodes), omega_0 clamped >= 1e-12. */
int gwo_grid(i64 n, double* omegas, double* weights) {
    if (n <= 0) return -1;
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    double* wy = (double*)malloc(sizeof(double) * (size_t)n);
    double* tv = (double*)malloc(sizeof(double) * (size_t)n);
    double* tw = (double*)malloc(sizeof(double) * (size_t)n);
    i64* order = (i64*)malloc(sizeof(i64) * (size_t)n);
    gauleg(-1.0, 1.0, n, y, wy);
    for (i64 i = 0; i < n; ++i) {
        tv[i] = 0.5 * (1.0 + y[i]) / (1.0 - y[i]);
        tw[i] = wy[i] / ((1.0 - y[i]) * (1.0 - y[i]));
        order[i] = i;
    }
    /* insertion sort on tv (n is small); strict < keeps equal keys in index order */
    for (i64 i = 1; i < n; ++i) {
        const i64 key = order[i];
        i64 j = i - 1;
        while (j >= 0 && tv[key] < tv[order[j]]) { order[j + 1] = order[j]; --j; }
        order[j + 1] = key;
    }
    for (i64 i = 0; i < n; ++i) { omegas[i] = tv[order[i]]; weights[i] = tw[order[i]]; }
    if (omegas[0] < 1e-12) omegas[0] = 1e-12;
    free(y); free(wy); free(tv); free(tw); free(order);
    return 0;
}

/* src/gw/pade.cpp:10-63: sample npar of n points (stride n/(npar-1), last = n-1) and
 * build the Thiele continued-fraction table; coeffs[i] = g(i,i).  Returns npar_actual. */
i64 gwo_pade_coeffs(i64 n, const double* x_c, const double* y_c, i64 npar, double* coeffs_c, double* xs_c) {
    const zc* x = (const zc*)x_c;
    const zc* y = (const zc*)y_c;
    zc* coeffs = (zc*)coeffs_c;
    zc* xs = (zc*)xs_c;
    if (n <= 0 || npar <= 0) return -1;
    const i64 na = npar < n ? npar : n;
    if (na == 1) { coeffs[0] = y[0]; xs[0] = x[0]; return 1; }
    zc* ys = (zc*)malloc(sizeof(zc) * (size_t)na);
    const i64 step = n / (na - 1);
    if (step == 0) {
        for (i64 i = 0; i < na; ++i) { xs[i] = x[i]; ys[i] = y[i]; }
    } else {
        i64 idat = 0;
        for (i64 ip = 0; ip < na - 1; ++ip) { xs[ip] = x[idat]; ys[ip] = y[idat]; idat += step; }
        xs[na - 1] = x[n - 1];
        ys[na - 1] = y[n - 1];
    }
    zc* g = (zc*)malloc(sizeof(zc) * (size_t)(na * na));
    for (i64 i = 0; i < na * na; ++i) g[i] = 0.0;
    for (i64 i = 0; i < na; ++i) g[i * na] = ys[i];
    for (i64 ip = 1; ip < na; ++ip) {
        for (i64 id = ip; id < na; ++id) {
            const zc num = g[(ip - 1) * na + ip - 1] - g[id * na + ip - 1];
            const zc den = (xs[id] - xs[ip - 1]) * g[id * na + ip - 1];
            if (cabs(den) < 1e-20) g[id * na + ip] = num / CMPLX(1e-20, 0.0);
            else g[id * na + ip] = num / den;
        }
    }
    for (i64 i = 0; i < na; ++i) coeffs[i] = g[i * na + i];
    free(ys); free(g);
    return na;
}

/* src/gw/pade.cpp:65-101: backward continued-fraction evaluation at real z. */
void gwo_pade_eval(i64 npar, const double* coeffs_c, double z, const double* xs_c, double* out_c) {
    const zc* coeffs = (const zc*)coeffs_c;
    const zc* xs = (const zc*)xs_c;
    zc* out = (zc*)out_c;
    if (npar == 0) { *out = 0.0; return; }
    if (npar == 1) { *out = coeffs[0]; return; }
    const zc zt = CMPLX(z, 0.0);
    zc val = CMPLX(1.0, 0.0);
    for (i64 kr = npar - 1; kr > 0; --kr) {
        const i64 k = kr - 1;
        const zc num = coeffs[k + 1] * (zt - xs[k]);
        if (cabs(val) < 1e-20) val = CMPLX(1e-20, 0.0);
        val = CMPLX(1.0, 0.0) + num / val;
    }
    if (cabs(val) < 1e-20) { *out = coeffs[0] / CMPLX(1e-20, 0.0); return; }
    *out = coeffs[0] / val;
}

/* src/gw/qp_solver.cpp:10-47: per requested state, fixed-point
 * E <- e_p + Re Sigma_c(E - E_F) + Sigma_x[p,p] - vxc[p,p], <= 200 iterations, tol 1e-6.
 * sigma is nmo x nfreq complex row-major; qp_out[nmo] is NaN for unrequested states. */
void gwo_qp(i64 nmo, const double* mo, double fermi, const double* sigma_x_diag, const double* vxc_diag,
            i64 nfreq, const double* omegas, const double* sigma_c, const i64* states, i64 nstates,
            i64 npar, double* qp_out) {
    const zc* sigma = (const zc*)sigma_c;
    zc* x = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    zc* y = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    zc* coeffs = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    zc* xs = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    for (i64 p = 0; p < nmo; ++p) qp_out[p] = NAN;
    for (i64 f = 0; f < nfreq; ++f) x[f] = CMPLX(0.0, omegas[f]);
    for (i64 s = 0; s < nstates; ++s) {
        const i64 p = states[s];
        double cur = mo[p];
        for (i64 f = 0; f < nfreq; ++f) y[f] = sigma[p * nfreq + f];
        const i64 na = gwo_pade_coeffs(nfreq, (const double*)x, (const double*)y, npar, (double*)coeffs, (double*)xs);
        for (int it = 0; it < 200; ++it) {
            const double target = cur - fermi;
            zc sc;
            gwo_pade_eval(na, (const double*)coeffs, target, (const double*)xs, (double*)&sc);
            const double nq = mo[p] + creal(sc) + sigma_x_diag[p] - vxc_diag[p];
            if (fabs(nq - cur) < 1e-6) { cur = nq; break; }
            cur = nq;
        }
        qp_out[p] = cur;
    }
    free(x); free(y); free(coeffs); free(xs);
}

/* src/io.cpp:94-108 (E_c.out): Pade of one state's Sigma_c sampled at
 * e = x_start + i*interval - E_F, i < npts; out is npts x 3 (e[eV], Re, Im). */
void gwo_ec_sweep(i64 nfreq, const double* omegas, const double* sigma_row_c, i64 npar, i64 npts,
                  double fermi, double x_start, double interval, double* out) {
    zc* x = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    zc* coeffs = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    zc* xs = (zc*)malloc(sizeof(zc) * (size_t)nfreq);
    for (i64 f = 0; f < nfreq; ++f) x[f] = CMPLX(0.0, omegas[f]);
    const i64 na = gwo_pade_coeffs(nfreq, (const double*)x, sigma_row_c, npar, (double*)coeffs, (double*)xs);
    for (i64 i = 0; i < npts; ++i) {
        const double e = x_start + (double)i * interval - fermi;
        zc v;
        gwo_pade_eval(na, (const double*)coeffs, e, (const double*)xs, (double*)&v);
        out[3 * i + 0] = (e + fermi) * 27.211386245988;
        out[3 * i + 1] = creal(v);
        out[3 * i + 2] = cimag(v);
    }
    free(x); free(coeffs); free(xs);
}
