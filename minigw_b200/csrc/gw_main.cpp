// gw_main.cpp -- `gw` command-line driver for the b200 backend.
//
// Drop-in for the reference executable (src/main.cpp:19-141, src/cli.cpp:33-104): same flags and
// defaults (include/cli.hpp:9-23), same input (gw_input.h5 in --input-dir) and the same output
// files in --output-dir: gw.out (stdout tee, src/io.cpp:13-57), E_c_before_Pade.out
// (src/io.cpp:86-92), E_c.out (19836 Pade samples, src/io.cpp:94-108) and the final energy table
// (src/io.cpp:110-126).  Only `--linalg-backend b200` is provided here; the numerical work is done
// by libgwb200 (include/gwb200.h) on one GPU.
#include <cerrno>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <streambuf>
#include <string>
#include <vector>

#include "gwb200.h"

namespace {

constexpr double kHartreeToEv = 27.211386245988;

struct Cli {
    std::string input_dir{"."};
    std::string output_dir{"./gw_output"};
    std::size_t freq_points{200};
    std::size_t pade_params{16};
    std::optional<std::size_t> selected_state_1based{5};
    std::vector<std::size_t> states_1based;  // extension: --states a,b,c
    double eta{0.0};
    std::string linalg_backend{"b200"};
    std::string frequency_parallel{"auto"};
    std::string kernel_parallel{"auto"};
    bool print_memory_footprint{true};
    std::size_t contraction_panel_size{32};
    std::size_t scalapack_ranks_per_group{4};
    std::size_t tasks_per_gpu{4};
    std::string precision{"fp64"};
};

void print_usage(const char* exe) {
    std::cerr << "Usage: " << exe << " [options]\n"
              << "Options:\n"
              << "  --input-dir PATH             Directory containing gw_input.h5\n"
              << "  --freq-points N              Number of imaginary-frequency points [default: 200]\n"
              << "  --pade-params N              Number of Pade parameters [default: 16]\n"
              << "  --state N                    1-based orbital index to calculate [default: 5]\n"
              << "  --states A,B,...             1-based orbital indices to calculate (b200 extension)\n"
              << "  --all-states                 Calculate all diagonal states\n"
              << "  --eta VALUE                  Infinitesimal broadening [default: 0.0; nonzero: complex symmetric path, fp64 only]\n"
              << "  --linalg-backend NAME        b200 [default: b200]\n"
              << "  --precision MODE             fp64, mixed or mixed-refined [default: fp64]\n"
              << "  --frequency-parallel MODE    auto or serial (the device batches all frequencies)\n"
              << "  --kernel-parallel MODE       auto, serial, or openmp (host loops; no effect on b200)\n"
              << "  --contraction-panel-size N   Accepted for compatibility; b200 solves all (p,k) columns at once\n"
              << "  --scalapack-ranks-per-group N  Accepted for compatibility (no ScaLAPACK in this build)\n"
              << "  --tasks-per-gpu N            Local-rank-to-GPU mapping block size [default: 4]\n"
              << "  --print-memory-footprint     Print the device memory estimate before running GW\n"
              << "  --output-dir PATH            Directory containing E_c_before_Pade.out, E_c.out, and gw.out\n"
              << "  --help                       Show this message\n";
}

std::size_t to_size(const std::string& s) { return static_cast<std::size_t>(std::stoull(s)); }

Cli parse_cli(int argc, char** argv) {
    Cli cli;
    for (int i = 1; i < argc; ++i) {
        const std::string arg = argv[i];
        auto require_value = [&](const std::string& name) -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("Missing value for " + name);
            return argv[++i];
        };
        if (arg == "--input-dir") cli.input_dir = require_value(arg);
        else if (arg == "--freq-points") cli.freq_points = to_size(require_value(arg));
        else if (arg == "--pade-params") cli.pade_params = to_size(require_value(arg));
        else if (arg == "--state") { cli.selected_state_1based = to_size(require_value(arg)); cli.states_1based.clear(); }
        else if (arg == "--states") {
            std::stringstream ss(require_value(arg));
            std::string tok;
            cli.states_1based.clear();
            while (std::getline(ss, tok, ',')) cli.states_1based.push_back(to_size(tok));
            if (cli.states_1based.empty()) throw std::runtime_error("--states needs at least one index");
        }
        else if (arg == "--all-states") { cli.selected_state_1based.reset(); cli.states_1based.clear(); }
        else if (arg == "--eta") cli.eta = std::stod(require_value(arg));
        else if (arg == "--linalg-backend") cli.linalg_backend = require_value(arg);
        else if (arg == "--precision") cli.precision = require_value(arg);
        else if (arg == "--frequency-parallel") cli.frequency_parallel = require_value(arg);
        else if (arg == "--kernel-parallel") cli.kernel_parallel = require_value(arg);
        else if (arg == "--contraction-panel-size") cli.contraction_panel_size = to_size(require_value(arg));
        else if (arg == "--scalapack-ranks-per-group") cli.scalapack_ranks_per_group = to_size(require_value(arg));
        else if (arg == "--tasks-per-gpu") cli.tasks_per_gpu = to_size(require_value(arg));
        else if (arg == "--print-memory-footprint") cli.print_memory_footprint = true;
        else if (arg == "--output-dir") cli.output_dir = require_value(arg);
        else if (arg == "--help" || arg == "-h") { print_usage(argv[0]); std::exit(EXIT_SUCCESS); }
        else throw std::runtime_error("Unknown option: " + arg);
    }
    std::filesystem::create_directories(cli.output_dir);
    if (cli.freq_points == 0) throw std::runtime_error("--freq-points must be positive");
    if (cli.pade_params == 0) throw std::runtime_error("--pade-params must be positive");
    if (cli.contraction_panel_size == 0) throw std::runtime_error("--contraction-panel-size must be positive");
    if (cli.scalapack_ranks_per_group == 0) throw std::runtime_error("--scalapack-ranks-per-group must be positive");
    if (cli.tasks_per_gpu == 0) throw std::runtime_error("--tasks-per-gpu must be positive");
    if (cli.frequency_parallel != "auto" && cli.frequency_parallel != "serial" && cli.frequency_parallel != "mpi" &&
        cli.frequency_parallel != "openmp")
        throw std::runtime_error("--frequency-parallel must be one of: auto, serial, mpi, openmp");
    if (cli.kernel_parallel != "auto" && cli.kernel_parallel != "serial" && cli.kernel_parallel != "openmp")
        throw std::runtime_error("--kernel-parallel must be one of: auto, serial, openmp");
    if (cli.linalg_backend != "b200")
        throw std::runtime_error("Unknown --linalg-backend value: " + cli.linalg_backend +
                                 ". This executable provides: b200 (use the reference build for reference, "
                                 "blas-lapack, scalapack, cosma, cublas).");
    if (cli.frequency_parallel == "openmp")
        throw std::runtime_error("OpenMP frequency parallelism is only supported for replicated local host backends. "
                                 "The b200 device backend batches all frequencies on the GPU.");
    if (cli.frequency_parallel == "mpi")
        throw std::runtime_error("--frequency-parallel mpi requires a build configured with MPI; the b200 driver runs "
                                 "one GPU per process");
    if (cli.precision != "fp64" && cli.precision != "mixed" && cli.precision != "mixed-refined")
        throw std::runtime_error("--precision must be fp64, mixed or mixed-refined");
    return cli;
}

std::string join_path(const std::string& dir, const std::string& file) {
    return (std::filesystem::path(dir) / file).string();
}

class TeeBuffer : public std::streambuf {
public:
    TeeBuffer(std::streambuf* a, std::streambuf* b) : a_(a), b_(b) {}

private:
    int overflow(int ch) override {
        if (ch == traits_type::eof()) return traits_type::not_eof(ch);
        const int r1 = a_->sputc(static_cast<char>(ch));
        const int r2 = b_->sputc(static_cast<char>(ch));
        return (r1 == traits_type::eof() || r2 == traits_type::eof()) ? traits_type::eof() : ch;
    }
    int sync() override { return (a_->pubsync() == 0 && b_->pubsync() == 0) ? 0 : -1; }
    std::streambuf* a_;
    std::streambuf* b_;
};

void check(int rc, const char* what) {
    if (rc != GWB200_OK) throw std::runtime_error(std::string(what) + ": " + gwb200_last_error());
}

int local_rank_from_env() {
    for (const char* name : {"OMPI_COMM_WORLD_LOCAL_RANK", "MPI_LOCALRANKID", "SLURM_LOCALID", "LOCAL_RANK"}) {
        if (const char* v = std::getenv(name)) return std::atoi(v);
    }
    return 0;
}

double seconds_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

} // namespace

int main(int argc, char** argv) {
    gwb200_handle* h = nullptr;
    try {
        const Cli cli = parse_cli(argc, argv);
        std::ofstream log_file(join_path(cli.output_dir, "gw.out"));
        if (!log_file) throw std::runtime_error("Could not open log file: " + join_path(cli.output_dir, "gw.out"));
        TeeBuffer tee(std::cout.rdbuf(), log_file.rdbuf());
        std::streambuf* old = std::cout.rdbuf(&tee);
        struct Restore {
            std::streambuf* o;
            ~Restore() { std::cout.rdbuf(o); }
        } restore{old};

        std::cout << "\n--- Begin of C++20 G0W0 Calculation ---\n";
        std::cout << "Loading data from: " << cli.input_dir << '\n';
        const auto t_read = std::chrono::steady_clock::now();
        const std::string path = join_path(cli.input_dir, "gw_input.h5");
        int64_t nmo = 0, nocc = 0;
        double fermi = 0.0;
        // Sizes first; the data is read once the state list is known, and only the slices the path
        // uses (gwb200_read_input_h5_slices), never the nmo^4 ERI tensor.
        check(gwb200_read_input_h5_slices(path.c_str(), nullptr, 0, &nmo, &nocc, &fermi, nullptr, nullptr, nullptr,
                                          nullptr, nullptr),
              "read_gw_input_hdf5");
        double read_seconds = seconds_since(t_read);
        const int64_t nvirt = nmo - nocc, n_ph = nocc * nvirt;
        std::cout << "  - Vxc MO basis shape: (" << nmo << ", " << nmo << ")\n";
        std::cout << "  - Fermi energy (eV): " << fermi * kHartreeToEv << '\n';
        std::cout << "  - Number of occupied orbitals: " << nocc << '\n';
        std::cout << "  - Number of virtual orbitals: " << nvirt << '\n';
        std::cout << "  - Number of MOs: " << nmo << '\n';
        std::cout << "  - Number of particle-hole states: " << n_ph << '\n';
        std::cout << "  - ERI MO shape: (" << nmo << ", " << nmo << ", " << nmo << ", " << nmo << ")\n";

        std::vector<int64_t> states;
        if (!cli.states_1based.empty()) {
            for (auto s : cli.states_1based) {
                if (s == 0) throw std::runtime_error("--states must be 1-based and positive");
                states.push_back(static_cast<int64_t>(s - 1));
            }
        } else if (cli.selected_state_1based.has_value()) {
            if (*cli.selected_state_1based == 0) throw std::runtime_error("--state must be 1-based and positive");
            states.push_back(static_cast<int64_t>(*cli.selected_state_1based - 1));
        } else {
            for (int64_t p = 0; p < nmo; ++p) states.push_back(p);
        }
        for (auto s : states)
            if (s >= nmo) throw std::runtime_error("Selected state is out of range");
        const auto t_slices = std::chrono::steady_clock::now();
        const size_t ns = states.size();
        std::vector<double> mo(static_cast<size_t>(nmo)), vxc_diag(static_cast<size_t>(nmo));
        std::vector<double> vph(static_cast<size_t>(n_ph) * n_ph), panel(ns * static_cast<size_t>(nmo) * n_ph);
        std::vector<double> xdiag(static_cast<size_t>(nmo) * nocc);
        check(gwb200_read_input_h5_slices(path.c_str(), states.data(), static_cast<int64_t>(ns), &nmo, &nocc, &fermi,
                                          mo.data(), vph.data(), panel.data(), xdiag.data(), vxc_diag.data()),
              "read_gw_input_hdf5");
        read_seconds += seconds_since(t_slices);

        int ndev = 1;
        const int device = (local_rank_from_env() / static_cast<int>(cli.tasks_per_gpu)) % std::max(1, ndev);
        check(gwb200_create(device, &h), "gwb200_create");
        std::cout << "Linear algebra backend: b200 (" << gwb200_version() << ")\n";
        std::cout << "Frequency parallel mode: device-batched (all frequencies per launch)\n";
        std::cout << "Precision: " << cli.precision << '\n';
        if (cli.print_memory_footprint) {
            const double res_gib = (static_cast<double>(n_ph) * n_ph + static_cast<double>(n_ph) * states.size() * nmo) *
                                   8.0 / (1024.0 * 1024.0 * 1024.0);
            std::cout << "Device memory estimate: V_ph + panel " << res_gib << " GiB resident, eps(iw)+panel "
                      << res_gib << " GiB per frequency (frequencies are chunked to fit)\n";
        }
        const auto t_total = std::chrono::steady_clock::now();
        auto t = std::chrono::steady_clock::now();
        check(gwb200_load_system_slices(h, nmo, nocc, mo.data(), vph.data(), panel.data(), xdiag.data(),
                                        vxc_diag.data(), fermi, states.data(), static_cast<int64_t>(ns)),
              "gwb200_load_system_slices");
        const double setup_seconds = seconds_since(t);
        std::vector<double> omega(cli.freq_points), weight(cli.freq_points);
        check(gwb200_grid(static_cast<int64_t>(cli.freq_points), omega.data(), weight.data()), "generate grid");
        std::cout << "Total number of Pade parameters: " << cli.pade_params << '\n';
        std::cout << "Total number of transformed Gauss-Legendre frequency points: " << cli.freq_points << '\n';
        std::cout << "\n--- Starting Sigma_c(iw) calculation... ---\n";
        std::vector<std::complex<double>> sigma(static_cast<size_t>(nmo) * cli.freq_points);
        gwb200_stats stats{};
        t = std::chrono::steady_clock::now();
        check(gwb200_sigma_c(h, omega.data(), weight.data(), static_cast<int64_t>(cli.freq_points), states.data(),
                             static_cast<int64_t>(states.size()), cli.eta,
                             cli.precision == "mixed"           ? GWB200_MIXED
                             : cli.precision == "mixed-refined" ? GWB200_MIXED_REFINED
                                                                : GWB200_FP64,
                             reinterpret_cast<double*>(sigma.data()), &stats),
              "gwb200_sigma_c");
        const double sigma_seconds = seconds_since(t);
        std::cout << "Sigma_c(iw) calculation complete.\n";
        std::vector<double> sigx(static_cast<size_t>(nmo)), qp(static_cast<size_t>(nmo));
        check(gwb200_sigma_x_diag(h, sigx.data()), "gwb200_sigma_x_diag");
        t = std::chrono::steady_clock::now();
        check(gwb200_qp(h, omega.data(), static_cast<int64_t>(cli.freq_points), reinterpret_cast<double*>(sigma.data()),
                        static_cast<int64_t>(cli.pade_params), states.data(), static_cast<int64_t>(states.size()),
                        qp.data()),
              "gwb200_qp");
        double pade_seconds = seconds_since(t);
        const double total_seconds = seconds_since(t_total);

        const int64_t out_state = states.size() == 1 || cli.selected_state_1based.has_value() ? states.front() : 0;
        {
            std::ofstream out(join_path(cli.output_dir, "E_c_before_Pade.out"));
            for (std::size_t f = 0; f < cli.freq_points; ++f) {
                const auto z = sigma[static_cast<size_t>(out_state) * cli.freq_points + f];
                out << '(' << std::setprecision(17) << z.real() << ',' << z.imag() << ")\n";
            }
        }
        t = std::chrono::steady_clock::now();
        {
            const int64_t npts = 19836;
            std::vector<double> sweep(static_cast<size_t>(npts) * 3);
            check(gwb200_pade_sweep(h, omega.data(), static_cast<int64_t>(cli.freq_points),
                                    reinterpret_cast<double*>(sigma.data() + static_cast<size_t>(out_state) * cli.freq_points),
                                    static_cast<int64_t>(cli.pade_params), npts, fermi, -6.5, 0.00065, sweep.data()),
                  "gwb200_pade_sweep");
            std::ofstream out(join_path(cli.output_dir, "E_c.out"));
            for (int64_t i = 0; i < npts; ++i)
                out << std::setprecision(17) << sweep[3 * i] << ' ' << sweep[3 * i + 1] << ' ' << sweep[3 * i + 2] << '\n';
        }
        pade_seconds += seconds_since(t);

        const auto old_flags = std::cout.flags();
        const auto old_prec = std::cout.precision();
        std::cout << "\n--- Profiling Baseline ---\n" << std::fixed << std::setprecision(2);
        auto row = [](const char* name, double v) {
            std::cout << std::left << std::setw(22) << name << std::right << std::setw(8) << v << " s\n";
        };
        row("read input:", read_seconds);
        row("total GW wall:", total_seconds);
        row("screening setup:", setup_seconds);
        row("build W_c accum:", stats.device_ms_screening * 1e-3);
        row("sigma_c accum:", stats.device_ms_contract * 1e-3);
        row("sigma_c wall:", sigma_seconds);
        row("pade/output pade:", pade_seconds);
        std::cout.flags(old_flags);
        std::cout.precision(old_prec);

        std::cout << "\n--- G0W0 Calculation Summary ---\n";
        std::cout << std::left << std::setw(10) << "Orbital" << std::setw(15) << "KS Energy" << std::setw(15)
                  << "Sigma_x" << std::setw(15) << "Sigma_c" << std::setw(15) << "Vxc" << std::setw(15) << "QP Energy"
                  << '\n';
        std::cout << std::left << std::setw(10) << "-------" << std::setw(15) << "---------" << std::setw(15)
                  << "-------" << std::setw(15) << "-------" << std::setw(15) << "-------" << std::setw(15)
                  << "---------" << '\n';
        for (const auto idx : states) {
            const size_t i = static_cast<size_t>(idx);
            const double vxx = vxc_diag[i];
            const double sigma_c_qp = qp[i] + vxx - mo[i] - sigx[i];
            std::cout << std::left << std::setw(10) << (idx + 1) << std::setw(15) << mo[i] * kHartreeToEv
                      << std::setw(15) << sigx[i] * kHartreeToEv << std::setw(15) << sigma_c_qp * kHartreeToEv
                      << std::setw(15) << vxx * kHartreeToEv << std::setw(15) << qp[i] * kHartreeToEv << '\n';
        }
        std::cout << "\n--- End of C++20 G0W0 Calculation ---\n";
        gwb200_destroy(h);
        h = nullptr;
    } catch (const std::exception& ex) {
        std::cerr << "Error: " << ex.what() << '\n';
        if (h) gwb200_destroy(h);
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}
