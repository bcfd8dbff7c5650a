"""Write b200-enabled copies of the reference's backend_factory.cpp and sigma_c_driver.cpp into
OUT_DIR (a temporary build directory; nothing is written into the repository or the reference).

    python oracle/b200_integration/patch.py REF_ROOT OUT_DIR

The insertions are the maintainer-side binding: the `b200` case of make_local_linalg_backend
and, in compute_sigma_c_with_backend, a branch that loads the system with the state list and
fills Sigma_c(iw) with one gwb200_sigma_c call.  They are placed at anchors found in the reference
files, and the script fails if an anchor is missing.
"""
import sys
from pathlib import Path

FACTORY_INCLUDE = '#include "linalg/linalg_b200.hpp"\n'
FACTORY_CASE = '''#ifdef GW_HAS_B200_BACKEND
    if (cli.linalg_backend == "b200") {
        return linalg::make_b200_backend();
    }
#endif
'''
DRIVER_INCLUDE = '#include "gwb200.h"\n#include <memory>\n'
DRIVER_BRANCH = '''#ifdef GW_HAS_B200_BACKEND
    if (linalg_backend.name() == "b200") {
        auto chk = [](int rc) { if (rc != GWB200_OK) throw std::runtime_error(gwb200_last_error()); };
        gwb200_handle* h = nullptr;
        chk(gwb200_create(static_cast<int>(settings.execution.mpi_local_rank / settings.execution.tasks_per_gpu), &h));
        std::unique_ptr<gwb200_handle, int (*)(gwb200_handle*)> guard(h, gwb200_destroy);
        const auto& eri = integrals.eri_tensor().data();
        const auto& vxc = integrals.vxc_matrix().data();
        std::vector<int64_t> st(states.begin(), states.end());
        chk(gwb200_load_system_states(h, static_cast<int64_t>(orbitals.nmo()), static_cast<int64_t>(orbitals.nocc()),
                                      orbitals.energies().data(), eri.data(), vxc.data(), orbitals.fermi_energy(),
                                      st.data(), static_cast<int64_t>(st.size())));
        std::vector<double> omega(omega_im.size());
        for (std::size_t f = 0; f < omega.size(); ++f) omega[f] = omega_im[f].imag();
        gwb200_stats stats{};
        chk(gwb200_sigma_c(h, omega.data(), weights.data(), static_cast<int64_t>(omega.size()), st.data(),
                           static_cast<int64_t>(st.size()), settings.eta, GWB200_FP64,
                           reinterpret_cast<double*>(sigma_c_im_points.data().data()), &stats));
        timings.invert_epsilon_seconds += stats.device_ms_screening * 1e-3;
        timings.sigma_c_seconds += stats.device_ms_contract * 1e-3;
        if (root_rank(settings)) {
            std::cout << "Using the b200 device backend: " << stats.nph << " particle-hole pairs, " << stats.ncols
                      << " right-hand sides, " << stats.frequency_chunks << " frequency chunk(s).\\n";
        }
        return;
    }
#endif
'''


def insert_after(text: str, anchor: str, block: str) -> str:
    i = text.index(anchor) + len(anchor)
    return text[:i] + block + text[i:]


def insert_before(text: str, anchor: str, block: str) -> str:
    i = text.index(anchor)
    return text[:i] + block + text[i:]


def main() -> None:
    ref, out = Path(sys.argv[1]), Path(sys.argv[2])
    out.mkdir(parents=True, exist_ok=True)
    f = (ref / "src/linalg/backend_factory.cpp").read_text()
    f = insert_after(f, "#include <stdexcept>\n", FACTORY_INCLUDE)
    f = insert_before(f, '    if (cli.linalg_backend == "cublas") {', FACTORY_CASE)
    (out / "backend_factory_b200.cpp").write_text(f)
    d = (ref / "src/gw/sigma_c_driver.cpp").read_text()
    d = insert_after(d, '#include "workspace/screening_workspace.hpp"\n', DRIVER_INCLUDE)
    anchor = '    if (std::string_view{linalg_backend.name()}.find("cublas")'
    i = d.index(anchor)
    j = d.rindex("#ifdef GW_HAS_CUDA_BACKEND", 0, i)
    d = d[:j] + DRIVER_BRANCH + "\n" + d[j:]
    (out / "sigma_c_driver_b200.cpp").write_text(d)


if __name__ == "__main__":
    main()
