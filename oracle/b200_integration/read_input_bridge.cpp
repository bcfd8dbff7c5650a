// read_input_bridge.cpp -- gw::read_gw_input_hdf5 (declared by the reference's include/hdf5_input.hpp)
// implemented with libgwb200's minimal HDF5 reader, so the reference's own main() links without
// libhdf5 (absent in this image).  Same validation messages path: failures throw std::runtime_error.
#include "gwb200.h"
#include "hdf5_input.hpp"

#include <stdexcept>
#include <string>

namespace gw {

GwInput read_gw_input_hdf5(const std::string& path) {
    int64_t nmo = 0, nocc = 0;
    double fermi = 0.0;
    if (gwb200_read_input_h5(path.c_str(), &nmo, &nocc, &fermi, nullptr, nullptr, nullptr) != GWB200_OK)
        throw std::runtime_error(gwb200_last_error());
    const auto n = static_cast<std::size_t>(nmo);
    GwInput in;
    in.mo_energy.assign(n, 0.0);
    std::vector<double> eri(n * n * n * n), vxc(n * n);
    if (gwb200_read_input_h5(path.c_str(), &nmo, &nocc, &fermi, in.mo_energy.data(), eri.data(), vxc.data()) !=
        GWB200_OK)
        throw std::runtime_error(gwb200_last_error());
    in.eri_mo = Tensor4Real(n, n, n, n, std::move(eri));
    in.vxc_mo = MatrixReal(n, n, std::move(vxc));
    in.nocc = static_cast<std::size_t>(nocc);
    in.fermi_energy = fermi;
    return in;
}

} // namespace gw
