// linalg_b200.hpp -- the `b200` backend object for the reference's backend factory
// (include/linalg/linalg.hpp:43-63).  A device backend: the patched driver routes it to
// gwb200_sigma_c (include/gwb200.h); the host-style primitives are not provided, as the reference's
// device screening workspace bypasses them too.
#pragma once

#include "gwb200.h"
#include "linalg/linalg.hpp"

#include <memory>
#include <stdexcept>

namespace gw::linalg {

class B200Backend final : public Backend {
public:
    [[nodiscard]] std::string_view name() const noexcept override { return "b200"; }
    [[nodiscard]] BackendCapabilities capabilities() const noexcept override {
        return BackendCapabilities{.family = BackendFamily::Device,
                                   .thread_safe = false,
                                   .uses_internal_threads = false,
                                   .distributed_mpi = false,
                                   .uses_device_memory = true};
    }
    [[nodiscard]] MatrixComplex inverse(MatrixComplex) const override { throw unsupported(); }
    [[nodiscard]] MatrixComplex gemm(const MatrixComplex&, const MatrixComplex&, MatrixTranspose,
                                     MatrixTranspose) const override {
        throw unsupported();
    }
    [[nodiscard]] std::vector<Complex> gemv(const MatrixComplex&, const std::vector<double>&,
                                            MatrixTranspose) const override {
        throw unsupported();
    }
    [[nodiscard]] Complex quadratic_form(const std::vector<double>&, const MatrixComplex&) const override {
        throw unsupported();
    }

private:
    static std::runtime_error unsupported() {
        return std::runtime_error("b200: host-style primitives are not provided; the driver calls gwb200_sigma_c");
    }
};

inline std::shared_ptr<const Backend> make_b200_backend() {
    static const std::shared_ptr<const Backend> backend = std::make_shared<B200Backend>();
    return backend;
}

} // namespace gw::linalg
