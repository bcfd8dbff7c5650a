// noalloc.cu -- gwb200_screened_forms_noalloc: the screened quadratic forms with no device
// allocation at all.
//
// Who needs it: callers that cannot call cudaMalloc.  A host framework whose caching allocator
// already owns (nearly) all device memory, where an outside cudaMalloc fails or fragments its
// pool; a serving loop that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
// imply; a process admitted under a fixed device-memory budget that must know its whole
// footprint before it starts.  Such callers pass their own device buffers for the inputs and
// outputs; every intermediate lives in one fixed, file-scope device array.
//
// The scratch is kStaticScratchBytes (4 MiB) of global memory that every GPU which loads
// libgwb200 holds until the process exits.  One frequency of the tall matrix
// [eps ; (D^1/2 X)^T] must fit in it (see the header for the size rule); frequencies are
// processed in chunks that fit.  All calls share the array: calls that overlap on the GPU
// (two streams, two host threads) race on it and must be serialised by the caller.
#include "internal.cuh"

namespace gwb200 {
namespace {

constexpr size_t kStaticScratchBytes = size_t{4} << 20;
constexpr size_t kStaticScratchDoubles = kStaticScratchBytes / sizeof(double);
constexpr size_t kHeaderDoubles = 32;  // 256 bytes: the failing-pivot flag

__device__ __align__(256) double g_noalloc_scratch[kStaticScratchDoubles];

// Device address of g_noalloc_scratch on the current device.  In host code the symbol is only a
// host-side stand-in: the address must come from cudaGetSymbolAddress with the device current.  It
// is looked up on every call (cheap next to a solve) rather than cached, so it stays right after the
// primary context of the device has been reset and the module loaded again.
double* scratch_for_current_device() {
    void* p = nullptr;
    GWB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    return static_cast<double*>(p);
}

void require_device_pointer(const void* p, const char* name) {
    if (!p) fail(GWB200_BAD_ARGUMENT, std::string("null ") + name);
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(GWB200_BAD_ARGUMENT, std::string(name) + " is not a CUDA pointer");
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        fail(GWB200_BAD_ARGUMENT, std::string(name) + " must be device memory");
    int dev = 0;
    GWB_CUDA(cudaGetDevice(&dev));
    if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
        fail(GWB200_BAD_ARGUMENT, std::string(name) + " is memory of device " + std::to_string(attr.device) +
                                      ", not of the current device " + std::to_string(dev));
}

} // namespace

size_t noalloc_scratch_bytes() { return kStaticScratchBytes; }

void screened_forms_noalloc(int64_t n, int64_t m, const double* d_v, const double* d_xt, const double* d_delta,
                            const double* d_omega, int64_t nfreq, double* d_q_out, cudaStream_t s) {
    if (n <= 0 || m <= 0 || nfreq <= 0) fail(GWB200_BAD_SHAPE, "n, m and nfreq must be positive");
    const TallGeometry g = make_geometry(n, m);
    const size_t per_freq = (size_t)g.stride + (size_t)g.n_pad + (size_t)kNb * kNb + (size_t)g.m_pad;
    if (per_freq > kStaticScratchDoubles - kHeaderDoubles)
        fail(GWB200_BAD_SHAPE, "system too large for the 4 MiB static scratch: one frequency needs " +
                                   std::to_string(per_freq * sizeof(double)) + " bytes ((n64+m64)*n64 + n64 + 4096 + "
                                   "m64 doubles with n64, m64 = n, m rounded up to 64)");
    require_device_pointer(d_v, "V_ph");
    require_device_pointer(d_xt, "panel");
    require_device_pointer(d_delta, "delta");
    require_device_pointer(d_omega, "omega");
    require_device_pointer(d_q_out, "output");

    double* base = scratch_for_current_device();
    auto* err = reinterpret_cast<unsigned long long*>(base);
    const int64_t fc = (int64_t)std::min<size_t>((size_t)nfreq, (kStaticScratchDoubles - kHeaderDoubles) / per_freq);
    double* a = base + kHeaderDoubles;
    double* dvec = a + (size_t)fc * g.stride;
    double* linv = dvec + (size_t)fc * g.n_pad;
    double* qacc = linv + (size_t)fc * kNb * kNb;

    // The scratch keeps the previous call's contents: reset the pivot flag; qacc is cleared per chunk.
    GWB_CUDA(cudaMemsetAsync(err, 0xFF, sizeof(unsigned long long), s));
    for (int64_t f0 = 0; f0 < nfreq; f0 += fc) {
        const int64_t nf = std::min(fc, nfreq - f0);
        launch_scale_vectors(d_delta, g.n, g.n_pad, d_omega + f0, nf, dvec, s);
        launch_build_tall(g, d_v, d_xt, dvec, nf, a, s);
        GWB_CUDA(cudaMemsetAsync(qacc, 0, sizeof(double) * (size_t)nf * g.m_pad, s));
        launch_factor_chunk(g, nf, a, linv, qacc, err, s, nullptr, -1);
        launch_negate_copy(qacc, nf, m, g.m_pad, d_q_out + (size_t)f0 * m, m, s);
    }
    unsigned long long piv = 0;
    GWB_CUDA(cudaMemcpyAsync(&piv, err, sizeof(piv), cudaMemcpyDeviceToHost, s));
    GWB_CUDA(cudaStreamSynchronize(s));
    if (piv != ~0ull)
        fail(GWB200_NOT_SPD, "eps(iw) is not positive definite: Cholesky pivot " + std::to_string(piv) + " <= 0");
}

} // namespace gwb200
