// qsb_ham_nonlocal_apply_static: the nonlocal apply (Hpsi += V_NL psi) with its
// scratch in a fixed, library-owned device array instead of the context's
// workspace, so the call itself allocates nothing.
//
// Who needs it: callers that must not allocate device memory once they are
// running — codes that reserve all device memory up front for their own
// arena (the way QUMASUN sub-allocates everything from one work arena) and
// callers that cannot afford the device-wide synchronization that
// cudaMalloc / cudaFree bring into a tight loop.  The regular entry point grows
// the context's workspace with cudaMalloc the first time a larger bundle is
// applied; this one never does.
//
// The scratch (per-chunk partial sums of <beta|psi> and the per-atom
// coefficients dV E_w <beta|psi>) is QSB_NL_STATIC_SCRATCH_BYTES of device
// memory, held by every GPU that loads the library until the process exits.
#include "qsb_internal.h"

#include <mutex>
#include <string>

namespace {

constexpr size_t kStaticScratchDoubles = QSB_NL_STATIC_SCRATCH_BYTES / sizeof(double);

// One copy per device.  Host code cannot use this name as a device address:
// its address is looked up with cudaGetSymbolAddress on each device.
static __device__ __align__(256) double g_nl_static_scratch[kStaticScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch on device `dev` (the current one), looked up
// once per device.
qsb_status static_scratch(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices) return qsb::fail(QSB_ERR_INVALID, "nonlocal_apply_static: device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_nl_static_scratch);
        if (e != cudaSuccess) return qsb::cuda_fail(e, "nonlocal_apply_static: cudaGetSymbolAddress");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return QSB_OK;
}

}  // namespace

extern "C" qsb_status qsb_ham_nonlocal_apply_static(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb,
                                                    const void* psi_dev, void* hpsi_dev, double gx, double gy,
                                                    double gz, void* stream) {
    QSB_TRY(qsb::check_apply(h, dtype, nb, psi_dev, hpsi_dev));
    // the projector tables live on the device the context was created on; the
    // scratch must be that device's copy of the array
    int dev = -1;
    QSB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != h->device)
        return qsb::fail(QSB_ERR_STATE, "nonlocal_apply_static: current device " + std::to_string(dev) +
                                            " is not the context's device " + std::to_string(h->device));
    if (nb == 0 || h->nl.n_points == 0) return QSB_OK;
    if (!is_complex) gx = gy = gz = 0.0;
    const int ncol = is_complex ? 2 * nb : nb;
    const size_t need = qsb::nl_workspace_bytes(h->nl, ncol);
    if (need > QSB_NL_STATIC_SCRATCH_BYTES)
        return qsb::fail(QSB_ERR_INVALID, "nonlocal_apply_static: this projector set and band count need " +
                                              std::to_string(need) + " bytes of scratch; the static scratch holds " +
                                              std::to_string((size_t)QSB_NL_STATIC_SCRATCH_BYTES) +
                                              " (use fewer bands per call, or qsb_ham_nonlocal_apply)");
    void* ws = nullptr;
    QSB_TRY(static_scratch(dev, &ws));
    cudaStream_t s = (cudaStream_t)stream;
    double* coef = nullptr;
    QSB_TRY(qsb::nl_project(dtype, h->nl, h->nx, h->ny, h->nz, nb, is_complex, psi_dev, h->dx * h->dy * h->dz,
                            gx * h->dx, gy * h->dy, gz * h->dz, false, ws, &coef, s));
    return qsb::nl_apply(dtype, h->nl, (int)h->N, nb, is_complex, hpsi_dev, coef, gx * h->dx, gy * h->dy, gz * h->dz, s);
}
