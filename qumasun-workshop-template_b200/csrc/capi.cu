// extern "C" entry points of libqumasun_b200 (declared in include/qumasun_b200.h).
#include "qsb_internal.h"

#include <cmath>
#include <cstring>
#include <algorithm>
#include <string>
#include <vector>

namespace qsb {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

qsb_status fail(qsb_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

qsb_status cuda_fail(cudaError_t e, const char* where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? QSB_ERR_NOMEM : QSB_ERR_CUDA;
}

// Error word written by kernels whose bounded waits ran out (bit 0); one per
// device, its address looked up once per device.
static __device__ int g_device_error = 0;

int* device_error_word() {
    static int* addr[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
        addr[dev] = (int*)p;
    }
    return addr[dev];
}

static qsb_status check_grid(int nx, int ny, int nz) {
    if (nx < 1 || ny < 1 || nz < 1) return fail(QSB_ERR_INVALID, "grid dimensions must be >= 1");
    if ((long long)nx * ny * nz >= (1LL << 31)) return fail(QSB_ERR_INVALID, "grid has 2^31 or more points");
    return QSB_OK;
}

static qsb_status ensure_ws(qsb_ham* h, size_t bytes) {
    if (bytes <= h->ws_bytes) return QSB_OK;
    if (h->ws) cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
    cudaError_t e = cudaMalloc(&h->ws, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "workspace cudaMalloc");
    h->ws_bytes = bytes;
    return QSB_OK;
}

// GTH projector radial part, one projector per channel (i = 1):
//   p_l(r) = sqrt(2) r^l exp(-r^2 / (2 r_l^2)) / (r_l^(l+3/2) sqrt(Gamma(l+3/2)))
// (Goedecker, Teter, Hutter, PRB 54, 1703 (1996); Hartwigsen, Goedecker, Hutter,
// PRB 58, 3641 (1998)) times real spherical harmonics
//   Y_00 = 1/sqrt(4 pi),  Y_1{x,y,z} = sqrt(3/(4 pi)) {x,y,z}/r.
static void gth_points(double Rx, double Ry, double Rz, int nl, const double* r_l, const double* h_l, double rcut_factor,
                       double dx, double dy, double dz, std::vector<int>& coords, std::vector<double>& beta_cols,
                       std::vector<double>& energy, int& npts, int& width, std::vector<double>& dbeta_cols) {
    width = (nl >= 1 ? 1 : 0) + (nl >= 2 ? 3 : 0);
    npts = 0;
    if (width == 0) return;
    const double pi = 3.14159265358979323846;
    double rmax = 0.0;
    for (int l = 0; l < nl; ++l) rmax = std::max(rmax, rcut_factor * r_l[l]);
    const int ix0 = (int)std::floor((Rx - rmax) / dx), ix1 = (int)std::ceil((Rx + rmax) / dx);
    const int iy0 = (int)std::floor((Ry - rmax) / dy), iy1 = (int)std::ceil((Ry + rmax) / dy);
    const int iz0 = (int)std::floor((Rz - rmax) / dz), iz1 = (int)std::ceil((Rz + rmax) / dz);
    std::vector<double> cols[4], grads[3][4];   // grads[d][w]: d beta_w / d(x, y, z)
    const double rc0 = rcut_factor * r_l[0];
    const double rc1 = nl >= 2 ? rcut_factor * r_l[1] : 0.0;
    const double pre0 = std::sqrt(2.0) / (std::pow(r_l[0], 1.5) * std::sqrt(std::sqrt(pi) / 2.0)) / std::sqrt(4.0 * pi);
    const double pre1 = nl >= 2 ? std::sqrt(2.0) / (std::pow(r_l[1], 2.5) * std::sqrt(3.0 * std::sqrt(pi) / 4.0)) *
                                      std::sqrt(3.0 / (4.0 * pi))
                                : 0.0;
    for (int iz = iz0; iz <= iz1; ++iz)
        for (int iy = iy0; iy <= iy1; ++iy)
            for (int ix = ix0; ix <= ix1; ++ix) {
                const double x = ix * dx - Rx, y = iy * dy - Ry, z = iz * dz - Rz;
                const double r2 = x * x + y * y + z * z;
                if (r2 > rmax * rmax) continue;
                coords.push_back(ix); coords.push_back(iy); coords.push_back(iz);
                const double r = std::sqrt(r2);
                const double v[3] = {x, y, z};
                const double b0 = r <= rc0 ? pre0 * std::exp(-r2 / (2.0 * r_l[0] * r_l[0])) : 0.0;
                cols[0].push_back(b0);
                const double s0 = 1.0 / (r_l[0] * r_l[0]);
                for (int d = 0; d < 3; ++d) grads[d][0].push_back(-v[d] * s0 * b0);   // grad of a Gaussian
                if (nl >= 2) {
                    const double e1 = r <= rc1 ? pre1 * std::exp(-r2 / (2.0 * r_l[1] * r_l[1])) : 0.0;
                    const double s1 = 1.0 / (r_l[1] * r_l[1]);
                    for (int m = 0; m < 3; ++m) {
                        cols[1 + m].push_back(e1 * v[m]);
                        // d(e1 v_m)/d v_d = e1 (delta_md - v_m v_d / r1^2)
                        for (int d = 0; d < 3; ++d)
                            grads[d][1 + m].push_back(e1 * ((m == d ? 1.0 : 0.0) - v[m] * v[d] * s1));
                    }
                }
                ++npts;
            }
    for (int w = 0; w < width; ++w) beta_cols.insert(beta_cols.end(), cols[w].begin(), cols[w].end());
    for (int d = 0; d < 3; ++d)
        for (int w = 0; w < width; ++w) dbeta_cols.insert(dbeta_cols.end(), grads[d][w].begin(), grads[d][w].end());
    energy.push_back(h_l[0]);
    if (nl >= 2) for (int m = 0; m < 3; ++m) energy.push_back(h_l[1]);
}

}  // namespace qsb

using namespace qsb;

extern "C" {

const char* qsb_last_error(void) { return g_last_error.c_str(); }

qsb_status qsb_device_status(int* code, int clear) {
    if (!code) return fail(QSB_ERR_INVALID, "device_status: null code");
    int v = 0;
    QSB_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)));
    *code = v;
    if (clear && v) {
        const int zero = 0;
        QSB_CUDA_TRY(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)));
    }
    return QSB_OK;
}
const char* qsb_version(void) { return "qumasun_b200 0.1.0 (sm_100a)"; }

qsb_status qsb_laplacian8th(qsb_dtype dtype, int nx, int ny, int nz, int nb, void* out_dev, const void* p_dev,
                            double coef, double dx, double dy, double dz, void* stream) {
    QSB_TRY(check_grid(nx, ny, nz));
    if (nb < 0 || (nb > 0 && (!out_dev || !p_dev))) return fail(QSB_ERR_INVALID, "laplacian8th: bad bands/pointers");
    if (dtype != QSB_F64 && dtype != QSB_F32) return fail(QSB_ERR_INVALID, "laplacian8th: bad dtype");
    if (dx <= 0 || dy <= 0 || dz <= 0) return fail(QSB_ERR_INVALID, "laplacian8th: spacing must be > 0");
    if (nb == 0) return QSB_OK;
    StencilLaunch L{nx, ny, nz, nb, 0, 0, p_dev, out_dev, nullptr};
    return launch_stencil(dtype, L, make_fd8_coef(coef, dx, dy, dz, 0, 0, 0), (cudaStream_t)stream);
}

qsb_status qsb_laplacian_kpoint8th(qsb_dtype dtype, int nx, int ny, int nz, int nb, void* out_dev, const void* src_dev,
                                   double coef, double dx, double dy, double dz, double gx, double gy, double gz,
                                   void* stream) {
    QSB_TRY(check_grid(nx, ny, nz));
    if (nb < 0 || (nb > 0 && (!out_dev || !src_dev))) return fail(QSB_ERR_INVALID, "laplacian_kpoint8th: bad bands/pointers");
    if (dtype != QSB_F64 && dtype != QSB_F32) return fail(QSB_ERR_INVALID, "laplacian_kpoint8th: bad dtype");
    if (dx <= 0 || dy <= 0 || dz <= 0) return fail(QSB_ERR_INVALID, "laplacian_kpoint8th: spacing must be > 0");
    if (nb == 0) return QSB_OK;
    StencilLaunch L{nx, ny, nz, nb, 1, 0, src_dev, out_dev, nullptr};
    return launch_stencil(dtype, L, make_fd8_coef(coef, dx, dy, dz, gx, gy, gz), (cudaStream_t)stream);
}

qsb_status qsb_ham_create(qsb_ham** ham, int nx, int ny, int nz, double dx, double dy, double dz) {
    if (!ham) return fail(QSB_ERR_INVALID, "ham_create: null handle pointer");
    *ham = nullptr;
    QSB_TRY(check_grid(nx, ny, nz));
    if (dx <= 0 || dy <= 0 || dz <= 0) return fail(QSB_ERR_INVALID, "ham_create: spacing must be > 0");
    // the device the tables will live on (host-only checks also work without one)
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        dev = -1;
        cudaGetLastError();
    }
    qsb_ham* h = new qsb_ham();
    h->device = dev;
    h->nx = nx; h->ny = ny; h->nz = nz;
    h->N = (size_t)nx * ny * nz;
    h->dx = dx; h->dy = dy; h->dz = dz;
    *ham = h;
    return QSB_OK;
}

qsb_status qsb_ham_destroy(qsb_ham* h) {
    if (!h) return QSB_OK;
    if (h->V64) cudaFree(h->V64);
    if (h->V32) cudaFree(h->V32);
    if (h->ws) cudaFree(h->ws);
    if (h->stage) cudaFree(h->stage);
    kinetic_fft_free(h);
    for (cudaEvent_t e : h->pev)
        if (e) cudaEventDestroy(e);
    if (h->up) cudaStreamDestroy(h->up);
    if (h->down) cudaStreamDestroy(h->down);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->ev_rec) cudaEventDestroy(e);
    nl_free(h->nl);
    delete h;
    return QSB_OK;
}

// V64 = V, V32 = (float)V, flag = 1 on a non-finite value
static __global__ void potential_copy_kernel(size_t N, const double* __restrict__ V, double* __restrict__ V64,
                                      float* __restrict__ V32, int* __restrict__ flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const double v = V[i];
        bad |= !isfinite(v);
        V64[i] = v;
        V32[i] = (float)v;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) *flag = 1;
}

qsb_status qsb_ham_set_potential(qsb_ham* h, const double* V, int on_device) {
    if (!h || !V) return fail(QSB_ERR_INVALID, "set_potential: null argument");
    if (!h->V64) QSB_CUDA_TRY(cudaMalloc((void**)&h->V64, h->N * sizeof(double)));
    if (!h->V32) QSB_CUDA_TRY(cudaMalloc((void**)&h->V32, h->N * sizeof(float)));
    if (on_device) {
        // stays on the device: copy, FP32 copy and a non-finite flag (4 bytes back)
        int* flag = nullptr;
        QSB_CUDA_TRY(cudaMalloc((void**)&flag, sizeof(int)));
        QSB_CUDA_TRY(cudaMemset(flag, 0, sizeof(int)));
        potential_copy_kernel<<<(unsigned)std::min<size_t>((h->N + 255) / 256, 148 * 8), 256>>>(h->N, V, h->V64,
                                                                                              h->V32, flag);
        int hf = 0;
        const cudaError_t e = cudaGetLastError();
        QSB_CUDA_TRY(cudaMemcpy(&hf, flag, sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(flag);
        if (e != cudaSuccess) return cuda_fail(e, "potential_copy_kernel");
        if (hf) return fail(QSB_ERR_NUMERIC, "set_potential: non-finite value");
        return QSB_OK;
    }
    std::vector<double> hv(h->N);
    std::memcpy(hv.data(), V, h->N * sizeof(double));
    for (size_t i = 0; i < h->N; ++i)
        if (!std::isfinite(hv[i])) return fail(QSB_ERR_NUMERIC, "set_potential: non-finite value");
    std::vector<float> hf(hv.begin(), hv.end());
    QSB_CUDA_TRY(cudaMemcpy(h->V64, hv.data(), h->N * sizeof(double), cudaMemcpyHostToDevice));
    QSB_CUDA_TRY(cudaMemcpy(h->V32, hf.data(), h->N * sizeof(float), cudaMemcpyHostToDevice));
    return QSB_OK;
}

qsb_status qsb_ham_set_projectors(qsb_ham* h, int n_atoms, const int* npts, const int* widths, const int* coords,
                                  const double* beta, const double* energy) {
    if (!h) return fail(QSB_ERR_INVALID, "set_projectors: null context");
    if (n_atoms > 0 && (!npts || !widths)) return fail(QSB_ERR_INVALID, "set_projectors: null npts/widths");
    long long tot = 0, totw = 0;
    for (int a = 0; a < n_atoms; ++a) { tot += npts[a]; totw += (long long)npts[a] * widths[a]; }
    if (tot > 0 && !coords) return fail(QSB_ERR_INVALID, "set_projectors: null coords");
    if (totw > 0 && (!beta || !energy)) return fail(QSB_ERR_INVALID, "set_projectors: null beta/energy");
    return nl_upload(h->nl, h->nx, h->ny, h->nz, n_atoms, npts, widths, coords, beta, energy);
}

qsb_status qsb_ham_set_gth_projectors(qsb_ham* h, int n_atoms, const double* pos, const int* species, int n_species,
                                      const int* nl, const double* r_l, const double* h_l, double rcut_factor) {
    if (!h) return fail(QSB_ERR_INVALID, "set_gth_projectors: null context");
    if (n_atoms < 0 || n_species < 0 || (n_atoms > 0 && (!pos || !species || !nl || !r_l || !h_l)))
        return fail(QSB_ERR_INVALID, "set_gth_projectors: bad arguments");
    if (!(rcut_factor > 0)) return fail(QSB_ERR_INVALID, "set_gth_projectors: rcut_factor must be > 0");
    std::vector<int> npts(n_atoms), widths(n_atoms), coords;
    std::vector<double> beta, energy, dbeta;
    for (int a = 0; a < n_atoms; ++a) {
        const int s = species[a];
        if (s < 0 || s >= n_species || nl[s] < 0 || nl[s] > 2)
            return fail(QSB_ERR_INVALID, "set_gth_projectors: bad species / channel count");
        for (int l = 0; l < nl[s]; ++l)
            if (!(r_l[2 * s + l] > 0)) return fail(QSB_ERR_INVALID, "set_gth_projectors: r_l must be > 0");
        gth_points(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], nl[s], r_l + 2 * s, h_l + 2 * s, rcut_factor, h->dx,
                   h->dy, h->dz, coords, beta, energy, npts[a], widths[a], dbeta);
    }
    QSB_TRY(nl_upload(h->nl, h->nx, h->ny, h->nz, n_atoms, npts.data(), widths.data(), coords.data(), beta.data(),
                      energy.data()));
    return nl_upload_gradients(h->nl, dbeta.data());
}

qsb_status qsb_ham_set_projector_gradients(qsb_ham* h, const double* dbeta) {
    if (!h) return fail(QSB_ERR_INVALID, "set_projector_gradients: null context");
    return nl_upload_gradients(h->nl, dbeta);
}

static qsb_status energy_force(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi,
                               const double* occupancies, double gx, double gy, double gz, double* energy,
                               double* forces, void* stream) {
    if (!h || !energy) return fail(QSB_ERR_INVALID, "nonlocal energy: null argument");
    if (dtype != QSB_F64 && dtype != QSB_F32) return fail(QSB_ERR_INVALID, "nonlocal energy: bad dtype");
    if (nb < 0 || (nb > 0 && (!psi || !occupancies))) return fail(QSB_ERR_INVALID, "nonlocal energy: bad bands/pointers");
    *energy = 0.0;
    if (nb == 0 || h->nl.n_points == 0) return QSB_OK;
    if (!is_complex) gx = gy = gz = 0.0;
    const int ncol = is_complex ? 2 * nb : nb;
    QSB_TRY(ensure_ws(h, nl_energy_force_bytes(h->nl, ncol, nb)));
    return nl_energy_force(dtype, h->nl, h->nx, h->ny, h->nz, nb, is_complex, psi, occupancies, h->dx * h->dy * h->dz,
                           gx * h->dx, gy * h->dy, gz * h->dz, energy, forces, h->ws, (cudaStream_t)stream);
}

qsb_status qsb_ham_nonlocal_energy(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi,
                                   const double* occupancies, double gx, double gy, double gz, double* energy,
                                   void* stream) {
    return energy_force(h, dtype, is_complex, nb, psi, occupancies, gx, gy, gz, energy, nullptr, stream);
}

qsb_status qsb_ham_nonlocal_energy_force(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi,
                                         const double* occupancies, double gx, double gy, double gz, double* energy,
                                         double* forces, void* stream) {
    if (!forces) return fail(QSB_ERR_INVALID, "nonlocal energy_force: null forces");
    return energy_force(h, dtype, is_complex, nb, psi, occupancies, gx, gy, gz, energy, forces, stream);
}

qsb_status qsb_ham_projector_info(const qsb_ham* h, int64_t* total_points, int* total_projectors) {
    if (!h) return fail(QSB_ERR_INVALID, "projector_info: null context");
    if (total_points) *total_points = h->nl.n_points;
    if (total_projectors) *total_projectors = h->nl.total_proj;
    return QSB_OK;
}

static qsb_status timing_event(qsb_ham* h, cudaStream_t s) {
    cudaEvent_t e;
    if (!h->ev_pool.empty()) {
        e = h->ev_pool.back();
        h->ev_pool.pop_back();
    } else {
        QSB_CUDA_TRY(cudaEventCreate(&e));
    }
    QSB_CUDA_TRY(cudaEventRecord(e, s));
    h->ev_rec.push_back(e);
    return QSB_OK;
}

}  // extern "C"

qsb_status qsb::check_apply(qsb_ham* h, qsb_dtype dtype, int nb, const void* a, const void* b) {
    if (!h) return fail(QSB_ERR_INVALID, "null context");
    if (dtype != QSB_F64 && dtype != QSB_F32) return fail(QSB_ERR_INVALID, "bad dtype");
    if (nb < 0 || (nb > 0 && (!a || !b))) return fail(QSB_ERR_INVALID, "bad bands/pointers");
    return QSB_OK;
}

extern "C" {

qsb_status qsb_ham_apply(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi_dev, void* hpsi_dev,
                         double gx, double gy, double gz, void* stream) {
    QSB_TRY(check_apply(h, dtype, nb, psi_dev, hpsi_dev));
    if (!h->V64) return fail(QSB_ERR_STATE, "ham_apply: potential not set");
    if (nb == 0) return QSB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (!is_complex) gx = gy = gz = 0.0;
    const double dV = h->dx * h->dy * h->dz;
    const bool has_nl = h->nl.n_points > 0;
    const int ncol = is_complex ? 2 * nb : nb;
    double* coef = nullptr;
    if (has_nl) QSB_TRY(ensure_ws(h, nl_workspace_bytes(h->nl, ncol)));
    if (h->timing) QSB_TRY(timing_event(h, s));
    // 1) <beta|psi>: deterministic chunked projection (mInnerNonlocalPsi_v4_bundle)
    if (has_nl) {
        QSB_TRY(nl_project(dtype, h->nl, h->nx, h->ny, h->nz, nb, is_complex, psi_dev, dV, gx * h->dx, gy * h->dy,
                           gz * h->dz, false, h->ws, &coef, s));
        h->launches += 2;
    }
    if (h->timing) QSB_TRY(timing_event(h, s));
    if (h->kinetic == 1) {
        // 2') hpsi = V psi + FFT kinetic   (mHamiltonianMatrix_ddm_bundle, algorithm 1)
        QSB_TRY(kinetic_fft_apply(h, dtype, is_complex, nb, psi_dev, hpsi_dev, gx, gy, gz, s, &h->launches));
    } else {
        // 2) hpsi = V psi - 1/2 FD8(psi)   (mPotentialMatrix_ddm + mKineticMatrixAdd_ddm_kpint)
        StencilLaunch L{h->nx, h->ny, h->nz, nb, is_complex ? 1 : 0, 1, psi_dev, hpsi_dev,
                        dtype == QSB_F64 ? (const void*)h->V64 : (const void*)h->V32};
        QSB_TRY(launch_stencil(dtype, L, make_fd8_coef(-0.5, h->dx, h->dy, h->dz, gx, gy, gz), s));
        h->launches += 1;
    }
    if (h->timing) QSB_TRY(timing_event(h, s));
    // 3) hpsi += sum |beta> E <beta|psi>   (ProjectionPP_bundle expansion, pull form)
    if (has_nl) {
        QSB_TRY(nl_apply(dtype, h->nl, (int)h->N, nb, is_complex, hpsi_dev, coef, gx * h->dx, gy * h->dy, gz * h->dz, s));
        h->launches += 1;
    }
    if (h->timing) QSB_TRY(timing_event(h, s));
    return QSB_OK;
}

// H psi of host bundles: band chunks go through two device staging slots, the
// host-to-device copy of chunk k + 1 (stream up), the apply of chunk k (the
// caller's stream) and the device-to-host copy of chunk k - 1 (stream down)
// overlapping, so that both copy directions of the host link run at once.
qsb_status qsb_ham_apply_host(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi_host,
                              void* hpsi_host, double gx, double gy, double gz, int chunk_bands, void* stream) {
    QSB_TRY(check_apply(h, dtype, nb, psi_host, hpsi_host));
    if (!h->V64) return fail(QSB_ERR_STATE, "ham_apply_host: potential not set");
    if (chunk_bands < 0) return fail(QSB_ERR_INVALID, "ham_apply_host: chunk_bands must be >= 0");
    if (nb == 0) return QSB_OK;
    const int chunk = std::min(nb, chunk_bands > 0 ? chunk_bands : std::max(1, (nb + 15) / 16));
    const size_t band_bytes = (is_complex ? 2 : 1) * h->N * (dtype == QSB_F64 ? 8 : 4);
    const size_t slot = (size_t)chunk * band_bytes;      // one psi or hpsi chunk
    if (h->stage_bytes < 4 * slot) {
        if (h->stage) QSB_CUDA_TRY(cudaFree(h->stage));
        h->stage = nullptr;
        h->stage_bytes = 0;
        QSB_CUDA_TRY(cudaMalloc(&h->stage, 4 * slot));
        h->stage_bytes = 4 * slot;
    }
    if (!h->up) QSB_CUDA_TRY(cudaStreamCreateWithFlags(&h->up, cudaStreamNonBlocking));
    if (!h->down) QSB_CUDA_TRY(cudaStreamCreateWithFlags(&h->down, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->pev)
        if (!e) QSB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t start = h->pev[0], *in_ready = h->pev + 1, *done = h->pev + 3, *out_free = h->pev + 5;
    char* d_in[2] = {(char*)h->stage, (char*)h->stage + slot};
    char* d_out[2] = {(char*)h->stage + 2 * slot, (char*)h->stage + 3 * slot};
    const char* src = (const char*)psi_host;
    char* dst = (char*)hpsi_host;
    // the staging slots are free once everything before this call on the caller's stream is done
    QSB_CUDA_TRY(cudaEventRecord(start, s));
    QSB_CUDA_TRY(cudaStreamWaitEvent(h->up, start, 0));
    QSB_CUDA_TRY(cudaStreamWaitEvent(h->down, start, 0));
    const int n_chunks = (nb + chunk - 1) / chunk;
    for (int k = 0; k < n_chunks; ++k) {
        const int j = k & 1;
        const int b0 = k * chunk, nbk = std::min(chunk, nb - b0);
        const size_t bytes = (size_t)nbk * band_bytes, off = (size_t)b0 * band_bytes;
        if (k >= 2) QSB_CUDA_TRY(cudaStreamWaitEvent(h->up, done[j], 0));        // apply k - 2 read slot j
        QSB_CUDA_TRY(cudaMemcpyAsync(d_in[j], src + off, bytes, cudaMemcpyHostToDevice, h->up));
        QSB_CUDA_TRY(cudaEventRecord(in_ready[j], h->up));
        QSB_CUDA_TRY(cudaStreamWaitEvent(s, in_ready[j], 0));
        if (k >= 2) QSB_CUDA_TRY(cudaStreamWaitEvent(s, out_free[j], 0));        // copy-out k - 2 left slot j
        QSB_TRY(qsb_ham_apply(h, dtype, is_complex, nbk, d_in[j], d_out[j], gx, gy, gz, s));
        QSB_CUDA_TRY(cudaEventRecord(done[j], s));
        QSB_CUDA_TRY(cudaStreamWaitEvent(h->down, done[j], 0));
        QSB_CUDA_TRY(cudaMemcpyAsync(dst + off, d_out[j], bytes, cudaMemcpyDeviceToHost, h->down));
        QSB_CUDA_TRY(cudaEventRecord(out_free[j], h->down));
    }
    // the caller's stream sees the last copies out (and the copy streams' work ends there)
    QSB_CUDA_TRY(cudaStreamWaitEvent(s, out_free[(n_chunks - 1) & 1], 0));
    if (n_chunks > 1) QSB_CUDA_TRY(cudaStreamWaitEvent(s, out_free[n_chunks & 1], 0));
    QSB_CUDA_TRY(cudaEventRecord(start, h->up));
    QSB_CUDA_TRY(cudaStreamWaitEvent(s, start, 0));
    return QSB_OK;
}

qsb_status qsb_ham_set_kinetic(qsb_ham* h, int algorithm) {
    if (!h) return fail(QSB_ERR_INVALID, "set_kinetic: null context");
    if (algorithm != 0 && algorithm != 1) return fail(QSB_ERR_INVALID, "set_kinetic: algorithm must be 0 (FD8) or 1 (FFT)");
    h->kinetic = algorithm;
    return QSB_OK;
}

qsb_status qsb_ham_set_timing(qsb_ham* h, int enable) {
    if (!h) return fail(QSB_ERR_INVALID, "set_timing: null context");
    h->timing = enable != 0;
    return QSB_OK;
}

qsb_status qsb_ham_get_timing(qsb_ham* h, double* project_ms, double* stencil_ms, double* expand_ms, int* applies,
                              int* kernel_launches) {
    if (!h) return fail(QSB_ERR_INVALID, "get_timing: null context");
    double pm = 0.0, sm = 0.0, em = 0.0;
    const size_t n = h->ev_rec.size() / 4;
    for (size_t i = 0; i < n; ++i) {
        float a = 0.f, b = 0.f, c = 0.f;
        QSB_CUDA_TRY(cudaEventSynchronize(h->ev_rec[4 * i + 3]));
        QSB_CUDA_TRY(cudaEventElapsedTime(&a, h->ev_rec[4 * i], h->ev_rec[4 * i + 1]));
        QSB_CUDA_TRY(cudaEventElapsedTime(&b, h->ev_rec[4 * i + 1], h->ev_rec[4 * i + 2]));
        QSB_CUDA_TRY(cudaEventElapsedTime(&c, h->ev_rec[4 * i + 2], h->ev_rec[4 * i + 3]));
        pm += a;
        sm += b;
        em += c;
    }
    h->ev_pool.insert(h->ev_pool.end(), h->ev_rec.begin(), h->ev_rec.end());
    h->ev_rec.clear();
    if (project_ms) *project_ms = pm;
    if (stencil_ms) *stencil_ms = sm;
    if (expand_ms) *expand_ms = em;
    if (applies) *applies = (int)n;
    if (kernel_launches) *kernel_launches = h->launches;
    h->launches = 0;
    return QSB_OK;
}

qsb_status qsb_ham_nonlocal_apply(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi_dev,
                                  void* hpsi_dev, double gx, double gy, double gz, void* stream) {
    QSB_TRY(check_apply(h, dtype, nb, psi_dev, hpsi_dev));
    if (nb == 0 || h->nl.n_points == 0) return QSB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (!is_complex) gx = gy = gz = 0.0;
    const int ncol = is_complex ? 2 * nb : nb;
    QSB_TRY(ensure_ws(h, nl_workspace_bytes(h->nl, ncol)));
    double* coef = nullptr;
    QSB_TRY(nl_project(dtype, h->nl, h->nx, h->ny, h->nz, nb, is_complex, psi_dev, h->dx * h->dy * h->dz, gx * h->dx,
                       gy * h->dy, gz * h->dz, false, h->ws, &coef, s));
    return nl_apply(dtype, h->nl, (int)h->N, nb, is_complex, hpsi_dev, coef, gx * h->dx, gy * h->dy, gz * h->dz, s);
}

qsb_status qsb_ham_nonlocal_project(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi_dev,
                                    double gx, double gy, double gz, double* out_host, void* stream) {
    QSB_TRY(check_apply(h, dtype, nb, psi_dev, out_host));
    if (nb == 0 || h->nl.total_proj == 0) return QSB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (!is_complex) gx = gy = gz = 0.0;
    const int ncol = is_complex ? 2 * nb : nb;
    const int P = h->nl.total_proj;
    std::vector<double> coef_h;
    if (h->nl.n_points > 0) {
        QSB_TRY(ensure_ws(h, nl_workspace_bytes(h->nl, ncol)));
        double* coef = nullptr;
        QSB_TRY(nl_project(dtype, h->nl, h->nx, h->ny, h->nz, nb, is_complex, psi_dev, h->dx * h->dy * h->dz,
                           gx * h->dx, gy * h->dy, gz * h->dz, true, h->ws, &coef, s));
        coef_h.resize((size_t)h->nl.n_atoms * h->nl.wmax * ncol);
        QSB_CUDA_TRY(cudaMemcpyAsync(coef_h.data(), coef, coef_h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        QSB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    std::memset(out_host, 0, sizeof(double) * (size_t)P * ncol);
    for (int a = 0; a < h->nl.n_atoms; ++a)
        for (int w = 0; w < h->nl.h_atom_width[a]; ++w)
            for (int c = 0; c < ncol; ++c)
                out_host[(size_t)c * P + h->nl.h_atom_proj_off[a] + w] =
                    coef_h.empty() ? 0.0 : coef_h[((size_t)a * h->nl.wmax + w) * ncol + c];
    return QSB_OK;
}

}  // extern "C"
