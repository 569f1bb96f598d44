// FFT kinetic operator: the reference's default Hamiltonian
// (mHamiltonianMatrix_ddm_bundle with m_algorithm_Laplacian = 1,
// source/qumasun_base1.matrix.h:171-228; source/qumasun_base1.h:243):
//   hpsi = IFFT( |G + k|^2 / 2 * FFT(psi) ) / N + V psi
// with G_d = 2 pi m / (n_d h_d), m folded as (2m > n ? m - n : m) -- the
// Nyquist index of an even grid stays +n/2 (OperateKineticInKspace_bundle,
// :96-123) -- and the 1/N applied after the inverse transform, as there.
//
// B200 form: bands go through batched cuFFT plans in chunks of FFT_CHUNK
// (plans and one spectrum buffer cached in the context).  Real Gamma-point
// bands go two to a complex field through the C2C transforms (the multiplier
// is real and even at k = 0, so the operator acts on real and imaginary parts
// apart); a single real band uses R2C / C2R (half the spectrum); complex SoA bands
// are interleaved into the spectrum buffer by one pass, transformed C2C, and
// the pass after the inverse transform de-interleaves, scales by 1/N and adds
// V psi in one read of psi and one write of hpsi.
#include "qsb_internal.h"
#include <cufft.h>
#include <algorithm>

namespace qsb {

namespace {

constexpr int FFT_CHUNK = 32;     // bands per batched transform
constexpr int KT = 256;

__device__ __forceinline__ double gfold(int m, int n, double c) { return c * (double)(2 * m > n ? m - n : m); }

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = cufftDoubleComplex; };
template <> struct Cplx<float> { using type = cufftComplex; };

// spectrum of real bands: batch x nz x ny x (nx/2 + 1), x fastest
template <typename C>
__global__ void __launch_bounds__(KT) kmul_half_kernel(C* __restrict__ spec, size_t total, int nx, int ny, int nz,
                                                       double cx, double cy, double cz) {
    const int nxh = nx / 2 + 1;
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const int kx = (int)(i % nxh);
        const size_t r = i / nxh;
        const int ky = (int)(r % ny);
        const int kz = (int)((r / ny) % nz);
        const double gx = gfold(kx, nx, cx), gy = gfold(ky, ny, cy), gz = gfold(kz, nz, cz);
        const double m = 0.5 * (gx * gx + gy * gy + gz * gz);
        C v = spec[i];
        v.x = (decltype(v.x))(v.x * m);
        v.y = (decltype(v.y))(v.y * m);
        spec[i] = v;
    }
}

// spectrum of complex bands: batch x nz x ny x nx
template <typename C>
__global__ void __launch_bounds__(KT) kmul_full_kernel(C* __restrict__ spec, size_t total, int nx, int ny, int nz,
                                                       double cx, double cy, double cz, double kx0, double ky0,
                                                       double kz0) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const int kx = (int)(i % nx);
        const size_t r = i / nx;
        const int ky = (int)(r % ny);
        const int kz = (int)((r / ny) % nz);
        const double gx = gfold(kx, nx, cx) + kx0, gy = gfold(ky, ny, cy) + ky0, gz = gfold(kz, nz, cz) + kz0;
        const double m = 0.5 * (gx * gx + gy * gy + gz * gz);
        C v = spec[i];
        v.x = (decltype(v.x))(v.x * m);
        v.y = (decltype(v.y))(v.y * m);
        spec[i] = v;
    }
}

// real bands: hpsi = hpsi / N + V psi (hpsi holds the unnormalised inverse transform)
template <typename T>
__global__ void __launch_bounds__(KT) finish_real_kernel(T* __restrict__ hpsi, const T* __restrict__ psi,
                                                         const T* __restrict__ V, size_t N, size_t total,
                                                         double inv_n) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT)
        hpsi[i] = (T)((double)hpsi[i] * inv_n) + V[i % N] * psi[i];
}

// complex SoA bands -> interleaved spectrum buffer
template <typename T, typename C>
__global__ void __launch_bounds__(KT) interleave_kernel(C* __restrict__ spec, const T* __restrict__ psi, size_t N,
                                                        size_t total) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const size_t b = i / N, p = i % N;
        C v;
        v.x = psi[2 * b * N + p];
        v.y = psi[(2 * b + 1) * N + p];
        spec[i] = v;
    }
}

// complex bands: hpsi (SoA) = spectrum / N + V psi
template <typename T, typename C>
__global__ void __launch_bounds__(KT) finish_cplx_kernel(T* __restrict__ hpsi, const C* __restrict__ spec,
                                                         const T* __restrict__ psi, const T* __restrict__ V,
                                                         size_t N, size_t total, double inv_n) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const size_t b = i / N, p = i % N;
        const C v = spec[i];
        const T vp = V[p];
        const size_t re = 2 * b * N + p, im = re + N;
        hpsi[re] = (T)((double)v.x * inv_n) + vp * psi[re];
        hpsi[im] = (T)((double)v.y * inv_n) + vp * psi[im];
    }
}

// real bands, two to a complex field: spec[p] = psi[2p] + i psi[2p+1] (zero
// imaginary part for an odd last band).  The multiplier is real and even at
// k = 0, so the kinetic operator is real and acts on the two bands
// independently: T(a + ib) = Ta + iTb.
template <typename T, typename C>
__global__ void __launch_bounds__(KT) pack_pairs_kernel(C* __restrict__ spec, const T* __restrict__ psi, size_t N,
                                                        int bands, size_t total) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const size_t pr = i / N, p = i - pr * N;
        const size_t b0 = 2 * pr;
        C v;
        v.x = psi[b0 * N + p];
        v.y = (int)b0 + 1 < bands ? psi[(b0 + 1) * N + p] : (T)0;
        spec[i] = v;
    }
}

// hpsi[2p] = Re spec[p] / N + V psi[2p], hpsi[2p+1] = Im spec[p] / N + V psi[2p+1]
template <typename T, typename C>
__global__ void __launch_bounds__(KT) finish_pairs_kernel(T* __restrict__ hpsi, const C* __restrict__ spec,
                                                          const T* __restrict__ psi, const T* __restrict__ V,
                                                          size_t N, int bands, size_t total, double inv_n) {
    for (size_t i = blockIdx.x * (size_t)KT + threadIdx.x; i < total; i += (size_t)gridDim.x * KT) {
        const size_t pr = i / N, p = i - pr * N;
        const size_t b0 = 2 * pr;
        const C v = spec[i];
        const T vp = V[p];
        hpsi[b0 * N + p] = (T)((double)v.x * inv_n) + vp * psi[b0 * N + p];
        if ((int)b0 + 1 < bands) hpsi[(b0 + 1) * N + p] = (T)((double)v.y * inv_n) + vp * psi[(b0 + 1) * N + p];
    }
}

unsigned grid_for(size_t total) {
    return (unsigned)std::max<size_t>(1, std::min<size_t>((total + KT - 1) / KT, 148 * 16));
}

#define QSB_FFT_TRY(expr)                                                                              \
    do {                                                                                               \
        const cufftResult r_ = (expr);                                                                 \
        if (r_ != CUFFT_SUCCESS)                                                                       \
            return fail(QSB_ERR_CUDA, std::string("cuFFT call failed (") + std::to_string((int)r_) +   \
                                          "): " + #expr);                                              \
    } while (0)

qsb_status get_plan(qsb_ham* h, int dtype, int cplx, int batch, qsb_ham::FftPlan** out) {
    for (auto& p : h->fft_plans)
        if (p.dtype == dtype && p.cplx == cplx && p.batch == batch) {
            *out = &p;
            return QSB_OK;
        }
    int n[3] = {h->nz, h->ny, h->nx};
    cufftHandle f = 0, b = 0;
    const bool dbl = dtype == QSB_F64;
    const cufftType tf = cplx ? (dbl ? CUFFT_Z2Z : CUFFT_C2C) : (dbl ? CUFFT_D2Z : CUFFT_R2C);
    const cufftType tb = cplx ? (dbl ? CUFFT_Z2Z : CUFFT_C2C) : (dbl ? CUFFT_Z2D : CUFFT_C2R);
    QSB_FFT_TRY(cufftPlanMany(&f, 3, n, nullptr, 1, 0, nullptr, 1, 0, tf, batch));
    if (cplx) {
        b = f;   // one C2C plan serves both directions
    } else {
        const cufftResult r = cufftPlanMany(&b, 3, n, nullptr, 1, 0, nullptr, 1, 0, tb, batch);
        if (r != CUFFT_SUCCESS) {
            cufftDestroy(f);
            return fail(QSB_ERR_CUDA, "cuFFT plan (inverse) failed: " + std::to_string((int)r));
        }
    }
    h->fft_plans.push_back(qsb_ham::FftPlan{dtype, cplx, batch, (int)f, (int)b});
    *out = &h->fft_plans.back();
    return QSB_OK;
}

template <typename T>
qsb_status apply_t(qsb_ham* h, qsb_dtype dtype, int cplx, int nb, const T* psi, T* hpsi, double gx, double gy,
                   double gz, cudaStream_t s, int* launches) {
    using C = typename Cplx<T>::type;
    const size_t N = h->N;
    if (!cplx && nb > 1) {
        // real bands in pairs through the complex transforms: cuFFT's complex
        // passes run at ~4.8 TB/s where its x-direction R2C / C2R kernels run
        // at ~1.65 TB/s on these grids
        const int chunk = std::min(nb, FFT_CHUNK);
        const int pmax = (chunk + 1) / 2;
        const size_t need = (size_t)pmax * N * sizeof(C);
        if (h->fft_buf_bytes < need) {
            if (h->fft_buf) QSB_CUDA_TRY(cudaFree(h->fft_buf));
            h->fft_buf = nullptr;
            h->fft_buf_bytes = 0;
            QSB_CUDA_TRY(cudaMalloc(&h->fft_buf, need));
            h->fft_buf_bytes = need;
        }
        C* spec = (C*)h->fft_buf;
        const T* V = dtype == QSB_F64 ? (const T*)h->V64 : (const T*)h->V32;
        const double cx = 2.0 * M_PI / (h->dx * h->nx), cy = 2.0 * M_PI / (h->dy * h->ny),
                     cz = 2.0 * M_PI / (h->dz * h->nz);
        const double inv_n = 1.0 / (double)N;
        for (int b0 = 0; b0 < nb; b0 += chunk) {
            const int bc = std::min(chunk, nb - b0);
            const int pairs = (bc + 1) / 2;
            qsb_ham::FftPlan* p = nullptr;
            QSB_TRY(get_plan(h, dtype, 1, pairs, &p));
            QSB_FFT_TRY(cufftSetStream((cufftHandle)p->forward, s));
            const T* x = psi + (size_t)b0 * N;
            T* y = hpsi + (size_t)b0 * N;
            const size_t npts = (size_t)pairs * N;
            pack_pairs_kernel<T, C><<<grid_for(npts), KT, 0, s>>>(spec, x, N, bc, npts);
            QSB_CUDA_TRY(cudaGetLastError());
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecZ2Z((cufftHandle)p->forward, spec, spec, CUFFT_FORWARD));
            } else {
                QSB_FFT_TRY(cufftExecC2C((cufftHandle)p->forward, spec, spec, CUFFT_FORWARD));
            }
            kmul_full_kernel<C><<<grid_for(npts), KT, 0, s>>>(spec, npts, h->nx, h->ny, h->nz, cx, cy, cz, 0.0, 0.0,
                                                               0.0);
            QSB_CUDA_TRY(cudaGetLastError());
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecZ2Z((cufftHandle)p->backward, spec, spec, CUFFT_INVERSE));
            } else {
                QSB_FFT_TRY(cufftExecC2C((cufftHandle)p->backward, spec, spec, CUFFT_INVERSE));
            }
            finish_pairs_kernel<T, C><<<grid_for(npts), KT, 0, s>>>(y, spec, x, V, N, bc, npts, inv_n);
            QSB_CUDA_TRY(cudaGetLastError());
            *launches += 3;
        }
        return QSB_OK;
    }
    const int nxh = h->nx / 2 + 1;
    const size_t spec_per_band = cplx ? N : (size_t)h->nz * h->ny * nxh;
    const int chunk = std::min(nb, FFT_CHUNK);
    const size_t need = (size_t)chunk * spec_per_band * sizeof(C);
    if (h->fft_buf_bytes < need) {
        if (h->fft_buf) QSB_CUDA_TRY(cudaFree(h->fft_buf));
        h->fft_buf = nullptr;
        h->fft_buf_bytes = 0;
        QSB_CUDA_TRY(cudaMalloc(&h->fft_buf, need));
        h->fft_buf_bytes = need;
    }
    C* spec = (C*)h->fft_buf;
    const T* V = dtype == QSB_F64 ? (const T*)h->V64 : (const T*)h->V32;
    const double cx = 2.0 * M_PI / (h->dx * h->nx), cy = 2.0 * M_PI / (h->dy * h->ny),
                 cz = 2.0 * M_PI / (h->dz * h->nz);
    const double inv_n = 1.0 / (double)N;
    const int cols = cplx ? 2 : 1;
    for (int b0 = 0; b0 < nb; b0 += chunk) {
        const int bc = std::min(chunk, nb - b0);
        qsb_ham::FftPlan* p = nullptr;
        QSB_TRY(get_plan(h, dtype, cplx, bc, &p));
        QSB_FFT_TRY(cufftSetStream((cufftHandle)p->forward, s));
        QSB_FFT_TRY(cufftSetStream((cufftHandle)p->backward, s));
        const T* x = psi + (size_t)b0 * cols * N;
        T* y = hpsi + (size_t)b0 * cols * N;
        const size_t nspec = (size_t)bc * spec_per_band, npts = (size_t)bc * N;
        if (!cplx) {
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecD2Z((cufftHandle)p->forward, (cufftDoubleReal*)x, (cufftDoubleComplex*)spec));
            } else {
                QSB_FFT_TRY(cufftExecR2C((cufftHandle)p->forward, (cufftReal*)x, (cufftComplex*)spec));
            }
            kmul_half_kernel<C><<<grid_for(nspec), KT, 0, s>>>(spec, nspec, h->nx, h->ny, h->nz, cx, cy, cz);
            QSB_CUDA_TRY(cudaGetLastError());
            // out of place into hpsi (the inverse real transform consumes the spectrum)
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecZ2D((cufftHandle)p->backward, (cufftDoubleComplex*)spec, (cufftDoubleReal*)y));
            } else {
                QSB_FFT_TRY(cufftExecC2R((cufftHandle)p->backward, (cufftComplex*)spec, (cufftReal*)y));
            }
            finish_real_kernel<T><<<grid_for(npts), KT, 0, s>>>(y, x, V, N, npts, inv_n);
            QSB_CUDA_TRY(cudaGetLastError());
            *launches += 2;
        } else {
            interleave_kernel<T, C><<<grid_for(npts), KT, 0, s>>>(spec, x, N, npts);
            QSB_CUDA_TRY(cudaGetLastError());
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecZ2Z((cufftHandle)p->forward, spec, spec, CUFFT_FORWARD));
            } else {
                QSB_FFT_TRY(cufftExecC2C((cufftHandle)p->forward, spec, spec, CUFFT_FORWARD));
            }
            kmul_full_kernel<C><<<grid_for(nspec), KT, 0, s>>>(spec, nspec, h->nx, h->ny, h->nz, cx, cy, cz, gx, gy,
                                                                gz);
            QSB_CUDA_TRY(cudaGetLastError());
            if constexpr (sizeof(T) == 8) {
                QSB_FFT_TRY(cufftExecZ2Z((cufftHandle)p->backward, spec, spec, CUFFT_INVERSE));
            } else {
                QSB_FFT_TRY(cufftExecC2C((cufftHandle)p->backward, spec, spec, CUFFT_INVERSE));
            }
            finish_cplx_kernel<T, C><<<grid_for(npts), KT, 0, s>>>(y, spec, x, V, N, npts, inv_n);
            QSB_CUDA_TRY(cudaGetLastError());
            *launches += 3;
        }
    }
    return QSB_OK;
}

}  // namespace

qsb_status kinetic_fft_apply(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi, void* hpsi,
                             double gx, double gy, double gz, cudaStream_t s, int* launches) {
    if (dtype == QSB_F64)
        return apply_t<double>(h, dtype, is_complex, nb, (const double*)psi, (double*)hpsi, gx, gy, gz, s, launches);
    return apply_t<float>(h, dtype, is_complex, nb, (const float*)psi, (float*)hpsi, gx, gy, gz, s, launches);
}

void kinetic_fft_free(qsb_ham* h) {
    for (auto& p : h->fft_plans) {
        cufftDestroy((cufftHandle)p.forward);
        if (p.backward != p.forward) cufftDestroy((cufftHandle)p.backward);
    }
    h->fft_plans.clear();
    if (h->fft_buf) cudaFree(h->fft_buf);
    h->fft_buf = nullptr;
    h->fft_buf_bytes = 0;
}

}  // namespace qsb
