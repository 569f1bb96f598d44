// qsb_orthonormalize: dV-weighted orthonormalisation of a band bundle in place,
// the role of GramSchmidt_ddm (source/GramSchmidt_mpi.h:56-96) before an SCF.
//
// The reference runs classical Gram-Schmidt band after band (nb sequential
// passes of inner products and updates over the grid).  On the device the same
// factorisation is formed as Cholesky QR, twice ("CholQR2"): G = dV X^H X on the
// tensor path of cuBLAS, G = U^H U (potrf), X <- X U^-1 (trsm, in place).  Both
// produce the Q factor of X = Q R with a positive diagonal R, which is unique,
// so the results agree to rounding for inputs that are not near rank-deficient;
// the second pass brings the orthogonality of the first (~cond(X)^2 eps) down to
// ~eps.  Complex SoA bundles (re plane, im plane per band) are packed into
// interleaved columns for the complex trsm and unpacked after.
#include "qsb_internal.h"

#include <cublas_v2.h>
#include <cusolverDn.h>
#include <cuComplex.h>
#include <algorithm>
#include <string>
#include <vector>

namespace {

// Hermitian Gram of a complex SoA bundle from its 2n-real view T = Xr^T Xr
// (2n x 2n, ld 2n): G_jk = <x_j|x_k> dV = (re_j.re_k + im_j.im_k) + i (re_j.im_k - im_j.re_k)
__global__ void hermitian_from_real_view(const double* __restrict__ T, int n, double dV, cuDoubleComplex* __restrict__ G) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j >= n) return;
    const int ld = 2 * n;
    const double rr = T[(2 * j) + (size_t)ld * (2 * k)], ii = T[(2 * j + 1) + (size_t)ld * (2 * k + 1)];
    const double ri = T[(2 * j) + (size_t)ld * (2 * k + 1)], ir = T[(2 * j + 1) + (size_t)ld * (2 * k)];
    G[j + (size_t)n * k] = make_cuDoubleComplex((rr + ii) * dV, (ri - ir) * dV);
}

// SoA bundle (band b: re at 2bN, im at (2b+1)N) <-> interleaved columns Z (N x n)
__global__ void soa_to_interleaved(const double* __restrict__ X, size_t N, int n, cuDoubleComplex* __restrict__ Z) {
    const int b = blockIdx.y;
    const double* re = X + (size_t)2 * b * N;
    const double* im = re + N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        Z[(size_t)b * N + i] = make_cuDoubleComplex(re[i], im[i]);
}
__global__ void interleaved_to_soa(const cuDoubleComplex* __restrict__ Z, size_t N, int n, double* __restrict__ X) {
    const int b = blockIdx.y;
    double* re = X + (size_t)2 * b * N;
    double* im = re + N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const cuDoubleComplex z = Z[(size_t)b * N + i];
        re[i] = z.x;
        im[i] = z.y;
    }
}

// d[k] = |U_kk| of the Cholesky factor (real, or complex with ld n)
__global__ void factor_diagonal(const double* __restrict__ U, int n, int cplx, double* __restrict__ d) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) d[k] = fabs(cplx ? U[2 * ((size_t)k + (size_t)n * k)] : U[(size_t)k + (size_t)n * k]);
}

struct Handles {
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t sol = nullptr;
    void* mem = nullptr;
    ~Handles() {
        if (mem) cudaFree(mem);
        if (blas) cublasDestroy(blas);
        if (sol) cusolverDnDestroy(sol);
    }
};

#define ORTH_BLAS(expr)                                                                               \
    do {                                                                                              \
        if ((expr) != CUBLAS_STATUS_SUCCESS) return qsb::fail(QSB_ERR_CUDA, "orthonormalize: " #expr); \
    } while (0)
#define ORTH_SOLVER(expr)                                                                               \
    do {                                                                                                \
        if ((expr) != CUSOLVER_STATUS_SUCCESS) return qsb::fail(QSB_ERR_CUDA, "orthonormalize: " #expr); \
    } while (0)

}  // namespace

extern "C" qsb_status qsb_orthonormalize(int64_t N, int nb, int is_complex, double* X, double dV, void* stream) {
    if (N < 1 || nb < 1 || !X || !(dV > 0.0)) return qsb::fail(QSB_ERR_INVALID, "orthonormalize: bad arguments");
    if (nb > N) return qsb::fail(QSB_ERR_INVALID, "orthonormalize: more bands than grid points");
    if (N > 0x7fffffffLL) return qsb::fail(QSB_ERR_INVALID, "orthonormalize: grid too large for the BLAS calls");
    cudaStream_t s = (cudaStream_t)stream;
    Handles h;
    if (cublasCreate(&h.blas) != CUBLAS_STATUS_SUCCESS) return qsb::fail(QSB_ERR_CUDA, "orthonormalize: cublasCreate");
    if (cusolverDnCreate(&h.sol) != CUSOLVER_STATUS_SUCCESS)
        return qsb::fail(QSB_ERR_CUDA, "orthonormalize: cusolverDnCreate");
    ORTH_BLAS(cublasSetStream(h.blas, s));
    ORTH_SOLVER(cusolverDnSetStream(h.sol, s));
    const int n = nb;
    const int ni = (int)N;
    // workspace: T (2n x 2n real view Gram), G (n x n complex), info, potrf work, interleaved bundle (complex)
    const size_t t_doubles = (size_t)(2 * n) * (2 * n);
    const size_t g_doubles = (size_t)2 * n * n;
    int lwork = 0;
    if (is_complex)
        ORTH_SOLVER(cusolverDnZpotrf_bufferSize(h.sol, CUBLAS_FILL_MODE_UPPER, n, nullptr, n, &lwork));
    else
        ORTH_SOLVER(cusolverDnDpotrf_bufferSize(h.sol, CUBLAS_FILL_MODE_UPPER, n, nullptr, n, &lwork));
    const size_t w_doubles = (size_t)lwork * (is_complex ? 2 : 1) + 2 + n;
    const size_t z_doubles = is_complex ? (size_t)2 * N * n : 0;
    QSB_CUDA_TRY(cudaMalloc(&h.mem, sizeof(double) * (t_doubles + g_doubles + w_doubles + z_doubles) + 64));
    double* T = (double*)h.mem;
    double* G = T + t_doubles;
    double* W = G + g_doubles;
    int* info = (int*)(W + w_doubles - 2 - n);
    double* diag = W + w_doubles - n;
    std::vector<double> hdiag(n);
    cuDoubleComplex* Z = (cuDoubleComplex*)(W + w_doubles);
    const double one = 1.0, zero = 0.0;
    const dim3 pgrid((unsigned)std::min<int64_t>((N + 255) / 256, 1024), n);
    for (int pass = 0; pass < 2; ++pass) {
        if (is_complex) {
            // T = Xr^T Xr over the 2n-real view (N x 2n, ld N)
            ORTH_BLAS(cublasDgemm(h.blas, CUBLAS_OP_T, CUBLAS_OP_N, 2 * n, 2 * n, ni, &one, X, ni, X, ni, &zero, T, 2 * n));
            hermitian_from_real_view<<<dim3((n + 127) / 128, n), 128, 0, s>>>(T, n, dV, (cuDoubleComplex*)G);
            QSB_CUDA_TRY(cudaGetLastError());
            ORTH_SOLVER(cusolverDnZpotrf(h.sol, CUBLAS_FILL_MODE_UPPER, n, (cuDoubleComplex*)G, n,
                                         (cuDoubleComplex*)W, lwork, info));
        } else {
            ORTH_BLAS(cublasDgemm(h.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, ni, &dV, X, ni, X, ni, &zero, G, n));
            ORTH_SOLVER(cusolverDnDpotrf(h.sol, CUBLAS_FILL_MODE_UPPER, n, G, n, W, lwork, info));
        }
        int hinfo = 0;
        factor_diagonal<<<(n + 127) / 128, 128, 0, s>>>(G, n, is_complex ? 1 : 0, diag);
        QSB_CUDA_TRY(cudaGetLastError());
        QSB_CUDA_TRY(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
        QSB_CUDA_TRY(cudaMemcpyAsync(hdiag.data(), diag, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        QSB_CUDA_TRY(cudaStreamSynchronize(s));
        // a pivot below 1e-7 of the largest: a direction below ~1e-14 of the
        // overlap's scale, which the classical Gram-Schmidt of the reference
        // would also turn into noise
        double dmax = 0.0, dmin = 1e300;
        for (double v : hdiag) {
            dmax = std::max(dmax, v);
            dmin = std::min(dmin, v);
        }
        if (hinfo != 0 || !(dmin > 1e-7 * dmax))
            return qsb::fail(QSB_ERR_NUMERIC, "orthonormalize: the bands are linearly dependent (Cholesky info " +
                                                  std::to_string(hinfo) + ", smallest pivot " + std::to_string(dmin) +
                                                  " of " + std::to_string(dmax) + ")");
        // X <- X U^-1
        if (is_complex) {
            soa_to_interleaved<<<pgrid, 256, 0, s>>>(X, (size_t)N, n, Z);
            QSB_CUDA_TRY(cudaGetLastError());
            const cuDoubleComplex zone = make_cuDoubleComplex(1.0, 0.0);
            ORTH_BLAS(cublasZtrsm(h.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, ni,
                                  n, &zone, (const cuDoubleComplex*)G, n, Z, ni));
            interleaved_to_soa<<<pgrid, 256, 0, s>>>(Z, (size_t)N, n, X);
            QSB_CUDA_TRY(cudaGetLastError());
        } else {
            ORTH_BLAS(cublasDtrsm(h.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, ni,
                                  n, &one, G, n, X, ni));
        }
    }
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    return QSB_OK;
}
