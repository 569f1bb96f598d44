/*
 * oracle/ref_fft.cpp -- extern "C" entries around the REFERENCE's own
 * QUMASUN_BASE1 object (its FFT-kinetic Hamiltonian, its GGA-PBE
 * exchange-correlation and its Hartree potential), compiled in place from the reference's source/
 * directory (never copied) into oracle/_ref/libqsref_fft.so.  Test
 * infrastructure only.
 *
 * What runs is QUMASUN_BASE1::mHamiltonianMatrix_ddm_bundle, algorithm 1
 * (source/qumasun_base1.matrix.h:142-228): the SoA bands gathered into
 * interleaved complex fields (DDMGatherScatter::GatherExchangeD2Z), the
 * FFTW_ExecutorMany3D forward transform (source/fftw_executor.h:359-425), the
 * k-space multiply QUMASUN::OperateKineticInKspace_bundle (:96-123), the
 * backward transform, the 1/N scaling, the scatter back
 * (ScatterExchangeZ2D) and mPotentialMatrixAdd_ddm_bundle (V psi).  The object
 * is the reference's own QUMASUN_BASE1, built by its own constructor from an
 * Input with no nuclei, on one rank (oracle/ref_shim/mpi.h).
 *
 * Two stand-ins make it build here:
 *   - FFTW 3 is not installed: oracle/ref_shim/fftw3.h + fftw_dft.cpp restate
 *     FFTW's documented DFT (direct sums, long double twiddles);
 *   - IGNORE_NONLOCAL (the reference's own switch, matrix.h:231) leaves out the
 *     SvF2 nonlocal part, which this entry does not exercise (no nuclei).
 * k enters as the reference takes it: integer k-point indices times
 * dk = 2 pi / (L * kpoint_sample) per axis (qumasun_base1.constructor.h:34-36).
 */
#include <mpi.h>
#include "mpi_helper.h"
#include "qumasun_base1.h"

#include <cstring>
#include <vector>

namespace {

class RefFFTHamiltonian : public QUMASUN_BASE1 {
public:
    RefFFTHamiltonian(const Input& input, const int ddm[4]) : QUMASUN_BASE1(input, MPI_COMM_WORLD, ddm) {}

    // the reference's spin-unpolarised GGA branch of mSetPotentialVxc on a given density
    void GgaPbe(const double* rho, double* vxc, double* e_x, double* e_c) {
        const size_t N = (size_t)m_size_3d;
        mInitializeWorkBuffer(16 * N + 64);
        for (size_t i = 0; i < N; ++i) {
            ml_rho[i] = rho[i];
            ml_pcc_rho[i] = 0.0;
        }
        mSetPotentialVxc();
        for (size_t i = 0; i < N; ++i) vxc[i] = ml_Vx[i] + ml_Vc[i];
        *e_x = m_E_x;
        *e_c = m_E_c;
    }

    // the reference's Hartree potential of a density (mSetPotentialVhart)
    void Hartree(const double* rho, double* vh) {
        const size_t N = (size_t)m_size_3d;
        const size_t hr = (size_t)m_HR_ratio_x * m_HR_ratio_y * m_HR_ratio_z;
        mInitializeWorkBuffer(16 * N * hr + 64);
        for (size_t i = 0; i < N; ++i) ml_rho[i] = rho[i];
        mSetPotentialVhart();
        for (size_t i = 0; i < N; ++i) vh[i] = ml_Vhart[i];
    }

    // H psi of nb SoA bands (band b: re at 2bN, im at (2b+1)N)
    void Apply(const double* V, int nb, const double* psi, double* hpsi, int kx, int ky, int kz) {
        const size_t N = (size_t)m_size_3d;
        mInitializeWorkBuffer(4 * N * (size_t)nb + 64);
        std::vector<SoAComplex> phi(nb), hp(nb);
        for (int b = 0; b < nb; ++b) {
            phi[b].re = const_cast<double*>(psi) + 2 * (size_t)b * N;
            phi[b].im = phi[b].re + N;
            hp[b].re = hpsi + 2 * (size_t)b * N;
            hp[b].im = hp[b].re + N;
        }
        mHamiltonianMatrix_ddm_bundle(hp.data(), V, phi.data(), nb, kx, ky, kz, 0);
    }
};

}  // namespace

extern "C" {

/* H psi = -1/2 (grad + i k)^2 psi + V psi on an nx x ny x nz periodic box of
 * side lengths (lx, ly, lz), k_d = kidx[d] * 2 pi / (L_d * ksample[d]).
 * psi and hpsi: nb complex SoA bands, 2 * nb * nx * ny * nz doubles. */
int qsref_ham_fft(int nx, int ny, int nz, double lx, double ly, double lz, const int* ksample, const int* kidx,
                  const double* V, int nb, const double* psi, double* hpsi) {
    if (nx < 1 || ny < 1 || nz < 1 || nb < 1 || !psi || !hpsi || !V) return 1;
    QUMASUN::Input in{};
    in.hamiltonian_type = QUMASUN::HAMILTONIAN::KohnSham_PP;
    in.grid_size[0] = nx;
    in.grid_size[1] = ny;
    in.grid_size[2] = nz;
    std::memset(in.box_axis, 0, sizeof(in.box_axis));
    in.box_axis[0] = lx;
    in.box_axis[4] = ly;
    in.box_axis[8] = lz;
    in.num_solutions = nb;
    in.num_electrons = 0;
    in.num_nuclei = 0;
    in.HR_ratio = 1;
    for (int d = 0; d < 3; ++d) in.kpoint_sample[d] = ksample ? ksample[d] : 1;
    in.test_algorithm_Laplacian = 1;
    const int ddm[4] = {1, 1, 1, 1};
    RefFFTHamiltonian H(in, ddm);
    H.Apply(V, nb, psi, hpsi, kidx ? kidx[0] : 0, kidx ? kidx[1] : 0, kidx ? kidx[2] : 0);
    return 0;
}

/* The reference's GGA-PBE exchange-correlation (XC_TYPE::GGA, spin off) of a
 * density rho on an nx x ny x nz periodic box of sides (lx, ly, lz):
 * vxc = V_x + V_c (N doubles), e_xc[0] = E_x, e_xc[1] = E_c (QUMASUN_BASE1::
 * mSetPotentialVxc, source/qumasun_base1.potential.h:376-640). */
int qsref_gga_pbe(int nx, int ny, int nz, double lx, double ly, double lz, const double* rho, double* vxc,
                  double* e_xc) {
    if (nx < 1 || ny < 1 || nz < 1 || !rho || !vxc || !e_xc) return 1;
    QUMASUN::Input in{};
    in.hamiltonian_type = QUMASUN::HAMILTONIAN::KohnSham_PP;
    in.xc_type = QUMASUN::XC_TYPE::GGA;
    in.grid_size[0] = nx;
    in.grid_size[1] = ny;
    in.grid_size[2] = nz;
    std::memset(in.box_axis, 0, sizeof(in.box_axis));
    in.box_axis[0] = lx;
    in.box_axis[4] = ly;
    in.box_axis[8] = lz;
    in.num_solutions = 1;
    in.num_nuclei = 0;
    in.HR_ratio = 1;
    in.test_algorithm_Laplacian = 1;
    const int ddm[4] = {1, 1, 1, 1};
    RefFFTHamiltonian H(in, ddm);
    H.GgaPbe(rho, vxc, &e_xc[0], &e_xc[1]);
    return 0;
}

/* The reference's Hartree potential V_H of rho (QUMASUN_BASE1::mSetPotentialVhart,
 * source/qumasun_base1.potential.h:32-100: the Poisson solve of
 * mPoissonDDMFFT_Upconvert on the high-resolution grid, then DownConvert_Realspace),
 * on an nx x ny x nz box of sides (lx, ly, lz) with the high-resolution ratio hr. */
int qsref_hartree(int nx, int ny, int nz, double lx, double ly, double lz, int hr, const double* rho, double* vh) {
    if (nx < 1 || ny < 1 || nz < 1 || hr < 1 || !rho || !vh) return 1;
    QUMASUN::Input in{};
    in.hamiltonian_type = QUMASUN::HAMILTONIAN::KohnSham_PP;
    in.grid_size[0] = nx;
    in.grid_size[1] = ny;
    in.grid_size[2] = nz;
    std::memset(in.box_axis, 0, sizeof(in.box_axis));
    in.box_axis[0] = lx;
    in.box_axis[4] = ly;
    in.box_axis[8] = lz;
    in.num_solutions = 1;
    in.num_nuclei = 0;
    in.HR_ratio = hr;
    in.test_algorithm_Laplacian = 1;
    const int ddm[4] = {1, 1, 1, 1};
    RefFFTHamiltonian H(in, ddm);
    H.Hartree(rho, vh);
    return 0;
}

}  // extern "C"
