// qumasun_dropin.hpp — the reference's hot-path call surfaces, re-declared over
// the C ABI of include/qumasun_b200.h, so a reference-style caller keeps its
// call sites and passes device pointers.
//
// Include it after the caller's own declarations of GridRange / GridRangeMPI
// (anything with SizeX/SizeY/SizeZ), SoAComplex {double* re, *im} and OneComplex
// (source/GridRange.h:14-44, source/soacomplex.h:4-9): the adapters are
// templates on those types and declare none of them.
//
// Layout requirement of the C ABI (the reference's own WaveSet layout,
// source/qumasun_base1.h:457-460): a complex band's imaginary plane follows its
// real plane (im == re + N) and bands of a bundle are consecutive.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "qumasun_b200.h"

namespace qsb_dropin {

inline void check(qsb_status st) {
    if (st != QSB_OK) throw std::runtime_error(std::string("qumasun_b200: ") + qsb_last_error());
}

template <class T>
constexpr qsb_dtype dtype_of() {
    static_assert(sizeof(T) == 8 || sizeof(T) == 4, "double or float");
    return sizeof(T) == 8 ? QSB_F64 : QSB_F32;
}

// Laplacian8th<T>(grid, out, p, coef, dx, dy, dz)  (source/GridDifference8th.h:177-184):
// out += coef * FD8 Laplacian(p), one band, device pointers.
template <class T, class Grid>
void Laplacian8th(const Grid& grid, T* out, const T* p, double coef, double dx, double dy, double dz,
                  void* stream = nullptr) {
    check(qsb_laplacian8th(dtype_of<T>(), grid.SizeX(), grid.SizeY(), grid.SizeZ(), 1, out, p, coef, dx, dy, dz,
                           stream));
}

// LaplacianKpoint8th_ddm(grid, out, src, coef, dx, dy, dz, gx, gy, gz)
// (source/GridDifferenceKpoint8th.h:324-366), split_dimension 0, device pointers.
template <class Grid, class SoA>
void LaplacianKpoint8th_ddm(const Grid& grid, SoA& out, const SoA& src, double coef, double dx, double dy, double dz,
                            double gx, double gy, double gz, void* stream = nullptr) {
    const size_t N = (size_t)grid.SizeX() * grid.SizeY() * grid.SizeZ();
    if (out.im != out.re + N || src.im != src.re + N)
        throw std::invalid_argument("LaplacianKpoint8th_ddm: im plane must follow re plane (WaveSet layout)");
    check(qsb_laplacian_kpoint8th(QSB_F64, grid.SizeX(), grid.SizeY(), grid.SizeZ(), 1, out.re, src.re, coef, dx, dy,
                                  dz, gx, gy, gz, stream));
}

// mHamiltonianMatrix_ddm / ProjectionPP_bundle (source/qumasun_base1.matrix.h:263-291,
// source/PseudoPotNonlocal_SvF2_kpoint.h:4239-4247) on a bundle of complex bands.
class Hamiltonian {
public:
    template <class Grid>
    Hamiltonian(const Grid& grid, double dx, double dy, double dz)
        : N_((size_t)grid.SizeX() * grid.SizeY() * grid.SizeZ()) {
        check(qsb_ham_create(&h_, grid.SizeX(), grid.SizeY(), grid.SizeZ(), dx, dy, dz));
    }
    ~Hamiltonian() { qsb_ham_destroy(h_); }
    Hamiltonian(const Hamiltonian&) = delete;
    Hamiltonian& operator=(const Hamiltonian&) = delete;

    void SetPotential(const double* Vtot_dev) { check(qsb_ham_set_potential(h_, Vtot_dev, 1)); }
    // projector_RY-style tables: per atom point list (unfolded grid coords) + column-major values
    void SetProjectors(int n_atoms, const int* npts, const int* widths, const int* coords, const double* beta,
                       const double* energy) {
        check(qsb_ham_set_projectors(h_, n_atoms, npts, widths, coords, beta, energy));
    }
    // Hp = H p for num_bundle SoA bands (k-point vector g in bohr^-1)
    template <class SoA>
    void Apply(SoA* Hp, const SoA* p, int num_bundle, double gx, double gy, double gz, void* stream = nullptr) {
        if (num_bundle <= 0) return;
        if (Hp[0].im != Hp[0].re + N_ || p[0].im != p[0].re + N_)
            throw std::invalid_argument("Hamiltonian::Apply: im plane must follow re plane (WaveSet layout)");
        check(qsb_ham_apply(h_, QSB_F64, 1, num_bundle, p[0].re, Hp[0].re, gx, gy, gz, stream));
    }
    // Hp += V_NL p  (ProjectionPP_bundle)
    template <class SoA>
    void ProjectionPP_bundle(SoA* Hp, const SoA* p, int begin_n, int end_n, double gx, double gy, double gz,
                             void* stream = nullptr) {
        if (end_n <= begin_n) return;
        check(qsb_ham_nonlocal_apply(h_, QSB_F64, 1, end_n - begin_n, p[begin_n].re, Hp[begin_n].re, gx, gy, gz,
                                     stream));
    }
    // m_algorithm_Laplacian (source/qumasun_base1.h:243): 1 makes Apply the FFT
    // kinetic of mHamiltonianMatrix_ddm_bundle (source/qumasun_base1.matrix.h:171-228),
    // 0 the FD8 form of mHamiltonianMatrix_ddm
    void SetKineticAlgorithm(int algorithm) { check(qsb_ham_set_kinetic(h_, algorithm)); }
    // Apply on bundles in host memory (the reference's CPU build), chunked
    // through the device; complete when `stream` is
    template <class SoA>
    void ApplyHost(SoA* Hp, const SoA* p, int num_bundle, double gx, double gy, double gz, void* stream = nullptr,
                   int chunk_bands = 0) {
        if (num_bundle <= 0) return;
        if (Hp[0].im != Hp[0].re + N_ || p[0].im != p[0].re + N_)
            throw std::invalid_argument("Hamiltonian::ApplyHost: im plane must follow re plane (WaveSet layout)");
        check(qsb_ham_apply_host(h_, QSB_F64, 1, num_bundle, p[0].re, Hp[0].re, gx, gy, gz, chunk_bands, stream));
    }
    qsb_ham* handle() const { return h_; }

private:
    qsb_ham* h_ = nullptr;
    size_t N_;
};

// CubeWriter::SaveCube(filename, frame, num_nuclei, nuclei, field)
// (source/cube_writer.h:27-90): the same Frame (box edge vectors in boxaxis),
// any Nucleus type with Z, Rx, Ry, Rz; byte-identical files.  Returns 1 like
// the reference; failures (unwritable path) throw instead of crashing.
struct CubeWriter {
    struct Frame {
        int grid_x;
        int grid_y;
        int grid_z;
        double boxaxis[9];
        double boxorg[3];
        char comment[256]{0};
    };
    template <class Nucleus>
    static int SaveCube(const char* filename, const Frame& frame, int num_nuclei, const Nucleus* nuclei,
                        const double* field) {
        std::vector<int> Z(num_nuclei > 0 ? num_nuclei : 0);
        std::vector<double> pos(3 * Z.size());
        for (size_t a = 0; a < Z.size(); ++a) {
            Z[a] = nuclei[a].Z;
            pos[3 * a] = nuclei[a].Rx;
            pos[3 * a + 1] = nuclei[a].Ry;
            pos[3 * a + 2] = nuclei[a].Rz;
        }
        check(qsb_cube_write(filename, frame.comment, frame.grid_x, frame.grid_y, frame.grid_z, frame.boxaxis,
                             frame.boxorg, num_nuclei, Z.empty() ? nullptr : Z.data(),
                             pos.empty() ? nullptr : pos.data(), field));
        return 1;
    }
};

// CubeReader3 (source/cube_reader3.h:11-124): LoadCube reads header and values
// (boxaxis = grid count x voxel vector, as there), GetMeshData copies the
// values in the x-fastest grid layout.  Where the reference returns a zeroed
// frame or leaves a short file's tail unread, these throw.
class CubeReader3 {
public:
    struct Frame {
        int grid_x;
        int grid_y;
        int grid_z;
        double boxaxis[9];
        double boxorg[3];
        char comment[1024];
    };
    Frame LoadCube(const char* filename) {
        Frame f{};
        int grid[3];
        check(qsb_cube_read_header(filename, grid, f.boxaxis, f.boxorg, nullptr));
        f.grid_x = grid[0];
        f.grid_y = grid[1];
        f.grid_z = grid[2];
        if (std::FILE* fp = std::fopen(filename, "r")) {      // the comment line, kept with its newline as there
            char line[1024];
            if (std::fgets(line, sizeof line, fp) && std::fgets(line, sizeof line, fp))
                std::snprintf(f.comment, sizeof f.comment, "%s", line);
            std::fclose(fp);
        }
        values_.resize((size_t)grid[0] * grid[1] * grid[2]);
        check(qsb_cube_read(filename, values_.data(), nullptr, nullptr));
        return f;
    }
    void GetMeshData(double* dest) const { std::copy(values_.begin(), values_.end(), dest); }

private:
    std::vector<double> values_;
};

// LOBPCG::Eigen_z_multi_mpi(l_grid, dVol, num_solution, iter_max, eigen_values,
// eigen_vectors, keep, work, temporary, p_num_fix, residual_threshold,
// keep_S_matrix, SCF_step, sk, OpeA, watch)  (source/lobpcg_z_multi_mpi.h:1732-1742)
// on one rank.  `work` / `temporary` / keep_S_matrix / sk / watch are accepted
// for call-site compatibility; the device solver keeps its own work bundles in
// `solver`, created once per (N, num_solution).  OpeA(SoA* Ax, SoA* x, int n)
// receives device bundles.
class EigenSolverZ {
public:
    EigenSolverZ(int64_t N, int n) { check(qsb_eigensolver_create(&es_, N, n, 1)); }
    ~EigenSolverZ() { qsb_eigensolver_destroy(es_); }
    EigenSolverZ(const EigenSolverZ&) = delete;
    EigenSolverZ& operator=(const EigenSolverZ&) = delete;
    qsb_eigensolver* handle() const { return es_; }

private:
    qsb_eigensolver* es_ = nullptr;
};

template <class SoA, class OperationA>
struct OpeABridge {
    OperationA* op;
    size_t N;
    static int call(void* user, int nb, const double* x, double* ax, void*) {
        auto* self = static_cast<OpeABridge*>(user);
        std::vector<SoA> X(nb), AX(nb);
        for (int k = 0; k < nb; ++k) {
            X[k].re = const_cast<double*>(x) + 2 * k * self->N;
            X[k].im = X[k].re + self->N;
            AX[k].re = ax + 2 * k * self->N;
            AX[k].im = AX[k].re + self->N;
        }
        try {
            (*self->op)(AX.data(), X.data(), nb);
        } catch (...) {
            return QSB_ERR_STATE;
        }
        return 0;
    }
};

template <class Grid, class SoA, class Complex, class OperationA, class WATCH>
void Eigen_z_multi_mpi(EigenSolverZ& solver, const Grid& l_grid, double dVol, int num_solution, int iter_max,
                       double* eigen_values, SoA* eigen_vectors, double* keep, double* /*work*/,
                       double* /*temporary*/, int* p_num_fix, double residual_threshold, Complex* /*keep_S_matrix*/,
                       int SCF_step, int /*sk*/, OperationA OpeA, WATCH& /*watch*/, void* stream = nullptr) {
    const size_t N = (size_t)l_grid.SizeX() * l_grid.SizeY() * l_grid.SizeZ();
    OpeABridge<SoA, OperationA> bridge{&OpeA, N};
    check(qsb_eigensolver_set_operator(solver.handle(), &OpeABridge<SoA, OperationA>::call, &bridge));
    check(qsb_lobpcg_z(solver.handle(), dVol, num_solution, iter_max, eigen_values, eigen_vectors[0].re, keep,
                       p_num_fix, residual_threshold, SCF_step, stream));
}

// EigenLOBPCG_d_multi(N, dVol, num_solution, iter_max, eigen_values,
// eigen_vectors, keep, work, is_first_time, OpeA, watch) (source/lobpcg_d_multi.h:23-27).
// OpeA(double* Ax, const double* x) is called per band on device vectors.
template <class OperationA>
struct OpeADBridge {
    OperationA* op;
    size_t N;
    static int call(void* user, int nb, const double* x, double* ax, void*) {
        auto* self = static_cast<OpeADBridge*>(user);
        try {
            for (int k = 0; k < nb; ++k) (*self->op)(ax + k * self->N, x + k * self->N);
        } catch (...) {
            return QSB_ERR_STATE;
        }
        return 0;
    }
};

template <class OperationA, class WATCH>
void EigenLOBPCG_d_multi(qsb_eigensolver* solver, const int N, const double dVol, const int num_solution,
                         const int iter_max, double* eigen_values, double* eigen_vectors, double* keep,
                         double* /*work*/, bool is_first_time, OperationA OpeA, WATCH& /*watch*/,
                         void* stream = nullptr) {
    OpeADBridge<OperationA> bridge{&OpeA, (size_t)N};
    check(qsb_eigensolver_set_operator(solver, &OpeADBridge<OperationA>::call, &bridge));
    check(qsb_lobpcg_d(solver, dVol, num_solution, iter_max, eigen_values, eigen_vectors, keep, is_first_time ? 1 : 0,
                       stream));
}

}  // namespace qsb_dropin
