/*
 * oracle/ref_entry.cpp — extern "C" entry points around the REFERENCE's own
 * hot-path templates, compiled from the reference source tree (never copied)
 * into oracle/_ref/libqsref.so by oracle/Makefile.
 *
 * TEST INFRASTRUCTURE ONLY.  The product never links or loads this library;
 * tests, the golden-fixture generator and bench.py's CPU reference arm do.
 *
 * What each entry point runs (paths relative to the reference's source/):
 *   qsref_laplacian8th        Laplacian8th<double>          GridDifference8th.h:177-184
 *   qsref_laplacian_kpoint8th LaplacianKpoint8th_halo<K..>  GridDifferenceKpoint8th.h:123-151
 *                             (dispatch on |g|<1e-8 as LaplacianKpoint8th_ddm does,
 *                              GridDifferenceKpoint8th.h:330-364, with per-call
 *                              halo buffers instead of its first-call statics)
 *   qsref_overlap_blocks      GetOverlapPeriodic            GridSubgrid.h:690-740
 *   qsref_nonlocal_apply      ProjectionPP_bundle_1's order of operations
 *                             (PseudoPotNonlocal_SvF2_kpoint.h:3911-4046 and
 *                              mInnerNonlocalPsi_v4_bundle :4463-4576) built from the
 *                              reference's CutSubgridByRanges / AddSubgridByRanges
 *                              (GridSubgrid.h:742,751) and blas_DGEMM_t/_n (w_dgemm.h)
 *   qsref_nonlocal_energy_force  EnergyPPnonlocal_bundle / ForceNonlocal_bundle (grad(p) form)
 *                             (PseudoPotNonlocal_SvF2_kpoint.h:5033-5135, :3629-3731)
 *   qsref_hamiltonian         mHamiltonianMatrix_ddm composition
 *                             (qumasun_base1.matrix.h:263-317): H = V.psi + NL + FD8(-1/2)
 *   qsref_lobpcg_d            EigenLOBPCG_d_multi           lobpcg_d_multi.h:23-545
 *   qsref_lobpcg_z            LOBPCG::Eigen_z_multi_mpi     lobpcg_z_multi_mpi.h:1732-2852
 *   qsref_lda_pz              Calc_XC_LDA (Perdew-Zunger)   Vxc.h:43-75
 *   qsref_set_occupancy       SetOccupancy (Fermi-Dirac)    SetOccupancy.h:7-18
 *   qsref_cube_write          CubeWriter::SaveCube          cube_writer.h:27-90
 *   qsref_cube_read           CubeReader3::LoadCube + GetMeshData  cube_reader3.h:38-124
 *   qsref_upf_load            LoadUPF_ONCV                  upf_oncv_loader.h:353-1050
 *
 * The nonlocal class itself (projector construction from UPF via SvF) is not
 * compiled: the projector values are supplied by the caller on the block
 * layout that GetOverlapPeriodic produces, exactly the layout of
 * PP_Proj_Ylm_each_atom::projector_RY (column-major, grid_sizes x width).
 */
#include <vector>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <algorithm>
#include <map>

#include "debug_print.h"
/* w_dsygvx.h's lapack_DSYGVX_mpi_split names lapack_DSYGVX_range before the
 * LAPACKE branch of that header declares it; it is never called here. */
int lapack_DSYGVX_range(double*, double*, double*, double*, int, int, int);
#include "GridDifference8th.h"
#include "GridDifferenceKpoint8th.h"
#include "GridSubgrid.h"
#include "w_dgemm.h"

/* lobpcg_d_multi.h calls an 8-argument lapack_DSYGVX (with a triangle-factor
 * scratch array) that w_dsygvx.h no longer defines; this overload forwards to
 * the 7-argument one and ignores the scratch, so the reference template
 * instantiates unchanged. */
#include "w_dsygvx.h"
inline int lapack_DSYGVX(double* A, double* B, double* w, double* Z, double* /*triangle_factors*/, int N, int il, int iu) {
    return lapack_DSYGVX(A, B, w, Z, N, il, iu);
}
#include "vecmath.h"
#include "lobpcg_d_multi.h"
#ifdef QSREF_WITH_Z
#include "lobpcg_z_multi_mpi.h"
#include "Vxc.h"
#include "SetOccupancy.h"
#include "GramSchmidt_mpi.h"
#endif
#include "cube_reader3.h"
#include "cube_writer.h"
#include "upf_oncv_loader.h"

namespace {

struct NullWatch {
    void Record(int) {}
    void Record(int, int) {}
    void Restart() {}
};

GridRangeMPI make_grid(int nx, int ny, int nz) {
    GridRangeMPI g{};
    g.begin_x = 0; g.begin_y = 0; g.begin_z = 0;
    g.end_x = nx; g.end_y = ny; g.end_z = nz;
    g.mpi_comm = MPI_COMM_WORLD;
    g.split_dimension = 0;
    g.num_split_x = g.num_split_y = g.num_split_z = 1;
    return g;
}

/* One atom's projector data on the reference block layout. */
struct RefAtom {
    std::vector<GridRange> ranges;
    std::vector<ShiftedGrid> shifts;
    int grid_size = 0;
    int width = 0;
    const double* proj = nullptr;     /* grid_size x width, column-major */
    const double* energy = nullptr;   /* width */
};

struct RefNonlocal {
    std::vector<RefAtom> atoms;
};

/* Bloch factor exp(i k.r) on the block layout, as mCreateBlochExp builds it
 * (PseudoPotNonlocal_SvF2_kpoint.h:3538-3605): r is the unfolded grid
 * coordinate (folded range minus the periodic shift). */
void bloch_exp(const RefAtom& a, double gx_dx, double gy_dy, double gz_dz, std::vector<double>& re, std::vector<double>& im) {
    re.assign(a.grid_size, 0.0);
    im.assign(a.grid_size, 0.0);
    int offset_i = 0;
    for (size_t ib = 0; ib < a.ranges.size(); ++ib) {
        const int ix_begin = a.ranges[ib].begin_x - a.shifts[ib].x;
        const int iy_begin = a.ranges[ib].begin_y - a.shifts[ib].y;
        const int iz_begin = a.ranges[ib].begin_z - a.shifts[ib].z;
        const int ix_end = a.ranges[ib].end_x - a.shifts[ib].x;
        const int iy_end = a.ranges[ib].end_y - a.shifts[ib].y;
        const int iz_end = a.ranges[ib].end_z - a.shifts[ib].z;
        const int size_x = ix_end - ix_begin;
        const int size_y = iy_end - iy_begin;
        for (int iz = iz_begin; iz < iz_end; ++iz) {
            const double kzz = gz_dz * (double)iz;
            for (int iy = iy_begin; iy < iy_end; ++iy) {
                const double kyy = gy_dy * (double)iy;
                for (int ix = ix_begin; ix < ix_end; ++ix) {
                    const double kxx = gx_dx * (double)ix;
                    const int i = offset_i + (ix - ix_begin) + size_x * ((iy - iy_begin) + size_y * (iz - iz_begin));
                    re[i] = cos(kxx + kyy + kzz);
                    im[i] = sin(kxx + kyy + kzz);
                }
            }
        }
        offset_i += (int)a.ranges[ib].Size3D();
    }
}

/* Hp += V_NL psi for a bundle of complex bands (SoA), following
 * ProjectionPP_bundle_1 + mInnerNonlocalPsi_v4_bundle step by step. */
void nonlocal_apply_bundle(const RefNonlocal& nl, const GridRange& grid, int num_bundle,
                           double* const* hp_re, double* const* hp_im,
                           const double* const* psi_re, const double* const* psi_im,
                           double dV, double gx_dx, double gy_dy, double gz_dz) {
    const bool is_gamma = (gx_dx == 0.0) && (gy_dy == 0.0) && (gz_dz == 0.0);
    for (const RefAtom& a : nl.atoms) {
        if (a.width == 0 || a.grid_size == 0) continue;
        const int grid_size = a.grid_size;
        std::vector<double> cut((size_t)grid_size * 2 * num_bundle);
        std::vector<double> l_inner((size_t)a.width * 2 * num_bundle);
        for (int n = 0; n < num_bundle; ++n) {
            CutSubgridByRanges(a.ranges, cut.data() + (size_t)grid_size * 2 * n, grid, psi_re[n]);
            CutSubgridByRanges(a.ranges, cut.data() + (size_t)grid_size * (2 * n + 1), grid, psi_im[n]);
        }
        std::vector<double> ere, eim;
        if (!is_gamma) {
            bloch_exp(a, gx_dx, gy_dy, gz_dz, ere, eim);
            for (int n = 0; n < num_bundle; ++n) {
                double* pr = cut.data() + (size_t)grid_size * 2 * n;
                double* pi = cut.data() + (size_t)grid_size * (2 * n + 1);
                for (int i = 0; i < grid_size; ++i) {
                    const double p_re = pr[i], p_im = pi[i];
                    pr[i] = ere[i] * p_re - eim[i] * p_im;
                    pi[i] = ere[i] * p_im + eim[i] * p_re;
                }
            }
        }
        /* <p|psi> dV : PseudoPotNonlocal_SvF2_kpoint.h:4528 */
        blas_DGEMM_t(a.width, 2 * num_bundle, grid_size, a.proj, cut.data(), l_inner.data(), a.width, dV, 0.0);
        /* c = E_w <p|psi> : :4003-4011 */
        for (int n = 0; n < num_bundle * 2; ++n)
            for (int w = 0; w < a.width; ++w)
                l_inner[(size_t)a.width * n + w] *= a.energy[w];
        /* |p> c : :4017 */
        blas_DGEMM_n(grid_size, 2 * num_bundle, a.width, a.proj, l_inner.data(), cut.data(), grid_size, 1.0, 0.0);
        if (!is_gamma) {
            for (int n = 0; n < num_bundle; ++n) {
                double* pr = cut.data() + (size_t)grid_size * 2 * n;
                double* pi = cut.data() + (size_t)grid_size * (2 * n + 1);
                for (int i = 0; i < grid_size; ++i) {
                    const double p_re = pr[i], p_im = pi[i];
                    pr[i] = ere[i] * p_re + eim[i] * p_im;
                    pi[i] = ere[i] * p_im - eim[i] * p_re;
                }
            }
        }
        for (int n = 0; n < num_bundle; ++n) {
            AddSubgridByRanges(grid, hp_re[n], a.ranges, cut.data() + (size_t)grid_size * 2 * n);
            AddSubgridByRanges(grid, hp_im[n], a.ranges, cut.data() + (size_t)grid_size * (2 * n + 1));
        }
    }
}

/* Same for real bands: the imaginary column of each band is zero, which is
 * how the reference's complex path treats a Gamma-point real state. */
void nonlocal_apply_real(const RefNonlocal& nl, const GridRange& grid, double* hp, const double* psi, double dV) {
    for (const RefAtom& a : nl.atoms) {
        if (a.width == 0 || a.grid_size == 0) continue;
        const int grid_size = a.grid_size;
        std::vector<double> cut(grid_size);
        std::vector<double> l_inner(a.width);
        CutSubgridByRanges(a.ranges, cut.data(), grid, psi);
        blas_DGEMM_t(a.width, 1, grid_size, a.proj, cut.data(), l_inner.data(), a.width, dV, 0.0);
        for (int w = 0; w < a.width; ++w) l_inner[w] *= a.energy[w];
        blas_DGEMM_n(grid_size, 1, a.width, a.proj, l_inner.data(), cut.data(), grid_size, 1.0, 0.0);
        AddSubgridByRanges(grid, hp, a.ranges, cut.data());
    }
}

RefNonlocal build_nonlocal(int nx, int ny, int nz, int n_atoms, const int* cubes, const int* widths,
                           const double* proj, const double* energy) {
    RefNonlocal nl;
    GridRange grid = MakeRange(nx, ny, nz);
    size_t proj_off = 0, e_off = 0;
    for (int a = 0; a < n_atoms; ++a) {
        RefAtom at;
        GridRange cube{cubes[6 * a + 0], cubes[6 * a + 1], cubes[6 * a + 2], cubes[6 * a + 3], cubes[6 * a + 4], cubes[6 * a + 5]};
        at.grid_size = GetOverlapPeriodic(grid, cube, nx, ny, nz, at.ranges, at.shifts);
        at.width = widths[a];
        at.proj = proj + proj_off;
        at.energy = energy + e_off;
        proj_off += (size_t)at.grid_size * at.width;
        e_off += at.width;
        nl.atoms.push_back(std::move(at));
    }
    return nl;
}

struct RefHamiltonian {
    int nx, ny, nz;
    double dx, dy, dz;
    const double* V;
    RefNonlocal nl;
    double gx, gy, gz;
};

/* mHamiltonianMatrix_ddm (qumasun_base1.matrix.h:263-291) for one real band:
 * Hp = 0; Hp = V p; Hp += NL p; Hp += FD8 Laplacian with coef -1/2. */
void apply_h_real(const RefHamiltonian& H, double* hp, const double* p) {
    GridRange grid = MakeRange(H.nx, H.ny, H.nz);
    const size_t n = grid.Size3D();
    for (size_t i = 0; i < n; ++i) hp[i] = H.V[i] * p[i];
    nonlocal_apply_real(H.nl, grid, hp, p, H.dx * H.dy * H.dz);
    Laplacian8th<double>(grid, hp, p, -0.5, H.dx, H.dy, H.dz);
}

template <int KX, int KY, int KZ>
void kpoint_call(const GridRange& grid, SoAComplex& out, const SoAComplex& src, double* re_h, double* im_h,
                 double coef, double dx, double dy, double dz, double gx, double gy, double gz) {
    LaplacianKpoint8th_halo<KX, KY, KZ>(grid, out, src, re_h, im_h, coef, dx, dy, dz, gx, gy, gz);
}

void kpoint_dispatch(const GridRange& grid, SoAComplex& out, const SoAComplex& src, double coef,
                     double dx, double dy, double dz, double gx, double gy, double gz) {
    const size_t over = (size_t)(grid.SizeX() + 8) * (grid.SizeY() + 8) * (grid.SizeZ() + 8);
    std::vector<double> re_h(over), im_h(over);
    constexpr double th = 1.0e-8;
    const int kx = fabs(gx) < th ? 0 : 1, ky = fabs(gy) < th ? 0 : 1, kz = fabs(gz) < th ? 0 : 1;
    const int sel = kx * 4 + ky * 2 + kz;
    switch (sel) {
    case 0: kpoint_call<0, 0, 0>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 1: kpoint_call<0, 0, 1>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 2: kpoint_call<0, 1, 0>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 3: kpoint_call<0, 1, 1>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 4: kpoint_call<1, 0, 0>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 5: kpoint_call<1, 0, 1>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    case 6: kpoint_call<1, 1, 0>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    default: kpoint_call<1, 1, 1>(grid, out, src, re_h.data(), im_h.data(), coef, dx, dy, dz, gx, gy, gz); break;
    }
}

/* mHamiltonianMatrix_ddm for a bundle of complex SoA bands at k = (gx,gy,gz). */
void apply_h_complex(const RefHamiltonian& H, SoAComplex* hp, const SoAComplex* p, int nb) {
    GridRange grid = MakeRange(H.nx, H.ny, H.nz);
    const size_t n = grid.Size3D();
    std::vector<double*> hr(nb), hi(nb);
    std::vector<const double*> pr(nb), pi(nb);
    for (int b = 0; b < nb; ++b) {
        for (size_t i = 0; i < n; ++i) { hp[b].re[i] = H.V[i] * p[b].re[i]; hp[b].im[i] = H.V[i] * p[b].im[i]; }
        hr[b] = hp[b].re; hi[b] = hp[b].im; pr[b] = p[b].re; pi[b] = p[b].im;
    }
    nonlocal_apply_bundle(H.nl, grid, nb, hr.data(), hi.data(), pr.data(), pi.data(), H.dx * H.dy * H.dz,
                          H.gx * H.dx, H.gy * H.dy, H.gz * H.dz);
    for (int b = 0; b < nb; ++b)
        kpoint_dispatch(grid, hp[b], p[b], -0.5, H.dx, H.dy, H.dz, H.gx, H.gy, H.gz);
}

} // namespace

extern "C" {

void qsref_set_threads(int n) { openblas_set_num_threads(n); }

/* out += coef * FD8 Laplacian(p), periodic, x fastest. */
void qsref_laplacian8th(int nx, int ny, int nz, double* out, const double* p, double coef, double dx, double dy, double dz) {
    GridRange grid = MakeRange(nx, ny, nz);
    Laplacian8th<double>(grid, out, p, coef, dx, dy, dz);
}

/* out += coef*(Laplacian + 2i g.grad - g^2) applied to src (SoA complex). */
void qsref_laplacian_kpoint8th(int nx, int ny, int nz, double* out_re, double* out_im, const double* src_re,
                               const double* src_im, double coef, double dx, double dy, double dz, double gx,
                               double gy, double gz) {
    GridRange grid = MakeRange(nx, ny, nz);
    SoAComplex out{out_re, out_im};
    SoAComplex src{(double*)src_re, (double*)src_im};
    kpoint_dispatch(grid, out, src, coef, dx, dy, dz, gx, gy, gz);
}

/* Block decomposition of one atom's cube [b,e) (global coordinates, may
 * extend past the cell) over the periodic grid.  Writes up to max_blocks
 * entries of {begin_x,begin_y,begin_z,end_x,end_y,end_z,shift_x,shift_y,shift_z}
 * and returns the number of blocks; *grid_size receives the total points. */
int qsref_overlap_blocks(int nx, int ny, int nz, const int* cube, int* out, int max_blocks, int* grid_size) {
    GridRange grid = MakeRange(nx, ny, nz);
    GridRange c{cube[0], cube[1], cube[2], cube[3], cube[4], cube[5]};
    std::vector<GridRange> ranges;
    std::vector<ShiftedGrid> shifts;
    *grid_size = GetOverlapPeriodic(grid, c, nx, ny, nz, ranges, shifts);
    const int nbk = (int)ranges.size();
    for (int b = 0; b < nbk && b < max_blocks; ++b) {
        const int v[9] = {ranges[b].begin_x, ranges[b].begin_y, ranges[b].begin_z, ranges[b].end_x, ranges[b].end_y,
                          ranges[b].end_z, shifts[b].x, shifts[b].y, shifts[b].z};
        std::memcpy(out + 9 * b, v, sizeof(v));
    }
    return nbk;
}

/* Hp += V_NL psi over nb complex SoA bands (band b: re at psi + 2bN, im at
 * psi + (2b+1)N).  cubes: 6 ints per atom; proj: per-atom block-layout
 * projector tables concatenated; energy: per-atom widths concatenated. */
void qsref_nonlocal_apply(int nx, int ny, int nz, double dx, double dy, double dz, int n_atoms, const int* cubes,
                          const int* widths, const double* proj, const double* energy, int nb, double* hp,
                          const double* psi, double gx, double gy, double gz) {
    RefNonlocal nl = build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy);
    GridRange grid = MakeRange(nx, ny, nz);
    const size_t N = grid.Size3D();
    std::vector<double*> hr(nb), hi(nb);
    std::vector<const double*> pr(nb), pi(nb);
    for (int b = 0; b < nb; ++b) {
        hr[b] = hp + 2 * b * N; hi[b] = hp + (2 * b + 1) * N;
        pr[b] = psi + 2 * b * N; pi[b] = psi + (2 * b + 1) * N;
    }
    nonlocal_apply_bundle(nl, grid, nb, hr.data(), hi.data(), pr.data(), pi.data(), dx * dy * dz, gx * dx, gy * dy, gz * dz);
}

/* Nonlocal energy and forces of nb complex SoA bands, following
 * EnergyPPnonlocal_bundle (PseudoPotNonlocal_SvF2_kpoint.h:5033-5135) and the
 * grad(p) form of ForceNonlocal_bundle (:3629-3731): per atom the cut psi
 * (Bloch phase as mInnerNonlocalPsi applies it) is projected with DGEMM_t on
 * projector_RY and on its three gradient tables (dV-scaled, the inner / diff_x,
 * diff_y, diff_z of mInnerNonlocalPsi_diff_bundle), then
 *   E += |inner|^2 E_w occ_n,   F_a += 2 (inner.r diff.r + inner.i diff.i) E_w occ_n.
 * grad: per atom three block-layout tables (d/dx, d/dy, d/dz), grid_size x width each. */
void qsref_nonlocal_energy_force(int nx, int ny, int nz, double dx, double dy, double dz, int n_atoms,
                                 const int* cubes, const int* widths, const double* proj, const double* grad,
                                 const double* energy, int nb, const double* psi, const double* occ, double gx,
                                 double gy, double gz, double* energy_out, double* forces) {
    RefNonlocal nl = build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy);
    GridRange grid = MakeRange(nx, ny, nz);
    const size_t N = grid.Size3D();
    const double dV = dx * dy * dz;
    const double gx_dx = gx * dx, gy_dy = gy * dy, gz_dz = gz * dz;
    const bool is_gamma = (gx_dx == 0.0) && (gy_dy == 0.0) && (gz_dz == 0.0);
    double E = 0.0;
    size_t goff = 0;
    for (int ai = 0; ai < n_atoms; ++ai) {
        const RefAtom& a = nl.atoms[ai];
        if (a.width == 0 || a.grid_size == 0) continue;
        const int gs = a.grid_size, w = a.width;
        std::vector<double> cut((size_t)gs * 2 * nb);
        for (int n = 0; n < nb; ++n) {
            CutSubgridByRanges(a.ranges, cut.data() + (size_t)gs * 2 * n, grid, psi + 2 * n * N);
            CutSubgridByRanges(a.ranges, cut.data() + (size_t)gs * (2 * n + 1), grid, psi + (2 * n + 1) * N);
        }
        if (!is_gamma) {
            std::vector<double> ere, eim;
            bloch_exp(a, gx_dx, gy_dy, gz_dz, ere, eim);
            for (int n = 0; n < nb; ++n) {
                double* pr = cut.data() + (size_t)gs * 2 * n;
                double* pi = cut.data() + (size_t)gs * (2 * n + 1);
                for (int i = 0; i < gs; ++i) {
                    const double p_re = pr[i], p_im = pi[i];
                    pr[i] = ere[i] * p_re - eim[i] * p_im;
                    pi[i] = ere[i] * p_im + eim[i] * p_re;
                }
            }
        }
        std::vector<double> inner((size_t)w * 2 * nb), diff[3];
        blas_DGEMM_t(w, 2 * nb, gs, a.proj, cut.data(), inner.data(), w, dV, 0.0);
        for (int k = 0; k < 3; ++k) {
            diff[k].resize((size_t)w * 2 * nb);
            blas_DGEMM_t(w, 2 * nb, gs, grad + goff + (size_t)k * gs * w, cut.data(), diff[k].data(), w, dV, 0.0);
        }
        for (int n = 0; n < nb; ++n)
            for (int wi = 0; wi < w; ++wi) {
                const double eo = a.energy[wi] * occ[n];
                const double ir = inner[(size_t)w * (2 * n) + wi], ii = inner[(size_t)w * (2 * n + 1) + wi];
                E += (ir * ir + ii * ii) * eo;
                for (int k = 0; k < 3; ++k)
                    forces[3 * ai + k] += 2.0 * (ir * diff[k][(size_t)w * (2 * n) + wi] +
                                                 ii * diff[k][(size_t)w * (2 * n + 1) + wi]) * eo;
            }
        goff += (size_t)3 * gs * w;
    }
    *energy_out = E;
}

/* H psi = V psi + V_NL psi - 1/2 FD8(psi) for nb real bands (band b at psi + bN). */
void qsref_hamiltonian_real(int nx, int ny, int nz, double dx, double dy, double dz, const double* V, int n_atoms,
                            const int* cubes, const int* widths, const double* proj, const double* energy, int nb,
                            double* hp, const double* psi) {
    RefHamiltonian H{nx, ny, nz, dx, dy, dz, V, build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy), 0, 0, 0};
    const size_t N = (size_t)nx * ny * nz;
    for (int b = 0; b < nb; ++b) apply_h_real(H, hp + b * N, psi + b * N);
}

/* H psi for nb complex SoA bands at Bloch vector g. */
void qsref_hamiltonian_complex(int nx, int ny, int nz, double dx, double dy, double dz, const double* V, int n_atoms,
                               const int* cubes, const int* widths, const double* proj, const double* energy, int nb,
                               double* hp, const double* psi, double gx, double gy, double gz) {
    RefHamiltonian H{nx, ny, nz, dx, dy, dz, V, build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy), gx, gy, gz};
    const size_t N = (size_t)nx * ny * nz;
    std::vector<SoAComplex> h(nb), p(nb);
    for (int b = 0; b < nb; ++b) {
        h[b] = SoAComplex{hp + 2 * b * N, hp + (2 * b + 1) * N};
        p[b] = SoAComplex{(double*)psi + 2 * b * N, (double*)psi + (2 * b + 1) * N};
    }
    apply_h_complex(H, h.data(), p.data(), nb);
}

/* EigenLOBPCG_d_multi on the reference Hamiltonian.  keep: n*N (P), work:
 * 5*n*N.  Prints of the reference go to stdout. */
void qsref_lobpcg_d(int nx, int ny, int nz, double dx, double dy, double dz, const double* V, int n_atoms,
                    const int* cubes, const int* widths, const double* proj, const double* energy, int n, int iter_max,
                    double* eigen_values, double* X, double* keep, double* work, int is_first_time) {
    RefHamiltonian H{nx, ny, nz, dx, dy, dz, V, build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy), 0, 0, 0};
    const int N = nx * ny * nz;
    NullWatch watch;
    EigenLOBPCG_d_multi(N, dx * dy * dz, n, iter_max, eigen_values, X, keep, work, is_first_time != 0,
                        [&](double* Ax, const double* x) { apply_h_real(H, Ax, x); }, watch);
}

#ifdef QSREF_WITH_Z
/* LOBPCG::Eigen_z_multi_mpi on the reference Hamiltonian at Bloch vector g:
 * X and keep are SoA complex bundles (2*n*N doubles each), eigen_values n,
 * num_fix in/out.  Work arenas sized by the reference's own WorkSize functions. */
void qsref_lobpcg_z(int nx, int ny, int nz, double dx, double dy, double dz, const double* V, int n_atoms,
                    const int* cubes, const int* widths, const double* proj, const double* energy, int n, int iter_max,
                    double* eigen_values, double* X, double* keep, int* num_fix, double residual_threshold,
                    int scf_step, double gx, double gy, double gz) {
    RefHamiltonian H{nx, ny, nz, dx, dy, dz, V, build_nonlocal(nx, ny, nz, n_atoms, cubes, widths, proj, energy), gx, gy, gz};
    GridRangeMPI grid = make_grid(nx, ny, nz);
    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> work(LOBPCG::WorkSize_z_multi_mpi_keep((int)N, n) + 1024);
    std::vector<double> temporary(LOBPCG::WorkSize_z_multi_mpi_temporary((int)N, n) + 1024);
    std::vector<SoAComplex> xs(n);
    for (int k = 0; k < n; ++k) xs[k] = SoAComplex{X + 2 * k * N, X + (2 * k + 1) * N};
    NullWatch watch;
    LOBPCG::Eigen_z_multi_mpi(grid, dx * dy * dz, n, iter_max, eigen_values, xs.data(), keep, work.data(),
                              temporary.data(), num_fix, residual_threshold, nullptr, scf_step, 0,
                              [&](SoAComplex* Ax, SoAComplex* x, int nb) { apply_h_complex(H, Ax, x, nb); }, watch);
}
#endif

/* GramSchmidt_ddm (GramSchmidt_mpi.h:56-96) on a real bundle (nb x N) or a
 * complex SoA bundle (2 nb x N), in place, dV-weighted. */
void qsref_gram_schmidt(int nx, int ny, int nz, int nb, int is_complex, double* X, double dVol) {
    GridRangeMPI grid = make_grid(nx, ny, nz);
    const size_t N = (size_t)nx * ny * nz;
    if (is_complex) {
        std::vector<SoAComplex> xs(nb);
        for (int k = 0; k < nb; ++k) xs[k] = SoAComplex{X + 2 * k * N, X + (2 * k + 1) * N};
        GramSchmidt_ddm(grid, nb, xs.data(), dVol);
    } else {
        std::vector<double*> xs(nb);
        for (int k = 0; k < nb; ++k) xs[k] = X + k * N;
        GramSchmidt_ddm(grid, nb, xs.data(), dVol);
    }
}

/* exc[i] = rho eps_xc (exchange + correlation energy density), vxc[i] = V_x + V_c. */
void qsref_lda_pz(int n, const double* rho, double* exc, double* vxc) {
    for (int i = 0; i < n; ++i) {
        const Return_XC r = Calc_XC_LDA(rho[i]);
        exc[i] = r.rho_E_den_x + r.rho_E_den_c;
        vxc[i] = r.V_x + r.V_c;
    }
}

/* Fermi-Dirac occupations at chemical potential mu; returns their sum. */
double qsref_set_occupancy(double coef, double kbT, int n, const double* eig, double mu, double* occ) {
    return SetOccupancy(coef, kbT, n, eig, mu, occ);
}

/* axis: the three box edge vectors (grid_x * voxel_x, ...), as the frames hold them */
int qsref_cube_write(const char* path, const char* comment, int nx, int ny, int nz, const double* axis,
                     const double* org, int n_atoms, const int* Z, const double* pos, double* field) {
    CubeWriter::Frame f{};
    f.grid_x = nx; f.grid_y = ny; f.grid_z = nz;
    for (int i = 0; i < 9; ++i) f.boxaxis[i] = axis[i];
    for (int i = 0; i < 3; ++i) f.boxorg[i] = org[i];
    std::snprintf(f.comment, sizeof(f.comment), "%s", comment);
    std::vector<Nucleus> nuc(n_atoms);
    for (int a = 0; a < n_atoms; ++a) nuc[a] = Nucleus{Z[a], pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    return CubeWriter::SaveCube(path, f, n_atoms, nuc.data(), field);
}

/* LoadUPF_ONCV's radial data: info = {n_proj, valence, n_grid}; cutoff[4];
 * xi[2] = {xi_min, xi_delta}; radius, v_local [n_grid]; l, energy [n_proj];
 * proj [n_proj x n_grid] (the up-spin copies).  Outputs after info may be NULL
 * (first call for the sizes).  Returns 0 when the file did not load. */
int qsref_upf_load(const char* path, int* info, double* cutoff, double* xi, double* radius, double* v_local, int* l,
                   double* energy, double* proj) {
    PseudoPot_MBK* p = LoadUPF_ONCV(path);
    if (!p) return 0;
    info[0] = p->num_radial_projectors;
    info[1] = (int)p->valence_electron;
    info[2] = p->num_radial_grids;
    if (cutoff) for (int i = 0; i < 4; ++i) cutoff[i] = p->cutoff_r[i];
    if (xi) { xi[0] = p->xi_min; xi[1] = p->xi_delta; }
    const int n = p->num_radial_grids;
    if (radius) for (int i = 0; i < n; ++i) radius[i] = p->radius[i];
    if (v_local) for (int i = 0; i < n; ++i) v_local[i] = p->V_local[i];
    for (int k = 0; k < p->num_radial_projectors; ++k) {
        if (l) l[k] = p->projector_quantum_l[k];
        if (energy) energy[k] = p->projector_energy_up[k];
        if (proj) for (int i = 0; i < n; ++i) proj[(size_t)k * n + i] = p->projector[2 * k][i];
    }
    return 1;
}

/* grid[3] and axis[9], org[3] out; field (x fastest) out when not NULL */
void qsref_cube_read(const char* path, int* grid, double* axis, double* org, double* field) {
    CubeReader3 r;
    const CubeReader3::Frame f = r.LoadCube(path);
    grid[0] = f.grid_x; grid[1] = f.grid_y; grid[2] = f.grid_z;
    for (int i = 0; i < 9; ++i) axis[i] = f.boxaxis[i];
    for (int i = 0; i < 3; ++i) org[i] = f.boxorg[i];
    if (field) r.GetMeshData(field);
}

} // extern "C"
