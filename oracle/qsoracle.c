/*
 * oracle/qsoracle.c — CPU restatement (plain C, FP64, single thread) of the
 * reference's H.psi hot path.  TEST INFRASTRUCTURE ONLY: the parity tests,
 * smoke() and bench.py's CPU baseline call it as the checker; the product
 * never links it.
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the
 * reference's own headers compiled from its source tree (oracle/_ref,
 * oracle/ref_entry.cpp) and tests/test_oracle.py checks this file against them.
 *
 * Each function names the reference code it restates (paths relative to the
 * reference's source/ directory).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

static inline int wrap(int v, int n) {
    int m = v % n;
    return m < 0 ? m + n : m;
}

/* out += coef * Laplacian_8th(p), periodic.
 * Laplacian8th -> PasteHalo_f4 + Laplacian8th_halo_f (GridDifference8th.h:19-148,177-184):
 * coefficients :89-101, summation order :140-144 (centre, x, y, z; offsets 4,3,2,1). */
void qso_laplacian8th(int nx, int ny, int nz, double* out, const double* p, double coef, double dx, double dy,
                      double dz) {
    const double c0 = -14350.0 / 5040.0 * coef * (1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz));
    const double c4x = -9.0 * coef / (5040.0 * dx * dx), c3x = 128.0 * coef / (5040.0 * dx * dx);
    const double c2x = -1008.0 * coef / (5040.0 * dx * dx), c1x = 8064.0 * coef / (5040.0 * dx * dx);
    const double c4y = -9.0 * coef / (5040.0 * dy * dy), c3y = 128.0 * coef / (5040.0 * dy * dy);
    const double c2y = -1008.0 * coef / (5040.0 * dy * dy), c1y = 8064.0 * coef / (5040.0 * dy * dy);
    const double c4z = -9.0 * coef / (5040.0 * dz * dz), c3z = 128.0 * coef / (5040.0 * dz * dz);
    const double c2z = -1008.0 * coef / (5040.0 * dz * dz), c1z = 8064.0 * coef / (5040.0 * dz * dz);
    const size_t nxy = (size_t)nx * ny;
#define P(X, Y, Z) p[(size_t)wrap(X, nx) + (size_t)nx * wrap(Y, ny) + nxy * wrap(Z, nz)]
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                double d = c0 * P(ix, iy, iz);
                d += c4x * (P(ix + 4, iy, iz) + P(ix - 4, iy, iz)) + c3x * (P(ix + 3, iy, iz) + P(ix - 3, iy, iz)) +
                     c2x * (P(ix + 2, iy, iz) + P(ix - 2, iy, iz)) + c1x * (P(ix + 1, iy, iz) + P(ix - 1, iy, iz));
                d += c4y * (P(ix, iy + 4, iz) + P(ix, iy - 4, iz)) + c3y * (P(ix, iy + 3, iz) + P(ix, iy - 3, iz)) +
                     c2y * (P(ix, iy + 2, iz) + P(ix, iy - 2, iz)) + c1y * (P(ix, iy + 1, iz) + P(ix, iy - 1, iz));
                d += c4z * (P(ix, iy, iz + 4) + P(ix, iy, iz - 4)) + c3z * (P(ix, iy, iz + 3) + P(ix, iy, iz - 3)) +
                     c2z * (P(ix, iy, iz + 2) + P(ix, iy, iz - 2)) + c1z * (P(ix, iy, iz + 1) + P(ix, iy, iz - 1));
                out[(size_t)ix + (size_t)nx * iy + nxy * iz] += d;
            }
#undef P
}

/* One pass of LaplacianKpoint8th_halo_f (GridDifferenceKpoint8th.h:17-120):
 * out += Lap_g(p) and out2 += sign * D_g(p), with the |g_d| < 1e-8 dispatch of
 * LaplacianKpoint8th_ddm (:330-364) deciding which first-derivative terms exist. */
static void kpoint_pass(int nx, int ny, int nz, double* out, double* out2, const double* p, double coef,
                        double sign1st, double dx, double dy, double dz, double gx, double gy, double gz) {
    const int KX = fabs(gx) >= 1.0e-8, KY = fabs(gy) >= 1.0e-8, KZ = fabs(gz) >= 1.0e-8;
    const double c0 = -14350.0 / 5040.0 * coef * (1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)) -
                      coef * (gx * gx + gy * gy + gz * gz);
    const double c4x = -9.0 * coef / (5040.0 * dx * dx), c3x = 128.0 * coef / (5040.0 * dx * dx);
    const double c2x = -1008.0 * coef / (5040.0 * dx * dx), c1x = 8064.0 * coef / (5040.0 * dx * dx);
    const double c4y = -9.0 * coef / (5040.0 * dy * dy), c3y = 128.0 * coef / (5040.0 * dy * dy);
    const double c2y = -1008.0 * coef / (5040.0 * dy * dy), c1y = 8064.0 * coef / (5040.0 * dy * dy);
    const double c4z = -9.0 * coef / (5040.0 * dz * dz), c3z = 128.0 * coef / (5040.0 * dz * dz);
    const double c2z = -1008.0 * coef / (5040.0 * dz * dz), c1z = 8064.0 * coef / (5040.0 * dz * dz);
    const double coef2 = sign1st * coef * 2.0;
    const double a1x = 672.0 * coef2 * gx / (840.0 * dx), a2x = -168.0 * coef2 * gx / (840.0 * dx);
    const double a3x = 32.0 * coef2 * gx / (840.0 * dx), a4x = -3.0 * coef2 * gx / (840.0 * dx);
    const double a1y = 672.0 * coef2 * gy / (840.0 * dy), a2y = -168.0 * coef2 * gy / (840.0 * dy);
    const double a3y = 32.0 * coef2 * gy / (840.0 * dy), a4y = -3.0 * coef2 * gy / (840.0 * dy);
    const double a1z = 672.0 * coef2 * gz / (840.0 * dz), a2z = -168.0 * coef2 * gz / (840.0 * dz);
    const double a3z = 32.0 * coef2 * gz / (840.0 * dz), a4z = -3.0 * coef2 * gz / (840.0 * dz);
    const size_t nxy = (size_t)nx * ny;
#define P(X, Y, Z) p[(size_t)wrap(X, nx) + (size_t)nx * wrap(Y, ny) + nxy * wrap(Z, nz)]
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const size_t io = (size_t)ix + (size_t)nx * iy + nxy * iz;
                double d = c0 * P(ix, iy, iz);
                d += c4x * (P(ix + 4, iy, iz) + P(ix - 4, iy, iz)) + c3x * (P(ix + 3, iy, iz) + P(ix - 3, iy, iz)) +
                     c2x * (P(ix + 2, iy, iz) + P(ix - 2, iy, iz)) + c1x * (P(ix + 1, iy, iz) + P(ix - 1, iy, iz));
                d += c4y * (P(ix, iy + 4, iz) + P(ix, iy - 4, iz)) + c3y * (P(ix, iy + 3, iz) + P(ix, iy - 3, iz)) +
                     c2y * (P(ix, iy + 2, iz) + P(ix, iy - 2, iz)) + c1y * (P(ix, iy + 1, iz) + P(ix, iy - 1, iz));
                d += c4z * (P(ix, iy, iz + 4) + P(ix, iy, iz - 4)) + c3z * (P(ix, iy, iz + 3) + P(ix, iy, iz - 3)) +
                     c2z * (P(ix, iy, iz + 2) + P(ix, iy, iz - 2)) + c1z * (P(ix, iy, iz + 1) + P(ix, iy, iz - 1));
                out[io] += d;
                double g = 0.0;
                if (KX)
                    g += a4x * (P(ix + 4, iy, iz) - P(ix - 4, iy, iz)) + a3x * (P(ix + 3, iy, iz) - P(ix - 3, iy, iz)) +
                         a2x * (P(ix + 2, iy, iz) - P(ix - 2, iy, iz)) + a1x * (P(ix + 1, iy, iz) - P(ix - 1, iy, iz));
                if (KY)
                    g += a4y * (P(ix, iy + 4, iz) - P(ix, iy - 4, iz)) + a3y * (P(ix, iy + 3, iz) - P(ix, iy - 3, iz)) +
                         a2y * (P(ix, iy + 2, iz) - P(ix, iy - 2, iz)) + a1y * (P(ix, iy + 1, iz) - P(ix, iy - 1, iz));
                if (KZ)
                    g += a4z * (P(ix, iy, iz + 4) - P(ix, iy, iz - 4)) + a3z * (P(ix, iy, iz + 3) - P(ix, iy, iz - 3)) +
                         a2z * (P(ix, iy, iz + 2) - P(ix, iy, iz - 2)) + a1z * (P(ix, iy, iz + 1) - P(ix, iy, iz - 1));
                if (KX || KY || KZ) out2[io] += g;
            }
#undef P
}

/* LaplacianKpoint8th_halo (GridDifferenceKpoint8th.h:123-151): the real part
 * with sign +1 (cross term into out.im), then the imaginary part with sign -1. */
void qso_laplacian_kpoint8th(int nx, int ny, int nz, double* out_re, double* out_im, const double* src_re,
                             const double* src_im, double coef, double dx, double dy, double dz, double gx, double gy,
                             double gz) {
    kpoint_pass(nx, ny, nz, out_re, out_im, src_re, coef, +1.0, dx, dy, dz, gx, gy, gz);
    kpoint_pass(nx, ny, nz, out_im, out_re, src_im, coef, -1.0, dx, dy, dz, gx, gy, gz);
}

/* hp += V_NL psi, projectors given as per-atom point lists (unfolded coords) and
 * column-major tables.  Order of operations of ProjectionPP_bundle_1 and
 * mInnerNonlocalPsi_v4_bundle (PseudoPotNonlocal_SvF2_kpoint.h:3911-4046,
 * :4463-4576): gather (:4493-4496), Bloch phase exp(+ikr) (:4503-4519),
 * inner = dV * P^T cut (DGEMM_t :4528), times E_w (:4003-4011),
 * cut = P inner (DGEMM_n :4017), phase exp(-ikr) (:4021-4037), scatter-add (:4046).
 * is_complex = 0: nb real bands; 1: nb complex SoA bands. */
void qso_nonlocal_apply(int nx, int ny, int nz, double dx, double dy, double dz, int n_atoms, const int* npts,
                        const int* widths, const int* coords, const double* beta, const double* energy, int nb,
                        int is_complex, double* hp, const double* psi, double gx, double gy, double gz) {
    const size_t N = (size_t)nx * ny * nz;
    const double dV = dx * dy * dz;
    const int is_gamma = (gx * dx == 0.0) && (gy * dy == 0.0) && (gz * dz == 0.0);
    const int ncomp = is_complex ? 2 : 1;
    size_t poff = 0, boff = 0, eoff = 0;
    for (int a = 0; a < n_atoms; ++a) {
        const int np = npts[a], w = widths[a];
        const int* c = coords + 3 * poff;
        const double* P = beta + boff;
        const double* E = energy + eoff;
        if (w > 0 && np > 0) {
            size_t* gi = (size_t*)malloc(sizeof(size_t) * np);
            double* er = (double*)malloc(sizeof(double) * np);
            double* ei = (double*)malloc(sizeof(double) * np);
            double* cut = (double*)malloc(sizeof(double) * np * ncomp);
            double* inner = (double*)malloc(sizeof(double) * w * ncomp);
            for (int i = 0; i < np; ++i) {
                gi[i] = (size_t)wrap(c[3 * i], nx) + (size_t)nx * wrap(c[3 * i + 1], ny) +
                        (size_t)nx * ny * wrap(c[3 * i + 2], nz);
                if (is_complex && !is_gamma) {
                    const double kxx = gx * dx * (double)c[3 * i], kyy = gy * dy * (double)c[3 * i + 1],
                                 kzz = gz * dz * (double)c[3 * i + 2];
                    er[i] = cos(kxx + kyy + kzz);
                    ei[i] = sin(kxx + kyy + kzz);
                }
            }
            for (int b = 0; b < nb; ++b) {
                const double* pr = psi + (size_t)(is_complex ? 2 * b : b) * N;
                const double* pim = is_complex ? psi + (size_t)(2 * b + 1) * N : NULL;
                for (int i = 0; i < np; ++i) {
                    cut[i] = pr[gi[i]];
                    if (is_complex) cut[np + i] = pim[gi[i]];
                }
                if (is_complex && !is_gamma)
                    for (int i = 0; i < np; ++i) {
                        const double p_re = cut[i], p_im = cut[np + i];
                        cut[i] = er[i] * p_re - ei[i] * p_im;
                        cut[np + i] = er[i] * p_im + ei[i] * p_re;
                    }
                for (int k = 0; k < ncomp; ++k)
                    for (int ww = 0; ww < w; ++ww) {
                        double s = 0.0;
                        for (int i = 0; i < np; ++i) s += P[(size_t)ww * np + i] * cut[(size_t)k * np + i];
                        inner[k * w + ww] = dV * s * E[ww];
                    }
                for (int k = 0; k < ncomp; ++k)
                    for (int i = 0; i < np; ++i) {
                        double s = 0.0;
                        for (int ww = 0; ww < w; ++ww) s += P[(size_t)ww * np + i] * inner[k * w + ww];
                        cut[(size_t)k * np + i] = s;
                    }
                if (is_complex && !is_gamma)
                    for (int i = 0; i < np; ++i) {
                        const double p_re = cut[i], p_im = cut[np + i];
                        cut[i] = er[i] * p_re + ei[i] * p_im;
                        cut[np + i] = er[i] * p_im - ei[i] * p_re;
                    }
                double* hr = hp + (size_t)(is_complex ? 2 * b : b) * N;
                double* him = is_complex ? hp + (size_t)(2 * b + 1) * N : NULL;
                for (int i = 0; i < np; ++i) {
                    hr[gi[i]] += cut[i];
                    if (is_complex) him[gi[i]] += cut[np + i];
                }
            }
            free(gi); free(er); free(ei); free(cut); free(inner);
        }
        poff += (size_t)np;
        boff += (size_t)np * w;
        eoff += (size_t)w;
    }
}

/* <beta|psi> dV per projector and column: out[col * P + proj], the quantity of
 * mInnerNonlocalPsi_v4_bundle (PseudoPotNonlocal_SvF2_kpoint.h:4463-4576). */
void qso_nonlocal_project(int nx, int ny, int nz, double dx, double dy, double dz, int n_atoms, const int* npts,
                          const int* widths, const int* coords, const double* beta, int nb, int is_complex,
                          const double* psi, double gx, double gy, double gz, double* out) {
    const size_t N = (size_t)nx * ny * nz;
    const double dV = dx * dy * dz;
    int P = 0;
    for (int a = 0; a < n_atoms; ++a) P += widths[a];
    const int ncol = is_complex ? 2 * nb : nb;
    memset(out, 0, sizeof(double) * (size_t)P * ncol);
    size_t poff = 0, boff = 0;
    int proj0 = 0;
    for (int a = 0; a < n_atoms; ++a) {
        const int np = npts[a], w = widths[a];
        const int* c = coords + 3 * poff;
        const double* Pt = beta + boff;
        for (int b = 0; b < nb; ++b)
            for (int ww = 0; ww < w; ++ww) {
                double sr = 0.0, si = 0.0;
                for (int i = 0; i < np; ++i) {
                    const size_t g = (size_t)wrap(c[3 * i], nx) + (size_t)nx * wrap(c[3 * i + 1], ny) +
                                     (size_t)nx * ny * wrap(c[3 * i + 2], nz);
                    if (is_complex) {
                        const double kxx = gx * dx * (double)c[3 * i], kyy = gy * dy * (double)c[3 * i + 1],
                                     kzz = gz * dz * (double)c[3 * i + 2];
                        const double er = cos(kxx + kyy + kzz), ei = sin(kxx + kyy + kzz);
                        const double pr = psi[(size_t)(2 * b) * N + g], pim = psi[(size_t)(2 * b + 1) * N + g];
                        sr += Pt[(size_t)ww * np + i] * (er * pr - ei * pim);
                        si += Pt[(size_t)ww * np + i] * (er * pim + ei * pr);
                    } else {
                        sr += Pt[(size_t)ww * np + i] * psi[(size_t)b * N + g];
                    }
                }
                if (is_complex) {
                    out[(size_t)(2 * b) * P + proj0 + ww] = dV * sr;
                    out[(size_t)(2 * b + 1) * P + proj0 + ww] = dV * si;
                } else {
                    out[(size_t)b * P + proj0 + ww] = dV * sr;
                }
            }
        poff += (size_t)np;
        boff += (size_t)np * w;
        proj0 += w;
    }
}

/* mHamiltonianMatrix_ddm (qumasun_base1.matrix.h:263-291) restated for a
 * bundle: hp = V psi; hp += V_NL psi; hp += -1/2 FD8 kinetic (k-point form
 * for complex bands). */
void qso_hamiltonian(int nx, int ny, int nz, double dx, double dy, double dz, const double* V, int n_atoms,
                     const int* npts, const int* widths, const int* coords, const double* beta, const double* energy,
                     int nb, int is_complex, double* hp, const double* psi, double gx, double gy, double gz) {
    const size_t N = (size_t)nx * ny * nz;
    const int ncomp = is_complex ? 2 : 1;
    for (int b = 0; b < nb * ncomp; ++b)
        for (size_t i = 0; i < N; ++i) hp[(size_t)b * N + i] = V[i] * psi[(size_t)b * N + i];
    qso_nonlocal_apply(nx, ny, nz, dx, dy, dz, n_atoms, npts, widths, coords, beta, energy, nb, is_complex, hp, psi,
                       gx, gy, gz);
    for (int b = 0; b < nb; ++b) {
        if (is_complex)
            qso_laplacian_kpoint8th(nx, ny, nz, hp + (size_t)(2 * b) * N, hp + (size_t)(2 * b + 1) * N,
                                    psi + (size_t)(2 * b) * N, psi + (size_t)(2 * b + 1) * N, -0.5, dx, dy, dz, gx,
                                    gy, gz);
        else
            qso_laplacian8th(nx, ny, nz, hp + (size_t)b * N, psi + (size_t)b * N, -0.5, dx, dy, dz);
    }
}
