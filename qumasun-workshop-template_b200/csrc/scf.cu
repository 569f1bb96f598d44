// Self-consistent-field driver on the device: Gamma point, spin-unpolarised,
// LDA (Perdew-Zunger), analytic GTH local part, Fermi-Dirac occupations,
// Kerker-preconditioned DIIS density mixing, the real LOBPCG of lobpcg.cu.
//
// Step order of QUMASUN_KPOINT::Execute (source/qumasun_kpoint.scfloop.h:61-230):
// eigensolver -> occupations -> density -> mixing -> potentials -> energy ->
// |dE| / atom test.  The wavefunctions, densities, potentials, the Poisson and
// XC steps and the mixing history stay on the device; per step only the band
// energies (nb values), a handful of inner products and the DIIS matrix cross
// to the host.
//
// Pieces and their sources:
//   * density: SetDensityOne (source/qumasun_SetDensityOne.h), rho = sum occ psi^2;
//   * LDA: Calc_XC_LDA (source/Vxc.h:43-75);
//   * occupations: SetOccupancy (source/SetOccupancy.h:7-18) with the bisection
//     of mSetOccupancyTemperature (source/qumasun_base1.occupancy.h:76-170);
//   * Hartree: lap V = -4 pi rho by the FFT (cuFFT), G = 0 removed;
//   * GTH local part in G space (published GTH form), Kerker-preconditioned
//     DIIS and the Kohn-Sham energy of the output density: restated from the
//     mathematics (the reference forms its local potential from core charges on
//     a finer grid, source/qumasun_base1.core.h, and mixes with DIIS or Kerker
//     separately, source/mixing_DIIS.h, source/mixing_kerker.h).
#include "qsb_internal.h"
#include <cufft.h>
#include <cmath>
#include <vector>
#include <algorithm>
#include <chrono>

namespace qsb {
namespace {

constexpr int RB = 256;          // reduction block
constexpr int RBLOCKS = 592;     // partial sums (4 x 148 SMs), fixed: deterministic order

// ---------------- pointwise kernels ----------------

// rho[i] = sum_n occ[n] X[n][i]^2, bands in order (deterministic)
__global__ void density_kernel(size_t N, int nb, const double* __restrict__ X, const double* __restrict__ occ,
                               double* __restrict__ rho) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        double r = 0.0;
        for (int n = 0; n < nb; ++n) {
            const double x = X[(size_t)n * N + i];
            r += occ[n] * (x * x);
        }
        rho[i] = r;
    }
}

// Perdew-Zunger LDA (Calc_XC_LDA, source/Vxc.h:43-75): exc = rho eps_xc, vxc = V_x + V_c
// continuous = true: the high-density correlation branch with C and D solved
// from value and slope continuity at rs = 1 (A, B kept); with the published
// C = 0.0020, D = -0.0116 the two branches miss each other there by 3.2e-5 Ha
// in eps_c, so E_xc jumps by rho dV 3.2e-5 whenever a grid point's density
// crosses 3 / (4 pi).
__device__ __forceinline__ void lda_pz_point(double rho, double& exc, double& vxc, double rho_min = 1.0e-8,
                                             bool continuous = false) {
    if (rho < rho_min) {
        exc = 0.0;
        vxc = 0.0;
        return;
    }
    const double c2 = 0.62035049089940001667;            // cbrt(3 / (4 pi))
    const double c3 = -0.45816529328314287;               // -(3 / (4 pi)) cbrt(9 pi / 4)
    const double rs = c2 / cbrt(rho);
    const double ex = c3 / rs;
    double ec, ndec;
    if (rs >= 1.0) {
        const double g = -0.1423, b1 = 1.0529, b2 = 0.3334;
        const double s = sqrt(rs);
        ec = g / (1.0 + b1 * s + b2 * rs);
        ndec = ec * ec * (b1 * 0.5 * s + b2 * rs) / (3.0 * g);
    } else {
        const double A = 0.0311, B = -0.0480;
        const double C = continuous ? 0.0020191519406228 : 0.0020;
        const double D = continuous ? -0.0116320663789130 : -0.0116;
        const double lr = log(rs);
        ec = B + A * lr + D * rs + C * rs * lr;
        ndec = -(A + (D + C) * rs + C * rs * lr) / 3.0;
    }
    exc = rho * ex + rho * ec;
    vxc = (ex + ex / 3.0) + (ec + ndec);
}

__global__ void lda_kernel(size_t N, const double* __restrict__ rho, double* __restrict__ exc,
                           double* __restrict__ vxc, double rho_min = 1.0e-8, bool continuous = false) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        double e, v;
        lda_pz_point(rho[i], e, v, rho_min, continuous);
        if (exc) exc[i] = e;
        vxc[i] = v;
    }
}

// ---------------------------------------------------------------------------
// GGA-PBE, spin-unpolarised, as the reference's mSetPotentialVxc takes it
// (source/qumasun_base1.potential.h:383-470, 585-640 with XC_IMPLE_VER2):
// exchange per spin channel on rho_s = rho / 2 (GGA_PBE::Potential_X_test3,
// source/xc_gga_pbe.h:326-356; E_x = 2 E_x[rho_s]), correlation on rho with
// |grad rho|^2 (EnergyDensityPotential_C_test3, :525-594, PW92 local part
// LDA_PW92, :7-76, at zeta = 0), gradients and divergences by the eighth-order
// central first derivative (GridGradient8th.h:23-26), V_xc = v_x + v_c
// - 2 div(P_x grad rho_s) - 2 div(P_c grad rho).  The published PBE (Perdew,
// Burke, Ernzerhof, PRL 77, 3865) and PW92 (Perdew, Wang, PRB 45, 13244)
// parameters as the reference rounds them.
// ---------------------------------------------------------------------------
struct Grid3 {
    int nx, ny, nz;
    double dx, dy, dz;
};

// first derivative along axis `axis` of f at point (x, y, z), periodic, FD8
__device__ __forceinline__ double fd8_d1(const double* __restrict__ f, const Grid3& g, int x, int y, int z, int axis,
                                         double scale) {
    const double h = axis == 0 ? g.dx : axis == 1 ? g.dy : g.dz;
    const double c4 = -3.0 / (840.0 * h), c3 = 32.0 / (840.0 * h), c2 = -168.0 / (840.0 * h), c1 = 672.0 / (840.0 * h);
    auto at = [&](int m) -> double {
        int xx = x, yy = y, zz = z;
        if (axis == 0) xx = (x + m + 4 * g.nx) % g.nx;
        else if (axis == 1) yy = (y + m + 4 * g.ny) % g.ny;
        else zz = (z + m + 4 * g.nz) % g.nz;
        return scale * f[(size_t)xx + (size_t)g.nx * (yy + (size_t)g.ny * zz)];
    };
    return c4 * (at(4) - at(-4)) + c3 * (at(3) - at(-3)) + c2 * (at(2) - at(-2)) + c1 * (at(1) - at(-1));
}

// grad rho_s (rho_s = rho / 2) into g[0..3N)
__global__ void gga_grad_kernel(Grid3 g, const double* __restrict__ rho, double* __restrict__ grad) {
    const size_t N = (size_t)g.nx * g.ny * g.nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / ((size_t)g.nx * g.ny));
        grad[i] = fd8_d1(rho, g, x, y, z, 0, 0.5);
        grad[N + i] = fd8_d1(rho, g, x, y, z, 1, 0.5);
        grad[2 * N + i] = fd8_d1(rho, g, x, y, z, 2, 0.5);
    }
}

// Per point: exc = 2 rho_s eps_x(rho_s, s_s) + rho (eps_c^PW92 + H), vxc = v_x + v_c
// (the local parts), and grad (in) -> the flux 2 P_x grad rho_s + 2 P_c grad rho (out).
__global__ void gga_pbe_point_kernel(size_t N, const double* __restrict__ rho, double* __restrict__ grad,
                                     double* __restrict__ exc, double* __restrict__ vxc) {
    const double kappa = 0.804, mu = 0.21951, beta = 0.066725, gamma = 0.031091;
    const double cut = 1.0e-8;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const double gx = grad[i], gy = grad[N + i], gz = grad[2 * N + i];
        const double rs_ = 0.5 * rho[i];
        // exchange, one spin channel
        double ex = 0.0, vx = 0.0, px = 0.0;
        if (rs_ >= cut) {
            const double s2 = gx * gx + gy * gy + gz * gz;
            const double r13 = cbrt(rs_);
            const double r43 = r13 * rs_;
            const double c6 = cbrt(6.0 / M_PI);
            const double c62 = (6.0 * M_PI) / c6;
            const double qm = 4.0 * c62 * r43 * r43;
            const double q = s2 / qm;
            const double den = 1.0 + q * mu / kappa;
            const double F = 1.0 + kappa - kappa / den;
            const double dF = mu / (den * den);
            const double dq_dr = -(8.0 / 3.0) * q / rs_;
            ex = -(3.0 / 4.0) * c6 * r43 * F;
            vx = -c6 * (r13 * F + (3.0 / 4.0) * r43 * dF * dq_dr);
            px = -(3.0 / 4.0) * c6 * r43 * dF * (1.0 / qm);
        }
        // correlation on rho = 2 rho_s with grad rho = 2 grad rho_s
        const double r = 2.0 * rs_;
        double ec = 0.0, vc = 0.0, pc = 0.0;
        if (r >= cut) {
            const double Gx = 2.0 * gx, Gy = 2.0 * gy, Gz = 2.0 * gz;
            const double s2 = Gx * Gx + Gy * Gy + Gz * Gz;
            // PW92, zeta = 0
            const double A = 0.031091, al = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
            const double rsw = cbrt(3.0 / (4.0 * M_PI * r));
            const double sq = sqrt(rsw);
            const double mother = 2.0 * A * (b1 * sq + b2 * rsw + b3 * rsw * sq + b4 * rsw * rsw);
            const double lnt = log(1.0 + 1.0 / mother);
            const double el = -2.0 * A * (1.0 + al * rsw) * lnt;
            const double dmo = 2.0 * A * (b1 / (2.0 * sq) + b2 + (3.0 / 2.0) * b3 * sq + 2.0 * b4 * rsw);
            const double dln = -dmo / ((mother + 1.0) * mother);
            const double de = -2.0 * A * (al * lnt + (1.0 + al * rsw) * dln);
            const double vl = el - (1.0 / 3.0) * rsw * de;
            // PBE gradient correction H, phi = 1 at zeta = 0
            const double ee = exp(-el / gamma);
            const double alpha = ee - 1.0;
            const double C = (beta / gamma) * cbrt(M_PI / 3.0) / 16.0;
            const double cr = cbrt(r);
            const double Y = C * s2;
            const double r73 = r * r * cr;
            const double B = alpha * r73;
            const double BeY = fmax(B + ee * Y, 1e-30);
            const double BY = fmax(B + Y, 1e-30);
            const double lg = log(BeY / BY);
            const double H = gamma * lg;
            const double dexp = (0.5 * r < cut) ? 0.0 : -(ee / gamma) * (vl - el) / r;
            const double dB = (7.0 / 3.0) * alpha * cr * r + r73 * dexp;
            const double vH = H + r * gamma * ((-alpha * Y / (BeY * BY)) * dB + Y / BeY * dexp);
            ec = el + H;
            vc = vl + vH;
            pc = r * gamma * (alpha * B / (BeY * BY)) * C;
        }
        if (exc) exc[i] = 2.0 * ex + r * ec;
        vxc[i] = vx + vc;
        const double f = 2.0 * px + 4.0 * pc;
        grad[i] = f * gx;
        grad[N + i] = f * gy;
        grad[2 * N + i] = f * gz;
    }
}

// vxc -= div(flux)
__global__ void gga_div_kernel(Grid3 g, const double* __restrict__ flux, double* __restrict__ vxc) {
    const size_t N = (size_t)g.nx * g.ny * g.nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / ((size_t)g.nx * g.ny));
        const double d = fd8_d1(flux, g, x, y, z, 0, 1.0) + fd8_d1(flux + N, g, x, y, z, 1, 1.0) +
                         fd8_d1(flux + 2 * N, g, x, y, z, 2, 1.0);
        vxc[i] -= d;
    }
}

// out = a + b + c
__global__ void sum3_kernel(size_t N, const double* __restrict__ a, const double* __restrict__ b,
                            const double* __restrict__ c, double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        out[i] = a[i] + b[i] + c[i];
}

// out = a - b
__global__ void sub_kernel(size_t N, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}

// out = sum_k coef[k] in[k], m <= 8 arrays, in the given order
struct Combo {
    const double* in[8];
    double coef[8];
    int m;
};
__global__ void combo_kernel(size_t N, Combo c, double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        double r = 0.0;
        for (int k = 0; k < c.m; ++k) r += c.coef[k] * c.in[k][i];
        out[i] = r;
    }
}

// out += in
__global__ void add_kernel(size_t N, const double* __restrict__ in, double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        out[i] += in[i];
}

// ---------------- deterministic reductions ----------------

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < RB / 32; ++w) r += sh[w];
    __syncthreads();
    return r;
}

// partial[j * gridDim.x + blockIdx.x] = sum over this block's points of a_j b (j < na; b null: of a_j)
__global__ void __launch_bounds__(RB) dot_partial_kernel(size_t N, int na, const double* const* __restrict__ a,
                                                         const double* __restrict__ b, double* __restrict__ partial) {
    __shared__ double sh[RB / 32];
    for (int j = 0; j < na; ++j) {
        double v = 0.0;
        for (size_t i = blockIdx.x * (size_t)RB + threadIdx.x; i < N; i += (size_t)gridDim.x * RB)
            v += b ? a[j][i] * b[i] : a[j][i];
        const double s = block_sum(v, sh);
        if (threadIdx.x == 0) partial[(size_t)j * gridDim.x + blockIdx.x] = s;
    }
}

// partial[blockIdx.x] = sum over this block's points of |a - b|
__global__ void __launch_bounds__(RB) l1_diff_partial_kernel(size_t N, const double* __restrict__ a,
                                                             const double* __restrict__ b,
                                                             double* __restrict__ partial) {
    __shared__ double sh[RB / 32];
    double v = 0.0;
    for (size_t i = blockIdx.x * (size_t)RB + threadIdx.x; i < N; i += (size_t)gridDim.x * RB) v += fabs(a[i] - b[i]);
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// per band n: partial[n][blk] = sum x_n y_n and sum x_n x_n over this block's points
__global__ void __launch_bounds__(RB) band_dot_kernel(size_t N, const double* __restrict__ X,
                                                      const double* __restrict__ Y, double* __restrict__ pxy,
                                                      double* __restrict__ pxx) {
    __shared__ double sh[RB / 32];
    const int n = blockIdx.y;
    const double* x = X + (size_t)n * N;
    const double* y = Y + (size_t)n * N;
    double vxy = 0.0, vxx = 0.0;
    for (size_t i = blockIdx.x * (size_t)RB + threadIdx.x; i < N; i += (size_t)gridDim.x * RB) {
        const double xi = x[i];
        vxy += xi * y[i];
        vxx += xi * xi;
    }
    const double s1 = block_sum(vxy, sh);
    const double s2 = block_sum(vxx, sh);
    if (threadIdx.x == 0) {
        pxy[(size_t)n * gridDim.x + blockIdx.x] = s1;
        pxx[(size_t)n * gridDim.x + blockIdx.x] = s2;
    }
}

// out[j] = sum over blk of partial[j][blk], fixed order (one warp per row)
__global__ void row_sum_kernel(int rows, int cols, const double* __restrict__ partial, double* __restrict__ out) {
    const int j = blockIdx.x;
    if (j >= rows) return;
    double v = 0.0;
    for (int k = threadIdx.x; k < cols; k += 32) v += partial[(size_t)j * cols + k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) out[j] = v;
}

// ---------------- reciprocal space (half-complex grid [nz][ny][nx/2+1]) ----------------

__device__ __forceinline__ double freq(int k, int n, double d) {
    // numpy fftfreq convention: k < n/2 -> k, else k - n (the Nyquist bin is -n/2)
    return 2.0 * M_PI * (double)(k < (n + 1) / 2 ? k : k - n) / ((double)n * d);
}

struct KGrid {
    int nx, ny, nz, nxh;
    double dx, dy, dz;
};

// a Nyquist plane (k = n/2 of an even n): there G and -G are the same grid
// point, so a structure-factor phase exp(-i G.R) has no real-field
// representation; the local part leaves these planes out (energy and force alike)
__device__ __forceinline__ bool on_nyquist(const KGrid& g, size_t idx) {
    const int kx = (int)(idx % g.nxh);
    const size_t r = idx / g.nxh;
    const int ky = (int)(r % g.ny);
    const int kz = (int)(r / g.ny);
    return (g.nx % 2 == 0 && kx == g.nx / 2) || (g.ny % 2 == 0 && ky == g.ny / 2) ||
           (g.nz % 2 == 0 && kz == g.nz / 2);
}

__device__ __forceinline__ void kvec(const KGrid& g, size_t idx, double& gx, double& gy, double& gz) {
    const int kx = (int)(idx % g.nxh);
    const size_t r = idx / g.nxh;
    const int ky = (int)(r % g.ny);
    const int kz = (int)(r / g.ny);
    gx = freq(kx, g.nx, g.dx);
    gy = freq(ky, g.ny, g.dy);
    gz = freq(kz, g.nz, g.dz);
}

// f *= 4 pi / G^2 / N (G != 0), 0 at G = 0
__global__ void hartree_k_kernel(KGrid g, size_t M, double inv_n, cufftDoubleComplex* __restrict__ f) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < M; i += (size_t)gridDim.x * blockDim.x) {
        double gx, gy, gz;
        kvec(g, i, gx, gy, gz);
        const double g2 = gx * gx + gy * gy + gz * gz;
        const double s = g2 > 0.0 ? 4.0 * M_PI / g2 * inv_n : 0.0;
        f[i].x *= s;
        f[i].y *= s;
    }
}

// f *= A G^2 / (G^2 + q0^2) / N, 0 at G = 0
__global__ void kerker_k_kernel(KGrid g, size_t M, double inv_n, double amp, double q02,
                                cufftDoubleComplex* __restrict__ f) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < M; i += (size_t)gridDim.x * blockDim.x) {
        double gx, gy, gz;
        kvec(g, i, gx, gy, gz);
        const double g2 = gx * gx + gy * gy + gz * gz;
        const double s = g2 > 0.0 ? amp * g2 / (g2 + q02) * inv_n : 0.0;
        f[i].x *= s;
        f[i].y *= s;
    }
}

// GTH local part: V(G) = (1/Omega) sum_a v_a(G) exp(-i G.R_a),
// v(G) = -4 pi Z exp(-G^2 r^2 / 2) / G^2 + (2 pi)^(3/2) r^3 exp(-G^2 r^2 / 2) (C1 + C2 (3 - G^2 r^2)),
// G = 0: 2 pi Z r^2 + (2 pi)^(3/2) r^3 (C1 + 3 C2)  (Coulomb tail neutralised by the Hartree G = 0 term)
struct GthAtom {
    double x, y, z, zion, rloc, c1, c2;
};
__global__ void vloc_k_kernel(KGrid g, size_t M, double inv_omega, int na, const GthAtom* __restrict__ atoms,
                              cufftDoubleComplex* __restrict__ f) {
    const double tp32 = 15.749609945722419;   // (2 pi)^(3/2)
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < M; i += (size_t)gridDim.x * blockDim.x) {
        double gx, gy, gz;
        kvec(g, i, gx, gy, gz);
        const double g2 = gx * gx + gy * gy + gz * gz;
        double re = 0.0, im = 0.0;
        if (on_nyquist(g, i)) {
            f[i].x = 0.0;
            f[i].y = 0.0;
            continue;
        }
        for (int a = 0; a < na; ++a) {
            const GthAtom at = atoms[a];
            const double r2 = at.rloc * at.rloc;
            const double e = exp(-0.5 * g2 * r2);
            const double coul = g2 > 0.0 ? -4.0 * M_PI * at.zion * e / g2 : 2.0 * M_PI * at.zion * r2;
            const double v = coul + tp32 * r2 * at.rloc * e * (at.c1 + at.c2 * (3.0 - g2 * r2));
            double sn, cs;
            sincos(gx * at.x + gy * at.y + gz * at.z, &sn, &cs);
            re += v * cs;
            im -= v * sn;
        }
        f[i].x = re * inv_omega;
        f[i].y = im * inv_omega;
    }
}

// Force of the local part on every atom from a density's half-complex transform
// f (f = D2Z(rho), rho_G = f / N): F_a = -d/dR_a int rho V_loc
//   = sum_G G v_a(G) [sin(G.R_a) Re rho_G + cos(G.R_a) Im rho_G],
// the exact derivative of dV sum_r rho(r) V_loc(r) with V_loc the Fourier
// series above (Nyquist planes left out as there).  The half grid counts the
// kx = 0 plane once and the others twice.  partial[(a * 3 + d) * gridDim.x + blockIdx.x].
__global__ void __launch_bounds__(RB) local_force_kernel(KGrid g, size_t M, double inv_n, int na,
                                                         const GthAtom* __restrict__ atoms,
                                                         const cufftDoubleComplex* __restrict__ f,
                                                         double* __restrict__ partial) {
    __shared__ double sh[RB / 32];
    const double tp32 = 15.749609945722419;   // (2 pi)^(3/2)
    for (int a = 0; a < na; ++a) {
        const GthAtom at = atoms[a];
        const double r2 = at.rloc * at.rloc;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (size_t i = blockIdx.x * (size_t)RB + threadIdx.x; i < M; i += (size_t)gridDim.x * RB) {
            double gx, gy, gz;
            kvec(g, i, gx, gy, gz);
            const double g2 = gx * gx + gy * gy + gz * gz;
            if (g2 == 0.0 || on_nyquist(g, i)) continue;
            const int kx = (int)(i % g.nxh);
            const double w = kx == 0 ? 1.0 : 2.0;   // +-G pairs: kx and nx - kx
            const double e = exp(-0.5 * g2 * r2);
            const double v = -4.0 * M_PI * at.zion * e / g2 + tp32 * r2 * at.rloc * e * (at.c1 + at.c2 * (3.0 - g2 * r2));
            double sn, cs;
            sincos(gx * at.x + gy * at.y + gz * at.z, &sn, &cs);
            const double t = w * v * (sn * f[i].x + cs * f[i].y) * inv_n;
            fx += gx * t;
            fy += gy * t;
            fz += gz * t;
        }
        const double sx = block_sum(fx, sh), sy = block_sum(fy, sh), sz = block_sum(fz, sh);
        if (threadIdx.x == 0) {
            partial[(size_t)(a * 3 + 0) * gridDim.x + blockIdx.x] = sx;
            partial[(size_t)(a * 3 + 1) * gridDim.x + blockIdx.x] = sy;
            partial[(size_t)(a * 3 + 2) * gridDim.x + blockIdx.x] = sz;
        }
    }
}

// Radial-table local parts (qsb_scf_set_radial_local).  Per species the table
// holds the smooth part s(G) = v(G) + 4 pi z exp(-G^2 sigma^2 / 2) / G^2 on
// |G| = j dg (s(0) = v(0) + 2 pi z sigma^2); v(G) is s(|G|), by cubic Lagrange
// interpolation through the four nearest samples (s is even in G: index -1 is
// index 1), minus the Gaussian charge's 4 pi z exp(-G^2 sigma^2 / 2) / G^2, and
// s(0) - 2 pi z sigma^2 at G = 0 -- the finite-part convention of the GTH path.
struct TabAtom {
    double x, y, z;
    int sp;
};
struct TabSpecies {
    double z, sigma;
};
__device__ __forceinline__ double table_v(const double* __restrict__ tab, int n_g, double dg, double z, double sigma,
                                          double g2) {
    const double g = sqrt(g2);
    const double u = g / dg;
    const int j = (int)u;
    const double t = u - (double)j;
    const int im = j == 0 ? 1 : j - 1;
    const int i1 = min(j + 1, n_g - 1), i2 = min(j + 2, n_g - 1);
    const double wm = -t * (t - 1.0) * (t - 2.0) / 6.0, w0 = (t + 1.0) * (t - 1.0) * (t - 2.0) / 2.0;
    const double w1 = -(t + 1.0) * t * (t - 2.0) / 2.0, w2 = (t + 1.0) * t * (t - 1.0) / 6.0;
    const double sg = wm * tab[im] + w0 * tab[min(j, n_g - 1)] + w1 * tab[i1] + w2 * tab[i2];
    if (g2 > 0.0) return sg - 4.0 * M_PI * z * exp(-0.5 * g2 * sigma * sigma) / g2;
    return sg - 2.0 * M_PI * z * sigma * sigma;
}

__global__ void vloc_table_kernel(KGrid g, size_t M, double inv_omega, int na, const TabAtom* __restrict__ atoms,
                                  const TabSpecies* __restrict__ sp, const double* __restrict__ tab, int n_g,
                                  double dg, cufftDoubleComplex* __restrict__ f) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < M; i += (size_t)gridDim.x * blockDim.x) {
        double gx, gy, gz;
        kvec(g, i, gx, gy, gz);
        const double g2 = gx * gx + gy * gy + gz * gz;
        if (on_nyquist(g, i)) {
            f[i].x = 0.0;
            f[i].y = 0.0;
            continue;
        }
        double re = 0.0, im = 0.0;
        int last = -1;
        double v = 0.0;
        for (int a = 0; a < na; ++a) {
            const TabAtom at = atoms[a];
            if (at.sp != last) {
                v = table_v(tab + (size_t)at.sp * n_g, n_g, dg, sp[at.sp].z, sp[at.sp].sigma, g2);
                last = at.sp;
            }
            double sn, cs;
            sincos(gx * at.x + gy * at.y + gz * at.z, &sn, &cs);
            re += v * cs;
            im -= v * sn;
        }
        f[i].x = re * inv_omega;
        f[i].y = im * inv_omega;
    }
}

// the force of the table local parts, as local_force_kernel for the GTH ones
__global__ void __launch_bounds__(RB) local_force_table_kernel(KGrid g, size_t M, double inv_n, int na,
                                                               const TabAtom* __restrict__ atoms,
                                                               const TabSpecies* __restrict__ sp,
                                                               const double* __restrict__ tab, int n_g, double dg,
                                                               const cufftDoubleComplex* __restrict__ f,
                                                               double* __restrict__ partial) {
    __shared__ double sh[RB / 32];
    for (int a = 0; a < na; ++a) {
        const TabAtom at = atoms[a];
        const double* ts = tab + (size_t)at.sp * n_g;
        const double z = sp[at.sp].z, sigma = sp[at.sp].sigma;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (size_t i = blockIdx.x * (size_t)RB + threadIdx.x; i < M; i += (size_t)gridDim.x * RB) {
            double gx, gy, gz;
            kvec(g, i, gx, gy, gz);
            const double g2 = gx * gx + gy * gy + gz * gz;
            if (g2 == 0.0 || on_nyquist(g, i)) continue;
            const int kx = (int)(i % g.nxh);
            const double w = kx == 0 ? 1.0 : 2.0;
            const double v = table_v(ts, n_g, dg, z, sigma, g2);
            double sn, cs;
            sincos(gx * at.x + gy * at.y + gz * at.z, &sn, &cs);
            const double t = w * v * (sn * f[i].x + cs * f[i].y) * inv_n;
            fx += gx * t;
            fy += gy * t;
            fz += gz * t;
        }
        const double sx = block_sum(fx, sh), sy = block_sum(fy, sh), sz = block_sum(fz, sh);
        if (threadIdx.x == 0) {
            partial[(size_t)(a * 3 + 0) * gridDim.x + blockIdx.x] = sx;
            partial[(size_t)(a * 3 + 1) * gridDim.x + blockIdx.x] = sy;
            partial[(size_t)(a * 3 + 2) * gridDim.x + blockIdx.x] = sz;
        }
    }
}

inline int pw_blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

}  // namespace
}  // namespace qsb

struct qsb_scf {
    qsb_ham* ham = nullptr;
    qsb_eigensolver* es = nullptr;
    int nx = 0, ny = 0, nz = 0, nb = 0;
    size_t N = 0, M = 0;          // grid points, half-complex points
    double dx = 0, dy = 0, dz = 0, dV = 0;
    double n_el = 0, kbt = 0.01;
    double amp = 0.5, q0 = 0.8;
    double rho_tol = 0.0;         // int |rho_out - rho_in| / N_e bound of the stop (0: off)
    double xc_rho_min = 1.0e-8;   // LDA: exc = vxc = 0 below this density (Calc_XC_LDA's cut)
    bool xc_continuous = false;   // PZ correlation made continuous at rs = 1 (qsb_scf_set_xc)
    int xc_kind = 0;              // 0 LDA-PZ, 2 GGA-PBE (qsb_scf_set_xc)
    double* gga = nullptr;        // GGA: grad rho_s, then the flux (3 N)
    // FP64 polish of a mixed-precision run (qsb_scf_set_polish)
    qsb_eigensolver* polish_es = nullptr;
    int polish_max = 0;
    double polish_tol = 0.0;      // |dE| / atom of the polish's stop (0: the run's)
    double polish_rho_tol = 0.0;
    int last_polish_first = -1, last_polish_steps = 0;
    int depth = 6;
    int n_atoms = 0;
    // device fields
    double *vloc = nullptr, *rho_in = nullptr, *rho_out = nullptr, *vh = nullptr, *vxc = nullptr, *veff = nullptr;
    double *exc = nullptr, *tmp = nullptr, *hx = nullptr, *hist = nullptr;   // hist: depth x (rho_in, R)
    double *partial = nullptr, *sums = nullptr, *occ_dev = nullptr;
    const double** ptrs = nullptr;
    cufftDoubleComplex* fk = nullptr;
    qsb::GthAtom* atoms = nullptr;     // GTH local parts (device), set_gth_local
    // radial-table local parts (device), set_radial_local; used when tab_atoms is set
    qsb::TabAtom* tab_atoms = nullptr;
    qsb::TabSpecies* tab_species = nullptr;
    double* tab = nullptr;
    int tab_ng = 0;
    double tab_dg = 0.0;
    cufftHandle plan_f = 0, plan_b = 0;
    bool have_plans = false;
    // host
    std::vector<int> slots;       // history slots, oldest first
    std::vector<double> B;        // depth x depth residual inner products (by slot)
    std::vector<double> step_s;   // wall seconds of each step of the last run
    std::vector<double> step_res; // int |rho_out - rho_in| dV / N_e of each step of the last run
    // k-point runs (qsb_scf_set_kpoints / qsb_scf_run_kpoints)
    int n_k = 0;
    std::vector<double> kvec, kw; // 3 n_k Bloch vectors (bohr^-1), n_k weights (sum 1)
    std::vector<int> kown;        // k-points this context computes
    std::vector<int> knfix;       // soft-locking count of each k-point's solver calls
    double* hxc = nullptr;        // H X of one k-point's complex bundle (2 nb N)
    double* occ2 = nullptr;       // per-plane weights w_k f_nk of a complex bundle (2 nb)
    qsb_reduce_fn reduce = nullptr;   // sum over the ranks sharing the k-points (host buffers)
    void* reduce_user = nullptr;
    std::vector<double> hbuf;     // host staging of the density for the reduction
};

namespace qsb {
namespace {

#define QSB_CUFFT_TRY(expr)                                                                          \
    do {                                                                                             \
        const cufftResult r_ = (expr);                                                               \
        if (r_ != CUFFT_SUCCESS) return fail(QSB_ERR_CUDA, std::string("cuFFT call failed: ") + #expr); \
    } while (0)

KGrid kgrid(const qsb_scf* c) { return KGrid{c->nx, c->ny, c->nz, c->nx / 2 + 1, c->dx, c->dy, c->dz}; }

// dots[j] = int a_j b dV (b null: int a_j dV), na <= 8, deterministic
qsb_status dots(qsb_scf* c, int na, const double* const* a, const double* b, double* out, cudaStream_t s) {
    QSB_CUDA_TRY(cudaMemcpyAsync((void*)c->ptrs, a, na * sizeof(double*), cudaMemcpyHostToDevice, s));
    dot_partial_kernel<<<RBLOCKS, RB, 0, s>>>(c->N, na, c->ptrs, b, c->partial);
    row_sum_kernel<<<na, 32, 0, s>>>(na, RBLOCKS, c->partial, c->sums);
    QSB_CUDA_TRY(cudaMemcpyAsync(out, c->sums, na * sizeof(double), cudaMemcpyDeviceToHost, s));
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    for (int j = 0; j < na; ++j) out[j] *= c->dV;
    return QSB_OK;
}

// out = FFT^-1 [ factor(G) FFT[in] ]  (factor kernels divide by N)
enum class KOp { hartree, kerker };
qsb_status kspace(qsb_scf* c, KOp op, const double* in, double* out, cudaStream_t s) {
    QSB_CUFFT_TRY(cufftSetStream(c->plan_f, s));
    QSB_CUFFT_TRY(cufftSetStream(c->plan_b, s));
    QSB_CUFFT_TRY(cufftExecD2Z(c->plan_f, const_cast<double*>(in), c->fk));
    const double inv_n = 1.0 / (double)c->N;
    if (op == KOp::hartree) hartree_k_kernel<<<pw_blocks(c->M), 256, 0, s>>>(kgrid(c), c->M, inv_n, c->fk);
    else kerker_k_kernel<<<pw_blocks(c->M), 256, 0, s>>>(kgrid(c), c->M, inv_n, c->amp, c->q0 * c->q0, c->fk);
    QSB_CUFFT_TRY(cufftExecZ2D(c->plan_b, c->fk, out));
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

// vxc = V_xc[rho], exc = its energy density (may be null): LDA-PZ or GGA-PBE
qsb_status xc_eval(qsb_scf* c, const double* rho, double* exc, double* vxc, cudaStream_t s) {
    if (c->xc_kind == 2) {
        const Grid3 g{c->nx, c->ny, c->nz, c->dx, c->dy, c->dz};
        gga_grad_kernel<<<pw_blocks(c->N), 256, 0, s>>>(g, rho, c->gga);
        gga_pbe_point_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, rho, c->gga, exc, vxc);
        gga_div_kernel<<<pw_blocks(c->N), 256, 0, s>>>(g, c->gga, vxc);
    } else {
        lda_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, rho, exc, vxc, c->xc_rho_min, c->xc_continuous);
    }
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

// veff = vloc + V_H[rho_in] + V_xc[rho_in]
qsb_status potentials(qsb_scf* c, cudaStream_t s) {
    QSB_TRY(kspace(c, KOp::hartree, c->rho_in, c->vh, s));
    QSB_TRY(xc_eval(c, c->rho_in, nullptr, c->vxc, s));
    sum3_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, c->vloc, c->vh, c->vxc, c->veff);
    QSB_CUDA_TRY(cudaGetLastError());
    return qsb_ham_set_potential(c->ham, c->veff, 1);
}

// Fermi-Dirac occupations (SetOccupancy, source/SetOccupancy.h:7-18) at the mu of
// the bisection of mSetOccupancyTemperature (source/qumasun_base1.occupancy.h:76-170),
// refined by Newton steps to the exact electron count.  w (may be empty: all 1):
// the weight of each level's k-point, so that sum_i w_i occ_i = n_el with
// occ_i in [0, 2] (spin-paired); returns mu.
double fermi_weighted(const std::vector<double>& eig, const std::vector<double>& w, double n_el, double kbt,
                      std::vector<double>& occ) {
    const int n = (int)eig.size();
    occ.resize(n);
    auto wt = [&](int k) { return w.empty() ? 1.0 : w[k]; };
    auto fill = [&](double mu) {
        double sum = 0.0;
        for (int k = 0; k < n; ++k) {
            const double p = std::min((eig[k] - mu) / kbt, 80.0);
            occ[k] = 2.0 / (std::exp(p) + 1.0);
            sum += wt(k) * occ[k];
        }
        return sum;
    };
    double mu_min = *std::min_element(eig.begin(), eig.end()), mu_max = *std::max_element(eig.begin(), eig.end());
    double mu = 0.5 * (mu_min + mu_max);
    bool go = std::fabs(mu_max - mu_min) > 1.0e-9;
    fill(mu);
    double mu_last = mu;
    while (go) {
        const double ne = fill(mu);
        mu_last = mu;
        if (ne < n_el) mu_min = mu;
        else if (ne > n_el) mu_max = mu;
        else break;
        mu = 0.5 * (mu_min + mu_max);
        go = std::fabs(mu_max - mu_min) > 1.0e-9;
    }
    // the bisection leaves the electron count off by dN/dmu x ~1e-9 (1e-7 electrons
    // with a partly filled level at the Fermi energy), which moves the energy by
    // ~mu 1e-7: Newton steps on sum f(mu) = N_e from the last bisection point
    mu = mu_last;
    for (int it = 0; it < 8; ++it) {
        const double ne = fill(mu);
        double dn = 0.0;
        for (int k = 0; k < n; ++k) dn += wt(k) * occ[k] * (1.0 - 0.5 * occ[k]) / kbt;
        const double r = ne - n_el;
        if (std::fabs(r) <= 1e-14 * n_el || !(dn > 1e-300)) break;
        mu -= r / dn;
    }
    fill(mu);
    return mu;
}

void fermi(const std::vector<double>& eig, double n_el, double kbt, std::vector<double>& occ) {
    fermi_weighted(eig, std::vector<double>(), n_el, kbt, occ);
}

// Gaussian elimination with partial pivoting of the bordered DIIS system
void solve_bordered(std::vector<double> M, std::vector<double> b, std::vector<double>& x) {
    const int n = (int)b.size();
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(M[i * n + k]) > std::fabs(M[p * n + k])) p = i;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(M[k * n + j], M[p * n + j]);
            std::swap(b[k], b[p]);
        }
        if (M[k * n + k] == 0.0) continue;
        for (int i = k + 1; i < n; ++i) {
            const double f = M[i * n + k] / M[k * n + k];
            for (int j = k; j < n; ++j) M[i * n + j] -= f * M[k * n + j];
            b[i] -= f * b[k];
        }
    }
    x.assign(n, 0.0);
    for (int i = n - 1; i >= 0; --i) {
        double r = b[i];
        for (int j = i + 1; j < n; ++j) r -= M[i * n + j] * x[j];
        x[i] = M[i * n + i] != 0.0 ? r / M[i * n + i] : 0.0;
    }
}

double* hist_rin(qsb_scf* c, int slot) { return c->hist + (size_t)(2 * slot) * c->N; }
double* hist_res(qsb_scf* c, int slot) { return c->hist + (size_t)(2 * slot + 1) * c->N; }

// Kerker-preconditioned DIIS: rho_in <- sum a_i rho_in_i + P[sum a_i R_i]
qsb_status mix(qsb_scf* c, cudaStream_t s) {
    const int D = c->depth;
    int slot;
    if ((int)c->slots.size() < D) {
        slot = (int)c->slots.size();
    } else {
        slot = c->slots.front();
        c->slots.erase(c->slots.begin());
    }
    c->slots.push_back(slot);
    const size_t bytes = c->N * sizeof(double);
    QSB_CUDA_TRY(cudaMemcpyAsync(hist_rin(c, slot), c->rho_in, bytes, cudaMemcpyDeviceToDevice, s));
    sub_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, c->rho_out, c->rho_in, hist_res(c, slot));
    QSB_CUDA_TRY(cudaGetLastError());
    // inner products of the new residual with every stored one
    const int m = (int)c->slots.size();
    const double* a[8];
    for (int k = 0; k < m; ++k) a[k] = hist_res(c, c->slots[k]);
    double d[8];
    QSB_TRY(dots(c, m, a, hist_res(c, slot), d, s));
    for (int k = 0; k < m; ++k) {
        c->B[slot * D + c->slots[k]] = d[k];
        c->B[c->slots[k] * D + slot] = d[k];
    }
    // bordered system in history order, B scaled by its largest diagonal
    double sc = 0.0;
    for (int k = 0; k < m; ++k) sc = std::max(sc, c->B[c->slots[k] * D + c->slots[k]]);
    sc = std::max(sc, 1e-300);
    const int n = m + 1;
    std::vector<double> Mt(n * n, 0.0), rhs(n, 0.0), x;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) Mt[i * n + j] = c->B[c->slots[i] * D + c->slots[j]] / sc;
        Mt[i * n + m] = 1.0;
        Mt[m * n + i] = 1.0;
    }
    rhs[m] = 1.0;
    solve_bordered(Mt, rhs, x);
    Combo cr{}, cq{};
    cr.m = cq.m = m;
    for (int k = 0; k < m; ++k) {
        cr.in[k] = hist_rin(c, c->slots[k]);
        cq.in[k] = hist_res(c, c->slots[k]);
        cr.coef[k] = cq.coef[k] = x[k];
    }
    combo_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, cr, c->rho_in);
    combo_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, cq, c->tmp);
    QSB_CUDA_TRY(cudaGetLastError());
    QSB_TRY(kspace(c, KOp::kerker, c->tmp, c->tmp, s));
    add_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, c->tmp, c->rho_in);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

}  // namespace
}  // namespace qsb

using namespace qsb;

extern "C" {

qsb_status qsb_density(int64_t N, int nb, const double* X, const double* occupations, double* rho, void* stream) {
    if (N <= 0 || nb < 0 || !X || !occupations || !rho) return fail(QSB_ERR_INVALID, "density: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    double* occ = nullptr;
    QSB_CUDA_TRY(cudaMallocAsync((void**)&occ, std::max(nb, 1) * sizeof(double), s));
    QSB_CUDA_TRY(cudaMemcpyAsync(occ, occupations, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    density_kernel<<<pw_blocks((size_t)N), 256, 0, s>>>((size_t)N, nb, X, occ, rho);
    QSB_CUDA_TRY(cudaGetLastError());
    QSB_CUDA_TRY(cudaFreeAsync(occ, s));
    return QSB_OK;
}

qsb_status qsb_lda_pz(int64_t n, const double* rho, double* exc, double* vxc, void* stream) {
    if (n <= 0 || !rho || !vxc) return fail(QSB_ERR_INVALID, "lda_pz: bad argument");
    lda_kernel<<<pw_blocks((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, rho, exc, vxc);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

qsb_status qsb_scf_create(qsb_scf** out, qsb_ham* ham, qsb_eigensolver* es, int nb, double num_electrons) {
    if (!out || !ham || !es || nb <= 0 || !(num_electrons > 0.0) || num_electrons > 2.0 * nb)
        return fail(QSB_ERR_INVALID, "scf_create: bad argument (need ham, solver, nb > 0, 0 < electrons <= 2 nb)");
    if (ham->nx < 2 || ham->ny < 2 || ham->nz < 2) return fail(QSB_ERR_INVALID, "scf_create: grid too small");
    auto* c = new qsb_scf;
    c->ham = ham;
    c->es = es;
    c->nx = ham->nx; c->ny = ham->ny; c->nz = ham->nz;
    c->dx = ham->dx; c->dy = ham->dy; c->dz = ham->dz;
    c->N = (size_t)c->nx * c->ny * c->nz;
    c->M = (size_t)c->nz * c->ny * (c->nx / 2 + 1);
    c->dV = c->dx * c->dy * c->dz;
    c->nb = nb;
    c->n_el = num_electrons;
    *out = c;
    auto cleanup = [&](qsb_status st) {
        qsb_scf_destroy(c);
        *out = nullptr;
        return st;
    };
    const size_t fb = c->N * sizeof(double);
    double** fields[] = {&c->vloc, &c->rho_in, &c->rho_out, &c->vh, &c->vxc, &c->veff, &c->exc, &c->tmp};
    for (double** f : fields) {
        if (cudaMalloc((void**)f, fb) != cudaSuccess) return cleanup(fail(QSB_ERR_NOMEM, "scf_create: device allocation"));
        cudaMemset(*f, 0, fb);
    }
    if (cudaMalloc((void**)&c->hist, 2 * (size_t)c->depth * fb) != cudaSuccess ||
        cudaMalloc((void**)&c->hx, (size_t)nb * fb) != cudaSuccess ||
        cudaMalloc((void**)&c->partial, (size_t)std::max(8, nb) * RBLOCKS * 2 * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c->sums, (size_t)std::max(8, 2 * nb) * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c->occ_dev, (size_t)nb * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c->ptrs, 8 * sizeof(double*)) != cudaSuccess ||
        cudaMalloc((void**)&c->fk, c->M * sizeof(cufftDoubleComplex)) != cudaSuccess)
        return cleanup(fail(QSB_ERR_NOMEM, "scf_create: device allocation"));
    if (cufftPlan3d(&c->plan_f, c->nz, c->ny, c->nx, CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&c->plan_b, c->nz, c->ny, c->nx, CUFFT_Z2D) != CUFFT_SUCCESS)
        return cleanup(fail(QSB_ERR_CUDA, "scf_create: cuFFT plan"));
    c->have_plans = true;
    c->B.assign((size_t)c->depth * c->depth, 0.0);
    return QSB_OK;
}

qsb_status qsb_scf_destroy(qsb_scf* c) {
    if (!c) return QSB_OK;
    double* fields[] = {c->vloc, c->rho_in, c->rho_out, c->vh, c->vxc, c->veff, c->exc, c->tmp, c->hist, c->hx,
                        c->partial, c->sums, c->occ_dev};
    for (double* f : fields)
        if (f) cudaFree(f);
    if (c->ptrs) cudaFree((void*)c->ptrs);
    if (c->hxc) cudaFree(c->hxc);
    if (c->occ2) cudaFree(c->occ2);
    if (c->fk) cudaFree(c->fk);
    void* loc[5] = {c->atoms, c->tab_atoms, c->tab_species, c->tab, c->gga};
    for (void* q : loc)
        if (q) cudaFree(q);
    if (c->have_plans) {
        cufftDestroy(c->plan_f);
        cufftDestroy(c->plan_b);
    }
    delete c;
    return QSB_OK;
}

qsb_status qsb_scf_set_mixing(qsb_scf* c, double amplitude, double q0, int depth) {
    if (!c || !(amplitude > 0.0) || !(q0 >= 0.0) || depth < 1 || depth > 8)
        return fail(QSB_ERR_INVALID, "scf_set_mixing: need amplitude > 0, q0 >= 0, 1 <= depth <= 8");
    if (depth != c->depth) {
        double* h = nullptr;
        if (cudaMalloc((void**)&h, 2 * (size_t)depth * c->N * sizeof(double)) != cudaSuccess)
            return fail(QSB_ERR_NOMEM, "scf_set_mixing: device allocation");
        cudaFree(c->hist);
        c->hist = h;
        c->depth = depth;
    }
    c->amp = amplitude;
    c->q0 = q0;
    c->B.assign((size_t)depth * depth, 0.0);
    c->slots.clear();
    return QSB_OK;
}

qsb_status qsb_scf_set_density_tolerance(qsb_scf* c, double rho_tol) {
    if (!c || !(rho_tol >= 0.0)) return fail(QSB_ERR_INVALID, "scf_set_density_tolerance: need rho_tol >= 0");
    c->rho_tol = rho_tol;
    return QSB_OK;
}

qsb_status qsb_scf_set_polish(qsb_scf* c, qsb_eigensolver* es_fp64, int max_steps, double tol_per_atom,
                              double rho_tol) {
    if (!c) return fail(QSB_ERR_INVALID, "scf_set_polish: null context");
    if (!es_fp64 || max_steps <= 0) {
        c->polish_es = nullptr;
        c->polish_max = 0;
        return QSB_OK;
    }
    if (!(rho_tol >= 0.0) || !(tol_per_atom >= 0.0))
        return fail(QSB_ERR_INVALID, "scf_set_polish: need tol_per_atom >= 0 and rho_tol >= 0");
    int64_t N = 0;
    int nmax = 0, cplx = 0, mixed = 0;
    eigensolver_shape(es_fp64, &N, &nmax, &cplx, &mixed);
    if (mixed || cplx || (size_t)N != c->N || nmax < c->nb)
        return fail(QSB_ERR_INVALID, "scf_set_polish: needs a real FP64 solver context of the SCF's grid and bands");
    c->polish_es = es_fp64;
    c->polish_max = max_steps;
    c->polish_tol = tol_per_atom;
    c->polish_rho_tol = rho_tol;
    return QSB_OK;
}

qsb_status qsb_scf_polish_stats(const qsb_scf* c, int* first_step, int* steps) {
    if (!c) return fail(QSB_ERR_INVALID, "scf_polish_stats: null context");
    if (first_step) *first_step = c->last_polish_first;
    if (steps) *steps = c->last_polish_steps;
    return QSB_OK;
}

qsb_status qsb_scf_set_xc(qsb_scf* c, int pz_variant, double rho_min) {
    if (!c || pz_variant < 0 || pz_variant > 2 || !(rho_min >= 1e-30))
        return fail(QSB_ERR_INVALID, "scf_set_xc: need variant 0, 1 (LDA-PZ) or 2 (GGA-PBE) and rho_min >= 1e-30");
    if (pz_variant == 2 && !c->gga) QSB_CUDA_TRY(cudaMalloc((void**)&c->gga, 3 * c->N * sizeof(double)));
    c->xc_kind = pz_variant == 2 ? 2 : 0;
    c->xc_continuous = pz_variant == 1;
    c->xc_rho_min = rho_min;
    return QSB_OK;
}

qsb_status qsb_gga_pbe(int nx, int ny, int nz, double dx, double dy, double dz, const double* rho, double* exc,
                       double* vxc, void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || !(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !rho || !vxc)
        return fail(QSB_ERR_INVALID, "gga_pbe: bad argument");
    const size_t N = (size_t)nx * ny * nz;
    cudaStream_t s = (cudaStream_t)stream;
    double* work = nullptr;
    QSB_CUDA_TRY(cudaMalloc((void**)&work, 3 * N * sizeof(double)));
    const Grid3 g{nx, ny, nz, dx, dy, dz};
    gga_grad_kernel<<<pw_blocks(N), 256, 0, s>>>(g, rho, work);
    gga_pbe_point_kernel<<<pw_blocks(N), 256, 0, s>>>(N, rho, work, exc, vxc);
    gga_div_kernel<<<pw_blocks(N), 256, 0, s>>>(g, work, vxc);
    const cudaError_t e = cudaGetLastError();
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(work);
    if (e != cudaSuccess) return cuda_fail(e, "gga_pbe");
    if (e2 != cudaSuccess) return cuda_fail(e2, "gga_pbe");
    return QSB_OK;
}

qsb_status qsb_scf_set_smearing(qsb_scf* c, double kbt) {
    if (!c || !(kbt > 0.0)) return fail(QSB_ERR_INVALID, "scf_set_smearing: need kbT > 0");
    c->kbt = kbt;
    return QSB_OK;
}

namespace {
void free_local_parts(qsb_scf* c) {
    void* p[4] = {c->atoms, c->tab_atoms, c->tab_species, c->tab};
    for (void* q : p)
        if (q) cudaFree(q);
    c->atoms = nullptr;
    c->tab_atoms = nullptr;
    c->tab_species = nullptr;
    c->tab = nullptr;
    c->n_atoms = 0;
}
}  // namespace

qsb_status qsb_scf_set_gth_local(qsb_scf* c, int n_atoms, const double* pos, const int* species, int n_species,
                                 const double* zion, const double* rloc, const double* c1, const double* c2) {
    if (!c || n_atoms <= 0 || !pos || !species || n_species <= 0 || !zion || !rloc || !c1 || !c2)
        return fail(QSB_ERR_INVALID, "scf_set_gth_local: bad argument");
    std::vector<GthAtom> at(n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
        const int sp = species[a];
        if (sp < 0 || sp >= n_species || !(rloc[sp] > 0.0)) return fail(QSB_ERR_INVALID, "scf_set_gth_local: bad species");
        at[a] = GthAtom{pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], zion[sp], rloc[sp], c1[sp], c2[sp]};
    }
    free_local_parts(c);
    GthAtom* d = nullptr;
    QSB_CUDA_TRY(cudaMalloc((void**)&d, n_atoms * sizeof(GthAtom)));
    QSB_CUDA_TRY(cudaMemcpy(d, at.data(), n_atoms * sizeof(GthAtom), cudaMemcpyHostToDevice));
    const double omega = (double)c->N * c->dV;
    vloc_k_kernel<<<pw_blocks(c->M), 256>>>(kgrid(c), c->M, 1.0 / omega, n_atoms, d, c->fk);
    const cudaError_t e = cudaGetLastError();
    QSB_CUFFT_TRY(cufftSetStream(c->plan_b, 0));
    QSB_CUFFT_TRY(cufftExecZ2D(c->plan_b, c->fk, c->vloc));
    QSB_CUDA_TRY(cudaDeviceSynchronize());
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "vloc_k_kernel");
    }
    c->atoms = d;
    c->n_atoms = n_atoms;
    return QSB_OK;
}

qsb_status qsb_scf_set_radial_local(qsb_scf* c, int n_atoms, const double* pos, const int* species, int n_species,
                                    const double* z, const double* sigma, int n_g, double dg, const double* table) {
    if (!c || n_atoms <= 0 || !pos || !species || n_species <= 0 || !z || !sigma || n_g < 4 || !(dg > 0.0) || !table)
        return fail(QSB_ERR_INVALID, "scf_set_radial_local: bad argument");
    // the table must reach past the largest |G| of the grid by the interpolation stencil
    const double gmax = std::sqrt(std::pow(M_PI / c->dx, 2) + std::pow(M_PI / c->dy, 2) + std::pow(M_PI / c->dz, 2));
    if ((double)(n_g - 3) * dg < gmax)
        return fail(QSB_ERR_INVALID, "scf_set_radial_local: table ends at |G| = " + std::to_string((n_g - 3) * dg) +
                                         " below the grid's " + std::to_string(gmax) + " (+ 3 samples)");
    std::vector<TabAtom> at(n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
        const int sp = species[a];
        if (sp < 0 || sp >= n_species) return fail(QSB_ERR_INVALID, "scf_set_radial_local: bad species");
        at[a] = TabAtom{pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], sp};
    }
    std::vector<TabSpecies> spc(n_species);
    std::vector<double> smooth((size_t)n_species * n_g);
    for (int k = 0; k < n_species; ++k) {
        if (!(sigma[k] > 0.0)) return fail(QSB_ERR_INVALID, "scf_set_radial_local: sigma must be > 0");
        spc[k] = TabSpecies{z[k], sigma[k]};
        for (int j = 0; j < n_g; ++j) {
            const double v = table[(size_t)k * n_g + j];
            if (!std::isfinite(v)) return fail(QSB_ERR_INVALID, "scf_set_radial_local: non-finite table value");
            const double g = j * dg;
            smooth[(size_t)k * n_g + j] =
                j == 0 ? v + 2.0 * M_PI * z[k] * sigma[k] * sigma[k]
                       : v + 4.0 * M_PI * z[k] * std::exp(-0.5 * g * g * sigma[k] * sigma[k]) / (g * g);
        }
    }
    free_local_parts(c);
    QSB_CUDA_TRY(cudaMalloc((void**)&c->tab_atoms, n_atoms * sizeof(TabAtom)));
    QSB_CUDA_TRY(cudaMalloc((void**)&c->tab_species, n_species * sizeof(TabSpecies)));
    QSB_CUDA_TRY(cudaMalloc((void**)&c->tab, smooth.size() * sizeof(double)));
    QSB_CUDA_TRY(cudaMemcpy(c->tab_atoms, at.data(), n_atoms * sizeof(TabAtom), cudaMemcpyHostToDevice));
    QSB_CUDA_TRY(cudaMemcpy(c->tab_species, spc.data(), n_species * sizeof(TabSpecies), cudaMemcpyHostToDevice));
    QSB_CUDA_TRY(cudaMemcpy(c->tab, smooth.data(), smooth.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->tab_ng = n_g;
    c->tab_dg = dg;
    const double omega = (double)c->N * c->dV;
    vloc_table_kernel<<<pw_blocks(c->M), 256>>>(kgrid(c), c->M, 1.0 / omega, n_atoms, c->tab_atoms, c->tab_species,
                                                c->tab, n_g, dg, c->fk);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        free_local_parts(c);
        return cuda_fail(e, "vloc_table_kernel");
    }
    QSB_CUFFT_TRY(cufftSetStream(c->plan_b, 0));
    QSB_CUFFT_TRY(cufftExecZ2D(c->plan_b, c->fk, c->vloc));
    QSB_CUDA_TRY(cudaDeviceSynchronize());
    c->n_atoms = n_atoms;
    return QSB_OK;
}

qsb_status qsb_scf_local_forces(qsb_scf* c, const double* rho_dev, double* forces) {
    if (!c || !forces) return fail(QSB_ERR_INVALID, "scf_local_forces: bad argument");
    if (c->n_atoms <= 0) return fail(QSB_ERR_STATE, "scf_local_forces: no local potential (qsb_scf_set_gth_local)");
    const double* rho = rho_dev ? rho_dev : c->rho_out;
    QSB_CUFFT_TRY(cufftSetStream(c->plan_f, 0));
    QSB_CUFFT_TRY(cufftExecD2Z(c->plan_f, const_cast<double*>(rho), c->fk));
    const int blocks = RBLOCKS / 4;
    const int rows = 3 * c->n_atoms;
    double* part = nullptr;
    double* sums = nullptr;
    QSB_CUDA_TRY(cudaMalloc((void**)&part, (size_t)rows * blocks * sizeof(double)));
    if (cudaMalloc((void**)&sums, (size_t)rows * sizeof(double)) != cudaSuccess) {
        cudaFree(part);
        return fail(QSB_ERR_NOMEM, "scf_local_forces: device allocation");
    }
    if (c->tab_atoms)
        local_force_table_kernel<<<blocks, RB>>>(kgrid(c), c->M, 1.0 / (double)c->N, c->n_atoms, c->tab_atoms,
                                                 c->tab_species, c->tab, c->tab_ng, c->tab_dg, c->fk, part);
    else
        local_force_kernel<<<blocks, RB>>>(kgrid(c), c->M, 1.0 / (double)c->N, c->n_atoms, c->atoms, c->fk, part);
    row_sum_kernel<<<rows, 32>>>(rows, blocks, part, sums);
    std::vector<double> h(rows);
    const cudaError_t e = cudaMemcpy(h.data(), sums, rows * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(part);
    cudaFree(sums);
    if (e != cudaSuccess) return cuda_fail(e, "scf_local_forces");
    for (int k = 0; k < rows; ++k) {
        if (!std::isfinite(h[k])) return fail(QSB_ERR_NUMERIC, "scf_local_forces: non-finite value");
        forces[k] += h[k];
    }
    return QSB_OK;
}

qsb_status qsb_scf_step_residuals(qsb_scf* c, double* residuals, int max, int* n) {
    if (!c || !n || (max > 0 && !residuals)) return fail(QSB_ERR_INVALID, "scf_step_residuals: bad argument");
    *n = (int)c->step_res.size();
    for (int k = 0; k < std::min(max, *n); ++k) residuals[k] = c->step_res[k];
    return QSB_OK;
}

qsb_status qsb_scf_step_seconds(qsb_scf* c, double* seconds, int max, int* n) {
    if (!c || !n || (max > 0 && !seconds)) return fail(QSB_ERR_INVALID, "scf_step_seconds: bad argument");
    *n = (int)c->step_s.size();
    for (int k = 0; k < std::min(max, *n); ++k) seconds[k] = c->step_s[k];
    return QSB_OK;
}

qsb_status qsb_scf_get_field(qsb_scf* c, int which, double* out_dev) {
    if (!c || !out_dev) return fail(QSB_ERR_INVALID, "scf_get_field: bad argument");
    const double* f = which == 0 ? c->rho_out : which == 1 ? c->vloc : which == 2 ? c->veff : which == 3 ? c->rho_in
                                                                                                        : nullptr;
    if (!f) return fail(QSB_ERR_INVALID, "scf_get_field: which is 0 (rho), 1 (V_loc), 2 (V_eff) or 3 (mixed rho)");
    QSB_CUDA_TRY(cudaMemcpy(out_dev, f, c->N * sizeof(double), cudaMemcpyDeviceToDevice));
    return QSB_OK;
}

qsb_status qsb_scf_run(qsb_scf* c, double* X, double* keep, int lobpcg_iters, int max_steps, double tol_per_atom,
                       double* energies, int* steps, double* eigen_values, double* occupations, void* stream) {
    if (!c || !X || !keep || lobpcg_iters <= 0 || max_steps <= 0 || !(tol_per_atom > 0.0) || !energies || !steps)
        return fail(QSB_ERR_INVALID, "scf_run: bad argument");
    if (c->n_atoms <= 0) return fail(QSB_ERR_STATE, "scf_run: no local potential (qsb_scf_set_gth_local)");
    QSB_TRY(qsb_eigensolver_set_hamiltonian(c->es, c->ham, 0.0, 0.0, 0.0));
    if (c->polish_es) QSB_TRY(qsb_eigensolver_set_hamiltonian(c->polish_es, c->ham, 0.0, 0.0, 0.0));
    c->last_polish_first = -1;
    c->last_polish_steps = 0;
    bool polishing = false;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = c->nb;
    const size_t N = c->N;
    std::vector<double> ev(nb, 0.0), rq(nb), occ(nb), pxy(nb), pxx(nb);
    // initial density: the input states with the zero-temperature filling
    // (mSetOccupancyZero, source/qumasun_base1.occupancy.h:35-66)
    {
        double left = c->n_el;
        for (int n = 0; n < nb; ++n) {
            occ[n] = std::min(2.0, std::max(left, 0.0));
            left -= occ[n];
        }
    }
    QSB_CUDA_TRY(cudaMemcpyAsync(c->occ_dev, occ.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s));
    density_kernel<<<pw_blocks(N), 256, 0, s>>>(N, nb, X, c->occ_dev, c->rho_in);
    QSB_CUDA_TRY(cudaGetLastError());
    c->slots.clear();
    std::fill(c->B.begin(), c->B.end(), 0.0);
    double e_prev = 0.0;
    *steps = 0;
    c->step_s.clear();
    c->step_res.clear();
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    auto t_prev = std::chrono::steady_clock::now();
    for (int step = 0; step < max_steps; ++step) {
        QSB_TRY(potentials(c, s));
        // the polish's first FP64 call starts without search directions: the kept
        // P of the mixed solver is a direction of its FP32 iterations
        const bool fresh = step == 0 || (polishing && c->last_polish_steps == 0);
        QSB_TRY(qsb_lobpcg_d(polishing ? c->polish_es : c->es, c->dV, nb, lobpcg_iters, ev.data(), X, keep,
                             fresh ? 1 : 0, stream));
        if (polishing) ++c->last_polish_steps;
        // FP64 Rayleigh quotients of the states (the energy and the occupations use these)
        QSB_TRY(qsb_ham_apply(c->ham, QSB_F64, 0, nb, X, c->hx, 0.0, 0.0, 0.0, stream));
        band_dot_kernel<<<dim3(RBLOCKS / 4, nb), RB, 0, s>>>(N, X, c->hx, c->partial, c->partial + (size_t)nb * (RBLOCKS / 4));
        row_sum_kernel<<<2 * nb, 32, 0, s>>>(2 * nb, RBLOCKS / 4, c->partial, c->sums);
        QSB_CUDA_TRY(cudaGetLastError());
        std::vector<double> sums(2 * nb);
        QSB_CUDA_TRY(cudaMemcpyAsync(sums.data(), c->sums, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, s));
        QSB_CUDA_TRY(cudaStreamSynchronize(s));
        for (int n = 0; n < nb; ++n) {
            if (!(sums[nb + n] > 0.0) || !std::isfinite(sums[n])) return fail(QSB_ERR_NUMERIC, "scf_run: bad band norm");
            rq[n] = sums[n] / sums[nb + n];
        }
        fermi(rq, c->n_el, c->kbt, occ);
        QSB_CUDA_TRY(cudaMemcpyAsync(c->occ_dev, occ.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s));
        density_kernel<<<pw_blocks(N), 256, 0, s>>>(N, nb, X, c->occ_dev, c->rho_out);
        // energy of the output density: sum occ rq - int (V_H + V_xc)[rho_in] rho_out + E_H + E_xc [rho_out]
        sub_kernel<<<pw_blocks(N), 256, 0, s>>>(N, c->veff, c->vloc, c->tmp);
        QSB_TRY(kspace(c, KOp::hartree, c->rho_out, c->vh, s));
        QSB_TRY(xc_eval(c, c->rho_out, c->exc, c->vxc, s));
        QSB_CUDA_TRY(cudaGetLastError());
        double d2[2], exc_int;
        {
            const double* a[2] = {c->tmp, c->vh};
            QSB_TRY(dots(c, 2, a, c->rho_out, d2, s));
            const double* e[1] = {c->exc};
            QSB_TRY(dots(c, 1, e, nullptr, &exc_int, s));
        }
        double eband = 0.0;
        for (int n = 0; n < nb; ++n) eband += occ[n] * rq[n];
        const double etot = eband - d2[0] + 0.5 * d2[1] + exc_int;
        energies[step] = etot;
        *steps = step + 1;
        // the step ends with the energy on the host (the inner products synchronized the stream)
        const auto t_now = std::chrono::steady_clock::now();
        c->step_s.push_back(std::chrono::duration<double>(t_now - t_prev).count());
        t_prev = t_now;
        // density residual int |rho_out - rho_in| dV / N_e, recorded every step
        // (the RHO_ETOT convergence quantity of the reference's loop)
        {
            l1_diff_partial_kernel<<<RBLOCKS, RB, 0, s>>>(N, c->rho_out, c->rho_in, c->partial);
            row_sum_kernel<<<1, 32, 0, s>>>(1, RBLOCKS, c->partial, c->sums);
            double l1 = 0.0;
            QSB_CUDA_TRY(cudaMemcpyAsync(&l1, c->sums, sizeof(double), cudaMemcpyDeviceToHost, s));
            QSB_CUDA_TRY(cudaStreamSynchronize(s));
            c->step_res.push_back(l1 * c->dV / c->n_el);
        }
        const double etol = polishing && c->polish_tol > 0.0 ? c->polish_tol : tol_per_atom;
        bool done = step > 0 && std::fabs(etot - e_prev) / c->n_atoms < etol;
        const double rho_tol = polishing ? c->polish_rho_tol : c->rho_tol;
        if (done && rho_tol > 0.0) done = c->step_res.back() < rho_tol;
        e_prev = etot;
        if (polishing && c->last_polish_steps >= c->polish_max) done = true;
        if (done && !polishing && c->polish_es && step + 1 < max_steps) {
            // the mixed run has met its stop: go on in FP64 from its states and
            // density, with a fresh mixing history (the kept residuals carry the
            // FP32 states' noise, which would stay in the DIIS extrapolation)
            polishing = true;
            c->last_polish_first = step + 1;
            c->slots.clear();
            std::fill(c->B.begin(), c->B.end(), 0.0);
            done = false;
        }
        if (done) break;
        QSB_TRY(mix(c, s));
    }
    if (eigen_values) std::copy(rq.begin(), rq.end(), eigen_values);
    if (occupations) std::copy(occ.begin(), occ.end(), occupations);
    return QSB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// k-point SCF: the loop of QUMASUN_KPOINT::Execute over (k) groups
// (source/qumasun_kpoint.scfloop.h:61-258, qumasun_kpoint.lobpcg.h:78-106), the
// density summed over k (qumasun_base1.density.h:19-105, mReduceFieldInSamePlace)
// and the Fermi level over all (k, band) levels with the k weights.
// ---------------------------------------------------------------------------
namespace qsb {
namespace {

// host-staged sum of n doubles over the ranks sharing the k-points (device buffer)
qsb_status reduce_device(qsb_scf* c, double* dev, size_t n, cudaStream_t s) {
    if (!c->reduce) return QSB_OK;
    c->hbuf.resize(n);
    QSB_CUDA_TRY(cudaMemcpyAsync(c->hbuf.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    if (c->reduce(c->reduce_user, c->hbuf.data(), (int64_t)n) != 0)
        return fail(QSB_ERR_STATE, "scf_run_kpoints: the reduction callback failed");
    QSB_CUDA_TRY(cudaMemcpyAsync(dev, c->hbuf.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    return QSB_OK;
}

qsb_status reduce_host(qsb_scf* c, double* h, size_t n) {
    if (!c->reduce) return QSB_OK;
    if (c->reduce(c->reduce_user, h, (int64_t)n) != 0)
        return fail(QSB_ERR_STATE, "scf_run_kpoints: the reduction callback failed");
    return QSB_OK;
}

// rho (+)= sum_n occ2[2n] re_n^2 + occ2[2n+1] im_n^2 over a complex SoA bundle
qsb_status density_complex(qsb_scf* c, int nb, const double* X, const std::vector<double>& wocc, double* rho,
                           bool accumulate, cudaStream_t s) {
    std::vector<double> o2(2 * (size_t)nb);
    for (int n = 0; n < nb; ++n) o2[2 * n] = o2[2 * n + 1] = wocc[n];
    QSB_CUDA_TRY(cudaMemcpyAsync(c->occ2, o2.data(), o2.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    double* dst = accumulate ? c->tmp : rho;
    density_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, 2 * nb, X, c->occ2, dst);
    if (accumulate) add_kernel<<<pw_blocks(c->N), 256, 0, s>>>(c->N, c->tmp, rho);
    QSB_CUDA_TRY(cudaGetLastError());
    // the host copy of o2 must outlive the copy: synchronize before it goes
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    return QSB_OK;
}

}  // namespace
}  // namespace qsb

extern "C" {

qsb_status qsb_fermi_occupations(int n, const double* eig, const double* weights, double n_el, double kbt,
                                 double* occ, double* mu) {
    if (n <= 0 || !eig || !occ || !(kbt > 0.0) || !(n_el > 0.0))
        return fail(QSB_ERR_INVALID, "fermi_occupations: bad argument");
    std::vector<double> e(eig, eig + n), w, o;
    if (weights) w.assign(weights, weights + n);
    double cap = 0.0;
    for (int k = 0; k < n; ++k) {
        if (!std::isfinite(e[k]) || (weights && !(w[k] >= 0.0))) return fail(QSB_ERR_INVALID, "fermi_occupations: bad value");
        cap += 2.0 * (weights ? w[k] : 1.0);
    }
    if (n_el > cap) return fail(QSB_ERR_INVALID, "fermi_occupations: more electrons than the levels hold");
    const double m = fermi_weighted(e, w, n_el, kbt, o);
    std::copy(o.begin(), o.end(), occ);
    if (mu) *mu = m;
    return QSB_OK;
}

qsb_status qsb_scf_set_kpoints(qsb_scf* c, int n_k, const double* kvec, const double* weights, const int* owned) {
    if (!c || n_k < 1 || !kvec || !weights) return fail(QSB_ERR_INVALID, "scf_set_kpoints: bad argument");
    int64_t N = 0;
    int nmax = 0, cplx = 0, mixed = 0;
    eigensolver_shape(c->es, &N, &nmax, &cplx, &mixed);
    if (!cplx) return fail(QSB_ERR_INVALID, "scf_set_kpoints: needs a complex eigensolver context");
    double wsum = 0.0;
    for (int k = 0; k < n_k; ++k) {
        if (!(weights[k] > 0.0)) return fail(QSB_ERR_INVALID, "scf_set_kpoints: weights must be > 0");
        wsum += weights[k];
    }
    if (std::fabs(wsum - 1.0) > 1e-12) return fail(QSB_ERR_INVALID, "scf_set_kpoints: weights must sum to 1");
    const size_t fb = c->N * sizeof(double);
    if (!c->hxc && cudaMalloc((void**)&c->hxc, 2 * (size_t)c->nb * fb) != cudaSuccess)
        return fail(QSB_ERR_NOMEM, "scf_set_kpoints: device allocation");
    if (!c->occ2 && cudaMalloc((void**)&c->occ2, 2 * (size_t)c->nb * sizeof(double)) != cudaSuccess)
        return fail(QSB_ERR_NOMEM, "scf_set_kpoints: device allocation");
    c->n_k = n_k;
    c->kvec.assign(kvec, kvec + 3 * (size_t)n_k);
    c->kw.assign(weights, weights + n_k);
    c->kown.assign(n_k, 1);
    if (owned)
        for (int k = 0; k < n_k; ++k) c->kown[k] = owned[k] != 0;
    c->knfix.assign(n_k, 0);
    return QSB_OK;
}

qsb_status qsb_scf_set_reduce(qsb_scf* c, qsb_reduce_fn fn, void* user) {
    if (!c) return fail(QSB_ERR_INVALID, "scf_set_reduce: null context");
    c->reduce = fn;
    c->reduce_user = user;
    return QSB_OK;
}

qsb_status qsb_scf_run_kpoints(qsb_scf* c, double* const* X, double* const* keep, int lobpcg_iters, int max_steps,
                               double tol_per_atom, double* energies, int* steps, double* eigen_values,
                               double* occupations, void* stream) {
    if (!c || !X || !keep || lobpcg_iters <= 0 || max_steps <= 0 || !(tol_per_atom > 0.0) || !energies || !steps)
        return fail(QSB_ERR_INVALID, "scf_run_kpoints: bad argument");
    if (c->n_k < 1) return fail(QSB_ERR_STATE, "scf_run_kpoints: no k-points (qsb_scf_set_kpoints)");
    if (c->n_atoms <= 0) return fail(QSB_ERR_STATE, "scf_run_kpoints: no local potential (qsb_scf_set_gth_local)");
    for (int k = 0; k < c->n_k; ++k) {
        if (c->kown[k] && (!X[k] || !keep[k])) return fail(QSB_ERR_INVALID, "scf_run_kpoints: null bundle of an owned k-point");
        if (!c->kown[k] && !c->reduce)
            return fail(QSB_ERR_STATE, "scf_run_kpoints: k-points owned elsewhere need a reduction (qsb_scf_set_reduce)");
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = c->nb, nk = c->n_k;
    const size_t N = c->N;
    std::vector<double> rq((size_t)nk * nb, 0.0), occ((size_t)nk * nb, 0.0), wl((size_t)nk * nb), wocc(nb);
    for (int k = 0; k < nk; ++k)
        for (int n = 0; n < nb; ++n) wl[(size_t)k * nb + n] = c->kw[k];
    std::vector<double> ev(nb), sums(2 * (size_t)nb);
    auto own_first = [&]() {
        for (int k = 0; k < nk; ++k)
            if (c->kown[k]) return k;
        return -1;
    };
    // initial density: the input states of every k-point with the lowest bands
    // doubly filled (mSetOccupancyZero), weighted by w_k, summed over the ranks
    {
        double left = c->n_el;
        std::vector<double> f0(nb);
        for (int n = 0; n < nb; ++n) {
            f0[n] = std::min(2.0, std::max(left, 0.0));
            left -= f0[n];
        }
        const int k0 = own_first();
        if (k0 < 0) QSB_CUDA_TRY(cudaMemsetAsync(c->rho_in, 0, N * sizeof(double), s));
        for (int k = 0; k < nk; ++k) {
            if (!c->kown[k]) continue;
            for (int n = 0; n < nb; ++n) wocc[n] = c->kw[k] * f0[n];
            QSB_TRY(density_complex(c, nb, X[k], wocc, c->rho_in, k != k0, s));
        }
        QSB_TRY(reduce_device(c, c->rho_in, N, s));
    }
    c->slots.clear();
    std::fill(c->B.begin(), c->B.end(), 0.0);
    std::fill(c->knfix.begin(), c->knfix.end(), 0);
    double e_prev = 0.0;
    *steps = 0;
    c->step_s.clear();
    c->step_res.clear();
    c->last_polish_first = -1;
    c->last_polish_steps = 0;
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    auto t_prev = std::chrono::steady_clock::now();
    for (int step = 0; step < max_steps; ++step) {
        QSB_TRY(potentials(c, s));
        std::fill(rq.begin(), rq.end(), 0.0);
        for (int k = 0; k < nk; ++k) {
            if (!c->kown[k]) continue;
            const double* g = &c->kvec[3 * (size_t)k];
            QSB_TRY(qsb_eigensolver_set_hamiltonian(c->es, c->ham, g[0], g[1], g[2]));
            QSB_TRY(qsb_lobpcg_z(c->es, c->dV, nb, lobpcg_iters, ev.data(), X[k], keep[k], &c->knfix[k], 0.0, step,
                                 stream));
            // FP64 Rayleigh quotients <x|Hx> / <x|x> of the complex bands (re and im
            // planes of a band are contiguous: one 2N-long dot per band)
            QSB_TRY(qsb_ham_apply(c->ham, QSB_F64, 1, nb, X[k], c->hxc, g[0], g[1], g[2], stream));
            band_dot_kernel<<<dim3(RBLOCKS / 4, nb), RB, 0, s>>>(2 * N, X[k], c->hxc, c->partial,
                                                                 c->partial + (size_t)nb * (RBLOCKS / 4));
            row_sum_kernel<<<2 * nb, 32, 0, s>>>(2 * nb, RBLOCKS / 4, c->partial, c->sums);
            QSB_CUDA_TRY(cudaGetLastError());
            QSB_CUDA_TRY(cudaMemcpyAsync(sums.data(), c->sums, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, s));
            QSB_CUDA_TRY(cudaStreamSynchronize(s));
            for (int n = 0; n < nb; ++n) {
                if (!(sums[nb + n] > 0.0) || !std::isfinite(sums[n]))
                    return fail(QSB_ERR_NUMERIC, "scf_run_kpoints: bad band norm");
                rq[(size_t)k * nb + n] = sums[n] / sums[nb + n];
            }
        }
        // every rank needs every level for the Fermi level: the levels of the
        // k-points a rank does not own are zero there, so a sum gathers them
        QSB_TRY(reduce_host(c, rq.data(), rq.size()));
        fermi_weighted(rq, wl, c->n_el, c->kbt, occ);
        const int k0 = own_first();
        if (k0 < 0) QSB_CUDA_TRY(cudaMemsetAsync(c->rho_out, 0, N * sizeof(double), s));
        for (int k = 0; k < nk; ++k) {
            if (!c->kown[k]) continue;
            for (int n = 0; n < nb; ++n) wocc[n] = c->kw[k] * occ[(size_t)k * nb + n];
            QSB_TRY(density_complex(c, nb, X[k], wocc, c->rho_out, k != k0, s));
        }
        QSB_TRY(reduce_device(c, c->rho_out, N, s));
        // energy of the output density, as the Gamma-point loop
        sub_kernel<<<pw_blocks(N), 256, 0, s>>>(N, c->veff, c->vloc, c->tmp);
        QSB_TRY(kspace(c, KOp::hartree, c->rho_out, c->vh, s));
        QSB_TRY(xc_eval(c, c->rho_out, c->exc, c->vxc, s));
        QSB_CUDA_TRY(cudaGetLastError());
        double d2[2], exc_int;
        {
            const double* a[2] = {c->tmp, c->vh};
            QSB_TRY(dots(c, 2, a, c->rho_out, d2, s));
            const double* e[1] = {c->exc};
            QSB_TRY(dots(c, 1, e, nullptr, &exc_int, s));
        }
        double eband = 0.0;
        for (size_t i = 0; i < rq.size(); ++i) eband += wl[i] * occ[i] * rq[i];
        const double etot = eband - d2[0] + 0.5 * d2[1] + exc_int;
        energies[step] = etot;
        *steps = step + 1;
        const auto t_now = std::chrono::steady_clock::now();
        c->step_s.push_back(std::chrono::duration<double>(t_now - t_prev).count());
        t_prev = t_now;
        {
            l1_diff_partial_kernel<<<RBLOCKS, RB, 0, s>>>(N, c->rho_out, c->rho_in, c->partial);
            row_sum_kernel<<<1, 32, 0, s>>>(1, RBLOCKS, c->partial, c->sums);
            double l1 = 0.0;
            QSB_CUDA_TRY(cudaMemcpyAsync(&l1, c->sums, sizeof(double), cudaMemcpyDeviceToHost, s));
            QSB_CUDA_TRY(cudaStreamSynchronize(s));
            c->step_res.push_back(l1 * c->dV / c->n_el);
        }
        bool done = step > 0 && std::fabs(etot - e_prev) / c->n_atoms < tol_per_atom;
        if (done && c->rho_tol > 0.0) done = c->step_res.back() < c->rho_tol;
        e_prev = etot;
        if (done) break;
        QSB_TRY(mix(c, s));
    }
    if (eigen_values) std::copy(rq.begin(), rq.end(), eigen_values);
    if (occupations) std::copy(occ.begin(), occ.end(), occupations);
    return QSB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ion-ion (Ewald) energy and forces, and LBFGS geometry relaxation.
// ---------------------------------------------------------------------------

extern "C" {

// Point charges in an orthorhombic cell with a neutralising background: the
// ion-ion term that goes with the G-space GTH local part (whose Coulomb tail is
// that of a point charge Z_ion).  Splitting alpha = 5 / min(L), real and
// reciprocal sums cut where erfc / the Gaussian fall below 1e-16.
qsb_status qsb_ewald(int n_atoms, const double* pos, const double* charge, const double* cell, double* energy,
                     double* forces) {
    if (n_atoms <= 0 || !pos || !charge || !cell || !energy) return fail(QSB_ERR_INVALID, "ewald: bad argument");
    const double L[3] = {cell[0], cell[1], cell[2]};
    if (!(L[0] > 0) || !(L[1] > 0) || !(L[2] > 0)) return fail(QSB_ERR_INVALID, "ewald: cell edges must be > 0");
    const double omega = L[0] * L[1] * L[2];
    const double alpha = 5.0 / std::min(L[0], std::min(L[1], L[2]));
    const double lt = std::sqrt(-std::log(1e-16));
    const double rc = lt / alpha, gc = 2.0 * alpha * lt;
    const double spi = std::sqrt(M_PI);
    double E = 0.0;
    std::vector<double> F(3 * (size_t)n_atoms, 0.0);
    int nimg[3];
    for (int d = 0; d < 3; ++d) nimg[d] = (int)std::ceil(rc / L[d]) + 1;
    for (int a = 0; a < n_atoms; ++a)
        for (int b = 0; b < n_atoms; ++b)
            for (int i = -nimg[0]; i <= nimg[0]; ++i)
                for (int j = -nimg[1]; j <= nimg[1]; ++j)
                    for (int k = -nimg[2]; k <= nimg[2]; ++k) {
                        if (a == b && i == 0 && j == 0 && k == 0) continue;
                        const double d[3] = {pos[3 * a] - pos[3 * b] + i * L[0], pos[3 * a + 1] - pos[3 * b + 1] + j * L[1],
                                             pos[3 * a + 2] - pos[3 * b + 2] + k * L[2]};
                        const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                        if (r > rc) continue;
                        const double zz = charge[a] * charge[b];
                        E += 0.5 * zz * std::erfc(alpha * r) / r;
                        const double g = zz * (std::erfc(alpha * r) / r + 2.0 * alpha / spi * std::exp(-alpha * alpha * r * r)) /
                                         (r * r);
                        for (int c = 0; c < 3; ++c) F[3 * a + c] += g * d[c];
                    }
    int m[3];
    for (int d = 0; d < 3; ++d) m[d] = (int)std::ceil(gc * L[d] / (2.0 * M_PI));
    for (int i = -m[0]; i <= m[0]; ++i)
        for (int j = -m[1]; j <= m[1]; ++j)
            for (int k = -m[2]; k <= m[2]; ++k) {
                if (i == 0 && j == 0 && k == 0) continue;
                const double G[3] = {2.0 * M_PI * i / L[0], 2.0 * M_PI * j / L[1], 2.0 * M_PI * k / L[2]};
                const double g2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
                if (g2 > gc * gc) continue;
                const double w = std::exp(-g2 / (4.0 * alpha * alpha)) / g2;
                double sr = 0.0, si = 0.0;
                for (int a = 0; a < n_atoms; ++a) {
                    const double ph = G[0] * pos[3 * a] + G[1] * pos[3 * a + 1] + G[2] * pos[3 * a + 2];
                    sr += charge[a] * std::cos(ph);
                    si += charge[a] * std::sin(ph);
                }
                E += 2.0 * M_PI / omega * w * (sr * sr + si * si);
                for (int a = 0; a < n_atoms; ++a) {
                    const double ph = G[0] * pos[3 * a] + G[1] * pos[3 * a + 1] + G[2] * pos[3 * a + 2];
                    // Im(conj(S) e^{i ph}) = sr sin(ph) - si cos(ph)
                    const double t = 4.0 * M_PI / omega * w * charge[a] * (sr * std::sin(ph) - si * std::cos(ph));
                    for (int c = 0; c < 3; ++c) F[3 * a + c] += t * G[c];
                }
            }
    double z2 = 0.0, zs = 0.0;
    for (int a = 0; a < n_atoms; ++a) {
        z2 += charge[a] * charge[a];
        zs += charge[a];
    }
    E += -alpha / spi * z2 - M_PI / (2.0 * omega * alpha * alpha) * zs * zs;
    *energy = E;
    if (forces)
        for (size_t q = 0; q < F.size(); ++q) forces[q] += F[q];
    return QSB_OK;
}

// LBFGS on the free energy E - kBT S + E_ewald with the forces local + nonlocal
// + Ewald (the relaxation the reference drives with damped dynamics,
// glips::Relaxation1Q..4Q::Evolve, source/Relaxation1.h:45-190): per iteration
// the projectors and the local part move to the new positions, the SCF runs
// warm from the previous states, the two-loop recursion (history `history`,
// initial scale s.y / y.y) proposes a step, capped at max_step bohr per atom
// (the reference's upper move limit); a step that raises the energy is halved
// (up to 5 times, rises under 10 scf_tol per atom count as noise) before
// the history is updated.  Fixed atoms (fixed[a] != 0)
// feel no force.  Stops at max |F| < fmax.
qsb_status qsb_relax_lbfgs(qsb_scf* c, int n_atoms, double* pos, const int* species, int n_species, const int* nl,
                           const double* r_l, const double* h_l, double rcut_factor, const double* zion,
                           const double* rloc, const double* c1, const double* c2, const int* fixed, double* X,
                           double* keep, int lobpcg_iters, int scf_max_steps, double scf_tol, int max_iter,
                           double fmax, double max_step, int history, double* energies, int* iters, double* forces,
                           void* stream) {
    if (!c || n_atoms <= 0 || !pos || !species || !X || !keep || max_iter <= 0 || !(fmax > 0) || !(max_step > 0) ||
        history < 1 || !energies || !iters || scf_max_steps <= 0)
        return fail(QSB_ERR_INVALID, "relax_lbfgs: bad argument");
    const int n3 = 3 * n_atoms;
    std::vector<double> q(n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
        if (species[a] < 0 || species[a] >= n_species) return fail(QSB_ERR_INVALID, "relax_lbfgs: bad species");
        q[a] = zion[species[a]];
    }
    const double cell[3] = {c->nx * c->dx, c->ny * c->dy, c->nz * c->dz};
    std::vector<double> e_scf(scf_max_steps), occ(c->nb), ev(c->nb);
    // free energy and gradient (g = -F) at x
    auto evaluate = [&](const double* x, double& E, std::vector<double>& g) -> qsb_status {
        QSB_TRY(qsb_ham_set_gth_projectors(c->ham, n_atoms, x, species, n_species, nl, r_l, h_l, rcut_factor));
        QSB_TRY(qsb_scf_set_gth_local(c, n_atoms, x, species, n_species, zion, rloc, c1, c2));
        int steps = 0;
        QSB_TRY(qsb_scf_run(c, X, keep, lobpcg_iters, scf_max_steps, scf_tol, e_scf.data(), &steps, ev.data(),
                            occ.data(), stream));
        if (steps < 1 || steps > scf_max_steps) return fail(QSB_ERR_STATE, "relax_lbfgs: the SCF ran no step");
        double ts = 0.0;
        for (int n = 0; n < c->nb; ++n) {
            const double f = std::min(std::max(occ[n] / 2.0, 1e-300), 1.0 - 1e-16);
            ts -= c->kbt * 2.0 * (f * std::log(f) + (1.0 - f) * std::log1p(-f));
        }
        std::vector<double> F(n3, 0.0);
        double ee = 0.0, enl = 0.0;
        QSB_TRY(qsb_ewald(n_atoms, x, q.data(), cell, &ee, F.data()));
        QSB_TRY(qsb_scf_local_forces(c, nullptr, F.data()));
        QSB_TRY(qsb_ham_nonlocal_energy_force(c->ham, QSB_F64, 0, c->nb, X, occ.data(), 0.0, 0.0, 0.0, &enl,
                                              F.data(), stream));
        E = e_scf[steps - 1] - ts + ee;
        g.assign(n3, 0.0);
        for (int a = 0; a < n_atoms; ++a)
            for (int k = 0; k < 3; ++k) g[3 * a + k] = (fixed && fixed[a]) ? 0.0 : -F[3 * a + k];
        return QSB_OK;
    };
    auto fmax_of = [&](const std::vector<double>& g) {
        double m = 0.0;
        for (int a = 0; a < n_atoms; ++a)
            m = std::max(m, std::sqrt(g[3 * a] * g[3 * a] + g[3 * a + 1] * g[3 * a + 1] + g[3 * a + 2] * g[3 * a + 2]));
        return m;
    };
    std::vector<double> x(pos, pos + n3), g, xn(n3), gn;
    std::vector<std::vector<double>> S, Y;
    double E = 0.0, En = 0.0;
    QSB_TRY(evaluate(x.data(), E, g));
    *iters = 0;
    energies[0] = E;
    for (int it = 1; it <= max_iter && fmax_of(g) >= fmax; ++it) {
        // two-loop recursion: d = -H g
        std::vector<double> d(g);
        const int m = (int)S.size();
        std::vector<double> al(m), rho(m);
        for (int i = m - 1; i >= 0; --i) {
            double sy = 0.0, sd = 0.0;
            for (int k = 0; k < n3; ++k) {
                sy += S[i][k] * Y[i][k];
                sd += S[i][k] * d[k];
            }
            rho[i] = 1.0 / sy;
            al[i] = rho[i] * sd;
            for (int k = 0; k < n3; ++k) d[k] -= al[i] * Y[i][k];
        }
        double h0 = 1.0;   // bohr^2 / Ha without history
        if (m > 0) {
            double sy = 0.0, yy = 0.0;
            for (int k = 0; k < n3; ++k) {
                sy += S[m - 1][k] * Y[m - 1][k];
                yy += Y[m - 1][k] * Y[m - 1][k];
            }
            h0 = sy / yy;
        }
        for (int k = 0; k < n3; ++k) d[k] *= h0;
        for (int i = 0; i < m; ++i) {
            double yd = 0.0;
            for (int k = 0; k < n3; ++k) yd += Y[i][k] * d[k];
            const double b = rho[i] * yd;
            for (int k = 0; k < n3; ++k) d[k] += S[i][k] * (al[i] - b);
        }
        for (int k = 0; k < n3; ++k) d[k] = -d[k];
        // cap the displacement per atom
        double dm = 0.0;
        for (int a = 0; a < n_atoms; ++a)
            dm = std::max(dm, std::sqrt(d[3 * a] * d[3 * a] + d[3 * a + 1] * d[3 * a + 1] + d[3 * a + 2] * d[3 * a + 2]));
        const double sc = dm > max_step ? max_step / dm : 1.0;
        double step = sc;
        bool ok = false;
        // energies carry the SCF stop's error (|dE| < scf_tol per atom per
        // step, a few steps' worth from the fixed point): rises below that are noise
        const double slack = 10.0 * scf_tol * n_atoms;
        for (int tries = 0; tries < 6; ++tries) {
            for (int k = 0; k < n3; ++k) xn[k] = x[k] + step * d[k];
            QSB_TRY(evaluate(xn.data(), En, gn));
            if (En <= E + slack || tries == 5) {
                ok = true;
                break;
            }
            step *= 0.5;
        }
        if (!ok) break;
        std::vector<double> s(n3), y(n3);
        double sy = 0.0;
        for (int k = 0; k < n3; ++k) {
            s[k] = xn[k] - x[k];
            y[k] = gn[k] - g[k];
            sy += s[k] * y[k];
        }
        if (sy > 1e-12) {
            S.push_back(s);
            Y.push_back(y);
            if ((int)S.size() > history) {
                S.erase(S.begin());
                Y.erase(Y.begin());
            }
        }
        x = xn;
        g = gn;
        E = En;
        energies[it] = E;
        *iters = it;
    }
    std::copy(x.begin(), x.end(), pos);
    if (forces)
        for (int k = 0; k < n3; ++k) forces[k] = -g[k];
    return QSB_OK;
}

}  // extern "C"
