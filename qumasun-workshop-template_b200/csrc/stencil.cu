// FD8 Laplacian (+ k-point first-derivative term, + local potential) stencil
// kernels for sm_100a.
//
// One CTA owns a TX x TY tile of the xy plane for one band and marches along
// z.  Each thread keeps the 9-deep z column of its grid rows in registers
// (z-4 .. z+4), so every psi value is loaded from HBM once for the z
// derivative; the current plane (with a 4-wide x/y halo) is staged in a
// double-buffered shared-memory tile for the x and y derivatives.  Periodic
// boundaries are handled by wrapped indexing on the halo loads, which replaces
// the reference's explicit (N+8)^3 halo copy (source/GridDifference8th.h:19-78,
// :152-169): the reference reads and writes every band twice to build that copy.
//
// Arithmetic follows Laplacian8th_halo_f (source/GridDifference8th.h:82-148)
// and LaplacianKpoint8th_halo_f (source/GridDifferenceKpoint8th.h:17-120):
//   d = c0 p; d += x terms (offsets 4,3,2,1); d += y terms; d += z terms.
#include "qsb_internal.h"
#include <cmath>

namespace qsb {

FD8Coef make_fd8_coef(double coef, double dx, double dy, double dz, double gx, double gy, double gz) {
    FD8Coef c{};
    // source/GridDifferenceKpoint8th.h:26-40 (reduces to GridDifference8th.h:89-101 at g = 0)
    c.c0 = -14350.0 / 5040.0 * coef * (1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)) -
           coef * (gx * gx + gy * gy + gz * gz);
    const double w2[4] = {8064.0, -1008.0, 128.0, -9.0};
    for (int m = 0; m < 4; ++m) {
        c.cx[m] = w2[m] * coef / (5040.0 * dx * dx);
        c.cy[m] = w2[m] * coef / (5040.0 * dy * dy);
        c.cz[m] = w2[m] * coef / (5040.0 * dz * dz);
    }
    // first derivative, sign +1 (GridDifferenceKpoint8th.h:45-57); the imaginary
    // pass of the reference uses sign -1, i.e. exactly the negation.
    const double w1[4] = {672.0, -168.0, 32.0, -3.0};
    const double coef2 = coef * 2.0;
    constexpr double th = 1.0e-8;  // GridDifferenceKpoint8th.h:330 dispatch threshold
    const bool kx = std::fabs(gx) >= th, ky = std::fabs(gy) >= th, kz = std::fabs(gz) >= th;
    for (int m = 0; m < 4; ++m) {
        c.ax[m] = kx ? w1[m] * coef2 * gx / (840.0 * dx) : 0.0;
        c.ay[m] = ky ? w1[m] * coef2 * gy / (840.0 * dy) : 0.0;
        c.az[m] = kz ? w1[m] * coef2 * gz / (840.0 * dz) : 0.0;
    }
    c.has_grad = kx || ky || kz;
    return c;
}

namespace {

constexpr int TX = 32;        // tile width (one warp)
constexpr int BY = 8;         // thread rows per CTA
constexpr int RY = 2;         // grid rows per thread
constexpr int TY = BY * RY;   // tile height
constexpr int HW = 4;         // halo width of the 8th-order stencil

template <typename T>
struct KC {
    T c0;
    T cx[4], cy[4], cz[4];
    T ax[4], ay[4], az[4];
};

template <typename T>
KC<T> to_kc(const FD8Coef& c) {
    KC<T> k;
    k.c0 = (T)c.c0;
    for (int m = 0; m < 4; ++m) {
        k.cx[m] = (T)c.cx[m]; k.cy[m] = (T)c.cy[m]; k.cz[m] = (T)c.cz[m];
        k.ax[m] = (T)c.ax[m]; k.ay[m] = (T)c.ay[m]; k.az[m] = (T)c.az[m];
    }
    return k;
}

__device__ __forceinline__ int wrapi(int v, int n) {
    int m = v % n;
    return m < 0 ? m + n : m;
}

// MODE 0: out += coef*L(psi).  MODE 1: out = V psi + coef*L(psi) [+ NL].
template <typename T, bool CPLX, int MODE, bool GRAD, bool NL>
__global__ void __launch_bounds__(TX * BY, 2)
fd8_kernel(const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ V,
           int nx, int ny, int nz, int zchunk, KC<T> k, NLView nl) {
    constexpr int NC = CPLX ? 2 : 1;
    __shared__ T sm[2][NC][TY + 2 * HW][TX + 2 * HW];

    const int ntx = (nx + TX - 1) / TX;
    const int x0 = (blockIdx.x % ntx) * TX;
    const int y0 = (blockIdx.x / ntx) * TY;
    const int wx = min(TX, nx - x0);
    const int wy = min(TY, ny - y0);
    const int z0 = blockIdx.y * zchunk;
    const int z1 = min(nz, z0 + zchunk);
    const int band = blockIdx.z;
    const size_t nxy = (size_t)nx * ny;
    const size_t N = nxy * nz;

    const T* src[NC];
    T* dst[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const size_t plane = CPLX ? (size_t)(2 * band + c) : (size_t)band;
        src[c] = in + plane * N;
        dst[c] = out + plane * N;
    }

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx;
    const bool xin = tx < wx;

    bool rvalid[RY];
    int yrow[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        yrow[r] = y0 + ty + BY * r;
        rvalid[r] = xin && (ty + BY * r < wy);
    }

    // register queue: q[c][r][j] = psi(x, y_r, z - 4 + j)
    T q[NC][RY][9];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            q[c][r][0] = T(0);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int zz = wrapi(z0 - HW + j, nz);
                q[c][r][j + 1] = rvalid[r] ? __ldg(src[c] + x + (size_t)nx * yrow[r] + nxy * zz) : T(0);
            }
        }

    // halo roles
    const int hx_left = (tx < HW);
    const int hx_right = (tx >= HW && tx < 2 * HW);
    const int xl = wrapi(x0 - HW + tx, nx);             // for left-halo threads
    const int xr = wrapi(x0 + wx + (tx - HW), nx);      // for right-halo threads
    const int ytop = wrapi(y0 - HW + ty, ny);           // ty < 4
    const int ybot = wrapi(y0 + wy + (ty - HW), ny);    // 4 <= ty < 8

    for (int z = z0; z < z1; ++z) {
        const int buf = (z - z0) & 1;
        const int zn = wrapi(z + HW, nz);
        const size_t zoff = nxy * (size_t)z;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int r = 0; r < RY; ++r) {
#pragma unroll
                for (int j = 0; j < 8; ++j) q[c][r][j] = q[c][r][j + 1];
                q[c][r][8] = rvalid[r] ? __ldg(src[c] + x + (size_t)nx * yrow[r] + nxy * zn) : T(0);
                sm[buf][c][ty + BY * r + HW][tx + HW] = q[c][r][4];
            }
        // x halos of this plane
        if (hx_left || hx_right) {
            const int xs = hx_left ? xl : xr;
            const int col = hx_left ? tx : (wx + HW + (tx - HW));
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                if (ty + BY * r < wy) {
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        sm[buf][c][ty + BY * r + HW][col] = __ldg(src[c] + xs + (size_t)nx * yrow[r] + zoff);
                }
            }
        }
        // y halos of this plane
        if (xin) {
            if (ty < HW) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    sm[buf][c][ty][tx + HW] = __ldg(src[c] + x + (size_t)nx * ytop + zoff);
            } else if (ty < 2 * HW) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    sm[buf][c][wy + HW + (ty - HW)][tx + HW] = __ldg(src[c] + x + (size_t)nx * ybot + zoff);
            }
        }
        __syncthreads();

#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!rvalid[r]) continue;
            const int sy = ty + BY * r + HW;
            const int sx = tx + HW;
            T lap[NC], grd[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const T(*s)[TX + 2 * HW] = sm[buf][c];
                const T* qq = q[c][r];
                T d = k.c0 * qq[4];
                d += k.cx[3] * (s[sy][sx + 4] + s[sy][sx - 4]) + k.cx[2] * (s[sy][sx + 3] + s[sy][sx - 3]) +
                     k.cx[1] * (s[sy][sx + 2] + s[sy][sx - 2]) + k.cx[0] * (s[sy][sx + 1] + s[sy][sx - 1]);
                d += k.cy[3] * (s[sy + 4][sx] + s[sy - 4][sx]) + k.cy[2] * (s[sy + 3][sx] + s[sy - 3][sx]) +
                     k.cy[1] * (s[sy + 2][sx] + s[sy - 2][sx]) + k.cy[0] * (s[sy + 1][sx] + s[sy - 1][sx]);
                d += k.cz[3] * (qq[8] + qq[0]) + k.cz[2] * (qq[7] + qq[1]) + k.cz[1] * (qq[6] + qq[2]) +
                     k.cz[0] * (qq[5] + qq[3]);
                lap[c] = d;
                if (GRAD) {
                    T g = k.ax[3] * (s[sy][sx + 4] - s[sy][sx - 4]) + k.ax[2] * (s[sy][sx + 3] - s[sy][sx - 3]) +
                          k.ax[1] * (s[sy][sx + 2] - s[sy][sx - 2]) + k.ax[0] * (s[sy][sx + 1] - s[sy][sx - 1]);
                    g += k.ay[3] * (s[sy + 4][sx] - s[sy - 4][sx]) + k.ay[2] * (s[sy + 3][sx] - s[sy - 3][sx]) +
                         k.ay[1] * (s[sy + 2][sx] - s[sy - 2][sx]) + k.ay[0] * (s[sy + 1][sx] - s[sy - 1][sx]);
                    g += k.az[3] * (qq[8] - qq[0]) + k.az[2] * (qq[7] - qq[1]) + k.az[1] * (qq[6] - qq[2]) +
                         k.az[0] * (qq[5] - qq[3]);
                    grd[c] = g;
                } else {
                    grd[c] = T(0);
                }
            }
            T res[NC];
            if (CPLX) {
                // out.re: Lap(re) - D(im);  out.im: Lap(im) + D(re)
                res[0] = GRAD ? lap[0] - grd[NC - 1] : lap[0];
                res[NC - 1] = GRAD ? lap[NC - 1] + grd[0] : lap[NC - 1];
            } else {
                res[0] = lap[0];
            }
            const size_t gidx = (size_t)x + (size_t)nx * yrow[r] + zoff;
            if (MODE == 0) {
#pragma unroll
                for (int c = 0; c < NC; ++c) dst[c][gidx] += res[c];
            } else {
                const T v = __ldg(V + gidx);
                T nlv[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) nlv[c] = T(0);
                if (NL) {
                    const int e0 = __ldg(nl.grid_ptr + gidx), e1 = __ldg(nl.grid_ptr + gidx + 1);
                    {
                        const T* beta = (const T*)nl.ent_beta;
                        for (int e = e0; e < e1; ++e) {
                            const int a = __ldg(nl.ent_atom + e);
                            const double* cf = nl.coef + (size_t)a * nl.wmax * nl.ncol;
                            double tr = 0.0, ti = 0.0;
                            for (int w = 0; w < nl.wmax; ++w) {
                                const double b = (double)__ldg(beta + (size_t)e * nl.wmax + w);
                                if (CPLX) {
                                    tr += b * __ldg(cf + (size_t)w * nl.ncol + 2 * band);
                                    ti += b * __ldg(cf + (size_t)w * nl.ncol + 2 * band + 1);
                                } else {
                                    tr += b * __ldg(cf + (size_t)w * nl.ncol + band);
                                }
                            }
                            if (CPLX) {
                                const int* xyz = nl.ent_xyz + 3 * (size_t)e;
                                const double kxx = nl.gx_dx * (double)__ldg(xyz + 0);
                                const double kyy = nl.gy_dy * (double)__ldg(xyz + 1);
                                const double kzz = nl.gz_dz * (double)__ldg(xyz + 2);
                                double sn, cs;
                                sincos(kxx + kyy + kzz, &sn, &cs);
                                // multiply by exp(-i k.r): (cs*tr + sn*ti, cs*ti - sn*tr)
                                nlv[0] += (T)(cs * tr + sn * ti);
                                nlv[NC - 1] += (T)(cs * ti - sn * tr);
                            } else {
                                nlv[0] += (T)tr;
                            }
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < NC; ++c) dst[c][gidx] = v * q[c][r][4] + nlv[c] + res[c];
            }
        }
    }
}

template <typename T, bool CPLX, int MODE, bool NL>
void launch_t(const StencilLaunch& L, const FD8Coef& c, const NLView& nv, cudaStream_t s) {
    const int ntx = (L.nx + TX - 1) / TX, nty = (L.ny + TY - 1) / TY;
    const int tiles = ntx * nty;
    // Enough CTAs to fill 148 SMs x 2 resident CTAs several times over;
    // split z only when tiles x bands is small.
    int zsplit = 1;
    const long long ctas = (long long)tiles * L.nb;
    while (ctas * zsplit < 148LL * 2 * 4 && L.nz / (zsplit * 2) >= 8) zsplit *= 2;
    const int zchunk = (L.nz + zsplit - 1) / zsplit;
    const int nzc = (L.nz + zchunk - 1) / zchunk;
    dim3 grid(tiles, nzc, L.nb), block(TX, BY);
    const KC<T> k = to_kc<T>(c);
    if (c.has_grad && CPLX)
        fd8_kernel<T, CPLX, MODE, CPLX, NL><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx, L.ny,
                                                                  L.nz, zchunk, k, nv);
    else
        fd8_kernel<T, CPLX, MODE, false, NL><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx, L.ny,
                                                                   L.nz, zchunk, k, nv);
}

template <typename T>
qsb_status launch_dtype(const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    NLView nv{};
    const bool nl = (L.nl != nullptr);
    if (nl) nv = *L.nl;
    if (L.mode == 0) {
        if (L.is_complex) launch_t<T, true, 0, false>(L, c, nv, s);
        else launch_t<T, false, 0, false>(L, c, nv, s);
    } else {
        if (L.is_complex) {
            if (nl) launch_t<T, true, 1, true>(L, c, nv, s);
            else launch_t<T, true, 1, false>(L, c, nv, s);
        } else {
            if (nl) launch_t<T, false, 1, true>(L, c, nv, s);
            else launch_t<T, false, 1, false>(L, c, nv, s);
        }
    }
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

}  // namespace

qsb_status launch_stencil(qsb_dtype dt, const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    if (L.nb > 65535) return fail(QSB_ERR_INVALID, "stencil: nb > 65535");
    if (dt == QSB_F64) return launch_dtype<double>(L, c, s);
    return launch_dtype<float>(L, c, s);
}

}  // namespace qsb
