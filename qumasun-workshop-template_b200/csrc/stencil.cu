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
constexpr int BY = 8;         // warps per CTA, stacked in y
constexpr int NT = TX * BY;   // threads per CTA
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

// One CTA: a TX x TY tile (TY = BY*RY) of one band (both SoA planes for
// complex), marching z over [z0, z1).  Thread (tx, ty) owns the RY
// consecutive grid rows y0 + ty*RY + i at x0 + tx and keeps their z columns
// (z-4 .. z+4) in registers; the current plane plus its 4-wide x/y halo sits in
// a double-buffered shared tile.  Every global load is issued ahead of use:
// centre values 4 planes ahead (the z queue), halo values 2 planes ahead (a
// register shift of two planes), so a single __syncthreads per plane is the
// only wait.  The y derivative of the RY rows is read as one column of RY+8
// shared values (instead of 8 per point).
//
// MODE 0: out += L(psi)      (Laplacian8th / LaplacianKpoint8th "+=")
// MODE 1: out = V psi + L(psi)   (the local part of mHamiltonianMatrix_ddm)
template <typename T, bool CPLX, int MODE, bool GRAD, int RY>
__global__ void __launch_bounds__(NT, 2)
fd8_kernel(const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ V,
           int nx, int ny, int nz, int zchunk, KC<T> k) {
    constexpr int NC = CPLX ? 2 : 1;
    constexpr int TY = BY * RY;
    constexpr int SW = TX + 2 * HW;
    constexpr int SH = TY + 2 * HW;
    __shared__ T sm[2][NC][SH][SW];

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
    const int t = ty * TX + tx;
    const int x = x0 + tx;
    const bool xin = tx < wx;
    bool rv[RY];
#pragma unroll
    for (int i = 0; i < RY; ++i) rv[i] = xin && (ty * RY + i < wy);
    const size_t rowoff = (size_t)x + (size_t)nx * (y0 + ty * RY);   // grid offset of row 0 of this thread

    // x-halo role: 8*TY positions (left/right, TY rows, 4 columns)
    bool xh_ok = false;
    size_t xh_g = 0;
    int xh_s = 0;
    if (t < 8 * TY) {
        const int side = t / (4 * TY), rem = t % (4 * TY), hrow = rem / 4, hk = rem % 4;
        xh_ok = hrow < wy;
        const int gxx = side == 0 ? wrapi(x0 - HW + hk, nx) : wrapi(x0 + wx + hk, nx);
        xh_g = (size_t)gxx + (size_t)nx * (y0 + min(hrow, wy - 1));
        xh_s = (HW + hrow) * SW + (side == 0 ? hk : wx + HW + hk);
    }
    // y-halo role: 8*TX positions (top/bottom, 4 rows, TX columns)
    bool yh_ok = false;
    size_t yh_g = 0;
    int yh_s = 0;
    if (t < 8 * TX) {
        const int side = t / (4 * TX), rem = t % (4 * TX), hr = rem / TX, hc = rem % TX;
        yh_ok = hc < wx;
        const int gyy = side == 0 ? wrapi(y0 - HW + hr, ny) : wrapi(y0 + wy + hr, ny);
        yh_g = (size_t)(x0 + min(hc, wx - 1)) + (size_t)nx * gyy;
        yh_s = (side == 0 ? hr : wy + HW + hr) * SW + HW + hc;
    }

    // prefetched halos of planes z (index 0) and z+1 (index 1)
    T hx[2][NC], hy[2][NC];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const size_t zo = nxy * (size_t)wrapi(z0 + d, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            hx[d][c] = xh_ok ? __ldg(src[c] + xh_g + zo) : T(0);
            hy[d][c] = yh_ok ? __ldg(src[c] + yh_g + zo) : T(0);
        }
    }
    // z queues: q[c][i][j] = psi(x, y_i, z - 4 + j)
    T q[NC][RY][9];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int i = 0; i < RY; ++i) {
            q[c][i][0] = T(0);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const size_t zo = nxy * (size_t)wrapi(z0 - HW + j, nz);
                q[c][i][j + 1] = rv[i] ? __ldg(src[c] + rowoff + (size_t)nx * i + zo) : T(0);
            }
        }

    for (int z = z0; z < z1; ++z) {
        const int buf = (z - z0) & 1;
        T* sb = &sm[buf][0][0][0];
        // halos of plane z into shared memory, then prefetch plane z+2
        const size_t zo2 = nxy * (size_t)wrapi(z + 2, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (xh_ok) sb[c * SH * SW + xh_s] = hx[0][c];
            if (yh_ok) sb[c * SH * SW + yh_s] = hy[0][c];
            hx[0][c] = hx[1][c];
            hy[0][c] = hy[1][c];
            hx[1][c] = xh_ok ? __ldg(src[c] + xh_g + zo2) : T(0);
            hy[1][c] = yh_ok ? __ldg(src[c] + yh_g + zo2) : T(0);
        }
        // advance the z queues (load plane z+4) and write the centre of plane z
        const size_t zo4 = nxy * (size_t)wrapi(z + HW, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int i = 0; i < RY; ++i) {
#pragma unroll
                for (int j = 0; j < 8; ++j) q[c][i][j] = q[c][i][j + 1];
                q[c][i][8] = rv[i] ? __ldg(src[c] + rowoff + (size_t)nx * i + zo4) : T(0);
                // only in-tile threads write centres: for a partial tile the cells of
                // out-of-tile threads alias the right / bottom halo
                if (rv[i]) sm[buf][c][ty * RY + i + HW][tx + HW] = q[c][i][4];
            }
        __syncthreads();

        T res[NC][RY];
        T grd[NC][RY];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const T(*s)[SW] = sm[buf][c];
            T col[RY + 8];
#pragma unroll
            for (int j = 0; j < RY + 8; ++j) col[j] = s[ty * RY + j][tx + HW];
#pragma unroll
            for (int i = 0; i < RY; ++i) {
                const int sy = ty * RY + i + HW, sx = tx + HW;
                const T* qq = q[c][i];
                const T xm4 = s[sy][sx - 4], xm3 = s[sy][sx - 3], xm2 = s[sy][sx - 2], xm1 = s[sy][sx - 1];
                const T xp1 = s[sy][sx + 1], xp2 = s[sy][sx + 2], xp3 = s[sy][sx + 3], xp4 = s[sy][sx + 4];
                T d = k.c0 * qq[4];
                d += k.cx[3] * (xp4 + xm4) + k.cx[2] * (xp3 + xm3) + k.cx[1] * (xp2 + xm2) + k.cx[0] * (xp1 + xm1);
                d += k.cy[3] * (col[i + 8] + col[i]) + k.cy[2] * (col[i + 7] + col[i + 1]) +
                     k.cy[1] * (col[i + 6] + col[i + 2]) + k.cy[0] * (col[i + 5] + col[i + 3]);
                d += k.cz[3] * (qq[8] + qq[0]) + k.cz[2] * (qq[7] + qq[1]) + k.cz[1] * (qq[6] + qq[2]) +
                     k.cz[0] * (qq[5] + qq[3]);
                res[c][i] = d;
                if (GRAD) {
                    T g = k.ax[3] * (xp4 - xm4) + k.ax[2] * (xp3 - xm3) + k.ax[1] * (xp2 - xm2) + k.ax[0] * (xp1 - xm1);
                    g += k.ay[3] * (col[i + 8] - col[i]) + k.ay[2] * (col[i + 7] - col[i + 1]) +
                         k.ay[1] * (col[i + 6] - col[i + 2]) + k.ay[0] * (col[i + 5] - col[i + 3]);
                    g += k.az[3] * (qq[8] - qq[0]) + k.az[2] * (qq[7] - qq[1]) + k.az[1] * (qq[6] - qq[2]) +
                         k.az[0] * (qq[5] - qq[3]);
                    grd[c][i] = g;
                }
            }
        }
        const size_t zo = nxy * (size_t)z;
#pragma unroll
        for (int i = 0; i < RY; ++i) {
            if (!rv[i]) continue;
            const size_t gidx = rowoff + (size_t)nx * i + zo;
            T r0 = res[0][i], r1 = res[NC - 1][i];
            if (CPLX && GRAD) {
                // out.re: Lap(re) - D(im);  out.im: Lap(im) + D(re)
                r0 = res[0][i] - grd[NC - 1][i];
                r1 = res[NC - 1][i] + grd[0][i];
            }
            if (MODE == 0) {
                dst[0][gidx] += r0;
                if (CPLX) dst[NC - 1][gidx] += r1;
            } else {
                const T v = __ldg(V + gidx);
                dst[0][gidx] = v * q[0][i][4] + r0;
                if (CPLX) dst[NC - 1][gidx] = v * q[NC - 1][i][4] + r1;
            }
        }
    }
}

template <typename T, bool CPLX, int MODE>
void launch_t(const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    constexpr int RY = CPLX ? 2 : 4;
    constexpr int TY = BY * RY;
    const int ntx = (L.nx + TX - 1) / TX, nty = (L.ny + TY - 1) / TY;
    const int tiles = ntx * nty;
    // enough CTAs for 148 SMs x 2 resident CTAs x 3 waves; split z only when
    // tiles x bands is small, keeping chunks of >= 16 planes
    int zsplit = 1;
    const long long ctas = (long long)tiles * L.nb;
    while (ctas * zsplit < 148LL * 2 * 3 && L.nz / (zsplit * 2) >= 16) zsplit *= 2;
    const int zchunk = (L.nz + zsplit - 1) / zsplit;
    const int nzc = (L.nz + zchunk - 1) / zchunk;
    dim3 grid(tiles, nzc, L.nb), block(TX, BY);
    const KC<T> k = to_kc<T>(c);
    if (CPLX && c.has_grad)
        fd8_kernel<T, CPLX, MODE, CPLX, RY><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx,
                                                                   L.ny, L.nz, zchunk, k);
    else
        fd8_kernel<T, CPLX, MODE, false, RY><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx,
                                                                    L.ny, L.nz, zchunk, k);
}

template <typename T>
qsb_status launch_dtype(const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    if (L.mode == 0) {
        if (L.is_complex) launch_t<T, true, 0>(L, c, s);
        else launch_t<T, false, 0>(L, c, s);
    } else {
        if (L.is_complex) launch_t<T, true, 1>(L, c, s);
        else launch_t<T, false, 1>(L, c, s);
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
