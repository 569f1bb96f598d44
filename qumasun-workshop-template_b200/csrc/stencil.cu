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
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cuda.h>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

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
//
// The work of one CTA (tile x0, y0 of band `band`, planes [z0, z1)) is the
// device function fd8_tile, shared by fd8_kernel (one item per CTA) and
// fd8_batch_kernel (a persistent CTA walking a list of items of many systems).
template <typename T, bool CPLX, int MODE, bool GRAD, int RY>
__device__ __forceinline__ void fd8_tile(const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ V,
                                         int nx, int ny, int nz, int x0, int y0, int z0, int z1, int band,
                                         const KC<T>& k, T* smraw) {
    constexpr int NC = CPLX ? 2 : 1;
    constexpr int TY = BY * RY;
    constexpr int SW = TX + 2 * HW;
    constexpr int SH = TY + 2 * HW;
    T(*sm)[NC][SH][SW] = reinterpret_cast<T(*)[NC][SH][SW]>(smraw);
    const int wx = min(TX, nx - x0);
    const int wy = min(TY, ny - y0);
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

    // Register rotation without moves: the z loop is unrolled by 9, so at phase
    // p (z = zb + p) plane z-4+k lives in queue slot (p+k) % 9 and the halo of
    // plane z+d in halo slot (p+d) % 3, all compile-time indices.  A load issued
    // at phase p is first read 4 (centre) or 2 (halo) planes later.
    T hx[3][NC], hy[3][NC];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const size_t zo = nxy * (size_t)wrapi(z0 + d, nz);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            hx[d][c] = xh_ok ? __ldg(src[c] + xh_g + zo) : T(0);
            hy[d][c] = yh_ok ? __ldg(src[c] + yh_g + zo) : T(0);
        }
    }
    // epilogue operand prefetched 2 planes ahead like the halos: V (MODE 1) or
    // the accumulated output (MODE 0), 3-slot rotation
    constexpr int NE = MODE == 0 ? NC : 1;
    T ep[3][NE][RY];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const size_t zo = nxy * (size_t)wrapi(z0 + d, nz);
#pragma unroll
        for (int i = 0; i < RY; ++i) {
            if (MODE == 0) {
#pragma unroll
                for (int c = 0; c < NE; ++c) ep[d][c][i] = rv[i] ? dst[c][rowoff + (size_t)nx * i + zo] : T(0);
            } else {
                ep[d][0][i] = rv[i] ? __ldg(V + rowoff + (size_t)nx * i + zo) : T(0);
            }
        }
    }
    T q[NC][RY][9];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int i = 0; i < RY; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const size_t zo = nxy * (size_t)wrapi(z0 - HW + j, nz);
                q[c][i][j] = rv[i] ? __ldg(src[c] + rowoff + (size_t)nx * i + zo) : T(0);
            }

    for (int zb = z0; zb < z1; zb += 9) {
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            const int z = zb + p;
            if (z < z1) {
                const int buf = (z - z0) & 1;
                T* sb = &sm[buf][0][0][0];
                const size_t zo2 = nxy * (size_t)wrapi(z + 2, nz);
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (xh_ok) sb[c * SH * SW + xh_s] = hx[p % 3][c];
                    if (yh_ok) sb[c * SH * SW + yh_s] = hy[p % 3][c];
                    hx[(p + 2) % 3][c] = xh_ok ? __ldg(src[c] + xh_g + zo2) : T(0);
                    hy[(p + 2) % 3][c] = yh_ok ? __ldg(src[c] + yh_g + zo2) : T(0);
                }
#pragma unroll
                for (int i = 0; i < RY; ++i) {
                    // z + 2 < z1 keeps MODE 0's read of out ahead of this CTA's own writes
                    const bool ok = rv[i] && (MODE == 1 || z + 2 < z1);
                    const size_t o2 = rowoff + (size_t)nx * i + zo2;
                    if (MODE == 0) {
#pragma unroll
                        for (int c = 0; c < NE; ++c) ep[(p + 2) % 3][c][i] = ok ? dst[c][o2] : T(0);
                    } else {
                        ep[(p + 2) % 3][0][i] = ok ? __ldg(V + o2) : T(0);
                    }
                }
                const size_t zo4 = nxy * (size_t)wrapi(z + HW, nz);
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i) {
                        q[c][i][(p + 8) % 9] = rv[i] ? __ldg(src[c] + rowoff + (size_t)nx * i + zo4) : T(0);
                        // only in-tile threads write centres: for a partial tile the cells of
                        // out-of-tile threads alias the right / bottom halo
                        if (rv[i]) sm[buf][c][ty * RY + i + HW][tx + HW] = q[c][i][(p + 4) % 9];
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
#define QZ(k) q[c][i][(p + (k)) % 9]
                        const T xm4 = s[sy][sx - 4], xm3 = s[sy][sx - 3], xm2 = s[sy][sx - 2], xm1 = s[sy][sx - 1];
                        const T xp1 = s[sy][sx + 1], xp2 = s[sy][sx + 2], xp3 = s[sy][sx + 3], xp4 = s[sy][sx + 4];
                        T d = k.c0 * QZ(4);
                        d += k.cx[3] * (xp4 + xm4) + k.cx[2] * (xp3 + xm3) + k.cx[1] * (xp2 + xm2) +
                             k.cx[0] * (xp1 + xm1);
                        d += k.cy[3] * (col[i + 8] + col[i]) + k.cy[2] * (col[i + 7] + col[i + 1]) +
                             k.cy[1] * (col[i + 6] + col[i + 2]) + k.cy[0] * (col[i + 5] + col[i + 3]);
                        d += k.cz[3] * (QZ(8) + QZ(0)) + k.cz[2] * (QZ(7) + QZ(1)) + k.cz[1] * (QZ(6) + QZ(2)) +
                             k.cz[0] * (QZ(5) + QZ(3));
                        if constexpr (sizeof(T) == 4) d = fmaf(k.c0lo, QZ(4), d);
                        res[c][i] = d;
                        if (GRAD) {
                            T g = k.ax[3] * (xp4 - xm4) + k.ax[2] * (xp3 - xm3) + k.ax[1] * (xp2 - xm2) +
                                  k.ax[0] * (xp1 - xm1);
                            g += k.ay[3] * (col[i + 8] - col[i]) + k.ay[2] * (col[i + 7] - col[i + 1]) +
                                 k.ay[1] * (col[i + 6] - col[i + 2]) + k.ay[0] * (col[i + 5] - col[i + 3]);
                            g += k.az[3] * (QZ(8) - QZ(0)) + k.az[2] * (QZ(7) - QZ(1)) + k.az[1] * (QZ(6) - QZ(2)) +
                                 k.az[0] * (QZ(5) - QZ(3));
                            grd[c][i] = g;
                        }
#undef QZ
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
                        dst[0][gidx] = ep[p % 3][0][i] + r0;
                        if (CPLX) dst[NC - 1][gidx] = ep[p % 3][NE - 1][i] + r1;
                    } else {
                        const T v = ep[p % 3][0][i];
                        dst[0][gidx] = v * q[0][i][(p + 4) % 9] + r0;
                        if (CPLX) dst[NC - 1][gidx] = v * q[NC - 1][i][(p + 4) % 9] + r1;
                    }
                }
            }
        }
    }
}

template <typename T, bool CPLX, int MODE, bool GRAD, int RY>
// three CTAs per SM for real FP32 bands (the mixed solver's operator): 0.533
// against 0.551 ms at 96^3 x 128 bands with two (same box, same output bits)
__global__ void __launch_bounds__(NT, (CPLX && sizeof(T) == 8) ? 1 : ((!CPLX && sizeof(T) == 4) ? 3 : 2))
fd8_kernel(const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ V,
           int nx, int ny, int nz, int zchunk, KC<T> k) {
    constexpr int NC = CPLX ? 2 : 1;
    constexpr int TY = BY * RY;
    __shared__ T sm[2 * NC * (TY + 2 * HW) * (TX + 2 * HW)];
    const int ntx = (nx + TX - 1) / TX;
    const int z0 = blockIdx.y * zchunk;
    fd8_tile<T, CPLX, MODE, GRAD, RY>(in, out, V, nx, ny, nz, (blockIdx.x % ntx) * TX, (blockIdx.x / ntx) * TY, z0,
                                      min(nz, z0 + zchunk), blockIdx.z, k, sm);
}

// Batched form (qsb_ham_apply_batch): real bands, MODE 1 (out = V psi + L psi),
// a persistent grid walking (system, tile, z chunk, band) items of many grids.
template <typename T>
struct BatchSys {
    const T* in;
    T* out;
    const T* V;
    int nx, ny, nz;
    KC<T> k;
};
struct BatchItem {
    int sys, x0, y0, z0, z1, band;
};
template <typename T>
constexpr int batch_ry() { return sizeof(T) == 8 ? 2 : 4; }

template <typename T>
__global__ void __launch_bounds__(NT, 2)
fd8_batch_kernel(const BatchSys<T>* __restrict__ sys, const BatchItem* __restrict__ items, int n_items) {
    constexpr int RY = batch_ry<T>();
    constexpr int TY = BY * RY;
    __shared__ T sm[2 * (TY + 2 * HW) * (TX + 2 * HW)];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem w = items[it];
        const BatchSys<T>& S = sys[w.sys];
        fd8_tile<T, false, 1, false, RY>(S.in, S.out, S.V, S.nx, S.ny, S.nz, w.x0, w.y0, w.z0, w.z1, w.band, S.k, sm);
        __syncthreads();   // the next item reuses the shared tiles
    }
}

// ---------------------------------------------------------------------------
// TMA-pipelined stencil (primary path on sm_100a).
//
// The planes of a CTA's tile, with the 4-wide x/y halo, stream through an
// 8-stage shared-memory ring: one 3-D tensor copy (cp.async.bulk.tensor, box
// (TX+8) x (TY+8) x 1) per plane and SoA component, completing on one mbarrier
// per stage.  The tensor copy zero-fills coordinates outside the grid; the
// periodic halo cells of edge tiles (the only out-of-range ones) are written by
// threads from values prefetched two planes ahead.  Plane j (z = z0-4+j) is read
// twice from shared memory: its tile centres into the register z queue when it
// is the newest plane (step j-8) and its x/y neighbours when it is the current
// plane (step j-4); its stage is refilled with plane j+8 once every thread has
// passed the barrier of step j-3 (one barrier per step).  The FD sums are
// evaluated as trees per direction (short FP64 dependency chains); the result
// differs from the reference's left-to-right order only by rounding.
//
// Every wait is bounded: a wait that runs out sets an error bit in *err, all
// threads leave together (a block-wide vote), and the producer first waits (also
// bounded) for the copies it still has in flight.
// ---------------------------------------------------------------------------
constexpr unsigned WAIT_LIMIT = 1u << 22;   // try_wait polls before declaring a timeout
constexpr int ERR_STENCIL_TIMEOUT = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false after WAIT_LIMIT (or `limit`) polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned limit = WAIT_LIMIT) {
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Test setting of the box-fed stencil's wait limits: the environment variable
// QSB_STENCIL_COMPUTE_POLLS (read once per process) makes the compute warps wait
// that many polls on a barrier that nothing arrives at, and the producer's
// stage-release waits give up after as many polls: the waits run out, the
// kernel sets bit 0 of the device error word and returns (the producer first
// waits, with the full limit, for its copies in flight).  Unset: WAIT_LIMIT.
unsigned compute_poll_limit() {
    static unsigned v = 0;
    if (v == 0) {
        v = WAIT_LIMIT;
        if (const char* e = std::getenv("QSB_STENCIL_COMPUTE_POLLS")) {
            const long n = std::strtol(e, nullptr, 10);
            if (n >= 1 && n < (long)WAIT_LIMIT) v = (unsigned)n;
        }
    }
    return v;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------------------
// fd8_zacc_kernel: a ring of TMA-loaded planes (tile + 4-wide halo, periodic
// halo cells written by the threads), consumed one plane per step, with the z
// derivative carried as pending OUTPUTS.
//
// A thread owns RY rows x 2 x-adjacent points and reads shared memory in
// 16-byte pairs.  When plane j lands, its x/y derivatives, centre and V terms
// go into output j, and w_m p_j into the pending outputs j-m and j+m (m = 1..4);
// output j-4 is then complete and stored.  A plane is read from shared memory
// only in the step that consumes it, so the ring needs only the prefetch depth,
// and no z queue of inputs is kept.  Shared memory read per point (RY = 2):
// x 5 pairs per 2 points (2.5 pairs = 5 values) + y 8 pairs per 2 x 2 points
// (4 values) = 9 values, against 14 for a per-point 9-deep z queue with one
// row of x and one column of y per thread.
//
// Same arithmetic terms as fd8_kernel (Laplacian8th_halo_f,
// source/GridDifference8th.h:82-148; LaplacianKpoint8th_halo_f,
// source/GridDifferenceKpoint8th.h:17-120); the z sums are accumulated in
// arrival order, which changes only the rounding (~1e-16 relative).
constexpr int ZX = 16;            // threads along x, two points each
constexpr int ZTX = 2 * ZX;       // tile width in points

template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};

// ZY threads along y, RY rows each; S ring stages; MINB resident CTAs per SM
template <typename T>
__device__ __forceinline__ typename Pair<T>::type lds2(uint32_t a);
template <>
__device__ __forceinline__ double2 lds2<double>(uint32_t a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}

template <typename T, bool CPLX, int ZY, int RY, int S, int MINB>
struct ZCfg {
    static constexpr int NT = ZX * ZY;
    static constexpr int NC = CPLX ? 2 : 1;
    static constexpr int TY = ZY * RY;
    static constexpr int SW = ZTX + 2 * HW;
    static constexpr int SH = TY + 2 * HW;
    static constexpr int COMP = SH * SW;
    static constexpr int STAGE = NC * COMP;
    static constexpr size_t SMEM = (size_t)S * STAGE * sizeof(T) + S * sizeof(uint64_t) + 128;
    static_assert((COMP * sizeof(T)) % 128 == 0, "stage components must stay 128-byte aligned");
    static_assert(8 * TY <= NT && 8 * ZTX <= NT, "one periodic halo cell of each kind per thread");
    static_assert(MINB * SMEM <= 227 * 1024, "MINB CTAs per SM");
};

template <typename T, bool CPLX, int MODE, bool GRAD, int ZY, int RY, int S, int MINB>
__global__ void __launch_bounds__(ZX * ZY, MINB)
fd8_zacc_kernel(const __grid_constant__ CUtensorMap tmap, T* __restrict__ out, const T* __restrict__ in,
                const T* __restrict__ V, int nx, int ny, int nz, int zchunk, KC<T> k, int* __restrict__ err) {
    using C = ZCfg<T, CPLX, ZY, RY, S, MINB>;
    using P2 = typename Pair<T>::type;
    constexpr int NC = C::NC, TY = C::TY, SW = C::SW;
    extern __shared__ unsigned char smraw_[];
    unsigned char* smraw = (unsigned char*)(((uintptr_t)smraw_ + 127) & ~(uintptr_t)127);
    T* ring = reinterpret_cast<T*>(smraw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + (size_t)S * C::STAGE * sizeof(T));

    const int ntx = (nx + ZTX - 1) / ZTX;
    const int x0 = (blockIdx.x % ntx) * ZTX;
    const int y0 = (blockIdx.x / ntx) * TY;
    const int wx = min(ZTX, nx - x0);
    const int wy = min(TY, ny - y0);
    const int z0 = blockIdx.y * zchunk;
    const int z1 = min(nz, z0 + zchunk);
    const int nsteps = z1 - z0;
    const int nplanes = nsteps + 2 * HW;
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
    const int t = ty * ZX + tx;
    // nx is even on this path (16-byte row pitch), so a pair is valid or not as a whole
    const bool xin = 2 * tx < wx;
    bool rv[RY];
#pragma unroll
    for (int i = 0; i < RY; ++i) rv[i] = xin && (ty * RY + i < wy);
    const size_t rowoff = (size_t)(x0 + 2 * tx) + (size_t)nx * (y0 + ty * RY);
    const int soff = (ty * RY + HW) * SW + 2 * tx + HW;   // first centre pair in a component box

    // periodic halo cells (outside [0,nx) x [0,ny), zero-filled by the tensor copy)
    bool xh_ok = false, yh_ok = false;
    size_t xh_g = 0, yh_g = 0;
    int xh_s = 0, yh_s = 0;
    if (t < 8 * TY) {
        const int side = t / (4 * TY), rem = t % (4 * TY), hrow = rem / 4, hk = rem % 4;
        const int gxu = side == 0 ? x0 - HW + hk : x0 + wx + hk;
        xh_ok = hrow < wy && (gxu < 0 || gxu >= nx);
        xh_g = (size_t)wrapi(gxu, nx) + (size_t)nx * (y0 + min(hrow, wy - 1));
        xh_s = (HW + hrow) * SW + (side == 0 ? hk : wx + HW + hk);
    }
    if (t < 8 * ZTX) {
        const int side = t / (4 * ZTX), rem = t % (4 * ZTX), hr = rem / ZTX, hc = rem % ZTX;
        const int gyu = side == 0 ? y0 - HW + hr : y0 + wy + hr;
        yh_ok = hc < wx && (gyu < 0 || gyu >= ny);
        yh_g = (size_t)(x0 + min(hc, wx - 1)) + (size_t)nx * wrapi(gyu, ny);
        yh_s = (side == 0 ? hr : wy + HW + hr) * SW + HW + hc;
    }

    if (t == 0) {
        for (int st = 0; st < S; ++st) mbar_init(&bar[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // producer (thread 0): plane j (z = z0 - 4 + j, wrapped) -> stage j % S
    constexpr uint32_t PLANE_BYTES = (uint32_t)(C::STAGE * sizeof(T));
    int issued = 0;
    auto issue = [&](int j) {
        issued = j + 1;
        const int st = j % S;
        T* stage = ring + (size_t)st * C::STAGE;
        const int zz = wrapi(z0 - HW + j, nz);
        // order the threads' earlier generic-proxy writes (halo cells) to this
        // stage before the tensor copy's async-proxy writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[st], PLANE_BYTES);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int zplane = (CPLX ? 2 * band + c : band) * nz + zz;
            tma_load_3d(stage + c * C::COMP, &tmap, x0 - HW, y0 - HW, zplane, &bar[st]);
        }
    };
    if (t == 0)
        for (int j = 0; j < min(S, nplanes); ++j) issue(j);

    int failed = 0;
    // periodic halo values of inner planes, loaded two planes ahead (4 slots)
    T hx[4][NC], hy[4][NC];
    // epilogue operand one step ahead: V of plane j+1 (MODE 1) or the old value
    // of the output stored at step j+1 (MODE 0)
    constexpr int NE = MODE == 0 ? NC : 1;
    P2 ep[2][NE][RY];
    // pending outputs: slot o % 8 holds output plane o (local index; plane j is
    // z = z0 - 4 + j, output o is stored at step o + 4)
    T A[NC][RY][2][8];
    static_assert(sizeof(T) == 8, "pending-output z sums are FP64 only (FP32 uses fd8_kernel's order)");
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int i = 0; i < RY; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int s8 = 0; s8 < 8; ++s8) A[c][i][h][s8] = T(0);

    for (int jb = 0; jb < nplanes; jb += 8) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = jb + u;
            if (j < nplanes) {
                if (!failed && !mbar_wait(&bar[j % S], (uint32_t)((j / S) & 1))) failed = 1;
                T* cur = ring + (size_t)(j % S) * C::STAGE;
                const bool inner = j >= HW && j < nsteps + HW;
                if (inner) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        if (xh_ok) cur[c * C::COMP + xh_s] = hx[u % 4][c];
                        if (yh_ok) cur[c * C::COMP + yh_s] = hy[u % 4][c];
                    }
                }
                {
                    const int j2 = j + 2;
                    if (j2 >= HW && j2 < nsteps + HW) {
                        const size_t zo2 = nxy * (size_t)(z0 + j2 - HW);
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            hx[(u + 2) % 4][c] = xh_ok ? __ldg(src[c] + xh_g + zo2) : T(0);
                            hy[(u + 2) % 4][c] = yh_ok ? __ldg(src[c] + yh_g + zo2) : T(0);
                        }
                    }
                }
                if (MODE == 1) {
                    const int j1 = j + 1;
                    if (j1 >= HW && j1 < nsteps + HW) {
                        const size_t zo1 = nxy * (size_t)(z0 + j1 - HW);
#pragma unroll
                        for (int i = 0; i < RY; ++i) {
                            P2 v{};
                            if (rv[i]) v = __ldg(reinterpret_cast<const P2*>(V + rowoff + (size_t)nx * i + zo1));
                            ep[(u + 1) % 2][0][i] = v;
                        }
                    }
                } else {
                    const int o1 = j + 1 - HW;
                    if (o1 >= HW && o1 < nsteps + HW) {
                        const size_t zo1 = nxy * (size_t)(z0 + o1 - HW);
#pragma unroll
                        for (int c = 0; c < NE; ++c)
#pragma unroll
                            for (int i = 0; i < RY; ++i) {
                                P2 v{};
                                if (rv[i]) v = *reinterpret_cast<const P2*>(dst[c] + rowoff + (size_t)nx * i + zo1);
                                ep[(u + 1) % 2][c][i] = v;
                            }
                    }
                }
                // halo cells of plane j are written, and every thread has finished
                // step j-1, so stage (j-1) % S is free
                if (__syncthreads_or(failed)) goto drain;
                if (t == 0 && j >= 1 && j + S - 1 < nplanes) issue(j + S - 1);

                P2 pc[NC][RY];
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i)
                        pc[c][i] = *reinterpret_cast<const P2*>(cur + c * C::COMP + soff + i * SW);
#define PV(c, i, h) ((h) ? pc[c][i].y : pc[c][i].x)

                if (inner) {
                    T lxy[NC][RY][2];
                    T gxy[NC][RY][2];
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const T* s = cur + c * C::COMP + soff;
                        P2 col[RY + 8];
#pragma unroll
                        for (int r = 0; r < RY + 8; ++r)
                            col[r] = (r >= HW && r < HW + RY) ? pc[c][r - HW]
                                                             : *reinterpret_cast<const P2*>(s + (r - HW) * SW);
#pragma unroll
                        for (int i = 0; i < RY; ++i) {
                            const T* row = s + i * SW;
                            const P2 L0 = *reinterpret_cast<const P2*>(row - 4);
                            const P2 L1 = *reinterpret_cast<const P2*>(row - 2);
                            const P2 R0 = *reinterpret_cast<const P2*>(row + 2);
                            const P2 R1 = *reinterpret_cast<const P2*>(row + 4);
                            const P2 Cc = pc[c][i];
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                // x neighbours -4..-1, +1..+4 of point h of the pair
                                const T xm4 = h ? L0.y : L0.x, xm3 = h ? L1.x : L0.y;
                                const T xm2 = h ? L1.y : L1.x, xm1 = h ? Cc.x : L1.y;
                                const T xp1 = h ? R0.x : Cc.y, xp2 = h ? R0.y : R0.x;
                                const T xp3 = h ? R1.x : R0.y, xp4 = h ? R1.y : R1.x;
                                const T ym4 = h ? col[i].y : col[i].x, yp4 = h ? col[i + 8].y : col[i + 8].x;
                                const T ym3 = h ? col[i + 1].y : col[i + 1].x, yp3 = h ? col[i + 7].y : col[i + 7].x;
                                const T ym2 = h ? col[i + 2].y : col[i + 2].x, yp2 = h ? col[i + 6].y : col[i + 6].x;
                                const T ym1 = h ? col[i + 3].y : col[i + 3].x, yp1 = h ? col[i + 5].y : col[i + 5].x;
                                const T sxx = (k.cx[3] * (xp4 + xm4) + k.cx[2] * (xp3 + xm3)) +
                                              (k.cx[1] * (xp2 + xm2) + k.cx[0] * (xp1 + xm1));
                                const T syy = (k.cy[3] * (yp4 + ym4) + k.cy[2] * (yp3 + ym3)) +
                                              (k.cy[1] * (yp2 + ym2) + k.cy[0] * (yp1 + ym1));
                                lxy[c][i][h] = sxx + syy;
                                if (GRAD) {
                                    const T gx_ = (k.ax[3] * (xp4 - xm4) + k.ax[2] * (xp3 - xm3)) +
                                                  (k.ax[1] * (xp2 - xm2) + k.ax[0] * (xp1 - xm1));
                                    const T gy_ = (k.ay[3] * (yp4 - ym4) + k.ay[2] * (yp3 - ym3)) +
                                                  (k.ay[1] * (yp2 - ym2) + k.ay[0] * (yp1 - ym1));
                                    gxy[c][i][h] = gx_ + gy_;
                                }
                            }
                        }
                    }
                    // centre, V and in-plane terms of output j (slot u)
#pragma unroll
                    for (int c = 0; c < NC; ++c)
#pragma unroll
                        for (int i = 0; i < RY; ++i)
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                const T p = PV(c, i, h);
                                T r = k.c0 * p + lxy[c][i][h];
                                if (MODE == 1) r += (h ? ep[u % 2][0][i].y : ep[u % 2][0][i].x) * p;
                                // out_re = L(re) - D(im), out_im = L(im) + D(re)
                                if (CPLX && GRAD) r += c == 0 ? -gxy[NC - 1][i][h] : gxy[0][i][h];
                                A[c][i][h][u] += r;
                            }
                }

                // plane j enters outputs j -+ m (m = 1..3); output j-4 takes its last term
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const T p = PV(c, i, h);
                            A[c][i][h][(u + 7) % 8] += k.cz[0] * p;
                            A[c][i][h][(u + 1) % 8] += k.cz[0] * p;
                            A[c][i][h][(u + 6) % 8] += k.cz[1] * p;
                            A[c][i][h][(u + 2) % 8] += k.cz[1] * p;
                            A[c][i][h][(u + 5) % 8] += k.cz[2] * p;
                            A[c][i][h][(u + 3) % 8] += k.cz[2] * p;
                            A[c][i][h][(u + 4) % 8] += k.cz[3] * p;
                            if (CPLX && GRAD) {
                                // D z-part: +a_m q[o+m] (o = j-m), -a_m q[o-m] (o = j+m)
                                const T q = PV(NC - 1 - c, i, h);
                                const T w = c == 0 ? -q : q;
                                A[c][i][h][(u + 7) % 8] += k.az[0] * w;
                                A[c][i][h][(u + 1) % 8] -= k.az[0] * w;
                                A[c][i][h][(u + 6) % 8] += k.az[1] * w;
                                A[c][i][h][(u + 2) % 8] -= k.az[1] * w;
                                A[c][i][h][(u + 5) % 8] += k.az[2] * w;
                                A[c][i][h][(u + 3) % 8] -= k.az[2] * w;
                                A[c][i][h][(u + 4) % 8] += k.az[3] * w;
                            }
                        }
                // output j-4 (z = z0 + j - 8) is complete
                if (j >= 2 * HW) {
                    const size_t zo = nxy * (size_t)(z0 + j - 2 * HW);
#pragma unroll
                    for (int i = 0; i < RY; ++i) {
                        if (!rv[i]) continue;
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            P2 r;
                            r.x = A[c][i][0][(u + 4) % 8];
                            r.y = A[c][i][1][(u + 4) % 8];
                            if (MODE == 0) {
                                r.x += ep[u % 2][c][i].x;
                                r.y += ep[u % 2][c][i].y;
                            }
                            *reinterpret_cast<P2*>(dst[c] + rowoff + (size_t)nx * i + zo) = r;
                        }
                    }
                }
                // the freed slot starts output j+4 with plane j's term
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            T a = k.cz[3] * PV(c, i, h);
                            if (CPLX && GRAD) {
                                const T q = PV(NC - 1 - c, i, h);
                                a -= k.az[3] * (c == 0 ? -q : q);
                            }
                            A[c][i][h][(u + 4) % 8] = a;
                        }
#undef PV
            }
        }
    }
    return;

drain:
    // a wait ran out: record it and wait (bounded) for this CTA's copies in flight
    if (t == 0) {
        atomicOr(err, ERR_STENCIL_TIMEOUT);
        for (int st = 0; st < S; ++st) {
            int jmax = -1;
            for (int j = st; j < issued; j += S) jmax = j;
            if (jmax >= 0) (void)mbar_wait(&bar[st], (uint32_t)((jmax / S) & 1));
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// fd8_ws_kernel: the pending-output z accumulation of fd8_zacc_kernel, fed
// only by the tensor-memory accelerator.
//
// Per plane, one producer lane issues into a ring stage:
//   * the 40 x (TY+8) psi box of the tile and its 4-wide halo; at a y boundary
//     as top / body / bottom boxes at wrapped y coordinates, so the periodic
//     halo rows land in place (same 40-element pitch);
//   * at an x boundary, the 4 wrapped columns of the tile's rows as a side box
//     (4-element pitch; only the tile's own rows need x neighbours); the
//     zero-filled columns of the main box there are never read;
//   * the 32 x TY tile of V (MODE 1) or of the old output (MODE 0).
// The eight compute warps read shared memory only (no global load in the z
// loop, whose latency measured as the stall of the register-prefetch form)
// and hand each stage back through an mbarrier: no CTA-wide barrier per plane.
// Issuing the copies from a compute warp instead (lane 0 probing the stage
// releases at every step, no producer warp, 255 registers per thread) measured
// 1.03 against 0.42 ms: plane issue then follows that warp's progress.
// Tiles that would pass the grid edge are shifted back inside it and store only
// the points of their own nominal tile.
constexpr int WCW = 8;                    // compute warps: 16 x 16 threads
constexpr int WNT = (WCW + 1) * 32;       // + one producer warp

template <typename T, bool CPLX, int MODE, int RY, int S>
struct WsCfg {
    static constexpr int NC = CPLX ? 2 : 1;
    static constexpr int NE = MODE == 0 ? NC : 1;
    static constexpr int TY = 16 * RY;
    static constexpr int SW = ZTX + 2 * HW;                 // main pitch (40)
    static constexpr int MROWS = TY + 2 * HW;
    static constexpr int MAIN = MROWS * SW;                 // one component's main box
    static constexpr int SIDE = TY * HW;                    // side buffer: the tile's rows x 4
    static constexpr int EBOX = TY * ZTX;                   // V / old-output tile
    static constexpr int OFF_SIDE = NC * MAIN;              // side[c][L|R]
    static constexpr int OFF_E = OFF_SIDE + NC * 2 * SIDE;
    static constexpr int STAGE = OFF_E + NE * EBOX;
    static constexpr size_t SMEM = (size_t)S * STAGE * sizeof(T) + (2 * S + 1) * sizeof(uint64_t) + 128;
    static constexpr uint32_t MAIN_BYTES = (uint32_t)(MAIN * sizeof(T));
    static constexpr uint32_t SIDE_BYTES = (uint32_t)(SIDE * sizeof(T));
    static constexpr uint32_t E_BYTES = (uint32_t)(EBOX * sizeof(T));
    // every tensor copy lands on a 128-byte boundary
    static_assert((MAIN * sizeof(T)) % 128 == 0 && (SIDE * sizeof(T)) % 128 == 0 && (EBOX * sizeof(T)) % 128 == 0,
                  "stage parts aligned");
    static_assert((HW * SW * sizeof(T)) % 128 == 0 && ((TY + HW) * SW * sizeof(T)) % 128 == 0, "main sub-boxes");
    static_assert(SMEM <= 227 * 1024, "one CTA per SM");
};

struct WsMaps {
    CUtensorMap full, body, four;      // psi: 40 x (TY+8), 40 x TY, 40 x 4
    CUtensorMap side;                  // psi: 4 x TY
    CUtensorMap e;                     // V (MODE 1) or out (MODE 0): 32 x TY
};

// Geometry of one work item (tile x z chunk x band) of fd8_ws_kernel.
struct WsItem {
    int x0n, y0n;          // nominal tile: the points this item stores
    int x0, y0;            // loaded tile, inside the grid
    int ytop, ybot;        // wrapped first rows of the top / bottom halo
    int z0, nsteps, band;
    bool ledge, redge, yedge;
};

template <int TY>
__device__ __forceinline__ WsItem ws_item(int w, int nx, int ny, int nz, int zchunk, int tiles, int nzc) {
    WsItem it;
    const int tile = w % tiles, rest = w / tiles;
    it.band = rest / nzc;
    const int ntx = (nx + ZTX - 1) / ZTX;
    it.x0n = (tile % ntx) * ZTX;
    it.y0n = (tile / ntx) * TY;
    it.x0 = min(it.x0n, nx - ZTX);
    it.y0 = min(it.y0n, ny - TY);
    it.ledge = it.x0 == 0;
    it.redge = it.x0 + ZTX == nx;
    it.yedge = it.y0 < HW || it.y0 + TY + HW > ny;
    it.ytop = it.y0 - HW < 0 ? it.y0 - HW + ny : it.y0 - HW;
    it.ybot = it.y0 + TY >= ny ? it.y0 + TY - ny : it.y0 + TY;
    it.z0 = (rest % nzc) * zchunk;
    it.nsteps = min(nz, it.z0 + zchunk) - it.z0;
    return it;
}

// One CTA per item (blockIdx.x).  A persistent form (one CTA per SM walking
// the items, the ring running on across them) measured slower: 0.49 against
// 0.42 ms at 96^3 x 128 bands.
// Register budget, given to the compiler as a cap (__maxnreg__) rather than
// through __launch_bounds__: 9 warps (8 compute + the producer) take the
// register file of 12 (the allocation rounds a CTA's warps up to a multiple of
// four), 65536 / 384 = 170 -> 168 per thread at one CTA per SM.  With the cap
// stated directly the compiler kept the 168-register form free of the spills
// the launch-bounds form had (0.450 -> 0.417 ms at 96^3 x 128 bands, FP64).
// WT: the wait-limit test form (compute_poll_limit set); a separate
// instantiation, so that the production kernel carries none of it.
template <typename T, bool CPLX, int MODE, bool GRAD, bool ISO, int RY, int S, bool WT>
__global__ void __maxnreg__(168)
fd8_ws_kernel(const __grid_constant__ WsMaps maps, T* __restrict__ out, int nx, int ny, int nz, int zchunk, int tiles,
              int nzc, int items, KC<T> k, int* __restrict__ err, unsigned cpolls) {
    using C = WsCfg<T, CPLX, MODE, RY, S>;
    using P2 = typename Pair<T>::type;
    constexpr int NC = C::NC, NE = C::NE, TY = C::TY, SW = C::SW;
    extern __shared__ unsigned char smraw_[];
    unsigned char* smraw = (unsigned char*)(((uintptr_t)smraw_ + 127) & ~(uintptr_t)127);
    T* ring = reinterpret_cast<T*>(smraw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smraw + (size_t)S * C::STAGE * sizeof(T));
    uint64_t* empty = full + S;
    uint64_t* never = empty + S;   // no thread ever arrives here (the wait-limit test)
    const size_t nxy = (size_t)nx * ny;
    const size_t N = nxy * nz;
    const int t = threadIdx.y * ZX + threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    // cpolls < WAIT_LIMIT: the test setting of the wait limits (compute_poll_limit):
    // the compute warps first wait, with that limit, on a barrier nothing
    // arrives at, and the producer's stage-release waits use it too; the
    // producer's drain of its own copies keeps the full limit
    constexpr bool wait_test = WT;

    if (t == 0) {
        for (int st = 0; st < S; ++st) {
            mbar_init(&full[st], 1);
            mbar_init(&empty[st], WCW);
        }
        if constexpr (WT) mbar_init(never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == WCW) {
        // ---------------- producer ----------------
        if (lane != 0) return;
        const WsItem it = ws_item<TY>(blockIdx.x, nx, ny, nz, zchunk, tiles, nzc);
        const int nplanes = it.nsteps + 2 * HW;
        const uint32_t psi_bytes =
            NC * (C::MAIN_BYTES + ((it.ledge ? 1 : 0) + (it.redge ? 1 : 0)) * C::SIDE_BYTES);
        int issued = 0;
        bool failed = false;
        for (int j = 0; j < nplanes; ++j) {
            const int st = j % S;
            // stage st last held plane j - S: wait until every compute warp released it
            if (j >= S && !mbar_wait(&empty[st], (uint32_t)(((j / S) - 1) & 1), WT ? cpolls : WAIT_LIMIT)) {
                failed = true;
                break;
            }
            const bool e_on = MODE == 1 ? (j >= HW && j < it.nsteps + HW) : (j >= 2 * HW);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&full[st], psi_bytes + (e_on ? NE * C::E_BYTES : 0u));
            T* stage = ring + (size_t)st * C::STAGE;
            const int zz = wrapi(it.z0 - HW + j, nz);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int zp = (CPLX ? 2 * it.band + c : it.band) * nz + zz;
                T* mb = stage + c * C::MAIN;
                if (!it.yedge) {
                    tma_load_3d(mb, &maps.full, it.x0 - HW, it.y0 - HW, zp, &full[st]);
                } else {
                    tma_load_3d(mb, &maps.four, it.x0 - HW, it.ytop, zp, &full[st]);
                    tma_load_3d(mb + HW * SW, &maps.body, it.x0 - HW, it.y0, zp, &full[st]);
                    tma_load_3d(mb + (TY + HW) * SW, &maps.four, it.x0 - HW, it.ybot, zp, &full[st]);
                }
#pragma unroll
                for (int sd = 0; sd < 2; ++sd) {
                    if (sd == 0 ? !it.ledge : !it.redge) continue;
                    tma_load_3d(stage + C::OFF_SIDE + (c * 2 + sd) * C::SIDE, &maps.side, sd == 0 ? nx - HW : 0,
                                it.y0, zp, &full[st]);
                }
            }
            if (e_on) {
                T* eb = stage + C::OFF_E;
                if (MODE == 1) {
                    tma_load_3d(eb, &maps.e, it.x0, it.y0, it.z0 + j - HW, &full[st]);
                } else {
#pragma unroll
                    for (int c = 0; c < NE; ++c)
                        tma_load_3d(eb + c * C::EBOX, &maps.e, it.x0, it.y0,
                                    (CPLX ? 2 * it.band + c : it.band) * nz + it.z0 + j - 2 * HW, &full[st]);
                }
            }
            issued = j + 1;
        }
        if (failed) {
            atomicOr(err, ERR_STENCIL_TIMEOUT);
            // copies in flight must land before the CTA may exit
            for (int st = 0; st < S && st < issued; ++st) {
                const int last = st + ((issued - 1 - st) / S) * S;
                (void)mbar_wait(&full[st], (uint32_t)((last / S) & 1));
            }
        }
        return;
    }

    // ---------------- compute warps ----------------
    // shared memory is addressed with 32-bit offsets (ld.shared) throughout
    constexpr uint32_t TB = sizeof(T);
    const uint32_t ring_u = smem_u32(ring);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const uint32_t soff = ((ty * RY + HW) * SW + 2 * tx + HW) * TB;    // centre pair (main box)
    const uint32_t eoff = (C::OFF_E + ty * RY * ZTX + 2 * tx) * TB;    // V / old output pair
    bool failed = false;
    if constexpr (WT) failed = __any_sync(0xffffffffu, !mbar_wait(never, 0, cpolls));
    {
    const WsItem it = ws_item<TY>(blockIdx.x, nx, ny, nz, zchunk, tiles, nzc);
    const int x0 = it.x0, y0 = it.y0, z0 = it.z0, nsteps = it.nsteps, band = it.band;
    const bool ledge = it.ledge, redge = it.redge;
    const int nplanes = nsteps + 2 * HW;
    const int gx = x0 + 2 * tx;
    bool own[RY];
#pragma unroll
    for (int i = 0; i < RY; ++i) own[i] = gx >= it.x0n && y0 + ty * RY + i >= it.y0n;
    // this thread's first output pair of each component, in plane z = 0
    T* dst[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
        dst[c] = out + (CPLX ? (size_t)(2 * band + c) : (size_t)band) * N + (size_t)gx + (size_t)nx * (y0 + ty * RY);
    // the five x pairs of the thread's first row: byte offset (component 0),
    // row pitch in bytes, and whether they sit in a side buffer
    uint32_t xo[5], xp[5];
    bool xs[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const int cm = 2 * tx + 2 * m;          // column in the 40-wide main box
        const int r = ty * RY + HW;             // row of the first point
        if (ledge && cm < HW) {
            xo[m] = (C::OFF_SIDE + (r - HW) * HW + cm) * TB;
            xp[m] = HW * TB;
            xs[m] = true;
        } else if (redge && cm >= ZTX + HW) {
            xo[m] = (C::OFF_SIDE + C::SIDE + (r - HW) * HW + (cm - ZTX - HW)) * TB;
            xp[m] = HW * TB;
            xs[m] = true;
        } else {
            xo[m] = (r * SW + cm) * TB;
            xp[m] = SW * TB;
            xs[m] = false;
        }
    }

    T A[NC][RY][2][8];
    static_assert(sizeof(T) == 8, "pending-output z sums are FP64 only (FP32 uses fd8_kernel's order)");
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int i = 0; i < RY; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int s8 = 0; s8 < 8; ++s8) A[c][i][h][s8] = T(0);
    for (int jb = 0; jb < nplanes && !failed; jb += 8) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = jb + u;
            if (j < nplanes && !failed) {
                const int st = j % S;
                const bool ok = mbar_wait(&full[st], (uint32_t)((j / S) & 1), WT ? cpolls : WAIT_LIMIT);
                if (__any_sync(0xffffffffu, !ok)) {
                    failed = true;
                    continue;
                }
                const uint32_t cur = ring_u + (uint32_t)st * (uint32_t)(C::STAGE * TB);
                const bool inner = j >= HW && j < nsteps + HW;
                P2 pc[NC][RY];
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i) pc[c][i] = lds2<T>(cur + c * C::MAIN * TB + soff + i * SW * TB);
#define PV(c, i, h) ((h) ? pc[c][i].y : pc[c][i].x)
                // in-plane sums per point: ISO, (x+y) pairs per offset m; else x and y apart
                T sm[NC][RY][2][4];
                T syy[NC][RY][2];
                T gxy[NC][RY][2];
                P2 ev[NE][RY];
                if (inner) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const uint32_t sc = cur + c * C::MAIN * TB + soff;
                        P2 col[RY + 8];
#pragma unroll
                        for (int r = 0; r < RY + 8; ++r)
                            col[r] = (r >= HW && r < HW + RY) ? pc[c][r - HW]
                                                             : lds2<T>(sc + (uint32_t)((r - HW) * SW * (int)TB));
#pragma unroll
                        for (int i = 0; i < RY; ++i) {
                            P2 xv[5];
#pragma unroll
                            for (int m = 0; m < 5; ++m)
                                xv[m] = m == 2 ? pc[c][i]
                                               : lds2<T>(cur + xo[m] + (xs[m] ? c * 2 * C::SIDE * TB : c * C::MAIN * TB) +
                                                         i * xp[m]);
                            const P2 L0 = xv[0], L1 = xv[1], Cc = xv[2], R0 = xv[3], R1 = xv[4];
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                // x neighbours -4..-1, +1..+4 of point h of the pair
                                const T xm4 = h ? L0.y : L0.x, xm3 = h ? L1.x : L0.y;
                                const T xm2 = h ? L1.y : L1.x, xm1 = h ? Cc.x : L1.y;
                                const T xp1 = h ? R0.x : Cc.y, xp2 = h ? R0.y : R0.x;
                                const T xp3 = h ? R1.x : R0.y, xp4 = h ? R1.y : R1.x;
                                const T ym4 = h ? col[i].y : col[i].x, yp4 = h ? col[i + 8].y : col[i + 8].x;
                                const T ym3 = h ? col[i + 1].y : col[i + 1].x, yp3 = h ? col[i + 7].y : col[i + 7].x;
                                const T ym2 = h ? col[i + 2].y : col[i + 2].x, yp2 = h ? col[i + 6].y : col[i + 6].x;
                                const T ym1 = h ? col[i + 3].y : col[i + 3].x, yp1 = h ? col[i + 5].y : col[i + 5].x;
                                if (ISO) {
                                    sm[c][i][h][0] = (xp1 + xm1) + (yp1 + ym1);
                                    sm[c][i][h][1] = (xp2 + xm2) + (yp2 + ym2);
                                    sm[c][i][h][2] = (xp3 + xm3) + (yp3 + ym3);
                                    sm[c][i][h][3] = (xp4 + xm4) + (yp4 + ym4);
                                } else {
                                    sm[c][i][h][0] = xp1 + xm1;
                                    sm[c][i][h][1] = xp2 + xm2;
                                    sm[c][i][h][2] = xp3 + xm3;
                                    sm[c][i][h][3] = xp4 + xm4;
                                    syy[c][i][h] = (k.cy[3] * (yp4 + ym4) + k.cy[2] * (yp3 + ym3)) +
                                                   (k.cy[1] * (yp2 + ym2) + k.cy[0] * (yp1 + ym1));
                                }
                                if (GRAD) {
                                    const T gx_ = (k.ax[3] * (xp4 - xm4) + k.ax[2] * (xp3 - xm3)) +
                                                  (k.ax[1] * (xp2 - xm2) + k.ax[0] * (xp1 - xm1));
                                    const T gy_ = (k.ay[3] * (yp4 - ym4) + k.ay[2] * (yp3 - ym3)) +
                                                  (k.ay[1] * (yp2 - ym2) + k.ay[0] * (yp1 - ym1));
                                    gxy[c][i][h] = gx_ + gy_;
                                }
                            }
                        }
                    }
                    if (MODE == 1) {
#pragma unroll
                        for (int i = 0; i < RY; ++i) ev[0][i] = lds2<T>(cur + eoff + i * ZTX * TB);
                    }
                }
                if (MODE == 0 && j >= 2 * HW) {
#pragma unroll
                    for (int c = 0; c < NE; ++c)
#pragma unroll
                        for (int i = 0; i < RY; ++i) ev[c][i] = lds2<T>(cur + eoff + (c * C::EBOX + i * ZTX) * TB);
                }
                // every value of plane j is in registers: hand the stage back
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[st]);

                if (inner) {
                    // centre, V and in-plane terms of output j (slot u), as two
                    // independent chains
#pragma unroll
                    for (int c = 0; c < NC; ++c)
#pragma unroll
                        for (int i = 0; i < RY; ++i)
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                const T p = PV(c, i, h);
                                const T v = MODE == 1 ? (h ? ev[0][i].y : ev[0][i].x) : T(0);
                                T r1 = (k.c0 + v) * p;
                                r1 += k.cx[0] * sm[c][i][h][0];
                                r1 += k.cx[1] * sm[c][i][h][1];
                                T r2 = k.cx[3] * sm[c][i][h][3];
                                r2 += k.cx[2] * sm[c][i][h][2];
                                if (!ISO) r2 += syy[c][i][h];
                                // out_re = L(re) - D(im), out_im = L(im) + D(re)
                                if (CPLX && GRAD) r2 += c == 0 ? -gxy[NC - 1][i][h] : gxy[0][i][h];
                                A[c][i][h][u] += r1 + r2;
                            }
                }
                // plane j enters outputs j -+ m (m = 1..3); output j-4 takes its last term
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const T p = PV(c, i, h);
                            A[c][i][h][(u + 7) % 8] += k.cz[0] * p;
                            A[c][i][h][(u + 1) % 8] += k.cz[0] * p;
                            A[c][i][h][(u + 6) % 8] += k.cz[1] * p;
                            A[c][i][h][(u + 2) % 8] += k.cz[1] * p;
                            A[c][i][h][(u + 5) % 8] += k.cz[2] * p;
                            A[c][i][h][(u + 3) % 8] += k.cz[2] * p;
                            A[c][i][h][(u + 4) % 8] += k.cz[3] * p;
                            if (CPLX && GRAD) {
                                // D z-part: +a_m q[o+m] (o = j-m), -a_m q[o-m] (o = j+m)
                                const T q = PV(NC - 1 - c, i, h);
                                const T w = c == 0 ? -q : q;
                                A[c][i][h][(u + 7) % 8] += k.az[0] * w;
                                A[c][i][h][(u + 1) % 8] -= k.az[0] * w;
                                A[c][i][h][(u + 6) % 8] += k.az[1] * w;
                                A[c][i][h][(u + 2) % 8] -= k.az[1] * w;
                                A[c][i][h][(u + 5) % 8] += k.az[2] * w;
                                A[c][i][h][(u + 3) % 8] -= k.az[2] * w;
                                A[c][i][h][(u + 4) % 8] += k.az[3] * w;
                            }
                        }
                // output j-4 (z = z0 + j - 8) is complete
                if (j >= 2 * HW) {
                    const size_t zo = nxy * (size_t)(z0 + j - 2 * HW);
#pragma unroll
                    for (int i = 0; i < RY; ++i) {
                        if (!own[i]) continue;
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            P2 r;
                            r.x = A[c][i][0][(u + 4) % 8];
                            r.y = A[c][i][1][(u + 4) % 8];
                            if (MODE == 0) {
                                r.x += ev[c][i].x;
                                r.y += ev[c][i].y;
                            }
                            *reinterpret_cast<P2*>(dst[c] + (size_t)nx * i + zo) = r;
                        }
                    }
                }
                // the freed slot starts output j+4 with plane j's term
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int i = 0; i < RY; ++i)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            T a = k.cz[3] * PV(c, i, h);
                            if (CPLX && GRAD) {
                                const T q = PV(NC - 1 - c, i, h);
                                a -= k.az[3] * (c == 0 ? -q : q);
                            }
                            A[c][i][h][(u + 4) % 8] = a;
                        }
#undef PV
            }
        }
    }
    }
    if (failed && lane == 0) atomicOr(err, ERR_STENCIL_TIMEOUT);
}


// cuTensorMapEncodeTiled, looked up once through the runtime (no libcuda link)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// 3-D map over the band bundle viewed as [planes*nz][ny][nx], box (TX+8, TY+8, 1)
template <typename T>
bool make_plane_map(CUtensorMap* map, const void* base, int nx, int ny, long long zplanes, int box_y) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)zplanes};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(T), (cuuint64_t)nx * ny * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)(TX + 2 * HW), (cuuint32_t)box_y, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Stencil kernel choice (FP64): 0 fd8_ws_kernel (default; fd8_zacc_kernel where its tiling
// does not apply, fd8_kernel without 16-byte alignment), 2 fd8_kernel (register
// prefetch, no TMA), 3 fd8_zacc_kernel; QSB_STENCIL=ws|reg|zacc overrides it for
// A/B timing.
int stencil_variant() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("QSB_STENCIL");
        v = 0;
        if (e && std::string(e) == "reg") v = 2;
        if (e && std::string(e) == "zacc") v = 3;

    }
    return v;
}

// 3-D map with a (bw, bh, 1) box over an array viewed as [zplanes][ny][nx]
template <typename T>
bool make_box_map(CUtensorMap* map, const void* base, int nx, int ny, long long zplanes, int bw, int bh) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)zplanes};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(T), (cuuint64_t)nx * ny * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// SMs of the current device (one persistent CTA each)
int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
}

// A grid extent the box-fed kernel covers: one tile, or tiles (the last one
// shifted back inside the grid) whose 4-wide halos never straddle the periodic
// boundary.
bool ws_dim_ok(int n, int tile) { return n == tile || (n >= tile + HW && (n % tile == 0 || n % tile >= HW)); }

template <typename T, bool CPLX, int MODE, int RY, int S, int MINB = 1>
bool launch_ws(const StencilLaunch& L, const FD8Coef& c, const KC<T>& k, cudaStream_t s) {
    using C = WsCfg<T, CPLX, MODE, RY, S>;
    if (!ws_dim_ok(L.nx, ZTX) || !ws_dim_ok(L.ny, C::TY) || L.nz < HW) return false;
    const long long planes = (long long)L.nz * L.nb * (CPLX ? 2 : 1);
    WsMaps m;
    bool ok = make_box_map<T>(&m.full, L.in, L.nx, L.ny, planes, C::SW, C::TY + 2 * HW) &&
              make_box_map<T>(&m.body, L.in, L.nx, L.ny, planes, C::SW, C::TY) &&
              make_box_map<T>(&m.four, L.in, L.nx, L.ny, planes, C::SW, HW) &&
              make_box_map<T>(&m.side, L.in, L.nx, L.ny, planes, HW, C::TY);
    if (MODE == 1) ok = ok && make_box_map<T>(&m.e, L.V, L.nx, L.ny, L.nz, ZTX, C::TY);
    else ok = ok && make_box_map<T>(&m.e, L.out, L.nx, L.ny, planes, ZTX, C::TY);
    if (!ok) return false;
    const int tiles = ((L.nx + ZTX - 1) / ZTX) * ((L.ny + C::TY - 1) / C::TY);
    // at least 3 CTAs per SM; split z only when tiles x bands is small,
    // keeping chunks of >= 16 planes
    const int sms = sm_count();
    int zsplit = 1;
    while ((long long)tiles * L.nb * zsplit < 3LL * sms && L.nz / (zsplit * 2) >= 16) zsplit *= 2;
    const int zchunk = (L.nz + zsplit - 1) / zsplit;
    const int nzc = (L.nz + zchunk - 1) / zchunk;
    const long long items = (long long)tiles * nzc * L.nb;
    if (items > (1LL << 30)) return false;
    dim3 grid((unsigned)items), block(ZX, WNT / ZX);
    // equal x and y weights (hx == hy): the x and y pairs of each offset are summed first
    bool iso = true;
    for (int q = 0; q < 4; ++q) iso = iso && k.cx[q] == k.cy[q];
    const bool wt = compute_poll_limit() < WAIT_LIMIT;
    auto kern = CPLX && c.has_grad ? (iso ? fd8_ws_kernel<T, CPLX, MODE, CPLX, true, RY, S, false>
                                          : fd8_ws_kernel<T, CPLX, MODE, CPLX, false, RY, S, false>)
                                   : (iso ? fd8_ws_kernel<T, CPLX, MODE, false, true, RY, S, false>
                                          : fd8_ws_kernel<T, CPLX, MODE, false, false, RY, S, false>);
    if (wt)
        kern = CPLX && c.has_grad ? (iso ? fd8_ws_kernel<T, CPLX, MODE, CPLX, true, RY, S, true>
                                         : fd8_ws_kernel<T, CPLX, MODE, CPLX, false, RY, S, true>)
                                  : (iso ? fd8_ws_kernel<T, CPLX, MODE, false, true, RY, S, true>
                                         : fd8_ws_kernel<T, CPLX, MODE, false, false, RY, S, true>);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    kern<<<grid, block, C::SMEM, s>>>(m, (T*)L.out, L.nx, L.ny, L.nz, zchunk, tiles, nzc, (int)items, k,
                                      device_error_word(), compute_poll_limit());
    return true;
}

template <typename T, bool CPLX, int MODE, int ZY, int RY, int SREQ, int MINB>
bool launch_zacc(const StencilLaunch& L, const FD8Coef& c, const KC<T>& k, cudaStream_t s) {
    // ring depth: SREQ stages, or as many as fit MINB CTAs per SM
    constexpr int STAGE_B = (CPLX ? 2 : 1) * (ZY * RY + 2 * HW) * (ZTX + 2 * HW) * (int)sizeof(T);
    constexpr int SFIT = (227 * 1024 / MINB - 256) / STAGE_B;
    constexpr int S = SREQ < SFIT ? SREQ : SFIT;
    static_assert(S >= 3, "ring too shallow");
    using C = ZCfg<T, CPLX, ZY, RY, S, MINB>;
    const int tiles = ((L.nx + ZTX - 1) / ZTX) * ((L.ny + C::TY - 1) / C::TY);
    // enough CTAs for 148 SMs x MINB x 3 waves; split z only when tiles x bands
    // is small, keeping chunks of >= 16 planes
    int zsplit = 1;
    while ((long long)tiles * L.nb * zsplit < 148LL * MINB * 3 && L.nz / (zsplit * 2) >= 16) zsplit *= 2;
    const int zchunk = (L.nz + zsplit - 1) / zsplit;
    dim3 grid(tiles, (L.nz + zchunk - 1) / zchunk, L.nb), block(ZX, ZY);
    CUtensorMap map;
    if (!make_plane_map<T>(&map, L.in, L.nx, L.ny, (long long)L.nz * L.nb * (CPLX ? 2 : 1), C::TY + 2 * HW))
        return false;
    if (CPLX && c.has_grad) {
        auto kern = fd8_zacc_kernel<T, CPLX, MODE, CPLX, ZY, RY, S, MINB>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        kern<<<grid, block, C::SMEM, s>>>(map, (T*)L.out, (const T*)L.in, (const T*)L.V, L.nx, L.ny, L.nz, zchunk, k,
                                          device_error_word());
    } else {
        auto kern = fd8_zacc_kernel<T, CPLX, MODE, false, ZY, RY, S, MINB>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        kern<<<grid, block, C::SMEM, s>>>(map, (T*)L.out, (const T*)L.in, (const T*)L.V, L.nx, L.ny, L.nz, zchunk, k,
                                          device_error_word());
    }
    return true;
}

template <typename T, bool CPLX, int MODE>
void launch_t(const StencilLaunch& L, const FD8Coef& c, cudaStream_t s, int variant) {
    // rows per thread: as many as fit 128 registers without spilling
    constexpr int RY = (CPLX || sizeof(T) == 8) ? 2 : 4;
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
    // TMA path: the tensor map needs 16-byte aligned base and row pitch
    const int vec = 16 / (int)sizeof(T);
    const bool aligned = (L.nx % vec == 0) && (((uintptr_t)L.in) % 16 == 0);
    // the pending-output kernel also moves out / V / old values in 16-byte pairs
    const bool pairs_ok = ((uintptr_t)L.out % 16 == 0) && (L.V == nullptr || (uintptr_t)L.V % 16 == 0);
    // FP64 only: the pending-output z sums round at 2^-24 of the ~|c0| partial
    // sums in FP32, which measured as a 4e-6..6e-6 Ha eigenvalue floor of the
    // mixed solver at h = 0.125 bohr against 8e-7 with fd8_kernel's order
    // (centre + (x + y neighbours + z neighbours), each completed first)
    if constexpr (sizeof(T) == 8) {
        if (aligned && pairs_ok && L.tma_ok && variant == 0) {
            // rows per thread: 2 (complex: 1, within the register file at one CTA per SM).
            // Measured alternatives (real, 96^3 x 128 bands, FP64): 1 row per thread
            // at two CTAs per SM 0.474-0.502 ms (more shared loads per point); 3 rows
            // need 224 registers, which 9 warps cannot have (launch out of
            // resources); ring depth 4 / 5 / 6 / 8 stages: 0.473 / 0.428 / 0.419 / 0.463 ms.
            constexpr int WRY = CPLX ? 1 : 2;
            constexpr int WS = CPLX ? 8 : 6;
            if (launch_ws<T, CPLX, MODE, WRY, WS>(L, c, k, s)) return;
        }

        if (aligned && pairs_ok && L.tma_ok && (variant == 0 || variant == 3)) {
            // real 2 rows / 1 CTA per SM (212 registers), complex 1 row
            const bool done = CPLX ? launch_zacc<T, CPLX, MODE, 16, 1, 8, 1>(L, c, k, s)
                                   : launch_zacc<T, CPLX, MODE, 16, 2, 8, 1>(L, c, k, s);
            if (done) return;
        }
    }
    if (CPLX && c.has_grad)
        fd8_kernel<T, CPLX, MODE, CPLX, RY><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx,
                                                                   L.ny, L.nz, zchunk, k);
    else
        fd8_kernel<T, CPLX, MODE, false, RY><<<grid, block, 0, s>>>((const T*)L.in, (T*)L.out, (const T*)L.V, L.nx,
                                                                    L.ny, L.nz, zchunk, k);
}

template <typename T>
qsb_status launch_dtype(const StencilLaunch& L, const FD8Coef& c, cudaStream_t s, int variant) {
    if (L.mode == 0) {
        if (L.is_complex) launch_t<T, true, 0>(L, c, s, variant);
        else launch_t<T, false, 0>(L, c, s, variant);
    } else {
        if (L.is_complex) launch_t<T, true, 1>(L, c, s, variant);
        else launch_t<T, false, 1>(L, c, s, variant);
    }
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

// ---------------------------------------------------------------------------
// Autotuner (qsb_set_autotune): for the H psi form of the stencil (MODE 1, whose
// output is overwritten, so a candidate can run on the caller's buffers) in
// FP64, the first launch of each shape (grid, band count rounded up to a power
// of two, real / complex, k-point terms) times the kernels that apply -- the
// TMA-box kernel with its producer warp, the TMA-plane kernel with pending
// outputs, the register-prefetch kernel -- two runs each after a warm one, on
// the caller's stream with CUDA events, keeps the fastest for that shape, and
// runs it once more so the output is its own.  Decisions are logged
// (qsb_autotune_report).  FP32 keeps the register-prefetch kernel (its summation
// order), MODE 0 ("+=") the default order of kernels.
struct TuneState {
    std::mutex mu;
    bool on = false;
    std::map<std::array<int, 8>, int> choice;
    std::string log;
};
TuneState& tune_state() {
    static TuneState t;
    return t;
}

const char* variant_name(int v) { return v == 0 ? "tma-box (fd8_ws)" : v == 3 ? "tma-plane (fd8_zacc)" : "register (fd8)"; }

qsb_status tune_and_launch(qsb_dtype dt, const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    TuneState& ts = tune_state();
    int nbb = 1;
    while (nbb < L.nb) nbb *= 2;
    const std::array<int, 8> key{L.nx, L.ny, L.nz, nbb, L.is_complex, c.has_grad ? 1 : 0, (int)dt, L.mode};
    {
        std::lock_guard<std::mutex> g(ts.mu);
        auto it = ts.choice.find(key);
        if (it != ts.choice.end()) return launch_dtype<double>(L, c, s, it->second);
    }
    const int cand[3] = {0, 3, 2};
    float best = 1e30f;
    int pick = 0;
    std::string line = "stencil " + std::to_string(L.nx) + "x" + std::to_string(L.ny) + "x" + std::to_string(L.nz) +
                       (L.is_complex ? " complex" : " real") + " x" + std::to_string(L.nb) + " bands:";
    cudaEvent_t e0, e1;
    QSB_CUDA_TRY(cudaEventCreate(&e0));
    QSB_CUDA_TRY(cudaEventCreate(&e1));
    for (int v : cand) {
        qsb_status st = launch_dtype<double>(L, c, s, v);   // warm
        float ms = 0.f;
        if (st == QSB_OK) {
            cudaEventRecord(e0, s);
            for (int r = 0; r < 2; ++r) st = st == QSB_OK ? launch_dtype<double>(L, c, s, v) : st;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            ms *= 0.5f;
        }
        if (st != QSB_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return st;
        }
        line += std::string(" ") + variant_name(v) + " " + std::to_string(ms) + " ms;";
        if (ms < best) {
            best = ms;
            pick = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    line += std::string(" -> ") + variant_name(pick) + "\n";
    {
        std::lock_guard<std::mutex> g(ts.mu);
        ts.choice[key] = pick;
        ts.log += line;
    }
    return launch_dtype<double>(L, c, s, pick);
}

}  // namespace

qsb_status launch_stencil(qsb_dtype dt, const StencilLaunch& L, const FD8Coef& c, cudaStream_t s) {
    if (L.nb > 65535) return fail(QSB_ERR_INVALID, "stencil: nb > 65535");
    const int forced = stencil_variant();   // QSB_STENCIL overrides the choice
    if (dt == QSB_F64 && L.mode == 1 && forced == 0 && tune_state().on) return tune_and_launch(dt, L, c, s);
    if (dt == QSB_F64) return launch_dtype<double>(L, c, s, forced);
    return launch_dtype<float>(L, c, s, forced);
}

template <typename T>
qsb_status stencil_batch_t(int n, const BatchSysDesc* d, cudaStream_t s) {
    constexpr int TY = BY * batch_ry<T>();
    constexpr int ZC = 32;   // planes per item
    std::vector<BatchSys<T>> hs(n);
    std::vector<BatchItem> items;
    std::vector<std::pair<long long, int>> order;
    for (int i = 0; i < n; ++i) {
        hs[i] = BatchSys<T>{(const T*)d[i].in, (T*)d[i].out, (const T*)d[i].V, d[i].nx, d[i].ny, d[i].nz,
                            to_kc<T>(d[i].coef)};
        order.push_back({(long long)d[i].nx * d[i].ny * d[i].nz * d[i].nb, i});
    }
    // largest systems first, so the smallest fill the tail
    std::sort(order.begin(), order.end(), [](const std::pair<long long, int>& a, const std::pair<long long, int>& b) {
        return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    for (const auto& o : order) {
        const BatchSysDesc& q = d[o.second];
        for (int b = 0; b < q.nb; ++b)
            for (int z0 = 0; z0 < q.nz; z0 += ZC)
                for (int y0 = 0; y0 < q.ny; y0 += TY)
                    for (int x0 = 0; x0 < q.nx; x0 += TX)
                        items.push_back(BatchItem{o.second, x0, y0, z0, std::min(q.nz, z0 + ZC), b});
    }
    if (items.empty()) return QSB_OK;
    if (items.size() > (size_t)0x7fffffff) return fail(QSB_ERR_INVALID, "stencil batch: too many work items");
    const size_t sys_bytes = hs.size() * sizeof(BatchSys<T>);
    const size_t off = (sys_bytes + 255) / 256 * 256;
    void* dmem = nullptr;
    QSB_CUDA_TRY(cudaMallocAsync(&dmem, off + items.size() * sizeof(BatchItem), s));
    QSB_CUDA_TRY(cudaMemcpyAsync(dmem, hs.data(), sys_bytes, cudaMemcpyHostToDevice, s));
    QSB_CUDA_TRY(cudaMemcpyAsync((char*)dmem + off, items.data(), items.size() * sizeof(BatchItem),
                                 cudaMemcpyHostToDevice, s));
    const int grid = (int)std::min<size_t>(items.size(), (size_t)sm_count() * 2);
    fd8_batch_kernel<T><<<grid, dim3(TX, BY), 0, s>>>((const BatchSys<T>*)dmem, (const BatchItem*)((char*)dmem + off),
                                                      (int)items.size());
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(dmem, s);
    if (e != cudaSuccess) return cuda_fail(e, "fd8_batch_kernel");
    return QSB_OK;
}

qsb_status launch_stencil_batch(qsb_dtype dt, int n, const BatchSysDesc* d, cudaStream_t s) {
    return dt == QSB_F64 ? stencil_batch_t<double>(n, d, s) : stencil_batch_t<float>(n, d, s);
}

bool autotune_enabled() { return tune_state().on; }

void autotune_log(const std::string& line) {
    TuneState& ts = tune_state();
    std::lock_guard<std::mutex> g(ts.mu);
    ts.log += line;
}

}  // namespace qsb

extern "C" qsb_status qsb_set_autotune(int enable) {
    qsb::TuneState& ts = qsb::tune_state();
    std::lock_guard<std::mutex> g(ts.mu);
    ts.on = enable != 0;
    return QSB_OK;
}

extern "C" qsb_status qsb_autotune_report(char* buf, int len, int* needed) {
    qsb::TuneState& ts = qsb::tune_state();
    std::lock_guard<std::mutex> g(ts.mu);
    if (needed) *needed = (int)ts.log.size() + 1;
    if (buf && len > 0) {
        const size_t n = std::min<size_t>((size_t)len - 1, ts.log.size());
        std::memcpy(buf, ts.log.data(), n);
        buf[n] = '\0';
    }
    return QSB_OK;
}

namespace qsb {

}  // namespace qsb
