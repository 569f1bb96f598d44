// Nonlocal Kleinman-Bylander projector apply for sm_100a.
//
//   Hpsi_c += sum_a sum_w |beta_aw> E_w dV <beta_aw | psi_c>
//
// The order of operations is the reference's ProjectionPP_bundle_1 /
// mInnerNonlocalPsi_v4_bundle (source/PseudoPotNonlocal_SvF2_kpoint.h:3911-4046,
// :4463-4576): gather psi on each atom's points, multiply by exp(+i k.r) (k != 0),
// contract with the projector table (DGEMM_t, times dV), scale by E_w, expand
// (DGEMM_n), multiply by exp(-i k.r), scatter-add.
//
// B200 layout: the projector points are held twice.
//  * atom-major ("gather") order, cut into chunks of one atom's points, for the
//    projection.  Each CTA reduces one chunk for a group of bands in registers
//    and shared memory and writes one partial sum per (chunk, w, column); a
//    second tiny kernel sums the chunks of each atom in a fixed order, so the
//    result is deterministic (no floating-point atomics).
//  * grid-ordered CSR (entries of grid point g are [grid_ptr[g], grid_ptr[g+1]))
//    for the expansion, done as a PULL: each output point sums its own entries.
//    Overlapping spheres (different atoms, or an atom and its own periodic
//    images) therefore need no atomics and no non-overlap grouping
//    (mCreateNonoverlapList, :3410-3487), and the pull can be fused into the H
//    stencil so Hpsi is written once.
#include "qsb_internal.h"
#include <cstdlib>
#include <string>

#include <cmath>
#include <algorithm>
#include <numeric>
#include <cstring>

namespace qsb {

namespace {

constexpr int PROJ_THREADS = 256;
constexpr int CHUNK = 8192;          // points per projection chunk (32 per thread: amortizes the block reduction)
constexpr int APPLY_THREADS = 256;

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

template <typename T>
qsb_status dupload(T*& dst, const T* src, size_t n) {
    dfree(dst);
    if (n == 0) return QSB_OK;
    cudaError_t e = cudaMalloc((void**)&dst, n * sizeof(T));
    if (e != cudaSuccess) { dst = nullptr; return fail(QSB_ERR_NOMEM, "nonlocal tables: cudaMalloc failed"); }
    QSB_CUDA_TRY(cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return QSB_OK;
}

inline int fold(int v, int n) {
    int m = v % n;
    return m < 0 ? m + n : m;
}

// ---------------------------------------------------------------------------
// projection: partial[chunk][w][col] = sum_{p in chunk} beta[p][w] * phi_col[idx_p]
// phi = psi (real) or psi*exp(+i k.r) (complex; columns 2b = re, 2b+1 = im)
// ---------------------------------------------------------------------------
template <typename T, bool CPLX, int WM, int CB, int UP, int MINB>
__global__ void __launch_bounds__(PROJ_THREADS, MINB)
nl_proj_kernel(const int* __restrict__ chunk_order, const int* __restrict__ chunk_begin,
               const int* __restrict__ chunk_end, const int* __restrict__ pt_idx, const int* __restrict__ pt_xyz,
               const T* __restrict__ pt_beta, int wmax, const T* __restrict__ psi, size_t N, int nb, double gx_dx,
               double gy_dy, double gz_dz, double* __restrict__ partial, int ncol) {
    constexpr int NCB = CPLX ? 2 * CB : CB;
    constexpr int NV = WM * NCB;
    // launch order: chunks of all atoms by their position along the grid, so
    // that the CTAs in flight together gather from the same region of psi and
    // the overlapping spheres of neighbouring atoms meet in L2; each CTA writes
    // the partials of its own chunk, so the sums do not depend on the order
    const int chunk = chunk_order[blockIdx.y];
    const int band0 = blockIdx.x * CB;
    const int nbl = min(CB, nb - band0);
    const int p0 = chunk_begin[chunk], p1 = chunk_end[chunk];

    double acc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = 0.0;

    // UP points per thread per pass: their index and psi loads are all issued
    // before the first use, so UP x CB (x2 complex) gathers are in flight.
    // Thread t takes the points t + 256 m in increasing m whatever UP is, so
    // the summation order does not depend on UP.
    // the grid indices of the next pass are loaded while this pass's psi
    // gathers are in flight (one dependent load latency per pass, not two)
    int idx_next[UP];
#pragma unroll
    for (int u = 0; u < UP; ++u) {
        const int p = p0 + threadIdx.x + u * PROJ_THREADS;
        idx_next[u] = p < p1 ? __ldg(pt_idx + p) : 0;
    }
    for (int pb = p0 + threadIdx.x; pb < p1; pb += PROJ_THREADS * UP) {
        int idx[UP];
        bool live[UP];
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            live[u] = pb + u * PROJ_THREADS < p1;
            idx[u] = idx_next[u];
        }
        double vals[UP][CPLX ? 2 * CB : CB];
#pragma unroll
        for (int u = 0; u < UP; ++u)
#pragma unroll
            for (int j = 0; j < CB; ++j) {
                const bool ok = live[u] && j < nbl;
                if (CPLX) {
                    const size_t base = (size_t)(2 * (band0 + j)) * N;
                    vals[u][2 * j] = ok ? (double)__ldg(psi + base + idx[u]) : 0.0;
                    vals[u][2 * j + 1] = ok ? (double)__ldg(psi + base + N + idx[u]) : 0.0;
                } else {
                    vals[u][j] = ok ? (double)__ldg(psi + (size_t)(band0 + j) * N + idx[u]) : 0.0;
                }
            }
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            const int p = pb + PROJ_THREADS * UP + u * PROJ_THREADS;
            idx_next[u] = p < p1 ? __ldg(pt_idx + p) : 0;
        }
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            if (!live[u]) continue;
            const int p = pb + u * PROJ_THREADS;
            double b[WM];
#pragma unroll
            for (int w = 0; w < WM; ++w) b[w] = (w < wmax) ? (double)__ldg(pt_beta + (size_t)p * wmax + w) : 0.0;
            double cs = 1.0, sn = 0.0;
            if (CPLX) {
                // mCreateBlochExp (source/PseudoPotNonlocal_SvF2_kpoint.h:3580-3590)
                const double kxx = gx_dx * (double)__ldg(pt_xyz + 3 * (size_t)p + 0);
                const double kyy = gy_dy * (double)__ldg(pt_xyz + 3 * (size_t)p + 1);
                const double kzz = gz_dz * (double)__ldg(pt_xyz + 3 * (size_t)p + 2);
                sincos(kxx + kyy + kzz, &sn, &cs);
            }
#pragma unroll
            for (int j = 0; j < CB; ++j) {
                if (CPLX) {
                    const double pr = vals[u][2 * j], pi = vals[u][2 * j + 1];
                    const double fr = cs * pr - sn * pi;   // :4514-4515
                    const double fi = cs * pi + sn * pr;
#pragma unroll
                    for (int w = 0; w < WM; ++w) {
                        acc[w * NCB + 2 * j] += b[w] * fr;
                        acc[w * NCB + 2 * j + 1] += b[w] * fi;
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < WM; ++w) acc[w * NCB + j] += b[w] * vals[u][j];
                }
            }
        }
    }

    __shared__ double red[PROJ_THREADS / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double v = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NV; i += PROJ_THREADS) {
        const int w = i / NCB, jc = i % NCB;
        if (w >= wmax) continue;
        const int col = (CPLX ? 2 * band0 : band0) + jc;
        if (jc >= (CPLX ? 2 * nbl : nbl)) continue;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < PROJ_THREADS / 32; ++k) s += red[k][i];
        partial[((size_t)chunk * wmax + w) * ncol + col] = s;
    }
}

// coef[a][w][col] = dV * (E_w) * sum_{chunks of a} partial
__global__ void nl_finalize_kernel(const int* __restrict__ atom_chunk_begin, const int* __restrict__ atom_chunk_end,
                                   const double* __restrict__ atom_E, const int* __restrict__ atom_width, int wmax,
                                   const double* __restrict__ partial, int ncol, double dV, int inner_only,
                                   double* __restrict__ coef) {
    const int a = blockIdx.x;
    const int c0 = atom_chunk_begin[a], c1 = atom_chunk_end[a];
    const int wa = atom_width[a];
    for (int i = threadIdx.x; i < wmax * ncol; i += blockDim.x) {
        const int w = i / ncol, col = i % ncol;
        double s = 0.0;
        if (w < wa)
            for (int ch = c0; ch < c1; ++ch) s += partial[((size_t)ch * wmax + w) * ncol + col];
        const double e = inner_only ? 1.0 : atom_E[(size_t)a * wmax + w];
        coef[((size_t)a * wmax + w) * ncol + col] = (w < wa) ? (s * dV) * e : 0.0;
    }
}

// ---------------------------------------------------------------------------
// expansion, pull form over covered grid points:
//   hpsi_col[g] += sum_{e on g} sum_w beta_e[w] * coef[atom_e][w][col]
// One thread per covered grid point loops over every band, so the point's
// entries (atom, beta, Bloch phase) are loaded once into registers and the
// band loop streams the read-modify-write of hpsi, coalesced along x.
// Entries are taken MAXE at a time (points covered by more spheres loop).
// ---------------------------------------------------------------------------
template <typename T, bool CPLX, int WM>
__global__ void __launch_bounds__(APPLY_THREADS, 2)
nl_apply_kernel(const int* __restrict__ cov_grid, int n_cov, const int* __restrict__ grid_ptr,
                const int* __restrict__ ent_atom, const int* __restrict__ ent_xyz, const T* __restrict__ ent_beta,
                int wmax, const double* __restrict__ coef, int ncol, T* __restrict__ hpsi, size_t N, int nb,
                double gx_dx, double gy_dy, double gz_dz) {
    // entries held in registers at a time
    constexpr int MAXE = CPLX ? (WM <= 4 ? 2 : 1) : (WM <= 4 ? 4 : (WM <= 9 ? 2 : 1));
    constexpr int BG = CPLX ? 4 : 8;   // bands per group
    constexpr int CG = 8;              // coefficient columns per group: BG real, 2 BG complex
    const int r = blockIdx.x * APPLY_THREADS + threadIdx.x;
    if (r >= n_cov) return;
    const int g = __ldg(cov_grid + r);
    const int e0 = __ldg(grid_ptr + g), e1 = __ldg(grid_ptr + g + 1);
    // coefficient rows are read 8 columns at a time as four 16-byte loads
    const bool vec = (ncol % 2 == 0) && (((uintptr_t)coef) % 16 == 0);
    for (int eb = e0; eb < e1; eb += MAXE) {
        const int ne = min(MAXE, e1 - eb);
        const double* cf[MAXE];
        double b[MAXE][WM];
        double cs[MAXE], sn[MAXE];
#pragma unroll
        for (int q = 0; q < MAXE; ++q) {
            const int e = eb + min(q, ne - 1);
            cf[q] = coef + (size_t)__ldg(ent_atom + e) * wmax * ncol;
#pragma unroll
            for (int w = 0; w < WM; ++w)
                b[q][w] = (q < ne && w < wmax) ? (double)__ldg(ent_beta + (size_t)e * wmax + w) : 0.0;
            cs[q] = 1.0;
            sn[q] = 0.0;
            if (CPLX) {
                const double kxx = gx_dx * (double)__ldg(ent_xyz + 3 * (size_t)e + 0);
                const double kyy = gy_dy * (double)__ldg(ent_xyz + 3 * (size_t)e + 1);
                const double kzz = gz_dz * (double)__ldg(ent_xyz + 3 * (size_t)e + 2);
                sincos(kxx + kyy + kzz, &sn[q], &cs[q]);
            }
        }
        for (int b0 = 0; b0 < nb; b0 += BG) {
            const int c0 = CPLX ? 2 * b0 : b0;
            const bool full = vec && (b0 + BG <= nb);
            // hpsi of the group first: CG independent loads in flight
            T cur[CG];
#pragma unroll
            for (int k = 0; k < CG; ++k) {
                const int col = c0 + k;
                cur[k] = (col < ncol) ? hpsi[(size_t)col * N + g] : T(0);
            }
            double acc[CG];
#pragma unroll
            for (int k = 0; k < CG; ++k) acc[k] = 0.0;
#pragma unroll
            for (int q = 0; q < MAXE; ++q) {
                if (q < ne) {
                    double tq[CG];
#pragma unroll
                    for (int k = 0; k < CG; ++k) tq[k] = 0.0;
#pragma unroll
                    for (int w = 0; w < WM; ++w) {
                        if (w < wmax) {
                            const double* row = cf[q] + (size_t)w * ncol + c0;
                            double c[CG];
                            if (full) {
#pragma unroll
                                for (int k = 0; k < CG; k += 2) {
                                    const double2 v = __ldg(reinterpret_cast<const double2*>(row + k));
                                    c[k] = v.x;
                                    c[k + 1] = v.y;
                                }
                            } else {
#pragma unroll
                                for (int k = 0; k < CG; ++k) c[k] = (c0 + k < ncol) ? __ldg(row + k) : 0.0;
                            }
#pragma unroll
                            for (int k = 0; k < CG; ++k) tq[k] += b[q][w] * c[k];
                        }
                    }
                    if (CPLX) {
                        // exp(-i k.r) (source/PseudoPotNonlocal_SvF2_kpoint.h:4026-4027)
#pragma unroll
                        for (int j = 0; j < BG; ++j) {
                            acc[2 * j] += cs[q] * tq[2 * j] + sn[q] * tq[2 * j + 1];
                            acc[2 * j + 1] += cs[q] * tq[2 * j + 1] - sn[q] * tq[2 * j];
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < CG; ++k) acc[k] += tq[k];
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < CG; ++k) {
                const int col = c0 + k;
                if (col < ncol) hpsi[(size_t)col * N + g] = cur[k] + (T)acc[k];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// expansion, v2: the pull of nl_apply_kernel with the coefficient rows of every
// atom staged in shared memory one APPLY_CW-column slice at a time (threads
// whose points share an atom read them as broadcasts instead of per-point L1
// loads), up to MAXE entries of the point held in registers across all slices,
// and SG columns of hpsi loaded before use.
// ---------------------------------------------------------------------------
constexpr int APPLY_CW = 32;

template <typename T, bool CPLX, int WM>
__global__ void __launch_bounds__(APPLY_THREADS, 2)
nl_apply2_kernel(const int* __restrict__ cov_grid, int n_cov, const int* __restrict__ grid_ptr,
                 const int* __restrict__ ent_atom, const int* __restrict__ ent_xyz, const T* __restrict__ ent_beta,
                 int wmax, int n_atoms, const double* __restrict__ coef, int ncol, T* __restrict__ hpsi, size_t N,
                 double gx_dx, double gy_dy, double gz_dz) {
    extern __shared__ double csm[];                          // [atom][w][APPLY_CW]
    constexpr int MAXE = CPLX ? 2 : (WM <= 4 ? 3 : 1);       // entries kept in registers
    constexpr int SG = CPLX ? 8 : 16;                        // columns per pass
    const int r = blockIdx.x * APPLY_THREADS + threadIdx.x;
    const bool active = r < n_cov;
    int g = 0, e0 = 0, e1 = 0;
    if (active) {
        g = __ldg(cov_grid + r);
        e0 = __ldg(grid_ptr + g);
        e1 = __ldg(grid_ptr + g + 1);
    }
    const int ne = min(MAXE, e1 - e0);
    double b[MAXE][WM];
    int ao[MAXE];
    double cs[MAXE], sn[MAXE];
    auto load_entry = [&](int e, double* bq, int& aq, double& cq, double& sq) {
        aq = __ldg(ent_atom + e) * wmax * APPLY_CW;
#pragma unroll
        for (int w = 0; w < WM; ++w) bq[w] = w < wmax ? (double)__ldg(ent_beta + (size_t)e * wmax + w) : 0.0;
        cq = 1.0;
        sq = 0.0;
        if (CPLX) {
            const double kxx = gx_dx * (double)__ldg(ent_xyz + 3 * (size_t)e + 0);
            const double kyy = gy_dy * (double)__ldg(ent_xyz + 3 * (size_t)e + 1);
            const double kzz = gz_dz * (double)__ldg(ent_xyz + 3 * (size_t)e + 2);
            sincos(kxx + kyy + kzz, &sq, &cq);
        }
    };
#pragma unroll
    for (int q = 0; q < MAXE; ++q) {
        if (q < ne) {
            load_entry(e0 + q, b[q], ao[q], cs[q], sn[q]);
        } else {
#pragma unroll
            for (int w = 0; w < WM; ++w) b[q][w] = 0.0;
            ao[q] = 0;
            cs[q] = 1.0;
            sn[q] = 0.0;
        }
    }
    // adds entry (bq, aq, phase) times the staged slice to acc[SG]
    auto contract = [&](const double* bq, int aq, double cq, double sq, int s0, double* acc) {
        if constexpr (!CPLX) {
            // real: no phase, accumulate in place
#pragma unroll
            for (int w = 0; w < WM; ++w) {
                if (w < wmax) {
                    const double* row = csm + aq + w * APPLY_CW + s0;
#pragma unroll
                    for (int k = 0; k < SG; k += 2) {
                        const double2 v = *reinterpret_cast<const double2*>(row + k);
                        acc[k] += bq[w] * v.x;
                        acc[k + 1] += bq[w] * v.y;
                    }
                }
            }
        } else {
        double tq[SG];
#pragma unroll
        for (int k = 0; k < SG; ++k) tq[k] = 0.0;
#pragma unroll
        for (int w = 0; w < WM; ++w) {
            if (w < wmax) {
                const double* row = csm + aq + w * APPLY_CW + s0;
#pragma unroll
                for (int k = 0; k < SG; k += 2) {
                    const double2 v = *reinterpret_cast<const double2*>(row + k);
                    tq[k] += bq[w] * v.x;
                    tq[k + 1] += bq[w] * v.y;
                }
            }
        }
        {
            // exp(-i k.r) (source/PseudoPotNonlocal_SvF2_kpoint.h:4026-4027)
#pragma unroll
            for (int j = 0; j < SG / 2; ++j) {
                acc[2 * j] += cq * tq[2 * j] + sq * tq[2 * j + 1];
                acc[2 * j + 1] += cq * tq[2 * j + 1] - sq * tq[2 * j];
            }
        }
        }
    };
    const int slice = n_atoms * wmax * APPLY_CW;
    for (int c0 = 0; c0 < ncol; c0 += APPLY_CW) {
        const int cw = min(APPLY_CW, ncol - c0);
        __syncthreads();   // the previous slice is no longer read
        for (int i = threadIdx.x; i < slice; i += APPLY_THREADS) {
            const int k = i % APPLY_CW, aw = i / APPLY_CW;
            csm[i] = k < cw ? __ldg(coef + (size_t)aw * ncol + c0 + k) : 0.0;
        }
        __syncthreads();
        if (!active) continue;
        for (int s0 = 0; s0 < cw; s0 += SG) {
            T cur[SG];
#pragma unroll
            for (int k = 0; k < SG; ++k) cur[k] = s0 + k < cw ? hpsi[(size_t)(c0 + s0 + k) * N + g] : T(0);
            double acc[SG];
#pragma unroll
            for (int k = 0; k < SG; ++k) acc[k] = 0.0;
#pragma unroll
            for (int q = 0; q < MAXE; ++q)
                if (q < ne) contract(b[q], ao[q], cs[q], sn[q], s0, acc);
            // points covered by more than MAXE spheres
            for (int e = e0 + MAXE; e < e1; ++e) {
                double bx[WM], cx, sx;
                int ax;
                load_entry(e, bx, ax, cx, sx);
                contract(bx, ax, cx, sx, s0, acc);
            }
#pragma unroll
            for (int k = 0; k < SG; ++k)
                if (s0 + k < cw) hpsi[(size_t)(c0 + s0 + k) * N + g] = cur[k] + (T)acc[k];
        }
    }
}

// table: -1 projects on beta, 0..2 on the gradient tables d beta / d(x, y, z)
template <typename T, bool CPLX, int WM>
void launch_proj(const NLDevice& d, int table, int nb, const void* psi, size_t N, double gx_dx, double gy_dy,
                 double gz_dz, double* partial, int ncol, cudaStream_t s) {
    const size_t toff = table < 0 ? 0 : (size_t)table * d.n_points * d.wmax;
    const T* beta = table < 0 ? (std::is_same<T, double>::value ? (const T*)d.pt_beta64 : (const T*)d.pt_beta32)
                              : (std::is_same<T, double>::value ? (const T*)d.pt_dbeta64 + toff
                                                                : (const T*)d.pt_dbeta32 + toff);
    // up to 4 projectors: 8 real bands (4 complex) x 2 (1) points per thread
    // in at most 128 registers, two CTAs per SM (at 136 registers, one CTA:
    // 0.50 ms instead of 0.34 at the 96^3 x 128-band workload; 4 bands x 3
    // points at 80 registers and three CTAs: 0.35 ms)
    constexpr int CB = CPLX ? 4 : 8;
    constexpr int UP = (WM <= 4 && !CPLX) ? 2 : 1;
    constexpr int MINB = WM <= 4 ? 2 : 1;
    dim3 grid((nb + CB - 1) / CB, d.n_chunks);
    nl_proj_kernel<T, CPLX, WM, CB, UP, MINB><<<grid, PROJ_THREADS, 0, s>>>(d.chunk_order, d.chunk_begin, d.chunk_end,
                                                                        d.pt_idx, d.pt_xyz,
                                                                        beta, d.wmax, (const T*)psi, N, nb, gx_dx,
                                                                        gy_dy, gz_dz, partial, ncol);
}

template <typename T, bool CPLX>
void launch_proj_w(const NLDevice& d, int table, int nb, const void* psi, size_t N, double gx_dx, double gy_dy,
                   double gz_dz, double* partial, int ncol, cudaStream_t s) {
    if (d.wmax <= 1) launch_proj<T, CPLX, 1>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
    else if (d.wmax <= 4) launch_proj<T, CPLX, 4>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
    else if (d.wmax <= 9) launch_proj<T, CPLX, 9>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
    else launch_proj<T, CPLX, 16>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
}

// Per atom (one block): energy = sum over bands and projectors of occ E_w |c|^2;
// force_d = sum 2 occ E_w Re(conj(c) g_d) with c = dV <beta|psi>, g_d = dV <d beta/dd|psi>
// (coefficient arrays [atom][w][col], complex bands as columns 2b, 2b+1).
// Fixed-order block reduction: the result does not depend on timing.
__global__ void nl_energy_force_kernel(const double* __restrict__ c, const double* __restrict__ gx,
                                       const double* __restrict__ gy, const double* __restrict__ gz,
                                       const double* __restrict__ atom_E, const int* __restrict__ atom_width, int wmax,
                                       int nb, int is_complex, const double* __restrict__ occ, double* __restrict__ out) {
    const int a = blockIdx.x;
    const int wa = atom_width[a];
    const int ncol = is_complex ? 2 * nb : nb;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < wa * nb; i += blockDim.x) {
        const int w = i / nb, b = i % nb;
        const double e = atom_E[(size_t)a * wmax + w] * occ[b];
        const size_t base = ((size_t)a * wmax + w) * ncol;
        const int c0 = is_complex ? 2 * b : b;
        const double cr = c[base + c0], ci = is_complex ? c[base + c0 + 1] : 0.0;
        acc[0] += e * (cr * cr + ci * ci);
        if (gx) {
            acc[1] += 2.0 * e * (cr * gx[base + c0] + (is_complex ? ci * gx[base + c0 + 1] : 0.0));
            acc[2] += 2.0 * e * (cr * gy[base + c0] + (is_complex ? ci * gy[base + c0 + 1] : 0.0));
            acc[3] += 2.0 * e * (cr * gz[base + c0] + (is_complex ? ci * gz[base + c0 + 1] : 0.0));
        }
    }
    __shared__ double red[4][256];
#pragma unroll
    for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
#pragma unroll
            for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[(size_t)a * 4 + threadIdx.x] = red[threadIdx.x][0];
}

}  // namespace

void nl_free(NLDevice& d) {
    dfree(d.pt_idx); dfree(d.pt_xyz); dfree(d.pt_beta64); dfree(d.pt_beta32);
    dfree(d.atom_width); dfree(d.atom_proj_off); dfree(d.atom_E);
    dfree(d.chunk_atom); dfree(d.chunk_begin); dfree(d.chunk_end); dfree(d.chunk_order);
    dfree(d.atom_chunk_begin); dfree(d.atom_chunk_end);
    dfree(d.grid_ptr); dfree(d.cov_grid); dfree(d.ent_atom); dfree(d.ent_xyz);
    dfree(d.ent_beta64); dfree(d.ent_beta32);
    dfree(d.pt_dbeta64); dfree(d.pt_dbeta32);
    d.n_atoms = 0; d.wmax = 0; d.n_points = 0; d.total_proj = 0; d.n_chunks = 0; d.n_cov = 0;
    d.h_atom_width.clear(); d.h_atom_proj_off.clear(); d.h_npts.clear(); d.h_src.clear();
}

qsb_status nl_upload(NLDevice& d, int nx, int ny, int nz, int n_atoms, const int* npts, const int* widths,
                     const int* coords, const double* beta, const double* energy) {
    nl_free(d);
    if (n_atoms < 0) return fail(QSB_ERR_INVALID, "set_projectors: n_atoms < 0");
    const size_t N = (size_t)nx * ny * nz;
    int64_t total = 0;
    int wmax = 0, total_proj = 0;
    for (int a = 0; a < n_atoms; ++a) {
        if (npts[a] < 0 || widths[a] < 0) return fail(QSB_ERR_INVALID, "set_projectors: negative npts/width");
        if (widths[a] > 16) return fail(QSB_ERR_INVALID, "set_projectors: width > 16 per atom is not supported");
        total += npts[a];
        wmax = std::max(wmax, widths[a]);
        total_proj += widths[a];
    }
    if (total >= (int64_t)1 << 31) return fail(QSB_ERR_INVALID, "set_projectors: more than 2^31 points");
    d.n_atoms = n_atoms;
    d.wmax = wmax;
    d.n_points = total;
    d.total_proj = total_proj;
    d.h_atom_width.assign(widths, widths + n_atoms);
    d.h_npts.assign(npts, npts + n_atoms);
    d.h_atom_proj_off.resize(n_atoms);
    {
        int off = 0;
        for (int a = 0; a < n_atoms; ++a) { d.h_atom_proj_off[a] = off; off += widths[a]; }
    }
    if (total == 0 || wmax == 0) {
        // nothing to apply; keep an empty CSR so the fused stencil can skip it
        d.n_points = 0;
        return QSB_OK;
    }

    // atom-major points, sorted by folded grid index within each atom
    std::vector<int> idx(total), xyz(3 * total), atom_of(total);
    d.h_src.assign(total, 0);
    std::vector<double> b64((size_t)total * wmax, 0.0);
    std::vector<double> E((size_t)n_atoms * wmax, 0.0);
    std::vector<int> chunk_atom, chunk_b, chunk_e, acb(n_atoms), ace(n_atoms);
    {
        int64_t off = 0, boff = 0;
        std::vector<int> order;
        for (int a = 0; a < n_atoms; ++a) {
            const int np = npts[a], w = widths[a];
            for (int k = 0; k < w; ++k) E[(size_t)a * wmax + k] = energy[d.h_atom_proj_off[a] + k];
            order.resize(np);
            std::vector<int> fidx(np);
            for (int i = 0; i < np; ++i) {
                const int* c = coords + 3 * (off + i);
                fidx[i] = fold(c[0], nx) + nx * (fold(c[1], ny) + ny * fold(c[2], nz));
            }
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return fidx[u] < fidx[v]; });
            for (int i = 0; i < np; ++i) {
                const int src = order[i];
                const int64_t dst = off + i;
                idx[dst] = fidx[src];
                atom_of[dst] = a;
                d.h_src[dst] = src;
                for (int c = 0; c < 3; ++c) xyz[3 * dst + c] = coords[3 * (off + src) + c];
                for (int k = 0; k < w; ++k) b64[(size_t)dst * wmax + k] = beta[boff + (int64_t)k * np + src];
            }
            acb[a] = (int)chunk_b.size();
            if (w > 0)
                for (int i = 0; i < np; i += CHUNK) {
                    chunk_atom.push_back(a);
                    chunk_b.push_back((int)(off + i));
                    chunk_e.push_back((int)(off + std::min(np, i + CHUNK)));
                }
            ace[a] = (int)chunk_b.size();
            off += np;
            boff += (int64_t)np * w;
        }
    }
    d.n_chunks = (int)chunk_b.size();
    // launch order of the projection: by the grid index of each chunk's middle point
    std::vector<int> corder(d.n_chunks);
    std::iota(corder.begin(), corder.end(), 0);
    {
        std::vector<int> mid(d.n_chunks);
        for (int c = 0; c < d.n_chunks; ++c) mid[c] = idx[(chunk_b[c] + chunk_e[c] - 1) / 2];
        std::stable_sort(corder.begin(), corder.end(), [&](int u, int v) { return mid[u] < mid[v]; });
    }

    // grid-ordered CSR (counting sort by folded index, stable in atom-major order)
    std::vector<int> gptr(N + 1, 0);
    for (int64_t p = 0; p < total; ++p) gptr[idx[p] + 1]++;
    for (size_t g = 0; g < N; ++g) gptr[g + 1] += gptr[g];
    std::vector<int> fillp(gptr.begin(), gptr.end() - 1);
    std::vector<int> e_atom(total), e_xyz(3 * total);
    std::vector<double> e_b64((size_t)total * wmax);
    for (int64_t p = 0; p < total; ++p) {
        const int e = fillp[idx[p]]++;
        e_atom[e] = atom_of[p];
        for (int c = 0; c < 3; ++c) e_xyz[3 * e + c] = xyz[3 * p + c];
        for (int k = 0; k < wmax; ++k) e_b64[(size_t)e * wmax + k] = b64[(size_t)p * wmax + k];
    }
    std::vector<int> cov;
    for (size_t g = 0; g < N; ++g)
        if (gptr[g + 1] > gptr[g]) cov.push_back((int)g);
    d.n_cov = (int)cov.size();

    std::vector<float> b32(b64.begin(), b64.end()), e_b32(e_b64.begin(), e_b64.end());
    QSB_TRY(dupload(d.pt_idx, idx.data(), idx.size()));
    QSB_TRY(dupload(d.pt_xyz, xyz.data(), xyz.size()));
    QSB_TRY(dupload(d.pt_beta64, b64.data(), b64.size()));
    QSB_TRY(dupload(d.pt_beta32, b32.data(), b32.size()));
    QSB_TRY(dupload(d.atom_width, widths, (size_t)n_atoms));
    QSB_TRY(dupload(d.atom_proj_off, d.h_atom_proj_off.data(), (size_t)n_atoms));
    QSB_TRY(dupload(d.atom_E, E.data(), E.size()));
    QSB_TRY(dupload(d.chunk_atom, chunk_atom.data(), chunk_atom.size()));
    QSB_TRY(dupload(d.chunk_order, corder.data(), corder.size()));
    QSB_TRY(dupload(d.chunk_begin, chunk_b.data(), chunk_b.size()));
    QSB_TRY(dupload(d.chunk_end, chunk_e.data(), chunk_e.size()));
    QSB_TRY(dupload(d.atom_chunk_begin, acb.data(), acb.size()));
    QSB_TRY(dupload(d.atom_chunk_end, ace.data(), ace.size()));
    QSB_TRY(dupload(d.grid_ptr, gptr.data(), gptr.size()));
    QSB_TRY(dupload(d.cov_grid, cov.data(), cov.size()));
    QSB_TRY(dupload(d.ent_atom, e_atom.data(), e_atom.size()));
    QSB_TRY(dupload(d.ent_xyz, e_xyz.data(), e_xyz.size()));
    QSB_TRY(dupload(d.ent_beta64, e_b64.data(), e_b64.size()));
    QSB_TRY(dupload(d.ent_beta32, e_b32.data(), e_b32.size()));
    return QSB_OK;
}

size_t nl_workspace_bytes(const NLDevice& d, int ncol) {
    if (d.n_points == 0) return 0;
    const size_t part = (size_t)d.n_chunks * d.wmax * ncol * sizeof(double);
    const size_t coef = (size_t)d.n_atoms * d.wmax * ncol * sizeof(double);
    return ((part + 255) / 256) * 256 + ((coef + 255) / 256) * 256;
}

namespace {
qsb_status nl_project_table(qsb_dtype dt, const NLDevice& d, int table, int nx, int ny, int nz, int nb,
                            int is_complex, const void* psi, double dV, double gx_dx, double gy_dy, double gz_dz,
                            bool inner_only, void* ws, double** coef_out, cudaStream_t s) {
    const size_t N = (size_t)nx * ny * nz;
    const int ncol = is_complex ? 2 * nb : nb;
    const size_t part = (size_t)d.n_chunks * d.wmax * ncol * sizeof(double);
    double* partial = (double*)ws;
    double* coef = (double*)((char*)ws + ((part + 255) / 256) * 256);
    *coef_out = coef;
    if (d.n_points == 0) return QSB_OK;
    if ((nb + 7) / 8 > 65535) return fail(QSB_ERR_INVALID, "nonlocal: too many bands");
    if (dt == QSB_F64) {
        if (is_complex) launch_proj_w<double, true>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
        else launch_proj_w<double, false>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
    } else {
        if (is_complex) launch_proj_w<float, true>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
        else launch_proj_w<float, false>(d, table, nb, psi, N, gx_dx, gy_dy, gz_dz, partial, ncol, s);
    }
    QSB_CUDA_TRY(cudaGetLastError());
    nl_finalize_kernel<<<d.n_atoms, 256, 0, s>>>(d.atom_chunk_begin, d.atom_chunk_end, d.atom_E, d.atom_width, d.wmax,
                                                 partial, ncol, dV, inner_only ? 1 : 0, coef);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}
}  // namespace

qsb_status nl_project(qsb_dtype dt, const NLDevice& d, int nx, int ny, int nz, int nb, int is_complex,
                      const void* psi, double dV, double gx_dx, double gy_dy, double gz_dz, bool inner_only, void* ws,
                      double** coef_out, cudaStream_t s) {
    return nl_project_table(dt, d, -1, nx, ny, nz, nb, is_complex, psi, dV, gx_dx, gy_dy, gz_dz, inner_only, ws,
                            coef_out, s);
}

qsb_status nl_upload_gradients(NLDevice& d, const double* dbeta) {
    if (d.n_points == 0 || d.wmax == 0) return QSB_OK;
    if (!dbeta) return fail(QSB_ERR_INVALID, "set_projector_gradients: null table");
    const size_t per_dir = (size_t)d.n_points * d.wmax;
    std::vector<double> g64(3 * per_dir, 0.0);
    int64_t off = 0, goff = 0;
    for (int a = 0; a < d.n_atoms; ++a) {
        const int np = d.h_npts[a], w = d.h_atom_width[a];
        for (int i = 0; i < np; ++i) {
            const int64_t dst = off + i;
            const int src = d.h_src[dst];
            for (int dir = 0; dir < 3; ++dir)
                for (int k = 0; k < w; ++k)
                    g64[dir * per_dir + (size_t)dst * d.wmax + k] =
                        dbeta[goff + (int64_t)dir * np * w + (int64_t)k * np + src];
        }
        off += np;
        goff += (int64_t)3 * np * w;
    }
    std::vector<float> g32(g64.begin(), g64.end());
    dfree(d.pt_dbeta64);
    dfree(d.pt_dbeta32);
    QSB_CUDA_TRY(cudaMalloc((void**)&d.pt_dbeta64, g64.size() * sizeof(double)));
    QSB_CUDA_TRY(cudaMalloc((void**)&d.pt_dbeta32, g32.size() * sizeof(float)));
    QSB_CUDA_TRY(cudaMemcpy(d.pt_dbeta64, g64.data(), g64.size() * sizeof(double), cudaMemcpyHostToDevice));
    QSB_CUDA_TRY(cudaMemcpy(d.pt_dbeta32, g32.data(), g32.size() * sizeof(float), cudaMemcpyHostToDevice));
    return QSB_OK;
}

size_t nl_energy_force_bytes(const NLDevice& d, int ncol, int nb) {
    const size_t one = nl_workspace_bytes(d, ncol);
    return 4 * one + (((size_t)d.n_atoms * 4 + nb) * sizeof(double) + 256);
}

qsb_status nl_energy_force(qsb_dtype dt, const NLDevice& d, int nx, int ny, int nz, int nb, int is_complex,
                           const void* psi, const double* occ_host, double dV, double gx_dx, double gy_dy,
                           double gz_dz, double* energy, double* forces, void* ws, cudaStream_t s) {
    *energy = 0.0;
    if (d.n_points == 0 || nb == 0) return QSB_OK;
    if (forces && !d.pt_dbeta64) return fail(QSB_ERR_STATE, "nonlocal forces: no projector gradients set");
    const int ncol = is_complex ? 2 * nb : nb;
    const size_t one = nl_workspace_bytes(d, ncol);
    unsigned char* w = (unsigned char*)ws;
    double* coef[4] = {nullptr, nullptr, nullptr, nullptr};
    const int ntab = forces ? 4 : 1;
    for (int t = 0; t < ntab; ++t)
        QSB_TRY(nl_project_table(dt, d, t - 1, nx, ny, nz, nb, is_complex, psi, dV, gx_dx, gy_dy, gz_dz, true,
                                 w + t * one, &coef[t], s));
    double* out = (double*)(w + 4 * one);
    double* occ = out + (size_t)d.n_atoms * 4;
    QSB_CUDA_TRY(cudaMemcpyAsync(occ, occ_host, sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    nl_energy_force_kernel<<<d.n_atoms, 256, 0, s>>>(coef[0], coef[1], coef[2], coef[3], d.atom_E, d.atom_width,
                                                     d.wmax, nb, is_complex, occ, out);
    QSB_CUDA_TRY(cudaGetLastError());
    std::vector<double> h((size_t)d.n_atoms * 4);
    QSB_CUDA_TRY(cudaMemcpyAsync(h.data(), out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    double e = 0.0;
    for (int a = 0; a < d.n_atoms; ++a) {
        e += h[(size_t)a * 4];
        if (forces)
            for (int k = 0; k < 3; ++k) forces[3 * a + k] += h[(size_t)a * 4 + 1 + k];
    }
    if (!std::isfinite(e)) return fail(QSB_ERR_NUMERIC, "nonlocal energy: non-finite value");
    *energy = e;
    return QSB_OK;
}

qsb_status nl_apply(qsb_dtype dt, const NLDevice& d, int N, int nb, int is_complex, void* hpsi, const double* coef,
                    double gx_dx, double gy_dy, double gz_dz, cudaStream_t s) {
    if (d.n_points == 0 || d.n_cov == 0) return QSB_OK;
    const int ncol = is_complex ? 2 * nb : nb;
    const dim3 grid((d.n_cov + APPLY_THREADS - 1) / APPLY_THREADS);
    // v2 (coefficients staged in shared memory) while one slice of every atom's
    // rows fits; QSB_NLAPPLY=v1 keeps the L1 form for A/B timing
    static const bool force_v1 = [] {
        const char* e = std::getenv("QSB_NLAPPLY");
        return e && std::string(e) == "v1";
    }();
    const size_t smem2 = (size_t)d.n_atoms * d.wmax * APPLY_CW * sizeof(double);
    const bool v2 = !force_v1 && smem2 <= 96 * 1024;
#define QSB_APPLY(T, C, W, B)                                                                                        \
    do {                                                                                                             \
        if (v2) {                                                                                                    \
            cudaFuncSetAttribute(nl_apply2_kernel<T, C, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2); \
            nl_apply2_kernel<T, C, W><<<grid, APPLY_THREADS, smem2, s>>>(d.cov_grid, d.n_cov, d.grid_ptr, d.ent_atom, \
                                                                         d.ent_xyz, B, d.wmax, d.n_atoms, coef, ncol, \
                                                                         (T*)hpsi, (size_t)N, gx_dx, gy_dy, gz_dz);   \
        } else {                                                                                                     \
            nl_apply_kernel<T, C, W><<<grid, APPLY_THREADS, 0, s>>>(d.cov_grid, d.n_cov, d.grid_ptr, d.ent_atom,      \
                                                                    d.ent_xyz, B, d.wmax, coef, ncol, (T*)hpsi,      \
                                                                    (size_t)N, nb, gx_dx, gy_dy, gz_dz);            \
        }                                                                                                            \
    } while (0)
#define QSB_APPLY_W(T, C, B)                      \
    do {                                          \
        if (d.wmax <= 1) QSB_APPLY(T, C, 1, B);   \
        else if (d.wmax <= 4) QSB_APPLY(T, C, 4, B); \
        else if (d.wmax <= 9) QSB_APPLY(T, C, 9, B); \
        else QSB_APPLY(T, C, 16, B);              \
    } while (0)
    if (dt == QSB_F64) {
        if (is_complex) QSB_APPLY_W(double, true, d.ent_beta64);
        else QSB_APPLY_W(double, false, d.ent_beta64);
    } else {
        if (is_complex) QSB_APPLY_W(float, true, d.ent_beta32);
        else QSB_APPLY_W(float, false, d.ent_beta32);
    }
#undef QSB_APPLY_W
#undef QSB_APPLY
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

}  // namespace qsb
