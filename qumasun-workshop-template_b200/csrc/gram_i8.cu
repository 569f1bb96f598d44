// Gram products T = U^T V on the INT8 tensor cores with exact INT32
// accumulation (tcgen05.mma kind::i8, accumulators in TMEM): the Ozaki splitting.
//
// Why not BF16 with FP32 accumulation: the FP32 accumulator of the tensor core
// rounds toward zero, so a same-sign sum (every diagonal entry u.u of an
// overlap matrix) loses about 4e-8 of itself per MMA chained into one
// accumulator; at the K ranges of a Gram over 10^5..10^6 grid points that is a
// systematic 1e-5..1e-4 relative shortfall, which shifts every eigenvalue of
// the overlap matrix down and breaks the LOBPCG Rayleigh-Ritz step near
// convergence.  Integer accumulation has no rounding at all.
//
// Splitting: column c of U gets a power-of-two scale 2^e_c with
// max_i |u_ic| 2^-e_c in [32, 64), and three int8 slices
//   x = u 2^-e = s0 + s1 2^-7 + s2 2^-14 + r,  |r| <= 2^-15,  |s_k| <= 64
// (each slice the round-to-nearest of the remainder, so r has no sign bias).
//   U^T V = 2^(e_u + e_v) sum_l 2^(-7 l) D_l,  D_l = sum_{i+j=l} S_i^T T_j,  l = 0, 1, 2
// Six MMAs per K step (s0t0 | s0t1 + s1t0 | s0t2 + s1t1 + s2t0) into three INT32
// accumulators; the omitted levels (i+j >= 3) are below 2^-21 of the scaled
// products, random-signed except s2.s2 (2^-28).  |D_l| <= 3 * 64 * 64 * K <
// 2^31 for K <= 131072 elements per CTA, which the K split guarantees.
//
// Pipeline per CTA (128 threads, one CTA per SM): warp 0 allocates 512 TMEM
// columns (three 128-column accumulators) and its lane 0 streams 128-wide K
// stages of the six slice tiles with 2-D TMA copies (128B swizzle) into a
// 2-stage ring; warp 1 lane 0 issues 24 MMAs per stage and frees the stage
// with tcgen05.commit; the four warps then combine the three accumulators into
// FP64 partial tiles.  A second kernel sums the K-split partials in fixed order
// and applies the column scales.  All waits are bounded; a wait that runs out
// sets the device error word and the CTA drains, frees TMEM and returns.
#include "qsb_internal.h"
#include "tc_common.cuh"

#include <algorithm>

namespace qsb {
namespace {
using namespace tc;

constexpr int OZ_M = 128, OZ_N = 128;
constexpr int OZ_K = 128;                      // int8 K elements per stage (one 128-byte swizzle row)
constexpr int OZ_SLICES = 3;
constexpr int OZ_STAGES = 2;
constexpr int OZ_THREADS = 128;
constexpr int OZ_TILE = OZ_M * OZ_K;           // 16 KB per slice tile (A and B tiles have 128 rows)
constexpr int OZ_STAGE_BYTES = 2 * OZ_SLICES * OZ_TILE;
constexpr size_t OZ_SMEM = (size_t)OZ_STAGES * OZ_STAGE_BYTES + 1024 + 256;
constexpr int OZ_MAX_STAGES_PER_CTA = 131072 / OZ_K;
constexpr unsigned OZ_WAIT_LIMIT = 1u << 22;
constexpr unsigned OZ_DRAIN_LIMIT = 1u << 16;
constexpr int ERR_GEMM_TIMEOUT = 2;

// kind::i8: signed 8-bit A and B, signed 32-bit D, both K-major, M = N = 128
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_N >> 3) << 17) |
                              ((uint32_t)(OZ_M >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(OZ_IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ int column_of(const ColumnSet& src, int col, const void** base) {
    int local = col;
    const void* b = src.base[0];
    bool found = false;
#pragma unroll
    for (int k = 0; k < kMaxSegments; ++k) {
        if (!found) {
            if (k + 1 >= src.nseg || local < src.cols[k]) {
                b = src.base[k];
                found = true;
            } else {
                local -= src.cols[k];
            }
        }
    }
    *base = b;
    return local;
}

// Four consecutive elements of a column (zero past N); one 16-byte (fp32) or
// two 16-byte (fp64) loads when the column start is 16-byte aligned.
template <typename T>
__device__ __forceinline__ void load4(const T* __restrict__ s, int64_t i, int64_t N, bool vec, double (&v)[4]) {
    if (vec && i + 3 < N) {
        if constexpr (sizeof(T) == 4) {
            const float4 f = __ldg(reinterpret_cast<const float4*>(s + i));
            v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
        } else {
            const double2 a = __ldg(reinterpret_cast<const double2*>(s + i));
            const double2 b = __ldg(reinterpret_cast<const double2*>(s + i + 2));
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = (i + j < N) ? (double)s[i + j] : 0.0;
    }
}

// maxbits[col] = bits of max_i |u_i,col| (non-negative doubles order like their bits)
template <typename T>
__global__ void column_absmax_kernel(ColumnSet src, int64_t N, unsigned long long* __restrict__ maxbits) {
    const void* b;
    const int local = column_of(src, blockIdx.y, &b);
    const T* s = static_cast<const T*>(b) + (size_t)local * N;
    const bool vec = ((uintptr_t)s % 16) == 0;
    double m = 0.0;
    const int64_t n4 = (N + 3) / 4;
    // unrolled so that several 16-byte loads per thread are in flight
#pragma unroll 4
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (int64_t)gridDim.x * blockDim.x) {
        double v[4];
        load4<T>(s, 4 * q, N, vec, v);
        m = fmax(m, fmax(fmax(fabs(v[0]), fabs(v[1])), fmax(fabs(v[2]), fabs(v[3]))));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        atomicMax(&maxbits[blockIdx.y], (unsigned long long)__double_as_longlong(m));
    }
}

__device__ __forceinline__ int column_exponent(unsigned long long bits) {
    const double m = __longlong_as_double((long long)bits);
    return m > 0.0 ? ilogb(m) - 5 : 0;   // max |u| 2^-e in [32, 64)
}

// Four int8 slices of column col (length ldk, a multiple of 4; rows N..ldk
// zero) and its exponent; four elements per thread, one 4-byte store per slice.
// The Gram products use the first three, the rotations all four.
template <typename T>
__global__ void slice_kernel(ColumnSet src, int64_t N, int64_t ldk, const unsigned long long* __restrict__ maxbits,
                             int8_t* __restrict__ slices, size_t slice_stride, int* __restrict__ exps) {
    const int col = blockIdx.y;
    const void* b;
    const int local = column_of(src, col, &b);
    const T* s = static_cast<const T*>(b) + (size_t)local * N;
    const bool vec = ((uintptr_t)s % 16) == 0;
    const int e = column_exponent(maxbits[col]);
    if (blockIdx.x == 0 && threadIdx.x == 0) exps[col] = e;
    int8_t* o0 = slices + (size_t)col * ldk;
    int8_t* o1 = o0 + slice_stride;
    int8_t* o2 = o0 + 2 * slice_stride;
    int8_t* o3 = o0 + 3 * slice_stride;
    const int64_t n4 = ldk / 4;
#pragma unroll 4
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 4 * q;
        double v[4];
        load4<T>(s, i, N, vec, v);
        char4 a, c, d, f;
        signed char* pa = &a.x;
        signed char* pc = &c.x;
        signed char* pd = &d.x;
        signed char* pf = &f.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double x = ldexp(v[j], -e);
            const double q0 = rint(x);
            const double r1 = (x - q0) * 128.0;
            const double q1 = rint(r1);
            const double r2 = (r1 - q1) * 128.0;
            const double q2 = rint(r2);
            pa[j] = (signed char)(int)q0;
            pc[j] = (signed char)(int)q1;
            pd[j] = (signed char)(int)q2;
            pf[j] = (signed char)(int)rint((r2 - q2) * 128.0);
        }
        *reinterpret_cast<char4*>(o0 + i) = a;
        *reinterpret_cast<char4*>(o1 + i) = c;
        *reinterpret_cast<char4*>(o2 + i) = d;
        *reinterpret_cast<char4*>(o3 + i) = f;
    }
}

// Output tile of list entry t (all tiles column order, or mt <= nt only)
__device__ __forceinline__ void oz_tile_of(int t, int mtiles, bool upper, int* mt, int* nt) {
    if (upper) {
        int c = 0;
        while (t > c) {
            t -= c + 1;
            ++c;
        }
        *mt = t;
        *nt = c;
    } else {
        *mt = t % mtiles;
        *nt = t / mtiles;
    }
}
__device__ __forceinline__ int oz_tile_index(int mt, int nt, int mtiles, bool upper) {
    return upper ? nt * (nt + 1) / 2 + mt : nt * mtiles + mt;
}

// One CTA: output tile t (blockIdx.x) over K stages [kb0, kb1) of split blockIdx.y;
// the FP64 tile D0 + D1 2^-7 + D2 2^-14 goes to partial[((split*ntl + t)*128 + row)*128 + col].
__global__ void __launch_bounds__(OZ_THREADS, 1)
gram_i8_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
               const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB0,
               const __grid_constant__ CUtensorMap mB1, const __grid_constant__ CUtensorMap mB2, int kstages,
               int ksplit, int mtiles, int upper, double* __restrict__ partial, int* __restrict__ err) {
    extern __shared__ unsigned char oz_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)oz_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)OZ_STAGES * OZ_STAGE_BYTES);
    uint64_t* empty = full + OZ_STAGES;
    uint64_t* done = empty + OZ_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x, ntl = gridDim.x, split = blockIdx.y;
    int mt, nt;
    oz_tile_of(t, mtiles, upper != 0, &mt, &nt);
    const int per = (kstages + ksplit - 1) / ksplit;
    const int kb0 = min(kstages, split * per), kb1 = min(kstages, kb0 + per);
    const int nk = kb1 - kb0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < OZ_STAGES; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        bar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    int issued = 0;
    if (warp == 0 && lane == 0) {
        // ---- TMA producer: six slice tiles per stage ----
        const CUtensorMap* maps[6] = {&mA0, &mA1, &mA2, &mB0, &mB1, &mB2};
        for (int it = 0; it < nk; ++it) {
            const int s = it % OZ_STAGES;
            if (it >= OZ_STAGES && !bar_wait(&empty[s], (uint32_t)(((it / OZ_STAGES) - 1) & 1), OZ_WAIT_LIMIT)) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int*)abort_flag) break;
            unsigned char* st = base + (size_t)s * OZ_STAGE_BYTES;
            const int kx = (kb0 + it) * OZ_K;
            bar_expect_tx(&full[s], OZ_STAGE_BYTES);
#pragma unroll
            for (int k = 0; k < 6; ++k) tma_2d(st + k * OZ_TILE, maps[k], kx, (k < 3 ? mt * OZ_M : nt * OZ_N), &full[s]);
            issued = it + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        const uint32_t d0 = tmem, d1 = tmem + 128, d2 = tmem + 256;
        for (int it = 0; it < nk; ++it) {
            const int s = it % OZ_STAGES;
            if (!bar_wait(&full[s], (uint32_t)((it / OZ_STAGES) & 1), OZ_WAIT_LIMIT)) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int*)abort_flag) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = su32(base + (size_t)s * OZ_STAGE_BYTES);
            const uint32_t a0 = st, a1 = st + OZ_TILE, a2 = st + 2 * OZ_TILE;
            const uint32_t b0 = st + 3 * OZ_TILE, b1 = st + 4 * OZ_TILE, b2 = st + 5 * OZ_TILE;
#pragma unroll
            for (int kk = 0; kk < OZ_K / 32; ++kk) {
                const uint32_t ko = kk * 32;   // 32 int8 = 32 bytes along the swizzled row
                const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
                umma_i8(d0, sw128_kmajor_desc(a0 + ko), sw128_kmajor_desc(b0 + ko), acc);
                umma_i8(d1, sw128_kmajor_desc(a0 + ko), sw128_kmajor_desc(b1 + ko), acc);
                umma_i8(d1, sw128_kmajor_desc(a1 + ko), sw128_kmajor_desc(b0 + ko), 1u);
                umma_i8(d2, sw128_kmajor_desc(a0 + ko), sw128_kmajor_desc(b2 + ko), acc);
                umma_i8(d2, sw128_kmajor_desc(a1 + ko), sw128_kmajor_desc(b1 + ko), 1u);
                umma_i8(d2, sw128_kmajor_desc(a2 + ko), sw128_kmajor_desc(b0 + ko), 1u);
            }
            umma_commit(&empty[s]);
        }
        umma_commit(done);
    }
    __syncwarp();

    // ---- epilogue: warp w owns TMEM lanes (rows) 32w .. 32w+31 ----
    bool ok = bar_wait(done, 0, OZ_WAIT_LIMIT);
    if (!ok) {
        atomicOr(err, ERR_GEMM_TIMEOUT);
        atomicExch(abort_flag, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = warp * 32 + lane;
    double* prow = partial + ((size_t)split * ntl + t) * (OZ_M * OZ_N) + (size_t)row * OZ_N;
    const bool have = ok && nk > 0;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
    for (int c0 = 0; c0 < OZ_N; c0 += 32) {
        uint32_t r0[32], r1[32], r2[32];
        tmem_ld32(tmem + lane_base + (uint32_t)c0, r0);
        tmem_ld32(tmem + lane_base + 128u + (uint32_t)c0, r1);
        tmem_ld32(tmem + lane_base + 256u + (uint32_t)c0, r2);
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            double2 v = make_double2(0.0, 0.0);
            if (have) {
                v.x = (double)(int)r0[j] + (double)(int)r1[j] * 0x1p-7 + (double)(int)r2[j] * 0x1p-14;
                v.y = (double)(int)r0[j + 1] + (double)(int)r1[j + 1] * 0x1p-7 + (double)(int)r2[j + 1] * 0x1p-14;
            }
            *reinterpret_cast<double2*>(prow + c0 + j) = v;
        }
    }

    // ---- teardown ----
    __syncthreads();
    if (threadIdx.x == 0 && *(volatile int*)abort_flag) {
        for (int it = max(0, issued - OZ_STAGES); it < issued; ++it)
            (void)bar_wait(&full[it % OZ_STAGES], (uint32_t)((it / OZ_STAGES) & 1), OZ_DRAIN_LIMIT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Rotation OUT = U C on the INT8 tensor cores (the NextVector products of the
// mixed-precision LOBPCG): U is an Ozaki-split operand (the Gram's slices of
// the basis, grid-contiguous columns, read as an MN-major A operand), C a
// small FP64 K x q matrix whose rows are first scaled by U's column exponents
// (so one exponent per output column remains) and split into int8 slices
// stored K-contiguous (K-major B operand).  Both enter with four slices
// (2^-27 of the column maxima, below FP32's rounding): near convergence
// P' = R Cr + P Cp is far smaller than its two terms, and P' and AP' must stay
// as consistent as FP32 arithmetic keeps them.  The ten products with
// i + j <= 3 go into four INT32 accumulators (64 output columns per CTA);
// the epilogue scales by the output column's exponent and stores FP32 planes.
// ---------------------------------------------------------------------------
constexpr int RT_K = 128;   // K per stage (rows of the MN-major A tile, bytes of the K-major B rows)
constexpr int RT_N = 64;    // output columns per CTA (UMMA N)
constexpr int RT_TILE_B = RT_N * RT_K;          // 8 KB per slice of C'
constexpr int RT_STAGE_BYTES = 4 * OZ_TILE + 4 * RT_TILE_B;   // four slices of U, four of C'
// Two stages of the ring of the persistent kernel (one CTA per SM).
constexpr int RT_STAGES = 2;
constexpr size_t RT_SMEM = (size_t)RT_STAGES * RT_STAGE_BYTES + 1024 + 256;
static_assert(RT_SMEM <= 232448, "rotation stages must fit the 227 KB of shared memory per CTA");

// kind::i8, A MN-major (bit 15), B K-major, S32 accumulate, M = 128, N = 64
constexpr uint32_t RT_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | ((uint32_t)(RT_N >> 3) << 17) |
                              ((uint32_t)(OZ_M >> 4) << 24);

__device__ __forceinline__ void umma_i8_mn(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(RT_IDESC), "r"(accumulate)
        : "memory");
}

// MN-major A tile: K rows of 128 bytes (128 int8 along M, one 128-byte swizzle
// atom wide), 8-row atoms 1024 bytes apart along K.  With a single atom along M
// only the K stride matters; it is written into both offset fields.
__device__ __forceinline__ uint64_t sw128_mnmajor_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(1024 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// C' = diag(2^e_U) C split per output column j: exponent f_j with max|C'_.j| 2^-f in
// [32, 64), four int8 slices, written [j][kpad] (rows K..kpad zero).  One block per column.
__global__ void rot_coef_split_kernel(const double* __restrict__ C, int ldc, int K, int kpad,
                                      const int* __restrict__ eu, int8_t* __restrict__ slices, size_t stride,
                                      double* __restrict__ fscale) {
    const int j = blockIdx.x;
    double m = 0.0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) m = fmax(m, fabs(ldexp(C[(size_t)k + (size_t)ldc * j], eu[k])));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double red[32];
    __shared__ int ef;
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        ef = m > 0.0 ? ilogb(m) - 5 : 0;
        fscale[j] = ldexp(1.0, ef);
    }
    __syncthreads();
    const int f = ef;
    int8_t* o0 = slices + (size_t)j * kpad;
    for (int k = threadIdx.x; k < kpad; k += blockDim.x) {
        int a = 0, b = 0, c = 0, d = 0;
        if (k < K) {
            const double x = ldexp(C[(size_t)k + (size_t)ldc * j], eu[k] - f);
            const double q0 = rint(x);
            const double r1 = (x - q0) * 128.0;
            const double q1 = rint(r1);
            const double r2 = (r1 - q1) * 128.0;
            const double q2 = rint(r2);
            a = (int)q0;
            b = (int)q1;
            c = (int)q2;
            d = (int)rint((r2 - q2) * 128.0);
        }
        o0[k] = (int8_t)a;
        o0[stride + k] = (int8_t)b;
        o0[2 * stride + k] = (int8_t)c;
        o0[3 * stride + k] = (int8_t)d;
    }
}

// Persistent rotation kernel: one CTA per SM walks the output tiles (rows
// [mt*128, +128) of OUT x columns [nt*64, +64), tile t = mt * ntn + nt, CTAs
// take t = blockIdx.x, blockIdx.x + gridDim.x, ...), all of K per tile.
// Warp 0 lane 0 streams the K stages of every tile into a 2-stage shared
// ring, warp 1 lane 0 issues the ten MMAs per 32-K step into one of two TMEM
// accumulator sets (4 x 64 columns each, 512 columns in all), and warps 2-9
// (two per TMEM lane quarter, 32 output columns each) read a finished set,
// store it and hand it back -- so the loads of the next
// stages, the MMAs of the next tile and the epilogue of the last one overlap.
// Every wait is bounded: one that runs out sets the device error word and the
// abort flag; all roles then stop, in-flight copies are drained and TMEM is
// freed.
constexpr int RT_THREADS = 320;   // producer warp, MMA warp, eight epilogue warps

__global__ void __launch_bounds__(RT_THREADS, 1)
rot_i8_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
              const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mA3,
              const __grid_constant__ CUtensorMap mB0, const __grid_constant__ CUtensorMap mB1,
              const __grid_constant__ CUtensorMap mB2, const __grid_constant__ CUtensorMap mB3, int kstages,
              int64_t N, int q, int ntn, int ntiles, const double* __restrict__ fscale, ColumnSet out,
              int* __restrict__ err) {
    extern __shared__ unsigned char rt_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)rt_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)RT_STAGES * RT_STAGE_BYTES);
    uint64_t* empty = full + RT_STAGES;
    uint64_t* tfull = empty + RT_STAGES;      // accumulator set ready for the epilogue
    uint64_t* tempty = tfull + 2;             // accumulator set read out
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = kstages;
    // tiles of this CTA: t_j = blockIdx.x + j * gridDim.x, j < my_tiles
    const int my_tiles = blockIdx.x < (unsigned)ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int st = 0; st < RT_STAGES; ++st) {
            bar_init(&full[st], 1);
            bar_init(&empty[st], 1);
        }
        for (int b = 0; b < 2; ++b) {
            bar_init(&tfull[b], 1);
            bar_init(&tempty[b], 8);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    int issued = 0;   // stages the producer issued (for the drain)
    if (warp == 0 && lane == 0) {
        // ---------------- producer ----------------
        const CUtensorMap* amaps[4] = {&mA0, &mA1, &mA2, &mA3};
        const CUtensorMap* bmaps[4] = {&mB0, &mB1, &mB2, &mB3};
        int g = 0;
        for (int j = 0; j < my_tiles && !*(volatile int*)abort_flag; ++j) {
            const int t = (int)blockIdx.x + j * (int)gridDim.x;
            const int mt = t / ntn, nt = t - mt * ntn;
            for (int it = 0; it < nk; ++it, ++g) {
                const int st = g % RT_STAGES;
                if (g >= RT_STAGES && !bar_wait(&empty[st], (uint32_t)(((g / RT_STAGES) - 1) & 1), OZ_WAIT_LIMIT)) {
                    atomicOr(err, ERR_GEMM_TIMEOUT);
                    atomicExch(abort_flag, 1);
                    break;
                }
                if (*(volatile int*)abort_flag) break;
                unsigned char* sp = base + (size_t)st * RT_STAGE_BYTES;
                bar_expect_tx(&full[st], RT_STAGE_BYTES);
                // A: box (128 grid points, 128 columns of U) at (mt*128, it*128); B: box (128 K, 64 columns of C')
#pragma unroll
                for (int k = 0; k < 4; ++k) tma_2d(sp + k * OZ_TILE, amaps[k], mt * OZ_M, it * RT_K, &full[st]);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    tma_2d(sp + 4 * OZ_TILE + k * RT_TILE_B, bmaps[k], it * RT_K, nt * RT_N, &full[st]);
                issued = g + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        int g = 0;
        for (int j = 0; j < my_tiles && !*(volatile int*)abort_flag; ++j) {
            const int ab = j & 1;
            // the epilogue must have read this accumulator set (two tiles ago)
            if (j >= 2 && !bar_wait(&tempty[ab], (uint32_t)(((j >> 1) - 1) & 1), OZ_WAIT_LIMIT)) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d0 = tmem + (uint32_t)(ab * 4 * RT_N), d1 = d0 + RT_N, d2 = d0 + 2 * RT_N,
                           d3 = d0 + 3 * RT_N;
            bool ok = true;
            for (int it = 0; it < nk; ++it, ++g) {
                const int st = g % RT_STAGES;
                if (!bar_wait(&full[st], (uint32_t)((g / RT_STAGES) & 1), OZ_WAIT_LIMIT)) {
                    atomicOr(err, ERR_GEMM_TIMEOUT);
                    atomicExch(abort_flag, 1);
                    ok = false;
                    break;
                }
                if (*(volatile int*)abort_flag) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sa = su32(base + (size_t)st * RT_STAGE_BYTES);
                uint32_t a[4], b[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    a[k] = sa + k * OZ_TILE;
                    b[k] = sa + 4 * OZ_TILE + k * RT_TILE_B;
                }
#pragma unroll
                for (int kk = 0; kk < RT_K / 32; ++kk) {
                    const uint32_t ao = kk * 4096;   // 32 K rows of 128 bytes (four 8-row atoms)
                    const uint32_t bo = kk * 32;     // 32 int8 along the K-major row
                    const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
#define RT_MMA(D, I, J, ACC) umma_i8_mn(D, sw128_mnmajor_desc(a[I] + ao), sw128_kmajor_desc(b[J] + bo), ACC)
                    RT_MMA(d0, 0, 0, acc);
                    RT_MMA(d1, 0, 1, acc);
                    RT_MMA(d1, 1, 0, 1u);
                    RT_MMA(d2, 0, 2, acc);
                    RT_MMA(d2, 1, 1, 1u);
                    RT_MMA(d2, 2, 0, 1u);
                    RT_MMA(d3, 0, 3, acc);
                    RT_MMA(d3, 1, 2, 1u);
                    RT_MMA(d3, 2, 1, 1u);
                    RT_MMA(d3, 3, 0, 1u);
#undef RT_MMA
                }
                umma_commit(&empty[st]);
            }
            if (!ok) break;
            umma_commit(&tfull[ab]);
        }
    } else if (warp >= 2) {
        // ---------------- epilogue (warps 2-9: TMEM lanes 32 (warp % 4) ..., column half (warp - 2) / 4) ----------------
        const int quarter = warp & 3;
        const int chalf = (warp - 2) >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        for (int j = 0; j < my_tiles; ++j) {
            const int ab = j & 1;
            const bool ok = bar_wait(&tfull[ab], (uint32_t)((j >> 1) & 1), OZ_WAIT_LIMIT);
            if (!ok) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
            }
            // the TMEM loads below are warp-collective: stop as one warp
            if (__any_sync(0xffffffffu, !ok || *(volatile int*)abort_flag)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int t = (int)blockIdx.x + j * (int)gridDim.x;
            const int mt = t / ntn, nt = t - mt * ntn;
            const int64_t gp = (int64_t)mt * OZ_M + quarter * 32 + lane;   // grid point of this TMEM lane
            const uint32_t dset = tmem + lane_base + (uint32_t)(ab * 4 * RT_N);
            {
                const int c0 = chalf * 32;
                uint32_t r0[32], r1[32], r2[32], r3[32];
                tmem_ld32(dset + (uint32_t)c0, r0);
                tmem_ld32(dset + (uint32_t)(RT_N + c0), r1);
                tmem_ld32(dset + (uint32_t)(2 * RT_N + c0), r2);
                tmem_ld32(dset + (uint32_t)(3 * RT_N + c0), r3);
                if (gp < N && nk > 0) {
                    const int j0 = nt * RT_N + c0;
                    // one destination lookup for the chunk when its 32 columns lie in one array
                    const void* bp;
                    const int local0 = column_of(out, j0, &bp);
                    const void* bl;
                    const int local31 = j0 + 31 < q ? column_of(out, j0 + 31, &bl) : -1;
                    const bool one = local31 == local0 + 31 && bl == bp;
                    float* dst0 = (float*)bp + (size_t)local0 * N + gp;
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        const int col = j0 + jj;
                        if (col >= q) continue;
                        float* dst;
                        if (one) {
                            dst = dst0 + (size_t)jj * N;
                        } else {
                            const void* bj;
                            const int lj = column_of(out, col, &bj);
                            dst = (float*)bj + (size_t)lj * N + gp;
                        }
                        // D0 + D1 2^-7 + D2 2^-14 + D3 2^-21 summed exactly as an integer in units of
                        // 2^-21, one rounding to FP32, then the column's power-of-two scale (exact)
                        const long long iv = (long long)(int)r0[jj] * 2097152LL + (long long)(int)r1[jj] * 16384LL +
                                             (long long)(int)r2[jj] * 128LL + (long long)(int)r3[jj];
                        *dst = (float)iv * (float)(__ldg(fscale + col) * 0x1p-21);
                    }
                }
            }
            // this warp is done with the set: hand it back to the MMA issuer
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(&tempty[ab])) : "memory");
        }
    }
    __syncwarp();
    __syncthreads();
    if (threadIdx.x == 0 && *(volatile int*)abort_flag) {
        // copies in flight must land before the CTA may exit
        for (int g = max(0, issued - RT_STAGES); g < issued; ++g)
            (void)bar_wait(&full[g % RT_STAGES], (uint32_t)((g / RT_STAGES) & 1), OZ_DRAIN_LIMIT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// T[m + ldt n] (+)= alpha 2^(ea[m] + eb[n]) sum over splits (fixed order, FP64)
__global__ void gram_i8_reduce_kernel(const double* __restrict__ partial, int ksplit, int ntl, int mtiles, int upper,
                                      int p, int q, const int* __restrict__ ea, const int* __restrict__ eb,
                                      double* __restrict__ T, int ldt, double alpha, int accumulate) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (m >= p || n >= q) return;
    const int mt = m / OZ_M, nt = n / OZ_N;
    if (upper && mt > nt) return;
    const int t = oz_tile_index(mt, nt, mtiles, upper != 0);
    const size_t off = (size_t)t * (OZ_M * OZ_N) + (size_t)(m % OZ_M) * OZ_N + (n % OZ_N);
    const size_t stride = (size_t)ntl * (OZ_M * OZ_N);
    double s = 0.0;
    for (int k = 0; k < ksplit; ++k) s += partial[off + (size_t)k * stride];
    s = ldexp(s, ea[m] + eb[n]) * alpha;
    double* d = T + m + (size_t)ldt * n;
    *d = accumulate ? *d + s : s;
}

int64_t oz_ldk(int64_t N) { return ((N + OZ_K - 1) / OZ_K) * OZ_K; }
size_t a1k(size_t b) { return (b + 1023) & ~(size_t)1023; }
size_t oz_stride(int64_t N, int cols) { return a1k((size_t)oz_ldk(N) * cols); }

struct OzPlan {
    int mtiles, ntiles, ntl, kstages, ksplit;
    size_t partial_bytes;
};

// Tile list; K split into at least enough pieces that no CTA's INT32
// accumulators can overflow, and otherwise into one wave of CTAs.
OzPlan plan_oz(int64_t N, int p, int q, bool upper) {
    OzPlan g{};
    g.mtiles = (p + OZ_M - 1) / OZ_M;
    g.ntiles = (q + OZ_N - 1) / OZ_N;
    g.ntl = upper ? g.ntiles * (g.ntiles + 1) / 2 : g.mtiles * g.ntiles;
    g.kstages = (int)(oz_ldk(N) / OZ_K);
    const int kmin = (g.kstages + OZ_MAX_STAGES_PER_CTA - 1) / OZ_MAX_STAGES_PER_CTA;
    g.ksplit = std::max(kmin, std::min(g.kstages, 148 / std::max(1, g.ntl)));
    g.ksplit = std::max(1, g.ksplit);
    g.partial_bytes = a1k((size_t)g.ksplit * g.ntl * OZ_M * OZ_N * sizeof(double));
    return g;
}

}  // namespace

size_t ozaki_split_bytes(int64_t N, int cols) {
    return 4 * oz_stride(N, cols) + a1k((size_t)cols * sizeof(int)) + a1k((size_t)cols * sizeof(unsigned long long));
}

qsb_status ozaki_split(qsb_dtype dt, int64_t N, const ColumnSet& src, void* dst, cudaStream_t s) {
    const int cols = column_count(src);
    if (cols <= 0) return QSB_OK;
    if (cols > 65535) return fail(QSB_ERR_INVALID, "ozaki_split: too many columns");
    const int64_t ldk = oz_ldk(N);
    const size_t stride = oz_stride(N, cols);
    unsigned char* w = (unsigned char*)dst;
    int* exps = (int*)(w + 4 * stride);
    unsigned long long* maxbits = (unsigned long long*)(w + 4 * stride + a1k((size_t)cols * sizeof(int)));
    QSB_CUDA_TRY(cudaMemsetAsync(maxbits, 0, (size_t)cols * sizeof(unsigned long long), s));
    const int cblocks = (int)std::min<int64_t>((ldk / 4 + 255) / 256, 256);
    if (dt == QSB_F64) {
        column_absmax_kernel<double><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, maxbits);
        slice_kernel<double><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, ldk, maxbits, (int8_t*)w, stride, exps);
    } else {
        column_absmax_kernel<float><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, maxbits);
        slice_kernel<float><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, ldk, maxbits, (int8_t*)w, stride, exps);
    }
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

size_t ozaki_partial_bytes_bound(int64_t N, int p, int q, bool upper) {
    const OzPlan g = plan_oz(N, p, q, upper);
    const int kmin = (g.kstages + OZ_MAX_STAGES_PER_CTA - 1) / OZ_MAX_STAGES_PER_CTA;
    // ksplit' * ntl' <= kmin * ntl' + 148 for every call with p' <= p, q' <= q
    return a1k(((size_t)kmin * g.ntl + 148) * OZ_M * OZ_N * sizeof(double));
}

qsb_status gram_ozaki_tc(int64_t N, const void* A, int p, const void* B, int q, bool upper, double* T, int ldt,
                         double alpha, bool accumulate, void* partial, size_t partial_bytes, cudaStream_t s) {
    if (p <= 0 || q <= 0 || N <= 0) return QSB_OK;
    if (upper && p != q) return fail(QSB_ERR_INVALID, "gram_ozaki_tc: upper mode needs p == q");
    const OzPlan g = plan_oz(N, p, q, upper);
    if (partial_bytes < g.partial_bytes) return fail(QSB_ERR_INVALID, "gram_ozaki_tc: partial workspace too small");
    const int64_t ldk = oz_ldk(N);
    const unsigned char* a = (const unsigned char*)A;
    const unsigned char* b = (const unsigned char*)B;
    const size_t sa = oz_stride(N, p), sb = oz_stride(N, q);
    CUtensorMap m[6];
    for (int k = 0; k < 3; ++k) {
        if (!make_kmajor_map(&m[k], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a + k * sa, ldk, p, OZ_K, OZ_M) ||
            !make_kmajor_map(&m[3 + k], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, b + k * sb, ldk, q, OZ_K, OZ_N))
            return fail(QSB_ERR_CUDA, "gram_ozaki_tc: tensor map encoding failed");
    }
    const int* ea = (const int*)(a + 4 * sa);
    const int* eb = (const int*)(b + 4 * sb);
    QSB_CUDA_TRY(cudaFuncSetAttribute(gram_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)OZ_SMEM));
    gram_i8_kernel<<<dim3(g.ntl, g.ksplit), OZ_THREADS, OZ_SMEM, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], g.kstages,
                                                                       g.ksplit, g.mtiles, upper ? 1 : 0,
                                                                       (double*)partial, device_error_word());
    QSB_CUDA_TRY(cudaGetLastError());
    gram_i8_reduce_kernel<<<dim3((q + 127) / 128, p), 128, 0, s>>>((const double*)partial, g.ksplit, g.ntl, g.mtiles,
                                                                    upper ? 1 : 0, p, q, ea, eb, T, ldt, alpha,
                                                                    accumulate ? 1 : 0);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

size_t gram_ozaki_workspace(int64_t N, int p, int q, bool same) {
    return ozaki_split_bytes(N, p) + (same ? 0 : ozaki_split_bytes(N, q)) + plan_oz(N, p, q, false).partial_bytes;
}

qsb_status gram_ozaki(qsb_dtype dt, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                      double alpha, bool accumulate, bool upper, void* ws, size_t ws_bytes, cudaStream_t s) {
    if (p <= 0 || q <= 0 || N <= 0) return QSB_OK;
    const bool same = (U == V) && (p == q);
    if (ws_bytes < gram_ozaki_workspace(N, p, q, same)) return fail(QSB_ERR_INVALID, "gram_ozaki: workspace too small");
    unsigned char* sa = (unsigned char*)ws;
    unsigned char* sb = same ? sa : sa + ozaki_split_bytes(N, p);
    unsigned char* part = sb + (same ? ozaki_split_bytes(N, p) : ozaki_split_bytes(N, q));
    QSB_TRY(ozaki_split(dt, N, column_set(U, p), sa, s));
    if (!same) QSB_TRY(ozaki_split(dt, N, column_set(V, q), sb, s));
    return gram_ozaki_tc(N, sa, p, sb, q, upper, T, ldt, alpha, accumulate, part, plan_oz(N, p, q, false).partial_bytes,
                         s);
}

size_t ozaki_rot_coef_bytes(int K, int q) {
    const size_t kpad = (size_t)((K + RT_K - 1) / RT_K) * RT_K;
    return 4 * a1k((size_t)q * kpad) + a1k((size_t)q * sizeof(double));
}

// OUT (fp32 columns, one every N elements, gathered destinations) = U C, with U
// an ozaki_split operand of K columns and C a K x q FP64 matrix (device, ld ldc).
// OUT may alias the arrays U was split from: only the slices are read.
qsb_status ozaki_rotate(int64_t N, const void* Usplit, int K, const double* C, int ldc, int q, const ColumnSet& out,
                        void* cws, size_t cws_bytes, cudaStream_t s) {
    if (N <= 0 || K <= 0 || q <= 0) return QSB_OK;
    if (column_count(out) != q) return fail(QSB_ERR_INVALID, "ozaki_rotate: output column count");
    if (cws_bytes < ozaki_rot_coef_bytes(K, q)) return fail(QSB_ERR_INVALID, "ozaki_rotate: workspace too small");
    const int kpad = ((K + RT_K - 1) / RT_K) * RT_K;
    const size_t cstride = a1k((size_t)q * kpad);
    const unsigned char* a = (const unsigned char*)Usplit;
    const size_t sa = oz_stride(N, K);
    const int* eu = (const int*)(a + 4 * sa);
    int8_t* cs = (int8_t*)cws;
    double* fscale = (double*)((unsigned char*)cws + 4 * cstride);
    rot_coef_split_kernel<<<q, 256, 0, s>>>(C, ldc, K, kpad, eu, cs, cstride, fscale);
    QSB_CUDA_TRY(cudaGetLastError());
    const int64_t ldk = oz_ldk(N);
    CUtensorMap m[8];
    for (int k = 0; k < 4; ++k)
        if (!make_kmajor_map(&m[k], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a + k * sa, ldk, K, OZ_M, RT_K) ||
            !make_kmajor_map(&m[4 + k], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, cs + k * cstride, kpad, q, RT_K, RT_N))
            return fail(QSB_ERR_CUDA, "ozaki_rotate: tensor map encoding failed");
    QSB_CUDA_TRY(cudaFuncSetAttribute(rot_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RT_SMEM));
    const int ntn = (q + RT_N - 1) / RT_N;
    const long long tiles = (long long)((N + OZ_M - 1) / OZ_M) * ntn;
    if (tiles > 0x7fffffffLL) return fail(QSB_ERR_INVALID, "ozaki_rotate: too many tiles");
    int dev = 0, sms = 148;
    QSB_CUDA_TRY(cudaGetDevice(&dev));
    QSB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int ctas = (int)std::min<long long>(tiles, (long long)sms);
    rot_i8_kernel<<<ctas, RT_THREADS, RT_SMEM, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], kpad / RT_K, N, q,
                                                    ntn, (int)tiles, fscale, out, device_error_word());
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

}  // namespace qsb

extern "C" {

qsb_status qsb_gram_ozaki_int8_workspace(int64_t N, int p, int q, int same, size_t* bytes) {
    if (!bytes || N < 1 || p < 1 || q < 1) return qsb::fail(QSB_ERR_INVALID, "gram_ozaki_int8_workspace: bad arguments");
    *bytes = qsb::gram_ozaki_workspace(N, p, q, same != 0);
    return QSB_OK;
}

qsb_status qsb_gram_ozaki_int8(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V, double* T,
                               int ldt, int upper, void* workspace, size_t workspace_bytes, void* stream) {
    if (dtype != QSB_F64 && dtype != QSB_F32) return qsb::fail(QSB_ERR_INVALID, "gram_ozaki_int8: bad dtype");
    if (N < 1 || p < 1 || q < 1 || !U || !V || !T || ldt < p || !workspace)
        return qsb::fail(QSB_ERR_INVALID, "gram_ozaki_int8: bad arguments");
    if (p > 65535 || q > 65535) return qsb::fail(QSB_ERR_INVALID, "gram_ozaki_int8: p, q must be < 65536");
    if (upper && p != q) return qsb::fail(QSB_ERR_INVALID, "gram_ozaki_int8: upper needs p == q");
    return qsb::gram_ozaki(dtype, N, p, q, U, V, T, ldt, 1.0, false, upper != 0, workspace, workspace_bytes,
                           (cudaStream_t)stream);
}

size_t qsb_rotate_ozaki_int8_bytes(int64_t N, int K, int q) {
    return qsb::ozaki_split_bytes(N, K) + qsb::ozaki_rot_coef_bytes(K, q);
}

qsb_status qsb_rotate_ozaki_int8_workspace(int64_t N, int K, int q, size_t* bytes) {
    if (!bytes || N < 1 || K < 1 || q < 1) return qsb::fail(QSB_ERR_INVALID, "rotate_ozaki_int8_workspace: bad arguments");
    *bytes = qsb_rotate_ozaki_int8_bytes(N, K, q);
    return QSB_OK;
}

qsb_status qsb_rotate_ozaki_int8(qsb_dtype dtype, int64_t N, int K, int q, const void* U, const double* C, float* out,
                                 void* workspace, size_t workspace_bytes, void* stream) {
    if (dtype != QSB_F64 && dtype != QSB_F32) return qsb::fail(QSB_ERR_INVALID, "rotate_ozaki_int8: bad dtype");
    if (N < 1 || K < 1 || q < 1 || !U || !C || !out || !workspace)
        return qsb::fail(QSB_ERR_INVALID, "rotate_ozaki_int8: bad arguments");
    if (K > 65535 || q > 65535) return qsb::fail(QSB_ERR_INVALID, "rotate_ozaki_int8: K, q must be < 65536");
    if (workspace_bytes < qsb_rotate_ozaki_int8_bytes(N, K, q))
        return qsb::fail(QSB_ERR_INVALID, "rotate_ozaki_int8: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* w = (unsigned char*)workspace;
    QSB_TRY(qsb::ozaki_split(dtype, N, qsb::column_set(U, K), w, s));
    return qsb::ozaki_rotate(N, w, K, C, K, q, qsb::column_set(out, q), w + qsb::ozaki_split_bytes(N, K),
                             qsb::ozaki_rot_coef_bytes(K, q), s);
}

}  // extern "C"
