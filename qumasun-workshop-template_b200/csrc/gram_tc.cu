// Gram products T = U^T V on the 5th-generation tensor cores (tcgen05 + TMEM),
// as split-BF16x3 compensated products with FP32 accumulation:
//   u = u_hi + u_lo (two bfloat16),  u.v ~ u_hi.v_hi + u_hi.v_lo + u_lo.v_hi
// This is the mixed-precision form of the LOBPCG Gram blocks (MakeMatrix_z_blas,
// source/lobpcg_z_multi_mpi.h:300-558: DGEMM_t(2n, 2n, N) on the 2n-real view;
// EigenLOBPCG_d_multi's pairwise inner products, source/lobpcg_d_multi.h:103-133).
//
// Shapes: U is N x p, V is N x q, column-major with leading dimension N (each
// column one grid plane); N is huge (grid points), p, q <= a few hundred.
// Both operands are K-major for the MMA (K = grid index is contiguous).
//
// Pipeline per CTA (128 threads): warp 0 allocates the TMEM accumulator
// (128 lanes x 128 fp32 columns) and its lane 0 streams 64-wide K stages of
// U_hi, U_lo, V_hi, V_lo tiles with 2-D TMA copies (128B swizzle) into a 3-stage
// ring; warp 1 lane 0 issues 12 tcgen05.mma (3 products x 4 K-steps of 16) per
// stage and frees the stage with tcgen05.commit; after the CTA's K range all
// four warps read the accumulator (tcgen05.ld) and write an FP32 partial tile.
// CTAs split K; a second kernel sums the partials in FP64 in fixed order.
//
// All waits are bounded; a wait that runs out sets the device error word, the
// CTA stops issuing, drains (bounded) and frees its TMEM before returning.
#include "qsb_internal.h"
#include "tc_common.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

namespace qsb {
namespace {
using namespace tc;

constexpr int GT_M = 128;          // UMMA M (rows of T per CTA)
constexpr int GT_N = 128;          // UMMA N (columns of T per CTA)
constexpr int GT_K = 64;           // K elements per stage (one 128-byte swizzle row of bf16)
constexpr int GT_STAGES = 3;
constexpr int GT_THREADS = 128;
constexpr int TILE_BYTES_A = GT_M * GT_K * 2;   // 16 KB
constexpr int TILE_BYTES_B = GT_N * GT_K * 2;   // 16 KB
constexpr int STAGE_BYTES = 2 * TILE_BYTES_A + 2 * TILE_BYTES_B;
constexpr size_t GT_SMEM = (size_t)GT_STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers, tmem addr*/;
constexpr unsigned GT_WAIT_LIMIT = 1u << 22;
constexpr unsigned GT_DRAIN_LIMIT = 1u << 16;
constexpr int ERR_GEMM_TIMEOUT = 2;

// Instruction descriptor: kind::f16 with bf16 A and B, fp32 D, both K-major,
// M = 128, N = 128.
constexpr uint32_t GT_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(GT_N >> 3) << 17) |
                              ((uint32_t)(GT_M >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(GT_IDESC), "r"(accumulate)
        : "memory");
}

// Column c of the gathered operand (fp32 or fp64, one column every N elements)
// -> hi, lo bf16 columns of length ldk (a multiple of 4; rows N..ldk zero).
// The columns come from up to kMaxSegments arrays, so the active bands of
// separate bundles form one operand without a copy.  Four elements per thread:
// 16-byte loads when the column start allows, one 8-byte store per half.
template <typename T>
__global__ void split_bf16_kernel(ColumnSet src, int64_t N, int64_t ldk, __nv_bfloat16* __restrict__ hi,
                                  __nv_bfloat16* __restrict__ lo) {
    const int col = blockIdx.y;
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
    const T* s = static_cast<const T*>(b) + (size_t)local * N;
    const bool vec = ((uintptr_t)s % 16) == 0;
    __nv_bfloat16* h = hi + (size_t)col * ldk;
    __nv_bfloat16* l = lo + (size_t)col * ldk;
    const int64_t n4 = ldk / 4;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 4 * q;
        double v[4];
        if (vec && i + 3 < N) {
            if constexpr (sizeof(T) == 4) {
                const float4 f = __ldg(reinterpret_cast<const float4*>(s + i));
                v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
            } else {
                const double2 x0 = __ldg(reinterpret_cast<const double2*>(s + i));
                const double2 x1 = __ldg(reinterpret_cast<const double2*>(s + i + 2));
                v[0] = x0.x; v[1] = x0.y; v[2] = x1.x; v[3] = x1.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = (i + j < N) ? (double)s[i + j] : 0.0;
        }
        __nv_bfloat162 h01, h23, l01, l23;
        __nv_bfloat16 hv[4], lv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            hv[j] = __float2bfloat16_rn((float)v[j]);
            lv[j] = __float2bfloat16_rn((float)(v[j] - (double)__bfloat162float(hv[j])));
        }
        h01.x = hv[0]; h01.y = hv[1]; h23.x = hv[2]; h23.y = hv[3];
        l01.x = lv[0]; l01.y = lv[1]; l23.x = lv[2]; l23.y = lv[3];
        reinterpret_cast<__nv_bfloat162*>(h + i)[0] = h01;
        reinterpret_cast<__nv_bfloat162*>(h + i)[1] = h23;
        reinterpret_cast<__nv_bfloat162*>(l + i)[0] = l01;
        reinterpret_cast<__nv_bfloat162*>(l + i)[1] = l23;
    }
}

// Output tile of list entry t: all mtiles x ntiles tiles (column order), or
// only the tiles on and above the diagonal (mt <= nt, column order).
__host__ __device__ __forceinline__ void tile_of(int t, int mtiles, bool upper, int* mt, int* nt) {
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
__host__ __device__ __forceinline__ int tile_index(int mt, int nt, int mtiles, bool upper) {
    return upper ? nt * (nt + 1) / 2 + mt : nt * mtiles + mt;
}

// One CTA: output tile t of the tile list (blockIdx.x) over the K stages
// [kb0, kb1) of split blockIdx.y (units of GT_K); the fp32 tile goes to
// partial[((split * ntl + t) * GT_M + row) * GT_N + col].
template <int PRODUCTS>
__global__ void __launch_bounds__(GT_THREADS, 1)
gram_tc_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
               const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, int kstages,
               int ksplit, int mtiles, int upper, float* __restrict__ partial, int* __restrict__ err) {
    extern __shared__ unsigned char gt_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)gt_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)GT_STAGES * STAGE_BYTES);
    uint64_t* empty = full + GT_STAGES;
    uint64_t* done = empty + GT_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x, ntl = gridDim.x, split = blockIdx.y;
    int mt, nt;
    tile_of(t, mtiles, upper != 0, &mt, &nt);
    // this CTA's K stages: a contiguous share of the kstages
    const int per = (kstages + ksplit - 1) / ksplit;
    const int kb0 = min(kstages, split * per), kb1 = min(kstages, kb0 + per);
    const int nk = kb1 - kb0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < GT_STAGES; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        bar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(GT_N)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    int issued = 0;   // stages issued by the producer
    if (warp == 0 && lane == 0) {
        // ---- TMA producer ----
        for (int it = 0; it < nk; ++it) {
            const int s = it % GT_STAGES;
            if (it >= GT_STAGES && !bar_wait(&empty[s], (uint32_t)(((it / GT_STAGES) - 1) & 1), GT_WAIT_LIMIT)) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int*)abort_flag) break;
            unsigned char* st = base + (size_t)s * STAGE_BYTES;
            const int kx = (kb0 + it) * GT_K;
            bar_expect_tx(&full[s], STAGE_BYTES);
            tma_2d(st, &mAhi, kx, mt * GT_M, &full[s]);
            tma_2d(st + TILE_BYTES_A, &mAlo, kx, mt * GT_M, &full[s]);
            tma_2d(st + 2 * TILE_BYTES_A, &mBhi, kx, nt * GT_N, &full[s]);
            tma_2d(st + 2 * TILE_BYTES_A + TILE_BYTES_B, &mBlo, kx, nt * GT_N, &full[s]);
            issued = it + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        for (int it = 0; it < nk; ++it) {
            const int s = it % GT_STAGES;
            if (!bar_wait(&full[s], (uint32_t)((it / GT_STAGES) & 1), GT_WAIT_LIMIT)) {
                atomicOr(err, ERR_GEMM_TIMEOUT);
                atomicExch(abort_flag, 1);
                break;
            }
            if (*(volatile int*)abort_flag) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = su32(base + (size_t)s * STAGE_BYTES);
            const uint32_t a_hi = st, a_lo = st + TILE_BYTES_A;
            const uint32_t b_hi = st + 2 * TILE_BYTES_A, b_lo = b_hi + TILE_BYTES_B;
#pragma unroll
            for (int kk = 0; kk < GT_K / 16; ++kk) {
                const uint32_t koff = kk * 32;   // 16 bf16 = 32 bytes along the swizzled row
                const uint32_t acc0 = (it > 0 || kk > 0) ? 1u : 0u;
                umma_bf16(tmem, sw128_kmajor_desc(a_hi + koff), sw128_kmajor_desc(b_hi + koff), acc0);
                umma_bf16(tmem, sw128_kmajor_desc(a_hi + koff), sw128_kmajor_desc(b_lo + koff), 1u);
                umma_bf16(tmem, sw128_kmajor_desc(a_lo + koff), sw128_kmajor_desc(b_hi + koff), 1u);
                if (PRODUCTS == 4)
                    umma_bf16(tmem, sw128_kmajor_desc(a_lo + koff), sw128_kmajor_desc(b_lo + koff), 1u);
            }
            umma_commit(&empty[s]);   // stage s free once these MMAs complete
        }
        umma_commit(done);            // accumulator complete (or nothing in flight after an abort)
    }
    __syncwarp();

    // ---- epilogue: all warps; warp w owns TMEM lanes (rows) 32w .. 32w+31 ----
    bool ok = bar_wait(done, 0, GT_WAIT_LIMIT);
    if (!ok) {
        atomicOr(err, ERR_GEMM_TIMEOUT);
        atomicExch(abort_flag, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = warp * 32 + lane;
    float* prow = partial + ((size_t)split * ntl + t) * (GT_M * GT_N) + (size_t)row * GT_N;
    const bool have = ok && nk > 0;
#pragma unroll 1
    for (int c0 = 0; c0 < GT_N; c0 += 32) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        tmem_ld32(taddr, r);
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
            float4 v = have ? make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                                          __uint_as_float(r[j + 3]))
                            : make_float4(0.f, 0.f, 0.f, 0.f);
            *reinterpret_cast<float4*>(prow + c0 + j) = v;
        }
    }

    // ---- teardown: drain copies still in flight after an abort, free TMEM ----
    __syncthreads();
    if (threadIdx.x == 0 && *(volatile int*)abort_flag) {
        // only the last phase of each stage can still have copies in flight
        for (int it = max(0, issued - GT_STAGES); it < issued; ++it)
            (void)bar_wait(&full[it % GT_STAGES], (uint32_t)((it / GT_STAGES) & 1), GT_DRAIN_LIMIT);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GT_N) : "memory");
    }
}

// T[m + ldt*n] (+)= alpha * sum over splits of the partial tiles (fixed order,
// FP64).  Threads run along n, the contiguous index of a partial tile row.
// Entries of tiles below the diagonal are left alone in upper mode.
__global__ void gram_reduce_kernel(const float* __restrict__ partial, int ksplit, int ntl, int mtiles, int upper,
                                   int p, int q, double* __restrict__ T, int ldt, double alpha, int accumulate) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (m >= p || n >= q) return;
    const int mt = m / GT_M, nt = n / GT_N;
    if (upper && mt > nt) return;
    const int t = tile_index(mt, nt, mtiles, upper != 0);
    const size_t off = (size_t)t * (GT_M * GT_N) + (size_t)(m % GT_M) * GT_N + (n % GT_N);
    const size_t stride = (size_t)ntl * (GT_M * GT_N);
    double s = 0.0;
    for (int k = 0; k < ksplit; ++k) s += (double)partial[off + (size_t)k * stride];
    double* d = T + m + (size_t)ldt * n;
    *d = accumulate ? *d + alpha * s : alpha * s;
}

bool make_operand_map(CUtensorMap* map, const void* base, int64_t ldk, int cols, int box_rows) {
    return make_kmajor_map(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, ldk, cols, GT_K, box_rows);
}

int64_t split_ldk(int64_t N) { return ((N + GT_K - 1) / GT_K) * GT_K; }
size_t align1k(size_t b) { return (b + 1023) & ~(size_t)1023; }
size_t split_half_bytes(int64_t N, int cols) { return align1k((size_t)split_ldk(N) * cols * 2); }

struct GramPlan {
    int mtiles, ntiles, ntl, kstages, ksplit;
    size_t partial_bytes;
};

// Tile list and K split: at most one wave of CTAs (one CTA per SM), each with
// a contiguous share of the K stages.
GramPlan plan_gram(int64_t N, int p, int q, bool upper) {
    GramPlan g{};
    g.mtiles = (p + GT_M - 1) / GT_M;
    g.ntiles = (q + GT_N - 1) / GT_N;
    g.ntl = upper ? g.ntiles * (g.ntiles + 1) / 2 : g.mtiles * g.ntiles;
    g.kstages = (int)(split_ldk(N) / GT_K);
    g.ksplit = std::max(1, std::min(g.kstages, 148 / std::max(1, g.ntl)));
    g.partial_bytes = align1k((size_t)g.ksplit * g.ntl * GT_M * GT_N * sizeof(float));
    return g;
}

}  // namespace

namespace tc {

EncodeTiledFn encode_tiled_fn() {
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

bool make_kmajor_map(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, const void* base, int64_t ldk,
                     int cols, int box_k, int box_rows) {
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)ldk, (cuuint64_t)cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ldk * elem_bytes};
    const cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tc

size_t split_bf16_bytes(int64_t N, int cols) { return 2 * split_half_bytes(N, cols); }

qsb_status split_bf16(qsb_dtype dt, int64_t N, const ColumnSet& src, void* dst, cudaStream_t s) {
    const int cols = column_count(src);
    if (cols <= 0) return QSB_OK;
    if (cols > 65535) return fail(QSB_ERR_INVALID, "split_bf16: too many columns");
    const int64_t ldk = split_ldk(N);
    __nv_bfloat16* hi = (__nv_bfloat16*)dst;
    __nv_bfloat16* lo = (__nv_bfloat16*)((unsigned char*)dst + split_half_bytes(N, cols));
    const int cblocks = (int)std::min<int64_t>((ldk / 4 + 255) / 256, 256);
    if (dt == QSB_F64)
        split_bf16_kernel<double><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, ldk, hi, lo);
    else
        split_bf16_kernel<float><<<dim3(cblocks, cols), 256, 0, s>>>(src, N, ldk, hi, lo);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

size_t gram_partial_bytes(int64_t N, int p, int q, bool upper) { return plan_gram(N, p, q, upper).partial_bytes; }

// ksplit * ntl <= max(148, ntl) for every call, and ntl grows with p and q.
size_t gram_partial_bytes_bound(int p, int q, bool upper) {
    const GramPlan g = plan_gram(GT_K, p, q, upper);
    return align1k((size_t)std::max(148, g.ntl) * GT_M * GT_N * sizeof(float));
}

qsb_status gram_split_tc(int64_t N, const void* A, int p, const void* B, int q, bool upper, double* T, int ldt,
                         double alpha, bool accumulate, void* partial, size_t partial_bytes, cudaStream_t s,
                         int products) {
    if (p <= 0 || q <= 0 || N <= 0) return QSB_OK;
    if (products != 3 && products != 4) return fail(QSB_ERR_INVALID, "gram_split_tc: products must be 3 or 4");
    if (upper && p != q) return fail(QSB_ERR_INVALID, "gram_split_tc: upper mode needs p == q");
    const GramPlan g = plan_gram(N, p, q, upper);
    if (partial_bytes < g.partial_bytes) return fail(QSB_ERR_INVALID, "gram_split_tc: partial workspace too small");
    const int64_t ldk = split_ldk(N);
    const unsigned char* a = (const unsigned char*)A;
    const unsigned char* b = (const unsigned char*)B;
    CUtensorMap mahi, malo, mbhi, mblo;
    if (!make_operand_map(&mahi, a, ldk, p, GT_M) || !make_operand_map(&malo, a + split_half_bytes(N, p), ldk, p, GT_M) ||
        !make_operand_map(&mbhi, b, ldk, q, GT_N) || !make_operand_map(&mblo, b + split_half_bytes(N, q), ldk, q, GT_N))
        return fail(QSB_ERR_CUDA, "gram_split_tc: tensor map encoding failed");
    auto kern = products == 4 ? gram_tc_kernel<4> : gram_tc_kernel<3>;
    QSB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GT_SMEM));
    kern<<<dim3(g.ntl, g.ksplit), GT_THREADS, GT_SMEM, s>>>(mahi, malo, mbhi, mblo, g.kstages, g.ksplit,
                                                                       g.mtiles, upper ? 1 : 0, (float*)partial,
                                                                       device_error_word());
    QSB_CUDA_TRY(cudaGetLastError());
    gram_reduce_kernel<<<dim3((q + 127) / 128, p), 128, 0, s>>>((const float*)partial, g.ksplit, g.ntl, g.mtiles,
                                                                 upper ? 1 : 0, p, q, T, ldt, alpha,
                                                                 accumulate ? 1 : 0);
    QSB_CUDA_TRY(cudaGetLastError());
    return QSB_OK;
}

size_t gram_bf16x3_workspace(int64_t N, int p, int q, bool same) {
    return split_bf16_bytes(N, p) + (same ? 0 : split_bf16_bytes(N, q)) + gram_partial_bytes(N, p, q, false);
}

// T (p x q, ld ldt, FP64) = alpha * U^T V  (+ T when accumulate), U: N x p, V: N x q
// (ld N, fp32 or fp64; V == U with p == q splits once).
qsb_status gram_bf16x3(qsb_dtype dt, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                       double alpha, bool accumulate, bool upper, void* ws, size_t ws_bytes, cudaStream_t s,
                       int products) {
    if (p <= 0 || q <= 0 || N <= 0) return QSB_OK;
    const bool same = (U == V) && (p == q);
    const size_t need = gram_bf16x3_workspace(N, p, q, same);
    if (ws_bytes < need) return fail(QSB_ERR_INVALID, "gram_bf16x3: workspace too small");
    unsigned char* w = (unsigned char*)ws;
    unsigned char* sa = w;
    unsigned char* sb = same ? sa : sa + split_bf16_bytes(N, p);
    unsigned char* part = sb + (same ? split_bf16_bytes(N, p) : split_bf16_bytes(N, q));
    QSB_TRY(split_bf16(dt, N, column_set(U, p), sa, s));
    if (!same) QSB_TRY(split_bf16(dt, N, column_set(V, q), sb, s));
    return gram_split_tc(N, sa, p, sb, q, upper, T, ldt, alpha, accumulate, part, gram_partial_bytes(N, p, q, false), s,
                         products);
}

}  // namespace qsb

extern "C" {

qsb_status qsb_gram_bf16x3_workspace(int64_t N, int p, int q, int same, size_t* bytes) {
    if (!bytes || N < 1 || p < 1 || q < 1) return qsb::fail(QSB_ERR_INVALID, "gram_bf16x3_workspace: bad arguments");
    *bytes = qsb::gram_bf16x3_workspace(N, p, q, same != 0);
    return QSB_OK;
}

namespace {
qsb_status gram_entry(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                      int upper, void* workspace, size_t workspace_bytes, void* stream, int products) {
    if (dtype != QSB_F64 && dtype != QSB_F32) return qsb::fail(QSB_ERR_INVALID, "gram_bf16x3: bad dtype");
    if (N < 1 || p < 1 || q < 1 || !U || !V || !T || ldt < p || !workspace)
        return qsb::fail(QSB_ERR_INVALID, "gram_bf16: bad arguments");
    if (p > 65535 || q > 65535) return qsb::fail(QSB_ERR_INVALID, "gram_bf16x3: p, q must be < 65536");
    if (upper && p != q) return qsb::fail(QSB_ERR_INVALID, "gram_bf16x3: upper needs p == q");
    return qsb::gram_bf16x3(dtype, N, p, q, U, V, T, ldt, 1.0, false, upper != 0, workspace, workspace_bytes,
                            (cudaStream_t)stream, products);
}
}  // namespace

qsb_status qsb_gram_bf16x3(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                           int upper, void* workspace, size_t workspace_bytes, void* stream) {
    return gram_entry(dtype, N, p, q, U, V, T, ldt, upper, workspace, workspace_bytes, stream, 3);
}

qsb_status qsb_gram_bf16x4(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                           int upper, void* workspace, size_t workspace_bytes, void* stream) {
    return gram_entry(dtype, N, p, q, U, V, T, ldt, upper, workspace, workspace_bytes, stream, 4);
}

}  // extern "C"
