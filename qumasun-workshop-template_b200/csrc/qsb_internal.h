// Internal declarations shared by the CUDA translation units of the
// qumasun_b200 library.  Not part of the public ABI (include/qumasun_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/qumasun_b200.h"

namespace qsb {

// Records the message for qsb_last_error() and returns the status.
qsb_status fail(qsb_status st, const std::string& msg);
void set_last_error(const std::string& msg);   // restore the calling thread's message
qsb_status cuda_fail(cudaError_t e, const char* where);

#define QSB_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t qsb_e_ = (expr);                         \
        if (qsb_e_ != cudaSuccess) return ::qsb::cuda_fail(qsb_e_, #expr); \
    } while (0)

#define QSB_TRY(expr)                                        \
    do {                                                     \
        qsb_status qsb_s_ = (expr);                          \
        if (qsb_s_ != QSB_OK) return qsb_s_;                 \
    } while (0)

// FD8 coefficients in the reference's formulas
// (source/GridDifference8th.h:89-101, source/GridDifferenceKpoint8th.h:26-57).
struct FD8Coef {
    double c0;        // centre (includes -coef*|g|^2 for the k-point form)
    double cx[4], cy[4], cz[4];   // second-derivative weights for offsets 1..4
    double ax[4], ay[4], az[4];   // first-derivative weights (k-point form), offsets 1..4
    bool has_grad;                // any |g_d| >= 1e-8
};
FD8Coef make_fd8_coef(double coef, double dx, double dy, double dz, double gx, double gy, double gz);

// Coefficients in the kernel's type.  In fp32 the centre weight is a pair
// c0 + c0lo equal (to ~2^-48) to -2 * (sum of the ROUNDED fp32 neighbour
// weights) - coef |g|^2, so the fp32 stencil still annihilates constants:
// rounding c0 on its own would shift every eigenvalue of the fp32 operator by
// ~|c0| 2^-24 (~1e-6 Ha at h = 0.5 bohr).  In fp64 c0lo is zero and unused.
template <typename T>
struct KC {
    T c0, c0lo;
    T cx[4], cy[4], cz[4];
    T ax[4], ay[4], az[4];
};

template <typename T>
KC<T> to_kc(const FD8Coef& c) {
    KC<T> k;
    double sum_exact = 0.0, sum_rounded = 0.0;
    for (int m = 0; m < 4; ++m) {
        k.cx[m] = (T)c.cx[m]; k.cy[m] = (T)c.cy[m]; k.cz[m] = (T)c.cz[m];
        k.ax[m] = (T)c.ax[m]; k.ay[m] = (T)c.ay[m]; k.az[m] = (T)c.az[m];
        sum_exact += c.cx[m] + c.cy[m] + c.cz[m];
        sum_rounded += (double)k.cx[m] + (double)k.cy[m] + (double)k.cz[m];
    }
    if (sizeof(T) == sizeof(double)) {
        k.c0 = (T)c.c0;
        k.c0lo = T(0);
    } else {
        // c.c0 = -2 * sum_exact - coef |g|^2 (14350 = 2 * (8064 - 1008 + 128 - 9))
        const double target = (c.c0 + 2.0 * sum_exact) - 2.0 * sum_rounded;
        k.c0 = (T)target;
        k.c0lo = (T)(target - (double)k.c0);
    }
    return k;
}

// Launch configuration of the stencil kernels.
struct StencilLaunch {
    int nx, ny, nz;
    int nb;                  // bands
    int is_complex;          // SoA complex bundle
    int mode;                // 0: out += coef*L(psi); 1: out = V psi + coef*L(psi)
    const void* in;
    void* out;
    const void* V;           // mode 1 only
    bool tma_ok = true;      // allow the TMA-pipelined kernel (else the register-prefetch one)
};

// Device-side error word (bit 0: a bounded wait in a kernel ran out), shared by
// all kernels of the library; read and cleared with qsb_device_status().
int* device_error_word();

qsb_status launch_stencil(qsb_dtype dt, const StencilLaunch& L, const FD8Coef& c, cudaStream_t s);
// One system of the batched stencil (stencil.cu): real bundle of nb bands,
// out = V in + FD8 coefficients applied to in (the H psi local part).
struct BatchSysDesc {
    const void* in;
    void* out;
    const void* V;
    int nx, ny, nz, nb;
    FD8Coef coef;
};
qsb_status launch_stencil_batch(qsb_dtype dt, int n, const BatchSysDesc* d, cudaStream_t s);
// Autotuner state (stencil.cu): whether qsb_set_autotune is on, and a line for
// the decision log qsb_autotune_report returns.
bool autotune_enabled();
void autotune_log(const std::string& line);

// Argument checks shared by the apply entry points (context, dtype, band count
// and the two bundle pointers).
qsb_status check_apply(qsb_ham* h, qsb_dtype dtype, int nb, const void* a, const void* b);

// Device-side nonlocal tables (owned by qsb_ham).
struct NLDevice {
    int n_atoms = 0;
    int wmax = 0;                  // max projectors per atom (tables padded to wmax)
    int64_t n_points = 0;          // total points over atoms
    int total_proj = 0;            // sum of widths
    // atom-major point arrays
    int* pt_idx = nullptr;         // folded grid index
    int* pt_xyz = nullptr;         // unfolded coords, 3 per point
    double* pt_beta64 = nullptr;   // [point][wmax]
    float* pt_beta32 = nullptr;
    // per-atom
    int* atom_width = nullptr;     // [n_atoms]
    int* atom_proj_off = nullptr;  // [n_atoms] offset in the global projector numbering
    double* atom_E = nullptr;      // [n_atoms][wmax], zero-padded
    // projection chunks: each chunk is a run of points of one atom
    int n_chunks = 0;
    int* chunk_atom = nullptr;
    int* chunk_order = nullptr;    // launch order of the projection's chunks (by grid position)
    int* chunk_begin = nullptr;
    int* chunk_end = nullptr;
    int* atom_chunk_begin = nullptr;  // [n_atoms]
    int* atom_chunk_end = nullptr;    // [n_atoms]
    // grid-ordered (CSR over all N grid points) view of the same points for
    // the pull-form apply: entries of grid point g are [grid_ptr[g], grid_ptr[g+1])
    int* grid_ptr = nullptr;       // [N+1]
    int n_cov = 0;                 // grid points with at least one entry
    int* cov_grid = nullptr;       // [n_cov]
    int* ent_atom = nullptr;       // [n_points]
    int* ent_xyz = nullptr;        // [n_points][3]
    double* ent_beta64 = nullptr;  // [n_points][wmax]
    float* ent_beta32 = nullptr;
    // projector gradients d beta / d(x, y, z) of the point coordinate, same
    // layout as pt_beta per direction: [3][point][wmax] (optional; forces)
    double* pt_dbeta64 = nullptr;
    float* pt_dbeta32 = nullptr;
    // host copies kept for bookkeeping
    std::vector<int> h_atom_width;
    std::vector<int> h_atom_proj_off;
    std::vector<int> h_npts;
    std::vector<int> h_src;        // per atom-major sorted point: its index in the caller's order within its atom
};

void nl_free(NLDevice& d);
qsb_status nl_upload(NLDevice& d, int nx, int ny, int nz, int n_atoms, const int* npts, const int* widths,
                     const int* coords, const double* beta, const double* energy);

// Workspace needed by nl_project for nb bands (bytes).
size_t nl_workspace_bytes(const NLDevice& d, int ncol);
// Gradient tables in the caller's layout: per atom three blocks (d/dx, d/dy,
// d/dz), each npts x width column-major, atoms concatenated in order.
qsb_status nl_upload_gradients(NLDevice& d, const double* dbeta);
// Workspace of nl_energy_force.
size_t nl_energy_force_bytes(const NLDevice& d, int ncol, int nb);
// Nonlocal band energy sum_n occ_n sum_a,w E_w |<beta|psi_n>|^2 and, when
// forces != nullptr (host, 3 per atom, "+="), F_a = sum 2 occ E_w Re(<psi|beta><grad beta|psi>).
qsb_status nl_energy_force(qsb_dtype dt, const NLDevice& d, int nx, int ny, int nz, int nb, int is_complex,
                           const void* psi, const double* occ_host, double dV, double gx_dx, double gy_dy,
                           double gz_dz, double* energy, double* forces, void* ws, cudaStream_t s);
// coef[atom][w][col] = dV * E_w * <beta|psi_col> (Bloch-phased for complex); ws must hold
// nl_workspace_bytes.  If inner_only, the E_w factor is omitted.
qsb_status nl_project(qsb_dtype dt, const NLDevice& d, int nx, int ny, int nz, int nb, int is_complex,
                      const void* psi, double dV, double gx_dx, double gy_dy, double gz_dz,
                      bool inner_only, void* ws, double** coef_out, cudaStream_t s);
// hpsi[grid][col] += sum_e beta_e . coef  (pull over covered grid points)
qsb_status nl_apply(qsb_dtype dt, const NLDevice& d, int N, int nb, int is_complex, void* hpsi,
                    const double* coef, double gx_dx, double gy_dy, double gz_dz, cudaStream_t s);

// Split-BF16x3 tensor-core Gram products (gram_tc.cu).
//
// A tall operand is a set of columns of N grid values (fp32 or fp64, one
// column every N elements) gathered from up to kMaxSegments separate arrays.
constexpr int kMaxSegments = 4;
struct ColumnSet {
    const void* base[kMaxSegments];
    int cols[kMaxSegments];
    int nseg;
};
inline ColumnSet column_set(const void* a, int na, const void* b = nullptr, int nb = 0, const void* c = nullptr,
                            int nc = 0) {
    ColumnSet s{};
    const void* bs[3] = {a, b, c};
    const int ns[3] = {na, nb, nc};
    for (int k = 0; k < 3; ++k)
        if (ns[k] > 0) {
            s.base[s.nseg] = bs[k];
            s.cols[s.nseg++] = ns[k];
        }
    return s;
}
inline int column_count(const ColumnSet& s) {
    int t = 0;
    for (int k = 0; k < s.nseg; ++k) t += s.cols[k];
    return t;
}
// Bytes of the bf16 hi/lo copy of a cols-column operand.
size_t split_bf16_bytes(int64_t N, int cols);
// dst (split_bf16_bytes) <- hi/lo bf16 copy of the gathered columns
qsb_status split_bf16(qsb_dtype dt, int64_t N, const ColumnSet& src, void* dst, cudaStream_t s);
// Bytes of the split-K partial tiles of one gram_split_tc call.
size_t gram_partial_bytes(int64_t N, int p, int q, bool upper);
// Partial bytes enough for every call with p' <= p, q' <= q (any N).
size_t gram_partial_bytes_bound(int p, int q, bool upper);
// T (p x q, FP64, ld ldt) = alpha * A^T B (+ T when accumulate) from split
// operands A (p columns) and B (q columns); upper: only entries in output tiles
// on or above the diagonal (128 x 128 tiles) are written.
// products: 3 (hi.hi + hi.lo + lo.hi) or 4 (+ lo.lo).
qsb_status gram_split_tc(int64_t N, const void* A, int p, const void* B, int q, bool upper, double* T, int ldt,
                         double alpha, bool accumulate, void* partial, size_t partial_bytes, cudaStream_t s,
                         int products);
// INT8 Ozaki form (gram_i8.cu): three int8 slices per column with a per-column
// power-of-two scale, exact INT32 accumulation on the tensor cores.
size_t ozaki_split_bytes(int64_t N, int cols);
qsb_status ozaki_split(qsb_dtype dt, int64_t N, const ColumnSet& src, void* dst, cudaStream_t s);
// FP64 partial bytes enough for every call with p' <= p, q' <= q at this N.
size_t ozaki_partial_bytes_bound(int64_t N, int p, int q, bool upper);
qsb_status gram_ozaki_tc(int64_t N, const void* A, int p, const void* B, int q, bool upper, double* T, int ldt,
                         double alpha, bool accumulate, void* partial, size_t partial_bytes, cudaStream_t s);
// OUT (q fp32 columns, one every N elements, gathered destinations) = U C on
// the INT8 tensor cores, U an ozaki_split operand of K columns, C K x q FP64
// (device, ld ldc); OUT may alias the arrays U was split from.
size_t ozaki_rot_coef_bytes(int K, int q);
qsb_status ozaki_rotate(int64_t N, const void* Usplit, int K, const double* C, int ldc, int q, const ColumnSet& out,
                        void* cws, size_t cws_bytes, cudaStream_t s);
size_t gram_ozaki_workspace(int64_t N, int p, int q, bool same);
qsb_status gram_ozaki(qsb_dtype dt, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                      double alpha, bool accumulate, bool upper, void* ws, size_t ws_bytes, cudaStream_t s);
// One-call form on plain operands U (N x p), V (N x q), ld N.
size_t gram_bf16x3_workspace(int64_t N, int p, int q, bool same);
qsb_status gram_bf16x3(qsb_dtype dt, int64_t N, int p, int q, const void* U, const void* V, double* T, int ldt,
                       double alpha, bool accumulate, bool upper, void* ws, size_t ws_bytes, cudaStream_t s,
                       int products);

}  // namespace qsb

struct qsb_ham {
    int device = -1;                       // CUDA device current at qsb_ham_create (holds the tables)
    int nx = 0, ny = 0, nz = 0;
    size_t N = 0;
    double dx = 0, dy = 0, dz = 0;
    double* V64 = nullptr;
    float* V32 = nullptr;
    qsb::NLDevice nl;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    // optional per-kernel event timing of qsb_ham_apply
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;      // free events
    std::vector<cudaEvent_t> ev_rec;       // recorded triples: start, after projection, after stencil
    int launches = 0;
    // qsb_ham_apply_host: two device staging slots (psi chunk, hpsi chunk) and
    // the copy streams / events of the pipeline (created on first use)
    void* stage = nullptr;
    size_t stage_bytes = 0;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t pev[7] = {};               // start, in_ready[2], done[2], out_free[2]
    // kinetic operator of qsb_ham_apply: 0 FD8 stencil, 1 FFT (qsb_ham_set_kinetic)
    int kinetic = 0;
    struct FftPlan {
        int dtype, cplx, batch;
        int forward, backward;             // cufftHandle values
    };
    std::vector<FftPlan> fft_plans;        // by (dtype, complex, batch)
    void* fft_buf = nullptr;               // spectra of one band chunk
    size_t fft_buf_bytes = 0;
};

namespace qsb {
// Shape of a solver context (lobpcg.cu): grid points, bands, complex, mixed precision.
void eigensolver_shape(const qsb_eigensolver* es, int64_t* N, int* nmax, int* cplx, int* mixed);
// FFT kinetic term of qsb_ham_apply (kinetic_fft.cu): hpsi = -1/2 (grad + i g)^2 psi
// + V psi ("=" semantics; the nonlocal part is added by the caller).
qsb_status kinetic_fft_apply(qsb_ham* h, qsb_dtype dtype, int is_complex, int nb, const void* psi, void* hpsi,
                             double gx, double gy, double gz, cudaStream_t s, int* launches);
void kinetic_fft_free(qsb_ham* h);
}  // namespace qsb
