/*
 * qumasun_b200.h — C ABI of the B200 (sm_100a) Kohn-Sham H.psi + LOBPCG path.
 *
 * Plain pointers and sizes only; every call returns a qsb_status and, on
 * failure, qsb_last_error() describes it.  All array arguments named *_dev
 * or documented as "device" are CUDA device pointers; "stream" is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Layouts are the reference's own, so a caller's buffers pass through unchanged
 * (source/qumasun_base1.h:457-460, source/soacomplex.h:4):
 *   - grid index i = ix + nx*(iy + ny*iz), x fastest, periodic in x, y, z;
 *   - real band bundle:    band b at  psi + b*N                    (N = nx*ny*nz);
 *   - complex band bundle: band b re at psi + 2*b*N, im at psi + (2*b+1)*N  (SoA).
 * dtype QSB_F64 means double arrays, QSB_F32 float arrays (same layouts).
 *
 * Reference interfaces each entry point replaces are cited as path:line
 * within the reference project (atsushi-m-ito/QUMASUN-workshop-template).
 */
#ifndef QUMASUN_B200_H
#define QUMASUN_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QSB_API __attribute__((visibility("default")))
#else
#define QSB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qsb_status {
    QSB_OK = 0,
    QSB_ERR_INVALID = 1,   /* bad argument (size, pointer, dtype) */
    QSB_ERR_CUDA = 2,      /* a CUDA runtime/library call failed */
    QSB_ERR_NOMEM = 3,     /* device allocation failed */
    QSB_ERR_STATE = 4,     /* call made on an incompletely set-up context */
    QSB_ERR_SOLVER = 5,    /* small dense eigensolver / Cholesky failed */
    QSB_ERR_NUMERIC = 6    /* non-finite values detected */
} qsb_status;

typedef enum qsb_dtype { QSB_F64 = 0, QSB_F32 = 1 } qsb_dtype;

/* Text of the last error raised on the calling thread ("" if none). */
QSB_API const char* qsb_last_error(void);
/* Library version string. */
QSB_API const char* qsb_version(void);

/* Device-side error word of the current device (synchronizes with it): bit 0
 * set means a kernel's bounded wait on an asynchronous copy ran out and that
 * kernel returned early (its output is incomplete).  clear != 0 resets it.
 * The reference has no counterpart (it exits on CUDA errors,
 * source/gyield/gy_cuda.h:95-100). */
QSB_API qsb_status qsb_device_status(int* code, int clear);

/* ---------------------------------------------------------------------------
 * FD8 stencils (stateless).
 * ------------------------------------------------------------------------- */

/* out += coef * Laplacian_8th(p) for nb real bands, periodic boundaries.
 * Replaces Laplacian8th<T>(grid, out, p, coef, dx, dy, dz)
 * (source/GridDifference8th.h:177-184; stencil :82-148, halo :19-78), applied
 * band by band; same accumulate ("+=") semantics. */
QSB_API qsb_status qsb_laplacian8th(qsb_dtype dtype, int nx, int ny, int nz, int nb,
                            void* out_dev, const void* p_dev, double coef,
                            double dx, double dy, double dz, void* stream);

/* out += coef * (Laplacian + 2 i g.grad - |g|^2) src for nb complex SoA bands:
 * out.re gets Lap_g(re) - D_g(im), out.im gets Lap_g(im) + D_g(re).
 * Replaces LaplacianKpoint8th_ddm(grid, out, src, coef, dx, dy, dz, gx, gy, gz)
 * (source/GridDifferenceKpoint8th.h:324-366, stencil :17-120) with
 * split_dimension 0, including its |g_d| < 1e-8 dispatch; no static buffers. */
QSB_API qsb_status qsb_laplacian_kpoint8th(qsb_dtype dtype, int nx, int ny, int nz, int nb,
                                   void* out_dev, const void* src_dev, double coef,
                                   double dx, double dy, double dz,
                                   double gx, double gy, double gz, void* stream);

/* ---------------------------------------------------------------------------
 * Hamiltonian context: local potential + nonlocal KB projectors on one grid.
 * Replaces the state QUMASUN_BASE1 / PseudoPotNonlocal_SvF2_kpoint hold for
 * mHamiltonianMatrix_ddm (source/qumasun_base1.matrix.h:263-317).
 * ------------------------------------------------------------------------- */
typedef struct qsb_ham qsb_ham;

QSB_API qsb_status qsb_ham_create(qsb_ham** ham, int nx, int ny, int nz, double dx, double dy, double dz);
QSB_API qsb_status qsb_ham_destroy(qsb_ham* ham);

/* V: N doubles (the total local potential Vtot), host (on_device = 0) or
 * device (on_device = 1) memory.  Copied into the context (FP64 and FP32). */
QSB_API qsb_status qsb_ham_set_potential(qsb_ham* ham, const double* V, int on_device);

/* Nonlocal Kleinman-Bylander projectors, host arrays, copied into the context.
 * Replaces PseudoPotNonlocal_SvF2_kpoint::UpdatePosition's products
 * (source/PseudoPotNonlocal_SvF2_kpoint.h:3315-3406): per atom a point list
 * and a projector table, like PP_Proj_Ylm_each_atom::projector_RY (:216-236).
 *   npts[a]    points of atom a (any shape: voxel sphere or the reference's cube blocks)
 *   widths[a]  projectors of atom a (sum of 2l+1 over channels; 0 allowed)
 *   coords     3 ints per point, UNFOLDED grid coordinates (may lie outside
 *              [0,n)); the point acts on grid point (coords mod n) and its Bloch
 *              phase is exp(i g.(ix*dx, iy*dy, iz*dz)) as in mCreateBlochExp (:3538-3605)
 *   beta       per atom npts[a] x widths[a] values, column-major (point fastest)
 *   energy     per atom widths[a] KB energies E_w (projector_energy_RY, :151)
 * Arrays are concatenated over atoms in atom order. */
QSB_API qsb_status qsb_ham_set_projectors(qsb_ham* ham, int n_atoms, const int* npts, const int* widths,
                                  const int* coords, const double* beta, const double* energy);

/* Same, building analytic GTH (Goedecker-Teter-Hutter) projectors with one
 * radial function per channel (l = 0: 1 projector, l = 1: 3 projectors with
 * real harmonics x, y, z) on voxel spheres of radius rcut_factor*r_l.
 *   pos[3a..]    atom positions in bohr (any real value; folded periodically)
 *   species[a]   index into the species tables
 *   nl[s]        channels of species s (0, 1 or 2)
 *   r_l[2s+l], h_l[2s+l]   GTH radius and h^l_11 of channel l of species s */
QSB_API qsb_status qsb_ham_set_gth_projectors(qsb_ham* ham, int n_atoms, const double* pos, const int* species,
                                      int n_species, const int* nl, const double* r_l, const double* h_l,
                                      double rcut_factor);

/* Number of projector points held (sum over atoms), and total projectors. */
QSB_API qsb_status qsb_ham_projector_info(const qsb_ham* ham, int64_t* total_points, int* total_projectors);

/* hpsi = V psi + V_NL psi - 1/2 Laplacian_8th(psi)   ("=" semantics)
 * is_complex = 0: nb real bands, Gamma point (g ignored).
 * is_complex = 1: nb complex SoA bands at Bloch vector g (bohr^-1), with the
 *                 k-point kinetic operator of LaplacianKpoint8th_ddm and the
 *                 Bloch-phased projectors of ProjectionPP_bundle.
 * Replaces mHamiltonianMatrix_ddm (source/qumasun_base1.matrix.h:263-291):
 * SetZero, mPotentialMatrix_ddm, ProjectionPP_bundle, mKineticMatrixAdd_ddm_kpint. */
QSB_API qsb_status qsb_ham_apply(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                         const void* psi_dev, void* hpsi_dev,
                         double gx, double gy, double gz, void* stream);

/* Kinetic operator of qsb_ham_apply (and of everything built on it: the
 * eigensolvers given this context, the SCF driver, qsb_ham_apply_host):
 *   0  FD8 Laplacian (default; mKineticMatrixAdd_ddm_kpint, the stencil path);
 *   1  FFT kinetic, the reference's default (m_algorithm_Laplacian = 1,
 *      source/qumasun_base1.h:243; mHamiltonianMatrix_ddm_bundle,
 *      source/qumasun_base1.matrix.h:171-228): forward 3-D FFT of each band,
 *      times |G + k|^2 / 2 with the Nyquist index of an even grid taken as
 *      +n/2 (OperateKineticInKspace_bundle :96-123), inverse FFT, times 1/N,
 *      + V psi, + the nonlocal part.  Batched cuFFT plans and a spectrum
 *      buffer for 32 bands are made on first use and kept in the context.
 *      FP64 and FP32 (the mixed solver's operator). */
QSB_API qsb_status qsb_ham_set_kinetic(qsb_ham* ham, int algorithm);

/* The same H psi for bundles in HOST memory, the call shape of the reference's
 * CPU build of mHamiltonianMatrix_ddm (source/qumasun_base1.matrix.h:263-291,
 * psi and hpsi in host arrays): the bands go through the device in chunks of
 * chunk_bands (0: nb / 16 rounded up), the host-to-device copy of the next
 * chunk, the apply of this one (on `stream`) and the device-to-host copy of the
 * previous one overlapping (two device staging slots of 2 chunks each, kept in
 * the context and grown with cudaMalloc; two copy streams of the context).
 * Asynchronous like cudaMemcpyAsync: hpsi_host is complete once `stream` has
 * reached this point.  Page-locked host buffers (cudaHostAlloc /
 * cudaHostRegister) let the copies overlap; pageable ones work but serialize.
 * Calls on one context must not overlap (they share the staging slots). */
QSB_API qsb_status qsb_ham_apply_host(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                                      const void* psi_host, void* hpsi_host,
                                      double gx, double gy, double gz, int chunk_bands, void* stream);

/* H psi of n_sys independent systems at once (real bands, Gamma point, FD8
 * kinetic): hpsi[i] = H_i psi[i] for nb[i] bands of system i (each its own
 * qsb_ham: grid, spacing, potential, projectors).  The FD8 + V part of all
 * systems runs in ONE persistent launch over a work list of (system, tile of
 * 32 x 16 points (FP32: 32 x 32), 32-plane z chunk, band) items, largest
 * systems first, each item the tile work of the register-prefetch stencil
 * (results equal the per-system FP32 stencil's bit for bit); each system's
 * nonlocal projection and expansion keep their own launches.  The reference
 * applies H system by system (mHamiltonianMatrix_ddm, source/qumasun_base1.matrix.h:263-291);
 * for many small, uneven cells a launch per system leaves most SMs idle.
 * Results equal qsb_ham_apply's to rounding (a different stencil kernel).
 * With qsb_set_autotune on, the first call for a set of shapes times this
 * form against the systems' own qsb_ham_apply and keeps the faster. */
QSB_API qsb_status qsb_ham_apply_batch(qsb_dtype dtype, int n_sys, qsb_ham* const* hams, const int* nb,
                                       const void* const* psi, void* const* hpsi, void* stream);

/* Autotuner.  On (enable != 0), the first launch of each stencil shape in the
 * H psi form (FP64; grid, bands rounded up to a power of two, real / complex)
 * times the stencil kernels that apply to it (the TMA-box kernel with a
 * producer warp, the TMA-plane kernel, the register-prefetch kernel) on the
 * caller's stream and keeps the fastest for that shape; qsb_ham_apply_batch
 * likewise chooses between its batched and per-system forms.  Tuning runs on
 * the caller's buffers (the outputs are rewritten, the last run is the chosen
 * kernel's), so make tuned first calls outside stream capture.  Off (the
 * default): the fixed choice (the TMA-box kernel where it applies).
 * qsb_autotune_report copies the decision log (one line per decision, with
 * the times) into buf (len bytes, NUL-terminated); *needed = its size + 1. */
QSB_API qsb_status qsb_set_autotune(int enable);
QSB_API qsb_status qsb_autotune_report(char* buf, int len, int* needed);

/* hpsi += V_NL psi.  Replaces PseudoPotNonlocal_SvF2_kpoint::ProjectionPP_bundle
 * (source/PseudoPotNonlocal_SvF2_kpoint.h:4239-4247, CPU :3911-4046, GPU :4053-4236). */
QSB_API qsb_status qsb_ham_nonlocal_apply(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                                  const void* psi_dev, void* hpsi_dev,
                                  double gx, double gy, double gz, void* stream);

/* Size of the fixed device scratch used by qsb_ham_nonlocal_apply_static. */
#define QSB_NL_STATIC_SCRATCH_BYTES (4u << 20)

/* hpsi += V_NL psi exactly like qsb_ham_nonlocal_apply, but the call allocates
 * no device memory: its scratch (the <beta|psi> partial sums and per-atom
 * coefficients) is a fixed array of QSB_NL_STATIC_SCRATCH_BYTES (4 MiB) in the
 * library's device memory, present on every GPU that loads the library until
 * the process exits.  No counterpart in the reference (its nonlocal apply
 * sub-allocates from the caller's work buffer).
 * For callers that cannot allocate device memory while they run: codes that
 * reserve the whole device memory for their own arena at start-up, and loops
 * that cannot take the device-wide synchronization of cudaMalloc/cudaFree (the
 * regular entry point grows its workspace with cudaMalloc when a larger bundle
 * first arrives).
 *   - Requests needing more scratch than the array holds are rejected with
 *     QSB_ERR_INVALID and a message giving both sizes; split the bands into
 *     smaller bundles.  The need is about 8*(projector points/8192 + atoms)*
 *     (max projectors per atom)*(nb, or 2*nb for complex) bytes.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) and caches it; make that first call before any
 *     stream capture on that device.
 *   - All calls share the one array: calls that overlap on the GPU (other
 *     streams, other host threads, without ordering between them) race on it.
 *     Nothing in it needs to start at zero (each call writes every element it
 *     reads before reading it); it keeps the last call's values. */
QSB_API qsb_status qsb_ham_nonlocal_apply_static(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                                                 const void* psi_dev, void* hpsi_dev,
                                                 double gx, double gy, double gz, void* stream);

/* <beta_aw | psi_c> * dV for every projector and column into out_host
 * (double, layout [column][projector], projectors in atom order, columns:
 * real -> band b; complex -> 2b (re), 2b+1 (im)), the quantity
 * mInnerNonlocalPsi_v4_bundle computes (source/PseudoPotNonlocal_SvF2_kpoint.h:4463-4576;
 * index layout there is per atom, here global). */
QSB_API qsb_status qsb_ham_nonlocal_project(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                                    const void* psi_dev, double gx, double gy, double gz,
                                    double* out_host, void* stream);

/* Projector gradients d beta / d(x, y, z) (of the grid point's coordinate) for
 * the tables given to qsb_ham_set_projectors, needed by the forces: host array,
 * per atom three blocks (d/dx, d/dy, d/dz), each npts[a] x widths[a]
 * column-major like beta, atoms concatenated in order.  The reference's
 * FORCE_DIFF_PROJ path builds the same gradients of projector_RY
 * (source/PseudoPotNonlocal_SvF2_kpoint.h:31-45).  qsb_ham_set_gth_projectors
 * sets them itself (analytic derivatives of the GTH projectors). */
QSB_API qsb_status qsb_ham_set_projector_gradients(qsb_ham* ham, const double* dbeta);

/* Nonlocal band energy E = sum_n occ_n sum_atoms sum_w E_w |dV <beta_w|psi_n>|^2
 * (the Bloch-phased projection for complex bands at vector g).  occupancies:
 * host, nb values.  Replaces EnergyPPnonlocal_bundle
 * (source/PseudoPotNonlocal_SvF2_kpoint.h:5033-5135). */
QSB_API qsb_status qsb_ham_nonlocal_energy(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb, const void* psi_dev,
                                           const double* occupancies, double gx, double gy, double gz,
                                           double* energy, void* stream);

/* Same energy and the nonlocal forces, "+=" into forces (host, 3 per atom):
 *   F_a += sum_n occ_n sum_w 2 E_w Re( conj(dV <beta_w|psi_n>) dV <grad beta_w|psi_n> )
 * i.e. -dE/dR_a at fixed psi, computed in reverse mode: the adjoint of the
 * projection (2 occ E_w conj(c)) contracted with the projector-gradient
 * projections.  Replaces ForceNonlocal_bundle (grad(p) form,
 * source/PseudoPotNonlocal_SvF2_kpoint.h:3629-3731).  Needs projector gradients. */
QSB_API qsb_status qsb_ham_nonlocal_energy_force(qsb_ham* ham, qsb_dtype dtype, int is_complex, int nb,
                                                 const void* psi_dev, const double* occupancies, double gx, double gy,
                                                 double gz, double* energy, double* forces, void* stream);

/* ---------------------------------------------------------------------------
 * Block LOBPCG eigensolvers (device resident).
 * ------------------------------------------------------------------------- */
typedef struct qsb_eigensolver qsb_eigensolver;

/* Operator callback: ax = A x for nb bands (device pointers, same layout as the
 * solver's bundles), enqueued on `stream`; returns 0 on success.  This is the
 * reference's OpeA functor (source/qumasun_kpoint.lobpcg.h:97-99,
 * source/lobpcg_d_multi.h:70), one call per bundle instead of per band. */
typedef int (*qsb_apply_fn)(void* user, int nb, const double* x_dev, double* ax_dev, void* stream);

/* Solver context for bundles of up to n bands of N grid points (complex SoA
 * when is_complex), holding the device work bundles R, AX, AR, AP and a
 * temporary (the reference's `work`/`temporary` arenas,
 * source/lobpcg_z_multi_mpi.h:2862-2881) and the cuBLAS / cuSOLVER handles. */
QSB_API qsb_status qsb_eigensolver_create(qsb_eigensolver** es, int64_t N, int n, int is_complex);

/* Precision of a solver context.
 *   QSB_PREC_FP64   everything in FP64 (the reference's arithmetic).
 *   QSB_PREC_MIXED  the bundles X, R, P, AX, AR, AP live in FP32 inside the
 *                   context and the operator runs in FP32 (qsb_ham_apply with
 *                   QSB_F32, or an fp32 callback); the Gram / Rayleigh-Ritz
 *                   products run on the tensor cores as split-BF16x3 products
 *                   with FP32 accumulation (qsb_gram_bf16x3); the rotations
 *                   X' = X Cx + R Cr + P Cp are FP32 GEMMs; the pencil solve,
 *                   Rayleigh quotients, norms and the convergence tests stay
 *                   FP64.  The caller's X, keep and eigenvalues stay FP64 and
 *                   the qsb_lobpcg_z / qsb_lobpcg_d calls are unchanged; X and
 *                   keep come back with FP32 resolution. */
typedef enum qsb_precision { QSB_PREC_FP64 = 0, QSB_PREC_MIXED = 1 } qsb_precision;
QSB_API qsb_status qsb_eigensolver_create_ex(qsb_eigensolver** es, int64_t N, int n, int is_complex,
                                             qsb_precision precision);
QSB_API qsb_status qsb_eigensolver_destroy(qsb_eigensolver* es);
/* H of a qsb_ham context (Bloch vector g for complex bands) as the operator. */
QSB_API qsb_status qsb_eigensolver_set_hamiltonian(qsb_eigensolver* es, qsb_ham* ham, double gx, double gy, double gz);
/* A user callback as the operator. */
QSB_API qsb_status qsb_eigensolver_set_operator(qsb_eigensolver* es, qsb_apply_fn op, void* user);
/* FP32 operator callback for QSB_PREC_MIXED contexts (fp32 bundles, same layouts). */
typedef int (*qsb_apply_f32_fn)(void* user, int nb, const float* x_dev, float* ax_dev, void* stream);
QSB_API qsb_status qsb_eigensolver_set_operator_f32(qsb_eigensolver* es, qsb_apply_f32_fn op, void* user);
/* Iterations done by the last solve, and whether it ended with the norm-check rollback. */
QSB_API qsb_status qsb_eigensolver_last_stats(const qsb_eigensolver* es, int* iterations, int* rolled_back);
/* Overlap-basis fallback of the Rayleigh-Ritz step.  When the Cholesky of
 * ZHEGVD / DSYGVD finds the overlap matrix not positive definite (mixed
 * precision: on the unit-diagonal-scaled pencil, where the tensor-core Gram
 * errors, ~2^-17 / sqrt(N) of the diagonal for split-BF16x3, make it fail once
 * the basis [X R P] turns ill-conditioned near convergence; FP64: a search
 * basis that has become numerically dependent, as when a run is continued
 * from states of another precision), the step scales the pencil to a unit
 * diagonal, eigendecomposes the overlap matrix and drops the directions whose
 * overlap eigenvalue is below tol * (largest); the Ritz pairs are taken in the
 * rest (Stathopoulos-Wu's SVQB basis, as Hetmaniuk-Lehoucq use it in LOBPCG).
 * Default: mixed 1e-5 / sqrt(N) within [1e-8, 1e-5]; FP64 1e-12. */
QSB_API qsb_status qsb_eigensolver_set_drop_tolerance(qsb_eigensolver* es, double tol);
/* QSB_PREC_MIXED: how the Gram / Rayleigh-Ritz products are formed.
 *   QSB_GRAM_BF16X3     split-BF16x3 on the tensor cores (qsb_gram_bf16x3)
 *   QSB_GRAM_BF16X4     the same plus lo.lo (qsb_gram_bf16x4)
 *   QSB_GRAM_INT8_OZAKI three int8 slices, exact INT32 accumulation
 *                       (qsb_gram_ozaki_int8); the default.
 * The BF16 forms accumulate in the tensor core's FP32, which rounds toward
 * zero: a same-sign sum loses ~4e-8 of itself per MMA in one accumulator chain,
 * measured -4.8e-5 relative on overlap diagonals at 8192 grid points per CTA.
 * That bias shifts all overlap eigenvalues; at 96^3 grids with 128 bands the
 * BF16 solvers diverge, the INT8 one converges. */
typedef enum qsb_gram_kind { QSB_GRAM_BF16X3 = 3, QSB_GRAM_BF16X4 = 4, QSB_GRAM_INT8_OZAKI = 8 } qsb_gram_kind;
QSB_API qsb_status qsb_eigensolver_set_gram_kind(qsb_eigensolver* es, qsb_gram_kind kind);
/* Of the last call: how many Rayleigh-Ritz steps were solved by the Cholesky
 * route (?hegvd / ?sygvd; mixed precision: on the unit-diagonal-scaled pencil)
 * and how many fell back to the overlap-basis solve because that Cholesky found
 * the overlap not positive definite. */
QSB_API qsb_status qsb_eigensolver_solve_stats(const qsb_eigensolver* es, int* cholesky_solves,
                                               int* overlap_basis_solves);
/* Of the last call (mixed precision): most directions dropped in one
 * iteration, smallest kept overlap eigenvalue relative to the largest, and the
 * tolerance in force. */
QSB_API qsb_status qsb_eigensolver_overlap_stats(const qsb_eigensolver* es, int* max_dropped, double* min_kept_ratio,
                                                 double* drop_tolerance);
/* FP64 complex solver: how the Rayleigh-Ritz pencil is formed between full
 * recomputes.  mode 1 (the default) is the reference's steady-state update
 * (NextMatrix_z, source/lobpcg_z_multi_mpi.h:579-794, used at :2782, and
 * MakeMatrix_z_blas's skips at :2091-2101): in iterations that are not a
 * multiple of 6 (S_MAT_REST_LIMIT, :1808) only X^H A R, R^H A R, R^H A P and
 * R^H R are formed from the bundles; the X/P blocks come from the previous
 * pencil and its eigenvectors, and X^H R, R^H P from R = AX - X E.  mode 0
 * forms every block from the bundles in every iteration.  The keep_S_matrix
 * reuse across calls (:1811) is not taken: the first iteration of each call
 * forms the whole pencil. */
QSB_API qsb_status qsb_eigensolver_set_pencil_update(qsb_eigensolver* es, int mode);
/* Of the last FP64 complex call: pencils formed in full from the bundles, and
 * pencils formed by the steady-state update. */
QSB_API qsb_status qsb_eigensolver_pencil_stats(const qsb_eigensolver* es, int* full, int* steady);

/* Complex block LOBPCG.  Replaces LOBPCG::Eigen_z_multi_mpi(l_grid, dVol,
 * num_solution, iter_max, eigen_values, eigen_vectors, keep, work, temporary,
 * p_num_fix, residual_threshold, keep_S_matrix, SCF_step, sk, OpeA, watch)
 * (source/lobpcg_z_multi_mpi.h:1732-1742) on one rank:
 *   eigen_values  host, n values; in: previous eigenvalues, out: Ritz values of
 *                 the active bands (fixed bands keep theirs)
 *   X             device, n complex SoA bands, in/out (returned normalized, dV-weighted)
 *   keep          device, n complex SoA bands: the P directions kept between
 *                 calls (zeroed when scf_step == 0)
 *   p_num_fix     in/out soft-locking count (leading converged bands), <= n/2
 *   residual_threshold  bands with ||r|| below it (leading run) are fixed
 * Errors: QSB_ERR_SOLVER when the overlap matrix is not positive definite. */
QSB_API qsb_status qsb_lobpcg_z(qsb_eigensolver* es, double dVol, int n, int iter_max, double* eigen_values,
                                double* X, double* keep, int* p_num_fix, double residual_threshold, int scf_step,
                                void* stream);

/* Real block LOBPCG.  Replaces EigenLOBPCG_d_multi(N, dVol, num_solution,
 * iter_max, eigen_values, eigen_vectors, keep, work, is_first_time, OpeA, watch)
 * (source/lobpcg_d_multi.h:23-27): X and keep are device real bundles (n x N),
 * eigen_values host; stops early when max ||r||^2 dV < 1e-10 dV (:525). */
QSB_API qsb_status qsb_lobpcg_d(qsb_eigensolver* es, double dVol, int n, int iter_max, double* eigen_values,
                                double* X, double* keep, int is_first_time, void* stream);

/* dV-weighted orthonormalisation of nb bands in place (X: device, real bundle
 * nb x N or complex SoA bundle), the starting states of an SCF.  Replaces
 * GramSchmidt_ddm (source/GramSchmidt_mpi.h:56-96: classical Gram-Schmidt band
 * after band) by Cholesky QR applied twice (G = dV X^H X, G = U^H U, X <- X U^-1):
 * the same Q factor with a positive-diagonal R, so the same states to rounding
 * for bands that are not near-dependent.  QSB_ERR_NUMERIC when the bands are
 * linearly dependent.  Allocates its scratch (2N nb doubles for complex bands)
 * and BLAS handles for the call; synchronizes the stream. */
QSB_API qsb_status qsb_orthonormalize(int64_t N, int nb, int is_complex, double* X, double dV, void* stream);

/* Gram product T = U^T V on the tcgen05 tensor cores as split-BF16x3
 * compensated products (u = u_hi + u_lo in bfloat16, three products
 * hi.hi + hi.lo + lo.hi) with FP32 accumulation per CTA and FP64 summation of
 * the split-K partials: the mixed-precision form of the LOBPCG Gram blocks
 * (MakeMatrix_z_blas's DGEMM_t(2n, 2n, N) on the 2n-real view,
 * source/lobpcg_z_multi_mpi.h:300-558).
 *   U (N x p), V (N x q): device, column-major with leading dimension N, FP32
 *   or FP64 (V == U with p == q converts once); T: device FP64, p x q, ld ldt.
 *   upper != 0 (p == q): only the 128 x 128 output tiles on or above the
 *   diagonal are computed and written (all upper-triangle entries among them),
 *   the form the symmetric / Hermitian pencils use; other entries are untouched.
 *   workspace: device, at least the bytes qsb_gram_bf16x3_workspace returns. */
QSB_API qsb_status qsb_gram_bf16x3_workspace(int64_t N, int p, int q, int same, size_t* bytes);
QSB_API qsb_status qsb_gram_bf16x3(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V,
                                   double* T, int ldt, int upper, void* workspace, size_t workspace_bytes,
                                   void* stream);
/* Same with the fourth product lo.lo.  The three-product form misses
 * sum(u_lo v_lo), which on a diagonal entry u.u is sum(u_lo^2) > 0: the
 * diagonal comes out low by ~2^-16/3 relative, a bias, not noise, that an
 * overlap matrix turns into a shift of all its eigenvalues.  With lo.lo the
 * remaining error is the rounding of u_lo (~2^-17 relative, no sign bias). */
QSB_API qsb_status qsb_gram_bf16x4(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V,
                                   double* T, int ldt, int upper, void* workspace, size_t workspace_bytes,
                                   void* stream);

/* Gram product T = U^T V on the INT8 tensor cores (tcgen05 kind::i8) by the
 * Ozaki splitting: each column of U and V gets a power-of-two scale 2^e with
 * max|u| 2^-e in [32, 64) and three int8 slices u 2^-e = s0 + s1 2^-7 + s2 2^-14
 * (+ |r| <= 2^-15, round-to-nearest, no sign bias); the six slice products with
 * i + j <= 2 accumulate exactly in INT32 (TMEM) and combine in FP64.  Relative
 * error ~2^-20 per element product, random-signed, so Gram entries over N
 * points carry ~1e-6 / sqrt(N) and no systematic part beyond ~2^-28.  Same
 * arguments and workspace query as qsb_gram_bf16x3. */
QSB_API qsb_status qsb_gram_ozaki_int8_workspace(int64_t N, int p, int q, int same, size_t* bytes);
QSB_API qsb_status qsb_gram_ozaki_int8(qsb_dtype dtype, int64_t N, int p, int q, const void* U, const void* V,
                                       double* T, int ldt, int upper, void* workspace, size_t workspace_bytes,
                                       void* stream);

/* Rotation OUT = U C (the NextVector_z2 / NextVector products,
 * source/lobpcg_z_multi_mpi.h:1515-1598) on the INT8 tensor cores: U (N x K,
 * column-major ld N, fp32 or fp64) split as in qsb_gram_ozaki_int8, C (K x q,
 * FP64, device, ld K) scaled by U's column exponents and split per output
 * column; OUT: N x q fp32, ld N.  Element error ~2^-20 of max|u| |c| per term
 * (round-to-nearest slices, exact integer accumulation). */
QSB_API qsb_status qsb_rotate_ozaki_int8_workspace(int64_t N, int K, int q, size_t* bytes);
QSB_API qsb_status qsb_rotate_ozaki_int8(qsb_dtype dtype, int64_t N, int K, int q, const void* U, const double* C,
                                         float* out, void* workspace, size_t workspace_bytes, void* stream);

/* Per-kernel device timing of qsb_ham_apply, in the spirit of the reference's
 * StopWatch sectors (source/StopWatch.h:11-60, watch_pp in
 * source/PseudoPotNonlocal_SvF2_kpoint.h:261-272).  While enabled, every
 * qsb_ham_apply records CUDA events on its stream around its three phases:
 * the nonlocal projection, the FD8 + V stencil, and the nonlocal expansion.
 * qsb_ham_get_timing synchronizes those events, returns the summed
 * milliseconds of each phase, the number of applies and of kernel launches
 * since the last call, and resets the counters. */
QSB_API qsb_status qsb_ham_set_timing(qsb_ham* ham, int enable);
QSB_API qsb_status qsb_ham_get_timing(qsb_ham* ham, double* project_ms, double* stencil_ms, double* expand_ms,
                                      int* applies, int* kernel_launches);

/* ---------------------------------------------------------------------------
 * Self-consistent field on the device (Gamma point, spin-unpolarised, LDA).
 *
 * Building blocks:
 *   qsb_density  rho = sum_n occ_n psi_n^2 over a real bundle (n x N, device;
 *                occupations on the host).  Replaces mSetDensityByPsi /
 *                SetDensityOne (source/qumasun_base1.density.h:19-105,
 *                source/qumasun_SetDensityOne.h).
 *   qsb_lda_pz   Perdew-Zunger LDA per point: exc = rho eps_xc (may be NULL),
 *                vxc = V_x + V_c; zero below rho = 1e-8.  Replaces Calc_XC_LDA
 *                (source/Vxc.h:43-75) as mSetPotentialVxc uses it.
 *
 * Driver (the loop of QUMASUN_KPOINT::Execute, source/qumasun_kpoint.scfloop.h:61-230,
 * with LOBPCG as the solver): per step V_eff = V_loc + V_H[rho_in] + V_xc[rho_in]
 * goes into the qsb_ham, qsb_lobpcg_d runs lobpcg_iters iterations on X (the
 * solver's precision decides FP64 or mixed), FP64 Rayleigh quotients of X give
 * the Fermi-Dirac occupations (bisection of mSetOccupancyTemperature,
 * source/qumasun_base1.occupancy.h:76-170, kbT set by qsb_scf_set_smearing,
 * default 0.01 Ha) and the output density, the Kohn-Sham energy of the output
 * density E = sum occ e - int (V_H + V_xc)[rho_in] rho_out + E_H + E_xc [rho_out]
 * (ion-ion term excluded: a constant) is recorded, and the run stops when
 * |dE| / atom < tol_per_atom; otherwise Kerker-preconditioned DIIS (depth, A,
 * q0 of qsb_scf_set_mixing; default 6, 0.5, 0.8 bohr^-1) gives the next rho_in.
 * The first density is that of the input X with the lowest bands doubly
 * filled (mSetOccupancyZero's filling).  V_loc: analytic GTH local parts,
 * qsb_scf_set_gth_local (per-species arrays indexed by species[atom]).
 * energies: host, max_steps values; eigen_values / occupations: host, nb
 * values (may be NULL).  qsb_scf_get_field copies rho_out (0), V_loc (1),
 * V_eff (2) or the mixed input density (3) to a device buffer of N doubles.
 * --------------------------------------------------------------------------- */
typedef struct qsb_scf qsb_scf;
QSB_API qsb_status qsb_density(int64_t N, int nb, const double* X, const double* occupations, double* rho,
                               void* stream);
QSB_API qsb_status qsb_lda_pz(int64_t n, const double* rho, double* exc, double* vxc, void* stream);
QSB_API qsb_status qsb_scf_create(qsb_scf** scf, qsb_ham* ham, qsb_eigensolver* es, int nb, double num_electrons);
QSB_API qsb_status qsb_scf_destroy(qsb_scf* scf);
QSB_API qsb_status qsb_scf_set_gth_local(qsb_scf* scf, int n_atoms, const double* pos, const int* species,
                                         int n_species, const double* zion, const double* rloc, const double* c1,
                                         const double* c2);
/* Local parts from radial tables instead of the analytic GTH form (replaces a
 * qsb_scf_set_gth_local; the last call of the two decides): per species k the
 * table v_k(G) of qsb_radial_local_table (n_g values on |G| = j dg, computed
 * with charge z[k] and Gaussian width sigma[k] -- for a UPF, its radius,
 * v_local and z_valence), V_loc(G) = (1/Omega) sum_a v_{species[a]}(|G|)
 * exp(-i G.R_a).  The smooth part v + 4 pi z exp(-G^2 sigma^2 / 2) / G^2 is
 * interpolated (cubic, four nearest samples) and the Gaussian charge's term is
 * added back exactly, so the 1/G^2 tail is not interpolated.  The table must
 * reach |G| = sqrt(sum_d (pi / h_d)^2) with three samples to spare.
 * qsb_scf_local_forces then returns the force of these local parts.  The
 * reference builds its local potential from core charges by a Poisson solve
 * on a finer grid (source/qumasun_base1.core.h:54,139, upf_oncv_loader.h:337);
 * this is the G-space route of the same potential. */
QSB_API qsb_status qsb_scf_set_radial_local(qsb_scf* scf, int n_atoms, const double* pos, const int* species,
                                            int n_species, const double* z, const double* sigma, int n_g, double dg,
                                            const double* table);
QSB_API qsb_status qsb_scf_set_mixing(qsb_scf* scf, double amplitude, double q0, int depth);
QSB_API qsb_status qsb_scf_set_smearing(qsb_scf* scf, double kbt);
/* The SCF's LDA.  pz_variant 0 (default): Perdew-Zunger with the published
 * constants, as Calc_XC_LDA (source/Vxc.h:43-75) has them; its two correlation
 * branches miss each other at rs = 1 by 3.2e-5 Ha in eps_c, so the energy
 * jumps by (3 / 4 pi) dV 3.2e-5 Ha whenever a grid point's density crosses
 * 3 / (4 pi) -- as atoms move, central differences of the energy see these
 * steps.  pz_variant 1: the high-density branch's C and D solved from value
 * and slope continuity at rs = 1 (C = 0.0020191519, D = -0.0116320664; A, B
 * and the low-density branch unchanged), which leaves the energy a smooth
 * function of the positions.  rho_min (default 1e-8, Calc_XC_LDA's cut,
 * >= 1e-30): exc = vxc = 0 below it.  pz_variant 2: GGA-PBE instead
 * (spin-unpolarised, as qsb_gga_pbe; rho_min not used). */
QSB_API qsb_status qsb_scf_set_xc(qsb_scf* scf, int pz_variant, double rho_min);
/* GGA-PBE exchange-correlation of a spin-unpolarised density on an
 * nx x ny x nz periodic grid (device arrays of N doubles; exc may be NULL):
 * exc = the energy density (E_xc = dV sum exc), vxc = the potential
 * v_x + v_c - 2 div(P_x grad rho_s) - 2 div(P_c grad rho), gradients and
 * divergences by the eighth-order central difference.  Replaces the GGA branch
 * of QUMASUN_BASE1::mSetPotentialVxc (source/qumasun_base1.potential.h:383-470,
 * 585-640, XC_IMPLE_VER2) with GGA_PBE::Potential_X_test3 and
 * EnergyDensityPotential_C_test3 (source/xc_gga_pbe.h:326-356, 525-594):
 * exchange per spin channel on rho / 2, correlation on rho, PW92 local part,
 * densities below 1e-8 contributing nothing.  Allocates 3 N doubles of
 * scratch per call and synchronizes the stream. */
QSB_API qsb_status qsb_gga_pbe(int nx, int ny, int nz, double dx, double dy, double dz, const double* rho,
                               double* exc, double* vxc, void* stream);
/* Also require int |rho_out - rho_in| dV / N_e < rho_tol to stop (the
 * reference's RHO_ETOT convergence mode, source/qumasun_kpoint.scfloop.h:182-213);
 * 0 (default) stops on the energy alone. */
QSB_API qsb_status qsb_scf_set_density_tolerance(qsb_scf* scf, double rho_tol);
/* FP64 polish of a mixed-precision run: once the run meets its own stop
 * (|dE| / atom below qsb_scf_run's tol and, if set, the density tolerance) the
 * loop goes on with es_fp64 -- a real QSB_PREC_FP64 solver context of the
 * SCF's grid and at least its bands -- from the mixed run's states and mixed
 * density, for at most max_steps further steps (counted within qsb_scf_run's
 * max_steps), until |dE| / atom < tol_per_atom (0: the run's tol) and
 * int |rho_out - rho_in| dV / N_e < rho_tol (0: the energy alone).  The first
 * FP64 call starts without the kept search directions (P = 0, the [X R]
 * pencil), as at an SCF's first step.  FP32 rounding in the mixed solver's
 * states sets a floor under its density residual (~1e-8 N_e) and so under its
 * force error; the polish takes the end point to the FP64 one.  es_fp64 = NULL
 * or max_steps = 0 switches the polish off (the default).  No counterpart in
 * the reference (its solver has one precision). */
QSB_API qsb_status qsb_scf_set_polish(qsb_scf* scf, qsb_eigensolver* es_fp64, int max_steps, double tol_per_atom,
                                      double rho_tol);
/* Of the last qsb_scf_run: index of the first FP64 polish step (-1: none) and
 * how many polish steps ran. */
QSB_API qsb_status qsb_scf_polish_stats(const qsb_scf* scf, int* first_step, int* steps);
QSB_API qsb_status qsb_scf_run(qsb_scf* scf, double* X, double* keep, int lobpcg_iters, int max_steps,
                               double tol_per_atom, double* energies, int* steps, double* eigen_values,
                               double* occupations, void* stream);
QSB_API qsb_status qsb_scf_get_field(qsb_scf* scf, int which, double* out);
/* Force of the local parts (GTH, or radial tables) on every atom, -d/dR_a int rho V_loc, from the
 * last output density (rho_dev = NULL) or a given device density: forces
 * (host, 3 x n_atoms) accumulate ("+="), so the nonlocal part
 * (qsb_ham_nonlocal_energy_force) adds on.  Exact derivative of the grid sum
 * dV sum rho V_loc (V_loc's Fourier series).  Replaces the local-potential
 * terms of the reference's mGetForce (source/qumasun_base1.force.h:23-205;
 * mGetForceOnNuclRho_HR :247-284 on its core-charge form of V_loc). */
QSB_API qsb_status qsb_scf_local_forces(qsb_scf* scf, const double* rho_dev, double* forces);
/* Ion-ion energy of point charges (the GTH Z_ion, host arrays) in the
 * orthorhombic cell cell[3] (bohr) with a neutralising background, by Ewald
 * summation (alpha = 5 / min(L), sums cut at 1e-16); forces (host, 3 x n_atoms,
 * may be NULL) accumulate ("+=").  Host code, no device work.  The ion-ion
 * term of the reference's total energy and force (mGetForce's nuclear part,
 * source/qumasun_base1.force.h:23-205). */
QSB_API qsb_status qsb_ewald(int n_atoms, const double* pos, const double* charge, const double* cell,
                             double* energy, double* forces);
/* Geometry relaxation by LBFGS on the free energy E - kBT S + E_ewald, forces
 * local + nonlocal + Ewald.  Replaces the relaxation drivers
 * glips::Relaxation1Q..4Q::Evolve (source/Relaxation1.h:45-190) as the
 * reference's SCF/relax loop uses them.  Each evaluation moves the projectors
 * (qsb_ham_set_gth_projectors with nl, r_l, h_l, rcut_factor) and the local
 * parts (qsb_scf_set_gth_local with zion, rloc, c1, c2) to the positions and
 * runs qsb_scf_run(X, keep, lobpcg_iters, scf_max_steps, scf_tol) warm from
 * the previous states.  Steps: two-loop recursion over the last `history`
 * pairs (initial scale s.y / y.y; 1 bohr^2/Ha before any pair), capped at
 * max_step bohr per atom, halved (up to 5 times) while the energy rises by
 * more than 10 scf_tol per atom (the SCF energies' own error).
 * fixed (may be NULL): atoms with fixed[a] != 0 do not move.  Stops at
 * max_a |F_a| < fmax or after max_iter steps.  pos (host) returns the last
 * geometry, energies (host, max_iter + 1 values) the energy after each
 * step (index 0: the start), *iters the steps taken, forces (host, may be
 * NULL) the last forces. */
QSB_API qsb_status qsb_relax_lbfgs(qsb_scf* scf, int n_atoms, double* pos, const int* species, int n_species,
                                   const int* nl, const double* r_l, const double* h_l, double rcut_factor,
                                   const double* zion, const double* rloc, const double* c1, const double* c2,
                                   const int* fixed, double* X, double* keep, int lobpcg_iters, int scf_max_steps,
                                   double scf_tol, int max_iter, double fmax, double max_step, int history,
                                   double* energies, int* iters, double* forces, void* stream);
/* k-point SCF (complex Bloch bands): the loop of QUMASUN_KPOINT::Execute over
 * its k groups (source/qumasun_kpoint.scfloop.h:61-258, the solver calls of
 * qumasun_kpoint.lobpcg.h:78-106) with the density summed over k
 * (mSetDensityByPsi, source/qumasun_base1.density.h:19-105) and the Fermi level
 * found over all (k, band) levels with the k weights.  Needs a complex solver
 * context (either precision) given to qsb_scf_create.
 *   qsb_scf_set_kpoints: kvec 3 n_k Bloch vectors (bohr^-1), weights n_k (> 0,
 *     summing to 1), owned (may be NULL: all) marks the k-points this context
 *     computes; with several contexts (one per GPU, or per rank) sharing a k
 *     list, each owns a part and qsb_scf_set_reduce joins them.
 *   qsb_scf_set_reduce: fn(user, buf, count) must replace the host buffer buf
 *     of count doubles by its sum over all contexts sharing the k-points (an
 *     allreduce) and return 0; called with the same sizes in the same order on
 *     every context, twice per step (the levels, n_k nb; the density, N) and
 *     once before the first (the starting density).  NULL: one context.
 *   qsb_scf_run_kpoints: X[k], keep[k] device complex SoA bundles of nb bands
 *     (owned k only; others may be NULL), updated in place; per step every owned
 *     k-point gets lobpcg_iters solver iterations at its Bloch vector (no soft
 *     locking), FP64 Rayleigh quotients of its bands, the occupations f_nk in
 *     [0, 2] from the weighted Fermi level (sum_k w_k sum_n f_nk = N_e), the
 *     output density sum_k w_k sum_n f_nk |psi_nk|^2, the energy as in qsb_scf_run
 *     with the band energy sum_k w_k sum_n f_nk e_nk; stop and mixing as there
 *     (the FP64 polish does not apply).  eigen_values, occupations: host, n_k x nb
 *     (k-major, may be NULL), all k-points after the reduction. */
typedef int (*qsb_reduce_fn)(void* user, double* buf, int64_t count);
QSB_API qsb_status qsb_scf_set_kpoints(qsb_scf* scf, int n_k, const double* kvec, const double* weights,
                                       const int* owned);
QSB_API qsb_status qsb_scf_set_reduce(qsb_scf* scf, qsb_reduce_fn fn, void* user);
QSB_API qsb_status qsb_scf_run_kpoints(qsb_scf* scf, double* const* X, double* const* keep, int lobpcg_iters,
                                       int max_steps, double tol_per_atom, double* energies, int* steps,
                                       double* eigen_values, double* occupations, void* stream);
/* Fermi-Dirac occupations of n levels (host code): occ_i = 2 / (exp((e_i - mu) / kbt) + 1)
 * with mu such that sum_i w_i occ_i = n_el (weights NULL: all 1) -- the bisection
 * of mSetOccupancyTemperature (source/qumasun_base1.occupancy.h:76-170) with
 * SetOccupancy's formula (source/SetOccupancy.h:7-18), refined by Newton steps to
 * the exact count.  mu may be NULL. */
QSB_API qsb_status qsb_fermi_occupations(int n, const double* eig, const double* weights, double n_el, double kbt,
                                         double* occ, double* mu);
/* Wall seconds of each step of the last qsb_scf_run (host clock; a step ends
 * when its energy is on the host): up to max values, *n = steps recorded. */
QSB_API qsb_status qsb_scf_step_seconds(qsb_scf* scf, double* seconds, int max, int* n);
/* Density residual int |rho_out - rho_in| dV / N_e of each step of the last
 * qsb_scf_run (the quantity of qsb_scf_set_density_tolerance), up to max
 * values; *n = steps recorded. */
QSB_API qsb_status qsb_scf_step_residuals(qsb_scf* scf, double* residuals, int max, int* n);

/* ---------------------------------------------------------------------------
 * UPF (v2, ONCV norm-conserving) pseudopotentials (host code; no device work).
 * qsb_upf_load reads the radial data LoadUPF_ONCV keeps
 * (source/upf_oncv_loader.h:353-520): per radial projector k its l_k, E_k =
 * D_kk / 2 (Ha) and beta_k(r) = (r beta_k)(r) / r resampled onto the log grid
 * r_i = exp(xi_min + i xi_delta), i < n_grid (xi_min = -9, 1000 points up to
 * the UPF mesh's end) with the reference's quintic uniform-grid interpolant;
 * cutoff_l[l] = the largest cutoff_radius of channel l; v_local: the UPF's
 * PP_LOCAL with its tail blended into -2 Z_v / r past the local cutoff, as the
 * reference corrects it (ONCV_CORRECT_VLOCAL 11, upf_oncv_loader.h:803-921,
 * 1022-1026), resampled the same way (Ha).
 * qsb_upf_grid_tables builds the tables qsb_ham_set_projectors and
 * qsb_ham_set_projector_gradients take: beta_k(|r - R|) Y_lm(r - R) (real
 * harmonics, m = -l..l) on the grid points within the atom's largest cutoff,
 * E_k per column, and the analytic gradient tables.  (The reference's own
 * grid construction, the SvF2 filter of PseudoPotNonlocal_SvF2_kpoint.h:911-1180,
 * goes through FFTW; this one samples directly.)  Atoms with more than 16
 * projector columns are split into table entries of whole radial projectors at
 * the same position; entry_atom[e] is the atom of entry e (H psi is a sum over
 * entries; per-entry nonlocal forces add up to the atom's).
 * Call once with entry_atom (or any output array) NULL for the sizes:
 * n_entries, n_points (sum of npts), n_values (sum of npts * widths); then with
 * entry_atom / npts / widths [n_entries], coords [3 n_points], beta [n_values],
 * energy [sum of widths <= 16 n_entries], dbeta [3 n_values] (may be NULL). */
typedef struct qsb_upf qsb_upf;
QSB_API qsb_status qsb_upf_load(qsb_upf** upf, const char* path);
QSB_API qsb_status qsb_upf_destroy(qsb_upf* upf);
/* cutoff_l[4]; xi_min_delta[2]; any output may be NULL */
QSB_API qsb_status qsb_upf_info(const qsb_upf* upf, int* n_projectors, double* z_valence, int* n_grid,
                                double* cutoff_l, double* xi_min_delta);
/* radius, v_local [n_grid]; l, energy [n_projectors]; projectors [n_projectors x n_grid]; any may be NULL */
QSB_API qsb_status qsb_upf_radial(const qsb_upf* upf, double* radius, double* v_local, int* l, double* energy,
                                  double* projectors);
/* Fourier transform of a radial local potential (Ha) with Coulomb tail -z/r,
 * v(G) = int V(r) exp(-i G.r) d^3r, on G = j dg, j < n_g, in the convention of
 * the SCF driver's GTH local part: for G > 0 the full transform (its
 * -4 pi z / G^2 included), at G = 0 the finite part lim (v(G) + 4 pi z / G^2).
 * Computed as 4 pi int r^2 [V + z erf(r / (sqrt2 sigma)) / r] j0(G r) dr
 * (Simpson in ln r on the log grid radius[n_r]) minus the Gaussian charge's
 * 4 pi z exp(-G^2 sigma^2 / 2) / G^2 (2 pi z sigma^2 at G = 0); the result
 * does not depend on sigma.  For a UPF: radius and v_local of qsb_upf_radial,
 * z = z_valence.  (The reference forms its local potential from core charges
 * by a Poisson solve on a finer grid, source/qumasun_base1.core.h; this table
 * is the G-space route the SCF driver takes.) */
QSB_API qsb_status qsb_radial_local_table(int n_r, const double* radius, const double* v, double z, double sigma,
                                          int n_g, double dg, double* table);
QSB_API qsb_status qsb_upf_grid_tables(const qsb_upf* const* upf, int n_species, int n_atoms, const double* pos,
                                       const int* species, double dx, double dy, double dz, int* n_entries,
                                       int64_t* n_points, int64_t* n_values, int* entry_atom, int* npts,
                                       int* widths, int* coords, double* beta, double* energy, double* dbeta);

/* ---------------------------------------------------------------------------
 * Cube files (host code; no device work).  The reference's state and density
 * exchange format: files written by qsb_cube_write are byte-identical to those
 * of CubeWriter::SaveCube (source/cube_writer.h:27-90; title "Generated by
 * QUMASUN", the same printf formats, values z fastest, 6 per line, each z row
 * ending its line), and qsb_cube_read returns the values CubeReader3::LoadCube
 * + GetMeshData (source/cube_reader3.h:38-124) return, in this library's grid
 * layout (x fastest).  Where the reference reader silently stops on a short or
 * malformed file, these return QSB_ERR_INVALID with the counts found.
 *   axis[9]    the three box edge vectors (grid count x voxel vector), bohr
 *   origin[3]  the volume origin, bohr
 *   Z, pos     n_atoms atomic numbers and positions (3 per atom)
 *   field      nx*ny*nz doubles, host memory, x fastest
 * The comment is one line.  Rows are formatted / parsed by up to 16 host
 * threads. */
QSB_API qsb_status qsb_cube_write(const char* path, const char* comment, int nx, int ny, int nz,
                                  const double* axis, const double* origin, int n_atoms, const int* Z,
                                  const double* pos, const double* field);
/* grid[3] out; axis, origin, n_atoms may be NULL. */
QSB_API qsb_status qsb_cube_read_header(const char* path, int* grid, double* axis, double* origin, int* n_atoms);
/* field (grid product doubles) out; Z (n_atoms ints) and pos (3 n_atoms) may be NULL. */
QSB_API qsb_status qsb_cube_read(const char* path, double* field, int* Z, double* pos);

#ifdef __cplusplus
}
#endif
#endif /* QUMASUN_B200_H */
