/*
 * cytnx_b200 -- C ABI of the B200-native tensor-network hot path.
 *
 * Plain C types only (pointers, sizes, status codes).  Every entry point that
 * touches the GPU takes an explicit cudaStream_t (passed as void*; NULL = the
 * legacy default stream) and never synchronises the device unless stated.
 * Device buffers are owned by the caller.  On failure a call returns a
 * non-zero ctn_status and ctn_last_error() holds a message for the calling
 * thread; nothing ever resets the device or exits the process.
 *
 * Reference interfaces replaced (Cytnx 1.1.1 source tree):
 *   ctn_permute / ctn_permute_blocks
 *       utils_internal::MoveMemoryGpu(in, old_shape, mapper, invmapper, inplace)
 *       src/backend/utils_internal_gpu/cuMovemem_gpu.cu:289-304, reached from
 *       StorageImplementation<T>::Move_memory (src/backend/StorageImplementation.cpp:144-176)
 *       and Tensor_impl::contiguous (include/backend/Tensor_impl.hpp:222-279).
 *   ctn_blocks_enumerate
 *       BlockUniTensor::Init block enumeration, src/BlockUniTensor.cpp:190-230,
 *       flux rule include/UniTensor.hpp:1139-1165.
 *   ctn_contract_plan_create / ctn_contract_execute
 *       BlockUniTensor::contract, src/BlockUniTensor.cpp:777-1235 (block pairing
 *       :994-1006, per-pair Matmul/Gemm_Batch :1114-1223), i.e. the dtype tables
 *       lii.cuMatmul_ii / cuGemm_Batch_ii (src/backend/linalg_internal_interface.hpp:203-239).
 *   ctn_gemm_grouped_f64
 *       linalg::Gemm_Batch (src/linalg/Gemm_Batch.cpp:14-236; GPU loop of cublasDgemm
 *       src/backend/linalg_internal_gpu/cuGemm_Batch_internal.cu:10-65).
 *   ctn_dot_f64 / ctn_nrm2_f64 / ctn_lanczos_update_f64
 *       linalg::Vectordot / Norm / the elementwise Sub/Mul used by Lanczos
 *       (cuVectordot_internal.cu:133-160, cuNorm_internal.cu:14-27,
 *        cuArithmeticDispatch.cuh:57-90).
 *   ctn_tridiag_eigh
 *       linalg::Tridiag (src/linalg/Tridiag.cpp:10-104; LAPACKE_dstev in
 *       src/backend/linalg_internal_cpu/Tridiag_internal.cpp:9-42).
 *   ctn_heff2_*
 *       the two-site effective-Hamiltonian matvec that example/DMRG/dmrg_two_sites_U1.py:18-23
 *       runs through Network::Launch (src/RegularNetwork.cpp:901-1007) inside
 *       LinOp::matvec (include/LinOp.hpp:163-167).
 *   ctn_lanczos_gnd
 *       linalg::Lanczos(..., method="Gnd") -> Lanczos_Gnd_Ut
 *       (src/linalg/Lanczos_Gnd_Ut.cpp:29-199).
 *   ctn_lanczos_exp
 *       linalg::Lanczos_Exp (src/linalg/Lanczos_Exp.cpp:264-453).
 *   ctn_lanczos_which / ctn_sym_eigh
 *       linalg::Lanczos(Hop, Tin, which = "SA" / "LA" / "LM", maxiter, cvg_crit, k, is_V, ncv)
 *       (src/linalg/Lanczos.cpp:250-402: ARPACK dsaupd/dseupd).
 */
#ifndef CYTNX_B200_H
#define CYTNX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int ctn_status;
enum {
  CTN_OK = 0,
  CTN_ERR_INVALID = 1,     /* bad argument / shape / label mismatch */
  CTN_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  CTN_ERR_UNSUPPORTED = 3, /* dtype / rank / precision not handled */
  CTN_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  CTN_ERR_NUMERIC = 5      /* non-finite value or breakdown in a solver */
};

/* dtype ids are the reference's Type list indices (include/Type.hpp:177-179) */
enum {
  CTN_COMPLEX128 = 1,
  CTN_COMPLEX64 = 2,
  CTN_FLOAT64 = 3,
  CTN_FLOAT32 = 4,
  CTN_INT64 = 5,
  CTN_UINT64 = 6,
  CTN_INT32 = 7,
  CTN_UINT32 = 8,
  CTN_INT16 = 9,
  CTN_UINT16 = 10,
  CTN_BOOL = 11
};

/* arithmetic forms of the block GEMMs */
enum {
  CTN_PREC_F64 = 0,    /* plain FP64 (the drop-in form) */
  CTN_PREC_3XTF32 = 1, /* split: a = hi + lo in TF32, 3 tensor-core products, FP32 accumulate */
  CTN_PREC_BF16X3 = 2  /* split: a = hi + lo in BF16, 3 tensor-core products, FP32 accumulate */
};

const char *ctn_last_error(void);
int ctn_version(void);
/* element size in bytes of a dtype id, 0 if unknown */
size_t ctn_dtype_size(int dtype);

/* ---------------------------------------------------------------- permute
 * dst[new] = src[old] with new_shape[i] = old_shape[mapper[i]] (row-major);
 * bit-exact for every dtype.  rank <= 16.  src and dst must not overlap. */
ctn_status ctn_permute(const void *src, void *dst, int dtype, int rank, const uint64_t *old_shape,
                       const uint64_t *mapper, void *stream);

/* the same permutation applied to nblocks blocks in one launch sequence;
 * block b has shape old_shapes[b*rank .. b*rank+rank) and lives at element
 * offsets src_offs[b] / dst_offs[b]. */
ctn_status ctn_permute_blocks(const void *src, void *dst, int dtype, int rank, int64_t nblocks,
                              const uint64_t *old_shapes, const int64_t *src_offs,
                              const int64_t *dst_offs, const uint64_t *mapper, void *stream);

/* ---------------------------------------------------------------- blocks
 * Enumerate the symmetry-allowed blocks of a tensor with `rank` bonds.
 * sym_types[s]: -1 = U1, 0 = Zn (with modulus sym_n[s]); bond_types[i]: -1 ket, +1 bra;
 * qnums[i] points to bond i's table [nqs[i]][nsym].  Tuples go to out_itoi
 * ([capacity][rank], last leg fastest); *out_count receives the count. */
ctn_status ctn_blocks_enumerate(int rank, int nsym, const int32_t *sym_types, const int64_t *sym_n,
                                const int32_t *bond_types, const int64_t *nqs,
                                const int64_t *const *qnums, int64_t *out_itoi, int64_t capacity,
                                int64_t *out_count);

/* ---------------------------------------------------------------- contract
 * Host description of a block-sparse operand.  Blocks are dense row-major in
 * their *physical* leg order; `perm` (length rank) maps logical leg i to
 * physical leg perm[i] (the lazy permutation of Tensor_impl's _mapper); NULL
 * means identity.  shapes are logical. */
typedef struct {
  int32_t rank;
  int64_t nblocks;
  const int64_t *itoi;   /* [nblocks][rank] logical qnum-index tuples */
  const int64_t *shapes; /* [nblocks][rank] logical block shapes */
  const int64_t *offs;   /* [nblocks] element offsets into the tensor storage */
  const int64_t *perm;   /* [rank] or NULL */
} ctn_block_desc;

typedef struct ctn_contract_plan ctn_contract_plan;

/* comm_l[i] / comm_r[i]: logical leg indices of the i-th common label (sorted by
 * label, as vec_intersect_ returns them).  `out` describes the output blocks in
 * the order BlockUniTensor::Init enumerates them (legs = noncomm(L) ++ noncomm(R),
 * perm must be NULL). */
ctn_status ctn_contract_plan_create(const ctn_block_desc *L, const ctn_block_desc *R, int ncomm,
                                    const int64_t *comm_l, const int64_t *comm_r,
                                    const ctn_block_desc *out, ctn_contract_plan **plan);
/* device bytes the plan needs as scratch (permuted operand copies + task tables) */
size_t ctn_contract_plan_scratch_bytes(const ctn_contract_plan *plan);
/* flops of the planned block GEMMs (2*m*n*k summed over block pairs) */
double ctn_contract_plan_flops(const ctn_contract_plan *plan);
/* run: out blocks that receive no pair are zero-filled; scratch >= scratch_bytes. */
ctn_status ctn_contract_execute(ctn_contract_plan *plan, int dtype, const void *L, const void *R,
                                void *out, void *scratch, void *stream);
void ctn_contract_plan_destroy(ctn_contract_plan *plan);

/* ---------------------------------------------------------------- grouped GEMM
 * C_t = sum_p op(A_p) op(B_p) for every task t (row-major, FP64, DMMA).
 * Each task: {c_off, m, n, ldc, pair_begin, pair_count}; a task with no pair
 * writes zeros.  Each pair: {a_off, b_off, k, lda, ldb, flags} with flags bit0:
 * A stored [k][m] (transposed), bit1: B stored [n][k].  Offsets are elements
 * from the A/B/C base pointers given at execution; all pairs of one plan share the
 * same flags (execution returns CTN_ERR_UNSUPPORTED otherwise).  The plan copies the tables
 * to the device on its first execution on a device (run that first call before
 * any stream capture). */
typedef struct {
  int64_t c_off;
  int32_t m, n, ldc;
  int32_t pair_begin, pair_count;
  int32_t pad_;
} ctn_gemm_task;
typedef struct {
  int64_t a_off, b_off;
  int32_t k, lda, ldb, flags;
} ctn_gemm_pair;
typedef struct ctn_gemm_plan ctn_gemm_plan;
ctn_status ctn_gemm_grouped_plan_create(int64_t ntasks, const ctn_gemm_task *tasks, int64_t npairs,
                                        const ctn_gemm_pair *pairs, ctn_gemm_plan **plan);
double ctn_gemm_grouped_plan_flops(const ctn_gemm_plan *plan);
ctn_status ctn_gemm_grouped_f64(ctn_gemm_plan *plan, const double *A, const double *B, double *C,
                                void *stream);
void ctn_gemm_grouped_plan_destroy(ctn_gemm_plan *plan);

/* ---------------------------------------------------------------- split-precision GEMM
 * C[M][N] (FP64, row-major) = A[M][K] B[K][N] (FP64, row-major) on the tcgen05 tensor
 * cores: operands split as x = hi + lo (TF32 for CTN_PREC_3XTF32, BF16 for
 * CTN_PREC_BF16X3), products lo*hi + hi*lo + hi*hi accumulated in FP32 (TMEM).
 * workspace >= ctn_split_gemm_workspace_bytes(M, N, K, precision) device bytes.
 * Synchronises the stream (reads back the kernel's error word). */
size_t ctn_split_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int precision);
ctn_status ctn_split_gemm_f64(int64_t M, int64_t N, int64_t K, const double *A, const double *B, double *C,
                              int precision, void *workspace, void *stream);

/* Allocation-free form of ctn_split_gemm_f64 for callers that cannot allocate device
 * memory (programs whose device memory is owned by their own pool, fixed memory
 * budgets, foreign-language callers without a device allocator).  No counterpart in
 * the reference.  Scratch lives in a 32 MiB static device array held by every GPU
 * that loads the library until exit; problems needing more are rejected with
 * CTN_ERR_INVALID.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress) and should come before any stream capture; the address is kept
 * for the process, so a device reset afterwards is not supported.  All calls share
 * the array: calls that overlap on the GPU race, so serialise them.  Synchronises
 * the stream. */
ctn_status ctn_split_gemm_f64_noalloc(int64_t M, int64_t N, int64_t K, const double *A, const double *B, double *C,
                                      int precision, void *stream);

/* Self-test of the bounded-wait error path of the tcgen05 GEMM: one 128 x 128 x 128 split GEMM
 * whose producer issues no copies, so the MMA warp's wait for its first operand stage runs out
 * after `spin_limit` probes; the kernel records the error, stops its other roles, frees its
 * TMEM and returns.  Returns CTN_ERR_TIMEOUT (with the code of the wait in ctn_last_error())
 * when that path works; the context stays usable.  Allocates a small device buffer.
 * Synchronises the stream.  No counterpart in the reference (its kernels do not wait). */
ctn_status ctn_selftest_wait_timeout(int precision, long long spin_limit, void *stream);

/* Self-test of the bounded grid barrier of the fused Krylov step of ctn_lanczos_refined:
 * one cooperative launch on a 16384-element vector whose barrier waits for an arrival that
 * never comes, so every CTA's wait runs out after `spin_limit` probes (about 64 ns each) and
 * raises the error word.  Returns CTN_ERR_TIMEOUT when that path works (CTN_ERR_UNSUPPORTED
 * without cooperative launch); the context stays usable.  Allocates a small device buffer and
 * synchronises the stream.  No counterpart in the reference. */
ctn_status ctn_selftest_barrier_timeout(long long spin_limit, void *stream);

/* ---------------------------------------------------------------- BLAS-1 (FP64)
 * Results of reductions land in device memory (out points to device doubles). */
ctn_status ctn_dot_f64(const double *x, const double *y, int64_t n, double *out, void *stream);
ctn_status ctn_nrm2_f64(const double *x, int64_t n, double *out, void *stream);
/* y = a*x + y with a read from device memory (a_dev) times a_scale */
ctn_status ctn_axpy_f64(const double *x, double *y, int64_t n, const double *a_dev, double a_scale,
                        void *stream);
ctn_status ctn_scal_f64(double *x, int64_t n, const double *a_dev, int invert, void *stream);

/* symmetric tridiagonal eigensolver (host, FP64): d[n] diagonal, e[n-1] off-diagonal.
 * Eigenvalues ascending into w[n]; if z != NULL the eigenvectors as rows of z[n][n]. */
ctn_status ctn_tridiag_eigh(int n, const double *d, const double *e, double *w, double *z);
/* dense symmetric eigenproblem (host, cyclic Jacobi): a n x n row-major, w eigenvalues in
 * no particular order, z n x n row-major with the eigenvectors as columns.  The projected
 * matrix solve of ctn_lanczos_which (the reference calls LAPACK inside ARPACK dseupd). */
ctn_status ctn_sym_eigh(int n, const double *a, double *w, double *z);

/* ---------------------------------------------------------------- two-site H_eff
 * Plan for out = H_eff psi with the network of example/DMRG/dmrg_two_sites_U1.py:
 *   psi[a,s1,s2,b]  L[w,a,a']  M1[w,w1,s1,s1']  M2[w1,w2,s2,s2']  R[w2,b,b']
 *   out[a',s1',s2',b'] = sum L M1 M2 R psi   (order L -> M1 -> M2 -> R).
 * Each leg is given as its sector degeneracies and its charge indices into a
 * shared charge table; blocks of psi/L/R are described by ctn_block_desc
 * (identity perm, blocks in enumeration order).  M1/M2 are given densely per
 * block (they are tiny).  See cytnx_b200/heff.py for the host-side builder. */
typedef struct ctn_heff2_plan ctn_heff2_plan;
typedef struct {
  const ctn_block_desc *psi, *L, *R, *M1, *M2, *out;
  const double *M1_host, *M2_host; /* block data of the MPO tensors (host, block order) */
} ctn_heff2_desc;
ctn_status ctn_heff2_plan_create(const ctn_heff2_desc *desc, ctn_heff2_plan **plan);
double ctn_heff2_flops(const ctn_heff2_plan *plan);
size_t ctn_heff2_psi_elems(const ctn_heff2_plan *plan);
size_t ctn_heff2_workspace_bytes(const ctn_heff2_plan *plan, int precision);
/* bind the (fixed) environments: device pointers to L and R storage (FP64).
 * For split precisions this converts them once into the split operand layout. */
ctn_status ctn_heff2_set_env(ctn_heff2_plan *plan, const double *L, const double *R,
                             void *workspace, int precision, void *stream);
ctn_status ctn_heff2_matvec(ctn_heff2_plan *plan, const double *psi, double *out, int precision,
                            void *stream);
/* measurement aid: run `reps` matvecs with CUDA events between the phases on
 * `stream`; ms_out[0..3] receive the median over the repetitions of the device time of operand packing (split
 * forms only, 0 for FP64), step 1 (grouped GEMM), steps 2+3 (MPO combination) and
 * step 4 (grouped GEMM); launches_out the number of kernel launches one matvec issues. */
ctn_status ctn_heff2_profile(ctn_heff2_plan *plan, const double *psi, double *out, int precision, int reps,
                             double *ms_out, int *launches_out, void *stream);
/* flops of the planned grouped GEMM of step 1 or step 4 (2*m*n*k over its block pairs) */
double ctn_heff2_gemm_flops(const ctn_heff2_plan *plan, int step);
/* the same for the stacked tensor-core GEMMs of a split precision (one product counted) */
double ctn_heff2_split_gemm_flops(ctn_heff2_plan *plan, int precision, int step);
/* work accounting of the split-precision GEMMs (step 1 in out[0..3], step 4 in out[4..7]):
 * useful flops (2*M*N*K, one product), executed MMA flops of the tiles including their padding
 * (one product), the operand panel bytes the tiles copy into shared memory per matvec (hi and
 * lo panels, with every re-read), and the operands' own bytes (hi and lo, each element once) */
ctn_status ctn_heff2_split_stats(ctn_heff2_plan *plan, int precision, double *out);
void ctn_heff2_plan_destroy(ctn_heff2_plan *plan);
/* tile widths (N of the UMMA tiles: 32, 48, 64, 96, 128, 144, 160, 192 or 256; negative -128, -192,
 * -256 select 2-CTA cta_group::2 tiles of 256 rows) of the step-1 and
 * step-4 tensor-core GEMMs of a split precision; drops that precision's binding (the
 * operand panels depend on the widths), so call ctn_heff2_set_env again.  Used by the
 * autotuner (TwoSiteHeff.autotune). */
ctn_status ctn_heff2_set_tiles(ctn_heff2_plan *plan, int precision, int bn_step1, int bn_step4);
/* epilogue form of the step-1 / step-4 tensor-core GEMMs: -1 automatic (staged through
 * shared memory when the tiles are at least half filled), 0 direct
 * (each lane stores its own accumulator row), 1 staged (whole row segments per store),
 * 2 fragments (16-lane TMEM fragments stored from registers, no shared memory; the 2-CTA
 * tiles run 2 as 1).  Takes effect on the next matvec; used by the autotuner. */
ctn_status ctn_heff2_set_epilogue(ctn_heff2_plan *plan, int precision, int epi_step1, int epi_step4);

/* ---------------------------------------------------------------- batched H_eff
 * Many independent two-site problems (uneven block structures) applied together: the
 * split-precision tables of every plan are concatenated, so each phase (pack, step-1
 * GEMM, MPO fold, step-4 GEMM) of all problems is one launch; the two tcgen05 GEMMs are
 * persistent grouped launches over the union of all problems' tiles.  The vectors and
 * environments of problem i live at element offsets psi_offs[i] / L_offs[i] / R_offs[i]
 * of shared flat buffers (the output uses psi's offsets).  fp32_io != 0: psi, L, R and
 * out are FP32 (else FP64).  ctn_heff2_batch_matvec issues no host synchronisation once
 * ctn_heff2_batch_set_env has run, so it may be recorded in a CUDA graph.  Creating a
 * batch (re)prepares each plan's split tables for the given tile widths.
 * No counterpart in the reference, which contracts one network at a time through
 * Network::Launch (src/RegularNetwork.cpp:901-1007); this batches the two-site matvec
 * of example/DMRG/dmrg_two_sites_U1.py:18-23 over many problems. */
typedef struct ctn_heff2_batch ctn_heff2_batch;
ctn_status ctn_heff2_batch_create(ctn_heff2_plan *const *plans, int nprob, const int64_t *psi_offs,
                                  const int64_t *L_offs, const int64_t *R_offs, int precision,
                                  int bn_step1, int bn_step4, int fp32_io, ctn_heff2_batch **batch);
size_t ctn_heff2_batch_workspace_bytes(const ctn_heff2_batch *batch);
/* useful flops of one batched matvec (2*M*N*K over the GEMM groups, one product) */
double ctn_heff2_batch_gemm_flops(const ctn_heff2_batch *batch);
/* the same accounting as ctn_heff2_split_stats for the batched GEMMs */
ctn_status ctn_heff2_batch_stats(const ctn_heff2_batch *batch, double *out);
ctn_status ctn_heff2_batch_set_env(ctn_heff2_batch *batch, const void *L_all, const void *R_all,
                                   void *workspace, void *stream);
ctn_status ctn_heff2_batch_matvec(ctn_heff2_batch *batch, const void *psi_all, void *out_all,
                                  void *stream);
/* average phase times over `reps` matvecs: ms[0..3] = pack, step-1 GEMM, MPO fold, step-4 GEMM */
ctn_status ctn_heff2_batch_profile(ctn_heff2_batch *batch, const void *psi_all, void *out_all,
                                   int reps, double *ms, void *stream);
void ctn_heff2_batch_destroy(ctn_heff2_batch *batch);

/* ---------------------------------------------------------------- Lanczos
 * Ground state by the Lanczos_Gnd_Ut recurrence on flat FP64 device vectors.
 * matvec(user, x, y, stream) must write y = H x on `stream`.  krylov must hold
 * (maxiter + 1) * n doubles (device); work >= 4 * n + 64 doubles (device).
 * On return *energy holds the lowest Ritz value, eigvec (device, n) the Ritz
 * vector, *iters the iterations done.  Semantics follow the reference: stop
 * when |E_i - E_{i-1}| < cvgcrit or beta == 0 or maxiter reached; matvec is called exactly
 * *iters times. */
typedef int (*ctn_matvec_fn)(void *user, const double *x, double *y, void *stream);
ctn_status ctn_lanczos_gnd(ctn_matvec_fn matvec, void *user, const double *psi0, int64_t n,
                           int maxiter, double cvgcrit, double *krylov, double *work,
                           double *eigvec, double *energy, int *iters, void *stream);
/* Restarted ground-state Lanczos with two matvecs: matvec_lo (e.g. split precision) builds
 * the Krylov space of each cycle, matvec_hi (FP64) is applied once per restart to the
 * current vector to give its FP64 Rayleigh quotient and eigen-residual r = Hv - Ev.  Each
 * cycle: q0 = v, q1 = r/|r|, krydim - 1 low-precision steps with three-term recurrence and
 * an FP64 re-orthogonalisation against q0, FP64 tridiagonal solve, v <- Ritz vector.  Stops
 * when |r| <= tol * |E| or after max_restarts FP64 matvecs.  krylov: krydim * n doubles;
 * work >= n + 3200 + 3 * krydim doubles.  The Krylov steps keep alpha / beta on the device
 * (one host synchronisation per restart); each step's two reductions and its update run as
 * one cooperative launch whose grid barrier is a bounded wait (CTN_ERR_TIMEOUT if it gives
 * up).  *energy / *residual: FP64 Rayleigh quotient and |r| of the returned unit vector;
 * matvecs[0..1] = low / FP64 products used.
 * No direct counterpart in the reference (its Lanczos_ER restarts in one precision,
 * src/linalg/Lanczos_ER.cpp); the recurrence is that of Lanczos_Gnd_Ut. */
ctn_status ctn_lanczos_refined(ctn_matvec_fn matvec_lo, void *user_lo, ctn_matvec_fn matvec_hi,
                               void *user_hi, const double *psi0, int64_t n, int krydim, int max_restarts,
                               double tol, double *krylov, double *work, double *eigvec, double *energy,
                               double *residual, int *restarts, int64_t *matvecs, void *stream);
/* k extreme eigenpairs of a symmetric operator (the "which" form of linalg::Lanczos,
 * src/linalg/Lanczos.cpp:250-402, which drives ARPACK dsaupd/dseupd there): thick-restart
 * Lanczos with full re-orthogonalisation on the device.  which: 0 = "SA" (smallest
 * algebraic), 1 = "LA" (largest algebraic), 2 = "LM" (largest magnitude).  ncv: basis size
 * (0: min(n, 2k + 10), the reference's default; otherwise k < ncv <= n).  A Ritz pair
 * counts as converged when |beta_m y_m| <= tol * max(eps^(2/3), |theta|) (tol = 0: machine
 * precision), as in ARPACK.  maxiter bounds the restart cycles.  basis: (ncv + 1) * n
 * doubles (device); work: ctn_lanczos_which_work_doubles(n, ncv) doubles (device, with the
 * resolved ncv).  evals (host, k) and evecs (device, k * n, or null) in the reference's
 * order (ascending for SA, descending value / magnitude for LA / LM).  *iters: restart
 * cycles run; *nconv: wanted pairs converged (k unless maxiter ran out). */
/* exp(tau H) v for a symmetric operator by Lanczos projection: linalg::Lanczos_Exp
 * (src/linalg/Lanczos_Exp.cpp:264-453, CPU and dense-only there).  Plain three-term
 * recurrence from v / |v| with the reference's breakdown rule and its stopping rule
 * |exp(tau T)[i][0]| < cvgcrit; result V exp(tau T) V^T v.  tau = tau_re + i tau_im (real
 * time needs tau_im != 0 and out_im).  basis: min(maxiter, n) * n doubles; work:
 * ctn_lanczos_exp_work_doubles(n, maxiter) doubles (device).  *iters: Krylov dimension used. */
size_t ctn_lanczos_exp_work_doubles(int64_t n, int maxiter);
ctn_status ctn_lanczos_exp(ctn_matvec_fn matvec, void *user, const double *v, int64_t n, double tau_re,
                           double tau_im, double cvgcrit, int maxiter, double *basis, double *work, double *out_re,
                           double *out_im, int *iters, void *stream);
size_t ctn_lanczos_which_work_doubles(int64_t n, int ncv);
ctn_status ctn_lanczos_which(ctn_matvec_fn matvec, void *user, const double *v0, int64_t n, int which, int k,
                             int ncv, int maxiter, double tol, double *basis, double *work, double *evals,
                             double *evecs, int *iters, int *nconv, void *stream);
/* the same on a planned H_eff: `precision` for the Krylov steps, FP64 for the refinement
 * (both must be bound with ctn_heff2_set_env) */
ctn_status ctn_heff2_lanczos_refined(ctn_heff2_plan *plan, int precision, const double *psi0, int krydim,
                                     int max_restarts, double tol, double *krylov, double *work,
                                     double *eigvec, double *energy, double *residual, int *restarts,
                                     int64_t *matvecs, void *stream);
/* the same driver on a planned H_eff (no callback).  Each next iteration is queued on the
 * device before the host solves the current tridiagonal, so the host solve overlaps the next
 * matvec; after the last iteration one queued matvec is discarded.  CTN_PREC_F64: the results
 * are those of ctn_lanczos_gnd with the same matvec, bit for bit.  Split precisions: the
 * matvec hands its result to the recurrence in FP32 (its own error, ~1e-5, is far above the
 * FP32 rounding); the recurrence itself is FP64. */
ctn_status ctn_heff2_lanczos_gnd(ctn_heff2_plan *plan, int precision, const double *psi0,
                                 int maxiter, double cvgcrit, double *krylov, double *work,
                                 double *eigvec, double *energy, int *iters, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CYTNX_B200_H */
