/*
 * dmhm_b200 — C ABI of the B200 (sm_100a) H-matrix engine.
 *
 * Plain pointers, sizes and opaque handles only.  Each entry point replaces
 * one operation of the reference C++ API of YingzhouLi/dmhm (cited per entry
 * as file:line inside that project).  All matrices are real double precision,
 * column-major; all vectors are in the H-matrix's hierarchical ordering
 * (the ordering BuildNaturalToHierarchicalMap produces).
 *
 * Every function returns an HM_* status (0 = success).  On failure,
 * hm_last_error() returns a message for the calling thread.  Work is issued on
 * the context's CUDA stream; functions taking host pointers (the *_host
 * variants) synchronize that stream before returning.
 */
#ifndef DMHM_B200_H
#define DMHM_B200_H

#include <stdint.h>
#include <stddef.h>

#if defined(__GNUC__)
#define HM_API __attribute__((visibility("default")))
#else
#define HM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define HM_OK 0
#define HM_ERR_ARGUMENT 1      /* bad argument / nonconformal shapes          */
#define HM_ERR_OOM 2           /* device allocation failed                    */
#define HM_ERR_CUDA 3          /* CUDA runtime error                          */
#define HM_ERR_UNSUPPORTED 4   /* combination the reference also rejects      */
#define HM_ERR_NUMERICAL 5     /* non-finite values met (NaN / Inf)           */
#define HM_ERR_TIMEOUT 6       /* a bounded device wait ran out               */
#define HM_ERR_INTERNAL 7

typedef struct hm_context_s* hm_context;  /* device, stream, generators     */
typedef struct hm_matrix_s* hm_matrix;    /* one H-matrix resident in HBM    */
typedef struct hm_rank_model_s* hm_rank_model;  /* learned rank predictor  */

/* Message of the last failed call on this thread ("" if none). */
HM_API const char* hm_last_error(void);

/* Library version: major*10000 + minor*100 + patch. */
HM_API int hm_version(void);

/*
 * Context: device, stream, the two global generators and Oversample().
 * Replaces Initialize (src/core/global.cpp:43-94): both generators start at
 * the reference seed {17, 21} (global.cpp:88-93); oversample starts at 4
 * (global.cpp:30).  stream == NULL creates a private non-blocking stream.
 */
HM_API int hm_context_create(int device, void* cuda_stream, hm_context* out);
HM_API int hm_context_destroy(hm_context ctx);
/* Waits for the context's stream; HM_ERR_NUMERICAL when a low-rank rounding
   since the last synchronization met NaN or Inf (non-finite block data),
   HM_ERR_TIMEOUT when a bounded device wait gave up. */
HM_API int hm_context_synchronize(hm_context ctx);
/* SetOversample / Oversample (src/core/global.cpp:155-159). */
HM_API int hm_set_oversample(hm_context ctx, int oversample);
HM_API int hm_get_oversample(hm_context ctx, int* oversample);
/* SetCompressionTolerance / CompressionTolerance (src/core/global.cpp:
   160-181), applied as the single-rank DistHMat truncation does
   (SVDTrunc, src/DistHMat2d/Truncation-incl.hpp:37-63): every H*H
   compression keeps the singular values above tol * sigma_0 (at least
   sigma_0; only sigma_0 when sigma_0 < tol^2), at most maxRank, and the
   product is stored at the ranks kept.  0 (the default) keeps HMat2d's fixed rank maxRank. */
HM_API int hm_set_compression_tolerance(hm_context ctx, double tol);
HM_API int hm_get_compression_tolerance(hm_context ctx, double* tol);
/* SeedSerialLcg (src/core/random.cpp:67-68) and the single-rank
   SeedParallelLcg (random.cpp:70-101); state is the next value drawn. */
HM_API int hm_set_lcg_states(hm_context ctx, uint64_t serial, uint64_t parallel);
HM_API int hm_get_lcg_states(hm_context ctx, uint64_t* serial, uint64_t* parallel);

/*
 * BuildNaturalToHierarchicalMap (src/HMat2d/HMat2d.cpp:69-87,
 * src/HMat3d/HMat3d.cpp:91-110): map[natural] = hierarchical index.
 * dim = 2 or 3; sizes[dim]; map has prod(sizes) entries.
 */
HM_API int hm_natural_to_hierarchical_map(int dim, const int* sizes, int num_levels,
                                   int* map);

/*
 * HMat2d(const Sparse&, numLevels, maxRank, strong, xSize, ySize)
 * (include/dmhm/hmat2d.hpp:55-58; ImportSparse src/HMat2d/HMat2d.cpp:961-1033)
 * and the HMat3d equivalent (include/dmhm/hmat3d.hpp).  The CSR matrix is in
 * hierarchical ordering, height = width = prod(sizes), non-symmetric storage.
 */
HM_API int hm_create_from_csr(hm_context ctx, int dim, const int* sizes,
                       int num_levels, int max_rank, int strongly_admissible,
                       const int64_t* row_offsets, const int32_t* col_indices,
                       const double* values, hm_matrix* out);
/*
 * HMat2d<std::complex<double>> / HMat3d<std::complex<double>> (explicit
 * instantiations, src/HMat2d/HMat2d.cpp:1321-1324) from a complex CSR in
 * hierarchical order: values[2k], values[2k+1] = real, imaginary part of
 * nonzero k (the memory of std::complex<double>[]).  Stored on the device in
 * real form (two rows per grid point, entry a + bi as [[a, -b], [b, a]], a
 * complex rank-r block as a real rank-2r block), so every H-matrix entry of
 * this header (products, H*H, SchulzInvert, EstimateTwoNorm, copy,
 * transpose = AdjointFrom, real Scale / AddConstantToDiagonal) applies to it
 * unchanged, on real vectors of twice the length, which are the complex
 * vectors in interleaved storage; hm_info reports that real form.  H*H
 * products draw 2 x Oversample() real samples per complex direction.
 */
HM_API int hm_create_from_csr_complex(hm_context ctx, int dim, const int* sizes, int num_levels,
                                      int max_rank, int strongly_admissible,
                                      const int64_t* row_offsets, const int32_t* col_indices,
                                      const double* values, hm_matrix* out);
HM_API int hm_is_complex(hm_matrix h, int* is_complex);

/*
 * The reference's wire format: PackedSize / Pack / Unpack and the
 * HMat2d(const Vector<byte>&) constructor (src/HMat2d/Pack-incl.hpp:16-364;
 * HMat3d: src/HMat3d/Pack-incl.hpp).  Byte-identical to what the reference
 * writes on the same host (native-endian ints, one-byte bools, column-major
 * doubles), so matrices move between the two in both directions.
 * hm_unpack builds the block structure from the header (dim = 2 for HMat2d,
 * 3 for HMat3d) and rejects a block tree that does not match it, symmetric
 * matrices (NODE_SYMMETRIC) and non-root sub-matrices.  Real matrices only.
 */
HM_API int hm_packed_size(hm_matrix h, size_t* bytes);

/*
 * One low-rank approximation F = U V^T of a whole product (the randomized
 * range finder hmat_tools::Multiply, include/dmhm/hmat_tools.hpp:1657-1746:
 * F := alpha A B; TransposeMultiply, :1848-1937: F := alpha A^T B;
 * AdjointMultiply, :2039-: F := alpha A^H B), sample_rank Gaussian samples
 * from the context's serial generator (SampleRank(r) = r + Oversample() in
 * the reference's callers), truncated to rank min(A.MaxRank, B.MaxRank,
 * height) (or by the compression tolerance when one is set).  op 0, 1, 2.
 * U, V: HOST, height x max_rank (leading dimensions ldu, ldv); *rank
 * receives the number of columns written.  Real matrices only.
 */
HM_API int hm_low_rank_product(hm_matrix A, int op, double alpha, hm_matrix B, int sample_rank,
                               double* U, int ldu, double* V, int ldv, int max_rank, int* rank);
HM_API int hm_pack(hm_matrix h, void* buffer, size_t capacity, size_t* written);
HM_API int hm_unpack(hm_context ctx, int dim, const void* buffer, size_t size, hm_matrix* out);
/*
 * Complex Multiply / TransposeMultiply / AdjointMultiply against dense
 * blocks (src/HMat2d/MultiplyDense-incl.hpp:12-260 for Scalar =
 * std::complex<double>): C := alpha op(A) B + beta C, op 0 = A, 1 = A^T,
 * 2 = A^H; B, C interleaved complex, leading dimensions in complex elements;
 * DEVICE pointers (stream-ordered) or HOST pointers (copies, synchronizes).
 */
HM_API int hm_multiply_dense_complex(hm_matrix h, int op, double alpha_re, double alpha_im,
                                     const double* B, int ldb, double beta_re, double beta_im,
                                     double* C, int ldc, int nrhs);
HM_API int hm_multiply_dense_complex_host(hm_matrix h, int op, double alpha_re,
                                          double alpha_im, const double* B, int ldb,
                                          double beta_re, double beta_im, double* C, int ldc,
                                          int nrhs);
/*
 * Complex scalars on a complex H-matrix: Scale (src/HMat2d/HMat2d.cpp:616-647)
 * and AddConstantToDiagonal (:704-744) with alpha = alpha_re + i alpha_im;
 * ConjugateFrom (:424-472) into *dst; TransposeFrom without conjugation
 * (:477-546; hm_transpose is AdjointFrom, :548-614, for a complex handle).
 * *dst == NULL creates a new handle.
 */
HM_API int hm_scale_complex(hm_matrix h, double alpha_re, double alpha_im);
/* UpdateWith(alpha, B) (src/HMat2d/HMat2d.cpp:749-781): A := alpha B + A,
   low-rank blocks by RoundedUpdate to maxRank (src/hmat_tools/
   RoundedUpdate.cpp:14-162), dense blocks by Update; A and B on one block
   structure.  SetToIdentity (HMat2d.cpp:652-702): empty low-rank blocks,
   identity dense diagonal.  Conjugate (HMat2d.cpp:396-422): A := conj(A) in
   place (nothing to do for a real matrix). */
HM_API int hm_update_with(hm_matrix A, double alpha, hm_matrix B);
HM_API int hm_set_to_identity(hm_matrix h);
HM_API int hm_conjugate_in_place(hm_matrix h);
HM_API int hm_add_constant_to_diagonal_complex(hm_matrix h, double alpha_re, double alpha_im);
HM_API int hm_conjugate(hm_matrix src, hm_matrix* dst);
HM_API int hm_transpose_complex(hm_matrix src, hm_matrix* dst);
HM_API int hm_destroy(hm_matrix h);

/* Grid of the block structure: dim (2 or 3), sizes[dim] (xSize, ySize[,
   zSize]), strong (1) or weak (0) admissibility (StronglyAdmissible,
   src/HMat2d/HMat2d.cpp:436), and unknowns per grid point (1, or 2 for the
   real form of a complex matrix).  Any pointer may be NULL. */
HM_API int hm_structure(hm_matrix h, int* dim, int* sizes, int* strongly_admissible,
                        int* unknowns_per_point);

/* Height, width, number of levels, max rank, and the block census:
   counts[0..2] = node / low-rank / dense blocks, counts[3] = sum of low-rank
   ranks, bytes = device bytes of the block data. */
HM_API int hm_info(hm_matrix h, int* height, int* width, int* num_levels,
            int* max_rank, int64_t* counts, int64_t* bytes);

/* SetToRandom (src/HMat2d/SetToRandom-incl.hpp:14-55): dense leaves and
   rank-maxRank U, V drawn from the context's parallel generator. */
HM_API int hm_set_to_random(hm_matrix h);

/*
 * C := alpha op(H) B + beta C, op = identity (transpose = 0) or transpose (1).
 * HMat2d::Multiply / TransposeMultiply against Dense and Vector
 * (src/HMat2d/MultiplyDense-incl.hpp:12-150, MultiplyVector-incl.hpp:12-124).
 * B: n x nrhs (ld ldb), C: m x nrhs (ld ldc), DEVICE pointers, stream-ordered.
 */
HM_API int hm_multiply_dense(hm_matrix h, int transpose, double alpha,
                      const double* B, int ldb, double beta, double* C,
                      int ldc, int nrhs);
/* Same with HOST pointers: copies in, multiplies, copies out, synchronizes. */
HM_API int hm_multiply_dense_host(hm_matrix h, int transpose, double alpha,
                           const double* B, int ldb, double beta, double* C,
                           int ldc, int nrhs);

/*
 * Mixed-precision form of hm_multiply_dense (no transpose): block data read
 * from an FP32 copy rounded to TF32 (made on first use), inputs rounded to
 * TF32, products on the tensor cores with FP32 accumulation, C in FP64.
 * DEVICE pointers; synchronizes the stream.  Relative error against the
 * FP64 product is about 1e-3 (TF32 has an 11-bit significand).  The
 * reference computes only in the matrix's own precision.
 * Two kernel forms: 1 = tcgen05.mma kind::tf32 with tensor-memory
 * accumulators (nrhs <= 64, ranks <= 256), 2 = persistent 64 x 64 tiles of
 * mma.sync m16n8k8 TF32 (any nrhs; below 9 columns the FP64 kernels run).
 * hm_set_tf32_kernel(ctx, 0) (the default) times both on the first product
 * of each (layout, column bucket 16/32/64/...) and keeps the faster;
 * hm_tf32_kernel_choice reports (and if need be tunes) the form used.
 */
HM_API int hm_multiply_dense_tf32(hm_matrix h, double alpha, const double* B, int ldb,
                                  double beta, double* C, int ldc, int nrhs);
HM_API int hm_set_tf32_kernel(hm_context ctx, int which);
HM_API int hm_tf32_kernel_choice(hm_matrix h, const double* B, int ldb, int nrhs, int* which);
/*
 * FP64 products of 9 to 16 columns (hm_multiply_dense and the H*H sampling
 * products) run either as one pass of the FP64 tensor-core 64 x 64 tiles (1)
 * or as passes of at most 8 columns through the streaming kernels (2); which
 * is faster depends on the operator.  hm_set_fp64_split(ctx, 0) (the
 * default) times both the first time a (layout, job count, column count)
 * occurs and keeps the faster; hm_fp64_split_choice reports (and if need be
 * tunes) the form hm_multiply_dense uses for nrhs columns (DEVICE B).  No
 * counterpart in the reference (it calls one BLAS routine per block).
 */
HM_API int hm_set_fp64_split(hm_context ctx, int which);
HM_API int hm_fp64_split_choice(hm_matrix h, const double* B, int ldb, int nrhs, int* which);

/*
 * H*H products with randomized low-rank compression.
 * hm_multiply_hmat: C := alpha A B, C rebuilt (HMat2d::Multiply(alpha,
 * const HMat2d& B, HMat2d& C), include/dmhm/hmat2d.hpp:260-263;
 * src/HMat2d/MultiplyHMat-incl.hpp:12-187).  *C == NULL creates a new
 * handle; otherwise its previous contents are replaced.
 * hm_multiply_hmat_update: C :~= alpha A B + beta C on C's existing structure
 * (hmat2d.hpp:265-268; MultiplyHMat-incl.hpp:189-380).
 * Sampled products draw their Gaussian test matrices from the context's
 * serial generator in the reference's recursion order; Oversample() extra
 * samples (SampleRank, hmat2d.hpp:32-33).  C must differ from A and B.
 */
HM_API int hm_multiply_hmat(hm_matrix A, double alpha, hm_matrix B, hm_matrix* C);
HM_API int hm_multiply_hmat_update(hm_matrix A, double alpha, hm_matrix B, double beta,
                                   hm_matrix C);

/* hmat_tools::EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548). */
HM_API int hm_estimate_two_norm(hm_matrix h, double theta, double confidence,
                                double* estimate);

/* DirectInvert (src/HMat2d/Invert-incl.hpp:17-125; HMat3d:
   src/HMat3d/Invert-incl.hpp:14-122): A := inv(A) by recursive block
   elimination with Schur complements, in the reference's order of block
   products (each truncated to maxRank, randomized compressions drawing from
   the context's serial generator as the reference's do), dense diagonal
   leaves inverted by partial-pivoting elimination (hmat_tools::Invert,
   src/hmat_tools/Invert.cpp:14-42).  Real matrices whose dense leaves have
   at most 96 rows; HM_ERR_NUMERICAL when a leaf is singular. */
HM_API int hm_direct_invert(hm_matrix h);

/*
 * SchulzInvert(numIterations, theta, confidence, stopTol)
 * (include/dmhm/hmat2d.hpp:275-276, src/HMat2d/Invert-incl.hpp:127-196;
 * HMat3d: pass stop_tol = 1e-4, src/HMat3d/Invert-incl.hpp:168).
 * numIterations <= 0 runs up to 30 iterations with the stop test.  h is
 * replaced by the approximate inverse.  Optional outputs: iterations run and
 * the estimates [||A||, ||I - X_k A|| per stop check] (up to trace_cap).
 */
HM_API int hm_schulz_invert(hm_matrix h, int num_iterations, double theta,
                            double confidence, double stop_tol, int* iterations,
                            double* trace, int trace_cap, int* trace_len);

/*
 * Mixed-precision SchulzInvert (same iteration and stop test as
 * hm_schulz_invert).  While the last ||I - X_k A|| estimate is above
 * mixed_switch (without the stop test: all but the last three iterations),
 * an iteration runs its two H*H products in the low-precision phase (range
 * samples on the TF32 tensor cores, block roundings in FP32); the others,
 * the norm estimates and the sample orthogonalisation are FP64.
 * mixed_switch = 0 is hm_schulz_invert.  low_iterations receives the number
 * of low-precision iterations.  The reference has only the FP64 method.
 */
HM_API int hm_schulz_invert_mixed(hm_matrix h, int num_iterations, double theta,
                                  double confidence, double stop_tol, double mixed_switch,
                                  int* iterations, int* low_iterations, double* trace,
                                  int trace_cap, int* trace_len);
/* Low-precision phase for the context's H*H products (on != 0): range
   samples in TF32, roundings in FP32 (relative block error about 1e-6 from
   the roundings, up to about 1e-3 in blocks whose spectrum reaches below
   TF32's resolution).  Off by default. */
HM_API int hm_set_low_precision(hm_context ctx, int on);

/* CopyFrom (src/HMat2d/HMat2d.cpp:331-391); AdjointFrom / TransposeFrom for
   real scalars (HMat2d.cpp:479-614); *dst == NULL creates a new handle. */
HM_API int hm_copy(hm_matrix src, hm_matrix* dst);
HM_API int hm_transpose(hm_matrix src, hm_matrix* dst);
/* Scale (HMat2d.cpp:616-647; alpha = 0 drops every low-rank block to rank 0)
   and AddConstantToDiagonal (HMat2d.cpp:704-744). */
HM_API int hm_scale(hm_matrix h, double alpha);
HM_API int hm_add_constant_to_diagonal(hm_matrix h, double alpha);

/*
 * y := alpha op(H) x + beta y for one vector (DEVICE pointers, stream-ordered)
 * without allocating any device memory.  No counterpart in the reference: it
 * is for callers that cannot allocate device memory during the call (their
 * memory manager already holds the GPU's memory, or a time-critical loop must
 * not call the allocator).  Intermediates live in one static 4 MiB device
 * array of the library, so the matrix may need at most 524288 entries of
 * (the sum of its low-rank ranks); larger matrices return
 * HM_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * address; make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race and must not be issued.
 * Results agree with hm_multiply_dense to rounding (atomic accumulation).
 */
HM_API int hm_multiply_vector_noalloc(hm_matrix h, int transpose, double alpha,
                                      const double* x, double beta, double* y);

/*
 * Learned sample counts for the randomized H*H compressions.  No counterpart
 * in the reference, whose randomized product always draws SampleRank =
 * maxRank + Oversample() samples (include/dmhm/hmat_tools.hpp:1657-1746).
 * A three-layer perceptron (hm_rank_feature_count() inputs, two hidden
 * layers of 64, FP32; hm_rank_param_count() parameters) predicts, from the
 * features of one compression, the fraction of its rank cap that the
 * tolerance truncation keeps; with the model attached (hm_use_rank_model)
 * each compression draws ceil(fraction * cap) + margin + Oversample()
 * samples, estimates its error with `probes` Gaussian probe vectors and is
 * redone with the full sample count when that estimate exceeds 10 * the
 * compression tolerance.  Training data come from runs with the log on
 * (hm_rank_log_enable; needs a tolerance): features and kept fractions of
 * every compression.  Forward, backward and Adam run on the GPU.
 * Features (float rows of hm_rank_feature_count()): level / numLevels,
 * log2(1+m)/16, log2(1+n)/16, min(1, admissibility distance / 8), mean rank
 * of the low-rank leaves below the A block / maxRank, the same below the B
 * block, dense share of the entries below A, the same below B, rank cap /
 * maxRank, dimension / 3.
 */
HM_API int hm_rank_feature_count(void);
HM_API int hm_rank_param_count(void);
HM_API int hm_rank_model_create(hm_context ctx, uint64_t seed, hm_rank_model* out);
HM_API int hm_rank_model_destroy(hm_rank_model m);
HM_API int hm_rank_model_set_params(hm_rank_model m, const float* params, int n);
HM_API int hm_rank_model_get_params(hm_rank_model m, float* params, int n);
/* Mean squared error of the predictions on (x: n rows, t: n targets) and its
   gradient (grad: hm_rank_param_count() floats, may be NULL). */
HM_API int hm_rank_model_loss_grad(hm_rank_model m, const float* x, const float* t, int n,
                                   float* loss, float* grad);
/* `epochs` full-batch Adam steps (learning rate lr); *loss = final loss. */
HM_API int hm_rank_model_train(hm_rank_model m, const float* x, const float* t, int n,
                               int epochs, float lr, float* loss);
HM_API int hm_rank_model_predict(hm_rank_model m, const float* x, int n, float* out);
/* Attach (m != NULL) or detach the model; margin: extra rank over the
   prediction; probes: probe vectors of the error check. */
HM_API int hm_use_rank_model(hm_context ctx, hm_rank_model m, int margin, int probes);
HM_API int hm_rank_log_enable(hm_context ctx, int on);
/* Copies min(cap, *n) logged rows (x: cap * features floats, t: cap floats);
   *n receives the number logged; clear = 1 empties the log afterwards. */
HM_API int hm_rank_log_read(hm_context ctx, float* x, float* t, int cap, int* n, int clear);
/* Compressions run, samples drawn, samples the fixed count would have drawn,
   compressions redone after a failed probe check (since context creation). */
HM_API int hm_rank_stats(hm_context ctx, int64_t* compressions, int64_t* samples,
                         int64_t* samples_plain, int64_t* fallbacks);

/* Diagnostics (no reference counterpart): number of kernels this library has
   launched so far in the process, and per-kernel CUDA-event timing on the
   context stream.  hm_profile_enable resets the totals; hm_profile_read
   synchronizes and returns kernel `index` (HM_ERR_ARGUMENT past the end). */
HM_API unsigned long long hm_kernel_launches(void);
HM_API int hm_profile_enable(hm_context ctx, int on);
HM_API int hm_profile_read(hm_context ctx, int index, char* name, int name_cap,
                           double* ms, int64_t* launches);

/* Measurement aid (no reference counterpart): FP64 throughput of one
   instruction form on `device`, from a register-only kernel of the library
   (4 CTAs of 256 threads per SM, 8 independent accumulators per thread,
   `iterations` rounds), timed with CUDA events on a private stream.
   form: 0 mma.sync m8n8k4 .f64, 1 m16n8k4 .f64, 2 m16n8k8 .f64,
   3 m16n8k16 .f64, 4 scalar fma.rn.f64.  *tflops receives 1e-12 flop/s;
   *ms (may be NULL) the launch time. */
/* Check of the failure path (no reference counterpart): runs the bounded
   mbarrier wait of the tensor-core kernels on a barrier that nothing arrives
   at, giving up after `polls` polls (1..2^26).  *timed_out = 1 when the wait
   gave up, recorded its timeout and returned, as it must; the GPU context
   stays usable.  A real kernel whose wait gives up reports HM_ERR_TIMEOUT. */
HM_API int hm_check_bounded_wait(int device, long long polls, int* timed_out);

HM_API int hm_measure_fp64_peak(int device, int form, int iterations, double* tflops,
                                double* ms);

#ifdef __cplusplus
}
#endif

#endif /* DMHM_B200_H */
