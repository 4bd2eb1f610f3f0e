// Engine objects behind the C ABI: the context (device, stream, generators,
// workspace) and the device-resident H-matrix.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "common.h"
#include "structure.h"

namespace hmb {

// Per-block table entry the kernels read (32 bytes).
struct DevBlock {
    int kind, m, n, rank;
    int row_off, col_off;
    int rank_before;   // sum of the low-rank ranks of the blocks before this one
    int pad1;
    long long off;   // element offset of U (low-rank, V follows at off+m*rank) or D
};

struct Context {
    int device = 0;
    cudaStream_t stream = 0;
    bool own_stream = false;
    int oversample = 4;
    // Next raw state of the serial / parallel LCG (src/core/random.cpp:13-25).
    uint64_t serial_state = 0, parallel_state = 0;
    int num_sms = 148;
    // Relative truncation tolerance of the H*H compressions: 0 keeps the
    // reference's fixed rank maxRank; > 0 drops singular values at or below
    // tol * sigma_0 (capped at maxRank) and stores the products at the ranks
    // kept (CompressionTolerance, src/core/global.cpp:155-181; SVDTrunc,
    // src/DistHMat2d/Truncation-incl.hpp:37-63).
    double compression_tol = 0.0;
    // Learned sample counts of the randomized H*H compressions (mlp.cu):
    // when set, each compression draws (predicted rank + margin) +
    // oversample samples, checked by probe vectors.
    struct RankModel* rank_model = nullptr;
    int rank_margin = 2;
    int rank_probes = 4;
    // Training log: features and kept-rank fractions of every compression
    // (filled when rank_log is on and a tolerance is set).
    bool rank_log = false;
    std::vector<float> log_x, log_t;
    struct RankStats {
        long long compressions = 0, samples = 0, samples_plain = 0, fallbacks = 0;
    } rank_stats;
    // Work lists and scratch are stream-ordered allocations (cudaMallocAsync
    // / cudaFreeAsync on `stream`), freed right after the launches that use
    // them are queued.

    // Optional per-kernel timing with CUDA events on `stream`.
    bool profiling = false;
    struct Pending { std::string name; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    struct Totals { double ms = 0; long long launches = 0; };
    std::map<std::string, Totals> totals;
    void collect();   // synchronizes, folds pending event pairs into totals

    // Completion counters of the split-work kernels: all zero between
    // launches (each user resets what it counted).  Returns >= n of them.
    int* zeroed_counters(long long n);
    DeviceBuffer<int> counters;
    long long counters_cap = 0;
    // Layout groups (structure + ranks) with their product work lists
    // (matmul.cu), most recently used last.
    std::vector<std::shared_ptr<struct LayoutGroup>> layouts;
    // Symbolic H*H plans of recent products (hh.cu).
    std::shared_ptr<struct HHPlanCache> hh_cache;
    // Low-precision phase: H*H products draw their range samples (B Omega,
    // A (B Omega)) on the TF32 tensor cores and round their blocks in FP32
    // (QR, core SVD); orthogonalisation of the samples, the projections and
    // everything else stay FP64.  Set by mixed-precision Schulz for its
    // early iterations, or by the caller for whole products.
    bool low_precision = false;
    // Kernels of the TF32 dense product: 0 autotuned per (layout, column
    // bucket), 1 tcgen05 (at most 64 columns, ranks <= 256), 2 mma.sync.
    int tf32_kernel = 0;
    std::map<std::pair<uint64_t, int>, int> tf32_tuned;
    // FP64 products of 9 to 16 columns: 0 autotuned per (layout of the first
    // job's matrix, job count, column count), 1 one pass of the tensor-core
    // 64 x 64 tiles, 2 passes of at most 8 columns through the streaming
    // kernels.
    int fp64_split = 0;
    std::map<std::tuple<uint64_t, int, int>, int> fp64_split_tuned;
    // Grow-only device scratch reused by consecutive H*H products on this
    // context's stream (W arena, sampling arena, state slots, rounding work):
    // a product's kernels finish before the next product's start.
    double* scratch(int slot, long long n);
    DeviceBuffer<double> scratch_bufs[4];
    // One double of pinned host memory for results read back asynchronously
    // (made on first use, freed with the context).
    double* pinned_scalar();
    double* pinned = nullptr;
    // Device word set by kernels whose bounded waits gave up (zero = fine);
    // read and cleared by check_numerical().
    int* error_word();
    DeviceBuffer<int> errword;
    // Device word set by a low-rank rounding whose core held NaN or Inf
    // (zero = fine); read and cleared by check_numerical().
    int* numerical_word();
    DeviceBuffer<int> numword;
    // Synchronizes the stream and throws HM_ERR_TIMEOUT when a bounded wait
    // gave up, HM_ERR_NUMERICAL when a rounding met a non-finite value, since
    // the last check (clearing the word).
    void check_numerical();
};

// Host-side wall time of a phase, recorded under `name` when profiling.
class HostScope {
  public:
    HostScope(Context& c, const char* name)
        : c_(c), name_(name), t0_(std::chrono::steady_clock::now()) {}
    ~HostScope() {
        if (!c_.profiling) return;
        auto dt = std::chrono::steady_clock::now() - t0_;
        auto& t = c_.totals[std::string("host:") + name_];
        t.ms += std::chrono::duration<double, std::milli>(dt).count();
        t.launches += 1;
    }
  private:
    Context& c_;
    const char* name_;
    std::chrono::steady_clock::time_point t0_;
};

// Counts every kernel launch of the library (all contexts).
extern std::atomic<unsigned long long> g_launches;

// Brackets one kernel launch: counts it and, when profiling, records events.
class LaunchScope {
  public:
    LaunchScope(Context& c, const char* name) : c_(c), name_(name) {
        g_launches.fetch_add(1, std::memory_order_relaxed);
        if (c_.profiling) {
            cudaEventCreate(&a_);
            cudaEventCreate(&b_);
            cudaEventRecord(a_, c_.stream);
        }
    }
    ~LaunchScope() {
        if (c_.profiling) {
            cudaEventRecord(b_, c_.stream);
            c_.pending.push_back({name_, a_, b_});
        }
    }
  private:
    Context& c_;
    const char* name_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
};

class HMatrix {
  public:
    Context* ctx = nullptr;
    std::shared_ptr<Structure> S;
    int max_rank = 0;
    std::vector<int> rank;          // per block (low-rank blocks)
    std::vector<long long> off;     // per block data offset (elements)
    long long total = 0;            // elements in `data`
    DeviceBuffer<double> data;
    DeviceBuffer<DevBlock> table;   // device copy of the per-block table
    // FP32 copy (rounded to TF32) of `data` for the tensor-core products;
    // made on first use, dropped whenever `data` changes.
    DeviceBuffer<float> data32;
    bool shadow_valid = false;
    // Work lists of the products with this matrix, shared by every matrix of
    // the context with the same structure and ranks (they hold storage
    // offsets); found on first use, dropped whenever the storage is re-laid
    // out.
    mutable std::shared_ptr<struct LayoutGroup> group;

    int height() const { return S->N; }
    int width() const { return S->N; }
    // Computes offsets from `rank`, (re)allocates `data` (uninitialized) and
    // uploads the table.
    void layout();
    void upload_table();
    double* U(int b) const { return data.get() + off[b]; }
    double* V(int b) const { return data.get() + off[b] + (long long)S->blocks[b].m * rank[b]; }
    double* D(int b) const { return data.get() + off[b]; }
};

// Multiplication jobs: out = alpha op(H restricted to subtree `root`) in
// (+ beta out).  `in` points at the input row that corresponds to the root's
// first column (first row for op = transpose); `out` likewise for its output.
struct MatJob {
    const HMatrix* H;
    int root;
    bool trans;
    double alpha, beta;
    const double* in;
    int ldin;
    double* out;
    int ldout;
    int k;
    const double* alpha_scale = nullptr;   // if set, alpha is multiplied by *alpha_scale
};

// Work lists of one subtree (root, op) of one H-matrix, kept on the device
// (matmul.cu).  Cached per H-matrix; dropped when its storage is re-laid out.
struct JobTemplate;
// Row tiles of the output hold at most `row_tile` rows (<= 64).
std::shared_ptr<JobTemplate> get_template(Context& ctx, const HMatrix& H, int root, bool trans,
                                          int row_tile = 64);

// Runs a batch of jobs as two level-batched launches (low-rank inner products,
// then one fused output pass per row tile).  Outputs of different jobs must
// not overlap; inputs may alias each other but not outputs.  tf32: jobs with
// more than 8 columns multiply on the TF32 tensor cores (FP32 copies of the
// blocks and inputs, FP32 accumulation, FP64 output).
void run_jobs(Context& ctx, const std::vector<MatJob>& jobs, bool tf32 = false);
// How run_jobs runs an FP64 job list (tuning it if need be): 1 one pass of
// the tensor-core tiles, 2 passes of at most 8 columns (matmul.cu).
int fp64_split_for(Context& ctx, const std::vector<MatJob>& jobs);
// One-vector product of one job streamed block by block (matvec.cu); false
// when the matrix does not fit that kernel (the caller uses run_jobs' lists).
bool multiply_vector_streamed(Context& ctx, const MatJob& job);

// Tensor-core (TF32, FP32 accumulation) H-matrix x dense, device pointers;
// synchronizes (checks the kernels' error word).  The kernel form comes from
// tf32_kernel_choice (tc_matmul.cu).
int tf32_kernel_choice(Context& ctx, HMatrix& H, const double* B, int ldb, int nrhs);
// FP32 copy of the block data rounded to TF32 (data32), made on first use
// and kept until the data change.
void ensure_tf32_copy(Context& ctx, HMatrix& H);
// Runs the tensor-core kernels' bounded mbarrier wait on a barrier nothing
// arrives at, with `limit` polls; true when the wait gave up as it must.
bool bounded_wait_times_out(int device, long long limit);

void multiply_dense_tf32(HMatrix& H, double alpha, const double* B, int ldb, double beta,
                         double* C, int ldc, int nrhs);

// Complex H-matrix (real form, structure dof 2) times complex dense blocks
// (interleaved re, im; leading dimensions in complex elements), device
// pointers: op 0 C = alpha A B + beta C, 1 with A^T, 2 with A^H (complex.cu).
void multiply_dense_complex(HMatrix& H, int op, double ar, double ai, const double* B, int ldb,
                            double br, double bi, double* C, int ldc, int nrhs);

// F := alpha op(A) B as one low-rank matrix U V^T (lrprod.cu; op 0 = A,
// 1 = A^T, 2 = A^H); U, V: height x rank on the device; returns the rank.
int low_rank_product(Context& ctx, const HMatrix& A, int op, double alpha, const HMatrix& B,
                     int sample_rank, DeviceBuffer<double>& U, DeviceBuffer<double>& V);

// The reference's Pack / Unpack wire format (pack.cpp).
size_t packed_size(const HMatrix& H);
size_t pack(const HMatrix& H, unsigned char* out, size_t cap);
void unpack(Context& ctx, int dim, const unsigned char* buf, size_t size, HMatrix& H);

// Complex helpers on the real form (complex.cu): Scale and
// AddConstantToDiagonal with complex alpha, in-place conjugation.
void complex_scale(Context& ctx, HMatrix& H, double a, double b);
void complex_add_diagonal(Context& ctx, HMatrix& H, double a, double b);
void complex_conjugate(Context& ctx, HMatrix& H);

// Device kernels driven from the host side (launchers).
void launch_fill_random(Context& ctx, HMatrix& H);

// Gaussian fills (SerialGaussianRandomVectors on Dense<Real>) of m x n
// column-major matrices, each starting at LCG state `base`.
struct FillOp {
    double* dst;
    uint64_t base;
    int m, n;
};
void launch_gaussian_fills(Context& ctx, const std::vector<FillOp>& fills, const char* name);

}  // namespace hmb
