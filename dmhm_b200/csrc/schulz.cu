// Schulz inversion, two-norm estimation and the elementwise H-matrix
// operations they use (CopyFrom, AdjointFrom, Scale, AddConstantToDiagonal).
//
// SchulzInvert (src/HMat2d/Invert-incl.hpp:127-196; 3-D
// src/HMat3d/Invert-incl.hpp:127-186):
//   X_0 = (2 / est^2) A^T with est = EstimateTwoNorm(A) (already >= ||A||),
//   X_{k+1} = (2I - X_k A) X_k,
// with the optional stop test on an estimate of ||I - X_k A||_2.
// EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548): k normalised
// power steps from a Gaussian start vector, est = theta * prod ||A x_i||^(1/k).
// Every step runs on the device; the host reads back one scalar per estimate.
#include "schulz.h"

#include <cmath>
#include <limits>

#include "dense_ops.h"
#include "hh.h"
#include "rng.cuh"

namespace hmb {

namespace {

constexpr int kT = 256;

__global__ void copy_tasks_kernel(const CopyTask* __restrict__ tasks) {
    const CopyTask t = tasks[blockIdx.x];
    const long long total = (long long)t.m * t.n;
    for (long long e = threadIdx.x; e < total; e += kT) {
        int i = (int)(e % t.m), j = (int)(e / t.m);
        double v = t.transpose ? t.src[j + (long long)i * t.lds] : t.src[i + (long long)j * t.lds];
        t.dst[e] = t.alpha * v;
    }
}

struct DiagTask {
    double* D;
    int m, n;
};

__global__ void add_diag_kernel(const DiagTask* __restrict__ tasks, int ntasks, double alpha) {
    const int t = blockIdx.x;
    if (t >= ntasks) return;
    const DiagTask d = tasks[t];
    const int k = min(d.m, d.n);
    for (int j = threadIdx.x; j < k; j += kT) d.D[j + (long long)j * d.m] += alpha;
}

// Gaussian vector (SerialGaussianRandomVector, random.hpp:344-364):
// pairs at rows (2i, 2i+1), the last pair (or single) at (n-2, n-1) / n-1.
__global__ void gaussian_vector_kernel(double* x, int n, unsigned long long base) {
    const int pairs = (n + 1) / 2;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < pairs; p += gridDim.x * blockDim.x) {
        double a, b;
        box_muller(lcg_skip(base, 2ULL * p), a, b);
        if (p < pairs - 1) {
            x[2 * p] = a;
            x[2 * p + 1] = b;
        } else if (n & 1) {
            x[n - 1] = a;
        } else {
            x[n - 2] = a;
            x[n - 1] = b;
        }
    }
}

// Sum of squares, deterministic two-stage reduction.
constexpr int kNormBlocks = 148;

__global__ void sumsq_partial_kernel(const double* __restrict__ x, int n, double* partial) {
    __shared__ double red[kT / 32];
    double s = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) s = fma(x[i], x[i], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kT / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// nrm = sqrt(sum partial); inv = 1/nrm; est *= nrm^root  (root < 0: start,
// est := theta unchanged and only inv is produced).
__global__ void norm_finalize_kernel(const double* partial, int np, double* inv, double* est,
                                     double root) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < np; ++i) s += partial[i];
    const double nrm = sqrt(s);
    *inv = 1.0 / nrm;
    if (root > 0.0) *est *= pow(nrm, root);
}

__global__ void scale_vector_kernel(double* x, int n, const double* inv) {
    const double a = *inv;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] *= a;
}

__global__ void set_scalar_kernel(double* p, double v) { *p = v; }

}  // namespace

void launch_copy_tasks(Context& ctx, const std::vector<CopyTask>& tasks, const char* name) {
    std::vector<CopyTask> live;
    for (const CopyTask& t : tasks)
        if (t.m > 0 && t.n > 0) live.push_back(t);
    if (live.empty()) return;
    DeviceBuffer<CopyTask> d;
    d.upload(live, ctx.stream);
    LaunchScope ls(ctx, name);
    copy_tasks_kernel<<<(unsigned)live.size(), kT, 0, ctx.stream>>>(d.get());
    HMB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Elementwise H-matrix operations
// ---------------------------------------------------------------------------
// Rank actually used by each listed low-rank block: 1 + the last column of U
// with a nonzero entry (tolerance truncation leaves zero columns behind).
__global__ void rank_scan_kernel(const double* const* __restrict__ U, const int* __restrict__ m,
                                 const int* __restrict__ r, int* __restrict__ out) {
    const int b = blockIdx.x;
    const double* u = U[b];
    const int rows = m[b];
    int used = 0;
    for (int c = r[b] - 1; c >= 0; --c) {
        int nz = 0;
        for (int i = threadIdx.x; i < rows; i += blockDim.x) nz |= u[i + (long long)c * rows] != 0.0;
        if (__syncthreads_or(nz)) {
            used = c + 1;
            break;
        }
    }
    if (threadIdx.x == 0) out[b] = used;
}

void compact_ranks(Context& ctx, HMatrix& H) {
    const Structure& S = *H.S;
    std::vector<int> blocks;
    std::vector<const double*> up;
    std::vector<int> ms, rs;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        if (B.kind != KIND_LOWRANK || H.rank[b] == 0 || B.m == 0 || B.n == 0) continue;
        blocks.push_back(b);
        up.push_back(H.U(b));
        ms.push_back(B.m);
        rs.push_back(H.rank[b]);
    }
    if (blocks.empty()) return;
    DeviceBuffer<const double*> du;
    DeviceBuffer<int> dm, dr, dout;
    du.upload(up, ctx.stream);
    dm.upload(ms, ctx.stream);
    dr.upload(rs, ctx.stream);
    dout.allocate(blocks.size(), ctx.stream);
    {
        LaunchScope ls(ctx, "rank_scan");
        rank_scan_kernel<<<(unsigned)blocks.size(), 128, 0, ctx.stream>>>(du.get(), dm.get(), dr.get(),
                                                                          dout.get());
        HMB_CHECK_LAUNCH();
    }
    std::vector<int> used(blocks.size());
    HMB_CUDA(cudaMemcpyAsync(used.data(), dout.get(), used.size() * sizeof(int),
                             cudaMemcpyDeviceToHost, ctx.stream));
    HMB_CUDA(cudaStreamSynchronize(ctx.stream));
    // Re-lay out only when it saves at least 5 % of the low-rank storage: a
    // re-layout changes the ranks, and with them the symbolic plans and cached
    // operation lists of every later product; below that saving the trailing
    // zero columns are kept (they add nothing to any product or rounding).
    long long before = 0, after = 0;
    for (size_t i = 0; i < blocks.size(); ++i) {
        const Block& B = S.blocks[blocks[i]];
        before += (long long)(B.m + B.n) * rs[i];
        after += (long long)(B.m + B.n) * used[i];
    }
    if (after == before || after * 20 >= before * 19) return;
    // re-lay out with the used ranks and copy the kept columns over
    DeviceBuffer<double> old = std::move(H.data);
    const std::vector<long long> old_off = H.off;
    const std::vector<int> old_rank = H.rank;
    for (size_t i = 0; i < blocks.size(); ++i) H.rank[blocks[i]] = used[i];
    H.layout();
    std::vector<CopyTask> tasks;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        const double* src = old.get() + old_off[b];
        if (B.kind == KIND_DENSE) {
            tasks.push_back({src, H.D(b), 1.0, B.m, B.n, B.m, 0});
        } else if (H.rank[b] > 0) {
            tasks.push_back({src, H.U(b), 1.0, B.m, H.rank[b], B.m, 0});
            tasks.push_back({src + (long long)B.m * old_rank[b], H.V(b), 1.0, B.n, H.rank[b], B.n, 0});
        }
    }
    launch_copy_tasks(ctx, tasks, "rank_compact");
}

void hmat_copy(Context& ctx, const HMatrix& src, HMatrix& dst) {
    HMB_REQUIRE(&src != &dst, HM_ERR_ARGUMENT, "copy onto itself");
    dst.ctx = &ctx;
    dst.S = src.S;
    dst.max_rank = src.max_rank;
    dst.rank = src.rank;
    dst.layout();
    if (src.total > 0)
        HMB_CUDA(cudaMemcpyAsync(dst.data.get(), src.data.get(), src.total * sizeof(double),
                                 cudaMemcpyDeviceToDevice, ctx.stream));
}

void hmat_transpose(Context& ctx, const HMatrix& src, HMatrix& dst) {
    HMB_REQUIRE(&src != &dst, HM_ERR_ARGUMENT, "transpose onto itself");
    const Structure& S = *src.S;
    dst.ctx = &ctx;
    dst.S = src.S;
    dst.max_rank = src.max_rank;
    dst.rank.assign(S.blocks.size(), 0);
    for (size_t b = 0; b < S.blocks.size(); ++b)
        if (S.blocks[b].kind == KIND_LOWRANK) dst.rank[b] = src.rank[S.blocks[b].transpose];
    dst.layout();
    std::vector<CopyTask> tasks;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        const int bt = B.transpose;
        if (B.kind == KIND_LOWRANK) {
            const int r = dst.rank[b];
            // (U V^T)^T = V U^T: new U = old V (m x r), new V = old U (n x r)
            tasks.push_back({src.V(bt), dst.U(b), 1.0, B.m, r, B.m, 0});
            tasks.push_back({src.U(bt), dst.V(b), 1.0, B.n, r, B.n, 0});
        } else {
            tasks.push_back({src.D(bt), dst.D(b), 1.0, B.m, B.n, S.blocks[bt].m, 1});
        }
    }
    launch_copy_tasks(ctx, tasks, "transpose_blocks");
}

void hmat_scale(Context& ctx, HMatrix& H, double alpha) {
    const Structure& S = *H.S;
    H.shadow_valid = false;
    if (alpha == 0.0) {
        // Scale(0, LowRank) drops the rank (hmat_tools.hpp, Scale); dense -> 0
        bool any = false;
        for (int b : S.leaves)
            if (S.blocks[b].kind == KIND_LOWRANK && H.rank[b] != 0) { H.rank[b] = 0; any = true; }
        if (any) H.layout();
        if (H.total > 0)
            HMB_CUDA(cudaMemsetAsync(H.data.get(), 0, H.total * sizeof(double), ctx.stream));
        return;
    }
    if (alpha == 1.0) return;
    std::vector<CopyTask> tasks;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        if (B.kind == KIND_LOWRANK)
            tasks.push_back({H.U(b), H.U(b), alpha, B.m, H.rank[b], B.m, 0});
        else
            tasks.push_back({H.D(b), H.D(b), alpha, B.m, B.n, B.m, 0});
    }
    launch_copy_tasks(ctx, tasks, "scale_blocks");
}

void hmat_add_diagonal(Context& ctx, HMatrix& H, double alpha) {
    const Structure& S = *H.S;
    H.shadow_valid = false;
    std::vector<DiagTask> tasks;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        if (B.kind == KIND_DENSE && B.tgt_box == B.src_box) tasks.push_back({H.D(b), B.m, B.n});
    }
    if (tasks.empty()) return;
    DeviceBuffer<DiagTask> d;
    d.upload(tasks, ctx.stream);
    LaunchScope ls(ctx, "add_diagonal");
    add_diag_kernel<<<(unsigned)tasks.size(), kT, 0, ctx.stream>>>(d.get(), (int)tasks.size(),
                                                                   alpha);
    HMB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// EstimateTwoNorm
// ---------------------------------------------------------------------------
// Issues the estimate: its result lands in *result (pinned host memory)
// once `done` completes.
void estimate_two_norm_issue(Context& ctx, HMatrix& A, double theta, double confidence,
                             double* result, cudaEvent_t done) {
    HMB_REQUIRE(theta > 1.0, HM_ERR_ARGUMENT, "theta must be > 1");
    HMB_REQUIRE(confidence > 0.0, HM_ERR_ARGUMENT, "confidence must be positive");
    const int n = A.height();
    // power steps from the matrix's own height (complex rows for the real
    // form of a complex matrix, as the reference's complex instantiation)
    const int nk = n / A.S->dof;
    const int k = (int)std::ceil(std::log(0.8 * std::sqrt((double)nk) * std::pow(10.0, confidence)) /
                                 std::log(theta));
    cudaStream_t st = ctx.stream;
    DeviceBuffer<double> x, y, partial, scal;
    x.allocate(n, st);
    y.allocate(n, st);
    partial.allocate(kNormBlocks, st);
    scal.allocate(2, st);   // [0] = 1/||.||, [1] = estimate
    {
        LaunchScope ls(ctx, "norm_start_vector");
        gaussian_vector_kernel<<<ceil_div((n + 1) / 2, kT), kT, 0, st>>>(x.get(), n,
                                                                        ctx.serial_state);
        HMB_CHECK_LAUNCH();
    }
    ctx.serial_state = lcg_skip_host(ctx.serial_state, 2ULL * (uint64_t)((n + 1) / 2));
    {
        LaunchScope ls(ctx, "norm_reduce");
        set_scalar_kernel<<<1, 1, 0, st>>>(scal.get() + 1, theta);
        sumsq_partial_kernel<<<kNormBlocks, kT, 0, st>>>(x.get(), n, partial.get());
        norm_finalize_kernel<<<1, 32, 0, st>>>(partial.get(), kNormBlocks, scal.get(),
                                               scal.get() + 1, -1.0);
        HMB_CHECK_LAUNCH();
    }
    // x currently unnormalised; its scale is folded into the first product
    // through alpha_scale = 1/||x||.
    const double root = 1.0 / (double)k;
    double* cur = x.get();
    double* nxt = y.get();
    for (int i = 0; i < k; ++i) {
        MatJob job{&A, 0, false, 1.0, 0.0, cur, n, nxt, n, 1, scal.get()};
        run_jobs(ctx, {job});
        LaunchScope ls(ctx, "norm_reduce");
        sumsq_partial_kernel<<<kNormBlocks, kT, 0, st>>>(nxt, n, partial.get());
        norm_finalize_kernel<<<1, 32, 0, st>>>(partial.get(), kNormBlocks, scal.get(),
                                               scal.get() + 1, root);
        HMB_CHECK_LAUNCH();
        std::swap(cur, nxt);
    }
    HMB_CUDA(cudaMemcpyAsync(result, scal.get() + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    HMB_CUDA(cudaEventRecord(done, st));
}

double estimate_two_norm(Context& ctx, HMatrix& A, double theta, double confidence) {
    double* slot = ctx.pinned_scalar();
    cudaEvent_t ev;
    HMB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    try {
        estimate_two_norm_issue(ctx, A, theta, confidence, slot, ev);
        HMB_CUDA(cudaEventSynchronize(ev));
    } catch (...) {
        cudaEventDestroy(ev);
        throw;
    }
    cudaEventDestroy(ev);
    const double est = *slot;
    HMB_REQUIRE(std::isfinite(est), HM_ERR_NUMERICAL,
                "EstimateTwoNorm met NaN or Inf (non-finite block data)");
    return est;
}

// ---------------------------------------------------------------------------
// SchulzInvert
// ---------------------------------------------------------------------------
SchulzResult schulz_invert(Context& ctx, HMatrix& A, int num_iterations, double theta,
                           double confidence, double stop_tol, double mixed_switch) {
    SchulzResult res;
    bool stop = false;
    if (num_iterations <= 0) {
        num_iterations = 30;
        stop = true;
    }
    const double est = estimate_two_norm(ctx, A, theta, confidence);
    res.trace.push_back(est);
    const double alpha = 2.0 / (est * est);
    auto X = std::make_unique<HMatrix>();
    hmat_transpose(ctx, A, *X);
    hmat_scale(ctx, *X, alpha);
    // Mixed precision: an iteration runs its two products in the
    // low-precision phase while the last ||I - X A|| estimate is above
    // mixed_switch (without stop checks: all but the last three
    // iterations).  Newton-Schulz corrects the perturbation of a low-precision
    // step (e_{k+1} ~ e_k^2 + its rounding level), so the FP64 iterations that
    // follow reach the FP64 method's accuracy; the estimates themselves are
    // always FP64.
    const bool was_low = ctx.low_precision;
    struct Restore {
        Context& c;
        bool v;
        ~Restore() { c.low_precision = v; }
    } restore{ctx, was_low};
    double last = std::numeric_limits<double>::infinity();
    cudaEvent_t est_done;
    HMB_CUDA(cudaEventCreateWithFlags(&est_done, cudaEventDisableTiming));
    struct EventGuard {
        cudaEvent_t e;
        ~EventGuard() { cudaEventDestroy(e); }
    } est_guard{est_done};
    int k = 0;
    for (; k < num_iterations; ++k) {
        const bool low = mixed_switch > 0.0 &&
                         (stop ? last > mixed_switch : k + 3 < num_iterations);
        ctx.low_precision = low || was_low;
        if (low) ++res.low_iterations;
        // Tolerance truncation: the products leave their unused trailing
        // columns in place (zero columns past the kept ranks, which later
        // products carry as such), and X is re-laid out at the kept ranks
        // once, after the loop.  Re-laying out inside the loop would change
        // the ranks, and with them every later symbolic plan and cached
        // list, whose rebuild costs more host time than the narrower
        // products save (256^2 mixed with tolerance 1e-10: 57.8 s with a
        // re-layout after every estimate, 39.5 s without).
        HMatrix Z;
        hh_multiply(ctx, *X, A, -1.0, 0.0, Z, true, false);
        if (stop) {
            // X_{k+1} = (2I - X A) X is the same whether or not the stop
            // test passes, so it is issued before the estimate is read: the
            // host prepares it while the device runs the power iteration
            hmat_add_diagonal(ctx, Z, 1.0);
            double* slot = ctx.pinned_scalar();
            estimate_two_norm_issue(ctx, Z, theta, confidence, slot, est_done);
            hmat_add_diagonal(ctx, Z, 1.0);
            auto Xn = std::make_unique<HMatrix>();
            hh_multiply(ctx, Z, *X, 1.0, 0.0, *Xn, true, false);
            HMB_CUDA(cudaEventSynchronize(est_done));
            const double ez = *slot;
            HMB_REQUIRE(std::isfinite(ez), HM_ERR_NUMERICAL,
                        "SchulzInvert: the estimate of ||I - X A|| is NaN or Inf");
            res.trace.push_back(ez);
            last = std::fabs(ez);
            X = std::move(Xn);
            if (std::fabs(ez) < stop_tol && !low) {
                ++k;
                break;
            }
            continue;
        }
        hmat_add_diagonal(ctx, Z, 2.0);
        auto Xn = std::make_unique<HMatrix>();
        hh_multiply(ctx, Z, *X, 1.0, 0.0, *Xn, true, false);
        X = std::move(Xn);
    }
    if (ctx.compression_tol > 0.0) compact_ranks(ctx, *X);
    res.iterations = k;
    // A := X (CopyFrom, Invert-incl.hpp:195): take over X's storage
    A.rank = X->rank;
    A.max_rank = X->max_rank;
    A.off = X->off;
    A.total = X->total;
    A.data = std::move(X->data);
    A.shadow_valid = false;
    A.table = std::move(X->table);
    A.group.reset();
    return res;
}

}  // namespace hmb
