// Low-rank approximation of a whole H-matrix product as ONE low-rank matrix:
// hmat_tools::Multiply (F := alpha A B, include/dmhm/hmat_tools.hpp:1657-1746),
// TransposeMultiply (F := alpha A^T B, :1848-1937) and AdjointMultiply
// (F := alpha A^H B, :2039-; the same as TransposeMultiply for real scalars).
//
// The randomized range finder of the reference, on the batched device paths:
//   Omega = SerialGaussianRandomVectors(n x sampleRank)   (context's generator)
//   Y     = A (alpha B Omega)       or A^T (alpha B Omega)  (H-matmat kernels)
//   Q     = orth(Y)                 (Householder QR; the reference's pivoted
//                                    QR spans the same space)
//   Z     = B^T (alpha A^T Q)       or B^T (alpha A Q)
//   F     = best rank-r of Q Z^T    (the rounding kernel's orthogonal form:
//                                    QR of Z, Jacobi SVD of the core)
// with r = min(A.MaxRank(), B.MaxRank(), n).  The reference truncates to r
// exactly; with a compression tolerance set on the context the singular
// values at or below tol * sigma_0 are dropped as in the H*H compressions.
#include "lowrank.h"
#include "rng.cuh"

namespace hmb {

int low_rank_product(Context& ctx, const HMatrix& A, int op, double alpha, const HMatrix& B,
                     int sample_rank, DeviceBuffer<double>& U, DeviceBuffer<double>& V) {
    HMB_REQUIRE(A.S && B.S && (A.S == B.S || same_structure(*A.S, *B.S)), HM_ERR_ARGUMENT,
                "the factors must share one block structure");
    HMB_REQUIRE(A.S->dof == 1, HM_ERR_UNSUPPORTED,
                "low-rank products of complex H-matrices are not supported");
    HMB_REQUIRE(op >= 0 && op <= 2, HM_ERR_ARGUMENT, "op must be 0 (A B), 1 (A^T B) or 2 (A^H B)");
    const int n = A.height();
    // SerialGaussianRandomVectors writes the tail of every column at rows
    // sampleRank-2, sampleRank-1 (random.hpp:440-443): more samples than rows
    // would write past the column
    HMB_REQUIRE(sample_rank >= 1 && sample_rank <= n, HM_ERR_ARGUMENT,
                "sample rank must be in [1, height]");
    const int s = sample_rank;
    const int kq = std::min(n, s);
    const int r = std::min(std::min(std::min(A.max_rank, B.max_rank), n), kq);
    cudaStream_t st = ctx.stream;
    DeviceBuffer<double> omega, X, Y, Q, tau, Z1, Z, work;
    DeviceBuffer<int> kept;
    omega.allocate((size_t)n * s, st);
    X.allocate((size_t)n * s, st);
    Y.allocate((size_t)n * s, st);
    Q.allocate((size_t)n * kq, st);
    tau.allocate((size_t)s, st);
    Z1.allocate((size_t)n * kq, st);
    Z.allocate((size_t)n * kq, st);
    U.allocate((size_t)std::max(n * r, 1), st);
    V.allocate((size_t)std::max(n * r, 1), st);
    launch_gaussian_fills(ctx, {FillOp{omega.get(), ctx.serial_state, n, s}}, "lrprod_omega");
    ctx.serial_state = lcg_skip_host(ctx.serial_state, (uint64_t)s * 2ULL * (uint64_t)((n + 1) / 2));
    const bool tr = op != 0;
    run_jobs(ctx, {MatJob{&B, 0, false, alpha, 0.0, omega.get(), n, X.get(), n, s}});
    run_jobs(ctx, {MatJob{&A, 0, tr, 1.0, 0.0, X.get(), n, Y.get(), n, s}});
    launch_qr_formq(ctx, {QrOp{Y.get(), Q.get(), tau.get(), n, s, n, 0}}, "lrprod_qr");
    run_jobs(ctx, {MatJob{&A, 0, !tr, alpha, 0.0, Q.get(), n, Z1.get(), n, kq}});
    run_jobs(ctx, {MatJob{&B, 0, true, 1.0, 0.0, Z1.get(), n, Z.get(), n, kq}});
    if (r == 0) return 0;
    RoundOp o{};
    o.kind = ROUND_ORTHO;
    o.m = n;
    o.n = n;
    o.u1 = Q.get();
    o.ldu1 = n;
    o.r1 = kq;
    o.v1 = Z.get();
    o.ldv1 = n;
    o.rout = r;
    o.uo = U.get();
    o.vo = V.get();
    o.alpha = 1.0;
    o.tol = ctx.compression_tol;
    work.allocate((size_t)std::max<long long>(round_work_size(o), 2), st);
    o.work = work.get();
    if (o.tol > 0.0) {
        kept.allocate(1, st);
        o.rank_out = kept.get();
    }
    std::vector<RoundOp> ops{o};
    launch_round_ops(ctx, ops, "lrprod_round");
    int rank = r;
    if (o.tol > 0.0) {
        HMB_CUDA(cudaMemcpyAsync(&rank, kept.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        HMB_CUDA(cudaStreamSynchronize(st));
    }
    return rank;
}

}  // namespace hmb
