// Block-wise H-matrix updates of the HMat2d / HMat3d API:
//   UpdateWith(alpha, B)   A := alpha B + A (src/HMat2d/HMat2d.cpp:749-781):
//                          low-rank blocks by RoundedUpdate to maxRank
//                          (src/hmat_tools/RoundedUpdate.cpp:14-162: the exact
//                          concatenation when the ranks fit, else QR, SVD,
//                          truncation), dense blocks by Update (D += alpha D_B);
//   SetToIdentity()        (HMat2d.cpp:652-702: every low-rank block empty, dense
//                          diagonal blocks I, the other dense blocks 0).
// Both run on the batched kernels of the H*H product: one rounding op per
// low-rank block in one launch, one worker per dense block for the
// accumulation.
#include "dense_ops.h"
#include "hh.h"
#include "lowrank.h"
#include "schulz.h"

namespace hmb {

void hmat_update_with(Context& ctx, HMatrix& A, double alpha, const HMatrix& B) {
    HMB_REQUIRE(A.S && B.S && (A.S == B.S || same_structure(*A.S, *B.S)), HM_ERR_ARGUMENT,
                "UpdateWith needs both matrices on the same block structure");
    HMB_REQUIRE(&A != &B, HM_ERR_ARGUMENT, "UpdateWith of a matrix with itself");
    const Structure& S = *A.S;
    cudaStream_t st = ctx.stream;
    // new storage: the rank after RoundedUpdate per low-rank block
    DeviceBuffer<double> old = std::move(A.data);
    const std::vector<long long> old_off = A.off;
    const std::vector<int> old_rank = A.rank;
    std::vector<int> rank = A.rank;
    for (int b : S.leaves)
        if (S.blocks[b].kind == KIND_LOWRANK)
            rank[b] = std::min(old_rank[b] + B.rank[b], A.max_rank);
    A.rank = rank;
    A.layout();
    const bool dyn = ctx.compression_tol > 0.0;
    std::vector<RoundOp> ops;
    std::vector<long long> work;
    long long wtotal = 0;
    std::vector<GemmOp> gops;
    std::vector<int> gbegin{0};
    for (int b : S.leaves) {
        const Block& Bl = S.blocks[b];
        if (Bl.m == 0 || Bl.n == 0) continue;
        if (Bl.kind == KIND_DENSE) {
            const double* ad = old.get() + old_off[b];
            gops.push_back({ad, nullptr, A.D(b), 1.0, 0.0, Bl.m, Bl.n, -1, Bl.m, 0, Bl.m, 0, 0});
            gops.push_back({B.D(b), nullptr, A.D(b), alpha, 1.0, Bl.m, Bl.n, -1, Bl.m, 0, Bl.m, 0,
                            0});
            gbegin.push_back((int)gops.size());
            continue;
        }
        const int ra = old_rank[b], rb = B.rank[b], rout = rank[b];
        if (rout == 0) continue;
        RoundOp o{};
        o.m = Bl.m;
        o.n = Bl.n;
        o.alpha = alpha;
        o.beta = 1.0;
        o.u1 = B.U(b);
        o.v1 = B.V(b);
        o.r1 = rb;
        o.ldu1 = Bl.m;
        o.ldv1 = Bl.n;
        o.u2 = old.get() + old_off[b];
        o.v2 = o.u2 + (long long)Bl.m * ra;
        o.r2 = ra;
        o.ldu2 = Bl.m;
        o.ldv2 = Bl.n;
        o.rout = rout;
        o.uo = A.U(b);
        o.vo = A.V(b);
        o.tol = ctx.compression_tol;
        // exact when the ranks fit (and no tolerance asks for a truncation),
        // else the rounding to maxRank
        if (ra + rb <= A.max_rank && !dyn) o.kind = ra == 0 ? ROUND_SET : ROUND_CONCAT;
        else o.kind = ROUND_GENERAL;
        work.push_back(wtotal);
        wtotal += round_work_size(o);
        ops.push_back(o);
    }
    DeviceBuffer<double> wbuf;
    DeviceBuffer<int> kept;
    if (!ops.empty()) {
        wbuf.allocate((size_t)std::max<long long>(wtotal, 2), st);
        if (dyn) kept.allocate(ops.size(), st);
        for (size_t i = 0; i < ops.size(); ++i) {
            ops[i].work = wbuf.get() + work[i];
            if (dyn) ops[i].rank_out = kept.get() + i;
        }
        launch_round_ops(ctx, ops, "update_round");
    }
    launch_gemm_workers(ctx, gops, gbegin, "update_dense");
    if (dyn) compact_ranks(ctx, A);
    HMB_CUDA(cudaStreamSynchronize(st));   // `old` is freed in stream order; B may be reused
}

void hmat_set_identity(Context& ctx, HMatrix& H) {
    HMB_REQUIRE(H.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
    H.rank.assign(H.S->blocks.size(), 0);
    H.layout();
    if (H.total > 0)
        HMB_CUDA(cudaMemsetAsync(H.data.get(), 0, (size_t)H.total * sizeof(double), ctx.stream));
    hmat_add_diagonal(ctx, H, 1.0);
}

}  // namespace hmb
