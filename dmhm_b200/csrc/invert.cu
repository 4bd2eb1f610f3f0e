// DirectInvert: A := inv(A) by recursive block Gauss-Jordan elimination
// with Schur complements, the reference's HMat2d::DirectInvert
// (src/HMat2d/Invert-incl.hpp:17-125; HMat3d: src/HMat3d/Invert-incl.hpp:
// 14-122), with the dense leaves inverted by partial-pivoting elimination as
// hmat_tools::Invert does (getrf + getri, src/hmat_tools/Invert.cpp:14-42).
//
// The reference recurses over the q x q children of every diagonal node
// (q = 4 in 2-D, 8 in 3-D), copying the node into B, setting it to the
// identity and running, for l = 0 .. q-1,
//   A_ll := inv(B_ll)                          (recursion)
//   A_lj := A_ll A_lj           for j < l      (H*H, the block rebuilt)
//   B_lj := A_ll B_lj           for j > l
//   for i > l:  A_ij -= B_il A_lj  (j <= l),   B_ij -= B_il B_lj  (j > l)
// and then, for l = q-1 .. 0 and i < l, A_ij -= B_il A_lj for every j.
// Here every one of those block products is a sub-tree product of the
// engine's H*H executor (hh_multiply_sub), on matrices that keep the whole
// block structure: the products of one statement that write different
// blocks and read none of them are planned and run as one batch, in the
// reference's order, so the serial generator hands every randomized
// compression the draws the reference's sequence of Multiply calls gives
// it.  Factors that would alias the output are read from a copy.
#include <algorithm>
#include <mutex>
#include <set>

#include "hh.h"
#include "schulz.h"

namespace hmb {

namespace {

constexpr int kInvThreads = 256;
constexpr int kMaxLeafInvert = 96;   // [A | I] of a 96 x 96 leaf: 144 KB of shared memory

// In-place inverse of one m x m column-major dense block by Gauss-Jordan
// elimination with partial pivoting on [A | I] in shared memory (row-major,
// 2m columns).  A zero pivot (a singular leaf) sets *numflag and leaves
// the block's non-finite quotient, as the reference's getri would fail.
__global__ void __launch_bounds__(kInvThreads) invert_leaf_kernel(double* D, int m, int* numflag) {
    extern __shared__ __align__(16) double aug[];   // m rows x 2m
    __shared__ double fac[kMaxLeafInvert];
    __shared__ int piv;
    const int w = 2 * m;
    for (int e = threadIdx.x; e < m * w; e += kInvThreads) {
        const int i = e / w, j = e % w;
        aug[e] = j < m ? D[i + (long long)j * m] : (j - m == i ? 1.0 : 0.0);
    }
    __syncthreads();
    for (int k = 0; k < m; ++k) {
        if (threadIdx.x < 32) {
            // pivot: largest |a_ik|, i >= k (first one on ties, as idamax)
            double best = -1.0;
            int bi = k;
            for (int i = k + threadIdx.x; i < m; i += 32) {
                const double v = fabs(aug[i * w + k]);
                if (v > best) { best = v; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (threadIdx.x == 0) {
                piv = bi;
                if (!(best > 0.0) && numflag) atomicOr(numflag, 1);
            }
        }
        __syncthreads();
        const int p = piv;
        if (p != k)
            for (int j = threadIdx.x; j < w; j += kInvThreads) {
                const double t = aug[k * w + j];
                aug[k * w + j] = aug[p * w + j];
                aug[p * w + j] = t;
            }
        __syncthreads();
        const double inv = 1.0 / aug[k * w + k];
        for (int i = threadIdx.x; i < m; i += kInvThreads) fac[i] = aug[i * w + k];
        __syncthreads();
        for (int j = threadIdx.x; j < w; j += kInvThreads) aug[k * w + j] *= inv;
        __syncthreads();
        for (int e = threadIdx.x; e < m * w; e += kInvThreads) {
            const int i = e / w, j = e % w;
            if (i != k) aug[e] = fma(-fac[i], aug[k * w + j], aug[e]);
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < m * m; e += kInvThreads) {
        const int i = e % m, j = e / m;
        D[e] = aug[i * w + m + j];
    }
}

void invert_dense_leaf(Context& ctx, HMatrix& X, int b) {
    const Block& B = X.S->blocks[b];
    HMB_REQUIRE(B.m == B.n, HM_ERR_ARGUMENT, "Cannot invert non-square matrices");
    HMB_REQUIRE(B.m <= kMaxLeafInvert, HM_ERR_UNSUPPORTED,
                "DirectInvert handles dense leaves of at most 96 rows");
    if (B.m == 0) return;
    const size_t smem = (size_t)B.m * 2 * B.m * sizeof(double);
    {
        // once per device (contexts on several host threads may get here at once)
        int dev = 0;
        HMB_CUDA(cudaGetDevice(&dev));
        static std::mutex mu;
        static std::set<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (done.insert(dev).second)
            HMB_CUDA(cudaFuncSetAttribute(
                invert_leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)(kMaxLeafInvert * 2 * kMaxLeafInvert * sizeof(double))));
    }
    X.shadow_valid = false;
    LaunchScope ls(ctx, "invert_leaf");
    invert_leaf_kernel<<<1, kInvThreads, smem, ctx.stream>>>(X.D(b), B.m, ctx.numerical_word());
    HMB_CHECK_LAUNCH();
}

// Re-lays X out with new ranks; every leaf is filled by `fill` (copy tasks
// appended for it) from the old storage or elsewhere.  Old storage is freed
// in stream order after the copies.
template <typename Fill>
void relayout(Context& ctx, HMatrix& X, const std::vector<int>& new_rank, Fill fill) {
    DeviceBuffer<double> old = std::move(X.data);
    const std::vector<long long> old_off = X.off;
    const std::vector<int> old_rank = X.rank;
    X.rank = new_rank;
    X.layout();
    if (X.total > 0)
        HMB_CUDA(cudaMemsetAsync(X.data.get(), 0, (size_t)X.total * sizeof(double), ctx.stream));
    std::vector<CopyTask> tasks;
    for (int b : X.S->leaves) fill(b, old.get() + old_off[b], old_rank[b], tasks);
    launch_copy_tasks(ctx, tasks, "subtree_copy");
}

void copy_block(const Structure& S, int b, const double* src, int src_rank, const HMatrix& X,
                std::vector<CopyTask>& tasks) {
    const Block& B = S.blocks[b];
    if (B.kind == KIND_DENSE) {
        tasks.push_back({src, X.D(b), 1.0, B.m, B.n, B.m, 0});
    } else if (X.rank[b] > 0) {
        tasks.push_back({src, X.U(b), 1.0, B.m, X.rank[b], B.m, 0});
        tasks.push_back({src + (long long)B.m * src_rank, X.V(b), 1.0, B.n, X.rank[b], B.n, 0});
    }
}

// X's sub-tree at `root` := src's (CopyFrom of a child, Invert-incl.hpp:44).
void subtree_assign(Context& ctx, HMatrix& X, const HMatrix& src, int root) {
    const Structure& S = *X.S;
    std::vector<int> nr = X.rank;
    for (int b : S.leaves)
        if (S.in_subtree(b, root)) nr[b] = src.rank[b];
    relayout(ctx, X, nr, [&](int b, const double* old, int old_rank, std::vector<CopyTask>& t) {
        if (S.in_subtree(b, root)) copy_block(S, b, src.data.get() + src.off[b], src.rank[b], X, t);
        else copy_block(S, b, old, old_rank, X, t);
    });
}

__global__ void unit_diagonal_kernel(double* const* __restrict__ D, const int* __restrict__ m) {
    double* d = D[blockIdx.x];
    const int n = m[blockIdx.x];
    for (int j = threadIdx.x; j < n; j += blockDim.x) d[j + (long long)j * n] = 1.0;
}

// X's sub-tree at `root` := identity (SetToIdentity of a node, Invert-incl.hpp:34;
// HMat2d.cpp:652-702: empty low-rank blocks, identity on the dense diagonal).
void subtree_set_identity(Context& ctx, HMatrix& X, int root) {
    const Structure& S = *X.S;
    std::vector<int> nr = X.rank;
    for (int b : S.leaves)
        if (S.in_subtree(b, root) && S.blocks[b].kind == KIND_LOWRANK) nr[b] = 0;
    relayout(ctx, X, nr, [&](int b, const double* old, int old_rank, std::vector<CopyTask>& t) {
        if (!S.in_subtree(b, root)) copy_block(S, b, old, old_rank, X, t);
    });
    std::vector<double*> d;
    std::vector<int> m;
    for (int b : S.leaves) {
        const Block& B = S.blocks[b];
        if (B.kind == KIND_DENSE && S.in_subtree(b, root) && B.row_off == B.col_off && B.m > 0) {
            d.push_back(X.D(b));
            m.push_back(B.m);
        }
    }
    if (d.empty()) return;
    DeviceBuffer<double*> dd;
    DeviceBuffer<int> dm;
    dd.upload(d, ctx.stream);
    dm.upload(m, ctx.stream);
    LaunchScope ls(ctx, "subtree_identity");
    unit_diagonal_kernel<<<(unsigned)d.size(), 128, 0, ctx.stream>>>(dd.get(), dm.get());
    HMB_CHECK_LAUNCH();
}

void invert_node(Context& ctx, HMatrix& X, int root) {
    const Structure& S = *X.S;
    const Block& R = S.blocks[root];
    if (R.kind == KIND_DENSE) {
        invert_dense_leaf(ctx, X, root);
        return;
    }
    HMB_REQUIRE(R.kind == KIND_NODE, HM_ERR_UNSUPPORTED, "Cannot invert low-rank matrices");
    const int q = S.q;
    auto ch = [&](int t, int s) { return S.child(root, t, s); };
    HMatrix B;
    hmat_copy(ctx, X, B);               // B.CopyFrom(*this)
    subtree_set_identity(ctx, X, root);  // SetToIdentity()
    for (int l = 0; l < q; ++l) {
        subtree_assign(ctx, X, B, ch(l, l));   // A_ll := B_ll
        invert_node(ctx, X, ch(l, l));         // A_ll := inv(A_ll)
        if (l > 0) {                           // A_lj := A_ll A_lj, j < l
            HMatrix Xc;
            hmat_copy(ctx, X, Xc);
            std::vector<HHRoot> r;
            for (int j = 0; j < l; ++j) r.push_back({ch(l, l), ch(l, j), ch(l, j)});
            hh_multiply_sub(ctx, Xc, Xc, 1.0, 0.0, X, true, r);
        }
        if (l + 1 < q) {                       // B_lj := A_ll B_lj, j > l
            HMatrix Bc;
            hmat_copy(ctx, B, Bc);
            std::vector<HHRoot> r;
            for (int j = l + 1; j < q; ++j) r.push_back({ch(l, l), ch(l, j), ch(l, j)});
            hh_multiply_sub(ctx, X, Bc, 1.0, 0.0, B, true, r);
        }
        for (int i = l + 1; i < q; ++i) {
            {                                  // A_ij -= B_il A_lj, j <= l
                HMatrix Xc;
                hmat_copy(ctx, X, Xc);
                std::vector<HHRoot> r;
                for (int j = 0; j <= l; ++j) r.push_back({ch(i, l), ch(l, j), ch(i, j)});
                hh_multiply_sub(ctx, B, Xc, -1.0, 1.0, X, false, r);
            }
            if (l + 1 < q) {                   // B_ij -= B_il B_lj, j > l
                HMatrix Bc;
                hmat_copy(ctx, B, Bc);
                std::vector<HHRoot> r;
                for (int j = l + 1; j < q; ++j) r.push_back({ch(i, l), ch(l, j), ch(i, j)});
                hh_multiply_sub(ctx, Bc, Bc, -1.0, 1.0, B, false, r);
            }
        }
    }
    for (int l = q - 1; l >= 0; --l) {         // A_ij -= B_il A_lj, i < l, all j
        if (l == 0) break;
        HMatrix Xc;
        hmat_copy(ctx, X, Xc);
        std::vector<HHRoot> r;
        for (int i = l - 1; i >= 0; --i)
            for (int j = 0; j < q; ++j) r.push_back({ch(i, l), ch(l, j), ch(i, j)});
        hh_multiply_sub(ctx, B, Xc, -1.0, 1.0, X, false, r);
    }
}

}  // namespace

void hmat_direct_invert(Context& ctx, HMatrix& X) {
    HMB_REQUIRE(X.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
    HMB_REQUIRE(X.S->dof == 1, HM_ERR_UNSUPPORTED, "DirectInvert is built for real matrices");
    HMB_REQUIRE(X.S->blocks[0].kind != KIND_LOWRANK, HM_ERR_UNSUPPORTED,
                "Cannot invert low-rank matrices");
    // the serial HMat2d / HMat3d products truncate to the fixed rank maxRank,
    // in FP64: the context's tolerance and low-precision phase are set aside
    // for the call and restored afterwards
    const double tol = ctx.compression_tol;
    const bool low = ctx.low_precision;
    ctx.compression_tol = 0.0;
    ctx.low_precision = false;
    try {
        invert_node(ctx, X, 0);
    } catch (...) {
        ctx.compression_tol = tol;
        ctx.low_precision = low;
        throw;
    }
    ctx.compression_tol = tol;
    ctx.low_precision = low;
    ctx.check_numerical();
}

}  // namespace hmb
