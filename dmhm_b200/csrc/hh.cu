// H*H product (HMat2d::Multiply against an H-matrix) as a host symbolic
// phase plus level-batched device phases.
//
// The reference (src/HMat2d/MultiplyHMat-incl.hpp:12-380; 3-D
// src/HMat3d/MultiplyHMat-incl.hpp) recurses over the t, s, u children of
// every non-admissible node, forming for each (A-block, B-block) pair a
// low-rank or dense product W and folding it into the matching C block in a
// fixed order: first product sets the block, later ones are added with
// RoundedUpdate (fixed-rank truncation to maxRank), pushed down through
// ImportLowRank / UpdateWithLowRank (src/HMat2d/HMat2d.cpp:811-959), or
// accumulated into dense leaves.  Randomized sampling
// (include/dmhm/hmat_tools.hpp:1657-1746) handles node x node products and
// draws its Gaussian test matrix from the serial generator in recursion
// order.
//
// Here the same recursion runs once on the host, on block ids only, and
// records (a) every product W with its kind, size and rank, (b) for every C
// leaf block the ordered list of operations it receives, and (c) the
// generator position of every sampled product.  All ranks follow from the
// structure, so every buffer is sized before any device work.  The device
// then
//   1. draws all Gaussian test matrices at once (skip-ahead LCG),
//   2. runs all H-matrix x dense products of all samplings as four batched
//      launch pairs (B Omega, A X, A^T Q, B^T Z), orthonormalizes all samples
//      in one launch and rounds all sampled products in one launch,
//   3. forms all leaf-level products in two batched GEMM launches,
//   4. applies the per-block operation lists in waves: wave j performs the
//      j-th operation of every C block (one rounding launch and one dense
//      launch per wave), which keeps the reference's order within each block
//      while all blocks proceed in parallel.
#include "hh.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "dense_ops.h"
#include "lowrank.h"
#include "schulz.h"
#include "mlp.h"
#include "rng.cuh"

namespace hmb {

namespace {

enum WType { W_LRLR, W_LRH, W_LRD, W_HLR, W_DLR, W_HH, W_DD };

struct WTask {
    int type;
    int a, b;
    int c = -1;           // the C block the product is folded into (sampled products)
    double alpha;
    int m, n, r;          // W: m x n; rank r (low-rank) or dense
    // storage: aliases into A/B or owned slots in the W arena
    const double* U = nullptr;
    const double* V = nullptr;
    const double* D = nullptr;
    int ldU = 0, ldV = 0;
    long long u_off = -1, v_off = -1, d_off = -1, g_off = -1;
    bool u_alias = false, v_alias = false;   // U is A's block's U / V is B's block's V
    // randomized sampling
    int k = 0, kq = 0;
    uint64_t omega = 0;
    uint64_t omega_steps = 0;   // serial-generator draws before this sample's
    long long s_omega = -1, s_x = -1, s_y = -1, s_q = -1, s_tau = -1, s_z1 = -1, s_z = -1,
              s_work = -1;
};

enum LType { L_SET, L_RUPD, L_DDC, L_RESET };
struct LOp {
    int type;
    int w;
    int row0, col0;   // restriction of W: rows of U / rows of V
    double beta;
};

enum DType { D_LR, D_DD, D_COPY };
struct DOp {
    int type;
    int w;
    int row0, col0;
    double alpha, beta;
    int a, b;
};

// Operations grouped per C block: appended in recursion order, then grouped
// by block with a stable counting sort (order inside a block is preserved).
template <typename T>
struct PerBlock {
    std::vector<int> blk;
    std::vector<T> raw;
    std::vector<int> begin;
    std::vector<T> ops;
    void push(int c, const T& op) {
        blk.push_back(c);
        raw.push_back(op);
    }
    void finalize(size_t nblocks) {
        begin.assign(nblocks + 1, 0);
        for (int c : blk) begin[c + 1]++;
        for (size_t c = 0; c < nblocks; ++c) begin[c + 1] += begin[c];
        ops.resize(raw.size());
        std::vector<int> fill(begin.begin(), begin.end() - 1);
        for (size_t i = 0; i < raw.size(); ++i) ops[fill[blk[i]]++] = raw[i];
        std::vector<int>().swap(blk);
        std::vector<T>().swap(raw);
    }
    int size(int c) const { return begin[c + 1] - begin[c]; }
    const T* of(int c) const { return ops.data() + begin[c]; }
};

struct Planner {
    const Structure& S;
    const HMatrix& A;
    const HMatrix& B;
    int maxRankC;
    int oversample;
    uint64_t serial;
    uint64_t steps = 0;   // serial-generator draws so far
    std::vector<WTask> w;
    PerBlock<LOp> lops;
    PerBlock<DOp> dops;

    Planner(const HMatrix& a, const HMatrix& b, int maxRank, int over, uint64_t st)
        : S(*a.S), A(a), B(b), maxRankC(maxRank), oversample(over), serial(st) {}

    int kind(int blk) const { return S.blocks[blk].kind; }

    int product(int a, int b, double alpha) {
        WTask t{};
        t.a = a;
        t.b = b;
        t.alpha = alpha;
        t.m = S.blocks[a].m;
        t.n = S.blocks[b].n;
        const int ka = kind(a), kb = kind(b);
        if (ka == KIND_LOWRANK && kb == KIND_LOWRANK) {
            t.type = W_LRLR;
            t.r = std::min(A.rank[a], B.rank[b]);
        } else if (ka == KIND_LOWRANK && kb == KIND_NODE) {
            t.type = W_LRH;
            t.r = A.rank[a];
        } else if (ka == KIND_LOWRANK && kb == KIND_DENSE) {
            t.type = W_LRD;
            t.r = A.rank[a];
        } else if (ka == KIND_NODE && kb == KIND_LOWRANK) {
            t.type = W_HLR;
            t.r = B.rank[b];
        } else if (ka == KIND_DENSE && kb == KIND_LOWRANK) {
            t.type = W_DLR;
            t.r = B.rank[b];
        } else if (ka == KIND_NODE && kb == KIND_NODE) {
            t.type = W_HH;
            const Block& BA = S.blocks[a];
            const Block& BB = S.blocks[b];
            t.r = std::min(std::min(A.max_rank, B.max_rank),
                           std::min(std::min(BA.m, BA.n), std::min(BB.m, BB.n)));
            t.k = maxRankC + oversample;
            HMB_REQUIRE(t.k <= BB.n, HM_ERR_UNSUPPORTED,
                        "sample count exceeds the sampled block width (the reference's "
                        "Gaussian fill would write past its columns)");
            t.kq = std::min(BA.m, t.k);
            t.omega = serial;
            t.omega_steps = steps;
            const uint64_t draws = (uint64_t)t.k * 2ULL * (uint64_t)((BB.n + 1) / 2);
            serial = lcg_skip_host(serial, draws);
            steps += draws;
        } else if (ka == KIND_DENSE && kb == KIND_DENSE) {
            t.type = W_DD;
            t.r = -1;
        } else {
            throw Error(HM_ERR_UNSUPPORTED, "invalid H-matrix combination");
        }
        w.push_back(t);
        return (int)w.size() - 1;
    }

    // Multiply(alpha, B, C): C rebuilt (MultiplyHMat-incl.hpp:12-187)
    void fresh(int a, int b, int c, double alpha) {
        const int kc = kind(c);
        if (kc == KIND_LOWRANK) {
            int t = product(a, b, alpha);
            w[t].c = c;
            lops.push(c, {w[t].type == W_DD ? L_DDC : L_SET, t, 0, 0, 0.0});
        } else if (kc == KIND_NODE) {
            HMB_REQUIRE(kind(a) != KIND_DENSE && kind(b) != KIND_DENSE, HM_ERR_UNSUPPORTED,
                        "invalid H-matrix combination");
            if (kind(a) == KIND_LOWRANK || kind(b) == KIND_LOWRANK) {
                int t = product(a, b, alpha);
                import_lowrank(c, t, 0, 0);
            } else {
                for (int ti = 0; ti < S.q; ++ti)
                    for (int si = 0; si < S.q; ++si) {
                        fresh(S.child(a, ti, 0), S.child(b, 0, si), S.child(c, ti, si), alpha);
                        for (int u = 1; u < S.q; ++u)
                            update(S.child(a, ti, u), S.child(b, u, si), S.child(c, ti, si),
                                   alpha, 1.0);
                    }
            }
        } else {
            dense_into(c, a, b, alpha, 0.0);
        }
    }

    // Multiply(alpha, B, beta, C) (MultiplyHMat-incl.hpp:189-380)
    void update(int a, int b, int c, double alpha, double beta) {
        const int kc = kind(c);
        if (kc == KIND_LOWRANK) {
            int t = product(a, b, alpha);
            w[t].c = c;
            lops.push(c, {w[t].type == W_DD ? L_DDC : L_RUPD, t, 0, 0, beta});
        } else if (kc == KIND_NODE) {
            HMB_REQUIRE(kind(a) != KIND_DENSE && kind(b) != KIND_DENSE, HM_ERR_UNSUPPORTED,
                        "invalid H-matrix combination");
            if (kind(a) == KIND_LOWRANK || kind(b) == KIND_LOWRANK) {
                int t = product(a, b, alpha);
                update_with_lowrank(c, t, 0, 0, beta);
            } else {
                for (int ti = 0; ti < S.q; ++ti)
                    for (int si = 0; si < S.q; ++si) {
                        update(S.child(a, ti, 0), S.child(b, 0, si), S.child(c, ti, si), alpha,
                               beta);
                        for (int u = 1; u < S.q; ++u)
                            update(S.child(a, ti, u), S.child(b, u, si), S.child(c, ti, si),
                                   alpha, 1.0);
                    }
            }
        } else {
            dense_into(c, a, b, alpha, beta);
        }
    }

    void dense_into(int c, int a, int b, double alpha, double beta) {
        HMB_REQUIRE(kind(a) != KIND_NODE && kind(b) != KIND_NODE, HM_ERR_UNSUPPORTED,
                    "invalid H-matrix combination");
        if (kind(a) == KIND_DENSE && kind(b) == KIND_DENSE) {
            dops.push(c, {D_DD, -1, 0, 0, alpha, beta, a, b});
        } else {
            int t = product(a, b, alpha);
            dops.push(c, {D_LR, t, 0, 0, 1.0, beta, -1, -1});
        }
    }

    // ImportLowRank (HMat2d.cpp:811-904)
    void import_lowrank(int c, int t, int row0, int col0) {
        const Block& C = S.blocks[c];
        if (C.kind == KIND_LOWRANK) {
            lops.push(c, {L_SET, t, row0, col0, 0.0});
        } else if (C.kind == KIND_NODE) {
            for (int ti = 0; ti < S.q; ++ti)
                for (int si = 0; si < S.q; ++si) {
                    int ch = S.child(c, ti, si);
                    import_lowrank(ch, t, row0 + S.blocks[ch].row_off - C.row_off,
                                   col0 + S.blocks[ch].col_off - C.col_off);
                }
        } else {
            dops.push(c, {D_LR, t, row0, col0, 1.0, 0.0, -1, -1});
        }
    }

    // Scale(beta) followed by UpdateWithLowRank(1, W) (HMat2d.cpp:906-959)
    void update_with_lowrank(int c, int t, int row0, int col0, double beta) {
        const Block& C = S.blocks[c];
        if (C.kind == KIND_LOWRANK) {
            if (beta == 0.0) lops.push(c, {L_RESET, -1, 0, 0, 0.0});
            lops.push(c, {L_RUPD, t, row0, col0, beta == 0.0 ? 1.0 : beta});
        } else if (C.kind == KIND_NODE) {
            for (int ti = 0; ti < S.q; ++ti)
                for (int si = 0; si < S.q; ++si) {
                    int ch = S.child(c, ti, si);
                    update_with_lowrank(ch, t, row0 + S.blocks[ch].row_off - C.row_off,
                                        col0 + S.blocks[ch].col_off - C.col_off, beta);
                }
        } else {
            dops.push(c, {D_LR, t, row0, col0, 1.0, beta, -1, -1});
        }
    }
};

// A slot of a scratch arena handed out by offsets (doubles), 16-byte aligned.
struct Arena {
    long long used = 0;
    long long take(long long n) {
        long long o = used;
        used += (std::max<long long>(n, 0) + 1) & ~1LL;
        return o;
    }
};

// Features of the randomized compressions (the rank predictor's inputs, all
// in [0, 1] roughly):
//   0 level / numLevels      1 log2(1 + m) / 16     2 log2(1 + n) / 16
//   3 admissibility distance max|coord_t - coord_s| / 8 (capped at 1)
//   4, 5 mean rank of the low-rank leaves below A's / B's block / maxRank
//   6, 7 share of dense entries below A's / B's block
//   8 rank cap of the product / maxRank             9 dimension / 3
//  10 mean rank of A's low-rank leaves at the C block's own position / maxRank
//     (in a Schulz iteration A is the previous iterate, so this is the rank
//     the same block kept one product earlier)
//  11 the same over the C block's siblings (the other children of its parent)
struct SubtreeStat {
    double rank_sum = 0, lr_count = 0, dense_entries = 0, lr_entries = 0;
    bool done = false;
};

void subtree_stats(const Structure& S, const HMatrix& H, int b, std::vector<SubtreeStat>& st) {
    if (st[b].done) return;
    SubtreeStat s;
    const Block& B = S.blocks[b];
    if (B.kind == KIND_NODE) {
        for (int c = 0; c < S.q * S.q; ++c) {
            const int ch = B.first_child + c;
            subtree_stats(S, H, ch, st);
            s.rank_sum += st[ch].rank_sum;
            s.lr_count += st[ch].lr_count;
            s.dense_entries += st[ch].dense_entries;
            s.lr_entries += st[ch].lr_entries;
        }
    } else if (B.kind == KIND_DENSE) {
        s.dense_entries = (double)B.m * B.n;
    } else {
        s.rank_sum = H.rank[b];
        s.lr_count = 1;
        s.lr_entries = (double)(B.m + B.n) * H.rank[b];
    }
    s.done = true;
    st[b] = s;
}

std::vector<float> rank_features(const Structure& S, const HMatrix& A, const HMatrix& B,
                                 const std::vector<WTask>& w, const std::vector<int>& ids,
                                 int maxRank) {
    std::vector<SubtreeStat> sa(S.blocks.size()), sb(S.blocks.size());
    std::vector<float> f;
    f.reserve(ids.size() * kMlpFeatures);
    const float mr = (float)std::max(1, maxRank);
    for (int i : ids) {
        const WTask& t = w[i];
        subtree_stats(S, A, t.a, sa);
        subtree_stats(S, B, t.b, sb);
        const Block& Ba = S.blocks[t.a];
        const Block& Bb = S.blocks[t.b];
        const Box& tb = S.boxes[Ba.tgt_box];
        const Box& xb = S.boxes[Bb.src_box];
        int dist = 0;
        for (int d = 0; d < S.dim; ++d) dist = std::max(dist, std::abs(tb.coord[d] - xb.coord[d]));
        const SubtreeStat& A1 = sa[t.a];
        const SubtreeStat& B1 = sb[t.b];
        auto frac = [](double d, double l) { return (float)(d + l > 0 ? d / (d + l) : 0.0); };
        f.push_back((float)Ba.level / (float)std::max(1, S.num_levels));
        f.push_back(std::log2(1.0f + (float)t.m) / 16.0f);
        f.push_back(std::log2(1.0f + (float)t.n) / 16.0f);
        f.push_back(std::min(1.0f, (float)dist / 8.0f));
        f.push_back(A1.lr_count > 0 ? (float)(A1.rank_sum / A1.lr_count) / mr : 0.0f);
        f.push_back(B1.lr_count > 0 ? (float)(B1.rank_sum / B1.lr_count) / mr : 0.0f);
        f.push_back(frac(A1.dense_entries, A1.lr_entries));
        f.push_back(frac(B1.dense_entries, B1.lr_entries));
        f.push_back((float)t.r / mr);
        f.push_back((float)S.dim / 3.0f);
        float own = 0.0f, sib = 0.0f;
        if (t.c >= 0) {
            subtree_stats(S, A, t.c, sa);
            if (sa[t.c].lr_count > 0) own = (float)(sa[t.c].rank_sum / sa[t.c].lr_count) / mr;
            const int par = S.blocks[t.c].parent;
            if (par >= 0) {
                double rs = 0.0, lc = 0.0;
                for (int q = 0; q < S.q * S.q; ++q) {
                    const int chb = S.blocks[par].first_child + q;
                    if (chb == t.c) continue;
                    subtree_stats(S, A, chb, sa);
                    rs += sa[chb].rank_sum;
                    lc += sa[chb].lr_count;
                }
                if (lc > 0) sib = (float)(rs / lc) / mr;
            }
        }
        f.push_back(own);
        f.push_back(sib);
    }
    return f;
}

__global__ void sq_norms_kernel(const double* const* __restrict__ p, const long long* __restrict__ n,
                                double* __restrict__ out) {
    __shared__ double red[256];
    const double* x = p[blockIdx.x];
    double s = 0.0;
    for (long long e = threadIdx.x; e < n[blockIdx.x]; e += 256) s = fma(x[e], x[e], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// Squared Frobenius norms of the listed arrays into out[0 .. n) on the
// device (no host synchronization).
void sq_norms_device(Context& ctx, const std::vector<const double*>& ptr,
                     const std::vector<long long>& len, double* out) {
    if (ptr.empty()) return;
    DeviceBuffer<const double*> dp;
    DeviceBuffer<long long> dl;
    dp.upload(ptr, ctx.stream);
    dl.upload(len, ctx.stream);
    LaunchScope ls(ctx, "probe_norms");
    sq_norms_kernel<<<(unsigned)ptr.size(), 256, 0, ctx.stream>>>(dp.get(), dl.get(), out);
    HMB_CHECK_LAUNCH();
}

// Relative error of every listed compression W ~= alpha A_a B_b, estimated
// with q Gaussian probe vectors G: ||A (alpha B G) - U (V^T G)|| / ||A (alpha B G)||.
std::vector<double> probe_errors(Context& ctx, const Structure& S, const HMatrix& A,
                                 const HMatrix& B, const std::vector<WTask>& w,
                                 const std::vector<int>& ids) {
    const int q = std::max(1, ctx.rank_probes);
    Arena ar;
    std::vector<long long> g_off(ids.size()), x_off(ids.size()), y_off(ids.size()), v_off(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) {
        const WTask& t = w[ids[i]];
        g_off[i] = ar.take((long long)S.blocks[t.b].n * q);
        x_off[i] = ar.take((long long)S.blocks[t.b].m * q);
        y_off[i] = ar.take((long long)t.m * q);
        v_off[i] = ar.take((long long)t.r * q);
    }
    DeviceBuffer<double> buf;
    buf.allocate((size_t)std::max<long long>(ar.used, 2), ctx.stream);
    double* P0 = buf.get();
    // probes from the parallel generator's stream, past the current state
    uint64_t state = lcg_skip_host(ctx.parallel_state, 0x5DEECE66DULL);
    std::vector<FillOp> fills;
    for (size_t i = 0; i < ids.size(); ++i) {
        const int n = S.blocks[w[ids[i]].b].n;
        fills.push_back({P0 + g_off[i], state, n, q});
        state = lcg_skip_host(state, 2ULL * (uint64_t)q * (uint64_t)(n + 1));
    }
    launch_gaussian_fills(ctx, fills, "probe_fill");
    std::vector<MatJob> jobs;
    for (size_t i = 0; i < ids.size(); ++i) {
        const WTask& t = w[ids[i]];
        const Block& Bb = S.blocks[t.b];
        jobs.push_back({&B, t.b, false, t.alpha, 0.0, P0 + g_off[i], Bb.n, P0 + x_off[i], Bb.m, q});
    }
    run_jobs(ctx, jobs);
    jobs.clear();
    for (size_t i = 0; i < ids.size(); ++i) {
        const WTask& t = w[ids[i]];
        const Block& Ba = S.blocks[t.a];
        jobs.push_back({&A, t.a, false, 1.0, 0.0, P0 + x_off[i], Ba.n, P0 + y_off[i], Ba.m, q});
    }
    run_jobs(ctx, jobs);
    std::vector<const double*> ptr(ids.size());
    std::vector<long long> len(ids.size());
    for (size_t i = 0; i < ids.size(); ++i) {
        ptr[i] = P0 + y_off[i];
        len[i] = (long long)w[ids[i]].m * q;
    }
    // both norms (before and after subtracting U V^T G) land in one device
    // array and come back with one synchronization
    DeviceBuffer<double> nrm;
    nrm.allocate(2 * ids.size(), ctx.stream);
    sq_norms_device(ctx, ptr, len, nrm.get());
    std::vector<GemmOp> g1, g2;
    for (size_t i = 0; i < ids.size(); ++i) {
        const WTask& t = w[ids[i]];
        // VG = V^T G (r x q); Y -= U VG
        g1.push_back({t.V, P0 + g_off[i], P0 + v_off[i], 1.0, 0.0, t.r, q, t.n, t.ldV, t.n, t.r, 1, 0});
        g2.push_back({t.U, P0 + v_off[i], P0 + y_off[i], -1.0, 1.0, t.m, q, t.r, t.ldU, t.r, t.m, 0, 0});
    }
    launch_gemm_ops(ctx, g1, "probe_vg");
    launch_gemm_ops(ctx, g2, "probe_residual");
    sq_norms_device(ctx, ptr, len, nrm.get() + ids.size());
    std::vector<double> both(2 * ids.size());
    HMB_CUDA(cudaMemcpyAsync(both.data(), nrm.get(), both.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, ctx.stream));
    HMB_CUDA(cudaStreamSynchronize(ctx.stream));
    const double* ref = both.data();
    const double* res = both.data() + ids.size();
    std::vector<double> rel(ids.size());
    for (size_t i = 0; i < ids.size(); ++i)
        rel[i] = ref[i] > 0.0 ? std::sqrt(res[i] / ref[i]) : (res[i] > 0.0 ? 1.0 : 0.0);
    return rel;
}

// The symbolic phase depends only on the structure, the ranks of the
// factors (and of C for the update form), alpha, beta, the rank cap and the
// oversampling; generator positions are kept as draw counts from the
// starting state.  Plans are cached per context (the last kHHPlans), so the
// iterations of SchulzInvert, whose ranks repeat, plan once.
// Per-block operation lists of a plan in position-independent form (pointer
// fields are tagged offsets into the product's buffers, see reloc.h): built
// by the first product that uses the plan, replayed by the next ones.
// Indices of the base table: doubles 0 W arena, 1 A, 2 B, 3 C, 4 state
// slots, 5 C's previous storage, 6 rounding work; ints 0 per-op ranks,
// 1 kept ranks of the sampled products.
struct BlockCache {
    RoundList rounds;
    GemmList gemms;
    GemmTileList leaf1, leaf2;   // leaf products (bases: 0 W arena, 1 A, 2 B)
    bool leaves_cached = false;
    long long pa_used = 0, wk_used = 0;
    double tol = 0.0;
    bool a_is_b = false;
};

struct SymPlan {
    std::vector<WTask> w;
    PerBlock<LOp> lops;
    PerBlock<DOp> dops;
    uint64_t serial_steps = 0;
    std::vector<int> crank, state_rank, op_kind;
    std::vector<int> k0, kq0;   // plain sample counts per task
    std::shared_ptr<BlockCache> blocks;
    // Fixed by the plan's ranks, set by its first product: the W arena and
    // sampling scratch layout (offsets in the tasks) and the tasks a cached
    // product touches on the host -- the sampled products (node x node of
    // nonzero rank) and the node x low-rank / low-rank x node products, whose
    // factor is an H x dense product.  A product in 3-D has millions of
    // tasks, nearly all of rank 0 or served by the cached leaf and block
    // lists, so the per-product host work follows these lists only.
    bool laid_out = false;
    long long wa_used = 0, sa_used = 0;
    std::vector<int> hh_ids, hlr_ids, lrh_ids;
    std::vector<int> hh_pos;   // per task: its index in hh_ids, or -1
};

struct SymKey {
    const Structure* S = nullptr;
    int fresh = 1, maxRankC = 0, oversample = 0, maxA = 0, maxB = 0;
    double alpha = 0, beta = 0;
    std::vector<int> ra, rb, rc;
    std::vector<int> roots;   // flattened (a, b, c) sub-tree roots; empty: the whole matrix
    uint64_t hash = 0;
    bool operator==(const SymKey& o) const {
        return hash == o.hash && S == o.S && fresh == o.fresh && maxRankC == o.maxRankC &&
               oversample == o.oversample && maxA == o.maxA && maxB == o.maxB &&
               alpha == o.alpha && beta == o.beta && ra == o.ra && rb == o.rb && rc == o.rc &&
               roots == o.roots;
    }
};

uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ULL;
    return h;
}

constexpr size_t kHHPlans = 8;

}  // namespace

struct HHPlanCache {
    std::vector<std::pair<SymKey, std::shared_ptr<SymPlan>>> entries;   // most recent last
};

namespace {

// roots empty: the product of the whole matrices (C rebuilt when fresh).
// Otherwise one product per listed sub-tree triple, in order (fresh: C_c :=
// alpha A_a B_b; else C_c := alpha A_a B_b + beta C_c), into an existing C
// whose other leaves keep their content.
std::shared_ptr<SymPlan> make_plan(const HMatrix& A, const HMatrix& B, const HMatrix& C,
                                   double alpha, double beta, bool fresh, int maxRankC,
                                   int oversample, const std::vector<HHRoot>& roots) {
    const Structure& S = *A.S;
    Planner P(A, B, maxRankC, oversample, 0);
    const bool exec_fresh = fresh && roots.empty();
    if (roots.empty()) {
        if (fresh)
            P.fresh(0, 0, 0, alpha);
        else
            P.update(0, 0, 0, alpha, beta);
    }
    for (const HHRoot& r : roots) {
        if (fresh)
            P.fresh(r.a, r.b, r.c, alpha);
        else
            P.update(r.a, r.b, r.c, alpha, beta);
    }
    P.lops.finalize(S.blocks.size());
    P.dops.finalize(S.blocks.size());
    auto plan = std::make_shared<SymPlan>();
    plan->serial_steps = P.steps;
    // final ranks of C, and the rank after each operation with its rounding
    // kind (-1: rank reset), parallel to lops.ops
    std::vector<int>& crank = plan->crank;
    std::vector<int>& state_rank = plan->state_rank;
    std::vector<int>& op_kind = plan->op_kind;
    crank.assign(S.blocks.size(), 0);
    state_rank.assign(P.lops.ops.size(), 0);
    op_kind.assign(P.lops.ops.size(), 0);
    for (int c : S.leaves) {
        const Block& Cb = S.blocks[c];
        if (Cb.kind != KIND_LOWRANK) continue;
        int rank = exec_fresh ? 0 : C.rank[c];
        const int minDim = std::min(Cb.m, Cb.n);
        const int nops = P.lops.size(c);
        const LOp* ops = P.lops.of(c);
        for (int j = 0; j < nops; ++j) {
            const LOp& op = ops[j];
            int kindr = -1;
            switch (op.type) {
                case L_SET:
                    rank = P.w[op.w].r;
                    kindr = ROUND_SET;
                    break;
                case L_RESET:
                    rank = 0;
                    kindr = -1;
                    break;
                case L_RUPD: {
                    int r = P.w[op.w].r + rank;
                    int rr = std::min(std::min(r, minDim), maxRankC);
                    kindr = (rr == r) ? ROUND_CONCAT : ROUND_GENERAL;
                    rank = rr;
                    break;
                }
                case L_DDC:
                    rank = std::min(minDim, maxRankC);
                    kindr = ROUND_DENSE;
                    break;
            }
            state_rank[P.lops.begin[c] + j] = rank;
            op_kind[P.lops.begin[c] + j] = kindr;
        }
        crank[c] = rank;
    }
    plan->w = std::move(P.w);
    plan->k0.resize(plan->w.size());
    plan->kq0.resize(plan->w.size());
    for (size_t i = 0; i < plan->w.size(); ++i) {
        plan->k0[i] = plan->w[i].k;
        plan->kq0[i] = plan->w[i].kq;
    }
    plan->lops = std::move(P.lops);
    plan->dops = std::move(P.dops);
    return plan;
}

std::shared_ptr<SymPlan> get_plan(Context& ctx, const HMatrix& A, const HMatrix& B,
                                  const HMatrix& C, double alpha, double beta, bool fresh,
                                  int maxRankC, const std::vector<HHRoot>& roots) {
    SymKey key;
    key.S = A.S.get();
    key.fresh = fresh ? 1 : 0;
    key.maxRankC = maxRankC;
    key.oversample = ctx.oversample;
    key.maxA = A.max_rank;
    key.maxB = B.max_rank;
    key.alpha = alpha;
    key.beta = beta;
    key.ra = A.rank;
    key.rb = B.rank;
    if (!fresh || !roots.empty()) key.rc = C.rank;
    for (const HHRoot& r : roots) {
        key.roots.push_back(r.a);
        key.roots.push_back(r.b);
        key.roots.push_back(r.c);
    }
    uint64_t h = 1469598103934665603ULL;
    h = fnv(h, &key.S, sizeof(key.S));
    h = fnv(h, &key.fresh, sizeof(int) * 5);
    h = fnv(h, &key.alpha, sizeof(double) * 2);
    h = fnv(h, key.ra.data(), key.ra.size() * sizeof(int));
    h = fnv(h, key.rb.data(), key.rb.size() * sizeof(int));
    h = fnv(h, key.rc.data(), key.rc.size() * sizeof(int));
    h = fnv(h, key.roots.data(), key.roots.size() * sizeof(int));
    key.hash = h;
    if (!ctx.hh_cache) ctx.hh_cache = std::make_shared<HHPlanCache>();
    auto& E = ctx.hh_cache->entries;
    for (size_t i = 0; i < E.size(); ++i) {
        if (E[i].first == key) {
            auto hit = E[i];
            E.erase(E.begin() + (long long)i);
            E.push_back(hit);
            return hit.second;
        }
    }
    // complex matrices (real form, 2 rows per point): oversample complex
    // directions = 2 x oversample real ones
    auto plan = make_plan(A, B, C, alpha, beta, fresh, maxRankC, ctx.oversample * A.S->dof, roots);
    E.emplace_back(std::move(key), plan);
    if (E.size() > kHHPlans) E.erase(E.begin());
    return plan;
}

// The W arena and sampling scratch layout of a plan (offsets kept in its
// tasks; the ranks, and with them every size, are part of the plan's key)
// and its short task lists.  Low-rank factors that a product passes through
// unchanged alias A's U or B's V instead of taking a slot.
void lay_out_tasks(const Structure& S, const HMatrix& A, const HMatrix& B, SymPlan& plan) {
    Arena wa, sa;
    plan.hh_pos.assign(plan.w.size(), -1);
    for (size_t i = 0; i < plan.w.size(); ++i) {
        WTask& t = plan.w[i];
        const Block& Ba = S.blocks[t.a];
        const Block& Bb = S.blocks[t.b];
        switch (t.type) {
            case W_LRLR:
                if (A.rank[t.a] <= B.rank[t.b]) {
                    t.u_alias = true; t.ldU = Ba.m;
                    t.v_off = wa.take((long long)t.n * t.r); t.ldV = t.n;
                } else {
                    t.u_off = wa.take((long long)t.m * t.r); t.ldU = t.m;
                    t.v_alias = true; t.ldV = Bb.n;
                }
                t.g_off = wa.take((long long)B.rank[t.b] * A.rank[t.a]);
                break;
            case W_LRH:
            case W_LRD:
                t.u_alias = true; t.ldU = Ba.m;
                t.v_off = wa.take((long long)t.n * t.r); t.ldV = t.n;
                if (t.type == W_LRH && t.r > 0) plan.lrh_ids.push_back((int)i);
                break;
            case W_HLR:
            case W_DLR:
                t.u_off = wa.take((long long)t.m * t.r); t.ldU = t.m;
                t.v_alias = true; t.ldV = Bb.n;
                if (t.type == W_HLR && t.r > 0) plan.hlr_ids.push_back((int)i);
                break;
            case W_HH: {
                // sampling scratch at the plain sample counts (the learned
                // counts are never larger)
                const int k = plan.k0[i], kq = plan.kq0[i];
                t.u_off = wa.take((long long)t.m * t.r); t.ldU = t.m;
                t.v_off = wa.take((long long)t.n * t.r); t.ldV = t.n;
                t.s_omega = sa.take((long long)Bb.n * k);
                t.s_x = sa.take((long long)Bb.m * k);
                t.s_y = sa.take((long long)Ba.m * k);
                t.s_q = sa.take((long long)Ba.m * kq);
                t.s_tau = sa.take(k);
                t.s_z1 = sa.take((long long)Ba.n * kq);
                t.s_z = sa.take((long long)Bb.n * kq);
                RoundOp probe{};
                probe.kind = ROUND_ORTHO; probe.m = t.m; probe.n = t.n; probe.r1 = kq;
                t.s_work = sa.take(round_work_size(probe));
                if (t.r > 0) {
                    plan.hh_pos[i] = (int)plan.hh_ids.size();
                    plan.hh_ids.push_back((int)i);
                }
                break;
            }
            case W_DD:
                t.d_off = wa.take((long long)t.m * t.n);
                break;
        }
    }
    plan.wa_used = wa.used;
    plan.sa_used = sa.used;
    plan.laid_out = true;
}

// A task's factor addresses in this product's buffers.
void bind_task(WTask& t, double* W0, const HMatrix& A, const HMatrix& B) {
    t.U = t.u_alias ? A.U(t.a) : (t.u_off >= 0 ? W0 + t.u_off : nullptr);
    t.V = t.v_alias ? B.V(t.b) : (t.v_off >= 0 ? W0 + t.v_off : nullptr);
    t.D = t.d_off >= 0 ? W0 + t.d_off : nullptr;
}

}  // namespace

void hh_multiply(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha, double beta,
                 HMatrix& C, bool fresh, bool compact) {
    hh_multiply_roots(ctx, A, B, alpha, beta, C, fresh, {}, compact);
}

void hh_multiply_sub(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha, double beta,
                     HMatrix& C, bool fresh, const std::vector<HHRoot>& roots) {
    HMB_REQUIRE(!roots.empty(), HM_ERR_ARGUMENT, "no sub-tree product listed");
    HMB_REQUIRE(C.S != nullptr, HM_ERR_ARGUMENT, "sub-tree products need an existing C");
    const Structure& S = *C.S;
    for (const HHRoot& r : roots) {
        HMB_REQUIRE(r.a >= 0 && r.b >= 0 && r.c >= 0 && r.a < (int)S.blocks.size() &&
                        r.b < (int)S.blocks.size() && r.c < (int)S.blocks.size(),
                    HM_ERR_ARGUMENT, "sub-tree root out of range");
        const Block& Ba = S.blocks[r.a];
        const Block& Bb = S.blocks[r.b];
        const Block& Bc = S.blocks[r.c];
        HMB_REQUIRE(Ba.m == Bc.m && Bb.n == Bc.n && Ba.n == Bb.m && Ba.row_off == Bc.row_off &&
                        Bb.col_off == Bc.col_off && Ba.col_off == Bb.row_off,
                    HM_ERR_ARGUMENT, "sub-tree product roots are not conformal");
    }
    hh_multiply_roots(ctx, A, B, alpha, beta, C, fresh, roots, false);
}

void hh_multiply_roots(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha,
                       double beta, HMatrix& C, bool fresh_plan,
                       const std::vector<HHRoot>& roots, bool compact) {
    HMB_REQUIRE(A.S && B.S && (A.S == B.S || same_structure(*A.S, *B.S)), HM_ERR_ARGUMENT,
                "H*H multiply needs both factors on the same block structure");
    HMB_REQUIRE(&C != &A && &C != &B, HM_ERR_ARGUMENT,
                "the product must not overwrite a factor");
    const Structure& S = *A.S;
    cudaStream_t st = ctx.stream;
    // sub-tree products update C in place (every other leaf is kept), so
    // they execute like the update form whatever their planner form
    const bool fresh = fresh_plan && roots.empty();
    if (!fresh) {
        HMB_REQUIRE(C.S && (C.S == A.S || same_structure(*C.S, *A.S)), HM_ERR_ARGUMENT,
                    "C must share the factors' block structure");
    }
    const int maxRankC = fresh ? A.max_rank : C.max_rank;

    // ---------------- symbolic phase ----------------
    std::unique_ptr<HostScope> hs(new HostScope(ctx, "hh_symbolic"));
    const std::shared_ptr<SymPlan> plan =
        get_plan(ctx, A, B, C, alpha, beta, fresh_plan, maxRankC, roots);
    hs.reset(new HostScope(ctx, "hh_plan_copy"));
    // The plan's task list is used in place: its arena offsets are fixed
    // with the plan; the per-product fields of the tasks this product reads
    // (generator positions, factor addresses, sample counts) are rewritten
    // below before they are read; sample counts start from the plan's.
    struct PlanView {
        std::vector<WTask>& w;
        const PerBlock<LOp>& lops;
        const PerBlock<DOp>& dops;
    } P{plan->w, plan->lops, plan->dops};
    if (!plan->laid_out) lay_out_tasks(S, A, B, *plan);
    const std::vector<int>& hh = plan->hh_ids;
    const std::vector<int>& hh_pos = plan->hh_pos;
    for (int i : hh) {
        WTask& t = P.w[i];
        // generator positions of the samples, from this call's starting state
        t.omega = lcg_skip_host(ctx.serial_state, t.omega_steps);
        t.k = plan->k0[i];
        t.kq = plan->kq0[i];
    }
    const uint64_t serial_after = lcg_skip_host(ctx.serial_state, plan->serial_steps);
    const std::vector<int>& crank = plan->crank;
    const std::vector<int>& state_rank = plan->state_rank;
    const std::vector<int>& op_kind = plan->op_kind;

    hs.reset(new HostScope(ctx, "hh_alloc"));
    // ---------------- allocation ----------------
    // keep the old C storage if C is updated in place
    DeviceBuffer<double> c_old_data;
    std::vector<long long> c_old_off;
    std::vector<int> c_old_rank;
    if (!fresh) {
        c_old_data = std::move(C.data);
        c_old_off = C.off;
        c_old_rank = C.rank;
    }
    if (fresh) {
        C.S = A.S;
        C.max_rank = A.max_rank;
        C.ctx = &ctx;
    }
    C.rank = crank;
    C.layout();

    // W arena and sampling scratch (laid out with the plan)
    double* W0 = ctx.scratch(0, plan->wa_used);
    double* S0 = ctx.scratch(1, plan->sa_used);
    // leaf and block lists cached with the plan replay position-independently;
    // building them reads every task's factors, a replay only the listed ones
    const bool a_is_b = A.data.get() == B.data.get();
    std::shared_ptr<BlockCache> bc = plan->blocks;
    if (bc && (bc->tol != ctx.compression_tol || bc->a_is_b != a_is_b)) bc.reset();
    if (bc && bc->leaves_cached) {
        for (int i : hh) bind_task(P.w[i], W0, A, B);
        for (int i : plan->hlr_ids) bind_task(P.w[i], W0, A, B);
        for (int i : plan->lrh_ids) bind_task(P.w[i], W0, A, B);
    } else {
        for (WTask& t : P.w) bind_task(t, W0, A, B);
    }

    // ---------------- randomized sampling ----------------
    hs.reset(new HostScope(ctx, "hh_sampling"));
    const bool log_ranks = ctx.rank_log && ctx.compression_tol > 0.0 && !hh.empty();
    const bool learned = ctx.rank_model != nullptr && !hh.empty();
    std::vector<float> feats;
    if (log_ranks || learned) feats = rank_features(S, A, B, P.w, hh, maxRankC);
    std::vector<int> k_plain(hh.size()), kq_plain(hh.size());
    for (size_t i = 0; i < hh.size(); ++i) {
        k_plain[i] = P.w[hh[i]].k;
        kq_plain[i] = P.w[hh[i]].kq;
    }
    if (learned) {
        // sample counts from the predicted kept-rank fractions
        std::vector<float> pred(hh.size());
        ctx.rank_model->predict(feats.data(), (int)hh.size(), pred.data());
        for (size_t i = 0; i < hh.size(); ++i) {
            WTask& t = P.w[hh[i]];
            int rp = (int)std::ceil(pred[i] * t.r) + ctx.rank_margin;
            rp = std::max(1, std::min(rp, t.r));
            t.k = std::min(k_plain[i], rp + ctx.oversample * S.dof);
            t.kq = std::min(S.blocks[t.a].m, t.k);
        }
    }
    // kept ranks of the sampled products (truncating runs: later operations
    // read them on the device, the log reads them back)
    DeviceBuffer<int> kept;
    if (ctx.compression_tol > 0.0 && !hh.empty()) kept.allocate(hh.size(), st);
    // the sampling pipeline for the listed tasks, at their current k
    auto sample = [&](const std::vector<int>& ids) {
        {
            // Gaussian test matrices: SerialGaussianRandomVectors(Omega), n_b x k
            std::vector<FillOp> fills;
            for (int i : ids) {
                const WTask& t = P.w[i];
                fills.push_back({S0 + t.s_omega, t.omega, S.blocks[t.b].n, t.k});
            }
            launch_gaussian_fills(ctx, fills, "omega_fill");
        }
        // X = alpha B Omega
        {
            std::vector<MatJob> jobs;
            for (int i : ids) {
                const WTask& t = P.w[i];
                const Block& Bb = S.blocks[t.b];
                jobs.push_back({&B, t.b, false, t.alpha, 0.0, S0 + t.s_omega, Bb.n, S0 + t.s_x,
                                Bb.m, t.k});
            }
            run_jobs(ctx, jobs, ctx.low_precision);
        }
        // Y = A X
        {
            std::vector<MatJob> jobs;
            for (int i : ids) {
                const WTask& t = P.w[i];
                const Block& Ba = S.blocks[t.a];
                jobs.push_back({&A, t.a, false, 1.0, 0.0, S0 + t.s_x, Ba.n, S0 + t.s_y, Ba.m, t.k});
            }
            run_jobs(ctx, jobs, ctx.low_precision);
        }
        // Q = orth(Y)
        {
            std::vector<QrOp> q;
            for (int i : ids) {
                const WTask& t = P.w[i];
                q.push_back({S0 + t.s_y, S0 + t.s_q, S0 + t.s_tau, t.m, t.k, t.m, 0});
            }
            launch_qr_formq(ctx, q, "sample_qr");
        }
        // Z1 = alpha A^T Q
        {
            std::vector<MatJob> jobs;
            for (int i : ids) {
                const WTask& t = P.w[i];
                const Block& Ba = S.blocks[t.a];
                jobs.push_back({&A, t.a, true, t.alpha, 0.0, S0 + t.s_q, Ba.m, S0 + t.s_z1, Ba.n,
                                t.kq});
            }
            run_jobs(ctx, jobs);
        }
        // Z = B^T Z1
        {
            std::vector<MatJob> jobs;
            for (int i : ids) {
                const WTask& t = P.w[i];
                const Block& Bb = S.blocks[t.b];
                jobs.push_back({&B, t.b, true, 1.0, 0.0, S0 + t.s_z1, Bb.m, S0 + t.s_z, Bb.n, t.kq});
            }
            run_jobs(ctx, jobs);
        }
        // W = best rank-r of Q Z^T (the gesvd truncation of hmat_tools.hpp:1712-1745)
        {
            std::vector<RoundOp> ops;
            for (size_t j = 0; j < ids.size(); ++j) {
                const WTask& t = P.w[ids[j]];
                RoundOp op{};
                op.kind = ROUND_ORTHO;
                op.m = t.m;
                op.n = t.n;
                op.u1 = S0 + t.s_q; op.ldu1 = t.m; op.r1 = t.kq;
                op.v1 = S0 + t.s_z; op.ldv1 = t.n;
                op.rout = t.r;
                op.uo = const_cast<double*>(t.U);
                op.vo = const_cast<double*>(t.V);
                op.work = S0 + t.s_work;
                op.alpha = 1.0;
                op.tol = ctx.compression_tol;
                if (kept.get()) op.rank_out = kept.get() + hh_pos[ids[j]];
                ops.push_back(op);
            }
            launch_round_ops(ctx, ops, "sample_round");
        }
    };
    hs.reset(new HostScope(ctx, "hh_lr_jobs"));
    // W.U = alpha A B.U for node x low-rank, W.V = alpha B^T A.V for
    // low-rank x node
    {
        std::vector<MatJob> jobs;
        for (int i : plan->hlr_ids) {
            const WTask& t = P.w[i];
            jobs.push_back({&A, t.a, false, t.alpha, 0.0, B.U(t.b), S.blocks[t.b].m,
                            const_cast<double*>(t.U), t.m, t.r});
        }
        run_jobs(ctx, jobs);
        jobs.clear();
        for (int i : plan->lrh_ids) {
            const WTask& t = P.w[i];
            jobs.push_back({&B, t.b, true, t.alpha, 0.0, A.V(t.a), S.blocks[t.a].n,
                            const_cast<double*>(t.V), t.n, t.r});
        }
        run_jobs(ctx, jobs);
    }
    hs.reset(new HostScope(ctx, "hh_sample_pipeline"));
    if (!hh.empty()) sample(hh);
    if (learned) {
        // probe check: redo with the plain sample count every compression
        // whose estimated error exceeds the tolerance's scale; in the
        // low-precision phase the FP32 roundings resolve no tolerance finer
        // than 1e-6, which is then the scale (a plain redo could not do
        // better there)
        const std::vector<double> err = probe_errors(ctx, S, A, B, P.w, hh);
        const double scale = ctx.low_precision ? std::max(ctx.compression_tol, kLowPrecisionTolFloor)
                                               : ctx.compression_tol;
        const double limit = std::max(10.0 * scale, 1e-13);
        std::vector<int> redo;
        for (size_t i = 0; i < hh.size(); ++i)
            if (!(err[i] <= limit) && P.w[hh[i]].k < k_plain[i]) redo.push_back((int)i);
        ctx.rank_stats.compressions += (long long)hh.size();
        ctx.rank_stats.fallbacks += (long long)redo.size();
        for (size_t i = 0; i < hh.size(); ++i) {
            ctx.rank_stats.samples += P.w[hh[i]].k;
            ctx.rank_stats.samples_plain += k_plain[i];
        }
        if (!redo.empty()) {
            std::vector<int> ids;
            for (int i : redo) {
                WTask& t = P.w[hh[i]];
                t.k = k_plain[i];
                t.kq = kq_plain[i];
                ctx.rank_stats.samples += t.k;
                ids.push_back(hh[i]);
            }
            sample(ids);
        }
    } else if (!hh.empty()) {
        ctx.rank_stats.compressions += (long long)hh.size();
        for (size_t i = 0; i < hh.size(); ++i) {
            ctx.rank_stats.samples += k_plain[i];
            ctx.rank_stats.samples_plain += k_plain[i];
        }
    }
    if (log_ranks) {
        std::vector<int> kh(hh.size());
        HMB_CUDA(cudaMemcpyAsync(kh.data(), kept.get(), kh.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
        HMB_CUDA(cudaStreamSynchronize(st));
        for (size_t i = 0; i < hh.size(); ++i) {
            ctx.log_x.insert(ctx.log_x.end(), feats.begin() + (long long)i * kMlpFeatures,
                             feats.begin() + (long long)(i + 1) * kMlpFeatures);
            ctx.log_t.push_back((float)kh[i] / (float)std::max(1, P.w[hh[i]].r));
        }
    }
    // HH products with rank 0 (empty blocks): nothing to compute.

    hs.reset(new HostScope(ctx, "hh_leaf_lists"));
    // ---------------- leaf products ----------------
    // Cached with the plan's block lists (position-independent, reloc.h):
    // they depend on the plan and on whether A and B are one matrix.
    RelocBases leaf_bases{};
    leaf_bases.d[0] = W0;
    leaf_bases.d[1] = const_cast<double*>(A.data.get());
    leaf_bases.d[2] = const_cast<double*>(B.data.get());
    std::unique_ptr<GemmTileList> pending_leaf1, pending_leaf2;
    if (bc && bc->leaves_cached) {
        launch_gemm_tiles(ctx, bc->leaf1, leaf_bases, "leaf_products");
        launch_gemm_tiles(ctx, bc->leaf2, leaf_bases, "leaf_products");
    } else {
        std::vector<GemmOp> g1, g2;
        for (const WTask& t : P.w) {
            const Block& Ba = S.blocks[t.a];
            const Block& Bb = S.blocks[t.b];
            const int ra = A.rank[t.a], rb = B.rank[t.b];
            switch (t.type) {
                case W_LRLR:
                    if (t.r == 0) break;
                    if (ra <= rb) {
                        // G = B.U^T A.V (rb x ra); V = alpha B.V G
                        g1.push_back({B.U(t.b), A.V(t.a), W0 + t.g_off, 1.0, 0.0, rb, ra, Bb.m,
                                      Bb.m, Ba.n, rb, 1, 0});
                        g2.push_back({B.V(t.b), W0 + t.g_off, const_cast<double*>(t.V), t.alpha,
                                      0.0, Bb.n, ra, rb, Bb.n, rb, t.n, 0, 0});
                    } else {
                        // G = A.V^T B.U (ra x rb); U = alpha A.U G
                        g1.push_back({A.V(t.a), B.U(t.b), W0 + t.g_off, 1.0, 0.0, ra, rb, Ba.n,
                                      Ba.n, Bb.m, ra, 1, 0});
                        g2.push_back({A.U(t.a), W0 + t.g_off, const_cast<double*>(t.U), t.alpha,
                                      0.0, Ba.m, rb, ra, Ba.m, ra, t.m, 0, 0});
                    }
                    break;
                case W_LRD:   // V = alpha B.D^T A.V
                    if (t.r == 0) break;
                    g1.push_back({B.D(t.b), A.V(t.a), const_cast<double*>(t.V), t.alpha, 0.0,
                                  Bb.n, t.r, Bb.m, Bb.m, Ba.n, t.n, 1, 0});
                    break;
                case W_DLR:   // U = alpha A.D B.U
                    if (t.r == 0) break;
                    g1.push_back({A.D(t.a), B.U(t.b), const_cast<double*>(t.U), t.alpha, 0.0,
                                  Ba.m, t.r, Ba.n, Ba.m, Bb.m, t.m, 0, 0});
                    break;
                case W_DD:    // D = alpha A.D B.D
                    g1.push_back({A.D(t.a), B.D(t.b), const_cast<double*>(t.D), t.alpha, 0.0,
                                  Ba.m, Bb.n, Ba.n, Ba.m, Bb.m, t.m, 0, 0});
                    break;
                default:
                    break;
            }
        }
        // position-independent copies; kept once the block lists are cached
        Relocator rel;
        rel.add(0, W0, plan->wa_used);
        rel.add(1, A.data.get(), A.total);
        rel.add(2, B.data.get(), B.total);
        std::vector<GemmOp> t1 = g1, t2 = g2;
        bool ok = true;
        for (GemmOp& g : t1) ok = ok && rel.tag(g.A) && rel.tag(g.B) && rel.tag(g.C);
        for (GemmOp& g : t2) ok = ok && rel.tag(g.A) && rel.tag(g.B) && rel.tag(g.C);
        if (ok) {
            pending_leaf1.reset(new GemmTileList);
            pending_leaf2.reset(new GemmTileList);
            upload_gemm_tiles(ctx, t1, *pending_leaf1);
            upload_gemm_tiles(ctx, t2, *pending_leaf2);
            launch_gemm_tiles(ctx, *pending_leaf1, leaf_bases, "leaf_products");
            launch_gemm_tiles(ctx, *pending_leaf2, leaf_bases, "leaf_products");
        } else {   // a pointer outside the registered buffers: run once, uncached
            launch_gemm_ops(ctx, g1, "leaf_products");
            launch_gemm_ops(ctx, g2, "leaf_products");
        }
    }

    hs.reset(new HostScope(ctx, "hh_block_lists"));
    // ---------------- per-block operation lists ----------------
    // One worker (CTA) per C leaf block runs that block's operations in the
    // reference's order; blocks proceed independently.  Low-rank states of a
    // block with several operations alternate between two scratch slots; the
    // last operation writes into C.  The lists depend only on the plan (and
    // the truncation tolerance): built once, cached with it, then replayed.
    const bool dyn = ctx.compression_tol > 0.0;
    double* parena = nullptr;   // state slots (scratch 2)
    double* wbuf = nullptr;     // rounding work (scratch 3)
    DeviceBuffer<int> rk;
    if (dyn) rk.allocate(std::max<size_t>(1, P.lops.ops.size()), st);
    auto bases_now = [&]() {
        RelocBases b{};
        b.d[0] = W0;
        b.d[1] = const_cast<double*>(A.data.get());
        b.d[2] = const_cast<double*>(B.data.get());
        b.d[3] = C.data.get();
        b.d[4] = parena;
        b.d[5] = c_old_data.get();
        b.d[6] = wbuf;
        b.i[0] = rk.get();
        b.i[1] = kept.get();
        return b;
    };
    if (bc) {
        HostScope replay(ctx, "hh_block_lists_replayed");
        parena = ctx.scratch(2, bc->pa_used);
        if (bc->rounds.nw > 0) wbuf = ctx.scratch(3, bc->wk_used);
    } else {
        Arena pa, wk;
        std::vector<long long> slot0(S.blocks.size(), -1), slot1(S.blocks.size(), -1);
        std::vector<long long> wslot(S.blocks.size(), -1);
        for (int c : S.leaves) {
            const Block& Cb = S.blocks[c];
            const int nops = P.lops.size(c);
            if (Cb.kind != KIND_LOWRANK || nops == 0) continue;
            int mr = 0;
            for (int j = 0; j + 1 < nops; ++j) mr = std::max(mr, state_rank[P.lops.begin[c] + j]);
            if (nops > 1) {
                slot0[c] = pa.take((long long)(Cb.m + Cb.n) * mr);
                slot1[c] = pa.take((long long)(Cb.m + Cb.n) * mr);
            }
        }
        parena = ctx.scratch(2, pa.used);
        double* P0 = parena;
        std::vector<RoundOp> rops;
        std::vector<int> rbegin{0};
        std::vector<long long> rwork;   // per op: offset into the work arena
        // truncating runs: every op leaves its output rank in rk, the next op of
        // the block (and a sampled W's kept rank) set its input ranks on the device
        std::vector<GemmOp> gops;
        std::vector<int> gbegin{0};
        for (int c : S.leaves) {
            const Block& Cb = S.blocks[c];
            if (Cb.kind == KIND_LOWRANK) {
                const int nops = P.lops.size(c);
                const LOp* ops = P.lops.of(c);
                const int obase = P.lops.begin[c];
                if (nops == 0) {
                    // outside every sub-tree of a sub-tree product: keep the
                    // block (an exact copy, the concatenation with nothing)
                    if (!fresh && c_old_rank[c] > 0 && Cb.m > 0 && Cb.n > 0) {
                        RoundOp r{};
                        r.kind = ROUND_CONCAT;
                        r.m = Cb.m;
                        r.n = Cb.n;
                        r.alpha = 1.0;
                        r.beta = 1.0;
                        r.r2 = c_old_rank[c];
                        r.rout = c_old_rank[c];
                        r.u2 = c_old_data.get() + c_old_off[c];
                        r.v2 = r.u2 + (long long)Cb.m * c_old_rank[c];
                        r.ldu2 = Cb.m;
                        r.ldv2 = Cb.n;
                        r.uo = C.U(c);
                        r.vo = C.V(c);
                        rops.push_back(r);
                        rwork.push_back(0);
                        rbegin.push_back((int)rops.size());
                    }
                    continue;
                }
                const double* cu = nullptr;
                const double* cv = nullptr;
                int cr = 0;
                if (!fresh) {
                    cu = c_old_data.get() + c_old_off[c];
                    cv = cu + (long long)Cb.m * c_old_rank[c];
                    cr = c_old_rank[c];
                }
                long long wmax = 0;
                const size_t first = rops.size();
                int prev = -1;   // op whose output is (cu, cv)
                // An update by a product of rank 0 with beta = 1 that keeps
                // the state's rank leaves the state as it is (its rounding
                // would be an exact copy): it is not emitted, and the last op
                // that may change the state writes into C (op 0 when none
                // may: a copy of C's storage).
                auto keeps_state = [&](int j) {
                    return ops[j].type == L_RUPD && P.w[ops[j].w].r == 0 && ops[j].beta == 1.0 &&
                           op_kind[obase + j] == ROUND_CONCAT;
                };
                int last = nops - 1;
                while (last > 0 && keeps_state(last)) --last;
                int written = 0;   // ops so far that took a state slot
                for (int j = 0; j <= last; ++j) {
                    const LOp& op = ops[j];
                    const int rnew = state_rank[obase + j];
                    if (op.type == L_RESET) {
                        cr = 0;
                        prev = -1;
                        continue;
                    }
                    if (j < last && keeps_state(j)) continue;
                    double* ou = (j == last) ? C.U(c)
                                             : P0 + ((written++ & 1) ? slot1[c] : slot0[c]);
                    double* ov = ou + (long long)Cb.m * rnew;
                    const WTask& t = P.w[op.w];
                    RoundOp r{};
                    r.kind = op_kind[obase + j];
                    r.m = Cb.m;
                    r.n = Cb.n;
                    r.alpha = 1.0;
                    r.beta = op.beta;
                    r.rout = rnew;
                    r.uo = ou;
                    r.vo = ov;
                    if (op.type == L_DDC) {
                        r.u1 = t.D;
                        r.ldu1 = t.m;
                    } else {
                        r.u1 = t.U ? t.U + op.row0 : nullptr;
                        r.v1 = t.V ? t.V + op.col0 : nullptr;
                        r.ldu1 = t.ldU;
                        r.ldv1 = t.ldV;
                        r.r1 = t.r;
                    }
                    r.u2 = cu;
                    r.v2 = cv;
                    r.tol = ctx.compression_tol;
                    r.r2 = (op.type == L_SET || (op.type == L_DDC && op.beta == 0.0)) ? 0 : cr;
                    r.ldu2 = Cb.m;
                    r.ldv2 = Cb.n;
                    if (dyn) {
                        r.rank_out = rk.get() + rops.size();
                        if (r.r2 > 0 && prev >= 0) r.r2_dev = rk.get() + prev;
                        if (op.type != L_DDC && hh_pos[op.w] >= 0) r.r1_dev = kept.get() + hh_pos[op.w];
                    }
                    prev = -1;
                    if (rnew > 0 && Cb.m > 0 && Cb.n > 0) {
                        prev = (int)rops.size();
                        rops.push_back(r);
                        wmax = std::max(wmax, round_work_size(r));
                    }
                    cu = ou;
                    cv = ov;
                    cr = rnew;
                }
                if (rops.size() > first) {
                    const long long w0 = wk.take(wmax);
                    for (size_t i = first; i < rops.size(); ++i) rwork.push_back(w0);
                    rbegin.push_back((int)rops.size());
                }
            } else {
                const size_t first = gops.size();
                if (!fresh)
                    gops.push_back({c_old_data.get() + c_old_off[c], nullptr, C.D(c), 1.0, 0.0, Cb.m,
                                    Cb.n, -1, Cb.m, 0, Cb.m, 0, 0});
                for (int j = 0; j < P.dops.size(c); ++j) {
                    const DOp& op = P.dops.of(c)[j];
                    if (op.type == D_DD) {
                        const Block& Ba = S.blocks[op.a];
                        const Block& Bb = S.blocks[op.b];
                        gops.push_back({A.D(op.a), B.D(op.b), C.D(c), op.alpha, op.beta, Cb.m, Cb.n,
                                        Ba.n, Ba.m, Bb.m, Cb.m, 0, 0});
                    } else {
                        const WTask& t = P.w[op.w];
                        if (t.r == 0) {
                            // a product of rank 0: C = beta C (nothing to do for beta = 1)
                            if (op.beta != 1.0)
                                gops.push_back({C.D(c), nullptr, C.D(c), op.beta, 0.0, Cb.m, Cb.n,
                                                -1, Cb.m, 0, Cb.m, 0, 0});
                        } else
                            gops.push_back({t.U + op.row0, t.V + op.col0, C.D(c), 1.0, op.beta, Cb.m,
                                            Cb.n, t.r, t.ldU, t.ldV, Cb.m, 0, 1});
                    }
                }
                if (gops.size() > first && Cb.m > 0 && Cb.n > 0) gbegin.push_back((int)gops.size());
                else gops.resize(first);
            }
        }
        if (!rops.empty()) {
            wbuf = ctx.scratch(3, wk.used);
            for (size_t i = 0; i < rops.size(); ++i) rops[i].work = wbuf + rwork[i];
        }

        // position-independent copy for the cache
        Relocator rel;
        rel.add(0, W0, plan->wa_used);
        rel.add(1, A.data.get(), A.total);
        rel.add(2, B.data.get(), B.total);
        rel.add(3, C.data.get(), C.total);
        rel.add(4, parena, pa.used);
        rel.add(5, c_old_data.get(), (long long)c_old_data.size());
        rel.add(6, wbuf, wk.used);
        rel.add(0, rk.get(), (long long)rk.size());
        rel.add(1, kept.get(), (long long)kept.size());
        std::vector<RoundOp> trops = rops;
        std::vector<GemmOp> tgops = gops;
        bool ok = true;
        for (RoundOp& r : trops) {
            ok = ok && rel.tag(r.u1) && rel.tag(r.v1) && rel.tag(r.u2) && rel.tag(r.v2) &&
                 rel.tag(r.uo) && rel.tag(r.vo) && rel.tag(r.work) && rel.tag(r.rank_out) &&
                 rel.tag(r.r1_dev) && rel.tag(r.r2_dev);
        }
        for (GemmOp& g : tgops) ok = ok && rel.tag(g.A) && rel.tag(g.B) && rel.tag(g.C);
        bc = std::make_shared<BlockCache>();
        upload_round_list(ctx, ok ? trops : rops, rbegin, bc->rounds);
        upload_gemm_list(ctx, ok ? tgops : gops, gbegin, bc->gemms);
        bc->pa_used = pa.used;
        bc->wk_used = wk.used;
        bc->tol = ctx.compression_tol;
        bc->a_is_b = a_is_b;
        if (pending_leaf1) {
            bc->leaf1 = std::move(*pending_leaf1);
            bc->leaf2 = std::move(*pending_leaf2);
            bc->leaves_cached = true;
        }
        // lists that point outside the registered buffers run once, uncached
        if (ok) plan->blocks = bc;
        else HostScope uncached(ctx, "hh_block_lists_uncached");
    }
    hs.reset(new HostScope(ctx, "hh_block_launch"));
    const RelocBases bases = bases_now();
    launch_round_list(ctx, bc->rounds, bases, "block_round");
    launch_gemm_list(ctx, bc->gemms, bases, "dense_update");
    // low-rank C blocks whose final rank is 0 or that received no operation
    // need nothing: their storage is empty.
    ctx.serial_state = serial_after;
    // tolerance truncation: store C at the ranks kept
    if (ctx.compression_tol > 0.0 && compact) compact_ranks(ctx, C);
}

}  // namespace hmb
