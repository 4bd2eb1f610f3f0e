// Level-batched H-matrix x dense products (the H-matvec / H-matmat hot path).
//
// Replaces the reference's recursive HMat2d::Multiply / TransposeMultiply
// (src/HMat2d/MultiplyVector-incl.hpp:12-124, MultiplyDense-incl.hpp:12-150),
// which issues one gemv/gemm per dense leaf (src/hmat_tools/MultiplyVector.cpp
// :14-69) and two per low-rank block (:71-128), recursing over the tree.
//
// A job is one subtree (root block, op) of one H-matrix applied to one dense
// input.  Each (H-matrix, root, op) has a template -- its work lists, built
// once and kept on the device -- and a batch of jobs runs as two launches:
//   phase 1: T_b = W_b^T X_b for every low-rank block b of every job
//            (W = V, or U for the transpose), one CTA per block;
//   phase 2: for every output row tile of every job, Y_tile = alpha * (sum
//            over the dense leaves and low-rank blocks covering the tile of
//            A_e(tile rows) * B_e) + beta * Y_tile, one CTA per tile, so each
//            output element is written once (no atomics, deterministic).
// Every stored matrix entry is read exactly once per launch pair.  A CTA finds
// its job by binary search over the jobs' first work-item indices.
#include <algorithm>
#include <cstring>

#include "engine.h"
#include "templates.h"

namespace hmb {

// What a CTA needs to run its share of one job.
struct JobExec {
    const P1T* p1;
    const P2T* p2;
    const P2Entry* ent;
    const double* in;
    double* out;
    double* T;
    const double* alpha_scale;
    double alpha, beta;
    long long p1_begin, p2_begin;   // first global work item of this job
    int n1, n2, ldin, ldout, k, ct1, ct2, pad;   // ct*: column tiles per item
};

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ int find_job(const JobExec* jobs, int njobs, long long idx,
                                        bool phase2) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const long long b = phase2 ? jobs[mid].p2_begin : jobs[mid].p1_begin;
        if (b <= idx) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Phase 1: T = W^T in
// ---------------------------------------------------------------------------
// Narrow: k <= NC.  Warps take columns of W; lanes stride over rows.
template <int NC>
__global__ void __launch_bounds__(kThreads)
p1_narrow_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0) {
    const long long gi = blockIdx.x;
    const JobExec& J = jobs ? jobs[find_job(jobs, njobs, gi, false)] : job0;
    const P1T it = J.p1[gi - J.p1_begin];
    const double* in = J.in + it.in_off;
    double* T = J.T + it.t_rel * J.k;
    const int K = J.k, ldin = J.ldin;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = warp; j < it.r; j += kWarps) {
        const double* w = it.W + (long long)j * it.ldw;
        double acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = 0.0;
        int p = lane;
        for (; p + 224 < it.nin; p += 256) {   // eight loads of W in flight per lane
            double wv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) wv[u] = __ldg(w + p + 32 * u);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (c < K) {
                    const double* x = in + (long long)c * ldin + p;
#pragma unroll
                    for (int u = 0; u < 8; ++u) acc[c] = fma(wv[u], __ldg(x + 32 * u), acc[c]);
                }
            }
        }
        for (; p < it.nin; p += 32) {
            double w0 = __ldg(w + p);
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (c < K) acc[c] = fma(w0, __ldg(in + (long long)c * ldin + p), acc[c]);
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double v = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && c < K) T[j + (long long)c * it.r] = v;
        }
    }
}

// Wide: any k.  Output tile 32 (r) x 32 (k) per CTA column-tile; inner dim
// staged through shared memory in chunks of 32.
__global__ void __launch_bounds__(kThreads)
p1_wide_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0) {
    const long long gi = blockIdx.x;
    const JobExec& J = jobs ? jobs[find_job(jobs, njobs, gi, false)] : job0;
    const long long local = gi - J.p1_begin;
    const P1T it = J.p1[local / J.ct1];
    const int c0 = (int)(local % J.ct1) * 32;
    const double* in = J.in + it.in_off;
    double* T = J.T + it.t_rel * J.k;
    const int K = J.k, ldin = J.ldin;
    if (c0 >= K) return;
    __shared__ double sW[32][33];
    __shared__ double sX[32][33];
    const int tid = threadIdx.x;
    const int tj = tid & 31;          // output row within tile
    const int tc = (tid >> 5) * 4;    // 4 consecutive output columns
    for (int j0 = 0; j0 < it.r; j0 += 32) {
        double acc[4] = {0, 0, 0, 0};
        for (int p0 = 0; p0 < it.nin; p0 += 32) {
            for (int e = tid; e < 32 * 32; e += kThreads) {
                int pp = e & 31, jj = e >> 5;
                int p = p0 + pp, j = j0 + jj, c = c0 + jj;
                sW[jj][pp] = (p < it.nin && j < it.r) ? it.W[p + (long long)j * it.ldw] : 0.0;
                sX[jj][pp] = (p < it.nin && c < K) ? in[p + (long long)c * ldin] : 0.0;
            }
            __syncthreads();
#pragma unroll 8
            for (int pp = 0; pp < 32; ++pp) {
                double w = sW[tj][pp];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(w, sX[tc + u][pp], acc[u]);
            }
            __syncthreads();
        }
        int j = j0 + tj;
        if (j < it.r)
            for (int u = 0; u < 4; ++u) {
                int c = c0 + tc + u;
                if (c < K) T[j + (long long)c * it.r] = acc[u];
            }
    }
}

// ---------------------------------------------------------------------------
// Phase 2: Y_tile = alpha sum_e A_e B_e + beta Y_tile
// ---------------------------------------------------------------------------
__device__ __forceinline__ double load_a(const P2Entry& e, int i, int p) {
    return e.transA ? __ldg(e.A + p + (long long)i * e.lda)
                    : __ldg(e.A + i + (long long)p * e.lda);
}

// B operand of an entry: (pointer to element (0,0), leading dimension).
__device__ __forceinline__ void entry_b(const P2Entry& e, const JobExec& J, const double*& B,
                                       int& ldb) {
    if (e.b_from_t) { B = J.T + e.b_off * J.k; ldb = e.ldt; }
    else { B = J.in + e.b_off; ldb = J.ldin; }
}

__device__ __forceinline__ void store_out(const JobExec& J, const P2T& it, int i, int c,
                                          double v) {
    double* y = J.out + it.out_off + (it.r0 + i) + (long long)c * J.ldout;
    const double al = J.alpha_scale ? J.alpha * *J.alpha_scale : J.alpha;
    *y = J.beta == 0.0 ? al * v : al * v + J.beta * *y;
}

// Narrow: columns <= NC, rows <= 64, a streaming (HBM-bound) kernel.  The
// tile's entries are concatenated along the inner dimension (entry e covers
// columns [cbeg, cbeg + inner)), and the columns are split evenly among
// "column workers" (sub-groups of lanes; lanes within a worker own rows).
// Each worker keeps eight columns of loads in flight; partial sums are
// reduced over workers through shuffles and shared memory.
template <int NC>
__global__ void __launch_bounds__(kThreads)
p2_narrow_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0) {
    const long long gi = blockIdx.x;
    const JobExec& J = jobs ? jobs[find_job(jobs, njobs, gi, true)] : job0;
    const long long local = gi - J.p2_begin;
    const P2T it = J.p2[local / J.ct2];
    const int c0 = (int)(local % J.ct2) * NC;
    const int cols = min(NC, J.k - c0);
    __shared__ double red[kWarps][64][NC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // rows-per-pass RL (power of two <= 32), column sub-groups 32/RL per warp
    int RL = 1;
    while (RL < it.rows && RL < 32) RL <<= 1;
    const int sub = lane / RL, rl = lane % RL, nsub = 32 / RL;
    const int rpt = (it.rows + RL - 1) / RL;   // rows per thread (<= 2)
    double acc[2][NC];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[a][c] = 0.0;
    if (it.e1 > it.e0) {
        const P2Entry last = J.ent[it.e1 - 1];
        const int total = last.cbeg + last.inner;
        const int nworkers = kWarps * nsub;
        const int worker = warp * nsub + sub;
        const int chunk = (total + nworkers - 1) / nworkers;
        int p = worker * chunk;
        const int pend = min(total, p + chunk);
        int ei = it.e0;
        while (ei + 1 < it.e1 && J.ent[ei + 1].cbeg <= p) ++ei;
        while (p < pend) {
            const P2Entry e = J.ent[ei];
            const double* EB;
            int ldb;
            entry_b(e, J, EB, ldb);
            const int stop = min(pend, e.cbeg + e.inner);
            int q = p - e.cbeg;                 // column within the entry
            const int qstop = stop - e.cbeg;
            for (; q + 7 < qstop; q += 8) {
                double av[2][8], bv[8][NC];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        bv[u][c] = (c < cols) ? __ldg(EB + (q + u) + (long long)(c0 + c) * ldb) : 0.0;
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const int i = rl + a * RL;
                        av[a][u] = (a < rpt && i < it.rows) ? load_a(e, it.r0 + i, q + u) : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
#pragma unroll
                    for (int a = 0; a < 2; ++a)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[a][c] = fma(av[a][u], bv[u][c], acc[a][c]);
            }
            for (; q < qstop; ++q) {
                double b[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    b[c] = (c < cols) ? __ldg(EB + q + (long long)(c0 + c) * ldb) : 0.0;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const int i = rl + a * RL;
                    if (a < rpt && i < it.rows) {
                        const double av = load_a(e, it.r0 + i, q);
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[a][c] = fma(av, b[c], acc[a][c]);
                    }
                }
            }
            p = stop;
            ++ei;
        }
    }
    // reduce over the column sub-groups within the warp (lanes with equal rl)
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double v = acc[a][c];
            for (int o = 16; o >= RL; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[a][c] = v;
        }
    if (sub == 0) {
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            int i = rl + a * RL;
            if (a < rpt && i < it.rows)
#pragma unroll
                for (int c = 0; c < NC; ++c) red[warp][i][c] = acc[a][c];
        }
    }
    __syncthreads();
    for (int o = threadIdx.x; o < it.rows * cols; o += kThreads) {
        int i = o % it.rows, c = o / it.rows;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) v += red[w][i][c];
        store_out(J, it, i, c0 + c, v);
    }
}

// Wide: tile 64 rows x 64 cols, inner staged in chunks of 16; each thread
// owns a 4x4 register tile.
__global__ void __launch_bounds__(kThreads)
p2_wide_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0) {
    const long long gi = blockIdx.x;
    const JobExec& J = jobs ? jobs[find_job(jobs, njobs, gi, true)] : job0;
    const long long local = gi - J.p2_begin;
    const P2T it = J.p2[local / J.ct2];
    const int c0 = (int)(local % J.ct2) * 64;
    const int cols = min(64, J.k - c0);
    __shared__ double sA[16][64 + 1];
    __shared__ double sB[16][64 + 1];
    const int tid = threadIdx.x;
    const int tr = (tid & 15) * 4;   // rows tr..tr+3
    const int tc = (tid >> 4) * 4;   // cols tc..tc+3
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int ei = it.e0; ei < it.e1; ++ei) {
        const P2Entry e = J.ent[ei];
        const double* EB;
        int ldb;
        entry_b(e, J, EB, ldb);
        for (int p0 = 0; p0 < e.inner; p0 += 16) {
            for (int x = tid; x < 16 * 64; x += kThreads) {
                int i, pp;
                if (e.transA) { pp = x & 15; i = x >> 4; }
                else { i = x & 63; pp = x >> 6; }
                int p = p0 + pp;
                sA[pp][i] = (i < it.rows && p < e.inner) ? load_a(e, it.r0 + i, p) : 0.0;
            }
            for (int x = tid; x < 16 * 64; x += kThreads) {
                int pp = x & 15, c = x >> 4;
                int p = p0 + pp;
                sB[pp][c] = (c < cols && p < e.inner)
                                ? __ldg(EB + p + (long long)(c0 + c) * ldb) : 0.0;
            }
            __syncthreads();
#pragma unroll 4
            for (int pp = 0; pp < 16; ++pp) {
                double av[4], bv[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) av[a] = sA[pp][tr + a];
#pragma unroll
                for (int b = 0; b < 4; ++b) bv[b] = sB[pp][tc + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int i = tr + a;
        if (i >= it.rows) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int c = tc + b;
            if (c >= cols) continue;
            store_out(J, it, i, c0 + c, acc[a][b]);
        }
    }
}

// Work lists of one subtree of one H-matrix.
std::shared_ptr<JobTemplate> build_template(Context& ctx, const HMatrix& H, int root,
                                            bool trans, int row_tile) {
    HostScope hs(ctx, "hmm_template");
    const Structure& S = *H.S;
    const Block& R = S.blocks[root];
    auto T = std::make_shared<JobTemplate>();
    // leaves of the subtree, depth-first
    std::vector<int> leaves;
    {
        std::vector<int> stack{root};
        while (!stack.empty()) {
            int b = stack.back();
            stack.pop_back();
            const Block& B = S.blocks[b];
            if (B.kind == KIND_NODE) {
                for (int c = S.q * S.q - 1; c >= 0; --c) stack.push_back(B.first_child + c);
            } else if (B.m > 0 && B.n > 0) {
                leaves.push_back(b);
            }
        }
    }
    // phase 1 items
    std::vector<P1T> p1;
    std::vector<long long> t_rel(leaves.size(), -1);
    long long t_rows = 0;
    for (size_t li = 0; li < leaves.size(); ++li) {
        const int b = leaves[li];
        const Block& B = S.blocks[b];
        if (B.kind != KIND_LOWRANK || H.rank[b] == 0) continue;
        P1T it{};
        if (!trans) {
            it.W = H.V(b);
            it.nin = B.n;
            it.ldw = B.n;
            it.in_off = B.col_off - R.col_off;
        } else {
            it.W = H.U(b);
            it.nin = B.m;
            it.ldw = B.m;
            it.in_off = B.row_off - R.row_off;
        }
        it.r = H.rank[b];
        it.t_rel = t_rows;
        t_rel[li] = t_rows;
        t_rows += it.r;
        p1.push_back(it);
    }
    // phase 2: bucket the leaves by the output clusters they cover
    const Box& outBox = S.boxes[trans ? R.src_box : R.tgt_box];
    const int outBase = trans ? R.col_off : R.row_off;
    const int c0 = outBox.leaf0, nc = outBox.leaf1 - outBox.leaf0;
    std::vector<int> count(nc + 1, 0);
    for (int b : leaves) {
        const Block& B = S.blocks[b];
        const Box& ob = S.boxes[trans ? B.src_box : B.tgt_box];
        for (int c = ob.leaf0; c < ob.leaf1; ++c) count[c - c0 + 1]++;
    }
    for (int c = 0; c < nc; ++c) count[c + 1] += count[c];
    std::vector<int> bucket(count[nc]);
    {
        std::vector<int> fill(count.begin(), count.end() - 1);
        for (size_t li = 0; li < leaves.size(); ++li) {
            const Block& B = S.blocks[leaves[li]];
            const Box& ob = S.boxes[trans ? B.src_box : B.tgt_box];
            for (int c = ob.leaf0; c < ob.leaf1; ++c) bucket[fill[c - c0]++] = (int)li;
        }
    }
    std::vector<P2T> p2;
    std::vector<P2Entry> ent;
    for (int c = outBox.leaf0; c < outBox.leaf1; ++c) {
        const Box& cl = S.boxes[S.leaf_box[c]];
        if (cl.count == 0) continue;
        const int e0 = (int)ent.size();
        int cbeg = 0;
        for (int bi = count[c - c0]; bi < count[c - c0 + 1]; ++bi) {
            const int li = bucket[bi];
            const int b = leaves[li];
            const Block& B = S.blocks[b];
            P2Entry e{};
            if (B.kind == KIND_DENSE) {
                if (!trans) {
                    e.A = H.D(b) + (cl.offset - B.row_off);
                    e.lda = B.m;
                    e.transA = 0;
                    e.inner = B.n;
                    e.b_off = B.col_off - R.col_off;
                } else {
                    e.A = H.D(b) + (long long)(cl.offset - B.col_off) * B.m;
                    e.lda = B.m;
                    e.transA = 1;
                    e.inner = B.m;
                    e.b_off = B.row_off - R.row_off;
                }
                e.b_from_t = 0;
            } else {
                if (H.rank[b] == 0) continue;
                if (!trans) {
                    e.A = H.U(b) + (cl.offset - B.row_off);
                    e.lda = B.m;
                } else {
                    e.A = H.V(b) + (cl.offset - B.col_off);
                    e.lda = B.n;
                }
                e.transA = 0;
                e.inner = H.rank[b];
                e.b_from_t = 1;
                e.b_off = t_rel[li];
                e.ldt = H.rank[b];
            }
            e.cbeg = cbeg;
            cbeg += e.inner;
            ent.push_back(e);
        }
        const int e1 = (int)ent.size();
        for (int r0 = 0; r0 < cl.count; r0 += row_tile) {
            P2T it{};
            it.out_off = cl.offset - outBase;
            it.r0 = r0;
            it.rows = std::min(row_tile, cl.count - r0);
            it.e0 = e0;
            it.e1 = e1;
            p2.push_back(it);
        }
    }
    T->n1 = (int)p1.size();
    T->n2 = (int)p2.size();
    T->t_rows = t_rows;
    T->p1.upload(p1, ctx.stream);
    T->p2.upload(p2, ctx.stream);
    T->ent.upload(ent, ctx.stream);
    return T;
}

}  // namespace

std::shared_ptr<JobTemplate> get_template(Context& ctx, const HMatrix& H, int root, bool trans,
                                          int row_tile) {
    HMB_REQUIRE(row_tile >= 1 && row_tile <= 64, HM_ERR_INTERNAL, "row tile out of range");
    auto key = std::make_tuple(root, trans ? 1 : 0, row_tile);
    auto it = H.templates.find(key);
    if (it != H.templates.end()) return it->second;
    auto T = build_template(ctx, H, root, trans, row_tile);
    H.templates.emplace(key, T);
    return T;
}

void run_jobs(Context& ctx, const std::vector<MatJob>& jobs) {
    if (jobs.empty()) return;
    cudaStream_t st = ctx.stream;
    std::vector<std::shared_ptr<JobTemplate>> tmpl;
    tmpl.reserve(jobs.size());
    int kmax = 0;
    for (const MatJob& J : jobs) {
        HMB_REQUIRE(J.k >= 0, HM_ERR_ARGUMENT, "negative column count");
        kmax = std::max(kmax, J.k);
    }
    // streaming (few right-hand sides): 32-row tiles for more CTAs in flight
    const int row_tile = kmax <= 8 ? 32 : 64;
    for (const MatJob& J : jobs) tmpl.push_back(get_template(ctx, *J.H, J.root, J.trans, row_tile));
    const bool wide = kmax > 8;
    const int NC2 = kmax <= 1 ? 1 : kmax <= 4 ? 4 : kmax <= 8 ? 8 : 64;
    long long t_total = 0;
    std::vector<long long> t_off(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
        t_off[j] = t_total;
        t_total += tmpl[j]->t_rows * jobs[j].k;
    }
    DeviceBuffer<double> tbuf;
    tbuf.allocate((size_t)std::max<long long>(t_total, 1), st);
    std::vector<JobExec> ex;
    ex.reserve(jobs.size());
    long long n1 = 0, n2 = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const MatJob& J = jobs[j];
        if (J.k == 0) continue;
        const JobTemplate& T = *tmpl[j];
        JobExec e{};
        e.p1 = T.p1.get();
        e.p2 = T.p2.get();
        e.ent = T.ent.get();
        e.in = J.in;
        e.out = J.out;
        e.T = tbuf.get() + t_off[j];
        e.alpha_scale = J.alpha_scale;
        e.alpha = J.alpha;
        e.beta = J.beta;
        e.ldin = J.ldin;
        e.ldout = J.ldout;
        e.k = J.k;
        e.n1 = T.n1;
        e.n2 = T.n2;
        e.ct1 = wide ? ceil_div(J.k, 32) : 1;
        e.ct2 = ceil_div(J.k, NC2);
        e.p1_begin = n1;
        e.p2_begin = n2;
        n1 += (long long)T.n1 * e.ct1;
        n2 += (long long)T.n2 * e.ct2;
        ex.push_back(e);
    }
    if (ex.empty()) return;
    HMB_REQUIRE(n1 < (1LL << 31) && n2 < (1LL << 31), HM_ERR_UNSUPPORTED, "batch too large");
    DeviceBuffer<JobExec> dex;
    const JobExec* jobs_d = nullptr;
    if (ex.size() > 1) {
        dex.upload(ex, st);
        jobs_d = dex.get();
    }
    const JobExec job0 = ex[0];
    const int nj = (int)ex.size();
    if (n1 > 0) {
        LaunchScope ls(ctx, "hmm_lowrank_inner");
        const unsigned g = (unsigned)n1;
        if (kmax <= 1) p1_narrow_kernel<1><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else if (kmax <= 4) p1_narrow_kernel<4><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else if (kmax <= 8) p1_narrow_kernel<8><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else p1_wide_kernel<<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        HMB_CHECK_LAUNCH();
    }
    if (n2 > 0) {
        LaunchScope ls(ctx, "hmm_row_tiles");
        const unsigned g = (unsigned)n2;
        if (kmax <= 1) p2_narrow_kernel<1><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else if (kmax <= 4) p2_narrow_kernel<4><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else if (kmax <= 8) p2_narrow_kernel<8><<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        else p2_wide_kernel<<<g, kThreads, 0, st>>>(jobs_d, nj, job0);
        HMB_CHECK_LAUNCH();
    }
}

}  // namespace hmb
