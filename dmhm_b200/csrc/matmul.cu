// Level-batched H-matrix x dense products (the H-matvec / H-matmat hot path).
//
// Replaces the reference's recursive HMat2d::Multiply / TransposeMultiply
// (src/HMat2d/MultiplyVector-incl.hpp:12-124, MultiplyDense-incl.hpp:12-150),
// which issues one gemv/gemm per dense leaf (src/hmat_tools/MultiplyVector.cpp
// :14-69) and two per low-rank block (:71-128), recursing over the tree.
// Here a batch of jobs (each: one subtree of one H-matrix against one dense
// input) runs as two launches over flat work lists:
//   phase 1: T_b = W_b^T X_b for every low-rank block b of every job
//            (W = V, or U for the transpose), one CTA per block;
//   phase 2: for every row tile of every job, Y_tile = alpha * (sum over the
//            dense leaves and low-rank blocks covering the tile of
//            A_e(tile rows) * B_e) + beta * Y_tile, one CTA per tile, so each
//            output element is written once (no atomics, deterministic).
// Every stored matrix entry is read exactly once per launch pair.
#include <algorithm>
#include <cstring>

#include "engine.h"

namespace hmb {

namespace {

struct P1Item {
    const double* W;   // nin x r, ld ldw
    long long in_off;  // row offset into the job input
    long long t_off;   // offset of T (r x k, ld r) in the plan's T buffer
    int nin, r, ldw, job;
};

struct P2Item {
    long long out_off;  // row offset of the tile's first row in the job output
    int job, r0, rows, c0, cols, e0, e1, pad;
};

struct P2Entry {
    const double* A;   // element (i,p) = transA ? A[p + i*lda] : A[i + p*lda]
    long long b_off;   // B = (b_from_t ? T : job input) + b_off
    int lda, inner, transA, b_from_t, ldt, pad;
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ const JobArgs& job_of(const JobArgs* jobs, const JobArgs& job0,
                                                 int j) {
    return jobs ? jobs[j] : job0;
}

// ---------------------------------------------------------------------------
// Phase 1: T = W^T in
// ---------------------------------------------------------------------------
// Narrow: k <= NC.  Warps take columns of W; lanes stride over rows.
template <int NC>
__global__ void __launch_bounds__(kThreads)
p1_narrow_kernel(const P1Item* __restrict__ items, const JobArgs* __restrict__ jobs,
                 const JobArgs job0, double* __restrict__ Tbuf) {
    const P1Item it = items[blockIdx.x];
    const JobArgs& J = job_of(jobs, job0, it.job);
    const double* in = J.in + it.in_off;
    double* T = Tbuf + it.t_off;
    const int K = J.k, ldin = J.ldin;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = warp; j < it.r; j += kWarps) {
        const double* w = it.W + (long long)j * it.ldw;
        double acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = 0.0;
        int p = lane;
        for (; p + 96 < it.nin; p += 128) {
            double w0 = __ldg(w + p), w1 = __ldg(w + p + 32);
            double w2 = __ldg(w + p + 64), w3 = __ldg(w + p + 96);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (c < K) {
                    const double* x = in + (long long)c * ldin + p;
                    acc[c] = fma(w0, __ldg(x), acc[c]);
                    acc[c] = fma(w1, __ldg(x + 32), acc[c]);
                    acc[c] = fma(w2, __ldg(x + 64), acc[c]);
                    acc[c] = fma(w3, __ldg(x + 96), acc[c]);
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
p1_wide_kernel(const P1Item* __restrict__ items, const JobArgs* __restrict__ jobs,
               const JobArgs job0, double* __restrict__ Tbuf, int ctiles) {
    const P1Item it = items[blockIdx.x / ctiles];
    const JobArgs& J = job_of(jobs, job0, it.job);
    const double* in = J.in + it.in_off;
    double* T = Tbuf + it.t_off;
    const int K = J.k, ldin = J.ldin;
    const int ct = blockIdx.x % ctiles;
    const int c0 = ct * 32;
    if (c0 >= K) return;
    __shared__ double sW[32][33];
    __shared__ double sX[32][33];
    const int tid = threadIdx.x;
    // thread -> outputs (j = tid%32 + 32*jt ... ) : each thread 4 outputs
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
__device__ __forceinline__ void entry_b(const P2Entry& e, const JobArgs& J,
                                       const double* Tbuf, const double*& B, int& ldb) {
    if (e.b_from_t) { B = Tbuf + e.b_off; ldb = e.ldt; }
    else { B = J.in + e.b_off; ldb = J.ldin; }
}

// Narrow: cols <= NC, rows <= 64.  Lanes map to (row, inner sub-lane); warps
// split the inner dimension; partial sums reduced through shared memory.
template <int NC>
__global__ void __launch_bounds__(kThreads)
p2_narrow_kernel(const P2Item* __restrict__ items, const P2Entry* __restrict__ entries,
                 const JobArgs* __restrict__ jobs, const JobArgs job0,
                 const double* __restrict__ Tbuf) {
    const P2Item it = items[blockIdx.x];
    const JobArgs& J = job_of(jobs, job0, it.job);
    __shared__ double red[kWarps][64][NC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // rows-per-pass RL (power of two <= 32), inner sub-lanes 32/RL
    int RL = 1;
    while (RL < it.rows && RL < 32) RL <<= 1;
    const int sub = lane / RL, rl = lane % RL, nsub = 32 / RL;
    const int rpt = (it.rows + RL - 1) / RL;   // rows per thread (<= 64/RL)
    double acc[2][NC];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[a][c] = 0.0;
    // rows handled by this thread: rl + a*RL for a < rpt (rpt <= 2 when RL = 32;
    // when RL < 32, rows <= RL so rpt = 1)
    for (int ei = it.e0; ei < it.e1; ++ei) {
        P2Entry e = entries[ei];
        const double* EB;
        int ldb;
        entry_b(e, J, Tbuf, EB, ldb);
        const int stride = kWarps * nsub;
        for (int p = warp * nsub + sub; p < e.inner; p += stride) {
            double b[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c)
                b[c] = (c < it.cols) ? __ldg(EB + p + (long long)(it.c0 + c) * ldb) : 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                int i = rl + a * RL;
                if (a < rpt && i < it.rows) {
                    double av = load_a(e, it.r0 + i, p);
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc[a][c] = fma(av, b[c], acc[a][c]);
                }
            }
        }
    }
    // reduce over sub-lanes within the warp (lanes with equal rl)
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
    for (int o = threadIdx.x; o < it.rows * it.cols; o += kThreads) {
        int i = o % it.rows, c = o / it.rows;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) v += red[w][i][c];
        double* y = J.out + it.out_off + (it.r0 + i) + (long long)(it.c0 + c) * J.ldout;
        const double al = J.alpha_scale ? J.alpha * *J.alpha_scale : J.alpha;
        *y = J.beta == 0.0 ? al * v : al * v + J.beta * *y;
    }
}

// Wide: tile 64 rows x 64 cols, inner staged in chunks of 16; each thread
// owns a 4x4 register tile.
__global__ void __launch_bounds__(kThreads)
p2_wide_kernel(const P2Item* __restrict__ items, const P2Entry* __restrict__ entries,
               const JobArgs* __restrict__ jobs, const JobArgs job0,
               const double* __restrict__ Tbuf) {
    const P2Item it = items[blockIdx.x];
    const JobArgs& J = job_of(jobs, job0, it.job);
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
        const P2Entry e = entries[ei];
        const double* EB;
        int ldb;
        entry_b(e, J, Tbuf, EB, ldb);
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
                sB[pp][c] = (c < it.cols && p < e.inner)
                                ? __ldg(EB + p + (long long)(it.c0 + c) * ldb) : 0.0;
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
            if (c >= it.cols) continue;
            double* y = J.out + it.out_off + (it.r0 + i) + (long long)(it.c0 + c) * J.ldout;
            const double al = J.alpha_scale ? J.alpha * *J.alpha_scale : J.alpha;
            *y = J.beta == 0.0 ? al * acc[a][b] : al * acc[a][b] + J.beta * *y;
        }
    }
}

template <typename T>
void upload_list(DeviceBuffer<unsigned char>& buf, const std::vector<T>& v, cudaStream_t s) {
    buf.allocate(v.size() * sizeof(T), s);
    if (!v.empty())
        HMB_CUDA(cudaMemcpyAsync(buf.get(), v.data(), v.size() * sizeof(T),
                                 cudaMemcpyHostToDevice, s));
}

}  // namespace

struct MatPlan {
    DeviceBuffer<unsigned char> p1, p2, ent;
    size_t n1 = 0, n2 = 0;
    DeviceBuffer<double> T;
    int kmax = 0;
    int njobs = 0;
};

void MatPlanDeleter::operator()(MatPlan* p) const { delete p; }

PlanPtr build_plan(Context& ctx, const std::vector<JobSpec>& jobs) {
    HostScope hs(ctx, "hmm_plan");
    cudaStream_t st = ctx.stream;
    PlanPtr plan(new MatPlan);
    plan->njobs = (int)jobs.size();
    // leaves of each job's subtree (depth-first)
    std::vector<std::vector<int>> sub_leaves(jobs.size());
    int kmax = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
        HMB_REQUIRE(jobs[j].k >= 0, HM_ERR_ARGUMENT, "negative column count");
        kmax = std::max(kmax, jobs[j].k);
        const Structure& S = *jobs[j].H->S;
        std::vector<int> stack{jobs[j].root};
        while (!stack.empty()) {
            int b = stack.back();
            stack.pop_back();
            const Block& B = S.blocks[b];
            if (B.kind == KIND_NODE) {
                for (int c = S.q * S.q - 1; c >= 0; --c) stack.push_back(B.first_child + c);
            } else {
                sub_leaves[j].push_back(b);
            }
        }
    }
    plan->kmax = kmax;
    // phase 1: one item per (job, low-rank block)
    std::vector<P1Item> p1;
    std::vector<std::vector<long long>> t_of(jobs.size());
    long long t_total = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const JobSpec& J = jobs[j];
        const HMatrix& H = *J.H;
        const Structure& S = *H.S;
        const Block& R = S.blocks[J.root];
        t_of[j].assign(S.blocks.size(), -1);
        if (J.k == 0) continue;
        for (int b : sub_leaves[j]) {
            const Block& B = S.blocks[b];
            if (B.kind != KIND_LOWRANK || H.rank[b] == 0 || B.m == 0 || B.n == 0) continue;
            P1Item it{};
            if (!J.trans) {
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
            it.job = (int)j;
            it.t_off = t_total;
            t_of[j][b] = t_total;
            t_total += (long long)it.r * J.k;
            p1.push_back(it);
        }
    }
    plan->T.allocate((size_t)std::max<long long>(t_total, 1), st);
    // phase 2: one item per (job, output row tile, column tile)
    std::vector<P2Item> p2;
    std::vector<P2Entry> ent;
    const int CT = kmax > 8 ? 64 : 8;
    const int RT = 64;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const JobSpec& J = jobs[j];
        const HMatrix& H = *J.H;
        const Structure& S = *H.S;
        const Block& R = S.blocks[J.root];
        const Box& outBox = S.boxes[J.trans ? R.src_box : R.tgt_box];
        const int outBase = J.trans ? R.col_off : R.row_off;
        if (J.k == 0) continue;
        // bucket the subtree's leaf blocks by the output clusters they cover
        const int c0 = outBox.leaf0, nc = outBox.leaf1 - outBox.leaf0;
        std::vector<int> count(nc + 1, 0);
        for (int b : sub_leaves[j]) {
            const Block& B = S.blocks[b];
            if (B.m == 0 || B.n == 0) continue;
            const Box& ob = S.boxes[J.trans ? B.src_box : B.tgt_box];
            for (int c = ob.leaf0; c < ob.leaf1; ++c) count[c - c0 + 1]++;
        }
        for (int c = 0; c < nc; ++c) count[c + 1] += count[c];
        std::vector<int> bucket(count[nc]);
        {
            std::vector<int> fill(count.begin(), count.end() - 1);
            for (int b : sub_leaves[j]) {
                const Block& B = S.blocks[b];
                if (B.m == 0 || B.n == 0) continue;
                const Box& ob = S.boxes[J.trans ? B.src_box : B.tgt_box];
                for (int c = ob.leaf0; c < ob.leaf1; ++c) bucket[fill[c - c0]++] = b;
            }
        }
        for (int c = outBox.leaf0; c < outBox.leaf1; ++c) {
            const Box& cl = S.boxes[S.leaf_box[c]];
            if (cl.count == 0) continue;
            int e0 = (int)ent.size();
            for (int bi = count[c - c0]; bi < count[c - c0 + 1]; ++bi) {
                const int b = bucket[bi];
                const Block& B = S.blocks[b];
                P2Entry e{};
                if (B.kind == KIND_DENSE) {
                    if (!J.trans) {
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
                    if (!J.trans) {
                        e.A = H.U(b) + (cl.offset - B.row_off);
                        e.lda = B.m;
                    } else {
                        e.A = H.V(b) + (cl.offset - B.col_off);
                        e.lda = B.n;
                    }
                    e.transA = 0;
                    e.inner = H.rank[b];
                    e.b_from_t = 1;
                    e.b_off = t_of[j][b];
                    e.ldt = H.rank[b];
                }
                ent.push_back(e);
            }
            int e1 = (int)ent.size();
            for (int r0 = 0; r0 < cl.count; r0 += RT)
                for (int c0 = 0; c0 < J.k; c0 += CT) {
                    P2Item it{};
                    it.out_off = cl.offset - outBase;
                    it.job = (int)j;
                    it.r0 = r0;
                    it.rows = std::min(RT, cl.count - r0);
                    it.c0 = c0;
                    it.cols = std::min(CT, J.k - c0);
                    it.e0 = e0;
                    it.e1 = e1;
                    p2.push_back(it);
                }
        }
    }
    plan->n1 = p1.size();
    plan->n2 = p2.size();
    upload_list(plan->p1, p1, st);
    upload_list(plan->p2, p2, st);
    upload_list(plan->ent, ent, st);
    return plan;
}

void execute_plan(Context& ctx, MatPlan& plan, const std::vector<JobArgs>& args) {
    HMB_REQUIRE((int)args.size() == plan.njobs, HM_ERR_INTERNAL, "job count mismatch");
    if (args.empty()) return;
    cudaStream_t st = ctx.stream;
    DeviceBuffer<JobArgs> dj;
    const JobArgs* jobs = nullptr;
    JobArgs job0 = args[0];
    if (args.size() > 1) {
        dj.upload(args, st);
        jobs = dj.get();
    }
    const int kmax = plan.kmax;
    double* T = plan.T.get();
    if (plan.n1) {
        LaunchScope ls(ctx, "hmm_lowrank_inner");
        const P1Item* pi = (const P1Item*)plan.p1.get();
        const unsigned n = (unsigned)plan.n1;
        if (kmax <= 1)
            p1_narrow_kernel<1><<<n, kThreads, 0, st>>>(pi, jobs, job0, T);
        else if (kmax <= 4)
            p1_narrow_kernel<4><<<n, kThreads, 0, st>>>(pi, jobs, job0, T);
        else if (kmax <= 8)
            p1_narrow_kernel<8><<<n, kThreads, 0, st>>>(pi, jobs, job0, T);
        else {
            int ct = ceil_div(kmax, 32);
            p1_wide_kernel<<<n * ct, kThreads, 0, st>>>(pi, jobs, job0, T, ct);
        }
        HMB_CHECK_LAUNCH();
    }
    if (plan.n2) {
        LaunchScope ls(ctx, "hmm_row_tiles");
        const P2Item* pi = (const P2Item*)plan.p2.get();
        const P2Entry* pe = (const P2Entry*)plan.ent.get();
        const unsigned n = (unsigned)plan.n2;
        if (kmax <= 1)
            p2_narrow_kernel<1><<<n, kThreads, 0, st>>>(pi, pe, jobs, job0, T);
        else if (kmax <= 4)
            p2_narrow_kernel<4><<<n, kThreads, 0, st>>>(pi, pe, jobs, job0, T);
        else if (kmax <= 8)
            p2_narrow_kernel<8><<<n, kThreads, 0, st>>>(pi, pe, jobs, job0, T);
        else
            p2_wide_kernel<<<n, kThreads, 0, st>>>(pi, pe, jobs, job0, T);
        HMB_CHECK_LAUNCH();
    }
}

void run_jobs(Context& ctx, const std::vector<MatJob>& jobs) {
    if (jobs.empty()) return;
    std::vector<JobSpec> specs;
    std::vector<JobArgs> args;
    for (const MatJob& J : jobs) {
        specs.push_back({J.H, J.root, J.trans, J.k});
        args.push_back({J.in, J.out, J.alpha, J.beta, J.ldin, J.ldout, J.k, 0, nullptr});
    }
    PlanPtr plan = build_plan(ctx, specs);
    execute_plan(ctx, *plan, args);
}

}  // namespace hmb
