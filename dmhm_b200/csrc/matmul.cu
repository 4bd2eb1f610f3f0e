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
//            (W = V, or U for the transpose): for few columns one warp per
//            row segment of a block, whole blocks per CTA; otherwise one
//            CTA per block and 32-column tile;
//   phase 2: for every output row tile of every job, Y_tile = alpha * (sum
//            over the dense leaves and low-rank blocks covering the tile of
//            A_e(tile rows) * B_e) + beta * Y_tile, one CTA per tile, so each
//            output element is written once (no atomics, deterministic).
// Every stored matrix entry is read exactly once per launch pair.  A CTA finds
// its job by binary search over the jobs' first work-item indices.
#include <algorithm>
#include <tuple>
#include <type_traits>
#include <cstring>
#include <map>
#include <mutex>

#include "engine.h"
#include "templates.h"

namespace hmb {

// What a CTA needs to run its share of one job.
struct JobExec {
    const double* hb;    // storage of the job's H-matrix (work lists hold offsets)
    const float* hb32;   // TF32 path: its TF32-rounded FP32 copy
    const float* in32;   // TF32 path: the input, rounded, ld ldin32
    float* T32;          // TF32 path: phase-1 results
    int ldin32, pad32;
    const P1T* p1;
    const W1Tile* w1;
    const int* w1cp;     // wide: chunk prefix over the W1 tiles (n_w1 + 1)
    const int* tcp;      // wide: chunk prefix over the row tiles (n2 + 1)
    const int* ekc;      // wide: first chunk of each entry within its tile
    double* part;        // wide: partials of tiles cut between CTAs (shared by all jobs)
    const P2T* p2;
    const P2Entry* ent;
    const double* in;
    double* out;
    double* T;
    int* cnt1;           // per item: pieces finished (zero between launches)
    int* cnt2;           // per row tile: pieces finished
    const double* alpha_scale;
    double alpha, beta;
    long long p1_begin, p2_begin;   // first global work item (row / column) of this job
    int n1, n2, ldin, ldout, k, ct1, ct2, pad;   // ct*: column tiles per item
};

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr size_t kLayoutGroups = 16;   // layout groups kept per context

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
// Sum of v[f] over the 32 lanes for 16 values at once (a transposing
// butterfly: 16 shuffles instead of 80).  Lanes 2f and 2f+1 end up holding
// the total of value f in v[0].
__device__ __forceinline__ void warp_transpose_sum16(double (&v)[16], int lane) {
#pragma unroll
    for (int h = 8, o = 16; h >= 1; h >>= 1, o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const double send = up ? v[i] : v[i + h];
            const double keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// Even split of a concatenation of C work items (rows of the phase-1 items,
// columns of the phase-2 tiles, over all jobs) among GW <= C warps: warp w
// takes [w C / GW, (w+1) C / GW), never empty.  An item or tile cut between
// warps wa..wb is summed by the piece that finishes last (a counter per item
// or tile, reset by that piece), over the warps in order; warp w leaves the
// partial sum of its first piece in scratch slot 2w, of its last in 2w + 1.
__device__ __forceinline__ long long split_start(long long w, long long GW, long long C) {
    return w * C / GW;
}
__device__ __forceinline__ long long split_owner(long long g, long long GW, long long C) {
    return ((g + 1) * GW + C - 1) / C - 1;
}
__device__ __forceinline__ long long piece_slot(long long q, long long wa, bool wa_starts_here) {
    return 2 * q + ((q == wa && !wa_starts_here) ? 1 : 0);
}

// Narrow: k <= NC.  Persistent warps stream their share of the items' rows.
// A lane owns rows p and p + 32 of a 64-row step and loads JC = 16/NC columns
// of W for both (2 JC loads in flight); the 16 partial sums of a column chunk
// are reduced across the warp by a transposing butterfly.
template <int NC>
__global__ void __launch_bounds__(kThreads, 2)
p1_stream_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0, long long C,
                 long long GW, double* __restrict__ S, int rmax,
                 const int* __restrict__ start) {
    constexpr int JC = 16 / NC;
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (w >= GW) return;
    const long long slot_len = (long long)rmax * NC;
    long long g = split_start(w, GW, C);
    const long long gend = split_start(w + 1, GW, C);
    bool first = true;
    // one job with precomputed starts: items follow one another
    const bool seq = jobs == nullptr && start != nullptr;
    int item = seq ? start[w] - 1 : 0;
    while (g < gend) {
        const JobExec& J = jobs ? jobs[find_job(jobs, njobs, g, false)] : job0;
        const long long local = g - J.p1_begin;
        if (seq) {
            ++item;
        } else {
            item = 0;
            int hi = J.n1 - 1;
            while (item < hi) {
                const int mid = (item + hi + 1) >> 1;
                if (J.p1[mid].c0 <= local) item = mid;
                else hi = mid - 1;
            }
        }
        const P1T it = J.p1[item];
        if (item + 1 < J.n1) asm volatile("prefetch.global.L1 [%0];" ::"l"(J.p1 + item + 1));
        const int K = J.k, ldin = J.ldin, r = it.r;
        const int p0 = (int)(local - it.c0);
        const int p1 = (int)min((long long)it.nin, gend - J.p1_begin - it.c0);
        const bool whole = p0 == 0 && p1 == it.nin;
        double* dst = whole ? J.T + it.t_rel * K : S + (2 * w + (first ? 0 : 1)) * slot_len;
        const double* in = J.in + it.in_off;
        for (int j0 = 0; j0 < r; j0 += JC) {
            double v[16];
#pragma unroll
            for (int f = 0; f < 16; ++f) v[f] = 0.0;
            const double* wp = J.hb + it.w + (long long)j0 * it.ldw;
            for (int pa = p0 + lane; pa < p1; pa += 64) {
                const int pb = pa + 32;
                const bool okb = pb < p1;
                double wa[JC], wb[JC], xa[NC], xb[NC];
#pragma unroll
                for (int jj = 0; jj < JC; ++jj) {
                    const bool cj = j0 + jj < r;
                    wa[jj] = cj ? __ldg(wp + pa + (long long)jj * it.ldw) : 0.0;
                    wb[jj] = (okb && cj) ? __ldg(wp + pb + (long long)jj * it.ldw) : 0.0;
                }
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    xa[c] = (c < K) ? __ldg(in + pa + (long long)c * ldin) : 0.0;
                    xb[c] = (okb && c < K) ? __ldg(in + pb + (long long)c * ldin) : 0.0;
                }
#pragma unroll
                for (int jj = 0; jj < JC; ++jj)
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        v[jj * NC + c] = fma(wb[jj], xb[c], fma(wa[jj], xa[c], v[jj * NC + c]));
            }
            warp_transpose_sum16(v, lane);
            if ((lane & 1) == 0) {
                const int f = lane >> 1, jj = f / NC, c = f % NC;
                if (j0 + jj < r && c < K) dst[(j0 + jj) + (long long)c * r] = v[0];
            }
        }
        if (!whole) {
            __threadfence();
            __syncwarp();
            const long long G0 = J.p1_begin + it.c0;
            const long long wa = split_owner(G0, GW, C), wb = split_owner(G0 + it.nin - 1, GW, C);
            int last = 0;
            if (lane == 0) last = atomicAdd(J.cnt1 + item, 1) == (int)(wb - wa);
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                __threadfence();
                const bool wa_here = split_start(wa, GW, C) == G0;
                double* T = J.T + it.t_rel * K;
                for (int o = lane; o < r * K; o += 32) {
                    double t = 0.0;
                    for (long long q = wa; q <= wb; ++q)
                        t += __ldcg(S + piece_slot(q, wa, wa_here) * slot_len + o);
                    T[o] = t;
                }
                if (lane == 0) J.cnt1[item] = 0;
            }
        }
        g = J.p1_begin + it.c0 + p1;
        first = false;
    }
}

// ---------------------------------------------------------------------------
// Phase 2: Y_tile = alpha sum_e A_e B_e + beta Y_tile
// ---------------------------------------------------------------------------
__device__ __forceinline__ double load_a(const double* hb, const P2Entry& e, int i, int p) {
    const double* A = hb + e.a;
    return e.transA ? __ldg(A + p + (long long)i * e.lda) : __ldg(A + i + (long long)p * e.lda);
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

// Narrow: columns <= NC, rows <= 32, a streaming (HBM-bound) kernel.
// Persistent warps stream their share of the tiles' concatenated inner
// dimensions (entry e of a tile covers [cbeg, cbeg + inner)).  Within a
// warp, "column workers" (sub-groups of lanes, one lane per row) split the
// piece evenly and keep U columns of loads in flight.
template <int NC>
__global__ void __launch_bounds__(kThreads, 2)
p2_stream_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0, long long C,
                 long long GW, double* __restrict__ S, const int2* __restrict__ start) {
    constexpr int U = NC == 1 ? 16 : 4;
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (w >= GW) return;
    constexpr long long slot_len = 32LL * NC;
    long long g = split_start(w, GW, C);
    const long long gend = split_start(w + 1, GW, C);
    bool first = true;
    // one job with precomputed starts: tiles follow one another
    const bool seq = jobs == nullptr && start != nullptr;
    int tile = 0, ent_first = -1;
    if (seq) {
        const int2 s0 = start[w];
        tile = s0.x;
        ent_first = s0.y;
    }
    while (g < gend) {
        const JobExec& J = jobs ? jobs[find_job(jobs, njobs, g, true)] : job0;
        const long long local = g - J.p2_begin;
        P2T it;
        if (seq) {
            if (!first) {
                do { it = J.p2[++tile]; } while (it.width == 0);
            } else {
                it = J.p2[tile];
            }
        } else {
            tile = 0;
            int hi = J.n2 - 1;
            while (tile < hi) {
                const int mid = (tile + hi + 1) >> 1;
                if (J.p2[mid].c0 <= local) tile = mid;
                else hi = mid - 1;
            }
            it = J.p2[tile];
        }
        const int cols = J.k;
        const int q0 = (int)(local - it.c0);
        const int q1 = (int)min((long long)it.width, gend - J.p2_begin - it.c0);
        const bool whole = q0 == 0 && q1 == it.width;
        // rows-per-pass RL (power of two <= 32), column sub-groups 32/RL
        int RL = 1;
        while (RL < it.rows && RL < 32) RL <<= 1;
        const int sub = lane / RL, rl = lane % RL, nsub = 32 / RL;
        const bool row_ok = rl < it.rows;
        const int row = it.r0 + rl;
        double acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = 0.0;
        {
            const int chunk = (q1 - q0 + nsub - 1) / nsub;
            int p = q0 + sub * chunk;
            const int pend = min(q1, p + chunk);
            int ei = it.e0;
            if (seq && nsub == 1) {
                if (first) ei = ent_first;
            } else {
                int hi = it.e1 - 1;
                while (ei < hi) {
                    const int mid = (ei + hi + 1) >> 1;
                    if (J.ent[mid].cbeg <= p) ei = mid;
                    else hi = mid - 1;
                }
            }
            while (p < pend) {
                const P2Entry e = J.ent[ei];
                if (ei + 1 < it.e1) asm volatile("prefetch.global.L1 [%0];" ::"l"(J.ent + ei + 1));
                const double* EB;
                int ldb;
                entry_b(e, J, EB, ldb);
                const int stop = min(pend, e.cbeg + e.inner);
                int q = p - e.cbeg;                 // column within the entry
                const int qstop = stop - e.cbeg;
                for (; q + U - 1 < qstop; q += U) {
                    double av[U], bv[U][NC];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
#pragma unroll
                        for (int c = 0; c < NC; ++c)
                            bv[u][c] = (c < cols) ? __ldg(EB + (q + u) + (long long)c * ldb) : 0.0;
                        av[u] = row_ok ? load_a(J.hb, e, row, q + u) : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[c] = fma(av[u], bv[u][c], acc[c]);
                }
                for (; q < qstop; ++q) {
                    const double av = row_ok ? load_a(J.hb, e, row, q) : 0.0;
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        if (c < cols) acc[c] = fma(av, __ldg(EB + q + (long long)c * ldb), acc[c]);
                }
                p = stop;
                ++ei;
            }
        }
        // reduce over the column sub-groups (lanes with equal rl)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double v = acc[c];
            for (int o = 16; o >= RL; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[c] = v;
        }
        if (whole) {
            if (sub == 0 && row_ok)
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    if (c < cols) store_out(J, it, rl, c, acc[c]);
        } else {
            double* P = S + (2 * w + (first ? 0 : 1)) * slot_len;   // 32 x NC, ld 32
            if (sub == 0 && row_ok)
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    if (c < cols) P[rl + 32 * c] = acc[c];
            __threadfence();
            __syncwarp();
            const long long G0 = J.p2_begin + it.c0;
            const long long wa = split_owner(G0, GW, C), wb = split_owner(G0 + it.width - 1, GW, C);
            int last = 0;
            if (lane == 0) last = atomicAdd(J.cnt2 + tile, 1) == (int)(wb - wa);
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                __threadfence();
                const bool wa_here = split_start(wa, GW, C) == G0;
                for (int o = lane; o < it.rows * cols; o += 32) {
                    const int i = o % it.rows, c = o / it.rows;
                    double t = 0.0;
                    for (long long q = wa; q <= wb; ++q)
                        t += __ldcg(S + piece_slot(q, wa, wa_here) * slot_len + i + 32 * c);
                    store_out(J, it, i, c, t);
                }
                if (lane == 0) J.cnt2[tile] = 0;
            }
        }
        g = J.p2_begin + it.c0 + q1;
        first = false;
    }
}

// Row tiles without entries, over all jobs of a launch (list of (job, tile)):
// output = beta * output (alpha times an empty sum).
__global__ void p2_zero_kernel(const JobExec* __restrict__ jobs, const JobExec job0,
                               const int2* __restrict__ list, int n) {
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const int2 jt = list[t];
        const JobExec& J = jobs ? jobs[jt.x] : job0;
        const P2T it = J.p2[jt.y];
        for (int o = threadIdx.x; o < it.rows * J.k; o += blockDim.x)
            store_out(J, it, o % it.rows, o / it.rows, 0.0);
    }
}

// One launch for the tiles without entries of every job.
void launch_zero_tiles(Context& ctx, const std::vector<std::shared_ptr<JobTemplate>>& tmpl,
                       const std::vector<MatJob>& jobs, const JobExec* jobs_d, const JobExec& job0) {
    std::vector<int2> list;
    int j = 0;
    for (size_t i = 0; i < jobs.size(); ++i) {
        if (jobs[i].k == 0) continue;
        for (int t : tmpl[i]->hzero) list.push_back(make_int2(j, t));
        ++j;
    }
    if (list.empty()) return;
    DeviceBuffer<int2> d;
    d.upload(list, ctx.stream);
    LaunchScope ls(ctx, "hmm_zero_tiles");
    p2_zero_kernel<<<std::min((int)list.size(), 4 * ctx.num_sms), 256, 0, ctx.stream>>>(
        jobs_d, job0, d.get(), (int)list.size());
    HMB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Wide (many columns): FP64 64 x 64 output tiles on the FP64 tensor cores
// (mma.m8n8k4.f64), 4 warps of 32 x 32 each (4 x 4 MMA blocks, 32
// accumulators a thread); operands staged through shared memory in chunks
// of KC inner indices by cp.async, two stages (the next chunk loads while
// this one is multiplied).
// ---------------------------------------------------------------------------
constexpr int WT = kWideTile;   // tile rows = tile columns
constexpr int KC = 16;          // inner chunk
constexpr int WTHREADS = 128;   // 2 x 2 warps of 32 x 32
constexpr int SP = WT + 8;      // smem row: fragment loads hit 32 distinct banks

constexpr int NSTAGE = 2;       // chunk buffers per CTA
template <typename E>
struct WideSmemT {
    E a[NSTAGE][KC][SP];   // a[buf][p][i] = A(i, p)
    E b[NSTAGE][KC][SP];   // b[buf][p][c] = B(p, c)
};
using WideSmem = WideSmemT<double>;

// The copies carry no "memory" clobber: their shared-memory destinations are
// read only after cp_async_wait (which has one) and a barrier, and without
// it the compiler may keep the work-list fields that address the copies in
// registers instead of reloading them from global memory after every copy.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src),
                 "r"(valid ? 4 : 0));
}

// TF32 tensor-core MMA 16 x 8 x 8, FP32 accumulation.  Fragments (g = lane/4,
// t = lane%4): A a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4); B b0 (t, g),
// b1 (t+4, g); C c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1).
__device__ __forceinline__ void tmma(float* d, const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float round_tf32(double x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"((float)x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src),
                 "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Accumulator slot s = (mb * 4 + nb) * 2 + h of a thread holds tile element
// (row_of(s), col_of(s)) (the m8n8k4 C fragment: row lane/4, columns
// 2 (lane%4) + h of MMA block (mb, nb) of the warp's 32 x 32 quarter).
__device__ __forceinline__ int acc_row(int s, int warp, int lane) {
    return (warp & 1) * 32 + (s >> 3) * 8 + (lane >> 2);
}
__device__ __forceinline__ int acc_col(int s, int warp, int lane) {
    return (warp >> 1) * 32 + ((s >> 1) & 3) * 8 + 2 * (lane & 3) + (s & 1);
}

// TF32 tiles: slot s = ((mb * 4 + nb) * 4 + e) of MMA block (mb, nb) (16 x 8)
// of the warp's 32 x 32 quarter, C fragment element e.
__device__ __forceinline__ int acc_row_tf(int s, int warp, int lane) {
    return (warp & 1) * 32 + (s >> 4) * 16 + (lane >> 2) + ((s & 2) ? 8 : 0);
}
__device__ __forceinline__ int acc_col_tf(int s, int warp, int lane) {
    return (warp >> 1) * 32 + ((s >> 2) & 3) * 8 + 2 * (lane & 3) + (s & 1);
}

__device__ __forceinline__ void wide_mma_tf(const WideSmemT<float>& sm, int buf, int warp, int lane,
                                            float (&acc)[32]) {
    const int g = lane >> 2, t = lane & 3;
    const int r0 = (warp & 1) * 32 + g, c0 = (warp >> 1) * 32 + g;
#pragma unroll
    for (int kb = 0; kb < KC; kb += 8) {
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
            a[mb][0] = __float_as_uint(sm.a[buf][kb + t][r0 + mb * 16]);
            a[mb][1] = __float_as_uint(sm.a[buf][kb + t][r0 + mb * 16 + 8]);
            a[mb][2] = __float_as_uint(sm.a[buf][kb + t + 4][r0 + mb * 16]);
            a[mb][3] = __float_as_uint(sm.a[buf][kb + t + 4][r0 + mb * 16 + 8]);
        }
#pragma unroll
        for (int nb = 0; nb < 4; ++nb) {
            b[nb][0] = __float_as_uint(sm.b[buf][kb + t][c0 + nb * 8]);
            b[nb][1] = __float_as_uint(sm.b[buf][kb + t + 4][c0 + nb * 8]);
        }
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
            for (int nb = 0; nb < 4; ++nb) tmma(&acc[(mb * 4 + nb) * 4], a[mb], b[nb]);
    }
}

// acc += A(warp rows, chunk) B(chunk, warp columns) over one staged chunk.
__device__ __forceinline__ void wide_mma(const WideSmem& sm, int buf, int warp, int lane,
                                         double (&acc)[32]) {
    const int r0 = (warp & 1) * 32 + (lane >> 2), c0 = (warp >> 1) * 32 + (lane >> 2);
#pragma unroll
    for (int ks = 0; ks < KC / 4; ++ks) {
        const int p = ks * 4 + (lane & 3);
        double a[4], b[4];
#pragma unroll
        for (int mb = 0; mb < 4; ++mb) a[mb] = sm.a[buf][p][r0 + mb * 8];
#pragma unroll
        for (int nb = 0; nb < 4; ++nb) b[nb] = sm.b[buf][p][c0 + nb * 8];
#pragma unroll
        for (int mb = 0; mb < 4; ++mb)
#pragma unroll
            for (int nb = 0; nb < 4; ++nb) {
                double (&d)[2] = *reinterpret_cast<double(*)[2]>(&acc[(mb * 4 + nb) * 2]);
                dmma(d, a[mb], b[nb]);
            }
    }
}

// B chunk: B(p, c) = Bp[p + c * ldb] for p < len, c < cols (p fastest).
__device__ __forceinline__ void load_b_chunk(WideSmem& sm, int buf, const double* Bp, int ldb,
                                             int len, int cols, int tid) {
#pragma unroll
    for (int e = tid; e < KC * WT; e += WTHREADS) {
        const int p = e % KC, c = e / KC;
        const bool v = p < len && c < cols;
        cp_async8(&sm.b[buf][p][c], v ? Bp + p + (long long)c * ldb : Bp, v);
    }
}

__device__ __forceinline__ void load_b_chunk(WideSmemT<float>& sm, int buf, const float* Bp, int ldb,
                                             int len, int cols, int tid) {
#pragma unroll
    for (int e = tid; e < KC * WT; e += WTHREADS) {
        const int p = e % KC, c = e / KC;
        const bool v = p < len && c < cols;
        cp_async4(&sm.b[buf][p][c], v ? Bp + p + (long long)c * ldb : Bp, v);
    }
}

// The wide kernels stream a sequence of KC-chunks: phase 1 the chunks of
// every W1 tile (its nin input rows), phase 2 the chunks of every row tile's
// entries (no chunk spans two entries), over all jobs.  A persistent CTA takes
// an even share [b C / G, (b+1) C / G) of the sequence; the next chunk (of the
// same or the next tile) loads while the current one is multiplied.  A tile
// whose chunks a CTA holds completely is written directly; a tile cut between
// CTAs b_a..b_b leaves 64 x 64 partials (slot 2b for a CTA's first piece,
// 2b + 1 for its last) that the piece finishing last adds up in CTA order.
struct ChunkPos {
    int job, tile, ei, pos;   // phase 1: ei unused, pos = row offset in the tile's input
};

template <int PHASE>
__device__ __forceinline__ int tiles_of(const JobExec& J) { return PHASE == 1 ? J.n1 : J.n2; }
template <int PHASE>
__device__ __forceinline__ const int* chunk_prefix(const JobExec& J) { return PHASE == 1 ? J.w1cp : J.tcp; }

// TF: the TF32 form (FP32 copy of the blocks and of the input, TF32
// tensor-core MMA, FP32 accumulation, FP64 output).
// At most 128 registers a thread, so that 4 CTAs share an SM (152 without
// the bound: 3 CTAs per SM, 2 % slower on the 128 x 128, 64-column product).
template <int PHASE, bool TF>
__global__ void __launch_bounds__(WTHREADS, 4)
wide_kernel(const JobExec* __restrict__ jobs, int njobs, const JobExec job0, long long C, int G) {
    using E = typename std::conditional<TF, float, double>::type;
    extern __shared__ __align__(16) unsigned char wide_smem[];
    WideSmemT<E>& sm = *reinterpret_cast<WideSmemT<E>*>(wide_smem);
    __shared__ int last_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = blockIdx.x, y = blockIdx.y;
    const long long g0 = split_start(b, G, C), g1 = split_start(b + 1, G, C);
    if (g0 >= g1) return;
    auto job = [&](int j) -> const JobExec& { return jobs ? jobs[j] : job0; };
    // locate the first chunk
    ChunkPos cur{};
    {
        cur.job = jobs ? find_job(jobs, njobs, g0, PHASE == 2) : 0;
        const JobExec& J = job(cur.job);
        const long long local = g0 - (PHASE == 1 ? J.p1_begin : J.p2_begin);
        const int* cp = chunk_prefix<PHASE>(J);
        int lo = 0, hi = tiles_of<PHASE>(J) - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cp[mid] <= local) lo = mid;
            else hi = mid - 1;
        }
        // skip tiles without chunks
        while (cp[lo + 1] <= local) ++lo;
        cur.tile = lo;
        const int kin = (int)(local - cp[lo]);
        if (PHASE == 1) {
            cur.pos = kin * KC;
        } else {
            const P2T it = J.p2[lo];
            int e = it.e0, eh = it.e1 - 1;
            while (e < eh) {
                const int mid = (e + eh + 1) >> 1;
                if (J.ekc[mid] <= kin) e = mid;
                else eh = mid - 1;
            }
            cur.ei = e;
            cur.pos = (kin - J.ekc[e]) * KC;
        }
    }
    // loads the chunk at `c` into buffer `buf`; returns whether it is the last
    // chunk of its tile; advances `c`
    auto load = [&](ChunkPos& c, int buf) -> bool {
        const JobExec& J = job(c.job);
        const int cols = min(WT, J.k - y * WT);
        bool last;
        if (PHASE == 1) {
            const W1Tile* t = J.w1 + c.tile;
            const int len = min(KC, t->nin - c.pos), rows = t->rows;
#pragma unroll
            for (int e = tid; e < WT * KC; e += WTHREADS) {
                const int p = e % KC, i = e / KC;   // W columns are contiguous
                const bool v = p < len && i < rows;
                const long long wo = t->wcol[v ? i : 0];
                if constexpr (TF) {
                    const float* w0 = J.hb32 + wo;
                    cp_async4(&sm.a[buf][p][i], v ? w0 + c.pos + p : w0, v);
                } else {
                    const double* w0 = J.hb + wo;
                    cp_async8(&sm.a[buf][p][i], v ? w0 + c.pos + p : w0, v);
                }
            }
            if constexpr (TF)
                load_b_chunk(sm, buf, J.in32 + t->in_off + c.pos + (long long)y * WT * J.ldin32,
                             J.ldin32, len, cols, tid);
            else
                load_b_chunk(sm, buf, J.in + t->in_off + c.pos + (long long)y * WT * J.ldin,
                             J.ldin, len, cols, tid);
            c.pos += len;
            last = c.pos >= t->nin;
        } else {
            const P2T it = J.p2[c.tile];
            const P2Entry e = J.ent[c.ei];
            const int len = min(KC, e.inner - c.pos);
            const E* Eb;
            if constexpr (TF) Eb = J.hb32 + e.a;
            else Eb = J.hb + e.a;
            if (!e.transA) {
                const E* A = Eb + it.r0 + (long long)c.pos * e.lda;
#pragma unroll
                for (int x = tid; x < WT * KC; x += WTHREADS) {
                    const int i = x % WT, p = x / WT;   // rows contiguous
                    const bool v = p < len && i < it.rows;
                    if constexpr (TF) cp_async4(&sm.a[buf][p][i], v ? A + i + (long long)p * e.lda : Eb, v);
                    else cp_async8(&sm.a[buf][p][i], v ? A + i + (long long)p * e.lda : Eb, v);
                }
            } else {
                const E* A = Eb + c.pos + (long long)it.r0 * e.lda;
#pragma unroll
                for (int x = tid; x < WT * KC; x += WTHREADS) {
                    const int p = x % KC, i = x / KC;   // inner index contiguous
                    const bool v = p < len && i < it.rows;
                    if constexpr (TF) cp_async4(&sm.a[buf][p][i], v ? A + p + (long long)i * e.lda : Eb, v);
                    else cp_async8(&sm.a[buf][p][i], v ? A + p + (long long)i * e.lda : Eb, v);
                }
            }
            if constexpr (TF) {
                const float* EB;
                int ldb;
                if (e.b_from_t) { EB = J.T32 + e.b_off * J.k; ldb = e.ldt; }
                else { EB = J.in32 + e.b_off; ldb = J.ldin32; }
                load_b_chunk(sm, buf, EB + c.pos + (long long)y * WT * ldb, ldb, len, cols, tid);
            } else {
                const double* EB;
                int ldb;
                entry_b(e, J, EB, ldb);
                load_b_chunk(sm, buf, EB + c.pos + (long long)y * WT * ldb, ldb, len, cols, tid);
            }
            c.pos += len;
            last = false;
            if (c.pos >= e.inner) {
                c.pos = 0;
                ++c.ei;
                last = c.ei >= it.e1;
            }
        }
        cp_async_commit();
        if (last) {   // move to the next tile with chunks (possibly of the next job)
            c.pos = 0;
            for (;;) {
                ++c.tile;
                if (c.tile >= tiles_of<PHASE>(job(c.job))) {
                    if (!jobs || c.job + 1 >= njobs) break;
                    ++c.job;
                    c.tile = -1;
                    continue;
                }
                const int* cp = chunk_prefix<PHASE>(job(c.job));
                if (cp[c.tile + 1] > cp[c.tile]) break;
            }
            if (PHASE == 2 && c.tile < tiles_of<PHASE>(job(c.job))) c.ei = job(c.job).p2[c.tile].e0;
        }
        return last;
    };
    E acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0;
    auto arow = [&](int k) { return TF ? acc_row_tf(k, warp, lane) : acc_row(k, warp, lane); };
    auto acol = [&](int k) { return TF ? acc_col_tf(k, warp, lane) : acc_col(k, warp, lane); };
    // NSTAGE-deep ring: chunk q sits in buffer q % NSTAGE and is issued
    // NSTAGE - 1 chunks ahead; one commit group per chunk slot (empty past
    // the end) keeps the wait count constant
    ChunkPos loaded[NSTAGE];
    bool lastc[NSTAGE];
    const long long n = g1 - g0;
#pragma unroll
    for (int s = 0; s < NSTAGE - 1; ++s) {
        if (s < n) {
            loaded[s] = cur;
            lastc[s] = load(cur, s);
        } else {
            cp_async_commit();
        }
    }
    bool first_piece = true;
    for (long long q = 0; q < n; ++q) {
        const long long qn = q + NSTAGE - 1;
        const int bn = (int)(qn % NSTAGE);
        if (qn < n) {
            loaded[bn] = cur;
            lastc[bn] = load(cur, bn);
        } else {
            cp_async_commit();
        }
        cp_async_wait<NSTAGE - 1>();
        __syncthreads();
        const int buf = (int)(q % NSTAGE);
        if constexpr (TF) wide_mma_tf(sm, buf, warp, lane, acc);
        else wide_mma(sm, buf, warp, lane, acc);
        __syncthreads();
        if (!lastc[buf] && q + 1 < n) continue;
        // flush the tile of this chunk
        const ChunkPos& t = loaded[buf];
        const JobExec& J = job(t.job);
        const int cols = min(WT, J.k - y * WT);
        const long long base = PHASE == 1 ? J.p1_begin : J.p2_begin;
        const int* cp = chunk_prefix<PHASE>(J);
        const long long T0 = base + cp[t.tile], T1 = base + cp[t.tile + 1];
        const bool whole = T0 >= g0 && T1 <= g1;
        int rows;
        const W1Tile* wt = nullptr;
        P2T it{};
        if (PHASE == 1) {
            wt = J.w1 + t.tile;
            rows = wt->rows;
        } else {
            it = J.p2[t.tile];
            rows = it.rows;
        }
        auto emit = [&](int i, int c, double v) {
            if (PHASE == 1) {
                const long long o = wt->trel[i] * J.k + wt->tj[i] + (long long)(y * WT + c) * wt->tr[i];
                if constexpr (TF) J.T32[o] = round_tf32(v);
                else J.T[o] = v;
            } else {
                store_out(J, it, i, y * WT + c, v);
            }
        };
        if (whole && PHASE == 1) {
            // the thread's 32 accumulators lie in 4 tile rows: their T
            // offsets are loaded once, before the stores (which the compiler
            // must otherwise assume may change them)
            auto rslot = [](int k) { return TF ? (((k >> 4) << 1) | ((k >> 1) & 1)) : (k >> 3); };
            long long rbase[4], rstep[4];
            const long long kk = J.k;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = arow(TF ? (((q >> 1) << 4) | ((q & 1) << 1)) : q * 8);
                const bool ok = i < rows;
                rbase[q] = ok ? wt->trel[i] * kk + wt->tj[i] : 0;
                rstep[q] = ok ? (long long)wt->tr[i] : 0;
            }
            double* Tp = J.T;
            float* T32p = J.T32;
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const int i = arow(k), c = acol(k);
                if (i < rows && c < cols) {
                    const long long o = rbase[rslot(k)] + (long long)(y * WT + c) * rstep[rslot(k)];
                    if constexpr (TF) T32p[o] = round_tf32((double)acc[k]);
                    else Tp[o] = (double)acc[k];
                }
            }
        } else if (whole) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const int i = arow(k), c = acol(k);
                if (i < rows && c < cols) emit(i, c, (double)acc[k]);
            }
        } else {
            double* part = J.part + ((long long)y * 2 * G) * (WT * WT);
            double* mine = part + (2LL * b + (first_piece ? 0 : 1)) * (WT * WT);
#pragma unroll
            for (int k = 0; k < 32; ++k) mine[arow(k) + WT * acol(k)] = (double)acc[k];
            __threadfence();
            __syncthreads();
            const long long wa = split_owner(T0, G, C), wb = split_owner(T1 - 1, G, C);
            int* cnt = (PHASE == 1 ? J.cnt1 : J.cnt2) + (long long)t.tile * gridDim.y + y;
            if (tid == 0) last_flag = atomicAdd(cnt, 1) == (int)(wb - wa);
            __syncthreads();
            if (last_flag) {
                __threadfence();
                const bool wa_here = split_start(wa, G, C) == T0;
                for (int x = tid; x < rows * cols; x += WTHREADS) {
                    const int i = x % rows, c = x / rows;
                    double v = 0.0;
                    for (long long w = wa; w <= wb; ++w)
                        v += __ldcg(part + piece_slot(w, wa, wa_here) * (WT * WT) + i + WT * c);
                    emit(i, c, v);
                }
                if (tid == 0) *cnt = 0;
            }
            __syncthreads();
        }
#pragma unroll
        for (int k = 0; k < 32; ++k) acc[k] = 0;
        first_piece = false;
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
            it.w = H.V(b) - H.data.get();
            it.nin = B.n;
            it.ldw = B.n;
            it.in_off = B.col_off - R.col_off;
        } else {
            it.w = H.U(b) - H.data.get();
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
    long long c1 = 0;
    int rmax = 0;
    for (P1T& it : p1) {
        it.c0 = c1;
        c1 += it.nin;
        rmax = std::max(rmax, it.r);
    }
    // wide phase-1 tiles: the columns of the W's that share a source box
    // (one input slice), 64 to a tile
    std::vector<W1Tile> w1;
    if (row_tile > 32) {
        std::map<std::pair<long long, int>, std::vector<int>> groups;
        for (int i = 0; i < (int)p1.size(); ++i) groups[{p1[i].in_off, p1[i].nin}].push_back(i);
        for (auto& g : groups) {
            W1Tile cur{};
            cur.in_off = g.first.first;
            cur.nin = g.first.second;
            for (int i : g.second) {
                for (int j = 0; j < p1[i].r; ++j) {
                    if (cur.rows == kWideTile) {
                        w1.push_back(cur);
                        const long long io = cur.in_off;
                        const int ni = cur.nin;
                        cur = W1Tile{};
                        cur.in_off = io;
                        cur.nin = ni;
                    }
                    cur.wcol[cur.rows] = p1[i].w + (long long)j * p1[i].ldw;
                    cur.trel[cur.rows] = p1[i].t_rel;
                    cur.tj[cur.rows] = j;
                    cur.tr[cur.rows] = p1[i].r;
                    ++cur.rows;
                }
            }
            if (cur.rows > 0) w1.push_back(cur);
        }
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
    std::vector<int> zero;
    std::vector<int> ent_block;
    long long c2 = 0;
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
                    e.a = H.D(b) - H.data.get() + (cl.offset - B.row_off);
                    e.lda = B.m;
                    e.transA = 0;
                    e.inner = B.n;
                    e.b_off = B.col_off - R.col_off;
                } else {
                    e.a = H.D(b) - H.data.get() + (long long)(cl.offset - B.col_off) * B.m;
                    e.lda = B.m;
                    e.transA = 1;
                    e.inner = B.m;
                    e.b_off = B.row_off - R.row_off;
                }
                e.b_from_t = 0;
            } else {
                if (H.rank[b] == 0) continue;
                if (!trans) {
                    e.a = H.U(b) - H.data.get() + (cl.offset - B.row_off);
                    e.lda = B.m;
                } else {
                    e.a = H.V(b) - H.data.get() + (cl.offset - B.col_off);
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
            ent_block.push_back(b);
        }
        const int e1 = (int)ent.size();
        for (int r0 = 0; r0 < cl.count; r0 += row_tile) {
            P2T it{};
            it.out_off = cl.offset - outBase;
            it.r0 = r0;
            it.rows = std::min(row_tile, cl.count - r0);
            it.e0 = e0;
            it.e1 = e1;
            it.c0 = c2;
            it.width = cbeg;
            c2 += cbeg;
            if (cbeg == 0) zero.push_back((int)p2.size());
            p2.push_back(it);
        }
    }
    T->n1 = (int)p1.size();
    T->n2 = (int)p2.size();
    T->t_rows = t_rows;
    T->nz = (int)zero.size();
    T->c1 = c1;
    T->c2 = c2;
    T->rmax = rmax;
    T->p1.upload(p1, ctx.stream);
    T->p2.upload(p2, ctx.stream);
    T->ent.upload(ent, ctx.stream);
    T->zero_tiles.upload(zero, ctx.stream);
    T->hzero = zero;
    T->nw1 = (int)w1.size();
    T->w1.upload(w1, ctx.stream);
    if (row_tile > 32) {
        // chunk prefixes of the wide kernels (chunks of KC inner indices,
        // none spanning two entries)
        std::vector<int> w1cp(w1.size() + 1, 0), tcp(p2.size() + 1, 0), ekc(ent.size(), 0);
        for (size_t i = 0; i < w1.size(); ++i) w1cp[i + 1] = w1cp[i] + ceil_div(w1[i].nin, KC);
        for (size_t t = 0; t < p2.size(); ++t) {
            int k = 0;
            for (int e = p2[t].e0; e < p2[t].e1; ++e) {
                ekc[e] = k;
                k += ceil_div(ent[e].inner, KC);
            }
            tcp[t + 1] = tcp[t] + k;
        }
        T->wc1 = w1cp.back();
        T->wc2 = tcp.back();
        T->w1cp.upload(w1cp, ctx.stream);
        T->tcp.upload(tcp, ctx.stream);
        T->ekc.upload(ekc, ctx.stream);
    }
    T->hp1 = std::move(p1);
    T->hp2 = std::move(p2);
    T->hent = std::move(ent);
    T->hent_block = std::move(ent_block);
    return T;
}

}  // namespace

// The layout group of H in its context (created on first use).
LayoutGroup& layout_group(Context& ctx, const HMatrix& H) {
    if (H.group) return *H.group;
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ULL;
    };
    const Structure* S = H.S.get();
    mix(&S, sizeof(S));
    mix(&H.max_rank, sizeof(int));
    mix(H.rank.data(), H.rank.size() * sizeof(int));
    auto& L = ctx.layouts;
    for (size_t i = 0; i < L.size(); ++i) {
        LayoutGroup& g = *L[i];
        if (g.hash == h && g.S == S && g.max_rank == H.max_rank && g.rank == H.rank) {
            auto keep = L[i];
            L.erase(L.begin() + (long long)i);
            L.push_back(keep);
            H.group = keep;
            return *keep;
        }
    }
    auto g = std::make_shared<LayoutGroup>();
    g->S = S;
    g->max_rank = H.max_rank;
    g->rank = H.rank;
    g->hash = h;
    L.push_back(g);
    if (L.size() > kLayoutGroups) L.erase(L.begin());
    H.group = g;
    return *g;
}

std::shared_ptr<JobTemplate> get_template(Context& ctx, const HMatrix& H, int root, bool trans,
                                          int row_tile) {
    HMB_REQUIRE(row_tile >= 1 && row_tile <= 64, HM_ERR_INTERNAL, "row tile out of range");
    LayoutGroup& G = layout_group(ctx, H);
    auto key = std::make_tuple(root, trans ? 1 : 0, row_tile);
    auto it = G.templates.find(key);
    if (it != G.templates.end()) return it->second;
    auto T = build_template(ctx, H, root, trans, row_tile);
    HMB_REQUIRE((T->n1 == 0 || T->p1.get()) && (T->n2 == 0 || (T->p2.get() && T->ent.get())) &&
                    (T->nz == 0 || T->zero_tiles.get()) && (T->nw1 == 0 || T->w1.get()),
                HM_ERR_INTERNAL, "work lists missing on the device");
    G.templates.emplace(key, T);
    return T;
}

namespace {

// Resident CTAs of a persistent kernel of `threads` threads a CTA.
template <typename K>
int persistent_grid_n(const Context& ctx, K kernel, int threads, size_t smem = 0) {
    static std::mutex mu;
    static std::map<const void*, int> per_sm;
    std::lock_guard<std::mutex> lock(mu);
    int& n = per_sm[(const void*)kernel];
    if (n == 0) {
        HMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem));
        n = std::max(1, n);
    }
    return n * ctx.num_sms;
}

// Resident CTAs of a persistent kernel (occupancy x SMs), cached per kernel.
template <typename K>
int persistent_grid(const Context& ctx, K kernel) {
    static std::mutex mu;
    static std::map<const void*, int> per_sm;
    std::lock_guard<std::mutex> lock(mu);
    int& n = per_sm[(const void*)kernel];
    if (n == 0) {
        HMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, 0));
        n = std::max(1, n);
    }
    return n * ctx.num_sms;
}

// First item of every warp of the narrow phase-1 kernel for split width GW.
const int* warp_starts1(Context& ctx, JobTemplate& T, long long GW) {
    auto f = T.start1.find(GW);
    if (f != T.start1.end()) return f->second.get();
    std::vector<int> st((size_t)GW);
    int item = 0;
    for (long long w = 0; w < GW; ++w) {
        const long long g = w * T.c1 / GW;
        while (item + 1 < (int)T.hp1.size() && T.hp1[item + 1].c0 <= g) ++item;
        st[(size_t)w] = item;
    }
    DeviceBuffer<int>& d = T.start1[GW];
    d.upload(st, ctx.stream);
    return d.get();
}

// First (tile, entry) of every warp of the narrow phase-2 kernel.
const int2* warp_starts2(Context& ctx, JobTemplate& T, long long GW) {
    auto f = T.start2.find(GW);
    if (f != T.start2.end()) return f->second.get();
    std::vector<int2> st((size_t)GW);
    int tile = 0;
    for (long long w = 0; w < GW; ++w) {
        const long long g = w * T.c2 / GW;
        while (tile + 1 < (int)T.hp2.size() && T.hp2[tile + 1].c0 <= g) ++tile;
        const P2T& it = T.hp2[tile];
        int e = it.e0;
        while (e + 1 < it.e1 && T.hent[e + 1].cbeg <= g - it.c0) ++e;
        st[(size_t)w] = make_int2(tile, e);
    }
    DeviceBuffer<int2>& d = T.start2[GW];
    d.upload(st, ctx.stream);
    return d.get();
}

template <int NC>
void launch_narrow(Context& ctx, const JobExec* jobs_d, int nj, const JobExec& job0,
                   long long c1, long long c2, int rmax, JobTemplate* single) {
    cudaStream_t st = ctx.stream;
    if (c1 > 0) {
        const long long g = std::min<long long>(ceil_div(c1, kWarps),
                                                persistent_grid(ctx, p1_stream_kernel<NC>));
        const long long GW = std::min<long long>(g * kWarps, c1);
        const int* starts = single ? warp_starts1(ctx, *single, GW) : nullptr;
        DeviceBuffer<double> S;
        S.allocate((size_t)(2 * GW * rmax * NC), st);
        LaunchScope ls(ctx, "hmm_lowrank_inner");
        p1_stream_kernel<NC><<<(unsigned)g, kThreads, 0, st>>>(jobs_d, nj, job0, c1, GW, S.get(),
                                                               rmax, starts);
        HMB_CHECK_LAUNCH();
    }
    if (c2 > 0) {
        const long long g = std::min<long long>(ceil_div(c2, kWarps),
                                                persistent_grid(ctx, p2_stream_kernel<NC>));
        const long long GW = std::min<long long>(g * kWarps, c2);
        const int2* starts = single ? warp_starts2(ctx, *single, GW) : nullptr;
        DeviceBuffer<double> S;
        S.allocate((size_t)(2 * GW * 32 * NC), st);
        LaunchScope ls(ctx, "hmm_row_tiles");
        p2_stream_kernel<NC><<<(unsigned)g, kThreads, 0, st>>>(jobs_d, nj, job0, c2, GW, S.get(),
                                                               starts);
        HMB_CHECK_LAUNCH();
    }
}

// Inputs of TF32 products: X (n x k, ld ldx, FP64) -> Xf (n x k, ld n,
// FP32 rounded to TF32), one launch for all distinct inputs (blockIdx.y).
struct InConv {
    const double* src;
    float* dst;
    long long ld, n, total;
};

__global__ void in_tf32_kernel(const InConv* __restrict__ cv) {
    const InConv c = cv[blockIdx.y];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e % c.n, j = e / c.n;
        c.dst[e] = round_tf32(c.src[i + j * c.ld]);
    }
}

template <bool TF>
using WideElem = typename std::conditional<TF, float, double>::type;

template <bool TF>
void wide_grids(Context& ctx, long long c1, long long c2, int& G1, int& G2) {
    constexpr size_t smem = sizeof(WideSmemT<WideElem<TF>>);
    static std::once_flag attr_once;
    std::call_once(attr_once, [] {
        cudaFuncSetAttribute(wide_kernel<1, TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(wide_kernel<2, TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    G1 = (int)std::min<long long>(c1, persistent_grid_n(ctx, wide_kernel<1, TF>, WTHREADS, smem));
    G2 = (int)std::min<long long>(c2, persistent_grid_n(ctx, wide_kernel<2, TF>, WTHREADS, smem));
}

template <bool TF>
void launch_wide(Context& ctx, const JobExec* jobs_d, int nj, const JobExec& job0, long long n1,
                 long long n2, int G1, int G2, int ct) {
    constexpr size_t smem = sizeof(WideSmemT<WideElem<TF>>);
    cudaStream_t st = ctx.stream;
    if (n1 > 0 && G1 > 0) {
        LaunchScope ls(ctx, TF ? "hmm_lowrank_inner_tf32" : "hmm_lowrank_inner");
        wide_kernel<1, TF><<<dim3((unsigned)G1, (unsigned)ct), WTHREADS, smem, st>>>(jobs_d, nj, job0,
                                                                                    n1, G1);
        HMB_CHECK_LAUNCH();
    }
    if (n2 > 0 && G2 > 0) {
        LaunchScope ls(ctx, TF ? "hmm_row_tiles_tf32" : "hmm_row_tiles");
        wide_kernel<2, TF><<<dim3((unsigned)G2, (unsigned)ct), WTHREADS, smem, st>>>(jobs_d, nj, job0,
                                                                                    n2, G2);
        HMB_CHECK_LAUNCH();
    }
}

}  // namespace

int* Context::error_word() {
    if (!errword.get()) {
        errword.allocate(1, stream);
        HMB_CUDA(cudaMemsetAsync(errword.get(), 0, sizeof(int), stream));
    }
    return errword.get();
}

int* Context::numerical_word() {
    if (!numword.get()) {
        numword.allocate(1, stream);
        HMB_CUDA(cudaMemsetAsync(numword.get(), 0, sizeof(int), stream));
    }
    return numword.get();
}

void Context::check_numerical() {
    HMB_CUDA(cudaStreamSynchronize(stream));
    if (errword.get()) {
        int e = 0;
        HMB_CUDA(cudaMemcpy(&e, errword.get(), sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            HMB_CUDA(cudaMemset(errword.get(), 0, sizeof(int)));
            throw Error(HM_ERR_TIMEOUT, "a bounded device wait gave up (no progress)");
        }
    }
    if (!numword.get()) return;
    int h = 0;
    HMB_CUDA(cudaMemcpy(&h, numword.get(), sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        HMB_CUDA(cudaMemset(numword.get(), 0, sizeof(int)));
        throw Error(HM_ERR_NUMERICAL,
                    "a low-rank rounding met NaN or Inf (non-finite block data entered an "
                    "H*H product)");
    }
}

double* Context::pinned_scalar() {
    if (!pinned) HMB_CUDA(cudaMallocHost((void**)&pinned, sizeof(double)));
    return pinned;
}

double* Context::scratch(int slot, long long n) {
    DeviceBuffer<double>& b = scratch_bufs[slot];
    n = std::max<long long>(n, 2);
    if ((long long)b.size() < n) b.allocate((size_t)(n + n / 4), stream);
    return b.get();
}

int* Context::zeroed_counters(long long n) {
    if (n > counters_cap) {
        const long long cap = std::max<long long>(n, 2 * counters_cap);
        counters.allocate((size_t)cap, stream);
        HMB_CUDA(cudaMemsetAsync(counters.get(), 0, (size_t)cap * sizeof(int), stream));
        counters_cap = cap;
    }
    return counters.get();
}

namespace {

void run_jobs_direct(Context& ctx, const std::vector<MatJob>& jobs, bool tf32);

// The jobs in passes of at most 8 columns (the streaming kernels).
void run_jobs_split(Context& ctx, const std::vector<MatJob>& jobs, int kmax) {
    for (int c0 = 0; c0 < kmax; c0 += 8) {
        std::vector<MatJob> pass(jobs);
        for (MatJob& J : pass) {
            J.k = std::max(0, std::min(8, J.k - c0));
            if (J.k == 0) continue;
            J.in += (long long)c0 * J.ldin;
            J.out += (long long)c0 * J.ldout;
        }
        run_jobs_direct(ctx, pass, false);
    }
}

// Wide pass (1) or 8-column passes (2) for an FP64 job list of 9 to 16
// columns.  Which is faster depends on the operator: on the 256^2 operator
// (maxRank 32) two streaming passes are 27 % faster at 9 columns and 7 % at
// 12; on 32^2 the tensor-core pass is faster from 9 columns.  Timed once per
// (layout, job count, column count) on copies of the jobs writing into
// scratch with beta = 0 (one untimed and three timed runs of each).
int fp64_split_choice(Context& ctx, const std::vector<MatJob>& jobs, int kmax) {
    if (ctx.fp64_split != 0) return ctx.fp64_split;
    get_template(ctx, *jobs[0].H, jobs[0].root, jobs[0].trans, 64);   // makes the layout group
    const auto key = std::make_tuple(jobs[0].H->group->hash, (int)jobs.size(), kmax);
    auto f = ctx.fp64_split_tuned.find(key);
    if (f != ctx.fp64_split_tuned.end()) return f->second;
    HostScope hs(ctx, "fp64_split_autotune");
    std::vector<MatJob> trial(jobs);
    long long total = 0;
    std::vector<long long> off(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
        const Block& R = jobs[j].H->S->blocks[jobs[j].root];
        const int nout = jobs[j].trans ? R.n : R.m;
        off[j] = total;
        total += (long long)std::max(nout, 1) * std::max(jobs[j].k, 0);
    }
    DeviceBuffer<double> scratch;
    scratch.allocate((size_t)std::max<long long>(total, 1), ctx.stream);
    for (size_t j = 0; j < jobs.size(); ++j) {
        const Block& R = jobs[j].H->S->blocks[jobs[j].root];
        trial[j].out = scratch.get() + off[j];
        trial[j].ldout = std::max(jobs[j].trans ? R.n : R.m, 1);
        trial[j].beta = 0.0;
    }
    cudaEvent_t e0, e1;
    HMB_CUDA(cudaEventCreate(&e0));
    HMB_CUDA(cudaEventCreate(&e1));
    float ms[2] = {0.0f, 0.0f};
    for (int which = 1; which <= 2; ++which) {
        auto run = [&] {
            if (which == 1) run_jobs_direct(ctx, trial, false);
            else run_jobs_split(ctx, trial, kmax);
        };
        run();
        HMB_CUDA(cudaEventRecord(e0, ctx.stream));
        for (int r = 0; r < 3; ++r) run();
        HMB_CUDA(cudaEventRecord(e1, ctx.stream));
        HMB_CUDA(cudaEventSynchronize(e1));
        HMB_CUDA(cudaEventElapsedTime(&ms[which - 1], e0, e1));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int best = ms[1] < ms[0] ? 2 : 1;
    ctx.fp64_split_tuned[key] = best;
    return best;
}

}  // namespace

int fp64_split_for(Context& ctx, const std::vector<MatJob>& jobs) {
    int kmax = 0;
    for (const MatJob& J : jobs) kmax = std::max(kmax, J.k);
    if (jobs.empty() || kmax <= 8 || kmax > 16) return kmax > 8 ? 1 : 2;
    return fp64_split_choice(ctx, jobs, kmax);
}

void run_jobs(Context& ctx, const std::vector<MatJob>& jobs, bool tf32) {
    if (jobs.empty()) return;
    if (!tf32) {
        int kmax = 0;
        for (const MatJob& J : jobs) kmax = std::max(kmax, J.k);
        if (kmax > 8 && kmax <= 16 && fp64_split_choice(ctx, jobs, kmax) == 2) {
            run_jobs_split(ctx, jobs, kmax);
            return;
        }
    }
    run_jobs_direct(ctx, jobs, tf32);
}

namespace {

void run_jobs_direct(Context& ctx, const std::vector<MatJob>& jobs, bool tf32) {
    if (jobs.empty()) return;
    cudaStream_t st = ctx.stream;
    std::vector<std::shared_ptr<JobTemplate>> tmpl;
    tmpl.reserve(jobs.size());
    int kmax = 0;
    for (const MatJob& J : jobs) {
        HMB_REQUIRE(J.k >= 0, HM_ERR_ARGUMENT, "negative column count");
        kmax = std::max(kmax, J.k);
    }
    // one vector, one job: stream the blocks (matvec.cu)
    if (!tf32 && jobs.size() == 1 && jobs[0].k == 1 && multiply_vector_streamed(ctx, jobs[0])) return;
    // few columns: 32-row tiles, work split evenly over all resident warps;
    // many columns: 64 x 64 tiles on the tensor cores (FP64, or TF32 when asked)
    const bool wide = kmax > 8;
    tf32 = tf32 && wide;
    const int row_tile = wide ? 64 : 32;
    for (const MatJob& J : jobs) tmpl.push_back(get_template(ctx, *J.H, J.root, J.trans, row_tile));
    const int ct = ceil_div(std::max(kmax, 1), kWideTile);   // wide column tiles
    long long t_total = 0, c_total = 0;
    std::vector<long long> t_off(jobs.size()), c1_off(jobs.size()), c2_off(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
        const JobTemplate& T = *tmpl[j];
        t_off[j] = t_total;
        t_total += T.t_rows * jobs[j].k;
        c1_off[j] = c_total;
        c_total += wide ? (long long)T.nw1 * ct : T.n1;
        c2_off[j] = c_total;
        c_total += wide ? (long long)T.n2 * ct : T.n2;
    }
    // wide: persistent grids, 2 partial slots of 64 x 64 per CTA and column tile
    int G1 = 0, G2 = 0;
    long long p_total = 0;
    if (wide) {
        long long c1 = 0, c2 = 0;
        for (size_t j = 0; j < jobs.size(); ++j)
            if (jobs[j].k > 0) {
                c1 += tmpl[j]->wc1;
                c2 += tmpl[j]->wc2;
            }
        if (tf32) wide_grids<true>(ctx, c1, c2, G1, G2);
        else wide_grids<false>(ctx, c1, c2, G1, G2);
        p_total = 2LL * std::max(G1, G2) * ct * kWideTile * kWideTile;
    }
    // TF32: the blocks' FP32 copies, the inputs rounded once (inputs shared
    // by several jobs converted once), an FP32 intermediate
    DeviceBuffer<double> tbuf;
    DeviceBuffer<float> tbuf32, inbuf32;
    std::vector<const float*> in32(jobs.size(), nullptr);
    std::vector<int> ldin32(jobs.size(), 0);
    if (tf32) {
        std::map<std::tuple<const double*, int, int, int>, long long> seen;
        std::vector<InConv> conv;
        std::vector<long long> conv_job(jobs.size(), -1), conv_off;
        long long in_total = 0, maxconv = 0;
        for (size_t j = 0; j < jobs.size(); ++j) {
            const MatJob& J = jobs[j];
            if (J.k == 0) continue;
            ensure_tf32_copy(ctx, const_cast<HMatrix&>(*J.H));
            const Block& R = J.H->S->blocks[J.root];
            const int nin = J.trans ? R.m : R.n;
            auto key = std::make_tuple(J.in, J.ldin, nin, J.k);
            auto f = seen.find(key);
            if (f == seen.end()) {
                InConv c{};
                c.src = J.in;
                c.ld = J.ldin;
                c.n = std::max(nin, 1);
                c.total = (long long)nin * J.k;
                f = seen.emplace(key, (long long)conv.size()).first;
                conv.push_back(c);
                conv_off.push_back(in_total);
                in_total += std::max<long long>(c.total, 1);
                maxconv = std::max(maxconv, c.total);
            }
            conv_job[j] = f->second;
            ldin32[j] = std::max(nin, 1);
        }
        inbuf32.allocate((size_t)std::max<long long>(in_total, 1), st);
        tbuf32.allocate((size_t)std::max<long long>(t_total, 1), st);
        for (size_t c = 0; c < conv.size(); ++c) conv[c].dst = inbuf32.get() + conv_off[c];
        for (size_t j = 0; j < jobs.size(); ++j)
            if (conv_job[j] >= 0) in32[j] = conv[(size_t)conv_job[j]].dst;
        HMB_REQUIRE(conv.size() < 65536, HM_ERR_UNSUPPORTED, "too many distinct inputs");
        if (!conv.empty() && maxconv > 0) {
            DeviceBuffer<InConv> dconv;
            dconv.upload(conv, st);
            const long long gx = std::min<long long>(ceil_div(maxconv, 256LL), 2LL * ctx.num_sms);
            LaunchScope ls(ctx, "input_tf32");
            in_tf32_kernel<<<dim3((unsigned)gx, (unsigned)conv.size()), 256, 0, st>>>(dconv.get());
            HMB_CHECK_LAUNCH();
        }
    }
    tbuf.allocate((size_t)std::max<long long>((tf32 ? 0 : t_total) + p_total, 1), st);
    int* cnt = ctx.zeroed_counters(std::max<long long>(c_total, 1));
    std::vector<JobExec> ex;
    ex.reserve(jobs.size());
    long long n1 = 0, n2 = 0;
    int rmax = 0;
    size_t first_job = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const MatJob& J = jobs[j];
        if (J.k == 0) continue;
        if (ex.empty()) first_job = j;
        const JobTemplate& T = *tmpl[j];
        JobExec e{};
        e.hb = J.H->data.get();
        e.p1 = T.p1.get();
        e.w1 = T.w1.get();
        e.p2 = T.p2.get();
        e.ent = T.ent.get();
        e.in = J.in;
        e.out = J.out;
        if (tf32) {
            e.hb32 = J.H->data32.get();
            e.in32 = in32[j];
            e.ldin32 = ldin32[j];
            e.T32 = tbuf32.get() + t_off[j];
            e.part = tbuf.get();
        } else {
            e.T = tbuf.get() + t_off[j];
            e.part = tbuf.get() + t_total;
        }
        e.w1cp = T.w1cp.get();
        e.tcp = T.tcp.get();
        e.ekc = T.ekc.get();
        e.cnt1 = cnt + c1_off[j];
        e.cnt2 = cnt + c2_off[j];
        e.alpha_scale = J.alpha_scale;
        e.alpha = J.alpha;
        e.beta = J.beta;
        e.ldin = J.ldin;
        e.ldout = J.ldout;
        e.k = J.k;
        e.n1 = wide ? T.nw1 : T.n1;
        e.n2 = T.n2;
        e.ct1 = 1;
        e.ct2 = 1;
        e.p1_begin = n1;
        e.p2_begin = n2;
        n1 += wide ? T.wc1 : T.c1;
        n2 += wide ? T.wc2 : T.c2;
        rmax = std::max(rmax, T.rmax);
        ex.push_back(e);
    }
    if (ex.empty()) return;
    DeviceBuffer<JobExec> dex;
    const JobExec* jobs_d = nullptr;
    if (ex.size() > 1) {
        dex.upload(ex, st);
        jobs_d = dex.get();
    }
    const JobExec job0 = ex[0];
    const int nj = (int)ex.size();
    if (!wide) {
        JobTemplate* single = nj == 1 ? tmpl[first_job].get() : nullptr;
        if (kmax <= 1) launch_narrow<1>(ctx, jobs_d, nj, job0, n1, n2, rmax, single);
        else if (kmax <= 4) launch_narrow<4>(ctx, jobs_d, nj, job0, n1, n2, rmax, single);
        else launch_narrow<8>(ctx, jobs_d, nj, job0, n1, n2, rmax, single);
        launch_zero_tiles(ctx, tmpl, jobs, jobs_d, job0);
        return;
    }
    HMB_REQUIRE(ct < 65536, HM_ERR_UNSUPPORTED, "too many columns");
    if (tf32) launch_wide<true>(ctx, jobs_d, nj, job0, n1, n2, G1, G2, ct);
    else launch_wide<false>(ctx, jobs_d, nj, job0, n1, n2, G1, G2, ct);
    // row tiles without entries: output = beta * output
    launch_zero_tiles(ctx, tmpl, jobs, jobs_d, job0);
}

}  // namespace

}  // namespace hmb
