// One-vector H-matrix products (H x, H^T x) streamed block by block.
//
// Same result as the reference's recursive HMat2d::Multiply /
// TransposeMultiply for a Vector (src/HMat2d/MultiplyVector-incl.hpp:12-124;
// a gemv per dense leaf, src/hmat_tools/MultiplyVector.cpp:14-69, and two per
// low-rank block, :71-128), organised for HBM: every block's storage is read
// as one contiguous stream by one warp, because the DRAM delivers full
// bandwidth only for contiguous runs of about 2 KB or more.
//
//   kernel 1 (persistent warps, dynamic queue of units):
//     low-rank block  -> t = W^T x (warp reduction), y_b = A t   (W, A = V, U or U, V)
//     dense leaf      -> y_b = D x      (or D^T x for the transpose)
//     large low-rank  -> slabs of <= 512 rows: t-slabs write partial t and
//                        count themselves; y-slabs wait for the count, add the
//                        partials in slab order and form their rows of A t
//     every y_b is a block-private partial (kept in L2), so no atomics on y.
//   kernel 2: y_tile = alpha * (sum over the blocks covering the tile of their
//     partial rows, in a fixed order) + beta * y_tile.
// Deterministic: each partial is formed by exactly one warp in a fixed order.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

#include "engine.h"
#include "templates.h"

namespace hmb {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxRows = 512;   // rows (or input rows) of one warp unit
constexpr int kMaxRank = 128;   // larger ranks use the general kernels
constexpr int kWaitLimit = 1 << 24;

enum : int { MU_LR = 0, MU_DENSE = 1, MU_DENSE_T = 2, MU_TSLAB = 3, MU_YSLAB = 4 };

// One warp's unit of work.
//  MU_LR:      t = M1^T x[in_off..] (M1: rows_in x r, ld ld1), y = M2 t (M2: rows_out x r, ld ld2)
//  MU_DENSE:   y = M1 x[in_off..]   (M1: rows_out x r, ld ld1)
//  MU_DENSE_T: y[j] = M1(:, j)^T x[in_off..] for j < r (M1: rows_in x r, ld ld1)
//  MU_TSLAB:   tpart[slab] = M1^T x[in_off..] (M1: rows_in x r)
//  MU_YSLAB:   y = M2 (sum of the big block's tparts) (M2: rows_out x r)
// y is the partial buffer at y_off.
struct MvUnit {
    long long m1, m2;   // element offsets of M1, M2 in the matrix storage
    long long in_off, y_off;
    int kind, rows_in, rows_out, r;
    int ld1, ld2, big, slab;
};

// A low-rank block too large for one warp: its t-slabs and partial t's.
struct MvBig {
    long long t_off;   // tparts at t_off + slab * r
    int nslab, r;
};

}  // namespace

struct MvPlan {
    DeviceBuffer<MvUnit> units;
    DeviceBuffer<MvBig> big;
    DeviceBuffer<long long> ent_off;   // per P2 entry: partial offset of the tile's first row
    DeviceBuffer<double> scratch;      // partials, then the big blocks' partial t
    int nunits = 0, nbig = 0;
    long long partial_len = 0, tpart_len = 0;
};

namespace {

// L2 policies: the streamed matrices are read once (evict first); the
// partials are read again by the combine (evict last).
__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_stream(const double* p, unsigned long long pol) {
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_keep(double* p, double v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

// gpu-scope release / acquire on the big blocks' counters (a __syncwarp
// before the release makes the whole warp's stores visible with it; one after
// the acquire extends it to the whole warp).
__device__ __forceinline__ void red_add_release(int* p, int v) {
    asm volatile("red.add.release.gpu.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void warp_sum16(double (&v)[16], int lane) {
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

// Column dots of a 16-column chunk: v[f] (summed over the warp afterwards)
// gets lane's share of sum_i M(i, j0+f) x_i.  A lane owns rows lane + 32 rb;
// one step loads CPS = 16/RB whole columns (RB row blocks each), so the warp
// reads contiguous runs of the column-major M.
template <int RB>
__device__ __forceinline__ void cd_chunk(const double* __restrict__ M, int ld, int R, int C, int j0,
                                         const double (&xr)[RB], int lane, double (&v)[16],
                                         unsigned long long pol) {
    constexpr int CPS = 16 / RB;
#pragma unroll
    for (int f = 0; f < 16; ++f) v[f] = 0.0;
#pragma unroll 1
    for (int s = 0; s < RB; ++s) {
        const int jb = j0 + s * CPS;
        if (jb >= C) break;
        double val[CPS][RB];
#pragma unroll
        for (int cc = 0; cc < CPS; ++cc)
#pragma unroll
            for (int rb = 0; rb < RB; ++rb) {
                const int i = lane + 32 * rb, j = jb + cc;
                val[cc][rb] = (j < C && i < R) ? ld_stream(M + i + (long long)j * ld, pol) : 0.0;
            }
        double sum[CPS];
#pragma unroll
        for (int cc = 0; cc < CPS; ++cc) {
            sum[cc] = 0.0;
#pragma unroll
            for (int rb = 0; rb < RB; ++rb) sum[cc] = fma(val[cc][rb], xr[rb], sum[cc]);
        }
#pragma unroll
        for (int ss = 0; ss < RB; ++ss)
            if (ss == s)
#pragma unroll
                for (int cc = 0; cc < CPS; ++cc) v[ss * CPS + cc] = sum[cc];
    }
}

// Row combinations: lane's rows lane + 32 rb of y = M t (M: R x C, ld ld).
// One step loads CPS = 16/RB whole columns.
template <int RB, bool TGLOBAL>
__device__ __forceinline__ void rc_rows(const double* __restrict__ M, int ld, int R, int C,
                                        const double* t, int lane, double (&acc)[RB],
                                        unsigned long long pol) {
    constexpr int CPS = 16 / RB;
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) acc[rb] = 0.0;
#pragma unroll 1
    for (int j0 = 0; j0 < C; j0 += CPS) {
        double val[CPS][RB], tv[CPS];
#pragma unroll
        for (int cc = 0; cc < CPS; ++cc) {
            const int j = j0 + cc;
            tv[cc] = j < C ? (TGLOBAL ? __ldg(t + j) : t[j]) : 0.0;
#pragma unroll
            for (int rb = 0; rb < RB; ++rb) {
                const int i = lane + 32 * rb;
                val[cc][rb] = (j < C && i < R) ? ld_stream(M + i + (long long)j * ld, pol) : 0.0;
            }
        }
#pragma unroll
        for (int cc = 0; cc < CPS; ++cc)
#pragma unroll
            for (int rb = 0; rb < RB; ++rb) acc[rb] = fma(val[cc][rb], tv[cc], acc[rb]);
    }
}

// out[j] = sum_i M(i, j) x_i for j < C (lanes 2f write out[j0 + f]).
template <int RB>
__device__ void column_dots(const double* __restrict__ M, int ld, int R, int C,
                            const double* __restrict__ x, double* out, int lane,
                            unsigned long long pol) {
    double xr[RB];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
        const int i = lane + 32 * rb;
        xr[rb] = i < R ? __ldg(x + i) : 0.0;
    }
    for (int j0 = 0; j0 < C; j0 += 16) {
        double v[16];
        cd_chunk<RB>(M, ld, R, C, j0, xr, lane, v, pol);
        warp_sum16(v, lane);
        const int f = lane >> 1;
        if ((lane & 1) == 0 && j0 + f < C) out[j0 + f] = v[0];
    }
}

template <int RB, bool TGLOBAL>
__device__ void row_combos(const double* __restrict__ M, int ld, int R, int C, const double* t,
                           double* __restrict__ y, int lane, unsigned long long pol,
                           unsigned long long keep) {
    double acc[RB];
    rc_rows<RB, TGLOBAL>(M, ld, R, C, t, lane, acc, pol);
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
        const int i = lane + 32 * rb;
        if (i < R) st_keep(y + i, acc[rb], keep);
    }
}

__device__ __forceinline__ int row_blocks(int R) {
    const int n = (R + 31) >> 5;
    return n <= 1 ? 1 : n <= 2 ? 2 : n <= 4 ? 4 : n <= 8 ? 8 : 16;
}

__device__ void dispatch_cd(const double* M, int ld, int R, int C, const double* x, double* out,
                            int lane, unsigned long long pol) {
    switch (row_blocks(R)) {
        case 1: column_dots<1>(M, ld, R, C, x, out, lane, pol); break;
        case 2: column_dots<2>(M, ld, R, C, x, out, lane, pol); break;
        case 4: column_dots<4>(M, ld, R, C, x, out, lane, pol); break;
        case 8: column_dots<8>(M, ld, R, C, x, out, lane, pol); break;
        default: column_dots<16>(M, ld, R, C, x, out, lane, pol); break;
    }
}

template <bool TGLOBAL>
__device__ void dispatch_rc(const double* M, int ld, int R, int C, const double* t, double* y,
                            int lane, unsigned long long pol, unsigned long long keep) {
    switch (row_blocks(R)) {
        case 1: row_combos<1, TGLOBAL>(M, ld, R, C, t, y, lane, pol, keep); break;
        case 2: row_combos<2, TGLOBAL>(M, ld, R, C, t, y, lane, pol, keep); break;
        case 4: row_combos<4, TGLOBAL>(M, ld, R, C, t, y, lane, pol, keep); break;
        case 8: row_combos<8, TGLOBAL>(M, ld, R, C, t, y, lane, pol, keep); break;
        default: row_combos<16, TGLOBAL>(M, ld, R, C, t, y, lane, pol, keep); break;
    }
}

struct MvArgs {
    const double* hb;  // matrix storage
    const MvUnit* units;
    const MvBig* big;
    const double* x;
    double* part;      // block partials
    double* tpart;     // partial t of the big blocks
    int* queue;        // next unit; then warps finished (both zero at launch)
    int* done;         // per big block: t-slabs finished (zero at launch)
    int* err;          // set when a wait gave up
    int nunits, nbig, nwarps;
};

__global__ void __launch_bounds__(kThreads, 2) mv_blocks_kernel(const MvArgs a) {
    __shared__ double ts[kWarps][kMaxRank];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* t = ts[warp];
    // the combine kernel may be scheduled now; it waits for this grid's end
    asm volatile("griddepcontrol.launch_dependents;");
    const unsigned long long pol = policy_evict_first(), keep = policy_evict_last();
    int u = 0;
    if (lane == 0) u = atomicAdd(a.queue, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    while (u < a.nunits) {
        // take the next unit now so that the queue's latency overlaps this one
        int un_next = 0;
        if (lane == 0) un_next = atomicAdd(a.queue, 1);
        un_next = __shfl_sync(0xffffffffu, un_next, 0);
        if (un_next < a.nunits && lane == 0)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(a.units + un_next));
        const MvUnit un = a.units[u];
        const double* M1 = a.hb + un.m1;
        const double* M2 = a.hb + un.m2;
        const double* x = a.x + un.in_off;
        double* y = a.part + un.y_off;
        switch (un.kind) {
            case MU_LR:
                dispatch_cd(M1, un.ld1, un.rows_in, un.r, x, t, lane, pol);
                __syncwarp();
                dispatch_rc<false>(M2, un.ld2, un.rows_out, un.r, t, y, lane, pol, keep);
                __syncwarp();
                break;
            case MU_DENSE:
                dispatch_rc<true>(M1, un.ld1, un.rows_out, un.r, x, y, lane, pol, keep);
                break;
            case MU_DENSE_T:
                dispatch_cd(M1, un.ld1, un.rows_in, un.r, x, y, lane, pol);
                break;
            case MU_TSLAB: {
                const MvBig B = a.big[un.big];
                dispatch_cd(M1, un.ld1, un.rows_in, un.r, x, a.tpart + B.t_off + (long long)un.slab * B.r,
                            lane, pol);
                __syncwarp();
                if (lane == 0) red_add_release(a.done + un.big, 1);
                break;
            }
            default: {   // MU_YSLAB
                const MvBig B = a.big[un.big];
                int ok = 1;
                if (lane == 0) {
                    int it = 0;
                    while (ld_acquire(a.done + un.big) < B.nslab && ++it < kWaitLimit) __nanosleep(64);
                    ok = ld_acquire(a.done + un.big) >= B.nslab;
                    if (!ok) atomicExch(a.err, 1);
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                if (!ok) break;
                for (int j = lane; j < B.r; j += 32) {
                    double s = 0.0;
                    for (int q = 0; q < B.nslab; ++q) s += __ldcg(a.tpart + B.t_off + (long long)q * B.r + j);
                    t[j] = s;
                }
                __syncwarp();
                dispatch_rc<false>(M2, un.ld2, un.rows_out, un.r, t, y, lane, pol, keep);
                __syncwarp();
                break;
            }
        }
        u = un_next;
    }
    // the last warp out rearms the queue and the big-block counters
    if (lane == 0 && atomicAdd(a.queue + 1, 1) == a.nwarps - 1) {
        *a.queue = 0;
        a.queue[1] = 0;
        for (int i = 0; i < a.nbig; ++i) a.done[i] = 0;
    }
}

struct CombArgs {
    const P2T* tiles;
    const long long* ent_off;
    const double* part;
    double* out;
    const double* alpha_scale;
    double alpha, beta;
    int ntiles;
};

// y_tile = alpha * sum_e partial_e(tile rows) + beta * y_tile, one CTA per
// row tile: warp w adds entries e0 + w, e0 + w + 8, ..., then warp 0 adds
// the eight warp sums in order.  Launched as a
// programmatic dependent of the blocks kernel: it waits for that grid here.
__global__ void __launch_bounds__(kThreads) mv_combine_kernel(const CombArgs a) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ double red[kWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile = blockIdx.x;
    if (tile >= a.ntiles) return;
    const P2T it = a.tiles[tile];
    const bool ok = lane < it.rows;
    const double* base = a.part + it.r0 + (ok ? lane : 0);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    // warp w takes entries e0 + w + 8q; lane q fetches the q-th offset, then
    // the warp issues all of its partial loads back to back
    for (int eb = it.e0 + warp; eb < it.e1; eb += 32 * kWarps) {
        const int mine = eb + kWarps * lane;
        const long long off = mine < it.e1 ? a.ent_off[mine] : -1;
        const int nq = min(32, (it.e1 - eb + kWarps - 1) / kWarps);
        int q = 0;
        for (; q + 3 < nq; q += 4) {
            s0 += __ldcg(base + __shfl_sync(0xffffffffu, off, q));
            s1 += __ldcg(base + __shfl_sync(0xffffffffu, off, q + 1));
            s2 += __ldcg(base + __shfl_sync(0xffffffffu, off, q + 2));
            s3 += __ldcg(base + __shfl_sync(0xffffffffu, off, q + 3));
        }
        for (; q < nq; ++q) s0 += __ldcg(base + __shfl_sync(0xffffffffu, off, q));
    }
    red[warp][lane] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    if (warp != 0 || !ok) return;
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) v += red[w][lane];
    double* yp = a.out + it.out_off + it.r0 + lane;
    const double al = a.alpha_scale ? a.alpha * *a.alpha_scale : a.alpha;
    *yp = a.beta == 0.0 ? al * v : al * v + a.beta * *yp;
}

std::shared_ptr<MvPlan> build_plan(Context& ctx, const HMatrix& H, int root, bool trans,
                                   const JobTemplate& T) {
    HostScope hs(ctx, "hmv_plan");
    const Structure& S = *H.S;
    const Block& R = S.blocks[root];
    // output rows (relative to the root) -> row tile of the template
    const int nrows = trans ? R.n : R.m;
    std::vector<int> tile_at(nrows, -1);
    for (int t = 0; t < (int)T.hp2.size(); ++t) {
        const P2T& it = T.hp2[t];
        for (int i = 0; i < it.rows; ++i) tile_at[it.out_off + it.r0 + i] = t;
    }
    for (int v : tile_at)
        if (v < 0) return nullptr;
    // [o0, o1) must be a union of whole tiles
    auto tiles_of = [&](long long o0, long long o1, int& t0, int& nt) {
        t0 = tile_at[o0];
        const int t1 = tile_at[o1 - 1];
        const P2T& a = T.hp2[t0];
        const P2T& b = T.hp2[t1];
        nt = t1 - t0 + 1;
        return a.out_off + a.r0 == o0 && b.out_off + b.r0 + b.rows == o1;
    };
    // pieces of [o0, o0 + n) made of whole tiles, at most kMaxRows rows each
    auto pieces = [&](long long o0, int n, std::vector<std::pair<int, int>>& out) {
        out.clear();
        int a = 0;
        while (a < n) {
            int b = a;
            while (b < n) {
                const P2T& it = T.hp2[tile_at[o0 + b]];
                const int tend = (int)(it.out_off + it.r0 + it.rows - o0);
                if (tend - a > kMaxRows && b > a) break;
                b = tend;
            }
            if (b - a > kMaxRows || b > n) return false;
            out.push_back({a, b});
            a = b;
        }
        return true;
    };
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
    auto P = std::make_shared<MvPlan>();
    std::vector<MvUnit> first, rest;
    std::vector<MvBig> bigs;
    std::map<int, long long> yoff;   // block -> partial offset of its first output row
    std::vector<std::pair<int, int>> pcs;
    long long part = 0, tpart = 0;
    auto cover = [&](long long o0, long long o1) {
        int t0, nt;
        return tiles_of(o0, o1, t0, nt);
    };
    for (int b : leaves) {
        const Block& B = S.blocks[b];
        const int nout = trans ? B.n : B.m;
        const int nin = trans ? B.m : B.n;
        const long long in_off = trans ? B.row_off - R.row_off : B.col_off - R.col_off;
        const long long out0 = trans ? B.col_off - R.col_off : B.row_off - R.row_off;
        if (B.kind == KIND_DENSE) {
            if (nout > kMaxRows || (trans && nin > kMaxRows)) return nullptr;
            yoff[b] = part;
            MvUnit u{};
            u.kind = trans ? MU_DENSE_T : MU_DENSE;
            u.m1 = H.D(b) - H.data.get();
            u.ld1 = B.m;
            if (!trans) {
                u.rows_out = nout;
                u.r = nin;
            } else {
                u.rows_in = nin;
                u.r = nout;
            }
            u.in_off = in_off;
            u.y_off = part;
            if (!cover(out0, out0 + nout)) return nullptr;
            rest.push_back(u);
            part += nout;
            continue;
        }
        const int r = H.rank[b];
        if (r == 0) continue;
        if (r > kMaxRank) return nullptr;
        const long long W = (trans ? H.U(b) : H.V(b)) - H.data.get();
        const long long A = (trans ? H.V(b) : H.U(b)) - H.data.get();
        yoff[b] = part;
        if (nin <= kMaxRows && nout <= kMaxRows) {
            MvUnit u{};
            u.kind = MU_LR;
            u.m1 = W;
            u.ld1 = nin;
            u.m2 = A;
            u.ld2 = nout;
            u.rows_in = nin;
            u.rows_out = nout;
            u.r = r;
            u.in_off = in_off;
            u.y_off = part;
            if (!cover(out0, out0 + nout)) return nullptr;
            rest.push_back(u);
        } else {
            MvBig g{};
            g.t_off = tpart;
            g.nslab = (nin + kMaxRows - 1) / kMaxRows;
            g.r = r;
            tpart += (long long)g.nslab * r;
            const int bi = (int)bigs.size();
            bigs.push_back(g);
            for (int sl = 0; sl < g.nslab; ++sl) {
                MvUnit u{};
                u.kind = MU_TSLAB;
                u.m1 = W + (long long)sl * kMaxRows;
                u.ld1 = nin;
                u.rows_in = std::min(kMaxRows, nin - sl * kMaxRows);
                u.r = r;
                u.in_off = in_off + (long long)sl * kMaxRows;
                u.big = bi;
                u.slab = sl;
                first.push_back(u);
            }
            if (!pieces(out0, nout, pcs)) return nullptr;
            for (auto [a0, a1] : pcs) {
                MvUnit u{};
                u.kind = MU_YSLAB;
                u.m2 = A + a0;
                u.ld2 = nout;
                u.rows_out = a1 - a0;
                u.r = r;
                u.y_off = part + a0;
                u.big = bi;
                if (!cover(out0 + a0, out0 + a1)) return nullptr;
                rest.push_back(u);
            }
        }
        part += nout;
    }
    // larger units first (shorter tail); the y-slabs of the big blocks last,
    // so that their t-slabs (first in the queue) are done when they start
    std::stable_sort(rest.begin(), rest.end(), [](const MvUnit& x, const MvUnit& y) {
        const int kx = x.kind == MU_YSLAB, ky = y.kind == MU_YSLAB;
        if (kx != ky) return kx < ky;
        auto bytes = [](const MvUnit& u) { return (long long)(u.rows_in + u.rows_out) * u.r; };
        return bytes(x) > bytes(y);
    });
    std::vector<MvUnit> units;
    units.reserve(first.size() + rest.size());
    units.insert(units.end(), first.begin(), first.end());
    units.insert(units.end(), rest.begin(), rest.end());
    // entry e's partial offset is that of its cluster's first row
    std::vector<long long> eo(T.hent.size(), 0);
    for (const P2T& it : T.hp2) {
        for (int e = it.e0; e < it.e1; ++e) {
            const int b = T.hent_block[e];
            const Block& B = S.blocks[b];
            const long long out_row0 = trans ? B.col_off - R.col_off : B.row_off - R.row_off;
            eo[e] = yoff.at(b) + (it.out_off - out_row0);
        }
    }
    P->units.upload(units, ctx.stream);
    P->big.upload(bigs, ctx.stream);
    P->ent_off.upload(eo, ctx.stream);
    P->scratch.allocate((size_t)std::max<long long>(part + tpart, 1), ctx.stream);
    P->nunits = (int)units.size();
    P->nbig = (int)bigs.size();
    P->partial_len = part;
    P->tpart_len = tpart;
    return P;
}

}  // namespace

bool multiply_vector_streamed(Context& ctx, const MatJob& J) {
    if (J.k != 1) return false;
    auto T = get_template(ctx, *J.H, J.root, J.trans, 32);
    if (!T->mv_tried) {
        T->mv_tried = true;
        T->mv = build_plan(ctx, *J.H, J.root, J.trans, *T);
    }
    if (!T->mv) return false;
    MvPlan& P = *T->mv;
    if (P.nunits == 0) return false;
    cudaStream_t st = ctx.stream;
    int* cnt = ctx.zeroed_counters(2 + P.nbig);
    static std::once_flag once;
    static int per_sm = 0;
    std::call_once(once, [] {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mv_blocks_kernel, kThreads, 0);
        per_sm = std::max(1, per_sm);
    });
    const int g = std::max(1, std::min(per_sm * ctx.num_sms, (P.nunits + kWarps - 1) / kWarps));
    MvArgs a{};
    a.hb = J.H->data.get();
    a.units = P.units.get();
    a.big = P.big.get();
    a.x = J.in;
    a.part = P.scratch.get();
    a.tpart = P.scratch.get() + P.partial_len;
    a.queue = cnt;
    a.done = cnt + 2;
    a.err = ctx.error_word();
    a.nunits = P.nunits;
    a.nbig = P.nbig;
    a.nwarps = g * kWarps;
    {
        LaunchScope ls(ctx, "hmv_blocks");
        mv_blocks_kernel<<<g, kThreads, 0, st>>>(a);
        HMB_CHECK_LAUNCH();
    }
    CombArgs c{};
    c.tiles = T->p2.get();
    c.ent_off = P.ent_off.get();
    c.part = P.scratch.get();
    c.out = J.out;
    c.alpha_scale = J.alpha_scale;
    c.alpha = J.alpha;
    c.beta = J.beta;
    c.ntiles = T->n2;
    {
        LaunchScope ls(ctx, "hmv_combine");
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)std::max(1, T->n2));
        cfg.blockDim = dim3(kThreads);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = ctx.profiling ? 0 : 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        HMB_CUDA(cudaLaunchKernelEx(&cfg, mv_combine_kernel, c));
    }
    return true;
}

}  // namespace hmb
