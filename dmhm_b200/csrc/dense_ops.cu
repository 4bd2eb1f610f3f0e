// Batched small dense products for the leaf algebra of the H*H product:
// C = alpha op(A) op(B) + beta C, one CTA per product, 64 x 64 output tiles.
//
// These replace the reference's per-leaf BLAS calls in the dense and
// low-rank leaf products (src/hmat_tools/MultiplyMatrix.cpp:31-450: D*D,
// D*F, F*D, F*F, and the dense updates of src/hmat_tools/Update.cpp:14-108),
// which the reference issues one gemm at a time.
#include "dense_ops.h"

#include <algorithm>

namespace hmb {

namespace {

constexpr int kT = 256;
constexpr int kKC = 16;   // inner chunk
constexpr int kLd = 68;   // smem row stride (doubles): conflict-free m8n8k4 fragment loads

// Shared tiles of one CTA: two stages of a 64 x kKC chunk of op(A) (A(i, p)
// at a[s][p][i]) and a kKC x 64 chunk of op(B) (B(p, j) at b[s][p][j]).
struct GemmSmem {
    double a[2][kKC][kLd];
    double b[2][kKC][kLd];
};

__device__ __forceinline__ double ld_op(const double* X, int ld, bool trans, int i, int j) {
    return trans ? X[j + (long long)i * ld] : X[i + (long long)j * ld];
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

// Stage the chunk p0 .. p0 + kKC of the tile at (i0, j0) (zero outside op's
// m, n, k); the global reads run along each operand's contiguous index.
__device__ __forceinline__ void gemm_load_chunk(const GemmOp& op, int i0, int j0, int p0,
                                                GemmSmem& sm, int s) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < (64 * kKC) / kT; ++q) {
        const int e = tid + q * kT;
        int i, p;
        if (op.transA) { p = e & (kKC - 1); i = e / kKC; }
        else { i = e & 63; p = e >> 6; }
        const int gi = i0 + i, gp = p0 + p;
        const bool v = gi < op.m && gp < op.k;
        cp_async8(&sm.a[s][p][i],
                  v ? (op.transA ? op.A + gp + (long long)gi * op.lda : op.A + gi + (long long)gp * op.lda)
                    : op.A,
                  v);
    }
#pragma unroll
    for (int q = 0; q < (64 * kKC) / kT; ++q) {
        const int e = tid + q * kT;
        int j, p;
        if (op.transB) { j = e & 63; p = e >> 6; }
        else { p = e & (kKC - 1); j = e / kKC; }
        const int gj = j0 + j, gp = p0 + p;
        const bool v = gj < op.n && gp < op.k;
        cp_async8(&sm.b[s][p][j],
                  v ? (op.transB ? op.B + gj + (long long)gp * op.ldb : op.B + gp + (long long)gj * op.ldb)
                    : op.B,
                  v);
    }
}

// One 64x64 output tile of one op, computed by the whole CTA.  k < 0 means
// C = alpha A + beta C.  k >= 0: the FP64 tensor cores (mma.sync m8n8k4),
// warp w owning rows 32 (w & 1) .. + 32 and columns 16 (w >> 1) .. + 16 of
// the tile, chunks of kKC staged by cp.async one chunk ahead.
__device__ void gemm_tile(const GemmOp& op, int tile, GemmSmem& sm) {
    const int tiles_m = (op.m + 63) / 64;
    const int i0 = (tile % tiles_m) * 64, j0 = (tile / tiles_m) * 64;
    const int tid = threadIdx.x;
    if (op.k < 0) {
        for (int e = tid; e < 64 * 64; e += kT) {
            int i = i0 + (e & 63), j = j0 + (e >> 6);
            if (i < op.m && j < op.n) {
                double a = op.alpha == 0.0 ? 0.0 : op.alpha * ld_op(op.A, op.lda, op.transA, i, j);
                double* c = op.C + i + (long long)j * op.ldc;
                *c = op.beta == 0.0 ? a : a + op.beta * *c;
            }
        }
        return;
    }
    const int warp = tid >> 5, lane = tid & 31;
    const int r0 = (warp & 1) * 32 + (lane >> 2), c0 = (warp >> 1) * 16 + (lane >> 2);
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int nch = (op.k + kKC - 1) / kKC;
    if (nch > 0) {
        gemm_load_chunk(op, i0, j0, 0, sm, 0);
        cp_async_commit();
    }
    for (int ch = 0; ch < nch; ++ch) {
        const int s = ch & 1;
        if (ch + 1 < nch) {
            gemm_load_chunk(op, i0, j0, (ch + 1) * kKC, sm, s ^ 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kKC / 4; ++ks) {
            const int p = ks * 4 + (lane & 3);
            double af[4], bf[2];
#pragma unroll
            for (int mb = 0; mb < 4; ++mb) af[mb] = sm.a[s][p][r0 + mb * 8];
#pragma unroll
            for (int nb = 0; nb < 2; ++nb) bf[nb] = sm.b[s][p][c0 + nb * 8];
#pragma unroll
            for (int mb = 0; mb < 4; ++mb)
#pragma unroll
                for (int nb = 0; nb < 2; ++nb) dmma(acc[mb][nb], af[mb], bf[nb]);
        }
        __syncthreads();   // stage s is refilled by the next iteration's load
    }
    // C fragment: row lane / 4, columns 2 (lane % 4) + h of each 8 x 8 block
#pragma unroll
    for (int mb = 0; mb < 4; ++mb) {
        const int i = i0 + (warp & 1) * 32 + mb * 8 + (lane >> 2);
        if (i >= op.m) continue;
#pragma unroll
        for (int nb = 0; nb < 2; ++nb)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + (warp >> 1) * 16 + nb * 8 + 2 * (lane & 3) + h;
                if (j >= op.n) continue;
                double* c = op.C + i + (long long)j * op.ldc;
                const double v = op.alpha * acc[mb][nb][h];
                *c = op.beta == 0.0 ? v : v + op.beta * *c;
            }
    }
}

// One CTA per (op, 64x64 output tile).
__global__ void __launch_bounds__(kT, 2)
gemm_ops_kernel(const GemmOp* __restrict__ ops, const int* __restrict__ tile_op,
                const int* __restrict__ tile_id, const RelocBases bases) {
    __shared__ __align__(16) GemmSmem sm;
    GemmOp op = ops[tile_op[blockIdx.x]];
    op.A = reloc(op.A, bases);
    op.B = reloc(op.B, bases);
    op.C = reloc(op.C, bases);
    gemm_tile(op, tile_id[blockIdx.x], sm);
}

// One CTA per worker: ops [begin[w], begin[w+1]) in order, all tiles of each.
__global__ void __launch_bounds__(kT, 2)
gemm_worker_kernel(const GemmOp* __restrict__ ops, const int* __restrict__ begin,
                   const RelocBases bases) {
    __shared__ __align__(16) GemmSmem sm;
    for (int i = begin[blockIdx.x]; i < begin[blockIdx.x + 1]; ++i) {
        GemmOp op = ops[i];
        op.A = reloc(op.A, bases);
        op.B = reloc(op.B, bases);
        op.C = reloc(op.C, bases);
        const int tiles = ((op.m + 63) / 64) * ((op.n + 63) / 64);
        for (int t = 0; t < tiles; ++t) {
            gemm_tile(op, t, sm);
            __syncthreads();
        }
    }
}

}  // namespace

void upload_gemm_tiles(Context& ctx, const std::vector<GemmOp>& ops, GemmTileList& out) {
    out.ntiles = 0;
    std::vector<int> tile_op, tile_id;
    for (size_t o = 0; o < ops.size(); ++o) {
        const GemmOp& g = ops[o];
        if (g.m <= 0 || g.n <= 0) continue;
        int tiles = ceil_div(g.m, 64) * ceil_div(g.n, 64);
        for (int t = 0; t < tiles; ++t) {
            tile_op.push_back((int)o);
            tile_id.push_back(t);
        }
    }
    if (tile_op.empty()) return;
    out.ops.upload(ops, ctx.stream);
    out.tile_op.upload(tile_op, ctx.stream);
    out.tile_id.upload(tile_id, ctx.stream);
    out.ntiles = (int)tile_op.size();
}

void launch_gemm_tiles(Context& ctx, const GemmTileList& L, const RelocBases& bases,
                       const char* name) {
    if (L.ntiles == 0) return;
    LaunchScope ls(ctx, name);
    gemm_ops_kernel<<<(unsigned)L.ntiles, kT, 0, ctx.stream>>>(L.ops.get(), L.tile_op.get(),
                                                               L.tile_id.get(), bases);
    HMB_CHECK_LAUNCH();
}

void launch_gemm_ops(Context& ctx, const std::vector<GemmOp>& ops, const char* name) {
    GemmTileList L;
    upload_gemm_tiles(ctx, ops, L);
    launch_gemm_tiles(ctx, L, RelocBases{}, name);
}

void upload_gemm_list(Context& ctx, const std::vector<GemmOp>& ops, const std::vector<int>& begin,
                      GemmList& out) {
    out.nw = 0;
    if (ops.empty() || begin.size() < 2) return;
    out.ops.upload(ops, ctx.stream);
    out.begin.upload(begin, ctx.stream);
    out.nw = (int)begin.size() - 1;
}

void launch_gemm_list(Context& ctx, const GemmList& L, const RelocBases& bases, const char* name) {
    if (L.nw == 0) return;
    LaunchScope ls(ctx, name);
    gemm_worker_kernel<<<(unsigned)L.nw, kT, 0, ctx.stream>>>(L.ops.get(), L.begin.get(), bases);
    HMB_CHECK_LAUNCH();
}

void launch_gemm_workers(Context& ctx, const std::vector<GemmOp>& ops,
                         const std::vector<int>& begin, const char* name) {
    GemmList L;
    upload_gemm_list(ctx, ops, begin, L);
    launch_gemm_list(ctx, L, RelocBases{}, name);
}

}  // namespace hmb
