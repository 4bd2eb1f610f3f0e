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

__device__ __forceinline__ double ld_op(const double* X, int ld, bool trans, int i, int j) {
    return trans ? X[j + (long long)i * ld] : X[i + (long long)j * ld];
}

// One 64x64 output tile of one op, computed by the whole CTA.  k < 0 means
// C = alpha A + beta C.
__device__ void gemm_tile(const GemmOp& op, int tile, double (*sA)[65], double (*sB)[65]) {
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
    const int tr = (tid & 15) * 4, tc = (tid >> 4) * 4;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int p0 = 0; p0 < op.k; p0 += 16) {
        for (int e = tid; e < 16 * 64; e += kT) {
            int i, p;
            if (op.transA) { p = e & 15; i = e >> 4; }
            else { i = e & 63; p = e >> 6; }
            int gi = i0 + i, gp = p0 + p;
            sA[p][i] = (gi < op.m && gp < op.k) ? ld_op(op.A, op.lda, op.transA, gi, gp) : 0.0;
        }
        for (int e = tid; e < 16 * 64; e += kT) {
            int p, j;
            if (op.transB) { j = e & 63; p = e >> 6; }
            else { p = e & 15; j = e >> 4; }
            int gj = j0 + j, gp = p0 + p;
            sB[p][j] = (gj < op.n && gp < op.k) ? ld_op(op.B, op.ldb, op.transB, gp, gj) : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int p = 0; p < 16; ++p) {
            double av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = sA[p][tr + a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = sB[p][tc + b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int i = i0 + tr + a;
        if (i >= op.m) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int j = j0 + tc + b;
            if (j >= op.n) continue;
            double* c = op.C + i + (long long)j * op.ldc;
            double v = op.alpha * acc[a][b];
            *c = op.beta == 0.0 ? v : v + op.beta * *c;
        }
    }
}

// One CTA per (op, 64x64 output tile).
__global__ void __launch_bounds__(kT)
gemm_ops_kernel(const GemmOp* __restrict__ ops, const int* __restrict__ tile_op,
                const int* __restrict__ tile_id, const RelocBases bases) {
    __shared__ double sA[16][65];
    __shared__ double sB[16][65];
    GemmOp op = ops[tile_op[blockIdx.x]];
    op.A = reloc(op.A, bases);
    op.B = reloc(op.B, bases);
    op.C = reloc(op.C, bases);
    gemm_tile(op, tile_id[blockIdx.x], sA, sB);
}

// One CTA per worker: ops [begin[w], begin[w+1]) in order, all tiles of each.
__global__ void __launch_bounds__(kT)
gemm_worker_kernel(const GemmOp* __restrict__ ops, const int* __restrict__ begin,
                   const RelocBases bases) {
    __shared__ double sA[16][65];
    __shared__ double sB[16][65];
    for (int i = begin[blockIdx.x]; i < begin[blockIdx.x + 1]; ++i) {
        GemmOp op = ops[i];
        op.A = reloc(op.A, bases);
        op.B = reloc(op.B, bases);
        op.C = reloc(op.C, bases);
        const int tiles = ((op.m + 63) / 64) * ((op.n + 63) / 64);
        for (int t = 0; t < tiles; ++t) {
            gemm_tile(op, t, sA, sB);
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
