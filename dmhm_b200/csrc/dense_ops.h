// Batched small dense products and elementwise updates (see dense_ops.cu).
#pragma once
#include <vector>

#include "engine.h"
#include "reloc.h"

namespace hmb {

// C = alpha op(A) op(B) + beta C (k >= 0), or C = alpha op(A) + beta C (k < 0).
// op(X) = X^T when trans is set.  All column-major.  beta == 0 never reads C.
struct GemmOp {
    const double* A;
    const double* B;
    double* C;
    double alpha, beta;
    int m, n, k, lda, ldb, ldc, transA, transB;
};

// Launches all ops in one kernel; ops must write disjoint C matrices.
void launch_gemm_ops(Context& ctx, const std::vector<GemmOp>& ops, const char* name);
// The same from a device-resident list (one CTA per 64 x 64 tile of every
// op) whose pointers may be tagged offsets (reloc.h).
struct GemmTileList {
    DeviceBuffer<GemmOp> ops;
    DeviceBuffer<int> tile_op, tile_id;
    int ntiles = 0;
};
void upload_gemm_tiles(Context& ctx, const std::vector<GemmOp>& ops, GemmTileList& out);
void launch_gemm_tiles(Context& ctx, const GemmTileList& L, const RelocBases& bases,
                       const char* name);

// One CTA per worker w running ops [begin[w], begin[w+1]) in order (ops of one
// worker may update the same C); different workers write disjoint C.
void launch_gemm_workers(Context& ctx, const std::vector<GemmOp>& ops,
                         const std::vector<int>& begin, const char* name);
// The same from a device-resident list whose pointers may be tagged offsets
// (reloc.h).
struct GemmList {
    DeviceBuffer<GemmOp> ops;
    DeviceBuffer<int> begin;
    int nw = 0;
};
void upload_gemm_list(Context& ctx, const std::vector<GemmOp>& ops, const std::vector<int>& begin,
                      GemmList& out);
void launch_gemm_list(Context& ctx, const GemmList& L, const RelocBases& bases, const char* name);

}  // namespace hmb
