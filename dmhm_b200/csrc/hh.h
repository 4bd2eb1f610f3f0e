// H*H product with randomized low-rank compression (see hh.cu).
#pragma once
#include "engine.h"

namespace hmb {

// C := alpha A B (fresh = true; C is rebuilt) or C := alpha A B + beta C
// (fresh = false; C keeps its structure).  A, B, C share one block structure
// and C must be a different object from A and B.  With a compression
// tolerance, compact = true drops C's unused trailing columns at the end
// (compact_ranks, which waits for the product); callers that reach a
// synchronisation point anyway pass false and compact there.
void hh_multiply(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha,
                 double beta, HMatrix& C, bool fresh, bool compact = true);

// Products of sub-trees (blocks a of A, b of B into block c of C, all on one
// structure), listed in the order the reference runs them: fresh: C_c :=
// alpha A_a B_b (the sub-tree rebuilt), else C_c := alpha A_a B_b + beta C_c.
// Every C leaf outside the listed c sub-trees keeps its content; the c
// sub-trees must be disjoint and must not be read by another listed product.
// The serial generator advances as the reference's sequence of Multiply
// calls would.  C must exist and differ from A and B.
struct HHRoot {
    int a, b, c;
};
void hh_multiply_sub(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha,
                     double beta, HMatrix& C, bool fresh, const std::vector<HHRoot>& roots);
void hh_multiply_roots(Context& ctx, const HMatrix& A, const HMatrix& B, double alpha,
                       double beta, HMatrix& C, bool fresh_plan,
                       const std::vector<HHRoot>& roots, bool compact);

// Elementwise / structural operations used by Schulz inversion.
void hmat_copy(Context& ctx, const HMatrix& src, HMatrix& dst);        // CopyFrom
void hmat_transpose(Context& ctx, const HMatrix& src, HMatrix& dst);   // TransposeFrom / AdjointFrom
void hmat_scale(Context& ctx, HMatrix& H, double alpha);               // Scale
void hmat_add_diagonal(Context& ctx, HMatrix& H, double alpha);        // AddConstantToDiagonal
void hmat_update_with(Context& ctx, HMatrix& A, double alpha, const HMatrix& B);  // UpdateWith
void hmat_set_identity(Context& ctx, HMatrix& H);                     // SetToIdentity
void hmat_direct_invert(Context& ctx, HMatrix& X);                    // DirectInvert

}  // namespace hmb
