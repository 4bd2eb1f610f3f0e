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

// Elementwise / structural operations used by Schulz inversion.
void hmat_copy(Context& ctx, const HMatrix& src, HMatrix& dst);        // CopyFrom
void hmat_transpose(Context& ctx, const HMatrix& src, HMatrix& dst);   // TransposeFrom / AdjointFrom
void hmat_scale(Context& ctx, HMatrix& H, double alpha);               // Scale
void hmat_add_diagonal(Context& ctx, HMatrix& H, double alpha);        // AddConstantToDiagonal
void hmat_update_with(Context& ctx, HMatrix& A, double alpha, const HMatrix& B);  // UpdateWith
void hmat_set_identity(Context& ctx, HMatrix& H);                     // SetToIdentity

}  // namespace hmb
