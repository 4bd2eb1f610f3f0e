// Device work lists of one subtree of one H-matrix (see matmul.cu), shared
// by the FP64 and the tensor-core H-matrix x dense products.
#pragma once
#include "engine.h"

namespace hmb {

// Work lists of one subtree (device arrays), independent of the operands.
struct P1T {
    const double* W;   // nin x r, ld ldw
    long long in_off;  // row offset into the job input
    long long t_rel;   // T_b = T + t_rel * k (r x k, ld r)
    int nin, r, ldw, pad;
};

struct P2T {
    long long out_off;  // row offset of the tile's first row in the job output
    int r0, rows, e0, e1;
};

struct P2Entry {
    const double* A;   // element (i,p) = transA ? A[p + i*lda] : A[i + p*lda]
    long long b_off;   // b_from_t ? T + b_off * k (ld ldt) : job input + b_off
    int lda, inner, transA, b_from_t, ldt;
    int cbeg;          // first column of this entry in its tile's concatenation
};

struct JobTemplate {
    DeviceBuffer<P1T> p1;
    DeviceBuffer<P2T> p2;
    DeviceBuffer<P2Entry> ent;
    int n1 = 0, n2 = 0;
    long long t_rows = 0;   // sum of the ranks: T holds t_rows * k entries
};

}  // namespace hmb
