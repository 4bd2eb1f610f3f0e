// Batched low-rank rounding on the device (see lowrank.cu).
#pragma once
#include <vector>

#include "engine.h"
#include "reloc.h"

namespace hmb {

// Finest relative truncation tolerance the FP32 roundings of the
// low-precision phase resolve (a coarser one applies as given).
constexpr double kLowPrecisionTolFloor = 1e-6;

enum RoundKind : int {
    ROUND_SET = 0,      // out = (alpha U1, V1)
    ROUND_CONCAT = 1,   // out = ([beta U2, alpha U1], [V2, V1])      (exact)
    ROUND_GENERAL = 2,  // out = best rank-rout of alpha U1 V1^T + beta U2 V2^T
    ROUND_DENSE = 3,    // out = best rank-rout of alpha D1 + beta U2 V2^T
    ROUND_ORTHO = 4,    // out = best rank-rout of Q1 V1^T, Q1 orthonormal
};

struct RoundOp {
    const double* u1;   // U1 (m x r1) / D1 (m x n) / Q1 (m x r1)
    const double* v1;   // V1 (n x r1)
    const double* u2;   // U2 (m x r2)
    const double* v2;   // V2 (n x r2)
    double* uo;         // m x rout, ld m
    double* vo;         // n x rout, ld n
    double* work;       // scratch, round_work_size() doubles
    double alpha, beta;
    int kind, m, n, r1, r2, rout;
    int ldu1, ldv1, ldu2, ldv2;
    // > 0: also drop the singular values at or below tol * sigma_0 (all but
    // sigma_0 when sigma_0 < tol^2), writing zero columns in their place
    // (GENERAL, DENSE, ORTHO).
    double tol;
    int* rank_out;      // if set: receives the rank of the output
    // if set: the ranks of the inputs are min(r1, *r1_dev) / min(r2, *r2_dev),
    // read when the op runs (ranks left by earlier ops of a truncating run);
    // outputs are zero beyond their rank
    const int* r1_dev;
    const int* r2_dev;
};

// A device-resident list of rounding ops in worker order (see
// launch_round_workers).
struct RoundList {
    DeviceBuffer<RoundOp> ops;
    DeviceBuffer<int> begin, workers;
    int nw = 0;
    long long smem_double = 0, smem_float = 0;   // shared elements per CTA
};
void upload_round_list(Context& ctx, const std::vector<RoundOp>& ops,
                       const std::vector<int>& begin, RoundList& out);
void launch_round_list(Context& ctx, const RoundList& L, const RelocBases& bases,
                       const char* name);

// Scratch doubles one op needs (0 for SET / CONCAT).
long long round_work_size(const RoundOp& op);

// Launches one CTA per op.  Ops must write disjoint outputs.
void launch_round_ops(Context& ctx, std::vector<RoundOp>& ops, const char* name);

// One CTA per worker w running ops [begin[w], begin[w+1]) in order; different
// workers must write disjoint outputs.
void launch_round_workers(Context& ctx, const std::vector<RoundOp>& ops,
                          const std::vector<int>& begin, const char* name);

// Orthonormal basis of the columns of Y (m x k, overwritten), written to Q
// (m x min(m,k)): Householder QR, then Q = H_1 ... H_kk [I; 0].
struct QrOp {
    double* Y;
    double* Q;
    double* tau;   // min(m,k) doubles of scratch
    int m, k, ldy, pad;
};
void launch_qr_formq(Context& ctx, const std::vector<QrOp>& ops, const char* name);

}  // namespace hmb
