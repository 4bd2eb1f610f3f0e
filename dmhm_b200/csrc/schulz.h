// Schulz inversion and two-norm estimation (see schulz.cu).
#pragma once
#include <vector>

#include "engine.h"

namespace hmb {

struct SchulzResult {
    int iterations = 0;
    int low_iterations = 0;      // iterations run in the low-precision phase
    std::vector<double> trace;   // [est ||A||, est ||I - X_k A|| per stop check]
};

// Block copies: dst (m x n, ld m) = alpha * (transpose ? src^T : src), src
// with leading dimension lds; one CTA per task, all tasks in one launch.
struct CopyTask {
    const double* src;
    double* dst;
    double alpha;
    int m, n, lds, transpose;
};
void launch_copy_tasks(Context& ctx, const std::vector<CopyTask>& tasks, const char* name);

double estimate_two_norm(Context& ctx, HMatrix& A, double theta, double confidence);
// Drops the trailing zero columns that tolerance truncation leaves in the
// low-rank blocks when that saves at least 5 % of the low-rank storage
// (synchronizes to read the ranks back).
void compact_ranks(Context& ctx, HMatrix& H);
// mixed_switch > 0: mixed precision (iterations in the low-precision phase
// while the last ||I - X A|| estimate is above mixed_switch).
SchulzResult schulz_invert(Context& ctx, HMatrix& A, int num_iterations, double theta,
                           double confidence, double stop_tol, double mixed_switch = 0.0);

}  // namespace hmb
