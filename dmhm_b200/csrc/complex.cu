// Complex-double H-matrices (HMat2d<std::complex<double>> / HMat3d, explicitly
// instantiated by the reference at src/HMat2d/HMat2d.cpp:1321-1324).
//
// A complex matrix A is stored in its real form R(A): every grid point owns
// two rows and two columns (real part, imaginary part), and the complex entry
// a + bi becomes the 2 x 2 block [[a, -b], [b, a]].  A complex vector stored
// as interleaved (re, im) pairs -- the memory of std::complex<double>[] -- is
// its own real form, so R(A) x_real is (A x) in place.  The map is an algebra
// homomorphism: R(A B) = R(A) R(B), R(A^H) = R(A)^T, ||R(A)||_2 = ||A||_2, and
// a complex rank-r block is a real rank-2r block (its singular values come in
// equal pairs), so products, rounding, truncation and Schulz run unchanged on
// the real form with maxRank 2r, on the FP64 tensor-core kernels.
//
// Complex scalars and the transpose without conjugation are applied around
// the real product:
//   A x    = R(A) x,               A^H x = R(A)^T x,
//   A^T x  = conj(R(A)^T conj(x)), y := alpha t + beta y (complex alpha, beta).
#include "engine.h"

namespace hmb {

namespace {

constexpr int kT = 256;

// C(:, j) := alpha * (conj_t ? conj(T(:, j)) : T(:, j)) + beta * C(:, j)
// over n complex rows and k columns (leading dimensions in complex elements).
__global__ void complex_combine_kernel(const double2* __restrict__ T, int ldt, double2* C, int ldc,
                                       int n, int k, double ar, double ai, double br, double bi,
                                       int conj_t) {
    const long long total = (long long)n * k;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        double2 t = T[i + (long long)j * ldt];
        if (conj_t) t.y = -t.y;
        double2* c = C + i + (long long)j * ldc;
        double2 r;
        r.x = ar * t.x - ai * t.y;
        r.y = ar * t.y + ai * t.x;
        if (br != 0.0 || bi != 0.0) {
            const double2 y = *c;
            r.x += br * y.x - bi * y.y;
            r.y += br * y.y + bi * y.x;
        }
        *c = r;
    }
}

// D = conj(S) (n complex rows, k columns).
__global__ void complex_conj_kernel(const double2* __restrict__ S, int lds, double2* __restrict__ D,
                                    int ldd, int n, int k) {
    const long long total = (long long)n * k;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        double2 s = S[i + (long long)j * lds];
        s.y = -s.y;
        D[i + (long long)j * ldd] = s;
    }
}

int grid_for(const Context& ctx, long long total) {
    return (int)std::max<long long>(1, std::min<long long>((total + kT - 1) / kT, 4LL * ctx.num_sms));
}

// Elementwise work on the real form of one stored matrix piece (column-major
// m x n, leading dimension m): kind 0 rows 2i, 2i+1 := [[a, -b], [b, a]] of
// them (left multiplication by alpha = a + bi), kind 1 negate odd rows (the
// conjugate of a factor: conj(U V^T) = (J U)(J V)^T with J = diag(1, -1)),
// kind 2 negate the entries with row + column odd (the conjugate of a dense
// block, J D J), kind 3 add [[a, -b], [b, a]] on the diagonal pairs (a dense
// diagonal block plus alpha I).
struct PieceTask {
    double* p;
    int m, n, kind, pad;
};

__global__ void complex_pieces_kernel(const PieceTask* __restrict__ tasks, double a, double b) {
    const PieceTask t = tasks[blockIdx.x];
    if (t.kind == 0) {
        const long long pairs = (long long)(t.m / 2) * t.n;
        for (long long e = threadIdx.x; e < pairs; e += blockDim.x) {
            const int i = (int)(e % (t.m / 2)), j = (int)(e / (t.m / 2));
            double* c = t.p + 2 * i + (long long)j * t.m;
            const double x = c[0], y = c[1];
            c[0] = a * x - b * y;
            c[1] = b * x + a * y;
        }
    } else if (t.kind == 1) {
        const long long total = (long long)(t.m / 2) * t.n;
        for (long long e = threadIdx.x; e < total; e += blockDim.x) {
            const int i = (int)(e % (t.m / 2)), j = (int)(e / (t.m / 2));
            t.p[2 * i + 1 + (long long)j * t.m] *= -1.0;
        }
    } else if (t.kind == 2) {
        const long long total = (long long)t.m * t.n;
        for (long long e = threadIdx.x; e < total; e += blockDim.x) {
            const int i = (int)(e % t.m), j = (int)(e / t.m);
            if ((i + j) & 1) t.p[e] = -t.p[e];
        }
    } else {
        for (int i = threadIdx.x; i < t.m / 2; i += blockDim.x) {
            double* d = t.p + 2 * i + (long long)(2 * i) * t.m;   // (2i, 2i)
            d[0] += a;
            d[1] += b;                           // (2i+1, 2i)
            d[t.m] -= b;                         // (2i, 2i+1)
            d[t.m + 1] += a;                     // (2i+1, 2i+1)
        }
    }
}

void run_pieces(Context& ctx, HMatrix& H, const std::vector<PieceTask>& tasks, double a, double b,
                const char* name) {
    if (tasks.empty()) return;
    DeviceBuffer<PieceTask> d;
    d.upload(tasks, ctx.stream);
    LaunchScope ls(ctx, name);
    complex_pieces_kernel<<<(unsigned)tasks.size(), kT, 0, ctx.stream>>>(d.get(), a, b);
    HMB_CHECK_LAUNCH();
    H.shadow_valid = false;   // the FP32 copy no longer matches
}

}  // namespace

// A := alpha A for complex alpha (Scale, HMat2d.cpp:616-647): every dense
// block and every U factor multiplied from the left by alpha I.
void complex_scale(Context& ctx, HMatrix& H, double a, double b) {
    HMB_REQUIRE(H.S && H.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
    std::vector<PieceTask> t;
    for (int blk : H.S->leaves) {
        const Block& B = H.S->blocks[blk];
        if (B.m == 0 || B.n == 0) continue;
        if (B.kind == KIND_DENSE) t.push_back({H.D(blk), B.m, B.n, 0, 0});
        else if (H.rank[blk] > 0) t.push_back({H.U(blk), B.m, H.rank[blk], 0, 0});
    }
    run_pieces(ctx, H, t, a, b, "complex_scale");
}

// A := A + alpha I for complex alpha (AddConstantToDiagonal, HMat2d.cpp:704-744).
void complex_add_diagonal(Context& ctx, HMatrix& H, double a, double b) {
    HMB_REQUIRE(H.S && H.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
    std::vector<PieceTask> t;
    for (int blk : H.S->leaves) {
        const Block& B = H.S->blocks[blk];
        if (B.kind == KIND_DENSE && B.row_off == B.col_off && B.m == B.n && B.m > 0)
            t.push_back({H.D(blk), B.m, B.n, 3, 0});
    }
    run_pieces(ctx, H, t, a, b, "complex_add_diagonal");
}

// A := conj(A) in place (the conjugation of ConjugateFrom, HMat2d.cpp:424-472).
void complex_conjugate(Context& ctx, HMatrix& H) {
    HMB_REQUIRE(H.S && H.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
    std::vector<PieceTask> t;
    for (int blk : H.S->leaves) {
        const Block& B = H.S->blocks[blk];
        if (B.m == 0 || B.n == 0) continue;
        if (B.kind == KIND_DENSE) {
            t.push_back({H.D(blk), B.m, B.n, 2, 0});
        } else if (H.rank[blk] > 0) {
            t.push_back({H.U(blk), B.m, H.rank[blk], 1, 0});
            t.push_back({H.V(blk), B.n, H.rank[blk], 1, 0});
        }
    }
    run_pieces(ctx, H, t, 0.0, 0.0, "complex_conjugate");
}

void multiply_dense(HMatrix& H, int transpose, double alpha, const double* B, int ldb, double beta,
                    double* C, int ldc, int nrhs);

void multiply_dense_complex(HMatrix& H, int op, double ar, double ai, const double* B, int ldb,
                            double br, double bi, double* C, int ldc, int nrhs) {
    HMB_REQUIRE(H.S && H.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
    HMB_REQUIRE(op >= 0 && op <= 2, HM_ERR_ARGUMENT, "op must be 0 (A), 1 (A^T) or 2 (A^H)");
    HMB_REQUIRE(nrhs >= 0, HM_ERR_ARGUMENT, "nrhs must be >= 0");
    Context& ctx = *H.ctx;
    const int n = H.height() / 2;   // complex rows (square)
    HMB_REQUIRE(ldb >= std::max(1, n) && ldc >= std::max(1, n), HM_ERR_ARGUMENT,
                "leading dimension too small");
    if (nrhs == 0 || n == 0) return;
    cudaStream_t st = ctx.stream;
    const int rt = op == 0 ? 0 : 1;   // real product: R(A) or R(A)^T
    if (op != 1 && ai == 0.0 && bi == 0.0) {
        multiply_dense(H, rt, ar, B, 2 * ldb, br, C, 2 * ldc, nrhs);
        return;
    }
    DeviceBuffer<double> tin, tout;
    const double* src = B;
    int lds = ldb;
    if (op == 1) {
        tin.allocate((size_t)2 * n * nrhs, st);
        LaunchScope ls(ctx, "complex_conj");
        complex_conj_kernel<<<grid_for(ctx, (long long)n * nrhs), kT, 0, st>>>(
            reinterpret_cast<const double2*>(B), ldb, reinterpret_cast<double2*>(tin.get()), n, n,
            nrhs);
        HMB_CHECK_LAUNCH();
        src = tin.get();
        lds = n;
    }
    tout.allocate((size_t)2 * n * nrhs, st);
    multiply_dense(H, rt, 1.0, src, 2 * lds, 0.0, tout.get(), 2 * n, nrhs);
    LaunchScope ls(ctx, "complex_combine");
    complex_combine_kernel<<<grid_for(ctx, (long long)n * nrhs), kT, 0, st>>>(
        reinterpret_cast<const double2*>(tout.get()), n, reinterpret_cast<double2*>(C), ldc, n,
        nrhs, ar, ai, br, bi, op == 1 ? 1 : 0);
    HMB_CHECK_LAUNCH();
}

}  // namespace hmb
