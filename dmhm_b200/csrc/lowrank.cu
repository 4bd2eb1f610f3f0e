// Batched low-rank rounding: the device replacement of the reference's
// per-block LAPACK sequences
//   RoundedUpdate   (src/hmat_tools/RoundedUpdate.cpp:14-162: two geqrf,
//                    R1 R2^T, gesvd, two ormqr),
//   Compress / D*D  (src/hmat_tools/Compress.cpp:14-53,
//                    MultiplyMatrix.cpp:405-550: gesvd of a dense block),
//   randomized H*H  (include/dmhm/hmat_tools.hpp:1690-1745: geqp3 + orgqr of
//                    the sample, gesvd of the projected block).
// One CTA (256 threads) owns one rounding: Householder QR of the stacked
// factors (FP64, rank-deficient safe: zero columns give tau = 0), the small
// core M = R_u R_v^T, a one-sided Jacobi SVD of M with the rotations
// accumulated, selection of the largest singular triplets, and the
// reflectors applied back.  The truncated result is the same best rank-r
// approximation the reference computes (its factors differ only by the
// usual sign / rotation freedom of an SVD).
//
// Every device routine is written for an arithmetic type R: double (the
// reference's precision) or float, the low-precision form used by the early
// iterations of a mixed-precision Schulz run (inputs and outputs stay FP64;
// stacks, reflectors, core and rotations are FP32 in the work area and in
// shared memory).
#include "lowrank.h"

#include <algorithm>
#include <mutex>
#include <set>

namespace hmb {

namespace {

constexpr int kT = 256;
constexpr int kW = kT / 32;
constexpr int kMaxK = 128;         // largest stacked rank handled
constexpr long long kSmemBytes = 65536;   // M and J up to 64 x 64 FP64
// FP32 (low-precision phase): M and J up to 101 x 101, so that the 96-column
// cores of complex matrices of rank 24 (real rank 48) stay in shared memory
// (2 CTAs an SM for such launches; 15 % less rounding time on them)
constexpr long long kSmemBytesF32 = 81920;
constexpr int kQB = 4;           // columns a warp updates together when applying reflectors
constexpr int kJacobiSweeps = 40;  // bounded; converges in ~6-12

// Per-precision constants: Jacobi's orthogonality threshold (relative to the
// column norms), the squared-norm level below which a column counts as
// rounding noise (relative to ||M||_F^2), and the smallest resolvable
// relative truncation tolerance.
template <typename R> struct Prec;
template <> struct Prec<double> {
    static constexpr double jtol = 1e-15, tiny = 1e-32, tol_floor = 0.0;
};
template <> struct Prec<float> {
    static constexpr float jtol = 1e-6f, tiny = 1e-12f;
    static constexpr double tol_floor = kLowPrecisionTolFloor;
};

__device__ __forceinline__ double r_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float r_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double r_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float r_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double r_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float r_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double r_abs(double x) { return fabs(x); }
__device__ __forceinline__ float r_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double r_copysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float r_copysign(float a, float b) { return copysignf(a, b); }

// f(i, c) for every entry of an m x cols column-major array: column c by
// warp c % kW, rows by lane (no integer division in the index arithmetic)
template <typename F>
__device__ __forceinline__ void for_each_entry(int m, int cols, F f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < cols; c += kW)
        for (int i = lane; i < m; i += 32) f(i, c);
}

template <typename R>
__device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R>
__device__ R block_sum(R v, R* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    R t = threadIdx.x < kW ? red[threadIdx.x] : R(0);
    if (warp == 0) t = warp_sum(t);
    if (threadIdx.x == 0) red[kW] = t;
    __syncthreads();
    R r = red[kW];
    __syncthreads();
    return r;
}

// In-place Householder QR (LAPACK dgeqr2 conventions: beta = -sign(alpha)
// ||x||, v(1) = 1 implicit, tau = (beta - alpha) / beta; tau = 0 when the
// column below the diagonal is zero).  Column c belongs to warp c % kW for
// the whole factorization: the owner of column j has applied reflectors
// 0..j-1 to it and forms reflector j with warp reductions only; one barrier
// per column publishes it; every warp then applies it to its own columns.
template <typename R>
__device__ void cta_qr(R* A, int m, int n, int ld, R* tau, R* red) {
    (void)red;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kk = min(m, n);
    for (int j = 0; j < kk; ++j) {
        R* col = A + j + (long long)j * ld;
        const int len = m - j;
        if (warp == j % kW) {
            __syncwarp();   // this warp's last update of column j used other lanes' rows
            R s = 0;
            for (int i = 1 + lane; i < len; i += 32) s += col[i] * col[i];
            s = warp_sum(s);
            const R alpha = col[0];
            R t = 0, beta = alpha;
            if (s != R(0)) {
                beta = -r_copysign(r_sqrt(alpha * alpha + s), alpha);
                t = (beta - alpha) / beta;
                const R scal = R(1) / (alpha - beta);
                for (int i = 1 + lane; i < len; i += 32) col[i] *= scal;
            }
            __syncwarp();
            if (lane == 0) {
                col[0] = beta;
                tau[j] = t;
            }
        }
        __syncthreads();
        const R t = tau[j];
        if (t != R(0)) {
            // first column > j owned by this warp
            int c = j + 1 + ((warp - (j + 1) % kW + kW) % kW);
            for (; c < n; c += kW) {
                R* cc = A + j + (long long)c * ld;
                const R c0 = cc[0];
                R w = 0;
                for (int i = 1 + lane; i < len; i += 32) w += col[i] * cc[i];
                w = warp_sum(w) + c0;
                const R tw = t * w;
                __syncwarp();
                if (lane == 0) cc[0] = c0 - tw;
                for (int i = 1 + lane; i < len; i += 32) cc[i] -= tw * col[i];
            }
        }
    }
    __syncthreads();
}

// B := Q B with Q = H_0 H_1 ... H_{kk-1} from cta_qr (B is m x p;
// arithmetic in R, B may be stored in another type).  Column c of B is
// updated by warp c % kW through all reflectors, so no barrier is needed
// between them; a warp with several columns takes NB of them at a time and
// reduces their inner products together (independent shuffle chains
// overlap).  Each column sees the same operations in the same order either
// way.
template <int NB, typename R, typename RB>
__device__ __forceinline__ void warp_apply_q(const R* A, int m, int kk, int lda, const R* tau,
                                             RB* B, int p, int ldb) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < p; c += NB * kW) {
        for (int j = kk - 1; j >= 0; --j) {
            const R t = tau[j];
            if (t == R(0)) continue;
            const R* v = A + j + (long long)j * lda;
            const int len = m - j;
            R w[NB], b0[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int cb = c + b * kW;
                w[b] = 0;
                b0[b] = 0;
                if (cb < p) {
                    const RB* bc = B + (long long)cb * ldb + j;
                    b0[b] = (R)bc[0];
                    for (int i = 1 + lane; i < len; i += 32) w[b] += v[i] * (R)bc[i];
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int b = 0; b < NB; ++b) w[b] += __shfl_xor_sync(0xffffffffu, w[b], o);
            __syncwarp();
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int cb = c + b * kW;
                if (cb < p) {
                    RB* bc = B + (long long)cb * ldb + j;
                    const R tw = t * (w[b] + b0[b]);
                    if (lane == 0) bc[0] = (RB)(b0[b] - tw);
                    for (int i = 1 + lane; i < len; i += 32) bc[i] = (RB)((R)bc[i] - tw * v[i]);
                }
            }
            __syncwarp();
        }
    }
}

template <typename R, typename RB>
__device__ void cta_apply_q(const R* A, int m, int kk, int lda, const R* tau, RB* B, int p,
                            int ldb) {
    if (p > kW) warp_apply_q<kQB>(A, m, kk, lda, tau, B, p, ldb);
    else warp_apply_q<1>(A, m, kk, lda, tau, B, p, ldb);
    __syncthreads();
}

__device__ __forceinline__ int rr_pos(int i, int step, int n) {
    // (i - 1 + step) mod (n - 1) for 0 <= i - 1 + step < 2 (n - 1)
    const int x = i - 1 + step;
    return i == 0 ? 0 : 1 + (x >= n - 1 ? x - (n - 1) : x);
}

// One column pair (p, q) of round-robin step `step` (pair index k of n/2),
// handled by LANES lanes of a warp (hl = this lane's index among them); all
// lanes of the warp take part in the shuffles, live pair or not.  Rotates
// the pair when its columns are not yet orthogonal to the threshold, with
// the rotation's cosine and sine written without a division:
// h = sqrt(d^2 + 4c^2), s = |d| + h, r = 1/sqrt(2hs) give cos = s r and
// sin = sign(dc) 2|c| r (the rotation by the angle whose tangent t is the
// smaller root of t^2 + 2 zeta t - 1 = 0, zeta = d / (2c), d = b - a), and
// t c = sign(d) 4 c^2 h r^2 updates the squared norms.
template <int LANES, typename R>
__device__ __forceinline__ void jacobi_pair(R* M, int rows, int cols, R* J, R* nrm, int* flag,
                                            int k, int hl, int step, int n, R tiny, R jt2) {
    int p = 0, q = 1;
    if (k < n / 2) {
        p = rr_pos(k, step, n);
        q = rr_pos(n - 1 - k, step, n);
    }
    const bool live = k < n / 2 && p < cols && q < cols;
    if (p > q) { int t = p; p = q; q = t; }
    R* gp = M + (long long)p * rows;
    R* gq = M + (long long)q * rows;
    R c = 0;
    if (live)
        for (int i = hl; i < rows; i += LANES) c = r_fma(gp[i], gq[i], c);
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    const R a = live ? nrm[p] : R(0), b = live ? nrm[q] : R(0);
    if (live && c != R(0) && a > tiny && b > tiny && c * c > jt2 * (a * b)) {
        const R d = b - a;
        const R h = r_sqrt(r_fma(d, d, R(4) * c * c));
        const R s = r_abs(d) + h;
        const R r = r_rsqrt(R(2) * h * s);
        const R cs = s * r;
        const R sn = r_copysign(R(2) * r_abs(c), d * c) * r;
        for (int i = hl; i < rows; i += LANES) {
            const R x = gp[i], y = gq[i];
            gp[i] = cs * x - sn * y;
            gq[i] = sn * x + cs * y;
        }
        R* jp = J + (long long)p * cols;
        R* jq = J + (long long)q * cols;
        for (int i = hl; i < cols; i += LANES) {
            const R x = jp[i], y = jq[i];
            jp[i] = cs * x - sn * y;
            jq[i] = sn * x + cs * y;
        }
        if (hl == 0) {
            const R tc = r_copysign(R(4) * c * c, d) * h * r * r;
            nrm[p] = a - tc;
            nrm[q] = b + tc;
            *flag = 1;
        }
    }
}

// One-sided (Hestenes) Jacobi: rotates the columns of M (rows x cols) until
// they are mutually orthogonal, accumulating the rotations in J (cols x cols,
// J starts as I), so M_in = M_out J^T.  Round-robin ordering: cols/2
// disjoint pairs per step, all pairs of a step at once (a half-warp per
// pair; up to 16 columns, all pairs in warp 0, a quarter-warp each, which
// spares the steps the CTA barrier).  Bounded number of sweeps.
// Pairs with a column below rounding level (squared norm under 1e-32 times
// the squared Frobenius norm of M) are left alone: rotating noise against
// noise never settles, and such columns carry no singular value above
// rounding level.
//
// A core holding NaN or Inf (non-finite block data) sets *numflag; the
// sweeps still end within their bound.
template <typename R>
__device__ void cta_jacobi(R* M, int rows, int cols, R* J, int* flag, R* red, R* nrm,
                           int* numflag) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for_each_entry(cols, cols, [&](int i, int c) { J[i + c * cols] = i == c ? R(1) : R(0); });
    R fro = 0;
    for (long long e = threadIdx.x; e < (long long)rows * cols; e += kT) fro = r_fma(M[e], M[e], fro);
    fro = block_sum(fro, red);
    if (threadIdx.x == 0 && numflag && !isfinite((double)fro)) atomicOr(numflag, 1);
    const R tiny = R(Prec<R>::tiny) * fro;
    __syncthreads();
    if (cols < 2) return;
    const int n = cols + (cols & 1);
    // Squared column norms are kept in nrm (exact at the start of every
    // sweep, then updated by the rotations), so a pair reduces only its
    // inner product.
    const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
    constexpr R jt2 = Prec<R>::jtol * Prec<R>::jtol;
    for (int sweep = 0; sweep < kJacobiSweeps; ++sweep) {
        for (int c = warp; c < cols; c += kW) {
            const R* g = M + (long long)c * rows;
            R sq = 0;
            for (int i = lane; i < rows; i += 32) sq = r_fma(g[i], g[i], sq);
            sq = warp_sum(sq);
            if (lane == 0) nrm[c] = sq;
        }
        if (threadIdx.x == 0) *flag = 0;
        __syncthreads();
        // Convergence test on all pairs at once (the off-diagonal of the
        // Gram matrix, each pair's inner product by one thread): the sweep
        // below runs only if some pair would rotate, so the sweep that finds
        // nothing left to rotate is never run.  The inner products start at
        // a row offset that differs per lane, so the lanes of a warp read
        // different shared-memory banks.
        {
            bool rotate = false;
            for (int idx = threadIdx.x; idx < cols * cols && !rotate; idx += kT) {
                const int p = idx / cols, q = idx % cols;
                if (q <= p) continue;
                const R a = nrm[p], b = nrm[q];
                if (!(a > tiny && b > tiny)) continue;
                const R* gp = M + (long long)p * rows;
                const R* gq = M + (long long)q * rows;
                R c = 0;
                int i = lane % rows;
                for (int t = 0; t < rows; ++t) {
                    c = r_fma(gp[i], gq[i], c);
                    i = (i + 1 == rows) ? 0 : i + 1;
                }
                rotate = c != R(0) && c * c > jt2 * (a * b);
            }
            if (rotate) *flag = 1;
            __syncthreads();
            const int needed = *flag;
            __syncthreads();
            if (!needed) break;
            if (threadIdx.x == 0) *flag = 0;
            __syncthreads();
        }
        if (n <= 16) {
            // at most 8 pairs a step: warp 0 alone, 4 lanes per pair, so the
            // steps need only warp-level synchronization
            if (warp == 0) {
                for (int step = 0; step < n - 1; ++step) {
                    jacobi_pair<4>(M, rows, cols, J, nrm, flag, lane >> 2, lane & 3, step, n, tiny,
                                   jt2);
                    __syncwarp();
                }
            }
            __syncthreads();
        } else {
            for (int step = 0; step < n - 1; ++step) {
                // warp-uniform trip count: both half-warps of a warp iterate
                // together (their shuffles span the whole warp)
                for (int kb = 2 * warp; kb < n / 2; kb += 2 * kW)
                    jacobi_pair<16>(M, rows, cols, J, nrm, flag, kb + (hw & 1), hl, step, n, tiny,
                                    jt2);
                __syncthreads();
            }
        }
        const int again = *flag;
        __syncthreads();
        if (!again) break;
    }
}

// order[0..cols) = column indices of M by decreasing norm (ties by index).
template <typename R>
__device__ void cta_order_columns(const R* M, int rows, int cols, R* norms, int* order) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < cols; c += kW) {
        const R* g = M + (long long)c * rows;
        R s = 0;
        for (int i = lane; i < rows; i += 32) s = r_fma(g[i], g[i], s);
        s = warp_sum(s);
        // a NaN norm (non-finite block data, which the numerical flag
        // reports) sorts last, so that order stays a permutation
        if (lane == 0) norms[c] = s == s ? s : R(-1);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cols; j += kT) {
        const R sj = norms[j];
        int pos = 0;
        for (int i = 0; i < cols; ++i) {
            const R si = norms[i];
            pos += (si > sj || (si == sj && i < j)) ? 1 : 0;
        }
        order[pos] = j;
    }
    __syncthreads();
}

template <typename R>
struct RoundShared {
    R red[kW + 1];
    R norms[kMaxK];
    R nrm[kMaxK];    // Jacobi's running squared column norms
    int order[kMaxK];
    int flag;
};

// One rounding operation, executed by the whole CTA.  `dyn` holds the core
// and the rotations in shared memory when they fit in `smem_elems` elements.
template <typename R>
__device__ void do_round(const RoundOp& op_in, R* dyn, long long smem_elems, RoundShared<R>& sh,
                         int* numflag) {
    R* red = sh.red;
    R* norms = sh.norms;
    int* order = sh.order;
    RoundOp op = op_in;
    if (op.r1_dev) op.r1 = min(op.r1, *op.r1_dev);
    if (op.r2_dev) op.r2 = min(op.r2, *op.r2_dev);
    const int m = op.m, n = op.n;
    const int tid = threadIdx.x;

    if (op.kind == ROUND_SET || op.kind == ROUND_CONCAT) {
        // exact: [beta U2, alpha U1], [V2, V1] (SET: r2 = 0), zero beyond
        const int r2 = op.kind == ROUND_SET ? 0 : op.r2, r = op.r1 + r2;
        const int cap = max(r, op.rout);
        for_each_entry(m, cap, [&](int i, int c) {
            op.uo[i + (long long)c * m] =
                c >= r    ? 0.0
                : c < r2 ? op.beta * op.u2[i + (long long)c * op.ldu2]
                         : op.alpha * op.u1[i + (long long)(c - r2) * op.ldu1];
        });
        for_each_entry(n, cap, [&](int i, int c) {
            op.vo[i + (long long)c * n] = c >= r    ? 0.0
                                          : c < r2 ? op.v2[i + (long long)c * op.ldv2]
                                                   : op.v1[i + (long long)(c - r2) * op.ldv1];
        });
        if (tid == 0 && op.rank_out) *op.rank_out = r;
        return;
    }

    const bool ortho = op.kind == ROUND_ORTHO;
    const bool dense = op.kind == ROUND_DENSE;
    const int k = dense ? n : op.r1 + (op.kind == ROUND_GENERAL ? op.r2 : 0);
    const int rout = op.rout;
    if (m == 0 || n == 0) return;
    const int ku = ortho ? op.r1 : min(m, k);
    const int kv = dense ? n : min(n, k);
    // A block no taller than its stack (m <= k): the QR of the U stack would
    // only rotate the core's rows (Q_u is m x m), which changes neither the
    // column inner products one-sided Jacobi works on nor the rounding, so
    // the core is formed from the stack itself, M = U_cat R_v^T (or the
    // dense block), and its rotated columns are the output U directly.
    const bool skip_u = !ortho && m <= k;
    // The core and the rotations live in shared memory when they fit in
    // `smem_elems`; the stacked factors in the (L1-cached) work area.
    const long long need_mj = (long long)ku * kv + (long long)kv * kv;
    const bool mj_smem = need_mj <= smem_elems;
    R* w = reinterpret_cast<R*>(op.work);
    R* Ucat = w;
    if (!ortho) w += (long long)m * k;
    R* Vcat = w;
    if (!dense) w += (long long)n * k;
    R* tauU = w;
    w += k;
    R* tauV = w;
    w += k;
    R* M;
    R* J;
    if (mj_smem) {
        M = dyn;
        J = dyn + (long long)ku * kv;
    } else {
        M = w;
        J = w + (long long)ku * kv;
    }

    // ---- stacked factors ---------------------------------------------------
    if (op.kind == ROUND_GENERAL) {
        // [beta U2, alpha U1], [V2, V1]: U2 (the block's current factors, the
        // output of an earlier rounding) has orthogonal columns and V2
        // orthonormal ones, so the leading part of the core is already
        // diagonal and the Jacobi sweeps mostly rotate the new columns in
        const int r2 = op.r2;
        for_each_entry(m, k, [&](int i, int c) {
            Ucat[i + (long long)c * m] =
                (R)(c < r2 ? op.beta * op.u2[i + (long long)c * op.ldu2]
                           : op.alpha * op.u1[i + (long long)(c - r2) * op.ldu1]);
        });
        for_each_entry(n, k, [&](int i, int c) {
            Vcat[i + (long long)c * n] = (R)(c < r2 ? op.v2[i + (long long)c * op.ldv2]
                                                    : op.v1[i + (long long)(c - r2) * op.ldv1]);
        });
    } else if (dense) {
        for_each_entry(m, n, [&](int i, int c) {
            double v = op.alpha * op.u1[i + (long long)c * op.ldu1];
            if (op.beta != 0.0)
                for (int l = 0; l < op.r2; ++l)
                    v = fma(op.beta * op.u2[i + (long long)l * op.ldu2],
                            op.v2[c + (long long)l * op.ldv2], v);
            Ucat[i + (long long)c * m] = (R)v;
        });
    } else {  // ortho: Q1 is used in place; Z is copied
        for_each_entry(n, k, [&](int i, int c) {
            Vcat[i + (long long)c * n] = (R)op.v1[i + (long long)c * op.ldv1];
        });
    }
    __syncthreads();

    // ---- a dense block that is exactly zero ------------------------------
    // (a product of two leaves whose couplings do not meet, as across a gap
    // in the A A of a sparse operator).  Its rounding is known: Jacobi finds
    // nothing to rotate (J = I), every column norm is zero, so the columns
    // keep their order, and the kept columns are U = 0 and V = the unit
    // vectors, with the rank the tolerance rule gives (1 with a tolerance,
    // else the rank cap).  It is written directly.
    if (dense) {
        if (tid == 0) sh.flag = 0;
        __syncthreads();
        for (long long e = tid; e < (long long)m * n; e += kT)
            if (!(Ucat[e] == R(0))) sh.flag = 1;
        __syncthreads();
        const bool zero = sh.flag == 0;
        __syncthreads();
        if (zero) {
            int keep = min(rout, min(m, n));
            if (op.tol > 0.0 && keep > 0) keep = 1;
            if (tid == 0 && op.rank_out) *op.rank_out = keep;
            for_each_entry(m, rout, [&](int i, int c) { op.uo[i + (long long)c * m] = 0.0; });
            for_each_entry(n, rout, [&](int i, int c) {
                op.vo[i + (long long)c * n] = (c < keep && i == c) ? 1.0 : 0.0;
            });
            return;
        }
    }

    // ---- QR of the stacks ------------------------------------------------
    if (!ortho && !skip_u) cta_qr(Ucat, m, k, m, tauU, red);
    if (!dense) cta_qr(Vcat, n, k, n, tauV, red);

    // ---- core M = R_u R_v^T (ku x kv) -------------------------------------
    if (ortho || dense) {
        for_each_entry(ku, kv, [&](int i, int l) {
            R v;
            if (ortho) v = (i >= l) ? Vcat[l + (long long)i * n] : R(0);  // R_v^T
            else if (skip_u) v = Ucat[i + (long long)l * m];                // the block itself
            else v = (l >= i) ? Ucat[i + (long long)l * m] : R(0);          // R_u (ku x n)
            M[i + (long long)l * ku] = v;
        });
    } else {
        // U_cat R_v^T (skip_u) or R_u R_v^T, entry (i, l) summed over p from
        // l (or max(i, l)) to k - 1; 2 x 2 entries a thread, so each loaded
        // factor entry serves several products.  The entries of a tile start
        // at the tile's smallest p, the factors' entries outside their
        // triangles entering as exact zeros, which leaves every sum as it
        // would be alone (0 + 0 x = 0 until its own first term).
        constexpr int TR = 2, TC = 2;
        const int tr = (ku + TR - 1) / TR, tc = (kv + TC - 1) / TC;
        for (int tile = threadIdx.x; tile < tr * tc; tile += kT) {
            const int i0 = TR * (tile % tr), l0 = TC * (tile / tr);
            R acc[TR][TC];
#pragma unroll
            for (int r = 0; r < TR; ++r)
#pragma unroll
                for (int c = 0; c < TC; ++c) acc[r][c] = R(0);
            for (int p = skip_u ? l0 : max(i0, l0); p < k; ++p) {
                R a[TR], b[TC];
#pragma unroll
                for (int r = 0; r < TR; ++r) {
                    const int i = i0 + r;
                    a[r] = (i < ku && (skip_u || p >= i)) ? Ucat[i + (long long)p * m] : R(0);
                }
#pragma unroll
                for (int c = 0; c < TC; ++c) {
                    const int l = l0 + c;
                    b[c] = (l < kv && p >= l) ? Vcat[l + (long long)p * n] : R(0);
                }
#pragma unroll
                for (int r = 0; r < TR; ++r)
#pragma unroll
                    for (int c = 0; c < TC; ++c) acc[r][c] = r_fma(a[r], b[c], acc[r][c]);
            }
#pragma unroll
            for (int r = 0; r < TR; ++r)
#pragma unroll
                for (int c = 0; c < TC; ++c)
                    if (i0 + r < ku && l0 + c < kv) M[i0 + r + (long long)(l0 + c) * ku] = acc[r][c];
        }
    }
    __syncthreads();

    // ---- SVD of the core ---------------------------------------------------
    cta_jacobi(M, ku, kv, J, &sh.flag, red, sh.nrm, numflag);
    cta_order_columns(M, ku, kv, norms, order);

    // ---- outputs -------------------------------------------------------------
    // columns kept: at most rout and the core's size; with a tolerance, the
    // singular values above tol * sigma_0 (norms holds squared values); in
    // FP32 the tolerance is at least the precision's resolvable level
    int keep = min(rout, min(ku, kv));
    if (op.tol > 0.0 && keep > 0) {
        const double s0 = norms[order[0]];
        const double tol = op.tol > Prec<R>::tol_floor ? op.tol : Prec<R>::tol_floor;
        const double t2 = tol * tol;
        // SVDTrunc keeps at least sigma_0: one column when sigma_0 < tol^2
        // (its cutoff index 0), else every sigma above tol * sigma_0
        int c = 1;
        if (s0 >= t2 * t2)
            while (c < keep && (double)norms[order[c]] > t2 * s0) ++c;
        keep = c;
    }
    if (tid == 0 && op.rank_out) *op.rank_out = keep;
    if (ortho) {
        for_each_entry(m, rout, [&](int i, int c) {
            double v = 0.0;
            if (c < keep) {
                const R* g = M + (long long)order[c] * ku;
                for (int p = 0; p < ku; ++p) v = fma(op.u1[i + (long long)p * op.ldu1], (double)g[p], v);
            }
            op.uo[i + (long long)c * m] = v;
        });
    } else {
        for_each_entry(m, rout, [&](int i, int c) {
            op.uo[i + (long long)c * m] =
                (i < ku && c < keep) ? (double)M[i + (long long)order[c] * ku] : 0.0;
        });
    }
    for_each_entry(n, rout, [&](int i, int c) {
        op.vo[i + (long long)c * n] =
            (i < kv && c < keep) ? (double)J[i + (long long)order[c] * kv] : 0.0;
    });
    __syncthreads();
    if (!ortho && !skip_u) cta_apply_q(Ucat, m, min(m, k), m, tauU, op.uo, rout, m);
    if (!dense) cta_apply_q(Vcat, n, min(n, k), n, tauV, op.vo, rout, n);
}

// One CTA per worker; worker w runs ops [begin[w], begin[w+1]) in order (a
// C block's whole operation list, each op reading the previous one's output).
template <typename R>
__global__ void __launch_bounds__(kT, 4)
round_worker_kernel(const RoundOp* __restrict__ ops, const int* __restrict__ begin,
                    const int* __restrict__ workers, long long smem_elems,
                    const RelocBases bases, int* numflag) {
    extern __shared__ __align__(16) unsigned char round_dyn[];
    R* dyn = reinterpret_cast<R*>(round_dyn);
    __shared__ RoundShared<R> sh;
    const int w = workers[blockIdx.x];
    const int b0 = begin[w], b1 = begin[w + 1];
    for (int i = b0; i < b1; ++i) {
        RoundOp op = ops[i];
        op.u1 = reloc(op.u1, bases);
        op.v1 = reloc(op.v1, bases);
        op.u2 = reloc(op.u2, bases);
        op.v2 = reloc(op.v2, bases);
        op.uo = reloc(op.uo, bases);
        op.vo = reloc(op.vo, bases);
        op.work = reloc(op.work, bases);
        op.rank_out = reloc(op.rank_out, bases);
        op.r1_dev = reloc(op.r1_dev, bases);
        op.r2_dev = reloc(op.r2_dev, bases);
        do_round(op, dyn, smem_elems, sh, numflag);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kT) qr_formq_kernel(const QrOp* __restrict__ ops) {
    __shared__ double red[kW + 1];
    const QrOp op = ops[blockIdx.x];
    const int kq = min(op.m, op.k);
    if (op.m == 0 || kq == 0) return;
    cta_qr(op.Y, op.m, op.k, op.ldy, op.tau, red);
    for_each_entry(op.m, kq, [&](int i, int c) { op.Q[i + (long long)c * op.m] = (i == c) ? 1.0 : 0.0; });
    __syncthreads();
    cta_apply_q(op.Y, op.m, kq, op.ldy, op.tau, op.Q, kq, op.m);
}

}  // namespace

long long round_work_size(const RoundOp& op) {
    if (op.kind == ROUND_SET || op.kind == ROUND_CONCAT) return 0;
    const bool ortho = op.kind == ROUND_ORTHO, dense = op.kind == ROUND_DENSE;
    const long long k = dense ? op.n : op.r1 + (op.kind == ROUND_GENERAL ? op.r2 : 0);
    long long w = 0;
    if (!ortho) w += (long long)op.m * k;
    if (!dense) w += (long long)op.n * k;
    w += 2 * k;
    const long long ku = ortho ? op.r1 : std::min<long long>(op.m, k);
    const long long kv = dense ? op.n : std::min<long long>(op.n, k);
    w += ku * kv + kv * kv;   // M, J when they do not fit in shared memory
    return (w + 1) & ~1LL;
}

void launch_round_ops(Context& ctx, std::vector<RoundOp>& ops, const char* name) {
    std::vector<int> begin(ops.size() + 1);
    for (size_t i = 0; i <= ops.size(); ++i) begin[i] = (int)i;
    launch_round_workers(ctx, ops, begin, name);
}


namespace {

template <typename R>
void launch_round_typed(Context& ctx, const RoundList& L, const RelocBases& bases,
                        const char* name) {
    const long long smem = sizeof(R) == 8 ? L.smem_double : L.smem_float;
    {
        // once per device (contexts on several host threads may get here at once)
        int dev = 0;
        cudaGetDevice(&dev);
        static std::mutex mu;
        static std::set<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (done.insert(dev).second)
            HMB_CUDA(cudaFuncSetAttribute(round_worker_kernel<R>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(sizeof(R) == 8 ? kSmemBytes : kSmemBytesF32)));
    }
    LaunchScope ls(ctx, name);
    round_worker_kernel<R><<<(unsigned)L.nw, kT, smem * sizeof(R), ctx.stream>>>(
        L.ops.get(), L.begin.get(), L.workers.get(), smem, bases, ctx.numerical_word());
    HMB_CHECK_LAUNCH();
}

}  // namespace

void upload_round_list(Context& ctx, const std::vector<RoundOp>& ops,
                       const std::vector<int>& begin, RoundList& out) {
    out.nw = 0;
    if (ops.empty() || begin.size() < 2) return;
    // The core and the rotations of an op live in shared memory when they
    // fit the launch's size, otherwise in the (L1-cached) global work area;
    // the size is the largest need of the non-dense ops (dense compressions
    // with larger cores take the global path), so that more CTAs share an SM.
    long long need_max = 0;
    for (const RoundOp& op : ops) {
        if (op.kind == ROUND_SET || op.kind == ROUND_CONCAT) continue;
        const bool dense = op.kind == ROUND_DENSE;
        const long long k = dense ? op.n : op.r1 + (op.kind == ROUND_GENERAL ? op.r2 : 0);
        HMB_REQUIRE(k <= kMaxK, HM_ERR_UNSUPPORTED,
                    "low-rank rounding of more than 128 stacked columns");
        const long long ku = op.kind == ROUND_ORTHO ? op.r1 : std::min<long long>(op.m, k);
        const long long kv = dense ? op.n : std::min<long long>(op.n, k);
        const long long need = ku * kv + kv * kv;
        if (!dense || need <= 3072) need_max = std::max(need_max, need);
    }
    out.smem_double = std::min<long long>(need_max, kSmemBytes / 8);
    out.smem_float = std::min<long long>(need_max, kSmemBytesF32 / 4);
    out.nw = (int)begin.size() - 1;
    std::vector<int> workers(out.nw);
    for (int w = 0; w < out.nw; ++w) workers[w] = w;
    out.ops.upload(ops, ctx.stream);
    out.begin.upload(begin, ctx.stream);
    out.workers.upload(workers, ctx.stream);
}

void launch_round_list(Context& ctx, const RoundList& L, const RelocBases& bases,
                       const char* name) {
    if (L.nw == 0) return;
    if (ctx.low_precision) launch_round_typed<float>(ctx, L, bases, name);
    else launch_round_typed<double>(ctx, L, bases, name);
}

void launch_round_workers(Context& ctx, const std::vector<RoundOp>& ops,
                          const std::vector<int>& begin, const char* name) {
    RoundList L;
    upload_round_list(ctx, ops, begin, L);
    launch_round_list(ctx, L, RelocBases{}, name);
}

void launch_qr_formq(Context& ctx, const std::vector<QrOp>& ops, const char* name) {
    if (ops.empty()) return;
    DeviceBuffer<QrOp> d;
    d.upload(ops, ctx.stream);
    LaunchScope ls(ctx, name);
    qr_formq_kernel<<<(unsigned)ops.size(), kT, 0, ctx.stream>>>(d.get());
    HMB_CHECK_LAUNCH();
}

}  // namespace hmb
