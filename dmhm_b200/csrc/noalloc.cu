// H-matrix x vector that allocates no device memory.
//
// Some callers cannot allocate device memory while they run: applications
// whose own memory manager has already reserved the GPU's memory, and
// time-critical loops where an allocator call may block or fail.
// hm_multiply_vector_noalloc serves them.  It computes the same product as
// hm_multiply_dense with one right-hand side, but keeps its intermediate
// values (the per-block inner products V^T x, placed by the rank offsets
// that the matrix's block table carries) in one statically allocated
// device array of this library instead of allocating per call.  Dense leaves and low-rank blocks are processed one
// CTA per block, and each block adds its contribution to the output with
// atomic additions, so the summation order may differ from
// hm_multiply_dense in the last bits.
//
// The array holds kNoAllocScratchDoubles doubles (4 MiB); every GPU that
// loads the library holds it until the process exits.  A matrix needs
// (sum of the low-rank ranks) entries; larger matrices are rejected with
// HM_ERR_UNSUPPORTED.  All calls share the array and the
// array keeps whatever the last call left in it, so calls that overlap on
// the GPU (on different streams, or from different host threads without
// ordering) race on it and must not be issued.
#include <mutex>

#include "engine.h"

namespace hmb {

namespace {

constexpr long long kNoAllocScratchDoubles = 1LL << 19;   // 4 MiB
constexpr int kT = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch, looked up once per device.
double* scratch_address(int device) {
    static std::mutex mu;
    static double* addr[kMaxDevices] = {nullptr};
    HMB_REQUIRE(device >= 0 && device < kMaxDevices, HM_ERR_ARGUMENT, "device index too large");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        int cur = -1;
        HMB_CUDA(cudaGetDevice(&cur));
        HMB_REQUIRE(cur == device, HM_ERR_INTERNAL, "scratch set-up with the wrong device current");
        void* p = nullptr;
        HMB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[device] = static_cast<double*>(p);
    }
    return addr[device];
}

__global__ void noalloc_scale_kernel(double* y, int n, double beta) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = beta == 0.0 ? 0.0 : beta * y[i];
}

// t_b = W_b^T x for every low-rank block (W = V, or U for the transpose).
__global__ void noalloc_inner_kernel(const DevBlock* __restrict__ table, int nblocks,
                                     const double* __restrict__ data,
                                     const double* __restrict__ x, double* scratch, int trans) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* T = scratch;
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const DevBlock B = table[b];
        if (B.kind != KIND_LOWRANK || B.rank == 0 || B.m == 0 || B.n == 0) continue;
        const long long t0 = B.rank_before;
        const int nin = trans ? B.m : B.n;
        const double* W = data + B.off + (trans ? 0LL : (long long)B.m * B.rank);
        const double* xs = x + (trans ? B.row_off : B.col_off);
        for (int l = warp; l < B.rank; l += kT / 32) {
            const double* w = W + (long long)l * nin;
            double s = 0.0;
            for (int i = lane; i < nin; i += 32) s = fma(w[i], xs[i], s);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) T[t0 + l] = s;
        }
    }
}

// y += alpha * (D x or U t) for every leaf block (transposed roles for the
// transpose product), accumulated with atomic additions.
__global__ void noalloc_outer_kernel(const DevBlock* __restrict__ table, int nblocks,
                                     const double* __restrict__ data,
                                     const double* __restrict__ x, const double* scratch,
                                     double* y, double alpha, int trans) {
    const double* T = scratch;
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const DevBlock B = table[b];
        if (B.kind == KIND_NODE || B.m == 0 || B.n == 0) continue;
        const int nout = trans ? B.n : B.m;
        double* ys = y + (trans ? B.col_off : B.row_off);
        if (B.kind == KIND_DENSE) {
            const double* D = data + B.off;
            const double* xs = x + (trans ? B.row_off : B.col_off);
            const int nin = trans ? B.m : B.n;
            if (!trans) {
                // row i of D: neighbouring threads read neighbouring rows
                for (int i = threadIdx.x; i < nout; i += kT) {
                    double s = 0.0;
                    for (int j = 0; j < nin; ++j) s = fma(D[i + (long long)j * B.m], xs[j], s);
                    atomicAdd(ys + i, alpha * s);
                }
            } else {
                // column i of D: one warp, lanes along the column
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                for (int i = warp; i < nout; i += kT / 32) {
                    const double* col = D + (long long)i * B.m;
                    double s = 0.0;
                    for (int j = lane; j < nin; j += 32) s = fma(col[j], xs[j], s);
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (lane == 0) atomicAdd(ys + i, alpha * s);
                }
            }
        } else if (B.rank > 0) {
            const long long t0 = B.rank_before;
            const double* W = data + B.off + (trans ? (long long)B.m * B.rank : 0LL);
            for (int i = threadIdx.x; i < nout; i += kT) {
                double s = 0.0;
                for (int l = 0; l < B.rank; ++l) s = fma(W[i + (long long)l * nout], T[t0 + l], s);
                atomicAdd(ys + i, alpha * s);
            }
        }
    }
}

}  // namespace

void multiply_vector_noalloc(HMatrix& H, int transpose, double alpha, const double* x,
                             double beta, double* y) {
    Context& ctx = *H.ctx;
    const Structure& S = *H.S;
    const int nblocks = (int)S.blocks.size();
    long long rank_sum = 0;
    for (int b : S.leaves)
        if (S.blocks[b].kind == KIND_LOWRANK) rank_sum += H.rank[b];
    const long long need = rank_sum;
    HMB_REQUIRE(need <= kNoAllocScratchDoubles, HM_ERR_UNSUPPORTED,
                "hm_multiply_vector_noalloc: the matrix needs " + std::to_string(need) +
                    " scratch entries (the sum of its low-rank ranks); the static scratch holds " +
                    std::to_string(kNoAllocScratchDoubles));
    HMB_REQUIRE(x != nullptr && y != nullptr, HM_ERR_ARGUMENT, "NULL vector");
    HMB_CUDA(cudaSetDevice(ctx.device));
    double* scratch = scratch_address(ctx.device);
    const int n_out = transpose ? H.width() : H.height();
    const int grid = std::max(1, std::min(nblocks, 8 * ctx.num_sms));
    cudaStream_t st = ctx.stream;
    g_launches.fetch_add(3, std::memory_order_relaxed);
    noalloc_scale_kernel<<<std::max(1, std::min(ceil_div(n_out, kT), 4 * ctx.num_sms)), kT, 0,
                           st>>>(y, n_out, beta);
    noalloc_inner_kernel<<<grid, kT, 0, st>>>(H.table.get(), nblocks, H.data.get(), x, scratch,
                                              transpose);
    noalloc_outer_kernel<<<grid, kT, 0, st>>>(H.table.get(), nblocks, H.data.get(), x, scratch,
                                              y, alpha, transpose);
    HMB_CHECK_LAUNCH();
}

}  // namespace hmb
