// Mixed-precision H-matrix x dense product on the 5th-generation tensor cores.
//
// The FP64 product (matmul.cu, the reference's HMat2d::Multiply against a
// Dense block, src/HMat2d/MultiplyDense-incl.hpp:12-68) is bound by FP64 FMA
// throughput when many right-hand sides share each block.  Here the block
// data are read from an FP32 copy (rounded to TF32) and every block product
// runs as tcgen05.mma kind::tf32 with FP32 accumulation in tensor memory:
//   phase 1, one CTA per low-rank block b:  T_b^T (k x r) = X_b^T V_b,
//   phase 2, one CTA per output row tile:   Y_tile^T (k x rows) =
//            sum_e A_e^T B_e^T over the tile's dense leaves (X rows, D rows)
//            and low-rank blocks (T_b, U_b rows),
// with the right-hand sides as the MMA's M dimension (M = 64), the tile rows
// or the rank as N, and the block's inner dimension as K.  Both operands are
// staged in shared memory in the canonical no-swizzle K-major layout (core
// matrices of 8 rows x 16 bytes); one thread issues the MMAs and
// commits them to an mbarrier; every wait on it is bounded and reports
// through an error word instead of hanging.
//
// Work lists come from the FP64 path's per-subtree templates; FP64 pointers
// are translated to the FP32 copy by their offset in the H-matrix storage.
#include <cuda_runtime.h>

#include <utility>

#include "engine.h"
#include "templates.h"

namespace hmb {

namespace {

constexpr int kTcThreads = 128;
constexpr int kM = 64;          // right-hand sides per MMA tile
constexpr int kKC = 32;         // K elements staged per round
constexpr long long kWaitLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
}

// Bounded wait for the given phase parity; false (and err set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          long long limit = kWaitLimit) {
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity));
        if (done) return true;
    }
    atomicExch(err, 1);
    return false;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100; no swizzle
    return d;
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, majors, N, M.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn_major << 15) |
           ((uint32_t)b_mn_major << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(bar)));
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Canonical no-swizzle shared-memory layouts (byte offsets).
// K-major (rows x KC): core matrices of 8 rows x 16 B; K-direction step 128 B,
// row-group step (KC/4)*128 B.
__device__ __forceinline__ int kmaj_off(int r, int k) {
    return (r >> 3) * ((kKC / 4) * 128) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}
struct TcArgs {
    const double* base64;    // H-matrix FP64 storage
    const float* base32;     // its TF32-rounded FP32 copy
    const float* X;          // input, FP32, column-major (n x k, ld ldx)
    float* T;                // phase-1 results T_b^T, k x r each (ld r)
    double* Y;               // output, FP64 (ld ldy)
    int* err;
    const P1T* p1;
    const P2T* p2;
    const P2Entry* ent;
    double alpha, beta;
    int ldx, ldy, k;
};


// ---------------------------------------------------------------------------
// Phase 1: T_b^T (k x r) = X_b^T (k x n) * V_b (n x r), one CTA per block.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTcThreads) tc_lowrank_inner_kernel(const TcArgs a) {
    __shared__ __align__(128) float sA[kM * kKC];
    __shared__ __align__(128) float sB[256 * kKC];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const P1T it = a.p1[blockIdx.x];
    const int r = it.r, n = it.nin;
    const int N = ((r + 7) / 8) * 8;           // MMA N (multiple of 8, <= 256)
    int cols = 32;
    while (cols < N) cols <<= 1;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const float* X = a.X + it.in_off;
    const float* V = a.base32 + it.w;
    const uint32_t idesc = idesc_tf32(kM, N, 0, 0);
    uint32_t phase = 0;
    bool ok = true;
    const int kpad = ((n + 7) / 8) * 8;
    for (int k0 = 0; k0 < kpad && ok; k0 += kKC) {
        const int kc = min(kKC, kpad - k0);
        // A: X^T rows j (rhs), K = matrix rows i
        for (int e = threadIdx.x; e < kM * kKC; e += kTcThreads) {
            const int j = e / kKC, kk = e % kKC;
            const int i = k0 + kk;
            float v = 0.f;
            if (j < a.k && i < n && kk < kc) v = X[i + (long long)j * a.ldx];
            sA[kmaj_off(j, kk) >> 2] = v;
        }
        // B: V^T rows l (rank), K = matrix rows i
        for (int e = threadIdx.x; e < N * kKC; e += kTcThreads) {
            const int l = e / kKC, kk = e % kKC;
            const int i = k0 + kk;
            float v = 0.f;
            if (l < r && i < n && kk < kc) v = V[i + (long long)l * it.ldw];
            sB[kmaj_off(l, kk) >> 2] = v;
        }
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int s = 0; s < kc / 8; ++s) {
                const uint64_t ad = smem_desc(a0 + s * 256, 128, (kKC / 4) * 128);
                const uint64_t bd = smem_desc(b0 + s * 256, 128, (kKC / 4) * 128);
                mma_tf32(tmem, ad, bd, idesc, (k0 > 0 || s > 0) ? 1u : 0u);
            }
            mma_commit(&bar);
        }
        ok = mbar_wait(&bar, phase, a.err);
        if (!ok) mbar_wait(&bar, phase, a.err);   // let in-flight MMAs drain
        phase ^= 1;
        tc_fence_after();
        ok = __syncthreads_and(ok);               // uniform across the CTA
    }
    // epilogue: M = 64 layout, rhs j = 16*warp + lane (lanes 0..15 of each warp)
    const int lane = threadIdx.x & 31;
    const int j = 16 * warp + lane;
    float* T = a.T + it.t_rel * a.k;
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + c0, v);
            if (lane < 16 && j < a.k)
                for (int c = 0; c < 16; ++c)
                    if (c0 + c < r) T[(c0 + c) + (long long)j * r] = kpad > 0 ? v[c] : 0.f;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

// ---------------------------------------------------------------------------
// Phase 2: Y_tile^T (k x rows) = sum_e A_e^T B_e^T, one CTA per row tile.
// ---------------------------------------------------------------------------
// Each template row tile (<= 64 rows) is split over gridDim.y CTAs of
// kTileRows rows: more CTAs in flight per SM, the small A operands (T_b, X
// rows) re-read from L2.
constexpr int kTileRows = 16;

__global__ void __launch_bounds__(kTcThreads) tc_row_tiles_kernel(const TcArgs a) {
    constexpr int N = kTileRows;               // MMA N: tile rows (zero-padded)
    constexpr int kCols = 32;                  // TMEM columns allocated (minimum 32)
    __shared__ __align__(128) float sA[kM * kKC];
    __shared__ __align__(128) float sB[N * kKC];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    P2T it = a.p2[blockIdx.x];
    it.r0 += kTileRows * blockIdx.y;
    it.rows = min(kTileRows, it.rows - kTileRows * (int)blockIdx.y);
    if (it.rows <= 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = idesc_tf32(kM, N, 0, 0);
    uint32_t phase = 0;
    bool ok = true, any = false;
    for (int ei = it.e0; ei < it.e1 && ok; ++ei) {
        const P2Entry e = a.ent[ei];
        const float* Bsrc = a.base32 + e.a;    // rows of U or D (staged K-major)
        const float* Asrc;                     // T_b^T or X rows
        int lda_src;
        if (e.b_from_t) { Asrc = a.T + e.b_off * a.k; lda_src = e.ldt; }
        else { Asrc = a.X + e.b_off; lda_src = a.ldx; }
        const int inner = e.inner;
        const int kpad = ((inner + 7) / 8) * 8;
        for (int k0 = 0; k0 < kpad && ok; k0 += kKC) {
            const int kc = min(kKC, kpad - k0);
            for (int x = threadIdx.x; x < kM * kKC; x += kTcThreads) {
                const int j = x / kKC, kk = x % kKC;
                const int p = k0 + kk;
                float v = 0.f;
                if (j < a.k && p < inner && kk < kc) v = Asrc[p + (long long)j * lda_src];
                sA[kmaj_off(j, kk) >> 2] = v;
            }
            for (int x = threadIdx.x; x < N * kKC; x += kTcThreads) {
                const int i = x % N, kk = x / N;
                const int p = k0 + kk;
                float v = 0.f;
                if (i < it.rows && p < inner && kk < kc)
                    v = Bsrc[(it.r0 + i) + (long long)p * e.lda];
                sB[kmaj_off(i, kk) >> 2] = v;
            }
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
                for (int s = 0; s < kc / 8; ++s) {
                    const uint64_t ad = smem_desc(a0 + s * 256, 128, (kKC / 4) * 128);
                    const uint64_t bd = smem_desc(b0 + s * 256, 128, (kKC / 4) * 128);
                    mma_tf32(tmem, ad, bd, idesc, (any || s > 0) ? 1u : 0u);
                }
                mma_commit(&bar);
            }
            any = true;
            ok = mbar_wait(&bar, phase, a.err);
            if (!ok) mbar_wait(&bar, phase, a.err);   // let in-flight MMAs drain
            phase ^= 1;
            tc_fence_after();
            ok = __syncthreads_and(ok);               // uniform across the CTA
        }
    }
    const int j = 16 * warp + lane;
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + c0, v);
            if (lane < 16 && j < a.k)
                for (int c = 0; c < 16; ++c) {
                    const int i = c0 + c;
                    if (i >= it.rows) continue;
                    double* y = a.Y + it.out_off + it.r0 + i + (long long)j * a.ldy;
                    const double acc = any ? (double)v[c] : 0.0;
                    *y = a.beta == 0.0 ? a.alpha * acc : a.alpha * acc + a.beta * *y;
                }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kCols));
}

__global__ void to_tf32_kernel(const double* __restrict__ src, float* __restrict__ dst,
                               long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = to_tf32((float)src[i]);
}

// X (n x k, ld ldx, FP64) -> Xf (n x k, ld n, FP32 rounded to TF32)
__global__ void input_tf32_kernel(const double* __restrict__ X, int ldx, float* __restrict__ Xf,
                                  int n, int k) {
    const long long total = (long long)n * k;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        Xf[e] = to_tf32((float)X[i + (long long)j * ldx]);
    }
}

// Check of the bounded wait itself: one warp initialises an mbarrier that
// expects one arrival, never arrives, and waits for it with a short limit.
// The wait gives up, records the timeout in *err and the kernel returns.
__global__ void bounded_wait_probe_kernel(long long limit, int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    mbar_wait(&bar, 0, err, limit);
}

}  // namespace

// Runs the bounded-wait check on `device` (its own stream and flag); returns
// whether the wait ran out, as it must.
bool bounded_wait_times_out(int device, long long limit) {
    HMB_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    HMB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int* d_err = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d_err, sizeof(int), s);
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        g_launches.fetch_add(1, std::memory_order_relaxed);
        bounded_wait_probe_kernel<<<1, 32, 0, s>>>(limit, d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (d_err) cudaFreeAsync(d_err, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    HMB_CUDA(e);
    HMB_CUDA(e2);
    return h_err != 0;
}

// FP32 (TF32-rounded) copy of the block data, made on first use.
void ensure_tf32_copy(Context& ctx, HMatrix& H) {
    if (H.shadow_valid && H.data32.size() >= (size_t)std::max<long long>(H.total, 1)) return;
    H.data32.allocate((size_t)std::max<long long>(H.total, 1), ctx.stream);
    if (H.total > 0) {
        LaunchScope ls(ctx, "to_tf32");
        to_tf32_kernel<<<4 * ctx.num_sms, 256, 0, ctx.stream>>>(H.data.get(), H.data32.get(),
                                                                H.total);
        HMB_CHECK_LAUNCH();
    }
    H.shadow_valid = true;
}

namespace {

// The tcgen05 form: nrhs <= 64, ranks <= 256; synchronizes.
void dense_tf32_tc(Context& ctx, HMatrix& H, double alpha, const double* B, int ldb, double beta,
                   double* Cout, int ldc, int nrhs) {
    ensure_tf32_copy(ctx, H);
    auto T = get_template(ctx, H, 0, false);
    const int n = H.width();
    cudaStream_t st = ctx.stream;
    DeviceBuffer<float> Xf, Tbuf;
    DeviceBuffer<int> err;
    Xf.allocate((size_t)n * nrhs, st);
    Tbuf.allocate((size_t)std::max<long long>(T->t_rows * nrhs, 1), st);
    err.allocate(1, st);
    HMB_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    {
        LaunchScope ls(ctx, "input_tf32");
        input_tf32_kernel<<<4 * ctx.num_sms, 256, 0, st>>>(B, ldb, Xf.get(), n, nrhs);
        HMB_CHECK_LAUNCH();
    }
    TcArgs a{};
    a.base64 = H.data.get();
    a.base32 = H.data32.get();
    a.X = Xf.get();
    a.T = Tbuf.get();
    a.Y = Cout;
    a.err = err.get();
    a.p1 = T->p1.get();
    a.p2 = T->p2.get();
    a.ent = T->ent.get();
    a.alpha = alpha;
    a.beta = beta;
    a.ldx = n;
    a.ldy = ldc;
    a.k = nrhs;
    if (T->n1 > 0) {
        LaunchScope ls(ctx, "tc_lowrank_inner");
        tc_lowrank_inner_kernel<<<T->n1, kTcThreads, 0, st>>>(a);
        HMB_CHECK_LAUNCH();
    }
    if (T->n2 > 0) {
        LaunchScope ls(ctx, "tc_row_tiles");
        tc_row_tiles_kernel<<<dim3(T->n2, 64 / kTileRows), kTcThreads, 0, st>>>(a);
        HMB_CHECK_LAUNCH();
    }
    int h_err = 0;
    HMB_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    HMB_CUDA(cudaStreamSynchronize(st));
    HMB_REQUIRE(h_err == 0, HM_ERR_TIMEOUT, "a tensor-core wait ran out (no progress)");
}

// The mma.sync form: persistent 64 x 64 tiles over all right-hand sides.
void dense_tf32_mma(Context& ctx, HMatrix& H, double alpha, const double* B, int ldb, double beta,
                    double* Cout, int ldc, int nrhs) {
    if (nrhs <= 8) {   // below the tile width the FP64 kernels are bandwidth-bound anyway
        run_jobs(ctx, {MatJob{&H, 0, false, alpha, beta, B, ldb, Cout, ldc, nrhs}});
    } else {
        run_jobs(ctx, {MatJob{&H, 0, false, alpha, beta, B, ldb, Cout, ldc, nrhs}}, true);
    }
    HMB_CUDA(cudaStreamSynchronize(ctx.stream));
}

// Right-hand-side bucket of the tuning table: 16, 32, 64, 128, ...
int rhs_bucket(int nrhs) {
    int b = 16;
    while (b < nrhs) b *= 2;
    return b;
}

// Times both forms on the matrix into a scratch output (beta = 0, three
// runs each after one untimed run) and returns the faster (1 tcgen05,
// 2 mma.sync).
int tune_tf32(Context& ctx, HMatrix& H, const double* B, int ldb, int nrhs) {
    HostScope hs(ctx, "tf32_autotune");
    const int m = H.height();
    DeviceBuffer<double> scratch;
    scratch.allocate((size_t)std::max(m, 1) * nrhs, ctx.stream);
    cudaEvent_t e0, e1;
    HMB_CUDA(cudaEventCreate(&e0));
    HMB_CUDA(cudaEventCreate(&e1));
    float best_ms = 0.0f;
    int best = 2;
    for (int which = 1; which <= 2; ++which) {
        auto run = [&] {
            if (which == 1) dense_tf32_tc(ctx, H, 1.0, B, ldb, 0.0, scratch.get(), std::max(m, 1), nrhs);
            else dense_tf32_mma(ctx, H, 1.0, B, ldb, 0.0, scratch.get(), std::max(m, 1), nrhs);
        };
        run();
        HMB_CUDA(cudaEventRecord(e0, ctx.stream));
        for (int r = 0; r < 3; ++r) run();
        HMB_CUDA(cudaEventRecord(e1, ctx.stream));
        HMB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        HMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (which == 1 || ms < best_ms) {
            best_ms = ms;
            best = which;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

int tf32_kernel_choice(Context& ctx, HMatrix& H, const double* B, int ldb, int nrhs) {
    bool tc_ok = nrhs <= kM;
    for (size_t b = 0; tc_ok && b < H.S->blocks.size(); ++b)
        tc_ok = H.S->blocks[b].kind != KIND_LOWRANK || H.rank[b] <= 256;
    if (!tc_ok) return 2;
    if (ctx.tf32_kernel != 0) return ctx.tf32_kernel;
    get_template(ctx, H, 0, false);   // makes H.group
    const auto key = std::make_pair(H.group->hash, rhs_bucket(nrhs));
    auto f = ctx.tf32_tuned.find(key);
    if (f != ctx.tf32_tuned.end()) return f->second;
    const int w = tune_tf32(ctx, H, B, ldb, nrhs);
    ctx.tf32_tuned[key] = w;
    return w;
}

void multiply_dense_tf32(HMatrix& H, double alpha, const double* B, int ldb, double beta,
                         double* Cout, int ldc, int nrhs) {
    Context& ctx = *H.ctx;
    HMB_REQUIRE(nrhs >= 0, HM_ERR_ARGUMENT, "nrhs must be >= 0");
    HMB_REQUIRE(ldb >= std::max(1, H.width()) && ldc >= std::max(1, H.height()), HM_ERR_ARGUMENT,
                "leading dimension too small");
    if (nrhs == 0 || H.height() == 0) return;
    const int which = tf32_kernel_choice(ctx, H, B, ldb, nrhs);
    if (which == 1) {
        HMB_REQUIRE(nrhs <= kM, HM_ERR_UNSUPPORTED,
                    "the tcgen05 product handles at most 64 right-hand sides per call");
        dense_tf32_tc(ctx, H, alpha, B, ldb, beta, Cout, ldc, nrhs);
    } else {
        dense_tf32_mma(ctx, H, alpha, B, ldb, beta, Cout, ldc, nrhs);
    }
}

}  // namespace hmb
