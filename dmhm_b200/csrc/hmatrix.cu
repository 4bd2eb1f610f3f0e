// Device storage of an H-matrix: layout, sparse import, random fill.
//
// Storage: one arena per H-matrix.  Low-rank block b keeps U (m x r) then V
// (n x r), column-major with leading dimensions m and n (A_b = U V^T,
// include/dmhm/core/low_rank.hpp:22-38); dense leaves keep D (m x n).  Blocks
// are laid out in depth-first order so that a subtree's data is contiguous.
#include <climits>
#include <algorithm>

#include <deque>
#include <map>
#include <mutex>
#include <cstring>
#include "engine.h"
#include "rng.cuh"

namespace hmb {

void HMatrix::layout() {
    const Structure& St = *S;
    group.reset();
    shadow_valid = false;
    off.assign(St.blocks.size(), -1);
    long long cur = 0;
    for (int b : St.leaves) {
        const Block& B = St.blocks[b];
        off[b] = cur;
        if (B.kind == KIND_DENSE)
            cur += (long long)B.m * B.n;
        else
            cur += (long long)(B.m + B.n) * rank[b];
        cur = (cur + 1) & ~1LL;   // 16-byte alignment of every block
    }
    total = cur;
    data.allocate((size_t)std::max<long long>(total, 2), ctx->stream);
    upload_table();
}

void HMatrix::upload_table() {
    const Structure& St = *S;
    std::vector<DevBlock> t(St.blocks.size());
    long long before = 0;
    for (size_t b = 0; b < St.blocks.size(); ++b) {
        const Block& B = St.blocks[b];
        DevBlock d{};
        d.kind = B.kind;
        d.m = B.m;
        d.n = B.n;
        d.rank = B.kind == KIND_LOWRANK ? rank[b] : 0;
        d.row_off = B.row_off;
        d.col_off = B.col_off;
        d.rank_before = (int)std::min<long long>(before, INT_MAX);
        d.off = off[b];
        before += d.rank;
        t[b] = d;
    }
    table.upload(t, ctx->stream);
}

namespace {

// Pinned staging ring of one stream: copies take [head, head + bytes) and
// record an event after their cudaMemcpyAsync; before a range of the ring is
// written again, the host waits for the events of the copies that read it
// (normally long done), never for the whole stream.
struct StagedCopy {
    size_t begin, end;
    cudaEvent_t done;
};
struct StagingRing {
    char* buf = nullptr;
    size_t cap = 0, head = 0;
    std::deque<StagedCopy> pending;   // in ring order
    std::vector<cudaEvent_t> spare;
};
constexpr size_t kStagingBytes = size_t(128) << 20;
std::mutex g_staging_mu;
std::map<cudaStream_t, StagingRing> g_staging;

void retire_front(StagingRing& R) {
    HMB_CUDA(cudaEventSynchronize(R.pending.front().done));
    R.spare.push_back(R.pending.front().done);
    R.pending.pop_front();
}

}  // namespace

void staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return;
    if (bytes > kStagingBytes / 4) {
        HMB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    std::lock_guard<std::mutex> lock(g_staging_mu);
    StagingRing& R = g_staging[s];
    if (!R.buf) {
        if (cudaMallocHost((void**)&R.buf, kStagingBytes) != cudaSuccess) {
            R.buf = nullptr;
            cudaGetLastError();
            HMB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
            return;
        }
        R.cap = kStagingBytes;
    }
    const size_t need = (bytes + 255) & ~size_t(255);
    if (R.head + need > R.cap) {
        // the tail [head, cap) is skipped this lap: copies of earlier laps
        // still pending there are the oldest and are retired first
        while (!R.pending.empty() && R.pending.front().begin >= R.head) retire_front(R);
        R.head = 0;
    }
    // copies of the previous lap that read the range about to be written
    while (!R.pending.empty() && R.pending.front().begin < R.head + need &&
           R.pending.front().end > R.head)
        retire_front(R);
    char* p = R.buf + R.head;
    std::memcpy(p, src, bytes);
    HMB_CUDA(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, s));
    cudaEvent_t ev;
    if (!R.spare.empty()) {
        ev = R.spare.back();
        R.spare.pop_back();
    } else {
        HMB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    HMB_CUDA(cudaEventRecord(ev, s));
    R.pending.push_back({R.head, R.head + need, ev});
    R.head += need;
    // retire copies that are already done (keeps the pending list short)
    for (int i = 0; i < 8 && R.pending.size() > 1; ++i) {
        const cudaError_t q = cudaEventQuery(R.pending.front().done);
        if (q == cudaErrorNotReady) break;
        HMB_CUDA(q);
        R.spare.push_back(R.pending.front().done);
        R.pending.pop_front();
    }
}

// Drops the staging ring of a stream that is about to be destroyed.
void release_staging(cudaStream_t s) {
    std::lock_guard<std::mutex> lock(g_staging_mu);
    auto it = g_staging.find(s);
    if (it == g_staging.end()) return;
    cudaStreamSynchronize(s);
    for (const StagedCopy& c : it->second.pending) cudaEventDestroy(c.done);
    for (cudaEvent_t e : it->second.spare) cudaEventDestroy(e);
    if (it->second.buf) cudaFreeHost(it->second.buf);
    g_staging.erase(it);
}

namespace {

struct FillTask {
    double* dst;
    const double* old;         // previous buffer contents (may be null)
    unsigned long long base;   // LCG state at the task's first draw
    long long old_count;       // entries of `old` still in the buffer
    int m, n;
};

// Gaussian fill; entries the reference's fill does not write keep the old
// buffer value (Dense::Resize keeps its std::vector, new entries are zero).
__global__ void fill_gaussian_kernel(const FillTask* __restrict__ tasks) {
    const FillTask t = tasks[blockIdx.x];
    const long long total = (long long)t.m * t.n;
    const int pairs = (t.m + 1) / 2;
    for (long long e = threadIdx.x; e < total; e += blockDim.x) {
        int i = (int)(e % t.m), j = (int)(e / t.m);
        bool written = (i < 2 * (pairs - 1)) || ((t.m & 1) ? i == t.n - 1
                                                           : (i == t.n - 2 || i == t.n - 1));
        double v;
        if (written)
            v = gaussian_fill_entry(t.base, t.m, t.n, i, j);
        else
            v = (t.old != nullptr && e < t.old_count) ? t.old[e] : 0.0;
        t.dst[e] = v;
    }
}

inline unsigned long long fill_draws(int m, int n) {
    return (unsigned long long)n * 2ULL * (unsigned long long)((m + 1) / 2);
}

}  // namespace

// SetToRandom (src/HMat2d/SetToRandom-incl.hpp:14-55): depth-first over the
// leaves, dense m x n fills, low-rank U (m x maxRank) then V (n x maxRank),
// all from the parallel stream.
void launch_fill_random(Context& ctx, HMatrix& H) {
    const Structure& St = *H.S;
    for (int b : St.leaves) {
        const Block& B = St.blocks[b];
        if (B.kind == KIND_DENSE)
            HMB_REQUIRE(B.n <= B.m || B.m == 0, HM_ERR_UNSUPPORTED,
                        "random fill of a dense block wider than tall");
        else
            HMB_REQUIRE((H.max_rank <= B.m || B.m == 0) && (H.max_rank <= B.n || B.n == 0),
                        HM_ERR_UNSUPPORTED, "random fill with max rank above the block size");
    }
    // keep the old storage alive until the fill has read it
    DeviceBuffer<double> old_data(std::move(H.data));
    std::vector<long long> old_off = H.off;
    std::vector<int> old_rank = H.rank;
    for (int b : St.leaves)
        if (St.blocks[b].kind == KIND_LOWRANK) H.rank[b] = H.max_rank;
    H.layout();
    std::vector<FillTask> tasks;
    uint64_t state = ctx.parallel_state;
    const double* od = old_data.get();
    for (int b : St.leaves) {
        const Block& B = St.blocks[b];
        if (B.kind == KIND_DENSE) {
            tasks.push_back({H.D(b), od + old_off[b], state, (long long)B.m * B.n, B.m, B.n});
            state = lcg_skip_host(state, fill_draws(B.m, B.n));
        } else {
            int r = H.max_rank, ro = old_rank[b];
            tasks.push_back({H.U(b), od + old_off[b], state, (long long)B.m * ro, B.m, r});
            state = lcg_skip_host(state, fill_draws(B.m, r));
            tasks.push_back({H.V(b), od + old_off[b] + (long long)B.m * ro, state,
                             (long long)B.n * ro, B.n, r});
            state = lcg_skip_host(state, fill_draws(B.n, r));
        }
    }
    ctx.parallel_state = state;
    tasks.erase(std::remove_if(tasks.begin(), tasks.end(),
                               [](const FillTask& t) { return t.m == 0 || t.n == 0; }),
                tasks.end());
    if (tasks.empty()) return;
    DeviceBuffer<FillTask> d;
    d.upload(tasks, ctx.stream);
    LaunchScope ls(ctx, "fill_gaussian");
    fill_gaussian_kernel<<<(unsigned)tasks.size(), 256, 0, ctx.stream>>>(d.get());
    HMB_CHECK_LAUNCH();
}

void launch_gaussian_fills(Context& ctx, const std::vector<FillOp>& fills, const char* name) {
    std::vector<FillTask> tasks;
    for (const FillOp& f : fills) {
        if (f.m == 0 || f.n == 0) continue;
        HMB_REQUIRE(f.n <= f.m, HM_ERR_UNSUPPORTED,
                    "Gaussian fill wider than tall (the reference would write past its columns)");
        tasks.push_back({f.dst, nullptr, f.base, 0, f.m, f.n});
    }
    if (tasks.empty()) return;
    DeviceBuffer<FillTask> d;
    d.upload(tasks, ctx.stream);
    LaunchScope ls(ctx, name);
    fill_gaussian_kernel<<<(unsigned)tasks.size(), 256, 0, ctx.stream>>>(d.get());
    HMB_CHECK_LAUNCH();
}

}  // namespace hmb
