// C ABI (include/dmhm_b200.h): argument checks, error capture, and the host
// side of each entry point.
#include <algorithm>
#include <cstring>
#include <set>
#include <string>

#include "engine.h"
#include "mlp.h"
#include "hh.h"
#include "rng.cuh"
#include "schulz.h"

struct hm_matrix_s;

struct hm_context_s {
    hmb::Context c;
    std::set<hm_matrix_s*> live;   // handles created on this context
    std::set<struct hm_rank_model_s*> models;
};

struct hm_matrix_s {
    hmb::HMatrix h;
    hm_context_s* owner = nullptr;
};

struct hm_rank_model_s {
    hmb::RankModel m;
    hm_context_s* owner = nullptr;
};

namespace {

hm_matrix_s* new_handle(hm_context_s* ctx) {
    auto* m = new hm_matrix_s;
    m->owner = ctx;
    m->h.ctx = &ctx->c;
    ctx->live.insert(m);
    return m;
}

// Releases the device storage of a handle (stream-ordered frees).
void release_storage(hm_matrix_s* m) {
    m->h.group.reset();
    m->h.data32.reset();
    m->h.data.reset();
    m->h.table.reset();
}

void delete_handle(hm_matrix_s* m) {
    if (m->owner) {
        m->owner->live.erase(m);
        release_storage(m);
    }
    delete m;
}

hm_context_s* owner_of(hm_matrix_s* m) {
    HMB_REQUIRE(m->owner != nullptr, HM_ERR_ARGUMENT,
                "the H-matrix's context was destroyed");
    return m->owner;
}

}  // namespace

namespace hmb {

namespace {
thread_local std::string g_last_error;
}

std::atomic<unsigned long long> g_launches{0};

void set_last_error(const std::string& msg) { g_last_error = msg; }

void Context::collect() {
    HMB_CUDA(cudaStreamSynchronize(stream));
    for (auto& p : pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        Totals& t = totals[p.name];
        t.ms += ms;
        t.launches += 1;
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pending.clear();
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return HM_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return HM_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return HM_ERR_INTERNAL;
    }
}

// Host-side import of a CSR matrix in hierarchical order
// (ImportSparse, src/HMat2d/HMat2d.cpp:961-1033; ConvertSubmatrix,
// src/hmat_tools/ConvertSubmatrix.cpp:14-119): dense leaves copy their
// entries; an admissible block gets one rank-1 term per nonzero it holds,
// U = unit column, V = value column.
void import_csr(HMatrix& H, const int64_t* rows, const int32_t* cols,
                const double* vals) {
    const Structure& S = *H.S;
    H.rank.assign(S.blocks.size(), 0);
    // count nonzeros per admissible block
    std::vector<std::vector<std::pair<int, int>>> lr_entries(S.blocks.size());
    auto find_leaf = [&](int i, int j) {
        int b = 0;
        while (S.blocks[b].kind == KIND_NODE) {
            const Block& B = S.blocks[b];
            int t = 0, s = 0;
            const Box& TB = S.boxes[B.tgt_box];
            const Box& SB = S.boxes[B.src_box];
            for (int c = 0; c < S.q; ++c) {
                const Box& cb = S.boxes[TB.first_child + c];
                if (i >= cb.offset && i < cb.offset + cb.count) { t = c; break; }
            }
            for (int c = 0; c < S.q; ++c) {
                const Box& cb = S.boxes[SB.first_child + c];
                if (j >= cb.offset && j < cb.offset + cb.count) { s = c; break; }
            }
            b = S.child(b, t, s);
        }
        return b;
    };
    const int N = S.N;
    std::vector<int> leaf_of_entry;
    leaf_of_entry.reserve((size_t)rows[N]);
    for (int i = 0; i < N; ++i)
        for (int64_t k = rows[i]; k < rows[i + 1]; ++k) {
            int j = cols[k];
            HMB_REQUIRE(j >= 0 && j < N, HM_ERR_ARGUMENT, "CSR column index out of range");
            int b = find_leaf(i, j);
            leaf_of_entry.push_back(b);
            if (S.blocks[b].kind == KIND_LOWRANK) H.rank[b]++;
        }
    H.layout();
    std::vector<double> host((size_t)std::max<long long>(H.total, 0), 0.0);
    std::vector<int> used(S.blocks.size(), 0);
    size_t e = 0;
    for (int i = 0; i < N; ++i)
        for (int64_t k = rows[i]; k < rows[i + 1]; ++k, ++e) {
            int b = leaf_of_entry[e];
            const Block& B = S.blocks[b];
            int li = i - B.row_off, lj = cols[k] - B.col_off;
            if (B.kind == KIND_DENSE) {
                host[H.off[b] + li + (long long)lj * B.m] = vals[k];
            } else {
                int r = used[b]++;
                host[H.off[b] + li + (long long)r * B.m] = 1.0;
                host[H.off[b] + (long long)B.m * H.rank[b] + lj + (long long)r * B.n] = vals[k];
            }
        }
    if (H.total > 0)
        HMB_CUDA(cudaMemcpyAsync(H.data.get(), host.data(), host.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, H.ctx->stream));
    HMB_CUDA(cudaStreamSynchronize(H.ctx->stream));
}

void multiply_vector_noalloc(HMatrix& H, int transpose, double alpha, const double* x,
                             double beta, double* y);

void multiply_dense(HMatrix& H, int transpose, double alpha, const double* B,
                    int ldb, double beta, double* C, int ldc, int nrhs) {
    HMB_REQUIRE(nrhs >= 0, HM_ERR_ARGUMENT, "nrhs must be >= 0");
    const int m = transpose ? H.width() : H.height();
    const int n = transpose ? H.height() : H.width();
    HMB_REQUIRE(ldb >= std::max(1, n) && ldc >= std::max(1, m), HM_ERR_ARGUMENT,
                "leading dimension too small");
    if (nrhs == 0 || m == 0) return;
    run_jobs(*H.ctx, {MatJob{&H, 0, transpose != 0, alpha, beta, B, ldb, C, ldc, nrhs}});
}

}  // namespace hmb

using namespace hmb;

extern "C" {

const char* hm_last_error(void) { return g_last_error.c_str(); }

int hm_version(void) { return 100; }

int hm_context_create(int device, void* cuda_stream, hm_context* out) {
    return guarded([&] {
        HMB_REQUIRE(out != nullptr, HM_ERR_ARGUMENT, "out is NULL");
        *out = nullptr;
        int count = 0;
        HMB_CUDA(cudaGetDeviceCount(&count));
        HMB_REQUIRE(device >= 0 && device < count, HM_ERR_ARGUMENT, "no such CUDA device");
        HMB_CUDA(cudaSetDevice(device));
        auto* c = new hm_context_s;
        c->c.device = device;
        c->c.serial_state = kLcgSeed;
        c->c.parallel_state = kLcgSeed;
        cudaDeviceGetAttribute(&c->c.num_sms, cudaDevAttrMultiProcessorCount, device);
        // Keep freed stream-ordered memory in this process's pool across
        // synchronizations instead of returning it at every sync (a process
        // setting of the pool, not of the GPU).
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t threshold = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        if (cuda_stream) {
            c->c.stream = (cudaStream_t)cuda_stream;
        } else {
            cudaError_t err = cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking);
            if (err != cudaSuccess) {
                delete c;
                throw Error(HM_ERR_CUDA, cudaGetErrorString(err));
            }
            c->c.own_stream = true;
        }
        *out = c;
    });
}

int hm_context_destroy(hm_context ctx) {
    return guarded([&] {
        if (!ctx) return;
        // H-matrices still alive lose their device storage and become
        // unusable (every later call on them reports HM_ERR_ARGUMENT).
        for (hm_matrix_s* m : ctx->live) {
            release_storage(m);
            m->owner = nullptr;
            m->h.ctx = nullptr;
        }
        ctx->live.clear();
        for (hm_rank_model_s* m : ctx->models) {
            m->m.params.reset();
            m->m.grad.reset();
            m->m.m.reset();
            m->m.v.reset();
            m->m.ctx = nullptr;
            m->owner = nullptr;
        }
        ctx->models.clear();
        ctx->c.rank_model = nullptr;
        ctx->c.collect();
        // everything holding device memory is freed on the stream before the
        // stream goes away
        ctx->c.layouts.clear();
        ctx->c.hh_cache.reset();
        for (auto& b : ctx->c.scratch_bufs) b.reset();
        if (ctx->c.pinned) {
            cudaStreamSynchronize(ctx->c.stream);
            cudaFreeHost(ctx->c.pinned);
            ctx->c.pinned = nullptr;
        }
        ctx->c.counters.reset();
        ctx->c.errword.reset();
        ctx->c.numword.reset();
        cudaStreamSynchronize(ctx->c.stream);
        hmb::release_staging(ctx->c.stream);
        if (ctx->c.own_stream) cudaStreamDestroy(ctx->c.stream);
        delete ctx;
    });
}

int hm_context_synchronize(hm_context ctx) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        ctx->c.check_numerical();
    });
}

int hm_set_oversample(hm_context ctx, int oversample) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_REQUIRE(oversample >= 0, HM_ERR_ARGUMENT, "oversample must be >= 0");
        ctx->c.oversample = oversample;
    });
}

int hm_get_oversample(hm_context ctx, int* oversample) {
    return guarded([&] {
        HMB_REQUIRE(ctx && oversample, HM_ERR_ARGUMENT, "NULL argument");
        *oversample = ctx->c.oversample;
    });
}

int hm_set_compression_tolerance(hm_context ctx, double tol) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_REQUIRE(tol >= 0.0 && tol < 1.0, HM_ERR_ARGUMENT, "tolerance must be in [0, 1)");
        ctx->c.compression_tol = tol;
    });
}

int hm_set_tf32_kernel(hm_context ctx, int which) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_REQUIRE(which >= 0 && which <= 2, HM_ERR_ARGUMENT, "which must be 0, 1 or 2");
        ctx->c.tf32_kernel = which;
    });
}

int hm_tf32_kernel_choice(hm_matrix h, const double* B, int ldb, int nrhs, int* which) {
    return guarded([&] {
        HMB_REQUIRE(h && which && (nrhs == 0 || B), HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        HMB_REQUIRE(nrhs > 0 && ldb >= std::max(1, h->h.width()), HM_ERR_ARGUMENT,
                    "bad right-hand sides");
        *which = tf32_kernel_choice(*h->h.ctx, h->h, B, ldb, nrhs);
    });
}

int hm_set_fp64_split(hm_context ctx, int which) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_REQUIRE(which >= 0 && which <= 2, HM_ERR_ARGUMENT, "which must be 0, 1 or 2");
        ctx->c.fp64_split = which;
    });
}

int hm_fp64_split_choice(hm_matrix h, const double* B, int ldb, int nrhs, int* which) {
    return guarded([&] {
        HMB_REQUIRE(h && which && (nrhs == 0 || B), HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        HMB_REQUIRE(nrhs > 0 && ldb >= std::max(1, h->h.width()), HM_ERR_ARGUMENT,
                    "bad right-hand sides");
        // the whole product, as hm_multiply_dense runs it (a tuning run
        // writes into scratch, so no output is needed)
        MatJob J{&h->h, 0, false, 1.0, 0.0, B, ldb, nullptr, std::max(1, h->h.height()), nrhs};
        *which = fp64_split_for(*h->h.ctx, {J});
    });
}

int hm_get_compression_tolerance(hm_context ctx, double* tol) {
    return guarded([&] {
        HMB_REQUIRE(ctx && tol, HM_ERR_ARGUMENT, "NULL argument");
        *tol = ctx->c.compression_tol;
    });
}

int hm_set_lcg_states(hm_context ctx, uint64_t serial, uint64_t parallel) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        ctx->c.serial_state = serial;
        ctx->c.parallel_state = parallel;
    });
}

int hm_get_lcg_states(hm_context ctx, uint64_t* serial, uint64_t* parallel) {
    return guarded([&] {
        HMB_REQUIRE(ctx && serial && parallel, HM_ERR_ARGUMENT, "NULL argument");
        *serial = ctx->c.serial_state;
        *parallel = ctx->c.parallel_state;
    });
}

int hm_natural_to_hierarchical_map(int dim, const int* sizes, int num_levels, int* map) {
    return guarded([&] {
        HMB_REQUIRE(sizes && map, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(num_levels >= 1, HM_ERR_ARGUMENT, "num_levels must be >= 1");
        natural_to_hierarchical(dim, sizes, num_levels, map);
    });
}

int hm_create_from_csr(hm_context ctx, int dim, const int* sizes, int num_levels,
                       int max_rank, int strongly_admissible, const int64_t* row_offsets,
                       const int32_t* col_indices, const double* values, hm_matrix* out) {
    return guarded([&] {
        HMB_REQUIRE(ctx && sizes && row_offsets && out, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(max_rank >= 0, HM_ERR_ARGUMENT, "max_rank must be >= 0");
        *out = nullptr;
        HMB_CUDA(cudaSetDevice(ctx->c.device));
        auto* m = new_handle(ctx);
        try {
            m->h.S = build_structure(dim, sizes, num_levels, strongly_admissible != 0);
            m->h.max_rank = max_rank;
            const int64_t nnz = row_offsets[m->h.S->N];
            HMB_REQUIRE(nnz == 0 || (col_indices && values), HM_ERR_ARGUMENT,
                        "NULL CSR arrays");
            import_csr(m->h, row_offsets, col_indices, values);
        } catch (...) {
            delete_handle(m);
            throw;
        }
        *out = m;
    });
}

int hm_create_from_csr_complex(hm_context ctx, int dim, const int* sizes, int num_levels,
                               int max_rank, int strongly_admissible, const int64_t* row_offsets,
                               const int32_t* col_indices, const double* values, hm_matrix* out) {
    return guarded([&] {
        HMB_REQUIRE(ctx && sizes && row_offsets && out, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(max_rank >= 0, HM_ERR_ARGUMENT, "max_rank must be >= 0");
        *out = nullptr;
        HMB_CUDA(cudaSetDevice(ctx->c.device));
        auto* m = new_handle(ctx);
        try {
            m->h.S = build_structure(dim, sizes, num_levels, strongly_admissible != 0, 2);
            m->h.max_rank = 2 * max_rank;
            const int n = m->h.S->N / 2;
            const int64_t nnz = row_offsets[n];
            HMB_REQUIRE(nnz == 0 || (col_indices && values), HM_ERR_ARGUMENT,
                        "NULL CSR arrays");
            // real form: entry a + bi at (i, j) -> [[a, -b], [b, a]] at rows
            // 2i, 2i+1 and columns 2j, 2j+1 (zero parts dropped)
            std::vector<int64_t> rows((size_t)2 * n + 1, 0);
            std::vector<int32_t> cols;
            std::vector<double> vals;
            cols.reserve((size_t)nnz * 4);
            vals.reserve((size_t)nnz * 4);
            for (int i = 0; i < n; ++i)
                for (int half = 0; half < 2; ++half) {
                    for (int64_t k = row_offsets[i]; k < row_offsets[i + 1]; ++k) {
                        const int j = col_indices[k];
                        HMB_REQUIRE(j >= 0 && j < n, HM_ERR_ARGUMENT,
                                    "CSR column index out of range");
                        const double a = values[2 * k], b = values[2 * k + 1];
                        const double re_col = half == 0 ? a : b;    // column 2j
                        const double im_col = half == 0 ? -b : a;   // column 2j + 1
                        if (re_col != 0.0) {
                            cols.push_back(2 * j);
                            vals.push_back(re_col);
                        }
                        if (im_col != 0.0) {
                            cols.push_back(2 * j + 1);
                            vals.push_back(im_col);
                        }
                    }
                    rows[(size_t)2 * i + half + 1] = (int64_t)cols.size();
                }
            import_csr(m->h, rows.data(), cols.data(), vals.data());
        } catch (...) {
            delete_handle(m);
            throw;
        }
        *out = m;
    });
}

int hm_low_rank_product(hm_matrix A, int op, double alpha, hm_matrix B, int sample_rank,
                        double* U, int ldu, double* V, int ldv, int max_rank, int* rank) {
    return guarded([&] {
        HMB_REQUIRE(A && B && U && V && rank, HM_ERR_ARGUMENT, "NULL argument");
        hm_context_s* ctx = owner_of(A);
        HMB_REQUIRE(owner_of(B) == ctx, HM_ERR_ARGUMENT, "factors live in different contexts");
        HMB_REQUIRE(A->h.S && B->h.S, HM_ERR_ARGUMENT, "empty H-matrix");
        const int n = A->h.height();
        HMB_REQUIRE(ldu >= std::max(1, n) && ldv >= std::max(1, n), HM_ERR_ARGUMENT,
                    "leading dimension too small");
        DeviceBuffer<double> dU, dV;
        const int r = low_rank_product(ctx->c, A->h, op, alpha, B->h, sample_rank, dU, dV);
        HMB_REQUIRE(r <= max_rank, HM_ERR_ARGUMENT, "max_rank is below the product's rank");
        cudaStream_t st = ctx->c.stream;
        if (r > 0) {
            HMB_CUDA(cudaMemcpy2DAsync(U, (size_t)ldu * sizeof(double), dU.get(),
                                       (size_t)n * sizeof(double), (size_t)n * sizeof(double), r,
                                       cudaMemcpyDeviceToHost, st));
            HMB_CUDA(cudaMemcpy2DAsync(V, (size_t)ldv * sizeof(double), dV.get(),
                                       (size_t)n * sizeof(double), (size_t)n * sizeof(double), r,
                                       cudaMemcpyDeviceToHost, st));
        }
        HMB_CUDA(cudaStreamSynchronize(st));
        *rank = r;
    });
}

int hm_packed_size(hm_matrix h, size_t* bytes) {
    return guarded([&] {
        HMB_REQUIRE(h && bytes, HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        *bytes = packed_size(h->h);
    });
}

int hm_pack(hm_matrix h, void* buffer, size_t capacity, size_t* written) {
    return guarded([&] {
        HMB_REQUIRE(h && buffer, HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        const size_t n = pack(h->h, static_cast<unsigned char*>(buffer), capacity);
        if (written) *written = n;
    });
}

int hm_unpack(hm_context ctx, int dim, const void* buffer, size_t size, hm_matrix* out) {
    return guarded([&] {
        HMB_REQUIRE(ctx && buffer && out, HM_ERR_ARGUMENT, "NULL argument");
        *out = nullptr;
        HMB_CUDA(cudaSetDevice(ctx->c.device));
        auto* m = new_handle(ctx);
        try {
            unpack(ctx->c, dim, static_cast<const unsigned char*>(buffer), size, m->h);
        } catch (...) {
            delete_handle(m);
            throw;
        }
        *out = m;
    });
}

int hm_is_complex(hm_matrix h, int* is_complex) {
    return guarded([&] {
        HMB_REQUIRE(h && is_complex, HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        *is_complex = h->h.S && h->h.S->dof == 2 ? 1 : 0;
    });
}

int hm_multiply_dense_complex(hm_matrix h, int op, double alpha_re, double alpha_im,
                              const double* B, int ldb, double beta_re, double beta_im, double* C,
                              int ldc, int nrhs) {
    return guarded([&] {
        HMB_REQUIRE(h && (nrhs == 0 || (B && C)), HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        multiply_dense_complex(h->h, op, alpha_re, alpha_im, B, ldb, beta_re, beta_im, C, ldc,
                               nrhs);
    });
}

int hm_multiply_dense_complex_host(hm_matrix h, int op, double alpha_re, double alpha_im,
                                   const double* B, int ldb, double beta_re, double beta_im,
                                   double* C, int ldc, int nrhs) {
    return guarded([&] {
        HMB_REQUIRE(h && (nrhs == 0 || (B && C)), HM_ERR_ARGUMENT, "NULL argument");
        Context& ctx = owner_of(h)->c;
        HMB_REQUIRE(h->h.S && h->h.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
        const int n = h->h.height() / 2;
        HMB_REQUIRE(ldb >= std::max(1, n) && ldc >= std::max(1, n), HM_ERR_ARGUMENT,
                    "leading dimension too small");
        if (nrhs == 0) return;
        const size_t col = (size_t)n * 2 * sizeof(double);
        DeviceBuffer<double> dB, dC;
        dB.allocate((size_t)2 * n * nrhs, ctx.stream);
        dC.allocate((size_t)2 * n * nrhs, ctx.stream);
        HMB_CUDA(cudaMemcpy2DAsync(dB.get(), col, B, (size_t)ldb * 2 * sizeof(double), col, nrhs,
                                   cudaMemcpyHostToDevice, ctx.stream));
        if (beta_re != 0.0 || beta_im != 0.0)
            HMB_CUDA(cudaMemcpy2DAsync(dC.get(), col, C, (size_t)ldc * 2 * sizeof(double), col,
                                       nrhs, cudaMemcpyHostToDevice, ctx.stream));
        multiply_dense_complex(h->h, op, alpha_re, alpha_im, dB.get(), n, beta_re, beta_im,
                               dC.get(), n, nrhs);
        HMB_CUDA(cudaMemcpy2DAsync(C, (size_t)ldc * 2 * sizeof(double), dC.get(), col, col, nrhs,
                                   cudaMemcpyDeviceToHost, ctx.stream));
        HMB_CUDA(cudaStreamSynchronize(ctx.stream));
    });
}

int hm_destroy(hm_matrix h) {
    return guarded([&] {
        if (!h) return;
        delete_handle(h);
    });
}

int hm_structure(hm_matrix h, int* dim, int* sizes, int* strongly_admissible,
                 int* unknowns_per_point) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        const Structure& S = *h->h.S;
        if (dim) *dim = S.dim;
        if (sizes)
            for (int d = 0; d < S.dim; ++d) sizes[d] = S.sizes[d];
        if (strongly_admissible) *strongly_admissible = S.strong ? 1 : 0;
        if (unknowns_per_point) *unknowns_per_point = S.dof;
    });
}

int hm_info(hm_matrix h, int* height, int* width, int* num_levels, int* max_rank,
            int64_t* counts, int64_t* bytes) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        const Structure& S = *h->h.S;
        if (height) *height = S.N;
        if (width) *width = S.N;
        if (num_levels) *num_levels = S.num_levels;
        if (max_rank) *max_rank = h->h.max_rank;
        if (counts) {
            int64_t c[4] = {0, 0, 0, 0};
            for (size_t b = 0; b < S.blocks.size(); ++b) {
                c[S.blocks[b].kind]++;
                if (S.blocks[b].kind == KIND_LOWRANK) c[3] += h->h.rank[b];
            }
            std::memcpy(counts, c, sizeof(c));
        }
        if (bytes) *bytes = h->h.total * (int64_t)sizeof(double);
    });
}

int hm_set_to_random(hm_matrix h) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        launch_fill_random(owner_of(h)->c, h->h);
    });
}

int hm_multiply_dense(hm_matrix h, int transpose, double alpha, const double* B, int ldb,
                      double beta, double* C, int ldc, int nrhs) {
    return guarded([&] {
        HMB_REQUIRE(h && (nrhs == 0 || (B && C)), HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        multiply_dense(h->h, transpose, alpha, B, ldb, beta, C, ldc, nrhs);
    });
}

int hm_multiply_dense_host(hm_matrix h, int transpose, double alpha, const double* B, int ldb,
                           double beta, double* C, int ldc, int nrhs) {
    return guarded([&] {
        HMB_REQUIRE(h && (nrhs == 0 || (B && C)), HM_ERR_ARGUMENT, "NULL argument");
        Context& ctx = owner_of(h)->c;
        const int m = transpose ? h->h.width() : h->h.height();
        const int n = transpose ? h->h.height() : h->h.width();
        HMB_REQUIRE(ldb >= std::max(1, n) && ldc >= std::max(1, m), HM_ERR_ARGUMENT,
                    "leading dimension too small");
        if (nrhs == 0) return;
        DeviceBuffer<double> dB, dC;
        dB.allocate((size_t)n * nrhs, ctx.stream);
        dC.allocate((size_t)m * nrhs, ctx.stream);
        HMB_CUDA(cudaMemcpy2DAsync(dB.get(), n * sizeof(double), B, ldb * sizeof(double),
                                   n * sizeof(double), nrhs, cudaMemcpyHostToDevice, ctx.stream));
        if (beta != 0.0)
            HMB_CUDA(cudaMemcpy2DAsync(dC.get(), m * sizeof(double), C, ldc * sizeof(double),
                                       m * sizeof(double), nrhs, cudaMemcpyHostToDevice,
                                       ctx.stream));
        multiply_dense(h->h, transpose, alpha, dB.get(), n, beta, dC.get(), m, nrhs);
        HMB_CUDA(cudaMemcpy2DAsync(C, ldc * sizeof(double), dC.get(), m * sizeof(double),
                                   m * sizeof(double), nrhs, cudaMemcpyDeviceToHost, ctx.stream));
        HMB_CUDA(cudaStreamSynchronize(ctx.stream));
    });
}

int hm_multiply_hmat(hm_matrix A, double alpha, hm_matrix B, hm_matrix* C) {
    return guarded([&] {
        HMB_REQUIRE(A && B && C, HM_ERR_ARGUMENT, "NULL argument");
        hm_context_s* ctx = owner_of(A);
        HMB_REQUIRE(owner_of(B) == ctx, HM_ERR_ARGUMENT, "factors live in different contexts");
        HMB_REQUIRE(*C != A && *C != B, HM_ERR_ARGUMENT,
                    "the product must not overwrite a factor");
        if (*C) HMB_REQUIRE(owner_of(*C) == ctx, HM_ERR_ARGUMENT, "C lives in another context");
        bool created = false;
        if (*C == nullptr) {
            *C = new_handle(ctx);
            created = true;
        }
        try {
            hh_multiply(ctx->c, A->h, B->h, alpha, 0.0, (*C)->h, true);
        } catch (...) {
            if (created) {
                delete_handle(*C);
                *C = nullptr;
            }
            throw;
        }
    });
}

int hm_multiply_hmat_update(hm_matrix A, double alpha, hm_matrix B, double beta, hm_matrix C) {
    return guarded([&] {
        HMB_REQUIRE(A && B && C, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(C != A && C != B, HM_ERR_ARGUMENT, "the product must not overwrite a factor");
        hm_context_s* ctx = owner_of(A);
        HMB_REQUIRE(owner_of(B) == ctx && owner_of(C) == ctx, HM_ERR_ARGUMENT,
                    "operands live in different contexts");
        HMB_REQUIRE(C->h.S != nullptr, HM_ERR_ARGUMENT, "C is empty");
        hh_multiply(ctx->c, A->h, B->h, alpha, beta, C->h, false);
    });
}

int hm_estimate_two_norm(hm_matrix h, double theta, double confidence, double* estimate) {
    return guarded([&] {
        HMB_REQUIRE(h && estimate, HM_ERR_ARGUMENT, "NULL argument");
        *estimate = estimate_two_norm(owner_of(h)->c, h->h, theta, confidence);
    });
}

int hm_schulz_invert(hm_matrix h, int num_iterations, double theta, double confidence,
                     double stop_tol, int* iterations, double* trace, int trace_cap,
                     int* trace_len) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        HMB_REQUIRE(h->h.height() == h->h.width(), HM_ERR_ARGUMENT,
                    "Cannot invert non-square matrices");
        HMB_REQUIRE(theta > 1.0, HM_ERR_ARGUMENT, "Theta must be > 1");
        HMB_REQUIRE(confidence > 0.0, HM_ERR_ARGUMENT, "Confidence must be positive");
        SchulzResult r = schulz_invert(owner_of(h)->c, h->h, num_iterations, theta, confidence,
                                       stop_tol);
        if (iterations) *iterations = r.iterations;
        if (trace_len) *trace_len = (int)r.trace.size();
        if (trace)
            for (int i = 0; i < trace_cap && i < (int)r.trace.size(); ++i) trace[i] = r.trace[i];
    });
}

int hm_schulz_invert_mixed(hm_matrix h, int num_iterations, double theta, double confidence,
                           double stop_tol, double mixed_switch, int* iterations,
                           int* low_iterations, double* trace, int trace_cap, int* trace_len) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        HMB_REQUIRE(h->h.height() == h->h.width(), HM_ERR_ARGUMENT,
                    "Cannot invert non-square matrices");
        HMB_REQUIRE(theta > 1.0, HM_ERR_ARGUMENT, "Theta must be > 1");
        HMB_REQUIRE(confidence > 0.0, HM_ERR_ARGUMENT, "Confidence must be positive");
        HMB_REQUIRE(mixed_switch >= 0.0, HM_ERR_ARGUMENT, "mixed_switch must be >= 0");
        SchulzResult r = schulz_invert(owner_of(h)->c, h->h, num_iterations, theta, confidence,
                                       stop_tol, mixed_switch);
        if (iterations) *iterations = r.iterations;
        if (low_iterations) *low_iterations = r.low_iterations;
        if (trace_len) *trace_len = (int)r.trace.size();
        if (trace)
            for (int i = 0; i < trace_cap && i < (int)r.trace.size(); ++i) trace[i] = r.trace[i];
    });
}

int hm_set_low_precision(hm_context ctx, int on) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        ctx->c.low_precision = on != 0;
    });
}

int hm_copy(hm_matrix src, hm_matrix* dst) {
    return guarded([&] {
        HMB_REQUIRE(src && dst, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(*dst != src, HM_ERR_ARGUMENT, "copy onto itself");
        hm_context_s* ctx = owner_of(src);
        if (*dst == nullptr) *dst = new_handle(ctx);
        HMB_REQUIRE(owner_of(*dst) == ctx, HM_ERR_ARGUMENT, "dst lives in another context");
        hmat_copy(ctx->c, src->h, (*dst)->h);
    });
}

int hm_transpose(hm_matrix src, hm_matrix* dst) {
    return guarded([&] {
        HMB_REQUIRE(src && dst, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(*dst != src, HM_ERR_ARGUMENT, "transpose onto itself");
        hm_context_s* ctx = owner_of(src);
        if (*dst == nullptr) *dst = new_handle(ctx);
        HMB_REQUIRE(owner_of(*dst) == ctx, HM_ERR_ARGUMENT, "dst lives in another context");
        hmat_transpose(ctx->c, src->h, (*dst)->h);
    });
}

int hm_scale_complex(hm_matrix h, double alpha_re, double alpha_im) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        complex_scale(owner_of(h)->c, h->h, alpha_re, alpha_im);
    });
}

int hm_add_constant_to_diagonal_complex(hm_matrix h, double alpha_re, double alpha_im) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        complex_add_diagonal(owner_of(h)->c, h->h, alpha_re, alpha_im);
    });
}

int hm_conjugate(hm_matrix src, hm_matrix* dst) {
    return guarded([&] {
        HMB_REQUIRE(src && dst, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(*dst != src, HM_ERR_ARGUMENT, "conjugate onto itself");
        hm_context_s* ctx = owner_of(src);
        HMB_REQUIRE(src->h.S && src->h.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
        if (*dst == nullptr) *dst = new_handle(ctx);
        HMB_REQUIRE(owner_of(*dst) == ctx, HM_ERR_ARGUMENT, "dst lives in another context");
        hmat_copy(ctx->c, src->h, (*dst)->h);
        complex_conjugate(ctx->c, (*dst)->h);
    });
}

int hm_transpose_complex(hm_matrix src, hm_matrix* dst) {
    return guarded([&] {
        HMB_REQUIRE(src && dst, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(*dst != src, HM_ERR_ARGUMENT, "transpose onto itself");
        hm_context_s* ctx = owner_of(src);
        HMB_REQUIRE(src->h.S && src->h.S->dof == 2, HM_ERR_ARGUMENT, "not a complex H-matrix");
        if (*dst == nullptr) *dst = new_handle(ctx);
        HMB_REQUIRE(owner_of(*dst) == ctx, HM_ERR_ARGUMENT, "dst lives in another context");
        // A^T = conj(A^H); the real form's transpose is A^H
        hmat_transpose(ctx->c, src->h, (*dst)->h);
        complex_conjugate(ctx->c, (*dst)->h);
    });
}

int hm_update_with(hm_matrix A, double alpha, hm_matrix B) {
    return guarded([&] {
        HMB_REQUIRE(A && B, HM_ERR_ARGUMENT, "NULL argument");
        hm_context_s* ctx = owner_of(A);
        HMB_REQUIRE(owner_of(B) == ctx, HM_ERR_ARGUMENT, "matrices live in different contexts");
        hmat_update_with(ctx->c, A->h, alpha, B->h);
    });
}

int hm_set_to_identity(hm_matrix h) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        hmat_set_identity(owner_of(h)->c, h->h);
    });
}

int hm_conjugate_in_place(hm_matrix h) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        if (h->h.S->dof == 2) complex_conjugate(owner_of(h)->c, h->h);
    });
}

int hm_scale(hm_matrix h, double alpha) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        hmat_scale(owner_of(h)->c, h->h, alpha);
    });
}

int hm_add_constant_to_diagonal(hm_matrix h, double alpha) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        hmat_add_diagonal(owner_of(h)->c, h->h, alpha);
    });
}

int hm_multiply_dense_tf32(hm_matrix h, double alpha, const double* B, int ldb, double beta,
                           double* C, int ldc, int nrhs) {
    return guarded([&] {
        HMB_REQUIRE(h && (nrhs == 0 || (B && C)), HM_ERR_ARGUMENT, "NULL argument");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        multiply_dense_tf32(h->h, alpha, B, ldb, beta, C, ldc, nrhs);
    });
}

int hm_multiply_vector_noalloc(hm_matrix h, int transpose, double alpha, const double* x,
                               double beta, double* y) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        multiply_vector_noalloc(h->h, transpose != 0, alpha, x, beta, y);
    });
}

int hm_direct_invert(hm_matrix h) {
    return guarded([&] {
        HMB_REQUIRE(h, HM_ERR_ARGUMENT, "h is NULL");
        hm_context ctx = owner_of(h);
        HMB_REQUIRE(h->h.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
        hmat_direct_invert(ctx->c, h->h);
    });
}

int hm_check_bounded_wait(int device, long long polls, int* timed_out) {
    return guarded([&] {
        HMB_REQUIRE(timed_out, HM_ERR_ARGUMENT, "timed_out is NULL");
        HMB_REQUIRE(polls > 0 && polls <= (1LL << 26), HM_ERR_ARGUMENT,
                    "polls must be in 1..2^26");
        *timed_out = bounded_wait_times_out(device, polls) ? 1 : 0;
    });
}

unsigned long long hm_kernel_launches(void) {
    return g_launches.load(std::memory_order_relaxed);
}

int hm_profile_enable(hm_context ctx, int on) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        ctx->c.collect();
        ctx->c.totals.clear();
        ctx->c.profiling = on != 0;
    });
}

int hm_profile_read(hm_context ctx, int index, char* name, int name_cap, double* ms,
                    int64_t* launches) {
    return guarded([&] {
        HMB_REQUIRE(ctx && name && ms && launches && name_cap > 0, HM_ERR_ARGUMENT,
                    "NULL argument");
        ctx->c.collect();
        HMB_REQUIRE(index >= 0 && index < (int)ctx->c.totals.size(), HM_ERR_ARGUMENT,
                    "profile index out of range");
        auto it = ctx->c.totals.begin();
        std::advance(it, index);
        std::snprintf(name, (size_t)name_cap, "%s", it->first.c_str());
        *ms = it->second.ms;
        *launches = it->second.launches;
    });
}

// ---------------------------------------------------------------------------
// Learned sample counts
// ---------------------------------------------------------------------------
int hm_rank_feature_count(void) { return hmb::kMlpFeatures; }
int hm_rank_param_count(void) { return hmb::kMlpParams; }

int hm_rank_model_create(hm_context ctx, uint64_t seed, hm_rank_model* out) {
    return guarded([&] {
        HMB_REQUIRE(ctx && out, HM_ERR_ARGUMENT, "NULL argument");
        auto* m = new hm_rank_model_s();
        m->owner = ctx;
        m->m.ctx = &ctx->c;
        try {
            m->m.init(seed);
        } catch (...) {
            delete m;
            throw;
        }
        ctx->models.insert(m);
        *out = m;
    });
}

int hm_rank_model_destroy(hm_rank_model m) {
    return guarded([&] {
        if (!m) return;
        if (m->owner) {
            if (m->owner->c.rank_model == &m->m) m->owner->c.rank_model = nullptr;
            m->owner->models.erase(m);
        }
        delete m;
    });
}

int hm_rank_model_set_params(hm_rank_model m, const float* params, int n) {
    return guarded([&] {
        HMB_REQUIRE(m && m->owner && params, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(n == hmb::kMlpParams, HM_ERR_ARGUMENT, "wrong parameter count");
        m->m.set_params(params);
    });
}

int hm_rank_model_get_params(hm_rank_model m, float* params, int n) {
    return guarded([&] {
        HMB_REQUIRE(m && m->owner && params, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(n == hmb::kMlpParams, HM_ERR_ARGUMENT, "wrong parameter count");
        m->m.get_params(params);
    });
}

int hm_rank_model_loss_grad(hm_rank_model m, const float* x, const float* t, int n, float* loss,
                            float* grad) {
    return guarded([&] {
        HMB_REQUIRE(m && m->owner && x && t && loss, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(n > 0, HM_ERR_ARGUMENT, "empty batch");
        *loss = m->m.loss_and_grad(x, t, n, grad);
    });
}

int hm_rank_model_train(hm_rank_model m, const float* x, const float* t, int n, int epochs,
                        float lr, float* loss) {
    return guarded([&] {
        HMB_REQUIRE(m && m->owner && x && t, HM_ERR_ARGUMENT, "NULL argument");
        const float l = m->m.train(x, t, n, epochs, lr);
        if (loss) *loss = l;
    });
}

int hm_rank_model_predict(hm_rank_model m, const float* x, int n, float* out) {
    return guarded([&] {
        HMB_REQUIRE(m && m->owner && x && out, HM_ERR_ARGUMENT, "NULL argument");
        HMB_REQUIRE(n >= 0, HM_ERR_ARGUMENT, "negative count");
        m->m.predict(x, n, out);
    });
}

int hm_use_rank_model(hm_context ctx, hm_rank_model m, int margin, int probes) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        HMB_REQUIRE(!m || m->owner == ctx, HM_ERR_ARGUMENT, "model belongs to another context");
        HMB_REQUIRE(margin >= 0 && probes >= 1, HM_ERR_ARGUMENT, "margin >= 0, probes >= 1");
        ctx->c.rank_model = m ? &m->m : nullptr;
        ctx->c.rank_margin = margin;
        ctx->c.rank_probes = probes;
    });
}

int hm_rank_log_enable(hm_context ctx, int on) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        ctx->c.rank_log = on != 0;
    });
}

int hm_rank_log_read(hm_context ctx, float* x, float* t, int cap, int* n, int clear) {
    return guarded([&] {
        HMB_REQUIRE(ctx && n, HM_ERR_ARGUMENT, "NULL argument");
        const int have = (int)ctx->c.log_t.size();
        const int take = std::min(std::max(cap, 0), have);
        if (take > 0) {
            HMB_REQUIRE(x && t, HM_ERR_ARGUMENT, "NULL buffers");
            std::copy(ctx->c.log_x.begin(), ctx->c.log_x.begin() + (long long)take * hmb::kMlpFeatures, x);
            std::copy(ctx->c.log_t.begin(), ctx->c.log_t.begin() + take, t);
        }
        *n = have;
        if (clear) {
            ctx->c.log_x.clear();
            ctx->c.log_t.clear();
        }
    });
}

int hm_rank_stats(hm_context ctx, int64_t* compressions, int64_t* samples, int64_t* samples_plain,
                  int64_t* fallbacks) {
    return guarded([&] {
        HMB_REQUIRE(ctx, HM_ERR_ARGUMENT, "ctx is NULL");
        const auto& s = ctx->c.rank_stats;
        if (compressions) *compressions = s.compressions;
        if (samples) *samples = s.samples;
        if (samples_plain) *samples_plain = s.samples_plain;
        if (fallbacks) *fallbacks = s.fallbacks;
    });
}

}  // extern "C"
