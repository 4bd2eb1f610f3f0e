// The reference's H-matrix wire format (Pack / Unpack / PackedSize,
// src/HMat2d/Pack-incl.hpp:27-364, src/HMat3d/Pack-incl.hpp): a header of
// ints and bools written as raw native bytes, then the block tree depth
// first (children t-major, s-minor), each block as its BlockType (int enum:
// NODE 0, NODE_SYMMETRIC 1, LOW_RANK 2, DENSE 3), then for LOW_RANK the rank
// and U, V column by column, for DENSE its MatrixType (GENERAL 0, SYMMETRIC
// 1) and the columns (the lower triangle for SYMMETRIC).  The layout has to
// be byte-identical to interoperate with the reference, so this file writes
// and reads exactly those fields in that order.
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace hmb {

namespace {

constexpr int kNode = 0, kNodeSymmetric = 1, kLowRank = 2, kDense = 3;
constexpr int kGeneral = 0, kSymmetric = 1;

class Writer {
  public:
    explicit Writer(unsigned char* p) : p_(p) {}
    template <typename T>
    void put(const T& v) {
        if (p_) std::memcpy(p_ + n_, &v, sizeof(T));
        n_ += sizeof(T);
    }
    void put(const double* v, long long count) {
        if (p_ && count > 0) std::memcpy(p_ + n_, v, (size_t)count * sizeof(double));
        n_ += (size_t)count * sizeof(double);
    }
    size_t size() const { return n_; }

  private:
    unsigned char* p_;
    size_t n_ = 0;
};

class Reader {
  public:
    Reader(const unsigned char* p, size_t n) : p_(p), n_(n) {}
    template <typename T>
    T get() {
        need(sizeof(T));
        T v;
        std::memcpy(&v, p_ + at_, sizeof(T));
        at_ += sizeof(T);
        return v;
    }
    void get(double* dst, long long count) {
        need((size_t)count * sizeof(double));
        if (count > 0) std::memcpy(dst, p_ + at_, (size_t)count * sizeof(double));
        at_ += (size_t)count * sizeof(double);
    }
    void skip(size_t bytes) {
        need(bytes);
        at_ += bytes;
    }
    size_t position() const { return at_; }

  private:
    void need(size_t k) const {
        HMB_REQUIRE(at_ + k <= n_, HM_ERR_ARGUMENT, "packed H-matrix is truncated");
    }
    const unsigned char* p_;
    size_t n_, at_ = 0;
};

// Header of the root block: numLevels, maxRank, source/target offsets,
// symmetric, stronglyAdmissible, per axis the source and target sizes, per
// axis the source and target box coordinates (2-D: Pack-incl.hpp:46-59;
// 3-D adds z sizes and coordinates).
void write_header(Writer& w, const HMatrix& H) {
    const Structure& S = *H.S;
    w.put<int>(S.num_levels);
    w.put<int>(H.max_rank);
    w.put<int>(0);
    w.put<int>(0);
    w.put<bool>(false);
    w.put<bool>(S.strong);
    for (int k = 0; k < S.dim; ++k) {
        w.put<int>(S.sizes[k]);
        w.put<int>(S.sizes[k]);
    }
    for (int k = 0; k < S.dim; ++k) {
        w.put<int>(0);
        w.put<int>(0);
    }
}

void write_blocks(Writer& w, const HMatrix& H, const std::vector<double>& host) {
    const Structure& S = *H.S;
    std::vector<int> stack{0};
    while (!stack.empty()) {
        const int b = stack.back();
        stack.pop_back();
        const Block& B = S.blocks[b];
        if (B.kind == KIND_NODE) {
            w.put<int>(kNode);
            for (int c = S.q * S.q - 1; c >= 0; --c) stack.push_back(B.first_child + c);
        } else if (B.kind == KIND_LOWRANK) {
            w.put<int>(kLowRank);
            const int r = H.rank[b];
            w.put<int>(r);
            const double* u = host.empty() ? nullptr : host.data() + H.off[b];
            w.put(u, (long long)B.m * r);
            w.put(u ? u + (long long)B.m * r : nullptr, (long long)B.n * r);
        } else {
            w.put<int>(kDense);
            w.put<int>(kGeneral);
            w.put(host.empty() ? nullptr : host.data() + H.off[b], (long long)B.m * B.n);
        }
    }
}

}  // namespace

// PackedSize counts one int more than the header holds (13 ints + 2 bools
// in 2-D, 17 + 2 in 3-D, Pack-incl.hpp:32 and the 3-D :32, against 12 / 16
// ints written), so the reference's Pack into a Vector<byte> of that size
// ends with 4 zero bytes; the same size and trailing zeros are kept here.
constexpr size_t kPackSlack = sizeof(int);

size_t packed_size(const HMatrix& H) {
    HMB_REQUIRE(H.S != nullptr, HM_ERR_ARGUMENT, "empty H-matrix");
    HMB_REQUIRE(H.S->dof == 1, HM_ERR_UNSUPPORTED,
                "Pack of complex H-matrices is not supported (real form on the device)");
    Writer w(nullptr);
    write_header(w, H);
    write_blocks(w, H, {});
    return w.size() + kPackSlack;
}

size_t pack(const HMatrix& H, unsigned char* out, size_t cap) {
    const size_t need = packed_size(H);
    HMB_REQUIRE(cap >= need, HM_ERR_ARGUMENT, "pack buffer too small");
    std::vector<double> host((size_t)std::max<long long>(H.total, 2), 0.0);
    if (H.total > 0) {
        HMB_CUDA(cudaMemcpyAsync(host.data(), H.data.get(), (size_t)H.total * sizeof(double),
                                 cudaMemcpyDeviceToHost, H.ctx->stream));
        HMB_CUDA(cudaStreamSynchronize(H.ctx->stream));
    }
    Writer w(out);
    write_header(w, H);
    write_blocks(w, H, host);
    std::memset(out + w.size(), 0, kPackSlack);
    return w.size() + kPackSlack;
}

void unpack(Context& ctx, int dim, const unsigned char* buf, size_t size, HMatrix& H) {
    HMB_REQUIRE(dim == 2 || dim == 3, HM_ERR_ARGUMENT, "dim must be 2 or 3");
    Reader r(buf, size);
    const int num_levels = r.get<int>();
    const int max_rank = r.get<int>();
    const int source_offset = r.get<int>();
    const int target_offset = r.get<int>();
    const bool symmetric = r.get<bool>();
    const bool strong = r.get<bool>();
    int sizes[3] = {1, 1, 1};
    for (int k = 0; k < dim; ++k) {
        const int src = r.get<int>(), tgt = r.get<int>();
        HMB_REQUIRE(src == tgt, HM_ERR_UNSUPPORTED, "packed H-matrix is not square");
        sizes[k] = src;
    }
    for (int k = 0; k < dim; ++k) {
        const int xs = r.get<int>(), xt = r.get<int>();
        HMB_REQUIRE(xs == 0 && xt == 0, HM_ERR_UNSUPPORTED, "packed H-matrix is not a root");
    }
    HMB_REQUIRE(source_offset == 0 && target_offset == 0, HM_ERR_UNSUPPORTED,
                "packed H-matrix is not a root");
    HMB_REQUIRE(!symmetric, HM_ERR_UNSUPPORTED,
                "symmetric H-matrices (NODE_SYMMETRIC blocks) are not supported");
    HMB_REQUIRE(max_rank >= 0, HM_ERR_ARGUMENT, "negative maxRank in packed H-matrix");
    H.ctx = &ctx;
    H.S = build_structure(dim, sizes, num_levels, strong);
    H.max_rank = max_rank;
    const Structure& S = *H.S;
    H.rank.assign(S.blocks.size(), 0);
    // first pass: block kinds and ranks, positions of the data
    struct Item { int b; size_t pos; int type; };
    std::vector<Item> items;
    std::vector<int> stack{0};
    while (!stack.empty()) {
        const int b = stack.back();
        stack.pop_back();
        const Block& B = S.blocks[b];
        const int type = r.get<int>();
        if (B.kind == KIND_NODE) {
            HMB_REQUIRE(type == kNode, HM_ERR_ARGUMENT,
                        "packed block tree does not match the grid's block structure");
            for (int c = S.q * S.q - 1; c >= 0; --c) stack.push_back(B.first_child + c);
        } else if (B.kind == KIND_LOWRANK) {
            HMB_REQUIRE(type == kLowRank, HM_ERR_ARGUMENT,
                        "packed block tree does not match the grid's block structure");
            const int rk = r.get<int>();
            HMB_REQUIRE(rk >= 0, HM_ERR_ARGUMENT, "negative rank in packed H-matrix");
            H.rank[b] = rk;
            items.push_back({b, r.position(), kGeneral});
            r.skip((size_t)(B.m + B.n) * rk * sizeof(double));
        } else {
            HMB_REQUIRE(type == kDense, HM_ERR_ARGUMENT,
                        "packed block tree does not match the grid's block structure");
            const int mt = r.get<int>();
            HMB_REQUIRE(mt == kGeneral || mt == kSymmetric, HM_ERR_ARGUMENT,
                        "unknown dense matrix type in packed H-matrix");
            HMB_REQUIRE(mt == kGeneral || B.m == B.n, HM_ERR_ARGUMENT,
                        "symmetric dense block that is not square");
            items.push_back({b, r.position(), mt});
            const long long cnt = mt == kGeneral ? (long long)B.m * B.n
                                                 : (long long)B.m * (B.m + 1) / 2;
            r.skip((size_t)cnt * sizeof(double));
        }
    }
    (void)kNodeSymmetric;
    H.layout();
    std::vector<double> host((size_t)std::max<long long>(H.total, 2), 0.0);
    for (const Item& it : items) {
        const Block& B = S.blocks[it.b];
        Reader d(buf + it.pos, size - it.pos);
        double* dst = host.data() + H.off[it.b];
        if (B.kind == KIND_LOWRANK) {
            d.get(dst, (long long)(B.m + B.n) * H.rank[it.b]);
        } else if (it.type == kGeneral) {
            d.get(dst, (long long)B.m * B.n);
        } else {
            // lower triangle, column j from row j (Pack-incl.hpp:356-360),
            // mirrored into the general storage
            for (int j = 0; j < B.n; ++j) {
                d.get(dst + j + (long long)j * B.m, B.m - j);
                for (int i = j + 1; i < B.m; ++i)
                    dst[j + (long long)i * B.m] = dst[i + (long long)j * B.m];
            }
        }
    }
    if (H.total > 0)
        HMB_CUDA(cudaMemcpyAsync(H.data.get(), host.data(), (size_t)H.total * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx.stream));
    HMB_CUDA(cudaStreamSynchronize(ctx.stream));
}

}  // namespace hmb
