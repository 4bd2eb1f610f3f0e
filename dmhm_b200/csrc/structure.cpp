// Block structure construction (see structure.h).
#include "structure.h"

#include <algorithm>
#include <cstdlib>
#include <functional>
#include <map>
#include <mutex>

#include "common.h"

namespace hmb {

namespace {

// Fills box `id` (already allocated) and, above the leaf level, allocates its
// q children contiguously and fills them in quadrant order, so leaf clusters
// are numbered in hierarchical (depth-first) order.
void fill_box(Structure& S, int id, int level, const int* coord,
              const int* size, int offset) {
    Box b{};
    b.level = level;
    b.count = 1;
    for (int k = 0; k < 3; ++k) {
        b.coord[k] = k < S.dim ? coord[k] : 0;
        b.size[k] = k < S.dim ? size[k] : 1;
        b.count *= b.size[k];
    }
    b.count *= S.dof;
    b.offset = offset;
    b.first_child = -1;
    b.leaf0 = S.num_clusters();
    S.boxes[id] = b;
    if (level == S.num_levels - 1) {
        S.leaf_box.push_back(id);
        S.boxes[id].leaf1 = S.num_clusters();
        return;
    }
    int lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = b.size[k] / 2;
        hi[k] = b.size[k] - lo[k];
    }
    int first = (int)S.boxes.size();
    S.boxes[id].first_child = first;
    S.boxes.resize(S.boxes.size() + S.q);
    int off = offset;
    for (int qd = 0; qd < S.q; ++qd) {
        int csize[3], ccoord[3];
        for (int k = 0; k < 3; ++k) {
            int bit = k < S.dim ? (qd >> k) & 1 : 0;
            csize[k] = k < S.dim ? (bit ? hi[k] : lo[k]) : 1;
            ccoord[k] = 2 * b.coord[k] + bit;
        }
        fill_box(S, first + qd, level + 1, ccoord, csize, off);
        off += S.boxes[first + qd].count;
    }
    S.boxes[id].leaf1 = S.num_clusters();
}

}  // namespace

bool Structure::in_subtree(int b, int root) const {
    int lr = blocks[root].level;
    while (b >= 0 && blocks[b].level > lr) b = blocks[b].parent;
    return b == root;
}

bool same_structure(const Structure& a, const Structure& b) {
    return a.dim == b.dim && a.num_levels == b.num_levels && a.strong == b.strong &&
           a.dof == b.dof &&
           a.sizes[0] == b.sizes[0] && a.sizes[1] == b.sizes[1] && a.sizes[2] == b.sizes[2];
}

std::shared_ptr<Structure> build_structure(int dim, const int* sizes, int num_levels,
                                           bool strong, int dof) {
    // H-matrices over the same grid share one structure object.
    static std::mutex mu;
    static std::map<std::vector<int>, std::weak_ptr<Structure>> cache;
    std::vector<int> key{dim, num_levels, strong ? 1 : 0, dof};
    for (int k = 0; k < dim; ++k) key.push_back(sizes[k]);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end())
            if (auto sp = it->second.lock()) return sp;
    }
    auto S = build_structure_uncached(dim, sizes, num_levels, strong, dof);
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = S;
    return S;
}

std::shared_ptr<Structure> build_structure_uncached(int dim, const int* sizes, int num_levels,
                                                    bool strong, int dof) {
    HMB_REQUIRE(dim == 2 || dim == 3, HM_ERR_ARGUMENT, "dim must be 2 or 3");
    HMB_REQUIRE(num_levels >= 1 && num_levels <= 16, HM_ERR_ARGUMENT,
                "num_levels must be in [1, 16]");
    auto S = std::make_shared<Structure>();
    S->dim = dim;
    S->num_levels = num_levels;
    S->strong = strong;
    S->q = 1 << dim;
    HMB_REQUIRE(dof == 1 || dof == 2, HM_ERR_ARGUMENT, "dof must be 1 or 2");
    S->dof = dof;
    long long N = dof;
    for (int k = 0; k < 3; ++k) {
        S->sizes[k] = k < dim ? sizes[k] : 1;
        HMB_REQUIRE(S->sizes[k] >= 1, HM_ERR_ARGUMENT, "grid sizes must be >= 1");
        N *= S->sizes[k];
    }
    HMB_REQUIRE(N < (1LL << 30), HM_ERR_ARGUMENT, "grid too large");
    S->N = (int)N;

    int zero[3] = {0, 0, 0};
    S->boxes.resize(1);
    fill_box(*S, 0, 0, zero, S->sizes, 0);

    // Blocks: recursion over (target box, source box) pairs.
    std::function<void(int, int, int, int)> rec = [&](int bid, int tb, int sbx,
                                                      int level) {
        const Box& T = S->boxes[tb];
        const Box& Sb = S->boxes[sbx];
        Block& B = S->blocks[bid];
        B.level = level;
        B.tgt_box = tb;
        B.src_box = sbx;
        B.row_off = T.offset;
        B.col_off = Sb.offset;
        B.m = T.count;
        B.n = Sb.count;
        B.first_child = -1;
        int maxd = 0;
        bool any = false;
        for (int k = 0; k < dim; ++k) {
            int d = std::abs(T.coord[k] - Sb.coord[k]);
            maxd = std::max(maxd, d);
            any = any || d != 0;
        }
        bool admissible = strong ? (maxd > 1) : any;
        if (admissible) {
            B.kind = KIND_LOWRANK;
        } else if (num_levels - level > 1) {
            B.kind = KIND_NODE;
            int first = (int)S->blocks.size();
            S->blocks[bid].first_child = first;
            S->blocks.resize(S->blocks.size() + S->q * S->q);
            int tf = S->boxes[tb].first_child, sf = S->boxes[sbx].first_child;
            for (int t = 0; t < S->q; ++t)
                for (int s = 0; s < S->q; ++s) {
                    int c = first + s + S->q * t;
                    S->blocks[c].parent = bid;
                    rec(c, tf + t, sf + s, level + 1);
                }
        } else {
            B.kind = KIND_DENSE;
        }
    };
    S->blocks.resize(1);
    S->blocks[0].parent = -1;
    rec(0, 0, 0, 0);

    // Transposes.
    for (auto& b : S->blocks) b.transpose = -1;
    std::function<void(int, int)> trec = [&](int b, int bt) {
        S->blocks[b].transpose = bt;
        if (S->blocks[b].kind != KIND_NODE) return;
        for (int t = 0; t < S->q; ++t)
            for (int s = 0; s < S->q; ++s)
                trec(S->child(b, t, s), S->child(bt, s, t));
    };
    trec(0, 0);

    // Leaves in depth-first (reference recursion) order, and covers.
    {
        std::vector<int> stack{0};
        while (!stack.empty()) {
            int b = stack.back();
            stack.pop_back();
            if (S->blocks[b].kind == KIND_NODE) {
                for (int c = S->q * S->q - 1; c >= 0; --c)
                    stack.push_back(S->blocks[b].first_child + c);
            } else {
                S->leaves.push_back(b);
            }
        }
    }
    std::vector<int> by_level = S->leaves;
    std::stable_sort(by_level.begin(), by_level.end(), [&](int a, int b) {
        return S->blocks[a].level < S->blocks[b].level;
    });
    int nc = S->num_clusters();
    S->row_cover.assign(nc, {});
    S->col_cover.assign(nc, {});
    for (int b : by_level) {
        const Block& B = S->blocks[b];
        if (B.m == 0 || B.n == 0) continue;
        const Box& T = S->boxes[B.tgt_box];
        const Box& Sb = S->boxes[B.src_box];
        for (int c = T.leaf0; c < T.leaf1; ++c) S->row_cover[c].push_back(b);
        for (int c = Sb.leaf0; c < Sb.leaf1; ++c) S->col_cover[c].push_back(b);
    }
    for (int c = 0; c < nc; ++c)
        S->max_cluster = std::max(S->max_cluster, S->boxes[S->leaf_box[c]].count);
    return S;
}

void natural_to_hierarchical(int dim, const int* sizes, int num_levels,
                             int* map) {
    HMB_REQUIRE(dim == 2 || dim == 3, HM_ERR_ARGUMENT, "dim must be 2 or 3");
    int sz[3] = {1, 1, 1};
    for (int k = 0; k < dim; ++k) sz[k] = sizes[k];
    int index = 0;
    std::function<void(int, const int*, const int*)> rec =
        [&](int level, const int* origin, const int* this_size) {
            if (level == num_levels - 1) {
                for (int z = 0; z < this_size[2]; ++z)
                    for (int y = 0; y < this_size[1]; ++y)
                        for (int x = 0; x < this_size[0]; ++x) {
                            long long nat =
                                (long long)(origin[2] + z) * sz[0] * sz[1] +
                                (long long)(origin[1] + y) * sz[0] + origin[0] + x;
                            map[nat] = index++;
                        }
                return;
            }
            int lo[3], hi[3];
            for (int k = 0; k < 3; ++k) {
                lo[k] = k < dim ? this_size[k] / 2 : 0;
                hi[k] = this_size[k] - lo[k];
            }
            for (int qd = 0; qd < (1 << dim); ++qd) {
                int o[3], s[3];
                for (int k = 0; k < 3; ++k) {
                    int bit = k < dim ? (qd >> k) & 1 : 0;
                    if (k < dim) {
                        s[k] = bit ? hi[k] : lo[k];
                        o[k] = origin[k] + (bit ? lo[k] : 0);
                    } else {
                        s[k] = 1;
                        o[k] = 0;
                    }
                }
                rec(level + 1, o, s);
            }
        };
    int origin[3] = {0, 0, 0};
    rec(0, origin, sz);
}

}  // namespace hmb
