// Host-side dump of the block structure (structure.cpp): for the grid given
// on the command line (dim levels strong dof x y [z]) prints one line per
// leaf block in depth-first order, "kind level row_off col_off m n", then
// a summary line "blocks B clusters C max_cluster M" and checks the
// invariants the device code relies on:
//   - every node's children tile its rows and columns exactly,
//   - transpose(transpose(b)) == b and a transpose swaps rows and columns,
//   - the leaf blocks tile the whole matrix,
//   - each leaf cluster's row cover lists exactly the leaves over its rows,
//     coarse levels first.
// Exits non-zero (and prints "fail ...") when an invariant breaks.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "structure.h"

using namespace hmb;

int main(int argc, char** argv) {
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s dim levels strong dof x y [z]\n", argv[0]);
        return 2;
    }
    const int dim = std::atoi(argv[1]), levels = std::atoi(argv[2]);
    const bool strong = std::atoi(argv[3]) != 0;
    const int dof = std::atoi(argv[4]);
    int sizes[3] = {std::atoi(argv[5]), std::atoi(argv[6]), argc > 7 ? std::atoi(argv[7]) : 1};
    auto S = build_structure_uncached(dim, sizes, levels, strong, dof);
    int fails = 0;
    const int q = S->q;
    for (size_t b = 0; b < S->blocks.size(); ++b) {
        const Block& B = S->blocks[b];
        const Block& T = S->blocks[B.transpose];
        if (S->blocks[T.transpose].transpose != B.transpose || T.transpose != (int)b ||
            T.m != B.n || T.n != B.m || T.row_off != B.col_off || T.col_off != B.row_off ||
            T.kind != B.kind) {
            std::printf("fail transpose of block %zu\n", b);
            ++fails;
        }
        if (B.kind != KIND_NODE) continue;
        int rows = 0;
        for (int t = 0; t < q; ++t) {
            int cols = 0;
            const Block& first = S->blocks[S->child((int)b, t, 0)];
            for (int s = 0; s < q; ++s) {
                const Block& C = S->blocks[S->child((int)b, t, s)];
                if (C.parent != (int)b || C.row_off != B.row_off + rows ||
                    C.col_off != B.col_off + cols || C.m != first.m || C.level != B.level + 1) {
                    std::printf("fail child (%d,%d) of block %zu\n", t, s, b);
                    ++fails;
                }
                cols += C.n;
            }
            if (cols != B.n) {
                std::printf("fail columns of block %zu\n", b);
                ++fails;
            }
            rows += first.m;
        }
        if (rows != B.m) {
            std::printf("fail rows of block %zu\n", b);
            ++fails;
        }
    }
    // leaves tile the matrix (N^2 entries, no overlap: a per-row count of
    // covered columns must reach N for every row)
    std::vector<long long> covered(S->N, 0);
    for (int b : S->leaves) {
        const Block& B = S->blocks[b];
        std::printf("%d %d %d %d %d %d\n", B.kind, B.level, B.row_off, B.col_off, B.m, B.n);
        for (int i = 0; i < B.m; ++i) covered[B.row_off + i] += B.n;
    }
    for (int i = 0; i < S->N; ++i)
        if (covered[i] != S->N) {
            std::printf("fail leaves cover row %d %lld times\n", i, covered[i]);
            ++fails;
            break;
        }
    // row covers
    for (int c = 0; c < S->num_clusters(); ++c) {
        const Box& L = S->boxes[S->leaf_box[c]];
        std::vector<int> expect;
        for (int b : S->leaves) {
            const Block& B = S->blocks[b];
            if (B.m > 0 && B.n > 0 && B.row_off <= L.offset && L.offset < B.row_off + B.m)
                expect.push_back(b);
        }
        const std::vector<int>& got = S->row_cover[c];
        bool same = got.size() == expect.size();
        for (size_t k = 0; same && k < got.size(); ++k) {
            bool found = false;
            for (int e : expect) found = found || e == got[k];
            same = found && (k == 0 || S->blocks[got[k - 1]].level <= S->blocks[got[k]].level);
        }
        if (!same) {
            std::printf("fail row cover of cluster %d\n", c);
            ++fails;
        }
    }
    std::printf("blocks %zu clusters %d max_cluster %d\n", S->blocks.size(),
                S->num_clusters(), S->max_cluster);
    return fails ? 1 : 0;
}
