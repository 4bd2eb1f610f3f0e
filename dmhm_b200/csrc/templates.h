// Device work lists of one subtree of one H-matrix (see matmul.cu), shared
// by the FP64 and the tensor-core H-matrix x dense products.
#pragma once
#include <map>
#include <tuple>
#include <memory>
#include <vector>

#include "engine.h"

namespace hmb {

// Work lists of one subtree (device arrays), independent of the operands and
// of where the matrix storage lives: every block is an element offset into
// the storage, so matrices with the same structure and ranks share them.
struct P1T {
    long long w;       // W: nin x r, ld ldw, at storage + w
    long long in_off;  // row offset into the job input
    long long t_rel;   // T_b = T + t_rel * k (r x k, ld r)
    long long c0;      // first row of this item in the concatenation of all items' rows
    int nin, r, ldw, pad;
};

struct P2T {
    long long out_off;  // row offset of the tile's first row in the job output
    long long c0;       // first column of this tile in the concatenation of all tiles
    int r0, rows, e0, e1;
    int width;          // columns of the tile's concatenation (sum of its entries' inner)
    int pad;
};

struct P2Entry {
    long long a;       // A at storage + a: element (i,p) = transA ? A[p + i*lda] : A[i + p*lda]
    long long b_off;   // b_from_t ? T + b_off * k (ld ldt) : job input + b_off
    int lda, inner, transA, b_from_t, ldt;
    int cbeg;          // first column of this entry in its tile's concatenation
};

// Phase-1 tile of the wide (many-column) product: 64 rows of T gathered from
// the low-rank blocks that share one source box (so one input slice, rows
// [in_off, in_off + nin)).  Row i is column wcol[i] of some W; its results
// go to T[trel[i] * k + tj[i] + c * tr[i]].  wcol: storage offsets.
constexpr int kWideTile = 64;
struct W1Tile {
    long long in_off;
    int nin, rows;
    long long wcol[kWideTile];
    long long trel[kWideTile];
    int tj[kWideTile];
    int tr[kWideTile];
};

struct JobTemplate {
    DeviceBuffer<P1T> p1;
    DeviceBuffer<P2T> p2;
    DeviceBuffer<P2Entry> ent;
    DeviceBuffer<int> zero_tiles;   // tiles without entries (output = beta * output)
    DeviceBuffer<W1Tile> w1;        // wide phase-1 tiles
    DeviceBuffer<int> w1cp;         // wide: chunk prefix over the W1 tiles
    DeviceBuffer<int> tcp;          // wide: chunk prefix over the row tiles
    DeviceBuffer<int> ekc;          // wide: first chunk of every entry within its tile
    int nw1 = 0;
    long long wc1 = 0, wc2 = 0;     // wide: chunks of phase 1 / phase 2
    // Host copies, and per split width GW the first item / (tile, entry) of
    // every warp of the narrow kernels (built on first use).
    std::vector<P1T> hp1;
    std::vector<P2T> hp2;
    std::vector<P2Entry> hent;
    std::vector<int> hent_block;    // leaf block of every entry
    std::vector<int> hzero;         // tiles without entries
    // Block-streamed one-vector product plan (matvec.cu); null when the
    // blocks do not fit its limits.
    std::shared_ptr<struct MvPlan> mv;
    bool mv_tried = false;
    std::map<long long, DeviceBuffer<int>> start1;
    std::map<long long, DeviceBuffer<int2>> start2;
    int n1 = 0, n2 = 0, nz = 0;
    long long c1 = 0, c2 = 0;       // rows of all items, columns of all tiles
    int rmax = 0;                   // largest rank among the items
    long long t_rows = 0;   // sum of the ranks: T holds t_rows * k entries
};

// Matrices of one context with the same structure, rank cap and ranks (so the
// same storage layout) and the work lists of their products.
struct LayoutGroup {
    const Structure* S = nullptr;
    int max_rank = 0;
    std::vector<int> rank;
    uint64_t hash = 0;
    std::map<std::tuple<int, int, int>, std::shared_ptr<JobTemplate>> templates;
};

}  // namespace hmb
