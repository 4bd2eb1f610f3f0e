// Block structure of a square H-matrix over a 2-D or 3-D box grid, flattened
// into arrays.  Follows the reference's tree exactly (quadtree/octree with
// children indexed s + 2^d t, strong admissibility max_k |dx_k| > 1, weak
// admissibility "any dx_k != 0", leaves at level numLevels-1:
// include/dmhm/hmat2d.hpp:288-341, src/HMat2d/HMat2d.cpp:797-809,
// include/dmhm/hmat3d.hpp:455-535, src/HMat3d/HMat3d.cpp:852-875).
#pragma once
#include <memory>
#include <vector>

namespace hmb {

enum BlockKind : int { KIND_NODE = 0, KIND_LOWRANK = 1, KIND_DENSE = 2 };

// One box of the spatial tree (a cluster of grid points / rows).
struct Box {
    int level;
    int coord[3];
    int size[3];
    int offset;      // first hierarchical index
    int count;       // number of points
    int first_child; // box id of child 0 (children contiguous), -1 at leaves
    int leaf0, leaf1;  // leaf clusters [leaf0, leaf1) below this box
};

struct Block {
    int kind;
    int level;
    int parent;
    int first_child;  // children contiguous: first_child + s + q*t
    int tgt_box, src_box;
    int row_off, col_off, m, n;
    int transpose;    // block id with target/source swapped
};

struct Structure {
    int dim = 2;
    int sizes[3] = {1, 1, 1};
    int num_levels = 1;
    bool strong = true;
    int q = 4;        // children per side of a node: 2^dim
    // Unknowns per grid point: 1, or 2 for the real form of a complex matrix
    // (point p owns rows dof*p .. dof*p + dof - 1; box offsets, counts and
    // block sizes are in rows)
    int dof = 1;
    int N = 0;        // rows = dof * grid points

    std::vector<Box> boxes;     // box 0 = the whole grid
    std::vector<int> leaf_box;  // leaf cluster -> box id (hierarchical order)
    std::vector<Block> blocks;  // block 0 = the root; children contiguous
    std::vector<int> leaves;    // low-rank and dense blocks, depth-first order
    // For leaf cluster c: leaf blocks whose rows (row_cover) or columns
    // (col_cover) contain it, coarse levels first.
    std::vector<std::vector<int>> row_cover, col_cover;
    int max_cluster = 0;        // largest leaf cluster

    int num_clusters() const { return (int)leaf_box.size(); }
    int child(int b, int t, int s) const { return blocks[b].first_child + s + q * t; }
    bool in_subtree(int b, int root) const;  // b == root or a descendant
};

// Builds the structure (shared by all H-matrices over the same grid and
// parameters); throws hmb::Error on bad arguments.
std::shared_ptr<Structure> build_structure(int dim, const int* sizes, int num_levels,
                                           bool strong, int dof = 1);
std::shared_ptr<Structure> build_structure_uncached(int dim, const int* sizes, int num_levels,
                                                    bool strong, int dof = 1);
bool same_structure(const Structure& a, const Structure& b);

// map[natural] = hierarchical index (x fastest in the natural order).
void natural_to_hierarchical(int dim, const int* sizes, int num_levels,
                             int* map);

}  // namespace hmb
