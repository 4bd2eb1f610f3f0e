"""Host-side logic that needs no GPU, compiled with the host compiler: the
tagged-offset encoding of the cached operation lists (dmhm_b200/csrc/reloc.h)
and the block structure builder (dmhm_b200/csrc/structure.cpp) against the
oracle's tree and the block counts of the benchmark grids."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import load
from oracle import dmhm_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dmhm_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_relocator(tmp_path):
    exe = tmp_path / "reloc_check"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "dmhm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "reloc_check.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


@pytest.fixture(scope="module")
def structure_check(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("structure") / "structure_check"
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", CSRC, "-I", cuda_inc,
                    os.path.join(ROOT, "tests", "cpp", "structure_check.cpp"),
                    os.path.join(CSRC, "structure.cpp"), "-o", str(exe)], check=True)

    def run(dim, levels, strong, sizes, dof=1):
        r = subprocess.run([str(exe), str(dim), str(levels), str(int(strong)), str(dof)]
                           + [str(s) for s in sizes], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr
        lines = r.stdout.strip().splitlines()
        leaves = np.array([[int(v) for v in ln.split()] for ln in lines[:-1]])
        return leaves, lines[-1]
    return run


KIND = {O.LOW_RANK: 1, O.DENSE: 2}


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_structure_matches_oracle_tree(structure_check, case):
    """Leaf blocks in the reference's depth-first order, with kind, level,
    offsets and sizes, equal the oracle's tree (which follows
    src/HMat2d/HMat2d.cpp:797-809, :961-1033 and the Node ctor of
    include/dmhm/hmat2d.hpp:362-389); the builder's own invariants hold."""
    fx = load(case)
    sizes = [int(s) for s in fx["sizes"]]
    L = int(fx["levels"])
    leaves, _ = structure_check(len(sizes), L, bool(fx["strong"]), sizes)
    top = O.top_level(len(sizes), sizes, L, int(fx["rank"]), bool(fx["strong"]))
    H = O.import_sparse(top, *O.stencil_csr(sizes, fx["coef"], L)[:3])
    want = np.array([[KIND[b.kind], L - b.num_levels, b.tgt_off, b.src_off, b.height, b.width]
                     for b in H.leaves()])
    assert leaves.shape == want.shape and np.array_equal(leaves, want)


def test_structure_real_form_of_complex(structure_check):
    """dof = 2 (a complex matrix in real form): the same tree with every
    offset and size doubled."""
    one, _ = structure_check(2, 3, True, [24, 20])
    two, _ = structure_check(2, 3, True, [24, 20], dof=2)
    assert np.array_equal(two[:, :2], one[:, :2])
    assert np.array_equal(two[:, 2:], 2 * one[:, 2:])


@pytest.mark.parametrize("dim,levels,sizes,dense,lowrank", [
    # grid, numLevels -> dense leaves, low-rank blocks per level (count, side)
    (2, 4, [32, 32], 484, {2: (156, 64), 3: (1116, 16)}),
    (2, 6, [128, 128], 8836, {2: (156, 1024), 3: (1116, 256), 4: (5628, 64), 5: (25020, 16)}),
    (2, 5, [128, 128], 2116, {2: (156, 1024), 3: (1116, 256), 4: (5628, 64)}),
    (3, 4, [32, 32, 32], 10648, {2: (3096, 512), 3: (53352, 64)}),
    (2, 6, [256, 256], 8836, {2: (156, 4096), 3: (1116, 1024), 4: (5628, 256), 5: (25020, 64)}),
])
def test_structure_block_counts(structure_check, dim, levels, sizes, dense, lowrank):
    """Block counts of the benchmark grids (strong admissibility): dense
    leaves and low-rank blocks per level with their sizes."""
    leaves, _ = structure_check(dim, levels, True, sizes)
    assert int(np.sum(leaves[:, 0] == 2)) == dense
    lr = leaves[leaves[:, 0] == 1]
    assert sorted(set(lr[:, 1].tolist())) == sorted(lowrank)
    for lev, (count, side) in lowrank.items():
        at = lr[lr[:, 1] == lev]
        assert len(at) == count and np.all(at[:, 4] == side) and np.all(at[:, 5] == side)
