"""Generates the golden fixtures in this folder from the reference itself.

Runs the unmodified reference library (compiled by ``oracle/Makefile`` into
``oracle/_ref/dmhm_ref_driver``) on small seeded cases and stores inputs and
outputs as ``<case>.npz``.  Only this script and the oracle pinning tests
touch the reference; the fixtures let the GPU tests check parity without it.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py c1 ragged  # some cases
    python tests/golden/make_golden.py cplx       # the complex-double case
    python tests/golden/make_golden.py d2s d2w d3s  # single-rank DistHMat cases
    python tests/golden/make_golden.py cfg2 cfg1s cfg3 cfg4   # benchmark sizes
                                                   # (not in the default set: cfg4
                                                   # runs for many minutes)
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from helpers import big_case_inputs  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "dmhm_ref_driver")
DIST_DRIVER = os.path.join(ROOT, "oracle", "_ref", "dmhm_ref_dist_driver")

# name: grid, levels, rank, oversample, strong, coefficient seed, probes
CASES = {
    "c1": dict(sizes=(32, 32), levels=4, rank=8, oversample=4, strong=1, seed=1, probes=4,
               ops=["matvec", "random", "hh_AA", "hh_AB", "schulz3", "schulz_stop", "lrprod",
                    "direct"]),
    "ragged": dict(sizes=(24, 20), levels=3, rank=6, oversample=4, strong=1, seed=5, probes=3,
                   ops=["matvec", "random", "hh_AA", "hh_AB", "schulz3", "lrprod", "direct"]),
    "weak": dict(sizes=(16, 16), levels=3, rank=4, oversample=4, strong=0, seed=7, probes=3,
                 ops=["matvec", "random", "hh_AA", "schulz3", "direct"]),
    "c3d": dict(sizes=(16, 16, 16), levels=3, rank=8, oversample=8, strong=1, seed=9, probes=2,
                ops=["matvec", "random", "hh_AA", "schulz2", "direct"]),
}


def run(args, out_prefix, driver=DRIVER):
    r = subprocess.run([driver] + [str(a) for a in args] + ["--out", out_prefix],
                       capture_output=True, text=True, env={**os.environ, "OPENBLAS_NUM_THREADS": "1"})
    if r.returncode != 0:
        raise RuntimeError(f"reference driver failed: {args}\n{r.stderr}")
    info = json.loads(r.stdout.strip().splitlines()[-1])
    return info, np.fromfile(out_prefix + ".bin")


def make_case(name, spec, tmp):
    sizes = spec["sizes"]
    dim = len(sizes)
    N = int(np.prod(sizes))
    rng = np.random.default_rng(spec["seed"])
    coef = 1.0 + rng.random(N)
    coefB = 1.0 + rng.random(N)
    P = rng.standard_normal((N, spec["probes"]))
    cpath, cbpath, ppath = (os.path.join(tmp, f) for f in ("c.bin", "cb.bin", "p.bin"))
    coef.tofile(cpath)
    coefB.tofile(cbpath)
    np.asfortranarray(P).T.copy().tofile(ppath)     # column-major
    base = ["--dim", dim, "--nx", sizes[0], "--ny", sizes[1],
            "--nz", sizes[2] if dim == 3 else 1, "--levels", spec["levels"],
            "--rank", spec["rank"], "--oversample", spec["oversample"],
            "--strong", spec["strong"], "--coef", cpath]
    k = spec["probes"]
    out = dict(sizes=np.array(sizes), levels=spec["levels"], rank=spec["rank"],
               oversample=spec["oversample"], strong=spec["strong"], coef=coef, coefB=coefB,
               probes=P)
    o = os.path.join(tmp, "o")

    def mat(v):
        return v.reshape(k, N).T.copy()

    for op in spec["ops"]:
        if op == "matvec":
            _, y = run(["matvec"] + base + ["--x", ppath, "--nrhs", k], o)
            out["matvec"] = mat(y)
            _, y1 = run(["matvec"] + base + ["--x", ppath, "--nrhs", 1], o)
            out["matvec1"] = y1
            _, yt = run(["transpose"] + base + ["--x", ppath, "--nrhs", k], o)
            out["matvec_T"] = mat(yt)
        elif op == "random":
            _, y = run(["matvec"] + base + ["--x", ppath, "--nrhs", k, "--random", 1], o)
            out["random"] = mat(y)
            _, yt = run(["transpose"] + base + ["--x", ppath, "--nrhs", k, "--random", 1], o)
            out["random_T"] = mat(yt)
        elif op == "hh_AA":
            _, y = run(["hh"] + base + ["--x", ppath, "--nrhs", k], o)
            out["hh_AA"] = mat(y)
        elif op == "lrprod":
            # hmat_tools::Multiply / TransposeMultiply: F := alpha op(A) B with
            # A SetToRandom and B from the second coefficient field
            for opn, tag in ((0, "lr_AB"), (1, "lr_AtB")):
                info, y = run(["lrprod"] + base + ["--x", ppath, "--nrhs", k, "--random", 1,
                                                   "--useB", 1, "--coefB", cbpath,
                                                   "--alpha", 0.75, "--iters", opn], o)
                out[tag] = mat(y)
                out[tag + "_rank"] = info["iterations"]
        elif op == "hh_AB":
            _, y = run(["hh"] + base + ["--x", ppath, "--nrhs", k, "--useB", 1,
                                        "--coefB", cbpath, "--alpha", -0.5], o)
            out["hh_AB"] = mat(y)
        elif op in ("schulz2", "schulz3"):
            its = int(op[-1])
            info, y = run(["schulz_trace"] + base + ["--x", ppath, "--nrhs", k, "--iters", its], o)
            out[op] = mat(y)
            out[op + "_trace"] = np.fromfile(o + ".trace.bin")
            out[op + "_seconds"] = info["seconds"]
        elif op == "direct":
            # DirectInvert (recursive Schur complements) applied to the probes
            info, y = run(["direct"] + base + ["--x", ppath, "--nrhs", k], o)
            out["direct"] = mat(y)
            out["direct_seconds"] = info["seconds"]
        elif op == "schulz_stop":
            info, y = run(["schulz_trace"] + base + ["--x", ppath, "--nrhs", k, "--iters", -1,
                                                     "--stopTol", 1e-4], o)
            out["schulz_stop"] = mat(y)
            out["schulz_stop_trace"] = np.fromfile(o + ".trace.bin")
            out["schulz_stop_iterations"] = info["iterations"]
            out["schulz_stop_seconds"] = info["seconds"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "ok", sorted(out))


# complex cases (HMat2d<std::complex<double>>, shifted Helmholtz-like operator)
COMPLEX_CASES = {
    "cplx": dict(sizes=(32, 32), levels=3, rank=12, oversample=4, kwave=6.0, seed=11, probes=2),
}


def make_complex_case(name, spec, tmp):
    sizes = spec["sizes"]
    N = int(np.prod(sizes))
    rng = np.random.default_rng(spec["seed"])
    k = spec["probes"]
    P = rng.standard_normal((N, k)) + 1j * rng.standard_normal((N, k))
    ppath = os.path.join(tmp, "cp.bin")
    np.asfortranarray(P).T.copy().view(np.float64).tofile(ppath)   # column-major, interleaved
    base = ["--nx", sizes[0], "--ny", sizes[1], "--levels", spec["levels"],
            "--rank", spec["rank"], "--oversample", spec["oversample"],
            "--kwave", spec["kwave"], "--x", ppath, "--nrhs", k]
    out = dict(sizes=np.array(sizes), levels=spec["levels"], rank=spec["rank"],
               oversample=spec["oversample"], kwave=spec["kwave"], probes=P)
    o = os.path.join(tmp, "co")

    def cmat(v):
        return v.view(np.complex128).reshape(k, N).T.copy()

    _, y = run(["cmatvec"] + base, o)
    out["matvec"] = cmat(y)
    _, y = run(["chh"] + base, o)
    out["hh_AA"] = cmat(y)
    info, y = run(["cschulz"] + base + ["--iters", -1, "--stopTol", 1e-8], o)
    out["schulz_stop"] = cmat(y)
    out["schulz_stop_seconds"] = info["seconds"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "ok", sorted(out))


# the reference's Pack wire format: (case, SetToRandom?)
PACK_CASES = (("ragged", 1), ("c3d", 0))


def make_pack(tmp):
    """Pack bytes written by the reference for two fixture matrices (a
    SetToRandom 2-D matrix and a sparse-built 3-D one), with the reference's
    own matvec of the packed matrices' Unpack on the fixture probes."""
    out = {}
    for name, random in PACK_CASES:
        spec = CASES[name]
        sizes = spec["sizes"]
        dim = len(sizes)
        N = int(np.prod(sizes))
        rng = np.random.default_rng(spec["seed"])
        coef = 1.0 + rng.random(N)
        rng.random(N)                                  # coefB
        P = rng.standard_normal((N, spec["probes"]))
        cpath, ppath = os.path.join(tmp, "pc.bin"), os.path.join(tmp, "pp.bin")
        coef.tofile(cpath)
        np.asfortranarray(P).T.copy().tofile(ppath)
        base = ["--dim", dim, "--nx", sizes[0], "--ny", sizes[1],
                "--nz", sizes[2] if dim == 3 else 1, "--levels", spec["levels"],
                "--rank", spec["rank"], "--oversample", spec["oversample"],
                "--strong", spec["strong"], "--coef", cpath, "--random", random]
        o = os.path.join(tmp, "pk")
        r = subprocess.run([DRIVER, "pack"] + [str(a) for a in base] + ["--out", o],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr)
        packed = np.fromfile(o + ".pack", dtype=np.uint8)
        _, y = run(["unpack_matvec"] + base + ["--coefB", o + ".pack", "--x", ppath,
                                                "--nrhs", spec["probes"]], o)
        out[name + "_pack"] = packed
        out[name + "_unpack_matvec"] = y.reshape(spec["probes"], N).T.copy()
    np.savez_compressed(os.path.join(HERE, "pack.npz"), **out)
    print("pack ok", sorted(out))


def make_lcg(tmp):
    o = os.path.join(tmp, "lcg")
    run(["lcg", "--count", 9], o)
    d = np.fromfile(o + ".bin")
    np.savez_compressed(os.path.join(HERE, "lcg.npz"), count=9, draws=d)
    print("lcg ok")


# single-rank DistHMat2d / DistHMat3d (the reference's distributed classes
# run as one process over the serial MPI stand-in), beside the serial HMat2d /
# HMat3d on the same operator: products with multType 0 and 2, a fixed-count
# SchulzInvert and the stop-test SchulzInvert, all under the global
# CompressionTolerance `tol`
DIST_CASES = {
    "d2s": dict(sizes=(32, 32), levels=3, rank=8, oversample=4, strong=1, seed=13, probes=3,
                tol=1e-8, iters=16),
    "d2w": dict(sizes=(32, 32), levels=4, rank=8, oversample=4, strong=0, seed=17, probes=3,
                tol=1e-8, iters=16),
    "d3s": dict(sizes=(16, 16, 16), levels=3, rank=8, oversample=8, strong=1, seed=19, probes=2,
                tol=1e-8, iters=14),
}


def make_dist_case(name, spec, tmp):
    sizes = spec["sizes"]
    dim = len(sizes)
    N = int(np.prod(sizes))
    rng = np.random.default_rng(spec["seed"])
    coef = 1.0 + rng.random(N)
    coefB = 1.0 + rng.random(N)
    P = rng.standard_normal((N, spec["probes"]))
    cpath, cbpath, ppath = (os.path.join(tmp, f) for f in ("dc.bin", "dcb.bin", "dp.bin"))
    coef.tofile(cpath)
    coefB.tofile(cbpath)
    np.asfortranarray(P).T.copy().tofile(ppath)
    k = spec["probes"]
    base = ["--dim", dim, "--nx", sizes[0], "--ny", sizes[1],
            "--nz", sizes[2] if dim == 3 else 1, "--levels", spec["levels"],
            "--rank", spec["rank"], "--oversample", spec["oversample"],
            "--strong", spec["strong"], "--coef", cpath, "--x", ppath, "--nrhs", k]
    dist = base + ["--tol", spec["tol"]]
    out = dict(sizes=np.array(sizes), levels=spec["levels"], rank=spec["rank"],
               oversample=spec["oversample"], strong=spec["strong"], coef=coef, coefB=coefB,
               probes=P, tol=spec["tol"], iters=spec["iters"])
    o = os.path.join(tmp, "d")

    def mat(v):
        return v.reshape(k, N).T.copy()

    def drun(args):
        info, y = run(args, o, DIST_DRIVER)
        print(f"  {name} {args[0]} {args[-4:]} {info['seconds']:.2f} s", flush=True)
        return mat(y)

    for m in (0, 2):
        out[f"dist_hh_AA_m{m}"] = drun(["dhh"] + dist + ["--mult", m])
    out["dist_hh_AB_m2"] = drun(["dhh"] + dist + ["--mult", 2, "--useB", 1, "--coefB", cbpath,
                                                  "--alpha", -0.5])
    out["dist_schulz"] = drun(["dschulz"] + dist + ["--mult", 2, "--iters", spec["iters"]])
    out["dist_schulz_stop"] = drun(["dschulz"] + dist + ["--mult", 2, "--iters", -1,
                                                         "--stopTol", 1e-4])
    _, y = run(["hh"] + base, o)
    out["serial_hh_AA"] = mat(y)
    _, y = run(["schulz"] + base + ["--iters", spec["iters"]], o)
    out["serial_schulz"] = mat(y)
    _, y = run(["schulz"] + base + ["--iters", -1, "--stopTol", 1e-4], o)
    out["serial_schulz_stop"] = mat(y)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "ok", sorted(out))


# Cases at the benchmark workloads' own sizes.  Their inputs (coefficient
# fields and right-hand sides) come from a counter-based hash
# (``hashed_uniform``), so the tests regenerate them exactly and the fixtures
# hold only the reference's outputs, reduced to a few full columns plus a
# sketch G^T Y of every column (G hashed too).
#   kind "matmat": y = H X and y = H^T X for a SetToRandom H (64 columns)
#   kind "schulz": SchulzInvert (iters, stopTol), X applied to the probes
#   kind "hh":     C = A A of the sparse-built operator, applied to the probes
BIG_CASES = {
    # 128^2 five-point grid, 64-point leaves, maxRank 16, 64 right-hand sides
    "cfg2": dict(sizes=(128, 128), levels=5, rank=16, oversample=4, kind="matmat", nrhs=64,
                 keep=2, coef="uniform", seed=202),
    # 32^2 five-point grid, 16-point leaves, maxRank 8: Schulz down to 1e-8
    "cfg1s": dict(sizes=(32, 32), levels=4, rank=8, oversample=4, kind="schulz", nrhs=4,
                  keep=4, coef="uniform", seed=101, iters=-1, stopTol=1e-8),
    # 32^3 seven-point grid, 64-point leaves, maxRank 24, oversample 8: A A
    "cfg3": dict(sizes=(32, 32, 32), levels=4, rank=24, oversample=8, kind="hh", nrhs=4,
                 keep=1, coef="uniform", seed=303),
    # 256^2 five-point grid, log-uniform c, 64-point leaves, maxRank 32:
    # two fixed Schulz iterations
    "cfg4": dict(sizes=(256, 256), levels=6, rank=32, oversample=4, kind="schulz", nrhs=4,
                 keep=1, coef="log_uniform", seed=404, iters=2, stopTol=1e-4),
}
def make_big_case(name, spec, tmp):
    sizes = spec["sizes"]
    dim = len(sizes)
    N = int(np.prod(sizes))
    k = spec["nrhs"]
    coef, X, G = big_case_inputs(spec)
    cpath, xpath = os.path.join(tmp, "bc.bin"), os.path.join(tmp, "bx.bin")
    coef.tofile(cpath)
    np.asfortranarray(X).T.copy().tofile(xpath)
    base = ["--dim", dim, "--nx", sizes[0], "--ny", sizes[1],
            "--nz", sizes[2] if dim == 3 else 1, "--levels", spec["levels"],
            "--rank", spec["rank"], "--oversample", spec["oversample"], "--strong", 1,
            "--coef", cpath, "--x", xpath, "--nrhs", k]
    o = os.path.join(tmp, "b")
    out = dict(sizes=np.array(sizes), levels=spec["levels"], rank=spec["rank"],
               oversample=spec["oversample"], nrhs=k, seed=spec["seed"], coef_kind=spec["coef"])

    def reduce(tag, y):
        Y = y.reshape(k, N).T
        out[tag] = Y[:, :spec["keep"]].copy()
        out[tag + "_sketch"] = G.T @ Y

    if spec["kind"] == "matmat":
        info, y = run(["matvec"] + base + ["--random", 1], o)
        reduce("Y", y)
        out["seconds"] = info["seconds"]
        info, y = run(["transpose"] + base + ["--random", 1], o)
        reduce("YT", y)
    elif spec["kind"] == "schulz":
        info, y = run(["schulz_trace"] + base + ["--iters", spec["iters"],
                                                 "--stopTol", spec["stopTol"]], o)
        reduce("XP", y)
        out["trace"] = np.fromfile(o + ".trace.bin")
        out["iterations"] = info["iterations"]
        out["seconds"] = info["seconds"]
        out["iters"] = spec["iters"]
        out["stopTol"] = spec["stopTol"]
    elif spec["kind"] == "hh":
        info, y = run(["hh"] + base, o)
        reduce("CP", y)
        out["seconds"] = info["seconds"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "ok", f"{out['seconds']:.1f} s", sorted(out), flush=True)


def main(argv):
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8"], check=True,
                   capture_output=True)
    names = argv or list(CASES) + list(COMPLEX_CASES) + ["lcg", "pack"] + list(DIST_CASES)
    if any(n in DIST_CASES for n in names):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "dist"], check=True,
                       capture_output=True)
    with tempfile.TemporaryDirectory() as tmp:
        for n in names:
            if n == "lcg":
                make_lcg(tmp)
            elif n == "pack":
                make_pack(tmp)
            elif n in COMPLEX_CASES:
                make_complex_case(n, COMPLEX_CASES[n], tmp)
            elif n in DIST_CASES:
                make_dist_case(n, DIST_CASES[n], tmp)
            elif n in BIG_CASES:
                make_big_case(n, BIG_CASES[n], tmp)
            else:
                make_case(n, CASES[n], tmp)


if __name__ == "__main__":
    main(sys.argv[1:])
