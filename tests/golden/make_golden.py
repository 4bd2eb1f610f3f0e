"""Generates the golden fixtures in this folder from the reference itself.

Runs the unmodified reference library (compiled by ``oracle/Makefile`` into
``oracle/_ref/dmhm_ref_driver``) on small seeded cases and stores inputs and
outputs as ``<case>.npz``.  Only this script and the oracle pinning tests
touch the reference; the fixtures let the GPU tests check parity without it.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py c1 ragged  # some cases
    python tests/golden/make_golden.py cplx       # the complex-double case
    python tests/golden/make_golden.py d2s d2w d3s  # single-rank DistHMat cases
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

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
            else:
                make_case(n, CASES[n], tmp)


if __name__ == "__main__":
    main(sys.argv[1:])
