// Exercises the C++ facade (include/dmhm_b200.hpp) the way the reference's
// drivers use dmhm::HMat2d (tests/HMat2d/MultiplyHMat.cpp, Invert.cpp):
// build the stencil operator from a Sparse matrix in hierarchical order,
// multiply vectors and dense blocks, form A*A, run SchulzInvert.
// Written against the reference's namespace dmhm (an alias of dmhm_b200),
// with an AbstractHMat reference for the norm estimate, views of dense
// blocks, and HMat2d<std::complex<double>> on the shifted Helmholtz-like
// operator.
// Usage: facade_check <dir> <nx> <ny> <levels> <rank> <nprobes>
//                     [<cside> <clevels> <crank> <kwave> <cprobes>]
// Reads <dir>/coef.bin (natural order), <dir>/probes.bin (column-major) and,
// for the complex part, <dir>/cprobes.bin (column-major, interleaved);
// writes <dir>/{matvec1,matvec,matvec_view,norm,hh,schulz3}.bin and
// <dir>/{cmatvec,cmatvec_adj}.bin.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dmhm_b200.hpp"

using namespace dmhm;

static std::vector<double> read_bin(const std::string& path, size_t n) {
    std::vector<double> v(n);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(double), n, f) != n) {
        std::fprintf(stderr, "cannot read %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

static void write_bin(const std::string& path, const double* p, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(p, sizeof(double), n, f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc < 7) return 2;
    const std::string dir = argv[1];
    const int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]);
    const int levels = std::atoi(argv[4]), rank = std::atoi(argv[5]);
    const int k = std::atoi(argv[6]);
    const int N = nx * ny;
    Initialize(argc, argv);
    SetOversample(4);
    std::vector<double> c = read_bin(dir + "/coef.bin", N);
    std::vector<double> P = read_bin(dir + "/probes.bin", (size_t)N * k);

    std::vector<int> map;
    HMat2d<double>::BuildNaturalToHierarchicalMap(map, nx, ny, levels);
    std::vector<int> inv(N);
    for (int i = 0; i < N; ++i) inv[map[i]] = i;
    Sparse<double> S;
    S.height = S.width = N;
    for (int i = 0; i < N; ++i) {
        S.rowOffsets.push_back((int)S.nonzeros.size());
        const int nat = inv[i], x = nat % nx, y = nat / nx;
        int nb[4], nn = 0;
        if (x > 0) nb[nn++] = nat - 1;
        if (x < nx - 1) nb[nn++] = nat + 1;
        if (y > 0) nb[nn++] = nat - nx;
        if (y < ny - 1) nb[nn++] = nat + nx;
        for (int q = 0; q < nn; ++q) {
            S.nonzeros.push_back(-(c[nat] < c[nb[q]] ? c[nat] : c[nb[q]]));
            S.columnIndices.push_back(map[nb[q]]);
        }
        S.nonzeros.push_back(4.0 * c[nat] + 0.1);
        S.columnIndices.push_back(map[nat]);
    }
    S.rowOffsets.push_back((int)S.nonzeros.size());

    HMat2d<double> A(S, levels, rank, true, nx, ny);
    Vector<double> x(N), y;
    for (int i = 0; i < N; ++i) x.Set(i, P[i]);
    A.Multiply(1.0, x, y);
    write_bin(dir + "/matvec1.bin", y.LockedBuffer(), N);

    Dense<double> B(N, k), Cd;
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < N; ++i) B.Set(i, j, P[i + (size_t)j * N]);
    A.Multiply(1.0, B, Cd);
    write_bin(dir + "/matvec.bin", Cd.LockedBuffer(), (size_t)N * k);
    // columns 1.. of B through a locked view, into a view of a wider block
    {
        Dense<double> Bv, Wide(N, k + 2), Cv;
        Bv.LockedView(B, 0, 1, N, k - 1);
        Cv.View(Wide, 0, 2, N, k - 1);
        A.Multiply(1.0, Bv, Cv);
        write_bin(dir + "/matvec_view.bin", Wide.LockedBuffer(0, 2), (size_t)N * (k - 1));
        bool threw = false;
        try {
            Bv.Set(0, 0, 1.0);
        } catch (const std::logic_error&) {
            threw = true;
        }
        if (!threw) {
            std::fprintf(stderr, "a locked view accepted a write\n");
            return 1;
        }
    }
    // the norm estimate through the AbstractHMat interface
    {
        const AbstractHMat<double>& abs = A;
        const double est = hmat_tools::EstimateTwoNorm(abs, 1.5, 6.0);
        write_bin(dir + "/norm.bin", &est, 1);
        if (abs.Height() != N || !abs.StronglyAdmissible() || abs.NumLevels() != levels) {
            std::fprintf(stderr, "AbstractHMat queries\n");
            return 1;
        }
    }

    HMat2d<double> C;
    A.Multiply(1.0, A, C);
    C.Multiply(1.0, B, Cd);
    write_bin(dir + "/hh.bin", Cd.LockedBuffer(), (size_t)N * k);

    HMat2d<double> X;
    X.CopyFrom(A);
    SeedSerialLcg((21ULL << 32) | 17ULL);   // as after Initialize
    X.SchulzInvert(3);
    X.Multiply(1.0, B, Cd);
    write_bin(dir + "/schulz3.bin", Cd.LockedBuffer(), (size_t)N * k);
    std::printf("norm estimate %.17g\n", hmat_tools::EstimateTwoNorm(A, 1.5, 6.0));
    // single-rank DistHMat2d: the same operator, A*A under the global
    // compression tolerance (exact for sparse-built factors), against the
    // HMat2d product C computed above
    {
        SetCompressionTolerance(1e-10);
        DistHMat2d<double>::Teams teams(0);
        DistHMat2d<double> DA(S, levels, rank, true, nx, ny, teams), DC;
        if (DA.LocalHeight() != N || DA.FirstLocalRow() != 0) {
            std::fprintf(stderr, "DistHMat2d local sizes\n");
            return 1;
        }
        DA.Multiply(1.0, DA, DC, 2);
        Dense<double> R1, R2;
        DC.Multiply(1.0, B, R1);
        C.Multiply(1.0, B, R2);
        double num = 0, den = 0;
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < N; ++i) {
                const double d = R1.Get(i, j) - R2.Get(i, j);
                num += d * d;
                den += R2.Get(i, j) * R2.Get(i, j);
            }
        if (!(num <= 1e-20 * den)) {
            std::fprintf(stderr, "DistHMat2d A*A differs from HMat2d's\n");
            return 1;
        }
        if (!(DA.ParallelEstimateTwoNorm(1.5, 6.0) > 0)) return 1;
        SetCompressionTolerance(1e-16);
    }
    // one low-rank approximation of X^T X (hmat_tools::TransposeMultiply)
    LowRank<double> F;
    hmat_tools::TransposeMultiply(HMat2d<double>::SampleRank(X.MaxRank()), 1.0, X, X, F);
    if (F.Height() != N || F.Rank() < 1 || F.Rank() > X.MaxRank()) {
        std::fprintf(stderr, "low-rank product has the wrong shape\n");
        return 1;
    }
    // wire format round trip: X packed, unpacked into a fresh matrix, packed again
    std::vector<unsigned char> p1, p2;
    X.Pack(p1);
    HMat2d<double> Y;
    Y.Unpack(p1);
    Y.Pack(p2);
    if (p1 != p2 || p1.size() != X.PackedSize()) {
        std::fprintf(stderr, "pack round trip differs\n");
        return 1;
    }
    if (argc >= 12) {
        // HMat2d<std::complex<double>>: diagonal 4 + 0.2i - (k h)^2, h = 1/(side+1),
        // off-diagonals -1, rows ordered x-1, x+1, y-1, y+1, diagonal
        typedef std::complex<double> Z;
        const int side = std::atoi(argv[7]), cl = std::atoi(argv[8]), cr = std::atoi(argv[9]);
        const double kw = std::atof(argv[10]);
        const int ck = std::atoi(argv[11]);
        const int n = side * side;
        std::vector<double> cp = read_bin(dir + "/cprobes.bin", (size_t)2 * n * ck);
        std::vector<int> cmap;
        HMat2d<Z>::BuildNaturalToHierarchicalMap(cmap, side, side, cl);
        std::vector<int> cinv(n);
        for (int i = 0; i < n; ++i) cinv[cmap[i]] = i;
        const double h = 1.0 / (side + 1);
        Sparse<Z> CS;
        CS.height = CS.width = n;
        for (int i = 0; i < n; ++i) {
            CS.rowOffsets.push_back((int)CS.nonzeros.size());
            const int nat = cinv[i], x = nat % side, y = nat / side;
            int nb[4], nn = 0;
            if (x > 0) nb[nn++] = nat - 1;
            if (x < side - 1) nb[nn++] = nat + 1;
            if (y > 0) nb[nn++] = nat - side;
            if (y < side - 1) nb[nn++] = nat + side;
            for (int q = 0; q < nn; ++q) {
                CS.nonzeros.push_back(Z(-1.0, 0.0));
                CS.columnIndices.push_back(cmap[nb[q]]);
            }
            CS.nonzeros.push_back(Z(4.0 - (kw * h) * (kw * h), 0.2));
            CS.columnIndices.push_back(cmap[nat]);
        }
        CS.rowOffsets.push_back((int)CS.nonzeros.size());
        HMat2d<Z> CA(CS, cl, cr, true, side, side);
        if (CA.Height() != n || CA.MaxRank() != cr) {
            std::fprintf(stderr, "complex sizes\n");
            return 1;
        }
        Dense<Z> CB(n, ck), CC, CD;
        for (int j = 0; j < ck; ++j)
            for (int i = 0; i < n; ++i)
                CB.Set(i, j, Z(cp[2 * (i + (size_t)j * n)], cp[2 * (i + (size_t)j * n) + 1]));
        CA.Multiply(Z(1.0, 0.0), CB, CC);
        write_bin(dir + "/cmatvec.bin", reinterpret_cast<const double*>(CC.LockedBuffer()),
                  (size_t)2 * n * ck);
        CA.AdjointMultiply(Z(0.5, -0.25), CB, CD);
        write_bin(dir + "/cmatvec_adj.bin", reinterpret_cast<const double*>(CD.LockedBuffer()),
                  (size_t)2 * n * ck);
        const AbstractHMat<Z>& cabs = CA;
        if (!(hmat_tools::EstimateTwoNorm(cabs, 1.5, 6.0) > 0)) return 1;
    }
    Finalize();
    return 0;
}
