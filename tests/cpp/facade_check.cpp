// Exercises the C++ facade (include/dmhm_b200.hpp) the way the reference's
// drivers use dmhm::HMat2d (tests/HMat2d/MultiplyHMat.cpp, Invert.cpp):
// build the stencil operator from a Sparse matrix in hierarchical order,
// multiply vectors and dense blocks, form A*A, run SchulzInvert.
// Usage: facade_check <dir> <nx> <ny> <levels> <rank> <nprobes>
// Reads <dir>/coef.bin (natural order) and <dir>/probes.bin (column-major);
// writes <dir>/{matvec1,matvec,hh,schulz3}.bin.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "dmhm_b200.hpp"

using namespace dmhm_b200;

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
    Finalize();
    return 0;
}
