/*
 * Oracle driver over the unmodified reference library (test infrastructure).
 *
 * Links the reference's serial HMat2d / HMat3d (compiled from the reference
 * sources by oracle/Makefile) and runs the three hot paths on inputs that the
 * Python side writes as raw little-endian float64 files:
 *
 *   matvec  y = H x            (HMat2d::Multiply, src/HMat2d/MultiplyVector-incl.hpp:54-64,
 *                               dense form src/HMat2d/MultiplyDense-incl.hpp:56-68)
 *   hh      C = alpha A B      (HMat2d::Multiply H.H, src/HMat2d/MultiplyHMat-incl.hpp:12-187)
 *   schulz  SchulzInvert       (src/HMat2d/Invert-incl.hpp:127-196; 3-D :127-186)
 *   direct  DirectInvert       (src/HMat2d/Invert-incl.hpp:17-125; 3-D src/HMat3d/
 *                               Invert-incl.hpp:14-122), X applied to the probes
 *   lcg     first draws of the serial generator (src/core/random.cpp:13-119,
 *           include/dmhm/core/random.hpp:238-445)
 *   cmatvec / chh / cschulz   the same on HMat2d<std::complex<double>> over a
 *           shifted Helmholtz-like operator (RunComplex below)
 *   dhh / dschulz / dnorm   single-rank DistHMat2d / DistHMat3d (built with
 *           -DORACLE_WITH_DIST, RunDist below): the H.H product with its
 *           multType, SchulzInvert and ParallelEstimateTwoNorm under the global
 *           CompressionTolerance
 *
 * The operator is the grid stencil the workloads use: a 5-point (2-D) or
 * 7-point (3-D) operator in natural x-fastest order, diagonal 2*d*c_i + shift,
 * off-diagonals -min(c_i, c_j), permuted to the hierarchical ordering with
 * BuildNaturalToHierarchicalMap (src/HMat2d/HMat2d.cpp:69-87), rows built the
 * way tests/HMat2d/Invert.cpp:140-181 builds them and imported with
 * S.symmetric = false.  All vectors in and out are in hierarchical order.
 *
 * Outputs go to <out>.bin (float64) plus one JSON line on stdout with timings.
 */
#include "dmhm.hpp"
#include <cstdio>
#include <cstdlib>
#include <complex>
#include <cstring>
#include <string>
#include <vector>
#include <sys/time.h>

using namespace dmhm;

namespace {

double Now()
{
    struct timeval tv;
    gettimeofday(&tv, 0);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

struct DriverArgs
{
    std::string cmd;
    int dim, nx, ny, nz, levels, rank, oversample, strong, random;
    int nrhs, repeat, iters, count, useB, mult;
    double shift, alpha, theta, conf, stopTol, kwave, absorption, tol;
    std::string coef, coefB, x, out;
    DriverArgs()
    : dim(2), nx(32), ny(32), nz(1), levels(4), rank(8), oversample(4),
      strong(1), random(0), nrhs(1), repeat(1), iters(-1), count(16), useB(0),
      mult(2), shift(0.1), alpha(1.0), theta(1.5), conf(6.0), stopTol(1e-4), kwave(5.0),
      absorption(0.2), tol(1e-16) { }
};

std::vector<double> ReadDoubles(const std::string& path, size_t n)
{
    std::vector<double> v(n);
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
    size_t got = fread(&v[0], sizeof(double), n, f);
    fclose(f);
    if (got != n)
    { fprintf(stderr, "%s: expected %zu doubles, got %zu\n", path.c_str(), n, got); exit(2); }
    return v;
}

void WriteDoubles(const std::string& path, const std::vector<double>& v)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (!v.empty()) fwrite(&v[0], sizeof(double), v.size(), f);
    fclose(f);
}

// Build the CSR operator in hierarchical order.
void BuildSparse
(const DriverArgs& a, const std::vector<double>& c, const Vector<int>& map,
 Sparse<double>& S)
{
    const int N = a.nx * a.ny * a.nz;
    Vector<int> inv(N);
    for (int i = 0; i < N; ++i) inv[map[i]] = i;
    S.height = N; S.width = N; S.symmetric = false;
    S.nonzeros.Clear(); S.columnIndices.Clear(); S.rowOffsets.Clear();
    const int sx = 1, sy = a.nx, sz = a.nx * a.ny;
    for (int i = 0; i < N; ++i)
    {
        S.rowOffsets.PushBack(S.nonzeros.Size());
        const int nat = inv[i];
        const int x = nat % a.nx;
        const int y = (nat / a.nx) % a.ny;
        const int z = nat / (a.nx * a.ny);
        const double ci = c[nat];
        int nb[6]; int nn = 0;
        if (x > 0) nb[nn++] = nat - sx;
        if (x < a.nx - 1) nb[nn++] = nat + sx;
        if (y > 0) nb[nn++] = nat - sy;
        if (y < a.ny - 1) nb[nn++] = nat + sy;
        if (a.dim == 3)
        {
            if (z > 0) nb[nn++] = nat - sz;
            if (z < a.nz - 1) nb[nn++] = nat + sz;
        }
        for (int k = 0; k < nn; ++k)
        {
            const double cj = c[nb[k]];
            S.nonzeros.PushBack(-(ci < cj ? ci : cj));
            S.columnIndices.PushBack(map[nb[k]]);
        }
        S.nonzeros.PushBack(2.0 * a.dim * ci + a.shift);
        S.columnIndices.PushBack(map[nat]);
    }
    S.rowOffsets.PushBack(S.nonzeros.Size());
}

template<typename HMat> struct Maker;

template<> struct Maker<HMat2d<double> >
{
    static void Map(const DriverArgs& a, Vector<int>& map)
    { HMat2d<double>::BuildNaturalToHierarchicalMap(map, a.nx, a.ny, a.levels); }
    static HMat2d<double>* Make(const DriverArgs& a, const Sparse<double>& S)
    { return new HMat2d<double>(S, a.levels, a.rank, a.strong != 0, a.nx, a.ny); }
    static void Schulz(HMat2d<double>& H, const DriverArgs& a)
    { H.SchulzInvert(a.iters, a.theta, a.conf, a.stopTol); }
};

template<> struct Maker<HMat3d<double> >
{
    static void Map(const DriverArgs& a, Vector<int>& map)
    { HMat3d<double>::BuildNaturalToHierarchicalMap(map, a.nx, a.ny, a.nz, a.levels); }
    static HMat3d<double>* Make(const DriverArgs& a, const Sparse<double>& S)
    { return new HMat3d<double>(S, a.levels, a.rank, a.strong != 0, a.nx, a.ny, a.nz); }
    static void Schulz(HMat3d<double>& H, const DriverArgs& a)
    { H.SchulzInvert(a.iters, a.theta, a.conf); }
};

template<typename HMat>
void ApplyToProbes
(const HMat& H, const std::vector<double>& P, int N, int k,
 std::vector<double>& out)
{
    Dense<double> B(N, k), C;
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < N; ++i) B.Set(i, j, P[i + (size_t)j * N]);
    H.Multiply(1.0, B, C);
    out.resize((size_t)N * k);
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < N; ++i) out[i + (size_t)j * N] = C.Get(i, j);
}

template<typename HMat>
int Run(const DriverArgs& a)
{
    const int N = a.nx * a.ny * a.nz;
    Vector<int> map;
    Maker<HMat>::Map(a, map);
    std::vector<double> c = ReadDoubles(a.coef, N);
    Sparse<double> S;
    BuildSparse(a, c, map, S);
    SetOversample(a.oversample);

    HMat* A = Maker<HMat>::Make(a, S);
    if (a.random) A->SetToRandom();
    std::vector<double> result;
    double seconds = 0;
    int extraInt = 0;
    double extra = 0;

    if (a.cmd == "matvec")
    {
        std::vector<double> x = ReadDoubles(a.x, (size_t)N * a.nrhs);
        Dense<double> X(N, a.nrhs), Y;
        for (int j = 0; j < a.nrhs; ++j)
            for (int i = 0; i < N; ++i) X.Set(i, j, x[i + (size_t)j * N]);
        double t0 = Now();
        for (int rep = 0; rep < a.repeat; ++rep)
        {
            if (a.nrhs == 1)
            {
                Vector<double> xv(N), yv;
                for (int i = 0; i < N; ++i) xv[i] = x[i];
                A->Multiply(a.alpha, xv, yv);
                if (rep == a.repeat - 1)
                {
                    result.resize(N);
                    for (int i = 0; i < N; ++i) result[i] = yv[i];
                }
            }
            else
            {
                A->Multiply(a.alpha, X, Y);
                if (rep == a.repeat - 1)
                {
                    result.resize((size_t)N * a.nrhs);
                    for (int j = 0; j < a.nrhs; ++j)
                        for (int i = 0; i < N; ++i)
                            result[i + (size_t)j * N] = Y.Get(i, j);
                }
            }
        }
        seconds = (Now() - t0) / a.repeat;
    }
    else if (a.cmd == "transpose")
    {
        std::vector<double> x = ReadDoubles(a.x, (size_t)N * a.nrhs);
        Dense<double> X(N, a.nrhs), Y;
        for (int j = 0; j < a.nrhs; ++j)
            for (int i = 0; i < N; ++i) X.Set(i, j, x[i + (size_t)j * N]);
        double t0 = Now();
        A->TransposeMultiply(a.alpha, X, Y);
        seconds = Now() - t0;
        result.resize((size_t)N * a.nrhs);
        for (int j = 0; j < a.nrhs; ++j)
            for (int i = 0; i < N; ++i) result[i + (size_t)j * N] = Y.Get(i, j);
    }
    else if (a.cmd == "hh")
    {
        // C := alpha A B with B = A, or B built from a second coefficient
        // field, or B = the SetToRandom of a fresh copy (--useB 2).
        HMat* B = A;
        if (a.useB == 1)
        {
            std::vector<double> cB = ReadDoubles(a.coefB, N);
            Sparse<double> SB;
            BuildSparse(a, cB, map, SB);
            B = Maker<HMat>::Make(a, SB);
        }
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        HMat C;
        double t0 = Now();
        for (int rep = 0; rep < a.repeat; ++rep)
            A->Multiply(a.alpha, *B, C);
        seconds = (Now() - t0) / a.repeat;
        ApplyToProbes(C, P, N, a.nrhs, result);
        if (B != A) delete B;
    }
    else if (a.cmd == "schulz")
    {
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        HMat X;
        X.CopyFrom(*A);
        double t0 = Now();
        Maker<HMat>::Schulz(X, a);
        seconds = Now() - t0;
        ApplyToProbes(X, P, N, a.nrhs, result);
    }
    else if (a.cmd == "direct")
    {
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        HMat X;
        X.CopyFrom(*A);
        double t0 = Now();
        X.DirectInvert();
        seconds = Now() - t0;
        ApplyToProbes(X, P, N, a.nrhs, result);
    }
    else if (a.cmd == "schulz_trace")
    {
        // The SchulzInvert loop (src/HMat2d/Invert-incl.hpp:127-196) spelled
        // out through the public API so the per-iteration estimates of
        // ||I - X_k A||_2 and the iteration count can be recorded.  It draws
        // from the serial generator in the same order as SchulzInvert, so its
        // X equals SchulzInvert's bit for bit.
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        int numIterations = a.iters;
        bool stopflag = false;
        if (numIterations <= 0) { numIterations = 30; stopflag = true; }
        double t0 = Now();
        const double estimate = hmat_tools::EstimateTwoNorm(*A, a.theta, a.conf);
        const double alpha = 2.0 / (estimate * estimate);
        HMat X;
        X.AdjointFrom(*A);
        X.Scale(alpha);
        std::vector<double> trace;
        trace.push_back(estimate);
        int k = 0;
        for (k = 0; k < numIterations; ++k)
        {
            HMat Z;
            X.Multiply(-1.0, *A, Z);
            if (stopflag)
            {
                Z.AddConstantToDiagonal(1.0);
                const double estimateZ =
                    hmat_tools::EstimateTwoNorm(Z, a.theta, a.conf);
                trace.push_back(estimateZ);
                const double tol = (a.dim == 3 ? 1e-4 : a.stopTol);
                if (std::abs(estimateZ) < tol)
                {
                    Z.AddConstantToDiagonal(1.0);
                    HMat XCopy;
                    XCopy.CopyFrom(X);
                    Z.Multiply(1.0, XCopy, X);
                    ++k;
                    break;
                }
                Z.AddConstantToDiagonal(1.0);
            }
            else
                Z.AddConstantToDiagonal(2.0);
            HMat XCopy;
            XCopy.CopyFrom(X);
            Z.Multiply(1.0, XCopy, X);
        }
        seconds = Now() - t0;
        extraInt = k;
        ApplyToProbes(X, P, N, a.nrhs, result);
        std::vector<double> tr = trace;
        WriteDoubles(a.out + ".trace.bin", tr);
    }
    else if (a.cmd == "pack")
    {
        // the reference's wire format (src/HMat2d/Pack-incl.hpp:37-61);
        // bytes written to <out>.pack
        std::vector<byte> packed;
        Vector<byte> buf;
        A->Pack(buf);
        packed.assign(&buf[0], &buf[0] + buf.Size());
        FILE* f = fopen((a.out + ".pack").c_str(), "wb");
        if (!f) { fprintf(stderr, "cannot write pack\n"); return 2; }
        fwrite(&packed[0], 1, packed.size(), f);
        fclose(f);
        extraInt = (int)packed.size();
    }
    else if (a.cmd == "unpack_matvec")
    {
        // Unpack <coefB> (raw bytes of a packed matrix) and multiply the probes
        FILE* f = fopen(a.coefB.c_str(), "rb");
        if (!f) { fprintf(stderr, "cannot open %s\n", a.coefB.c_str()); return 2; }
        std::vector<byte> raw;
        int ch;
        while ((ch = fgetc(f)) != EOF) raw.push_back((byte)ch);
        fclose(f);
        Vector<byte> buf(raw.size());
        for (size_t i = 0; i < raw.size(); ++i) buf[i] = raw[i];
        HMat U;
        U.Unpack(buf);
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        ApplyToProbes(U, P, N, a.nrhs, result);
    }
    else if (a.cmd == "lrprod")
    {
        // F := alpha op(A) B as one low-rank matrix (hmat_tools::Multiply /
        // TransposeMultiply, include/dmhm/hmat_tools.hpp:1657-1937), sample
        // rank maxRank + Oversample(); B from --coefB (--useB 1) or A itself;
        // F applied to the probes: F.U (F.V^T P)
        HMat* B = A;
        if (a.useB == 1)
        {
            std::vector<double> cB = ReadDoubles(a.coefB, N);
            Sparse<double> SB;
            BuildSparse(a, cB, map, SB);
            B = Maker<HMat>::Make(a, SB);
        }
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        LowRank<double> F;
        const int sampleRank = a.rank + Oversample();
        double t0 = Now();
        if (a.iters == 1)
            hmat_tools::TransposeMultiply(sampleRank, a.alpha, *A, *B, F);
        else
            hmat_tools::Multiply(sampleRank, a.alpha, *A, *B, F);
        seconds = Now() - t0;
        const int r = F.U.Width();
        result.assign((size_t)N * a.nrhs, 0.0);
        for (int j = 0; j < a.nrhs; ++j)
            for (int l = 0; l < r; ++l)
            {
                double w = 0;
                for (int i = 0; i < N; ++i) w += F.V.Get(i, l) * P[i + (size_t)j * N];
                for (int i = 0; i < N; ++i) result[i + (size_t)j * N] += F.U.Get(i, l) * w;
            }
        extraInt = r;
        if (B != A) delete B;
    }
    else if (a.cmd == "norm")
    {
        double t0 = Now();
        extra = hmat_tools::EstimateTwoNorm(*A, a.theta, a.conf);
        seconds = Now() - t0;
    }
    else
    {
        fprintf(stderr, "unknown command %s\n", a.cmd.c_str());
        return 2;
    }
    if (!a.out.empty()) WriteDoubles(a.out + ".bin", result);
    printf("{\"cmd\": \"%s\", \"N\": %d, \"seconds\": %.9g, \"iterations\": %d,"
           " \"value\": %.17g}\n", a.cmd.c_str(), N, seconds, extraInt, extra);
    delete A;
    return 0;
}

#ifdef ORACLE_WITH_DIST
// Single-rank distributed classes over the serial MPI stand-in: one process
// owns the whole matrix (LocalHeight() == Height(), FirstLocalRow() == 0), so
// vectors and probes are the same hierarchical-order arrays as above.
template<typename HMat> struct DistMaker;

template<> struct DistMaker<HMat2d<double> >
{
    typedef DistHMat2d<double> D;
    static D* Make(const DriverArgs& a, const Sparse<double>& S, const D::Teams& t)
    { return new D(S, a.levels, a.rank, a.strong != 0, a.nx, a.ny, t); }
    // src/DistHMat2d/Invert-incl.hpp:14-105
    static void Schulz(D& H, const DriverArgs& a)
    { H.SchulzInvert(a.iters, a.mult, a.theta, a.conf, a.stopTol); }
};

template<> struct DistMaker<HMat3d<double> >
{
    typedef DistHMat3d<double> D;
    static D* Make(const DriverArgs& a, const Sparse<double>& S, const D::Teams& t)
    { return new D(S, a.levels, a.rank, a.strong != 0, a.nx, a.ny, a.nz, t); }
    // src/DistHMat3d/Invert-incl.hpp (stop test fixed at 1e-4)
    static void Schulz(D& H, const DriverArgs& a)
    { H.SchulzInvert(a.iters, a.mult, a.theta, a.conf); }
};

template<typename HMat>
int RunDist(const DriverArgs& a)
{
    typedef typename DistMaker<HMat>::D DHMat;
    const int N = a.nx * a.ny * a.nz;
    Vector<int> map;
    Maker<HMat>::Map(a, map);
    std::vector<double> c = ReadDoubles(a.coef, N);
    Sparse<double> S;
    BuildSparse(a, c, map, S);
    SetOversample(a.oversample);
    SetCompressionTolerance<double>(a.tol);
    typename DHMat::Teams teams(mpi::COMM_WORLD);
    DHMat* A = DistMaker<HMat>::Make(a, S, teams);
    if (A->LocalHeight() != N || A->FirstLocalRow() != 0)
    { fprintf(stderr, "single-rank DistHMat is not whole\n"); return 3; }
    std::vector<double> result;
    double seconds = 0, extra = 0;
    double t0 = Now();
    if (a.cmd == "dhh")
    {
        // C := alpha A B, B = A or built from --coefB (--useB 1)
        // (src/DistHMat2d/MultiplyHMat-incl.hpp:28-53)
        DHMat* B = A;
        if (a.useB == 1)
        {
            std::vector<double> cB = ReadDoubles(a.coefB, N);
            Sparse<double> SB;
            BuildSparse(a, cB, map, SB);
            B = DistMaker<HMat>::Make(a, SB, teams);
        }
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        DHMat C(teams);
        t0 = Now();
        A->Multiply(a.alpha, *B, C, a.mult);
        seconds = Now() - t0;
        ApplyToProbes(C, P, N, a.nrhs, result);
        if (B != A) delete B;
    }
    else if (a.cmd == "dschulz")
    {
        std::vector<double> P = ReadDoubles(a.x, (size_t)N * a.nrhs);
        t0 = Now();
        DistMaker<HMat>::Schulz(*A, a);
        seconds = Now() - t0;
        ApplyToProbes(*A, P, N, a.nrhs, result);
    }
    else if (a.cmd == "dnorm")
    {
        extra = A->ParallelEstimateTwoNorm(a.theta, a.conf);
        seconds = Now() - t0;
    }
    else
    {
        fprintf(stderr, "unknown command %s\n", a.cmd.c_str());
        return 2;
    }
    if (!a.out.empty()) WriteDoubles(a.out + ".bin", result);
    printf("{\"cmd\": \"%s\", \"N\": %d, \"seconds\": %.9g, \"iterations\": 0,"
           " \"value\": %.17g}\n", a.cmd.c_str(), N, seconds, extra);
    delete A;
    return 0;
}
#endif

// Complex-double path (HMat2d<std::complex<double>>, explicitly instantiated
// at src/HMat2d/HMat2d.cpp:1321-1324) on the shifted five-point
// Helmholtz-like operator: diagonal 4 + absorption i - (k h)^2 with
// h = 1 / (nx + 1), off-diagonals -1, natural x-fastest order permuted to the
// hierarchical order.  Commands: cmatvec (y = A x), chh (C = A A applied to
// the probes), cschulz (SchulzInvert applied to the probes).  Complex vectors
// are read and written as interleaved (re, im) float64.
int RunComplex(const DriverArgs& a)
{
    typedef std::complex<double> C;
    const int N = a.nx * a.ny;
    Vector<int> map;
    HMat2d<C>::BuildNaturalToHierarchicalMap(map, a.nx, a.ny, a.levels);
    Vector<int> inv(N);
    for (int i = 0; i < N; ++i) inv[map[i]] = i;
    const double h = 1.0 / (a.nx + 1);
    const C diag(4.0 - (a.kwave * h) * (a.kwave * h), a.absorption);
    Sparse<C> S;
    S.height = N; S.width = N; S.symmetric = false;
    for (int i = 0; i < N; ++i)
    {
        S.rowOffsets.PushBack(S.nonzeros.Size());
        const int nat = inv[i];
        const int x = nat % a.nx, y = nat / a.nx;
        int nb[4]; int nn = 0;
        if (x > 0) nb[nn++] = nat - 1;
        if (x < a.nx - 1) nb[nn++] = nat + 1;
        if (y > 0) nb[nn++] = nat - a.nx;
        if (y < a.ny - 1) nb[nn++] = nat + a.nx;
        for (int k = 0; k < nn; ++k)
        {
            S.nonzeros.PushBack(C(-1.0, 0.0));
            S.columnIndices.PushBack(map[nb[k]]);
        }
        S.nonzeros.PushBack(diag);
        S.columnIndices.PushBack(map[nat]);
    }
    S.rowOffsets.PushBack(S.nonzeros.Size());
    SetOversample(a.oversample);
    HMat2d<C> A(S, a.levels, a.rank, a.strong != 0, a.nx, a.ny);
    std::vector<double> raw = ReadDoubles(a.x, (size_t)2 * N * a.nrhs);
    Dense<C> P(N, a.nrhs), R;
    for (int j = 0; j < a.nrhs; ++j)
        for (int i = 0; i < N; ++i)
            P.Set(i, j, C(raw[2 * (i + (size_t)j * N)], raw[2 * (i + (size_t)j * N) + 1]));
    double t0 = Now();
    int its = 0;
    if (a.cmd == "cmatvec")
        A.Multiply(C(1.0, 0.0), P, R);
    else if (a.cmd == "chh")
    {
        HMat2d<C> B;
        A.Multiply(C(1.0, 0.0), A, B);
        B.Multiply(C(1.0, 0.0), P, R);
    }
    else if (a.cmd == "cschulz")
    {
        HMat2d<C> X;
        X.CopyFrom(A);
        X.SchulzInvert(a.iters, a.theta, a.conf, a.stopTol);
        X.Multiply(C(1.0, 0.0), P, R);
    }
    else { fprintf(stderr, "unknown command %s\n", a.cmd.c_str()); return 2; }
    const double seconds = Now() - t0;
    std::vector<double> out((size_t)2 * N * a.nrhs);
    for (int j = 0; j < a.nrhs; ++j)
        for (int i = 0; i < N; ++i)
        {
            const C v = R.Get(i, j);
            out[2 * (i + (size_t)j * N)] = v.real();
            out[2 * (i + (size_t)j * N) + 1] = v.imag();
        }
    if (!a.out.empty()) WriteDoubles(a.out + ".bin", out);
    printf("{\"cmd\": \"%s\", \"N\": %d, \"seconds\": %.9g, \"iterations\": %d}\n",
           a.cmd.c_str(), N, seconds, its);
    return 0;
}

int RunLcg(const DriverArgs& a)
{
    // Draw `count` serial uniforms, then `count` Gaussians of a vector and a
    // count x 3 Gaussian matrix, from the freshly seeded serial generator.
    std::vector<double> out;
    for (int i = 0; i < a.count; ++i) out.push_back(SerialUniform<double>());
    Vector<double> v(a.count);
    SerialGaussianRandomVector(v);
    for (int i = 0; i < a.count; ++i) out.push_back(v[i]);
    Dense<double> D(a.count, 3);
    SerialGaussianRandomVectors(D);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < a.count; ++i) out.push_back(D.Get(i, j));
    Dense<double> E(a.count, 3);
    ParallelGaussianRandomVectors(E);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < a.count; ++i) out.push_back(E.Get(i, j));
    WriteDoubles(a.out + ".bin", out);
    printf("{\"cmd\": \"lcg\", \"count\": %d}\n", a.count);
    return 0;
}

} // anonymous namespace

int main(int argc, char* argv[])
{
    DriverArgs a;
    if (argc < 2) { fprintf(stderr, "usage: %s cmd [--key value ...]\n", argv[0]); return 2; }
    a.cmd = argv[1];
    for (int i = 2; i + 1 < argc; i += 2)
    {
        std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "--dim") a.dim = atoi(v);
        else if (k == "--nx") a.nx = atoi(v);
        else if (k == "--ny") a.ny = atoi(v);
        else if (k == "--nz") a.nz = atoi(v);
        else if (k == "--levels") a.levels = atoi(v);
        else if (k == "--rank") a.rank = atoi(v);
        else if (k == "--oversample") a.oversample = atoi(v);
        else if (k == "--strong") a.strong = atoi(v);
        else if (k == "--random") a.random = atoi(v);
        else if (k == "--nrhs") a.nrhs = atoi(v);
        else if (k == "--repeat") a.repeat = atoi(v);
        else if (k == "--iters") a.iters = atoi(v);
        else if (k == "--count") a.count = atoi(v);
        else if (k == "--useB") a.useB = atoi(v);
        else if (k == "--mult") a.mult = atoi(v);
        else if (k == "--tol") a.tol = atof(v);
        else if (k == "--shift") a.shift = atof(v);
        else if (k == "--alpha") a.alpha = atof(v);
        else if (k == "--theta") a.theta = atof(v);
        else if (k == "--conf") a.conf = atof(v);
        else if (k == "--stopTol") a.stopTol = atof(v);
        else if (k == "--kwave") a.kwave = atof(v);
        else if (k == "--absorption") a.absorption = atof(v);
        else if (k == "--coef") a.coef = v;
        else if (k == "--coefB") a.coefB = v;
        else if (k == "--x") a.x = v;
        else if (k == "--out") a.out = v;
        else { fprintf(stderr, "unknown option %s\n", k.c_str()); return 2; }
    }
    int fakeArgc = 1;
    char** fakeArgv = argv;
    Initialize(fakeArgc, fakeArgv);
    int rc = 0;
    try
    {
        if (a.cmd == "lcg") rc = RunLcg(a);
        else if (a.cmd[0] == 'c') rc = RunComplex(a);
#ifdef ORACLE_WITH_DIST
        else if (a.cmd[0] == 'd') rc = a.dim == 2 ? RunDist<HMat2d<double> >(a)
                                                  : RunDist<HMat3d<double> >(a);
#endif
        else if (a.dim == 2) rc = Run<HMat2d<double> >(a);
        else rc = Run<HMat3d<double> >(a);
    }
    catch (std::exception& e)
    {
        fprintf(stderr, "reference threw: %s\n", e.what());
        rc = 3;
    }
    Finalize();
    return rc;
}
