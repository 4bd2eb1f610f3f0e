/*
 * dmhm_b200.hpp — header-only C++ facade with the reference's API
 * (YingzhouLi/dmhm: include/dmhm/hmat2d.hpp, hmat3d.hpp, core/dense.hpp,
 * core/vector.hpp, core/sparse.hpp, src/core/global.cpp) over the C ABI of
 * dmhm_b200.h.  Code written against dmhm::HMat2d<double> compiles against
 * dmhm_b200::HMat2d<double> after changing the namespace; every numeric
 * operation runs in the sm_100a kernels of libdmhm_b200.so.
 *
 * Scalar must be double.  Errors throw std::runtime_error (the reference
 * throws std::logic_error / std::runtime_error in the same places when built
 * without RELEASE).  Vectors are in hierarchical ordering.
 */
#ifndef DMHM_B200_HPP
#define DMHM_B200_HPP

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "dmhm_b200.h"

namespace dmhm_b200 {

inline void Check(int status) {
    if (status != HM_OK)
        throw std::runtime_error(std::string("dmhm_b200: ") + hm_last_error());
}

// ----- global state (src/core/global.cpp) ---------------------------------
namespace detail {
inline hm_context& Ctx() {
    static hm_context ctx = nullptr;
    return ctx;
}
}  // namespace detail

inline void Initialize(int& /*argc*/, char**& /*argv*/, int device = 0) {
    if (!detail::Ctx()) Check(hm_context_create(device, nullptr, &detail::Ctx()));
}
inline void Finalize() {
    if (detail::Ctx()) {
        hm_context_destroy(detail::Ctx());
        detail::Ctx() = nullptr;
    }
}
inline hm_context Context() {
    if (!detail::Ctx()) throw std::runtime_error("dmhm_b200: Initialize was not called");
    return detail::Ctx();
}
inline int Oversample() {
    int p = 0;
    Check(hm_get_oversample(Context(), &p));
    return p;
}
inline void SetOversample(int oversample) { Check(hm_set_oversample(Context(), oversample)); }
// SetCompressionTolerance / CompressionTolerance (src/core/global.cpp:
// 160-181): the global relative tolerance of the DistHMat products (default
// 1e-16, global.cpp:34).  As in the reference it does not change HMat2d /
// HMat3d, whose H*H products truncate to the fixed rank maxRank; the
// engine's per-context tolerance (hm_set_compression_tolerance) is set to it
// for the duration of each DistHMat product or inversion.
namespace detail {
inline double& DistTol() {
    static double t = 1e-16;
    return t;
}
// sets the context's tolerance for one scope and restores it
class ScopedTolerance {
  public:
    explicit ScopedTolerance(double tol) {
        Check(hm_get_compression_tolerance(Context(), &old_));
        Check(hm_set_compression_tolerance(Context(), tol));
    }
    ~ScopedTolerance() { hm_set_compression_tolerance(Context(), old_); }
    ScopedTolerance(const ScopedTolerance&) = delete;
    ScopedTolerance& operator=(const ScopedTolerance&) = delete;

  private:
    double old_ = 0.0;
};
}  // namespace detail
inline void SetCompressionTolerance(double tol) {
    if (!(tol >= 0.0 && tol < 1.0))
        throw std::runtime_error("dmhm_b200: compression tolerance must be in [0, 1)");
    detail::DistTol() = tol;
}
inline double CompressionTolerance() { return detail::DistTol(); }

// SeedSerialLcg (src/core/random.cpp:67-68): restart the serial generator
// (the one the randomized H*H sampling and EstimateTwoNorm draw from).
inline void SeedSerialLcg(uint64_t seed) {
    uint64_t s = 0, p = 0;
    Check(hm_get_lcg_states(Context(), &s, &p));
    Check(hm_set_lcg_states(Context(), seed, p));
}

// ----- containers (include/dmhm/core/vector.hpp, dense.hpp, sparse.hpp) ----
template <typename T>
class Vector {
  public:
    Vector() {}
    explicit Vector(int height) : data_(height, T(0)) {}
    int Height() const { return (int)data_.size(); }
    int Size() const { return Height(); }
    void Resize(int height) { data_.resize(height); }
    T Get(int i) const { return data_[i]; }
    void Set(int i, T v) { data_[i] = v; }
    T& operator[](int i) { return data_[i]; }
    const T& operator[](int i) const { return data_[i]; }
    T* Buffer() { return data_.data(); }
    const T* LockedBuffer() const { return data_.data(); }

  private:
    std::vector<T> data_;
};

template <typename T>
class Dense {
  public:
    Dense() : height_(0), width_(0), ldim_(1) {}
    Dense(int height, int width)
        : height_(height), width_(width), ldim_(height > 1 ? height : 1),
          data_((size_t)ldim_ * width, T(0)) {}
    int Height() const { return height_; }
    int Width() const { return width_; }
    int LDim() const { return ldim_; }
    void Resize(int height, int width) {
        if (height > ldim_) ldim_ = height > 1 ? height : 1;
        height_ = height;
        width_ = width;
        data_.resize((size_t)ldim_ * width);
    }
    T Get(int i, int j) const { return data_[i + (size_t)j * ldim_]; }
    void Set(int i, int j, T v) { data_[i + (size_t)j * ldim_] = v; }
    T* Buffer() { return data_.data(); }
    const T* LockedBuffer() const { return data_.data(); }

  private:
    int height_, width_, ldim_;
    std::vector<T> data_;
};

template <typename T>
struct Sparse {
    bool symmetric = false;
    int height = 0, width = 0;
    std::vector<T> nonzeros;
    std::vector<int> columnIndices;
    std::vector<int> rowOffsets;
};

// ----- H-matrices ------------------------------------------------------------
template <typename Scalar, int Dim>
class HMatBase {
    static_assert(sizeof(Scalar) == sizeof(double) && Scalar(0.5) != Scalar(0),
                  "dmhm_b200 supports Scalar = double");

  public:
    typedef Scalar Real;

    HMatBase() : h_(nullptr) {}
    ~HMatBase() {
        if (h_) hm_destroy(h_);
    }
    HMatBase(const HMatBase&) = delete;
    HMatBase& operator=(const HMatBase&) = delete;

    static int SampleRank(int approxRank) { return approxRank + Oversample(); }

    int Height() const { return Info().height; }
    int Width() const { return Info().width; }
    int NumLevels() const { return Info().levels; }
    int MaxRank() const { return Info().max_rank; }
    int SourceOffset() const { return 0; }
    int TargetOffset() const { return 0; }
    bool Symmetric() const { return false; }
    bool IsEmpty() const { return h_ == nullptr; }
    hm_matrix Handle() const { return h_; }

    void SetToRandom() { Check(hm_set_to_random(Need())); }

    // y := alpha H x (+ beta y)
    void Multiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const {
        y.Resize(Height());
        Check(hm_multiply_dense_host(Need(), 0, alpha, x.LockedBuffer(), x.Height(), 0.0,
                                     y.Buffer(), y.Height(), 1));
    }
    void Multiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta, Vector<Scalar>& y) const {
        Check(hm_multiply_dense_host(Need(), 0, alpha, x.LockedBuffer(), x.Height(), beta,
                                     y.Buffer(), y.Height(), 1));
    }
    void TransposeMultiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const {
        y.Resize(Width());
        Check(hm_multiply_dense_host(Need(), 1, alpha, x.LockedBuffer(), x.Height(), 0.0,
                                     y.Buffer(), y.Height(), 1));
    }
    void AdjointMultiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const {
        TransposeMultiply(alpha, x, y);
    }
    // C := alpha H B (+ beta C)
    void Multiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const {
        C.Resize(Height(), B.Width());
        Check(hm_multiply_dense_host(Need(), 0, alpha, B.LockedBuffer(), B.LDim(), 0.0,
                                     C.Buffer(), C.LDim(), B.Width()));
    }
    void Multiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta, Dense<Scalar>& C) const {
        Check(hm_multiply_dense_host(Need(), 0, alpha, B.LockedBuffer(), B.LDim(), beta,
                                     C.Buffer(), C.LDim(), B.Width()));
    }
    void TransposeMultiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const {
        C.Resize(Width(), B.Width());
        Check(hm_multiply_dense_host(Need(), 1, alpha, B.LockedBuffer(), B.LDim(), 0.0,
                                     C.Buffer(), C.LDim(), B.Width()));
    }
    void AdjointMultiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const {
        TransposeMultiply(alpha, B, C);
    }
    // C :~= alpha A B (C rebuilt) / C :~= alpha A B + beta C
    void Multiply(Scalar alpha, const HMatBase& B, HMatBase& C) const {
        Check(hm_multiply_hmat(Need(), alpha, B.Need(), &C.h_));
    }
    void Multiply(Scalar alpha, const HMatBase& B, Scalar beta, HMatBase& C) const {
        Check(hm_multiply_hmat_update(Need(), alpha, B.Need(), beta, C.Need()));
    }

    // Wire format (PackedSize / Pack / Unpack, src/HMat2d/Pack-incl.hpp:27-153):
    // the reference's bytes, readable by the reference's Unpack and back.
    std::size_t PackedSize() const {
        std::size_t n = 0;
        Check(hm_packed_size(Need(), &n));
        return n;
    }
    std::size_t Pack(std::vector<unsigned char>& packed) const {
        packed.resize(PackedSize());
        std::size_t written = 0;
        Check(hm_pack(Need(), packed.data(), packed.size(), &written));
        return written;
    }
    std::size_t Unpack(const std::vector<unsigned char>& packed) {
        hm_matrix h = nullptr;
        Check(hm_unpack(Context(), Dim, packed.data(), packed.size(), &h));
        if (h_) hm_destroy(h_);
        h_ = h;
        return packed.size();
    }

    void CopyFrom(const HMatBase& B) { Check(hm_copy(B.Need(), &h_)); }
    void AdjointFrom(const HMatBase& B) { Check(hm_transpose(B.Need(), &h_)); }
    void TransposeFrom(const HMatBase& B) { Check(hm_transpose(B.Need(), &h_)); }
    void Scale(Scalar alpha) { Check(hm_scale(Need(), alpha)); }
    // UpdateWith (HMat2d.cpp:749-781): A := alpha B + A
    void UpdateWith(Scalar alpha, const HMatBase& B) { Check(hm_update_with(Need(), alpha, B.Need())); }
    // SetToIdentity (HMat2d.cpp:652-702)
    void SetToIdentity() { Check(hm_set_to_identity(Need())); }
    // Conjugate / ConjugateFrom (HMat2d.cpp:396-472): nothing to do for real scalars
    void Conjugate() { Check(hm_conjugate_in_place(Need())); }
    void ConjugateFrom(const HMatBase& B) { CopyFrom(B); }
    void AddConstantToDiagonal(Scalar alpha) { Check(hm_add_constant_to_diagonal(Need(), alpha)); }

  protected:
    struct InfoT { int height, width, levels, max_rank; };
    InfoT Info() const {
        InfoT i{};
        Check(hm_info(Need(), &i.height, &i.width, &i.levels, &i.max_rank, nullptr, nullptr));
        return i;
    }
    hm_matrix Need() const {
        if (!h_) throw std::runtime_error("dmhm_b200: empty H-matrix");
        return h_;
    }
    void FromSparse(const Sparse<Scalar>& S, int numLevels, int maxRank, bool strong,
                    const int* sizes) {
        if (S.symmetric)
            throw std::runtime_error("dmhm_b200: symmetric storage (NODE_SYMMETRIC) "
                                     "is not supported by the H*H product and inversion");
        std::vector<int64_t> rows(S.rowOffsets.begin(), S.rowOffsets.end());
        std::vector<int32_t> cols(S.columnIndices.begin(), S.columnIndices.end());
        Check(hm_create_from_csr(Context(), Dim, sizes, numLevels, maxRank, strong ? 1 : 0,
                                 rows.data(), cols.data(), S.nonzeros.data(), &h_));
    }
    hm_matrix h_;
};

template <typename Scalar>
class HMat2d : public HMatBase<Scalar, 2> {
  public:
    HMat2d() {}
    HMat2d(const Sparse<Scalar>& S, int numLevels, int maxRank, bool stronglyAdmissible,
           int xSize, int ySize) {
        int sizes[2] = {xSize, ySize};
        this->FromSparse(S, numLevels, maxRank, stronglyAdmissible, sizes);
    }
    static void BuildNaturalToHierarchicalMap(std::vector<int>& map, int xSize, int ySize,
                                              int numLevels) {
        map.resize((size_t)xSize * ySize);
        int sizes[2] = {xSize, ySize};
        Check(hm_natural_to_hierarchical_map(2, sizes, numLevels, map.data()));
    }
    // SchulzInvert (include/dmhm/hmat2d.hpp:275-276)
    void SchulzInvert(int numIterations, Scalar theta = 1.5, Scalar confidence = 6,
                      Scalar stopTol = 1e-4) {
        Check(hm_schulz_invert(this->Need(), numIterations, theta, confidence, stopTol, nullptr,
                               nullptr, 0, nullptr));
    }
    // Mixed-precision SchulzInvert (no reference counterpart): iterations in
    // the low-precision phase while ||I - X A|| > mixedSwitch, then FP64;
    // returns the number of low-precision iterations.
    int SchulzInvertMixed(int numIterations, Scalar theta = 1.5, Scalar confidence = 6,
                          Scalar stopTol = 1e-4, Scalar mixedSwitch = 0.1) {
        int its = 0, low = 0;
        Check(hm_schulz_invert_mixed(this->Need(), numIterations, theta, confidence, stopTol,
                                     mixedSwitch, &its, &low, nullptr, 0, nullptr));
        return low;
    }
};

template <typename Scalar>
class HMat3d : public HMatBase<Scalar, 3> {
  public:
    HMat3d() {}
    HMat3d(const Sparse<Scalar>& S, int numLevels, int maxRank, bool stronglyAdmissible,
           int xSize, int ySize, int zSize) {
        int sizes[3] = {xSize, ySize, zSize};
        this->FromSparse(S, numLevels, maxRank, stronglyAdmissible, sizes);
    }
    static void BuildNaturalToHierarchicalMap(std::vector<int>& map, int xSize, int ySize,
                                              int zSize, int numLevels) {
        map.resize((size_t)xSize * ySize * zSize);
        int sizes[3] = {xSize, ySize, zSize};
        Check(hm_natural_to_hierarchical_map(3, sizes, numLevels, map.data()));
    }
    // SchulzInvert (include/dmhm/hmat3d.hpp:283): stop tolerance fixed at 1e-4
    // (src/HMat3d/Invert-incl.hpp:168)
    void SchulzInvert(int numIterations, Scalar theta = 1.5, Scalar confidence = 6) {
        Check(hm_schulz_invert(this->Need(), numIterations, theta, confidence, 1e-4, nullptr,
                               nullptr, 0, nullptr));
    }
};

// ----- single-rank DistHMat2d / DistHMat3d ----------------------------------
// include/dmhm/dist_hmat2d.hpp (and dist_hmat3d.hpp) on one process: the
// whole matrix is local (LocalHeight() = Height(), FirstLocalRow() = 0), the
// products truncate by the global CompressionTolerance (SVDTrunc,
// src/DistHMat2d/Truncation-incl.hpp:37-63) instead of to the fixed rank,
// and multType (the reference's accumulation schedules, MultiplyHMat-incl.hpp:
// 28-52) has no effect on the result here.  The reference compresses with
// two-sided sketches and Gram eigendecompositions; this engine rounds with
// QR and a Jacobi SVD under the same truncation rule, so results agree to
// the tolerance's scale, not bit for bit.
// Teams(mpi::Comm) of the distributed classes: one team of one process.
class DistTeams {
  public:
    explicit DistTeams(int comm = 0) { (void)comm; }
    int NumLevels() const { return 1; }
    int TeamLevel(int) const { return 0; }
};

namespace detail {
template <typename Base>
class DistOps : public Base {
  public:
    typedef typename Base::Real Real;
    typedef DistTeams Teams;

    int LocalHeight() const { return this->Height(); }
    int LocalWidth() const { return this->Width(); }
    int FirstLocalRow() const { return 0; }
    int FirstLocalCol() const { return 0; }

    // ParallelEstimateTwoNorm (src/DistHMat2d/Norm-incl.hpp:12-77)
    Real ParallelEstimateTwoNorm(Real theta, Real confidence) {
        double est = 0;
        Check(hm_estimate_two_norm(this->Handle(), theta, confidence, &est));
        return est;
    }
    using Base::Multiply;
    // C := alpha A B (MultiplyHMat-incl.hpp:28-52)
    void Multiply(double alpha, DistOps& B, DistOps& C, int multType = 2) {
        (void)multType;
        ScopedTolerance tol(CompressionTolerance());
        Base::Multiply(alpha, B, C);
    }
    // SchulzInvert (src/DistHMat2d/Invert-incl.hpp:14-105)
    void SchulzInvert(int numIterations, int multType = 2, Real theta = 1.5,
                      Real confidence = 6, Real stopTol = 1e-4, bool printRank = false) {
        (void)multType;
        (void)printRank;
        ScopedTolerance tol(CompressionTolerance());
        Check(hm_schulz_invert(this->Handle(), numIterations, theta, confidence, stopTol,
                               nullptr, nullptr, 0, nullptr));
    }
};
}  // namespace detail

template <typename Scalar>
class DistHMat2d : public detail::DistOps<HMat2d<Scalar>> {
  public:
    DistHMat2d() {}
    DistHMat2d(const Sparse<Scalar>& S, int numLevels, int maxRank, bool stronglyAdmissible,
               int xSize, int ySize, const DistTeams& teams) {
        (void)teams;
        int sizes[2] = {xSize, ySize};
        this->FromSparse(S, numLevels, maxRank, stronglyAdmissible, sizes);
    }
};

template <typename Scalar>
class DistHMat3d : public detail::DistOps<HMat3d<Scalar>> {
  public:
    DistHMat3d() {}
    DistHMat3d(const Sparse<Scalar>& S, int numLevels, int maxRank, bool stronglyAdmissible,
               int xSize, int ySize, int zSize, const DistTeams& teams) {
        (void)teams;
        int sizes[3] = {xSize, ySize, zSize};
        this->FromSparse(S, numLevels, maxRank, stronglyAdmissible, sizes);
    }
};

// LowRank<Scalar> (include/dmhm/core/low_rank.hpp:22-38): A = U V^T.
template <typename Scalar>
struct LowRank {
    Dense<Scalar> U, V;
    int Height() const { return U.Height(); }
    int Width() const { return V.Height(); }
    int Rank() const { return U.Width(); }
};

namespace hmat_tools {
// EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548)
template <typename Scalar, int Dim>
Scalar EstimateTwoNorm(const HMatBase<Scalar, Dim>& A, Scalar theta, Scalar confidence) {
    double est = 0;
    Check(hm_estimate_two_norm(A.Handle(), theta, confidence, &est));
    return est;
}


namespace detail {
template <typename Scalar, int Dim>
void LowRankProduct(int op, int sampleRank, Scalar alpha, const HMatBase<Scalar, Dim>& A,
                    const HMatBase<Scalar, Dim>& B, LowRank<Scalar>& F) {
    const int n = A.Height();
    const int cap = std::max(1, std::min(std::min(A.MaxRank(), B.MaxRank()), n));
    F.U.Resize(n, cap);
    F.V.Resize(n, cap);
    int r = 0;
    Check(hm_low_rank_product(A.Handle(), op, alpha, B.Handle(), sampleRank, F.U.Buffer(),
                              F.U.LDim(), F.V.Buffer(), F.V.LDim(), cap, &r));
    F.U.Resize(n, r);
    F.V.Resize(n, r);
}
}  // namespace detail

// F := alpha A B, alpha A^T B, alpha A^H B as one low-rank matrix
// (include/dmhm/hmat_tools.hpp:1657-1746, 1848-1937, 2039-)
template <typename Scalar, int Dim>
void Multiply(int sampleRank, Scalar alpha, const HMatBase<Scalar, Dim>& A,
              const HMatBase<Scalar, Dim>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(0, sampleRank, alpha, A, B, F);
}
template <typename Scalar, int Dim>
void TransposeMultiply(int sampleRank, Scalar alpha, const HMatBase<Scalar, Dim>& A,
                       const HMatBase<Scalar, Dim>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(1, sampleRank, alpha, A, B, F);
}
template <typename Scalar, int Dim>
void AdjointMultiply(int sampleRank, Scalar alpha, const HMatBase<Scalar, Dim>& A,
                     const HMatBase<Scalar, Dim>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(2, sampleRank, alpha, A, B, F);
}
}  // namespace hmat_tools

}  // namespace dmhm_b200

#endif  // DMHM_B200_HPP
