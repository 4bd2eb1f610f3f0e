/*
 * dmhm_b200.hpp — header-only C++ facade with the reference's API
 * (YingzhouLi/dmhm: include/dmhm/hmat2d.hpp, hmat3d.hpp,
 * core/abstract_hmat.hpp, core/dense.hpp, core/vector.hpp, core/sparse.hpp,
 * core/low_rank.hpp, hmat_tools.hpp, src/core/global.cpp) over the C ABI of
 * dmhm_b200.h.  Code written against dmhm::HMat2d<double> compiles against
 * it unchanged (namespace dmhm is an alias of dmhm_b200, see the end of this
 * file); every numeric operation runs in the sm_100a kernels of
 * libdmhm_b200.so.
 *
 * Scalar = double or std::complex<double> (the reference's explicit
 * instantiations, src/HMat2d/HMat2d.cpp:1321-1324, without the float ones).
 * A complex matrix takes real alpha / beta in the H*H product and in
 * UpdateWith, and cannot be packed; the hmat_tools low-rank products are
 * real.  Errors throw std::runtime_error (the reference throws
 * std::logic_error / std::runtime_error in the same places when built
 * without RELEASE); misuse of a view throws std::logic_error.  Vectors are
 * in hierarchical ordering.
 */
#ifndef DMHM_B200_HPP
#define DMHM_B200_HPP

#include <algorithm>
#include <complex>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <type_traits>
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
// Owning storage or a view of another container's memory (View: writable,
// LockedView: read-only), with the reference's method names.  Resizing a
// view, or writing through a locked view, throws std::logic_error.
template <typename T>
class Vector {
  public:
    Vector() : height_(0), viewing_(false), locked_(false), buf_(nullptr), lbuf_(nullptr) {}
    explicit Vector(int height, T x = T(0))
        : height_(height), viewing_(false), locked_(false), mem_(height, x) {
        Own();
    }
    Vector(int height, T* buffer)
        : height_(height), viewing_(true), locked_(false), buf_(buffer), lbuf_(buffer) {}
    Vector(int height, const T* lockedBuffer)
        : height_(height), viewing_(true), locked_(true), buf_(nullptr), lbuf_(lockedBuffer) {}
    Vector(const Vector& x)
        : height_(x.height_), viewing_(false), locked_(false),
          mem_(x.lbuf_, x.lbuf_ + x.height_) {
        Own();
    }
    Vector& operator=(const Vector& x) {
        if (this != &x) {
            if (viewing_) throw std::logic_error("dmhm_b200: cannot assign to a view");
            mem_.assign(x.lbuf_, x.lbuf_ + x.height_);
            height_ = x.height_;
            Own();
        }
        return *this;
    }
    int Height() const { return height_; }
    int Size() const { return height_; }
    void Resize(int height) {
        if (viewing_ && height != height_)
            throw std::logic_error("dmhm_b200: cannot resize a view");
        if (!viewing_) {
            mem_.resize(height);
            height_ = height;
            Own();
        }
    }
    void Clear() {
        mem_.clear();
        height_ = 0;
        viewing_ = locked_ = false;
        Own();
    }
    T Get(int i) const { return lbuf_[i]; }
    void Set(int i, T v) { Writable()[i] = v; }
    T& operator[](int i) { return Writable()[i]; }
    const T& operator[](int i) const { return lbuf_[i]; }
    T* Buffer(int i = 0) { return Writable() + i; }
    const T* LockedBuffer(int i = 0) const { return lbuf_ + i; }
    void View(Vector& x) { View(x, 0, x.Height()); }
    void View(Vector& x, int i, int height) {
        mem_.clear();
        height_ = height;
        viewing_ = true;
        locked_ = false;
        buf_ = x.Buffer(i);
        lbuf_ = buf_;
    }
    void LockedView(const Vector& x) { LockedView(x, 0, x.Height()); }
    void LockedView(const Vector& x, int i, int height) {
        mem_.clear();
        height_ = height;
        viewing_ = true;
        locked_ = true;
        buf_ = nullptr;
        lbuf_ = x.LockedBuffer(i);
    }
    void Print(const std::string tag, std::ostream& os = std::cout) const {
        os << tag << "\n";
        for (int i = 0; i < height_; ++i) os << lbuf_[i] << "\n";
        os << std::endl;
    }

  private:
    void Own() {
        buf_ = mem_.data();
        lbuf_ = buf_;
    }
    T* Writable() {
        if (locked_) throw std::logic_error("dmhm_b200: cannot write through a locked view");
        return buf_;
    }
    int height_;
    bool viewing_, locked_;
    std::vector<T> mem_;
    T* buf_;
    const T* lbuf_;
};

template <typename T>
class Dense {
  public:
    Dense() : height_(0), width_(0), ldim_(1), viewing_(false), locked_(false) { Own(); }
    Dense(int height, int width) : Dense(height, width, height > 1 ? height : 1) {}
    Dense(int height, int width, int ldim)
        : height_(height), width_(width), ldim_(ldim), viewing_(false), locked_(false),
          mem_((size_t)ldim * width, T(0)) {
        if (ldim < std::max(height, 1))
            throw std::logic_error("dmhm_b200: leading dimension smaller than the height");
        Own();
    }
    Dense(T* buffer, int height, int width, int ldim)
        : height_(height), width_(width), ldim_(ldim), viewing_(true), locked_(false),
          buf_(buffer), lbuf_(buffer) {}
    Dense(const T* lockedBuffer, int height, int width, int ldim)
        : height_(height), width_(width), ldim_(ldim), viewing_(true), locked_(true),
          buf_(nullptr), lbuf_(lockedBuffer) {}
    Dense(const Dense& A) : height_(0), width_(0), ldim_(1), viewing_(false), locked_(false) {
        CopyFrom(A);
    }
    Dense& operator=(const Dense& A) {
        if (this != &A) {
            if (viewing_) throw std::logic_error("dmhm_b200: cannot assign to a view");
            CopyFrom(A);
        }
        return *this;
    }
    int Height() const { return height_; }
    int Width() const { return width_; }
    int LDim() const { return ldim_; }
    int Size() const { return height_ * width_; }
    bool IsEmpty() const { return height_ == 0 || width_ == 0; }
    void Resize(int height, int width) {
        Resize(height, width, std::max(std::max(height, 1), viewing_ ? ldim_ : 1));
    }
    void Resize(int height, int width, int ldim) {
        if (viewing_) {
            if (height != height_ || width != width_)
                throw std::logic_error("dmhm_b200: cannot resize a view");
            return;
        }
        if (ldim < std::max(height, 1))
            throw std::logic_error("dmhm_b200: leading dimension smaller than the height");
        if (ldim != ldim_) {   // keep the entries that stay (as the reference's Resize)
            std::vector<T> m((size_t)ldim * width, T(0));
            for (int j = 0; j < std::min(width, width_); ++j)
                for (int i = 0; i < std::min(height, height_); ++i)
                    m[i + (size_t)j * ldim] = mem_[i + (size_t)j * ldim_];
            mem_.swap(m);
        } else {
            mem_.resize((size_t)ldim * width);
        }
        height_ = height;
        width_ = width;
        ldim_ = ldim;
        Own();
    }
    void Clear() {
        mem_.clear();
        height_ = width_ = 0;
        ldim_ = 1;
        viewing_ = locked_ = false;
        Own();
    }
    T Get(int i, int j) const { return lbuf_[i + (size_t)j * ldim_]; }
    void Set(int i, int j, T v) { Writable()[i + (size_t)j * ldim_] = v; }
    T* Buffer(int i = 0, int j = 0) { return Writable() + i + (size_t)j * ldim_; }
    const T* LockedBuffer(int i = 0, int j = 0) const { return lbuf_ + i + (size_t)j * ldim_; }
    void View(Dense& A) { View(A, 0, 0, A.Height(), A.Width()); }
    void View(Dense& A, int i, int j, int height, int width) {
        mem_.clear();
        height_ = height;
        width_ = width;
        ldim_ = A.LDim();
        viewing_ = true;
        locked_ = false;
        buf_ = A.Buffer(i, j);
        lbuf_ = buf_;
    }
    void LockedView(const Dense& A) { LockedView(A, 0, 0, A.Height(), A.Width()); }
    void LockedView(const Dense& A, int i, int j, int height, int width) {
        mem_.clear();
        height_ = height;
        width_ = width;
        ldim_ = A.LDim();
        viewing_ = true;
        locked_ = true;
        buf_ = nullptr;
        lbuf_ = A.LockedBuffer(i, j);
    }
    void Print(const std::string tag, std::ostream& os = std::cout) const {
        os << tag << "\n";
        for (int i = 0; i < height_; ++i) {
            for (int j = 0; j < width_; ++j) os << Get(i, j) << " ";
            os << "\n";
        }
        os << std::endl;
    }

  private:
    void Own() {
        buf_ = mem_.data();
        lbuf_ = buf_;
    }
    void CopyFrom(const Dense& A) {
        height_ = A.height_;
        width_ = A.width_;
        ldim_ = std::max(A.height_, 1);
        mem_.assign((size_t)ldim_ * width_, T(0));
        for (int j = 0; j < width_; ++j)
            for (int i = 0; i < height_; ++i) mem_[i + (size_t)j * ldim_] = A.Get(i, j);
        viewing_ = locked_ = false;
        Own();
    }
    T* Writable() {
        if (locked_) throw std::logic_error("dmhm_b200: cannot write through a locked view");
        return buf_;
    }
    int height_, width_, ldim_;
    bool viewing_, locked_;
    std::vector<T> mem_;
    T* buf_ = nullptr;
    const T* lbuf_ = nullptr;
};

template <typename T>
struct Sparse {
    bool symmetric = false;
    int height = 0, width = 0;
    std::vector<T> nonzeros;
    std::vector<int> columnIndices;
    std::vector<int> rowOffsets;
};

// LowRank<Scalar> (include/dmhm/core/low_rank.hpp:22-38): A = U V^T.
template <typename Scalar>
struct LowRank {
    Dense<Scalar> U, V;
    int Height() const { return U.Height(); }
    int Width() const { return V.Height(); }
    int Rank() const { return U.Width(); }
};

// ----- AbstractHMat (include/dmhm/core/abstract_hmat.hpp:20-93) --------------
// The virtual interface hmat_tools::EstimateTwoNorm and the randomized
// hmat_tools products take; HMat2d, HMat3d and the single-rank DistHMat
// classes implement it.  Handle() exposes the engine matrix behind it.
template <typename Scalar>
class AbstractHMat {
  public:
    virtual ~AbstractHMat() {}
    virtual int Height() const = 0;
    virtual int Width() const = 0;
    virtual int NumLevels() const = 0;
    virtual int MaxRank() const = 0;
    virtual int SourceOffset() const = 0;
    virtual int TargetOffset() const = 0;
    virtual bool Symmetric() const = 0;
    virtual bool StronglyAdmissible() const = 0;
    virtual void Print(const std::string tag, std::ostream& os = std::cout) const = 0;
    virtual void Multiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                          Vector<Scalar>& y) const = 0;
    virtual void Multiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const = 0;
    virtual void TransposeMultiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                                   Vector<Scalar>& y) const = 0;
    virtual void TransposeMultiply(Scalar alpha, const Vector<Scalar>& x,
                                   Vector<Scalar>& y) const = 0;
    virtual void AdjointMultiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                                 Vector<Scalar>& y) const = 0;
    virtual void AdjointMultiply(Scalar alpha, const Vector<Scalar>& x,
                                 Vector<Scalar>& y) const = 0;
    virtual void Multiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                          Dense<Scalar>& C) const = 0;
    virtual void Multiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const = 0;
    virtual void TransposeMultiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                                   Dense<Scalar>& C) const = 0;
    virtual void TransposeMultiply(Scalar alpha, const Dense<Scalar>& B,
                                   Dense<Scalar>& C) const = 0;
    virtual void AdjointMultiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                                 Dense<Scalar>& C) const = 0;
    virtual void AdjointMultiply(Scalar alpha, const Dense<Scalar>& B,
                                 Dense<Scalar>& C) const = 0;
    virtual hm_matrix Handle() const = 0;
};

// ----- H-matrices ------------------------------------------------------------
namespace detail {
// Scalar = double or std::complex<double> (the complex matrix lives on the
// device in real form: two rows per grid point, rank 2r; the engine's
// complex entry points take interleaved complex arrays)
template <typename S> struct ScalarTraits;
template <> struct ScalarTraits<double> {
    static const bool is_complex = false;
    static const int dof = 1;
};
template <> struct ScalarTraits<std::complex<double>> {
    static const bool is_complex = true;
    static const int dof = 2;
};
inline double Re(double a) { return a; }
inline double Im(double) { return 0.0; }
inline double Re(const std::complex<double>& a) { return a.real(); }
inline double Im(const std::complex<double>& a) { return a.imag(); }
inline const double* Doubles(const double* p) { return p; }
inline double* Doubles(double* p) { return p; }
inline const double* Doubles(const std::complex<double>* p) {
    return reinterpret_cast<const double*>(p);
}
inline double* Doubles(std::complex<double>* p) { return reinterpret_cast<double*>(p); }
template <typename S> double RealOnly(const S& a, const char* what) {
    if (Im(a) != 0.0)
        throw std::runtime_error(std::string("dmhm_b200: ") + what +
                                 " takes a real scalar for a complex matrix");
    return Re(a);
}
}  // namespace detail

template <typename Scalar, int Dim>
class HMatBase : public AbstractHMat<Scalar> {
    typedef detail::ScalarTraits<Scalar> Traits;

  public:
    typedef double Real;

    HMatBase() : h_(nullptr) {}
    ~HMatBase() {
        if (h_) hm_destroy(h_);
    }
    HMatBase(const HMatBase&) = delete;
    HMatBase& operator=(const HMatBase&) = delete;

    static int SampleRank(int approxRank) { return approxRank + Oversample(); }

    int Height() const override { return Info().height / Traits::dof; }
    int Width() const override { return Info().width / Traits::dof; }
    int NumLevels() const override { return Info().levels; }
    int MaxRank() const override { return Info().max_rank / Traits::dof; }
    int SourceOffset() const override { return 0; }
    int TargetOffset() const override { return 0; }
    bool Symmetric() const override { return false; }
    bool StronglyAdmissible() const override {
        int s = 0;
        Check(hm_structure(Need(), nullptr, nullptr, &s, nullptr));
        return s != 0;
    }
    bool IsEmpty() const { return h_ == nullptr; }
    hm_matrix Handle() const override { return h_; }

    // The equivalent dense matrix, row by row (formed by products with
    // unit vectors; meant for small matrices, as the reference's Print).
    void Print(const std::string tag, std::ostream& os = std::cout) const override {
        const int n = Height(), w = Width();
        os << tag << "\n";
        const int nb = 64;
        std::vector<std::vector<Scalar>> rows((size_t)n, std::vector<Scalar>((size_t)w));
        for (int j0 = 0; j0 < w; j0 += nb) {
            const int k = std::min(nb, w - j0);
            Dense<Scalar> E(w, k), C;
            for (int j = 0; j < k; ++j) E.Set(j0 + j, j, Scalar(1));
            Multiply(Scalar(1), E, C);
            for (int j = 0; j < k; ++j)
                for (int i = 0; i < n; ++i) rows[i][j0 + j] = C.Get(i, j);
        }
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < w; ++j) os << rows[i][j] << " ";
            os << "\n";
        }
        os << std::endl;
    }

    void SetToRandom() { Check(hm_set_to_random(Need())); }

    // y := alpha op(H) x (+ beta y), C := alpha op(H) B (+ beta C)
    void Multiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const override {
        y.Resize(Height());
        Apply(0, alpha, x.LockedBuffer(), x.Height(), Scalar(0), y.Buffer(), y.Height(), 1);
    }
    void Multiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                  Vector<Scalar>& y) const override {
        Apply(0, alpha, x.LockedBuffer(), x.Height(), beta, y.Buffer(), y.Height(), 1);
    }
    void TransposeMultiply(Scalar alpha, const Vector<Scalar>& x,
                           Vector<Scalar>& y) const override {
        y.Resize(Width());
        Apply(1, alpha, x.LockedBuffer(), x.Height(), Scalar(0), y.Buffer(), y.Height(), 1);
    }
    void TransposeMultiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                           Vector<Scalar>& y) const override {
        Apply(1, alpha, x.LockedBuffer(), x.Height(), beta, y.Buffer(), y.Height(), 1);
    }
    void AdjointMultiply(Scalar alpha, const Vector<Scalar>& x, Vector<Scalar>& y) const override {
        y.Resize(Width());
        Apply(2, alpha, x.LockedBuffer(), x.Height(), Scalar(0), y.Buffer(), y.Height(), 1);
    }
    void AdjointMultiply(Scalar alpha, const Vector<Scalar>& x, Scalar beta,
                         Vector<Scalar>& y) const override {
        Apply(2, alpha, x.LockedBuffer(), x.Height(), beta, y.Buffer(), y.Height(), 1);
    }
    void Multiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const override {
        C.Resize(Height(), B.Width());
        Apply(0, alpha, B.LockedBuffer(), B.LDim(), Scalar(0), C.Buffer(), C.LDim(), B.Width());
    }
    void Multiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                  Dense<Scalar>& C) const override {
        Apply(0, alpha, B.LockedBuffer(), B.LDim(), beta, C.Buffer(), C.LDim(), B.Width());
    }
    void TransposeMultiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const override {
        C.Resize(Width(), B.Width());
        Apply(1, alpha, B.LockedBuffer(), B.LDim(), Scalar(0), C.Buffer(), C.LDim(), B.Width());
    }
    void TransposeMultiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                           Dense<Scalar>& C) const override {
        Apply(1, alpha, B.LockedBuffer(), B.LDim(), beta, C.Buffer(), C.LDim(), B.Width());
    }
    void AdjointMultiply(Scalar alpha, const Dense<Scalar>& B, Dense<Scalar>& C) const override {
        C.Resize(Width(), B.Width());
        Apply(2, alpha, B.LockedBuffer(), B.LDim(), Scalar(0), C.Buffer(), C.LDim(), B.Width());
    }
    void AdjointMultiply(Scalar alpha, const Dense<Scalar>& B, Scalar beta,
                         Dense<Scalar>& C) const override {
        Apply(2, alpha, B.LockedBuffer(), B.LDim(), beta, C.Buffer(), C.LDim(), B.Width());
    }
    // C :~= alpha A B (C rebuilt) / C :~= alpha A B + beta C (a complex
    // matrix takes real alpha and beta here)
    void Multiply(Scalar alpha, const HMatBase& B, HMatBase& C) const {
        Check(hm_multiply_hmat(Need(), detail::RealOnly(alpha, "the H*H product"), B.Need(),
                               &C.h_));
    }
    void Multiply(Scalar alpha, const HMatBase& B, Scalar beta, HMatBase& C) const {
        Check(hm_multiply_hmat_update(Need(), detail::RealOnly(alpha, "the H*H product"),
                                      B.Need(), detail::RealOnly(beta, "the H*H product"),
                                      C.Need()));
    }

    // Wire format (PackedSize / Pack / Unpack, src/HMat2d/Pack-incl.hpp:27-153):
    // the reference's bytes, readable by the reference's Unpack and back
    // (real matrices).
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
        if (Traits::is_complex)
            throw std::runtime_error("dmhm_b200: Unpack reads real matrices only");
        hm_matrix h = nullptr;
        Check(hm_unpack(Context(), Dim, packed.data(), packed.size(), &h));
        if (h_) hm_destroy(h_);
        h_ = h;
        return packed.size();
    }

    void CopyFrom(const HMatBase& B) { Check(hm_copy(B.Need(), &h_)); }
    // AdjointFrom (HMat2d.cpp:548-614); for a complex matrix TransposeFrom
    // (:477-546) does not conjugate
    void AdjointFrom(const HMatBase& B) { Check(hm_transpose(B.Need(), &h_)); }
    void TransposeFrom(const HMatBase& B) {
        if (Traits::is_complex) Check(hm_transpose_complex(B.Need(), &h_));
        else Check(hm_transpose(B.Need(), &h_));
    }
    void Scale(Scalar alpha) {
        if (Traits::is_complex)
            Check(hm_scale_complex(Need(), detail::Re(alpha), detail::Im(alpha)));
        else Check(hm_scale(Need(), detail::Re(alpha)));
    }
    // UpdateWith (HMat2d.cpp:749-781): A := alpha B + A
    void UpdateWith(Scalar alpha, const HMatBase& B) {
        Check(hm_update_with(Need(), detail::RealOnly(alpha, "UpdateWith"), B.Need()));
    }
    // SetToIdentity (HMat2d.cpp:652-702)
    void SetToIdentity() { Check(hm_set_to_identity(Need())); }
    // Conjugate / ConjugateFrom (HMat2d.cpp:396-472)
    void Conjugate() { Check(hm_conjugate_in_place(Need())); }
    void ConjugateFrom(const HMatBase& B) {
        if (Traits::is_complex) Check(hm_conjugate(B.Need(), &h_));
        else CopyFrom(B);
    }
    // DirectInvert (src/HMat2d/Invert-incl.hpp:17-125; HMat3d :14-122):
    // A := inv(A) by recursive Schur complements (real matrices)
    void DirectInvert() {
        if (Traits::is_complex)
            throw std::runtime_error("dmhm_b200: DirectInvert is built for real matrices");
        Check(hm_direct_invert(Need()));
    }
    void AddConstantToDiagonal(Scalar alpha) {
        if (Traits::is_complex)
            Check(hm_add_constant_to_diagonal_complex(Need(), detail::Re(alpha),
                                                      detail::Im(alpha)));
        else Check(hm_add_constant_to_diagonal(Need(), detail::Re(alpha)));
    }

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
    // op: 0 = H, 1 = H^T, 2 = H^H
    void Apply(int op, Scalar alpha, const Scalar* B, int ldb, Scalar beta, Scalar* C, int ldc,
               int k) const {
        if (Traits::is_complex)
            Check(hm_multiply_dense_complex_host(Need(), op, detail::Re(alpha), detail::Im(alpha),
                                                 detail::Doubles(B), ldb, detail::Re(beta),
                                                 detail::Im(beta), detail::Doubles(C), ldc, k));
        else
            Check(hm_multiply_dense_host(Need(), op == 0 ? 0 : 1, detail::Re(alpha),
                                         detail::Doubles(B), ldb, detail::Re(beta),
                                         detail::Doubles(C), ldc, k));
    }
    void FromSparse(const Sparse<Scalar>& S, int numLevels, int maxRank, bool strong,
                    const int* sizes) {
        if (S.symmetric)
            throw std::runtime_error("dmhm_b200: symmetric storage (NODE_SYMMETRIC) "
                                     "is not supported by the H*H product and inversion");
        std::vector<int64_t> rows(S.rowOffsets.begin(), S.rowOffsets.end());
        std::vector<int32_t> cols(S.columnIndices.begin(), S.columnIndices.end());
        if (Traits::is_complex)
            Check(hm_create_from_csr_complex(Context(), Dim, sizes, numLevels, maxRank,
                                             strong ? 1 : 0, rows.data(), cols.data(),
                                             detail::Doubles(S.nonzeros.data()), &h_));
        else
            Check(hm_create_from_csr(Context(), Dim, sizes, numLevels, maxRank, strong ? 1 : 0,
                                     rows.data(), cols.data(), detail::Doubles(S.nonzeros.data()),
                                     &h_));
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
    void SchulzInvert(int numIterations, double theta = 1.5, double confidence = 6,
                      double stopTol = 1e-4) {
        Check(hm_schulz_invert(this->Need(), numIterations, theta, confidence, stopTol, nullptr,
                               nullptr, 0, nullptr));
    }
    // Mixed-precision SchulzInvert (no reference counterpart): iterations in
    // the low-precision phase while ||I - X A|| > mixedSwitch, then FP64;
    // returns the number of low-precision iterations.
    int SchulzInvertMixed(int numIterations, double theta = 1.5, double confidence = 6,
                          double stopTol = 1e-4, double mixedSwitch = 0.1) {
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
    void SchulzInvert(int numIterations, double theta = 1.5, double confidence = 6) {
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

namespace hmat_tools {
// EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548) of any
// AbstractHMat (real, or complex in its real form: the same norm)
template <typename Scalar>
double EstimateTwoNorm(const AbstractHMat<Scalar>& A, double theta, double confidence) {
    double est = 0;
    Check(hm_estimate_two_norm(A.Handle(), theta, confidence, &est));
    return est;
}

namespace detail {
template <typename Scalar>
void LowRankProduct(int op, int sampleRank, Scalar alpha, const AbstractHMat<Scalar>& A,
                    const AbstractHMat<Scalar>& B, LowRank<Scalar>& F) {
    static_assert(std::is_same<Scalar, double>::value,
                  "dmhm_b200: the hmat_tools low-rank products are built for real matrices");
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
template <typename Scalar>
void Multiply(int sampleRank, Scalar alpha, const AbstractHMat<Scalar>& A,
              const AbstractHMat<Scalar>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(0, sampleRank, alpha, A, B, F);
}
template <typename Scalar>
void TransposeMultiply(int sampleRank, Scalar alpha, const AbstractHMat<Scalar>& A,
                       const AbstractHMat<Scalar>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(1, sampleRank, alpha, A, B, F);
}
template <typename Scalar>
void AdjointMultiply(int sampleRank, Scalar alpha, const AbstractHMat<Scalar>& A,
                     const AbstractHMat<Scalar>& B, LowRank<Scalar>& F) {
    detail::LowRankProduct(2, sampleRank, alpha, A, B, F);
}
}  // namespace hmat_tools

}  // namespace dmhm_b200

// Code written against the reference's namespace compiles unchanged: dmhm
// names this library unless the including program defines
// DMHM_B200_NO_DMHM_ALIAS (for instance to link the reference beside it).
#ifndef DMHM_B200_NO_DMHM_ALIAS
namespace dmhm = dmhm_b200;
#endif

#endif  // DMHM_B200_HPP
