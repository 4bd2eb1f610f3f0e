// Position-independent operation lists (used by lowrank.cu and dense_ops.cu).
#pragma once
#include <type_traits>
#include <vector>

namespace hmb {

// Position-independent operation lists.  A pointer field of a cached op may
// hold (tag << 56) | element offset with tag = base index + 1; the kernels
// resolve it against the base table passed at launch (tag 0: an ordinary
// pointer, or null).  Lists built once per H*H plan are then replayed for
// every product with the same plan, only the base table changing.
constexpr int kRelocDouble = 8, kRelocInt = 2;
struct RelocBases {
    double* d[kRelocDouble];
    int* i[kRelocInt];
};

#ifdef __CUDACC__
__device__ __forceinline__ double* reloc(double* p, const RelocBases& b) {
    const unsigned long long v = reinterpret_cast<unsigned long long>(p);
    const unsigned tag = (unsigned)(v >> 56);
    return tag == 0 ? p : b.d[tag - 1] + (long long)(v & ((1ULL << 56) - 1));
}
__device__ __forceinline__ const double* reloc(const double* p, const RelocBases& b) {
    return reloc(const_cast<double*>(p), b);
}
__device__ __forceinline__ int* reloc(int* p, const RelocBases& b) {
    const unsigned long long v = reinterpret_cast<unsigned long long>(p);
    const unsigned tag = (unsigned)(v >> 56);
    return tag == 0 ? p : b.i[tag - 1] + (long long)(v & ((1ULL << 56) - 1));
}
__device__ __forceinline__ const int* reloc(const int* p, const RelocBases& b) {
    return reloc(const_cast<int*>(p), b);
}
#endif

// Host side: turns pointers into tagged offsets against registered ranges.
class Relocator {
  public:
    void add(int index, const double* base, long long count) { d_.push_back({index, base, count}); }
    void add(int index, const int* base, long long count) { i_.push_back({index, base, count}); }
    // false when p lies in no registered range (then the list is not
    // cached).  A pointer one past the end of a range (an empty block's
    // factor) is tagged to that range when no range contains it.
    template <typename T>
    bool tag(T*& p) const {
        if (p == nullptr) return true;
        using U = typename std::remove_const<T>::type;
        const auto& rs = ranges(static_cast<U*>(nullptr));
        for (int pass = 0; pass < 2; ++pass)
            for (const auto& r : rs) {
                const U* b = static_cast<const U*>(r.base);
                if (b && p >= b && (pass == 0 ? p < b + r.count : p == b + r.count)) {
                    const unsigned long long v =
                        ((unsigned long long)(r.index + 1) << 56) | (unsigned long long)(p - b);
                    p = reinterpret_cast<T*>(v);
                    return true;
                }
            }
        return false;
    }
  private:
    struct Range { int index; const void* base; long long count; };
    std::vector<Range> d_, i_;
    const std::vector<Range>& ranges(double*) const { return d_; }
    const std::vector<Range>& ranges(int*) const { return i_; }
};

}  // namespace hmb
