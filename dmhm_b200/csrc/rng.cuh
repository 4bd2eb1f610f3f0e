// The reference's 64-bit LCG and Box-Muller Gaussians, evaluated on the device
// by skip-ahead so every element of a random fill is computed independently.
//
// Generator: X_{k+1} = a X_k + c mod 2^64 with Knuth's a, c
// (src/core/random.cpp:13-25, emulated there in 16-bit limbs); a draw returns
// the state before advancing (SerialLcg, random.cpp:103-109).  Uniform on
// (0,1]: (upper 32 bits + 1) / 2^32 (include/dmhm/core/random.hpp:250-258).
// Box-Muller pair from (U, V): sqrt(-2 ln U) * (cos 2piV, sin 2piV)
// (random.hpp:280-292).  Skip-ahead composes the affine maps
// x -> a^(2^j) x + c_j, the same idea as IntegerPowerWith64BitMod
// (random.cpp:32-65).
#pragma once
#include <cstdint>

namespace hmb {

constexpr uint64_t kLcgMult = 6364136223846793005ULL;
constexpr uint64_t kLcgAdd = 1442695040888963407ULL;
constexpr uint64_t kLcgSeed = (21ULL << 32) | 17ULL;   // global.cpp:88-93

// Host: advance `state` by n draws.
inline uint64_t lcg_skip_host(uint64_t state, uint64_t n) {
    uint64_t a = kLcgMult, c = kLcgAdd, am = 1, cm = 0;
    while (n) {
        if (n & 1) { am = a * am; cm = a * cm + c; }
        c = a * c + c;
        a = a * a;
        n >>= 1;
    }
    return am * state + cm;
}

__device__ __forceinline__ uint64_t lcg_skip(uint64_t state, uint64_t n) {
    uint64_t a = kLcgMult, c = kLcgAdd;
    while (n) {
        if (n & 1) state = a * state + c;
        c = a * c + c;
        a = a * a;
        n >>= 1;
    }
    return state;
}

__device__ __forceinline__ double lcg_uniform(uint64_t state) {
    return ((double)(uint32_t)(state >> 32) + 1.0) / 4294967296.0;
}

// Gaussian pair from the two draws starting at `state`.
__device__ __forceinline__ void box_muller(uint64_t state, double& x, double& y) {
    const double u = lcg_uniform(state);
    const uint64_t s2 = kLcgMult * state + kLcgAdd;
    const double v = lcg_uniform(s2);
    const double a = sqrt(-2.0 * log(u));
    const double t = 2.0 * 3.14159265358979323846 * v;
    x = a * cos(t);
    y = a * sin(t);
}

// Element (i, j) of an m x n real Gaussian fill (SerialGaussianRandomVectors /
// ParallelGaussianRandomVectors on Dense<Real>, random.hpp:418-474) whose
// first draw is at `base`.  Each column draws 2*ceil(m/2) uniforms; the
// column's final pair (or single, for odd m) lands at rows n-2, n-1 (the
// WIDTH, a reference quirk), so rows m-2, m-1 keep zero.  Requires n <= m.
__device__ __forceinline__ double gaussian_fill_entry(uint64_t base, int m, int n,
                                                      int i, int j) {
    const int pairs = (m + 1) / 2;
    const uint64_t col = base;  // state at the column's first draw computed below
    int pair = -1, which = 0;
    if ((m & 1) && i == n - 1) { pair = pairs - 1; which = 0; }
    else if (!(m & 1) && i == n - 2) { pair = pairs - 1; which = 0; }
    else if (!(m & 1) && i == n - 1) { pair = pairs - 1; which = 1; }
    else if (i < 2 * (pairs - 1)) { pair = i / 2; which = i & 1; }
    if (pair < 0) return 0.0;
    const uint64_t st = lcg_skip(col, (uint64_t)j * 2 * pairs + 2 * (uint64_t)pair);
    double x, y;
    box_muller(st, x, y);
    return which ? y : x;
}

}  // namespace hmb
