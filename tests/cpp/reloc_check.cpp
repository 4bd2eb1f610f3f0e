// Host-side check of the position-independent list encoding (reloc.h):
// pointers into registered ranges become tagged offsets that resolve back
// against a new base table; a pointer one past a range's end is tagged to
// that range only when no range contains it; pointers outside every range
// are refused.  Prints "ok" on success.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "reloc.h"

using namespace hmb;

static const double* resolve(const double* p, double* const* bases) {
    const unsigned long long v = reinterpret_cast<unsigned long long>(p);
    const unsigned tag = (unsigned)(v >> 56);
    return tag == 0 ? p : bases[tag - 1] + (long long)(v & ((1ULL << 56) - 1));
}

int main() {
    std::vector<double> a(100), b(50), a2(100), b2(50);
    std::vector<int> ri(10);
    Relocator rel;
    rel.add(0, a.data(), 100);
    rel.add(1, b.data(), 50);
    rel.add(0, ri.data(), 10);
    int fails = 0;
    // inside a range
    const double* p = a.data() + 37;
    if (!rel.tag(p)) ++fails;
    double* bases[2] = {a2.data(), b2.data()};
    if (resolve(p, bases) != a2.data() + 37) ++fails;
    // one past the end of b: tagged to b
    const double* q = b.data() + 50;
    if (!rel.tag(q) || resolve(q, bases) != b2.data() + 50) ++fails;
    // null stays null
    const double* z = nullptr;
    if (!rel.tag(z) || z != nullptr) ++fails;
    // outside every range: refused
    double other[4];
    const double* o = other + 1;
    if (rel.tag(o)) ++fails;
    // int ranges are separate
    int* ip = ri.data() + 3;
    if (!rel.tag(ip) || (reinterpret_cast<unsigned long long>(ip) >> 56) != 1 ||
        (reinterpret_cast<unsigned long long>(ip) & 0xff) != 3)
        ++fails;
    std::printf(fails ? "fail %d\n" : "ok\n", fails);
    return fails ? 1 : 0;
}
