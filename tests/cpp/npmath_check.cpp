// Host build of zdx_npmath.cuh for tests/test_npmath_cpu.py.  Reads lines of 6 doubles as hex bit
// patterns (3-vectors a and b) and prints, as hex bit patterns, dot3(a, b), norm3(a), norm4 of
// (a0, a1, a2, b0), row_norm3(a) and cross3(a, b).
#include <cinttypes>
#include <cstdio>
#include <cstring>

#include "zdx_npmath.cuh"

static double from_bits(uint64_t u) {
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
static uint64_t to_bits(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
}

int main() {
    uint64_t u[6];
    while (std::scanf("%" SCNx64 " %" SCNx64 " %" SCNx64 " %" SCNx64 " %" SCNx64 " %" SCNx64, &u[0], &u[1], &u[2],
                      &u[3], &u[4], &u[5]) == 6) {
        double a[3] = {from_bits(u[0]), from_bits(u[1]), from_bits(u[2])};
        double b[3] = {from_bits(u[3]), from_bits(u[4]), from_bits(u[5])};
        double q[4] = {a[0], a[1], a[2], b[0]};
        double c[3];
        zdx::np::cross3(a, b, c);
        std::printf("%016" PRIx64 " %016" PRIx64 " %016" PRIx64 " %016" PRIx64 " %016" PRIx64 " %016" PRIx64
                    " %016" PRIx64 "\n",
                    to_bits(zdx::np::dot3(a, b)), to_bits(zdx::np::norm3(a)), to_bits(zdx::np::norm4(q)),
                    to_bits(zdx::np::row_norm3(a)), to_bits(c[0]), to_bits(c[1]), to_bits(c[2]));
    }
    return 0;
}
