// Checks zdx_format.h against std::ostream: for each value, the "%.6g" of the value cast to float (what
// `out << static_cast<float>(v)` prints), "%.6g" of the double, "%.9f" under std::fixed, and integers.
// Then formats one block of lines on 1 and on 7 threads through write_sliced and compares the files.
// Prints "ok <count>" or the first mismatch; exit status 0 only when everything matched.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "zdx_format.h"

static int fail(const char* what, double v, const std::string& a, const std::string& b) {
    std::printf("mismatch %s value %.17g: stream '%s' to_chars '%s'\n", what, v, a.c_str(), b.c_str());
    return 1;
}

int main() {
    std::vector<double> vals = {0.0, -0.0, 1.0, -1.0, 0.5, 1e-5, 5e-5, 999999.5, 9.999995, 99999.95, 1234567.0,
                                0.1, 1.0 / 3.0, 2.0 / 3.0, 1e-310, -4.9e-324, 1e300, -1e300, DBL_MAX, -DBL_MAX,
                                DBL_MIN, FLT_MAX, FLT_MIN, 1e-45, 0.0000015, 0.00000149999, 2.5e-7, 123456.5,
                                0.0010000005, 1.0000005, 8.0000005e-8,
                                std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity()};
    std::mt19937_64 rng(12345);
    for (int i = 0; i < 300000; ++i) {
        uint64_t bits = rng();
        double v;
        std::memcpy(&v, &bits, 8);
        if (std::isnan(v)) continue;
        vals.push_back(v);
    }
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (int e = -40; e <= 40; ++e)
        for (int i = 0; i < 2000; ++i) vals.push_back(u(rng) * std::pow(10.0, e));
    for (int i = 0; i < 20000; ++i) {  // values on a 6- and 9-digit rounding boundary
        const double m = std::floor(u(rng) * 1e6) + 0.5;
        vals.push_back(m * std::pow(10.0, (int)(rng() % 20) - 10));
        vals.push_back((std::floor(u(rng) * 1e9) + 0.5) * 1e-9);
    }
    long n = 0;
    for (double v : vals) {
        std::ostringstream a1, a2, a3;
        a1 << static_cast<float>(v);
        a2 << v;
        a3.setf(std::ios::fixed);
        a3 << std::setprecision(9) << v;
        zdx::TextBuf b1, b2, b3;
        b1.f6(v);
        b2.g6(v);
        b3.fixed9(v);
        if (a1.str() != b1.s) return fail("float %.6g", v, a1.str(), b1.s);
        if (a2.str() != b2.s) return fail("%.6g", v, a2.str(), b2.s);
        if (a3.str() != b3.s) return fail("%.9f", v, a3.str(), b3.s);
        n += 3;
    }
    for (long long k : {0LL, 1LL, -1LL, 9LL, 10LL, 123456789LL, -987654321012LL, (long long)INT64_MAX, (long long)INT64_MIN}) {
        std::ostringstream a;
        a << k;
        zdx::TextBuf b;
        b.integer(k);
        if (a.str() != b.s) return fail("integer", (double)k, a.str(), b.s);
        n++;
    }
    // sliced writing: same bytes on 1 and on 7 threads
    const int64_t items = 50000;
    std::string files[2];
    for (int pass = 0; pass < 2; ++pass) {
        std::FILE* f = std::tmpfile();
        if (!f) return 2;
        bool ok = zdx::write_sliced(f, items, pass ? 7 : 1, [&](int64_t b, int64_t e, zdx::TextBuf& o) {
            for (int64_t i = b; i < e; ++i) {
                o.integer(i);
                o.ch(' ');
                o.f6(vals[(size_t)i] * 1e-3);
                o.ch('\n');
            }
        });
        if (!ok) return 3;
        std::fflush(f);
        long len = std::ftell(f);
        std::rewind(f);
        files[pass].resize(len);
        if (std::fread(&files[pass][0], 1, len, f) != (size_t)len) return 4;
        std::fclose(f);
    }
    if (files[0] != files[1] || files[0].empty()) {
        std::printf("sliced output differs between 1 and 7 threads\n");
        return 1;
    }
    std::printf("ok %ld\n", n);
    return 0;
}
