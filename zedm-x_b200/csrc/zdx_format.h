// zdx_format.h -- the text of the output files, built with std::to_chars instead of std::ostream.
//
// The reference writes its particle VTK and state txt files through std::ofstream (src/main.cpp:1710-1870):
// a double in the default format is printf's "%.6g" of it, and under std::fixed with setprecision(9) it is
// "%.9f".  std::to_chars with chars_format::general / fixed and an explicit precision is specified to give
// the characters printf gives for the same conversion in the "C" locale, so the files are byte-identical;
// it runs without the stream's locale and sentry machinery, and each thread formats its own slice.
#pragma once

#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace zdx {

struct TextBuf {
    std::string s;
    void lit(const char* p) { s.append(p); }
    void ch(char c) { s.push_back(c); }
    // ostream << double, default flags: "%.6g"
    void g6(double v) {
        char b[48];
        auto r = std::to_chars(b, b + sizeof(b), v, std::chars_format::general, 6);
        s.append(b, r.ptr);
    }
    // ostream << float: promoted to double, then "%.6g"
    void f6(double v) { g6(static_cast<double>(static_cast<float>(v))); }
    // ostream << double under std::fixed and setprecision(9): "%.9f"
    void fixed9(double v) {
        char b[352];  // DBL_MAX has 309 integer digits
        auto r = std::to_chars(b, b + sizeof(b), v, std::chars_format::fixed, 9);
        s.append(b, r.ptr);
    }
    template <class I>
    void integer(I v) {
        char b[24];
        auto r = std::to_chars(b, b + sizeof(b), v);
        s.append(b, r.ptr);
    }
};

// Formats items [0, n) into consecutive slices on up to `threads` threads and writes the slices to `f` in
// order.  fn(begin, end, TextBuf&) appends the text of items [begin, end).  Returns false on a write error.
template <class Fn>
bool write_sliced(std::FILE* f, int64_t n, int threads, Fn&& fn) {
    if (n <= 0) return true;
    const int64_t min_items = 4096;
    int t = (int)std::min<int64_t>(threads, (n + min_items - 1) / min_items);
    if (t < 1) t = 1;
    std::unique_ptr<TextBuf[]> parts(new TextBuf[t]);
    auto run = [&](int k) {
        const int64_t b = n * k / t, e = n * (k + 1) / t;
        fn(b, e, parts[k]);
    };
    if (t == 1) {
        run(0);
    } else {
        std::vector<std::thread> pool;
        pool.reserve(t - 1);
        for (int k = 1; k < t; ++k) pool.emplace_back(run, k);
        run(0);
        for (auto& th : pool) th.join();
    }
    bool ok = true;
    for (int k = 0; k < t; ++k) {
        const std::string& p = parts[k].s;
        if (!p.empty()) ok = std::fwrite(p.data(), 1, p.size(), f) == p.size() && ok;
    }
    return ok;
}

}  // namespace zdx
