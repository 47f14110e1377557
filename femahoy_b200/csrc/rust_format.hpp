// Floating point text as Rust's formatter writes it, for the reference's error messages.
//
// The reference builds its messages with `format!`: "{residual:.2e}" (multigrid.rs:730-732)
// and "{:e}" (cholesky.rs:92-97). Rust's LowerExp writes the exponent as a plain integer with
// a minus sign only when negative (1.23e-5, 2.5e0, 1e10), not C's signed two-digit form
// (1.23e-05); "{:e}" without a precision writes the fewest digits that read back to the same
// double; NaN is "NaN" and the infinities "inf" and "-inf".
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace femgpu {

// C's "%.*e" text with its exponent rewritten in Rust's form.
inline std::string rust_exponent_text(const char* c) {
    std::string s(c);
    size_t e = s.find('e');
    if (e == std::string::npos) return s;
    std::string mant = s.substr(0, e);
    const char* p = s.c_str() + e + 1;
    bool neg = *p == '-';
    if (*p == '+' || *p == '-') ++p;
    while (*p == '0' && p[1] != '\0') ++p;
    return mant + "e" + (neg ? "-" : "") + p;
}

// Rust's "{:.Ne}" of v (N = digits after the point).
inline std::string rust_exp(double v, int digits) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", digits, v);
    return rust_exponent_text(buf);
}

// Rust's "{:e}" of v: the shortest digits that read back to v.
inline std::string rust_exp_shortest(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    for (int digits = 0; digits < 17; ++digits) {
        std::snprintf(buf, sizeof buf, "%.*e", digits, v);
        if (std::strtod(buf, nullptr) == v) return rust_exponent_text(buf);
    }
    std::snprintf(buf, sizeof buf, "%.16e", v);
    return rust_exponent_text(buf);
}

// Rust's "{}" (Display) of v: the shortest digits that read back to v, written out in full
// positional notation with no exponent (1e-7 is 0.0000001, 1e21 twenty-two digits, 2.0 is 2).
inline std::string rust_display(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    int digits = 0;
    for (; digits < 17; ++digits) {
        std::snprintf(buf, sizeof buf, "%.*e", digits, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    if (digits == 17) std::snprintf(buf, sizeof buf, "%.16e", v);
    // buf: [-]D[.DDD]e(+|-)XX
    std::string t(buf);
    const bool neg = t[0] == '-';
    if (neg) t.erase(0, 1);
    const size_t e = t.find('e');
    const int ex = std::atoi(t.c_str() + e + 1);
    std::string d;
    for (size_t k = 0; k < e; ++k)
        if (t[k] != '.') d += t[k];
    while (d.size() > 1 && d.back() == '0') d.pop_back();
    std::string out;
    if (ex >= 0) {
        if ((int)d.size() <= ex + 1) {
            out = d + std::string(ex + 1 - d.size(), '0');
        } else {
            out = d.substr(0, ex + 1) + "." + d.substr(ex + 1);
        }
    } else {
        out = "0." + std::string(-ex - 1, '0') + d;
    }
    return (neg ? "-" : "") + out;
}

}  // namespace femgpu
