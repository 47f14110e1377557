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

}  // namespace femgpu
