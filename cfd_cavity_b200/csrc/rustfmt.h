// rustfmt.h -- the float formats of Rust's core::fmt that the reference
// driver's text outputs use (progress lines, CSV, VTK, JSON), so that a run
// of this driver writes the same bytes for the same values:
//   fixed(x, p)    {:.p}   round-to-nearest-even on the exact binary value
//   exp(x, p)      {:.pe}  d.ddd + 'e' + exponent without '+' or padding
//   exp_short(x)   {:e}    shortest round-trip digits, scientific
//   display(x)     {}      shortest round-trip digits, positional, no ".0"
// NaN prints "NaN", infinities "inf" / "-inf", negative zero keeps its sign.
#pragma once

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

namespace rf {

inline bool special(double x, std::string& out) {
    if (std::isnan(x)) {
        out = "NaN";
        return true;
    }
    if (std::isinf(x)) {
        out = x < 0 ? "-inf" : "inf";
        return true;
    }
    return false;
}

// "1.50e-05" / "1.5e+08" -> "1.50e-5" / "1.5e8"
inline std::string rust_exponent(const char* s) {
    const char* e = std::strchr(s, 'e');
    if (!e) return s;
    std::string out(s, e - s);
    out += 'e';
    const char* p = e + 1;
    bool neg = false;
    if (*p == '+' || *p == '-') {
        neg = *p == '-';
        ++p;
    }
    while (*p == '0' && p[1] != '\0') ++p;
    if (neg) out += '-';
    out += p;
    return out;
}

inline std::string fixed(double x, int prec) {
    std::string s;
    if (special(x, s)) return s;
    char buf[400];
    std::snprintf(buf, sizeof(buf), "%.*f", prec, x);
    return buf;
}

inline std::string exp(double x, int prec) {
    std::string s;
    if (special(x, s)) return s;
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*e", prec, x);
    return rust_exponent(buf);
}

// Shortest round-trip digits and decimal exponent: x = d[0].d[1..] x 10^e.
inline void shortest(double x, bool& neg, std::string& digits, int& e10) {
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::scientific);
    *r.ptr = '\0';
    const char* p = buf;
    neg = *p == '-';
    if (neg) ++p;
    digits.clear();
    for (; *p && *p != 'e'; ++p)
        if (*p != '.') digits += *p;
    e10 = *p == 'e' ? std::atoi(p + 1) : 0;
}

inline std::string exp_short(double x) {
    std::string s;
    if (special(x, s)) return s;
    bool neg;
    std::string d;
    int e;
    shortest(x, neg, d, e);
    s = neg ? "-" : "";
    s += d[0];
    if (d.size() > 1) s += "." + d.substr(1);
    s += "e" + std::to_string(e);
    return s;
}

inline std::string display(double x) {
    std::string s;
    if (special(x, s)) return s;
    bool neg;
    std::string d;
    int e;
    shortest(x, neg, d, e);
    s = neg ? "-" : "";
    if (d == "0") return s + "0";
    if (e >= 0) {
        const size_t ip = size_t(e) + 1;
        if (d.size() <= ip) return s + d + std::string(ip - d.size(), '0');
        return s + d.substr(0, ip) + "." + d.substr(ip);
    }
    return s + "0." + std::string(size_t(-e - 1), '0') + d;
}

// {:>w}
inline std::string right(const std::string& v, size_t w) {
    return v.size() >= w ? v : std::string(w - v.size(), ' ') + v;
}

}  // namespace rf
