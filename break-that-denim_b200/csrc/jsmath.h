// Host helpers that reproduce the reference's JavaScript number semantics where the scene compiler
// depends on them bit for bit: Math.hypot (V8's normalised Kahan sum), ToInt32 for the integer
// hashes, and Number.prototype.toString for the material JSON folded into sceneHash.
#pragma once

#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace btd {

// Math.hypot as V8 computes it: magnitudes normalised by the largest, squared and summed with Kahan
// compensation, then sqrt(sum) * max. It differs from libm hypot in the last ulp, which matters for
// the Worley distance comparisons and the float32 positions hashed by sceneHash.
inline double jsHypot(const double* v, int n) {
  double mx = 0;
  for (int i = 0; i < n; ++i) {
    double a = std::fabs(v[i]);
    if (std::isnan(v[i])) return NAN;
    if (a > mx) mx = a;
  }
  if (std::isinf(mx)) return INFINITY;
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (int i = 0; i < n; ++i) {
    double q = std::fabs(v[i]) / mx;
    double summand = q * q - comp;
    double pre = sum + summand;
    comp = (pre - sum) - summand;
    sum = pre;
  }
  return std::sqrt(sum) * mx;
}
inline double jsHypot2(double a, double b) {
  double v[2] = {a, b};
  return jsHypot(v, 2);
}
inline double jsHypot3(double a, double b, double c) {
  double v[3] = {a, b, c};
  return jsHypot(v, 3);
}

// ECMAScript ToInt32 of an integral double.
inline int32_t toInt32(double d) {
  if (!std::isfinite(d)) return 0;
  double m = std::fmod(std::trunc(d), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return static_cast<int32_t>(static_cast<uint32_t>(m));
}

// Number.prototype.toString(10) of a finite double: shortest round-trip digits laid out by the
// ECMAScript Number::toString rules (fixed notation for exponents 1e-6 <= |x| < 1e21).
inline std::string jsNumber(double v) {
  if (v == 0) return "0";
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
  std::string out;
  if (v < 0) {
    out = "-";
    v = -v;
  }
  char buf[64];
  auto res = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string sci(buf, res.ptr);
  size_t epos = sci.find('e');
  std::string mant = sci.substr(0, epos);
  int e10 = std::atoi(sci.c_str() + epos + 1);
  std::string digits;
  for (char c : mant)
    if (c != '.') digits += c;
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  int k = static_cast<int>(digits.size());
  int n = e10 + 1;
  if (k <= n && n <= 21) {
    out += digits + std::string(n - k, '0');
  } else if (0 < n && n <= 21) {
    out += digits.substr(0, n) + "." + digits.substr(n);
  } else if (-6 < n && n <= 0) {
    out += "0." + std::string(-n, '0') + digits;
  } else {
    int e = n - 1;
    std::string es = (e >= 0 ? "+" : "-") + std::to_string(e >= 0 ? e : -e);
    if (k == 1)
      out += digits + "e" + es;
    else
      out += digits.substr(0, 1) + "." + digits.substr(1) + "e" + es;
  }
  return out;
}

}  // namespace btd
