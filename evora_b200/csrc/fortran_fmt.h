// fortran_fmt.h -- the output edit descriptors of Fortran formatted I/O that
// the reference's text files use (Ew.d, Fw.d, Iw, Lw, Aw), rendered the way
// gfortran renders them, so that screen lines, evolution files, snapshots
// and cuts compare byte for byte with the reference's.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace evora {
namespace fortran {

inline std::string pad_left(const std::string& s, int w) {
  if ((int)s.size() >= w) return s;
  return std::string((size_t)(w - (int)s.size()), ' ') + s;
}

inline std::string stars(int w) { return std::string((size_t)w, '*'); }

// Ew.d: [-]0.<d digits>E[+-]xx right-justified in w.  The d significant
// digits are the correctly rounded decimal of x (the C library's %e).  An
// exponent of three digits is written [+-]xxx without the letter E; when the
// field is one short the optional leading zero is dropped, and a field that
// is still too narrow is filled with asterisks.
inline std::string E(double x, int w, int d) {
  std::string s;
  if (std::isnan(x)) {
    s = "NaN";
  } else if (std::isinf(x)) {
    s = w >= 9 ? "Infinity" : "Inf";
    if (x < 0) s = "-" + s;
  } else {
    char buf[64];
    std::string digits;
    int e10 = 0;
    if (x == 0.0) {
      digits.assign((size_t)d, '0');
    } else {
      std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(x));   // "D.DDDe+XX"
      digits += buf[0];
      if (d > 1) digits.append(buf + 2, (size_t)(d - 1));
      e10 = std::atoi(std::strchr(buf, 'e') + 1) + 1;                 // 0.D... form
    }
    const char sign = e10 < 0 ? '-' : '+';
    const int ae = std::abs(e10);
    if (ae <= 99) std::snprintf(buf, sizeof buf, "E%c%02d", sign, ae);
    else if (ae <= 999) std::snprintf(buf, sizeof buf, "%c%03d", sign, ae);
    else return stars(w);
    s = std::string(std::signbit(x) ? "-" : "") + "0." + digits + buf;
    if ((int)s.size() > w) {
      const size_t z = s.find("0.");
      s.erase(z, 1);   // the leading zero is optional
    }
  }
  if ((int)s.size() > w) return stars(w);
  return pad_left(s, w);
}

// Fw.d
inline std::string F(double x, int w, int d) {
  char buf[512];
  if (std::isnan(x)) return pad_left("NaN", w);
  if (std::isinf(x)) return pad_left(x < 0 ? "-Inf" : "Inf", w);
  std::snprintf(buf, sizeof buf, "%.*f", d, x);
  std::string s = buf;
  if ((int)s.size() > w && (s.rfind("0.", 0) == 0 || s.rfind("-0.", 0) == 0)) s.erase(s.find("0."), 1);
  if ((int)s.size() > w) return stars(w);
  return pad_left(s, w);
}

// Iw
inline std::string I(long long v, int w) {
  std::string s = std::to_string(v);
  if ((int)s.size() > w) return stars(w);
  return pad_left(s, w);
}

// I0.m (at least m digits, zero-padded, no blanks), as in '(I0.3)'.
inline std::string I0(long long v, int m) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "%0*lld", m, v);
  return buf;
}

// Lw
inline std::string L(bool v, int w) { return pad_left(v ? "T" : "F", w); }

// Aw: a shorter string is right-justified, a longer one cut to its first w
// characters.
inline std::string A(const std::string& s, int w) {
  if ((int)s.size() >= w) return s.substr(0, (size_t)w);
  return pad_left(s, w);
}

}  // namespace fortran
}  // namespace evora
