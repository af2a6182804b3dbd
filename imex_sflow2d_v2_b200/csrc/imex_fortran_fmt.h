// Fortran edit descriptors used by the reference's output files
// (src/inpout_2d.f90: '(2e20.12,100(e20.12))' for .q_2d, '100ES15.7E2' for
// .p_2d, '(2000ES12.3E3)', '(A,I5)', '(A,F15.3)' for the ESRI grids), as
// gfortran writes them: the decimal digits are the correctly rounded ones
// (std::to_chars for %e-style digits, %f for Fw.d), Ew.d writes 0.d1...dd with a two-
// digit exponent after 'E' (three digits and no 'E' from 100 to 999),
// ESw.dEe writes d1.d2...E with exactly e exponent digits, a value whose
// exponent does not fit and any field too narrow become w asterisks, a
// negative value (negative zero included) gets '-', NaN and infinities are
// written as NaN / Infinity right-justified.  Host code only.
#pragma once

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace imex {
namespace ffmt {

inline void stars(std::string& out, int w) { out.append((size_t)w, '*'); }

inline void right(std::string& out, const char* s, int w) {
  const int n = (int)std::strlen(s);
  if (n > w) {
    stars(out, w);
    return;
  }
  out.append((size_t)(w - n), ' ');
  out.append(s, (size_t)n);
}

inline bool special(std::string& out, double v, int w) {
  if (std::isnan(v)) {
    right(out, "NaN", w);
    return true;
  }
  if (std::isinf(v)) {
    const char* s = v < 0 ? (w >= 9 ? "-Infinity" : "-Inf") : (w >= 8 ? "Infinity" : "Inf");
    right(out, s, w);
    return true;
  }
  return false;
}

// Decimal digits and exponent of |v| with `sig` significant digits,
// correctly rounded: |v| = 0.D1D2..Dsig x 10^E10 (E10 for the 0.d form).
inline void digits(double a, int sig, char* dig, int& e10) {
  char buf[64];
  const auto r = std::to_chars(buf, buf + sizeof buf - 1, a, std::chars_format::scientific,
                               sig - 1);   // d.ddde+XX, correctly rounded
  *r.ptr = 0;
  int k = 0;
  const char* p = buf;
  for (; *p && *p != 'e'; ++p)
    if (*p >= '0' && *p <= '9') dig[k++] = *p;
  dig[k] = 0;
  e10 = std::atoi(p + 1);
}

// Ew.d
inline void E(std::string& out, double v, int w, int d) {
  if (special(out, v, w)) return;
  char dig[64], s[96];
  int x;
  const double a = std::fabs(v);
  int ex;
  if (a == 0.0) {
    std::memset(dig, '0', (size_t)d);
    dig[d] = 0;
    ex = 0;
  } else {
    digits(a, d, dig, x);
    ex = x + 1;
  }
  char es[16];
  const int ae = std::abs(ex);
  if (ae <= 99) std::snprintf(es, sizeof es, "E%c%02d", ex < 0 ? '-' : '+', ae);
  else if (ae <= 999) std::snprintf(es, sizeof es, "%c%03d", ex < 0 ? '-' : '+', ae);
  else {
    stars(out, w);
    return;
  }
  std::snprintf(s, sizeof s, "%s0.%s%s", std::signbit(v) ? "-" : "", dig, es);
  right(out, s, w);
}

// ESw.dEe
inline void ES(std::string& out, double v, int w, int d, int e) {
  if (special(out, v, w)) return;
  char dig[64], s[96];
  int x = 0;
  const double a = std::fabs(v);
  if (a == 0.0) {
    std::memset(dig, '0', (size_t)d + 1);
    dig[d + 1] = 0;
  } else {
    digits(a, d + 1, dig, x);
  }
  const int ae = std::abs(x);
  int lim = 1;
  for (int i = 0; i < e; ++i) lim *= 10;
  if (ae >= lim) {
    stars(out, w);
    return;
  }
  std::snprintf(s, sizeof s, "%s%c.%sE%c%0*d", std::signbit(v) ? "-" : "", dig[0], dig + 1,
                x < 0 ? '-' : '+', e, ae);
  right(out, s, w);
}

// Iw
inline void I(std::string& out, long long v, int w) {
  char s[32];
  std::snprintf(s, sizeof s, "%lld", v);
  right(out, s, w);
}

// Fw.d
inline void F(std::string& out, double v, int w, int d) {
  if (special(out, v, w)) return;
  char s[64];
  std::snprintf(s, sizeof s, "%.*f", d, v);
  right(out, s, w);
}

// lettera(k): four characters CHAR(48+digit) of k (src/inpout_2d.f90:6642-6661)
inline std::string lettera(int k) {
  const int ithou = k / 1000;
  const int ihund = (k - ithou * 1000) / 100;
  const int iten = (k - ithou * 1000 - ihund * 100) / 10;
  const int ione = k - ithou * 1000 - ihund * 100 - iten * 10;
  std::string s(4, ' ');
  s[0] = (char)(ithou + 48);
  s[1] = (char)(ihund + 48);
  s[2] = (char)(iten + 48);
  s[3] = (char)(ione + 48);
  return s;
}

}  // namespace ffmt
}  // namespace imex
