// Oracle test infrastructure (CPU only): an FP64 scalar that counts the
// floating-point operations it performs.  Compiling fluxo_oracle.cpp with
// -DFLUXO_COUNT makes every `real` in the right-hand-side path a Counted, so
// one oracle RHS evaluation yields the exact algorithmic operation count F_alg
// used as the numerator of the FP64 roofline.
//
// Counting rules (fixed for the whole project):
//   + - * /                         1 each
//   sqrt log exp pow abs min max    1 each
//   a*b+c written in source         2 (one * and one +)
//   comparisons, unary minus, index arithmetic, copies   0
#pragma once
#include <cmath>
#include <cstdint>

extern "C" uint64_t g_oracle_flops;

struct Counted {
  double v;
  Counted() : v(0.0) {}
  Counted(double x) : v(x) {}  // NOLINT: implicit on purpose (literals)
  explicit operator double() const { return v; }
};

inline Counted cnt(double x) { ++g_oracle_flops; return Counted(x); }

inline Counted operator+(Counted a, Counted b) { return cnt(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { return cnt(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { return cnt(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { return cnt(a.v / b.v); }
inline Counted operator+(Counted a, double b) { return cnt(a.v + b); }
inline Counted operator-(Counted a, double b) { return cnt(a.v - b); }
inline Counted operator*(Counted a, double b) { return cnt(a.v * b); }
inline Counted operator/(Counted a, double b) { return cnt(a.v / b); }
inline Counted operator+(double a, Counted b) { return cnt(a + b.v); }
inline Counted operator-(double a, Counted b) { return cnt(a - b.v); }
inline Counted operator*(double a, Counted b) { return cnt(a * b.v); }
inline Counted operator/(double a, Counted b) { return cnt(a / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted& operator-=(Counted& a, Counted b) { a = a - b; return a; }
inline Counted& operator*=(Counted& a, Counted b) { a = a * b; return a; }
inline Counted& operator/=(Counted& a, Counted b) { a = a / b; return a; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator<(Counted a, double b) { return a.v < b; }
inline bool operator>(Counted a, double b) { return a.v > b; }
inline bool operator<=(Counted a, double b) { return a.v <= b; }
inline bool operator>=(Counted a, double b) { return a.v >= b; }
inline Counted sqrt(Counted a) { return cnt(std::sqrt(a.v)); }
inline Counted log(Counted a) { return cnt(std::log(a.v)); }
inline Counted exp(Counted a) { return cnt(std::exp(a.v)); }
inline Counted pow(Counted a, double b) { return cnt(std::pow(a.v, b)); }
inline Counted fabs(Counted a) { return cnt(std::fabs(a.v)); }
inline Counted fmax(Counted a, Counted b) { return cnt(a.v > b.v ? a.v : b.v); }
inline Counted fmin(Counted a, Counted b) { return cnt(a.v < b.v ? a.v : b.v); }
inline bool isnan(Counted a) { return std::isnan(a.v); }
inline double val(Counted a) { return a.v; }
