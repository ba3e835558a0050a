// Operation-counting scalar for the oracle (C++ build of shock_oracle.c):
// every +, -, *, /, sqrt, fabs and pow on a `real` adds one to the counter,
// comparisons add nothing.  Test infrastructure: produces the algorithmic
// FLOP count per cell-stage used as the roofline numerator.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>

struct FlopCounter {
    static uint64_t &n() { static uint64_t v = 0; return v; }
    static std::map<std::string, uint64_t> &phases() { static std::map<std::string, uint64_t> m; return m; }
    static uint64_t &mark() { static uint64_t v = 0; return v; }
};

struct CReal {
    double v;
    CReal() : v(0) {}
    CReal(double x) : v(x) {}
    explicit operator double() const { return v; }
    CReal &operator+=(const CReal &o) { FlopCounter::n()++; v += o.v; return *this; }
    CReal &operator-=(const CReal &o) { FlopCounter::n()++; v -= o.v; return *this; }
};
inline CReal operator+(CReal a, CReal b) { FlopCounter::n()++; return CReal(a.v + b.v); }
inline CReal operator-(CReal a, CReal b) { FlopCounter::n()++; return CReal(a.v - b.v); }
inline CReal operator*(CReal a, CReal b) { FlopCounter::n()++; return CReal(a.v * b.v); }
inline CReal operator/(CReal a, CReal b) { FlopCounter::n()++; return CReal(a.v / b.v); }
inline CReal operator-(CReal a) { return CReal(-a.v); }
inline bool operator<(CReal a, CReal b) { return a.v < b.v; }
inline bool operator>(CReal a, CReal b) { return a.v > b.v; }
inline CReal R_SQRT(CReal a) { FlopCounter::n()++; return CReal(std::sqrt(a.v)); }
inline CReal R_FABS(CReal a) { FlopCounter::n()++; return CReal(std::fabs(a.v)); }
inline CReal R_POW(CReal a, double e) { FlopCounter::n()++; return CReal(std::pow(a.v, e)); }
typedef CReal real;

inline void oracle_phase(const char *name)
{
    uint64_t now = FlopCounter::n();
    FlopCounter::phases()[name] += now - FlopCounter::mark();
    FlopCounter::mark() = now;
}
#define ORACLE_PHASE(name) oracle_phase(name)
