/*
 * orc_counted.h -- op-counting scalar for the oracle (TEST INFRASTRUCTURE).
 *
 * A standard-layout wrapper around one double: arrays of Counted have the
 * memory layout of arrays of double, so the counting build of the oracle
 * reads the same caller-owned buffers as the plain FP64 build. Every
 * arithmetic operator bumps a per-kind counter; the value arithmetic is
 * ordinary double arithmetic, so a counted run also reproduces the FP64 run.
 */
#ifndef ORC_COUNTED_H
#define ORC_COUNTED_H

#include <cmath>
#include <cstdint>

namespace orc {

extern thread_local uint64_t g_ops[6]; /* add/sub, mul, div, sqrt, compare, other */

struct Counted {
    double v;
    Counted() : v(0) {}
    Counted(double d) : v(d) {}          /* implicit from literals and ints */
    explicit operator double() const { return v; }
    explicit operator float() const { return float(v); }
    explicit operator int() const { return int(v); }
};

inline Counted operator+(Counted a, Counted b) { ++g_ops[0]; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_ops[0]; return Counted(a.v - b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted operator*(Counted a, Counted b) { ++g_ops[1]; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_ops[2]; return Counted(a.v / b.v); }
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted& operator-=(Counted& a, Counted b) { a = a - b; return a; }
inline Counted& operator*=(Counted& a, Counted b) { a = a * b; return a; }
inline bool operator<(Counted a, Counted b) { ++g_ops[4]; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++g_ops[4]; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++g_ops[4]; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { ++g_ops[4]; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { ++g_ops[4]; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { ++g_ops[4]; return a.v != b.v; }
inline Counted sqrt(Counted a) { ++g_ops[3]; return Counted(std::sqrt(a.v)); }
inline Counted floor(Counted a) { ++g_ops[5]; return Counted(std::floor(a.v)); }
inline Counted exp(Counted a) { ++g_ops[5]; return Counted(std::exp(a.v)); }
inline Counted cos(Counted a) { ++g_ops[5]; return Counted(std::cos(a.v)); }
inline Counted sin(Counted a) { ++g_ops[5]; return Counted(std::sin(a.v)); }

}  // namespace orc

#endif
