// rs_opcount.hpp -- TEST / MEASUREMENT INFRASTRUCTURE ONLY: an op-counting scalar for the
// oracle. rso::Sim<OpCount> runs the restated substep in double precision while counting
// every floating-point operation, which gives the algorithmic FLOP figure of a workload
// (add/sub/mul/div = 1 each, sqrt and transcendental calls counted separately; comparisons,
// min/max and clamps are not FLOPs and are counted apart).
#pragma once

#include <cmath>
#include <limits>

namespace rso {

struct OpTally {
    long long add = 0, mul = 0, div = 0, sqrt = 0, trans = 0, cmp = 0;
    void reset() { *this = OpTally(); }
};
inline OpTally& op_tally() {
    static thread_local OpTally t;
    return t;
}

struct OpCount {
    double v;
    OpCount() : v(0) {}
    OpCount(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
    OpCount operator-() const { return OpCount(-v); }
    OpCount& operator+=(const OpCount& o) { op_tally().add++; v += o.v; return *this; }
    OpCount& operator-=(const OpCount& o) { op_tally().add++; v -= o.v; return *this; }
    OpCount& operator*=(const OpCount& o) { op_tally().mul++; v *= o.v; return *this; }
    OpCount& operator/=(const OpCount& o) { op_tally().div++; v /= o.v; return *this; }
};
inline OpCount operator+(OpCount a, OpCount b) { op_tally().add++; return OpCount(a.v + b.v); }
inline OpCount operator-(OpCount a, OpCount b) { op_tally().add++; return OpCount(a.v - b.v); }
inline OpCount operator*(OpCount a, OpCount b) { op_tally().mul++; return OpCount(a.v * b.v); }
inline OpCount operator/(OpCount a, OpCount b) { op_tally().div++; return OpCount(a.v / b.v); }
inline bool operator<(OpCount a, OpCount b) { op_tally().cmp++; return a.v < b.v; }
inline bool operator>(OpCount a, OpCount b) { op_tally().cmp++; return a.v > b.v; }
inline bool operator<=(OpCount a, OpCount b) { op_tally().cmp++; return a.v <= b.v; }
inline bool operator>=(OpCount a, OpCount b) { op_tally().cmp++; return a.v >= b.v; }
inline bool operator==(OpCount a, OpCount b) { op_tally().cmp++; return a.v == b.v; }
inline bool operator!=(OpCount a, OpCount b) { op_tally().cmp++; return a.v != b.v; }
inline OpCount sqrt(OpCount a) { op_tally().sqrt++; return OpCount(std::sqrt(a.v)); }
inline OpCount log(OpCount a) { op_tally().trans++; return OpCount(std::log(a.v)); }
inline OpCount sin(OpCount a) { op_tally().trans++; return OpCount(std::sin(a.v)); }
inline OpCount cos(OpCount a) { op_tally().trans++; return OpCount(std::cos(a.v)); }
inline OpCount acos(OpCount a) { op_tally().trans++; return OpCount(std::acos(a.v)); }
inline OpCount atan2(OpCount a, OpCount b) { op_tally().trans++; return OpCount(std::atan2(a.v, b.v)); }
inline bool isfinite(OpCount a) { return std::isfinite(a.v); }

}  // namespace rso

namespace std {
template <>
class numeric_limits<rso::OpCount> {
public:
    static constexpr bool is_specialized = true;
    static rso::OpCount infinity() { return rso::OpCount(std::numeric_limits<double>::infinity()); }
    static rso::OpCount max() { return rso::OpCount(std::numeric_limits<float>::max()); }
};
}  // namespace std
