/*
 * oracle_ad.h -- TEST INFRASTRUCTURE ONLY (CPU oracle, see oracle_common.h).
 *
 * A minimal tape-based reverse-mode differentiation type for the FP64 twin of the model-1
 * prognostic path (oracle/adjoint.cpp).  Every arithmetic operation on tape values appends one
 * node holding the indices of its (at most two) operands and the local partial derivatives; the
 * reverse sweep walks the tape backwards.  Values that depend on no input (grid constants) carry
 * index -1 and record nothing.  Comparisons act on values, so the branches of the solver differentiate
 * along the branch taken; max/min at a tie and |x| at zero take the mean of the one-sided
 * derivatives.
 *
 * This is an independent derivation of the gradient: it differentiates the oracle's own
 * operations, not the library's hand-written adjoint.
 */
#ifndef GRAL_ORACLE_AD_H
#define GRAL_ORACLE_AD_H

#include <cmath>
#include <cstdint>
#include <vector>

namespace oracle {

struct TapeNode {
    int32_t a, b;     /* operand node indices (-1: none) */
    double da, db;    /* d(result)/d(operand) */
};

/* The tape of the current recording (one per thread; the twin records single-threaded). */
struct Tape {
    std::vector<TapeNode> nodes;
    int32_t push(int32_t a, double da, int32_t b, double db) {
        nodes.push_back({a, b, da, db});
        return (int32_t)nodes.size() - 1;
    }
    /* a fresh input (leaf) node */
    int32_t leaf() { return push(-1, 0.0, -1, 0.0); }
    void clear() { nodes.clear(); }
    /* adjoints of every node from the seeds already placed in adj (same length as the tape) */
    void reverse(std::vector<double> &adj) const {
        for (size_t n = nodes.size(); n-- > 0;) {
            const double g = adj[n];
            if (g == 0.0) continue;
            const TapeNode &t = nodes[n];
            if (t.a >= 0) adj[(size_t)t.a] += g * t.da;
            if (t.b >= 0) adj[(size_t)t.b] += g * t.db;
        }
    }
};

extern thread_local Tape *g_tape;

struct AD {
    double v = 0.0;
    int32_t i = -1;
    AD() = default;
    AD(double x) : v(x), i(-1) {}   /* constants: no node */
    AD(float x) : v((double)x), i(-1) {}
    AD(int x) : v((double)x), i(-1) {}
    static AD make(double v, int32_t a, double da, int32_t b, double db) {
        AD r;
        r.v = v;
        if (a < 0 && b < 0) return r;
        r.i = g_tape->push(a, da, b, db);
        return r;
    }
    static AD input(double v) {
        AD r;
        r.v = v;
        r.i = g_tape->leaf();
        return r;
    }
};

inline AD operator+(const AD &x, const AD &y) { return AD::make(x.v + y.v, x.i, 1.0, y.i, 1.0); }
inline AD operator-(const AD &x, const AD &y) { return AD::make(x.v - y.v, x.i, 1.0, y.i, -1.0); }
inline AD operator*(const AD &x, const AD &y) { return AD::make(x.v * y.v, x.i, y.v, y.i, x.v); }
inline AD operator/(const AD &x, const AD &y) {
    const double q = x.v / y.v;
    return AD::make(q, x.i, 1.0 / y.v, y.i, -q / y.v);
}
inline AD operator-(const AD &x) { return AD::make(-x.v, x.i, -1.0, -1, 0.0); }
inline AD &operator+=(AD &x, const AD &y) { return x = x + y; }
inline AD &operator-=(AD &x, const AD &y) { return x = x - y; }
inline AD &operator*=(AD &x, const AD &y) { return x = x * y; }
inline bool operator<(const AD &x, const AD &y) { return x.v < y.v; }
inline bool operator>(const AD &x, const AD &y) { return x.v > y.v; }
inline bool operator<=(const AD &x, const AD &y) { return x.v <= y.v; }
inline bool operator>=(const AD &x, const AD &y) { return x.v >= y.v; }
inline bool operator==(const AD &x, const AD &y) { return x.v == y.v; }
inline bool operator!=(const AD &x, const AD &y) { return x.v != y.v; }

/* At a tie of max/min and at the kink of |x| the derivative is the mean of the two one-sided
 * ones, which is what a central difference across the kink measures (and the true derivative
 * where two kinks cancel, as |F| and max(F, 0) do in the power law at F = 0). */
inline AD vmax(const AD &a, const AD &b) {
    if (a.v == b.v) return AD::make(a.v, a.i, 0.5, b.i, 0.5);
    return (a > b) ? a : b;
}
inline AD vmin(const AD &a, const AD &b) {
    if (a.v == b.v) return AD::make(a.v, a.i, 0.5, b.i, 0.5);
    return (a < b) ? a : b;
}
inline AD osqrt(const AD &x) {
    const double r = std::sqrt(x.v);
    return AD::make(r, x.i, r > 0.0 ? 0.5 / r : 0.0, -1, 0.0);   /* subgradient 0 at the root */
}
inline AD ofabs(const AD &x) {
    return AD::make(std::fabs(x.v), x.i, x.v < 0.0 ? -1.0 : (x.v > 0.0 ? 1.0 : 0.0), -1, 0.0);
}
inline AD ofma(const AD &a, const AD &b, const AD &c) { return a * b + c; }

/* Forward-mode dual number (value, derivative along one direction): the tangent of the same
 * operations, an independent check of the tape's reverse sweep. */
struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x), d(0.0) {}
    Dual(float x) : v((double)x), d(0.0) {}
    Dual(int x) : v((double)x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(const Dual &x, const Dual &y) { return Dual(x.v + y.v, x.d + y.d); }
inline Dual operator-(const Dual &x, const Dual &y) { return Dual(x.v - y.v, x.d - y.d); }
inline Dual operator*(const Dual &x, const Dual &y) { return Dual(x.v * y.v, x.d * y.v + x.v * y.d); }
inline Dual operator/(const Dual &x, const Dual &y) {
    const double q = x.v / y.v;
    return Dual(q, (x.d - q * y.d) / y.v);
}
inline Dual operator-(const Dual &x) { return Dual(-x.v, -x.d); }
inline Dual &operator+=(Dual &x, const Dual &y) { return x = x + y; }
inline Dual &operator-=(Dual &x, const Dual &y) { return x = x - y; }
inline Dual &operator*=(Dual &x, const Dual &y) { return x = x * y; }
inline bool operator<(const Dual &x, const Dual &y) { return x.v < y.v; }
inline bool operator>(const Dual &x, const Dual &y) { return x.v > y.v; }
inline bool operator<=(const Dual &x, const Dual &y) { return x.v <= y.v; }
inline bool operator>=(const Dual &x, const Dual &y) { return x.v >= y.v; }
inline bool operator==(const Dual &x, const Dual &y) { return x.v == y.v; }
inline bool operator!=(const Dual &x, const Dual &y) { return x.v != y.v; }
inline Dual vmax(const Dual &a, const Dual &b) {
    if (a.v == b.v) return Dual(a.v, 0.5 * (a.d + b.d));
    return (a > b) ? a : b;
}
inline Dual vmin(const Dual &a, const Dual &b) {
    if (a.v == b.v) return Dual(a.v, 0.5 * (a.d + b.d));
    return (a < b) ? a : b;
}
inline Dual osqrt(const Dual &x) {
    const double r = std::sqrt(x.v);
    return Dual(r, r > 0.0 ? 0.5 * x.d / r : 0.0);
}
inline Dual ofabs(const Dual &x) { return Dual(std::fabs(x.v), x.v < 0.0 ? -x.d : (x.v > 0.0 ? x.d : 0.0)); }
inline Dual ofma(const Dual &a, const Dual &b, const Dual &c) { return a * b + c; }

}  // namespace oracle

#endif
