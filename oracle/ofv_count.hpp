// ofv_count.hpp -- counting scalar used to fix the algorithmic flop figure of the oracle.
//
// TEST INFRASTRUCTURE ONLY.  When wenofv_oracle.c is compiled as C++ with -DOFV_COUNTING,
// every arithmetic scalar of the restated path is an ofv_cnt: each +, -, *, /, sqrt, fabs
// and comparison increments a global counter.  Division and sqrt count as one flop each
// (the convention of the roofline table), and so do exp, log and tanh (PRIMITIVE3's THINC
// profile); comparisons and fabs are counted separately and are not flops.
#ifndef OFV_COUNT_HPP
#define OFV_COUNT_HPP
#include <cmath>

struct ofv_counters {
    unsigned long long add, mul, div, sqrt, cmp, abs, tr;
};
extern ofv_counters g_ofv_cnt;

struct ofv_cnt {
    double v;
    ofv_cnt() : v(0.0) {}
    ofv_cnt(double x) : v(x) {}
    operator double() const { return v; }
    ofv_cnt &operator+=(ofv_cnt o) { g_ofv_cnt.add++; v += o.v; return *this; }
    ofv_cnt &operator-=(ofv_cnt o) { g_ofv_cnt.add++; v -= o.v; return *this; }
    ofv_cnt &operator*=(ofv_cnt o) { g_ofv_cnt.mul++; v *= o.v; return *this; }
    ofv_cnt &operator/=(ofv_cnt o) { g_ofv_cnt.div++; v /= o.v; return *this; }
    ofv_cnt operator-() const { return ofv_cnt(-v); }
};

#define OFV_BIN(op, field)                                                                 \
    inline ofv_cnt operator op(ofv_cnt a, ofv_cnt b) { g_ofv_cnt.field++; return ofv_cnt(a.v op b.v); } \
    inline ofv_cnt operator op(double a, ofv_cnt b) { g_ofv_cnt.field++; return ofv_cnt(a op b.v); }    \
    inline ofv_cnt operator op(ofv_cnt a, double b) { g_ofv_cnt.field++; return ofv_cnt(a.v op b); }    \
    inline ofv_cnt operator op(int a, ofv_cnt b) { g_ofv_cnt.field++; return ofv_cnt((double)a op b.v); } \
    inline ofv_cnt operator op(ofv_cnt a, int b) { g_ofv_cnt.field++; return ofv_cnt(a.v op (double)b); }
OFV_BIN(+, add)
OFV_BIN(-, add)
OFV_BIN(*, mul)
OFV_BIN(/, div)
#undef OFV_BIN

#define OFV_CMP(op)                                                                          \
    inline bool operator op(ofv_cnt a, ofv_cnt b) { g_ofv_cnt.cmp++; return a.v op b.v; }   \
    inline bool operator op(double a, ofv_cnt b) { g_ofv_cnt.cmp++; return a op b.v; }      \
    inline bool operator op(ofv_cnt a, double b) { g_ofv_cnt.cmp++; return a.v op b; }      \
    inline bool operator op(int a, ofv_cnt b) { g_ofv_cnt.cmp++; return (double)a op b.v; } \
    inline bool operator op(ofv_cnt a, int b) { g_ofv_cnt.cmp++; return a.v op (double)b; }
OFV_CMP(<)
OFV_CMP(>)
OFV_CMP(<=)
OFV_CMP(>=)
#undef OFV_CMP

inline ofv_cnt sqrt(ofv_cnt a) { g_ofv_cnt.sqrt++; return ofv_cnt(std::sqrt(a.v)); }
inline ofv_cnt fabs(ofv_cnt a) { g_ofv_cnt.abs++; return ofv_cnt(std::fabs(a.v)); }
// pow(x, n): with a small integer n (the WENO kernels) n - 1 multiplications, otherwise (the
// stiffened-gas isentropes) one transcendental
inline ofv_cnt pow(ofv_cnt a, double n)
{
    if (n >= 1 && n <= 8 && n == (double)(int)n) g_ofv_cnt.mul += (unsigned long long)(n - 1);
    else g_ofv_cnt.tr++;
    return ofv_cnt(std::pow(a.v, n));
}
inline ofv_cnt pow(ofv_cnt a, ofv_cnt n) { return pow(a, n.v); }
inline bool ofv_isnan(ofv_cnt a) { return std::isnan(a.v); }
inline ofv_cnt exp(ofv_cnt a) { g_ofv_cnt.tr++; return ofv_cnt(std::exp(a.v)); }
inline ofv_cnt log(ofv_cnt a) { g_ofv_cnt.tr++; return ofv_cnt(std::log(a.v)); }
inline ofv_cnt tanh(ofv_cnt a) { g_ofv_cnt.tr++; return ofv_cnt(std::tanh(a.v)); }

#endif
