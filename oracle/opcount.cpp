/*
 * opcount.cpp -- TEST INFRASTRUCTURE ONLY: an operation-counting build of
 * the CPU oracle (wq3d_oracle.cpp).
 *
 * The oracle is compiled a second time with every "double" replaced by
 * Counted, a one-double wrapper whose arithmetic and math functions bump
 * global counters.  Counted has the layout of a double, so the oracle's C
 * entry points keep their binary interface and the same ctypes binding
 * drives this library.  Two extra entry points read and clear the
 * counters:
 *   oracle_opcount_read(uint64_t out[4][6])   per phase of the step (0 the
 *                                             ray step, 1 target distances,
 *                                             2 CPA search, 3 eigenray
 *                                             construction): adds,
 *                                             multiplies, divides, square
 *                                             roots, other math calls (sin,
 *                                             cos, exp, log, atan2, pow ...),
 *                                             compares
 *   oracle_opcount_reset()
 * The oracle marks its phases with ORACLE_PHASE, which expands to nothing
 * in its own build (tests/test_oracle_opcount.py reads the counts).
 *
 * The math overloads below sit in namespace std because the oracle calls
 * them qualified (std::sqrt, std::sin ...); they exist only in this
 * counting build.  The Rayleigh loss's complex arithmetic stays in plain
 * double (oracle_plain_double) and is not counted.
 */
#include "../include/wq3d.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace wq3d_opcount {

enum { OPC_ADD, OPC_MUL, OPC_DIV, OPC_SQRT, OPC_MATH, OPC_CMP, OPC_N };
enum { OPC_PHASES = 4 };
uint64_t g_counts[OPC_PHASES][OPC_N];
uint64_t* g_count = g_counts[0];

/* a scope whose operations count toward phase p */
struct Phase {
    uint64_t* saved;
    explicit Phase(int p) : saved(g_count) { g_count = g_counts[p]; }
    ~Phase() { g_count = saved; }
};

struct Counted {
    double v;
    Counted() = default;
    constexpr Counted(double x) : v(x) {}
    operator double() const { return v; }
    Counted& operator+=(Counted o) { ++g_count[OPC_ADD]; v += o.v; return *this; }
    Counted& operator-=(Counted o) { ++g_count[OPC_ADD]; v -= o.v; return *this; }
    Counted& operator*=(Counted o) { ++g_count[OPC_MUL]; v *= o.v; return *this; }
    Counted& operator/=(Counted o) { ++g_count[OPC_DIV]; v /= o.v; return *this; }
    Counted& operator++() { ++g_count[OPC_ADD]; v += 1.0; return *this; }
    Counted operator-() const { return Counted(-v); }
    Counted operator+() const { return *this; }
};
static_assert(sizeof(Counted) == sizeof(double) && std::is_trivially_copyable<Counted>::value,
              "Counted must have the layout of a double");

template <class T>
using if_num = typename std::enable_if<std::is_arithmetic<T>::value, int>::type;

#define OPC_BINARY(OP, KIND)                                                                  \
    inline Counted operator OP(Counted a, Counted b) { ++g_count[KIND]; return Counted(a.v OP b.v); } \
    template <class T, if_num<T> = 0>                                                         \
    inline Counted operator OP(Counted a, T b) { ++g_count[KIND]; return Counted(a.v OP (double)b); } \
    template <class T, if_num<T> = 0>                                                         \
    inline Counted operator OP(T a, Counted b) { ++g_count[KIND]; return Counted((double)a OP b.v); }
OPC_BINARY(+, OPC_ADD)
OPC_BINARY(-, OPC_ADD)
OPC_BINARY(*, OPC_MUL)
OPC_BINARY(/, OPC_DIV)
#undef OPC_BINARY

#define OPC_COMPARE(OP)                                                                       \
    inline bool operator OP(Counted a, Counted b) { ++g_count[OPC_CMP]; return a.v OP b.v; }   \
    template <class T, if_num<T> = 0>                                                         \
    inline bool operator OP(Counted a, T b) { ++g_count[OPC_CMP]; return a.v OP (double)b; }  \
    template <class T, if_num<T> = 0>                                                         \
    inline bool operator OP(T a, Counted b) { ++g_count[OPC_CMP]; return (double)a OP b.v; }
OPC_COMPARE(<)
OPC_COMPARE(>)
OPC_COMPARE(<=)
OPC_COMPARE(>=)
OPC_COMPARE(==)
OPC_COMPARE(!=)
#undef OPC_COMPARE

/* the Rayleigh loss mixes the scalar type into plain complex arithmetic */
typedef std::complex<double> cplx;
inline cplx operator*(Counted a, const cplx& b) { return a.v * b; }
inline cplx operator*(const cplx& a, Counted b) { return a * b.v; }
inline cplx operator/(Counted a, const cplx& b) { return a.v / b; }
inline cplx operator/(const cplx& a, Counted b) { return a / b.v; }
inline cplx operator+(Counted a, const cplx& b) { return a.v + b; }
inline cplx operator+(const cplx& a, Counted b) { return a + b.v; }
inline cplx operator-(Counted a, const cplx& b) { return a.v - b; }
inline cplx operator-(const cplx& a, Counted b) { return a - b.v; }

}  // namespace wq3d_opcount

namespace std {
using wq3d_opcount::Counted;
using wq3d_opcount::g_count;
#define OPC_UNARY(NAME, KIND)                                                               \
    inline Counted NAME(Counted a) { ++g_count[wq3d_opcount::KIND]; return Counted(::NAME(a.v)); }
OPC_UNARY(sqrt, OPC_SQRT)
OPC_UNARY(sin, OPC_MATH)
OPC_UNARY(cos, OPC_MATH)
OPC_UNARY(tan, OPC_MATH)
OPC_UNARY(asin, OPC_MATH)
OPC_UNARY(acos, OPC_MATH)
OPC_UNARY(atan, OPC_MATH)
OPC_UNARY(exp, OPC_MATH)
OPC_UNARY(log, OPC_MATH)
OPC_UNARY(log10, OPC_MATH)
OPC_UNARY(cosh, OPC_MATH)
OPC_UNARY(sinh, OPC_MATH)
OPC_UNARY(tanh, OPC_MATH)
#undef OPC_UNARY
inline Counted fabs(Counted a) { return Counted(::fabs(a.v)); }
inline Counted abs(Counted a) { return Counted(::fabs(a.v)); }
inline Counted floor(Counted a) { return Counted(::floor(a.v)); }
inline Counted ceil(Counted a) { return Counted(::ceil(a.v)); }
inline Counted round(Counted a) { return Counted(::round(a.v)); }
inline bool isnan(Counted a) { return __builtin_isnan(a.v); }
inline bool isfinite(Counted a) { return __builtin_isfinite(a.v); }
inline bool isinf(Counted a) { return __builtin_isinf(a.v); }
inline Counted atan2(Counted y, Counted x) { ++g_count[wq3d_opcount::OPC_MATH]; return Counted(::atan2(y.v, x.v)); }
inline Counted pow(Counted a, Counted b) { ++g_count[wq3d_opcount::OPC_MATH]; return Counted(::pow(a.v, b.v)); }
inline Counted pow(Counted a, double b) { ++g_count[wq3d_opcount::OPC_MATH]; return Counted(::pow(a.v, b)); }
inline Counted pow(double a, Counted b) { ++g_count[wq3d_opcount::OPC_MATH]; return Counted(::pow(a, b.v)); }
inline Counted fmod(Counted a, Counted b) { ++g_count[wq3d_opcount::OPC_DIV]; return Counted(::fmod(a.v, b.v)); }
inline Counted fmod(Counted a, double b) { ++g_count[wq3d_opcount::OPC_DIV]; return Counted(::fmod(a.v, b)); }
inline Counted hypot(Counted a, Counted b) { ++g_count[wq3d_opcount::OPC_SQRT]; return Counted(::hypot(a.v, b.v)); }
inline Counted copysign(Counted a, Counted b) { return Counted(::copysign(a.v, b.v)); }
inline Counted fmax(Counted a, Counted b) { ++g_count[wq3d_opcount::OPC_CMP]; return Counted(::fmax(a.v, b.v)); }
inline Counted fmin(Counted a, Counted b) { ++g_count[wq3d_opcount::OPC_CMP]; return Counted(::fmin(a.v, b.v)); }
}  // namespace std

typedef double oracle_plain_double;
#define ORACLE_OPCOUNT 1
#define double wq3d_opcount::Counted
#include "wq3d_oracle.cpp"
#undef double

extern "C" {
int oracle_opcount_read(uint64_t* out) {
    for (int p = 0; p < wq3d_opcount::OPC_PHASES; ++p)
        for (int k = 0; k < wq3d_opcount::OPC_N; ++k) out[p * wq3d_opcount::OPC_N + k] = wq3d_opcount::g_counts[p][k];
    return 0;
}
int oracle_opcount_reset(void) {
    for (int p = 0; p < wq3d_opcount::OPC_PHASES; ++p)
        for (int k = 0; k < wq3d_opcount::OPC_N; ++k) wq3d_opcount::g_counts[p][k] = 0;
    return 0;
}
}
