// Forward-mode dual numbers for the tangent (JVP) kernels: a value and N directional
// derivatives, with the arithmetic the level-set and chemistry updates use.  Branches
// (comparisons, min / max, clamps) follow the value, so a dual evaluation takes exactly the
// primal's branch and carries the derivative of that branch.
#pragma once
#include <cmath>

namespace petch {

// Elementary float operations, each rounded on its own on the device (no fused multiply-add), so
// an expression gives the same bits in every kernel that inlines it; double keeps the plain
// operators (the chemistry duals follow the plain double kernels' code generation).
__host__ __device__ inline float rn_add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ inline float rn_sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ inline float rn_mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ inline double rn_add(double a, double b) { return a + b; }
__host__ __device__ inline double rn_sub(double a, double b) { return a - b; }
__host__ __device__ inline double rn_mul(double a, double b) { return a * b; }

template <class S, int N>
struct Dual {
    S v;
    S d[N];
};

template <class S, int N>
__host__ __device__ inline Dual<S, N> dconst(S v) {
    Dual<S, N> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = S(0);
    return r;
}

#define PETCH_DUAL_BINOP(OP, VAL, DER)                                                           \
    template <class S, int N>                                                                    \
    __host__ __device__ inline Dual<S, N> operator OP(const Dual<S, N>& a, const Dual<S, N>& b) { \
        Dual<S, N> r;                                                                            \
        r.v = VAL;                                                                               \
        _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DER;                              \
        return r;                                                                                \
    }
PETCH_DUAL_BINOP(+, rn_add(a.v, b.v), rn_add(a.d[k], b.d[k]))
PETCH_DUAL_BINOP(-, rn_sub(a.v, b.v), rn_sub(a.d[k], b.d[k]))
PETCH_DUAL_BINOP(*, rn_mul(a.v, b.v), rn_add(rn_mul(a.d[k], b.v), rn_mul(a.v, b.d[k])))
#undef PETCH_DUAL_BINOP

template <class S, int N>
__host__ __device__ inline Dual<S, N> operator/(const Dual<S, N>& a, const Dual<S, N>& b) {
    Dual<S, N> r;
    r.v = a.v / b.v;
    const S ib = S(1) / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = rn_mul(rn_sub(a.d[k], rn_mul(r.v, b.d[k])), ib);
    return r;
}

template <class S, int N>
__host__ __device__ inline Dual<S, N> operator-(const Dual<S, N>& a) {
    Dual<S, N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}

// mixed scalar forms
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator+(const Dual<S, N>& a, S b) { return a + dconst<S, N>(b); }
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator+(S a, const Dual<S, N>& b) { return dconst<S, N>(a) + b; }
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator-(const Dual<S, N>& a, S b) { return a - dconst<S, N>(b); }
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator-(S a, const Dual<S, N>& b) { return dconst<S, N>(a) - b; }
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator*(const Dual<S, N>& a, S b) {
    Dual<S, N> r;
    r.v = rn_mul(a.v, b);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = rn_mul(a.d[k], b);
    return r;
}
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator*(S a, const Dual<S, N>& b) { return b * a; }
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator/(const Dual<S, N>& a, S b) {
    Dual<S, N> r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <class S, int N>
__host__ __device__ inline Dual<S, N> operator/(S a, const Dual<S, N>& b) { return dconst<S, N>(a) / b; }

// ---- generic helpers: plain overloads for float / double, dual ones following the value ----
__host__ __device__ inline float vval(float x) { return x; }
__host__ __device__ inline double vval(double x) { return x; }
template <class S, int N>
__host__ __device__ inline S vval(const Dual<S, N>& x) { return x.v; }

__host__ __device__ inline float vmax(float a, float b) { return fmaxf(a, b); }
__host__ __device__ inline float vmin(float a, float b) { return fminf(a, b); }
__host__ __device__ inline float vsqrt(float a) { return sqrtf(a); }
__host__ __device__ inline float vabs(float a) { return fabsf(a); }
__host__ __device__ inline double vmax(double a, double b) { return fmax(a, b); }
__host__ __device__ inline double vmin(double a, double b) { return fmin(a, b); }
__host__ __device__ inline double vsqrt(double a) { return sqrt(a); }
__host__ __device__ inline double vabs(double a) { return fabs(a); }

// max / min pick an operand (ties: the first, as fmaxf / fminf return either when equal)
template <class S, int N>
__host__ __device__ inline Dual<S, N> vmax(const Dual<S, N>& a, const Dual<S, N>& b) {
    return (b.v > a.v) ? b : a;
}
template <class S, int N>
__host__ __device__ inline Dual<S, N> vmin(const Dual<S, N>& a, const Dual<S, N>& b) {
    return (b.v < a.v) ? b : a;
}
template <class S, int N>
__host__ __device__ inline Dual<S, N> vmax(const Dual<S, N>& a, S b) { return vmax(a, dconst<S, N>(b)); }
template <class S, int N>
__host__ __device__ inline Dual<S, N> vmin(const Dual<S, N>& a, S b) { return vmin(a, dconst<S, N>(b)); }

// sqrt: derivative 0 at 0 (where the primal's one-sided differences vanish)
template <class S, int N>
__host__ __device__ inline Dual<S, N> vsqrt(const Dual<S, N>& a) {
    Dual<S, N> r;
    r.v = sqrt(a.v);
    const S g = r.v > S(0) ? S(0.5) / r.v : S(0);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = rn_mul(a.d[k], g);
    return r;
}

template <class S, int N>
__host__ __device__ inline Dual<S, N> vabs(const Dual<S, N>& a) {
    return signbit(a.v) ? -a : a;
}

}  // namespace petch
