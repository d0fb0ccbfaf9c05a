// g4b_dual.cuh - forward-mode dual numbers for the gradient replay.
//
// Dual<T> carries a value and its derivative with respect to one parameter
// (the refractive index of the material whose index is differentiated). The
// value part goes through exactly the operations the plain T path performs,
// so a replay with Dual<float> follows the FP32 history bit for bit while the
// derivative rides along. Comparisons look at values only: discrete choices
// are not differentiated here; their probabilities enter as score terms.
#pragma once

#include <cuda_runtime.h>

namespace g4b {
namespace dev {

template<class T>
struct Dual {
    T v;
    T d;
    Dual() = default;
    __device__ __forceinline__ constexpr Dual(float value) : v(static_cast<T>(value)), d(T(0)) {}
    __device__ __forceinline__ constexpr Dual(double value) : v(static_cast<T>(value)), d(T(0)) {}
    __device__ __forceinline__ constexpr Dual(int value) : v(static_cast<T>(value)), d(T(0)) {}
    __device__ __forceinline__ constexpr Dual(T value, T derivative, int) : v(value), d(derivative) {}
    __device__ __forceinline__ explicit operator double() const { return static_cast<double>(v); }
    __device__ __forceinline__ explicit operator float() const { return static_cast<float>(v); }
};

template<class T>
__device__ __forceinline__ Dual<T> MakeDual(T value, T derivative) {
    return Dual<T>(value, derivative, 0);
}

template<class T>
struct IsDualType {
    static constexpr bool value = false;
};
template<class T>
struct IsDualType<Dual<T>> {
    static constexpr bool value = true;
};

template<class T>
__device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return MakeDual(a.v + b.v, a.d + b.d); }
template<class T>
__device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return MakeDual(a.v - b.v, a.d - b.d); }
template<class T>
__device__ __forceinline__ Dual<T> operator-(Dual<T> a) { return MakeDual(-a.v, -a.d); }
template<class T>
__device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) {
    return MakeDual(a.v * b.v, a.d * b.v + a.v * b.d);
}
template<class T>
__device__ __forceinline__ Dual<T> operator/(Dual<T> a, Dual<T> b) {
    const T q{a.v / b.v};
    return MakeDual(q, (a.d - q * b.d) / b.v);
}
template<class T>
__device__ __forceinline__ Dual<T>& operator+=(Dual<T>& a, Dual<T> b) { return a = a + b; }
template<class T>
__device__ __forceinline__ Dual<T>& operator-=(Dual<T>& a, Dual<T> b) { return a = a - b; }

template<class T>
__device__ __forceinline__ bool operator<(Dual<T> a, Dual<T> b) { return a.v < b.v; }
template<class T>
__device__ __forceinline__ bool operator>(Dual<T> a, Dual<T> b) { return a.v > b.v; }
template<class T>
__device__ __forceinline__ bool operator<=(Dual<T> a, Dual<T> b) { return a.v <= b.v; }
template<class T>
__device__ __forceinline__ bool operator>=(Dual<T> a, Dual<T> b) { return a.v >= b.v; }
template<class T>
__device__ __forceinline__ bool operator==(Dual<T> a, Dual<T> b) { return a.v == b.v; }
template<class T>
__device__ __forceinline__ bool operator!=(Dual<T> a, Dual<T> b) { return a.v != b.v; }

template<class T>
__device__ __forceinline__ bool IsFinite(Dual<T> a) { return IsFinite(a.v); }

template<class T>
__device__ __forceinline__ Dual<T> Sqrt(Dual<T> a) {
    const T r{Sqrt(a.v)};
    return MakeDual(r, a.d == T(0) ? T(0) : a.d / (T(2) * r));
}
template<class T>
__device__ __forceinline__ Dual<T> Fabs(Dual<T> a) { return a.v < T(0) ? -a : a; }
template<class T>
__device__ __forceinline__ Dual<T> Fmin(Dual<T> a, Dual<T> b) {
    // fmin's value (NaN-aware) with the derivative of the operand it returned
    const T m{Fmin(a.v, b.v)};
    return MakeDual(m, (m == a.v && !(a.v != a.v)) ? a.d : b.d);
}
template<class T>
__device__ __forceinline__ Dual<T> Fmax(Dual<T> a, Dual<T> b) {
    const T m{Fmax(a.v, b.v)};
    return MakeDual(m, (m == a.v && !(a.v != a.v)) ? a.d : b.d);
}
template<class T>
__device__ __forceinline__ Dual<T> Log(Dual<T> a) { return MakeDual(Log(a.v), a.d / a.v); }
template<class T>
__device__ __forceinline__ Dual<T> Exp(Dual<T> a) {
    const T e{Exp(a.v)};
    return MakeDual(e, a.d * e);
}
template<class T>
__device__ __forceinline__ void SinCosTurn(Dual<T> t, Dual<T>* s, Dual<T>* c) {
    T sv, cv;
    SinCosTurn(t.v, &sv, &cv);
    const T twoPi{T(6.28318530717958647692)};
    *s = MakeDual(sv, twoPi * cv * t.d);
    *c = MakeDual(cv, -twoPi * sv * t.d);
}

template<>
__device__ __forceinline__ Dual<float> Infinity<Dual<float>>() { return Dual<float>(Infinity<float>()); }
template<>
__device__ __forceinline__ Dual<double> Infinity<Dual<double>>() { return Dual<double>(Infinity<double>()); }
template<>
__device__ __forceinline__ Dual<float> QuietNaN<Dual<float>>() { return Dual<float>(QuietNaN<float>()); }
template<>
__device__ __forceinline__ Dual<double> QuietNaN<Dual<double>>() { return Dual<double>(QuietNaN<double>()); }

template<>
__device__ __forceinline__ Dual<float> Uniform<Dual<float>>(unsigned long long seed, unsigned long long key,
                                                            std::uint32_t bounce, std::uint32_t process,
                                                            std::uint32_t draw) {
    return Dual<float>(Uniform<float>(seed, key, bounce, process, draw));
}
template<>
__device__ __forceinline__ Dual<double> Uniform<Dual<double>>(unsigned long long seed, unsigned long long key,
                                                              std::uint32_t bounce, std::uint32_t process,
                                                              std::uint32_t draw) {
    return Dual<double>(Uniform<double>(seed, key, bounce, process, draw));
}

// UniformFromWord for plain and dual numbers (a draw carries no derivative).
template<class R>
__device__ __forceinline__ R UniformSample(std::uint32_t word) {
    if constexpr (IsDualType<R>::value) {
        return R(UniformFromWord<decltype(R{}.v)>(word));
    } else {
        return UniformFromWord<R>(word);
    }
}

// The value of a plain or dual number, and the value of one with the
// derivative of another (used where the value comes from an FP64 side
// computation the dual arithmetic cannot see).
template<class R>
__device__ __forceinline__ double ValueOf(R x) {
    return static_cast<double>(x);
}
template<class R>
__device__ __forceinline__ R WithDerivativeOf(R value, R source) {
    if constexpr (IsDualType<R>::value) {
        value.d = source.d;
    }
    return value;
}

}  // namespace dev
}  // namespace g4b
