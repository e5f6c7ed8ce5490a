// Analytic radial forms on the device: the 34 closed forms of the reference
// (include/forcesmith/potentials/analytic_potential.hpp:304-806), written once
// over a hyper-dual scalar so that one expression yields the value, d/dr,
// d²/dr² and the parameter partials ∂/∂θ_k, ∂²/∂r∂θ_k that the reference
// derives symbolically (AnalyticForm::eval / deriv / deriv2 / param_grad /
// dderiv_dparam, analytic_potential.hpp:156-298).
//
// A hyper-dual number is a + b ε1 + c ε2 + d ε1ε2 with ε1² = ε2² = 0.  Seeding
// r = (r, 1, 0, 0) gives (v, dv/dr); r = (r, 1, 1, 0) puts d²v/dr² in d; r =
// (r, 1, 0, 0) with θ_k = (θ_k, 0, 1, 0) gives ∂v/∂θ_k in c and ∂²v/∂r∂θ_k in d.
//
// No device function here recurses (the smooth-cutoff forms call form_base,
// never form_expr), so every kernel's stack size is known at compile time.
#pragma once

#include <cuda_runtime.h>

namespace fsg {

template <class T> struct Hd {
  T a, b, c, d;
};

template <class T> __device__ __forceinline__ Hd<T> hd_c(T v) { return Hd<T>{v, T(0), T(0), T(0)}; }

template <class T> __device__ __forceinline__ Hd<T> operator+(Hd<T> x, Hd<T> y) {
  return {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d};
}
template <class T> __device__ __forceinline__ Hd<T> operator-(Hd<T> x, Hd<T> y) {
  return {x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d};
}
template <class T> __device__ __forceinline__ Hd<T> operator-(Hd<T> x) { return {-x.a, -x.b, -x.c, -x.d}; }
template <class T> __device__ __forceinline__ Hd<T> operator*(Hd<T> x, Hd<T> y) {
  return {x.a * y.a, x.a * y.b + x.b * y.a, x.a * y.c + x.c * y.a, x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a};
}
template <class T> __device__ __forceinline__ Hd<T> operator*(T s, Hd<T> x) { return {s * x.a, s * x.b, s * x.c, s * x.d}; }
template <class T> __device__ __forceinline__ Hd<T> operator+(T s, Hd<T> x) { return {s + x.a, x.b, x.c, x.d}; }
template <class T> __device__ __forceinline__ Hd<T> operator-(T s, Hd<T> x) { return {s - x.a, -x.b, -x.c, -x.d}; }
template <class T> __device__ __forceinline__ Hd<T> operator-(Hd<T> x, T s) { return {x.a - s, x.b, x.c, x.d}; }

// f(x) with f, f', f'' at x.a
template <class T> __device__ __forceinline__ Hd<T> hd_lift(Hd<T> x, T f, T f1, T f2) {
  return {f, f1 * x.b, f1 * x.c, f1 * x.d + f2 * x.b * x.c};
}
template <class T> __device__ __forceinline__ Hd<T> hd_recip(Hd<T> x) {
  const T i = T(1) / x.a;
  return hd_lift(x, i, -i * i, T(2) * i * i * i);
}
template <class T> __device__ __forceinline__ Hd<T> operator/(Hd<T> x, Hd<T> y) { return x * hd_recip(y); }
template <class T> __device__ __forceinline__ Hd<T> hd_exp(Hd<T> x) {
  const T e = exp(x.a);
  return hd_lift(x, e, e, e);
}
template <class T> __device__ __forceinline__ Hd<T> hd_sqrt(Hd<T> x) {
  const T s = sqrt(x.a);
  return hd_lift(x, s, T(0.5) / s, T(-0.25) / (s * x.a));
}
template <class T> __device__ __forceinline__ Hd<T> hd_cos(Hd<T> x) {
  T sn, cs;
  if constexpr (sizeof(T) == 4) sincosf(x.a, &sn, &cs);
  else sincos(x.a, &sn, &cs);
  return hd_lift(x, cs, -sn, -cs);
}
// min / max: the selected operand with its derivative parts (ties take x)
template <class T> __device__ __forceinline__ Hd<T> hd_min(Hd<T> x, Hd<T> y) { return x.a <= y.a ? x : y; }
template <class T> __device__ __forceinline__ Hd<T> hd_max(Hd<T> x, Hd<T> y) { return x.a >= y.a ? x : y; }
// x^p with a constant exponent
template <class T> __device__ __forceinline__ Hd<T> hd_powc(Hd<T> x, T p) {
  const T v = pow(x.a, p);
  return hd_lift(x, v, p * pow(x.a, p - T(1)), p * (p - T(1)) * pow(x.a, p - T(2)));
}
// x^p with a variable exponent: the value is pow(x, p) (so a negative base
// with an integral exponent keeps its value); ln x enters only through the
// exponent's own derivative parts
template <class T> __device__ __forceinline__ Hd<T> hd_pow(Hd<T> x, Hd<T> p) {
  const T v = pow(x.a, p.a);
  const T fx = p.a * pow(x.a, p.a - T(1));
  const T fxx = p.a * (p.a - T(1)) * pow(x.a, p.a - T(2));
  Hd<T> o{v, fx * x.b, fx * x.c, fx * x.d + fxx * x.b * x.c};
  if (p.b != T(0) || p.c != T(0) || p.d != T(0)) {
    const T L = log(x.a);
    const T fp = v * L, fpp = v * L * L, fxp = pow(x.a, p.a - T(1)) * (T(1) + p.a * L);
    o.b += fp * p.b;
    o.c += fp * p.c;
    o.d += fp * p.d + fxp * (x.b * p.c + p.b * x.c) + fpp * p.b * p.c;
  }
  return o;
}

constexpr int kFormCount = 34;
constexpr int kFormMaxParams = 16;

__host__ __device__ __forceinline__ int form_param_count(int form) {
  constexpr int np[kFormCount] = {2, 3, 2, 2, 2, 3, 2, 3, 3, 1, 3, 5,  // 0-11
                                  4, 6, 6, 7, 5, 7, 5, 6, 5, 6, 2,     // 12-22
                                  11, 2, 16, 9, 12, 2, 5, 3, 4, 3, 7}; // 23-33
  return (form >= 0 && form < kFormCount) ? np[form] : -1;
}

// detail::cosine_cutoff (analytic_potential.hpp:142-145)
template <class T> __device__ __forceinline__ Hd<T> hd_cos_cut(Hd<T> r, Hd<T> lo, Hd<T> hi) {
  const T pi = T(3.14159265358979323846);
  return T(0.5) + T(0.5) * hd_cos(pi * (hd_min(hd_max(r, lo), hi) - lo) / (hi - lo));
}
// detail::switching_factor (analytic_potential.hpp:147-151): u⁴/(1 + u⁴), u = min((r − r0)/h, 0)
template <class T> __device__ __forceinline__ Hd<T> hd_switch(Hd<T> r, T r0, Hd<T> h) {
  const Hd<T> u = hd_min((r - r0) / h, hd_c(T(0)));
  const Hd<T> u4 = (u * u) * (u * u);
  return u4 / (T(1) + u4);
}

// The expressions of forms 0-29 at r; p holds the form's parameters.
template <class T> __device__ Hd<T> form_base(int form, const Hd<T> *p, Hd<T> r) {
  using H = Hd<T>;
  const T one = T(1);
  switch (form) {
  case 0: { // LennardJones 4ε(sr6² − sr6), sr6 = (σ/r)^6
    const H sr6 = hd_powc(p[1] / r, T(6));
    return (T(4) * p[0]) * (sr6 * sr6 - sr6);
  }
  case 1: { // Morse De(1 − e)² − De, e = exp(−a(r − re))
    const H e = hd_exp(-(p[1] * (r - p[2])));
    return p[0] * (one - e) * (one - e) - p[0];
  }
  case 2: return p[0] * hd_exp(-(p[1] * r));                          // ExpDecay
  case 3: return p[0] * hd_sqrt(r / p[1]);                            // SqrtFunc
  case 4: return p[0] / hd_pow(r, p[1]);                              // PowerDecay
  case 5: return p[0] * hd_exp(-(p[1] * (r - p[2])));                 // MexpDecay
  case 6: return p[0] * (r - p[1]) * (r - p[1]);                      // Harmonic
  case 7: return p[0] * hd_exp(-(p[1] * r)) + p[2];                   // ExpPlus
  case 8: return p[0] * r * r + p[1] * r + p[2];                      // Parabola
  case 9: return p[0] + T(0) * r;                                     // ConstFunc
  case 10: { // Buckingham A exp(−r/ρ) − C (ρ²/r²)³
    const H x = (p[1] * p[1]) / (r * r);
    return p[0] * hd_exp(-(r / p[1])) - p[2] * x * x * x;
  }
  case 11: { // Born A exp((C − r)/B) − D/r⁶ + E/r⁸
    const H r2 = r * r, r6 = r2 * r2 * r2;
    return p[0] * hd_exp((p[2] - r) / p[1]) - p[3] / r6 + p[4] / (r6 * r2);
  }
  case 12: // Universal {E0, a, b, c}
    return p[0] * (p[2] / (p[2] - p[1]) * hd_pow(r, p[1]) - p[1] / (p[2] - p[1]) * hd_pow(r, p[2])) + p[3] * r;
  case 13: // Eopp {A, n, B, m, k, phi}
    return p[0] / hd_pow(r, p[1]) + (p[2] / hd_pow(r, p[3])) * hd_cos(p[4] * r + p[5]);
  case 14: // EoppExp {A, B, C, m, k, phi}
    return p[0] * hd_exp(-(p[1] * r)) + (p[2] / hd_pow(r, p[3])) * hd_cos(p[4] * r + p[5]);
  case 15: // Meopp {A, n, B, m, k, phi, r0}
    return p[0] / hd_pow(r - p[6], p[1]) + (p[2] / hd_pow(r, p[3])) * hd_cos(p[4] * r + p[5]);
  case 16: { // GenLJ {A, n, m, r0, B}
    const H x = r / p[3];
    return p[0] / (p[2] - p[1]) * (p[2] * hd_pow(x, -p[1]) - p[1] * hd_pow(x, -p[2])) + p[4];
  }
  case 17: { // DoubleMorse {D1, a1, r1, D2, a2, r2, C}
    const H e1 = hd_exp(-(p[1] * (r - p[2]))), e2 = hd_exp(-(p[4] * (r - p[5])));
    return p[0] * ((one - e1) * (one - e1) - one) + p[3] * ((one - e2) * (one - e2) - one) + p[6];
  }
  case 18: { // DoubleExp {A, B, r1, C, r2}
    const H dr = r - p[2];
    return p[0] * hd_exp(-(p[1] * dr * dr)) + hd_exp(-(p[3] * (r - p[4])));
  }
  case 19: { // Mishin {A, B, C, r0, n, d}
    const H z = r - p[3];
    const H e = hd_exp(-(p[5] * z));
    return p[0] * hd_pow(z, p[4]) * e * (one + p[1] * e) + p[2];
  }
  case 20: { // Poly5 {a0..a4}, s = r − 1
    const H s = r - one, s2 = s * s;
    return p[0] + (T(0.5) * p[1]) * s2 + p[2] * s * s2 + p[3] * s2 * s2 + p[4] * s2 * s2 * s;
  }
  case 21: // StiwWeb2 {A, B, p, q, delta, rc}
    return (p[0] * hd_pow(r, -p[2]) - p[1] * hd_pow(r, -p[3])) * hd_exp(p[4] / (r - p[5]));
  case 22: return hd_exp(p[0] / (r - p[1]));                          // StiwWeb3 {gamma, a}
  case 23: // TersoffPot {A, B, lambda, mu, beta, n, c, d, h, R, S}
    return hd_cos_cut(r, p[9], p[10]) * (p[0] * hd_exp(-(p[2] * r)) - p[1] * hd_exp(-(p[3] * r)));
  case 24: return p[0] * hd_exp(-(p[1] * r));                         // TersoffMix {chi, omega}
  case 25: { // TersoffModPot: TersoffPot × (1 + c1 r + … + c5 r⁵)
    const H r2 = r * r, r3 = r2 * r, r4 = r3 * r, r5 = r4 * r;
    return hd_cos_cut(r, p[9], p[10]) * (p[0] * hd_exp(-(p[2] * r)) - p[1] * hd_exp(-(p[3] * r))) *
           (one + p[11] * r + p[12] * r2 + p[13] * r3 + p[14] * r4 + p[15] * r5);
  }
  case 26: { // Kawamura {A..I}
    const H s = p[5] + p[6], t = p[3] + p[4];
    return p[0] * p[1] / r + p[2] * s * hd_exp((t - r) / s) - p[7] * p[8] / hd_powc(r, T(6));
  }
  case 27: { // KawamuraMix {A..L}
    const H s = p[5] + p[6], t = p[3] + p[4], w = r - p[11];
    return p[0] * p[1] / r + p[2] * s * hd_exp((t - r) / s) - p[7] * p[8] / hd_powc(r, T(6)) +
           p[2] * p[9] * (hd_exp(T(-2) * (p[10] * w)) - T(2) * hd_exp(-(p[10] * w)));
  }
  case 28: return hd_pow(p[0] / r, p[1]);                             // Softshell {A, n}
  case 29: { // Strmm {A, B, C, D, E}
    const H s = r - p[4];
    return (T(2) * p[0]) * hd_exp((T(-0.5) * p[1]) * s) - p[2] * (one + p[3] * s) * hd_exp(-(p[3] * s));
  }
  }
  return hd_c(T(0));
}

// Every form at r (rmax: the table's upper gate bound, where the `_sc` forms
// switch off).  The smooth-cutoff forms are their base form times the
// switching factor (SmoothCutoff, analytic_potential.hpp:782-793).
template <class T> __device__ __forceinline__ Hd<T> form_expr(int form, const Hd<T> *p, Hd<T> r, T rmax) {
  switch (form) {
  case 30: return form_base<T>(0, p, r) * hd_switch(r, rmax, p[2]);  // LennardJonesSC
  case 31: return form_base<T>(1, p, r) * hd_switch(r, rmax, p[3]);  // MorseSC
  case 32: return form_base<T>(2, p, r) * hd_switch(r, rmax, p[2]);  // ExpDecaySC
  case 33: return form_base<T>(13, p, r) * hd_switch(r, rmax, p[6]); // EoppSC
  }
  return form_base<T>(form, p, r);
}

// StiwWeb2 / StiwWeb3 are exactly zero past their cut-off, or where the
// exponent would underflow (StiwWeb2::outside, analytic_potential.hpp:587-590);
// their parameter partials are zero there as well.
template <class T> __device__ __forceinline__ bool form_outside(int form, const double *pp, T r) {
  if (form == 21 || form == 22) {
    const int k = form == 21 ? 5 : 1;
    const T d = r - static_cast<T>(pp[k]);
    return d >= T(0) || static_cast<T>(pp[k - 1]) / d < T(-708);
  }
  return false;
}

// Evaluate with r seeded as (r, 1, s2, 0) and parameter kp (if ≥ 0) seeded
// as (θ, 0, 1, 0).
template <class T>
__device__ __forceinline__ Hd<T> form_seeded(int form, const double *pp, int n, T r, T rmax, T s2, int kp) {
  Hd<T> p[kFormMaxParams];
#pragma unroll
  for (int k = 0; k < kFormMaxParams; ++k)
    p[k] = Hd<T>{k < n ? static_cast<T>(pp[k]) : T(0), T(0), (k == kp) ? T(1) : T(0), T(0)};
  return form_expr<T>(form, p, Hd<T>{r, T(1), s2, T(0)}, rmax);
}

} // namespace fsg
