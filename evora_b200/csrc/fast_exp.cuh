// fast_exp.cuh -- exp(x) by the table-driven method of Tang (ACM TOMS
// 15(2), 1989, "Table-driven implementation of the exponential function in
// IEEE floating-point arithmetic"), for the FP64 fast forms: the default
// mode's chemistry (chem_fast.cu, table staged in shared memory) and the
// dual-energy powers rho^(g-1) of the FP64 hydro kernels (hydro_math.cuh,
// table read through the read-only cache).  About 1 ulp, no branch.
#pragma once

namespace evora {

// 2^(j/32), j = 0..31, rounded to nearest double (from 60-digit decimal
// arithmetic).
__device__ const double kExp2Frac[32] = {
    0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0,
    0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0,
    0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0,
    0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0,
    0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0,
    0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0,
    0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0,
    0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0,
};

// exp(x) by Tang's table-driven method: x = (32 m + j) ln2/32 + r with
// n = 32 m + j = rint(32 x / ln2), so |r| <= ln2/64 (a little more when the
// product rounds across a half), then exp(x) = 2^m 2^(j/32) (1 + p(r)).
// ln2/32 is split in a leading and a trailing double so that r is exact to
// about 2^-100 relative to x.  x is clamped to [-746, 710] (NaN passes
// through the comparisons), outside of which exp rounds to 0 or overflows;
// 2^m is applied as two powers of two so that a subnormal result rounds
// once.  tab(j) returns 2^(j/32) (kExp2Frac[j]).
template <class Tab>
__device__ __forceinline__ double exp_tang(double x, const Tab& tab) {
  constexpr double kInvL = 0x1.71547652b82fep+5;     // 32 / ln 2
  constexpr double kLhi = 0x1.62e42fefa39efp-6;      // ln 2 / 32, leading part
  constexpr double kLlo = 0x1.abc9e3b39803fp-61;     // ... and trailing part
  x = x < -746.0 ? -746.0 : x;
  x = x > 710.0 ? 710.0 : x;
  const double nd = rint(x * kInvL);
  const int n = __double2int_rn(nd);
  double r = fma(-nd, kLhi, x);
  r = fma(-nd, kLlo, r);
  // e^r - 1 = r + r^2/2 + ... + r^6/720
  double p = fma(r, 1.0 / 720.0, 1.0 / 120.0);
  p = fma(p, r, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = p * r;
  const double s = tab(n & 31);
  const double y = fma(s, p, s);
  const int m = n >> 5;   // floor(n / 32): -1077 .. 1024 after the clamp (NaN: any; y is NaN)
  const int m1 = m >> 1, m2 = m - m1;
  const double s1 = __longlong_as_double((long long)((unsigned long long)(m1 + 1023) << 52));
  const double s2 = __longlong_as_double((long long)((unsigned long long)(m2 + 1023) << 52));
  return (y * s1) * s2;
}

// Tang's exp with the table staged at tab (shared memory).
struct ExpTable {
  const double* tab;
  __device__ __forceinline__ double operator()(double x) const {
    return exp_tang(x, [this](int j) { return tab[j]; });
  }
};

// Tang's exp with the table read from global memory through the read-only
// cache.
__device__ __forceinline__ double exp_global(double x) {
  return exp_tang(x, [](int j) { return __ldg(&kExp2Frac[j]); });
}

}  // namespace evora
