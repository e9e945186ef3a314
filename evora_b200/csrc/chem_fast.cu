// chem_fast.cu -- chem(q) (chemistry.f90:72-121) of the default (not
// STRICT) mode on a resident SoA state: the cell update of chem_cell.cuh with
// the CIE cooling sub-cycles (cie.f90:26-56) evaluating fewer FP64
// operations per cycle than the reference's order of operations (chem.cu):
//
//   * the rates (rates.f90:80-158) share their powers of T: T^-3/2 =
//     T^-1 T^-1/2 and T^-1/2 = T^-1 sqrt(T) are products instead of an
//     exponential and a division; T^0.3647 = T T^-0.6353 exp(-2^-25 ln T)
//     (the single-precision literals 0.3647 and -0.6353 differ by exactly
//     1 - 2^-25), e^(-2^-25 ln T) by its cubic Taylor polynomial;
//     T^-0.397 exp(-473638/T) is one exponential of the summed arguments;
//   * the remaining nine exponentials per cycle use the table-driven method
//     of Tang (ACM TOMS 15(2), 1989, "Table-driven implementation of the
//     exponential function in IEEE floating-point arithmetic") with 32
//     table entries and the degree-6 Taylor polynomial of e^r - 1 on
//     |r| <= ln2/64 (truncation below 4e-18), about 1 ulp;
//   * 8 reciprocals (rcp64: the hardware's approximation and two Newton
//     steps, within an ulp) instead of 12 divisions per cycle: those of p
//     and sum(n) are shared by T, 1/T and the pressure update, and the
//     equilibrium abundances take one per element;
//   * products and sums contract to FMAs (this unit is compiled with them).
//
// Results stay within a few ulp of the reference order per rate; the cells'
// trajectories agree with the oracle to the chemistry tests' tolerances.
// Species and cooling are FP64 whatever the state precision.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/evora_gpu.h"
#include "chem.h"
#include "chem_cell.cuh"
#include "chemistry.cuh"
#include "common.h"
#include "fast_exp.cuh"

namespace evora {
namespace {

// 128-thread blocks, 4 per SM (128 registers per thread, a few spills):
// measured at 256^3 against 5 and 6 blocks per SM (96 and 80 registers,
// more spills), which ran about 3 and 2 % slower.
constexpr int kChemThreads = 128;
constexpr int kChemMinBlocks = 4;

// 1/x from the hardware's approximate FP64 reciprocal (rcp.approx.ftz.f64,
// relative error about 1e-6, checked below 2^-16 by evora_selftest_exp) and
// two Newton steps (e -> e^2 -> e^4, past 2^-64): within an ulp of the
// quotient for normal x and results, with no branch to a slow path.  x = +-0, +-inf and NaN give the
// approximation itself (+-inf, +-0, NaN: the residual is NaN there); a
// subnormal x (flushed) gives +-inf.
__device__ __forceinline__ double rcp64(double x) {
  double r0;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(x));
  double e = fma(-x, r0, 1.0);
  double r = fma(r0, e, r0);
  e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  return e == e ? r : r0;
}

// The rate coefficients staged in shared memory (c[i][j] at 2 i + j), read
// where they are used: a volatile load is not hoisted out of the sub-cycle
// loop, so the 26 coefficients hold no registers across it.
struct CoefShared {
  const double* c;
  __device__ __forceinline__ double operator()(int i, int j) const {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"((unsigned)__cvta_generic_to_shared(c + 2 * i + j)));
    return v;
  }
};

// comprates (rates.f90:80-158) at temperature temp (tempinv = 1/temp) with
// the shared powers of T described above; the same outputs as
// chemistry.cuh's comprates.  kc(i, j) = k.c[i][j].
template <class Exp, class Coef>
__device__ __forceinline__ void comprates_fast(double temp, double tempinv, const Coef& kc, int background,
                                               int cooling, const Exp& ex, double* chemrate, double* coolrate) {
  const double lt = log(temp);
  const double temproot = sqrt(temp);
  const double tmhalf = tempinv * temproot;   // T^-1/2
  const double temp15 = tempinv * tmhalf;     // T^-3/2
  // sqrt(T 1e-5) = sqrt(T) sqrt(1e-5)
  const double fec = rcp64(1.0 + temproot * 3.1622776601683794e-3);
  const double fc1 = temproot * fec;
  const double e1 = ex(-((double)157809.1f * tempinv));
  const double e2 = ex(-((double)286335.4f * tempinv));
  const double e3 = ex(-((double)631515.0f * tempinv));
  const double ln1e3 = -6.907755278982137, ln1e6 = -13.815510557964274;   // ln 1e-3, ln 1e-6
  const double fr = ex((double)(-0.2f) * (lt + ln1e3)) * rcp64(1.0 + ex((double)0.7f * (lt + ln1e6)));
  const double fr1 = fr * tmhalf;
  const double fr2 = fr * temproot;
  const float c3 = 0.3f * (-94000.0f);   // a product of two default reals
  const double edr = ex((double)(-470000.0f) * tempinv) * (1.0 + (double)c3 * tempinv);
  const double p6353 = ex((double)(-0.6353f) * lt);   // T^-0.6353
  chemrate[0] = kc(0, 0) * fc1 * e1;
  chemrate[1] = kc(1, 0) * fc1 * e2;
  chemrate[2] = kc(2, 0) * fc1 * e3;
  chemrate[3] = kc(3, 0) * fr1;
  chemrate[4] = kc(4, 0) * p6353 + kc(6, 0) * temp15 * edr;
  chemrate[5] = kc(5, 0) * fr1;
  if (background) {
    chemrate[6] = kc(10, 0);
    chemrate[7] = kc(11, 0);
    chemrate[8] = kc(12, 0);
  } else {
    chemrate[6] = chemrate[7] = chemrate[8] = 0.0;
  }
  if (cooling) {
    // T^0.3647 = T T^-0.6353 e^u, u = -2^-25 ln T (|u| < 2.3e-5 for any
    // finite T > 0): e^u by 1 + u + u^2/2 + u^3/6, error below 2e-20
    const double u = -0x1p-25 * lt;
    const double eu = fma(fma(fma(u, 1.0 / 6.0, 0.5), u, 1.0), u, 1.0);
    coolrate[0] = kc(0, 1) * fc1 * e1;
    coolrate[1] = kc(1, 1) * fc1 * e2;
    coolrate[2] = kc(2, 1) * fc1 * e3;
    coolrate[3] = kc(3, 1) * fr2;
    coolrate[4] = kc(4, 1) * (temp * p6353 * eu);
    coolrate[5] = kc(5, 1) * fr2;
    coolrate[6] = kc(6, 1) * temp15 * edr;
    coolrate[7] = kc(7, 1) * fec * ex((double)(-118348.0f) * tempinv);
    coolrate[8] = kc(8, 1) * fec * ex((double)(-0.397f) * lt + (double)(-473638.0f) * tempinv);
    coolrate[9] = kc(9, 1) * temproot;
    if (background) {
      coolrate[10] = kc(10, 1);
      coolrate[11] = kc(11, 1);
      coolrate[12] = kc(12, 1);
    } else {
      coolrate[10] = coolrate[11] = coolrate[12] = 0.0;
    }
  }
}

// cieabundance (cie.f90:58-85) without a UV background, with one
// reciprocal per element: n(H) = nH cr3 / (cr0 + cr3), n(H+) = nH cr0 /
// (cr0 + cr3), and with D = cr4 cr5 + cr1 cr5 + cr1 cr2, n(He) = nHe cr4 cr5
// / D, n(He+) = nHe cr1 cr5 / D, n(He++) = nHe cr1 cr2 / D (the reference's
// fractions cr0/cr3, cr1/cr4, cr2/cr5 multiplied out); with a background,
// chemistry.cuh's (implicitcie's electron-density root).
__device__ __forceinline__ void cieabundance_fast(double nH, double nHe, double* n, const double* cr,
                                                  int background, double uv, unsigned& err) {
  if (background && uv > 0.0) {
    cieabundance(nH, nHe, n, cr, background, uv, err);
    return;
  }
  const double dH = nH * rcp64(cr[0] + cr[3]);
  n[0] = cr[3] * dH;
  n[1] = cr[0] * dH;
  const double a = cr[4] * cr[5], b = cr[1] * cr[5], c = cr[1] * cr[2];
  const double dHe = nHe * rcp64(a + b + c);
  n[2] = a * dHe;
  n[3] = b * dHe;
  n[4] = c * dHe;
  n[5] = n[1] + n[3] + 2 * n[4];
  check_floor(n, err);
}

// cie (cie.f90:26-56) with comprates_fast and cieabundance_fast: the same
// sub-cycle schedule and pressure update as chemistry.cuh's cie, with the
// reciprocals of p and sum(n) shared: T = p / sum(n) temp0, 1/T =
// sum(n) / p / temp0, cdt Lambda / p.
template <class Exp, class Coef>
struct CieFast {
  Exp ex;
  Coef kc;
  // pressure() (comp.f90:45-85) with the fast forms: kin/E as kin (1/E),
  // rho^(g-1) = exp((g-1) ln rho), the divisions as products with
  // reciprocals; the same write-back of E or S
  __device__ __forceinline__ double pressure(double* q, const Gas<double>& c, bool de, unsigned& err) const {
    const double m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
    const double kin = 0.5 * m2 * rcp64(q[0]);
    double press;
    if (de) {
      const double pg = ex(c.g1 * log(q[0]));
      if (kin * rcp64(q[4]) > c.de_thresh1) {
        press = q[5] * pg;
        q[4] = kin + press * c.g1inv;
      } else {
        press = c.g1 * (q[4] - kin);
        q[5] = press * rcp64(pg);
      }
    } else {
      press = c.g1 * (q[4] - kin);
    }
    if (press <= 0.0) err |= EVORA_ERR_PRESSURE;
    return press;
  }
  __device__ __forceinline__ double div_pow(double a, double x, double y) const { return a * rcp64(ex(y * log(x))); }
  __device__ __forceinline__ double div(double a, double, double binv) const { return a * binv; }
  __device__ __forceinline__ void run(const ChemParams& C, const ChemCoef& k, double temp0, double dt, double rho,
                                      double& press, double* n, unsigned& err) const {
    const double nH = C.chiH * rho, nHe = C.chiHe * rho;
    const double temp0inv = rcp64(temp0);
    double chemrate[kNchem], coolrate[kNcool];
    if (!C.cooling) {
      const double ns = nsum(n);
      comprates_fast(press * rcp64(ns) * temp0, ns * rcp64(press) * temp0inv, kc, C.background, 0, ex,
                     chemrate, coolrate);
      cieabundance_fast(nH, nHe, n, chemrate, C.background, k.uv, err);
      return;
    }
    double ct = 0.0;
    int cycles = 0;
    while (ct < dt) {
      if (++cycles > kCoolMaxCycles) {
        err |= EVORA_ERR_CHEM;
        break;
      }
      const double ns = nsum(n);
      const double pinv = rcp64(press);
      comprates_fast(press * rcp64(ns) * temp0, ns * pinv * temp0inv, kc, C.background, 1, ex, chemrate,
                     coolrate);
      cieabundance_fast(nH, nHe, n, chemrate, C.background, k.uv, err);
      double lambda, gamma;
      cool(n, coolrate, C.background, lambda, gamma);
      const double coolio = gamma - lambda;
      const double cooltime = fabs(press * rcp64(coolio));
      double cdt = C.c_chem * cooltime;
      const double rest = dt - ct, cap = dt * C.substep;
      if (rest < cdt) cdt = rest;   // min(c_chem * cooltime, dt - ct, dt * substep)
      if (cap < cdt) cdt = cap;
      ct = ct + cdt;
      press = (press + cdt * gamma) * rcp64(1.0 + cdt * lambda * pinv);
    }
  }
};

// chem(q) on the resident SoA state, with Tang's exponential (its table
// staged in shared memory) and the rate coefficients read from shared
// memory where they are used.  Both measured faster in the 256^3
// cosmological box: with the library's exp the kernel ran about 14 % slower,
// with the coefficients in registers about 5 %.  expand: the expansion
// terms in the same pass.
template <typename T, int MINB>
__global__ void __launch_bounds__(kChemThreads, MINB)
k_chem_fast(T* __restrict__ q, int64_t n, int nf, double* __restrict__ species, HydroParams P, const GridCtl* ctl,
            unsigned* err, bool expand) {
  if (ctl_skip(ctl)) return;
  __shared__ double tab[32];
  __shared__ double coef[2 * kNcool];
  if (threadIdx.x < 32) tab[threadIdx.x] = kExp2Frac[threadIdx.x];
  if (threadIdx.x < 2 * kNcool) coef[threadIdx.x] = ctl->coef.c[threadIdx.x >> 1][threadIdx.x & 1];
  __syncthreads();
  chem_soa(q, n, nf, species, P, ctl, CieFast<ExpTable, CoefShared>{ExpTable{tab}, CoefShared{coef}}, err, expand);
}

// The self-test of the error bounds over x[0..n): out[i] = Tang's exp(x[i]),
// out[n + i] = rcp64(x[i]), out[2n + i] = the hardware's approximate
// reciprocal it starts from.
__global__ void k_math_selftest(const double* __restrict__ x, double* __restrict__ out, int64_t n) {
  __shared__ double tab[32];
  if (threadIdx.x < 32) tab[threadIdx.x] = kExp2Frac[threadIdx.x];
  __syncthreads();
  const ExpTable ex{tab};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    double r0;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(v));
    out[i] = ex(v);
    out[n + i] = rcp64(v);
    out[2 * n + i] = r0;
  }
}

}  // namespace

int chem_step_fast(const HydroParams& P, void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
                   cudaStream_t st, bool expand) {
  const int64_t want = (n + kChemThreads - 1) / kChemThreads, cap = (int64_t)148 * kChemMinBlocks * 4;
  const int blocks = (int)(want < cap ? (want < 1 ? 1 : want) : cap);
  if (f32)
    k_chem_fast<float, kChemMinBlocks>
        <<<blocks, kChemThreads, 0, st>>>((float*)q, n, nf, species, P, ctl, &ctl->err, expand);
  else
    k_chem_fast<double, kChemMinBlocks>
        <<<blocks, kChemThreads, 0, st>>>((double*)q, n, nf, species, P, ctl, &ctl->err, expand);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "chem");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

}  // namespace evora

extern "C" int evora_selftest_exp(const double* x, double* out, int64_t n) {
  if (!x || !out || n < 0) return EVORA_ERR_ARG;
  if (n == 0) return 0;
  double *dx = nullptr, *dy = nullptr;
  cudaError_t e = cudaMalloc(&dx, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dy, 3 * sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    evora::k_math_selftest<<<148 * 4, 256>>>(dx, dy, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dy, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dy);
  if (e != cudaSuccess) {
    evora::set_cuda_error(e, "evora_selftest_exp");
    return EVORA_ERR_CUDA;
  }
  return 0;
}
