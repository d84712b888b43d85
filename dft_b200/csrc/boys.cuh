// Boys function F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt on the device.
//
// Method (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978), sec. 4;
// the tabulated-Taylor scheme used by most MD codes):
//   T < 36: F_L(T) = sum_{j=0}^{6} F_{L+j}(T_k) (T_k - T)^j / j!  around the
//           nearest grid point T_k = k / 10 (|T_k - T| <= 0.05, truncation
//           ~1e-15 relative), exp(-T) = exp(-T_k) exp(T_k - T) with a 7-term
//           Taylor series, then the downward recursion
//           F_m = (2T F_{m+1} + exp(-T)) / (2m + 1), which is stable.
//   T >= 36: F_0 = sqrt(pi / T) / 2 (erfc(6) < 2e-17), upward recursion
//           F_{m+1} = ((2m + 1) F_m - exp(-T)) / (2T), stable for T > m.
// The table holds F_0..F_14 and exp(-T_k) for T_k = 0, 0.1, ..., 36; it is
// computed on the host in long double from the all-positive series
// F_m(T) = exp(-T) sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)).
// FP32 uses the same scheme with 5 Taylor terms and a float table built at
// the float grid points.
#pragma once

#include "common.cuh"

#define DFTK_BOYS_ROWS 361
#define DFTK_BOYS_COLS 16
#define DFTK_BOYS_EXPCOL 15
#define DFTK_BOYS_TMAX 36.0

__device__ double g_boys64[DFTK_BOYS_ROWS * DFTK_BOYS_COLS];
__device__ float g_boys32[DFTK_BOYS_ROWS * DFTK_BOYS_COLS];

template <typename T, int L> struct Boys;

template <int L> struct Boys<double, L> {
    static_assert(L + 6 < DFTK_BOYS_EXPCOL, "Boys table too narrow");
    __device__ __forceinline__ static void eval(double x, double *F)
    {
        if (x < DFTK_BOYS_TMAX) {
            const int k = __double2int_rn(x * 10.0);
            const double d = (double)k * 0.1 - x;
            const double *row = g_boys64 + k * DFTK_BOYS_COLS;
            double f = __ldg(row + L + 6);
            f = fma(f, d * (1.0 / 6.0), __ldg(row + L + 5));
            f = fma(f, d * 0.2, __ldg(row + L + 4));
            f = fma(f, d * 0.25, __ldg(row + L + 3));
            f = fma(f, d * (1.0 / 3.0), __ldg(row + L + 2));
            f = fma(f, d * 0.5, __ldg(row + L + 1));
            f = fma(f, d, __ldg(row + L));
            F[L] = f;
            if (L > 0) {
                double e = fma(d, 1.0 / 7.0, 1.0);
                e = fma(d * (1.0 / 6.0), e, 1.0);
                e = fma(d * 0.2, e, 1.0);
                e = fma(d * 0.25, e, 1.0);
                e = fma(d * (1.0 / 3.0), e, 1.0);
                e = fma(d * 0.5, e, 1.0);
                e = fma(d, e, 1.0);
                e *= __ldg(row + DFTK_BOYS_EXPCOL);
                const double x2 = x + x;
#pragma unroll
                for (int m = L - 1; m >= 0; --m) F[m] = fma(x2, F[m + 1], e) * (1.0 / (2 * m + 1));
            }
        } else {
            const double rs = ::rsqrt(x);
            F[0] = 0.88622692545275801365 * rs;
            if (L > 0) {
                const double e = ::exp(-x);
                const double h = 0.5 * rs * rs;
#pragma unroll
                for (int m = 0; m < L; ++m) F[m + 1] = fma((double)(2 * m + 1), F[m], -e) * h;
            }
        }
    }
};

template <int L> struct Boys<float, L> {
    static_assert(L + 4 < DFTK_BOYS_EXPCOL, "Boys table too narrow");
    __device__ __forceinline__ static void eval(float x, float *F)
    {
        if (x < (float)DFTK_BOYS_TMAX) {
            const int k = __float2int_rn(x * 10.0f);
            const float d = (float)k * 0.1f - x;
            const float *row = g_boys32 + k * DFTK_BOYS_COLS;
            float f = __ldg(row + L + 4);
            f = fmaf(f, d * 0.25f, __ldg(row + L + 3));
            f = fmaf(f, d * (1.0f / 3.0f), __ldg(row + L + 2));
            f = fmaf(f, d * 0.5f, __ldg(row + L + 1));
            f = fmaf(f, d, __ldg(row + L));
            F[L] = f;
            if (L > 0) {
                float e = fmaf(d, 0.25f, 1.0f);
                e = fmaf(d * (1.0f / 3.0f), e, 1.0f);
                e = fmaf(d * 0.5f, e, 1.0f);
                e = fmaf(d, e, 1.0f);
                e *= __ldg(row + DFTK_BOYS_EXPCOL);
                const float x2 = x + x;
#pragma unroll
                for (int m = L - 1; m >= 0; --m) F[m] = fmaf(x2, F[m + 1], e) * (1.0f / (2 * m + 1));
            }
        } else {
            const float rs = ::rsqrtf(x);
            F[0] = 0.886226925f * rs;
            if (L > 0) {
                const float e = __expf(-x);
                const float h = 0.5f * rs * rs;
#pragma unroll
                for (int m = 0; m < L; ++m) F[m + 1] = fmaf((float)(2 * m + 1), F[m], -e) * h;
            }
        }
    }
};

// Runtime-order Boys (orders up to 14) for the generic drop-in kernels and the
// one-electron kernel: same scheme, loop instead of unrolled code.
__device__ __forceinline__ void boys_runtime(int L, double x, double *F)
{
    if (x < DFTK_BOYS_TMAX) {
        const int k = __double2int_rn(x * 10.0);
        const double d = (double)k * 0.1 - x;
        const double *row = g_boys64 + k * DFTK_BOYS_COLS;
        const int top = L + 6 < DFTK_BOYS_EXPCOL ? 6 : DFTK_BOYS_EXPCOL - 1 - L;
        double f = __ldg(row + L + top);
        for (int j = top; j >= 1; --j) f = fma(f, d / j, __ldg(row + L + j - 1));
        F[L] = f;
        double e = 1.0;
        for (int j = 7; j >= 1; --j) e = fma(d / j, e, 1.0);
        e *= __ldg(row + DFTK_BOYS_EXPCOL);
        for (int m = L - 1; m >= 0; --m) F[m] = (2.0 * x * F[m + 1] + e) / (2 * m + 1);
    } else {
        const double rs = ::rsqrt(x);
        F[0] = 0.88622692545275801365 * rs;
        const double e = ::exp(-x);
        const double h = 0.5 * rs * rs;
        for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
    }
}
