// Boys function F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt on the device.
//
// Method (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978), sec. 4;
// the tabulated-Taylor scheme used by most MD codes):
//   T < 50: F_L(T) = sum_{j=0}^{7} F_{L+j}(T_k) (T_k - T)^j / j!  around the
//           nearest grid point T_k = k / 10 (|T_k - T| <= 0.05, truncation
//           < 2e-15 relative).  The table stores, per order L, the eight
//           coefficients F_{L+j}(T_k) / j! of one grid point contiguously, so
//           the polynomial is a plain FMA Horner chain fed by 128-bit loads
//           (order 0: two 256-bit loads, measured 4 % faster on (ss|ss); the
//           other orders measured slower with them).
//           exp(-T) = exp(-T_k) exp(T_k - T) with a 7-term Taylor series,
//           then the downward recursion F_m = (2T F_{m+1} + exp(-T)) / (2m+1),
//           which is stable.
//   T >= 50: F_0 = sqrt(pi / T) / 2 (erfc(7) < 5e-23) and the upward
//           recursion F_{m+1} = (2m + 1) F_m / (2T); the exp(-T) < 2e-22 term
//           it drops changes F_m by < 2e-14 relative for m <= 7.
// Tables (internal linkage: each device module of the library -- dftk.cu and
// the hlc_part_*.cu units -- holds its own copy, filled by dftk_init):
// orders L = 0..12, grid points T_k = 0, 0.1, ..., 50, computed on the
// host in long double from the all-positive series
// F_m(T) = exp(-T) sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)).
// Orders >= 1 in FP64 read a half-step table instead (T_k = k / 20, so
// |T_k - T| <= 0.025): seven coefficients F_{L+j}(T_k) / j! and exp(-T_k) in
// one 64-byte row, two 256-bit loads and no separate exp table load; the
// seven-term series truncate below 1e-16 relative (measured 1-4 % faster on
// the p classes than the full-step rows).
// FP32 uses the same scheme with the first five coefficients of a float table
// built at the float grid points, and a 5-term exp series; slot 5 of each
// 32-byte FP32 row holds exp(-T_k), so one 256-bit load serves both.
#pragma once

#include "common.cuh"

#define DFTK_BOYS_ROWS 501
#define DFTK_BOYS_NL 13        // orders 0..12 ((ff|ff) quartets)
#define DFTK_BOYS_W 8          // coefficients per grid point
#define DFTK_BOYS_TMAX 50.0

static __device__ __align__(128) double g_boys64[DFTK_BOYS_NL * DFTK_BOYS_ROWS * DFTK_BOYS_W];
static __device__ double g_bexp64[DFTK_BOYS_ROWS];
#ifndef DFTK_BOYS_HALFSTEP
#define DFTK_BOYS_HALFSTEP 1
#endif
#define DFTK_BOYS_HROWS 1001   // half-step grid T_k = k / 20, k = 0..1000
// half-step rows (orders >= 1): F_{L+j}(T_k) / j!, j = 0..6, then exp(-T_k)
static __device__ __align__(128) double g_boys64h[DFTK_BOYS_NL * DFTK_BOYS_HROWS * DFTK_BOYS_W];
static __device__ __align__(128) float g_boys32[DFTK_BOYS_NL * DFTK_BOYS_ROWS * DFTK_BOYS_W];
static __device__ float g_bexp32[DFTK_BOYS_ROWS];

// 32-byte read-only vector loads (sm_100: ld.global.nc.v4.f64 / .v8.f32);
// the address must be 32-byte aligned (table rows are)
__device__ __forceinline__ void ldg_v4d(const double *p, double &a, double &b, double &c, double &d)
{
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void ldg_v8f(const float *p, float (&v)[8])
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
}

// One packed core record of a primitive pair (P x/y/z, p, K, q, 1/(2p), 0):
// 64 bytes in FP64 (two 256-bit loads), 32 bytes in FP32 (one).
__device__ __forceinline__ void core_ld(const double *p, double &a, double &b, double &c, double &d, double &e,
                                        double &f, double &g, double &h)
{
    ldg_v4d(p, a, b, c, d);
    ldg_v4d(p + 4, e, f, g, h);
}
__device__ __forceinline__ void core_ld(const float *p, float &a, float &b, float &c, float &d, float &e, float &f,
                                        float &g, float &h)
{
    float v[8];
    ldg_v8f(p, v);
    a = v[0]; b = v[1]; c = v[2]; d = v[3]; e = v[4]; f = v[5]; g = v[6]; h = v[7];
}

template <typename T, int L> struct Boys;

template <int L> struct Boys<double, L> {
    static_assert(L < DFTK_BOYS_NL, "Boys order beyond the table");
    __device__ __forceinline__ static void eval(double x, double *F)
    {
        if (DFTK_BOYS_HALFSTEP && L > 0 && x < DFTK_BOYS_TMAX) {
            // one 64-byte row: seven Taylor coefficients of F_L and exp(-T_k)
            const double shifted = fma(x, 20.0, DFTK_ROUND_MAGIC64);  // x >= 0
            const int k = __double2loint(shifted);
            const double d = (shifted - DFTK_ROUND_MAGIC64) * 0.05 - x;
            const double *rowp = g_boys64h + ((size_t)L * DFTK_BOYS_HROWS + k) * DFTK_BOYS_W;
            double c0, c1, c2, c3, c4, c5, c6, ek;
            ldg_v4d(rowp, c0, c1, c2, c3);
            ldg_v4d(rowp + 4, c4, c5, c6, ek);
            double f = fma(c6, d, c5);
            f = fma(f, d, c4);
            f = fma(f, d, c3);
            f = fma(f, d, c2);
            f = fma(f, d, c1);
            F[L] = fma(f, d, c0);
            double e = fma(d, 1.0 / 5040.0, 1.0 / 720.0);
            e = fma(e, d, 1.0 / 120.0);
            e = fma(e, d, 1.0 / 24.0);
            e = fma(e, d, 1.0 / 6.0);
            e = fma(e, d, 0.5);
            e = fma(e, d, 1.0);
            e = fma(e, d, 1.0);
            e *= ek;
            const double x2 = x + x;
#pragma unroll
            for (int m = L - 1; m >= 0; --m) F[m] = fma(x2, F[m + 1], e) * (1.0 / (2 * m + 1));
        } else if (x < DFTK_BOYS_TMAX) {
            const double shifted = fma(x, 10.0, DFTK_ROUND_MAGIC64);  // x >= 0
            const int k = __double2loint(shifted);
            const double d = (shifted - DFTK_ROUND_MAGIC64) * 0.1 - x;
            const double *rowp = g_boys64 + ((size_t)L * DFTK_BOYS_ROWS + k) * DFTK_BOYS_W;
            double c0, c1, c2, c3, c4, c5, c6, c7;
            if constexpr (L == 0) {
                // (ss|ss): two 256-bit loads per row (measured faster for this
                // order only; the higher orders keep 128-bit loads)
                ldg_v4d(rowp, c0, c1, c2, c3);
                ldg_v4d(rowp + 4, c4, c5, c6, c7);
            } else {
                const double2 *row = reinterpret_cast<const double2 *>(rowp);
                const double2 c01 = __ldg(row), c23 = __ldg(row + 1), c45 = __ldg(row + 2), c67 = __ldg(row + 3);
                c0 = c01.x; c1 = c01.y; c2 = c23.x; c3 = c23.y; c4 = c45.x; c5 = c45.y; c6 = c67.x; c7 = c67.y;
            }
            double f = fma(c7, d, c6);
            f = fma(f, d, c5);
            f = fma(f, d, c4);
            f = fma(f, d, c3);
            f = fma(f, d, c2);
            f = fma(f, d, c1);
            F[L] = fma(f, d, c0);
            if (L > 0) {
                double e = fma(d, 1.0 / 5040.0, 1.0 / 720.0);
                e = fma(e, d, 1.0 / 120.0);
                e = fma(e, d, 1.0 / 24.0);
                e = fma(e, d, 1.0 / 6.0);
                e = fma(e, d, 0.5);
                e = fma(e, d, 1.0);
                e = fma(e, d, 1.0);
                e *= __ldg(g_bexp64 + k);
                const double x2 = x + x;
#pragma unroll
                for (int m = L - 1; m >= 0; --m) F[m] = fma(x2, F[m + 1], e) * (1.0 / (2 * m + 1));
            }
        } else {
            const double rs = Math<double>::rsqrt(x);
            F[0] = 0.88622692545275801365 * rs;
            const double h = 0.5 * rs * rs;
#pragma unroll
            for (int m = 0; m < L; ++m) F[m + 1] = ((double)(2 * m + 1) * h) * F[m];
        }
    }
};

template <int L> struct Boys<float, L> {
    static_assert(L < DFTK_BOYS_NL, "Boys order beyond the table");
    __device__ __forceinline__ static void eval(float x, float *F)
    {
        if (x < (float)DFTK_BOYS_TMAX) {
            const float shifted = fmaf(x, 10.0f, DFTK_ROUND_MAGIC32);  // x >= 0
            const int k = __float_as_int(shifted) - 0x4B400000;
            const float d = (shifted - DFTK_ROUND_MAGIC32) * 0.1f - x;
            float c[8];
            ldg_v8f(g_boys32 + ((size_t)L * DFTK_BOYS_ROWS + k) * DFTK_BOYS_W, c);
            float f = fmaf(c[4], d, c[3]);
            f = fmaf(f, d, c[2]);
            f = fmaf(f, d, c[1]);
            F[L] = fmaf(f, d, c[0]);
            if (L > 0) {
                float e = fmaf(d, 1.0f / 24.0f, 1.0f / 6.0f);
                e = fmaf(e, d, 0.5f);
                e = fmaf(e, d, 1.0f);
                e = fmaf(e, d, 1.0f);
                e *= c[5];  // exp(-T_k)
                const float x2 = x + x;
#pragma unroll
                for (int m = L - 1; m >= 0; --m) F[m] = fmaf(x2, F[m + 1], e) * (1.0f / (2 * m + 1));
            }
        } else {
            const float rs = ::rsqrtf(x);
            F[0] = 0.886226925f * rs;
            const float h = 0.5f * rs * rs;
#pragma unroll
            for (int m = 0; m < L; ++m) F[m + 1] = ((float)(2 * m + 1) * h) * F[m];
        }
    }
};

// Runtime-order Boys (orders 0..8) for the generic drop-in kernels and the
// one-electron kernel: same scheme and tables, order chosen at run time.
__device__ __forceinline__ void boys_runtime(int L, double x, double *F)
{
    if (x < DFTK_BOYS_TMAX) {
        const int k = max(__double2int_rn(x * 10.0), 0);
        const double d = (double)k * 0.1 - x;
        const double *row = g_boys64 + ((size_t)L * DFTK_BOYS_ROWS + k) * DFTK_BOYS_W;
        double f = __ldg(row + 7);
        for (int j = 6; j >= 0; --j) f = fma(f, d, __ldg(row + j));
        F[L] = f;
        double e = 1.0;
        for (int j = 7; j >= 1; --j) e = fma(d / j, e, 1.0);
        e *= __ldg(g_bexp64 + k);
        for (int m = L - 1; m >= 0; --m) F[m] = (2.0 * x * F[m + 1] + e) / (2 * m + 1);
    } else {
        const double rs = ::rsqrt(x);
        F[0] = 0.88622692545275801365 * rs;
        const double h = 0.5 * rs * rs;
        for (int m = 0; m < L; ++m) F[m + 1] = (2 * m + 1) * h * F[m];
    }
}
