// Loop-based McMurchie-Davidson pieces for runtime angular momenta: used by
// the one-electron kernel and by the drop-in replacements of the reference's
// nuclear_kernel / eri_kernel.  The s/p ERI hot path uses the generated
// straight-line code in eri_classes.cuh instead.
#pragma once

#include "boys.cuh"
#include "common.cuh"

#define DFTK_E_SLOTS 7     // Hermite slots per axis in the reference layout (max_e)
#define DFTK_GENERIC_LMAX 8

// 1-D Hermite coefficients E^{la,lb}_t, t = 0..la+lb, with the factor
// exp(-mu X_AB^2) in E^{00}_0; a raised first, then b (shelled.py:228-294).
__device__ __forceinline__ void herm_E1d(double al, double be, double A, double B, int la, int lb,
                                         double *E)
{
    const double p = al + be;
    const double X = A - B;
    const double PA = -be * X / p, PB = al * X / p, h = 0.5 / p;
    double cur[16], nxt[16];
    for (int t = 0; t < 16; ++t) cur[t] = 0.0;
    cur[0] = exp(-al * be / p * X * X);
    int order = 0;
    for (int step = 0; step < la + lb; ++step) {
        const double sh = step < la ? PA : PB;
        for (int t = 0; t <= order + 1; ++t) {
            double v = 0.0;
            if (t <= order) v = sh * cur[t];
            if (t > 0) v = fma(h, cur[t - 1], v);
            if (t + 1 <= order) v = fma((double)(t + 1), cur[t + 1], v);
            nxt[t] = v;
        }
        ++order;
        for (int t = 0; t <= order; ++t) cur[t] = nxt[t];
    }
    for (int t = 0; t <= la + lb; ++t) E[t] = cur[t];
}

// R^{(0)}_{tuv}(alpha, X, Y, Z) for t + u + v <= L <= LM, dense cube index
// (t * (LM + 1) + u) * (LM + 1) + v, computed level by level from n = L down.
template <int LM>
__device__ __forceinline__ void herm_R(int L, double alpha, double X, double Y, double Z, double *R)
{
    constexpr int D = LM + 1;
    double F[LM + 1];
    boys_runtime(L, alpha * (X * X + Y * Y + Z * Z), F);
    double prev[D * D * D];
    for (int i = 0; i < D * D * D; ++i) prev[i] = 0.0;  // entries beyond order L read as zero
    double scale[LM + 1];
    scale[0] = 1.0;
    for (int n = 1; n <= L; ++n) scale[n] = scale[n - 1] * (-2.0 * alpha);
    prev[0] = scale[L] * F[L];
    for (int n = L - 1; n >= 0; --n) {
        const int top = L - n;
        // fill in decreasing t+u+v so the level-(n+1) values are read before overwrite
        for (int s = top; s >= 1; --s)
            for (int t = s; t >= 0; --t)
                for (int u = s - t; u >= 0; --u) {
                    const int v = s - t - u;
                    double r;
                    if (t > 0) {
                        r = X * prev[((t - 1) * D + u) * D + v];
                        if (t > 1) r = fma((double)(t - 1), prev[((t - 2) * D + u) * D + v], r);
                    } else if (u > 0) {
                        r = Y * prev[(t * D + u - 1) * D + v];
                        if (u > 1) r = fma((double)(u - 1), prev[(t * D + u - 2) * D + v], r);
                    } else {
                        r = Z * prev[(t * D + u) * D + v - 1];
                        if (v > 1) r = fma((double)(v - 1), prev[(t * D + u) * D + v - 2], r);
                    }
                    prev[(t * D + u) * D + v] = r;
                }
        prev[0] = scale[n] * F[n];
    }
    for (int i = 0; i < D * D * D; ++i) R[i] = prev[i];
}
