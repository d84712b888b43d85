// Orbitals on a grid of points (the reference's evaluation script,
// shelled_eval.py:88-131): AO values, then (after the MO GEMM the host does
// with the library GEMM) per-orbital densities.
//
// k_grid_ao: one thread per point, all shells of the molecule in order (the
// shell table is read as warp-uniform broadcasts).  Like the reference, the
// point comes in FP32 and everything after the centre difference is FP64:
//   ao[a][g] = x^i y^j z^k * sum_p cn_p exp(-alpha_p r^2) * g(i, j, k)
// with cn_p = contraction coefficient x radial norm and g the component's
// 1/sqrt(prod (2 l_i - 1)!!) (1 for s and p); shells up to f, a generally
// contracted shell arriving as one shell per contraction row.  Rows are AOs,
// columns points, so the stores of a warp are contiguous.
//
// k_grid_density: psi_a, psi_b are the MO values (rows = orbitals); for
// orbital k < n_mo and point g
//   total[k][g] = [k < n_a] psi_a^2 + [k < n_b] psi_b^2   (FP64, stored FP32)
//   phase[k][g] = psi_a                                     (k < n_a only)
#pragma once

#include "common.cuh"
#include "hl.cuh"

__global__ void __launch_bounds__(128) k_grid_ao(const dftk_shells_t sh, long long n, const float *pts, double *ao,
                                                 long long ld)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double x = (double)pts[3 * g], y = (double)pts[3 * g + 1], z = (double)pts[3 * g + 2];
    for (int s = 0; s < sh.n_shells; ++s) {
        const double dx = x - __ldg(sh.xyz + 3 * s), dy = y - __ldg(sh.xyz + 3 * s + 1),
                     dz = z - __ldg(sh.xyz + 3 * s + 2);
        // the reference's sum of squares, without contraction into FMAs
        const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        const int p0 = __ldg(sh.prim_off + s), np = __ldg(sh.nprim + s);
        double rad = 0.0;
        for (int p = 0; p < np; ++p) rad += __ldg(sh.prim_cn + p0 + p) * exp(-__ldg(sh.prim_exp + p0 + p) * r2);
        const int l = __ldg(sh.l + s);
        double *row = ao + (long long)__ldg(sh.ao + s) * ld + g;
        if (l == 0) {
            row[0] = rad;
        } else if (l == 1) {
            row[0] = dx * rad;
            row[ld] = dy * rad;
            row[2 * ld] = dz * rad;
        } else if (l <= HL_LMAX) {
            const int nc = hl_ncomp(l);
            for (int k = 0; k < nc; ++k) {
                double v = 1.0;
                for (int i = 0; i < hl_pow(l, k, 0); ++i) v *= dx;
                for (int i = 0; i < hl_pow(l, k, 1); ++i) v *= dy;
                for (int i = 0; i < hl_pow(l, k, 2); ++i) v *= dz;
                row[(long long)k * ld] = v * rad * c_hl_cnorm[l][k];
            }
        }
        // momenta beyond f are rejected by the host before launch
    }
}

// GRID_DENSITY_UNROLL points per thread, blockDim apart (coalesced), so each
// thread has that many independent loads in flight
#define GRID_DENSITY_UNROLL 4

__global__ void __launch_bounds__(256) k_grid_density(int n_a, int n_b, long long n, const double *psi_a,
                                                      const double *psi_b, long long ld_psi, float *total,
                                                      float *phase, long long ld_out)
{
    const int k = blockIdx.y;
    const long long g0 = (long long)blockIdx.x * blockDim.x * GRID_DENSITY_UNROLL + threadIdx.x;
    const double *ra = psi_a + (long long)k * ld_psi;
    const double *rb = psi_b + (long long)k * ld_psi;
    const bool same = psi_b == psi_a;  // closed shells pass one matrix twice: read it once
    double pa[GRID_DENSITY_UNROLL], pb[GRID_DENSITY_UNROLL];
#pragma unroll
    for (int j = 0; j < GRID_DENSITY_UNROLL; ++j) {
        const long long g = g0 + (long long)j * blockDim.x;
        pa[j] = g < n ? ra[g] : 0.0;
        pb[j] = g < n ? (same ? pa[j] : rb[g]) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < GRID_DENSITY_UNROLL; ++j) {
        const long long g = g0 + (long long)j * blockDim.x;
        if (g >= n) break;
        const double da = k < n_a ? pa[j] * pa[j] : 0.0, db = k < n_b ? pb[j] * pb[j] : 0.0;
        total[(long long)k * ld_out + g] = (float)(da + db);
        if (k < n_a) phase[(long long)k * ld_out + g] = (float)pa[j];
    }
}
