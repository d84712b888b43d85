// Shared definitions for libdftk (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dftk.h"

#define DFTK_PI 3.14159265358979323846
#define DFTK_FULL_MASK 0xffffffffu

// sqrt(2 pi^{5/2}): split evenly between the bra and ket pair prefactors so
// that (bra K)(ket K) rsqrt(p+q) = 2 pi^{5/2} / (p q sqrt(p+q)) K_AB K_CD.
#define DFTK_SQRT_2PI52 5.9149671727956128778

// Field indices of a primitive-pair record (see dftk_pairs_t).
enum { F_PX = 0, F_PY, F_PZ, F_P, F_K, F_H, F_AX, F_AY, F_AZ, F_BX, F_BY, F_BZ };

// The molecule a shell belongs to (the single molecule when sh.mol is NULL):
// offset and AO count of its matrix blocks, its first shell and shell count,
// and the offset of its shell-block (n_s x n_s) arrays.
struct MolView {
    long long mat;
    int nao;
    int s0;
    int ns;
    long long dsh;
};

__device__ __forceinline__ MolView mol_view(const dftk_shells_t &sh, int s)
{
    MolView v;
    if (sh.mol == nullptr) {
        v.mat = 0;
        v.nao = sh.n_ao;
        v.s0 = 0;
        v.ns = sh.n_shells;
        v.dsh = 0;
        return v;
    }
    const int m = __ldg(sh.mol + s);
    v.mat = __ldg(sh.mol_mat + m);
    v.nao = __ldg(sh.mol_nao + m);
    v.s0 = __ldg(sh.mol_shell0 + m);
    v.ns = __ldg(sh.mol_ns + m);
    v.dsh = __ldg(sh.mol_dsh + m);
    return v;
}

// max |D| over the six shell blocks of the quartet (ab|cd) from the
// shell-block maxima Dsh (all four shells lie in one molecule)
__device__ __forceinline__ float quartet_dmax(const dftk_shells_t &sh, const float *Dsh, int a, int b, int c, int d)
{
    const MolView v = mol_view(sh, a);
    const float *B = Dsh + v.dsh;
    const int ns = v.ns;
    const int la = a - v.s0, lb = b - v.s0, lc = c - v.s0, ld = d - v.s0;
    return fmaxf(fmaxf(__ldg(B + la * ns + lb), __ldg(B + lc * ns + ld)),
                 fmaxf(fmaxf(__ldg(B + la * ns + lc), __ldg(B + la * ns + ld)),
                       fmaxf(__ldg(B + lb * ns + lc), __ldg(B + lb * ns + ld))));
}

// Element counts of the N x N matrices and of the shell-block arrays.
inline long long shells_mat_elems(const dftk_shells_t &sh)
{
    return sh.mol ? sh.mat_elems : (long long)sh.n_ao * sh.n_ao;
}
inline long long shells_dsh_elems(const dftk_shells_t &sh)
{
    return sh.mol ? sh.dsh_elems : (long long)sh.n_shells * sh.n_shells;
}
inline int shells_n_mol(const dftk_shells_t &sh) { return sh.mol ? sh.n_mol : 1; }

// Stored fields per pair class: the ERI fields (ss 5, ps 9, pp 12) plus the
// bra-side exponent alpha last (read only by the gradient kernels).
__host__ __device__ constexpr int pair_fields(int pc) { return pc == 0 ? 6 : (pc == 1 ? 10 : 13); }
__host__ __device__ constexpr int pair_alpha_field(int pc) { return pair_fields(pc) - 1; }

// Inverse square root for the positive, normal, float-range arguments of the
// integral kernels (p + q, and T beyond the Boys table): an FP32 estimate
// refined by two Newton-Raphson steps r <- r (3 - x r^2) / 2, each of which
// squares the relative error (2^-22 -> 2^-43 -> below double rounding).  No
// special-case branches, unlike a general-purpose rsqrt.
template <typename T> struct Math;
template <> struct Math<double> {
    __device__ __forceinline__ static double rsqrt(double x)
    {
        double r = (double)::rsqrtf((float)x);
        const double h = 0.5 * x;
        r = r * fma(-h * r, r, 1.5);
        r = r * fma(-h * r, r, 1.5);
        return r;
    }
};
template <> struct Math<float> {
    __device__ __forceinline__ static float rsqrt(float x) { return ::rsqrtf(x); }
};

// Round-to-nearest of 0 <= v < 2^31 by adding 1.5 * 2^52: the sum's low
// mantissa bits hold the integer, and subtracting the constant again gives it
// as a double, so the table index needs no double<->int conversion.
#define DFTK_ROUND_MAGIC64 6755399441055744.0
#define DFTK_ROUND_MAGIC32 12582912.0f  // 1.5 * 2^23, bit pattern 0x4B400000

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(DFTK_FULL_MASK, v, o);
    return v;
}
