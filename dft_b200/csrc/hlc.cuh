// Thread-per-quartet J/K kernels of the classes (ds|ss), (ds|ps), (ds|pp),
// (dp|ss), (dp|ps), (dp|pp): the generated straight-line bodies of
// hl_classes.cuh (gen_hl.py) over candidate spaces indexed through the d
// path's pair sets (class rows of the hi set, class kets of the lo set), and
// the s/p digestion (digest_block).  One warp takes 32 consecutive
// candidates of one class (and one split of the ket components), as the s/p
// scan kernel does; the quartets of a row are consecutive, so the bra pair is
// usually warp-uniform.
#pragma once

#include "hl.cuh"
#include "hl_classes.cuh"

struct HlcParams {
    dftk_shells_t sh;
    const int *shell_ao;
    dftk_pairs_t hi, lo;
    const int *rows[2];
    long long n_rows[2];
    const int *kets[3];
    const long long *off[HLC_N_CLASSES];
    long long total[HLC_N_CLASSES];
    float tau_prim;
    const double *D, *Da, *Db;
    double *Y, *Za, *Zb;
    const float *Dsh;
    int uhf;
    double tau;
    long long *counts;  // [2]: quartets evaluated, primitive quartets (NULL = not counted)
};

template <int C, int S>
__device__ __forceinline__ void hlc_one(const HlcParams &P, bool valid, int row, int ket)
{
    using E = HlClass<double, C, S>;
    const int lead = __ffs(__ballot_sync(DFTK_FULL_MASK, valid)) - 1;
    const int row0 = __shfl_sync(DFTK_FULL_MASK, row, lead < 0 ? 0 : lead);
    const bool uniform = __all_sync(DFTK_FULL_MASK, !valid || row == row0);
    const int brow = valid ? row : row0;
    const int a = P.hi.ab[2 * brow], b = P.hi.ab[2 * brow + 1];
    const int c = valid ? P.lo.ab[2 * ket] : 0, d = valid ? P.lo.ab[2 * ket + 1] : 0;
    double I[E::NI];
    int evaluated = 0;
    if (valid) {
        evaluated = E::run(P.hi.rec64, P.hi.qp, P.hi.n_pairs, P.hi.kmax, row, P.hi.nprim[row], P.lo.rec64, P.lo.qp,
                           P.lo.n_pairs, P.lo.kmax, ket, P.lo.nprim[ket], P.tau_prim, I);
    } else {
#pragma unroll
        for (int q = 0; q < E::NI; ++q) I[q] = 0.0;
    }
    // a hi pair never equals a lo pair, and a != b (different momenta)
    const int ew = c == d;
    digest_block<E>(P, valid, uniform, a, b, c, d, (double)(1 << ew), I);
    if (P.counts) {
        // each split evaluates the same primitive quartets: count split 0
        int tot = S == 0 ? evaluated : 0;
        int nq = (S == 0 && valid) ? 1 : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tot += __shfl_xor_sync(DFTK_FULL_MASK, tot, o);
            nq += __shfl_xor_sync(DFTK_FULL_MASK, nq, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (nq) atomicAdd((unsigned long long *)P.counts, (unsigned long long)nq);
            if (tot) atomicAdd((unsigned long long *)(P.counts + 1), (unsigned long long)tot);
        }
    }
}

template <int C, int S>
__device__ __forceinline__ void hlc_split(const HlcParams &P, int split, bool valid, int row, int ket)
{
    if (split == S) {
        hlc_one<C, S>(P, valid, row, ket);
    } else if constexpr (S + 1 < HlClass<double, C, 0>::NSPLIT) {
        hlc_split<C, S + 1>(P, split, valid, row, ket);
    }
}

template <int C>
__global__ void __launch_bounds__(128) k_hlc(const HlcParams P)
{
    using E0 = HlClass<double, C, 0>;
    constexpr int NS = E0::NSPLIT;
    constexpr int X = E0::BRA_L, Yc = E0::KET_CLASS;
    const long long ncand = P.total[C];
    const long long nwork = ((ncand + 31) >> 5) * NS;
    const int lane = threadIdx.x & 31;
    const long long wstride = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gw < nwork; gw += wstride) {
        const int split = (int)(gw % NS);
        const long long cand = (gw / NS) * 32 + lane;
        bool valid = cand < ncand;
        int row = 0, ket = 0;
        if (valid) {
            const int r = find_row(P.off[C], P.n_rows[X], cand);
            row = __ldg(P.rows[X] + r);
            ket = __ldg(P.kets[Yc] + (cand - __ldg(P.off[C] + r)));
            const int a = P.hi.ab[2 * row], b = P.hi.ab[2 * row + 1];
            const int c = P.lo.ab[2 * ket], d = P.lo.ab[2 * ket + 1];
            const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
            valid = __ldg(P.hi.q + row) * __ldg(P.lo.q + ket) * (double)dm >= P.tau;
        }
        if (!__any_sync(DFTK_FULL_MASK, valid)) continue;
        hlc_split<C, 0>(P, split, valid, row, ket);
    }
}
