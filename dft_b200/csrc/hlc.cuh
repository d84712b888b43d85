// Thread-per-quartet J/K kernels of the fifteen d classes without an f shell
// ((ds|ss) .. (dd|dd), hl_classes.cuh, written by gen_hl.py at build time):
// candidate spaces indexed through the d path's pair sets (the hi rows of one
// pair kind as bras; the lo rows of one kind, or the hi rows of one kind, as
// kets, grouped by primitive-count bucket), and the s/p digestion generalised
// to threads that hold a chunk of bra and of ket components.  One warp takes
// 32 consecutive candidates of one class and component chunk, as the s/p scan
// kernel does; the quartets of a (row, bucket) segment are consecutive, so
// the bra pair is usually warp-uniform.  The kernels are instantiated in the
// hlc_part_*.cu units (hlc_part.cuh), one kernel per chunk.
//
// Pair kinds: 0 ss, 1 ps, 2 pp (lo set), 3 ds, 4 dp, 5 dd (hi set); pairs
// with an f shell have no kind and stay with the warp-per-quartet kernel.
#pragma once

#include "hl.cuh"
#include "hl_classes.cuh"

#define HLC_N_KINDS 6

struct HlcParams {
    dftk_shells_t sh;
    const int *shell_ao;
    dftk_pairs_t hi, lo;
    const int *rows[3];  // hi rows of kinds ds, dp, dd (bras, Schwarz order)
    long long n_rows[3];
    const int *kets[HLC_N_KINDS];  // rows of each kind grouped by primitive-count bucket
    long long seg[HLC_N_KINDS][DFTK_HLC_NB + 1];
    const long long *off[HLC_N_CLASSES];  // over (bra position, bucket)
    long long total[HLC_N_CLASSES];
    float tau_prim;
    const double *D, *Da, *Db;
    double *Y, *Za, *Zb;
    const float *Dsh;
    int uhf;
    double tau;
    long long *counts;  // [2]: quartets evaluated, primitive quartets (NULL = not counted)
};

// whether a thread's chunk of class E holds bra component ia (a) / ib (b)
template <typename E>
__device__ __forceinline__ constexpr bool chunk_has_a(int ia)
{
    for (int n = 0; n < E::NAB; ++n)
        if (E::ab_a(n) == ia) return true;
    return false;
}
template <typename E>
__device__ __forceinline__ constexpr bool chunk_has_b(int ib)
{
    for (int n = 0; n < E::NAB; ++n)
        if (E::ab_b(n) == ib) return true;
    return false;
}

// Digest a chunk I[n NCD + m] (bra components ab_a/ab_b(n), ket components
// cd_c/cd_d(m)) into Y and Z with the identities of digest_block; each
// thread adds its chunk's partial sums.
template <typename E>
__device__ __forceinline__ void hlc_digest(const HlcParams &P, bool valid, bool uniform_bra, int a, int b, int c,
                                           int d, double w, const double (&I)[E::NI])
{
    constexpr int NA = E::NA, NB = E::NB, NC = E::NC, ND = E::ND, NAB = E::NAB, NCD = E::NCD;
    const MolView mv = mol_view(P.sh, a);
    const int N = mv.nao;
    const int oa = P.shell_ao[a], ob = P.shell_ao[b], oc = P.shell_ao[c], od = P.shell_ao[d];
    const double fJ = valid ? 2.0 / w : 0.0;
    const double fK = valid ? 1.0 / w : 0.0;
    double v[E::NI];
#pragma unroll
    for (int q = 0; q < E::NI; ++q) v[q] = valid ? I[q] : 0.0;
    const double *D = P.D + mv.mat;
    double *Yb = P.Y + mv.mat;
    // Y_cd
#pragma unroll
    for (int m = 0; m < NCD; ++m) {
        double s = 0.0;
#pragma unroll
        for (int n = 0; n < NAB; ++n)
            s = fma(v[n * NCD + m], __ldg(D + (long long)(oa + E::ab_a(n)) * N + ob + E::ab_b(n)), s);
        if (valid) atomicAdd(Yb + (long long)(oc + E::cd_c(m)) * N + od + E::cd_d(m), fJ * s);
    }
    // Y_ab
#pragma unroll
    for (int n = 0; n < NAB; ++n) {
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < NCD; ++m)
            s = fma(v[n * NCD + m], __ldg(D + (long long)(oc + E::cd_c(m)) * N + od + E::cd_d(m)), s);
        s *= fJ;
        if (uniform_bra) {
            s = warp_sum(s);
            if ((threadIdx.x & 31) == 0) atomicAdd(Yb + (long long)(oa + E::ab_a(n)) * N + ob + E::ab_b(n), s);
        } else if (valid) {
            atomicAdd(Yb + (long long)(oa + E::ab_a(n)) * N + ob + E::ab_b(n), s);
        }
    }
    for (int spin = 0; spin < (P.uhf ? 2 : 1); ++spin) {
        const double *Ds = (spin ? P.Db : P.Da) + mv.mat;
        double *Z = (spin ? P.Zb : P.Za) + mv.mat;
        double zac[NA][NC], zad[NA][ND], zbc[NB][NC], zbd[NB][ND];
#pragma unroll
        for (int i = 0; i < NA; ++i) {
#pragma unroll
            for (int j = 0; j < NC; ++j) zac[i][j] = 0.0;
#pragma unroll
            for (int j = 0; j < ND; ++j) zad[i][j] = 0.0;
        }
#pragma unroll
        for (int i = 0; i < NB; ++i) {
#pragma unroll
            for (int j = 0; j < NC; ++j) zbc[i][j] = 0.0;
#pragma unroll
            for (int j = 0; j < ND; ++j) zbd[i][j] = 0.0;
        }
#pragma unroll
        for (int n = 0; n < NAB; ++n)
#pragma unroll
            for (int m = 0; m < NCD; ++m) {
                const int ia = E::ab_a(n), ib = E::ab_b(n), cc = E::cd_c(m), dd = E::cd_d(m);
                const double val = v[n * NCD + m] * fK;
                zac[ia][cc] = fma(val, __ldg(Ds + (long long)(ob + ib) * N + od + dd), zac[ia][cc]);
                zad[ia][dd] = fma(val, __ldg(Ds + (long long)(ob + ib) * N + oc + cc), zad[ia][dd]);
                zbc[ib][cc] = fma(val, __ldg(Ds + (long long)(oa + ia) * N + od + dd), zbc[ib][cc]);
                zbd[ib][dd] = fma(val, __ldg(Ds + (long long)(oa + ia) * N + oc + cc), zbd[ib][dd]);
            }
        if (valid) {
#pragma unroll
            for (int ia = 0; ia < NA; ++ia) {
                if (!chunk_has_a<E>(ia)) continue;
#pragma unroll
                for (int cc = 0; cc < NC; ++cc)
                    if (split_has_c<E>(cc)) atomicAdd(Z + (long long)(oa + ia) * N + oc + cc, zac[ia][cc]);
#pragma unroll
                for (int dd = 0; dd < ND; ++dd)
                    if (split_has_d<E>(dd)) atomicAdd(Z + (long long)(oa + ia) * N + od + dd, zad[ia][dd]);
            }
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) {
                if (!chunk_has_b<E>(ib)) continue;
#pragma unroll
                for (int cc = 0; cc < NC; ++cc)
                    if (split_has_c<E>(cc)) atomicAdd(Z + (long long)(ob + ib) * N + oc + cc, zbc[ib][cc]);
#pragma unroll
                for (int dd = 0; dd < ND; ++dd)
                    if (split_has_d<E>(dd)) atomicAdd(Z + (long long)(ob + ib) * N + od + dd, zbd[ib][dd]);
            }
        }
    }
}

template <int C, int S>
__device__ __forceinline__ void hlc_one(const HlcParams &P, bool valid, int row, int ket)
{
    using E = HlClass<double, C, S>;
    constexpr bool KET_HI = E::KET_KIND >= 3;
    const dftk_pairs_t &K = KET_HI ? P.hi : P.lo;
    const int lead = __ffs(__ballot_sync(DFTK_FULL_MASK, valid)) - 1;
    const int row0 = __shfl_sync(DFTK_FULL_MASK, row, lead < 0 ? 0 : lead);
    const bool uniform = __all_sync(DFTK_FULL_MASK, !valid || row == row0);
    const int brow = valid ? row : row0;
    const int a = P.hi.ab[2 * brow], b = P.hi.ab[2 * brow + 1];
    const int c = valid ? K.ab[2 * ket] : 0, d = valid ? K.ab[2 * ket + 1] : 0;
    double I[E::NI];
    int evaluated = 0;
    if (valid) {
        evaluated = E::run(P.hi.rec64, P.hi.qp, P.hi.n_pairs, P.hi.kmax, row, P.hi.nprim[row], K.rec64, K.qp,
                           K.n_pairs, K.kmax, ket, K.nprim[ket], P.tau_prim, I);
    } else {
#pragma unroll
        for (int q = 0; q < E::NI; ++q) I[q] = 0.0;
    }
    const int ew = (a == b) + (c == d) + ((E::BRA_KIND == E::KET_KIND) && row == ket);
    hlc_digest<E>(P, valid, uniform, a, b, c, d, (double)(1 << ew), I);
    if (P.counts) {
        // every chunk evaluates the same primitive quartets: count chunk 0
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

// resident 128-thread blocks per SM the class kernels are compiled for
// (register cap 65536 / (128 x value))
#ifndef DFTK_HLC_MINB
#define DFTK_HLC_MINB 1
#endif

// One component chunk S of class C over every candidate: one kernel per
// chunk, so an SM holds a single straight-line body in its instruction cache
// (measured on B200, (dp|pp) with nine chunks: instruction-fetch stalls of
// 37 cycles per issue with the chunks interleaved in one kernel).
template <int C, int S>
__global__ void __launch_bounds__(128, DFTK_HLC_MINB) k_hlc(const HlcParams P)
{
    using E0 = HlClass<double, C, 0>;
    constexpr int X = E0::BRA_KIND - 3, Yk = E0::KET_KIND;
    constexpr bool KET_HI = Yk >= 3;
    const dftk_pairs_t &K = KET_HI ? P.hi : P.lo;
    const int *kets = P.kets[Yk];
    const long long ncand = P.total[C];
    const long long nwork = (ncand + 31) >> 5;
    const int lane = threadIdx.x & 31;
    const long long wstride = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gw < nwork; gw += wstride) {
        const long long cand = gw * 32 + lane;
        bool valid = cand < ncand;
        int row = 0, ket = 0;
        if (valid) {
            const int rb = find_row(P.off[C], P.n_rows[X] * DFTK_HLC_NB, cand);
            row = __ldg(P.rows[X] + rb / DFTK_HLC_NB);
            ket = __ldg(kets + P.seg[Yk][rb % DFTK_HLC_NB] + (cand - __ldg(P.off[C] + rb)));
            const int a = P.hi.ab[2 * row], b = P.hi.ab[2 * row + 1];
            const int c = K.ab[2 * ket], d = K.ab[2 * ket + 1];
            const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
            valid = __ldg(P.hi.q + row) * __ldg(K.q + ket) * (double)dm >= P.tau;
        }
        if (!__any_sync(DFTK_FULL_MASK, valid)) continue;
        hlc_one<C, S>(P, valid, row, ket);
    }
}
