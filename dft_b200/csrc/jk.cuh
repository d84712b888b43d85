// Pair data, Schwarz factors, integral-direct J/K and ERI-block kernels.
#pragma once

#include "boys.cuh"
#include "common.cuh"
#include "eri_classes.cuh"

// Packed core record of primitive slot (k * n_pairs + pair): P, p, K, the
// primitive Schwarz factor and 1/(2p) in both precisions.
__device__ __forceinline__ void write_core(const dftk_pairs_t &pr, long long slot, double Px, double Py, double Pz,
                                           double p, double K, float qp)
{
    const double v[8] = {Px, Py, Pz, p, K, (double)qp, p > 0.0 ? 0.5 / p : 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        pr.core64[slot * 8 + i] = v[i];
        pr.core32[slot * 8 + i] = (float)v[i];
    }
}

// ----------------------------------------------------------------- pair data
// One thread per (primitive slot k, pair); pair index fastest so the SoA
// record writes are coalesced.  Replaces the per-pair nuclear_kernel launch
// and pair_cache dict (shelled.py:1000-1059) for the ERI path.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_pair_data(const dftk_shells_t sh, const dftk_pairs_t pr, int nfields)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = pr.n_pairs;
    if (t >= (long long)n * pr.kmax) return;
    const int pair = (int)(t % n);
    const int k = (int)(t / n);
    const int a = pr.ab[2 * pair], b = pr.ab[2 * pair + 1];
    const int na = sh.nprim[a], nb = sh.nprim[b];
    if (k == 0) pr.nprim[pair] = na * nb;
    double f[13];
#pragma unroll
    for (int i = 0; i < 13; ++i) f[i] = 0.0;
    if (k < na * nb) {
        const int ia = k / nb, ib = k % nb;
        const double al = sh.prim_exp[sh.prim_off[a] + ia];
        const double be = sh.prim_exp[sh.prim_off[b] + ib];
        const double ca = sh.prim_cn[sh.prim_off[a] + ia];
        const double cb = sh.prim_cn[sh.prim_off[b] + ib];
        const double Ax = sh.xyz[3 * a], Ay = sh.xyz[3 * a + 1], Az = sh.xyz[3 * a + 2];
        const double Bx = sh.xyz[3 * b], By = sh.xyz[3 * b + 1], Bz = sh.xyz[3 * b + 2];
        const double p = al + be;
        const double ip = 1.0 / p;
        const double Px = (al * Ax + be * Bx) * ip;
        const double Py = (al * Ay + be * By) * ip;
        const double Pz = (al * Az + be * Bz) * ip;
        const double ab2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
        f[F_PX] = Px; f[F_PY] = Py; f[F_PZ] = Pz; f[F_P] = p;
        f[F_K] = DFTK_SQRT_2PI52 * ca * cb * exp(-al * be * ip * ab2) * ip;
        f[F_H] = 0.5 * ip;
        f[F_AX] = Px - Ax; f[F_AY] = Py - Ay; f[F_AZ] = Pz - Az;
        f[F_BX] = Px - Bx; f[F_BY] = Py - By; f[F_BZ] = Pz - Bz;
        f[nfields - 1] = al;  // overwrites nothing the class reads (alpha field is last)
    }
    for (int i = 0; i < nfields; ++i) {
        const long long o = ((long long)i * pr.kmax + k) * n + pair;
        pr.rec64[o] = f[i];
        pr.rec32[o] = (float)f[i];
    }
    if (pr.core64) write_core(pr, (long long)k * n + pair, f[F_PX], f[F_PY], f[F_PZ], f[F_P], f[F_K], 0.0f);
}
#endif

// ------------------------------------------------------------------ helpers
template <int C, typename T, int S>
__device__ __forceinline__ int eri_run(const T *bra, const T *bra_core, const float *bra_q, int bra_n_pairs,
                                       int bra_kmax, int bra_row, int bra_np, const T *ket, const T *ket_core,
                                       const float *ket_q, int ket_n_pairs, int ket_kmax, int ket_row, int ket_np,
                                       float eps, T (&I)[EriClass<T, C, S>::NI])
{
    return EriClass<T, C, S>::run(bra, bra_core, bra_q, bra_n_pairs, bra_kmax, bra_row, bra_np, ket, ket_core, ket_q,
                                  ket_n_pairs, ket_kmax, ket_row, ket_np, eps, I);
}

// Diagonal class of a pair class: ss -> (ss|ss), ps -> (ps|ps), pp -> (pp|pp).
template <int PC> struct DiagClass { static constexpr int C = PC == 0 ? 0 : (PC == 1 ? 2 : 5); };

// max |(ab|ab)| over components, primitives k0 .. k0 + np - 1 of the pair
template <int C, int S>
__device__ __forceinline__ double diag_max(const dftk_pairs_t &pr, int pair, int k0, int np)
{
    double I[EriClass<double, C, S>::NI];
    const double *rec = pr.rec64 + (long long)k0 * pr.n_pairs;
    const double *core = pr.core64 + 8LL * k0 * pr.n_pairs;
    const float *q = pr.qp + (long long)k0 * pr.n_pairs;
    eri_run<C, double, S>(rec, core, q, pr.n_pairs, pr.kmax, pair, np, rec, core, q, pr.n_pairs, pr.kmax, pair, np,
                          0.0f, I);
    double m = 0.0;
#pragma unroll
    for (int q2 = 0; q2 < EriClass<double, C, S>::NI; ++q2) m = fmax(m, fabs(I[q2]));
    return m;
}

template <int C>
__device__ __forceinline__ double diag_max_all(const dftk_pairs_t &pr, int pair, int k0, int np)
{
    double m = diag_max<C, 0>(pr, pair, k0, np);
    if constexpr (EriClass<double, C, 0>::NSPLIT > 1) {
        m = fmax(m, diag_max<C, 1>(pr, pair, k0, np));
        m = fmax(m, diag_max<C, 2>(pr, pair, k0, np));
    }
    return m;
}

#define DFTK_MAX_KPAIR 128

// Schwarz factors, one thread per pair: Q_ab = sqrt(max |(ab|ab)|) of the
// contracted pair, and per primitive pair q_k = sqrt(max |(ab_k|ab_k)|); the
// primitive records of the pair are then reordered by descending q_k (both
// copies) so the ERI loops can stop at the first negligible primitive.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
template <int PC>
static __global__ void k_schwarz(const dftk_pairs_t pr, int nfields)
{
    const int pair = blockIdx.x * blockDim.x + threadIdx.x;
    if (pair >= pr.n_pairs) return;
    constexpr int C = DiagClass<PC>::C;
    const int np = pr.nprim[pair];
    const long long n = pr.n_pairs;
    for (int k = 0; k < pr.kmax; ++k) pr.qp[k * n + pair] = 0.0f;  // no screening while measuring
    pr.q[pair] = sqrt(diag_max_all<C>(pr, pair, 0, np));
    float qk[DFTK_MAX_KPAIR];
    int order[DFTK_MAX_KPAIR];
    const int kk = min(pr.kmax, DFTK_MAX_KPAIR);
    for (int k = 0; k < kk; ++k) {
        qk[k] = k < np ? (float)sqrt(diag_max_all<C>(pr, pair, k, 1)) : 0.0f;
        order[k] = k;
    }
    // insertion sort, descending q (kmax <= DFTK_MAX_KPAIR)
    for (int a = 1; a < kk; ++a) {
        const int o = order[a];
        int b = a - 1;
        while (b >= 0 && qk[order[b]] < qk[o]) { order[b + 1] = order[b]; --b; }
        order[b + 1] = o;
    }
    for (int f = 0; f < nfields; ++f) {
        double v64[DFTK_MAX_KPAIR];
        float v32[DFTK_MAX_KPAIR];
        for (int k = 0; k < kk; ++k) {
            v64[k] = pr.rec64[((long long)f * pr.kmax + k) * n + pair];
            v32[k] = pr.rec32[((long long)f * pr.kmax + k) * n + pair];
        }
        for (int k = 0; k < kk; ++k) {
            pr.rec64[((long long)f * pr.kmax + k) * n + pair] = v64[order[k]];
            pr.rec32[((long long)f * pr.kmax + k) * n + pair] = v32[order[k]];
        }
    }
    for (int k = 0; k < kk; ++k) pr.qp[k * n + pair] = qk[order[k]];
    if (pr.core64)
        for (int k = 0; k < kk; ++k) {
            const long long o = (long long)k * n + pair;
            write_core(pr, o, pr.rec64[o], pr.rec64[(long long)pr.kmax * n + o], pr.rec64[2LL * pr.kmax * n + o],
                       pr.rec64[3LL * pr.kmax * n + o], pr.rec64[4LL * pr.kmax * n + o], qk[order[k]]);
        }
}
#endif

// ------------------------------------------------------------------- J / K
struct JkParams {
    dftk_shells_t sh;  // shells (and molecule table of a batch)
    const int *shell_ao;
    const int *ab[3];
    const int *np[3];
    const double *rec64[3];
    const float *rec32[3];
    const double *core64[3];
    const float *core32[3];
    const double *q[3];
    const float *qp[3];
    int n_pairs[3];
    int kmax[3];
    float tau_prim;
    long long n_rows[DFTK_N_QCLASS];
    long long total[DFTK_N_QCLASS];
    const long long *row_off[DFTK_N_QCLASS];
    const double *D, *Da, *Db;
    double *Y, *Za, *Zb;
    const float *Dsh;
    int uhf;
    double tau_lo, tau_hi;  // scan path: quartet processed if tau_lo <= bound < tau_hi
    double tau, tau32;      // select path: FP64 if bound >= tau32, FP32 if tau <= bound < tau32
    int dm_pow2;            // select path: bound Q_ab Q_cd max|D|^2 (gradients) instead of max|D|
    int bucket;             // select path: group survivors by the ket's primitive-count bucket
    long long *counts;
    // select path: per class one list of (bra row, ket) with capacity total[C];
    // FP64 entries fill it from the front, FP32 entries from the back
    int2 *list[DFTK_N_QCLASS];
    unsigned long long *heads;  // [2 * DFTK_N_QCLASS]: FP64 then FP32 entry counts
    const int *ket_base[DFTK_N_QCLASS];  // batches: first ket pair of each row's molecule (NULL = 0)
    const unsigned char *mol_active;     // batches: molecules still iterating (NULL = all)
    int tile[2 * DFTK_N_QCLASS];         // list kernels: consecutive work items per warp step (FP64, FP32)
};

// ket pair of candidate `cand` in bra row `row` of class C
template <int C>
__device__ __forceinline__ int cand_ket(const JkParams &P, int row, long long cand)
{
    const int k = (int)(cand - __ldg(P.row_off[C] + row));
    return P.ket_base[C] ? k + __ldg(P.ket_base[C] + row) : k;
}

// whether the molecule of shell a still takes part (per-molecule convergence)
__device__ __forceinline__ bool mol_is_active(const JkParams &P, int a)
{
    return P.mol_active == nullptr || P.sh.mol == nullptr || __ldg(P.mol_active + __ldg(P.sh.mol + a)) != 0;
}

// largest r in [0, n_rows) with off[r] <= cand
__device__ __forceinline__ int find_row(const long long *off, long long n_rows, long long cand)
{
    long long lo = 0, hi = n_rows - 1;
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= cand) lo = mid; else hi = mid - 1;
    }
    return (int)lo;
}

// Shell-block maxima of |D| (and |D_a|, |D_b| for UHF): Dsh[dsh + x * ns + y]
// per molecule (x, y molecule-local shells).  Thread t = (x global, y local),
// y < max_ns.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_dsh(const dftk_shells_t sh, int max_ns, const double *D, const double *Da, const double *Db,
                      int uhf, float *Dsh)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)sh.n_shells * max_ns) return;
    const int x = (int)(t / max_ns), yl = (int)(t % max_ns);
    const MolView v = mol_view(sh, x);
    if (yl >= v.ns) return;
    const int y = v.s0 + yl;
    const int ox = sh.ao[x], oy = sh.ao[y];
    const int nx = (sh.l[x] + 1) * (sh.l[x] + 2) / 2, ny = (sh.l[y] + 1) * (sh.l[y] + 2) / 2;
    const int N = v.nao;
    double m = 0.0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const long long o = v.mat + (long long)(ox + i) * N + oy + j;
            m = fmax(m, fabs(D[o]));
            m = fmax(m, fabs(Da[o]));
            if (uhf) m = fmax(m, fabs(Db[o]));
        }
    Dsh[v.dsh + (long long)(x - v.s0) * v.ns + yl] = (float)m;
}
#endif

// Digest one contracted block into the half-accumulators Y (J) and Z (K):
//   Y_ab += 2/w sum_cd I D_cd,  Y_cd += 2/w sum_ab I D_ab,
//   Z_ac += 1/w sum_bd I D_bd,  Z_ad += 1/w sum_bc I D_bc,
//   Z_bc += 1/w sum_ad I D_ad,  Z_bd += 1/w sum_ac I D_ac,
// w = 2^{[a=b]+[c=d]+[ab=cd]}; J = Y + Y^T and K = Z + Z^T afterwards give the
// eight orientations of fill_matrices (shelled.py:791-859) with its weights.
// Whether a thread's share of the ket components (one split of class E)
// holds ket component cc (c) or dd (d).
template <typename E>
__device__ __forceinline__ constexpr bool split_has_c(int cc)
{
    for (int m = 0; m < E::NCD; ++m)
        if (E::cd_c(m) == cc) return true;
    return false;
}
template <typename E>
__device__ __forceinline__ constexpr bool split_has_d(int dd)
{
    for (int m = 0; m < E::NCD; ++m)
        if (E::cd_d(m) == dd) return true;
    return false;
}

// The digestion of one block of class E (EriClass or HlClass: NA..ND, NCD,
// cd_c, cd_d); PT holds sh, shell_ao, D, Da, Db, Y, Za, Zb and uhf.
template <typename E, typename PT, typename T>
__device__ __forceinline__ void digest_block(const PT &P, bool valid, bool uniform_bra, int a, int b, int c, int d,
                                             double w, const T (&I)[E::NI])
{
    constexpr int NA = E::NA, NB = E::NB, NC = E::NC, ND = E::ND, NCD = E::NCD;
    const MolView mv = mol_view(P.sh, a);
    const int N = mv.nao;
    const int oa = P.shell_ao[a], ob = P.shell_ao[b], oc = P.shell_ao[c], od = P.shell_ao[d];
    const double fJ = valid ? 2.0 / w : 0.0;
    const double fK = valid ? 1.0 / w : 0.0;
    double v[E::NI];
#pragma unroll
    for (int q = 0; q < E::NI; ++q) v[q] = valid ? (double)I[q] : 0.0;
    const double *D = P.D + mv.mat;
    double *Yb = P.Y + mv.mat;
    // Y_cd
#pragma unroll
    for (int m = 0; m < NCD; ++m) {
        double s = 0.0;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
                s = fma(v[(ia * NB + ib) * NCD + m], __ldg(D + (long long)(oa + ia) * N + ob + ib), s);
        if (valid) atomicAdd(Yb + (long long)(oc + E::cd_c(m)) * N + od + E::cd_d(m), fJ * s);
    }
    // Y_ab
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < NCD; ++m)
                s = fma(v[(ia * NB + ib) * NCD + m],
                        __ldg(D + (long long)(oc + E::cd_c(m)) * N + od + E::cd_d(m)), s);
            s *= fJ;
            if (uniform_bra) {
                s = warp_sum(s);
                if ((threadIdx.x & 31) == 0) atomicAdd(Yb + (long long)(oa + ia) * N + ob + ib, s);
            } else if (valid) {
                atomicAdd(Yb + (long long)(oa + ia) * N + ob + ib, s);
            }
        }
    // K, one or two spins
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
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int ib = 0; ib < NB; ++ib)
#pragma unroll
                for (int m = 0; m < NCD; ++m) {
                    const int cc = E::cd_c(m), dd = E::cd_d(m);
                    const double val = v[(ia * NB + ib) * NCD + m] * fK;
                    zac[ia][cc] = fma(val, __ldg(Ds + (long long)(ob + ib) * N + od + dd), zac[ia][cc]);
                    zad[ia][dd] = fma(val, __ldg(Ds + (long long)(ob + ib) * N + oc + cc), zad[ia][dd]);
                    zbc[ib][cc] = fma(val, __ldg(Ds + (long long)(oa + ia) * N + od + dd), zbc[ib][cc]);
                    zbd[ib][dd] = fma(val, __ldg(Ds + (long long)(oa + ia) * N + oc + cc), zbd[ib][dd]);
                }
        if (valid) {
#pragma unroll
            for (int ia = 0; ia < NA; ++ia) {
#pragma unroll
                for (int cc = 0; cc < NC; ++cc)
                    if (split_has_c<E>(cc)) atomicAdd(Z + (long long)(oa + ia) * N + oc + cc, zac[ia][cc]);
#pragma unroll
                for (int dd = 0; dd < ND; ++dd)
                    if (split_has_d<E>(dd)) atomicAdd(Z + (long long)(oa + ia) * N + od + dd, zad[ia][dd]);
            }
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) {
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

template <int C, typename T, int S>
__device__ __forceinline__ void digest(const JkParams &P, bool valid, bool uniform_bra, int a, int b,
                                       int c, int d, double w, const T (&I)[EriClass<T, C, S>::NI])
{
    digest_block<EriClass<T, C, S>>(P, valid, uniform_bra, a, b, c, d, w, I);
}

template <int C, typename T> struct RecOf;
template <int C> struct RecOf<C, double> {
    __device__ static const double *get(const JkParams &P, int pc) { return P.rec64[pc]; }
    __device__ static const double *core(const JkParams &P, int pc) { return P.core64[pc]; }
};
template <int C> struct RecOf<C, float> {
    __device__ static const float *get(const JkParams &P, int pc) { return P.rec32[pc]; }
    __device__ static const float *core(const JkParams &P, int pc) { return P.core32[pc]; }
};

template <int C, typename T, int S>
__device__ __forceinline__ void jk_one(const JkParams &P, bool valid, int row, int ket)
{
    using E = EriClass<T, C, S>;
    constexpr int X = E::BRA_CLASS, Yc = E::KET_CLASS;
    const int *abX = P.ab[X];
    const int *abY = P.ab[Yc];
    // warp-uniform bra pair lets the Y_ab reduction happen in registers; the
    // caller guarantees at least one valid lane
    const int lead = __ffs(__ballot_sync(DFTK_FULL_MASK, valid)) - 1;
    const int row0 = __shfl_sync(DFTK_FULL_MASK, row, lead < 0 ? 0 : lead);
    const bool uniform = __all_sync(DFTK_FULL_MASK, !valid || row == row0);
    // screened-out lanes take the bra shells of the warp's lead row: lane 0
    // writes the reduced Y_ab block with its own a, b even when it is invalid
    const int brow = valid ? row : row0;
    const int a = abX[2 * brow], b = abX[2 * brow + 1];
    const int c = valid ? abY[2 * ket] : 0, d = valid ? abY[2 * ket + 1] : 0;
    T I[E::NI];
    int evaluated = 0;
    if (valid) {
        // FP32 quartets (bound Q_ab Q_cd max|D| < tau_fp32): also skip the
        // primitive quartets whose qp product is below 2^-20 Q_ab Q_cd, i.e.
        // whose share of the quartet is below a few FP32 roundings; with the
        // bound below tau_fp32 that is < 1e-12 absolute per quartet
        float eps = P.tau_prim;
        if constexpr (sizeof(T) == 4)
            eps = fmaxf(eps, 9.5367431640625e-7f * (float)(__ldg(P.q[X] + row) * __ldg(P.q[Yc] + ket)));
        evaluated = eri_run<C, T, S>(RecOf<C, T>::get(P, X), RecOf<C, T>::core(P, X), P.qp[X], P.n_pairs[X],
                                     P.kmax[X], row, P.np[X][row], RecOf<C, T>::get(P, Yc),
                                     RecOf<C, T>::core(P, Yc), P.qp[Yc], P.n_pairs[Yc], P.kmax[Yc], ket,
                                     P.np[Yc][ket], eps, I);
    } else {
#pragma unroll
        for (int q = 0; q < E::NI; ++q) I[q] = T(0);
    }
    const int ew = (a == b) + (c == d) + ((X == Yc) && (row == ket));
    digest<C, T, S>(P, valid, uniform, a, b, c, d, (double)(1 << ew), I);
    if (P.counts) {
        // evaluated primitive quartets: slot 12 + class (the FP32 launch's
        // counts pointer is offset by 6)
        int tot = evaluated;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(DFTK_FULL_MASK, tot, o);
        if ((threadIdx.x & 31) == 0 && tot)
            atomicAdd((unsigned long long *)(P.counts + 2 * DFTK_N_QCLASS + C), (unsigned long long)tot);
    }
}

// One warp per 32 consecutive candidates of class C (and one split of the
// c components for the split classes); quartets whose density-weighted
// Schwarz bound falls outside [tau_lo, tau_hi) are skipped.
template <int C, typename T>
__global__ void __launch_bounds__(128) k_jk(const JkParams P)
{
    using E0 = EriClass<T, C, 0>;
    constexpr int NS = E0::NSPLIT;
    constexpr int X = E0::BRA_CLASS, Yc = E0::KET_CLASS;
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
            row = find_row(P.row_off[C], P.n_rows[C], cand);
            ket = cand_ket<C>(P, row, cand);
            const int a = P.ab[X][2 * row], b = P.ab[X][2 * row + 1];
            const int c = P.ab[Yc][2 * ket], d = P.ab[Yc][2 * ket + 1];
            const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
            const double bound = __ldg(P.q[X] + row) * __ldg(P.q[Yc] + ket) * (double)dm * (P.dm_pow2 ? (double)dm : 1.0);
            valid = bound >= P.tau_lo && bound < P.tau_hi && mol_is_active(P, a);
        }
        if (P.counts && split == 0) {
            const unsigned bal = __ballot_sync(DFTK_FULL_MASK, valid);
            if (lane == 0 && bal) atomicAdd((unsigned long long *)(P.counts + C), (unsigned long long)__popc(bal));
        }
        if (!__any_sync(DFTK_FULL_MASK, valid)) continue;
        if constexpr (NS == 1) {
            jk_one<C, T, 0>(P, valid, row, ket);
        } else {
            if (split == 0) jk_one<C, T, 0>(P, valid, row, ket);
            else if (split == 1) jk_one<C, T, 1>(P, valid, row, ket);
            else jk_one<C, T, 2>(P, valid, row, ket);
        }
    }
}

// Selection pass: one scan of class C's candidate space computes each
// quartet's density-weighted Schwarz bound and appends the survivors to the
// FP64 or FP32 end of the class list.  A block compacts a tile of
// SELECT_TILE consecutive candidates with a block-wide prefix sum and
// reserves its output range with one atomic, so the lists keep the candidate
// order within every tile: the class kernels then see long runs of one bra
// row with neighbouring kets (shared bra data, warp-uniform J reduction).
#define SELECT_THREADS 256
#define SELECT_PER_WARP 8
#define SELECT_TILE (SELECT_THREADS * SELECT_PER_WARP)

template <int C>
__device__ __forceinline__ void select_classify(const JkParams &P, long long cand, int &row, int &ket, bool &is64,
                                                bool &is32, int r0)
{
    using E0 = EriClass<double, C, 0>;
    constexpr int X = E0::BRA_CLASS, Yc = E0::KET_CLASS;
    const long long *off = P.row_off[C];
    row = r0;
    if (cand >= __ldg(off + r0 + 1)) row = find_row(off, P.n_rows[C], cand);
    ket = cand_ket<C>(P, row, cand);
    const int a = P.ab[X][2 * row], b = P.ab[X][2 * row + 1];
    const int c = P.ab[Yc][2 * ket], d = P.ab[Yc][2 * ket + 1];
    const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
    const double bound = __ldg(P.q[X] + row) * __ldg(P.q[Yc] + ket) * (double)dm * (P.dm_pow2 ? (double)dm : 1.0);
    const bool active = mol_is_active(P, a);
    is64 = active && bound >= P.tau32;
    is32 = active && !is64 && bound >= P.tau;
}

// One tile of class C's candidates (the block's SELECT_TILE consecutive
// candidates starting at tile * SELECT_TILE), with P.bucket set: within the
// tile the survivors are grouped by the ket pair's primitive-pair-count
// bucket (select_bucket:
// nprim <= 1, 4, 9, 16, 36, more), candidate order kept inside a bucket, so
// the 32 lanes of a class-kernel warp loop over similar primitive counts
// (generally contracted bases mix 1- and 81-primitive pairs; with one
// primitive count, as in STO-3G, the order is the candidate order).
#define SELECT_NB 6
__device__ __forceinline__ int select_bucket(int nprim)
{
    return nprim <= 1 ? 0 : nprim <= 4 ? 1 : nprim <= 9 ? 2 : nprim <= 16 ? 3 : nprim <= 36 ? 4 : 5;
}

template <int C>
__device__ __forceinline__ void select_tile_bucketed(const JkParams &P, long long tile, unsigned (*s_cnt)[2 * SELECT_NB],
                                            unsigned long long &s_base64, unsigned long long &s_base32)
{
    using E0 = EriClass<double, C, 0>;
    constexpr int Yc = E0::KET_CLASS;
    const long long ncand = P.total[C];
    const long long cap = ncand;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const long long *off = P.row_off[C];
    {
        const long long wfirst = tile * SELECT_TILE + (long long)warp * 32 * SELECT_PER_WARP;
        int r0 = 0;
        if (lane == 0 && wfirst < ncand) r0 = find_row(off, P.n_rows[C], wfirst);
        r0 = __shfl_sync(DFTK_FULL_MASK, r0, 0);
        if (lane < 2 * SELECT_NB) s_cnt[warp][lane] = 0;
        __syncwarp();
        int rows[SELECT_PER_WARP], kets[SELECT_PER_WARP], keys[SELECT_PER_WARP];
        unsigned pos[SELECT_PER_WARP];
#pragma unroll
        for (int it = 0; it < SELECT_PER_WARP; ++it) {
            const long long cand = wfirst + it * 32 + lane;
            bool is64 = false, is32 = false;
            rows[it] = 0;
            kets[it] = 0;
            if (cand < ncand) {
                select_classify<C>(P, cand, rows[it], kets[it], is64, is32, r0);
                r0 = rows[it];  // later candidates of this lane lie at or beyond this row
            }
            // key = bucket x 2 + precision for a survivor (bucket 0 when the
            // caller passes no primitive counts), -1 for a dropped candidate
            int key = -1;
            if (is64 || is32) key = 2 * (P.np[Yc] ? select_bucket(__ldg(P.np[Yc] + kets[it])) : 0) + (is32 ? 1 : 0);
            const unsigned same = __match_any_sync(DFTK_FULL_MASK, key);
            pos[it] = key >= 0 ? s_cnt[warp][key] + __popc(same & below) : 0u;
            __syncwarp();
            if (key >= 0 && (same & below) == 0) s_cnt[warp][key] += __popc(same);
            __syncwarp();
            keys[it] = key;
            r0 = __shfl_sync(DFTK_FULL_MASK, r0, 0);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // exclusive offsets in (precision, bucket, warp) order
            unsigned t[2] = {0u, 0u};
            for (int key = 0; key < 2 * SELECT_NB; ++key)
                for (int w = 0; w < SELECT_THREADS / 32; ++w) {
                    const unsigned n = s_cnt[w][key];
                    s_cnt[w][key] = t[key & 1];
                    t[key & 1] += n;
                }
            s_base64 = t[0] ? atomicAdd(P.heads + C, (unsigned long long)t[0]) : 0ull;
            s_base32 = t[1] ? atomicAdd(P.heads + DFTK_N_QCLASS + C, (unsigned long long)t[1]) : 0ull;
            if (P.counts) {
                if (t[0]) atomicAdd((unsigned long long *)(P.counts + C), (unsigned long long)t[0]);
                if (t[1]) atomicAdd((unsigned long long *)(P.counts + DFTK_N_QCLASS + C), (unsigned long long)t[1]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < SELECT_PER_WARP; ++it) {
            const int key = keys[it];
            if (key < 0) continue;
            const unsigned long long p = s_cnt[warp][key] + pos[it];
            if ((key & 1) == 0) P.list[C][s_base64 + p] = make_int2(rows[it], kets[it]);
            else P.list[C][cap - 1 - (long long)(s_base32 + p)] = make_int2(rows[it], kets[it]);
        }
        __syncthreads();  // s_base/s_cnt are rewritten by the next tile
    }
}

// The same in candidate order (P.bucket == 0): per warp and precision one
// ballot-compacted run.
template <int C>
__device__ __forceinline__ void select_tile_plain(const JkParams &P, long long tile, unsigned (*s_cnt)[2 * SELECT_NB],
                                                  unsigned long long &s_base64, unsigned long long &s_base32)
{
    const long long ncand = P.total[C];
    const long long cap = ncand;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const long long *off = P.row_off[C];
    const long long wfirst = tile * SELECT_TILE + (long long)warp * 32 * SELECT_PER_WARP;
    int r0 = 0;
    if (lane == 0 && wfirst < ncand) r0 = find_row(off, P.n_rows[C], wfirst);
    r0 = __shfl_sync(DFTK_FULL_MASK, r0, 0);
    unsigned m64[SELECT_PER_WARP], m32[SELECT_PER_WARP];
    int rows[SELECT_PER_WARP], kets[SELECT_PER_WARP];
    unsigned n64 = 0, n32 = 0;
#pragma unroll
    for (int it = 0; it < SELECT_PER_WARP; ++it) {
        const long long cand = wfirst + it * 32 + lane;
        bool is64 = false, is32 = false;
        rows[it] = 0;
        kets[it] = 0;
        if (cand < ncand) {
            select_classify<C>(P, cand, rows[it], kets[it], is64, is32, r0);
            r0 = rows[it];  // later candidates of this lane lie at or beyond this row
        }
        m64[it] = __ballot_sync(DFTK_FULL_MASK, is64);
        m32[it] = __ballot_sync(DFTK_FULL_MASK, is32);
        n64 += __popc(m64[it]);
        n32 += __popc(m32[it]);
        r0 = __shfl_sync(DFTK_FULL_MASK, r0, 0);
    }
    if (lane == 0) {
        s_cnt[warp][0] = n64;
        s_cnt[warp][1] = n32;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t64 = 0, t32 = 0;
        for (int w = 0; w < SELECT_THREADS / 32; ++w) {
            const unsigned a = s_cnt[w][0], b = s_cnt[w][1];
            s_cnt[w][0] = t64;
            s_cnt[w][1] = t32;
            t64 += a;
            t32 += b;
        }
        s_base64 = t64 ? atomicAdd(P.heads + C, (unsigned long long)t64) : 0ull;
        s_base32 = t32 ? atomicAdd(P.heads + DFTK_N_QCLASS + C, (unsigned long long)t32) : 0ull;
        if (P.counts) {
            if (t64) atomicAdd((unsigned long long *)(P.counts + C), (unsigned long long)t64);
            if (t32) atomicAdd((unsigned long long *)(P.counts + DFTK_N_QCLASS + C), (unsigned long long)t32);
        }
    }
    __syncthreads();
    unsigned long long p64 = s_base64 + s_cnt[warp][0];
    unsigned long long p32 = s_base32 + s_cnt[warp][1];
#pragma unroll
    for (int it = 0; it < SELECT_PER_WARP; ++it) {
        if (m64[it] & (1u << lane)) P.list[C][p64 + __popc(m64[it] & below)] = make_int2(rows[it], kets[it]);
        if (m32[it] & (1u << lane))
            P.list[C][cap - 1 - (long long)(p32 + __popc(m32[it] & below))] = make_int2(rows[it], kets[it]);
        p64 += __popc(m64[it]);
        p32 += __popc(m32[it]);
    }
    __syncthreads();  // s_base/s_cnt are rewritten by the next tile
}

template <int C>
__device__ __forceinline__ void select_tile(const JkParams &P, long long tile, unsigned (*s_cnt)[2 * SELECT_NB],
                                            unsigned long long &s_base64, unsigned long long &s_base32)
{
    if (P.bucket) select_tile_bucketed<C>(P, tile, s_cnt, s_base64, s_base32);
    else select_tile_plain<C>(P, tile, s_cnt, s_base64, s_base32);
}

template <int C>
__global__ void __launch_bounds__(SELECT_THREADS) k_select(const JkParams P)
{
    __shared__ unsigned s_cnt[SELECT_THREADS / 32][2 * SELECT_NB];
    __shared__ unsigned long long s_base64, s_base32;
    const long long ntiles = (P.total[C] + SELECT_TILE - 1) / SELECT_TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        select_tile<C>(P, tile, s_cnt, s_base64, s_base32);
}

// All classes' selection passes in one launch: block b takes tile b of the
// concatenated tile ranges (tile_base[c] .. tile_base[c + 1] for class c),
// grid-striding over the total.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void __launch_bounds__(SELECT_THREADS) k_select_all(const JkParams P)
{
    __shared__ unsigned s_cnt[SELECT_THREADS / 32][2 * SELECT_NB];
    __shared__ unsigned long long s_base64, s_base32;
    long long base[DFTK_N_QCLASS + 1];
    base[0] = 0;
#pragma unroll
    for (int c = 0; c < DFTK_N_QCLASS; ++c) base[c + 1] = base[c] + (P.total[c] + SELECT_TILE - 1) / SELECT_TILE;
    for (long long t = blockIdx.x; t < base[DFTK_N_QCLASS]; t += gridDim.x) {
        int c = 0;
        while (t >= base[c + 1]) ++c;
        const long long tile = t - base[c];
        switch (c) {
        case 0: select_tile<0>(P, tile, s_cnt, s_base64, s_base32); break;
        case 1: select_tile<1>(P, tile, s_cnt, s_base64, s_base32); break;
        case 2: select_tile<2>(P, tile, s_cnt, s_base64, s_base32); break;
        case 3: select_tile<3>(P, tile, s_cnt, s_base64, s_base32); break;
        case 4: select_tile<4>(P, tile, s_cnt, s_base64, s_base32); break;
        default: select_tile<5>(P, tile, s_cnt, s_base64, s_base32); break;
        }
    }
}
#endif

// Minimum resident 128-thread blocks per SM requested from the compiler for
// each class kernel (caps its registers; 1 = no cap).  Measured on B200 for
// (H2O)_64: caps that force 64 registers help the light classes most; the
// p-rich classes lose to spills beyond these values.
#ifndef DFTK_MINB_D0
#define DFTK_MINB_D0 8
#endif
#ifndef DFTK_MINB_D1
#define DFTK_MINB_D1 8
#endif
#ifndef DFTK_MINB_D2
#define DFTK_MINB_D2 5
#endif
#ifndef DFTK_MINB_D3
#define DFTK_MINB_D3 5
#endif
#ifndef DFTK_MINB_D4
#define DFTK_MINB_D4 4
#endif
#ifndef DFTK_MINB_D5
#define DFTK_MINB_D5 2
#endif
#ifndef DFTK_MINB_F0
#define DFTK_MINB_F0 8
#endif
#ifndef DFTK_MINB_F1
#define DFTK_MINB_F1 8
#endif
#ifndef DFTK_MINB_F2
#define DFTK_MINB_F2 8
#endif
#ifndef DFTK_MINB_F3
#define DFTK_MINB_F3 8
#endif
#ifndef DFTK_MINB_F4
#define DFTK_MINB_F4 4
#endif
#ifndef DFTK_MINB_F5
#define DFTK_MINB_F5 3
#endif
template <int C, typename T> struct JkMinBlocks {
    static constexpr int d[6] = {DFTK_MINB_D0, DFTK_MINB_D1, DFTK_MINB_D2, DFTK_MINB_D3, DFTK_MINB_D4, DFTK_MINB_D5};
    static constexpr int f[6] = {DFTK_MINB_F0, DFTK_MINB_F1, DFTK_MINB_F2, DFTK_MINB_F3, DFTK_MINB_F4, DFTK_MINB_F5};
    static constexpr int value = sizeof(T) == 8 ? d[C] : f[C];
};

// J/K over the selected quartets of class C in precision T: warp w takes
// list entries 32w .. 32w + 31 (one split of the c components at a time).
template <int C, typename T>
__global__ void __launch_bounds__(128, JkMinBlocks<C, T>::value) k_jk_list(const JkParams P)
{
    constexpr int NS = EriClass<T, C, 0>::NSPLIT;
    constexpr bool fp32 = sizeof(T) == 4;
    const long long n = (long long)P.heads[(fp32 ? DFTK_N_QCLASS : 0) + C];
    const long long cap = P.total[C];
    const int2 *list = P.list[C];
    const long long nq = (n + 31) >> 5;
    const long long nwork = nq * NS;
    const int lane = threadIdx.x & 31;
    // each warp step takes `tile` consecutive work items (32-entry groups, or
    // their c-component splits), so a warp stays on neighbouring list entries;
    // split-major order: the grid sweeps the list with split 0's code, then
    // split 1's, so resident warps share one straight-line body
    const int tile = P.tile[(fp32 ? DFTK_N_QCLASS : 0) + C] > 0 ? P.tile[(fp32 ? DFTK_N_QCLASS : 0) + C] : 1;
    const long long wstride = (((long long)gridDim.x * blockDim.x) >> 5) * tile;
    for (long long g0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * tile; g0 < nwork; g0 += wstride) {
        for (int k = 0; k < tile; ++k) {
            const long long gw = g0 + k;
            if (gw >= nwork) break;
            const int split = (int)(gw / nq);
            const long long idx = (gw % nq) * 32 + lane;
            const bool valid = idx < n;
            int row = 0, ket = 0;
            if (valid) {
                const int2 e = __ldg(list + (fp32 ? cap - 1 - idx : idx));
                row = e.x;
                ket = e.y;
            }
            if constexpr (NS == 1) {
                jk_one<C, T, 0>(P, valid, row, ket);
            } else {
                if (split == 0) jk_one<C, T, 0>(P, valid, row, ket);
                else if (split == 1) jk_one<C, T, 1>(P, valid, row, ket);
                else jk_one<C, T, 2>(P, valid, row, ket);
            }
        }
    }
}

// One 32-entry tile of class C's list in precision T (split S of the c
// components for the split class): the body of k_jk_list for one warp.
template <int C, typename T>
__device__ __forceinline__ void list_tile(const JkParams &P, long long t)
{
    constexpr int NS = EriClass<T, C, 0>::NSPLIT;
    constexpr bool fp32 = sizeof(T) == 4;
    const long long n = (long long)P.heads[(fp32 ? DFTK_N_QCLASS : 0) + C];
    const long long cap = P.total[C];
    const int lane = threadIdx.x & 31;
    const int split = (int)(t % NS);
    const long long idx = (t / NS) * 32 + lane;
    const bool valid = idx < n;
    int row = 0, ket = 0;
    if (valid) {
        const int2 e = __ldg(P.list[C] + (fp32 ? cap - 1 - idx : idx));
        row = e.x;
        ket = e.y;
    }
    if constexpr (NS == 1) {
        jk_one<C, T, 0>(P, valid, row, ket);
    } else {
        if (split == 0) jk_one<C, T, 0>(P, valid, row, ket);
        else if (split == 1) jk_one<C, T, 1>(P, valid, row, ket);
        else jk_one<C, T, 2>(P, valid, row, ket);
    }
}

// Persistent J/K over the selected quartets of every class in precision T:
// a grid of resident blocks whose warps pull 32-entry tiles from one device
// work counter (P.heads[2 * DFTK_N_QCLASS + fp32]) over the concatenated
// tile ranges of all classes, heaviest class first, so the classes share the
// SMs without a launch per class and the tail of each class overlaps the next.
// MINB caps the registers of the whole kernel (every class runs under it).
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) k_jk_persist(const JkParams P)
{
    constexpr bool fp32 = sizeof(T) == 4;
    constexpr int order[DFTK_N_QCLASS] = {5, 4, 3, 2, 1, 0};
    constexpr int nsplit[DFTK_N_QCLASS] = {EriClass<T, 0, 0>::NSPLIT, EriClass<T, 1, 0>::NSPLIT,
                                           EriClass<T, 2, 0>::NSPLIT, EriClass<T, 3, 0>::NSPLIT,
                                           EriClass<T, 4, 0>::NSPLIT, EriClass<T, 5, 0>::NSPLIT};
    long long base[DFTK_N_QCLASS + 1];
    base[0] = 0;
#pragma unroll
    for (int k = 0; k < DFTK_N_QCLASS; ++k) {
        const int c = order[k];
        const long long n = (long long)P.heads[(fp32 ? DFTK_N_QCLASS : 0) + c];
        base[k + 1] = base[k] + ((n + 31) >> 5) * nsplit[c];
    }
    unsigned long long *ctr = P.heads + 2 * DFTK_N_QCLASS + (fp32 ? 1 : 0);
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(ctr, 1ull);
        t = __shfl_sync(DFTK_FULL_MASK, t, 0);
        if ((long long)t >= base[DFTK_N_QCLASS]) break;
        int k = 0;
        while ((long long)t >= base[k + 1]) ++k;
        const long long local = (long long)t - base[k];
        switch (order[k]) {
        case 0: list_tile<0, T>(P, local); break;
        case 1: list_tile<1, T>(P, local); break;
        case 2: list_tile<2, T>(P, local); break;
        case 3: list_tile<3, T>(P, local); break;
        case 4: list_tile<4, T>(P, local); break;
        default: list_tile<5, T>(P, local); break;
        }
    }
}

// J = Y + Y^T, K = Z + Z^T within each molecule's block (blockIdx.y = molecule)
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_symmetrize(const dftk_shells_t sh, const double *Y, const double *Za, const double *Zb, double *J,
                             double *Ka, double *Kb, int uhf)
{
    const int m = blockIdx.y;
    const long long base = sh.mol ? sh.mol_mat[m] : 0;
    const int N = sh.mol ? sh.mol_nao[m] : sh.n_ao;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)N * N;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / N), j = (int)(t % N);
        const long long o = base + t, ot = base + (long long)j * N + i;
        J[o] = Y[o] + Y[ot];
        Ka[o] = Za[o] + Za[ot];
        if (uhf) Kb[o] = Zb[o] + Zb[ot];
    }
}
#endif

// ------------------------------------------------------------- ERI blocks
struct EmitParams {
    const int *shell_ao;
    const int *shell_l;
    const int *ab[3];
    const int *np[3];
    const double *rec64[3];
    const float *rec32[3];
    const double *core64[3];
    const float *core32[3];
    const float *qp[3];
    int n_pairs[3];
    int kmax[3];
    long long nq;
    const int *desc;
    const long long *out_off;
    double *out;
};

__device__ __forceinline__ int ncomp(int l) { return (l + 1) * (l + 2) / 2; }

template <typename T> struct EmitRec;
template <> struct EmitRec<double> {
    __device__ static const double *get(const EmitParams &P, int pc) { return P.rec64[pc]; }
    __device__ static const double *core(const EmitParams &P, int pc) { return P.core64[pc]; }
};
template <> struct EmitRec<float> {
    __device__ static const float *get(const EmitParams &P, int pc) { return P.rec32[pc]; }
    __device__ static const float *core(const EmitParams &P, int pc) { return P.core32[pc]; }
};

template <int C, typename T, int S>
__device__ __forceinline__ void emit_split(const EmitParams &P, int row, int ket, const int (&slot)[4],
                                           const int (&stride)[4], double *out)
{
    using E = EriClass<T, C, S>;
    constexpr int X = E::BRA_CLASS, Yc = E::KET_CLASS;
    T I[E::NI];
    eri_run<C, T, S>(EmitRec<T>::get(P, X), EmitRec<T>::core(P, X), P.qp[X], P.n_pairs[X], P.kmax[X], row,
                     P.np[X][row], EmitRec<T>::get(P, Yc), EmitRec<T>::core(P, Yc), P.qp[Yc], P.n_pairs[Yc],
                     P.kmax[Yc], ket, P.np[Yc][ket], 0.0f, I);
#pragma unroll
    for (int ia = 0; ia < E::NA; ++ia)
#pragma unroll
        for (int ib = 0; ib < E::NB; ++ib)
#pragma unroll
            for (int m = 0; m < E::NCD; ++m) {
                const int comp[4] = {ia, ib, E::cd_c(m), E::cd_d(m)};
                long long o = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) o += (long long)comp[k] * stride[slot[k]];
                out[o] = (double)I[(ia * E::NB + ib) * E::NCD + m];
            }
}

template <int C, typename T>
__device__ __forceinline__ void emit_class(const EmitParams &P, int row, int ket, const int (&slot)[4],
                                           const int (&stride)[4], double *out)
{
    emit_split<C, T, 0>(P, row, ket, slot, stride, out);
    if constexpr (EriClass<T, C, 0>::NSPLIT > 1) {
        emit_split<C, T, 1>(P, row, ket, slot, stride, out);
        emit_split<C, T, 2>(P, row, ket, slot, stride, out);
    }
}

template <typename T>
__device__ __forceinline__ void emit_any(int C, const EmitParams &P, int row, int ket, const int (&slot)[4],
                                         const int (&stride)[4], double *out)
{
    switch (C) {
    case 0: emit_class<0, T>(P, row, ket, slot, stride, out); break;
    case 1: emit_class<1, T>(P, row, ket, slot, stride, out); break;
    case 2: emit_class<2, T>(P, row, ket, slot, stride, out); break;
    case 3: emit_class<3, T>(P, row, ket, slot, stride, out); break;
    case 4: emit_class<4, T>(P, row, ket, slot, stride, out); break;
    default: emit_class<5, T>(P, row, ket, slot, stride, out); break;
    }
}

// One thread per quartet; desc flags bit 3 selects the FP32 evaluation.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_emit(const EmitParams P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.nq) return;
    const int C = P.desc[4 * t], row = P.desc[4 * t + 1], ket = P.desc[4 * t + 2], flags = P.desc[4 * t + 3];
    if (C < 0 || C >= DFTK_N_QCLASS) return;
    constexpr int bra_pc[6] = {0, 1, 1, 2, 2, 2};
    constexpr int ket_pc[6] = {0, 0, 1, 0, 1, 2};
    const int X = bra_pc[C], Yc = ket_pc[C];
    if (row < 0 || row >= P.n_pairs[X] || ket < 0 || ket >= P.n_pairs[Yc]) return;
    // my (a', b', c', d') -> reference slots
    int slot[4];
    const int bra0 = (flags & 4) ? 2 : 0, ket0 = (flags & 4) ? 0 : 2;
    slot[0] = bra0 + ((flags & 1) ? 1 : 0);
    slot[1] = bra0 + ((flags & 1) ? 0 : 1);
    slot[2] = ket0 + ((flags & 2) ? 1 : 0);
    slot[3] = ket0 + ((flags & 2) ? 0 : 1);
    const int sh[4] = {P.ab[X][2 * row], P.ab[X][2 * row + 1], P.ab[Yc][2 * ket], P.ab[Yc][2 * ket + 1]};
    int nref[4];
    for (int k = 0; k < 4; ++k) nref[slot[k]] = ncomp(P.shell_l[sh[k]]);
    int stride[4];
    stride[3] = 1;
    stride[2] = nref[3];
    stride[1] = nref[3] * nref[2];
    stride[0] = nref[3] * nref[2] * nref[1];
    double *out = P.out + P.out_off[t];
    if (flags & 8) emit_any<float>(C, P, row, ket, slot, stride, out);
    else emit_any<double>(C, P, row, ket, slot, stride, out);
}
#endif
