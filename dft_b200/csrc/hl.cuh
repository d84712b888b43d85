// Shell quartets with a d or f shell (l <= 3): one warp per quartet,
// McMurchie-Davidson with run-time momenta, the Cartesian block and the
// Hermite intermediates in shared memory.  J/K builds send it the quartets
// with an f shell (every d class without one has generated thread-per-quartet
// code, hlc.cuh), or every d/f quartet when the caller gives no class spaces;
// the ERI-block emission, Schwarz factors and one-electron integrals of d and
// f shells use it throughout.
//
// Per primitive quartet (bra primitive pair i outside, ket pair j inside):
//   R^{(n)}_{tuv}, t+u+v+n <= L, level by level over the warp's lanes
//   (R^{(n)}_{000} = pre (-2 rho)^n F_n(rho |PQ|^2), then the recursion on
//   the first non-zero of t, u, v; shelled.py:296-348 restated), and the
//   ket-side Hermite-to-Cartesian transform
//     W[tuv][cd] += sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi} R_{t+tau,u+nu,v+phi};
// after the ket loop the bra transform I[ab][cd] += sum_tuv E^{ab}_tuv W[tuv][cd].
// E coefficients come from the record's PA, PB and 1/(2p) through the
// Obara-Saika-style recursion of calc_E (shelled.py:228-294), with the
// Gaussian product factor carried in the record's K.  Cartesian components
// of a d shell follow combinations() (shelled.py:15-23) and carry the
// factor 1/sqrt(prod (2 l_i - 1)!!) of normal() (shelled.py:95-101) that the
// per-primitive coefficient (coefficient x radial norm) leaves out.
#pragma once

#include "boys.cuh"
#include "common.cuh"
#include "generic.cuh"
#include "jk.cuh"

#define HL_LMAX 3          // largest shell momentum the kernels take (f)
#define HL_NC 10           // components of an f shell
#define HL_MAX_KPAIR 128   // primitive pairs per pair (Schwarz sort)
#define HL_FIELDS 13       // record fields (generic layout, alpha last)

// Sizes of the per-warp scratch for quartets of shells up to momentum LM:
// LM = 2 (d) takes 26.6 KB of shared memory per warp, LM = 3 (f) 167 KB, so
// a molecule runs the smallest instantiation that covers its shells.
template <int LM> struct HlDims {
    static constexpr int NC = (LM + 1) * (LM + 2) / 2;                    // components of one shell
    static constexpr int LP = 2 * LM;                                     // pair momentum
    static constexpr int L = 4 * LM;                                      // quartet momentum (Boys order)
    static constexpr int NH = (LP + 1) * (LP + 2) * (LP + 3) / 6;         // (t,u,v), t+u+v <= LP
    static constexpr int NR = (L + 1) * (L + 2) * (L + 3) * (L + 4) / 24;  // R^{(n)}_{tuv}, t+u+v+n <= L
    static constexpr int NE = 3 * (LM + 1) * (LM + 1) * (LP + 1);         // E^{ij}_t of one pair, 3 axes
};
static_assert(HlDims<HL_LMAX>::L < DFTK_BOYS_NL, "Boys table too short for the f quartets");

template <int LM> struct HlScratch {
    using D = HlDims<LM>;
    double Eb[D::NE];
    double Ek[D::NE];
    double R[D::NR];
    double W[D::NH * D::NC * D::NC];
    double I[D::NC * D::NC * D::NC * D::NC];
};

// Cartesian powers of component k of momentum l, in combinations() order
// (z power outer, then y, x innermost); packed x | y << 4 | z << 8.
static __constant__ int c_hl_comp[HL_LMAX + 1][HL_NC] = {
    {0x000},
    {0x001, 0x010, 0x100},
    {0x002, 0x011, 0x020, 0x101, 0x110, 0x200},
    {0x003, 0x012, 0x021, 0x030, 0x102, 0x111, 0x120, 0x201, 0x210, 0x300},
};
// 1 / sqrt(prod (2 l_i - 1)!!) per component (1/sqrt(3), 1/sqrt(15))
#define HL_R3 0.57735026918962576451
#define HL_R15 0.25819888974716112568
static __constant__ double c_hl_cnorm[HL_LMAX + 1][HL_NC] = {
    {1.0},
    {1.0, 1.0, 1.0},
    {HL_R3, 1.0, HL_R3, 1.0, 1.0, HL_R3},
    {HL_R15, HL_R3, HL_R3, HL_R15, HL_R3, 1.0, HL_R3, HL_R3, HL_R3, HL_R15},
};

__device__ __forceinline__ int hl_ncomp(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int hl_pow(int l, int k, int axis) { return (c_hl_comp[l][k] >> (4 * axis)) & 15; }

// Index of (t,u,v) among all triples with t+u+v <= s_max, ordered by
// s = t+u+v, then w = u+v, then v.
__device__ __forceinline__ int hl_tet(int t, int u, int v)
{
    const int s = t + u + v, w = u + v;
    return s * (s + 1) * (s + 2) / 6 + w * (w + 1) / 2 + v;
}
// inverse of hl_tet
__device__ __forceinline__ void hl_untet(int h, int &t, int &u, int &v)
{
    int s = 0;
    while ((s + 1) * (s + 2) * (s + 3) / 6 <= h) ++s;
    int k = h - s * (s + 1) * (s + 2) / 6;
    int w = 0;
    while ((w + 1) * (w + 2) / 2 <= k) ++w;
    v = k - w * (w + 1) / 2;
    u = w - v;
    t = s - w;
}
__device__ __forceinline__ int hl_c4(int x) { return x * (x - 1) * (x - 2) * (x - 3) / 24; }
// first entry of level n in the R array of a quartet of momentum L
__device__ __forceinline__ int hl_rbase(int L, int n) { return hl_c4(L + 4) - hl_c4(L - n + 4); }
template <int LM>
__device__ __forceinline__ int hl_eidx(int axis, int i, int j, int t)
{
    return ((axis * (LM + 1) + i) * (LM + 1) + j) * (2 * LM + 1) + t;
}

// E^{ij}_t for every axis, i <= la, j <= lb of one primitive pair: lane
// (axis, i, j) raises a i times from E^{00}_0 = 1, then b j times.
template <int LM>
__device__ __forceinline__ void hl_hermite_E(double *E, int la, int lb, double h, const double (&PA)[3],
                                             const double (&PB)[3], int lane)
{
    constexpr int LP = 2 * LM;
    const int nij = (la + 1) * (lb + 1);
    for (int e = lane; e < 3 * nij; e += 32) {
        const int axis = e / nij, r = e % nij, i = r / (lb + 1), j = r % (lb + 1);
        double cur[LP + 1];
#pragma unroll
        for (int t = 0; t <= LP; ++t) cur[t] = 0.0;
        cur[0] = 1.0;
        int order = 0;
        for (int step = 0; step < i + j; ++step) {
            const double sh = step < i ? PA[axis] : PB[axis];
            double nxt[LP + 1];
#pragma unroll
            for (int t = 0; t <= LP; ++t) {
                double v = 0.0;
                if (t <= order) v = sh * cur[t];
                if (t > 0 && t <= order + 1) v = fma(h, cur[t - 1], v);
                if (t + 1 <= order) v = fma((double)(t + 1), cur[t + 1], v);
                nxt[t] = v;
            }
            ++order;
#pragma unroll
            for (int t = 0; t <= LP; ++t) cur[t] = nxt[t];
        }
        for (int t = 0; t <= i + j; ++t) E[hl_eidx<LM>(axis, i, j, t)] = cur[t];
    }
}

// One primitive-pair record (generic 13-field layout): rec points at the
// pair's slot k (rec64 + k * n_pairs + pair), fs = kmax * n_pairs.
struct HlRec {
    double P[3], p, K, h, A[3], B[3];
};
__device__ __forceinline__ HlRec hl_load_rec(const double *rec, long long fs)
{
    HlRec r;
    r.P[0] = __ldg(rec);
    r.P[1] = __ldg(rec + fs);
    r.P[2] = __ldg(rec + 2 * fs);
    r.p = __ldg(rec + 3 * fs);
    r.K = __ldg(rec + 4 * fs);
    r.h = __ldg(rec + 5 * fs);
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        r.A[x] = __ldg(rec + (6 + x) * fs);
        r.B[x] = __ldg(rec + (9 + x) * fs);
    }
    return r;
}

// Contracted Cartesian block of the quartet (ab|cd) into s.I[(ia nb + ib) ncd + ic nd + id]
// (component normalisation applied).  bra/ket point at primitive slot 0 of
// their pair (rec64 + pair, qp + pair); st = n_pairs, fs = kmax * n_pairs.
// Primitive pairs come sorted by descending qp; both loops stop once
// qp_bra * qp_ket < eps.  Every lane of the warp must call this.
template <int LM>
__device__ void hl_quartet(HlScratch<LM> &s, int la, int lb, int lc, int ld, const double *bra, const float *bra_qp,
                           long long bst, long long bfs, int bra_n, const double *ket, const float *ket_qp,
                           long long kst, long long kfs, int ket_n, float eps)
{
    const int lane = threadIdx.x & 31;
    const int na = hl_ncomp(la), nb = hl_ncomp(lb), nc = hl_ncomp(lc), nd = hl_ncomp(ld);
    const int nab = na * nb, ncd = nc * nd;
    const int Lab = la + lb, Lcd = lc + ld, L = Lab + Lcd;
    const int nhb = (Lab + 1) * (Lab + 2) * (Lab + 3) / 6;
    for (int e = lane; e < nab * ncd; e += 32) s.I[e] = 0.0;
    const float kq0 = __ldg(ket_qp);
    for (int i = 0; i < bra_n; ++i) {
        const float qb = __ldg(bra_qp + i * bst);
        if (qb * kq0 < eps) break;
        const HlRec br = hl_load_rec(bra + i * bst, bfs);
        __syncwarp();
        hl_hermite_E<LM>(s.Eb, la, lb, br.h, br.A, br.B, lane);
        for (int e = lane; e < nhb * ncd; e += 32) s.W[e] = 0.0;
        for (int j = 0; j < ket_n; ++j) {
            const float qk = __ldg(ket_qp + j * kst);
            if (qb * qk < eps) break;
            const HlRec kr = hl_load_rec(ket + j * kst, kfs);
            __syncwarp();  // the previous primitive quartet is done with Ek and R
            hl_hermite_E<LM>(s.Ek, lc, ld, kr.h, kr.A, kr.B, lane);
            const double sum = br.p + kr.p;
            const double rho = br.p * kr.p / sum;
            const double X = br.P[0] - kr.P[0], Y = br.P[1] - kr.P[1], Z = br.P[2] - kr.P[2];
            const double pre = br.K * kr.K / sqrt(sum);
            double F[4 * LM + 1];
            boys_runtime(L, rho * (X * X + Y * Y + Z * Z), F);
            if (lane <= L) {
                double sc = pre;
                for (int n = 0; n < lane; ++n) sc *= -2.0 * rho;
                s.R[hl_rbase(L, lane)] = sc * F[lane];
            }
            __syncwarp();
            // levels t+u+v = 1..L: entry (component k of the level, order n)
            for (int lev = 1; lev <= L; ++lev) {
                const int ncomp_lev = (lev + 1) * (lev + 2) / 2, norder = L - lev + 1;
                for (int e = lane; e < ncomp_lev * norder; e += 32) {
                    const int k = e % ncomp_lev, n = e / ncomp_lev;
                    int w = 0;
                    while ((w + 1) * (w + 2) / 2 <= k) ++w;
                    const int v = k - w * (w + 1) / 2, u = w - v, t = lev - w;
                    const double *Rn1 = s.R + hl_rbase(L, n + 1);
                    double r;
                    if (t > 0) {
                        r = X * Rn1[hl_tet(t - 1, u, v)];
                        if (t > 1) r = fma((double)(t - 1), Rn1[hl_tet(t - 2, u, v)], r);
                    } else if (u > 0) {
                        r = Y * Rn1[hl_tet(t, u - 1, v)];
                        if (u > 1) r = fma((double)(u - 1), Rn1[hl_tet(t, u - 2, v)], r);
                    } else {
                        r = Z * Rn1[hl_tet(t, u, v - 1)];
                        if (v > 1) r = fma((double)(v - 1), Rn1[hl_tet(t, u, v - 2)], r);
                    }
                    s.R[hl_rbase(L, n) + hl_tet(t, u, v)] = r;
                }
                __syncwarp();
            }
            // ket transform into W[h][cd]
            for (int e = lane; e < nhb * ncd; e += 32) {
                const int h = e / ncd, cd = e % ncd, ic = cd / nd, id = cd % nd;
                int t, u, v;
                hl_untet(h, t, u, v);
                const int cx = hl_pow(lc, ic, 0), cy = hl_pow(lc, ic, 1), cz = hl_pow(lc, ic, 2);
                const int dx = hl_pow(ld, id, 0), dy = hl_pow(ld, id, 1), dz = hl_pow(ld, id, 2);
                double acc = 0.0;
                for (int tt = 0; tt <= cx + dx; ++tt) {
                    const double ex = s.Ek[hl_eidx<LM>(0, cx, dx, tt)];
                    for (int uu = 0; uu <= cy + dy; ++uu) {
                        const double exy = ex * s.Ek[hl_eidx<LM>(1, cy, dy, uu)];
                        for (int vv = 0; vv <= cz + dz; ++vv) {
                            const double c = exy * s.Ek[hl_eidx<LM>(2, cz, dz, vv)];
                            const double r = s.R[hl_tet(t + tt, u + uu, v + vv)];
                            acc = ((tt + uu + vv) & 1) ? fma(-c, r, acc) : fma(c, r, acc);
                        }
                    }
                }
                s.W[e] += acc;
            }
        }
        __syncwarp();
        // bra transform I[ab][cd] += E^{ab}_{tuv} W[tuv][cd]
        for (int e = lane; e < nab * ncd; e += 32) {
            const int ab = e / ncd, cd = e % ncd, ia = ab / nb, ib = ab % nb;
            const int ax = hl_pow(la, ia, 0), ay = hl_pow(la, ia, 1), az = hl_pow(la, ia, 2);
            const int bx = hl_pow(lb, ib, 0), by = hl_pow(lb, ib, 1), bz = hl_pow(lb, ib, 2);
            double acc = 0.0;
            for (int t = 0; t <= ax + bx; ++t) {
                const double ex = s.Eb[hl_eidx<LM>(0, ax, bx, t)];
                for (int u = 0; u <= ay + by; ++u) {
                    const double exy = ex * s.Eb[hl_eidx<LM>(1, ay, by, u)];
                    for (int v = 0; v <= az + bz; ++v)
                        acc = fma(exy * s.Eb[hl_eidx<LM>(2, az, bz, v)], s.W[hl_tet(t, u, v) * ncd + cd], acc);
                }
            }
            s.I[e] += acc;
        }
        __syncwarp();
    }
    // component normalisation
    for (int e = lane; e < nab * ncd; e += 32) {
        const int ab = e / ncd, cd = e % ncd;
        s.I[e] *= c_hl_cnorm[la][ab / nb] * c_hl_cnorm[lb][ab % nb] * c_hl_cnorm[lc][cd / nd] *
                  c_hl_cnorm[ld][cd % nd];
    }
    __syncwarp();
}

// ------------------------------------------------------------ Schwarz factors
// One warp per pair of a 13-field pair set (any momenta <= HL_LMAX): Q_ab =
// sqrt(max |(ab|ab)|) over the block, per primitive pair q_k likewise, then
// the pair's primitive records reordered by descending q_k (both copies).
extern __shared__ __align__(16) unsigned char hl_smem[];

template <int LM>
__global__ void __launch_bounds__(32) k_hl_schwarz(const dftk_shells_t sh, const dftk_pairs_t pr)
{
    HlScratch<LM> &s = *reinterpret_cast<HlScratch<LM> *>(hl_smem);
    __shared__ float qk[HL_MAX_KPAIR];
    __shared__ int order[HL_MAX_KPAIR];
    __shared__ double tmp[HL_MAX_KPAIR];
    __shared__ float tmp32[HL_MAX_KPAIR];
    const int pair = blockIdx.x, lane = threadIdx.x;
    const long long n = pr.n_pairs, fs = (long long)pr.kmax * n;
    const int np = pr.nprim[pair], kk = pr.kmax;
    const int a = pr.ab[2 * pair], b = pr.ab[2 * pair + 1];
    const int la = sh.l[a], lb = sh.l[b];
    const int nab = hl_ncomp(la) * hl_ncomp(lb);
    for (int k = lane; k < kk; k += 32) pr.qp[k * n + pair] = 0.0f;  // no screening while measuring
    __syncwarp();
    const double *rec = pr.rec64 + pair;
    const float *qp = pr.qp + pair;
    auto block_max = [&]() {
        double m = 0.0;
        for (int e = lane; e < nab * nab; e += 32) m = fmax(m, fabs(s.I[e]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(DFTK_FULL_MASK, m, o));
        __syncwarp();
        return m;
    };
    hl_quartet<LM>(s, la, lb, la, lb, rec, qp, n, fs, np, rec, qp, n, fs, np, 0.0f);
    const double qfull = sqrt(block_max());
    for (int k = 0; k < kk; ++k) {
        float v = 0.0f;
        if (k < np) {
            hl_quartet<LM>(s, la, lb, la, lb, rec + k * n, qp + k * n, n, fs, 1, rec + k * n, qp + k * n, n, fs, 1,
                           0.0f);
            v = (float)sqrt(block_max());
        }
        if (lane == 0) {
            qk[k] = v;
            order[k] = k;
        }
    }
    __syncwarp();
    if (lane == 0) {
        pr.q[pair] = qfull;
        for (int x = 1; x < kk; ++x) {
            const int o = order[x];
            int y = x - 1;
            while (y >= 0 && qk[order[y]] < qk[o]) { order[y + 1] = order[y]; --y; }
            order[y + 1] = o;
        }
    }
    __syncwarp();
    for (int f = 0; f < HL_FIELDS; ++f) {
        for (int k = lane; k < kk; k += 32) {
            tmp[k] = pr.rec64[(f * (long long)kk + k) * n + pair];
            tmp32[k] = pr.rec32[(f * (long long)kk + k) * n + pair];
        }
        __syncwarp();
        for (int k = lane; k < kk; k += 32) {
            pr.rec64[(f * (long long)kk + k) * n + pair] = tmp[order[k]];
            pr.rec32[(f * (long long)kk + k) * n + pair] = tmp32[order[k]];
        }
        __syncwarp();
    }
    for (int k = lane; k < kk; k += 32) pr.qp[k * n + pair] = qk[order[k]];
}

// --------------------------------------------------------------------- J / K
struct HlJkParams {
    dftk_shells_t sh;
    dftk_pairs_t hi, lo;
    long long n_rows;
    long long total[2];
    const long long *row_off[2];
    float tau_prim;
    const double *D, *Da, *Db;
    double *Y, *Za, *Zb;
    const float *Dsh;
    int uhf;
    double tau;
    long long *counts;  // [2]: quartets evaluated, primitive quartets (NULL = not counted)
    // bit 6 x + y: quartets of bra pair kind x and ket pair kind y belong to
    // a thread-per-quartet class kernel (pair kinds: hlc_kind)
    unsigned long long cover;
};

// Kind of the pair (a, b), l_a >= l_b: 0 ss, 1 ps, 2 pp, 3 ds, 4 dp, 5 dd;
// -1 with an f shell.
__device__ __forceinline__ int hlc_kind(int la, int lb)
{
    if (la > 2) return -1;
    return la == 0 ? 0 : (la == 1 ? 1 + lb : 3 + lb);
}

// Digest the block s.I of quartet (ab|cd) into Y (J) and Z (K) with the
// weights of the unique-quartet enumeration (same identities as the s/p
// digestion: J = Y + Y^T, K = Z + Z^T afterwards).
template <int LM>
__device__ void hl_digest(const HlJkParams &P, const HlScratch<LM> &s, int a, int b, int c, int d, bool same_pair)
{
    const int lane = threadIdx.x & 31;
    const int la = P.sh.l[a], lb = P.sh.l[b], lc = P.sh.l[c], ld = P.sh.l[d];
    const int na = hl_ncomp(la), nb = hl_ncomp(lb), nc = hl_ncomp(lc), nd = hl_ncomp(ld);
    const int ncd = nc * nd;
    const MolView mv = mol_view(P.sh, a);
    const int N = mv.nao;
    const int oa = P.sh.ao[a], ob = P.sh.ao[b], oc = P.sh.ao[c], od = P.sh.ao[d];
    const int ew = (a == b) + (c == d) + (same_pair ? 1 : 0);
    const double w = (double)(1 << ew), fJ = 2.0 / w, fK = 1.0 / w;
    const double *D = P.D + mv.mat;
    double *Y = P.Y + mv.mat;
    // Y_ab += fJ sum_cd I D_cd
    for (int ab = lane; ab < na * nb; ab += 32) {
        double acc = 0.0;
        for (int cd = 0; cd < ncd; ++cd)
            acc = fma(s.I[ab * ncd + cd], __ldg(D + (long long)(oc + cd / nd) * N + od + cd % nd), acc);
        atomicAdd(Y + (long long)(oa + ab / nb) * N + ob + ab % nb, fJ * acc);
    }
    // Y_cd += fJ sum_ab I D_ab
    for (int cd = lane; cd < ncd; cd += 32) {
        double acc = 0.0;
        for (int ab = 0; ab < na * nb; ++ab)
            acc = fma(s.I[ab * ncd + cd], __ldg(D + (long long)(oa + ab / nb) * N + ob + ab % nb), acc);
        atomicAdd(Y + (long long)(oc + cd / nd) * N + od + cd % nd, fJ * acc);
    }
    for (int spin = 0; spin < (P.uhf ? 2 : 1); ++spin) {
        const double *Ds = (spin ? P.Db : P.Da) + mv.mat;
        double *Z = (spin ? P.Zb : P.Za) + mv.mat;
        // Z_ac += fK sum_{b,d} I D_bd ; Z_ad += fK sum_{b,c} I D_bc
        for (int e = lane; e < na * (nc + nd); e += 32) {
            const int ia = e / (nc + nd), r = e % (nc + nd);
            double acc = 0.0;
            if (r < nc) {
                for (int ib = 0; ib < nb; ++ib)
                    for (int id = 0; id < nd; ++id)
                        acc = fma(s.I[(ia * nb + ib) * ncd + r * nd + id],
                                  __ldg(Ds + (long long)(ob + ib) * N + od + id), acc);
                atomicAdd(Z + (long long)(oa + ia) * N + oc + r, fK * acc);
            } else {
                const int id = r - nc;
                for (int ib = 0; ib < nb; ++ib)
                    for (int ic = 0; ic < nc; ++ic)
                        acc = fma(s.I[(ia * nb + ib) * ncd + ic * nd + id],
                                  __ldg(Ds + (long long)(ob + ib) * N + oc + ic), acc);
                atomicAdd(Z + (long long)(oa + ia) * N + od + id, fK * acc);
            }
        }
        // Z_bc += fK sum_{a,d} I D_ad ; Z_bd += fK sum_{a,c} I D_ac
        for (int e = lane; e < nb * (nc + nd); e += 32) {
            const int ib = e / (nc + nd), r = e % (nc + nd);
            double acc = 0.0;
            if (r < nc) {
                for (int ia = 0; ia < na; ++ia)
                    for (int id = 0; id < nd; ++id)
                        acc = fma(s.I[(ia * nb + ib) * ncd + r * nd + id],
                                  __ldg(Ds + (long long)(oa + ia) * N + od + id), acc);
                atomicAdd(Z + (long long)(ob + ib) * N + oc + r, fK * acc);
            } else {
                const int id = r - nc;
                for (int ia = 0; ia < na; ++ia)
                    for (int ic = 0; ic < nc; ++ic)
                        acc = fma(s.I[(ia * nb + ib) * ncd + ic * nd + id],
                                  __ldg(Ds + (long long)(oa + ia) * N + oc + ic), acc);
                atomicAdd(Z + (long long)(ob + ib) * N + od + id, fK * acc);
            }
        }
    }
}

// One block (one warp) per candidate at a time over the two candidate
// spaces: (hi | lo) then (hi | hi); quartets whose density-weighted Schwarz
// bound Q_ab Q_cd max|D| falls below tau are skipped.
template <int LM>
__global__ void __launch_bounds__(32) k_hl_jk(const HlJkParams P)
{
    HlScratch<LM> &s = *reinterpret_cast<HlScratch<LM> *>(hl_smem);
    const long long total = P.total[0] + P.total[1];
    const long long hfs = (long long)P.hi.kmax * P.hi.n_pairs;
    const long long lfs = (long long)P.lo.kmax * P.lo.n_pairs;
    long long evaluated = 0;
    for (long long cand = blockIdx.x; cand < total; cand += gridDim.x) {
        const int kind = cand >= P.total[0];
        const long long cc = kind ? cand - P.total[0] : cand;
        const int row = find_row(P.row_off[kind], P.n_rows, cc);
        const int ket = (int)(cc - __ldg(P.row_off[kind] + row));
        const dftk_pairs_t &K = kind ? P.hi : P.lo;
        const int a = P.hi.ab[2 * row], b = P.hi.ab[2 * row + 1];
        const int c = K.ab[2 * ket], d = K.ab[2 * ket + 1];
        if (P.cover) {
            const int x = hlc_kind(P.sh.l[a], P.sh.l[b]), y = hlc_kind(P.sh.l[c], P.sh.l[d]);
            if (x >= 0 && y >= 0 && ((P.cover >> (6 * x + y)) & 1)) continue;
        }
        const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
        if (P.hi.q[row] * K.q[ket] * (double)dm < P.tau) continue;
        hl_quartet<LM>(s, P.sh.l[a], P.sh.l[b], P.sh.l[c], P.sh.l[d], P.hi.rec64 + row, P.hi.qp + row, P.hi.n_pairs,
                   hfs, P.hi.nprim[row], K.rec64 + ket, K.qp + ket, K.n_pairs, kind ? hfs : lfs, K.nprim[ket],
                   P.tau_prim);
        hl_digest<LM>(P, s, a, b, c, d, kind == 1 && row == ket);
        __syncwarp();
        ++evaluated;
    }
    if (P.counts && threadIdx.x == 0 && evaluated)
        atomicAdd((unsigned long long *)P.counts, (unsigned long long)evaluated);
}

// ---------------------------------------------------------------- ERI blocks
// desc per quartet: {kind (0 = (hi|lo), 1 = (hi|hi)), bra row, ket row,
// flags, n0, n1, n2, n3}; flags bit 0: the reference's first bra shell is
// the pair's second, bit 1 likewise for the ket, bit 2: the reference's bra
// is this quartet's ket.  n0..n3 are the reference slot AO counts (strides of
// the flat block), out_off[q] the block's first element.
template <int LM>
__global__ void __launch_bounds__(32) k_hl_emit(const dftk_shells_t sh, const dftk_pairs_t hi, const dftk_pairs_t lo,
                                                long long nq, const int *desc, const long long *out_off, double *out)
{
    HlScratch<LM> &s = *reinterpret_cast<HlScratch<LM> *>(hl_smem);
    const long long hfs = (long long)hi.kmax * hi.n_pairs, lfs = (long long)lo.kmax * lo.n_pairs;
    for (long long q = blockIdx.x; q < nq; q += gridDim.x) {
        const int *dq = desc + 8 * q;
        const int kind = dq[0], row = dq[1], ket = dq[2], flags = dq[3];
        if (kind < 0 || kind > 1 || row < 0 || row >= hi.n_pairs) continue;
        const dftk_pairs_t &K = kind ? hi : lo;
        if (ket < 0 || ket >= K.n_pairs) continue;
        const int sha[4] = {hi.ab[2 * row], hi.ab[2 * row + 1], K.ab[2 * ket], K.ab[2 * ket + 1]};
        const int l4[4] = {sh.l[sha[0]], sh.l[sha[1]], sh.l[sha[2]], sh.l[sha[3]]};
        hl_quartet<LM>(s, l4[0], l4[1], l4[2], l4[3], hi.rec64 + row, hi.qp + row, hi.n_pairs, hfs, hi.nprim[row],
                   K.rec64 + ket, K.qp + ket, K.n_pairs, kind ? hfs : lfs, K.nprim[ket], 0.0f);
        int slot[4];
        const int bra0 = (flags & 4) ? 2 : 0, ket0 = (flags & 4) ? 0 : 2;
        slot[0] = bra0 + ((flags & 1) ? 1 : 0);
        slot[1] = bra0 + ((flags & 1) ? 0 : 1);
        slot[2] = ket0 + ((flags & 2) ? 1 : 0);
        slot[3] = ket0 + ((flags & 2) ? 0 : 1);
        long long stride[4];
        stride[3] = 1;
        stride[2] = dq[7];
        stride[1] = (long long)dq[7] * dq[6];
        stride[0] = (long long)dq[7] * dq[6] * dq[5];
        const int n1 = hl_ncomp(l4[1]), n2 = hl_ncomp(l4[2]), n3 = hl_ncomp(l4[3]);
        const int tot = hl_ncomp(l4[0]) * n1 * n2 * n3;
        double *o = out + out_off[q];
        for (int e = threadIdx.x; e < tot; e += 32) {
            const int c3 = e % n3, c2 = (e / n3) % n2, c1 = (e / (n3 * n2)) % n1, c0 = e / (n3 * n2 * n1);
            const int comp[4] = {c0, c1, c2, c3};
            long long off = 0;
            for (int k = 0; k < 4; ++k) off += comp[k] * stride[slot[k]];
            o[off] = s.I[e];
        }
        __syncwarp();
    }
}

// ------------------------------------------------------- one-electron blocks
// R^{(0)}_{tuv}(alpha, X, Y, Z), t+u+v <= L <= 2 HL_LMAX, for one thread,
// tet-indexed (hl_tet): the same level-by-level recursion as hl_quartet.
#define HL_NR1 210  // R^{(n)}_{tuv} with t+u+v+n <= 2 HL_LMAX
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __device__ void hl_R_thread(int L, double alpha, double X, double Y, double Z, double *R0)
{
    double F[2 * HL_LMAX + 1];
    boys_runtime(L, alpha * (X * X + Y * Y + Z * Z), F);
    double R[HL_NR1];
    double sc = 1.0;
#pragma unroll 1
    for (int n = 0; n <= L; ++n) {
        R[hl_rbase(L, n)] = sc * F[n];
        sc *= -2.0 * alpha;
    }
#pragma unroll 1
    for (int lev = 1; lev <= L; ++lev)
#pragma unroll 1
        for (int w = 0; w <= lev; ++w)
#pragma unroll 1
            for (int v = 0; v <= w; ++v) {
                const int u = w - v, t = lev - w;
#pragma unroll 1
                for (int n = 0; n + lev <= L; ++n) {
                    const double *Rn1 = R + hl_rbase(L, n + 1);
                    double r;
                    if (t > 0) {
                        r = X * Rn1[hl_tet(t - 1, u, v)];
                        if (t > 1) r = fma((double)(t - 1), Rn1[hl_tet(t - 2, u, v)], r);
                    } else if (u > 0) {
                        r = Y * Rn1[hl_tet(t, u - 1, v)];
                        if (u > 1) r = fma((double)(u - 1), Rn1[hl_tet(t, u - 2, v)], r);
                    } else {
                        r = Z * Rn1[hl_tet(t, u, v - 1)];
                        if (v > 1) r = fma((double)(v - 1), Rn1[hl_tet(t, u, v - 2)], r);
                    }
                    R[hl_rbase(L, n) + hl_tet(t, u, v)] = r;
                }
            }
    const int n0 = (L + 1) * (L + 2) * (L + 3) / 6;
#pragma unroll 1
    for (int k = 0; k < n0; ++k) R0[k] = R[k];
}
#endif

// S, T, V of the shell pairs (i, j), j <= i, with a d shell (the s/p pairs
// are k_one_electron's): the same MD overlap / kinetic / nuclear-attraction
// formulas with run-time component loops (overlap_1d and T_raw,
// shelled.py:104-155; nuclear_kernel's V, shelled.py:420-436), the component
// normalisation applied per Cartesian function.  One thread per pair.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_one_electron_hl(const dftk_shells_t sh, int n_atoms, const double *atom_xyz,
                                  const double *atom_z, double *S, double *T, double *V)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npair = (long long)sh.n_shells * (sh.n_shells + 1) / 2;
    if (t >= npair) return;
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)i * (i + 1) / 2 > t) --i;
    while ((long long)(i + 1) * (i + 2) / 2 <= t) ++i;
    const int j = (int)(t - (long long)i * (i + 1) / 2);
    const int la = sh.l[i], lb = sh.l[j];
    if (la > HL_LMAX || lb > HL_LMAX || la < 0 || lb < 0 || (la < 2 && lb < 2)) return;
    if (sh.mol) return;  // batches carry s/p shells only
    const int ca = hl_ncomp(la), cb = hl_ncomp(lb);
    const int N = sh.n_ao;
    const double A[3] = {sh.xyz[3 * i], sh.xyz[3 * i + 1], sh.xyz[3 * i + 2]};
    const double B[3] = {sh.xyz[3 * j], sh.xyz[3 * j + 1], sh.xyz[3 * j + 2]};
    double s_acc[HL_NC * HL_NC], t_acc[HL_NC * HL_NC], v_acc[HL_NC * HL_NC];
#pragma unroll 1
    for (int x = 0; x < ca * cb; ++x) s_acc[x] = t_acc[x] = v_acc[x] = 0.0;
    const int L = la + lb;
#pragma unroll 1
    for (int ia = 0; ia < sh.nprim[i]; ++ia)
#pragma unroll 1
        for (int ib = 0; ib < sh.nprim[j]; ++ib) {
            const double al = sh.prim_exp[sh.prim_off[i] + ia], be = sh.prim_exp[sh.prim_off[j] + ib];
            const double w = sh.prim_cn[sh.prim_off[i] + ia] * sh.prim_cn[sh.prim_off[j] + ib];
            const double p = al + be;
            const double sq = sqrt(DFTK_PI / p);
            double Pc[3];
            for (int x = 0; x < 3; ++x) Pc[x] = (al * A[x] + be * B[x]) / p;
            // ov[axis][a power][b power 0..lb+2]; eh = E^{ab}_t for V
            double ov[3 * (HL_LMAX + 1) * (HL_LMAX + 3)];
            double eh[HlDims<HL_LMAX>::NE];
#pragma unroll 1
            for (int x = 0; x < 3; ++x)
#pragma unroll 1
                for (int pa = 0; pa <= la; ++pa)
#pragma unroll 1
                    for (int pb = 0; pb <= lb + 2; ++pb) {
                        double E[16];
                        herm_E1d(al, be, A[x], B[x], pa, pb, E);
                        ov[(x * (HL_LMAX + 1) + pa) * (HL_LMAX + 3) + pb] = E[0] * sq;
                        if (pb <= lb)
                            for (int tt = 0; tt <= pa + pb; ++tt) eh[hl_eidx<HL_LMAX>(x, pa, pb, tt)] = E[tt];
                    }
            double vv[HL_NC * HL_NC];
#pragma unroll 1
            for (int x = 0; x < ca * cb; ++x) vv[x] = 0.0;
#pragma unroll 1
            for (int c = 0; c < n_atoms; ++c) {
                double R[HlDims<HL_LMAX>::NH];
                hl_R_thread(L, p, Pc[0] - atom_xyz[3 * c], Pc[1] - atom_xyz[3 * c + 1], Pc[2] - atom_xyz[3 * c + 2],
                            R);
#pragma unroll 1
                for (int k = 0; k < ca * cb; ++k) {
                    const int ka = k / cb, kb = k % cb;
                    const int ax = hl_pow(la, ka, 0), ay = hl_pow(la, ka, 1), az = hl_pow(la, ka, 2);
                    const int bx = hl_pow(lb, kb, 0), by = hl_pow(lb, kb, 1), bz = hl_pow(lb, kb, 2);
                    double s = 0.0;
#pragma unroll 1
                    for (int tx = 0; tx <= ax + bx; ++tx)
#pragma unroll 1
                        for (int ty = 0; ty <= ay + by; ++ty)
#pragma unroll 1
                            for (int tz = 0; tz <= az + bz; ++tz)
                                s += eh[hl_eidx<HL_LMAX>(0, ax, bx, tx)] * eh[hl_eidx<HL_LMAX>(1, ay, by, ty)] *
                                     eh[hl_eidx<HL_LMAX>(2, az, bz, tz)] * R[hl_tet(tx, ty, tz)];
                    vv[k] += atom_z[c] * s;
                }
            }
#pragma unroll 1
            for (int k = 0; k < ca * cb; ++k) {
                const int ka = k / cb, kb = k % cb;
                double o[3], kk[3];
                for (int x = 0; x < 3; ++x) {
                    const int a_ = hl_pow(la, ka, x), b_ = hl_pow(lb, kb, x);
                    const double *ovx = ov + (x * (HL_LMAX + 1) + a_) * (HL_LMAX + 3);
                    o[x] = ovx[b_];
                    kk[x] = be * (2 * b_ + 1) * ovx[b_] - 2.0 * be * be * ovx[b_ + 2] -
                            (b_ >= 2 ? 0.5 * b_ * (b_ - 1) * ovx[b_ - 2] : 0.0);
                }
                s_acc[k] += w * o[0] * o[1] * o[2];
                t_acc[k] += w * (kk[0] * o[1] * o[2] + o[0] * kk[1] * o[2] + o[0] * o[1] * kk[2]);
                v_acc[k] += w * (-2.0 * DFTK_PI / p) * vv[k];
            }
        }
    const int oi = sh.ao[i], oj = sh.ao[j];
#pragma unroll 1
    for (int k = 0; k < ca * cb; ++k) {
        const int ka = k / cb, kb = k % cb;
        const double g = c_hl_cnorm[la][ka] * c_hl_cnorm[lb][kb];
        const long long r = (long long)(oi + ka) * N + oj + kb, c = (long long)(oj + kb) * N + oi + ka;
        S[r] = S[c] = g * s_acc[k];
        T[r] = T[c] = g * t_acc[k];
        V[r] = V[c] = g * v_acc[k];
    }
}
#endif

// J += Y + Y^T, K += Z + Z^T (one molecule): the d-quartet part added to the
// s/p part dftk_jk wrote.
#ifndef DFTK_HLC_PART  // not compiled into the hlc_part_*.cu units (unused there)
static __global__ void k_symmetrize_add(int N, const double *Y, const double *Za, const double *Zb, double *J, double *Ka,
                                 double *Kb, int uhf)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)N * N;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / N), j = (int)(t % N);
        const long long ot = (long long)j * N + i;
        J[t] += Y[t] + Y[ot];
        Ka[t] += Za[t] + Za[ot];
        if (uhf) Kb[t] += Zb[t] + Zb[ot];
    }
}
#endif
