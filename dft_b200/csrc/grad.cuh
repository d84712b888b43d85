// Analytic nuclear gradient of the RHF / UHF energy (FP64):
//   dE/dX = sum D (dT + dV)/dX - sum W dS/dX + sum Gamma d(mu nu|la si)/dX + dE_NN/dX
// with D the total density, W the energy-weighted density and, symmetrised
// over the eight index orientations,
//   Gamma = 1/2 D_mn D_ls - 1/4 (Da_ml Da_ns + Db_ml Db_ns + Da_ms Da_nl + Db_ms Db_nl)
// (RHF, Da = Db = D/2: 1/2 D D - 1/8 (D_ml D_ns + D_ms D_nl)).
//
// Derivatives of a primitive Cartesian Gaussian w.r.t. its centre raise and
// lower the power on that axis, d/dA_x x_A^i e^{-a x_A^2} = 2a x_A^{i+1} - i x_A^{i-1},
// so every derivative integral is an MD integral at L + 1 whose Hermite
// coefficients on the differentiated side are 2a E^{i+1,j} - i E^{i-1,j}
// (exponent-shifted E), recomputed per primitive pair from the pair records
// (P, p, K_AB, alpha) and the shell centres; nothing is stored per quartet.
//
// Two-electron part, one thread per Schwarz candidate shell quartet of a
// class (compile-time angular momenta, so every Hermite loop unrolls into
// registers).  Per bra primitive pair the Gamma-weighted bra Hermite density
// Eg[m][T] = sum_n Gamma[n][m] E^n_T is formed once; per primitive quartet
//   H[n][T]  += sum_T' (sum_m Gamma[n][m] (-1)^|T'| E^m_T') R_{T+T'}   (|T| <= L_ab + 1)
//   dE/dC    += sum_m sum_T' dE^m_T'(C) (-1)^|T'| sum_T Eg[m][T] R_{T+T'}
// and after the ket loop dE/dA, dE/dB = sum_n sum_T dE^n_T(A or B) H[n][T]
// (adjoint order: no derivative integral is formed).  dE/dD = -(A + B + C)
// by translational invariance.  Gradient sums go through a block-private
// shared-memory copy of the gradient (one global atomic per atom coordinate
// and block) when 3 n_atoms doubles fit, else straight to global atomics.
#pragma once

#include "boys.cuh"
#include "common.cuh"

#define GRAD_THREADS 128
#define GRAD_SMEM_ATOMS 2048  // 48 KB of shared memory

struct GradParams {
    dftk_shells_t sh;
    const int *shell_atom;
    int n_atoms;
    const int *ab[3];
    const double *q[3];
    const double *rec[3];
    const float *rec32[3];  // FP32 copies of the records (mixed gradient)
    const int *nprim[3];
    int n_pairs[3];
    int kmax;
    long long n_rows[DFTK_N_QCLASS];
    long long total[DFTK_N_QCLASS];
    const long long *row_off[DFTK_N_QCLASS];
    const double *D, *Da, *Db;  // total and spin densities (Da == Db for RHF)
    const float *Dsh;
    const float *qp[3];  // primitive Schwarz factors, descending per pair
    float tau_prim;      // primitive quartets with qp_bra qp_ket < tau_prim are skipped
    double tau;
    double *grad;  // [n_atoms * 3], accumulated
    // list path: per class the selected (bra row, ket) entries and their count
    const int2 *list[DFTK_N_QCLASS];
    const unsigned long long *heads;
    const int *ket_base[DFTK_N_QCLASS];  // batches: first ket pair of each row's molecule (NULL = 0)
};

template <typename T> struct GradRec;
template <> struct GradRec<double> {
    __device__ static const double *get(const GradParams &P, int pc) { return P.rec[pc]; }
};
template <> struct GradRec<float> {
    __device__ static const float *get(const GradParams &P, int pc) { return P.rec32[pc]; }
};

// Quartet classes (ss|ss)..(pp|pp): angular momenta and pair classes.
template <int C> struct GradClassOf;
template <> struct GradClassOf<0> { static constexpr int LA = 0, LB = 0, LC = 0, LD = 0, X = 0, Y = 0; };
template <> struct GradClassOf<1> { static constexpr int LA = 1, LB = 0, LC = 0, LD = 0, X = 1, Y = 0; };
template <> struct GradClassOf<2> { static constexpr int LA = 1, LB = 0, LC = 1, LD = 0, X = 1, Y = 1; };
template <> struct GradClassOf<3> { static constexpr int LA = 1, LB = 1, LC = 0, LD = 0, X = 2, Y = 0; };
template <> struct GradClassOf<4> { static constexpr int LA = 1, LB = 1, LC = 1, LD = 0, X = 2, Y = 1; };
template <> struct GradClassOf<5> { static constexpr int LA = 1, LB = 1, LC = 1, LD = 1, X = 2, Y = 2; };

// power of axis x of Cartesian component k of an s or p shell (x, y, z order)
__device__ __forceinline__ constexpr int g_cp(int l, int k, int x) { return l == 0 ? 0 : (k == x ? 1 : 0); }

// 1-D Hermite coefficients E^{i,j}_t without the Gaussian product factor,
// i <= IA, j <= JB, t <= i + j:
//   E^{i+1,j}_t = h E^{ij}_{t-1} + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}   (h = 1/2p)
// and the same in j with X_PB.
template <typename T, int IA, int JB>
__device__ __forceinline__ void g_etab(T PA, T PB, T h, T (&E)[IA + 1][JB + 1][IA + JB + 1])
{
    E[0][0][0] = T(1);
#pragma unroll
    for (int i = 0; i < IA; ++i)
#pragma unroll
        for (int t = 0; t <= i + 1; ++t) {
            T v;
            if (t <= i) {
                v = PA * E[i][0][t];
                if (t > 0) v = fma(h, E[i][0][t - 1], v);
            } else {
                v = h * E[i][0][t - 1];
            }
            if (t + 1 <= i) v = fma((T)(t + 1), E[i][0][t + 1], v);
            E[i + 1][0][t] = v;
        }
#pragma unroll
    for (int j = 0; j < JB; ++j)
#pragma unroll
        for (int i = 0; i <= IA; ++i)
#pragma unroll
            for (int t = 0; t <= i + j + 1; ++t) {
                T v;
                if (t <= i + j) {
                    v = PB * E[i][j][t];
                    if (t > 0) v = fma(h, E[i][j][t - 1], v);
                } else {
                    v = h * E[i][j][t - 1];
                }
                if (t + 1 <= i + j) v = fma((T)(t + 1), E[i][j][t + 1], v);
                E[i][j + 1][t] = v;
            }
}

// R_{tuv} = R^{(0)}_{tuv}(rho, X, Y, Z) for t + u + v <= LM, times `pre`:
// R^{(n)}_{000} = pre (-2 rho)^n F_n and
// R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X R^{(n+1)}_{t,u,v} (first non-zero index).
// Computed in place, one order n at a time from n = LM down to 0: order n's
// entries of index sum s need order n + 1's entries of sums s - 1 and s - 2,
// so writing the sums in decreasing order never overwrites an entry still to
// be read.  One cube of storage (no per-order copies), every index fixed at
// compile time.
template <typename T, int LM>
__device__ __forceinline__ void g_rcube(T X, T Y, T Z, T m2rho, T pre, const T *F,
                                        T (&R)[LM + 1][LM + 1][LM + 1])
{
    T cp[LM + 1];
    cp[0] = pre;
#pragma unroll
    for (int n = 1; n <= LM; ++n) cp[n] = cp[n - 1] * m2rho;
    R[0][0][0] = cp[LM] * F[LM];
#pragma unroll
    for (int n = LM - 1; n >= 0; --n) {
#pragma unroll
        for (int s = LM - n; s >= 1; --s)
#pragma unroll
            for (int t = 0; t <= s; ++t)
#pragma unroll
                for (int u = 0; u <= s - t; ++u) {
                    const int v = s - t - u;
                    T r;
                    if (t > 0) {
                        r = X * R[t - 1][u][v];
                        if (t > 1) r = fma((T)(t - 1), R[t - 2][u][v], r);
                    } else if (u > 0) {
                        r = Y * R[t][u - 1][v];
                        if (u > 1) r = fma((T)(u - 1), R[t][u - 2][v], r);
                    } else {
                        r = Z * R[t][u][v - 1];
                        if (v > 1) r = fma((T)(v - 1), R[t][u][v - 2], r);
                    }
                    R[t][u][v] = r;
                }
        R[0][0][0] = cp[n] * F[n];
    }
}

// gradient accumulation into the block's shared copy (or global memory)
__device__ __forceinline__ void g_add(double *s_grad, double *grad, int idx, double v)
{
    if (s_grad) atomicAdd(s_grad + idx, v);
    else atomicAdd(grad + idx, v);
}

__device__ __forceinline__ void g_smem_begin(double *s_grad, int n3)
{
    if (s_grad)
        for (int i = threadIdx.x; i < n3; i += blockDim.x) s_grad[i] = 0.0;
    __syncthreads();
}

__device__ __forceinline__ void g_smem_end(const double *s_grad, double *grad, int n3)
{
    __syncthreads();
    if (s_grad)
        for (int i = threadIdx.x; i < n3; i += blockDim.x)
            if (s_grad[i] != 0.0) atomicAdd(grad + i, s_grad[i]);
}

// gA, gB += sum_T dE^n_T(A), dE^n_T(B) V[T] over the derivative region of bra
// component n = (ka, kb): T in the box s_n + 1 per axis with |T| <= |s_n| + 1.
template <typename T, int LA, int LB, bool WITH_B = true>
__device__ __forceinline__ void g_ab_contract(int ka, int kb, const T (&Eb)[3][LA + 2][LB + 2][LA + LB + 3],
                                              T al, T be, const T (&V)[LA + LB + 2][LA + LB + 2][LA + LB + 2],
                                              T *gA, T *gB)
{
    const int sx = g_cp(LA, ka, 0) + g_cp(LB, kb, 0), sy = g_cp(LA, ka, 1) + g_cp(LB, kb, 1),
              sz = g_cp(LA, ka, 2) + g_cp(LB, kb, 2);
#pragma unroll
    for (int t = 0; t <= sx + 1; ++t)
#pragma unroll
        for (int u = 0; u <= sy + 1; ++u)
#pragma unroll
            for (int v = 0; v <= sz + 1; ++v) {
                if (t + u + v > sx + sy + sz + 1) continue;
                const T h = V[t][u][v];
#pragma unroll
                for (int dir = 0; dir < 3; ++dir) {
                    T ea = T(1), eb = T(1);
                    bool zero = false;
#pragma unroll
                    for (int x = 0; x < 3; ++x) {
                        const int i = g_cp(LA, ka, x), j = g_cp(LB, kb, x), tx = x == 0 ? t : (x == 1 ? u : v);
                        if (x != dir) {
                            if (tx > i + j) zero = true;
                            else {
                                ea *= Eb[x][i][j][tx];
                                eb *= Eb[x][i][j][tx];
                            }
                        } else {
                            T fa = T(2) * al * Eb[x][i + 1][j][tx];
                            if (i > 0 && tx <= i + j - 1) fa = fma(-(T)i, Eb[x][i - 1][j][tx], fa);
                            ea *= fa;
                            if constexpr (WITH_B) {
                                T fb = T(2) * be * Eb[x][i][j + 1][tx];
                                if (j > 0 && tx <= i + j - 1) fb = fma(-(T)j, Eb[x][i][j - 1][tx], fb);
                                eb *= fb;
                            }
                        }
                    }
                    if (!zero) {
                        gA[dir] = fma(ea, h, gA[dir]);
                        if constexpr (WITH_B) gB[dir] = fma(eb, h, gB[dir]);
                    }
                }
            }
}

// Two-electron gradient contributions gA, gB, gC of one shell quartet (bra
// row, ket) of class C (gD = -(gA + gB + gC)).  Classes with an s bra (<= 3
// bra components) hold H[n][T] across the ket primitives; the pp-bra classes
// contract each primitive quartet's V[T] with the bra derivative
// coefficients at once (less register state).  Both sides' primitive pairs
// come sorted by descending primitive Schwarz factor, and the loops stop once
// qp_bra qp_ket < tau_prim.
template <int C, typename T>
__device__ __forceinline__ void grad_quartet(const GradParams &P, int row, int ket, T *gA, T *gB,
                                             T *gC)
{
    using G = GradClassOf<C>;
    constexpr int LA = G::LA, LB = G::LB, LC = G::LC, LD = G::LD, X = G::X, Y = G::Y;
    constexpr int NA = LA ? 3 : 1, NB = LB ? 3 : 1, NC = LC ? 3 : 1, ND = LD ? 3 : 1;
    constexpr int NN = NA * NB, NM = NC * ND;
    constexpr int LAB = LA + LB, LCD = LC + LD, LM = LAB + LCD + 1;
    const int nX = P.n_pairs[X], nY = P.n_pairs[Y];
    const long long fsX = (long long)P.kmax * nX, fsY = (long long)P.kmax * nY;
    constexpr int faX = pair_alpha_field(X), faY = pair_alpha_field(Y);
    {
        const int a = P.ab[X][2 * row], b = P.ab[X][2 * row + 1];
        const int c = P.ab[Y][2 * ket], d = P.ab[Y][2 * ket + 1];
        const MolView mv = mol_view(P.sh, a);
        const long long N = mv.nao;
        const double *Dt = P.D + mv.mat, *Dta = P.Da + mv.mat, *Dtb = P.Db + mv.mat;
        const int oa = P.sh.ao[a], ob = P.sh.ao[b], oc = P.sh.ao[c], od = P.sh.ao[d];
        const int ew = (a == b) + (c == d) + ((X == Y) && (row == ket));
        const double f = 8.0 / (double)(1 << ew);  // orientations of the unique quartet
        T Gm[NN][NM];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j)
#pragma unroll
                for (int k = 0; k < NC; ++k)
#pragma unroll
                    for (int l = 0; l < ND; ++l) {
                        const long long I = oa + i, J = ob + j, K = oc + k, Lq = od + l;
                        const double coul = 0.5 * Dt[I * N + J] * Dt[K * N + Lq];
                        const double exch = 0.25 * (Dta[I * N + K] * Dta[J * N + Lq] + Dtb[I * N + K] * Dtb[J * N + Lq] +
                                                    Dta[I * N + Lq] * Dta[J * N + K] + Dtb[I * N + Lq] * Dtb[J * N + K]);
                        Gm[i * NB + j][k * ND + l] = (T)(f * (coul - exch));
                    }
        T cA[3], cB[3], cC[3], cD[3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            cA[x] = P.sh.xyz[3 * a + x];
            cB[x] = P.sh.xyz[3 * b + x];
            cC[x] = P.sh.xyz[3 * c + x];
            cD[x] = P.sh.xyz[3 * d + x];
        }
#pragma unroll
        for (int x = 0; x < 3; ++x) gA[x] = gB[x] = gC[x] = T(0);
        const T *brec = GradRec<T>::get(P, X) + row;
        const T *krec = GradRec<T>::get(P, Y) + ket;
        const float *bq = P.qp[X] + row, *kq = P.qp[Y] + ket;
        const int nbp = P.nprim[X][row], nkp = P.nprim[Y][ket];
        const float kq0 = __ldg(kq);
#pragma unroll 1
        for (int ip = 0; ip < nbp; ++ip) {
            const float qb = __ldg(bq + (long long)ip * nX);
            if (qb * kq0 < P.tau_prim) break;
            const T *br = brec + (long long)ip * nX;
            const T bP[3] = {__ldg(br), __ldg(br + fsX), __ldg(br + 2 * fsX)};
            const T bp = __ldg(br + F_P * fsX), bK = __ldg(br + F_K * fsX), bal = __ldg(br + faX * fsX);
            const T bbe = bp - bal, bh = T(0.5) / bp;
            T Eb[3][LA + 2][LB + 2][LAB + 3];
#pragma unroll
            for (int x = 0; x < 3; ++x) g_etab<T, LA + 1, LB + 1>(bP[x] - cA[x], bP[x] - cB[x], bh, Eb[x]);
            // Gamma-weighted bra Hermite density
            T Eg[NM][LAB + 1][LAB + 1][LAB + 1];
#pragma unroll
            for (int m = 0; m < NM; ++m)
#pragma unroll
                for (int t = 0; t <= LAB; ++t)
#pragma unroll
                    for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                        for (int v = 0; v <= LAB - t - u; ++v) {
                            bool first = true;
                            T s = T(0);
#pragma unroll
                            for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                                for (int kb = 0; kb < NB; ++kb) {
                                    const int ax = g_cp(LA, ka, 0), ay = g_cp(LA, ka, 1), az = g_cp(LA, ka, 2);
                                    const int bx = g_cp(LB, kb, 0), by = g_cp(LB, kb, 1), bz = g_cp(LB, kb, 2);
                                    if (t <= ax + bx && u <= ay + by && v <= az + bz) {
                                        const T e = Eb[0][ax][bx][t] * Eb[1][ay][by][u] * Eb[2][az][bz][v];
                                        s = first ? Gm[ka * NB + kb][m] * e : fma(Gm[ka * NB + kb][m], e, s);
                                        first = false;
                                    }
                                }
                            Eg[m][t][u][v] = s;
                        }
            if constexpr (LC == 0 && LD == 0 && NN > 3) {
                // (pp|ss): the ket is one s-s component, so the bra side folds
                // Gamma into the derivative Hermite density once per bra
                // primitive, DA[dir][T] = sum_n Gamma_n dE^n_T(A, dir); a
                // primitive quartet then costs sum_T DA R_T per direction.
                // C and D come from Hc[T'] = sum_T Eg[T] R_{T+T'}, and
                // dE/dB = -(A + C + D) (translational invariance).
                T DA[3][LAB + 2][LAB + 2][LAB + 2];
#pragma unroll
                for (int dir = 0; dir < 3; ++dir)
#pragma unroll
                    for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll
                        for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll
                            for (int v = 0; v <= LAB + 1 - t - u; ++v) DA[dir][t][u][v] = T(0);
#pragma unroll
                for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < NB; ++kb) {
                        const T gn = Gm[ka * NB + kb][0];
                        const int sx = g_cp(LA, ka, 0) + g_cp(LB, kb, 0), sy = g_cp(LA, ka, 1) + g_cp(LB, kb, 1),
                                  sz = g_cp(LA, ka, 2) + g_cp(LB, kb, 2);
#pragma unroll
                        for (int dir = 0; dir < 3; ++dir)
#pragma unroll
                            for (int t = 0; t <= sx + (dir == 0); ++t)
#pragma unroll
                                for (int u = 0; u <= sy + (dir == 1); ++u)
#pragma unroll
                                    for (int v = 0; v <= sz + (dir == 2); ++v) {
                                        T e = gn;
#pragma unroll
                                        for (int x = 0; x < 3; ++x) {
                                            const int i = g_cp(LA, ka, x), j = g_cp(LB, kb, x),
                                                      tx = x == 0 ? t : (x == 1 ? u : v);
                                            if (x != dir) {
                                                e *= Eb[x][i][j][tx];
                                            } else {
                                                T fa = T(2) * bal * Eb[x][i + 1][j][tx];
                                                if (i > 0 && tx <= i + j - 1) fa = fma(-(T)i, Eb[x][i - 1][j][tx], fa);
                                                e *= fa;
                                            }
                                        }
                                        DA[dir][t][u][v] += e;
                                    }
                    }
#pragma unroll 1
                for (int jp = 0; jp < nkp; ++jp) {
                    if (qb * __ldg(kq + (long long)jp * nY) < P.tau_prim) break;
                    const T *kr = krec + (long long)jp * nY;
                    const T kP[3] = {__ldg(kr), __ldg(kr + fsY), __ldg(kr + 2 * fsY)};
                    const T kp = __ldg(kr + F_P * fsY), kK = __ldg(kr + F_K * fsY), kal = __ldg(kr + faY * fsY);
                    const T kbe = kp - kal, kh = T(0.5) / kp;
                    const T s2 = bp + kp;
                    const T rs = Math<T>::rsqrt(s2);
                    const T rho = bp * kp * (rs * rs);
                    const T PQx = bP[0] - kP[0], PQy = bP[1] - kP[1], PQz = bP[2] - kP[2];
                    T F[LM + 1];
                    Boys<T, LM>::eval(rho * (PQx * PQx + PQy * PQy + PQz * PQz), F);
                    T R[LM + 1][LM + 1][LM + 1];
                    g_rcube<T, LM>(PQx, PQy, PQz, T(-2) * rho, bK * kK * rs, F, R);
#pragma unroll
                    for (int dir = 0; dir < 3; ++dir) {
                        T acc = T(0);
#pragma unroll
                        for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll
                            for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll
                                for (int v = 0; v <= LAB + 1 - t - u; ++v) acc = fma(DA[dir][t][u][v], R[t][u][v], acc);
                        gA[dir] += acc;
                    }
                    // Hc at T' = 0 and T' = e_dir
                    T h0 = T(0), h1[3] = {T(0), T(0), T(0)};
#pragma unroll
                    for (int t = 0; t <= LAB; ++t)
#pragma unroll
                        for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
                            for (int v = 0; v <= LAB - t - u; ++v) {
                                const T e = Eg[0][t][u][v];
                                h0 = fma(e, R[t][u][v], h0);
                                h1[0] = fma(e, R[t + 1][u][v], h1[0]);
                                h1[1] = fma(e, R[t][u + 1][v], h1[1]);
                                h1[2] = fma(e, R[t][u][v + 1], h1[2]);
                            }
                    // s-s ket: dE/dC_x = 2 gamma (X_QC h0 - h h1_x), dE/dD_x = 2 delta (X_QD h0 - h h1_x)
#pragma unroll
                    for (int dir = 0; dir < 3; ++dir) {
                        const T qc = kP[dir] - cC[dir], qd = kP[dir] - cD[dir];
                        gC[dir] = fma(T(2) * kal, fma(qc, h0, -kh * h1[dir]), gC[dir]);
                        gB[dir] = fma(T(2) * kbe, fma(qd, h0, -kh * h1[dir]), gB[dir]);  // gD for now
                    }
                }
                continue;
            }
            constexpr bool kHoldH = NN <= 3;
            constexpr int NH = kHoldH ? NN : 1;
            T H[NH][LAB + 2][LAB + 2][LAB + 2];
            if constexpr (kHoldH) {
#pragma unroll
                for (int n = 0; n < NH; ++n)
#pragma unroll
                    for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll
                        for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll
                            for (int v = 0; v <= LAB + 1 - t - u; ++v) H[n][t][u][v] = T(0);
            }
#pragma unroll 1
            for (int jp = 0; jp < nkp; ++jp) {
                if (qb * __ldg(kq + (long long)jp * nY) < P.tau_prim) break;
                const T *kr = krec + (long long)jp * nY;
                const T kP[3] = {__ldg(kr), __ldg(kr + fsY), __ldg(kr + 2 * fsY)};
                const T kp = __ldg(kr + F_P * fsY), kK = __ldg(kr + F_K * fsY), kal = __ldg(kr + faY * fsY);
                const T kh = T(0.5) / kp;
                // streaming (pp-bra) classes also need d raised: dE/dD from the ket side
                constexpr int JD = kHoldH ? LD : LD + 1;
                T Ek[3][LC + 2][JD + 1][LC + JD + 2];
#pragma unroll
                for (int x = 0; x < 3; ++x) g_etab<T, LC + 1, JD>(kP[x] - cC[x], kP[x] - cD[x], kh, Ek[x]);
                const T kbe = kp - kal;
                const T s2 = bp + kp;
                const T rs = Math<T>::rsqrt(s2);
                const T rho = bp * kp * (rs * rs);
                const T PQx = bP[0] - kP[0], PQy = bP[1] - kP[1], PQz = bP[2] - kP[2];
                T F[LM + 1];
                Boys<T, LM>::eval(rho * (PQx * PQx + PQy * PQy + PQz * PQz), F);
                T R[LM + 1][LM + 1][LM + 1];
                g_rcube<T, LM>(PQx, PQy, PQz, T(-2) * rho, bK * kK * rs, F, R);
                // bra side: H[n][T] += sum_T' Gk[T'] R[T + T']
#pragma unroll
                for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < NB; ++kb) {
                        const int n = ka * NB + kb;
                        T Gk[LCD + 1][LCD + 1][LCD + 1];
#pragma unroll
                        for (int t = 0; t <= LCD; ++t)
#pragma unroll
                            for (int u = 0; u <= LCD - t; ++u)
#pragma unroll
                                for (int v = 0; v <= LCD - t - u; ++v) {
                                    bool first = true;
                                    T s = T(0);
#pragma unroll
                                    for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                                        for (int kd = 0; kd < ND; ++kd) {
                                            const int cx = g_cp(LC, kc, 0), cy = g_cp(LC, kc, 1), cz = g_cp(LC, kc, 2);
                                            const int dx = g_cp(LD, kd, 0), dy = g_cp(LD, kd, 1), dz = g_cp(LD, kd, 2);
                                            if (t <= cx + dx && u <= cy + dy && v <= cz + dz) {
                                                T e = Ek[0][cx][dx][t] * Ek[1][cy][dy][u] * Ek[2][cz][dz][v];
                                                if ((t + u + v) & 1) e = -e;
                                                s = first ? Gm[n][kc * ND + kd] * e : fma(Gm[n][kc * ND + kd], e, s);
                                                first = false;
                                            }
                                        }
                                    Gk[t][u][v] = s;
                                }
                        const int sx = g_cp(LA, ka, 0) + g_cp(LB, kb, 0), sy = g_cp(LA, ka, 1) + g_cp(LB, kb, 1),
                                  sz = g_cp(LA, ka, 2) + g_cp(LB, kb, 2);
#pragma unroll
                        for (int t = 0; t <= sx + 1; ++t)
#pragma unroll
                            for (int u = 0; u <= sy + 1; ++u)
#pragma unroll
                                for (int v = 0; v <= sz + 1; ++v) {
                                    if (t + u + v > sx + sy + sz + 1) continue;
                                    T acc = kHoldH ? H[kHoldH ? n : 0][t][u][v] : T(0);
#pragma unroll
                                    for (int t2 = 0; t2 <= LCD; ++t2)
#pragma unroll
                                        for (int u2 = 0; u2 <= LCD - t2; ++u2)
#pragma unroll
                                            for (int v2 = 0; v2 <= LCD - t2 - u2; ++v2)
                                                acc = fma(Gk[t2][u2][v2], R[t + t2][u + u2][v + v2], acc);
                                    H[kHoldH ? n : 0][t][u][v] = acc;
                                }
                        // streaming classes: dE/dA only, dE/dB by translational invariance
                        if constexpr (!kHoldH) g_ab_contract<T, LA, LB, false>(ka, kb, Eb, bal, bbe, H[0], gA, gB);
                    }
                // ket side: dE/dC
#pragma unroll
                for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                    for (int kd = 0; kd < ND; ++kd) {
                        const int m = kc * ND + kd;
                        const int cx = g_cp(LC, kc, 0), cy = g_cp(LC, kc, 1), cz = g_cp(LC, kc, 2);
                        const int dx = g_cp(LD, kd, 0), dy = g_cp(LD, kd, 1), dz = g_cp(LD, kd, 2);
#pragma unroll
                        for (int t = 0; t <= cx + dx + 1; ++t)
#pragma unroll
                            for (int u = 0; u <= cy + dy + 1; ++u)
#pragma unroll
                                for (int v = 0; v <= cz + dz + 1; ++v) {
                                    if (t + u + v > cx + dx + cy + dy + cz + dz + 1) continue;
                                    T hc = T(0);
                                    bool first = true;
#pragma unroll
                                    for (int t1 = 0; t1 <= LAB; ++t1)
#pragma unroll
                                        for (int u1 = 0; u1 <= LAB - t1; ++u1)
#pragma unroll
                                            for (int v1 = 0; v1 <= LAB - t1 - u1; ++v1) {
                                                hc = first ? Eg[m][t1][u1][v1] * R[t + t1][u + u1][v + v1]
                                                           : fma(Eg[m][t1][u1][v1], R[t + t1][u + u1][v + v1], hc);
                                                first = false;
                                            }
                                    if ((t + u + v) & 1) hc = -hc;
#pragma unroll
                                    for (int dir = 0; dir < 3; ++dir) {
                                        T e = T(1), ed = T(1);
                                        bool zero = false;
#pragma unroll
                                        for (int x = 0; x < 3; ++x) {
                                            const int i = g_cp(LC, kc, x), j = g_cp(LD, kd, x), tx = x == 0 ? t : (x == 1 ? u : v);
                                            if (x != dir) {
                                                if (tx > i + j) zero = true;
                                                else {
                                                    e *= Ek[x][i][j][tx];
                                                    if constexpr (!kHoldH) ed *= Ek[x][i][j][tx];
                                                }
                                            } else {
                                                T fd = tx <= i + j + 1 ? T(2) * kal * Ek[x][i + 1][j][tx] : T(0);
                                                if (i > 0 && tx <= i + j - 1) fd = fma(-(T)i, Ek[x][i - 1][j][tx], fd);
                                                e *= fd;
                                                if constexpr (!kHoldH) {
                                                    T fdd = tx <= i + j + 1 ? T(2) * kbe * Ek[x][i][j + 1][tx] : T(0);
                                                    if (j > 0 && tx <= i + j - 1) fdd = fma(-(T)j, Ek[x][i][j - 1][tx], fdd);
                                                    ed *= fdd;
                                                }
                                            }
                                        }
                                        if (!zero) {
                                            gC[dir] = fma(e, hc, gC[dir]);
                                            if constexpr (!kHoldH) gB[dir] = fma(ed, hc, gB[dir]);  // dE/dD for now
                                        }
                                    }
                                }
                    }
            }
            // dE/dA and dE/dB from the bra intermediates
            if constexpr (kHoldH) {
#pragma unroll
                for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < NB; ++kb) g_ab_contract<T, LA, LB>(ka, kb, Eb, bal, bbe, H[ka * NB + kb], gA, gB);
            }
        }
        if constexpr (NN > 3) {
            // pp-bra classes: gB holds dE/dD here; dE/dB = -(A + C + D)
#pragma unroll
            for (int x = 0; x < 3; ++x) gB[x] = -(gA[x] + gC[x] + gB[x]);
        }
    }
}

// Two-electron gradient of class C over the Schwarz candidates (scan path:
// quartets with Q_ab Q_cd max|D|^2 < tau are skipped) or over the entries
// the selection pass kept (list path; warp w takes entries 32w .. 32w + 31,
// and a warp whose entries share the bra pair sums dE/dA, dE/dB in registers).
// Minimum resident blocks per SM requested per class (caps registers).
// Measured on B200 for (H2O)_64: 4 (128 registers) speeds up the s-bra
// classes by ~20 %; the p-rich classes lose to spills under any cap.
#ifndef DFTK_GMINB_0
#define DFTK_GMINB_0 4
#endif
#ifndef DFTK_GMINB_1
#define DFTK_GMINB_1 4
#endif
#ifndef DFTK_GMINB_2
#define DFTK_GMINB_2 1
#endif
#ifndef DFTK_GMINB_3
#define DFTK_GMINB_3 1
#endif
#ifndef DFTK_GMINB_4
#define DFTK_GMINB_4 1
#endif
#ifndef DFTK_GMINB_5
#define DFTK_GMINB_5 1
#endif
template <int C> struct GradMinBlocks {
    static constexpr int v[6] = {DFTK_GMINB_0, DFTK_GMINB_1, DFTK_GMINB_2, DFTK_GMINB_3, DFTK_GMINB_4, DFTK_GMINB_5};
    static constexpr int value = v[C];
};

// T = float (list path only): the FP32 entries the selection pass wrote at
// the back of the class list (mixed gradient); sums stay FP64.
template <int C, bool LIST, typename T = double>
__global__ void __launch_bounds__(GRAD_THREADS, GradMinBlocks<C>::value) k_grad_eri(const GradParams P)
{
    using G = GradClassOf<C>;
    constexpr int X = G::X, Y = G::Y;
    extern __shared__ double s_grad[];
    double *sg = P.n_atoms <= GRAD_SMEM_ATOMS ? s_grad : nullptr;
    g_smem_begin(sg, 3 * P.n_atoms);
    if constexpr (LIST) {
        constexpr bool fp32 = sizeof(T) == 4;
        const long long n = (long long)P.heads[(fp32 ? DFTK_N_QCLASS : 0) + C];
        const long long cap = P.total[C];
        const int2 *list = P.list[C];
        const long long nwork = (n + 31) >> 5;
        const int lane = threadIdx.x & 31;
        const long long wstride = ((long long)gridDim.x * blockDim.x) >> 5;
        for (long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gw < nwork; gw += wstride) {
            const long long idx = gw * 32 + lane;
            const bool valid = idx < n;
            int row = 0, ket = 0;
            if (valid) {
                const int2 e = __ldg(list + (fp32 ? cap - 1 - idx : idx));
                row = e.x;
                ket = e.y;
            }
            double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0}, gC[3] = {0.0, 0.0, 0.0};
            if (valid) {
                T tA[3], tB[3], tC[3];
                grad_quartet<C, T>(P, row, ket, tA, tB, tC);
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    gA[x] = (double)tA[x];
                    gB[x] = (double)tB[x];
                    gC[x] = (double)tC[x];
                }
            }
            const int row0 = __shfl_sync(DFTK_FULL_MASK, row, 0);  // lane 0 is valid whenever any lane is
            const bool uniform = __all_sync(DFTK_FULL_MASK, !valid || row == row0);
            if (valid) {
                const int c = P.ab[Y][2 * ket], d = P.ab[Y][2 * ket + 1];
                const int atC = P.shell_atom[c], atD = P.shell_atom[d];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    g_add(sg, P.grad, 3 * atC + x, gC[x]);
                    g_add(sg, P.grad, 3 * atD + x, -(gA[x] + gB[x] + gC[x]));
                }
            }
            const int a = P.ab[X][2 * row0], b = P.ab[X][2 * row0 + 1];
            const int atA = P.shell_atom[a], atB = P.shell_atom[b];
            if (uniform) {
#pragma unroll
                for (int x = 0; x < 3; ++x)
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        gA[x] += __shfl_xor_sync(DFTK_FULL_MASK, gA[x], o);
                        gB[x] += __shfl_xor_sync(DFTK_FULL_MASK, gB[x], o);
                    }
                if (lane == 0) {
#pragma unroll
                    for (int x = 0; x < 3; ++x) {
                        g_add(sg, P.grad, 3 * atA + x, gA[x]);
                        g_add(sg, P.grad, 3 * atB + x, gB[x]);
                    }
                }
            } else if (valid) {
                const int ra = P.ab[X][2 * row], rb = P.ab[X][2 * row + 1];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    g_add(sg, P.grad, 3 * P.shell_atom[ra] + x, gA[x]);
                    g_add(sg, P.grad, 3 * P.shell_atom[rb] + x, gB[x]);
                }
            }
        }
    } else {
        const long long ncand = P.total[C];
        const long long stride = (long long)gridDim.x * blockDim.x;
        for (long long cand = (long long)blockIdx.x * blockDim.x + threadIdx.x; cand < ncand; cand += stride) {
            const int row = find_row(P.row_off[C], P.n_rows[C], cand);
            const int ket = (int)(cand - P.row_off[C][row]) + (P.ket_base[C] ? P.ket_base[C][row] : 0);
            const int a = P.ab[X][2 * row], b = P.ab[X][2 * row + 1];
            const int c = P.ab[Y][2 * ket], d = P.ab[Y][2 * ket + 1];
            const float dm = quartet_dmax(P.sh, P.Dsh, a, b, c, d);
            if (P.q[X][row] * P.q[Y][ket] * (double)dm * (double)dm < P.tau) continue;
            double gA[3], gB[3], gC[3];
            grad_quartet<C, double>(P, row, ket, gA, gB, gC);
            const int at[4] = {P.shell_atom[a], P.shell_atom[b], P.shell_atom[c], P.shell_atom[d]};
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                g_add(sg, P.grad, 3 * at[0] + x, gA[x]);
                g_add(sg, P.grad, 3 * at[1] + x, gB[x]);
                g_add(sg, P.grad, 3 * at[2] + x, gC[x]);
                g_add(sg, P.grad, 3 * at[3] + x, -(gA[x] + gB[x] + gC[x]));
            }
        }
    }
    g_smem_end(sg, P.grad, 3 * P.n_atoms);
}

// Nuclear-attraction gradient of pair class PC: one thread per (shell pair,
// nucleus), nucleus fastest.  Per primitive pair,
//   V_n = -2 pi / p Z K_ab sum_T E^n_T R_T(p, P - C)
// with d/dA, d/dB from exponent-shifted E and d/dC_x = -sum_T E^n_T R_{T + 1_x}.
// Both orientations of an off-diagonal shell pair are counted (factor 2).
template <int PC>
__global__ void __launch_bounds__(GRAD_THREADS) k_grad_nuclear(const dftk_shells_t sh, const int *ab, int n_pairs,
                                                              const int *shell_atom, int n_atoms,
                                                              const double *atom_xyz, const double *atom_z,
                                                              const double *D, double *grad)
{
    constexpr int LA = PC == 0 ? 0 : 1, LB = PC == 2 ? 1 : 0;
    constexpr int NA = LA ? 3 : 1, NB = LB ? 3 : 1;
    constexpr int LM = LA + LB + 1;
    extern __shared__ double s_grad[];
    double *sg = n_atoms <= GRAD_SMEM_ATOMS ? s_grad : nullptr;
    g_smem_begin(sg, 3 * n_atoms);
    // a batch pairs each shell pair with the nuclei of its own molecule only
    const int nat_stride = sh.mol ? sh.max_natom : n_atoms;
    const long long total = (long long)n_pairs * nat_stride;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int pair = (int)(t / nat_stride), cl = (int)(t % nat_stride);
        const int a = ab[2 * pair], b = ab[2 * pair + 1];
        int cn = cl;
        if (sh.mol) {
            const int m = __ldg(sh.mol + a);
            if (cl >= __ldg(sh.mol_natom + m)) continue;
            cn = __ldg(sh.mol_atom0 + m) + cl;
        }
        const MolView mv = mol_view(sh, a);
        const long long N = mv.nao;
        const double cA[3] = {sh.xyz[3 * a], sh.xyz[3 * a + 1], sh.xyz[3 * a + 2]};
        const double cB[3] = {sh.xyz[3 * b], sh.xyz[3 * b + 1], sh.xyz[3 * b + 2]};
        const double cC[3] = {atom_xyz[3 * cn], atom_xyz[3 * cn + 1], atom_xyz[3 * cn + 2]};
        const double fpair = (a == b) ? 1.0 : 2.0;
        double Dm[NA][NB];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j) Dm[i][j] = fpair * D[mv.mat + (long long)(sh.ao[a] + i) * N + sh.ao[b] + j];
        const double ab2 = (cA[0] - cB[0]) * (cA[0] - cB[0]) + (cA[1] - cB[1]) * (cA[1] - cB[1]) +
                           (cA[2] - cB[2]) * (cA[2] - cB[2]);
        double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0}, gC[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia < sh.nprim[a]; ++ia)
            for (int ib = 0; ib < sh.nprim[b]; ++ib) {
                const double al = sh.prim_exp[sh.prim_off[a] + ia], be = sh.prim_exp[sh.prim_off[b] + ib];
                const double p = al + be, ip = 1.0 / p;
                const double pre = -2.0 * DFTK_PI * ip * atom_z[cn] * sh.prim_cn[sh.prim_off[a] + ia] *
                                   sh.prim_cn[sh.prim_off[b] + ib] * exp(-al * be * ip * ab2);
                double Pc[3], E[3][LA + 2][LB + 2][LA + LB + 3];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Pc[x] = (al * cA[x] + be * cB[x]) * ip;
                    g_etab<double, LA + 1, LB + 1>(Pc[x] - cA[x], Pc[x] - cB[x], 0.5 * ip, E[x]);
                }
                const double X = Pc[0] - cC[0], Y = Pc[1] - cC[1], Z = Pc[2] - cC[2];
                double F[LM + 1];
                Boys<double, LM>::eval(p * (X * X + Y * Y + Z * Z), F);
                double R[LM + 1][LM + 1][LM + 1];
                g_rcube<double, LM>(X, Y, Z, -2.0 * p, pre, F, R);
#pragma unroll
                for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < NB; ++kb) {
                        const double dm = Dm[ka][kb];
                        double tA[3] = {0.0, 0.0, 0.0}, tB[3] = {0.0, 0.0, 0.0};
                        g_ab_contract<double, LA, LB>(ka, kb, E, al, be, R, tA, tB);
                        // operator centre: -E^n_T R_{T + 1_dir}
                        const int sx = g_cp(LA, ka, 0) + g_cp(LB, kb, 0), sy = g_cp(LA, ka, 1) + g_cp(LB, kb, 1),
                                  sz = g_cp(LA, ka, 2) + g_cp(LB, kb, 2);
                        double tC[3] = {0.0, 0.0, 0.0};
#pragma unroll
                        for (int t = 0; t <= sx; ++t)
#pragma unroll
                            for (int u = 0; u <= sy; ++u)
#pragma unroll
                                for (int v = 0; v <= sz; ++v) {
                                    const double e = E[0][g_cp(LA, ka, 0)][g_cp(LB, kb, 0)][t] *
                                                     E[1][g_cp(LA, ka, 1)][g_cp(LB, kb, 1)][u] *
                                                     E[2][g_cp(LA, ka, 2)][g_cp(LB, kb, 2)][v];
                                    tC[0] = fma(e, R[t + 1][u][v], tC[0]);
                                    tC[1] = fma(e, R[t][u + 1][v], tC[1]);
                                    tC[2] = fma(e, R[t][u][v + 1], tC[2]);
                                }
#pragma unroll
                        for (int x = 0; x < 3; ++x) {
                            gA[x] = fma(dm, tA[x], gA[x]);
                            gB[x] = fma(dm, tB[x], gB[x]);
                            gC[x] = fma(-dm, tC[x], gC[x]);
                        }
                    }
            }
        const int atA = shell_atom[a], atB = shell_atom[b];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            g_add(sg, grad, 3 * atA + x, gA[x]);
            g_add(sg, grad, 3 * atB + x, gB[x]);
            g_add(sg, grad, 3 * cn + x, gC[x]);
        }
    }
    g_smem_end(sg, grad, 3 * n_atoms);
}

// Overlap and kinetic gradient of pair class PC: one thread per shell pair.
// S and T depend on A - B only, so d/dB = -d/dA.  1-D overlaps
// S_ij = E^{ij}_0 sqrt(pi / p) and the 1-D kinetic
// T_ij = b (2j+1) S_ij - 2 b^2 S_{i,j+2} - j (j-1)/2 S_{i,j-2}.
template <int PC>
__global__ void __launch_bounds__(GRAD_THREADS) k_grad_overlap_kinetic(const dftk_shells_t sh, const int *ab,
                                                                      int n_pairs, const int *shell_atom,
                                                                      int n_atoms, const double *D,
                                                                      const double *W, double *grad)
{
    constexpr int LA = PC == 0 ? 0 : 1, LB = PC == 2 ? 1 : 0;
    constexpr int NA = LA ? 3 : 1, NB = LB ? 3 : 1;
    extern __shared__ double s_grad[];
    double *sg = n_atoms <= GRAD_SMEM_ATOMS ? s_grad : nullptr;
    g_smem_begin(sg, 3 * n_atoms);
    for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < n_pairs; pair += gridDim.x * blockDim.x) {
        const int a = ab[2 * pair], b = ab[2 * pair + 1];
        const MolView mv = mol_view(sh, a);
        const long long N = mv.nao;
        const double cA[3] = {sh.xyz[3 * a], sh.xyz[3 * a + 1], sh.xyz[3 * a + 2]};
        const double cB[3] = {sh.xyz[3 * b], sh.xyz[3 * b + 1], sh.xyz[3 * b + 2]};
        const double fpair = (a == b) ? 1.0 : 2.0;
        const double ab2 = (cA[0] - cB[0]) * (cA[0] - cB[0]) + (cA[1] - cB[1]) * (cA[1] - cB[1]) +
                           (cA[2] - cB[2]) * (cA[2] - cB[2]);
        double gA[3] = {0.0, 0.0, 0.0};
        for (int ia = 0; ia < sh.nprim[a]; ++ia)
            for (int ib = 0; ib < sh.nprim[b]; ++ib) {
                const double al = sh.prim_exp[sh.prim_off[a] + ia], be = sh.prim_exp[sh.prim_off[b] + ib];
                const double p = al + be, ip = 1.0 / p;
                const double w = sh.prim_cn[sh.prim_off[a] + ia] * sh.prim_cn[sh.prim_off[b] + ib] *
                                 exp(-al * be * ip * ab2) * DFTK_PI * ip * sqrt(DFTK_PI * ip);
                // S1[x][i][j] = E^{ij}_0 for i <= LA + 1, j <= LB + 3
                double E[3][LA + 2][LB + 4][LA + LB + 5];
                double Pc[3];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Pc[x] = (al * cA[x] + be * cB[x]) * ip;
                    g_etab<double, LA + 1, LB + 3>(Pc[x] - cA[x], Pc[x] - cB[x], 0.5 * ip, E[x]);
                }
#pragma unroll
                for (int ka = 0; ka < NA; ++ka)
#pragma unroll
                    for (int kb = 0; kb < NB; ++kb) {
                        const long long mu = sh.ao[a] + ka, nu = sh.ao[b] + kb;
                        const double dm = fpair * w * D[mv.mat + mu * N + nu], wm = fpair * w * W[mv.mat + mu * N + nu];
                        double S[3][3], T[3][3];  // [axis][i = a - 1 .. a + 1 -> 0..2] at j = b
#pragma unroll
                        for (int x = 0; x < 3; ++x)
#pragma unroll
                            for (int di = -1; di <= 1; ++di) {
                                const int i = g_cp(LA, ka, x) + di, j = g_cp(LB, kb, x);
                                if (i < 0) {
                                    S[x][di + 1] = 0.0;
                                    T[x][di + 1] = 0.0;
                                    continue;
                                }
                                const double s = E[x][i][j][0];
                                double tk = be * (2 * j + 1) * s - 2.0 * be * be * E[x][i][j + 2][0];
                                if (j >= 2) tk -= 0.5 * j * (j - 1) * E[x][i][j - 2][0];
                                S[x][di + 1] = s;
                                T[x][di + 1] = tk;
                            }
#pragma unroll
                        for (int dir = 0; dir < 3; ++dir) {
                            const int o1 = (dir + 1) % 3, o2 = (dir + 2) % 3;
                            const int i = g_cp(LA, ka, dir);
                            double dS = 2.0 * al * S[dir][2], dT = 2.0 * al * T[dir][2];
                            if (i > 0) {
                                dS -= i * S[dir][0];
                                dT -= i * T[dir][0];
                            }
                            const double dSf = dS * S[o1][1] * S[o2][1];
                            const double dTf = dT * S[o1][1] * S[o2][1] + dS * (T[o1][1] * S[o2][1] + S[o1][1] * T[o2][1]);
                            gA[dir] += dm * dTf - wm * dSf;
                        }
                    }
            }
        const int atA = shell_atom[a], atB = shell_atom[b];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            g_add(sg, grad, 3 * atA + x, gA[x]);
            g_add(sg, grad, 3 * atB + x, -gA[x]);
        }
    }
    g_smem_end(sg, grad, 3 * n_atoms);
}
