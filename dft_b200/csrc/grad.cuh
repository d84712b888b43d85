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
// (exponent-shifted E), recomputed from the shells per primitive pair.  Two
// electron part: per quartet, Gamma is formed once; the ket-transformed
// Hermite integrals are contracted with Gamma into bra-Hermite intermediates
// H[mu nu][tuv] summed over ket primitives, which the derivative E of one bra
// primitive turns into dE/dA and dE/dB (adjoint order: no derivative integral
// is stored).  dE/dC comes from the mirrored pass, dE/dD = -(A + B + C) by
// translational invariance.
#pragma once

#include "generic.cuh"

#define GRAD_LMAX 5   // L + 1 for s/p shell quartets

__device__ __forceinline__ int g_ncomp(int l) { return (l + 1) * (l + 2) / 2; }

__device__ __forceinline__ void g_pow(int l, int k, int *pw)
{
    if (l == 0) { pw[0] = pw[1] = pw[2] = 0; return; }
    pw[0] = (k == 0); pw[1] = (k == 1); pw[2] = (k == 2);
}

// 1-D Hermite E^{i,j}_t for i <= 2, j <= 2 (powers up to l + 1) on one axis:
// E[(i * 3 + j) * 5 + t], t <= 4, zero beyond t = i + j.
__device__ __forceinline__ void g_E_table(double al, double be, double A, double B, double *E)
{
    for (int i = 0; i <= 2; ++i)
        for (int j = 0; j <= 2; ++j) {
            double e[16];
            herm_E1d(al, be, A, B, i, j, e);
            for (int t = 0; t < 5; ++t) E[(i * 3 + j) * 5 + t] = t <= i + j ? e[t] : 0.0;
        }
}

// Hermite index of (t, u, v) with t + u + v <= 3 in a dense 4^3 box
#define HIDX(t, u, v) (((t) * 4 + (u)) * 4 + (v))
#define RIDX5(t, u, v) (((t) * (GRAD_LMAX + 1) + (u)) * (GRAD_LMAX + 1) + (v))

struct GradParams {
    dftk_shells_t sh;
    const int *shell_atom;
    const int *ab[3];
    const double *q[3];
    int n_pairs[3];
    long long n_rows[DFTK_N_QCLASS];
    long long total[DFTK_N_QCLASS];
    const long long *row_off[DFTK_N_QCLASS];
    const double *D, *Da, *Db;  // total and spin densities (Da == Db for RHF)
    const float *Dsh;
    int N, ns;
    double tau;
    double *grad;  // [n_atoms * 3], accumulated
};

// Bra-side pass: g_A and g_B of one shell quartet.
__device__ void grad_quartet_bra(const GradParams &P, int a, int b, int c, int d, const double *G, double *gA,
                                 double *gB)
{
    const dftk_shells_t &sh = P.sh;
    const int la = sh.l[a], lb = sh.l[b], lc = sh.l[c], ld = sh.l[d];
    const int na = g_ncomp(la), nb = g_ncomp(lb), nc = g_ncomp(lc), nd = g_ncomp(ld);
    const int Lab = la + lb + 1;  // bra Hermite order after differentiation
    const int L = la + lb + lc + ld + 1;
    const double *A = sh.xyz + 3 * a, *B = sh.xyz + 3 * b, *C = sh.xyz + 3 * c, *Dd = sh.xyz + 3 * d;
    for (int k = 0; k < 3; ++k) gA[k] = gB[k] = 0.0;
    for (int ia = 0; ia < sh.nprim[a]; ++ia)
        for (int ib = 0; ib < sh.nprim[b]; ++ib) {
            const double al = sh.prim_exp[sh.prim_off[a] + ia], be = sh.prim_exp[sh.prim_off[b] + ib];
            const double cab = sh.prim_cn[sh.prim_off[a] + ia] * sh.prim_cn[sh.prim_off[b] + ib];
            const double p = al + be;
            double Pc[3], Eab[3][45];
            for (int x = 0; x < 3; ++x) {
                Pc[x] = (al * A[x] + be * B[x]) / p;
                g_E_table(al, be, A[x], B[x], Eab[x]);
            }
            // H[n][tuv] = sum over ket primitives and components m of
            //             Gamma[n][m] sum_tau (-1)^tau E^m_tau R_{t+tau}
            double H[9 * 64];
            for (int i = 0; i < na * nb * 64; ++i) H[i] = 0.0;
            for (int ic = 0; ic < sh.nprim[c]; ++ic)
                for (int id = 0; id < sh.nprim[d]; ++id) {
                    const double ga = sh.prim_exp[sh.prim_off[c] + ic], de = sh.prim_exp[sh.prim_off[d] + id];
                    const double ccd = sh.prim_cn[sh.prim_off[c] + ic] * sh.prim_cn[sh.prim_off[d] + id];
                    const double qq = ga + de;
                    double Qc[3], Ecd[3][45];
                    for (int x = 0; x < 3; ++x) {
                        Qc[x] = (ga * C[x] + de * Dd[x]) / qq;
                        g_E_table(ga, de, C[x], Dd[x], Ecd[x]);
                    }
                    const double rho = p * qq / (p + qq);
                    const double pre = 2.0 * DFTK_PI * DFTK_PI * sqrt(DFTK_PI) / (p * qq * sqrt(p + qq)) * cab * ccd;
                    double R[(GRAD_LMAX + 1) * (GRAD_LMAX + 1) * (GRAD_LMAX + 1)];
                    herm_R<GRAD_LMAX>(L, rho, Pc[0] - Qc[0], Pc[1] - Qc[1], Pc[2] - Qc[2], R);
                    for (int kc = 0; kc < nc; ++kc)
                        for (int kd = 0; kd < nd; ++kd) {
                            int pc[3], pd[3];
                            g_pow(lc, kc, pc);
                            g_pow(ld, kd, pd);
                            double Tt[64];
                            for (int t = 0; t <= Lab; ++t)
                                for (int u = 0; u + t <= Lab; ++u)
                                    for (int v = 0; v + u + t <= Lab; ++v) {
                                        double s = 0.0;
                                        for (int tx = 0; tx <= pc[0] + pd[0]; ++tx)
                                            for (int ty = 0; ty <= pc[1] + pd[1]; ++ty)
                                                for (int tz = 0; tz <= pc[2] + pd[2]; ++tz) {
                                                    const double e = Ecd[0][(pc[0] * 3 + pd[0]) * 5 + tx] *
                                                                     Ecd[1][(pc[1] * 3 + pd[1]) * 5 + ty] *
                                                                     Ecd[2][(pc[2] * 3 + pd[2]) * 5 + tz];
                                                    const double sg = ((tx + ty + tz) & 1) ? -1.0 : 1.0;
                                                    s += sg * e * R[RIDX5(t + tx, u + ty, v + tz)];
                                                }
                                        Tt[HIDX(t, u, v)] = s * pre;
                                    }
                            const int m = kc * nd + kd;
                            for (int n = 0; n < na * nb; ++n) {
                                const double g = G[n * 9 + m];
                                if (g == 0.0) continue;
                                for (int t = 0; t <= Lab; ++t)
                                    for (int u = 0; u + t <= Lab; ++u)
                                        for (int v = 0; v + u + t <= Lab; ++v)
                                            H[n * 64 + HIDX(t, u, v)] += g * Tt[HIDX(t, u, v)];
                            }
                        }
                }
            // contract with the exponent-shifted bra E coefficients
            for (int ka = 0; ka < na; ++ka)
                for (int kb = 0; kb < nb; ++kb) {
                    int pa[3], pb[3];
                    g_pow(la, ka, pa);
                    g_pow(lb, kb, pb);
                    const double *Hn = H + (ka * nb + kb) * 64;
                    for (int dir = 0; dir < 3; ++dir)
                        for (int side = 0; side < 2; ++side) {
                            double s = 0.0;
                            for (int t = 0; t <= Lab; ++t)
                                for (int u = 0; u + t <= Lab; ++u)
                                    for (int v = 0; v + u + t <= Lab; ++v) {
                                        const int tt[3] = {t, u, v};
                                        double e = 1.0;
                                        for (int x = 0; x < 3 && e != 0.0; ++x) {
                                            const int i = pa[x], j = pb[x];
                                            double f;
                                            if (x != dir) {
                                                f = Eab[x][(i * 3 + j) * 5 + tt[x]];
                                            } else if (side == 0) {
                                                f = 2.0 * al * Eab[x][((i + 1) * 3 + j) * 5 + tt[x]];
                                                if (i > 0) f -= i * Eab[x][((i - 1) * 3 + j) * 5 + tt[x]];
                                            } else {
                                                f = 2.0 * be * Eab[x][(i * 3 + j + 1) * 5 + tt[x]];
                                                if (j > 0) f -= j * Eab[x][(i * 3 + j - 1) * 5 + tt[x]];
                                            }
                                            e *= f;
                                        }
                                        s += e * Hn[HIDX(t, u, v)];
                                    }
                            if (side == 0) gA[dir] += s; else gB[dir] += s;
                        }
                }
        }
}

// Ket-side pass: g_C of one shell quartet (mirror image of the bra pass).
__device__ void grad_quartet_ket(const GradParams &P, int a, int b, int c, int d, const double *G, double *gC)
{
    const dftk_shells_t &sh = P.sh;
    const int la = sh.l[a], lb = sh.l[b], lc = sh.l[c], ld = sh.l[d];
    const int na = g_ncomp(la), nb = g_ncomp(lb), nc = g_ncomp(lc), nd = g_ncomp(ld);
    const int Lcd = lc + ld + 1;
    const int L = la + lb + lc + ld + 1;
    const double *A = sh.xyz + 3 * a, *B = sh.xyz + 3 * b, *C = sh.xyz + 3 * c, *Dd = sh.xyz + 3 * d;
    for (int k = 0; k < 3; ++k) gC[k] = 0.0;
    for (int ic = 0; ic < sh.nprim[c]; ++ic)
        for (int id = 0; id < sh.nprim[d]; ++id) {
            const double ga = sh.prim_exp[sh.prim_off[c] + ic], de = sh.prim_exp[sh.prim_off[d] + id];
            const double ccd = sh.prim_cn[sh.prim_off[c] + ic] * sh.prim_cn[sh.prim_off[d] + id];
            const double qq = ga + de;
            double Qc[3], Ecd[3][45];
            for (int x = 0; x < 3; ++x) {
                Qc[x] = (ga * C[x] + de * Dd[x]) / qq;
                g_E_table(ga, de, C[x], Dd[x], Ecd[x]);
            }
            double H[9 * 64];
            for (int i = 0; i < nc * nd * 64; ++i) H[i] = 0.0;
            for (int ia = 0; ia < sh.nprim[a]; ++ia)
                for (int ib = 0; ib < sh.nprim[b]; ++ib) {
                    const double al = sh.prim_exp[sh.prim_off[a] + ia], be = sh.prim_exp[sh.prim_off[b] + ib];
                    const double cab = sh.prim_cn[sh.prim_off[a] + ia] * sh.prim_cn[sh.prim_off[b] + ib];
                    const double p = al + be;
                    double Pc[3], Eab[3][45];
                    for (int x = 0; x < 3; ++x) {
                        Pc[x] = (al * A[x] + be * B[x]) / p;
                        g_E_table(al, be, A[x], B[x], Eab[x]);
                    }
                    const double rho = p * qq / (p + qq);
                    const double pre = 2.0 * DFTK_PI * DFTK_PI * sqrt(DFTK_PI) / (p * qq * sqrt(p + qq)) * cab * ccd;
                    double R[(GRAD_LMAX + 1) * (GRAD_LMAX + 1) * (GRAD_LMAX + 1)];
                    herm_R<GRAD_LMAX>(L, rho, Pc[0] - Qc[0], Pc[1] - Qc[1], Pc[2] - Qc[2], R);
                    for (int ka = 0; ka < na; ++ka)
                        for (int kb = 0; kb < nb; ++kb) {
                            int pa[3], pb[3];
                            g_pow(la, ka, pa);
                            g_pow(lb, kb, pb);
                            double Tt[64];
                            for (int t = 0; t <= Lcd; ++t)
                                for (int u = 0; u + t <= Lcd; ++u)
                                    for (int v = 0; v + u + t <= Lcd; ++v) {
                                        double s = 0.0;
                                        for (int tx = 0; tx <= pa[0] + pb[0]; ++tx)
                                            for (int ty = 0; ty <= pa[1] + pb[1]; ++ty)
                                                for (int tz = 0; tz <= pa[2] + pb[2]; ++tz) {
                                                    const double e = Eab[0][(pa[0] * 3 + pb[0]) * 5 + tx] *
                                                                     Eab[1][(pa[1] * 3 + pb[1]) * 5 + ty] *
                                                                     Eab[2][(pa[2] * 3 + pb[2]) * 5 + tz];
                                                    s += e * R[RIDX5(t + tx, u + ty, v + tz)];
                                                }
                                        Tt[HIDX(t, u, v)] = s * pre;
                                    }
                            const int n = ka * nb + kb;
                            for (int m = 0; m < nc * nd; ++m) {
                                const double g = G[n * 9 + m];
                                if (g == 0.0) continue;
                                for (int t = 0; t <= Lcd; ++t)
                                    for (int u = 0; u + t <= Lcd; ++u)
                                        for (int v = 0; v + u + t <= Lcd; ++v)
                                            H[m * 64 + HIDX(t, u, v)] += g * Tt[HIDX(t, u, v)];
                            }
                        }
                }
            for (int kc = 0; kc < nc; ++kc)
                for (int kd = 0; kd < nd; ++kd) {
                    int pc[3], pd[3];
                    g_pow(lc, kc, pc);
                    g_pow(ld, kd, pd);
                    const double *Hm = H + (kc * nd + kd) * 64;
                    for (int dir = 0; dir < 3; ++dir) {
                        double s = 0.0;
                        for (int t = 0; t <= Lcd; ++t)
                            for (int u = 0; u + t <= Lcd; ++u)
                                for (int v = 0; v + u + t <= Lcd; ++v) {
                                    const int tt[3] = {t, u, v};
                                    double e = ((t + u + v) & 1) ? -1.0 : 1.0;
                                    for (int x = 0; x < 3 && e != 0.0; ++x) {
                                        const int i = pc[x], j = pd[x];
                                        double f;
                                        if (x != dir) {
                                            f = Ecd[x][(i * 3 + j) * 5 + tt[x]];
                                        } else {
                                            f = 2.0 * ga * Ecd[x][((i + 1) * 3 + j) * 5 + tt[x]];
                                            if (i > 0) f -= i * Ecd[x][((i - 1) * 3 + j) * 5 + tt[x]];
                                        }
                                        e *= f;
                                    }
                                    s += e * Hm[HIDX(t, u, v)];
                                }
                        gC[dir] += s;
                    }
                }
        }
}

// Two-electron gradient: one thread per Schwarz candidate quartet of class C;
// quartets with Q_ab Q_cd max|D|^2 < tau are skipped.
template <int C>
__global__ void __launch_bounds__(64) k_grad_eri(const GradParams P)
{
    constexpr int bra_pc[6] = {0, 1, 1, 2, 2, 2};
    constexpr int ket_pc[6] = {0, 0, 1, 0, 1, 2};
    const int X = bra_pc[C], Yc = ket_pc[C];
    const long long ncand = P.total[C];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long cand = (long long)blockIdx.x * blockDim.x + threadIdx.x; cand < ncand; cand += stride) {
        const int row = find_row(P.row_off[C], P.n_rows[C], cand);
        const int ket = (int)(cand - P.row_off[C][row]);
        const int a = P.ab[X][2 * row], b = P.ab[X][2 * row + 1];
        const int c = P.ab[Yc][2 * ket], d = P.ab[Yc][2 * ket + 1];
        const int ns = P.ns;
        const float dm = fmaxf(fmaxf(P.Dsh[a * ns + b], P.Dsh[c * ns + d]),
                               fmaxf(fmaxf(P.Dsh[a * ns + c], P.Dsh[a * ns + d]),
                                     fmaxf(P.Dsh[b * ns + c], P.Dsh[b * ns + d])));
        if (P.q[X][row] * P.q[Yc][ket] * (double)dm * (double)dm < P.tau) continue;
        const int N = P.N;
        const int oa = P.sh.ao[a], ob = P.sh.ao[b], oc = P.sh.ao[c], od = P.sh.ao[d];
        const int na = g_ncomp(P.sh.l[a]), nb = g_ncomp(P.sh.l[b]), nc = g_ncomp(P.sh.l[c]), nd = g_ncomp(P.sh.l[d]);
        const int ew = (a == b) + (c == d) + ((X == Yc) && (row == ket));
        const double f = 8.0 / (double)(1 << ew);  // orientations of the unique quartet
        double G[81];
        for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j)
                for (int k = 0; k < nc; ++k)
                    for (int l = 0; l < nd; ++l) {
                        const long long I = oa + i, Jn = ob + j, K = oc + k, Ln = od + l;
                        const double coul = 0.5 * P.D[I * N + Jn] * P.D[K * N + Ln];
                        const double exch = 0.25 * (P.Da[I * N + K] * P.Da[Jn * N + Ln] + P.Db[I * N + K] * P.Db[Jn * N + Ln] +
                                                    P.Da[I * N + Ln] * P.Da[Jn * N + K] + P.Db[I * N + Ln] * P.Db[Jn * N + K]);
                        G[(i * nb + j) * 9 + k * nd + l] = f * (coul - exch);
                    }
        double gA[3], gB[3], gC[3];
        grad_quartet_bra(P, a, b, c, d, G, gA, gB);
        grad_quartet_ket(P, a, b, c, d, G, gC);
        const int at[4] = {P.shell_atom[a], P.shell_atom[b], P.shell_atom[c], P.shell_atom[d]};
        for (int x = 0; x < 3; ++x) {
            atomicAdd(P.grad + 3 * at[0] + x, gA[x]);
            atomicAdd(P.grad + 3 * at[1] + x, gB[x]);
            atomicAdd(P.grad + 3 * at[2] + x, gC[x]);
            atomicAdd(P.grad + 3 * at[3] + x, -(gA[x] + gB[x] + gC[x]));
        }
    }
}

// One-electron gradient: one thread per shell pair (i >= j).  S and T are
// two-centre (d/dB = -d/dA); V is summed over nuclei with d/dC = -(d/dA + d/dB).
__global__ void k_grad_onee(const dftk_shells_t sh, const int *shell_atom, int n_atoms, const double *atom_xyz,
                            const double *atom_z, const double *D, const double *W, double *grad)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npair = (long long)sh.n_shells * (sh.n_shells + 1) / 2;
    if (t >= npair) return;
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)i * (i + 1) / 2 > t) --i;
    while ((long long)(i + 1) * (i + 2) / 2 <= t) ++i;
    const int j = (int)(t - (long long)i * (i + 1) / 2);
    const int la = sh.l[i], lb = sh.l[j];
    if (la > 1 || lb > 1 || la < 0 || lb < 0) return;
    const int na = g_ncomp(la), nb = g_ncomp(lb);
    const int N = sh.n_ao;
    const double fpair = (i == j) ? 1.0 : 2.0;
    const double *A = sh.xyz + 3 * i, *B = sh.xyz + 3 * j;
    double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
    for (int ia = 0; ia < sh.nprim[i]; ++ia)
        for (int ib = 0; ib < sh.nprim[j]; ++ib) {
            const double al = sh.prim_exp[sh.prim_off[i] + ia], be = sh.prim_exp[sh.prim_off[j] + ib];
            const double w = sh.prim_cn[sh.prim_off[i] + ia] * sh.prim_cn[sh.prim_off[j] + ib];
            const double p = al + be;
            const double sq = sqrt(DFTK_PI / p);
            double Pc[3];
            double S1[3][3][4], Eh[3][45];  // 1-D overlaps S(i <= 2, j <= 3); Hermite E (i, j <= 2)
            for (int x = 0; x < 3; ++x) {
                Pc[x] = (al * A[x] + be * B[x]) / p;
                for (int pi = 0; pi <= 2; ++pi)
                    for (int pj = 0; pj <= 3; ++pj) {
                        double e[16];
                        herm_E1d(al, be, A[x], B[x], pi, pj, e);
                        S1[x][pi][pj] = e[0] * sq;
                    }
                g_E_table(al, be, A[x], B[x], Eh[x]);
            }
            // 1-D kinetic T(i, j) = b(2j+1) S(i,j) - 2b^2 S(i,j+2) - j(j-1)/2 S(i,j-2), j <= 1
            auto T1 = [&](int x, int pi, int pj) {
                double v = be * (2 * pj + 1) * S1[x][pi][pj] - 2.0 * be * be * S1[x][pi][pj + 2];
                if (pj >= 2) v -= 0.5 * pj * (pj - 1) * S1[x][pi][pj - 2];
                return v;
            };
            for (int ka = 0; ka < na; ++ka)
                for (int kb = 0; kb < nb; ++kb) {
                    int pa[3], pb[3];
                    g_pow(la, ka, pa);
                    g_pow(lb, kb, pb);
                    const long long mu = sh.ao[i] + ka, nu = sh.ao[j] + kb;
                    const double Dm = fpair * w * D[mu * N + nu], Wm = fpair * w * W[mu * N + nu];
                    double Sx[3], Tx[3];
                    for (int x = 0; x < 3; ++x) {
                        Sx[x] = S1[x][pa[x]][pb[x]];
                        Tx[x] = T1(x, pa[x], pb[x]);
                    }
                    for (int dir = 0; dir < 3; ++dir) {
                        const int ii = pa[dir], jj = pb[dir];
                        const double dS = 2.0 * al * S1[dir][ii + 1][jj] - (ii > 0 ? ii * S1[dir][ii - 1][jj] : 0.0);
                        const double dT = 2.0 * al * T1(dir, ii + 1, jj) - (ii > 0 ? ii * T1(dir, ii - 1, jj) : 0.0);
                        const int o1 = (dir + 1) % 3, o2 = (dir + 2) % 3;
                        const double dSfull = dS * Sx[o1] * Sx[o2];
                        const double dTfull = dT * Sx[o1] * Sx[o2] + dS * (Tx[o1] * Sx[o2] + Sx[o1] * Tx[o2]);
                        gA[dir] += Dm * dTfull - Wm * dSfull;
                        gB[dir] -= Dm * dTfull - Wm * dSfull;
                    }
                    const int L = la + lb + 1;
                    for (int cnuc = 0; cnuc < n_atoms; ++cnuc) {
                        double R[(GRAD_LMAX + 1) * (GRAD_LMAX + 1) * (GRAD_LMAX + 1)];
                        herm_R<GRAD_LMAX>(L, p, Pc[0] - atom_xyz[3 * cnuc], Pc[1] - atom_xyz[3 * cnuc + 1],
                                          Pc[2] - atom_xyz[3 * cnuc + 2], R);
                        const double pref = -2.0 * DFTK_PI / p * atom_z[cnuc] * Dm;
                        double dA[3], dB[3];
                        for (int dir = 0; dir < 3; ++dir)
                            for (int side = 0; side < 2; ++side) {
                                double s = 0.0;
                                for (int tx = 0; tx <= L; ++tx)
                                    for (int ty = 0; ty + tx <= L; ++ty)
                                        for (int tz = 0; tz + ty + tx <= L; ++tz) {
                                            const int tt[3] = {tx, ty, tz};
                                            double e = 1.0;
                                            for (int x = 0; x < 3 && e != 0.0; ++x) {
                                                const int ii = pa[x], jj = pb[x];
                                                double f;
                                                if (x != dir) {
                                                    f = Eh[x][(ii * 3 + jj) * 5 + tt[x]];
                                                } else if (side == 0) {
                                                    f = 2.0 * al * Eh[x][((ii + 1) * 3 + jj) * 5 + tt[x]];
                                                    if (ii > 0) f -= ii * Eh[x][((ii - 1) * 3 + jj) * 5 + tt[x]];
                                                } else {
                                                    f = 2.0 * be * Eh[x][(ii * 3 + jj + 1) * 5 + tt[x]];
                                                    if (jj > 0) f -= jj * Eh[x][(ii * 3 + jj - 1) * 5 + tt[x]];
                                                }
                                                e *= f;
                                            }
                                            s += e * R[RIDX5(tx, ty, tz)];
                                        }
                                (side == 0 ? dA : dB)[dir] = pref * s;
                            }
                        for (int dir = 0; dir < 3; ++dir) {
                            gA[dir] += dA[dir];
                            gB[dir] += dB[dir];
                            atomicAdd(grad + 3 * cnuc + dir, -(dA[dir] + dB[dir]));
                        }
                    }
                }
        }
    for (int dir = 0; dir < 3; ++dir) {
        atomicAdd(grad + 3 * shell_atom[i] + dir, gA[dir]);
        atomicAdd(grad + 3 * shell_atom[j] + dir, gB[dir]);
    }
}
