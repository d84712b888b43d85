// One-electron integrals and the drop-in replacements of the reference's
// nuclear_kernel / eri_kernel.
#pragma once

#include "generic.cuh"

__device__ __forceinline__ void cart_comp(int l, int k, int *pw)
{
    // combinations(l) order (shelled.py:15-23): s; p = x, y, z
    if (l == 0) { pw[0] = pw[1] = pw[2] = 0; return; }
    pw[0] = (k == 0); pw[1] = (k == 1); pw[2] = (k == 2);
}

// S, T, V for shell pair t = (i, j), j <= i: MD overlap E^{ij}_0 sqrt(pi/p)
// per axis, kinetic by the l +- 2 rule of T_raw (shelled.py:149-155) halved
// with sign (shelled.py:998), V = -(2 pi / p) sum_C Z_C sum E_t E_u E_v R_tuv
// (nuclear_kernel, shelled.py:420-436), contracted with coefficient x norm.
__global__ void k_one_electron(const dftk_shells_t sh, int n_atoms, const double *atom_xyz,
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
    if (la > 1 || lb > 1 || la < 0 || lb < 0) return;  // s and p only; blocks left untouched
    // a batch: pairs within one molecule, with that molecule's nuclei
    int atom0 = 0, natom = n_atoms;
    if (sh.mol) {
        const int mi = sh.mol[i];
        if (sh.mol[j] != mi) return;
        atom0 = sh.mol_atom0[mi];
        natom = sh.mol_natom[mi];
    }
    const MolView mv = mol_view(sh, i);
    const int ca = (la + 1) * (la + 2) / 2, cb = (lb + 1) * (lb + 2) / 2;
    const int N = mv.nao;
    const double A[3] = {sh.xyz[3 * i], sh.xyz[3 * i + 1], sh.xyz[3 * i + 2]};
    const double B[3] = {sh.xyz[3 * j], sh.xyz[3 * j + 1], sh.xyz[3 * j + 2]};
    double s_acc[3][3], t_acc[3][3], v_acc[3][3];
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) s_acc[x][y] = t_acc[x][y] = v_acc[x][y] = 0.0;
    for (int ia = 0; ia < sh.nprim[i]; ++ia)
        for (int ib = 0; ib < sh.nprim[j]; ++ib) {
            const double al = sh.prim_exp[sh.prim_off[i] + ia], be = sh.prim_exp[sh.prim_off[j] + ib];
            const double w = sh.prim_cn[sh.prim_off[i] + ia] * sh.prim_cn[sh.prim_off[j] + ib];
            const double p = al + be;
            const double sq = sqrt(DFTK_PI / p);
            double Pc[3];
            for (int x = 0; x < 3; ++x) Pc[x] = (al * A[x] + be * B[x]) / p;
            // per-axis overlaps S(la_x, lb_x + k), k = -2..2 (stored at k+2)
            double ov[3][2][5];   // [axis][a power][b power 0..4]
            double eh[3][2][2][3];  // Hermite E^{a,b}_t per axis for V
            for (int x = 0; x < 3; ++x) {
                for (int pa = 0; pa <= 1; ++pa)
                    for (int pb = 0; pb <= 3; ++pb) {
                        double E[16];
                        herm_E1d(al, be, A[x], B[x], pa, pb, E);
                        ov[x][pa][pb] = E[0] * sq;
                        if (pb <= 1)
                            for (int tt = 0; tt < 3; ++tt) eh[x][pa][pb][tt] = tt <= pa + pb ? E[tt] : 0.0;
                    }
            }
            // V needs R up to L = la + lb per pair; sum over nuclei
            double Rv[27];
            double vv[3][3];
            for (int x = 0; x < 3; ++x)
                for (int y = 0; y < 3; ++y) vv[x][y] = 0.0;
            const int L = la + lb;
            for (int c = atom0; c < atom0 + natom; ++c) {
                double R[27];
                herm_R<2>(L, p, Pc[0] - atom_xyz[3 * c], Pc[1] - atom_xyz[3 * c + 1],
                          Pc[2] - atom_xyz[3 * c + 2], R);
                for (int k = 0; k < 27; ++k) Rv[k] = R[k];
                for (int ka = 0; ka < ca; ++ka)
                    for (int kb = 0; kb < cb; ++kb) {
                        int pa[3], pb[3];
                        cart_comp(la, ka, pa);
                        cart_comp(lb, kb, pb);
                        double s = 0.0;
                        for (int tx = 0; tx <= pa[0] + pb[0]; ++tx)
                            for (int ty = 0; ty <= pa[1] + pb[1]; ++ty)
                                for (int tz = 0; tz <= pa[2] + pb[2]; ++tz)
                                    s += eh[0][pa[0]][pb[0]][tx] * eh[1][pa[1]][pb[1]][ty] *
                                         eh[2][pa[2]][pb[2]][tz] * Rv[(tx * 3 + ty) * 3 + tz];
                        vv[ka][kb] += atom_z[c] * s;
                    }
            }
            for (int ka = 0; ka < ca; ++ka)
                for (int kb = 0; kb < cb; ++kb) {
                    int pa[3], pb[3];
                    cart_comp(la, ka, pa);
                    cart_comp(lb, kb, pb);
                    double o[3], k[3];
                    for (int x = 0; x < 3; ++x) {
                        const int a_ = pa[x], b_ = pb[x];
                        o[x] = ov[x][a_][b_];
                        k[x] = be * (2 * b_ + 1) * ov[x][a_][b_] - 2.0 * be * be * ov[x][a_][b_ + 2] -
                               (b_ >= 2 ? 0.5 * b_ * (b_ - 1) * ov[x][a_][b_ - 2] : 0.0);
                    }
                    s_acc[ka][kb] += w * o[0] * o[1] * o[2];
                    t_acc[ka][kb] += w * (k[0] * o[1] * o[2] + o[0] * k[1] * o[2] + o[0] * o[1] * k[2]);
                    v_acc[ka][kb] += w * (-2.0 * DFTK_PI / p) * vv[ka][kb];
                }
        }
    const int oi = sh.ao[i], oj = sh.ao[j];
    for (int ka = 0; ka < ca; ++ka)
        for (int kb = 0; kb < cb; ++kb) {
            const long long r = mv.mat + (long long)(oi + ka) * N + oj + kb, c = mv.mat + (long long)(oj + kb) * N + oi + ka;
            S[r] = s_acc[ka][kb]; S[c] = s_acc[ka][kb];
            T[r] = t_acc[ka][kb]; T[c] = t_acc[ka][kb];
            V[r] = v_acc[ka][kb]; V[c] = v_acc[ka][kb];
        }
}

// Drop-in for the reference's nuclear_kernel (shelled.py:350-450): same
// arguments, one thread per primitive-component pair q = a * num_funcs_b + b.
__global__ void k_nuclear_dropin(const double *exp_a, const double *exp_b, const double *cen_a,
                                 const double *cen_b, const int *pow_a, const int *pow_b,
                                 const int *atoms, const double *atom_centers, int num_atoms,
                                 int num_funcs_a, int num_funcs_b, double *V_out, double *Ex_out,
                                 double *Ey_out, double *Ez_out, double *p_out, double *P_out,
                                 int *nx_out, int *ny_out, int *nz_out)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)num_funcs_a * num_funcs_b) return;
    const int a = (int)(q / num_funcs_b), b = (int)(q % num_funcs_b);
    const double al = exp_a[a], be = exp_b[b];
    double E[3][16];
    int len[3];
    bool ok = true;
    for (int x = 0; x < 3; ++x) {
        const int la = pow_a[3 * a + x], lb = pow_b[3 * b + x];
        ok = ok && la >= 0 && lb >= 0 && la + lb < DFTK_E_SLOTS;
    }
    for (int x = 0; x < 3; ++x) {
        const int la = ok ? pow_a[3 * a + x] : 0, lb = ok ? pow_b[3 * b + x] : 0;
        herm_E1d(al, be, cen_a[x], cen_b[x], la, lb, E[x]);
        len[x] = la + lb + 1;
        for (int t = len[x]; t < 16; ++t) E[x][t] = 0.0;
    }
    const double p = al + be;
    const double Px = (al * cen_a[0] + be * cen_b[0]) / p;
    const double Py = (al * cen_a[1] + be * cen_b[1]) / p;
    const double Pz = (al * cen_a[2] + be * cen_b[2]) / p;
    const int L = len[0] + len[1] + len[2] - 3;
    double value = 0.0;
    if (ok && L <= DFTK_GENERIC_LMAX) {
        constexpr int D = DFTK_GENERIC_LMAX + 1;
        for (int c = 0; c < num_atoms; ++c) {
            double R[D * D * D];
            herm_R<DFTK_GENERIC_LMAX>(L, p, Px - atom_centers[3 * c], Py - atom_centers[3 * c + 1],
                                      Pz - atom_centers[3 * c + 2], R);
            double s = 0.0;
            for (int t = 0; t < len[0]; ++t)
                for (int u = 0; u < len[1]; ++u)
                    for (int v = 0; v < len[2]; ++v) s += E[0][t] * E[1][u] * E[2][v] * R[(t * D + u) * D + v];
            value += atoms[c] * s;
        }
        value *= -2.0 * DFTK_PI / p;
    } else {
        value = __longlong_as_double(0x7ff8000000000000ULL);  // beyond the supported order
    }
    V_out[q] = value;
    for (int t = 0; t < DFTK_E_SLOTS; ++t) {
        Ex_out[q * DFTK_E_SLOTS + t] = E[0][t];
        Ey_out[q * DFTK_E_SLOTS + t] = E[1][t];
        Ez_out[q * DFTK_E_SLOTS + t] = E[2][t];
    }
    p_out[q] = p;
    P_out[3 * q] = Px; P_out[3 * q + 1] = Py; P_out[3 * q + 2] = Pz;
    nx_out[q] = len[0]; ny_out[q] = len[1]; nz_out[q] = len[2];
}

// Drop-in for the reference's eri_kernel (shelled.py:452-532): same arguments,
// one thread per primitive quartet q = i * K_cd + j.
__global__ void k_eri_dropin(int K_ab, const double *p_ab, const double *P_ab, const double *Exab,
                             const double *Eyab, const double *Ezab, const int *nxab,
                             const int *nyab, const int *nzab, int K_cd, const double *p_cd,
                             const double *P_cd, const double *Excd, const double *Eycd,
                             const double *Ezcd, const int *nxcd, const int *nycd, const int *nzcd,
                             double *out)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)K_ab * K_cd) return;
    const int i = (int)(q / K_cd), j = (int)(q % K_cd);
    const int ni[3] = {nxab[i], nyab[i], nzab[i]}, nj[3] = {nxcd[j], nycd[j], nzcd[j]};
    const double *Ei[3] = {Exab + DFTK_E_SLOTS * i, Eyab + DFTK_E_SLOTS * i, Ezab + DFTK_E_SLOTS * i};
    const double *Ej[3] = {Excd + DFTK_E_SLOTS * j, Eycd + DFTK_E_SLOTS * j, Ezcd + DFTK_E_SLOTS * j};
    int len[3];
    bool ok = true;
    for (int x = 0; x < 3; ++x) {
        len[x] = ni[x] + nj[x] - 1;
        ok = ok && ni[x] >= 1 && nj[x] >= 1 && ni[x] <= DFTK_E_SLOTS && nj[x] <= DFTK_E_SLOTS;
    }
    const int L = len[0] + len[1] + len[2] - 3;
    if (!ok || L > DFTK_GENERIC_LMAX) {
        out[q] = __longlong_as_double(0x7ff8000000000000ULL);
        return;
    }
    const double pi_ = p_ab[i], pj = p_cd[j];
    const double rho = pi_ * pj / (pi_ + pj);
    constexpr int D = DFTK_GENERIC_LMAX + 1;
    double R[D * D * D];
    herm_R<DFTK_GENERIC_LMAX>(L, rho, P_ab[3 * i] - P_cd[3 * j], P_ab[3 * i + 1] - P_cd[3 * j + 1],
                              P_ab[3 * i + 2] - P_cd[3 * j + 2], R);
    double Cc[3][2 * DFTK_E_SLOTS];
    for (int x = 0; x < 3; ++x) {
        for (int s = 0; s < len[x]; ++s) Cc[x][s] = 0.0;
        for (int t = 0; t < ni[x]; ++t)
            for (int k = 0; k < nj[x]; ++k) Cc[x][t + k] += Ei[x][t] * Ej[x][k] * ((k & 1) ? -1.0 : 1.0);
    }
    double sum = 0.0;
    for (int t = 0; t < len[0]; ++t)
        for (int u = 0; u < len[1]; ++u)
            for (int v = 0; v < len[2]; ++v) sum += Cc[0][t] * Cc[1][u] * Cc[2][v] * R[(t * D + u) * D + v];
    out[q] = sum * (2.0 * DFTK_PI * DFTK_PI * sqrt(DFTK_PI)) / (pi_ * pj * sqrt(pi_ + pj));
}

// FMA-pipe microbenchmark: 8 independent chains per thread.
template <typename T>
__global__ void k_fma_burn(int iters, double *sink)
{
    T a[8];
    const T b = (T)0.999999, c = (T)1e-7;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (T)(threadIdx.x + k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = a[k] * b + c;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    sink[(long long)blockIdx.x * blockDim.x + threadIdx.x] = (double)s;
}

template <int L>
__device__ __forceinline__ void boys64_store(double x, double *out)
{
    double f[L + 1];
    Boys<double, L>::eval(x, f);
    for (int m = 0; m <= L; ++m) out[m] = f[m];
}

// F_0..F_mmax through the same unrolled evaluator the ERI kernels use.
__global__ void k_boys_test(int mmax, long long n, const double *T, double *F)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double *o = F + t * (mmax + 1);
    // caller-supplied arguments: T < 0 is evaluated at 0 (the table index
    // stays in range); NaN takes the asymptotic branch and stays NaN
    const double x = T[t] < 0.0 ? 0.0 : T[t];
    switch (mmax) {
    case 0: boys64_store<0>(x, o); break;
    case 1: boys64_store<1>(x, o); break;
    case 2: boys64_store<2>(x, o); break;
    case 3: boys64_store<3>(x, o); break;
    case 4: boys64_store<4>(x, o); break;
    case 5: boys64_store<5>(x, o); break;
    case 6: boys64_store<6>(x, o); break;
    case 7: boys64_store<7>(x, o); break;
    default: boys64_store<8>(x, o); break;
    }
}

template <int L>
__device__ __forceinline__ void boys32_store(float x, float *out)
{
    float f[L + 1];
    Boys<float, L>::eval(x, f);
    for (int m = 0; m <= L; ++m) out[m] = f[m];
}

__global__ void k_boys32_test(int mmax, long long n, const float *T, float *F)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float *o = F + t * (mmax + 1);
    const float x = T[t] < 0.0f ? 0.0f : T[t];
    switch (mmax) {
    case 0: boys32_store<0>(x, o); break;
    case 1: boys32_store<1>(x, o); break;
    case 2: boys32_store<2>(x, o); break;
    case 3: boys32_store<3>(x, o); break;
    case 4: boys32_store<4>(x, o); break;
    case 5: boys32_store<5>(x, o); break;
    case 6: boys32_store<6>(x, o); break;
    case 7: boys32_store<7>(x, o); break;
    default: boys32_store<8>(x, o); break;
    }
}
