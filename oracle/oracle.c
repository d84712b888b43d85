/*
 * oracle.c -- CPU oracle for the Boys / Hermite / ERI / J-K digestion path.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library as the checker.  The product
 * (the dft_b200 package and its libdftk.so) never links, loads or calls it.
 *
 * This is a plain-C restatement of the reference's algorithm (yegor-gondhal/DFT,
 * shelled.py).  Every function names the reference lines it follows.  It is
 * pinned by tests/test_oracle_golden.py against fixtures produced by running
 * the reference itself (tests/golden/make_golden.py).
 *
 * Conventions shared with the reference:
 *   - Cartesian components of a shell come in combinations(l) order
 *     (shelled.py:15-23): x before y before z, e.g. p = x, y, z.
 *   - Primitive index inside a shell = component * n_exp + exponent
 *     (xp.tile / xp.repeat, shelled.py:948-949, :965-968).
 *   - AO index inside a shell = contraction * n_comp + component
 *     (einsum "apbqcrds,ip,jq,kr,ls->iajbkcld", shelled.py:682-689).
 *   - Hermite arrays carry 7 slots per primitive pair (max_e, shelled.py:170).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_E 7
#define ORC_MAXR 2048
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------ Boys */
/* F_m(T) for m = 0..n-1 with the reference's three regimes
 * (shelled.py:174-211): T < 1e-14 -> 1/(2m+1); T < 6 -> 40-term series for
 * the highest order then downward recursion; otherwise F_0 from erf and
 * upward recursion. */
static double orc_boys_series(int m, double T)
{
    double sum = 1.0 / (2.0 * m + 1.0);
    double term = 1.0;
    for (int k = 1; k < 40; ++k) {
        term *= -T / (double)k;
        sum += term / (2.0 * m + 2.0 * k + 1.0);
    }
    return sum;
}

void orc_boys(int n, double T, double *F)
{
    double e = exp(-T);
    if (T < 1e-14) {
        for (int m = 0; m < n; ++m) F[m] = 1.0 / (2.0 * m + 1.0);
        return;
    }
    if (T < 6.0) {
        double f = orc_boys_series(n - 1, T);
        F[n - 1] = f;
        for (int m = n - 2; m >= 0; --m) {
            f = (2.0 * T * f + e) / (2.0 * m + 1);
            F[m] = f;
        }
        return;
    }
    double f = sqrt(ORC_PI) * erf(sqrt(T)) / (2.0 * sqrt(T));
    F[0] = f;
    for (int m = 0; m + 1 < n; ++m) {
        f = ((2.0 * m + 1.0) * f - e) / (2.0 * T);
        F[m + 1] = f;
    }
}

/* --------------------------------------------------------- Hermite E (1-D) */
/* E^{la,lb}_t, t = 0..la+lb, for one Cartesian axis, with the Gaussian
 * product factor exp(-q Q^2) folded into E_0^{00} (shelled.py:228-294):
 * raise a first (X_PA = -beta Q / p), then b (X_PB = alpha Q / p). */
void orc_hermite_E(double alpha, double beta, double A, double B, int la, int lb, double *E)
{
    double cur[ORC_E], nxt[ORC_E];
    double p = alpha + beta;
    double Q = A - B;
    for (int t = 0; t < ORC_E; ++t) { cur[t] = 0.0; E[t] = 0.0; }
    cur[0] = exp(-(alpha * beta / p) * Q * Q);
    int order = 0;
    for (int step = 0; step < la + lb; ++step) {
        double shift = (step < la) ? -(beta * Q / p) : (alpha * Q / p);
        for (int t = 0; t <= order + 1; ++t) {
            double v = 0.0;
            if (t <= order) v += shift * cur[t];
            if (t > 0) v += cur[t - 1] / (2.0 * p);
            if (t + 1 <= order) v += (t + 1) * cur[t + 1];
            nxt[t] = v;
        }
        ++order;
        for (int t = 0; t <= order; ++t) cur[t] = nxt[t];
    }
    for (int t = 0; t <= order; ++t) E[t] = cur[t];
}

/* ------------------------------------------------------------- Hermite R */
/* R^{n}_{tuv} on a dense (nx, ny, nz, nn) box, index ((t*ny+u)*nz+v)*nn+n
 * (shelled.py:172, :296-348): R^{n}_{000} = (-2 param)^n F_n(param |PQ|^2),
 * then recursion on the first non-zero of t, u, v in that order. */
void orc_hermite_R(int nx, int ny, int nz, int nn, double dx, double dy, double dz,
                   double param, double *R)
{
#define RI(t, u, v, n) ((((t) * ny + (u)) * nz + (v)) * nn + (n))
    double F[32];
    double T = param * (dx * dx + dy * dy + dz * dz);
    orc_boys(nn, T, F);
    double s = 1.0;
    for (int n = 0; n < nn; ++n) { R[RI(0, 0, 0, n)] = s * F[n]; s *= -2.0 * param; }
    for (int t = 0; t < nx; ++t)
        for (int u = 0; u < ny; ++u)
            for (int v = 0; v < nz; ++v) {
                if (t == 0 && u == 0 && v == 0) continue;
                int top = nn - (t + u + v);
                for (int n = 0; n < top; ++n) {
                    double r;
                    if (t > 0) {
                        r = dx * R[RI(t - 1, u, v, n + 1)];
                        if (t > 1) r += (t - 1) * R[RI(t - 2, u, v, n + 1)];
                    } else if (u > 0) {
                        r = dy * R[RI(t, u - 1, v, n + 1)];
                        if (u > 1) r += (u - 1) * R[RI(t, u - 2, v, n + 1)];
                    } else {
                        r = dz * R[RI(t, u, v - 1, n + 1)];
                        if (v > 1) r += (v - 1) * R[RI(t, u, v - 2, n + 1)];
                    }
                    R[RI(t, u, v, n)] = r;
                }
            }
#undef RI
}

/* ------------------------------------------------- primitive pair records */
/* Pair data of the reference's nuclear_kernel (shelled.py:350-450): for every
 * primitive pair q = a * nb + b: E^{x,y,z} (7 slots each), p, P, per-axis
 * lengths l_a + l_b + 1 and, if natoms > 0, the primitive nuclear attraction
 * V = -2 pi / p * sum_C Z_C sum_tuv E_t E_u E_v R_tuv(p, P - C). */
void orc_pair_prims(int na, const double *exp_a, const int *pow_a, const double *cen_a,
                    int nb, const double *exp_b, const int *pow_b, const double *cen_b,
                    int natoms, const int *Z, const double *atom_xyz, double *V,
                    double *Ex, double *Ey, double *Ez, double *p_out, double *P_out,
                    int *nx_out, int *ny_out, int *nz_out)
{
    for (int a = 0; a < na; ++a)
        for (int b = 0; b < nb; ++b) {
            long q = (long)a * nb + b;
            double ea = exp_a[a], eb = exp_b[b];
            double ex[ORC_E], ey[ORC_E], ez[ORC_E];
            orc_hermite_E(ea, eb, cen_a[0], cen_b[0], pow_a[3 * a], pow_b[3 * b], ex);
            orc_hermite_E(ea, eb, cen_a[1], cen_b[1], pow_a[3 * a + 1], pow_b[3 * b + 1], ey);
            orc_hermite_E(ea, eb, cen_a[2], cen_b[2], pow_a[3 * a + 2], pow_b[3 * b + 2], ez);
            double p = ea + eb;
            double Px = (ea * cen_a[0] + eb * cen_b[0]) / p;
            double Py = (ea * cen_a[1] + eb * cen_b[1]) / p;
            double Pz = (ea * cen_a[2] + eb * cen_b[2]) / p;
            int lx = pow_a[3 * a] + pow_b[3 * b] + 1;
            int ly = pow_a[3 * a + 1] + pow_b[3 * b + 1] + 1;
            int lz = pow_a[3 * a + 2] + pow_b[3 * b + 2] + 1;
            if (V) {
                double R[ORC_MAXR];
                int nn = lx + ly + lz - 2;
                double acc = 0.0;
                for (int c = 0; c < natoms; ++c) {
                    orc_hermite_R(lx, ly, lz, nn, Px - atom_xyz[3 * c], Py - atom_xyz[3 * c + 1],
                                  Pz - atom_xyz[3 * c + 2], p, R);
                    double s = 0.0;
                    for (int t = 0; t < lx; ++t)
                        for (int u = 0; u < ly; ++u)
                            for (int v = 0; v < lz; ++v)
                                s += ex[t] * ey[u] * ez[v] * R[((t * ly + u) * lz + v) * nn];
                    acc += Z[c] * s;
                }
                V[q] = -2.0 * ORC_PI / p * acc;
            }
            for (int t = 0; t < ORC_E; ++t) {
                Ex[q * ORC_E + t] = ex[t];
                Ey[q * ORC_E + t] = ey[t];
                Ez[q * ORC_E + t] = ez[t];
            }
            p_out[q] = p;
            P_out[3 * q] = Px; P_out[3 * q + 1] = Py; P_out[3 * q + 2] = Pz;
            nx_out[q] = lx; ny_out[q] = ly; nz_out[q] = lz;
        }
}

/* ----------------------------------------------------- primitive ERIs */
/* One primitive x component quartet (shelled.py:452-532): ket-signed
 * convolution of the 1-D Hermite coefficients per axis, contraction with
 * R_{tuv}^{0}, times 2 pi^{5/2} / (p q sqrt(p + q)). */
static double orc_eri_one(double pi, const double *Pi, const double *exi, const double *eyi,
                          const double *ezi, int nxi, int nyi, int nzi,
                          double pj, const double *Pj, const double *exj, const double *eyj,
                          const double *ezj, int nxj, int nyj, int nzj, double *R)
{
    int lx = nxi + nxj - 1, ly = nyi + nyj - 1, lz = nzi + nzj - 1;
    int nn = lx + ly + lz - 2;
    double rho = pi * pj / (pi + pj);
    orc_hermite_R(lx, ly, lz, nn, Pi[0] - Pj[0], Pi[1] - Pj[1], Pi[2] - Pj[2], rho, R);
    double cx[16], cy[16], cz[16];
    for (int s = 0; s < lx; ++s) cx[s] = 0.0;
    for (int s = 0; s < ly; ++s) cy[s] = 0.0;
    for (int s = 0; s < lz; ++s) cz[s] = 0.0;
    for (int t = 0; t < nxi; ++t)
        for (int k = 0; k < nxj; ++k) cx[t + k] += exi[t] * exj[k] * ((k & 1) ? -1.0 : 1.0);
    for (int t = 0; t < nyi; ++t)
        for (int k = 0; k < nyj; ++k) cy[t + k] += eyi[t] * eyj[k] * ((k & 1) ? -1.0 : 1.0);
    for (int t = 0; t < nzi; ++t)
        for (int k = 0; k < nzj; ++k) cz[t + k] += ezi[t] * ezj[k] * ((k & 1) ? -1.0 : 1.0);
    double sum = 0.0;
    for (int t = 0; t < lx; ++t)
        for (int u = 0; u < ly; ++u) {
            double cxy = cx[t] * cy[u];
            for (int v = 0; v < lz; ++v) sum += cxy * cz[v] * R[((t * ly + u) * lz + v) * nn];
        }
    double pre = 2.0 * ORC_PI * ORC_PI * sqrt(ORC_PI);
    return sum * pre / (pi * pj * sqrt(pi + pj));
}

/* Primitive ERIs of one shell quartet from two pair records (the reference's
 * eri_kernel launch, shelled.py:640-662): out[i * K_cd + j]. */
void orc_eri_prims(int K_ab, const double *p_ab, const double *P_ab, const double *Exab,
                   const double *Eyab, const double *Ezab, const int *nxab, const int *nyab,
                   const int *nzab, int K_cd, const double *p_cd, const double *P_cd,
                   const double *Excd, const double *Eycd, const double *Ezcd, const int *nxcd,
                   const int *nycd, const int *nzcd, double *out)
{
    double R[ORC_MAXR];
    for (int i = 0; i < K_ab; ++i)
        for (int j = 0; j < K_cd; ++j)
            out[(long)i * K_cd + j] = orc_eri_one(
                p_ab[i], P_ab + 3 * i, Exab + ORC_E * i, Eyab + ORC_E * i, Ezab + ORC_E * i,
                nxab[i], nyab[i], nzab[i], p_cd[j], P_cd + 3 * j, Excd + ORC_E * j,
                Eycd + ORC_E * j, Ezcd + ORC_E * j, nxcd[j], nycd[j], nzcd[j], R);
}

/* ------------------------------------------------------------ shells */
typedef struct {
    int ns;
    const double *center;  /* 3 * ns */
    const int *l;          /* angular momentum */
    const int *nexp;       /* primitives per shell */
    const int *ncontr;     /* contractions per shell */
    const int *exp_off;    /* offset into exps */
    const int *coef_off;   /* offset into coefs (ncontr x nexp, row-major) */
    const int *ao;         /* first AO of the shell */
    const double *exps;
    const double *coefs;
} OrcShells;

static int orc_ncomp(int l) { return (l + 1) * (l + 2) / 2; }

/* combinations(l), shelled.py:15-23 */
static void orc_components(int l, int *pow)
{
    int k = 0;
    for (int n = 0; n <= l; ++n)
        for (int m = 0; m <= l; ++m)
            for (int i = 0; i <= l; ++i)
                if (i + m + n == l) { pow[3 * k] = i; pow[3 * k + 1] = m; pow[3 * k + 2] = n; ++k; }
}

static double orc_dfact(int n) /* (n)!! with (-1)!! = 1 */
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

/* normal(alpha, pow), shelled.py:95-101 */
static double orc_norm(double alpha, const int *pw)
{
    int L = pw[0] + pw[1] + pw[2];
    double t = pow(4.0 * alpha, L) /
               (orc_dfact(2 * pw[0] - 1) * orc_dfact(2 * pw[1] - 1) * orc_dfact(2 * pw[2] - 1));
    return sqrt(t) * pow(2.0 * alpha / ORC_PI, 0.75);
}

int orc_shell_nao(const OrcShells *S, int s) { return orc_ncomp(S->l[s]) * S->ncontr[s]; }

/* Primitive records of the ordered shell pair (a, b), like the reference's
 * per-pair nuclear_kernel launch (shelled.py:1000-1036) minus V. */
typedef struct {
    int K;
    double *p, *P, *Ex, *Ey, *Ez;
    int *nx, *ny, *nz;
    double *norm; /* normalisation product per primitive pair */
} OrcPair;

static void orc_pair_build(const OrcShells *S, int a, int b, OrcPair *pr)
{
    int ca = orc_ncomp(S->l[a]), cb = orc_ncomp(S->l[b]);
    int ea = S->nexp[a], eb = S->nexp[b];
    int na = ca * ea, nb = cb * eb;
    int powa[3 * 28], powb[3 * 28];
    double expa[256], expb[256], nrma[256], nrmb[256];
    int pa[3 * 256], pb[3 * 256];
    orc_components(S->l[a], powa);
    orc_components(S->l[b], powb);
    for (int c = 0; c < ca; ++c)
        for (int e = 0; e < ea; ++e) {
            int i = c * ea + e;
            expa[i] = S->exps[S->exp_off[a] + e];
            pa[3 * i] = powa[3 * c]; pa[3 * i + 1] = powa[3 * c + 1]; pa[3 * i + 2] = powa[3 * c + 2];
            nrma[i] = orc_norm(expa[i], pa + 3 * i);
        }
    for (int c = 0; c < cb; ++c)
        for (int e = 0; e < eb; ++e) {
            int i = c * eb + e;
            expb[i] = S->exps[S->exp_off[b] + e];
            pb[3 * i] = powb[3 * c]; pb[3 * i + 1] = powb[3 * c + 1]; pb[3 * i + 2] = powb[3 * c + 2];
            nrmb[i] = orc_norm(expb[i], pb + 3 * i);
        }
    int K = na * nb;
    pr->K = K;
    pr->p = (double *)malloc(sizeof(double) * K * (1 + 3 + 3 * ORC_E + 1));
    pr->P = pr->p + K;
    pr->Ex = pr->P + 3 * K;
    pr->Ey = pr->Ex + ORC_E * K;
    pr->Ez = pr->Ey + ORC_E * K;
    pr->norm = pr->Ez + ORC_E * K;
    pr->nx = (int *)malloc(sizeof(int) * 3 * K);
    pr->ny = pr->nx + K;
    pr->nz = pr->ny + K;
    orc_pair_prims(na, expa, pa, S->center + 3 * a, nb, expb, pb, S->center + 3 * b, 0, NULL, NULL,
                   NULL, pr->Ex, pr->Ey, pr->Ez, pr->p, pr->P, pr->nx, pr->ny, pr->nz);
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) pr->norm[i * nb + j] = nrma[i] * nrmb[j];
}

static void orc_pair_free(OrcPair *pr)
{
    free(pr->p);
    free(pr->nx);
}

/* Contracted Cartesian block of the shell quartet (ab|cd), layout
 * (n_ao_a, n_ao_b, n_ao_c, n_ao_d) with AO = contraction * n_comp + component
 * (calc_eri, shelled.py:640-691: eri_kernel, normalisation, einsum). */
/* Signature of the reference's host-compiled eri_kernel launch loop
 * (oracle/_ref ref_run_eri_kernel): primitive ERIs from two pair records. */
typedef void (*orc_ref_eri_fn)(long long, int, const double *, const double *, const double *,
                               const double *, const double *, const int *, const int *,
                               const int *, int, const double *, const double *, const double *,
                               const double *, const double *, const int *, const int *,
                               const int *, double *);

static void orc_quartet_block_fn(const OrcShells *S, const OrcPair *ab, const OrcPair *cd,
                                 int a, int b, int c, int d, double *prim, double *out,
                                 orc_ref_eri_fn fn);

static void orc_quartet_block(const OrcShells *S, const OrcPair *ab, const OrcPair *cd,
                              int a, int b, int c, int d, double *prim, double *out)
{
    orc_quartet_block_fn(S, ab, cd, a, b, c, d, prim, out, NULL);
}

static void orc_quartet_block_fn(const OrcShells *S, const OrcPair *ab, const OrcPair *cd,
                                 int a, int b, int c, int d, double *prim, double *out,
                                 orc_ref_eri_fn fn)
{
    if (fn)
        fn((long long)ab->K * cd->K, ab->K, ab->p, ab->P, ab->Ex, ab->Ey, ab->Ez, ab->nx, ab->ny,
           ab->nz, cd->K, cd->p, cd->P, cd->Ex, cd->Ey, cd->Ez, cd->nx, cd->ny, cd->nz, prim);
    else
        orc_eri_prims(ab->K, ab->p, ab->P, ab->Ex, ab->Ey, ab->Ez, ab->nx, ab->ny, ab->nz, cd->K,
                      cd->p, cd->P, cd->Ex, cd->Ey, cd->Ez, cd->nx, cd->ny, cd->nz, prim);
    int cmp[4] = {orc_ncomp(S->l[a]), orc_ncomp(S->l[b]), orc_ncomp(S->l[c]), orc_ncomp(S->l[d])};
    int ne[4] = {S->nexp[a], S->nexp[b], S->nexp[c], S->nexp[d]};
    int nc[4] = {S->ncontr[a], S->ncontr[b], S->ncontr[c], S->ncontr[d]};
    int sh[4] = {a, b, c, d};
    int nao[4];
    for (int k = 0; k < 4; ++k) nao[k] = cmp[k] * nc[k];
    long total = (long)nao[0] * nao[1] * nao[2] * nao[3];
    for (long t = 0; t < total; ++t) out[t] = 0.0;
    int Kb = cmp[1] * ne[1], Kd = cmp[3] * ne[3];
    for (int ia = 0; ia < cmp[0] * ne[0]; ++ia)
        for (int ib = 0; ib < Kb; ++ib)
            for (int ic = 0; ic < cmp[2] * ne[2]; ++ic)
                for (int id = 0; id < Kd; ++id) {
                    int pi = ia * Kb + ib, pj = ic * Kd + id;
                    double v = prim[(long)pi * cd->K + pj] * ab->norm[pi] * cd->norm[pj];
                    int prm[4] = {ia, ib, ic, id};
                    /* split primitive index into (component, exponent) */
                    int comp[4], ex[4];
                    for (int k = 0; k < 4; ++k) { comp[k] = prm[k] / ne[k]; ex[k] = prm[k] % ne[k]; }
                    for (int ka = 0; ka < nc[0]; ++ka) {
                        double va = v * S->coefs[S->coef_off[sh[0]] + ka * ne[0] + ex[0]];
                        int oa = ka * cmp[0] + comp[0];
                        for (int kb = 0; kb < nc[1]; ++kb) {
                            double vb = va * S->coefs[S->coef_off[sh[1]] + kb * ne[1] + ex[1]];
                            int ob = kb * cmp[1] + comp[1];
                            for (int kc = 0; kc < nc[2]; ++kc) {
                                double vc = vb * S->coefs[S->coef_off[sh[2]] + kc * ne[2] + ex[2]];
                                int oc = kc * cmp[2] + comp[2];
                                for (int kd = 0; kd < nc[3]; ++kd) {
                                    double vd = vc * S->coefs[S->coef_off[sh[3]] + kd * ne[3] + ex[3]];
                                    int od = kd * cmp[3] + comp[3];
                                    out[((long)(oa * nao[1] + ob) * nao[2] + oc) * nao[3] + od] += vd;
                                }
                            }
                        }
                    }
                }
}

static OrcShells orc_shells(int ns, const double *center, const int *l, const int *nexp,
                            const int *ncontr, const int *exp_off, const int *coef_off,
                            const int *ao, const double *exps, const double *coefs)
{
    OrcShells S = {ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs};
    return S;
}

/* Contracted ERI blocks of a list of shell quartets quads[4*t..4*t+3];
 * block t is written at out + offsets[t]. */
void orc_eri_quartets(int ns, const double *center, const int *l, const int *nexp,
                      const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                      const double *exps, const double *coefs, long nq, const int *quads,
                      const long *offsets, double *out)
{
    OrcShells S = orc_shells(ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs);
    #pragma omp parallel
    {
        double *prim = (double *)malloc(sizeof(double) * ((size_t)1 << 20));
        #pragma omp for schedule(dynamic, 8)
        for (long t = 0; t < nq; ++t) {
            const int *q = quads + 4 * t;
            OrcPair ab, cd;
            orc_pair_build(&S, q[0], q[1], &ab);
            orc_pair_build(&S, q[2], q[3], &cd);
            orc_quartet_block(&S, &ab, &cd, q[0], q[1], q[2], q[3], prim, out + offsets[t]);
            orc_pair_free(&ab);
            orc_pair_free(&cd);
        }
        free(prim);
    }
}

/* ------------------------------------------------------------ J/K digestion */
/* fill_matrices (shelled.py:770-877): each unique quartet contributes in its 8
 * orientations (shelled.py:791-800), each divided by the duplicate weight
 * 2^{[a=b] + [c=d] + [ab=cd]} (shelled.py:826-831):
 *   J[s0, s1] += sum eri * P[s2, s3],  K_sigma[s0, s2] += sum eri * P_sigma[s1, s3]. */
static void orc_digest_one(const OrcShells *S, const int *q, const double *blk, int N,
                           const double *P, const double *Pa, const double *Pb, double *J,
                           double *Ka, double *Kb)
{
    static const int orient[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                                     {2, 3, 0, 1}, {3, 2, 0, 1}, {2, 3, 1, 0}, {3, 2, 1, 0}};
    int nao[4], ao0[4];
    for (int k = 0; k < 4; ++k) { nao[k] = orc_shell_nao(S, q[k]); ao0[k] = S->ao[q[k]]; }
    int pw = (q[0] == q[1]) + (q[2] == q[3]) + (q[0] == q[2] && q[1] == q[3]);
    double inv_w = 1.0 / (double)(1 << pw);
    int idx[4];
    for (idx[0] = 0; idx[0] < nao[0]; ++idx[0])
        for (idx[1] = 0; idx[1] < nao[1]; ++idx[1])
            for (idx[2] = 0; idx[2] < nao[2]; ++idx[2])
                for (idx[3] = 0; idx[3] < nao[3]; ++idx[3]) {
                    double v = blk[((idx[0] * nao[1] + idx[1]) * nao[2] + idx[2]) * nao[3] + idx[3]] * inv_w;
                    for (int o = 0; o < 8; ++o) {
                        int s0 = ao0[orient[o][0]] + idx[orient[o][0]];
                        int s1 = ao0[orient[o][1]] + idx[orient[o][1]];
                        int s2 = ao0[orient[o][2]] + idx[orient[o][2]];
                        int s3 = ao0[orient[o][3]] + idx[orient[o][3]];
                        J[s0 * N + s1] += v * P[s2 * N + s3];
                        Ka[s0 * N + s2] += v * Pa[s1 * N + s3];
                        Kb[s0 * N + s2] += v * Pb[s1 * N + s3];
                    }
                }
}

static void orc_reduce(int nthreads, long NN, double *acc, double *J, double *Ka, double *Kb)
{
    for (int t = 0; t < nthreads; ++t) {
        double *aj = acc + (long)t * 3 * NN;
        for (long i = 0; i < NN; ++i) { J[i] += aj[i]; Ka[i] += aj[NN + i]; Kb[i] += aj[2 * NN + i]; }
    }
}

/* Digest stored blocks (the reference's stored-ERI fill_matrices). */
void orc_fill_matrices(int ns, const double *center, const int *l, const int *nexp,
                       const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                       const double *exps, const double *coefs, long nq, const int *quads,
                       const long *offsets, const double *values, int N, const double *P,
                       const double *Pa, const double *Pb, double *J, double *Ka, double *Kb)
{
    OrcShells S = orc_shells(ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs);
    long NN = (long)N * N;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    double *acc = (double *)calloc((size_t)nthreads * 3 * NN, sizeof(double));
    #pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *aj = acc + (long)tid * 3 * NN;
        #pragma omp for schedule(dynamic, 64)
        for (long t = 0; t < nq; ++t)
            orc_digest_one(&S, quads + 4 * t, values + offsets[t], N, P, Pa, Pb, aj, aj + NN, aj + 2 * NN);
    }
    orc_reduce(nthreads, NN, acc, J, Ka, Kb);
    free(acc);
}

/* Integral-direct J/K over a quartet list: the reference's calc_eri quartet
 * block (shelled.py:640-691) digested at once by fill_matrices' rule
 * (shelled.py:826-859), without storing the integrals. */
void orc_direct_jk_fn(int ns, const double *center, const int *l, const int *nexp,
                      const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                      const double *exps, const double *coefs, long nq, const int *quads, int N,
                      const double *P, const double *Pa, const double *Pb, double *J, double *Ka,
                      double *Kb, orc_ref_eri_fn fn);

void orc_direct_jk(int ns, const double *center, const int *l, const int *nexp,
                   const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                   const double *exps, const double *coefs, long nq, const int *quads, int N,
                   const double *P, const double *Pa, const double *Pb, double *J, double *Ka,
                   double *Kb)
{
    orc_direct_jk_fn(ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs, nq, quads, N,
                     P, Pa, Pb, J, Ka, Kb, NULL);
}

/* Same, with the primitive ERIs from `fn` (the reference's own eri_kernel
 * compiled as host code) when it is not NULL. */
void orc_direct_jk_fn(int ns, const double *center, const int *l, const int *nexp,
                      const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                      const double *exps, const double *coefs, long nq, const int *quads, int N,
                      const double *P, const double *Pa, const double *Pb, double *J, double *Ka,
                      double *Kb, orc_ref_eri_fn fn)
{
    OrcShells S = orc_shells(ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs);
    long NN = (long)N * N;
    /* largest contracted block and primitive block of any quartet */
    size_t nao_max = 1, np_max = 1;
    for (int s = 0; s < ns; ++s) {
        size_t a = (size_t)orc_shell_nao(&S, s), p = (size_t)orc_ncomp(l[s]) * nexp[s];
        if (a > nao_max) nao_max = a;
        if (p > np_max) np_max = p;
    }
    const size_t blk_max = nao_max * nao_max * nao_max * nao_max;
    const size_t prim_max = np_max * np_max * np_max * np_max;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    double *acc = (double *)calloc((size_t)nthreads * 3 * NN, sizeof(double));
    #pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *aj = acc + (long)tid * 3 * NN;
        double *prim = (double *)malloc(sizeof(double) * prim_max);
        double *blk = (double *)malloc(sizeof(double) * blk_max);
        #pragma omp for schedule(dynamic, 16)
        for (long t = 0; t < nq; ++t) {
            const int *q = quads + 4 * t;
            OrcPair ab, cd;
            orc_pair_build(&S, q[0], q[1], &ab);
            orc_pair_build(&S, q[2], q[3], &cd);
            orc_quartet_block_fn(&S, &ab, &cd, q[0], q[1], q[2], q[3], prim, blk, fn);
            orc_digest_one(&S, q, blk, N, P, Pa, Pb, aj, aj + NN, aj + 2 * NN);
            orc_pair_free(&ab);
            orc_pair_free(&cd);
        }
        free(prim);
        free(blk);
    }
    orc_reduce(nthreads, NN, acc, J, Ka, Kb);
    free(acc);
}

/* ------------------------------------------------------------ one-electron */
/* 1-D overlap of two Cartesian Gaussians by the binomial expansion of the
 * reference's overlap() (shelled.py:104-146):
 *   exp(-ab/p (A-B)^2) sum_{i<=la, j<=lb, i+j even} C(la,i) C(lb,j) PA^{la-i} PB^{lb-j}
 *   (i+j-1)!! / (2p)^{(i+j)/2} sqrt(pi/p). */
static double orc_binom(int n, int k)
{
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

static double orc_overlap_1d(double al, double be, double A, double B, int la, int lb)
{
    if (la < 0 || lb < 0) return 0.0;
    double p = al + be;
    double P = (al * A + be * B) / p;
    double PA = P - A, PB = P - B;
    double s = 0.0;
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j) {
            int u = i + j;
            if (u & 1) continue;
            s += orc_binom(la, i) * orc_binom(lb, j) * pow(PA, la - i) * pow(PB, lb - j) *
                 orc_dfact(u - 1) / pow(2.0 * p, u / 2) * sqrt(ORC_PI / p);
        }
    return s * exp(-al * be / p * (A - B) * (A - B));
}

/* Contracted S, T, V over all shell pairs into full N x N matrices
 * (shelled.py:961-1069): primitive blocks times normalisation, contracted
 * with the coefficients; T by the l+-2 rule of T_raw (shelled.py:149-155)
 * summed over axes and halved with sign (shelled.py:989-998); V from the
 * pair kernel's nuclear sum (shelled.py:1015-1045). */
void orc_one_electron(int ns, const double *center, const int *l, const int *nexp,
                      const int *ncontr, const int *exp_off, const int *coef_off, const int *ao,
                      const double *exps, const double *coefs, int natoms, const int *Z,
                      const double *atom_xyz, int N, double *Smat, double *Tmat, double *Vmat)
{
    (void)ncontr;
    #pragma omp parallel for schedule(dynamic, 4)
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b <= a; ++b) {
            int ca = orc_ncomp(l[a]), cb = orc_ncomp(l[b]);
            int ea = nexp[a], eb = nexp[b];
            int na = ca * ea, nb = cb * eb;
            int powa[3 * 28], powb[3 * 28];
            orc_components(l[a], powa);
            orc_components(l[b], powb);
            double expa[256], expb[256];
            int pa[3 * 256], pb[3 * 256];
            for (int c = 0; c < ca; ++c)
                for (int e = 0; e < ea; ++e) {
                    int i = c * ea + e;
                    expa[i] = exps[exp_off[a] + e];
                    for (int k = 0; k < 3; ++k) pa[3 * i + k] = powa[3 * c + k];
                }
            for (int c = 0; c < cb; ++c)
                for (int e = 0; e < eb; ++e) {
                    int i = c * eb + e;
                    expb[i] = exps[exp_off[b] + e];
                    for (int k = 0; k < 3; ++k) pb[3 * i + k] = powb[3 * c + k];
                }
            int K = na * nb;
            double *V = (double *)malloc(sizeof(double) * K * (4 + 3 * ORC_E));
            double *Ex = V + K, *Ey = Ex + ORC_E * K, *Ez = Ey + ORC_E * K, *pp = Ez + ORC_E * K;
            double *PP = (double *)malloc(sizeof(double) * 3 * K);
            int *nn = (int *)malloc(sizeof(int) * 3 * K);
            orc_pair_prims(na, expa, pa, center + 3 * a, nb, expb, pb, center + 3 * b, natoms, Z,
                           atom_xyz, V, Ex, Ey, Ez, pp, PP, nn, nn + K, nn + 2 * K);
            int nca = ncontr[a], ncb = ncontr[b];
            for (int ka = 0; ka < nca; ++ka)
                for (int kb = 0; kb < ncb; ++kb)
                    for (int c1 = 0; c1 < ca; ++c1)
                        for (int c2 = 0; c2 < cb; ++c2) {
                            double s = 0.0, t = 0.0, v = 0.0;
                            for (int e1 = 0; e1 < ea; ++e1)
                                for (int e2 = 0; e2 < eb; ++e2) {
                                    int i = c1 * ea + e1, j = c2 * eb + e2;
                                    double al = expa[i], be = expb[j];
                                    double ov[3], kin[3];
                                    for (int d = 0; d < 3; ++d) {
                                        double A = center[3 * a + d], B = center[3 * b + d];
                                        int la_ = pa[3 * i + d], lb_ = pb[3 * j + d];
                                        ov[d] = orc_overlap_1d(al, be, A, B, la_, lb_);
                                        kin[d] = -2.0 * be * (2 * lb_ + 1) * ov[d] +
                                                 4.0 * be * be * orc_overlap_1d(al, be, A, B, la_, lb_ + 2) +
                                                 (lb_ >= 2 ? lb_ * (lb_ - 1) * orc_overlap_1d(al, be, A, B, la_, lb_ - 2) : 0.0);
                                    }
                                    double w = orc_norm(al, pa + 3 * i) * orc_norm(be, pb + 3 * j) *
                                               coefs[coef_off[a] + ka * ea + e1] *
                                               coefs[coef_off[b] + kb * eb + e2];
                                    s += w * ov[0] * ov[1] * ov[2];
                                    t += w * (kin[0] * ov[1] * ov[2] + kin[1] * ov[2] * ov[0] +
                                              kin[2] * ov[0] * ov[1]);
                                    v += w * V[(long)i * nb + j];
                                }
                            int r = ao[a] + ka * ca + c1, q = ao[b] + kb * cb + c2;
                            Smat[(long)r * N + q] = s; Smat[(long)q * N + r] = s;
                            Tmat[(long)r * N + q] = -0.5 * t; Tmat[(long)q * N + r] = -0.5 * t;
                            Vmat[(long)r * N + q] = v; Vmat[(long)q * N + r] = v;
                        }
            free(V); free(PP); free(nn);
        }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------ gradients */
/* Nuclear gradient of the SCF energy (no counterpart in the reference; the
 * reference has no gradients).  Restated from the definitions, independently
 * of the GPU kernels' adjoint ordering: every derivative integral is formed
 * explicitly by the centre-derivative rule of a Cartesian Gaussian,
 *   d/dA_x [a] = 2 alpha [a + 1_x] - a_x [a - 1_x],
 * applied on every centre (all four ERI centres, both one-electron centres
 * and the nuclear-attraction operator centre, whose derivative is
 * -sum E E E R_{t+1,u,v}), with the MD primitives of this file.  The caller
 * passes the total density D, the spin densities Da, Db and the
 * energy-weighted density W; grad[3 * atom + x] receives
 *   sum D dH - sum W dS + 1/2 sum d(mn|ls) [D_mn D_ls - Da_ml Da_ns - Db_ml Db_ns]. */

/* 1-D E^{i,j}_t for i, j <= 3 of one primitive pair: E[((i * 4) + j) * ORC_E + t] */
static void orc_E_table(double al, double be, double A, double B, double *E)
{
    for (int i = 0; i <= 3; ++i)
        for (int j = 0; j <= 3; ++j) orc_hermite_E(al, be, A, B, i, j, E + (i * 4 + j) * ORC_E);
}

/* unnormalised primitive (ab|cd) with powers pa..pd from E tables and an R box
 * (box side 6, index ((t * 6 + u) * 6 + v) * 6 + n) */
static double orc_eri_from_tables(const double *Eb[3], const double *Ek[3], const int *pa,
                                  const int *pb, const int *pc, const int *pd, const double *R,
                                  double pre)
{
    for (int x = 0; x < 3; ++x)
        if (pa[x] < 0 || pb[x] < 0 || pc[x] < 0 || pd[x] < 0) return 0.0;
    const double *ex = Eb[0] + (pa[0] * 4 + pb[0]) * ORC_E, *ey = Eb[1] + (pa[1] * 4 + pb[1]) * ORC_E,
                 *ez = Eb[2] + (pa[2] * 4 + pb[2]) * ORC_E;
    const double *fx = Ek[0] + (pc[0] * 4 + pd[0]) * ORC_E, *fy = Ek[1] + (pc[1] * 4 + pd[1]) * ORC_E,
                 *fz = Ek[2] + (pc[2] * 4 + pd[2]) * ORC_E;
    double s = 0.0;
    for (int t = 0; t <= pa[0] + pb[0]; ++t)
        for (int u = 0; u <= pa[1] + pb[1]; ++u)
            for (int v = 0; v <= pa[2] + pb[2]; ++v) {
                double e = ex[t] * ey[u] * ez[v];
                if (e == 0.0) continue;
                for (int tau = 0; tau <= pc[0] + pd[0]; ++tau)
                    for (int nu = 0; nu <= pc[1] + pd[1]; ++nu)
                        for (int phi = 0; phi <= pc[2] + pd[2]; ++phi) {
                            double f = fx[tau] * fy[nu] * fz[phi];
                            if ((tau + nu + phi) & 1) f = -f;
                            s += e * f * R[(((t + tau) * 6 + (u + nu)) * 6 + (v + phi)) * 6];
                        }
            }
    return s * pre;
}

/* derivative of a primitive integral w.r.t. centre k (0..3) along axis x */
static double orc_deri(const double *Eb[3], const double *Ek[3], const int *p4[4], const double *ex4,
                       int k, int x, const double *R, double pre)
{
    int q[4][3];
    for (int m = 0; m < 4; ++m)
        for (int y = 0; y < 3; ++y) q[m][y] = p4[m][y];
    q[k][x] += 1;
    double v = 2.0 * ex4[k] * orc_eri_from_tables(Eb, Ek, q[0], q[1], q[2], q[3], R, pre);
    if (p4[k][x] > 0) {
        q[k][x] -= 2;
        v -= p4[k][x] * orc_eri_from_tables(Eb, Ek, q[0], q[1], q[2], q[3], R, pre);
    }
    return v;
}

/* one primitive of a shell: exponent, powers, and the contraction x norm weight */
typedef struct {
    double ex, w;
    int pw[3];
    int aoi;
} OrcPrim;

static int orc_shell_prims(const OrcShells *S, int s, OrcPrim *out)
{
    int cmp = orc_ncomp(S->l[s]), ne = S->nexp[s], n = 0;
    int pw[3 * 28];
    orc_components(S->l[s], pw);
    for (int k = 0; k < S->ncontr[s]; ++k)
        for (int c = 0; c < cmp; ++c)
            for (int e = 0; e < ne; ++e) {
                OrcPrim *p = out + n++;
                p->ex = S->exps[S->exp_off[s] + e];
                for (int y = 0; y < 3; ++y) p->pw[y] = pw[3 * c + y];
                p->w = S->coefs[S->coef_off[s] + k * ne + e] * orc_norm(p->ex, p->pw);
                p->aoi = S->ao[s] + k * cmp + c;
            }
    return n;
}

/* 1-D overlap and kinetic pieces for the one-electron derivatives */
static double orc_kin_1d(double al, double be, double A, double B, int la, int lb)
{
    if (la < 0 || lb < 0) return 0.0;
    double v = -2.0 * be * (2 * lb + 1) * orc_overlap_1d(al, be, A, B, la, lb) +
               4.0 * be * be * orc_overlap_1d(al, be, A, B, la, lb + 2);
    if (lb >= 2) v += lb * (lb - 1) * orc_overlap_1d(al, be, A, B, la, lb - 2);
    return v;
}

static double orc_S_prim(double al, double be, const double *A, const double *B, const int *pa, const int *pb)
{
    double s = 1.0;
    for (int d = 0; d < 3; ++d) s *= orc_overlap_1d(al, be, A[d], B[d], pa[d], pb[d]);
    return s;
}

static double orc_T_prim(double al, double be, const double *A, const double *B, const int *pa, const int *pb)
{
    double ov[3], kin[3];
    for (int d = 0; d < 3; ++d) {
        if (pa[d] < 0 || pb[d] < 0) return 0.0;
        ov[d] = orc_overlap_1d(al, be, A[d], B[d], pa[d], pb[d]);
        kin[d] = orc_kin_1d(al, be, A[d], B[d], pa[d], pb[d]);
    }
    return -0.5 * (kin[0] * ov[1] * ov[2] + kin[1] * ov[0] * ov[2] + kin[2] * ov[0] * ov[1]);
}

/* -2 pi / p Z sum_tuv E_t E_u E_v R_{t + sx, u + sy, v + sz}(p, P - C): the
 * nuclear attraction primitive (shift 0) or, with a unit shift, minus its
 * derivative w.r.t. the nuclear centre C. */
static double orc_V_prim(double al, double be, const double *A, const double *B, const int *pa, const int *pb,
                         const double *C, double Z, const int *shift)
{
    for (int d = 0; d < 3; ++d)
        if (pa[d] < 0 || pb[d] < 0) return 0.0;
    double p = al + be, E[3][ORC_E], P[3];
    for (int d = 0; d < 3; ++d) {
        orc_hermite_E(al, be, A[d], B[d], pa[d], pb[d], E[d]);
        P[d] = (al * A[d] + be * B[d]) / p;
    }
    double R[6 * 6 * 6 * 6];
    orc_hermite_R(6, 6, 6, 6, P[0] - C[0], P[1] - C[1], P[2] - C[2], p, R);
    double s = 0.0;
    for (int t = 0; t <= pa[0] + pb[0]; ++t)
        for (int u = 0; u <= pa[1] + pb[1]; ++u)
            for (int v = 0; v <= pa[2] + pb[2]; ++v)
                s += E[0][t] * E[1][u] * E[2][v] * R[(((t + shift[0]) * 6 + u + shift[1]) * 6 + v + shift[2]) * 6];
    return -2.0 * ORC_PI / p * Z * s;
}

void orc_gradient(int ns, const double *center, const int *l, const int *nexp, const int *ncontr,
                  const int *exp_off, const int *coef_off, const int *ao, const double *exps,
                  const double *coefs, const int *shell_atom, int natoms, const int *Z,
                  const double *atom_xyz, int N, const double *D, const double *Da, const double *Db,
                  const double *W, double *grad)
{
    OrcShells S = orc_shells(ns, center, l, nexp, ncontr, exp_off, coef_off, ao, exps, coefs);
    int nthreads = orc_num_threads();
    double *acc = (double *)calloc((size_t)nthreads * 3 * natoms, sizeof(double));
    const int npair = ns * (ns + 1) / 2;
    /* ---- one-electron part over all ordered shell pairs */
    #pragma omp parallel for schedule(dynamic, 1)
    for (int a = 0; a < ns; ++a) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *g = acc + (size_t)tid * 3 * natoms;
        OrcPrim PA[256], PB[256];
        int na = orc_shell_prims(&S, a, PA);
        const double *A = center + 3 * a;
        for (int b = 0; b < ns; ++b) {
            int nb = orc_shell_prims(&S, b, PB);
            const double *B = center + 3 * b;
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    const OrcPrim *pi = PA + i, *pj = PB + j;
                    double w = pi->w * pj->w;
                    double dm = D[(long)pi->aoi * N + pj->aoi] * w, wm = W[(long)pi->aoi * N + pj->aoi] * w;
                    for (int x = 0; x < 3; ++x) {
                        int up[3] = {pi->pw[0], pi->pw[1], pi->pw[2]}, dn[3] = {pi->pw[0], pi->pw[1], pi->pw[2]};
                        up[x] += 1;
                        dn[x] -= 1;
                        int bup[3] = {pj->pw[0], pj->pw[1], pj->pw[2]}, bdn[3] = {pj->pw[0], pj->pw[1], pj->pw[2]};
                        bup[x] += 1;
                        bdn[x] -= 1;
                        /* d/dA and d/dB of S and T */
                        double dSa = 2.0 * pi->ex * orc_S_prim(pi->ex, pj->ex, A, B, up, pj->pw) -
                                     pi->pw[x] * orc_S_prim(pi->ex, pj->ex, A, B, dn, pj->pw);
                        double dSb = 2.0 * pj->ex * orc_S_prim(pi->ex, pj->ex, A, B, pi->pw, bup) -
                                     pj->pw[x] * orc_S_prim(pi->ex, pj->ex, A, B, pi->pw, bdn);
                        double dTa = 2.0 * pi->ex * orc_T_prim(pi->ex, pj->ex, A, B, up, pj->pw) -
                                     pi->pw[x] * orc_T_prim(pi->ex, pj->ex, A, B, dn, pj->pw);
                        double dTb = 2.0 * pj->ex * orc_T_prim(pi->ex, pj->ex, A, B, pi->pw, bup) -
                                     pj->pw[x] * orc_T_prim(pi->ex, pj->ex, A, B, pi->pw, bdn);
                        g[3 * shell_atom[a] + x] += dm * dTa - wm * dSa;
                        g[3 * shell_atom[b] + x] += dm * dTb - wm * dSb;
                        const int zero[3] = {0, 0, 0};
                        int unit[3] = {0, 0, 0};
                        unit[x] = 1;
                        for (int c = 0; c < natoms; ++c) {
                            const double *Cc = atom_xyz + 3 * c;
                            double zc = Z[c];
                            double dVa = 2.0 * pi->ex * orc_V_prim(pi->ex, pj->ex, A, B, up, pj->pw, Cc, zc, zero) -
                                         pi->pw[x] * orc_V_prim(pi->ex, pj->ex, A, B, dn, pj->pw, Cc, zc, zero);
                            double dVb = 2.0 * pj->ex * orc_V_prim(pi->ex, pj->ex, A, B, pi->pw, bup, Cc, zc, zero) -
                                         pj->pw[x] * orc_V_prim(pi->ex, pj->ex, A, B, pi->pw, bdn, Cc, zc, zero);
                            /* d/dC_x R_tuv(P - C) = -R_{t+1,u,v} */
                            double dVc = -orc_V_prim(pi->ex, pj->ex, A, B, pi->pw, pj->pw, Cc, zc, unit);
                            g[3 * shell_atom[a] + x] += dm * dVa;
                            g[3 * shell_atom[b] + x] += dm * dVb;
                            g[3 * c + x] += dm * dVc;
                        }
                    }
                }
        }
    }
    /* ---- two-electron part over unique quartets */
    #pragma omp parallel for schedule(dynamic, 1)
    for (int ab = 0; ab < npair; ++ab) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *g = acc + (size_t)tid * 3 * natoms;
        int a = (int)((sqrt(8.0 * ab + 1.0) - 1.0) / 2.0);
        while (a * (a + 1) / 2 > ab) --a;
        while ((a + 1) * (a + 2) / 2 <= ab) ++a;
        int b = ab - a * (a + 1) / 2;
        OrcPrim PA[256], PB[256], PC[256], PD[256];
        int na = orc_shell_prims(&S, a, PA), nb = orc_shell_prims(&S, b, PB);
        for (int cd = 0; cd <= ab; ++cd) {
            int c = (int)((sqrt(8.0 * cd + 1.0) - 1.0) / 2.0);
            while (c * (c + 1) / 2 > cd) --c;
            while ((c + 1) * (c + 2) / 2 <= cd) ++c;
            int d = cd - c * (c + 1) / 2;
            int nc = orc_shell_prims(&S, c, PC), nd = orc_shell_prims(&S, d, PD);
            int ew = (a == b) + (c == d) + (ab == cd);
            double f = 8.0 / (double)(1 << ew);
            const double *Ac = center + 3 * a, *Bc = center + 3 * b, *Cc = center + 3 * c, *Dc = center + 3 * d;
            int at[4] = {shell_atom[a], shell_atom[b], shell_atom[c], shell_atom[d]};
            /* loop over exponent quadruples, then over the components that share them */
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    double Eb[3][16 * ORC_E];
                    const OrcPrim *pi = PA + i, *pj = PB + j;
                    double p = pi->ex + pj->ex, P[3];
                    for (int x = 0; x < 3; ++x) {
                        orc_E_table(pi->ex, pj->ex, Ac[x], Bc[x], Eb[x]);
                        P[x] = (pi->ex * Ac[x] + pj->ex * Bc[x]) / p;
                    }
                    const double *Ebp[3] = {Eb[0], Eb[1], Eb[2]};
                    for (int k = 0; k < nc; ++k)
                        for (int m = 0; m < nd; ++m) {
                            const OrcPrim *pk = PC + k, *pm = PD + m;
                            const int mu = pi->aoi, nu = pj->aoi, la = pk->aoi, si = pm->aoi;
                            double gam = 0.5 * D[(long)mu * N + nu] * D[(long)la * N + si] -
                                         0.25 * (Da[(long)mu * N + la] * Da[(long)nu * N + si] +
                                                 Db[(long)mu * N + la] * Db[(long)nu * N + si] +
                                                 Da[(long)mu * N + si] * Da[(long)nu * N + la] +
                                                 Db[(long)mu * N + si] * Db[(long)nu * N + la]);
                            gam *= f * pi->w * pj->w * pk->w * pm->w;
                            if (gam == 0.0) continue;
                            double Ek[3][16 * ORC_E];
                            double q = pk->ex + pm->ex, Q[3];
                            for (int x = 0; x < 3; ++x) {
                                orc_E_table(pk->ex, pm->ex, Cc[x], Dc[x], Ek[x]);
                                Q[x] = (pk->ex * Cc[x] + pm->ex * Dc[x]) / q;
                            }
                            const double *Ekp[3] = {Ek[0], Ek[1], Ek[2]};
                            double R[6 * 6 * 6 * 6];
                            orc_hermite_R(6, 6, 6, 6, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], p * q / (p + q), R);
                            double pre = 2.0 * ORC_PI * ORC_PI * sqrt(ORC_PI) / (p * q * sqrt(p + q));
                            const int *p4[4] = {pi->pw, pj->pw, pk->pw, pm->pw};
                            double ex4[4] = {pi->ex, pj->ex, pk->ex, pm->ex};
                            for (int cen = 0; cen < 4; ++cen)
                                for (int x = 0; x < 3; ++x)
                                    g[3 * at[cen] + x] += gam * orc_deri(Ebp, Ekp, p4, ex4, cen, x, R, pre);
                        }
                }
        }
    }
    for (int k = 0; k < 3 * natoms; ++k) {
        double s = 0.0;
        for (int t = 0; t < nthreads; ++t) s += acc[(size_t)t * 3 * natoms + k];
        grad[k] = s;
    }
    free(acc);
}
