/*
 * dftk.h -- C-ABI of libdftk.so, the B200 (sm_100a) Gaussian-integral and
 * Fock-build library.
 *
 * Every entry point returns an int status (DFTK_OK = 0); dftk_last_error()
 * gives a message for the calling host thread.  All array arguments are
 * DEVICE pointers owned by the caller unless stated otherwise; nothing here
 * allocates device memory except dftk_init's one-off constant tables.  Work is
 * issued on the given stream (NULL = legacy default stream) and is
 * asynchronous unless stated otherwise.
 *
 * Reference interfaces replaced (yegor-gondhal/DFT, shelled.py):
 *   dftk_nuclear_kernel   <- RawKernel nuclear_kernel         shelled.py:350-450 (launch :1015)
 *   dftk_eri_kernel       <- RawKernel eri_kernel             shelled.py:452-532 (launch :642)
 *   dftk_boys             <- device boys()/taylor()           shelled.py:174-211
 *   dftk_pair_data        <- per-pair nuclear_kernel launch + pair_cache   shelled.py:1000-1059
 *   dftk_one_electron     <- overlap/T_raw/V block loop       shelled.py:961-1069
 *   dftk_schwarz          <- (absent in the reference: screening bounds)
 *   dftk_eri_blocks       <- calc_eri quartet blocks          shelled.py:596-700
 *   dftk_hl_eri_blocks    <- the same for quartets with a d or f shell
 *   dftk_jk_hl            <- fill_matrices, quartets with a d or f shell (adds to dftk_jk's J/K)
 *   dftk_hl_schwarz       <- (absent in the reference: screening bounds, generic pair layout)
 *   dftk_jk               <- fill_matrices                    shelled.py:770-877
 *   dftk_jk_noalloc       <- (absent in the reference: dftk_jk with fixed in-library scratch)
 *   dftk_grad             <- (absent in the reference: analytic nuclear gradients)
 *   dftk_workspace_bytes  <- (absent: workspace size of one molecule or a batch)
 *   dftk_prepare          <- pair_list + pair_cache setup and the quartet enumeration
 *                            shelled.py:599-603, 962-964, 1000-1059 (one call, Schwarz-sorted)
 *   dftk_grid_ao          <- AO loop of the evaluation script     shelled_eval.py:88-107
 *   dftk_grid_density     <- its density lines                    shelled_eval.py:108-131
 */
#ifndef DFTK_H
#define DFTK_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t-compatible opaque stream handle */
typedef struct CUstream_st *dftk_stream_t;

enum {
    DFTK_OK = 0,
    DFTK_ERR_ARG = 1,          /* bad argument (null pointer, negative size, ...) */
    DFTK_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed */
    DFTK_ERR_UNSUPPORTED = 3,  /* basis feature outside what the kernels handle */
    DFTK_ERR_WORKSPACE = 4,    /* workspace too small */
    DFTK_ERR_SIZE = 5          /* size beyond a fixed maximum */
};

/* dftk_jk flags */
#define DFTK_JK_UHF 1          /* K_a from D_a and K_b from D_b; else K_b untouched and D_b unused */
#define DFTK_JK_MIXED 2        /* FP32 for quartets with Q_ab Q_cd Dmax < tau_fp32 */
#define DFTK_JK_PERSIST 4      /* list path: one selection launch over every class, then one persistent
                                  launch per precision whose warps pull 32-quartet tiles of all classes
                                  (heaviest first) from a device work counter, instead of a selection
                                  and a class kernel per class (timing hook: slot 0 / 6 holds the
                                  persistent FP64 / FP32 launch) */

/* Quartet classes, in the order dftk_jk and dftk_queue_t use them:
 * 0 (ss|ss), 1 (ps|ss), 2 (ps|ps), 3 (pp|ss), 4 (pp|ps), 5 (pp|pp). */
#define DFTK_N_QCLASS 6
#define DFTK_N_PCLASS 3

/* Shells of one molecule, or of a batch of molecules (device arrays).  l <= 1
 * (s, p) for dftk_jk's class kernels and the gradient, l <= 3 for
 * dftk_jk_hl, dftk_hl_eri_blocks and dftk_one_electron (one molecule).  One
 * contraction per shell: the reference splits sp shells (shelled.py:66-75),
 * and a generally contracted shell (a coefficient matrix, shelled.py:49-64)
 * is passed as one shell per contraction row with consecutive AO offsets,
 * which is the reference's AO order (contraction-major, :663-691).
 *
 * One molecule: mol == NULL; every N x N matrix argument is n_ao x n_ao.
 * A batch: the shells of each molecule are contiguous, ao[] holds
 * molecule-local AO indices, and every "N x N" matrix argument (densities,
 * J, K, S, T, V, W) is the concatenation of the molecules' own n x n blocks,
 * block m at element offset mol_mat[m].  Shell pairs and quartets never mix
 * molecules (dftk_queue_t.ket_base).  The workspace functions size the
 * shell-block arrays per molecule (mol_dsh). */
typedef struct {
    int n_shells;
    int n_ao;               /* one molecule: AO count; a batch: largest molecule's */
    const double *xyz;      /* [3 * n_shells] centre of each shell, bohr */
    const int *l;           /* [n_shells] angular momentum */
    const int *nprim;       /* [n_shells] primitives */
    const int *prim_off;    /* [n_shells] first primitive in prim_exp/prim_cn */
    const int *ao;          /* [n_shells] first AO (reference ao_start) */
    const double *prim_exp; /* [total primitives] exponents */
    const double *prim_cn;  /* [total primitives] coefficient x radial norm sqrt((4a)^l) (2a/pi)^{3/4}, which is
                               normal() of every component for s and p (shelled.py:95-101) */
    /* batch description (n_mol = 0 and NULL pointers for one molecule) */
    int n_mol;
    int max_ns;                /* largest shell count of a molecule */
    int max_natom;             /* largest atom count of a molecule */
    long long mat_elems;       /* sum of n_ao^2 over the molecules */
    long long dsh_elems;       /* sum of n_shells^2 over the molecules */
    const int *mol;            /* [n_shells] molecule of each shell */
    const long long *mol_mat;  /* [n_mol] offset of the molecule's n_ao x n_ao block */
    const int *mol_nao;        /* [n_mol] AO count */
    const int *mol_shell0;     /* [n_mol] first shell */
    const int *mol_ns;         /* [n_mol] shell count */
    const long long *mol_dsh;  /* [n_mol] offset of its n_shells x n_shells block in shell-block arrays */
    const int *mol_atom0;      /* [n_mol] first atom (atom arrays are concatenated too) */
    const int *mol_natom;      /* [n_mol] atom count */
} dftk_shells_t;

/* Shell pairs of one pair class (0 ss, 1 ps, 2 pp) with l_a >= l_b, and their
 * primitive-pair records in SoA layout rec[(field * kmax + k) * n_pairs + pair]
 * (fields: P x/y/z, p, K, 1/(2p), PA x/y/z, PB x/y/z, of which ss uses 5, ps 9,
 * pp 12, followed by the bra exponent alpha: 6 / 10 / 13 fields stored). */
typedef struct {
    int n_pairs;
    int kmax;               /* primitive-pair slots per pair (max nprim_a * nprim_b) */
    const int *ab;          /* [2 * n_pairs] shells (a, b) */
    int *nprim;             /* [n_pairs] primitive pairs in use (written by dftk_pair_data) */
    double *rec64;          /* [nfields * kmax * n_pairs] (written by dftk_pair_data) */
    float *rec32;           /* same, FP32 copy for the mixed path */
    double *q;              /* [n_pairs] Schwarz factor sqrt(max|(ab|ab)|) (written by dftk_schwarz) */
    float *qp;              /* [kmax * n_pairs] primitive Schwarz factors sqrt(max|(ab_k|ab_k)|), each
                               pair's primitives reordered by descending qp (written by dftk_schwarz) */
    /* packed core records core[(k * n_pairs + pair) * 8 + slot], slots P x/y/z, p, K, qp, 1/(2p), 0:
       what the class kernels' inner primitive loops read in one or two vector loads (written by
       dftk_pair_data and, sorted, by dftk_schwarz; 64-byte aligned; NULL for the generic layout) */
    double *core64;         /* [8 * kmax * n_pairs] */
    float *core32;          /* [8 * kmax * n_pairs] */
} dftk_pairs_t;

/* Candidate quartets of each class: bra pair `row` of the bra pair class pairs
 * with ket pairs 0 .. (row_off[row+1] - row_off[row] - 1) of the ket class,
 * both classes sorted by descending Schwarz factor (so the Schwarz-surviving
 * kets of a row form a prefix).  For bra class == ket class the prefix stops
 * at the row itself, which enumerates each unique quartet once. */
typedef struct {
    long long n_rows[DFTK_N_QCLASS];
    long long total[DFTK_N_QCLASS];           /* host copy of row_off[n_rows] */
    const long long *row_off[DFTK_N_QCLASS];  /* device [n_rows + 1] */
    double tau_prim;                          /* skip primitive quartets with qp_ab * qp_cd < tau_prim
                                                 (0 keeps all); each skipped one is bounded by it */
    /* batches: ket k of row r is ket pair ket_base[c][r] + k (the first pair of
     * the row's molecule in the ket class, each molecule's pairs contiguous and
     * sorted by descending Schwarz factor); NULL = 0 */
    const int *ket_base[DFTK_N_QCLASS];
    /* batches: molecules m with mol_active[m] == 0 are skipped by the
     * selection pass (per-molecule convergence); NULL = all active */
    const unsigned char *mol_active;
    /* 1: the selection pass groups each tile's surviving quartets by the ket
     * pair's primitive-pair count (nprim <= 1, 4, 9, 16, 36, more), so a
     * warp's lanes loop over similar primitive counts (bases whose pairs
     * differ in primitive count, e.g. general contractions); 0: candidate
     * order (every pair has the same count, e.g. STO-3G) */
    int bucket_kets;
} dftk_queue_t;

/* Shell quartets with a d or f shell (l <= 3).  The reference's eri_kernel takes
 * any momenta (shelled.py:452-532, max_e = 7); here the s/p classes run the
 * generated kernels behind dftk_jk and every quartet with a d or f shell runs a
 * warp-per-quartet kernel with run-time momenta behind dftk_jk_hl (shared
 * scratch per warp: 26.6 KB when lmax = 2, 167 KB when lmax = 3).  Both
 * pair sets use the generic record layout (pair_class DFTK_PCLASS_GENERIC in
 * dftk_pair_data: the 12 ERI fields and alpha, 13 fields) and are sorted by
 * descending Schwarz factor (dftk_hl_schwarz).  Shells may carry l <= 3;
 * prim_cn holds coefficient x radial norm sqrt((4a)^l) (2a/pi)^{3/4}, and the
 * kernels apply each Cartesian component's 1/sqrt(prod (2 l_i - 1)!!) (for
 * s and p shells both conventions agree). */
#define DFTK_PCLASS_GENERIC 3
#define DFTK_HL_LMAX 3
/* primitive-pair-count buckets of the class ket lists (upper bounds) */
#define DFTK_HLC_NB 6
#define DFTK_HLC_BUCKET_BOUNDS {1, 4, 9, 16, 36, 1 << 30}
typedef struct {
    dftk_pairs_t hi;              /* pairs with a d or f shell, l_a >= l_b */
    dftk_pairs_t lo;              /* every s/p pair of the molecule, same layout */
    long long n_rows;             /* hi.n_pairs */
    long long total[2];           /* candidates of (hi|lo) and of (hi|hi) (ket <= row) */
    const long long *row_off[2];  /* device [n_rows + 1] each: Schwarz prefixes as in dftk_queue_t */
    double tau_prim;              /* primitive-quartet cut, as in dftk_queue_t */
    int lmax;                     /* largest shell momentum, 2 (d) or 3 (f): selects the kernels' scratch layout */
    /* Thread-per-quartet classes (generated code): class c = 0 (ds|ss),
     * 1 (ds|ps), 2 (ds|pp), 3 (dp|ss), 4 (dp|ps), 5 (dp|pp), 6 (dd|ss),
     * 7 (dd|ps), 8 (ds|ds), 9 (dp|ds), 10 (dp|dp), 11 (dd|pp), 12 (dd|ds),
     * 13 (dd|dp), 14 (dd|dd); f quartets run in the warp kernel.  Pair kinds: 0 (s,s),
     * 1 (p,s), 2 (p,p) in the lo set, 3 (d,s), 4 (d,p), 5 (d,d) in the hi set.
     * cls_rows[x] lists the hi rows of kind 3 + x ascending (the bras, by
     * descending Schwarz factor).  cls_kets[y] lists the rows of kind y (lo
     * rows for y < 3, hi rows for y >= 3) grouped by primitive-pair count
     * (bucket b holds nprim in (bound[b - 1], bound[b]] of DFTK_HLC_BUCKET_BOUNDS),
     * ascending within a bucket; bucket b starts at cls_ket_seg[y][b].
     * cls_off[c] are the candidate offsets over (bra position r, bucket b),
     * entry r * DFTK_HLC_NB + b: the quartets of bra r with the Schwarz
     * prefix of bucket b's kets (for (ds|ds), (dp|dp) and (dd|dd) only kets
     * whose hi row is <= the bra's, so each unique quartet appears once); cls_total[c] = the last
     * offset.  Bucketing keeps the 32 lanes of a warp on kets with similar
     * primitive counts.  A class whose cls_off is non-NULL takes every
     * quartet of its two pair kinds: the warp-per-quartet kernel skips them,
     * and a host may give the hi rows whose every (hi|lo) quartet belongs to a
     * class zero candidates in row_off[0].  All NULL: every d quartet runs in
     * the warp kernel. */
    const int *cls_rows[3];
    long long n_cls_rows[3];
    const int *cls_kets[6];
    long long cls_ket_seg[6][7];
    const long long *cls_off[15];
    long long cls_total[15];
} dftk_hl_t;

/* library version (integer, 100 * major + minor) */
int dftk_version(void);

/* message of the last failing call on this host thread ("" if none) */
const char *dftk_last_error(void);

/* Load the Boys tables on the current device.  Called implicitly by every
 * compute entry point; call it once yourself before any stream capture. */
int dftk_init(void);

/* F_0..F_mmax(T) for n arguments: F[i * (mmax + 1) + m] (boys/taylor,
 * shelled.py:174-211), through the evaluators the ERI kernels use:
 * mmax 0..8 in FP64 and (dftk_boys32) FP32.  T < 0 is evaluated at 0. */
int dftk_boys(int mmax, long long n, const double *T, double *F, dftk_stream_t stream);
int dftk_boys32(int mmax, long long n, const float *T, float *F, dftk_stream_t stream);

/* Primitive-pair records of every pair in `pairs` (the pair part of
 * nuclear_kernel and pair_cache, shelled.py:1000-1059). */
int dftk_pair_data(const dftk_shells_t *shells, int pair_class, dftk_pairs_t *pairs,
                   dftk_stream_t stream);

/* Schwarz factors pairs->q from the diagonal quartets (ab|ab), primitive
 * factors pairs->qp, and the primitive records of each pair reordered by
 * descending qp.  At most 128 primitive pairs per pair. */
int dftk_schwarz(const dftk_shells_t *shells, int pair_class, dftk_pairs_t *pairs,
                 dftk_stream_t stream);

/* One-call setup of a molecule's pairs and queue for dftk_jk / dftk_grad,
 * everything a host would otherwise do itself: the shell pairs of each pair
 * class in the reference's pair order (i, j <= i; pair_list, shelled.py:962-964,
 * stored with l_a >= l_b), their records and Schwarz factors
 * (dftk_pair_data, dftk_schwarz), the pairs sorted by descending Schwarz
 * factor (stable) with the records rebuilt in that order, and the candidate
 * offsets of every quartet class at tau_schwarz (the unique-quartet
 * enumeration cd <= ab of shelled.py:599-603, Schwarz-screened).  All arrays
 * live in the caller's device `storage` (dftk_prepare_bytes bytes); pairs[3]
 * and *queue are filled with pointers into it.  One molecule; the pairs with
 * a d or f shell are left to dftk_prepare_hl.
 * Reads shells->l and shells->nprim back to the host and synchronises
 * `stream`.  No counterpart in the reference as one call. */
int dftk_prepare_bytes(const dftk_shells_t *shells, size_t *bytes);
int dftk_prepare(const dftk_shells_t *shells, double tau_schwarz, double tau_prim, void *storage,
                 size_t storage_bytes, dftk_pairs_t pairs[DFTK_N_PCLASS], dftk_queue_t *queue,
                 dftk_stream_t stream);

/* Contracted Cartesian S, T, V (N x N, row-major) over all shell pairs
 * (shelled.py:961-1069); atom_z are the nuclear charges as doubles. */
int dftk_one_electron(const dftk_shells_t *shells, int n_atoms, const double *atom_xyz,
                      const double *atom_z, double *S, double *T, double *V,
                      dftk_stream_t stream);

/* AO values at points (the AO loop of the reference's orbital evaluation,
 * shelled_eval.py:88-107): ao[a * ld + g] = x^i y^j z^k sum_p cn_p
 * exp(-alpha_p r^2) / sqrt(prod (2 l_i - 1)!!) for every AO a of the molecule
 * and point g < n_points, with (x, y, z) = point g - the shell centre.  Points
 * are FP32 xyz triples (the reference's grid dtype), the arithmetic and ao
 * are FP64.  One molecule (shells->n_mol == 0) with shells up to f (else
 * DFTK_ERR_UNSUPPORTED); ao
 * holds shells->n_ao rows of ld >= n_points doubles.  Reads shells->l back to
 * the host to check the momenta (synchronises the stream). */
int dftk_grid_ao(const dftk_shells_t *shells, long long n_points, const float *points, double *ao,
                 long long ld, dftk_stream_t stream);

/* Per-orbital densities on points (shelled_eval.py:110-131), from MO values
 * psi_a, psi_b (n_mo rows of ld_psi >= n_points doubles; the MO step
 * psi = C^T ao is a plain GEMM left to the caller's BLAS): for k < n_mo
 *   total[k * ld_out + g] = [k < n_a] psi_a^2 + [k < n_b] psi_b^2  (FP64, stored FP32)
 *   phase[k * ld_out + g] = psi_a (FP32), rows k < n_a only (others untouched). */
int dftk_grid_density(int n_mo, int n_a, int n_b, long long n_points, const double *psi_a,
                      const double *psi_b, long long ld_psi, float *total, float *phase,
                      long long ld_out, dftk_stream_t stream);

/* Contracted ERI blocks of explicit quartets (debug / parity path of calc_eri,
 * shelled.py:640-691).  desc[4 * t] = {quartet class, bra row, ket row, flags}
 * with flags bit0 = bra pair stored as (b, a), bit1 = ket pair stored as
 * (d, c), bit2 = bra and ket exchanged, all relative to the reference quartet
 * (a, b, c, d), and bit3 = evaluate with the FP32 kernels (the mixed path);
 * block t is written at out + out_off[t] in the reference's
 * (n_ao_a, n_ao_b, n_ao_c, n_ao_d) row-major layout.  Descriptors out of
 * range are skipped (their block is left untouched). */
int dftk_eri_blocks(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS],
                    long long n_quartets, const int *desc, const long long *out_off,
                    double *out, dftk_stream_t stream);

/* Workspace bytes dftk_jk needs for n_shells shells and n_ao AOs (direct
 * path: each class kernel scans its candidate space and skips screened
 * quartets itself). */
size_t dftk_jk_workspace_bytes(int n_shells, int n_ao);

/* Workspace bytes for the selection path: a workspace at least this large
 * makes dftk_jk run one selection pass that writes the surviving quartets of
 * every class into FP64/FP32 lists, then class kernels over the lists (no
 * per-kernel scan; one scan for both precisions).  8 bytes per candidate
 * quartet of the queue on top of dftk_jk_workspace_bytes. */
size_t dftk_jk_workspace_bytes_queue(int n_shells, int n_ao, const dftk_queue_t *queue);

/* The same two sizes for any shell set, one molecule or a batch: queue NULL
 * gives the direct-path size (dftk_jk_workspace_bytes), a queue the
 * selection-path size (dftk_jk_workspace_bytes_queue). */
size_t dftk_workspace_bytes(const dftk_shells_t *shells, const dftk_queue_t *queue);

/* Integral-direct J and K (fill_matrices, shelled.py:770-877, without stored
 * ERIs): J = (mu nu|la si) D_la,si and K_s = (mu la|nu si) Ds_la,si over the
 * unique Schwarz-surviving quartets of `queue` whose bound
 * Q_ab Q_cd max|D block| >= tau.  J, K_a (and K_b with DFTK_JK_UHF) are
 * overwritten, N x N row-major, symmetric.  With DFTK_JK_MIXED the quartets
 * with bound < tau_fp32 run in FP32 (accumulation stays FP64).
 * counts (optional device array of 4 * DFTK_N_QCLASS long long, zeroed by
 * the caller) receives per class: shell quartets evaluated in FP64, then in
 * FP32, then primitive quartets evaluated in FP64, then in FP32.
 * With the selection workspace the class kernels may run on a second,
 * library-owned stream of the same device, forked from and joined back into
 * `stream` with events (dftk_grad does the same): the call's work still
 * completes in `stream` order, and concurrent calls on one device take turns
 * at the fork. */
int dftk_jk(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS],
            const dftk_queue_t *queue, const double *D, const double *D_a, const double *D_b,
            double *J, double *K_a, double *K_b, int flags, double tau, double tau_fp32,
            void *workspace, size_t workspace_bytes, long long *counts, dftk_stream_t stream);

/* dftk_jk for callers that cannot allocate device memory (no counterpart in
 * the reference).  Same arguments as dftk_jk without the workspace: the
 * scratch is a fixed device array inside the library (about 7 MB, held on
 * every GPU that loads the library until exit), so the molecule may have at
 * most 512 basis functions and 512 shells (DFTK_ERR_SIZE otherwise).  All
 * calls share that array: calls that overlap on the GPU race, so keep them on
 * one stream.  The first call on a device looks up the array's address with
 * that device current; make it before any stream capture.  The address is
 * kept for the life of the process, so it assumes the device's primary
 * context is not reset (cudaDeviceReset) between calls. */
int dftk_jk_noalloc(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS],
                    const dftk_queue_t *queue, const double *D, const double *D_a,
                    const double *D_b, double *J, double *K_a, double *K_b, int flags,
                    double tau, double tau_fp32, long long *counts, dftk_stream_t stream);

/* The d/f part of one molecule's setup for C hosts (dftk_prepare does the
 * s/p part and skips the pairs with a d or f shell): both generic-layout pair
 * sets built, Schwarz-sorted and described, with the two candidate spaces'
 * row offsets, inside caller storage of dftk_prepare_hl_bytes bytes (device
 * memory, 256-byte aligned).  Shells must already be one per contraction row.
 * Synchronises the stream; storage must outlive the calls that use *hl.
 * No counterpart in the reference beyond pair_list / pair_cache setup. */
int dftk_prepare_hl_bytes(const dftk_shells_t *shells, size_t *bytes);
int dftk_prepare_hl(const dftk_shells_t *shells, double tau_schwarz, double tau_prim, void *storage,
                    size_t storage_bytes, dftk_hl_t *hl, dftk_stream_t stream);

/* Schwarz factors of a generic-layout pair set (momenta <= lmax <= 3), with each
 * pair's primitive records reordered by descending primitive factor (no
 * counterpart in the reference: screening bounds).  kmax <= 128. */
int dftk_hl_schwarz(const dftk_shells_t *shells, dftk_pairs_t *pairs, int lmax, dftk_stream_t stream);

/* Adds the Coulomb and exchange contributions of every quartet with a d or f shell
 * to J, K_a (, K_b): the rest of fill_matrices (shelled.py:770-877) after
 * dftk_jk has written the s/p part.  FP64; quartets whose bound
 * Q_ab Q_cd max|D| is below tau are skipped.  Workspace: at least
 * dftk_jk_workspace_bytes(n_shells, n_ao).  One molecule per call. */
int dftk_jk_hl(const dftk_shells_t *shells, const dftk_hl_t *hl, const double *D, const double *D_a,
               const double *D_b, double *J, double *K_a, double *K_b, int flags, double tau, void *workspace,
               size_t workspace_bytes, long long *counts, dftk_stream_t stream);

/* Contracted ERI blocks of quartets with a d or f shell <- calc_eri quartet blocks
 * shelled.py:596-700.  desc[8 q ..]: {0 = (hi|lo) / 1 = (hi|hi), hi row, ket
 * row, flags (bit 0: the reference's first bra shell is the pair's second,
 * bit 1 the same for the ket, bit 2: the reference's bra is the ket pair),
 * n0, n1, n2, n3 (AO counts of the reference's four shells, the block's
 * strides)}; block q starts at out[out_off[q]]. */
int dftk_hl_eri_blocks(const dftk_shells_t *shells, const dftk_hl_t *hl, long long n_quartets, const int *desc,
                       const long long *out_off, double *out, dftk_stream_t stream);

/* Profiling aid: with timing enabled, later dftk_jk calls record CUDA events
 * around each class kernel on their stream.  dftk_jk_timing_read waits for
 * the last recorded call and writes ms[2 * DFTK_N_QCLASS] (FP64 launches,
 * then FP32 launches; 0 where a class did not launch).  A dftk_grad call
 * records its FP64 / FP32 class kernels in slots 0..5 / 6..11 and its
 * one-electron part in slot 12 (written when n >= 13). */
int dftk_jk_timing(int enable);
int dftk_jk_timing_read(float *ms, int n);

/* Launch shapes of the quartet kernels (no counterpart in the reference):
 * per kernel family, quartet class and precision (fp32 0/1), the threads per
 * block (64 or 128) and the grid cap in resident blocks per SM (1..32).  The
 * autotuner (dft_b200/autotune.py) times candidates and sets the fastest;
 * the table is process-wide, guarded by a mutex, and read at each launch, so
 * set it before capturing a CUDA graph.  Defaults: J/K 128 x 16, gradient
 * 128 x 8. */
#define DFTK_FAMILY_JK 0      /* dftk_jk class kernels (list path) */
#define DFTK_FAMILY_GRAD 1    /* dftk_grad class kernels (list path; fp32 = 0 only) */
#define DFTK_N_FAMILY 2
int dftk_set_launch(int family, int qclass, int fp32, int threads, int blocks_per_sm);
int dftk_get_launch(int family, int qclass, int fp32, int *threads, int *blocks_per_sm);
/* Tile of the J/K list kernels (no counterpart in the reference): per class
 * and precision, how many consecutive 32-quartet work items a warp takes per
 * step of its grid-stride loop (1, 2, 4 or 8; default 1) -- larger tiles keep
 * a warp on neighbouring list entries (same bra pairs).  Set by the
 * autotuner beside the launch shape. */
int dftk_set_tile(int qclass, int fp32, int tile);
int dftk_get_tile(int qclass, int fp32, int *tile);

/* Analytic nuclear gradient (no counterpart in the reference): grad[3 * atom
 * + x] is overwritten with sum D dH/dX - sum W dS/dX + sum Gamma d(ab|cd)/dX
 * (electronic part; the nuclear repulsion term is the caller's).  D is the
 * total density, D_a / D_b the spin densities (both D/2 for RHF), W the
 * energy-weighted density; shell_atom maps shells to atoms, atom_z are the
 * nuclear charges.  Mixed form: with tau_fp32 > tau, quartets whose bound
 * Q_ab Q_cd max|D|^2 lies in [tau, tau_fp32) are differentiated in FP32
 * (list path only; sums in FP64); tau_fp32 <= tau keeps all of them FP64.
 * Quartets of `queue` with Q_ab Q_cd max|D|^2 < tau are
 * skipped; primitive quartets with qp_bra qp_ket < queue->tau_prim too.
 * workspace: at least dftk_jk_workspace_bytes(n_shells, n_ao) bytes; with
 * dftk_jk_workspace_bytes_queue bytes the surviving quartets are compacted
 * by dftk_jk's selection pass first (the faster path). */
int dftk_grad(const dftk_shells_t *shells, const int *shell_atom, int n_atoms, const double *atom_xyz,
              const double *atom_z, const dftk_pairs_t pairs[DFTK_N_PCLASS], const dftk_queue_t *queue,
              const double *D, const double *D_a, const double *D_b, const double *W, double tau,
              double tau_fp32, double *grad, void *workspace, size_t workspace_bytes, dftk_stream_t stream);

/* Drop-in for the reference's nuclear_kernel (same arguments and output
 * layout, shelled.py:350-371): one thread per primitive-component pair,
 * E arrays with 7 slots per pair, num_atoms nuclei with integer charges. */
int dftk_nuclear_kernel(const double *exp_a, const double *exp_b, const double *cen_a,
                        const double *cen_b, const int *pow_a, const int *pow_b,
                        const int *atoms, const double *atom_centers, int num_atoms,
                        int num_funcs_a, int num_funcs_b, double *V_output, double *Ex_output,
                        double *Ey_output, double *Ez_output, double *p_output,
                        double *P_output, int *nx_output, int *ny_output, int *nz_output,
                        dftk_stream_t stream);

/* Drop-in for the reference's eri_kernel (same arguments and output layout,
 * shelled.py:452-473): eri_output[i * K_cd + j] for primitive pair records
 * i of ab and j of cd. */
int dftk_eri_kernel(int K_ab, const double *p_ab, const double *P_ab, const double *Exab,
                    const double *Eyab, const double *Ezab, const int *nxab, const int *nyab,
                    const int *nzab, int K_cd, const double *p_cd, const double *P_cd,
                    const double *Excd, const double *Eycd, const double *Ezcd,
                    const int *nxcd, const int *nycd, const int *nzcd, double *eri_output,
                    dftk_stream_t stream);

/* FMA-pipe microbenchmark used to measure the FP64/FP32 roofline denominator:
 * `iters` dependent-chain-free FMAs per thread (8 chains), result in sink[]
 * (blocks * threads doubles).  precision 64 or 32. */
int dftk_fma_burn(int precision, int blocks, int threads, int iters, double *sink,
                  dftk_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DFTK_H */
