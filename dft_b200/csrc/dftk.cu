// libdftk: C-ABI entry points (declared in include/dftk.h).
//
// One translation unit: the device tables (g_boys64/g_boys32) and all kernels
// live here, so the library needs no relocatable device code.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "boys.cuh"
#include "common.cuh"
#include "generic.cuh"
#include "jk.cuh"
#include "grad.cuh"
#include "onee.cuh"
#include "grid.cuh"
#include "hl.cuh"
#include "hlc.cuh"
#include "hlc_parts.h"

namespace {

thread_local std::string g_last_error;
std::mutex g_init_mutex;
bool g_init_done[128] = {false};

// Auxiliary streams per device: dftk_jk runs independent class kernels side
// by side on them (their FP64 atomics into Y/Z commute), forked from and
// joined back into the caller's stream with events, so the call still
// behaves as one ordered piece of work on that stream.  Created once per
// device by dftk_init (before any stream capture).
struct StreamPool {
    bool ready = false;
    std::mutex mutex;  // held from fork to join: the events are shared by all callers on the device
    cudaStream_t aux[2];
    cudaEvent_t fork;
    cudaEvent_t join[2];
};
StreamPool g_pool[128];
std::vector<double> g_tab64;
std::vector<float> g_tab32;

int fail(int code, const char *what)
{
    g_last_error = what;
    return code;
}

int fail_cuda(cudaError_t e, const char *where)
{
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return DFTK_ERR_CUDA;
}

#define DFTK_CUDA(call)                                                     \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call);                 \
    } while (0)

#define DFTK_LAUNCHED(name)                                                 \
    do {                                                                    \
        cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess) return fail_cuda(e_, name);                  \
    } while (0)

// F_m(T) = exp(-T) sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)), all terms
// positive, summed in long double until they stop contributing.
long double boys_series_ld(int m, long double T)
{
    long double term = 1.0L / (2 * m + 1);
    long double sum = term;
    for (int i = 1; i < 2000; ++i) {
        term *= 2.0L * T / (2 * m + 2 * i + 1);
        sum += term;
        if (term < sum * 1e-22L && i > T) break;
    }
    return expl(-T) * sum;
}

std::vector<double> g_exp64;
std::vector<float> g_exp32;
std::vector<double> g_tab64h;

// Per-order Taylor coefficients F_{L+j}(T_k) / j! (see boys.cuh).
void build_tables()
{
    if (!g_tab64.empty()) return;
    const int R = DFTK_BOYS_ROWS, W = DFTK_BOYS_W, NL = DFTK_BOYS_NL;
    g_tab64.assign((size_t)NL * R * W, 0.0);
    g_tab32.assign((size_t)NL * R * W, 0.0f);
    g_exp64.assign(R, 0.0);
    g_exp32.assign(R, 0.0f);
    std::vector<long double> F64(NL + W), F32(NL + W);
    for (int k = 0; k < R; ++k) {
        const long double t64 = (long double)((double)k * 0.1);  // grid the FP64 evaluator rounds to
        const long double t32 = (long double)((float)k * 0.1f);  // grid the FP32 evaluator rounds to
        for (int m = 0; m < NL + W; ++m) {
            F64[m] = boys_series_ld(m, t64);
            F32[m] = boys_series_ld(m, t32);
        }
        for (int L = 0; L < NL; ++L) {
            long double fact = 1.0L;
            for (int j = 0; j < W; ++j) {
                if (j > 0) fact *= j;
                g_tab64[((size_t)L * R + k) * W + j] = (double)(F64[L + j] / fact);
                g_tab32[((size_t)L * R + k) * W + j] = (float)(F32[L + j] / fact);
            }
        }
        g_exp64[k] = (double)expl(-t64);
        g_exp32[k] = (float)expl(-t32);
        // FP32 rows use coefficients 0..4; slot 5 carries exp(-T_k) (see boys.cuh)
        for (int L = 0; L < NL; ++L) g_tab32[((size_t)L * R + k) * W + 5] = g_exp32[k];
    }
    // half-step FP64 rows: F_{L+j}(T_k) / j! for j = 0..6 and exp(-T_k) in slot 7
    const int RH = DFTK_BOYS_HROWS;
    g_tab64h.assign((size_t)NL * RH * W, 0.0);
    for (int k = 0; k < RH; ++k) {
        const long double t = (long double)((double)k * 0.05);  // grid the evaluator rounds to
        for (int m = 0; m < NL + W; ++m) F64[m] = boys_series_ld(m, t);
        const double ek = (double)expl(-t);
        for (int L = 0; L < NL; ++L) {
            long double fact = 1.0L;
            for (int j = 0; j < W - 1; ++j) {
                if (j > 0) fact *= j;
                g_tab64h[((size_t)L * RH + k) * W + j] = (double)(F64[L + j] / fact);
            }
            g_tab64h[((size_t)L * RH + k) * W + W - 1] = ek;
        }
    }
}

int ensure_init()
{
    int dev = 0;
    DFTK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return fail(DFTK_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_init_mutex);
    if (g_init_done[dev]) return DFTK_OK;
    build_tables();
    DFTK_CUDA(cudaMemcpyToSymbol(g_boys64, g_tab64.data(), sizeof(double) * g_tab64.size()));
    DFTK_CUDA(cudaMemcpyToSymbol(g_boys32, g_tab32.data(), sizeof(float) * g_tab32.size()));
    DFTK_CUDA(cudaMemcpyToSymbol(g_bexp64, g_exp64.data(), sizeof(double) * g_exp64.size()));
    DFTK_CUDA(cudaMemcpyToSymbol(g_bexp32, g_exp32.data(), sizeof(float) * g_exp32.size()));
    DFTK_CUDA(cudaMemcpyToSymbol(g_boys64h, g_tab64h.data(), sizeof(double) * g_tab64h.size()));
    {
        const BoysTables t = {g_tab64.data(), g_tab64.size(), g_tab32.data(), g_tab32.size(), g_exp64.data(),
                              g_exp64.size(), g_exp32.data(), g_exp32.size(), g_tab64h.data(), g_tab64h.size()};
        int st;
        if ((st = hlc_part_a_init(t)) || (st = hlc_part_b_init(t)) || (st = hlc_part_c_init(t)) ||
            (st = hlc_part_d_init(t)))
            return st;
    }
    StreamPool &sp = g_pool[dev];
    for (int i = 0; i < 2; ++i) {
        DFTK_CUDA(cudaStreamCreateWithFlags(&sp.aux[i], cudaStreamNonBlocking));
        DFTK_CUDA(cudaEventCreateWithFlags(&sp.join[i], cudaEventDisableTiming));
    }
    DFTK_CUDA(cudaEventCreateWithFlags(&sp.fork, cudaEventDisableTiming));
    sp.ready = true;
    g_init_done[dev] = true;
    return DFTK_OK;
}

// Launch shapes of the quartet kernels, per (family, class, precision):
// threads per block (64 or 128) and resident blocks per SM of the grid cap.
// Set by dftk_set_launch (the autotuner); read at every launch.
struct LaunchShape {
    int threads;
    int blocks_per_sm;
    int tile = 1;  // J/K list kernels: consecutive 32-entry work items per warp step
};
LaunchShape g_shape[DFTK_N_FAMILY][DFTK_N_QCLASS][2];
bool g_shape_init = false;
std::mutex g_shape_mutex;
int g_sm_count = 0;

void init_shapes_locked()
{
    if (g_shape_init) return;
    for (int c = 0; c < DFTK_N_QCLASS; ++c)
        for (int p = 0; p < 2; ++p) {
            g_shape[DFTK_FAMILY_JK][c][p] = {128, 16, 1};
            g_shape[DFTK_FAMILY_GRAD][c][p] = {128, 8, 1};
        }
    g_shape_init = true;
}

LaunchShape launch_shape(int family, int c, int fp32)
{
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    init_shapes_locked();
    return g_shape[family][c][fp32 ? 1 : 0];
}

int sm_count()
{
    if (g_sm_count > 0) return g_sm_count;
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        n > 0)
        g_sm_count = n;
    return g_sm_count > 0 ? g_sm_count : 148;
}

// grid of a quartet kernel: enough blocks for `threads_needed` threads, at
// most blocks_per_sm x SM count
unsigned shaped_grid(const LaunchShape &sh, long long threads_needed)
{
    long long blocks = (threads_needed + sh.threads - 1) / sh.threads;
    const long long cap = (long long)sm_count() * sh.blocks_per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

#define DFTK_INIT()                                                         \
    do {                                                                    \
        int s_ = ensure_init();                                             \
        if (s_ != DFTK_OK) return s_;                                       \
    } while (0)

inline unsigned blocks_for(long long n, int threads)
{
    return (unsigned)((n + threads - 1) / threads);
}

// Workspace layout of dftk_jk: Y, Za, Zb (N*N doubles each), then Dsh (ns*ns floats).
size_t ws_bytes(int ns, int n_ao)
{
    const size_t nn = (size_t)n_ao * n_ao;
    size_t b = 3 * nn * sizeof(double);
    b += (size_t)ns * ns * sizeof(float);
    return (b + 255) & ~(size_t)255;
}

#ifndef DFTK_JK_STREAMS_DEFAULT
#define DFTK_JK_STREAMS_DEFAULT 2  // measured on (H2O)_64: 23.6 -> 22.4 ms per FP64 build
#endif

// Optional per-class event timing of dftk_jk (dftk_jk_timing).
// slots: FP64 class launches 0..5, FP32 ones 6..11, one-electron part of a gradient 12
#define DFTK_TIMING_SLOTS (2 * DFTK_N_QCLASS + 1)
struct JkTiming {
    bool enabled = false;
    bool created = false;
    bool launched[DFTK_TIMING_SLOTS] = {false};
    cudaEvent_t start[DFTK_TIMING_SLOTS];
    cudaEvent_t stop[DFTK_TIMING_SLOTS];
};
JkTiming g_timing;
std::mutex g_timing_mutex;

template <int C, typename T>
int launch_jk_class(const JkParams &P, cudaStream_t s)
{
    const long long ncand = P.total[C];
    const int slot = C + (sizeof(T) == 4 ? DFTK_N_QCLASS : 0);
    if (g_timing.enabled) g_timing.launched[slot] = false;
    if (ncand <= 0) return DFTK_OK;
    const long long warps = ((ncand + 31) / 32) * EriClass<T, C, 0>::NSPLIT;
    long long blocks = (warps * 32 + 127) / 128;
    const long long cap = 148LL * 16;
    if (blocks > cap) blocks = cap;
    if (g_timing.enabled) DFTK_CUDA(cudaEventRecord(g_timing.start[slot], s));
    k_jk<C, T><<<(unsigned)blocks, 128, 0, s>>>(P);
    DFTK_LAUNCHED("k_jk");
    if (g_timing.enabled) {
        DFTK_CUDA(cudaEventRecord(g_timing.stop[slot], s));
        g_timing.launched[slot] = true;
    }
    return DFTK_OK;
}

template <int C, typename T>
int launch_jk_list_class(const JkParams &P, cudaStream_t s)
{
    const long long ncand = P.total[C];
    const int slot = C + (sizeof(T) == 4 ? DFTK_N_QCLASS : 0);
    if (g_timing.enabled) g_timing.launched[slot] = false;
    if (ncand <= 0) return DFTK_OK;
    const long long warps = ((ncand + 31) / 32) * EriClass<T, C, 0>::NSPLIT;
    const LaunchShape sh = launch_shape(DFTK_FAMILY_JK, C, sizeof(T) == 4);
    const unsigned blocks = shaped_grid(sh, warps * 32);
    if (g_timing.enabled) DFTK_CUDA(cudaEventRecord(g_timing.start[slot], s));
    k_jk_list<C, T><<<blocks, sh.threads, 0, s>>>(P);
    DFTK_LAUNCHED("k_jk_list");
    if (g_timing.enabled) {
        DFTK_CUDA(cudaEventRecord(g_timing.stop[slot], s));
        g_timing.launched[slot] = true;
    }
    return DFTK_OK;
}

template <int C>
int launch_select_class(const JkParams &P, cudaStream_t s)
{
    const long long ncand = P.total[C];
    if (ncand <= 0) return DFTK_OK;
    long long blocks = (ncand + SELECT_TILE - 1) / SELECT_TILE;
    const long long cap = 148LL * 8;
    if (blocks > cap) blocks = cap;
    k_select<C><<<(unsigned)blocks, SELECT_THREADS, 0, s>>>(P);
    DFTK_LAUNCHED("k_select");
    return DFTK_OK;
}


// One class of the list path on stream cs: its selection pass, then its FP64
// class kernel and, for a mixed build, its FP32 one (counts slots as in dftk_jk).
template <int C>
int launch_class_pipeline(JkParams P, bool mixed, long long *counts, cudaStream_t cs)
{
    int st;
    P.counts = counts;
    if ((st = launch_select_class<C>(P, cs))) return st;
    if ((st = launch_jk_list_class<C, double>(P, cs))) return st;
    if (mixed) {
        P.counts = counts ? counts + DFTK_N_QCLASS : nullptr;
        if ((st = launch_jk_list_class<C, float>(P, cs))) return st;
    }
    return DFTK_OK;
}

// Streams the class kernels go to: 1 = all on the caller's stream; 2 or 3
// split the classes by measured cost, so one class's tail overlaps the next
// class's work (default 2; the environment variable DFTK_JK_STREAMS = 1..3
// overrides it).  Timing mode (dftk_jk_timing) keeps them on one stream so
// per-class times stay clean.
int jk_stream_count()
{
    static int n = -1;
    if (n < 0) {
        const char *e = getenv("DFTK_JK_STREAMS");
        n = e ? atoi(e) : DFTK_JK_STREAMS_DEFAULT;
        if (n < 1) n = 1;
        if (n > 3) n = 3;
    }
    return g_timing.enabled ? 1 : n;
}

int fork_class_streams(cudaStream_t s, cudaStream_t *cls, int &n_aux, bool gradient = false)
{
    int dev = 0;
    DFTK_CUDA(cudaGetDevice(&dev));
    const int n = jk_stream_count();
    n_aux = 0;
    for (int c = 0; c < DFTK_N_QCLASS; ++c) cls[c] = s;
    if (n == 1 || dev < 0 || dev >= 128 || !g_pool[dev].ready) return DFTK_OK;
    StreamPool &sp = g_pool[dev];
    n_aux = n - 1;
    DFTK_CUDA(cudaEventRecord(sp.fork, s));
    for (int i = 0; i < n_aux; ++i) DFTK_CUDA(cudaStreamWaitEvent(sp.aux[i], sp.fork, 0));
    // classes by cost on (H2O)_64: (ps|ss) 9.1 ms, (ss|ss) 6.0, (ps|ps) 3.3, (pp|ss) 1.8, (pp|ps) 1.8, (pp|pp) 0.5
    static const int two[DFTK_N_QCLASS] = {1, 0, 1, 0, 1, 0};
    static const int three[DFTK_N_QCLASS] = {1, 0, 2, 2, 1, 2};
    // gradient classes: (ss|ss) 12.5 ms, (ps|ss) 17.4, (ps|ps) 8.1, (pp|ss) 4.9, (pp|ps) 14.0, (pp|pp) 11.6
    static const int two_g[DFTK_N_QCLASS] = {1, 0, 1, 0, 1, 0};
    static const int three_g[DFTK_N_QCLASS] = {1, 0, 2, 2, 1, 2};
    for (int c = 0; c < DFTK_N_QCLASS; ++c) {
        const int k = gradient ? (n == 2 ? two_g[c] : three_g[c]) : (n == 2 ? two[c] : three[c]);
        cls[c] = k == 0 ? s : sp.aux[k - 1];
    }
    return DFTK_OK;
}

int join_class_streams(cudaStream_t s, int n_aux)
{
    if (n_aux == 0) return DFTK_OK;
    int dev = 0;
    DFTK_CUDA(cudaGetDevice(&dev));
    StreamPool &sp = g_pool[dev];
    for (int i = 0; i < n_aux; ++i) {
        DFTK_CUDA(cudaEventRecord(sp.join[i], sp.aux[i]));
        DFTK_CUDA(cudaStreamWaitEvent(s, sp.join[i], 0));
    }
    return DFTK_OK;
}

// Workspace with room for the selection lists: the base layout, then the
// 2 * DFTK_N_QCLASS list counters, then one int2 per candidate of every class.
// the same for a shell set that may be a batch (matrix and shell-block sizes summed per molecule)
size_t ws_bytes_sh(const dftk_shells_t &sh)
{
    size_t b = 3 * (size_t)shells_mat_elems(sh) * sizeof(double);
    b += (size_t)shells_dsh_elems(sh) * sizeof(float);
    return (b + 255) & ~(size_t)255;
}

size_t ws_list_bytes_sh(const dftk_shells_t &sh, const dftk_queue_t *q)
{
    size_t b = ws_bytes_sh(sh) + 256;
    for (int c = 0; c < DFTK_N_QCLASS; ++c)
        if (q->n_rows[c] > 0 && q->total[c] > 0) b += (((size_t)q->total[c] * sizeof(int2)) + 255) & ~(size_t)255;
    return b;
}

// shell-block maxima of |D| for every molecule (before the selection or scan)
int launch_dsh(const dftk_shells_t &sh, const double *D, const double *Da, const double *Db, int uhf, float *Dsh,
               cudaStream_t s)
{
    const int max_ns = sh.mol ? sh.max_ns : sh.n_shells;
    const long long n = (long long)sh.n_shells * max_ns;
    if (n == 0) return DFTK_OK;
    k_dsh<<<blocks_for(n, 128), 128, 0, s>>>(sh, max_ns, D, Da, Db, uhf, Dsh);
    DFTK_LAUNCHED("k_dsh");
    return DFTK_OK;
}

int launch_symmetrize(const dftk_shells_t &sh, const double *Y, const double *Za, const double *Zb, double *J,
                      double *Ka, double *Kb, int uhf, cudaStream_t s)
{
    const long long nn = (long long)sh.n_ao * sh.n_ao;  // the largest molecule's block in a batch
    long long bx = (nn + 255) / 256;
    if (bx > 148 * 8) bx = 148 * 8;
    if (bx < 1) bx = 1;
    const dim3 grid((unsigned)bx, (unsigned)shells_n_mol(sh));
    k_symmetrize<<<grid, 256, 0, s>>>(sh, Y, Za, Zb, J, Ka, Kb, uhf);
    DFTK_LAUNCHED("k_symmetrize");
    return DFTK_OK;
}

size_t ws_list_bytes(int ns, int n_ao, const dftk_queue_t *q)
{
    size_t b = ws_bytes(ns, n_ao) + 256;
    for (int c = 0; c < DFTK_N_QCLASS; ++c)
        if (q->n_rows[c] > 0 && q->total[c] > 0) b += (((size_t)q->total[c] * sizeof(int2)) + 255) & ~(size_t)255;
    return b;
}

// The persistent class kernel: every block resident (SM count x MINB blocks
// of 128 threads).  MINB (the register cap shared by all classes) comes from
// DFTK_PERSIST_MINB64 / DFTK_PERSIST_MINB32 (instantiated: FP64 4 or 6,
// FP32 6 or 8; defaults 4 and 6).
template <typename T>
int launch_jk_persist(const JkParams &P, cudaStream_t s)
{
    static int minb64 = -1, minb32 = -1;
    if (minb64 < 0) {
        const char *e = getenv("DFTK_PERSIST_MINB64");
        minb64 = (e && atoi(e) == 6) ? 6 : 4;
        e = getenv("DFTK_PERSIST_MINB32");
        minb32 = (e && atoi(e) == 8) ? 8 : 6;
    }
    const int slot = sizeof(T) == 4 ? DFTK_N_QCLASS : 0;
    if (g_timing.enabled) DFTK_CUDA(cudaEventRecord(g_timing.start[slot], s));
    if constexpr (sizeof(T) == 8) {
        if (minb64 == 6) k_jk_persist<double, 6><<<(unsigned)(sm_count() * 6), 128, 0, s>>>(P);
        else k_jk_persist<double, 4><<<(unsigned)(sm_count() * 4), 128, 0, s>>>(P);
    } else {
        if (minb32 == 8) k_jk_persist<float, 8><<<(unsigned)(sm_count() * 8), 128, 0, s>>>(P);
        else k_jk_persist<float, 6><<<(unsigned)(sm_count() * 6), 128, 0, s>>>(P);
    }
    DFTK_LAUNCHED("k_jk_persist");
    if (g_timing.enabled) {
        DFTK_CUDA(cudaEventRecord(g_timing.stop[slot], s));
        g_timing.launched[slot] = true;
        for (int c = 1; c < DFTK_N_QCLASS; ++c) g_timing.launched[slot + c] = false;
    }
    return DFTK_OK;
}

template <typename T>
int launch_jk_all(const JkParams &P, cudaStream_t s)
{
    int st;
    if ((st = launch_jk_class<0, T>(P, s))) return st;
    if ((st = launch_jk_class<1, T>(P, s))) return st;
    if ((st = launch_jk_class<2, T>(P, s))) return st;
    if ((st = launch_jk_class<3, T>(P, s))) return st;
    if ((st = launch_jk_class<4, T>(P, s))) return st;
    if ((st = launch_jk_class<5, T>(P, s))) return st;
    return DFTK_OK;
}

}  // namespace

// Lets the other translation units of the library report errors through
// dftk_last_error(); hidden, not part of the C-ABI.
extern "C" __attribute__((visibility("hidden"))) void dftk_internal_set_error(const char *msg)
{
    g_last_error = msg ? msg : "";
}

extern "C" {

int dftk_version(void) { return 100; }

const char *dftk_last_error(void) { return g_last_error.c_str(); }

int dftk_init(void)
{
    g_last_error.clear();
    return ensure_init();
}

int dftk_boys(int mmax, long long n, const double *T, double *F, dftk_stream_t stream)
{
    if (mmax < 0 || mmax > 8 || n < 0 || (n > 0 && (!T || !F))) return fail(DFTK_ERR_ARG, "dftk_boys: bad arguments (mmax 0..8)");
    DFTK_INIT();
    if (n == 0) return DFTK_OK;
    k_boys_test<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(mmax, n, T, F);
    DFTK_LAUNCHED("k_boys_test");
    return DFTK_OK;
}

int dftk_boys32(int mmax, long long n, const float *T, float *F, dftk_stream_t stream)
{
    if (mmax < 0 || mmax > 8 || n < 0 || (n > 0 && (!T || !F))) return fail(DFTK_ERR_ARG, "dftk_boys32: bad arguments (mmax 0..8)");
    DFTK_INIT();
    if (n == 0) return DFTK_OK;
    k_boys32_test<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(mmax, n, T, F);
    DFTK_LAUNCHED("k_boys32_test");
    return DFTK_OK;
}

int dftk_pair_data(const dftk_shells_t *shells, int pair_class, dftk_pairs_t *pairs, dftk_stream_t stream)
{
    if (!shells || !pairs || pair_class < 0 || pair_class > DFTK_PCLASS_GENERIC)
        return fail(DFTK_ERR_ARG, "dftk_pair_data: bad arguments");
    if (pairs->n_pairs < 0 || pairs->kmax <= 0) return fail(DFTK_ERR_ARG, "dftk_pair_data: bad pair counts");
    const int nf = pair_class == DFTK_PCLASS_GENERIC ? HL_FIELDS : pair_fields(pair_class);
    if ((long long)pairs->n_pairs * pairs->kmax * nf >= (1LL << 31))
        return fail(DFTK_ERR_SIZE, "dftk_pair_data: records exceed 2^31 elements (32-bit offsets)");
    DFTK_INIT();
    const long long n = (long long)pairs->n_pairs * pairs->kmax;
    if (n == 0) return DFTK_OK;
    k_pair_data<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(*shells, *pairs, nf);
    DFTK_LAUNCHED("k_pair_data");
    return DFTK_OK;
}

int dftk_schwarz(const dftk_shells_t *shells, int pair_class, dftk_pairs_t *pairs, dftk_stream_t stream)
{
    if (!shells || !pairs || pair_class < 0 || pair_class > 2) return fail(DFTK_ERR_ARG, "dftk_schwarz: bad arguments");
    DFTK_INIT();
    const int n = pairs->n_pairs;
    if (n == 0) return DFTK_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (pairs->kmax > DFTK_MAX_KPAIR) return fail(DFTK_ERR_SIZE, "dftk_schwarz: more than 128 primitive pairs per pair");
    if (!pairs->qp) return fail(DFTK_ERR_ARG, "dftk_schwarz: null qp");
    if (!pairs->core64 || !pairs->core32) return fail(DFTK_ERR_ARG, "dftk_schwarz: null core records");
    const int nf = pair_fields(pair_class);
    if (pair_class == 0) k_schwarz<0><<<blocks_for(n, 64), 64, 0, s>>>(*pairs, nf);
    else if (pair_class == 1) k_schwarz<1><<<blocks_for(n, 64), 64, 0, s>>>(*pairs, nf);
    else k_schwarz<2><<<blocks_for(n, 64), 64, 0, s>>>(*pairs, nf);
    DFTK_LAUNCHED("k_schwarz");
    return DFTK_OK;
}

}  // extern "C" (the setup helpers below are C++)

namespace {

// One molecule's setup plan: the pair lists of each pair class in the
// reference's pair order (i, j <= i; stored with l_a >= l_b) and the byte
// offsets of every array in the caller's storage.
struct PreparePlan {
    int kmax = 1;
    std::vector<int> ab[DFTK_N_PCLASS];
    size_t off_ab[DFTK_N_PCLASS], off_np[DFTK_N_PCLASS], off_r64[DFTK_N_PCLASS], off_r32[DFTK_N_PCLASS],
        off_q[DFTK_N_PCLASS], off_qp[DFTK_N_PCLASS], off_c64[DFTK_N_PCLASS], off_c32[DFTK_N_PCLASS],
        off_row[DFTK_N_QCLASS];
    int bucket_kets = 0;  // the s/p pairs span more than one primitive-count bucket
    size_t bytes = 0;
};

constexpr int kQX[DFTK_N_QCLASS] = {0, 1, 1, 2, 2, 2}, kQY[DFTK_N_QCLASS] = {0, 0, 1, 0, 1, 2};

size_t carve(size_t &at, size_t n)
{
    const size_t o = at;
    at += (n + 255) / 256 * 256;
    return o;
}

int prepare_plan(const dftk_shells_t *shells, PreparePlan &pl)
{
    const int ns = shells->n_shells;
    std::vector<int> l(ns), np(ns);
    if (ns > 0) {
        DFTK_CUDA(cudaMemcpy(l.data(), shells->l, sizeof(int) * ns, cudaMemcpyDeviceToHost));
        DFTK_CUDA(cudaMemcpy(np.data(), shells->nprim, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    }
    int pmax = 1;
    for (int i = 0; i < ns; ++i) {
        if (l[i] < 0 || l[i] > HL_LMAX) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare: shells beyond f");
        if (np[i] < 1) return fail(DFTK_ERR_ARG, "dftk_prepare: a shell without primitives");
        pmax = std::max(pmax, np[i]);
    }
    pl.kmax = pmax * pmax;
    if (pl.kmax > DFTK_MAX_KPAIR) return fail(DFTK_ERR_SIZE, "dftk_prepare: more than 128 primitive pairs per pair");
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) {
            const bool swap = l[i] < l[j];
            const int a = swap ? j : i, b = swap ? i : j;
            if (l[a] >= 2) continue;  // pairs with a d or f shell: dftk_prepare_hl
            auto &v = pl.ab[l[a] + l[b]];
            v.push_back(a);
            v.push_back(b);
        }
    {
        // primitive-count buckets of the s/p pairs (as the selection pass forms them)
        static const long long bounds[DFTK_HLC_NB] = DFTK_HLC_BUCKET_BOUNDS;
        int first = -1;
        for (int pc = 0; pc < DFTK_N_PCLASS && !pl.bucket_kets; ++pc)
            for (size_t k = 0; k < pl.ab[pc].size() / 2; ++k) {
                const long long n = (long long)np[pl.ab[pc][2 * k]] * np[pl.ab[pc][2 * k + 1]];
                int b = 0;
                while (b + 1 < DFTK_HLC_NB && n > bounds[b]) ++b;
                if (first < 0) first = b;
                if (b != first) {
                    pl.bucket_kets = 1;
                    break;
                }
            }
    }
    size_t at = 0;
    for (int pc = 0; pc < DFTK_N_PCLASS; ++pc) {
        const size_t n = pl.ab[pc].size() / 2, rec = (size_t)pair_fields(pc) * pl.kmax * n;
        pl.off_ab[pc] = carve(at, sizeof(int) * 2 * std::max<size_t>(n, 1));
        pl.off_np[pc] = carve(at, sizeof(int) * std::max<size_t>(n, 1));
        pl.off_r64[pc] = carve(at, sizeof(double) * std::max<size_t>(rec, 1));
        pl.off_r32[pc] = carve(at, sizeof(float) * std::max<size_t>(rec, 1));
        pl.off_q[pc] = carve(at, sizeof(double) * std::max<size_t>(n, 1));
        pl.off_qp[pc] = carve(at, sizeof(float) * std::max<size_t>((size_t)pl.kmax * n, 1));
        pl.off_c64[pc] = carve(at, sizeof(double) * 8 * std::max<size_t>((size_t)pl.kmax * n, 1));
        pl.off_c32[pc] = carve(at, sizeof(float) * 8 * std::max<size_t>((size_t)pl.kmax * n, 1));
    }
    for (int c = 0; c < DFTK_N_QCLASS; ++c) pl.off_row[c] = carve(at, sizeof(long long) * (pl.ab[kQX[c]].size() / 2 + 1));
    pl.bytes = at;
    return DFTK_OK;
}

// The d/f part of a molecule's setup: the pairs with a d or f shell ("hi")
// and every s/p pair ("lo") in the generic 13-field layout.
struct PrepareHlPlan {
    int kmax = 1, lmax = 2;
    std::vector<int> l;      // shell momenta
    std::vector<int> ab[2];  // 0 hi, 1 lo
    size_t off_ab[2], off_np[2], off_r64[2], off_r32[2], off_q[2], off_qp[2], off_row[2];
    size_t off_cls_rows[3], off_cls_kets[HLC_N_KINDS], off_cls_off[HLC_N_CLASSES];
    std::vector<int> np;  // primitives per shell
    size_t bytes = 0;
};

int prepare_hl_plan(const dftk_shells_t *shells, PrepareHlPlan &pl)
{
    const int ns = shells->n_shells;
    std::vector<int> l(ns), np(ns);
    if (ns > 0) {
        DFTK_CUDA(cudaMemcpy(l.data(), shells->l, sizeof(int) * ns, cudaMemcpyDeviceToHost));
        DFTK_CUDA(cudaMemcpy(np.data(), shells->nprim, sizeof(int) * ns, cudaMemcpyDeviceToHost));
    }
    int pmax = 1;
    for (int i = 0; i < ns; ++i) {
        if (l[i] < 0 || l[i] > HL_LMAX) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare_hl: shells beyond f");
        if (np[i] < 1) return fail(DFTK_ERR_ARG, "dftk_prepare_hl: a shell without primitives");
        pmax = std::max(pmax, np[i]);
        pl.lmax = std::max(pl.lmax, l[i]);
    }
    pl.kmax = pmax * pmax;
    if (pl.kmax > HL_MAX_KPAIR) return fail(DFTK_ERR_SIZE, "dftk_prepare_hl: more than 128 primitive pairs per pair");
    for (int i = 0; i < ns; ++i)
        for (int j = 0; j <= i; ++j) {
            const bool swap = l[i] < l[j];
            const int a = swap ? j : i, b = swap ? i : j;
            auto &v = pl.ab[l[a] >= 2 ? 0 : 1];
            v.push_back(a);
            v.push_back(b);
        }
    size_t at = 0;
    for (int k = 0; k < 2; ++k) {
        const size_t n = pl.ab[k].size() / 2, rec = (size_t)HL_FIELDS * pl.kmax * n;
        pl.off_ab[k] = carve(at, sizeof(int) * 2 * std::max<size_t>(n, 1));
        pl.off_np[k] = carve(at, sizeof(int) * std::max<size_t>(n, 1));
        pl.off_r64[k] = carve(at, sizeof(double) * std::max<size_t>(rec, 1));
        pl.off_r32[k] = carve(at, sizeof(float) * std::max<size_t>(rec, 1));
        pl.off_q[k] = carve(at, sizeof(double) * std::max<size_t>(n, 1));
        pl.off_qp[k] = carve(at, sizeof(float) * std::max<size_t>((size_t)pl.kmax * n, 1));
    }
    for (int k = 0; k < 2; ++k) pl.off_row[k] = carve(at, sizeof(long long) * (pl.ab[0].size() / 2 + 1));
    const size_t nhi = pl.ab[0].size() / 2, nlo = pl.ab[1].size() / 2;
    for (int x = 0; x < 3; ++x) pl.off_cls_rows[x] = carve(at, sizeof(int) * std::max<size_t>(nhi, 1));
    for (int y = 0; y < HLC_N_KINDS; ++y) pl.off_cls_kets[y] = carve(at, sizeof(int) * std::max<size_t>(y < 3 ? nlo : nhi, 1));
    for (int c = 0; c < HLC_N_CLASSES; ++c) pl.off_cls_off[c] = carve(at, sizeof(long long) * (nhi * DFTK_HLC_NB + 1));
    pl.l = l;
    pl.np = np;
    pl.bytes = at;
    return DFTK_OK;
}

// Row offsets of one candidate space: bra row r keeps the ket prefix with
// q_ket >= tau / q_bra[r] (both sorted descending), cut at k <= r when
// `same` (bra and ket are one pair set) so each unique quartet appears once.
std::vector<long long> prefix_offsets(const std::vector<double> &qx, const std::vector<double> &qy, bool same,
                                      double tau)
{
    const size_t nr = qx.size(), nk = qy.size();
    std::vector<long long> off(nr + 1, 0);
    for (size_t r = 0; r < nr; ++r) {
        long long cnt = 0;
        if (nk > 0 && qx[r] > 0.0) {
            const double thr = tau / qx[r];
            size_t lo = 0, hi = nk;
            while (lo < hi) {
                const size_t mid = (lo + hi) / 2;
                if (qy[mid] >= thr) lo = mid + 1;
                else hi = mid;
            }
            cnt = (long long)lo;
        }
        if (same) cnt = std::min<long long>(cnt, (long long)r + 1);
        off[r + 1] = off[r] + cnt;
    }
    return off;
}

// Candidate spaces of the thread-per-quartet d classes over one pair
// layout (hi / lo lists of (a, b) in Schwarz order with their q): bra lists
// per hi kind, ket lists per kind grouped by primitive-count bucket, and the
// offsets over (bra position, bucket), as dftk_hl_t documents them.
struct ClassSpaces {
    std::vector<int> rows[3], kets[HLC_N_KINDS];
    long long seg[HLC_N_KINDS][DFTK_HLC_NB + 1];
    std::vector<long long> off[HLC_N_CLASSES];
};

int hlc_bucket(long long nprim)
{
    static const long long bounds[DFTK_HLC_NB] = DFTK_HLC_BUCKET_BOUNDS;
    for (int b = 0; b < DFTK_HLC_NB; ++b)
        if (nprim <= bounds[b]) return b;
    return DFTK_HLC_NB - 1;
}

void class_spaces(const std::vector<int> &l, const std::vector<int> &np, const std::vector<int> (&ab)[2],
                  const std::vector<double> (&qs)[2], double tau, ClassSpaces &cs)
{
    std::vector<int> kind_lists[HLC_N_KINDS];
    for (int set = 0; set < 2; ++set)
        for (size_t r = 0; r < qs[set].size(); ++r) {
            const int la = l[ab[set][2 * r]], lb = l[ab[set][2 * r + 1]];
            if (la > 2) continue;
            const int kind = la == 0 ? 0 : (la == 1 ? 1 + lb : 3 + lb);
            if (kind >= 3) cs.rows[kind - 3].push_back((int)r);
            kind_lists[kind].push_back((int)r);
        }
    for (int y = 0; y < HLC_N_KINDS; ++y) {
        const int set = y < 3 ? 1 : 0;
        std::vector<int> &kl = cs.kets[y];
        kl.clear();
        for (int b = 0; b < DFTK_HLC_NB; ++b) {
            cs.seg[y][b] = (long long)kl.size();
            for (int r : kind_lists[y]) {
                const long long n = (long long)np[ab[set][2 * r]] * np[ab[set][2 * r + 1]];
                if (hlc_bucket(n) == b) kl.push_back(r);
            }
        }
        cs.seg[y][DFTK_HLC_NB] = (long long)kl.size();
    }
    for (int c = 0; c < HLC_N_CLASSES; ++c) {
        const int bk = hlc_class_kinds[c][0], kk = hlc_class_kinds[c][1];
        const std::vector<int> &bra = cs.rows[bk - 3];
        const std::vector<double> &qk = kk < 3 ? qs[1] : qs[0];
        const std::vector<int> &kl = cs.kets[kk];
        std::vector<long long> &off = cs.off[c];
        off.assign(bra.size() * DFTK_HLC_NB + 1, 0);
        for (size_t i = 0; i < bra.size(); ++i) {
            const int r = bra[i];
            for (int b = 0; b < DFTK_HLC_NB; ++b) {
                long long lo = cs.seg[kk][b], hi = cs.seg[kk][b + 1], cnt = 0;
                if (qs[0][r] > 0.0) {
                    const double thr = tau / qs[0][r];
                    long long x = lo, y = hi;  // first ket of the segment with q < thr
                    while (x < y) {
                        const long long mid = (x + y) / 2;
                        if (qk[kl[mid]] >= thr) x = mid + 1;
                        else y = mid;
                    }
                    long long end = x;
                    if (bk == kk) {  // same pair set: kets whose row is <= the bra's
                        long long u = lo, v = hi;
                        while (u < v) {
                            const long long mid = (u + v) / 2;
                            if (kl[mid] <= r) u = mid + 1;
                            else v = mid;
                        }
                        end = std::min(end, u);
                    }
                    cnt = end - lo;
                }
                off[i * DFTK_HLC_NB + b + 1] = off[i * DFTK_HLC_NB + b] + cnt;
            }
        }
    }
}

}  // namespace

int dftk_internal_fail_cuda(cudaError_t e, const char *where) { return fail_cuda(e, where); }

extern "C" {

int dftk_prepare_hl_bytes(const dftk_shells_t *shells, size_t *bytes)
{
    if (!shells || !bytes || shells->n_shells < 0 || (shells->n_shells > 0 && (!shells->l || !shells->nprim)))
        return fail(DFTK_ERR_ARG, "dftk_prepare_hl_bytes: bad arguments");
    if (shells->n_mol > 0) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare_hl_bytes: one molecule at a time");
    DFTK_INIT();
    PrepareHlPlan pl;
    const int st = prepare_hl_plan(shells, pl);
    if (st != DFTK_OK) return st;
    *bytes = pl.bytes;
    return DFTK_OK;
}

int dftk_prepare_hl(const dftk_shells_t *shells, double tau_schwarz, double tau_prim, void *storage,
                    size_t storage_bytes, dftk_hl_t *hl, dftk_stream_t stream)
{
    if (!shells || !hl || !(tau_schwarz >= 0.0) || !(tau_prim >= 0.0) || shells->n_shells < 0 ||
        (shells->n_shells > 0 && (!shells->l || !shells->nprim)))
        return fail(DFTK_ERR_ARG, "dftk_prepare_hl: bad arguments");
    if (shells->n_mol > 0) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare_hl: one molecule at a time");
    DFTK_INIT();
    cudaStream_t s = (cudaStream_t)stream;
    DFTK_CUDA(cudaStreamSynchronize(s));
    PrepareHlPlan pl;
    int st = prepare_hl_plan(shells, pl);
    if (st != DFTK_OK) return st;
    if (!storage || storage_bytes < pl.bytes) return fail(DFTK_ERR_WORKSPACE, "dftk_prepare_hl: storage too small");
    char *base = (char *)storage;
    std::vector<double> qs[2];
    dftk_pairs_t *sets[2] = {&hl->hi, &hl->lo};
    for (int k = 0; k < 2; ++k) {
        dftk_pairs_t &P = *sets[k];
        std::vector<int> &ab = pl.ab[k];
        const int n = (int)(ab.size() / 2);
        memset(&P, 0, sizeof(P));
        P.n_pairs = n;
        P.kmax = pl.kmax;
        P.ab = (const int *)(base + pl.off_ab[k]);
        P.nprim = (int *)(base + pl.off_np[k]);
        P.rec64 = (double *)(base + pl.off_r64[k]);
        P.rec32 = (float *)(base + pl.off_r32[k]);
        P.q = (double *)(base + pl.off_q[k]);
        P.qp = (float *)(base + pl.off_qp[k]);
        if (n == 0) continue;
        for (int pass = 0; pass < 2; ++pass) {
            DFTK_CUDA(cudaMemcpyAsync(base + pl.off_ab[k], ab.data(), sizeof(int) * ab.size(), cudaMemcpyHostToDevice, s));
            if ((st = dftk_pair_data(shells, DFTK_PCLASS_GENERIC, &P, stream)) != DFTK_OK) return st;
            if ((st = dftk_hl_schwarz(shells, &P, pl.lmax, stream)) != DFTK_OK) return st;
            qs[k].assign(n, 0.0);
            DFTK_CUDA(cudaMemcpyAsync(qs[k].data(), P.q, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            DFTK_CUDA(cudaStreamSynchronize(s));
            if (pass == 1) break;
            std::vector<int> order(n);
            for (int i = 0; i < n; ++i) order[i] = i;
            const std::vector<double> &q = qs[k];
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return q[x] > q[y]; });
            std::vector<int> sorted(ab.size());
            for (int i = 0; i < n; ++i) {
                sorted[2 * i] = ab[2 * order[i]];
                sorted[2 * i + 1] = ab[2 * order[i] + 1];
            }
            ab.swap(sorted);
        }
    }
    std::vector<long long> off_lo = prefix_offsets(qs[0], qs[1], false, tau_schwarz);
    std::vector<long long> off_hi = prefix_offsets(qs[0], qs[0], true, tau_schwarz);
    // thread-per-quartet classes
    ClassSpaces cs;
    class_spaces(pl.l, pl.np, pl.ab, qs, tau_schwarz, cs);
    for (int c = 0; c < HLC_N_CLASSES; ++c) {
        hl->cls_off[c] = (const long long *)(base + pl.off_cls_off[c]);
        hl->cls_total[c] = cs.off[c].back();
        DFTK_CUDA(cudaMemcpyAsync(base + pl.off_cls_off[c], cs.off[c].data(), sizeof(long long) * cs.off[c].size(),
                                  cudaMemcpyHostToDevice, s));
    }
    for (int x = 0; x < 3; ++x) {
        hl->cls_rows[x] = (const int *)(base + pl.off_cls_rows[x]);
        hl->n_cls_rows[x] = (long long)cs.rows[x].size();
        if (!cs.rows[x].empty())
            DFTK_CUDA(cudaMemcpyAsync(base + pl.off_cls_rows[x], cs.rows[x].data(), sizeof(int) * cs.rows[x].size(),
                                      cudaMemcpyHostToDevice, s));
    }
    for (int y = 0; y < HLC_N_KINDS; ++y) {
        hl->cls_kets[y] = (const int *)(base + pl.off_cls_kets[y]);
        for (int b = 0; b <= DFTK_HLC_NB; ++b) hl->cls_ket_seg[y][b] = cs.seg[y][b];
        if (!cs.kets[y].empty())
            DFTK_CUDA(cudaMemcpyAsync(base + pl.off_cls_kets[y], cs.kets[y].data(), sizeof(int) * cs.kets[y].size(),
                                      cudaMemcpyHostToDevice, s));
    }
    {
        std::vector<long long> cnt(qs[0].size());
        for (size_t r = 0; r < cnt.size(); ++r) cnt[r] = off_lo[r + 1] - off_lo[r];
        for (int x = 0; x < 3; ++x) {
            // rows of kind x leave (hi|lo) when classes (x|ss), (x|ps), (x|pp) all exist
            int n = 0;
            for (int c = 0; c < HLC_N_CLASSES; ++c) n += hlc_class_kinds[c][0] == x + 3 && hlc_class_kinds[c][1] < 3;
            if (n == 3)
                for (int r : cs.rows[x]) cnt[r] = 0;
        }
        for (size_t r = 0; r < cnt.size(); ++r) off_lo[r + 1] = off_lo[r] + cnt[r];
        // (hi|hi) likewise, for rows of a kind that has a class with every
        // hi kind, when no hi pair has an f shell
        bool has_f = false;
        for (size_t r = 0; r < qs[0].size(); ++r) has_f = has_f || pl.l[pl.ab[0][2 * r]] > 2;
        for (size_t r = 0; r < cnt.size(); ++r) cnt[r] = off_hi[r + 1] - off_hi[r];
        for (int x = 0; x < 3 && !has_f; ++x) {
            int n = 0;
            for (int c = 0; c < HLC_N_CLASSES; ++c) {
                const int bk = hlc_class_kinds[c][0], kk = hlc_class_kinds[c][1];
                n += (bk == x + 3 && kk >= 3) || (kk == x + 3 && bk >= 3 && bk != kk);
            }
            if (n == 3)
                for (int r : cs.rows[x]) cnt[r] = 0;
        }
        for (size_t r = 0; r < cnt.size(); ++r) off_hi[r + 1] = off_hi[r] + cnt[r];
    }
    long long *d_lo = (long long *)(base + pl.off_row[0]), *d_hi = (long long *)(base + pl.off_row[1]);
    DFTK_CUDA(cudaMemcpyAsync(d_lo, off_lo.data(), sizeof(long long) * off_lo.size(), cudaMemcpyHostToDevice, s));
    DFTK_CUDA(cudaMemcpyAsync(d_hi, off_hi.data(), sizeof(long long) * off_hi.size(), cudaMemcpyHostToDevice, s));
    hl->n_rows = (long long)qs[0].size();
    hl->total[0] = off_lo.back();
    hl->total[1] = off_hi.back();
    hl->row_off[0] = d_lo;
    hl->row_off[1] = d_hi;
    hl->tau_prim = tau_prim;
    hl->lmax = pl.lmax;
    DFTK_CUDA(cudaStreamSynchronize(s));  // the host vectors above are sources of the copies
    return DFTK_OK;
}

int dftk_prepare_bytes(const dftk_shells_t *shells, size_t *bytes)
{
    if (!shells || !bytes || shells->n_shells < 0 || (shells->n_shells > 0 && (!shells->l || !shells->nprim)))
        return fail(DFTK_ERR_ARG, "dftk_prepare_bytes: bad arguments");
    if (shells->n_mol > 0) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare_bytes: one molecule at a time");
    DFTK_INIT();
    PreparePlan pl;
    const int st = prepare_plan(shells, pl);
    if (st != DFTK_OK) return st;
    *bytes = pl.bytes;
    return DFTK_OK;
}

int dftk_prepare(const dftk_shells_t *shells, double tau_schwarz, double tau_prim, void *storage,
                 size_t storage_bytes, dftk_pairs_t pairs[DFTK_N_PCLASS], dftk_queue_t *queue, dftk_stream_t stream)
{
    if (!shells || !pairs || !queue || !(tau_schwarz >= 0.0) || !(tau_prim >= 0.0) || shells->n_shells < 0 ||
        (shells->n_shells > 0 && (!shells->l || !shells->nprim)))
        return fail(DFTK_ERR_ARG, "dftk_prepare: bad arguments");
    if (shells->n_mol > 0) return fail(DFTK_ERR_UNSUPPORTED, "dftk_prepare: one molecule at a time");
    DFTK_INIT();
    cudaStream_t s = (cudaStream_t)stream;
    DFTK_CUDA(cudaStreamSynchronize(s));  // the shell arrays may still be in flight on the caller's stream
    PreparePlan pl;
    int st = prepare_plan(shells, pl);
    if (st != DFTK_OK) return st;
    if (!storage || storage_bytes < pl.bytes) return fail(DFTK_ERR_WORKSPACE, "dftk_prepare: storage too small");
    char *base = (char *)storage;
    std::vector<double> qs[DFTK_N_PCLASS];
    for (int pc = 0; pc < DFTK_N_PCLASS; ++pc) {
        dftk_pairs_t &P = pairs[pc];
        std::vector<int> &ab = pl.ab[pc];
        const int n = (int)(ab.size() / 2);
        P.n_pairs = n;
        P.kmax = pl.kmax;
        P.ab = (const int *)(base + pl.off_ab[pc]);
        P.nprim = (int *)(base + pl.off_np[pc]);
        P.rec64 = (double *)(base + pl.off_r64[pc]);
        P.rec32 = (float *)(base + pl.off_r32[pc]);
        P.q = (double *)(base + pl.off_q[pc]);
        P.qp = (float *)(base + pl.off_qp[pc]);
        P.core64 = (double *)(base + pl.off_c64[pc]);
        P.core32 = (float *)(base + pl.off_c32[pc]);
        if (n == 0) continue;
        // Schwarz factors in enumeration order, then the pairs sorted by
        // descending factor (stable) and their records rebuilt in that order
        for (int pass = 0; pass < 2; ++pass) {
            DFTK_CUDA(cudaMemcpyAsync(base + pl.off_ab[pc], ab.data(), sizeof(int) * ab.size(), cudaMemcpyHostToDevice, s));
            if ((st = dftk_pair_data(shells, pc, &P, stream)) != DFTK_OK) return st;
            if ((st = dftk_schwarz(shells, pc, &P, stream)) != DFTK_OK) return st;
            qs[pc].assign(n, 0.0);
            DFTK_CUDA(cudaMemcpyAsync(qs[pc].data(), P.q, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            DFTK_CUDA(cudaStreamSynchronize(s));
            if (pass == 1) break;
            std::vector<int> order(n);
            for (int i = 0; i < n; ++i) order[i] = i;
            const std::vector<double> &q = qs[pc];
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return q[x] > q[y]; });
            std::vector<int> sorted(ab.size());
            for (int i = 0; i < n; ++i) {
                sorted[2 * i] = ab[2 * order[i]];
                sorted[2 * i + 1] = ab[2 * order[i] + 1];
            }
            ab.swap(sorted);
        }
    }
    // candidate offsets: bra row r keeps the ket prefix with q_ket >= tau / q_bra[r]
    // (the ket factors are sorted descending), cut at k <= r when bra and ket
    // share a pair class so each unique quartet appears once
    for (int c = 0; c < DFTK_N_QCLASS; ++c) {
        const std::vector<double> &qx = qs[kQX[c]], &qy = qs[kQY[c]];
        const size_t nr = pl.ab[kQX[c]].size() / 2, nk = pl.ab[kQY[c]].size() / 2;
        std::vector<long long> off(nr + 1, 0);
        for (size_t r = 0; r < nr; ++r) {
            long long cnt = 0;
            if (nk > 0 && qx[r] > 0.0) {
                const double thr = tau_schwarz / qx[r];
                // first index with qy < thr (qy descending)
                size_t lo = 0, hi = nk;
                while (lo < hi) {
                    const size_t mid = (lo + hi) / 2;
                    if (qy[mid] >= thr) lo = mid + 1;
                    else hi = mid;
                }
                cnt = (long long)lo;
            }
            if (kQX[c] == kQY[c]) cnt = std::min<long long>(cnt, (long long)r + 1);
            off[r + 1] = off[r] + cnt;
        }
        long long *d_off = (long long *)(base + pl.off_row[c]);
        DFTK_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, s));
        queue->total[c] = off[nr];
        queue->n_rows[c] = off[nr] > 0 ? (long long)nr : 0;
        queue->row_off[c] = d_off;
        queue->ket_base[c] = nullptr;
    }
    queue->tau_prim = tau_prim;
    queue->mol_active = nullptr;
    queue->bucket_kets = pl.bucket_kets;
    DFTK_CUDA(cudaStreamSynchronize(s));  // the host vectors above are sources of the copies
    return DFTK_OK;
}

int dftk_one_electron(const dftk_shells_t *shells, int n_atoms, const double *atom_xyz,
                      const double *atom_z, double *S, double *T, double *V, dftk_stream_t stream)
{
    if (!shells || n_atoms < 0 || !S || !T || !V || (n_atoms > 0 && (!atom_xyz || !atom_z)))
        return fail(DFTK_ERR_ARG, "dftk_one_electron: bad arguments");
    DFTK_INIT();
    const long long npair = (long long)shells->n_shells * (shells->n_shells + 1) / 2;
    if (npair == 0) return DFTK_OK;
    k_one_electron<<<blocks_for(npair, 64), 64, 0, (cudaStream_t)stream>>>(*shells, n_atoms, atom_xyz, atom_z, S, T, V);
    DFTK_LAUNCHED("k_one_electron");
    if (!shells->mol) {
        // pairs with a d shell (the kernel returns at once for the others)
        k_one_electron_hl<<<blocks_for(npair, 64), 64, 0, (cudaStream_t)stream>>>(*shells, n_atoms, atom_xyz, atom_z,
                                                                                 S, T, V);
        DFTK_LAUNCHED("k_one_electron_hl");
    }
    return DFTK_OK;
}

int dftk_grid_ao(const dftk_shells_t *shells, long long n_points, const float *points, double *ao, long long ld,
                 dftk_stream_t stream)
{
    if (!shells || n_points < 0 || ld < n_points || (n_points > 0 && (!points || !ao)) || shells->n_shells < 0 ||
        (shells->n_shells > 0 && (!shells->xyz || !shells->l || !shells->nprim || !shells->prim_off || !shells->ao ||
                                  !shells->prim_exp || !shells->prim_cn)))
        return fail(DFTK_ERR_ARG, "dftk_grid_ao: bad arguments");
    if (shells->n_mol > 0) return fail(DFTK_ERR_UNSUPPORTED, "dftk_grid_ao: one molecule at a time");
    DFTK_INIT();
    if (n_points == 0 || shells->n_shells == 0) return DFTK_OK;
    if ((n_points + 127) / 128 > 0x7fffffffLL) return fail(DFTK_ERR_SIZE, "dftk_grid_ao: too many points in one call");
    // momenta beyond f have no AO code here: refuse them before launch
    std::vector<int> l(shells->n_shells);
    DFTK_CUDA(cudaMemcpyAsync(l.data(), shells->l, sizeof(int) * l.size(), cudaMemcpyDeviceToHost,
                              (cudaStream_t)stream));
    DFTK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    for (int v : l)
        if (v < 0 || v > HL_LMAX) return fail(DFTK_ERR_UNSUPPORTED, "dftk_grid_ao: shells beyond f");
    k_grid_ao<<<blocks_for(n_points, 128), 128, 0, (cudaStream_t)stream>>>(*shells, n_points, points, ao, ld);
    DFTK_LAUNCHED("k_grid_ao");
    return DFTK_OK;
}

int dftk_grid_density(int n_mo, int n_a, int n_b, long long n_points, const double *psi_a, const double *psi_b,
                      long long ld_psi, float *total, float *phase, long long ld_out, dftk_stream_t stream)
{
    if (n_mo < 0 || n_mo > 65535 || n_a < 0 || n_b < 0 || n_a > n_mo || n_b > n_mo || n_points < 0 ||
        ld_psi < n_points || ld_out < n_points ||
        (n_points > 0 && n_mo > 0 && (!psi_a || !psi_b || !total || (n_a > 0 && !phase))))
        return fail(DFTK_ERR_ARG, "dftk_grid_density: bad arguments");
    DFTK_INIT();
    if (n_points == 0 || n_mo == 0) return DFTK_OK;
    const long long per_block = 256LL * GRID_DENSITY_UNROLL;
    const long long bx = (n_points + per_block - 1) / per_block;
    if (bx > 0x7fffffffLL) return fail(DFTK_ERR_SIZE, "dftk_grid_density: too many points in one call");
    k_grid_density<<<dim3((unsigned)bx, (unsigned)n_mo), 256, 0, (cudaStream_t)stream>>>(n_a, n_b, n_points, psi_a,
                                                                                         psi_b, ld_psi, total, phase,
                                                                                         ld_out);
    DFTK_LAUNCHED("k_grid_density");
    return DFTK_OK;
}

int dftk_eri_blocks(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS], long long n_quartets,
                    const int *desc, const long long *out_off, double *out, dftk_stream_t stream)
{
    if (!shells || !pairs || n_quartets < 0 || (n_quartets > 0 && (!desc || !out_off || !out)))
        return fail(DFTK_ERR_ARG, "dftk_eri_blocks: bad arguments");
    DFTK_INIT();
    if (n_quartets == 0) return DFTK_OK;
    EmitParams P;
    P.shell_ao = shells->ao;
    P.shell_l = shells->l;
    for (int k = 0; k < 3; ++k) {
        if (pairs[k].n_pairs > 0 && (!pairs[k].core64 || !pairs[k].core32))
            return fail(DFTK_ERR_ARG, "dftk_eri_blocks: pair class without core records");
        P.ab[k] = pairs[k].ab;
        P.np[k] = pairs[k].nprim;
        P.rec64[k] = pairs[k].rec64;
        P.rec32[k] = pairs[k].rec32;
        P.core64[k] = pairs[k].core64;
        P.core32[k] = pairs[k].core32;
        P.qp[k] = pairs[k].qp;
        P.n_pairs[k] = pairs[k].n_pairs;
        P.kmax[k] = pairs[k].kmax;
    }
    P.nq = n_quartets;
    P.desc = desc;
    P.out_off = out_off;
    P.out = out;
    k_emit<<<blocks_for(n_quartets, 64), 64, 0, (cudaStream_t)stream>>>(P);
    DFTK_LAUNCHED("k_emit");
    return DFTK_OK;
}

size_t dftk_jk_workspace_bytes(int n_shells, int n_ao)
{
    if (n_shells < 0 || n_ao < 0) return 0;
    return ws_bytes(n_shells, n_ao);
}

size_t dftk_jk_workspace_bytes_queue(int n_shells, int n_ao, const dftk_queue_t *queue)
{
    if (n_shells < 0 || n_ao < 0 || !queue) return 0;
    return ws_list_bytes(n_shells, n_ao, queue);
}

size_t dftk_workspace_bytes(const dftk_shells_t *shells, const dftk_queue_t *queue)
{
    if (!shells || shells->n_shells < 0 || shells->n_ao < 0) return 0;
    return queue ? ws_list_bytes_sh(*shells, queue) : ws_bytes_sh(*shells);
}

int dftk_jk(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS], const dftk_queue_t *queue,
            const double *D, const double *D_a, const double *D_b, double *J, double *K_a, double *K_b,
            int flags, double tau, double tau_fp32, void *workspace, size_t workspace_bytes,
            long long *counts, dftk_stream_t stream)
{
    if (!shells || !pairs || !queue || !D || !D_a || !J || !K_a || !workspace)
        return fail(DFTK_ERR_ARG, "dftk_jk: null argument");
    const int uhf = (flags & DFTK_JK_UHF) != 0;
    const int mixed = (flags & DFTK_JK_MIXED) != 0;
    if (uhf && (!D_b || !K_b)) return fail(DFTK_ERR_ARG, "dftk_jk: UHF needs D_b and K_b");
    if (!(tau >= 0.0) || (mixed && !(tau_fp32 >= tau))) return fail(DFTK_ERR_ARG, "dftk_jk: bad thresholds");
    if (shells->mol && (shells->n_mol <= 0 || !shells->mol_mat || !shells->mol_nao || !shells->mol_shell0 ||
                        !shells->mol_ns || !shells->mol_dsh))
        return fail(DFTK_ERR_ARG, "dftk_jk: incomplete molecule table");
    if (workspace_bytes < ws_bytes_sh(*shells)) return fail(DFTK_ERR_WORKSPACE, "dftk_jk: workspace too small");
    DFTK_INIT();
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nn = (size_t)shells_mat_elems(*shells);
    double *Y = (double *)workspace;
    double *Za = Y + nn;
    double *Zb = Za + nn;
    float *Dsh = (float *)(Zb + nn);
    DFTK_CUDA(cudaMemsetAsync(Y, 0, 3 * nn * sizeof(double), s));
    int st;
    if ((st = launch_dsh(*shells, D, D_a, uhf ? D_b : D_a, uhf, Dsh, s))) return st;
    JkParams P;
    memset(&P, 0, sizeof(P));
    P.sh = *shells;
    for (int c = 0; c < DFTK_N_QCLASS; ++c) P.ket_base[c] = queue->ket_base[c];
    P.mol_active = queue->mol_active;
    P.bucket = queue->bucket_kets;
    P.shell_ao = shells->ao;
    for (int k = 0; k < 3; ++k) {
        if (pairs[k].n_pairs > 0 && (!pairs[k].core64 || !pairs[k].core32))
            return fail(DFTK_ERR_ARG, "dftk_jk: pair class without core records");
        P.ab[k] = pairs[k].ab;
        P.np[k] = pairs[k].nprim;
        P.rec64[k] = pairs[k].rec64;
        P.rec32[k] = pairs[k].rec32;
        P.core64[k] = pairs[k].core64;
        P.core32[k] = pairs[k].core32;
        P.q[k] = pairs[k].q;
        P.qp[k] = pairs[k].qp;
        P.n_pairs[k] = pairs[k].n_pairs;
        P.kmax[k] = pairs[k].kmax;
    }
    for (int c = 0; c < DFTK_N_QCLASS; ++c) {
        P.n_rows[c] = queue->n_rows[c];
        P.row_off[c] = queue->row_off[c];
        P.total[c] = queue->n_rows[c] > 0 ? queue->total[c] : 0;
        if (P.total[c] < 0) return fail(DFTK_ERR_ARG, "dftk_jk: negative candidate total");
        if (P.total[c] > 0 && !queue->row_off[c]) return fail(DFTK_ERR_ARG, "dftk_jk: missing row offsets");
    }
    P.tau_prim = (float)queue->tau_prim;
    for (int c = 0; c < DFTK_N_QCLASS; ++c)
        for (int p = 0; p < 2; ++p) P.tile[p * DFTK_N_QCLASS + c] = launch_shape(DFTK_FAMILY_JK, c, p).tile;
    P.D = D;
    P.Da = D_a;
    P.Db = uhf ? D_b : D_a;
    P.Y = Y;
    P.Za = Za;
    P.Zb = Zb;
    P.Dsh = Dsh;
    P.uhf = uhf;
    if (workspace_bytes >= ws_list_bytes_sh(*shells, queue)) {
        // selection pass + list-driven class kernels
        unsigned char *cur = (unsigned char *)workspace + ws_bytes_sh(*shells);
        P.heads = (unsigned long long *)cur;
        cur += 256;
        for (int c = 0; c < DFTK_N_QCLASS; ++c) {
            P.list[c] = (int2 *)cur;
            if (P.total[c] > 0) cur += (((size_t)P.total[c] * sizeof(int2)) + 255) & ~(size_t)255;
        }
        // list counters, then the persistent kernel's two work counters
        DFTK_CUDA(cudaMemsetAsync(P.heads, 0, (2 * DFTK_N_QCLASS + 2) * sizeof(unsigned long long), s));
        P.tau = tau;
        P.tau32 = mixed ? tau_fp32 : tau;
        P.counts = counts;
        if (flags & DFTK_JK_PERSIST) {
            // one selection launch over every class, then one persistent launch per precision
            long long tiles = 0;
            for (int c = 0; c < DFTK_N_QCLASS; ++c) tiles += (P.total[c] + SELECT_TILE - 1) / SELECT_TILE;
            if (tiles > 0) {
                long long sb = tiles < 148LL * 8 ? tiles : 148LL * 8;
                k_select_all<<<(unsigned)sb, SELECT_THREADS, 0, s>>>(P);
                DFTK_LAUNCHED("k_select_all");
                if ((st = launch_jk_persist<double>(P, s))) return st;
                if (mixed) {
                    P.counts = counts ? counts + DFTK_N_QCLASS : nullptr;
                    if ((st = launch_jk_persist<float>(P, s))) return st;
                }
            }
            return launch_symmetrize(*shells, Y, Za, Zb, J, K_a, K_b, uhf, s);
        }
        // per class on its stream: selection, then the FP64 (and FP32) list kernel
        cudaStream_t cls[DFTK_N_QCLASS];
        int n_aux = 0;
        int dev = 0;
        DFTK_CUDA(cudaGetDevice(&dev));
        std::unique_lock<std::mutex> fork_lock(g_pool[dev].mutex);
        if ((st = fork_class_streams(s, cls, n_aux))) return st;
        if ((st = launch_class_pipeline<1>(P, mixed, counts, cls[1]))) return st;
        if ((st = launch_class_pipeline<0>(P, mixed, counts, cls[0]))) return st;
        if ((st = launch_class_pipeline<2>(P, mixed, counts, cls[2]))) return st;
        if ((st = launch_class_pipeline<3>(P, mixed, counts, cls[3]))) return st;
        if ((st = launch_class_pipeline<4>(P, mixed, counts, cls[4]))) return st;
        if ((st = launch_class_pipeline<5>(P, mixed, counts, cls[5]))) return st;
        if ((st = join_class_streams(s, n_aux))) return st;
        return launch_symmetrize(*shells, Y, Za, Zb, J, K_a, K_b, uhf, s);
    }
    P.tau_lo = tau;
    P.tau_hi = INFINITY;
    if (mixed) {
        P.tau_lo = tau_fp32;
        P.counts = counts;
        if ((st = launch_jk_all<double>(P, s))) return st;
        P.tau_lo = tau;
        P.tau_hi = tau_fp32;
        P.counts = counts ? counts + DFTK_N_QCLASS : nullptr;
        if ((st = launch_jk_all<float>(P, s))) return st;
    } else {
        P.counts = counts;
        if ((st = launch_jk_all<double>(P, s))) return st;
    }
    return launch_symmetrize(*shells, Y, Za, Zb, J, K_a, K_b, uhf, s);
}

}  // extern "C"

namespace {
// Shared scratch of the d/f kernels: the LM = 2 layout fits the default
// 48 KB, the LM = 3 one needs the opt-in (set before each launch).
template <int LM, typename K> int hl_smem_optin(K kernel, size_t extra_static = 0)
{
    const size_t bytes = sizeof(HlScratch<LM>);
    if (bytes + extra_static > 48 * 1024)
        DFTK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return DFTK_OK;
}

// One class kernel of the thread-per-quartet d classes: 128-thread blocks,
// a grid of at most 16 resident blocks per SM striding over the class's
// warp work items (32 candidates x ket-component split).
static_assert(HLC_N_CLASSES == sizeof(((dftk_hl_t *)nullptr)->cls_off) / sizeof(void *),
              "dftk_hl_t holds one candidate space per generated d class");
}  // namespace

extern "C" {

int dftk_hl_schwarz(const dftk_shells_t *shells, dftk_pairs_t *pairs, int lmax, dftk_stream_t stream)
{
    if (!shells || !pairs || !pairs->qp || !pairs->q || !pairs->rec64 || !pairs->rec32 || pairs->n_pairs < 0 ||
        lmax < 0 || lmax > HL_LMAX)
        return fail(DFTK_ERR_ARG, "dftk_hl_schwarz: bad arguments (lmax 0..3)");
    if (pairs->kmax > HL_MAX_KPAIR) return fail(DFTK_ERR_SIZE, "dftk_hl_schwarz: more than 128 primitive pairs per pair");
    if (shells->mol) return fail(DFTK_ERR_UNSUPPORTED, "dftk_hl_schwarz: one molecule at a time");
    DFTK_INIT();
    if (pairs->n_pairs == 0) return DFTK_OK;
    int st;
    if (lmax <= 2) {
        k_hl_schwarz<2><<<(unsigned)pairs->n_pairs, 32, sizeof(HlScratch<2>), (cudaStream_t)stream>>>(*shells, *pairs);
    } else {
        if ((st = hl_smem_optin<3>(k_hl_schwarz<3>, 4096))) return st;
        k_hl_schwarz<3><<<(unsigned)pairs->n_pairs, 32, sizeof(HlScratch<3>), (cudaStream_t)stream>>>(*shells, *pairs);
    }
    DFTK_LAUNCHED("k_hl_schwarz");
    return DFTK_OK;
}

int dftk_jk_hl(const dftk_shells_t *shells, const dftk_hl_t *hl, const double *D, const double *D_a,
               const double *D_b, double *J, double *K_a, double *K_b, int flags, double tau, void *workspace,
               size_t workspace_bytes, long long *counts, dftk_stream_t stream)
{
    if (!shells || !hl || !D || !D_a || !J || !K_a || !workspace) return fail(DFTK_ERR_ARG, "dftk_jk_hl: null argument");
    const int uhf = (flags & DFTK_JK_UHF) != 0;
    if (uhf && (!D_b || !K_b)) return fail(DFTK_ERR_ARG, "dftk_jk_hl: UHF needs D_b and K_b");
    if (!(tau >= 0.0)) return fail(DFTK_ERR_ARG, "dftk_jk_hl: bad threshold");
    if (shells->mol) return fail(DFTK_ERR_UNSUPPORTED, "dftk_jk_hl: one molecule at a time");
    if (hl->lmax < 2 || hl->lmax > HL_LMAX || hl->n_rows < 0 || hl->n_rows != hl->hi.n_pairs || hl->total[0] < 0 ||
        hl->total[1] < 0 ||
        ((hl->total[0] > 0 || hl->total[1] > 0) && (!hl->row_off[0] || !hl->row_off[1])))
        return fail(DFTK_ERR_ARG, "dftk_jk_hl: inconsistent candidate spaces");
    if (workspace_bytes < ws_bytes(shells->n_shells, shells->n_ao))
        return fail(DFTK_ERR_WORKSPACE, "dftk_jk_hl: workspace too small");
    long long cls_sum = 0;
    unsigned long long cover = 0;
    for (int c = 0; c < HLC_N_CLASSES; ++c) {
        const int bk = hlc_class_kinds[c][0], kk = hlc_class_kinds[c][1];
        const long long nb = hl->n_cls_rows[bk - 3], nk = hl->cls_ket_seg[kk][DFTK_HLC_NB];
        bool seg_ok = hl->cls_ket_seg[kk][0] == 0;
        for (int b = 0; b < DFTK_HLC_NB; ++b) seg_ok = seg_ok && hl->cls_ket_seg[kk][b] <= hl->cls_ket_seg[kk][b + 1];
        if (hl->cls_total[c] < 0 ||
            (hl->cls_total[c] > 0 && (!hl->cls_off[c] || !hl->cls_rows[bk - 3] || !hl->cls_kets[kk] || !seg_ok ||
                                      nb <= 0 || nb > hl->n_rows || nk <= 0 ||
                                      nk > (kk < 3 ? hl->lo.n_pairs : hl->n_rows))))
            return fail(DFTK_ERR_ARG, "dftk_jk_hl: inconsistent class spaces");
        cls_sum += hl->cls_total[c];
        if (hl->cls_off[c]) cover |= (1ull << (6 * bk + kk)) | (1ull << (6 * kk + bk));
    }
    DFTK_INIT();
    const long long total = hl->total[0] + hl->total[1];
    if ((total == 0 && cls_sum == 0) || hl->n_rows == 0) return DFTK_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int N = shells->n_ao;
    const size_t nn = (size_t)N * N;
    double *Y = (double *)workspace;
    double *Za = Y + nn;
    double *Zb = Za + nn;
    float *Dsh = (float *)(Zb + nn);
    DFTK_CUDA(cudaMemsetAsync(Y, 0, 3 * nn * sizeof(double), s));
    int st;
    if ((st = launch_dsh(*shells, D, D_a, uhf ? D_b : D_a, uhf, Dsh, s))) return st;
    HlJkParams P;
    memset(&P, 0, sizeof(P));
    P.sh = *shells;
    P.hi = hl->hi;
    P.lo = hl->lo;
    P.n_rows = hl->n_rows;
    for (int k = 0; k < 2; ++k) {
        P.total[k] = hl->total[k];
        P.row_off[k] = hl->row_off[k];
    }
    P.tau_prim = (float)hl->tau_prim;
    P.D = D;
    P.Da = D_a;
    P.Db = uhf ? D_b : D_a;
    P.Y = Y;
    P.Za = Za;
    P.Zb = Zb;
    P.Dsh = Dsh;
    P.uhf = uhf;
    P.tau = tau;
    P.counts = counts;
    P.cover = cover;
    if (cls_sum > 0) {
        HlcParams C;
        memset(&C, 0, sizeof(C));
        C.sh = *shells;
        C.shell_ao = shells->ao;
        C.hi = hl->hi;
        C.lo = hl->lo;
        for (int x = 0; x < 3; ++x) {
            C.rows[x] = hl->cls_rows[x];
            C.n_rows[x] = hl->n_cls_rows[x];
        }
        for (int y = 0; y < HLC_N_KINDS; ++y) {
            C.kets[y] = hl->cls_kets[y];
            for (int b = 0; b <= DFTK_HLC_NB; ++b) C.seg[y][b] = hl->cls_ket_seg[y][b];
        }
        for (int c = 0; c < HLC_N_CLASSES; ++c) {
            C.off[c] = hl->cls_off[c];
            C.total[c] = hl->cls_total[c];
        }
        C.tau_prim = (float)hl->tau_prim;
        C.D = D;
        C.Da = D_a;
        C.Db = uhf ? D_b : D_a;
        C.Y = Y;
        C.Za = Za;
        C.Zb = Zb;
        C.Dsh = Dsh;
        C.uhf = uhf;
        C.tau = tau;
        C.counts = counts;
        // the library's class streams (as dftk_jk forks them), joined below
        cudaStream_t cls[DFTK_N_QCLASS];
        int n_aux = 0, dev = 0, next = 0;
        DFTK_CUDA(cudaGetDevice(&dev));
        std::unique_lock<std::mutex> fork_lock(g_pool[dev].mutex);
        if ((st = fork_class_streams(s, cls, n_aux))) return st;
        cudaStream_t sts[4] = {s, s, s, s};
        int ns = 1;
        for (int c = 0; c < DFTK_N_QCLASS && ns < 4; ++c) {
            bool seen = false;
            for (int k = 0; k < ns; ++k) seen = seen || sts[k] == cls[c];
            if (!seen) sts[ns++] = cls[c];
        }
        // the chunk kernels live in the separately compiled hlc_part_*.cu units
        if ((st = hlc_part_a_launch(C, sts, ns, next)) || (st = hlc_part_b_launch(C, sts, ns, next)) ||
            (st = hlc_part_c_launch(C, sts, ns, next)) || (st = hlc_part_d_launch(C, sts, ns, next)))
            return st;
        if ((st = join_class_streams(s, n_aux))) return st;
    }
    if (total > 0) {
        long long blocks = total;
        // one-warp blocks: 8 per SM with the d layout (26.6 KB shared each), 1 with the f one (167 KB)
        const long long cap = (long long)sm_count() * (hl->lmax <= 2 ? 8 : 1);
        if (blocks > cap) blocks = cap;
        if (hl->lmax <= 2) {
            k_hl_jk<2><<<(unsigned)blocks, 32, sizeof(HlScratch<2>), s>>>(P);
        } else {
            if ((st = hl_smem_optin<3>(k_hl_jk<3>))) return st;
            k_hl_jk<3><<<(unsigned)blocks, 32, sizeof(HlScratch<3>), s>>>(P);
        }
        DFTK_LAUNCHED("k_hl_jk");
    }
    long long bx = ((long long)nn + 255) / 256;
    if (bx > 148 * 8) bx = 148 * 8;
    k_symmetrize_add<<<(unsigned)bx, 256, 0, s>>>(N, Y, Za, Zb, J, K_a, K_b, uhf);
    DFTK_LAUNCHED("k_symmetrize_add");
    return DFTK_OK;
}

int dftk_hl_eri_blocks(const dftk_shells_t *shells, const dftk_hl_t *hl, long long n_quartets, const int *desc,
                       const long long *out_off, double *out, dftk_stream_t stream)
{
    if (!shells || !hl || n_quartets < 0 || (n_quartets > 0 && (!desc || !out_off || !out)) || hl->lmax < 2 ||
        hl->lmax > HL_LMAX)
        return fail(DFTK_ERR_ARG, "dftk_hl_eri_blocks: bad arguments");
    DFTK_INIT();
    if (n_quartets == 0) return DFTK_OK;
    long long blocks = n_quartets;
    const long long cap = (long long)sm_count() * (hl->lmax <= 2 ? 8 : 1);
    if (blocks > cap) blocks = cap;
    cudaStream_t s = (cudaStream_t)stream;
    if (hl->lmax <= 2) {
        k_hl_emit<2><<<(unsigned)blocks, 32, sizeof(HlScratch<2>), s>>>(*shells, hl->hi, hl->lo, n_quartets, desc,
                                                                        out_off, out);
    } else {
        int st;
        if ((st = hl_smem_optin<3>(k_hl_emit<3>))) return st;
        k_hl_emit<3><<<(unsigned)blocks, 32, sizeof(HlScratch<3>), s>>>(*shells, hl->hi, hl->lo, n_quartets, desc,
                                                                        out_off, out);
    }
    DFTK_LAUNCHED("k_hl_emit");
    return DFTK_OK;
}

int dftk_jk_timing(int enable)
{
    std::lock_guard<std::mutex> lock(g_timing_mutex);
    if (enable && !g_timing.created) {
        for (int k = 0; k < DFTK_TIMING_SLOTS; ++k) {
            DFTK_CUDA(cudaEventCreate(&g_timing.start[k]));
            DFTK_CUDA(cudaEventCreate(&g_timing.stop[k]));
        }
        g_timing.created = true;
    }
    g_timing.enabled = enable != 0;
    for (int k = 0; k < DFTK_TIMING_SLOTS; ++k) g_timing.launched[k] = false;
    return DFTK_OK;
}

int dftk_jk_timing_read(float *ms, int n)
{
    if (!ms || n < 2 * DFTK_N_QCLASS) return fail(DFTK_ERR_ARG, "dftk_jk_timing_read: need 12 floats");
    std::lock_guard<std::mutex> lock(g_timing_mutex);
    const int nslots = n < DFTK_TIMING_SLOTS ? n : DFTK_TIMING_SLOTS;
    for (int k = 0; k < nslots; ++k) {
        ms[k] = 0.0f;
        if (g_timing.created && g_timing.launched[k]) {
            DFTK_CUDA(cudaEventSynchronize(g_timing.stop[k]));
            DFTK_CUDA(cudaEventElapsedTime(&ms[k], g_timing.start[k], g_timing.stop[k]));
        }
    }
    return DFTK_OK;
}

int dftk_set_launch(int family, int qclass, int fp32, int threads, int blocks_per_sm)
{
    if (family < 0 || family >= DFTK_N_FAMILY || qclass < 0 || qclass >= DFTK_N_QCLASS || (fp32 != 0 && fp32 != 1))
        return fail(DFTK_ERR_ARG, "dftk_set_launch: bad family / class / precision");
    if ((threads != 64 && threads != 128) || blocks_per_sm < 1 || blocks_per_sm > 32)
        return fail(DFTK_ERR_ARG, "dftk_set_launch: threads must be 64 or 128, blocks_per_sm 1..32");
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    init_shapes_locked();
    g_shape[family][qclass][fp32].threads = threads;
    g_shape[family][qclass][fp32].blocks_per_sm = blocks_per_sm;
    return DFTK_OK;
}

int dftk_set_tile(int qclass, int fp32, int tile)
{
    if (qclass < 0 || qclass >= DFTK_N_QCLASS || (fp32 != 0 && fp32 != 1) || (tile != 1 && tile != 2 && tile != 4 &&
                                                                               tile != 8))
        return fail(DFTK_ERR_ARG, "dftk_set_tile: bad class / precision, or tile not 1, 2, 4, 8");
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    init_shapes_locked();
    g_shape[DFTK_FAMILY_JK][qclass][fp32].tile = tile;
    return DFTK_OK;
}

int dftk_get_tile(int qclass, int fp32, int *tile)
{
    if (qclass < 0 || qclass >= DFTK_N_QCLASS || (fp32 != 0 && fp32 != 1) || !tile)
        return fail(DFTK_ERR_ARG, "dftk_get_tile: bad arguments");
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    init_shapes_locked();
    *tile = g_shape[DFTK_FAMILY_JK][qclass][fp32].tile;
    return DFTK_OK;
}

int dftk_get_launch(int family, int qclass, int fp32, int *threads, int *blocks_per_sm)
{
    if (family < 0 || family >= DFTK_N_FAMILY || qclass < 0 || qclass >= DFTK_N_QCLASS || (fp32 != 0 && fp32 != 1) ||
        !threads || !blocks_per_sm)
        return fail(DFTK_ERR_ARG, "dftk_get_launch: bad arguments");
    std::lock_guard<std::mutex> lock(g_shape_mutex);
    init_shapes_locked();
    *threads = g_shape[family][qclass][fp32].threads;
    *blocks_per_sm = g_shape[family][qclass][fp32].blocks_per_sm;
    return DFTK_OK;
}

int dftk_grad(const dftk_shells_t *shells, const int *shell_atom, int n_atoms, const double *atom_xyz,
              const double *atom_z, const dftk_pairs_t pairs[DFTK_N_PCLASS], const dftk_queue_t *queue,
              const double *D, const double *D_a, const double *D_b, const double *W, double tau, double tau_fp32,
              double *grad, void *workspace, size_t workspace_bytes, dftk_stream_t stream)
{
    if (!shells || !shell_atom || n_atoms <= 0 || !atom_xyz || !atom_z || !pairs || !queue || !D || !D_a || !D_b ||
        !W || !grad || !workspace)
        return fail(DFTK_ERR_ARG, "dftk_grad: null argument");
    const int ns = shells->n_shells;
    if (workspace_bytes < ws_bytes_sh(*shells)) return fail(DFTK_ERR_WORKSPACE, "dftk_grad: workspace too small");
    if (!(tau >= 0.0)) return fail(DFTK_ERR_ARG, "dftk_grad: bad threshold");
    const bool mixed = tau_fp32 > tau;
    DFTK_INIT();
    cudaStream_t s = (cudaStream_t)stream;
    // same workspace layout as dftk_jk: Dsh after three N x N blocks, then
    // the selection heads and lists when the workspace holds them
    float *Dsh = (float *)((double *)workspace + 3 * (size_t)shells_mat_elems(*shells));
    const bool use_list = workspace_bytes >= ws_list_bytes_sh(*shells, queue);
    DFTK_CUDA(cudaMemsetAsync(grad, 0, 3 * sizeof(double) * n_atoms, s));
    if (ns == 0) return DFTK_OK;
    // block-private gradient copies in shared memory when they fit
    const size_t smem = n_atoms <= GRAD_SMEM_ATOMS ? 3 * sizeof(double) * n_atoms : 0;
    const long long cap = (long long)sm_count() * 8;
    const int nat_stride = shells->mol ? shells->max_natom : n_atoms;
    auto grid = [cap](long long work) {
        long long b = (work + GRAD_THREADS - 1) / GRAD_THREADS;
        return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
    };
    {
        const int st = launch_dsh(*shells, D, D_a, D_b, 1, Dsh, s);
        if (st) return st;
    }
    // with dftk_jk_timing on: slots 0..5 time the class kernels, slot 6 the one-electron part
    const bool timed = g_timing.enabled;
    if (timed) {
        for (int k = 0; k < DFTK_TIMING_SLOTS; ++k) g_timing.launched[k] = false;
        DFTK_CUDA(cudaEventRecord(g_timing.start[2 * DFTK_N_QCLASS], s));
    }
#define DFTK_GRAD_ONEE(PC)                                                                                   \
    if (pairs[PC].n_pairs > 0) {                                                                             \
        k_grad_overlap_kinetic<PC><<<grid(pairs[PC].n_pairs), GRAD_THREADS, smem, s>>>(                       \
            *shells, pairs[PC].ab, pairs[PC].n_pairs, shell_atom, n_atoms, D, W, grad);                      \
        DFTK_LAUNCHED("k_grad_overlap_kinetic");                                                             \
        k_grad_nuclear<PC><<<grid((long long)pairs[PC].n_pairs * nat_stride), GRAD_THREADS, smem, s>>>(      \
            *shells, pairs[PC].ab, pairs[PC].n_pairs, shell_atom, n_atoms, atom_xyz, atom_z, D, grad);       \
        DFTK_LAUNCHED("k_grad_nuclear");                                                                     \
    }
    DFTK_GRAD_ONEE(0)
    DFTK_GRAD_ONEE(1)
    DFTK_GRAD_ONEE(2)
#undef DFTK_GRAD_ONEE
    if (timed) {
        DFTK_CUDA(cudaEventRecord(g_timing.stop[2 * DFTK_N_QCLASS], s));
        g_timing.launched[2 * DFTK_N_QCLASS] = true;
    }
    GradParams P;
    memset(&P, 0, sizeof(P));
    P.sh = *shells;
    P.shell_atom = shell_atom;
    P.n_atoms = n_atoms;
    P.kmax = pairs[0].kmax;
    for (int k = 0; k < 3; ++k) {
        if (pairs[k].kmax != P.kmax) return fail(DFTK_ERR_ARG, "dftk_grad: pair classes with different kmax");
        P.ab[k] = pairs[k].ab;
        P.q[k] = pairs[k].q;
        P.rec[k] = pairs[k].rec64;
        P.rec32[k] = pairs[k].rec32;
        P.nprim[k] = pairs[k].nprim;
        P.n_pairs[k] = pairs[k].n_pairs;
    }
    for (int c = 0; c < DFTK_N_QCLASS; ++c) {
        P.n_rows[c] = queue->n_rows[c];
        P.total[c] = queue->n_rows[c] > 0 ? queue->total[c] : 0;
        P.row_off[c] = queue->row_off[c];
    }
    P.D = D;
    P.Da = D_a;
    P.Db = D_b;
    P.Dsh = Dsh;
    P.tau = tau;
    P.grad = grad;
    P.tau_prim = (float)queue->tau_prim;
    for (int k = 0; k < 3; ++k) P.qp[k] = pairs[k].qp;
    for (int c = 0; c < DFTK_N_QCLASS; ++c) P.ket_base[c] = queue->ket_base[c];
    if (use_list) {
        // selection pass of dftk_jk with the gradient bound Q_ab Q_cd max|D|^2 >= tau
        JkParams S;
        memset(&S, 0, sizeof(S));
        S.sh = *shells;
        for (int c = 0; c < DFTK_N_QCLASS; ++c) S.ket_base[c] = queue->ket_base[c];
        S.mol_active = queue->mol_active;
        for (int k = 0; k < 3; ++k) {
            S.ab[k] = pairs[k].ab;
            S.q[k] = pairs[k].q;
            S.np[k] = pairs[k].nprim;  // the selection groups survivors by the ket's primitive count
        }
        S.bucket = queue->bucket_kets;
        for (int c = 0; c < DFTK_N_QCLASS; ++c) {
            S.n_rows[c] = P.n_rows[c];
            S.row_off[c] = P.row_off[c];
            S.total[c] = P.total[c];
        }
        S.Dsh = Dsh;
        S.tau = tau;
        S.tau32 = mixed ? tau_fp32 : tau;  // FP32 entries: tau <= bound < tau_fp32
        S.dm_pow2 = 1;
        unsigned char *cur = (unsigned char *)workspace + ws_bytes_sh(*shells);
        S.heads = (unsigned long long *)cur;
        cur += 256;
        for (int c = 0; c < DFTK_N_QCLASS; ++c) {
            S.list[c] = (int2 *)cur;
            if (S.total[c] > 0) cur += (((size_t)S.total[c] * sizeof(int2)) + 255) & ~(size_t)255;
        }
        DFTK_CUDA(cudaMemsetAsync(S.heads, 0, 2 * DFTK_N_QCLASS * sizeof(unsigned long long), s));
        int st;
        if ((st = launch_select_class<0>(S, s))) return st;
        if ((st = launch_select_class<1>(S, s))) return st;
        if ((st = launch_select_class<2>(S, s))) return st;
        if ((st = launch_select_class<3>(S, s))) return st;
        if ((st = launch_select_class<4>(S, s))) return st;
        if ((st = launch_select_class<5>(S, s))) return st;
        for (int c = 0; c < DFTK_N_QCLASS; ++c) P.list[c] = S.list[c];
        P.heads = S.heads;
    }
#define DFTK_GRAD_LAUNCH(CC)                                                  \
    if (P.total[CC] > 0) {                                                    \
        if (timed) DFTK_CUDA(cudaEventRecord(g_timing.start[CC], cls[CC]));         \
        if (use_list) {                                                       \
            const LaunchShape gs = launch_shape(DFTK_FAMILY_GRAD, CC, 0);     \
            k_grad_eri<CC, true><<<shaped_grid(gs, P.total[CC]), gs.threads, smem, cls[CC]>>>(P); \
        } else {                                                              \
            k_grad_eri<CC, false><<<grid(P.total[CC]), GRAD_THREADS, smem, cls[CC]>>>(P); \
        }                                                                     \
        DFTK_LAUNCHED("k_grad_eri");                                          \
        if (timed) {                                                          \
            DFTK_CUDA(cudaEventRecord(g_timing.stop[CC], cls[CC]));                 \
            g_timing.launched[CC] = true;                                     \
        }                                                                     \
        if (use_list && mixed) {                                              \
            const LaunchShape gs = launch_shape(DFTK_FAMILY_GRAD, CC, 1);     \
            if (timed) DFTK_CUDA(cudaEventRecord(g_timing.start[DFTK_N_QCLASS + CC], cls[CC])); \
            k_grad_eri<CC, true, float><<<shaped_grid(gs, P.total[CC]), gs.threads, smem, cls[CC]>>>(P); \
            DFTK_LAUNCHED("k_grad_eri");                                      \
            if (timed) {                                                      \
                DFTK_CUDA(cudaEventRecord(g_timing.stop[DFTK_N_QCLASS + CC], cls[CC])); \
                g_timing.launched[DFTK_N_QCLASS + CC] = true;                 \
            }                                                                 \
        }                                                                     \
    }
    // class kernels on the forked streams (their gradient sums are atomics, which commute)
    cudaStream_t cls[DFTK_N_QCLASS];
    int n_aux = 0;
    int dev = 0;
    DFTK_CUDA(cudaGetDevice(&dev));
    std::unique_lock<std::mutex> fork_lock(g_pool[dev].mutex);
    {
        const int st = fork_class_streams(s, cls, n_aux, true);
        if (st) return st;
    }
    DFTK_GRAD_LAUNCH(1)
    DFTK_GRAD_LAUNCH(0)
    DFTK_GRAD_LAUNCH(4)
    DFTK_GRAD_LAUNCH(5)
    DFTK_GRAD_LAUNCH(2)
    DFTK_GRAD_LAUNCH(3)
#undef DFTK_GRAD_LAUNCH
    return join_class_streams(s, n_aux);
}

int dftk_nuclear_kernel(const double *exp_a, const double *exp_b, const double *cen_a, const double *cen_b,
                        const int *pow_a, const int *pow_b, const int *atoms, const double *atom_centers,
                        int num_atoms, int num_funcs_a, int num_funcs_b, double *V_output, double *Ex_output,
                        double *Ey_output, double *Ez_output, double *p_output, double *P_output, int *nx_output,
                        int *ny_output, int *nz_output, dftk_stream_t stream)
{
    if (num_funcs_a < 0 || num_funcs_b < 0 || num_atoms < 0) return fail(DFTK_ERR_ARG, "dftk_nuclear_kernel: negative size");
    DFTK_INIT();
    const long long n = (long long)num_funcs_a * num_funcs_b;
    if (n == 0) return DFTK_OK;
    k_nuclear_dropin<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        exp_a, exp_b, cen_a, cen_b, pow_a, pow_b, atoms, atom_centers, num_atoms, num_funcs_a, num_funcs_b,
        V_output, Ex_output, Ey_output, Ez_output, p_output, P_output, nx_output, ny_output, nz_output);
    DFTK_LAUNCHED("k_nuclear_dropin");
    return DFTK_OK;
}

int dftk_eri_kernel(int K_ab, const double *p_ab, const double *P_ab, const double *Exab, const double *Eyab,
                    const double *Ezab, const int *nxab, const int *nyab, const int *nzab, int K_cd,
                    const double *p_cd, const double *P_cd, const double *Excd, const double *Eycd,
                    const double *Ezcd, const int *nxcd, const int *nycd, const int *nzcd, double *eri_output,
                    dftk_stream_t stream)
{
    if (K_ab < 0 || K_cd < 0) return fail(DFTK_ERR_ARG, "dftk_eri_kernel: negative size");
    DFTK_INIT();
    const long long n = (long long)K_ab * K_cd;
    if (n == 0) return DFTK_OK;
    k_eri_dropin<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        K_ab, p_ab, P_ab, Exab, Eyab, Ezab, nxab, nyab, nzab, K_cd, p_cd, P_cd, Excd, Eycd, Ezcd, nxcd, nycd,
        nzcd, eri_output);
    DFTK_LAUNCHED("k_eri_dropin");
    return DFTK_OK;
}

int dftk_fma_burn(int precision, int blocks, int threads, int iters, double *sink, dftk_stream_t stream)
{
    if ((precision != 64 && precision != 32) || blocks <= 0 || threads <= 0 || threads > 1024 || iters < 0 || !sink)
        return fail(DFTK_ERR_ARG, "dftk_fma_burn: bad arguments");
    if (precision == 64) k_fma_burn<double><<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, sink);
    else k_fma_burn<float><<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, sink);
    DFTK_LAUNCHED("k_fma_burn");
    return DFTK_OK;
}

}  // extern "C"
