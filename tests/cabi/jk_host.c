/*
 * A C host of libdftk.so, the way a non-Python caller would drive it: read a
 * molecule's shells and densities (written by tests/test_gpu_cabi_host.py),
 * set up pairs and queue with dftk_prepare, build J and K with dftk_jk and
 * write them back.  Uses nothing but include/dftk.h and the CUDA runtime.
 *
 * Input (binary, native endianness): int32 n_shells, n_ao, n_prim; then
 * double xyz[3 n_shells]; int32 l, nprim, prim_off, ao [n_shells each];
 * double prim_exp[n_prim], prim_cn[n_prim], D[n_ao^2], D_a[n_ao^2].
 * Output: double J[n_ao^2], K[n_ao^2].
 *
 * usage: jk_host input.bin output.bin
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "dftk.h"

#define CK(x)                                                                     \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));              \
            return 2;                                                             \
        }                                                                         \
    } while (0)
#define DK(x)                                                                     \
    do {                                                                          \
        int s_ = (x);                                                             \
        if (s_ != DFTK_OK) {                                                      \
            fprintf(stderr, "%s: status %d: %s\n", #x, s_, dftk_last_error());    \
            return 3;                                                             \
        }                                                                         \
    } while (0)

static int read_all(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes ? 0 : 1; }

static int to_device(void **d, const void *h, size_t bytes)
{
    if (cudaMalloc(d, bytes ? bytes : 8) != cudaSuccess) return 1;
    if (bytes && cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 1;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 1;
    int hdr[3];
    if (read_all(f, hdr, sizeof hdr)) return 1;
    const int ns = hdr[0], nao = hdr[1], np = hdr[2];
    if (ns <= 0 || nao <= 0 || np <= 0 || nao > 4096) return 1;
    const size_t nn = (size_t)nao * nao;
    double *xyz = malloc(sizeof(double) * 3 * ns), *ex = malloc(sizeof(double) * np), *cn = malloc(sizeof(double) * np);
    int *l = malloc(sizeof(int) * ns), *npr = malloc(sizeof(int) * ns), *off = malloc(sizeof(int) * ns),
        *ao = malloc(sizeof(int) * ns);
    double *D = malloc(sizeof(double) * nn), *Da = malloc(sizeof(double) * nn), *J = malloc(sizeof(double) * nn),
           *K = malloc(sizeof(double) * nn);
    if (!xyz || !ex || !cn || !l || !npr || !off || !ao || !D || !Da || !J || !K) return 1;
    if (read_all(f, xyz, sizeof(double) * 3 * ns) || read_all(f, l, sizeof(int) * ns) ||
        read_all(f, npr, sizeof(int) * ns) || read_all(f, off, sizeof(int) * ns) || read_all(f, ao, sizeof(int) * ns) ||
        read_all(f, ex, sizeof(double) * np) || read_all(f, cn, sizeof(double) * np) ||
        read_all(f, D, sizeof(double) * nn) || read_all(f, Da, sizeof(double) * nn))
        return 1;
    fclose(f);

    void *d_xyz, *d_l, *d_np, *d_off, *d_ao, *d_ex, *d_cn, *d_D, *d_Da, *d_J, *d_K;
    if (to_device(&d_xyz, xyz, sizeof(double) * 3 * ns) || to_device(&d_l, l, sizeof(int) * ns) ||
        to_device(&d_np, npr, sizeof(int) * ns) || to_device(&d_off, off, sizeof(int) * ns) ||
        to_device(&d_ao, ao, sizeof(int) * ns) || to_device(&d_ex, ex, sizeof(double) * np) ||
        to_device(&d_cn, cn, sizeof(double) * np) || to_device(&d_D, D, sizeof(double) * nn) ||
        to_device(&d_Da, Da, sizeof(double) * nn) || to_device(&d_J, NULL, 0) || to_device(&d_K, NULL, 0))
        return 2;
    CK(cudaFree(d_J));
    CK(cudaFree(d_K));
    CK(cudaMalloc(&d_J, sizeof(double) * nn));
    CK(cudaMalloc(&d_K, sizeof(double) * nn));

    dftk_shells_t sh;
    memset(&sh, 0, sizeof sh);  /* one molecule: the batch fields stay zero */
    sh.n_shells = ns;
    sh.n_ao = nao;
    sh.xyz = d_xyz;
    sh.l = d_l;
    sh.nprim = d_np;
    sh.prim_off = d_off;
    sh.ao = d_ao;
    sh.prim_exp = d_ex;
    sh.prim_cn = d_cn;

    size_t store_bytes = 0;
    DK(dftk_prepare_bytes(&sh, &store_bytes));
    void *store;
    CK(cudaMalloc(&store, store_bytes));
    dftk_pairs_t pairs[DFTK_N_PCLASS];
    dftk_queue_t queue;
    DK(dftk_prepare(&sh, 1e-12, 1e-15, store, store_bytes, pairs, &queue, NULL));
    const size_t ws_bytes = dftk_jk_workspace_bytes_queue(ns, nao, &queue);
    void *ws;
    CK(cudaMalloc(&ws, ws_bytes));
    DK(dftk_jk(&sh, pairs, &queue, d_D, d_Da, NULL, d_J, d_K, NULL, 0, 1e-14, 1e-14, ws, ws_bytes, NULL, NULL));
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(J, d_J, sizeof(double) * nn, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(K, d_K, sizeof(double) * nn, cudaMemcpyDeviceToHost));

    FILE *o = fopen(argv[2], "wb");
    if (!o || fwrite(J, sizeof(double), nn, o) != nn || fwrite(K, sizeof(double), nn, o) != nn) return 1;
    fclose(o);
    printf("jk_host: %d shells, %d AOs, quartets %lld %lld %lld %lld %lld %lld\n", ns, nao, queue.total[0],
           queue.total[1], queue.total[2], queue.total[3], queue.total[4], queue.total[5]);
    return 0;
}
