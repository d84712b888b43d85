// Body of one hlc_part_*.cu: the chunk kernels of the generated d classes
// HLC_FIRST .. HLC_LAST, their launcher HLC_PART_LAUNCH and the table
// initialiser HLC_PART_INIT (the including file defines the four macros).
#pragma once

// leaves out the shared headers' non-template kernels, which only dftk.cu launches
#define DFTK_HLC_PART 1

#include "dftk.h"
#include "hlc.cuh"
#include "hlc_parts.h"

namespace {

int part_sm_count()
{
    static const int n = [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            v <= 0)
            v = 148;
        return v;
    }();
    return n;
}

// The chunk kernels of class C: 128-thread blocks, a grid of at most 16
// resident blocks per SM striding over the class's 32-candidate work items,
// one launch per component chunk dealt round-robin over the streams.
template <int C, int S = 0> int launch_hlc(const HlcParams &P, const cudaStream_t *st, int ns, int &next)
{
    if (P.total[C] == 0) return DFTK_OK;
    const long long items = (P.total[C] + 31) / 32;
    long long blocks = (items + 3) / 4;
    const long long cap = (long long)part_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    k_hlc<C, S><<<(unsigned)blocks, 128, 0, st[next++ % ns]>>>(P);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dftk_internal_fail_cuda(e, "k_hlc");
    if constexpr (S + 1 < HlClass<double, C, 0>::NSPLIT) return launch_hlc<C, S + 1>(P, st, ns, next);
    return DFTK_OK;
}

template <int C> int launch_from(const HlcParams &P, const cudaStream_t *st, int ns, int &next)
{
    if constexpr (C > HLC_LAST) {
        return DFTK_OK;
    } else {
        const int r = launch_hlc<C>(P, st, ns, next);
        if (r != DFTK_OK) return r;
        return launch_from<C + 1>(P, st, ns, next);
    }
}

}  // namespace

int HLC_PART_LAUNCH(const HlcParams &P, const cudaStream_t *st, int ns, int &next)
{
    return launch_from<HLC_FIRST>(P, st, ns, next);
}

int HLC_PART_INIT(const BoysTables &t)
{
    if (t.n64 * sizeof(double) != sizeof(g_boys64) || t.n32 * sizeof(float) != sizeof(g_boys32) ||
        t.ne64 * sizeof(double) != sizeof(g_bexp64) || t.ne32 * sizeof(float) != sizeof(g_bexp32) ||
        t.n64h * sizeof(double) != sizeof(g_boys64h))
        return dftk_internal_fail_cuda(cudaErrorInvalidValue, "hlc part: Boys table sizes");
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(g_boys64, t.t64, sizeof(g_boys64))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(g_boys32, t.t32, sizeof(g_boys32))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(g_bexp64, t.e64, sizeof(g_bexp64))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(g_bexp32, t.e32, sizeof(g_bexp32))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(g_boys64h, t.t64h, sizeof(g_boys64h))) != cudaSuccess)
        return dftk_internal_fail_cuda(e, "hlc part: Boys tables");
    return DFTK_OK;
}
