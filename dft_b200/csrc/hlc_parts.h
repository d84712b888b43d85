// Host interface between dftk.cu and the translation units that hold the
// generated d-class kernels (hlc_part_*.cu, compiled side by side by
// build.py).  Each part is its own device module: it keeps its own copy of
// the Boys tables, which dftk_init fills through the part's init function.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

struct HlcParams;

// host copies of the Boys tables (boys.cuh layouts)
struct BoysTables {
    const double *t64;
    size_t n64;
    const float *t32;
    size_t n32;
    const double *e64;
    size_t ne64;
    const float *e32;
    size_t ne32;
    const double *t64h;
    size_t n64h;
};

// records a CUDA failure as the library's last error; returns DFTK_ERR_CUDA
int dftk_internal_fail_cuda(cudaError_t e, const char *where);

// Launch the chunk kernels of the part's classes, dealt round-robin over the
// ns streams in st (`next` carries the round-robin position between parts).
int hlc_part_a_launch(const HlcParams &P, const cudaStream_t *st, int ns, int &next);
int hlc_part_b_launch(const HlcParams &P, const cudaStream_t *st, int ns, int &next);
int hlc_part_c_launch(const HlcParams &P, const cudaStream_t *st, int ns, int &next);
int hlc_part_d_launch(const HlcParams &P, const cudaStream_t *st, int ns, int &next);

// copy the Boys tables into the part's device module (current device)
int hlc_part_a_init(const BoysTables &t);
int hlc_part_b_init(const BoysTables &t);
int hlc_part_c_init(const BoysTables &t);
int hlc_part_d_init(const BoysTables &t);
