// dftk_jk_noalloc: the integral-direct J/K build for callers that cannot
// allocate device memory.
//
// dftk_jk wants a caller-allocated workspace (dftk_jk_workspace_bytes).  Some
// callers cannot make that allocation: a host program that runs the library
// inside a fixed device-memory budget it has already carved up, or a plugin
// host whose own memory pool must account for every byte and where a
// cudaMalloc from inside the plugin would also synchronize the device.  This
// entry point takes the same inputs and outputs as dftk_jk and uses a
// file-scope device array as its workspace instead, so it allocates nothing.
//
// Limits and sharing:
//   * at most DFTK_NOALLOC_MAX_AO basis functions and DFTK_NOALLOC_MAX_SHELLS
//     shells; larger molecules get DFTK_ERR_SIZE and an error message;
//   * the array (DFTK_NOALLOC_SCRATCH_BYTES, about 7 MB) lives in every GPU
//     that loads the library until the process exits;
//   * every call shares it: two calls whose work overlaps on the GPU (other
//     streams, other host threads on the same device) race, so issue them on
//     one stream or order them yourself.  Each call clears the parts that must
//     start at zero, so the contents a previous call left behind do no harm;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is cached for the life of the
//     process, which assumes the device's primary context is not reset
//     (cudaDeviceReset) in between.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dftk.h"

#define DFTK_NOALLOC_MAX_AO 512
#define DFTK_NOALLOC_MAX_SHELLS 512
// Y, Z_a, Z_b (N^2 doubles each) and the shell-block density maxima (ns^2 floats)
#define DFTK_NOALLOC_SCRATCH_BYTES                                                          \
    (3ull * DFTK_NOALLOC_MAX_AO * DFTK_NOALLOC_MAX_AO * sizeof(double) +                    \
     1ull * DFTK_NOALLOC_MAX_SHELLS * DFTK_NOALLOC_MAX_SHELLS * sizeof(float))

// In host code this name is only a host-side stand-in for the device array;
// the kernels get the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_jk_scratch[DFTK_NOALLOC_SCRATCH_BYTES];

extern "C" __attribute__((visibility("hidden"))) void dftk_internal_set_error(const char *msg);

namespace {
std::mutex g_noalloc_mutex;
void *g_scratch_ptr[128] = {nullptr};
}  // namespace

extern "C" int dftk_jk_noalloc(const dftk_shells_t *shells, const dftk_pairs_t pairs[DFTK_N_PCLASS],
                               const dftk_queue_t *queue, const double *D, const double *D_a,
                               const double *D_b, double *J, double *K_a, double *K_b, int flags,
                               double tau, double tau_fp32, long long *counts, dftk_stream_t stream)
{
    if (!shells) {
        dftk_internal_set_error("dftk_jk_noalloc: null shells");
        return DFTK_ERR_ARG;
    }
    const bool batch_too_big =
        shells->mol && (shells->mat_elems > (long long)DFTK_NOALLOC_MAX_AO * DFTK_NOALLOC_MAX_AO ||
                        shells->dsh_elems > (long long)DFTK_NOALLOC_MAX_SHELLS * DFTK_NOALLOC_MAX_SHELLS);
    if (shells->n_ao < 0 || shells->n_shells < 0 || batch_too_big ||
        (!shells->mol && (shells->n_ao > DFTK_NOALLOC_MAX_AO || shells->n_shells > DFTK_NOALLOC_MAX_SHELLS))) {
        // a batch is limited by its packed matrix and density-maxima sizes,
        // a single molecule by its basis functions and shells
        const std::string lim = std::to_string(DFTK_NOALLOC_MAX_AO);
        const std::string lims = std::to_string(DFTK_NOALLOC_MAX_SHELLS);
        const std::string msg =
            shells->mol
                ? "dftk_jk_noalloc: the batch's packed matrices (" + std::to_string(shells->mat_elems) +
                      " elements) or density maxima (" + std::to_string(shells->dsh_elems) +
                      " elements) exceed the fixed scratch limit of " + lim + "^2 / " + lims +
                      "^2; use dftk_jk with a workspace"
                : "dftk_jk_noalloc: " + std::to_string(shells->n_ao) + " basis functions / " +
                      std::to_string(shells->n_shells) + " shells exceed the fixed scratch limit of " + lim +
                      " / " + lims + "; use dftk_jk with a workspace";
        dftk_internal_set_error(msg.c_str());
        return DFTK_ERR_SIZE;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        dftk_internal_set_error((std::string("dftk_jk_noalloc: cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
        return DFTK_ERR_CUDA;
    }
    if (dev < 0 || dev >= 128) {
        dftk_internal_set_error("dftk_jk_noalloc: device index out of range");
        return DFTK_ERR_ARG;
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_scratch_ptr[dev]) {
            e = cudaGetSymbolAddress(&g_scratch_ptr[dev], g_jk_scratch);
            if (e != cudaSuccess) {
                g_scratch_ptr[dev] = nullptr;
                dftk_internal_set_error(
                    (std::string("dftk_jk_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
                return DFTK_ERR_CUDA;
            }
        }
        scratch = g_scratch_ptr[dev];
    }
    return dftk_jk(shells, pairs, queue, D, D_a, D_b, J, K_a, K_b, flags, tau, tau_fp32, scratch,
                   (size_t)DFTK_NOALLOC_SCRATCH_BYTES, counts, stream);
}
