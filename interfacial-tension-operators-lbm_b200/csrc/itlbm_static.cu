// itlbm_static.cu -- the fixed device scratch of itlbm_case_diag_drop_static.
//
// One file-scope device array per device holds everything a drop diagnostic needs besides the case
// itself: the per-node fields (6 doubles a node), the per-block partials, the shell histogram, the
// running state and the device copy of the result.  Its size covers cases of up to
// ITLBM_STATIC_DIAG_MAX_NODES nodes with sides of up to ITLBM_STATIC_DIAG_MAX_SIDE (14 MiB).  Nothing
// in it has to start at zero: each diagnostic clears the shell histogram and the output on its
// stream before use, and writes the partials and the state before it reads them.
#include "itlbm_internal.h"

#include <mutex>

namespace itlbm {

namespace {

constexpr size_t STATIC_DIAG_BYTES = (size_t)14 << 20;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_static_diag[STATIC_DIAG_BYTES];

std::mutex g_mu;
void *g_addr[MAX_DEVICES] = {};

}  // namespace

cudaError_t static_diag_scratch(int device, void **base, size_t *bytes) {
    if (device < 0 || device >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[device]) {
        // the device must be current: the address is that of this device's copy of the array
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_diag);
        if (e != cudaSuccess) return e;
        g_addr[device] = p;
    }
    *base = g_addr[device];
    *bytes = STATIC_DIAG_BYTES;
    return cudaSuccess;
}

}  // namespace itlbm
