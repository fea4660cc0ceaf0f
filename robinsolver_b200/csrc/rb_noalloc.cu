// rb_noalloc.cu -- leaf Robin-to-Robin maps without any device allocation.
//
// Some callers cannot call cudaMalloc: a host framework that owns all device memory through its
// own pool (or has reserved the device's memory up front) and forbids allocations from plugins,
// and loops on a latency-critical path, where cudaMalloc's implicit device synchronisation is
// not acceptable.  They bring their own input and output buffers; rb_leaf_rtr_noalloc then runs
// the leaf factor kernel (rb_leaf.cu) with its working memory -- the inverted diagonal blocks,
// the intermediate of the transposed block sweep and the zero-pivot flag -- in a file-scope
// __device__ array instead of handle-owned allocations.
//
// The array is RB_NOALLOC_SCRATCH_BYTES (32 MiB) and is part of the module image: every GPU on
// which the library is loaded holds it until the process exits.  All calls share it and it keeps
// the last call's contents, so calls whose device work overlaps (different streams, or different
// host threads on one device) race on it.  Only the zero-pivot flag must start at zero; it is
// cleared on the caller's stream before each launch.  In host code the array's name is not a
// device address: its device address is looked up with cudaGetSymbolAddress once per device, on
// the first call made while that device is current.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "robin_b200.h"
#include "rb_kernels.h"

namespace rb {

constexpr size_t RB_NOALLOC_SCRATCH_BYTES = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[RB_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[128] = {};

// failures are reported like rb_tree_create's: rb_last_error(NULL) on the calling thread
static int noalloc_fail(int code, const char* msg) {
    set_thread_error(msg);
    return code;
}

}  // namespace rb

using namespace rb;

extern "C" int rb_leaf_rtr_noalloc(int a, int b, double kb, const double* d_h, const double* d_k, int nleaves,
                                   double* d_rtr, void* stream) {
    if (a < 3 || b < 3 || nleaves < 1 || !d_h || !d_k || !d_rtr)
        return noalloc_fail(RB_ERR_INVALID, "rb_leaf_rtr_noalloc: grid must be at least 3x3, nleaves >= 1, pointers non-null");
    // sizes in 64-bit arithmetic: a grid this large cannot fit the scratch array anyway
    if ((int64_t)a * a > 1024 || 2 * ((int64_t)a + b) > 512)
        return noalloc_fail(RB_ERR_INVALID, "rb_leaf_rtr_noalloc: leaf grid too large for the leaf kernel");
    LeafGeom g{a, b, 2 * (a + b), 2 * (a + b) + a * b, kb};
    const size_t per_leaf = ((size_t)b * a * a + (size_t)g.nb * g.n) * sizeof(z);
    const size_t need = 256 + (size_t)nleaves * per_leaf;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
        return noalloc_fail(RB_ERR_CUDA, "rb_leaf_rtr_noalloc: no current CUDA device");
    if (a != 16) {
        // leaves other than 16 wide run the one-CTA-per-leaf kernel, whose shared memory grows
        // with a and nb: refuse a grid it cannot hold on this device
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            return noalloc_fail(RB_ERR_CUDA, "rb_leaf_rtr_noalloc: cannot query the device's shared memory");
        if (leaf_block_factor_smem(g) > (size_t)optin) {
            char msg[200];
            std::snprintf(msg, sizeof(msg),
                          "rb_leaf_rtr_noalloc: a %dx%d leaf needs %zu bytes of shared memory, the device allows %d",
                          a, b, leaf_block_factor_smem(g), optin);
            return noalloc_fail(RB_ERR_INVALID, msg);
        }
    }
    if (need > RB_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "rb_leaf_rtr_noalloc: %d leaves of %dx%d need %zu bytes of scratch, the limit is %zu "
                      "(at most %zu leaves of this size per call)",
                      nleaves, a, b, need, RB_NOALLOC_SCRATCH_BYTES, (RB_NOALLOC_SCRATCH_BYTES - 256) / per_leaf);
        return noalloc_fail(RB_ERR_INVALID, msg);
    }
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mutex);
        if (!g_noalloc_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return noalloc_fail(RB_ERR_CUDA, "rb_leaf_rtr_noalloc: cudaGetSymbolAddress of the scratch array failed");
            }
            g_noalloc_addr[dev] = p;
        }
        base = g_noalloc_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* status = static_cast<int*>(base);
    z* sinv = reinterpret_cast<z*>(static_cast<unsigned char*>(base) + 256);
    z* Y = sinv + (size_t)nleaves * b * a * a;
    // per-leaf grid spacings come from the caller (2 doubles per leaf: hx, hy)
    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess)
        return noalloc_fail(RB_ERR_CUDA, "rb_leaf_rtr_noalloc: clearing the status flag failed");
    cudaError_t e = leaf_block_factor(g, nleaves, d_h, reinterpret_cast<const z*>(d_k), sinv, Y, status, s);
    if (e != cudaSuccess) return noalloc_fail(RB_ERR_CUDA, cudaGetErrorString(e));
    // the leaf RtR is the first nb columns of each leaf's Y (nb x n, ld nb)
    e = cudaMemcpy2DAsync(d_rtr, (size_t)g.nb * g.nb * sizeof(z), Y, (size_t)g.nb * g.n * sizeof(z),
                          (size_t)g.nb * g.nb * sizeof(z), nleaves, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return noalloc_fail(RB_ERR_CUDA, cudaGetErrorString(e));
    int st = 0;
    e = cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return noalloc_fail(RB_ERR_CUDA, cudaGetErrorString(e));
    if (st) return noalloc_fail(RB_ERR_NUMERIC, "rb_leaf_rtr_noalloc: zero pivot in a leaf block inverse");
    return RB_OK;
}
