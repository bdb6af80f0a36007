// gx_search_device_noalloc: the plain query path with no device allocation at all.
//
// Some callers cannot call cudaMalloc: a host that hands this library a CUDA stream from
// inside a memory-pool-managed framework (pool allocators that own every byte of the
// device), a real-time or embedded caller whose memory budget is fixed when the process
// starts, or code running where an allocation could block or fail at an unsafe moment.
// This entry point lets them search with only the buffers they already own: the
// resident index, their queries and their result arrays.  Its scratch lives in a
// file-scope device array of fixed size instead of a workspace.
//
// The scratch holds the per-(spectrum, length) candidate windows, the hyperscore table
// and the device guard word.  It is a static __device__ array, so in host code its name
// is only a host-side stand-in: the kernels receive the device address that
// cudaGetSymbolAddress returns, looked up once per device (with that device current) on
// the first call that runs on it, and again after a cudaDeviceReset has replaced the
// device's context (the new context holds a fresh, zeroed copy of the array).
//
// Limits and sharing:
//  * at most GX_NOALLOC_MAX_WINDOWS (spectra x lengths) per call;
//  * every call on a device uses the same array, which keeps the previous call's
//    contents: the guard word is cleared at the start of each call, the window table is
//    rewritten completely, the hyperscore table is written once at set-up;
//  * calls whose kernels overlap on the GPU (other streams, or other host threads on the
//    same device) race on the array and must be serialised by the caller.

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/gicops_b200.h"
#include "gx_device.cuh"
#include "gx_device_scope.cuh"
#include "gx_index.cuh"
#include "gx_internal.h"

namespace gx {
// kernels of the plain path (gx_search.cu)
__global__ void k_windows(SearchArgs a, int2 *win);
__global__ void __launch_bounds__(512) k_search_plain(SearchArgs a, int tile);
}  // namespace gx

using namespace gx;

namespace {

constexpr int kPlainBlock = 512;
constexpr int kPlainTile = 8192;
constexpr size_t kHeadBytes = 1024;  // lgfact (81 doubles) at 0, guard word at 768
constexpr size_t kScratchBytes = kHeadBytes + sizeof(int2) * (size_t)GX_NOALLOC_MAX_WINDOWS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct DeviceSetUp {
    unsigned char *addr = nullptr;   // the array's device address in that context
    unsigned long long ctx_id = 0;   // the context it was set up in (0: never)
};
DeviceSetUp g_setup[kMaxDevices];

// Unique id of the calling thread's current context (0 when none or when the driver has no
// such query).  A cudaDeviceReset replaces the device's primary context, and with it the
// module's copy of the array: a new id says that the set-up must run again.
unsigned long long current_context_id()
{
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {   // under g_mu
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
        looked_up = true;
    }
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array on `device` (the current device), set up on the
// first call in each context: the address is looked up and the hyperscore table written.
gx_status scratch_for(int device, unsigned char **out)
{
    if (device < 0 || device >= kMaxDevices) return fail(GX_ERR_INVLD_PARAM, "gx_search_device_noalloc: device id");
    std::lock_guard<std::mutex> g(g_mu);
    DeviceSetUp &d = g_setup[device];
    const unsigned long long ctx = current_context_id();
    if (!d.addr || ctx == 0 || ctx != d.ctx_id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "gx_search_device_noalloc: cudaGetSymbolAddress");
        double lg[81];
        gx_lgfact(lg);
        if ((e = cudaMemcpy(p, lg, sizeof(lg), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "gx_search_device_noalloc: hyperscore table");
        if ((e = cudaFuncSetAttribute(k_search_plain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kPlainTile * 8)) != cudaSuccess)
            return cuda_fail(e, "gx_search_device_noalloc: kernel attributes");
        d.addr = static_cast<unsigned char *>(p);
        d.ctx_id = current_context_id();   // the lookup above made the context current
    }
    *out = d.addr;
    return GX_SUCCESS;
}

}  // namespace

extern "C" gx_status gx_search_device_noalloc(gx_index *ix, const gx_queries *q, const gx_params *p, gx_result *out,
                                              gx_cell *heap, uint32_t *hist, void *stream)
{
    if (!ix || !q || !p || !out) return fail(GX_ERR_INVLD_PTR, "gx_search_device_noalloc: null argument");
    const int32_t cap = gx_heap_capacity(p->topmatches);
    if (cap < 1 || cap > GX_MAX_HEAP)
        return fail(GX_ERR_INVLD_PARAM, "gx_search_device_noalloc: topmatches gives a heap capacity outside 1..31");
    if (p->scale == 0 || p->dF > 255 || p->min_shp == 0)
        return fail(GX_ERR_INVLD_PARAM, "gx_search_device_noalloc: scale must be > 0, dF <= 255, min_shp >= 1");
    const double top = p->max_mass * (double)p->scale;
    if (!(top >= 1.0) || top + 1.0 > (double)ix->nbins + 0.5)
        return fail(GX_ERR_INVLD_PARAM, "gx_search_device_noalloc: max_mass*scale+1 exceeds the index's bins");
    if ((2.0 * p->dF + 1.0) * ix->maxz >= 57.02 * p->scale)
        return fail(GX_ERR_INVLD_PARAM, "gx_search_device_noalloc: fragment tolerance wider than a residue");
    const uint64_t nwin = (uint64_t)q->nspec * (uint64_t)ix->nlen;
    if (nwin > (uint64_t)GX_NOALLOC_MAX_WINDOWS)
        return fail(GX_ERR_INVLD_SIZE, "gx_search_device_noalloc: spectra x lengths = " + std::to_string(nwin) +
                                           " exceeds the fixed scratch of " +
                                           std::to_string(GX_NOALLOC_MAX_WINDOWS) + " windows; split the batch");
    if (q->nspec == 0) return GX_SUCCESS;
    DeviceScope ds(ix->device);
    cudaError_t e = ds.status();
    if (e != cudaSuccess) return cuda_fail(e, "gx_search_device_noalloc: cudaSetDevice");
    cudaGetLastError();   // an earlier call's error is not ours to report
    unsigned char *scratch = nullptr;
    gx_status rc = scratch_for(ix->device, &scratch);
    if (rc != GX_SUCCESS) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int32_t *err = reinterpret_cast<int32_t *>(scratch + 768);
    int2 *win = reinterpret_cast<int2 *>(scratch + kHeadBytes);
    if ((e = cudaMemsetAsync(err, 0, sizeof(int32_t), st)) != cudaSuccess)
        return cuda_fail(e, "gx_search_device_noalloc: clear guard word");

    SearchArgs a{};
    a.bA = ix->bA; a.iA = ix->iA; a.mass = ix->mass; a.lens = ix->lens; a.nlen = ix->nlen; a.nbins = ix->nbins;
    a.maxz = ix->maxz;
    a.qidx = q->idx; a.moz = q->moz; a.intn = q->intn; a.prec = q->prec; a.dMq = q->dM; a.nspec = q->nspec;
    a.dM = p->dM;
    a.upper = (p->max_mass * (double)p->scale) - 1.0 - (double)p->dF;
    a.dF = p->dF; a.min_shp = p->min_shp; a.min_cpsm = p->min_cpsm; a.heap_cap = cap;
    a.expect_max = p->expect_max; a.flags = p->flags;
    a.lgfact = reinterpret_cast<const double *>(scratch);
    a.win = win; a.out = out; a.heap_out = heap; a.hist_out = hist; a.err = err;

    k_windows<<<(unsigned)((nwin + 255) / 256), 256, 0, st>>>(a, win);
    count_launch();
    k_search_plain<<<q->nspec, kPlainBlock, (size_t)kPlainTile * 8, st>>>(a, kPlainTile);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "gx_search_device_noalloc: launch");
    return GX_SUCCESS;
}
