// ising_sweep_static: the measured sweep on caller-owned device arrays, allocating nothing.
//
// Some callers cannot call cudaMalloc: an application whose device memory is all owned by a
// memory pool it does not control (a framework's caching allocator that has reserved the HBM,
// or a host process with a fixed device-memory budget), or a tight serving/timing loop where
// the implicit device synchronisation of cudaMalloc/cudaFree is not acceptable.  For them this
// entry point runs sweeps directly on the two colour arrays they pass in, and keeps the (M, E)
// accumulators of the measured sweeps in a fixed device array compiled into the library, so no
// call allocates device or pinned host memory.
//
// The scratch array is a file-scope __device__ symbol: every GPU that loads the library holds
// its 64 KiB until the process exits.  Host code cannot use the symbol's name as an address
// (on the host it names a host-side stand-in), so each device's real address is looked up with
// cudaGetSymbolAddress, with that device current, on the first call there, and cached with the
// CUDA context it belongs to: after cudaDeviceReset the device has a new context, and the next
// call looks the address up again.  The first call on a device does this set-up, so it should
// come before any stream capture.
//
// Caller arrays are checked before any launch: they must be device (or managed) memory of the
// current device, 16-byte aligned, and lie inside one allocation of at least the bytes the
// shape needs (cuMemGetAddressRange through the runtime's driver entry points).
#include <cstring>
#include <mutex>

#include "capi_internal.h"

namespace ising {
namespace {

// At most this many (M, E) measurements per call: 2 x 8 bytes each, 64 KiB in total.
constexpr int64_t kStaticSeriesMaxPairs = 4096;

__device__ __align__(256) unsigned long long g_static_series[2 * kStaticSeriesMaxPairs];

constexpr int kMaxDevices = 64;
std::mutex g_static_setup_mutex;
unsigned long long* g_static_series_addr[kMaxDevices] = {};
void* g_static_series_ctx[kMaxDevices] = {};

// Driver entry points, looked up through the runtime (no link against libcuda).
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*MemGetAddressRangeFn)(unsigned long long* base, size_t* size,
                                    unsigned long long ptr);

template <typename Fn>
Fn driver_entry(const char* name)
{
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return reinterpret_cast<Fn>(fn);
}

// Device address of g_static_series on `device` (which must be current), looked up on the
// first call for that device and again whenever the device's current context has changed.
int static_series_address(int device, unsigned long long** out)
{
    std::lock_guard<std::mutex> lock(g_static_setup_mutex);
    static CtxGetCurrentFn ctx_get = driver_entry<CtxGetCurrentFn>("cuCtxGetCurrent");
    void* ctx = nullptr;
    if (ctx_get && ctx_get(&ctx) != 0) ctx = nullptr;
    if (!g_static_series_addr[device] || ctx != g_static_series_ctx[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_series);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static series scratch)");
        g_static_series_addr[device] = static_cast<unsigned long long*>(p);
        g_static_series_ctx[device] = ctx;
    }
    *out = g_static_series_addr[device];
    return ISING_OK;
}

// A caller array of at least `need` bytes on `device`: checked on the host before any launch,
// so that a pointer to host memory, to another GPU or to a too-short buffer is an
// ISING_ERR_INVALID and not a kernel reading out of bounds.
int check_device_array(const void* p, const char* name, int device, size_t need)
{
    if (!p) return fail(ISING_ERR_INVALID, "%s is null", name);
    if (reinterpret_cast<uintptr_t>(p) % 16)
        return fail(ISING_ERR_INVALID, "%s must be 16-byte aligned", name);
    cudaPointerAttributes a;
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ISING_ERR_INVALID, "%s is not a CUDA pointer", name);
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        return fail(ISING_ERR_INVALID, "%s must be device memory", name);
    if (a.type == cudaMemoryTypeDevice && a.device != device)
        return fail(ISING_ERR_INVALID, "%s lives on device %d, but device %d is current", name,
                    a.device, device);
    static MemGetAddressRangeFn range = driver_entry<MemGetAddressRangeFn>("cuMemGetAddressRange");
    if (!range) return fail(ISING_ERR_CUDA, "cuMemGetAddressRange is not available");
    unsigned long long base = 0;
    size_t size = 0;
    const unsigned long long ptr = reinterpret_cast<uintptr_t>(p);
    if (range(&base, &size, ptr) != 0)
        return fail(ISING_ERR_INVALID, "%s is not inside a device allocation", name);
    if (ptr < base || ptr - base > size || size - (ptr - base) < need)
        return fail(ISING_ERR_INVALID,
                    "%s holds %llu bytes to the end of its allocation; the shape needs %llu",
                    name, (unsigned long long)(size - (ptr - base)), (unsigned long long)need);
    return ISING_OK;
}

}  // namespace
}  // namespace ising

using namespace ising;

extern "C" int ising_sweep_static(int ndim, const int64_t* shape, int variant, int algorithm,
                                  uint64_t seed, const uint32_t* table, int table_n, void* c0,
                                  void* c1, uint64_t t0, int64_t n_sweeps, int64_t measure_every,
                                  int64_t* series_out, void* stream)
{
    if (!shape || !table) return fail(ISING_ERR_INVALID, "null shape or table");
    if (ndim != 2 && ndim != 3)
        return fail(ISING_ERR_INVALID, "only 2D and 3D lattices are supported, got ndim=%d", ndim);
    for (int i = 0; i < ndim; ++i)
        if (shape[i] < 2 || shape[i] % 2)
            return fail(ISING_ERR_INVALID, "all extents must be even and >= 2");
    if (variant != ISING_VARIANT_INT8 && variant != ISING_VARIANT_MSC)
        return fail(ISING_ERR_INVALID, "unknown variant %d", variant);
    if (algorithm != ISING_METROPOLIS && algorithm != ISING_HEATBATH)
        return fail(ISING_ERR_INVALID, "unknown algorithm %d", algorithm);
    if (variant == ISING_VARIANT_MSC && (ndim != 2 || algorithm != ISING_METROPOLIS))
        return fail(ISING_ERR_INVALID, "msc supports 2D Metropolis only");
    const int64_t lx = shape[ndim - 1];
    const int multiple = variant == ISING_VARIANT_MSC ? 128 : 8;
    if (lx % multiple)
        return fail(ISING_ERR_INVALID, "last extent must be a multiple of %d", multiple);
    if (table_n != 2 * ndim + 1)
        return fail(ISING_ERR_INVALID, "table must have %d entries, got %d", 2 * ndim + 1, table_n);
    const int64_t ly = shape[ndim - 2], lz = ndim == 3 ? shape[0] : 1, rows = ly * lz;
    if (rows > (int64_t)0x7FFFFFFF || lx / 2 > (int64_t)0x7FFFFFFF)
        return fail(ISING_ERR_INVALID, "lattice too large for 32-bit row indices");
    if (n_sweeps < 0 || measure_every < 0)
        return fail(ISING_ERR_INVALID, "negative sweep count or measurement interval");
    const int64_t n_meas = measure_every > 0 ? n_sweeps / measure_every : 0;
    if (n_meas > kStaticSeriesMaxPairs)
        return fail(ISING_ERR_INVALID,
                    "at most %lld measurements per call (n_sweeps / measure_every = %lld); "
                    "split the run into several calls",
                    (long long)kStaticSeriesMaxPairs, (long long)n_meas);
    if (n_meas > 0 && !series_out)
        return fail(ISING_ERR_INVALID, "measure_every > 0 needs series_out");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices)
        return fail(ISING_ERR_INVALID, "device ordinal %d not supported", device);
    // bytes of one colour array: rows x Lx/2 int8, or rows x Lx/128 uint64 words
    const size_t colour_bytes = variant == ISING_VARIANT_MSC
                                    ? (size_t)rows * (size_t)(lx / 128) * sizeof(u64)
                                    : (size_t)rows * (size_t)(lx / 2);
    int rc = check_device_array(c0, "c0", device, colour_bytes);
    if (rc == ISING_OK) rc = check_device_array(c1, "c1", device, colour_bytes);
    if (rc != ISING_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int max_blocks = device_sm_count(device) * 8;

    unsigned long long* scratch = nullptr;
    if (n_meas > 0) {
        rc = static_series_address(device, &scratch);
        if (rc != ISING_OK) return rc;
        // the array keeps the previous call's sums: clear the part this call accumulates into
        e = cudaMemsetAsync(scratch, 0, (size_t)n_meas * 2 * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(static series scratch)");
    }

    u32 tab[7];
    for (int i = 0; i < 7; ++i) tab[i] = i < table_n ? table[i] : 0xFFFFFFFFu;
    const int rule = select_rule(variant, algorithm, ndim, tab);
    const u32 k0 = (u32)seed, k1 = (u32)(seed >> 32);
    int64_t k = 0;
    for (int64_t s = 0; s < n_sweeps; ++s) {
        const u32 t = (u32)(t0 + (uint64_t)s);
        const bool meas = measure_every > 0 && (s + 1) % measure_every == 0;
        for (int color = 0; color < 2; ++color) {
            unsigned long long* m = (meas && color == 1) ? scratch + 2 * k : nullptr;
            void* own = color == 0 ? c0 : c1;
            void* other = color == 0 ? c1 : c0;
            if (variant == ISING_VARIANT_MSC) {
                MscHalf p;
                p.own = static_cast<u64*>(own);
                p.other = static_cast<const u64*>(other);
                p.rows = (int)rows;
                p.nw = (int)(lx / 128);
                p.t = t;
                p.color = (u32)color;
                p.k0 = k0;
                p.k1 = k1;
                p.thr4 = tab[3];
                p.thr8 = tab[4];
                p.nw_magic = magic_for(p.nw);
                p.meas = m;
                p.stats = nullptr;
                p.ctl = nullptr;
                e = launch_msc_half(true, p, max_blocks, max_blocks / 8, 1, st);
            } else {
                Int8Half p;
                memset(&p, 0, sizeof p);
                p.own = static_cast<int8_t*>(own);
                p.other = static_cast<const int8_t*>(other);
                p.rows = rows;
                p.lh = (int)(lx / 2);
                p.ly = (int)ly;
                p.lz = (int)lz;
                p.vw = int8_chunk_width(p.lh);  // caller arrays are contiguous: V divides lh
                p.pitch = p.lh;
                p.cpr = p.lh / p.vw;
                p.t = t;
                p.color = (u32)color;
                p.k0 = k0;
                p.k1 = k1;
                for (int i = 0; i < 7; ++i) p.table[i] = tab[i];
                p.meas = m;
                p.ctl = nullptr;
                e = launch_int8_half(ndim, rule, p, max_blocks, max_blocks / 8, st);
            }
            if (e != cudaSuccess) return cuda_fail(e, "static sweep launch");
        }
        if (meas) ++k;
    }
    if (n_meas > 0) {
        e = cudaMemcpyAsync(series_out, scratch, (size_t)n_meas * 2 * sizeof(long long),
                            cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "static sweep series copy");
    }
    return ISING_OK;
}
