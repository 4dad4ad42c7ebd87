// C ABI (include/ising_b200.h): handle management, layout transfers, the sweep loop and the
// device probes.  All device work of a handle runs on its stream.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "capi_internal.h"

namespace ising {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(ISING_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

// Device memory of simulation handles comes from one stream-ordered pool per device that keeps
// up to kPoolKeep bytes of freed memory for reuse: creating and destroying many simulations
// (a scan, a validation run, jobs one at a time) then maps no memory and synchronises nothing.
constexpr unsigned long long kPoolKeep = 8ull << 30;
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64] = {};

cudaError_t pool_alloc(int device, void** p, size_t bytes, cudaStream_t st)
{
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
        if (!g_pool[device]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = device;
            const cudaError_t e = cudaMemPoolCreate(&g_pool[device], &props);
            if (e != cudaSuccess) return e;
            unsigned long long keep = kPoolKeep;
            cudaMemPoolSetAttribute(g_pool[device], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = g_pool[device];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

// Pinned host buffers of the measured series, by size class (powers of two from 4 KiB), kept
// for reuse (at most kPinnedKept per class).
constexpr size_t kPinnedKept = 8;
static std::mutex g_pinned_mu;
static std::map<size_t, std::vector<void*>> g_pinned;

static size_t pinned_class(size_t bytes)
{
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    return c;
}

cudaError_t host_pinned_get(void** p, size_t bytes)
{
    const size_t c = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        auto& v = g_pinned[c];
        if (!v.empty()) {
            *p = v.back();
            v.pop_back();
            return cudaSuccess;
        }
    }
    return cudaMallocHost(p, c);
}

void host_pinned_put(void* p, size_t bytes)
{
    if (!p) return;
    const size_t c = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        auto& v = g_pinned[c];
        if (v.size() < kPinnedKept) {
            v.push_back(p);
            return;
        }
    }
    cudaFreeHost(p);
}

int device_sm_count(int device)
{
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return 148;
    return n > 0 ? n : 148;
}

int select_rule(int variant, int algorithm, int ndim, const u32* table)
{
    if (variant == ISING_VARIANT_MSC) return kMetroFast;
    const int d = ndim;
    if (algorithm == ISING_METROPOLIS) {
        // the fast rule needs T(a) = table[2d - a] non-decreasing in a < d
        for (int i = d + 1; i < 2 * d; ++i)
            if (table[i] < table[i + 1]) return kMetroGeneric;
        return kMetroFast;
    }
    for (int i = 0; i < 2 * d; ++i)
        if (table[i] > table[i + 1]) return kHeatGeneric;
    return kHeatFast;
}

}  // namespace ising

namespace ising {

// Longest chunk of sweeps captured in one graph (the chunk length of unmeasured runs is the
// handle's graph_chunk knob, 32 by default); shortest remainder of a call replayed as a graph;
// graphs a handle keeps before remainders are launched directly.
constexpr int64_t kGraphChunkMax = 256;
constexpr int64_t kGraphRemainderMin = 4;
constexpr size_t kGraphsKept = 16;

// Reads the error word of the last persistent run (waits for the handle's stream).
static int check_pending(ising_sim* h)
{
    if (!h->pending_err) return ISING_OK;
    h->pending_err = false;
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, h->d_flags + h->sm_count, sizeof(int),
                                    cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "persistent sweep");
    if (err)
        return fail(ISING_ERR_TIMEOUT,
                    "a bounded wait of the persistent sweep expired; the lattice is not valid");
    return ISING_OK;
}

__global__ void ctl_set_kernel(unsigned long long* ctl, unsigned long long t,
                               unsigned long long k)
{
    ctl[0] = t;
    ctl[1] = k;
}

__global__ void ctl_advance_kernel(unsigned long long* ctl, unsigned long long dt,
                                   unsigned long long dk)
{
    ctl[0] += dt;
    ctl[1] += dk;
}

void clear_graphs(ising_sim* h)
{
    for (auto& g : h->graphs) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
}

// Two unmeasured sweeps per launch on shared-memory tiles: when asked for, and by default for
// eligible lattices of up to 512K sites per colour (1024^2), where a half-sweep is too short to
// hide its launch (larger ones measured faster with single half-sweeps).
constexpr long long kTemporalAutoSites = 512 * 1024;

static bool use_temporal(const ising_sim* h)
{
    if (!temporal_ok(h)) return false;
    if (h->schedule == ISING_SCHEDULE_TEMPORAL) return true;
    return h->schedule == ISING_SCHEDULE_AUTO && h->rows * (long long)h->lh <= kTemporalAutoSites;
}

// The captured chunk of G sweeps of this handle: 2G half-sweeps with counters relative to the
// control block d_acc[6] (sweep) / d_acc[7] (series slot), then one node advancing it.
static int chunk_graph(ising_sim* h, int64_t G, bool measured, cudaGraphExec_t* out)
{
    for (auto& g : h->graphs)
        if (g.sweeps == G && g.measured == measured) {
            *out = g.exec;
            return ISING_OK;
        }
    const unsigned long long* ctl = h->d_acc + 6;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
    int rc = ISING_OK;
    const bool tb = use_temporal(h);
    const int K = temporal_sweeps();
    int64_t s = 0;
    if (tb) {  // K unmeasured sweeps per launch, up to the measured last sweep
        const int64_t runs = (G - (measured ? 1 : 0)) / K;
        const cudaError_t le = launch_temporal_run(h, 0u, runs, ctl);
        if (le != cudaSuccess) rc = cuda_fail(le, "temporal half-sweeps");
        s = runs * K;
    }
    for (; s < G && rc == ISING_OK;) {
        unsigned long long* m =
            (measured && s == G - 1) ? (unsigned long long*)h->d_series : nullptr;
        rc = half_sweep(h, 0, (u32)s, nullptr, nullptr, ctl);
        if (rc == ISING_OK) rc = half_sweep(h, 1, (u32)s, m, nullptr, ctl);
        ++s;
    }
    if (rc == ISING_OK) {
        ctl_advance_kernel<<<1, 1, 0, h->stream>>>(h->d_acc + 6, (unsigned long long)G,
                                                   measured ? 1ull : 0ull);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "graph capture");
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(h->stream, &graph);
    if (rc != ISING_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    h->graphs.push_back({G, measured, exec});
    *out = exec;
    return ISING_OK;
}

}  // namespace ising

using namespace ising;

#define TRY_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

#define CHECK_HANDLE(h)                                                    \
    do {                                                                   \
        if (!(h)) return fail(ISING_ERR_INVALID, "null simulation handle"); \
    } while (0)

extern "C" {

const char* ising_last_error(void) { return g_last_error.c_str(); }

int ising_version(void) { return 100; }

int ising_device_name(int device, char* buf, int buflen)
{
    if (!buf || buflen < 1) return fail(ISING_ERR_INVALID, "null or empty output buffer");
    cudaDeviceProp prop;
    const cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "cudaGetDeviceProperties");
    }
    snprintf(buf, (size_t)buflen, "%s sm_%d%d %d SMs", prop.name, prop.major, prop.minor,
             prop.multiProcessorCount);
    return ISING_OK;
}

int ising_device_count(int* n)
{
    if (!n) return fail(ISING_ERR_INVALID, "null output pointer");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *n = 0;
        cudaGetLastError();
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *n = c;
    return ISING_OK;
}

int ising_create(int ndim, const int64_t* shape, int variant, int algorithm, uint64_t seed,
                 int device, ising_sim** out)
{
    if (!out || !shape) return fail(ISING_ERR_INVALID, "null pointer argument");
    *out = nullptr;
    if (ndim != 2 && ndim != 3)
        return fail(ISING_ERR_INVALID, "only 2D and 3D lattices are supported, got ndim=%d", ndim);
    for (int i = 0; i < ndim; ++i)
        if (shape[i] < 2 || shape[i] % 2)
            return fail(ISING_ERR_INVALID, "all extents must be even and >= 2");
    if (variant != ISING_VARIANT_INT8 && variant != ISING_VARIANT_MSC)
        return fail(ISING_ERR_INVALID, "unknown variant %d", variant);
    if (algorithm != ISING_METROPOLIS && algorithm != ISING_HEATBATH)
        return fail(ISING_ERR_INVALID, "unknown algorithm %d", algorithm);
    const int64_t lx = shape[ndim - 1];
    const int multiple = variant == ISING_VARIANT_MSC ? 128 : 8;
    if (lx % multiple)
        return fail(ISING_ERR_INVALID, "last extent must be a multiple of %d, got %lld", multiple,
                    (long long)lx);
    if (variant == ISING_VARIANT_MSC && (ndim != 2 || algorithm != ISING_METROPOLIS))
        return fail(ISING_ERR_INVALID, "msc supports 2D Metropolis only");
    const int64_t ly = shape[ndim - 2];
    const int64_t lz = ndim == 3 ? shape[0] : 1;
    const int64_t rows = ly * lz;
    if (rows > (int64_t)0x7FFFFFFF || lx / 2 > (int64_t)0x7FFFFFFF)
        return fail(ISING_ERR_INVALID, "lattice too large for 32-bit row indices");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(ISING_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev)
        return fail(ISING_ERR_INVALID, "device %d out of range (%d devices)", device, ndev);
    TRY_CUDA(cudaSetDevice(device));

    ising_sim* h = new ising_sim();
    h->device = device;
    h->ndim = ndim;
    h->variant = variant;
    h->algorithm = algorithm;
    for (int i = 0; i < 3; ++i) h->shape[i] = i < ndim ? shape[i] : 0;
    h->rows = rows;
    h->lh = (int)(lx / 2);
    h->ly = (int)ly;
    h->lz = (int)lz;
    h->nw = (int)(lx / 128);
    h->vw = 16;                        // int8 rows padded to 16 bytes: 128-bit chunks everywhere
    h->pitch = (h->lh + 15) / 16 * 16;
    h->seed = seed;
    h->table_n = 2 * ndim + 1;
    for (int i = 0; i < 7; ++i) h->table[i] = 0xFFFFFFFFu;
    h->rule = select_rule(variant, algorithm, ndim, h->table);
    h->sm_count = device_sm_count(device);
    h->max_blocks = h->sm_count * 8;
    h->colour_bytes = variant == ISING_VARIANT_MSC ? (size_t)rows * h->nw * 8
                                                  : (size_t)rows * (size_t)h->pitch;
    cudaError_t e = cudaStreamCreateWithFlags(&h->own_stream_handle, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    h->stream = h->own_stream_handle;
    for (int c = 0; c < 2; ++c) {
        e = pool_alloc(device, &h->c[c], h->colour_bytes, h->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            h->c[c] = nullptr;
            ising_destroy(h);
            return fail(ISING_ERR_NOMEM, "allocation of %zu bytes failed: %s", h->colour_bytes,
                        cudaGetErrorString(e));
        }
    }
    e = pool_alloc(device, (void**)&h->d_acc, 8 * sizeof(unsigned long long), h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->d_acc = nullptr;
        ising_destroy(h);
        return fail(ISING_ERR_NOMEM, "allocation of the accumulators failed");
    }
    e = cudaMemsetAsync(h->d_acc, 0, 8 * sizeof(unsigned long long), h->stream);
    // the arrays are usable from any stream once their allocation has completed
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        ising_destroy(h);
        return cuda_fail(e, "initialising the accumulators");
    }
    *out = h;
    return ISING_OK;
}

int ising_destroy(ising_sim* h)
{
    if (!h) return ISING_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    // pool memory goes back to the pool, stream-ordered on the handle's own stream
    cudaStream_t fs = h->own_stream_handle;
    for (int c = 0; c < 2; ++c)
        if (h->c[c]) cudaFreeAsync(h->c[c], fs);
    if (h->d_acc) cudaFreeAsync(h->d_acc, fs);
    if (h->d_series) cudaFreeAsync(h->d_series, fs);
    for (int c = 0; c < 2; ++c)
        if (h->tb_scratch[c]) cudaFreeAsync(h->tb_scratch[c], fs);
    if (h->h_series) host_pinned_put(h->h_series, (size_t)h->series_cap * 2 * sizeof(long long));
    if (fs) cudaStreamSynchronize(fs);
    clear_graphs(h);
    if (h->d_flags) cudaFree(h->d_flags);
    if (h->d_label) cudaFree(h->d_label);
    if (h->own_stream_handle) cudaStreamDestroy(h->own_stream_handle);
    cudaGetLastError();
    delete h;
    return ISING_OK;
}

int ising_set_stream(ising_sim* h, void* stream)
{
    CHECK_HANDLE(h);
    h->stream = stream ? (cudaStream_t)stream : h->own_stream_handle;
    return ISING_OK;
}

int ising_set_table(ising_sim* h, const uint32_t* table, int n)
{
    CHECK_HANDLE(h);
    if (!table) return fail(ISING_ERR_INVALID, "null table");
    if (n != h->table_n)
        return fail(ISING_ERR_INVALID, "table must have %d entries, got %d", h->table_n, n);
    for (int i = 0; i < 7; ++i) h->table[i] = i < n ? table[i] : 0xFFFFFFFFu;
    h->rule = select_rule(h->variant, h->algorithm, h->ndim, h->table);
    clear_graphs(h);  // the table is part of the captured launches
    return ISING_OK;
}

int ising_set_seed(ising_sim* h, uint64_t seed)
{
    CHECK_HANDLE(h);
    h->seed = seed;
    clear_graphs(h);
    return ISING_OK;
}

// Bytes of one colour row in host arrays (contiguous) and on the device (pitched for int8).
static size_t host_row_bytes(const ising_sim* h)
{
    return h->variant == ISING_VARIANT_MSC ? (size_t)h->nw * 8 : (size_t)h->lh;
}

static size_t device_row_bytes(const ising_sim* h)
{
    return h->variant == ISING_VARIANT_MSC ? (size_t)h->nw * 8 : (size_t)h->pitch;
}

// Full lattices move through a bounded device staging buffer, a block of rows at a time.
static const size_t kStagingBytes = (size_t)256 << 20;

static long long rows_per_chunk(const ising_sim* h)
{
    const size_t row_bytes = (size_t)2 * h->lh;
    long long r = (long long)(kStagingBytes / row_bytes);
    if (r < 1) r = 1;
    if (h->variant == ISING_VARIANT_MSC && r > 1) r &= ~1LL;  // keep row parity aligned
    return r > h->rows ? h->rows : r;
}

int ising_set_lattice(ising_sim* h, const int8_t* full)
{
    CHECK_HANDLE(h);
    if (!full) return fail(ISING_ERR_INVALID, "null lattice");
    TRY_CUDA(cudaSetDevice(h->device));
    const long long rpc = rows_per_chunk(h);
    const size_t row_bytes = (size_t)2 * h->lh;
    int8_t* stage = nullptr;
    TRY_CUDA(pool_alloc(h->device, (void**)&stage, rpc * row_bytes, h->stream));
    int rc = ISING_OK;
    for (long long r0 = 0; r0 < h->rows && rc == ISING_OK; r0 += rpc) {
        const long long nr = (r0 + rpc > h->rows) ? h->rows - r0 : rpc;
        cudaError_t e = cudaMemcpyAsync(stage, full + r0 * row_bytes, nr * row_bytes,
                                        cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) {
            if (h->variant == ISING_VARIANT_MSC)
                e = launch_msc_pack(stage, (u64*)h->c[0] + r0 * h->nw,
                                    (u64*)h->c[1] + r0 * h->nw, (int)nr, (int)r0, h->nw,
                                    h->max_blocks, h->stream);
            else
                e = launch_int8_split(stage, (int8_t*)h->c[0] + r0 * h->pitch,
                                      (int8_t*)h->c[1] + r0 * h->pitch, nr, r0, h->lh, h->pitch,
                                      h->ly, h->max_blocks, h->stream);
        }
        if (e != cudaSuccess) rc = cuda_fail(e, "set_lattice");
    }
    cudaFreeAsync(stage, h->stream);
    if (rc == ISING_OK) TRY_CUDA(cudaStreamSynchronize(h->stream));
    return rc;
}

int ising_get_lattice(ising_sim* h, int8_t* full)
{
    CHECK_HANDLE(h);
    {
        const int prc = check_pending(h);
        if (prc != ISING_OK) return prc;
    }
    if (!full) return fail(ISING_ERR_INVALID, "null lattice");
    TRY_CUDA(cudaSetDevice(h->device));
    const long long rpc = rows_per_chunk(h);
    const size_t row_bytes = (size_t)2 * h->lh;
    int8_t* stage = nullptr;
    TRY_CUDA(pool_alloc(h->device, (void**)&stage, rpc * row_bytes, h->stream));
    int rc = ISING_OK;
    for (long long r0 = 0; r0 < h->rows && rc == ISING_OK; r0 += rpc) {
        const long long nr = (r0 + rpc > h->rows) ? h->rows - r0 : rpc;
        cudaError_t e;
        if (h->variant == ISING_VARIANT_MSC)
            e = launch_msc_unpack((const u64*)h->c[0] + r0 * h->nw,
                                  (const u64*)h->c[1] + r0 * h->nw, stage, (int)nr, (int)r0,
                                  h->nw, h->max_blocks, h->stream);
        else
            e = launch_int8_merge((const int8_t*)h->c[0] + r0 * h->pitch,
                                  (const int8_t*)h->c[1] + r0 * h->pitch, stage, nr, r0, h->lh,
                                  h->pitch,
                                  h->ly, h->max_blocks, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(full + r0 * row_bytes, stage, nr * row_bytes,
                                cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "get_lattice");
    }
    cudaFreeAsync(stage, h->stream);
    cudaStreamSynchronize(h->stream);
    return rc;
}

int ising_upload(ising_sim* h, const void* c0, const void* c1)
{
    CHECK_HANDLE(h);
    if (!c0 || !c1) return fail(ISING_ERR_INVALID, "null colour array");
    TRY_CUDA(cudaSetDevice(h->device));
    // host rows are contiguous (width) on the host, `pitch` apart on the device
    const size_t width = host_row_bytes(h), rows = (size_t)h->rows;
    const size_t dp = device_row_bytes(h);
    TRY_CUDA(cudaMemcpy2DAsync(h->c[0], dp, c0, width, width, rows, cudaMemcpyHostToDevice,
                               h->stream));
    TRY_CUDA(cudaMemcpy2DAsync(h->c[1], dp, c1, width, width, rows, cudaMemcpyHostToDevice,
                               h->stream));
    TRY_CUDA(cudaStreamSynchronize(h->stream));
    return ISING_OK;
}

int ising_download(ising_sim* h, void* c0, void* c1)
{
    CHECK_HANDLE(h);
    {
        const int prc = check_pending(h);
        if (prc != ISING_OK) return prc;
    }
    if (!c0 || !c1) return fail(ISING_ERR_INVALID, "null colour array");
    TRY_CUDA(cudaSetDevice(h->device));
    const size_t width = host_row_bytes(h), rows = (size_t)h->rows;
    const size_t dp = device_row_bytes(h);
    TRY_CUDA(cudaMemcpy2DAsync(c0, width, h->c[0], dp, width, rows, cudaMemcpyDeviceToHost,
                               h->stream));
    TRY_CUDA(cudaMemcpy2DAsync(c1, width, h->c[1], dp, width, rows, cudaMemcpyDeviceToHost,
                               h->stream));
    TRY_CUDA(cudaStreamSynchronize(h->stream));
    return ISING_OK;
}

int ising_fill_cold(ising_sim* h)
{
    CHECK_HANDLE(h);
    TRY_CUDA(cudaSetDevice(h->device));
    const int v = h->variant == ISING_VARIANT_MSC ? 0xFF : 0x01;
    for (int c = 0; c < 2; ++c) TRY_CUDA(cudaMemsetAsync(h->c[c], v, h->colour_bytes, h->stream));
    return ISING_OK;
}

int ising_fill_philox(ising_sim* h, uint64_t start_seed)
{
    CHECK_HANDLE(h);
    TRY_CUDA(cudaSetDevice(h->device));
    TRY_CUDA(launch_philox_start(h->c[0], h->c[1], h->rows, h->lh, h->pitch,
                                 h->variant == ISING_VARIANT_MSC, (u32)start_seed,
                                 (u32)(start_seed >> 32), h->max_blocks, h->stream));
    return ISING_OK;
}

int ising_set_schedule(ising_sim* h, int schedule, int test_mute_band)
{
    CHECK_HANDLE(h);
    if (schedule < ISING_SCHEDULE_AUTO || schedule > ISING_SCHEDULE_TEMPORAL)
        return fail(ISING_ERR_INVALID, "unknown schedule %d", schedule);
    h->schedule = schedule;
    h->mute_band = test_mute_band;
    return ISING_OK;
}

int ising_set_knob(ising_sim* h, int knob, int value)
{
    CHECK_HANDLE(h);
    switch (knob) {
    case ISING_KNOB_BAND:
        if (h->variant != ISING_VARIANT_INT8) return fail(ISING_ERR_INVALID, "band: int8 only");
        if (value < 0 || value > 1024) return fail(ISING_ERR_INVALID, "band must be 0..1024");
        h->band = value;
        break;
    case ISING_KNOB_CHUNK_WIDTH:
        if (h->variant != ISING_VARIANT_INT8)
            return fail(ISING_ERR_INVALID, "chunk width: int8 only");
        if (value != 16 && value != 8 && value != 4)
            return fail(ISING_ERR_INVALID, "chunk width must be 16, 8 or 4 bytes");
        if (value == 8 && h->lh % 8)
            return fail(ISING_ERR_INVALID, "chunk width 8 needs Lx/2 to be a multiple of 8");
        h->vw = value;
        break;
    case ISING_KNOB_BLOCKS_PER_SM:
        if (value < 1 || value > 32) return fail(ISING_ERR_INVALID, "blocks per SM must be 1..32");
        h->blocks_per_sm = value;
        h->max_blocks = h->sm_count * value;
        break;
    case ISING_KNOB_MSC_WAVES:
        if (value < 1 || value > 16) return fail(ISING_ERR_INVALID, "msc waves must be 1..16");
        h->msc_waves = value;
        break;
    case ISING_KNOB_GRAPH_CHUNK:
        if (value < 1 || value > kGraphChunkMax)
            return fail(ISING_ERR_INVALID, "graph chunk must be 1..%d sweeps", (int)kGraphChunkMax);
        h->graph_chunk = value;
        break;
    case ISING_KNOB_CLUSTER_TILE:
        if (value != 0 && value != 1 && (value < 32 || value > 6144))
            return fail(ISING_ERR_INVALID,
                        "cluster tile must be 0 (automatic), 1 (no tiles) or 32..6144");
        h->cluster_tile = value;
        break;
    case ISING_KNOB_MSC_KERNEL:
        if (value < 0 || value > 7) return fail(ISING_ERR_INVALID, "msc kernel must be 0..7");
        h->msc_kernel = value;
        break;
    case ISING_KNOB_TEST_LABEL_CYCLE:
        if (value != 0 && value != 1) return fail(ISING_ERR_INVALID, "test hook is 0 or 1");
        h->test_label_cycle = value;
        break;
    default: return fail(ISING_ERR_INVALID, "unknown knob %d", knob);
    }
    clear_graphs(h);  // captured graphs hold the old launch parameters
    return ISING_OK;
}

int ising_get_knob(ising_sim* h, int knob, int* value)
{
    CHECK_HANDLE(h);
    if (!value) return fail(ISING_ERR_INVALID, "null output pointer");
    switch (knob) {
    case ISING_KNOB_BAND: *value = h->band; break;
    case ISING_KNOB_CHUNK_WIDTH: *value = h->vw; break;
    case ISING_KNOB_BLOCKS_PER_SM: *value = h->blocks_per_sm; break;
    case ISING_KNOB_MSC_WAVES: *value = h->msc_waves; break;
    case ISING_KNOB_GRAPH_CHUNK: *value = (int)h->graph_chunk; break;
    case ISING_KNOB_CLUSTER_TILE: *value = h->cluster_tile; break;
    case ISING_KNOB_MSC_KERNEL: *value = h->msc_kernel; break;
    case ISING_KNOB_TEST_LABEL_CYCLE: *value = h->test_label_cycle; break;
    default: return fail(ISING_ERR_INVALID, "unknown knob %d", knob);
    }
    return ISING_OK;
}

int ising_time_sweeps(ising_sim* h, uint64_t t0, int64_t n_sweeps, float* ms)
{
    CHECK_HANDLE(h);
    if (!ms || n_sweeps <= 0) return fail(ISING_ERR_INVALID, "bad arguments");
    TRY_CUDA(cudaSetDevice(h->device));
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    int rc = ISING_OK;
    if (e == cudaSuccess) e = cudaEventRecord(a, h->stream);
    if (e == cudaSuccess) {
        rc = ising_sweep(h, t0, n_sweeps, 0, nullptr);
        if (rc == ISING_OK) e = cudaEventRecord(b, h->stream);
        if (rc == ISING_OK && e == cudaSuccess) e = cudaEventSynchronize(b);
        if (rc == ISING_OK && e == cudaSuccess) e = cudaEventElapsedTime(ms, a, b);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (rc != ISING_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "timed sweeps");
    return ISING_OK;
}

int ising_selftest_bounded_wait(int device, int* timed_out)
{
    if (!timed_out) return fail(ISING_ERR_INVALID, "null output pointer");
    return selftest_bounded_wait(device, timed_out);
}

int ising_sweep(ising_sim* h, uint64_t t0, int64_t n_sweeps, int64_t measure_every,
                int64_t* series_out)
{
    CHECK_HANDLE(h);
    {
        int rc = check_pending(h);
        if (rc != ISING_OK) return rc;
    }
    if (n_sweeps < 0) return fail(ISING_ERR_INVALID, "negative sweep count");
    if (measure_every < 0) return fail(ISING_ERR_INVALID, "negative measurement interval");
    if (measure_every > 0 && !series_out)
        return fail(ISING_ERR_INVALID, "measure_every > 0 needs series_out");
    TRY_CUDA(cudaSetDevice(h->device));
    const int64_t n_meas = measure_every > 0 ? n_sweeps / measure_every : 0;
    if (n_meas > 0) {
        int rc = ensure_series(h, n_meas);
        if (rc != ISING_OK) return rc;
        TRY_CUDA(cudaMemsetAsync(h->d_series, 0, (size_t)n_meas * 2 * sizeof(long long),
                                 h->stream));
    }
    if (use_temporal(h)) {  // before any graph capture
        int rc = temporal_scratch(h);
        if (rc != ISING_OK) return rc;
    }
    int64_t k = 0, s0 = 0;
    // Small 2D int8 lattices: all sweeps in one persistent cooperative launch.
    const bool persistent_ok = h->variant == ISING_VARIANT_INT8 && h->ndim == 2 &&
                               n_sweeps > 0 && n_sweeps < (1LL << 30);
    // (The automatic schedule uses graphs: on B200 the per-half-sweep chain of flag, halo
    // reads and fence of the persistent kernel measured 1.9x slower than replayed graphs at
    // 1024^2: 141 against 273 flips/ns, and 320 for the temporal tiles.)
    const bool want_persistent = h->schedule == ISING_SCHEDULE_PERSISTENT;
    if (persistent_ok && want_persistent) {
        if (!h->d_flags) {
            cudaError_t e = cudaMalloc(&h->d_flags, (h->sm_count + 2) * sizeof(unsigned int));
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(ISING_ERR_NOMEM, "cudaMalloc of the persistent progress flags");
            }
        }
        int* err = reinterpret_cast<int*>(h->d_flags + h->sm_count);
        int rc = run_persistent_int8(h, t0, n_sweeps, measure_every,
                                     n_meas > 0 ? (unsigned long long*)h->d_series : nullptr,
                                     h->d_flags, err, h->mute_band);
        if (rc == ISING_OK) {
            h->pending_err = true;
            if (n_meas > 0) {
                TRY_CUDA(cudaMemcpyAsync(h->h_series, h->d_series,
                                         (size_t)n_meas * 2 * sizeof(long long),
                                         cudaMemcpyDeviceToHost, h->stream));
                rc = check_pending(h);
                if (rc != ISING_OK) return rc;
                memcpy(series_out, h->h_series, (size_t)n_meas * 2 * sizeof(long long));
            }
            return ISING_OK;
        }
        if (rc != ISING_ERR_STATE) return rc;  // ISING_ERR_STATE: not resident, fall back
    }
    // Whole chunks of G sweeps replay one captured graph (G = the measurement interval, so each
    // chunk ends with its measurement); the rest is launched directly.
    const int64_t G = measure_every > 0 ? measure_every : h->graph_chunk;
    if (h->schedule != ISING_SCHEDULE_LAUNCHES && G <= kGraphChunkMax && n_sweeps >= 2 * G) {
        cudaGraphExec_t exec = nullptr;
        int rc = chunk_graph(h, G, measure_every > 0, &exec);
        if (rc != ISING_OK) return rc;
        ctl_set_kernel<<<1, 1, 0, h->stream>>>(h->d_acc + 6, t0, 0);
        TRY_CUDA(cudaGetLastError());
        const int64_t chunks = n_sweeps / G;
        for (int64_t c = 0; c < chunks; ++c) TRY_CUDA(cudaGraphLaunch(exec, h->stream));
        s0 = chunks * G;
        k = measure_every > 0 ? chunks : 0;
        // the rest (no measurement falls in it) as one more graph, captured once per length
        // and kept while the handle holds few graphs: a repeated call then issues no single
        // launches at all
        const int64_t rem = n_sweeps - s0;
        if (rem >= kGraphRemainderMin && h->graphs.size() < kGraphsKept) {
            cudaGraphExec_t rexec = nullptr;
            rc = chunk_graph(h, rem, false, &rexec);
            if (rc != ISING_OK) return rc;
            TRY_CUDA(cudaGraphLaunch(rexec, h->stream));
            s0 = n_sweeps;
        }
    }
    const bool tb = use_temporal(h);
    const int K = temporal_sweeps();
    // sweeps s .. s + K - 1 hold no measurement
    auto unmeasured = [&](int64_t s) {
        if (measure_every <= 0) return true;
        for (int i = 0; i < K; ++i)
            if ((s + i + 1) % measure_every == 0) return false;
        return true;
    };
    for (int64_t s = s0; s < n_sweeps; ++s) {
        const u32 t = (u32)(t0 + (uint64_t)s);
        const bool meas = measure_every > 0 && (s + 1) % measure_every == 0;
        if (tb && s + K <= n_sweeps && unmeasured(s)) {
            int64_t runs = 0;  // consecutive launches of K unmeasured sweeps from s
            while (s + (runs + 1) * K <= n_sweeps && unmeasured(s + runs * K)) ++runs;
            TRY_CUDA(launch_temporal_run(h, t, runs, nullptr));
            s += runs * K - 1;
            continue;
        }
        unsigned long long* m = meas ? (unsigned long long*)(h->d_series + 2 * k) : nullptr;
        int rc = half_sweep(h, 0, t, nullptr, nullptr);
        if (rc == ISING_OK) rc = half_sweep(h, 1, t, m, nullptr);
        if (rc != ISING_OK) return rc;
        if (meas) ++k;
    }
    if (n_meas > 0) {
        TRY_CUDA(cudaMemcpyAsync(h->h_series, h->d_series, (size_t)n_meas * 2 * sizeof(long long),
                                 cudaMemcpyDeviceToHost, h->stream));
        TRY_CUDA(cudaStreamSynchronize(h->stream));
        memcpy(series_out, h->h_series, (size_t)n_meas * 2 * sizeof(long long));
    }
    return ISING_OK;
}

int ising_half_sweep(ising_sim* h, int color, uint64_t t)
{
    CHECK_HANDLE(h);
    {
        const int prc = check_pending(h);
        if (prc != ISING_OK) return prc;
    }
    if (color != 0 && color != 1) return fail(ISING_ERR_INVALID, "colour must be 0 or 1");
    TRY_CUDA(cudaSetDevice(h->device));
    return half_sweep(h, color, (u32)t, nullptr, nullptr);
}

int ising_observables(ising_sim* h, int64_t* m, int64_t* e)
{
    CHECK_HANDLE(h);
    {
        const int prc = check_pending(h);
        if (prc != ISING_OK) return prc;
    }
    if (!m || !e) return fail(ISING_ERR_INVALID, "null output pointer");
    TRY_CUDA(cudaSetDevice(h->device));
    TRY_CUDA(cudaMemsetAsync(h->d_acc, 0, 2 * sizeof(unsigned long long), h->stream));
    int rc = observe(h, h->d_acc);
    if (rc != ISING_OK) return rc;
    long long out[2];
    TRY_CUDA(cudaMemcpyAsync(out, h->d_acc, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    TRY_CUDA(cudaStreamSynchronize(h->stream));
    *m = out[0];
    *e = out[1];
    return ISING_OK;
}

int ising_sync(ising_sim* h)
{
    CHECK_HANDLE(h);
    {
        const int prc = check_pending(h);
        if (prc != ISING_OK) return prc;
    }
    TRY_CUDA(cudaSetDevice(h->device));
    TRY_CUDA(cudaStreamSynchronize(h->stream));
    return ISING_OK;
}

int ising_device_bytes(ising_sim* h, int64_t* bytes)
{
    CHECK_HANDLE(h);
    if (!bytes) return fail(ISING_ERR_INVALID, "null output pointer");
    *bytes = (int64_t)(2 * h->colour_bytes + 8 * sizeof(unsigned long long) +
                       (size_t)h->series_cap * 2 * sizeof(long long));
    return ISING_OK;
}

int ising_msc_calls_per_word(ising_sim* h, uint64_t t0, int64_t n_sweeps, double* mean,
                             double* warp_max)
{
    CHECK_HANDLE(h);
    if (h->variant != ISING_VARIANT_MSC) return fail(ISING_ERR_INVALID, "not an msc simulation");
    if (n_sweeps <= 0 || !mean || !warp_max) return fail(ISING_ERR_INVALID, "bad arguments");
    TRY_CUDA(cudaSetDevice(h->device));
    unsigned long long* stats = h->d_acc + 2;
    TRY_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), h->stream));
    for (int64_t s = 0; s < n_sweeps; ++s) {
        const u32 t = (u32)(t0 + (uint64_t)s);
        int rc = half_sweep(h, 0, t, nullptr, stats);
        if (rc == ISING_OK) rc = half_sweep(h, 1, t, nullptr, stats);
        if (rc != ISING_OK) return rc;
    }
    unsigned long long out[2];
    TRY_CUDA(cudaMemcpyAsync(out, stats, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    TRY_CUDA(cudaStreamSynchronize(h->stream));
    const double words = 2.0 * (double)n_sweeps * (double)h->rows * (double)h->nw;
    *mean = (double)out[0] / words;
    *warp_max = (double)out[1] / words;
    return ISING_OK;
}

int ising_philox_rate(int device, int calls_per_thread, int repeats, double* calls_per_ns)
{
    if (!calls_per_ns || calls_per_thread <= 0 || repeats <= 0)
        return fail(ISING_ERR_INVALID, "bad arguments");
    TRY_CUDA(cudaSetDevice(device));
    const int sms = device_sm_count(device);
    const int threads = 256, blocks = sms * 8 * 4;
    u32* out = nullptr;
    TRY_CUDA(cudaMalloc(&out, (size_t)threads * blocks * sizeof(u32)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 0.0;
    cudaError_t e = launch_philox_probe(out, blocks, threads, calls_per_thread, 1u, 2u, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    for (int i = 0; i < repeats && e == cudaSuccess; ++i) {
        cudaEventRecord(a, 0);
        e = launch_philox_probe(out, blocks, threads, calls_per_thread, 1u, 2u, 0);
        cudaEventRecord(b, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double rate = (double)threads * blocks * calls_per_thread / (ms * 1e6);
        if (rate > best) best = rate;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "philox probe");
    *calls_per_ns = best;
    return ISING_OK;
}

int ising_philox_range(int device, uint32_t q0, int64_t n, uint32_t c1, uint32_t c2, uint32_t c3,
                       uint32_t k0, uint32_t k1, uint32_t* out)
{
    if (!out || n < 0) return fail(ISING_ERR_INVALID, "bad arguments");
    if (n == 0) return ISING_OK;
    TRY_CUDA(cudaSetDevice(device));
    u32* d = nullptr;
    TRY_CUDA(cudaMalloc(&d, (size_t)n * 16));
    cudaError_t e = launch_philox_range(d, n, q0, c1, c2, c3, k0, k1,
                                        device_sm_count(device) * 8, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, (size_t)n * 16, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "philox range");
    return ISING_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- internal helpers --------
namespace ising {

int ensure_series(ising_sim* h, int64_t pairs)
{
    if (pairs <= h->series_cap) return ISING_OK;
    clear_graphs(h);  // captured measured chunks point into the old buffer
    if (h->d_series) cudaFreeAsync(h->d_series, h->stream);
    if (h->h_series) {
        cudaStreamSynchronize(h->stream);  // no copy into it is still in flight
        host_pinned_put(h->h_series, (size_t)h->series_cap * 2 * sizeof(long long));
    }
    h->d_series = nullptr;
    h->h_series = nullptr;
    h->series_cap = 0;
    const size_t bytes = (size_t)pairs * 2 * sizeof(long long);
    cudaError_t e = pool_alloc(h->device, (void**)&h->d_series, bytes, h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->d_series = nullptr;
        return fail(ISING_ERR_NOMEM, "allocation of %zu series bytes failed", bytes);
    }
    e = host_pinned_get((void**)&h->h_series, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->h_series = nullptr;
        return fail(ISING_ERR_NOMEM, "cudaMallocHost of %zu bytes failed", bytes);
    }
    h->series_cap = pairs;
    return ISING_OK;
}

int half_sweep(ising_sim* h, int color, u32 t, unsigned long long* meas,
               unsigned long long* stats, const unsigned long long* ctl)
{
    const u32 k0 = (u32)h->seed, k1 = (u32)(h->seed >> 32);
    cudaError_t e;
    if (h->variant == ISING_VARIANT_MSC) {
        MscHalf p;
        p.own = (u64*)h->c[color];
        p.other = (const u64*)h->c[1 - color];
        p.rows = (int)h->rows;
        p.nw = h->nw;
        p.t = t;
        p.color = (u32)color;
        p.k0 = k0;
        p.k1 = k1;
        p.thr4 = h->table[3];
        p.thr8 = h->table[4];
        p.nw_magic = magic_for(h->nw);
        p.meas = meas;
        p.stats = stats;
        p.ctl = ctl;
        e = launch_msc_half(true, p, h->max_blocks, h->sm_count, h->msc_waves, h->stream,
                            h->msc_kernel);
    } else {
        Int8Half p;
        p.own = (int8_t*)h->c[color];
        p.other = (const int8_t*)h->c[1 - color];
        p.rows = h->rows;
        p.lh = h->lh;
        p.ly = h->ly;
        p.lz = h->lz;
        p.pitch = h->pitch;
        p.vw = h->vw;
        p.cpr = (h->lh + h->vw - 1) / h->vw;
        p.band = h->band;
        p.t = t;
        p.color = (u32)color;
        p.k0 = k0;
        p.k1 = k1;
        for (int i = 0; i < 7; ++i) p.table[i] = h->table[i];
        p.meas = meas;
        p.ctl = ctl;
        e = launch_int8_half(h->ndim, h->rule, p, h->max_blocks, h->sm_count, h->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "half-sweep launch");
    return ISING_OK;
}

int observe(ising_sim* h, unsigned long long* acc)
{
    cudaError_t e;
    if (h->variant == ISING_VARIANT_MSC) {
        MscHalf p;
        memset(&p, 0, sizeof p);
        p.own = (u64*)h->c[1];
        p.other = (const u64*)h->c[0];
        p.rows = (int)h->rows;
        p.nw = h->nw;
        p.color = 1;
        p.meas = acc;
        e = launch_msc_half(false, p, h->max_blocks, h->sm_count, 1, h->stream);
    } else {
        Int8Half p;
        memset(&p, 0, sizeof p);
        p.own = (int8_t*)h->c[1];
        p.other = (const int8_t*)h->c[0];
        p.rows = h->rows;
        p.lh = h->lh;
        p.ly = h->ly;
        p.lz = h->lz;
        p.pitch = h->pitch;
        p.vw = h->vw;
        p.cpr = (h->lh + h->vw - 1) / h->vw;
        p.color = 1;
        p.meas = acc;
        e = launch_int8_half(h->ndim, kObserve, p, h->max_blocks, h->sm_count, h->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "observables launch");
    return ISING_OK;
}

}  // namespace ising
