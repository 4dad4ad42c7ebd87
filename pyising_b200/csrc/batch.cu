// Batched ensembles and continuous-batching serving: many independent lattices of uneven size,
// dimension, variant and temperature advanced together, one grouped launch per half-sweep
// "epoch" over a (lattice, tile) work list.
//
// Every lattice keeps its own seed, table, sweep counter and measurement interval.  Its sweep
// counter at epoch e is t0 + (e - join) / 2 (lattices join at even epochs, so every launch
// updates one colour, e % 2, of every active lattice); its (M, E) after sweep s lands in its
// own series slot.  The random numbers depend only on (site, sweep, colour, seed), so each
// lattice is bit-identical to running it alone with the single-lattice kernels.
//
// Work items are tiles of ~16K int8 sites (whole rows) or ~4K packed words; items of one
// kernel class (variant, chunk width, dims, decision rule) share a launch; a block walks its
// items grid-stride.  The host engine decides membership deterministically from sweep counts,
// so it never waits for the device except to hand results back (events) and to bound how far
// it runs ahead.
#include <algorithm>
#include <climits>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "capi_internal.h"
#include "int8_core.cuh"
#include "msc_core.cuh"

namespace ising {

// One msc lattice of a batch (read from global memory by the msc kernel).
struct BatchLattice {
    void* c[2];
    long long* series;     // (M, E) pairs, or nullptr
    long long join_epoch;  // even epoch of the first half-sweep
    int rows, nw, nw_shift;
    u64 nw_magic;          // ceil(2^64 / nw)
    int every;             // measurement interval in sweeps (0 = none)
    u32 t0;
    u32 k0, k1;
    u32 table[7];
};

// Work-item sizes follow the work of each kernel class: about kItemsPerSlot items per resident
// block of the class's kernel (so a launch has no long tail and small lattices still fill the
// GPU), within these bounds; both are multiples of 256 chunks or words.
constexpr long long kInt8ItemMin = 512, kInt8ItemMax = 4096;    // band slots
constexpr long long kMscItemMin = 2048, kMscItemMax = 16384;    // words
constexpr long long kItemsPerSlot = 6;  // default of the ISING_KNOB_ITEMS_PER_SLOT knob
constexpr int kBandCap = 8;             // default of the ISING_KNOB_BAND knob (batch)

// Item size for `total` units of work over `slots` resident blocks, `per_slot` items each.
inline long long item_size(long long total, long long slots, long long per_slot, long long lo,
                           long long hi)
{
    long long want = (total + per_slot * slots - 1) / (per_slot * slots);
    return want < lo ? lo : (want > hi ? hi : want);
}

// ----------------------------------------------------------------------------- int8 -------
// An int8 launch covers up to kInt8PerLaunch lattices of one kernel class; their descriptors are
// the launch's parameter block (constant memory), so every field a block reads is uniform, as
// in the single-lattice kernel.  Block b belongs to the last lattice whose block_begin <= b (a
// uniform binary search) and updates its slots [(b - block_begin) * per, ...), a slot being a
// band of L.band rows of one plane in one chunk column (int8_band), band-major.
struct Int8Desc {
    void* c[2];
    long long* series;     // (M, E) pairs, or nullptr
    long long join_epoch;  // even epoch of the first half-sweep
    int every;             // measurement interval in sweeps (0 = none)
    u32 t0, k0, k1;
    u32 table[7];
    int rows, lh, ly, lz, pitch, cpr, band, bpp;
    u32 cpr_magic, bpp_magic;  // fast_div magics of cpr and bpp
    int block_begin;           // first block of this lattice in the launch
    int per_block;             // band slots per block (a multiple of 256)
    int nslots;                // band slots of the lattice: lz * bpp * cpr
};

// Parameter blocks come in three capacities; a launch passes the smallest that holds its
// lattices, since the host cost of a launch grows with the size of its parameters.
constexpr int kInt8PerLaunch = 240;

template <int N>
struct Int8LaunchN {
    long long epoch;               // the launch's epoch, relative to *epoch_base when set
    const long long* epoch_base;   // replayed graph chunks: device epoch counter, else nullptr
    int n;  // lattices
    int pad;
    Int8Desc lat[N];
};
using Int8Launch = Int8LaunchN<kInt8PerLaunch>;
static_assert(sizeof(Int8Launch) <= 32764, "kernel parameter block over the 32 KB limit");

template <int V, int NDIM, int RULE, bool MIXED, bool MEAS>
__device__ __forceinline__ void batch_int8_slots(const Int8Half& p, const Int8Desc& L, u32 s0,
                                                 u32 s1, const u32* stab, long long& m_acc,
                                                 long long& e_acc)
{
    const u32 cpr = (u32)L.cpr, bpp = (u32)L.bpp;
    for (u32 slot = s0 + threadIdx.x; slot < s1; slot += 256u) {
        const u32 band = fast_div(slot, cpr, L.cpr_magic);
        const int j0 = (int)(slot - band * cpr) * V;
        int z = 0, yb = (int)band;
        if constexpr (NDIM == 3) {
            z = (int)fast_div(band, bpp, L.bpp_magic);
            yb = (int)(band - (u32)z * bpp);
        }
        const int y0 = yb * L.band;
        const int y1 = y0 + L.band < L.ly ? y0 + L.band : L.ly;
        int8_band<V, NDIM, RULE, MIXED, MEAS>(p, z, y0, y1, j0, stab, m_acc, e_acc);
    }
}

#ifndef ISING_BATCH_MIN_BLOCKS
#define ISING_BATCH_MIN_BLOCKS 4
#endif
template <int V, int NDIM, int RULE, bool MIXED, int N>
__global__ void __launch_bounds__(256, ISING_BATCH_MIN_BLOCKS)
    batch_int8_kernel(const __grid_constant__ Int8LaunchN<N> P)
{
    __shared__ u32 stab[8];  // acceptance table for the per-site lookup rules
    // launched with programmatic stream serialization: wait for the previous kernel of the
    // stream (every kernel of the engine's stream waits on its predecessor in turn, so this
    // class's previous half-sweep has completed too), then let the next launch start
    pdl_wait();
    pdl_trigger();
    const int b = (int)blockIdx.x;
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.lat[mid].block_begin <= b) lo = mid;
        else hi = mid - 1;
    }
    const Int8Desc& L = P.lat[lo];
    if constexpr (RULE != kMetroFast) {
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < 7; ++i) stab[i] = L.table[i];
        }
        __syncthreads();
    }
    const long long epoch = P.epoch + (P.epoch_base ? *P.epoch_base : 0);
    const u32 color = (u32)(epoch & 1);
    const u32 s = (u32)((epoch - L.join_epoch) >> 1);  // sweeps done (< 2^31)
    const bool meas = color == 1 && L.every > 0 && ((s + 1u) % (u32)L.every) == 0;
    Int8Half p;
    p.own = static_cast<int8_t*>(L.c[color]);
    p.other = static_cast<const int8_t*>(L.c[color ^ 1]);
    p.rows = L.rows;
    p.lh = L.lh;
    p.ly = L.ly;
    p.lz = L.lz;
    p.cpr = L.cpr;
    p.pitch = L.pitch;
    p.vw = V;
    p.t = L.t0 + s;
    p.color = color;
    p.k0 = L.k0;
    p.k1 = L.k1;
#pragma unroll
    for (int i = 0; i < 7; ++i) p.table[i] = L.table[i];
    p.meas = meas ? reinterpret_cast<unsigned long long*>(
                        L.series + 2 * ((s + 1u) / (u32)L.every - 1u))
                  : nullptr;
    p.ctl = nullptr;
    const u32 s0 = (u32)(b - L.block_begin) * (u32)L.per_block;
    const u32 s1 = s0 + (u32)L.per_block < (u32)L.nslots ? s0 + (u32)L.per_block : (u32)L.nslots;
    long long m_acc = 0, e_acc = 0;
    if (meas) {
        batch_int8_slots<V, NDIM, RULE, MIXED, true>(p, L, s0, s1, stab, m_acc, e_acc);
        block_accumulate2(m_acc, e_acc, p.meas);
    } else {
        batch_int8_slots<V, NDIM, RULE, MIXED, false>(p, L, s0, s1, stab, m_acc, e_acc);
    }
}

// ------------------------------------------------------------------------------ msc -------
struct BatchItem {
    int lat;
    int pad;
    long long begin, end;  // words
};

constexpr int kBatchWarps = 8;

__global__ void __launch_bounds__(kBatchWarps * 32) batch_msc_kernel(
    const BatchLattice* __restrict__ lats, const BatchItem* __restrict__ items, int n_items,
    long long epoch_rel, const long long* epoch_base)
{
    __shared__ QueueSlots q_all[kBatchWarps];
    __shared__ uint4 lvmask[16];
    // (launched without programmatic serialization: its early-launched blocks would hold their
    // 17 KB work stacks while waiting, and the batch measured slower with it)
    // the epoch, relative to the device counter in replayed graph chunks
    const long long epoch = epoch_rel + (epoch_base ? *epoch_base : 0);
    const u32 color = (u32)(epoch & 1);
    const int warp = threadIdx.x >> 5;
    long long m_acc = 0, e_acc = 0;  // flushed per lattice, as in batch_int8_kernel
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const BatchLattice& L = lats[item.lat];
        const u32 s = (u32)((epoch - L.join_epoch) >> 1);  // sweeps done (< 2^31)
        const bool meas = color == 1 && L.every > 0 && ((s + 1u) % (u32)L.every) == 0;
        MscHalf p;
        p.own = static_cast<u64*>(L.c[color]);
        p.other = static_cast<const u64*>(L.c[color ^ 1]);
        p.rows = L.rows;
        p.nw = L.nw;
        p.t = L.t0 + s;
        p.color = color;
        p.k0 = L.k0;
        p.k1 = L.k1;
        p.thr4 = L.table[3];
        p.thr8 = L.table[4];
        p.nw_magic = L.nw_magic;
        p.stats = nullptr;
        p.ctl = nullptr;
        p.meas = meas ? reinterpret_cast<unsigned long long*>(
                            L.series + 2 * ((s + 1u) / (u32)L.every - 1u))
                      : nullptr;
        if (threadIdx.x < 16) lvmask[threadIdx.x] = level_masks(p.thr4, p.thr8, threadIdx.x);
        __syncthreads();
        const long long len = item.end - item.begin;
        long long per = (len + kBatchWarps - 1) / kBatchWarps;
        per = (per + 31) / 32 * 32;
        const long long b = item.begin + warp * per;
        const long long e = min(b + per, item.end);
        msc_queue_range(p, b, e, L.nw_shift, q_all[warp], lvmask);
        if (meas) {
            // the warp's words are final: measure them (the other colour is unchanged)
            __syncwarp();
            msc_measure_range(p, b, e, L.nw_shift, m_acc, e_acc);
            if (it + (int)gridDim.x >= n_items || items[it + gridDim.x].lat != item.lat) {
                block_accumulate2(m_acc, e_acc, p.meas);
                m_acc = e_acc = 0;
            }
        }
        __syncthreads();
    }
}

__global__ void batch_epoch_set(long long* counter, long long epoch) { *counter = epoch; }

// ----------------------------------------------------------------------------- host engine ---

using Clock = std::chrono::steady_clock;

struct Job {
    int64_t id = 0;
    int state = ISING_JOB_PENDING;
    ising_job spec;
    std::vector<int8_t> init;  // host copy of an initial lattice (ISING_INIT_LATTICE)
    int rows = 0, lh = 0, ly = 0, lz = 1, nw = 0;
    int pitch = 0;  // int8: bytes between rows on the device (lh rounded up to 16)
    size_t colour_bytes = 0, series_pairs = 0, device_bytes = 0;
    void* c[2] = {nullptr, nullptr};
    long long* d_series = nullptr;
    long long* h_series = nullptr;  // pinned
    int8_t* h_lattice = nullptr;    // pinned, keep_lattice only
    long long join_epoch = -1;
    cudaEvent_t done_event = nullptr;
    Clock::time_point t_submit, t_start, t_done;
    std::string error;
};

struct KernelClass {
    int variant, v, ndim, rule, mixed;  // mixed: rows padded (lh % 16 != 0)
    bool operator<(const KernelClass& o) const
    {
        return std::tie(variant, v, ndim, rule, mixed) <
               std::tie(o.variant, o.v, o.ndim, o.rule, o.mixed);
    }
};

class Engine {
public:
    Engine(int device, int64_t budget) : device_(device), budget_(budget) {}

    int init()
    {
        cudaError_t e = cudaSetDevice(device_);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
        sms_ = device_sm_count(device_);
        // The engine's own stream-ordered pool keeps freed lattice memory (up to the budget)
        // mapped across synchronisations, so admitting a job after another finished reuses it
        // instead of mapping fresh pages; the device's default pool is left untouched.
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device_;
        e = cudaMemPoolCreate(&pool_, &props);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
        uint64_t keep = (uint64_t)budget_;
        e = cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolSetAttribute");
        e = cudaMalloc((void**)&d_epoch_, sizeof(long long));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (epoch counter)");
        return ISING_OK;
    }

    ~Engine()
    {
        cudaSetDevice(device_);
        if (stream_) cudaStreamSynchronize(stream_);
        for (auto& kv : jobs_) free_job(*kv.second);
        if (d_lats_) cudaFreeAsync(d_lats_, stream_);
        if (d_items_) cudaFreeAsync(d_items_, stream_);
        if (stream_) cudaStreamSynchronize(stream_);
        if (chunk_exec_) cudaGraphExecDestroy(chunk_exec_);
        for (auto& x : old_execs_) {
            cudaGraphExecDestroy(x.first);
            cudaEventDestroy(x.second);
        }
        if (d_epoch_) cudaFree(d_epoch_);
        for (auto& kv : pinned_free_) cudaFreeHost(kv.second);
        for (cudaEvent_t ev : epoch_events_) cudaEventDestroy(ev);
        if (stream_) cudaStreamDestroy(stream_);
        if (pool_) cudaMemPoolDestroy(pool_);
        cudaGetLastError();
    }

    // Validates the job and queues it; returns its id.
    int submit(const ising_job& spec, int64_t* id)
    {
        auto j = std::make_unique<Job>();
        int rc = validate(spec, *j);
        if (rc != ISING_OK) return rc;
        j->spec = spec;
        if (spec.init == ISING_INIT_LATTICE) {
            const size_t n = (size_t)j->rows * 2 * j->lh;
            j->init.assign(spec.lattice, spec.lattice + n);
        }
        j->spec.lattice = nullptr;
        if ((int64_t)j->device_bytes > budget_)
            return fail(ISING_ERR_NOMEM, "job needs %zu device bytes, over the %lld-byte budget",
                        j->device_bytes, (long long)budget_);
        // the pinned host buffers of the results are taken now, on the submitting thread:
        // page-locking memory while the job finishes would stall the sweeps in flight
        cudaError_t e = cudaSuccess;
        if (j->series_pairs)
            e = pinned_get((void**)&j->h_series, j->series_pairs * 2 * sizeof(long long));
        if (e == cudaSuccess && spec.keep_lattice)
            e = pinned_get((void**)&j->h_lattice, (size_t)j->rows * 2 * j->lh);
        if (e != cudaSuccess) {
            cudaGetLastError();
            free_job(*j);
            return fail(ISING_ERR_NOMEM, "pinned result buffers of a job");
        }
        j->id = ++last_id_;
        j->t_submit = Clock::now();
        *id = j->id;
        pending_.push_back(j->id);
        jobs_[j->id] = std::move(j);
        return ISING_OK;
    }

    bool busy() const { return !active_.empty() || !pending_.empty() || !finishing_.empty(); }
    bool has_work() const { return !active_.empty() || !pending_.empty(); }
    size_t active_count() const { return active_.size(); }
    size_t pending_count() const { return pending_.size(); }
    long long epoch() const { return epoch_; }
    int64_t used_bytes() const { return used_; }

    // One half-sweep of every active lattice (admitting pending jobs at even epochs).
    // Issues the next epoch, or the next replayed chunk of 2 * chunk_sweeps_ epochs when the
    // batch is stable and `budget` (epochs the caller still allows; <= 0: no limit) holds it.
    int step(long long budget = 0)
    {
        cudaError_t e = cudaSetDevice(device_);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
        if ((epoch_ & 1) == 0) {
            int rc = admit();
            if (rc != ISING_OK) return rc;
        }
        if (active_.empty()) return ISING_OK;
        if (dirty_) {
            drop_chunk();
            int rc = rebuild();
            if (rc != ISING_OK) return rc;
        }
        reap_chunks();
        if (chunk_ready() && (budget <= 0 || 2 * chunk_sweeps_ <= budget)) {
            int rc = run_chunk();
            if (rc == ISING_OK) rc = retire();
            if (rc == ISING_OK) rc = throttle();
            return rc;
        }
        e = launch_epoch(epoch_, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "batch launch");
        ++epoch_;
        if ((epoch_ & 1) == 0) {
            int rc = retire();
            if (rc != ISING_OK) return rc;
            rc = throttle();
            if (rc != ISING_OK) return rc;
        }
        return ISING_OK;
    }

    // Marks finished result copies as done; returns how many completed.
    int poll()
    {
        int n = 0;
        for (auto it = finishing_.begin(); it != finishing_.end();) {
            Job& j = *jobs_[*it];
            const cudaError_t e = cudaEventQuery(j.done_event);
            if (e == cudaSuccess) {
                j.state = ISING_JOB_DONE;
                j.t_done = Clock::now();
                cudaEventDestroy(j.done_event);
                j.done_event = nullptr;
                it = finishing_.erase(it);
                ++n;
            } else if (e == cudaErrorNotReady) {
                ++it;
            } else {
                return cuda_fail(e, "result event");
            }
        }
        return n;
    }

    int wait_finishing()
    {
        cudaError_t e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
        poll();
        return ISING_OK;
    }

    Job* find(int64_t id)
    {
        auto it = jobs_.find(id);
        return it == jobs_.end() ? nullptr : it->second.get();
    }

    int result(int64_t id, int64_t* series_out, int8_t* lattice_out, double* latency)
    {
        Job* j = find(id);
        if (!j) return fail(ISING_ERR_INVALID, "unknown job %lld", (long long)id);
        if (j->state != ISING_JOB_DONE)
            return fail(ISING_ERR_STATE, "job %lld is not done", (long long)id);
        if (series_out && j->series_pairs)
            memcpy(series_out, j->h_series, j->series_pairs * 2 * sizeof(long long));
        if (lattice_out) {
            if (!j->h_lattice)
                return fail(ISING_ERR_STATE, "job %lld was not submitted with keep_lattice",
                            (long long)id);
            memcpy(lattice_out, j->h_lattice, (size_t)j->rows * 2 * j->lh);
        }
        if (latency)
            *latency = std::chrono::duration<double>(j->t_done - j->t_submit).count();
        return ISING_OK;
    }

    int release(int64_t id)
    {
        auto it = jobs_.find(id);
        if (it == jobs_.end()) return fail(ISING_ERR_INVALID, "unknown job %lld", (long long)id);
        Job& j = *it->second;
        if (j.state == ISING_JOB_ACTIVE || j.state == ISING_JOB_FINISHING)
            return fail(ISING_ERR_STATE, "job %lld is still running", (long long)id);
        if (j.state == ISING_JOB_PENDING)
            pending_.erase(std::remove(pending_.begin(), pending_.end(), id), pending_.end());
        free_job(j);
        jobs_.erase(it);
        return ISING_OK;
    }

    int64_t budget() const { return budget_; }
    cudaStream_t stream() const { return stream_; }

    // Launch knobs of the batch (identical results for every value); applied at the next
    // rebuild of the work list.
    int set_knob(int knob, int value)
    {
        if (knob == ISING_KNOB_BAND) {
            if (value < 1 || value > 64) return fail(ISING_ERR_INVALID, "band cap must be 1..64");
            band_cap_ = value;
        } else if (knob == ISING_KNOB_ITEMS_PER_SLOT) {
            if (value < 1 || value > 64)
                return fail(ISING_ERR_INVALID, "items per slot must be 1..64");
            items_per_slot_ = value;
        } else if (knob == ISING_KNOB_GRAPH_CHUNK) {
            if (value < 0 || value > 64)
                return fail(ISING_ERR_INVALID, "batch graph chunk must be 0..64 sweeps");
            chunk_sweeps_ = value;
            drop_chunk();
        } else {
            return fail(ISING_ERR_INVALID, "knob %d does not apply to a batch", knob);
        }
        dirty_ = true;
        return ISING_OK;
    }

    int get_knob(int knob, int* value) const
    {
        if (knob == ISING_KNOB_BAND) *value = band_cap_;
        else if (knob == ISING_KNOB_ITEMS_PER_SLOT) *value = (int)items_per_slot_;
        else if (knob == ISING_KNOB_GRAPH_CHUNK) *value = (int)chunk_sweeps_;
        else return fail(ISING_ERR_INVALID, "knob %d does not apply to a batch", knob);
        return ISING_OK;
    }

private:
    int validate(const ising_job& s, Job& j)
    {
        if (s.ndim != 2 && s.ndim != 3)
            return fail(ISING_ERR_INVALID, "only 2D and 3D lattices are supported");
        for (int i = 0; i < s.ndim; ++i)
            if (s.shape[i] < 2 || s.shape[i] % 2)
                return fail(ISING_ERR_INVALID, "all extents must be even and >= 2");
        if (s.variant != ISING_VARIANT_INT8 && s.variant != ISING_VARIANT_MSC)
            return fail(ISING_ERR_INVALID, "unknown variant %d", s.variant);
        if (s.algorithm != ISING_METROPOLIS && s.algorithm != ISING_HEATBATH)
            return fail(ISING_ERR_INVALID, "unknown algorithm %d", s.algorithm);
        if (s.variant == ISING_VARIANT_MSC && (s.ndim != 2 || s.algorithm != ISING_METROPOLIS))
            return fail(ISING_ERR_INVALID, "msc supports 2D Metropolis only");
        const int64_t lx = s.shape[s.ndim - 1];
        if (lx % (s.variant == ISING_VARIANT_MSC ? 128 : 8))
            return fail(ISING_ERR_INVALID, "last extent must be a multiple of %d",
                        s.variant == ISING_VARIANT_MSC ? 128 : 8);
        if (s.table_n != 2 * s.ndim + 1)
            return fail(ISING_ERR_INVALID, "table must have %d entries", 2 * s.ndim + 1);
        if (s.n_sweeps < 0 || s.measure_every < 0)
            return fail(ISING_ERR_INVALID, "negative sweep count or interval");
        if (s.init != ISING_INIT_COLD && s.init != ISING_INIT_PHILOX && s.init != ISING_INIT_LATTICE)
            return fail(ISING_ERR_INVALID, "unknown init %d", s.init);
        if (s.init == ISING_INIT_LATTICE && !s.lattice)
            return fail(ISING_ERR_INVALID, "ISING_INIT_LATTICE needs a lattice");
        const int64_t ly = s.shape[s.ndim - 2], lz = s.ndim == 3 ? s.shape[0] : 1;
        if (ly * lz > 0x7FFFFFFF || lx / 2 > 0x7FFFFFFF)
            return fail(ISING_ERR_INVALID, "lattice too large");
        if (s.variant == ISING_VARIANT_INT8 && ly * lz * ((lx / 2 + 15) / 16) > 0x7FFFFFFF)
            return fail(ISING_ERR_INVALID, "lattice too large for the batch (2^31 chunks)");
        j.rows = (int)(ly * lz);
        j.lh = (int)(lx / 2);
        j.ly = (int)ly;
        j.lz = (int)lz;
        j.nw = (int)(lx / 128);
        j.pitch = (j.lh + 15) / 16 * 16;
        j.colour_bytes = s.variant == ISING_VARIANT_MSC ? (size_t)j.rows * j.nw * 8
                                                       : (size_t)j.rows * j.pitch;
        j.series_pairs = s.measure_every > 0 ? (size_t)(s.n_sweeps / s.measure_every) : 0;
        j.device_bytes = 2 * j.colour_bytes + j.series_pairs * 2 * sizeof(long long);
        return ISING_OK;
    }

    int admit()
    {
        for (auto it = pending_.begin(); it != pending_.end();) {
            Job& j = *jobs_[*it];
            if (used_ + (int64_t)j.device_bytes > budget_) {
                ++it;  // later, smaller jobs may still fit
                continue;
            }
            int rc = start_job(j);
            if (rc != ISING_OK) return rc;
            it = pending_.erase(it);
        }
        return ISING_OK;
    }

    int start_job(Job& j)
    {
        cudaError_t e;
        for (int c = 0; c < 2; ++c) {
            e = dev_alloc(&j.c[c], j.colour_bytes);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync (job lattice)");
        }
        if (j.series_pairs) {
            const size_t sb = j.series_pairs * 2 * sizeof(long long);
            e = dev_alloc((void**)&j.d_series, sb);
            if (e == cudaSuccess) e = cudaMemsetAsync(j.d_series, 0, sb, stream_);
            if (e != cudaSuccess) return cuda_fail(e, "job series");
        }
        const ising_job& s = j.spec;
        const int max_blocks = sms_ * 8;
        if (s.init == ISING_INIT_COLD) {
            const int v = s.variant == ISING_VARIANT_MSC ? 0xFF : 0x01;
            for (int c = 0; c < 2 && e == cudaSuccess; ++c)
                e = cudaMemsetAsync(j.c[c], v, j.colour_bytes, stream_);
        } else if (s.init == ISING_INIT_PHILOX) {
            e = launch_philox_start(j.c[0], j.c[1], j.rows, j.lh, j.pitch,
                                    s.variant == ISING_VARIANT_MSC, (u32)s.seed,
                                    (u32)(s.seed >> 32), max_blocks, stream_);
        } else {
            const size_t full = (size_t)j.rows * 2 * j.lh;
            int8_t* stage = nullptr;
            e = dev_alloc((void**)&stage, full);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(stage, j.init.data(), full, cudaMemcpyHostToDevice, stream_);
            if (e == cudaSuccess) {
                if (s.variant == ISING_VARIANT_MSC)
                    e = launch_msc_pack(stage, (u64*)j.c[0], (u64*)j.c[1], j.rows, 0, j.nw,
                                        max_blocks, stream_);
                else
                    e = launch_int8_split(stage, (int8_t*)j.c[0], (int8_t*)j.c[1], j.rows, 0,
                                          j.lh, j.pitch, j.ly, max_blocks, stream_);
            }
            if (stage) cudaFreeAsync(stage, stream_);
            std::vector<int8_t>().swap(j.init);
        }
        if (e != cudaSuccess) return cuda_fail(e, "job start");
        used_ += (int64_t)j.device_bytes;
        j.join_epoch = epoch_;
        j.state = ISING_JOB_ACTIVE;
        j.t_start = Clock::now();
        if (s.n_sweeps == 0) {
            j.state = ISING_JOB_ACTIVE;
            return finish_job(j);
        }
        active_.push_back(j.id);
        dirty_ = true;
        return ISING_OK;
    }

    // Builds the launch lists, grouped by kernel class: for int8 classes the lattice
    // descriptors of each launch (chunks of kInt8PerLaunch), for msc the lattice table and the
    // work items in device memory.
    int rebuild()
    {
        std::vector<BatchLattice> lats;              // msc lattices
        std::map<KernelClass, std::vector<Int8Desc>> int8_descs;
        std::map<KernelClass, long long> class_units;  // chunk-rows (int8) or words (msc)
        std::vector<std::pair<KernelClass, int>> msc_of;  // (class, index in lats)
        for (int64_t id : active_) {
            Job& j = *jobs_[id];
            const ising_job& s = j.spec;
            u32 table[7];
            for (int i = 0; i < 7; ++i) table[i] = i < s.table_n ? s.table[i] : 0xFFFFFFFFu;
            KernelClass kc{s.variant, 0, s.ndim, 0, 0};
            if (s.variant == ISING_VARIANT_MSC) {
                BatchLattice L;
                memset(&L, 0, sizeof L);
                L.c[0] = j.c[0];
                L.c[1] = j.c[1];
                L.series = j.d_series;
                L.join_epoch = j.join_epoch;
                L.rows = j.rows;
                L.nw = j.nw;
                L.nw_shift = (j.nw & (j.nw - 1)) == 0 ? __builtin_ctz((unsigned)j.nw) : -1;
                L.nw_magic = magic_for(j.nw);
                L.every = (int)s.measure_every;
                L.t0 = (u32)s.t0;
                L.k0 = (u32)s.seed;
                L.k1 = (u32)(s.seed >> 32);
                memcpy(L.table, table, sizeof table);
                class_units[kc] += (long long)j.rows * j.nw;
                msc_of.emplace_back(kc, (int)lats.size());
                lats.push_back(L);
            } else {
                Int8Desc D;
                memset(&D, 0, sizeof D);
                D.c[0] = j.c[0];
                D.c[1] = j.c[1];
                D.series = j.d_series;
                D.join_epoch = j.join_epoch;
                D.every = (int)s.measure_every;
                D.t0 = (u32)s.t0;
                D.k0 = (u32)s.seed;
                D.k1 = (u32)(s.seed >> 32);
                memcpy(D.table, table, sizeof table);
                D.rows = j.rows;
                D.lh = j.lh;
                D.ly = j.ly;
                D.lz = j.lz;
                D.pitch = j.pitch;  // rows padded to 16 bytes: chunk width 16
                D.cpr = (j.lh + 15) / 16;
                kc.v = 16;
                kc.mixed = (j.lh % 16) != 0;
                kc.rule = select_rule(s.variant, s.algorithm, s.ndim, table);
                class_units[kc] += (long long)j.rows * D.cpr;
                int8_descs[kc].push_back(D);
            }
        }
        // int8: the class's band height is the longest power of two up to the band cap that
        // still leaves items_per_slot blocks of one slot per thread per resident block; blocks
        // of a lattice hold per_block slots, sized the same way
        int8_launches_.clear();
        for (auto& kv : int8_descs) {
            const KernelClass& kc = kv.first;
            const long long units = class_units[kc];
            const long long want = items_per_slot_ * 256 * slots(kc);
            int band = 1;
            while (band * 2 <= band_cap_) band *= 2;
            while (band > 1 && units / band < want) band >>= 1;
            long long per = item_size(units / band, slots(kc), items_per_slot_, kInt8ItemMin,
                                      kInt8ItemMax);
            per = (per + 255) / 256 * 256;
            std::vector<Int8Launch> launches;
            for (size_t i = 0; i < kv.second.size(); ++i) {
                if (i % kInt8PerLaunch == 0) {
                    launches.emplace_back();
                    memset(&launches.back(), 0, sizeof(Int8Launch));
                }
                Int8Launch& P = launches.back();
                Int8Desc D = kv.second[i];
                D.band = band < D.ly ? band : D.ly;
                D.bpp = (D.ly + D.band - 1) / D.band;
                const long long nslots = (long long)D.lz * D.bpp * D.cpr;
                D.nslots = (int)nslots;
                D.cpr_magic = fast_div_magic((u32)D.cpr, (unsigned long long)nslots);
                D.bpp_magic = fast_div_magic((u32)D.bpp, (unsigned long long)D.lz * D.bpp);
                D.per_block = (int)per;
                const int prev = P.n ? P.lat[P.n - 1].block_begin +
                                           (P.lat[P.n - 1].nslots + P.lat[P.n - 1].per_block - 1) /
                                               P.lat[P.n - 1].per_block
                                     : 0;
                D.block_begin = prev;
                P.lat[P.n++] = D;
            }
            int8_launches_.emplace_back(kc, std::move(launches));
        }
        // msc: work items of whole 256-word runs over the class's lattices
        std::map<KernelClass, std::vector<BatchItem>> by_class;
        for (const auto& m : msc_of) {
            const KernelClass& kc = m.first;
            const BatchLattice& L = lats[m.second];
            const long long words = (long long)L.rows * L.nw;
            long long per = item_size(class_units[kc], slots(kc), items_per_slot_, kMscItemMin,
                                      kMscItemMax);
            per = (per + 255) / 256 * 256;
            for (long long b = 0; b < words; b += per)
                by_class[kc].push_back(BatchItem{m.second, 0, b, std::min(words, b + per)});
        }
        std::vector<BatchItem> items;
        classes_.clear();
        for (auto& kv : by_class) {
            classes_.emplace_back(kv.first, std::make_pair((int)items.size(), (int)kv.second.size()));
            items.insert(items.end(), kv.second.begin(), kv.second.end());
        }
        int rc = upload(lats.data(), lats.size() * sizeof(BatchLattice), (void**)&d_lats_, &lats_cap_);
        if (rc == ISING_OK)
            rc = upload(items.data(), items.size() * sizeof(BatchItem), (void**)&d_items_, &items_cap_);
        dirty_ = false;
        return rc;
    }

    // Blocks of an int8 launch: the last lattice's block_begin plus its blocks.
    static unsigned int8_grid(const Int8Launch& P)
    {
        const Int8Desc& L = P.lat[P.n - 1];
        return (unsigned)(L.block_begin + (L.nslots + L.per_block - 1) / L.per_block);
    }

    // Resident blocks of a class's kernel on the whole device.
    long long slots(const KernelClass& kc)
    {
        const void* fn = kc.variant == ISING_VARIANT_MSC
                             ? (const void*)batch_msc_kernel
                             : (const void*)batch_int8_kernel<16, 2, kMetroFast, false, 16>;
        // (one occupancy for all int8 classes: they share the launch bounds)
        return (long long)sms_ * blocks_per_sm(fn, kc.variant == ISING_VARIANT_MSC
                                                       ? kBatchWarps * 32 : 256);
    }

    int upload(const void* src, size_t bytes, void** dst, size_t* cap)
    {
        if (bytes == 0) return ISING_OK;
        if (bytes > *cap) {
            if (*dst) cudaFreeAsync(*dst, stream_);
            size_t nc = std::max(bytes, *cap * 2);
            cudaError_t e = dev_alloc(dst, nc);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync (work list)");
            *cap = nc;
        }
        // pageable source: staged by the driver before the call returns
        cudaError_t e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream_);
        if (e != cudaSuccess) return cuda_fail(e, "work list upload");
        return ISING_OK;
    }

    int blocks_per_sm(const void* fn, int threads)
    {
        int& per_sm = occupancy_[fn];
        if (per_sm < 1 &&
            (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess ||
             per_sm < 1)) {
            cudaGetLastError();
            per_sm = 2;
        }
        return per_sm;
    }

    int grid_for(const void* fn, int n_items, int threads = 256)
    {
        const int g = sms_ * blocks_per_sm(fn, threads);
        return n_items < g ? n_items : g;
    }

    template <int V, int NDIM, bool MIXED, int N>
    cudaError_t launch_int8_cap(int rule, const Int8Launch& full)
    {
        Int8LaunchN<N> P;
        P.epoch = full.epoch;
        P.epoch_base = full.epoch_base;
        P.n = full.n;
        P.pad = 0;
        memcpy(P.lat, full.lat, (size_t)full.n * sizeof(Int8Desc));
        const dim3 grid(int8_grid(full)), block(256);
        switch (rule) {
        case kMetroFast:
            return launch_pdl(batch_int8_kernel<V, NDIM, kMetroFast, MIXED, N>, grid, block, stream_, P);
        case kHeatFast:
            return launch_pdl(batch_int8_kernel<V, NDIM, kHeatFast, MIXED, N>, grid, block, stream_, P);
        case kMetroGeneric:
            return launch_pdl(batch_int8_kernel<V, NDIM, kMetroGeneric, MIXED, N>, grid, block,
                              stream_, P);
        case kHeatGeneric:
            return launch_pdl(batch_int8_kernel<V, NDIM, kHeatGeneric, MIXED, N>, grid, block,
                              stream_, P);
        default: return cudaErrorInvalidValue;
        }
    }

    template <int V, int NDIM, bool MIXED>
    cudaError_t launch_int8_rule(int rule, const Int8Launch& P)
    {
        if (P.n <= 16) return launch_int8_cap<V, NDIM, MIXED, 16>(rule, P);
        if (P.n <= 64) return launch_int8_cap<V, NDIM, MIXED, 64>(rule, P);
        return launch_int8_cap<V, NDIM, MIXED, kInt8PerLaunch>(rule, P);
    }

    // int8 rows are padded to 16 bytes, so the chunk width is always 16; lattices whose rows are
    // a multiple of 16 get the kernel without the partial-chunk code.
    cudaError_t launch_int8(const KernelClass& kc, const Int8Launch& P)
    {
        if (kc.ndim == 3)
            return kc.mixed ? launch_int8_rule<16, 3, true>(kc.rule, P)
                            : launch_int8_rule<16, 3, false>(kc.rule, P);
        return kc.mixed ? launch_int8_rule<16, 2, true>(kc.rule, P)
                        : launch_int8_rule<16, 2, false>(kc.rule, P);
    }

    cudaError_t launch_msc(int off, int n, long long epoch, const long long* epoch_base)
    {
        auto fn = batch_msc_kernel;
        const dim3 grid(grid_for((const void*)fn, n, kBatchWarps * 32)), block(kBatchWarps * 32);
        fn<<<grid, block, 0, stream_>>>(d_lats_, d_items_ + off, n, epoch, epoch_base);
        return cudaGetLastError();
    }

    // Every class's launches of one epoch (absolute, or relative to *epoch_base).
    cudaError_t launch_epoch(long long epoch, const long long* epoch_base)
    {
        cudaError_t e = cudaSuccess;
        for (auto& cl : int8_launches_) {
            for (Int8Launch& P : cl.second) {
                P.epoch = epoch;
                P.epoch_base = epoch_base;
                e = launch_int8(cl.first, P);
                if (e != cudaSuccess) return e;
            }
        }
        for (const auto& cl : classes_) {
            e = launch_msc(cl.second.first, cl.second.second, epoch, epoch_base);
            if (e != cudaSuccess) return e;
        }
        return e;
    }

    // ---- graph chunks: kChunkSweeps sweeps of a stable batch replayed from one graph ----
    // While no job can join (admission happens at even epochs, and pending jobs that did not
    // fit can only fit after a job retires) and every active job has kChunkSweeps sweeps left,
    // the batch's launches repeat with only the epoch changing: they are captured once per
    // membership, reading the epoch from a device counter set before each replay.
    static constexpr long long kChunkSweeps = 32;  // default of the ISING_KNOB_GRAPH_CHUNK knob
    static constexpr long long kChunkReplays = 4;  // chunks of sweeps left needed for a capture

    long long min_sweeps_left() const
    {
        long long m = LLONG_MAX;
        for (int64_t id : active_) {
            const Job& j = *jobs_.at(id);
            m = std::min(m, (long long)j.spec.n_sweeps - (epoch_ - j.join_epoch) / 2);
        }
        return m;
    }

    bool chunk_ready() const
    {
        if ((epoch_ & 1) || active_.empty() || chunk_sweeps_ == 0) return false;
        return min_sweeps_left() >= chunk_sweeps_ * (chunk_exec_ ? 1 : kChunkReplays);
    }

    int run_chunk()
    {
        cudaError_t e;
        if (!chunk_exec_) {
            e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture (batch)");
            cudaError_t le = cudaSuccess;
            for (long long k = 0; k < 2 * chunk_sweeps_ && le == cudaSuccess; ++k)
                le = launch_epoch(k, d_epoch_);
            cudaGraph_t graph = nullptr;
            e = cudaStreamEndCapture(stream_, &graph);
            if (le != cudaSuccess || e != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                return cuda_fail(le != cudaSuccess ? le : e, "batch graph capture");
            }
            e = cudaGraphInstantiate(&chunk_exec_, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) {
                chunk_exec_ = nullptr;
                return cuda_fail(e, "cudaGraphInstantiate (batch)");
            }
        }
        batch_epoch_set<<<1, 1, 0, stream_>>>(d_epoch_, epoch_);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaGraphLaunch(chunk_exec_, stream_);
        if (e != cudaSuccess) return cuda_fail(e, "batch graph launch");
        epoch_ += 2 * chunk_sweeps_;
        return ISING_OK;
    }

    // Drops the chunk graph (membership changed); it is destroyed once its launches are done.
    void drop_chunk()
    {
        if (!chunk_exec_) return;
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventRecord(ev, stream_) == cudaSuccess) {
            old_execs_.emplace_back(chunk_exec_, ev);
        } else {
            cudaStreamSynchronize(stream_);
            cudaGraphExecDestroy(chunk_exec_);
            if (ev) cudaEventDestroy(ev);
        }
        chunk_exec_ = nullptr;
    }

    void reap_chunks()
    {
        for (auto it = old_execs_.begin(); it != old_execs_.end();) {
            if (cudaEventQuery(it->second) == cudaSuccess) {
                cudaGraphExecDestroy(it->first);
                cudaEventDestroy(it->second);
                it = old_execs_.erase(it);
            } else {
                ++it;
            }
        }
        cudaGetLastError();  // cudaErrorNotReady from the queries
    }

    int retire()
    {
        for (auto it = active_.begin(); it != active_.end();) {
            Job& j = *jobs_[*it];
            if ((epoch_ - j.join_epoch) / 2 >= j.spec.n_sweeps) {
                int rc = finish_job(j);
                if (rc != ISING_OK) return rc;
                it = active_.erase(it);
                dirty_ = true;
            } else {
                ++it;
            }
        }
        return ISING_OK;
    }

    // Enqueues the result copies after the job's last half-sweep and frees its lattice.
    int finish_job(Job& j)
    {
        cudaError_t e = cudaSuccess;
        if (j.series_pairs) {
            const size_t sb = j.series_pairs * 2 * sizeof(long long);
            if (!j.h_series) e = pinned_get((void**)&j.h_series, sb);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(j.h_series, j.d_series, sb, cudaMemcpyDeviceToHost, stream_);
        }
        if (e == cudaSuccess && j.spec.keep_lattice) {
            const size_t full = (size_t)j.rows * 2 * j.lh;
            int8_t* stage = nullptr;
            if (!j.h_lattice) e = pinned_get((void**)&j.h_lattice, full);
            if (e == cudaSuccess) e = dev_alloc((void**)&stage, full);
            if (e == cudaSuccess) {
                if (j.spec.variant == ISING_VARIANT_MSC)
                    e = launch_msc_unpack((const u64*)j.c[0], (const u64*)j.c[1], stage, j.rows, 0,
                                          j.nw, sms_ * 8, stream_);
                else
                    e = launch_int8_merge((const int8_t*)j.c[0], (const int8_t*)j.c[1], stage,
                                          j.rows, 0, j.lh, j.pitch, j.ly, sms_ * 8, stream_);
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(j.h_lattice, stage, full, cudaMemcpyDeviceToHost, stream_);
            if (stage) cudaFreeAsync(stage, stream_);
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j.done_event, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(j.done_event, stream_);
        if (e != cudaSuccess) return cuda_fail(e, "job results");
        for (int c = 0; c < 2; ++c) {
            cudaFreeAsync(j.c[c], stream_);
            j.c[c] = nullptr;
        }
        if (j.d_series) {
            cudaFreeAsync(j.d_series, stream_);
            j.d_series = nullptr;
        }
        used_ -= (int64_t)j.device_bytes;
        j.state = ISING_JOB_FINISHING;
        finishing_.push_back(j.id);
        return ISING_OK;
    }

    // Records the end of the sweep (or graph chunk) just issued; the host stays at most about
    // kMaxAhead sweeps ahead of the device (see throttle_event), so a newly admitted job starts
    // soon after it joins.
    static constexpr long long kMaxAhead = 8;

    int throttle()
    {
        cudaEvent_t ev = nullptr;
        if (!free_events_.empty()) {
            ev = free_events_.back();
            free_events_.pop_back();
        } else {
            cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
            epoch_events_.push_back(ev);
        }
        cudaEventRecord(ev, stream_);
        inflight_.emplace_back(ev, epoch_);
        return ISING_OK;
    }

public:
    // The event to wait for before issuing more work (nullptr: not too far ahead).  Callers
    // wait without holding any lock the submitters need, then call throttle_done().
    cudaEvent_t throttle_event() const
    {
        return !inflight_.empty() && epoch_ - inflight_.front().second > 2 * kMaxAhead
                   ? inflight_.front().first
                   : nullptr;
    }

    void throttle_done()
    {
        free_events_.push_back(inflight_.front().first);
        inflight_.pop_front();
    }

    int wait_throttle()
    {
        while (cudaEvent_t ev = throttle_event()) {
            const cudaError_t e = cudaEventSynchronize(ev);
            if (e != cudaSuccess) return cuda_fail(e, "throttle");
            throttle_done();
        }
        return ISING_OK;
    }

private:

    void free_job(Job& j)
    {
        if (j.done_event) cudaEventDestroy(j.done_event);
        j.done_event = nullptr;
        for (int c = 0; c < 2; ++c)
            if (j.c[c]) cudaFreeAsync(j.c[c], stream_);
        if (j.d_series) cudaFreeAsync(j.d_series, stream_);
        if (j.h_series) pinned_put(j.h_series, j.series_pairs * 2 * sizeof(long long));
        if (j.h_lattice) pinned_put(j.h_lattice, (size_t)j.rows * 2 * j.lh);
        j.c[0] = j.c[1] = nullptr;
        j.d_series = nullptr;
        j.h_series = nullptr;
        j.h_lattice = nullptr;
    }

    cudaError_t dev_alloc(void** p, size_t bytes)
    {
        return cudaMallocFromPoolAsync(p, bytes, pool_, stream_);
    }

    // Pinned host buffers for results are reused across jobs (size classes of powers of two
    // from 4 KiB): page-locking memory for every finished job would stall the serving loop.
    static size_t pinned_class(size_t bytes)
    {
        size_t c = 4096;
        while (c < bytes) c <<= 1;
        return c;
    }

    cudaError_t pinned_get(void** p, size_t bytes)
    {
        const size_t c = pinned_class(bytes);
        auto it = pinned_free_.find(c);
        if (it != pinned_free_.end()) {
            *p = it->second;
            pinned_free_.erase(it);
            return cudaSuccess;
        }
        return cudaMallocHost(p, c);
    }

    void pinned_put(void* p, size_t bytes) { pinned_free_.emplace(pinned_class(bytes), p); }

    int device_;
    int64_t budget_;
    int64_t used_ = 0;
    int sms_ = 148;
    cudaStream_t stream_ = nullptr;
    cudaMemPool_t pool_ = nullptr;
    std::multimap<size_t, void*> pinned_free_;  // reusable pinned result buffers by size class
    long long epoch_ = 0;
    int64_t last_id_ = 0;
    int band_cap_ = kBandCap;
    long long items_per_slot_ = kItemsPerSlot;
    long long* d_epoch_ = nullptr;       // device epoch counter of replayed graph chunks
    cudaGraphExec_t chunk_exec_ = nullptr;
    std::vector<std::pair<cudaGraphExec_t, cudaEvent_t>> old_execs_;
    long long chunk_sweeps_ = kChunkSweeps;  // 0: no graph chunks
    std::map<int64_t, std::unique_ptr<Job>> jobs_;
    std::deque<int64_t> pending_;
    std::vector<int64_t> active_;
    std::vector<int64_t> finishing_;
    bool dirty_ = false;
    BatchLattice* d_lats_ = nullptr;
    BatchItem* d_items_ = nullptr;
    size_t lats_cap_ = 0, items_cap_ = 0;
    std::vector<std::pair<KernelClass, std::pair<int, int>>> classes_;  // msc work items
    std::vector<std::pair<KernelClass, std::vector<Int8Launch>>> int8_launches_;
    std::vector<cudaEvent_t> epoch_events_, free_events_;
    std::map<const void*, int> occupancy_;
    std::deque<std::pair<cudaEvent_t, long long>> inflight_;  // (event, epoch recorded at)
};

}  // namespace ising

using namespace ising;

// ------------------------------------------------------------------------------- batch API ---
struct ising_batch {
    std::unique_ptr<Engine> eng;
};

extern "C" {

int ising_batch_create(int device, int64_t memory_budget, ising_batch** out)
{
    if (!out) return fail(ISING_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (memory_budget <= 0) return fail(ISING_ERR_INVALID, "memory budget must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(ISING_ERR_INVALID, "device %d not available", device);
    }
    auto b = new ising_batch();
    b->eng.reset(new Engine(device, memory_budget));
    int rc = b->eng->init();
    if (rc != ISING_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return ISING_OK;
}

int ising_batch_add(ising_batch* b, const ising_job* job, int64_t* id)
{
    if (!b || !job || !id) return fail(ISING_ERR_INVALID, "null argument");
    return b->eng->submit(*job, id);
}

int ising_batch_run(ising_batch* b, int64_t max_epochs, int64_t* epochs_run)
{
    if (!b) return fail(ISING_ERR_INVALID, "null batch");
    int64_t n = 0;  // half-sweep epochs issued (a replayed chunk issues many)
    while (b->eng->has_work() && (max_epochs <= 0 || n < max_epochs)) {
        const size_t before = b->eng->active_count() + b->eng->pending_count();
        const long long e0 = b->eng->epoch();
        int rc = b->eng->step(max_epochs > 0 ? max_epochs - n : 0);
        if (rc == ISING_OK) rc = b->eng->wait_throttle();
        if (rc != ISING_OK) return rc;
        n += b->eng->epoch() - e0;
        if (b->eng->active_count() == 0 && b->eng->pending_count() > 0 &&
            b->eng->pending_count() == before)
            return fail(ISING_ERR_NOMEM, "pending jobs do not fit the memory budget");
    }
    if (epochs_run) *epochs_run = n;
    return b->eng->wait_finishing();
}

int ising_batch_status(ising_batch* b, int64_t id, int* state, int64_t* sweeps_done)
{
    if (!b || !state) return fail(ISING_ERR_INVALID, "null argument");
    b->eng->poll();
    Job* j = b->eng->find(id);
    if (!j) return fail(ISING_ERR_INVALID, "unknown job %lld", (long long)id);
    *state = j->state;
    if (sweeps_done) {
        long long s = 0;
        if (j->state == ISING_JOB_DONE || j->state == ISING_JOB_FINISHING) s = j->spec.n_sweeps;
        else if (j->state == ISING_JOB_ACTIVE) s = (b->eng->epoch() - j->join_epoch) / 2;
        *sweeps_done = s;
    }
    return ISING_OK;
}

int ising_batch_result(ising_batch* b, int64_t id, int64_t* series_out, int8_t* lattice_out)
{
    if (!b) return fail(ISING_ERR_INVALID, "null batch");
    b->eng->poll();
    return b->eng->result(id, series_out, lattice_out, nullptr);
}

int ising_batch_release(ising_batch* b, int64_t id)
{
    if (!b) return fail(ISING_ERR_INVALID, "null batch");
    return b->eng->release(id);
}

int ising_batch_set_knob(ising_batch* b, int knob, int value)
{
    if (!b) return fail(ISING_ERR_INVALID, "null batch");
    return b->eng->set_knob(knob, value);
}

int ising_batch_get_knob(ising_batch* b, int knob, int* value)
{
    if (!b || !value) return fail(ISING_ERR_INVALID, "null argument");
    return b->eng->get_knob(knob, value);
}

int ising_batch_destroy(ising_batch* b)
{
    delete b;
    return ISING_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------- serving API ---
struct ising_server {
    std::unique_ptr<Engine> eng;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    int error = ISING_OK;
    std::string error_msg;
};

static void server_loop(ising_server* s)
{
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        s->cv_work.wait(lk, [s] { return s->stop || s->eng->busy(); });
        if (s->stop && !s->eng->busy()) break;
        if (s->eng->has_work()) {
            // one sweep (two half-sweeps) per turn, then let submitters in
            for (int k = 0; k < 2 && s->error == ISING_OK; ++k) {
                const int rc = s->eng->step();
                if (rc != ISING_OK) {
                    s->error = rc;
                    s->error_msg = g_last_error;
                }
            }
            // bound the run-ahead without holding the lock submitters and waiters need
            while (cudaEvent_t ev = s->eng->throttle_event()) {
                lk.unlock();
                const cudaError_t e = cudaEventSynchronize(ev);
                lk.lock();
                if (e != cudaSuccess) {
                    s->error = cuda_fail(e, "throttle");
                    s->error_msg = g_last_error;
                    break;
                }
                s->eng->throttle_done();
            }
        } else {
            lk.unlock();
            cudaStreamSynchronize(s->eng->stream());
            lk.lock();
        }
        if (s->eng->poll() > 0) s->cv_done.notify_all();
        if (s->error != ISING_OK) {
            s->cv_done.notify_all();
            break;
        }
        // brief release so submitters and waiters can take the lock
        lk.unlock();
        std::this_thread::yield();
        lk.lock();
    }
}

extern "C" {

int ising_server_create(int device, int64_t memory_budget, ising_server** out)
{
    if (!out) return fail(ISING_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (memory_budget <= 0) return fail(ISING_ERR_INVALID, "memory budget must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return fail(ISING_ERR_INVALID, "device %d not available", device);
    }
    auto s = new ising_server();
    s->eng.reset(new Engine(device, memory_budget));
    int rc = s->eng->init();
    if (rc != ISING_OK) {
        delete s;
        return rc;
    }
    s->worker = std::thread([s, device] {
        cudaSetDevice(device);
        server_loop(s);
    });
    *out = s;
    return ISING_OK;
}

int ising_server_submit(ising_server* s, const ising_job* job, int64_t* id)
{
    if (!s || !job || !id) return fail(ISING_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error != ISING_OK) return fail(s->error, "server stopped: %s", s->error_msg.c_str());
    int rc = s->eng->submit(*job, id);
    if (rc == ISING_OK) s->cv_work.notify_one();
    return rc;
}

int ising_server_wait(ising_server* s, int64_t id, double timeout_s, int* state)
{
    if (!s || !state) return fail(ISING_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    Job* j = s->eng->find(id);
    if (!j) return fail(ISING_ERR_INVALID, "unknown job %lld", (long long)id);
    auto done = [&] { return s->error != ISING_OK || s->eng->find(id)->state == ISING_JOB_DONE; };
    if (timeout_s < 0) s->cv_done.wait(lk, done);
    else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    *state = s->eng->find(id)->state;
    if (s->error != ISING_OK) return fail(s->error, "server stopped: %s", s->error_msg.c_str());
    return ISING_OK;
}

int ising_server_result(ising_server* s, int64_t id, int64_t* series_out, int8_t* lattice_out,
                        double* latency_s)
{
    if (!s) return fail(ISING_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    return s->eng->result(id, series_out, lattice_out, latency_s);
}

int ising_server_release(ising_server* s, int64_t id)
{
    if (!s) return fail(ISING_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    return s->eng->release(id);
}

int ising_server_status(ising_server* s, int64_t* pending, int64_t* active, int64_t* used_bytes,
                        int64_t* epoch)
{
    if (!s) return fail(ISING_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (pending) *pending = (int64_t)s->eng->pending_count();
    if (active) *active = (int64_t)s->eng->active_count();
    if (used_bytes) *used_bytes = s->eng->used_bytes();
    if (epoch) *epoch = s->eng->epoch();
    return ISING_OK;
}

int ising_server_set_knob(ising_server* s, int knob, int value)
{
    if (!s) return fail(ISING_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    return s->eng->set_knob(knob, value);
}

int ising_server_destroy(ising_server* s)
{
    if (!s) return ISING_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    delete s;
    return ISING_OK;
}

}  // extern "C"
