// Internal declarations shared by the C-ABI translation units (not part of the public ABI).
#pragma once

#include <string>
#include <vector>

#include "common.cuh"
#include "ising_b200.h"

// A simulation handle: one lattice, its two colour arrays on one device, one stream.
struct ising_sim {
    int device = 0;
    int ndim = 2;
    int variant = ISING_VARIANT_INT8;
    int algorithm = ISING_METROPOLIS;
    int64_t shape[3] = {0, 0, 0};
    long long rows = 0;  // prod(shape[:-1])
    int lh = 0;          // Lx / 2
    int ly = 0;          // rows per plane
    int lz = 1;          // planes (1 in 2D)
    int nw = 0;          // packed words per row (msc)
    int pitch = 0;       // int8: bytes between rows on the device (lh rounded up to 16)
    int vw = 16;         // int8: chunk width of the kernels
    int band = 0;        // int8: rows per band of the band schedule (0: the launcher's default)
    uint64_t seed = 0;
    uint32_t table[7] = {0, 0, 0, 0, 0, 0, 0};
    int table_n = 5;
    int rule = 0;        // ising::Rule chosen from the table
    void* c[2] = {nullptr, nullptr};
    size_t colour_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream_handle = nullptr;
    unsigned long long* d_acc = nullptr;  // [0,1] observables, [2,3] msc call statistics
    long long* d_series = nullptr;        // (M, E) pairs of one ising_sweep call
    long long* h_series = nullptr;        // pinned copy of d_series
    int64_t series_cap = 0;               // pairs
    int sm_count = 148;
    int max_blocks = 148 * 8;           // grid cap: sm_count * blocks_per_sm
    // Launch knobs (ising_set_knob); every value gives identical results.
    int blocks_per_sm = 8;
    int msc_waves = 1;                  // msc: warp ranges per resident warp
    int msc_kernel = 0;                 // msc: schedule (ISING_KNOB_MSC_KERNEL)
    int64_t graph_chunk = 32;           // sweeps per captured graph of an unmeasured run
    // Captured chunks of `sweeps` sweeps (one measurement at the end when `measured`), replayed
    // with the sweep counter and series slot in d_acc[6], d_acc[7].
    struct Graph {
        int64_t sweeps;
        bool measured;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    int schedule = ISING_SCHEDULE_AUTO;
    int mute_band = -1;                 // test hook of the persistent schedule
    unsigned int* d_flags = nullptr;    // persistent schedule: per-band progress + error word
    int* d_label = nullptr;             // cluster updates: a label per site, error word, masks
    int cluster_tile = 0;               // cluster updates: positions per tile (0: automatic)
    void* tb_scratch[2] = {nullptr, nullptr};  // temporal schedule: second pair of colour arrays
    int test_label_cycle = 0;           // test hook: a cycle in the cluster labels
    bool pending_err = false;           // a persistent run's error word not yet read
};

namespace ising {

extern thread_local std::string g_last_error;
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
int device_sm_count(int device);
int select_rule(int variant, int algorithm, int ndim, const u32* table);

int ensure_series(ising_sim* h, int64_t pairs);
int half_sweep(ising_sim* h, int color, u32 t, unsigned long long* meas,
               unsigned long long* stats, const unsigned long long* ctl = nullptr);
void clear_graphs(ising_sim* h);
int observe(ising_sim* h, unsigned long long* acc);
bool temporal_ok(const ising_sim* h);
// Stream-ordered device memory from the per-device pool that single-lattice handles share.
cudaError_t pool_alloc(int device, void** p, size_t bytes, cudaStream_t st);
// The temporal schedule's second pair of colour arrays (allocated once, outside any capture).
int temporal_scratch(ising_sim* h);
// `count` temporal launches of kTbSteps / 2 sweeps each from sweep t; the lattice ends in the
// handle's arrays.
cudaError_t launch_temporal_run(const ising_sim* h, u32 t, int64_t count,
                                const unsigned long long* ctl);
int temporal_sweeps();  // sweeps per temporal launch
int run_persistent_int8(ising_sim* h, uint64_t t0, int64_t n_sweeps, int64_t measure_every,
                        unsigned long long* series, unsigned int* flags, int* err, int mute_band);
int selftest_bounded_wait(int device, int* timed_out);

// kernel launchers
int int8_chunk_width(int lh);
int int8_default_band(long long rows, int ly, int cpr, int sm_count);
unsigned int8_band_geometry(Int8Half& p, int max_blocks, int sm_count);
cudaError_t launch_int8_half(int ndim, int rule, const Int8Half& p, int max_blocks, int sm_count,
                             cudaStream_t st);
// kernel: 0 = automatic (the strip schedule where the rows hold whole 32-word strips), 1 = the
// range schedule, 2..7 = the strip schedule with (Philox blocks per word at intake, resident
// blocks the registers are bounded for) = (4, 2), (4, 3), (4, 4), (3, 2), (3, 3), (3, 4).
cudaError_t launch_msc_half(bool update, const MscHalf& p, int max_blocks, int sm_count,
                            int waves, cudaStream_t st, int kernel = 0);
cudaError_t launch_int8_split(const int8_t* full, int8_t* c0, int8_t* c1, long long rows,
                              long long row0, int lh, int pitch, int ly, int max_blocks,
                              cudaStream_t st);
cudaError_t launch_int8_merge(const int8_t* c0, const int8_t* c1, int8_t* full, long long rows,
                              long long row0, int lh, int pitch, int ly, int max_blocks,
                              cudaStream_t st);
cudaError_t launch_msc_pack(const int8_t* full, u64* w0, u64* w1, int rows, int row0, int nw,
                            int max_blocks, cudaStream_t st);
cudaError_t launch_msc_unpack(const u64* w0, const u64* w1, int8_t* full, int rows, int row0,
                              int nw, int max_blocks, cudaStream_t st);
cudaError_t launch_philox_start(void* c0, void* c1, long long rows, int lh, int pitch, int packed,
                                u32 k0, u32 k1, int max_blocks, cudaStream_t st);
cudaError_t launch_philox_probe(u32* out, int blocks, int threads, int calls, u32 k0, u32 k1,
                                cudaStream_t st);
cudaError_t launch_philox_range(u32* out, long long n, u32 q0, u32 c1, u32 c2, u32 c3, u32 k0,
                                u32 k1, int max_blocks, cudaStream_t st);

}  // namespace ising
