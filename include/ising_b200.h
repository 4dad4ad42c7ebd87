/*
 * ising_b200.h — C ABI of the B200 (sm_100a) backend for pyising's sweep hot path.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status (ISING_OK = 0).  Every call
 * that fails leaves a message readable with ising_last_error() (thread-local).  A handle
 * belongs to one host thread at a time and issues all its work on one CUDA stream; the library
 * owns all device memory it allocates and never keeps a host pointer after a call returns.
 *
 * The reference interface each entry point replaces is cited as file:line inside the pyising
 * project (github.com/walidhemati/pyising).  The Python host layer (pyising_b200.backend)
 * binds these through ctypes.
 */
#ifndef ISING_B200_H
#define ISING_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
#define ISING_OK 0
#define ISING_ERR_INVALID 1   /* bad argument: shape, variant, algorithm, size, null pointer */
#define ISING_ERR_CUDA 2      /* a CUDA runtime call failed; message has the CUDA error */
#define ISING_ERR_NOMEM 3     /* device allocation failed or over the memory budget */
#define ISING_ERR_TIMEOUT 4   /* a bounded device-side wait expired (kernel returned early) */
#define ISING_ERR_STATE 5     /* call not valid in the object's current state */

/* ---- enums --------------------------------------------------------------------------- */
#define ISING_VARIANT_INT8 0  /* compressed checkerboard, one int8 per spin (2D/3D) */
#define ISING_VARIANT_MSC 1   /* multi-spin coding, 64 spins per uint64 (2D Metropolis) */
#define ISING_METROPOLIS 0
#define ISING_HEATBATH 1

typedef struct ising_sim ising_sim;

/* Message of the last failed call on this thread ("" if none).
 * Replaces: exceptions raised by pyising (src/pyising/lattice.py:25-34,
 * src/pyising/backends/base.py:54-57, src/pyising/backends/__init__.py:37-38,60-61). */
const char* ising_last_error(void);

/* Library ABI version (major * 10000 + minor * 100 + patch). */
int ising_version(void);

/* Number of visible CUDA devices.
 * Replaces: pyising.backends._gpu.cuda_available (src/pyising/backends/_gpu.py:39-45). */
int ising_device_count(int* n);

/* "<name> sm_<major><minor> <n> SMs" of a device (the autotuner's cache key).  No counterpart
 * in the reference. */
int ising_device_name(int device, char* buf, int buflen);

/* Create a simulation: ndim 2 or 3; shape is (Ly, Lx) or (Lz, Ly, Lx); every extent even and
 * >= 2; Lx % 8 == 0 (int8) or Lx % 128 == 0 (msc, 2D Metropolis only).  Device arrays are
 * allocated but not initialised: call ising_set_lattice / ising_upload / ising_fill_cold.
 * Replaces: IsingSimulation.__init__ + _setup (src/pyising/backends/base.py:44-73;
 * src/pyising/backends/cupy_backend.py:53-66,114-123) and check_shape
 * (src/pyising/lattice.py:25-34). */
int ising_create(int ndim, const int64_t* shape, int variant, int algorithm, uint64_t seed,
                 int device, ising_sim** out);

/* Free the device arrays and the handle (NULL is accepted). */
int ising_destroy(ising_sim* h);

/* Use an existing CUDA stream (cudaStream_t passed as void*; NULL = the handle's own stream).
 * The caller keeps the stream alive while the handle uses it. */
int ising_set_stream(ising_sim* h, void* stream);

/* Acceptance table, uint32[2*ndim+1] indexed by (X + 2 ndim) / 2 (threshold_table,
 * src/pyising/lattice.py:128-142).  The table is copied.
 * Replaces: IsingSimulation.set_beta/_upload_table (src/pyising/backends/base.py:79-83,
 * src/pyising/backends/cupy_backend.py:74-75). */
int ising_set_table(ising_sim* h, const uint32_t* table, int n);

/* Change the Philox key (seed, 64 bit). */
int ising_set_seed(ising_sim* h, uint64_t seed);

/* Load / read a full int8 lattice (+1/-1, C order, prod(shape) bytes) from / into host memory.
 * The colour split (and bit packing for msc) runs on the device.
 * Replaces: set_lattice / get_lattice (src/pyising/backends/numpy_backend.py:46-51,126-131;
 * src/pyising/backends/cupy_backend.py:77-82,146-152) with to/from_compressed and
 * pack/unpack_bits (src/pyising/lattice.py:50-90). */
int ising_set_lattice(ising_sim* h, const int8_t* full);
int ising_get_lattice(ising_sim* h, int8_t* full);

/* Copy the two colour arrays in their device layout: int8 (rows, Lx/2) or packed uint64
 * (rows, Lx/128) — the same arrays as to_compressed / pack_bits produce. */
int ising_upload(ising_sim* h, const void* c0, const void* c1);
int ising_download(ising_sim* h, void* c0, void* c1);

/* All spins +1.  Replaces: _fill_cold (src/pyising/backends/base.py:119-120). */
int ising_fill_cold(ising_sim* h);

/* Run n_sweeps full sweeps (colour 0 then colour 1) with sweep counters t0, t0+1, ...
 * If measure_every > 0, (M, E) as exact int64 after every measure_every-th sweep are written
 * to series_out[2*i], series_out[2*i+1] (host memory, n_sweeps / measure_every pairs) and the
 * call blocks until they are there; otherwise the call only enqueues the work.
 * Replaces: IsingSimulation.sweep (src/pyising/backends/base.py:85-90) with _half_sweep
 * (src/pyising/backends/cupy_backend.py:68-72,125-135) and the measurement loop of
 * pyising.observables.sample (src/pyising/observables.py:61-74). */
int ising_sweep(ising_sim* h, uint64_t t0, int64_t n_sweeps, int64_t measure_every,
                int64_t* series_out);

/* One colour's half-sweep with sweep counter t (asynchronous).
 * Replaces: the _half_sweep hook (src/pyising/backends/base.py:101-103;
 * src/pyising/backends/cupy_backend.py:68-72,125-135). */
int ising_half_sweep(ising_sim* h, int color, uint64_t t);

/* How ising_sweep issues its half-sweeps (no counterpart in the reference, which launches one
 * kernel per half-sweep from Python):
 *   ISING_SCHEDULE_AUTO       graphs for whole chunks of sweeps, launches for the rest (the
 *                             temporal tiles below for eligible lattices up to 1024^2);
 *   ISING_SCHEDULE_LAUNCHES   one kernel launch per half-sweep;
 *   ISING_SCHEDULE_GRAPHS     replayed CUDA graphs of whole chunks of sweeps;
 *   ISING_SCHEDULE_PERSISTENT one cooperative launch for all sweeps (2D int8; others fall back):
 *                             bands of rows wait only for their neighbours, every wait bounded;
 *   ISING_SCHEDULE_TEMPORAL   graphs whose launches each run two unmeasured sweeps on
 *                             shared-memory tiles with recomputed halos (small 2D int8
 *                             lattices with rows a multiple of 16 bytes; others fall back).
 * All schedules give identical results.  test_mute_band >= 0 makes that band of a persistent
 * run stop publishing its progress, so its neighbours' bounded waits expire: the sweep then
 * reports ISING_ERR_TIMEOUT (the lattice is no longer valid); pass -1 otherwise. */
#define ISING_SCHEDULE_AUTO 0
#define ISING_SCHEDULE_LAUNCHES 1
#define ISING_SCHEDULE_GRAPHS 2
#define ISING_SCHEDULE_PERSISTENT 3
#define ISING_SCHEDULE_TEMPORAL 4
int ising_set_schedule(ising_sim* h, int schedule, int test_mute_band);

/* Launch knobs of a handle, picked by the autotuner (pyising_b200.autotune) or by hand.  Every
 * value gives identical spins and observables; only the speed changes.  Setting a knob drops
 * the handle's captured graphs.  No counterpart in the reference, whose kernels have a fixed
 * launch shape (src/pyising/backends/cupy_backend.py:68-72,129-135).
 *   ISING_KNOB_BAND           int8: rows of one plane a thread walks, reusing the opposite
 *                             colour's rows (halo depth); 0 = occupancy-based default
 *   ISING_KNOB_CHUNK_WIDTH    int8: bytes (4 sites each per 32-bit word) per thread: 16, 8, 4
 *   ISING_KNOB_BLOCKS_PER_SM  grid cap in blocks of 256 threads per SM (default 8)
 *   ISING_KNOB_MSC_WAVES      msc: warp ranges per resident warp (default 1)
 *   ISING_KNOB_GRAPH_CHUNK    sweeps per captured graph of an unmeasured run (default 32) */
#define ISING_KNOB_BAND 1
#define ISING_KNOB_CHUNK_WIDTH 2
#define ISING_KNOB_BLOCKS_PER_SM 3
#define ISING_KNOB_MSC_WAVES 4
#define ISING_KNOB_GRAPH_CHUNK 5
/* Cluster updates: sites per colour in a tile of the shared-memory union-find (0 = automatic,
 * 1 = no tiles: one union-find in global memory, else 32..6144); the labels are the same for
 * every value. */
#define ISING_KNOB_CLUSTER_TILE 7
/* msc schedule: 0 = automatic (strips where each row holds a multiple of 32 words, ranges
 * elsewhere), 1 = word ranges per warp, 2..7 = 32-word column strips walked down a band of rows two
 * rows per step, with (Philox blocks per word before the work stack, resident blocks of 256
 * threads the registers are bounded for) = (4, 2), (4, 3), (4, 4), (3, 2), (3, 3), (3, 4). */
#define ISING_KNOB_MSC_KERNEL 9
/* Test hook of the bounded union-find loops (0 = off): 1 makes every cluster labeling write a
 * two-site cycle into the labels (sites 0 and S) after the unions, so the root walks that follow
 * run out of their step budgets and the call returns ISING_ERR_TIMEOUT, with the context intact.
 * Never set outside tests. */
#define ISING_KNOB_TEST_LABEL_CYCLE 8
/* Batch and server knobs (ising_batch_set_knob, ising_server_set_knob): ISING_KNOB_BAND is the
 * longest band a kernel class may use (default 8); ISING_KNOB_ITEMS_PER_SLOT the work items per
 * resident block a launch aims at (default 6; smaller items balance better, larger ones cost
 * less per item); ISING_KNOB_GRAPH_CHUNK the sweeps of a stable batch replayed from one
 * captured graph (default 32, 0 = every epoch launched directly). */
#define ISING_KNOB_ITEMS_PER_SLOT 6
int ising_set_knob(ising_sim* h, int knob, int value);
int ising_get_knob(ising_sim* h, int knob, int* value);

/* n_sweeps unmeasured sweeps from sweep counter t0, timed on the device with CUDA events on the
 * handle's stream; blocks until done and returns the elapsed milliseconds in *ms.  Used by the
 * autotuner; the sweeps are real (the lattice advances).  No counterpart in the reference. */
int ising_time_sweeps(ising_sim* h, uint64_t t0, int64_t n_sweeps, float* ms);

/* n_steps Swendsen-Wang cluster updates of an int8 lattice (2D/3D, fewer than 2^31 sites),
 * steps step0 .. step0+n-1, random numbers keyed by `seed`: bonds between aligned neighbours
 * are active when a Philox uniform is below p_bond (the integer threshold of
 * p = 1 - exp(-2 beta)), the connected clusters are found on the device by a lock-free
 * union-find, and each cluster flips with probability 1/2.  Labels take 4 bytes per site,
 * allocated on the first call.  With series_out non-null, the exact (M, E) after every step
 * lands in series_out[2k], series_out[2k+1] (the call then blocks until done).
 * ISING_ERR_TIMEOUT if a bounded union-find loop gave up.
 * Replaces: the CPU Wolff sampler used for equilibrated starts and Binder scans
 * (src/pyising/cluster.py:32-104; src/pyising/validate.py:45-50,127-150). */
int ising_cluster_sweep(ising_sim* h, uint64_t step0, int64_t n_steps, uint64_t seed,
                        uint32_t p_bond, int64_t* series_out);

/* One labeling of step `step` without the flips (diagnostics and tests): labels_out (2*S
 * int32, S = sites per colour; site g = c*S + row*Lx/2 + j) gets each site's cluster root,
 * bonds_out (S bytes) the active bonds of each colour-0 site (bit k: same-index colour-1 site,
 * the other horizontal one, y+1, y-1, z+1, z-1).  No counterpart in the reference. */
int ising_cluster_labels(ising_sim* h, uint64_t step, uint64_t seed, uint32_t p_bond,
                         int32_t* labels_out, uint8_t* bonds_out);

/* Exact magnetisation M = sum s and energy E = -sum_<ij> s_i s_j (blocks until done).
 * Replaces: observables / magnetization / energy (src/pyising/backends/base.py:125-135;
 * src/pyising/backends/observables_torch.py:46-111). */
int ising_observables(ising_sim* h, int64_t* m, int64_t* e);

/* Block until the handle's queued work is done.
 * Replaces: synchronize (src/pyising/backends/cupy_backend.py:86-87). */
int ising_sync(ising_sim* h);

/* Bytes of device memory the handle holds (spin arrays and buffers).
 * Replaces: device_bytes (src/pyising/backends/base.py:137-139). */
int ising_device_bytes(ising_sim* h, int64_t* bytes);

/* Mean Philox calls per word of the msc kernel over n_sweeps sweeps (also advances the
 * lattice: t0, t0+1, ...); *mean and *warp_max as in the reference's diagnostic.
 * Replaces: CupyMultiSpin.philox_calls_per_word (src/pyising/backends/cupy_backend.py:137-144).
 */
int ising_msc_calls_per_word(ising_sim* h, uint64_t t0, int64_t n_sweeps, double* mean,
                             double* warp_max);

/* Sweeps on caller-owned device arrays that allocate nothing.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc (device memory owned by a pool they do not
 * control, or a loop that must not take cudaMalloc/cudaFree's implicit synchronisation).
 * c0, c1: the two colour arrays in device memory of the current device, laid out as
 * ising_upload expects (int8 (rows, Lx/2): rows * Lx/2 bytes each, or packed uint64
 * (rows, Lx/128): rows * Lx/16 bytes each), 16-byte aligned, updated in place.  Each must lie
 * inside one device allocation with at least that many bytes from the pointer to the
 * allocation's end; host memory, another GPU's memory or a shorter buffer is rejected with
 * ISING_ERR_INVALID before any work is issued.  Arguments
 * otherwise as ising_create + ising_set_table + ising_sweep; the work runs on `stream`
 * (cudaStream_t, NULL = default stream) on the calling thread's current device.
 * Measured (M, E) sums live in a fixed 64 KiB device array inside the library (held by every
 * GPU that loads it until exit): at most 4096 measurements (n_sweeps / measure_every) per call,
 * more is rejected with ISING_ERR_INVALID.  The first call on a device looks the array's address
 * up (cudaGetSymbolAddress), and so does the first call after the device's context changed
 * (cudaDeviceReset); make that first call before any stream capture.  Every call shares
 * the array, so calls that overlap on the GPU (other streams, other threads) race; the
 * measured part is cleared at the start of each call.  Blocks until series_out is written when
 * measure_every > 0, otherwise only enqueues the work. */
int ising_sweep_static(int ndim, const int64_t* shape, int variant, int algorithm, uint64_t seed,
                       const uint32_t* table, int table_n, void* c0, void* c1, uint64_t t0,
                       int64_t n_sweeps, int64_t measure_every, int64_t* series_out,
                       void* stream);

/* Device-side seeded start (not in the reference, whose hot start is NumPy's PCG64 and stays
 * the default of the Python layer): compressed site n of colour c is +1 iff bit n % 32 of word
 * (n / 32) % 4 of Philox4x32-10((n / 128, 0, c, 0xFFFFFFFF), start_seed) is set.  The same
 * spins for the int8 and the packed layout; no host work, so multi-GB starts cost a kernel. */
int ising_fill_philox(ising_sim* h, uint64_t start_seed);

/* ---- batched ensembles and serving ----------------------------------------------------- */
/* No counterpart in the reference (which runs one lattice per launch): many independent
 * lattices of uneven size, dimension, variant and temperature advance together, one grouped
 * launch per half-sweep over a (lattice, tile) work list; each lattice stays bit-identical to
 * running it alone (the random numbers depend only on site, sweep, colour and seed). */

#define ISING_INIT_COLD 0     /* all +1 */
#define ISING_INIT_PHILOX 1   /* the device seeded start of ising_fill_philox, seed = job seed */
#define ISING_INIT_LATTICE 2  /* a full int8 lattice, copied when the job is added */

#define ISING_JOB_PENDING 0   /* waiting for memory (admission at the next sweep boundary) */
#define ISING_JOB_ACTIVE 1
#define ISING_JOB_FINISHING 2 /* last sweep issued, results on their way to the host */
#define ISING_JOB_DONE 3

typedef struct ising_job {
    int ndim;                 /* 2 or 3 */
    int64_t shape[3];         /* (Ly, Lx) or (Lz, Ly, Lx) */
    int variant;              /* ISING_VARIANT_* */
    int algorithm;            /* ISING_METROPOLIS / ISING_HEATBATH */
    uint64_t seed;            /* Philox key */
    uint32_t table[7];        /* threshold_table(beta, ndim, algorithm) */
    int table_n;              /* 2 * ndim + 1 */
    uint64_t t0;              /* sweep counter of the first sweep */
    int64_t n_sweeps;
    int64_t measure_every;    /* (M, E) after every measure_every-th sweep; 0 = none */
    int init;                 /* ISING_INIT_* */
    const int8_t* lattice;    /* ISING_INIT_LATTICE: full lattice, C order (copied) */
    int keep_lattice;         /* non-zero: copy the final lattice back for *_result */
} ising_job;

typedef struct ising_batch ising_batch;

/* A batch on `device` whose lattices and series may hold at most memory_budget device bytes.
 * Replaces running lattices one at a time through create()/sweep() (bench/run.py:121-142). */
int ising_batch_create(int device, int64_t memory_budget, ising_batch** out);
/* Queue a job (validated like ising_create); it joins at the next sweep boundary with room. */
int ising_batch_add(ising_batch* b, const ising_job* job, int64_t* id);
/* Advance every job until all are done (max_epochs <= 0) or for max_epochs half-sweeps. */
int ising_batch_run(ising_batch* b, int64_t max_epochs, int64_t* epochs_run);
int ising_batch_status(ising_batch* b, int64_t id, int* state, int64_t* sweeps_done);
/* Results of a done job: series (n_sweeps / measure_every pairs of (M, E)), final lattice. */
int ising_batch_result(ising_batch* b, int64_t id, int64_t* series_out, int8_t* lattice_out);
int ising_batch_release(ising_batch* b, int64_t id);
/* Launch knobs of a batch (ISING_KNOB_BAND cap, ISING_KNOB_ITEMS_PER_SLOT), applied at the next
 * rebuild of its work list; identical results for every value.  No counterpart in the reference
 * (it has no batch). */
int ising_batch_set_knob(ising_batch* b, int knob, int value);
int ising_batch_get_knob(ising_batch* b, int knob, int* value);
int ising_batch_destroy(ising_batch* b);

typedef struct ising_server ising_server;

/* A serving loop on its own host thread: submitted jobs are admitted by the memory budget at
 * sweep boundaries while others run (continuous batching), results stay on the host until
 * released.  Submit, wait, result, status and release are thread-safe. */
int ising_server_create(int device, int64_t memory_budget, ising_server** out);
int ising_server_submit(ising_server* s, const ising_job* job, int64_t* id);
/* Wait up to timeout_s seconds (< 0: no limit) for the job; *state is its ISING_JOB_* state. */
int ising_server_wait(ising_server* s, int64_t id, double timeout_s, int* state);
/* Results of a done job and its submit-to-done latency in seconds. */
int ising_server_result(ising_server* s, int64_t id, int64_t* series_out, int8_t* lattice_out,
                        double* latency_s);
int ising_server_release(ising_server* s, int64_t id);
int ising_server_status(ising_server* s, int64_t* pending, int64_t* active, int64_t* used_bytes,
                        int64_t* epoch);
/* Finish the jobs already submitted, stop the thread and free everything. */
/* The batch knobs of a server's engine (see ising_batch_set_knob). */
int ising_server_set_knob(ising_server* s, int knob, int value);
int ising_server_destroy(ising_server* s);

/* ---- slab decomposition of one lattice over several devices ---------------------------- */
/* No counterpart in the reference (one lattice lives on one device there).  A slab handle owns
 * rows [begin, begin + count) of the first axis of the whole lattice `shape` (rows y in 2D,
 * planes z in 3D) plus one halo row (2D) or plane (3D) of each colour on each side.  A
 * half-sweep of colour c reads the opposite colour's halos, so before it the caller copies the
 * opposite colour's edge rows of the neighbouring slabs into them (periodic along the axis), by
 * NCCL, a peer copy or a local copy; the half-sweep itself never wraps along the slab axis.
 * Random numbers use global site indices, so the slabs together give exactly the results of one
 * ising_sim holding the whole lattice, and the lattice's (M, E) is the sum over the slabs.
 * Per-slab calls mirror ising_create / ising_set_table / ising_upload / ising_download /
 * ising_fill_cold / ising_fill_philox / ising_half_sweep / ising_observables / ising_sync; host
 * colour arrays hold the owned rows only ((rows, Lx/2) int8 or (rows, Lx/128) uint64). */
typedef struct ising_slab ising_slab;

#define ISING_SLAB_HALO_LOW 0   /* halo before owned row 0 (receives the previous slab's edge) */
#define ISING_SLAB_HALO_HIGH 1  /* halo after the last owned row (the next slab's edge) */
#define ISING_SLAB_EDGE_LOW 2   /* first owned row or plane (sent to the previous slab) */
#define ISING_SLAB_EDGE_HIGH 3  /* last owned row or plane (sent to the next slab) */

int ising_slab_create(int ndim, const int64_t* shape, int variant, int algorithm, uint64_t seed,
                      int64_t begin, int64_t count, int device, ising_slab** out);
int ising_slab_destroy(ising_slab* s);
int ising_slab_set_stream(ising_slab* s, void* stream);
int ising_slab_set_table(ising_slab* s, const uint32_t* table, int n);
int ising_slab_upload(ising_slab* s, const void* c0, const void* c1);
int ising_slab_download(ising_slab* s, void* c0, void* c1);
int ising_slab_fill_cold(ising_slab* s);
int ising_slab_fill_philox(ising_slab* s, uint64_t start_seed);
/* Device address and byte count of one halo or edge region of colour `color` (`which`: one of
 * ISING_SLAB_HALO_* / ISING_SLAB_EDGE_*); the region is contiguous and the same size on every
 * slab of a lattice. */
int ising_slab_halo(ising_slab* s, int color, int which, void** ptr, int64_t* bytes);
/* Read the neighbouring slab n's edge rows in place instead of this slab's halos: side 0 = the
 * previous slab (its last rows become this slab's low halo), 1 = the next one (periodic); NULL
 * goes back to the own halos.  Both must be slabs of the same lattice; on another device, peer
 * access is enabled (NVLink loads).  No copy is made: the caller orders each half-sweep after the
 * neighbours' previous half-sweeps (one stream, or events), and keeps n alive while it is set. */
int ising_slab_set_peer(ising_slab* s, int side, ising_slab* n);
/* Zero `pairs` (M, E) slots on the device (allocating them on first use). */
int ising_slab_series_reset(ising_slab* s, int64_t pairs);
/* One half-sweep of colour `color` at sweep counter t on the slab's stream; with slot >= 0 the
 * half-sweep also adds the slab's exact (M, E) after it to series slot `slot` (measure on
 * colour 1, the second half of a sweep, as ising_sweep does). */
int ising_slab_half_sweep(ising_slab* s, int color, uint64_t t, int64_t slot);
/* The same over rows (2D) or planes (3D) first .. first + count - 1 of the slab only: the rows
 * that read no halo (all but the first and the last) can run while the halos are still being
 * exchanged, the two edge rows after it. */
int ising_slab_half_sweep_rows(ising_slab* s, int color, uint64_t t, int64_t slot, int64_t first,
                               int64_t count);
/* Copy `pairs` series slots to the host (blocks). */
int ising_slab_series_read(ising_slab* s, int64_t pairs, int64_t* out);
/* The slab's (M, E) over its owned sites (blocks); the colour-0 halos must be current. */
int ising_slab_observables(ising_slab* s, int64_t* m, int64_t* e);
int ising_slab_sync(ising_slab* s);

/* ---- device probes (roofline ceilings and generator checks) ---------------------------- */

/* Self-test of the bounded device-side wait used by the persistent schedule: one CTA waits for
 * a flag that nothing sets, gives up after ~1 ms and records the time-out; *timed_out = 1 when
 * that happened and the context is still usable. */
int ising_selftest_bounded_wait(int device, int* timed_out);

/* Philox4x32-10 throughput of this device in calls/ns (best of `repeats`).
 * Replaces: bench/roofline.py:59-78 (philox_rate). */
int ising_philox_rate(int device, int calls_per_thread, int repeats, double* calls_per_ns);

/* out[4*i + k] = word k of Philox4x32-10((q0 + i, c1, c2, c3), (k0, k1)), i < n, computed on
 * the device (checks the device generator against philox4x32, src/pyising/philox.py:26-51). */
int ising_philox_range(int device, uint32_t q0, int64_t n, uint32_t c1, uint32_t c2, uint32_t c3,
                       uint32_t k0, uint32_t k1, uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* ISING_B200_H */
