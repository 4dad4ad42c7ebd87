// Persistent multi-sweep kernel for small 2D int8 lattices.
//
// A 1024^2 half-sweep is ~0.5 M sites: well under a microsecond of work, so even replayed
// graphs spend most of their time between launches.  Here one cooperative launch runs all
// 2n half-sweeps.  CTA b owns a band of rows; before half-sweep k it waits until both
// neighbouring bands (periodic in y) have published k finished half-sweeps, which covers both
// hazards of the checkerboard: the rows it reads (the other colour, written in half-sweep k-1)
// are final, and the rows it overwrites (its colour, read by the neighbours in half-sweep k-1)
// are no longer needed.  Bands exchange nothing but these flags; opposite-colour rows are read
// from L2 (ld.global.cg), so rows cached in L1 from two half-sweeps ago are never used.
//
// Publishing follows the grid-barrier pattern: __syncthreads, then one thread fences and stores
// the flag with release semantics; the waiter acquires it before its CTA reads.
// Every wait is bounded: after kSpinLimit polls the CTA records a time-out in the error word
// and leaves; a CTA that sees the error leaves too, so the launch always ends and the host turns
// the error into ISING_ERR_TIMEOUT.  Cooperative launch guarantees that all CTAs are resident.
#include "capi_internal.h"
#include "int8_core.cuh"


namespace ising {

struct PersistArgs {
    Int8Half p;          // geometry, key and table (own/other/colour/t/meas set per step)
    int8_t* c0;
    int8_t* c1;
    long long n_half;    // 2 * sweeps
    u32 t0;
    int every;           // measurement interval (0 = none)
    unsigned long long* series;
    unsigned int* flags; // per CTA: half-sweeps finished
    int* err;            // non-zero: a wait timed out
    int rows_per_cta;
    int bx_log2;
    int mute_band;       // -1; otherwise a band that stops publishing (time-out test)
};

constexpr unsigned long long kSpinLimit = 1ull << 21;  // ~1 s of polls (one L2 round trip each)

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 of a CTA waits until flags[x] >= k and flags[y] >= k, polling at most
// kSpinLimit times; returns false (and sets *err, which makes every other waiter give up too)
// on a time-out or when another CTA already timed out.
__device__ __forceinline__ bool wait_flags(const unsigned int* flags, int x, int y, unsigned k,
                                           volatile int* err, unsigned long long limit)
{
    unsigned long long spins = 0;
    while (true) {
        const unsigned int fx = ld_acquire(flags + x), fy = ld_acquire(flags + y);
        if (fx >= k && fy >= k) return true;
        if (*err || ++spins > limit) {
            *err = 1;
            return false;
        }
    }
}

// Self-test of the bounded wait: CTA 0 waits for a flag that CTA 1 never sets; the wait must
// give up, set *err and return, leaving the context usable.
__global__ void wait_selftest_kernel(unsigned int* flags, int* err, unsigned long long limit)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) wait_flags(flags, 1, 1, 1u, err, limit);
}

template <int RULE>
__global__ void __launch_bounds__(256) int8_persistent_kernel(const PersistArgs a)
{
    __shared__ u32 stab[8];
    __shared__ int s_abort;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) stab[i] = a.p.table[i];
        s_abort = 0;
    }
    __syncthreads();
    const int nb = gridDim.x, b = blockIdx.x;
    const int up = (b + nb - 1) % nb, dn = (b + 1) % nb;
    const long long r0 = (long long)b * a.rows_per_cta;
    const long long r1 = min(r0 + a.rows_per_cta, a.p.rows);
    const int bx = 1 << a.bx_log2, by = 256 >> a.bx_log2;
    const int tx = threadIdx.x & (bx - 1), ty = threadIdx.x >> a.bx_log2;
    volatile int* err = a.err;

    for (long long k = 0; k < a.n_half; ++k) {
        if (k > 0) {
            if (threadIdx.x == 0 && !wait_flags(a.flags, up, dn, (unsigned)k, err, kSpinLimit))
                s_abort = 1;
            __syncthreads();
            if (s_abort) break;
        }
        const u32 color = (u32)(k & 1);
        const long long s = k >> 1;
        Int8Half p = a.p;
        p.own = color ? a.c1 : a.c0;
        p.other = color ? a.c0 : a.c1;
        p.color = color;
        p.t = a.t0 + (u32)s;
        const bool meas = color == 1 && a.every > 0 && ((s + 1) % a.every) == 0;
        p.meas = meas ? a.series + 2 * ((s + 1) / a.every - 1) : nullptr;
        long long m_acc = 0, e_acc = 0;
        if (b == a.mute_band) break;  // test hook: this band never publishes (neighbours time out)
        for (long long row = r0 + ty; row < r1; row += by)
            for (int jc = tx; jc < p.cpr; jc += bx) {
                if (meas)
                    int8_chunk<16, 2, RULE, true, true, true>(p, row, (int)row, 0, jc * 16, stab,
                                                              m_acc, e_acc);
                else
                    int8_chunk<16, 2, RULE, true, true, false>(p, row, (int)row, 0, jc * 16, stab,
                                                               m_acc, e_acc);
            }
        if (meas) block_accumulate2(m_acc, e_acc, p.meas);
        __syncthreads();  // every row of the band is written (CTA scope) ...
        if (threadIdx.x == 0) {
            __threadfence();  // ... and, cumulatively, visible GPU-wide before the flag moves
            st_release(a.flags + b, (unsigned int)(k + 1));
        }
    }
}

// Runs n sweeps of a small 2D int8 lattice in one cooperative launch; returns ISING_ERR_STATE
// (no work done) when the device cannot hold one CTA per band, so the caller falls back.
int run_persistent_int8(ising_sim* h, uint64_t t0, int64_t n_sweeps, int64_t measure_every,
                        unsigned long long* series, unsigned int* flags, int* err, int mute_band)
{
    const int max_bands = h->sm_count;
    int nb = (int)std::min<long long>(max_bands, (h->rows + 1) / 2);
    if (nb < 1) nb = 1;
    const int rpc = (int)((h->rows + nb - 1) / nb);
    nb = (int)((h->rows + rpc - 1) / rpc);
    PersistArgs a;
    memset(&a, 0, sizeof a);
    a.p.rows = h->rows;
    a.p.lh = h->lh;
    a.p.ly = h->ly;
    a.p.lz = 1;
    a.p.pitch = h->pitch;
    a.p.vw = 16;
    a.p.cpr = (h->lh + 15) / 16;
    a.p.k0 = (u32)h->seed;
    a.p.k1 = (u32)(h->seed >> 32);
    for (int i = 0; i < 7; ++i) a.p.table[i] = h->table[i];
    a.p.ctl = nullptr;
    a.c0 = (int8_t*)h->c[0];
    a.c1 = (int8_t*)h->c[1];
    a.n_half = 2 * n_sweeps;
    a.t0 = (u32)t0;
    a.every = (int)measure_every;
    a.series = series;
    a.flags = flags;
    a.err = err;
    a.rows_per_cta = rpc;
    int bx = 1;
    while (bx < a.p.cpr && bx < 128) bx <<= 1;
    a.bx_log2 = __builtin_ctz((unsigned)bx);
    a.mute_band = mute_band;

    const void* fn;
    switch (h->rule) {
    case kMetroFast: fn = (const void*)int8_persistent_kernel<kMetroFast>; break;
    case kHeatFast: fn = (const void*)int8_persistent_kernel<kHeatFast>; break;
    case kMetroGeneric: fn = (const void*)int8_persistent_kernel<kMetroGeneric>; break;
    default: fn = (const void*)int8_persistent_kernel<kHeatGeneric>; break;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess ||
        per_sm < 1 || nb > per_sm * h->sm_count) {
        cudaGetLastError();
        return ISING_ERR_STATE;
    }
    cudaError_t e = cudaMemsetAsync(flags, 0, (size_t)nb * sizeof(unsigned int), h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "persistent sweep set-up");
    void* args[] = {&a};
    e = cudaLaunchCooperativeKernel(fn, dim3(nb), dim3(256), args, 0, h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ISING_ERR_STATE;
    }
    return ISING_OK;
}

int selftest_bounded_wait(int device, int* timed_out)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    unsigned int* flags = nullptr;
    e = cudaMalloc(&flags, 2 * sizeof(unsigned int) + sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    int* err = reinterpret_cast<int*>(flags + 2);
    e = cudaMemset(flags, 0, 2 * sizeof(unsigned int) + sizeof(int));
    if (e == cudaSuccess) {
        unsigned long long limit = 1ull << 14;  // short: ~1 ms of polling
        void* args[] = {&flags, &err, &limit};
        e = cudaLaunchCooperativeKernel((const void*)wait_selftest_kernel, dim3(2), dim3(32),
                                        args, 0, 0);
    }
    int host_err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(flags);
    if (e != cudaSuccess) return cuda_fail(e, "bounded-wait self-test");
    *timed_out = host_err;
    return ISING_OK;
}

}  // namespace ising
