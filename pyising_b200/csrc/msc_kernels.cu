// Single-lattice multi-spin-coded half-sweep kernels: the work-stack kernel (every sweep; a
// measured half-sweep measures each warp's words after updating them) and the one-word-per-
// thread kernel (the observables reduction and the call statistics).  Device code in
// msc_core.cuh.
#include "msc_core.cuh"

#ifndef ISING_MSC_MIN_BLOCKS
#define ISING_MSC_MIN_BLOCKS 1
#endif

namespace ising {

template <bool UPDATE>
__global__ void __launch_bounds__(256) msc_half_kernel(const MscHalf p_in)
{
    MscHalf p = p_in;
    resolve_ctl(p);
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    long long m_acc = 0, e_acc = 0;
    long long calls_acc = 0, wmax_acc = 0;
    if (x < p.nw) {
        for (int y = blockIdx.y * blockDim.y + threadIdx.y; y < p.rows;
             y += gridDim.y * blockDim.y)
            msc_word<UPDATE>(p, y, x, m_acc, e_acc, calls_acc, wmax_acc);
    }
    if (p.meas) block_accumulate2(m_acc, e_acc, p.meas);
    if (UPDATE && p.stats) block_accumulate2(calls_acc, wmax_acc, p.stats);
}

constexpr int kQueueWarps = 8;

template <bool MEAS>
__global__ void __launch_bounds__(kQueueWarps * 32, ISING_MSC_MIN_BLOCKS)
    msc_half_queue_kernel(const MscHalf p_in, long long total, long long per_warp, int nw_shift)
{
    MscHalf p = p_in;
    __shared__ QueueSlots q_all[kQueueWarps];
    __shared__ uint4 lvmask[16];
    if (threadIdx.x < 16) lvmask[threadIdx.x] = level_masks(p.thr4, p.thr8, threadIdx.x);
    pdl_wait();  // the previous half-sweep has completed
    pdl_trigger();
    resolve_ctl(p);
    __syncthreads();
    const long long begin = ((long long)blockIdx.x * kQueueWarps + (threadIdx.x >> 5)) * per_warp;
    const long long end = min(begin + per_warp, total);
    msc_queue_range(p, begin, end, nw_shift, q_all[threadIdx.x >> 5], lvmask);
    if constexpr (MEAS) {
        // the warp's words are final: measure them (the other colour is unchanged)
        __syncwarp();
        long long m_acc = 0, e_acc = 0;
        msc_measure_range(p, begin, end, nw_shift, m_acc, e_acc);
        block_accumulate2(m_acc, e_acc, p.meas);
    }
}

// Strip schedule: warp g walks rows [band (g / strips), band (g / strips + 1)) of strip
// g % strips; K Philox blocks per word at intake; registers bounded for MINB resident blocks.
template <bool MEAS, int K, int MINB>
__global__ void __launch_bounds__(kQueueWarps * 32, MINB)
    msc_strip_kernel(const MscHalf p_in, int strips, int band)
{
    MscHalf p = p_in;
    __shared__ StripSlots q_all[kQueueWarps];
    __shared__ uint4 lvmask[16];
    if (threadIdx.x < 16) lvmask[threadIdx.x] = level_masks(p.thr4, p.thr8, threadIdx.x);
    pdl_wait();  // the previous half-sweep has completed
    pdl_trigger();
    resolve_ctl(p);
    __syncthreads();
    const int g = blockIdx.x * kQueueWarps + (threadIdx.x >> 5);
    const int strip = g % strips;
    const int y0 = (g / strips) * band;
    const int y1 = min(y0 + band, p.rows);
    if (y0 < p.rows) msc_strip_band<K>(p, strip, y0, y1, q_all[threadIdx.x >> 5], lvmask);
    if constexpr (MEAS) {
        __syncwarp();
        long long m_acc = 0, e_acc = 0;
        if (y0 < p.rows) msc_measure_strip(p, strip, y0, y1, m_acc, e_acc);
        block_accumulate2(m_acc, e_acc, p.meas);
    }
}

void msc_geometry(int rows, int nw, int max_blocks, dim3* grid, dim3* block)
{
    int bx = 1;
    while (bx < nw && bx < 128) bx <<= 1;
    const int by = 256 / bx;
    const int gx = (nw + bx - 1) / bx;
    long long gy = ((long long)rows + by - 1) / by;
    long long cap = max_blocks / gx;
    if (cap < 1) cap = 1;
    if (gy > cap) gy = cap;
    if (gy > 65535) gy = 65535;
    *grid = dim3((unsigned)gx, (unsigned)gy, 1);
    *block = dim3((unsigned)bx, (unsigned)by, 1);
}

// Resident blocks per SM of the work-stack kernel (occupancy query, cached per device).
static int queue_blocks_per_sm()
{
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, msc_half_queue_kernel<false>,
                                                          kQueueWarps * 32, 0) != cudaSuccess ||
            b < 1) {
            cudaGetLastError();
            b = 2;
        }
        cached[dev] = b;
    }
    return cached[dev];
}

int msc_nw_shift(int nw) { return (nw & (nw - 1)) == 0 ? __builtin_ctz((unsigned)nw) : -1; }

template <bool MEAS, int K, int MINB>
static int strip_blocks_per_sm()
{
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, msc_strip_kernel<MEAS, K, MINB>,
                                                          kQueueWarps * 32, 0) != cudaSuccess ||
            b < 1) {
            cudaGetLastError();
            b = 2;
        }
        cached[dev] = b;
    }
    return cached[dev];
}

template <bool MEAS, int K, int MINB>
static cudaError_t launch_strip(const MscHalf& p, int sm_count, int waves, cudaStream_t st)
{
    const int strips = p.nw / 32;
    const long long units = (long long)p.rows * strips;  // (row, strip) steps
    const long long warps = (long long)(sm_count > 0 ? sm_count : 1) *
                            strip_blocks_per_sm<MEAS, K, MINB>() * kQueueWarps * (waves > 0 ? waves : 1);
    long long band = (units + warps - 1) / warps;
    if (band < 1) band = 1;
    const long long nwarps = (long long)strips * ((p.rows + band - 1) / band);
    const unsigned blocks = (unsigned)((nwarps + kQueueWarps - 1) / kQueueWarps);
    return launch_pdl(msc_strip_kernel<MEAS, K, MINB>, dim3(blocks), dim3(kQueueWarps * 32), st, p,
                      strips, (int)band);
}

template <int K, int MINB>
static cudaError_t strip_launch(const MscHalf& p, int sm_count, int waves, cudaStream_t st)
{
    return p.meas ? launch_strip<true, K, MINB>(p, sm_count, waves, st)
                  : launch_strip<false, K, MINB>(p, sm_count, waves, st);
}

cudaError_t launch_msc_half(bool update, const MscHalf& p, int max_blocks, int sm_count,
                            int waves, cudaStream_t st, int kernel)
{
    // the strip schedule needs rows of whole 32-word strips and word indices below 2^32
    const bool strip_ok = p.nw % 32 == 0 && (long long)p.rows * p.nw <= 0xFFFFFFFFll;
    // automatic: the strips (4 intake blocks, registers for 2 blocks per SM) wherever the rows
    // hold whole 32-word strips, the word ranges elsewhere
    if (kernel == 0) kernel = strip_ok ? 2 : 1;
    if (update && !p.stats && strip_ok && kernel >= 2) {
        switch (kernel) {
        case 2: return strip_launch<4, 2>(p, sm_count, waves, st);
        case 3: return strip_launch<4, 3>(p, sm_count, waves, st);
        case 4: return strip_launch<4, 4>(p, sm_count, waves, st);
        case 5: return strip_launch<3, 2>(p, sm_count, waves, st);
        case 6: return strip_launch<3, 3>(p, sm_count, waves, st);
        default: return strip_launch<3, 4>(p, sm_count, waves, st);
        }
    }
    if (update && !p.stats) {
        // `waves` resident waves of warps (one by default), each warp with an equal contiguous
        // range of words
        const long long total = (long long)p.rows * p.nw;
        const long long warps = (long long)(sm_count > 0 ? sm_count : 1) * queue_blocks_per_sm() *
                                kQueueWarps * (waves > 0 ? waves : 1);
        long long per_warp = (total + warps - 1) / warps;
        per_warp = (per_warp + 31) / 32 * 32;
        if (per_warp < 32) per_warp = 32;
        const long long nwarps = (total + per_warp - 1) / per_warp;
        const unsigned blocks = (unsigned)((nwarps + kQueueWarps - 1) / kQueueWarps);
        if (p.meas)
            return launch_pdl(msc_half_queue_kernel<true>, dim3(blocks), dim3(kQueueWarps * 32),
                              st, p, total, per_warp, msc_nw_shift(p.nw));
        return launch_pdl(msc_half_queue_kernel<false>, dim3(blocks), dim3(kQueueWarps * 32), st,
                          p, total, per_warp, msc_nw_shift(p.nw));
    }
    dim3 grid, block;
    msc_geometry(p.rows, p.nw, max_blocks, &grid, &block);
    if (update) msc_half_kernel<true><<<grid, block, 0, st>>>(p);
    else msc_half_kernel<false><<<grid, block, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace ising
