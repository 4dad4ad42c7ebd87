// Shared device code: Philox4x32-10, SWAR helpers, reductions and launch-parameter structs.
//
// Philox4x32-10 follows Salmon et al., SC'11 (the published Random123 algorithm) with the
// counter/key conventions of pyising's oracle: src/pyising/philox.py:26-51 (multipliers,
// Weyl key increments, key bumped between rounds but not after the last one).
#pragma once

#include <cstdint>
#include <utility>

#include <cuda_runtime.h>

namespace ising {

typedef uint32_t u32;
typedef uint64_t u64;

constexpr u32 kPhiloxM0 = 0xD2511F53u;
constexpr u32 kPhiloxM1 = 0xCD9E8D57u;
constexpr u32 kPhiloxW0 = 0x9E3779B9u;
constexpr u32 kPhiloxW1 = 0xBB67AE85u;

struct u32x4 {
    u32 x, y, z, w;
};

// One Philox4x32-10 block.  The counter words c1..c3 and the key are usually uniform across a
// warp (sweep, colour, stream selector, seed), so the compiler keeps the first two rounds'
// products in the uniform datapath; only the site/word index c0 varies per thread.
// SPLIT: each 32x32->64 product as a separate high and low multiply (the same values); on
// B200 that measured 4% faster inside the 2D int8 kernels, 1% slower in 3D and equal in msc.
template <bool SPLIT = false>
__device__ __forceinline__ u32x4 philox4x32_10(u32 c0, u32 c1, u32 c2, u32 c3, u32 k0, u32 k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        u32 h0, l0, h1, l1;
        if constexpr (SPLIT) {
            asm("mul.hi.u32 %0, %1, %2;" : "=r"(h0) : "r"(c0), "n"(kPhiloxM0));
            asm("mul.lo.u32 %0, %1, %2;" : "=r"(l0) : "r"(c0), "n"(kPhiloxM0));
            asm("mul.hi.u32 %0, %1, %2;" : "=r"(h1) : "r"(c2), "n"(kPhiloxM1));
            asm("mul.lo.u32 %0, %1, %2;" : "=r"(l1) : "r"(c2), "n"(kPhiloxM1));
        } else {
            const u64 p0 = (u64)kPhiloxM0 * c0;
            const u64 p1 = (u64)kPhiloxM1 * c2;
            h0 = (u32)(p0 >> 32);
            l0 = (u32)p0;
            h1 = (u32)(p1 >> 32);
            l1 = (u32)p1;
        }
        const u32 n0 = h1 ^ c1 ^ k0;
        const u32 n2 = h0 ^ c3 ^ k1;
        c1 = l1;
        c3 = l0;
        c0 = n0;
        c2 = n2;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return u32x4{c0, c1, c2, c3};
}

// Byte lanes of packed int8 spins: +1 is 0x01, -1 is 0xFF, so bit 1 of a byte is the
// "spin down" flag and (a ^ b) & 0x02 is the "anti-aligned" flag of two spins.
constexpr u32 kBit1 = 0x02020202u;
constexpr u32 kBit7 = 0x80808080u;

// 0x80 per selected byte -> 0xFE per selected byte (the XOR that flips a +-1 byte).
__device__ __forceinline__ u32 flip_mask_from_bit7(u32 m7) { return m7 | (m7 - (m7 >> 6)); }

// Sum of the four bytes of v (each byte small and non-negative).
__device__ __forceinline__ int byte_sum(u32 v) { return (int)__dp4a(v, 0x01010101u, 0u); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Block-wide sum of two int64 values, then one atomicAdd per block into out[0], out[1].
// Every thread of the block must call it.
__device__ __forceinline__ void block_accumulate2(long long a, long long b,
                                                  unsigned long long* out)
{
    __shared__ long long sa[32], sb[32];
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    const int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
    __syncthreads();  // a previous call's readers of sa/sb are done
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        a = lane < nwarps ? sa[lane] : 0;
        b = lane < nwarps ? sb[lane] : 0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (lane == 0) {
            atomicAdd(out, (unsigned long long)a);
            atomicAdd(out + 1, (unsigned long long)b);
        }
    }
}

// Decision rule selected on the host.
enum Rule : int {
    kMetroFast = 0,    // Metropolis, table[d+1..2d] non-increasing (always true for tables
                       // built by threshold_table)
    kHeatFast = 1,     // heat bath, table non-decreasing (beta >= 0)
    kMetroGeneric = 2, // any table, one lookup per site
    kHeatGeneric = 3,
    kObserve = 4,      // no update: measurement only
};

// Parameters of one int8 half-sweep launch over a (rows, lh) colour array pair.
struct Int8Half {
    int8_t* own;
    const int8_t* other;
    long long rows;
    int lh;      // Lx / 2 (bytes per row)
    int ly;      // rows per z plane
    int lz;      // planes (1 in 2D)
    int cpr;     // chunks per row = ceil(lh / V)
    int pitch;   // bytes between rows in memory (lh, or lh rounded up to 16 with V = 16)
    int vw;      // chunk width V: 16, 8 or 4 bytes
    int band;    // band schedule: rows of one plane a thread walks (0: the launcher picks)
    int bpp;     // band schedule: bands per plane = ceil(ly / band)
    u32 cpr_magic, bpp_magic;  // fast_div magics of cpr and bpp (0: divide)
    u32 t;       // sweep counter (Philox counter word 1)
    u32 color;   // colour being updated (Philox counter word 2)
    u32 k0, k1;  // Philox key (seed lo, hi)
    u32 table[7];
    unsigned long long* meas;  // (M, E) accumulators, or nullptr
    // Graph-replay control block, or nullptr: when set, the sweep counter is ctl[0] + t and the
    // accumulators are meas + 2 * ctl[1] (a captured chunk of sweeps advances ctl itself).
    const unsigned long long* ctl;
};

// Parameters of one packed (msc) half-sweep launch over (rows, nw) uint64 words.
struct MscHalf {
    u64* own;
    const u64* other;
    int rows;
    int nw;     // words per row = Lx / 128
    u32 t, color, k0, k1;
    u32 thr4;   // table[3]: acceptance for one anti-aligned neighbour (dE = 4)
    u32 thr8;   // table[4]: acceptance for none (dE = 8)
    u64 nw_magic;  // ceil(2^64 / nw): w / nw = umulhi64(w, nw_magic) for w < 2^32
    unsigned long long* meas;   // (M, E) accumulators, or nullptr
    unsigned long long* stats;  // (calls, warp-max calls) diagnostics, or nullptr
    const unsigned long long* ctl;  // graph-replay control block, as in Int8Half
};

// w / d with m = ceil(2^64 / d): for 0 <= w < 2^32 and 1 < d < 2^32 the error of w * m / 2^64
// is below w / 2^64 < 1/d, so it never crosses the next integer; larger w divide directly.
__device__ __forceinline__ long long div_magic(long long w, u64 m, int d)
{
    return ((u64)w >> 32) ? w / d : (long long)__umul64hi((u64)w, m);
}

inline u64 magic_for(int d) { return d > 1 ? ~0ull / (u64)d + 1ull : 0ull; }

// n / d with m = ceil(2^32 / d) when n * d < 2^32 holds for every n passed (then
// floor(n * m / 2^32) is exact: the error n * (m * d - 2^32) / (d * 2^32) stays below 1/d),
// else m = 0 and a plain division.
__device__ __forceinline__ u32 fast_div(u32 n, u32 d, u32 m) { return m ? __umulhi(n, m) : n / d; }

inline u32 fast_div_magic(u32 d, unsigned long long n_max)
{
    if (d < 2 || n_max * d >= (1ull << 32)) return 0;
    return (u32)(((1ull << 32) + d - 1) / d);
}

// Programmatic dependent launch.  Half-sweep kernels are launched with programmatic stream
// serialization (launch_pdl), so a half-sweep's grid may be launched while the previous kernel
// of the stream is still running: hiding the launch latency, which for small lattices is most
// of a half-sweep.  Each such kernel waits in pdl_wait (griddepcontrol.wait: the previous grid
// has completed and its writes are visible) before it reads the lattice or the control block,
// then lets its own successor launch (pdl_trigger).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                              Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Resolve the graph-replay control block of a launch (see Int8Half::ctl).
template <typename P>
__device__ __forceinline__ void resolve_ctl(P& p)
{
    if (p.ctl) {
        p.t += (u32)p.ctl[0];
        if (p.meas) p.meas += 2 * p.ctl[1];
    }
}

}  // namespace ising
