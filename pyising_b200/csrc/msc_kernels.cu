// Multi-spin-coded (64 spins per uint64) 2D Metropolis half-sweep with the lazy bitwise
// uniform comparison, and its fused integer (M, E) reduction.
//
// Same results as pyising's NumpyMultiSpin (src/pyising/backends/numpy_backend.py:54-124) and
// the CUDA C msc_half kernel (src/pyising/backends/cuda/ising.cu:92-150): word w at bit level
// k uses call k/2 of Philox((w, t, c, 1 + k/2), seed); even levels take r0 | r1 << 32, odd
// levels r2 | r3 << 32 (src/pyising/philox.py:67-78).  Level k decides the lanes whose
// uniform's bit 31-k differs from the threshold's: u < thr exactly when, at the first
// differing bit, u has 0 and the threshold has 1.
#include "common.cuh"

namespace ising {

// Bit-sliced anti-aligned count of the four neighbours: a0 = none, a1 = exactly one,
// a2 = two or more (numpy_backend.py:63-69).
struct Slices {
    u64 a0, a1, a2;
};

__device__ __forceinline__ Slices slice4(u64 o, u64 n1, u64 n2, u64 n3, u64 n4)
{
    const u64 x1 = o ^ n1, x2 = o ^ n2, x3 = o ^ n3, x4 = o ^ n4;
    const u64 any = x1 | x2 | x3 | x4;
    const u64 s1 = x1 ^ x2, c1 = x1 & x2, s2 = x3 ^ x4, c2 = x3 & x4;
    Slices s;
    s.a2 = c1 | c2 | (s1 & s2);
    s.a1 = any & ~s.a2;
    s.a0 = ~any;
    return s;
}

__device__ __forceinline__ void lazy_level(u64 r, int bit, u32 thr4, u32 thr8, const Slices& s,
                                           u64& acc, u64& und)
{
    const u64 t4 = ((thr4 >> bit) & 1u) ? ~0ull : 0ull;
    const u64 t8 = ((thr8 >> bit) & 1u) ? ~0ull : 0ull;
    const u64 tm = (s.a1 & t4) | (s.a0 & t8);
    acc |= und & ~r & tm;
    und &= ~(r ^ tm);
}

// Flip mask of one word; `calls` returns the Philox blocks drawn.
__device__ __forceinline__ u64 msc_flip(const Slices& s, u32 w, u32 t, u32 color, u32 k0,
                                        u32 k1, u32 thr4, u32 thr8, int& calls)
{
    u64 acc = 0, und = s.a0 | s.a1;
    int lp = 0;
    for (; lp < 16 && und; ++lp) {
        const u32x4 r = philox4x32_10(w, t, color, 1u + (u32)lp, k0, k1);
        lazy_level((u64)r.x | ((u64)r.y << 32), 31 - 2 * lp, thr4, thr8, s, acc, und);
        lazy_level((u64)r.z | ((u64)r.w << 32), 30 - 2 * lp, thr4, thr8, s, acc, und);
    }
    calls = lp;
    return s.a2 | acc;
}

template <bool UPDATE>
__global__ void __launch_bounds__(256) msc_half_kernel(const MscHalf p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    long long m_acc = 0, e_acc = 0;
    long long calls_acc = 0, wmax_acc = 0;
    if (x < p.nw) {
        const int nw = p.nw;
        for (int y = blockIdx.y * blockDim.y + threadIdx.y; y < p.rows;
             y += gridDim.y * blockDim.y) {
            const long long rb = (long long)y * nw;
            const u64* orow = p.other + rb;
            const u64 o = p.own[rb + x];
            const u64 c = __ldg(orow + x);
            const int par = (y + (int)p.color) & 1;
            u64 hz;
            if (par) hz = (c >> 1) | (__ldg(orow + (x + 1 == nw ? 0 : x + 1)) << 63);
            else hz = (c << 1) | (__ldg(orow + (x == 0 ? nw - 1 : x - 1)) >> 63);
            const u64 up = __ldg(p.other + (long long)(y == 0 ? p.rows - 1 : y - 1) * nw + x);
            const u64 dn = __ldg(p.other + (long long)(y + 1 == p.rows ? 0 : y + 1) * nw + x);
            u64 ns = o;
            if constexpr (UPDATE) {
                const Slices s = slice4(o, c, hz, up, dn);
                int calls = 0;
                ns = o ^ msc_flip(s, (u32)(rb + x), p.t, p.color, p.k0, p.k1, p.thr4, p.thr8,
                                  calls);
                p.own[rb + x] = ns;
                if (p.stats) {
                    calls_acc += calls;
                    wmax_acc += __reduce_max_sync(__activemask(), calls);
                }
            }
            if (p.meas) {
                const int anti = __popcll(ns ^ c) + __popcll(ns ^ hz) + __popcll(ns ^ up) +
                                 __popcll(ns ^ dn);
                m_acc += 2 * (__popcll(ns) + __popcll(c)) - 128;
                e_acc += 2 * anti - 256;
            }
        }
    }
    if (p.meas) block_accumulate2(m_acc, e_acc, p.meas);
    if (UPDATE && p.stats) block_accumulate2(calls_acc, wmax_acc, p.stats);
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

cudaError_t launch_msc_half(bool update, const MscHalf& p, int max_blocks, cudaStream_t st)
{
    dim3 grid, block;
    msc_geometry(p.rows, p.nw, max_blocks, &grid, &block);
    if (update) msc_half_kernel<true><<<grid, block, 0, st>>>(p);
    else msc_half_kernel<false><<<grid, block, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace ising
