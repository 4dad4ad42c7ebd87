// Layout conversion between a full int8 lattice and the per-colour device arrays, done on the
// device so that set_lattice/get_lattice move one array across PCIe and no host-side reshuffle
// of a multi-GB lattice is needed.
//
// Colour c of row r (row parity rp = (y + z) % 2) holds x = 2j + ((rp + c) % 2)
// (src/pyising/lattice.py:50-72).  The packed layout sets bit b of word w for compressed site
// 64w + b when that spin is +1 (src/pyising/lattice.py:75-90).  Also: the Philox throughput
// probe (the measured RNG ceiling, like bench/roofline.py:24-36 in the reference).
#include "common.cuh"

namespace ising {

// full (rows, 2*lh) -> c0, c1 (rows, lh); one thread per 4 compressed sites of both colours.
__global__ void int8_split_kernel(const int8_t* __restrict__ full, int8_t* __restrict__ c0,
                                  int8_t* __restrict__ c1, long long rows, long long row0,
                                  int lh, int pitch, int ly)
{
    const int qpr = lh / 4;
    const long long total = rows * qpr;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / qpr;
        const int q = (int)(i - row * qpr);
        const long long ar = row0 + row;
        const int y = (int)(ar % ly), z = (int)(ar / ly);
        const int rp = (y + z) & 1;
        const uint2 v = *reinterpret_cast<const uint2*>(full + row * 2 * lh + 8 * q);
        const u32 even = __byte_perm(v.x, v.y, 0x6420);
        const u32 odd = __byte_perm(v.x, v.y, 0x7531);
        *reinterpret_cast<u32*>(c0 + row * pitch + 4 * q) = rp ? odd : even;
        *reinterpret_cast<u32*>(c1 + row * pitch + 4 * q) = rp ? even : odd;
    }
}

__global__ void int8_merge_kernel(const int8_t* __restrict__ c0, const int8_t* __restrict__ c1,
                                  int8_t* __restrict__ full, long long rows, long long row0,
                                  int lh, int pitch, int ly)
{
    const int qpr = lh / 4;
    const long long total = rows * qpr;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / qpr;
        const int q = (int)(i - row * qpr);
        const long long ar = row0 + row;
        const int y = (int)(ar % ly), z = (int)(ar / ly);
        const int rp = (y + z) & 1;
        const u32 a = *reinterpret_cast<const u32*>(c0 + row * pitch + 4 * q);
        const u32 b = *reinterpret_cast<const u32*>(c1 + row * pitch + 4 * q);
        const u32 e = rp ? b : a;  // sites at even x
        const u32 o = rp ? a : b;  // sites at odd x
        uint2 v;
        v.x = __byte_perm(e, o, 0x5140);
        v.y = __byte_perm(e, o, 0x7362);
        *reinterpret_cast<uint2*>(full + row * 2 * lh + 8 * q) = v;
    }
}

// full (rows, 128*nw) -> packed w0, w1 (rows, nw).  One warp per output word pair position:
// lane l tests compressed sites 64w + l and 64w + 32 + l with two ballots per colour.
__global__ void msc_pack_kernel(const int8_t* __restrict__ full, u64* __restrict__ w0,
                                u64* __restrict__ w1, int rows, int row0, int nw)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long total = (long long)rows * nw;
    for (long long i = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
         i < total; i += warps) {
        const int row = (int)(i / nw);
        const int w = (int)(i - (long long)row * nw);
        const int rp = (row0 + row) & 1;
        const int8_t* src = full + (long long)row * 128 * nw;
        const int j0 = 64 * w + lane, j1 = 64 * w + 32 + lane;
        // colour c sits at x = 2j + ((rp + c) & 1)
        const u32 c0lo = __ballot_sync(0xFFFFFFFFu, src[2 * j0 + rp] > 0);
        const u32 c0hi = __ballot_sync(0xFFFFFFFFu, src[2 * j1 + rp] > 0);
        const u32 c1lo = __ballot_sync(0xFFFFFFFFu, src[2 * j0 + (rp ^ 1)] > 0);
        const u32 c1hi = __ballot_sync(0xFFFFFFFFu, src[2 * j1 + (rp ^ 1)] > 0);
        if (lane == 0) {
            w0[i] = (u64)c0lo | ((u64)c0hi << 32);
            w1[i] = (u64)c1lo | ((u64)c1hi << 32);
        }
    }
}

// packed -> full; one thread per compressed site pair (both colours of index j).
__global__ void msc_unpack_kernel(const u64* __restrict__ w0, const u64* __restrict__ w1,
                                  int8_t* __restrict__ full, int rows, int row0, int nw)
{
    const long long lh = 64LL * nw;
    const long long total = (long long)rows * lh;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / lh;
        const long long j = i - row * lh;
        const int rp = (int)((row0 + row) & 1);
        const long long wi = row * nw + (j >> 6);
        const int b = (int)(j & 63);
        const int8_t s0 = ((w0[wi] >> b) & 1ull) ? 1 : -1;
        const int8_t s1 = ((w1[wi] >> b) & 1ull) ? 1 : -1;
        int8_t* dst = full + row * 2 * lh + 2 * j;
        dst[rp] = s0;
        dst[rp ^ 1] = s1;
    }
}

static unsigned grid_for(long long total, int threads, int max_blocks);

// Device seeded start (not in the reference, whose hot start is NumPy's PCG64): compressed site
// n of colour c is +1 iff bit n % 32 of word (n / 32) % 4 of Philox((n / 128, 0, c, 0xFFFFFFFF),
// seed) is set.  Counter word 3 = 0xFFFFFFFF is never used by a sweep, and int8 and packed
// layouts get the same spins.  n is the logical index row * lh + j whatever the row pitch.
__global__ void philox_start_int8_kernel(int8_t* c0, int8_t* c1, long long rows, int lh,
                                         int pitch, u32 k0, u32 k1)
{
    const int qpr = lh / 4;  // 4-site quads per row (lh % 4 == 0)
    const long long quads = rows * qpr;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * quads;
         i += (long long)gridDim.x * blockDim.x) {
        const u32 color = (u32)(i / quads);
        const long long qi = i - (long long)color * quads;
        const long long row = qi / qpr;
        const int q = (int)(qi - row * qpr);
        const long long n = row * lh + 4LL * q;
        const u32x4 r = philox4x32_10((u32)(n >> 7), 0u, color, 0xFFFFFFFFu, k0, k1);
        const int word = (int)((n >> 5) & 3);
        const u32 rw = word == 0 ? r.x : (word == 1 ? r.y : (word == 2 ? r.z : r.w));
        const u32 nib = (rw >> (n & 31)) & 0xFu;
        const u32 ones = (nib * 0x00204081u) & 0x01010101u;  // bit i -> byte i
        int8_t* dst = (color ? c1 : c0) + row * pitch + 4 * q;
        *reinterpret_cast<u32*>(dst) = 0xFFFFFFFFu ^ (ones * 0xFEu);  // 1 -> +1, 0 -> -1
    }
}

// Packed layout: words 2g, 2g+1 of a colour come from call g (sites 128g .. 128g + 127).
__global__ void philox_start_msc_kernel(u64* w0, u64* w1, long long words, u32 k0, u32 k1)
{
    const long long groups = words / 2;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * groups;
         i += (long long)gridDim.x * blockDim.x) {
        const u32 color = (u32)(i / groups);
        const long long g = i - (long long)color * groups;
        const u32x4 r = philox4x32_10((u32)g, 0u, color, 0xFFFFFFFFu, k0, k1);
        u64* w = (color ? w1 : w0) + 2 * g;
        w[0] = (u64)r.x | ((u64)r.y << 32);
        w[1] = (u64)r.z | ((u64)r.w << 32);
    }
}

// rows x lh sites per colour (int8, rows `pitch` bytes apart) or rows x nw words (packed).
cudaError_t launch_philox_start(void* c0, void* c1, long long rows, int lh, int pitch, int packed,
                                u32 k0, u32 k1, int max_blocks, cudaStream_t st)
{
    if (packed) {
        const long long words = rows * (lh / 64);
        philox_start_msc_kernel<<<grid_for(words, 256, max_blocks), 256, 0, st>>>(
            static_cast<u64*>(c0), static_cast<u64*>(c1), words, k0, k1);
    } else {
        const long long work = 2 * rows * (lh / 4);
        philox_start_int8_kernel<<<grid_for(work, 256, max_blocks), 256, 0, st>>>(
            static_cast<int8_t*>(c0), static_cast<int8_t*>(c1), rows, lh, pitch, k0, k1);
    }
    return cudaGetLastError();
}

// Throughput probe: `calls` Philox blocks per thread, outputs xor-folded so nothing is dead.
__global__ void philox_probe_kernel(u32* __restrict__ out, int calls, u32 k0, u32 k1)
{
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    u32 acc = 0;
    for (int i = 0; i < calls; ++i) {
        const u32x4 r = philox4x32_10(tid, (u32)i, 0u, 0u, k0, k1);
        acc ^= r.x ^ r.y ^ r.z ^ r.w;
    }
    out[tid] = acc;
}

// Philox over a counter range for testing the device generator against the oracle:
// out[4 i + k] = word k of Philox((q0 + i, c1, c2, c3), (k0, k1)).
__global__ void philox_range_kernel(u32* __restrict__ out, long long n, u32 q0, u32 c1, u32 c2,
                                    u32 c3, u32 k0, u32 k1)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const u32x4 r = philox4x32_10(q0 + (u32)i, c1, c2, c3, k0, k1);
        reinterpret_cast<uint4*>(out)[i] = make_uint4(r.x, r.y, r.z, r.w);
    }
}

static unsigned grid_for(long long total, int threads, int max_blocks)
{
    long long g = (total + threads - 1) / threads;
    if (g > max_blocks) g = max_blocks;
    if (g < 1) g = 1;
    return (unsigned)g;
}

cudaError_t launch_int8_split(const int8_t* full, int8_t* c0, int8_t* c1, long long rows,
                              long long row0, int lh, int pitch, int ly, int max_blocks,
                              cudaStream_t st)
{
    const long long total = rows * (lh / 4);
    int8_split_kernel<<<grid_for(total, 256, max_blocks), 256, 0, st>>>(full, c0, c1, rows,
                                                                        row0, lh, pitch, ly);
    return cudaGetLastError();
}

cudaError_t launch_int8_merge(const int8_t* c0, const int8_t* c1, int8_t* full, long long rows,
                              long long row0, int lh, int pitch, int ly, int max_blocks,
                              cudaStream_t st)
{
    const long long total = rows * (lh / 4);
    int8_merge_kernel<<<grid_for(total, 256, max_blocks), 256, 0, st>>>(c0, c1, full, rows,
                                                                        row0, lh, pitch, ly);
    return cudaGetLastError();
}

cudaError_t launch_msc_pack(const int8_t* full, u64* w0, u64* w1, int rows, int row0, int nw,
                            int max_blocks, cudaStream_t st)
{
    const long long total = (long long)rows * nw * 32;
    msc_pack_kernel<<<grid_for(total, 256, max_blocks), 256, 0, st>>>(full, w0, w1, rows, row0,
                                                                      nw);
    return cudaGetLastError();
}

cudaError_t launch_msc_unpack(const u64* w0, const u64* w1, int8_t* full, int rows, int row0,
                              int nw, int max_blocks, cudaStream_t st)
{
    const long long total = (long long)rows * nw * 64;
    msc_unpack_kernel<<<grid_for(total, 256, max_blocks), 256, 0, st>>>(w0, w1, full, rows,
                                                                        row0, nw);
    return cudaGetLastError();
}

cudaError_t launch_philox_probe(u32* out, int blocks, int threads, int calls, u32 k0, u32 k1,
                                cudaStream_t st)
{
    philox_probe_kernel<<<blocks, threads, 0, st>>>(out, calls, k0, k1);
    return cudaGetLastError();
}

cudaError_t launch_philox_range(u32* out, long long n, u32 q0, u32 c1, u32 c2, u32 c3, u32 k0,
                                u32 k1, int max_blocks, cudaStream_t st)
{
    philox_range_kernel<<<grid_for(n, 256, max_blocks), 256, 0, st>>>(out, n, q0, c1, c2, c3,
                                                                      k0, k1);
    return cudaGetLastError();
}

}  // namespace ising
