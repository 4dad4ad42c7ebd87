// int8 compressed-checkerboard half-sweep kernel (2D/3D, Metropolis/heat bath) with the fused
// integer (M, E) reduction; the per-chunk update is int8_update in int8_core.cuh.
//
// Band schedule: the work of one launch is a list of slots (band, chunk column), band-major; a
// band is `band` consecutive rows of one plane.  A thread takes slots grid-stride and walks its
// band's rows top to bottom (int8_band), so consecutive threads of a warp read consecutive
// 16-byte chunks of the same rows.  Longer bands reuse more opposite-colour rows but leave fewer
// slots to fill the GPU; the launcher's default picks the longest band (up to 16 rows) that
// still gives every SM a wave of resident threads, and a tuned value can replace it.
#include "int8_core.cuh"

namespace ising {

template <int V, int NDIM, int RULE, bool MIXED, bool MEAS>
__global__ void __launch_bounds__(256, 4) int8_half_kernel(const Int8Half p_in)
{
    Int8Half p = p_in;
    __shared__ u32 stab[8];  // acceptance table for the per-site lookup rules
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) stab[i] = p.table[i];  // constant indices: p stays in registers
    }
    pdl_wait();  // the previous half-sweep has completed
    pdl_trigger();
    resolve_ctl(p);
    __syncthreads();
    long long m_acc = 0, e_acc = 0;
    const u32 cpr = (u32)p.cpr, bpp = (u32)p.bpp;
    const u32 nslots = (u32)p.lz * bpp * cpr;
    for (u32 slot = blockIdx.x * blockDim.x + threadIdx.x; slot < nslots;
         slot += gridDim.x * blockDim.x) {
        const u32 band = fast_div(slot, cpr, p.cpr_magic);
        const int j0 = (int)(slot - band * cpr) * V;
        int z = 0, yb = (int)band;
        if constexpr (NDIM == 3) {
            z = (int)fast_div(band, bpp, p.bpp_magic);
            yb = (int)(band - (u32)z * bpp);
        }
        const int y0 = yb * p.band;
        const int y1 = y0 + p.band < p.ly ? y0 + p.band : p.ly;
        int8_band<V, NDIM, RULE, MIXED, MEAS>(p, z, y0, y1, j0, stab, m_acc, e_acc);
    }
    if constexpr (MEAS) block_accumulate2(m_acc, e_acc, p.meas);
}

// ------------------------------------------------------------------------- host side ---
template <int V, int NDIM, bool MIXED, bool MEAS>
static cudaError_t launch_rule(int rule, const Int8Half& p, unsigned grid, cudaStream_t st)
{
    switch (rule) {
    case kMetroFast: return launch_pdl(int8_half_kernel<V, NDIM, kMetroFast, MIXED, MEAS>, grid, 256, st, p);
    case kHeatFast: return launch_pdl(int8_half_kernel<V, NDIM, kHeatFast, MIXED, MEAS>, grid, 256, st, p);
    case kMetroGeneric:
        return launch_pdl(int8_half_kernel<V, NDIM, kMetroGeneric, MIXED, MEAS>, grid, 256, st, p);
    case kHeatGeneric:
        return launch_pdl(int8_half_kernel<V, NDIM, kHeatGeneric, MIXED, MEAS>, grid, 256, st, p);
    default: return launch_pdl(int8_half_kernel<V, NDIM, kObserve, MIXED, true>, grid, 256, st, p);
    }
}

template <int V, bool MIXED = false>
static cudaError_t launch_v(int ndim, int rule, const Int8Half& p, unsigned grid, cudaStream_t st)
{
    const bool meas = p.meas != nullptr;
    if (ndim == 3)
        return meas ? launch_rule<V, 3, MIXED, true>(rule, p, grid, st)
                    : launch_rule<V, 3, MIXED, false>(rule, p, grid, st);
    return meas ? launch_rule<V, 2, MIXED, true>(rule, p, grid, st)
                : launch_rule<V, 2, MIXED, false>(rule, p, grid, st);
}

// Chunk width used for a row of lh bytes: the widest of 16/8/4 that divides it.
int int8_chunk_width(int lh) { return lh % 16 == 0 ? 16 : (lh % 8 == 0 ? 8 : 4); }

// Default band height: the longest of 16, 8, 4, 2, 1 rows whose slots still give every SM one
// wave of resident threads (4 blocks of 256 at 64 registers).
int int8_default_band(long long rows, int ly, int cpr, int sm_count)
{
    const long long want = 1024LL * sm_count;
    int b = 16;
    while (b > 1 && (rows / ly) * ((ly + b - 1) / b) * (long long)cpr < want) b >>= 1;
    return b;
}

// Fills in the band fields of p (band from p.band, or the default when p.band <= 0) and
// returns the grid: one block per 256 slots, at most max_blocks.
unsigned int8_band_geometry(Int8Half& p, int max_blocks, int sm_count)
{
    if (p.band <= 0) p.band = int8_default_band(p.rows, p.ly, p.cpr, sm_count);
    if (p.band > p.ly) p.band = p.ly;
    p.bpp = (p.ly + p.band - 1) / p.band;
    const unsigned long long nslots = (unsigned long long)p.lz * p.bpp * p.cpr;
    p.cpr_magic = fast_div_magic((u32)p.cpr, nslots);
    p.bpp_magic = fast_div_magic((u32)p.bpp, (unsigned long long)p.lz * p.bpp);
    unsigned long long g = (nslots + 255) / 256;
    if (g > (unsigned long long)max_blocks) g = (unsigned long long)max_blocks;
    return (unsigned)(g < 1 ? 1 : g);
}

cudaError_t launch_int8_half(int ndim, int rule, const Int8Half& p_in, int max_blocks, int sm_count,
                             cudaStream_t st)
{
    Int8Half p = p_in;
    const unsigned grid = int8_band_geometry(p, max_blocks, sm_count);
    const int v = p.vw;
    if (v == 16) {  // padded rows (lh % 16 != 0) need the partial-chunk code
        return (p.lh % 16) ? launch_v<16, true>(ndim, rule, p, grid, st)
                           : launch_v<16, false>(ndim, rule, p, grid, st);
    }
    if (v == 8) return launch_v<8>(ndim, rule, p, grid, st);
    return launch_v<4>(ndim, rule, p, grid, st);
}

}  // namespace ising
