// int8 compressed-checkerboard half-sweep kernel (2D/3D, Metropolis/heat bath) with the fused
// integer (M, E) reduction; the per-chunk update is int8_chunk in int8_core.cuh.
#include "int8_core.cuh"

namespace ising {

template <int V, int NDIM, int RULE, bool MIXED>
__global__ void __launch_bounds__(256, 4) int8_half_kernel(const Int8Half p_in)
{
    Int8Half p = p_in;
    resolve_ctl(p);
    __shared__ u32 stab[8];  // acceptance table for the per-site lookup rules
    if (threadIdx.x == 0 && threadIdx.y == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) stab[i] = p.table[i];  // constant indices: stays in params
    }
    __syncthreads();
    const int jc = blockIdx.x * blockDim.x + threadIdx.x;
    long long m_acc = 0, e_acc = 0;
    if (jc < p.cpr) {
        const int j0 = jc * V;
        const int row_step = gridDim.y * blockDim.y;
        const int row0 = blockIdx.y * blockDim.y + threadIdx.y;
        // (y, z) of the row, advanced without divisions in the loop (rows < 2^31)
        int y = row0, z = 0, sy = row_step, sz = 0;
        if constexpr (NDIM == 3) {
            z = row0 / p.ly;
            y = row0 - z * p.ly;
            sz = row_step / p.ly;
            sy = row_step - sz * p.ly;
        }
        for (long long row = row0; row < p.rows; row += row_step) {
            if constexpr (NDIM == 3) {
                if (row != row0) {
                    y += sy;
                    z += sz;
                    if (y >= p.ly) {
                        y -= p.ly;
                        ++z;
                    }
                }
            } else {
                y = (int)row;
            }
            int8_chunk<V, NDIM, RULE, false, MIXED>(p, row, y, z, j0, stab, m_acc, e_acc);
        }
    }
    if (p.meas) block_accumulate2(m_acc, e_acc, p.meas);
}

// ------------------------------------------------------------------------- host side ---
template <int V, int NDIM, bool MIXED>
static cudaError_t launch_rule(int rule, const Int8Half& p, dim3 grid, dim3 block,
                               cudaStream_t st)
{
    switch (rule) {
    case kMetroFast: int8_half_kernel<V, NDIM, kMetroFast, MIXED><<<grid, block, 0, st>>>(p); break;
    case kHeatFast: int8_half_kernel<V, NDIM, kHeatFast, MIXED><<<grid, block, 0, st>>>(p); break;
    case kMetroGeneric:
        int8_half_kernel<V, NDIM, kMetroGeneric, MIXED><<<grid, block, 0, st>>>(p);
        break;
    case kHeatGeneric:
        int8_half_kernel<V, NDIM, kHeatGeneric, MIXED><<<grid, block, 0, st>>>(p);
        break;
    default: int8_half_kernel<V, NDIM, kObserve, MIXED><<<grid, block, 0, st>>>(p); break;
    }
    return cudaGetLastError();
}

template <int V, bool MIXED = false>
static cudaError_t launch_v(int ndim, int rule, const Int8Half& p, dim3 grid, dim3 block,
                            cudaStream_t st)
{
    return ndim == 3 ? launch_rule<V, 3, MIXED>(rule, p, grid, block, st)
                     : launch_rule<V, 2, MIXED>(rule, p, grid, block, st);
}

// Chunk width used for a row of lh bytes: the widest of 16/8/4 that divides it.
int int8_chunk_width(int lh) { return lh % 16 == 0 ? 16 : (lh % 8 == 0 ? 8 : 4); }

// Launch geometry: x threads along a row (chunks), y rows per block, grid-stride over rows.
void int8_geometry(long long rows, int cpr, int max_blocks, dim3* grid, dim3* block)
{
    int bx = 1;
    while (bx < cpr && bx < 128) bx <<= 1;
    const int by = 256 / bx;
    const int gx = (cpr + bx - 1) / bx;
    long long gy = (rows + by - 1) / by;
    long long cap = max_blocks / gx;
    if (cap < 1) cap = 1;
    if (gy > cap) gy = cap;
    if (gy > 65535) gy = 65535;
    *grid = dim3((unsigned)gx, (unsigned)gy, 1);
    *block = dim3((unsigned)bx, (unsigned)by, 1);
}

cudaError_t launch_int8_half(int ndim, int rule, const Int8Half& p, int max_blocks,
                             cudaStream_t st)
{
    dim3 grid, block;
    int8_geometry(p.rows, p.cpr, max_blocks, &grid, &block);
    const int v = p.vw;
    if (v == 16) {  // padded rows (lh % 16 != 0) need the partial-chunk code
        return (p.lh % 16) ? launch_v<16, true>(ndim, rule, p, grid, block, st)
                           : launch_v<16, false>(ndim, rule, p, grid, block, st);
    }
    if (v == 8) return launch_v<8>(ndim, rule, p, grid, block, st);
    return launch_v<4>(ndim, rule, p, grid, block, st);
}

}  // namespace ising
