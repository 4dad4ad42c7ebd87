// Slab decomposition of one lattice over several devices (or several handles on one device).
//
// A slab handle owns a contiguous range [begin, begin + count) of the lattice's first axis: rows
// y of a 2D lattice, planes z of a 3D one.  Its colour arrays hold the owned rows plus one halo
// of the opposite side's neighbours on each side: one row (2D) or one plane of ly rows (3D),
//
//     [ low halo | owned rows 0 .. rows-1 | high halo ]     (rows `row_bytes` apart)
//
// A half-sweep of colour c reads only the opposite colour, so before it the caller copies the
// opposite colour's boundary rows of the neighbouring slabs into this slab's halos (periodic
// along the axis: the first slab's low halo is the last slab's last row or plane), over NCCL,
// a peer copy or a local copy: ising_slab_halo gives the device addresses of the halos and of
// the boundary rows to send.  The kernels never wrap along the slab axis: they read the halos.
// Random numbers use the global site index (the local row plus the slab's first global row) and
// the global row parity, so the slabs together are bit-identical to one handle holding the
// whole lattice (src/pyising/philox.py:54-78 keys every site by its index, not by who owns it).
// The (M, E) sums of a slab cover its owned sites; the lattice's are the sums over slabs.
#include <cstring>

#include "capi_internal.h"
#include "int8_core.cuh"
#include "msc_core.cuh"

struct ising_slab {
    int device = 0;
    int ndim = 2;
    int variant = ISING_VARIANT_INT8;
    int algorithm = ISING_METROPOLIS;
    int64_t shape[3] = {0, 0, 0};  // the whole lattice
    int64_t begin = 0, count = 0;  // owned range of the first axis
    long long rows = 0;            // owned rows: count (2D) or count * ly (3D)
    long long halo = 0;            // rows per halo: 1 (2D) or ly (3D)
    long long row0 = 0;            // global row index of owned row 0
    int lh = 0, ly = 0, lz = 1;    // ly, lz: the local extents the kernels walk
    int nw = 0, pitch = 0;
    size_t row_bytes = 0;          // device bytes per row: pitch (int8) or 8 nw (msc)
    size_t host_row = 0;           // host bytes per row: lh (int8) or 8 nw (msc)
    uint64_t seed = 0;
    uint32_t table[7] = {0, 0, 0, 0, 0, 0, 0};
    int table_n = 5;
    int rule = 0;
    void* base[2] = {nullptr, nullptr};  // halo + rows + halo rows per colour
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    unsigned long long* d_acc = nullptr;  // (M, E) of ising_slab_observables
    long long* d_series = nullptr;        // measured (M, E) pairs
    int64_t series_cap = 0;
    int sm_count = 148;
    int max_blocks = 148 * 8;
    int queue_blocks = 2;  // resident blocks per SM of the msc work-stack kernel
    int strip_blocks = 2;  // ... of the msc strip kernel
    // Neighbouring slabs whose edge rows the kernels read in place of this slab's halos
    // (ising_slab_set_peer), per colour; nullptr: the own halo rows.
    const char* peer_lo[2] = {nullptr, nullptr};
    const char* peer_hi[2] = {nullptr, nullptr};

    char* owned(int c) const { return static_cast<char*>(base[c]) + halo * row_bytes; }
    // Where the kernels read the rows before and after the owned ones, in colour c.
    const char* low_rows(int c) const { return peer_lo[c] ? peer_lo[c] : owned(c) - halo * row_bytes; }
    const char* high_rows(int c) const
    {
        return peer_hi[c] ? peer_hi[c] : owned(c) + rows * (long long)row_bytes;
    }
};

namespace ising {

struct SlabGeo {
    long long row0;  // global row of local row 0: the Philox site index is (row0 + row) * lh + j
    int par0;        // parity of the slab's first global y (2D) or z (3D)
    long long halo;  // rows before (and after) the owned ones that a half-sweep reads
    const void* lo;  // those rows of the opposite colour: rows -halo .. -1
    const void* hi;  // and rows `rows` .. rows + halo - 1
    int a0, an;      // the launch updates rows (2D) or planes (3D) a0 .. a0 + an - 1
};

// int8 half-sweep of a slab: the band schedule of int8_half_kernel, with the rows next to the
// slab (row -1 and row `rows` in 2D, planes -1 and lz in 3D) read from the halos instead of
// wrapping.  Rows are 16-byte chunks with the partial-chunk code for padded rows.
template <int NDIM, int RULE, bool MEAS>
__global__ void __launch_bounds__(256, 4) int8_slab_kernel(const Int8Half p_in, const SlabGeo g)
{
    constexpr int V = 16, W = 4;
    Int8Half p = p_in;
    __shared__ u32 stab[8];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) stab[i] = p.table[i];
    }
    pdl_wait();  // the previous kernel of the stream has completed
    pdl_trigger();
    __syncthreads();
    long long m_acc = 0, e_acc = 0;
    const u32 cpr = (u32)p.cpr, bpp = (u32)p.bpp;
    // bands over rows a0 .. a0 + an - 1 (2D) or over all rows of planes a0 .. a0 + an - 1 (3D)
    const u32 nslots = (u32)(NDIM == 3 ? g.an : 1) * bpp * cpr;
    const int ly = p.ly;
    const int ybase = NDIM == 2 ? g.a0 : 0, yend = NDIM == 2 ? g.a0 + g.an : ly;
    for (u32 slot = blockIdx.x * blockDim.x + threadIdx.x; slot < nslots;
         slot += gridDim.x * blockDim.x) {
        const u32 band = fast_div(slot, cpr, p.cpr_magic);
        const int j0 = (int)(slot - band * cpr) * V;
        int z = 0, yb = (int)band;
        if constexpr (NDIM == 3) {
            const int zs = (int)fast_div(band, bpp, p.bpp_magic);
            yb = (int)(band - (u32)zs * bpp);
            z = g.a0 + zs;
        }
        const int y0 = ybase + yb * p.band;
        const int y1 = y0 + p.band < yend ? y0 + p.band : yend;
        const int wv = valid_words<true, W>(p, j0);
        const long long plane = (long long)z * ly;
        const int8_t* oth = p.other + j0;
        const int8_t* lo = static_cast<const int8_t*>(g.lo) + j0;
        const int8_t* hi = static_cast<const int8_t*>(g.hi) + j0;
        // opposite-colour row r: rows -halo .. -1 from lo, rows .. rows + halo - 1 from hi
        auto orow = [&](long long r) -> const int8_t* {
            return r < 0 ? lo + (r + g.halo) * p.pitch
                         : (r >= p.rows ? hi + (r - p.rows) * p.pitch : oth + r * p.pitch);
        };
        // 2D: y is the slab axis, rows -1 and ly are halo rows; 3D: y wraps inside its plane
        const long long yprev = NDIM == 2 ? y0 - 1 : (y0 == 0 ? ly - 1 : y0 - 1);
        Words<W> nd = load_words_ro<W>(orow(plane + yprev));
        Words<W> c = load_words_ro<W>(oth + (plane + y0) * p.pitch);
        for (int y = y0; y < y1; ++y) {
            const long long row = plane + y;
            const long long ynext = NDIM == 2 ? y + 1 : (y + 1 == ly ? 0 : y + 1);
            const Words<W> nu = load_words_ro<W>(orow(plane + ynext));
            Words<W> zu = nu, zd = nd;
            if constexpr (NDIM == 3) {  // planes z +- 1: plane -1 and plane lz are the halos
                zu = load_words_ro<W>(orow(row + ly));
                zd = load_words_ro<W>(orow(row - ly));
            }
            const int par = (g.par0 + y + z + (int)p.color) & 1;
            const u32 edge =
                (u32)(uint8_t)__ldg(p.other + row * p.pitch + edge_index(p, par, j0, wv));
            const Words<W> s = load_words<W>(p.own + row * p.pitch + j0);
            const Words<W> ns = int8_update<V, NDIM, RULE, true, MEAS, false>(
                p, g.row0 + row, par, j0, wv, s, c, nu, nd, zu, zd, edge, stab, m_acc, e_acc);
            if constexpr (RULE != kObserve) store_words<W>(p.own + row * p.pitch + j0, ns);
            nd = c;
            c = nu;
        }
    }
    if constexpr (MEAS) block_accumulate2(m_acc, e_acc, p.meas);
}

// msc half-sweep of a 2D slab, one word per thread; rows -1 and `rows` are the halo rows.
template <bool UPDATE, bool MEAS>
__global__ void __launch_bounds__(256) msc_slab_kernel(const MscHalf p, const SlabGeo g)
{
    pdl_wait();
    pdl_trigger();
    long long m_acc = 0, e_acc = 0;
    const int nw = p.nw;
    const long long w_end = (long long)(g.a0 + g.an) * nw;
    for (long long w = (long long)g.a0 * nw + blockIdx.x * (long long)blockDim.x + threadIdx.x;
         w < w_end; w += (long long)gridDim.x * blockDim.x) {
        const long long y = w / nw;
        const int x = (int)(w - y * nw);
        const long long rb = y * nw;
        const u64* orow = p.other + rb;
        const u64 o = p.own[rb + x];
        const u64 c = __ldg(orow + x);
        u64 hz;
        if ((g.par0 + (int)(y & 1) + (int)p.color) & 1)
            hz = (c >> 1) | (__ldg(orow + (x + 1 == nw ? 0 : x + 1)) << 63);
        else hz = (c << 1) | (__ldg(orow + (x == 0 ? nw - 1 : x - 1)) >> 63);
        const u64 up = __ldg((y == 0 ? static_cast<const u64*>(g.lo) : orow - nw) + x);
        const u64 dn = __ldg((y + 1 == p.rows ? static_cast<const u64*>(g.hi) : orow + nw) + x);
        u64 ns = o;
        if constexpr (UPDATE) {
            const Slices s = slice4(o, c, hz, up, dn);
            int calls = 0;
            ns = o ^ msc_flip(s, (u32)((g.row0 + y) * nw + x), p.t, p.color, p.k0, p.k1, p.thr4,
                              p.thr8, calls);
            p.own[rb + x] = ns;
        }
        if constexpr (MEAS) {
            const int anti =
                __popcll(ns ^ c) + __popcll(ns ^ hz) + __popcll(ns ^ up) + __popcll(ns ^ dn);
            m_acc += 2 * (__popcll(ns) + __popcll(c)) - 128;
            e_acc += 2 * anti - 256;
        }
    }
    if constexpr (MEAS) block_accumulate2(m_acc, e_acc, p.meas);
}

// Unmeasured msc half-sweep of a slab on the work stack of msc_half_queue_kernel: each warp walks
// a contiguous range of the slab's words, with global Philox word indices and halo rows.
constexpr int kSlabQueueWarps = 8;

__global__ void __launch_bounds__(kSlabQueueWarps * 32)
    msc_slab_queue_kernel(const MscHalf p, const SlabOffset so, long long first,
                          long long total, long long per_warp, int nw_shift)
{
    __shared__ QueueSlots q_all[kSlabQueueWarps];
    __shared__ uint4 lvmask[16];
    if (threadIdx.x < 16) lvmask[threadIdx.x] = level_masks(p.thr4, p.thr8, threadIdx.x);
    pdl_wait();
    pdl_trigger();
    __syncthreads();
    const long long begin =
        ((long long)blockIdx.x * kSlabQueueWarps + (threadIdx.x >> 5)) * per_warp;
    const long long end = begin + per_warp < total ? begin + per_warp : total;
    msc_queue_range<true>(p, first + begin, first + end, nw_shift, q_all[threadIdx.x >> 5],
                          lvmask, so);
}

// Words a0 * nw .. (a0 + an) * nw - 1 (rows a0 .. a0 + an - 1).
static cudaError_t launch_msc_slab_queue(const MscHalf& p, const SlabOffset& so, int a0, int an,
                                         int sm_count, int blocks_per_sm, cudaStream_t st)
{
    const long long total = (long long)an * p.nw;
    const long long warps = (long long)sm_count * blocks_per_sm * kSlabQueueWarps;
    long long per_warp = (total + warps - 1) / warps;
    per_warp = (per_warp + 31) / 32 * 32;
    const long long nwarps = (total + per_warp - 1) / per_warp;
    const unsigned blocks = (unsigned)((nwarps + kSlabQueueWarps - 1) / kSlabQueueWarps);
    const int shift = (p.nw & (p.nw - 1)) == 0 ? __builtin_ctz((unsigned)p.nw) : -1;
    return launch_pdl(msc_slab_queue_kernel, dim3(blocks), dim3(kSlabQueueWarps * 32), st, p, so,
                      (long long)a0 * p.nw, total, per_warp, shift);
}

// Unmeasured msc half-sweep of a slab on the strip schedule of msc_strip_kernel (rows holding
// whole 32-word strips): warp g walks rows a0 + band (g / strips) .. of strip g % strips, two
// rows per step, with global Philox word indices and the slab's halo rows.
constexpr int kSlabStripWarps = 8;

__global__ void __launch_bounds__(kSlabStripWarps * 32, 2)
    msc_slab_strip_kernel(const MscHalf p, const SlabOffset so, int a0, int an, int strips,
                          int band)
{
    __shared__ StripSlots q_all[kSlabStripWarps];
    __shared__ uint4 lvmask[16];
    if (threadIdx.x < 16) lvmask[threadIdx.x] = level_masks(p.thr4, p.thr8, threadIdx.x);
    pdl_wait();
    pdl_trigger();
    __syncthreads();
    const int g = blockIdx.x * kSlabStripWarps + (threadIdx.x >> 5);
    const int y0 = a0 + (g / strips) * band;
    const int y1 = min(y0 + band, a0 + an);
    if (y0 < a0 + an)
        msc_strip_band<4, true>(p, g % strips, y0, y1, q_all[threadIdx.x >> 5], lvmask, so);
}

// Rows a0 .. a0 + an - 1 on the strip schedule, bands sized for one wave of resident warps.
static cudaError_t launch_msc_slab_strip(const MscHalf& p, const SlabOffset& so, int a0, int an,
                                         int sm_count, int blocks_per_sm, cudaStream_t st)
{
    const int strips = p.nw / 32;
    const long long units = (long long)an * strips;
    const long long warps = (long long)sm_count * blocks_per_sm * kSlabStripWarps;
    long long band = (units + warps - 1) / warps;
    if (band < 1) band = 1;
    const long long nwarps = (long long)strips * ((an + band - 1) / band);
    const unsigned blocks = (unsigned)((nwarps + kSlabStripWarps - 1) / kSlabStripWarps);
    return launch_pdl(msc_slab_strip_kernel, dim3(blocks), dim3(kSlabStripWarps * 32), st, p, so,
                      a0, an, strips, (int)band);
}

// The device seeded start of ising_fill_philox at global site indices.
__global__ void slab_philox_int8_kernel(int8_t* c0, int8_t* c1, long long rows, long long row0,
                                        int lh, int pitch, u32 k0, u32 k1)
{
    const int qpr = lh / 4;
    const long long quads = rows * qpr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * quads;
         i += (long long)gridDim.x * blockDim.x) {
        const u32 color = (u32)(i / quads);
        const long long qi = i - (long long)color * quads;
        const long long row = qi / qpr;
        const int q = (int)(qi - row * qpr);
        const long long n = (row0 + row) * lh + 4LL * q;
        const u32x4 r = philox4x32_10((u32)(n >> 7), 0u, color, 0xFFFFFFFFu, k0, k1);
        const int word = (int)((n >> 5) & 3);
        const u32 rw = word == 0 ? r.x : (word == 1 ? r.y : (word == 2 ? r.z : r.w));
        const u32 nib = (rw >> (n & 31)) & 0xFu;
        const u32 ones = (nib * 0x00204081u) & 0x01010101u;
        *reinterpret_cast<u32*>((color ? c1 : c0) + row * pitch + 4 * q) =
            0xFFFFFFFFu ^ (ones * 0xFEu);
    }
}

__global__ void slab_philox_msc_kernel(u64* w0, u64* w1, long long rows, long long row0, int nw,
                                       u32 k0, u32 k1)
{
    const long long words = rows * nw;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * words;
         i += (long long)gridDim.x * blockDim.x) {
        const u32 color = (u32)(i / words);
        const long long wl = i - (long long)color * words;
        const long long wg = row0 * nw + wl;  // global word index
        const u32x4 r = philox4x32_10((u32)(wg >> 1), 0u, color, 0xFFFFFFFFu, k0, k1);
        (color ? w1 : w0)[wl] =
            (wg & 1) ? ((u64)r.z | ((u64)r.w << 32)) : ((u64)r.x | ((u64)r.y << 32));
    }
}

static unsigned slab_grid(long long work, int max_blocks)
{
    long long g = (work + 255) / 256;
    if (g > max_blocks) g = max_blocks;
    return (unsigned)(g < 1 ? 1 : g);
}

template <int NDIM, bool MEAS>
static void launch_int8_slab_rule(int rule, const Int8Half& p, const SlabGeo& g, unsigned grid,
                                  cudaStream_t st)
{
    auto go = [&](auto kernel) { launch_pdl(kernel, dim3(grid), dim3(256), st, p, g); };
    switch (rule) {
    case kMetroFast: go(int8_slab_kernel<NDIM, kMetroFast, MEAS>); break;
    case kHeatFast: go(int8_slab_kernel<NDIM, kHeatFast, MEAS>); break;
    case kMetroGeneric: go(int8_slab_kernel<NDIM, kMetroGeneric, MEAS>); break;
    case kHeatGeneric: go(int8_slab_kernel<NDIM, kHeatGeneric, MEAS>); break;
    default: go(int8_slab_kernel<NDIM, kObserve, true>); break;
    }
}

// One half-sweep of colour `color` (rule kObserve: measurement of colour `color` only) over
// rows (2D) or planes (3D) a0 .. a0 + an - 1 of the slab.
static int slab_half(ising_slab* s, int color, u32 t, int rule, unsigned long long* meas, int a0,
                     int an)
{
    const SlabGeo g{s->row0, (int)(s->begin & 1), s->halo, s->low_rows(1 - color),
                    s->high_rows(1 - color), a0, an};
    if (s->variant == ISING_VARIANT_MSC) {
        MscHalf p;
        memset(&p, 0, sizeof p);
        p.own = reinterpret_cast<u64*>(s->owned(color));
        p.other = reinterpret_cast<const u64*>(s->owned(1 - color));
        p.rows = (int)s->rows;
        p.nw = s->nw;
        p.t = t;
        p.color = (u32)color;
        p.k0 = (u32)s->seed;
        p.k1 = (u32)(s->seed >> 32);
        p.thr4 = s->table[3];
        p.thr8 = s->table[4];
        p.meas = meas;
        p.nw_magic = magic_for(s->nw);
        if (rule != kObserve && !meas) {
            const SlabOffset so{s->row0 * s->nw, (int)(s->begin & 1),
                                reinterpret_cast<const u64*>(s->low_rows(1 - color)),
                                reinterpret_cast<const u64*>(s->high_rows(1 - color))};
            // strips where the rows hold whole 32-word strips (as for whole lattices)
            const bool strips = s->nw % 32 == 0 && s->rows * s->nw <= 0xFFFFFFFFll;
            const cudaError_t e =
                strips ? launch_msc_slab_strip(p, so, a0, an, s->sm_count, s->strip_blocks,
                                               s->stream)
                       : launch_msc_slab_queue(p, so, a0, an, s->sm_count, s->queue_blocks,
                                               s->stream);
            return e == cudaSuccess ? ISING_OK : cuda_fail(e, "slab half-sweep launch");
        }
        const unsigned grid = slab_grid((long long)an * s->nw, s->max_blocks);
        auto go = [&](auto kernel) { launch_pdl(kernel, dim3(grid), dim3(256), s->stream, p, g); };
        if (rule == kObserve) go(msc_slab_kernel<false, true>);
        else if (meas) go(msc_slab_kernel<true, true>);
        else go(msc_slab_kernel<true, false>);
    } else {
        Int8Half p;
        memset(&p, 0, sizeof p);
        p.own = reinterpret_cast<int8_t*>(s->owned(color));
        p.other = reinterpret_cast<const int8_t*>(s->owned(1 - color));
        p.rows = s->rows;
        p.lh = s->lh;
        p.ly = s->ly;
        p.lz = s->lz;
        p.pitch = s->pitch;
        p.vw = 16;
        p.cpr = (s->lh + 15) / 16;
        p.t = t;
        p.color = (u32)color;
        p.k0 = (u32)s->seed;
        p.k1 = (u32)(s->seed >> 32);
        for (int i = 0; i < 7; ++i) p.table[i] = s->table[i];
        p.meas = meas;
        // band geometry of the updated range; the kernel keeps the slab's own extents
        Int8Half q = p;
        if (s->ndim == 2) q.ly = an;
        else q.lz = an;
        q.rows = (long long)q.ly * q.lz;
        const unsigned grid = int8_band_geometry(q, s->max_blocks, s->sm_count);
        p.band = q.band;
        p.bpp = q.bpp;
        p.cpr_magic = q.cpr_magic;
        p.bpp_magic = q.bpp_magic;
        const bool m = meas != nullptr;
        if (s->ndim == 3) {
            if (m) launch_int8_slab_rule<3, true>(rule, p, g, grid, s->stream);
            else launch_int8_slab_rule<3, false>(rule, p, g, grid, s->stream);
        } else {
            if (m) launch_int8_slab_rule<2, true>(rule, p, g, grid, s->stream);
            else launch_int8_slab_rule<2, false>(rule, p, g, grid, s->stream);
        }
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ISING_OK : cuda_fail(e, "slab half-sweep launch");
}

}  // namespace ising

using namespace ising;

#define SLAB_TRY(call)                                       \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
    } while (0)

#define SLAB_CHECK(s)                                                   \
    do {                                                                \
        if (!(s)) return fail(ISING_ERR_INVALID, "null slab handle");  \
    } while (0)

extern "C" {

int ising_slab_create(int ndim, const int64_t* shape, int variant, int algorithm, uint64_t seed,
                      int64_t begin, int64_t count, int device, ising_slab** out)
{
    if (!out || !shape) return fail(ISING_ERR_INVALID, "null pointer argument");
    *out = nullptr;
    if (ndim != 2 && ndim != 3)
        return fail(ISING_ERR_INVALID, "only 2D and 3D lattices are supported, got ndim=%d", ndim);
    for (int i = 0; i < ndim; ++i)
        if (shape[i] < 2 || shape[i] % 2)
            return fail(ISING_ERR_INVALID, "all extents must be even and >= 2");
    if (variant != ISING_VARIANT_INT8 && variant != ISING_VARIANT_MSC)
        return fail(ISING_ERR_INVALID, "unknown variant %d", variant);
    if (algorithm != ISING_METROPOLIS && algorithm != ISING_HEATBATH)
        return fail(ISING_ERR_INVALID, "unknown algorithm %d", algorithm);
    const int64_t lx = shape[ndim - 1];
    const int multiple = variant == ISING_VARIANT_MSC ? 128 : 8;
    if (lx % multiple)
        return fail(ISING_ERR_INVALID, "last extent must be a multiple of %d, got %lld", multiple,
                    (long long)lx);
    if (variant == ISING_VARIANT_MSC && (ndim != 2 || algorithm != ISING_METROPOLIS))
        return fail(ISING_ERR_INVALID, "msc supports 2D Metropolis only");
    const int64_t ly = shape[ndim - 2];
    const int64_t lz = ndim == 3 ? shape[0] : 1;
    if (ly * lz > (int64_t)0x7FFFFFFF || lx / 2 > (int64_t)0x7FFFFFFF)
        return fail(ISING_ERR_INVALID, "lattice too large for 32-bit row indices");
    if (count < 1 || begin < 0 || begin + count > shape[0])
        return fail(ISING_ERR_INVALID, "slab [%lld, %lld) outside the first axis (extent %lld)",
                    (long long)begin, (long long)(begin + count), (long long)shape[0]);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(ISING_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev)
        return fail(ISING_ERR_INVALID, "device %d out of range (%d devices)", device, ndev);
    SLAB_TRY(cudaSetDevice(device));

    ising_slab* s = new ising_slab();
    s->device = device;
    s->ndim = ndim;
    s->variant = variant;
    s->algorithm = algorithm;
    for (int i = 0; i < 3; ++i) s->shape[i] = i < ndim ? shape[i] : 0;
    s->begin = begin;
    s->count = count;
    s->lh = (int)(lx / 2);
    s->nw = (int)(lx / 128);
    s->pitch = (s->lh + 15) / 16 * 16;
    if (ndim == 2) {
        s->ly = (int)count;  // the kernels walk the owned rows as one plane
        s->lz = 1;
        s->halo = 1;
        s->row0 = begin;
    } else {
        s->ly = (int)ly;
        s->lz = (int)count;
        s->halo = ly;
        s->row0 = begin * ly;
    }
    s->rows = (long long)s->ly * s->lz;
    s->row_bytes = variant == ISING_VARIANT_MSC ? (size_t)s->nw * 8 : (size_t)s->pitch;
    s->host_row = variant == ISING_VARIANT_MSC ? (size_t)s->nw * 8 : (size_t)s->lh;
    s->seed = seed;
    s->table_n = 2 * ndim + 1;
    for (int i = 0; i < 7; ++i) s->table[i] = 0xFFFFFFFFu;
    s->rule = select_rule(variant, algorithm, ndim, s->table);
    s->sm_count = device_sm_count(device);
    s->max_blocks = s->sm_count * 8;
    {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, msc_slab_queue_kernel,
                                                          kSlabQueueWarps * 32, 0) == cudaSuccess &&
            b > 0)
            s->queue_blocks = b;
        cudaGetLastError();
        b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, msc_slab_strip_kernel,
                                                          kSlabStripWarps * 32, 0) == cudaSuccess &&
            b > 0)
            s->strip_blocks = b;
        cudaGetLastError();
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    s->stream = s->own_stream;
    const size_t bytes = (size_t)(s->rows + 2 * s->halo) * s->row_bytes;
    for (int c = 0; c < 2; ++c) {
        e = cudaMalloc(&s->base[c], bytes);
        if (e == cudaSuccess) e = cudaMemset(s->base[c], 0, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ising_slab_destroy(s);
            return fail(ISING_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", bytes,
                        cudaGetErrorString(e));
        }
    }
    e = cudaMalloc(&s->d_acc, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaGetLastError();
        ising_slab_destroy(s);
        return fail(ISING_ERR_NOMEM, "cudaMalloc of the accumulators failed");
    }
    *out = s;
    return ISING_OK;
}

int ising_slab_destroy(ising_slab* s)
{
    if (!s) return ISING_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int c = 0; c < 2; ++c)
        if (s->base[c]) cudaFree(s->base[c]);
    if (s->d_acc) cudaFree(s->d_acc);
    if (s->d_series) cudaFree(s->d_series);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    cudaGetLastError();
    delete s;
    return ISING_OK;
}

int ising_slab_set_stream(ising_slab* s, void* stream)
{
    SLAB_CHECK(s);
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    return ISING_OK;
}

int ising_slab_set_table(ising_slab* s, const uint32_t* table, int n)
{
    SLAB_CHECK(s);
    if (!table) return fail(ISING_ERR_INVALID, "null table");
    if (n != s->table_n)
        return fail(ISING_ERR_INVALID, "table must have %d entries, got %d", s->table_n, n);
    for (int i = 0; i < 7; ++i) s->table[i] = i < n ? table[i] : 0xFFFFFFFFu;
    s->rule = select_rule(s->variant, s->algorithm, s->ndim, s->table);
    return ISING_OK;
}

int ising_slab_upload(ising_slab* s, const void* c0, const void* c1)
{
    SLAB_CHECK(s);
    if (!c0 || !c1) return fail(ISING_ERR_INVALID, "null colour array");
    SLAB_TRY(cudaSetDevice(s->device));
    const void* src[2] = {c0, c1};
    for (int c = 0; c < 2; ++c)
        SLAB_TRY(cudaMemcpy2DAsync(s->owned(c), s->row_bytes, src[c], s->host_row, s->host_row,
                                   (size_t)s->rows, cudaMemcpyHostToDevice, s->stream));
    SLAB_TRY(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

int ising_slab_download(ising_slab* s, void* c0, void* c1)
{
    SLAB_CHECK(s);
    if (!c0 || !c1) return fail(ISING_ERR_INVALID, "null colour array");
    SLAB_TRY(cudaSetDevice(s->device));
    void* dst[2] = {c0, c1};
    for (int c = 0; c < 2; ++c)
        SLAB_TRY(cudaMemcpy2DAsync(dst[c], s->host_row, s->owned(c), s->row_bytes, s->host_row,
                                   (size_t)s->rows, cudaMemcpyDeviceToHost, s->stream));
    SLAB_TRY(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

int ising_slab_fill_cold(ising_slab* s)
{
    SLAB_CHECK(s);
    SLAB_TRY(cudaSetDevice(s->device));
    const int v = s->variant == ISING_VARIANT_MSC ? 0xFF : 0x01;
    const size_t bytes = (size_t)(s->rows + 2 * s->halo) * s->row_bytes;
    for (int c = 0; c < 2; ++c) SLAB_TRY(cudaMemsetAsync(s->base[c], v, bytes, s->stream));
    return ISING_OK;
}

int ising_slab_fill_philox(ising_slab* s, uint64_t start_seed)
{
    SLAB_CHECK(s);
    SLAB_TRY(cudaSetDevice(s->device));
    const u32 k0 = (u32)start_seed, k1 = (u32)(start_seed >> 32);
    if (s->variant == ISING_VARIANT_MSC) {
        slab_philox_msc_kernel<<<slab_grid(2 * s->rows * s->nw, s->max_blocks), 256, 0,
                                 s->stream>>>(reinterpret_cast<u64*>(s->owned(0)),
                                              reinterpret_cast<u64*>(s->owned(1)), s->rows,
                                              s->row0, s->nw, k0, k1);
    } else {
        slab_philox_int8_kernel<<<slab_grid(2 * s->rows * (s->lh / 4), s->max_blocks), 256, 0,
                                  s->stream>>>(reinterpret_cast<int8_t*>(s->owned(0)),
                                               reinterpret_cast<int8_t*>(s->owned(1)), s->rows,
                                               s->row0, s->lh, s->pitch, k0, k1);
    }
    SLAB_TRY(cudaGetLastError());
    return ISING_OK;
}

int ising_slab_halo(ising_slab* s, int color, int which, void** ptr, int64_t* bytes)
{
    SLAB_CHECK(s);
    if (!ptr || !bytes) return fail(ISING_ERR_INVALID, "null output pointer");
    if (color != 0 && color != 1) return fail(ISING_ERR_INVALID, "colour must be 0 or 1");
    char* own = s->owned(color);
    const long long hb = s->halo * (long long)s->row_bytes;
    switch (which) {
    case ISING_SLAB_HALO_LOW: *ptr = own - hb; break;
    case ISING_SLAB_HALO_HIGH: *ptr = own + s->rows * (long long)s->row_bytes; break;
    case ISING_SLAB_EDGE_LOW: *ptr = own; break;
    case ISING_SLAB_EDGE_HIGH: *ptr = own + (s->rows - s->halo) * (long long)s->row_bytes; break;
    default: return fail(ISING_ERR_INVALID, "unknown halo selector %d", which);
    }
    *bytes = hb;
    return ISING_OK;
}

int ising_slab_set_peer(ising_slab* s, int side, ising_slab* n)
{
    SLAB_CHECK(s);
    if (side != 0 && side != 1) return fail(ISING_ERR_INVALID, "side must be 0 (low) or 1 (high)");
    if (!n) {
        for (int c = 0; c < 2; ++c) (side ? s->peer_hi : s->peer_lo)[c] = nullptr;
        return ISING_OK;
    }
    bool same = n->variant == s->variant && n->ndim == s->ndim && n->row_bytes == s->row_bytes &&
                n->halo == s->halo && n->lh == s->lh;
    for (int i = 0; i < 3; ++i) same = same && n->shape[i] == s->shape[i];
    if (!same) return fail(ISING_ERR_INVALID, "peer slab of a different lattice");
    const int64_t extent = s->shape[0];
    const bool adjacent = side == 0 ? (n->begin + n->count) % extent == s->begin
                                    : (s->begin + s->count) % extent == n->begin;
    if (!adjacent)
        return fail(ISING_ERR_INVALID, "peer slab [%lld, %lld) is not the %s neighbour of [%lld, %lld)",
                    (long long)n->begin, (long long)(n->begin + n->count), side ? "high" : "low",
                    (long long)s->begin, (long long)(s->begin + s->count));
    if (n->device != s->device) {
        int can = 0;
        SLAB_TRY(cudaDeviceCanAccessPeer(&can, s->device, n->device));
        if (!can)
            return fail(ISING_ERR_INVALID, "device %d cannot read device %d's memory", s->device,
                        n->device);
        SLAB_TRY(cudaSetDevice(s->device));
        const cudaError_t e = cudaDeviceEnablePeerAccess(n->device, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
        else if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceEnablePeerAccess");
    }
    for (int c = 0; c < 2; ++c) {
        if (side == 0) s->peer_lo[c] = n->owned(c) + (n->rows - n->halo) * (long long)n->row_bytes;
        else s->peer_hi[c] = n->owned(c);
    }
    return ISING_OK;
}

int ising_slab_series_reset(ising_slab* s, int64_t pairs)
{
    SLAB_CHECK(s);
    if (pairs < 0) return fail(ISING_ERR_INVALID, "negative series length");
    SLAB_TRY(cudaSetDevice(s->device));
    if (pairs > s->series_cap) {
        if (s->d_series) {
            SLAB_TRY(cudaStreamSynchronize(s->stream));
            cudaFree(s->d_series);
            s->d_series = nullptr;
            s->series_cap = 0;
        }
        cudaError_t e = cudaMalloc((void**)&s->d_series, (size_t)pairs * 2 * sizeof(long long));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(ISING_ERR_NOMEM, "cudaMalloc of a series of %lld pairs", (long long)pairs);
        }
        s->series_cap = pairs;
    }
    if (pairs > 0)
        SLAB_TRY(cudaMemsetAsync(s->d_series, 0, (size_t)pairs * 2 * sizeof(long long), s->stream));
    return ISING_OK;
}

int ising_slab_half_sweep_rows(ising_slab* s, int color, uint64_t t, int64_t slot,
                               int64_t first, int64_t count)
{
    SLAB_CHECK(s);
    if (color != 0 && color != 1) return fail(ISING_ERR_INVALID, "colour must be 0 or 1");
    if (slot >= s->series_cap)
        return fail(ISING_ERR_INVALID, "series slot %lld beyond the %lld reset pairs",
                    (long long)slot, (long long)s->series_cap);
    if (first < 0 || count < 0 || first + count > s->count)
        return fail(ISING_ERR_INVALID, "rows [%lld, %lld) outside the slab's %lld",
                    (long long)first, (long long)(first + count), (long long)s->count);
    if (count == 0) return ISING_OK;
    SLAB_TRY(cudaSetDevice(s->device));
    unsigned long long* m =
        slot >= 0 ? reinterpret_cast<unsigned long long*>(s->d_series + 2 * slot) : nullptr;
    return slab_half(s, color, (u32)t, s->rule, m, (int)first, (int)count);
}

int ising_slab_half_sweep(ising_slab* s, int color, uint64_t t, int64_t slot)
{
    SLAB_CHECK(s);
    return ising_slab_half_sweep_rows(s, color, t, slot, 0, s->count);
}

int ising_slab_series_read(ising_slab* s, int64_t pairs, int64_t* out)
{
    SLAB_CHECK(s);
    if (pairs < 0 || pairs > s->series_cap)
        return fail(ISING_ERR_INVALID, "series of %lld pairs, %lld reset", (long long)pairs,
                    (long long)s->series_cap);
    if (pairs > 0 && !out) return fail(ISING_ERR_INVALID, "null output pointer");
    SLAB_TRY(cudaSetDevice(s->device));
    if (pairs > 0)
        SLAB_TRY(cudaMemcpyAsync(out, s->d_series, (size_t)pairs * 2 * sizeof(long long),
                                 cudaMemcpyDeviceToHost, s->stream));
    SLAB_TRY(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

int ising_slab_observables(ising_slab* s, int64_t* m, int64_t* e)
{
    SLAB_CHECK(s);
    if (!m || !e) return fail(ISING_ERR_INVALID, "null output pointer");
    SLAB_TRY(cudaSetDevice(s->device));
    SLAB_TRY(cudaMemsetAsync(s->d_acc, 0, 2 * sizeof(unsigned long long), s->stream));
    const int rc = slab_half(s, 1, 0u, kObserve, s->d_acc, 0, (int)s->count);
    if (rc != ISING_OK) return rc;
    long long out[2];
    SLAB_TRY(cudaMemcpyAsync(out, s->d_acc, sizeof out, cudaMemcpyDeviceToHost, s->stream));
    SLAB_TRY(cudaStreamSynchronize(s->stream));
    *m = out[0];
    *e = out[1];
    return ISING_OK;
}

int ising_slab_sync(ising_slab* s)
{
    SLAB_CHECK(s);
    SLAB_TRY(cudaSetDevice(s->device));
    SLAB_TRY(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

}  // extern "C"
