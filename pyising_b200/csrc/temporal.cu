// Temporally blocked int8 2D half-sweeps: two sweeps (four half-sweeps) per launch.
//
// A small lattice's half-sweep is a few microseconds of work, about as long as a launch, even
// with graphs and programmatic dependent launch.  Here one launch does kTbSteps half-sweeps: a
// CTA loads a band of kTbBand rows plus kTbSteps halo rows on each side (periodic in y) of both
// colours into shared memory, runs the half-sweeps there on a row range that shrinks by one
// row per half-sweep (half-sweep k updates tile rows [k+1, rows-1-k): exactly what the band's
// rows need after the last one, since each half-sweep reads the opposite colour one row
// further out), and writes back only the band.  Halo rows are updated by two CTAs with the
// same random numbers, keyed by (site, sweep, colour) as everywhere else, so every result is
// bit-identical to four single half-sweeps.
//
// Conditions (temporal_ok): int8 2D, a fast decision rule, rows a multiple of 16 bytes (no
// padding, whole 16-byte chunks), Ly a multiple of kTbBand and at least kTbRows (no row twice
// in a tile), the tile within the shared memory of a CTA.  Unmeasured sweeps only: measured
// ones run the single half-sweep kernels.
#include "capi_internal.h"
#include "int8_core.cuh"

namespace ising {

#ifndef ISING_TB_BAND
#define ISING_TB_BAND 8
#endif
constexpr int kTbBand = ISING_TB_BAND;           // rows a CTA writes back
#ifndef ISING_TB_STEPS
#define ISING_TB_STEPS 4
#endif
constexpr int kTbSteps = ISING_TB_STEPS;         // half-sweeps per launch (even: whole sweeps)
static_assert(kTbSteps % 2 == 0, "whole sweeps per launch");
constexpr int kTbRows = kTbBand + 2 * kTbSteps;  // tile rows per colour
constexpr int kTbMaxSmem = 96 * 1024;
#ifndef ISING_TB_THREADS
#define ISING_TB_THREADS 1024
#endif
constexpr int kTbThreads = ISING_TB_THREADS;  // 32 warps (512 and 1024 measured alike)

#ifndef ISING_TB_CHUNK
#define ISING_TB_CHUNK 16
#endif
// Bytes a thread updates per tile step (4 sites per 32-bit word); 16 measured best of 4/8/16
// (1024^2: 315 / 309 / 256 flips/ns for 16 / 8 / 4).
constexpr int kTbChunk = ISING_TB_CHUNK;

template <int V>
__device__ __forceinline__ Words<V / 4> lds_words(const int8_t* p)
{
    Words<V / 4> r;
    if constexpr (V == 16) {
        const uint4 q = *reinterpret_cast<const uint4*>(p);
        r.v[0] = q.x;
        r.v[1] = q.y;
        r.v[2] = q.z;
        r.v[3] = q.w;
    } else if constexpr (V == 8) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        r.v[0] = q.x;
        r.v[1] = q.y;
    } else {
        r.v[0] = *reinterpret_cast<const u32*>(p);
    }
    return r;
}

template <int V>
__device__ __forceinline__ void sts_words(int8_t* p, const Words<V / 4>& w)
{
    if constexpr (V == 16) *reinterpret_cast<uint4*>(p) = make_uint4(w.v[0], w.v[1], w.v[2], w.v[3]);
    else if constexpr (V == 8) *reinterpret_cast<uint2*>(p) = make_uint2(w.v[0], w.v[1]);
    else *reinterpret_cast<u32*>(p) = w.v[0];
}

// Reads both colours from in0/in1 and writes the band to out0/out1: separate arrays, since a
// CTA's halo rows are other CTAs' bands, which those write back in the same launch.
template <int RULE>
__global__ void __launch_bounds__(kTbThreads) int8_temporal_kernel(const Int8Half p_in,
                                                           const int8_t* in0, const int8_t* in1,
                                                           int8_t* out0, int8_t* out1)
{
    constexpr int V = kTbChunk;
    extern __shared__ __align__(16) int8_t tile[];  // [colour][kTbRows][lh]
    __shared__ u32 stab[8];
    Int8Half p = p_in;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) stab[i] = p.table[i];
    }
    pdl_wait();  // the previous launch of the stream has completed
    pdl_trigger();
    resolve_ctl(p);  // p.t: the sweep of the first half-sweep (colour 0)
    const int lh = p.lh, ly = p.ly, cpr = lh >> 4;
    const int r0 = blockIdx.x * kTbBand;
    const int chunks = kTbRows * cpr;
    for (int i = threadIdx.x; i < 2 * chunks; i += blockDim.x) {
        const int c = i >= chunks;
        const int rem = i - c * chunks;
        const int tr = rem / cpr, jc = rem - tr * cpr;
        int gr = r0 - kTbSteps + tr;
        gr = gr < 0 ? gr + ly : (gr >= ly ? gr - ly : gr);
        const int8_t* src = (c ? in1 : in0) + (long long)gr * p.pitch + 16 * jc;
        *reinterpret_cast<uint4*>(tile + (c * kTbRows + tr) * lh + 16 * jc) =
            __ldcg(reinterpret_cast<const uint4*>(src));
    }
    __syncthreads();
    long long m_acc = 0, e_acc = 0;  // unused (no measurement here)
#pragma unroll 1
    for (int k = 0; k < kTbSteps; ++k) {
        const int color = k & 1;
        Int8Half q = p;
        q.t = p.t + (u32)(k >> 1);
        q.color = (u32)color;
        int8_t* own = tile + color * kTbRows * lh;
        const int8_t* oth = tile + (color ^ 1) * kTbRows * lh;
        const int vpr = lh / V;  // chunks per row at this step's width
        const int lo = k + 1, n = (kTbRows - 2 - 2 * k) * vpr;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int tr = lo + i / vpr, jc = i - (i / vpr) * vpr, j0 = V * jc;
            int gr = r0 - kTbSteps + tr;
            gr = gr < 0 ? gr + ly : (gr >= ly ? gr - ly : gr);
            const int par = (gr + color) & 1;
            const Words<V / 4> s = lds_words<V>(own + tr * lh + j0);
            const Words<V / 4> c = lds_words<V>(oth + tr * lh + j0);
            const Words<V / 4> nu = lds_words<V>(oth + (tr + 1) * lh + j0);
            const Words<V / 4> nd = lds_words<V>(oth + (tr - 1) * lh + j0);
            const int je = par ? (j0 + V == lh ? 0 : j0 + V) : (j0 == 0 ? lh - 1 : j0 - 1);
            const u32 edge = (u32)(uint8_t)oth[tr * lh + je];
            const Words<V / 4> ns = int8_update<V, 2, RULE, false, false, false>(
                q, gr, par, j0, V / 4, s, c, nu, nd, nu, nd, edge, stab, m_acc, e_acc);
            sts_words<V>(own + tr * lh + j0, ns);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < 2 * kTbBand * cpr; i += blockDim.x) {
        const int c = i >= kTbBand * cpr;
        const int rem = i - c * kTbBand * cpr;
        const int b = rem / cpr, jc = rem - b * cpr;
        *reinterpret_cast<uint4*>((c ? out1 : out0) + (long long)(r0 + b) * p.pitch + 16 * jc) =
            *reinterpret_cast<const uint4*>(tile + (c * kTbRows + kTbSteps + b) * lh + 16 * jc);
    }
}

bool temporal_ok(const ising_sim* h)
{
    return h->variant == ISING_VARIANT_INT8 && h->ndim == 2 &&
           (h->rule == kMetroFast || h->rule == kHeatFast) && h->lh % 16 == 0 &&
           h->pitch == h->lh && h->ly % kTbBand == 0 && h->ly >= kTbRows &&
           2 * kTbRows * h->lh <= kTbMaxSmem;
}

int temporal_sweeps() { return kTbSteps / 2; }

// kTbSteps / 2 sweeps from sweep t (relative to ctl[0] when ctl is set), colour 0 first,
// from the handle's arrays into its scratch pair (to_scratch) or back.
static cudaError_t launch_int8_temporal(const ising_sim* h, u32 t, const unsigned long long* ctl,
                                        bool to_scratch)
{
    Int8Half p;
    memset(&p, 0, sizeof p);
    p.own = (int8_t*)h->c[0];
    p.other = (const int8_t*)h->c[1];
    p.rows = h->rows;
    p.lh = h->lh;
    p.ly = h->ly;
    p.lz = 1;
    p.pitch = h->pitch;
    p.vw = 16;
    p.cpr = h->lh / 16;
    p.t = t;
    p.k0 = (u32)h->seed;
    p.k1 = (u32)(h->seed >> 32);
    for (int i = 0; i < 7; ++i) p.table[i] = h->table[i];
    p.ctl = ctl;
    const size_t smem = (size_t)2 * kTbRows * h->lh;
    const dim3 grid((unsigned)(h->ly / kTbBand)), block(kTbThreads);
    int8_t* a0 = (int8_t*)h->c[0];
    int8_t* a1 = (int8_t*)h->c[1];
    int8_t* b0 = (int8_t*)h->tb_scratch[0];
    int8_t* b1 = (int8_t*)h->tb_scratch[1];
    const int8_t* i0 = to_scratch ? a0 : b0;
    const int8_t* i1 = to_scratch ? a1 : b1;
    int8_t* o0 = to_scratch ? b0 : a0;
    int8_t* o1 = to_scratch ? b1 : a1;
    auto launch = [&](auto kernel) -> cudaError_t {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = h->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kernel, p, i0, i1, o0, o1);
    };
    return h->rule == kHeatFast ? launch(int8_temporal_kernel<kHeatFast>)
                                : launch(int8_temporal_kernel<kMetroFast>);
}

int temporal_scratch(ising_sim* h)
{
    for (int c = 0; c < 2; ++c) {
        if (h->tb_scratch[c]) continue;
        const cudaError_t e = pool_alloc(h->device, &h->tb_scratch[c], h->colour_bytes, h->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            h->tb_scratch[c] = nullptr;
            return fail(ISING_ERR_NOMEM, "allocation of the temporal schedule's second arrays");
        }
    }
    return ISING_OK;
}

// `count` temporal launches from sweep t (each kTbSteps / 2 sweeps), alternating between the
// handle's arrays and the scratch pair; an odd count ends with the lattice copied back.
cudaError_t launch_temporal_run(const ising_sim* h, u32 t, int64_t count,
                                const unsigned long long* ctl)
{
    const u32 K = (u32)(kTbSteps / 2);
    for (int64_t i = 0; i < count; ++i) {
        const cudaError_t e = launch_int8_temporal(h, t + (u32)i * K, ctl, (i & 1) == 0);
        if (e != cudaSuccess) return e;
    }
    if (count & 1) {
        for (int c = 0; c < 2; ++c) {
            const cudaError_t e = cudaMemcpyAsync(h->c[c], h->tb_scratch[c], h->colour_bytes,
                                                  cudaMemcpyDeviceToDevice, h->stream);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace ising
