// int8 compressed-checkerboard half-sweep (2D/3D, Metropolis/heat bath) with the fused
// integer (M, E) reduction.
//
// Same results as pyising's NumpyCheckerboard._half_sweep (src/pyising/backends/
// numpy_backend.py:26-44) and the CUDA C int8_half kernel (src/pyising/backends/cuda/
// ising.cu:25-87): site n = row*Lh + j of colour c draws word n%4 of
// Philox((n/4, t, c, 0), seed) (src/pyising/philox.py:54-64).
//
// Work split: a thread owns V consecutive colour sites of one row (V = 16: one 128-bit load
// per array, four Philox blocks).  Spins stay packed in 32-bit words and the neighbour
// counting is byte-parallel (SWAR): with +1 = 0x01 and -1 = 0xFF, bit 1 of each byte is the
// "down" flag, so (a ^ b) & 0x02020202 marks anti-aligned pairs of four sites at once.
//
// Metropolis decision without lookups.  Metropolis flips iff X <= 0 or u < table[(X + 2d)/2]
// with X = s*h = 2d - 2A (A = anti-aligned neighbours).  Let T(a) = table[2d - a] for a < d;
// threshold tables built by threshold_table() make T non-decreasing in a, so with
// L = #{a < d : u < T(a)} the rule is exactly "flip iff A + L >= d", evaluated byte-parallel.
// Heat bath (+1 iff u < table[U], U = up neighbours = 2d - D) and Metropolis with a table that
// is not monotone read table[.] per site from a shared-memory copy of the table.
#pragma once

#include "common.cuh"

namespace ising {

template <int W>
struct Words {
    u32 v[W];
};

template <int W>
__device__ __forceinline__ Words<W> load_words(const int8_t* p)
{
    Words<W> r;
    if constexpr (W == 4) {
        const uint4 q = *reinterpret_cast<const uint4*>(p);
        r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
    } else if constexpr (W == 2) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        r.v[0] = q.x; r.v[1] = q.y;
    } else {
        r.v[0] = *reinterpret_cast<const u32*>(p);
    }
    return r;
}

template <int W>
__device__ __forceinline__ Words<W> load_words_ro(const int8_t* p)
{
    Words<W> r;
    if constexpr (W == 4) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(p));
        r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
    } else if constexpr (W == 2) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
        r.v[0] = q.x; r.v[1] = q.y;
    } else {
        r.v[0] = __ldg(reinterpret_cast<const unsigned int*>(p));
    }
    return r;
}

// The opposite colour read from L2, bypassing L1: needed inside one launch that runs several
// half-sweeps, where other SMs rewrite rows this SM may have cached.
template <int W>
__device__ __forceinline__ Words<W> load_words_cg(const int8_t* p)
{
    Words<W> r;
    if constexpr (W == 4) {
        const uint4 q = __ldcg(reinterpret_cast<const uint4*>(p));
        r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
    } else if constexpr (W == 2) {
        const uint2 q = __ldcg(reinterpret_cast<const uint2*>(p));
        r.v[0] = q.x; r.v[1] = q.y;
    } else {
        r.v[0] = __ldcg(reinterpret_cast<const unsigned int*>(p));
    }
    return r;
}

template <int W, bool CG>
__device__ __forceinline__ Words<W> load_other(const int8_t* p)
{
    if constexpr (CG) return load_words_cg<W>(p);
    else return load_words_ro<W>(p);
}

template <int W>
__device__ __forceinline__ void store_words(int8_t* p, const Words<W>& r)
{
    if constexpr (W == 4) {
        *reinterpret_cast<uint4*>(p) = make_uint4(r.v[0], r.v[1], r.v[2], r.v[3]);
    } else if constexpr (W == 2) {
        *reinterpret_cast<uint2*>(p) = make_uint2(r.v[0], r.v[1]);
    } else {
        *reinterpret_cast<u32*>(p) = r.v[0];
    }
}

// 32-bit load from a shared-memory byte address.
__device__ __forceinline__ u32 lds_u32(u32 addr)
{
    u32 v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

// 4-bit mask (bit i = site i) -> XOR pattern 0xFE in byte i (the flip of a +-1 byte).
__device__ __forceinline__ u32 flip_bytes(u32 m4)
{
    return ((m4 * 0x00204081u) & 0x01010101u) * 0xFEu;  // bit i -> byte i, then 0x01 -> 0xFE
}

// New spins of the four sites in word `s` given their anti-aligned (Metropolis) or down
// (heat bath) neighbour counts `cnt` (one byte per site) and their four uniforms.  `stab` is
// the acceptance table in shared memory (used by the lookup rules).
//   kMetroFast: byte-parallel "A + #{a<d : u < T(a)} >= d" (monotone Metropolis tables);
//   heat bath and kMetroGeneric: one shared-memory lookup per site, valid for any table.
template <int NDIM, int RULE>
__device__ __forceinline__ u32 decide4(const Int8Half& p, u32 s, u32 cnt, const u32x4& r,
                                       const u32* stab)
{
    constexpr int d = NDIM;
    if constexpr (RULE == kObserve) {
        return s;
    } else if constexpr (RULE == kMetroFast) {
        u32 l[4] = {0, 0, 0, 0};
        const u32 uu[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int a = 0; a < d; ++a) {
            const u32 thr = p.table[2 * d - a];
#pragma unroll
            for (int i = 0; i < 4; ++i) l[i] += uu[i] < thr ? 1u : 0u;
        }
        const u32 lw = l[0] | (l[1] << 8) | (l[2] << 16) | (l[3] << 24);
        const u32 m7 = (cnt + lw + (u32)(0x80 - d) * 0x01010101u) & kBit7;
        return s ^ flip_mask_from_bit7(m7);
    } else if constexpr (RULE == kHeatFast || RULE == kHeatGeneric) {
        // +1 iff u < table[U], U = up neighbours = 2d - D; rt[k] = table[2d - k]
        const u32 base = (u32)__cvta_generic_to_shared(stab) + 8u * d;  // &table[2d]
        const u32 b0 = r.x < lds_u32(base - 4u * (cnt & 0xFFu)) ? 1u : 0u;
        const u32 b1 = r.y < lds_u32(base - 4u * ((cnt >> 8) & 0xFFu)) ? 2u : 0u;
        const u32 b2 = r.z < lds_u32(base - 4u * ((cnt >> 16) & 0xFFu)) ? 4u : 0u;
        const u32 b3 = r.w < lds_u32(base - 4u * (cnt >> 24)) ? 8u : 0u;
        return 0xFFFFFFFFu ^ flip_bytes(b0 | b1 | b2 | b3);
    } else {
        // Metropolis, any table: flip iff A >= d or u < table[2d - A]
        const u32 base = (u32)__cvta_generic_to_shared(stab) + 8u * d;  // &table[2d]
        const u32 a0 = cnt & 0xFFu, a1 = (cnt >> 8) & 0xFFu, a2 = (cnt >> 16) & 0xFFu,
                  a3 = cnt >> 24;
        const u32 f0 = (a0 >= (u32)d || r.x < lds_u32(base - 4u * a0)) ? 1u : 0u;
        const u32 f1 = (a1 >= (u32)d || r.y < lds_u32(base - 4u * a1)) ? 2u : 0u;
        const u32 f2 = (a2 >= (u32)d || r.z < lds_u32(base - 4u * a2)) ? 4u : 0u;
        const u32 f3 = (a3 >= (u32)d || r.w < lds_u32(base - 4u * a3)) ? 8u : 0u;
        return s ^ flip_bytes(f0 | f1 | f2 | f3);
    }
}

// New spins of the V colour sites starting at j0 in row `row` (parity `par` = (y + z + colour)
// & 1) from their own words `s`, the opposite colour's words of the same row `c`, of the rows
// above/below `nu`/`nd` and planes above/below `zu`/`zd` (3D), and the horizontal neighbour byte
// outside the chunk `edge`; stores them, and with MEAS adds the chunk's (M, E) contribution to
// m_acc / e_acc.  With RULE == kObserve nothing is updated (measurement only).
//
// MIXED = false: every chunk is full (lh % V == 0).  MIXED = true: rows are padded to a multiple
// of V bytes and a row's last chunk holds wv < W valid words; such a chunk runs the same
// instructions as a full one (no divergence inside a warp), with the padding words selected
// away: their random numbers are drawn and discarded, their bytes stored back unchanged, and
// the right-hand neighbour of the last valid word is the row's wrapped edge byte.
// Returns the new words; STORE = false leaves storing them to the caller (the tiles of the
// temporally blocked kernel live in shared memory).
template <int V, int NDIM, int RULE, bool MIXED, bool MEAS, bool STORE = true>
__device__ __forceinline__ Words<V / 4> int8_update(const Int8Half& p, long long row, int par,
                                                    int j0, int wv, const Words<V / 4>& s,
                                                    const Words<V / 4>& c,
                                                    const Words<V / 4>& nu,
                                                    const Words<V / 4>& nd,
                                                    const Words<V / 4>& zu,
                                                    const Words<V / 4>& zd, u32 edge,
                                                    const u32* stab, long long& m_acc,
                                                    long long& e_acc)
{
    constexpr int W = V / 4;
    constexpr bool kHeat = (RULE == kHeatFast || RULE == kHeatGeneric);
    Words<W> hz;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        if (par) {
            u32 nx = edge;
            if (k + 1 < W) nx = (!MIXED || k + 1 < wv) ? c.v[k + 1] : edge;
            hz.v[k] = __funnelshift_r(c.v[k], nx, 8);
        } else {
            const u32 pv = (k > 0) ? c.v[k - 1] : (edge << 24);
            hz.v[k] = __funnelshift_l(pv, c.v[k], 8);
        }
    }

    // Neighbour counts first, so the neighbour words are dead before the Philox blocks.
    u32 cnt[W];
    int other_down = 0;  // down spins of the opposite colour at the same indices (for M)
#pragma unroll
    for (int k = 0; k < W; ++k) {
        if constexpr (kHeat) {
            u32 acc = (c.v[k] & kBit1) + (hz.v[k] & kBit1) + (nu.v[k] & kBit1) +
                      (nd.v[k] & kBit1);
            if constexpr (NDIM == 3) acc += (zu.v[k] & kBit1) + (zd.v[k] & kBit1);
            cnt[k] = acc >> 1;  // down neighbours per site
        } else {
            const u32 sv = s.v[k];
            u32 acc = ((c.v[k] ^ sv) & kBit1) + ((hz.v[k] ^ sv) & kBit1) +
                      ((nu.v[k] ^ sv) & kBit1) + ((nd.v[k] ^ sv) & kBit1);
            if constexpr (NDIM == 3)
                acc += ((zu.v[k] ^ sv) & kBit1) + ((zd.v[k] ^ sv) & kBit1);
            cnt[k] = acc >> 1;  // anti-aligned neighbours per site
        }
        if constexpr (MEAS) {
            const int od = __popc(c.v[k] & kBit1);
            other_down += (!MIXED || k < wv) ? od : 0;
        }
    }

    Words<W> ns;
    // Philox counters use the logical site index row*lh + j, independent of the pitch
    const u32 q0 = (u32)((unsigned long long)(row * p.lh + j0) >> 2);
#pragma unroll
    for (int k = 0; k < W; ++k) {
        if constexpr (RULE == kObserve) {
            ns.v[k] = s.v[k];
        } else {
            const u32x4 r =
                philox4x32_10<NDIM == 2>(q0 + (u32)k, p.t, p.color, 0u, p.k0, p.k1);
            const u32 d = decide4<NDIM, RULE>(p, s.v[k], cnt[k], r, stab);
            ns.v[k] = (!MIXED || k < wv) ? d : s.v[k];
        }
    }
    if constexpr (RULE != kObserve && STORE) store_words<W>(p.own + row * p.pitch + j0, ns);

    if constexpr (MEAS) {
        // Bonds of this colour's sites: s*h = 2d - 2A' per site (A' = anti-aligned neighbours
        // of the new spin); E = -sum s*h.  A' follows from the counts: a flipped site's
        // anti-aligned neighbours are the previously aligned ones (2d - A), and for heat bath
        // A' = D for a +1 site, 2d - D for a -1 site.
        constexpr u32 k2d = 0x01010101u * (u32)(2 * NDIM);
        int anti = 0, down = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const u32 sv = ns.v[k];
            u32 sel;  // 0xFF in the bytes whose count is replaced by 2d - count
            if constexpr (kHeat) sel = ((sv & kBit1) >> 1) * 0xFFu;
            else sel = (((sv ^ s.v[k]) & kBit1) >> 1) * 0xFFu;
            const u32 ap = (cnt[k] & ~sel) | ((k2d - cnt[k]) & sel);
            const bool valid = !MIXED || k < wv;
            anti += valid ? byte_sum(ap) : 0;
            down += valid ? __popc(sv & kBit1) : 0;
        }
        const int nv = 4 * wv;                      // valid sites of this chunk
        m_acc += 2 * nv - 2 * (down + other_down);  // this colour's sites + the other's
        e_acc += 2 * anti - 2 * NDIM * nv;          // -(2d n - 2 anti)
    }
    return ns;
}

template <bool MIXED, int W>
__device__ __forceinline__ int valid_words(const Int8Half& p, int j0)
{
    if constexpr (!MIXED) return W;
    const int left = (p.lh - j0) >> 2;
    return left < W ? left : W;
}

// Horizontal neighbour byte outside a chunk's wv valid words (periodic in x).
__device__ __forceinline__ int edge_index(const Int8Half& p, int par, int j0, int wv)
{
    return par ? (j0 + 4 * wv == p.lh ? 0 : j0 + 4 * wv) : (j0 == 0 ? p.lh - 1 : j0 - 1);
}

// One chunk (V sites from j0) of row `row` = (z, y): loads its neighbourhood, then int8_update.
// CG reads the opposite colour from L2 (needed when one launch runs several half-sweeps).
template <int V, int NDIM, int RULE, bool CG, bool MIXED, bool MEAS>
__device__ __forceinline__ void int8_chunk(const Int8Half& p, long long row, int y, int z, int j0,
                                           const u32* stab, long long& m_acc, long long& e_acc)
{
    constexpr int W = V / 4;
    const int par = (y + z + (int)p.color) & 1;
    const int wv = valid_words<MIXED, W>(p, j0);
    const long long rb = row * p.pitch;
    const int8_t* orow = p.other + rb;
    const Words<W> s = load_words<W>(p.own + rb + j0);
    const Words<W> c = load_other<W, CG>(orow + j0);
    const int yu = z * p.ly + (y + 1 == p.ly ? 0 : y + 1);
    const int yd = z * p.ly + (y == 0 ? p.ly - 1 : y - 1);
    const Words<W> nu = load_other<W, CG>(p.other + (long long)yu * p.pitch + j0);
    const Words<W> nd = load_other<W, CG>(p.other + (long long)yd * p.pitch + j0);
    Words<W> zu = nu, zd = nd;
    if constexpr (NDIM == 3) {
        const int pu = (z + 1 == p.lz ? 0 : z + 1) * p.ly + y;
        const int pd = (z == 0 ? p.lz - 1 : z - 1) * p.ly + y;
        zu = load_other<W, CG>(p.other + (long long)pu * p.pitch + j0);
        zd = load_other<W, CG>(p.other + (long long)pd * p.pitch + j0);
    }
    const int je = edge_index(p, par, j0, wv);
    const u32 edge = CG ? (u32)(uint8_t)__ldcg(orow + je) : (u32)(uint8_t)__ldg(orow + je);
    int8_update<V, NDIM, RULE, MIXED, MEAS>(p, row, par, j0, wv, s, c, nu, nd, zu, zd, edge, stab,
                                            m_acc, e_acc);
}

// Band schedule: chunk column j0 of rows y0 .. y1-1 of plane z, top to bottom.  The three
// opposite-colour rows a row needs (y-1, y, y+1) slide down the band, so each row loads one new
// opposite-colour row (plus the planes z +- 1 in 3D) instead of three.
template <int V, int NDIM, int RULE, bool MIXED, bool MEAS>
__device__ __forceinline__ void int8_band(const Int8Half& p, int z, int y0, int y1, int j0,
                                          const u32* stab, long long& m_acc, long long& e_acc)
{
    constexpr int W = V / 4;
    const int wv = valid_words<MIXED, W>(p, j0);
    const int ly = p.ly;
    const long long plane = (long long)z * ly;
    const int8_t* oth = p.other + j0;
    Words<W> nd = load_words_ro<W>(oth + (plane + (y0 == 0 ? ly - 1 : y0 - 1)) * p.pitch);
    Words<W> c = load_words_ro<W>(oth + (plane + y0) * p.pitch);
    const long long zup = NDIM == 3 ? (long long)(z + 1 == p.lz ? 0 : z + 1) * ly : 0;
    const long long zdn = NDIM == 3 ? (long long)(z == 0 ? p.lz - 1 : z - 1) * ly : 0;
    for (int y = y0; y < y1; ++y) {
        const long long row = plane + y;
        const Words<W> nu = load_words_ro<W>(oth + (plane + (y + 1 == ly ? 0 : y + 1)) * p.pitch);
        Words<W> zu = nu, zd = nd;
        if constexpr (NDIM == 3) {
            zu = load_words_ro<W>(oth + (zup + y) * p.pitch);
            zd = load_words_ro<W>(oth + (zdn + y) * p.pitch);
        }
        const int par = (y + z + (int)p.color) & 1;
        const u32 edge = (u32)(uint8_t)__ldg(p.other + row * p.pitch + edge_index(p, par, j0, wv));
        const Words<W> s = load_words<W>(p.own + row * p.pitch + j0);
        int8_update<V, NDIM, RULE, MIXED, MEAS>(p, row, par, j0, wv, s, c, nu, nd, zu, zd, edge,
                                                stab, m_acc, e_acc);
        nd = c;
        c = nu;
    }
}

}  // namespace ising
