// Device code of the multi-spin-coded (64 spins per uint64) 2D Metropolis half-sweep with the
// lazy bitwise uniform comparison, shared by the single-lattice and the batched kernels.
//
// Same results as pyising's NumpyMultiSpin (src/pyising/backends/numpy_backend.py:54-124) and
// the CUDA C msc_half kernel (src/pyising/backends/cuda/ising.cu:92-150): word w at bit level
// k uses call k/2 of Philox((w, t, c, 1 + k/2), seed); even levels take r0 | r1 << 32, odd
// levels r2 | r3 << 32 (src/pyising/philox.py:67-78).  Level k decides the lanes whose
// uniform's bit 31-k differs from the threshold's: u < thr exactly when, at the first
// differing bit, u has 0 and the threshold has 1.
#pragma once

#include "common.cuh"

#ifndef ISING_MSC_INTAKE_CALLS
#define ISING_MSC_INTAKE_CALLS 4
#endif

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

// Flip mask of one word drawing Philox blocks until every lane is decided; `calls` returns
// the blocks drawn.
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

// One word (row y, word x): update when UPDATE, then the (M, E) contribution of its 64 sites'
// bonds when p.meas (every bond has exactly one colour-1 end; the other colour's same-index
// word is counted once for M), and the call statistics when p.stats.
template <bool UPDATE>
__device__ __forceinline__ void msc_word(const MscHalf& p, int y, int x, long long& m_acc,
                                         long long& e_acc, long long& calls_acc,
                                         long long& wmax_acc)
{
    const int nw = p.nw;
    const long long rb = (long long)y * nw;
    const u64* orow = p.other + rb;
    const u64 o = p.own[rb + x];
    const u64 c = __ldg(orow + x);
    u64 hz;
    if ((y + (int)p.color) & 1) hz = (c >> 1) | (__ldg(orow + (x + 1 == nw ? 0 : x + 1)) << 63);
    else hz = (c << 1) | (__ldg(orow + (x == 0 ? nw - 1 : x - 1)) >> 63);
    const u64 up = __ldg(p.other + (long long)(y == 0 ? p.rows - 1 : y - 1) * nw + x);
    const u64 dn = __ldg(p.other + (long long)(y + 1 == p.rows ? 0 : y + 1) * nw + x);
    u64 ns = o;
    if constexpr (UPDATE) {
        const Slices s = slice4(o, c, hz, up, dn);
        int calls = 0;
        ns = o ^ msc_flip(s, (u32)(rb + x), p.t, p.color, p.k0, p.k1, p.thr4, p.thr8, calls);
        p.own[rb + x] = ns;
        if (p.stats) {
            calls_acc += calls;
            wmax_acc += __reduce_max_sync(__activemask(), calls);
        }
    }
    if (p.meas) {
        const int anti =
            __popcll(ns ^ c) + __popcll(ns ^ hz) + __popcll(ns ^ up) + __popcll(ns ^ dn);
        m_acc += 2 * (__popcll(ns) + __popcll(c)) - 128;
        e_acc += 2 * anti - 256;
    }
}

// ---------------------------------------------------------------------------------------------
// Work-stack schedule (no measurement): keeps every lane busy with a Philox block.
//
// Per word, the lazy comparison needs a data-dependent number of Philox blocks (3.8 on average
// at T_c, but 6.3 for the slowest word of a warp), so a one-word-per-lane kernel idles most
// lanes in its last iterations.  Here a warp walks a contiguous range of words:
//   * intake: the next 32 words of the range (their global loads were issued when the previous
//     batch was consumed) are bit-sliced and get four Philox blocks each unconditionally (at
//     T_c half of the words need four or more); decided words are stored, the others pushed on
//     the warp's 64-entry stack in shared memory;
//   * while the stack holds 32 or more entries: pop 32, draw one Philox block each at the
//     entry's own level pair, store finished words, push back the rest;
//   * when the range is done and at most 32 entries are left: each lane runs one entry to the
//     end (stack_drain).
// The random numbers, bit levels and their order are the reference's; only the schedule
// differs, so results are identical.  Lanes are handled as two independent 32-bit halves.

#ifndef ISING_MSC_POP
#define ISING_MSC_POP 1
#endif
constexpr int kPop = 32 * ISING_MSC_POP;  // entries popped per pass (two per lane: two chains)
constexpr int kQueueCap = kPop + 32;
constexpr int kIntakeCalls = ISING_MSC_INTAKE_CALLS;  // Philox blocks per word before queueing

// One more slot than entries: lanes with nothing to push write to slot kQueueCap, so a push is
// stores without a branch.
struct QueueSlots {
    u32 idx[kQueueCap + 1];
    u32 lp[kQueueCap + 1];
    u64 a1[kQueueCap + 1];
    u64 und[kQueueCap + 1];
    u64 res[kQueueCap + 1];
};

// Threshold bit masks of the even and odd level of each level pair: (t4e, t8e, t4o, t8o).
__device__ __forceinline__ uint4 level_masks(u32 thr4, u32 thr8, u32 lp)
{
    const u32 se = 31u - 2u * lp, so = se - 1u;
    return make_uint4(((thr4 >> se) & 1u) ? ~0u : 0u, ((thr8 >> se) & 1u) ? ~0u : 0u,
                      ((thr4 >> so) & 1u) ? ~0u : 0u, ((thr8 >> so) & 1u) ? ~0u : 0u);
}

// One bit level on 32 lanes: tm selects each lane's threshold bit (thr4 for lanes with one
// anti-aligned neighbour, thr8 for none); an undecided lane is decided when its random bit
// differs from tm, and accepted (flipped) when that bit is 0 and tm is 1.
__device__ __forceinline__ void level32(u32 r, u32 t4m, u32 t8m, u32 a1, u32& und, u32& res)
{
    const u32 tm = (a1 & t4m) | (~a1 & t8m);
    res ^= und & ~r & tm;
    und &= ~(r ^ tm);
}

__device__ __forceinline__ void call_levels(const u32x4& r, const uint4& m, u32 a1l, u32 a1h,
                                            u32& undl, u32& undh, u32& resl, u32& resh)
{
    level32(r.x, m.x, m.y, a1l, undl, resl);  // even level: r0 | r1 << 32
    level32(r.y, m.x, m.y, a1h, undh, resh);
    level32(r.z, m.z, m.w, a1l, undl, resl);  // odd level: r2 | r3 << 32
    level32(r.w, m.z, m.w, a1h, undh, resh);
}

// Both levels of one Philox block on 32 lanes: the even level uses r_e, the odd one r_o.
__device__ __forceinline__ void level_pair(u32 re, u32 ro, u32 t4e, u32 t8e, u32 t4o, u32 t8o,
                                           u32 a1, u32& und, u32& acc)
{
    const u32 tme = (a1 & t4e) | (~a1 & t8e);
    const u32 tmo = (a1 & t4o) | (~a1 & t8o);
    const u32 ae = und & ~re & tme;       // decided at the even level, accepted
    const u32 u1 = und & ~(re ^ tme);     // still undecided after it
    const u32 ao = u1 & ~ro & tmo;
    und = u1 & ~(ro ^ tmo);
    acc |= ae | ao;
}

__device__ __forceinline__ void block_levels(const u32x4& r, const uint4& m, u32 a1l, u32 a1h,
                                             u32& undl, u32& undh, u32& accl, u32& acch)
{
    level_pair(r.x, r.z, m.x, m.y, m.z, m.w, a1l, undl, accl);  // r0 | r1 << 32, r2 | r3 << 32
    level_pair(r.y, r.w, m.x, m.y, m.z, m.w, a1h, undh, acch);
}

// Where a lattice piece sits in a bigger lattice (slab decomposition): the Philox word index is
// w0 + the local word index and the row parity that of the global row (par0 + local row); rows
// -1 and `rows` are not wrapped but read from lo and hi (the slab's halo rows, or a neighbouring
// slab's edge rows in place).  Unused (and compiled out) for whole lattices.
struct SlabOffset {
    long long w0;
    int par0;
    const u64* lo;
    const u64* hi;
};

// Global words of one intake batch (one per lane), loaded ahead of use.
struct IntakeLoads {
    u64 o, c, side, up, dn;
    int y;  // row of the word
};

template <bool SLAB = false>
__device__ __forceinline__ void intake_load(const MscHalf& p, long long w, bool valid, int nw,
                                            int nw_shift, IntakeLoads& L,
                                            const SlabOffset& so = {0, 0, nullptr, nullptr})
{
    if (!valid) {
        L.o = L.c = L.side = L.up = L.dn = 0;
        L.y = 0;
        return;
    }
    int y, x;
    if (nw_shift >= 0) {
        y = (int)(w >> nw_shift);
        x = (int)(w & (nw - 1));
    } else {
        y = (int)div_magic(w, p.nw_magic, nw);
        x = (int)(w - (long long)y * nw);
    }
    L.y = y;
    const u64* orow = p.other + (long long)y * nw;
    L.o = p.own[w];
    L.c = __ldg(orow + x);
    const int py = SLAB ? y + so.par0 : y;
    const int xs = ((py + (int)p.color) & 1) ? (x + 1 == nw ? 0 : x + 1) : (x == 0 ? nw - 1 : x - 1);
    L.side = __ldg(orow + xs);
    if constexpr (SLAB) {
        L.up = __ldg((y == 0 ? so.lo : orow - nw) + x);
        L.dn = __ldg((y + 1 == p.rows ? so.hi : orow + nw) + x);
    } else {
        L.up = __ldg(p.other + (long long)(y == 0 ? p.rows - 1 : y - 1) * nw + x);
        L.dn = __ldg(p.other + (long long)(y + 1 == p.rows ? 0 : y + 1) * nw + x);
    }
}

// The end of a warp's work: the at most 32 stack entries left take one lane each, and each lane
// draws its entry's Philox blocks one after another until the entry is decided, without going
// back to the stack.  Draining by stack passes instead (pop, one block, push back the undecided)
// spends a pop, a ballot and a push per block on a warp whose lanes are mostly idle; here the
// passes' bookkeeping is gone and only the lanes' longest chain remains (measured on B200 with
// the strip walker: 16384^2 3546 -> 3647 flips/ns, 8192^2 2535 -> 2790, 4096^2 1387 -> 1716;
// drawing two or more of an entry's blocks at a time was no faster).  Works on both stack
// layouts (QueueSlots, StripSlots).
template <class Slots>
__device__ __forceinline__ void stack_drain(const MscHalf& p, Slots& q, int& n,
                                            const uint4* lvmask, u32 wg)
{
    const int lane = threadIdx.x & 31;
    const bool act = lane < n;
    u32 idx = 0, lp = 0, undl = 0, undh = 0, accl = 0, acch = 0;
    u64 a1 = 0, res = 0;
    if (act) {
        idx = q.idx[lane];
        lp = q.lp[lane];
        a1 = q.a1[lane];
        res = q.res[lane];
        const u64 und = q.und[lane];
        undl = (u32)und;
        undh = (u32)(und >> 32);
    }
    __syncwarp();
    n = 0;
    if (act) {
        const u32 a1l = (u32)a1, a1h = (u32)(a1 >> 32);
        do {  // an entry has lp < 16 and an undecided lane
            const u32x4 r = philox4x32_10<true>(wg + idx, p.t, p.color, 1u + lp, p.k0, p.k1);
            block_levels(r, lvmask[lp], a1l, a1h, undl, undh, accl, acch);
        } while ((undl | undh) != 0 && ++lp < 16u);
        p.own[idx] = res ^ ((u64)accl | ((u64)acch << 32));
    }
    __syncwarp();
}

// The whole warp updates words [begin, end) of the lattice in p.  `lvmask` holds
// level_masks(p.thr4, p.thr8, lp) for lp = 0..15; `q` is this warp's stack.
template <bool SLAB = false>
__device__ __forceinline__ void msc_queue_range(const MscHalf& p, long long begin, long long end,
                                                int nw_shift, QueueSlots& q,
                                                const uint4* lvmask,
                                                const SlabOffset& so = {0, 0, nullptr, nullptr})
{
    const u32 wg = SLAB ? (u32)so.w0 : 0u;  // Philox word index = wg + local index (mod 2^32)
    const int lane = threadIdx.x & 31;
    const u32 lt = (1u << lane) - 1u;
    const int nw = p.nw;
    long long next = begin;
    int n = 0;
    IntakeLoads L;
    long long w = next + lane;
    bool more = next < end;
    if (more) intake_load<SLAB>(p, w, w < end, nw, nw_shift, L, so);
    while (true) {
        if (n < kPop && more) {
            const bool valid = w < end;
            u32 a1l = 0, a1h = 0, undl = 0, undh = 0, resl = 0, resh = 0;
            if (valid) {
                const bool par = ((SLAB ? L.y + so.par0 : L.y) + (int)p.color) & 1;
                const u64 hz = par ? ((L.c >> 1) | (L.side << 63)) : ((L.c << 1) | (L.side >> 63));
                const Slices s = slice4(L.o, L.c, hz, L.up, L.dn);
                a1l = (u32)s.a1;
                a1h = (u32)(s.a1 >> 32);
                undl = ~(u32)s.a2;
                undh = ~(u32)(s.a2 >> 32);
                const u64 r0 = L.o ^ s.a2;
                resl = (u32)r0;
                resh = (u32)(r0 >> 32);
            }
            const long long wc = w;
            next += 32;
            more = next < end;
            w = next + lane;
            if (more) intake_load<SLAB>(p, w, w < end, nw, nw_shift, L, so);
            if (valid) {
#pragma unroll
                for (int c3 = 0; c3 < kIntakeCalls; ++c3) {
                    const u32x4 r =
                        philox4x32_10(wg + (u32)wc, p.t, p.color, 1u + (u32)c3, p.k0, p.k1);
                    call_levels(r, lvmask[c3], a1l, a1h, undl, undh, resl, resh);
                }
            }
            const bool keep = valid && (undl | undh) != 0;
            if (valid && !keep) p.own[wc] = (u64)resl | ((u64)resh << 32);
            const u32 km = __ballot_sync(0xFFFFFFFFu, keep);
            {
                const int pos = keep ? n + __popc(km & lt) : kQueueCap;
                q.idx[pos] = (u32)wc;
                q.lp[pos] = (u32)kIntakeCalls;
                q.a1[pos] = (u64)a1l | ((u64)a1h << 32);
                q.und[pos] = (u64)undl | ((u64)undh << 32);
                q.res[pos] = (u64)resl | ((u64)resh << 32);
            }
            n += __popc(km);
            __syncwarp();
        } else if (!more && n <= 32) {
            if (n > 0) stack_drain(p, q, n, lvmask, wg);
            break;
        } else {
            // pop up to kPop entries: lane l takes entries base + l and base + 32 + l
            const int take = n < kPop ? n : kPop;
            const int base = n - take;
            u32 idx[ISING_MSC_POP], lp[ISING_MSC_POP];
            u64 a1[ISING_MSC_POP];
            u32 undl[ISING_MSC_POP], undh[ISING_MSC_POP], resl[ISING_MSC_POP], resh[ISING_MSC_POP];
            bool act[ISING_MSC_POP];
#pragma unroll
            for (int m = 0; m < ISING_MSC_POP; ++m) {
                const int e = base + 32 * m + lane;
                act[m] = 32 * m + lane < take;
                idx[m] = act[m] ? q.idx[e] : 0u;
                lp[m] = act[m] ? q.lp[e] : 0u;
                a1[m] = act[m] ? q.a1[e] : 0ull;
                const u64 und = act[m] ? q.und[e] : 0ull, res = act[m] ? q.res[e] : 0ull;
                undl[m] = (u32)und;
                undh[m] = (u32)(und >> 32);
                resl[m] = (u32)res;
                resh[m] = (u32)(res >> 32);
            }
            __syncwarp();
#pragma unroll
            for (int m = 0; m < ISING_MSC_POP; ++m) {
                if (act[m]) {
                    const u32x4 r =
                        philox4x32_10(wg + idx[m], p.t, p.color, 1u + lp[m], p.k0, p.k1);
                    call_levels(r, lvmask[lp[m]], (u32)a1[m], (u32)(a1[m] >> 32), undl[m],
                                undh[m], resl[m], resh[m]);
                    ++lp[m];
                }
            }
            int kept = 0;
#pragma unroll
            for (int m = 0; m < ISING_MSC_POP; ++m) {
                const bool keep = act[m] && (undl[m] | undh[m]) != 0 && lp[m] < 16u;
                if (act[m] && !keep) p.own[idx[m]] = (u64)resl[m] | ((u64)resh[m] << 32);
                const u32 km = __ballot_sync(0xFFFFFFFFu, keep);
                {
                    const int pos = keep ? base + kept + __popc(km & lt) : kQueueCap;
                    q.idx[pos] = idx[m];
                    q.lp[pos] = lp[m];
                    q.a1[pos] = a1[m];
                    q.und[pos] = (u64)undl[m] | ((u64)undh[m] << 32);
                    q.res[pos] = (u64)resl[m] | ((u64)resh[m] << 32);
                }
                kept += __popc(km);
            }
            n = base + kept;
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Strip schedule (lattices whose rows hold a multiple of 32 words): a warp walks a band of rows
// of one 32-word column strip, lane l owning word x0 + l of every row.  The opposite colour's
// rows y - 1, y, y + 1 slide through registers (one new row per step), so a word costs three
// loads (its own word, the opposite colour's next row, the horizontal neighbour word) instead
// of five, and the row parity, the row index and the wrap of the vertical neighbours are
// warp-uniform.  The bit-sliced count takes seven operations per 32-bit half: with
// x_k = o ^ n_k, x1 ^ x2 = n1 ^ n2 and x1 & x2 = (o ^ n1) & (o ^ n2), so the pair sums need
// no x_k.  The lazy comparison handles both levels of a Philox block together (seven
// operations per half).  Words still undecided after the intake go to the warp's stack as in
// the range schedule.  Random numbers, levels and their order are the reference's, so the
// results are identical.

// Pair sums of two anti-aligned flags: s = exactly one, c = both.
struct HalfSlices {
    u32 a1, a2;  // exactly one / two or more anti-aligned neighbours
};

__device__ __forceinline__ HalfSlices slice_half(u32 o, u32 n1, u32 n2, u32 n3, u32 n4)
{
    const u32 s1 = n1 ^ n2, c1 = (o ^ n1) & (o ^ n2);
    const u32 s2 = n3 ^ n4, c2 = (o ^ n3) & (o ^ n4);
    const u32 cc = c1 | c2;
    HalfSlices h;
    h.a1 = (s1 ^ s2) & ~cc;
    h.a2 = cc | (s1 & s2);
    return h;
}

// The warp walks its band two rows per step: each lane takes word x of rows y and y + 1, so
// eight Philox chains are in flight at intake and the per-step loop, ballot and stack
// bookkeeping are shared by two words.  The stack takes up to 64 entries per intake, so it holds
// kPop + 64.  The Philox products are separate high and low multiplies and the intake's level
// masks come from the block's shared table: measured faster here (16384^2: 3610 flips/ns
// against 3260 for one row per step with the products as wide multiplies and the masks derived
// in uniform registers).
constexpr int kStripCap = kPop + 64;

// One more slot than entries: lanes with nothing to push write their entry to slot kStripCap,
// so a push is stores without a branch (measured 1.2% faster than the per-lane branch, in the
// word-range walker too).
struct StripSlots {
    u32 idx[kStripCap + 1];
    u32 lp[kStripCap + 1];
    u64 a1[kStripCap + 1];
    u64 und[kStripCap + 1];
    u64 res[kStripCap + 1];
};

// One pass over the stack: a Philox block for each of up to 32 entries at its own level pair;
// the result word of an entry already holds every decision made so far.
__device__ __forceinline__ void strip_pop(const MscHalf& p, StripSlots& q, int& n,
                                          const uint4* lvmask, u32 wg)
{
    const int lane = threadIdx.x & 31;
    const u32 lt = (1u << lane) - 1u;
    const int take = n < 32 ? n : 32;
    const int base = n - take;
    const bool act = lane < take;
    const int e = base + lane;
    const u32 idx = act ? q.idx[e] : 0u;
    u32 lp = act ? q.lp[e] : 0u;
    const u64 a1 = act ? q.a1[e] : 0ull;
    const u64 und = act ? q.und[e] : 0ull, res = act ? q.res[e] : 0ull;
    __syncwarp();
    u32 undl = (u32)und, undh = (u32)(und >> 32), accl = 0, acch = 0;
    if (act) {
        const u32x4 r = philox4x32_10<true>(wg + idx, p.t, p.color, 1u + lp, p.k0, p.k1);
        block_levels(r, lvmask[lp], (u32)a1, (u32)(a1 >> 32), undl, undh, accl, acch);
        ++lp;
    }
    const u64 nres = res ^ ((u64)accl | ((u64)acch << 32));
    const bool keep = act && (undl | undh) != 0 && lp < 16u;
    if (act && !keep) p.own[idx] = nres;
    const u32 km = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) {
        const int pos = base + __popc(km & lt);
        q.idx[pos] = idx;
        q.lp[pos] = lp;
        q.a1[pos] = a1;
        q.und[pos] = (u64)undl | ((u64)undh << 32);
        q.res[pos] = nres;
    }
    n = base + __popc(km);
    __syncwarp();
}

// The warp updates rows [y0, y1) of strip `strip` (words 32 strip .. 32 strip + 31 of a row).
// SLAB: the lattice is a slab of a bigger one (SlabOffset): Philox word indices are so.w0 + the
// local index, row parities those of the global rows, and rows -1 and `rows` of the opposite
// colour are read from so.lo and so.hi instead of wrapping.
template <int K, bool SLAB = false>
__device__ __forceinline__ void msc_strip_band(const MscHalf& p, int strip, int y0, int y1,
                                               StripSlots& q, const uint4* lvmask,
                                               const SlabOffset& so = {0, 0, nullptr, nullptr})
{
    const int lane = threadIdx.x & 31;
    const u32 lt = (1u << lane) - 1u;
    const int nw = p.nw, rows = p.rows;
    const int x = strip * 32 + lane;
    const int xr = x + 1 == nw ? 0 : x + 1, xl = x == 0 ? nw - 1 : x - 1;
    const u64* other = p.other;
    const u32 wg = SLAB ? (u32)so.w0 : 0u;
    const int odd0 = ((SLAB ? so.par0 : 0) + (int)p.color) & 1;  // parity of local row 0
    // opposite-colour row r, r in [-1, rows]
    auto orow = [&](int r) -> const u64* {
        if constexpr (SLAB) {
            if (r < 0) return so.lo;
            if (r >= rows) return so.hi;
        } else {
            r = r < 0 ? rows - 1 : (r >= rows ? 0 : r);
        }
        return other + (long long)r * nw;
    };
    u64 up = __ldg(orow(y0 - 1) + x);
    u64 c = __ldg(orow(y0) + x);
    u64 f_o0 = 0, f_o1 = 0, f_d1 = 0, f_d2 = 0, f_s0 = 0, f_s1 = 0;
    auto fetch = [&](int y) {
        f_o0 = p.own[(long long)y * nw + x];
        f_d1 = __ldg(orow(y + 1) + x);
        f_s0 = __ldg(orow(y) + (((y + odd0) & 1) ? xr : xl));
        if (y + 1 < y1) {
            f_o1 = p.own[(long long)(y + 1) * nw + x];
            f_d2 = __ldg(orow(y + 2) + x);
            f_s1 = __ldg(orow(y + 1) + (((y + 1 + odd0) & 1) ? xr : xl));
        }
    };
    int y = y0;
    if (y < y1) fetch(y);
    int n = 0;
    while (true) {
        if (n < kPop && y < y1) {
            const bool two = y + 1 < y1;
            const u64 o0 = f_o0, o1 = f_o1, d1 = f_d1, d2 = f_d2, s0 = f_s0, s1 = f_s1;
            const bool odd = ((y + odd0) & 1) != 0;  // row y; row y + 1 has the other parity
            const u64 hz0 = odd ? ((c >> 1) | (s0 << 63)) : ((c << 1) | (s0 >> 63));
            const u64 hz1 = odd ? ((d1 << 1) | (s1 >> 63)) : ((d1 >> 1) | (s1 << 63));
            const int yc = y;
            y += two ? 2 : 1;
            if (y < y1) fetch(y);
            const HalfSlices al = slice_half((u32)o0, (u32)c, (u32)hz0, (u32)up, (u32)d1);
            const HalfSlices ah = slice_half((u32)(o0 >> 32), (u32)(c >> 32), (u32)(hz0 >> 32),
                                             (u32)(up >> 32), (u32)(d1 >> 32));
            const HalfSlices bl = slice_half((u32)o1, (u32)d1, (u32)hz1, (u32)c, (u32)d2);
            const HalfSlices bh = slice_half((u32)(o1 >> 32), (u32)(d1 >> 32), (u32)(hz1 >> 32),
                                             (u32)(c >> 32), (u32)(d2 >> 32));
            up = two ? d1 : c;
            c = two ? d2 : d1;
            u32 ual = ~al.a2, uah = ~ah.a2, aal = 0, aah = 0;
            u32 ubl = ~bl.a2, ubh = ~bh.a2, abl = 0, abh = 0;
            const u32 wa = (u32)((long long)yc * nw + x), wb = wa + (u32)nw;
#pragma unroll
            for (int b = 0; b < K; ++b) {
                const uint4 m = lvmask[b];
                const u32x4 ra =
                    philox4x32_10<true>(wg + wa, p.t, p.color, 1u + (u32)b, p.k0, p.k1);
                const u32x4 rb =
                    philox4x32_10<true>(wg + wb, p.t, p.color, 1u + (u32)b, p.k0, p.k1);
                block_levels(ra, m, al.a1, ah.a1, ual, uah, aal, aah);
                block_levels(rb, m, bl.a1, bh.a1, ubl, ubh, abl, abh);
            }
            const u32 ral = (u32)o0 ^ al.a2 ^ aal, rah = (u32)(o0 >> 32) ^ ah.a2 ^ aah;
            const u32 rbl = (u32)o1 ^ bl.a2 ^ abl, rbh = (u32)(o1 >> 32) ^ bh.a2 ^ abh;
            const bool ka = (ual | uah) != 0, kb = two && (ubl | ubh) != 0;
            // every word is stored, decided or not: an undecided word's entry ends with the
            // store of its final value, and nothing else reads this colour during the
            // half-sweep (measured 0.6-0.8% faster than storing only the decided words here; in
            // the word-range walker 0.5% slower, so that one keeps the predicated store)
            p.own[wa] = (u64)ral | ((u64)rah << 32);
            if (two) p.own[wb] = (u64)rbl | ((u64)rbh << 32);
            const u32 kma = __ballot_sync(0xFFFFFFFFu, ka);
            const u32 kmb = __ballot_sync(0xFFFFFFFFu, kb);
            {
                const int pos = ka ? n + __popc(kma & lt) : kStripCap;
                q.idx[pos] = wa;
                q.lp[pos] = (u32)K;
                q.a1[pos] = (u64)al.a1 | ((u64)ah.a1 << 32);
                q.und[pos] = (u64)ual | ((u64)uah << 32);
                q.res[pos] = (u64)ral | ((u64)rah << 32);
            }
            n += __popc(kma);
            {
                const int pos = kb ? n + __popc(kmb & lt) : kStripCap;
                q.idx[pos] = wb;
                q.lp[pos] = (u32)K;
                q.a1[pos] = (u64)bl.a1 | ((u64)bh.a1 << 32);
                q.und[pos] = (u64)ubl | ((u64)ubh << 32);
                q.res[pos] = (u64)rbl | ((u64)rbh << 32);
            }
            n += __popc(kmb);
            __syncwarp();
        } else if (y >= y1 && n <= 32) {
            if (n > 0) stack_drain(p, q, n, lvmask, wg);
            break;
        } else {
            strip_pop(p, q, n, lvmask, wg);
        }
    }
}

// (M, E) contributions of rows [y0, y1) of a strip after the warp updated them.
__device__ __forceinline__ void msc_measure_strip(const MscHalf& p, int strip, int y0, int y1,
                                                  long long& m_acc, long long& e_acc)
{
    long long calls = 0, wmax = 0;
    const int x = strip * 32 + (threadIdx.x & 31);
    for (int y = y0; y < y1; ++y) msc_word<false>(p, y, x, m_acc, e_acc, calls, wmax);
}

// (M, E) contributions of words [begin, end) as they are now, one word per lane of the warp:
// run after the warp's msc_queue_range (and a __syncwarp) to measure the updated colour.
__device__ __forceinline__ void msc_measure_range(const MscHalf& p, long long begin, long long end,
                                                  int nw_shift, long long& m_acc,
                                                  long long& e_acc)
{
    long long calls = 0, wmax = 0;
    for (long long w = begin + (threadIdx.x & 31); w < end; w += 32) {
        const int y = (int)(nw_shift >= 0 ? (w >> nw_shift) : div_magic(w, p.nw_magic, p.nw));
        msc_word<false>(p, y, (int)(w - (long long)y * p.nw), m_acc, e_acc, calls, wmax);
    }
}

}  // namespace ising
