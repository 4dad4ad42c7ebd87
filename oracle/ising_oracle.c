/*
 * CPU oracle for the pyising sweep hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the algorithm of pyising's NumPy backend so that the CUDA
 * product can be checked bit for bit.  Only tests/, __graft_entry__.smoke() and the CPU legs
 * of bench.py load it; the product library never links or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py compares every function here with golden
 * vectors that tests/golden/make_golden.py produced by running the reference itself.
 *
 * Reference algorithm (file:line inside the pyising project):
 *   Philox4x32-10 ............ src/pyising/philox.py:26-51
 *   split_seed ............... src/pyising/philox.py:20-23
 *   int8 site stream ......... src/pyising/philox.py:54-64
 *   msc word stream .......... src/pyising/philox.py:67-78
 *   threshold table .......... src/pyising/lattice.py:121-142
 *   int8 half-sweep .......... src/pyising/backends/numpy_backend.py:26-44
 *   msc flip mask/half-sweep . src/pyising/backends/numpy_backend.py:54-83,103-124
 *   sweep loop ............... src/pyising/backends/base.py:85-90
 *   observables .............. src/pyising/lattice.py:108-118 and
 *                              src/pyising/backends/observables_torch.py:46-111
 *
 * Layout: colour arrays are (rows, Lh) with rows = prod(shape[:-1]), Lh = Lx/2.  For 3D the
 * shape is (Lz, Ly, Lx) and row r = z*Ly + y; in 2D the shape is (Ly, Lx) and r = y.  Colour c
 * of row r sits at x = 2j + ((y + z + c) % 2).  Packed (msc) rows hold Lh/64 uint64 words, bit b
 * of word w being compressed site 64w+b (1 = spin +1).
 *
 * Threads: the row loops are OpenMP-parallel (orc_set_threads); results do not depend on the
 * thread count because every site's random number is keyed by (site, sweep, colour, seed).
 * The int8 sweeps use an AVX-512 variant of the half-sweep on hosts that have it (orc_set_fast;
 * bit-identical to the plain one, both pinned to the golden vectors).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

/* Philox4x32-10: ten rounds, key bumped between rounds (philox.py:40-50). */
static inline void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                          uint32_t k1, uint32_t out[4])
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        const uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_philox(const uint32_t *ctr, uint32_t k0, uint32_t k1, uint32_t *out)
{
    philox(ctr[0], ctr[1], ctr[2], ctr[3], k0, k1, out);
}

/* Bulk Philox over counters (q0+i, c1, c2, c3), i < n: out is (n, 4). */
void orc_philox_range(uint64_t q0, int64_t n, uint32_t c1, uint32_t c2, uint32_t c3,
                      uint32_t k0, uint32_t k1, uint32_t *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        philox((uint32_t)(q0 + (uint64_t)i), c1, c2, c3, k0, k1, out + 4 * i);
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* prob_to_threshold / threshold_table (lattice.py:121-142). algorithm 0 = Metropolis, 1 = heat
 * bath. Out has 2*ndim+1 entries indexed by (X + 2 ndim) / 2. */
static uint32_t prob_to_threshold(double p)
{
    if (p >= 1.0) return 0xFFFFFFFFu;
    double v = floor(p * 4294967296.0);
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

void orc_threshold_table(double beta, int ndim, int algorithm, uint32_t *out)
{
    const int z = 2 * ndim;
    for (int i = 0; i <= z; ++i) {
        const int x = -z + 2 * i;
        if (algorithm == 0)
            out[i] = x <= 0 ? 0xFFFFFFFFu : prob_to_threshold(exp(-2.0 * beta * x));
        else
            out[i] = prob_to_threshold(1.0 / (1.0 + exp(-2.0 * beta * x)));
    }
}

typedef struct {
    int ndim;
    int64_t lz, ly, lh, rows;
} geom_t;

static geom_t make_geom(int ndim, const int64_t *shape)
{
    geom_t g;
    g.ndim = ndim;
    if (ndim == 3) { g.lz = shape[0]; g.ly = shape[1]; g.lh = shape[2] / 2; }
    else { g.lz = 1; g.ly = shape[0]; g.lh = shape[1] / 2; }
    g.rows = g.lz * g.ly;
    return g;
}

/* One colour of the int8 checkerboard (numpy_backend.py:26-44). */
void orc_int8_half(int8_t *own, const int8_t *other, int ndim, const int64_t *shape, int color,
                   uint32_t t, uint64_t seed, const uint32_t *table, int heatbath)
{
    const geom_t g = make_geom(ndim, shape);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int z2 = 2 * ndim;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < g.rows; ++r) {
        const int64_t y = r % g.ly, zz = r / g.ly;
        const int p = (int)((y + zz + color) & 1);
        const int64_t ryu = zz * g.ly + (y + 1 == g.ly ? 0 : y + 1);
        const int64_t ryd = zz * g.ly + (y == 0 ? g.ly - 1 : y - 1);
        const int64_t rzu = (zz + 1 == g.lz ? 0 : zz + 1) * g.ly + y;
        const int64_t rzd = (zz == 0 ? g.lz - 1 : zz - 1) * g.ly + y;
        const int8_t *o = other + r * g.lh;
        uint32_t rnd[4];
        int64_t last_q = -1;
        for (int64_t j = 0; j < g.lh; ++j) {
            int h = o[j];
            if (p) h += o[j + 1 == g.lh ? 0 : j + 1];
            else h += o[j == 0 ? g.lh - 1 : j - 1];
            h += other[ryu * g.lh + j] + other[ryd * g.lh + j];
            if (ndim == 3) h += other[rzu * g.lh + j] + other[rzd * g.lh + j];
            const int64_t n = r * g.lh + j;
            const int64_t q = n >> 2;
            if (q != last_q) {
                philox((uint32_t)q, t, (uint32_t)color, 0u, k0, k1, rnd);
                last_q = q;
            }
            const uint32_t u = rnd[n & 3];
            const int s = own[n];
            if (heatbath) {
                own[n] = (u < table[(h + z2) / 2]) ? 1 : -1;
            } else {
                const int x = s * h;
                own[n] = (x <= 0 || u < table[(x + z2) / 2]) ? (int8_t)-s : (int8_t)s;
            }
        }
    }
}

/* ---- the same half-sweep, vectorised with AVX-512 (x86-64 hosts that have it) -----------------
 * Bit-identical to orc_int8_half (tests/test_oracle_golden.py checks both against each other
 * and the golden vectors); it only makes the full-size parity runs affordable.  Per row: the
 * row's Philox blocks sixteen at a time (32x32->64 products of even and odd lanes with
 * vpmuludq), transposed into site order; then 64 sites per step: int8 neighbour sums, the
 * table entry by a permute, an unsigned compare. */
#if defined(__x86_64__) && defined(__GNUC__)
#include <immintrin.h>
#define ORC_AVX512 __attribute__((target("avx512f,avx512bw")))

ORC_AVX512 static inline __m512i mulhi_lo(__m512i x, __m512i m, __m512i *lo)
{
    const __m512i pe = _mm512_mul_epu32(x, m);
    const __m512i po = _mm512_mul_epu32(_mm512_srli_epi64(x, 32), m);
    *lo = _mm512_mask_blend_epi32(0xAAAA, pe, _mm512_slli_epi64(po, 32));
    return _mm512_mask_blend_epi32(0xAAAA, _mm512_srli_epi64(pe, 32), po);
}

/* Philox blocks (q0 + i, c1, c2, c3), i < 16, written in site order: out[4 i + w] = word w of
 * block i. */
ORC_AVX512 static void philox16(uint32_t q0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                uint32_t k1, uint32_t *out)
{
    __m512i x0 = _mm512_add_epi32(_mm512_set1_epi32((int)q0),
                                  _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13,
                                                    14, 15));
    __m512i x1 = _mm512_set1_epi32((int)c1), x2 = _mm512_set1_epi32((int)c2);
    __m512i x3 = _mm512_set1_epi32((int)c3);
    const __m512i m0 = _mm512_set1_epi32((int)PHILOX_M0), m1 = _mm512_set1_epi32((int)PHILOX_M1);
    for (int r = 0; r < 10; ++r) {
        __m512i lo0, lo1;
        const __m512i hi0 = mulhi_lo(x0, m0, &lo0);
        const __m512i hi1 = mulhi_lo(x2, m1, &lo1);
        const __m512i n0 = _mm512_ternarylogic_epi32(hi1, x1, _mm512_set1_epi32((int)k0), 0x96);
        const __m512i n2 = _mm512_ternarylogic_epi32(hi0, x3, _mm512_set1_epi32((int)k1), 0x96);
        x1 = lo1;
        x3 = lo0;
        x0 = n0;
        x2 = n2;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    /* 4 x 16 -> site order: 128-bit lane k of u_m holds block 4k + m after the unpacks */
    const __m512i t0 = _mm512_unpacklo_epi32(x0, x1), t1 = _mm512_unpackhi_epi32(x0, x1);
    const __m512i t2 = _mm512_unpacklo_epi32(x2, x3), t3 = _mm512_unpackhi_epi32(x2, x3);
    const __m512i u0 = _mm512_unpacklo_epi64(t0, t2), u1 = _mm512_unpackhi_epi64(t0, t2);
    const __m512i u2 = _mm512_unpacklo_epi64(t1, t3), u3 = _mm512_unpackhi_epi64(t1, t3);
    const __m512i a = _mm512_shuffle_i32x4(u0, u1, 0x44), b = _mm512_shuffle_i32x4(u2, u3, 0x44);
    const __m512i c = _mm512_shuffle_i32x4(u0, u1, 0xEE), d = _mm512_shuffle_i32x4(u2, u3, 0xEE);
    _mm512_storeu_si512((void *)(out + 0), _mm512_shuffle_i32x4(a, b, 0x88));
    _mm512_storeu_si512((void *)(out + 16), _mm512_shuffle_i32x4(a, b, 0xDD));
    _mm512_storeu_si512((void *)(out + 32), _mm512_shuffle_i32x4(c, d, 0x88));
    _mm512_storeu_si512((void *)(out + 48), _mm512_shuffle_i32x4(c, d, 0xDD));
}

/* 16 sites: flip / set mask from int8 values v (x = s h for Metropolis, h for heat bath). */
ORC_AVX512 static inline __mmask16 decide16(__m128i v8, const uint32_t *u, __m512i tab,
                                            int z2, int heatbath)
{
    const __m512i v = _mm512_cvtepi8_epi32(v8);
    const __m512i idx = _mm512_srai_epi32(_mm512_add_epi32(v, _mm512_set1_epi32(z2)), 1);
    const __m512i thr = _mm512_permutexvar_epi32(idx, tab);
    const __mmask16 lt = _mm512_cmplt_epu32_mask(_mm512_loadu_si512((const void *)u), thr);
    if (heatbath) return lt;
    return lt | _mm512_cmple_epi32_mask(v, _mm512_setzero_si512());
}

ORC_AVX512 static void int8_half_avx512(int8_t *own, const int8_t *other, int ndim,
                                        const int64_t *shape, int color, uint32_t t,
                                        uint64_t seed, const uint32_t *table, int heatbath)
{
    const geom_t g = make_geom(ndim, shape);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int z2 = 2 * ndim;
    uint32_t tab16[16];
    for (int i = 0; i < 16; ++i) tab16[i] = i <= z2 ? table[i] : 0u;
    const __m512i tab = _mm512_loadu_si512((const void *)tab16);
#pragma omp parallel
    {
        uint32_t *ubuf = (uint32_t *)malloc((size_t)(g.lh + 128) * sizeof(uint32_t));
        int8_t *row = (int8_t *)malloc((size_t)g.lh + 2);
#pragma omp for schedule(static)
        for (int64_t r = 0; r < g.rows; ++r) {
            const int64_t y = r % g.ly, zz = r / g.ly;
            const int p = (int)((y + zz + color) & 1);
            const int8_t *o = other + r * g.lh;
            const int8_t *yu = other + (zz * g.ly + (y + 1 == g.ly ? 0 : y + 1)) * g.lh;
            const int8_t *yd = other + (zz * g.ly + (y == 0 ? g.ly - 1 : y - 1)) * g.lh;
            const int8_t *zu = other + ((zz + 1 == g.lz ? 0 : zz + 1) * g.ly + y) * g.lh;
            const int8_t *zd = other + ((zz == 0 ? g.lz - 1 : zz - 1) * g.ly + y) * g.lh;
            /* site uniforms of the row: ubuf[off + j] for site n = r lh + j */
            const int64_t n0 = r * g.lh, q0 = n0 >> 2, q1 = (n0 + g.lh + 3) >> 2;
            for (int64_t q = q0; q < q1; q += 16)
                philox16((uint32_t)q, t, (uint32_t)color, 0u, k0, k1, ubuf + 4 * (q - q0));
            const uint32_t *u = ubuf + (n0 & 3);
            /* the row with its wrapped ends: row[1 + j] = o[j] */
            row[0] = o[g.lh - 1];
            memcpy(row + 1, o, (size_t)g.lh);
            row[g.lh + 1] = o[0];
            const int8_t *side = p ? row + 2 : row;
            int8_t *s = own + r * g.lh;
            for (int64_t j = 0; j < g.lh; j += 64) {
                const int64_t left = g.lh - j;
                const __mmask64 m = left >= 64 ? ~(__mmask64)0 : (((__mmask64)1 << left) - 1);
                __m512i h = _mm512_add_epi8(_mm512_maskz_loadu_epi8(m, o + j),
                                            _mm512_maskz_loadu_epi8(m, side + j));
                h = _mm512_add_epi8(h, _mm512_maskz_loadu_epi8(m, yu + j));
                h = _mm512_add_epi8(h, _mm512_maskz_loadu_epi8(m, yd + j));
                if (ndim == 3) {
                    h = _mm512_add_epi8(h, _mm512_maskz_loadu_epi8(m, zu + j));
                    h = _mm512_add_epi8(h, _mm512_maskz_loadu_epi8(m, zd + j));
                }
                const __m512i sv = _mm512_maskz_loadu_epi8(m, s + j);
                const __mmask64 neg = _mm512_movepi8_mask(sv);
                /* Metropolis decides on x = s h, heat bath on h */
                const __m512i v =
                    heatbath ? h : _mm512_mask_sub_epi8(h, neg, _mm512_setzero_si512(), h);
                __mmask64 f = 0;
                for (int k = 0; k < 4; ++k)
                    f |= (__mmask64)decide16(_mm512_extracti32x4_epi32(v, k), u + j + 16 * k, tab,
                                             z2, heatbath)
                         << (16 * k);
                __m512i out;
                if (heatbath) /* +1 where u < table, else -1 */
                    out = _mm512_mask_blend_epi8(f, _mm512_set1_epi8(-1), _mm512_set1_epi8(1));
                else
                    out = _mm512_mask_sub_epi8(sv, f, _mm512_setzero_si512(), sv);
                _mm512_mask_storeu_epi8(s + j, m, out);
            }
        }
        free(ubuf);
        free(row);
    }
}

static int avx512_ok(void)
{
    static int ok = -1;
    if (ok < 0) {
        __builtin_cpu_init();
        ok = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw");
    }
    return ok;
}
#else
static int avx512_ok(void) { return 0; }
static void int8_half_avx512(int8_t *own, const int8_t *other, int ndim, const int64_t *shape,
                             int color, uint32_t t, uint64_t seed, const uint32_t *table,
                             int heatbath)
{
    (void)own; (void)other; (void)ndim; (void)shape; (void)color; (void)t; (void)seed;
    (void)table; (void)heatbath;
}
#endif

/* 0 = the plain restatement above, 1 = the AVX-512 variant where the host has it (default). */
static int g_fast = 1;

void orc_set_fast(int on) { g_fast = on; }

int orc_fast_active(void) { return g_fast && avx512_ok(); }

static void int8_half(int8_t *own, const int8_t *other, int ndim, const int64_t *shape,
                      int color, uint32_t t, uint64_t seed, const uint32_t *table, int heatbath)
{
    if (orc_fast_active())
        int8_half_avx512(own, other, ndim, shape, color, t, seed, table, heatbath);
    else
        orc_int8_half(own, other, ndim, shape, color, t, seed, table, heatbath);
}

/* Integer observables of the int8 layout: M = sum of spins, E = -sum over bonds s_i s_j.
 * Every bond has exactly one colour-0 end (observables_torch.py:3-4). */
void orc_int8_observables(const int8_t *c0, const int8_t *c1, int ndim, const int64_t *shape,
                          int64_t *m_out, int64_t *e_out)
{
    const geom_t g = make_geom(ndim, shape);
    int64_t msum = 0, esum = 0;
#pragma omp parallel for schedule(static) reduction(+ : msum, esum)
    for (int64_t r = 0; r < g.rows; ++r) {
        const int64_t y = r % g.ly, zz = r / g.ly;
        const int p = (int)((y + zz) & 1);
        const int64_t ryu = zz * g.ly + (y + 1 == g.ly ? 0 : y + 1);
        const int64_t ryd = zz * g.ly + (y == 0 ? g.ly - 1 : y - 1);
        const int64_t rzu = (zz + 1 == g.lz ? 0 : zz + 1) * g.ly + y;
        const int64_t rzd = (zz == 0 ? g.lz - 1 : zz - 1) * g.ly + y;
        const int8_t *o = c1 + r * g.lh;
        for (int64_t j = 0; j < g.lh; ++j) {
            int h = o[j];
            if (p) h += o[j + 1 == g.lh ? 0 : j + 1];
            else h += o[j == 0 ? g.lh - 1 : j - 1];
            h += c1[ryu * g.lh + j] + c1[ryd * g.lh + j];
            if (ndim == 3) h += c1[rzu * g.lh + j] + c1[rzd * g.lh + j];
            const int s = c0[r * g.lh + j];
            msum += s + o[j];
            esum += s * h;
        }
    }
    *m_out = msum;
    *e_out = -esum;
}

/* n full sweeps from sweep counter t0 (base.py:85-90); when measure_every > 0 the observables
 * after every measure_every-th sweep go to series[2*i] (M) and series[2*i+1] (E). */
void orc_int8_sweeps(int8_t *c0, int8_t *c1, int ndim, const int64_t *shape, uint64_t t0,
                     int64_t n, uint64_t seed, const uint32_t *table, int heatbath,
                     int64_t measure_every, int64_t *series)
{
    int64_t k = 0;
    for (int64_t s = 0; s < n; ++s) {
        const uint32_t t = (uint32_t)(t0 + (uint64_t)s);
        int8_half(c0, c1, ndim, shape, 0, t, seed, table, heatbath);
        int8_half(c1, c0, ndim, shape, 1, t, seed, table, heatbath);
        if (measure_every > 0 && (s + 1) % measure_every == 0 && series) {
            orc_int8_observables(c0, c1, ndim, shape, series + 2 * k, series + 2 * k + 1);
            ++k;
        }
    }
}

/* ------------------------------------------------ multi-spin coding (2D Metropolis) ------ */

/* Bit-sliced decision with the lazy MSB-first comparison (numpy_backend.py:54-83).  Level k
 * uses call k/2 of Philox(w, t, colour, 1 + k/2): even levels r0|r1<<32, odd r2|r3<<32
 * (philox.py:67-78).  Returns the flip mask; *calls gets the Philox calls used. */
static uint64_t msc_flip(uint64_t own, uint64_t n1, uint64_t n2, uint64_t n3, uint64_t n4,
                         uint32_t w, uint32_t t, uint32_t color, uint32_t k0, uint32_t k1,
                         uint32_t thr4, uint32_t thr8, int *calls)
{
    const uint64_t x1 = own ^ n1, x2 = own ^ n2, x3 = own ^ n3, x4 = own ^ n4;
    const uint64_t any = x1 | x2 | x3 | x4;
    const uint64_t a0 = ~any;
    const uint64_t s1 = x1 ^ x2, cy1 = x1 & x2, s2 = x3 ^ x4, cy2 = x3 & x4;
    const uint64_t a2 = cy1 | cy2 | (s1 & s2);
    const uint64_t a1 = any & ~a2;
    uint64_t acc = 0, und = a0 | a1;
    int nc = 0;
    for (int lp = 0; lp < 16 && und; ++lp) {
        uint32_t r[4];
        philox(w, t, color, 1u + (uint32_t)lp, k0, k1, r);
        ++nc;
        for (int half = 0; half < 2; ++half) {
            const int bit = 31 - (2 * lp + half);
            const uint64_t rv = half == 0 ? ((uint64_t)r[0] | ((uint64_t)r[1] << 32))
                                          : ((uint64_t)r[2] | ((uint64_t)r[3] << 32));
            const uint64_t t4 = ((thr4 >> bit) & 1u) ? ~0ull : 0ull;
            const uint64_t t8 = ((thr8 >> bit) & 1u) ? ~0ull : 0ull;
            const uint64_t tm = (a1 & t4) | (a0 & t8);
            acc |= und & ~rv & tm;
            und &= ~(rv ^ tm);
        }
    }
    if (calls) *calls = nc;
    return a2 | acc;
}

/* One colour of the packed lattice (numpy_backend.py:103-124); shape (Ly, Lx), Lx % 128 == 0.
 * Returns the total Philox calls (diagnostic). */
int64_t orc_msc_half(uint64_t *own, const uint64_t *other, const int64_t *shape, int color,
                     uint32_t t, uint64_t seed, uint32_t thr4, uint32_t thr8)
{
    const int64_t ly = shape[0], nw = shape[1] / 128;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    int64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int64_t y = 0; y < ly; ++y) {
        const int p = (int)((y + color) & 1);
        const uint64_t *o = other + y * nw;
        const uint64_t *up = other + (y == 0 ? ly - 1 : y - 1) * nw;
        const uint64_t *dn = other + (y + 1 == ly ? 0 : y + 1) * nw;
        for (int64_t x = 0; x < nw; ++x) {
            const uint64_t c = o[x];
            uint64_t hz;
            if (p) hz = (c >> 1) | (o[x + 1 == nw ? 0 : x + 1] << 63);
            else hz = (c << 1) | (o[x == 0 ? nw - 1 : x - 1] >> 63);
            const int64_t w = y * nw + x;
            int nc = 0;
            const uint64_t f = msc_flip(own[w], c, hz, up[x], dn[x], (uint32_t)w, t,
                                        (uint32_t)color, k0, k1, thr4, thr8, &nc);
            own[w] ^= f;
            total += nc;
        }
    }
    return total;
}

static inline int popc64(uint64_t v) { return __builtin_popcountll(v); }

/* Packed observables (observables_torch.py:85-111): M = 2 up - N, E = -(2N - 2 anti). */
void orc_msc_observables(const uint64_t *w0, const uint64_t *w1, const int64_t *shape,
                         int64_t *m_out, int64_t *e_out)
{
    const int64_t ly = shape[0], nw = shape[1] / 128;
    const int64_t n = shape[0] * shape[1];
    int64_t up = 0, anti = 0;
#pragma omp parallel for schedule(static) reduction(+ : up, anti)
    for (int64_t y = 0; y < ly; ++y) {
        const int p = (int)(y & 1);
        const uint64_t *o = w1 + y * nw;
        const uint64_t *u = w1 + (y == 0 ? ly - 1 : y - 1) * nw;
        const uint64_t *d = w1 + (y + 1 == ly ? 0 : y + 1) * nw;
        for (int64_t x = 0; x < nw; ++x) {
            const uint64_t s = w0[y * nw + x], c = o[x];
            uint64_t hz;
            if (p) hz = (c >> 1) | (o[x + 1 == nw ? 0 : x + 1] << 63);
            else hz = (c << 1) | (o[x == 0 ? nw - 1 : x - 1] >> 63);
            up += popc64(s) + popc64(c);
            anti += popc64(s ^ c) + popc64(s ^ hz) + popc64(s ^ u[x]) + popc64(s ^ d[x]);
        }
    }
    *m_out = 2 * up - n;
    *e_out = -(2 * n - 2 * anti);
}

int64_t orc_msc_sweeps(uint64_t *w0, uint64_t *w1, const int64_t *shape, uint64_t t0, int64_t n,
                       uint64_t seed, uint32_t thr4, uint32_t thr8, int64_t measure_every,
                       int64_t *series)
{
    int64_t k = 0, calls = 0;
    for (int64_t s = 0; s < n; ++s) {
        const uint32_t t = (uint32_t)(t0 + (uint64_t)s);
        calls += orc_msc_half(w0, w1, shape, 0, t, seed, thr4, thr8);
        calls += orc_msc_half(w1, w0, shape, 1, t, seed, thr4, thr8);
        if (measure_every > 0 && (s + 1) % measure_every == 0 && series) {
            orc_msc_observables(w0, w1, shape, series + 2 * k, series + 2 * k + 1);
            ++k;
        }
    }
    return calls;
}
