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
        orc_int8_half(c0, c1, ndim, shape, 0, t, seed, table, heatbath);
        orc_int8_half(c1, c0, ndim, shape, 1, t, seed, table, heatbath);
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
