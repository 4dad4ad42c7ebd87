// Swendsen-Wang cluster updates of an int8 lattice (2D/3D), in its checkerboard layout.
//
// Local updates slow down critically near T_c (autocorrelation ~ L^2.17 sweeps in 2D); pyising
// equilibrates its starts and measures its Binder cumulants with a CPU Wolff sampler
// (src/pyising/cluster.py:32-104, src/pyising/validate.py:45-50,127-150).  Here the cluster
// update runs on the device: Swendsen-Wang (Phys. Rev. Lett. 58, 86 (1987)) with the
// connected components found by a lock-free union-find.
//
// One update at step t:
//   1. every bond joins a colour-0 site to a colour-1 site (the lattice is bipartite), so each
//      colour-0 site owns its 2d bonds and each bond is seen once.  A bond between aligned
//      spins is active with probability p = 1 - exp(-2 beta) (threshold p_bond on a uniform
//      u32 from Philox((n, t, kBondTag, k), key)).  The union-find runs on two levels, so that
//      the near-spanning clusters of the critical region do not funnel every union through a
//      few global roots: a CTA owns a tile of R rows x W positions of one plane, both colours
//      (16 x 32 by default), unites the active bonds inside the tile in shared memory, then
//      writes each site's tile-local root as its global label (sw_local_kernel); a second
//      kernel unites the active bonds that leave their tile in global memory (sw_cross_kernel).
//      Within a tile, pointer jumping then makes every node point at its root.  (The
//      single-level variant, every bond united in global memory by sw_bond_kernel, is kept
//      behind the cluster_tile knob.)
//      On both levels roots are linked larger-under-smaller with atomicCAS and finds halve
//      paths with plain stores (parents only ever move up the tree, so a stale read is still
//      an ancestor); the tile order of sites is their global order, so the final root of a
//      cluster is its smallest site whatever the tile size;
//   2. every label is replaced by its root (a read-only walk: only thread i writes label[i]);
//      in 2D the flips walk to the roots themselves instead;
//   3. every cluster flips with probability 1/2: bit (root & 127) of
//      Philox((root >> 7, t, kFlipTag, 0), key), the same for all its sites.
// Site g = c * S + row * lh + j (S = rows * lh sites per colour, the logical compressed index).
// Labels are int32 (lattices of fewer than 2^31 sites).  Every retry loop is bounded: a thread
// that exceeds the bound sets the error word and stops, and the host reports ISING_ERR_TIMEOUT.
#include "capi_internal.h"

namespace ising {

constexpr u32 kBondTag = 0x53570001u;  // Philox counter word 2 of the bond uniforms
constexpr u32 kFlipTag = 0x53570002u;  // ... of the cluster flip bits
// Bounded loops: one union (its finds and retries) or one root walk may take at most kStepLimit
// steps (about 0.3 s of dependent L2 reads; legitimate walks are far shorter), and every loop
// gives up as soon as any thread has set the error word, which it reads every kErrPoll steps.
// A thread that runs out sets the error word, so one cycle in the labels (which a correct
// union-find never makes) ends the whole launch within milliseconds and the host reports
// ISING_ERR_TIMEOUT with the context intact.
constexpr int kStepLimit = 1 << 20;
constexpr int kErrPoll = 64;

struct StepBudget {
    int left = kStepLimit;
    bool dead = false;
};

// One more step of a bounded loop; false (and the error word set) when the budget is spent or
// another thread has set the error word.
__device__ __forceinline__ bool step(StepBudget& b, int* err)
{
    if (b.dead) return false;
    if (--b.left < 0) {
        atomicExch(err, 1);
        b.dead = true;
        return false;
    }
    if ((b.left & (kErrPoll - 1)) == 0 && *(volatile int*)err) {
        b.dead = true;
        return false;
    }
    return true;
}

struct ClusterArgs {
    int8_t* c[2];
    int* label;
    unsigned char* bonds;  // per colour-0 site, bit k = bond k active
    int* err;
    long long S;           // sites per colour
    long long rows;
    int lh, ly, lz, pitch, ndim;
    u32 t, k0, k1, p_bond;
};

__device__ __forceinline__ int uf_find(int* label, int x, int* err, StepBudget& b)
{
    while (step(b, err)) {
        const int p = __ldcg(label + x);
        if (p == x) return x;
        const int gp = __ldcg(label + p);
        if (gp != p) label[x] = gp;  // path halving
        x = gp;
    }
    return x;
}

// The root of x without writing anything: flattening must not halve paths, or a halving store
// (label[x] = grandparent) could overwrite the root another thread has just written to label[x].
__device__ __forceinline__ int uf_root(const int* label, int x, int* err)
{
    StepBudget b;
    while (step(b, err)) {
        const int p = __ldcg(label + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ __forceinline__ void uf_union(int* label, int a, int b, int* err)
{
    StepBudget budget;  // shared by the finds and the retries of this union
    while (step(budget, err)) {
        a = uf_find(label, a, err, budget);
        b = uf_find(label, b, err, budget);
        if (budget.dead || a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        // link root b under root a, unless b stopped being a root meanwhile
        const int old = atomicCAS(label + b, b, a);
        if (old == b) return;
        b = old;
    }
}

// Test hook (ISING_KNOB_TEST_LABEL_CYCLE): a two-site cycle in the labels, which the root walks
// after it can only leave through their step budgets.
__global__ void sw_cycle_kernel(int* label, long long S)
{
    label[0] = (int)S;
    label[S] = 0;
}

// Colour-1 positions of the 2d bonds of colour-0 site n (the order of the bond bits): the same
// index, the other horizontal neighbour, y + 1, y - 1, z + 1, z - 1 (periodic).
__device__ __forceinline__ void bond_ends(const ClusterArgs& a, long long n, long long nb[6])
{
    const long long row = n / a.lh;
    const int j = (int)(n - row * a.lh);
    const int y = (int)(row % a.ly), z = (int)(row / a.ly);
    const int par = (y + z) & 1;  // colour 0
    const long long plane = (long long)z * a.ly;
    nb[0] = row * a.lh + j;
    nb[1] = row * a.lh + (par ? (j + 1 == a.lh ? 0 : j + 1) : (j == 0 ? a.lh - 1 : j - 1));
    nb[2] = (plane + (y + 1 == a.ly ? 0 : y + 1)) * a.lh + j;
    nb[3] = (plane + (y == 0 ? a.ly - 1 : y - 1)) * a.lh + j;
    nb[4] = ((long long)(z + 1 == a.lz ? 0 : z + 1) * a.ly + y) * a.lh + j;
    nb[5] = ((long long)(z == 0 ? a.lz - 1 : z - 1) * a.ly + y) * a.lh + j;
}

__device__ __forceinline__ int8_t colour1_spin(const ClusterArgs& a, long long m)
{
    const long long mrow = m / a.lh;
    return a.c[1][mrow * a.pitch + (m - mrow * a.lh)];
}

// Shared-memory union-find of one tile (same rules and bounds as the global one).
__device__ __forceinline__ int tile_find(volatile int* lab, int x, int* err, StepBudget& b)
{
    while (step(b, err)) {
        const int p = lab[x];
        if (p == x) return x;
        const int gp = lab[p];
        if (gp != p) lab[x] = gp;
        x = gp;
    }
    return x;
}

__device__ __forceinline__ int tile_root(const volatile int* lab, int x, int* err)
{
    StepBudget b;
    while (step(b, err)) {
        const int p = lab[x];
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ __forceinline__ void tile_union(int* lab, int a, int b, int* err)
{
    StepBudget budget;
    while (step(budget, err)) {
        a = tile_find(lab, a, err, budget);
        b = tile_find(lab, b, err, budget);
        if (budget.dead || a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicCAS(lab + b, b, a);
        if (old == b) return;
        b = old;
    }
}

// Rectangular tiles: a tile is R rows x W positions of one plane (y in [y0, y0 + R), j in
// [j0, j0 + W), clipped at the plane's edges), of both colours; its local index of position
// (r, c) is r * W + c for colour 0 and R * W + r * W + c for colour 1, which orders a tile's
// sites as their global indices do.
struct TileGeo {
    int R, W;        // rows and positions per tile
    int tx, ty;      // tiles per row of positions, per plane
};

__device__ __forceinline__ void tile_origin(const ClusterArgs& a, const TileGeo& g, long long b,
                                           int& z, int& y0, int& j0)
{
    const long long per_plane = (long long)g.tx * g.ty;
    z = (int)(b / per_plane);
    const int rem = (int)(b - (long long)z * per_plane);
    const int by = rem / g.tx;
    y0 = by * g.R;
    j0 = (rem - by * g.tx) * g.W;
}

// Colour-1 coordinates (y, j, z) of bond k of colour-0 site (y, j, z) (the order of the bond
// bits), periodic.
__device__ __forceinline__ void bond_end(const ClusterArgs& a, int k, int y, int j, int z,
                                         int& ny, int& nj, int& nz)
{
    ny = y;
    nj = j;
    nz = z;
    if (k == 1) {
        const int par = (y + z) & 1;  // colour 0
        nj = par ? (j + 1 == a.lh ? 0 : j + 1) : (j == 0 ? a.lh - 1 : j - 1);
    } else if (k == 2) {
        ny = y + 1 == a.ly ? 0 : y + 1;
    } else if (k == 3) {
        ny = y == 0 ? a.ly - 1 : y - 1;
    } else if (k == 4) {
        nz = z + 1 == a.lz ? 0 : z + 1;
    } else if (k == 5) {
        nz = z == 0 ? a.lz - 1 : z - 1;
    }
}

// Tile b: draws the bonds of the tile's colour-0 sites, stores their masks, unites the active
// bonds that stay in the tile (shared memory), flattens the tile's trees and writes every tile
// site's label: the global index of its tile-local root.
__global__ void __launch_bounds__(256) sw_local_kernel(const ClusterArgs a, const TileGeo g)
{
    extern __shared__ int lab[];  // [2 R W]
    int z, y0, j0;
    tile_origin(a, g, blockIdx.x, z, y0, j0);
    const int R = g.R, W = g.W, RW = R * W;
    const int rn = a.ly - y0 < R ? a.ly - y0 : R;  // rows of this tile
    const int wn = a.lh - j0 < W ? a.lh - j0 : W;  // positions per row of this tile
    for (int i = threadIdx.x; i < 2 * RW; i += blockDim.x) lab[i] = i;
    __syncthreads();
    const int nbonds = 2 * a.ndim;
    const long long plane = (long long)z * a.ly;
    for (int i = threadIdx.x; i < rn * wn; i += blockDim.x) {
        const int r = i / wn, c = i - (i / wn) * wn;
        const int y = y0 + r, j = j0 + c;
        const long long row = plane + y;
        const long long q = row * a.lh + j;
        const int8_t s = a.c[0][row * a.pitch + j];
        const u32x4 r0 = philox4x32_10((u32)q, a.t, kBondTag, 0u, a.k0, a.k1);
        u32x4 r1 = {0u, 0u, 0u, 0u};
        if (a.ndim == 3) r1 = philox4x32_10((u32)q, a.t, kBondTag, 1u, a.k0, a.k1);
        const u32 u[6] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y};
        unsigned mask = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k >= nbonds) break;
            if (u[k] >= a.p_bond) continue;
            int ny, nj, nz;
            bond_end(a, k, y, j, z, ny, nj, nz);
            const long long nrow = (long long)nz * a.ly + ny;
            if (a.c[1][nrow * a.pitch + nj] != s) continue;
            mask |= 1u << k;
            if (nz == z && ny >= y0 && ny < y0 + rn && nj >= j0 && nj < j0 + wn)
                tile_union(lab, r * W + c, RW + (ny - y0) * W + (nj - j0), a.err);
        }
        a.bonds[q] = (unsigned char)mask;
    }
    __syncthreads();
    // Pointer jumping until every node points at its root: a concurrent reader sees the old
    // parent or the grandparent, both ancestors, so walks stay valid; log2(depth) rounds.
    volatile int* vlab = lab;
    for (int round = 0; round < 32; ++round) {
        int changed = 0;
        for (int i = threadIdx.x; i < 2 * rn * wn; i += blockDim.x) {
            const int cc = i >= rn * wn;
            const int ii = i - cc * rn * wn;
            const int li = cc * RW + (ii / wn) * W + (ii - (ii / wn) * wn);
            const int p = vlab[li];
            const int gp = vlab[p];
            if (gp != p) {
                vlab[li] = gp;
                changed = 1;
            }
        }
        if (!__syncthreads_or(changed && !*(volatile int*)a.err)) break;
    }
    for (int i = threadIdx.x; i < 2 * rn * wn; i += blockDim.x) {
        const int cc = i >= rn * wn;
        const int ii = i - cc * rn * wn;
        const int r = ii / wn, c = ii - (ii / wn) * wn;
        const int li = cc * RW + r * W + c;
        const int root = tile_root(lab, li, a.err);
        const int rc = root >= RW;
        const int rl = root - rc * RW;
        const long long gi = (long long)cc * a.S + (plane + y0 + r) * a.lh + j0 + c;
        const long long gr = (long long)rc * a.S + (plane + y0 + rl / W) * a.lh + j0 + rl % W;
        a.label[gi] = (int)gr;
    }
}

// Single-level variant (cluster_tile knob 1): every site its own tree, then every colour-0 site
// draws its bonds and unites the active ones in global memory directly.
__global__ void sw_init_kernel(int* label, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        label[i] = (int)i;
}

__global__ void sw_bond_kernel(const ClusterArgs a)
{
    const int nbonds = 2 * a.ndim;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.S;
         q += (long long)gridDim.x * blockDim.x) {
        const long long row = q / a.lh;
        const int8_t s = a.c[0][row * a.pitch + (q - row * a.lh)];
        long long nb[6];
        bond_ends(a, q, nb);
        const u32x4 r0 = philox4x32_10((u32)q, a.t, kBondTag, 0u, a.k0, a.k1);
        u32x4 r1 = {0u, 0u, 0u, 0u};
        if (a.ndim == 3) r1 = philox4x32_10((u32)q, a.t, kBondTag, 1u, a.k0, a.k1);
        const u32 u[6] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y};
        unsigned mask = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k >= nbonds) break;
            if (u[k] < a.p_bond && colour1_spin(a, nb[k]) == s) {
                mask |= 1u << k;
                uf_union(a.label, (int)q, (int)(a.S + nb[k]), a.err);
            }
        }
        a.bonds[q] = (unsigned char)mask;
    }
}

// The active bonds that leave their colour-0 site's tile, united in global memory.
__global__ void sw_cross_kernel(const ClusterArgs a, const TileGeo g)
{
    const int nbonds = 2 * a.ndim;
    const u32 S = (u32)a.S, lh = (u32)a.lh, ly = (u32)a.ly;  // S < 2^31
    for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q < S; q += gridDim.x * blockDim.x) {
        const unsigned mask = a.bonds[q];
        if (!mask) continue;
        const u32 row = q / lh;
        const int j = (int)(q - row * lh);
        const int y = (int)(row % ly), z = (int)(row / ly);
        const int y0 = y / g.R * g.R, j0 = j / g.W * g.W;
        const int y1 = y0 + g.R < (int)ly ? y0 + g.R : (int)ly;  // the tile, clipped
        const int j1 = j0 + g.W < (int)lh ? j0 + g.W : (int)lh;
        // in 2D only sites on a tile's border rows or columns have bonds that leave it
        if (a.ndim == 2 && y > y0 && y < y1 - 1 && j > j0 && j < j1 - 1) continue;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k >= nbonds) break;
            if (!((mask >> k) & 1u)) continue;
            int ny, nj, nz;
            bond_end(a, k, y, j, z, ny, nj, nz);
            if (nz == z && ny >= y0 && ny < y1 && nj >= j0 && nj < j1) continue;
            const long long m = ((long long)nz * a.ly + ny) * a.lh + nj;
            uf_union(a.label, (int)q, (int)(a.S + m), a.err);
        }
    }
}

// Every label becomes its root; only thread i writes label[i], and every value it can hold
// meanwhile (its old parent or the root) is an ancestor, so other threads' walks stay valid.
__global__ void sw_flatten_kernel(int* label, long long n, int* err)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        label[i] = uf_root(label, (int)i, err);
}

// Step 3.  WALK: each site walks up to its root itself (read-only), with no flattening pass
// before; otherwise the labels are flat already.
template <bool WALK>
__global__ void sw_flip_kernel(const ClusterArgs a)
{
    const long long n = 2 * a.S;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
         g += (long long)gridDim.x * blockDim.x) {
        const int root = WALK ? uf_root(a.label, (int)g, a.err) : a.label[g];
        const u32x4 r = philox4x32_10((u32)root >> 7, a.t, kFlipTag, 0u, a.k0, a.k1);
        const u32 w = (root & 64) ? ((root & 32) ? r.w : r.z) : ((root & 32) ? r.y : r.x);
        if ((w >> (root & 31)) & 1u) {
            const int c = g >= a.S ? 1 : 0;
            const long long m = g - (long long)c * a.S;
            const long long row = m / a.lh;
            int8_t* p = (c ? a.c[1] : a.c[0]) + row * a.pitch + (m - row * a.lh);
            *p = (int8_t)(*p ^ (int8_t)0xFE);  // +1 <-> -1
        }
    }
}

static int cluster_setup(ising_sim* h)
{
    if (h->variant != ISING_VARIANT_INT8)
        return fail(ISING_ERR_INVALID, "cluster updates: int8 lattices only");
    const long long n = 2 * h->rows * (long long)h->lh;
    if (n >= 0x7FFFFFFFll)
        return fail(ISING_ERR_INVALID, "cluster updates: lattices of fewer than 2^31 sites");
    if (!h->d_label) {  // labels, the error word, then one bond mask per colour-0 site
        cudaError_t e =
            cudaMalloc((void**)&h->d_label, (size_t)n * sizeof(int) + 256 + (size_t)(n / 2));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(ISING_ERR_NOMEM, "cudaMalloc of the cluster labels (%lld sites)", n);
        }
    }
    return ISING_OK;
}

// Tile shape of the shared-memory union-find: about T positions (the handle's cluster_tile
// knob, else kTileAuto) as R rows x W positions, W = 32 (16 for small T) or the row length;
// T = 0: the single-level union-find in global memory (knob value 1).  Small tiles give many
// CTAs and short trees, square-ish ones keep most bonds inside their tile.  Measured per update
// on B200 (single-level / 16 x 32 tiles): 256^2 52 / 39 us, 1024^2 199 / 85 us, 4096^2 2969 /
// 813 us, 256^3 2996 / 1062 us.
constexpr int kTileAuto = 512;

static int cluster_tiles(const ising_sim* h, TileGeo* g)
{
    if (h->cluster_tile == 1) return 0;
    const int T = h->cluster_tile > 0 ? h->cluster_tile : kTileAuto;
    g->W = T >= 256 ? 32 : 16;
    if (g->W > h->lh) g->W = h->lh;
    g->R = T / g->W;
    if (g->R < 1) g->R = 1;
    if (g->R > h->ly) g->R = h->ly;
    g->tx = (h->lh + g->W - 1) / g->W;
    g->ty = (h->ly + g->R - 1) / g->R;
    return g->tx * g->ty * h->lz;
}

static unsigned char* cluster_masks(ising_sim* h, long long S)
{
    return reinterpret_cast<unsigned char*>(h->d_label) + 2 * S * sizeof(int) + 256;
}

// One labeling (step 1-2) and, when `flip`, the cluster flips (step 3).
static int cluster_step(ising_sim* h, u32 t, u64 seed, u32 p_bond, bool flip)
{
    ClusterArgs a;
    a.c[0] = (int8_t*)h->c[0];
    a.c[1] = (int8_t*)h->c[1];
    a.S = h->rows * (long long)h->lh;
    a.label = h->d_label;
    a.err = reinterpret_cast<int*>(reinterpret_cast<char*>(h->d_label) + 2 * a.S * sizeof(int));
    a.bonds = cluster_masks(h, a.S);
    a.rows = h->rows;
    a.lh = h->lh;
    a.ly = h->ly;
    a.lz = h->lz;
    a.pitch = h->pitch;
    a.ndim = h->ndim;
    a.t = t;
    a.k0 = (u32)seed;
    a.k1 = (u32)(seed >> 32);
    a.p_bond = p_bond;
    const int grid = h->sm_count * 8;
    TileGeo g;
    const int tiles = cluster_tiles(h, &g);
    if (tiles > 0) {
        sw_local_kernel<<<(unsigned)tiles, 256, (size_t)2 * g.R * g.W * sizeof(int), h->stream>>>(
            a, g);
        sw_cross_kernel<<<grid, 256, 0, h->stream>>>(a, g);
    } else {
        sw_init_kernel<<<grid, 256, 0, h->stream>>>(a.label, 2 * a.S);
        sw_bond_kernel<<<grid, 256, 0, h->stream>>>(a);
    }
    if (h->test_label_cycle) sw_cycle_kernel<<<1, 1, 0, h->stream>>>(a.label, a.S);
    // 2D: the flips walk to the roots themselves (no flattening pass); 3D, where the trees of
    // the tiles' roots are deeper (every z bond leaves its tile), measured faster flattened first
    // (256^3: 1046 vs 1131 us per update; 1024^2: 79 vs 85 us the other way round)
    const bool walk = flip && h->ndim == 2;
    if (!walk) sw_flatten_kernel<<<grid, 256, 0, h->stream>>>(a.label, 2 * a.S, a.err);
    if (walk) sw_flip_kernel<true><<<grid, 256, 0, h->stream>>>(a);
    else if (flip) sw_flip_kernel<false><<<grid, 256, 0, h->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "cluster update launch");
    return ISING_OK;
}

static int cluster_error(ising_sim* h)
{
    const long long S = h->rows * (long long)h->lh;
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, reinterpret_cast<char*>(h->d_label) + 2 * S * sizeof(int),
                                    sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cluster update");
    if (err) return fail(ISING_ERR_TIMEOUT, "a bounded union-find loop of the cluster update gave up");
    return ISING_OK;
}

}  // namespace ising

using namespace ising;

extern "C" int ising_cluster_sweep(ising_sim* h, uint64_t step0, int64_t n_steps, uint64_t seed,
                                   uint32_t p_bond, int64_t* series_out)
{
    if (!h) return fail(ISING_ERR_INVALID, "null handle");
    if (n_steps < 0) return fail(ISING_ERR_INVALID, "negative step count");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    int rc = cluster_setup(h);
    if (rc != ISING_OK) return rc;
    if (series_out && n_steps > 0) {
        rc = ensure_series(h, n_steps);
        if (rc != ISING_OK) return rc;
        e = cudaMemsetAsync(h->d_series, 0, (size_t)n_steps * 2 * sizeof(long long), h->stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync (series)");
    }
    const long long S = h->rows * (long long)h->lh;
    e = cudaMemsetAsync(reinterpret_cast<char*>(h->d_label) + 2 * S * sizeof(int), 0, sizeof(int),
                        h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    for (int64_t k = 0; k < n_steps; ++k) {
        rc = cluster_step(h, (u32)(step0 + (uint64_t)k), seed, p_bond, true);
        if (rc == ISING_OK && series_out)
            rc = observe(h, reinterpret_cast<unsigned long long*>(h->d_series + 2 * k));
        if (rc != ISING_OK) return rc;
    }
    rc = cluster_error(h);
    if (rc == ISING_OK && series_out && n_steps > 0) {
        e = cudaMemcpyAsync(series_out, h->d_series, (size_t)n_steps * 2 * sizeof(long long),
                            cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(e, "cluster series copy");
    }
    return rc;
}

extern "C" int ising_cluster_labels(ising_sim* h, uint64_t step, uint64_t seed, uint32_t p_bond,
                                    int32_t* labels_out, uint8_t* bonds_out)
{
    if (!h || !labels_out || !bonds_out) return fail(ISING_ERR_INVALID, "null argument");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    int rc = cluster_setup(h);
    if (rc != ISING_OK) return rc;
    const long long S = h->rows * (long long)h->lh;
    e = cudaMemsetAsync(reinterpret_cast<char*>(h->d_label) + 2 * S * sizeof(int), 0, sizeof(int),
                        h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    rc = cluster_step(h, (u32)step, seed, p_bond, false);
    if (rc == ISING_OK) rc = cluster_error(h);
    if (rc == ISING_OK) {
        e = cudaMemcpyAsync(labels_out, h->d_label, (size_t)(2 * S) * sizeof(int),
                            cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(bonds_out, cluster_masks(h, S), (size_t)S, cudaMemcpyDeviceToHost,
                                h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "cluster labels copy");
    }
    return rc;
}
