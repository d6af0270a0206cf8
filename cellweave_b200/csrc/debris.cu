// Debris loss on the device: break_down_debris and drain_shut_in of
// crates/engine/src/simulation.rs (1746-1826) over every history at once.
//
// A dead cell kept with a debris loss holds the volume it died with, and the
// dead tissue of a history owes the fluid `loss` of that volume each step
// (simulation.rs:1226-1244, 1255-1275).  Every whole pixel owed is taken at
// the tissue's edge: a dead pixel with living tissue of another cell across
// a face goes to one of those neighbours (close_over, cpm.rs:560-574), and
// once the edge is spent the pixels it laid bare, up to EDGE_PASSES times.
// The reference draws the pixels one at a time without replacement; here a
// pass takes each edge pixel with probability (owed - paid) / edge pixels,
// all of a pass decided against the lattice as it stood, so that a pass pays
// what is owed on average and the next pass (or step, through the carried
// debt) pays the difference.  Each dead cell then asks for what it gave up
// less.  Fluid shut in the tissue (medium the bath does not reach) with
// living tissue across a face goes to one of those neighbours, one layer a
// step (close_in, cpm.rs:592-606), decided against the lattice as it stood.
//
// Three passes over the sites per edge pass (find, draw, apply) and two for
// the fluid; the decisions go through a per-site scratch so that no pass
// reads what it writes.
#include <algorithm>
#include <cmath>

#include "cw_internal.cuh"

using namespace cw;

namespace {

constexpr int T = 256;
constexpr int EDGE_PASSES = 8;  // simulation.rs:151
constexpr int32_t OBST = -1;
constexpr int32_t EDGE = -2;  // a claim: an edge pixel, not drawn yet

__device__ __forceinline__ void xyz_of(int64_t i, int4 dm, int &x, int &y, int &z) {
    const int64_t slice = (int64_t)dm.x * dm.y;
    z = (int)(i / slice);
    const int64_t r = i - (int64_t)z * slice;
    y = (int)(r / dm.x);
    x = (int)(r - (int64_t)y * dm.x);
}

// The face neighbours of local pixel i (von_neumann, clipped at the walls)
// that are living tissue of a cell other than `self`: not the medium, an
// obstacle or necrotic (living_around, cpm.rs:709-722).  Their local indices
// into out[], their number returned.
__device__ __forceinline__ int living_around(const int32_t *g, int4 dm, int64_t i, int32_t self,
                                             const int32_t *type, int64_t cap, int necrotic, int64_t out[6]) {
    int x, y, z;
    xyz_of(i, dm, x, y, z);
    const int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    int64_t nb[6];
    int m = 0;
    if (x > 0) nb[m++] = i - 1;
    if (x + 1 < dm.x) nb[m++] = i + 1;
    if (y > 0) nb[m++] = i - w;
    if (y + 1 < dm.y) nb[m++] = i + w;
    if (dm.z > 1 && z > 0) nb[m++] = i - slice;
    if (dm.z > 1 && z + 1 < dm.z) nb[m++] = i + slice;
    int n = 0;
    for (int k = 0; k < m; ++k) {
        const int32_t o = g[nb[k]];
        if (o == self || o == 0 || o == OBST || o >= cap) continue;
        if (necrotic >= 0 && type[o] == necrotic) continue;
        out[n++] = nb[k];
    }
    return n;
}

__device__ __forceinline__ int history_of(const int32_t *blk, int nh) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    return s_h;
}

// What the kept dead of each history hold, and the share of it owed this
// step (simulation.rs:1243, 1272): one block per history.
__global__ void k_debris_owe(const int64_t *cell_off, const uint8_t *kept, const int32_t *volume, double loss,
                             double *owed, int64_t *held, int32_t *active) {
    const int h = blockIdx.x;
    const int64_t c0 = cell_off[h], c1 = cell_off[h + 1];
    unsigned long long v = 0;
    for (int64_t c = c0 + 1 + threadIdx.x; c < c1; c += blockDim.x)
        if (kept[c] && volume[c] > 0) v += (unsigned long long)volume[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ unsigned long long s[T / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s[k];
        held[h] = (int64_t)t;
        owed[h] += loss * (double)t;
        active[h] = floor(owed[h]) >= 1.0;
    }
}

// After a pass: a history that has paid what it owes sits out the rest.
__global__ void k_debris_still(int nh, const double *owed, const int32_t *paid, int32_t *active) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < nh && active[h] && (int64_t)floor(owed[h]) - (int64_t)paid[h] <= 0) active[h] = 0;
}

__device__ __forceinline__ int64_t still_owed(const double *owed, const int32_t *paid, int h) {
    return (int64_t)floor(owed[h]) - (int64_t)paid[h];
}

// Mark the edge: kept dead pixels with living tissue across a face.
__global__ void k_debris_edges(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                               const int32_t *blk, int nh, const int32_t *type, const uint8_t *kept, int necrotic,
                               const double *owed, const int32_t *paid, const int32_t *active, int32_t *claim,
                               int32_t *edges) {
    const int h = history_of(blk, nh);
    if (!active[h]) return;  // the whole block: its claims are not read this step
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int64_t gi = off[h] + i;
    claim[gi] = -1;
    if (still_owed(owed, paid, h) <= 0) return;
    const int32_t *g = grid + off[h];
    const int32_t id = g[i];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    if (id <= 0 || id >= cap || !kept[c0 + id]) return;
    int64_t nb[6];
    if (living_around(g, dims[h], i, id, type + c0, cap, necrotic, nb) == 0) return;
    claim[gi] = EDGE;
    atomicAdd(edges + h, 1);
}

// Draw the pixels this pass takes and who takes each.
__global__ void k_debris_draw(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                              const int32_t *blk, int nh, const int32_t *type, int necrotic, const double *owed,
                              const int32_t *paid, const int32_t *edges, const uint2 *keys, const uint32_t *step,
                              int pass, const int32_t *active, int32_t *claim) {
    const int h = history_of(blk, nh);
    if (!active[h]) return;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int64_t gi = off[h] + i;
    if (claim[gi] != EDGE) return;
    const int64_t want = still_owed(owed, paid, h);
    const int32_t e = edges[h];
    const uint4 r = philox((uint32_t)i, *step, 6u, (uint32_t)pass, keys[h].x, keys[h].y);
    if (want <= 0 || (want < e && u01(r.x, r.y) * (double)e >= (double)want)) {
        claim[gi] = -1;
        return;
    }
    const int32_t *g = grid + off[h];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    int64_t nb[6];
    const int n = living_around(g, dims[h], i, g[i], type + c0, cap, necrotic, nb);
    const int k = min((int)(u01(r.z, r.w) * n), n - 1);
    claim[gi] = g[nb[k]];
}

// Fluid shut in the tissue with living tissue across a face, and who takes
// each pixel (shut_in, can_close_in, close_in; cpm.rs:592-660).
__global__ void k_drain_draw(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                             const int32_t *blk, int nh, const int32_t *type, int necrotic, const uint8_t *bath,
                             const uint2 *keys, const uint32_t *step, int32_t *claim) {
    const int h = history_of(blk, nh);
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int64_t gi = off[h] + i;
    claim[gi] = -1;
    const int32_t *g = grid + off[h];
    if (g[i] != 0 || bath[gi]) return;
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    int64_t nb[6];
    const int n = living_around(g, dims[h], i, 0, type + c0, cap, necrotic, nb);
    if (n == 0) return;
    const uint4 r = philox((uint32_t)i, *step, 7u, 0u, keys[h].x, keys[h].y);
    claim[gi] = g[nb[min((int)(u01(r.x, r.y) * n), n - 1)]];
}

// Hand each claimed pixel to its taker; a cell's loss counted in `given`
// and the history's in `paid` (the medium's is not counted).
__global__ void k_claims_apply(int32_t *grid, const int64_t *off, const int64_t *cell_off, const int32_t *blk, int nh,
                               const int32_t *claim, int32_t *volume, int32_t *given, int32_t *paid,
                               const int32_t *active) {
    const int h = history_of(blk, nh);
    if (active && !active[h]) return;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int64_t gi = off[h] + i;
    const int32_t to = claim[gi];
    if (to < 0) return;
    const int64_t c0 = cell_off[h];
    const int32_t from = grid[gi];
    grid[gi] = to;
    atomicAdd(volume + c0 + to, 1);
    if (from > 0) {
        atomicSub(volume + c0 + from, 1);
        atomicAdd(given + c0 + from, 1);
        atomicAdd(paid + h, 1);
    }
}

// What is still owed, carried, never more than the dead tissue still holds;
// each dead cell asks for what it gave up less (simulation.rs:1793-1808).
__global__ void k_debris_settle_cells(int64_t nc, int32_t *given, int32_t *target) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int32_t g = given[c];
    if (g <= 0) return;
    target[c] = target[c] > g ? target[c] - g : 0;
    given[c] = 0;
}
__global__ void k_debris_settle_histories(int nh, double *owed, const int64_t *held, int32_t *paid) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const double p = (double)paid[h];
    owed[h] = fmin(owed[h] - p, (double)held[h] - p);
    paid[h] = 0;
}

}  // namespace

namespace cw {

int DebrisState::ensure(int64_t ncells, int nh, int64_t sites) {
    int rc;
    if ((rc = dalloc(&kept, ncells)) || (rc = dalloc(&given, ncells)) || (rc = dalloc(&owed, nh)) ||
        (rc = dalloc(&held, nh)) || (rc = dalloc(&paid, nh)) || (rc = dalloc(&edges, nh)) ||
        (rc = dalloc(&active, nh)) || (rc = dalloc(&claim, sites)))
        return rc;
    CW_CUDA(cudaMemsetAsync(kept, 0, sizeof(uint8_t) * ncells, stream()));
    CW_CUDA(cudaMemsetAsync(given, 0, sizeof(int32_t) * ncells, stream()));
    CW_CUDA(cudaMemsetAsync(owed, 0, sizeof(double) * nh, stream()));
    CW_CUDA(cudaMemsetAsync(held, 0, sizeof(int64_t) * nh, stream()));
    CW_CUDA(cudaMemsetAsync(paid, 0, sizeof(int32_t) * nh, stream()));
    return CW_OK;
}

void DebrisState::release() {
    dfree(kept); dfree(given); dfree(owed); dfree(held); dfree(paid); dfree(edges); dfree(active); dfree(claim);
    kept = nullptr; given = nullptr; owed = nullptr; held = nullptr; paid = nullptr; edges = nullptr;
    active = nullptr; claim = nullptr;
}

static int site_plan_of(cw_lattice_s *l) {
    Plan &p = l->site_plan;
    if (p.nblocks != 0) return CW_OK;
    std::vector<int64_t> per(l->g.nh);
    for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
    return p.build(per, T);
}

// break_down_debris for every history (no host synchronisation): the debt
// booked from the kept dead's volumes, up to EDGE_PASSES passes over the
// edge, the debt carried and the dead cells' targets lowered.
int debris_break_down_enqueue(cw_lattice_s *l, DebrisState &D, double loss, int necrotic, const uint32_t *step) {
    int rc;
    if ((rc = site_plan_of(l)) != CW_OK) return rc;
    const Plan &p = l->site_plan;
    const int nh = (int)l->g.nh;
    k_debris_owe<<<nh, T, 0, stream()>>>(l->d_cell_off, D.kept, l->volume, loss, D.owed, D.held, D.active);
    CW_LAUNCHED();
    for (int pass = 0; pass < EDGE_PASSES; ++pass) {
        CW_CUDA(cudaMemsetAsync(D.edges, 0, sizeof(int32_t) * nh, stream()));
        k_debris_edges<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh,
                                                      l->type, D.kept, necrotic, D.owed, D.paid, D.active, D.claim,
                                                      D.edges);
        CW_LAUNCHED();
        k_debris_draw<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh,
                                                     l->type, necrotic, D.owed, D.paid, D.edges, l->d_keys, step,
                                                     pass, D.active, D.claim);
        CW_LAUNCHED();
        k_claims_apply<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_off, l->d_cell_off, p.d_blk, nh, D.claim,
                                                      l->volume, D.given, D.paid, D.active);
        CW_LAUNCHED();
        k_debris_still<<<(unsigned)((nh + T - 1) / T), T, 0, stream()>>>(nh, D.owed, D.paid, D.active);
        CW_LAUNCHED();
    }
    const int64_t nc = l->ncells;
    k_debris_settle_cells<<<(unsigned)((nc + T - 1) / T), T, 0, stream()>>>(nc, D.given, l->target);
    CW_LAUNCHED();
    k_debris_settle_histories<<<(unsigned)((nh + T - 1) / T), T, 0, stream()>>>(nh, D.owed, D.held, D.paid);
    CW_LAUNCHED();
    return CW_OK;
}

// drain_shut_in for every history: `bath` is the bath mask of the lattice as
// it stands (lattice_bath_enqueue); medium outside it is shut in.
int debris_drain_enqueue(cw_lattice_s *l, DebrisState &D, const uint8_t *bath, int necrotic, const uint32_t *step) {
    int rc;
    if ((rc = site_plan_of(l)) != CW_OK) return rc;
    const Plan &p = l->site_plan;
    const int nh = (int)l->g.nh;
    k_drain_draw<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh, l->type,
                                                necrotic, bath, l->d_keys, step, D.claim);
    CW_LAUNCHED();
    k_claims_apply<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_off, l->d_cell_off, p.d_blk, nh, D.claim,
                                                  l->volume, D.given, D.paid, nullptr);
    CW_LAUNCHED();
    return CW_OK;
}

}  // namespace cw
