// Cell division on the device: divide_across of crates/engine/src/cpm.rs
// (1087-1160) for many cells of many histories at once, and the division
// step of Simulation::step (simulation.rs:1338-1347, divide_ready_cells
// 1603-1716) on top of it.
//
// A cell splits across the plane through its centre of mass with a given
// normal: its pixels with (x - cx) nx + (y - cy) ny [+ (z - cz) nz] > 0 go to a
// new cell of the same kind with the parent's volume parameters; a plane that
// leaves one side empty, a cell under 8 pixels or the medium is no division.
// The centre is the mean of the pixel coordinates; their sums are integers,
// so the device's atomic sums equal the reference's ordered f64 sums, and
// the side test is the reference's arithmetic (this file is built without
// fused multiply-add).  Daughters take the next free record of their
// history, in the order of their parents' ids, so ids match the
// reference's push order.
//
// Passes (every pixel of the batch each): the coordinate sums of the
// dividing cells; the count each plane moves; the daughters chosen per
// history (parents in id order, as far as the living-cell limit and the
// record capacity allow); the relabelling; then the records (and, given, a
// copy of the parent's network state).
#include <algorithm>
#include <cmath>

#include "cw_internal.cuh"

using namespace cw;

namespace {

constexpr int T = 256;
constexpr int32_t MIN_DIVIDE_VOLUME = 8;  // cpm.rs:132

__device__ __forceinline__ void pixel_xyz(int64_t i, int4 dm, int &x, int &y, int &z) {
    const int64_t slice = (int64_t)dm.x * dm.y;
    z = (int)(i / slice);
    const int64_t r = i - (int64_t)z * slice;
    y = (int)(r / dm.x);
    x = (int)(r - (int64_t)y * dm.x);
}

// The coordinate sums and pixel counts of the flagged cells.
__global__ void k_div_sums(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                           const int32_t *blk, int nh, const uint8_t *flag, unsigned long long *sums, int32_t *npix,
                           const int32_t *count) {
    if (*count == 0) return;
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int32_t id = grid[off[h] + i];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    if (id <= 0 || id >= cap || !flag[c0 + id]) return;
    int x, y, z;
    pixel_xyz(i, dims[h], x, y, z);
    const int64_t c = c0 + id;
    atomicAdd(sums + 3 * c + 0, (unsigned long long)x);
    atomicAdd(sums + 3 * c + 1, (unsigned long long)y);
    atomicAdd(sums + 3 * c + 2, (unsigned long long)z);
    atomicAdd(npix + c, 1);
}

// divide_across's side of pixel (x, y, z) for cell c: > 0 goes to the daughter.
__device__ __forceinline__ double side_of(const unsigned long long *sums, const int32_t *npix, const double *normal,
                                          int64_t c, bool volume, int x, int y, int z) {
    const double n = (double)npix[c];
    const double cx = (double)sums[3 * c + 0] / n, cy = (double)sums[3 * c + 1] / n;
    double side = ((double)x - cx) * normal[3 * c + 0] + ((double)y - cy) * normal[3 * c + 1];
    if (volume) {
        const double cz = (double)sums[3 * c + 2] / n;
        side += ((double)z - cz) * normal[3 * c + 2];
    }
    return side;
}

// How many pixels each flagged cell's plane moves.
__global__ void k_div_moved(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                            const int32_t *blk, int nh, const uint8_t *flag, const unsigned long long *sums,
                            const int32_t *npix, const double *normal, int32_t *moved, const int32_t *count) {
    if (*count == 0) return;
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int32_t id = grid[off[h] + i];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    if (id <= 0 || id >= cap || !flag[c0 + id]) return;
    const int4 dm = dims[h];
    int x, y, z;
    pixel_xyz(i, dm, x, y, z);
    if (side_of(sums, npix, normal, c0 + id, dm.z > 1, x, y, z) > 0.0) atomicAdd(moved + c0 + id, 1);
}

// One block per history: the flagged cells in id order whose plane divides
// them get the next free records, as far as `max_living` (living cells,
// daughters counted as they are born; <= 0: no limit) and the capacity
// allow; daughter[c] = the new id or -1.  used[h] advances.
__global__ void k_div_select(const int64_t *cell_off, int nh, const uint8_t *flag, const int32_t *npix,
                             const int32_t *moved, const uint8_t *alive, int max_living, int32_t *used,
                             int32_t *daughter, const int32_t *count) {
    if (*count == 0) return;
    __shared__ int s_scan[T];
    __shared__ int s_base, s_living, s_room;
    const int h = blockIdx.x;
    if (h >= nh) return;
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    // living cells now (the reference's self.living(), simulation.rs:2354-2367)
    int living = 0;
    if (alive)
        for (int64_t k = threadIdx.x; k < cap; k += blockDim.x) living += alive[c0 + k] ? 1 : 0;
    living = (int)warp_sum((double)living);
    if (threadIdx.x == 0) { s_living = 0; s_base = 0; }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_living, living);
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t room = cap - used[h];
        if (alive && max_living > 0) {
            const int64_t left = max_living - s_living > 0 ? max_living - s_living : 0;
            room = room < left ? room : left;
        }
        s_room = (int)(room > 0 ? room : 0);
    }
    __syncthreads();
    const int room = s_room;
    const int first = used[h];
    for (int64_t k0 = 0; k0 < cap; k0 += blockDim.x) {
        const int64_t k = k0 + threadIdx.x;
        const int64_t c = c0 + k;
        bool splits = false;
        if (k > 0 && k < cap && flag[c]) {
            const int32_t n = npix[c], m = moved[c];
            splits = n >= MIN_DIVIDE_VOLUME && m > 0 && m < n;
        }
        // rank among the block's splitting cells, in id order
        s_scan[threadIdx.x] = splits ? 1 : 0;
        __syncthreads();
        for (int d = 1; d < (int)blockDim.x; d <<= 1) {
            const int v = threadIdx.x >= (unsigned)d ? s_scan[threadIdx.x - d] : 0;
            __syncthreads();
            s_scan[threadIdx.x] += v;
            __syncthreads();
        }
        const int rank = s_base + s_scan[threadIdx.x] - (splits ? 1 : 0);
        if (k < cap) daughter[c] = splits && rank < room ? first + rank : -1;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_base += s_scan[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) used[h] = first + min(s_base, room);
}

// The dividing cells' pixels on the far side of their planes to the daughters.
__global__ void k_div_relabel(int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                              const int32_t *blk, int nh, const int32_t *daughter, const unsigned long long *sums,
                              const int32_t *npix, const double *normal, const int32_t *count) {
    if (*count == 0) return;
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    int32_t *g = grid + off[h];
    const int32_t id = g[i];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    if (id <= 0 || id >= cap) return;
    const int32_t dg = daughter[c0 + id];
    if (dg < 0) return;
    const int4 dm = dims[h];
    int x, y, z;
    pixel_xyz(i, dm, x, y, z);
    if (side_of(sums, npix, normal, c0 + id, dm.z > 1, x, y, z) > 0.0) g[i] = dg;
}

// The records of each division (cpm.rs:1147-1157): the parent keeps what
// stayed, the daughter takes what moved, its kind and volume parameters the
// parent's; its network state (when given, [S][nc]) a copy of the parent's.
__global__ void k_div_records(const int64_t *cell_off, int nh, int64_t nc, const int32_t *daughter,
                              const int32_t *npix, const int32_t *moved, int32_t *type, int32_t *volume,
                              int32_t *target, double *lambda, int32_t *tsurf, double *lsurf, double *state, int S,
                              uint8_t *alive, const int32_t *count) {
    if (*count == 0) return;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int32_t dg = daughter[c];
    if (dg < 0) return;
    int lo = 0, hi = nh - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
    const int64_t d = cell_off[lo] + dg;
    volume[c] = npix[c] - moved[c];
    volume[d] = moved[c];
    type[d] = type[c];
    target[d] = target[c];
    lambda[d] = lambda[c];
    if (tsurf) { tsurf[d] = tsurf[c]; lsurf[d] = lsurf[c]; }
    if (state)
        for (int i = 0; i < S; ++i) state[(int64_t)i * nc + d] = state[(int64_t)i * nc + c];
    if (alive) alive[d] = 1;
}

// Surfaces counted again after divisions (two cells' surfaces change with
// each): zeroed, then every pixel adds its faces against other ids.
__global__ void k_div_surface_zero(int32_t *surface, int64_t nc, const int32_t *count) {
    if (*count == 0) return;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) surface[c] = 0;
}

__global__ void k_div_surface_count(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                                    const int32_t *blk, int nh, int32_t *surface, const int32_t *count) {
    if (*count == 0) return;
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int64_t i = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (i >= off[h + 1] - off[h]) return;
    const int32_t *g = grid + off[h];
    const int32_t id = g[i];
    const int64_t c0 = cell_off[h], cap = cell_off[h + 1] - c0;
    if (id <= 0 || id >= cap) return;
    const int4 dm = dims[h];
    int x, y, z;
    pixel_xyz(i, dm, x, y, z);
    const int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    int faces = 0;
    if (y > 0) faces += g[i - w] != id;
    if (y + 1 < dm.y) faces += g[i + w] != id;
    if (x > 0) faces += g[i - 1] != id;
    if (x + 1 < dm.x) faces += g[i + 1] != id;
    if (z > 0) faces += g[i - slice] != id;
    if (z + 1 < dm.z) faces += g[i + slice] != id;
    if (faces) atomicAdd(surface + c0 + id, faces);
}

}  // namespace

namespace cw {

int DivScratch::ensure(int64_t nc) {
    if (cap >= nc) return CW_OK;
    release();
    int rc;
    if ((rc = dalloc(&flag, nc)) || (rc = dalloc(&normal, 3 * nc)) || (rc = dalloc(&sums, 3 * nc)) ||
        (rc = dalloc(&npix, nc)) || (rc = dalloc(&moved, nc)) || (rc = dalloc(&daughter, nc)) ||
        (rc = dalloc(&count, 1)))
        return rc;
    CW_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t), stream()));
    cap = nc;
    return CW_OK;
}

void DivScratch::release() {
    dfree(flag); dfree(normal); dfree(sums); dfree(npix); dfree(moved); dfree(daughter); dfree(count);
    cap = 0;
}

// Divide the cells flagged in l->div.flag (l->div.count of them) across the
// planes in l->div.normal (no host synchronisation); with none flagged every
// pass returns at once.  alive / max_living: the living-cell limit
// (null: none); state ([S][nc]) is copied to daughters when given.
int lattice_divide_enqueue(cw_lattice_s *l, const uint8_t *alive, int max_living, double *state, int S) {
    DivScratch &D = l->div;
    const int64_t nc = l->ncells;
    Plan &p = l->site_plan;
    if (p.nblocks == 0) {
        std::vector<int64_t> per(l->g.nh);
        for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
        int rc = p.build(per, T);
        if (rc != CW_OK) return rc;
    }
    const int nh = (int)l->g.nh;
    const int32_t *cnt = D.count;
    CW_CUDA(cudaMemsetAsync(D.sums, 0, sizeof(unsigned long long) * 3 * nc, stream()));
    CW_CUDA(cudaMemsetAsync(D.npix, 0, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(D.moved, 0, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(D.daughter, 0xFF, sizeof(int32_t) * nc, stream()));
    k_div_sums<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh, D.flag,
                                              D.sums, D.npix, cnt);
    CW_LAUNCHED();
    k_div_moved<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh, D.flag,
                                               D.sums, D.npix, D.normal, D.moved, cnt);
    CW_LAUNCHED();
    k_div_select<<<nh, T, 0, stream()>>>(l->d_cell_off, nh, D.flag, D.npix, D.moved, alive, max_living, l->d_used,
                                         D.daughter, cnt);
    CW_LAUNCHED();
    k_div_relabel<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, nh,
                                                 D.daughter, D.sums, D.npix, D.normal, cnt);
    CW_LAUNCHED();
    const unsigned cb = (unsigned)((nc + T - 1) / T);
    k_div_records<<<cb, T, 0, stream()>>>(l->d_cell_off, nh, nc, D.daughter, D.npix, D.moved, l->type, l->volume,
                                          l->target, l->lambda, l->surface_on ? l->tsurf : nullptr,
                                          l->surface_on ? l->lsurf : nullptr, state, S,
                                          const_cast<uint8_t *>(alive), cnt);
    CW_LAUNCHED();
    if (l->surface_on) {
        k_div_surface_zero<<<cb, T, 0, stream()>>>(l->surface, nc, cnt);
        CW_LAUNCHED();
        k_div_surface_count<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk,
                                                           nh, l->surface, cnt);
        CW_LAUNCHED();
    }
    return CW_OK;
}

}  // namespace cw

extern "C" {

int cw_lattice_divide(cw_lattice l, uint32_t hist, uint32_t n, const int32_t *ids, const double *normals,
                      int32_t *daughters) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    const int64_t c0 = l->cell_off[hist], cap = l->cell_off[hist + 1] - c0, nc = l->ncells;
    std::vector<uint8_t> flag(nc, 0);
    std::vector<double> normal(3 * nc, 0.0);
    for (uint32_t k = 0; k < n; ++k) {
        if (ids[k] < 0 || ids[k] >= cap) return fail(CW_ERR_NOT_FOUND, "no cell " + std::to_string(ids[k]));
        if (ids[k] == 0) continue;  // the medium divides into nothing (cpm.rs:1099-1101)
        flag[c0 + ids[k]] = 1;
        for (int a = 0; a < 3; ++a) normal[3 * (c0 + ids[k]) + a] = normals[3 * k + a];
    }
    int rc = l->div.ensure(nc);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(l->div.flag, flag.data(), nc, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(l->div.normal, normal.data(), sizeof(double) * 3 * nc, cudaMemcpyHostToDevice,
                            stream()));
    int32_t flagged = 0;
    for (uint8_t f : flag) flagged += f;
    CW_CUDA(cudaMemcpyAsync(l->div.count, &flagged, sizeof flagged, cudaMemcpyHostToDevice, stream()));
    if ((rc = lattice_divide_enqueue(l, nullptr, 0, nullptr, 0)) != CW_OK) return rc;
    std::vector<int32_t> dg(nc);
    CW_CUDA(cudaMemcpyAsync(dg.data(), l->div.daughter, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (uint32_t k = 0; k < n; ++k) daughters[k] = ids[k] > 0 ? dg[c0 + ids[k]] : -1;
    return CW_OK;
}

int cw_lattice_cell_count(cw_lattice l, uint32_t hist, uint32_t *n) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int32_t v = 0;
    CW_CUDA(cudaMemcpy(&v, l->d_used + hist, sizeof v, cudaMemcpyDeviceToHost));
    *n = (uint32_t)v;
    return CW_OK;
}

}  // extern "C"
