// Lattice <-> field coupling: crates/engine/src/coupling.rs on the device.
// Each kernel is one pass over the pixels of every history; nothing leaves
// the device between the lattice, the field and the per-cell means.
#include <cmath>

#include "cw_internal.cuh"
#include "field_kernels.cuh"

using namespace cw;

namespace {

constexpr int T = 256;

struct Pair {
    const int32_t *grid;
    const int32_t *type;
    const int4 *dims;
    const int64_t *off;
    const int64_t *cell_off;
};

Pair pair_of(cw_lattice_s *l) { return Pair{l->grid, l->type, l->g.d_dims, l->g.d_off, l->d_cell_off}; }

// apply_uptake (coupling.rs:26-39): every pixel of a cell whose type has a
// rate sinks it, floored at zero as set_uptake_at does; the rest nothing.
__global__ void k_paint_uptake(Pair p, const int32_t *blk, int nh, const double *rate_by_type, int K, double *dst) {
    __shared__ int s_h;
    __shared__ double sr[8];
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    if (threadIdx.x < 8) sr[threadIdx.x] = threadIdx.x < K ? rate_by_type[threadIdx.x] : 0.0;
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= p.off[h + 1] - p.off[h]) return;
    int64_t i = p.off[h] + local;
    int32_t id = p.grid[i];
    int64_t c0 = p.cell_off[h], cap = p.cell_off[h + 1] - c0;
    double v = 0.0;
    if (id > 0 && id < cap) {
        double r = sr[p.type[c0 + id]];
        if (r != 0.0) v = fmax(r, 0.0);
    }
    dst[i] = v;
}

// apply_background_uptake (coupling.rs:47-53): every medium pixel sinks `rate`.
__global__ void k_paint_background(Pair p, int64_t n, double rate, double *dst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && p.grid[i] == 0) dst[i] = fmax(rate, 0.0);
}

// apply_production (coupling.rs:61-73) from per-cell rates laid out like the
// lattice's records (global cell index).
__global__ void k_paint_production(Pair p, const int32_t *blk, int nh, const double *per_cell, double *dst) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= p.off[h + 1] - p.off[h]) return;
    int64_t i = p.off[h] + local;
    int32_t id = p.grid[i];
    int64_t c0 = p.cell_off[h], cap = p.cell_off[h + 1] - c0;
    double v = 0.0;
    if (id > 0 && id < cap) {
        double r = per_cell[c0 + id];
        if (r > 0.0) v = r;
    }
    dst[i] = v;
}

// hold_obstacles_at (coupling.rs:80-82).
__global__ void k_hold_obstacles(const int32_t *grid, int64_t n, double v, uint8_t *held, double *c) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && grid[i] == -1) { held[i] = 1; c[i] = v; }
}

// hold_vessels_by (coupling.rs:114-150) on planes: an obstacle pixel with a
// delivery share above zero is held at value x min(share, 1) unless the mean
// of the field over its in-box neighbours that are not obstacles (x-1, x+1,
// y-1, y+1, summed in that order) already reaches that level.  Only obstacle
// pixels are written and only the others read, so one pass decides on the
// field as it stood, as the reference's two passes do.
__global__ void k_hold_vessels_by(Pair p, const int32_t *blk, int nh, double value, const double *delivery,
                                  uint8_t *held, double *c) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= p.off[h + 1] - p.off[h]) return;
    const int64_t i = p.off[h] + local;
    if (p.grid[i] != -1) return;
    const double share = delivery[i];
    if (share <= 0.0) return;
    const double level = value * fmin(share, 1.0);
    const int4 dm = p.dims[h];
    const int x = (int)(local % dm.x), y = (int)(local / dm.x);
    const int nx[4] = {x - 1, x + 1, x, x};
    const int ny[4] = {y, y, y - 1, y + 1};
    double sum = 0.0;
    int n = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (nx[q] < 0 || nx[q] >= dm.x || ny[q] < 0 || ny[q] >= dm.y) continue;
        const int64_t j = p.off[h] + (int64_t)ny[q] * dm.x + nx[q];
        if (p.grid[j] == -1) continue;
        sum += c[j];
        n += 1;
    }
    if (n > 0 && sum / (double)n >= level) return;  // richer around it: left free
    held[i] = 1;
    c[i] = level;
}

__global__ void k_open_medium(const int32_t *grid, int64_t n, uint8_t *open) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) open[i] = grid[i] == 0;
}

// mean_per_cell (coupling.rs:164-182): sums and counts per cell, one atomic
// per distinct cell per warp; the medium and the obstacle are skipped.
__global__ void k_cell_sums(Pair p, const int32_t *blk, int nh, const double *c, double *sum, int32_t *count) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    int64_t c0 = p.cell_off[h], cap = p.cell_off[h + 1] - c0;
    int64_t key = -1;
    double v = 0.0;
    if (local < p.off[h + 1] - p.off[h]) {
        int64_t i = p.off[h] + local;
        int32_t id = p.grid[i];
        if (id > 0 && id < cap) { key = c0 + id; v = c[i]; }
    }
    // Cells are compact, so a warp's 32 consecutive pixels hold a few runs of
    // one id: a segmented inclusive scan along the warp gives each run's sum
    // and length at its last lane, which alone touches global memory.
    const int lane = threadIdx.x & 31;
    if (!__any_sync(0xffffffffu, key >= 0)) return;
    const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool head = lane == 0 || prev != key;
    unsigned heads = __ballot_sync(0xffffffffu, head);
    // distance back to this lane's run head
    const unsigned below = heads & ((2u << lane) - 1u);
    const int start = 31 - __clz(below);
    double s = v;
    int n = 1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double sv = __shfl_up_sync(0xffffffffu, s, o);
        int nv = __shfl_up_sync(0xffffffffu, n, o);
        if (lane - o >= start) { s += sv; n += nv; }
    }
    const long long next = __shfl_down_sync(0xffffffffu, key, 1);
    const bool tail = lane == 31 || next != key;
    if (key >= 0 && tail) {
        atomicAdd(sum + key, s);
        atomicAdd(count + key, n);
    }
}

__global__ void k_cell_means(const double *sum, const int32_t *count, int64_t n, double *mean) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) mean[k] = count[k] == 0 ? 0.0 : sum[k] / (double)count[k];
}

int site_plan(const Geom &g, Plan &p) {
    std::vector<int64_t> per(g.nh);
    for (uint32_t k = 0; k < g.nh; ++k) per[k] = g.sites(k);
    return p.build(per, T);
}

int check_pair(cw_field_s *f, cw_lattice_s *l) {
    if (!f->g.same(l->g)) return fail(CW_ERR_CONFIG, "the field and the lattice hold different histories");
    return CW_OK;
}

}  // namespace

namespace cw {

// Device versions for the simulation driver.
int couple_uptake_device(cw_field_s *f, cw_lattice_s *l, const double *d_rate_by_type, int K, double *dst,
                         const Plan &p) {
    k_paint_uptake<<<p.nblocks, T, 0, stream()>>>(pair_of(l), p.d_blk, l->g.nh, d_rate_by_type, K, dst);
    CW_LAUNCHED();
    return CW_OK;
}

int couple_production_device(cw_field_s *f, cw_lattice_s *l, const double *d_per_cell, const Plan &p) {
    f->production_on = true;
    k_paint_production<<<p.nblocks, T, 0, stream()>>>(pair_of(l), p.d_blk, l->g.nh, d_per_cell, f->production);
    CW_LAUNCHED();
    return CW_OK;
}

int couple_background_device(cw_field_s *f, cw_lattice_s *l, double rate, double *dst) {
    int64_t n = f->g.total;
    k_paint_background<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(pair_of(l), n, rate, dst);
    CW_LAUNCHED();
    return CW_OK;
}

// Per-cell means over all histories into `mean` (global cell index);
// `sum` and `count` are scratch of the lattice's record count.
int couple_means_device(cw_field_s *f, cw_lattice_s *l, double *sum, int32_t *count, double *mean, const Plan &p) {
    CW_CUDA(cudaMemsetAsync(sum, 0, sizeof(double) * l->ncells, stream()));
    CW_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t) * l->ncells, stream()));
    k_cell_sums<<<p.nblocks, T, 0, stream()>>>(pair_of(l), p.d_blk, l->g.nh, f->c, sum, count);
    CW_LAUNCHED();
    k_cell_means<<<(unsigned)((l->ncells + T - 1) / T), T, 0, stream()>>>(sum, count, l->ncells, mean);
    CW_LAUNCHED();
    return CW_OK;
}

}  // namespace cw

extern "C" {

int cw_couple_uptake(cw_field f, cw_lattice l, int32_t K, const double *rate_by_type, int32_t first_order) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    if (K < 1 || K > 8) return fail(CW_ERR_CONFIG, "rates for 1 to 8 types");
    double *d_rate;
    if ((rc = dalloc(&d_rate, 8)) != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_rate, 0, 8 * sizeof(double), stream()));
    CW_CUDA(cudaMemcpyAsync(d_rate, rate_by_type, sizeof(double) * K, cudaMemcpyHostToDevice, stream()));
    Plan p;
    if ((rc = site_plan(f->g, p)) != CW_OK) return rc;
    double *dst = first_order ? f->lin_sink : f->uptake;
    if (first_order) f->lin_sink_on = true;
    else f->uptake_on = true;
    rc = couple_uptake_device(f, l, d_rate, l->K > K ? K : l->K, dst, p);
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_rate);
    p.release();
    return rc;
}

int cw_couple_background_uptake(cw_field f, cw_lattice l, double rate) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    int64_t n = f->g.total;
    f->uptake_on = true;
    k_paint_background<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(pair_of(l), n, rate, f->uptake);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_couple_production(cw_field f, cw_lattice l, uint32_t hist, uint32_t n, const double *per_cell) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int64_t cap = l->cell_off[hist + 1] - l->cell_off[hist];
    double *d_pc;
    if ((rc = dalloc(&d_pc, l->ncells)) != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_pc, 0, sizeof(double) * l->ncells, stream()));
    CW_CUDA(cudaMemcpyAsync(d_pc + l->cell_off[hist], per_cell, sizeof(double) * (n < cap ? n : cap),
                            cudaMemcpyHostToDevice, stream()));
    // only history `hist` is repainted: paint all into scratch, copy its slice
    double *d_out;
    if ((rc = dalloc(&d_out, f->g.total)) != CW_OK) return rc;
    Plan p;
    if ((rc = site_plan(f->g, p)) != CW_OK) return rc;
    k_paint_production<<<p.nblocks, T, 0, stream()>>>(pair_of(l), p.d_blk, l->g.nh, d_pc, d_out);
    CW_LAUNCHED();
    f->production_on = true;
    CW_CUDA(cudaMemcpyAsync(f->production + f->g.off[hist], d_out + f->g.off[hist], sizeof(double) * f->g.sites(hist),
                            cudaMemcpyDeviceToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_pc);
    dfree(d_out);
    p.release();
    return CW_OK;
}

int cw_couple_hold_obstacles(cw_field f, cw_lattice l, double value) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    int64_t n = f->g.total;
    f->held_dirty = true;
    k_hold_obstacles<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(l->grid, n, value, f->held, f->c);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_couple_hold_vessels_by(cw_field f, cw_lattice l, double value, const double *delivery) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    if (!delivery) return fail(CW_ERR_CONFIG, "hold_vessels_by needs a delivery share for every pixel");
    for (uint32_t k = 0; k < f->g.nh; ++k)
        if (f->g.d[k] > 1)
            return fail(CW_ERR_CONFIG, "hold_vessels_by holds the vessels of a plane; history " + std::to_string(k) +
                                           " is a volume");
    const int64_t n = f->g.total;
    double *d_share;
    if ((rc = dalloc(&d_share, n)) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(d_share, delivery, sizeof(double) * n, cudaMemcpyHostToDevice, stream()));
    Plan p;
    if ((rc = site_plan(f->g, p)) != CW_OK) return rc;
    f->held_dirty = true;
    k_hold_vessels_by<<<p.nblocks, T, 0, stream()>>>(pair_of(l), p.d_blk, l->g.nh, value, d_share, f->held, f->c);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_share);
    p.release();
    return CW_OK;
}

int cw_couple_hold_medium_bath(cw_field f, cw_lattice l, double value) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    int64_t n = f->g.total;
    uint8_t *open;
    if ((rc = dalloc(&open, n)) != CW_OK) return rc;
    k_open_medium<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(l->grid, n, open);
    CW_LAUNCHED();
    rc = field_hold_bath_device(f, open, -1, value);
    dfree(open);
    return rc;
}

int cw_couple_mean_per_cell(cw_field f, cw_lattice l, uint32_t hist, uint32_t n, double *out) {
    CW_SCOPE(f);
    CW_JOIN(l);
    int rc = check_pair(f, l);
    if (rc != CW_OK) return rc;
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int64_t cap = l->cell_off[hist + 1] - l->cell_off[hist];
    if ((int64_t)n > cap) return fail(CW_ERR_CONFIG, "more cells asked for than the history holds");
    double *sum, *mean;
    int32_t *count;
    if ((rc = dalloc(&sum, l->ncells)) || (rc = dalloc(&mean, l->ncells)) || (rc = dalloc(&count, l->ncells)))
        return rc;
    Plan p;
    if ((rc = site_plan(f->g, p)) != CW_OK) return rc;
    if ((rc = couple_means_device(f, l, sum, count, mean, p)) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(out, mean + l->cell_off[hist], sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    if (n > 0) out[0] = 0.0;  // the medium reads zero (coupling.rs:160-163)
    dfree(sum); dfree(mean); dfree(count);
    p.release();
    return CW_OK;
}

}  // extern "C"
