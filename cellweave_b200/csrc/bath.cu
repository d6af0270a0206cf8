// The bath on the device: the medium pixels joined to the box's outer layer
// through medium, 4-connected in the plane and 6-connected in a volume —
// what hold_bath_at (crates/engine/src/pde.rs:550-631) holds when the open
// pixels are the medium (hold_medium_bath, coupling.rs:156-158).
//
// The reference floods from the outer layer one pixel at a time.  Here the
// medium's connected components are found by union-find over the whole batch
// at once: every medium pixel starts as its own root, each joins its right,
// lower (and next-slice) medium neighbour by atomicMin on the roots (a root's
// label only falls, so the retries end), the labels are flattened to their
// roots, the roots of every outer-layer medium pixel are marked, and a pixel
// is bath when its root is marked.  Five plain launches over the sites, no
// convergence loop on the host, so the bath can be taken inside a captured
// step.  The same pixels as the reference's flood: a component is held
// exactly when it reaches the outer layer.
//
// In a volume the union-find covers the occupied span (the box around every
// pixel that is not medium, one wider on every side) only: the medium outside
// it is bath (from any pixel outside the span a straight line away from it
// stays outside and ends on the outer layer), and a medium component inside
// is bath exactly when it reaches the span's border layer (next to the
// outside) or the outer layer.  The same mask for a fraction of the work
// when a small tissue sits in a large box.
#include "cw_internal.cuh"

using namespace cw;

namespace {

constexpr int T = 256;
constexpr int FIND_LIMIT = 1 << 26;  // a chase or retry longer than any batch's pixel count is a fault

__device__ int g_bath_error;

__device__ __forceinline__ int32_t find_root(const int32_t *L, int32_t i) {
    for (int n = 0; n < FIND_LIMIT; ++n) {
        const int32_t p = __ldcg(L + i);
        if (p == i) return i;
        i = p;
    }
    atomicExch(&g_bath_error, 1);
    return i;
}

__device__ __forceinline__ void unite(int32_t *L, int32_t a, int32_t b) {
    for (int n = 0; n < FIND_LIMIT; ++n) {
        a = find_root(L, a);
        b = find_root(L, b);
        if (a == b) return;
        if (a < b) {
            const int32_t old = atomicMin(L + b, a);
            if (old == b) return;
            b = old;
        } else {
            const int32_t old = atomicMin(L + a, b);
            if (old == a) return;
            a = old;
        }
    }
    atomicExch(&g_bath_error, 1);
}

constexpr int32_t OUTSIDE = -2;  // a label: medium outside the span, bath

// Inside the span of history h (always, without one or in a plane).
__device__ __forceinline__ bool inside(const int32_t *span, int h, int4 dm, int x, int y, int z) {
    if (!span || dm.z <= 1) return true;
    const int32_t *s = span + 6 * h;
    return x >= s[0] && x <= s[3] && y >= s[1] && y <= s[4] && z >= s[2] && z <= s[5];
}

__device__ __forceinline__ bool site_of(const int32_t *blk, int nh, const int4 *dims, const int64_t *off,
                                        int &h, int64_t &i, int &x, int &y, int &z) {
    h = plan_history(blk, nh, blockIdx.x);
    const int4 dm = dims[h];
    const int64_t local = (int64_t)(blockIdx.x - blk[h]) * T + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return false;
    x = (int)(local % dm.x);
    y = (int)((local / dm.x) % dm.y);
    z = (int)(local / ((int64_t)dm.x * dm.y));
    i = off[h] + local;
    return true;
}

__global__ void k_cc_init(const int32_t *blk, int nh, const int4 *dims, const int64_t *off, const int32_t *span,
                          const int32_t *grid, int32_t *L, uint8_t *mark) {
    int h, x, y, z;
    int64_t i;
    if (!site_of(blk, nh, dims, off, h, i, x, y, z)) return;
    L[i] = grid[i] != 0 ? -1 : inside(span, h, dims[h], x, y, z) ? (int32_t)i : OUTSIDE;
    mark[i] = 0;
}

__global__ void k_cc_merge(const int32_t *blk, int nh, const int4 *dims, const int64_t *off, int32_t *L) {
    int h, x, y, z;
    int64_t i;
    if (!site_of(blk, nh, dims, off, h, i, x, y, z)) return;
    if (L[i] < 0) return;
    const int4 dm = dims[h];
    if (x + 1 < dm.x && L[i + 1] >= 0) unite(L, (int32_t)i, (int32_t)(i + 1));
    if (y + 1 < dm.y && L[i + dm.x] >= 0) unite(L, (int32_t)i, (int32_t)(i + dm.x));
    const int64_t slice = (int64_t)dm.x * dm.y;
    if (z + 1 < dm.z && L[i + slice] >= 0) unite(L, (int32_t)i, (int32_t)(i + slice));
}

__global__ void k_cc_flatten(int64_t n, int32_t *L) {
    const int64_t i = (int64_t)blockIdx.x * T + threadIdx.x;
    if (i >= n || L[i] < 0) return;
    L[i] = find_root(L, (int32_t)i);
}

// the roots of the medium on the box's outer layer (a flat box's one slice
// is its whole area: its first and last slice are not a layer)
// (and, in a volume with a span, the roots of the medium on its border layer)
__global__ void k_cc_mark(const int32_t *blk, int nh, const int4 *dims, const int64_t *off, const int32_t *span,
                          const int32_t *L, uint8_t *mark) {
    int h, x, y, z;
    int64_t i;
    if (!site_of(blk, nh, dims, off, h, i, x, y, z)) return;
    const int32_t r = L[i];
    if (r < 0) return;
    const int4 dm = dims[h];
    bool outer = x == 0 || y == 0 || x + 1 == dm.x || y + 1 == dm.y || (dm.z > 1 && (z == 0 || z + 1 == dm.z));
    if (span && dm.z > 1) {
        const int32_t *s = span + 6 * h;
        outer = outer || x == s[0] || x == s[3] || y == s[1] || y == s[4] || z == s[2] || z == s[5];
    }
    if (outer) mark[r] = 1;
}

__global__ void k_cc_bath(int64_t n, const int32_t *L, const uint8_t *mark, uint8_t *bath) {
    const int64_t i = (int64_t)blockIdx.x * T + threadIdx.x;
    if (i >= n) return;
    const int32_t r = L[i];
    bath[i] = r == OUTSIDE || (r >= 0 && mark[r]) ? 1 : 0;
}

}  // namespace

namespace cw {

// The bath mask of every history into `bath` (one byte per site, 1 = held by
// the bath), enqueued on the library's stream without synchronisation.
int lattice_bath_enqueue(cw_lattice_s *l, uint8_t *bath) {
    const int64_t n = l->g.total;
    if (n >= (int64_t)INT32_MAX) return fail(CW_ERR_CONFIG, "the bath labels pixels with 32-bit indices");
    int rc;
    if (!l->bath_label) {
        if ((rc = dalloc(&l->bath_label, (size_t)n)) != CW_OK) return rc;
        if ((rc = dalloc(&l->bath_mark, (size_t)n)) != CW_OK) return rc;
    }
    Plan &p = l->site_plan;
    if (p.nblocks == 0) {
        std::vector<int64_t> per(l->g.nh);
        for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
        if ((rc = p.build(per, T)) != CW_OK) return rc;
    }
    const unsigned flat = (unsigned)((n + T - 1) / T);
    const int nh = (int)l->g.nh;
    // the span of the lattice as it stands (a step's may be out of date)
    if ((rc = lattice_span_enqueue(l)) != CW_OK) return rc;
    k_cc_init<<<p.nblocks, T, 0, stream()>>>(p.d_blk, nh, l->g.d_dims, l->g.d_off, l->d_span, l->grid, l->bath_label,
                                            l->bath_mark);
    CW_LAUNCHED();
    k_cc_merge<<<p.nblocks, T, 0, stream()>>>(p.d_blk, nh, l->g.d_dims, l->g.d_off, l->bath_label);
    CW_LAUNCHED();
    k_cc_flatten<<<flat, T, 0, stream()>>>(n, l->bath_label);
    CW_LAUNCHED();
    k_cc_mark<<<p.nblocks, T, 0, stream()>>>(p.d_blk, nh, l->g.d_dims, l->g.d_off, l->d_span, l->bath_label,
                                             l->bath_mark);
    CW_LAUNCHED();
    k_cc_bath<<<flat, T, 0, stream()>>>(n, l->bath_label, l->bath_mark, bath);
    CW_LAUNCHED();
    return CW_OK;
}

// CW_ERR_SIMULATION if a bath's union-find met a chase longer than any
// lattice (synchronous; clears the record).
int lattice_bath_error() {
    int v = 0;
    CW_CUDA(cudaMemcpyFromSymbol(&v, g_bath_error, sizeof v));
    if (v) {
        const int zero = 0;
        CW_CUDA(cudaMemcpyToSymbol(g_bath_error, &zero, sizeof zero));
        return fail(CW_ERR_SIMULATION, "the bath's union-find did not settle");
    }
    return CW_OK;
}

}  // namespace cw

extern "C" int cw_lattice_bath(cw_lattice l, uint32_t hist, uint8_t *out) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    uint8_t *d;
    int rc;
    if ((rc = dalloc(&d, (size_t)l->g.total)) != CW_OK) return rc;
    if ((rc = lattice_bath_enqueue(l, d)) != CW_OK) {
        dfree(d);
        return rc;
    }
    CW_CUDA(cudaMemcpyAsync(out, d + l->g.off[hist], (size_t)l->g.sites(hist), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d);
    return lattice_bath_error();
}
