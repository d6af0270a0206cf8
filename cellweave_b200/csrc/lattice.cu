// CPM lattice: CpmLattice of crates/engine/src/cpm.rs on the device.
//
// The reference's Monte Carlo step is sequential: N attempts at random
// pixels, each seeing every flip before it (cpm.rs:734-772).  Here one step
// is a sequence of sublattice passes.  Pixels are coloured so that no pixel
// of a colour lies within the contact reach of another (the chessboard for
// contact across faces; a period R+1 in every axis for a reach of Chebyshev
// radius R); a pass makes one copy attempt at every pixel of one colour.
// Attempts of one pass never read a pixel another of them writes; they meet
// only through the volume and surface records of cells they share.  A pass
// runs its attempts as the sequence in a per-pass priority order would (each
// seeing the records every earlier one left): attempts that share no cell run
// at once, the others in rounds, in priority order (k_cpm_pass).  So a pass is
// deterministic whatever the thread schedule, and keeps the sequential
// sweep's volume statistics.  The colours are swept in an order shuffled anew
// every step.
//
// Each attempt is the reference's try_flip (cpm.rs:797-838): a neighbour
// across a face drawn uniformly, no proposal from or into an obstacle or
// within one cell, Delta-H = contact (cpm.rs:851-876) + volume
// (cpm.rs:879-894) [+ surface, an extension], accepted when Delta-H <= 0 or
// u < exp(-Delta-H / T).  Draws come from Philox4x32-10 keyed by the
// history's seed, counter (pixel, step, 0, 0).  This file is built without
// fused multiply-add so that Delta-H rounds as the reference's does.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

#include "cw_internal.cuh"

using namespace cw;

namespace {

constexpr int T = 256;
constexpr int32_t OBST = -1;

struct LatView {
    int32_t *grid;
    const int32_t *type;
    int32_t *volume;
    const int32_t *vsnap;
    const int32_t *target;
    const double *lambda;
    int32_t *surface;
    const int32_t *ssnap;
    const int32_t *tsurf;
    const double *lsurf;
    const int4 *dims;
    const int64_t *off;
    const int64_t *cell_off;
    const uint2 *keys;
    int32_t K;
    int32_t nreach;
    int32_t period;
    int32_t ncol;
    double across;
    double temperature;
    int32_t surface_on;
    int32_t copy_moore;
    uint32_t take_below;   // sub-sweeps: a pixel attempts when its draw is below this (0: every pixel)
    const int32_t *span;   // volumes: the pixels a Monte Carlo step visits (x0 y0 z0 x1 y1 z1 a history)
};

struct Tables {
    double J[64];
    int8_t reach[3 * 124];
};

__device__ __forceinline__ int32_t kind_of(const int32_t *type_h, int64_t cap, int32_t id) {
    if (id < 0 || id >= cap) return 0;  // the obstacle reads as the medium (cpm.rs:908-917)
    return type_h[id];
}

// von_neumann, cpm.rs:922-944: y-1, y+1, x-1, x+1, z-1, z+1, clipped; as a
// mask of the six directions in that order (bit k: direction k exists), so
// that the neighbours live in registers.
struct Vn {
    unsigned mask;
    int64_t w, slice;
    __device__ __forceinline__ int count() const { return __popc(mask); }
    __device__ __forceinline__ bool has(int k) const { return (mask >> k) & 1u; }
    __device__ __forceinline__ int64_t step(int k) const {
        return k == 0 ? -w : k == 1 ? w : k == 2 ? -1 : k == 3 ? 1 : k == 4 ? -slice : slice;
    }
    // the offset of the j-th existing neighbour (j < count)
    __device__ __forceinline__ int64_t nth(int j) const { return step(__fns(mask, 0, j + 1)); }
};
// The copy neighbourhood with Moore copies: every in-box pixel at Chebyshev
// distance 1, bit k = (dz + 1) 9 + (dy + 1) 3 + (dx + 1) (the centre, 13, never
// set), taken in that order (the oracle's or_copy_neighbours).
struct Moore {
    unsigned mask;
    int64_t w, slice;
    __device__ __forceinline__ int count() const { return __popc(mask); }
    __device__ __forceinline__ int64_t step(int k) const {
        return (int64_t)(k / 9 - 1) * slice + (int64_t)((k / 3) % 3 - 1) * w + (k % 3 - 1);
    }
    __device__ __forceinline__ int64_t nth(int j) const { return step(__fns(mask, 0, j + 1)); }
};
__device__ __forceinline__ Moore moore_of(int4 dm, int x, int y, int z) {
    Moore m;
    m.w = dm.x;
    m.slice = (int64_t)dm.x * dm.y;
    m.mask = 0u;
    const int deep = dm.z > 1 ? 1 : 0;
    for (int dz = -deep; dz <= deep; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if ((dx | dy | dz) == 0) continue;
                if (x + dx < 0 || x + dx >= dm.x || y + dy < 0 || y + dy >= dm.y || z + dz < 0 || z + dz >= dm.z)
                    continue;
                m.mask |= 1u << ((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
            }
    return m;
}

__device__ __forceinline__ Vn vn_of(int4 dm, int x, int y, int z) {
    Vn v;
    v.w = dm.x;
    v.slice = (int64_t)dm.x * dm.y;
    v.mask = (y > 0 ? 1u : 0u) | (y + 1 < dm.y ? 2u : 0u) | (x > 0 ? 4u : 0u) | (x + 1 < dm.x ? 8u : 0u) |
             (z > 0 ? 16u : 0u) | (z + 1 < dm.z ? 32u : 0u);
    return v;
}

// contact_delta_h (cpm.rs:851-876) on history grid `g`; *num before the division.
__device__ __forceinline__ double contact_delta(const int32_t *__restrict__ g, int4 dm, int x, int y, int z, int32_t src,
                                int32_t dst, const int32_t *type_h, int64_t cap, const double *sJ, int K,
                                const int8_t *reach, int nreach, double across, int64_t i, Vn vn, double *num) {
    int32_t ks = kind_of(type_h, cap, src), kd = kind_of(type_h, cap, dst);
    double dh = 0.0;
    if (nreach > 0) {
        for (int k = 0; k < nreach; ++k) {
            int a = x + reach[3 * k], b = y + reach[3 * k + 1], c = z + reach[3 * k + 2];
            if (a < 0 || b < 0 || c < 0 || a >= dm.x || b >= dm.y || c >= dm.z) continue;
            int32_t nb = g[((int64_t)c * dm.y + b) * dm.x + a];
            int32_t kn = kind_of(type_h, cap, nb);
            double ed = dst == nb ? 0.0 : sJ[kd * K + kn];
            double es = src == nb ? 0.0 : sJ[ks * K + kn];
            dh += ed - es;
        }
        *num = dh;
        return dh / across;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (!vn.has(k)) continue;
        int32_t nb = g[i + vn.step(k)];
        int32_t kn = kind_of(type_h, cap, nb);
        double ed = dst == nb ? 0.0 : sJ[kd * K + kn];
        double es = src == nb ? 0.0 : sJ[ks * K + kn];
        dh += ed - es;
    }
    *num = dh;
    return dh;
}

// volume_delta_h, cpm.rs:879-894, on the volumes given (c0: the history's first cell).
__device__ __forceinline__ double volume_delta(const int32_t *vol, const int32_t *target, const double *lambda,
                                               int64_t c0, int32_t src, int32_t dst) {
    double dh = 0.0;
    if (src != 0) {
        double v = (double)vol[c0 + src], vt = (double)target[c0 + src];
        double a = v - 1.0 - vt, b = v - vt;
        dh += lambda[c0 + src] * (a * a - b * b);
    }
    if (dst != 0) {
        double v = (double)vol[c0 + dst], vt = (double)target[c0 + dst];
        double a = v + 1.0 - vt, b = v - vt;
        dh += lambda[c0 + dst] * (a * a - b * b);
    }
    return dh;
}

__device__ __forceinline__ void surface_change(const int32_t *g, int64_t i, Vn vn, int32_t src, int32_t dst,
                                               int32_t &dsrc, int32_t &ddst) {
    int eq_s = 0, eq_d = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (!vn.has(k)) continue;
        int32_t nb = g[i + vn.step(k)];
        eq_s += nb == src;
        eq_d += nb == dst;
    }
    const int nvn = vn.count();
    dsrc = eq_s - (nvn - eq_s);
    ddst = (nvn - eq_d) - eq_d;
}

__device__ __forceinline__ double surface_delta(const int32_t *surf, const int32_t *tsurf, const double *lsurf,
                                                int64_t c0, int32_t src, int32_t dst, int32_t dsrc, int32_t ddst) {
    double dh = 0.0;
    if (src > 0) {
        double s = (double)surf[c0 + src], st = (double)tsurf[c0 + src];
        double a = s + (double)dsrc - st, b = s - st;
        dh += lsurf[c0 + src] * (a * a - b * b);
    }
    if (dst > 0) {
        double s = (double)surf[c0 + dst], st = (double)tsurf[c0 + dst];
        double a = s + (double)ddst - st, b = s - st;
        dh += lsurf[c0 + dst] * (a * a - b * b);
    }
    return dh;
}

// The colour order of the current step for every history: a Fisher-Yates
// shuffle driven by Philox(all-ones, step, 1, i); with `pass_keys`, each
// pass's priority key, word 0 of Philox(all-ones - 1, step, 2, colour);
// advances the step counter.
__global__ void k_colour_order(const uint2 *keys, int nh, int ncol, uint32_t *mcs_ctr, uint32_t *mcs_cur,
                               int32_t *perm, uint32_t *pass_keys) {
    // one block: every thread reads the counter before thread 0 advances it
    uint32_t m = *mcs_ctr;
    for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        int32_t p[27];
        for (int i = 0; i < ncol; ++i) p[i] = i;
        uint2 k = keys[h];
        for (int i = ncol - 1; i > 0; --i) {
            uint4 r = philox(0xFFFFFFFFu, m, 1u, (uint32_t)i, k.x, k.y);
            int j = (int)(((uint64_t)r.x * (uint64_t)(i + 1)) >> 32);
            int32_t t = p[i]; p[i] = p[j]; p[j] = t;
        }
        for (int i = 0; i < ncol; ++i) perm[h * ncol + i] = p[i];
        if (pass_keys)
            for (int i = 0; i < ncol; ++i)
                pass_keys[h * ncol + i] = philox(0xFFFFFFFEu, m, 2u, (uint32_t)p[i], k.x, k.y).x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *mcs_cur = m;
        *mcs_ctr = m + 1;
    }
}

// The pixel with index k among the pixels of colour `colour` inside the box
// b = (x0, y0, z0, x1, y1, z1) (inclusive) of a history; false past the end.
// Colour classes: the chessboard (x + y + z) mod 2 for period 0, else the
// residues of x, y, z modulo the period.  (32-bit index arithmetic: a
// history holds fewer than 2^31 pixels.)
__device__ __forceinline__ bool colour_site_box(const int (&b)[6], int period, int colour, uint32_t k, int &x, int &y,
                                                int &z) {
    if (b[3] < b[0] || b[4] < b[1] || b[5] < b[2]) return false;
    if (period == 0) {
        const uint32_t hw = ((uint32_t)(b[3] - b[0]) + 2u) >> 1;
        const uint32_t wy = (uint32_t)(b[4] - b[1] + 1);
        const uint32_t row = k / hw;
        if (row >= wy * (uint32_t)(b[5] - b[2] + 1)) return false;
        y = b[1] + (int)(row % wy);
        z = b[2] + (int)(row / wy);
        x = b[0] + ((colour - b[0] - y - z) & 1) + 2 * (int)(k - row * hw);
        return x <= b[3];
    }
    const int c[3] = {colour % period, (colour / period) % period, colour / (period * period)};
    int f[3];
    uint32_t n[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        f[a] = b[a] + ((c[a] - b[a] % period + period) % period);
        n[a] = f[a] <= b[3 + a] ? (uint32_t)((b[3 + a] - f[a]) / period + 1) : 0u;
    }
    if (n[0] == 0 || n[1] == 0 || n[2] == 0 || k >= n[0] * n[1] * n[2]) return false;
    const uint32_t r = k / n[0];
    x = f[0] + period * (int)(k - r * n[0]);
    y = f[1] + period * (int)(r % n[1]);
    z = f[2] + period * (int)(r / n[1]);
    return true;
}

// The most pixels one colour holds in a box of sides (wx, wy, wz): the plan
// of a pass gives each history that many sites.
__host__ __device__ __forceinline__ int64_t colour_sites_max(int64_t wx, int64_t wy, int64_t wz, int period) {
    if (wx <= 0 || wy <= 0 || wz <= 0) return 0;
    if (period == 0) return ((wx + 1) / 2) * wy * wz;
    return ((wx + period - 1) / period) * ((wy + period - 1) / period) * ((wz + period - 1) / period);
}

// MurmurHash3's 32-bit finaliser (Appleby): a bijection of 32-bit words, so
// the pixels of one history get distinct priorities in a pass.
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// One copy attempt of a pass, with everything about it that the pass cannot
// change: the pixels of a colour lie outside one another's reach, so the
// contact term, the surface counts' changes and the draws are fixed when the
// pass starts; only the volume and surface records move.
struct __align__(16) Attempt {
    int64_t c0;        // the history's first cell record
    int32_t src, dst;  // source and copied ids
    uint32_t prio;     // the pass priority
    int32_t dsurf;     // surface changes of source and copied cell (int16 each)
    uint32_t u0, u1;   // the acceptance draw's words
    int64_t gi;        // the pixel in the batch's flat order
    union {
        double contact;  // contact Delta-H (cpm.rs:851-876)
        uint2 where;     // until the contact is taken: history | z << 16, x | y << 16
    };
};
static_assert(sizeof(Attempt) == 48, "an attempt is three 16-byte words");

constexpr int PT = 1024;           // threads of a pass block; one block per SM
constexpr int PEND_SMEM = 4096;    // pending attempts a block lists in shared memory (else in its global segment)
constexpr int PLAN_SMEM = 1024;    // pass plans of up to 1023 histories sit in shared memory
constexpr int ILP = 2;             // attempts a thread carries at once through a round
constexpr int MAX_ROUNDS = 256;
constexpr uint32_t ROUND_SPAN = MAX_ROUNDS + 2;  // claim tags one pass may use
// passes before the claim tags would overflow 32 bits: the pass that reaches
// it clears the claims and starts the count again
constexpr uint32_t SEQ_LIMIT = 0xFFFFFFFFu / ROUND_SPAN - 1u;
constexpr unsigned long long BARRIER_NS = 2000000000ull;

// Scratch of the passes.  Claims: two words per cell (by round parity), each
// (tag << 32 | priority) with the tag (pass sequence x ROUND_SPAN + round)
// rising from pass to pass, so that old claims lose to new ones and nothing
// needs clearing.  Attempts: a segment of `seg` per block.  Pending lists:
// indices into the block's segment, in shared memory or, for a block with
// more than PEND_SMEM attempts, in two segments of `seg` in `idx`.
struct PassScratch {
    unsigned long long *claim[2];  // ncells each
    Attempt *list;
    uint32_t *idx;
    uint32_t seg;
    int64_t ncells;
    uint32_t *ctl;                 // CTL_* below, then the pass keys (history x colour)
    const int32_t *vplan;          // nh + 1: each history's first chunk of PT sites; vplan[nh]: all chunks
    unsigned long long barrier_ns; // a grid barrier's wait limit
    int32_t withhold;              // a block that never arrives at a barrier (failure tests; -1: none)
    int32_t max_rounds;            // rounds before a pass gives up (CW_ERR_SIMULATION)
};
// control words: list counts and the barrier's arrivals share a line (both
// left at zero when a pass ends); the barrier's generation (only ever
// compared with itself) another; the error, round and sequence records a
// third; then the pass keys
enum { CTL_COUNT = 0, CTL_BAR = 3, CTL_GEN = 32, CTL_ERR = 48, CTL_ROUNDS = 49, CTL_SEQ = 50, CTL_KEYS = 64 };

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// A barrier over the whole (co-resident, cooperatively launched) grid whose
// wait gives up after S.barrier_ns; false then, on every thread of the block.
// The block S.withhold (a failure test) never arrives and returns false.
__device__ __forceinline__ bool grid_barrier(const PassScratch &S, int *s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if ((int)blockIdx.x == S.withhold) {
            ok = 0;
        } else {
            uint32_t *ctl = S.ctl;
            const uint32_t g0 = ld_acquire_gpu(ctl + CTL_GEN);
            __threadfence();
            if (atomicAdd(ctl + CTL_BAR, 1u) == gridDim.x - 1) {
                ctl[CTL_BAR] = 0u;
                __threadfence();
                atomicAdd(ctl + CTL_GEN, 1u);
            } else {
                uint32_t spins = 0;
                uint64_t t0 = 0;
                while (ld_acquire_gpu(ctl + CTL_GEN) == g0) {
                    if ((++spins & 255u) == 0) {  // the clock only now and then
                        const uint64_t t = global_ns();
                        if (t0 == 0) t0 = t;
                        else if (t - t0 > S.barrier_ns) { ok = 0; break; }
                    }
                }
            }
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Append `v` (where `take`) to `list` at a slot counted by *s_n, one
// shared-memory atomic per warp.
template <typename V>
__device__ __forceinline__ void warp_append(V *list, uint32_t *s_n, bool take, const V &v) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    uint32_t base = 0;
    if (lane == 0 && m) base = atomicAdd(s_n, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// The history whose chunks hold chunk vb (plan: nh + 1 prefix of chunks).
__device__ __forceinline__ int plan_find(const int32_t *plan, int nh, int vb) {
    int lo = 0, hi = nh - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (plan[mid] <= vb) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// occupied_span (cpm.rs:774-793) of every volume history, at the start of a
// Monte Carlo step: min and max of x, y, z over the pixels that are not
// medium (the obstacle counts), reduced per warp, one atomic a warp; then one
// pixel wider on every side, clipped, or empty (x0 > x1) when all is medium.
__global__ void k_span_reset(int32_t *span, int nh) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    for (int a = 0; a < 3; ++a) {
        span[6 * h + a] = 0x7fffffff;
        span[6 * h + 3 + a] = -1;
    }
}
__global__ void k_span_occupied(const int32_t *grid, const int4 *dims, const int64_t *off, const int32_t *blk, int nh,
                                int32_t *span) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    const int4 dm = dims[h];
    if (dm.z <= 1) return;  // the whole block: a plane visits its whole box
    const int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {-1, -1, -1};
    if (local < off[h + 1] - off[h] && grid[off[h] + local] != 0) {
        const int64_t slice = (int64_t)dm.x * dm.y;
        const int z = (int)(local / slice);
        const int64_t r = local - (int64_t)z * slice;
        const int y = (int)(r / dm.x), x = (int)(r - (int64_t)y * dm.x);
        mn[0] = mx[0] = x;
        mn[1] = mx[1] = y;
        mn[2] = mx[2] = z;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = __reduce_min_sync(0xffffffffu, mn[a]);
        mx[a] = __reduce_max_sync(0xffffffffu, mx[a]);
    }
    if ((threadIdx.x & 31) == 0 && mx[0] >= 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(span + 6 * h + a, mn[a]);
            atomicMax(span + 6 * h + 3 + a, mx[a]);
        }
}
__global__ void k_span_finish(int32_t *span, const int4 *dims, int nh) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    int32_t *s = span + 6 * h;
    if (s[3] < 0) {  // all medium: nothing to visit
        s[0] = 1;
        s[3] = 0;
        return;
    }
    const int lim[3] = {dims[h].x, dims[h].y, dims[h].z};
    for (int a = 0; a < 3; ++a) {
        s[a] = s[a] > 0 ? s[a] - 1 : 0;
        s[3 + a] = s[3 + a] + 1 < lim[a] - 1 ? s[3 + a] + 1 : lim[a] - 1;
    }
}

// The pass plan of every volume history from its span: the chunks of PT sites
// the largest colour of the span holds, as a prefix over the histories
// (vplan[nh] = all of them).  One block: each thread sums a run of
// histories, the runs' totals are scanned, then each run is written.
__global__ void __launch_bounds__(1024) k_pass_plan(const int32_t *span, int nh, int period, int32_t *vplan) {
    __shared__ int32_t s_run[1024];
    const int per = (nh + blockDim.x - 1) / blockDim.x;
    const int h0 = threadIdx.x * per, h1 = min(h0 + per, nh);
    auto chunks = [&](int h) -> int32_t {
        const int32_t *s = span + 6 * h;
        const int64_t n = colour_sites_max(s[3] - s[0] + 1, s[4] - s[1] + 1, s[5] - s[2] + 1, period);
        return (int32_t)((n + PT - 1) / PT);
    };
    int32_t tot = 0;
    for (int h = h0; h < h1; ++h) tot += chunks(h);
    s_run[threadIdx.x] = tot;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t acc = 0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            const int32_t v = s_run[t];
            s_run[t] = acc;
            acc += v;
        }
        vplan[nh] = acc;
    }
    __syncthreads();
    int32_t acc = s_run[threadIdx.x];
    for (int h = h0; h < h1; ++h) {
        vplan[h] = acc;
        acc += chunks(h);
    }
}

// One sublattice pass: one copy attempt at every pixel of this pass's colour
// (the reference's try_flip, cpm.rs:797-838) inside each history's box (a
// volume's occupied span, a plane's whole box), the attempts ordered by a
// per-pass priority and run as that sequence would run them.  The pixels of
// a colour lie outside one another's reach, so two attempts meet only
// through the records of a cell they both involve (volume, surface).
//
// Propose: every attempt that copies (source and copied ids differ, neither
// the obstacle) claims its cells other than the medium with its priority and
// is packed into its block's segment; then the terms the pass cannot change
// (contact, surface counts) are taken over the packed attempts.  Rounds: an
// attempt holding the claim on all its cells runs against the live records;
// the others claim again for the next round.  An attempt runs only after
// every higher-priority attempt sharing a cell with it, which is the
// sequence in decreasing priority, whatever the thread schedule.  The blocks
// meet at a grid barrier between rounds and count what is left in one word;
// each block lists its pending attempts by index, in shared memory when they
// fit.
__global__ void __launch_bounds__(PT, 1) k_cpm_pass(LatView L, Tables tabs, int nh, const int32_t *perm, int pass,
                                                    const uint32_t *mcs_cur, PassScratch S) {
    // a pass queued after one that gave up does nothing: the barrier's count
    // and the claims that one left behind are cleared by the host first
    if (__ldcg(S.ctl + CTL_ERR) != 0u) return;
    __shared__ double sJ[64];
    __shared__ int8_t sreach[3 * 124];
    __shared__ int s_ok;
    __shared__ uint32_t s_n[2];
    __shared__ int32_t s_plan[PLAN_SMEM];
    __shared__ uint32_t s_pend[2][PEND_SMEM];
    for (int i = threadIdx.x; i < L.K * L.K; i += blockDim.x) sJ[i] = tabs.J[i];
    for (int i = threadIdx.x; i < 3 * L.nreach; i += blockDim.x) sreach[i] = tabs.reach[i];
    const bool plan_shared = nh + 1 <= PLAN_SMEM;
    if (plan_shared)
        for (int i = threadIdx.x; i <= nh; i += blockDim.x) s_plan[i] = S.vplan[i];
    if (threadIdx.x == 0) s_n[0] = s_n[1] = 0u;
    __syncthreads();
    const int32_t *plan = plan_shared ? s_plan : S.vplan;
    const int nvb = plan[nh];
    const uint32_t mcs = *mcs_cur;
    const uint32_t seq = S.ctl[CTL_SEQ];
    const uint32_t tag0 = seq * ROUND_SPAN;  // round r claims with tag tag0 + r
    const uint32_t *pass_key = S.ctl + CTL_KEYS;
    Attempt *mine = S.list + (size_t)blockIdx.x * S.seg;
    // ---- propose and claim (round 1's claims); a block's chunks come in
    // increasing order, so its history only moves forward
    int h = blockIdx.x < nvb ? plan_find(plan, nh, blockIdx.x) : 0;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        while (h + 1 < nh && plan[h + 1] <= vb) ++h;
        const int4 dm = L.dims[h];
        int box[6] = {0, 0, 0, dm.x - 1, dm.y - 1, dm.z - 1};
        if (L.span && dm.z > 1)
#pragma unroll
            for (int a = 0; a < 6; ++a) box[a] = L.span[6 * h + a];
        const int colour = perm[h * L.ncol + pass];
        const uint32_t k = (uint32_t)(vb - plan[h]) * PT + threadIdx.x;
        const int32_t *g = L.grid + L.off[h];
        int x = 0, y = 0, z = 0;
        bool copies = false;
        Attempt a;
        if (colour_site_box(box, L.period, colour, k, x, y, z)) {
            const int64_t i = ((int64_t)z * dm.y + y) * dm.x + x;
            const int32_t src = __ldg(g + i);
            // a pixel whose copy neighbours all hold its own id cannot copy: no draw needed
            bool edge = false;
            int nvn = 0;
            Vn vn;
            Moore mo;
            // every neighbour read at once (no read waits on another's test)
            if (!L.copy_moore) {
                vn = vn_of(dm, x, y, z);
                nvn = vn.count();
                int32_t nb[6];
#pragma unroll
                for (int q = 0; q < 6; ++q) nb[q] = vn.has(q) ? __ldg(g + i + vn.step(q)) : src;
#pragma unroll
                for (int q = 0; q < 6; ++q) edge |= nb[q] != src;
            } else {
                mo = moore_of(dm, x, y, z);
                nvn = mo.count();
                int32_t nb[27];
#pragma unroll
                for (int q = 0; q < 27; ++q)
                    nb[q] = q != 13 && ((mo.mask >> q) & 1u) ? __ldg(g + i + mo.step(q)) : src;
#pragma unroll
                for (int q = 0; q < 27; ++q) edge |= nb[q] != src;
            }
            // with sub-sweeps, a pixel attempts in this one with probability
            // 1 / subsweeps (its own draw), so that over the Monte Carlo step
            // its attempts are Binomial(subsweeps, 1 / subsweeps), near the
            // Poisson(1) of random pixels
            if (edge && src != OBST && L.take_below &&
                philox((uint32_t)i, mcs, 4u, 0u, L.keys[h].x, L.keys[h].y).x >= L.take_below)
                edge = false;
            if (edge && src != OBST) {
                const uint2 key = L.keys[h];
                const uint4 r = philox((uint32_t)i, mcs, 0u, 0u, key.x, key.y);
                const int j = (int)(((uint64_t)r.x * (uint64_t)nvn) >> 32);
                const int32_t dst = __ldg(g + i + (L.copy_moore ? mo.nth(j) : vn.nth(j)));
                if (src != dst && dst != OBST) {
                    copies = true;
                    const uint32_t prio = fmix32((uint32_t)i ^ pass_key[h * L.ncol + pass]);
                    const int64_t c0 = L.cell_off[h];
                    const unsigned long long claim = ((unsigned long long)(tag0 + 1u) << 32) | prio;
                    if (src > 0) atomicMax(S.claim[1] + c0 + src, claim);
                    if (dst > 0) atomicMax(S.claim[1] + c0 + dst, claim);
                    a.c0 = c0;
                    a.src = src;
                    a.dst = dst;
                    a.prio = prio;
                    a.dsurf = 0;
                    a.u0 = r.y;
                    a.u1 = r.z;
                    a.gi = L.off[h] + i;
                    a.where = make_uint2((uint32_t)h | ((uint32_t)z << 16), (uint32_t)x | ((uint32_t)y << 16));
                }
            }
        }
        warp_append(mine, &s_n[0], copies, a);
    }
    __syncthreads();
    const uint32_t n = s_n[0];
    // ---- what the pass cannot change, over the block's attempts packed
    // together (a contact term reads no pixel of the colour, which only the
    // rounds write)
    for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
        Attempt &a = mine[e];
        const uint2 wh = a.where;
        const int hh = (int)(wh.x & 0xFFFFu);
        const int x = (int)(wh.y & 0xFFFFu), y = (int)(wh.y >> 16), z = (int)(wh.x >> 16);
        const int4 dm = L.dims[hh];
        const int64_t cap = L.cell_off[hh + 1] - a.c0;
        const int64_t i = ((int64_t)z * dm.y + y) * dm.x + x;
        const int32_t *g = L.grid + L.off[hh];
        const Vn vn = vn_of(dm, x, y, z);
        double num;
        const double contact = contact_delta(g, dm, x, y, z, a.src, a.dst, L.type + a.c0, cap, sJ, L.K, sreach,
                                             L.nreach, L.across, i, vn, &num);
        int32_t ds = 0, dd = 0;
        if (L.surface_on) surface_change(g, i, vn, a.src, a.dst, ds, dd);
        a.contact = contact;
        a.dsurf = (int32_t)((uint32_t)(uint16_t)(int16_t)ds | ((uint32_t)(uint16_t)(int16_t)dd << 16));
    }
    if (threadIdx.x == 0 && n) atomicAdd(S.ctl + CTL_COUNT + 0, n);
    uint32_t *pend[2] = {s_pend[0], s_pend[1]};
    if (n > PEND_SMEM) {
        pend[0] = S.idx + (size_t)blockIdx.x * 2 * S.seg;
        pend[1] = pend[0] + S.seg;
    }
    if (!grid_barrier(S, &s_ok)) {
        if (threadIdx.x == 0) atomicExch(S.ctl + CTL_ERR, 1u);
        return;
    }
    // ---- rounds
    uint32_t npend = n;  // this block's attempts entering the round
    for (int r = 1;; ++r) {
        const uint32_t left = __ldcg(S.ctl + CTL_COUNT + (r - 1) % 3);
        if (left == 0) break;
        if (r > S.max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(S.ctl + CTL_ERR, 2u);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            S.ctl[CTL_COUNT + (r + 1) % 3] = 0u;  // round r + 1's count; last read as round r - 1's
            atomicMax(S.ctl + CTL_ROUNDS, (uint32_t)r);
        }
        if (threadIdx.x == 0) s_n[r & 1] = 0u;
        __syncthreads();
        const unsigned long long *cl = S.claim[r & 1];
        unsigned long long *next = S.claim[(r + 1) & 1];
        const uint32_t *pin = pend[(r - 1) & 1];
        uint32_t *pout = pend[r & 1];
        const unsigned long long key_tag = (unsigned long long)(tag0 + (uint32_t)r) << 32;
        const unsigned long long next_tag = (unsigned long long)(tag0 + (uint32_t)r + 1u) << 32;
        for (uint32_t e0 = 0; e0 < npend; e0 += ILP * PT) {
            uint32_t id[ILP];
            bool has[ILP], win[ILP];
            Attempt a[ILP];
            unsigned long long cs[ILP], cd[ILP];
#pragma unroll
            for (int j = 0; j < ILP; ++j) {
                const uint32_t e = e0 + (uint32_t)j * PT + threadIdx.x;
                has[j] = e < npend;
                id[j] = has[j] ? (r == 1 ? e : pin[e]) : 0u;
            }
#pragma unroll
            for (int j = 0; j < ILP; ++j)
                if (has[j]) a[j] = mine[id[j]];
#pragma unroll
            for (int j = 0; j < ILP; ++j) {
                cs[j] = cd[j] = 0ull;
                if (has[j]) {
                    if (a[j].src > 0) cs[j] = __ldcg(cl + a[j].c0 + a[j].src);
                    if (a[j].dst > 0) cd[j] = __ldcg(cl + a[j].c0 + a[j].dst);
                }
            }
#pragma unroll
            for (int j = 0; j < ILP; ++j) {
                win[j] = false;
                if (has[j]) {
                    const unsigned long long key = key_tag | a[j].prio;
                    win[j] = (a[j].src <= 0 || cs[j] == key) && (a[j].dst <= 0 || cd[j] == key);
                }
            }
#pragma unroll
            for (int j = 0; j < ILP; ++j) {
                bool again = false;
                if (win[j]) {
                    const Attempt &t = a[j];
                    const int32_t ds = (int32_t)(int16_t)(t.dsurf & 0xFFFF), dd = (int32_t)(int16_t)(t.dsurf >> 16);
                    double delta = t.contact + volume_delta(L.volume, L.target, L.lambda, t.c0, t.src, t.dst);
                    if (L.surface_on) delta += surface_delta(L.surface, L.tsurf, L.lsurf, t.c0, t.src, t.dst, ds, dd);
                    bool accept = delta <= 0.0;
                    if (!accept) accept = u01(t.u0, t.u1) < own_exp(-delta / L.temperature);
                    if (accept) {
                        L.grid[t.gi] = t.dst;
                        // the records: its cells are its own this round
                        if (t.src != 0) L.volume[t.c0 + t.src] -= 1;
                        if (t.dst != 0) L.volume[t.c0 + t.dst] += 1;
                        if (L.surface_on) {
                            if (t.src > 0) L.surface[t.c0 + t.src] += ds;
                            if (t.dst > 0) L.surface[t.c0 + t.dst] += dd;
                        }
                    }
                } else if (has[j]) {
                    const unsigned long long claim = next_tag | a[j].prio;
                    if (a[j].src > 0) atomicMax(next + a[j].c0 + a[j].src, claim);
                    if (a[j].dst > 0) atomicMax(next + a[j].c0 + a[j].dst, claim);
                    again = true;
                }
                warp_append(pout, &s_n[r & 1], again, id[j]);
            }
        }
        __syncthreads();
        npend = s_n[r & 1];
        if (threadIdx.x == 0 && npend) atomicAdd(S.ctl + CTL_COUNT + r % 3, npend);
        if (!grid_barrier(S, &s_ok)) {
            if (threadIdx.x == 0) atomicExch(S.ctl + CTL_ERR, 1u);
            return;
        }
    }
    // ---- the pass is over on every block: the counts go back to zero for the
    // next pass (no block reads them again), the sequence advances; at the
    // sequence's limit the claims are cleared and it starts again
    if (seq + 1u >= SEQ_LIMIT) {
        for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < S.ncells;
             c += (int64_t)gridDim.x * blockDim.x)
            S.claim[0][c] = S.claim[1][c] = 0ull;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.ctl[CTL_COUNT + 0] = S.ctl[CTL_COUNT + 1] = S.ctl[CTL_COUNT + 2] = 0u;
        S.ctl[CTL_SEQ] = seq + 1u >= SEQ_LIMIT ? 0u : seq + 1u;
    }
}


// The first staged pixel of histories h0..h1 (n sites from `a`) whose id is
// below -1 or at least its history's cell capacity, as an offset from `a`.
__global__ void k_check_ids(const int32_t *stage, int64_t a, int64_t n, const int64_t *off, const int64_t *cell_off,
                            int h0, int h1, unsigned long long *first_bad) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t i = a + k;
    int lo = h0, hi = h1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (off[mid] <= i) lo = mid; else hi = mid - 1; }
    const int32_t v = stage[i];
    if (v < -1 || (int64_t)v >= cell_off[lo + 1] - cell_off[lo]) atomicMin(first_bad, (unsigned long long)k);
}

__global__ void k_delta_h(LatView L, Tables tabs, int h, int64_t n, const int64_t *site, const int32_t *dstv,
                          double *out) {
    __shared__ double sJ[64];
    __shared__ int8_t sreach[3 * 124];
    for (int i = threadIdx.x; i < L.K * L.K; i += blockDim.x) sJ[i] = tabs.J[i];
    for (int i = threadIdx.x; i < 3 * L.nreach; i += blockDim.x) sreach[i] = tabs.reach[i];
    __syncthreads();
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int4 dm = L.dims[h];
    const int64_t c0 = L.cell_off[h], cap = L.cell_off[h + 1] - c0;
    const int32_t *g = L.grid + L.off[h];
    int64_t i = site[q];
    int x = (int)(i % dm.x), y = (int)((i / dm.x) % dm.y), z = (int)(i / ((int64_t)dm.x * dm.y));
    const Vn vn = vn_of(dm, x, y, z);
    int32_t src = g[i], dst = dstv[q];
    double num;
    double c = contact_delta(g, dm, x, y, z, src, dst, L.type + c0, cap, sJ, L.K, sreach, L.nreach, L.across, i, vn,
                             &num);
    double v = volume_delta(L.volume, L.target, L.lambda, c0, src, dst);
    double s = 0.0;
    if (L.surface_on) {
        int32_t ds, dd;
        surface_change(g, i, vn, src, dst, ds, dd);
        s = surface_delta(L.surface, L.tsurf, L.lsurf, c0, src, dst, ds, dd);
    }
    double *o = out + 6 * q;
    o[0] = num; o[1] = c; o[2] = v; o[3] = s; o[4] = c + v; o[5] = (c + v) + s;
}

// Recount volumes (and surfaces) from the grid: recount, cpm.rs:1262-1270.
__global__ void k_recount(const int32_t *grid, const int4 *dims, const int64_t *off, const int64_t *cell_off,
                          const int32_t *blk, int nh, int32_t *vol, int32_t *surf) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    const int32_t *g = grid + off[h];
    int32_t id = g[local];
    int64_t cap = cell_off[h + 1] - cell_off[h];
    if (id < 0 || id >= cap) return;
    atomicAdd(vol + cell_off[h] + id, 1);
    if (surf && id > 0) {
        const int4 dm = dims[h];
        int x = (int)(local % dm.x), y = (int)((local / dm.x) % dm.y), z = (int)(local / ((int64_t)dm.x * dm.y));
        const Vn vn = vn_of(dm, x, y, z);
        int c = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (vn.has(k)) c += g[local + vn.step(k)] != id;
        if (c) atomicAdd(surf + cell_off[h] + id, c);
    }
}

__global__ void k_compare(const int32_t *a, const int32_t *b, const int64_t *cell_off, int h, int *bad) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t c0 = cell_off[h], n = cell_off[h + 1] - c0;
    if (i >= 1 && i < n && a[c0 + i] != b[c0 + i]) atomicAdd(bad, 1);
}

// set_contact_order, cpm.rs:274-301.
int make_reach(int order, bool volume, int8_t *off, double *across) {
    *across = 1.0;
    if (order <= 1) return 0;
    int deep = volume ? 2 : 0;
    std::vector<std::array<int, 3>> cand;
    std::vector<int64_t> dist;
    for (int dz = -deep; dz <= deep; ++dz)
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                cand.push_back({dx, dy, dz});
                dist.push_back((int64_t)dx * dx + dy * dy + dz * dz);
            }
    std::vector<int64_t> u = dist;
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    int64_t limit = u[std::min<size_t>((size_t)(order - 1), u.size() - 1)];
    int n = 0;
    int64_t acr = 0;
    for (size_t i = 0; i < cand.size(); ++i)
        if (dist[i] <= limit) {
            for (int a = 0; a < 3; ++a) off[3 * n + a] = (int8_t)cand[i][a];
            acr += std::max(cand[i][0], 0);
            ++n;
        }
    *across = (double)acr;
    return n;
}

}  // namespace

int cw_lattice_s::build_plans() {
    bool volume = g.d[0] > 1;
    nreach = make_reach(order, volume, reach, &across);
    if (nreach == 0 && !copy_moore) {
        period = 0;
        ncol = 2;
    } else if (nreach == 0) {
        // face contact with diagonal copies: a copy's source must not be a
        // pixel of the same colour, so the chessboard gives way to period 2
        period = 2;
        ncol = volume ? 8 : 4;
    } else {
        int r = 1;
        for (int k = 0; k < 3 * nreach; ++k) r = std::max(r, (int)std::abs(reach[k]));
        period = r + 1;
        ncol = volume ? period * period * period : period * period;
    }
    // the pass plan: chunks of PT sites, as many as the largest colour of each
    // history's box holds (a plane's plan; in a volume a bound of the plan the
    // device takes from the occupied span every Monte Carlo step)
    std::vector<int32_t> vp(g.nh + 1, 0);
    for (uint32_t k = 0; k < g.nh; ++k) {
        const int64_t sites = colour_sites_max(g.w[k], g.h[k], g.d[k], period);
        vp[k + 1] = vp[k] + (int32_t)((sites + PT - 1) / PT);
    }
    int rc;
    if (pass_grid == 0) {
        int per_sm = 0, dev = 0, nsm = 0;
        CW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_cpm_pass, PT, 0));
        CW_CUDA(cudaGetDevice(&dev));
        CW_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        pass_grid = std::max(1, per_sm * nsm);
    }
    // the pass scratch: a block's segment holds every site of the chunks it
    // visits, (chunks / blocks launched, rounded up) x PT
    const int32_t nvb = vp[g.nh];
    pass_blocks = std::max(1, std::min(nvb, pass_grid));
    pass_seg = (int64_t)((nvb + pass_blocks - 1) / pass_blocks) * PT;
    const int64_t need = (int64_t)pass_blocks * pass_seg;
    if (need > plist_cap) {
        dfree(plist);
        dfree(pidx);
        plist_cap = 0;
        if ((rc = dalloc(&plist, 3 * (size_t)need)) != CW_OK) return rc;  // an attempt is 3 uint4
        if ((rc = dalloc(&pidx, 2 * (size_t)need)) != CW_OK) return rc;   // two pending lists
        plist_cap = need;
    }
    if (!d_vplan && (rc = dalloc(&d_vplan, (size_t)g.nh + 1)) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(d_vplan, vp.data(), sizeof(int32_t) * (g.nh + 1), cudaMemcpyHostToDevice, stream()));
    if (!claim) {
        if ((rc = dalloc(&claim, 2 * (size_t)ncells)) != CW_OK) return rc;
        CW_CUDA(cudaMemsetAsync(claim, 0, sizeof(unsigned long long) * 2 * (size_t)ncells, stream()));
    }
    if (!pctl) {
        if ((rc = dalloc(&pctl, CTL_KEYS + 27 * (size_t)g.nh)) != CW_OK) return rc;
        CW_CUDA(cudaMemsetAsync(pctl, 0, sizeof(uint32_t) * (CTL_KEYS + 27 * (size_t)g.nh), stream()));
    }
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

namespace {
struct LatExtra {
    uint32_t *mcs_ctr = nullptr, *mcs_cur = nullptr;
    int32_t *perm = nullptr;
};
}  // namespace

static LatView lat_view(cw_lattice_s *l) {
    LatView v;
    v.grid = l->grid; v.type = l->type; v.volume = l->volume; v.vsnap = l->vsnap; v.target = l->target;
    v.lambda = l->lambda; v.surface = l->surface; v.ssnap = l->ssnap; v.tsurf = l->tsurf; v.lsurf = l->lsurf;
    v.dims = l->g.d_dims; v.off = l->g.d_off; v.cell_off = l->d_cell_off; v.keys = l->d_keys;
    v.K = l->K; v.nreach = l->nreach; v.period = l->period; v.ncol = l->ncol; v.across = l->across;
    v.temperature = l->temperature; v.surface_on = l->surface_on ? 1 : 0; v.copy_moore = l->copy_moore ? 1 : 0;
    v.take_below = l->subsweeps > 1 ? (uint32_t)(4294967296.0 / (double)l->subsweeps) : 0u;
    v.span = l->d_span;
    return v;
}

static Tables lat_tables(const cw_lattice_s *l) {
    Tables t;
    std::memcpy(t.J, l->J, sizeof t.J);
    std::memcpy(t.reach, l->reach, sizeof t.reach);
    return t;
}

// mcs counter (2 words) and colour permutations live in d_flag's neighbours
struct LatDevice {
    uint32_t *mcs;   // [0] counter, [1] current
    int32_t *perm;   // nh * 27
};
static LatDevice dev_of(cw_lattice_s *l) {
    LatDevice d;
    d.mcs = (uint32_t *)l->d_flag;
    d.perm = l->d_flag + 4;
    return d;
}

namespace cw {
int lattice_recount_surfaces(cw_lattice_s *l) {
    Plan &p = l->site_plan;
    if (p.nblocks == 0) {
        std::vector<int64_t> per(l->g.nh);
        for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
        int rc = p.build(per, T);
        if (rc != CW_OK) return rc;
    }
    CW_CUDA(cudaMemsetAsync(l->vsnap, 0, sizeof(int32_t) * l->ncells, stream()));
    CW_CUDA(cudaMemsetAsync(l->surface, 0, sizeof(int32_t) * l->ncells, stream()));
    k_recount<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, l->g.nh,
                                             l->vsnap, l->surface);
    CW_LAUNCHED();
    return CW_OK;
}

int lattice_recount(cw_lattice_s *l, int32_t *vol_out, int32_t *surf_out) {
    std::vector<int64_t> per(l->g.nh);
    for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
    Plan p;
    int rc = p.build(per, T);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(vol_out, 0, sizeof(int32_t) * l->ncells, stream()));
    if (surf_out) CW_CUDA(cudaMemsetAsync(surf_out, 0, sizeof(int32_t) * l->ncells, stream()));
    k_recount<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, l->d_cell_off, p.d_blk, l->g.nh,
                                             vol_out, surf_out);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    p.release();
    return CW_OK;
}

// One Monte Carlo step of every history (no host synchronisation): the
// colour order, then one cooperative launch per colour (its rounds meet at a
// grid barrier), the claims and control words cleared before each.
int lattice_span_enqueue(cw_lattice_s *l) {
    if (!l->d_span) return CW_OK;
    Plan &p = l->site_plan;
    if (p.nblocks == 0) {
        std::vector<int64_t> per(l->g.nh);
        for (uint32_t k = 0; k < l->g.nh; ++k) per[k] = l->g.sites(k);
        int rc = p.build(per, T);
        if (rc != CW_OK) return rc;
    }
    const int nh = (int)l->g.nh;
    k_span_reset<<<(nh + 127) / 128, 128, 0, stream()>>>(l->d_span, nh);
    CW_LAUNCHED();
    k_span_occupied<<<p.nblocks, T, 0, stream()>>>(l->grid, l->g.d_dims, l->g.d_off, p.d_blk, nh, l->d_span);
    CW_LAUNCHED();
    k_span_finish<<<(nh + 127) / 128, 128, 0, stream()>>>(l->d_span, l->g.d_dims, nh);
    CW_LAUNCHED();
    k_pass_plan<<<1, 1024, 0, stream()>>>(l->d_span, nh, l->period, l->d_vplan);
    CW_LAUNCHED();
    return CW_OK;
}

int lattice_sweep(cw_lattice_s *l) {
    int rc0 = lattice_span_enqueue(l);
    if (rc0 != CW_OK) return rc0;
    for (int s = 0; s < std::max(l->subsweeps, 1); ++s) {
        int rc = lattice_subsweep(l);
        if (rc != CW_OK) return rc;
    }
    l->mcs += 1;
    return CW_OK;
}

// One sweep of every colour (a whole Monte Carlo step with one sub-sweep);
// the device's step counter advances by one per sub-sweep.
int lattice_subsweep(cw_lattice_s *l) {
    LatDevice d = dev_of(l);
    k_colour_order<<<1, 128, 0, stream()>>>(l->d_keys, l->g.nh, l->ncol, d.mcs, d.mcs + 1, d.perm,
                                            l->pctl + CTL_KEYS);
    CW_LAUNCHED();
    LatView v = lat_view(l);
    Tables t = lat_tables(l);
    PassScratch S;
    S.claim[0] = l->claim;
    S.claim[1] = l->claim + l->ncells;
    S.list = (Attempt *)l->plist;
    S.idx = l->pidx;
    S.seg = (uint32_t)l->pass_seg;
    S.ncells = l->ncells;
    S.ctl = l->pctl;
    S.vplan = l->d_vplan;
    const TestFaults &tf = test_faults();
    S.barrier_ns = tf.wait_ns ? tf.wait_ns : BARRIER_NS;
    S.withhold = tf.withhold_block;
    S.max_rounds = tf.max_rounds > 0 ? tf.max_rounds : MAX_ROUNDS;
    int nh = (int)l->g.nh;
    const uint32_t *cur = d.mcs + 1;
    for (int q = 0; q < l->ncol; ++q) {
        void *args[] = {&v, &t, &nh, &d.perm, &q, (void *)&cur, &S};
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.gridDim = dim3((unsigned)l->pass_blocks);
        cfg.blockDim = dim3(PT);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream();
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CW_CUDA(cudaLaunchKernelExC(&cfg, (const void *)k_cpm_pass, args));
        count_launch(1);
    }
    return CW_OK;
}

// CW_ERR_TIMEOUT (or CW_ERR_SIMULATION) if a pass gave up since the last
// call: a grid barrier that waited too long, or more rounds than allowed.
int lattice_pass_error(cw_lattice_s *l) {
    uint32_t e = 0;
    CW_CUDA(cudaMemcpy(&e, l->pctl + CTL_ERR, sizeof e, cudaMemcpyDeviceToHost));
    if (!e) return CW_OK;
    // a pass that gave up left its counts, the barrier's arrivals and its
    // claims behind: all start again from zero
    CW_CUDA(cudaMemset(l->pctl, 0, sizeof(uint32_t) * CTL_KEYS));
    CW_CUDA(cudaMemset(l->claim, 0, sizeof(unsigned long long) * 2 * (size_t)l->ncells));
    return e == 1 ? fail(CW_ERR_TIMEOUT, "a sublattice pass waited too long at a grid barrier")
                  : fail(CW_ERR_SIMULATION, "a sublattice pass needed more rounds than allowed");
}
}  // namespace cw

extern "C" {

int cw_lattice_create(uint32_t nh, const uint32_t *w, const uint32_t *h, const uint32_t *d,
                      const uint32_t *cell_capacity, double temperature, cw_lattice *out) {
    *out = nullptr;
    if (nh > 65535) return fail(CW_ERR_CONFIG, "a lattice batch holds at most 65535 histories");
    cw_lattice_s *l = new cw_lattice_s();
    if (l->hs.init() != CW_OK) { delete l; return CW_ERR_CUDA; }
    CW_SCOPE(l);
    int rc = l->g.init(nh, w, h, d);
    if (rc != CW_OK) { delete l; return rc; }
    bool volume = l->g.d[0] > 1;
    for (uint32_t k = 1; k < nh; ++k)
        if ((l->g.d[k] > 1) != volume) {
            l->g.release();
            delete l;
            return fail(CW_ERR_CONFIG, "a batch holds flat lattices or volumes, not both");
        }
    l->cell_off.assign(nh + 1, 0);
    for (uint32_t k = 0; k < nh; ++k) {
        uint32_t cap = std::max<uint32_t>(cell_capacity ? cell_capacity[k] : 1, 1);
        l->cell_off[k + 1] = l->cell_off[k] + cap;
    }
    l->ncells = l->cell_off[nh];
    l->temperature = temperature;
    l->seed.assign(nh, 0);
    int64_t n = l->g.total, nc = l->ncells;
    if ((rc = dalloc(&l->grid, n)) || (rc = dalloc(&l->type, nc)) || (rc = dalloc(&l->volume, nc)) ||
        (rc = dalloc(&l->target, nc)) || (rc = dalloc(&l->lambda, nc)) || (rc = dalloc(&l->vsnap, nc)) ||
        (rc = dalloc(&l->d_cell_off, nh + 1)) || (rc = dalloc(&l->d_keys, nh)) ||
        (rc = dalloc(&l->d_flag, 4 + 27 * (size_t)nh)) || (rc = dalloc(&l->d_used, nh)) ||
        (volume && (rc = dalloc(&l->d_span, 6 * (size_t)nh)))) {
        cw_lattice_destroy(l);
        return rc;
    }
    CW_CUDA(cudaMemsetAsync(l->grid, 0, sizeof(int32_t) * n, stream()));
    CW_CUDA(cudaMemsetAsync(l->type, 0, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(l->volume, 0, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(l->target, 0, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(l->lambda, 0, sizeof(double) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(l->d_keys, 0, sizeof(uint2) * nh, stream()));
    CW_CUDA(cudaMemsetAsync(l->d_flag, 0, sizeof(int32_t) * (4 + 27 * (size_t)nh), stream()));
    l->used.assign(nh, 1);  // the medium's record
    CW_CUDA(cudaMemcpyAsync(l->d_used, l->used.data(), sizeof(int32_t) * nh, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(l->d_cell_off, l->cell_off.data(), sizeof(int64_t) * (nh + 1), cudaMemcpyHostToDevice,
                            stream()));
    l->K = 1;
    l->J[0] = 0.0;
    l->order = 1;
    if ((rc = l->build_plans()) != CW_OK) { cw_lattice_destroy(l); return rc; }
    CW_CUDA(cudaStreamSynchronize(stream()));
    *out = l;
    return CW_OK;
}

int cw_lattice_destroy(cw_lattice l) {
    if (!l) return CW_OK;
    CW_SCOPE(l);
    dfree(l->grid); dfree(l->type); dfree(l->volume); dfree(l->target); dfree(l->lambda); dfree(l->vsnap);
    dfree(l->surface); dfree(l->ssnap); dfree(l->tsurf); dfree(l->lsurf); dfree(l->d_cell_off); dfree(l->d_keys);
    dfree(l->d_flag); dfree(l->claim); dfree(l->plist); dfree(l->pidx); dfree(l->d_vplan); dfree(l->pctl); dfree(l->d_used);
    dfree(l->bath_label); dfree(l->bath_mark); dfree(l->stage); dfree(l->d_bad); dfree(l->d_span);
    l->div.release();
    l->site_plan.release();
    l->g.release();
    l->hs.release();
    delete l;
    return CW_OK;
}

int cw_lattice_capacity(cw_lattice l, uint32_t hist, uint32_t *cap) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    *cap = (uint32_t)(l->cell_off[hist + 1] - l->cell_off[hist]);
    return CW_OK;
}

int cw_lattice_pass_rounds(cw_lattice l, uint32_t *rounds) {
    CW_SCOPE(l);
    uint32_t zero = 0;
    CW_CUDA(cudaStreamSynchronize(stream()));
    CW_CUDA(cudaMemcpy(rounds, l->pctl + CTL_ROUNDS, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    CW_CUDA(cudaMemcpy(l->pctl + CTL_ROUNDS, &zero, sizeof zero, cudaMemcpyHostToDevice));
    return CW_OK;
}

int cw_lattice_set_stream(cw_lattice l, void *stream) {
    CW_SCOPE(l);
    return l->hs.set((cudaStream_t)stream);
}

void *cw_lattice_get_stream(cw_lattice l) { return (void *)l->hs.stream; }

const char *cw_lattice_last_error(cw_lattice l) { return l->hs.err.c_str(); }

int cw_lattice_count(cw_lattice l, uint32_t *nh) {
    CW_SCOPE(l);
    *nh = l->g.nh;
    return CW_OK;
}

int cw_lattice_set_contact(cw_lattice l, int32_t K, const double *J, int32_t order) {
    CW_SCOPE(l);
    if (K < 1 || K > 8) return fail(CW_ERR_CONFIG, "the contact table holds 1 to 8 types, got " + std::to_string(K));
    for (int a = 0; a < K; ++a)
        for (int b = 0; b < K; ++b)
            if (!std::isfinite(J[a * K + b]) || J[a * K + b] != J[b * K + a])
                return fail(CW_ERR_CONFIG, "the contact table must be finite and symmetric");
    l->K = K;
    std::memset(l->J, 0, sizeof l->J);
    std::memcpy(l->J, J, sizeof(double) * K * K);
    l->order = order < 1 ? 1 : order;
    return l->build_plans();
}

int cw_lattice_set_copy_nbhd(cw_lattice l, int32_t nbhd) {
    CW_SCOPE(l);
    if (nbhd != CW_COPY_VON_NEUMANN && nbhd != CW_COPY_MOORE)
        return fail(CW_ERR_CONFIG, "copy neighbourhood " + std::to_string(nbhd) + " is neither von Neumann nor Moore");
    l->copy_moore = nbhd == CW_COPY_MOORE;
    return l->build_plans();
}

int cw_lattice_set_subsweeps(cw_lattice l, int32_t subsweeps) {
    CW_SCOPE(l);
    if (subsweeps < 1 || subsweeps > 64) return fail(CW_ERR_CONFIG, "1 to 64 sub-sweeps a Monte Carlo step");
    l->subsweeps = subsweeps;
    return CW_OK;
}

int cw_lattice_set_temperature(cw_lattice l, double temperature) {
    CW_SCOPE(l);
    if (!(temperature > 0.0)) return fail(CW_ERR_CONFIG, "the temperature must be positive");
    l->temperature = temperature;
    return CW_OK;
}

// Histories h0..h1's sites, staged at `off[h0]`, copied into the grid when
// every id lies in [-1, capacity): the host data lands in the staging buffer,
// a kernel records the first pixel that does not, and only a clean upload
// becomes the grid.
static int upload_range(cw_lattice l, uint32_t h0, uint32_t h1, const int32_t *grid) {
    int rc;
    if (!l->stage && ((rc = dalloc(&l->stage, (size_t)l->g.total)) || (rc = dalloc(&l->d_bad, 1)))) return rc;
    const int64_t a = l->g.off[h0], n = l->g.off[h1 + 1] - a;
    const unsigned long long none = ~0ull;
    CW_CUDA(cudaMemcpyAsync(l->stage + a, grid, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(l->d_bad, &none, sizeof none, cudaMemcpyHostToDevice, stream()));
    k_check_ids<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(l->stage, a, n, l->g.d_off, l->d_cell_off, (int)h0,
                                                                 (int)h1, l->d_bad);
    CW_LAUNCHED();
    unsigned long long bad = none;
    CW_CUDA(cudaMemcpyAsync(&bad, l->d_bad, sizeof bad, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    if (bad != none) {
        uint32_t h = h0;
        while (h < h1 && l->g.off[h + 1] <= a + (int64_t)bad) ++h;
        const int64_t i = a + (int64_t)bad - l->g.off[h];
        return fail(CW_ERR_CONFIG, "pixel " + std::to_string(i) + " holds id " + std::to_string(grid[bad]) +
                                       ", past the history's cell capacity " +
                                       std::to_string(l->cell_off[h + 1] - l->cell_off[h]));
    }
    CW_CUDA(cudaMemcpyAsync(l->grid + a, l->stage + a, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, stream()));
    return CW_OK;
}

int cw_lattice_upload(cw_lattice l, uint32_t hist, const int32_t *grid) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    return upload_range(l, hist, hist, grid);
}

int cw_lattice_upload_all(cw_lattice l, const int32_t *grids) {
    CW_SCOPE(l);
    if (l->g.nh == 0) return CW_OK;
    return upload_range(l, 0, l->g.nh - 1, grids);
}

int cw_lattice_download(cw_lattice l, uint32_t hist, int32_t *grid) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    CW_CUDA(cudaMemcpyAsync(grid, l->grid + l->g.off[hist], sizeof(int32_t) * l->g.sites(hist), cudaMemcpyDeviceToHost,
                            stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_lattice_download_all(cw_lattice l, int32_t *grids) {
    CW_SCOPE(l);
    CW_CUDA(cudaMemcpyAsync(grids, l->grid, sizeof(int32_t) * l->g.total, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

static int check_cells(cw_lattice l, uint32_t hist, uint32_t n) {
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    if ((int64_t)n > l->cell_off[hist + 1] - l->cell_off[hist])
        return fail(CW_ERR_CONFIG, "more records than the history's cell capacity");
    return CW_OK;
}

int cw_cells_set(cw_lattice l, uint32_t hist, uint32_t n, const int32_t *type, const int32_t *volume,
                 const int32_t *target, const double *lambda) {
    CW_SCOPE(l);
    int rc = check_cells(l, hist, n);
    if (rc != CW_OK) return rc;
    for (uint32_t i = 0; i < n; ++i)
        if (type && (type[i] < 0 || type[i] >= l->K))
            return fail(CW_ERR_CONFIG, "cell " + std::to_string(i) + " has type " + std::to_string(type[i]) +
                                           " outside the contact table");
    int64_t c0 = l->cell_off[hist];
    if ((int32_t)n > l->used[hist]) {
        l->used[hist] = (int32_t)n;
        CW_CUDA(cudaMemcpyAsync(l->d_used + hist, &l->used[hist], sizeof(int32_t), cudaMemcpyHostToDevice, stream()));
    }
    if (type) CW_CUDA(cudaMemcpyAsync(l->type + c0, type, 4 * n, cudaMemcpyHostToDevice, stream()));
    if (volume) CW_CUDA(cudaMemcpyAsync(l->volume + c0, volume, 4 * n, cudaMemcpyHostToDevice, stream()));
    if (target) CW_CUDA(cudaMemcpyAsync(l->target + c0, target, 4 * n, cudaMemcpyHostToDevice, stream()));
    if (lambda) CW_CUDA(cudaMemcpyAsync(l->lambda + c0, lambda, 8 * n, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_cells_get(cw_lattice l, uint32_t hist, uint32_t n, int32_t *type, int32_t *volume, int32_t *target,
                 double *lambda) {
    CW_SCOPE(l);
    int rc = check_cells(l, hist, n);
    if (rc != CW_OK) return rc;
    int64_t c0 = l->cell_off[hist];
    if (type) CW_CUDA(cudaMemcpyAsync(type, l->type + c0, 4 * n, cudaMemcpyDeviceToHost, stream()));
    if (volume) CW_CUDA(cudaMemcpyAsync(volume, l->volume + c0, 4 * n, cudaMemcpyDeviceToHost, stream()));
    if (target) CW_CUDA(cudaMemcpyAsync(target, l->target + c0, 4 * n, cudaMemcpyDeviceToHost, stream()));
    if (lambda) CW_CUDA(cudaMemcpyAsync(lambda, l->lambda + c0, 8 * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_cells_set_surface(cw_lattice l, uint32_t hist, uint32_t n, const int32_t *target_surface,
                         const double *lambda_surface) {
    CW_SCOPE(l);
    int rc = check_cells(l, hist, n);
    if (rc != CW_OK) return rc;
    if (!l->surface_on) {
        int64_t nc = l->ncells;
        if ((rc = dalloc(&l->surface, nc)) || (rc = dalloc(&l->ssnap, nc)) || (rc = dalloc(&l->tsurf, nc)) ||
            (rc = dalloc(&l->lsurf, nc)))
            return rc;
        CW_CUDA(cudaMemsetAsync(l->tsurf, 0, 4 * nc, stream()));
        CW_CUDA(cudaMemsetAsync(l->lsurf, 0, 8 * nc, stream()));
        l->surface_on = true;
    }
    int64_t c0 = l->cell_off[hist];
    CW_CUDA(cudaMemcpyAsync(l->tsurf + c0, target_surface, 4 * n, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(l->lsurf + c0, lambda_surface, 8 * n, cudaMemcpyHostToDevice, stream()));
    return lattice_recount(l, l->vsnap, l->surface);  // vsnap is scratch until the next pass
}

int cw_cells_get_surface(cw_lattice l, uint32_t hist, uint32_t n, int32_t *surface) {
    CW_SCOPE(l);
    int rc = check_cells(l, hist, n);
    if (rc != CW_OK) return rc;
    if (!l->surface_on) return fail(CW_ERR_NOT_FOUND, "the surface constraint is off");
    CW_CUDA(cudaMemcpyAsync(surface, l->surface + l->cell_off[hist], 4 * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_lattice_set_seed(cw_lattice l, uint32_t hist, uint64_t seed) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    l->seed[hist] = seed;
    uint2 k = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    CW_CUDA(cudaMemcpyAsync(l->d_keys + hist, &k, sizeof k, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_lattice_set_mcs(cw_lattice l, uint32_t mcs) {
    CW_SCOPE(l);
    l->mcs = mcs;
    // the draws count sub-sweeps
    const uint32_t eff = mcs * (uint32_t)std::max(l->subsweeps, 1);
    CW_CUDA(cudaMemcpyAsync(l->d_flag, &eff, sizeof eff, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_lattice_get_mcs(cw_lattice l, uint32_t *mcs) {
    CW_SCOPE(l);
    *mcs = l->mcs;
    return CW_OK;
}

int cw_lattice_mcs(cw_lattice l, uint32_t sweeps) {
    CW_SCOPE(l);
    for (uint32_t s = 0; s < sweeps; ++s) {
        int rc = lattice_sweep(l);
        if (rc != CW_OK) return rc;
    }
    CW_CUDA(cudaStreamSynchronize(stream()));
    return lattice_pass_error(l);
}

int cw_lattice_delta_h_batch(cw_lattice l, uint32_t hist, uint32_t n, const int64_t *site, const int32_t *dst,
                             double *out) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    if (n == 0) return CW_OK;
    int64_t ns = l->g.sites(hist), cap = l->cell_off[hist + 1] - l->cell_off[hist];
    for (uint32_t q = 0; q < n; ++q)
        if (site[q] < 0 || site[q] >= ns || dst[q] < -1 || dst[q] >= cap)
            return fail(CW_ERR_CONFIG, "proposal " + std::to_string(q) + " is outside the lattice or the records");
    int64_t *d_site;
    int32_t *d_dst;
    double *d_out;
    int rc;
    if ((rc = dalloc(&d_site, n)) || (rc = dalloc(&d_dst, n)) || (rc = dalloc(&d_out, 6 * (size_t)n))) return rc;
    CW_CUDA(cudaMemcpyAsync(d_site, site, 8 * (size_t)n, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(d_dst, dst, 4 * (size_t)n, cudaMemcpyHostToDevice, stream()));
    k_delta_h<<<(n + T - 1) / T, T, 0, stream()>>>(lat_view(l), lat_tables(l), (int)hist, n, d_site, d_dst, d_out);
    CW_LAUNCHED();
    CW_CUDA(cudaMemcpyAsync(out, d_out, 48 * (size_t)n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_site); dfree(d_dst); dfree(d_out);
    return CW_OK;
}

int cw_lattice_verify(cw_lattice l, uint32_t hist, int32_t *ok) {
    CW_SCOPE(l);
    if (hist >= l->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int32_t *vol, *surf = nullptr;
    int *bad;
    int rc;
    if ((rc = dalloc(&vol, l->ncells)) || (rc = dalloc(&bad, 1))) return rc;
    if (l->surface_on && (rc = dalloc(&surf, l->ncells)) != CW_OK) return rc;
    if ((rc = lattice_recount(l, vol, surf)) != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), stream()));
    int64_t cap = l->cell_off[hist + 1] - l->cell_off[hist];
    unsigned nb = (unsigned)((cap + T - 1) / T);
    k_compare<<<nb, T, 0, stream()>>>(vol, l->volume, l->d_cell_off, (int)hist, bad);
    CW_LAUNCHED();
    if (surf) {
        k_compare<<<nb, T, 0, stream()>>>(surf, l->surface, l->d_cell_off, (int)hist, bad);
        CW_LAUNCHED();
    }
    int hbad = 0;
    CW_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    *ok = hbad == 0;
    dfree(vol); dfree(bad); dfree(surf);
    return CW_OK;
}

}  // extern "C"
