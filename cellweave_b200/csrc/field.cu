// Diffusion field: ScalarField of crates/engine/src/pde.rs on the device.
//
// Two solvers stand side by side:
//  * CW_FP64: the reference's red-black SOR (relax / sor_sweep / half_sweep,
//    pde.rs:245-405) pixel for pixel in FP64.  This file is built without
//    fused multiply-add, so each pixel's update rounds exactly as the Rust
//    does, and red-black order makes the in-place update equal to the
//    reference's read-one-buffer/write-the-other (pde.rs:322-328): the field
//    and the sweep count are bit-identical to the reference's.
//  * CW_FP32_DC: defect correction.  The FP64 residual r = b - A c is formed,
//    A d = r is relaxed in FP32 by red-black SOR sweeps (field32.cu, kept in
//    shared memory several half-sweeps deep), and c += d in FP64, until the
//    projected residual is below the tolerance.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "cw_internal.cuh"
#include "field_kernels.cuh"
#include "tma.cuh"

using namespace cw;

namespace {

struct RelaxState {
    unsigned long long moved[2];  // max |change| of the red and the black half-sweep
    unsigned long long resid;     // max projected residual
    double omega;
    double tol;
    int64_t sweeps;               // sweeps taken, final once done
    int32_t done;                 // 0 running, 1 converged
    int32_t stop;
    double last_change;
    double last_resid;
    int64_t inner;                // FP32 sweeps taken (defect correction)
    // the error estimate of the defect-correction solve (the wide sweeps'
    // apply): the largest |correction| of the last outer iteration and the
    // largest |c| it left, as the bits of non-negative doubles (atomic max),
    // the previous iteration's largest correction, and the bound asked
    unsigned long long corr;
    unsigned long long cmax;
    double prev_corr;
    double etol;
};

// (a history holds fewer than 2^31 pixels: 32-bit division is enough)
__device__ __forceinline__ void locate(const int4 dm, int64_t local, int &x, int &y, int &z) {
    const uint32_t l = (uint32_t)local, w = (uint32_t)dm.x, h = (uint32_t)dm.y;
    const uint32_t r = l / w;
    x = (int)(l - r * w);
    y = (int)(r % h);
    z = (int)(r / h);
}

// The box around every free pixel (free_span, pde.rs:305-320).
__global__ void k_span(const uint8_t *__restrict__ held, const int4 *dims, const int64_t *off, const int32_t *blk,
                       int nh, Span *span) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    int64_t n = off[h + 1] - off[h];
    bool ok = local < n && !held[off[h] + local];
    int x = 0, y = 0, z = 0;
    if (ok) locate(dims[h], local, x, y, z);
    // warp-level reduction first, then one atomic per warp
    int xmin = ok ? x : INT_MAX, xmax = ok ? x : -1, ymin = ok ? y : INT_MAX, ymax = ok ? y : -1;
    int zmin = ok ? z : INT_MAX, zmax = ok ? z : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
        xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
        ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
        ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
        zmin = min(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
        zmax = max(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    }
    if ((threadIdx.x & 31) == 0 && xmax >= 0) {
        atomicMin(&span[h].x0, xmin); atomicMax(&span[h].x1, xmax);
        atomicMin(&span[h].y0, ymin); atomicMax(&span[h].y1, ymax);
        atomicMin(&span[h].z0, zmin); atomicMax(&span[h].z1, zmax);
        span[h].found = 1;
    }
}

__global__ void k_span_reset(Span *span, int nh) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < nh) span[h] = Span{INT_MAX, -1, INT_MAX, -1, INT_MAX, -1, 0, 0};
}

// One half-sweep of the reference's SOR, in place, FP64 (half_sweep,
// pde.rs:329-405).  Items enumerate the pixels of `colour` inside the span.
__global__ void k_sor64_half(FieldView fv, const int32_t *blk, int nh, const Span *span, RelaxState *st,
                             int colour) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    if (st[h].done) return;
    const Span sp = span[h];
    const int4 dm = fv.dims[h];
    int sw = sp.x1 - sp.x0 + 1, hw = (sw + 1) >> 1, ny = sp.y1 - sp.y0 + 1;
    int64_t k = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    double moved = 0.0;
    int64_t rows = (int64_t)ny * (sp.z1 - sp.z0 + 1);
    if (k < rows * hw) {
        int64_t row = k / hw;
        int j = (int)(k - row * hw);
        int y = sp.y0 + (int)(row % ny), z = sp.z0 + (int)(row / ny);
        int x = sp.x0 + ((colour - (sp.x0 + y + z)) & 1) + 2 * j;
        if (x <= sp.x1) {
            int64_t i = fv.off[h] + ((int64_t)z * dm.y + y) * dm.x + x;
            if (!fv.held[i]) {
                double before = fv.c[i];
                double sum, real;
                pixel_sums64(fv.c, i, x, y, z, dm, sum, real);
                double den = real * fv.d + fv.decay;
                if (fv.ks) den = den + fv.ks[i];
                double balanced = add_sources(fv, i, fv.d * sum) / den;
                double om = st[h].omega;
                double after = (1.0 - om) * before + om * balanced;
                if (fv.floor) after = fmax(after, 0.0);
                fv.c[i] = after;
                moved = fabs(after - before);
            }
        }
    }
    block_max_to(&st[h].moved[colour], moved);
}

// Rows per block of the residual kernel (and of its launch plan, row_plan).
constexpr int RES_ROWS = 4;

// Projected residual max |b - A c| over the free pixels of each history;
// optionally writes the FP32 coefficients of the defect-correction solve's
// SOR on A d = r, the relaxation factor folded in: omega r / den and
// omega D / den (both 0 on held pixels), and zeroes the correction.
// The FP32 coefficients of the defect-correction sweep at a free pixel:
// b = omega r / den and a = omega D / den, scaled by q = omega / den formed
// in FP32 by the fast reciprocal division (within 2 ulp; the same q for a and
// b of a pixel, so the FP32 equation is only rescaled, and its error is the
// FP32 solve's, removed by the FP64 residual; r itself is FP64).
__device__ __forceinline__ void dc_coefficients(double om, double den, double r, double d, float &b, float &a) {
    b = a = 0.0f;
    if (den > 0.0) {
        const float q = __fdividef((float)om, (float)den);
        b = q * (float)r;
        a = q * (float)d;
    }
}

__global__ void __launch_bounds__(256) k_residual64(FieldView fv, const int32_t *blk, int nh, RelaxState *st,
                                                    float *r32, float *inv32, float *dz, int skip_done) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    if (skip_done && st[h].done) return;
    const int4 dm = fv.dims[h];
    const double om = st[h].omega;
    // one block: 256 consecutive pixels of each of RES_ROWS consecutive rows
    const uint32_t segs = ((uint32_t)dm.x + 255u) / 256u;
    const uint32_t lb = blockIdx.x - blk[h];
    const uint32_t row0 = (lb / segs) * RES_ROWS;
    const uint32_t nrows = (uint32_t)dm.y * (uint32_t)dm.z;
    const int x = (int)((lb % segs) * 256u + threadIdx.x);
    double worst = 0.0;
    for (uint32_t row = row0; row < row0 + RES_ROWS && row < nrows; ++row) {
        if (x >= dm.x) break;
        const int y = (int)(row % (uint32_t)dm.y), z = (int)(row / (uint32_t)dm.y);
        int64_t i = fv.off[h] + (int64_t)row * dm.x + x;
        float r_out = 0.0f, inv_out = 0.0f;
        if (!fv.held[i]) {
            double sum, real;
            pixel_sums64(fv.c, i, x, y, z, dm, sum, real);
            double den = real * fv.d + fv.decay;
            if (fv.ks) den = den + fv.ks[i];
            double cv = fv.c[i];
            double r = add_sources(fv, i, fv.d * sum) - den * cv;
            if (fv.floor && cv <= 0.0 && r < 0.0) r = 0.0;
            worst = fmax(worst, fabs(r));
            dc_coefficients(om, den, r, fv.d, r_out, inv_out);
        }
        if (r32) r32[i] = r_out;
        if (inv32) inv32[i] = inv_out;
        if (dz) dz[i] = 0.0f;
    }
    block_max_to(&st[h].resid, worst);
}

// After sweep `index`: decide convergence (relax's `moved < tolerance`,
// pde.rs:280-283, or the residual rule) and reset the accumulators.
// The stop test after each FP64 sweep; a running history counts the sweep
// (so that a chunk of sweeps launches with the same arguments every time).
__global__ void k_check(RelaxState *st, int nh, int residual_counted) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    RelaxState &s = st[h];
    if (!s.done) {
        double m = fmax(__longlong_as_double((long long)s.moved[0]), __longlong_as_double((long long)s.moved[1]));
        double r = __longlong_as_double((long long)s.resid);
        s.last_change = m;
        if (residual_counted) s.last_resid = r;
        bool conv = s.stop == CW_STOP_RESIDUAL ? r < s.tol : m < s.tol;
        s.sweeps += 1;
        if (conv) s.done = 1;
    }
    s.moved[0] = s.moved[1] = 0ull;
    s.resid = 0ull;
}

// Defect correction fused with the next residual, in two launches, one per
// colour: c += d (floored at zero as the reference's update is, pde.rs:395),
// then r = b - A c at the corrected field, written in FP32 as omega r / den
// for the next FP32 solve, with the correction zeroed behind it.  The first launch corrects the
// red pixels and reads its black neighbours as c + d; the second corrects the
// black ones and reads its red neighbours as they now stand, so no thread
// reads a value another thread of the same launch writes.  One block takes
// 512 consecutive pixels of one row, a thread the pair (2t, 2t+1): one
// pixel of each colour.
__global__ void __launch_bounds__(256) k_dc_update(FieldView fv, const int32_t *blk, int nh, RelaxState *st,
                                                   float *dlt, float *r32, int colour) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    if (st[h].done) return;
    const int4 dm = fv.dims[h];
    const uint32_t segs = ((uint32_t)dm.x + 511u) / 512u;
    const uint32_t lb = blockIdx.x - blk[h];
    const uint32_t row = lb / segs, seg = lb - row * segs;
    const int y = (int)(row % (uint32_t)dm.y), z = (int)(row / (uint32_t)dm.y);
    const int x = (int)seg * 512 + 2 * (int)threadIdx.x + ((colour + y + z) & 1);
    double worst = 0.0;
    if (x < dm.x) {
        const int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
        const int64_t i = fv.off[h] + (int64_t)row * w + x;
        if (!fv.held[i]) {
            const bool red = colour == 0;
            const bool fl = fv.floor;
            auto nb = [&](int64_t j) -> double {
                double cj = fv.c[j];
                if (red && !fv.held[j]) {
                    cj = cj + (double)dlt[j];
                    if (fl) cj = fmax(cj, 0.0);
                }
                return cj;
            };
            double ci = fv.c[i] + (double)dlt[i];
            if (fl) ci = fmax(ci, 0.0);
            double sum = 0.0, real = 0.0;
            if (x > 0) { sum += nb(i - 1); real += 1.0; }
            if (x + 1 < dm.x) { sum += nb(i + 1); real += 1.0; }
            if (y > 0) { sum += nb(i - w); real += 1.0; }
            if (y + 1 < dm.y) { sum += nb(i + w); real += 1.0; }
            if (z > 0) { sum += nb(i - slice); real += 1.0; }
            if (z + 1 < dm.z) { sum += nb(i + slice); real += 1.0; }
            double den = real * fv.d + fv.decay;
            if (fv.ks) den = den + fv.ks[i];
            double r = add_sources(fv, i, fv.d * sum) - den * ci;
            if (fl && ci <= 0.0 && r < 0.0) r = 0.0;
            worst = fabs(r);
            fv.c[i] = ci;
            float b32, a32;
            dc_coefficients(st[h].omega, den, r, fv.d, b32, a32);
            r32[i] = b32;
            dlt[i] = 0.f;
        }
    }
    block_max_to(&st[h].resid, worst);
}

// The error a contraction leaves after a correction of largest size c whose
// ratio to the one before is q < 1: the corrections to come sum to at most
// c q / (1 - q) if the ratio holds; doubled for the ratio's wobble.  A zero
// correction leaves nothing; no ratio (the first correction, or q >= 1)
// gives no estimate (a huge one).
__device__ __forceinline__ double error_estimate(double c, double prev) {
    if (c == 0.0) return 0.0;
    if (!(prev > 0.0) || c >= prev) return 1e308;
    double q = c / prev;
    return 2.0 * c * q / (1.0 - q);
}

// `estimated`: the sweeps report their corrections (the wide apply), and a
// history with etol > 0 also waits for its error estimate to fall below etol
// times its largest |c|.
__global__ void k_dc_check(RelaxState *st, int nh, int inner, int64_t max_sweeps, int estimated) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    RelaxState &s = st[h];
    if (!s.done) {
        double r = __longlong_as_double((long long)s.resid);
        s.last_resid = r;
        double c = __longlong_as_double((long long)s.corr);
        bool close = true;
        if (estimated && s.etol > 0.0)
            close = s.inner > 0 && error_estimate(c, s.prev_corr) < s.etol * __longlong_as_double((long long)s.cmax);
        if (r < s.tol && close) s.done = 1;
        else if (s.inner >= max_sweeps) s.done = 2;  // out of sweeps: reported as not settled
        else { s.inner += inner; s.sweeps = s.inner; }
        s.prev_corr = c;
    }
    s.resid = 0ull;
    s.corr = 0ull;
    s.cmax = 0ull;
}

// The test of k_dc_check without its bookkeeping: marks what settled and
// records the residual, leaving the accumulator for the next k_dc_check.
__global__ void k_dc_peek(RelaxState *st, int nh, int estimated) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    RelaxState &s = st[h];
    if (!s.done) {
        double r = __longlong_as_double((long long)s.resid);
        s.last_resid = r;
        bool close = true;
        if (estimated && s.etol > 0.0)
            close = s.inner > 0 && error_estimate(__longlong_as_double((long long)s.corr), s.prev_corr) <
                                       s.etol * __longlong_as_double((long long)s.cmax);
        if (r < s.tol && close) s.done = 1;
    }
}

// inflow (pde.rs:415-456): flux from held pixels into free ones; with
// `free_count`, the free pixels counted too (free_count, pde.rs:459-462).
__global__ void k_inflow(FieldView fv, const int32_t *blk, int nh, double *out,
                         unsigned long long *free_count = nullptr) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    const int4 dm = fv.dims[h];
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    double flux = 0.0;
    if (local < fv.off[h + 1] - fv.off[h]) {
        int64_t i = fv.off[h] + local;
        if (!fv.held[i]) {
            int x, y, z;
            locate(dm, local, x, y, z);
            int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
            double ci = fv.c[i];
            if (x > 0 && fv.held[i - 1]) flux += fv.d * (fv.c[i - 1] - ci);
            if (x + 1 < dm.x && fv.held[i + 1]) flux += fv.d * (fv.c[i + 1] - ci);
            if (y > 0 && fv.held[i - w]) flux += fv.d * (fv.c[i - w] - ci);
            if (y + 1 < dm.y && fv.held[i + w]) flux += fv.d * (fv.c[i + w] - ci);
            if (z > 0 && fv.held[i - slice]) flux += fv.d * (fv.c[i - slice] - ci);
            if (z + 1 < dm.z && fv.held[i + slice]) flux += fv.d * (fv.c[i + slice] - ci);
        }
    }
    flux = warp_sum(flux);
    if ((threadIdx.x & 31) == 0 && flux != 0.0) atomicAdd(out + h, flux);
    if (free_count) {
        const bool free = local < fv.off[h + 1] - fv.off[h] && !fv.held[fv.off[h] + local];
        const unsigned n = __popc(__ballot_sync(0xffffffffu, free));
        if ((threadIdx.x & 31) == 0 && n) atomicAdd(free_count + h, (unsigned long long)n);
    }
}

// DiffusionField::step (pde.rs:705-728), out of place.
__global__ void k_explicit(FieldView fv, const int32_t *blk, int nh, double dt, double *next) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    const int4 dm = fv.dims[h];
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= fv.off[h + 1] - fv.off[h]) return;
    int64_t i = fv.off[h] + local;
    double c = fv.c[i];
    if (fv.held[i]) { next[i] = c; return; }
    int x, y, z;
    locate(dm, local, x, y, z);
    int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    double a = x > 0 ? fv.c[i - 1] : c;
    double b = x + 1 < dm.x ? fv.c[i + 1] : c;
    double e = y > 0 ? fv.c[i - w] : c;
    double g = y + 1 < dm.y ? fv.c[i + w] : c;
    double lap = a + b + e + g - 4.0 * c;
    if (dm.z > 1) {
        double p = z > 0 ? fv.c[i - slice] : c;
        double q = z + 1 < dm.z ? fv.c[i + slice] : c;
        lap += p + q - 2.0 * c;
    }
    double change = add_sources(fv, i, fv.d * lap - fv.decay * c);
    next[i] = fmax(c + dt * change, 0.0);
}

__global__ void k_fill64(double *p, int64_t n, double v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_hold_mask(double *c, uint8_t *held, const uint8_t *mask, int64_t n, double v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && mask[i]) { held[i] = 1; c[i] = v; }
}

// ---- bath (hold_bath_at, pde.rs:550-631) ------------------------------------
__global__ void k_bath_box(const uint8_t *open, const int4 *dims, const int64_t *off, const int32_t *blk, int nh,
                           Span *box) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    if (open[off[h] + local]) return;
    int x, y, z;
    locate(dims[h], local, x, y, z);
    atomicMin(&box[h].x0, x); atomicMax(&box[h].x1, x);
    atomicMin(&box[h].y0, y); atomicMax(&box[h].y1, y);
    atomicMin(&box[h].z0, z); atomicMax(&box[h].z1, z);
    box[h].found = 1;
}

__device__ __forceinline__ bool in_box(const Span &b, const int4 dm, int x, int y, int z, Span &e) {
    e.x0 = max(b.x0 - 1, 0); e.x1 = min(b.x1 + 1, dm.x - 1);
    e.y0 = max(b.y0 - 1, 0); e.y1 = min(b.y1 + 1, dm.y - 1);
    e.z0 = max(b.z0 - 1, 0); e.z1 = min(b.z1 + 1, dm.z - 1);
    return b.found && e.x0 <= x && x <= e.x1 && e.y0 <= y && y <= e.y1 && e.z0 <= z && z <= e.z1;
}

__global__ void k_bath_init(const uint8_t *open, uint8_t *held, const int4 *dims, const int64_t *off,
                            const int32_t *blk, int nh, const Span *box, int only_hist) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    if (only_hist >= 0 && h != only_hist) return;
    const int4 dm = dims[h];
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    int64_t i = off[h] + local;
    int x, y, z;
    locate(dm, local, x, y, z);
    Span e;
    if (!in_box(box[h], dm, x, y, z, e)) { held[i] = 1; return; }
    bool outer = x == e.x0 || x == e.x1 || y == e.y0 || y == e.y1 || (dm.z > 1 && (z == e.z0 || z == e.z1));
    if (outer && open[i]) held[i] = 1;
}

// Spread the bath one step through faces, in place (monotone, so stale reads
// only delay); `changed` counts pixels newly reached.
__global__ void k_bath_spread(const uint8_t *open, uint8_t *held, const int4 *dims, const int64_t *off,
                              const int32_t *blk, int nh, const Span *box, int only_hist, int *changed) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    if (only_hist >= 0 && h != only_hist) return;
    const int4 dm = dims[h];
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    int64_t i = off[h] + local;
    if (held[i] || !open[i]) return;
    int x, y, z;
    locate(dm, local, x, y, z);
    int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    bool r = (x > 0 && held[i - 1]) || (x + 1 < dm.x && held[i + 1]) || (y > 0 && held[i - w]) ||
             (y + 1 < dm.y && held[i + w]) || (z > 0 && held[i - slice]) || (z + 1 < dm.z && held[i + slice]);
    if (r) {
        held[i] = 1;
        atomicAdd(changed, 1);
    }
}

__global__ void k_bath_values(double *c, const uint8_t *held, const int64_t *off, const int32_t *blk, int nh,
                              int only_hist, double v) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    int h = s_h;
    if (only_hist >= 0 && h != only_hist) return;
    int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    int64_t i = off[h] + local;
    if (held[i]) c[i] = v;
}

constexpr int T = 256;

int64_t blocks_for(int64_t n) { return (n + T - 1) / T; }

struct SitePlan {
    // per-handle plan over every site of every history, built once
    Plan p;
};

}  // namespace

// ---------------------------------------------------------------------------
namespace cw {

FieldView view(cw_field_s *f) {
    FieldView v;
    v.c = f->c; v.held = f->held; v.up = f->uptake_on ? f->uptake : nullptr;
    v.pr = f->production_on ? f->production : nullptr;
    v.ks = f->lin_sink_on ? f->lin_sink : nullptr;
    v.d = f->dcoef; v.decay = f->decay; v.source = f->source;
    v.floor = f->floor ? 1 : 0;
    v.dims = f->g.d_dims; v.off = f->g.d_off;
    return v;
}

// One block per 256 consecutive pixels of a row (k_residual64's mapping).
static int row_plan(cw_field_s *f, Plan &p) {
    std::vector<int64_t> per(f->g.nh);
    for (uint32_t k = 0; k < f->g.nh; ++k)
        per[k] = ((int64_t)f->g.h[k] * f->g.d[k] + RES_ROWS - 1) / RES_ROWS * ((f->g.w[k] + 255) / 256);
    return p.build(per, 1);
}

static int site_plan(cw_field_s *f, Plan &p) {
    std::vector<int64_t> per(f->g.nh);
    for (uint32_t k = 0; k < f->g.nh; ++k) per[k] = f->g.sites(k);
    return p.build(per, T);
}

int field_span(cw_field_s *f, std::vector<Span> &spans) {
    Plan p;
    int rc = site_plan(f, p);
    if (rc != CW_OK) return rc;
    k_span_reset<<<(f->g.nh + 63) / 64, 64, 0, stream()>>>(f->d_span, f->g.nh);
    CW_LAUNCHED();
    k_span<<<p.nblocks, T, 0, stream()>>>(f->held, f->g.d_dims, f->g.d_off, p.d_blk, f->g.nh, f->d_span);
    CW_LAUNCHED();
    spans.resize(f->g.nh);
    CW_CUDA(cudaMemcpyAsync(spans.data(), f->d_span, sizeof(Span) * f->g.nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    p.release();
    return CW_OK;
}

}  // namespace cw

int cw_field_s::alloc_fp32() {
    if (r32) return CW_OK;
    int rc;
    int64_t n = g.total;
    if ((rc = dalloc(&r32, n)) != CW_OK) return rc;
    if ((rc = dalloc(&d32a, n)) != CW_OK) return rc;
    if ((rc = dalloc(&d32b, n)) != CW_OK) return rc;
    if ((rc = dalloc(&inv32, n)) != CW_OK) return rc;
    return CW_OK;
}

// The reference's relaxation factor (pde.rs:267-277), on the host.
static double auto_omega(const cw_field_s *f, uint32_t k, const Span &s) {
    if (f->g.d[k] > 1) {
        int32_t l = std::max({s.x1 - s.x0 + 1, s.y1 - s.y0 + 1, s.z1 - s.z0 + 1});
        l = std::max(l, 2);
        return 2.0 / (1.0 + std::sin(3.14159265358979323846 / (double)l));
    }
    double n = (double)std::max(f->g.w[k], f->g.h[k]);
    return std::min(2.0 / (1.0 + std::sin(3.14159265358979323846 / n)), 1.95);
}

static int relax_fp64(cw_field_s *f, const cw_relax_opts &o, std::vector<Span> &spans, RelaxState *d_st,
                      std::vector<RelaxState> &hs) {
    uint32_t nh = f->g.nh;
    FieldView fv = view(f);
    // per-colour plans over the span
    Plan pc[2], ps;
    for (int colour = 0; colour < 2; ++colour) {
        std::vector<int64_t> per(nh, 0);
        for (uint32_t k = 0; k < nh; ++k) {
            const Span &s = spans[k];
            if (!s.found) continue;
            int64_t hw = (s.x1 - s.x0 + 2) / 2;
            per[k] = hw * (int64_t)(s.y1 - s.y0 + 1) * (s.z1 - s.z0 + 1);
        }
        int rc = pc[colour].build(per, T);
        if (rc != CW_OK) return rc;
    }
    int rc = site_plan(f, ps);
    if (rc != CW_OK) return rc;
    Plan prow;
    if ((rc = row_plan(f, prow)) != CW_OK) return rc;
    bool resid = o.stop == CW_STOP_RESIDUAL;
    auto sweep = [&]() -> int {
        for (int colour = 0; colour < 2; ++colour) {
            if (pc[colour].nblocks == 0) continue;
            k_sor64_half<<<pc[colour].nblocks, T, 0, stream()>>>(fv, pc[colour].d_blk, nh, f->d_span, d_st, colour);
            CW_LAUNCHED();
        }
        if (resid) {
            k_residual64<<<prow.nblocks, T, 0, stream()>>>(fv, prow.d_blk, nh, d_st, nullptr, nullptr, nullptr, 1);
            CW_LAUNCHED();
        }
        k_check<<<(nh + 63) / 64, 64, 0, stream()>>>(d_st, nh, resid ? 1 : 0);
        CW_LAUNCHED();
        return CW_OK;
    };
    // The first GRAPH_SWEEPS sweeps launched one by one; a solve that goes on
    // replays them captured as one graph (the same launches with the same
    // arguments), 1, 2, 4, ... up to 32 replays between checks, the last few
    // sweeps below a whole chunk launched one by one again.
    constexpr int64_t GRAPH_SWEEPS = 8;
    cudaGraphExec_t chunk_graph = nullptr;
    int64_t done_sweeps = 0, reps = 1;
    bool first = true;
    while (done_sweeps < o.max_sweeps) {
        const int64_t left = o.max_sweeps - done_sweeps;
        if (first || left < GRAPH_SWEEPS) {
            const int64_t n = std::min(GRAPH_SWEEPS, left);
            for (int64_t s = 0; s < n; ++s)
                if ((rc = sweep()) != CW_OK) return rc;
            done_sweeps += n;
            first = false;
        } else {
            if (!chunk_graph) {
                cudaGraph_t g = nullptr;
                CW_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
                for (int64_t s = 0; s < GRAPH_SWEEPS && rc == CW_OK; ++s) rc = sweep();
                cudaError_t e = cudaStreamEndCapture(stream(), &g);
                if (rc != CW_OK) { if (g) cudaGraphDestroy(g); return rc; }
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
                e = cudaGraphInstantiate(&chunk_graph, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
            }
            const int64_t n = std::min(reps, left / GRAPH_SWEEPS);
            for (int64_t r = 0; r < n; ++r) {
                cudaError_t e = cudaGraphLaunch(chunk_graph, stream());
                if (e != cudaSuccess) { cudaGraphExecDestroy(chunk_graph); return cuda_fail(e, "cudaGraphLaunch"); }
            }
            done_sweeps += n * GRAPH_SWEEPS;
            reps = std::min<int64_t>(reps * 2, 32);
        }
        cudaError_t e = cudaMemcpyAsync(hs.data(), d_st, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
        if (e != cudaSuccess) {
            if (chunk_graph) cudaGraphExecDestroy(chunk_graph);
            return cuda_fail(e, "relax state");
        }
        bool all = true;
        for (uint32_t k = 0; k < nh; ++k) all = all && hs[k].done;
        if (all) break;
    }
    if (chunk_graph) cudaGraphExecDestroy(chunk_graph);
    pc[0].release(); pc[1].release(); ps.release(); prow.release();
    return CW_OK;
}

// ------------------------------------------------------------------ residual by TMA tiles
//
// k_residual64 with its reads staged by the TMA engine.  Persistent blocks,
// two per SM (34 warps an SM: twice the consumers to hide the FP64 chains
// behind; measured 1.7% faster a campaign step than one block of five
// stages), walk 128 x 16 tiles with a producer warp and 16 consumer warps:
// the producer looks up the block's next tiles 32 at a time (a lane per
// candidate: its record, then whether its history has settled), and for each
// live one waits for a free stage and has the TMA engine bring in the tile's
// values (with a ring of neighbours: x from x0 - 2, so that the box starts on
// 16 bytes), held mask and per-pixel coefficients, with the tile's scalars
// beside them.  A consumer warp takes one row of the tile, four pixels a
// lane, folds its maximum into the history's with one atomic and frees the
// stage.  No block-wide barrier after the start, and no global load on a
// consumer's path but its outputs.  Per pixel the arithmetic is
// k_residual64's, in the same order: the same bits.  Used for flat histories
// whose width is a multiple of 16 (the held mask's rows must start on 16
// bytes), the campaign's case.

constexpr int RT_X = 128, RT_Y = 16;               // pixels of a tile
constexpr int RT_CX = RT_X + 4, RT_CY = RT_Y + 2;  // its values' box: x0 - 2 .. x0 + 129, y0 - 1 .. y0 + 16
constexpr int RT_CONSUMERS = RT_Y;                 // a warp per row of a tile
constexpr int RT_THREADS = 32 * (RT_CONSUMERS + 1);
constexpr int RT_MAX_STAGES = 6;
constexpr int RT_MAPS = 5;                         // per history: values, held, sink, production, uptake
constexpr int RT_SMEM = 100 * 1024;                // two blocks per SM: the stages of a block fit in this

__device__ int g_rt_wait_failed;

// A tile as the host lays it out: its history, corner and the history's
// shape and first pixel.
struct RtTile {
    int h, x0, y0, w, ht, pad;
    long long off;
};

// What a stage holds besides the boxes: the tile, or h < 0 for no more tiles.
struct RtStaged {
    RtTile t;
    double omega;
};

struct RtArgs {
    const CUtensorMap *maps;  // RT_MAPS per history
    const RtTile *tiles;
    int ntiles;
    int stages;               // tiles in flight per block
    int stage;                // bytes of one stage
    int o_held, o_ks, o_pr, o_up;  // offsets in a stage, -1 for an absent array
    uint32_t tx;              // bytes one stage receives
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(RT_THREADS, 2)
    k_residual64_tiles(RtArgs a, FieldView fv, RelaxState *st, float *r32, float *inv32, float *dz, int skip_done) {
    extern __shared__ __align__(128) unsigned char rsm[];
    __shared__ __align__(8) uint64_t full[RT_MAX_STAGES], empty[RT_MAX_STAGES];
    __shared__ RtStaged s_tile[RT_MAX_STAGES];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int k = 0; k < a.stages; ++k) {
            mbar_init(sh_addr(&full[k]), 1);
            mbar_init(sh_addr(&empty[k]), RT_CONSUMERS);
        }
        mbar_init_fence();
    }
    __syncthreads();
    if (warp == RT_CONSUMERS) {
        // ---- producer
        int it = 0;
        bool stop = false;
        for (int base = blockIdx.x; !stop; base += 32 * gridDim.x) {
            const int t = base + lane * gridDim.x;
            RtStaged c;
            c.t = RtTile{-1, 0, 0, 0, 0, 0, 0};
            c.omega = 0.0;
            if (t < a.ntiles) {
                c.t = a.tiles[t];
                if (skip_done && st[c.t.h].done) c.t.h = -1;
                else c.omega = st[c.t.h].omega;
            }
            unsigned live = __ballot_sync(0xffffffffu, c.t.h >= 0);
            const bool last = __shfl_sync(0xffffffffu, t, 31) >= a.ntiles;
            while (live && !stop) {
                const int src = __ffs(live) - 1;
                live &= live - 1;
                RtStaged v;
                v.t.h = __shfl_sync(0xffffffffu, c.t.h, src);
                v.t.x0 = __shfl_sync(0xffffffffu, c.t.x0, src);
                v.t.y0 = __shfl_sync(0xffffffffu, c.t.y0, src);
                v.t.w = __shfl_sync(0xffffffffu, c.t.w, src);
                v.t.ht = __shfl_sync(0xffffffffu, c.t.ht, src);
                v.t.off = __shfl_sync(0xffffffffu, c.t.off, src);
                v.omega = __shfl_sync(0xffffffffu, c.omega, src);
                int ok = 1;
                if (lane == 0) {
                    const int slot = it % a.stages;
                    if (it >= a.stages && !mbar_wait_bounded(sh_addr(&empty[slot]), (uint32_t)((it / a.stages) - 1) & 1u))
                        ok = 0;
                    if (ok) {
                        s_tile[slot] = v;
                        const uint32_t bar = sh_addr(&full[slot]);
                        unsigned char *stage = rsm + (size_t)slot * a.stage;
                        const CUtensorMap *m = a.maps + RT_MAPS * v.t.h;
                        // the consumers' reads of this stage before the copies' writes
                        fence_proxy_async_shared();
                        mbar_expect_tx(bar, a.tx);
                        tma_load_2d(stage, m, bar, v.t.x0 - 2, v.t.y0 - 1);
                        tma_load_2d(stage + a.o_held, m + 1, bar, v.t.x0, v.t.y0);
                        if (a.o_ks >= 0) tma_load_2d(stage + a.o_ks, m + 2, bar, v.t.x0, v.t.y0);
                        if (a.o_pr >= 0) tma_load_2d(stage + a.o_pr, m + 3, bar, v.t.x0, v.t.y0);
                        if (a.o_up >= 0) tma_load_2d(stage + a.o_up, m + 4, bar, v.t.x0, v.t.y0);
                    } else {
                        atomicExch(&g_rt_wait_failed, 1);
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) stop = true;
                ++it;
            }
            if (last && !stop) {
                // no more tiles: the next stage says so
                if (lane == 0) {
                    const int slot = it % a.stages;
                    if (it < a.stages || mbar_wait_bounded(sh_addr(&empty[slot]), (uint32_t)((it / a.stages) - 1) & 1u)) {
                        s_tile[slot].t.h = -1;
                        mbar_arrive(sh_addr(&full[slot]));
                    } else {
                        atomicExch(&g_rt_wait_failed, 1);
                    }
                }
                stop = true;
            }
        }
        return;
    }
    // ---- consumers: warp `warp` takes row `warp` of each tile
    for (int it = 0;; ++it) {
        const int slot = it % a.stages;
        if (!mbar_wait_bounded(sh_addr(&full[slot]), (uint32_t)(it / a.stages) & 1u)) {
            atomicExch(&g_rt_wait_failed, 1);
            break;
        }
        const RtStaged v = s_tile[slot];
        if (v.t.h < 0) break;
        const unsigned char *stage = rsm + (size_t)slot * a.stage;
        const double *sc = (const double *)stage;
        const uint8_t *sheld = stage + a.o_held;
        const double *sks = (const double *)(stage + a.o_ks), *spr = (const double *)(stage + a.o_pr),
                     *sup = (const double *)(stage + a.o_up);
        const double den4 = 4.0 * fv.d + fv.decay;
        const int row = warp, y = v.t.y0 + row;
        double worst = 0.0;
        if (y < v.t.ht) {
            const int64_t rowbase = v.t.off + (int64_t)y * v.t.w;
#pragma unroll
            for (int j = 0; j < RT_X / 32; ++j) {
                const int col = lane + 32 * j, x = v.t.x0 + col, k = row * RT_X + col;
                if (x >= v.t.w) continue;
                const int64_t i = rowbase + x;
                float r_out = 0.0f, inv_out = 0.0f;
                if (!sheld[k]) {
                    // pixel_sums64's order onto zero: x-1, x+1, y-1, y+1; a
                    // pixel with all four neighbours real has real = 4, and
                    // real d + decay is then one number
                    const double *p = sc + (row + 1) * RT_CX + (col + 2);
                    double sum, den;
                    if (x > 0 && x + 1 < v.t.w && y > 0 && y + 1 < v.t.ht) {
                        sum = 0.0 + p[-1];
                        sum = sum + p[1];
                        sum = sum + p[-RT_CX];
                        sum = sum + p[RT_CX];
                        den = den4;
                    } else {
                        double real = 0.0;
                        sum = 0.0;
                        if (x > 0) { sum += p[-1]; real += 1.0; }
                        if (x + 1 < v.t.w) { sum += p[1]; real += 1.0; }
                        if (y > 0) { sum += p[-RT_CX]; real += 1.0; }
                        if (y + 1 < v.t.ht) { sum += p[RT_CX]; real += 1.0; }
                        den = real * fv.d + fv.decay;
                    }
                    if (a.o_ks >= 0) den = den + sks[k];
                    const double cv = p[0];
                    // add_sources' order
                    double t = fv.d * sum + fv.source;
                    if (a.o_pr >= 0) t = t + spr[k];
                    if (a.o_up >= 0) t = t - sup[k];
                    double r = t - den * cv;
                    if (fv.floor && cv <= 0.0 && r < 0.0) r = 0.0;
                    worst = fmax(worst, fabs(r));
                    dc_coefficients(v.omega, den, r, fv.d, r_out, inv_out);
                }
                if (r32) r32[i] = r_out;
                if (inv32) inv32[i] = inv_out;
                if (dz) dz[i] = 0.0f;
            }
        }
        worst = warp_max(worst);
        __syncwarp();
        if (lane == 0) {
            if (worst > 0.0) atomic_max_nonneg(&st[v.t.h].resid, worst);
            mbar_arrive(sh_addr(&empty[slot]));
        }
    }
}

// The tensor maps and tiles of k_residual64_tiles for a field, built where
// every history allows it, with the arrays they were built on.
struct ResTiles {
    bool ok = false;
    CUtensorMap *maps = nullptr;
    RtTile *tiles = nullptr;
    RtArgs args{};
    int grid = 0, smem = 0;
    const void *built_on[RT_MAPS] = {};

    void release() {
        dfree(maps);
        dfree(tiles);
        ok = false;
    }
};

static bool rt_matches(const ResTiles &rt, const FieldView &fv) {
    const void *now[RT_MAPS] = {fv.c, fv.held, fv.ks, fv.pr, fv.up};
    for (int m = 0; m < RT_MAPS; ++m)
        if (now[m] != rt.built_on[m]) return false;
    return rt.ok;
}

static int rt_prepare(cw_field_s *f, ResTiles &rt) {
    const FieldView fv = view(f);
    if (rt.ok && rt_matches(rt, fv)) return CW_OK;
    rt.release();
    const Geom &g = f->g;
    for (uint32_t k = 0; k < g.nh; ++k)
        if (g.d[k] != 1 || g.w[k] % 16 != 0 || g.off[k] % 16 != 0) return CW_OK;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return CW_OK;
    // the stage: values, held mask, then each present coefficient array
    RtArgs &a = rt.args;
    int at = ((RT_CX * RT_CY * 8) + 127) / 128 * 128;
    a.o_held = at;
    at += RT_X * RT_Y;
    a.tx = RT_CX * RT_CY * 8 + RT_X * RT_Y;
    const void *arrays[3] = {fv.ks, fv.pr, fv.up};
    int *slots[3] = {&a.o_ks, &a.o_pr, &a.o_up};
    for (int m = 0; m < 3; ++m) {
        *slots[m] = -1;
        if (!arrays[m]) continue;
        *slots[m] = at;
        at += RT_X * RT_Y * 8;
        a.tx += RT_X * RT_Y * 8;
    }
    a.stage = at;
    a.stages = std::min(RT_MAX_STAGES, RT_SMEM / a.stage);
    if (a.stages < 2) return CW_OK;
    rt.smem = a.stages * a.stage;
    std::vector<CUtensorMap> maps((size_t)RT_MAPS * g.nh);
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (uint32_t k = 0; k < g.nh; ++k) {
        for (int m = 0; m < RT_MAPS; ++m) {
            const void *base = m == 0 ? (const void *)fv.c : m == 1 ? (const void *)fv.held : arrays[m - 2];
            if (!base) continue;
            const bool u8 = m == 1;
            const size_t es = u8 ? 1 : 8;
            cuuint64_t dim[2] = {(cuuint64_t)g.w[k], (cuuint64_t)g.h[k]};
            cuuint64_t stride[1] = {(cuuint64_t)g.w[k] * es};
            cuuint32_t box[2] = {m == 0 ? (cuuint32_t)RT_CX : (cuuint32_t)RT_X,
                                 m == 0 ? (cuuint32_t)RT_CY : (cuuint32_t)RT_Y};
            cuuint32_t estride[2] = {1, 1};
            CUresult r = enc(&maps[(size_t)RT_MAPS * k + m],
                             u8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                             (void *)((const char *)base + (size_t)g.off[k] * es), dim, stride, box, estride,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return CW_OK;  // k_residual64 serves
        }
    }
    std::vector<RtTile> tiles;
    for (uint32_t k = 0; k < g.nh; ++k)
        for (int y = 0; y < (int)g.h[k]; y += RT_Y)
            for (int x = 0; x < (int)g.w[k]; x += RT_X)
                tiles.push_back(RtTile{(int)k, x, y, (int)g.w[k], (int)g.h[k], 0, (long long)g.off[k]});
    CW_CUDA(cudaFuncSetAttribute((const void *)k_residual64_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 RT_SMEM));
    int per_sm = 0, dev = 0, nsm = 0;
    CW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_residual64_tiles, RT_THREADS,
                                                          rt.smem));
    if (per_sm < 1) return CW_OK;
    CW_CUDA(cudaGetDevice(&dev));
    CW_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int rc;
    if ((rc = dalloc(&rt.maps, maps.size())) != CW_OK) return rc;
    if ((rc = dalloc(&rt.tiles, tiles.size())) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(rt.maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                            stream()));
    CW_CUDA(cudaMemcpyAsync(rt.tiles, tiles.data(), tiles.size() * sizeof(RtTile), cudaMemcpyHostToDevice,
                            stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    a.maps = rt.maps;
    a.tiles = rt.tiles;
    a.ntiles = (int)tiles.size();
    rt.grid = std::min<int>(a.ntiles, per_sm * nsm);
    const void *on[RT_MAPS] = {fv.c, fv.held, fv.ks, fv.pr, fv.up};
    for (int m = 0; m < RT_MAPS; ++m) rt.built_on[m] = on[m];
    rt.ok = true;
    return CW_OK;
}

static int rt_wait_failed();

// Whether a staged copy of the FP32 sweeps or of the residual timed out.
static int dc_waits_failed() {
    int rc = sor32_wait_failed();
    return rc != CW_OK ? rc : rt_wait_failed();
}

static int rt_wait_failed() {
    int v = 0;
    CW_CUDA(cudaMemcpyFromSymbol(&v, g_rt_wait_failed, sizeof v));
    if (v) {
        const int zero = 0;
        CW_CUDA(cudaMemcpyToSymbol(g_rt_wait_failed, &zero, sizeof zero));
        return fail(CW_ERR_TIMEOUT, "a residual tile's copy did not land in time");
    }
    return CW_OK;
}

// Launch plans and the FP32 solver of the defect-correction solve, built on a
// field's first FP32 solve and kept: no allocation in later solves, so that
// a whole step can be captured in a CUDA graph.
struct DcCache {
    Plan pr, prow;
    Sor32 solver;
    ResTiles rt;
    int depth = -1, window = 0;
    std::vector<double> omega;
    double *d_omega = nullptr;  // per history, for the state initialisation on the device
};

__global__ void k_dc_state_init(RelaxState *st, int nh, const double *omega, double tol, double etol) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    RelaxState s{};
    s.omega = omega[h];
    s.tol = tol;
    s.etol = etol;
    s.stop = CW_STOP_RESIDUAL;
    st[h] = s;
}

static int dc_prepare(cw_field_s *f, int depth, int window, const std::vector<double> &om, DcCache **out) {
    uint32_t nh = f->g.nh;
    int rc = f->alloc_fp32();
    if (rc != CW_OK) return rc;
    DcCache *c = (DcCache *)f->dc_cache;
    if (c && (c->depth != depth || c->window != window)) {
        c->solver.release();
        c->depth = -1;
    }
    if (!c) {
        c = new DcCache();
        f->dc_cache = c;
        if ((rc = row_plan(f, c->prow)) != CW_OK) return rc;
        std::vector<int64_t> per(nh);
        for (uint32_t k = 0; k < nh; ++k) per[k] = (int64_t)f->g.h[k] * f->g.d[k] * ((f->g.w[k] + 511) / 512);
        if ((rc = c->pr.build(per, 1)) != CW_OK) return rc;
        if ((rc = dalloc(&c->d_omega, nh)) != CW_OK) return rc;
    }
    if (c->depth < 0) {
        if ((rc = c->solver.init(f, depth, om, window)) != CW_OK) return rc;
        c->depth = depth;
        c->window = window;
        c->omega.clear();
    }
    if ((rc = rt_prepare(f, c->rt)) != CW_OK) return rc;
    if (c->omega != om) {
        std::vector<float> omf(om.begin(), om.end());
        CW_CUDA(cudaMemcpyAsync(c->solver.omega, omf.data(), sizeof(float) * nh, cudaMemcpyHostToDevice, stream()));
        CW_CUDA(cudaMemcpyAsync(c->d_omega, om.data(), sizeof(double) * nh, cudaMemcpyHostToDevice, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        c->omega = om;
    }
    *out = c;
    return CW_OK;
}

// The defect-correction solve's residual: by TMA tiles where they were built
// on the field's current arrays, else k_residual64.
static void dc_residual(DcCache *c, const FieldView &fv, uint32_t nh, RelaxState *d_st, float *r32, float *inv32,
                        float *dz) {
    if (rt_matches(c->rt, fv))
        k_residual64_tiles<<<c->rt.grid, RT_THREADS, c->rt.smem, stream()>>>(c->rt.args, fv, d_st, r32, inv32, dz, 1);
    else
        k_residual64<<<c->prow.nblocks, T, 0, stream()>>>(fv, c->prow.d_blk, (int)nh, d_st, r32, inv32, dz, 1);
}

// One outer iteration: the convergence test, `inner` FP32 sweeps, the fused
// correction and residual.  No host synchronisation.
static int dc_outer(cw_field_s *f, DcCache *c, RelaxState *d_st, int inner, int64_t max_sweeps, float *&start) {
    uint32_t nh = f->g.nh;
    FieldView fv = view(f);
    const int32_t *done_ptr = (const int32_t *)((const char *)d_st + offsetof(RelaxState, done));
    const int stride = (int)(sizeof(RelaxState) / sizeof(int32_t));
    k_dc_check<<<(nh + 63) / 64, 64, 0, stream()>>>(d_st, nh, inner, max_sweeps, c->solver.wide ? 1 : 0);
    CW_LAUNCHED();
    if (c->solver.vol) {
        // volumes: the last sweep launch adds the correction to c, then the
        // residual at the corrected field in one pass
        int rc = c->solver.sweeps(f, inner, done_ptr, stride, start, true);
        if (rc != CW_OK) return rc;
        dc_residual(c, fv, nh, d_st, f->r32, nullptr, nullptr);
        CW_LAUNCHED();
        return CW_OK;
    }
    if (c->solver.wide) {
        // the last sweep launch adds the correction to c, recording its
        // largest size and the largest |c| for the error estimate; then the
        // residual at the corrected field, in one pass (the correction buffer
        // needs no zeroing: the next solve's first launch does not read it)
        unsigned long long *corr = (unsigned long long *)((char *)d_st + offsetof(RelaxState, corr));
        int rc = c->solver.sweeps(f, inner, done_ptr, stride, start, true, corr,
                                  (int)(sizeof(RelaxState) / sizeof(unsigned long long)));
        if (rc != CW_OK) return rc;
        dc_residual(c, fv, nh, d_st, f->r32, nullptr, nullptr);
        CW_LAUNCHED();
        return CW_OK;
    }
    int rc = c->solver.sweeps(f, inner, done_ptr, stride, start);
    if (rc != CW_OK) return rc;
    float *d = c->solver.result();
    for (int colour = 0; colour < 2; ++colour) {
        k_dc_update<<<c->pr.nblocks, 256, 0, stream()>>>(fv, c->pr.d_blk, nh, d_st, d, f->r32, colour);
        CW_LAUNCHED();
    }
    start = d;  // zeroed behind the update
    return CW_OK;
}

static int relax_fp32dc(cw_field_s *f, const cw_relax_opts &o, RelaxState *d_st, std::vector<RelaxState> &hs) {
    uint32_t nh = f->g.nh;
    int inner = o.inner_sweeps > 0 ? o.inner_sweeps : 16;
    int depth = o.block_depth > 0 ? o.block_depth : 4;
    std::vector<double> om(nh);
    for (uint32_t k = 0; k < nh; ++k) om[k] = hs[k].omega;
    DcCache *c = nullptr;
    int rc = dc_prepare(f, depth, o.window, om, &c);
    if (rc != CW_OK) return rc;
    FieldView fv = view(f);
    int64_t outer = 0;
    int64_t max_outer = o.max_sweeps / inner + 2;
    int queue = 2;
    // the first residual also sets the inverse diagonal and zeroes d32a
    dc_residual(c, fv, nh, d_st, f->r32, f->inv32, f->d32a);
    CW_LAUNCHED();
    float *start = f->d32a;
    while (outer < max_outer) {
        for (int q = 0; q < queue && outer < max_outer; ++q, ++outer)
            if ((rc = dc_outer(f, c, d_st, inner, o.max_sweeps, start)) != CW_OK) return rc;
        CW_CUDA(cudaMemcpyAsync(hs.data(), d_st, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        if ((rc = dc_waits_failed()) != CW_OK) return rc;
        bool all = true;
        for (uint32_t k = 0; k < nh; ++k) all = all && hs[k].done;
        if (all) break;
        queue = std::min(queue * 2, 16);
    }
    return CW_OK;
}

namespace cw {
// Build (or update) a field's FP32 plans for `depth` and its factors per history.
int field_dc_prepare(cw_field_s *f, int depth, int window, const std::vector<double> &omega) {
    DcCache *c = nullptr;
    return dc_prepare(f, depth, window, omega, &c);
}

// The defect-correction solve enqueued with a fixed number of outer
// iterations and no host synchronisation (every kernel skips a history once
// it has settled), for capture in a CUDA graph.  A previous field_relax with
// the same options must have built the field's plans; omega is unchanged.
int field_relax_enqueue(cw_field_s *f, const cw_relax_opts *opts, int outer, float **start_out) {
    DcCache *c = (DcCache *)f->dc_cache;
    if (!c || c->depth < 0) return fail(CW_ERR_CONFIG, "the field has not been solved in FP32 yet");
    uint32_t nh = f->g.nh;
    RelaxState *d_st = (RelaxState *)f->stats;
    int inner = opts->inner_sweeps > 0 ? opts->inner_sweeps : 16;
    k_dc_state_init<<<(nh + 63) / 64, 64, 0, stream()>>>(d_st, nh, c->d_omega, opts->tolerance,
                                                         opts->error_tolerance);
    CW_LAUNCHED();
    FieldView fv = view(f);
    dc_residual(c, fv, nh, d_st, f->r32, f->inv32, f->d32a);
    CW_LAUNCHED();
    float *start = f->d32a;
    for (int q = 0; q < outer; ++q) {
        int rc = dc_outer(f, c, d_st, inner, opts->max_sweeps, start);
        if (rc != CW_OK) return rc;
    }
    // a last test marks what settled
    k_dc_peek<<<(nh + 63) / 64, 64, 0, stream()>>>(d_st, nh, c->solver.wide ? 1 : 0);
    CW_LAUNCHED();
    if (start_out) *start_out = start;
    return CW_OK;
}

// Carry an enqueued solve on, host-driven, until every history has settled
// (or max_sweeps is spent): for the rare step that needs more outer
// iterations than a captured graph holds.  `start` is the zeroed correction
// buffer the enqueued solve ended on.
int field_relax_finish(cw_field_s *f, const cw_relax_opts *opts, float *start) {
    DcCache *c = (DcCache *)f->dc_cache;
    uint32_t nh = f->g.nh;
    RelaxState *d_st = (RelaxState *)f->stats;
    int inner = opts->inner_sweeps > 0 ? opts->inner_sweeps : 16;
    std::vector<RelaxState> hs(nh);
    for (int64_t outer = 0; outer < opts->max_sweeps / inner + 2; ++outer) {
        CW_CUDA(cudaMemcpyAsync(hs.data(), d_st, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        bool all = true;
        for (uint32_t k = 0; k < nh; ++k) all = all && hs[k].done;
        if (all) return CW_OK;
        int rc = dc_outer(f, c, d_st, inner, opts->max_sweeps, start);
        if (rc != CW_OK) return rc;
        k_dc_peek<<<(nh + 63) / 64, 64, 0, stream()>>>(d_st, nh, c->solver.wide ? 1 : 0);
        CW_LAUNCHED();
    }
    return CW_OK;
}

// The state an enqueued solve left: per history sweeps, residual, settled.
int field_relax_collect(cw_field_s *f, std::vector<cw_relax_stats> &out, bool &all_settled) {
    uint32_t nh = f->g.nh;
    std::vector<RelaxState> hs(nh);
    CW_CUDA(cudaMemcpyAsync(hs.data(), f->stats, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    int rc = dc_waits_failed();
    if (rc != CW_OK) return rc;
    out.resize(nh);
    all_settled = true;
    for (uint32_t k = 0; k < nh; ++k) {
        out[k].sweeps = hs[k].sweeps;
        out[k].last_change = 0.0;
        out[k].residual = hs[k].last_resid;
        out[k].status = hs[k].done == 1 ? CW_OK : CW_ERR_SIMULATION;
        out[k].omega = hs[k].omega;
        all_settled = all_settled && hs[k].done == 1;
    }
    return CW_OK;
}
}  // namespace cw

extern "C" {

int cw_field_create(uint32_t nh, const uint32_t *w, const uint32_t *h, const uint32_t *d, double dcoef,
                    double decay, double initial, cw_field *out) {
    *out = nullptr;
    if (!std::isfinite(dcoef) || !std::isfinite(decay) || dcoef < 0.0 || decay < 0.0)
        return fail(CW_ERR_CONFIG, "diffusion and decay must be finite and not negative, got D = " +
                                       std::to_string(dcoef) + ", decay = " + std::to_string(decay));
    cw_field_s *f = new cw_field_s();
    if (f->hs.init() != CW_OK) { delete f; return CW_ERR_CUDA; }
    CW_SCOPE(f);
    int rc = f->g.init(nh, w, h, d);
    if (rc != CW_OK) { delete f; return rc; }
    f->dcoef = dcoef; f->decay = decay;
    int64_t n = f->g.total;
    if ((rc = dalloc(&f->c, n)) || (rc = dalloc(&f->held, n)) || (rc = dalloc(&f->uptake, n)) ||
        (rc = dalloc(&f->production, n)) || (rc = dalloc(&f->lin_sink, n)) || (rc = dalloc(&f->d_span, nh)) ||
        (rc = dalloc((RelaxState **)&f->stats, nh))) {
        cw_field_destroy(f);
        return rc;
    }
    k_fill64<<<(unsigned)blocks_for(n), T, 0, stream()>>>(f->c, n, initial);
    CW_LAUNCHED();
    CW_CUDA(cudaMemsetAsync(f->held, 0, n, stream()));
    CW_CUDA(cudaMemsetAsync(f->uptake, 0, n * sizeof(double), stream()));
    CW_CUDA(cudaMemsetAsync(f->production, 0, n * sizeof(double), stream()));
    CW_CUDA(cudaMemsetAsync(f->lin_sink, 0, n * sizeof(double), stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    *out = f;
    return CW_OK;
}

int cw_field_destroy(cw_field f) {
    if (!f) return CW_OK;
    CW_SCOPE(f);
    dfree(f->c); dfree(f->held); dfree(f->uptake); dfree(f->production); dfree(f->lin_sink);
    dfree(f->r32); dfree(f->d32a); dfree(f->d32b); dfree(f->inv32); dfree(f->tmp64); dfree(f->d_span);
    if (f->dc_cache) {
        DcCache *c = (DcCache *)f->dc_cache;
        c->solver.release();
        c->pr.release();
        c->prow.release();
        c->rt.release();
        dfree(c->d_omega);
        delete c;
    }
    RelaxState *st = (RelaxState *)f->stats;
    dfree(st);
    if (f->adjoint) cw_field_destroy(f->adjoint);
    f->inflow_plan.release();
    f->g.release();
    f->hs.release();
    delete f;
    return CW_OK;
}

int cw_field_set_stream(cw_field f, void *stream) {
    CW_SCOPE(f);
    return f->hs.set((cudaStream_t)stream);
}

void *cw_field_get_stream(cw_field f) { return (void *)f->hs.stream; }

const char *cw_field_last_error(cw_field f) { return f->hs.err.c_str(); }

int cw_field_set_source(cw_field f, double source) {
    CW_SCOPE(f);
    f->source = source;
    return CW_OK;
}

int cw_field_set_floor(cw_field f, int32_t on) {
    CW_SCOPE(f);
    f->floor = on != 0;
    return CW_OK;
}

int cw_field_set_diffusion(cw_field f, double dcoef) {
    CW_SCOPE(f);
    if (!std::isfinite(dcoef) || dcoef < 0.0) return fail(CW_ERR_CONFIG, "diffusion must be finite and not negative");
    f->dcoef = dcoef;
    return CW_OK;
}

static double *array_of(cw_field f, int32_t which) {
    switch (which) {
    case CW_VALUES: return f->c;
    case CW_UPTAKE: return f->uptake;
    case CW_PRODUCTION: return f->production;
    case CW_LIN_SINK: return f->lin_sink;
    default: return nullptr;
    }
}

int cw_field_upload(cw_field f, uint32_t hist, int32_t which, const double *host) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    double *p = array_of(f, which);
    if (!p) return fail(CW_ERR_CONFIG, "unknown field array");
    if (which == CW_LIN_SINK) f->lin_sink_on = true;
    if (which == CW_UPTAKE) f->uptake_on = true;
    if (which == CW_PRODUCTION) f->production_on = true;
    CW_CUDA(cudaMemcpyAsync(p + f->g.off[hist], host, sizeof(double) * f->g.sites(hist), cudaMemcpyHostToDevice,
                            stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_field_download(cw_field f, uint32_t hist, int32_t which, double *host) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    double *p = array_of(f, which);
    if (!p) return fail(CW_ERR_CONFIG, "unknown field array");
    CW_CUDA(cudaMemcpyAsync(host, p + f->g.off[hist], sizeof(double) * f->g.sites(hist), cudaMemcpyDeviceToHost,
                            stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_field_upload_held(cw_field f, uint32_t hist, const uint8_t *held) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    f->held_dirty = true;
    CW_CUDA(cudaMemcpyAsync(f->held + f->g.off[hist], held, f->g.sites(hist), cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_field_download_held(cw_field f, uint32_t hist, uint8_t *held) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    CW_CUDA(cudaMemcpyAsync(held, f->held + f->g.off[hist], f->g.sites(hist), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

int cw_field_fill(cw_field f, double value) {
    CW_SCOPE(f);
    int64_t n = f->g.total;
    k_fill64<<<(unsigned)blocks_for(n), T, 0, stream()>>>(f->c, n, value);
    CW_LAUNCHED();
    return CW_OK;
}

int cw_field_clear(cw_field f, int32_t which) {
    CW_SCOPE(f);
    double *p = array_of(f, which);
    if (!p || which == CW_VALUES) return fail(CW_ERR_CONFIG, "only uptake, production and the linear sink clear");
    CW_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * f->g.total, stream()));
    if (which == CW_UPTAKE) f->uptake_on = false;
    if (which == CW_PRODUCTION) f->production_on = false;
    if (which == CW_LIN_SINK) f->lin_sink_on = false;
    return CW_OK;
}

int cw_field_release_all(cw_field f) {
    CW_SCOPE(f);
    f->held_dirty = true;
    CW_CUDA(cudaMemsetAsync(f->held, 0, f->g.total, stream()));
    return CW_OK;
}

int cw_field_hold_mask(cw_field f, uint32_t hist, const uint8_t *mask, double value) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int64_t n = f->g.sites(hist);
    uint8_t *dm;
    int rc = dalloc(&dm, n);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, stream()));
    f->held_dirty = true;
    k_hold_mask<<<(unsigned)blocks_for(n), T, 0, stream()>>>(f->c + f->g.off[hist], f->held + f->g.off[hist], dm, n,
                                                             value);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(dm);
    return CW_OK;
}

int cw_field_relax(cw_field f, const cw_relax_opts *opts, cw_relax_stats *stats) {
    CW_SCOPE(f);
    return cw::field_relax(f, opts, nullptr, stats);
}

// The operator restricted to the free pixels is symmetric (den_i on the
// diagonal, -D between neighbours), so its adjoint solve is the same solver
// on a twin with dl_dc as the source, zero on the held pixels and no floor.
int cw_field_relax_adjoint(cw_field f, const double *dl_dc, double *lambda, const cw_relax_opts *opts,
                           cw_relax_stats *stats) {
    CW_SCOPE(f);
    int rc;
    cw_field_s *a = f->adjoint;
    const int64_t n = f->g.total;
    if (!a) {
        std::vector<uint32_t> W(f->g.w.begin(), f->g.w.end()), H(f->g.h.begin(), f->g.h.end()),
            D(f->g.d.begin(), f->g.d.end());
        if ((rc = cw_field_create(f->g.nh, W.data(), H.data(), D.data(), f->dcoef, f->decay, 0.0, &a)) != CW_OK)
            return rc;
        f->adjoint = a;
    }
    a->dcoef = f->dcoef;
    a->decay = f->decay;
    a->source = 0.0;
    a->floor = false;
    CW_CUDA(cudaMemcpyAsync(a->held, f->held, (size_t)n, cudaMemcpyDeviceToDevice, stream()));
    a->held_dirty = true;
    CW_CUDA(cudaMemsetAsync(a->c, 0, sizeof(double) * n, stream()));
    a->lin_sink_on = f->lin_sink_on;
    if (f->lin_sink_on)
        CW_CUDA(cudaMemcpyAsync(a->lin_sink, f->lin_sink, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream()));
    a->uptake_on = false;
    a->production_on = true;
    CW_CUDA(cudaMemcpyAsync(a->production, dl_dc, sizeof(double) * n, cudaMemcpyHostToDevice, stream()));
    rc = cw::field_relax(a, opts, nullptr, stats);
    if (rc != CW_OK && rc != CW_ERR_SIMULATION) return rc;
    CW_CUDA(cudaMemcpyAsync(lambda, a->c, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return rc;
}

}  // extern "C"

// relax on every history; omega_h (nh entries, may be null) overrides the
// options' factor history by history.
int cw::field_relax(cw_field_s *f, const cw_relax_opts *opts, const double *omega_h, cw_relax_stats *stats) {
    cw_relax_opts o = *opts;
    if (o.max_sweeps <= 0) o.max_sweeps = 1;
    if (o.precision != CW_FP64 && o.precision != CW_FP32_DC) return fail(CW_ERR_CONFIG, "unknown precision");
    if (o.precision == CW_FP32_DC && o.stop != CW_STOP_RESIDUAL)
        return fail(CW_ERR_CONFIG, "the FP32 defect-correction solve stops on the residual only");
    if (!(o.tolerance > 0.0 && o.tolerance < INFINITY))
        return fail(CW_ERR_CONFIG, "the tolerance must be finite and above zero, got " + std::to_string(o.tolerance));
    if (!(o.error_tolerance >= 0.0 && o.error_tolerance < INFINITY))
        return fail(CW_ERR_CONFIG, "the error tolerance must be finite and not negative, got " +
                                       std::to_string(o.error_tolerance));
    if (!(o.omega < 2.0))
        return fail(CW_ERR_CONFIG, "the relaxation factor must lie in (0, 2) (or be <= 0 for the rule), got " +
                                       std::to_string(o.omega));
    uint32_t nh = f->g.nh;
    if (omega_h)
        for (uint32_t k = 0; k < nh; ++k)
            if (!(omega_h[k] < 2.0))
                return fail(CW_ERR_CONFIG, "a history's relaxation factor must lie below 2, got " +
                                               std::to_string(omega_h[k]));
    int rc;
    if (f->held_dirty || f->spans.size() != nh) {
        if ((rc = field_span(f, f->spans)) != CW_OK) return rc;
        f->held_dirty = false;
    }
    std::vector<Span> &spans = f->spans;
    std::vector<RelaxState> hs(nh);
    for (uint32_t k = 0; k < nh; ++k) {
        RelaxState &s = hs[k];
        std::memset(&s, 0, sizeof s);
        s.tol = o.tolerance;
        s.etol = o.error_tolerance;
        s.stop = o.stop;
        if (!spans[k].found) {  // nothing to balance: one sweep that moves nothing (pde.rs:256-259)
            s.done = 1;
            s.sweeps = 1;
            s.omega = 0.0;
            continue;
        }
        s.omega = (omega_h && omega_h[k] > 0.0) ? omega_h[k] : o.omega > 0.0 ? o.omega : auto_omega(f, k, spans[k]);
    }
    RelaxState *d_st = (RelaxState *)f->stats;
    CW_CUDA(cudaMemcpyAsync(d_st, hs.data(), sizeof(RelaxState) * nh, cudaMemcpyHostToDevice, stream()));
    if (o.precision == CW_FP64) rc = relax_fp64(f, o, spans, d_st, hs);
    else rc = relax_fp32dc(f, o, d_st, hs);
    if (rc != CW_OK) return rc;
    // final residual of every history, for the report (the defect-correction
    // loop ends on one it has just computed)
    std::vector<double> res(nh);
    if (o.precision == CW_FP32_DC) {
        for (uint32_t k = 0; k < nh; ++k) res[k] = hs[k].last_resid;
    } else if ((rc = cw_field_residual(f, res.data())) != CW_OK) {
        return rc;
    }
    bool bad = false;
    for (uint32_t k = 0; k < nh; ++k) {
        bool ok = hs[k].done == 1;
        bad = bad || !ok;
        if (stats) {
            stats[k].sweeps = hs[k].sweeps;
            stats[k].last_change = hs[k].last_change;
            stats[k].residual = res[k];
            stats[k].status = ok ? CW_OK : CW_ERR_SIMULATION;
            stats[k].omega = hs[k].omega;
        }
    }
    if (bad)
        return fail(CW_ERR_SIMULATION, "diffusion did not settle within " + std::to_string(o.max_sweeps) +
                                           " sweeps at tolerance " + std::to_string(o.tolerance));
    return CW_OK;
}

namespace cw {
int field_inflow_enqueue(cw_field_s *f, double *inflow, unsigned long long *free_count) {
    Plan &ps = f->inflow_plan;
    int rc;
    if (ps.nblocks == 0 && (rc = site_plan(f, ps)) != CW_OK) return rc;
    k_inflow<<<ps.nblocks, T, 0, stream()>>>(view(f), ps.d_blk, (int)f->g.nh, inflow, free_count);
    CW_LAUNCHED();
    return CW_OK;
}
}  // namespace cw

extern "C" {

int cw_field_residual(cw_field f, double *out) {
    CW_SCOPE(f);
    uint32_t nh = f->g.nh;
    RelaxState *d_st = (RelaxState *)f->stats;
    std::vector<RelaxState> hs(nh);
    CW_CUDA(cudaMemcpyAsync(hs.data(), d_st, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (auto &s : hs) { s.resid = 0ull; s.done = 0; }
    CW_CUDA(cudaMemcpyAsync(d_st, hs.data(), sizeof(RelaxState) * nh, cudaMemcpyHostToDevice, stream()));
    Plan prow;
    int rc = row_plan(f, prow);
    if (rc != CW_OK) return rc;
    k_residual64<<<prow.nblocks, T, 0, stream()>>>(view(f), prow.d_blk, nh, d_st, nullptr, nullptr, nullptr, 0);
    CW_LAUNCHED();
    CW_CUDA(cudaMemcpyAsync(hs.data(), d_st, sizeof(RelaxState) * nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (uint32_t k = 0; k < nh; ++k) out[k] = __builtin_bit_cast(double, (uint64_t)hs[k].resid);
    prow.release();
    return CW_OK;
}

int cw_field_inflow(cw_field f, double *out) {
    CW_SCOPE(f);
    uint32_t nh = f->g.nh;
    double *d_out;
    int rc = dalloc(&d_out, nh);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * nh, stream()));
    Plan ps;
    if ((rc = site_plan(f, ps)) != CW_OK) return rc;
    k_inflow<<<ps.nblocks, T, 0, stream()>>>(view(f), ps.d_blk, nh, d_out);
    CW_LAUNCHED();
    CW_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_out);
    ps.release();
    return CW_OK;
}

int cw_field_step(cw_field f, double dt) {
    CW_SCOPE(f);
    if (std::isnan(dt) || dt <= 0.0) return fail(CW_ERR_CONFIG, "time step must be positive, got " + std::to_string(dt));
    bool volume = false;
    for (uint32_t k = 0; k < f->g.nh; ++k) volume = volume || f->g.d[k] > 1;
    double limit = volume ? 0.25 * 2.0 / 3.0 : 0.25;
    if (f->dcoef * dt > limit)
        return fail(CW_ERR_CONFIG, "unstable time step: D*dt = " + std::to_string(f->dcoef * dt) + " is above " +
                                       std::to_string(limit));
    if (f->decay * dt > 1.0)
        return fail(CW_ERR_CONFIG, "unstable time step: decay*dt = " + std::to_string(f->decay * dt) + " is above 1");
    int rc;
    if (!f->tmp64 && (rc = dalloc(&f->tmp64, f->g.total)) != CW_OK) return rc;
    Plan ps;
    if ((rc = site_plan(f, ps)) != CW_OK) return rc;
    k_explicit<<<ps.nblocks, T, 0, stream()>>>(view(f), ps.d_blk, f->g.nh, dt, f->tmp64);
    CW_LAUNCHED();
    std::swap(f->c, f->tmp64);
    CW_CUDA(cudaStreamSynchronize(stream()));
    ps.release();
    return CW_OK;
}

}  // extern "C"

namespace cw {
// The bath flood of one history (or all, hist < 0) from an open mask on the device.
int field_hold_bath_device(cw_field_s *f, const uint8_t *d_open, int hist, double value) {
    Plan ps;
    int rc = site_plan(f, ps);
    if (rc != CW_OK) return rc;
    uint32_t nh = f->g.nh;
    f->held_dirty = true;  // the span buffer is the box's scratch, and holds change
    Span *box = f->d_span;
    k_span_reset<<<(nh + 63) / 64, 64, 0, stream()>>>(box, nh);
    CW_LAUNCHED();
    k_bath_box<<<ps.nblocks, T, 0, stream()>>>(d_open, f->g.d_dims, f->g.d_off, ps.d_blk, nh, box);
    CW_LAUNCHED();
    k_bath_init<<<ps.nblocks, T, 0, stream()>>>(d_open, f->held, f->g.d_dims, f->g.d_off, ps.d_blk, nh, box, hist);
    CW_LAUNCHED();
    int *d_changed;
    if ((rc = dalloc(&d_changed, 1)) != CW_OK) return rc;
    int64_t limit = f->g.total + 2;
    int64_t iters = 0;
    for (;;) {
        CW_CUDA(cudaMemsetAsync(d_changed, 0, sizeof(int), stream()));
        for (int r = 0; r < 16; ++r) {
            k_bath_spread<<<ps.nblocks, T, 0, stream()>>>(d_open, f->held, f->g.d_dims, f->g.d_off, ps.d_blk, nh, box,
                                                          hist, d_changed);
            CW_LAUNCHED();
        }
        iters += 16;
        int changed = 0;
        CW_CUDA(cudaMemcpyAsync(&changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        if (!changed) break;
        if (iters > limit) {
            dfree(d_changed);
            return fail(CW_ERR_TIMEOUT, "the bath flood did not finish");
        }
    }
    dfree(d_changed);
    k_bath_values<<<ps.nblocks, T, 0, stream()>>>(f->c, f->held, f->g.d_off, ps.d_blk, nh, hist, value);
    CW_LAUNCHED();
    CW_CUDA(cudaStreamSynchronize(stream()));
    ps.release();
    return CW_OK;
}
}  // namespace cw

extern "C" int cw_field_hold_bath(cw_field f, uint32_t hist, const uint8_t *open, double value) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    uint8_t *d_open;
    int rc = dalloc(&d_open, f->g.total);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_open, 1, f->g.total, stream()));
    CW_CUDA(cudaMemcpyAsync(d_open + f->g.off[hist], open, f->g.sites(hist), cudaMemcpyHostToDevice, stream()));
    rc = field_hold_bath_device(f, d_open, (int)hist, value);
    dfree(d_open);
    return rc;
}

// Measurement hook: `sweeps` FP32 red-black sweeps of the correction
// equation on the field's current residual, every history active, timed
// with events around the sweep launches alone.  The field is not changed.
extern "C" int cw_field_time_inner(cw_field f, int32_t sweeps, int32_t depth, int32_t window, double omega, float *ms,
                                   int64_t *launches) {
    CW_SCOPE(f);
    uint32_t nh = f->g.nh;
    int rc = f->alloc_fp32();
    if (rc != CW_OK) return rc;
    std::vector<RelaxState> hs(nh);
    for (auto &s : hs) { std::memset(&s, 0, sizeof s); s.omega = omega; s.stop = CW_STOP_RESIDUAL; }
    RelaxState *d_st = (RelaxState *)f->stats;
    CW_CUDA(cudaMemcpyAsync(d_st, hs.data(), sizeof(RelaxState) * nh, cudaMemcpyHostToDevice, stream()));
    Plan prow;
    if ((rc = row_plan(f, prow)) != CW_OK) return rc;
    k_residual64<<<prow.nblocks, T, 0, stream()>>>(view(f), prow.d_blk, nh, d_st, f->r32, f->inv32, f->d32a, 0);
    CW_LAUNCHED();
    Sor32 solver;
    std::vector<double> om(nh, omega);
    if ((rc = solver.init(f, depth, om, window)) != CW_OK) return rc;
    const int32_t *done_ptr = (const int32_t *)((const char *)d_st + offsetof(RelaxState, done));
    cudaEvent_t a, b;
    CW_CUDA(cudaEventCreate(&a));
    CW_CUDA(cudaEventCreate(&b));
    uint64_t before = cw_launch_count();
    CW_CUDA(cudaEventRecord(a, stream()));
    if ((rc = solver.sweeps(f, sweeps, done_ptr, (int)(sizeof(RelaxState) / sizeof(int32_t)))) != CW_OK) return rc;
    CW_CUDA(cudaEventRecord(b, stream()));
    CW_CUDA(cudaEventSynchronize(b));
    CW_CUDA(cudaEventElapsedTime(ms, a, b));
    *launches = (int64_t)(cw_launch_count() - before);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    f->last_inner = solver.result();
    solver.release();
    prow.release();
    return dc_waits_failed();
}

extern "C" int cw_field_inner_correction(cw_field f, uint32_t hist, float *out) {
    CW_SCOPE(f);
    if (hist >= f->g.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    if (!f->last_inner) return fail(CW_ERR_CONFIG, "no inner solve has run on this field");
    CW_CUDA(cudaMemcpy(out, f->last_inner + f->g.off[hist], sizeof(float) * f->g.sites(hist), cudaMemcpyDeviceToHost));
    return CW_OK;
}
