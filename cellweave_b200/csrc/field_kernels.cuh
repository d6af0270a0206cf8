// Field views and the FP32 inner solver shared by field.cu and field32.cu.
#pragma once

#include "cw_internal.cuh"

namespace cw {

// What a field kernel reads: the values, the held mask, the per-pixel
// coefficients and the scalars of pde.rs:30-53 (ks: first-order sink or null).
struct FieldView {
    double *c;
    const uint8_t *held;
    const double *up, *pr, *ks;
    double d, decay, source;
    const int4 *dims;
    const int64_t *off;
    int floor;  // 1: updates floored at zero, residual projected (the reference); 0: a linear solve
};

FieldView view(cw_field_s *f);
int field_hold_bath_device(cw_field_s *f, const uint8_t *d_open, int hist, double value);

// The source side of a pixel's balance after `t` (d*sum or d*lap - decay*c):
// t + source + production - uptake, added in the reference's order
// (pde.rs:393-394, 717-718); an absent array is an exact zero.
__device__ __forceinline__ double add_sources(const FieldView &fv, int64_t i, double t) {
    t = t + fv.source;
    if (fv.pr) t = t + fv.pr[i];
    if (fv.up) t = t - fv.up[i];
    return t;
}

// Neighbour sum and count of real neighbours in the reference's order:
// x-1, x+1, y-1, y+1, z-1, z+1 (pde.rs:361-390).
__device__ __forceinline__ void pixel_sums64(const double *__restrict__ c, int64_t i, int x, int y, int z, int4 dm,
                                             double &sum, double &real) {
    int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    double s = 0.0, r = 0.0;
    if (x > 0) { s += c[i - 1]; r += 1.0; }
    if (x + 1 < dm.x) { s += c[i + 1]; r += 1.0; }
    if (y > 0) { s += c[i - w]; r += 1.0; }
    if (y + 1 < dm.y) { s += c[i + w]; r += 1.0; }
    if (z > 0) { s += c[i - slice]; r += 1.0; }
    if (z + 1 < dm.z) { s += c[i + slice]; r += 1.0; }
    sum = s;
    real = r;
}

// Red-black SOR sweeps on the correction equation A d = r in FP32.  Flat
// histories are swept `depth` half-sweeps per launch, each tile held on chip
// with a halo `depth` deep (temporal blocking): 128 x 64 windows fed by TMA
// to persistent blocks where every history's rows are 16-byte aligned,
// 64 x 64 windows read by plain loads otherwise; volumes by 64 x 32 (or
// 64 x 16) tiles marched along z, two or four half-sweeps per launch, or at
// depth 1 one half-sweep per launch, in place.
struct Sor32 {
    int depth = 4;
    bool blocked = true;
    bool wide = false;          // the TMA-fed kernel
    bool vol = false;           // volumes: the tiles marched along z
    int4 *vtiles = nullptr;     // vol: (history, x0, y0, z0) per tile, device
    int nvtiles = 0, vy = 32, vz = 32, vdepth = 2;
    Plan tiles;                 // 64 x 64 windows: tiles per history
    Plan sites;                 // volumes: pixels per history
    void *maps = nullptr;       // wide: 4 tensor maps per history (d32a, d32b, r32, inv32), device
    int4 *wtiles = nullptr;     // wide: (history, x0, y0, 0) per window, device
    int nwtiles = 0, wgrid = 0;
    int wwarps = 8;             // wide: warps per block (8: 128 x 64 windows, 16: 128 x 128)
    float *omega = nullptr;
    float *ping = nullptr, *pong = nullptr, *out = nullptr;
    int init(cw_field_s *f, int depth, const std::vector<double> &omega_per_history, int window = CW_WINDOW_AUTO);
    // n sweeps from the zeroed correction buffer `start` (or the last result);
    // `apply` (wide only): the last launch adds the correction to the field's
    // values instead of writing it, and result() is null
    // corr (optional, apply only): per history, with stride corr_stride, the
    // largest |correction| the launch added, as the bits of a non-negative
    // double (atomic max)
    int sweeps(cw_field_s *f, int n, const int32_t *done, int done_stride, float *start = nullptr,
               bool apply = false, unsigned long long *corr = nullptr, int corr_stride = 0);
    float *result() const { return out; }
    void release();
};

// CW_ERR_TIMEOUT if a wide-kernel block gave up waiting for its window since
// the last call (synchronous; clears the record).
int sor32_wait_failed();

}  // namespace cw
