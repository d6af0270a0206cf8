// FP32 red-black SOR on the correction equation of the defect-correction
// solve (see field.cu).  Built with fused multiply-add: this is the fast
// path, and its error is removed by the FP64 residual and correction steps.
//
// Temporal blocking.  A flat history is cut into tiles whose interior is
// (64 - 2 DEPTH) pixels square; a block loads the tile with a halo DEPTH
// pixels deep (a 64 x 64 window) and runs DEPTH half-sweeps on it before
// writing the interior back to the other buffer.  Every window pixel is
// updated at every half-sweep, its missing neighbours read as zero; the
// error this makes at the window's edge moves in by one ring per half-sweep,
// so after DEPTH of them the interior is exactly what DEPTH global
// half-sweeps give.  The correction crosses HBM once per DEPTH half-sweeps.
//
// Layout.  Warp w owns window rows 8w .. 8w+7, lane l the column pair
// (2l, 2l+1): one pixel of each colour per row, so every half-sweep gives
// every thread the same work.  The correction, the right-hand side and the
// inverse diagonal of a thread's sixteen pixels stay in registers for the
// whole launch.  Neighbours come from the thread's own registers (the other
// pixel of the pair, the rows above and below), from the next lane by a warp
// shuffle, and across a warp boundary from the one row each neighbouring
// warp publishes in shared memory after every half-sweep (double-buffered,
// so one barrier per half-sweep suffices).
#include "cw_internal.cuh"
#include "field_kernels.cuh"

namespace cw {
namespace {

constexpr int WIN = 64;            // window side
constexpr int WARPS = 8;           // warps per block
constexpr int ROWS = WIN / WARPS;  // window rows per warp

// One half-sweep of colour C over the thread's rows (C known at compile
// time: the colour of each row's pixels is then fixed and no branch is left).
// ab/be: the rows just above and below this warp's, from the neighbours.
template <int C>
__device__ __forceinline__ void half_sweep(float (&d0)[ROWS], float (&d1)[ROWS], const float (&r0)[ROWS],
                                           const float (&r1)[ROWS], const float (&i0)[ROWS],
                                           const float (&i1)[ROWS], float ab0, float ab1, float be0, float be1,
                                           int lane, float om, float dcoef) {
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        if (((C + j) & 1) == 0) {  // the even column of the pair
            float left = __shfl_up_sync(0xffffffffu, d1[j], 1);
            left = lane == 0 ? 0.f : left;
            const float up = j > 0 ? d0[j - 1] : ab0, down = j < ROWS - 1 ? d0[j + 1] : be0;
            const float old = d0[j];
            d0[j] = fmaf(om, fmaf(fmaf(dcoef, (left + d1[j]) + (up + down), r0[j]), i0[j], -old), old);
        } else {  // the odd column
            float right = __shfl_down_sync(0xffffffffu, d0[j], 1);
            right = lane == 31 ? 0.f : right;
            const float up = j > 0 ? d1[j - 1] : ab1, down = j < ROWS - 1 ? d1[j + 1] : be1;
            const float old = d1[j];
            d1[j] = fmaf(om, fmaf(fmaf(dcoef, (d0[j] + right) + (up + down), r1[j]), i1[j], -old), old);
        }
    }
}

template <int DEPTH>
__global__ void __launch_bounds__(32 * WARPS) k_sor32_tb(const float *__restrict__ src, float *__restrict__ dst,
                                                         const float *__restrict__ rhs, const float *__restrict__ inv,
                                                         const int4 *__restrict__ dims,
                                                         const int64_t *__restrict__ off,
                                                         const int32_t *__restrict__ blk, int nh,
                                                         const float *__restrict__ omega, const int32_t *done,
                                                         int done_stride, int nhalf, int start_colour, float dcoef) {
    constexpr int IN = WIN - 2 * DEPTH;  // interior side
    // edge rows each warp publishes, double-buffered by half-sweep parity:
    // [buffer][warp][0 top, 1 bottom][column]
    __shared__ float edge[2][WARPS][2][WIN];
    __shared__ int s_h;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    if (done[(int64_t)h * done_stride]) return;
    const int4 dm = dims[h];
    const int ntx = (dm.x + IN - 1) / IN;
    const int t = blockIdx.x - blk[h];
    const int gx0 = (t % ntx) * IN - DEPTH, gy0 = (t / ntx) * IN - DEPTH;
    const int64_t base = off[h];
    const float om = omega[h];
    const int gx = gx0 + 2 * lane;
    const bool in0 = gx >= 0 && gx < dm.x, in1 = gx + 1 >= 0 && gx + 1 < dm.x;
    float d0[ROWS], d1[ROWS], r0[ROWS], r1[ROWS], i0[ROWS], i1[ROWS];
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int gy = gy0 + ROWS * warp + j;
        d0[j] = d1[j] = r0[j] = r1[j] = i0[j] = i1[j] = 0.f;
        if (gy >= 0 && gy < dm.y) {
            const int64_t row = base + (int64_t)gy * dm.x + gx;
            if (in0) { d0[j] = src[row]; r0[j] = rhs[row]; i0[j] = inv[row]; }
            if (in1) { d1[j] = src[row + 1]; r1[j] = rhs[row + 1]; i1[j] = inv[row + 1]; }
        }
    }
    auto publish = [&](int buf) {
        edge[buf][warp][0][2 * lane] = d0[0];
        edge[buf][warp][0][2 * lane + 1] = d1[0];
        edge[buf][warp][1][2 * lane] = d0[ROWS - 1];
        edge[buf][warp][1][2 * lane + 1] = d1[ROWS - 1];
    };
    publish(0);
    __syncthreads();
    // window pixel (ex, ey) has colour (gx0 + gy0 + ex + ey) mod 2, and gx0 + gy0
    // and 8 warp are even: in row j the pixel of colour c is the pair's (c + j) mod 2
    for (int s = 0; s < nhalf; ++s) {
        const int buf = s & 1;
        const float ab0 = warp > 0 ? edge[buf][warp - 1][1][2 * lane] : 0.f;
        const float ab1 = warp > 0 ? edge[buf][warp - 1][1][2 * lane + 1] : 0.f;
        const float be0 = warp < WARPS - 1 ? edge[buf][warp + 1][0][2 * lane] : 0.f;
        const float be1 = warp < WARPS - 1 ? edge[buf][warp + 1][0][2 * lane + 1] : 0.f;
        if (((start_colour + s) & 1) == 0)
            half_sweep<0>(d0, d1, r0, r1, i0, i1, ab0, ab1, be0, be1, lane, om, dcoef);
        else
            half_sweep<1>(d0, d1, r0, r1, i0, i1, ab0, ab1, be0, be1, lane, om, dcoef);
        // the other buffer was last read before the previous barrier
        publish(buf ^ 1);
        __syncthreads();
    }
    // the interior back to global memory
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int ey = ROWS * warp + j, gy = gy0 + ey;
        if (ey < DEPTH || ey >= DEPTH + IN || gy >= dm.y) continue;
        const int64_t row = base + (int64_t)gy * dm.x + gx;
        const int ex = 2 * lane;
        if (ex >= DEPTH && ex < DEPTH + IN && gx < dm.x) dst[row] = d0[j];
        if (ex + 1 >= DEPTH && ex + 1 < DEPTH + IN && gx + 1 < dm.x) dst[row + 1] = d1[j];
    }
}

// One half-sweep in place, any depth of lattice (volumes).
__global__ void k_sor32_half(float *__restrict__ dlt, const float *__restrict__ rhs, const float *__restrict__ inv,
                             const int4 *__restrict__ dims, const int64_t *__restrict__ off,
                             const int32_t *__restrict__ blk, int nh, const float *__restrict__ omega,
                             const int32_t *done, int done_stride, int colour, float dcoef) {
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    if (done[(int64_t)h * done_stride]) return;
    const int4 dm = dims[h];
    const int hw = (dm.x + 1) >> 1;
    int64_t k = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    int64_t rows = (int64_t)dm.y * dm.z;
    if (k >= rows * hw) return;
    int64_t row = k / hw;
    int y = (int)(row % dm.y), z = (int)(row / dm.y);
    int x = ((colour - y - z) & 1) + 2 * (int)(k - row * hw);
    if (x >= dm.x) return;
    int64_t w = dm.x, slice = (int64_t)dm.x * dm.y;
    int64_t i = off[h] + row * w + x;
    float iv = inv[i];
    if (iv == 0.f) return;
    float sum = 0.f;
    if (x > 0) sum += dlt[i - 1];
    if (x + 1 < dm.x) sum += dlt[i + 1];
    if (y > 0) sum += dlt[i - w];
    if (y + 1 < dm.y) sum += dlt[i + w];
    if (z > 0) sum += dlt[i - slice];
    if (z + 1 < dm.z) sum += dlt[i + slice];
    float old = dlt[i];
    dlt[i] = old + omega[h] * ((rhs[i] + dcoef * sum) * iv - old);
}

typedef void (*TbKernel)(const float *, float *, const float *, const float *, const int4 *, const int64_t *,
                         const int32_t *, int, const float *, const int32_t *, int, int, int, float);

TbKernel tb_kernel(int depth) {
    switch (depth) {
    case 2: return k_sor32_tb<2>;
    case 4: return k_sor32_tb<4>;
    case 6: return k_sor32_tb<6>;
    default: return k_sor32_tb<8>;
    }
}

}  // namespace

int Sor32::init(cw_field_s *f, int d, const std::vector<double> &om) {
    depth = d < 1 ? 1 : d;
    if (depth > 1) depth = depth >= 8 ? 8 : (depth >= 6 ? 6 : (depth >= 4 ? 4 : 2));
    blocked = depth > 1;
    for (uint32_t k = 0; k < f->g.nh; ++k) blocked = blocked && f->g.d[k] == 1;
    std::vector<float> omf(om.begin(), om.end());
    int rc = dalloc(&omega, omf.size());
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(omega, omf.data(), sizeof(float) * omf.size(), cudaMemcpyHostToDevice, stream()));
    std::vector<int64_t> per(f->g.nh);
    if (blocked) {
        const int in = WIN - 2 * depth;
        for (uint32_t k = 0; k < f->g.nh; ++k)
            per[k] = (int64_t)((f->g.w[k] + in - 1) / in) * ((f->g.h[k] + in - 1) / in);
        rc = tiles.build(per, 1);
    } else {
        for (uint32_t k = 0; k < f->g.nh; ++k) per[k] = (int64_t)((f->g.w[k] + 1) / 2) * f->g.h[k] * f->g.d[k];
        rc = sites.build(per, 256);
    }
    ping = f->d32a;
    pong = f->d32b;
    out = ping;
    return rc;
}

int Sor32::sweeps(cw_field_s *f, int n, const int32_t *done, int done_stride, float *start) {
    float dcoef = (float)f->dcoef;
    if (start) {  // begin from this (zeroed) buffer; the other is scratch
        ping = start;
        pong = start == f->d32a ? f->d32b : f->d32a;
    }
    if (!blocked) {
        for (int s = 0; s < n; ++s)
            for (int colour = 0; colour < 2; ++colour) {
                k_sor32_half<<<sites.nblocks, 256, 0, stream()>>>(ping, f->r32, f->inv32, f->g.d_dims, f->g.d_off,
                                                                  sites.d_blk, f->g.nh, omega, done, done_stride,
                                                                  colour, dcoef);
                CW_LAUNCHED();
            }
        out = ping;
        return CW_OK;
    }
    // 2n half-sweeps, `depth` per launch (fewer in the last), starting from
    // the zeroed buffer; the tiles are those of `depth`, whose window halo is
    // deep enough for a shorter last launch too
    TbKernel kern = tb_kernel(depth);
    float *a = ping, *b = pong;
    int remaining = 2 * n, done_half = 0;
    while (remaining > 0) {
        int dd = remaining < depth ? remaining : depth;
        kern<<<tiles.nblocks, 32 * WARPS, 0, stream()>>>(a, b, f->r32, f->inv32, f->g.d_dims, f->g.d_off, tiles.d_blk,
                                                         f->g.nh, omega, done, done_stride, dd, done_half & 1, dcoef);
        CW_LAUNCHED();
        remaining -= dd;
        done_half += dd;
        float *t = a; a = b; b = t;
    }
    out = a;
    return CW_OK;
}

void Sor32::release() {
    dfree(omega);
    tiles.release();
    sites.release();
}

}  // namespace cw
