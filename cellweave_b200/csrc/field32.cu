// FP32 red-black SOR on the correction equation A d = r of the
// defect-correction solve (see field.cu).  Built with fused multiply-add:
// this is the fast path, and its error is removed by the FP64 residual and
// correction steps.  The coefficients come with the relaxation factor folded
// in (field.cu writes them): b = omega r / den and a = omega D / den, so one
// update is d' = (1 - omega) d + a (sum of the four neighbours) + b, two
// fused multiply-adds after the neighbour sum.
//
// Temporal blocking.  A flat history is cut into windows; a block takes a
// window and runs DEPTH half-sweeps on it before writing its interior back to
// the other buffer.  Every window pixel is updated at every half-sweep, its
// missing neighbours read as zero; the error this makes at a window edge that
// lies inside the history moves in by one ring per half-sweep, so after DEPTH
// of them every pixel at least DEPTH from such an edge is exactly what DEPTH
// global half-sweeps give.  A window edge on or beyond the history's border
// makes no error (outside pixels are zero there too), so the interior reaches
// that border.  The correction crosses HBM once per DEPTH half-sweeps.
//
// The wide kernel (rows 16-byte aligned in every history, the campaign's
// case): 128 x 64 windows, a warp per 8 rows, a lane per 4 consecutive
// columns held as float4 registers (two pixels of each colour per row, one
// warp shuffle per two updates).  Blocks are persistent, two per SM; while a
// block sweeps one window in registers, the TMA engine brings the next
// window's correction and coefficients into shared memory (one mbarrier,
// 96 KB), so the HBM reads overlap the sweeps.  Windows start at x = k (128 -
// 2 DEPTH), a multiple of 4 floats as TMA needs, and at y = k (64 - 2 DEPTH).
//
// The narrow kernel (any width): 64 x 64 windows, a lane per column pair,
// plain loads, one window per block.
//
// Between warps, each warp publishes its top and bottom rows in shared memory
// after every half-sweep (double-buffered, so one barrier per half-sweep).

#include <mutex>

#include "cw_internal.cuh"
#include "field_kernels.cuh"
#include "tma.cuh"

namespace cw {
namespace {

// ------------------------------------------------------------------ narrow windows

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
                                           float lm, float rm, float omc) {
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        if (((C + j) & 1) == 0) {  // the even column of the pair
            const float left = __shfl_up_sync(0xffffffffu, d1[j], 1);
            const float up = j > 0 ? d0[j - 1] : ab0, down = j < ROWS - 1 ? d0[j + 1] : be0;
            d0[j] = fmaf(i0[j], fmaf(lm, left, d1[j]) + (up + down), fmaf(omc, d0[j], r0[j]));
        } else {  // the odd column
            const float right = __shfl_down_sync(0xffffffffu, d0[j], 1);
            const float up = j > 0 ? d1[j - 1] : ab1, down = j < ROWS - 1 ? d1[j + 1] : be1;
            d1[j] = fmaf(i1[j], fmaf(rm, right, d0[j]) + (up + down), fmaf(omc, d1[j], r1[j]));
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
                                                         int done_stride, int nhalf, int start_colour) {
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
    const float omc = 1.f - omega[h];
    // the lanes at the window's sides have no neighbour across it (a zero);
    // the shuffle's own value, finite, is multiplied by zero instead
    const float lm = lane == 0 ? 0.f : 1.f, rm = lane == 31 ? 0.f : 1.f;
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
            half_sweep<0>(d0, d1, r0, r1, i0, i1, ab0, ab1, be0, be1, lm, rm, omc);
        else
            half_sweep<1>(d0, d1, r0, r1, i0, i1, ab0, ab1, be0, be1, lm, rm, omc);
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

// ------------------------------------------------------------------ wide windows (TMA)

constexpr int WX = 128;              // window columns
constexpr int WROWS = 8;             // rows per warp; a window has 8 rows per warp of its block
// Two shapes: 8 warps (128 x 64 windows, two blocks per SM) or 16 warps
// (128 x 128 windows, one block per SM: a smaller share of the window is
// halo, 1.31 pixels swept per interior pixel at depth 8 against 1.52).
constexpr size_t wide_smem(int warps) {
    return (size_t)3 * WX * WROWS * warps * sizeof(float) + (size_t)2 * warps * 2 * (WX / 4) * sizeof(float4);
}
__device__ int g_wide_wait_failed;

// The first window at or after `t`, in steps of `step`, whose history is not settled.
__device__ __forceinline__ int next_live(int t, int ntiles, int step, const int4 *tiles, const int32_t *done,
                                         int stride) {
    while (t < ntiles && done[(int64_t)tiles[t].x * stride]) t += step;
    return t;
}

// One half-sweep of colour C over rows J0..J1-1 of a lane's 8 rows x 4
// columns.  Column c of row j has colour (c + j) mod 2 (windows start at even
// x and y): colour C takes columns 0 and 2 of the rows with C + j even, 1 and
// 3 of the others.  Every update reads only pixels of the other colour, which
// this half-sweep does not change.
template <int C, int J0, int J1>
__device__ __forceinline__ void rows4(float4 (&d)[WROWS], const float4 (&a)[WROWS], const float4 (&b)[WROWS],
                                      const float4 ab, const float4 be, float lm, float rm, float omc) {
    // the across-lane neighbours first: they are of the other colour, which
    // this half-sweep does not change, and their latency then overlaps
    float nb[WROWS];
#pragma unroll
    for (int j = J0; j < J1; ++j)
        nb[j] = ((C + j) & 1) == 0 ? __shfl_up_sync(0xffffffffu, d[j].w, 1) : __shfl_down_sync(0xffffffffu, d[j].x, 1);
#pragma unroll
    for (int j = J0; j < J1; ++j) {
        const float4 up = j > 0 ? d[j - 1] : ab, dn = j < WROWS - 1 ? d[j + 1] : be;
        if (((C + j) & 1) == 0) {
            const float left = nb[j];
            const float s0 = fmaf(lm, left, d[j].y) + (up.x + dn.x);
            const float s2 = (d[j].y + d[j].w) + (up.z + dn.z);
            d[j].x = fmaf(a[j].x, s0, fmaf(omc, d[j].x, b[j].x));
            d[j].z = fmaf(a[j].z, s2, fmaf(omc, d[j].z, b[j].z));
        } else {
            const float right = nb[j];
            const float s1 = (d[j].x + d[j].z) + (up.y + dn.y);
            const float s3 = fmaf(rm, right, d[j].z) + (up.w + dn.w);
            d[j].y = fmaf(a[j].y, s1, fmaf(omc, d[j].y, b[j].y));
            d[j].w = fmaf(a[j].w, s3, fmaf(omc, d[j].w, b[j].w));
        }
    }
}

// What a block needs of a window, staged in shared memory by thread 0 one
// window ahead, so that no thread waits on a global load at a window's start.
struct WideTile {
    int4 tl;      // (history, x0, y0, 0); history < 0: no window left
    int4 dm;      // the history's dimensions
    int64_t off;  // its first pixel
    float omc;    // 1 - omega
};

// maps: 4 per history (d32a, d32b, r32, inv32); src_map picks the buffer
// read (0 or 1), dst is the other.  tiles: (history, x0, y0, 0) per window.
// zero_start: the correction starts at zero (the first launch of a solve):
// it is not read.  apply_c: the last launch of a solve adds its correction to
// the FP64 field (floored at zero when `floor`) instead of writing it to dst.
template <int DEPTH, int WWARPS>
__global__ void __launch_bounds__(32 * WWARPS, WWARPS == 8 ? 2 : 1)
    k_sor32_wide(const CUtensorMap *__restrict__ maps, int src_map, float *__restrict__ dst,
                 const int4 *__restrict__ tiles, int ntiles, const int4 *__restrict__ dims,
                 const int64_t *__restrict__ off, const float *__restrict__ omega, const int32_t *done,
                 int done_stride, int nhalf, int start_colour, int zero_start, double *__restrict__ apply_c,
                 int floor, unsigned long long wait_ns, int skip_copies, unsigned long long *corr, int corr_stride) {
    constexpr int WY = WROWS * WWARPS;  // window rows
    constexpr int STAGE = WX * WY;      // floats per array of the staged window
    extern __shared__ __align__(128) float smem[];
    const float4 *sd = (const float4 *)smem, *sb = (const float4 *)(smem + STAGE),
                 *sa = (const float4 *)(smem + 2 * STAGE);
    float4 *edge = (float4 *)(smem + 3 * STAGE);  // [buffer][warp][0 top, 1 bottom][lane]
    __shared__ __align__(8) uint64_t bar_word;
    __shared__ WideTile s_info[2];
    __shared__ int s_fail;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t bar = sh_addr(&bar_word);
    const uint32_t boxes = zero_start ? 2u : 3u;
    // thread 0: find the next live window at or after t, stage its scalars
    // in s_info[slot] and start its copies
    auto stage_next = [&](int t, int slot) {
        t = next_live(t, ntiles, gridDim.x, tiles, done, done_stride);
        WideTile w;
        w.tl = make_int4(-1, 0, 0, 0);
        if (t < ntiles) {
            w.tl = tiles[t];
            w.tl.w = t;
            w.dm = dims[w.tl.x];
            w.off = off[w.tl.x];
            w.omc = 1.f - omega[w.tl.x];
            const CUtensorMap *m = maps + 4 * w.tl.x;
            mbar_expect_tx(bar, (uint32_t)(boxes * STAGE * sizeof(float)));
            // skip_copies (a failure test): the bytes announced never come,
            // and the wait below runs out
            if (!skip_copies) {
                if (!zero_start) tma_load_2d(smem, m + src_map, bar, w.tl.y, w.tl.z);
                tma_load_2d(smem + STAGE, m + 2, bar, w.tl.y, w.tl.z);
                tma_load_2d(smem + 2 * STAGE, m + 3, bar, w.tl.y, w.tl.z);
            }
        }
        s_info[slot] = w;
    };
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
        s_fail = 0;
        stage_next(blockIdx.x, 0);
    }
    __syncthreads();
    uint32_t parity = 0;
    const float lm = lane == 0 ? 0.f : 1.f, rm = lane == 31 ? 0.f : 1.f;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    auto ed = [&](int buf, int w, int side) -> float4 & { return edge[((buf * WWARPS + w) * 2 + side) * 32 + lane]; };
    for (int slot = 0;; slot ^= 1) {
        const WideTile info = s_info[slot];
        if (info.tl.x < 0) break;
        if (!mbar_wait_bounded(bar, parity, wait_ns)) s_fail = 1;
        float4 d[WROWS], a[WROWS], b[WROWS];
#pragma unroll
        for (int j = 0; j < WROWS; ++j) {
            const int k = (warp * WROWS + j) * 32 + lane;
            d[j] = zero_start ? z4 : sd[k];
            b[j] = sb[k];
            a[j] = sa[k];
        }
        __syncthreads();  // the stage is read: free for the next window
        if (s_fail) {
            // leave no copy in flight into this block's shared memory
            if (threadIdx.x == 0) {
                mbar_wait_bounded(bar, parity, wait_ns);
                atomicExch(&g_wide_wait_failed, 1);
            }
            return;
        }
        parity ^= 1u;
        if (threadIdx.x == 0) {
            // the generic-proxy reads of the stage before the async-proxy writes
            fence_proxy_async_shared();
            stage_next(info.tl.w + gridDim.x, slot ^ 1);
        }
        const float omc = info.omc;
        ed(0, warp, 0) = d[0];
        ed(0, warp, 1) = d[WROWS - 1];
        __syncthreads();
        for (int s = 0; s < nhalf; ++s) {
            const int buf = s & 1;
            const float4 ab = warp > 0 ? ed(buf, warp - 1, 1) : z4;
            const float4 be = warp < WWARPS - 1 ? ed(buf, warp + 1, 0) : z4;
            if (((start_colour + s) & 1) == 0)
                rows4<0, 0, WROWS>(d, a, b, ab, be, lm, rm, omc);
            else
                rows4<1, 0, WROWS>(d, a, b, ab, be, lm, rm, omc);
            if (s + 1 < nhalf) {
                // the other buffer was last read before the previous barrier
                ed(buf ^ 1, warp, 0) = d[0];
                ed(buf ^ 1, warp, 1) = d[WROWS - 1];
                __syncthreads();
            }
        }
        // the interior back to global memory: the warp's rows inside it (a
        // range uniform over the warp), the lane's columns inside it (all four,
        // none, or a few at a history border that cuts a float4)
        const int x0 = info.tl.y, y0 = info.tl.z;
        const int4 dm = info.dm;
        const int ix0 = x0 == 0 ? 0 : x0 + DEPTH, ix1 = x0 + WX >= dm.x ? dm.x : x0 + WX - DEPTH;
        const int iy0 = y0 == 0 ? 0 : y0 + DEPTH, iy1 = y0 + WY >= dm.y ? dm.y : y0 + WY - DEPTH;
        const int wy = y0 + warp * WROWS;
        const int j0 = max(iy0 - wy, 0), j1 = min(iy1 - wy, WROWS);
        const int gx = x0 + 4 * lane;
        const bool full = gx >= ix0 && gx + 4 <= ix1;
        const bool part = !full && gx + 4 > ix0 && gx < ix1;
        const int64_t first = info.off + (int64_t)wy * dm.x + gx;
        if (apply_c) {
            // c += d on the free pixels (held ones have a = 0 and d = 0 throughout)
            double *row = apply_c + first;
            float most = 0.f;   // the largest |d| the window adds
            double top = 0.0;   // and the largest |c| it leaves
#pragma unroll
            for (int j = 0; j < WROWS; ++j, row += dm.x) {
                if (j < j0 || j >= j1 || !(full || part)) continue;
                const float dv[4] = {d[j].x, d[j].y, d[j].z, d[j].w};
                const float av[4] = {a[j].x, a[j].y, a[j].z, a[j].w};
                if (corr) {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (full || (gx + e >= ix0 && gx + e < ix1)) most = fmaxf(most, fabsf(dv[e]));
                }
                if (full) {
                    double2 c01 = *(double2 *)row, c23 = *(double2 *)(row + 2);
                    double cv[4] = {c01.x, c01.y, c23.x, c23.y};
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (dv[e] != 0.f || av[e] != 0.f) {
                            cv[e] = cv[e] + (double)dv[e];
                            if (floor) cv[e] = fmax(cv[e], 0.0);
                            top = fmax(top, fabs(cv[e]));
                        }
                    *(double2 *)row = make_double2(cv[0], cv[1]);
                    *(double2 *)(row + 2) = make_double2(cv[2], cv[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (gx + e >= ix0 && gx + e < ix1 && (dv[e] != 0.f || av[e] != 0.f)) {
                            double v = row[e] + (double)dv[e];
                            row[e] = floor ? fmax(v, 0.0) : v;
                            top = fmax(top, fabs(row[e]));
                        }
                }
            }
            if (corr) {
                // one atomic per warp and window
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) most = fmaxf(most, __shfl_xor_sync(0xffffffffu, most, o));
                for (int o = 16; o > 0; o >>= 1) top = fmax(top, __shfl_xor_sync(0xffffffffu, top, o));
                if (lane == 0) {
                    unsigned long long *mine = corr + (int64_t)info.tl.x * corr_stride;
                    if (most > 0.f) atomicMax(mine, (unsigned long long)__double_as_longlong((double)most));
                    if (top > 0.0) atomicMax(mine + 1, (unsigned long long)__double_as_longlong(top));
                }
            }
        } else {
            float *row = dst + first;
#pragma unroll
            for (int j = 0; j < WROWS; ++j, row += dm.x) {
                if (j < j0 || j >= j1) continue;
                if (full) {
                    *(float4 *)row = d[j];
                } else if (part) {
                    if (gx >= ix0 && gx < ix1) row[0] = d[j].x;
                    if (gx + 1 >= ix0 && gx + 1 < ix1) row[1] = d[j].y;
                    if (gx + 2 >= ix0 && gx + 2 < ix1) row[2] = d[j].z;
                    if (gx + 3 >= ix0 && gx + 3 < ix1) row[3] = d[j].w;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ volumes

// One half-sweep in place, any depth of lattice (volumes).
__global__ void k_sor32_half(float *__restrict__ dlt, const float *__restrict__ rhs, const float *__restrict__ inv,
                             const int4 *__restrict__ dims, const int64_t *__restrict__ off,
                             const int32_t *__restrict__ blk, int nh, const float *__restrict__ omega,
                             const int32_t *done, int done_stride, int colour) {
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
    // (x pair) + (y pair) [+ (z pair)]: in 2D the windowed kernels' order
    const float xm = x > 0 ? dlt[i - 1] : 0.f, xp = x + 1 < dm.x ? dlt[i + 1] : 0.f;
    const float ym = y > 0 ? dlt[i - w] : 0.f, yp = y + 1 < dm.y ? dlt[i + w] : 0.f;
    float sum = (xm + xp) + (ym + yp);
    if (dm.z > 1) sum += (z > 0 ? dlt[i - slice] : 0.f) + (z + 1 < dm.z ? dlt[i + slice] : 0.f);
    dlt[i] = fmaf(inv[i], sum, fmaf(1.f - omega[h], dlt[i], rhs[i]));
}

// ------------------------------------------------------------------ volumes, blocked

// Temporal blocking in a volume (2.5-D: tiles across x and y marched along
// z).  A block takes a VX x VY tile of a history's columns over a chunk of
// its slices [z0, z1) and runs S <= D half-sweeps on it in one pass along z:
// at step t, stage s (the s-th half-sweep) updates slice t - 2 (s - 1), its
// pixels of that half-sweep's colour, in place in a ring of slices in shared
// memory.  Two slices between stages keep every read at the right level:
// stage s reads slices p - 1, p, p + 1 after stage s - 1 (slice p + 1 was
// done a step ago, slice p - 1 holds stage s's own colour, which stage s
// does not read), and no slice a stage reads is written in the same step.
// The tile's halo is D pixels across x and y and D slices along z beyond
// the chunk; what lies beyond the loaded slices or the tile reads as zero,
// exact at the history's border and an error that moves in one ring per
// half-sweep inside it, so every pixel D or more from such an edge equals S
// in-place half-sweeps of the whole history (as k_sor32_half gives them,
// to the bit: the same sums in the same order).  A thread owns a pair of
// columns (one pixel of each colour per slice); the next slice is brought
// into registers while the stages run, then into the ring, one barrier a
// step.  The stage's coefficients are read from global memory (L1 keeps a
// slice's for the S steps that use it).
constexpr int VX = 64;  // tile columns: 32 lanes x 2

template <int D, int VY>
__global__ void __launch_bounds__(32 * VY) k_sor32_vol(const float *__restrict__ src, float *__restrict__ dst,
                                                       const float *__restrict__ rhs, const float *__restrict__ inv,
                                                       const int4 *__restrict__ dims, const int64_t *__restrict__ off,
                                                       const int4 *__restrict__ tiles, int vz,
                                                       const float *__restrict__ omega, const int32_t *done,
                                                       int done_stride, int nhalf, int start_colour, int zero_start,
                                                       double *__restrict__ apply_c, int floor) {
    constexpr int R = 2 * D + 2;  // ring slots: slices t - 2 D + 1 .. t + 2 in use at step t
    extern __shared__ __align__(16) float ring[];  // [R][VY][VX]
    const int4 tl = tiles[blockIdx.x];
    const int h = tl.x;
    if (done[(int64_t)h * done_stride]) return;
    const int4 dm = dims[h];
    const int x0 = tl.y, y0 = tl.z, z0 = tl.w;
    const int z1 = min(z0 + vz, dm.z);
    const int zlo = max(z0 - D, 0), zhi = min(z1 + D, dm.z);
    const int S = nhalf;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int lx = 2 * tx, gx = x0 + lx, gy = y0 + ty;
    const bool in0 = gx < dm.x && gy < dm.y, in1 = gx + 1 < dm.x && gy < dm.y;
    // offsets inside the history in 32 bits (a history holds fewer than 2^31
    // pixels), its arrays from their first pixel
    const int plane = dm.x * dm.y;
    const int col = gy * dm.x + gx;  // this thread's first pixel in slice 0
    const int64_t base = off[h];
    const float *hsrc = src + base, *hrhs = rhs + base, *hinv = inv + base;
    float *hdst = dst + base;
    double *hc = apply_c ? apply_c + base : nullptr;
    const float omc = 1.f - omega[h];
    // the output interior of the tile (a window edge on the history's border makes no error)
    const int ix0 = x0 == 0 ? 0 : x0 + D, ix1 = x0 + VX >= dm.x ? dm.x : x0 + VX - D;
    const int iy0 = y0 == 0 ? 0 : y0 + D, iy1 = y0 + VY >= dm.y ? dm.y : y0 + VY - D;
    const bool out_y = gy >= iy0 && gy < iy1;
    const bool out0 = in0 && out_y && gx >= ix0 && gx < ix1, out1 = in1 && out_y && gx + 1 >= ix0 && gx + 1 < ix1;
    // this thread's pair in ring slot k
    float2 *const mine = (float2 *)(ring + ty * VX) + tx;
    auto at = [&](int k) -> float2 * { return mine + k * (VY * VX / 2); };
    auto wrap = [](int k) { return k < 0 ? k + R : (k >= R ? k - R : k); };
    auto load = [&](int o, float &v0, float &v1) {  // o: the slice's offset
        v0 = v1 = 0.f;
        if (!zero_start) {
            if (in0) v0 = __ldg(hsrc + o + col);
            if (in1) v1 = __ldg(hsrc + o + col + 1);
        }
    };
    // the first two slices
    for (int z = zlo; z < min(zlo + 2, zhi); ++z) {
        float v0, v1;
        load(z * plane, v0, v1);
        *at(z % R) = make_float2(v0, v1);
    }
    __syncthreads();
    const int tend = zhi - 1 + 2 * (S - 1);
    int rt = zlo % R;     // ring slot of slice t
    int toff = zlo * plane;  // offset of slice t
    for (int t = zlo; t <= tend; ++t, rt = wrap(rt + 1), toff += plane) {
        // the slice after next into registers while the stages run
        const int zn = t + 2;
        float n0 = 0.f, n1 = 0.f;
        if (zn < zhi) load(toff + 2 * plane, n0, n1);
#pragma unroll
        for (int s = 1; s <= D; ++s) {
            if (s > S) break;
            const int p = t - 2 * (s - 1);  // the same for the whole block
            if (p < zlo || p >= zhi) continue;
            const int c = (start_colour + s - 1) & 1;
            // the pixel of colour c in this thread's pair ((x + y + z) mod 2 == c,
            // x0 even): the same e for a warp, which holds one row
            const int e = (c + gy + p) & 1;
            const int k = wrap(rt - 2 * (s - 1));
            float2 *row = at(k);
            const float2 me = *row;
            // x neighbours: the left pair's second pixel, the right pair's first
            const float left = __shfl_up_sync(0xffffffffu, me.y, 1);
            const float right = __shfl_down_sync(0xffffffffu, me.x, 1);
            const float2 z2 = make_float2(0.f, 0.f);
            const float2 ym2 = ty > 0 ? row[-VX / 2] : z2, yp2 = ty + 1 < VY ? row[VX / 2] : z2;
            const float2 zm2 = p - 1 >= zlo ? *at(wrap(k - 1)) : z2;
            const float2 zp2 = p + 1 < zhi ? *at(wrap(k + 1)) : z2;
            if (!(e ? in1 : in0)) continue;  // outside the history: stays zero
            float xm, xp, ym, yp, zm, zp, cur;
            if (e == 0) {
                xm = tx > 0 ? left : 0.f; xp = me.y; ym = ym2.x; yp = yp2.x; zm = zm2.x; zp = zp2.x; cur = me.x;
            } else {
                xm = me.x; xp = tx < 31 ? right : 0.f; ym = ym2.y; yp = yp2.y; zm = zm2.y; zp = zp2.y; cur = me.y;
            }
            // k_sor32_half's sums, in its order
            float sum = (xm + xp) + (ym + yp);
            sum += (zm + zp);
            const int i = toff - 2 * (s - 1) * plane + col + e;
            const float v = fmaf(__ldg(hinv + i), sum, fmaf(omc, cur, __ldg(hrhs + i)));
            *row = e == 0 ? make_float2(v, me.y) : make_float2(me.x, v);
        }
        // slice t - 2 (S - 1) has had every half-sweep: its interior out
        const int pf = t - 2 * (S - 1);
        if (pf >= z0 && pf < z1) {
            const float2 q = *at(wrap(rt - 2 * (S - 1)));
            const int i = toff - 2 * (S - 1) * plane + col;
            if (hc) {
                // the last launch of a correction: c += d on the free pixels
                // (a held pixel has a = 0 and d = 0 throughout), floored as
                // the reference's update is (pde.rs:395)
                if (out0 && (q.x != 0.f || __ldg(hinv + i) != 0.f)) {
                    const double v = hc[i] + (double)q.x;
                    hc[i] = floor ? fmax(v, 0.0) : v;
                }
                if (out1 && (q.y != 0.f || __ldg(hinv + i + 1) != 0.f)) {
                    const double v = hc[i + 1] + (double)q.y;
                    hc[i + 1] = floor ? fmax(v, 0.0) : v;
                }
            } else {
                if (out0) hdst[i] = q.x;
                if (out1) hdst[i + 1] = q.y;
            }
        }
        if (zn < zhi) *at(wrap(rt + 2)) = make_float2(n0, n1);
        __syncthreads();
    }
}

typedef void (*TbKernel)(const float *, float *, const float *, const float *, const int4 *, const int64_t *,
                         const int32_t *, int, const float *, const int32_t *, int, int, int);
typedef void (*WideKernel)(const CUtensorMap *, int, float *, const int4 *, int, const int4 *, const int64_t *,
                           const float *, const int32_t *, int, int, int, int, double *, int, unsigned long long,
                           int, unsigned long long *, int);

TbKernel tb_kernel(int depth) {
    switch (depth) {
    case 2: return k_sor32_tb<2>;
    case 4: return k_sor32_tb<4>;
    case 6: return k_sor32_tb<6>;
    default: return k_sor32_tb<8>;
    }
}

template <int W>
WideKernel wide_kernel_of(int depth) {
    switch (depth) {
    case 2: return k_sor32_wide<2, W>;
    case 4: return k_sor32_wide<4, W>;
    case 6: return k_sor32_wide<6, W>;
    default: return k_sor32_wide<8, W>;
    }
}

typedef void (*VolKernel)(const float *, float *, const float *, const float *, const int4 *, const int64_t *,
                          const int4 *, int, const float *, const int32_t *, int, int, int, int, double *, int);

VolKernel vol_kernel(int depth, int vy) {
    if (vy == 16) return depth >= 4 ? k_sor32_vol<4, 16> : k_sor32_vol<2, 16>;
    return depth >= 4 ? k_sor32_vol<4, 32> : k_sor32_vol<2, 32>;
}

size_t vol_smem(int depth, int vy) { return (size_t)(2 * depth + 2) * vy * VX * sizeof(float); }

WideKernel wide_kernel(int depth, int warps) { return warps == 16 ? wide_kernel_of<16>(depth) : wide_kernel_of<8>(depth); }

// Window starts along one axis of n pixels for windows of `win` with a halo
// of `depth`: the first at 0, then every win - 2 depth until one reaches n.
void axis_starts(int n, int win, int depth, std::vector<int> &out) {
    out.clear();
    out.push_back(0);
    if (n <= win) return;
    const int step = win - 2 * depth;
    const int last = (n - win + step - 1) / step;
    for (int k = 1; k <= last; ++k) out.push_back(k * step);
}

// The wide kernel's tensor maps, windows and grid, if every history allows it.
int wide_init(Sor32 &s, cw_field_s *f, int warps) {
    s.wide = false;
    s.wwarps = warps;
    const int WY = WROWS * warps;
    const size_t smem = wide_smem(warps);
    const Geom &g = f->g;
    for (uint32_t k = 0; k < g.nh; ++k)
        if (g.d[k] != 1 || g.w[k] % 4 != 0 || g.off[k] % 4 != 0) return CW_OK;
    if (s.depth % 2 != 0 || s.depth > 8) return CW_OK;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return CW_OK;
    std::vector<CUtensorMap> maps(4 * (size_t)g.nh);
    float *arrays[4] = {f->d32a, f->d32b, f->r32, f->inv32};
    for (uint32_t k = 0; k < g.nh; ++k)
        for (int m = 0; m < 4; ++m) {
            cuuint64_t dim[2] = {(cuuint64_t)g.w[k], (cuuint64_t)g.h[k]};
            cuuint64_t stride[1] = {(cuuint64_t)g.w[k] * sizeof(float)};
            cuuint32_t box[2] = {(cuuint32_t)WX, (cuuint32_t)WY};
            cuuint32_t estride[2] = {1, 1};
            CUresult r = enc(&maps[4 * k + m], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, arrays[m] + g.off[k], dim, stride,
                             box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return CW_OK;  // the narrow kernel serves
        }
    WideKernel kern = wide_kernel(s.depth, warps);
    if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
        (void)cudaGetLastError();
        return CW_OK;  // the narrow kernel serves
    }
    int per_sm = 0, dev = 0, nsm = 0;
    CW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)kern, 32 * warps, smem));
    if (per_sm < 1) return CW_OK;
    CW_CUDA(cudaGetDevice(&dev));
    CW_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    std::vector<int4> tiles;
    std::vector<int> xs, ys;
    for (uint32_t k = 0; k < g.nh; ++k) {
        axis_starts(g.w[k], WX, s.depth, xs);
        axis_starts(g.h[k], WY, s.depth, ys);
        for (int y : ys)
            for (int x : xs) tiles.push_back(make_int4((int)k, x, y, 0));
    }
    int rc;
    CUtensorMap *dm = nullptr;
    if ((rc = dalloc(&dm, maps.size())) != CW_OK) return rc;
    s.maps = dm;
    if ((rc = dalloc(&s.wtiles, tiles.size())) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(s.maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                            stream()));
    CW_CUDA(cudaMemcpyAsync(s.wtiles, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    s.nwtiles = (int)tiles.size();
    s.wgrid = std::min<int>(s.nwtiles, per_sm * nsm);
    s.wide = true;
    return CW_OK;
}

// The volume kernel's tiles: VX x vy columns (halo `depth`) by chunks of vz
// slices, vz the largest of 64, 32, 16 that still gives the device three
// tiles for every block it holds at once.
int vol_init(Sor32 &s, cw_field_s *f, int window) {
    s.vol = false;
    const Geom &g = f->g;
    for (uint32_t k = 0; k < g.nh; ++k)
        if (g.d[k] < 2) return CW_OK;
    s.vdepth = s.depth >= 4 ? 4 : 2;
    s.vy = window == CW_WINDOW_64 ? 16 : 32;
    VolKernel kern = vol_kernel(s.vdepth, s.vy);
    const size_t smem = vol_smem(s.vdepth, s.vy);
    CW_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, dev = 0, nsm = 0;
    CW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)kern, 32 * s.vy, smem));
    if (per_sm < 1) return CW_OK;  // one half-sweep per launch serves
    CW_CUDA(cudaGetDevice(&dev));
    CW_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    std::vector<int> xs, ys;
    std::vector<int64_t> columns(g.nh);
    for (uint32_t k = 0; k < g.nh; ++k) {
        axis_starts(g.w[k], VX, s.vdepth, xs);
        axis_starts(g.h[k], s.vy, s.vdepth, ys);
        columns[k] = (int64_t)xs.size() * ys.size();
    }
    // chunks: the longest of 64, 32, 16 slices that still gives three tiles
    // for every block the device holds at once (one tile a block, for less of
    // the z halo's redundant work, measured 11 % slower on the 256^3 spheroid)
    const int64_t want = 3LL * per_sm * nsm;
    s.vz = 16;
    for (int vz : {64, 32}) {
        int64_t n = 0;
        for (uint32_t k = 0; k < g.nh; ++k) n += columns[k] * ((g.d[k] + vz - 1) / vz);
        if (n >= want) {
            s.vz = vz;
            break;
        }
    }
    std::vector<int4> tiles;
    for (uint32_t k = 0; k < g.nh; ++k) {
        axis_starts(g.w[k], VX, s.vdepth, xs);
        axis_starts(g.h[k], s.vy, s.vdepth, ys);
        for (int z = 0; z < g.d[k]; z += s.vz)
            for (int y : ys)
                for (int x : xs) tiles.push_back(make_int4((int)k, x, y, z));
    }
    int rc;
    if ((rc = dalloc(&s.vtiles, tiles.size())) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(s.vtiles, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    s.nvtiles = (int)tiles.size();
    s.vol = true;
    return CW_OK;
}

}  // namespace

int Sor32::init(cw_field_s *f, int d, const std::vector<double> &om, int window) {
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
        wide = false;
        if ((window == CW_WINDOW_AUTO || window == CW_WINDOW_TALL) &&
            (rc = wide_init(*this, f, window == CW_WINDOW_TALL ? 16 : 8)) != CW_OK)
            return rc;
        if (!wide) {
            const int in = WIN - 2 * depth;
            for (uint32_t k = 0; k < f->g.nh; ++k)
                per[k] = (int64_t)((f->g.w[k] + in - 1) / in) * ((f->g.h[k] + in - 1) / in);
            rc = tiles.build(per, 1);
        }
    } else {
        vol = false;
        if (depth > 1 && (rc = vol_init(*this, f, window)) != CW_OK) return rc;
        if (!vol) {
            for (uint32_t k = 0; k < f->g.nh; ++k) per[k] = (int64_t)((f->g.w[k] + 1) / 2) * f->g.h[k] * f->g.d[k];
            rc = sites.build(per, 256);
        }
    }
    ping = f->d32a;
    pong = f->d32b;
    out = ping;
    return rc;
}

int Sor32::sweeps(cw_field_s *f, int n, const int32_t *done, int done_stride, float *start, bool apply,
                  unsigned long long *corr, int corr_stride) {
    if (apply && !wide && !vol) return fail(CW_ERR_CONFIG, "only the wide and volume FP32 kernels apply their correction");
    if (start) {  // begin from this (zeroed) buffer; the other is scratch
        ping = start;
        pong = start == f->d32a ? f->d32b : f->d32a;
    }
    if (vol) {
        // 2n half-sweeps, vdepth per launch (fewer in the last), ping-pong
        // between the buffers; the first launch starts from zero
        float *a = ping, *b = pong;
        int remaining = 2 * n, done_half = 0;
        VolKernel kern = vol_kernel(vdepth, vy);
        const size_t smem = vol_smem(vdepth, vy);
        while (remaining > 0) {
            const int dd = remaining < vdepth ? remaining : vdepth;
            // with `apply` the last launch adds its correction to the field
            const bool last = remaining == dd;
            kern<<<nvtiles, 32 * vy, smem, stream()>>>(a, b, f->r32, f->inv32, f->g.d_dims, f->g.d_off, vtiles, vz,
                                                       omega, done, done_stride, dd, done_half & 1,
                                                       done_half == 0 ? 1 : 0, apply && last ? f->c : nullptr,
                                                       f->floor ? 1 : 0);
            CW_LAUNCHED();
            remaining -= dd;
            done_half += dd;
            float *t = a; a = b; b = t;
        }
        out = apply ? nullptr : a;
        return CW_OK;
    }
    if (!blocked) {
        for (int s = 0; s < n; ++s)
            for (int colour = 0; colour < 2; ++colour) {
                k_sor32_half<<<sites.nblocks, 256, 0, stream()>>>(ping, f->r32, f->inv32, f->g.d_dims, f->g.d_off,
                                                                  sites.d_blk, f->g.nh, omega, done, done_stride,
                                                                  colour);
                CW_LAUNCHED();
            }
        out = ping;
        return CW_OK;
    }
    // 2n half-sweeps, `depth` per launch (fewer in the last), starting from
    // the zeroed buffer; the windows are those of `depth`, whose halo is deep
    // enough for a shorter last launch too
    float *a = ping, *b = pong;
    int remaining = 2 * n, done_half = 0;
    while (remaining > 0) {
        int dd = remaining < depth ? remaining : depth;
        if (wide) {
            // the first launch starts from zero without reading it; with
            // `apply` the last adds its correction to the field
            const bool last = remaining == dd;
            wide_kernel(depth, wwarps)<<<wgrid, 32 * wwarps, wide_smem(wwarps), stream()>>>(
                (const CUtensorMap *)maps, a == f->d32a ? 0 : 1, b, wtiles, nwtiles, f->g.d_dims, f->g.d_off, omega,
                done, done_stride, dd, done_half & 1, done_half == 0 ? 1 : 0, apply && last ? f->c : nullptr,
                f->floor ? 1 : 0, test_faults().wait_ns ? test_faults().wait_ns : TMA_WAIT_NS, test_faults().skip_tma,
                apply && last ? corr : nullptr, corr_stride);
        } else {
            tb_kernel(depth)<<<tiles.nblocks, 32 * WARPS, 0, stream()>>>(a, b, f->r32, f->inv32, f->g.d_dims,
                                                                         f->g.d_off, tiles.d_blk, f->g.nh, omega,
                                                                         done, done_stride, dd, done_half & 1);
        }
        CW_LAUNCHED();
        remaining -= dd;
        done_half += dd;
        float *t = a; a = b; b = t;
    }
    out = apply ? nullptr : a;
    return CW_OK;
}

void Sor32::release() {
    dfree(omega);
    tiles.release();
    sites.release();
    CUtensorMap *m = (CUtensorMap *)maps;
    dfree(m);
    maps = nullptr;
    dfree(wtiles);
    wide = false;
    dfree(vtiles);
    vol = false;
}

// Whether a wide-kernel block gave up waiting for its window (and clears the record).
int sor32_wait_failed() {
    int v = 0, zero = 0;
    CW_CUDA(cudaMemcpyFromSymbol(&v, g_wide_wait_failed, sizeof v));
    if (v) {
        CW_CUDA(cudaMemcpyToSymbol(g_wide_wait_failed, &zero, sizeof zero));
        return fail(CW_ERR_TIMEOUT, "an FP32 SOR block waited too long for its window's TMA copies");
    }
    return CW_OK;
}

}  // namespace cw
