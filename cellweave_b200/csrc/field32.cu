// FP32 red-black SOR on the correction equation of the defect-correction
// solve (see field.cu).  Built with fused multiply-add: this is the fast
// path, and its error is removed by the FP64 residual and correction steps.
//
// A flat history is cut into TX x TY tiles.  Each launch loads a tile with a
// halo `depth` pixels deep into shared memory (correction, right-hand side
// and inverse diagonal), runs `depth` half-sweeps there, the valid region
// shrinking by one ring per half-sweep, and writes the tile's interior to
// the other buffer.  The interior is exactly what `depth` global half-sweeps
// would give, and the correction makes one round trip through HBM per
// `depth` half-sweeps instead of one per half-sweep.
#include "cw_internal.cuh"
#include "field_kernels.cuh"

namespace cw {
namespace {

constexpr int TX = 128;
constexpr int TY = 32;
constexpr int THREADS = 512;

__global__ void __launch_bounds__(THREADS) k_sor32_tb(const float *__restrict__ src, float *__restrict__ dst,
                                                      const float *__restrict__ rhs, const float *__restrict__ inv,
                                                      const int4 *__restrict__ dims, const int64_t *__restrict__ off,
                                                      const int32_t *__restrict__ blk, int nh,
                                                      const float *__restrict__ omega, const int32_t *done,
                                                      int done_stride, int depth, int start_colour, float dcoef) {
    extern __shared__ float sm[];
    __shared__ int s_h;
    if (threadIdx.x == 0) s_h = plan_history(blk, nh, blockIdx.x);
    __syncthreads();
    const int h = s_h;
    if (done[(int64_t)h * done_stride]) return;
    const int4 dm = dims[h];
    const int ntx = (dm.x + TX - 1) / TX;
    const int t = blockIdx.x - blk[h];
    const int tx0 = (t % ntx) * TX, ty0 = (t / ntx) * TY;
    const int EW = TX + 2 * depth, EH = TY + 2 * depth, E = EW * EH;
    float *sd = sm, *sr = sm + E, *si = sm + 2 * E;
    const int64_t base = off[h];
    const float om = omega[h];
    // load the tile and its halo; outside the grid everything is zero, which
    // drops the missing neighbours from the sum (their count is in `inv`)
    for (int e = threadIdx.x; e < E; e += THREADS) {
        int ex = e % EW, ey = e / EW;
        int gx = tx0 - depth + ex, gy = ty0 - depth + ey;
        float a = 0.f, b = 0.f, c = 0.f;
        if (gx >= 0 && gx < dm.x && gy >= 0 && gy < dm.y) {
            int64_t i = base + (int64_t)gy * dm.x + gx;
            a = src[i];
            b = rhs[i];
            c = inv[i];
        }
        sd[e] = a; sr[e] = b; si[e] = c;
    }
    __syncthreads();
    // half-sweeps: pixels of one colour, at least s rings in from the edge.
    // Threads take the pixels of the colour directly: row ey holds the
    // colour at ex = p, p + 2, ... with p fixed by the row's parity.
    const int HW = EW / 2 + 1;
    for (int s = 1; s <= depth; ++s) {
        const int colour = (start_colour + s - 1) & 1;
        const int rows = EH - 2 * s;
        for (int e = threadIdx.x; e < rows * HW; e += THREADS) {
            int ey = s + e / HW;
            int gy = ty0 - depth + ey;
            int par = (colour - (tx0 - depth) - gy) & 1;  // ex parity giving (gx + gy) % 2 == colour
            int ex = par + 2 * (e % HW);
            if (ex < s || ex >= EW - s) continue;
            int k = ey * EW + ex;
            float iv = si[k];
            if (iv == 0.f) continue;
            float sum = (sd[k - 1] + sd[k + 1]) + (sd[k - EW] + sd[k + EW]);
            float old = sd[k];
            sd[k] = old + om * ((sr[k] + dcoef * sum) * iv - old);
        }
        __syncthreads();
    }
    // store the interior
    for (int e = threadIdx.x; e < TX * TY; e += THREADS) {
        int ix = e % TX, iy = e / TX;
        int gx = tx0 + ix, gy = ty0 + iy;
        if (gx < dm.x && gy < dm.y) dst[base + (int64_t)gy * dm.x + gx] = sd[(iy + depth) * EW + ix + depth];
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

}  // namespace

int Sor32::init(cw_field_s *f, int d, const std::vector<double> &om) {
    depth = d < 1 ? 1 : (d > 16 ? 16 : d);
    blocked = depth > 1;
    for (uint32_t k = 0; k < f->g.nh; ++k) blocked = blocked && f->g.d[k] == 1;
    std::vector<float> omf(om.begin(), om.end());
    int rc = dalloc(&omega, omf.size());
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(omega, omf.data(), sizeof(float) * omf.size(), cudaMemcpyHostToDevice, stream()));
    std::vector<int64_t> per(f->g.nh);
    if (blocked) {
        for (uint32_t k = 0; k < f->g.nh; ++k)
            per[k] = (int64_t)((f->g.w[k] + TX - 1) / TX) * ((f->g.h[k] + TY - 1) / TY);
        rc = tiles.build(per, 1);
        if (rc == CW_OK) {
            size_t smem = 3 * sizeof(float) * (TX + 2 * depth) * (TY + 2 * depth);
            if (cudaFuncSetAttribute(k_sor32_tb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess)
                return fail(CW_ERR_CUDA, "shared memory for the blocked sweep");
        }
    } else {
        for (uint32_t k = 0; k < f->g.nh; ++k)
            per[k] = (int64_t)((f->g.w[k] + 1) / 2) * f->g.h[k] * f->g.d[k];
        rc = sites.build(per, 256);
    }
    ping = f->d32a;
    pong = f->d32b;
    out = ping;
    return rc;
}

int Sor32::sweeps(cw_field_s *f, int n, const int32_t *done, int done_stride) {
    float dcoef = (float)f->dcoef;
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
    // 2n half-sweeps, `depth` per launch, starting from the zeroed buffer
    float *a = ping, *b = pong;
    int remaining = 2 * n, done_half = 0;
    while (remaining > 0) {
        int dd = remaining < depth ? remaining : depth;
        size_t smem = 3 * sizeof(float) * (TX + 2 * dd) * (TY + 2 * dd);
        k_sor32_tb<<<tiles.nblocks, THREADS, smem, stream()>>>(a, b, f->r32, f->inv32, f->g.d_dims, f->g.d_off,
                                                                tiles.d_blk, f->g.nh, omega, done, done_stride, dd,
                                                                done_half & 1, dcoef);
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
