// An allocation-free entry point: the FP32 defect-correction solve of one
// flat field, with its scratch in a fixed array compiled into the library.
//
// Some callers cannot let a library allocate device memory.  A host whose
// device memory is all owned by another allocator (a framework's caching
// pool, an arena sized once at start-up) cannot have cudaMalloc and cudaFree
// called behind its back: they take memory the pool thinks is free and
// synchronise the whole device on the way.  The same holds for a caller in a
// loop with a fixed time budget, where an allocation's stall is not
// affordable.  cw_field_relax_noalloc serves them: the caller passes the
// field and its coefficients in device memory it owns, and everything the
// solve needs besides (the FP32 right-hand side, inverse diagonal and the two
// correction buffers, the convergence record) lives in `g_scratch` below.
//
// That array is NA_MAX_PIXELS * 16 bytes plus a 256-byte record, about 16 MiB,
// and every GPU that loads the library keeps it until the process exits.
// All calls share it: two calls whose work overlaps on the GPU (on two
// streams, or from two threads) corrupt each other's results, so calls must
// be serialised.  Each call overwrites every part of it it reads before
// reading it, so nothing a previous call left there matters.
#include <cmath>
#include <cstring>
#include <mutex>

#include "cw_internal.cuh"
#include "field_kernels.cuh"

namespace {

constexpr int64_t NA_MAX_PIXELS = 1 << 20;  // 1,048,576 pixels, a 1024 x 1024 field
constexpr size_t NA_RECORD = 256;
constexpr size_t NA_BYTES = NA_RECORD + 16 * (size_t)NA_MAX_PIXELS;

__device__ __align__(256) unsigned char g_scratch[NA_BYTES];

// The device address of g_scratch, found once per device (cudaGetSymbolAddress
// with that device current) on the first call made on it.
std::mutex g_mu;
void *g_addr[64] = {nullptr};

struct NaState {
    unsigned long long resid;  // max projected residual of the last pass (bits of a non-negative double)
    int32_t done;              // 0 running, 1 settled, 2 out of sweeps
    int32_t pad;
    int64_t inner;             // FP32 sweeps taken
    double last_resid;
};

struct NaField {
    double *c;
    const uint8_t *held;
    const double *up, *pr, *ks;
    double d, decay, source;
    int w, h;
};

__device__ __forceinline__ double na_sources(const NaField &f, int i, double t) {
    t = t + f.source;
    if (f.pr) t = t + f.pr[i];
    if (f.up) t = t - f.up[i];
    return t;
}

// FP64 residual r = b - A c (projected at the floor) into r32; the inverse
// diagonal on the first pass; zeroes the correction.
__global__ void k_na_residual(NaField f, NaState *st, float *r32, float *inv32, float *dz, int first) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double worst = 0.0;
    if (i < f.w * f.h && !st->done) {
        int x = i % f.w, y = i / f.w;
        float r_out = 0.f, inv_out = 0.f;
        if (!f.held[i]) {
            double sum, real;
            cw::pixel_sums64(f.c, i, x, y, 0, make_int4(f.w, f.h, 1, 0), sum, real);
            double den = real * f.d + f.decay;
            if (f.ks) den = den + f.ks[i];
            double cv = f.c[i];
            double r = na_sources(f, i, f.d * sum) - den * cv;
            if (cv <= 0.0 && r < 0.0) r = 0.0;
            worst = fabs(r);
            r_out = (float)r;
            inv_out = den > 0.0 ? (float)(1.0 / den) : 0.f;
        }
        r32[i] = r_out;
        if (first) inv32[i] = inv_out;
        dz[i] = 0.f;
    }
    worst = cw::warp_max(worst);
    if ((threadIdx.x & 31) == 0 && worst > 0.0) cw::atomic_max_nonneg(&st->resid, worst);
}

__global__ void k_na_check(NaState *st, double tol, int inner, int64_t max_sweeps) {
    if (threadIdx.x || blockIdx.x) return;
    if (!st->done) {
        double r = __longlong_as_double((long long)st->resid);
        st->last_resid = r;
        if (r < tol) st->done = 1;
        else if (st->inner >= max_sweeps) st->done = 2;
        else st->inner += inner;
    }
    st->resid = 0ull;
}

// `nhalf` red-black half-sweeps of A d = r on 64 x 64 windows with a halo of
// 8, the window's rows in registers: the single-field form of the batched
// kernel in field32.cu, reading its buffers from the fixed scratch.
constexpr int WIN = 64, WARPS = 8, ROWS = 8, DEPTH = 8, IN = WIN - 2 * DEPTH;

__global__ void __launch_bounds__(256) k_na_sweep(const float *__restrict__ src, float *__restrict__ dst,
                                                  const float *__restrict__ rhs, const float *__restrict__ inv,
                                                  int w, int h, float om, const NaState *st, int nhalf,
                                                  int start_colour, float dcoef) {
    __shared__ float edge[WARPS][2][WIN];
    if (st->done) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntx = (w + IN - 1) / IN;
    const int gx0 = (blockIdx.x % ntx) * IN - DEPTH, gy0 = (blockIdx.x / ntx) * IN - DEPTH;
    const int gx = gx0 + 2 * lane;
    const bool in0 = gx >= 0 && gx < w, in1 = gx + 1 >= 0 && gx + 1 < w;
    float d0[ROWS], d1[ROWS], r0[ROWS], r1[ROWS], i0[ROWS], i1[ROWS];
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int gy = gy0 + ROWS * warp + j;
        d0[j] = d1[j] = r0[j] = r1[j] = i0[j] = i1[j] = 0.f;
        if (gy >= 0 && gy < h) {
            const int row = gy * w + gx;
            if (in0) { d0[j] = src[row]; r0[j] = rhs[row]; i0[j] = inv[row]; }
            if (in1) { d1[j] = src[row + 1]; r1[j] = rhs[row + 1]; i1[j] = inv[row + 1]; }
        }
    }
    edge[warp][0][2 * lane] = d0[0];
    edge[warp][0][2 * lane + 1] = d1[0];
    edge[warp][1][2 * lane] = d0[ROWS - 1];
    edge[warp][1][2 * lane + 1] = d1[ROWS - 1];
    __syncthreads();
    for (int s = 0; s < nhalf; ++s) {
        const int c = (start_colour + s) & 1;
        const float ab0 = warp > 0 ? edge[warp - 1][1][2 * lane] : 0.f;
        const float ab1 = warp > 0 ? edge[warp - 1][1][2 * lane + 1] : 0.f;
        const float be0 = warp < WARPS - 1 ? edge[warp + 1][0][2 * lane] : 0.f;
        const float be1 = warp < WARPS - 1 ? edge[warp + 1][0][2 * lane + 1] : 0.f;
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            if (((c + j) & 1) == 0) {
                float left = __shfl_up_sync(0xffffffffu, d1[j], 1);
                if (lane == 0) left = 0.f;
                const float up = j > 0 ? d0[j - 1] : ab0, down = j < ROWS - 1 ? d0[j + 1] : be0;
                const float old = d0[j];
                d0[j] = old + om * ((r0[j] + dcoef * ((left + d1[j]) + (up + down))) * i0[j] - old);
            } else {
                float right = __shfl_down_sync(0xffffffffu, d0[j], 1);
                if (lane == 31) right = 0.f;
                const float up = j > 0 ? d1[j - 1] : ab1, down = j < ROWS - 1 ? d1[j + 1] : be1;
                const float old = d1[j];
                d1[j] = old + om * ((r1[j] + dcoef * ((d0[j] + right) + (up + down))) * i1[j] - old);
            }
        }
        __syncthreads();
        edge[warp][0][2 * lane] = d0[0];
        edge[warp][0][2 * lane + 1] = d1[0];
        edge[warp][1][2 * lane] = d0[ROWS - 1];
        edge[warp][1][2 * lane + 1] = d1[ROWS - 1];
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int ey = ROWS * warp + j, gy = gy0 + ey;
        if (ey < DEPTH || ey >= DEPTH + IN || gy >= h) continue;
        const int row = gy * w + gx;
        const int ex = 2 * lane;
        if (ex >= DEPTH && ex < DEPTH + IN && gx < w) dst[row] = d0[j];
        if (ex + 1 >= DEPTH && ex + 1 < DEPTH + IN && gx + 1 < w) dst[row + 1] = d1[j];
    }
}

__global__ void k_na_correct(NaField f, const NaState *st, const float *dlt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= f.w * f.h || st->done || f.held[i]) return;
    f.c[i] = fmax(f.c[i] + (double)dlt[i], 0.0);
}

int scratch_address(void **out) {
    int dev = 0;
    CW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cw::fail(CW_ERR_CUDA, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cw::cuda_fail(e, "cudaGetSymbolAddress(g_scratch)");
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return CW_OK;
}

}  // namespace

extern "C" int cw_field_relax_noalloc(double *values, const uint8_t *held, const double *lin_sink, const double *uptake,
                                      const double *production, uint32_t width, uint32_t height, double dcoef,
                                      double decay, double source, double omega, double tolerance,
                                      int64_t max_sweeps, int32_t inner_sweeps, int64_t *sweeps_out,
                                      double *residual_out) {
    if (!values || !held) return cw::fail(CW_ERR_CONFIG, "the values and the held mask are required");
    if (width == 0 || height == 0)
        return cw::fail(CW_ERR_CONFIG, "field dimensions must be positive, got " + std::to_string(width) + "x" +
                                           std::to_string(height));
    if ((int64_t)width * height > NA_MAX_PIXELS)
        return cw::fail(CW_ERR_CONFIG, "cw_field_relax_noalloc takes at most " + std::to_string(NA_MAX_PIXELS) +
                                           " pixels (its fixed scratch holds 1024 x 1024), got " +
                                           std::to_string(width) + "x" + std::to_string(height));
    if (!std::isfinite(dcoef) || !std::isfinite(decay) || dcoef < 0.0 || decay < 0.0)
        return cw::fail(CW_ERR_CONFIG, "diffusion and decay must be finite and not negative");
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != CW_OK) return rc;
    const int n = (int)(width * height);
    NaState *st = (NaState *)base;
    float *r32 = (float *)((char *)base + NA_RECORD);
    float *inv32 = r32 + NA_MAX_PIXELS;
    float *da = inv32 + NA_MAX_PIXELS;
    float *db = da + NA_MAX_PIXELS;
    if (omega <= 0.0) {  // the reference's rule for a flat field (pde.rs:275-276)
        double m = (double)(width > height ? width : height);
        omega = std::fmin(2.0 / (1.0 + std::sin(3.14159265358979323846 / m)), 1.95);
    }
    if (!(omega > 0.0 && omega < 2.0))
        return cw::fail(CW_ERR_CONFIG, "the relaxation factor must lie in (0, 2) (or be <= 0 for the rule), got " +
                                           std::to_string(omega));
    if (!(tolerance > 0.0 && tolerance < INFINITY))
        return cw::fail(CW_ERR_CONFIG, "the tolerance must be finite and above zero, got " + std::to_string(tolerance));
    const int inner = inner_sweeps > 0 ? inner_sweeps : 16;
    if (max_sweeps <= 0) max_sweeps = 1;
    NaField f{values, held, uptake, production, lin_sink, dcoef, decay, source, (int)width, (int)height};
    cudaStream_t s = cw::stream();
    if (s) {
        // the library stream is created on the device current at its first
        // use (or handed in by cw_set_stream): it must be this device's
        int dev = -1, sdev = -1;
        CW_CUDA(cudaGetDevice(&dev));
        CW_CUDA(cudaStreamGetDevice(s, &sdev));
        if (sdev != dev)
            return cw::fail(CW_ERR_CONFIG, "the library stream belongs to device " + std::to_string(sdev) +
                                               ", the current device is " + std::to_string(dev) +
                                               ": give this device's stream to cw_set_stream first");
    }
    NaState init{};
    CW_CUDA(cudaMemcpyAsync(st, &init, sizeof init, cudaMemcpyHostToDevice, s));
    const int T = 256, nb = (n + T - 1) / T;
    const int ntiles = (int)(((width + IN - 1) / IN) * ((height + IN - 1) / IN));
    NaState host{};
    bool first = true;
    for (int64_t outer = 0; outer < max_sweeps / inner + 2; ++outer) {
        k_na_residual<<<nb, T, 0, s>>>(f, st, r32, inv32, da, first ? 1 : 0);
        CW_LAUNCHED();
        first = false;
        k_na_check<<<1, 32, 0, s>>>(st, tolerance, inner, max_sweeps);
        CW_LAUNCHED();
        float *a = da, *b = db;
        int remaining = 2 * inner, half = 0;
        while (remaining > 0) {
            int dd = remaining < DEPTH ? remaining : DEPTH;
            k_na_sweep<<<ntiles, 256, 0, s>>>(a, b, r32, inv32, (int)width, (int)height, (float)omega, st, dd,
                                              half & 1, (float)dcoef);
            CW_LAUNCHED();
            remaining -= dd;
            half += dd;
            float *t = a; a = b; b = t;
        }
        k_na_correct<<<nb, T, 0, s>>>(f, st, a);
        CW_LAUNCHED();
        CW_CUDA(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s));
        CW_CUDA(cudaStreamSynchronize(s));
        if (host.done) break;
    }
    if (sweeps_out) *sweeps_out = host.inner;
    if (residual_out) *residual_out = host.last_resid;
    if (host.done != 1)
        return cw::fail(CW_ERR_SIMULATION, "diffusion did not settle within " + std::to_string(max_sweeps) +
                                               " sweeps at tolerance " + std::to_string(tolerance));
    return CW_OK;
}
