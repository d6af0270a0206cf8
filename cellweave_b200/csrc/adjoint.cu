// Differentiation of the frozen-geometry step: a hand-written adjoint of the
// steady field solves and of the RK4 network, for fitting the diffusion
// coefficient, the per-type uptake and network rates.  The reference has no
// adjoint, no loss and no autodiff; this is an extension on its model.
//
// Forward, on one history's lattice held fixed:
//   oxygen   A(D, k) c = b: D lap c - k_type c = 0, held where the lattice is
//            an obstacle (the vessel), relaxed by the field solver;
//   o_j      the mean of c over cell j (mean_per_cell, coupling.rs:164-182);
//   x_j(T)   T RK4 steps of the network with oxygen input o_j (network.rs:777),
//            checkpointed every K steps;
//   signal   A_s s = p, p = sigma x_j(T)[angiogenic] on cell j's pixels;
//   loss     L = sum_b (h_b - h*_b)^2 + w sum_b (g_b - g*_b)^2, with h_b the
//            fraction of bin b's cell pixels that are hypoxic, smoothed as
//            sigmoid((level - c) / tau), g_b their mean signal, bins by the
//            distance from the vessel column.
// Adjoint: A_s lam_s = dL/ds; dL/dx(T)[angio] = sigma sum_cell lam_s; reverse
// RK4 over each checkpointed segment (recomputed forward) gives dL/dtheta and
// dL/do_j; A lam = dL/dc (direct term + the means' share); then
// dL/dD = -lam . dA/dD c and dL/dk_t = -lam . dA/dk_t c.  A and A_s are
// symmetric, so each adjoint solve is the forward solver with another source
// (and no floor).  Gradient reductions are in FP64.
#include <cmath>
#include <cstring>

#include "cw_internal.cuh"
#include "field_kernels.cuh"
#include "network_kernels.cuh"

using namespace cw;

struct cw_fit_s {
    cw::HandleStream hs;  // its lattice's stream and its last error
    cw_lattice_s *lat = nullptr;
    cw_network_s *net = nullptr;
    cw_fit_config cfg;
    int64_t n = 0, nc = 0;
    int S = 0, ntheta = 0, angio = -1;
    cw_field_s *o2 = nullptr, *sig = nullptr, *ao2 = nullptr, *asig = nullptr;
    double Dc = 1.0, k[3] = {0, 0, 0};
    std::vector<double> theta, base_par_rate;
    int4 *term = nullptr;
    double4 *par = nullptr;
    double *d_rate = nullptr;
    double *sum = nullptr, *mean = nullptr, *sum2 = nullptr, *mean2 = nullptr, *inputs = nullptr;
    int32_t *count = nullptr, *count2 = nullptr;
    double *x0 = nullptr, *xT = nullptr, *lam = nullptr, *gin = nullptr, *ck = nullptr, *seg = nullptr;
    double *bins = nullptr;  // [3][nbins]: hypoxic sum, signal sum, cell pixels
    double *coef = nullptr;  // [2][nbins]: dL/dh_b / N_b, dL/dg_b / N_b
    double *grad = nullptr;  // [4 + ntheta]
    std::vector<double> target_h, target_g, h, g, cnt;
    Plan sites;
    // the frozen lattice's pixels listed by cell and by bin, in pixel order:
    // the means and the bins' sums are then taken in one fixed order, so that a
    // forward pass gives the same loss to the bit every time (central
    // differences of it resolve the smallest derivatives)
    int64_t *cell_ptr = nullptr, *bin_ptr = nullptr;
    int32_t *cell_px = nullptr, *bin_px = nullptr;
    bool forward_done = false;
};

namespace {

constexpr int T = 256;
constexpr int RB = 64;  // cells per block in the RK4 kernels
constexpr int MAXTH = 32;

NetDev fit_net(const cw_fit_s *f) { return NetDev{f->net->node_ptr, f->term, f->par, f->S, f->net->nterms}; }

__device__ __forceinline__ int bin_of(int x, int xc, double width, int nbins) {
    int b = (int)(fabs((double)(x - xc)) / width);
    return b < nbins ? b : nbins - 1;
}

__device__ __forceinline__ double sigmoid(double u) { return 1.0 / (1.0 + exp(-u)); }

__global__ void k_fit_inputs(const double *mean, int64_t nc, double egf, double *inputs) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    inputs[c] = mean[c];
    inputs[nc + c] = egf;
    for (int q = 2; q < 6; ++q) inputs[q * nc + c] = 0.0;
}

// One RK4 step of the thread's cell (rk4, network.rs:777-799) on shared
// columns x (in/out), with k and m as scratch: the same arithmetic as k_rk4_lanes.
__device__ void rk4_step(const NetDev &N, const int4 *sterm, const double4 *spar, const int32_t *sptr, double *x,
                         double *m, double *k, double *acc, const double *in, double dt) {
    const int S = N.S;
    derivatives(N, sterm, spar, sptr, x, in, k, RB);
    for (int i = 0; i < S; ++i) { acc[i * RB] = k[i * RB]; m[i * RB] = x[i * RB] + 0.5 * dt * k[i * RB]; }
    for (int stage = 1; stage < 4; ++stage) {
        derivatives(N, sterm, spar, sptr, m, in, k, RB);
        double step = stage < 2 ? 0.5 * dt : dt;
        for (int i = 0; i < S; ++i) {
            double kv = k[i * RB];
            if (stage < 3) { acc[i * RB] = acc[i * RB] + 2.0 * kv; m[i * RB] = x[i * RB] + step * kv; }
            else acc[i * RB] = acc[i * RB] + kv;
        }
    }
    for (int i = 0; i < S; ++i) x[i * RB] = fmin(fmax(x[i * RB] + (dt / 6.0) * acc[i * RB], 0.0), 1.0);
}

__device__ void load_net(const NetDev &N, int4 *sterm, double4 *spar, int32_t *sptr) {
    for (int t = threadIdx.x; t < N.nterms; t += blockDim.x) { sterm[t] = N.term[t]; spar[t] = N.par[t]; }
    for (int t = threadIdx.x; t <= N.S; t += blockDim.x) sptr[t] = N.node_ptr[t];
}

// Forward: T steps from the initial state, checkpoint every K steps.
__global__ void __launch_bounds__(RB) k_fit_forward(NetDev N, const double *x0, const double *inputs, int64_t nc,
                                                    int steps, int K, double dt, double *ck, double *xT) {
    extern __shared__ double sm[];
    const int S = N.S;
    double *x = sm, *m = sm + S * RB, *k = sm + 2 * S * RB, *acc = sm + 3 * S * RB;
    int4 *sterm = (int4 *)(sm + 4 * S * RB);
    double4 *spar = (double4 *)(sterm + N.nterms);
    int32_t *sptr = (int32_t *)(spar + N.nterms);
    load_net(N, sterm, spar, sptr);
    __syncthreads();
    int64_t c = (int64_t)blockIdx.x * RB + threadIdx.x;
    if (c >= nc) return;
    double in[6];
    for (int q = 0; q < 6; ++q) in[q] = inputs[q * nc + c];
    const int t = threadIdx.x;
    for (int i = 0; i < S; ++i) x[i * RB + t] = x0[i];
    for (int s = 0; s < steps; ++s) {
        if (s % K == 0)
            for (int i = 0; i < S; ++i) ck[((int64_t)(s / K) * S + i) * nc + c] = x[i * RB + t];
        rk4_step(N, sterm, spar, sptr, x + t, m + t, k + t, acc + t, in, dt);
    }
    for (int i = 0; i < S; ++i) xT[i * nc + c] = x[i * RB + t];
}

// Hill response and its slope in s (driver, network.rs:56-64).
__device__ __forceinline__ void hill_d(double s, double n, double half, double &v, double &dv) {
    if (s <= 0.0) { v = 0.0; dv = 0.0; return; }
    double sn, hn, dsn;
    if (n == 2.0) { sn = s * s; hn = half * half; dsn = 2.0 * s; }
    else { sn = pow(s, n); hn = pow(half, n); dsn = n * pow(s, n - 1.0); }
    double den = hn + sn;
    v = sn / den;
    dv = dsn * hn / (den * den);
}

// Vector-Jacobian product of the network's right-hand side at z with the
// adjoint a: adds a . df/dz to gx, a . df/dtheta (the first ntheta rates) to
// gth, and a . df/d(oxygen input) to *gin.  Columns have stride RB.
__device__ void vjp_f(const NetDev &N, const int4 *sterm, const double4 *spar, const int32_t *sptr, const double *z,
                      const double *in, const double *a, double *gx, double *gth, int ntheta, double &gin) {
    const int S = N.S;
    const double o2 = in[0];
    const double o2_slope = (o2 > 0.0 && o2 < 1.0) ? 1.0 : 0.0;  // read clamps oxygen to [0, 1]
    for (int i = 0; i < S; ++i) {
        const double ai = a[i * RB];
        if (ai == 0.0) continue;
        const double own = z[i * RB];
        for (int t = sptr[i]; t < sptr[i + 1]; ++t) {
            const int4 tm = sterm[t];
            const double4 p = spar[t];
            const double k = p.x;
            double s = 0.0, ds = 0.0;  // the source and d(read)/d(its variable)
            if (tm.x != CW_DECAYS && tm.x != CW_RELAXES_TO) {
                s = read_source(tm.y, in, z, RB);
                ds = tm.y >= 0 ? 1.0 : (tm.y == -1 ? o2_slope : 0.0);
            }
            double g_own = 0.0, g_s = 0.0, g_k = 0.0;
            switch (tm.x) {
            case CW_ACTIVATED_BY:
            case CW_INHIBITED_BY: {
                double drv = s, ddrv = 1.0;
                if (tm.z) hill_d(s, p.y, p.z, drv, ddrv);
                if (tm.x == CW_ACTIVATED_BY) { g_own = -k * drv; g_s = k * ddrv * (1.0 - own); g_k = drv * (1.0 - own); }
                else { g_own = -k * drv; g_s = -k * ddrv * own; g_k = -drv * own; }
                break;
            }
            case CW_ACTIVATED_BY_ABSENCE_OF: g_own = -k * (1.0 - s); g_s = -k * (1.0 - own); g_k = (1.0 - s) * (1.0 - own); break;
            case CW_PRODUCED_BY: g_s = k; g_k = s; break;
            case CW_DECAYS: g_own = -k; g_k = -own; break;
            case CW_RELAXES_TO: g_own = -k; g_k = -(own - p.w); break;
            case CW_DAMAGED_BELOW: {
                double u = (p.w - s) / p.w;
                if (u > 0.0) { g_s = k / p.w; g_k = -u; }
                break;
            }
            default: {
                double u = (s - p.w) / p.w;
                if (u > 0.0) { g_s = -k / p.w; g_k = -u; }
                break;
            }
            }
            gx[i * RB] += ai * g_own;
            if (tm.y >= 0 && tm.x != CW_DECAYS && tm.x != CW_RELAXES_TO) gx[tm.y * RB] += ai * g_s * ds;
            else if (tm.y == -1 && tm.x != CW_DECAYS && tm.x != CW_RELAXES_TO) gin += ai * g_s * ds;
            if (t < ntheta) gth[t * RB] += ai * g_k;
        }
    }
}

// Reverse RK4 over one checkpointed segment of K steps.  lam holds
// dL/dx at the segment's end on entry and at its start on return.
__global__ void __launch_bounds__(RB) k_fit_backward(NetDev N, const double *ckm, const double *inputs, int64_t nc,
                                                     int K, double dt, double *seg, double *lam, double *gin_out,
                                                     double *gth_out, int ntheta) {
    extern __shared__ double sm[];
    const int S = N.S;
    double *x = sm, *m = x + S * RB, *k1 = m + S * RB, *k2 = k1 + S * RB, *k3 = k2 + S * RB, *ln = k3 + S * RB;
    double *mu = ln + S * RB, *a = mu + S * RB, *gx = a + S * RB, *gth = gx + S * RB, *acc = gth + MAXTH * RB;
    int4 *sterm = (int4 *)(acc + S * RB);
    double4 *spar = (double4 *)(sterm + N.nterms);
    int32_t *sptr = (int32_t *)(spar + N.nterms);
    load_net(N, sterm, spar, sptr);
    const int t = threadIdx.x;
    for (int q = 0; q < ntheta; ++q) gth[q * RB + t] = 0.0;
    __syncthreads();
    int64_t c = (int64_t)blockIdx.x * RB + t;
    double gin = 0.0;
    if (c < nc) {
        double in[6];
        for (int q = 0; q < 6; ++q) in[q] = inputs[q * nc + c];
        double *X = x + t, *M = m + t, *K1 = k1 + t, *K2 = k2 + t, *K3 = k3 + t, *LN = ln + t, *MU = mu + t;
        double *A = a + t, *GX = gx + t, *G = gth + t, *ACC = acc + t;
        // recompute the segment's states
        for (int i = 0; i < S; ++i) { X[i * RB] = ckm[i * nc + c]; seg[(int64_t)i * nc + c] = X[i * RB]; }
        for (int s = 0; s < K; ++s) {
            rk4_step(N, sterm, spar, sptr, X, M, K1, ACC, in, dt);
            for (int i = 0; i < S; ++i) seg[((int64_t)(s + 1) * S + i) * nc + c] = X[i * RB];
        }
        for (int s = K - 1; s >= 0; --s) {
            for (int i = 0; i < S; ++i) X[i * RB] = seg[((int64_t)s * S + i) * nc + c];
            // forward stages of this step
            derivatives(N, sterm, spar, sptr, X, in, K1, RB);
            for (int i = 0; i < S; ++i) M[i * RB] = X[i * RB] + 0.5 * dt * K1[i * RB];
            derivatives(N, sterm, spar, sptr, M, in, K2, RB);
            for (int i = 0; i < S; ++i) M[i * RB] = X[i * RB] + 0.5 * dt * K2[i * RB];
            derivatives(N, sterm, spar, sptr, M, in, K3, RB);
            for (int i = 0; i < S; ++i) M[i * RB] = X[i * RB] + dt * K3[i * RB];
            derivatives(N, sterm, spar, sptr, M, in, GX, RB);  // k4 in GX for the moment
            for (int i = 0; i < S; ++i) {
                double y = X[i * RB] + (dt / 6.0) * (K1[i * RB] + 2.0 * K2[i * RB] + 2.0 * K3[i * RB] + GX[i * RB]);
                double l = lam[(int64_t)i * nc + c];
                MU[i * RB] = (y > 0.0 && y < 1.0) ? l : 0.0;  // the clamp to [0, 1]
                LN[i * RB] = MU[i * RB];                       // x_{t+1} = y: dy/dx = 1
            }
            // stage 4 at m3 = x + dt k3, adjoint mu dt/6
            for (int i = 0; i < S; ++i) { A[i * RB] = MU[i * RB] * (dt / 6.0); GX[i * RB] = 0.0; }
            vjp_f(N, sterm, spar, sptr, M, in, A, GX, G, ntheta, gin);
            for (int i = 0; i < S; ++i) { LN[i * RB] += GX[i * RB]; A[i * RB] = MU[i * RB] * (dt / 3.0) + dt * GX[i * RB]; }
            // stage 3 at m2 = x + dt/2 k2
            for (int i = 0; i < S; ++i) { M[i * RB] = X[i * RB] + 0.5 * dt * K2[i * RB]; GX[i * RB] = 0.0; }
            vjp_f(N, sterm, spar, sptr, M, in, A, GX, G, ntheta, gin);
            for (int i = 0; i < S; ++i) { LN[i * RB] += GX[i * RB]; A[i * RB] = MU[i * RB] * (dt / 3.0) + 0.5 * dt * GX[i * RB]; }
            // stage 2 at m1 = x + dt/2 k1
            for (int i = 0; i < S; ++i) { M[i * RB] = X[i * RB] + 0.5 * dt * K1[i * RB]; GX[i * RB] = 0.0; }
            vjp_f(N, sterm, spar, sptr, M, in, A, GX, G, ntheta, gin);
            for (int i = 0; i < S; ++i) { LN[i * RB] += GX[i * RB]; A[i * RB] = MU[i * RB] * (dt / 6.0) + 0.5 * dt * GX[i * RB]; }
            // stage 1 at x
            for (int i = 0; i < S; ++i) GX[i * RB] = 0.0;
            vjp_f(N, sterm, spar, sptr, X, in, A, GX, G, ntheta, gin);
            for (int i = 0; i < S; ++i) lam[(int64_t)i * nc + c] = LN[i * RB] + GX[i * RB];
        }
        gin_out[c] += gin;
    }
    // FP64 reduction of the rate gradients over the block's cells
    __syncthreads();
    for (int q = 0; q < ntheta; ++q) {
        double v = gth[q * RB + t];
        v = warp_sum(v);
        if ((t & 31) == 0 && v != 0.0) atomicAdd(gth_out + q, v);
    }
}

// Every cell's mean of `v` over its pixels (mean_per_cell, coupling.rs:164-182),
// summed in pixel order from the cell's pixel list; count: its pixels; sum
// (optional): the sum itself.
__global__ void k_fit_cell_means(const int64_t *ptr, const int32_t *px, int64_t nc, const double *v, double *mean,
                                 int32_t *count, double *sum_out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int64_t a = ptr[c], b = ptr[c + 1];
    double sum = 0.0;
    for (int64_t k = a; k < b; ++k) sum += v[px[k]];
    const int32_t n = (int32_t)(b - a);
    count[c] = n;
    mean[c] = n == 0 ? 0.0 : sum / (double)n;
    if (sum_out) sum_out[c] = sum;
}

// Bin statistics, one block per bin over the bin's cell pixels: hypoxic sum,
// signal sum and pixels, each a fixed-order tree sum.
constexpr int BIN_T = 256;
__global__ void __launch_bounds__(BIN_T) k_fit_bins_fixed(const int64_t *ptr, const int32_t *px, const double *c,
                                                         const double *s, int nbins, double level, double tau,
                                                         double *bins) {
    __shared__ double sh[BIN_T], sg[BIN_T];
    const int b = blockIdx.x;
    const int64_t a = ptr[b], e = ptr[b + 1];
    double h = 0.0, g = 0.0;
    for (int64_t k = a + threadIdx.x; k < e; k += BIN_T) {
        const int32_t i = px[k];
        h += sigmoid((level - c[i]) / tau);
        g += s[i];
    }
    sh[threadIdx.x] = h;
    sg[threadIdx.x] = g;
    __syncthreads();
    for (int w = BIN_T / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[threadIdx.x] += sh[threadIdx.x + w];
            sg[threadIdx.x] += sg[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bins[b] = sh[0];
        bins[nbins + b] = sg[0];
        bins[2 * nbins + b] = (double)(e - a);
    }
}

// Signal production p = sigma x(T)[angio] on the cell's pixels.
__global__ void k_fit_production(const int32_t *grid, int64_t n, const double *xT, int64_t nc, int angio, double sigma,
                                 double *prod) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t id = grid[i];
    prod[i] = (id > 0 && id < nc && angio >= 0) ? sigma * xT[(int64_t)angio * nc + id] : 0.0;
}

// dL/ds on cell pixels (the signal adjoint's source).
__global__ void k_fit_gs(const int32_t *grid, int W, int64_t n, int xc, double width, int nbins, const double *coef,
                         double *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = grid[i] > 0 ? coef[nbins + bin_of((int)(i % W), xc, width, nbins)] : 0.0;
}

// dL/dx(T): sigma times the cell's sum of the signal adjoint, on the angiogenic node.
__global__ void k_fit_lam_init(const double *sum_lam_s, int64_t nc, int S, int angio, double sigma, double *lam,
                               double *gin) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    for (int i = 0; i < S; ++i) lam[(int64_t)i * nc + c] = (i == angio && c > 0) ? sigma * sum_lam_s[c] : 0.0;
    gin[c] = 0.0;
}

// dL/dc on cell pixels: the hypoxic term and the cell mean's share of dL/do.
__global__ void k_fit_gc(const int32_t *grid, const double *c, int W, int64_t n, int64_t nc, int xc, double width,
                         int nbins, double level, double tau, const double *coef, const double *gin,
                         const int32_t *count, double *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t id = grid[i];
    double g = 0.0;
    if (id > 0) {
        double sg = sigmoid((level - c[i]) / tau);
        g = coef[bin_of((int)(i % W), xc, width, nbins)] * sg * (1.0 - sg) * (-1.0 / tau);
        if (id < nc && count[id] > 0) g += gin[id] / (double)count[id];
    }
    out[i] = g;
}

// dL/dD = -sum lam (real c - sum of neighbours), dL/dk_t = -sum lam c over type t.
__global__ void k_fit_param_grads(const double *lam, const double *c, const uint8_t *held, const int32_t *grid,
                                  const int32_t *type, int W, int H, int D, int64_t nc, double *grad) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t n = (int64_t)W * H * D;
    double gD = 0.0, gk[3] = {0.0, 0.0, 0.0};
    if (i < n && !held[i]) {
        int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((int64_t)W * H));
        double sum = 0.0, real = 0.0;
        int64_t slice = (int64_t)W * H;
        if (x > 0) { sum += c[i - 1]; real += 1.0; }
        if (x + 1 < W) { sum += c[i + 1]; real += 1.0; }
        if (y > 0) { sum += c[i - W]; real += 1.0; }
        if (y + 1 < H) { sum += c[i + W]; real += 1.0; }
        if (z > 0) { sum += c[i - slice]; real += 1.0; }
        if (z + 1 < D) { sum += c[i + slice]; real += 1.0; }
        gD = -lam[i] * (real * c[i] - sum);
        int32_t id = grid[i];
        if (id > 0 && id < nc) {
            int ty = type[id];
            if (ty >= 1 && ty <= 3) gk[ty - 1] = -lam[i] * c[i];
        }
    }
    gD = warp_sum(gD);
    for (int q = 0; q < 3; ++q) gk[q] = warp_sum(gk[q]);
    if ((threadIdx.x & 31) == 0) {
        if (gD != 0.0) atomicAdd(grad, gD);
        for (int q = 0; q < 3; ++q)
            if (gk[q] != 0.0) atomicAdd(grad + 1 + q, gk[q]);
    }
}

size_t fwd_smem(const cw_fit_s *f) {
    return sizeof(double) * 4 * f->S * RB + f->net->nterms * (sizeof(int4) + sizeof(double4)) +
           sizeof(int32_t) * (f->S + 1);
}
size_t bwd_smem(const cw_fit_s *f) {
    return sizeof(double) * (10 * f->S + MAXTH) * RB + f->net->nterms * (sizeof(int4) + sizeof(double4)) +
           sizeof(int32_t) * (f->S + 1);
}

int fit_relax(cw_fit_s *f, cw_field_s *fld, double tol) {
    cw_relax_opts o{};
    o.omega = f->cfg.omega;
    o.stop = CW_STOP_RESIDUAL;
    o.tolerance = tol;
    o.max_sweeps = 2000000;
    o.precision = f->cfg.precision;
    o.inner_sweeps = 32;
    o.block_depth = 8;
    return field_relax(fld, &o, nullptr, nullptr);
}

int blocks(int64_t n) { return (int)((n + T - 1) / T); }

}  // namespace

extern "C" {

int cw_fit_create(cw_lattice lat, cw_network net, const cw_fit_config *cfg, cw_fit *out) {
    CW_SCOPE(lat);  // the fit and its fields work on the lattice's stream
    *out = nullptr;
    if (lat->g.nh != 1) return fail(CW_ERR_CONFIG, "a fit takes a lattice of one history");
    if (cfg->steps <= 0 || cfg->checkpoint_every <= 0 || cfg->steps % cfg->checkpoint_every)
        return fail(CW_ERR_CONFIG, "the RK4 steps must be a positive multiple of the checkpoint interval");
    if (cfg->nbins <= 0 || cfg->nbins > 4096) return fail(CW_ERR_CONFIG, "1 to 4096 bins");
    cw_fit_s *f = new cw_fit_s();
    f->hs.init();
    f->lat = lat;
    f->net = net;
    f->cfg = *cfg;
    f->n = lat->g.total;
    f->nc = lat->ncells;
    f->S = net->S;
    f->angio = net->roles[5];
    f->ntheta = std::min(std::min(cfg->network_params, MAXTH), net->nterms);
    if (f->ntheta < 0) f->ntheta = 0;
    const uint32_t W = lat->g.w[0], H = lat->g.h[0], D = lat->g.d[0];
    int rc;
    if ((rc = cw_field_create(1, &W, &H, &D, cfg->dcoef, 0.0, 1.0, &f->o2)) ||
        (rc = cw_field_create(1, &W, &H, &D, cfg->signal_dcoef, cfg->signal_decay, 0.0, &f->sig)) ||
        (rc = cw_field_create(1, &W, &H, &D, cfg->dcoef, 0.0, 0.0, &f->ao2)) ||
        (rc = cw_field_create(1, &W, &H, &D, cfg->signal_dcoef, cfg->signal_decay, 0.0, &f->asig))) {
        cw_fit_destroy(f);
        return rc;
    }
    f->ao2->floor = false;
    f->asig->floor = false;
    // the vessel: the lattice's obstacle pixels hold the oxygen
    if ((rc = cw_couple_hold_obstacles(f->o2, lat, cfg->vessel_value)) ||
        (rc = cw_couple_hold_obstacles(f->ao2, lat, 0.0))) {
        cw_fit_destroy(f);
        return rc;
    }
    f->Dc = cfg->dcoef;
    for (int q = 0; q < 3; ++q) f->k[q] = cfg->uptake[q];
    std::vector<int4> tv(net->nterms);
    std::vector<double4> pv(net->nterms);
    if (net->nterms > 0) {
        CW_CUDA(cudaMemcpy(tv.data(), net->term, sizeof(int4) * net->nterms, cudaMemcpyDeviceToHost));
        CW_CUDA(cudaMemcpy(pv.data(), net->par, sizeof(double4) * net->nterms, cudaMemcpyDeviceToHost));
    }
    for (int t = 0; t < f->ntheta; ++t) f->theta.push_back(pv[t].x);
    int64_t nc = f->nc, S = f->S, M = cfg->steps / cfg->checkpoint_every;
    if ((rc = dalloc(&f->term, net->nterms)) || (rc = dalloc(&f->par, net->nterms)) || (rc = dalloc(&f->d_rate, 8)) ||
        (rc = dalloc(&f->sum, nc)) || (rc = dalloc(&f->mean, nc)) || (rc = dalloc(&f->sum2, nc)) ||
        (rc = dalloc(&f->mean2, nc)) || (rc = dalloc(&f->count, nc)) || (rc = dalloc(&f->count2, nc)) ||
        (rc = dalloc(&f->inputs, 6 * nc)) || (rc = dalloc(&f->x0, S)) || (rc = dalloc(&f->xT, S * nc)) ||
        (rc = dalloc(&f->lam, S * nc)) || (rc = dalloc(&f->gin, nc)) || (rc = dalloc(&f->ck, M * S * nc)) ||
        (rc = dalloc(&f->seg, (cfg->checkpoint_every + 1) * S * nc)) || (rc = dalloc(&f->bins, 3 * cfg->nbins)) ||
        (rc = dalloc(&f->coef, 2 * cfg->nbins)) || (rc = dalloc(&f->grad, 4 + MAXTH))) {
        cw_fit_destroy(f);
        return rc;
    }
    if (net->nterms > 0) {
        CW_CUDA(cudaMemcpy(f->term, tv.data(), sizeof(int4) * net->nterms, cudaMemcpyHostToDevice));
        CW_CUDA(cudaMemcpy(f->par, pv.data(), sizeof(double4) * net->nterms, cudaMemcpyHostToDevice));
    }
    CW_CUDA(cudaMemcpy(f->x0, net->initial.data(), sizeof(double) * S, cudaMemcpyHostToDevice));
    f->target_h.assign(cfg->nbins, 0.0);
    f->target_g.assign(cfg->nbins, 0.0);
    std::vector<int64_t> per(1, f->n);
    if ((rc = f->sites.build(per, T)) != CW_OK) { cw_fit_destroy(f); return rc; }
    {
        // pixel lists of the frozen lattice, by cell and by bin, in pixel order
        std::vector<int32_t> grid(f->n);
        CW_CUDA(cudaMemcpyAsync(grid.data(), lat->grid, sizeof(int32_t) * f->n, cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        const int nb = cfg->nbins;
        std::vector<int64_t> cp(nc + 1, 0), bp(nb + 1, 0);
        auto bin_of_host = [&](int64_t i) {
            int b = (int)(std::fabs((double)((int)(i % W) - cfg->vessel_x)) / cfg->bin_width);
            return b < nb ? b : nb - 1;
        };
        for (int64_t i = 0; i < f->n; ++i) {
            const int32_t id = grid[i];
            if (id > 0 && id < nc) cp[id + 1] += 1;
            if (id > 0) bp[bin_of_host(i) + 1] += 1;
        }
        for (int64_t c2 = 0; c2 < nc; ++c2) cp[c2 + 1] += cp[c2];
        for (int b = 0; b < nb; ++b) bp[b + 1] += bp[b];
        std::vector<int32_t> cpx(std::max<int64_t>(cp[nc], 1)), bpx(std::max<int64_t>(bp[nb], 1));
        std::vector<int64_t> cn(cp.begin(), cp.end() - 1), bn(bp.begin(), bp.end() - 1);
        for (int64_t i = 0; i < f->n; ++i) {
            const int32_t id = grid[i];
            if (id > 0 && id < nc) cpx[cn[id]++] = (int32_t)i;
            if (id > 0) bpx[bn[bin_of_host(i)]++] = (int32_t)i;
        }
        if ((rc = dalloc(&f->cell_ptr, nc + 1)) || (rc = dalloc(&f->bin_ptr, nb + 1)) ||
            (rc = dalloc(&f->cell_px, cpx.size())) || (rc = dalloc(&f->bin_px, bpx.size()))) {
            cw_fit_destroy(f);
            return rc;
        }
        CW_CUDA(cudaMemcpyAsync(f->cell_ptr, cp.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, stream()));
        CW_CUDA(cudaMemcpyAsync(f->bin_ptr, bp.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, stream()));
        CW_CUDA(cudaMemcpyAsync(f->cell_px, cpx.data(), sizeof(int32_t) * cpx.size(), cudaMemcpyHostToDevice,
                                stream()));
        CW_CUDA(cudaMemcpyAsync(f->bin_px, bpx.data(), sizeof(int32_t) * bpx.size(), cudaMemcpyHostToDevice,
                                stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
    }
    size_t sb = bwd_smem(f), sf = fwd_smem(f);
    if (sb > 48 * 1024 && cudaFuncSetAttribute(k_fit_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb))
        return fail(CW_ERR_CONFIG, "the network is too large for the adjoint's shared memory");
    if (sf > 48 * 1024 && cudaFuncSetAttribute(k_fit_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sf))
        return fail(CW_ERR_CONFIG, "the network is too large for the forward's shared memory");
    *out = f;
    return CW_OK;
}

int cw_fit_destroy(cw_fit f) {
    if (!f) return CW_OK;
    CW_SCOPE(f);
    cw_field_destroy(f->o2); cw_field_destroy(f->sig); cw_field_destroy(f->ao2); cw_field_destroy(f->asig);
    dfree(f->term); dfree(f->par); dfree(f->d_rate); dfree(f->sum); dfree(f->mean); dfree(f->sum2); dfree(f->mean2);
    dfree(f->count); dfree(f->count2); dfree(f->inputs); dfree(f->x0); dfree(f->xT); dfree(f->lam); dfree(f->gin);
    dfree(f->ck); dfree(f->seg); dfree(f->bins); dfree(f->coef); dfree(f->grad);
    dfree(f->cell_ptr); dfree(f->bin_ptr); dfree(f->cell_px); dfree(f->bin_px);
    f->sites.release();
    f->hs.release();
    delete f;
    return CW_OK;
}

const char *cw_fit_last_error(cw_fit f) { return f->hs.err.c_str(); }

int cw_fit_nparams(cw_fit f, int32_t *n) {
    CW_SCOPE(f);
    *n = 4 + f->ntheta;
    return CW_OK;
}

int cw_fit_get_params(cw_fit f, double *p) {
    CW_SCOPE(f);
    p[0] = f->Dc;
    for (int q = 0; q < 3; ++q) p[1 + q] = f->k[q];
    for (int t = 0; t < f->ntheta; ++t) p[4 + t] = f->theta[t];
    return CW_OK;
}

int cw_fit_set_params(cw_fit f, const double *p) {
    CW_SCOPE(f);
    if (!(p[0] > 0.0)) return fail(CW_ERR_CONFIG, "the diffusion coefficient must be positive");
    f->Dc = p[0];
    for (int q = 0; q < 3; ++q) f->k[q] = p[1 + q];
    for (int t = 0; t < f->ntheta; ++t) f->theta[t] = p[4 + t];
    f->forward_done = false;
    return CW_OK;
}

int cw_fit_set_target(cw_fit f, const double *h, const double *g) {
    CW_SCOPE(f);
    f->target_h.assign(h, h + f->cfg.nbins);
    f->target_g.assign(g, g + f->cfg.nbins);
    return CW_OK;
}

int cw_fit_forward(cw_fit f, double *loss, double *h_out, double *g_out) {
    CW_SCOPE(f);
    const cw_fit_config &c = f->cfg;
    const int nb = c.nbins;
    int rc;
    // parameters onto the device
    f->o2->dcoef = f->Dc;
    f->ao2->dcoef = f->Dc;
    double rate[8] = {0, f->k[0], f->k[1], f->k[2], 0, 0, 0, 0};
    CW_CUDA(cudaMemcpyAsync(f->d_rate, rate, sizeof rate, cudaMemcpyHostToDevice, stream()));
    for (int t = 0; t < f->ntheta; ++t)
        CW_CUDA(cudaMemcpyAsync((char *)(f->par + t), &f->theta[t], sizeof(double), cudaMemcpyHostToDevice, stream()));
    // oxygen
    if ((rc = couple_uptake_device(f->o2, f->lat, f->d_rate, 8, f->o2->lin_sink, f->sites)) != CW_OK) return rc;
    f->o2->lin_sink_on = true;
    if ((rc = fit_relax(f, f->o2, c.tolerance)) != CW_OK) return rc;
    k_fit_cell_means<<<blocks(f->nc), T, 0, stream()>>>(f->cell_ptr, f->cell_px, f->nc, f->o2->c, f->mean, f->count,
                                                        nullptr);
    CW_LAUNCHED();
    k_fit_inputs<<<blocks(f->nc), T, 0, stream()>>>(f->mean, f->nc, c.egf, f->inputs);
    CW_LAUNCHED();
    // the network, checkpointed
    NetDev N = fit_net(f);
    k_fit_forward<<<(unsigned)((f->nc + RB - 1) / RB), RB, fwd_smem(f), stream()>>>(
        N, f->x0, f->inputs, f->nc, c.steps, c.checkpoint_every, c.dt, f->ck, f->xT);
    CW_LAUNCHED();
    // the signal
    k_fit_production<<<blocks(f->n), T, 0, stream()>>>(f->lat->grid, f->n, f->xT, f->nc, f->angio, c.secretion,
                                                       f->sig->production);
    CW_LAUNCHED();
    f->sig->production_on = true;
    if ((rc = fit_relax(f, f->sig, c.tolerance)) != CW_OK) return rc;
    // profiles and the loss
    k_fit_bins_fixed<<<nb, BIN_T, 0, stream()>>>(f->bin_ptr, f->bin_px, f->o2->c, f->sig->c, nb, c.hypoxic_level,
                                                 c.tau, f->bins);
    CW_LAUNCHED();
    std::vector<double> hb(3 * nb);
    CW_CUDA(cudaMemcpyAsync(hb.data(), f->bins, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    f->h.assign(nb, 0.0);
    f->g.assign(nb, 0.0);
    f->cnt.assign(hb.begin() + 2 * nb, hb.end());
    double L = 0.0;
    for (int b = 0; b < nb; ++b) {
        if (f->cnt[b] <= 0) continue;
        f->h[b] = hb[b] / f->cnt[b];
        f->g[b] = hb[nb + b] / f->cnt[b];
        double dh = f->h[b] - f->target_h[b], dg = f->g[b] - f->target_g[b];
        L += dh * dh + c.signal_weight * dg * dg;
    }
    if (loss) *loss = L;
    if (h_out) std::memcpy(h_out, f->h.data(), sizeof(double) * nb);
    if (g_out) std::memcpy(g_out, f->g.data(), sizeof(double) * nb);
    f->forward_done = true;
    return CW_OK;
}

int cw_fit_gradient(cw_fit f, double *loss, double *grad) {
    CW_SCOPE(f);
    int rc;
    if ((rc = cw_fit_forward(f, loss, nullptr, nullptr)) != CW_OK) return rc;
    const cw_fit_config &c = f->cfg;
    const int nb = c.nbins;
    const int W = f->lat->g.w[0];
    // dL/dh_b / N_b and dL/dg_b / N_b
    std::vector<double> coef(2 * nb, 0.0);
    for (int b = 0; b < nb; ++b) {
        if (f->cnt[b] <= 0) continue;
        coef[b] = 2.0 * (f->h[b] - f->target_h[b]) / f->cnt[b];
        coef[nb + b] = 2.0 * c.signal_weight * (f->g[b] - f->target_g[b]) / f->cnt[b];
    }
    CW_CUDA(cudaMemcpyAsync(f->coef, coef.data(), sizeof(double) * 2 * nb, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemsetAsync(f->grad, 0, sizeof(double) * (4 + MAXTH), stream()));
    // signal adjoint
    k_fit_gs<<<blocks(f->n), T, 0, stream()>>>(f->lat->grid, W, f->n, c.vessel_x, c.bin_width, nb, f->coef,
                                               f->asig->production);
    CW_LAUNCHED();
    f->asig->production_on = true;
    if ((rc = fit_relax(f, f->asig, c.adjoint_tolerance)) != CW_OK) return rc;
    k_fit_cell_means<<<blocks(f->nc), T, 0, stream()>>>(f->cell_ptr, f->cell_px, f->nc, f->asig->c, f->mean2,
                                                        f->count2, f->sum2);
    CW_LAUNCHED();
    k_fit_lam_init<<<blocks(f->nc), T, 0, stream()>>>(f->sum2, f->nc, f->S, f->angio, c.secretion, f->lam, f->gin);
    CW_LAUNCHED();
    // reverse RK4, segment by segment
    NetDev N = fit_net(f);
    const int M = c.steps / c.checkpoint_every;
    for (int m = M - 1; m >= 0; --m) {
        k_fit_backward<<<(unsigned)((f->nc + RB - 1) / RB), RB, bwd_smem(f), stream()>>>(
            N, f->ck + (int64_t)m * f->S * f->nc, f->inputs, f->nc, c.checkpoint_every, c.dt, f->seg, f->lam, f->gin,
            f->grad + 4, f->ntheta);
        CW_LAUNCHED();
    }
    // oxygen adjoint
    k_fit_gc<<<blocks(f->n), T, 0, stream()>>>(f->lat->grid, f->o2->c, W, f->n, f->nc, c.vessel_x, c.bin_width, nb,
                                               c.hypoxic_level, c.tau, f->coef, f->gin, f->count, f->ao2->production);
    CW_LAUNCHED();
    f->ao2->production_on = true;
    CW_CUDA(cudaMemcpyAsync(f->ao2->lin_sink, f->o2->lin_sink, sizeof(double) * f->n, cudaMemcpyDeviceToDevice,
                            stream()));
    f->ao2->lin_sink_on = true;
    if ((rc = fit_relax(f, f->ao2, c.adjoint_tolerance)) != CW_OK) return rc;
    const int4 dm = make_int4(f->lat->g.w[0], f->lat->g.h[0], f->lat->g.d[0], 0);
    k_fit_param_grads<<<blocks(f->n), T, 0, stream()>>>(f->ao2->c, f->o2->c, f->o2->held, f->lat->grid, f->lat->type,
                                                        dm.x, dm.y, dm.z, f->nc, f->grad);
    CW_LAUNCHED();
    std::vector<double> g(4 + MAXTH);
    CW_CUDA(cudaMemcpyAsync(g.data(), f->grad, sizeof(double) * (4 + MAXTH), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    std::memcpy(grad, g.data(), sizeof(double) * (4 + f->ntheta));
    return CW_OK;
}

}  // extern "C"

extern "C" int cw_network_backward_batch(cw_network net, int64_t ncells, const double *state, const double *inputs,
                                         double dt, int32_t substeps, double *adjoint, double *d_oxygen,
                                         int32_t nrates, double *d_rates) {
    CW_SCOPE(net);
    if (ncells < 0 || substeps < 1 || !(dt > 0.0))
        return fail(CW_ERR_CONFIG, "a backward step needs cells >= 0, substeps >= 1 and dt > 0");
    if (nrates < 0 || nrates > std::min(MAXTH, net->nterms))
        return fail(CW_ERR_CONFIG, "rates to differentiate: 0 to " + std::to_string(std::min(MAXTH, net->nterms)));
    if (ncells == 0) {
        for (int32_t t = 0; t < nrates; ++t) d_rates[t] = 0.0;
        return CW_OK;
    }
    const int64_t nc = ncells, S = net->S;
    // cell-major host arrays to node-major device columns
    std::vector<double> xs(S * nc), in(6 * nc), lam(S * nc);
    for (int64_t c = 0; c < nc; ++c) {
        for (int64_t i = 0; i < S; ++i) {
            xs[i * nc + c] = state[c * S + i];
            lam[i * nc + c] = adjoint[c * S + i];
        }
        for (int q = 0; q < 6; ++q) in[q * nc + c] = inputs[c * 6 + q];
    }
    double *d_x = nullptr, *d_in = nullptr, *d_seg = nullptr, *d_lam = nullptr, *d_gin = nullptr, *d_gth = nullptr;
    auto release = [&]() { dfree(d_x); dfree(d_in); dfree(d_seg); dfree(d_lam); dfree(d_gin); dfree(d_gth); };
    int rc;
    if ((rc = dalloc(&d_x, S * nc)) || (rc = dalloc(&d_in, 6 * nc)) || (rc = dalloc(&d_seg, (substeps + 1) * S * nc)) ||
        (rc = dalloc(&d_lam, S * nc)) || (rc = dalloc(&d_gin, nc)) || (rc = dalloc(&d_gth, MAXTH))) {
        release();
        return rc;
    }
    CW_CUDA(cudaMemcpyAsync(d_x, xs.data(), sizeof(double) * S * nc, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(d_in, in.data(), sizeof(double) * 6 * nc, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemcpyAsync(d_lam, lam.data(), sizeof(double) * S * nc, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemsetAsync(d_gin, 0, sizeof(double) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(d_gth, 0, sizeof(double) * MAXTH, stream()));
    const size_t smem = sizeof(double) * (10 * S + MAXTH) * RB + net->nterms * (sizeof(int4) + sizeof(double4)) +
                        sizeof(int32_t) * (S + 1);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_fit_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        release();
        return fail(CW_ERR_CONFIG, "the network is too large for the backward step's shared memory");
    }
    NetDev N{net->node_ptr, net->term, net->par, net->S, net->nterms};
    k_fit_backward<<<(unsigned)((nc + RB - 1) / RB), RB, smem, stream()>>>(N, d_x, d_in, nc, substeps, dt, d_seg,
                                                                          d_lam, d_gin, d_gth, nrates);
    count_launch();
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) { release(); return cuda_fail(le, "kernel launch"); }
    std::vector<double> gin(nc), gth(MAXTH);
    CW_CUDA(cudaMemcpyAsync(lam.data(), d_lam, sizeof(double) * S * nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(gin.data(), d_gin, sizeof(double) * nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(gth.data(), d_gth, sizeof(double) * MAXTH, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    release();
    for (int64_t c = 0; c < nc; ++c)
        for (int64_t i = 0; i < S; ++i) adjoint[c * S + i] = lam[i * nc + c];
    if (d_oxygen)
        for (int64_t c = 0; c < nc; ++c) d_oxygen[c] = gin[c];
    for (int32_t t = 0; t < nrates; ++t) d_rates[t] = gth[t];
    return CW_OK;
}
