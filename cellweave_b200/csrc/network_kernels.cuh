// The compiled network and its device-side term evaluation, shared by the
// RK4 step (network.cu) and its adjoint (adjoint.cu).
#pragma once

#include <cmath>
#include <string>
#include <vector>

#include "cw_internal.cuh"

struct cw_network_s {
    cw::HandleStream hs;  // its stream and last error
    int32_t S = 0, nterms = 0;
    std::vector<std::string> names;
    std::vector<double> initial;
    int32_t roles[7] = {-1, -1, -1, -1, -1, -1, -1};
    double growth_coefficient = 0.0, lambda_volume = 0.0, max_target = NAN;
    uint32_t reference_volume = 0;
    // the compiled terms on the host (node_ptr, term, par below), for the
    // mutations that derive a network from this one
    std::vector<int32_t> h_ptr;
    std::vector<int4> h_term;
    std::vector<double4> h_par;
    // device copies of the compiled terms
    int32_t *node_ptr = nullptr;  // S + 1
    int4 *term = nullptr;         // (kind, source, has_hill, 0)
    double4 *par = nullptr;       // (rate, hill_n, hill_k, param)
};

namespace cw {

struct NetDev {
    const int32_t *node_ptr;
    const int4 *term;
    const double4 *par;
    int32_t S, nterms;
};

// read, network.rs:670-680.
__device__ __forceinline__ double read_source(int32_t src, const double *in, const double *st, int stride) {
    if (src >= 0) return st[src * stride];
    switch (-1 - src) {
    case 0: return fmin(fmax(in[0], 0.0), 1.0);
    case 1: return in[1];
    case 2: return fmin(fmax(in[2], 0.0), 1.0);
    case 3: return fmax(in[3], 0.0);
    case 4: return fmax(in[4], 0.0);
    default: return fmax(in[5], 0.0);
    }
}

// driver, network.rs:56-64.  A Hill exponent of exactly two is a square.
__device__ __forceinline__ double hill(double s, double n, double half) {
    double sp = fmax(s, 0.0);
    double sn, hn;
    if (n == 2.0) { sn = sp * sp; hn = half * half; }
    else { sn = pow(sp, n); hn = pow(half, n); }
    return sn / (hn + sn);
}

// derivatives + term_rate, network.rs:686-734, for the thread's cell.
// st/out point at node 0 of this thread's column (stride = threads).
__device__ __forceinline__ void derivatives(const NetDev &N, const int4 *sterm, const double4 *spar, const int32_t *sptr,
                            const double *st, const double *in, double *out, int stride) {
    for (int i = 0; i < N.S; ++i) {
        double own = st[i * stride], rate = 0.0;
        for (int t = sptr[i]; t < sptr[i + 1]; ++t) {
            int4 tm = sterm[t];
            double4 p = spar[t];
            double k = p.x, r;
            switch (tm.x) {
            case CW_ACTIVATED_BY: {
                double s = read_source(tm.y, in, st, stride);
                double drv = tm.z ? hill(s, p.y, p.z) : s;
                r = k * drv * (1.0 - own);
                break;
            }
            case CW_INHIBITED_BY: {
                double s = read_source(tm.y, in, st, stride);
                double drv = tm.z ? hill(s, p.y, p.z) : s;
                r = -k * drv * own;
                break;
            }
            case CW_ACTIVATED_BY_ABSENCE_OF:
                r = k * (1.0 - read_source(tm.y, in, st, stride)) * (1.0 - own);
                break;
            case CW_PRODUCED_BY: r = k * read_source(tm.y, in, st, stride); break;
            case CW_DECAYS: r = -k * own; break;
            case CW_RELAXES_TO: r = -k * (own - p.w); break;
            case CW_DAMAGED_BELOW: {
                double s = read_source(tm.y, in, st, stride);
                r = -k * fmax((p.w - s) / p.w, 0.0);
                break;
            }
            default: {
                double s = read_source(tm.y, in, st, stride);
                r = -k * fmax((s - p.w) / p.w, 0.0);
                break;
            }
            }
            rate += r;
        }
        out[i * stride] = rate;
    }
}

}  // namespace cw
