// Protein network: Network of crates/engine/src/network.rs on the device.
//
// Compilation (from_spec, network.rs:283-445) runs once on the host: names
// are resolved to indices, terms laid out per node in file order.  The RK4
// step (rk4, network.rs:777-799) runs one cell per thread when there are many
// cells (k_rk4: every cell of a launch walks the same term list, so a warp
// never diverges; state, midpoint, stage slope and accumulated slope in
// shared memory laid out [node][thread]), and a lane per node when there are
// few (k_rk4_lanes: 8, 16 or 32 lanes a cell, source nodes by shuffle).
// Built without fused multiply-add: the sums round as the reference's do.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>

#include "cw_internal.cuh"
#include "network_kernels.cuh"

using namespace cw;

namespace {

const char *INPUTS[6] = {"oxygen", "egf", "crowding", "stress", "waste", "necrotic_factor"};

constexpr int MAXS = 32;

constexpr int RT = 64;  // cells per block of the one-cell-per-thread kernels

// One cell's `substeps` RK4 steps (rk4, network.rs:777-799) on its column of
// the block's shared arrays (xs: state, ms: midpoint, ks: stage slope, as:
// accumulated slope, each [node][RT]), under the terms at sterm/spar/sptr.
__device__ __forceinline__ void rk4_cell(const NetDev &N, const int4 *sterm, const double4 *spar, const int32_t *sptr,
                                         double *xs, double *ms, double *ks, double *as, const double *in, double dt,
                                         int substeps) {
    const int S = N.S;
    for (int sub = 0; sub < substeps; ++sub) {
        // k1 at x
        derivatives(N, sterm, spar, sptr, xs, in, ks, RT);
        for (int i = 0; i < S; ++i) {
            double k1 = ks[i * RT];
            as[i * RT] = k1;
            ms[i * RT] = xs[i * RT] + 0.5 * dt * k1;
        }
        // k2 at x + dt/2 k1, k3 at x + dt/2 k2, k4 at x + dt k3
        for (int stage = 1; stage < 4; ++stage) {
            derivatives(N, sterm, spar, sptr, ms, in, ks, RT);
            double step = stage < 2 ? 0.5 * dt : dt;
            for (int i = 0; i < S; ++i) {
                double kv = ks[i * RT];
                if (stage < 3) {
                    as[i * RT] = as[i * RT] + 2.0 * kv;
                    ms[i * RT] = xs[i * RT] + step * kv;
                } else {
                    as[i * RT] = as[i * RT] + kv;
                }
            }
        }
        for (int i = 0; i < S; ++i) {
            double delta = (dt / 6.0) * as[i * RT];
            xs[i * RT] = fmin(fmax(xs[i * RT] + delta, 0.0), 1.0);
        }
    }
}

// state: [S][ncells] (node-major, coalesced); inputs: [6][ncells].
// alive (optional): cells whose entry is zero are left as they are.
__global__ void __launch_bounds__(RT) k_rk4(NetDev N, double *state, const double *inputs, int64_t ncells,
                                            int64_t state_stride, int64_t input_stride, double dt, int substeps,
                                            const uint8_t *alive) {
    extern __shared__ double sm[];
    const int S = N.S;
    double *x = sm, *mid = sm + S * RT, *kk = sm + 2 * S * RT, *acc = sm + 3 * S * RT;
    int4 *sterm = (int4 *)(sm + 4 * S * RT);
    double4 *spar = (double4 *)(sterm + N.nterms);
    int32_t *sptr = (int32_t *)(spar + N.nterms);
    for (int t = threadIdx.x; t < N.nterms; t += RT) { sterm[t] = N.term[t]; spar[t] = N.par[t]; }
    for (int t = threadIdx.x; t <= S; t += RT) sptr[t] = N.node_ptr[t];
    __syncthreads();
    int64_t c = (int64_t)blockIdx.x * RT + threadIdx.x;
    if (c >= ncells) return;
    if (alive && !alive[c]) return;
    const int tid = threadIdx.x;
    double in[6];
    for (int q = 0; q < 6; ++q) in[q] = inputs[q * input_stride + c];
    double *xs = x + tid, *ms = mid + tid, *ks = kk + tid, *as = acc + tid;
    for (int i = 0; i < S; ++i) xs[i * RT] = state[i * state_stride + c];
    rk4_cell(N, sterm, spar, sptr, xs, ms, ks, as, in, dt, substeps);
    for (int i = 0; i < S; ++i) state[i * state_stride + c] = xs[i * RT];
}

// The same for cells of many networks: cell c under nets[clone[c]], its
// terms read from global memory (a network's tables are a few KB: they stay
// in L1 across the block's cells of that network).
// state: [S][state_stride], inputs: [6][input_stride]; alive (optional):
// cells whose entry is zero are left as they are.
__global__ void __launch_bounds__(RT) k_rk4_clones(const NetDev *nets, const int32_t *clone, int S, double *state,
                                                   const double *inputs, int64_t ncells, int64_t state_stride,
                                                   int64_t input_stride, double dt, int substeps,
                                                   const uint8_t *alive) {
    extern __shared__ double sm[];
    double *x = sm, *mid = sm + S * RT, *kk = sm + 2 * S * RT, *acc = sm + 3 * S * RT;
    int64_t c = (int64_t)blockIdx.x * RT + threadIdx.x;
    if (c >= ncells) return;
    if (alive && !alive[c]) return;
    const NetDev N = nets[clone[c]];
    const int tid = threadIdx.x;
    double in[6];
    for (int q = 0; q < 6; ++q) in[q] = inputs[q * input_stride + c];
    double *xs = x + tid, *ms = mid + tid, *ks = kk + tid, *as = acc + tid;
    for (int i = 0; i < S; ++i) xs[i * RT] = state[i * state_stride + c];
    rk4_cell(N, N.term, N.par, N.node_ptr, xs, ms, ks, as, in, dt, substeps);
    for (int i = 0; i < S; ++i) state[i * state_stride + c] = xs[i * RT];
}

// RK4 with a lane per node (derivatives and term_rate, network.rs:686-734;
// rk4, 777-799): W lanes (W >= S, a power of two) hold one cell, lane i its
// node i's state, midpoint and accumulated slope in registers; a node's
// terms read their source nodes from the other lanes by shuffle.  A term
// loop runs to the most terms any node of the warp has, every lane taking
// part in each shuffle, and a lane adds its own node's terms in file order:
// the same operations in the same order as one cell per thread, to the bit.
// nets null: every cell under N; else cell c under nets[clone[c]].
template <int W>
__global__ void __launch_bounds__(128) k_rk4_lanes(NetDev N, const NetDev *nets, const int32_t *clone, double *state,
                                                   const double *inputs, int64_t ncells, int64_t state_stride,
                                                   int64_t input_stride, double dt, int substeps,
                                                   const uint8_t *alive) {
    const int lane = threadIdx.x & 31, node = lane % W, base = lane - node;
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / W;
    const bool cell = c < ncells;
    const NetDev M = (nets && cell) ? nets[clone[c]] : N;
    const int S = M.S;
    const bool live = cell && node < S && !(alive && !alive[c]);
    int p0 = 0, cnt = 0;
    if (cell && node < S) {
        p0 = M.node_ptr[node];
        cnt = M.node_ptr[node + 1] - p0;
    }
    int tmax = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tmax = max(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
    double in[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) in[q] = cell ? inputs[q * input_stride + c] : 0.0;
    double x = live ? state[node * state_stride + c] : 0.0;
    // the rate of this lane's node at the cell's values v (one value a lane)
    auto rate_of = [&](double own) -> double {
        double rate = 0.0;
        for (int t = 0; t < tmax; ++t) {
            const bool has = t < cnt;
            const int4 tm = has ? M.term[p0 + t] : make_int4(-1, -1, 0, 0);
            const int from = (has && tm.y >= 0 && tm.y < S) ? base + tm.y : lane;
            const double nodev = __shfl_sync(0xffffffffu, own, from);
            if (!has) continue;
            const double4 p = M.par[p0 + t];
            // read, network.rs:670-680
            double s = 0.0;
            if (tm.y >= 0) s = nodev;
            else switch (-1 - tm.y) {
                case 0: s = fmin(fmax(in[0], 0.0), 1.0); break;
                case 1: s = in[1]; break;
                case 2: s = fmin(fmax(in[2], 0.0), 1.0); break;
                case 3: s = fmax(in[3], 0.0); break;
                case 4: s = fmax(in[4], 0.0); break;
                default: s = fmax(in[5], 0.0); break;
                }
            const double k = p.x;
            double r;
            switch (tm.x) {
            case CW_ACTIVATED_BY: {
                const double drv = tm.z ? hill(s, p.y, p.z) : s;
                r = k * drv * (1.0 - own);
                break;
            }
            case CW_INHIBITED_BY: {
                const double drv = tm.z ? hill(s, p.y, p.z) : s;
                r = -k * drv * own;
                break;
            }
            case CW_ACTIVATED_BY_ABSENCE_OF: r = k * (1.0 - s) * (1.0 - own); break;
            case CW_PRODUCED_BY: r = k * s; break;
            case CW_DECAYS: r = -k * own; break;
            case CW_RELAXES_TO: r = -k * (own - p.w); break;
            case CW_DAMAGED_BELOW: r = -k * fmax((p.w - s) / p.w, 0.0); break;
            default: r = -k * fmax((s - p.w) / p.w, 0.0); break;
            }
            rate += r;
        }
        return rate;
    };
    for (int sub = 0; sub < substeps; ++sub) {
        // k1 at x
        double k1 = rate_of(x);
        double acc = k1;
        double mid = x + 0.5 * dt * k1;
        // k2 at x + dt/2 k1, k3 at x + dt/2 k2, k4 at x + dt k3
        for (int stage = 1; stage < 4; ++stage) {
            const double kv = rate_of(mid);
            const double step = stage < 2 ? 0.5 * dt : dt;
            if (stage < 3) {
                acc = acc + 2.0 * kv;
                mid = x + step * kv;
            } else {
                acc = acc + kv;
            }
        }
        const double delta = (dt / 6.0) * acc;
        x = fmin(fmax(x + delta, 0.0), 1.0);
    }
    if (live) state[node * state_stride + c] = x;
}

// Cells above this many take one thread each (the warps walk one term list
// together, no divergence); below it a lane per node puts more threads on
// the few cells (measured: 2,144 cells of 12 nodes 384 -> 178 us; 136,384
// cells of 8 nodes 521 -> 2,430 us with lanes, whose nodes diverge by term).
constexpr int64_t LANES_BELOW = 16384;

int rk4_lanes(const NetDev &N, const NetDev *nets, const int32_t *clone, int S, double *state, const double *inputs,
              int64_t ncells, int64_t state_stride, int64_t input_stride, double dt, int substeps,
              const uint8_t *alive, size_t cell_smem) {
    if (ncells >= LANES_BELOW) {
        const unsigned grid = (unsigned)((ncells + RT - 1) / RT);
        if (nets) {
            const size_t smem = sizeof(double) * 4 * S * RT;
            if (smem > 48 * 1024)
                CW_CUDA(cudaFuncSetAttribute(k_rk4_clones, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_rk4_clones<<<grid, RT, smem, stream()>>>(nets, clone, S, state, inputs, ncells, state_stride,
                                                       input_stride, dt, substeps, alive);
        } else {
            k_rk4<<<grid, RT, cell_smem, stream()>>>(N, state, inputs, ncells, state_stride, input_stride, dt, substeps,
                                                     alive);
        }
        CW_LAUNCHED();
        return CW_OK;
    }
    const int W = S <= 8 ? 8 : S <= 16 ? 16 : 32;
    const int64_t threads = ncells * W;
    const unsigned grid = (unsigned)((threads + 127) / 128);
    if (W == 8)
        k_rk4_lanes<8><<<grid, 128, 0, stream()>>>(N, nets, clone, state, inputs, ncells, state_stride, input_stride,
                                                   dt, substeps, alive);
    else if (W == 16)
        k_rk4_lanes<16><<<grid, 128, 0, stream()>>>(N, nets, clone, state, inputs, ncells, state_stride,
                                                    input_stride, dt, substeps, alive);
    else
        k_rk4_lanes<32><<<grid, 128, 0, stream()>>>(N, nets, clone, state, inputs, ncells, state_stride,
                                                    input_stride, dt, substeps, alive);
    CW_LAUNCHED();
    return CW_OK;
}

// mechanics, network.rs:811-821.
__global__ void k_mechanics(const double *state, int64_t ncells, int64_t stride, int growth, double coefficient,
                            double max_target, int has_max, uint32_t reference_volume, uint32_t *target) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    double g = state[growth * stride + c];
    double ratio = 1.0 + coefficient * g;
    if (has_max) ratio = fmin(ratio, max_target);
    double t = fmax((double)reference_volume * ratio, 0.0);
    target[c] = isnan(t) ? 0u : (t >= 4294967295.0 ? 4294967295u : (uint32_t)t);
}

size_t rk4_smem(const cw_network_s *n) {
    return sizeof(double) * 4 * n->S * RT + n->nterms * (sizeof(int4) + sizeof(double4)) + sizeof(int32_t) * (n->S + 1);
}

// The device copies of a network's host tables (h_ptr, h_term, h_par).
int network_upload(cw_network_s *n) {
    n->nterms = (int32_t)n->h_term.size();
    int rc;
    if ((rc = dalloc(&n->node_ptr, n->S + 1)) || (rc = dalloc(&n->term, n->nterms)) ||
        (rc = dalloc(&n->par, n->nterms)))
        return rc;
    CW_CUDA(cudaMemcpy(n->node_ptr, n->h_ptr.data(), sizeof(int32_t) * (n->S + 1), cudaMemcpyHostToDevice));
    if (n->nterms > 0) {
        CW_CUDA(cudaMemcpy(n->term, n->h_term.data(), sizeof(int4) * n->nterms, cudaMemcpyHostToDevice));
        CW_CUDA(cudaMemcpy(n->par, n->h_par.data(), sizeof(double4) * n->nterms, cudaMemcpyHostToDevice));
    }
    size_t smem = rk4_smem(n);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_rk4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(CW_ERR_CONFIG, "the network is too large for one block's shared memory");
    return CW_OK;
}

// A network like `n` with host tables to be changed and uploaded: every
// field but the device copies.
cw_network_s *network_derive(const cw_network_s *n) {
    cw_network_s *m = new cw_network_s();
    m->hs.init(false);
    m->S = n->S;
    m->names = n->names;
    m->initial = n->initial;
    std::memcpy(m->roles, n->roles, sizeof m->roles);
    m->growth_coefficient = n->growth_coefficient;
    m->lambda_volume = n->lambda_volume;
    m->max_target = n->max_target;
    m->reference_volume = n->reference_volume;
    m->h_ptr = n->h_ptr;
    m->h_term = n->h_term;
    m->h_par = n->h_par;
    return m;
}

// `(u * n as f64) as usize`, at most n - 1 (network.rs:488, 521): Rust's
// cast truncates and saturates (below zero and NaN give 0).
size_t pick_of(size_t n, double u) {
    if (n == 0) return 0;
    const double v = u * (double)n;
    if (!(v > 0.0)) return 0;
    if (v >= (double)n) return n - 1;
    return std::min<size_t>((size_t)v, n - 1);
}

// The node holding the term at global index t (terms in node order).
int node_of_term(const cw_network_s *n, int32_t t) {
    int i = 0;
    while (i + 1 < n->S && n->h_ptr[i + 1] <= t) ++i;
    return i;
}

constexpr double MUTATION_SPREAD = 2.0;  // network.rs:158
constexpr double GAINED_RATE = 0.1;      // network.rs:163
constexpr int REWIRED_INPUTS = 4;        // network.rs:169: oxygen, egf, crowding, stress

}  // namespace

namespace cw {
NetDev net_dev(const cw_network_s *n) { return NetDev{n->node_ptr, n->term, n->par, n->S, n->nterms}; }

// Device-side RK4 on node-major state (used by the simulation driver).
int network_step_device(const cw_network_s *n, double *state, const double *inputs, int64_t ncells,
                        int64_t state_stride, int64_t input_stride, double dt, int substeps, const uint8_t *alive) {
    if (ncells <= 0) return CW_OK;
    return rk4_lanes(net_dev(n), nullptr, nullptr, n->S, state, inputs, ncells, state_stride, input_stride, dt,
                     substeps, alive, rk4_smem(n));
}

// RK4 for cells of many networks on node-major state (the driver's evolving
// histories): cell c under nets[clone[c]], living cells only.
int network_step_clones_device(const NetDev *nets, const int32_t *clone, int S, double *state, const double *inputs,
                               int64_t ncells, int64_t state_stride, int64_t input_stride, double dt, int substeps,
                               const uint8_t *alive) {
    if (ncells <= 0) return CW_OK;
    NetDev none{};
    none.S = S;
    return rk4_lanes(none, nets, clone, S, state, inputs, ncells, state_stride, input_stride, dt, substeps, alive, 0);
}

int network_mechanics_device(const cw_network_s *n, const double *state, int64_t ncells, int64_t stride,
                             uint32_t *target) {
    if (ncells <= 0) return CW_OK;
    bool has = !std::isnan(n->max_target);
    k_mechanics<<<(unsigned)((ncells + 255) / 256), 256, 0, stream()>>>(state, ncells, stride, n->roles[0],
                                                                       n->growth_coefficient,
                                                                       has ? n->max_target : 0.0, has ? 1 : 0,
                                                                       n->reference_volume, target);
    CW_LAUNCHED();
    return CW_OK;
}
int32_t network_nodes(const cw_network_s *n) { return n->S; }
double network_lambda(const cw_network_s *n) { return n->lambda_volume; }
int32_t network_role(const cw_network_s *n, int k) { return n->roles[k]; }
uint32_t network_reference_volume(const cw_network_s *n) { return n->reference_volume; }
const std::vector<double> &network_initial(const cw_network_s *n) { return n->initial; }
}  // namespace cw

extern "C" {

int cw_network_compile(int32_t nnodes, const char *const *names, const double *initial, int32_t nterms,
                       const cw_term_spec *terms, const char *growth, const char *survival, const char *hypoxia,
                       const char *differentiation, const char *apoptosis, const char *angiogenic,
                       const char *evasion, double growth_coefficient, double lambda_volume, double max_target,
                       uint32_t reference_volume, cw_network *out) {
    *out = nullptr;
    if (nnodes <= 0) return fail(CW_ERR_CONFIG, "a network needs a node");
    if (nnodes > MAXS) return fail(CW_ERR_CONFIG, "at most " + std::to_string(MAXS) + " nodes");
    if (!growth || !survival || !hypoxia)
        return fail(CW_ERR_CONFIG,
                    "the network declares no roles, and inherits none: say which node is growth, which is survival, "
                    "and which is the hypoxia response");
    std::map<std::string, int> index;
    for (int i = 0; i < nnodes; ++i) {
        std::string nm = names[i];
        for (auto in : INPUTS)
            if (nm == in)
                return fail(CW_ERR_CONFIG, "node `" + nm +
                                               "` takes the name of an environment input; inputs are [\"oxygen\", "
                                               "\"egf\", \"crowding\", \"stress\", \"waste\", \"necrotic_factor\"]");
        if (!index.emplace(nm, i).second) return fail(CW_ERR_CONFIG, "two nodes are named `" + nm + "`");
    }
    auto resolve = [&](const char *name, const std::string &whose, int32_t *src) -> int {
        std::string nm = name ? name : "";
        for (int q = 0; q < 6; ++q)
            if (nm == INPUTS[q]) { *src = -1 - q; return CW_OK; }
        auto it = index.find(nm);
        if (it != index.end()) { *src = it->second; return CW_OK; }
        std::string known = "[\"oxygen\", \"egf\", \"crowding\", \"stress\", \"waste\", \"necrotic_factor\"";
        for (int i = 0; i < nnodes; ++i) known += std::string(", \"") + names[i] + "\"";
        return fail(CW_ERR_CONFIG, "node `" + whose + "` reads `" + nm +
                                       "`, which is neither a node nor an input; known names are " + known + "]");
    };
    std::vector<int32_t> ptr(nnodes + 1, 0);
    std::vector<int4> tv(nterms);
    std::vector<double4> pv(nterms);
    int prev = 0;
    for (int t = 0; t < nterms; ++t) {
        const cw_term_spec &s = terms[t];
        if (s.node < prev || s.node >= nnodes) return fail(CW_ERR_CONFIG, "terms must be listed in node order");
        prev = s.node;
        ptr[s.node + 1] += 1;
        std::string whose = names[s.node];
        if (s.kind < CW_ACTIVATED_BY || s.kind > CW_DAMAGED_ABOVE)
            return fail(CW_ERR_CONFIG, "node `" + whose + "` has an unknown kind of term");
        int32_t src = 0;
        bool reads = s.kind != CW_DECAYS && s.kind != CW_RELAXES_TO;
        if (reads) {
            int rc = resolve(s.source, whose, &src);
            if (rc != CW_OK) return rc;
        }
        int has_hill = 0;
        if ((s.kind == CW_ACTIVATED_BY || s.kind == CW_INHIBITED_BY) && s.has_hill) {
            if (s.hill_n <= 0.0 || s.hill_k <= 0.0)
                return fail(CW_ERR_CONFIG, "node `" + whose + "` has a Hill term with n = " + std::to_string(s.hill_n) +
                                               " and k = " + std::to_string(s.hill_k) + "; both must be positive");
            has_hill = 1;
        }
        if ((s.kind == CW_DAMAGED_BELOW || s.kind == CW_DAMAGED_ABOVE) && s.param <= 0.0)
            return fail(CW_ERR_CONFIG, "node `" + whose + "` is damaged " +
                                           (s.kind == CW_DAMAGED_BELOW ? "below " : "above ") +
                                           std::to_string(s.param) + ", which must be positive");
        tv[t] = make_int4(s.kind, src, has_hill, 0);
        pv[t] = make_double4(s.rate, has_hill ? s.hill_n : 0.0, has_hill ? s.hill_k : 0.0, s.param);
    }
    for (int i = 0; i < nnodes; ++i) ptr[i + 1] += ptr[i];
    cw_network_s *n = new cw_network_s();
    if (n->hs.init(false) != CW_OK) { delete n; return CW_ERR_CUDA; }
    auto role = [&](const char *name, const char *which, int32_t *dst) -> int {
        if (!name) { *dst = -1; return CW_OK; }
        auto it = index.find(name);
        if (it == index.end())
            return fail(CW_ERR_CONFIG, std::string("the ") + which + " role names `" + name + "`, which is not a node");
        *dst = it->second;
        return CW_OK;
    };
    const char *rn[7] = {growth, survival, hypoxia, differentiation, apoptosis, angiogenic, evasion};
    const char *rw[7] = {"growth", "survival", "hypoxia response", "differentiation", "apoptosis", "angiogenic",
                         "evasion"};
    for (int k = 0; k < 7; ++k) {
        int rc = role(rn[k], rw[k], &n->roles[k]);
        if (rc != CW_OK) { delete n; return rc; }
    }
    n->S = nnodes;
    n->nterms = nterms;
    for (int i = 0; i < nnodes; ++i) {
        n->names.push_back(names[i]);
        double v = initial ? initial[i] : 0.0;
        n->initial.push_back(std::fmin(std::fmax(v, 0.0), 1.0));
    }
    n->growth_coefficient = growth_coefficient;
    n->lambda_volume = lambda_volume;
    n->max_target = max_target;
    n->reference_volume = reference_volume;
    n->h_ptr = ptr;
    n->h_term = tv;
    n->h_par = pv;
    int rc = network_upload(n);
    if (rc != CW_OK) {
        cw_network_destroy(n);
        return rc;
    }
    *out = n;
    return CW_OK;
}

int cw_network_destroy(cw_network n) {
    if (!n) return CW_OK;
    CW_SCOPE(n);
    dfree(n->node_ptr); dfree(n->term); dfree(n->par);
    n->hs.release();
    delete n;
    return CW_OK;
}

int cw_network_set_stream(cw_network n, void *stream) {
    CW_SCOPE(n);
    return n->hs.set((cudaStream_t)stream);
}

void *cw_network_get_stream(cw_network n) { return (void *)n->hs.stream; }

const char *cw_network_last_error(cw_network n) { return n->hs.err.c_str(); }

int cw_network_info(cw_network n, int32_t *nnodes, int32_t *roles7, double *initial) {
    CW_SCOPE(n);
    if (nnodes) *nnodes = n->S;
    if (roles7) std::memcpy(roles7, n->roles, sizeof n->roles);
    if (initial) std::memcpy(initial, n->initial.data(), sizeof(double) * n->S);
    return CW_OK;
}

int cw_network_step_batch(cw_network n, int64_t ncells, double *state, const double *inputs, double dt,
                          int32_t substeps) {
    CW_SCOPE(n);
    if (ncells <= 0) return CW_OK;
    const int S = n->S;
    double *d_state, *d_in;
    int rc;
    if ((rc = dalloc(&d_state, (size_t)ncells * S)) || (rc = dalloc(&d_in, (size_t)ncells * 6))) return rc;
    // host rows are [cell][node]; the device works node-major
    std::vector<double> t((size_t)ncells * (S > 6 ? S : 6));
    for (int64_t c = 0; c < ncells; ++c)
        for (int i = 0; i < S; ++i) t[(size_t)i * ncells + c] = state[c * S + i];
    CW_CUDA(cudaMemcpyAsync(d_state, t.data(), sizeof(double) * ncells * S, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (int64_t c = 0; c < ncells; ++c)
        for (int q = 0; q < 6; ++q) t[(size_t)q * ncells + c] = inputs[c * 6 + q];
    CW_CUDA(cudaMemcpyAsync(d_in, t.data(), sizeof(double) * ncells * 6, cudaMemcpyHostToDevice, stream()));
    if ((rc = network_step_device(n, d_state, d_in, ncells, ncells, ncells, dt, substeps, nullptr)) != CW_OK)
        return rc;
    CW_CUDA(cudaMemcpyAsync(t.data(), d_state, sizeof(double) * ncells * S, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (int64_t c = 0; c < ncells; ++c)
        for (int i = 0; i < S; ++i) state[c * S + i] = t[(size_t)i * ncells + c];
    dfree(d_state);
    dfree(d_in);
    return CW_OK;
}

int cw_network_mechanics_batch(cw_network n, int64_t ncells, const double *state, uint32_t *target,
                               double *lambda) {
    CW_SCOPE(n);
    if (ncells <= 0) return CW_OK;
    const int S = n->S;
    double *d_state;
    uint32_t *d_t;
    int rc;
    if ((rc = dalloc(&d_state, (size_t)ncells * S)) || (rc = dalloc(&d_t, (size_t)ncells))) return rc;
    std::vector<double> t((size_t)ncells * S);
    for (int64_t c = 0; c < ncells; ++c)
        for (int i = 0; i < S; ++i) t[(size_t)i * ncells + c] = state[c * S + i];
    CW_CUDA(cudaMemcpyAsync(d_state, t.data(), sizeof(double) * ncells * S, cudaMemcpyHostToDevice, stream()));
    if ((rc = network_mechanics_device(n, d_state, ncells, ncells, d_t)) != CW_OK) return rc;
    CW_CUDA(cudaMemcpyAsync(target, d_t, sizeof(uint32_t) * ncells, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    if (lambda)
        for (int64_t c = 0; c < ncells; ++c) lambda[c] = n->lambda_volume;
    dfree(d_state);
    dfree(d_t);
    return CW_OK;
}

int cw_network_mutate(cw_network n, double which, double how, cw_network *out, cw_mutation *rec) {
    CW_SCOPE(n);
    if (!out) return fail(CW_ERR_CONFIG, "no place for the mutated network");
    *out = nullptr;
    const size_t count = n->h_term.size();
    if (count == 0) return fail(CW_ERR_NOT_FOUND, "a network without a single term has nothing a mutation could change");
    const int32_t pick = (int32_t)pick_of(count, which);
    const double factor = std::pow(MUTATION_SPREAD, 2.0 * how - 1.0);
    cw_network_s *m = network_derive(n);
    m->h_par[pick].x = m->h_par[pick].x * factor;
    const int node = node_of_term(n, pick);
    int rc = network_upload(m);
    if (rc != CW_OK) {
        cw_network_destroy(m);
        return rc;
    }
    if (rec) *rec = cw_mutation{node, pick - n->h_ptr[node], n->h_term[pick].x, CW_CHANGE_SCALED, factor, 0, 0};
    *out = m;
    return CW_OK;
}

int cw_network_rewire(cw_network n, const double draws[5], cw_network *out, cw_mutation *rec) {
    CW_SCOPE(n);
    if (!out || !draws) return fail(CW_ERR_CONFIG, "rewiring takes five draws and a place for the network");
    *out = nullptr;
    const double mode = draws[0], which = draws[1], source = draws[2], sign = draws[3], how = draws[4];
    cw_network_s *m = network_derive(n);
    cw_mutation r{};
    if (mode < 0.5) {
        // a gained link, the node's last term
        const int node = (int)pick_of((size_t)n->S, which);
        const int s = (int)pick_of((size_t)(REWIRED_INPUTS + n->S), source);
        const int32_t src = s < REWIRED_INPUTS ? -1 - s : s - REWIRED_INPUTS;
        const double rate = GAINED_RATE * std::pow(MUTATION_SPREAD, 2.0 * how - 1.0);
        const int32_t kind = sign < 0.5 ? CW_ACTIVATED_BY : CW_ACTIVATED_BY_ABSENCE_OF;
        const int32_t at = m->h_ptr[node + 1];
        m->h_term.insert(m->h_term.begin() + at, make_int4(kind, src, 0, 0));
        m->h_par.insert(m->h_par.begin() + at, make_double4(rate, 0.0, 0.0, 0.0));
        for (int i = node + 1; i <= n->S; ++i) m->h_ptr[i] += 1;
        r = cw_mutation{node, at - n->h_ptr[node], kind, CW_CHANGE_GAINED, rate, src, 0};
    } else {
        const size_t count = n->h_term.size();
        if (count == 0) {
            delete m;
            return fail(CW_ERR_NOT_FOUND, "a network without a single term has no term to lose");
        }
        const int32_t at = (int32_t)pick_of(count, which);
        const int node = node_of_term(n, at);
        r = cw_mutation{node, at - n->h_ptr[node], n->h_term[at].x, CW_CHANGE_LOST, 0.0, 0, 0};
        m->h_term.erase(m->h_term.begin() + at);
        m->h_par.erase(m->h_par.begin() + at);
        for (int i = node + 1; i <= n->S; ++i) m->h_ptr[i] -= 1;
    }
    int rc = network_upload(m);
    if (rc != CW_OK) {
        cw_network_destroy(m);
        return rc;
    }
    if (rec) *rec = r;
    *out = m;
    return CW_OK;
}

int cw_network_step_clones(int32_t nnets, const cw_network *nets, int64_t ncells, const int32_t *clone,
                           double *state, const double *inputs, double dt, int32_t substeps) {
    if (ncells <= 0) return CW_OK;
    if (nnets <= 0 || !nets) return fail(CW_ERR_CONFIG, "no networks to step the cells under");
    const int S = nets[0]->S;
    std::vector<NetDev> dev(nnets);
    for (int k = 0; k < nnets; ++k) {
        if (!nets[k] || nets[k]->S != S) return fail(CW_ERR_CONFIG, "every network of a batch has the same nodes");
        dev[k] = net_dev(nets[k]);
    }
    for (int64_t c = 0; c < ncells; ++c)
        if (clone[c] < 0 || clone[c] >= nnets)
            return fail(CW_ERR_CONFIG, "cell " + std::to_string(c) + " names network " + std::to_string(clone[c]) +
                                           " of " + std::to_string(nnets));
    NetDev *d_nets;
    int32_t *d_clone;
    double *d_state, *d_in;
    int rc;
    if ((rc = dalloc(&d_nets, (size_t)nnets)) || (rc = dalloc(&d_clone, (size_t)ncells)) ||
        (rc = dalloc(&d_state, (size_t)ncells * S)) || (rc = dalloc(&d_in, (size_t)ncells * 6)))
        return rc;
    std::vector<double> t((size_t)ncells * (S > 6 ? S : 6));
    for (int64_t c = 0; c < ncells; ++c)
        for (int i = 0; i < S; ++i) t[(size_t)i * ncells + c] = state[c * S + i];
    CW_CUDA(cudaMemcpy(d_state, t.data(), sizeof(double) * ncells * S, cudaMemcpyHostToDevice));
    for (int64_t c = 0; c < ncells; ++c)
        for (int q = 0; q < 6; ++q) t[(size_t)q * ncells + c] = inputs[c * 6 + q];
    CW_CUDA(cudaMemcpy(d_in, t.data(), sizeof(double) * ncells * 6, cudaMemcpyHostToDevice));
    CW_CUDA(cudaMemcpy(d_nets, dev.data(), sizeof(NetDev) * nnets, cudaMemcpyHostToDevice));
    CW_CUDA(cudaMemcpy(d_clone, clone, sizeof(int32_t) * ncells, cudaMemcpyHostToDevice));
    NetDev none{};
    none.S = S;
    if ((rc = rk4_lanes(none, d_nets, d_clone, S, d_state, d_in, ncells, ncells, ncells, dt, substeps, nullptr, 0)) !=
        CW_OK)
        return rc;
    CW_CUDA(cudaGetLastError());
    CW_CUDA(cudaMemcpyAsync(t.data(), d_state, sizeof(double) * ncells * S, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    for (int64_t c = 0; c < ncells; ++c)
        for (int i = 0; i < S; ++i) state[c * S + i] = t[(size_t)i * ncells + c];
    dfree(d_nets);
    dfree(d_clone);
    dfree(d_state);
    dfree(d_in);
    return CW_OK;
}

}  // extern "C"
