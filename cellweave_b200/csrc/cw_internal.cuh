// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/cellweave_b200.h"

namespace cw {

// ------------------------------------------------------------------ errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
cudaStream_t stream();
void count_launch(uint64_t n = 1);

// ------------------------------------------------------------------ streams and errors per handle
// Every handle queues its work on its own CUDA stream (created with it, or
// the stream of the handle that created it: a simulation's lattice and
// fields share the simulation's) and keeps the message of its last failure.
// A public entry point opens a Scope on its handle: stream() is then that
// stream, and a failure is recorded on the handle as well as on the calling
// thread.  A call that also reads another handle's buffers joins that
// handle's stream on entry and on exit (Join), so the two queues stay ordered.
struct HandleStream {
    cudaStream_t stream = nullptr;  // null: the library stream
    bool own = false;               // created for this handle (destroyed with it)
    std::string err;                // the last failure of a call on this handle
    int init(bool adopt = true);    // the current scope's stream (adopt), else a new one
    int set(cudaStream_t s);        // the caller's stream (null: a new one of its own)
    void release();
    HandleStream() = default;
    HandleStream(const HandleStream &) = delete;
    HandleStream &operator=(const HandleStream &) = delete;
    ~HandleStream() { release(); }
};
class Scope {
  public:
    explicit Scope(HandleStream *hs);
    ~Scope();
    Scope(const Scope &) = delete;
    Scope &operator=(const Scope &) = delete;

  private:
    cudaStream_t prev_stream_;
    std::string *prev_err_;
    bool prev_set_;
};
class Join {
  public:
    explicit Join(const HandleStream *other);
    ~Join();
    Join(const Join &) = delete;
    Join &operator=(const Join &) = delete;

  private:
    cudaStream_t mine_, other_;
};
#define CW_SCOPE(h) ::cw::Scope cw_scope_(&(h)->hs)
#define CW_JOIN(h) ::cw::Join cw_join_(&(h)->hs)

// Failure-test settings (cw_test_faults): all off by default.  wait_ns
// shortens every bounded device wait (grid barriers, TMA copies) from its
// 2 s; withhold_block keeps one block of a pass from arriving at its grid
// barriers; max_rounds caps a pass's priority rounds; skip_tma makes the
// FP32 sweep kernels issue no copy, so that their waits run out.
struct TestFaults {
    unsigned long long wait_ns = 0;
    int32_t withhold_block = -1;
    int32_t max_rounds = 0;
    int32_t skip_tma = 0;
};
const TestFaults &test_faults();

#define CW_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return ::cw::cuda_fail(e_, #call);          \
    } while (0)

#define CW_LAUNCHED()                                                      \
    do {                                                                   \
        ::cw::count_launch();                                              \
        cudaError_t e_ = cudaGetLastError();                               \
        if (e_ != cudaSuccess) return ::cw::cuda_fail(e_, "kernel launch"); \
    } while (0)

// ------------------------------------------------------------------ device memory
template <class T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    return CW_OK;
}
template <class T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

// ------------------------------------------------------------------ batch geometry
// Histories packed one after another in flat site order; each history's
// pixels keep the reference's order: x fastest, then y, then z.
struct Geom {
    uint32_t nh = 0;
    std::vector<int32_t> w, h, d;
    std::vector<int64_t> off;  // nh + 1
    int64_t total = 0;
    int4 *d_dims = nullptr;    // (w, h, d, 0) per history
    int64_t *d_off = nullptr;  // nh + 1
    int init(uint32_t n, const uint32_t *W, const uint32_t *H, const uint32_t *D);
    void release();
    int64_t sites(uint32_t k) const { return off[k + 1] - off[k]; }
    bool same(const Geom &o) const { return w == o.w && h == o.h && d == o.d; }
};

// Blocks of a launch distributed over histories: history k owns blocks
// [blk[k], blk[k+1]).  Built on the host from per-history item counts.
struct Plan {
    uint32_t nh = 0;
    int32_t nblocks = 0;
    std::vector<int32_t> blk;     // nh + 1
    std::vector<int32_t> table;   // what d_blk holds (kept for the asynchronous copy)
    std::vector<int64_t> items;   // per history
    int32_t *d_blk = nullptr;     // nh + 1 prefix entries, then the history of each of the nblocks blocks
    size_t cap = 0;               // entries allocated at d_blk
    int build(const std::vector<int64_t> &items_per_history, int threads);
    void release();
};

// The history of block b of a plan (Plan::build lays the table after the prefix).
__device__ __forceinline__ int plan_history(const int32_t *blk, int nh, int b) { return __ldg(blk + nh + 1 + b); }

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3"
// (SC'11): ten rounds of two 32x32->64 multiplies and a Weyl key schedule.
__host__ __device__ __forceinline__ uint4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                 uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32), lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}

// 53 random bits from two words as a double in [0, 1).
__host__ __device__ __forceinline__ double u01(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// exp(x) from + - * and a power-of-two scaling only, so that host and device
// round alike (the translation units that use it build without fused
// multiply-add): Cody-Waite reduction by ln 2 split into a 20-bit head and
// its tail, then a degree-17 Taylor polynomial of e^r, |r| <= ln2 / 2.
__host__ __device__ __forceinline__ double own_exp(double x) {
    if (!(x > -745.0)) return 0.0;
    if (x > 709.0) return HUGE_VAL;
    const double log2e = 1.4426950408889634;
    const double ln2_hi = 0.6931467056274414;
    const double ln2_lo = 4.7493250390316726e-07;
    double kf = floor(x * log2e + 0.5);
    double r = (x - kf * ln2_hi) - kf * ln2_lo;
    double p = 1.0 / 355687428096000.0;
    p = p * r + 1.0 / 20922789888000.0;
    p = p * r + 1.0 / 1307674368000.0;
    p = p * r + 1.0 / 87178291200.0;
    p = p * r + 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return ldexp(p, (int)kf);
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v) {
    if (!(v >= 0.0)) return;
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// The block's maximum of a non-negative v into *addr with one atomic (every
// thread of the block calls it; at most 1024 threads).  Many atomics per
// history on its one word would queue in L2.
__device__ __forceinline__ void block_max_to(unsigned long long *addr, double v) {
    __shared__ double s_part[32];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < ((blockDim.x + 31) >> 5) ? s_part[threadIdx.x] : 0.0;
        v = warp_max(v);
        if (threadIdx.x == 0 && v > 0.0) atomic_max_nonneg(addr, v);
    }
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ handles
struct Span {
    int32_t x0, x1, y0, y1, z0, z1;
    int32_t found, pad;
};

}  // namespace cw

namespace cw {
// Per-cell scratch of a division round (division.cu).
struct DivScratch {
    uint8_t *flag = nullptr;               // cells to divide
    double *normal = nullptr;              // 3 per cell: the plane's normal
    unsigned long long *sums = nullptr;    // 3 per cell: coordinate sums
    int32_t *npix = nullptr, *moved = nullptr, *daughter = nullptr;
    int32_t *count = nullptr;              // cells flagged: the passes skip all work at 0
    int64_t cap = 0;
    int ensure(int64_t ncells);
    void release();
};
}  // namespace cw

struct cw_lattice_s {
    cw::HandleStream hs;             // its stream and last error
    cw::Geom g;
    std::vector<int64_t> cell_off;   // nh + 1
    int64_t ncells = 0;              // all histories
    int32_t *grid = nullptr;
    int32_t *type = nullptr, *volume = nullptr, *target = nullptr;
    double *lambda = nullptr;
    int32_t *vsnap = nullptr;
    int32_t *surface = nullptr, *ssnap = nullptr, *tsurf = nullptr;
    double *lsurf = nullptr;
    bool surface_on = false;
    int64_t *d_cell_off = nullptr;
    int32_t K = 1;
    double J[64] = {0};
    int32_t order = 1;
    double temperature = 10.0;
    bool copy_moore = false;         // copies from any Chebyshev neighbour, not only across faces
    int32_t subsweeps = 1;           // sweeps of every colour a Monte Carlo step, each pixel in each with 1 / this
    uint32_t mcs = 0;
    std::vector<uint64_t> seed;
    uint2 *d_keys = nullptr;         // Philox key per history
    // the colouring: ncol colours of period `period` (0: the chessboard)
    int32_t ncol = 0, period = 0;
    int32_t nreach = 0;
    int8_t reach[3 * 124] = {0};
    double across = 1.0;
    int32_t *d_flag = nullptr;       // scratch flag / counters
    // scratch of the sublattice passes (lattice.cu): claims, pending lists, control words
    unsigned long long *claim = nullptr;  // 2 * ncells
    uint4 *plist = nullptr;               // plist_cap attempts of 3 uint4 (lattice.cu)
    uint32_t *pidx = nullptr;             // 2 * plist_cap pending-attempt indices
    int64_t plist_cap = 0;
    int32_t *d_vplan = nullptr;           // nh + 1: the pass plan (first chunk of each history)
    uint32_t *pctl = nullptr;             // control words, then 27 pass keys per history (lattice.cu)
    int pass_grid = 0;                    // blocks the device holds at once in a cooperative pass launch
    int pass_blocks = 0;                  // blocks of the pass launch
    int64_t pass_seg = 0;                 // attempts a block's segment holds
    // records in use per history (the medium's included): cw_cells_set raises
    // it, divisions advance it on the device
    std::vector<int32_t> used;
    int32_t *d_used = nullptr;
    cw::DivScratch div;
    cw::Plan site_plan;                   // every pixel of every history, T per block
    int32_t *stage = nullptr;             // uploads land here and are checked before they become the grid
    int32_t *d_span = nullptr;            // volumes: the occupied span of each history (x0 y0 z0 x1 y1 z1)
    unsigned long long *d_bad = nullptr;  // the first pixel of an upload past its history's capacity
    int32_t *bath_label = nullptr;        // the bath's union-find labels, one per site (bath.cu)
    uint8_t *bath_mark = nullptr;         // roots that reach the outer layer (bath.cu)
    int build_plans();
};

struct cw_field_s {
    cw::HandleStream hs;             // its stream and last error
    cw::Geom g;
    double *c = nullptr;             // values
    uint8_t *held = nullptr;
    double *uptake = nullptr, *production = nullptr, *lin_sink = nullptr;
    bool lin_sink_on = false, uptake_on = false, production_on = false;
    bool held_dirty = true;          // the span cache is stale
    bool floor = true;               // updates floored at zero (pde.rs:395); off for adjoint solves
    std::vector<cw::Span> spans;     // free_span of every history, cached
    double dcoef = 0.2, decay = 0.0, source = 0.0;
    // scratch of the FP32 defect-correction solve and the explicit step:
    // r32 = omega r / den, inv32 = omega D / den (the SOR's coefficients, 0 on
    // held pixels), d32a / d32b the correction, ping-ponged
    float *r32 = nullptr, *d32a = nullptr, *d32b = nullptr, *inv32 = nullptr;
    float *last_inner = nullptr;     // d32a or d32b: where cw_field_time_inner's correction is
    double *tmp64 = nullptr;
    void *stats = nullptr;           // per-history solve state (device)
    cw::Span *d_span = nullptr;
    void *dc_cache = nullptr;        // plans and solver of the FP32 solve (field.cu)
    cw_field_s *adjoint = nullptr;   // twin of cw_field_relax_adjoint, made on its first call
    cw::Plan inflow_plan;            // every site, for the inflow enqueued inside a step
    int alloc_fp32();
};

namespace cw {
// translation-unit entry points used across files
int field_span(cw_field_s *f, std::vector<Span> &spans);
int field_relax(cw_field_s *f, const cw_relax_opts *opts, const double *omega_h, cw_relax_stats *stats);
int field_relax_enqueue(cw_field_s *f, const cw_relax_opts *opts, int outer, float **start_out);
int field_relax_finish(cw_field_s *f, const cw_relax_opts *opts, float *start);
int field_dc_prepare(cw_field_s *f, int depth, int window, const std::vector<double> &omega);
int field_relax_collect(cw_field_s *f, std::vector<cw_relax_stats> &out, bool &all_settled);
int lattice_recount(cw_lattice_s *lat, int32_t *vol_out, int32_t *surf_out);
int lattice_sweep(cw_lattice_s *lat);
int lattice_subsweep(cw_lattice_s *lat);
int lattice_pass_error(cw_lattice_s *l);
int lattice_recount_surfaces(cw_lattice_s *l);  // surfaces from the grid into the records, no sync
int lattice_divide_enqueue(cw_lattice_s *l, const uint8_t *alive, int max_living, double *state, int S);
int lattice_span_enqueue(cw_lattice_s *l);  // volumes: the occupied span of the lattice as it stands, into d_span
int lattice_bath_enqueue(cw_lattice_s *l, uint8_t *bath);  // bath.cu: medium joined to the box's outer layer
int lattice_bath_error();
// debris.cu: the dead tissue's debris lost at its edge, the fluid shut in drained
struct DebrisState {
    uint8_t *kept = nullptr;   // per cell: dead, keeping the volume it died with
    int32_t *given = nullptr;  // per cell: pixels given up this step
    double *owed = nullptr;    // per history: pixels owed to the fluid, carried
    int64_t *held = nullptr;   // per history: what the kept dead hold
    int32_t *paid = nullptr, *edges = nullptr;  // per history, this step / this pass
    int32_t *active = nullptr; // per history: still owes this step (the passes skip the others whole)
    int32_t *claim = nullptr;  // per site: the cell taking it this pass (-1: none)
    int ensure(int64_t ncells, int nh, int64_t sites);
    void release();
};
int debris_break_down_enqueue(cw_lattice_s *l, DebrisState &D, double loss, int necrotic, const uint32_t *step);
int debris_drain_enqueue(cw_lattice_s *l, DebrisState &D, const uint8_t *bath, int necrotic, const uint32_t *step);
// field.cu: inflow (pde.rs:415-456) and free_count per history, added into inflow / free_count
int field_inflow_enqueue(cw_field_s *f, double *inflow, unsigned long long *free_count);
// coupling (coupling.cu), device-resident
int couple_uptake_device(cw_field_s *f, cw_lattice_s *l, const double *d_rate_by_type, int K, double *dst,
                         const Plan &p);
int couple_production_device(cw_field_s *f, cw_lattice_s *l, const double *d_per_cell, const Plan &p);
int couple_background_device(cw_field_s *f, cw_lattice_s *l, double rate, double *dst);
int couple_means_device(cw_field_s *f, cw_lattice_s *l, double *sum, int32_t *count, double *mean, const Plan &p);
}  // namespace cw

struct cw_network_s;
namespace cw {
// network (network.cu), device-resident, node-major state [S][stride]
int network_step_device(const cw_network_s *n, double *state, const double *inputs, int64_t ncells,
                        int64_t state_stride, int64_t input_stride, double dt, int substeps, const uint8_t *alive);
struct NetDev;
NetDev net_dev(const cw_network_s *n);
int network_step_clones_device(const NetDev *nets, const int32_t *clone, int S, double *state, const double *inputs,
                               int64_t ncells, int64_t state_stride, int64_t input_stride, double dt, int substeps,
                               const uint8_t *alive);
int network_mechanics_device(const cw_network_s *n, const double *state, int64_t ncells, int64_t stride,
                             uint32_t *target);
int32_t network_nodes(const cw_network_s *n);
double network_lambda(const cw_network_s *n);
int32_t network_role(const cw_network_s *n, int k);
uint32_t network_reference_volume(const cw_network_s *n);
const std::vector<double> &network_initial(const cw_network_s *n);
}  // namespace cw
