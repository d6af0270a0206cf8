// Simulation driver: Simulation<Running>::step (simulation.rs:1129-1350)
// reduced to the data-parallel hot path, device-resident, for a batch of
// independent histories (the campaign of src/campaign.rs:196-205 run as one
// batch instead of one history per CPU thread).
//
// Per lattice step: (1) every field is painted from the lattice and relaxed
// to its residual tolerance (declare_sources + relax); (2) every cell reads
// its field means (mean_per_cell); (3) every living network takes
// `substeps` RK4 steps; (4) survival below the threshold turns a cell
// necrotic, every other cell's mechanics set its target volume; (5) the
// lattice takes `sweeps` Monte Carlo steps.  Division, vessels, immune cells
// and the rest of the reference's biology are not part of this path.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <random>

#include "cw_internal.cuh"
#include "network_kernels.cuh"

using namespace cw;

struct cw_sim_s {
    cw::HandleStream hs;  // its stream (its lattice's and fields' too) and last error
    cw_sim_config cfg;
    std::vector<uint32_t> w, h, d, ncells;
    std::vector<uint64_t> obstacles;  // obstacle pixels seeded per history (a vessel's)
    std::vector<uint64_t> seeds;
    std::vector<double> J, sink;
    cw_lattice_s *lat = nullptr;
    cw_field_s *o2 = nullptr, *sig = nullptr;
    cw_field_s *wst = nullptr, *nfc = nullptr;  // the released fields: waste, necrotic factor
    double *cell_wst = nullptr, *cell_nfc = nullptr, *wst_rate = nullptr, *nfc_rate = nullptr;
    int32_t *died_at = nullptr;     // the step a cell turned necrotic (-1: not yet)
    int32_t *began = nullptr, *due = nullptr;  // a cell's cycle: the step it began and the step it is over
    cw_field_s *str = nullptr;      // the stress field of an exposure
    double *cell_str = nullptr, *d_str_uptake = nullptr;
    double str_level = 0.0;         // the level the stress field was last solved at
    std::vector<cw_relax_stats> last_str;
    cw::DebrisState debris;         // with a debris loss
    bool debris_on = false;
    double *level = nullptr;        // per history: the level the bath holds (1, or a still medium's)
    double *d_inflow = nullptr;     // per history: what the tissue takes up from the held pixels
    unsigned long long *d_free = nullptr;  // per history: the oxygen's free pixels
    uint32_t *d_step = nullptr;     // the step being taken, on the device
    uint8_t *bath = nullptr;        // the bath of the current lattice, one byte per site
    std::vector<cw_relax_stats> last_wst, last_nfc;
    cw_network_s *net = nullptr;
    double *d_sink = nullptr;       // 8 rates by type
    double *d_uptake = nullptr;     // 8 zero-order uptakes by type (the living types at o2_uptake)
    double *cell_o2 = nullptr, *cell_sig = nullptr, *sum = nullptr, *secretion = nullptr;
    int32_t *count = nullptr;
    double *state = nullptr, *inputs = nullptr;
    uint8_t *alive = nullptr;
    uint32_t *target32 = nullptr;
    int64_t nc = 0;                 // records over all histories
    // types that are no longer living (necrotic, differentiated, apoptotic), as bits
    uint32_t leaving = 0;
    // clones: tracked with mutation or a lineage; with mutation (evolve) every
    // clone also steps under its own network (0: the founding one, not owned;
    // a lineage's founders all share it)
    bool track = false;
    bool evolve = false;
    bool clone_nets = false;        // every cell steps under its clone's network (mutation or a lesion)
    std::vector<cw_network_s *> clones;
    std::vector<uint8_t> clone_owned;   // the simulation made it (a mutation), and destroys it
    std::vector<uint8_t> clone_lesion;  // a lesion's clone, or descended from one
    std::vector<int32_t> clone_parent;
    std::vector<cw_mutation> clone_mutation;
    // lineage tracing: every record's mark (-1: none), set at the marking
    // step and carried by daughters
    bool tracing = false;
    std::vector<int32_t> h_mark;
    // a lesion (Lesion, simulation.rs:348-360): its network (the caller's), the
    // step it appears at (-1: none), its radius and centre (NaN: the box's)
    cw_network_s *lesion_net = nullptr;
    int64_t lesion_at = -1;
    double lesion_radius = 0.0, lesion_cx = 0.0, lesion_cy = 0.0;
    std::vector<int32_t> h_clone;
    int32_t *d_clone = nullptr;
    cw::NetDev *d_nets = nullptr;
    size_t nets_cap = 0;
    Plan sites;
    std::vector<cw_relax_stats> last;
    uint32_t steps = 0;
    // autotuner: relaxation factor per history and field, blocking depth
    struct Tune {
        bool active = false;
        int steps = 0, done = 0;
        std::vector<double> cand;
        std::vector<int> cls, rank;             // class of each history, its index within the class
        int nclass = 0;
        std::vector<double> sum[2], cnt[2];     // [field][class * ncand + candidate]
    } tune;
    std::vector<double> omega[2];               // per history, per field
    int32_t depth = 8;
    bool depth_tuned = false;
    int sor_window = CW_WINDOW_AUTO;  // FP32 sweep windows, tuned with the depth
    // a step as three captured CUDA graphs (oxygen solve; means and signal
    // solve; network, fates and lattice), each solve with a fixed budget of
    // outer iterations checked, and finished host-side if ever short
    cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};
    uint64_t gkernels[3] = {0, 0, 0};
    bool graphs = false;
    int budget[2] = {0, 0};
    float *gstart[2] = {nullptr, nullptr};
    std::vector<cw_relax_stats> last_sig;
    uint64_t graph_steps = 0, budget_misses = 0;
    int need[2] = {0, 0};        // most outer iterations a solve needed over the current window
    int window = 0;              // graph steps in the window
};

extern "C" {
static void tune_begin(cw_sim_s *s);
static int upload_clones(cw_sim_s *s, bool tables);
static void drop_graphs(cw_sim_s *s);
}

namespace {

constexpr int T = 256;

// A cell's inputs (cell_inputs, simulation.rs:2511-2527): its mean oxygen,
// EGF everywhere the same, crowding 1 - volume / reference volume clamped to
// [0, 1]; no stress, waste or necrotic factor on this path.
__global__ void k_inputs(const int32_t *type, const int32_t *volume, const int64_t *cell_off, int nh, int64_t nc,
                         uint32_t leaving, const double *cell_o2, double egf, double reference, double *inputs,
                         uint8_t *alive) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    // the medium slot of every history is not a cell
    int lo = 0, hi = nh - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
    bool medium = c == cell_off[lo];
    bool a = !medium && volume[c] > 0 && !((leaving >> (type[c] & 31)) & 1u);
    alive[c] = a;
    inputs[0 * nc + c] = cell_o2[c];
    inputs[1 * nc + c] = egf;
    inputs[2 * nc + c] = a ? fmin(fmax(1.0 - (double)volume[c] / reference, 0.0), 1.0) : 0.0;
    inputs[3 * nc + c] = 0.0;
    inputs[4 * nc + c] = 0.0;
    inputs[5 * nc + c] = 0.0;
}

// What each cell releases into the released fields this step
// (settle_released, simulation.rs:2546-2570): a living cell's pixels the
// waste's production; a necrotic cell's the factor's, for `release_for`
// steps after the one it died at (for as long as it is there when < 0).
__global__ void k_release_rates(const uint8_t *alive, const int32_t *type, const int32_t *volume,
                                const int32_t *died_at, const uint32_t *step, int64_t nc, int necrotic,
                                double waste, double factor, int release_for, double *wst_rate, double *nfc_rate) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    if (wst_rate) wst_rate[c] = alive[c] ? waste : 0.0;
    if (nfc_rate) {
        const bool dead = necrotic >= 0 && type[c] == necrotic && volume[c] > 0;
        const bool releasing = release_for < 0 || died_at[c] < 0 || (int64_t)*step <= (int64_t)died_at[c] + release_for;
        nfc_rate[c] = dead && releasing ? factor : 0.0;
    }
}

// The cells' waste and necrotic-factor inputs (cell_inputs, simulation.rs:2511-2521).
__global__ void k_inputs_stress(const double *cell_str, int64_t nc, double *inputs) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    inputs[3 * nc + c] = cell_str ? cell_str[c] : 0.0;
}

// A field held where `src` is held, at `level` (the stress where the oxygen
// comes in: hold_medium_bath or hold_vessels_at at the exposure's level).
__global__ void k_hold_like(const uint8_t *src, int64_t n, double level, uint8_t *held, double *c) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t m = src[i];
    held[i] = m;
    if (m) c[i] = level;
}

__global__ void k_inputs_released(const double *cell_wst, const double *cell_nfc, int64_t nc, double *inputs) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    if (cell_wst) inputs[4 * nc + c] = cell_wst[c];
    if (cell_nfc) inputs[5 * nc + c] = cell_nfc[c];
}

// A field held exactly on `mask` at `value` (release_all, then hold_bath_at),
// or, given `level`, at its history's level (off: the histories' sites).
__global__ void k_hold_from_mask(const uint8_t *mask, int64_t n, double value, uint8_t *held, double *c,
                                 const double *level = nullptr, const int64_t *off = nullptr, int nh = 0) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t m = mask[i];
    held[i] = m;
    if (!m) return;
    if (level) {
        int lo = 0, hi = nh - 1;
        while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (off[mid] <= i) lo = mid; else hi = mid - 1; }
        value = level[lo];
    }
    c[i] = value;
}

// settle_bath_level (simulation.rs:2114-2125): a still medium of diffusion
// `dm` around the tissue holds 1 - inflow / (4 pi dm r), r the radius of a
// ball of the free pixels, at zero at least.
__global__ void k_bath_level(int nh, const double *inflow, const unsigned long long *free_count, double dm,
                             double *level) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const double four_pi = 4.0 * 3.141592653589793;
    const double r = cbrt(3.0 * (double)free_count[h] / four_pi);
    level[h] = r > 0.0 ? fmax(1.0 - inflow[h] / (four_pi * dm * r), 0.0) : 1.0;
}

__global__ void k_step_advance(uint32_t *step) { *step += 1u; }

// A cell on the box's sides (and faces, with `faces`) of each history.
__global__ void k_touches_edge(const int32_t *grid, const int4 *dims, const int64_t *off, int nh, int faces,
                               int32_t *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= off[nh] || grid[i] <= 0) return;
    int lo = 0, hi = nh - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (off[mid] <= i) lo = mid; else hi = mid - 1; }
    const int4 dm = dims[lo];
    const int64_t local = i - off[lo], slice = (int64_t)dm.x * dm.y;
    const int z = (int)(local / slice);
    const int64_t r = local - (int64_t)z * slice;
    const int y = (int)(r / dm.x), x = (int)(r - (int64_t)y * dm.x);
    const bool side = x == 0 || x == dm.x - 1 || y == 0 || y == dm.y - 1;
    const bool face = faces && dm.z > 1 && (z == 0 || z == dm.z - 1);
    if (side || face) out[lo] = 1;
}

__global__ void k_secretion(const uint8_t *alive, const double *cell_o2, int64_t nc, double level, double rate,
                            double *secretion) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) secretion[c] = (alive[c] && cell_o2[c] < level) ? rate : 0.0;
}

constexpr int32_t RESORPTION_RATE = 2;    // pixels a necrotic cell gives up a step (simulation.rs:127)
constexpr int32_t SHEDDING_RATE = 6;      // a differentiated cell leaving the layer (simulation.rs:135)
constexpr int32_t FRAGMENTATION_RATE = 8; // an apoptotic cell breaking up (simulation.rs:142)
constexpr double DIVISION_RATIO = 1.4;    // of the reference volume (simulation.rs:45)
constexpr double QUIESCENCE_THRESHOLD = 0.45;  // hypoxia response that stops cycling (simulation.rs:117)
constexpr int DEFAULT_MAX_CELLS = 2000;   // simulation.rs:61

// Measure::measure's counts per history (measure.rs:133-170): one block a
// history over its records; out[8 h ..] = cycling, quiescent, necrotic,
// living area, necrotic area, born, gone, lines holding living pixels.
// out[MEASURES h ..]: cycling, quiescent, necrotic, living area, necrotic
// area, born, gone, lines holding living pixels, differentiating, apoptotic,
// leaving area (measure.rs:115-170).
constexpr int MEASURES = 12;
__global__ void k_measure(const int32_t *type, const int32_t *volume, const int64_t *cell_off, const int32_t *used,
                          int necrotic, int differentiated, int apoptotic, const double *state, int hyp, int64_t nc,
                          const uint8_t *lines, const int64_t *line_off, unsigned long long *out) {
    const int h = blockIdx.x;
    __shared__ unsigned long long acc[MEASURES];
    if (threadIdx.x < MEASURES) acc[threadIdx.x] = 0ull;
    __syncthreads();
    const int64_t c0 = cell_off[h];
    const int32_t n = used[h];
    unsigned long long v[MEASURES] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t k = 1 + threadIdx.x; k < n; k += blockDim.x) {
        const int64_t c = c0 + k;
        const int32_t vol = volume[c];
        const bool dead = necrotic >= 0 && type[c] == necrotic;
        const bool diff = differentiated >= 0 && type[c] == differentiated;
        const bool apop = apoptotic >= 0 && type[c] == apoptotic;
        if (vol == 0) {
            if (dead || diff || apop) v[6] += 1;  // resorbed, shed or broken up: gone for good
            continue;
        }
        if (diff || apop) {
            v[diff ? 8 : 9] += 1;
            v[10] += (unsigned long long)vol;
        } else if (dead) {
            v[2] += 1;
            v[4] += (unsigned long long)vol;
        } else {
            if (hyp < 0 || state[(int64_t)hyp * nc + c] < QUIESCENCE_THRESHOLD) v[0] += 1;
            else v[1] += 1;
            v[3] += (unsigned long long)vol;
        }
    }
    if (lines)
        for (int64_t q = line_off[h] + threadIdx.x; q < line_off[h + 1]; q += blockDim.x) v[7] += lines[q];
    for (int j = 0; j < MEASURES; ++j)
        if (v[j]) atomicAdd(&acc[j], v[j]);
    __syncthreads();
    if (threadIdx.x < MEASURES) out[MEASURES * h + threadIdx.x] = acc[threadIdx.x];
    if (threadIdx.x == 0) out[MEASURES * h + 5] = (unsigned long long)(n - 1);
}

// The columns (by_row 0) or rows (1) of each history that hold a living pixel.
__global__ void k_measure_lines(const int32_t *grid, const int32_t *type, const int32_t *volume,
                                const int64_t *cell_off, const int4 *dims, const int64_t *off, const int32_t *blk,
                                int nh, int necrotic, int by_row, const int64_t *line_off, uint8_t *lines) {
    const int h = plan_history(blk, nh, blockIdx.x);
    const int4 dm = dims[h];
    const int64_t local = (int64_t)(blockIdx.x - blk[h]) * blockDim.x + threadIdx.x;
    if (local >= off[h + 1] - off[h]) return;
    const int32_t id = grid[off[h] + local];
    if (id <= 0) return;
    const int64_t c = cell_off[h] + id;
    if (volume[c] <= 0 || (necrotic >= 0 && type[c] == necrotic)) return;
    const int x = (int)(local % dm.x), y = (int)((local / dm.x) % dm.y);
    lines[line_off[h] + (by_row ? y : x)] = 1;
}

// Fate and upward coupling (simulation.rs:1212-1309, the necrosis and
// mechanics branches): a necrotic cell gives up RESORPTION_RATE pixels a step
// until it is gone; survival below the threshold makes a living cell
// necrotic; every other living cell takes the target its mechanics give.
// With a cycle (simulation.rs:1301-1304) the target is grown(): half the
// network's target when the cycle begins, all of it when it is over.
// Cells leaving the layer or breaking up (simulation.rs:1209-1296): a cell
// committed to differentiate sheds SHEDDING_RATE pixels a step, one in
// apoptosis FRAGMENTATION_RATE, until gone; a living cell whose network has the
// apoptosis (or else the differentiation) node commits with that node's level
// as its chance this step, drawn from Philox(record, step, 9 / 10, 0) under its
// history's key.
struct Leaving {
    int32_t differentiated, apoptotic;  // types, -1: none
    int32_t role_diff, role_apop;       // network nodes, -1: none
    const uint2 *keys;
    const int64_t *cell_off;
    int32_t nh;
};

__global__ void k_fates(const uint8_t *alive, const double *state, int64_t nc, int survival, double death,
                        int necrotic, const uint32_t *mech_target, int32_t *type, const int32_t *volume,
                        int32_t *target, double *lambda, double lam, int32_t *died_at, const uint32_t *step,
                        const int32_t *began, const int32_t *due, uint8_t *kept, Leaving lv) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    if ((lv.differentiated >= 0 && type[c] == lv.differentiated) || (lv.apoptotic >= 0 && type[c] == lv.apoptotic)) {
        const int32_t v = volume[c];
        const int32_t rate = type[c] == lv.apoptotic ? FRAGMENTATION_RATE : SHEDDING_RATE;
        if (v > 0) {
            target[c] = v > rate ? v - rate : 0;
            lambda[c] = lam;
        }
        return;
    }
    if (necrotic >= 0 && type[c] == necrotic) {
        const int32_t v = volume[c];
        if (v > 0 && kept) {
            // with a debris loss the dead keep what they held (simulation.rs:1226-1244)
            if (!kept[c]) { kept[c] = 1; target[c] = v; lambda[c] = lam; }
        } else if (v > 0) {
            target[c] = v > RESORPTION_RATE ? v - RESORPTION_RATE : 0;
            lambda[c] = lam;
        }
        return;
    }
    if (!alive[c]) return;
    if (necrotic >= 0 && state[survival * nc + c] < death) {
        type[c] = necrotic;
        if (died_at) died_at[c] = (int32_t)*step;
        if (kept) { kept[c] = 1; target[c] = volume[c]; lambda[c] = lam; }  // simulation.rs:1264-1275
        return;
    }
    if ((lv.apoptotic >= 0 && lv.role_apop >= 0) || (lv.differentiated >= 0 && lv.role_diff >= 0)) {
        int lo = 0, hi = lv.nh - 1;
        while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (lv.cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
        const uint32_t local = (uint32_t)(c - lv.cell_off[lo]);
        const uint2 k = lv.keys[lo];
        if (lv.apoptotic >= 0 && lv.role_apop >= 0) {
            const uint4 r = philox(local, *step, 9u, 0u, k.x, k.y);
            if (u01(r.x, r.y) < state[(int64_t)lv.role_apop * nc + c]) { type[c] = lv.apoptotic; return; }
        }
        if (lv.differentiated >= 0 && lv.role_diff >= 0) {
            const uint4 r = philox(local, *step, 10u, 0u, k.x, k.y);
            if (u01(r.x, r.y) < state[(int64_t)lv.role_diff * nc + c]) { type[c] = lv.differentiated; return; }
        }
    }
    uint32_t full = min(mech_target[c], 0x7fffffffu);
    if (began && due[c] > began[c]) {
        // grown (simulation.rs:2534-2540)
        const double passed = fmin((double)((int64_t)*step - began[c]) / (double)(due[c] - began[c]), 1.0);
        full = (uint32_t)round((double)full * (0.5 + 0.5 * passed));
    }
    target[c] = (int32_t)full;
    lambda[c] = lam;
}

// The cycle lengths of each division (simulation.rs:1701-1713, 1739-1745):
// the parent's and the daughter's begin at this step and last median x
// exp(spread z), z a standard normal by Box and Muller from two uniform draws
// (Philox(parent, step, 5, 0) under the history's key), rounded, a step at
// least.
__device__ __forceinline__ int32_t cycle_length(double u, double v, double median, double spread) {
    const double z = sqrt(-2.0 * log(1.0 - u)) * cos(6.283185307179586 * v);
    return (int32_t)fmax(round(median * exp(spread * z)), 1.0);
}
__global__ void k_cycle_births(const int64_t *cell_off, int nh, int64_t nc, const int32_t *daughter, const uint2 *keys,
                               const uint32_t *step, double median, double spread, int32_t *began, int32_t *due,
                               const int32_t *count) {
    if (*count == 0) return;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc || daughter[c] < 0) return;
    int lo = 0, hi = nh - 1;
    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
    const int64_t d = cell_off[lo] + daughter[c];
    const uint2 k = keys[lo];
    const uint32_t now = *step;
    const uint4 r = philox((uint32_t)(c - cell_off[lo]), now, 5u, 0u, k.x, k.y);
    const uint4 q = philox((uint32_t)(c - cell_off[lo]), now, 5u, 1u, k.x, k.y);
    began[c] = began[d] = (int32_t)now;
    due[c] = (int32_t)now + cycle_length(u01(r.x, r.y), u01(r.z, r.w), median, spread);
    due[d] = (int32_t)now + cycle_length(u01(q.x, q.y), u01(q.z, q.w), median, spread);
}

// Which cells divide this step (divide_ready_cells, simulation.rs:1603-1626):
// living, of at least DIVISION_RATIO times the reference volume, cycling
// (hypoxia response under QUIESCENCE_THRESHOLD); the plane's normal from
// Philox(cell, step, 3, 0) under the history's key: a uniform angle in the
// plane, a uniform direction in a volume (simulation.rs:1631-1642).  Also
// refreshes `alive` for the living-cell limit.
__global__ void k_div_ready(const int32_t *type, const int32_t *volume, const int64_t *cell_off, const uint2 *keys,
                            const int4 *dims, int nh, int64_t nc, uint32_t leaving, const double *state, int hyp,
                            double threshold, const uint32_t *mcs_ctr, uint8_t *alive, uint8_t *flag,
                            double *normal, int32_t *count, const uint32_t *step, int every, const int32_t *due_at) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    int lo = 0, hi = nh - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cell_off[mid] <= c) lo = mid; else hi = mid - 1; }
    const int64_t local = c - cell_off[lo];
    const bool a = local > 0 && volume[c] > 0 && !((leaving >> (type[c] & 31)) & 1u);
    alive[c] = a;
    // the check on the steps it is taken on (every > 1: step % every == 0)
    const bool due = every <= 1 || (*step % (uint32_t)every) == 0u;
    const bool ready = due && a && (double)volume[c] >= threshold && (!due_at || due_at[c] <= (int32_t)*step) &&
                       (hyp < 0 || state[(int64_t)hyp * nc + c] < QUIESCENCE_THRESHOLD);
    flag[c] = ready;
    if (!ready) return;
    atomicAdd(count, 1);  // few cells are ready at once
    const uint2 k = keys[lo];
    const uint4 r = philox((uint32_t)local, *mcs_ctr, 3u, 0u, k.x, k.y);
    const double u0 = u01(r.x, r.y), u1 = u01(r.z, r.w);
    if (dims[lo].z > 1) {
        const double z = 2.0 * u0 - 1.0, around = u1 * 6.283185307179586;
        const double rr = sqrt(fmax(1.0 - z * z, 0.0));
        normal[3 * c + 0] = rr * cos(around);
        normal[3 * c + 1] = rr * sin(around);
        normal[3 * c + 2] = z;
    } else {
        const double angle = u0 * 3.141592653589793;
        normal[3 * c + 0] = cos(angle);
        normal[3 * c + 1] = sin(angle);
        normal[3 * c + 2] = 0.0;
    }
}

__global__ void k_stats(const uint8_t *alive, const double *cell_o2, const int32_t *volume, const int64_t *cell_off,
                        int nh, double *out) {
    int h = blockIdx.x;
    int64_t c0 = cell_off[h], c1 = cell_off[h + 1];
    double living = 0.0, o2 = 0.0, vol = 0.0;
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        if (alive[c]) living += 1.0;
        if (c > c0 && volume[c] > 0) { o2 += cell_o2[c] * volume[c]; vol += volume[c]; }
    }
    living = warp_sum(living); o2 = warp_sum(o2); vol = warp_sum(vol);
    __shared__ double s[3][32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s[0][wid] = living; s[1][wid] = o2; s[2][wid] = vol; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, v = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += s[0][k]; b += s[1][k]; v += s[2][k]; }
        out[4 * h + 0] = a;
        out[4 * h + 1] = v > 0 ? b / v : 0.0;
    }
}

__global__ void k_fill_u8(uint8_t *p, int64_t n, uint8_t v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Seed one history on the host: squares (or cubes) of side s of random type
// 1..types at random places that overlap nothing, `n` of them or as many as
// fit (seeding 0); a regular packing of squares with a gap of (pitch - s)
// (seeding 1); cubes packed in a ball around the centre (seeding 2).
void seed_history(const cw_sim_config &c, uint32_t W, uint32_t H, uint32_t D, uint32_t n, uint64_t seed,
                  std::vector<int32_t> &grid, std::vector<int32_t> &type, int ncelltypes) {
    std::mt19937_64 rng(seed);
    grid.assign((size_t)W * H * D, 0);
    type.assign(1, 0);
    const int s = c.seed_side > 0 ? c.seed_side : 7;
    auto pick_type = [&]() { return 1 + (int)(rng() % (uint64_t)ncelltypes); };
    // vessel column as obstacle (held by the oxygen field)
    if (c.o2_hold == 1)
        for (uint32_t z = 0; z < D; ++z)
            for (uint32_t y = 0; y < H; ++y) grid[((size_t)z * H + y) * W + W / 2] = -1;
    // a vessel: an obstacle disc at the centre through every slice (add_obstacle_disc, cpm.rs:389-415)
    if (c.o2_hold == 4) {
        const int64_t cx = W / 2, cy = H / 2, r2 = (int64_t)c.vessel_radius * c.vessel_radius;
        for (uint32_t z = 0; z < D; ++z)
            for (uint32_t y = 0; y < H; ++y)
                for (uint32_t x = 0; x < W; ++x) {
                    const int64_t dx = (int64_t)x - cx, dy = (int64_t)y - cy;
                    if (dx * dx + dy * dy <= r2) grid[((size_t)z * H + y) * W + x] = -1;
                }
    }
    // one cell (Seeding::Single, simulation.rs:666-694): a ball of radius s at
    // the centre, or against the vessel's wall (add_ball, cpm.rs:323-354)
    if (c.seeding == 3) {
        const int64_t cx = (int64_t)(W / 2) + (c.o2_hold == 4 ? c.vessel_radius + s : 0), cy = H / 2, cz = D / 2;
        const int64_t r2 = (int64_t)s * s;
        for (uint32_t z = 0; z < D; ++z)
            for (uint32_t y = 0; y < H; ++y)
                for (uint32_t x = 0; x < W; ++x) {
                    const int64_t dx = (int64_t)x - cx, dy = (int64_t)y - cy, dz = (int64_t)z - cz;
                    int32_t &g = grid[((size_t)z * H + y) * W + x];
                    if (dx * dx + dy * dy + dz * dz <= r2 && g != -1) g = 1;
                }
        type.push_back(1);
        return;
    }
    // a sheet (Seeding::Sheet, simulation.rs:696-740): the box tiled with
    // side x side blocks of normal tissue (type 2), row by row
    if (c.seeding == 4) {
        for (uint32_t y = 0; y < H; y += (uint32_t)s)
            for (uint32_t x = 0; x < W; x += (uint32_t)s) {
                const int32_t id = (int32_t)type.size();
                for (uint32_t yy = y; yy < y + (uint32_t)s && yy < H; ++yy)
                    for (uint32_t xx = x; xx < x + (uint32_t)s && xx < W; ++xx) grid[(size_t)yy * W + xx] = id;
                type.push_back(2);
            }
        return;
    }
    auto free_box = [&](uint32_t x0, uint32_t y0, uint32_t z0, uint32_t sx, uint32_t sy, uint32_t sz) {
        if (x0 + sx > W || y0 + sy > H || z0 + sz > D) return false;
        for (uint32_t z = z0; z < z0 + sz; ++z)
            for (uint32_t y = y0; y < y0 + sy; ++y)
                for (uint32_t x = x0; x < x0 + sx; ++x)
                    if (grid[((size_t)z * H + y) * W + x] != 0) return false;
        return true;
    };
    auto put = [&](uint32_t x0, uint32_t y0, uint32_t z0, uint32_t sx, uint32_t sy, uint32_t sz) {
        int32_t id = (int32_t)type.size();
        for (uint32_t z = z0; z < z0 + sz; ++z)
            for (uint32_t y = y0; y < y0 + sy; ++y)
                for (uint32_t x = x0; x < x0 + sx; ++x) grid[((size_t)z * H + y) * W + x] = id;
        type.push_back(pick_type());
    };
    uint32_t sz = D > 1 ? (uint32_t)s : 1;
    if (c.seeding == 1) {
        uint32_t pitch = (uint32_t)s + 2;
        for (uint32_t z = 0; z + sz <= D; z += (D > 1 ? pitch : 1))
            for (uint32_t y = 1; y + s <= H; y += pitch)
                for (uint32_t x = 1; x + s <= W; x += pitch)
                    if (type.size() - 1 < n && free_box(x, y, z, s, s, sz)) put(x, y, z, s, s, sz);
    } else if (c.seeding == 2 && D > 1) {
        // cubes on a grid of pitch s inside a ball of radius R around the centre
        double R = std::cbrt(3.0 * n * s * s * s / (4.0 * 3.14159265358979)) + 0.5 * s;
        double cx = W / 2.0, cy = H / 2.0, cz = D / 2.0;
        for (uint32_t z = 0; z + s <= D; z += s)
            for (uint32_t y = 0; y + s <= H; y += s)
                for (uint32_t x = 0; x + s <= W; x += s) {
                    double dx = x + s / 2.0 - cx, dy = y + s / 2.0 - cy, dz = z + s / 2.0 - cz;
                    if (dx * dx + dy * dy + dz * dz <= R * R && type.size() - 1 < n && free_box(x, y, z, s, s, s))
                        put(x, y, z, s, s, s);
                }
    } else {
        uint64_t tries = 0, cap = 200ull * n + 1000;
        while (type.size() - 1 < n && tries++ < cap) {
            uint32_t x = (uint32_t)(rng() % (W - s + 1)), y = (uint32_t)(rng() % (H - s + 1));
            uint32_t z = D > 1 ? (uint32_t)(rng() % (D - sz + 1)) : 0;
            if (free_box(x, y, z, s, s, sz)) put(x, y, z, s, s, sz);
        }
    }
}

int64_t blocks(int64_t n) { return (n + T - 1) / T; }

}  // namespace

extern "C" {

int cw_sim_create(const cw_sim_config *cfg, cw_network net, cw_sim *out) {
    *out = nullptr;
    const cw_sim_config &c = *cfg;
    if (c.nh == 0) return fail(CW_ERR_CONFIG, "a simulation needs a history");
    if (c.K < 2 || c.K > 8) return fail(CW_ERR_CONFIG, "2 to 8 types, the medium included");
    if (c.nfields < 1 || c.nfields > 2) return fail(CW_ERR_CONFIG, "one or two fields");
    if (!(c.error_tolerance >= 0.0 && c.error_tolerance < INFINITY))
        return fail(CW_ERR_CONFIG, "the error tolerance must be finite and not negative");
    if (c.o2_hold < 0 || c.o2_hold > 4)
        return fail(CW_ERR_CONFIG, "the oxygen is held on a row, a column, the faces, the bath or a vessel");
    if (c.o2_hold == 4 && c.vessel_radius < 1) return fail(CW_ERR_CONFIG, "a vessel needs a radius of a pixel or more");
    if (c.stop_rule == CW_STOP_MAX_CHANGE && c.precision != CW_FP64)
        return fail(CW_ERR_CONFIG, "the largest change a sweep is the FP64 solve's stopping rule");
    if (c.cycle_median != 0.0 && !(c.cycle_median >= 1.0 && c.cycle_median < 1e9 && c.cycle_spread >= 0.0 &&
                                   c.cycle_spread < 1e3))
        return fail(CW_ERR_CONFIG, "a cycle lasts a step at least, and its spread is not below zero");
    if (c.debris_loss != 0.0 && !(c.debris_loss > 0.0 && c.debris_loss <= 1.0))
        return fail(CW_ERR_CONFIG, "debris loss is the share of a dead cell lost per step, above zero and at most one");
    if (c.debris_loss > 0.0 && c.necrotic_type < 0) return fail(CW_ERR_CONFIG, "debris loss needs a necrotic type");
    if (c.exposure_intensity != 0.0) {
        if (!(c.exposure_intensity > 0.0 && c.exposure_intensity < 1e300))
            return fail(CW_ERR_CONFIG, "the exposure's intensity must be zero or more");
        if (!(c.exposure_uptake > 0.0 && c.exposure_uptake < 1e300))
            return fail(CW_ERR_CONFIG, "the exposure's uptake must be above zero, or it fills the box");
        if (c.exposure_start < 0 || c.exposure_on < 0 || c.exposure_off < 0)
            return fail(CW_ERR_CONFIG, "an exposure's start and schedule are counts of steps");
        if (c.exposure_on == 0 && c.exposure_off > 0)
            return fail(CW_ERR_CONFIG, "a periodic exposure that is on for zero steps is never on");
    }
    if (c.still_medium != 0.0) {
        if (!(c.still_medium > 0.0 && c.still_medium < 1e300))
            return fail(CW_ERR_CONFIG, "the still medium's diffusion is above zero");
        if (c.o2_hold != 3) return fail(CW_ERR_CONFIG, "a still medium is the bath's, and this scenario has none");
        for (uint32_t k = 0; k < c.nh; ++k)
            if (!c.d || c.d[k] <= 1)
                return fail(CW_ERR_CONFIG, "a still medium is solved around a ball, and a plane has none");
    }
    if (c.seeding == 4) {
        // simulation.rs:696-731
        if (c.seed_side < 4)
            return fail(CW_ERR_CONFIG, "a sheet of cells " + std::to_string(c.seed_side) +
                                           " pixels across is too fine for any of them to divide");
        for (uint32_t k = 0; k < c.nh; ++k) {
            if ((c.d && c.d[k] > 1))
                return fail(CW_ERR_CONFIG, "a sheet, which is a layer one cell thick, runs only in the plane");
            if (c.w[k] % (uint32_t)c.seed_side || c.h[k] % (uint32_t)c.seed_side)
                return fail(CW_ERR_CONFIG, "a sheet of cells " + std::to_string(c.seed_side) +
                                               " pixels across does not tile a " + std::to_string(c.w[k]) + "x" +
                                               std::to_string(c.h[k]) + " box");
        }
        if (!c.field_off)
            return fail(CW_ERR_CONFIG, "a sheet fills the box and leaves no medium to supply oxygen; "
                                       "it runs with the field off");
    }
    if (c.field_off && c.nfields != 1)
        return fail(CW_ERR_CONFIG, "with the field off there is only the oxygen, at its start");
    for (int32_t t : {c.differentiated_type, c.apoptotic_type})
        if (t >= c.K || t == 0 || t < -1 || (t >= 0 && t == c.necrotic_type))
            return fail(CW_ERR_CONFIG, "a leaving type is a cell type of the contact table, apart from the necrotic");
    if (c.differentiated_type >= 0 && c.differentiated_type == c.apoptotic_type)
        return fail(CW_ERR_CONFIG, "differentiated and apoptotic cells take different types");
    if (!(c.mutation_rate >= 0.0 && c.mutation_rate <= 1.0) || !(c.rewiring >= 0.0 && c.rewiring <= 1.0))
        return fail(CW_ERR_CONFIG, "the mutation rate and the rewiring share lie in [0, 1]");
    if (c.mutation_rate > 0.0 && !c.divide)
        return fail(CW_ERR_CONFIG, "mutations come at divisions, and this simulation does not divide");
    if (c.tracing && c.tracing_at < 0) return fail(CW_ERR_CONFIG, "lineage tracing marks the cells at a step, 0 or later");
    if (!net) return fail(CW_ERR_CONFIG, "a simulation needs a network");
    int32_t survival = network_role(net, 1);
    cw_sim_s *s = new cw_sim_s();
    if (s->hs.init() != CW_OK) { delete s; return CW_ERR_CUDA; }
    CW_SCOPE(s);  // its lattice and fields take its stream
    s->cfg = c;
    s->w.assign(c.w, c.w + c.nh);
    s->h.assign(c.h, c.h + c.nh);
    s->d.assign(c.nh, 1);
    if (c.d) s->d.assign(c.d, c.d + c.nh);
    s->ncells.assign(c.ncells, c.ncells + c.nh);
    s->seeds.assign(c.seeds, c.seeds + c.nh);
    s->J.assign(c.J, c.J + c.K * c.K);
    s->sink.assign(8, 0.0);
    for (int k = 0; k < c.K; ++k) s->sink[k] = c.o2_sink_by_type[k];
    s->cfg.w = s->w.data(); s->cfg.h = s->h.data(); s->cfg.d = s->d.data();
    s->cfg.ncells = s->ncells.data(); s->cfg.seeds = s->seeds.data(); s->cfg.J = s->J.data();
    s->cfg.o2_sink_by_type = s->sink.data();
    s->net = net;
    int ncelltypes = c.necrotic_type > 0 ? c.necrotic_type - 1 : c.K - 1;
    if (ncelltypes < 1) ncelltypes = 1;
    // seed every history on the host
    std::vector<std::vector<int32_t>> grids(c.nh), types(c.nh);
    std::vector<uint32_t> cap(c.nh);
    for (uint32_t k = 0; k < c.nh; ++k) {
        seed_history(c, s->w[k], s->h[k], s->d[k], s->ncells[k], s->seeds[k], grids[k], types[k], ncelltypes);
        // records for the daughters of divisions too
        const int32_t spare = !c.divide ? 0 : c.spare_cells > 0 ? c.spare_cells : c.max_cells > 0 ? c.max_cells
                                                                                              : DEFAULT_MAX_CELLS;
        cap[k] = (uint32_t)(types[k].size() + spare);
        s->obstacles.push_back((uint64_t)std::count(grids[k].begin(), grids[k].end(), -1));
    }
    int rc = cw_lattice_create(c.nh, s->w.data(), s->h.data(), s->d.data(), cap.data(), c.temperature, &s->lat);
    if (rc != CW_OK) { cw_sim_destroy(s); return rc; }
    if ((rc = cw_lattice_set_contact(s->lat, c.K, c.J, c.contact_order)) != CW_OK) { cw_sim_destroy(s); return rc; }
    if (c.subsweeps > 1 && (rc = cw_lattice_set_subsweeps(s->lat, c.subsweeps)) != CW_OK) { cw_sim_destroy(s); return rc; }
    if (c.divide && (rc = s->lat->div.ensure(s->lat->ncells)) != CW_OK) { cw_sim_destroy(s); return rc; }
    for (uint32_t k = 0; k < c.nh; ++k) {
        uint32_t n = (uint32_t)types[k].size();  // the seeded records; the spares stay free
        std::vector<int32_t> vol(n, 0), tgt(n, c.target_volume);
        std::vector<double> lam(n, c.lambda_volume);
        for (int32_t id : grids[k]) if (id > 0) vol[id] += 1;
        if (c.seeding == 3 || c.target_volume <= 0) tgt = vol;  // a seeded cell aims at what it holds
        tgt[0] = 0;
        lam[0] = 0.0;
        if ((rc = cw_lattice_upload(s->lat, k, grids[k].data())) ||
            (rc = cw_cells_set(s->lat, k, n, types[k].data(), vol.data(), tgt.data(), lam.data())) ||
            (rc = cw_lattice_set_seed(s->lat, k, s->seeds[k]))) {
            cw_sim_destroy(s);
            return rc;
        }
        if (c.surface_target > 0) {
            std::vector<int32_t> ts(n, c.surface_target);
            std::vector<double> ls(n, c.lambda_surface);
            if ((rc = cw_cells_set_surface(s->lat, k, n, ts.data(), ls.data())) != CW_OK) {
                cw_sim_destroy(s);
                return rc;
            }
        }
    }
    // fields: the oxygen starts at the source's level, or at zero around a vessel (simulation.rs:786-793)
    if ((rc = cw_field_create(c.nh, s->w.data(), s->h.data(), s->d.data(), c.o2_dcoef, 0.0, c.o2_hold == 4 ? 0.0 : 1.0,
                              &s->o2)) != CW_OK) {
        cw_sim_destroy(s);
        return rc;
    }
    for (uint32_t k = 0; k < c.nh; ++k) {
        int64_t n = (int64_t)s->w[k] * s->h[k] * s->d[k];
        std::vector<uint8_t> held(n, 0);
        uint32_t W = s->w[k], H = s->h[k], D = s->d[k];
        for (uint32_t z = 0; z < D; ++z)
            for (uint32_t y = 0; y < H; ++y)
                for (uint32_t x = 0; x < W; ++x) {
                    bool on = c.o2_hold == 0 ? y == 0
                            : c.o2_hold == 1 ? x == W / 2
                            : c.o2_hold == 2 ? (x == 0 || y == 0 || x + 1 == W || y + 1 == H || z == 0 || z + 1 == D)
                            : c.o2_hold == 4 ? grids[k][((size_t)z * H + y) * W + x] == -1  // the vessel's pixels
                                             : false;  // 3: the bath, taken every step
                    held[((size_t)z * H + y) * W + x] = on;
                }
        if ((rc = cw_field_hold_mask(s->o2, k, held.data(), 1.0)) != CW_OK) { cw_sim_destroy(s); return rc; }
    }
    if (c.nfields == 2 &&
        (rc = cw_field_create(c.nh, s->w.data(), s->h.data(), s->d.data(), c.signal_dcoef, c.signal_decay, 0.0,
                              &s->sig)) != CW_OK) {
        cw_sim_destroy(s);
        return rc;
    }
    if (c.waste_production > 0.0 &&
        (rc = cw_field_create(c.nh, s->w.data(), s->h.data(), s->d.data(), c.o2_dcoef, 0.0, 0.0, &s->wst)) != CW_OK) {
        cw_sim_destroy(s);
        return rc;
    }
    if (c.exposure_intensity > 0.0) {
        // STRESS_DIFFUSION = OXYGEN_DIFFUSION (simulation.rs:157), from zero
        if ((rc = cw_field_create(c.nh, s->w.data(), s->h.data(), s->d.data(), c.o2_dcoef, 0.0, 0.0, &s->str)) !=
            CW_OK) {
            cw_sim_destroy(s);
            return rc;
        }
        std::vector<double> up(8, 0.0);
        for (int k = 1; k < c.K; ++k) up[k] = k == c.necrotic_type ? 0.0 : c.exposure_uptake;
        if ((rc = dalloc(&s->d_str_uptake, 8)) != CW_OK) { cw_sim_destroy(s); return rc; }
        CW_CUDA(cudaMemcpy(s->d_str_uptake, up.data(), 8 * sizeof(double), cudaMemcpyHostToDevice));
        s->str->uptake_on = true;
        CW_CUDA(cudaMemset(s->str->uptake, 0, sizeof(double) * (size_t)s->str->g.total));
    }
    if (c.necrotic_production > 0.0) {
        if (c.necrotic_type < 0) {
            cw_sim_destroy(s);
            return fail(CW_ERR_CONFIG, "a necrotic factor is released by necrotic cells, and this simulation has none");
        }
        if ((rc = cw_field_create(c.nh, s->w.data(), s->h.data(), s->d.data(), c.o2_dcoef, 0.0, 0.0, &s->nfc)) !=
            CW_OK) {
            cw_sim_destroy(s);
            return rc;
        }
    }
    // per-cell device state
    s->nc = s->lat->ncells;
    int S = network_nodes(net);
    int64_t nc = s->nc;
    if ((rc = dalloc(&s->d_sink, 8)) || (rc = dalloc(&s->cell_o2, nc)) || (rc = dalloc(&s->cell_sig, nc)) ||
        (rc = dalloc(&s->sum, nc)) || (rc = dalloc(&s->secretion, nc)) || (rc = dalloc(&s->count, nc)) ||
        (rc = dalloc(&s->state, nc * S)) || (rc = dalloc(&s->inputs, nc * 6)) || (rc = dalloc(&s->alive, nc)) ||
        (rc = dalloc(&s->target32, nc))) {
        cw_sim_destroy(s);
        return rc;
    }
    if ((rc = dalloc(&s->d_step, 1)) || (rc = dalloc(&s->died_at, nc)) || (rc = dalloc(&s->cell_wst, nc)) ||
        (rc = dalloc(&s->cell_nfc, nc)) || (rc = dalloc(&s->wst_rate, nc)) || (rc = dalloc(&s->nfc_rate, nc))) {
        cw_sim_destroy(s);
        return rc;
    }
    s->debris_on = c.debris_loss > 0.0;
    if ((c.o2_hold == 3 || s->wst || s->nfc || s->debris_on) &&
        (rc = dalloc(&s->bath, (size_t)s->lat->g.total)) != CW_OK) {
        cw_sim_destroy(s);
        return rc;
    }
    if (s->debris_on && (rc = s->debris.ensure(nc, (int)c.nh, s->lat->g.total)) != CW_OK) {
        cw_sim_destroy(s);
        return rc;
    }
    if ((rc = dalloc(&s->level, c.nh)) || (rc = dalloc(&s->d_inflow, c.nh)) || (rc = dalloc(&s->d_free, c.nh)) ||
        (rc = dalloc(&s->cell_str, nc))) {
        cw_sim_destroy(s);
        return rc;
    }
    {
        std::vector<double> ones(c.nh, 1.0);
        CW_CUDA(cudaMemcpy(s->level, ones.data(), sizeof(double) * c.nh, cudaMemcpyHostToDevice));
    }
    if (c.cycle_median > 0.0) {
        if ((rc = dalloc(&s->began, nc)) || (rc = dalloc(&s->due, nc))) {
            cw_sim_destroy(s);
            return rc;
        }
        // the cells the tissue starts with: no cycle behind them (simulation.rs:1055-1056)
        CW_CUDA(cudaMemsetAsync(s->began, 0, sizeof(int32_t) * nc, stream()));
        CW_CUDA(cudaMemsetAsync(s->due, 0, sizeof(int32_t) * nc, stream()));
    }
    for (int32_t t : {c.necrotic_type, c.differentiated_type, c.apoptotic_type})
        if (t >= 0 && t < 32) s->leaving |= 1u << t;
    if (c.tracing) {
        s->tracing = true;
        s->h_mark.assign(nc, -1);
    }
    if (c.mutation_rate > 0.0 || c.lineage || c.tracing) {
        // every record starts in the founding clone, or (a lineage) every seeded
        // cell founds its own: its clone is its record's index in the batch
        s->track = true;
        s->evolve = c.mutation_rate > 0.0;
        s->h_clone.assign(nc, 0);
        if (c.lineage)
            for (uint32_t k = 0; k < c.nh; ++k)
                for (size_t id = 1; id < types[k].size(); ++id) {
                    const int64_t g = s->lat->cell_off[k] + (int64_t)id;
                    s->h_clone[g] = (int32_t)g;
                }
        s->clones.assign(c.lineage ? (size_t)nc : 1, net);
        s->clone_owned.assign(s->clones.size(), 0);
        s->clone_lesion.assign(s->clones.size(), 0);
        s->clone_nets = s->evolve;
        if ((rc = dalloc(&s->d_clone, nc)) != CW_OK || (rc = upload_clones(s, true)) != CW_OK) {
            cw_sim_destroy(s);
            return rc;
        }
    }
    CW_CUDA(cudaMemsetAsync(s->d_step, 0, sizeof(uint32_t), stream()));
    CW_CUDA(cudaMemsetAsync(s->died_at, 0xFF, sizeof(int32_t) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(s->cell_wst, 0, sizeof(double) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(s->cell_nfc, 0, sizeof(double) * nc, stream()));
    CW_CUDA(cudaMemcpyAsync(s->d_sink, s->sink.data(), 8 * sizeof(double), cudaMemcpyHostToDevice, stream()));
    {
        // the zero-order uptake of the living types (not the medium, not the dead)
        std::vector<double> up(8, 0.0);
        for (int k = 1; k < c.K; ++k) up[k] = k == c.necrotic_type ? 0.0 : std::max(c.o2_uptake, 0.0);
        if ((rc = dalloc(&s->d_uptake, 8)) != CW_OK) { cw_sim_destroy(s); return rc; }
        CW_CUDA(cudaMemcpyAsync(s->d_uptake, up.data(), 8 * sizeof(double), cudaMemcpyHostToDevice, stream()));
        if (c.o2_uptake > 0.0) {
            s->o2->uptake_on = true;
            CW_CUDA(cudaMemsetAsync(s->o2->uptake, 0, sizeof(double) * (size_t)s->o2->g.total, stream()));
        }
    }
    std::vector<double> st((size_t)nc * S);
    const std::vector<double> &init = network_initial(net);
    for (int i = 0; i < S; ++i) std::fill(st.begin() + (size_t)i * nc, st.begin() + (size_t)(i + 1) * nc, init[i]);
    CW_CUDA(cudaMemcpyAsync(s->state, st.data(), sizeof(double) * nc * S, cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaMemsetAsync(s->cell_o2, 0, sizeof(double) * nc, stream()));
    CW_CUDA(cudaMemsetAsync(s->cell_sig, 0, sizeof(double) * nc, stream()));
    std::vector<int64_t> per(c.nh);
    for (uint32_t k = 0; k < c.nh; ++k) per[k] = (int64_t)s->w[k] * s->h[k] * s->d[k];
    if ((rc = s->sites.build(per, T)) != CW_OK) { cw_sim_destroy(s); return rc; }
    s->last.assign(c.nh, cw_relax_stats{});
    // relaxation factors: the configuration's, or the reference's rule
    // until the autotuner has chosen one per lattice size
    for (int f = 0; f < 2; ++f) s->omega[f].assign(c.nh, 0.0);
    if (c.omega <= 0.0 && c.precision == CW_FP32_DC) tune_begin(s);
    else s->depth_tuned = true;
    (void)survival;
    CW_CUDA(cudaStreamSynchronize(stream()));
    *out = s;
    return CW_OK;
}

int cw_sim_set_lesion(cw_sim s, cw_network net, uint32_t at, double radius, double cx, double cy) {
    CW_SCOPE(s);
    const cw_sim_config &c = s->cfg;
    if (!net) return fail(CW_ERR_CONFIG, "a lesion needs a network");
    for (uint32_t k = 0; k < c.nh; ++k) {
        if (s->d[k] > 1)
            return fail(CW_ERR_CONFIG, "a lesion is placed in a plane; history " + std::to_string(k) + " is a volume");
        // simulation.rs:751-770
        if ((!std::isnan(cx) || !std::isnan(cy)) &&
            !(cx >= 0.0 && cx < (double)s->w[k] && cy >= 0.0 && cy < (double)s->h[k]))
            return fail(CW_ERR_CONFIG, "a lesion centred at (" + std::to_string(cx) + ", " + std::to_string(cy) +
                                           ") lies outside the " + std::to_string(s->w[k]) + "x" +
                                           std::to_string(s->h[k]) + " box");
    }
    if (std::isnan(cx) != std::isnan(cy)) return fail(CW_ERR_CONFIG, "a lesion's centre names both coordinates");
    if (!(std::isfinite(radius) && radius > 0.0))
        return fail(CW_ERR_CONFIG, "a lesion of radius " + std::to_string(radius) + " holds no cell");
    // every cell steps under its clone's network with the tissue's roles and
    // mechanics: the lesion's network must share them
    const cw_network_s *a = s->net, *b = net;
    bool same = a->S == b->S && a->growth_coefficient == b->growth_coefficient &&
                a->lambda_volume == b->lambda_volume && a->reference_volume == b->reference_volume &&
                (a->max_target == b->max_target || (std::isnan(a->max_target) && std::isnan(b->max_target)));
    for (int r = 0; r < 7; ++r) same = same && a->roles[r] == b->roles[r];
    if (!same)
        return fail(CW_ERR_CONFIG, "the device steps a lesion whose network has the tissue's nodes, roles, "
                                   "mechanics and reference volume");
    if (s->steps > at) return fail(CW_ERR_CONFIG, "the lesion's step " + std::to_string(at) + " has passed");
    if (!s->track) {
        // from now on every record's clone is followed (all in the founding one)
        s->track = true;
        s->h_clone.assign(s->nc, 0);
        s->clones.assign(1, s->net);
        s->clone_owned.assign(1, 0);
        s->clone_lesion.assign(1, 0);
        int rc = dalloc(&s->d_clone, s->nc);
        if (rc != CW_OK) return rc;
    }
    s->clone_nets = true;
    s->lesion_net = net;
    s->lesion_at = (int64_t)at;
    s->lesion_radius = radius;
    s->lesion_cx = cx;
    s->lesion_cy = cy;
    drop_graphs(s);
    return upload_clones(s, true);
}

int cw_sim_destroy(cw_sim s) {
    if (!s) return CW_OK;
    CW_SCOPE(s);
    drop_graphs(s);
    cw_lattice_destroy(s->lat);
    cw_field_destroy(s->o2);
    cw_field_destroy(s->sig);
    cw_field_destroy(s->wst);
    cw_field_destroy(s->nfc);
    dfree(s->cell_wst); dfree(s->cell_nfc); dfree(s->wst_rate); dfree(s->nfc_rate); dfree(s->died_at); dfree(s->began); dfree(s->due);
    s->debris.release(); dfree(s->level); dfree(s->d_inflow); dfree(s->d_free);
    cw_field_destroy(s->str); dfree(s->cell_str); dfree(s->d_str_uptake);
    dfree(s->d_step); dfree(s->bath); dfree(s->d_uptake);
    dfree(s->d_sink); dfree(s->cell_o2); dfree(s->cell_sig); dfree(s->sum); dfree(s->secretion); dfree(s->count);
    dfree(s->state); dfree(s->inputs); dfree(s->alive); dfree(s->target32);
    // the networks mutations made; the founders, a lesion's clone and the
    // clones of suppressed mutations share networks the simulation does not own
    for (size_t k = 0; k < s->clones.size(); ++k)
        if (k < s->clone_owned.size() && s->clone_owned[k]) cw_network_destroy(s->clones[k]);
    dfree(s->d_clone); dfree(s->d_nets);
    s->sites.release();
    s->hs.release();
    delete s;
    return CW_OK;
}

// The autotuner: while it runs, the histories of one lattice size share the
// candidate factors among them (history q of a size class takes candidate
// (q + step) mod n), and each solve's sweep count is booked against its
// candidate; afterwards every history takes its class's best factor.
static void tune_begin(cw_sim_s *s) {
    auto &t = s->tune;
    // volumes take larger factors (the reference's rule gives 1.94 for a span
    // of 100 voxels, 1.976 for 256)
    if (s->d[0] > 1) t.cand = {1.88, 1.91, 1.93, 1.95, 1.96, 1.97, 1.98};
    else t.cand = {1.80, 1.85, 1.88, 1.90, 1.92, 1.94, 1.96};
    uint32_t nh = s->cfg.nh;
    t.cls.assign(nh, 0);
    t.rank.assign(nh, 0);
    std::vector<std::array<uint32_t, 3>> keys;
    std::vector<int> members;
    for (uint32_t k = 0; k < nh; ++k) {
        std::array<uint32_t, 3> key{s->w[k], s->h[k], s->d[k]};
        size_t c = std::find(keys.begin(), keys.end(), key) - keys.begin();
        if (c == keys.size()) { keys.push_back(key); members.push_back(0); }
        t.cls[k] = (int)c;
        t.rank[k] = members[c]++;
    }
    t.nclass = (int)keys.size();
    int smallest = *std::min_element(members.begin(), members.end());
    int n = (int)t.cand.size();
    t.steps = std::max(2, (n + smallest - 1) / smallest);
    for (int f = 0; f < 2; ++f) { t.sum[f].assign(t.nclass * n, 0.0); t.cnt[f].assign(t.nclass * n, 0.0); }
    t.active = true;
    t.done = 0;
}

static void tune_assign(cw_sim_s *s) {
    auto &t = s->tune;
    int n = (int)t.cand.size();
    for (int f = 0; f < 2; ++f)
        for (uint32_t k = 0; k < s->cfg.nh; ++k) s->omega[f][k] = t.cand[(t.rank[k] + t.done) % n];
}

static void tune_book(cw_sim_s *s, int f, const std::vector<cw_relax_stats> &st) {
    auto &t = s->tune;
    int n = (int)t.cand.size();
    for (uint32_t k = 0; k < s->cfg.nh; ++k) {
        int c = (t.rank[k] + t.done) % n;
        t.sum[f][t.cls[k] * n + c] += (double)st[k].sweeps;
        t.cnt[f][t.cls[k] * n + c] += 1.0;
    }
}

static void tune_finish(cw_sim_s *s) {
    auto &t = s->tune;
    int n = (int)t.cand.size();
    for (int f = 0; f < 2; ++f)
        for (uint32_t k = 0; k < s->cfg.nh; ++k) {
            int best = -1;
            double bv = 0.0;
            for (int c = 0; c < n; ++c) {
                double cnt = t.cnt[f][t.cls[k] * n + c];
                if (cnt <= 0) continue;
                double v = t.sum[f][t.cls[k] * n + c] / cnt;
                if (best < 0 || v < bv) { best = c; bv = v; }
            }
            if (best >= 0) s->omega[f][k] = t.cand[best];
        }
    t.active = false;
}

// Blocking depth: the fastest of the candidates on the oxygen field's
// current residual.
static int tune_depth(cw_sim_s *s) {
    if (s->cfg.precision != CW_FP32_DC) return CW_OK;
    float best = 0.f;
    int bd = 8, bw = CW_WINDOW_AUTO;
    // volumes march tiles along z at two or four half-sweeps a launch
    const bool volume = s->d[0] > 1;
    for (int w : {CW_WINDOW_AUTO, CW_WINDOW_64})
        for (int d : {volume ? 2 : 6, 4, 8}) {
            float ms = 0.f;
            int64_t launches = 0;
            int rc = cw_field_time_inner(s->o2, 8, d, w, 1.9, &ms, &launches);
            if (rc != CW_OK) return rc;
            if (best == 0.f || ms < best) { best = ms; bd = d; bw = w; }
        }
    s->depth = bd;
    s->sor_window = bw;
    s->depth_tuned = true;
    return CW_OK;
}

static void drop_graphs(cw_sim_s *s) {
    for (auto &g : s->gexec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    s->graphs = false;
}

// The clone of every record and the clones' network tables onto the device
// (all of the tables when `tables`).
static int upload_clones(cw_sim_s *s, bool tables) {
    if (tables) {
        if (s->clones.size() > s->nets_cap) {
            dfree(s->d_nets);
            s->nets_cap = std::max<size_t>(2 * s->clones.size(), 16);
            int rc = dalloc(&s->d_nets, s->nets_cap);
            if (rc != CW_OK) { s->nets_cap = 0; return rc; }
        }
        std::vector<cw::NetDev> dev(s->clones.size());
        for (size_t k = 0; k < s->clones.size(); ++k) dev[k] = cw::net_dev(s->clones[k]);
        CW_CUDA(cudaMemcpyAsync(s->d_nets, dev.data(), sizeof(cw::NetDev) * dev.size(), cudaMemcpyHostToDevice,
                                stream()));
    }
    CW_CUDA(cudaMemcpyAsync(s->d_clone, s->h_clone.data(), sizeof(int32_t) * s->h_clone.size(),
                            cudaMemcpyHostToDevice, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

// Daughters that are not quite copies (simulation.rs:1655-1700): after a
// division step, each daughter joins its parent's clone; with chance
// mutation_rate its network changes (mutate, or with chance `rewiring`
// rewire) and it founds a clone of its own.  The draws come from Philox
// under the history's key, counter (parent id, step, 6 / 7 / 8, 0): the rate
// test and `which` from the first, `how` and the rewiring test from the
// second, the gained link's source and sign from the third.
static int evolve_after_division(cw_sim_s *s) {
    cw_lattice_s *l = s->lat;
    int32_t count = 0;
    CW_CUDA(cudaMemcpyAsync(&count, l->div.count, sizeof(int32_t), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    if (count == 0) return CW_OK;  // no cell was ready: the daughters' table is last step's
    std::vector<int32_t> dg(s->nc);
    CW_CUDA(cudaMemcpyAsync(dg.data(), l->div.daughter, sizeof(int32_t) * s->nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    const cw_sim_config &c = s->cfg;
    const uint32_t step = (uint32_t)s->steps;
    bool grown = false, moved = false;
    for (uint32_t h = 0; h < c.nh; ++h) {
        const int64_t c0 = l->cell_off[h], cap = l->cell_off[h + 1] - c0;
        const uint64_t seed = l->seed[h];
        const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
        for (int64_t id = 1; id < cap; ++id) {
            const int32_t d = dg[c0 + id];
            if (d < 0) continue;
            const int32_t parent_clone = s->h_clone[c0 + id];
            s->h_clone[c0 + d] = parent_clone;
            if (s->tracing) s->h_mark[c0 + d] = s->h_mark[c0 + id];  // simulation.rs:1711
            moved = true;
            if (!s->evolve) continue;
            const uint4 r0 = cw::philox((uint32_t)id, step, 6u, 0u, k0, k1);
            if (!(cw::u01(r0.x, r0.y) < c.mutation_rate)) continue;
            const double which = cw::u01(r0.z, r0.w);
            const uint4 r1 = cw::philox((uint32_t)id, step, 7u, 0u, k0, k1);
            const double how = cw::u01(r1.x, r1.y);
            cw_network nn = nullptr;
            cw_mutation rec{};
            int rc;
            double u = c.rewiring > 0.0 ? cw::u01(r1.z, r1.w) : 1.0;
            if (c.rewiring > 0.0 && u < c.rewiring) {
                const uint4 r2 = cw::philox((uint32_t)id, step, 8u, 0u, k0, k1);
                const double draws[5] = {u / c.rewiring, which, cw::u01(r2.x, r2.y), cw::u01(r2.z, r2.w), how};
                rc = cw_network_rewire(s->clones[parent_clone], draws, &nn, &rec);
            } else {
                rc = cw_network_mutate(s->clones[parent_clone], which, how, &nn, &rec);
            }
            if (rc == CW_ERR_NOT_FOUND) continue;  // nothing to change: the daughter stays in its parent's clone
            if (rc != CW_OK) return rc;
            // a mutation founded before suppress_before is drawn and recorded,
            // but made on a copy that is thrown away: the daughter founds its
            // clone with its parent's network unchanged (simulation.rs:1671-1694)
            const bool suppressed = c.suppress_before > 0 && (int64_t)step < (int64_t)c.suppress_before;
            if (suppressed) {
                cw_network_destroy(nn);
                nn = s->clones[parent_clone];
                rec.suppressed = 1;
            }
            s->clones.push_back(nn);
            s->clone_owned.push_back(suppressed ? 0 : 1);
            s->clone_lesion.push_back(s->clone_lesion[parent_clone]);
            s->clone_parent.push_back(parent_clone);
            s->clone_mutation.push_back(rec);
            s->h_clone[c0 + d] = (int32_t)(s->clones.size() - 1);
            grown = true;
        }
    }
    return moved ? upload_clones(s, grown) : CW_OK;
}

// Whether record g of the batch is in the layer (in_layer, simulation.rs:
// 2400-2405): holding pixels, and cycling, quiescent or committed to
// differentiate (not necrotic, not apoptotic).
static bool in_layer(const cw_sim_s *s, const std::vector<int32_t> &ty, const std::vector<int32_t> &vo, int64_t g) {
    const cw_sim_config &c = s->cfg;
    return vo[g] > 0 && ty[g] != c.necrotic_type && !(c.apoptotic_type >= 0 && ty[g] == c.apoptotic_type);
}

// The records' types and volumes on the host.
static int records_to_host(cw_sim_s *s, std::vector<int32_t> &ty, std::vector<int32_t> &vo) {
    ty.resize(s->nc);
    vo.resize(s->nc);
    CW_CUDA(cudaMemcpyAsync(ty.data(), s->lat->type, sizeof(int32_t) * s->nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(vo.data(), s->lat->volume, sizeof(int32_t) * s->nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

// mark_every_cell (simulation.rs:1908-1918): every cell in the layer takes
// its own mark (its id less one, the reference's slot), every other record
// none.  Draws nothing.
static int mark_every_cell(cw_sim_s *s) {
    std::vector<int32_t> ty, vo;
    int rc = records_to_host(s, ty, vo);
    if (rc != CW_OK) return rc;
    cw_lattice_s *l = s->lat;
    for (uint32_t h = 0; h < s->cfg.nh; ++h) {
        const int64_t c0 = l->cell_off[h], cap = l->cell_off[h + 1] - c0;
        for (int64_t id = 0; id < cap; ++id)
            s->h_mark[c0 + id] = id > 0 && in_layer(s, ty, vo, c0 + id) ? (int32_t)(id - 1) : -1;
    }
    return CW_OK;
}

// place_lesion (simulation.rs:1920-1970), before anything else in the step
// it appears at: in every history, each living cell (not necrotic, not
// leaving the layer, holding pixels) whose centre of mass lies within the
// lesion's radius of its centre joins one new clone carrying the lesion's
// network, fresh (its state the network's initial one).  Centres are the
// reference's: x + 1/2 and y + 1/2 summed in row order per cell, over the
// count.  A history with no such cell founds no clone.  Draws nothing.
static int place_lesion(cw_sim_s *s) {
    cw_lattice_s *l = s->lat;
    const cw_sim_config &c = s->cfg;
    const int64_t nc = s->nc, total = l->g.total;
    const int S = network_nodes(s->net);
    std::vector<int32_t> grid(total), ty(nc), vo(nc);
    std::vector<double> state((size_t)S * nc);
    CW_CUDA(cudaMemcpyAsync(grid.data(), l->grid, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(ty.data(), l->type, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(vo.data(), l->volume, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(state.data(), s->state, sizeof(double) * state.size(), cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    const std::vector<double> &fresh = network_initial(s->lesion_net);
    bool joined = false;
    for (uint32_t h = 0; h < c.nh; ++h) {
        const int64_t c0 = l->cell_off[h], cap = l->cell_off[h + 1] - c0;
        const int32_t W = s->w[h], H = s->h[h];
        const double cx = std::isnan(s->lesion_cx) ? (double)W / 2.0 : s->lesion_cx;
        const double cy = std::isnan(s->lesion_cy) ? (double)H / 2.0 : s->lesion_cy;
        std::vector<double> sx(cap, 0.0), sy(cap, 0.0);
        std::vector<uint32_t> n(cap, 0u);
        const int32_t *g = grid.data() + l->g.off[h];
        for (int32_t y = 0; y < H; ++y)
            for (int32_t x = 0; x < W; ++x) {
                const int32_t id = g[(int64_t)y * W + x];
                if (id < 0 || id >= cap) continue;
                sx[id] += (double)x + 0.5;
                sy[id] += (double)y + 0.5;
                n[id] += 1u;
            }
        std::vector<int64_t> joining;
        for (int64_t id = 1; id < cap; ++id) {
            const int64_t gi = c0 + id;
            const bool alive = vo[gi] > 0 && !((s->leaving >> (ty[gi] & 31)) & 1u);
            if (alive && n[id] > 0 &&
                std::hypot(sx[id] / (double)n[id] - cx, sy[id] / (double)n[id] - cy) <= s->lesion_radius)
                joining.push_back(gi);
        }
        if (joining.empty()) continue;
        const int32_t founded = (int32_t)s->clones.size();
        s->clones.push_back(s->lesion_net);
        s->clone_owned.push_back(0);
        s->clone_lesion.push_back(1);
        s->clone_parent.push_back(-1);
        cw_mutation none{};
        none.node = none.term = none.kind = none.change = none.source = -1;
        s->clone_mutation.push_back(none);
        for (int64_t gi : joining) {
            s->h_clone[gi] = founded;
            for (int k = 0; k < S; ++k) state[(size_t)k * nc + gi] = fresh[k];
        }
        joined = true;
    }
    if (!joined) return CW_OK;
    CW_CUDA(cudaMemcpyAsync(s->state, state.data(), sizeof(double) * state.size(), cudaMemcpyHostToDevice, stream()));
    return upload_clones(s, true);
}

// The division step (simulation.rs:1338-1347): every step, the ready cells
// of each history in id order as far as the living-cell limit allows, each
// daughter taking a copy of its parent's network state.
static int division_step(cw_sim_s *s) {
    const cw_sim_config &c = s->cfg;
    if (!c.divide) return CW_OK;
    const int64_t nc = s->nc;
    cw_lattice_s *l = s->lat;
    CW_CUDA(cudaMemsetAsync(l->div.count, 0, sizeof(int32_t), stream()));
    k_div_ready<<<(unsigned)blocks(nc), T, 0, stream()>>>(
        l->type, l->volume, l->d_cell_off, l->d_keys, l->g.d_dims, (int)c.nh, nc, s->leaving, s->state,
        network_role(s->net, 2), DIVISION_RATIO * (double)network_reference_volume(s->net),
        (const uint32_t *)l->d_flag, s->alive, l->div.flag, l->div.normal, l->div.count, s->d_step, c.divide_every,
        s->due);
    CW_LAUNCHED();
    int rc = lattice_divide_enqueue(l, s->alive, c.max_cells > 0 ? c.max_cells : DEFAULT_MAX_CELLS, s->state,
                                    network_nodes(s->net));
    if (rc == CW_OK && s->track) rc = evolve_after_division(s);
    if (rc != CW_OK || !s->due) return rc;
    k_cycle_births<<<(unsigned)blocks(nc), T, 0, stream()>>>(l->d_cell_off, (int)c.nh, nc, l->div.daughter, l->d_keys,
                                                             s->d_step, c.cycle_median, c.cycle_spread, s->began,
                                                             s->due, l->div.count);
    CW_LAUNCHED();
    return CW_OK;
}

// Exposure::level_at (types.rs:319-332): the intensity while on, else 0.
static double exposure_level(const cw_sim_config &c, uint64_t mcs) {
    if (c.exposure_intensity <= 0.0 || mcs < (uint64_t)c.exposure_start) return 0.0;
    if (c.exposure_on <= 0) return c.exposure_intensity;  // continuous
    const uint64_t period = std::max<uint64_t>((uint64_t)c.exposure_on + (uint64_t)c.exposure_off, 1);
    return (mcs - (uint64_t)c.exposure_start) % period < (uint64_t)c.exposure_on ? c.exposure_intensity : 0.0;
}

// settle_stress (simulation.rs:2015-2055) for the step `mcs`: zero while the
// exposure is off; otherwise the living (and, around a vessel, the medium)
// take it up, it is held at the level where the oxygen is held, and solved,
// from scratch and tightly when the level changed.
static int settle_stress(cw_sim_s *s, const cw_relax_opts &o, uint64_t mcs) {
    const cw_sim_config &c = s->cfg;
    cw_field_s *f = s->str;
    const double level = exposure_level(c, mcs);
    int rc;
    if (level == 0.0) {
        CW_CUDA(cudaMemsetAsync(f->c, 0, sizeof(double) * (size_t)f->g.total, stream()));
        s->str_level = 0.0;
    } else {
        if ((rc = couple_uptake_device(f, s->lat, s->d_str_uptake, 8, f->uptake, s->sites)) != CW_OK) return rc;
        if (c.o2_hold == 4 &&
            (rc = couple_background_device(f, s->lat, c.exposure_uptake, f->uptake)) != CW_OK)
            return rc;
        k_hold_like<<<(unsigned)blocks(f->g.total), T, 0, stream()>>>(s->o2->held, f->g.total, level, f->held, f->c);
        CW_LAUNCHED();
        f->held_dirty = true;
        cw_relax_opts os = o;
        os.tolerance = 0.01 * c.exposure_uptake;  // OXYGEN_TOLERANCE x the exposure's uptake
        if (level != s->str_level) { os.tolerance = 1e-8; os.max_sweeps = 2000000; }
        s->last_str.resize(c.nh);
        const double *om = c.omega > 0.0 ? nullptr : s->omega[0].data();
        if ((rc = field_relax(f, &os, om, s->last_str.data())) != CW_OK) return rc;
        s->str_level = level;
    }
    if ((rc = couple_means_device(f, s->lat, s->sum, s->count, s->cell_str, s->sites)) != CW_OK) return rc;
    k_inputs_stress<<<(unsigned)blocks(s->nc), T, 0, stream()>>>(s->cell_str, s->nc, s->inputs);
    CW_LAUNCHED();
    return CW_OK;
}

// settle_bath_level (simulation.rs:2114-2125) from the field as solved.
static int settle_bath_level(cw_sim_s *s) {
    const int nh = (int)s->cfg.nh;
    CW_CUDA(cudaMemsetAsync(s->d_inflow, 0, sizeof(double) * nh, stream()));
    CW_CUDA(cudaMemsetAsync(s->d_free, 0, sizeof(unsigned long long) * nh, stream()));
    int rc = field_inflow_enqueue(s->o2, s->d_inflow, s->d_free);
    if (rc != CW_OK) return rc;
    k_bath_level<<<(unsigned)blocks(nh), T, 0, stream()>>>(nh, s->d_inflow, s->d_free, s->cfg.still_medium, s->level);
    CW_LAUNCHED();
    return CW_OK;
}

// Who takes up oxygen (declare_sources, simulation.rs:2138-2163): the
// first-order sinks by type (and of the medium), and with o2_uptake the
// zero-order uptake of every living cell's pixel (apply_uptake) and, around a
// vessel, of the medium too (apply_background_uptake).
static int paint_oxygen(cw_sim_s *s) {
    const cw_sim_config &c = s->cfg;
    int rc;
    if ((rc = couple_uptake_device(s->o2, s->lat, s->d_sink, 8, s->o2->lin_sink, s->sites)) != CW_OK) return rc;
    if (c.o2_background_sink > 0.0 &&
        (rc = couple_background_device(s->o2, s->lat, c.o2_background_sink, s->o2->lin_sink)) != CW_OK)
        return rc;
    s->o2->lin_sink_on = true;
    if (c.o2_uptake > 0.0) {
        if ((rc = couple_uptake_device(s->o2, s->lat, s->d_uptake, 8, s->o2->uptake, s->sites)) != CW_OK) return rc;
        if (c.o2_hold == 4 && (rc = couple_background_device(s->o2, s->lat, c.o2_uptake, s->o2->uptake)) != CW_OK)
            return rc;
    }
    return CW_OK;
}

static Leaving leaving_of(const cw_sim_s *s) {
    const cw_sim_config &c = s->cfg;
    return Leaving{c.differentiated_type, c.apoptotic_type, network_role(s->net, 3), network_role(s->net, 4),
                   s->lat->d_keys, s->lat->d_cell_off, (int32_t)c.nh};
}

// Every living cell's network: the one network, or in an evolving batch each
// cell under its clone's.
static int step_networks(cw_sim_s *s) {
    const cw_sim_config &c = s->cfg;
    const int64_t nc = s->nc;
    if (s->clone_nets)
        return network_step_clones_device(s->d_nets, s->d_clone, network_nodes(s->net), s->state, s->inputs, nc, nc,
                                          nc, c.dt, c.substeps, s->alive);
    return network_step_device(s->net, s->state, s->inputs, nc, nc, nc, c.dt, c.substeps, s->alive);
}

// One of the three phases of a step, enqueued without host synchronisation.
static int enqueue_phase(cw_sim_s *s, int p, const cw_relax_opts &o) {
    const cw_sim_config &c = s->cfg;
    const int64_t nc = s->nc;
    int rc;
    if (p == 0) {
        if ((rc = paint_oxygen(s)) != CW_OK) return rc;
        return field_relax_enqueue(s->o2, &o, s->budget[0], &s->gstart[0]);
    }
    if (p == 1) {
        if ((rc = couple_means_device(s->o2, s->lat, s->sum, s->count, s->cell_o2, s->sites)) != CW_OK) return rc;
        k_inputs<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->lat->type, s->lat->volume, s->lat->d_cell_off, c.nh, nc,
                                                           s->leaving, s->cell_o2, 0.2,
                                                           (double)std::max(network_reference_volume(s->net), 1u),
                                                           s->inputs, s->alive);
        CW_LAUNCHED();
        if (!s->sig) return CW_OK;
        k_secretion<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->alive, s->cell_o2, nc, c.hypoxic_level,
                                                              c.signal_secretion, s->secretion);
        CW_LAUNCHED();
        if ((rc = couple_production_device(s->sig, s->lat, s->secretion, s->sites)) != CW_OK) return rc;
        return field_relax_enqueue(s->sig, &o, s->budget[1], &s->gstart[1]);
    }
    if (s->sig && (rc = couple_means_device(s->sig, s->lat, s->sum, s->count, s->cell_sig, s->sites)) != CW_OK)
        return rc;
    if ((rc = step_networks(s)) != CW_OK) return rc;
    if ((rc = network_mechanics_device(s->net, s->state, nc, nc, s->target32)) != CW_OK) return rc;
    k_fates<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->alive, s->state, nc, network_role(s->net, 1),
                                                      c.death_threshold, c.necrotic_type, s->target32, s->lat->type,
                                                      s->lat->volume, s->lat->target, s->lat->lambda, c.lambda_volume,
                                                      s->died_at, s->d_step, s->began, s->due,
                                                          s->debris_on ? s->debris.kept : nullptr, leaving_of(s));
    CW_LAUNCHED();
    for (int k = 0; k < c.sweeps; ++k)
        if ((rc = lattice_sweep(s->lat)) != CW_OK) return rc;
    if ((rc = division_step(s)) != CW_OK) return rc;
    k_step_advance<<<1, 1, 0, stream()>>>(s->d_step);
    CW_LAUNCHED();
    return CW_OK;
}

static int outer_budget(const std::vector<cw_relax_stats> &st, int inner) {
    int64_t most = 0;
    for (auto &x : st) most = std::max<int64_t>(most, x.sweeps);
    return (int)((most + inner - 1) / inner) + 1;
}

static int build_graphs(cw_sim_s *s, const cw_relax_opts &o) {
    drop_graphs(s);
    if (s->budget[0] <= 0) s->budget[0] = outer_budget(s->last, o.inner_sweeps);
    if (s->budget[1] <= 0) s->budget[1] = outer_budget(s->last_sig, o.inner_sweeps);
    // the factors the graphs will use: the configuration's or the tuned ones
    int rc0;
    for (int fi = 0; fi < 2; ++fi) {
        cw_field_s *f = fi == 0 ? s->o2 : s->sig;
        if (!f) continue;
        std::vector<double> om(s->cfg.nh, s->cfg.omega);
        if (s->cfg.omega <= 0.0) om = s->omega[fi];
        if ((rc0 = field_dc_prepare(f, s->depth, s->sor_window, om)) != CW_OK) return rc0;
    }
    const uint32_t mcs = s->lat->mcs;
    for (int p = 0; p < 3; ++p) {
        cudaGraph_t g = nullptr;
        CW_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
        const uint64_t before = cw_launch_count();
        int rc = enqueue_phase(s, p, o);
        cudaError_t e = cudaStreamEndCapture(stream(), &g);
        if (rc != CW_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        s->gkernels[p] = cw_launch_count() - before;
        e = cudaGraphInstantiate(&s->gexec[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    s->lat->mcs = mcs;  // the capture ran no sweep
    s->graphs = true;
    return CW_OK;
}

// Collect a graph's solve; finish it host-side if its budget fell short.
static int settle(cw_sim_s *s, int which, const cw_relax_opts &o, std::vector<cw_relax_stats> &st) {
    cw_field_s *f = which == 0 ? s->o2 : s->sig;
    bool ok = false;
    int rc = field_relax_collect(f, st, ok);
    if (rc != CW_OK) return rc;
    s->need[which] = std::max(s->need[which], outer_budget(st, o.inner_sweeps) - 1);
    if (ok) return CW_OK;
    s->budget_misses += 1;
    if ((rc = field_relax_finish(f, &o, s->gstart[which])) != CW_OK) return rc;
    if ((rc = field_relax_collect(f, st, ok)) != CW_OK) return rc;
    if (!ok) return fail(CW_ERR_SIMULATION, "diffusion did not settle within the sweep limit");
    s->budget[which] += 1;  // rebuilt with room for one more next step
    drop_graphs(s);
    return CW_OK;
}

static int step_graph(cw_sim_s *s, const cw_relax_opts &o) {
    int rc;
    CW_CUDA(cudaGraphLaunch(s->gexec[0], stream()));
    count_launch(s->gkernels[0]);
    if ((rc = settle(s, 0, o, s->last)) != CW_OK) return rc;
    if (!s->graphs) {  // rebuilt below; finish this step on the plain path
        for (int p = 1; p < 3; ++p) {
            if ((rc = enqueue_phase(s, p, o)) != CW_OK) return rc;
            if (p == 1 && s->sig && (rc = settle(s, 1, o, s->last_sig)) != CW_OK) return rc;
        }
        return CW_OK;
    }
    CW_CUDA(cudaGraphLaunch(s->gexec[1], stream()));
    count_launch(s->gkernels[1]);
    if (s->sig && (rc = settle(s, 1, o, s->last_sig)) != CW_OK) return rc;
    if (!s->graphs) return enqueue_phase(s, 2, o);
    CW_CUDA(cudaGraphLaunch(s->gexec[2], stream()));
    count_launch(s->gkernels[2]);
    s->lat->mcs += (uint32_t)s->cfg.sweeps;
    s->graph_steps += 1;
    // every 8 steps, trim a budget well above what the solves needed: kernels
    // of a settled history exit at once, but their launches still cost
    if (++s->window >= 8) {
        bool rebuild = false;
        for (int w = 0; w < 2; ++w)
            if (s->need[w] > 0 && s->budget[w] > s->need[w] + 2) { s->budget[w] = s->need[w] + 1; rebuild = true; }
        s->need[0] = s->need[1] = 0;
        s->window = 0;
        if (rebuild) drop_graphs(s);
    }
    return CW_OK;
}

int cw_sim_step(cw_sim s, uint32_t nsteps) {
    CW_SCOPE(s);
    const cw_sim_config &c = s->cfg;
    int64_t nc = s->nc;
    int S = network_nodes(s->net);
    int survival = network_role(s->net, 1);
    cw_relax_opts o{};
    o.omega = c.omega;
    o.stop = c.stop_rule == CW_STOP_MAX_CHANGE ? CW_STOP_MAX_CHANGE : CW_STOP_RESIDUAL;
    o.tolerance = c.tolerance;
    o.error_tolerance = c.error_tolerance;
    o.max_sweeps = 200000;
    o.precision = c.precision;
    // 64 FP32 sweeps a correction: a volume's solve takes hundreds of sweeps,
    // and on the plane's batched campaign (fields to residual 1e-8) 64 took
    // 12.3 ms a step against 12.8 for 48, 13.1 for 32 and 14.8 for 16
    o.inner_sweeps = c.inner_sweeps > 0 ? c.inner_sweeps : 64;
    int rc;
    for (uint32_t step = 0; step < nsteps; ++step, ++s->steps) {
        if (s->lesion_net && (int64_t)s->steps == s->lesion_at && (rc = place_lesion(s)) != CW_OK) return rc;
        if (s->tracing && (int64_t)s->steps == (int64_t)c.tracing_at && (rc = mark_every_cell(s)) != CW_OK)
            return rc;
        bool solve = c.relax_every <= 1 || (s->steps % (uint32_t)c.relax_every) == 0;
        o.block_depth = s->depth;
        o.window = s->sor_window;
        const bool graph_ok = c.use_graphs && c.precision == CW_FP32_DC && c.relax_every <= 1 && !s->tune.active &&
                              s->depth_tuned && s->steps >= 2 && !s->last.empty() &&
                              (!s->sig || !s->last_sig.empty()) && !s->wst && !s->nfc && c.o2_hold != 3 &&
                              !s->debris_on && !s->str && !s->track && !c.field_off;
        if (graph_ok) {
            if (!s->graphs && (rc = build_graphs(s, o)) != CW_OK) return rc;
            if ((rc = step_graph(s, o)) != CW_OK) return rc;
            continue;
        }
        bool tuning = solve && s->tune.active && s->steps > 0;  // the first solve starts from scratch: not booked
        if (tuning) tune_assign(s);
        // with the field off nothing consumes: the oxygen stays at its start
        // and is not solved (field_is_off, simulation.rs:2127-2131)
        const bool o2_solve = solve && !c.field_off;
        if (o2_solve && s->bath) {
            // the bath of the lattice as it stands (hold_medium_bath, coupling.rs:156-158)
            if ((rc = lattice_bath_enqueue(s->lat, s->bath)) != CW_OK) return rc;
            if (c.o2_hold == 3) {
                k_hold_from_mask<<<(unsigned)blocks(s->o2->g.total), T, 0, stream()>>>(
                    s->bath, s->o2->g.total, 1.0, s->o2->held, s->o2->c, s->level, s->lat->g.d_off, (int)c.nh);
                CW_LAUNCHED();
                s->o2->held_dirty = true;
            }
        }
        if (o2_solve) {
            // 1. downward coupling and the oxygen solve
            if ((rc = paint_oxygen(s)) != CW_OK) return rc;
            const double *om = c.omega > 0.0 ? nullptr : s->omega[0].data();
            cw_relax_opts o1 = o;
            const bool warm = s->steps == 0 && c.first_tolerance > 0.0;
            if (warm) {
                // settled tightly once, from scratch (OXYGEN_WARMUP_*, simulation.rs:91-98)
                o1.tolerance = std::min(c.first_tolerance, c.tolerance);
                o1.max_sweeps = 2000000;
            }
            if ((rc = field_relax(s->o2, &o1, om, s->last.data())) != CW_OK) return rc;
            if (c.still_medium > 0.0) {
                // the level a step behind the field (settle_bath_level after start() and each solve)
                if ((rc = settle_bath_level(s)) != CW_OK) return rc;
                if (warm) {
                    k_hold_from_mask<<<(unsigned)blocks(s->o2->g.total), T, 0, stream()>>>(
                        s->bath, s->o2->g.total, 1.0, s->o2->held, s->o2->c, s->level, s->lat->g.d_off, (int)c.nh);
                    CW_LAUNCHED();
                    if ((rc = field_relax(s->o2, &o, om, s->last.data())) != CW_OK) return rc;
                    if ((rc = settle_bath_level(s)) != CW_OK) return rc;
                }
            }
            if (tuning) tune_book(s, 0, s->last);
            if (!s->depth_tuned && (rc = tune_depth(s)) != CW_OK) return rc;
        }
        // 2. what each cell sits in
        if ((rc = couple_means_device(s->o2, s->lat, s->sum, s->count, s->cell_o2, s->sites)) != CW_OK) return rc;
        k_inputs<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->lat->type, s->lat->volume, s->lat->d_cell_off, c.nh, nc,
                                                           s->leaving, s->cell_o2, 0.2,
                                                           (double)std::max(network_reference_volume(s->net), 1u),
                                                           s->inputs, s->alive);
        CW_LAUNCHED();
        if (s->sig && solve) {
            k_secretion<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->alive, s->cell_o2, nc, c.hypoxic_level,
                                                                  c.signal_secretion, s->secretion);
            CW_LAUNCHED();
            if ((rc = couple_production_device(s->sig, s->lat, s->secretion, s->sites)) != CW_OK) return rc;
            std::vector<cw_relax_stats> &st2 = s->last_sig;
            st2.resize(c.nh);
            const double *om = c.omega > 0.0 ? nullptr : s->omega[1].data();
            if ((rc = field_relax(s->sig, &o, om, st2.data())) != CW_OK) return rc;
            if (tuning) tune_book(s, 1, st2);
            if ((rc = couple_means_device(s->sig, s->lat, s->sum, s->count, s->cell_sig, s->sites)) != CW_OK)
                return rc;
        }
        // 2a. an exposure's stress (settle_stress, simulation.rs:1158-1162)
        if (s->str && solve) {
            if ((rc = settle_stress(s, o, s->steps)) != CW_OK) return rc;
        } else if (s->str) {
            k_inputs_stress<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->cell_str, nc, s->inputs);
            CW_LAUNCHED();
        }
        // 2b. the released fields: the waste from the living, the necrotic
        // factor from the dead, held at zero on the bath (settle_waste,
        // settle_necrotic_factor; simulation.rs:2057-2113)
        if ((s->wst || s->nfc) && solve) {
            k_release_rates<<<(unsigned)blocks(nc), T, 0, stream()>>>(
                s->alive, s->lat->type, s->lat->volume, s->died_at, s->d_step, nc, c.necrotic_type,
                c.waste_production, c.necrotic_production, c.necrotic_release_for, s->wst ? s->wst_rate : nullptr,
                s->nfc ? s->nfc_rate : nullptr);
            CW_LAUNCHED();
            cw_field_s *fs[2] = {s->wst, s->nfc};
            double *rates[2] = {s->wst_rate, s->nfc_rate};
            double *means[2] = {s->cell_wst, s->cell_nfc};
            std::vector<cw_relax_stats> *sts[2] = {&s->last_wst, &s->last_nfc};
            for (int q = 0; q < 2; ++q) {
                cw_field_s *f = fs[q];
                if (!f) continue;
                if ((rc = couple_production_device(f, s->lat, rates[q], s->sites)) != CW_OK) return rc;
                k_hold_from_mask<<<(unsigned)blocks(f->g.total), T, 0, stream()>>>(s->bath, f->g.total, 0.0, f->held,
                                                                                  f->c);
                CW_LAUNCHED();
                f->held_dirty = true;
                sts[q]->resize(c.nh);
                const double *om = c.omega > 0.0 ? nullptr : s->omega[0].data();
                if ((rc = field_relax(f, &o, om, sts[q]->data())) != CW_OK) return rc;
                if ((rc = couple_means_device(f, s->lat, s->sum, s->count, means[q], s->sites)) != CW_OK) return rc;
            }
            k_inputs_released<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->wst ? s->cell_wst : nullptr,
                                                                        s->nfc ? s->cell_nfc : nullptr, nc, s->inputs);
            CW_LAUNCHED();
        } else if (s->wst || s->nfc) {
            // a step between solves: the cells read the last means
            k_inputs_released<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->wst ? s->cell_wst : nullptr,
                                                                        s->nfc ? s->cell_nfc : nullptr, nc, s->inputs);
            CW_LAUNCHED();
        }
        // 3. every living network
        if ((rc = step_networks(s)) != CW_OK) return rc;
        // 4. fates and mechanics
        if ((rc = network_mechanics_device(s->net, s->state, nc, nc, s->target32)) != CW_OK) return rc;
        k_fates<<<(unsigned)blocks(nc), T, 0, stream()>>>(s->alive, s->state, nc, survival, c.death_threshold,
                                                          c.necrotic_type, s->target32, s->lat->type,
                                                          s->lat->volume, s->lat->target, s->lat->lambda,
                                                          c.lambda_volume, s->died_at, s->d_step, s->began, s->due,
                                                          s->debris_on ? s->debris.kept : nullptr, leaving_of(s));
        CW_LAUNCHED();
        // 4b. with a debris loss, the dead tissue's debris lost at its edge and
        // the fluid shut in drained (simulation.rs:1311-1315)
        if (s->debris_on) {
            if ((rc = debris_break_down_enqueue(s->lat, s->debris, c.debris_loss, c.necrotic_type, s->d_step)) !=
                CW_OK)
                return rc;
            if ((rc = lattice_bath_enqueue(s->lat, s->bath)) != CW_OK) return rc;
            if ((rc = debris_drain_enqueue(s->lat, s->debris, s->bath, c.necrotic_type, s->d_step)) != CW_OK)
                return rc;
            if (s->lat->surface_on && (rc = lattice_recount_surfaces(s->lat)) != CW_OK) return rc;
        }
        // 5. the lattice, then 6. division
        for (int k = 0; k < c.sweeps; ++k)
            if ((rc = lattice_sweep(s->lat)) != CW_OK) return rc;
        if ((rc = division_step(s)) != CW_OK) return rc;
        k_step_advance<<<1, 1, 0, stream()>>>(s->d_step);
        CW_LAUNCHED();
        if (tuning && ++s->tune.done >= s->tune.steps) tune_finish(s);
        (void)S;
    }
    return CW_OK;
}

int cw_sim_graph_info(cw_sim s, uint64_t *graph_steps, uint64_t *budget_misses, int32_t *budgets) {
    CW_SCOPE(s);
    if (graph_steps) *graph_steps = s->graph_steps;
    if (budget_misses) *budget_misses = s->budget_misses;
    if (budgets) { budgets[0] = s->budget[0]; budgets[1] = s->budget[1]; }
    return CW_OK;
}

int cw_sim_tuning(cw_sim s, double *omega_o2, double *omega_signal, int32_t *depth, int32_t *window,
                  int32_t *tuning) {
    CW_SCOPE(s);
    for (uint32_t k = 0; k < s->cfg.nh; ++k) {
        if (omega_o2) omega_o2[k] = s->omega[0][k];
        if (omega_signal) omega_signal[k] = s->omega[1][k];
    }
    if (depth) *depth = s->depth;
    if (window) *window = s->sor_window;
    if (tuning) *tuning = s->tune.active ? 1 : 0;
    return CW_OK;
}

// The simulation's stream is its lattice's and fields' too.
int cw_sim_set_stream(cw_sim s, void *stream) {
    CW_SCOPE(s);
    // the old stream's work finishes first (set synchronises it)
    int rc = s->hs.set((cudaStream_t)stream);
    if (rc != CW_OK) return rc;
    // the children follow the simulation's stream without owning it
    if (s->lat) { s->lat->hs.stream = s->hs.stream; s->lat->hs.own = false; }
    cw_field_s *fs[5] = {s->o2, s->sig, s->wst, s->nfc, s->str};
    for (cw_field_s *f : fs)
        if (f) { f->hs.stream = s->hs.stream; f->hs.own = false; }
    return CW_OK;
}

void *cw_sim_get_stream(cw_sim s) { return (void *)s->hs.stream; }

const char *cw_sim_last_error(cw_sim s) { return s->hs.err.c_str(); }

int cw_sim_clones(cw_sim s, uint32_t hist, uint32_t n, int32_t *clone) {
    CW_SCOPE(s);
    if (hist >= s->cfg.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    const int64_t c0 = s->lat->cell_off[hist], cap = s->lat->cell_off[hist + 1] - c0;
    if ((int64_t)n > cap) return fail(CW_ERR_CONFIG, "history " + std::to_string(hist) + " holds " +
                                                         std::to_string(cap) + " records");
    for (uint32_t k = 0; k < n; ++k) clone[k] = s->track ? s->h_clone[c0 + k] : 0;
    return CW_OK;
}

int cw_sim_clone_count(cw_sim s, uint32_t *nclones) {
    *nclones = s->track ? (uint32_t)s->clones.size() : 1u;
    return CW_OK;
}

int cw_sim_clone_records(cw_sim s, uint32_t *count, int32_t *parent, cw_mutation *mutation) {
    if (count) *count = (uint32_t)s->clone_parent.size();
    for (size_t k = 0; k < s->clone_parent.size(); ++k) {
        if (parent) parent[k] = s->clone_parent[k];
        if (mutation) mutation[k] = s->clone_mutation[k];
    }
    return CW_OK;
}

int cw_sim_traced(cw_sim s, uint32_t hist, uint32_t cap, uint32_t *marks, uint64_t *cells, uint32_t *n) {
    CW_SCOPE(s);
    if (!s->tracing) return fail(CW_ERR_CONFIG, "this simulation traces no lineage");
    if (hist >= s->cfg.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    std::vector<int32_t> ty, vo;
    int rc = records_to_host(s, ty, vo);
    if (rc != CW_OK) return rc;
    const int64_t c0 = s->lat->cell_off[hist], c1 = s->lat->cell_off[hist + 1];
    std::map<int32_t, uint64_t> count;
    for (int64_t g = c0 + 1; g < c1; ++g)
        if (s->h_mark[g] >= 0 && in_layer(s, ty, vo, g)) count[s->h_mark[g]] += 1;
    uint32_t k = 0;
    for (const auto &mc : count) {
        if (k < cap) {
            if (marks) marks[k] = (uint32_t)mc.first;
            if (cells) cells[k] = mc.second;
        }
        ++k;
    }
    *n = k;
    return CW_OK;
}

int cw_sim_lattice(cw_sim s, cw_lattice *lat) {
    CW_SCOPE(s);
    *lat = s->lat;
    return CW_OK;
}

int cw_sim_field(cw_sim s, int32_t which, cw_field *f) {
    CW_SCOPE(s);
    *f = which == 0 ? s->o2 : which == 1 ? s->sig : which == 2 ? s->wst : which == 3 ? s->nfc
       : which == 4 ? s->str : nullptr;
    if (!*f) return fail(CW_ERR_NOT_FOUND, "no such field");
    return CW_OK;
}

int cw_sim_stats(cw_sim s, double *out) {
    CW_SCOPE(s);
    uint32_t nh = s->cfg.nh;
    double *d_out;
    int rc = dalloc(&d_out, 4 * (size_t)nh);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * 4 * nh, stream()));
    k_stats<<<nh, 256, 0, stream()>>>(s->alive, s->cell_o2, s->lat->volume, s->lat->d_cell_off, nh, d_out);
    CW_LAUNCHED();
    CW_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * 4 * nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_out);
    if ((rc = lattice_pass_error(s->lat)) != CW_OK) return rc;
    if (s->bath && (rc = lattice_bath_error()) != CW_OK) return rc;
    for (uint32_t k = 0; k < nh; ++k) {
        out[4 * k + 2] = (double)s->last[k].sweeps;
        out[4 * k + 3] = s->last[k].residual;
    }
    return CW_OK;
}

int cw_sim_touches_edge(cw_sim s, int32_t *out) {
    CW_SCOPE(s);
    const cw_sim_config &c = s->cfg;
    int32_t *d_out = nullptr;
    int rc = dalloc(&d_out, c.nh);
    if (rc != CW_OK) return rc;
    CW_CUDA(cudaMemsetAsync(d_out, 0, sizeof(int32_t) * c.nh, stream()));
    const int64_t n = s->lat->g.total;
    // in a volume the vessel runs through the front and back faces
    k_touches_edge<<<(unsigned)((n + T - 1) / T), T, 0, stream()>>>(s->lat->grid, s->lat->g.d_dims, s->lat->g.d_off,
                                                                   (int)c.nh, c.o2_hold == 4 ? 0 : 1, d_out);
    CW_LAUNCHED();
    CW_CUDA(cudaMemcpyAsync(out, d_out, sizeof(int32_t) * c.nh, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_out);
    return CW_OK;
}

int cw_sim_measure(cw_sim s, cw_measurements *out) {
    CW_SCOPE(s);
    const cw_sim_config &c = s->cfg;
    const uint32_t nh = c.nh;
    cw_lattice_s *l = s->lat;
    const bool lined = c.o2_hold == 0 || c.o2_hold == 1;
    std::vector<int64_t> loff(nh + 1, 0);
    for (uint32_t k = 0; k < nh; ++k) loff[k + 1] = loff[k] + (c.o2_hold == 1 ? s->h[k] : s->w[k]);
    unsigned long long *d_out;
    uint8_t *d_lines = nullptr;
    int64_t *d_loff = nullptr;
    int rc;
    if ((rc = dalloc(&d_out, MEASURES * (size_t)nh)) != CW_OK) return rc;
    if (lined && ((rc = dalloc(&d_lines, (size_t)loff[nh])) || (rc = dalloc(&d_loff, nh + 1)))) return rc;
    if (lined) {
        CW_CUDA(cudaMemsetAsync(d_lines, 0, (size_t)loff[nh], stream()));
        CW_CUDA(cudaMemcpyAsync(d_loff, loff.data(), sizeof(int64_t) * (nh + 1), cudaMemcpyHostToDevice, stream()));
        k_measure_lines<<<s->sites.nblocks, T, 0, stream()>>>(l->grid, l->type, l->volume, l->d_cell_off, l->g.d_dims,
                                                              l->g.d_off, s->sites.d_blk, (int)nh, c.necrotic_type,
                                                              c.o2_hold == 1 ? 1 : 0, d_loff, d_lines);
        CW_LAUNCHED();
    }
    k_measure<<<nh, 256, 0, stream()>>>(l->type, l->volume, l->d_cell_off, l->d_used, c.necrotic_type,
                                        c.differentiated_type, c.apoptotic_type, s->state, network_role(s->net, 2),
                                        s->nc, d_lines, d_loff, d_out);
    CW_LAUNCHED();
    std::vector<unsigned long long> h(MEASURES * (size_t)nh);
    CW_CUDA(cudaMemcpyAsync(h.data(), d_out, sizeof(unsigned long long) * MEASURES * nh, cudaMemcpyDeviceToHost,
                            stream()));
    // clones with a living cell (measure.rs: clone_sizes), from the records on the host
    std::vector<int32_t> ty, vo;
    if (s->track) {
        ty.resize(s->nc);
        vo.resize(s->nc);
        CW_CUDA(cudaMemcpyAsync(ty.data(), l->type, sizeof(int32_t) * s->nc, cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaMemcpyAsync(vo.data(), l->volume, sizeof(int32_t) * s->nc, cudaMemcpyDeviceToHost, stream()));
    }
    CW_CUDA(cudaStreamSynchronize(stream()));
    dfree(d_out);
    dfree(d_lines);
    dfree(d_loff);
    const double pi = 3.14159265358979323846;
    for (uint32_t k = 0; k < nh; ++k) {
        const unsigned long long *v = &h[MEASURES * (size_t)k];
        cw_measurements &m = out[k];
        m.mcs = s->steps > 0 ? s->steps - 1 : 0;
        m.exposure = exposure_level(c, m.mcs);
        m.cycling = v[0];
        m.quiescent = v[1];
        m.necrotic = v[2];
        m.born = v[5];
        m.gone = v[6];
        m.differentiating = v[8];
        m.apoptotic = v[9];
        if (s->track) {
            std::vector<int32_t> seen;
            uint64_t lesion = 0;
            const int64_t c0 = l->cell_off[k], c1 = l->cell_off[k + 1];
            for (int64_t g = c0 + 1; g < c1; ++g)
                if (vo[g] > 0 && !((s->leaving >> (ty[g] & 31)) & 1u)) {
                    seen.push_back(s->h_clone[g]);
                    lesion += s->clone_lesion[s->h_clone[g]];
                }
            std::sort(seen.begin(), seen.end());
            m.clones = (uint64_t)(std::unique(seen.begin(), seen.end()) - seen.begin());
            // living cells descended from a lesion (lesion_cells, evolution.rs:182-197)
            m.lesion = lesion;
        } else {
            m.clones = v[0] + v[1] > 0 ? 1 : 0;
            m.lesion = 0;
        }
        // the held column of o2_hold 1, the vessel of 4: the lattice's only obstacles
        m.vessel = (c.o2_hold == 1 || c.o2_hold == 4) ? s->obstacles[k] : 0;
        const uint32_t D = s->d[k];
        // radius_of (measure.rs:103-113): a disc in the plane, a ball in a volume
        auto radius = [&](uint64_t size) {
            if (D <= 1) return std::sqrt((double)size / pi);
            if (c.o2_hold == 4) return std::sqrt((double)size / (pi * (double)D));  // a cylinder as long as the box
            return std::cbrt(3.0 * (double)size / (4.0 * pi));
        };
        const uint64_t living = v[3], dead = v[4], leaving = v[10];
        m.tissue_radius = radius(m.vessel + living + dead + leaving);
        m.necrotic_radius = radius(dead);
        if (c.o2_hold == 0) m.viable_depth = v[7] == 0 ? 0.0 : (double)living / (double)v[7];
        else if (c.o2_hold == 1) m.viable_depth = v[7] == 0 ? 0.0 : (double)living / (2.0 * (double)v[7]);
        else if (c.o2_hold == 4) m.viable_depth = radius(m.vessel + living) - radius(m.vessel);
        else m.viable_depth = m.tissue_radius - m.necrotic_radius;
    }
    return CW_OK;
}

int cw_sim_network_state(cw_sim s, uint32_t hist, uint32_t n, double *state) {
    CW_SCOPE(s);
    if (hist >= s->cfg.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    int S = network_nodes(s->net);
    int64_t c0 = s->lat->cell_off[hist], cap = s->lat->cell_off[hist + 1] - c0;
    if ((int64_t)n > cap) return fail(CW_ERR_CONFIG, "more cells asked for than the history holds");
    std::vector<double> col(n);
    for (int i = 0; i < S; ++i) {
        CW_CUDA(cudaMemcpyAsync(col.data(), s->state + (size_t)i * s->nc + c0, sizeof(double) * n,
                                cudaMemcpyDeviceToHost, stream()));
        CW_CUDA(cudaStreamSynchronize(stream()));
        for (uint32_t cc = 0; cc < n; ++cc) state[(size_t)cc * S + i] = col[cc];
    }
    return CW_OK;
}

int cw_sim_cycle(cw_sim s, uint32_t hist, uint32_t n, int32_t *began, int32_t *due) {
    CW_SCOPE(s);
    if (hist >= s->cfg.nh) return fail(CW_ERR_NOT_FOUND, "no history " + std::to_string(hist));
    if (!s->due) return fail(CW_ERR_CONFIG, "this simulation has no cell cycle");
    int64_t c0 = s->lat->cell_off[hist], cap = s->lat->cell_off[hist + 1] - c0;
    if ((int64_t)n > cap) return fail(CW_ERR_CONFIG, "more cells asked for than the history holds");
    CW_CUDA(cudaMemcpyAsync(began, s->began + c0, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaMemcpyAsync(due, s->due + c0, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream()));
    CW_CUDA(cudaStreamSynchronize(stream()));
    return CW_OK;
}

}  // extern "C"
