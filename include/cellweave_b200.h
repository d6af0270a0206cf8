/*
 * cellweave_b200.h -- the C ABI of cellweave's per-step hot path on one B200.
 *
 * The reference (ngodzik/cellweave v0.3.0) is a Rust library whose hot path
 * is three objects and the glue between them:
 *   CpmLattice   crates/engine/src/cpm.rs:187-1041     -> cw_lattice
 *   ScalarField  crates/engine/src/pde.rs:30-640        -> cw_field
 *   Network      crates/engine/src/network.rs:247-822   -> cw_network
 *   coupling::*  crates/engine/src/coupling.rs:26-182   -> cw_couple_*
 *   Simulation<Running>::step, simulation.rs:1129-1350  -> cw_sim (driver)
 * Each entry point below names the reference method it replaces.
 *
 * Conventions.
 *  - Every function returns a status: CW_OK, or the CellweaveError variant
 *    the reference would return (crates/core/src/error.rs:7-23), plus
 *    CW_ERR_CUDA and CW_ERR_TIMEOUT.  cw_last_error() gives the message of
 *    the last failure on the calling thread.
 *  - Handles own their device buffers (as the reference's objects own their
 *    Vecs).  Host pointers are borrowed for the duration of the call only.
 *  - One handle holds one history or a batch of independent histories of
 *    uneven sizes ("hist" selects one); a plain single history is a batch of
 *    one.  Cell ids are per history, 0 the medium, -1 the obstacle
 *    (u32::MAX in the reference: the same bits).
 *  - Every handle queues its work on its own CUDA stream, created with it
 *    (a simulation's lattice and fields share the simulation's; a fit takes
 *    its lattice's); cw_*_set_stream hands in the caller's stream instead.
 *    A call that reads two handles (cw_couple_*) orders their streams with
 *    events.  Calls that return host data synchronise the handle's stream.
 *    One host thread at a time per handle, as the reference's &mut receivers
 *    require (simulation.rs:456); different handles may be driven from
 *    different threads at once.  cw_*_last_error(h) gives the message of the
 *    last failure of a call on h, cw_last_error() that of the calling thread.
 *    Calls without a handle (cw_field_relax_noalloc, cw_event_record,
 *    cw_network_step_clones) use the library stream (cw_set_stream).
 *  - No CPU path: without a usable CUDA device every call that would launch
 *    work returns CW_ERR_CUDA.
 */
#ifndef CELLWEAVE_B200_H
#define CELLWEAVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CW_OK = 0,
    CW_ERR_CONFIG = 1,     /* CellweaveError::Config */
    CW_ERR_SIMULATION = 2, /* CellweaveError::Simulation, e.g. a field that did not settle */
    CW_ERR_ODE = 3,        /* CellweaveError::OdeSolver */
    CW_ERR_NOT_FOUND = 4,  /* CellweaveError::NotFound */
    CW_ERR_CUDA = 5,       /* a CUDA call failed, or no device */
    CW_ERR_TIMEOUT = 6     /* a bounded device loop ran out of iterations */
};

typedef struct cw_lattice_s *cw_lattice;
typedef struct cw_field_s *cw_field;
typedef struct cw_network_s *cw_network;
typedef struct cw_sim_s *cw_sim;
typedef struct cw_fit_s *cw_fit;

/* ------------------------------------------------------------------ library */
const char *cw_last_error(void);
int cw_version(void);
/* The library stream, for calls without a handle (a cudaStream_t); NULL
 * restores the library's own. */
int cw_set_stream(void *stream);
/* Each handle's stream (a cudaStream_t): the caller's, or NULL for a new one
 * of the handle's own; work queued before finishes first.  A simulation's
 * lattice and fields follow cw_sim_set_stream (do not set theirs apart).
 * The per-handle streams stand for the reference's exclusive &mut borrow of
 * each object (simulation.rs:456): handles on different streams run at once. */
int cw_lattice_set_stream(cw_lattice lat, void *stream);
int cw_field_set_stream(cw_field f, void *stream);
int cw_network_set_stream(cw_network net, void *stream);
int cw_sim_set_stream(cw_sim sim, void *stream);
void *cw_lattice_get_stream(cw_lattice lat);
void *cw_field_get_stream(cw_field f);
void *cw_network_get_stream(cw_network net);
void *cw_sim_get_stream(cw_sim sim);
/* The message of the last failure of a call on the handle ("" if none). */
const char *cw_lattice_last_error(cw_lattice lat);
const char *cw_field_last_error(cw_field f);
const char *cw_network_last_error(cw_network net);
const char *cw_sim_last_error(cw_sim sim);
const char *cw_fit_last_error(cw_fit fit);
/* The CUDA device the library works on (one per process). */
int cw_set_device(int32_t device);
void *cw_get_stream(void);
int cw_synchronize(void);
/* Kernels this library has launched since it was loaded. */
uint64_t cw_launch_count(void);
/* Failure tests, no counterpart in the reference (its loops cannot hang):
 * make the library's bounded device waits run out without faulting the GPU.
 * wait_ns (1 ms to 2 s; 0: the default 2 s) limits every grid-barrier and
 * TMA-copy wait; withhold_block >= 0 keeps that block of each sublattice pass
 * from arriving at its grid barriers (the others give up: CW_ERR_TIMEOUT);
 * max_rounds > 0 caps a pass's priority rounds (past it: CW_ERR_SIMULATION);
 * skip_tma != 0 makes the FP32 sweeps issue no TMA copy, so their waits run
 * out (CW_ERR_TIMEOUT).  Every call replaces all four; (0, -1, 0, 0) is the
 * default.  Work captured in a CUDA graph keeps the settings of its capture. */
int cw_test_faults(uint64_t wait_ns, int32_t withhold_block, int32_t max_rounds, int32_t skip_tma);
/* CUDA events on the library stream, in slots 0..15, for timing.  cw_synchronize
 * waits for every stream of the device. */
int cw_event_record(int32_t slot);
/* The same on a given stream (a handle's, from cw_*_get_stream); NULL: the library stream. */
int cw_event_record_on(void *stream, int32_t slot);
int cw_event_elapsed(int32_t a, int32_t b, float *ms);
/* cudaProfilerStart / cudaProfilerStop around a region (for ncu --profile-from-start off). */
int cw_profiler_start(void);
int cw_profiler_stop(void);

/* ------------------------------------------------------------------ lattice
 * CpmLattice::with_depth (cpm.rs:231-259) for `nh` histories at once.  A
 * side of 0 or above 65535 is CW_ERR_CONFIG (CpmError::InvalidDims,
 * cpm.rs:18-22).  cell_capacity[h] bounds the ids of history h (medium
 * included); the grid starts as medium, with no records but the medium's. */
int cw_lattice_create(uint32_t nh, const uint32_t *w, const uint32_t *h, const uint32_t *d,
                      const uint32_t *cell_capacity, double temperature, cw_lattice *out);
int cw_lattice_destroy(cw_lattice lat);
int cw_lattice_count(cw_lattice lat, uint32_t *nh);
/* The cell records history `hist` holds (its capacity, the medium's included). */
int cw_lattice_capacity(cw_lattice lat, uint32_t hist, uint32_t *cap);
/* The most rounds a sublattice pass needed since the last call (a pass runs
 * its attempts that share no cell at once, the others in later rounds);
 * resets the count.  A diagnostic; no counterpart in the reference. */
int cw_lattice_pass_rounds(cw_lattice lat, uint32_t *rounds);
/* ContactEnergy (cpm.rs:30-129) generalised to a K x K table over cell types
 * (K <= 8, symmetric, J[0] the medium-medium 0), and set_contact_order
 * (cpm.rs:274-301): 1 faces only, 2 and 3 the wider reach and its divisor. */
int cw_lattice_set_contact(cw_lattice lat, int32_t K, const double *J, int32_t order);
int cw_lattice_set_temperature(cw_lattice lat, double temperature);
/* The medium the bath reaches in history `hist`: out[i] = 1 for the pixels
 * hold_medium_bath would hold (coupling.rs:156-158, pde.rs:550-631: medium
 * joined to the box's outer layer through medium, 4-connected in the plane,
 * 6-connected in a volume), 0 elsewhere.  out holds one byte per pixel. */
int cw_lattice_bath(cw_lattice lat, uint32_t hist, uint8_t *out);
/* divide_across (cpm.rs:1087-1160) for cells `ids` of history `hist`, each
 * across the plane through its centre of mass with normal normals[3k..3k+2]
 * (the third component counts in a volume only): the pixels on the side the
 * normal points to go to a new cell of the same kind and volume parameters,
 * whose id (the next free record, in the order of `ids` sorted by id) is
 * written to daughters[k]; -1 where nothing changed (the medium, fewer than
 * 8 pixels, a plane that leaves one side empty, no free record). */
int cw_lattice_divide(cw_lattice lat, uint32_t hist, uint32_t n, const int32_t *ids, const double *normals,
                      int32_t *daughters);
/* The records history `hist` uses (the medium's included): cells set, plus
 * the daughters of divisions. */
int cw_lattice_cell_count(cw_lattice lat, uint32_t hist, uint32_t *n);
/* Where a copy attempt takes its id from: CW_COPY_VON_NEUMANN, a face
 * neighbour as try_flip does (cpm.rs:797-838, 922-944; the default), or
 * CW_COPY_MOORE, any in-box pixel at Chebyshev distance 1 (an extension). */
enum { CW_COPY_VON_NEUMANN = 0, CW_COPY_MOORE = 1 };
int cw_lattice_set_copy_nbhd(cw_lattice lat, int32_t nbhd);
/* The update order's kinetics (no counterpart in the reference, whose
 * random pixels attempt each pixel Poisson(1) times a Monte Carlo step).
 * 1, the default: a Monte Carlo step sweeps every colour once and attempts
 * every pixel once, so a favoured copy happens at once where random pixels
 * take it with probability 1 - 1/e; driven shrinking and growth run faster.
 * n > 1: n sweeps of every colour, a pixel attempting in each with
 * probability 1/n (its own Philox draw), Binomial(n, 1/n) attempts a step,
 * which nears Poisson(1) as n grows; n times the passes. */
int cw_lattice_set_subsweeps(cw_lattice lat, int32_t subsweeps);
/* The grid of history `hist`, w*h*d int32 in the reference's flat order.  An upload holding an id
 * past the history's cell capacity (or below -1, the obstacle) is refused with CW_ERR_CONFIG naming
 * the first such pixel, and the lattice keeps its grid; the check runs on the device. */
int cw_lattice_upload(cw_lattice lat, uint32_t hist, const int32_t *grid);
int cw_lattice_download(cw_lattice lat, uint32_t hist, int32_t *grid);
/* Every history's grid at once, one after another in history order (the sum of w*h*d int32): one
 * copy, one check and one synchronisation for the whole batch (a campaign's grids in one buffer). */
int cw_lattice_upload_all(cw_lattice lat, const int32_t *grids);
int cw_lattice_download_all(cw_lattice lat, int32_t *grids);
/* Cell records (CellRecord, cpm.rs:171-181) for ids [0, n) of history `hist`:
 * type, volume, target volume, lambda_volume (set_volume_target, set_kind:
 * cpm.rs:997-1041). */
int cw_cells_set(cw_lattice lat, uint32_t hist, uint32_t n, const int32_t *type, const int32_t *volume,
                 const int32_t *target, const double *lambda);
int cw_cells_get(cw_lattice lat, uint32_t hist, uint32_t n, int32_t *type, int32_t *volume, int32_t *target,
                 double *lambda);
/* Surface constraint (an extension; off until set): lambda_S (S - S_target)^2,
 * S the number of faces a cell shares with other ids.  Surfaces are
 * recounted from the grid when this is called. */
int cw_cells_set_surface(cw_lattice lat, uint32_t hist, uint32_t n, const int32_t *target_surface,
                         const double *lambda_surface);
int cw_cells_get_surface(cw_lattice lat, uint32_t hist, uint32_t n, int32_t *surface);
/* Seed of history `hist`'s Philox stream, and the step counter of all. */
int cw_lattice_set_seed(cw_lattice lat, uint32_t hist, uint64_t seed);
int cw_lattice_set_mcs(cw_lattice lat, uint32_t mcs);
int cw_lattice_get_mcs(cw_lattice lat, uint32_t *mcs);
/* monte_carlo_step (cpm.rs:748-772) `sweeps` times on every history: one
 * copy attempt per pixel per step, made in sublattice passes so that no two
 * concurrent attempts share a contact neighbourhood. */
int cw_lattice_mcs(cw_lattice lat, uint32_t sweeps);
/* Delta-H (cpm.rs:841-894) of copying dst[k] into site[k] on history
 * `hist` as it stands, for n proposals: out[6k..6k+5] = contact numerator,
 * contact term, volume term, surface term, adhesion+volume, total. */
int cw_lattice_delta_h_batch(cw_lattice lat, uint32_t hist, uint32_t n, const int64_t *site, const int32_t *dst,
                             double *out);
/* records_match_grid (cpm.rs:1272-1279): *ok = 1 when every record's volume
 * (and surface, if on) equals the recount of history `hist`'s grid. */
int cw_lattice_verify(cw_lattice lat, uint32_t hist, int32_t *ok);

/* ------------------------------------------------------------------ field
 * ScalarField::with_depth (pde.rs:98-131) for `nh` histories. */
int cw_field_create(uint32_t nh, const uint32_t *w, const uint32_t *h, const uint32_t *d, double dcoef,
                    double decay, double initial, cw_field *out);
int cw_field_destroy(cw_field f);
/* with_source (pde.rs:135-138), and the diffusion coefficient (for fits). */
int cw_field_set_source(cw_field f, double source);
int cw_field_set_diffusion(cw_field f, double dcoef);
/* The floor at zero of every update (pde.rs:395), on by default; off makes
 * relax a plain linear solve (values may go negative), as an adjoint needs. */
int cw_field_set_floor(cw_field f, int32_t on);
enum { CW_VALUES = 0, CW_UPTAKE = 1, CW_PRODUCTION = 2, CW_LIN_SINK = 3 };
/* Per-pixel arrays of history `hist`: values, uptake (zero-order sink,
 * set_uptake_at), production (set_production_at) and the first-order sink
 * k_i of the extension D lap c - k_i c (zero by default: the reference). */
int cw_field_upload(cw_field f, uint32_t hist, int32_t which, const double *host);
int cw_field_download(cw_field f, uint32_t hist, int32_t which, double *host);
int cw_field_upload_held(cw_field f, uint32_t hist, const uint8_t *held);
int cw_field_download_held(cw_field f, uint32_t hist, uint8_t *held);
/* fill, clear_uptake, clear_production, release_all (pde.rs:205-220, 468-470). */
int cw_field_fill(cw_field f, double value);
int cw_field_clear(cw_field f, int32_t which);
int cw_field_release_all(cw_field f);
/* hold_where (pde.rs:491-498): hold every pixel mask names at value. */
int cw_field_hold_mask(cw_field f, uint32_t hist, const uint8_t *mask, double value);
/* hold_bath_at (pde.rs:550-631) with an explicit open mask of history `hist`. */
int cw_field_hold_bath(cw_field f, uint32_t hist, const uint8_t *open, double value);

enum { CW_STOP_MAX_CHANGE = 0, CW_STOP_RESIDUAL = 1 };
enum { CW_FP64 = 0, CW_FP32_DC = 1 };
/* CW_FP32_DC sweep windows: the widest the batch allows (128 x 64, fed by
 * TMA, where every history's rows are 16-byte aligned; else 64 x 64),
 * 64 x 64 always, or 128 x 128 TMA-fed windows, one block per SM, where the
 * rows allow (else 64 x 64). */
enum { CW_WINDOW_AUTO = 0, CW_WINDOW_64 = 1, CW_WINDOW_TALL = 2 };
typedef struct {
    double omega;        /* <= 0: the reference's rule (pde.rs:267-277) */
    int32_t stop;        /* CW_STOP_MAX_CHANGE (the reference) or CW_STOP_RESIDUAL */
    double tolerance;    /* converged when the stop quantity is below it */
    int64_t max_sweeps;  /* pde.rs:279-287: past it, CW_ERR_SIMULATION */
    int32_t precision;   /* CW_FP64 (bit-exact with the reference) or CW_FP32_DC */
    int32_t inner_sweeps;/* CW_FP32_DC: FP32 sweeps per FP64 defect correction (0: 16) */
    int32_t block_depth; /* CW_FP32_DC: half-sweeps per launch kept in shared memory (0: 4) */
    int32_t window;      /* CW_FP32_DC: a CW_WINDOW_* */
    double error_tolerance; /* CW_FP32_DC on flat fields (the TMA-fed sweeps): > 0 also asks that the
                               error left, estimated from the last two corrections (the largest
                               change c_k and their ratio q: c_k q / (1 - q), doubled), be below this,
                               so that a solve stops once its field is that close to the converged
                               one whatever the residual says; the residual rule still holds.
                               0: the residual alone.  No counterpart in the reference */
} cw_relax_opts;
typedef struct {
    int64_t sweeps;      /* the count relax returns (pde.rs:279-283) */
    double last_change;  /* max |change| of the last sweep (FP64 mode) */
    double residual;     /* max projected |b - A c| at the end */
    int32_t status;      /* CW_OK or CW_ERR_SIMULATION */
    double omega;        /* the factor used */
} cw_relax_stats;
/* relax (pde.rs:245-288) on every history; stats has nh entries (may be
 * NULL).  Returns CW_ERR_SIMULATION when any history failed to settle. */
int cw_field_relax(cw_field f, const cw_relax_opts *opts, cw_relax_stats *stats);
/* The adjoint of the steady solve (no counterpart in the reference, which has
 * no derivatives): lambda solves A^T lambda = dl_dc for the field's operator
 * as it stands (diffusion, decay, first-order sink, held pixels), with
 * lambda = 0 on held pixels; then dL/dtheta = -lambda . (dA/dtheta c -
 * db/dtheta) for any coefficient theta.  dl_dc and lambda hold every
 * history's pixels in the batch's flat order.  Exact where the forward
 * solve's floor at zero does not bind.  Options and errors as cw_field_relax
 * (lambda is written also when CW_ERR_SIMULATION reports it unsettled). */
int cw_field_relax_adjoint(cw_field f, const double *dl_dc, double *lambda, const cw_relax_opts *opts,
                           cw_relax_stats *stats);
/* No counterpart in the reference: the FP32 defect-correction relax of one
 * flat field (width x height <= 1,048,576 pixels) that allocates no device
 * memory, for callers whose device memory belongs to another allocator (a
 * framework's caching pool, an arena sized at start-up) or whose loop cannot
 * afford the device-wide stall of cudaMalloc/cudaFree.  The caller passes
 * device pointers it owns: values (w*h doubles, relaxed in place), the held
 * mask (w*h bytes), and the first-order sink, uptake and production (w*h
 * doubles each, or NULL for zero).  The solve's scratch is a fixed array of
 * about 16 MiB inside the library, which every GPU that loads it keeps until
 * exit; its device address is looked up on the first call made on each
 * device.  All calls share that array, so calls whose work overlaps on the
 * GPU (two streams, two threads) race: serialise them.  The work runs on the
 * library stream (cw_set_stream chooses it), which must belong to the current
 * device (else CW_ERR_CONFIG), and the caller's buffers must be ready for
 * that stream: synchronise whatever stream wrote them first.  Larger fields
 * return CW_ERR_CONFIG; a field that does not settle within max_sweeps
 * returns CW_ERR_SIMULATION.  omega <= 0 takes the reference's rule; an
 * omega of 2 or more, or a tolerance that is not finite and above zero,
 * returns CW_ERR_CONFIG. */
int cw_field_relax_noalloc(double *values, const uint8_t *held, const double *lin_sink, const double *uptake,
                           const double *production, uint32_t width, uint32_t height, double dcoef, double decay,
                           double source, double omega, double tolerance, int64_t max_sweeps, int32_t inner_sweeps,
                           int64_t *sweeps_out, double *residual_out);
/* The projected residual max |b - A c| of every history (nh entries). */
int cw_field_residual(cw_field f, double *out);
/* inflow (pde.rs:415-456) of every history (nh entries). */
int cw_field_inflow(cw_field f, double *out);
/* Measurement: time `sweeps` FP32 sweeps of the defect-correction kernel
 * (`depth` half-sweeps per launch, `window` a CW_WINDOW_*) on the current
 * residual of every history, without changing the field.  *ms is the kernels'
 * time, *launches their count. */
int cw_field_time_inner(cw_field f, int32_t sweeps, int32_t depth, int32_t window, double omega, float *ms,
                        int64_t *launches);
/* The FP32 correction the last cw_field_time_inner left, history `hist`
 * (w*h*d floats).  A check of the sweep kernels: every depth gives the same
 * correction as one half-sweep per launch.  No counterpart in the reference. */
int cw_field_inner_correction(cw_field f, uint32_t hist, float *out);
/* DiffusionField::step (pde.rs:705-728): one explicit step; CW_ERR_CONFIG for
 * a step the scheme cannot take (pde.rs:673-701). */
int cw_field_step(cw_field f, double dt);

/* ------------------------------------------------------------------ coupling
 * The lattice and the field must hold the same histories and sizes. */
/* apply_uptake (coupling.rs:26-39) with a rate per cell type (K entries;
 * 0 for a type that does not consume).  first_order = 0 writes the
 * zero-order uptake, as the reference; 1 writes the first-order sink k_i. */
int cw_couple_uptake(cw_field f, cw_lattice lat, int32_t K, const double *rate_by_type, int32_t first_order);
/* apply_background_uptake (coupling.rs:47-53). */
int cw_couple_background_uptake(cw_field f, cw_lattice lat, double rate);
/* apply_production (coupling.rs:61-73): per-cell rates of history `hist`. */
int cw_couple_production(cw_field f, cw_lattice lat, uint32_t hist, uint32_t n, const double *per_cell);
/* hold_obstacles_at (coupling.rs:80-82) and hold_medium_bath (coupling.rs:156-158). */
int cw_couple_hold_obstacles(cw_field f, cw_lattice lat, double value);
int cw_couple_hold_medium_bath(cw_field f, cw_lattice lat, double value);
/* hold_vessels_by (coupling.rs:114-150) on planes: every obstacle pixel whose
 * delivery share (host array, one double per pixel of the batch, flat in the
 * batch's order) is above zero is held at value x min(share, 1), unless the
 * field's mean over its in-box neighbours that are not obstacles is already
 * at least that; it is left as it is otherwise.  CW_ERR_CONFIG for a volume. */
int cw_couple_hold_vessels_by(cw_field f, cw_lattice lat, double value, const double *delivery);
/* mean_per_cell (coupling.rs:164-182) for ids [0, n) of history `hist`. */
int cw_couple_mean_per_cell(cw_field f, cw_lattice lat, uint32_t hist, uint32_t n, double *out);

/* ------------------------------------------------------------------ network */
enum {
    CW_ACTIVATED_BY = 0, CW_INHIBITED_BY = 1, CW_ACTIVATED_BY_ABSENCE_OF = 2, CW_PRODUCED_BY = 3,
    CW_DECAYS = 4, CW_RELAXES_TO = 5, CW_DAMAGED_BELOW = 6, CW_DAMAGED_ABOVE = 7
};
/* One term of a NetworkSpec (crates/core/src/network.rs:51-135). */
typedef struct {
    int32_t node;        /* index of the node it belongs to; terms listed in node order, file order */
    int32_t kind;        /* CW_ACTIVATED_BY ... */
    const char *source;  /* node or input name; NULL for decays / relaxes_to */
    double rate;
    double hill_n;       /* <= 0 and hill_k <= 0: no Hill response */
    double hill_k;
    double param;        /* relaxes_to value, or damaged_* threshold */
    int32_t has_hill;
} cw_term_spec;
/* Network::from_spec (network.rs:283-445): resolves names once and refuses
 * what the reference refuses (CW_ERR_CONFIG, message naming the culprit).
 * Optional roles may be NULL; max_target NaN means none. */
int cw_network_compile(int32_t nnodes, const char *const *names, const double *initial, int32_t nterms,
                       const cw_term_spec *terms, const char *growth, const char *survival, const char *hypoxia,
                       const char *differentiation, const char *apoptosis, const char *angiogenic,
                       const char *evasion, double growth_coefficient, double lambda_volume, double max_target,
                       uint32_t reference_volume, cw_network *out);
int cw_network_destroy(cw_network net);
/* Node count and the role indices (growth, survival, hypoxia,
 * differentiation, apoptosis, angiogenic, evasion; -1 when absent). */
int cw_network_info(cw_network net, int32_t *nnodes, int32_t *roles7, double *initial);
/* SignalingNetwork::step (network.rs:802-805) = rk4 (network.rs:777-799),
 * `substeps` times on each of `ncells` cells.  state is [ncells][S] and is
 * updated in place; inputs is [ncells][6]: oxygen, egf, crowding, stress,
 * waste, necrotic factor (CellInputs, crates/core/src/types.rs:414-433). */
int cw_network_step_batch(cw_network net, int64_t ncells, double *state, const double *inputs, double dt,
                          int32_t substeps);
/* mechanics (network.rs:811-821) of each cell: target volume and lambda. */
int cw_network_mechanics_batch(cw_network net, int64_t ncells, const double *state, uint32_t *target,
                               double *lambda);
/* The adjoint of cw_network_step_batch (no counterpart in the reference,
 * which has no derivatives): for `substeps` RK4 steps from `state` ([ncells][S],
 * the state before them) under `inputs` ([ncells][6]), `adjoint` ([ncells][S])
 * holds dL/d(state after) on entry and dL/d(state before) on return; d_oxygen
 * (ncells, or NULL) receives dL/d(oxygen input); d_rates the first `nrates`
 * terms' dL/d(rate) summed over the cells (terms in compile order: node by
 * node, each node's in file order; nrates <= 32).  The forward steps are
 * recomputed; the clamp to [0, 1] passes no gradient where it binds. */
int cw_network_backward_batch(cw_network net, int64_t ncells, const double *state, const double *inputs, double dt,
                              int32_t substeps, double *adjoint, double *d_oxygen, int32_t nrates, double *d_rates);

/* ------------------------------------------------------------------ mutated networks
 * A heritable change to a network (Mutation, network.rs:171-199). */
enum { CW_CHANGE_SCALED = 0, CW_CHANGE_GAINED = 1, CW_CHANGE_LOST = 2 };
typedef struct {
    int32_t node;    /* the node whose terms changed */
    int32_t term;    /* which of its terms, from zero in file order; a gained link is the last */
    int32_t kind;    /* CW_ACTIVATED_BY ... */
    int32_t change;  /* CW_CHANGE_* */
    double value;    /* the factor of a scaled rate, or the rate of a gained link */
    int32_t source;  /* a gained link's source: a node index, or -1 - input (oxygen, egf, crowding, stress) */
    int32_t suppressed; /* a simulation's mutation drawn and recorded but not made (suppress_before) */
} cw_mutation;
/* Network::mutate (network.rs:479-501): one rate, picked by `which` among
 * every node's terms in file order, scaled by 2^(2 how - 1); `which` and `how`
 * are uniform draws in [0, 1) taken by the caller.  *out is a new network;
 * `net` is unchanged.  CW_ERR_NOT_FOUND (and *out NULL) for a network
 * without a single term. */
int cw_network_mutate(cw_network net, double which, double how, cw_network *out, cw_mutation *rec);
/* Network::rewire (network.rs:503-575), draws = (mode, which, source, sign,
 * how): below one half a node gains an activated_by (sign < 1/2) or
 * activated_by_absence_of link from one of the first four inputs or any
 * node, at 0.1 x 2^(2 how - 1); otherwise one term is lost.  *out is a new
 * network; CW_ERR_NOT_FOUND for a loss from a network without a term. */
int cw_network_rewire(cw_network net, const double draws[5], cw_network *out, cw_mutation *rec);
/* RK4 for cells of many networks at once (the per-cell mutated networks of
 * an evolving run, network.rs:487-616): cell c steps under nets[clone[c]].
 * Every network has the same node count; state [ncells][S], inputs
 * [ncells][6], as cw_network_step_batch. */
int cw_network_step_clones(int32_t nnets, const cw_network *nets, int64_t ncells, const int32_t *clone,
                           double *state, const double *inputs, double dt, int32_t substeps);

/* ------------------------------------------------------------------ simulation driver
 * A device-resident Simulation<Running>::step (simulation.rs:1129-1350)
 * reduced to the hot path: per lattice step, every field is painted from the
 * lattice and relaxed, cells read their field means, every living network
 * takes `substeps` RK4 steps, survival and mechanics set kind and target
 * volume (a necrotic cell's shrinking by 2 pixels a step until it is gone),
 * the lattice takes `sweeps` Monte Carlo steps, and cells grown past 1.4
 * times the network's reference volume, not too hypoxic to cycle, divide
 * (simulation.rs:1338-1347, 1603-1716). */
typedef struct {
    uint32_t nh;                 /* histories (a batch of uneven sizes) */
    const uint32_t *w, *h, *d;   /* per history */
    const uint32_t *ncells;      /* initial cells per history */
    const uint64_t *seeds;       /* per history */
    double temperature;
    int32_t K;                   /* cell types; type 0 is the medium */
    const double *J;             /* K x K */
    int32_t contact_order;
    int32_t target_volume;       /* of every seeded cell */
    double lambda_volume;
    int32_t surface_target;      /* <= 0: no surface constraint */
    double lambda_surface;
    int32_t seeding;             /* 0 squares at random free places, 1 a packed ball of cubes, 3 one cell (below),
                                    4 a sheet: the plane tiled by seed_side-square cells of type 2 (simulation.rs:
                                    696-731; needs field_off) */
    int32_t seed_side;           /* side of a seeded square / cube */
    int32_t nfields;             /* 1 (oxygen) or 2 (oxygen and a secreted signal) */
    double o2_dcoef;
    const double *o2_sink_by_type; /* K first-order sinks k per type (0 for the medium) */
    double o2_background_sink;   /* first-order sink of medium pixels (stroma around a vessel) */
    int32_t o2_hold;             /* 0 row y=0, 1 column x=w/2, 2 every face of the box, 4 a vessel (below), 3 the bath: the
                                    medium joined to the box's outer layer, taken every step
                                    (declare_sources with OxygenSource::Bath, simulation.rs:2138-2146) */
    double signal_dcoef, signal_decay, signal_secretion, hypoxic_level;
    double tolerance;            /* residual tolerance of every field solve */
    int32_t precision;           /* CW_FP64 or CW_FP32_DC */
    double omega;                /* <= 0: chosen by the autotuner (CW_FP32_DC) or the reference's rule */
    int32_t inner_sweeps;        /* CW_FP32_DC: FP32 sweeps per defect correction (0: 64) */
    int32_t relax_every;         /* solve the fields every this many steps (1: each) */
    double dt;                   /* network time step */
    int32_t substeps;            /* RK4 steps per lattice step */
    int32_t sweeps;              /* Monte Carlo steps per lattice step */
    double death_threshold;      /* survival below it: the necrotic type */
    int32_t necrotic_type;       /* type a dead cell takes (-1: none) */
    int32_t use_graphs;          /* once tuned, replay each step as captured CUDA graphs */
    int32_t divide;              /* 1: the division step; 0: none */
    int32_t max_cells;           /* living cells a history divides up to (<= 0: 2000, the reference's default) */
    int32_t spare_cells;         /* records per history for daughters (<= 0: max_cells) */
    /* The released fields (settle_waste / settle_necrotic_factor and
     * settle_released, simulation.rs:2057-2113, 2546-2570), each diffusing as
     * oxygen does, held at zero on the bath, solved like the other fields, its
     * mean over a cell the cell's `waste` / `necrotic_factor` input.  They run
     * on the step's un-captured path (no CUDA graphs). */
    double waste_production;     /* > 0: what a living cell's pixel releases a step (Waste, types.rs:240-244) */
    double necrotic_production;  /* > 0: what a necrotic cell's pixel releases (NecroticFactor, types.rs:256-266) */
    int32_t necrotic_release_for;/* steps after the one it died at a necrotic cell releases; < 0: while it is there */
    int32_t subsweeps;           /* <= 1: one sweep of every colour a Monte Carlo step; n: cw_lattice_set_subsweeps */
    /* The reference's scenarios (Simulation::new, simulation.rs:510-1066):
     * seeding 3 is one cell (a disc in the plane, a ball in a volume, of
     * radius seed_side) at the centre, or against the vessel's wall with
     * o2_hold 4, its target its own volume; o2_hold 4 is a vessel, an
     * obstacle disc of vessel_radius at the centre through every slice, held
     * at the source's level (add_obstacle_disc, cpm.rs:389-415). */
    double o2_uptake;            /* > 0: zero-order uptake of every living cell's pixel (apply_uptake,
                                    coupling.rs:22-40), and of the medium around a vessel (apply_background_uptake) */
    int32_t divide_every;        /* the division check every this many steps (<= 1: every step; the reference
                                    checks a single seeded tissue every 20, simulation.rs:1338-1345) */
    int32_t vessel_radius;       /* o2_hold 4 */
    int32_t stop_rule;           /* CW_STOP_RESIDUAL, or CW_STOP_MAX_CHANGE with CW_FP64: the reference's
                                    relax, pixel for pixel (no pixel moves by more than `tolerance` a sweep) */
    double first_tolerance;      /* > 0: the first step's oxygen solved to this, up to 2,000,000 sweeps, from the
                                    field's initial level (start(), simulation.rs:1068-1083) */
    double cycle_median;         /* > 0: a cell cycle (Cycle, simulation.rs:1701-1745, 2529-2540): each division
                                    draws the two cells' lengths, median x exp(spread z), a cell divides once its
                                    cycle is over and asks meanwhile for half to all of its target */
    double cycle_spread;
    double debris_loss;          /* (0, 1]: the share of a dead cell's volume its debris loses a step, taken at the
                                    tissue's edge, and the fluid the tissue shuts in drained (break_down_debris,
                                    drain_shut_in, simulation.rs:1746-1826); 0: dead cells resorb RESORPTION_RATE
                                    pixels a step.  Needs necrotic_type */
    double still_medium;         /* > 0: the bath is still medium of this diffusion, and the level it holds falls
                                    with what the tissue takes up (settle_bath_level, simulation.rs:2104-2125);
                                    o2_hold 3 in volumes only */
    double exposure_intensity;   /* > 0: an exposure (Exposure, types.rs:92-104, 319-332; settle_stress,
                                    simulation.rs:2006-2056): a stress field, diffusing as oxygen does, held at
                                    this level where the oxygen is held from step exposure_start on (with
                                    exposure_on > 0, for exposure_on steps of every exposure_on + exposure_off),
                                    zero while off, taken up at exposure_uptake by every living pixel (and the
                                    medium around a vessel); a cell's mean is its network's stress input */
    double exposure_uptake;
    int32_t exposure_start, exposure_on, exposure_off;
    double mutation_rate;        /* (0, 1]: at each division the daughter's network changes with this chance and
                                    the daughter founds a clone (simulation.rs:1655-1700): one rate scaled by up
                                    to MUTATION_SPREAD either way (Network::mutate, network.rs:479-501), or, with
                                    `rewiring`, that share of the changes a link gained or lost
                                    (Network::rewire, network.rs:503-575); every clone's cells step under its
                                    own network.  The draws: Philox under the history's key, counters (parent
                                    id, step, 6 / 7 / 8, 0).  0: every cell under the one network */
    double rewiring;             /* [0, 1]: the share of the changes that rewire */
    int32_t field_off;           /* nothing consumes: the oxygen is not solved and stays at its start, 1 (the
                                    field left off, simulation.rs:786-793, 2127-2131) */
    int32_t differentiated_type; /* >= 0: the type a cell takes when it commits to differentiate (its network's
                                    differentiation node's level its chance a step), then shedding SHEDDING_RATE
                                    pixels a step until gone; -1: no such fate (simulation.rs:1209-1296) */
    int32_t apoptotic_type;      /* >= 0: the same for apoptosis (the apoptosis node; FRAGMENTATION_RATE) */
    int32_t lineage;             /* every seeded cell founds a clone of its own (a lineage-tracing sheet,
                                    simulation.rs:780-785): cw_sim_clones and the measurements count them */
    double error_tolerance;      /* the FP32 solves' error_tolerance (cw_relax_opts); 0: the residual alone */
    int32_t suppress_before;     /* > 0: every mutation founded before this step is drawn and recorded (its
                                    clone founded, cw_mutation.suppressed set) but not made: the daughter keeps
                                    its parent's network (Scenario::suppress_before, simulation.rs:240-244,
                                    1671-1694); <= 0: none */
    int32_t tracing;             /* 1: lineage tracing (Tracing, types.rs:208-214; mark_every_cell,
                                    simulation.rs:1908-1918): at the start of step tracing_at every cell in the
                                    layer (holding pixels, neither necrotic nor apoptotic) is marked with its
                                    record's id less one, and daughters carry their parent's mark
                                    (cw_sim_traced); 0: none */
    int32_t tracing_at;
} cw_sim_config;
int cw_sim_create(const cw_sim_config *cfg, cw_network net, cw_sim *out);
/* A lesion (Lesion, simulation.rs:348-360; place_lesion 1920-1970): at the
 * start of step `at`, before anything else in it, every living cell of each
 * history whose centre of mass lies within `radius` pixels of (cx, cy) (both
 * NaN: the centre of the box) joins one new clone carrying `net`, its state
 * the network's initial one; the clone is recorded with parent -1 and a
 * mutation whose change is -1, and measurements count the lesion's living
 * descendants.  Planes only.  `net` stays the caller's and must outlive the
 * simulation; it has the simulation network's nodes, roles, mechanics and
 * reference volume (every cell steps under its clone's network, with the
 * tissue's roles).  CW_ERR_CONFIG for a centre outside the box, a radius not
 * finite and above zero, a volume, another network frame, or a step past. */
int cw_sim_set_lesion(cw_sim sim, cw_network net, uint32_t at, double radius, double cx, double cy);
int cw_sim_destroy(cw_sim sim);
/* `steps` lattice steps on every history. */
int cw_sim_step(cw_sim sim, uint32_t steps);
/* The clones of a simulation with mutation or a lineage (CloneRecord,
 * simulation.rs:780-785, 1686-1694): the clone of records 0..n-1 of history
 * `hist` (0: the founding clone; with a lineage a seeded cell's clone is its
 * record's index in the batch); the clones in the whole batch; and the clones
 * clones founded during the run, in the order they were founded, which are
 * the last *count clone indices: each one's parent clone and its mutation
 * (cw_mutation as cw_network_mutate gives it; a lesion's clone has parent -1
 * and change -1; parent and mutation may be NULL). */
int cw_sim_clones(cw_sim sim, uint32_t hist, uint32_t n, int32_t *clone);
int cw_sim_clone_count(cw_sim sim, uint32_t *nclones);
int cw_sim_clone_records(cw_sim sim, uint32_t *count, int32_t *parent, cw_mutation *mutation);
/* traced_clones (simulation.rs:2407-2421) of history `hist`: for every mark
 * a cell in the layer still carries, in increasing order, the mark and the
 * cells in the layer carrying it (cycling, quiescent or differentiating,
 * holding pixels).  *n receives the number of marks; at most `cap` pairs are
 * written.  Empty before the marking step; CW_ERR_CONFIG without tracing. */
int cw_sim_traced(cw_sim sim, uint32_t hist, uint32_t cap, uint32_t *marks, uint64_t *cells, uint32_t *n);
/* What the autotuner chose: the SOR relaxation factor of every history for
 * the oxygen and the signal field (0 until chosen: the reference's rule),
 * the FP32 blocking depth and window (CW_WINDOW_*), and whether it is still
 * trying candidates.  It runs when cfg.omega <= 0 with CW_FP32_DC, over the
 * first few steps. */
int cw_sim_tuning(cw_sim sim, double *omega_o2, double *omega_signal, int32_t *depth, int32_t *window,
                  int32_t *tuning);
/* Steps replayed from CUDA graphs, solves whose graph budget of outer
 * iterations fell short (finished host-side), and the budgets (2 entries). */
int cw_sim_graph_info(cw_sim sim, uint64_t *graph_steps, uint64_t *budget_misses, int32_t *budgets);
/* Handles the driver owns, for inspection with the calls above; fields 0 oxygen, 1 signal, 2 waste,
   3 necrotic factor, 4 stress (CW_ERR_NOT_FOUND for one the simulation does not have). */
int cw_sim_lattice(cw_sim sim, cw_lattice *lat);
int cw_sim_field(cw_sim sim, int32_t which, cw_field *f);
/* Per history: living cells, mean oxygen over cells, sweeps of the last
 * oxygen solve, its residual (4 doubles per history). */
int cw_sim_stats(cw_sim sim, double *out);
/* Measurements (crates/engine/src/measure.rs:21-90, Simulation::measure
 * 133-236) of every history as it stands after the last step: the counts of
 * cycling (hypoxia response under 0.45), quiescent and necrotic cells with
 * pixels, cells ever born and gone (resorbed to nothing), the obstacle
 * pixels, and the equivalent radii of the tissue and of the necrotic area
 * (a disc in the plane, a ball in a volume).  viable_depth is the
 * reference's for the source the oxygen hold stands for: the tissue radius
 * less the necrotic one around the faces or the bath (o2_hold 2, 3), the
 * radius of vessel and living together less the vessel's around a vessel
 * (4; in a volume the radii are of cylinders as long as the box), the living
 * area over the columns living cells hold along a held row (0, the
 * reference's capillary), and over twice the rows they hold beside the held
 * column (1, tissue on either side). */
typedef struct {
    uint64_t mcs;        /* index of the step last taken (0 before the first) */
    uint64_t cycling, quiescent, necrotic;
    uint64_t born, gone;
    uint64_t vessel;
    double tissue_radius, necrotic_radius, viable_depth;
    double exposure;     /* the exposure's level at the step last taken (0 without one or while off) */
    uint64_t differentiating, apoptotic;  /* cells leaving the layer, cells breaking up */
    uint64_t clones;     /* clones with a living cell (with lineage or mutation; else 1 while any cell lives) */
    uint64_t lesion;     /* living cells descended from a lesion (lesion_cells, evolution.rs:182-197) */
} cw_measurements;
int cw_sim_measure(cw_sim sim, cw_measurements *out);
/* touches_the_edge (simulation.rs:2165-2198) of every history, one int32 each: a cell on a pixel of
 * the box's sides, or, in a volume around no vessel, of its faces; one pass over the sites. */
int cw_sim_touches_edge(cw_sim sim, int32_t *out);
/* Network state of history `hist`, [ncells][S]. */
int cw_sim_network_state(cw_sim sim, uint32_t hist, uint32_t n, double *state);
/* The cycle of records 0..n-1 of history `hist`: the step each began and the step it is over (the
   reference's began / due, simulation.rs:486-491); CW_ERR_CONFIG without a cycle. */
int cw_sim_cycle(cw_sim sim, uint32_t hist, uint32_t n, int32_t *began, int32_t *due);

/* ------------------------------------------------------------------ differentiation
 * No counterpart in the reference (it has no adjoint, loss or autodiff): a
 * hand-written adjoint of one frozen lattice's step, for fitting.  Oxygen
 * solves D lap c - k_type c = 0 with the lattice's obstacles held at
 * vessel_value; each cell's network runs `steps` RK4 steps of dt on its mean
 * oxygen, checkpointed every `checkpoint_every`; the cells secrete
 * secretion * (angiogenic node) into a signal field (signal_dcoef,
 * signal_decay).  The loss is sum_b (h_b - h*_b)^2 + signal_weight *
 * sum_b (g_b - g*_b)^2 over `nbins` bins of |x - vessel_x| / bin_width, h_b
 * the bin's hypoxic fraction of cell pixels, smoothed as
 * sigmoid((hypoxic_level - c) / tau), g_b their mean signal.  Parameters:
 * D, k for types 1..3, and the rates of the network's first
 * `network_params` terms (file order). */
typedef struct {
    double dcoef;               /* D (the first parameter's initial value) */
    double uptake[3];           /* k of types 1, 2, 3 */
    double vessel_value;        /* oxygen held on the lattice's obstacles */
    int32_t vessel_x;           /* bins measure the distance from this column */
    double egf;
    double signal_dcoef, signal_decay, secretion;
    int32_t steps, checkpoint_every;
    double dt;
    int32_t nbins;
    double bin_width, hypoxic_level, tau, signal_weight;
    double tolerance;           /* forward solves: residual */
    double adjoint_tolerance;   /* adjoint solves: residual */
    int32_t precision;          /* CW_FP64 or CW_FP32_DC for every solve */
    double omega;               /* <= 0: the reference's rule */
    int32_t network_params;     /* rates fitted, at most 32 */
} cw_fit_config;
/* The lattice (one history) and the network are borrowed, not copied: keep
 * them alive, and the lattice unchanged, while the fit lives. */
int cw_fit_create(cw_lattice lat, cw_network net, const cw_fit_config *cfg, cw_fit *out);
int cw_fit_destroy(cw_fit fit);
int cw_fit_nparams(cw_fit fit, int32_t *n);
int cw_fit_get_params(cw_fit fit, double *params);
int cw_fit_set_params(cw_fit fit, const double *params);
/* Target profiles h* and g*, nbins each. */
int cw_fit_set_target(cw_fit fit, const double *hypoxic, const double *signal);
/* Forward: the loss and the profiles h, g (nbins each; either may be NULL). */
int cw_fit_forward(cw_fit fit, double *loss, double *hypoxic, double *signal);
/* Forward and adjoint: the loss and dL/dparams (cw_fit_nparams entries). */
int cw_fit_gradient(cw_fit fit, double *loss, double *grad);

#ifdef __cplusplus
}
#endif
#endif
