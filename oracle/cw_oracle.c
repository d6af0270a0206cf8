/*
 * cw_oracle.c -- CPU restatement of cellweave's per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
 * CUDA library in cellweave_b200/: only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it, always as the checker or as the
 * timed CPU reference, never as a product code path.
 *
 * It restates, function by function and in the same floating-point order,
 * the Rust sources of the reference (ngodzik/cellweave v0.3.0):
 *   crates/engine/src/pde.rs      ScalarField relax / half_sweep / free_span /
 *                                 inflow / hold_bath_at / explicit step
 *   crates/engine/src/cpm.rs      ContactEnergy, set_contact_order (Reach),
 *                                 contact_delta_h, volume_delta_h, try_flip,
 *                                 monte_carlo_step, occupied_span
 *   crates/engine/src/network.rs  driver (Hill), read, derivatives,
 *                                 term_rate, rk4, mechanics
 *   crates/engine/src/coupling.rs apply_uptake, apply_background_uptake,
 *                                 apply_production, hold_obstacles_at,
 *                                 hold_vessels_by, hold_medium_bath,
 *                                 mean_per_cell
 * Build with -ffp-contract=off so that no multiply-add is fused, as in Rust.
 *
 * Parity status.  RK4 is pinned by the reference's golden table
 * (network.rs:866-891, 1e-12); the SOR by the closed forms and invariants of
 * pde.rs:783-1248; Delta-H by the closed forms of cpm.rs:1232-1258 and the
 * "Delta-H equals the change of total boundary energy" test (cpm.rs:1912-1943).
 * The Metropolis trajectory itself is unpinned: it depends on the rand 0.10.3
 * StdRng stream (a third-party crate that is not vendored), so the sequential
 * sweep here draws from splitmix64 and is compared statistically only.
 *
 * Extensions that the reference does not have (each off by default, each
 * reducing to the reference when off): a first-order sink k_i in the SOR
 * denominator, a residual stopping rule, a K x K contact table indexed by
 * cell type, a surface constraint, and the sublattice (checkerboard)
 * Metropolis scheme that the GPU runs, with Philox4x32-10 draws, restated
 * here so the GPU lattice can be compared bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_CONFIG 1
#define OR_ERR_SIMULATION 2

/* ======================================================================
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11) and the derived draws the sublattice sweep uses.
 * ====================================================================== */
typedef struct { uint32_t v[4]; } or_u32x4;

static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

or_u32x4 or_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    or_u32x4 out = {{c0, c1, c2, c3}};
    return out;
}

void or_philox_batch(uint32_t n, const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
    for (uint32_t i = 0; i < n; ++i) {
        or_u32x4 r = or_philox(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], key[0], key[1]);
        memcpy(out + 4 * i, r.v, sizeof r.v);
    }
}

/* Uniform double in [0, 1) from 53 random bits taken from two words. */
static inline double or_u01(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* exp(x) for x <= 0, the same operations as the device's: Cody-Waite
 * reduction by ln 2 split into a 20-bit head and a tail, a degree-17 Taylor
 * polynomial of e^r on |r| <= ln2/2 in Horner form, and a power-of-two
 * scaling.  Only + - * and ldexp, so host and device agree to the bit. */
double or_cw_exp(double x) {
    if (!(x > -745.0)) return 0.0; /* also catches NaN */
    if (x > 709.0) return INFINITY;
    const double log2e = 1.4426950408889634;
    const double ln2_hi = 0.6931467056274414;     /* 0x1.62e42p-1: 20 significant bits */
    const double ln2_lo = 4.7493250390316726e-07; /* ln 2 - ln2_hi */
    double kf = floor(x * log2e + 0.5);
    double r = (x - kf * ln2_hi) - kf * ln2_lo;
    double p = 1.0 / 355687428096000.0; /* 1/17! */
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

/* ======================================================================
 * Diffusion field: pde.rs
 * ====================================================================== */
typedef struct {
    int32_t w, h, d;
    double *values;     /* n */
    uint8_t *held;      /* n */
    double *uptake;     /* n, zero-order sink (pde.rs:48) */
    double *production; /* n, zero-order source (pde.rs:50) */
    double *lin_sink;   /* n or NULL: first-order sink k_i (extension) */
    double dcoef, decay, source;
} or_field;

typedef struct { int32_t x0, x1, y0, y1, z0, z1; } or_span;

/* free_span, pde.rs:305-320: the box around every pixel not held.  The z
 * range keeps the reference's form: the first free z, then the last one. */
int or_free_span(const or_field *f, or_span *s) {
    int64_t n = (int64_t)f->w * f->h * f->d;
    int found = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (f->held[i]) continue;
        int32_t x = (int32_t)(i % f->w), y = (int32_t)((i / f->w) % f->h), z = (int32_t)(i / ((int64_t)f->w * f->h));
        if (!found) {
            s->x0 = s->x1 = x; s->y0 = s->y1 = y; s->z0 = s->z1 = z;
            found = 1;
        }
        if (x < s->x0) s->x0 = x;
        if (x > s->x1) s->x1 = x;
        if (y < s->y0) s->y0 = y;
        if (y > s->y1) s->y1 = y;
        s->z1 = z;
    }
    return found;
}

/* The relaxation factor of relax, pde.rs:267-277. */
double or_auto_omega(const or_field *f, const or_span *s) {
    if (f->d > 1) {
        int32_t l = s->x1 - s->x0 + 1;
        if (s->y1 - s->y0 + 1 > l) l = s->y1 - s->y0 + 1;
        if (s->z1 - s->z0 + 1 > l) l = s->z1 - s->z0 + 1;
        if (l < 2) l = 2;
        return 2.0 / (1.0 + sin(3.14159265358979323846 / (double)l));
    }
    double n = (double)(f->w > f->h ? f->w : f->h);
    double om = 2.0 / (1.0 + sin(3.14159265358979323846 / n));
    return om < 1.95 ? om : 1.95;
}

/* One pixel's balance, pde.rs:361-395 (sum order x-1, x+1, y-1, y+1, z-1, z+1). */
static inline void or_pixel_sums(const or_field *f, const double *v, int64_t i, int32_t x, int32_t y, int32_t z,
                                 double *sum_out, double *real_out) {
    int64_t w = f->w, slice = (int64_t)f->w * f->h;
    double sum = 0.0, real = 0.0;
    if (x > 0) { sum += v[i - 1]; real += 1.0; }
    if (x + 1 < f->w) { sum += v[i + 1]; real += 1.0; }
    if (y > 0) { sum += v[i - w]; real += 1.0; }
    if (y + 1 < f->h) { sum += v[i + w]; real += 1.0; }
    if (z > 0) { sum += v[i - slice]; real += 1.0; }
    if (z + 1 < f->d) { sum += v[i + slice]; real += 1.0; }
    *sum_out = sum;
    *real_out = real;
}

static inline double or_denominator(const or_field *f, double real, int64_t i) {
    double den = real * f->dcoef + f->decay;
    if (f->lin_sink) den = den + f->lin_sink[i];
    return den;
}

/* half_sweep, pde.rs:329-405: reads `cur`, writes `nxt`; returns max |change|. */
static double or_half_sweep(const or_field *f, const double *cur, double *nxt, double omega, int colour,
                            const or_span *s) {
    int64_t w = f->w, h = f->h;
    int64_t first = (int64_t)s->z0 * h + s->y0, last = (int64_t)s->z1 * h + s->y1;
    double moved_all = 0.0;
#pragma omp parallel for schedule(static) reduction(max : moved_all)
    for (int64_t stacked = first; stacked <= last; ++stacked) {
        int32_t y = (int32_t)(stacked % h), z = (int32_t)(stacked / h);
        if (y < s->y0 || y > s->y1) continue;
        double moved = 0.0;
        for (int32_t x = s->x0; x <= s->x1; ++x) {
            int64_t i = stacked * w + x;
            double before = cur[i];
            if ((x + y + z) % 2 != colour || f->held[i]) {
                nxt[i] = before;
                continue;
            }
            double sum, real;
            or_pixel_sums(f, cur, i, x, y, z, &sum, &real);
            double balanced = (f->dcoef * sum + f->source + f->production[i] - f->uptake[i]) / or_denominator(f, real, i);
            double after = fmax((1.0 - omega) * before + omega * balanced, 0.0);
            nxt[i] = after;
            double dlt = fabs(after - before);
            moved = fmax(moved, dlt);
        }
        if (moved > moved_all) moved_all = moved;
    }
    return moved_all;
}

/* Largest projected residual |b - A c| over the free pixels: at a pixel held
 * at zero by the floor a residual that points below zero counts as met. */
double or_field_residual(const or_field *f) {
    int64_t w = f->w, h = f->h, d = f->d;
    double worst = 0.0;
#pragma omp parallel for schedule(static) reduction(max : worst)
    for (int64_t stacked = 0; stacked < h * d; ++stacked) {
        int32_t y = (int32_t)(stacked % h), z = (int32_t)(stacked / h);
        for (int32_t x = 0; x < w; ++x) {
            int64_t i = stacked * w + x;
            if (f->held[i]) continue;
            double sum, real;
            or_pixel_sums(f, f->values, i, x, y, z, &sum, &real);
            double c = f->values[i];
            double r = (f->dcoef * sum + f->source + f->production[i] - f->uptake[i]) - or_denominator(f, real, i) * c;
            if (c <= 0.0 && r < 0.0) r = 0.0;
            r = fabs(r);
            if (r > worst) worst = r;
        }
    }
    return worst;
}

/* relax, pde.rs:245-288.  omega <= 0 selects the reference's automatic rule.
 * stop_kind 0: max per-sweep change < tol (the reference); 1: projected
 * residual < tol after the sweep.  Returns the sweep count in *sweeps. */
int or_field_relax(or_field *f, double omega, int stop_kind, double tol, int64_t max_sweeps, int threads,
                   int64_t *sweeps) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    or_span s;
    if (!or_free_span(f, &s)) {
        *sweeps = 1;
        return OR_OK;
    }
    if (!(omega > 0.0)) omega = or_auto_omega(f, &s);
    int64_t n = (int64_t)f->w * f->h * f->d;
    double *next = (double *)malloc(sizeof(double) * (size_t)n);
    if (!next) return OR_ERR_SIMULATION;
    memcpy(next, f->values, sizeof(double) * (size_t)n);
    double *cur = f->values, *nxt = next;
    int rc = OR_ERR_SIMULATION;
    *sweeps = max_sweeps;
    for (int64_t done = 1; done <= max_sweeps; ++done) {
        double red = or_half_sweep(f, cur, nxt, omega, 0, &s);
        double *t = cur; cur = nxt; nxt = t;
        double black = or_half_sweep(f, cur, nxt, omega, 1, &s);
        t = cur; cur = nxt; nxt = t;
        double moved = fmax(red, black);
        int settled;
        if (stop_kind == 1) {
            double *keep = f->values;
            f->values = cur;
            settled = or_field_residual(f) < tol;
            f->values = keep;
        } else {
            settled = moved < tol;
        }
        if (settled) {
            *sweeps = done;
            rc = OR_OK;
            break;
        }
    }
    if (cur != f->values) memcpy(f->values, cur, sizeof(double) * (size_t)n);
    free(next);
    return rc;
}

/* inflow, pde.rs:415-456, summed in the same fixed order. */
double or_field_inflow(const or_field *f) {
    or_span s;
    if (!or_free_span(f, &s)) return 0.0;
    int64_t w = f->w, slice = (int64_t)f->w * f->h;
    double flux = 0.0;
    for (int32_t z = s.z0; z <= s.z1; ++z)
        for (int32_t y = s.y0; y <= s.y1; ++y)
            for (int32_t x = s.x0; x <= s.x1; ++x) {
                int64_t i = z * slice + y * w + x;
                if (f->held[i]) continue;
#define OR_ACROSS(j) do { if (f->held[(j)]) flux += f->dcoef * (f->values[(j)] - f->values[i]); } while (0)
                if (x > 0) OR_ACROSS(i - 1);
                if (x + 1 < f->w) OR_ACROSS(i + 1);
                if (y > 0) OR_ACROSS(i - w);
                if (y + 1 < f->h) OR_ACROSS(i + w);
                if (z > 0) OR_ACROSS(i - slice);
                if (z + 1 < f->d) OR_ACROSS(i + slice);
#undef OR_ACROSS
            }
    return flux;
}

/* DiffusionField::step, pde.rs:646-728: one explicit Euler step with mirror
 * walls.  Returns OR_ERR_CONFIG for a step the scheme cannot take. */
int or_field_step_explicit(or_field *f, double dt) {
    if (isnan(dt) || dt <= 0.0) return OR_ERR_CONFIG;
    double limit = f->d > 1 ? 0.25 * 2.0 / 3.0 : 0.25;
    if (f->dcoef * dt > limit) return OR_ERR_CONFIG;
    if (f->decay * dt > 1.0) return OR_ERR_CONFIG;
    int64_t w = f->w, h = f->h, slice = w * h, n = slice * f->d;
    double *next = (double *)malloc(sizeof(double) * (size_t)n);
    if (!next) return OR_ERR_SIMULATION;
    for (int64_t i = 0; i < n; ++i) {
        double c = f->values[i];
        if (f->held[i]) { next[i] = c; continue; }
        int64_t x = i % w, y = (i / w) % h, z = i / slice;
        double a = x > 0 ? f->values[i - 1] : c;
        double b = x + 1 < w ? f->values[i + 1] : c;
        double e = y > 0 ? f->values[i - w] : c;
        double g = y + 1 < h ? f->values[i + w] : c;
        double lap = a + b + e + g - 4.0 * c;
        if (f->d > 1) {
            double p = z > 0 ? f->values[i - slice] : c;
            double q = z + 1 < f->d ? f->values[i + slice] : c;
            lap += p + q - 2.0 * c;
        }
        double change = f->dcoef * lap - f->decay * c + f->source + f->production[i] - f->uptake[i];
        next[i] = fmax(c + dt * change, 0.0);
    }
    memcpy(f->values, next, sizeof(double) * (size_t)n);
    free(next);
    return OR_OK;
}

/* hold_bath_at, pde.rs:550-631: hold every pixel a bath flooding in from the
 * edge of the box around the closed pixels can reach, at `value`.  `open` is
 * one byte per pixel.  Holds accumulate in `held`. */
int or_hold_bath(or_field *f, const uint8_t *open, double value) {
    int64_t w = f->w, h = f->h, d = f->d, slice = w * h, n = slice * d;
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    int closed = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (open[i]) continue;
        int64_t p[3] = {i % w, (i / w) % h, i / slice};
        if (!closed) {
            for (int a = 0; a < 3; ++a) lo[a] = hi[a] = p[a];
            closed = 1;
        }
        for (int a = 0; a < 3; ++a) {
            if (p[a] < lo[a]) lo[a] = p[a];
            if (p[a] > hi[a]) hi[a] = p[a];
        }
    }
    int64_t lim[3] = {w, h, d};
    if (closed)
        for (int a = 0; a < 3; ++a) {
            lo[a] = lo[a] > 0 ? lo[a] - 1 : 0;
            hi[a] = hi[a] + 1 < lim[a] - 1 ? hi[a] + 1 : lim[a] - 1;
        }
    for (int64_t i = 0; i < n; ++i) {
        int64_t p[3] = {i % w, (i / w) % h, i / slice};
        int inside = closed;
        for (int a = 0; a < 3 && inside; ++a) inside = lo[a] <= p[a] && p[a] <= hi[a];
        if (!inside) f->held[i] = 1;
    }
    int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!stack) return OR_ERR_SIMULATION;
    int64_t top = 0;
#define OR_REACH(j) do { int64_t jj = (j); if (!f->held[jj] && open[jj]) { f->held[jj] = 1; stack[top++] = jj; } } while (0)
    if (closed) {
        for (int64_t z = lo[2]; z <= hi[2]; ++z)
            for (int64_t y = lo[1]; y <= hi[1]; ++y)
                for (int64_t x = lo[0]; x <= hi[0]; ++x) {
                    int outer = x == lo[0] || x == hi[0] || y == lo[1] || y == hi[1] || (d > 1 && (z == lo[2] || z == hi[2]));
                    if (outer) OR_REACH(z * slice + y * w + x);
                }
    }
    while (top > 0) {
        int64_t i = stack[--top];
        int64_t x = i % w, y = (i / w) % h, z = i / slice;
        if (x > 0) OR_REACH(i - 1);
        if (x + 1 < w) OR_REACH(i + 1);
        if (y > 0) OR_REACH(i - w);
        if (y + 1 < h) OR_REACH(i + w);
        if (z > 0) OR_REACH(i - slice);
        if (z + 1 < d) OR_REACH(i + slice);
    }
#undef OR_REACH
    free(stack);
    for (int64_t i = 0; i < n; ++i)
        if (f->held[i]) f->values[i] = value;
    return OR_OK;
}

/* ======================================================================
 * CPM lattice: cpm.rs
 * ====================================================================== */
#define OR_OBSTACLE (-1)
#define OR_MAX_REACH 124

typedef struct {
    int32_t w, h, d;
    int32_t *grid;    /* n; -1 is the obstacle (u32::MAX in the reference) */
    int32_t ncells;   /* records, medium slot 0 included */
    int32_t *type;    /* [ncells], index into the K x K table */
    int32_t *volume;  /* [ncells] */
    int32_t *target;  /* [ncells] */
    double *lambda;   /* [ncells] */
    int32_t *surface; /* [ncells] or NULL: the surface constraint is off */
    int32_t *target_surface;
    double *lambda_surface;
    int32_t K;
    double *J;        /* K*K, row-major, symmetric, J[0] = 0 */
    int32_t order;    /* contact order, cpm.rs:274 */
    double temperature;
    int32_t copy_moore; /* 0: copy from a face neighbour (cpm.rs:922-944); 1: from any of the
                           8 (26) Chebyshev neighbours, an extension */
} or_lattice;

/* set_contact_order, cpm.rs:274-301.  Returns the offsets (x, y, z) and the
 * divisor; *n = 0 for order <= 1 (faces only, no divisor). */
int or_reach(int order, int volume, int32_t *offsets, double *across) {
    if (order <= 1) { *across = 1.0; return 0; }
    int deep = volume ? 2 : 0;
    int32_t cand[OR_MAX_REACH][3];
    int64_t dist[OR_MAX_REACH];
    int nc = 0;
    for (int dz = -deep; dz <= deep; ++dz)
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                cand[nc][0] = dx; cand[nc][1] = dy; cand[nc][2] = dz;
                dist[nc] = (int64_t)dx * dx + (int64_t)dy * dy + (int64_t)dz * dz;
                ++nc;
            }
    /* sorted, deduplicated distances */
    int64_t uniq[OR_MAX_REACH];
    int nu = 0;
    for (int i = 0; i < nc; ++i) {
        int seen = 0;
        for (int j = 0; j < nu; ++j) seen |= uniq[j] == dist[i];
        if (!seen) uniq[nu++] = dist[i];
    }
    for (int i = 1; i < nu; ++i)
        for (int j = i; j > 0 && uniq[j - 1] > uniq[j]; --j) {
            int64_t t = uniq[j]; uniq[j] = uniq[j - 1]; uniq[j - 1] = t;
        }
    int idx = order - 1 < nu - 1 ? order - 1 : nu - 1;
    int64_t limit = uniq[idx];
    int n = 0;
    int64_t acr = 0;
    for (int i = 0; i < nc; ++i)
        if (dist[i] <= limit) {
            offsets[3 * n] = cand[i][0]; offsets[3 * n + 1] = cand[i][1]; offsets[3 * n + 2] = cand[i][2];
            acr += cand[i][0] > 0 ? cand[i][0] : 0;
            ++n;
        }
    *across = (double)acr;
    return n;
}

static inline int32_t or_kind(const or_lattice *l, int32_t id) {
    if (id == OR_OBSTACLE) return 0;
    if (id < 0 || id >= l->ncells) return 0;
    return l->type[id];
}

/* contact_energy, cpm.rs:901-906: zero inside one cell, else J by kinds. */
static inline double or_energy(const or_lattice *l, int32_t a, int32_t b) {
    if (a == b) return 0.0;
    return l->J[or_kind(l, a) * l->K + or_kind(l, b)];
}

/* von_neumann, cpm.rs:922-944: y-1, y+1, x-1, x+1, z-1, z+1, clipped. */
static inline int or_von_neumann(const or_lattice *l, int32_t x, int32_t y, int32_t z, int64_t *out) {
    int64_t w = l->w, slice = (int64_t)l->w * l->h, i = (int64_t)z * slice + (int64_t)y * w + x;
    int n = 0;
    if (y > 0) out[n++] = i - w;
    if (y + 1 < l->h) out[n++] = i + w;
    if (x > 0) out[n++] = i - 1;
    if (x + 1 < l->w) out[n++] = i + 1;
    if (z > 0) out[n++] = i - slice;
    if (z + 1 < l->d) out[n++] = i + slice;
    return n;
}

/* The pixels a copy may come from: the face neighbours of von_neumann, or
 * with copy_moore every in-box pixel at Chebyshev distance 1, in the order
 * dz, dy, dx = -1, 0, 1 (an extension; the reference copies across faces). */
static inline int or_copy_neighbours(const or_lattice *l, int32_t x, int32_t y, int32_t z, int64_t *out) {
    if (!l->copy_moore) return or_von_neumann(l, x, y, z, out);
    int64_t w = l->w, slice = (int64_t)l->w * l->h, i = (int64_t)z * slice + (int64_t)y * w + x;
    int n = 0;
    int deep = l->d > 1 ? 1 : 0;
    for (int dz = -deep; dz <= deep; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                if (x + dx < 0 || x + dx >= l->w || y + dy < 0 || y + dy >= l->h || z + dz < 0 || z + dz >= l->d)
                    continue;
                out[n++] = i + dz * slice + dy * w + dx;
            }
    return n;
}

/* contact_delta_h, cpm.rs:851-876.  *num is the sum before the division. */
static double or_contact_delta(const or_lattice *l, const int32_t *reach, int nreach, double across, int32_t x,
                               int32_t y, int32_t z, int32_t src, int32_t dst, double *num) {
    double dh = 0.0;
    if (nreach > 0) {
        for (int k = 0; k < nreach; ++k) {
            int64_t a = (int64_t)x + reach[3 * k], b = (int64_t)y + reach[3 * k + 1], c = (int64_t)z + reach[3 * k + 2];
            if (a < 0 || b < 0 || c < 0 || a >= l->w || b >= l->h || c >= l->d) continue;
            int32_t nb = l->grid[(c * l->h + b) * l->w + a];
            dh += or_energy(l, dst, nb) - or_energy(l, src, nb);
        }
        *num = dh;
        return dh / across;
    }
    int64_t nbr[6];
    int nn = or_von_neumann(l, x, y, z, nbr);
    for (int k = 0; k < nn; ++k) {
        int32_t nb = l->grid[nbr[k]];
        dh += or_energy(l, dst, nb) - or_energy(l, src, nb);
    }
    *num = dh;
    return dh;
}

/* volume_delta_h, cpm.rs:879-894, on the volumes given. */
static double or_volume_delta(const or_lattice *l, const int32_t *vol, int32_t src, int32_t dst) {
    double dh = 0.0;
    if (src != 0) {
        double v = (double)vol[src], vt = (double)l->target[src];
        double a = v - 1.0 - vt, b = v - vt;
        dh += l->lambda[src] * (a * a - b * b);
    }
    if (dst != 0) {
        double v = (double)vol[dst], vt = (double)l->target[dst];
        double a = v + 1.0 - vt, b = v - vt;
        dh += l->lambda[dst] * (a * a - b * b);
    }
    return dh;
}

/* Surface constraint (extension): a cell's surface is the number of faces
 * between its pixels and pixels of any other id, lattice walls excluded.
 * Copying dst into a pixel of src changes only the surfaces of src and dst. */
static void or_surface_change(const or_lattice *l, int32_t x, int32_t y, int32_t z, int32_t src, int32_t dst,
                              int32_t *dsrc, int32_t *ddst) {
    int64_t nbr[6];
    int nn = or_von_neumann(l, x, y, z, nbr);
    int eq_src = 0, eq_dst = 0;
    for (int k = 0; k < nn; ++k) {
        int32_t nb = l->grid[nbr[k]];
        eq_src += nb == src;
        eq_dst += nb == dst;
    }
    *dsrc = eq_src - (nn - eq_src);
    *ddst = (nn - eq_dst) - eq_dst;
}

static double or_surface_delta(const or_lattice *l, const int32_t *surf, int32_t src, int32_t dst, int32_t dsrc,
                               int32_t ddst) {
    double dh = 0.0;
    if (src > 0) {
        double s = (double)surf[src], st = (double)l->target_surface[src];
        double a = s + (double)dsrc - st, b = s - st;
        dh += l->lambda_surface[src] * (a * a - b * b);
    }
    if (dst > 0) {
        double s = (double)surf[dst], st = (double)l->target_surface[dst];
        double a = s + (double)ddst - st, b = s - st;
        dh += l->lambda_surface[dst] * (a * a - b * b);
    }
    return dh;
}

/* Delta-H for copying the id `dst` into `site`, on the lattice as it
 * stands (contact_delta_h + volume_delta_h, cpm.rs:841-894, with no skip
 * rule): out[0] contact numerator, out[1] contact term, out[2] volume term,
 * out[3] surface term, out[4] adhesion+volume total, out[5] with surface. */
void or_lattice_delta_h(const or_lattice *l, int64_t site, int32_t dst, double *out) {
    int32_t reach[3 * OR_MAX_REACH];
    double across;
    int nreach = or_reach(l->order, l->d > 1, reach, &across);
    int64_t w = l->w, slice = (int64_t)l->w * l->h;
    int32_t x = (int32_t)(site % w), y = (int32_t)((site / w) % l->h), z = (int32_t)(site / slice);
    int32_t src = l->grid[site];
    double num;
    out[1] = or_contact_delta(l, reach, nreach, across, x, y, z, src, dst, &num);
    out[0] = num;
    out[2] = or_volume_delta(l, l->volume, src, dst);
    out[3] = 0.0;
    out[4] = out[1] + out[2];
    if (l->surface) {
        int32_t ds, dd;
        or_surface_change(l, x, y, z, src, dst, &ds, &dd);
        out[3] = or_surface_delta(l, l->surface, src, dst, ds, dd);
    }
    out[5] = out[4] + out[3];
}

/* splitmix64 (Steele, Lea, Flood 2014) for the sequential sweep. */
static inline uint64_t or_splitmix(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t or_range(uint64_t *s, uint64_t n) {
    return (uint64_t)(((unsigned __int128)or_splitmix(s) * n) >> 64);
}

/* occupied_span, cpm.rs:777-793. */
int or_occupied_span(const or_lattice *l, int32_t *span6) {
    int64_t w = l->w, slice = (int64_t)l->w * l->h, n = slice * l->d;
    int found = 0;
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
        if (l->grid[i] == 0) continue;
        int32_t p[3] = {(int32_t)(i % w), (int32_t)((i / w) % l->h), (int32_t)(i / slice)};
        if (!found) {
            for (int a = 0; a < 3; ++a) lo[a] = hi[a] = p[a];
            found = 1;
        }
        for (int a = 0; a < 3; ++a) {
            if (p[a] < lo[a]) lo[a] = p[a];
            if (p[a] > hi[a]) hi[a] = p[a];
        }
    }
    int32_t lim[3] = {l->w, l->h, l->d};
    for (int a = 0; a < 3 && found; ++a) {
        span6[2 * a] = lo[a] > 0 ? lo[a] - 1 : 0;
        span6[2 * a + 1] = hi[a] + 1 < lim[a] - 1 ? hi[a] + 1 : lim[a] - 1;
    }
    return found;
}

/* try_flip, cpm.rs:797-838, drawing from splitmix64.  Immune chemotaxis
 * (cpm.rs:816-822) belongs to the immune scenarios and is not restated. */
static void or_try_flip(or_lattice *l, const int32_t *reach, int nreach, double across, int32_t x, int32_t y,
                        int32_t z, uint64_t *rng) {
    int64_t w = l->w, slice = (int64_t)l->w * l->h, site = (int64_t)z * slice + (int64_t)y * w + x;
    int32_t src = l->grid[site];
    int64_t nbr[26];
    int nn = or_copy_neighbours(l, x, y, z, nbr);
    if (nn == 0) return;
    int32_t dst = l->grid[nbr[or_range(rng, (uint64_t)nn)]];
    if (src == dst || src == OR_OBSTACLE || dst == OR_OBSTACLE) return;
    double num;
    double delta = or_contact_delta(l, reach, nreach, across, x, y, z, src, dst, &num) + or_volume_delta(l, l->volume, src, dst);
    int32_t ds = 0, dd = 0;
    if (l->surface) {
        or_surface_change(l, x, y, z, src, dst, &ds, &dd);
        delta += or_surface_delta(l, l->surface, src, dst, ds, dd);
    }
    int accept = delta <= 0.0;
    if (!accept) accept = (double)(or_splitmix(rng) >> 11) * (1.0 / 9007199254740992.0) < exp(-delta / l->temperature);
    if (accept) {
        l->grid[site] = dst;
        if (src != 0) l->volume[src] -= 1;
        if (dst != 0) l->volume[dst] += 1;
        if (l->surface) {
            if (src > 0) l->surface[src] += ds;
            if (dst > 0) l->surface[dst] += dd;
        }
    }
}

/* monte_carlo_step, cpm.rs:748-772, `sweeps` times: the reference's
 * sequential random-site Metropolis. */
void or_lattice_mcs_sequential(or_lattice *l, uint64_t seed, int32_t sweeps) {
    int32_t reach[3 * OR_MAX_REACH];
    double across;
    int nreach = or_reach(l->order, l->d > 1, reach, &across);
    uint64_t rng = seed;
    for (int32_t s = 0; s < sweeps; ++s) {
        if (l->d > 1) {
            int32_t sp[6];
            if (!or_occupied_span(l, sp)) continue;
            int64_t n = (int64_t)(sp[1] - sp[0] + 1) * (sp[3] - sp[2] + 1) * (sp[5] - sp[4] + 1);
            for (int64_t k = 0; k < n; ++k) {
                int32_t x = sp[0] + (int32_t)or_range(&rng, (uint64_t)(sp[1] - sp[0] + 1));
                int32_t y = sp[2] + (int32_t)or_range(&rng, (uint64_t)(sp[3] - sp[2] + 1));
                int32_t z = sp[4] + (int32_t)or_range(&rng, (uint64_t)(sp[5] - sp[4] + 1));
                or_try_flip(l, reach, nreach, across, x, y, z, &rng);
            }
        } else {
            int64_t n = (int64_t)l->w * l->h;
            for (int64_t k = 0; k < n; ++k) {
                int32_t x = (int32_t)or_range(&rng, (uint64_t)l->w);
                int32_t y = (int32_t)or_range(&rng, (uint64_t)l->h);
                or_try_flip(l, reach, nreach, across, x, y, 0, &rng);
            }
        }
    }
}

/* ---- the sublattice scheme the GPU runs, restated on the CPU ----------- */

/* Colouring: with faces only (contact and copy), the chessboard (x+y+z) mod
 * 2; otherwise a period p = R+1 in every axis, R the Chebyshev radius of the
 * contact reach (1 for face contact with Moore copy), so that no pixel of a
 * colour lies within the reach, or the copy neighbourhood, of another. */
int or_colouring(const or_lattice *l, int32_t *period) {
    int32_t reach[3 * OR_MAX_REACH];
    double across;
    int n = or_reach(l->order, l->d > 1, reach, &across);
    if (n == 0 && !l->copy_moore) { *period = 0; return 2; }
    int32_t r = 1;
    for (int k = 0; k < 3 * n; ++k) {
        int32_t a = reach[k] < 0 ? -reach[k] : reach[k];
        if (a > r) r = a;
    }
    int32_t p = r + 1;
    *period = p;
    return l->d > 1 ? p * p * p : p * p;
}

static inline int32_t or_colour_of(int32_t period, int32_t x, int32_t y, int32_t z) {
    if (period == 0) return (x + y + z) & 1;
    return (x % period) + period * (y % period) + period * period * (z % period);
}

/* The order the colours are swept in during lattice step `mcs`: a
 * Fisher-Yates shuffle driven by Philox with the site word all ones. */
void or_colour_order(int32_t ncol, uint32_t mcs, uint32_t k0, uint32_t k1, int32_t *perm) {
    for (int32_t i = 0; i < ncol; ++i) perm[i] = i;
    for (int32_t i = ncol - 1; i > 0; --i) {
        or_u32x4 r = or_philox(0xFFFFFFFFu, mcs, 1u, (uint32_t)i, k0, k1);
        int32_t j = (int32_t)(((uint64_t)r.v[0] * (uint64_t)(i + 1)) >> 32);
        int32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t;
    }
}

/* MurmurHash3's 32-bit finaliser (Appleby): a bijection of 32-bit words, so
 * distinct pixels of one pass get distinct priorities. */
static inline uint32_t or_fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

/* A pass's priority of pixel `site`: the pass's key is word 0 of
 * Philox(0xFFFFFFFE, step, 2, colour) under the history's key. */
uint32_t or_pass_priority(uint32_t site, uint32_t mcs, int32_t colour, uint32_t k0, uint32_t k1) {
    or_u32x4 r = or_philox(0xFFFFFFFEu, mcs, 2u, (uint32_t)colour, k0, k1);
    return or_fmix32(site ^ r.v[0]);
}

typedef struct {
    uint32_t prio;
    int64_t site;
} or_ranked;

static int or_by_priority_desc(const void *a, const void *b) {
    uint32_t pa = ((const or_ranked *)a)->prio, pb = ((const or_ranked *)b)->prio;
    return pa < pb ? 1 : (pa > pb ? -1 : 0);
}

/* `sweeps` lattice steps of the sublattice scheme, starting at step counter
 * `mcs0`.  Per colour pass every pixel of the colour makes one attempt from
 * draws Philox(site, mcs, 0, 0) under key (k0, k1), the pixels taken one at a
 * time in decreasing pass priority (or_pass_priority), each seeing the
 * volumes and surfaces every earlier one left.  The pixels of a colour lie
 * outside one another's reach, so two attempts of a pass meet only through
 * the records of a cell they share; the device runs the attempts that share
 * no cell at once and settles the others in priority order, which is this
 * sequence.
 *
 * `snapshot` != 0 is a planted mistake for the statistical tests: every
 * attempt of a pass reads the volumes and surfaces the pass started with. */
void or_lattice_mcs_checkerboard(or_lattice *l, uint32_t k0, uint32_t k1, uint32_t mcs0, int32_t sweeps,
                                 int32_t snapshot, int32_t subsweeps) {
    int32_t reach[3 * OR_MAX_REACH];
    double across;
    int nreach = or_reach(l->order, l->d > 1, reach, &across);
    int32_t period;
    int32_t ncol = or_colouring(l, &period);
    int32_t perm[27];
    int64_t w = l->w, slice = (int64_t)l->w * l->h, n = slice * l->d;
    or_ranked *order = (or_ranked *)malloc(sizeof(or_ranked) * (size_t)(n > 0 ? n : 1));
    int32_t *vsnap = snapshot ? (int32_t *)malloc(sizeof(int32_t) * (size_t)l->ncells) : NULL;
    int32_t *ssnap = snapshot && l->surface ? (int32_t *)malloc(sizeof(int32_t) * (size_t)l->ncells) : NULL;
    /* subsweeps > 1: every colour swept that many times a Monte Carlo step, a
     * pixel attempting in each sweep when its draw (counter word 2 = 4) is
     * below 2^32 / subsweeps; the draws count sub-sweeps */
    if (subsweeps < 1) subsweeps = 1;
    const uint32_t take_below = subsweeps > 1 ? (uint32_t)(4294967296.0 / (double)subsweeps) : 0u;
    /* in a volume a Monte Carlo step visits the occupied span at its start
     * (monte_carlo_step, cpm.rs:748-763): the box around every pixel that is
     * not medium, one wider on every side; nothing when all is medium.  A
     * plane visits the whole box. */
    int32_t sp[6] = {0, l->w - 1, 0, l->h - 1, 0, l->d - 1};
    int occupied = 1;
    for (int32_t s = 0; s < sweeps * subsweeps; ++s) {
        uint32_t mcs = mcs0 * (uint32_t)subsweeps + (uint32_t)s;
        if (l->d > 1 && s % subsweeps == 0) occupied = or_occupied_span(l, sp);
        or_colour_order(ncol, mcs, k0, k1, perm);
        for (int32_t q = 0; q < ncol; ++q) {
            int32_t colour = perm[q];
            if (vsnap) memcpy(vsnap, l->volume, sizeof(int32_t) * (size_t)l->ncells);
            if (ssnap) memcpy(ssnap, l->surface, sizeof(int32_t) * (size_t)l->ncells);
            const int32_t *vol = vsnap ? vsnap : l->volume;
            const int32_t *surf = ssnap ? ssnap : l->surface;
            int64_t m = 0;
            for (int32_t z = sp[4]; occupied && z <= sp[5]; ++z)
                for (int32_t y = sp[2]; y <= sp[3]; ++y)
                    for (int32_t x = sp[0]; x <= sp[1]; ++x) {
                        if (or_colour_of(period, x, y, z) != colour) continue;
                        int64_t site = (int64_t)z * slice + (int64_t)y * w + x;
                        order[m].site = site;
                        order[m].prio = or_pass_priority((uint32_t)site, mcs, colour, k0, k1);
                        ++m;
                    }
            qsort(order, (size_t)m, sizeof(or_ranked), or_by_priority_desc);
            for (int64_t e = 0; e < m; ++e) {
                int64_t site = order[e].site;
                int32_t x = (int32_t)(site % w), y = (int32_t)((site / w) % l->h), z = (int32_t)(site / slice);
                int64_t nbr[26];
                int nn = or_copy_neighbours(l, x, y, z, nbr);
                if (nn == 0) continue;
                if (take_below && or_philox((uint32_t)site, mcs, 4u, 0u, k0, k1).v[0] >= take_below) continue;
                or_u32x4 r = or_philox((uint32_t)site, mcs, 0u, 0u, k0, k1);
                int32_t src = l->grid[site];
                int32_t dst = l->grid[nbr[((uint64_t)r.v[0] * (uint64_t)nn) >> 32]];
                if (src == dst || src == OR_OBSTACLE || dst == OR_OBSTACLE) continue;
                double num;
                double delta = or_contact_delta(l, reach, nreach, across, x, y, z, src, dst, &num) +
                               or_volume_delta(l, vol, src, dst);
                int32_t ds = 0, dd = 0;
                if (l->surface) {
                    or_surface_change(l, x, y, z, src, dst, &ds, &dd);
                    delta += or_surface_delta(l, surf, src, dst, ds, dd);
                }
                int accept = delta <= 0.0;
                if (!accept) accept = or_u01(r.v[1], r.v[2]) < or_cw_exp(-delta / l->temperature);
                if (accept) {
                    l->grid[site] = dst;
                    if (src != 0) l->volume[src] -= 1;
                    if (dst != 0) l->volume[dst] += 1;
                    if (l->surface) {
                        if (src > 0) l->surface[src] += ds;
                        if (dst > 0) l->surface[dst] += dd;
                    }
                }
            }
        }
    }
    free(order);
    free(vsnap);
    free(ssnap);
}

/* divide_across, cpm.rs:1094-1160: split cell `id` across the plane through
 * its centre of mass with normal (nx, ny, nz) (nz counts in a volume only);
 * the pixels with (x - cx) nx + (y - cy) ny [+ (z - cz) nz] > 0 go to a new
 * record *used (which then advances), of the parent's kind and volume
 * parameters.  -1, nothing changed: the medium, an unknown id, fewer than 8
 * pixels (cpm.rs:132), a plane leaving one side empty, or no free record. */
int32_t or_lattice_divide_across(or_lattice *l, int32_t id, double nx, double ny, double nz, int32_t *used) {
    if (id <= 0 || id >= *used) return -1;
    int64_t w = l->w, slice = (int64_t)l->w * l->h, n = slice * l->d;
    int64_t total = 0;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int64_t i = 0; i < n; ++i)
        if (l->grid[i] == id) {
            sx += (double)(i % w);
            sy += (double)((i / w) % l->h);
            sz += (double)(i / slice);
            ++total;
        }
    if (total < 8) return -1;
    if (*used >= l->ncells) return -1;
    double fn = (double)total, cx = sx / fn, cy = sy / fn, cz = l->d > 1 ? sz / fn : 0.0;
    int32_t daughter = *used;
    int64_t moved = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (l->grid[i] != id) continue;
        double x = (double)(i % w), y = (double)((i / w) % l->h), z = (double)(i / slice);
        double side = (x - cx) * nx + (y - cy) * ny;
        if (l->d > 1) side += (z - cz) * nz;
        if (side > 0.0) { l->grid[i] = daughter; ++moved; }
    }
    if (moved == 0 || moved == total) {
        for (int64_t i = 0; i < n; ++i)
            if (l->grid[i] == daughter) l->grid[i] = id;
        return -1;
    }
    l->volume[id] = (int32_t)(total - moved);
    l->type[daughter] = l->type[id];
    l->volume[daughter] = (int32_t)moved;
    l->target[daughter] = l->target[id];
    l->lambda[daughter] = l->lambda[id];
    if (l->surface) {
        l->target_surface[daughter] = l->target_surface[id];
        l->lambda_surface[daughter] = l->lambda_surface[id];
    }
    *used += 1;
    return daughter;
}

/* Recount volumes (and surfaces) from the grid: records_match_grid,
 * cpm.rs:1262-1279.  Obstacles are skipped; ids past ncells are ignored. */
void or_lattice_recount(const or_lattice *l, int32_t *volume, int32_t *surface) {
    int64_t w = l->w, slice = (int64_t)l->w * l->h, n = slice * l->d;
    memset(volume, 0, sizeof(int32_t) * (size_t)l->ncells);
    if (surface) memset(surface, 0, sizeof(int32_t) * (size_t)l->ncells);
    for (int64_t i = 0; i < n; ++i) {
        int32_t id = l->grid[i];
        if (id == OR_OBSTACLE || id < 0 || id >= l->ncells) continue;
        volume[id] += 1;
        if (surface && id > 0) {
            int32_t x = (int32_t)(i % w), y = (int32_t)((i / w) % l->h), z = (int32_t)(i / slice);
            int64_t nbr[6];
            int nn = or_von_neumann(l, x, y, z, nbr);
            for (int k = 0; k < nn; ++k) surface[id] += l->grid[nbr[k]] != id;
        }
    }
}

/* ======================================================================
 * Protein network: network.rs
 * ====================================================================== */
enum { OR_ACTIVATED_BY = 0, OR_INHIBITED_BY, OR_ACTIVATED_BY_ABSENCE_OF, OR_PRODUCED_BY, OR_DECAYS,
       OR_RELAXES_TO, OR_DAMAGED_BELOW, OR_DAMAGED_ABOVE };

typedef struct {
    int32_t S;          /* nodes */
    int32_t *node_ptr;  /* S+1: terms of node i are [node_ptr[i], node_ptr[i+1]) in file order */
    int32_t *kind;      /* per term, the enum above */
    int32_t *source;    /* >= 0 a node; -1-k an input: 0 oxygen, 1 egf, 2 crowding, 3 stress, 4 waste, 5 necrotic_factor */
    double *rate;
    double *hill_n;     /* <= 0: no Hill response */
    double *hill_k;
    double *param;      /* relaxes_to value, or damaged_* threshold */
} or_network;

/* driver, network.rs:56-64. */
static inline double or_driver(double s, double n, double half) {
    if (!(n > 0.0)) return s;
    double sn = pow(fmax(s, 0.0), n);
    return sn / (pow(half, n) + sn);
}

/* read, network.rs:670-680; `in` holds o2, egf, crowding, stress, waste, necrotic factor. */
static inline double or_read(const double *state, const double *in, int32_t source) {
    if (source >= 0) return state[source];
    switch (-1 - source) {
    case 0: return fmin(fmax(in[0], 0.0), 1.0);
    case 1: return in[1];
    case 2: return fmin(fmax(in[2], 0.0), 1.0);
    case 3: return fmax(in[3], 0.0);
    case 4: return fmax(in[4], 0.0);
    default: return fmax(in[5], 0.0);
    }
}

/* derivatives + term_rate, network.rs:686-734. */
static void or_derivatives(const or_network *net, const double *state, const double *in, double *out) {
    for (int32_t i = 0; i < net->S; ++i) {
        double own = state[i], rate = 0.0;
        for (int32_t t = net->node_ptr[i]; t < net->node_ptr[i + 1]; ++t) {
            double k = net->rate[t], r;
            switch (net->kind[t]) {
            case OR_ACTIVATED_BY:
                r = k * or_driver(or_read(state, in, net->source[t]), net->hill_n[t], net->hill_k[t]) * (1.0 - own);
                break;
            case OR_INHIBITED_BY:
                r = -k * or_driver(or_read(state, in, net->source[t]), net->hill_n[t], net->hill_k[t]) * own;
                break;
            case OR_ACTIVATED_BY_ABSENCE_OF:
                r = k * (1.0 - or_read(state, in, net->source[t])) * (1.0 - own);
                break;
            case OR_PRODUCED_BY: r = k * or_read(state, in, net->source[t]); break;
            case OR_DECAYS: r = -k * own; break;
            case OR_RELAXES_TO: r = -k * (own - net->param[t]); break;
            case OR_DAMAGED_BELOW: {
                double s = or_read(state, in, net->source[t]), th = net->param[t];
                r = -k * fmax((th - s) / th, 0.0);
                break;
            }
            default: {
                double s = or_read(state, in, net->source[t]), th = net->param[t];
                r = -k * fmax((s - th) / th, 0.0);
                break;
            }
            }
            rate += r;
        }
        out[i] = rate;
    }
}

/* rk4, network.rs:777-799, `substeps` times per cell.  state is [ncells][S]
 * row-major, inputs [ncells][6]. */
void or_network_step(const or_network *net, int64_t ncells, double *state, const double *inputs, double dt,
                     int32_t substeps) {
    int32_t S = net->S;
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * (size_t)S * 6);
        double *x = buf, *mid = buf + S, *k0 = buf + 2 * S, *k1 = buf + 3 * S, *k2 = buf + 4 * S, *k3 = buf + 5 * S;
        double *k[4] = {k0, k1, k2, k3};
#pragma omp for schedule(static)
        for (int64_t c = 0; c < ncells; ++c) {
            double *st = state + c * S;
            const double *in = inputs + c * 6;
            for (int32_t sub = 0; sub < substeps; ++sub) {
                for (int32_t i = 0; i < S; ++i) x[i] = st[i];
                or_derivatives(net, x, in, k[0]);
                for (int stage = 0; stage < 3; ++stage) {
                    double step = stage < 2 ? 0.5 * dt : dt;
                    for (int32_t i = 0; i < S; ++i) mid[i] = x[i] + step * k[stage][i];
                    or_derivatives(net, mid, in, k[stage + 1]);
                }
                for (int32_t i = 0; i < S; ++i) {
                    double delta = (dt / 6.0) * (k0[i] + 2.0 * k1[i] + 2.0 * k2[i] + k3[i]);
                    st[i] = fmin(fmax(x[i] + delta, 0.0), 1.0);
                }
            }
        }
        free(buf);
    }
}

/* mechanics, network.rs:811-821: target = (ref * min(1 + c*growth, max)) as u32. */
void or_network_mechanics(int64_t ncells, int32_t S, const double *state, int32_t growth, double coefficient,
                          double max_target, int has_max, uint32_t reference_volume, uint32_t *target) {
    for (int64_t c = 0; c < ncells; ++c) {
        double g = state[c * S + growth];
        double ratio = 1.0 + coefficient * g;
        if (has_max) ratio = fmin(ratio, max_target);
        double t = fmax((double)reference_volume * ratio, 0.0);
        target[c] = isnan(t) ? 0u : (t >= 4294967295.0 ? 4294967295u : (uint32_t)t);
    }
}

/* ======================================================================
 * Coupling: coupling.rs
 * ====================================================================== */

/* apply_uptake (coupling.rs:26-39) with a rate per kind: every pixel of a
 * cell whose kind has a positive rate sinks it; rates are floored at zero as
 * set_uptake_at does.  Clears the sinks first. */
void or_apply_uptake(int64_t n, const int32_t *grid, int32_t ncells, const int32_t *type, const double *rate_by_type,
                     double *uptake) {
    for (int64_t i = 0; i < n; ++i) {
        uptake[i] = 0.0;
        int32_t id = grid[i];
        if (id == 0 || id == OR_OBSTACLE || id < 0 || id >= ncells) continue;
        double r = rate_by_type[type[id]];
        if (r != 0.0) uptake[i] = fmax(r, 0.0);
    }
}

/* apply_background_uptake, coupling.rs:47-53. */
void or_apply_background_uptake(int64_t n, const int32_t *grid, double rate, double *uptake) {
    for (int64_t i = 0; i < n; ++i)
        if (grid[i] == 0) uptake[i] = fmax(rate, 0.0);
}

/* apply_production, coupling.rs:61-73. */
void or_apply_production(int64_t n, const int32_t *grid, int64_t nrates, const double *per_cell, double *production) {
    for (int64_t i = 0; i < n; ++i) {
        production[i] = 0.0;
        int32_t id = grid[i];
        if (id == 0 || id == OR_OBSTACLE || id < 0 || id >= nrates) continue;
        if (per_cell[id] > 0.0) production[i] = per_cell[id];
    }
}

/* hold_obstacles_at, coupling.rs:80-82 (hold_where, pde.rs:491-498). */
void or_hold_obstacles(int64_t n, const int32_t *grid, double value, uint8_t *held, double *values) {
    for (int64_t i = 0; i < n; ++i)
        if (grid[i] == OR_OBSTACLE) { held[i] = 1; values[i] = value; }
}

/* hold_vessels_by, coupling.rs:114-150, on a w x h plane: every obstacle pixel
 * whose delivery share is above zero is held at value x min(share, 1), unless
 * the mean of the field over its in-box, non-obstacle neighbours (x-1, x+1,
 * y-1, y+1, summed in that order) is at least that level.  Every decision
 * reads the field as it stood before any hold (the holds are applied after,
 * hold_pixels_by, pde.rs:504-514); only obstacle pixels are written and only
 * other pixels are read, so deciding and holding in one loop is the same. */
void or_hold_vessels_by(int32_t w, int32_t h, const int32_t *grid, double value, const double *delivery,
                        uint8_t *held, double *values) {
    for (int32_t y = 0; y < h; ++y)
        for (int32_t x = 0; x < w; ++x) {
            const int64_t i = (int64_t)y * w + x;
            if (grid[i] != OR_OBSTACLE) continue;
            const double share = delivery[i];
            if (share <= 0.0) continue;
            /* f64::min and fmin both give the number when one side is NaN */
            const double level = value * fmin(share, 1.0);
            const int32_t nx[4] = {x - 1, x + 1, x, x};
            const int32_t ny[4] = {y, y, y - 1, y + 1};
            double sum = 0.0;
            int n = 0;
            for (int q = 0; q < 4; ++q) {
                if (nx[q] < 0 || nx[q] >= w || ny[q] < 0 || ny[q] >= h) continue;
                const int64_t j = (int64_t)ny[q] * w + nx[q];
                if (grid[j] == OR_OBSTACLE) continue;
                sum += values[j];
                n += 1;
            }
            const int richer = n > 0 && sum / (double)n >= level;
            if (!richer) { held[i] = 1; values[i] = level; }
        }
}

/* mean_per_cell, coupling.rs:164-182: sums in lattice order. */
void or_mean_per_cell(int64_t n, const int32_t *grid, const double *values, int32_t ncells, double *out) {
    double *sum = (double *)calloc((size_t)ncells, sizeof(double));
    uint32_t *count = (uint32_t *)calloc((size_t)ncells, sizeof(uint32_t));
    for (int64_t i = 0; i < n; ++i) {
        int32_t id = grid[i];
        if (id == 0 || id == OR_OBSTACLE || id < 0 || id >= ncells) continue;
        sum[id] += values[i];
        count[id] += 1;
    }
    for (int32_t c = 0; c < ncells; ++c) out[c] = count[c] == 0 ? 0.0 : sum[c] / (double)count[c];
    free(sum);
    free(count);
}

int or_version(void) { return 1; }
