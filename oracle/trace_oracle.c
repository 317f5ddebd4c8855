/*
 * ORACLE -- test infrastructure only.  Nothing in the trench_b200 product links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it, as the checker.
 *
 * Scalar FP64 restatement of the reference CPU particle tracer
 * (trench_charging_2d.py:542-702, `trace_cpu`), one particle at a time.  The
 * reference advances all live particles together with NumPy; every particle is
 * independent, so running each particle to completion gives identical values.
 * Each arithmetic expression keeps the reference's operand order so results are
 * bit-identical to NumPy (no FMA contraction: built with -ffp-contract=off).
 *
 *   interp()      trench_charging_2d.py:492-509  (vacuum-weighted bilinear)
 *   wall_entry()  trench_charging_2d.py:512-539  (first solid face crossed)
 *   rf_coeff()    trench_rf.py:5-11              (periodic linear interpolation)
 *   trace_one()   trench_charging_2d.py:579-694  (step loop, barrier, record)
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <pthread.h>

typedef struct {
    const double *ex, *ey;          /* (nx, ny) C order */
    const uint8_t *vac;             /* 1 = vacuum */
    const double *phi, *wface;      /* barrier; NULL = absorb model */
    const double *rf_ex, *rf_ey, *rf_phi;   /* (2, nx, ny) or NULL */
    const double *wave;             /* (n_phase, 2) */
    int n_phase;
    double period, dt_max, bound_vs, bound_vm;
    int nx, ny;
    double dx, cfl;
    int max_steps, tapered, record;
    int path_stride;
} oracle_case;

/* numpy float remainder for a positive modulus (npy_divmod). */
static double pymod(double a, double b) {
    double m = fmod(a, b);
    if (m != 0.0) {
        if ((m < 0.0) != (b < 0.0)) m += b;
    } else {
        m = copysign(0.0, b);
    }
    return m;
}

static int64_t clip64(int64_t i, int64_t n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); }
static int64_t pmod64(int64_t i, int64_t n) { int64_t r = i % n; return r < 0 ? r + n : r; }

/* F = (E*vac, vac) gathered at the 4 corners; trench_charging_2d.py:492-509. */
static void interp(const oracle_case *c, const double *ex, const double *ey, double x, double y,
                   double *ox, double *oy) {
    const int nx = c->nx, ny = c->ny;
    double fx = x / c->dx - 0.5, fy = y / c->dx - 0.5;
    int64_t i0 = (int64_t)floor(fx), j0 = (int64_t)floor(fy);
    double tx = fx - (double)i0, ty = fy - (double)j0;
    int64_t i1 = pmod64(i0 + 1, nx);
    i0 = pmod64(i0, nx);
    int64_t j1 = clip64(j0 + 1, ny);
    j0 = clip64(j0, ny);
    int64_t k[4] = {i0 * ny + j0, i1 * ny + j0, i0 * ny + j1, i1 * ny + j1};
    double w[4] = {(1.0 - tx) * (1.0 - ty), tx * (1.0 - ty), (1.0 - tx) * ty, tx * ty};
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int q = 0; q < 4; ++q) {
        double v = (double)c->vac[k[q]];
        a0 = (q ? a0 + w[q] * (ex[k[q]] * v) : w[q] * (ex[k[q]] * v));
        a1 = (q ? a1 + w[q] * (ey[k[q]] * v) : w[q] * (ey[k[q]] * v));
        a2 = (q ? a2 + w[q] * v : w[q] * v);
    }
    double s = a2 > 1e-12 ? a2 : 1e-12;
    *ox = a0 / s;
    *oy = a1 / s;
}

/* trench_charging_2d.py:512-539 */
static void wall_entry(const oracle_case *c, double x0, double y0, double sx, double sy,
                       int64_t *cx, int64_t *cy, int64_t *vx_, int64_t *vy_, int *face_x) {
    const int nx = c->nx, ny = c->ny;
    const double dx = c->dx;
    int64_t ix0 = (int64_t)(x0 / dx); if (ix0 > nx - 1) ix0 = nx - 1;
    int64_t iy0 = clip64((int64_t)(y0 / dx), ny);
    double xu = x0 + sx, yu = y0 + sy;
    int64_t dix = (int64_t)floor(xu / dx) - ix0;
    int64_t diy = clip64((int64_t)floor(yu / dx), ny) - iy0;
    double fx = dix != 0 ? ((double)(ix0 + (dix > 0)) * dx - x0) / sx : INFINITY;
    double fy = diy != 0 ? ((double)(iy0 + (diy > 0)) * dx - y0) / sy : INFINITY;
    int x_first = fx < fy;
    int64_t ax = x_first ? pmod64(ix0 + dix, nx) : ix0;
    int64_t ay = x_first ? iy0 : iy0 + diy;
    int diag = (dix != 0) && (diy != 0);
    int first_solid = !c->vac[ax * ny + ay];
    int64_t lx = pmod64(ix0 + dix, nx), ly = iy0 + diy;
    int use_last = diag && !first_solid;
    *cx = use_last ? lx : ax;
    *cy = use_last ? ly : ay;
    *vx_ = use_last ? ax : ix0;
    *vy_ = use_last ? ay : iy0;
    *face_x = use_last ? !x_first : x_first;
}

/* trench_rf.py:5-11 */
static void rf_coeff(const oracle_case *c, double at, double *vs, double *vm) {
    double f = pymod(at, c->period) / c->period * (double)c->n_phase;
    int64_t i = pmod64((int64_t)floor(f), c->n_phase);
    int64_t j = pmod64(i + 1, c->n_phase);
    double w = f - floor(f);
    *vs = c->wave[2 * i] * (1.0 - w) + c->wave[2 * j] * w;
    *vm = c->wave[2 * i + 1] * (1.0 - w) + c->wave[2 * j + 1] * w;
}

/* One particle, trench_charging_2d.py:579-694.  Returns status 1/2/3. */
static int trace_one(const oracle_case *c, double *px, double *py, double *pvx, double *pvy, double qm,
                     double *pclock, double *pelapsed, int32_t *hit, int32_t *nsteps,
                     double *endpoint, double *path, int32_t *path_len) {
    const int nx = c->nx, ny = c->ny;
    const double dx = c->dx, Lx = nx * dx, Ly = ny * dx;
    double x = *px, y = *py, vx = *pvx, vy = *pvy;
    double clock = pclock ? *pclock : 0.0, elapsed = pelapsed ? *pelapsed : 0.0;
    const int rf = c->n_phase > 0;
    int status = 3, k;
    int32_t plen = path_len ? *path_len : 0;
    for (k = 0; k < c->max_steps; ++k) {
        double ex, ey;
        interp(c, c->ex, c->ey, x, y, &ex, &ey);
        double ax = qm * ex, ay = qm * ey;
        double speed = hypot(vx, vy);
        double dt;
        if (!rf) {
            dt = c->cfl * dx / (speed + sqrt(2.0 * dx * hypot(ax, ay)) + 1.0);
        } else {
            const size_t cells = (size_t)nx * ny;
            double exs, eys, exm, eym;
            interp(c, c->rf_ex, c->rf_ey, x, y, &exs, &eys);
            interp(c, c->rf_ex + cells, c->rf_ey + cells, x, y, &exm, &eym);
            double bx = fabs(ex) + (c->bound_vs * fabs(exs) + c->bound_vm * fabs(exm));
            double by = fabs(ey) + (c->bound_vs * fabs(eys) + c->bound_vm * fabs(eym));
            double accel = fabs(qm) * hypot(bx, by);
            double d = c->cfl * dx / (speed + sqrt(2 * dx * accel) + 1);
            dt = c->dt_max < d ? c->dt_max : d;
            double vs, vm;
            rf_coeff(c, clock + dt / 2, &vs, &vm);
            ex = ex + (vs * exs + vm * exm);
            ey = ey + (vs * eys + vm * eym);
            ax = qm * ex; ay = qm * ey;
            clock = pymod(clock + dt, c->period);
            elapsed = elapsed + dt;
        }
        double vxn = vx + ax * dt, vyn = vy + ay * dt;
        double x0 = x, y0 = y;
        double sx = 0.5 * (vx + vxn) * dt, sy = 0.5 * (vy + vyn) * dt;
        x = pymod(x + sx, Lx);
        y = y + sy;
        vx = vxn; vy = vyn;

        int escaped = y >= Ly;
        int64_t ix = (int64_t)(x / dx); if (ix > nx - 1) ix = nx - 1;
        int64_t iy = clip64((int64_t)(y / dx), ny);
        int is_hit = !escaped && !c->vac[ix * ny + iy];
        int64_t cx, cy, vcx, vcy; int face_x;
        if (c->tapered && !is_hit && !escaped) {
            int64_t ix0 = (int64_t)(x0 / dx); if (ix0 > nx - 1) ix0 = nx - 1;
            int64_t iy0 = clip64((int64_t)(y0 / dx), ny);
            if (ix != ix0 && iy != iy0) {
                wall_entry(c, x0, y0, sx, sy, &cx, &cy, &vcx, &vcy, &face_x);
                is_hit = !c->vac[cx * ny + cy];
            }
        }
        if (c->phi && is_hit) {
            wall_entry(c, x0, y0, sx, sy, &cx, &cy, &vcx, &vcy, &face_x);
            double vn = face_x ? vx : vy;
            int64_t cc = cx * ny + cy, vv = vcx * ny + vcy;
            double dphi = c->wface[cc] * (c->phi[cc] - c->phi[vv]);
            if (rf) {
                const size_t cells = (size_t)nx * ny;
                double vs, vm;
                rf_coeff(c, clock, &vs, &vm);
                double d0 = c->rf_phi[cc] - c->rf_phi[vv];
                double d1 = c->rf_phi[cells + cc] - c->rf_phi[cells + vv];
                dphi += c->wface[cc] * (vs * d0 + vm * d1);
            }
            if (0.5 * (vn * vn) < qm * dphi) {
                if (face_x) vx = -vx; else vy = -vy;
                x = x0; y = y0;
                is_hit = 0;
            }
            ix = cx; iy = cy;
        }
        if ((c->record || c->tapered) && !c->phi && is_hit) {
            wall_entry(c, x0, y0, sx, sy, &cx, &cy, &vcx, &vcy, &face_x);
            ix = cx; iy = cy;
        }
        if (c->record) {
            double xp = x, yp = y, tf = 1.0;
            if (is_hit) {
                wall_entry(c, x0, y0, sx, sy, &cx, &cy, &vcx, &vcy, &face_x);
                double frac;
                if (face_x) {
                    double xb = (double)(cx + (sx < 0)) * dx;
                    xb += nearbyint((x0 - xb) / Lx) * Lx;
                    frac = (xb - x0) / sx;
                } else {
                    frac = ((double)(cy + (sy < 0)) * dx - y0) / sy;
                }
                frac = frac < 0 ? 0 : (frac > 1 ? 1 : frac);
                tf = frac;
                xp = pymod(x0 + frac * sx, Lx);
                yp = y0 + frac * sy;
            } else if (escaped) {
                double frac = (Ly - y0) / sy;
                frac = frac < 0 ? 0 : (frac > 1 ? 1 : frac);
                tf = frac;
                xp = pymod(x0 + frac * sx, Lx);
                yp = Ly;
            }
            if (endpoint) { endpoint[0] = xp; endpoint[1] = yp; }
            if (rf && (is_hit || escaped)) {
                clock = pymod(clock - (1 - tf) * dt, c->period);
                elapsed = elapsed - (1 - tf) * dt;
            }
            if (path && plen < c->path_stride) {
                path[2 * plen] = xp; path[2 * plen + 1] = yp;
                ++plen;
            }
        }
        if (is_hit) {
            status = 1;
            *hit = (int32_t)(ix * ny + iy);
            ++k;
            break;
        }
        if (escaped) {
            status = 2;
            ++k;
            break;
        }
    }
    *px = x; *py = y; *pvx = vx; *pvy = vy;
    if (pclock) *pclock = clock;
    if (pelapsed) *pelapsed = elapsed;
    if (nsteps) *nsteps = k;
    if (path_len) *path_len = plen;
    return status;
}

/* Work shared by the worker threads: particles are handed out in blocks of 64
 * through an atomic counter; each particle is independent of every other. */
typedef struct {
    const oracle_case *c;
    int64_t n;
    double *x, *y, *vx, *vy, *clock, *elapsed, *endpoints, *paths;
    const double *qm;
    const int32_t *slots;
    int32_t *path_len, *hit, *steps;
    int8_t *status;
    int64_t next;   /* atomic */
} oracle_job;

static void *worker(void *arg) {
    oracle_job *j = (oracle_job *)arg;
    const oracle_case *c = j->c;
    for (;;) {
        int64_t b = __atomic_fetch_add(&j->next, 64, __ATOMIC_RELAXED);
        if (b >= j->n) break;
        int64_t e = b + 64 < j->n ? b + 64 : j->n;
        for (int64_t i = b; i < e; ++i) {
            int32_t slot = (c->record && j->slots) ? j->slots[i] : -1;
            j->hit[i] = -1;
            j->status[i] = (int8_t)trace_one(
                c, j->x + i, j->y + i, j->vx + i, j->vy + i, j->qm[i],
                c->n_phase ? j->clock + i : NULL, c->n_phase ? j->elapsed + i : NULL, j->hit + i,
                j->steps ? j->steps + i : NULL, c->record && j->endpoints ? j->endpoints + 2 * i : NULL,
                slot >= 0 ? j->paths + (size_t)2 * slot * c->path_stride : NULL,
                slot >= 0 ? j->path_len + slot : NULL);
        }
    }
    return NULL;
}

/*
 * Trace n particles in place.  status: 1 absorbed, 2 escaped, 3 still live after
 * max_steps (reference convention, trench_cuda.py:73).  hit[i] = ix*ny+iy of the
 * absorbing cell (or -1).  steps[i] = steps taken.  Optional arrays may be NULL.
 * n_threads host threads share the particles; results do not depend on it.
 */
int oracle_trace(int64_t n, double *x, double *y, double *vx, double *vy, const double *qm,
                 const double *ex, const double *ey, const uint8_t *vac, int nx, int ny,
                 double dx, double cfl, int max_steps, int tapered,
                 const double *phi, const double *wface,
                 const double *rf_ex, const double *rf_ey, const double *rf_phi,
                 const double *wave, int n_phase, double period, double dt_max,
                 double bound_vs, double bound_vm, double *clock, double *elapsed,
                 int record, double *endpoints, const int32_t *slots, double *paths,
                 int32_t *path_len, int path_stride,
                 int8_t *status, int32_t *hit, int32_t *steps, int n_threads) {
    if (n < 0 || nx < 1 || ny < 1) return 1;
    oracle_case c = {ex, ey, vac, phi, wface, rf_ex, rf_ey, rf_phi, wave, n_phase, period,
                     dt_max, bound_vs, bound_vm, nx, ny, dx, cfl, max_steps, tapered, record,
                     path_stride};
    oracle_job job = {&c, n, x, y, vx, vy, clock, elapsed, endpoints, paths, qm, slots,
                      path_len, hit, steps, status, 0};
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 1; t < n_threads; ++t)
        if (pthread_create(&tid[started], NULL, worker, &job) == 0) ++started;
    worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    return 0;
}
