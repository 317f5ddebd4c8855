// Reference-exact FP64 tracer (precision TB_PRECISION_F64).
//
// Compiled with -fmad=false: every product and sum is rounded separately, in the
// operand order of the reference CPU tracer (trench_charging_2d.py:542-702), so a
// particle traced here follows the same FP64 trajectory as the reference.  The
// work distribution is B200-first: a persistent grid of warps whose lanes each
// hold one particle and refill from a global atomic queue the moment their
// particle ends, so no lane idles behind a long electron trajectory and there is
// no host round trip per 256-step chunk (trench_cuda.py:100-117).  Hits are
// deposited on the device with integer atomics instead of a host bincount
// (trench_cuda.py:118-121), so counts are exact and order-independent.  Quotients by
// the cell size and by the RF period, which sit on the step's dependency chain, come
// from the rounded reciprocal and one exact correction (tb_div_by): the same quotient
// as the division in three dependent operations, which is what bounds a small batch of
// long trajectories.
#include "tb_internal.cuh"

namespace {

struct K64 {
    tb_trace_args a;
    int nx, ny;
    double dx;
    double rdx, rperiod;            // RN(1/dx), RN(1/period): quotients by tb_div_by, exact
    const uint8_t *vac;
    unsigned long long *queue;
    int *err;
};

// NumPy float remainder for a positive modulus (trench_charging_2d.py:606).  A value at
// most one period outside [0, b) -- every position after one step and every clock -- is
// wrapped by one exact subtraction (b <= a < 2b: exact by Sterbenz's lemma) or by the same
// rounded addition NumPy makes for a negative remainder; FP64 fmod, an iterative routine,
// is left for the rest.  Results are identical to the general form, including +0 for a
// remainder of zero.
__device__ __forceinline__ double pymod(double a, double b) {
    if (a >= 0.0 && a < b) return a == 0.0 ? 0.0 : a;
    if (a >= b && a < 2.0 * b) {
        const double m = a - b;
        return m == 0.0 ? 0.0 : m;
    }
    if (a < 0.0 && a >= -b) {
        const double m = a + b;
        return m == 0.0 ? 0.0 : m;
    }
    double m = fmod(a, b);
    if (m != 0.0) {
        if ((m < 0.0) != (b < 0.0)) m += b;
    } else {
        m = copysign(0.0, b);
    }
    return m;
}

__device__ __forceinline__ int clipll(int i, int n) {
    return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
}
// i mod n in [0, n); indices at most one period out are wrapped without a division.
// Cell indices are 32-bit, as in the reference kernel (grids hold fewer than 2^31 cells).
__device__ __forceinline__ int pmodll(int i, int n) {
    if (i >= 0 && i < n) return i;
    if (i >= n && i < 2 * n) return i - n;
    if (i < 0 && i >= -n) return i + n;
    int r = i % n;
    return r < 0 ? r + n : r;
}

// Vacuum-weighted bilinear field (trench_charging_2d.py:492-509).
__device__ __forceinline__ void interp(const K64 &k, const double *ex, const double *ey, double x, double y,
                                       double &ox, double &oy) {
    const int nx = k.nx, ny = k.ny;
    double fx = tb_div_by(x, k.dx, k.rdx) - 0.5, fy = tb_div_by(y, k.dx, k.rdx) - 0.5;
    int i0 = (int)floor(fx), j0 = (int)floor(fy);
    double tx = fx - (double)i0, ty = fy - (double)j0;
    int i1 = pmodll(i0 + 1, nx);
    i0 = pmodll(i0, nx);
    int j1 = clipll(j0 + 1, ny);
    j0 = clipll(j0, ny);
    const int c[4] = {i0 * ny + j0, i1 * ny + j0, i0 * ny + j1, i1 * ny + j1};
    const double w[4] = {(1.0 - tx) * (1.0 - ty), tx * (1.0 - ty), (1.0 - tx) * ty, tx * ty};
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double v = (double)__ldg(k.vac + c[q]);
        const double t0 = w[q] * (__ldg(ex + c[q]) * v);
        const double t1 = w[q] * (__ldg(ey + c[q]) * v);
        const double t2 = w[q] * v;
        a0 = q ? a0 + t0 : t0;
        a1 = q ? a1 + t1 : t1;
        a2 = q ? a2 + t2 : t2;
    }
    const double s = a2 > 1e-12 ? a2 : 1e-12;
    ox = a0 / s;
    oy = a1 / s;
}

// First solid face crossed by a move (trench_charging_2d.py:512-539).
__device__ __forceinline__ void wall_entry(const K64 &k, double x0, double y0, double sx, double sy,
                                           int &cx, int &cy, int &vcx, int &vcy,
                                           bool &face_x) {
    const int nx = k.nx, ny = k.ny;
    const double dx = k.dx;
    int ix0 = (int)tb_div_by(x0, dx, k.rdx);
    if (ix0 > nx - 1) ix0 = nx - 1;
    const int iy0 = clipll((int)tb_div_by(y0, dx, k.rdx), ny);
    const double xu = x0 + sx, yu = y0 + sy;
    const int dix = (int)floor(tb_div_by(xu, dx, k.rdx)) - ix0;
    const int diy = clipll((int)floor(tb_div_by(yu, dx, k.rdx)), ny) - iy0;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    const double fx = dix != 0 ? ((double)(ix0 + (dix > 0)) * dx - x0) / sx : inf;
    const double fy = diy != 0 ? ((double)(iy0 + (diy > 0)) * dx - y0) / sy : inf;
    const bool x_first = fx < fy;
    const int ax = x_first ? pmodll(ix0 + dix, nx) : ix0;
    const int ay = x_first ? iy0 : iy0 + diy;
    const bool use_last = dix != 0 && diy != 0 && __ldg(k.vac + ax * ny + ay);
    cx = use_last ? pmodll(ix0 + dix, nx) : ax;
    cy = use_last ? iy0 + diy : ay;
    vcx = use_last ? ax : ix0;
    vcy = use_last ? ay : iy0;
    face_x = use_last ? !x_first : x_first;
}

// Periodic linear interpolation of the electrode voltage deltas (trench_rf.py:5-11).
__device__ __forceinline__ void rf_coeff(const K64 &k, double at, double &vs, double &vm) {
    const double f = tb_div_by(pymod(at, k.a.period), k.a.period, k.rperiod) * (double)k.a.n_phase;
    const int i = pmodll((int)floor(f), k.a.n_phase);
    const int j = pmodll(i + 1, k.a.n_phase);
    const double w = f - floor(f);
    vs = k.a.d_wave[2 * i] * (1.0 - w) + k.a.d_wave[2 * j] * w;
    vm = k.a.d_wave[2 * i + 1] * (1.0 - w) + k.a.d_wave[2 * j + 1] * w;
}

__global__ void __launch_bounds__(256) trace_f64_kernel(const __grid_constant__ K64 k) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const tb_trace_args &a = k.a;
    const int nx = k.nx, ny = k.ny;
    const int cells = nx * ny;
    const double dx = k.dx, Lx = (double)nx * dx, Ly = (double)ny * dx;
    const bool rf = a.n_phase > 0;

    long long pid = -1;
    double x = 0, y = 0, vx = 0, vy = 0, qm = 0, clock = 0, elapsed = 0, xp = 0, yp = 0;
    int steps = 0, stop_at = 0, spc = 0, slot = -1, plen = 0;
    bool open = true;
    unsigned long long my_steps = 0, my_esc_i = 0, my_esc_e = 0, my_lost = 0, my_hit_i = 0, my_hit_e = 0;

    // One step of this lane's particle (trench_charging_2d.py:584-650); on absorption,
    // escape or the step budget the outputs are written and pid becomes -1.
    auto step = [&]() {
        double ex, ey;
        interp(k, a.d_ex, a.d_ey, x, y, ex, ey);
        double ax = qm * ex, ay = qm * ey;
        const double speed = hypot(vx, vy);
        double dt;
        if (!rf) {
            dt = a.cfl * dx / (speed + sqrt(2.0 * dx * hypot(ax, ay)) + 1.0);
        } else {
            double exs, eys, exm, eym;
            interp(k, a.d_rf_ex, a.d_rf_ey, x, y, exs, eys);
            interp(k, a.d_rf_ex + cells, a.d_rf_ey + cells, x, y, exm, eym);
            const double bx = fabs(ex) + (a.bound_vs * fabs(exs) + a.bound_vm * fabs(exm));
            const double by = fabs(ey) + (a.bound_vs * fabs(eys) + a.bound_vm * fabs(eym));
            const double accel = fabs(qm) * hypot(bx, by);
            const double d = a.cfl * dx / (speed + sqrt(2 * dx * accel) + 1);
            dt = a.dt_max < d ? a.dt_max : d;
            double vs, vm;
            rf_coeff(k, clock + dt / 2, vs, vm);
            ex = ex + (vs * exs + vm * exm);
            ey = ey + (vs * eys + vm * eym);
            ax = qm * ex; ay = qm * ey;
            clock = pymod(clock + dt, a.period);
            elapsed = elapsed + dt;
        }
        const double vxn = vx + ax * dt, vyn = vy + ay * dt;
        const double x0 = x, y0 = y;
        const double sx = 0.5 * (vx + vxn) * dt, sy = 0.5 * (vy + vyn) * dt;
        x = pymod(x + sx, Lx);
        y = y + sy;
        vx = vxn; vy = vyn;
        ++steps;
        ++my_steps;

        const bool escaped = y >= Ly;
        int ix = (int)tb_div_by(x, dx, k.rdx);
        if (ix > nx - 1) ix = nx - 1;
        int iy = clipll((int)tb_div_by(y, dx, k.rdx), ny);
        bool hit = !escaped && !__ldg(k.vac + ix * ny + iy);
        int cx = 0, cy = 0, vcx = 0, vcy = 0;
        bool face_x = false;
        if (a.tapered && !hit && !escaped) {
            int ix0 = (int)tb_div_by(x0, dx, k.rdx);
            if (ix0 > nx - 1) ix0 = nx - 1;
            const int iy0 = clipll((int)tb_div_by(y0, dx, k.rdx), ny);
            if (ix != ix0 && iy != iy0) {
                wall_entry(k, x0, y0, sx, sy, cx, cy, vcx, vcy, face_x);
                hit = !__ldg(k.vac + cx * ny + cy);
            }
        }
        if (a.d_phi && hit) {
            wall_entry(k, x0, y0, sx, sy, cx, cy, vcx, vcy, face_x);
            const double vn = face_x ? vx : vy;
            const int cc = cx * ny + cy, vv = vcx * ny + vcy;
            double dphi = a.d_wface[cc] * (a.d_phi[cc] - a.d_phi[vv]);
            if (rf) {
                double vs, vm;
                rf_coeff(k, clock, vs, vm);
                const double d0 = a.d_rf_phi[cc] - a.d_rf_phi[vv];
                const double d1 = a.d_rf_phi[cells + cc] - a.d_rf_phi[cells + vv];
                dphi += a.d_wface[cc] * (vs * d0 + vm * d1);
            }
            if (0.5 * (vn * vn) < qm * dphi) {
                if (face_x) vx = -vx; else vy = -vy;
                x = x0; y = y0;
                hit = false;
            }
            ix = cx; iy = cy;
        }
        if ((a.record || a.tapered) && !a.d_phi && hit) {
            wall_entry(k, x0, y0, sx, sy, cx, cy, vcx, vcy, face_x);
            ix = cx; iy = cy;
        }
        if (a.record) {
            // trench_charging_2d.py:652-685
            double tf = 1.0;
            xp = x; yp = y;
            if (hit) {
                wall_entry(k, x0, y0, sx, sy, cx, cy, vcx, vcy, face_x);
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
            if (rf && (hit || escaped)) {
                clock = pymod(clock - (1 - tf) * dt, a.period);
                elapsed = elapsed - (1 - tf) * dt;
            }
            if (slot >= 0 && plen < a.path_stride) {
                const size_t o = (size_t)2 * ((size_t)slot * a.path_stride + plen);
                a.d_paths[o] = xp;
                a.d_paths[o + 1] = yp;
                ++plen;
            }
        }

        int done = 0;  // 1 absorbed, 2 escaped, 3 budget or step cap reached
        if (hit) {
            const int cell = ix * ny + iy;
            if (cell < 0 || cell >= cells) {
                atomicCAS(k.err, TB_DERR_NONE, TB_DERR_BAD_CELL);
            } else {
                tb_deposit(a.d_counts, (size_t)spc * cells + cell);
            }
            if (a.d_hit) a.d_hit[pid] = (int32_t)cell;
            if (spc == 0) ++my_hit_i; else ++my_hit_e;
            done = 1;
        } else if (escaped) {
            if (spc == 0) ++my_esc_i; else ++my_esc_e;
            done = 2;
        } else if (steps >= stop_at) {
            if (steps >= a.max_steps) ++my_lost;
            done = 3;
        }
        if (done) {
            a.d_steps[pid] = steps;
            if (done != 3) a.d_status[pid] = (int8_t)done;
            if (done == 3 || a.write_state) {
                a.d_x[pid] = x; a.d_y[pid] = y; a.d_vx[pid] = vx; a.d_vy[pid] = vy;
            }
            if (rf) { a.d_clock[2 * pid] = clock; a.d_clock[2 * pid + 1] = elapsed; }
            if (a.record) {
                a.d_endpoints[2 * pid] = xp;
                a.d_endpoints[2 * pid + 1] = yp;
                if (slot >= 0) a.d_path_len[slot] = plen;
            }
            pid = -1;
        }
    };

    for (;;) {
        // Refill empty lanes from the global queue (one atomic per warp).
        const unsigned need = __ballot_sync(FULL, pid < 0);
        if (need != 0u && !open) break;  // queue drained: the lanes finish their particles below
        if (need != 0u) {
            const int leader = __ffs(need) - 1;
            const int cnt = __popc(need);
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(k.queue, (unsigned long long)cnt);
            base = __shfl_sync(FULL, base, leader);
            if (base + (unsigned long long)cnt >= (unsigned long long)a.n) open = false;
            if (pid < 0) {
                const unsigned long long idx = base + __popc(need & ((1u << lane) - 1u));
                if (idx < (unsigned long long)a.n && a.d_status[idx] == 3 && a.d_steps[idx] < a.max_steps) {
                    pid = (long long)idx;
                    x = a.d_x[pid]; y = a.d_y[pid]; vx = a.d_vx[pid]; vy = a.d_vy[pid];
                    qm = a.d_qm[pid];
                    spc = a.d_spc[pid];
                    steps = a.d_steps[pid];
                    stop_at = min(a.max_steps, steps + a.step_budget);
                    if (rf) { clock = a.d_clock[2 * pid]; elapsed = a.d_clock[2 * pid + 1]; }
                    slot = (a.record && a.d_slots) ? a.d_slots[pid] : -1;
                    plen = slot >= 0 ? a.d_path_len[slot] : 0;
                    if (a.record) { xp = a.d_endpoints[2 * pid]; yp = a.d_endpoints[2 * pid + 1]; }
                }
            }
        }
        if (__all_sync(FULL, pid >= 0)) {
            // every lane holds a particle: step them all until one of them ends
            do {
                step();
            } while (__all_sync(FULL, pid >= 0));
        } else if (pid >= 0) {
            step();
        }
    }
    // The queue is drained: each lane runs its particle to the end with no warp-level
    // bookkeeping, so the last, longest trajectories step at the latency of the step
    // itself (a small batch of long trajectories is bound by exactly that).
    while (pid >= 0) step();

    // Warp-reduce the per-lane tallies, one atomic per warp and counter.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        my_steps += __shfl_down_sync(FULL, my_steps, o);
        my_esc_i += __shfl_down_sync(FULL, my_esc_i, o);
        my_esc_e += __shfl_down_sync(FULL, my_esc_e, o);
        my_lost += __shfl_down_sync(FULL, my_lost, o);
        my_hit_i += __shfl_down_sync(FULL, my_hit_i, o);
        my_hit_e += __shfl_down_sync(FULL, my_hit_e, o);
    }
    if (lane == 0) {
        unsigned long long *t = reinterpret_cast<unsigned long long *>(a.d_totals);
        if (my_esc_i) atomicAdd(t + 0, my_esc_i);
        if (my_esc_e) atomicAdd(t + 1, my_esc_e);
        if (my_lost) atomicAdd(t + 2, my_lost);
        if (my_steps) atomicAdd(t + 3, my_steps);
        if (my_hit_i) atomicAdd(t + 4, (unsigned long long)my_hit_i);
        if (my_hit_e) atomicAdd(t + 5, (unsigned long long)my_hit_e);
    }
}

}  // namespace

int tb_launch_trace_f64(tb_ctx *ctx, const tb_trace_args *a, cudaStream_t s) {
    K64 k;
    k.a = *a;
    k.nx = ctx->nx;
    k.ny = ctx->ny;
    k.dx = ctx->dx;
    k.rdx = 1.0 / ctx->dx;
    k.rperiod = a->n_phase > 0 ? 1.0 / a->period : 0.0;
    k.vac = ctx->d_vac;
    k.queue = ctx->d_queue;
    k.err = ctx->d_err;
    TB_CUDA(ctx, cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned long long), s));
    // a batch too small to give every SM a 256-thread CTA is spread over more SMs in
    // 128-thread CTAs (FP64 issue per SM is the limit while the batch is full)
    const int threads = a->n >= (long long)ctx->num_sms * 256 ? 256 : 128;
    long long want = (a->n + threads - 1) / threads;
    long long cap = (long long)ctx->num_sms * 8;
    int blocks = (int)(want < cap ? want : cap);
    if (blocks < 1) blocks = 1;
    trace_f64_kernel<<<blocks, threads, 0, s>>>(k);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}
