// FP32 tracer (precision TB_PRECISION_F32): the throughput path.
//
// Compiled with -prec-div=false -prec-sqrt=false -ftz=true: divisions and square
// roots are the hardware approximations (max 2 ulp), denormals flush to zero (the
// vacuum flag stored in the low bit of a zero field is such a denormal).
// Design (B200-first):
//  * Position = integer cell + FP32 offset in [0,1) cell units, so the cell
//    index, periodic wrap and floor are exact integer operations and the offset
//    keeps 2^-24-cell resolution everywhere in the grid.
//  * Velocities in units of vscale (m/s); time in dx/vscale; the packed field is
//    E*vac*dx/vscale^2 so qm*field is the acceleration in these units.
//  * The packed field (8 bytes per cell, vacuum flag in bit 0 of Ex) is staged
//    once per block into shared memory with a bulk async copy (TMA engine,
//    cp.async.bulk + mbarrier); every bilinear gather is a shared-memory load.
//    Grids too large for shared memory read the same layout from global memory
//    (L2-resident).
//  * Persistent warps, one particle per lane, lanes refill from a global atomic
//    queue as soon as their particle ends (no lane waits for a slow electron); a warp
//    reserves a small block of ranks at a time and prefetches their particles into
//    L1, so most refills wait neither for the atomic nor for the particle's loads.
//  * Claim order (tb_set_claim_order): index, reverse, or learned -- electrons first,
//    then ions longest predicted first from per-bin step means of the previous trace,
//    claimed through FP32 claim records written in that order by a scatter kernel.
//  * Absorbed particles are deposited with integer atomics (bit-exact counts).
//  * The x/y-symmetric arithmetic of a step (half-cell shift, the bilinear sums of
//    (Ex, Ey), acceleration, velocity and position updates, cell remainder) runs on
//    packed FP32 pairs (sm_100 f32x2 add/mul/fma): one instruction per pair, which
//    cuts the issued instructions of this issue-bound loop by about an eighth.
// The step follows the reference algorithm (trench_charging_2d.py:584-650,
// trench_trace.cu:92-148): vacuum-weighted bilinear field, CFL step, trapezoid
// update, periodic x, escape at the top, staircase corner crossing, first-face
// wall entry and the potential-barrier reflection.
#include <algorithm>
#include <vector>

#include "tb_internal.cuh"

namespace {

constexpr int F32_THREADS = 1024;
constexpr float ONE_BELOW = 0x1.fffffep-1f;  // largest float < 1

struct K32 {
    tb_trace_args a;
    int nx, ny;
    double dx, vscale;
    float inv_v;                    // the reference's "+1 m/s" in velocity units
    double inv_dx, inv_v64;         // metres -> cells, m/s -> velocity units
    const tb_fcell *field;          // packed field (global)
    const float4 *barrier;          // per-cell face barrier, potential / vscale^2
    unsigned long long *queue;
    int *err;
    int bytes;                      // packed field bytes (multiple of 16)
    int pool_off;                   // byte offset of the drain pool in dynamic shared memory, -1 = none
    int reverse;                    // claim particles from the last index down
    // learned claim order (nullptr rec = none): claim records in claim order, their number,
    // each particle's key, the ion bins' classes, per-block class starts, per-bin step sums,
    // 1 / domain width and the ordering kernels' blocks
    uint4 *rec;
    unsigned *n_rec;
    uint16_t *okey;
    uint8_t *oclass;
    unsigned *oblk, *oacc;
    double inv_lx;
    int onb;
    // circuit_rf in flight (kernels with RF = true): the unit-voltage basis fields
    // (exs, eys, exm, eym) x vac in field units per padded cell, their per-face wall
    // barriers (substrate basis then mask basis, nx*ny each), the waveform per table
    // interval and the clock units.  The clock is a 32-bit fixed-point fraction of the
    // period: 2^-32 period resolution, and the wrap at the period is the integer wrap.
    const float4 *rf_field;
    const float4 *rf_barrier;
    const float4 *rf_wave;          // (vs_i, vm_i, vs_i+1 - vs_i, vm_i+1 - vm_i), i < n_phase
    float t_clock;                  // clock units (2^-32 period) per unit of step time
    float wave_scale;               // n_phase * 2^-32: clock -> table position
    int n_phase_m1;
    float t_sec;                    // seconds per unit of step time (dx / vscale)
    float dt_max;                   // step bound of the in-flight field, in step time
    float bvs, bvm;                 // largest voltage deltas of the waveform
};

// 1.0f for a vacuum cell, 0.0f for a solid one, with integer operations only
__device__ __forceinline__ float vac_of(const tb_fcell &c) {
    return __uint_as_float((__float_as_uint(c.ex) & 1u) ? 0x3f800000u : 0u);
}

template <bool SMEM>
struct FieldView {
    const tb_fcell *p;
    __device__ __forceinline__ tb_fcell at(int c) const {
        if (SMEM) return p[c];
        const float2 v = __ldg(reinterpret_cast<const float2 *>(p) + c);
        return tb_fcell{v.x, v.y};
    }
    __device__ __forceinline__ bool vac(int c) const {
        float x;
        if (SMEM) x = p[c].ex; else x = __ldg(&p[c].ex);
        return __float_as_uint(x) & 1u;
    }
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bulk-copies `bytes` (multiple of 16) from global to shared memory through the
// async copy engine and waits on an mbarrier with a bounded number of polls.
// Returns false if the copy did not complete within the bound.
__device__ bool stage_field(void *dst, const void *src, int bytes, uint64_t *mbar, bool reuse = false) {
    const uint32_t bar = smem_u32(mbar);
    if (threadIdx.x == 0) {
        if (reuse) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        const int chunk = 32768;
        for (int off = 0; off < bytes; off += chunk) {
            const int sz = bytes - off < chunk ? bytes - off : chunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                ::"r"(smem_u32((char *)dst + off)), "l"((const char *)src + off), "r"(sz), "r"(bar)
                : "memory");
        }
    }
    uint32_t done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
            : "=r"(done) : "r"(bar) : "memory");
        if (!done) __nanosleep(32);
    }
    return __syncthreads_and(done) != 0;
}

// One lane's particle: cell (ix, iy) and FP32 offset (ox, oy) in [0,1) cell units,
// velocity in vscale units; pid < 0 = no particle.
struct LaneState {
    int pid, ix, iy, steps, stop_at, spc;
    float2 o, v;                    // offset (ox, oy) and velocity (vx, vy), packed pairs
    float qm;
    uint32_t clock;                 // circuit_rf: clock in 2^-32 of the period
    float elapsed;                  // circuit_rf: seconds in flight
};

// The four bilinear corners a lane loaded last and their base index (-1 = none).  With
// the field in global memory a step that stays in the same cell quad reuses them: a
// move is under half a cell at the usual CFL, so about half the steps skip the gathers.
struct QuadCache {
    int base;
    tb_fcell c00, c01, c10, c11;
};

// Per-lane event counts, reduced over the warp at the end.
struct LaneTally {
    unsigned steps, esc_i, esc_e, lost, hit_i, hit_e;
};

// Loop-invariant parameters of one case.
template <bool SMEM>
struct CaseView {
    FieldView<SMEM> F;
    int nx, ny, cells, P;
    float inv_v, cfl;
    bool barrier, tapered, first_face;
    bool small_steps;   // cfl < 1/2: a step ends in a corner cell of its start quad
};

// One step of one particle (trench_charging_2d.py:584-650): vacuum-weighted bilinear
// field, CFL step, trapezoid update, periodic x, escape, staircase corner, first-face
// wall entry and barrier reflection; on absorption, escape or the step cap the
// particle's outputs are written and s.pid becomes -1.
// Waveform table position of a clock: interval i and the position within it
// (trench_rf.py:5-11: periodic linear interpolation of n_phase samples; the last
// interval runs to the first sample).
__device__ __forceinline__ int rf_interval(const K32 &k, uint32_t clock, float &w) {
    const float f = (float)clock * k.wave_scale;
    const int i = min((int)f, k.n_phase_m1);  // a clock just below 2^32 may round up to n
    w = f - (float)i;
    return i;
}

// Voltage deltas (substrate, mask) of the waveform at a clock.
__device__ __forceinline__ void rf_voltages(const K32 &k, uint32_t clock, float &vs, float &vm) {
    float w;
    const float4 e = __ldg(k.rf_wave + rf_interval(k, clock, w));
    vs = fmaf(w, e.z, e.x);
    vm = fmaf(w, e.w, e.y);
}

template <bool SMEM, bool RF>
__device__ __forceinline__ void step_particle(const K32 &k, const CaseView<SMEM> &C, LaneState &s, LaneTally &t,
                                              QuadCache &q) {
    const tb_trace_args &a = k.a;
    const int nx = C.nx, ny = C.ny, P = C.P;
    // ---- vacuum-weighted bilinear field (trench_charging_2d.py:492-509) ----
    // corners (i0, j0) = (ix - 1 + hx, iy - 1 + hy) .. (i0 + 1, j0 + 1); in the halo-padded
    // field i0 + 1 = ix + hx needs no wrap and the clipped rows need one clamp
    const int hx = s.o.x >= 0.5f ? 1 : 0, hy = s.o.y >= 0.5f ? 1 : 0;
    const float2 tq = __fadd2_rn(s.o, make_float2(hx ? -0.5f : 0.5f, hy ? -0.5f : 0.5f));
    const float tx = tq.x, ty = tq.y;
    const int base = (s.ix + hx) * P + max(s.iy + hy, 0);
    tb_fcell c00, c01, c10, c11;
    if (SMEM) {
        c00 = C.F.at(base); c01 = C.F.at(base + 1);
        c10 = C.F.at(base + P); c11 = C.F.at(base + P + 1);
    } else {
        if (base != q.base) {
            q.c00 = C.F.at(base); q.c01 = C.F.at(base + 1);
            q.c10 = C.F.at(base + P); q.c11 = C.F.at(base + P + 1);
            q.base = base;
        }
        c00 = q.c00; c01 = q.c01; c10 = q.c10; c11 = q.c11;
    }
    // A step moves at most cfl cells (|v| dt + |a| dt^2 / 2 <= cfl for the CFL dt), so with
    // cfl below one half a step that starts inside this quad of cell centres ends in one of
    // its four corner cells.  The quad flag (bit 0 of the lower-left corner's ey) says all
    // four are vacuum: then the step cannot reach a wall and the vacuum weights sum to one,
    // and both the normalisation and the end-cell checks are skipped.
    const bool near = !(C.small_steps && (__float_as_uint(c00.ey) & 1u));
    // bilinear sum of the (vacuum-premultiplied) field with (ex, ey) as one packed pair:
    // along y in both columns, then along x
    const float2 M1 = make_float2(-1.f, -1.f);
    const float2 tyy = make_float2(ty, ty), txx = make_float2(tx, tx);
    const float2 f00 = make_float2(c00.ex, c00.ey), f01 = make_float2(c01.ex, c01.ey);
    const float2 f10 = make_float2(c10.ex, c10.ey), f11 = make_float2(c11.ex, c11.ey);
    const float2 e0 = __ffma2_rn(tyy, __ffma2_rn(f00, M1, f01), f00);
    const float2 e1 = __ffma2_rn(tyy, __ffma2_rn(f10, M1, f11), f10);
    const float2 E = __ffma2_rn(txx, __ffma2_rn(e0, M1, e1), e0);
    const float sex = E.x, sey = E.y;
    float inv_sw = 1.f;
    if (near) {
        const float v00 = vac_of(c00), v01 = vac_of(c01), v10 = vac_of(c10), v11 = vac_of(c11);
        const float s0 = fmaf(ty, v01 - v00, v00), s1 = fmaf(ty, v11 - v10, v10);
        inv_sw = __fdividef(1.f, fmaxf(fmaf(tx, s1 - s0, s0), 1e-12f));
    }
    float2 A;
    float dt;
    const float speed = sqrtf(fmaf(s.v.x, s.v.x, s.v.y * s.v.y));
    if (!RF) {
        const float qs = s.qm * inv_sw;
        A = __fmul2_rn(make_float2(qs, qs), E);
        const float acc = sqrtf(fmaf(A.x, A.x, A.y * A.y));
        dt = __fdividef(C.cfl, speed + sqrtf(2.f * acc) + C.inv_v);
    } else {
        const float ux = 1.f - tx, uy = 1.f - ty;
        const float w00 = ux * uy, w10 = tx * uy, w01 = ux * ty, w11 = tx * ty;
        // in-flight RF field (trench_trace.cu:97-110): the basis fields at the same corners
        // and weights bound the step, and the field is taken at the mid-step clock.  The
        // waveform interval of the start clock is loaded before the step is known: a
        // CFL-limited step is far shorter than an interval, so the mid-step clock is
        // nearly always in it and the lookup leaves the step's dependency chain.
        const uint32_t c0 = s.clock;
        float w0;
        const int i0 = rf_interval(k, c0, w0);
        const float4 e0 = __ldg(k.rf_wave + i0);
        const float4 b00 = __ldg(k.rf_field + base), b01 = __ldg(k.rf_field + base + 1);
        const float4 b10 = __ldg(k.rf_field + base + P), b11 = __ldg(k.rf_field + base + P + 1);
        // weighted sums like the field's; the vacuum normalisation 1/sw is applied once
        const float sxs = w00 * b00.x + w10 * b10.x + w01 * b01.x + w11 * b11.x;
        const float sys = w00 * b00.y + w10 * b10.y + w01 * b01.y + w11 * b11.y;
        const float sxm = w00 * b00.z + w10 * b10.z + w01 * b01.z + w11 * b11.z;
        const float sym = w00 * b00.w + w10 * b10.w + w01 * b01.w + w11 * b11.w;
        const float bx = fabsf(sex) + (k.bvs * fabsf(sxs) + k.bvm * fabsf(sxm));
        const float by = fabsf(sey) + (k.bvs * fabsf(sys) + k.bvm * fabsf(sym));
        const float accel = fabsf(s.qm) * inv_sw * sqrtf(bx * bx + by * by);
        dt = fminf(k.dt_max, __fdividef(C.cfl, speed + sqrtf(2.f * accel) + C.inv_v));
        const unsigned long long inc = __float2ull_rn(dt * k.t_clock);
        const uint32_t mid = c0 + (uint32_t)(inc >> 1);
        float w;
        const int im = rf_interval(k, mid, w);
        const float4 e = im == i0 ? e0 : __ldg(k.rf_wave + im);
        const float vs = fmaf(w, e.z, e.x), vm = fmaf(w, e.w, e.y);
        const float qs = s.qm * inv_sw;
        A = make_float2(qs * (sex + (vs * sxs + vm * sxm)), qs * (sey + (vs * sys + vm * sym)));
        s.clock = c0 + (uint32_t)inc;
        s.elapsed += dt * k.t_sec;
    }

    // ---- CFL step and trapezoid update (trench_charging_2d.py:587-608) ----
    // v' = v + a dt and the move (v + v') dt / 2 = (v + a dt / 2) dt, each a packed pair.
    // A step moves less than one cell, so the new offset lies in (-1, 2): the cell change
    // is its floor (-1, 0 or 1) and the new offset the remainder (exact for the shift by
    // 1; a remainder that rounds up to 1 is clamped below 1)
    const float2 dtt = make_float2(dt, dt);
    const float hdt = 0.5f * dt;
    const float2 vn = __ffma2_rn(A, dtt, s.v);
    const float2 S = __fmul2_rn(__ffma2_rn(A, make_float2(hdt, hdt), s.v), dtt);
    const float vxn = vn.x, vyn = vn.y, sx = S.x, sy = S.y;
    const float2 pos = __fadd2_rn(s.o, S);
    const float fnx = floorf(pos.x), fny = floorf(pos.y);
    const int dix = (int)fnx, diy = (int)fny;
    const float2 rem = __ffma2_rn(make_float2(fnx, fny), M1, pos);
    const float nox = fminf(rem.x, ONE_BELOW), noy = fminf(rem.y, ONE_BELOW);
    int nix = s.ix + dix;
    nix = nix < 0 ? nx - 1 : (nix >= nx ? 0 : nix);
    const int niy = s.iy + diy;
    ++s.steps;
    const bool escaped = niy >= ny;
    bool hit_end = false, corner = false;
    if (near && !escaped) {
        hit_end = !C.F.vac((nix + 1) * P + max(niy, -1) + 1);
        // both the column and the (clipped) row changed: a staircase corner may lie on
        // the path between two vacuum cells (trench_charging_2d.py:614-621).  The move
        // reaches the wall only if the cell beyond the first boundary crossed is solid
        // (the first-face rule of the rare path below, same expressions), so that is
        // decided here and the rare path runs only for an actual corner contact.
        corner = C.tapered && !hit_end && dix != 0 && max(niy, 0) != max(s.iy, 0);
        if (corner) {
            const int y0c = min(max(s.iy, 0), ny - 1);
            const int iyn = min(max(niy, 0), ny - 1);
            const float fx = ((dix > 0 ? 1.f : 0.f) - s.o.x) / sx;
            const float fy = ((iyn > y0c ? 1.f : 0.f) - s.o.y) / sy;
            const bool x_first = fx < fy;
            corner = !C.F.vac((x_first ? nix + 1 : s.ix + 1) * P + (x_first ? y0c : iyn) + 1);
        }
    }

    if (!(hit_end || corner || escaped || s.steps >= s.stop_at)) {
        s.ix = nix; s.iy = niy; s.o = make_float2(nox, noy); s.v = vn;
        return;
    }

    // ---- rare path: wall contact, escape, or step cap ----
    const int y0c = min(max(s.iy, 0), ny - 1);
    const int iyn = min(max(niy, 0), ny - 1);
    const int diy_e = iyn - y0c;     // rows clipped like the reference
    bool hit = hit_end;
    int dcell = nix * ny + iyn;
    bool reflected = false;
    if (hit ? C.first_face : corner) {
        // first solid face crossed (trench_charging_2d.py:512-539) in cell units
        const float inf = __int_as_float(0x7f800000);
        const float fx = dix != 0 ? ((dix > 0 ? 1.f : 0.f) - s.o.x) / sx : inf;
        const float fy = diy_e != 0 ? ((diy_e > 0 ? 1.f : 0.f) - s.o.y) / sy : inf;
        const bool x_first = fx < fy;
        const int ax_ = x_first ? nix : s.ix, ay_ = x_first ? y0c : y0c + diy_e;
        const bool use_last = dix != 0 && diy_e != 0 && C.F.vac((ax_ + 1) * P + ay_ + 1);
        const int cx = use_last ? nix : ax_, cy = use_last ? y0c + diy_e : ay_;
        const bool face_x = use_last ? !x_first : x_first;
        const int ccell = cx * ny + cy;
        hit = !C.F.vac((cx + 1) * P + cy + 1);
        dcell = ccell;
        if (hit && C.barrier) {
            const float4 b = __ldg(k.barrier + ccell);
            // neighbour the particle came from: W/E across an x face, S/N across a y face
            float dphi = face_x ? (dix > 0 ? b.x : b.y) : (diy_e > 0 ? b.z : b.w);
            if (RF) {
                // barrier of the instantaneous potential at the clock after the step
                // (trench_trace.cu:131-136)
                float vs, vm;
                rf_voltages(k, s.clock, vs, vm);
                const float4 bs = __ldg(k.rf_barrier + ccell), bm = __ldg(k.rf_barrier + C.cells + ccell);
                const float ds = face_x ? (dix > 0 ? bs.x : bs.y) : (diy_e > 0 ? bs.z : bs.w);
                const float dm = face_x ? (dix > 0 ? bm.x : bm.y) : (diy_e > 0 ? bm.z : bm.w);
                dphi += vs * ds + vm * dm;
            }
            const float vn = face_x ? vxn : vyn;
            if (0.5f * vn * vn < s.qm * dphi) {
                // reflect: the normal velocity flips, the position stays at the start point
                s.v.x = face_x ? -vxn : vxn;
                s.v.y = face_x ? vyn : -vyn;
                hit = false;
                reflected = true;
            }
        }
    }
    if (!reflected) { s.ix = nix; s.iy = niy; s.o = make_float2(nox, noy); s.v = vn; }

    int done = 0;
    if (hit) {
        if (dcell < 0 || dcell >= C.cells) {
            atomicCAS(k.err, TB_DERR_NONE, TB_DERR_BAD_CELL);
        } else {
            tb_deposit(a.d_counts, (size_t)s.spc * C.cells + dcell);
        }
        if (a.d_hit) a.d_hit[s.pid] = dcell;
        if (s.spc == 0) ++t.hit_i; else ++t.hit_e;
        done = 1;
    } else if (escaped && !reflected) {
        if (s.spc == 0) ++t.esc_i; else ++t.esc_e;
        done = 2;
    } else if (s.steps >= s.stop_at) {
        if (s.steps >= a.max_steps) ++t.lost;
        done = 3;
    }
    if (done) {
        const int pid = s.pid;
        t.steps += (unsigned)s.steps;   // the claim subtracted the particle's earlier steps
        a.d_steps[pid] = s.steps;
        if (done != 3) a.d_status[pid] = (int8_t)done;
        if (done == 3 || a.write_state) {
            a.d_x[pid] = ((double)s.ix + (double)s.o.x) * k.dx;
            a.d_y[pid] = ((double)s.iy + (double)s.o.y) * k.dx;
            a.d_vx[pid] = (double)s.v.x * k.vscale;
            a.d_vy[pid] = (double)s.v.y * k.vscale;
        }
        if (RF) {
            a.d_clock[2 * pid] = (double)s.clock * 0x1p-32 * a.period;
            a.d_clock[2 * pid + 1] = (double)s.elapsed;
        }
        s.pid = -1;
    }
}

// Shared-memory pool of particle states for the drain of a case: 9 words per lane
// (struct of arrays over the block's threads): pid; ix | iy << 16 (grids below 32768
// cells a side, iy >= -1); steps; stop_at | spc << 31; ox, oy, vx, vy, qm.
constexpr int POOL_WORDS = 9;
constexpr int POOL_WORDS_RF = 11;   // + phase, elapsed
#ifndef TB_TAIL_ROUND_STEPS
#define TB_TAIL_ROUND_STEPS 64
#endif
constexpr int TAIL_ROUND_STEPS = TB_TAIL_ROUND_STEPS;

template <bool RF>
__device__ __forceinline__ void pool_put(uint32_t *P, int T, int q, const LaneState &s) {
    P[0 * T + q] = (uint32_t)s.pid;
    P[1 * T + q] = ((uint32_t)s.ix & 0xffffu) | ((uint32_t)s.iy << 16);
    P[2 * T + q] = (uint32_t)s.steps;
    P[3 * T + q] = (uint32_t)s.stop_at | ((uint32_t)s.spc << 31);
    P[4 * T + q] = __float_as_uint(s.o.x);
    P[5 * T + q] = __float_as_uint(s.o.y);
    P[6 * T + q] = __float_as_uint(s.v.x);
    P[7 * T + q] = __float_as_uint(s.v.y);
    P[8 * T + q] = __float_as_uint(s.qm);
    if (RF) {
        P[9 * T + q] = s.clock;
        P[10 * T + q] = __float_as_uint(s.elapsed);
    }
}

template <bool RF>
__device__ __forceinline__ void pool_get(const uint32_t *P, int T, int q, LaneState &s) {
    s.pid = (int)P[0 * T + q];
    const uint32_t xy = P[1 * T + q];
    s.ix = (int)(xy & 0xffffu);
    s.iy = (int)xy >> 16;  // arithmetic shift keeps iy = -1
    s.steps = (int)P[2 * T + q];
    const uint32_t w = P[3 * T + q];
    s.stop_at = (int)(w & 0x7fffffffu);
    s.spc = (int)(w >> 31);
    s.o.x = __uint_as_float(P[4 * T + q]);
    s.o.y = __uint_as_float(P[5 * T + q]);
    s.v.x = __uint_as_float(P[6 * T + q]);
    s.v.y = __uint_as_float(P[7 * T + q]);
    s.qm = __uint_as_float(P[8 * T + q]);
    if (RF) {
        s.clock = P[9 * T + q];
        s.elapsed = __uint_as_float(P[10 * T + q]);
    }
}

// Traces particles of one case with the calling block until the case's queue is
// drained and every particle has ended, then adds the warps' tallies to the case's
// totals.  `fieldp` is the packed field in shared or global memory.  Every thread of
// the block calls it.
//
// Main phase: each lane takes a particle from the case's global queue whenever its
// particle ends.  Drain: once the queue is empty a warp keeps only the lanes whose
// particles are still in flight, so with independent warps the block would issue
// nearly full instruction streams for a few live lanes each until the longest
// particle ends.  With a shared-memory pool (pool != nullptr) the block instead runs
// rounds: the live particles are packed into the first warps, those warps take up
// to TAIL_ROUND_STEPS steps, and the rest wait at the barrier.  A particle's
// arithmetic does not depend on its lane, so the results are the same either way.
template <bool SMEM, bool RF, bool REC = false>
__device__ __forceinline__ void run_case(const K32 &k, const tb_fcell *fieldp, uint32_t *pool) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const tb_trace_args &a = k.a;
    unsigned long long *const queue = k.queue;

    CaseView<SMEM> C;
    C.F.p = fieldp;
    C.nx = k.nx;
    C.ny = k.ny;
    C.cells = k.nx * k.ny;
    C.P = k.ny + 2;  // padded column stride
    C.inv_v = k.inv_v;
    C.cfl = (float)a.cfl;
    C.barrier = a.d_phi != nullptr;
    C.tapered = a.tapered != 0;
    C.first_face = C.barrier || C.tapered;
    C.small_steps = a.cfl <= 0.45;

    LaneState s;
    s.pid = -1;
    s.ix = s.iy = s.steps = s.stop_at = s.spc = 0;
    s.o.x = s.o.y = s.v.x = s.v.y = s.qm = 0.f;
    s.clock = 0u;
    s.elapsed = 0.f;
    LaneTally t = {0u, 0u, 0u, 0u, 0u, 0u};
    QuadCache q;
    q.base = -1;
    q.c00 = q.c01 = q.c10 = q.c11 = tb_fcell{0.f, 0.f};
    bool open = true;
    // The warp's reserved block of claim ranks [wc, we): empty lanes are refilled from it
    // without an atomic, and a new block is reserved only when it runs short.  While the
    // queue is long a block keeps up to one rank per lane beyond the lanes being served
    // (guided: the reserve shrinks with the work left, so little is held back from other
    // warps at the end), and the particle data of the kept ranks is prefetched into L1, so
    // a refill waits neither for the queue atomic nor for the particle's loads.
    unsigned long long wc = 0, we = 0;
    const unsigned long long n_all = REC ? (unsigned long long)*k.n_rec : (unsigned long long)a.n;
    const unsigned long long warps_all = (unsigned long long)gridDim.x * (blockDim.x >> 5);

    for (;;) {
        unsigned need = __ballot_sync(FULL, s.pid < 0);
        if (need != 0u) {
            if (!open && wc >= we) {
                if (pool != nullptr || need == FULL) break;
            } else {
                const unsigned cnt = __popc(need);
                const unsigned long long avail = we - wc;
                const bool reserve = avail < cnt && open;
                unsigned long long nb = 0, nwc = wc + (avail < cnt ? avail : cnt), nwe = we;
                if (reserve) {
                    const unsigned long long left = n_all > we ? n_all - we : 0ULL;
                    const unsigned long long extra = min(32ULL, left / (4ULL * warps_all));
                    const unsigned long long size = (cnt - avail) + extra;
                    const int leader = __ffs(need) - 1;
                    if (lane == leader) nb = atomicAdd(queue, size);
                    nb = __shfl_sync(FULL, nb, leader);
                    if (nb + size >= n_all) open = false;
                    nwc = nb + (cnt - avail);
                    nwe = nb + size;
                    // prefetch the particle data of the ranks kept for later refills
                    if (REC) {
                        // four 32-byte records to a 128-byte line
                        const unsigned long long r = nwc + 4ULL * (unsigned)lane;
                        if (r < nwe && r < n_all) asm volatile("prefetch.global.L1 [%0];" ::"l"(k.rec + 2 * r));
                    }
                    const unsigned long long r = nwc + 8ULL * (unsigned)lane;
                    if (!REC && r < nwe && r < n_all) {
                        const unsigned long long i = k.reverse ? n_all - 1 - r : r;
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_x + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_y + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_vx + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_vy + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_qm + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_steps + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_status + i));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_spc + i));
                        if (RF) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.d_clock + 2 * i));
                    }
                }
                if (s.pid < 0) {
                    // the j-th empty lane takes the block's next rank, then the reservation's
                    const unsigned j = __popc(need & ((1u << lane) - 1u));
                    const unsigned long long rank = j < avail ? wc + j : (reserve ? nb + (j - avail) : n_all);
                    if (REC && rank < n_all) {
                        // learned order: the record holds the particle's FP32 start state,
                        // converted by the scatter with the expressions below
                        const uint4 r0 = __ldg(k.rec + 2 * rank), r1 = __ldg(k.rec + 2 * rank + 1);
                        s.pid = (int)r0.x;
                        q.base = -1;
                        s.ix = (int)(r0.y & 0xffffu);
                        s.iy = (int)r0.y >> 16;  // arithmetic shift keeps a negative row
                        s.o = make_float2(__uint_as_float(r0.z), __uint_as_float(r0.w));
                        s.v = make_float2(__uint_as_float(r1.x), __uint_as_float(r1.y));
                        s.qm = __uint_as_float(r1.z);
                        s.spc = (int)(r1.w >> 31);
                        s.steps = (int)(r1.w & 0x7fffffffu);
                        s.stop_at = min(a.max_steps, s.steps + a.step_budget);
                        t.steps -= (unsigned)s.steps;
                    }
                    // claim order: index order, or from the last index down (k.reverse)
                    const unsigned long long idx = (k.reverse && rank < n_all) ? n_all - 1 - rank : rank;
                    if (!REC && idx < n_all && a.d_status[idx] == 3 && a.d_steps[idx] < a.max_steps) {
                        const int pid = (int)idx;
                        s.pid = pid;
                        q.base = -1;
                        // metres -> cells: x lies in cell min(int(x/dx), nx-1) as in the
                        // reference (trench_charging_2d.py:611)
                        const double xc = a.d_x[pid] * k.inv_dx, yc = a.d_y[pid] * k.inv_dx;
                        s.ix = min(max((int)xc, 0), C.nx - 1);
                        s.iy = min((int)floor(yc), C.ny - 1);  // a start above the grid escapes at once
                        s.o.x = fminf(fmaxf((float)(xc - (double)s.ix), 0.f), ONE_BELOW);
                        s.o.y = fminf(fmaxf((float)(yc - (double)s.iy), 0.f), ONE_BELOW);
                        s.v.x = (float)(a.d_vx[pid] * k.inv_v64);
                        s.v.y = (float)(a.d_vy[pid] * k.inv_v64);
                        s.qm = (float)a.d_qm[pid];
                        s.spc = a.d_spc[pid];
                        s.steps = a.d_steps[pid];
                        s.stop_at = min(a.max_steps, s.steps + a.step_budget);
                        t.steps -= (unsigned)s.steps;   // steps are tallied when the particle stops
                        if (RF) {
                            // clock in [0, period) seconds -> 2^-32 of the period
                            const double c = a.d_clock[2 * pid] / a.period * 4294967296.0 + 0.5;
                            s.clock = (uint32_t)(unsigned long long)fmin(fmax(c, 0.0), 4294967295.0);
                            s.elapsed = (float)a.d_clock[2 * pid + 1];
                        }
                    }
                }
                wc = nwc;
                we = nwe;
            }
            need = __ballot_sync(FULL, s.pid < 0);
        }
        if (need == 0u) {
            // every lane holds a particle: step them all until one of them ends, one vote
            // per step instead of the refill bookkeeping
            do {
                step_particle<SMEM, RF>(k, C, s, t, q);
            } while (__all_sync(FULL, s.pid >= 0));
        } else if (s.pid >= 0) {
            step_particle<SMEM, RF>(k, C, s, t, q);
        }
    }

    if (pool != nullptr) {
        __shared__ int s_live;
        const int T = blockDim.x;
        if (threadIdx.x == 0) s_live = 0;
        for (;;) {
            __syncthreads();
            if (s.pid >= 0) {
                pool_put<RF>(pool, T, atomicAdd(&s_live, 1), s);
                s.pid = -1;
            }
            __syncthreads();
            const int live = s_live;
            if (live == 0) break;
            if ((int)threadIdx.x < live) pool_get<RF>(pool, T, threadIdx.x, s);
            q.base = -1;
            __syncthreads();
            if (threadIdx.x == 0) s_live = 0;
            if ((int)(threadIdx.x & ~31u) < live) {  // warp-uniform: this warp holds particles
                for (int r = 0; r < TAIL_ROUND_STEPS; ++r) {
                    if (__ballot_sync(FULL, s.pid >= 0) == 0u) break;
                    if (s.pid >= 0) step_particle<SMEM, RF>(k, C, s, t, q);
                }
            }
        }
    }

#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t.steps += __shfl_down_sync(FULL, t.steps, o);
        t.esc_i += __shfl_down_sync(FULL, t.esc_i, o);
        t.esc_e += __shfl_down_sync(FULL, t.esc_e, o);
        t.lost += __shfl_down_sync(FULL, t.lost, o);
        t.hit_i += __shfl_down_sync(FULL, t.hit_i, o);
        t.hit_e += __shfl_down_sync(FULL, t.hit_e, o);
    }
    if (lane == 0) {
        unsigned long long *tot = reinterpret_cast<unsigned long long *>(a.d_totals);
        if (t.esc_i) atomicAdd(tot + 0, (unsigned long long)t.esc_i);
        if (t.esc_e) atomicAdd(tot + 1, (unsigned long long)t.esc_e);
        if (t.lost) atomicAdd(tot + 2, (unsigned long long)t.lost);
        if (t.steps) atomicAdd(tot + 3, (unsigned long long)t.steps);
        if (t.hit_i) atomicAdd(tot + 4, (unsigned long long)t.hit_i);
        if (t.hit_e) atomicAdd(tot + 5, (unsigned long long)t.hit_e);
    }
}

template <bool SMEM, int THREADS, bool RF, bool REC = false>
__global__ void __launch_bounds__(THREADS, 1) trace_f32_kernel(const __grid_constant__ K32 k) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    const tb_fcell *fieldp = k.field;
    if (SMEM) {
        if (!stage_field(smem_raw, k.field, k.bytes, &mbar)) {
            if (threadIdx.x == 0) atomicCAS(k.err, TB_DERR_NONE, TB_DERR_BULK_TIMEOUT);
            return;
        }
        fieldp = reinterpret_cast<const tb_fcell *>(smem_raw);
    }
    uint32_t *pool = k.pool_off >= 0 ? reinterpret_cast<uint32_t *>(smem_raw + k.pool_off) : nullptr;
    run_case<SMEM, RF, REC>(k, fieldp, pool);
}

// Many cases in one persistent launch: each CTA repeatedly takes the case with the
// most particles left in its queue, stages that case's field into shared memory and
// traces from the case's queue; CTAs meet on large cases and spread over small ones.
template <bool SMEM>
__global__ void __launch_bounds__(F32_THREADS, 1)
    trace_f32_batch_kernel(const K32 *__restrict__ cases, int n_cases, int *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int s_case;
    bool staged = false;
    for (;;) {
        if (threadIdx.x < 32) {
            // warp 0: the case with the most unclaimed particles
            long long best_rem = 0;
            int best = -1;
            for (int c = threadIdx.x; c < n_cases; c += 32) {
                const unsigned long long q = *reinterpret_cast<volatile const unsigned long long *>(cases[c].queue);
                // a case in the learned order queues only its traced particles (its records)
                const long long lim = cases[c].rec ? (long long)*cases[c].n_rec : cases[c].a.n;
                const long long rem = lim - (long long)q;
                if (rem > best_rem) { best_rem = rem; best = c; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const long long r2 = __shfl_down_sync(0xffffffffu, best_rem, o);
                const int b2 = __shfl_down_sync(0xffffffffu, best, o);
                if (r2 > best_rem || (r2 == best_rem && b2 >= 0 && (best < 0 || b2 < best))) {
                    best_rem = r2;
                    best = b2;
                }
            }
            if (threadIdx.x == 0) s_case = best;
        }
        __syncthreads();
        const int c = s_case;
        if (c < 0) return;
        const K32 &k = cases[c];
        const tb_fcell *fieldp = k.field;
        if (SMEM) {
            if (!stage_field(smem_raw, k.field, k.bytes, &mbar, staged)) {
                if (threadIdx.x == 0) atomicCAS(err, TB_DERR_NONE, TB_DERR_BULK_TIMEOUT);
                return;
            }
            staged = true;
            fieldp = reinterpret_cast<const tb_fcell *>(smem_raw);
        }
        uint32_t *pool = k.pool_off >= 0 ? reinterpret_cast<uint32_t *>(smem_raw + k.pool_off) : nullptr;
        if (k.a.n_phase > 0) run_case<SMEM, true>(k, fieldp, pool);  // block-uniform: one case per CTA
        else if (SMEM && k.rec) run_case<SMEM, false, SMEM>(k, fieldp, pool);
        else run_case<SMEM, false>(k, fieldp, pool);
        __syncthreads();  // every warp is done with this case's field
    }
}

// Packs FP64 fields into the halo-padded FP32 tracer layout; one thread per cell.
__global__ void pack_fields_kernel(int nx, int ny, double scale_e, double scale_phi, const uint8_t *vac,
                                   const double *ex, const double *ey, const double *phi,
                                   const double *wface, tb_fcell *out, float4 *bar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = nx * ny;
    if (c >= cells) return;
    const int ix = c / ny, iy = c - ix * ny;
    const int v = vac[c] ? 1 : 0;
    tb_store_packed(out, vac, nx, ny, ix, iy, tb_pack_cell(ex[c], ey[c], v, scale_e));
    float4 b = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!v && phi != nullptr) {
        const int w = (ix == 0 ? nx - 1 : ix - 1) * ny + iy;
        const int e = (ix == nx - 1 ? 0 : ix + 1) * ny + iy;
        const double f = wface[c], pc = phi[c];
        b.x = (float)(f * (pc - phi[w]) * scale_phi);
        b.y = (float)(f * (pc - phi[e]) * scale_phi);
        b.z = iy > 0 ? (float)(f * (pc - phi[c - 1]) * scale_phi) : 0.f;
        b.w = iy < ny - 1 ? (float)(f * (pc - phi[c + 1]) * scale_phi) : 0.f;
    }
    bar[c] = b;
}

// Packs the waveform ((n, 2) voltage deltas per phase sample) into one float4 per
// table interval: the samples at its start and the differences to the next sample
// (the last interval runs to the first).
__global__ void pack_wave_kernel(const double *wave, int n, float4 *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = i + 1 == n ? 0 : i + 1;
    out[i] = make_float4((float)wave[2 * i], (float)wave[2 * i + 1], (float)(wave[2 * j] - wave[2 * i]),
                         (float)(wave[2 * j + 1] - wave[2 * i + 1]));
}

// Packs the circuit_rf unit-voltage basis fields ((2, nx, ny) each: substrate, mask)
// into one float4 per halo-padded cell, (exs, eys, exm, eym) x vac x scale_e, and the
// per-face barriers of the two basis potentials like pack_fields_kernel.
__global__ void pack_rf_fields_kernel(int nx, int ny, double scale_e, double scale_phi, const uint8_t *vac,
                                      const double *ex, const double *ey, const double *phi, const double *wface,
                                      float4 *out, float4 *bar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = nx * ny;
    if (c >= cells) return;
    const int ix = c / ny, iy = c - ix * ny;
    const double v = vac[c] ? scale_e : 0.0;
    tb_store_halo(out, nx, ny, ix, iy,
                  make_float4((float)(ex[c] * v), (float)(ey[c] * v), (float)(ex[cells + c] * v),
                              (float)(ey[cells + c] * v)));
    for (int b = 0; b < 2; ++b) {
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!vac[c] && wface != nullptr) {
            const double *ph = phi + (size_t)b * cells;
            const int w = (ix == 0 ? nx - 1 : ix - 1) * ny + iy;
            const int e = (ix == nx - 1 ? 0 : ix + 1) * ny + iy;
            const double f = wface[c], pc = ph[c];
            r.x = (float)(f * (pc - ph[w]) * scale_phi);
            r.y = (float)(f * (pc - ph[e]) * scale_phi);
            r.z = iy > 0 ? (float)(f * (pc - ph[c - 1]) * scale_phi) : 0.f;
            r.w = iy < ny - 1 ? (float)(f * (pc - ph[c + 1]) * scale_phi) : 0.f;
        }
        bar[(size_t)b * cells + c] = r;
    }
}

}  // namespace

int tb_launch_pack_rf_fields(tb_ctx *ctx, const double *rf_ex, const double *rf_ey, const double *rf_phi,
                             const double *wface, const double *wave, int n_phase, cudaStream_t s) {
    const int cells = ctx->nx * ctx->ny;
    const double vscale = ctx->vscale;
    const int threads = 256;
    pack_rf_fields_kernel<<<(cells + threads - 1) / threads, threads, 0, s>>>(
        ctx->nx, ctx->ny, ctx->dx / (vscale * vscale), 1.0 / (vscale * vscale), ctx->d_vac, rf_ex, rf_ey, rf_phi,
        wface, ctx->d_rf_field, ctx->d_rf_barrier);
    pack_wave_kernel<<<(n_phase + threads - 1) / threads, threads, 0, s>>>(wave, n_phase, ctx->d_rf_wave);
    TB_CUDA(ctx, cudaGetLastError());
    ctx->rf_wave_src = wave;
    ctx->rf_n_phase = n_phase;
    ctx->rf_vscale = vscale;
    ctx->rf_ready = 1;
    return TB_OK;
}

int tb_launch_pack_fields(tb_ctx *ctx, const double *ex, const double *ey, const double *phi,
                          const double *wface, double vscale, cudaStream_t s) {
    const int cells = ctx->nx * ctx->ny;
    const double scale_e = ctx->dx / (vscale * vscale);
    const double scale_phi = 1.0 / (vscale * vscale);
    const int threads = 256;
    pack_fields_kernel<<<(cells + threads - 1) / threads, threads, 0, s>>>(
        ctx->nx, ctx->ny, scale_e, scale_phi, ctx->d_vac, ex, ey, phi, wface, ctx->d_field, ctx->d_barrier);
    TB_CUDA(ctx, cudaGetLastError());
    ctx->vscale = vscale;
    ctx->fields_ready = 1;
    return TB_OK;
}

// Raises the dynamic shared-memory limit of the FP32 tracer to the device maximum.
// Called from tb_create, so launches (also inside a CUDA graph capture) make no
// attribute calls; the attribute is per function and device, always this value.
int tb_configure_trace_f32(tb_ctx *ctx) {
    const int limit = ctx->max_smem - 1024;
#define TB_SMEM_ATTR(T, RF)                                                                                  \
    TB_CUDA(ctx, cudaFuncSetAttribute(trace_f32_kernel<true, T, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                      limit));                                                               \
    if (!RF)                                                                                                 \
    TB_CUDA(ctx, cudaFuncSetAttribute(trace_f32_kernel<true, T, false, true>,                                \
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, limit))
    TB_SMEM_ATTR(1024, false);
    TB_SMEM_ATTR(768, false);
    TB_SMEM_ATTR(512, false);
    TB_SMEM_ATTR(256, false);
    TB_SMEM_ATTR(128, false);
    TB_SMEM_ATTR(1024, true);
    TB_SMEM_ATTR(768, true);
    TB_SMEM_ATTR(512, true);
    TB_SMEM_ATTR(256, true);
    TB_SMEM_ATTR(128, true);
#undef TB_SMEM_ATTR
    TB_CUDA(ctx, cudaFuncSetAttribute(trace_f32_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      limit));
    ctx->smem_attr_bytes = limit;
    return TB_OK;
}

namespace {

K32 make_k32(const tb_ctx *ctx, const tb_trace_args *a) {
    K32 k;
    k.a = *a;
    k.nx = ctx->nx;
    k.ny = ctx->ny;
    k.dx = ctx->dx;
    k.vscale = ctx->vscale;
    k.inv_v = (float)(1.0 / ctx->vscale);
    k.inv_dx = 1.0 / ctx->dx;
    k.inv_v64 = 1.0 / ctx->vscale;
    k.field = ctx->d_field;
    k.barrier = ctx->d_barrier;
    k.queue = ctx->d_queue;
    k.err = ctx->d_err;
    k.bytes = tb_halo_count(ctx->nx, ctx->ny) * (int)sizeof(tb_fcell);
    k.pool_off = -1;
    k.reverse = ctx->tune_reverse == 1;
    k.rec = nullptr;
    k.n_rec = nullptr;
    k.okey = nullptr;
    k.oclass = nullptr;
    k.oblk = k.oacc = nullptr;
    k.inv_lx = 0.0;
    k.onb = 0;
    k.rf_field = ctx->d_rf_field;
    k.rf_barrier = ctx->d_rf_barrier;
    k.rf_wave = ctx->d_rf_wave;
    k.t_clock = k.wave_scale = k.t_sec = k.dt_max = k.bvs = k.bvm = 0.f;
    k.n_phase_m1 = 0;
    if (a->n_phase > 0) {
        // step time unit dx / vscale: in seconds, in clock units, and the in-flight step bound
        const double unit = ctx->dx / ctx->vscale;
        k.t_sec = (float)unit;
        k.t_clock = (float)(unit / a->period * 4294967296.0);
        k.wave_scale = (float)(a->n_phase * 0x1p-32);
        k.n_phase_m1 = a->n_phase - 1;
        k.dt_max = (float)(a->dt_max / unit);
        k.bvs = (float)a->bound_vs;
        k.bvm = (float)a->bound_vm;
    }
    return k;
}

// Bytes of the drain pool for a block of `threads`.
int pool_bytes(int threads, bool rf = false) { return (rf ? POOL_WORDS_RF : POOL_WORDS) * 4 * threads; }

// ---- learned claim order ----------------------------------------------------------------
// A launch ends with the particles still in flight when the queue runs dry.  Claimed in
// index order the ions of a batch come last in random columns, and those above the
// opening travel the whole trench (three to four times the steps of those stopped by the
// mask), so they set the end.  The learned order claims every electron first (in index
// order, as the reverse order does for a batch of ions then electrons) and then the ions
// longest predicted first; the prediction is the mean step count of the ion's bin (128
// starting column bands x 4 bands of vx / |vy|) in the previous trace on this context.
constexpr uint16_t KEY_NONE = 0xffff, KEY_ELECTRON = 0xfffe;

__device__ __forceinline__ int ion_bin(double x, double vx, double vy, double inv_lx) {
    const int xb = min(max((int)(x * inv_lx * 128.0), 0), 127);
    const double h = 0.1 * fabs(vy);
    const int db = vx < 0.0 ? (vx < -h ? 0 : 1) : (vx > h ? 3 : 2);
    return xb * 4 + db;
}

__device__ __forceinline__ int claim_class(uint16_t key, const uint8_t *ion_class) {
    return key == KEY_NONE ? TB_ORDER_CLASSES : (key == KEY_ELECTRON ? 0 : 1 + ion_class[key]);
}

// Blocks of the ordering kernels (k_claim_bins and k_claim_scatter walk the particles
// with the same grid, so each block meets the same particles in both).
constexpr int CLAIM_THREADS = 256;
constexpr int PACK_CLAIM_BLOCKS = 64;   // ordering blocks per case of a pack
int claim_blocks(const tb_ctx *ctx, long long n) {
    return (int)std::max<long long>(1, std::min<long long>((n + CLAIM_THREADS - 1) / CLAIM_THREADS,
                                                           4LL * std::max(ctx->num_sms, 1)));
}

// Each particle's key (ion bin, electron, or not traced) and, per block, the number of
// its particles in each class (blk[block][class]; warp-aggregated shared-memory counts).
// (block b of nb for the case of k)
__device__ __forceinline__ void claim_bins_body(const K32 &k, int b, int nb) {
    __shared__ unsigned h[TB_ORDER_CLASSES];
    const tb_trace_args &a = k.a;
    uint16_t *key = k.okey;
    const uint8_t *ion_class = k.oclass;
    const double inv_lx = k.inv_lx;
    if (threadIdx.x < TB_ORDER_CLASSES) h[threadIdx.x] = 0;
    __syncthreads();
    for (long long i0 = (long long)b * blockDim.x; i0 < a.n; i0 += (long long)nb * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        int c = TB_ORDER_CLASSES;
        if (i < a.n) {
            // every load of the particle issued at once (one memory round trip)
            const int8_t st = a.d_status[i], sp = a.d_spc[i];
            const int32_t n_steps = a.d_steps[i];
            const double x = a.d_x[i], vx = a.d_vx[i], vy = a.d_vy[i];
            uint16_t kk = KEY_NONE;
            if (st == 3 && n_steps < a.max_steps) kk = sp ? KEY_ELECTRON : (uint16_t)ion_bin(x, vx, vy, inv_lx);
            key[i] = kk;
            c = claim_class(kk, ion_class);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        if (c < TB_ORDER_CLASSES && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[c], __popc(peers));
    }
    __syncthreads();
    if (threadIdx.x < TB_ORDER_CLASSES) k.oblk[b * TB_ORDER_CLASSES + threadIdx.x] = h[threadIdx.x];
}

// One block of 1024 threads (thread b for ordering block b, nb <= 1024): the start of
// each ordering block's share of each class in the claim order (classes in turn, blocks
// in turn within a class), written over the counts, and the number of records.  Each
// thread scans its 16 counts within its warp; warp c then scans the warps' totals of
// class c.
__device__ __forceinline__ void claim_scan_body(unsigned *blk, int nb, unsigned *n_rec) {
    constexpr int C = TB_ORDER_CLASSES;
    __shared__ unsigned s_wsum[32][C + 1];   // per warp and class: the warp's total, then the warps before it
    __shared__ unsigned s_tot[C], s_start[C];
    const unsigned FULL = 0xffffffffu;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    unsigned v[C], x[C];
    if (t < nb) {
        const uint4 *row = reinterpret_cast<const uint4 *>(blk + (size_t)t * C);
#pragma unroll
        for (int q = 0; q < C / 4; ++q) {
            const uint4 u = row[q];
            v[4 * q] = u.x;
            v[4 * q + 1] = u.y;
            v[4 * q + 2] = u.z;
            v[4 * q + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = 0u;
    }
#pragma unroll
    for (int c = 0; c < C; ++c) {
        unsigned y = v[c];  // inclusive scan within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned z = __shfl_up_sync(FULL, y, o);
            if (lane >= o) y += z;
        }
        x[c] = y;
        if (lane == 31) s_wsum[w][c] = y;
    }
    __syncthreads();
    if (w < C) {  // warp c: exclusive scan of class c over the 32 warps
        const unsigned own = s_wsum[lane][w];
        unsigned y = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned z = __shfl_up_sync(FULL, y, o);
            if (lane >= o) y += z;
        }
        __syncwarp();
        s_wsum[lane][w] = y - own;
        if (lane == 31) s_tot[w] = y;
    }
    __syncthreads();
    if (t == 0) {
        unsigned off = 0;
        for (int c = 0; c < C; ++c) {
            s_start[c] = off;
            off += s_tot[c];
        }
        *n_rec = off;
    }
    __syncthreads();
    if (t < nb) {
        uint4 *row = reinterpret_cast<uint4 *>(blk + (size_t)t * C);
#pragma unroll
        for (int q = 0; q < C / 4; ++q) {
            uint4 u;
            u.x = s_start[4 * q] + s_wsum[w][4 * q] + x[4 * q] - v[4 * q];
            u.y = s_start[4 * q + 1] + s_wsum[w][4 * q + 1] + x[4 * q + 1] - v[4 * q + 1];
            u.z = s_start[4 * q + 2] + s_wsum[w][4 * q + 2] + x[4 * q + 2] - v[4 * q + 2];
            u.w = s_start[4 * q + 3] + s_wsum[w][4 * q + 3] + x[4 * q + 3] - v[4 * q + 3];
            row[q] = u;
        }
    }
}

// Each traced particle's claim record at its place in the claim order: the FP32 start
// state converted with the claim's expressions (cell, offset, velocity in vscale units,
// q/m), the step count and species, and the particle index.  Places are handed out from
// the block's starts with shared-memory counters.
__device__ __forceinline__ void claim_scatter_body(const K32 &k, int b, int nb) {
    __shared__ unsigned fill[TB_ORDER_CLASSES];
    const tb_trace_args &a = k.a;
    const uint16_t *key = k.okey;
    const uint8_t *ion_class = k.oclass;
    uint4 *rec = k.rec;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < TB_ORDER_CLASSES) fill[threadIdx.x] = k.oblk[b * TB_ORDER_CLASSES + threadIdx.x];
    __syncthreads();
    for (long long i0 = (long long)b * blockDim.x; i0 < a.n; i0 += (long long)nb * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        int c = TB_ORDER_CLASSES;
        uint4 r0 = make_uint4(0u, 0u, 0u, 0u), r1 = r0;
        if (i < a.n) {
            // the key and the particle's data loaded together (one memory round trip)
            const uint16_t kk = key[i];
            const double x = a.d_x[i], y = a.d_y[i], vx64 = a.d_vx[i], vy64 = a.d_vy[i], qm64 = a.d_qm[i];
            const int32_t n_steps = a.d_steps[i];
            const int8_t sp = a.d_spc[i];
            c = claim_class(kk, ion_class);
            const double xc = x * k.inv_dx, yc = y * k.inv_dx;
            const int ix = min(max((int)xc, 0), k.nx - 1);
            const int iy = min((int)floor(yc), k.ny - 1);
            const float ox = fminf(fmaxf((float)(xc - (double)ix), 0.f), ONE_BELOW);
            const float oy = fminf(fmaxf((float)(yc - (double)iy), 0.f), ONE_BELOW);
            const float vx = (float)(vx64 * k.inv_v64), vy = (float)(vy64 * k.inv_v64);
            const float qm = (float)qm64;
            r0 = make_uint4((unsigned)i, ((unsigned)ix & 0xffffu) | ((unsigned)iy << 16), __float_as_uint(ox),
                            __float_as_uint(oy));
            r1 = make_uint4(__float_as_uint(vx), __float_as_uint(vy), __float_as_uint(qm),
                            (unsigned)n_steps | (sp ? 0x80000000u : 0u));
        }
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int leader = __ffs(peers) - 1;
        unsigned base = 0;
        if (lane == leader && c < TB_ORDER_CLASSES) base = atomicAdd(&fill[c], __popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (c < TB_ORDER_CLASSES) {
            const unsigned slot = base + __popc(peers & ((1u << lane) - 1u));
            rec[2 * (size_t)slot] = r0;
            rec[2 * (size_t)slot + 1] = r1;
        }
    }
}

// After the trace: step sum and count of each ion bin (shared-memory histogram per block,
// one global add per bin and block).
__device__ __forceinline__ void claim_learn_body(const K32 &k, int blk_i, int nblk) {
    __shared__ unsigned h[2 * TB_ORDER_ION_BINS];
    const long long n = k.a.n;
    const uint16_t *key = k.okey;
    const int32_t *steps = k.a.d_steps;
    unsigned *acc = k.oacc;
    for (int b = threadIdx.x; b < 2 * TB_ORDER_ION_BINS; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (long long i = (long long)blk_i * blockDim.x + threadIdx.x; i < n; i += (long long)nblk * blockDim.x) {
        const uint16_t kk = key[i];
        if (kk < TB_ORDER_ION_BINS) {
            atomicAdd(&h[2 * kk], (unsigned)steps[i]);
            atomicAdd(&h[2 * kk + 1], 1u);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 2 * TB_ORDER_ION_BINS; b += blockDim.x)
        if (h[b]) atomicAdd(&acc[b], h[b]);
}

// Class of each ion bin for the next launch: 1 for the longest mean step count, then in
// equal steps of that mean down to 15; bins without ions take the mean of all ions.  The
// sums are cleared.
__device__ __forceinline__ void claim_classes_body(unsigned *acc, uint8_t *ion_class) {
    __shared__ float s_sum[TB_ORDER_ION_BINS], s_cnt[TB_ORDER_ION_BINS], s_max[TB_ORDER_ION_BINS];
    const int b = threadIdx.x;
    const float sum = (float)acc[2 * b], cnt = (float)acc[2 * b + 1];
    s_sum[b] = sum;
    s_cnt[b] = cnt;
    s_max[b] = cnt > 0.f ? sum / cnt : 0.f;
    __syncthreads();
    for (int o = TB_ORDER_ION_BINS / 2; o > 0; o >>= 1) {
        if (b < o) {
            s_sum[b] += s_sum[b + o];
            s_cnt[b] += s_cnt[b + o];
            s_max[b] = fmaxf(s_max[b], s_max[b + o]);
        }
        __syncthreads();
    }
    const float mean = s_cnt[0] > 0.f ? s_sum[0] / s_cnt[0] : 0.f, mx = s_max[0];
    const float m = cnt > 0.f ? sum / cnt : mean;
    const int c = mx > 0.f ? (int)(15.f * (1.f - m / (mx * 1.0001f))) : 0;
    ion_class[b] = (uint8_t)min(max(c, 0), 14);
    acc[2 * b] = 0u;
    acc[2 * b + 1] = 0u;
}

// The ordering kernels of one case (grid = the case's ordering blocks) ...
__global__ void __launch_bounds__(CLAIM_THREADS) k_claim_bins(const K32 k) { claim_bins_body(k, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(1024) k_claim_scan(const K32 k) { claim_scan_body(k.oblk, k.onb, k.n_rec); }
__global__ void __launch_bounds__(CLAIM_THREADS) k_claim_scatter(const K32 k) {
    claim_scatter_body(k, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(1024) k_claim_learn(const K32 k) { claim_learn_body(k, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(TB_ORDER_ION_BINS) k_claim_classes(const K32 k) {
    claim_classes_body(k.oacc, k.oclass);
}

// ... and of every case of a pack that claims in the learned order (blockIdx.y or
// blockIdx.x = case; cases without the order and surplus blocks return at once).
__global__ void __launch_bounds__(CLAIM_THREADS) k_pack_claim_bins(const K32 *__restrict__ cases) {
    const K32 &k = cases[blockIdx.y];
    if (k.rec && (int)blockIdx.x < k.onb) claim_bins_body(k, blockIdx.x, k.onb);
}
__global__ void __launch_bounds__(1024) k_pack_claim_scan(const K32 *__restrict__ cases) {
    const K32 &k = cases[blockIdx.x];
    if (k.rec) claim_scan_body(k.oblk, k.onb, k.n_rec);
}
__global__ void __launch_bounds__(CLAIM_THREADS) k_pack_claim_scatter(const K32 *__restrict__ cases) {
    const K32 &k = cases[blockIdx.y];
    if (k.rec && (int)blockIdx.x < k.onb) claim_scatter_body(k, blockIdx.x, k.onb);
}
__global__ void __launch_bounds__(1024) k_pack_claim_learn(const K32 *__restrict__ cases) {
    const K32 &k = cases[blockIdx.y];
    if (k.rec) claim_learn_body(k, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(TB_ORDER_ION_BINS) k_pack_claim_classes(const K32 *__restrict__ cases) {
    const K32 &k = cases[blockIdx.x];
    if (k.rec) claim_classes_body(k.oacc, k.oclass);
}

// Learned-order buffers for n particles, allocated outside stream capture only; a failed
// allocation leaves the order unused (the launch claims in index order).
bool claim_buffers(tb_ctx *ctx, long long n, cudaStream_t s) {
    if (ctx->d_claim_cls && n <= ctx->claim_cap) return true;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return false;
    if (!ctx->d_claim_cls) {
        unsigned *cls = nullptr, *blk = nullptr, *acc = nullptr;
        uint8_t *ion = nullptr;
        const size_t blk_b = (size_t)TB_ORDER_CLASSES * 4 * std::max(ctx->num_sms, 1) * sizeof(unsigned);
        const size_t acc_b = 2 * TB_ORDER_ION_BINS * sizeof(unsigned);
        const bool ok = cudaMalloc(&cls, sizeof(unsigned)) == cudaSuccess && cudaMalloc(&blk, blk_b) == cudaSuccess &&
                        cudaMalloc(&acc, acc_b) == cudaSuccess && cudaMalloc(&ion, TB_ORDER_ION_BINS) == cudaSuccess &&
                        cudaMemset(cls, 0, sizeof(unsigned)) == cudaSuccess && cudaMemset(blk, 0, blk_b) == cudaSuccess &&
                        cudaMemset(acc, 0, acc_b) == cudaSuccess && cudaMemset(ion, 0, TB_ORDER_ION_BINS) == cudaSuccess;
        if (!ok) {
            cudaFree(cls);
            cudaFree(blk);
            cudaFree(acc);
            cudaFree(ion);
            cudaGetLastError();
            return false;
        }
        ctx->d_claim_cls = cls;
        ctx->d_claim_blk = blk;
        ctx->d_ion_acc = acc;
        ctx->d_ion_class = ion;
    }
    if (n > ctx->claim_cap) {
        cudaFree(ctx->d_claim_rec);
        cudaFree(ctx->d_claim_key);
        ctx->d_claim_rec = nullptr;
        ctx->d_claim_key = nullptr;
        ctx->claim_cap = 0;
        if (cudaMalloc(&ctx->d_claim_rec, (size_t)n * 2 * sizeof(uint4)) != cudaSuccess ||
            cudaMalloc(&ctx->d_claim_key, (size_t)n * sizeof(uint16_t)) != cudaSuccess) {
            cudaFree(ctx->d_claim_rec);
            cudaFree(ctx->d_claim_key);
            ctx->d_claim_rec = nullptr;
            ctx->d_claim_key = nullptr;
            cudaGetLastError();
            return false;
        }
        ctx->claim_cap = n;
    }
    return true;
}

// The learned order's fields of a case's kernel arguments (its buffers must exist).
void claim_fields(const tb_ctx *ctx, long long n, int nb, K32 *k) {
    (void)n;
    k->rec = ctx->d_claim_rec;
    k->n_rec = ctx->d_claim_cls;
    k->okey = ctx->d_claim_key;
    k->oclass = ctx->d_ion_class;
    k->oblk = ctx->d_claim_blk;
    k->oacc = ctx->d_ion_acc;
    k->inv_lx = 1.0 / (ctx->nx * ctx->dx);
    k->onb = nb;
}

}  // namespace

int tb_launch_trace_f32(tb_ctx *ctx, const tb_trace_args *a, cudaStream_t s) {
    K32 k = make_k32(ctx, a);
    const bool rf = a->n_phase > 0;
    TB_CUDA(ctx, cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned long long), s));
    // learned claim order (not for circuit_rf launches): records written in claim order
    const bool learned = ctx->tune_reverse == 2 && !rf && a->n > 0 && a->n <= 0x7fffffffLL && ctx->nx < 65536 &&
                         ctx->ny < 32767 && 4 * ctx->num_sms <= 1024 && claim_buffers(ctx, a->n, s);
    if (learned) {
        claim_fields(ctx, a->n, claim_blocks(ctx, a->n), &k);  // at most 4 x SMs <= 1024 blocks
        k_claim_bins<<<k.onb, CLAIM_THREADS, 0, s>>>(k);
        k_claim_scan<<<1, 1024, 0, s>>>(k);
        k_claim_scatter<<<k.onb, CLAIM_THREADS, 0, s>>>(k);
    }
    const bool smem = k.bytes <= ctx->smem_attr_bytes;
    // CTA size and CTAs per SM come from the context's tuning (tb_set_tuning)
    int threads = ctx->tune_threads;
    if (threads == 0) {
        // by batch size: the largest CTA that still puts one on every SM
        const long long per_sm_n = (a->n + ctx->num_sms - 1) / std::max(ctx->num_sms, 1);
        threads = per_sm_n >= 768 ? 1024 : per_sm_n >= 384 ? 512 : per_sm_n >= 192 ? 256 : 128;
    }
    // the drain pool goes after the field when both fit (without the field it always fits
    // under the default 48 KB)
    const int pb = pool_bytes(threads, rf);
    size_t shm = smem ? (size_t)k.bytes : 0;
    k.pool_off = -1;
    if (ctx->nx < 65536 && ctx->ny < 32767 && (!smem || k.bytes + pb <= ctx->smem_attr_bytes)) {
        k.pool_off = (int)shm;
        shm += pb;
    }
    // several CTAs per SM only when their shared memory fits side by side
    int per_sm = ctx->tune_ctas_per_sm;
    if ((long long)per_sm * ((long long)shm + 1024) > ctx->smem_per_sm) per_sm = 1;
    long long want = (a->n + threads - 1) / threads;
    long long cap = (long long)ctx->num_sms * per_sm;
    int blocks = (int)(want < cap ? want : cap);
    if (blocks < 1) blocks = 1;
#define TB_LAUNCH_F32(T)                                                                        \
    do {                                                                                        \
        if (rf) {                                                                               \
            if (smem) trace_f32_kernel<true, T, true><<<blocks, T, shm, s>>>(k);               \
            else trace_f32_kernel<false, T, true><<<blocks, T, shm, s>>>(k);                   \
        } else {                                                                                \
            if (k.rec) {                                                                        \
                if (smem) trace_f32_kernel<true, T, false, true><<<blocks, T, shm, s>>>(k);     \
                else trace_f32_kernel<false, T, false, true><<<blocks, T, shm, s>>>(k);         \
            } else if (smem) trace_f32_kernel<true, T, false><<<blocks, T, shm, s>>>(k);       \
            else trace_f32_kernel<false, T, false><<<blocks, T, shm, s>>>(k);                  \
        }                                                                                       \
    } while (0)
    if (threads == 128) TB_LAUNCH_F32(128);
    else if (threads == 256) TB_LAUNCH_F32(256);
    else if (threads == 512) TB_LAUNCH_F32(512);
    else if (threads == 768) TB_LAUNCH_F32(768);
    else TB_LAUNCH_F32(1024);
#undef TB_LAUNCH_F32
    if (learned) {
        k_claim_learn<<<std::max(ctx->num_sms, 1), 1024, 0, s>>>(k);
        k_claim_classes<<<1, TB_ORDER_ION_BINS, 0, s>>>(k);
    }
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

// ---------------------------------------------------------------------------------
// No-allocation variant of the FP32 tracer.
//
// Some callers cannot call cudaMalloc: a host application that hands every byte of
// device memory to its own pool at start-up, or a caller on a latency-critical
// path where cudaMalloc/cudaFree may synchronise the whole device.  For them
// tb_trace_f32_noalloc keeps the tracer's scratch -- the packed FP32 field, the
// per-face wall barrier, the work-queue counter and the check flag -- in the
// file-scope array below instead of a context.  Every GPU that loads this
// library holds the array (about 2.5 MiB) until the process exits.

namespace {

// a grid of at most MAX cells has a halo-padded field of at most 3*MAX + 6 cells
constexpr size_t NOALLOC_FIELD_BYTES = ((size_t)3 * TB_NOALLOC_MAX_CELLS + 8) * sizeof(tb_fcell);
constexpr size_t NOALLOC_BARRIER_BYTES = (size_t)TB_NOALLOC_MAX_CELLS * sizeof(float4);
constexpr size_t NOALLOC_COUNTER_BYTES = 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_FIELD_BYTES + NOALLOC_BARRIER_BYTES + NOALLOC_COUNTER_BYTES;

// Host code must not pass this name to a kernel: on the host it is a stand-in,
// not a device address.  The per-device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

}  // namespace

extern "C" int tb_trace_f32_noalloc(int nx, int ny, double dx, const uint8_t *d_vac, const tb_trace_args *a,
                                    double vscale, void *stream) {
    if (nx < 1 || ny < 1 || !(dx > 0) || !d_vac || !a || !(vscale > 0))
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: invalid grid, mask or arguments");
    if ((long long)nx * ny > TB_NOALLOC_MAX_CELLS)
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: grid of %lld cells exceeds the %d-cell maximum",
                       (long long)nx * ny, TB_NOALLOC_MAX_CELLS);
    if (a->n < 0 || !(a->cfl > 0 && a->cfl <= 1) || a->max_steps < 1 || a->step_budget < 1)
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: needs n >= 0, 0 < cfl <= 1, max_steps >= 1");
    if (a->n > 0 && (!a->d_x || !a->d_y || !a->d_vx || !a->d_vy || !a->d_qm || !a->d_spc || !a->d_ex ||
                     !a->d_ey || !a->d_counts || !a->d_totals || !a->d_status || !a->d_steps))
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: a required array is missing");
    if ((a->d_phi == nullptr) != (a->d_wface == nullptr))
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: phi and wface must be given together");
    if (a->n_phase > 0 || a->record)
        return tb_fail(nullptr, TB_ERR_ARG, "tb_trace_f32_noalloc: RF clock and record are not supported");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0)
        return tb_fail(nullptr, TB_ERR_DEVICE, "tb_trace_f32_noalloc: no usable current device");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->n == 0) {
        // nothing to trace; the check-flag slot still reports this call
        if (a->d_totals) {
            e = cudaMemsetAsync(a->d_totals + 6, 0, sizeof(int64_t), s);
            if (e != cudaSuccess) return tb_cuda_check(nullptr, e, "cudaMemsetAsync(totals[6])");
        }
        return TB_OK;
    }
    // The array's device address and the kernels' shared-memory attribute are looked up
    // and set on every call (host-side calls that allocate nothing), so a call after a
    // device reset, which reloads the module, uses the new address and attribute.
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return tb_cuda_check(nullptr, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    int num_sms = 0, max_smem = 0;
    e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return tb_cuda_check(nullptr, e, "cudaDeviceGetAttribute");
    tb_ctx tmp;  // a view of the static scratch; owns nothing and is never released
    tmp.device = dev;
    tmp.max_smem = max_smem;
    if (tb_configure_trace_f32(&tmp) != TB_OK) return tb_fail(nullptr, TB_ERR_CUDA, "%s", tmp.err);
    unsigned char *base = static_cast<unsigned char *>(ptr);
    tmp.nx = nx;
    tmp.ny = ny;
    tmp.dx = dx;
    tmp.num_sms = num_sms;
    tmp.d_vac = const_cast<uint8_t *>(d_vac);
    tmp.d_field = reinterpret_cast<tb_fcell *>(base);
    tmp.d_barrier = reinterpret_cast<float4 *>(base + NOALLOC_FIELD_BYTES);
    tmp.d_queue = reinterpret_cast<unsigned long long *>(base + NOALLOC_FIELD_BYTES + NOALLOC_BARRIER_BYTES);
    tmp.d_err = reinterpret_cast<int *>(tmp.d_queue + 8);
    // the array keeps the previous call's contents: clear the counters that must start at zero
    e = cudaMemsetAsync(tmp.d_queue, 0, NOALLOC_COUNTER_BYTES, s);
    if (e != cudaSuccess) return tb_cuda_check(nullptr, e, "cudaMemsetAsync(scratch counters)");
    if (tb_launch_pack_fields(&tmp, a->d_ex, a->d_ey, a->d_phi, a->d_wface, vscale, s) != TB_OK ||
        tb_launch_trace_f32(&tmp, a, s) != TB_OK)
        return tb_fail(nullptr, TB_ERR_CUDA, "%s", tmp.err);
    // the device check flag goes to totals[6] (0 = every bound held)
    e = cudaMemsetAsync(a->d_totals + 6, 0, sizeof(int64_t), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a->d_totals + 6, tmp.d_err, sizeof(int), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return tb_cuda_check(nullptr, e, "copy of the check flag");
    return TB_OK;
}

// ---------------------------------------------------------------------------------
// Case packs: many trench cases traced by one persistent launch.

struct tb_pack {
    int device = 0;
    int n = 0;
    std::vector<tb_ctx *> ctxs;
    K32 *d_cases = nullptr;
    unsigned long long *d_queues = nullptr;  // one work counter per case
    int *d_err = nullptr;
    int max_bytes = 0;
    int max_particles = 0;
    bool smem = false;
    int pool_off = -1;   // drain pool offset in dynamic shared memory, -1 = none
    size_t shm = 0;      // dynamic shared memory without RF cases
    bool small_sides = true;
    int smem_limit = 0;
    int launch_pool_off = -1;  // pool offset and dynamic shared memory of the launch (tb_pack_set_args)
    size_t launch_shm = 0;
    int num_sms = 0;
    int ready = 0;
    int n_learned = 0;   // cases claimed in the learned order (tb_pack_set_args)
    tb_pack_steps *steps = nullptr;  // per-batch update of every case (tb_pack_set_steps)
    char err[512] = {0};
};

namespace {

// status = live, steps = 0, counts = 0, totals = 0 for every case (blockIdx.y = case)
__global__ void k_pack_reset(const K32 *cases, int n_cases) {
    const int c = blockIdx.y;
    if (c >= n_cases) return;
    const K32 &k = cases[c];
    const long long n = k.a.n;
    const int cells2 = 2 * k.nx * k.ny;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n || i < cells2;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < n) { k.a.d_status[i] = 3; k.a.d_steps[i] = 0; }
        if (i < cells2) k.a.d_counts[i] = 0;
        if (i < 8) k.a.d_totals[i] = 0;
    }
}

}  // namespace

static int pack_fail(tb_pack *p, int code, const char *msg) {
    if (p) snprintf(p->err, sizeof(p->err), "%s", msg);
    return tb_fail(nullptr, code, "%s", msg);
}

extern "C" int tb_pack_create(tb_pack **out, int n_cases, tb_ctx *const *ctxs) {
    if (!out || n_cases < 1 || !ctxs) return tb_fail(nullptr, TB_ERR_ARG, "tb_pack_create: no cases");
    *out = nullptr;
    const int dev = ctxs[0] ? ctxs[0]->device : -1;
    for (int i = 0; i < n_cases; ++i)
        if (!ctxs[i] || ctxs[i]->device != dev)
            return tb_fail(nullptr, TB_ERR_ARG, "tb_pack_create: every case needs a context on the same device");
    tb_pack *p = new tb_pack();
    p->device = dev;
    p->n = n_cases;
    p->ctxs.assign(ctxs, ctxs + n_cases);
    p->num_sms = ctxs[0]->num_sms;
    for (int i = 0; i < n_cases; ++i)
        p->max_bytes = std::max(p->max_bytes, tb_halo_count(ctxs[i]->nx, ctxs[i]->ny) * (int)sizeof(tb_fcell));
    p->smem = p->max_bytes <= ctxs[0]->smem_attr_bytes;
    p->shm = p->smem ? (size_t)p->max_bytes : 0;
    bool small_sides = true;
    for (int i = 0; i < n_cases; ++i) small_sides = small_sides && ctxs[i]->nx < 65536 && ctxs[i]->ny < 32767;
    p->small_sides = small_sides;
    p->smem_limit = ctxs[0]->smem_attr_bytes;
    if (small_sides && (!p->smem || p->max_bytes + pool_bytes(F32_THREADS) <= ctxs[0]->smem_attr_bytes)) {
        p->pool_off = (int)p->shm;
        p->shm += pool_bytes(F32_THREADS);
    }
    p->launch_pool_off = p->pool_off;
    p->launch_shm = p->shm;
    cudaError_t e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_cases, sizeof(K32) * n_cases);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_queues, sizeof(unsigned long long) * n_cases);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cudaFree(p->d_cases); cudaFree(p->d_queues); cudaFree(p->d_err);
        delete p;
        return tb_cuda_check(nullptr, e, "tb_pack_create");
    }
    *out = p;
    return TB_OK;
}

extern "C" int tb_pack_destroy(tb_pack *p) {
    if (!p) return TB_OK;
    cudaSetDevice(p->device);
    cudaFree(p->d_cases);
    cudaFree(p->d_queues);
    cudaFree(p->d_err);
    tb_pack_steps_free(p->steps);
    delete p;
    return TB_OK;
}

extern "C" const char *tb_pack_last_error(const tb_pack *p) { return p ? p->err : tb_last_error(nullptr); }

extern "C" int tb_pack_set_args(tb_pack *p, const tb_trace_args *args) {
    if (!p || !args) return TB_ERR_ARG;
    std::vector<K32> ks(p->n);
    p->max_particles = 0;
    for (int i = 0; i < p->n; ++i) {
        const tb_trace_args &a = args[i];
        if (a.n < 0 || a.n > 0x7fffffffLL || !(a.cfl > 0 && a.cfl <= 1) || a.max_steps < 1 || a.step_budget < 1)
            return pack_fail(p, TB_ERR_ARG, "tb_pack_set_args: invalid particle count, cfl or step counts");
        if (a.record) return pack_fail(p, TB_ERR_ARG, "tb_pack_set_args: the case pack traces without record");
        const tb_ctx *c = p->ctxs[i];
        if (a.n_phase > 0 && (!c->rf_ready || c->rf_vscale != c->vscale || a.d_wave != c->rf_wave_src ||
                              a.n_phase != c->rf_n_phase || !a.d_clock || !(a.period > 0) || !(a.dt_max > 0)))
            return pack_fail(p, TB_ERR_ARG,
                             "tb_pack_set_args: an RF case needs tb_set_rf_fields with its waveform, and its clock");
        if (!a.d_x || !a.d_y || !a.d_vx || !a.d_vy || !a.d_qm || !a.d_spc || !a.d_counts || !a.d_totals ||
            !a.d_status || !a.d_steps)
            return pack_fail(p, TB_ERR_ARG, "tb_pack_set_args: a required array is missing");
        if ((a.d_phi == nullptr) != (a.d_wface == nullptr))
            return pack_fail(p, TB_ERR_ARG, "tb_pack_set_args: phi and wface must be given together");
        if (!p->ctxs[i]->fields_ready)
            return pack_fail(p, TB_ERR_ARG, "tb_pack_set_args: a case has no packed field yet");
        ks[i] = make_k32(p->ctxs[i], &a);
        ks[i].queue = p->d_queues + i;
        ks[i].err = p->d_err;
        // the learned claim order, for a case whose context asks for it and holds its buffers
        // (tb_reserve_claim_order); its ordering kernels run over all such cases at once
        // (shared-memory packs only: the global-memory pack kernel keeps its registers)
        if (p->smem && c->tune_reverse == 2 && a.n_phase == 0 && a.n > 0 && c->nx < 65536 && c->ny < 32767 &&
            c->d_claim_cls && a.n <= c->claim_cap)
            claim_fields(c, a.n, (int)std::min<long long>((a.n + CLAIM_THREADS - 1) / CLAIM_THREADS, PACK_CLAIM_BLOCKS),
                         &ks[i]);
        p->max_particles = std::max<int>(p->max_particles, (int)a.n);
    }
    // RF cases keep two more words per lane in the drain pool
    bool rf_any = false;
    for (int i = 0; i < p->n; ++i) rf_any = rf_any || args[i].n_phase > 0;
    p->launch_pool_off = p->pool_off;
    p->launch_shm = p->shm;
    if (rf_any && p->pool_off >= 0) {
        const size_t base = p->smem ? (size_t)p->max_bytes : 0;
        if (base + pool_bytes(F32_THREADS, true) <= (size_t)p->smem_limit) {
            p->launch_shm = base + pool_bytes(F32_THREADS, true);
        } else {
            p->launch_pool_off = -1;
            p->launch_shm = base;
        }
    }
    for (int i = 0; i < p->n; ++i) ks[i].pool_off = p->launch_pool_off;
    p->n_learned = 0;
    for (int i = 0; i < p->n; ++i) p->n_learned += ks[i].rec != nullptr;
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_cases, ks.data(), sizeof(K32) * p->n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return pack_fail(p, TB_ERR_CUDA, cudaGetErrorString(e));
    p->ready = 1;
    return TB_OK;
}

extern "C" int tb_pack_trace(tb_pack *p, int reset, void *stream) {
    if (!p) return TB_ERR_ARG;
    if (!p->ready) return pack_fail(p, TB_ERR_ARG, "tb_pack_trace: call tb_pack_set_args first");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_queues, 0, sizeof(unsigned long long) * p->n, s);
    if (e != cudaSuccess) return pack_fail(p, TB_ERR_CUDA, cudaGetErrorString(e));
    if (reset) {
        const int blocks = std::max(1, std::min(64, (p->max_particles + 255) / 256));
        k_pack_reset<<<dim3(blocks, p->n), 256, 0, s>>>(p->d_cases, p->n);
    }
    if (p->n_learned) {  // claim records of the learned-order cases (after the reset)
        k_pack_claim_bins<<<dim3(PACK_CLAIM_BLOCKS, p->n), CLAIM_THREADS, 0, s>>>(p->d_cases);
        k_pack_claim_scan<<<p->n, 1024, 0, s>>>(p->d_cases);
        k_pack_claim_scatter<<<dim3(PACK_CLAIM_BLOCKS, p->n), CLAIM_THREADS, 0, s>>>(p->d_cases);
    }
    if (p->smem)
        trace_f32_batch_kernel<true><<<p->num_sms, F32_THREADS, p->launch_shm, s>>>(p->d_cases, p->n, p->d_err);
    else
        trace_f32_batch_kernel<false><<<p->num_sms, F32_THREADS, p->launch_shm, s>>>(p->d_cases, p->n, p->d_err);
    if (p->n_learned) {
        k_pack_claim_learn<<<dim3(PACK_CLAIM_BLOCKS / 4, p->n), 1024, 0, s>>>(p->d_cases);
        k_pack_claim_classes<<<p->n, TB_ORDER_ION_BINS, 0, s>>>(p->d_cases);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return pack_fail(p, TB_ERR_CUDA, cudaGetErrorString(e));
    return TB_OK;
}

extern "C" int tb_pack_set_steps(tb_pack *p, const tb_step_desc *descs) {
    if (!p || !descs) return TB_ERR_ARG;
    const int code = tb_pack_steps_set(&p->steps, p->n, p->ctxs.data(), descs, p->err, sizeof(p->err));
    if (code != TB_OK) return tb_fail(nullptr, code, "%s", p->err);
    return TB_OK;
}

extern "C" int tb_pack_step(tb_pack *p, void *stream) {
    if (!p) return TB_ERR_ARG;
    if (!p->steps) return pack_fail(p, TB_ERR_ARG, "tb_pack_step: call tb_pack_set_steps first");
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return pack_fail(p, TB_ERR_CUDA, cudaGetErrorString(e));
    const int code = tb_pack_steps_run(p->steps, (cudaStream_t)stream, p->err, sizeof(p->err));
    if (code != TB_OK) return tb_fail(nullptr, code, "%s", p->err);
    return TB_OK;
}

extern "C" int tb_pack_check(tb_pack *p, void *stream) {
    if (!p) return TB_ERR_ARG;
    int flag = 0;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pack_fail(p, TB_ERR_CUDA, cudaGetErrorString(e));
    if (flag != TB_DERR_NONE) {
        cudaMemsetAsync(p->d_err, 0, sizeof(int), s);
        return pack_fail(p, TB_ERR_KERNEL, "a kernel check failed in the case pack");
    }
    return TB_OK;
}


extern "C" int tb_reserve_claim_order(tb_ctx *ctx, long long n) {
    if (!ctx || n < 0 || n > 0x7fffffffLL) return TB_ERR_ARG;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!claim_buffers(ctx, n > 0 ? n : 1, 0))
        return tb_fail(ctx, TB_ERR_CUDA, "tb_reserve_claim_order: could not allocate the claim-order buffers for %lld particles", n);
    return TB_OK;
}

extern "C" int tb_set_claim_order(tb_ctx *ctx, int order) {
    if (!ctx) return TB_ERR_ARG;
    if (order < 0 || order > 2) return tb_fail(ctx, TB_ERR_ARG, "tb_set_claim_order: order must be 0, 1 or 2");
    ctx->tune_reverse = order;
    return TB_OK;
}

extern "C" int tb_set_tuning(tb_ctx *ctx, int threads, int ctas_per_sm) {
    if (!ctx) return TB_ERR_ARG;
    if ((threads != 0 && threads != 128 && threads != 256 && threads != 512 && threads != 768 && threads != 1024) ||
        ctas_per_sm < 1 || ctas_per_sm > 2)
        return tb_fail(ctx, TB_ERR_ARG,
                       "tb_set_tuning: threads must be 0 (by batch size), 128, 256, 512, 768 or 1024 and CTAs "
                       "per SM 1 or 2");
    ctx->tune_threads = threads;
    ctx->tune_ctas_per_sm = ctas_per_sm;
    return TB_OK;
}
