// Per-batch charge and field update on the device (everything after the trace).
//
// Restates the reference batch loop body (trench_charging_2d.py:1239-1285):
//   deposit     drho = (cnt_i - cnt_e) q / dx^2, zero on conductors      (:1240-1243)
//   leakage     Qs_new = M (rho_s dx^2 + dt G phi_ext)                    (:1246-1256)
//   conductor   driven: rho = 0 on it; floating: semi-implicit step       (:1257-1266, :815-830)
//   potential   phi = solve(-rho/eps0) + external                         (:1268)
//   field       E = -grad phi over vacuum neighbours                      (:1269, :429-454)
//   history     bottom flux ratios, escapes, lost, leak, probe potentials (:1272-1280)
//
// Charge only ever sits on surface cells (every absorbing cell is a solid cell
// next to vacuum), so the state is the surface vector rho_s (m entries, FP64)
// and the potential is phi = external + G rho_s, with G the surface Green's
// operator (built once with the multigrid solver).  Both products are
// bandwidth-bound GEMVs, one warp per row.  The field kernel writes the FP64
// field (reference layout) and the packed FP32 tracer field in one pass.
//
// Compiled with -fmad=false so the field and deposit arithmetic rounds like
// the reference's NumPy expressions.
#include <cooperative_groups.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "tb_internal.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int ONE_BLOCK = 1024;

enum { H_RATIO_I = 0, H_RATIO_E = 1, H_ESC_E = 2, H_LOST = 3, H_LEAK = 4, H_STEPS = 5, H_PROBE0 = 6 };

__device__ double block_reduce(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    __syncthreads();
    return t;  // valid in thread 0
}

// numpy.logaddexp
__device__ double logaddexp(double x, double y) {
    if (x == y) return x + 0.693147180559945309417232121458176568;
    const double t = x - y;
    if (t > 0) return x + log1p(exp(-t));
    if (t <= 0) return y + log1p(exp(t));
    return t;  // NaN
}

// Semi-implicit floating-conductor potential step (trench_charging_2d.py:815-830).
__device__ double conductor_step(double n_i, double n_e, double q, double C, double Te, double drift) {
    const double x_i = q * n_i / C + drift, x_e = q * n_e / C;
    if (n_e == 0) return x_i;
    const double k = x_i / Te;
    const double frac = k != 0 ? -expm1(-k) / k : 1.0;
    return -Te * logaddexp(-k, log(x_e / Te * frac));
}

// K1: deposit counts on the surface vector, leakage input, tallies.
__global__ void __launch_bounds__(ONE_BLOCK) k_deposit(const tb_step_desc d, int ncell, double *tally, int *err) {
    __shared__ double sh[32];
    if (threadIdx.x == 0) *d.d_batch += 1;
    const double dx2 = d.dx * d.dx;
    double ni = 0, ne = 0, bi = 0, be = 0, hi = 0, he = 0, reg = 0;
    for (int s = threadIdx.x; s < d.m; s += blockDim.x) {
        const int c = d.d_surf[s];
        const int ci = d.d_counts[c], ce = d.d_counts[ncell + c];
        const uint8_t f = d.d_sflag[s];
        const double rp = d.d_rho_s[s];
        d.d_rho_prev[s] = rp;
        double drho = ((double)(ci - ce) * d.q_macro) / dx2;
        if (f & TB_SFLAG_COND) drho = 0.0;
        const double r = rp + drho;
        d.d_rho_s[s] = r;
        const double qs = r * dx2;
        d.d_work[s] = d.d_leak_h ? qs + d.d_leak_h[s] : qs;
        if (f & TB_SFLAG_COND) { ni += ci; ne += ce; }
        if (f & TB_SFLAG_BOTTOM) { bi += ci; be += ce; }
        if (f & TB_SFLAG_REGION) reg += qs;
        hi += ci;
        he += ce;
    }
    ni = block_reduce(ni, sh); ne = block_reduce(ne, sh);
    bi = block_reduce(bi, sh); be = block_reduce(be, sh);
    hi = block_reduce(hi, sh); he = block_reduce(he, sh);
    reg = block_reduce(reg, sh);
    if (threadIdx.x == 0) {
        tally[0] = ni; tally[1] = ne; tally[2] = bi; tally[3] = be; tally[4] = reg;
        // every absorbed particle must have landed on a surface cell
        if ((long long)hi != d.d_totals[4] || (long long)he != d.d_totals[5])
            atomicCAS(err, TB_DERR_NONE, TB_DERR_OFF_SURFACE);
    }
}

// y = A x with A row-major (rows, cols); one warp per row, FP64 accumulation.  Row
// `warp` of the product; with `scatter`, y[scatter[warp]] = y0[scatter[warp]] + row.
template <typename T>
__device__ __forceinline__ void gemv_row(int warp, int lane, int cols, const T *A, const double *x, double *y,
                                         const double *y0, const int32_t *scatter) {
    const T *a = A + (size_t)warp * cols;
    double acc = 0.0;
    for (int c = lane; c < cols; c += 32) acc += (double)a[c] * x[c];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        if (scatter) {
            const int cell = scatter[warp];
            y[cell] = y0[cell] + acc;
        } else {
            y[warp] = acc;
        }
    }
}

template <typename T>
__global__ void k_gemv(int rows, int cols, const T *A, const double *x, double *y, const double *y0,
                       const int32_t *scatter) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= rows) return;
    gemv_row<T>(warp, lane, cols, A, x, y, y0, scatter);
}

// K3: leakage result, conductor step, history scalars.
__global__ void __launch_bounds__(ONE_BLOCK) k_finish(const tb_step_desc d, const double *tally) {
    __shared__ double sh[32];
    const double dx2 = d.dx * d.dx;
    const bool leak = d.d_leak_M != nullptr;
    double reg_new = 0, drift = 0;
    for (int s = threadIdx.x; s < d.m; s += blockDim.x) {
        const uint8_t f = d.d_sflag[s];
        double r = d.d_rho_s[s];
        if (leak) {
            const double qn = d.d_work[d.m + s];
            r = qn / dx2;
            if (f & TB_SFLAG_REGION) reg_new += qn;
        }
        if (d.driven && (f & TB_SFLAG_COND)) r = 0.0;
        d.d_rho_s[s] = r;
        if (d.floating) drift += (r - d.d_rho_prev[s]) * d.d_g_s[s];
    }
    reg_new = block_reduce(reg_new, sh);
    drift = block_reduce(drift, sh);
    if (threadIdx.x == 0) {
        const int row = *d.d_batch;
        double leak_ratio = 0.0;
        if (leak) leak_ratio = (tally[4] - reg_new) / d.dt_batch / d.leak_norm;
        if (d.floating && d.c_slot >= 0) {
            drift = drift * dx2;
            const double dV = conductor_step(tally[0], tally[1], d.q_macro, d.C_cond, d.Te, drift);
            d.d_rho_s[d.c_slot] += d.C_cond * (dV - drift) / dx2;
        }
        if (row >= 0 && row < d.max_batches) {
            double *h = d.d_hist + (size_t)row * d.hist_cols;
            h[H_RATIO_I] = tally[2] / d.bottom_norm;
            h[H_RATIO_E] = tally[3] / d.bottom_norm;
            h[H_ESC_E] = (double)d.d_totals[1] / d.n_per_batch;
            h[H_LOST] = (double)d.d_totals[2] / (2.0 * d.n_per_batch);
            h[H_LEAK] = leak_ratio;
            h[H_STEPS] = (double)d.d_totals[3];
        }
    }
}

// Fused charge update (K1 + leakage GEMV + K3 in one launch) for m <= FUSED_MAX_M
// surface slots: one cluster of FUSED_CTAS blocks.  Each block takes a contiguous range
// of slots for the per-slot work and every warp of the cluster a share of the leakage
// rows; the phases are separated by cluster barriers (release/acquire at cluster scope,
// which orders the global-memory writes of one phase before the reads of the next).
// Per-block partial sums are combined by block 0 through distributed shared memory in
// rank order, so the result does not depend on scheduling.
constexpr int FUSED_CTAS = 8;
constexpr int FUSED_MAX_M = 1024;

__device__ __forceinline__ void charge_fused(const tb_step_desc &d, int ncell, int *err) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    __shared__ double sh[32];
    __shared__ double part[10];  // ni, ne, bi, be, hi, he, reg | reg_new, drift
    const double dx2 = d.dx * d.dx;
    const int m = d.m;
    const int per = (m + FUSED_CTAS - 1) / FUSED_CTAS;
    const int s0 = rank * per, s1 = min(m, s0 + per);
    // ---- deposit and leakage input (k_deposit) ----
    double ni = 0, ne = 0, bi = 0, be = 0, hi = 0, he = 0, reg = 0;
    for (int s = s0 + (int)threadIdx.x; s < s1; s += blockDim.x) {
        const int c = d.d_surf[s];
        const int ci = d.d_counts[c], ce = d.d_counts[ncell + c];
        const uint8_t f = d.d_sflag[s];
        const double rp = d.d_rho_s[s];
        d.d_rho_prev[s] = rp;
        double drho = ((double)(ci - ce) * d.q_macro) / dx2;
        if (f & TB_SFLAG_COND) drho = 0.0;
        const double r = rp + drho;
        d.d_rho_s[s] = r;
        const double qs = r * dx2;
        d.d_work[s] = d.d_leak_h ? qs + d.d_leak_h[s] : qs;
        if (f & TB_SFLAG_COND) { ni += ci; ne += ce; }
        if (f & TB_SFLAG_BOTTOM) { bi += ci; be += ce; }
        if (f & TB_SFLAG_REGION) reg += qs;
        hi += ci;
        he += ce;
    }
    ni = block_reduce(ni, sh); ne = block_reduce(ne, sh);
    bi = block_reduce(bi, sh); be = block_reduce(be, sh);
    hi = block_reduce(hi, sh); he = block_reduce(he, sh);
    reg = block_reduce(reg, sh);
    if (threadIdx.x == 0) {
        part[0] = ni; part[1] = ne; part[2] = bi; part[3] = be; part[4] = hi; part[5] = he; part[6] = reg;
    }
    cl.sync();
    // ---- leakage: work[m + r] = M[r] . work[0, m), one warp per row over the cluster ----
    const bool leak = d.d_leak_M != nullptr;
    if (leak) {
        const int wpb = blockDim.x >> 5, lane = threadIdx.x & 31;
        for (int r = rank * wpb + (int)(threadIdx.x >> 5); r < m; r += FUSED_CTAS * wpb) {
            const double *row = d.d_leak_M + (size_t)r * m;
            double acc = 0.0;
            for (int c = lane; c < m; c += 32) acc += row[c] * d.d_work[c];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) d.d_work[m + r] = acc;
        }
    }
    cl.sync();
    // ---- leakage result, driven conductor, drift (k_finish, per slot) ----
    double reg_new = 0, drift = 0;
    for (int s = s0 + (int)threadIdx.x; s < s1; s += blockDim.x) {
        const uint8_t f = d.d_sflag[s];
        double r = d.d_rho_s[s];
        if (leak) {
            const double qn = d.d_work[m + s];
            r = qn / dx2;
            if (f & TB_SFLAG_REGION) reg_new += qn;
        }
        if (d.driven && (f & TB_SFLAG_COND)) r = 0.0;
        d.d_rho_s[s] = r;
        if (d.floating) drift += (r - d.d_rho_prev[s]) * d.d_g_s[s];
    }
    reg_new = block_reduce(reg_new, sh);
    drift = block_reduce(drift, sh);
    if (threadIdx.x == 0) { part[7] = reg_new; part[8] = drift; }
    cl.sync();
    // ---- conductor step and history (k_finish, block 0 thread 0) ----
    if (rank == 0 && threadIdx.x == 0) {
        double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int b = 0; b < FUSED_CTAS; ++b) {
            const double *pb = cl.map_shared_rank(part, b);
            for (int i = 0; i < 9; ++i) t[i] += pb[i];
        }
        // every absorbed particle must have landed on a surface cell
        if ((long long)t[4] != d.d_totals[4] || (long long)t[5] != d.d_totals[5])
            atomicCAS(err, TB_DERR_NONE, TB_DERR_OFF_SURFACE);
        const int row = ++*d.d_batch;
        double leak_ratio = 0.0;
        if (leak) leak_ratio = (t[6] - t[7]) / d.dt_batch / d.leak_norm;
        if (d.floating && d.c_slot >= 0) {
            const double dr = t[8] * dx2;
            const double dV = conductor_step(t[0], t[1], d.q_macro, d.C_cond, d.Te, dr);
            d.d_rho_s[d.c_slot] += d.C_cond * (dV - dr) / dx2;
        }
        if (row >= 0 && row < d.max_batches) {
            double *h = d.d_hist + (size_t)row * d.hist_cols;
            h[H_RATIO_I] = t[2] / d.bottom_norm;
            h[H_RATIO_E] = t[3] / d.bottom_norm;
            h[H_ESC_E] = (double)d.d_totals[1] / d.n_per_batch;
            h[H_LOST] = (double)d.d_totals[2] / (2.0 * d.n_per_batch);
            h[H_LEAK] = leak_ratio;
            h[H_STEPS] = (double)d.d_totals[3];
        }
    }
    cl.sync();  // block 0 has read every block's partial sums before any block exits
}

__global__ void __cluster_dims__(FUSED_CTAS, 1, 1) __launch_bounds__(ONE_BLOCK)
    k_charge_fused(const tb_step_desc d, int ncell, int *err) {
    charge_fused(d, ncell, err);
}

// Charge monitors of the history (trench_charging_2d.py:871-874, 1281-1285): for each
// monitor r, dx^2 sum_s w[r][s] x (|rho_s| if absolute[r] else rho_s) into row
// *d_batch of out.  Charge only sits on surface slots, so the monitors' cell sets are
// weights over the slots; one warp per monitor.
__global__ void k_monitors(const tb_step_desc d, const double *w, const uint8_t *absolute, int n, double *out) {
    const int row = *d.d_batch;
    if (row < 0 || row >= d.max_batches) return;
    const int lane = threadIdx.x & 31;
    for (int r = threadIdx.x >> 5; r < n; r += blockDim.x >> 5) {
        const double *wr = w + (size_t)r * d.m;
        const bool ab = absolute[r] != 0;
        double acc = 0.0;
        for (int s = lane; s < d.m; s += 32) {
            const double v = d.d_rho_s[s];
            acc += wr[s] * (ab ? fabs(v) : v);
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) out[(size_t)row * n + r] = acc * (d.dx * d.dx);
    }
}

// K5: E = -grad phi over vacuum neighbours (trench_charging_2d.py:429-454), the
// packed FP32 tracer field, the per-face wall barrier and the probe history.
__device__ __forceinline__ void field_cell(const tb_step_desc &d, int c, int nx, int ny, const uint8_t *vac,
                                           double scale_e, double scale_phi, tb_fcell *out, float4 *bar) {
    const int n = nx * ny;
    if (c == 0) {
        const int row = *d.d_batch;
        if (row >= 0 && row < d.max_batches)
            for (int k = 0; k < d.n_probes; ++k)
                d.d_hist[(size_t)row * d.hist_cols + H_PROBE0 + k] = d.d_phi[d.d_probes[k]];
    }
    if (c >= n) return;
    const int ix = c / ny, iy = c - ix * ny;
    const int w = (ix == 0 ? nx - 1 : ix - 1) * ny + iy, e = (ix == nx - 1 ? 0 : ix + 1) * ny + iy;
    const double *phi = d.d_phi;
    const double pc = phi[c];
    const double dx = d.dx;
    // x: neighbours west (m) and east (pl)
    double gx = 0.0;
    {
        const bool vm = vac[w], vp = vac[e];
        const double m = phi[w], pl = phi[e];
        if (vm && vp) gx = (pl - m) / (2 * dx);
        else if (vp) gx = (pl - pc) / dx;
        else if (vm) gx = (pc - m) / dx;
    }
    double gy = 0.0;
    {
        const bool vm = iy > 0 ? vac[c - 1] : false;
        const bool vp = iy < ny - 1 ? vac[c + 1] : true;
        const double m = iy > 0 ? phi[c - 1] : 2 * d.v_sub - pc;
        const double pl = iy < ny - 1 ? phi[c + 1] : (d.top_dirichlet ? 2 * d.v_top - pc : pc);
        if (vm && vp) gy = (pl - m) / (2 * dx);
        else if (vp) gy = (pl - pc) / dx;
        else if (vm) gy = (pc - m) / dx;
    }
    const double ex = -gx, ey = -gy;
    if (d.d_ex) { d.d_ex[c] = ex; d.d_ey[c] = ey; }
    const int v = vac[c] ? 1 : 0;
    tb_store_packed(out, vac, nx, ny, ix, iy, tb_pack_cell(ex, ey, v, scale_e));
    float4 b = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!v && d.d_wface) {
        const double f = d.d_wface[c];
        b.x = (float)(f * (pc - phi[w]) * scale_phi);
        b.y = (float)(f * (pc - phi[e]) * scale_phi);
        b.z = iy > 0 ? (float)(f * (pc - phi[c - 1]) * scale_phi) : 0.f;
        b.w = iy < ny - 1 ? (float)(f * (pc - phi[c + 1]) * scale_phi) : 0.f;
    }
    bar[c] = b;
}

__global__ void k_field(const tb_step_desc d, int nx, int ny, const uint8_t *vac, double scale_e, double scale_phi,
                        tb_fcell *out, float4 *bar) {
    field_cell(d, blockIdx.x * blockDim.x + threadIdx.x, nx, ny, vac, scale_e, scale_phi, out, bar);
}

// ---- the same update for every case of a pack, one launch per stage ----------------
// Case = blockIdx.y; each case's descriptor, grid and packed-field outputs in one entry.
constexpr int PACK_THREADS = 256;

__global__ void __cluster_dims__(FUSED_CTAS, 1, 1) __launch_bounds__(ONE_BLOCK)
    k_pack_charge(const tb_pack_step_entry *E) {
    const tb_pack_step_entry &e = E[blockIdx.y];
    charge_fused(e.d, e.nx * e.ny, e.err);
}

__global__ void __launch_bounds__(PACK_THREADS) k_pack_green(const tb_pack_step_entry *E) {
    const tb_pack_step_entry &e = E[blockIdx.y];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= e.d.n_rows) return;
    if (e.d.d_green)
        gemv_row<float>(warp, lane, e.d.m, e.d.d_green, e.d.d_rho_s, e.d.d_phi, e.d.d_ext, e.d.d_rows);
    else
        gemv_row<double>(warp, lane, e.d.m, e.d.d_green64, e.d.d_rho_s, e.d.d_phi, e.d.d_ext, e.d.d_rows);
}

__global__ void __launch_bounds__(PACK_THREADS) k_pack_field(const tb_pack_step_entry *E) {
    const tb_pack_step_entry &e = E[blockIdx.y];
    field_cell(e.d, blockIdx.x * blockDim.x + threadIdx.x, e.nx, e.ny, e.vac, e.scale_e, e.scale_phi, e.field,
               e.bar);
}

}  // namespace

extern "C" int tb_step_charge(tb_ctx *ctx, const tb_step_desc *d, void *stream) {
    if (!ctx || !d) return TB_ERR_ARG;
    if (d->m < 1 || !d->d_surf || !d->d_sflag || !d->d_rho_s || !d->d_rho_prev || !d->d_work || !d->d_counts ||
        !d->d_totals || !d->d_batch || !d->d_hist || d->hist_cols < 6 || !(d->dx > 0) || !(d->bottom_norm > 0) ||
        !(d->n_per_batch > 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_step_charge: incomplete step descriptor");
    if (d->floating && (!d->d_g_s || !(d->C_cond > 0)))
        return tb_fail(ctx, TB_ERR_ARG, "tb_step_charge: floating conductor needs g_s and C_cond");
    if (d->d_leak_M && !(d->dt_batch > 0 && d->leak_norm > 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_step_charge: leakage needs dt_batch and leak_norm");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (d->m <= FUSED_MAX_M) {
        k_charge_fused<<<FUSED_CTAS, ONE_BLOCK, 0, s>>>(*d, ctx->nx * ctx->ny, ctx->d_err);
        TB_CUDA(ctx, cudaGetLastError());
        return TB_OK;
    }
    // many surface slots: the leakage GEMV runs over the whole GPU between two one-block kernels
    double *tally = reinterpret_cast<double *>(ctx->d_queue + 2);  // 5 doubles of context scratch
    k_deposit<<<1, ONE_BLOCK, 0, s>>>(*d, ctx->nx * ctx->ny, tally, ctx->d_err);
    if (d->d_leak_M) {
        const int threads = 256, wpb = threads / 32;
        k_gemv<double><<<(d->m + wpb - 1) / wpb, threads, 0, s>>>(d->m, d->m, d->d_leak_M, d->d_work,
                                                                  d->d_work + d->m, nullptr, nullptr);
    }
    k_finish<<<1, ONE_BLOCK, 0, s>>>(*d, tally);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

extern "C" int tb_step_potential(tb_ctx *ctx, const tb_step_desc *d, void *stream) {
    if (!ctx || !d) return TB_ERR_ARG;
    if (d->n_rows < 1 || !d->d_rows || (!d->d_green && !d->d_green64) || !d->d_ext || !d->d_phi ||
        !(d->vscale > 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_step_potential: incomplete step descriptor");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256, wpb = threads / 32;
    const int blocks = (d->n_rows + wpb - 1) / wpb;
    if (d->d_green)
        k_gemv<float><<<blocks, threads, 0, s>>>(d->n_rows, d->m, d->d_green, d->d_rho_s, d->d_phi, d->d_ext,
                                                 d->d_rows);
    else
        k_gemv<double><<<blocks, threads, 0, s>>>(d->n_rows, d->m, d->d_green64, d->d_rho_s, d->d_phi, d->d_ext,
                                                  d->d_rows);
    const int cells = ctx->nx * ctx->ny;
    const double scale_e = ctx->dx / (d->vscale * d->vscale), scale_phi = 1.0 / (d->vscale * d->vscale);
    k_field<<<(cells + 255) / 256, 256, 0, s>>>(*d, ctx->nx, ctx->ny, ctx->d_vac, scale_e, scale_phi, ctx->d_field,
                                               ctx->d_barrier);
    TB_CUDA(ctx, cudaGetLastError());
    ctx->vscale = d->vscale;
    ctx->fields_ready = 1;
    return TB_OK;
}

// The per-batch state before a trace, in one launch: every particle untraced (status 3,
// no steps), the hit counts and the totals zero.
__global__ void k_batch_reset(int8_t *status, int32_t *steps, long long n, int32_t *counts, long long n_counts,
                              unsigned long long *totals, int n_totals) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long end = n > n_counts ? n : n_counts;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
        if (i < n) {
            status[i] = 3;
            steps[i] = 0;
        }
        if (i < n_counts) counts[i] = 0;
        if (i < n_totals) totals[i] = 0ULL;
    }
}

extern "C" int tb_batch_reset(tb_ctx *ctx, int8_t *d_status, int32_t *d_steps, long long n, int32_t *d_counts,
                              long long n_counts, unsigned long long *d_totals, int n_totals, void *stream) {
    if (!ctx || n < 0 || n_counts < 0 || n_totals < 0 || n_totals > 64 || (n > 0 && (!d_status || !d_steps)) ||
        (n_counts > 0 && !d_counts) || (n_totals > 0 && !d_totals))
        return tb_fail(ctx, TB_ERR_ARG, "tb_batch_reset: invalid arguments");
    const long long end = std::max(std::max(n, n_counts), (long long)n_totals);
    if (end == 0) return TB_OK;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    const int threads = 256;
    const long long want = (end + threads - 1) / threads;
    const int blocks = (int)std::min<long long>(want, 8LL * std::max(ctx->num_sms, 1));
    k_batch_reset<<<blocks, threads, 0, (cudaStream_t)stream>>>(d_status, d_steps, n, d_counts, n_counts, d_totals,
                                                                 n_totals);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

extern "C" int tb_step_monitors(tb_ctx *ctx, const tb_step_desc *d, const double *d_weights,
                                const uint8_t *d_absolute, int n_monitors, double *d_out, void *stream) {
    if (!ctx || !d) return TB_ERR_ARG;
    if (n_monitors < 0 || (n_monitors > 0 && (!d_weights || !d_absolute || !d_out)) || d->m < 1 || !d->d_rho_s ||
        !d->d_batch || !(d->dx > 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_step_monitors: invalid arguments");
    if (n_monitors == 0) return TB_OK;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    k_monitors<<<1, 256, 0, (cudaStream_t)stream>>>(*d, d_weights, d_absolute, n_monitors, d_out);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}


// ---- case packs: the per-batch update of every case, one launch per stage ---------------

struct tb_pack_steps {
    int n = 0;
    std::vector<tb_ctx *> ctxs;
    std::vector<tb_step_desc> descs;
    std::vector<int> own_charge;     // cases whose charge update runs alone (m > FUSED_MAX_M)
    tb_pack_step_entry *d_entries = nullptr;
    tb_pack_step_entry *d_fused = nullptr;  // the cases of the batched charge launch
    int n_fused = 0;
    int green_blocks = 0, field_blocks = 0;
};

void tb_pack_steps_free(tb_pack_steps *ps) {
    if (!ps) return;
    cudaFree(ps->d_entries);
    cudaFree(ps->d_fused);
    delete ps;
}

int tb_pack_steps_set(tb_pack_steps **out, int n, tb_ctx *const *ctxs, const tb_step_desc *descs, char *err,
                      size_t errlen) {
    auto fail = [&](const char *msg) {
        snprintf(err, errlen, "%s", msg);
        return TB_ERR_ARG;
    };
    if (n < 1 || n > 65535 || !ctxs || !descs) return fail("tb_pack_set_steps: needs 1 to 65535 cases");
    std::vector<tb_pack_step_entry> entries(n), fused;
    std::vector<int> own;
    int green_blocks = 0, field_blocks = 0;
    const int wpb = PACK_THREADS / 32;
    for (int i = 0; i < n; ++i) {
        const tb_step_desc &d = descs[i];
        const tb_ctx *c = ctxs[i];
        if (d.m < 1 || !d.d_surf || !d.d_sflag || !d.d_rho_s || !d.d_rho_prev || !d.d_work || !d.d_counts ||
            !d.d_totals || !d.d_batch || !d.d_hist || d.hist_cols < 6 || !(d.dx > 0) || !(d.bottom_norm > 0) ||
            !(d.n_per_batch > 0) || d.n_rows < 1 || !d.d_rows || (!d.d_green && !d.d_green64) || !d.d_ext ||
            !d.d_phi || !(d.vscale > 0))
            return fail("tb_pack_set_steps: incomplete step descriptor");
        if (d.floating && (!d.d_g_s || !(d.C_cond > 0)))
            return fail("tb_pack_set_steps: floating conductor needs g_s and C_cond");
        if (d.d_leak_M && !(d.dt_batch > 0 && d.leak_norm > 0))
            return fail("tb_pack_set_steps: leakage needs dt_batch and leak_norm");
        tb_pack_step_entry &e = entries[i];
        e.d = d;
        e.nx = c->nx;
        e.ny = c->ny;
        e.vac = c->d_vac;
        e.scale_e = c->dx / (d.vscale * d.vscale);
        e.scale_phi = 1.0 / (d.vscale * d.vscale);
        e.field = c->d_field;
        e.bar = c->d_barrier;
        e.err = c->d_err;
        if (d.m <= FUSED_MAX_M) fused.push_back(e);
        else own.push_back(i);
        green_blocks = std::max(green_blocks, (d.n_rows + wpb - 1) / wpb);
        field_blocks = std::max(field_blocks, (c->nx * c->ny + PACK_THREADS - 1) / PACK_THREADS);
    }
    tb_pack_steps *ps = new tb_pack_steps();
    cudaError_t e = cudaSetDevice(ctxs[0]->device);
    if (e == cudaSuccess) e = cudaMalloc(&ps->d_entries, sizeof(tb_pack_step_entry) * n);
    if (e == cudaSuccess && !fused.empty()) e = cudaMalloc(&ps->d_fused, sizeof(tb_pack_step_entry) * fused.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(ps->d_entries, entries.data(), sizeof(tb_pack_step_entry) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !fused.empty())
        e = cudaMemcpy(ps->d_fused, fused.data(), sizeof(tb_pack_step_entry) * fused.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        tb_pack_steps_free(ps);
        snprintf(err, errlen, "tb_pack_set_steps: %s", cudaGetErrorString(e));
        return TB_ERR_CUDA;
    }
    ps->n = n;
    ps->ctxs.assign(ctxs, ctxs + n);
    ps->descs.assign(descs, descs + n);
    ps->own_charge = own;
    ps->n_fused = (int)fused.size();
    ps->green_blocks = green_blocks;
    ps->field_blocks = field_blocks;
    tb_pack_steps_free(*out);
    *out = ps;
    return TB_OK;
}

int tb_pack_steps_run(tb_pack_steps *ps, cudaStream_t s, char *err, size_t errlen) {
    if (ps->n_fused > 0) k_pack_charge<<<dim3(FUSED_CTAS, ps->n_fused), ONE_BLOCK, 0, s>>>(ps->d_fused);
    for (int i : ps->own_charge) {
        const int code = tb_step_charge(ps->ctxs[i], &ps->descs[i], s);
        if (code != TB_OK) {
            snprintf(err, errlen, "%s", ps->ctxs[i]->err);
            return code;
        }
    }
    k_pack_green<<<dim3(ps->green_blocks, ps->n), PACK_THREADS, 0, s>>>(ps->d_entries);
    k_pack_field<<<dim3(ps->field_blocks, ps->n), PACK_THREADS, 0, s>>>(ps->d_entries);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(err, errlen, "tb_pack_step: %s", cudaGetErrorString(e));
        return TB_ERR_CUDA;
    }
    for (int i = 0; i < ps->n; ++i) {
        ps->ctxs[i]->vscale = ps->descs[i].vscale;
        ps->ctxs[i]->fields_ready = 1;
    }
    return TB_OK;
}
