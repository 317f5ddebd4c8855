// Adjoint of the charging loop: history tallies, the surrogate recurrence over the
// stored histories, and its reverse sweep.
//
// Likelihood-ratio reweighting.  Ion energies and angles are drawn from histogram
// tables with bin probabilities p_k.  Changing them to r_k p_k reweights every
// traced ion by r(bin); with the trajectories held fixed, the expected ion deposit
// of batch b on surface slot s becomes
//     ci_b[s](r) = Ni_b[s] + sum_k (rE_k - 1) TE_b[k][s] + sum_l (rA_l - 1) TA_b[l][s]
// (first order in r - 1; at r = 1 it is the traced count), TE/TA the per-bin
// tallies of the absorbed ions.  d ci_b / d r_k = T_b[k] is the score-function
// (likelihood-ratio) estimator of the deposit's sensitivity to the bin weight.
//
// The charge update over those deposits is the recurrence of tb_step_charge
// (trench_charging_2d.py:1239-1266: deposit, leakage, driven or floating
// conductor), same arithmetic, so at r = 1 it reproduces the traced run's surface
// charge (to the rounding of the real-valued sums, which tb_step_charge may add in
// another order).  Its adjoint, per batch in reverse, with
// lambda = dJ / d rho_{b+1}:
//   floating conductor  rho_{b+1} = r' + e_c C (dV - drift) / dx^2,
//                       drift = dx^2 sum_s g_s (r'_s - rho_b,s), dV = f(ni, ne, drift)
//     => lambda'_s = lambda_s + kappa g_s, kappa = lambda_c C (df/dx_i - 1),
//        dJ/d ni = lambda_c (q / dx^2) df/dx_i, dJ/d ne = lambda_c (q / dx^2) df/dx_e,
//        and -kappa g_s flows to rho_b
//   driven conductor    lambda'_s = 0 on conductor slots
//   leakage             r' = M (r dx^2 + h) / dx^2  =>  u = M^T lambda'
//   deposit             r = rho_b + (ci - ce) q / dx^2 (0 on conductors)
//     => lambda_b = u - kappa g,  mu_s = dJ/d ci_s = u_s q / dx^2 (+ dJ/d ni on the
//        conductor, + dJ/d bottom_b on bottom slots)
//   parameters          dJ/d r_k += sum_s T_b[k][s] mu_s.
// Field feedback (optional): the traced deposits themselves depend on rho_b through
// the field.  With their response measured along orthonormal surface-charge modes V
// (ci(rho) ~ ci + Ui V^T (rho - rho_b), ce likewise with Ue),
//     lambda_b += V (Ui^T mu + Ue^T mu_e),  mu_e_s = dJ/d ce_s
// (-u_s q / dx^2 off the conductor, dJ/d ne on it).
// f is the semi-implicit conductor step (trench_charging_2d.py:815-830):
//   x_i = q ni / C + drift, x_e = q ne / C, k = x_i / Te, frac = (1 - e^-k) / k,
//   f = -Te logaddexp(-k, L), L = log(x_e frac / Te);
//   df/dx_i = s1 - s2 (1/(e^k - 1) - 1/k), df/dx_e = -Te s2 / x_e,
//   s1 = 1 / (1 + e^(k + L)), s2 = 1 - s1 (the weights of logaddexp's arguments).
//
// Compiled with -fmad=false, like the step kernels it mirrors.
#include <math.h>

#include "tb_internal.cuh"

namespace {

constexpr int ONE_BLOCK = 1024;

__device__ double block_sum(double v, double *sh) {
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

__device__ double logaddexp(double x, double y) {
    if (x == y) return x + 0.693147180559945309417232121458176568;
    const double t = x - y;
    if (t > 0) return x + log1p(exp(-t));
    if (t <= 0) return y + log1p(exp(t));
    return t;  // NaN
}

__device__ double conductor_step(double n_i, double n_e, double q, double C, double Te, double drift) {
    const double x_i = q * n_i / C + drift, x_e = q * n_e / C;
    if (n_e == 0) return x_i;
    const double k = x_i / Te;
    const double frac = k != 0 ? -expm1(-k) / k : 1.0;
    return -Te * logaddexp(-k, log(x_e / Te * frac));
}

// d(conductor_step)/d x_i (= d/d drift) and d/d x_e.  With no electron deposit the
// step is x_i itself.
__device__ void conductor_partials(double n_i, double n_e, double q, double C, double Te, double drift,
                                   double *f_xi, double *f_xe) {
    if (n_e == 0) { *f_xi = 1.0; *f_xe = 0.0; return; }
    const double x_i = q * n_i / C + drift, x_e = q * n_e / C;
    const double k = x_i / Te;
    const double frac = k != 0 ? -expm1(-k) / k : 1.0;
    const double L = log(x_e / Te * frac);
    const double s1 = 1.0 / (1.0 + exp(k + L)), s2 = 1.0 / (1.0 + exp(-(k + L)));
    // d log(frac) / dk = 1/(e^k - 1) - 1/k; Laurent series near k = 0
    const double k2 = k * k;
    const double dlf = fabs(k) < 1e-2 ? -0.5 + k * (1.0 / 12.0 - k2 * (1.0 / 720.0 - k2 / 30240.0))
                                      : 1.0 / expm1(k) - 1.0 / k;
    *f_xi = s1 - s2 * dlf;
    *f_xe = -Te * s2 / x_e;
}

__global__ void k_tally(const tb_tally_args a, int ncell, int *err) {
    const long long n = a.n_species;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n || a.d_status[i] != 1) return;
    const int c = a.d_hit[i];
    const int s = (c >= 0 && c < ncell) ? a.d_slot[c] : -1;
    if (s < 0 || s >= a.m) { atomicCAS(err, TB_DERR_NONE, TB_DERR_OFF_SURFACE); return; }
    const int ne = a.n_energy, na = a.n_angle;
    if (i < n) {
        const int be = a.d_bin_e ? a.d_bin_e[i] : 0, ba = a.d_bin_a ? a.d_bin_a[i] : 0;
        if ((ne > 0 && be >= ne) || (na > 0 && ba >= na)) { atomicCAS(err, TB_DERR_NONE, TB_DERR_BAD_CELL); return; }
        if (ne > 0) atomicAdd(&a.d_table[(size_t)be * a.m + s], 1);
        if (na > 0) atomicAdd(&a.d_table[(size_t)(ne + ba) * a.m + s], 1);
        atomicAdd(&a.d_table[(size_t)(ne + na) * a.m + s], 1);
    } else {
        atomicAdd(&a.d_table[(size_t)(ne + na + 1) * a.m + s], 1);
    }
}

// Reweighted ion deposit on slot s of one table.
__device__ double ion_deposit(const tb_adjoint_args &a, const int32_t *T, int m, int s) {
    const int ne = a.n_energy, na = a.n_angle;
    double ci = (double)T[(size_t)(ne + na) * m + s];
    if (a.d_rE)
        for (int k = 0; k < ne; ++k) ci += (a.d_rE[k] - 1.0) * (double)T[(size_t)k * m + s];
    if (a.d_rA)
        for (int l = 0; l < na; ++l) ci += (a.d_rA[l] - 1.0) * (double)T[(size_t)(ne + l) * m + s];
    return ci;
}

// Forward 1/2: deposit and leakage input (tb_step.cu k_deposit, over table deposits).
__global__ void __launch_bounds__(ONE_BLOCK) k_fwd_deposit(const tb_step_desc d, const tb_adjoint_args a, int b) {
    __shared__ double sh[32];
    const int m = d.m;
    const int32_t *T = a.d_tables + (size_t)b * (a.n_energy + a.n_angle + 2) * m;
    const double dx2 = d.dx * d.dx;
    double ni = 0, ne = 0, bi = 0;
    for (int s = threadIdx.x; s < m; s += blockDim.x) {
        const double ci = ion_deposit(a, T, m, s);
        const double ce = (double)T[(size_t)(a.n_energy + a.n_angle + 1) * m + s];
        const uint8_t f = d.d_sflag[s];
        const double rp = a.d_rho[s];
        d.d_rho_prev[s] = rp;
        double drho = ((ci - ce) * d.q_macro) / dx2;
        if (f & TB_SFLAG_COND) drho = 0.0;
        const double r = rp + drho;
        a.d_rho[s] = r;
        const double qs = r * dx2;
        d.d_work[s] = d.d_leak_h ? qs + d.d_leak_h[s] : qs;
        if (f & TB_SFLAG_COND) { ni += ci; ne += ce; }
        if (f & TB_SFLAG_BOTTOM) bi += ci;
    }
    ni = block_sum(ni, sh);
    ne = block_sum(ne, sh);
    bi = block_sum(bi, sh);
    if (threadIdx.x == 0) {
        a.d_scal[4 * b + 0] = ni;
        a.d_scal[4 * b + 1] = ne;
        a.d_bottom[b] = bi;
    }
}

// y = A x, A row-major (rows, cols), one warp per row; with acc != 0, y += A x.
template <typename T>
__global__ void k_gemv(int rows, int cols, const T *A, const double *x, double *y, int acc) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const T *r = A + (size_t)warp * cols;
    double s = 0.0;
    for (int c = lane; c < cols; c += 32) s += (double)r[c] * x[c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y[warp] = acc ? y[warp] + s : s;
}

// Forward 2/2: leakage result, driven conductor, floating-conductor step (k_finish).
__global__ void __launch_bounds__(ONE_BLOCK) k_fwd_finish(const tb_step_desc d, const tb_adjoint_args a, int b) {
    __shared__ double sh[32];
    const double dx2 = d.dx * d.dx;
    const bool leak = d.d_leak_M != nullptr;
    double drift = 0;
    for (int s = threadIdx.x; s < d.m; s += blockDim.x) {
        const uint8_t f = d.d_sflag[s];
        double r = a.d_rho[s];
        if (leak) r = d.d_work[d.m + s] / dx2;
        if (d.driven && (f & TB_SFLAG_COND)) r = 0.0;
        a.d_rho[s] = r;
        if (d.floating) drift += (r - d.d_rho_prev[s]) * d.d_g_s[s];
    }
    drift = block_sum(drift, sh);
    if (threadIdx.x == 0) {
        double dr = 0.0;
        if (d.floating && d.c_slot >= 0) {
            dr = drift * dx2;
            const double ni = a.d_scal[4 * b + 0], ne = a.d_scal[4 * b + 1];
            const double dV = conductor_step(ni, ne, d.q_macro, d.C_cond, d.Te, dr);
            a.d_rho[d.c_slot] += d.C_cond * (dV - dr) / dx2;
        }
        a.d_scal[4 * b + 2] = dr;
    }
}

// Scratch layout of the reverse sweep: [0, m) mu (ion deposits), [m, 2m) mu_e
// (electron deposits), 2m kappa, 2m + 1 dJ/d ni, 2m + 2 dJ/d ne, [2m + 4, ...) the
// feedback coefficients.

// Reverse 1/3: through the conductor step; lambda' into work[0, m).
__global__ void __launch_bounds__(ONE_BLOCK) k_rev_conductor(const tb_step_desc d, const tb_adjoint_args a, int b,
                                                             const double *lambda, double *scratch) {
    __shared__ double kap_sh;
    if (threadIdx.x == 0) {
        double kap = 0.0, jni = 0.0, jne = 0.0;
        if (d.floating && d.c_slot >= 0) {
            double f_xi, f_xe;
            conductor_partials(a.d_scal[4 * b + 0], a.d_scal[4 * b + 1], d.q_macro, d.C_cond, d.Te,
                               a.d_scal[4 * b + 2], &f_xi, &f_xe);
            const double lc = lambda[d.c_slot];
            kap = lc * d.C_cond * (f_xi - 1.0);
            jni = lc * f_xi * d.q_macro / (d.dx * d.dx);
            jne = lc * f_xe * d.q_macro / (d.dx * d.dx);
        }
        kap_sh = kap;
        scratch[2 * d.m] = kap;
        scratch[2 * d.m + 1] = jni;
        scratch[2 * d.m + 2] = jne;
    }
    __syncthreads();
    const double kap = kap_sh;
    for (int s = threadIdx.x; s < d.m; s += blockDim.x) {
        double l = lambda[s];
        if (d.floating) l += kap * d.d_g_s[s];
        if (d.driven && (d.d_sflag[s] & TB_SFLAG_COND)) l = 0.0;
        d.d_work[s] = l;
    }
}

// Reverse 2/3: through the deposit; lambda <- dJ/d rho_b, mu and mu_e into scratch.
__global__ void __launch_bounds__(ONE_BLOCK) k_rev_deposit(const tb_step_desc d, const tb_adjoint_args a, int b,
                                                           double *lambda, const double *gbottom, double *scratch) {
    const double dx2 = d.dx * d.dx;
    const bool leak = d.d_leak_M != nullptr;
    const double kap = scratch[2 * d.m], jni = scratch[2 * d.m + 1], jne = scratch[2 * d.m + 2];
    const double gb = gbottom ? gbottom[b] : 0.0;
    for (int s = threadIdx.x; s < d.m; s += blockDim.x) {
        const uint8_t f = d.d_sflag[s];
        const double u = leak ? d.d_work[d.m + s] : d.d_work[s];
        const bool cond = f & TB_SFLAG_COND;
        double mu = cond ? (d.floating ? jni : 0.0) : u * d.q_macro / dx2;
        if (f & TB_SFLAG_BOTTOM) mu += gb;
        scratch[s] = mu;
        scratch[d.m + s] = cond ? (d.floating ? jne : 0.0) : -(u * d.q_macro / dx2);
        lambda[s] = d.floating ? u - kap * d.d_g_s[s] : u;
    }
}

// Reverse 3/3 (field feedback): lambda += V (Ui^T mu + Ue^T mu_e) with the batch's
// response set; one warp per mode for the coefficients.
__global__ void __launch_bounds__(ONE_BLOCK) k_rev_feedback(const tb_step_desc d, const tb_adjoint_args a, int b,
                                                            double *lambda, double *scratch) {
    const int set = a.d_resp_index[b];
    if (set < 0) return;
    const int m = d.m, K = a.n_basis;
    const double *Ui = a.d_resp_i + (size_t)set * m * K, *Ue = a.d_resp_e + (size_t)set * m * K;
    double *coef = scratch + 2 * m + 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int j = warp; j < K; j += warps) {
        double c = 0.0;
        for (int s = lane; s < m; s += 32)
            c += Ui[(size_t)s * K + j] * scratch[s] + Ue[(size_t)s * K + j] * scratch[m + s];
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) coef[j] = c;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < m; s += blockDim.x) {
        double add = 0.0;
        for (int j = 0; j < K; ++j) add += a.d_basis[(size_t)s * K + j] * coef[j];
        lambda[s] += add;
    }
}

int check_step(tb_ctx *ctx, const tb_step_desc *d, const tb_adjoint_args *a, const char *who) {
    if (d->m < 1 || !d->d_sflag || !d->d_rho_prev || !d->d_work || !(d->dx > 0))
        return tb_fail(ctx, TB_ERR_ARG, "%s: incomplete step descriptor", who);
    if (d->floating && (!d->d_g_s || !(d->C_cond > 0)))
        return tb_fail(ctx, TB_ERR_ARG, "%s: floating conductor needs g_s and C_cond", who);
    if (a->n_batches < 1 || a->n_energy < 0 || a->n_angle < 0 || !a->d_tables || !a->d_rho || !a->d_scal ||
        !a->d_bottom)
        return tb_fail(ctx, TB_ERR_ARG, "%s: incomplete adjoint arguments", who);
    if ((a->d_rE && a->n_energy < 1) || (a->d_rA && a->n_angle < 1))
        return tb_fail(ctx, TB_ERR_ARG, "%s: reweighting factors for an empty table", who);
    if (a->n_basis < 0 || (a->n_basis > 0 && (!a->d_basis || !a->d_resp_i || !a->d_resp_e || !a->d_resp_index)))
        return tb_fail(ctx, TB_ERR_ARG, "%s: incomplete field-feedback arguments", who);
    return TB_OK;
}

}  // namespace

extern "C" int tb_tally(tb_ctx *ctx, const tb_tally_args *a, void *stream) {
    if (!ctx || !a) return TB_ERR_ARG;
    if (a->n_species < 0 || a->m < 1 || a->n_energy < 0 || a->n_angle < 0 || !a->d_table || !a->d_slot)
        return tb_fail(ctx, TB_ERR_ARG, "tb_tally: invalid arguments");
    if (a->n_species == 0) return TB_OK;
    if (!a->d_status || !a->d_hit || (a->n_energy > 0 && !a->d_bin_e) || (a->n_angle > 0 && !a->d_bin_a))
        return tb_fail(ctx, TB_ERR_ARG, "tb_tally: a particle array is missing");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    const long long total = 2 * a->n_species;
    k_tally<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a, ctx->nx * ctx->ny, ctx->d_err);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

extern "C" int tb_adjoint_forward(tb_ctx *ctx, const tb_step_desc *d, const tb_adjoint_args *a, void *stream) {
    if (!ctx || !d || !a) return TB_ERR_ARG;
    int rc = check_step(ctx, d, a, "tb_adjoint_forward");
    if (rc != TB_OK) return rc;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int wpb = 8, blocks = (d->m + wpb - 1) / wpb;
    for (int b = 0; b < a->n_batches; ++b) {
        k_fwd_deposit<<<1, ONE_BLOCK, 0, s>>>(*d, *a, b);
        if (d->d_leak_M)
            k_gemv<double><<<blocks, 32 * wpb, 0, s>>>(d->m, d->m, d->d_leak_M, d->d_work, d->d_work + d->m, 0);
        k_fwd_finish<<<1, ONE_BLOCK, 0, s>>>(*d, *a, b);
    }
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

extern "C" int tb_adjoint_reverse(tb_ctx *ctx, const tb_step_desc *d, const tb_adjoint_args *a, double *d_lambda,
                                  const double *d_gbottom, double *d_grad, double *d_scratch, void *stream) {
    if (!ctx || !d || !a) return TB_ERR_ARG;
    int rc = check_step(ctx, d, a, "tb_adjoint_reverse");
    if (rc != TB_OK) return rc;
    if (!d_lambda || !d_scratch || (a->n_energy + a->n_angle > 0 && !d_grad))
        return tb_fail(ctx, TB_ERR_ARG, "tb_adjoint_reverse: lambda, grad and scratch are required");
    if (d->d_leak_M && !a->d_leak_MT)
        return tb_fail(ctx, TB_ERR_ARG, "tb_adjoint_reverse: leakage needs the transposed operator");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int wpb = 8, blocks = (d->m + wpb - 1) / wpb;
    const int rows = a->n_energy + a->n_angle;
    const size_t per = (size_t)(rows + 2) * d->m;
    for (int b = a->n_batches - 1; b >= 0; --b) {
        k_rev_conductor<<<1, ONE_BLOCK, 0, s>>>(*d, *a, b, d_lambda, d_scratch);
        if (d->d_leak_M)
            k_gemv<double><<<blocks, 32 * wpb, 0, s>>>(d->m, d->m, a->d_leak_MT, d->d_work, d->d_work + d->m, 0);
        k_rev_deposit<<<1, ONE_BLOCK, 0, s>>>(*d, *a, b, d_lambda, d_gbottom, d_scratch);
        if (a->n_basis > 0) k_rev_feedback<<<1, ONE_BLOCK, 0, s>>>(*d, *a, b, d_lambda, d_scratch);
        if (rows > 0)
            k_gemv<int32_t><<<(rows + wpb - 1) / wpb, 32 * wpb, 0, s>>>(rows, d->m, a->d_tables + (size_t)b * per,
                                                                        d_scratch, d_grad, 1);
    }
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}
