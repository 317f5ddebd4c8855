// Device-side particle injection at the top boundary.
//
// Restates the sampling of the reference's `inject` (trench_charging_2d.py:458-489)
// on the GPU, so a batch needs no host-to-device particle copy:
//   ions       x ~ U(0, Lx); energy from a tabulated inverse CDF (or fixed),
//              polar angle from a tabulated inverse CDF (optionally with a random
//              sign) or a lateral thermal velocity N(0, sigma);
//              v = sqrt(2 E e / m_i), vx = v sin(theta), vy = -v cos(theta)
//   electrons  x ~ U(0, Lx); vx ~ N(0, s); vy = -s sqrt(-2 ln(1 - u)) (flux-weighted
//              Maxwellian, trench_charging_2d.py:478-481)
//   y = Ly - 1e-3 dx for all; qm = e/m_i or -e/m_e.
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), a counter-based generator: particle i of
// batch b uses counter (i, b_lo, b_hi, 0) and the 64-bit seed as key, so every
// particle's draws are independent of launch shape and order.
#include <math.h>

#include "tb_internal.cuh"

namespace {

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}

// Philox4x32 with 10 rounds; round constants from the SC'11 paper.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += W0; k1 += W1; }
        const uint32_t hi0 = mulhi32(M0, c[0]), lo0 = M0 * c[0];
        const uint32_t hi1 = mulhi32(M1, c[2]), lo1 = M1 * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

// (0, 1) open-interval double from 32 random bits
__device__ __forceinline__ double unit(uint32_t r) { return ((double)r + 0.5) * 2.3283064365386963e-10; }

// Inverse CDF of a histogram: cdf[0..nb] increasing from 0 to 1 over bin edges
// edges[0..nb]; linear within a bin.  *bin receives the bin drawn (a bin of zero
// weight is never drawn: the search ends on cdf[lo] <= u < cdf[lo + 1]).
__device__ double sample_table(const double *edges, const double *cdf, int nb, double u, int *bin) {
    int lo = 0, hi = nb;  // cdf[lo] <= u < cdf[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (cdf[mid] <= u) lo = mid; else hi = mid;
    }
    *bin = lo;
    const double w = cdf[hi] - cdf[lo];
    const double f = w > 0 ? (u - cdf[lo]) / w : 0.5;
    return edges[lo] + f * (edges[hi] - edges[lo]);
}

__global__ void k_inject(const tb_inject_args a) {
    const long long n = a.n_species;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n) return;
    const unsigned long long batch = a.batch + (a.d_counter ? (unsigned long long)(*a.d_counter + 1) : 0ull);
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(batch & 0xffffffffu), (uint32_t)(batch >> 32), (uint32_t)(i >> 32)};
    philox4x32_10(c, (uint32_t)(a.seed & 0xffffffffu), (uint32_t)(a.seed >> 32));
    const double u0 = unit(c[0]), u1 = unit(c[1]), u2 = unit(c[2]), u3 = unit(c[3]);
    double x = u0 * a.lx, vx, vy, qm;
    int8_t spc;
    if (i < n) {
        int be = 0, ba = 0;
        const double e = a.n_energy > 0 ? sample_table(a.d_energy_edges, a.d_energy_cdf, a.n_energy, u1, &be)
                                        : a.ion_energy_eV;
        if (a.d_bin_e) a.d_bin_e[i] = (uint16_t)be;
        const double v = sqrt(2.0 * fmax(e, 0.0) * a.e_charge / a.ion_mass);
        if (a.n_angle > 0) {
            double th = sample_table(a.d_angle_edges, a.d_angle_cdf, a.n_angle, u2, &ba);
            if (a.angle_random_sign && u3 < 0.5) th = -th;
            vx = v * sin(th);
            vy = -v * cos(th);
        } else {
            // lateral thermal velocity (Box-Muller)
            vx = a.ion_lateral_sigma * sqrt(-2.0 * log(u2)) * cos(6.283185307179586 * u3);
            vy = -v;
        }
        if (a.d_bin_a) a.d_bin_a[i] = (uint16_t)ba;
        qm = a.qm_ion;
        spc = 0;
    } else {
        const double s = a.electron_sigma;
        vx = s * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        vy = -s * sqrt(-2.0 * log(1.0 - u3));
        qm = a.qm_electron;
        spc = 1;
    }
    if (a.d_clock) {
        // stratified launch time: stratum k of the species' n, offset by a fifth draw
        // (counter word 3 with its top bit set, disjoint from the particle counters)
        uint32_t d[4] = {(uint32_t)i, (uint32_t)(batch & 0xffffffffu), (uint32_t)(batch >> 32),
                         (uint32_t)(i >> 32) | 0x80000000u};
        philox4x32_10(d, (uint32_t)(a.seed & 0xffffffffu), (uint32_t)(a.seed >> 32));
        const long long k = i < n ? i : i - n;
        const double t = ((double)k + unit(d[0])) * a.period / (double)n;
        a.d_clock[2 * i] = t < a.period ? t : 0.0;
        a.d_clock[2 * i + 1] = 0.0;
    }
    a.d_x[i] = x;
    a.d_y[i] = a.y0;
    a.d_vx[i] = vx;
    a.d_vy[i] = vy;
    a.d_qm[i] = qm;
    a.d_spc[i] = spc;
}

__global__ void k_philox(unsigned long long seed, unsigned long long batch, int n, uint32_t *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(batch & 0xffffffffu), (uint32_t)(batch >> 32), 0u};
    philox4x32_10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
    for (int k = 0; k < 4; ++k) out[4 * i + k] = c[k];
}

}  // namespace

extern "C" int tb_inject(tb_ctx *ctx, const tb_inject_args *a, void *stream) {
    if (!ctx || !a) return TB_ERR_ARG;
    if (a->n_species < 0 || !a->d_x || !a->d_y || !a->d_vx || !a->d_vy || !a->d_qm || !a->d_spc ||
        !(a->lx > 0) || !(a->ion_mass > 0) || !(a->electron_sigma >= 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_inject: invalid arguments");
    if ((a->n_energy > 0 && (!a->d_energy_edges || !a->d_energy_cdf)) ||
        (a->n_angle > 0 && (!a->d_angle_edges || !a->d_angle_cdf)))
        return tb_fail(ctx, TB_ERR_ARG, "tb_inject: a sampling table is missing");
    if (a->d_clock && !(a->period > 0))
        return tb_fail(ctx, TB_ERR_ARG, "tb_inject: RF launch times need a positive period");
    if (a->n_energy > 65536 || a->n_angle > 65536)
        return tb_fail(ctx, TB_ERR_ARG, "tb_inject: a table has more than 65536 bins");
    if (a->n_species == 0) return TB_OK;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    const long long total = 2 * a->n_species;
    k_inject<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}

extern "C" int tb_philox_fill(tb_ctx *ctx, unsigned long long seed, unsigned long long batch, int n,
                              uint32_t *d_out, void *stream) {
    if (!ctx || n < 0 || (n > 0 && !d_out)) return TB_ERR_ARG;
    if (n == 0) return TB_OK;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    k_philox<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(seed, batch, n, d_out);
    TB_CUDA(ctx, cudaGetLastError());
    return TB_OK;
}
