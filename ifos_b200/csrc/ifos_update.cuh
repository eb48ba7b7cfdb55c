// Model update of the step-length search (src/calc_mat_change_test.c:26-334):
// the test model of a trial step, or the accepted update, on the device.
#pragma once

#include <cuda_runtime.h>

namespace ifos {

// Parameters of one update (the reference's globals and arguments).
struct KMatChange {
    long long n;      // NX*NY
    int nx, ny;
    int acoustic;
    float eps_scale;
    int iter, itest;
    int inv_vp_iter, inv_vs_iter, inv_rho_iter;
    int lbfgs_unnormalised;
    float vp_lower, vp_upper, vs_lower, vs_upper, rho_lower, rho_upper;
    float vp_vs_ratio;
    int limit_update;
    float s_vp, s_vs, s_rho;
    int lbfgs_npar;
    float vs_avg, rho_avg, vp_avg;
};

// Bits of a non-negative float, whose order is that of the unsigned ints.
__device__ __forceinline__ unsigned pos_bits(float v) { return v > 0.0f ? __float_as_uint(v) : 0u; }

// The six maxima of src/calc_mat_change_test.c:80-139 into mx[0..5]:
// max(0, vp), max|g_vp|, max(0, vs), max|g_vs|, max(0, rho), max|g_rho|
// (mx zeroed by the caller; the reference's running maxima start at 0 and
// its gradient maximum restarts from |g| while it is still 0, which for
// finite values is the plain maximum).
__global__ void k_mc_maxima(KMatChange m, const float *vp, const float *gvp, const float *vs, const float *gvs,
                            const float *rho, const float *grho, unsigned *mx) {
    unsigned a[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m.n;
         k += (long long)gridDim.x * blockDim.x) {
        a[0] = max(a[0], pos_bits(vp[k]));
        a[1] = max(a[1], pos_bits(fabsf(gvp[k])));
        if (!m.acoustic) {
            a[2] = max(a[2], pos_bits(vs[k]));
            a[3] = max(a[3], pos_bits(fabsf(gvs[k])));
        }
        a[4] = max(a[4], pos_bits(rho[k]));
        a[5] = max(a[5], pos_bits(fabsf(grho[k])));
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const unsigned w = __reduce_max_sync(0xffffffffu, a[q]);
        if ((threadIdx.x & 31) == 0 && w) atomicMax(mx + q, w);
    }
}

// EPSILON of one parameter (src/calc_mat_change_test.c:144-211): the scaled
// ratio of the maxima, zero before the parameter's first iteration, and
// eps_scale itself under unnormalised L-BFGS steps.
__device__ __forceinline__ float mc_step(const KMatChange &m, unsigned mmax, unsigned gmax, int inv_iter) {
    float e = m.eps_scale * (__uint_as_float(mmax) / __uint_as_float(gmax));
    if (m.iter < inv_iter) e = 0.0f;
    if (m.lbfgs_unnormalised) {
        e = m.eps_scale;
        if (m.iter < inv_iter) e = 0.0f;
    }
    return e;
}

// A limited update (src/calc_mat_change_test.c:265-289): the change relative
// to the start model, in percent, is held to `lim`.
__device__ __forceinline__ float mc_limit(float start, float v, float lim) {
    const float pro = (float)((double)((start - v) / start) * 100.0);
    if ((fabs((double)pro) > (double)lim) && ((double)pro > 0.0))
        v = (float)((double)start - (double)(start * lim) / 100.0);
    if ((fabs((double)pro) > (double)lim) && ((double)pro < 0.0))
        v = (float)((double)start + (double)(start * lim) / 100.0);
    return v;
}

// One cell of the update loop (src/calc_mat_change_test.c:223-330) in the
// reference's order of rules; k is the row-major cell, l the reference's
// column-major running index of the L-BFGS difference vectors.
__global__ void k_mc_update(KMatChange m, const unsigned *mx, float *vp, float *vs, float *rho, const float *gvp,
                            const float *gvs, const float *grho, const float *vp0, const float *vs0,
                            const float *rho0, float *vp1, float *vs1, float *rho1, float *s, float *eps_out,
                            int *ratio_hit) {
    const float e_vp = mc_step(m, mx[0], mx[1], m.inv_vp_iter);
    const float e_vs = m.acoustic ? 0.0f : mc_step(m, mx[2], mx[3], m.inv_vs_iter);
    const float e_rho = mc_step(m, mx[4], mx[5], m.inv_rho_iter);
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k == 0) {
        eps_out[0] = e_vp;
        eps_out[1] = e_vs;
        eps_out[2] = e_rho;
    }
    if (k >= m.n) return;
    const float pi = vp[k], r = rho[k], u = m.acoustic ? 0.0f : vs[k];
    float pn = pi - e_vp * gvp[k];
    float un = m.acoustic ? 0.0f : u - e_vs * gvs[k];
    float rn = r - e_rho * grho[k];
    if (pn < m.vp_lower) pn = m.vp_lower;
    if (pn > m.vp_upper) pn = m.vp_upper;
    if (!m.acoustic) {
        if ((un < m.vs_lower) && ((double)un > 1e-6)) un = m.vs_lower;
        if (un > m.vs_upper) un = u;
        if (m.vp_vs_ratio > 1) {  // the Poisson-ratio check
            if ((pn / un) < m.vp_vs_ratio) {
                pn = un * m.vp_vs_ratio;
                atomicOr(ratio_hit, 1);
            }
        }
    }
    if (m.limit_update == 1) {
        if (!m.acoustic) un = mc_limit(vs0[k], un, m.s_vs);
        pn = mc_limit(vp0[k], pn, m.s_vp);
        rn = mc_limit(rho0[k], rn, m.s_rho);
    }
    if ((rn < m.rho_lower) && (m.inv_rho_iter < m.iter)) rn = r;
    if ((rn > m.rho_upper) && (m.inv_rho_iter < m.iter)) rn = r;
    if ((double)pn < 0.0) pn = pi;
    if (!m.acoustic && (double)un < 0.0) un = u;
    if ((double)rn < 0.0) rn = r;
    vp1[k] = pn;
    if (!m.acoustic) vs1[k] = un;
    rho1[k] = rn;
    if (m.itest == 0) {
        if (s && m.lbfgs_npar > 0) {
            const long long j = k / m.nx, i = k % m.nx, l = i * m.ny + j;
            if (!m.acoustic) s[l] = (un - u) / m.vs_avg;
            if (m.lbfgs_npar > 1) s[m.n + l] = (rn - r) / m.rho_avg;
            if (m.lbfgs_npar > 2) s[2 * m.n + l] = (pn - pi) / m.vp_avg;
        }
        if (!m.acoustic) vs[k] = un;
        rho[k] = rn;
        vp[k] = pn;
    }
}

}  // namespace ifos
