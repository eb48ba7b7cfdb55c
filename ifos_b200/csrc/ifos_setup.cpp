// Host-side set-up of the propagation path.  See ifos_setup.h.
#include "ifos_setup.h"

#include <cmath>
#include <cstdint>
#include <cstdlib>

namespace ifos {

static const double kPi = 3.141592653589793;

// Holberg (1987) group-velocity-optimised staggered weights for a maximum
// relative error of 0.1, 0.5, 1 and 3 percent (MAXRELERROR 1..4); the same
// published values the reference tabulates (src/holbergcoeff.c:51-84).
static const double kHolberg[4][6][6] = {
    {{1.0010}, {1.1382, -0.046414}, {1.1965, -0.078804, 0.0081781},
     {1.2257, -0.099537, 0.018063, -0.0026274}, {1.2415, -0.11231, 0.026191, -0.0064682, 0.001191},
     {1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
    {{1.0050}, {1.1534, -0.052806}, {1.2111, -0.088313, 0.011768},
     {1.2367, -0.10815, 0.023113, -0.0046905}, {1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161},
     {1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
    {{1.0100}, {1.1640, -0.057991}, {1.2192, -0.094070, 0.014608},
     {1.2422, -0.11269, 0.026140, -0.0064054}, {1.2534, -0.12257, 0.033755, -0.011081, 0.0036784},
     {1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
    {{1.0300}, {1.1876, -0.072518}, {1.2341, -0.10569, 0.022589},
     {1.2516, -0.12085, 0.032236, -0.011459}, {1.2596, -0.12829, 0.038533, -0.014681, 0.0072580},
     {1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}},
};
// The reference's leading column (grid points per wavelength), hc[0].
static const double kPpw[5][6] = {{23.0, 8.0, 6.0, 5.0, 5.0, 4.0},
                                  {49.7, 8.32, 4.77, 3.69, 3.19, 2.91},
                                  {22.2, 5.65, 3.74, 3.11, 2.80, 2.62},
                                  {15.8, 4.80, 3.39, 2.90, 2.65, 2.51},
                                  {9.16, 3.47, 2.91, 2.61, 2.45, 2.36}};

static int64_t gcd64(int64_t a, int64_t b) {
    if (a < 0) a = -a;
    if (b < 0) b = -b;
    while (b) {
        int64_t t = a % b;
        a = b;
        b = t;
    }
    return a ? a : 1;
}

// Taylor weights of the 2M-th order staggered first derivative, exactly as a
// rational number: c_m = 1/(2m-1) * prod_{k != m} (2k-1)^2 / ((2k-1)^2 - (2m-1)^2).
static double taylor_weight(int M, int m) {
    int64_t num = 1, den = 2 * m - 1;
    for (int k = 1; k <= M; k++) {
        if (k == m) continue;
        int64_t a = (int64_t)(2 * k - 1) * (2 * k - 1);
        int64_t b = a - (int64_t)(2 * m - 1) * (2 * m - 1);
        num *= a;
        den *= b;
        int64_t g = gcd64(num, den);
        num /= g;
        den /= g;
    }
    return (double)num / (double)den;
}

bool fd_coefficients(int fdorder, int maxrelerror, float hc[7]) {
    if (fdorder < 2 || fdorder > 12 || (fdorder & 1) || maxrelerror < 0 || maxrelerror > 4) return false;
    int M = fdorder / 2;
    for (int k = 0; k < 7; k++) hc[k] = 0.0f;
    hc[0] = (float)kPpw[maxrelerror][M - 1];
    for (int m = 1; m <= M; m++)
        hc[m] = (float)(maxrelerror == 0 ? taylor_weight(M, m) : kHolberg[maxrelerror - 1][M - 1][m - 1]);
    return true;
}

// One side of the CPML profile set (src/PML_pro.c:117-221 for x, :226-313 for
// y), arrays 1-based at h = i - base.  The reference tests `abs(d) > 1e-6`
// with the integer abs(), i.e. (int)d != 0.
static void cpml_side(const ifos_params &p, float d0, float d0_half, float thick, float origin, int lo, int hi,
                      int base, bool from_left, bool clamp_alpha, float amax, float *K, float *a, float *b,
                      float *Kh, float *ah, float *bh) {
    const float DH = p.dh, DT = p.dt, npw = p.npower, kmax = p.k_max_pml;
    for (int i = lo; i <= hi; i++) {
        const int h = i - base;
        float d = 0.0f, dh = 0.0f, al = 0.0f, alh = 0.0f;
        K[h] = 1.0f;
        Kh[h] = 1.0f;
        const float x = DH * (i - 1);
        float absc = from_left ? origin - x : x - origin;
        if (absc >= 0.0) {
            float nrm = absc / thick;
            d = d0 * std::pow((double)nrm, (double)npw);
            K[h] = 1.0 + (kmax - 1.0) * std::pow((double)nrm, (double)npw);
            al = amax * (1.0 - nrm);
        }
        absc = from_left ? origin - (x + DH / 2.0) : x + DH / 2.0 - origin;
        if (absc >= 0.0) {
            float nrm = absc / thick;
            dh = d0_half * std::pow((double)nrm, (double)npw);
            Kh[h] = 1.0 + (kmax - 1.0) * std::pow((double)nrm, (double)npw);
            alh = amax * (1.0 - nrm);
        }
        if (clamp_alpha) {
            if (al < 0.0) al = 0.0;
            if (alh < 0.0) alh = 0.0;
        }
        b[h] = std::exp((double)(-(d / K[h] + al) * DT));
        bh[h] = std::exp((double)(-(dh / Kh[h] + alh) * DT));
        a[h] = 0.0f;
        ah[h] = 0.0f;
        if ((int)d != 0) a[h] = d * (b[h] - 1.0) / (K[h] * (d + K[h] * al));
        if ((int)dh != 0) ah[h] = dh * (bh[h] - 1.0) / (Kh[h] * (dh + Kh[h] * alh));
    }
}

CpmlProfiles cpml_profiles(const ifos_params &p) {
    CpmlProfiles pr;
    pr.n = 2 * p.fw;
    for (auto &v : pr.arr) v.assign((size_t)pr.n + 1, 0.0f);
    if (p.fw <= 0) return pr;
    const float thick = p.fw * p.dh;
    const float rc = 0.001f;
    const float d0 = -(p.npower + 1) * p.vppml * std::log((double)rc) / (2.0 * thick);
    const float amax = 2.0 * kPi * (p.fpml / 2.0);
    float *A[12];
    for (int k = 0; k < 12; k++) A[k] = pr.arr[k].data();
    const float xr = (p.nx - 1) * p.dh - thick, yb = (p.ny - 1) * p.dh - thick;
    cpml_side(p, d0, d0, thick, thick, 1, p.fw, 0, true, true, amax, A[0], A[1], A[2], A[3], A[4], A[5]);
    cpml_side(p, d0, d0, thick, xr, p.nx - p.fw + 1, p.nx, p.nx - 2 * p.fw, false, true, amax, A[0], A[1], A[2],
              A[3], A[4], A[5]);
    cpml_side(p, d0, d0, thick, thick, 1, p.fw, 0, true, false, amax, A[6], A[7], A[8], A[9], A[10], A[11]);
    cpml_side(p, d0, d0, thick, yb, p.ny - p.fw + 1, p.ny, p.ny - 2 * p.fw, false, false, amax, A[6], A[7], A[8],
              A[9], A[10], A[11]);
    return pr;
}

ViscoScalars visco_scalars(const ifos_params &p) {
    ViscoScalars v{};
    float pts[IFOS_MAX_L + 1] = {0};
    for (int l = 1; l <= p.L; l++) {
        pts[l] = 1.0 / (2.0 * kPi * p.fl[l - 1]);  // src/readmod.c:44-49
        v.eta[l] = p.dt / pts[l];
    }
    const float ws = 2.0 * kPi * p.f_ref;  // src/prepare_update_s.c:38-45
    float su = 0.0f, sp = 0.0f;
    for (int l = 1; l <= p.L; l++) {
        su = su + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        sp = sp + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
    }
    v.sumu = su;
    v.sumpi = sp;
    for (int l = 1; l <= p.L; l++) {
        v.bip[l] = 1.0 / (1.0 + (v.eta[l] * 0.5));
        v.bjm[l] = 1.0 / (1.0 + (v.eta[l] * 0.5));
        v.cip[l] = 1.0 - (v.eta[l] * 0.5);
        v.cjm[l] = 1.0 - (v.eta[l] * 0.5);
        v.bjm_srf[l] = v.eta[l] / (1.0 + (v.eta[l] * 0.5));  // src/surface_PML.c:150
    }
    return v;
}

bool build_model(const ifos_params &p, const float *vp, const float *vs, const float *rho, const float *taup,
                 const float *taus, ModelPlanes &o) {
    const int NX = p.nx, NY = p.ny;
    const size_t N = (size_t)NX * NY;
    if (!vp || !rho || (!p.acoustic && !vs)) return false;
    // ghost-ring view: one rank's periodic copy of rows 1/NY and columns 1/NX
    // into rows 0/NY+1 and columns 0/NX+1 (src/matcopy_elastic.c:59-141)
    auto gi = [&](int j, int i) -> size_t {
        if (j == 0) j = NY;
        if (j == NY + 1) j = 1;
        if (i == 0) i = NX;
        if (i == NX + 1) i = 1;
        return (size_t)(j - 1) * NX + (i - 1);
    };
    o.rho.assign(rho, rho + N);
    o.vp.assign(vp, vp + N);
    o.vs.assign(N, 0.0f);
    if (!p.acoustic) o.vs.assign(vs, vs + N);
    const float *R = o.rho.data(), *U = o.vs.data(), *PI = o.vp.data();
    o.rip.resize(N);
    o.rjp.resize(N);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {  // src/av_rho.c:26-33
            size_t k = gi(j, i);
            o.rjp[k] = 1.0 / (0.5 * (R[k] + R[gi(j + 1, i)]));
            o.rip[k] = 1.0 / (0.5 * (R[k] + R[gi(j, i + 1)]));
        }
    if (p.acoustic) {
        o.g_ac.resize(N);
        for (size_t k = 0; k < N; k++) o.g_ac[k] = R[k] * (PI[k] * PI[k]);  // src/update_p_PML.c:98
        if (!p.L) return true;
        // viscoacoustic (src/prepare_update_p.c:44-64): the relaxed modulus pi
        // and g = pi*DT*(1+L*taup); e_l = pi*eta_l*taup is formed in the kernels
        const ViscoScalars vs_ = visco_scalars(p);
        std::vector<float> tp(N);
        for (size_t k = 0; k < N; k++) tp[k] = taup ? taup[k] : p.tau;
        o.g_v.resize(N);
        o.pi_r.resize(N);
        for (size_t k = 0; k < N; k++) {
            float pi = (PI[k] * PI[k] * R[k]) / (1.0 + vs_.sumpi * tp[k]);
            o.g_v[k] = pi * p.dt * (1.0 + p.L * tp[k]);
            o.pi_r[k] = pi;
        }
        o.tau_uniform = true;
        for (size_t k = 1; k < N && o.tau_uniform; k++)
            if (tp[k] != tp[0]) o.tau_uniform = false;
        o.taus0 = o.tausipjp0 = 0.0f;
        o.taup0 = tp[0];
        if (!o.tau_uniform) o.taup = tp;
        return true;
    }
    // PARAMETERIZATION 3: PI and U hold lambda and mu themselves; the
    // reference's correlation weights (mm, ll) keep their vp/vs form under
    // both parameterizations (src/IFOS2D.c:2395-2396 has no branch)
    const bool lame = p.parameterization == 3;
    o.uipjp.resize(N);
    o.f_el.resize(N);
    o.g_el.resize(N);
    o.mm.resize(N);
    o.ll.resize(N);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {  // src/av_mue.c:28-61
            size_t k = gi(j, i), k2 = gi(j, i + 1), k3 = gi(j + 1, i), k4 = gi(j + 1, i + 1);
            float u1 = lame ? U[k] : R[k] * U[k] * U[k];
            float u2 = lame ? U[k2] : R[k2] * U[k2] * U[k2];
            float u3 = lame ? U[k3] : R[k3] * U[k3] * U[k3];
            float u4 = lame ? U[k4] : R[k4] * U[k4] * U[k4];
            float v = 4.0 / ((1.0 / u1) + (1.0 / u2) + (1.0 / u3) + (1.0 / u4));
            if ((u1 == 0.0) || (u2 == 0.0) || (u3 == 0.0) || (u4 == 0.0)) v = 0.0;
            o.uipjp[k] = v;
        }
    for (size_t k = 0; k < N; k++) {
        // src/update_s_elastic_PML.c:224-230 (and the SH update's f)
        o.f_el[k] = lame ? U[k] : R[k] * U[k] * U[k];
        o.g_el[k] = lame ? PI[k] : R[k] * ((PI[k] * PI[k]) - 2 * U[k] * U[k]);
        float muss = R[k] * U[k] * U[k];  // src/IFOS2D.c:2395-2396
        float lamss = R[k] * PI[k] * PI[k] - 2.0 * muss;
        o.mm[k] = (U[k] > 0.0) ? muss * muss : 0.0f;
        o.ll[k] = (lamss + muss) * (lamss + muss);
    }
    // free-surface row coefficients, elastic (src/surface_elastic_PML.c:94-100)
    o.srf_fjm.resize(NX);
    o.srf_g.resize(NX);
    for (int i = 0; i < NX; i++) {
        o.srf_fjm[i] = lame ? U[i] * 2.0 : R[i] * U[i] * U[i] * 2.0;
        o.srf_g[i] = lame ? PI[i] : R[i] * ((PI[i] * PI[i]) - 2 * U[i] * U[i]);
    }
    if (!p.L) return true;

    ViscoScalars vs_ = visco_scalars(p);
    std::vector<float> ts(N), tp(N), tsij(N);
    for (size_t k = 0; k < N; k++) {
        ts[k] = taus ? taus[k] : p.tau;
        tp[k] = taup ? taup[k] : p.tau;
    }
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++)  // src/av_tau.c:25-29
            tsij[gi(j, i)] = 0.25 * (ts[gi(j, i)] + ts[gi(j, i + 1)] + ts[gi(j + 1, i)] + ts[gi(j + 1, i + 1)]);
    o.fipjp_v.resize(N);
    o.f_v.resize(N);
    o.g_v.resize(N);
    o.mu_r.resize(N);
    o.pi_r.resize(N);
    o.muipjp_r.resize(N);
    const float DT = p.dt;
    const int L = p.L;
    for (size_t k = 0; k < N; k++) {  // src/prepare_update_s.c:60-93
        float mu = lame ? U[k] / (1.0 + vs_.sumu * ts[k]) : (U[k] * U[k] * R[k]) / (1.0 + vs_.sumu * ts[k]);
        float pi = lame ? (PI[k] + 2 * U[k]) / (1.0 + vs_.sumpi * tp[k])
                        : (PI[k] * PI[k] * R[k]) / (1.0 + vs_.sumpi * tp[k]);
        float muipjp = o.uipjp[k] / (1.0 + vs_.sumu * tsij[k]);
        o.fipjp_v[k] = muipjp * DT * (1.0 + L * tsij[k]);
        o.f_v[k] = mu * DT * (1.0 + L * ts[k]);
        o.g_v[k] = pi * DT * (1.0 + L * tp[k]);
        o.mu_r[k] = mu;
        o.pi_r[k] = pi;
        o.muipjp_r[k] = muipjp;
    }
    o.tau_uniform = true;
    for (size_t k = 1; k < N && o.tau_uniform; k++)
        if (ts[k] != ts[0] || tp[k] != tp[0] || tsij[k] != tsij[0]) o.tau_uniform = false;
    o.taus0 = ts[0];
    o.taup0 = tp[0];
    o.tausipjp0 = tsij[0];
    if (!o.tau_uniform) {
        o.taus = ts;
        o.taup = tp;
        o.tausipjp = tsij;
    }
    // visco free-surface row (src/surface_PML.c:125-147)
    o.srf_djm.resize(NX);
    o.srf_e.resize(NX);
    for (int i = 0; i < NX; i++) {
        float mu = lame ? U[i] / (1.0 + vs_.sumu * ts[i]) : (U[i] * U[i] * R[i]) / (1.0 + vs_.sumu * ts[i]);
        float pi = lame ? (PI[i] + 2 * U[i]) / (1.0 + vs_.sumpi * tp[i])
                        : (PI[i] * PI[i] * R[i]) / (1.0 + vs_.sumpi * tp[i]);
        o.srf_fjm[i] = mu * 2.0 * (1.0 + L * ts[i]);
        o.srf_g[i] = pi * (1.0 + L * tp[i]);
        o.srf_djm[i] = 2.0 * mu * ts[i];
        o.srf_e[i] = pi * tp[i];
    }
    return true;
}

}  // namespace ifos
