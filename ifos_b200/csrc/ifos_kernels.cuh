// Device kernels of the shot solver.
//
// Every kernel covers all shot slots of a context (blockIdx.z = slot), so a
// single shot and a batch of shots run the same code.  The per-cell arithmetic
// keeps the operation order and the float/double promotions of the
// reference's kernels (cited per function); the library is compiled with
// --fmad=false, so in fp32 mode each cell update rounds exactly as the
// reference's C code does.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ifos {

// Programmatic dependent launch.  pdl_wait: block until the preceding kernel
// of the stream has completed and its writes are visible (a no-op when this
// kernel was not launched as a dependent); pdl_launch: let the next kernel
// of the stream start its blocks before this one has finished.  Every kernel
// the solver launches as a dependent calls pdl_wait before it touches memory
// the preceding kernels write, and pdl_launch only after that wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// halo around every state plane (>= FDORDER/2 + 1 for FDORDER 12)
constexpr int HX = 8;
constexpr int HY = 8;

// state plane ids
enum : int {
    P_VX = 0, P_VY, P_SXX, P_SYY, P_SXY, P_VXP1, P_VYP1, P_VZ, P_SXZ, P_SYZ, P_VZP1, P_SP, NP_FIELD
};
// model plane ids
enum : int {
    M_RHO = 0, M_VP, M_VS, M_RIP, M_RJP, M_UIPJP, M_F, M_G, M_GAC, M_FIPJPV, M_FV, M_GV, M_MUR, M_PIR,
    M_MUIPJPR, M_TAUS, M_TAUP, M_TAUSIPJP, M_MM, M_LL, NM_PLANE
};
// CPML strip ids: x strips (NY x 2FW), y strips (2FW x NX)
enum : int { X_SXX = 0, X_SXY, X_VXX, X_VYX, X_VXXS, X_SXZ, X_VZX, NX_STRIP };
enum : int { Y_SYY = 0, Y_SXY, Y_VYY, Y_VXY, Y_SYZ, Y_VZY, NY_STRIP };
// profile ids (arrays of 2FW+1, 1-based)
enum : int { K_X = 0, A_X, B_X, K_XH, A_XH, B_XH, K_Y, A_Y, B_Y, K_YH, A_YH, B_YH };

struct KGrid {
    int nx, ny, pitch, fw, free_surf, boundary, fdoh, L, quirk_hi, nt_total;
    long long plane;  // elements per state/model plane
    float dt, dh;
    float hc[7];
    float eta[9], bip[9], bjm[9], cip[9], cjm[9], bjm_srf[9];
    float taus0, taup0, tausipjp0;  // used when the tau planes are absent
    int adjoint_type;
    int k_one;       // every CPML K profile value is 1: d/K == d exactly
    int dh_pow2;     // DH is a power of two: x/DH == x*inv_dh exactly
    float inv_dh;    // 1/DH (exact when dh_pow2)
    int tile_order;  // pipelined stencils: 0 slot-major tile sequence, 1 slot-minor
    int prod_polls;  // pipelined stencils: polls of the producer's stage-release wait (0: the default limit)
    int mu_fix;      // the mu correlation with the corrected grouping (ifos_params.mu_corrected)
    int lame;        // PARAMETERIZATION 3: the model planes hold lambda and mu, the assembly stops at the moduli
};

// x / DH, exact in both branches: multiplying by the reciprocal of a power of
// two rounds exactly as the division does.
template <typename T>
__device__ __forceinline__ T div_dh(const KGrid &g, T x) {
    return g.dh_pow2 ? x * (T)g.inv_dh : x / (T)g.dh;
}

template <typename T>
struct KState {
    T *base;                  // slot 0
    long long slot_stride;    // elements between slots
    long long off[NP_FIELD];  // plane offsets within a slot (-1 absent)
    long long mem_off[5];     // first plane of r,p,q,t,o (L planes each), -1 absent
    T *psix[NX_STRIP];        // slot 0 strip, NY x 2FW each
    T *psiy[NY_STRIP];        // slot 0 strip, 2FW x NX each
    long long psix_slot, psiy_slot;  // elements between slots of one strip
};

template <typename T>
struct KModel {
    const T *m[NM_PLANE];  // model 0 planes (NULL absent)
    long long model_stride;
    const int *slot_model;  // model index of every slot
    const T *prof;          // 12 x (2FW+1)
    const T *srf;           // 4 x NX per model: fjm, g, djm, e (row j=1)
    long long srf_stride;
};

__host__ __device__ inline long long pidx(const KGrid &g, int j, int i) {
    return (long long)(j - 1 + HY) * g.pitch + (i - 1 + HX);
}

template <typename T>
__device__ inline T *fieldp(const KState<T> &s, int slot, int id) {
    return s.base + slot * s.slot_stride + s.off[id];
}
template <typename T>
__device__ inline T *memp(const KState<T> &s, const KGrid &g, int slot, int which, int l /*1-based*/) {
    return s.base + slot * s.slot_stride + s.mem_off[which] + (long long)(l - 1) * g.plane;
}
template <typename T>
__device__ inline const T *modelp(const KModel<T> &m, int slot, int id) {
    return m.m[id] ? m.m[id] + (long long)m.slot_model[slot] * m.model_stride : nullptr;
}
template <typename T>
__device__ inline T prof(const KModel<T> &m, const KGrid &g, int which, int h) {
    return m.prof[which * (2 * g.fw + 1) + h];
}

// Running sum of the FD taps: the m=1 term starts the sum, as in the
// reference's written-out expressions (src/update_v_PML.c:164-175); with z0
// it is added to zero, as in its generic loops (the FDORDER 10/12 default
// branches of src/update_v_acoustic_PML.c, src/update_p_PML.c and
// src/update_s_visc_PML.c).  The two differ only in the sign of a zero sum.
template <typename T>
__device__ __forceinline__ T tap(int m, T s, T t, bool z0 = false) {
    return (m == 1 && !z0) ? t : s + t;
}

// IEEE round-to-nearest division (what `/` compiles to) that the compiler
// may not hoist out of the branch it is written in: a speculated division of
// a zero or tiny dividend (the CPML strips before the wavefield reaches
// them) takes its slow path even when its result is not used.
__device__ __forceinline__ float div_rn_pinned(float x, float y) {
    float q;
    asm volatile("div.rn.f32 %0, %1, %2;" : "=f"(q) : "f"(x), "f"(y));
    return q;
}
__device__ __forceinline__ double div_rn_pinned(double x, double y) {
    double q;
    asm volatile("div.rn.f64 %0, %1, %2;" : "=d"(q) : "d"(x), "d"(y));
    return q;
}

// CPML recursion of every kernel: psi = b*psi + a*d; d = d/K + psi.  With
// every K equal to 1 (k_one) the quotient is d itself and no division runs.
template <typename T>
__device__ inline T cpml(T *psi, T b, T a, T K, T d, int k_one = 0) {
    const T ps = b * *psi + a * d;
    *psi = ps;
    if (k_one) return d + ps;
    return div_rn_pinned(d, K) + ps;
}

// CPML on precomputed strip indices (0: not in the strip): hx is the 1-based
// profile index of the x strip (left: i, right: i-NX+2FW), hy that of the y
// strip (top without free surface: j, bottom: j-NY+2FW).
__device__ __forceinline__ int strip_x(const KGrid &g, int i) {
    if (g.boundary || g.fw == 0) return 0;
    if (i <= g.fw) return i;
    if (i >= g.nx - g.fw + 1) return i - g.nx + 2 * g.fw;
    return 0;
}
__device__ __forceinline__ int strip_y(const KGrid &g, int j) {
    if (g.fw == 0) return 0;
    if (!g.free_surf && j <= g.fw) return j;
    if (j >= g.ny - g.fw + 1) return j - g.ny + 2 * g.fw;
    return 0;
}

// x strips (left: i<=FW, right: i>=NX-FW+1 at h1=i-NX+2FW), src/update_v_PML.c:177-200
template <typename T>
__device__ inline T cpml_x(const KGrid &g, const KModel<T> &M, T *strip, int j, int i, int kk, int ka, int kb,
                           T d) {
    const int n2 = 2 * g.fw;
    if (!g.boundary && i <= g.fw)
        d = cpml(strip + (long long)(j - 1) * n2 + (i - 1), prof(M, g, kb, i), prof(M, g, ka, i), prof(M, g, kk, i),
                 d);
    if (!g.boundary && i >= g.nx - g.fw + 1) {
        int h = i - g.nx + 2 * g.fw;
        d = cpml(strip + (long long)(j - 1) * n2 + (h - 1), prof(M, g, kb, h), prof(M, g, ka, h), prof(M, g, kk, h),
                 d);
    }
    return d;
}
// y strips (top only without free surface: j<=FW; bottom: j>=NY-FW+1 at h1=j-NY+2FW)
template <typename T>
__device__ inline T cpml_y(const KGrid &g, const KModel<T> &M, T *strip, int j, int i, int kk, int ka, int kb,
                           T d) {
    if (!g.free_surf && j <= g.fw)
        d = cpml(strip + (long long)(j - 1) * g.nx + (i - 1), prof(M, g, kb, j), prof(M, g, ka, j),
                 prof(M, g, kk, j), d);
    if (j >= g.ny - g.fw + 1) {
        int h = j - g.ny + 2 * g.fw;
        d = cpml(strip + (long long)(h - 1) * g.nx + (i - 1), prof(M, g, kb, h), prof(M, g, ka, h),
                 prof(M, g, kk, h), d);
    }
    return d;
}

// Reads of a stress plane above the free surface.  The reference mirrors
// syy, sxy (and syz, sp) into the ghost rows after every stress update
// (src/surface_elastic_PML.c:53-63: syy[1-m] = -syy[1+m], sxy[1-m] = -sxy[m]);
// here the velocity kernel reads the mirrored value directly.
template <typename T>
__device__ inline T ld_mirror_even(const KGrid &g, const T *f, int j, int i) {  // syy, syz, sp
    if (g.free_surf && j <= 0) return -f[pidx(g, 2 - j, i)];
    return f[pidx(g, j, i)];
}
template <typename T>
__device__ inline T ld_mirror_odd(const KGrid &g, const T *f, int j, int i) {  // sxy, sxz
    if (g.free_surf && j <= 0) return -f[pidx(g, 1 - j, i)];
    return f[pidx(g, j, i)];
}

// ---------------------------------------------------------------------------
// velocity half step, P-SV (src/update_v_PML.c:161-252; reference FDORDER
// 10/12 branches :466-528 when quirk_hi).  sw: 0 forward, 1 adjoint.
template <typename T, int FDOH>
__global__ void k_v_psv(KGrid g, KState<T> S, KModel<T> M, int sw, int want_p1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY), *sxy = fieldp(S, slot, P_SXY);
    T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    const long long c = pidx(g, j, i);
    const T rip = modelp(M, slot, M_RIP)[c], rjp = modelp(M, slot, M_RJP)[c];
    const T DT = g.dt, DH = g.dh;
    if (g.quirk_hi) {
        const T dtdh = DT * DT / DH;
        T ax = 0, ay = 0;
#pragma unroll
        for (int m = 1; m <= FDOH; m++) ax = tap(m, ax, (T)g.hc[m] * (sxx[pidx(g, j, i + m)] - sxx[pidx(g, j, i - m + 1)]));
#pragma unroll
        for (int m = 1; m <= FDOH; m++)
            ax += (T)g.hc[m] * (ld_mirror_odd(g, sxy, j + m - 1, i) - ld_mirror_odd(g, sxy, j - m, i));
#pragma unroll
        for (int m = 1; m <= FDOH; m++)
            ay = tap(m, ay, (T)g.hc[m] * (ld_mirror_even(g, syy, j + m, i) - ld_mirror_even(g, syy, j - m + 1, i)));
#pragma unroll
        for (int m = 1; m <= FDOH; m++) ay += (T)g.hc[m] * (sxy[pidx(g, j, i + m - 1)] - sxy[pidx(g, j, i - m)]);
        vx[c] += ax * dtdh * rip;
        vy[c] += ay * dtdh * rjp;
        return;
    }
    T sxx_x = 0, sxy_x = 0, sxy_y = 0, syy_y = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) sxx_x = tap(m, sxx_x, (T)g.hc[m] * (sxx[pidx(g, j, i + m)] - sxx[pidx(g, j, i - m + 1)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++) sxy_x = tap(m, sxy_x, (T)g.hc[m] * (sxy[pidx(g, j, i + m - 1)] - sxy[pidx(g, j, i - m)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++)
        sxy_y = tap(m, sxy_y, (T)g.hc[m] * (ld_mirror_odd(g, sxy, j + m - 1, i) - ld_mirror_odd(g, sxy, j - m, i)));
#pragma unroll
    for (int m = 1; m <= FDOH; m++)
        syy_y = tap(m, syy_y, (T)g.hc[m] * (ld_mirror_even(g, syy, j + m, i) - ld_mirror_even(g, syy, j - m + 1, i)));
    sxx_x = cpml_x(g, M, S.psix[X_SXX] + slot * S.psix_slot, j, i, K_XH, A_XH, B_XH, sxx_x);
    sxy_x = cpml_x(g, M, S.psix[X_SXY] + slot * S.psix_slot, j, i, K_X, A_X, B_X, sxy_x);
    syy_y = cpml_y(g, M, S.psiy[Y_SYY] + slot * S.psiy_slot, j, i, K_YH, A_YH, B_YH, syy_y);
    sxy_y = cpml_y(g, M, S.psiy[Y_SXY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, sxy_y);
    T *vxp1 = fieldp(S, slot, P_VXP1), *vyp1 = fieldp(S, slot, P_VYP1);
    if (sw == 0) {
        if (want_p1) {
            vxp1[c] = rip * (sxx_x + sxy_y) / DH;
            vyp1[c] = rjp * (sxy_x + syy_y) / DH;
        }
    } else {
        vxp1[c] += vx[c] * DT;
        vyp1[c] += vy[c] * DT;
    }
    vx[c] += DT * rip * (sxx_x + sxy_y) / DH;
    vy[c] += DT * rjp * (sxy_x + syy_y) / DH;
}

// velocity half step, SH (src/update_v_PML_SH.c:61-297, CPML on every order)
template <typename T, int FDOH>
__global__ void k_v_sh(KGrid g, KState<T> S, KModel<T> M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *sxz = fieldp(S, slot, P_SXZ), *syz = fieldp(S, slot, P_SYZ);
    T *vz = fieldp(S, slot, P_VZ), *vzp1 = fieldp(S, slot, P_VZP1);
    const long long c = pidx(g, j, i);
    const T rjp = modelp(M, slot, M_RJP)[c];
    const T DT = g.dt, DH = g.dh;
    T sxz_x = 0, syz_y = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) sxz_x = tap(m, sxz_x, (T)g.hc[m] * (sxz[pidx(g, j, i + m - 1)] - sxz[pidx(g, j, i - m)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++)
        syz_y = tap(m, syz_y, (T)g.hc[m] * (ld_mirror_even(g, syz, j + m, i) - ld_mirror_even(g, syz, j - m + 1, i)));
    sxz_x = cpml_x(g, M, S.psix[X_SXZ] + slot * S.psix_slot, j, i, K_X, A_X, B_X, sxz_x);
    syz_y = cpml_y(g, M, S.psiy[Y_SYZ] + slot * S.psiy_slot, j, i, K_YH, A_YH, B_YH, syz_y);
    vzp1[c] = vz[c];
    vz[c] += rjp * DT * (sxz_x + syz_y) / (DH);
}

// velocity half step, acoustic (src/update_v_acoustic_PML.c:72-148; the
// reference 10/12 default :396-409 when quirk_hi)
template <typename T, int FDOH>
__global__ void k_v_ac(KGrid g, KState<T> S, KModel<T> M, int sw, int want_p1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *sp = fieldp(S, slot, P_SP);
    T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    const long long c = pidx(g, j, i);
    const T rip = modelp(M, slot, M_RIP)[c], rjp = modelp(M, slot, M_RJP)[c];
    const T DT = g.dt, DH = g.dh;
    T sp_x = 0, sp_y = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) sp_x = tap(m, sp_x, (T)g.hc[m] * (sp[pidx(g, j, i + m)] - sp[pidx(g, j, i - m + 1)]), g.quirk_hi != 0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++)
        sp_y = tap(m, sp_y, (T)g.hc[m] * (ld_mirror_even(g, sp, j + m, i) - ld_mirror_even(g, sp, j - m + 1, i)), g.quirk_hi != 0);
    if (g.quirk_hi) {
        const T dtdh = DT * DT / DH;
        vx[c] += sp_x * dtdh * rip;
        vy[c] += sp_y * dtdh * rjp;
        return;
    }
    sp_x = cpml_x(g, M, S.psix[X_SXX] + slot * S.psix_slot, j, i, K_XH, A_XH, B_XH, sp_x);
    sp_y = cpml_y(g, M, S.psiy[Y_SYY] + slot * S.psiy_slot, j, i, K_YH, A_YH, B_YH, sp_y);
    T *vxp1 = fieldp(S, slot, P_VXP1), *vyp1 = fieldp(S, slot, P_VYP1);
    if (sw == 0) {
        if (want_p1) {
            vxp1[c] = rip * (sp_x) / DH;
            vyp1[c] = rjp * (sp_y) / DH;
        }
    } else {
        vxp1[c] += vx[c] * DT;
        vyp1[c] += vy[c] * DT;
    }
    vx[c] += DT * rip * (sp_x) / DH;
    vy[c] += DT * rjp * (sp_y) / DH;
}

// ---------------------------------------------------------------------------
// stress half step, P-SV elastic (src/update_s_elastic_PML.c:151-241; the
// reference 10/12 branches :442-535 when quirk_hi)
template <typename T, int FDOH>
__global__ void k_s_psv_el(KGrid g, KState<T> S, KModel<T> M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY), *sxy = fieldp(S, slot, P_SXY);
    const long long c = pidx(g, j, i);
    const T DT = g.dt, DH = g.dh;
    const T dhi = DT / DH;
    T vxx = 0, vyx = 0, vxy = 0, vyy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxx = tap(m, vxx, (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyx = tap(m, vyx, (T)g.hc[m] * (vy[pidx(g, j, i + m)] - vy[pidx(g, j, i - m + 1)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxy = tap(m, vxy, (T)g.hc[m] * (vx[pidx(g, j + m, i)] - vx[pidx(g, j - m + 1, i)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyy = tap(m, vyy, (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]));
    vxx = vxx * dhi;
    vyx = vyx * dhi;
    vxy = vxy * dhi;
    vyy = vyy * dhi;
    if (g.quirk_hi) {
        const T fipjp = modelp(M, slot, M_UIPJP)[c] * DT, f = modelp(M, slot, M_VS)[c] * DT,
                gg = modelp(M, slot, M_VP)[c] * DT;
        sxy[c] += (fipjp * (vxy + vyx));
        sxx[c] = (T)((double)sxx[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vyy)));
        syy[c] = (T)((double)syy[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vxx)));
        return;
    }
    vxx = cpml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, i, K_X, A_X, B_X, vxx);
    vyx = cpml_x(g, M, S.psix[X_VYX] + slot * S.psix_slot, j, i, K_XH, A_XH, B_XH, vyx);
    vyy = cpml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, vyy);
    vxy = cpml_y(g, M, S.psiy[Y_VXY] + slot * S.psiy_slot, j, i, K_YH, A_YH, B_YH, vxy);
    const T fipjp = modelp(M, slot, M_UIPJP)[c], f = modelp(M, slot, M_F)[c], gg = modelp(M, slot, M_G)[c];
    sxy[c] += fipjp * (vyx + vxy);
    sxx[c] = (T)((double)sxx[c] + ((double)(gg * (vxx + vyy)) + (2.0 * (double)f * (double)vxx)));
    syy[c] = (T)((double)syy[c] + ((double)(gg * (vxx + vyy)) + (2.0 * (double)f * (double)vyy)));
}

// stress half step, P-SV viscoelastic with L SLS (src/update_s_visc_PML.c:
// orders 2-8 :62-516 with CPML; the reference 10/12 default :518-660 has none)
template <typename T, int FDOH>
__global__ void k_s_psv_visc(KGrid g, KState<T> S, KModel<T> M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY), *sxy = fieldp(S, slot, P_SXY);
    const long long c = pidx(g, j, i);
    const T DT = g.dt, DH = g.dh;
    const T dhi = (T)(1.0 / (double)DH), dthalbe = (T)((double)DT / 2.0);
    T vxx = 0, vyx = 0, vxy = 0, vyy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxx = tap(m, vxx, (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]), g.quirk_hi != 0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyx = tap(m, vyx, (T)g.hc[m] * (vy[pidx(g, j, i + m)] - vy[pidx(g, j, i - m + 1)]), g.quirk_hi != 0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxy = tap(m, vxy, (T)g.hc[m] * (vx[pidx(g, j + m, i)] - vx[pidx(g, j - m + 1, i)]), g.quirk_hi != 0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyy = tap(m, vyy, (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]), g.quirk_hi != 0);
    vxx = vxx * dhi;
    vyx = vyx * dhi;
    vxy = vxy * dhi;
    vyy = vyy * dhi;
    if (!g.quirk_hi) {
        vxx = cpml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, i, K_X, A_X, B_X, vxx);
        vyx = cpml_x(g, M, S.psix[X_VYX] + slot * S.psix_slot, j, i, K_XH, A_XH, B_XH, vyx);
        vyy = cpml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, vyy);
        vxy = cpml_y(g, M, S.psiy[Y_VXY] + slot * S.psiy_slot, j, i, K_YH, A_YH, B_YH, vxy);
    }
    const int L = g.L;
    T sumr = 0, sump = 0, sumq = 0;
    for (int l = 1; l <= L; l++) {
        sumr += memp(S, g, slot, 0, l)[c];
        sump += memp(S, g, slot, 1, l)[c];
        sumq += memp(S, g, slot, 2, l)[c];
    }
    const T fipjp = modelp(M, slot, M_FIPJPV)[c], f = modelp(M, slot, M_FV)[c], gg = modelp(M, slot, M_GV)[c];
    sxy[c] += (fipjp * (vxy + vyx)) + (dthalbe * sumr);
    sxx[c] = (T)((double)sxx[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vyy) + (double)(dthalbe * sump)));
    syy[c] = (T)((double)syy[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vxx) + (double)(dthalbe * sumq)));
    const T mu = modelp(M, slot, M_MUR)[c], pi = modelp(M, slot, M_PIR)[c], muij = modelp(M, slot, M_MUIPJPR)[c];
    const T *tsp = modelp(M, slot, M_TAUS), *tpp = modelp(M, slot, M_TAUP), *tsijp = modelp(M, slot, M_TAUSIPJP);
    const T ts = tsp ? tsp[c] : (T)g.taus0, tp = tpp ? tpp[c] : (T)g.taup0, tsij = tsijp ? tsijp[c] : (T)g.tausipjp0;
    sumr = sump = sumq = 0;
    for (int l = 1; l <= L; l++) {
        const T eta = g.eta[l];
        // dip, d, e of src/prepare_update_s.c:57-59, formed in the same order
        const T dip = muij * eta * tsij, d = mu * eta * ts, e = pi * eta * tp;
        T *rr = memp(S, g, slot, 0, l) + c, *pp = memp(S, g, slot, 1, l) + c, *qq = memp(S, g, slot, 2, l) + c;
        T r = (T)g.bip[l] * (*rr * (T)g.cip[l] - (dip * (vxy + vyx)));
        T p = (T)((double)g.bjm[l] * ((double)(*pp * (T)g.cjm[l] - (e * (vxx + vyy))) + (2.0 * (double)d * (double)vyy)));
        T q = (T)((double)g.bjm[l] * ((double)(*qq * (T)g.cjm[l] - (e * (vxx + vyy))) + (2.0 * (double)d * (double)vxx)));
        *rr = r;
        *pp = p;
        *qq = q;
        sumr += r;
        sump += p;
        sumq += q;
    }
    sxy[c] += (dthalbe * sumr);
    sxx[c] += (dthalbe * sump);
    syy[c] += (dthalbe * sumq);
}

// stress half step, SH elastic / viscoelastic (src/update_s_elastic_PML_SH.c:
// 60-400, src/update_s_visc_PML_SH.c:59-476)
template <typename T, int FDOH>
__global__ void k_s_sh(KGrid g, KState<T> S, KModel<T> M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *vz = fieldp(S, slot, P_VZ);
    T *sxz = fieldp(S, slot, P_SXZ), *syz = fieldp(S, slot, P_SYZ);
    const long long c = pidx(g, j, i);
    const T DT = g.dt, DH = g.dh;
    const int L = g.L;
    const T dhi = L ? (T)(1.0 / (double)DH) : DT / DH, dthalbe = (T)((double)DT / 2.0);
    T vzx = 0, vzy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vzx = tap(m, vzx, (T)g.hc[m] * (vz[pidx(g, j, i + m)] - vz[pidx(g, j, i - m + 1)]));
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vzy = tap(m, vzy, (T)g.hc[m] * (vz[pidx(g, j + m - 1, i)] - vz[pidx(g, j - m, i)]));
    vzx = vzx * dhi;
    vzy = vzy * dhi;
    vzx = cpml_x(g, M, S.psix[X_VZX] + slot * S.psix_slot, j, i, K_XH, A_XH, B_XH, vzx);
    vzy = cpml_y(g, M, S.psiy[Y_VZY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, vzy);
    if (!L) {
        const T fipjp = modelp(M, slot, M_UIPJP)[c], f = modelp(M, slot, M_F)[c];
        sxz[c] += (fipjp * vzx);
        syz[c] += (f * vzy);
        return;
    }
    T sumo = 0, sumt = 0;
    for (int l = 1; l <= L; l++) {
        sumo += memp(S, g, slot, 4, l)[c];
        sumt += memp(S, g, slot, 3, l)[c];
    }
    sxz[c] += (modelp(M, slot, M_FIPJPV)[c] * vzx) + (dthalbe * sumo);
    syz[c] += (modelp(M, slot, M_FV)[c] * vzy) + (dthalbe * sumt);
    const T mu = modelp(M, slot, M_MUR)[c], muij = modelp(M, slot, M_MUIPJPR)[c];
    const T *tsp = modelp(M, slot, M_TAUS), *tsijp = modelp(M, slot, M_TAUSIPJP);
    const T ts = tsp ? tsp[c] : (T)g.taus0, tsij = tsijp ? tsijp[c] : (T)g.tausipjp0;
    sumo = sumt = 0;
    for (int l = 1; l <= L; l++) {
        const T eta = g.eta[l];
        const T dip = muij * eta * tsij, d = mu * eta * ts;
        T *oo = memp(S, g, slot, 4, l) + c, *tt = memp(S, g, slot, 3, l) + c;
        T o = (T)g.bip[l] * (*oo * (T)g.cip[l] - (dip * vzx));
        T t = (T)g.bjm[l] * (*tt * (T)g.cjm[l] - (d * vzy));
        *oo = o;
        *tt = t;
        sumt += t;
        sumo += o;
    }
    sxz[c] += (dthalbe * sumo);
    syz[c] += (dthalbe * sumt);
}

// pressure half step, acoustic (src/update_p_PML.c:55-273; the reference
// 10/12 default :275-287 when quirk_hi)
template <typename T, int FDOH>
__global__ void k_p_ac(KGrid g, KState<T> S, KModel<T> M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    T *sp = fieldp(S, slot, P_SP);
    const long long c = pidx(g, j, i);
    const T DT = g.dt, DH = g.dh;
    const T dhi = DT / DH;
    T vxx = 0, vyy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxx = tap(m, vxx, (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]), g.quirk_hi != 0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyy = tap(m, vyy, (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]), g.quirk_hi != 0);
    if (g.quirk_hi) {
        const T gg = modelp(M, slot, M_VP)[c] * DT;
        sp[c] += (gg * (vxx + vyy)) * dhi;
        return;
    }
    vxx = vxx * dhi;
    vyy = vyy * dhi;
    vxx = cpml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, i, K_X, A_X, B_X, vxx);
    vyy = cpml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, vyy);
    sp[c] += modelp(M, slot, M_GAC)[c] * (vxx + vyy);
}

// pressure half step, viscoacoustic with L relaxation mechanisms
// (src/update_p_visc_PML.c: FDORDER 2 :61-146 with CPML; every other order
// :148-182, sums from zero and no CPML).  The CPML memories of vyx and vxy
// that its FDORDER 2 branch also advances feed nothing else and are not kept.
template <typename T, int FDOH>
__global__ void k_p_visc(KGrid g, KState<T> S, KModel<T> M) {
    constexpr bool Z0 = FDOH != 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    T *sp = fieldp(S, slot, P_SP);
    const long long c = pidx(g, j, i);
    const T DT = g.dt, DH = g.dh;
    const T dhi = (T)(1.0 / (double)DH), dthalbe = (T)((double)DT / 2.0);
    T vxx = 0, vyy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vxx = tap(m, vxx, (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]), Z0);
#pragma unroll
    for (int m = 1; m <= FDOH; m++) vyy = tap(m, vyy, (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]), Z0);
    vxx = vxx * dhi;
    vyy = vyy * dhi;
    if (FDOH == 1) {
        vxx = cpml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, i, K_X, A_X, B_X, vxx);
        vyy = cpml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, j, i, K_Y, A_Y, B_Y, vyy);
    }
    const int L = g.L;
    T sump = 0;
    for (int l = 1; l <= L; l++) sump += memp(S, g, slot, 1, l)[c];
    const T gg = modelp(M, slot, M_GV)[c], pi = modelp(M, slot, M_PIR)[c];
    const T *tpp = modelp(M, slot, M_TAUP);
    const T tp = tpp ? tpp[c] : (T)g.taup0;
    sp[c] += (gg * (vxx + vyy)) + (dthalbe * sump);
    sump = 0;
    for (int l = 1; l <= L; l++) {
        const T e = pi * (T)g.eta[l] * tp;  // e of src/prepare_update_p.c:62, formed in the same order
        T *pp = memp(S, g, slot, 1, l) + c;
        const T p = (T)g.bjm[l] * (*pp * (T)g.cjm[l] - (e * (vxx + vyy)));
        *pp = p;
        sump += p;
    }
    sp[c] += (dthalbe * sump);
}

// Cells of a snapshot that the stencil kernels stored and a later kernel of
// the same step changes (explosive sources, the free surface): base of the
// snapshot of slot 0 being stored (NULL: nothing to patch), floats between
// slots, NX*NY, and the component index of every patched field (-1 absent).
// fp16 snapshot segments (IFOS_SNAP_F16S).  The 64 consecutive cells of a
// row that one pipelined tile covers share one fp32 scale: the segment's
// absolute maximum m is mapped to kSegTop, just below fp16's largest finite
// value (65504), so the segment's largest values sit at the top of fp16's
// top binade, where its relative precision is best.  A value v is stored as
// fp16(v * (kSegTop / m)), rounded to nearest even, and read back as
// float(h) * (m / kSegTop); a segment whose maximum is below 1e-30 (or NaN)
// is stored as zeros.
constexpr int kSegCells = 64;
constexpr float kSegTop = 65472.0f;  // 2^15 (2 - 2^-9)
// int16 segments (IFOS_SNAP_I16S): the same segments and scales, the maximum
// mapped to 32767 and each value stored as the nearest integer of
// v * (32767 / m): an absolute error of at most about m / 65534, 32 times
// below fp16's m / 2048 at the top of the segment (fp16 keeps more relative
// precision only for values below m / 32).
constexpr float kSegTopI16 = 32767.0f;
// all 32 lanes of a warp, each with a column pair of one segment: its maximum |v|
__device__ __forceinline__ float seg_absmax_warp(float v0, float v1, bool ok0, bool ok1) {
    const unsigned a0 = ok0 ? (__float_as_uint(v0) & 0x7fffffffu) : 0u;
    const unsigned a1 = ok1 ? (__float_as_uint(v1) & 0x7fffffffu) : 0u;
    return __uint_as_float(__reduce_max_sync(0xffffffffu, a0 > a1 ? a0 : a1));
}
// The quantisation factor q and the stored read-back scale inv of a segment
// maximum m.  Neither needs to be correctly rounded: q * inv = 1 within a few
// ulps of fp32 (far below fp16's 2^-11) and m * q stays below 65504, so the
// fast approximate division (a reciprocal and a multiply) serves; it is exact
// enough for m below 2^126 (a wavefield amplitude of 8.5e37).
__device__ __forceinline__ void seg_scales(float m, float &q, float &inv, float top = kSegTop) {
    if (m >= 1e-30f) {
        q = __fdividef(top, m);
        inv = m * (1.0f / top);
    } else {
        q = 0.0f;
        inv = 0.0f;
    }
}

// the 16-bit pattern of a scaled value x (|x| <= top) and back: fp16 rounded
// to nearest even, or the nearest integer (clamped to +-32767 against the
// approximate scale)
__device__ __forceinline__ unsigned short seg_pack(float x, bool i16) {
    if (i16) return (unsigned short)(short)__float2int_rn(fminf(fmaxf(x, -kSegTopI16), kSegTopI16));
    return __half_as_ushort(__float2half_rn(x));
}
__device__ __forceinline__ float seg_unpack(unsigned short u, bool i16) {
    return i16 ? (float)(short)u : __half2float(__ushort_as_half(u));
}

struct KSnapPatch {
    float *base;
    long long slot_floats;
    long long n;
    int c_sxx, c_syy, c_sp, c_syz;
};
__device__ __forceinline__ void snap_patch(const KSnapPatch &pt, int slot, int comp, const KGrid &g, int j, int i,
                                           float v) {
    if (pt.base && comp >= 0) pt.base[slot * pt.slot_floats + comp * pt.n + (long long)(j - 1) * g.nx + (i - 1)] = v;
}

// ---------------------------------------------------------------------------
// Sources.  Forward force sources after the velocity update
// (src/update_v_PML.c:553-564, src/update_v_PML_SH.c:327-333); adjoint
// residual injection at the receivers (:567-578, unscaled).  One thread per
// slot walks its sources in order, so coincident sources add in the
// reference's order.
struct KSrc {
    const float *pos;    // slot-major: slot * 8 * max_src
    const float *sig;    // slot * max_src * NT
    const int *nsrc;     // per slot
    int max_src, nt_total;
};
struct KRec {
    const int *pos;      // slot * 2 * max_rec
    const int *ntr;      // per slot
    int max_rec;
    const float *adj;    // slot * 3 * max_rec * NT
    float *sec;          // slot * NS * max_rec * NT
    // the cell -> receiver map the velocity ops use to sample or inject the
    // receivers in place: per slot map_stride ints, first NY row entries
    // (-1: no receiver in the row, else the row's index among the slot's
    // receiver rows), then rmax rows of NX cell entries (-1 or the index of
    // the receiver in the cell)
    const int *map;
    long long map_stride;
    int rmax;
};

// receiver indices of cells (j, i) and (j, i+1) of `slot` (-1: none)
__device__ __forceinline__ int2 rec_pair(const KRec &r, int nx, int ny, int slot, int j, int i, bool v0, bool v1) {
    const int *m = r.map + (long long)slot * r.map_stride;
    const int rr = m[j - 1];
    if (rr < 0) return make_int2(-1, -1);
    const int *cells = m + ny + (long long)rr * nx + (i - 1);
    return make_int2(v0 ? cells[0] : -1, v1 ? cells[1] : -1);
}

template <typename T>
__global__ void k_inject_v_fwd(KGrid g, KState<T> S, KModel<T> M, KSrc src, int nt, int psv, int sh) {
    pdl_wait();
    pdl_launch();
    const int slot = blockIdx.x;
    if (threadIdx.x) return;
    const int n = src.nsrc[slot];
    const float *pos = src.pos + (long long)slot * 8 * src.max_src;
    const float *sig = src.sig + (long long)slot * src.max_src * src.nt_total;
    T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY), *vz = fieldp(S, slot, P_VZ);
    const T DT = g.dt, DH = g.dh;
    const T *rip = modelp(M, slot, M_RIP), *rjp = modelp(M, slot, M_RJP);
    for (int l = 0; l < n; l++) {
        const int i = (int)pos[l], j = (int)pos[src.max_src + l];
        const long long c = pidx(g, j, i);
        const T s = sig[(long long)l * src.nt_total + nt - 1];
        if (psv) {
            const int type = (int)pos[7 * src.max_src + l];
            const float azi_rad = (double)pos[6 * src.max_src + l] * 3.141592653589793 / 180;
            if (type == 2) vx[c] += (DT * rip[c] * s) / (DH * DH);
            if (type == 3) vy[c] += (DT * rjp[c] * s) / (DH * DH);
            if (type == 4) {
                vx[c] = (T)((double)vx[c] + ((double)(DT * rip[c]) * sin((double)azi_rad) * (double)s) / (double)(DH * DH));
                vy[c] = (T)((double)vy[c] + ((double)(DT * rjp[c]) * cos((double)azi_rad) * (double)s) / (double)(DH * DH));
            }
        }
        if (sh) vz[c] = (T)((double)vz[c] + ((double)(rjp[c] * DT) * 1.0 * (double)s) / (double)(DH * DH));
    }
}

template <typename T>
__global__ void k_inject_v_adj(KGrid g, KState<T> S, KRec rec, int nt, int psv, int sh) {
    pdl_wait();
    pdl_launch();
    const int slot = blockIdx.y;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= rec.ntr[slot]) return;
    const int *pos = rec.pos + (long long)slot * 2 * rec.max_rec;
    const long long c = pidx(g, pos[rec.max_rec + l], pos[l]);
    const float *adj = rec.adj + (long long)slot * 3 * rec.max_rec * g.nt_total;
    const long long o = (long long)l * g.nt_total + nt - 1;
    const long long cs = (long long)rec.max_rec * g.nt_total;
    if (psv) {
        T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
        const int at = g.adjoint_type;
        if (at == 1) {
            vx[c] += (T)adj[o];
            vy[c] += (T)adj[cs + o];
        }
        if (at == 2) vy[c] += (T)adj[cs + o];
        if (at == 3) vx[c] += (T)adj[o];
    }
    if (sh) fieldp(S, slot, P_VZ)[c] += (T)adj[2 * cs + o];
}

// Explosive source after the stress update (src/psource.c:37-58).
// update_v_PML assigns the global SOURCE_TYPE from the type column of each
// source it visits (src/update_v_PML.c:558); psource then fires when the last
// one is explosive (src/IFOS2D.c:1758).
__device__ __forceinline__ bool psource_fires(const KSrc &src, int slot) {
    const int n = src.nsrc[slot];
    if (n <= 0) return false;
    const float *pos = src.pos + (long long)slot * 8 * src.max_src;
    return (int)pos[7 * src.max_src + n - 1] == 1;
}
// the explosive source term of source l at step nt (src/psource.c:47-52):
// the centred difference of its signal over 2 DH^2, one-sided at the ends
__device__ __forceinline__ float psource_amp(const KSrc &src, int slot, int l, int nt, float DH) {
    const float *sig = src.sig + (long long)slot * src.max_src * src.nt_total;
    const int NT = src.nt_total;
    const float *sl = sig + (long long)l * NT - 1;
    float amp = 0.0f;
    if (nt == 1) amp = sl[nt + 1] / (2.0 * DH * DH);
    if ((nt > 1) && (nt < NT)) amp = (sl[nt + 1] - sl[nt - 1]) / (2.0 * DH * DH);
    if (nt == NT) amp = -sl[nt - 1] / (2.0 * DH * DH);
    return amp;
}
// source l of a slot at its cell
template <typename T>
__device__ void psource_apply(const KGrid &g, const KState<T> &S, const KSrc &src, int nt, int acoustic,
                              const KSnapPatch &pt, int slot, int l) {
    const float *pos = src.pos + (long long)slot * 8 * src.max_src;
    const int i = (int)pos[l], j = (int)pos[src.max_src + l];
    const float amp = psource_amp(src, slot, l, nt, g.dh);
    const long long c = pidx(g, j, i);
    if (!acoustic) {
        T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY);
        sxx[c] = (T)((double)sxx[c] + 0.5 * (double)amp);
        syy[c] = (T)((double)syy[c] + 0.5 * (double)amp);
        snap_patch(pt, slot, pt.c_sxx, g, j, i, (float)sxx[c]);
        snap_patch(pt, slot, pt.c_syy, g, j, i, (float)syy[c]);
    } else {
        T *sp = fieldp(S, slot, P_SP);
        sp[c] += (T)amp;
        snap_patch(pt, slot, pt.c_sp, g, j, i, (float)sp[c]);
    }
}

// pressure residual at receiver l, ADJOINT_TYPE 4 (src/psource.c:61-74)
template <typename T>
__device__ void psource_adj_rec(const KGrid &g, const KState<T> &S, const KRec &rec, int nt, int acoustic, int slot,
                                int l) {
    const int *pos = rec.pos + (long long)slot * 2 * rec.max_rec;
    const long long c = pidx(g, pos[rec.max_rec + l], pos[l]);
    const float *adj = rec.adj + (long long)slot * 3 * rec.max_rec * g.nt_total;
    const float amp = adj[2LL * rec.max_rec * g.nt_total + (long long)l * g.nt_total + nt - 1];
    if (!acoustic) {
        T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY);
        sxx[c] = (T)((double)sxx[c] + 0.5 * (double)amp);
        syy[c] = (T)((double)syy[c] + 0.5 * (double)amp);
    } else {
        fieldp(S, slot, P_SP)[c] += (T)amp;
    }
}

// free surface at j=1 after the source (src/surface_elastic_PML.c:47-106,
// src/surface_PML.c:61-173, src/surface_acoustic_PML.c:28-38).  The mirrored
// ghost rows are not stored: the velocity kernels read them via ld_mirror_*.
template <typename T, int FDOH>
__device__ void surface_cell(const KGrid &g, const KState<T> &S, const KModel<T> &M, int psv, int sh, int acoustic,
                             const KSnapPatch &pt, int slot, int i) {
    const int j = 1;
    const long long c = pidx(g, j, i);
    if (acoustic) {
        fieldp(S, slot, P_SP)[c] = 0;
        snap_patch(pt, slot, pt.c_sp, g, j, i, 0.0f);
        return;
    }
    if (sh) {
        fieldp(S, slot, P_SYZ)[c] = 0;
        snap_patch(pt, slot, pt.c_syz, g, j, i, 0.0f);
    }
    if (!psv) return;
    snap_patch(pt, slot, pt.c_syy, g, j, i, 0.0f);
    const T DT = g.dt, DH = g.dh;
    const T dh24 = (T)(1.0 / (double)DH), dthalbe = (T)((double)DT / 2.0);
    const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
    T *sxx = fieldp(S, slot, P_SXX), *syy = fieldp(S, slot, P_SYY);
    syy[c] = 0;
    const int L = g.L;
    if (L)
        for (int l = 1; l <= L; l++) memp(S, g, slot, 2, l)[c] = 0;
    T vxx = 0, vyy = 0;
#pragma unroll
    for (int m = 1; m <= FDOH; m++) {
        vxx += (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]);
        vyy += (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]);
    }
    vxx *= dh24;
    vyy *= dh24;
    vxx = cpml_x(g, M, S.psix[X_VXXS] + slot * S.psix_slot, j, i, K_X, A_X, B_X, vxx);
    const T *srf = M.srf + (long long)M.slot_model[slot] * M.srf_stride;
    const T fjm = srf[i - 1], gg = srf[g.nx + i - 1];
    if (!L) {
        sxx[c] += -DT * ((gg * gg) / (gg + fjm) * vxx + gg * vyy);
        snap_patch(pt, slot, pt.c_sxx, g, j, i, (float)sxx[c]);
        return;
    }
    const T djm = srf[2 * g.nx + i - 1], e = srf[3 * g.nx + i - 1];
    T sump = 0;
    for (int l = 1; l <= L; l++) sump += memp(S, g, slot, 1, l)[c];
    sxx[c] += -(DT * (gg - fjm) * (gg - fjm) * vxx / gg) - (DT * (gg - fjm) * vyy) - (dthalbe * sump);
    sump = 0;
    for (int l = 1; l <= L; l++) {
        T *pp = memp(S, g, slot, 1, l) + c;
        const T bjm = g.bjm_srf[l];
        *pp = (T)((double)*pp + (double)bjm * (((double)(djm - e) * ((double)(fjm / gg) - 1.0) * (double)vxx) -
                                                (double)((djm - e) * vyy)));
        sump += *pp;
    }
    sxx[c] += (dthalbe * sump);
    snap_patch(pt, slot, pt.c_sxx, g, j, i, (float)sxx[c]);
}

// the instability probe of src/IFOS2D.c:1660-1672 (vy or vz at the grid centre)
template <typename T>
__device__ void nan_probe(const KGrid &g, const KState<T> &S, int psv, int slot, int *bad) {
    const long long cc = pidx(g, g.ny / 2, g.nx / 2);
    T v = psv ? fieldp(S, slot, P_VY)[cc] : fieldp(S, slot, P_VZ)[cc];
    if (isnan((double)v)) atomicExch(bad, 1);
}

// receiver l (src/seismo_ssg.c:26-140)
template <typename T, int FDOH>
__device__ void seismo_rec(const KGrid &g, const KState<T> &S, const KModel<T> &M, const KRec &rec, int nt, int seismo,
                           int psv, int sh, int acoustic, int slot, int l) {
    const int *pos = rec.pos + (long long)slot * 2 * rec.max_rec;
    const int i = pos[l], j = pos[rec.max_rec + l];
    const long long c = pidx(g, j, i);
    const long long cs = (long long)rec.max_rec * g.nt_total;
    float *sec = rec.sec + (long long)slot * 6 * cs + (long long)l * g.nt_total + nt - 1;
    const bool want_v = seismo == 1 || seismo == 4 || seismo == 5;
    const bool want_p = seismo == 2 || seismo == 4 || seismo == 5;
    const bool want_cd = seismo == 3 || seismo == 4;
    if (want_cd) {
        const T *vx = fieldp(S, slot, P_VX), *vy = fieldp(S, slot, P_VY);
        T vxx = 0, vyy = 0, vyx = 0, vxy = 0;
#pragma unroll
        for (int m = 1; m <= FDOH; m++) {
            vxx += (T)g.hc[m] * (vx[pidx(g, j, i + m - 1)] - vx[pidx(g, j, i - m)]);
            vyy += (T)g.hc[m] * (vy[pidx(g, j + m - 1, i)] - vy[pidx(g, j - m, i)]);
            vyx += (T)g.hc[m] * (vy[pidx(g, j, i + m)] - vy[pidx(g, j, i - m + 1)]);
            vxy += (T)g.hc[m] * (vx[pidx(g, j + m, i)] - vx[pidx(g, j - m + 1, i)]);
        }
        const T dhi = (T)g.dt / (T)g.dh;
        vxx *= dhi;
        vyy *= dhi;
        vyx *= dhi;
        vxy *= dhi;
        sec[5 * cs] = (float)((double)(vxx + vyy) * sqrt((double)modelp(M, slot, M_VP)[c]));
        sec[4 * cs] = !acoustic ? (float)((double)(vxy - vyx) * sqrt((double)modelp(M, slot, M_VS)[c])) : 0.0f;
    }
    if (want_v) {
        if (seismo == 4 || psv) {
            sec[0] = (float)fieldp(S, slot, P_VX)[c];
            sec[cs] = (float)fieldp(S, slot, P_VY)[c];
        }
        if (sh) sec[2 * cs] = (float)fieldp(S, slot, P_VZ)[c];
    }
    if (want_p && (seismo != 5 || psv)) {
        if (!acoustic) sec[3 * cs] = (float)(-fieldp(S, slot, P_SXX)[c] - fieldp(S, slot, P_SYY)[c]);
        else sec[3 * cs] = (float)(-fieldp(S, slot, P_SP)[c]);
    }
}

// After the stress update: the explosive sources and the free surface
// (src/IFOS2D.c:1758-1768), one thread per column of row 1.  A column thread
// first applies the sources located in its row-1 cell, in source order, then
// the surface update of that cell; the thread of column 1 applies the sources
// below row 1.  Every cell is thus changed by one thread, in the reference's
// order.  grid: x over columns, y = slot.
template <typename T, int FDOH>
__global__ void k_surface_src(KGrid g, KState<T> S, KModel<T> M, KSrc src, int nt, int psv, int sh, int acoustic,
                              int do_ps, int do_surf, KSnapPatch pt) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int slot = blockIdx.y;
    if (i > g.nx) return;
    if (do_ps && psource_fires(src, slot)) {
        const int n = src.nsrc[slot];
        const float *pos = src.pos + (long long)slot * 8 * src.max_src;
        for (int l = 0; l < n; l++) {
            const int il = (int)pos[l], jl = (int)pos[src.max_src + l];
            if (jl == 1 ? il == i : i == 1) psource_apply<T>(g, S, src, nt, acoustic, pt, slot, l);
        }
    }
    if (do_surf) surface_cell<T, FDOH>(g, S, M, psv, sh, acoustic, pt, slot, i);
}

// the pressure residual at the receivers, ADJOINT_TYPE 4; grid: x over receivers, y = slot
template <typename T>
__global__ void k_psource_adj(KGrid g, KState<T> S, KRec rec, int nt, int acoustic) {
    pdl_wait();
    pdl_launch();
    const int slot = blockIdx.y;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < rec.ntr[slot]) psource_adj_rec<T>(g, S, rec, nt, acoustic, slot, l);
}

// receivers and the instability probe; grid: x over receivers, y = slot
template <typename T, int FDOH>
__global__ void k_seismo(KGrid g, KState<T> S, KModel<T> M, KRec rec, int nt, int seismo, int psv, int sh,
                         int acoustic, int *bad) {
    pdl_wait();
    pdl_launch();
    const int slot = blockIdx.y;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l == 0) nan_probe<T>(g, S, psv, slot, bad);
    if (seismo && l < rec.ntr[slot]) seismo_rec<T, FDOH>(g, S, M, rec, nt, seismo, psv, sh, acoustic, slot, l);
}

}  // namespace ifos
