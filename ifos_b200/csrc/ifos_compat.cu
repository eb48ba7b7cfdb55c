// libifos_compat: the reference's per-kernel functions under their own names
// and signatures (include/ifos_compat.h), computed on the device.
//
// Each entry point mirrors the caller's arrays it reads into device buffers
// (kept per host block for reuse), runs one thread per cell on the
// reference's own array layout, and copies the arrays it writes back before
// returning.  The arithmetic follows the reference functions term by term
// (operation order, float/double promotions, the sums of the written-out
// FDORDER cases and of the generic loops), so results are bit-identical; the
// library is compiled with --fmad=false like libifos_b200.
//
// Layout (src/util.c matrix()/f3tensor()): a wavefield or model matrix of
// rows -nd+1..NY+nd and columns -nd+1..NX+nd (nd = FDORDER/2+1,
// src/IFOS2D.c:310,375-518) is one contiguous block starting at
// &m[-nd+1][-nd+1] with row stride NX+2nd; an f3tensor keeps the mechanism
// index innermost; CPML psi arrays are matrix(1,NY,1,2FW) (x strips) and
// matrix(1,2FW,1,NX) (y strips); profiles are vector(1,2FW).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "ifos_compat.h"

// globals of the reference driver (src/globvar.h), defined by the program
extern "C" {
extern int NX, NY, NT, FDORDER, FW, FREE_SURF, BOUNDARY, L, NPROCX, NPROCY, SOURCE_TYPE, ADJOINT_TYPE, VELOCITY,
    PARAMETERIZATION, WAVETYPE, SEISMO, ACOUSTIC;
extern int POS[3];
extern float DT, DH, F_REF;
extern float *FL;
}

namespace {

constexpr double kPi = 3.141592653589793;  // PI of src/fd.h:20

void die(const char *what, cudaError_t e) {
    std::fprintf(stderr, "libifos_compat: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
}
#define CC(call)                           \
    do {                                   \
        cudaError_t e_ = (call);           \
        if (e_ != cudaSuccess) die(#call, e_); \
    } while (0)

// ---------------------------------------------------------------------------
// device mirrors of host blocks
struct Mirror {
    void *d = nullptr;
    size_t bytes = 0;
};
std::unordered_map<const void *, Mirror> g_mirrors;
cudaStream_t g_st = nullptr;

cudaStream_t stream() {
    if (!g_st) CC(cudaStreamCreateWithFlags(&g_st, cudaStreamNonBlocking));
    return g_st;
}
// device buffer for a host block (allocated on first use, grown as needed)
float *mirror(const void *host, size_t bytes) {
    Mirror &m = g_mirrors[host];
    if (m.bytes < bytes) {
        if (m.d) CC(cudaFree(m.d));
        CC(cudaMalloc(&m.d, bytes));
        m.bytes = bytes;
    }
    return (float *)m.d;
}
// the host block copied in
float *up(const void *host, size_t bytes) {
    if (!host) return nullptr;
    float *d = mirror(host, bytes);
    CC(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, stream()));
    return d;
}
// a device mirror copied back out
void down(void *host, size_t bytes) {
    if (!host) return;
    CC(cudaMemcpyAsync(host, g_mirrors[host].d, bytes, cudaMemcpyDeviceToHost, stream()));
}
void finish() { CC(cudaStreamSynchronize(stream())); }

// block start and size of the driver's arrays
int nd_of() { return FDORDER / 2 + 1; }
size_t field_bytes() {
    const int nd = nd_of();
    return (size_t)(NY + 2 * nd) * (NX + 2 * nd) * sizeof(float);
}
void *fblk(float **m) { return m ? (void *)&m[-nd_of() + 1][-nd_of() + 1] : nullptr; }
void *tblk(float ***t) { return t ? (void *)&t[-nd_of() + 1][-nd_of() + 1][1] : nullptr; }
size_t tensor_bytes() { return field_bytes() * (size_t)L; }
void *pblk(float **psi) { return psi ? (void *)&psi[1][1] : nullptr; }
size_t psix_bytes() { return (size_t)NY * 2 * FW * sizeof(float); }
size_t psiy_bytes() { return (size_t)2 * FW * NX * sizeof(float); }

// ---------------------------------------------------------------------------
// device side
struct RG {
    int nd, stride, nx, ny;  // layout; NX, NY
    int nx1, nx2, ny1, ny2;  // updated range
    int fw, left, right, top, bottom;
    int fdoh, L;
    float dt, dh;
    float hc[7];
};

RG make_rg(int nx1, int nx2, int ny1, int ny2, const float *hc) {
    RG g{};
    g.nd = nd_of();
    g.stride = NX + 2 * g.nd;
    g.nx = NX;
    g.ny = NY;
    g.nx1 = nx1;
    g.nx2 = nx2;
    g.ny1 = ny1;
    g.ny2 = ny2;
    g.fw = FW;
    g.left = !BOUNDARY && POS[1] == 0;
    g.right = !BOUNDARY && POS[1] == NPROCX - 1;
    g.top = POS[2] == 0 && !FREE_SURF;
    g.bottom = POS[2] == NPROCY - 1;
    g.fdoh = FDORDER / 2;
    g.L = L;
    g.dt = DT;
    g.dh = DH;
    for (int m = 0; m < 7; m++) g.hc[m] = (hc && m >= 1 && m <= g.fdoh) ? hc[m] : 0.0f;
    return g;
}

__device__ __forceinline__ long long ri(const RG &g, int j, int i) {
    return (long long)(j + g.nd - 1) * g.stride + (i + g.nd - 1);
}

// CPML profiles gathered as 12 rows of 2FW (index h-1)
enum { PK_X = 0, PA_X, PB_X, PK_XH, PA_XH, PB_XH, PK_Y, PA_Y, PB_Y, PK_YH, PA_YH, PB_YH };
struct Prof {
    const float *p;
    int n;  // 2FW
    __device__ __forceinline__ float operator()(int k, int h) const { return p[k * n + h - 1]; }
};
const float *g_prof_dev = nullptr;
size_t g_prof_bytes = 0;
Prof upload_prof(float *const *vecs /*12, 1-based*/) {
    const int n = 2 * FW;
    Prof P{nullptr, n};
    if (n <= 0) return P;
    std::vector<float> h((size_t)12 * n, 0.0f);
    for (int k = 0; k < 12; k++)
        if (vecs[k])
            for (int q = 1; q <= n; q++) h[(size_t)k * n + q - 1] = vecs[k][q];
    const size_t bytes = h.size() * sizeof(float);
    if (g_prof_bytes < bytes) {
        if (g_prof_dev) CC(cudaFree((void *)g_prof_dev));
        CC(cudaMalloc((void **)&g_prof_dev, bytes));
        g_prof_bytes = bytes;
    }
    CC(cudaMemcpyAsync((void *)g_prof_dev, h.data(), bytes, cudaMemcpyHostToDevice, stream()));
    // the copy must complete before h goes out of scope
    finish();
    P.p = g_prof_dev;
    return P;
}

// psi = b*psi + a*d; d = d/K + psi (src/update_v_PML.c:180-181)
__device__ __forceinline__ float cp(float *psi, float b, float a, float K, float d) {
    *psi = b * *psi + a * d;
    return d / K + *psi;
}
// x strips: left i <= FW at h = i, right i >= nx2-FW+1 at h = i-nx2+2FW
__device__ __forceinline__ float pmlx(const RG &g, const Prof &P, float *psi, int j, int i, int kK, int ka, int kb,
                                      float d) {
    const int n2 = 2 * g.fw;
    if (g.left && i <= g.fw) d = cp(psi + (long long)(j - 1) * n2 + (i - 1), P(kb, i), P(ka, i), P(kK, i), d);
    if (g.right && i >= g.nx2 - g.fw + 1) {
        const int h = i - g.nx2 + n2;
        d = cp(psi + (long long)(j - 1) * n2 + (h - 1), P(kb, h), P(ka, h), P(kK, h), d);
    }
    return d;
}
// y strips: top j <= FW (no free surface) at h = j, bottom j >= ny2-FW+1 at h = j-ny2+2FW
__device__ __forceinline__ float pmly(const RG &g, const Prof &P, float *psi, int j, int i, int kK, int ka, int kb,
                                      float d) {
    if (g.top && j <= g.fw) d = cp(psi + (long long)(j - 1) * g.nx + (i - 1), P(kb, j), P(ka, j), P(kK, j), d);
    if (g.bottom && j >= g.ny2 - g.fw + 1) {
        const int h = j - g.ny2 + 2 * g.fw;
        d = cp(psi + (long long)(h - 1) * g.nx + (i - 1), P(kb, h), P(ka, h), P(kK, h), d);
    }
    return d;
}

// Staggered sums: fwd sum_m hc[m](f[k+m] - f[k-m+1]), bwd sum_m hc[m](f[k+m-1] - f[k-m])
// along stride s.  Z0 false: the m=1 term starts the sum (the written-out
// FDORDER cases); true: accumulated from zero (the generic loops).
template <int FD, bool Z0>
__device__ __forceinline__ float sfwd(const RG &g, const float *f, long long c, long long s) {
    float a = g.hc[1] * (f[c + s] - f[c]);
    if (Z0) a = 0.0f + a;
#pragma unroll
    for (int m = 2; m <= FD; m++) a += g.hc[m] * (f[c + m * s] - f[c - (m - 1) * s]);
    return a;
}
template <int FD, bool Z0>
__device__ __forceinline__ float sbwd(const RG &g, const float *f, long long c, long long s) {
    float a = g.hc[1] * (f[c] - f[c - s]);
    if (Z0) a = 0.0f + a;
#pragma unroll
    for (int m = 2; m <= FD; m++) a += g.hc[m] * (f[c + (m - 1) * s] - f[c - m * s]);
    return a;
}

#define CELL_IJ(g)                                                    \
    const int i = (g).nx1 + (int)(blockIdx.x * blockDim.x + threadIdx.x); \
    const int j = (g).ny1 + (int)(blockIdx.y * blockDim.y + threadIdx.y); \
    if (i > (g).nx2 || j > (g).ny2) return;                           \
    const long long c = ri((g), j, i);

dim3 grid_of(int nx1, int nx2, int ny1, int ny2) {
    return dim3((unsigned)((nx2 - nx1 + 1 + 31) / 32), (unsigned)((ny2 - ny1 + 1 + 7) / 8));
}
const dim3 kBlk(32, 8);

#define DISPATCH_FD(fdoh, ...)                                  \
    switch (fdoh) {                                             \
        case 1: { constexpr int FD = 1; __VA_ARGS__; } break;   \
        case 2: { constexpr int FD = 2; __VA_ARGS__; } break;   \
        case 3: { constexpr int FD = 3; __VA_ARGS__; } break;   \
        case 4: { constexpr int FD = 4; __VA_ARGS__; } break;   \
        case 5: { constexpr int FD = 5; __VA_ARGS__; } break;   \
        default: { constexpr int FD = 6; __VA_ARGS__; } break;  \
    }

}  // namespace

// ---------------------------------------------------------------------------
// kernels (one thread per cell of nx1..nx2 x ny1..ny2)
namespace {

// update_v_PML (src/update_v_PML.c:161-252 per written-out order; FDORDER
// 10/12 :466-528, one sum per component, no CPML and no vxp1) and
// update_v_acoustic_PML (AC; orders 2-8 written out, 10/12 generic loops
// :396-409).  PSV: P-SV stresses sxx/syy/sxy; AC: pressure sp.
template <int FD, bool HI, bool AC>
__global__ void kc_v(RG g, Prof P, float *vx, float *vy, float *vxp1, float *vyp1, const float *sxx, const float *syy,
                     const float *sxy, const float *rip, const float *rjp, float *ps_xx, float *ps_yy, float *ps_xy_y,
                     float *ps_xy_x, int sw, int velocity) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    if (HI) {
        const float dtdh = DT * DT / DH;
        float ax, ay;
        if (AC) {
            // vxtmp += hc[m]*(sp[j][i+m]-sp[j][i-m+1]); vytmp likewise along y, from zero
            ax = sfwd<FD, true>(g, sxx, c, 1);
            ay = sfwd<FD, true>(g, sxx, c, s);
        } else {
            ax = sfwd<FD, false>(g, sxx, c, 1);
#pragma unroll
            for (int m = 1; m <= FD; m++) ax += g.hc[m] * (sxy[c + (m - 1) * s] - sxy[c - m * s]);
            ay = sfwd<FD, false>(g, syy, c, s);
#pragma unroll
            for (int m = 1; m <= FD; m++) ay += g.hc[m] * (sxy[c + (m - 1)] - sxy[c - m]);
        }
        vx[c] += ax * dtdh * rip[c];
        vy[c] += ay * dtdh * rjp[c];
        return;
    }
    float sxx_x, syy_y, sxy_x = 0.0f, sxy_y = 0.0f;
    if (AC) {
        sxx_x = sfwd<FD, false>(g, sxx, c, 1);
        syy_y = sfwd<FD, false>(g, sxx, c, s);
        sxx_x = pmlx(g, P, ps_xx, j, i, PK_XH, PA_XH, PB_XH, sxx_x);
        syy_y = pmly(g, P, ps_yy, j, i, PK_YH, PA_YH, PB_YH, syy_y);
    } else {
        sxx_x = sfwd<FD, false>(g, sxx, c, 1);
        sxy_x = sbwd<FD, false>(g, sxy, c, 1);
        sxy_y = sbwd<FD, false>(g, sxy, c, s);
        syy_y = sfwd<FD, false>(g, syy, c, s);
        if (g.left && i <= g.fw) {
            const long long q = (long long)(j - 1) * 2 * g.fw + (i - 1);
            sxx_x = cp(ps_xx + q, P(PB_XH, i), P(PA_XH, i), P(PK_XH, i), sxx_x);
            sxy_x = cp(ps_xy_x + q, P(PB_X, i), P(PA_X, i), P(PK_X, i), sxy_x);
        }
        if (g.right && i >= g.nx2 - g.fw + 1) {
            const int h = i - g.nx2 + 2 * g.fw;
            const long long q = (long long)(j - 1) * 2 * g.fw + (h - 1);
            sxx_x = cp(ps_xx + q, P(PB_XH, h), P(PA_XH, h), P(PK_XH, h), sxx_x);
            sxy_x = cp(ps_xy_x + q, P(PB_X, h), P(PA_X, h), P(PK_X, h), sxy_x);
        }
        if (g.top && j <= g.fw) {
            const long long q = (long long)(j - 1) * g.nx + (i - 1);
            syy_y = cp(ps_yy + q, P(PB_YH, j), P(PA_YH, j), P(PK_YH, j), syy_y);
            sxy_y = cp(ps_xy_y + q, P(PB_Y, j), P(PA_Y, j), P(PK_Y, j), sxy_y);
        }
        if (g.bottom && j >= g.ny2 - g.fw + 1) {
            const int h = j - g.ny2 + 2 * g.fw;
            const long long q = (long long)(h - 1) * g.nx + (i - 1);
            syy_y = cp(ps_yy + q, P(PB_YH, h), P(PA_YH, h), P(PK_YH, h), syy_y);
            sxy_y = cp(ps_xy_y + q, P(PB_Y, h), P(PA_Y, h), P(PK_Y, h), sxy_y);
        }
    }
    const float fx = AC ? (sxx_x) : (sxx_x + sxy_y), fy = AC ? (syy_y) : (sxy_x + syy_y);
    if (sw == 0) {
        vxp1[c] = rip[c] * fx / DH;
        vyp1[c] = rjp[c] * fy / DH;
    }
    if (sw == 1) {
        if (velocity == 0) {
            vxp1[c] += vx[c] * DT;
            vyp1[c] += vy[c] * DT;
        } else {
            vxp1[c] = vx[c];
            vyp1[c] = vy[c];
        }
    }
    vx[c] += DT * rip[c] * fx / DH;
    vy[c] += DT * rjp[c] * fy / DH;
}

// one source of update_v_PML / update_v_acoustic_PML / update_v_PML_SH
struct SrcI {
    int i, j, type;
    float s, s1;       // signals[l][nt], signals1[l][nt]
    double sn, cs;     // sin/cos of the azimuth, evaluated by the host's libm as the reference does
};
// sources in order (src/update_v_PML.c:553-578, src/update_v_PML_SH.c:327-343)
__global__ void kc_src_v(RG g, const SrcI *src, int n, float *vx, float *vy, float *vz, const float *rip,
                         const float *rjp, int sw, int adjoint_type) {
    if (blockIdx.x || threadIdx.x) return;
    const float DT = g.dt, DH = g.dh;
    for (int l = 0; l < n; l++) {
        const SrcI q = src[l];
        const long long c = ri(g, q.j, q.i);
        if (vz) {  // SH
            if (sw == 0) vz[c] = (float)((double)vz[c] + ((double)(rjp[c] * DT) * 1.0 * (double)q.s1) / (double)(DH * DH));
            if (sw == 1) vz[c] += q.s;
            continue;
        }
        if (sw == 0) {
            if (q.type == 2) vx[c] += (DT * rip[c] * q.s1) / (DH * DH);
            if (q.type == 3) vy[c] += (DT * rjp[c] * q.s1) / (DH * DH);
            if (q.type == 4) {
                vx[c] = (float)((double)vx[c] + ((double)(DT * rip[c]) * q.sn * (double)q.s) / (double)(DH * DH));
                vy[c] = (float)((double)vy[c] + ((double)(DT * rjp[c]) * q.cs * (double)q.s) / (double)(DH * DH));
            }
        }
        if (sw == 1) {
            if (adjoint_type == 1) {
                vx[c] += q.s;
                vy[c] += q.s1;
            }
            if (adjoint_type == 2) vy[c] += q.s1;
            if (adjoint_type == 3) vx[c] += q.s;
        }
    }
}

// update_s_elastic_PML (src/update_s_elastic_PML.c:151-241; FDORDER 10/12
// :442-535 without CPML, rates ux += DT*vxx, uy += DT*vyy)
template <int FD, bool HI>
__global__ void kc_s_el(RG g, Prof P, const float *vx, const float *vy, float *ux, float *uy, float *uxy, float *sxx,
                        float *syy, float *sxy, const float *pi, const float *u, const float *uipjp,
                        const float *rho, float *ps_vxx, float *ps_vyy, float *ps_vxy, float *ps_vyx, int param) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dhi = DT / DH;
    float vxx = sbwd<FD, false>(g, vx, c, 1) * dhi;
    float vyx = sfwd<FD, false>(g, vy, c, 1) * dhi;
    float vxy = sfwd<FD, false>(g, vx, c, s) * dhi;
    float vyy = sbwd<FD, false>(g, vy, c, s) * dhi;
    if (HI) {
        if (ux) ux[c] += DT * vxx;
        if (uy) uy[c] += DT * vyy;
        const float fipjp = uipjp[c] * DT, f = u[c] * DT, gg = pi[c] * DT;
        sxy[c] += (fipjp * (vxy + vyx));
        sxx[c] = (float)((double)sxx[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vyy)));
        syy[c] = (float)((double)syy[c] + ((double)(gg * (vxx + vyy)) - (2.0 * (double)f * (double)vxx)));
        return;
    }
    vxx = pmlx(g, P, ps_vxx, j, i, PK_X, PA_X, PB_X, vxx);
    vyx = pmlx(g, P, ps_vyx, j, i, PK_XH, PA_XH, PB_XH, vyx);
    vyy = pmly(g, P, ps_vyy, j, i, PK_Y, PA_Y, PB_Y, vyy);
    vxy = pmly(g, P, ps_vxy, j, i, PK_YH, PA_YH, PB_YH, vxy);
    const float fipjp = uipjp[c];
    float f = 0.0f, gg = 0.0f;
    if (param == 3) {
        f = u[c];
        gg = pi[c];
    }
    if (param == 1) {
        f = rho[c] * u[c] * u[c];
        gg = rho[c] * ((pi[c] * pi[c]) - 2 * u[c] * u[c]);
    }
    sxy[c] += fipjp * (vyx + vxy);
    sxx[c] = (float)((double)sxx[c] + ((double)(gg * (vxx + vyy)) + (2.0 * (double)f * (double)vxx)));
    syy[c] = (float)((double)syy[c] + ((double)(gg * (vxx + vyy)) + (2.0 * (double)f * (double)vyy)));
    if (uxy) uxy[c] = (fipjp / DT) * (vyx + vxy);
    if (ux) ux[c] = (float)((double)((gg / DT) * (vxx + vyy)) + ((2.0 * (double)f / (double)DT) * (double)vxx));
    if (uy) uy[c] = (float)((double)((gg / DT) * (vxx + vyy)) + ((2.0 * (double)f / (double)DT) * (double)vyy));
}

// update_s_visc_PML (src/update_s_visc_PML.c:171-276 written out for 2-8 with
// CPML and rates; FDORDER 10/12 generic loops :615-660 without either)
template <int FD, bool HI>
__global__ void kc_s_visc(RG g, Prof P, const float *vx, const float *vy, float *ux, float *uy, float *uxy,
                          float *sxx, float *syy, float *sxy, float *r, float *p, float *q, const float *fipjp,
                          const float *f, const float *gv, const float *bip, const float *bjm, const float *cip,
                          const float *cjm, const float *d, const float *e, const float *dip, float *ps_vxx,
                          float *ps_vyy, float *ps_vxy, float *ps_vyx) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dhi = 1.0 / DH, dthalbe = DT / 2.0;  // src/update_s_visc_PML.c:50-52
    float vxx = sbwd<FD, HI>(g, vx, c, 1) * dhi;
    float vyx = sfwd<FD, HI>(g, vy, c, 1) * dhi;
    float vxy = sfwd<FD, HI>(g, vx, c, s) * dhi;
    float vyy = sbwd<FD, HI>(g, vy, c, s) * dhi;
    if (!HI) {
        vxx = pmlx(g, P, ps_vxx, j, i, PK_X, PA_X, PB_X, vxx);
        vyx = pmlx(g, P, ps_vyx, j, i, PK_XH, PA_XH, PB_XH, vyx);
        vyy = pmly(g, P, ps_vyy, j, i, PK_Y, PA_Y, PB_Y, vyy);
        vxy = pmly(g, P, ps_vxy, j, i, PK_YH, PA_YH, PB_YH, vxy);
    }
    const int L = g.L;
    const long long t0 = c * L;
    float sumr = 0.0f, sump = 0.0f, sumq = 0.0f;
    for (int l = 0; l < L; l++) {
        sumr += r[t0 + l];
        sump += p[t0 + l];
        sumq += q[t0 + l];
    }
    sxy[c] += (fipjp[c] * (vxy + vyx)) + (dthalbe * sumr);
    sxx[c] = (float)((double)sxx[c] + ((double)(gv[c] * (vxx + vyy)) - (2.0 * (double)f[c] * (double)vyy) +
                                      (double)(dthalbe * sump)));
    syy[c] = (float)((double)syy[c] + ((double)(gv[c] * (vxx + vyy)) - (2.0 * (double)f[c] * (double)vxx) +
                                      (double)(dthalbe * sumq)));
    if (!HI) {
        if (uxy) uxy[c] = (float)((double)((fipjp[c] / DT) * (vxy + vyx)) + (0.5 * (double)sumr));
        if (ux)
            ux[c] = (float)((double)((gv[c] / DT) * (vxx + vyy)) - ((2.0 * (double)f[c] / (double)DT) * (double)vyy) +
                            (0.5 * (double)sump));
        if (uy)
            uy[c] = (float)((double)((gv[c] / DT) * (vxx + vyy)) - ((2.0 * (double)f[c] / (double)DT) * (double)vxx) +
                            (0.5 * (double)sumq));
    }
    sumr = sump = sumq = 0.0f;
    for (int l = 0; l < L; l++) {
        r[t0 + l] = bip[l] * (r[t0 + l] * cip[l] - (dip[t0 + l] * (vxy + vyx)));
        p[t0 + l] = (float)((double)bjm[l] * ((double)(p[t0 + l] * cjm[l] - (e[t0 + l] * (vxx + vyy))) +
                                              (2.0 * (double)d[t0 + l] * (double)vyy)));
        q[t0 + l] = (float)((double)bjm[l] * ((double)(q[t0 + l] * cjm[l] - (e[t0 + l] * (vxx + vyy))) +
                                              (2.0 * (double)d[t0 + l] * (double)vxx)));
        sumr += r[t0 + l];
        sump += p[t0 + l];
        sumq += q[t0 + l];
    }
    sxy[c] += (dthalbe * sumr);
    sxx[c] += (dthalbe * sump);
    syy[c] += (dthalbe * sumq);
    if (!HI) {
        if (uxy) uxy[c] = (float)((double)uxy[c] + (0.5 * (double)sumr));
        if (ux) ux[c] = (float)((double)ux[c] + (0.5 * (double)sump));
        if (uy) uy[c] = (float)((double)uy[c] + (0.5 * (double)sumq));
    }
}

}  // namespace

namespace {

// surface_elastic_PML (src/surface_elastic_PML.c:45-121), one thread per column
__global__ void kc_surf_el(RG g, Prof P, int j, const float *vx, const float *vy, float *sxx, float *syy, float *sxy,
                           float *ux, float *uy, float *uxy, const float *pi, const float *u, const float *rho,
                           float *ps_vxx, float *syz, float *sxz, float *uyz, float *uxz, int param, int psv, int sh) {
    const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i > g.nx) return;
    const long long c = ri(g, j, i), s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dh24 = 1.0 / DH;
    if (psv) {
        syy[c] = 0.0f;
        if (uy) uy[c] = 0.0f;
        float vxx = 0.0f, vyy = 0.0f;
        for (int m = 1; m <= g.fdoh; m++) {
            syy[c - m * s] = -syy[c + m * s];
            sxy[c - m * s] = -sxy[c + (m - 1) * s];
            if (uy) uy[c - m * s] = -uy[c + m * s];
            if (uxy) uxy[c - m * s] = -uxy[c + (m - 1) * s];
            vxx += g.hc[m] * (vx[c + m - 1] - vx[c - m]);
            vyy += g.hc[m] * (vy[c + (m - 1) * s] - vy[c - m * s]);
        }
        vxx *= dh24;
        vyy *= dh24;
        if (g.left && i <= g.fw) vxx = cp(ps_vxx + (long long)(j - 1) * 2 * g.fw + (i - 1), P(PB_X, i), P(PA_X, i), P(PK_X, i), vxx);
        if (g.right && i >= g.nx - g.fw + 1) {
            const int h = i - g.nx + 2 * g.fw;
            vxx = cp(ps_vxx + (long long)(j - 1) * 2 * g.fw + (h - 1), P(PB_X, h), P(PA_X, h), P(PK_X, h), vxx);
        }
        float fjm = 0.0f, gg = 0.0f;
        if (param == 3) {
            fjm = u[c] * 2.0;
            gg = pi[c];
        }
        if (param == 1) {
            fjm = rho[c] * u[c] * u[c] * 2.0;
            gg = rho[c] * ((pi[c] * pi[c]) - 2 * u[c] * u[c]);
        }
        sxx[c] += -DT * ((gg * gg) / (gg + fjm) * vxx + gg * vyy);
        if (ux) ux[c] = (float)(((2.0 * (double)gg * (double)fjm + (double)(fjm * fjm)) / (double)(gg + fjm)) * (double)vxx);
    }
    if (sh) {
        syz[c] = 0.0f;
        if (uyz) uyz[c] = 0.0f;
        for (int m = 1; m <= g.fdoh; m++) {
            syz[c - m * s] = -syz[c + m * s];
            sxz[c - m * s] = -sxz[c + (m - 1) * s];
            if (uyz) uyz[c - m * s] = -uyz[c + m * s];
            if (uxz) uxz[c - m * s] = -uxz[c + (m - 1) * s];
        }
    }
}

// surface_PML (src/surface_PML.c:61-173), one thread per column; etajm holds
// peta (the reference copies it in), sumu/sumpi as formed there (:48-57)
__global__ void kc_surf_visc(RG g, Prof P, int j, const float *vx, const float *vy, float *sxx, float *syy,
                             float *sxy, float *ux, float *uy, float *uxy, float *p, float *q, const float *ppi,
                             const float *pu, const float *prho, const float *ptaup, const float *ptaus,
                             const float *etajm, float sumu, float sumpi, float *ps_vxx, float *syz, float *sxz,
                             float *uyz, float *uxz, int param, int psv, int sh) {
    const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i > g.nx) return;
    const long long c = ri(g, j, i), s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dh24 = 1.0 / DH, dthalbe = DT / 2.0;
    const int L = g.L;
    const long long t0 = c * L;
    if (psv) {
        syy[c] = 0.0f;
        if (uy) uy[c] = 0.0f;
        for (int l = 0; l < L; l++) q[t0 + l] = 0.0f;
        float vxx = 0.0f, vyy = 0.0f;
        for (int m = 1; m <= g.fdoh; m++) {
            syy[c - m * s] = -syy[c + m * s];
            sxy[c - m * s] = -sxy[c + (m - 1) * s];
            if (uy) uy[c - m * s] = -uy[c + m * s];
            if (uxy) uxy[c - m * s] = -uxy[c + (m - 1) * s];
            vxx += g.hc[m] * (vx[c + m - 1] - vx[c - m]);
            vyy += g.hc[m] * (vy[c + (m - 1) * s] - vy[c - m * s]);
        }
        vxx *= dh24;
        vyy *= dh24;
        if (g.left && i <= g.fw) vxx = cp(ps_vxx + (long long)(j - 1) * 2 * g.fw + (i - 1), P(PB_X, i), P(PA_X, i), P(PK_X, i), vxx);
        if (g.right && i >= g.nx - g.fw + 1) {
            const int h = i - g.nx + 2 * g.fw;
            vxx = cp(ps_vxx + (long long)(j - 1) * 2 * g.fw + (h - 1), P(PB_X, h), P(PA_X, h), P(PK_X, h), vxx);
        }
        float mu = 0.0f, pi = 0.0f;
        if (param == 1) {
            mu = (float)((double)(pu[c] * pu[c] * prho[c]) / (1.0 + (double)(sumu * ptaus[c])));
            pi = (float)((double)(ppi[c] * ppi[c] * prho[c]) / (1.0 + (double)(sumpi * ptaup[c])));
        }
        if (param == 3) {
            mu = (float)((double)pu[c] / (1.0 + (double)(sumu * ptaus[c])));
            pi = (float)((double)(ppi[c] + 2 * pu[c]) / (1.0 + (double)(sumpi * ptaup[c])));
        }
        float sump = 0.0f;
        for (int l = 0; l < L; l++) sump += p[t0 + l];
        const float fjm = (float)((double)mu * 2.0 * (1.0 + (double)((float)L * ptaus[c])));
        const float gg = (float)((double)pi * (1.0 + (double)((float)L * ptaup[c])));
        sxx[c] += -(DT * (gg - fjm) * (gg - fjm) * vxx / gg) - (DT * (gg - fjm) * vyy) - (dthalbe * sump);
        if (ux)
            ux[c] = (float)((double)ux[c] + ((double)(-((gg - fjm) * (gg - fjm) * vxx / gg) - ((gg - fjm) * vyy)) -
                                             (0.5 * (double)sump)));
        sump = 0.0f;
        for (int l = 0; l < L; l++) {
            const float bjm = (float)((double)etajm[l] / (1.0 + ((double)etajm[l] * 0.5)));
            const float djm = (float)(2.0 * (double)mu * (double)ptaus[c]);
            const float e = pi * ptaup[c];
            p[t0 + l] = (float)((double)p[t0 + l] +
                                (double)bjm * (((double)(djm - e) * ((double)(fjm / gg) - 1.0) * (double)vxx) -
                                               (double)((djm - e) * vyy)));
            sump += p[t0 + l];
        }
        sxx[c] += (dthalbe * sump);
        if (ux) ux[c] = (float)((double)ux[c] + (0.5 * (double)sump));
    }
    if (sh) {
        syz[c] = 0.0f;
        if (uyz) uyz[c] = 0.0f;
        for (int m = 1; m <= g.fdoh; m++) {
            syz[c - m * s] = -syz[c + m * s];
            sxz[c - m * s] = -sxz[c + (m - 1) * s];
            if (uyz) uyz[c - m * s] = -uyz[c + m * s];
            if (uxz) uxz[c - m * s] = -uxz[c + (m - 1) * s];
        }
    }
}

// one source of psource: the samples at nt-1, nt, nt+1
struct PsrcI {
    int i, j;
    float sm, s0, sp;
};
// psource (src/psource.c:26-75), sources in order
__global__ void kc_psource(RG g, const PsrcI *src, int n, int nt, int ntot, int sw, int acoustic, float *sxx,
                           float *syy, float *spr) {
    if (blockIdx.x || threadIdx.x) return;
    const float DH = g.dh;
    for (int l = 0; l < n; l++) {
        const PsrcI q = src[l];
        float amp = 0.0f;
        if (sw == 0) {
            if (nt == 1) amp = (float)((double)q.sp / (2.0 * DH * DH));
            if ((nt > 1) && (nt < ntot)) amp = (float)((double)(q.sp - q.sm) / (2.0 * DH * DH));
            if (nt == ntot) amp = (float)((double)(-q.sm) / (2.0 * DH * DH));
        } else if (sw == 1) {
            amp = q.s0;
        } else {
            continue;
        }
        const long long c = ri(g, q.j, q.i);
        if (!acoustic) {
            sxx[c] = (float)((double)sxx[c] + 0.5 * (double)amp);
            syy[c] = (float)((double)syy[c] + 0.5 * (double)amp);
        } else {
            spr[c] += amp;
        }
    }
}

// seismo_ssg (src/seismo_ssg.c:26-140): the six samples of receiver itr
// (vx vy vz p curl div) into out[6*itr..]; the host copies those the
// reference writes for SEISMO
__global__ void kc_seismo(RG g, const int *rec, int ntr, int seismo, int acoustic, const float *vx, const float *vy,
                          const float *vz, const float *sxx, const float *syy, const float *sp, const float *pi,
                          const float *u, float *out) {
    const int itr = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (itr >= ntr) return;
    const int i = rec[2 * itr], j = rec[2 * itr + 1];
    const long long c = ri(g, j, i), s = g.stride;
    float *o = out + 6 * itr;
    if (vx) o[0] = vx[c];
    if (vy) o[1] = vy[c];
    if (vz) o[2] = vz[c];
    if (!acoustic) {
        if (sxx && syy) o[3] = -sxx[c] - syy[c];
    } else if (sp) {
        o[3] = -sp[c];
    }
    if ((seismo == 3 || seismo == 4) && vx && vy) {
        const float dhi = g.dt / g.dh;
        float vxx = 0, vyy = 0, vyx = 0, vxy = 0;
        for (int m = 1; m <= g.fdoh; m++) {
            vxx += g.hc[m] * (vx[c + m - 1] - vx[c - m]);
            vyy += g.hc[m] * (vy[c + (m - 1) * s] - vy[c - m * s]);
            vyx += g.hc[m] * (vy[c + m] - vy[c - m + 1]);
            vxy += g.hc[m] * (vx[c + m * s] - vx[c - (m - 1) * s]);
        }
        vxx *= dhi;
        vyy *= dhi;
        vyx *= dhi;
        vxy *= dhi;
        o[5] = (float)((double)(vxx + vyy) * sqrt((double)pi[c]));
        o[4] = !acoustic ? (float)((double)(vxy - vyx) * sqrt((double)u[c])) : 0.0f;
    }
}

// update_v_PML_SH (src/update_v_PML_SH.c:106-150 per written-out order, CPML on all orders)
template <int FD>
__global__ void kc_v_sh(RG g, Prof P, float *vz, float *vzp1, const float *sxz, const float *syz, const float *rjp,
                        float *ps_sxz_x, float *ps_syz_y) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    float sxz_x = sbwd<FD, false>(g, sxz, c, 1);
    float syz_y = sfwd<FD, false>(g, syz, c, s);
    sxz_x = pmlx(g, P, ps_sxz_x, j, i, PK_X, PA_X, PB_X, sxz_x);
    syz_y = pmly(g, P, ps_syz_y, j, i, PK_YH, PA_YH, PB_YH, syz_y);
    vzp1[c] = vz[c];
    vz[c] += rjp[c] * DT * (sxz_x + syz_y) / (DH);
}

// update_s_elastic_PML_SH (src/update_s_elastic_PML_SH.c:114-168) and
// update_s_visc_PML_SH (VISC, src/update_s_visc_PML_SH.c)
template <int FD, bool VISC>
__global__ void kc_s_sh(RG g, Prof P, const float *vz, float *sxz, float *syz, float *uxz, float *uyz,
                        const float *uipjp, const float *u, const float *rho, float *t, float *o, const float *bip,
                        const float *bjm, const float *cip, const float *cjm, const float *d, const float *dip,
                        const float *fipjp_v, const float *f_v, float *ps_vzx, float *ps_vzy, int param) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dhi = VISC ? (float)(1.0 / DH) : DT / DH;
    float vzx = sfwd<FD, false>(g, vz, c, 1) * dhi;
    float vzy = sbwd<FD, false>(g, vz, c, s) * dhi;
    vzx = pmlx(g, P, ps_vzx, j, i, PK_XH, PA_XH, PB_XH, vzx);
    vzy = pmly(g, P, ps_vzy, j, i, PK_Y, PA_Y, PB_Y, vzy);
    if (!VISC) {
        const float fipjp = uipjp[c];
        float f = 0.0f;
        if (param == 3) f = u[c];
        if (param == 1) f = rho[c] * u[c] * u[c];
        sxz[c] += (fipjp * vzx);
        syz[c] += (f * vzy);
        if (uxz) uxz[c] = (fipjp * vzx) / DT;
        if (uyz) uyz[c] = (f * vzy) / DT;
        return;
    }
    const float dthalbe = DT / 2.0;
    const int L = g.L;
    const long long t0 = c * L;
    float sumo = 0.0f, sumt = 0.0f;
    for (int l = 0; l < L; l++) {
        sumo += o[t0 + l];
        sumt += t[t0 + l];
    }
    sxz[c] += (fipjp_v[c] * vzx) + (dthalbe * sumo);
    syz[c] += (f_v[c] * vzy) + (dthalbe * sumt);
    sumt = sumo = 0.0f;
    for (int l = 0; l < L; l++) {
        o[t0 + l] = bip[l] * (o[t0 + l] * cip[l] - (dip[t0 + l] * vzx));
        t[t0 + l] = bjm[l] * (t[t0 + l] * cjm[l] - (d[t0 + l] * vzy));
        sumt += t[t0 + l];
        sumo += o[t0 + l];
    }
    sxz[c] += (dthalbe * sumo);
    syz[c] += (dthalbe * sumt);
}

// update_p_PML (src/update_p_PML.c:107-160 written out for 2-8, the rate in u;
// FDORDER 10/12 generic loop :275-287)
template <int FD, bool HI>
__global__ void kc_p(RG g, Prof P, const float *vx, const float *vy, float *sp, float *u, const float *pi,
                     const float *rho, float *ps_vxx, float *ps_vyy, int param) {
    CELL_IJ(g)
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dhi = DT / DH;
    if (HI) {
        const float vxx = sbwd<FD, true>(g, vx, c, 1), vyy = sbwd<FD, true>(g, vy, c, s);
        const float gg = pi[c] * DT;
        sp[c] += (gg * (vxx + vyy)) * dhi;
        return;
    }
    float vxx = sbwd<FD, false>(g, vx, c, 1) * dhi;
    float vyy = sbwd<FD, false>(g, vy, c, s) * dhi;
    vxx = pmlx(g, P, ps_vxx, j, i, PK_X, PA_X, PB_X, vxx);
    vyy = pmly(g, P, ps_vyy, j, i, PK_Y, PA_Y, PB_Y, vyy);
    float gg = 0.0f;
    if (param == 1) gg = rho[c] * (pi[c] * pi[c]);
    sp[c] += gg * (vxx + vyy);
    if (u) u[c] = (gg / DT) * (vxx + vyy);
}

// update_p_visc_PML (src/update_p_visc_PML.c:61-146 at FDORDER 2, with CPML
// on all four velocity derivatives; :148-182 for every other order, the
// generic loop from zero without CPML)
template <int FD>
__global__ void kc_p_visc(RG g, Prof P, const float *vx, const float *vy, float *sp, float *p, const float *gv,
                          const float *bjm, const float *cjm, const float *e, float *ps_vxx, float *ps_vyy,
                          float *ps_vxy, float *ps_vyx) {
    CELL_IJ(g)
    constexpr bool Z0 = FD != 1;
    const long long s = g.stride;
    const float DT = g.dt, DH = g.dh;
    const float dhi = 1.0 / DH, dthalbe = DT / 2.0;  // src/update_p_visc_PML.c:49-51
    float vxx = sbwd<FD, Z0>(g, vx, c, 1) * dhi;
    float vyy = sbwd<FD, Z0>(g, vy, c, s) * dhi;
    if (FD == 1 && ps_vxx) {
        float vyx = sfwd<FD, false>(g, vy, c, 1) * dhi;
        float vxy = sfwd<FD, false>(g, vx, c, s) * dhi;
        vxx = pmlx(g, P, ps_vxx, j, i, PK_X, PA_X, PB_X, vxx);
        vyx = pmlx(g, P, ps_vyx, j, i, PK_XH, PA_XH, PB_XH, vyx);
        vyy = pmly(g, P, ps_vyy, j, i, PK_Y, PA_Y, PB_Y, vyy);
        vxy = pmly(g, P, ps_vxy, j, i, PK_YH, PA_YH, PB_YH, vxy);
        (void)vyx, (void)vxy;
    }
    const int L = g.L;
    const long long t0 = c * L;
    float sump = 0.0f;
    for (int l = 0; l < L; l++) sump += p[t0 + l];
    sp[c] += (gv[c] * (vxx + vyy)) + (dthalbe * sump);
    sump = 0.0f;
    for (int l = 0; l < L; l++) {
        p[t0 + l] = bjm[l] * (p[t0 + l] * cjm[l] - (e[t0 + l] * (vxx + vyy)));
        sump += p[t0 + l];
    }
    sp[c] += (dthalbe * sump);
}

// surface_acoustic_PML (src/surface_acoustic_PML.c:36-42): zero at the
// surface, imaged above it
__global__ void kc_surf_ac(RG g, int j, float *sp) {
    const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i > g.nx) return;
    const long long c = ri(g, j, i), s = g.stride;
    sp[c] = 0.0f;
    for (int m = 1; m <= g.fdoh; m++) sp[c - m * s] = -sp[c + m * s];
}

}  // namespace

// ---------------------------------------------------------------------------
// entry points
namespace {

void *g_small = nullptr;  // per-call source / receiver tables
size_t g_small_bytes = 0;
void *small_up(const void *h, size_t bytes) {
    if (g_small_bytes < bytes) {
        if (g_small) CC(cudaFree(g_small));
        CC(cudaMalloc(&g_small, bytes));
        g_small_bytes = bytes;
    }
    CC(cudaMemcpyAsync(g_small, h, bytes, cudaMemcpyHostToDevice, stream()));
    return g_small;
}
float *g_small_out = nullptr;
size_t g_small_out_bytes = 0;
float *small_out(size_t bytes) {
    if (g_small_out_bytes < bytes) {
        if (g_small_out) CC(cudaFree(g_small_out));
        CC(cudaMalloc((void **)&g_small_out, bytes));
        g_small_out_bytes = bytes;
    }
    CC(cudaMemsetAsync(g_small_out, 0, bytes, stream()));
    return g_small_out;
}
// a 1-based vector(1,L) of the driver on the device (index 0..L-1)
float *vec_up(const float *v) { return v ? up(&v[1], (size_t)L * sizeof(float)) : nullptr; }

void check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) die(what, e);
}

// sources of update_v_PML / update_v_acoustic_PML / update_v_PML_SH at sample nt.
// Only the forward (sw 0) reads the azimuth and type rows 7 and 8: the
// adjoint's sources are the receivers, a matrix(1,6,...) of positions only
// (src/IFOS2D.c:2183), as src/update_v_PML.c:552-578 reads them.
std::vector<SrcI> gather_src(float **srcpos_loc, float **signals, float **signals1, int nsrc, int nt, int sw) {
    std::vector<SrcI> v;
    for (int l = 1; l <= nsrc; l++) {
        SrcI q{};
        q.i = (int)srcpos_loc[1][l];
        q.j = (int)srcpos_loc[2][l];
        q.type = sw == 0 ? (int)srcpos_loc[8][l] : 0;
        // azi_rad = srcpos_loc[7][l]*PI/180, a float, then sin/cos of it (src/update_v_PML.c:556,562)
        const float azi = sw == 0 ? (float)(srcpos_loc[7][l] * kPi / 180) : 0.0f;
        q.sn = std::sin((double)azi);
        q.cs = std::cos((double)azi);
        q.s = signals ? signals[l][nt] : 0.0f;
        q.s1 = signals1 ? signals1[l][nt] : 0.0f;
        v.push_back(q);
    }
    return v;
}

}  // namespace

extern "C" void update_v_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vx, float **vxp1, float **vxm1,
                             float **vy, float **vyp1, float **vym1, float **uttx, float **utty, float **sxx,
                             float **syy, float **sxy, float **rip, float **rjp, float **srcpos_loc, float **signals,
                             float **signals1, int nsrc, float **absorb_coeff, float *hc, int infoout, int sw,
                             float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half, float *b_x_half,
                             float *K_y, float *a_y, float *b_y, float *K_y_half, float *a_y_half, float *b_y_half,
                             float **psi_sxx_x, float **psi_syy_y, float **psi_sxy_y, float **psi_sxy_x) {
    (void)vxm1, (void)vym1, (void)uttx, (void)utty, (void)absorb_coeff, (void)infoout;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool hi = FDORDER >= 10;
    const bool pml = !hi && FW > 0;
    float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_vxp1 = hi ? nullptr : up(fblk(vxp1), fb), *d_vyp1 = hi ? nullptr : up(fblk(vyp1), fb);
    const float *d_sxx = up(fblk(sxx), fb), *d_syy = up(fblk(syy), fb), *d_sxy = up(fblk(sxy), fb);
    const float *d_rip = up(fblk(rip), fb), *d_rjp = up(fblk(rjp), fb);
    float *ps[4] = {nullptr, nullptr, nullptr, nullptr};
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps[0] = up(pblk(psi_sxx_x), psix_bytes());
        ps[1] = up(pblk(psi_syy_y), psiy_bytes());
        ps[2] = up(pblk(psi_sxy_y), psiy_bytes());
        ps[3] = up(pblk(psi_sxy_x), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, {
            if (hi) kc_v<FD, true, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_vxp1, d_vyp1, d_sxx, d_syy, d_sxy, d_rip, d_rjp, ps[0], ps[1], ps[2], ps[3], sw, VELOCITY);
            else kc_v<FD, false, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_vxp1, d_vyp1, d_sxx, d_syy, d_sxy, d_rip, d_rjp, ps[0], ps[1], ps[2], ps[3], sw, VELOCITY);
        });
        check_launch("update_v_PML");
    }
    if (nsrc > 0 && (sw == 0 || sw == 1)) {
        const std::vector<SrcI> src = gather_src(srcpos_loc, signals, signals1, nsrc, nt, sw);
        const SrcI *d_src = (const SrcI *)small_up(src.data(), src.size() * sizeof(SrcI));
        kc_src_v<<<1, 1, 0, stream()>>>(g, d_src, nsrc, d_vx, d_vy, nullptr, d_rip, d_rjp, sw, ADJOINT_TYPE);
        check_launch("update_v_PML sources");
        // the reference sets the global SOURCE_TYPE from each source it visits (src/update_v_PML.c:558)
        if (sw == 0) SOURCE_TYPE = (int)srcpos_loc[8][nsrc];
    }
    down(fblk(vx), fb);
    down(fblk(vy), fb);
    if (!hi && (sw == 0 || sw == 1)) {
        down(fblk(vxp1), fb);
        down(fblk(vyp1), fb);
    }
    if (pml) {
        down(pblk(psi_sxx_x), psix_bytes());
        down(pblk(psi_syy_y), psiy_bytes());
        down(pblk(psi_sxy_y), psiy_bytes());
        down(pblk(psi_sxy_x), psix_bytes());
    }
    finish();
}

extern "C" void update_v_acoustic_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vx, float **vxp1,
                                      float **vxm1, float **vy, float **vyp1, float **vym1, float **sp, float **rip,
                                      float **rjp, float **srcpos_loc, float **signals, float **signals1, int nsrc,
                                      float **absorb_coeff, float *hc, int infoout, int sw, float *K_x_half,
                                      float *a_x_half, float *b_x_half, float *K_y_half, float *a_y_half,
                                      float *b_y_half, float **psi_sxx_x, float **psi_syy_y) {
    (void)vxm1, (void)vym1, (void)absorb_coeff, (void)infoout;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool hi = FDORDER >= 10;
    const bool pml = !hi && FW > 0;
    float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_vxp1 = hi ? nullptr : up(fblk(vxp1), fb), *d_vyp1 = hi ? nullptr : up(fblk(vyp1), fb);
    const float *d_sp = up(fblk(sp), fb);
    const float *d_rip = up(fblk(rip), fb), *d_rjp = up(fblk(rjp), fb);
    float *ps_x = nullptr, *ps_y = nullptr;
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps_x = up(pblk(psi_sxx_x), psix_bytes());
        ps_y = up(pblk(psi_syy_y), psiy_bytes());
        float *const pv[12] = {nullptr, nullptr, nullptr, K_x_half, a_x_half, b_x_half,
                               nullptr, nullptr, nullptr, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, {
            if (hi) kc_v<FD, true, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_vxp1, d_vyp1, d_sp, d_sp, d_sp, d_rip, d_rjp, ps_x, ps_y, nullptr, nullptr, sw, VELOCITY);
            else kc_v<FD, false, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_vxp1, d_vyp1, d_sp, d_sp, d_sp, d_rip, d_rjp, ps_x, ps_y, nullptr, nullptr, sw, VELOCITY);
        });
        check_launch("update_v_acoustic_PML");
    }
    if (nsrc > 0 && (sw == 0 || sw == 1)) {
        const std::vector<SrcI> src = gather_src(srcpos_loc, signals, signals1, nsrc, nt, sw);
        const SrcI *d_src = (const SrcI *)small_up(src.data(), src.size() * sizeof(SrcI));
        kc_src_v<<<1, 1, 0, stream()>>>(g, d_src, nsrc, d_vx, d_vy, nullptr, d_rip, d_rjp, sw, ADJOINT_TYPE);
        check_launch("update_v_acoustic_PML sources");
        if (sw == 0) SOURCE_TYPE = (int)srcpos_loc[8][nsrc];
    }
    down(fblk(vx), fb);
    down(fblk(vy), fb);
    if (!hi && (sw == 0 || sw == 1)) {
        down(fblk(vxp1), fb);
        down(fblk(vyp1), fb);
    }
    if (pml) {
        down(pblk(psi_sxx_x), psix_bytes());
        down(pblk(psi_syy_y), psiy_bytes());
    }
    finish();
}

extern "C" void update_s_elastic_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux,
                                     float **uy, float **uxy, float **uyx, float **sxx, float **syy, float **sxy,
                                     float **pi, float **u, float **uipjp, float **absorb_coeff, float **rho,
                                     float *hc, int infoout, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                     float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                                     float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx,
                                     float **psi_vyy, float **psi_vxy, float **psi_vyx) {
    (void)uyx, (void)absorb_coeff, (void)infoout;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool hi = FDORDER >= 10;
    const bool pml = !hi && FW > 0;
    const float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_ux = up(fblk(ux), fb), *d_uy = up(fblk(uy), fb), *d_uxy = hi ? nullptr : up(fblk(uxy), fb);
    float *d_sxx = up(fblk(sxx), fb), *d_syy = up(fblk(syy), fb), *d_sxy = up(fblk(sxy), fb);
    const float *d_pi = up(fblk(pi), fb), *d_u = up(fblk(u), fb), *d_uipjp = up(fblk(uipjp), fb);
    const float *d_rho = up(fblk(rho), fb);
    float *ps[4] = {nullptr, nullptr, nullptr, nullptr};
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps[0] = up(pblk(psi_vxx), psix_bytes());
        ps[1] = up(pblk(psi_vyy), psiy_bytes());
        ps[2] = up(pblk(psi_vxy), psiy_bytes());
        ps[3] = up(pblk(psi_vyx), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, {
            if (hi) kc_s_el<FD, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_ux, d_uy, d_uxy, d_sxx, d_syy, d_sxy, d_pi, d_u, d_uipjp, d_rho, ps[0], ps[1], ps[2], ps[3], PARAMETERIZATION);
            else kc_s_el<FD, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_ux, d_uy, d_uxy, d_sxx, d_syy, d_sxy, d_pi, d_u, d_uipjp, d_rho, ps[0], ps[1], ps[2], ps[3], PARAMETERIZATION);
        });
        check_launch("update_s_elastic_PML");
    }
    down(fblk(sxx), fb);
    down(fblk(syy), fb);
    down(fblk(sxy), fb);
    down(fblk(ux), fb);
    down(fblk(uy), fb);
    if (!hi) down(fblk(uxy), fb);
    if (pml) {
        down(pblk(psi_vxx), psix_bytes());
        down(pblk(psi_vyy), psiy_bytes());
        down(pblk(psi_vxy), psiy_bytes());
        down(pblk(psi_vyx), psix_bytes());
    }
    finish();
}

extern "C" void update_s_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux, float **uy,
                                  float **uxy, float **uyx, float **sxx, float **syy, float **sxy, float **pi,
                                  float **u, float **uipjp, float **rho, float *hc, int infoout, float ***r,
                                  float ***p, float ***q, float **fipjp, float **f, float **g_, float *bip,
                                  float *bjm, float *cip, float *cjm, float ***d, float ***e, float ***dip,
                                  float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half,
                                  float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                                  float *a_y_half, float *b_y_half, float **psi_vxx, float **psi_vyy,
                                  float **psi_vxy, float **psi_vyx) {
    (void)uyx, (void)pi, (void)u, (void)uipjp, (void)rho, (void)infoout;
    const size_t fb = field_bytes(), tb = tensor_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool hi = FDORDER >= 10;
    const bool pml = !hi && FW > 0;
    const float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_ux = hi ? nullptr : up(fblk(ux), fb), *d_uy = hi ? nullptr : up(fblk(uy), fb);
    float *d_uxy = hi ? nullptr : up(fblk(uxy), fb);
    float *d_sxx = up(fblk(sxx), fb), *d_syy = up(fblk(syy), fb), *d_sxy = up(fblk(sxy), fb);
    float *d_r = up(tblk(r), tb), *d_p = up(tblk(p), tb), *d_q = up(tblk(q), tb);
    const float *d_d = up(tblk(d), tb), *d_e = up(tblk(e), tb), *d_dip = up(tblk(dip), tb);
    const float *d_fipjp = up(fblk(fipjp), fb), *d_f = up(fblk(f), fb), *d_g = up(fblk(g_), fb);
    const float *d_bip = vec_up(bip), *d_bjm = vec_up(bjm), *d_cip = vec_up(cip), *d_cjm = vec_up(cjm);
    float *ps[4] = {nullptr, nullptr, nullptr, nullptr};
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps[0] = up(pblk(psi_vxx), psix_bytes());
        ps[1] = up(pblk(psi_vyy), psiy_bytes());
        ps[2] = up(pblk(psi_vxy), psiy_bytes());
        ps[3] = up(pblk(psi_vyx), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, {
            if (hi) kc_s_visc<FD, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_ux, d_uy, d_uxy, d_sxx, d_syy, d_sxy, d_r, d_p, d_q, d_fipjp, d_f, d_g, d_bip, d_bjm, d_cip, d_cjm, d_d, d_e, d_dip, ps[0], ps[1], ps[2], ps[3]);
            else kc_s_visc<FD, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_ux, d_uy, d_uxy, d_sxx, d_syy, d_sxy, d_r, d_p, d_q, d_fipjp, d_f, d_g, d_bip, d_bjm, d_cip, d_cjm, d_d, d_e, d_dip, ps[0], ps[1], ps[2], ps[3]);
        });
        check_launch("update_s_visc_PML");
    }
    down(fblk(sxx), fb);
    down(fblk(syy), fb);
    down(fblk(sxy), fb);
    down(tblk(r), tb);
    down(tblk(p), tb);
    down(tblk(q), tb);
    if (!hi) {
        down(fblk(ux), fb);
        down(fblk(uy), fb);
        down(fblk(uxy), fb);
    }
    if (pml) {
        down(pblk(psi_vxx), psix_bytes());
        down(pblk(psi_vyy), psiy_bytes());
        down(pblk(psi_vxy), psiy_bytes());
        down(pblk(psi_vyx), psix_bytes());
    }
    finish();
}

extern "C" void surface_elastic_PML(int ndepth, float **vx, float **vy, float **sxx, float **syy, float **sxy,
                                    float **syz, float **pi, float **u, float **rho, float *hc, float *K_x,
                                    float *a_x, float *b_x, float **psi_vxx, float **ux, float **uy, float **uxy,
                                    float **uyz, float **sxz, float **uxz) {
    const size_t fb = field_bytes();
    const RG g = make_rg(1, NX, 1, NY, hc);
    const int psv = WAVETYPE == 1 || WAVETYPE == 3, sh = WAVETYPE == 2 || WAVETYPE == 3;
    float *d[13] = {};
    if (psv) {
        d[0] = up(fblk(vx), fb);
        d[1] = up(fblk(vy), fb);
        d[2] = up(fblk(sxx), fb);
        d[3] = up(fblk(syy), fb);
        d[4] = up(fblk(sxy), fb);
        d[5] = up(fblk(ux), fb);
        d[6] = up(fblk(uy), fb);
        d[7] = up(fblk(uxy), fb);
        d[8] = up(fblk(pi), fb);
        d[9] = up(fblk(u), fb);
        d[10] = up(fblk(rho), fb);
    }
    float *s_syz = nullptr, *s_sxz = nullptr, *s_uyz = nullptr, *s_uxz = nullptr;
    if (sh) {
        s_syz = up(fblk(syz), fb);
        s_sxz = up(fblk(sxz), fb);
        s_uyz = up(fblk(uyz), fb);
        s_uxz = up(fblk(uxz), fb);
    }
    float *ps = nullptr;
    Prof P{nullptr, 2 * FW};
    if (psv && FW > 0 && !BOUNDARY) {
        ps = up(pblk(psi_vxx), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x};
        P = upload_prof(pv);
    }
    kc_surf_el<<<(NX + 127) / 128, 128, 0, stream()>>>(g, P, ndepth, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7],
                                                        d[8], d[9], d[10], ps, s_syz, s_sxz, s_uyz, s_uxz,
                                                        PARAMETERIZATION, psv, sh);
    check_launch("surface_elastic_PML");
    if (psv) {
        down(fblk(sxx), fb);
        down(fblk(syy), fb);
        down(fblk(sxy), fb);
        down(fblk(ux), fb);
        down(fblk(uy), fb);
        down(fblk(uxy), fb);
        if (ps) down(pblk(psi_vxx), psix_bytes());
    }
    if (sh) {
        down(fblk(syz), fb);
        down(fblk(sxz), fb);
        down(fblk(uyz), fb);
        down(fblk(uxz), fb);
    }
    finish();
}

extern "C" void surface_PML(int ndepth, float **vx, float **vy, float **sxx, float **syy, float **sxy, float **syz,
                            float ***p, float ***q, float **ppi, float **pu, float **prho, float **ptaup,
                            float **ptaus, float *etajm, float *peta, float *hc, float *K_x, float *a_x, float *b_x,
                            float **psi_vxx, float **ux, float **uy, float **uxy, float **uyz, float **sxz,
                            float **uxz) {
    const size_t fb = field_bytes(), tb = tensor_bytes();
    const RG g = make_rg(1, NX, 1, NY, hc);
    const int psv = WAVETYPE == 1 || WAVETYPE == 3, sh = WAVETYPE == 2 || WAVETYPE == 3;
    float sumu = 0.0f, sumpi = 0.0f;
    float *d_eta = nullptr;
    float *d[15] = {};
    if (psv) {
        // relaxation sums as src/surface_PML.c:44-57 forms them
        std::vector<float> pts((size_t)L + 1);
        for (int l = 1; l <= L; l++) pts[l] = 1.0 / (2.0 * kPi * FL[l]);
        const float ws = 2.0 * kPi * F_REF;
        for (int l = 1; l <= L; l++) {
            sumu = sumu + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
            sumpi = sumpi + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        }
        for (int l = 1; l <= L; l++) etajm[l] = peta[l];
        d_eta = vec_up(etajm);
        d[0] = up(fblk(vx), fb);
        d[1] = up(fblk(vy), fb);
        d[2] = up(fblk(sxx), fb);
        d[3] = up(fblk(syy), fb);
        d[4] = up(fblk(sxy), fb);
        d[5] = up(fblk(ux), fb);
        d[6] = up(fblk(uy), fb);
        d[7] = up(fblk(uxy), fb);
        d[8] = up(tblk(p), tb);
        d[9] = up(tblk(q), tb);
        d[10] = up(fblk(ppi), fb);
        d[11] = up(fblk(pu), fb);
        d[12] = up(fblk(prho), fb);
        d[13] = up(fblk(ptaup), fb);
        d[14] = up(fblk(ptaus), fb);
    }
    float *s_syz = nullptr, *s_sxz = nullptr, *s_uyz = nullptr, *s_uxz = nullptr;
    if (sh) {
        s_syz = up(fblk(syz), fb);
        s_sxz = up(fblk(sxz), fb);
        s_uyz = up(fblk(uyz), fb);
        s_uxz = up(fblk(uxz), fb);
    }
    float *ps = nullptr;
    Prof P{nullptr, 2 * FW};
    if (psv && FW > 0 && !BOUNDARY) {
        ps = up(pblk(psi_vxx), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x};
        P = upload_prof(pv);
    }
    kc_surf_visc<<<(NX + 127) / 128, 128, 0, stream()>>>(
        g, P, ndepth, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], d[10], d[11], d[12], d[13], d[14],
        d_eta, sumu, sumpi, ps, s_syz, s_sxz, s_uyz, s_uxz, PARAMETERIZATION, psv, sh);
    check_launch("surface_PML");
    if (psv) {
        down(fblk(sxx), fb);
        down(fblk(syy), fb);
        down(fblk(sxy), fb);
        down(fblk(ux), fb);
        down(fblk(uy), fb);
        down(fblk(uxy), fb);
        down(tblk(p), tb);
        down(tblk(q), tb);
        if (ps) down(pblk(psi_vxx), psix_bytes());
    }
    if (sh) {
        down(fblk(syz), fb);
        down(fblk(sxz), fb);
        down(fblk(uyz), fb);
        down(fblk(uxz), fb);
    }
    finish();
}

extern "C" void psource(int nt, float **sxx, float **syy, float **sp, float **srcpos_loc, float **signals, int nsrc,
                        int sw) {
    if (nsrc <= 0 || (sw != 0 && sw != 1)) return;
    const size_t fb = field_bytes();
    const RG g = make_rg(1, NX, 1, NY, nullptr);
    std::vector<PsrcI> src;
    for (int l = 1; l <= nsrc; l++) {
        PsrcI q{};
        q.i = (int)srcpos_loc[1][l];
        q.j = (int)srcpos_loc[2][l];
        q.sm = (nt - 1 >= 1 && nt - 1 <= NT) ? signals[l][nt - 1] : 0.0f;
        q.s0 = (nt >= 1 && nt <= NT) ? signals[l][nt] : 0.0f;
        q.sp = (nt + 1 >= 1 && nt + 1 <= NT) ? signals[l][nt + 1] : 0.0f;
        src.push_back(q);
    }
    float *d_sxx = nullptr, *d_syy = nullptr, *d_sp = nullptr;
    if (!ACOUSTIC) {
        d_sxx = up(fblk(sxx), fb);
        d_syy = up(fblk(syy), fb);
    } else {
        d_sp = up(fblk(sp), fb);
    }
    const PsrcI *d_src = (const PsrcI *)small_up(src.data(), src.size() * sizeof(PsrcI));
    kc_psource<<<1, 1, 0, stream()>>>(g, d_src, nsrc, nt, NT, sw, ACOUSTIC, d_sxx, d_syy, d_sp);
    check_launch("psource");
    if (!ACOUSTIC) {
        down(fblk(sxx), fb);
        down(fblk(syy), fb);
    } else {
        down(fblk(sp), fb);
    }
    finish();
}

extern "C" void seismo_ssg(int lsamp, int ntr, int **recpos, float **sectionvx, float **sectionvy,
                           float **sectionvz, float **sectionp, float **sectioncurl, float **sectiondiv, float **vx,
                           float **vy, float **vz, float **sxx, float **syy, float **sp, float **pi, float **u,
                           float *hc) {
    if (ntr <= 0) return;
    const size_t fb = field_bytes();
    const RG g = make_rg(1, NX, 1, NY, hc);
    std::vector<int> rec((size_t)2 * ntr);
    for (int itr = 1; itr <= ntr; itr++) {
        rec[2 * (itr - 1)] = recpos[1][itr];
        rec[2 * (itr - 1) + 1] = recpos[2][itr];
    }
    const int psv = WAVETYPE == 1 || WAVETYPE == 3, sh = WAVETYPE == 2 || WAVETYPE == 3;
    const bool curl = SEISMO == 3 || SEISMO == 4;
    const float *d_vx = psv || SEISMO == 4 ? up(fblk(vx), fb) : nullptr;
    const float *d_vy = psv || SEISMO == 4 ? up(fblk(vy), fb) : nullptr;
    const float *d_vz = sh ? up(fblk(vz), fb) : nullptr;
    const float *d_sxx = !ACOUSTIC ? up(fblk(sxx), fb) : nullptr, *d_syy = !ACOUSTIC ? up(fblk(syy), fb) : nullptr;
    const float *d_sp = ACOUSTIC ? up(fblk(sp), fb) : nullptr;
    const float *d_pi = curl ? up(fblk(pi), fb) : nullptr;
    const float *d_u = curl && !ACOUSTIC ? up(fblk(u), fb) : nullptr;
    const int *d_rec = (const int *)small_up(rec.data(), rec.size() * sizeof(int));
    float *d_out = small_out((size_t)6 * ntr * sizeof(float));
    kc_seismo<<<(ntr + 127) / 128, 128, 0, stream()>>>(g, d_rec, ntr, SEISMO, ACOUSTIC, d_vx, d_vy, d_vz, d_sxx,
                                                        d_syy, d_sp, d_pi, d_u, d_out);
    check_launch("seismo_ssg");
    std::vector<float> out((size_t)6 * ntr);
    CC(cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(float), cudaMemcpyDeviceToHost, stream()));
    finish();
    // the samples src/seismo_ssg.c writes for each SEISMO mode
    const int ins = lsamp;
    for (int itr = 1; itr <= ntr; itr++) {
        const float *o = &out[(size_t)6 * (itr - 1)];
        switch (SEISMO) {
            case 1:
                if (psv) {
                    sectionvx[itr][ins] = o[0];
                    sectionvy[itr][ins] = o[1];
                }
                if (sh) sectionvz[itr][ins] = o[2];
                break;
            case 2: sectionp[itr][ins] = o[3]; break;
            case 3:
                sectiondiv[itr][ins] = o[5];
                sectioncurl[itr][ins] = o[4];
                break;
            case 4:
                sectiondiv[itr][ins] = o[5];
                sectioncurl[itr][ins] = o[4];
                sectionvx[itr][ins] = o[0];
                sectionvy[itr][ins] = o[1];
                if (sh) sectionvz[itr][ins] = o[2];
                sectionp[itr][ins] = o[3];
                break;
            case 5:
                if (psv) {
                    sectionvx[itr][ins] = o[0];
                    sectionvy[itr][ins] = o[1];
                    sectionp[itr][ins] = o[3];
                }
                if (sh) sectionvz[itr][ins] = o[2];
                break;
        }
    }
}

extern "C" void update_v_PML_SH(int nx1, int nx2, int ny1, int ny2, int nt, float **vz, float **vzp1, float **vzm1,
                                float **sxz, float **syz, float **rjp, float **srcpos_loc, float **signals,
                                float **signals1, int nsrc, float **absorb_coeff, float *hc, int infoout, int sw,
                                float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half,
                                float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                                float *a_y_half, float *b_y_half, float **psi_sxz_x, float **psi_syz_y) {
    (void)vzm1, (void)absorb_coeff, (void)infoout;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool pml = FW > 0;
    float *d_vz = up(fblk(vz), fb), *d_vzp1 = up(fblk(vzp1), fb);
    const float *d_sxz = up(fblk(sxz), fb), *d_syz = up(fblk(syz), fb), *d_rjp = up(fblk(rjp), fb);
    float *ps_x = nullptr, *ps_y = nullptr;
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps_x = up(pblk(psi_sxz_x), psix_bytes());
        ps_y = up(pblk(psi_syz_y), psiy_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, kc_v_sh<FD><<<gr, kBlk, 0, stream()>>>(g, P, d_vz, d_vzp1, d_sxz, d_syz, d_rjp, ps_x, ps_y));
        check_launch("update_v_PML_SH");
    }
    if (nsrc > 0 && (sw == 0 || sw == 1)) {
        const std::vector<SrcI> src = gather_src(srcpos_loc, signals, signals1, nsrc, nt, sw);
        const SrcI *d_src = (const SrcI *)small_up(src.data(), src.size() * sizeof(SrcI));
        kc_src_v<<<1, 1, 0, stream()>>>(g, d_src, nsrc, nullptr, nullptr, d_vz, nullptr, d_rjp, sw, ADJOINT_TYPE);
        check_launch("update_v_PML_SH sources");
    }
    down(fblk(vz), fb);
    down(fblk(vzp1), fb);
    if (pml) {
        down(pblk(psi_sxz_x), psix_bytes());
        down(pblk(psi_syz_y), psiy_bytes());
    }
    finish();
}

extern "C" void update_s_elastic_PML_SH(int nx1, int nx2, int ny1, int ny2, float **vz, float **sxz, float **syz,
                                        float **uxz, float **uyz, float *hc, int infoout, float *K_x, float *a_x,
                                        float *b_x, float *K_x_half, float *a_x_half, float *b_x_half, float *K_y,
                                        float *a_y, float *b_y, float *K_y_half, float *a_y_half, float *b_y_half,
                                        float **psi_vzx, float **psi_vzy, float **uipjp, float **u, float **rho) {
    (void)infoout;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool pml = FW > 0;
    const float *d_vz = up(fblk(vz), fb);
    float *d_sxz = up(fblk(sxz), fb), *d_syz = up(fblk(syz), fb);
    float *d_uxz = up(fblk(uxz), fb), *d_uyz = up(fblk(uyz), fb);
    const float *d_uipjp = up(fblk(uipjp), fb), *d_u = up(fblk(u), fb), *d_rho = up(fblk(rho), fb);
    float *ps_x = nullptr, *ps_y = nullptr;
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps_x = up(pblk(psi_vzx), psix_bytes());
        ps_y = up(pblk(psi_vzy), psiy_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, kc_s_sh<FD, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vz, d_sxz, d_syz, d_uxz, d_uyz, d_uipjp, d_u, d_rho, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, ps_x, ps_y, PARAMETERIZATION));
        check_launch("update_s_elastic_PML_SH");
    }
    down(fblk(sxz), fb);
    down(fblk(syz), fb);
    down(fblk(uxz), fb);
    down(fblk(uyz), fb);
    if (pml) {
        down(pblk(psi_vzx), psix_bytes());
        down(pblk(psi_vzy), psiy_bytes());
    }
    finish();
}

extern "C" void update_s_visc_PML_SH(int nx1, int nx2, int ny1, int ny2, float **vz, float **sxz, float **syz,
                                     float ***t, float ***o, float *bip, float *bjm, float *cip, float *cjm,
                                     float ***d, float ***dip, float **fipjp, float **f, float *hc, int infoout,
                                     float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half,
                                     float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                                     float *a_y_half, float *b_y_half, float **psi_vzx, float **psi_vzy) {
    (void)infoout;
    const size_t fb = field_bytes(), tb = tensor_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool pml = FW > 0;
    const float *d_vz = up(fblk(vz), fb);
    float *d_sxz = up(fblk(sxz), fb), *d_syz = up(fblk(syz), fb);
    float *d_t = up(tblk(t), tb), *d_o = up(tblk(o), tb);
    const float *d_d = up(tblk(d), tb), *d_dip = up(tblk(dip), tb);
    const float *d_fipjp = up(fblk(fipjp), fb), *d_f = up(fblk(f), fb);
    const float *d_bip = vec_up(bip), *d_bjm = vec_up(bjm), *d_cip = vec_up(cip), *d_cjm = vec_up(cjm);
    float *ps_x = nullptr, *ps_y = nullptr;
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps_x = up(pblk(psi_vzx), psix_bytes());
        ps_y = up(pblk(psi_vzy), psiy_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, kc_s_sh<FD, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vz, d_sxz, d_syz, nullptr, nullptr, nullptr, nullptr, nullptr, d_t, d_o, d_bip, d_bjm, d_cip, d_cjm, d_d, d_dip, d_fipjp, d_f, ps_x, ps_y, PARAMETERIZATION));
        check_launch("update_s_visc_PML_SH");
    }
    down(fblk(sxz), fb);
    down(fblk(syz), fb);
    down(tblk(t), tb);
    down(tblk(o), tb);
    if (pml) {
        down(pblk(psi_vzx), psix_bytes());
        down(pblk(psi_vzy), psiy_bytes());
    }
    finish();
}

extern "C" void update_p_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **sp, float **u,
                             float **pi, float **absorb_coeff, float **rho, float *hc, int infoout, float *K_x,
                             float *a_x, float *b_x, float *K_x_half, float *a_x_half, float *b_x_half, float *K_y,
                             float *a_y, float *b_y, float *K_y_half, float *a_y_half, float *b_y_half,
                             float **psi_vxx, float **psi_vyy, float **psi_vxy, float **psi_vyx) {
    (void)absorb_coeff, (void)infoout, (void)psi_vxy, (void)psi_vyx;
    const size_t fb = field_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool hi = FDORDER >= 10;
    const bool pml = !hi && FW > 0;
    const float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_sp = up(fblk(sp), fb), *d_u = hi ? nullptr : up(fblk(u), fb);
    const float *d_pi = up(fblk(pi), fb), *d_rho = up(fblk(rho), fb);
    float *ps_x = nullptr, *ps_y = nullptr;
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps_x = up(pblk(psi_vxx), psix_bytes());
        ps_y = up(pblk(psi_vyy), psiy_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, {
            if (hi) kc_p<FD, true><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_sp, d_u, d_pi, d_rho, ps_x, ps_y, PARAMETERIZATION);
            else kc_p<FD, false><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_sp, d_u, d_pi, d_rho, ps_x, ps_y, PARAMETERIZATION);
        });
        check_launch("update_p_PML");
    }
    down(fblk(sp), fb);
    if (!hi) down(fblk(u), fb);
    if (pml) {
        down(pblk(psi_vxx), psix_bytes());
        down(pblk(psi_vyy), psiy_bytes());
    }
    finish();
}

extern "C" void update_p_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **sp,
                                  float **pi, float **rho, float *hc, int infoout, float ***p, float **g_, float *bjm,
                                  float *cjm, float ***e, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                  float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                                  float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx,
                                  float **psi_vyy, float **psi_vxy, float **psi_vyx) {
    (void)pi, (void)rho, (void)infoout;
    const size_t fb = field_bytes(), tb = tensor_bytes();
    const RG g = make_rg(nx1, nx2, ny1, ny2, hc);
    const bool pml = FDORDER == 2 && FW > 0;
    const float *d_vx = up(fblk(vx), fb), *d_vy = up(fblk(vy), fb);
    float *d_sp = up(fblk(sp), fb), *d_p = up(tblk(p), tb);
    const float *d_g = up(fblk(g_), fb), *d_e = up(tblk(e), tb);
    const float *d_bjm = vec_up(bjm), *d_cjm = vec_up(cjm);
    float *ps[4] = {nullptr, nullptr, nullptr, nullptr};
    Prof P{nullptr, 2 * FW};
    if (pml) {
        ps[0] = up(pblk(psi_vxx), psix_bytes());
        ps[1] = up(pblk(psi_vyy), psiy_bytes());
        ps[2] = up(pblk(psi_vxy), psiy_bytes());
        ps[3] = up(pblk(psi_vyx), psix_bytes());
        float *const pv[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
        P = upload_prof(pv);
    }
    if (nx2 >= nx1 && ny2 >= ny1) {
        const dim3 gr = grid_of(nx1, nx2, ny1, ny2);
        DISPATCH_FD(g.fdoh, kc_p_visc<FD><<<gr, kBlk, 0, stream()>>>(g, P, d_vx, d_vy, d_sp, d_p, d_g, d_bjm, d_cjm, d_e, ps[0], ps[1], ps[2], ps[3]));
        check_launch("update_p_visc_PML");
    }
    down(fblk(sp), fb);
    down(tblk(p), tb);
    if (pml) {
        down(pblk(psi_vxx), psix_bytes());
        down(pblk(psi_vyy), psiy_bytes());
        down(pblk(psi_vxy), psiy_bytes());
        down(pblk(psi_vyx), psix_bytes());
    }
    finish();
}

extern "C" void surface_acoustic_PML(int ndepth, float **sp) {
    const size_t fb = field_bytes();
    const RG g = make_rg(1, NX, 1, NY, nullptr);
    float *d_sp = up(fblk(sp), fb);
    kc_surf_ac<<<(NX + 127) / 128, 128, 0, stream()>>>(g, ndepth, d_sp);
    check_launch("surface_acoustic_PML");
    down(fblk(sp), fb);
    finish();
}

extern "C" void ifos_compat_release(void) {
    if (g_st) cudaStreamSynchronize(g_st);
    for (auto &kv : g_mirrors)
        if (kv.second.d) cudaFree(kv.second.d);
    g_mirrors.clear();
    if (g_prof_dev) cudaFree((void *)g_prof_dev);
    g_prof_dev = nullptr;
    g_prof_bytes = 0;
    if (g_small) cudaFree(g_small);
    g_small = nullptr;
    g_small_bytes = 0;
    if (g_small_out) cudaFree(g_small_out);
    g_small_out = nullptr;
    g_small_out_bytes = 0;
}
