// Snapshot store, zero-lag correlation, gradient assembly and FP64
// reductions of the shot solver.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "ifos_kernels.cuh"

namespace ifos {

// snapshot component lists: P-SV elastic (vxp1, vyp1, sxx, syy, sxy), acoustic
// (vxp1, vyp1, sp), SH (vzp1, sxz, syz) -- the arrays copied at
// src/IFOS2D.c:1805-1871
struct KSnap {
    void *base;            // slot 0, slot 0 snapshot
    long long slot_bytes;  // bytes between slots
    long long snap_bytes;  // bytes between snapshots of one slot
    float *scale;          // [slot][snap][comp] absmax (bf16 / fp16 formats)
    int ncomp, ntdtinv, format;
    int comp_plane[8];     // state plane of every component
    long long n;           // NX*NY
    int nx, ny, segs;      // fp16 segments: row segments of kSegCells cells
    long long ex_off;      // fp16 segments: bytes from a snapshot to its scales [comp][NY][segs]
};

template <typename T>
__device__ inline T snap_load(const KSnap &s, int slot, int snap, int k, long long q) {
    const char *b = (const char *)s.base + slot * s.slot_bytes + snap * s.snap_bytes;
    if (s.format == 0) return ((const T *)b)[k * s.n + q];
    if (s.format == 3 || s.format == 4) {
        const long long row = q / s.nx, col = q - row * s.nx;
        const float sc = ((const float *)(b + s.ex_off))[((long long)k * s.ny + row) * s.segs + col / kSegCells];
        return (T)(seg_unpack(((const unsigned short *)b)[k * s.n + q], s.format == 4) * sc);
    }
    const float sc = s.scale[((long long)slot * s.ntdtinv + snap) * s.ncomp + k];
    if (s.format == 1) return (T)(__bfloat162float(((const __nv_bfloat16 *)b)[k * s.n + q]) * sc);
    return (T)(__half2float(((const __half *)b)[k * s.n + q]) * sc);
}

// fp16 segments: one warp re-quantises the row-j segment `seg` of the listed
// components from the state planes (lane l holds cells 2l, 2l+1 of it).
template <typename T>
__device__ __forceinline__ void quant_seg(const KGrid &g, const KState<T> &S, const KSnap &sn, int slot, int hin,
                                          int j, int seg, const int *comps, int ncomps) {
    const int lane = threadIdx.x & 31;
    const int i = seg * kSegCells + 2 * lane + 1;
    const bool ok0 = i <= g.nx, ok1 = i + 1 <= g.nx;
    char *b = (char *)sn.base + slot * sn.slot_bytes + hin * sn.snap_bytes;
    unsigned short *h = (unsigned short *)b;
    float *ex = (float *)(b + sn.ex_off);
    const bool i16 = sn.format == 4;
    const long long q = (long long)(j - 1) * g.nx + (i - 1);
    for (int t = 0; t < ncomps; t++) {
        const int k = comps[t];
        if (k < 0) continue;
        const T *f = fieldp(S, slot, sn.comp_plane[k]);
        const float v0 = ok0 ? (float)f[pidx(g, j, i)] : 0.0f, v1 = ok1 ? (float)f[pidx(g, j, i + 1)] : 0.0f;
        float qf, inv;
        seg_scales(seg_absmax_warp(v0, v1, ok0, ok1), qf, inv, i16 ? kSegTopI16 : kSegTop);
        if (ok0) h[k * sn.n + q] = seg_pack(v0 * qf, i16);
        if (ok1) h[k * sn.n + q + 1] = seg_pack(v1 * qf, i16);
        if (lane == 0) ex[((long long)k * g.ny + (j - 1)) * sn.segs + seg] = inv;
    }
}

// fp16-segment snapshot store of the unpipelined paths: one warp per row
// segment, all components.  Grid (segs, ceil(NY/8), slots), block (32, 8).
template <typename T>
__global__ void k_snap_seg16(KGrid g, KState<T> S, KSnap sn, int hin) {
    pdl_wait();
    pdl_launch();
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (j > g.ny) return;
    const int comps[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    quant_seg<T>(g, S, sn, blockIdx.z, hin, j, blockIdx.x, comps, sn.ncomp);
}

// fp16 segments written by the stencil kernels: the free-surface and
// explosive-source kernel changes the stresses of row 1 and of the source
// cells after the stress kernel stored them, so those segments are stored
// again from the final state.  Grid (segs + max_src, 1, slots), one warp.
template <typename T>
__global__ void k_snap_fix16(KGrid g, KState<T> S, KSnap sn, int hin, KSrc src, int surf, int4 patched) {
    pdl_wait();
    pdl_launch();
    const int slot = blockIdx.z;
    const int comps[4] = {patched.x, patched.y, patched.z, patched.w};
    int j, seg;
    if ((int)blockIdx.x < sn.segs) {
        if (!surf) return;
        j = 1;
        seg = blockIdx.x;
    } else {
        const int l = blockIdx.x - sn.segs;
        if (l >= src.nsrc[slot]) return;
        const float *pos = src.pos + (long long)slot * 8 * src.max_src;
        const int i = (int)pos[l];
        j = (int)pos[src.max_src + l];
        if (i < 1 || i > g.nx || j < 1 || j > g.ny) return;
        seg = (i - 1) / kSegCells;
    }
    quant_seg<T>(g, S, sn, slot, hin, j, seg, comps, 4);
}

// fp32/fp64 snapshot copy (one thread per cell, all components)
template <typename T>
__global__ void k_snap_store(KGrid g, KState<T> S, KSnap sn, int hin) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1);
    T *b = (T *)((char *)sn.base + slot * sn.slot_bytes + hin * sn.snap_bytes);
    for (int k = 0; k < sn.ncomp; k++) b[k * sn.n + q] = fieldp(S, slot, sn.comp_plane[k])[c];
}

// low-precision snapshots, pass 1: absolute maximum of every component
template <typename T>
__global__ void k_snap_absmax(KGrid g, KState<T> S, KSnap sn, int hin) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    const bool in = i <= g.nx && j <= g.ny;
    const long long c = in ? pidx(g, j, i) : 0;
    for (int k = 0; k < sn.ncomp; k++) {
        float v = in ? fabsf((float)fieldp(S, slot, sn.comp_plane[k])[c]) : 0.0f;
        for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0 && v > 0.0f)
            atomicMax((unsigned int *)&sn.scale[((long long)slot * sn.ntdtinv + hin) * sn.ncomp + k],
                      __float_as_uint(v));
    }
}

// low-precision snapshots, pass 2: scaled conversion (round to nearest even)
template <typename T>
__global__ void k_snap_quant(KGrid g, KState<T> S, KSnap sn, int hin) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1);
    char *b = (char *)sn.base + slot * sn.slot_bytes + hin * sn.snap_bytes;
    for (int k = 0; k < sn.ncomp; k++) {
        const float sc = sn.scale[((long long)slot * sn.ntdtinv + hin) * sn.ncomp + k];
        const float inv = sc > 0.0f ? 1.0f / sc : 0.0f;
        const float v = (float)fieldp(S, slot, sn.comp_plane[k])[c] * inv;
        if (sn.format == 1) ((__nv_bfloat16 *)b)[k * sn.n + q] = __float2bfloat16_rn(v);
        else ((__half *)b)[k * sn.n + q] = __float2half_rn(v);
    }
}

// gradient accumulators per slot: 5 planes of NX*NY (lam', mu', rho', mu_z', rho_z')
struct KGrad {
    float *acc;             // slot * 5 * n
    float *out;             // slot * 10 * n (IFOS_G_* planes)
    long long n;
    double *acc64;          // slot * 5 * n: the sums in double (grad_acc64), else NULL
};

// The correlation of an fp64 context (the error oracle): the terms of
// src/IFOS2D.c:2379-2419 in double from double fields and snapshots, summed
// in double (gr.acc64), so that the oracle's gradients carry no float
// rounding at all.
__device__ __forceinline__ void correlate_f64(const KGrid &g, const KState<double> &S, const KModel<double> &M,
                                              const KSnap &sn, const KGrad &gr, int snap, int psv, int sh,
                                              int acoustic, int slot, long long c, long long q) {
    double *acc = gr.acc64 + (long long)slot * 5 * gr.n;
    int k = 0;
    if (psv) {
        const double frx = snap_load<double>(sn, slot, snap, k++, q), fry = snap_load<double>(sn, slot, snap, k++, q);
        acc[2 * gr.n + q] += (fieldp(S, slot, P_VXP1)[c] * frx) + (fieldp(S, slot, P_VYP1)[c] * fry);
        if (!acoustic) {
            const double fx = snap_load<double>(sn, slot, snap, k++, q), fy = snap_load<double>(sn, slot, snap, k++, q),
                         fu = snap_load<double>(sn, slot, snap, k++, q);
            const double sxx = fieldp(S, slot, P_SXX)[c], syy = fieldp(S, slot, P_SYY)[c],
                         sxy = fieldp(S, slot, P_SXY)[c];
            acc[q] += (fx + fy) * (sxx + syy);
            const double mm = modelp(M, slot, M_MM)[c], ll = modelp(M, slot, M_LL)[c];
            if (mm != 0.0) {
                const double t1 = (1.0 / mm) * (fu * sxy);
                const double t2 = (.25 * (g.mu_fix ? (fx + fy) * (sxx + syy) : fx + fy * (sxx + syy))) / ll;
                const double t3 = (.25 * (g.mu_fix ? (fx - fy) * (sxx - syy) : fx - fy * (sxx - syy))) / mm;
                acc[gr.n + q] += (t1 + t2) + t3;
            }
        } else {
            const double fp = snap_load<double>(sn, slot, snap, k++, q);
            acc[q] += fp * fieldp(S, slot, P_SP)[c];
        }
    }
    if (sh) {
        const double frz = snap_load<double>(sn, slot, snap, k++, q), fxz = snap_load<double>(sn, slot, snap, k++, q),
                     fyz = snap_load<double>(sn, slot, snap, k++, q);
        acc[4 * gr.n + q] += fieldp(S, slot, P_VZP1)[c] * frz;
        const double *rho = modelp(M, slot, M_RHO), *u = modelp(M, slot, M_VS);
        const double muss = rho[c] * u[c] * u[c];
        acc[3 * gr.n + q] += (1.0 / (muss * muss)) * (fxz * fieldp(S, slot, P_SXZ)[c] + fyz * fieldp(S, slot, P_SYZ)[c]);
    }
}

// zero-lag correlation with the stored forward wavefield (src/IFOS2D.c:2379-2419)
template <typename T>
__global__ void k_correlate(KGrid g, KState<T> S, KModel<T> M, KSnap sn, KGrad gr, int snap, int psv, int sh,
                            int acoustic) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1);
    if constexpr (std::is_same<T, double>::value) {
        if (gr.acc64) {
            correlate_f64(g, S, M, sn, gr, snap, psv, sh, acoustic, slot, c, q);
            return;
        }
    }
    float *acc = gr.acc + (long long)slot * 5 * gr.n;
    int k = 0;
    if (psv) {
        const T frx = snap_load<T>(sn, slot, snap, k++, q), fry = snap_load<T>(sn, slot, snap, k++, q);
        acc[2 * gr.n + q] += (float)((fieldp(S, slot, P_VXP1)[c] * frx) + (fieldp(S, slot, P_VYP1)[c] * fry));
        if (!acoustic) {
            const T fx = snap_load<T>(sn, slot, snap, k++, q), fy = snap_load<T>(sn, slot, snap, k++, q),
                    fu = snap_load<T>(sn, slot, snap, k++, q);
            const T sxx = fieldp(S, slot, P_SXX)[c], syy = fieldp(S, slot, P_SYY)[c], sxy = fieldp(S, slot, P_SXY)[c];
            acc[q] += (float)((fx + fy) * (sxx + syy));
            const T mm = modelp(M, slot, M_MM)[c], ll = modelp(M, slot, M_LL)[c];
            if (mm != (T)0) {
                const double t1 = (1.0 / (double)mm) * (double)(fu * sxy);
                const double t2 = (.25 * (double)(g.mu_fix ? (fx + fy) * (sxx + syy) : fx + fy * (sxx + syy))) /
                                  (double)ll;
                const double t3 = (.25 * (double)(g.mu_fix ? (fx - fy) * (sxx - syy) : fx - fy * (sxx - syy))) /
                                  (double)mm;
                acc[gr.n + q] = (float)((double)acc[gr.n + q] + ((t1 + t2) + t3));
            }
        } else {
            const T fp = snap_load<T>(sn, slot, snap, k++, q);
            acc[q] += (float)((fp) * (fieldp(S, slot, P_SP)[c]));
        }
    }
    if (sh) {
        const T frz = snap_load<T>(sn, slot, snap, k++, q), fxz = snap_load<T>(sn, slot, snap, k++, q),
                fyz = snap_load<T>(sn, slot, snap, k++, q);
        acc[4 * gr.n + q] += (float)(fieldp(S, slot, P_VZP1)[c] * frz);
        const T *rho = modelp(M, slot, M_RHO), *u = modelp(M, slot, M_VS);
        const T muss = rho[c] * u[c] * u[c];
        acc[3 * gr.n + q] = (float)((double)acc[3 * gr.n + q] +
                                    (1.0 / (double)(muss * muss)) *
                                        (double)(fxz * fieldp(S, slot, P_SXZ)[c] + fyz * fieldp(S, slot, P_SYZ)[c]));
    }
}

// Zero-lag correlation for fp32 state and fp32 snapshots: the arithmetic of
// k_correlate per cell, two adjacent cells of a row per thread with 8-byte
// loads and stores (rows of NX cells, NX even; the pitched state planes are
// always pair-aligned).  Grid: x over pairs of a row, y = row, z = slot.
struct CorrCell {
    float vxp1, vyp1, sxx, syy, sxy, sp, vzp1, sxz, syz;  // adjoint state
    float f[8];                                           // stored forward components
};
// W: the accumulator type -- float as the reference accumulates (each
// step's term is formed in float and added in float, or in double and
// rounded, exactly as src/IFOS2D.c:2379-2419 writes it), or double for the
// grad_acc64 sums (the same terms added in double, rounded once at the end)
template <int PSV, int SH, int AC, typename W = float>
__device__ __forceinline__ void correlate_cell(const CorrCell &a, float mm, float ll, float rho, float u, W *w0,
                                               W *w1, W *w2, W *w3, W *w4, bool mufix = false) {
    constexpr int KS = PSV ? (AC ? 3 : 5) : 0;  // first SH component
    if (PSV) {
        const float frx = a.f[0], fry = a.f[1];
        *w2 += (W)(float)((a.vxp1 * frx) + (a.vyp1 * fry));
        if (!AC) {
            const float fx = a.f[2], fy = a.f[3], fu = a.f[4];
            *w0 += (W)(float)((fx + fy) * (a.sxx + a.syy));
            if (mm != 0.0f) {
                const double t1 = (1.0 / (double)mm) * (double)(fu * a.sxy);
                // mufix: the grouping the mu gradient needs (sums of forward times adjoint stresses)
                const double t2 = (.25 * (double)(mufix ? (fx + fy) * (a.sxx + a.syy) : fx + fy * (a.sxx + a.syy))) /
                                  (double)ll;
                const double t3 = (.25 * (double)(mufix ? (fx - fy) * (a.sxx - a.syy) : fx - fy * (a.sxx - a.syy))) /
                                  (double)mm;
                *w1 = (W)((double)*w1 + ((t1 + t2) + t3));
            }
        } else {
            const float fp = a.f[2];
            *w0 += (W)(float)((fp) * (a.sp));
        }
    }
    if (SH) {
        const float frz = a.f[KS], fxz = a.f[KS + 1], fyz = a.f[KS + 2];
        *w4 += (W)(float)(a.vzp1 * frz);
        const float muss = rho * u * u;
        *w3 = (W)((double)*w3 + (1.0 / (double)(muss * muss)) * (double)(fxz * a.sxz + fyz * a.syz));
    }
}

// SEG: 0 fp32 snapshots, 1 fp16 segments, 2 int16 segments; ACC64: the sums
// in double (gr.acc64)
template <int PSV, int SH, int AC, int SEG, bool ACC64 = false>
__global__ void k_correlate_pairs(KGrid g, KState<float> S, KModel<float> M, KSnap sn, KGrad gr, int snap) {
    pdl_wait();
    pdl_launch();
    constexpr int NC = (PSV ? (AC ? 3 : 5) : 0) + (SH ? 3 : 0);
    // accumulators in use: lambda', mu', rho' (P-SV; acoustic: lambda', rho'), mu_z', rho_z' (SH)
    constexpr bool use[5] = {PSV != 0, PSV && !AC, PSV != 0, SH != 0, SH != 0};
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    const int j = blockIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1), n = gr.n;
    const float *st = S.base + slot * S.slot_stride + c;
    const char *sb = (const char *)sn.base + slot * sn.slot_bytes + snap * sn.snap_bytes;
    float *acc = gr.acc + (long long)slot * 5 * n + q;
    auto ld2 = [](const float *p) { return *reinterpret_cast<const float2 *>(p); };
    CorrCell a0{}, a1{};
    auto field = [&](int id, float &x0, float &x1) {
        const float2 v = ld2(st + S.off[id]);
        x0 = v.x;
        x1 = v.y;
    };
    if (PSV) {
        field(P_VXP1, a0.vxp1, a1.vxp1);
        field(P_VYP1, a0.vyp1, a1.vyp1);
        if (!AC) {
            field(P_SXX, a0.sxx, a1.sxx);
            field(P_SYY, a0.syy, a1.syy);
            field(P_SXY, a0.sxy, a1.sxy);
        } else {
            field(P_SP, a0.sp, a1.sp);
        }
    }
    if (SH) {
        field(P_VZP1, a0.vzp1, a1.vzp1);
        field(P_SXZ, a0.sxz, a1.sxz);
        field(P_SYZ, a0.syz, a1.syz);
    }
    if constexpr (SEG != 0) {
        // 16-bit segments: a pair never straddles a segment (both start at odd i)
        const unsigned short *hs = (const unsigned short *)sb + q;
        const float *ex = (const float *)(sb + sn.ex_off) + (long long)(j - 1) * sn.segs + (i - 1) / kSegCells;
#pragma unroll
        for (int k = 0; k < NC; k++) {
            const unsigned u = *reinterpret_cast<const unsigned *>(hs + k * sn.n);
            const float sc = ex[(long long)k * g.ny * sn.segs];
            a0.f[k] = seg_unpack((unsigned short)(u & 0xffffu), SEG == 2) * sc;
            a1.f[k] = seg_unpack((unsigned short)(u >> 16), SEG == 2) * sc;
        }
    } else {
        const float *fs = (const float *)sb + q;
#pragma unroll
        for (int k = 0; k < NC; k++) {
            const float2 v = ld2(fs + k * sn.n);
            a0.f[k] = v.x;
            a1.f[k] = v.y;
        }
    }
    const long long mo = (long long)M.slot_model[slot] * M.model_stride + c;
    float2 mm{0, 0}, ll{0, 0}, rho{0, 0}, u{0, 0};
    if (PSV && !AC) {
        mm = ld2(M.m[M_MM] + mo);
        ll = ld2(M.m[M_LL] + mo);
    }
    if (SH) {
        rho = ld2(M.m[M_RHO] + mo);
        u = ld2(M.m[M_VS] + mo);
    }
    const bool pair = i + 1 <= g.nx;
    if constexpr (ACC64) {
        double *acd = gr.acc64 + (long long)slot * 5 * n + q;
        double2 w[5] = {};
#pragma unroll
        for (int k = 0; k < 5; k++)
            if (use[k]) w[k] = *reinterpret_cast<const double2 *>(acd + k * n);
        correlate_cell<PSV, SH, AC, double>(a0, mm.x, ll.x, rho.x, u.x, &w[0].x, &w[1].x, &w[2].x, &w[3].x, &w[4].x,
                                            g.mu_fix != 0);
        if (pair)
            correlate_cell<PSV, SH, AC, double>(a1, mm.y, ll.y, rho.y, u.y, &w[0].y, &w[1].y, &w[2].y, &w[3].y,
                                                &w[4].y, g.mu_fix != 0);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            if (!use[k]) continue;
            if (pair) *reinterpret_cast<double2 *>(acd + k * n) = w[k];
            else acd[k * n] = w[k].x;
        }
        return;
    }
    float2 w[5] = {};
#pragma unroll
    for (int k = 0; k < 5; k++)
        if (use[k]) w[k] = ld2(acc + k * n);
    correlate_cell<PSV, SH, AC>(a0, mm.x, ll.x, rho.x, u.x, &w[0].x, &w[1].x, &w[2].x, &w[3].x, &w[4].x, g.mu_fix != 0);
    if (pair)
        correlate_cell<PSV, SH, AC>(a1, mm.y, ll.y, rho.y, u.y, &w[0].y, &w[1].y, &w[2].y, &w[3].y, &w[4].y,
                                    g.mu_fix != 0);
#pragma unroll
    for (int k = 0; k < 5; k++) {
        if (!use[k]) continue;
        if (pair) *reinterpret_cast<float2 *>(acc + k * n) = w[k];
        else acc[k * n] = w[k].x;
    }
}



// The assembly of an fp64 context (the error oracle): the formulas of
// src/IFOS2D.c:2477-2601 in double from the double sums, rounded once into
// the float output planes.
__device__ __forceinline__ void assemble_f64(const KGrid &g, const KModel<double> &M, const KGrad &gr, int psv,
                                             int sh, int acoustic, int slot, long long c, long long q) {
    const long long n = gr.n;
    const double *acc = gr.acc64 + (long long)slot * 5 * n;
    float *o = gr.out + (long long)slot * 10 * n;
    const double wl = acc[q], wm = acc[n + q], wr = acc[2 * n + q], wmz = acc[3 * n + q], wrz = acc[4 * n + q];
    o[0 * n + q] = (float)wl;
    o[1 * n + q] = (float)wm;
    o[2 * n + q] = (float)wr;
    o[6 * n + q] = (float)wmz;
    o[7 * n + q] = (float)wrz;
    const double DT = (double)g.dt;
    if (g.lame) {  // PARAMETERIZATION 3: the lambda, mu and rho gradients (src/IFOS2D.c:2498-2608)
        o[3 * n + q] = psv ? (float)(-DT * wl) : 0.0f;
        o[4 * n + q] = psv ? (float)(-DT * wm) : 0.0f;
        o[5 * n + q] = psv ? (float)(-DT * wr) : 0.0f;
        o[8 * n + q] = sh ? (float)(-DT * wmz) : (float)wmz;
        o[9 * n + q] = sh ? (float)(-DT * wrz) : (float)wrz;
        return;
    }
    const double rho = modelp(M, slot, M_RHO)[c], u = modelp(M, slot, M_VS)[c], pi = modelp(M, slot, M_VP)[c];
    double vp_g = 0, vs_g = 0, rho_g = 0;
    if (psv) {
        double lam = -DT * wl, mu = 0;
        const double muss = !acoustic ? rho * u * u : 0;
        const double lamss = rho * pi * pi - 2.0 * muss;
        lam = !acoustic ? lam / (4.0 * (lamss + muss) * (lamss + muss)) : lam / ((lamss + muss) * (lamss + muss));
        vp_g = 2.0 * pi * rho * lam;
        if (!acoustic) {
            mu = -DT * wm;
            vs_g = -4.0 * rho * u * lam + 2.0 * rho * u * mu;
        } else {
            vs_g = wm;
        }
        const double rho_s = -DT * wr;
        rho_g = !acoustic ? (pi * pi - 2.0 * u * u) * lam + u * u * mu + rho_s : (pi * pi) * lam + rho_s;
    }
    o[3 * n + q] = (float)vp_g;
    o[4 * n + q] = (float)vs_g;
    o[5 * n + q] = (float)rho_g;
    if (sh && !acoustic) {
        const double mu_z = -DT * wmz;
        o[8 * n + q] = (float)(2.0 * rho * u * mu_z);
        o[9 * n + q] = (float)(u * u * mu_z + (-DT * wrz));
    } else {
        o[8 * n + q] = (float)wmz;
        o[9 * n + q] = (float)wrz;
    }
}

// per-shot gradient assembly, PARAMETERIZATION 1 and 3 (src/IFOS2D.c:2477-2608)
template <typename T>
__global__ void k_assemble(KGrid g, KModel<T> M, KGrad gr, int psv, int sh, int acoustic) {
    pdl_wait();
    pdl_launch();
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int slot = blockIdx.z;
    if (i > g.nx || j > g.ny) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1), n = gr.n;
    const float *acc = gr.acc + (long long)slot * 5 * n;
    float *o = gr.out + (long long)slot * 10 * n;
    if constexpr (std::is_same<T, double>::value) {
        if (gr.acc64) {  // the fp64 oracle: the assembly in double from the double sums
            assemble_f64(g, M, gr, psv, sh, acoustic, slot, c, q);
            return;
        }
    }
    const double *acd = gr.acc64 ? gr.acc64 + (long long)slot * 5 * n : nullptr;
    // grad_acc64: the double sums rounded once, then the reference's assembly
    auto w = [&](int k) { return acd ? (float)acd[k * n + q] : acc[k * n + q]; };
    const float wl = w(0), wm = w(1), wr = w(2), wmz = w(3), wrz = w(4);
    o[0 * n + q] = wl;
    o[1 * n + q] = wm;
    o[2 * n + q] = wr;
    o[6 * n + q] = wmz;
    o[7 * n + q] = wrz;
    const float DT = g.dt;
    if (g.lame) {
        // PARAMETERIZATION 3 (src/IFOS2D.c:2498-2500, :2527-2530, :2551-2554,
        // :2581-2584, :2605-2608): each gradient is -DT times its sum; the
        // reference leaves the vp / vs / rho planes as zero where the wave type
        // is not modelled, and the SH planes as the raw sums
        o[3 * n + q] = psv ? -DT * wl : 0.0f;
        o[4 * n + q] = psv ? -DT * wm : 0.0f;
        o[5 * n + q] = psv ? -DT * wr : 0.0f;
        o[8 * n + q] = sh ? -DT * wmz : wmz;
        o[9 * n + q] = sh ? -DT * wrz : wrz;
        return;
    }
    const float rho = (float)modelp(M, slot, M_RHO)[c], u = (float)modelp(M, slot, M_VS)[c],
                pi = (float)modelp(M, slot, M_VP)[c];
    float vp_g = 0, vs_g = 0, rho_g = 0;
    if (psv) {
        float lam = -DT * wl, mu = 0;
        const float muss = !acoustic ? rho * u * u : 0;
        const float lamss = (float)((double)(rho * pi * pi) - 2.0 * (double)muss);
        if (!acoustic) lam = (float)((1.0 / (4.0 * (double)(lamss + muss) * (double)(lamss + muss))) * (double)lam);
        else lam = (float)((1.0 / (double)((lamss + muss) * (lamss + muss))) * (double)lam);
        vp_g = (float)(2.0 * (double)pi * (double)rho * (double)lam);
        if (!acoustic) {
            mu = -DT * wm;
            vs_g = (float)(-4.0 * (double)rho * (double)u * (double)lam + 2.0 * (double)rho * (double)u * (double)mu);
        } else {
            vs_g = wm;
        }
        const float rho_s = -DT * wr;
        if (!acoustic)
            rho_g = (float)(((double)(pi * pi) - (2.0 * (double)u * (double)u)) * (double)lam +
                            (double)(u * u * mu) + (double)rho_s);
        else
            rho_g = ((pi * pi) * lam) + rho_s;
    }
    o[3 * n + q] = vp_g;
    o[4 * n + q] = vs_g;
    o[5 * n + q] = rho_g;
    if (sh && !acoustic) {
        const float mu_z = -DT * wmz;
        o[8 * n + q] = (float)(2.0 * (double)rho * (double)u * (double)mu_z);
        const float rho_s_z = -DT * wrz;
        o[9 * n + q] = ((u * u * mu_z) + rho_s_z);
    } else {
        o[8 * n + q] = wmz;
        o[9 * n + q] = wrz;
    }
}

// The host-called kernels below are compiled into the solver unit only (the
// per-width stencil units define IFOS_PIPE_FD and do not launch them).
#ifndef IFOS_PIPE_FD

// sum of the assembled gradients over slots (src/IFOS2D.c:2703-2724), in slot
// order so the float additions match the reference's shot loop
__global__ void k_grad_sum(const float *grads, int nshots, long long n, float *out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int planes[5] = {3, 4, 5, 8, 9};
    for (int k = 0; k < 5; k++) {
        float s = 0.0f;
        for (int sl = 0; sl < nshots; sl++) s += grads[(long long)sl * 10 * n + planes[k] * n + q];
        out[k * n + q] = s;
    }
}

// FP64 dot product, pass 1: one double partial per block (deterministic)
__global__ void k_dot_partial(const float *a, const float *b, long long n, double *partial) {
    double acc = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const double x = a[k];
        acc += x * (b ? (double)b[k] : x);
    }
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}
// pass 2: fixed-order sum of the partials
__global__ void k_dot_final(const double *partial, int nb, double *out) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += partial[k];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) *out = v;
    }
}

// residuals of one component, LNORM=2, VELOCITY=0 (src/calc_res.c:137-281):
// per trace, running float sums times DT, time-reversed difference; the
// misfit and energy partial sums per trace in double
// The time window of src/time_window.c:135-210 on one sample: v at 1-based
// sample j (j >= 2) of trace i, picks [np][ntr]; returns the windowed value
// and the taper bits (1/2 late/early of the first window, 4/8 of the second).
__device__ __forceinline__ float tw_sample(float v, int j, int i, int ntr, int tw_ind, const float *picks, float dt,
                                          float gamma, float twl_plus, float twl_minus, unsigned char &m) {
    const float time = (float)(j * dt);
    m = 0;
    float p1, l1, l2;
    if (tw_ind == 1 || tw_ind == 2) {
        p1 = picks[i];
        l1 = picks[ntr + i];
        l2 = picks[2 * ntr + i];
    } else {
        p1 = picks[i];
        l1 = twl_plus;
        l2 = twl_minus;
    }
    const float dumpa = (time - p1 - l1);
    const float taper = (float)exp((double)(-gamma * dumpa));
    const float dumpb = (time - p1 + l2);
    const float taper1 = (float)exp((double)(-gamma * dumpb));
    if (tw_ind != 2) {
        if (time >= p1 + l1) {
            v = v * taper;
            m |= 1;
        }
        if (time <= p1 - l2) {
            v = v * taper1;
            m |= 2;
        }
        return v;
    }
    float dummy = v;
    if (time >= p1 + l1) {
        dummy = v * taper;
        m |= 1;
    }
    if (time <= p1 - l2) {
        dummy = v * taper1;
        m |= 2;
    }
    const float p4 = picks[3 * ntr + i], l5 = picks[4 * ntr + i], l6 = picks[5 * ntr + i];
    const float dumpc = (time - p4 - l5);
    const float taper2 = (float)exp((double)(-gamma * dumpc));
    const float dumpd = (time - p4 + l6);
    const float taper3 = (float)exp((double)(-gamma * dumpd));
    if (time >= p4 + l5) {
        v = v * taper2;
        m |= 4;
    }
    if (time <= p4 - l6) {
        v = v * taper3;
        m |= 8;
    }
    return v + dummy;
}

// time window of the residual step (TIMEWIN=1): picks [np][ntr] of one shot
struct KWindow {
    const float *picks;  // NULL: no window
    int stride;          // traces between the pick rows
    int tw_ind;
    float gamma, twl_plus, twl_minus;
};
__global__ void k_calc_res(const float *obs, const float *syn, float *diff, int ntr, int ns, float dt,
                           double *l2_tr, double *en_tr, const int *kill = nullptr, KWindow win = KWindow{}) {
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= ntr) return;
    if (kill && kill[tr]) {  // a killed trace keeps a zero residual and adds nothing (src/calc_res.c:196-197)
        l2_tr[tr] = 0.0;
        en_tr[tr] = 0.0;
        return;
    }
    const float *s = syn + (long long)tr * ns, *d = obs + (long long)tr * ns;
    float *df = diff + (long long)tr * ns;
    float rs = 0.0f, rd = 0.0f;
    double l2 = 0.0, en = 0.0;
    for (int j = 0; j < ns; j++) {
        rs += s[j];
        rd += d[j];
        float is = rs * dt, id = rd * dt;
        if (win.picks && j >= 1) {  // windowed after the integration (src/calc_res.c:157-160)
            unsigned char m;
            is = tw_sample(is, j + 1, tr, win.stride, win.tw_ind, win.picks, dt, win.gamma, win.twl_plus,
                           win.twl_minus, m);
            id = tw_sample(id, j + 1, tr, win.stride, win.tw_ind, win.picks, dt, win.gamma, win.twl_plus,
                           win.twl_minus, m);
        }
        const float r = is - id;
        df[ns - 1 - j] = r;
        l2 += (double)r * (double)r;
        en += (double)id * (double)id;
    }
    l2_tr[tr] = l2;
    en_tr[tr] = en;
}

// Offset-based trace kill (src/create_trkill_table.c:35-46): killtable[r][s]
// is set to 1 where the source-receiver offset, formed in float and taken
// through a double sqrt as the reference does, lies strictly inside
// (lower, upper); other entries are left as they are.  One thread per pair.
__global__ void k_trkill(int ntr, const int *rx, const int *ry, int nsrc, const float *sx, const float *sy, float dh,
                         float lower, float upper, int *killtable) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= (long long)ntr * nsrc) return;
    const int r = (int)(k / nsrc), s = (int)(k % nsrc);
    const float ddx = sx[s] - rx[r] * dh, ddy = sy[s] - ry[r] * dh;
    const float offset = (float)fabs(sqrt((double)(ddx * ddx + ddy * ddy)));
    if (offset > lower && offset < upper) killtable[k] = 1;
}

// Time windows around picked first arrivals (src/time_window.c:146-220),
// one thread per sample j = 2..ns of a trace; tw_ind 0: one pick per trace
// with lengths twl_plus/twl_minus; 1: (pick, length+, length-); 2: two such
// windows, the first one's tapered copy added to the second's.  mask (if
// not NULL) records the tapers applied: bits 0/1 the first window's late/early
// taper, bits 2/3 the second window's.
__global__ void k_time_window(float *sec, int ntr, int ns, int tw_ind, const float *picks, float dt, float gamma,
                              float twl_plus, float twl_minus, unsigned char *mask) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= (long long)ntr * ns) return;
    const int i = (int)(k / ns), j = (int)(k % ns) + 1;  // trace, 1-based sample
    if (j < 2) {  // the reference's loops start at sample 2
        if (mask) mask[k] = 0;
        return;
    }
    unsigned char m;
    sec[k] = tw_sample(sec[k], j, i, ntr, tw_ind, picks, dt, gamma, twl_plus, twl_minus, m);
    if (mask) mask[k] = m;
}

// Butterworth filtering of traces (src/timedomain_filt.c with the vendored
// libcseife): every trace is one thread's sequential recursion, in double.
// The reference filters the ns+1 values [0, x_1..x_ns] (its dvector has a
// zero element before the samples), with each section of the cascade in
// turn: y_j = f0 x_j + f1 x_{j-1} + f2 x_{j-2} + g1 y_{j-1} + g2 y_{j-2}
// (contrib/libcseife/cseife_rekfl.c), evaluated left to right.
struct KIIR {
    double c[8][5];  // sections: f0 f1 f2 g1 g2
    int n;
};
__global__ void k_butterworth(float *data, double *work, int ntr, int ns, KIIR lp, KIIR hp) {
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= ntr) return;
    float *d = data + (long long)tr * ns;
    double *x = work + (long long)tr * (ns + 1);
    for (int pass = 0; pass < 2; pass++) {
        const KIIR &f = pass ? hp : lp;
        if (f.n == 0) continue;
        x[0] = 0.0;
        for (int j = 1; j <= ns; j++) x[j] = (double)d[j - 1];
        // a highpass first subtracts x[0] from every value (contrib/libcseife/cseife.c:156-161); x[0] is 0
        for (int s = 0; s < f.n; s++) {
            const double f0 = f.c[s][0], f1 = f.c[s][1], f2 = f.c[s][2], g1 = f.c[s][3], g2 = f.c[s][4];
            double xa = 0.0, xaa = 0.0, ya = 0.0, yaa = 0.0;
            for (int j = 0; j <= ns; j++) {
                const double xn = x[j];
                const double y = f0 * xn + f1 * xa + f2 * xaa + g1 * ya + g2 * yaa;
                x[j] = y;
                xaa = xa;
                xa = xn;
                yaa = ya;
                ya = y;
            }
        }
        for (int j = 1; j <= ns; j++) d[j - 1] = (float)x[j];
    }
}

// Per-shot gradient taper around the source (src/taper_grad_shot.c:52-197,
// sws=1): the taper matrix (gp x gp values, formed on the host as the
// reference forms it) is centred on the source cell, every cell outside it
// has the value 1, the field is shifted by its minimum and divided by its
// maximum, the gradient is multiplied by it, and the cells within `filtsize`
// of the source are set to zero.
struct KTaperShot {
    int i0, j0, ijc, gp;  // source cell, centre index of the taper matrix, its size
    float minm, maxm;     // minimum of the tapered field and maximum after the shift
    int filtsize;
};
__global__ void k_taper_shot(float *gout, long long n, int nx, int ny, unsigned planes, const KTaperShot *tp,
                             const float *mats) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int slot = blockIdx.y;
    if (q >= n) return;
    const KTaperShot t = tp[slot];
    const int i = (int)(q % nx) + 1, j = (int)(q / nx) + 1;
    float msum = 1.0f;
    const int ix = i - t.i0 + t.ijc, iy = j - t.j0 + t.ijc;
    if (ix >= 1 && ix <= t.gp && iy >= 1 && iy <= t.gp) {
        const float m = mats[(long long)slot * t.gp * t.gp + (long long)(iy - 1) * t.gp + (ix - 1)];
        if (msum > m) msum = m;
    }
    const float coeff = (msum - t.minm) / t.maxm;
    const bool zero = i >= t.i0 - t.filtsize && i <= t.i0 + t.filtsize && j >= t.j0 - t.filtsize &&
                      j <= t.j0 + t.filtsize;
    float *g = gout + (long long)slot * 10 * n + q;
    for (int k = 0; k < 10; k++) {
        if (!(planes >> k & 1u)) continue;
        g[k * n] = zero ? 0.0f : g[k * n] * coeff;
    }
    (void)ny;
}

// Per-shot gradient taper read from a file (src/taper_grad_shot.c:206-289,
// sws 2-4): the planes of `planes` of one slot's stored gradients times the
// coefficient plane, one float product per cell as waveconv *= taper_coeff.
__global__ void k_taper_coeff(float *g, long long n, unsigned planes, const float *coeff) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float t = coeff[q];
    for (int k = 0; k < 10; k++)
        if (planes >> k & 1u) g[k * n + q] *= t;
}

// Median smoothing of a gradient or model plane (src/smooth.c with
// src/median2D.c).  Every cell takes the window of fs x fs values around it
// (edges extended by the nearest row / column), gathered x-major as the
// reference's filterpart is.  The reference sorts its vector t[0..k-1] with
// t[0] = 0 (a zeroed element before the copied window) and t[1..k-1] the
// first k-1 window values, leaving the last window value at t[k], and returns
// t[k/2+1]; the same non-recursive quicksort (src/util.c:437-466) runs here
// so that ties of +0 and -0 resolve as they do there.
constexpr int kMedianMax = 31 * 31 + 1;
__device__ __forceinline__ void quicksort_dev(float *arr, int elements) {
    int beg[64], end[64], i = 0;
    beg[0] = 0;
    end[0] = elements;
    while (i >= 0) {
        int L = beg[i], R = end[i] - 1;
        if (L < R) {
            const float piv = arr[L];
            while (L < R) {
                while (arr[R] >= piv && L < R) R--;
                if (L < R) arr[L++] = arr[R];
                while (arr[L] <= piv && L < R) L++;
                if (L < R) arr[R--] = arr[L];
            }
            arr[L] = piv;
            beg[i + 1] = L + 1;
            end[i + 1] = end[i];
            end[i++] = L;
            if (end[i] - beg[i] > end[i - 1] - beg[i - 1]) {
                int sw = beg[i];
                beg[i] = beg[i - 1];
                beg[i - 1] = sw;
                sw = end[i];
                end[i] = end[i - 1];
                end[i - 1] = sw;
            }
        } else {
            i--;
        }
    }
}
__global__ void k_median_smooth(const float *in, float *out, int nx, int ny, int fs) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nx * ny) return;
    const int i = (int)(q % nx) + 1, j = (int)(q / nx) + 1;
    const int hfs = fs / 2, k = fs * fs;
    float t[kMedianMax];
    t[0] = 0.0f;
    int n = 1;
    for (int ii = -hfs; ii <= hfs; ii++)
        for (int jj = -hfs; jj <= hfs; jj++) {
            const int x = min(max(i + ii, 1), nx), y = min(max(j + jj, 1), ny);
            t[n++] = in[(long long)(y - 1) * nx + (x - 1)];
        }
    quicksort_dev(t, k);
    out[q] = t[k / 2 + 1];
}

#endif  // IFOS_PIPE_FD
}  // namespace ifos
