// Persistent, TMA-pipelined stencil kernels.
//
// Each block loops over 32 x TY tiles of the grid (all shot slots).  A
// producer warp issues bulk tensor loads (cp.async.bulk.tensor, no multicast)
// of every input plane of a tile into a ring of NST shared-memory stages: the
// planes that need neighbours (the stresses in the velocity update, the
// velocities in the stress update) as tile + halo boxes, and the per-cell
// streams (the updated fields, memory variables, coefficients) as plain tile
// boxes.  Eight compute warps consume the stages in order and release each
// one to the producer, so HBM latency is hidden by the ring rather than by
// occupancy.  Results are written back with coalesced 128-byte warp stores.
// The per-cell arithmetic is the reference's, in the same order and with the
// same float/double promotions as ifos_kernels.cuh.
#pragma once
#include <type_traits>

#include "ifos_kernels.cuh"
#include "ifos_tma.cuh"

// 1: the reference's double-promoted terms are evaluated in double (bit-exact);
// 0: in the kernel's own precision
#ifndef IFOS_EXACT
#define IFOS_EXACT 1
#endif

namespace ifos {

template <typename T>
using Dbl = typename std::conditional<IFOS_EXACT != 0, double, T>::type;

// Plane ids for the TMA z coordinate: state plane = slot * planes_per_slot + pid,
// model plane = model * model_planes + mid.
struct KTma {
    int planes_per_slot;
    int pid[NP_FIELD];
    int mem_pid[5];
    int model_planes;
    int mid[NM_PLANE];
};

template <typename T, int FDOH, int TY, int NH, int NP, int NST>
struct Pipe {
    static constexpr int TX = 32, H = FDOH, XH = ((FDOH + 3) / 4) * 4;
    static constexpr int BW = TX + 2 * XH, BH = TY + 2 * H;
    static constexpr int ES = (int)sizeof(T);
    // tensor-copy destinations in shared memory must be 128-byte aligned
    static constexpr int BOXS = ((BW * BH * ES + 127) / 128) * 128 / ES;
    static constexpr int PLS = TX * TY;
    static constexpr int STAGE = NH * BOXS + NP * PLS;
    static constexpr int RT = TY / 8;  // rows per thread (eight compute warps)
    static constexpr uint32_t TXB = (uint32_t)((NH * BW * BH + NP * PLS) * ES);
    static constexpr size_t bytes() { return (size_t)NST * STAGE * ES; }
};

struct KMaps {
    CUtensorMap halo;   // state planes, box (32+2XH) x (TY+2H)
    CUtensorMap plain;  // state planes, box 32 x TY
    CUtensorMap model;  // model planes, box 32 x TY
};

struct TileIdx {
    int slot, i0, j0;
};
__device__ __forceinline__ TileIdx tile_of(int t, int ntx, int nty, int TY) {
    TileIdx r;
    const int per = ntx * nty;
    r.slot = t / per;
    const int rem = t - r.slot * per;
    const int tyi = rem / ntx;
    r.i0 = (rem - tyi * ntx) * 32 + 1;
    r.j0 = tyi * TY + 1;
    return r;
}

// source of a plain-box load: a state plane or a model plane
struct PlainSrc {
    int z;
    bool model;
};

// Warp-specialised persistent driver.  Warps 0-7 compute, warp 8 produces:
// its lane 0 walks the same tile sequence, waits until a stage has been
// released by all eight compute warps ("empty" barrier, one arrival per warp),
// and issues the bulk tensor loads of the next tile into it ("full" barrier,
// completed by the transaction bytes).  The tile's model index is passed
// through shared memory.  Every wait is bounded.
constexpr int kComputeThreads = 256;
constexpr int kBlockThreads = kComputeThreads + 32;

template <typename T, int FDOH, int TY, int NH, int NP, int NST, typename Op>
__device__ __forceinline__ void run_pipeline(const KGrid &g, const KMaps &mp, int nshots, const Op &op,
                                             const int *slot_model, int *err) {
    using P = Pipe<T, FDOH, TY, NH, NP, NST>;
    extern __shared__ __align__(1024) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ int tile_model[NST];
    __shared__ int abort_flag;
    T *smem = reinterpret_cast<T *>(sm_raw);
    const int ntx = (g.nx + 31) / 32, nty = (g.ny + TY - 1) / TY;
    const int ntiles = ntx * nty * nshots;
    const int warp = threadIdx.y;  // block is 32 x 9
    if (warp == 8 && threadIdx.x == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);
        }
        abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == 8) {
        if (threadIdx.x != 0) return;
        for (int k = 0;; k++) {
            const int t = blockIdx.x + k * gridDim.x;
            if (t >= ntiles) break;
            const int st = k % NST;
            if (k >= NST && !mbar_wait_bounded(&empty[st], (uint32_t)(((k / NST) - 1) & 1), err, 18)) {
                abort_flag = 1;
                break;
            }
            const TileIdx ti = tile_of(t, ntx, nty, TY);
            const int model = slot_model[ti.slot];
            tile_model[st] = model;
            T *stage = smem + st * P::STAGE;
            uint64_t *bar = &full[st];
            int hz[NH > 0 ? NH : 1];
            PlainSrc pz[NP > 0 ? NP : 1];
            op.planes(ti, model, hz, pz);
            const int bx = HX + ti.i0 - 1 - P::XH, by = HY + ti.j0 - 1 - P::H;
            const int px = HX + ti.i0 - 1, py = HY + ti.j0 - 1;
            mbar_expect_tx(bar, P::TXB);
#pragma unroll
            for (int h = 0; h < NH; h++) tma_load_3d(stage + h * P::BOXS, &mp.halo, bx, by, hz[h], bar);
#pragma unroll
            for (int q = 0; q < NP; q++)
                tma_load_3d(stage + NH * P::BOXS + q * P::PLS, pz[q].model ? &mp.model : &mp.plain, px, py,
                            pz[q].z, bar);
        }
        return;
    }
    for (int k = 0;; k++) {
        const int t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int st = k % NST;
        const uint32_t parity = (uint32_t)((k / NST) & 1);
        if (!mbar_wait_bounded(&full[st], parity, err, 16)) {
            mbar_wait_bounded(&full[st], parity, err, 17);
            return;
        }
        if (abort_flag) return;
        const TileIdx ti = tile_of(t, ntx, nty, TY);
        T *stage = smem + st * P::STAGE;
        op.compute(ti, tile_model[st], stage, stage + NH * P::BOXS);
        __syncwarp();
        if (threadIdx.x == 0) mbar_arrive(&empty[st]);
    }
}

// y-tap of a staged halo tile.  In the top row of tiles with a free surface
// (MIR) rows j<=0 read the imaged value the reference's ghost rows hold when
// the velocity is updated: -f(2-j) for syy, syz, sp
// (src/surface_elastic_PML.c:59) and -f(1-j) for sxy (:60).
template <bool MIR, bool ODD, typename P, typename T>
__device__ __forceinline__ T ldy(const T *t, int jj, int col, int dy) {
    const int rr = jj + P::H + dy;
    if (MIR && rr < P::H) {
        const int src = ODD ? 2 * P::H - rr - 1 : 2 * P::H - rr;
        return -t[src * P::BW + col];
    }
    return t[rr * P::BW + col];
}

// FD weights of one launch, in registers
template <typename T, int FDOH>
struct Hc {
    T w[FDOH + 1];
    __device__ __forceinline__ explicit Hc(const KGrid &g) {
#pragma unroll
        for (int m = 0; m <= FDOH; m++) w[m] = (T)g.hc[m];
    }
};

// ---------------------------------------------------------------------------
// velocity, P-SV (src/update_v_PML.c:161-252; 10/12 reference branches :466-528)
// halo: sxx syy sxy; plain: vx vy rip rjp [+ vxp1 vyp1 in the adjoint, NP=6]
template <typename T, int FDOH, int TY, int NP, int NST>
struct OpVPsv {
    using P = Pipe<T, FDOH, TY, 3, NP, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    int sw, want_p1;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_SXX];
        hz[1] = zb + tm.pid[P_SYY];
        hz[2] = zb + tm.pid[P_SXY];
        pz[0] = {zb + tm.pid[P_VX], false};
        pz[1] = {zb + tm.pid[P_VY], false};
        pz[2] = {mb + tm.mid[M_RIP], true};
        pz[3] = {mb + tm.mid[M_RJP], true};
        if (NP > 4) {
            pz[4 % NP] = {zb + tm.pid[P_VXP1], false};
            pz[5 % NP] = {zb + tm.pid[P_VYP1], false};
        }
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        if (g.free_surf && ti.j0 == 1) rows<true>(ti, h, pl);
        else rows<false>(ti, h, pl);
    }
    template <bool MIR>
    __device__ __forceinline__ void rows(const TileIdx &ti, const T *h, const T *pl) const {
        const T *t_sxx = h, *t_syy = h + P::BOXS, *t_sxy = h + 2 * P::BOXS;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ vx = S.base + so + S.off[P_VX];
        T *__restrict__ vy = S.base + so + S.off[P_VY];
        T *__restrict__ vxp1 = S.base + so + S.off[P_VXP1];
        T *__restrict__ vyp1 = S.base + so + S.off[P_VYP1];
        T *ps_sxx = S.psix[X_SXX] + slot * S.psix_slot, *ps_sxy = S.psix[X_SXY] + slot * S.psix_slot;
        T *ps_syy = S.psiy[Y_SYY] + slot * S.psiy_slot, *ps_syx = S.psiy[Y_SXY] + slot * S.psiy_slot;
        const T DT = g.dt, DH = g.dh;
        const int col = tx + P::XH;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + col, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            const T vxo = pl[pc], vyo = pl[P::PLS + pc];
            const T rip = pl[2 * P::PLS + pc], rjp = pl[3 * P::PLS + pc];
            if (g.quirk_hi) {
                const T dtdh = DT * DT / DH;
                T ax = 0, ay = 0;
#pragma unroll
                for (int m = 1; m <= FDOH; m++) ax += hc.w[m] * (t_sxx[rc + m] - t_sxx[rc - m + 1]);
#pragma unroll
                for (int m = 1; m <= FDOH; m++)
                    ax += hc.w[m] * (ldy<MIR, true, P>(t_sxy, jj, col, m - 1) - ldy<MIR, true, P>(t_sxy, jj, col, -m));
#pragma unroll
                for (int m = 1; m <= FDOH; m++)
                    ay += hc.w[m] * (ldy<MIR, false, P>(t_syy, jj, col, m) - ldy<MIR, false, P>(t_syy, jj, col, 1 - m));
#pragma unroll
                for (int m = 1; m <= FDOH; m++) ay += hc.w[m] * (t_sxy[rc + m - 1] - t_sxy[rc - m]);
                vx[c] = vxo + ax * dtdh * rip;
                vy[c] = vyo + ay * dtdh * rjp;
                continue;
            }
            T sxx_x = 0, sxy_x = 0, sxy_y = 0, syy_y = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) sxx_x += hc.w[m] * (t_sxx[rc + m] - t_sxx[rc - m + 1]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++) sxy_x += hc.w[m] * (t_sxy[rc + m - 1] - t_sxy[rc - m]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++)
                sxy_y += hc.w[m] * (ldy<MIR, true, P>(t_sxy, jj, col, m - 1) - ldy<MIR, true, P>(t_sxy, jj, col, -m));
#pragma unroll
            for (int m = 1; m <= FDOH; m++)
                syy_y += hc.w[m] * (ldy<MIR, false, P>(t_syy, jj, col, m) - ldy<MIR, false, P>(t_syy, jj, col, 1 - m));
            sxx_x = cpml_xh(g, M, ps_sxx, j, hx, K_XH, A_XH, B_XH, sxx_x);
            sxy_x = cpml_xh(g, M, ps_sxy, j, hx, K_X, A_X, B_X, sxy_x);
            syy_y = cpml_yh(g, M, ps_syy, i, hy, K_YH, A_YH, B_YH, syy_y);
            sxy_y = cpml_yh(g, M, ps_syx, i, hy, K_Y, A_Y, B_Y, sxy_y);
            if (sw == 0) {
                if (want_p1) {
                    vxp1[c] = div_dh(g, rip * (sxx_x + sxy_y));
                    vyp1[c] = div_dh(g, rjp * (sxy_x + syy_y));
                }
            } else if (NP > 4) {
                vxp1[c] = pl[(4 % NP) * P::PLS + pc] + vxo * DT;
                vyp1[c] = pl[(5 % NP) * P::PLS + pc] + vyo * DT;
            }
            vx[c] = vxo + div_dh(g, DT * rip * (sxx_x + sxy_y));
            vy[c] = vyo + div_dh(g, DT * rjp * (sxy_x + syy_y));
        }
    }
};

// velocity, SH (src/update_v_PML_SH.c:61-297); halo: sxz syz; plain: vz rjp
template <typename T, int FDOH, int TY, int NST>
struct OpVSh {
    using P = Pipe<T, FDOH, TY, 2, 2, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_SXZ];
        hz[1] = zb + tm.pid[P_SYZ];
        pz[0] = {zb + tm.pid[P_VZ], false};
        pz[1] = {mb + tm.mid[M_RJP], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        if (g.free_surf && ti.j0 == 1) rows<true>(ti, h, pl);
        else rows<false>(ti, h, pl);
    }
    template <bool MIR>
    __device__ __forceinline__ void rows(const TileIdx &ti, const T *h, const T *pl) const {
        const T *t_sxz = h, *t_syz = h + P::BOXS;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ vz = S.base + so + S.off[P_VZ];
        T *__restrict__ vzp1 = S.base + so + S.off[P_VZP1];
        T *ps_x = S.psix[X_SXZ] + slot * S.psix_slot, *ps_y = S.psiy[Y_SYZ] + slot * S.psiy_slot;
        const T DT = g.dt;
        const int col = tx + P::XH;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + col, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            T sxz_x = 0, syz_y = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) sxz_x += hc.w[m] * (t_sxz[rc + m - 1] - t_sxz[rc - m]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++)
                syz_y += hc.w[m] * (ldy<MIR, false, P>(t_syz, jj, col, m) - ldy<MIR, false, P>(t_syz, jj, col, 1 - m));
            sxz_x = cpml_xh(g, M, ps_x, j, hx, K_X, A_X, B_X, sxz_x);
            syz_y = cpml_yh(g, M, ps_y, i, hy, K_YH, A_YH, B_YH, syz_y);
            const T vzo = pl[pc];
            vzp1[c] = vzo;
            vz[c] = vzo + div_dh(g, pl[P::PLS + pc] * DT * (sxz_x + syz_y));
        }
    }
};

// velocity, acoustic (src/update_v_acoustic_PML.c:72-148, default :396-409)
// halo: sp; plain: vx vy rip rjp [+ vxp1 vyp1 in the adjoint, NP=6]
template <typename T, int FDOH, int TY, int NP, int NST>
struct OpVAc {
    using P = Pipe<T, FDOH, TY, 1, NP, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    int sw, want_p1;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_SP];
        pz[0] = {zb + tm.pid[P_VX], false};
        pz[1] = {zb + tm.pid[P_VY], false};
        pz[2] = {mb + tm.mid[M_RIP], true};
        pz[3] = {mb + tm.mid[M_RJP], true};
        if (NP > 4) {
            pz[4 % NP] = {zb + tm.pid[P_VXP1], false};
            pz[5 % NP] = {zb + tm.pid[P_VYP1], false};
        }
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        if (g.free_surf && ti.j0 == 1) rows<true>(ti, h, pl);
        else rows<false>(ti, h, pl);
    }
    template <bool MIR>
    __device__ __forceinline__ void rows(const TileIdx &ti, const T *h, const T *pl) const {
        const T *t_sp = h;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ vx = S.base + so + S.off[P_VX];
        T *__restrict__ vy = S.base + so + S.off[P_VY];
        T *__restrict__ vxp1 = S.base + so + S.off[P_VXP1];
        T *__restrict__ vyp1 = S.base + so + S.off[P_VYP1];
        T *ps_x = S.psix[X_SXX] + slot * S.psix_slot, *ps_y = S.psiy[Y_SYY] + slot * S.psiy_slot;
        const T DT = g.dt, DH = g.dh;
        const int col = tx + P::XH;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + col, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            const T rip = pl[2 * P::PLS + pc], rjp = pl[3 * P::PLS + pc];
            T sp_x = 0, sp_y = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) sp_x += hc.w[m] * (t_sp[rc + m] - t_sp[rc - m + 1]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++)
                sp_y += hc.w[m] * (ldy<MIR, false, P>(t_sp, jj, col, m) - ldy<MIR, false, P>(t_sp, jj, col, 1 - m));
            const T vxo = pl[pc], vyo = pl[P::PLS + pc];
            if (g.quirk_hi) {
                const T dtdh = DT * DT / DH;
                vx[c] = vxo + sp_x * dtdh * rip;
                vy[c] = vyo + sp_y * dtdh * rjp;
                continue;
            }
            sp_x = cpml_xh(g, M, ps_x, j, hx, K_XH, A_XH, B_XH, sp_x);
            sp_y = cpml_yh(g, M, ps_y, i, hy, K_YH, A_YH, B_YH, sp_y);
            if (sw == 0) {
                if (want_p1) {
                    vxp1[c] = div_dh(g, rip * (sp_x));
                    vyp1[c] = div_dh(g, rjp * (sp_y));
                }
            } else if (NP > 4) {
                vxp1[c] = pl[(4 % NP) * P::PLS + pc] + vxo * DT;
                vyp1[c] = pl[(5 % NP) * P::PLS + pc] + vyo * DT;
            }
            vx[c] = vxo + div_dh(g, DT * rip * (sp_x));
            vy[c] = vyo + div_dh(g, DT * rjp * (sp_y));
        }
    }
};

// velocity derivatives of the stress kernels from the staged vx, vy tiles
template <typename P, typename T, int FDOH>
struct VDer {
    T vxx, vyx, vxy, vyy;
    __device__ __forceinline__ VDer(const Hc<T, FDOH> &hc, const T *t_vx, const T *t_vy, int rc) {
        vxx = 0;
        vyx = 0;
        vxy = 0;
        vyy = 0;
#pragma unroll
        for (int m = 1; m <= FDOH; m++) vxx += hc.w[m] * (t_vx[rc + m - 1] - t_vx[rc - m]);
#pragma unroll
        for (int m = 1; m <= FDOH; m++) vyx += hc.w[m] * (t_vy[rc + m] - t_vy[rc - m + 1]);
#pragma unroll
        for (int m = 1; m <= FDOH; m++) vxy += hc.w[m] * (t_vx[rc + m * P::BW] - t_vx[rc - (m - 1) * P::BW]);
#pragma unroll
        for (int m = 1; m <= FDOH; m++) vyy += hc.w[m] * (t_vy[rc + (m - 1) * P::BW] - t_vy[rc - m * P::BW]);
    }
};

// stress, P-SV elastic (src/update_s_elastic_PML.c:151-241; 10/12: :442-535)
// halo: vx vy; plain: sxx syy sxy uipjp f g (reference 10/12 branch: uipjp vs vp)
template <typename T, int FDOH, int TY, int NST>
struct OpSEl {
    using P = Pipe<T, FDOH, TY, 2, 6, NST>;
    using D = Dbl<T>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SXX], false};
        pz[1] = {zb + tm.pid[P_SYY], false};
        pz[2] = {zb + tm.pid[P_SXY], false};
        pz[3] = {mb + tm.mid[M_UIPJP], true};
        pz[4] = {mb + tm.mid[g.quirk_hi ? M_VS : M_F], true};
        pz[5] = {mb + tm.mid[g.quirk_hi ? M_VP : M_G], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        const T *t_vx = h, *t_vy = h + P::BOXS;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ sxx = S.base + so + S.off[P_SXX];
        T *__restrict__ syy = S.base + so + S.off[P_SYY];
        T *__restrict__ sxy = S.base + so + S.off[P_SXY];
        T *ps_vxx = S.psix[X_VXX] + slot * S.psix_slot, *ps_vyx = S.psix[X_VYX] + slot * S.psix_slot;
        T *ps_vyy = S.psiy[Y_VYY] + slot * S.psiy_slot, *ps_vxy = S.psiy[Y_VXY] + slot * S.psiy_slot;
        const T DT = g.dt, DH = g.dh;
        const T dhi = DT / DH;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + tx + P::XH, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            VDer<P, T, FDOH> d(hc, t_vx, t_vy, rc);
            T vxx = d.vxx * dhi, vyx = d.vyx * dhi, vxy = d.vxy * dhi, vyy = d.vyy * dhi;
            const T sxx0 = pl[pc], syy0 = pl[P::PLS + pc], sxy0 = pl[2 * P::PLS + pc];
            if (g.quirk_hi) {
                const T fipjp = pl[3 * P::PLS + pc] * DT, f = pl[4 * P::PLS + pc] * DT, gg = pl[5 * P::PLS + pc] * DT;
                sxy[c] = sxy0 + (fipjp * (vxy + vyx));
                sxx[c] = (T)((D)sxx0 + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vyy)));
                syy[c] = (T)((D)syy0 + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vxx)));
                continue;
            }
            vxx = cpml_xh(g, M, ps_vxx, j, hx, K_X, A_X, B_X, vxx);
            vyx = cpml_xh(g, M, ps_vyx, j, hx, K_XH, A_XH, B_XH, vyx);
            vyy = cpml_yh(g, M, ps_vyy, i, hy, K_Y, A_Y, B_Y, vyy);
            vxy = cpml_yh(g, M, ps_vxy, i, hy, K_YH, A_YH, B_YH, vxy);
            const T fipjp = pl[3 * P::PLS + pc], f = pl[4 * P::PLS + pc], gg = pl[5 * P::PLS + pc];
            sxy[c] = sxy0 + fipjp * (vyx + vxy);
            sxx[c] = (T)((D)sxx0 + ((D)(gg * (vxx + vyy)) + ((D)2 * (D)f * (D)vxx)));
            syy[c] = (T)((D)syy0 + ((D)(gg * (vxx + vyy)) + ((D)2 * (D)f * (D)vyy)));
        }
    }
};

// stress, P-SV viscoelastic with LL SLS (src/update_s_visc_PML.c)
// halo: vx vy; plain: sxx syy sxy, r[LL] p[LL] q[LL], fipjp f g mu pi muipjp
// (non-uniform tau planes are read directly from HBM)
template <typename T, int FDOH, int TY, int LL, int NST>
struct OpSVisc {
    static constexpr int NP = 3 + 3 * LL + 6;
    using P = Pipe<T, FDOH, TY, 2, NP, NST>;
    using D = Dbl<T>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SXX], false};
        pz[1] = {zb + tm.pid[P_SYY], false};
        pz[2] = {zb + tm.pid[P_SXY], false};
#pragma unroll
        for (int l = 0; l < LL; l++) {
            pz[3 + l] = {zb + tm.mem_pid[0] + l, false};
            pz[3 + LL + l] = {zb + tm.mem_pid[1] + l, false};
            pz[3 + 2 * LL + l] = {zb + tm.mem_pid[2] + l, false};
        }
        pz[3 + 3 * LL + 0] = {mb + tm.mid[M_FIPJPV], true};
        pz[3 + 3 * LL + 1] = {mb + tm.mid[M_FV], true};
        pz[3 + 3 * LL + 2] = {mb + tm.mid[M_GV], true};
        pz[3 + 3 * LL + 3] = {mb + tm.mid[M_MUR], true};
        pz[3 + 3 * LL + 4] = {mb + tm.mid[M_PIR], true};
        pz[3 + 3 * LL + 5] = {mb + tm.mid[M_MUIPJPR], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        const T *t_vx = h, *t_vy = h + P::BOXS;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        const long long mo = (long long)model * M.model_stride;
        T *__restrict__ sxx = S.base + so + S.off[P_SXX];
        T *__restrict__ syy = S.base + so + S.off[P_SYY];
        T *__restrict__ sxy = S.base + so + S.off[P_SXY];
        T *__restrict__ mr = S.base + so + S.mem_off[0];
        T *__restrict__ mp = S.base + so + S.mem_off[1];
        T *__restrict__ mq = S.base + so + S.mem_off[2];
        T *ps_vxx = S.psix[X_VXX] + slot * S.psix_slot, *ps_vyx = S.psix[X_VYX] + slot * S.psix_slot;
        T *ps_vyy = S.psiy[Y_VYY] + slot * S.psiy_slot, *ps_vxy = S.psiy[Y_VXY] + slot * S.psiy_slot;
        const T *ts_p = M.m[M_TAUS] ? M.m[M_TAUS] + mo : nullptr, *tp_p = M.m[M_TAUP] ? M.m[M_TAUP] + mo : nullptr,
                *tsij_p = M.m[M_TAUSIPJP] ? M.m[M_TAUSIPJP] + mo : nullptr;
        const long long PL = g.plane;
        const T DT = g.dt, DH = g.dh;
        const T dhi = (T)(1.0 / (double)DH), dthalbe = (T)((double)DT / 2.0);
        constexpr int CO = 3 + 3 * LL;  // first coefficient plane
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + tx + P::XH, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            VDer<P, T, FDOH> d(hc, t_vx, t_vy, rc);
            T vxx = d.vxx * dhi, vyx = d.vyx * dhi, vxy = d.vxy * dhi, vyy = d.vyy * dhi;
            if (!g.quirk_hi) {
                vxx = cpml_xh(g, M, ps_vxx, j, hx, K_X, A_X, B_X, vxx);
                vyx = cpml_xh(g, M, ps_vyx, j, hx, K_XH, A_XH, B_XH, vyx);
                vyy = cpml_yh(g, M, ps_vyy, i, hy, K_Y, A_Y, B_Y, vyy);
                vxy = cpml_yh(g, M, ps_vxy, i, hy, K_YH, A_YH, B_YH, vxy);
            }
            T sumr = 0, sump = 0, sumq = 0;
#pragma unroll
            for (int l = 0; l < LL; l++) {
                sumr += pl[(3 + l) * P::PLS + pc];
                sump += pl[(3 + LL + l) * P::PLS + pc];
                sumq += pl[(3 + 2 * LL + l) * P::PLS + pc];
            }
            const T fipjp = pl[CO * P::PLS + pc], f = pl[(CO + 1) * P::PLS + pc], gg = pl[(CO + 2) * P::PLS + pc];
            const T mu = pl[(CO + 3) * P::PLS + pc], pi = pl[(CO + 4) * P::PLS + pc],
                    muij = pl[(CO + 5) * P::PLS + pc];
            const T ts = ts_p ? ts_p[c] : (T)g.taus0, tp = tp_p ? tp_p[c] : (T)g.taup0,
                    tsij = tsij_p ? tsij_p[c] : (T)g.tausipjp0;
            const T s_xy = pl[2 * P::PLS + pc] + ((fipjp * (vxy + vyx)) + (dthalbe * sumr));
            const T s_xx = (T)((D)pl[pc] + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vyy) + (D)(dthalbe * sump)));
            const T s_yy =
                (T)((D)pl[P::PLS + pc] + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vxx) + (D)(dthalbe * sumq)));
            sumr = sump = sumq = 0;
#pragma unroll
            for (int l = 0; l < LL; l++) {
                const T eta = g.eta[l + 1];
                const T dip = muij * eta * tsij, dd = mu * eta * ts, e = pi * eta * tp;
                const T rr = (T)g.bip[l + 1] * (pl[(3 + l) * P::PLS + pc] * (T)g.cip[l + 1] - (dip * (vxy + vyx)));
                const T pp = (T)((D)g.bjm[l + 1] *
                                 ((D)(pl[(3 + LL + l) * P::PLS + pc] * (T)g.cjm[l + 1] - (e * (vxx + vyy))) +
                                  ((D)2 * (D)dd * (D)vyy)));
                const T qq = (T)((D)g.bjm[l + 1] *
                                 ((D)(pl[(3 + 2 * LL + l) * P::PLS + pc] * (T)g.cjm[l + 1] - (e * (vxx + vyy))) +
                                  ((D)2 * (D)dd * (D)vxx)));
                mr[c + l * PL] = rr;
                mp[c + l * PL] = pp;
                mq[c + l * PL] = qq;
                sumr += rr;
                sump += pp;
                sumq += qq;
            }
            sxy[c] = s_xy + (dthalbe * sumr);
            sxx[c] = s_xx + (dthalbe * sump);
            syy[c] = s_yy + (dthalbe * sumq);
        }
    }
};

// stress, SH elastic (src/update_s_elastic_PML_SH.c); halo: vz; plain: sxz syz uipjp f
template <typename T, int FDOH, int TY, int NST>
struct OpSShEl {
    using P = Pipe<T, FDOH, TY, 1, 4, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VZ];
        pz[0] = {zb + tm.pid[P_SXZ], false};
        pz[1] = {zb + tm.pid[P_SYZ], false};
        pz[2] = {mb + tm.mid[M_UIPJP], true};
        pz[3] = {mb + tm.mid[M_F], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        const T *t_vz = h;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ sxz = S.base + so + S.off[P_SXZ];
        T *__restrict__ syz = S.base + so + S.off[P_SYZ];
        T *ps_x = S.psix[X_VZX] + slot * S.psix_slot, *ps_y = S.psiy[Y_VZY] + slot * S.psiy_slot;
        const T dhi = (T)g.dt / (T)g.dh;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + tx + P::XH, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            T vzx = 0, vzy = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vzx += hc.w[m] * (t_vz[rc + m] - t_vz[rc - m + 1]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vzy += hc.w[m] * (t_vz[rc + (m - 1) * P::BW] - t_vz[rc - m * P::BW]);
            vzx = vzx * dhi;
            vzy = vzy * dhi;
            vzx = cpml_xh(g, M, ps_x, j, hx, K_XH, A_XH, B_XH, vzx);
            vzy = cpml_yh(g, M, ps_y, i, hy, K_Y, A_Y, B_Y, vzy);
            sxz[c] = pl[pc] + (pl[2 * P::PLS + pc] * vzx);
            syz[c] = pl[P::PLS + pc] + (pl[3 * P::PLS + pc] * vzy);
        }
    }
};

// stress, SH viscoelastic (src/update_s_visc_PML_SH.c); halo: vz;
// plain: sxz syz t[LL] o[LL] fipjp f mu muipjp
template <typename T, int FDOH, int TY, int LL, int NST>
struct OpSShVisc {
    static constexpr int NP = 2 + 2 * LL + 4;
    using P = Pipe<T, FDOH, TY, 1, NP, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VZ];
        pz[0] = {zb + tm.pid[P_SXZ], false};
        pz[1] = {zb + tm.pid[P_SYZ], false};
#pragma unroll
        for (int l = 0; l < LL; l++) {
            pz[2 + l] = {zb + tm.mem_pid[3] + l, false};       // t
            pz[2 + LL + l] = {zb + tm.mem_pid[4] + l, false};  // o
        }
        pz[2 + 2 * LL + 0] = {mb + tm.mid[M_FIPJPV], true};
        pz[2 + 2 * LL + 1] = {mb + tm.mid[M_FV], true};
        pz[2 + 2 * LL + 2] = {mb + tm.mid[M_MUR], true};
        pz[2 + 2 * LL + 3] = {mb + tm.mid[M_MUIPJPR], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        const T *t_vz = h;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        const long long mo = (long long)model * M.model_stride;
        T *__restrict__ sxz = S.base + so + S.off[P_SXZ];
        T *__restrict__ syz = S.base + so + S.off[P_SYZ];
        T *__restrict__ mt = S.base + so + S.mem_off[3];
        T *__restrict__ mo_ = S.base + so + S.mem_off[4];
        T *ps_x = S.psix[X_VZX] + slot * S.psix_slot, *ps_y = S.psiy[Y_VZY] + slot * S.psiy_slot;
        const T *ts_p = M.m[M_TAUS] ? M.m[M_TAUS] + mo : nullptr,
                *tsij_p = M.m[M_TAUSIPJP] ? M.m[M_TAUSIPJP] + mo : nullptr;
        const long long PL = g.plane;
        const T DT = g.dt, DH = g.dh;
        const T dhi = (T)(1.0 / (double)DH), dthalbe = (T)((double)DT / 2.0);
        constexpr int CO = 2 + 2 * LL;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + tx + P::XH, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            T vzx = 0, vzy = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vzx += hc.w[m] * (t_vz[rc + m] - t_vz[rc - m + 1]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vzy += hc.w[m] * (t_vz[rc + (m - 1) * P::BW] - t_vz[rc - m * P::BW]);
            vzx = vzx * dhi;
            vzy = vzy * dhi;
            vzx = cpml_xh(g, M, ps_x, j, hx, K_XH, A_XH, B_XH, vzx);
            vzy = cpml_yh(g, M, ps_y, i, hy, K_Y, A_Y, B_Y, vzy);
            T sumo = 0, sumt = 0;
#pragma unroll
            for (int l = 0; l < LL; l++) {
                sumo += pl[(2 + LL + l) * P::PLS + pc];
                sumt += pl[(2 + l) * P::PLS + pc];
            }
            const T fipjp = pl[CO * P::PLS + pc], f = pl[(CO + 1) * P::PLS + pc];
            const T mu = pl[(CO + 2) * P::PLS + pc], muij = pl[(CO + 3) * P::PLS + pc];
            const T ts = ts_p ? ts_p[c] : (T)g.taus0, tsij = tsij_p ? tsij_p[c] : (T)g.tausipjp0;
            const T s_xz = pl[pc] + ((fipjp * vzx) + (dthalbe * sumo));
            const T s_yz = pl[P::PLS + pc] + ((f * vzy) + (dthalbe * sumt));
            sumo = sumt = 0;
#pragma unroll
            for (int l = 0; l < LL; l++) {
                const T eta = g.eta[l + 1];
                const T dip = muij * eta * tsij, dd = mu * eta * ts;
                const T o = (T)g.bip[l + 1] * (pl[(2 + LL + l) * P::PLS + pc] * (T)g.cip[l + 1] - (dip * vzx));
                const T t = (T)g.bjm[l + 1] * (pl[(2 + l) * P::PLS + pc] * (T)g.cjm[l + 1] - (dd * vzy));
                mo_[c + l * PL] = o;
                mt[c + l * PL] = t;
                sumt += t;
                sumo += o;
            }
            sxz[c] = s_xz + (dthalbe * sumo);
            syz[c] = s_yz + (dthalbe * sumt);
        }
    }
};

// pressure, acoustic (src/update_p_PML.c:55-273; default :275-287)
// halo: vx vy; plain: sp g (reference 10/12 branch: vp)
template <typename T, int FDOH, int TY, int NST>
struct OpPAc {
    using P = Pipe<T, FDOH, TY, 2, 2, NST>;
    KGrid g;
    KState<T> S;
    KModel<T> M;
    KTma tm;
    __device__ void planes(const TileIdx &ti, int model, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SP], false};
        pz[1] = {mb + tm.mid[g.quirk_hi ? M_VP : M_GAC], true};
    }
    __device__ void compute(const TileIdx &ti, int model, T *h, const T *pl) const {
        const T *t_vx = h, *t_vy = h + P::BOXS;
        const int tx = threadIdx.x, i = ti.i0 + tx, slot = ti.slot;
        if (i > g.nx) return;
        const int hx = strip_x(g, i);
        const Hc<T, FDOH> hc(g);
        const long long so = (long long)slot * S.slot_stride;
        T *__restrict__ sp = S.base + so + S.off[P_SP];
        T *ps_x = S.psix[X_VXX] + slot * S.psix_slot, *ps_y = S.psiy[Y_VYY] + slot * S.psiy_slot;
        const T DT = g.dt, DH = g.dh;
        const T dhi = DT / DH;
#pragma unroll
        for (int r = 0; r < P::RT; r++) {
            const int jj = threadIdx.y + 8 * r, j = ti.j0 + jj;
            if (j > g.ny) break;
            const int hy = strip_y(g, j);
            const int rc = (jj + P::H) * P::BW + tx + P::XH, pc = jj * 32 + tx;
            const int c = (int)pidx(g, j, i);
            T vxx = 0, vyy = 0;
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vxx += hc.w[m] * (t_vx[rc + m - 1] - t_vx[rc - m]);
#pragma unroll
            for (int m = 1; m <= FDOH; m++) vyy += hc.w[m] * (t_vy[rc + (m - 1) * P::BW] - t_vy[rc - m * P::BW]);
            if (g.quirk_hi) {
                const T gg = pl[P::PLS + pc] * DT;
                sp[c] = pl[pc] + (gg * (vxx + vyy)) * dhi;
                continue;
            }
            vxx = vxx * dhi;
            vyy = vyy * dhi;
            vxx = cpml_xh(g, M, ps_x, j, hx, K_X, A_X, B_X, vxx);
            vyy = cpml_yh(g, M, ps_y, i, hy, K_Y, A_Y, B_Y, vyy);
            sp[c] = pl[pc] + pl[P::PLS + pc] * (vxx + vyy);
        }
    }
};

// the kernel: one Op per launch, persistent over all tiles of all slots
template <typename T, int FDOH, int TY, int NH, int NP, int NST, typename Op>
__global__ void __launch_bounds__(kBlockThreads) kp_stencil(const __grid_constant__ KMaps maps,
                                                            const __grid_constant__ Op op, int nshots, int *err) {
    run_pipeline<T, FDOH, TY, NH, NP, NST>(op.g, maps, nshots, op, op.M.slot_model, err);
}

}  // namespace ifos
