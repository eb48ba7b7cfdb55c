// Persistent, TMA-pipelined stencil kernels (fp32).
//
// Each block loops over 64 x TY tiles of the grid (all shot slots).  A
// producer warp streams every input plane of a tile into a ring of NST
// shared-memory stages with bulk tensor loads (cp.async.bulk.tensor, never
// with cluster multicast): the planes that need neighbours (the stresses in
// the velocity update, the velocities in the stress update) as tile + halo
// boxes, the per-cell planes (fields, memory variables, coefficients) as
// plain tile boxes.  The compute warps release a stage as soon as they have
// read it and write their results straight to HBM with 8-byte stores (on
// snapshot steps also the stored wavefield components, into the snapshot
// buffer), so the ring only ever waits on loads.
//
// A thread owns two adjacent columns (float2 shared-memory accesses) of the
// RT = TY / (compute warps) consecutive rows of its warp: the x-taps of both
// columns come from one aligned window, the y-taps of neighbouring rows from
// the same words, and the cells of a thread are independent work.  Interior
// tiles (no CPML strip cell) take a path without strip code.  The per-cell
// arithmetic is the reference's, in the same order and with the same
// float/double promotions as the one-thread-per-cell kernels of
// ifos_kernels.cuh.
#pragma once
#include <type_traits>

#include "ifos_kernels.cuh"
#include "ifos_snap.cuh"
#include "ifos_tma.cuh"

// 1: the reference's double-promoted terms are evaluated in double (bit-exact);
// 0: in single precision
#ifndef IFOS_EXACT
#define IFOS_EXACT 1
#endif

// compute warps per block (the block adds one producer warp)
#ifndef IFOS_NCW
#define IFOS_NCW 8
#endif

namespace ifos {

constexpr int kComputeWarps = IFOS_NCW;
// Resident blocks per SM the elastic stress op's launch bounds aim for: four
// for FDORDER <= 4 (400 x 160 batch of 128: 100-105 vs 109 us per launch),
// three otherwise.
constexpr int sblocks(int fdoh) {
#ifdef IFOS_SBLOCKS
    return IFOS_SBLOCKS + 0 * fdoh;
#else
    return fdoh <= 2 ? 4 : 3;
#endif
}
// Resident blocks per SM the velocity ops' launch bounds aim for.  Four
// (registers capped at 56, two ring stages) were faster for FDORDER <= 4
// (400 x 160 batch of 128: 94 vs 103 us per launch), three for the wider
// stencils (2000 x 600, FDORDER 8, one shot: 22.3 vs 24.6 us).
constexpr int vblocks(int fdoh) {
#ifdef IFOS_VBLOCKS
    return IFOS_VBLOCKS + 0 * fdoh;
#else
    return fdoh <= 2 ? 4 : 3;
#endif
}
constexpr int kBlockThreads = 32 * kComputeWarps + 32;
constexpr int kTileX = 64;

using D = std::conditional<IFOS_EXACT != 0, double, float>::type;

// Plane ids for the TMA z coordinate: state plane = slot * planes_per_slot + pid,
// model plane = model * model_planes + mid; snap_comp: the snapshot
// component of a state plane.
struct KTma {
    int planes_per_slot;
    int pid[NP_FIELD];
    int mem_pid[5];
    int model_planes;
    int mid[NM_PLANE];
    int snap_ntd, snap_ncomp;
    int snap_comp[NP_FIELD];  // component index of a state plane (-1: not stored)
};

struct KMaps {
    CUtensorMap halo;   // state planes, box (64+2XH) x (TY+2H)
    CUtensorMap plain;  // state planes, box 64 x TY (loads and stores)
    CUtensorMap model;  // model planes, box 64 x TY
};

// fp32 snapshot written by a launch: snapshot of slot 0 being stored (NULL:
// none), floats between slots, NX*NY, and whether rows start 8-byte aligned
// (NX even) for pair stores.
// the snapshot a stencil launch stores (base NULL: none)
struct KSnapOut {
    char *base;            // this snapshot of slot 0
    long long slot_bytes;  // bytes between slots
    long long n;           // NX*NY
    int pairs;             // NX even: column pairs are aligned for vector stores
    int f16;               // fp16 segments (IFOS_SNAP_F16S); else fp32
    long long ex_off;      // fp16: bytes from a snapshot to its segment scales [comp][NY][segs]
    int segs;              // fp16: segments per row
};

// NH halo boxes, NP loaded plain boxes, NO output-only plain boxes, NST stages
template <int FDOH, int TY, int NH, int NP, int NO, int NST, int BCAP = 3>
struct Pipe {
    static constexpr int TX = kTileX, H = FDOH;
    static constexpr int HE = (FDOH + 1) & ~1;       // x window half width (even)
    static constexpr int XH = ((FDOH + 3) / 4) * 4;  // staged x halo (16-byte TMA alignment)
    static constexpr int BW = TX + 2 * XH, BH = TY + 2 * H;
    static constexpr int BOXS = ((BW * BH * 4 + 127) / 128) * 32;  // 128-byte aligned box stride
    static constexpr int PLS = TX * TY;
    static constexpr int NHALO = NH, NLOAD = NP, NPL = NP + NO, STAGES = NST;
    static constexpr int STAGE = NH * BOXS + NPL * PLS;
    static constexpr int RT = TY / kComputeWarps;  // rows per thread
    static constexpr int TILE_Y = TY;
    static constexpr uint32_t TXB = (uint32_t)((NH * BW * BH + NP * PLS) * 4);
    static constexpr size_t bytes() { return (size_t)NST * STAGE * 4; }
    static constexpr int BLOCK_CAP = BCAP;  // resident blocks per SM the launch bounds aim for
    static_assert(TY % kComputeWarps == 0, "tile height must be a multiple of the compute warps");
    static_assert(HE <= XH, "x window exceeds the staged halo");
};

// One tile as the producer hands it to the compute warps.
struct __align__(16) TileInfo {
    int slot, i0, j0;
    int model;   // model index of the slot
    int ystrip;  // some row of the tile lies in a CPML y strip
    int pad[3];
};

// Tile t of a launch.  Slot-major order walks all tiles of slot 0, then of
// slot 1, ...; slot-minor order gives consecutive t the same tile of
// consecutive slots, so the CTAs resident at one time share the model tiles
// of shots over the same model (one HBM read, the rest from L2).
//
// CPML-first order (tile order bit 1): the spatial rank runs over the tiles
// that meet a CPML strip first -- the tile rows in a y strip (top without a
// free surface, bottom), then the x-strip columns (left, right) of the other
// rows -- and the interior last, each region row by row.  Strip tiles take
// the slower CPML path of every op; ranked first, the round-robin of tiles
// over the persistent CTAs hands each CTA the same number of them (within
// one), so the CTAs finish together instead of the ones that drew the strip
// columns finishing last.  A bijection on [0, ntx*nty).
__device__ __forceinline__ int cpml_first(int rank, int ntx, int nty, int TY, const KGrid &g) {
    if (g.fw <= 0) return rank;
    const int cl = min(ntx, (g.fw - 1) / kTileX + 1);  // tile columns with i0 <= FW
    const int vx = g.nx - g.fw + 1 - kTileX;            // right strip: min(i0+63, NX) >= NX-FW+1
    const int xr0 = max(cl, vx <= 0 ? 0 : (vx + kTileX - 1) / kTileX);
    const int rt = g.free_surf ? 0 : min(nty, (g.fw - 1) / TY + 1);  // tile rows with j0 <= FW
    const int vy = g.ny - g.fw + 1 - TY;                              // bottom strip: j0+TY-1 >= NY-FW+1
    const int yb0 = min(nty, max(rt, vy <= 0 ? 0 : (vy + TY - 1) / TY));
    const int nys = rt + (nty - yb0);  // rows in a y strip
    if (rank < nys * ntx) {
        const int r = rank / ntx;
        return (r < rt ? r : yb0 + (r - rt)) * ntx + (rank - r * ntx);
    }
    rank -= nys * ntx;
    const int ce = cl + (ntx - xr0);  // x-strip columns
    const int mid = nty - nys;        // rows between the y strips: rt .. yb0-1
    if (rank < mid * ce) {
        const int r = rank / ce, c = rank - r * ce;
        return (rt + r) * ntx + (c < cl ? c : xr0 + (c - cl));
    }
    rank -= mid * ce;
    const int w = ntx - ce;  // > 0 here: the regions above hold every tile when it is 0
    const int r = rank / w;
    return (rt + r) * ntx + cl + (rank - r * w);
}

__device__ __forceinline__ void tile_of(int t, int ntx, int nty, int TY, int nshots, int order, const KGrid &g,
                                        TileInfo &r) {
    int rem;
    if (order & 1) {
        rem = t / nshots;
        r.slot = t - rem * nshots;
    } else {
        const int per = ntx * nty;
        r.slot = t / per;
        rem = t - r.slot * per;
    }
    if (order & 2) rem = cpml_first(rem, ntx, nty, TY, g);
    const int tyi = rem / ntx;
    r.i0 = (rem - tyi * ntx) * kTileX + 1;
    r.j0 = tyi * TY + 1;
}

// rows j0 .. j0+TY-1 meet a y strip (top: j <= FW without free surface,
// bottom: j >= NY-FW+1)
__device__ __forceinline__ int tile_in_ystrip(const KGrid &g, int j0, int TY) {
    if (g.fw == 0) return 0;
    if (!g.free_surf && j0 <= g.fw) return 1;
    return j0 + TY - 1 >= g.ny - g.fw + 1 ? 1 : 0;
}

// source of a plain-box load: a state plane or a model plane
struct PlainSrc {
    int z;
    bool model;
};

// Warp-specialised persistent driver.  Warps 0..kComputeWarps-1 compute; lane
// 0 of the last warp produces: it walks the same tile sequence, waits until a
// stage has been released by all compute warps ("empty" barrier, one arrival
// per warp), and issues the bulk tensor loads of the next tile into it
// ("full" barrier, completed by the transaction bytes).  The tile's indices
// travel through shared memory with the stage.  Every wait is bounded: a
// wait that gives up records its code in *err (16/17: a compute warp on a
// stage's loads, 18: the producer on a stage's release) and the block winds
// down after its copies in flight: when the producer gives up before tile
// k_stop it records k_stop (stop_at) and issues nothing more; the compute
// warps still wait for every tile it issued (so that no copy into the ring is
// in flight when the block exits), compute none of them, and leave at k_stop.
template <typename P, typename Op>
__device__ __forceinline__ void run_pipeline(const KGrid &g, const KMaps &mp, int nshots, const Op &op, int *err) {
    constexpr int NST = P::STAGES, NH = P::NHALO, NP = P::NLOAD, TY = P::TILE_Y;
    extern __shared__ __align__(1024) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[NST], empty[NST];
    __shared__ TileInfo tinfo[NST];
    __shared__ int stop_at;  // -1 while the producer runs, else the first tile it did not issue
    float *smem = reinterpret_cast<float *>(sm_raw);
    const int ntx = (g.nx + kTileX - 1) / kTileX, nty = (g.ny + TY - 1) / TY;
    const int ntiles = ntx * nty * nshots;
    const int warp = threadIdx.y;
    if (warp == kComputeWarps && threadIdx.x == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kComputeWarps);
        }
        stop_at = -1;
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == kComputeWarps) {
        if (threadIdx.x != 0) return;
        // Tile k in stage k % NST.  The per-cell planes of the first NST tiles
        // are not written by the preceding kernel of the stream, so they are
        // requested before waiting for it; everything else after.
        auto issue = [&](int k, bool halo, bool plain) {
            const int st = k % NST;
            TileInfo ti;
            tile_of(blockIdx.x + k * gridDim.x, ntx, nty, TY, nshots, g.tile_order, g, ti);
            float *stage = smem + st * P::STAGE;
            uint64_t *bar = &full[st];
            if (plain) {
                ti.model = op.M.slot_model[ti.slot];
                ti.ystrip = tile_in_ystrip(g, ti.j0, TY);
                tinfo[st] = ti;
                mbar_expect_tx(bar, P::TXB);
            } else {
                ti.model = tinfo[st].model;
            }
            int hz[NH > 0 ? NH : 1];
            PlainSrc pz[NP > 0 ? NP : 1];
            op.planes(ti, hz, pz);
            if (halo) {
                const int bx = HX + ti.i0 - 1 - P::XH, by = HY + ti.j0 - 1 - P::H;
#pragma unroll
                for (int h = 0; h < NH; h++) tma_load_3d(stage + h * P::BOXS, &mp.halo, bx, by, hz[h], bar);
            }
            if (plain) {
                const int px = HX + ti.i0 - 1, py = HY + ti.j0 - 1;
#pragma unroll
                for (int q = 0; q < NP; q++)
                    tma_load_3d(stage + NH * P::BOXS + q * P::PLS, pz[q].model ? &mp.model : &mp.plain, px, py,
                                pz[q].z, bar);
            }
        };
        int npre = 0;
        while (npre < NST && blockIdx.x + npre * gridDim.x < ntiles) issue(npre++, false, true);
        pdl_wait();
        for (int k = 0; k < npre; k++) issue(k, true, false);
        pdl_launch();
        for (int k = npre;; k++) {
            const int t = blockIdx.x + k * gridDim.x;
            if (t >= ntiles) break;
            const int st = k % NST;
            if (!mbar_wait_bounded(&empty[st], (uint32_t)(((k / NST) - 1) & 1), err, 18, (long)g.prod_polls)) {
                *(volatile int *)&stop_at = k;
                break;
            }
            issue(k, true, true);
        }
        return;
    }
    volatile int *stop = &stop_at;
    for (int k = 0;; k++) {
        const int t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int st = k % NST;
        const uint32_t parity = (uint32_t)((k / NST) & 1);
        bool landed = false;
        for (long it = 0; it < (1L << 16) && !landed; it++) {
            landed = mbar_try_wait(&full[st], parity);
            if (!landed && *stop >= 0 && k >= *stop) return;  // never issued: nothing in flight for it
        }
        if (!landed) {
            if (err) atomicExch(err, 16);
            mbar_wait_bounded(&full[st], parity, err, 17);
            return;
        }
        if (*stop >= 0) continue;  // the producer stopped: drain the tiles it issued, compute none
        const TileInfo ti = tinfo[st];
        const float *stage = smem + st * P::STAGE;
        op.compute(ti, stage, stage + NH * P::BOXS, &empty[st]);
    }
}

// ---------------------------------------------------------------------------
// Difference stencils of a thread's column pair (cells e = 0, 1 at staged
// columns c0 + e).  The m=1 term starts each sum and the others are added in
// order, as in the reference's written-out expressions
// (src/update_v_PML.c:164-175); Z0: the sum is accumulated from zero, as in
// its generic loops (the FDORDER 10/12 default branches, e.g.
// src/update_p_PML.c:275-287).  fwd: sum_m w_m (f[+m] - f[-m+1]);
// bwd: sum_m w_m (f[+m-1] - f[-m]).

// FD weights of one launch, in registers
template <int FDOH>
struct Hc {
    float w[FDOH + 1];
    __device__ __forceinline__ explicit Hc(const KGrid &g) {
#pragma unroll
        for (int m = 0; m <= FDOH; m++) w[m] = g.hc[m];
    }
};

// staged values of one row at columns c0-HE .. c0+HE+1 (c0 - HE even)
template <int HE>
struct XWin {
    float v[2 * HE + 2];
    __device__ __forceinline__ void load(const float *row, int c0) {
#pragma unroll
        for (int q = 0; q <= HE; q++) {
            const float2 a = *reinterpret_cast<const float2 *>(row + c0 - HE + 2 * q);
            v[2 * q] = a.x;
            v[2 * q + 1] = a.y;
        }
    }
};
template <int FDOH, int HE, bool Z0 = false>
__device__ __forceinline__ float xfwd(const Hc<FDOH> &hc, const XWin<HE> &W, int e) {
    float s = hc.w[1] * (W.v[HE + e + 1] - W.v[HE + e]);
    if (Z0) s = 0.0f + s;
#pragma unroll
    for (int m = 2; m <= FDOH; m++) s += hc.w[m] * (W.v[HE + e + m] - W.v[HE + e - m + 1]);
    return s;
}
template <int FDOH, int HE, bool Z0 = false>
__device__ __forceinline__ float xbwd(const Hc<FDOH> &hc, const XWin<HE> &W, int e) {
    float s = hc.w[1] * (W.v[HE + e] - W.v[HE + e - 1]);
    if (Z0) s = 0.0f + s;
#pragma unroll
    for (int m = 2; m <= FDOH; m++) s += hc.w[m] * (W.v[HE + e + m - 1] - W.v[HE + e - m]);
    return s;
}

// Column pair of a staged halo box at row offset dy from tile row jj.  In the
// top row of tiles with a free surface (MIR) rows j<=0 read the imaged value
// the reference's ghost rows hold when the velocity is updated: -f(2-j) for
// syy, syz, sp (src/surface_elastic_PML.c:59) and -f(1-j) for sxy (:60).
template <bool MIR, bool ODD, typename P>
__device__ __forceinline__ float2 ldy2(const float *t, int jj, int c0, int dy) {
    const int rr = jj + P::H + dy;
    if (MIR && rr < P::H) {
        const int src = ODD ? 2 * P::H - rr - 1 : 2 * P::H - rr;
        const float2 a = *reinterpret_cast<const float2 *>(t + src * P::BW + c0);
        return make_float2(-a.x, -a.y);
    }
    return *reinterpret_cast<const float2 *>(t + rr * P::BW + c0);
}
template <bool MIR, bool ODD, typename P, int FDOH, bool Z0 = false>
__device__ __forceinline__ float2 yfwd2(const Hc<FDOH> &hc, const float *t, int jj, int c0) {
    float2 a = ldy2<MIR, ODD, P>(t, jj, c0, 1), b = ldy2<MIR, ODD, P>(t, jj, c0, 0);
    float2 s = make_float2(hc.w[1] * (a.x - b.x), hc.w[1] * (a.y - b.y));
    if (Z0) s = make_float2(0.0f + s.x, 0.0f + s.y);
#pragma unroll
    for (int m = 2; m <= FDOH; m++) {
        a = ldy2<MIR, ODD, P>(t, jj, c0, m);
        b = ldy2<MIR, ODD, P>(t, jj, c0, 1 - m);
        s.x += hc.w[m] * (a.x - b.x);
        s.y += hc.w[m] * (a.y - b.y);
    }
    return s;
}
template <bool MIR, bool ODD, typename P, int FDOH, bool Z0 = false>
__device__ __forceinline__ float2 ybwd2(const Hc<FDOH> &hc, const float *t, int jj, int c0) {
    float2 a = ldy2<MIR, ODD, P>(t, jj, c0, 0), b = ldy2<MIR, ODD, P>(t, jj, c0, -1);
    float2 s = make_float2(hc.w[1] * (a.x - b.x), hc.w[1] * (a.y - b.y));
    if (Z0) s = make_float2(0.0f + s.x, 0.0f + s.y);
#pragma unroll
    for (int m = 2; m <= FDOH; m++) {
        a = ldy2<MIR, ODD, P>(t, jj, c0, m - 1);
        b = ldy2<MIR, ODD, P>(t, jj, c0, -m);
        s.x += hc.w[m] * (a.x - b.x);
        s.y += hc.w[m] * (a.y - b.y);
    }
    return s;
}

__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void sts2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
__device__ __forceinline__ float pick(const float2 &v, int e) { return e ? v.y : v.x; }

// CPML on a cell known to lie in the strip (hx / hy > 0), src/update_v_PML.c:177-226
__device__ __forceinline__ float pml_x(const KGrid &g, const KModel<float> &M, float *strip, int j, int hx, int kk,
                                       int ka, int kb, float d) {
    return cpml(strip + (j - 1) * (2 * g.fw) + (hx - 1), prof(M, g, kb, hx), prof(M, g, ka, hx), prof(M, g, kk, hx),
                d, g.k_one);
}
__device__ __forceinline__ float pml_y(const KGrid &g, const KModel<float> &M, float *strip, int i, int hy, int kk,
                                       int ka, int kb, float d) {
    return cpml(strip + (hy - 1) * g.nx + (i - 1), prof(M, g, kb, hy), prof(M, g, ka, hy), prof(M, g, kk, hy), d,
                g.k_one);
}

// Per-thread geometry of a tile: the column pair, its validity and strip
// indices, and whether the tile needs the CPML path at all.
struct Cols {
    int lane, c0, i;
    bool v0, v1;
    int hx0, hx1;
    __device__ __forceinline__ Cols(const KGrid &g, const TileInfo &ti, int XH, bool strips) {
        lane = threadIdx.x;
        c0 = XH + 2 * lane;
        i = ti.i0 + 2 * lane;
        v0 = i <= g.nx;
        v1 = i + 1 <= g.nx;
        hx0 = (strips && v0) ? strip_x(g, i) : 0;
        hx1 = (strips && v1) ? strip_x(g, i + 1) : 0;
    }
    __device__ __forceinline__ int hx(int e) const { return e ? hx1 : hx0; }
    __device__ __forceinline__ bool valid(int e) const { return e ? v1 : v0; }
};

// Store a column pair: both cells (8-byte store) or only the first one
// (the last column of an odd NX).
__device__ __forceinline__ void gput2(float *p, float n0, float n1, bool pair, bool v0) {
    if (pair) *reinterpret_cast<float2 *>(p) = make_float2(n0, n1);
    else if (v0) *p = n0;
}

// Row addresses of a thread's column pair: the cell (j, i) in the state of a
// slot and, on snapshot steps, in the snapshot being stored.
struct RowOut {
    float *st;          // state plane 0 at (j, i)
    float *sn;          // fp32 snapshot component 0 at (j, i), NULL when not storing fp32
    __half *sh;         // fp16 snapshot component 0 at (j, i), NULL when not storing fp16
    float *se;          // fp16: scale of component 0 for this row segment
    long long se_comp;  // fp16: scales between components
    bool pair, v0, spair;
    __device__ __forceinline__ RowOut(const KGrid &g, const KState<float> &S, const KSnapOut &so, int slot, int j,
                                      const Cols &cl) {
        st = S.base + (long long)slot * S.slot_stride + ((j - 1 + HY) * g.pitch + (cl.i - 1 + HX));
        sn = nullptr;
        sh = nullptr;
        se = nullptr;
        se_comp = 0;
        if (so.base) {
            char *b = so.base + slot * so.slot_bytes;
            const long long q = (long long)(j - 1) * g.nx + (cl.i - 1);
            if (so.f16) {
                sh = reinterpret_cast<__half *>(b) + q;
                se = reinterpret_cast<float *>(b + so.ex_off) + (long long)(j - 1) * so.segs + (cl.i - 1) / kSegCells;
                se_comp = (long long)g.ny * so.segs;
            } else {
                sn = reinterpret_cast<float *>(b) + q;
            }
        }
        pair = cl.v1;
        v0 = cl.v0;
        spair = cl.v1 && so.pairs;
    }
    __device__ __forceinline__ void put(long long off, float n0, float n1) const { gput2(st + off, n0, n1, pair, v0); }
    // every lane of the warp calls this for its column pair of the row
    __device__ __forceinline__ void snap(long long n, int comp, float n0, float n1) const {
        if (comp < 0) return;
        if (sn) {
            float *p = sn + comp * n;
            if (spair) *reinterpret_cast<float2 *>(p) = make_float2(n0, n1);
            else {
                if (v0) p[0] = n0;
                if (pair) p[1] = n1;
            }
        } else if (sh) {
            float q, inv;
            seg_scales(seg_absmax_warp(n0, n1, v0, pair), q, inv);
            __half *p = sh + comp * n;
            if (spair) *reinterpret_cast<__half2 *>(p) = __floats2half2_rn(n0 * q, n1 * q);
            else {
                if (v0) p[0] = __float2half_rn(n0 * q);
                if (pair) p[1] = __float2half_rn(n1 * q);
            }
            if (threadIdx.x == 0) se[comp * se_comp] = inv;
        }
    }
};

// release a stage once every lane of the warp has read its part of it
__device__ __forceinline__ void release_stage(uint64_t *empty) {
    __syncwarp();
    if (threadIdx.x == 0) mbar_arrive(empty);
}

// Explosive sources of step nt on row j, as src/psource.c:47-55 applies
// them after the stress update and before the free surface
// (src/IFOS2D.c:1758-1764): the lane holding a source cell adds half the
// source term to its sxx and syy, sources in list order (psource_apply).
__device__ __forceinline__ void psource_row(const KGrid &g, const KSrc &src, int slot, int nt, int j, const Cols &cl,
                                            float (&sxx)[2], float (&syy)[2]) {
    if (!psource_fires(src, slot)) return;
    const int n = src.nsrc[slot];
    const float *pos = src.pos + (long long)slot * 8 * src.max_src;
    for (int l = 0; l < n; l++) {
        if ((int)pos[src.max_src + l] != j) continue;
        const int e = (int)pos[l] - cl.i;
        if ((e != 0 && e != 1) || !cl.valid(e)) continue;
        const float amp = psource_amp(src, slot, l, nt, g.dh);
        if (e == 0) {
            sxx[0] = (float)((double)sxx[0] + 0.5 * (double)amp);
            syy[0] = (float)((double)syy[0] + 0.5 * (double)amp);
        } else {
            sxx[1] = (float)((double)sxx[1] + 0.5 * (double)amp);
            syy[1] = (float)((double)syy[1] + 0.5 * (double)amp);
        }
    }
}

// The free surface of row 1 on a stress op's results (surface_cell: the
// elastic src/surface_elastic_PML.c:53-104 and, with L memory variables, the
// viscoelastic src/surface_PML.c:60-157), from the staged velocities (wx:
// the vx window of row 1; vy2: the zero-started y difference of vy, formed
// before the stage was released): the derivatives are zero-started sums
// scaled by 1/DH, vxx carries its own x CPML (psi_vxxs).  p and q are the
// p and q memory variables (LL each).
template <int FDOH, int HE, int LL>
__device__ __forceinline__ void surface_row(const KGrid &g, const KState<float> &S, const KModel<float> &M,
                                            const Hc<FDOH> &hc, const XWin<HE> &wx, float2 vy2, const Cols &cl,
                                            int slot, int model, float (&sxx)[2], float (&syy)[2], float (*p)[2],
                                            float (*q)[2]) {
    const float DT = g.dt, DH = g.dh;
    const float dh24 = (float)(1.0 / (double)DH), dthalbe = (float)((double)DT / 2.0);
    const float *srf = M.srf + (long long)model * M.srf_stride;
#pragma unroll
    for (int e = 0; e < 2; e++) {
        if (!cl.valid(e)) continue;
        const int i = cl.i + e;
        syy[e] = 0.0f;
#pragma unroll
        for (int l = 0; l < LL; l++) q[l][e] = 0.0f;
        float vxx = xbwd<FDOH, HE, true>(hc, wx, e) * dh24;
        const float vyy = pick(vy2, e) * dh24;
        const int hx = strip_x(g, i);  // the surface has its x CPML also where the stress update has none (10/12)
        if (hx) vxx = pml_x(g, M, S.psix[X_VXXS] + slot * S.psix_slot, 1, hx, K_X, A_X, B_X, vxx);
        const float fjm = srf[i - 1], gg = srf[g.nx + i - 1];
        if (LL == 0) {
            sxx[e] += -DT * ((gg * gg) / (gg + fjm) * vxx + gg * vyy);
            continue;
        }
        const float djm = srf[2 * g.nx + i - 1], ee = srf[3 * g.nx + i - 1];
        float sump = 0;
#pragma unroll
        for (int l = 0; l < LL; l++) sump += p[l][e];
        sxx[e] += -(DT * (gg - fjm) * (gg - fjm) * vxx / gg) - (DT * (gg - fjm) * vyy) - (dthalbe * sump);
        sump = 0;
#pragma unroll
        for (int l = 0; l < LL; l++) {
            const float bjm = g.bjm_srf[l + 1];
            p[l][e] = (float)((double)p[l][e] + (double)bjm * (((double)(djm - ee) * ((double)(fjm / gg) - 1.0) *
                                                                 (double)vxx) - (double)((djm - ee) * vyy)));
            sump += p[l][e];
        }
        sxx[e] += (dthalbe * sump);
    }
}

// By-value forms of the two for out-of-line calls from the viscoelastic
// stress op: its rarely taken source and surface rows then do not add to the
// register budget of its main path (the elastic op has room and inlines them).
template <int LL>
struct RowVals {
    float sxx[2], syy[2], p[LL > 0 ? LL : 1][2], q[LL > 0 ? LL : 1][2];
};
static __device__ __noinline__ float4 psource_row_v(const KGrid &g, const KSrc &src, int slot, int nt, int j, Cols cl,
                                             float4 v) {
    float sxx[2] = {v.x, v.y}, syy[2] = {v.z, v.w};
    psource_row(g, src, slot, nt, j, cl, sxx, syy);
    return make_float4(sxx[0], sxx[1], syy[0], syy[1]);
}
// Receiver indices of the thread's column pair in row j (-1: none) when
// the velocity op samples or injects the receivers in place (rec_mode), read
// from the slot's cell map at the start of the row so that the two loads are
// in flight while the row is computed.
__device__ __forceinline__ int2 rec_lookup(const KGrid &g, const KRec &rec, int mode, int rec_j0, int rec_j1,
                                           int slot, int j, const Cols &cl) {
    if (!mode || j < rec_j0 || j > rec_j1 || j > g.ny) return make_int2(-1, -1);
    return rec_pair(rec, g.nx, g.ny, slot, j, cl.i, cl.v0, cl.v1);
}

// The receivers of the thread's cells in row j (rl: their indices) on the
// new vx, vy before they are stored: mode 1 copies them into the seismograms
// of step nt, as src/seismo_ssg.c:26-140 samples vx, vy after the step
// (SEISMO 1); mode 2 adds the adjoint sources of step nt, as
// src/update_v_PML.c:567-578 does after the velocity update (ADJOINT_TYPE 1:
// both components, 2: vy, 3: vx).
__device__ __forceinline__ void rec_apply(const KGrid &g, const KRec &rec, int mode, int slot, int nt, int2 rl,
                                          float (&vx)[2], float (&vy)[2]) {
    const long long cs = (long long)rec.max_rec * g.nt_total;
#pragma unroll
    for (int e = 0; e < 2; e++) {
        const int l = e ? rl.y : rl.x;
        if (l < 0) continue;
        const long long o = (long long)l * g.nt_total + nt - 1;
        if (mode == 2) {
            const float *adj = rec.adj + (long long)slot * 3 * cs + o;
            const int at = g.adjoint_type;
            if (at == 1 || at == 3) vx[e] += adj[0];
            if (at == 1 || at == 2) vy[e] += adj[cs];
        } else {
            float *sec = rec.sec + (long long)slot * 6 * cs + o;
            sec[0] = vx[e];
            sec[cs] = vy[e];
        }
    }
}

template <int FDOH, int HE, int LL>
__device__ __noinline__ RowVals<LL> surface_row_v(const KGrid &g, const KState<float> &S, const KModel<float> &M,
                                                  Hc<FDOH> hc, XWin<HE> wx, float2 vy2, Cols cl, int slot, int model,
                                                  RowVals<LL> v) {
    surface_row<FDOH, HE, LL>(g, S, M, hc, wx, vy2, cl, slot, model, v.sxx, v.syy, v.p, v.q);
    return v;
}

// Interior tiles take rows<false>; tiles with a strip cell rows<true>.
// The path is chosen per warp (all lanes take the same one, so that the
// warp-wide operations of the snapshot store and the stage release meet):
// lanes outside the strips of a strip tile see hx = 0 and no y strip.
#define IFOS_TILE_COMPUTE(NOPML_)                                                                     \
    __device__ __forceinline__ void compute(const TileInfo &ti, const float *h, const float *pl,      \
                                            uint64_t *empty) const {                                  \
        const Cols cl(g, ti, P::XH, !(NOPML_));                                                       \
        if ((NOPML_) || (!__any_sync(0xffffffffu, cl.hx0 != 0 || cl.hx1 != 0) && !ti.ystrip))         \
            rows<false>(ti, cl, h, pl, empty);                                                        \
        else                                                                                          \
            rows<true>(ti, cl, h, pl, empty);                                                         \
    }

// the common members of an op
// src, nt, fsurf, fps: the stress ops apply the explosive sources of step nt
// (fps; rows src_j0..src_j1 hold every slot's sources) and the free surface
// of row 1 (fsurf) themselves
// rec_mode (P-SV velocity ops): 1 the forward samples vx, vy at the
// receivers into the seismograms (SEISMO 1) and probes the centre cell for
// NaN, 2 the adjoint adds the residual sources at the receivers; rows
// rec_j0..rec_j1 hold every slot's receivers.
#define IFOS_OP_MEMBERS \
    KGrid g;            \
    KState<float> S;    \
    KModel<float> M;    \
    KTma tm;            \
    KSnapOut so;        \
    KSrc src;           \
    int nt;             \
    int fsurf;          \
    int fps;            \
    int src_j0, src_j1; \
    KRec rec;           \
    int rec_mode;       \
    int rec_j0, rec_j1; \
    int *bad;

// ---------------------------------------------------------------------------
// stress, P-SV viscoelastic with LL SLS (src/update_s_visc_PML.c; the
// reference 10/12 default :615-660 has no CPML and zero-started sums: QUIRK)
// halo: vx vy; plain: sxx syy sxy, r[LL] p[LL] q[LL], fipjp f g mu pi muipjp;
// writes sxx syy sxy r p q.  Non-uniform tau planes are read from HBM.
template <int FDOH, int TY, int LL, int NST, bool QUIRK>
struct OpSVisc {
    static constexpr int NH_ = 2, NP_ = 3 + 3 * LL + 6, NOUT = 3 + 3 * LL;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
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
    IFOS_TILE_COMPUTE(QUIRK)
    template <bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_vx = h, *t_vy = h + P::BOXS;
        float2 vys = make_float2(0.0f, 0.0f);  // the free surface's vy difference (row 1)
        const Hc<FDOH> hc(g);
        // everything this warp needs from the stage, then release it
        XWin<P::HE> wx[RT], wy[RT];
        float2 dxy[RT], dyy[RT], in[RT][NP_];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wx[r].load(t_vx + (jj + P::H) * P::BW, cl.c0);
            wy[r].load(t_vy + (jj + P::H) * P::BW, cl.c0);
            dxy[r] = yfwd2<false, false, P, FDOH, QUIRK>(hc, t_vx, jj, cl.c0);
            dyy[r] = ybwd2<false, false, P, FDOH, QUIRK>(hc, t_vy, jj, cl.c0);
            if (fsurf && ti.j0 + jj == 1) vys = ybwd2<false, false, P, FDOH, true>(hc, t_vy, jj, cl.c0);
#pragma unroll
            for (int q = 0; q < NP_; q++) in[r][q] = lds2(pl + q * P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const long long mo = (long long)ti.model * M.model_stride;
        const float *ts_p = M.m[M_TAUS] ? M.m[M_TAUS] + mo : nullptr;
        const float *tp_p = M.m[M_TAUP] ? M.m[M_TAUP] + mo : nullptr;
        const float *tsij_p = M.m[M_TAUSIPJP] ? M.m[M_TAUSIPJP] + mo : nullptr;
        const float DT = g.dt, DH = g.dh;
        const float dhi = (float)(1.0 / (double)DH), dthalbe = (float)((double)DT / 2.0);
        constexpr int CO = 3 + 3 * LL;  // first coefficient plane
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[NOUT][2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const float2 *v = in[r];
                float vxx = xbwd<FDOH, P::HE, QUIRK>(hc, wx[r], e) * dhi;
                float vyx = xfwd<FDOH, P::HE, QUIRK>(hc, wy[r], e) * dhi;
                float vxy = pick(dxy[r], e) * dhi, vyy = pick(dyy[r], e) * dhi;
                const bool ok = cl.valid(e);
                if (PML && ok) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) {
                        vxx = pml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, vxx);
                        vyx = pml_x(g, M, S.psix[X_VYX] + slot * S.psix_slot, j, hx, K_XH, A_XH, B_XH, vyx);
                    }
                    const int hy = strip_y(g, j);
                    if (hy) {
                        vyy = pml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, vyy);
                        vxy = pml_y(g, M, S.psiy[Y_VXY] + slot * S.psiy_slot, ii, hy, K_YH, A_YH, B_YH, vxy);
                    }
                }
                float sumr = 0, sump = 0, sumq = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) {
                    sumr += pick(v[3 + l], e);
                    sump += pick(v[3 + LL + l], e);
                    sumq += pick(v[3 + 2 * LL + l], e);
                }
                const float fipjp = pick(v[CO], e), f = pick(v[CO + 1], e), gg = pick(v[CO + 2], e);
                const float mu = pick(v[CO + 3], e), pi = pick(v[CO + 4], e), muij = pick(v[CO + 5], e);
                float ts = g.taus0, tp = g.taup0, tsij = g.tausipjp0;
                if (ok && (ts_p || tp_p || tsij_p)) {
                    const int c = (j - 1 + HY) * g.pitch + (cl.i + e - 1 + HX);
                    if (ts_p) ts = ts_p[c];
                    if (tp_p) tp = tp_p[c];
                    if (tsij_p) tsij = tsij_p[c];
                }
                const float s_xy = pick(v[2], e) + ((fipjp * (vxy + vyx)) + (dthalbe * sumr));
                const float s_xx = (float)((D)pick(v[0], e) + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vyy) +
                                                              (D)(dthalbe * sump)));
                const float s_yy = (float)((D)pick(v[1], e) + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vxx) +
                                                              (D)(dthalbe * sumq)));
                sumr = sump = sumq = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) {
                    const float eta = g.eta[l + 1];
                    // dip, d, e of src/prepare_update_s.c:57-59, formed in the same order
                    const float dip = muij * eta * tsij, dd = mu * eta * ts, ee = pi * eta * tp;
                    const float rr = g.bip[l + 1] * (pick(v[3 + l], e) * g.cip[l + 1] - (dip * (vxy + vyx)));
                    const float pp = (float)((D)g.bjm[l + 1] *
                                             ((D)(pick(v[3 + LL + l], e) * g.cjm[l + 1] - (ee * (vxx + vyy))) +
                                              ((D)2 * (D)dd * (D)vyy)));
                    const float qq = (float)((D)g.bjm[l + 1] *
                                             ((D)(pick(v[3 + 2 * LL + l], e) * g.cjm[l + 1] - (ee * (vxx + vyy))) +
                                              ((D)2 * (D)dd * (D)vxx)));
                    o[3 + l][e] = rr;
                    o[3 + LL + l][e] = pp;
                    o[3 + 2 * LL + l][e] = qq;
                    sumr += rr;
                    sump += pp;
                    sumq += qq;
                }
                o[0][e] = s_xx + (dthalbe * sump);
                o[1][e] = s_yy + (dthalbe * sumq);
                o[2][e] = s_xy + (dthalbe * sumr);
            }
            if (fps && j >= src_j0 && j <= src_j1) {
                const float4 r4 = psource_row_v(g, src, slot, nt, j, cl, make_float4(o[0][0], o[0][1], o[1][0], o[1][1]));
                o[0][0] = r4.x, o[0][1] = r4.y, o[1][0] = r4.z, o[1][1] = r4.w;
            }
            if (fsurf && j == 1) {
                RowVals<LL> rv;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    rv.sxx[e] = o[0][e];
                    rv.syy[e] = o[1][e];
#pragma unroll
                    for (int l = 0; l < LL; l++) {
                        rv.p[l][e] = o[3 + LL + l][e];
                        rv.q[l][e] = o[3 + 2 * LL + l][e];
                    }
                }
                rv = surface_row_v<FDOH, P::HE, LL>(g, S, M, hc, wx[r], vys, cl, slot, ti.model, rv);
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    o[0][e] = rv.sxx[e];
                    o[1][e] = rv.syy[e];
#pragma unroll
                    for (int l = 0; l < LL; l++) {
                        o[3 + LL + l][e] = rv.p[l][e];
                        o[3 + 2 * LL + l][e] = rv.q[l][e];
                    }
                }
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_SXX], o[0][0], o[0][1]);
            out.put(S.off[P_SYY], o[1][0], o[1][1]);
            out.put(S.off[P_SXY], o[2][0], o[2][1]);
#pragma unroll
            for (int l = 0; l < LL; l++) {
                out.put(S.mem_off[0] + l * g.plane, o[3 + l][0], o[3 + l][1]);
                out.put(S.mem_off[1] + l * g.plane, o[3 + LL + l][0], o[3 + LL + l][1]);
                out.put(S.mem_off[2] + l * g.plane, o[3 + 2 * LL + l][0], o[3 + 2 * LL + l][1]);
            }
            out.snap(so.n, tm.snap_comp[P_SXX], o[0][0], o[0][1]);
            out.snap(so.n, tm.snap_comp[P_SYY], o[1][0], o[1][1]);
            out.snap(so.n, tm.snap_comp[P_SXY], o[2][0], o[2][1]);
        }
    }
};

// stress, P-SV elastic (src/update_s_elastic_PML.c:151-241; 10/12: :442-535)
// halo: vx vy; plain: sxx syy sxy uipjp f g (reference 10/12 branch: uipjp vs vp);
// writes sxx syy sxy
template <int FDOH, int TY, int NST, bool QUIRK>
struct OpSEl {
    static constexpr int NH_ = 2, NP_ = 6;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST, sblocks(FDOH)>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SXX], false};
        pz[1] = {zb + tm.pid[P_SYY], false};
        pz[2] = {zb + tm.pid[P_SXY], false};
        pz[3] = {mb + tm.mid[M_UIPJP], true};
        pz[4] = {mb + tm.mid[QUIRK ? M_VS : M_F], true};
        pz[5] = {mb + tm.mid[QUIRK ? M_VP : M_G], true};
    }
    IFOS_TILE_COMPUTE(QUIRK)
    template <bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_vx = h, *t_vy = h + P::BOXS;
        float2 vys = make_float2(0.0f, 0.0f);  // the free surface's vy difference (row 1)
        const Hc<FDOH> hc(g);
        XWin<P::HE> wx[RT], wy[RT];
        float2 dxy[RT], dyy[RT], in[RT][NP_];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wx[r].load(t_vx + (jj + P::H) * P::BW, cl.c0);
            wy[r].load(t_vy + (jj + P::H) * P::BW, cl.c0);
            dxy[r] = yfwd2<false, false, P, FDOH>(hc, t_vx, jj, cl.c0);
            dyy[r] = ybwd2<false, false, P, FDOH>(hc, t_vy, jj, cl.c0);
            if (fsurf && ti.j0 + jj == 1) vys = ybwd2<false, false, P, FDOH, true>(hc, t_vy, jj, cl.c0);
#pragma unroll
            for (int q = 0; q < NP_; q++) in[r][q] = lds2(pl + q * P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const float DT = g.dt, DH = g.dh;
        const float dhi = DT / DH;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[3][2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const float2 *v = in[r];
                float vxx = xbwd<FDOH, P::HE>(hc, wx[r], e) * dhi;
                float vyx = xfwd<FDOH, P::HE>(hc, wy[r], e) * dhi;
                float vxy = pick(dxy[r], e) * dhi, vyy = pick(dyy[r], e) * dhi;
                const float sxx0 = pick(v[0], e), syy0 = pick(v[1], e), sxy0 = pick(v[2], e);
                if (QUIRK) {
                    const float fipjp = pick(v[3], e) * DT, f = pick(v[4], e) * DT, gg = pick(v[5], e) * DT;
                    o[2][e] = sxy0 + (fipjp * (vxy + vyx));
                    o[0][e] = (float)((D)sxx0 + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vyy)));
                    o[1][e] = (float)((D)syy0 + ((D)(gg * (vxx + vyy)) - ((D)2 * (D)f * (D)vxx)));
                    continue;
                }
                if (PML && cl.valid(e)) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) {
                        vxx = pml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, vxx);
                        vyx = pml_x(g, M, S.psix[X_VYX] + slot * S.psix_slot, j, hx, K_XH, A_XH, B_XH, vyx);
                    }
                    const int hy = strip_y(g, j);
                    if (hy) {
                        vyy = pml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, vyy);
                        vxy = pml_y(g, M, S.psiy[Y_VXY] + slot * S.psiy_slot, ii, hy, K_YH, A_YH, B_YH, vxy);
                    }
                }
                const float fipjp = pick(v[3], e), f = pick(v[4], e), gg = pick(v[5], e);
                o[2][e] = sxy0 + fipjp * (vyx + vxy);
                o[0][e] = (float)((D)sxx0 + ((D)(gg * (vxx + vyy)) + ((D)2 * (D)f * (D)vxx)));
                o[1][e] = (float)((D)syy0 + ((D)(gg * (vxx + vyy)) + ((D)2 * (D)f * (D)vyy)));
            }
            if (fps && j >= src_j0 && j <= src_j1) psource_row(g, src, slot, nt, j, cl, o[0], o[1]);
            if (fsurf && j == 1)
                surface_row<FDOH, P::HE, 0>(g, S, M, hc, wx[r], vys, cl, slot, ti.model, o[0], o[1], nullptr, nullptr);
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_SXX], o[0][0], o[0][1]);
            out.put(S.off[P_SYY], o[1][0], o[1][1]);
            out.put(S.off[P_SXY], o[2][0], o[2][1]);
            out.snap(so.n, tm.snap_comp[P_SXX], o[0][0], o[0][1]);
            out.snap(so.n, tm.snap_comp[P_SYY], o[1][0], o[1][1]);
            out.snap(so.n, tm.snap_comp[P_SXY], o[2][0], o[2][1]);
        }
    }
};

// ---------------------------------------------------------------------------
// velocity, P-SV (src/update_v_PML.c:161-252; 10/12 reference branches
// :466-528 when QUIRK) and acoustic (src/update_v_acoustic_PML.c:72-148,
// default :396-409 when QUIRK; AC).  halo: sxx syy sxy (acoustic: sp);
// plain: vx vy rip rjp [+ vxp1 vyp1 in the adjoint].  SW: 0 forward,
// 1 adjoint; P1: this forward step forms vxp1/vyp1 for a snapshot (written to
// the snapshot when the launch stores one, else to the state).
template <int FDOH, int TY, int NST, bool QUIRK, int SW, bool P1, bool AC>
struct OpVPsv {
    static constexpr int NH_ = AC ? 1 : 3;
    static constexpr int NP_ = (SW == 1 && !QUIRK) ? 6 : 4;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST, vblocks(FDOH)>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        if (AC) {
            hz[0] = zb + tm.pid[P_SP];
        } else {
            hz[0] = zb + tm.pid[P_SXX];
            hz[(1 < NH_) ? 1 : 0] = zb + tm.pid[P_SYY];
            hz[(2 < NH_) ? 2 : 0] = zb + tm.pid[P_SXY];
        }
        pz[0] = {zb + tm.pid[P_VX], false};
        pz[1] = {zb + tm.pid[P_VY], false};
        pz[2] = {mb + tm.mid[M_RIP], true};
        pz[3] = {mb + tm.mid[M_RJP], true};
        if (NP_ > 4) {
            pz[4 % NP_] = {zb + tm.pid[P_VXP1], false};
            pz[5 % NP_] = {zb + tm.pid[P_VYP1], false};
        }
    }
    __device__ __forceinline__ void compute(const TileInfo &ti, const float *h, const float *pl,
                                            uint64_t *empty) const {
        const Cols cl(g, ti, P::XH, !QUIRK);
        const bool mir = g.free_surf && ti.j0 == 1;
        if (QUIRK || (cl.hx0 == 0 && cl.hx1 == 0 && !ti.ystrip)) {
            if (mir) rows<true, false>(ti, cl, h, pl, empty);
            else rows<false, false>(ti, cl, h, pl, empty);
        } else {
            if (mir) rows<true, true>(ti, cl, h, pl, empty);
            else rows<false, true>(ti, cl, h, pl, empty);
        }
    }
    template <bool MIR, bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        // P-SV: sxx, syy, sxy boxes; acoustic: the sp box serves as all three
        const float *t_sxx = h, *t_syy = AC ? h : h + P::BOXS, *t_sxy = AC ? h : h + 2 * P::BOXS;
        const Hc<FDOH> hc(g);
        int2 rl[RT];  // receivers of the thread's cells (rec_mode)
#pragma unroll
        for (int r = 0; r < RT; r++)
            rl[r] = rec_lookup(g, rec, rec_mode, rec_j0, rec_j1, ti.slot, ti.j0 + threadIdx.y * RT + r, cl);
        XWin<P::HE> wxx[RT], wxy[RT];
        float2 dyy[RT], dxy[RT], in[RT][NP_];
        float2 qa[RT][QUIRK && !AC ? FDOH : 1];  // reference 10/12 P-SV form: the sxy y-taps one by one
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wxx[r].load(t_sxx + (jj + P::H) * P::BW, cl.c0);
            if (!AC) wxy[r].load(t_sxy + (jj + P::H) * P::BW, cl.c0);
            dyy[r] = yfwd2<MIR, false, P, FDOH, QUIRK && AC>(hc, t_syy, jj, cl.c0);
            if (!AC && !QUIRK) dxy[r] = ybwd2<MIR, true, P, FDOH>(hc, t_sxy, jj, cl.c0);
            if (!AC && QUIRK) {
#pragma unroll
                for (int m = 1; m <= (QUIRK && !AC ? FDOH : 1); m++) {
                    const float2 a = ldy2<MIR, true, P>(t_sxy, jj, cl.c0, m - 1);
                    const float2 b = ldy2<MIR, true, P>(t_sxy, jj, cl.c0, -m);
                    qa[r][m - 1] = make_float2(a.x - b.x, a.y - b.y);
                }
            }
#pragma unroll
            for (int q = 0; q < NP_; q++) in[r][q] = lds2(pl + q * P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const float DT = g.dt, DH = g.dh;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[4][2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const float2 *v = in[r];
                const float vxo = pick(v[0], e), vyo = pick(v[1], e), rip = pick(v[2], e), rjp = pick(v[3], e);
                float a_x, a_y, b_x = 0.0f, b_y = 0.0f;  // P-SV: sxx_x, syy_y, sxy_x, sxy_y; acoustic: sp_x, sp_y
                if (QUIRK) {
                    const float dtdh = DT * DT / DH;
                    if (AC) {
                        a_x = xfwd<FDOH, P::HE, true>(hc, wxx[r], e);
                        a_y = pick(dyy[r], e);
                    } else {
                        // one written-out sum per component (src/update_v_PML.c:469-490)
                        a_x = xfwd<FDOH, P::HE>(hc, wxx[r], e);
#pragma unroll
                        for (int m = 1; m <= (QUIRK && !AC ? FDOH : 1); m++) a_x += hc.w[m] * pick(qa[r][m - 1], e);
                        a_y = pick(dyy[r], e);
#pragma unroll
                        for (int m = 1; m <= FDOH; m++)
                            a_y += hc.w[m] * (wxy[r].v[P::HE + e + m - 1] - wxy[r].v[P::HE + e - m]);
                    }
                    o[0][e] = vxo + a_x * dtdh * rip;
                    o[1][e] = vyo + a_y * dtdh * rjp;
                    continue;
                }
                a_x = xfwd<FDOH, P::HE>(hc, wxx[r], e);
                a_y = pick(dyy[r], e);
                if (!AC) {
                    b_x = xbwd<FDOH, P::HE>(hc, wxy[r], e);
                    b_y = pick(dxy[r], e);
                }
                if (PML && cl.valid(e)) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) {
                        a_x = pml_x(g, M, S.psix[X_SXX] + slot * S.psix_slot, j, hx, K_XH, A_XH, B_XH, a_x);
                        if (!AC) b_x = pml_x(g, M, S.psix[X_SXY] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, b_x);
                    }
                    const int hy = strip_y(g, j);
                    if (hy) {
                        a_y = pml_y(g, M, S.psiy[Y_SYY] + slot * S.psiy_slot, ii, hy, K_YH, A_YH, B_YH, a_y);
                        if (!AC) b_y = pml_y(g, M, S.psiy[Y_SXY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, b_y);
                    }
                }
                // P-SV: x force sxx_x + sxy_y, y force sxy_x + syy_y; acoustic: sp_x, sp_y
                const float fx = AC ? (a_x) : (a_x + b_y), fy = AC ? (a_y) : (b_x + a_y);
                if (SW == 0) {
                    if (P1) {
                        o[2][e] = div_dh(g, rip * fx);
                        o[3][e] = div_dh(g, rjp * fy);
                    }
                } else {
                    o[2][e] = pick(v[4 % NP_], e) + vxo * DT;
                    o[3][e] = pick(v[5 % NP_], e) + vyo * DT;
                }
                o[0][e] = vxo + div_dh(g, DT * rip * fx);
                o[1][e] = vyo + div_dh(g, DT * rjp * fy);
            }
            if (rl[r].x >= 0 || rl[r].y >= 0) rec_apply(g, rec, rec_mode, slot, nt, rl[r], o[0], o[1]);
            if (rec_mode == 1 && j == g.ny / 2) {  // the instability probe of the driver (src/IFOS2D.c:1660-1672)
                const int e = g.nx / 2 - cl.i;
                if ((e == 0 || e == 1) && cl.valid(e) && isnan(e ? o[1][1] : o[1][0])) atomicExch(bad, 1);
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_VX], o[0][0], o[0][1]);
            out.put(S.off[P_VY], o[1][0], o[1][1]);
            if (!QUIRK && (SW == 1 || (P1 && !out.sn && !out.sh))) {
                out.put(S.off[P_VXP1], o[2][0], o[2][1]);
                out.put(S.off[P_VYP1], o[3][0], o[3][1]);
            }
            if (!QUIRK && SW == 0 && P1) {
                out.snap(so.n, tm.snap_comp[P_VXP1], o[2][0], o[2][1]);
                out.snap(so.n, tm.snap_comp[P_VYP1], o[3][0], o[3][1]);
            }
        }
    }
};

// velocity, SH (src/update_v_PML_SH.c:61-297, CPML on every order);
// halo: sxz syz; plain: vz rjp; writes vz and vzp1 = previous vz
template <int FDOH, int TY, int NST>
struct OpVSh {
    static constexpr int NH_ = 2, NP_ = 2;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST, vblocks(FDOH)>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        hz[0] = zb + tm.pid[P_SXZ];
        hz[1] = zb + tm.pid[P_SYZ];
        pz[0] = {zb + tm.pid[P_VZ], false};
        pz[1] = {mb + tm.mid[M_RJP], true};
    }
    __device__ __forceinline__ void compute(const TileInfo &ti, const float *h, const float *pl,
                                            uint64_t *empty) const {
        const Cols cl(g, ti, P::XH, true);
        const bool mir = g.free_surf && ti.j0 == 1;
        if (cl.hx0 == 0 && cl.hx1 == 0 && !ti.ystrip) {
            if (mir) rows<true, false>(ti, cl, h, pl, empty);
            else rows<false, false>(ti, cl, h, pl, empty);
        } else {
            if (mir) rows<true, true>(ti, cl, h, pl, empty);
            else rows<false, true>(ti, cl, h, pl, empty);
        }
    }
    template <bool MIR, bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_sxz = h, *t_syz = h + P::BOXS;
        const Hc<FDOH> hc(g);
        XWin<P::HE> wxz[RT];
        float2 dyz[RT], vz2[RT], rjp2[RT];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wxz[r].load(t_sxz + (jj + P::H) * P::BW, cl.c0);
            dyz[r] = yfwd2<MIR, false, P, FDOH>(hc, t_syz, jj, cl.c0);
            vz2[r] = lds2(pl + jj * kTileX + 2 * cl.lane);
            rjp2[r] = lds2(pl + P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const float DT = g.dt;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                float sxz_x = xbwd<FDOH, P::HE>(hc, wxz[r], e), syz_y = pick(dyz[r], e);
                if (PML && cl.valid(e)) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) sxz_x = pml_x(g, M, S.psix[X_SXZ] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, sxz_x);
                    const int hy = strip_y(g, j);
                    if (hy) syz_y = pml_y(g, M, S.psiy[Y_SYZ] + slot * S.psiy_slot, ii, hy, K_YH, A_YH, B_YH, syz_y);
                }
                o[e] = pick(vz2[r], e) + div_dh(g, pick(rjp2[r], e) * DT * (sxz_x + syz_y));
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_VZP1], vz2[r].x, vz2[r].y);
            out.put(S.off[P_VZ], o[0], o[1]);
            out.snap(so.n, tm.snap_comp[P_VZP1], vz2[r].x, vz2[r].y);
        }
    }
};

// stress, SH elastic / viscoelastic (src/update_s_elastic_PML_SH.c,
// src/update_s_visc_PML_SH.c); halo: vz; plain: sxz syz [t[LL] o[LL]] and the
// coefficients (elastic: uipjp f; visco: fipjp f mu muipjp); writes sxz syz [t o]
template <int FDOH, int TY, int LL, int NST>
struct OpSSh {
    static constexpr int NH_ = 1, NP_ = LL ? 2 + 2 * LL + 4 : 4, NOUT = 2 + 2 * LL;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VZ];
        pz[0] = {zb + tm.pid[P_SXZ], false};
        pz[1] = {zb + tm.pid[P_SYZ], false};
        if (LL == 0) {
            pz[2] = {mb + tm.mid[M_UIPJP], true};
            pz[3] = {mb + tm.mid[M_F], true};
        } else {
#pragma unroll
            for (int l = 0; l < LL; l++) {
                pz[(2 + l) % NP_] = {zb + tm.mem_pid[3] + l, false};       // t
                pz[(2 + LL + l) % NP_] = {zb + tm.mem_pid[4] + l, false};  // o
            }
            pz[(2 + 2 * LL + 0) % NP_] = {mb + tm.mid[M_FIPJPV], true};
            pz[(2 + 2 * LL + 1) % NP_] = {mb + tm.mid[M_FV], true};
            pz[(2 + 2 * LL + 2) % NP_] = {mb + tm.mid[M_MUR], true};
            pz[(2 + 2 * LL + 3) % NP_] = {mb + tm.mid[M_MUIPJPR], true};
        }
    }
    IFOS_TILE_COMPUTE(false)
    template <bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_vz = h;
        const Hc<FDOH> hc(g);
        XWin<P::HE> wz[RT];
        float2 dzy[RT], in[RT][NP_];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wz[r].load(t_vz + (jj + P::H) * P::BW, cl.c0);
            dzy[r] = ybwd2<false, false, P, FDOH>(hc, t_vz, jj, cl.c0);
#pragma unroll
            for (int q = 0; q < NP_; q++) in[r][q] = lds2(pl + q * P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const long long mo = (long long)ti.model * M.model_stride;
        const float *ts_p = M.m[M_TAUS] ? M.m[M_TAUS] + mo : nullptr;
        const float *tsij_p = M.m[M_TAUSIPJP] ? M.m[M_TAUSIPJP] + mo : nullptr;
        const float DT = g.dt, DH = g.dh;
        const float dhi = LL ? (float)(1.0 / (double)DH) : DT / DH, dthalbe = (float)((double)DT / 2.0);
        constexpr int CO = 2 + 2 * LL;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[NOUT][2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const float2 *v = in[r];
                float vzx = xfwd<FDOH, P::HE>(hc, wz[r], e) * dhi, vzy = pick(dzy[r], e) * dhi;
                const bool ok = cl.valid(e);
                if (PML && ok) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) vzx = pml_x(g, M, S.psix[X_VZX] + slot * S.psix_slot, j, hx, K_XH, A_XH, B_XH, vzx);
                    const int hy = strip_y(g, j);
                    if (hy) vzy = pml_y(g, M, S.psiy[Y_VZY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, vzy);
                }
                if (LL == 0) {
                    o[0][e] = pick(v[0], e) + (pick(v[2], e) * vzx);
                    o[1][e] = pick(v[1], e) + (pick(v[3], e) * vzy);
                    continue;
                }
                float sumo = 0, sumt = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) {
                    sumo += pick(v[(2 + LL + l) % NP_], e);
                    sumt += pick(v[(2 + l) % NP_], e);
                }
                const float fipjp = pick(v[CO % NP_], e), f = pick(v[(CO + 1) % NP_], e);
                const float mu = pick(v[(CO + 2) % NP_], e), muij = pick(v[(CO + 3) % NP_], e);
                float ts = g.taus0, tsij = g.tausipjp0;
                if (ok && (ts_p || tsij_p)) {
                    const int c = (j - 1 + HY) * g.pitch + (cl.i + e - 1 + HX);
                    if (ts_p) ts = ts_p[c];
                    if (tsij_p) tsij = tsij_p[c];
                }
                const float s_xz = pick(v[0], e) + ((fipjp * vzx) + (dthalbe * sumo));
                const float s_yz = pick(v[1], e) + ((f * vzy) + (dthalbe * sumt));
                sumo = sumt = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) {
                    const float eta = g.eta[l + 1];
                    const float dip = muij * eta * tsij, dd = mu * eta * ts;
                    const float oo = g.bip[l + 1] * (pick(v[(2 + LL + l) % NP_], e) * g.cip[l + 1] - (dip * vzx));
                    const float tt = g.bjm[l + 1] * (pick(v[(2 + l) % NP_], e) * g.cjm[l + 1] - (dd * vzy));
                    o[(2 + LL + l) % NOUT][e] = oo;
                    o[(2 + l) % NOUT][e] = tt;
                    sumt += tt;
                    sumo += oo;
                }
                o[0][e] = s_xz + (dthalbe * sumo);
                o[1][e] = s_yz + (dthalbe * sumt);
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_SXZ], o[0][0], o[0][1]);
            out.put(S.off[P_SYZ], o[1][0], o[1][1]);
#pragma unroll
            for (int l = 0; l < LL; l++) {
                out.put(S.mem_off[3] + l * g.plane, o[(2 + l) % NOUT][0], o[(2 + l) % NOUT][1]);
                out.put(S.mem_off[4] + l * g.plane, o[(2 + LL + l) % NOUT][0], o[(2 + LL + l) % NOUT][1]);
            }
            out.snap(so.n, tm.snap_comp[P_SXZ], o[0][0], o[0][1]);
            out.snap(so.n, tm.snap_comp[P_SYZ], o[1][0], o[1][1]);
        }
    }
};

// pressure, acoustic (src/update_p_PML.c:55-273; default :275-287 when QUIRK)
// halo: vx vy; plain: sp g (reference 10/12 branch: vp); writes sp
template <int FDOH, int TY, int NST, bool QUIRK>
struct OpPAc {
    static constexpr int NH_ = 2, NP_ = 2;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SP], false};
        pz[1] = {mb + tm.mid[QUIRK ? M_VP : M_GAC], true};
    }
    IFOS_TILE_COMPUTE(QUIRK)
    template <bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_vx = h, *t_vy = h + P::BOXS;
        const Hc<FDOH> hc(g);
        XWin<P::HE> wx[RT];
        float2 dyy[RT], sp2[RT], g2[RT];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wx[r].load(t_vx + (jj + P::H) * P::BW, cl.c0);
            dyy[r] = ybwd2<false, false, P, FDOH, QUIRK>(hc, t_vy, jj, cl.c0);
            sp2[r] = lds2(pl + jj * kTileX + 2 * cl.lane);
            g2[r] = lds2(pl + P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const float DT = g.dt, DH = g.dh;
        const float dhi = DT / DH;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                float vxx = xbwd<FDOH, P::HE, QUIRK>(hc, wx[r], e), vyy = pick(dyy[r], e);
                if (QUIRK) {
                    const float gg = pick(g2[r], e) * DT;
                    o[e] = pick(sp2[r], e) + (gg * (vxx + vyy)) * dhi;
                    continue;
                }
                vxx = vxx * dhi;
                vyy = vyy * dhi;
                if (PML && cl.valid(e)) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) vxx = pml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, vxx);
                    const int hy = strip_y(g, j);
                    if (hy) vyy = pml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, vyy);
                }
                o[e] = pick(sp2[r], e) + pick(g2[r], e) * (vxx + vyy);
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_SP], o[0], o[1]);
            out.snap(so.n, tm.snap_comp[P_SP], o[0], o[1]);
        }
    }
};
// pressure, viscoacoustic with LL relaxation mechanisms
// (src/update_p_visc_PML.c:61-146 at FDORDER 2, with CPML; :148-182 for every
// other order: sums from zero and no CPML, hence Z0 and no strip path)
// halo: vx vy; plain: sp p[LL] g pi; writes sp p[LL].  Non-uniform taup is
// read from HBM.
template <int FDOH, int TY, int LL, int NST>
struct OpPVisc {
    static constexpr bool Z0 = FDOH != 1;
    static constexpr int NH_ = 2, NP_ = 3 + LL;
    using P = Pipe<FDOH, TY, NH_, NP_, 0, NST>;
    IFOS_OP_MEMBERS
    __device__ void planes(const TileInfo &ti, int *hz, PlainSrc *pz) const {
        const int zb = ti.slot * tm.planes_per_slot;
        const int mb = ti.model * tm.model_planes;
        hz[0] = zb + tm.pid[P_VX];
        hz[1] = zb + tm.pid[P_VY];
        pz[0] = {zb + tm.pid[P_SP], false};
#pragma unroll
        for (int l = 0; l < LL; l++) pz[1 + l] = {zb + tm.mem_pid[1] + l, false};
        pz[1 + LL] = {mb + tm.mid[M_GV], true};
        pz[2 + LL] = {mb + tm.mid[M_PIR], true};
    }
    IFOS_TILE_COMPUTE(Z0)
    template <bool PML>
    __device__ __forceinline__ void rows(const TileInfo &ti, const Cols &cl, const float *h, const float *pl,
                                         uint64_t *empty) const {
        constexpr int RT = P::RT;
        const float *t_vx = h, *t_vy = h + P::BOXS;
        const Hc<FDOH> hc(g);
        XWin<P::HE> wx[RT];
        float2 dyy[RT], in[RT][NP_];
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int jj = threadIdx.y * RT + r;
            wx[r].load(t_vx + (jj + P::H) * P::BW, cl.c0);
            dyy[r] = ybwd2<false, false, P, FDOH, Z0>(hc, t_vy, jj, cl.c0);
#pragma unroll
            for (int q = 0; q < NP_; q++) in[r][q] = lds2(pl + q * P::PLS + jj * kTileX + 2 * cl.lane);
        }
        release_stage(empty);
        const int slot = ti.slot;
        const float *tp_p = M.m[M_TAUP] ? M.m[M_TAUP] + (long long)ti.model * M.model_stride : nullptr;
        const float DT = g.dt, DH = g.dh;
        const float dhi = (float)(1.0 / (double)DH), dthalbe = (float)((double)DT / 2.0);
#pragma unroll
        for (int r = 0; r < RT; r++) {
            const int j = ti.j0 + threadIdx.y * RT + r;
            if (j > g.ny) break;
            float o[1 + LL][2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const float2 *v = in[r];
                float vxx = xbwd<FDOH, P::HE, Z0>(hc, wx[r], e) * dhi, vyy = pick(dyy[r], e) * dhi;
                const bool ok = cl.valid(e);
                if (PML && ok) {
                    const int hx = cl.hx(e), ii = cl.i + e;
                    if (hx) vxx = pml_x(g, M, S.psix[X_VXX] + slot * S.psix_slot, j, hx, K_X, A_X, B_X, vxx);
                    const int hy = strip_y(g, j);
                    if (hy) vyy = pml_y(g, M, S.psiy[Y_VYY] + slot * S.psiy_slot, ii, hy, K_Y, A_Y, B_Y, vyy);
                }
                float sump = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) sump += pick(v[1 + l], e);
                const float gg = pick(v[1 + LL], e), pi = pick(v[2 + LL], e);
                float tp = g.taup0;
                if (ok && tp_p) tp = tp_p[(j - 1 + HY) * g.pitch + (cl.i + e - 1 + HX)];
                const float s = pick(v[0], e) + ((gg * (vxx + vyy)) + (dthalbe * sump));
                sump = 0;
#pragma unroll
                for (int l = 0; l < LL; l++) {
                    const float ee = pi * g.eta[l + 1] * tp;  // e of src/prepare_update_p.c:62
                    const float pp = g.bjm[l + 1] * (pick(v[1 + l], e) * g.cjm[l + 1] - (ee * (vxx + vyy)));
                    o[1 + l][e] = pp;
                    sump += pp;
                }
                o[0][e] = s + (dthalbe * sump);
            }
            const RowOut out(g, S, so, slot, j, cl);
            out.put(S.off[P_SP], o[0][0], o[0][1]);
#pragma unroll
            for (int l = 0; l < LL; l++) out.put(S.mem_off[1] + l * g.plane, o[1 + l][0], o[1 + l][1]);
            out.snap(so.n, tm.snap_comp[P_SP], o[0][0], o[0][1]);
        }
    }
};
#undef IFOS_TILE_COMPUTE
#undef IFOS_OP_MEMBERS

// Blocks per SM for the register budget: as many as the shared-memory ring
// allows (227 KB per SM), at most 3, and no more than leave 64 registers a
// thread.
template <typename P>
constexpr int ring_blocks() {
    constexpr int by_smem = (int)(232448 / (P::bytes() + 1024));
    constexpr int by_regs = 65536 / (kBlockThreads * (P::BLOCK_CAP > 3 ? 56 : 64));
    constexpr int b = by_smem < by_regs ? by_smem : by_regs;
    return b < 1 ? 1 : (b > P::BLOCK_CAP ? P::BLOCK_CAP : b);
}

// the kernel: one Op per launch, persistent over all tiles of all slots
template <typename Op>
__global__ void __launch_bounds__(kBlockThreads, ring_blocks<typename Op::P>())
    kp_stencil(const __grid_constant__ KMaps maps, const __grid_constant__ Op op, int nshots, int *err) {
    run_pipeline<typename Op::P>(op.g, maps, nshots, op, err);
}

}  // namespace ifos
