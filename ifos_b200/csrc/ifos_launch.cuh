// Device context and stencil launcher of libifos_b200, shared by the solver
// (ifos_solver.cu) and the per-FDORDER stencil translation units
// (ifos_pipe.cu, compiled once per half stencil width FD = FDORDER/2 so that
// the pipelined kernels of the six widths compile in parallel).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "ifos_gpu.h"
#include "ifos_kernels.cuh"
#include "ifos_setup.h"
#include "ifos_snap.cuh"
#include "ifos_tile.cuh"
#ifndef IFOS_PIPE_FD
#include "ifos_update.cuh"
#endif

using namespace ifos;

// rows of a pipelined tile (kTileX = 64 columns x kTileY rows)
#ifndef IFOS_TILE_Y
#define IFOS_TILE_Y 8
#endif
static constexpr int kTileY = IFOS_TILE_Y;
// rows of the velocity ops' tiles (their own tensor maps when they differ)
#ifndef IFOS_VTILE_Y
#define IFOS_VTILE_Y 8
#endif
static constexpr int kTileYV = IFOS_VTILE_Y;

// Stages of an op's shared-memory ring: as many as fit when kRingBlocks
// blocks share an SM's 227 KB (2..6).  Loads stay in flight in every stage
// but the one being computed, so deeper rings keep more bytes in flight.
#ifndef IFOS_RING_BLOCKS
#define IFOS_RING_BLOCKS 3
#endif
constexpr int kRingBlocks = IFOS_RING_BLOCKS;
template <int FD, int NH, int NP, int NO, int TY = kTileY, int RB = kRingBlocks>
constexpr int ring_stages() {
    constexpr size_t stage = Pipe<FD, TY, NH, NP, NO, 1>::bytes();
    constexpr int n = (int)((232448 / RB - 1024) / stage);
    return n < 2 ? 2 : (n > 6 ? 6 : n);
}

// Launch a kernel of the time loop as a programmatic dependent of the
// preceding one (it starts while that one drains; its own griddepcontrol.wait
// orders every dependent access).  Without IFOS_PDL (=0) a plain launch.
template <typename... KArgs, typename... Args>
inline void launch_dep(cudaStream_t st, bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, args...);
}
// largest L on the pipelined path (more SLS fall back to one thread per cell)
static constexpr int kPipeMaxL = 5;

// receiver rows a slot's cell map holds: slots whose receivers lie on more
// rows are sampled and injected by the separate receiver kernels
constexpr int kRecMapRows = 8;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// a sampled kernel-class interval (start and end event)
struct TimedPair {
    int cls;
    cudaEvent_t e0, e1;
};
// one captured time loop: the instantiated graph, the launch sequence it was
// captured for (key), the kernels it launches, and its timing events
struct LoopGraph {
    std::string key;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
    std::vector<cudaEvent_t> events;
    std::vector<TimedPair> pairs;
};

struct ifos_ctx {
    ifos_params p{};
    int device = 0;
    bool dbl = false;  // fp64 arithmetic
    size_t esz = 4;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    int last_code = 0;  // code of the last failed call, read and cleared by ifos_status
    KGrid g{};
    int psv = 0, sh = 0, ac = 0;
    // state
    DevBuf state, psi, models, prof, srf, slot_model, src_pos, src_sig, src_n, rec_pos, rec_n, rec_map, adj, sec,
        snap, snap_scale, gacc, gacc64, gout, bad, dot_partial, dot_out, res_tr;
    long long slot_stride = 0, psix_len = 0, psiy_len = 0, psi_slot = 0, model_stride = 0;
    long long off[NP_FIELD];
    long long mem_off[5];
    bool mplane[NM_PLANE];
    long long moff[NM_PLANE];
    bool tau_planes = false;
    ViscoScalars vsc{};
    // snapshots
    bool with_snap = false;
    int ncomp = 0, comp_plane[8] = {0};
    long long snap_bytes = 0, snap_slot_bytes = 0, snap_ex_off = 0;
    bool snaps_valid = false;
    int fwd_nshots = 0;
    // host mirrors
    std::vector<int> nsrc_h, ntr_h, slot_model_h;
    std::vector<int> rec_row_lo, rec_row_hi;  // per slot: rows holding its receivers (lo > hi: none)
    std::vector<char> rec_mapped;             // per slot: its receivers fit the cell map (kRecMapRows rows)
    std::vector<float> srcpos_h;
    bool adj_staged = false;
    float last_ms = 0.0f;
    long long launches = 0;
    cudaStream_t own_st = nullptr;  // the context's own stream (st may be a caller's)
    // asynchronous fetches: a copy stream, the event a copy waits for, and
    // per buffer the completion of its latest copy (pending until a later
    // writer of the buffer has been ordered after it)
    cudaStream_t cp_st = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_sec_done = nullptr, ev_grad_done = nullptr;
    bool sec_pending = false, grad_pending = false;
    // sampled per-kernel timing
    int prof_stride = 0;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<TimedPair> ev_pairs;
    double kt_ms[4] = {0, 0, 0, 0};
    long long kt_n[4] = {0, 0, 0, 0};
    // pipelined (TMA) stencil path: fp32, L <= kPipeMaxL
    bool pipe = false;
    bool fused_snap = false;  // fp32 snapshots written by the stencil kernels
    bool pdl = true;          // time-loop kernels launched as programmatic dependents
    KMaps maps{};
    KMaps maps_v{};  // tensor maps of the velocity ops' tile height
    KTma ktma{};
    int num_sms = 148;
    // execution options (IFOS_OPT_*)
    bool graphs = true;     // time loops captured once and replayed as CUDA graphs
    int blocks_per_sm = 0;  // persistent stencil CTAs per SM (0: as many as fit)
    cudaStream_t cap_st = nullptr;  // capture stream (the caller's may be the legacy default stream)
    bool capturing = false;         // a loop is being captured: timing events become graph nodes
    LoopGraph gfwd, gadj;
};

// ----------------------------------------------------------------------------
template <typename T>
inline KState<T> kstate(const ifos_ctx *c) {
    KState<T> s{};
    s.base = (T *)c->state.p;
    s.slot_stride = c->slot_stride;
    for (int k = 0; k < NP_FIELD; k++) s.off[k] = c->off[k] < 0 ? 0 : c->off[k];
    for (int k = 0; k < 5; k++) s.mem_off[k] = c->mem_off[k] < 0 ? 0 : c->mem_off[k];
    T *psi = (T *)c->psi.p;
    for (int k = 0; k < NX_STRIP; k++) s.psix[k] = psi + k * c->psix_len;
    for (int k = 0; k < NY_STRIP; k++) s.psiy[k] = psi + NX_STRIP * c->psix_len + k * c->psiy_len;
    s.psix_slot = c->psi_slot;
    s.psiy_slot = c->psi_slot;
    return s;
}
template <typename T>
inline KModel<T> kmodel(const ifos_ctx *c) {
    KModel<T> m{};
    for (int k = 0; k < NM_PLANE; k++) {
        bool use = c->mplane[k];
        if ((k == M_TAUS || k == M_TAUP || k == M_TAUSIPJP) && !c->tau_planes) use = false;
        m.m[k] = use ? (const T *)c->models.p + c->moff[k] : nullptr;
    }
    m.model_stride = c->model_stride;
    m.slot_model = (const int *)c->slot_model.p;
    m.prof = (const T *)c->prof.p;
    m.srf = (const T *)c->srf.p;
    m.srf_stride = 4LL * c->p.nx;
    return m;
}
inline KSrc ksrc(const ifos_ctx *c) {
    KSrc s{};
    s.pos = (const float *)c->src_pos.p;
    s.sig = (const float *)c->src_sig.p;
    s.nsrc = (const int *)c->src_n.p;
    s.max_src = std::max(1, c->p.max_src);
    s.nt_total = c->p.nt;
    return s;
}
inline KRec krec(const ifos_ctx *c) {
    KRec r{};
    r.pos = (const int *)c->rec_pos.p;
    r.ntr = (const int *)c->rec_n.p;
    r.max_rec = std::max(1, c->p.max_rec);
    r.adj = (const float *)c->adj.p;
    r.sec = (float *)c->sec.p;
    r.map = (const int *)c->rec_map.p;
    r.map_stride = (long long)c->p.ny + (long long)kRecMapRows * c->p.nx;
    r.rmax = kRecMapRows;
    return r;
}
inline KSnap ksnap(const ifos_ctx *c) {
    KSnap s{};
    s.base = c->snap.p;
    s.slot_bytes = c->snap_slot_bytes;
    s.snap_bytes = c->snap_bytes;
    s.scale = (float *)c->snap_scale.p;
    s.ncomp = c->ncomp;
    s.ntdtinv = c->p.nt / c->p.dtinv;
    s.format = c->p.snap_format;
    for (int k = 0; k < 8; k++) s.comp_plane[k] = c->comp_plane[k];
    s.n = (long long)c->p.nx * c->p.ny;
    s.nx = c->p.nx;
    s.ny = c->p.ny;
    s.segs = (c->p.nx + 63) / 64;
    s.ex_off = c->snap_ex_off;
    return s;
}

#define DISPATCH_FDOH(fdoh, ...)                 \
    switch (fdoh) {                              \
        case 1: { constexpr int FD = 1; __VA_ARGS__; } break; \
        case 2: { constexpr int FD = 2; __VA_ARGS__; } break; \
        case 3: { constexpr int FD = 3; __VA_ARGS__; } break; \
        case 4: { constexpr int FD = 4; __VA_ARGS__; } break; \
        case 5: { constexpr int FD = 5; __VA_ARGS__; } break; \
        default: { constexpr int FD = 6; __VA_ARGS__; } break; \
    }

template <typename T>
struct Launcher {
    ifos_ctx *c;
    KState<T> S;
    KModel<T> M;
    KSrc src;
    KRec rec;
    dim3 blk{32, 8, 1}, grd;
    int nshots;
    // the stress ops apply the explosive sources (fps) and the free surface
    // (fsurf) of step nt_cur themselves: P-SV elastic and viscoelastic only
    int nt_cur = 0, fsurf = 0, fps = 0;
    int src_j0 = 1, src_j1 = 0;  // rows holding the slots' sources (empty range: none)
    // the P-SV velocity ops sample (1) or inject (2) the receivers of rows
    // rec_j0..rec_j1 themselves (the setting of the step being launched)
    int rec_mode = 0, rec_j0 = 1, rec_j1 = 0;
    bool seis_fused = false;  // the forward's velocity ops sample the receivers (no seismogram kernel)
    // rows holding the receivers of slots [0, nshots); false when a slot's
    // receivers do not fit its cell map
    bool receiver_rows() {
        rec_j0 = c->p.ny + 1;
        rec_j1 = 0;
        bool ok = true;
        for (int s = 0; s < nshots; s++) {
            if (c->ntr_h[s] <= 0) continue;
            ok = ok && c->rec_mapped[s];
            rec_j0 = std::min(rec_j0, c->rec_row_lo[s]);
            rec_j1 = std::max(rec_j1, c->rec_row_hi[s]);
        }
        return ok;
    }
    Launcher(ifos_ctx *cc, int ns) : c(cc), nshots(ns) {
        S = kstate<T>(c);
        M = kmodel<T>(c);
        src = ksrc(c);
        rec = krec(c);
        grd = dim3((c->p.nx + 31) / 32, (c->p.ny + 7) / 8, ns);
    }
    // one persistent launch of a pipelined stencil op over all tiles of all slots
    template <typename Op>
    void pipelined(const Op &op0) {
        using P = typename Op::P;
        Op op = op0;
        op.nt = nt_cur;
        op.rec = rec;
        op.rec_mode = rec_mode;
        op.rec_j0 = rec_j0;
        op.rec_j1 = rec_j1;
        op.bad = (int *)c->bad.p;
        static_assert(P::bytes() + 1024 <= 232448, "shared-memory ring exceeds 227 KB");
        auto kern = kp_stencil<Op>;
        constexpr int kMaxDev = 64;
        static int occ[kMaxDev] = {0};  // resident blocks per SM, per device (0: not queried)
        const int d = c->device < kMaxDev ? c->device : kMaxDev - 1;
        if (!occ[d]) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::bytes());
            int o = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, kBlockThreads, P::bytes());
            occ[d] = o > 0 ? o : 1;
        }
        const long long ntiles =
            (long long)((c->p.nx + kTileX - 1) / kTileX) * ((c->p.ny + P::TILE_Y - 1) / P::TILE_Y) * nshots;
        const int bps = c->blocks_per_sm > 0 ? std::min(c->blocks_per_sm, occ[d]) : occ[d];
        const int grid = (int)std::min<long long>(ntiles, (long long)bps * c->num_sms);
        const KMaps &mp = P::TILE_Y == kTileY ? c->maps : c->maps_v;
        launch_dep(c->st, c->pdl, kern, dim3(grid), dim3(32, kComputeWarps + 1), P::bytes(), mp, op, nshots,
                   (int *)c->bad.p);
    }
    // the snapshot a launch stores (hin < 0: none)
    KSnapOut snap_out(int hin) const {
        KSnapOut so{};
        if (hin >= 0) {
            so.base = (char *)c->snap.p + (size_t)hin * c->snap_bytes;
            so.slot_bytes = c->snap_slot_bytes;
            so.n = (long long)c->p.nx * c->p.ny;
            so.pairs = (c->p.nx % 2) == 0;
            so.f16 = c->p.snap_format == IFOS_SNAP_F16S;
            so.ex_off = c->snap_ex_off;
            so.segs = (c->p.nx + 63) / 64;
        }
        return so;
    }
    template <int FD, bool Q, int SW, bool P1>
    void v_one(int hin) {
        const KGrid &g = c->g;
        const KTma &t = c->ktma;
        if (c->ac) {
            constexpr int NP = (SW == 1 && !Q) ? 6 : 4;
            pipelined(OpVPsv<FD, kTileYV, ring_stages<FD, 1, NP, 0, kTileYV, vblocks(FD)>(), Q, SW, P1, true>{g, S, M, t, snap_out(hin)});
            return;
        }
        if (c->psv) {
            constexpr int NP = (SW == 1 && !Q) ? 6 : 4;
            pipelined(OpVPsv<FD, kTileYV, ring_stages<FD, 3, NP, 0, kTileYV, vblocks(FD)>(), Q, SW, P1, false>{g, S, M, t, snap_out(hin)});
        }
    }
    // hin: snapshot index stored by this step's kernels (-1 none)
    template <int FD>
    void v_pipe(int sw, int want_p1, int hin) {
        bool done = false;
        if constexpr (FD >= 5) {
            if (c->g.quirk_hi) {
                v_one<FD, true, 0, false>(-1);
                done = true;
            }
        }
        if (!done) {
            if (sw) v_one<FD, false, 1, false>(-1);
            else if (want_p1) v_one<FD, false, 0, true>(hin);
            else v_one<FD, false, 0, false>(-1);
        }
        if (c->sh) pipelined(OpVSh<FD, kTileYV, ring_stages<FD, 2, 2, 0, kTileYV, vblocks(FD)>()>{c->g, S, M, c->ktma, snap_out(hin)});
    }
    template <int FD, int LL>
    void s_visc_pipe(int hin) {
        const KGrid &g = c->g;
        constexpr int NST = ring_stages<FD, 2, 3 + 3 * LL + 6, 0>();
        if (c->psv) {
            bool done = false;
            if constexpr (FD >= 5) {
                if (g.quirk_hi) {
                    pipelined(OpSVisc<FD, kTileY, LL, NST, true>{g, S, M, c->ktma, snap_out(hin), src, nt_cur, fsurf,
                                                                 fps, src_j0, src_j1});
                    done = true;
                }
            }
            if (!done)
                pipelined(OpSVisc<FD, kTileY, LL, NST, false>{g, S, M, c->ktma, snap_out(hin), src, nt_cur, fsurf, fps, src_j0,
                                                              src_j1});
        }
        if (c->sh) pipelined(OpSSh<FD, kTileY, LL, ring_stages<FD, 1, 2 + 2 * LL + 4, 0>()>{g, S, M, c->ktma, snap_out(hin)});
    }
    template <int FD, int LL>
    void p_visc_pipe(int hin) {
        pipelined(OpPVisc<FD, kTileY, LL, ring_stages<FD, 2, 3 + LL, 0>()>{c->g, S, M, c->ktma, snap_out(hin)});
    }
    template <int FD>
    void s_pipe(int hin) {
        const KGrid &g = c->g;
        const KTma &t = c->ktma;
        bool quirk = false;
        if constexpr (FD >= 5) quirk = g.quirk_hi != 0;
        if (c->ac && g.L) {
            switch (g.L) {
                case 1: p_visc_pipe<FD, 1>(hin); break;
                case 2: p_visc_pipe<FD, 2>(hin); break;
                case 3: p_visc_pipe<FD, 3>(hin); break;
                case 4: p_visc_pipe<FD, 4>(hin); break;
                default: p_visc_pipe<FD, 5>(hin); break;
            }
            return;
        }
        if (c->ac) {
            constexpr int NST = ring_stages<FD, 2, 2, 0>();
            if constexpr (FD >= 5) {
                if (quirk) {
                    pipelined(OpPAc<FD, kTileY, NST, true>{g, S, M, t, snap_out(hin)});
                    return;
                }
            }
            pipelined(OpPAc<FD, kTileY, NST, false>{g, S, M, t, snap_out(hin)});
            return;
        }
        switch (g.L) {
            case 0:
                if (c->psv) {
                    constexpr int NST = ring_stages<FD, 2, 6, 0, kTileY, sblocks(FD)>();
                    bool done = false;
                    if constexpr (FD >= 5) {
                        if (quirk) {
                            pipelined(OpSEl<FD, kTileY, NST, true>{g, S, M, t, snap_out(hin), src, nt_cur, fsurf, fps, src_j0, src_j1});
                            done = true;
                        }
                    }
                    if (!done) pipelined(OpSEl<FD, kTileY, NST, false>{g, S, M, t, snap_out(hin), src, nt_cur, fsurf, fps, src_j0, src_j1});
                }
                if (c->sh) pipelined(OpSSh<FD, kTileY, 0, ring_stages<FD, 1, 4, 0>()>{g, S, M, t, snap_out(hin)});
                break;
            case 1: s_visc_pipe<FD, 1>(hin); break;
            case 2: s_visc_pipe<FD, 2>(hin); break;
            case 3: s_visc_pipe<FD, 3>(hin); break;
            case 4: s_visc_pipe<FD, 4>(hin); break;
            default: s_visc_pipe<FD, 5>(hin); break;
        }
    }
    void v_step(int sw, int want_p1, int hin = -1) {
        const KGrid &g = c->g;
        if constexpr (std::is_same<T, float>::value) {
            if (c->pipe) {
                DISPATCH_FDOH(g.fdoh, v_pipe<FD>(sw, want_p1, hin));
                c->launches += (c->ac ? 1 : c->psv + c->sh);
                return;
            }
        }
        DISPATCH_FDOH(g.fdoh, {
            if (c->ac) k_v_ac<T, FD><<<grd, blk, 0, c->st>>>(g, S, M, sw, want_p1);
            else {
                if (c->psv) k_v_psv<T, FD><<<grd, blk, 0, c->st>>>(g, S, M, sw, want_p1);
                if (c->sh) k_v_sh<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
            }
        });
        c->launches += (c->ac ? 1 : c->psv + c->sh);
    }
    void s_step(int hin = -1) {
        const KGrid &g = c->g;
        if constexpr (std::is_same<T, float>::value) {
            if (c->pipe) {
                DISPATCH_FDOH(g.fdoh, s_pipe<FD>(hin));
                c->launches += (c->ac ? 1 : c->psv + c->sh);
                return;
            }
        }
        DISPATCH_FDOH(g.fdoh, {
            if (c->ac && g.L) k_p_visc<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
            else if (c->ac) k_p_ac<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
            else {
                if (c->psv) {
                    if (g.L) k_s_psv_visc<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
                    else k_s_psv_el<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
                }
                if (c->sh) k_s_sh<T, FD><<<grd, blk, 0, c->st>>>(g, S, M);
            }
        });
        c->launches += (c->ac ? 1 : c->psv + c->sh);
    }
    // the explosive sources, free surface and receivers of a forward step
    void post_fwd(int nt, bool psource, const KSnapPatch &pt) {
        const KGrid &g = c->g;
        if (!fps && (psource || c->p.free_surf)) {
            const dim3 gs((unsigned)((c->p.nx + 127) / 128), (unsigned)nshots);
            DISPATCH_FDOH(g.fdoh, launch_dep(c->st, c->pdl, k_surface_src<T, FD>, gs, dim3(128), 0, g, S, M, src, nt,
                                             c->psv, c->sh, c->ac, psource ? 1 : 0, c->p.free_surf ? 1 : 0, pt));
            c->launches++;
        }
        if (seis_fused) return;  // the velocity op sampled the receivers and probed for NaN
        const dim3 gr((unsigned)((std::max(1, c->p.max_rec) + 127) / 128), (unsigned)nshots);
        DISPATCH_FDOH(g.fdoh, launch_dep(c->st, c->pdl, k_seismo<T, FD>, gr, dim3(128), 0, g, S, M, rec, nt,
                                         c->p.seismo, c->psv, c->sh, c->ac, (int *)c->bad.p));
        c->launches++;
    }
    // the residual pressure source and free surface of an adjoint step
    void post_adj(int nt, bool psource) {
        const KGrid &g = c->g;
        if (psource) {
            const dim3 gr((unsigned)((std::max(1, c->p.max_rec) + 127) / 128), (unsigned)nshots);
            launch_dep(c->st, c->pdl, k_psource_adj<T>, gr, dim3(128), 0, g, S, rec, nt, c->ac);
            c->launches++;
        }
        if (c->p.free_surf && !fsurf) {
            const dim3 gs((unsigned)((c->p.nx + 127) / 128), (unsigned)nshots);
            DISPATCH_FDOH(g.fdoh, launch_dep(c->st, c->pdl, k_surface_src<T, FD>, gs, dim3(128), 0, g, S, M, src, nt,
                                             c->psv, c->sh, c->ac, 0, 1, KSnapPatch{}));
            c->launches++;
        }
    }
};

// The pipelined stencil launches of each width are instantiated in their own
// translation unit (ifos_pipe.cu with IFOS_PIPE_FD set); everywhere else they
// are only declared.
#ifndef IFOS_PIPE_FD
#define IFOS_EXTERN_PIPE(FD)                                      \
    extern template void Launcher<float>::v_pipe<FD>(int, int, int); \
    extern template void Launcher<float>::s_pipe<FD>(int);
IFOS_EXTERN_PIPE(1)
IFOS_EXTERN_PIPE(2)
IFOS_EXTERN_PIPE(3)
IFOS_EXTERN_PIPE(4)
IFOS_EXTERN_PIPE(5)
IFOS_EXTERN_PIPE(6)
#undef IFOS_EXTERN_PIPE
#endif
