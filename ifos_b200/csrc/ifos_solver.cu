// libifos_b200: device context, time loops and the C ABI (include/ifos_gpu.h).
#include "ifos_launch.cuh"

namespace {
thread_local std::string g_create_error;
}  // namespace


// Events for the sampled kernel timing come from a pool that grows on demand;
// a captured loop takes the events it recorded out of the pool and owns them.
static cudaEvent_t pool_event(ifos_ctx *c) {
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}
struct KTimer {
    ifos_ctx *c;
    int cls;
    cudaEvent_t e0 = nullptr;
    KTimer(ifos_ctx *cc, int k, bool sample) : c(cc), cls(k) {
        if (!(sample && cc->prof_stride > 0)) return;
        e0 = pool_event(c);
        if (e0) cudaEventRecordWithFlags(e0, c->st, c->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
    ~KTimer() {
        if (!e0) return;
        cudaEvent_t e1 = pool_event(c);
        if (!e1) return;
        cudaEventRecordWithFlags(e1, c->st, c->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
        c->ev_pairs.push_back({cls, e0, e1});
    }
};
static void collect_kernel_times(ifos_ctx *c) {
    for (auto &pr : c->ev_pairs) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, pr.e0, pr.e1) == cudaSuccess) {
            c->kt_ms[pr.cls] += ms;
            c->kt_n[pr.cls]++;
        } else {
            cudaGetLastError();  // an unusable sample is dropped, not reported later
        }
    }
    c->ev_pairs.clear();
    c->ev_used = 0;
}
static void drop_graph(LoopGraph &lg) {
    if (lg.exec) cudaGraphExecDestroy(lg.exec);
    for (cudaEvent_t e : lg.events) cudaEventDestroy(e);
    lg = LoopGraph{};
}

// ----------------------------------------------------------------------------
static int fail(ifos_ctx *c, int code, const std::string &msg) {
    if (c) {
        c->err = msg;
        c->last_code = code;
    } else {
        g_create_error = msg;
    }
    return code;
}
#define CK(call)                                                                                            \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return fail(c, IFOS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static int dev_alloc(ifos_ctx *c, DevBuf &b, size_t bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if (!bytes) return IFOS_OK;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(c, IFOS_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    }
    b.bytes = bytes;
    return IFOS_OK;
}
static void dev_free(DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

// Grow-only per-context scratch (the res_tr buffer): a call that needs no more
// than any call before it allocates nothing, so concurrent contexts on other
// streams are not stalled by the device-wide synchronisation of cudaFree.
static int scratch(ifos_ctx *c, size_t bytes, void **out) {
    if (c->res_tr.bytes < bytes) {
        CK(cudaStreamSynchronize(c->st));
        if (int rc = dev_alloc(c, c->res_tr, bytes)) return rc;
    }
    *out = c->res_tr.p;
    return IFOS_OK;
}

static int check_params(const ifos_params &p, std::string &why) {
    auto bad = [&](const char *m) {
        why = m;
        return IFOS_ERR_ARG;
    };
    if (p.nx < 1 || p.ny < 1 || p.nt < 1) return bad("NX, NY and NT must be positive");
    if (p.grad_acc64 && (p.precision != 0 || (p.nx & 1) ||
                         (p.snap_format != IFOS_SNAP_F32 && p.snap_format != IFOS_SNAP_F16S &&
                          p.snap_format != IFOS_SNAP_I16S)))
        return bad("grad_acc64 needs fp32 arithmetic, an even NX and fp32 or 16-bit segment snapshots");
    if (p.fdorder < 2 || p.fdorder > 12 || (p.fdorder & 1)) return bad("FDORDER must be 2, 4, 6, 8, 10 or 12");
    if (p.maxrelerror < 0 || p.maxrelerror > 4) return bad("MAXRELERROR must be 0..4");
    if (p.fw < 0 || 2 * p.fw > p.nx || 2 * p.fw > p.ny) return bad("FW does not fit the grid");
    if (p.L < 0 || p.L > IFOS_MAX_L) return bad("L must be 0..8");
    if (p.wavetype < 1 || p.wavetype > 3) return bad("WAVETYPE must be 1, 2 or 3");
    if (p.acoustic && p.wavetype != 1) return bad("acoustic modelling is P-SV only");
    // PARAMETERIZATION 2 has no branch in the reference's stress updates, av_mue or
    // prepare_update_s (src/update_s_elastic_PML.c:132-137 leave f and g unset), and
    // acoustic PARAMETERIZATION 3 none in update_p_PML (src/update_p_PML.c:96-98):
    // no run of the reference defines those results
    if (p.parameterization == 2)
        return bad("PARAMETERIZATION=2 is not defined by the reference's stress updates; use 1 or 3");
    if (p.parameterization != 1 && p.parameterization != 3) return bad("PARAMETERIZATION must be 1 or 3");
    if (p.parameterization == 3 && p.acoustic)
        return bad("acoustic modelling has no PARAMETERIZATION=3 branch in the reference; use 1");
    if (p.velocity != 0) return bad("only VELOCITY=0 is implemented");
    if (p.dtinv < 1 || p.nt % p.dtinv) return bad("NT must be a multiple of DTINV");
    if (p.seismo < 0 || p.seismo > 5) return bad("SEISMO must be 0..5");
    if (p.max_shots < 1 || p.max_models < 1) return bad("max_shots and max_models must be >= 1");
    if (p.max_src < 0 || p.max_rec < 0) return bad("max_src/max_rec must be >= 0");
    if (p.snap_format < 0 || p.snap_format > 4) return bad("snap_format must be 0, 1, 2, 3 or 4");
    if (p.precision < 0 || p.precision > 1) return bad("precision must be 0 or 1");
    if (!(p.dt > 0) || !(p.dh > 0)) return bad("DT and DH must be positive");
    for (int l = 0; l < p.L; l++)
        if (!(p.fl[l] > 0)) return bad("FL1..FLL must be positive");
    return IFOS_OK;
}

struct Layout {
    long long pitch, rows, plane, slot_elems, psix, psiy, psi_slot, model_elems;
    int nfield, nmem, nmodel;
    long long snap_bytes_per, snap_slot_bytes;
    long long snap_ex_off;  // fp16 segments: bytes from a snapshot to its exponents
    int ncomp, segs;
};

static Layout layout_of(const ifos_params &p) {
    Layout L{};
    L.pitch = ((p.nx + 2 * HX) + 31) / 32 * 32;
    L.rows = p.ny + 2 * HY;
    L.plane = L.pitch * L.rows;
    const int psv = p.wavetype != 2, sh = p.wavetype != 1;
    L.nfield = 0;
    if (psv) L.nfield += p.acoustic ? 5 : 7;
    if (sh) L.nfield += 4;
    L.nmem = p.L ? (psv ? (p.acoustic ? 1 : 3) * p.L : 0) + (sh ? 2 * p.L : 0) : 0;
    L.slot_elems = (long long)(L.nfield + L.nmem) * L.plane;
    L.psix = (long long)p.ny * 2 * p.fw;
    L.psiy = (long long)2 * p.fw * p.nx;
    L.psi_slot = NX_STRIP * L.psix + NY_STRIP * L.psiy;
    // model planes: rho vp vs rip rjp always; + elastic (uipjp f g mm ll) or acoustic g;
    // + visco (fipjp f g mu pi muipjp [taus taup tausipjp]) or viscoacoustic (g pi [taup])
    L.nmodel = 5 + (p.acoustic ? 1 : 5) + (p.L ? (p.acoustic ? 3 : 9) : 0);
    L.model_elems = (long long)L.nmodel * L.plane;
    L.ncomp = (psv ? (p.acoustic ? 3 : 5) : 0) + (sh ? 3 : 0);
    const int bytes = p.snap_format == 0 ? (p.precision ? 8 : 4) : 2;
    L.snap_bytes_per = (long long)L.ncomp * p.nx * p.ny * bytes;
    L.segs = (p.nx + 63) / 64;
    if (p.snap_format == IFOS_SNAP_F16S || p.snap_format == IFOS_SNAP_I16S) {
        // 16-bit values [comp][NY*NX], then one fp32 scale per component, row and segment
        L.snap_ex_off = (L.snap_bytes_per + 15) / 16 * 16;
        L.snap_bytes_per = (L.snap_ex_off + (long long)L.ncomp * p.ny * L.segs * 4 + 255) / 256 * 256;
    }
    L.snap_slot_bytes = L.snap_bytes_per * (p.nt / p.dtinv);
    return L;
}

extern "C" void ifos_params_default(ifos_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->nx = 100;
    p->ny = 100;
    p->nt = 1000;
    p->dh = 1.0f;
    p->dt = 1e-4f;
    p->fdorder = 4;
    p->fw = 10;
    p->free_surf = 1;
    p->vppml = 1800.0f;
    p->fpml = 20.0f;
    p->npower = 2.0f;
    p->k_max_pml = 1.0f;
    p->wavetype = 1;
    p->parameterization = 1;
    p->seismo = 1;
    p->source_type = 1;
    p->adjoint_type = 1;
    p->dtinv = 1;
    p->max_shots = 1;
    p->max_models = 1;
    p->max_src = 1;
    p->max_rec = 1;
}

extern "C" size_t ifos_ctx_bytes(const ifos_params *p, int with_snapshots) {
    if (!p) return 0;
    Layout L = layout_of(*p);
    const size_t e = p->precision ? 8 : 4;
    size_t b = (size_t)p->max_shots * (L.slot_elems + L.psi_slot) * e;
    b += (size_t)p->max_models * (L.model_elems * e + 4 * (size_t)p->nx * e);
    b += (size_t)p->max_shots * ((size_t)8 * p->max_src * 4 + (size_t)p->max_src * p->nt * 4 + (size_t)2 * p->max_rec * 4 +
                                 (size_t)3 * p->max_rec * p->nt * 4 + (size_t)IFOS_NS * p->max_rec * p->nt * 4);
    b += (size_t)p->max_shots * (size_t)15 * p->nx * p->ny * 4;
    if (with_snapshots) b += (size_t)p->max_shots * L.snap_slot_bytes;
    return b;
}

// error text of context-free entry points, read back by ifos_last_error(NULL)
void ifos_internal_set_error(const std::string &msg) { g_create_error = msg; }

extern "C" const char *ifos_last_error(const ifos_ctx *ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

extern "C" int ifos_ctx_destroy(ifos_ctx *c) {
    if (!c) return IFOS_OK;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->cp_st) cudaStreamSynchronize(c->cp_st);  // asynchronous fetches still reading the buffers
    DevBuf *bufs[] = {&c->state, &c->psi, &c->models, &c->prof, &c->srf, &c->slot_model, &c->src_pos, &c->src_sig,
                      &c->src_n, &c->rec_pos, &c->rec_n, &c->rec_map, &c->adj, &c->sec, &c->snap, &c->snap_scale,
                      &c->gacc, &c->gacc64, &c->gout, &c->bad, &c->dot_partial, &c->dot_out, &c->res_tr};
    for (DevBuf *b : bufs) dev_free(*b);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    drop_graph(c->gfwd);
    drop_graph(c->gadj);
    if (c->cap_st) cudaStreamDestroy(c->cap_st);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->cp_st) cudaStreamDestroy(c->cp_st);
    for (cudaEvent_t e : {c->ev_ready, c->ev_sec_done, c->ev_grad_done})
        if (e) cudaEventDestroy(e);
    if (c->own_st) cudaStreamDestroy(c->own_st);
    delete c;
    return IFOS_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// fp32 planes of `pitch` x `rows` elements, `planes` of them back to back;
// boxes of box_w x box_h x 1, zero fill outside
static bool encode_planes(CUtensorMap *m, void *base, long long pitch, long long rows, long long planes, int box_w,
                          int box_h) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)rows, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)(pitch * rows) * 4};
    const cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Plane tables and tensor maps of the pipelined kernels.  Leaves c->pipe
// false (one thread per cell) for fp64 and for L > kPipeMaxL.
static void setup_pipeline(ifos_ctx *c, const Layout &L) {
    c->pipe = false;
    if (c->dbl || c->p.L > kPipeMaxL || L.slot_elems >= (1LL << 31)) return;
    KTma &t = c->ktma;
    t.planes_per_slot = (int)(L.slot_elems / L.plane);
    for (int k = 0; k < NP_FIELD; k++) t.pid[k] = c->off[k] < 0 ? 0 : (int)(c->off[k] / L.plane);
    for (int k = 0; k < 5; k++) t.mem_pid[k] = c->mem_off[k] < 0 ? 0 : (int)(c->mem_off[k] / L.plane);
    t.model_planes = (int)(L.model_elems / L.plane);
    for (int m = 0; m < NM_PLANE; m++) t.mid[m] = c->moff[m] < 0 ? 0 : (int)(c->moff[m] / L.plane);
    const int fdoh = c->g.fdoh, xh = ((fdoh + 3) / 4) * 4;
    const long long st_planes = (long long)t.planes_per_slot * c->p.max_shots;
    const long long md_planes = (long long)t.model_planes * c->p.max_models;
    if (!encode_planes(&c->maps.halo, c->state.p, L.pitch, L.rows, st_planes, kTileX + 2 * xh, kTileY + 2 * fdoh) ||
        !encode_planes(&c->maps.plain, c->state.p, L.pitch, L.rows, st_planes, kTileX, kTileY) ||
        !encode_planes(&c->maps.model, c->models.p, L.pitch, L.rows, md_planes, kTileX, kTileY))
        return;
    c->maps_v = c->maps;
    if (kTileYV != kTileY &&
        (!encode_planes(&c->maps_v.halo, c->state.p, L.pitch, L.rows, st_planes, kTileX + 2 * xh, kTileYV + 2 * fdoh) ||
         !encode_planes(&c->maps_v.plain, c->state.p, L.pitch, L.rows, st_planes, kTileX, kTileYV) ||
         !encode_planes(&c->maps_v.model, c->models.p, L.pitch, L.rows, md_planes, kTileX, kTileYV)))
        return;
    // fp32 snapshots are written by the stencil kernels themselves
    t.snap_ntd = c->p.nt / c->p.dtinv;
    t.snap_ncomp = c->ncomp;
    for (int k = 0; k < NP_FIELD; k++) t.snap_comp[k] = -1;
    for (int k = 0; k < c->ncomp; k++) t.snap_comp[c->comp_plane[k]] = k;
    // int16 segments are stored by k_snap_seg16 after the step, which keeps
    // their packing out of the stencil kernels
    c->fused_snap = c->with_snap && (c->p.snap_format == IFOS_SNAP_F32 || c->p.snap_format == IFOS_SNAP_F16S);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) == cudaSuccess && sms > 0)
        c->num_sms = sms;
    c->pipe = true;
}

extern "C" int ifos_ctx_create(const ifos_params *pp, int device, int with_snapshots, ifos_ctx **out) {
    ifos_ctx *c = nullptr;
    if (!pp || !out) return fail(c, IFOS_ERR_ARG, "null argument");
    *out = nullptr;
    std::string why;
    if (int rc = check_params(*pp, why)) return fail(c, rc, why);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(c, IFOS_ERR_CUDA, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(c, IFOS_ERR_ARG, "bad device index");
    c = new (std::nothrow) ifos_ctx();
    if (!c) return fail(nullptr, IFOS_ERR_NOMEM, "host allocation failed");
    c->p = *pp;
    c->device = device;
    const ifos_params &p = c->p;
    c->dbl = p.precision == 1;
    c->esz = c->dbl ? 8 : 4;
    c->psv = p.wavetype != 2;
    c->sh = p.wavetype != 1;
    c->ac = p.acoustic;
    c->with_snap = with_snapshots != 0;
    auto bail = [&](int rc) {
        g_create_error = c->err;
        ifos_ctx_destroy(c);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->cap_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess)
        return bail(fail(c, IFOS_ERR_CUDA, "stream/event creation failed"));
    c->st = c->own_st;

    Layout L = layout_of(p);
    KGrid &g = c->g;
    g.nx = p.nx;
    g.ny = p.ny;
    g.pitch = (int)L.pitch;
    g.plane = L.plane;
    g.fw = p.fw;
    g.free_surf = p.free_surf;
    g.boundary = p.boundary;
    g.fdoh = p.fdorder / 2;
    g.L = p.L;
    g.quirk_hi = (p.fdorder >= 10 && !p.hi_order_corrected && (c->psv || c->ac)) ? 1 : 0;
    g.mu_fix = p.mu_corrected ? 1 : 0;
    g.lame = p.parameterization == 3 ? 1 : 0;
    g.tile_order = 2;  // CPML strip tiles first, slot-major (IFOS_OPT_TILE_ORDER)
    g.nt_total = p.nt;
    g.dt = p.dt;
    g.dh = p.dh;
    g.adjoint_type = p.adjoint_type;
    if (!fd_coefficients(p.fdorder, p.maxrelerror, g.hc)) return bail(fail(c, IFOS_ERR_ARG, "bad FD order"));
    c->vsc = visco_scalars(p);
    for (int l = 0; l <= IFOS_MAX_L; l++) {
        g.eta[l] = c->vsc.eta[l];
        g.bip[l] = c->vsc.bip[l];
        g.bjm[l] = c->vsc.bjm[l];
        g.cip[l] = c->vsc.cip[l];
        g.cjm[l] = c->vsc.cjm[l];
        g.bjm_srf[l] = c->vsc.bjm_srf[l];
    }

    // state plane table
    for (auto &o : c->off) o = -1;
    for (auto &o : c->mem_off) o = -1;
    long long k = 0;
    if (c->psv) {
        c->off[P_VX] = k++ * L.plane;
        c->off[P_VY] = k++ * L.plane;
        if (!c->ac) {
            c->off[P_SXX] = k++ * L.plane;
            c->off[P_SYY] = k++ * L.plane;
            c->off[P_SXY] = k++ * L.plane;
        } else {
            c->off[P_SP] = k++ * L.plane;
        }
        c->off[P_VXP1] = k++ * L.plane;
        c->off[P_VYP1] = k++ * L.plane;
    }
    if (c->sh) {
        c->off[P_VZ] = k++ * L.plane;
        c->off[P_SXZ] = k++ * L.plane;
        c->off[P_SYZ] = k++ * L.plane;
        c->off[P_VZP1] = k++ * L.plane;
    }
    if (p.L) {
        if (c->psv)
            for (int w = 0; w < 3; w++) {
                if (c->ac && w != 1) continue;  // viscoacoustic: the pressure memories only
                c->mem_off[w] = k * L.plane;
                k += p.L;
            }
        if (c->sh)
            for (int w = 3; w < 5; w++) {
                c->mem_off[w] = k * L.plane;
                k += p.L;
            }
    }
    c->slot_stride = L.slot_elems;
    c->psix_len = L.psix;
    c->psiy_len = L.psiy;
    c->psi_slot = L.psi_slot;
    // snapshot components
    c->ncomp = 0;
    if (c->psv) {
        c->comp_plane[c->ncomp++] = P_VXP1;
        c->comp_plane[c->ncomp++] = P_VYP1;
        if (!c->ac) {
            c->comp_plane[c->ncomp++] = P_SXX;
            c->comp_plane[c->ncomp++] = P_SYY;
            c->comp_plane[c->ncomp++] = P_SXY;
        } else {
            c->comp_plane[c->ncomp++] = P_SP;
        }
    }
    if (c->sh) {
        c->comp_plane[c->ncomp++] = P_VZP1;
        c->comp_plane[c->ncomp++] = P_SXZ;
        c->comp_plane[c->ncomp++] = P_SYZ;
    }
    c->snap_bytes = L.snap_bytes_per;
    c->snap_slot_bytes = L.snap_slot_bytes;
    c->snap_ex_off = L.snap_ex_off;

    const size_t e = c->esz;
    const int S = p.max_shots;
    int rc = IFOS_OK;
    if ((rc = dev_alloc(c, c->state, (size_t)S * L.slot_elems * e))) return bail(rc);
    if ((rc = dev_alloc(c, c->psi, (size_t)S * L.psi_slot * e + e))) return bail(rc);
    c->model_stride = L.model_elems;
    if ((rc = dev_alloc(c, c->models, (size_t)p.max_models * L.model_elems * e))) return bail(rc);
    if ((rc = dev_alloc(c, c->prof, (size_t)12 * (2 * p.fw + 1) * e))) return bail(rc);
    if ((rc = dev_alloc(c, c->srf, (size_t)p.max_models * 4 * p.nx * e))) return bail(rc);
    if ((rc = dev_alloc(c, c->slot_model, (size_t)S * sizeof(int)))) return bail(rc);
    const int ms = std::max(1, p.max_src), mr = std::max(1, p.max_rec);
    if ((rc = dev_alloc(c, c->src_pos, (size_t)S * 8 * ms * 4))) return bail(rc);
    if ((rc = dev_alloc(c, c->src_sig, (size_t)S * ms * p.nt * 4))) return bail(rc);
    if ((rc = dev_alloc(c, c->src_n, (size_t)S * sizeof(int)))) return bail(rc);
    if ((rc = dev_alloc(c, c->rec_pos, (size_t)S * 2 * mr * 4))) return bail(rc);
    if ((rc = dev_alloc(c, c->rec_n, (size_t)S * sizeof(int)))) return bail(rc);
    if ((rc = dev_alloc(c, c->rec_map, (size_t)S * ((size_t)p.ny + (size_t)kRecMapRows * p.nx) * sizeof(int))))
        return bail(rc);
    if (cudaMemsetAsync(c->rec_map.p, 0xff, c->rec_map.bytes, c->st) != cudaSuccess)  // -1: no receiver
        return bail(fail(c, IFOS_ERR_CUDA, "receiver map clear failed"));
    if ((rc = dev_alloc(c, c->adj, (size_t)S * 3 * mr * p.nt * 4))) return bail(rc);
    if ((rc = dev_alloc(c, c->sec, (size_t)S * IFOS_NS * mr * p.nt * 4))) return bail(rc);
    const long long N = (long long)p.nx * p.ny;
    if ((rc = dev_alloc(c, c->gacc, (size_t)S * 5 * N * 4))) return bail(rc);
    // the double sums: grad_acc64, and always in an fp64 context (the error oracle sums and assembles in double)
    if ((p.grad_acc64 || p.precision == 1) && (rc = dev_alloc(c, c->gacc64, (size_t)S * 5 * N * 8))) return bail(rc);
    if ((rc = dev_alloc(c, c->gout, (size_t)S * IFOS_NG * N * 4))) return bail(rc);
    if ((rc = dev_alloc(c, c->bad, sizeof(int)))) return bail(rc);
    if ((rc = dev_alloc(c, c->dot_partial, 1024 * sizeof(double)))) return bail(rc);
    if ((rc = dev_alloc(c, c->dot_out, 2 * sizeof(double)))) return bail(rc);
    if (c->with_snap) {
        if ((rc = dev_alloc(c, c->snap, (size_t)S * L.snap_slot_bytes))) return bail(rc);
        // components a loop never writes (vxp1/vyp1 of the FDORDER 10/12
        // branches) read as zero, as the reference's zeroed arrays do
        if (cudaMemsetAsync(c->snap.p, 0, (size_t)S * L.snap_slot_bytes, c->st) != cudaSuccess)
            return bail(fail(c, IFOS_ERR_CUDA, "snapshot clear failed"));
        if ((rc = dev_alloc(c, c->snap_scale, (size_t)S * (p.nt / p.dtinv) * c->ncomp * sizeof(float) + 4)))
            return bail(rc);
    }
    // zero everything that is read before it is written (halos stay zero)
    DevBuf *zb[] = {&c->state, &c->psi, &c->models, &c->srf, &c->slot_model, &c->src_pos, &c->src_sig, &c->src_n,
                    &c->rec_pos, &c->rec_n, &c->adj, &c->sec, &c->gacc, &c->gout, &c->bad};
    for (DevBuf *b : zb)
        if (b->p) CK(cudaMemsetAsync(b->p, 0, b->bytes, c->st));
    // CPML profiles
    CpmlProfiles pr = cpml_profiles(p);
    {
        std::vector<char> hb((size_t)12 * (2 * p.fw + 1) * e);
        for (int a = 0; a < 12; a++)
            for (int h = 0; h <= 2 * p.fw; h++) {
                size_t idx = (size_t)a * (2 * p.fw + 1) + h;
                if (c->dbl) ((double *)hb.data())[idx] = pr.arr[a][h];
                else ((float *)hb.data())[idx] = pr.arr[a][h];
            }
        CK(cudaMemcpyAsync(c->prof.p, hb.data(), hb.size(), cudaMemcpyHostToDevice, c->st));
        // exact shortcuts of the kernels: d/K with K == 1 everywhere, x/DH with DH a power of two
        g.k_one = 1;
        for (int a : {K_X, K_XH, K_Y, K_YH})
            for (int h = 1; h <= 2 * p.fw; h++)  // the profiles are 1-based (index 0 is unused)
                if (pr.arr[a][h] != 1.0) g.k_one = 0;
        int ex = 0;
        g.dh_pow2 = std::frexp(p.dh, &ex) == 0.5f ? 1 : 0;
        g.inv_dh = g.dh_pow2 ? 1.0f / p.dh : 0.0f;
    }
    // model plane table
    for (int m = 0; m < NM_PLANE; m++) {
        c->mplane[m] = false;
        c->moff[m] = -1;
    }
    std::vector<int> present = {M_RHO, M_VP, M_VS, M_RIP, M_RJP};
    if (c->ac) present.push_back(M_GAC);
    else {
        present.push_back(M_UIPJP);
        present.push_back(M_F);
        present.push_back(M_G);
        present.push_back(M_MM);
        present.push_back(M_LL);
    }
    if (p.L && c->ac)
        for (int m : {M_GV, M_PIR, M_TAUP}) present.push_back(m);
    else if (p.L)
        for (int m : {M_FIPJPV, M_FV, M_GV, M_MUR, M_PIR, M_MUIPJPR, M_TAUS, M_TAUP, M_TAUSIPJP}) present.push_back(m);
    for (size_t q = 0; q < present.size(); q++) {
        c->mplane[present[q]] = true;
        c->moff[present[q]] = (long long)q * L.plane;
    }
    c->nsrc_h.assign(S, 0);
    c->ntr_h.assign(S, 0);
    c->rec_row_lo.assign(S, 1);
    c->rec_row_hi.assign(S, 0);
    c->rec_mapped.assign(S, 1);
    c->slot_model_h.assign(S, 0);
    c->srcpos_h.assign((size_t)S * 8 * ms, 0.0f);
    setup_pipeline(c, L);
    if (const char *e = std::getenv("IFOS_PDL")) c->pdl = std::atoi(e) != 0;
    if (const char *e = std::getenv("IFOS_GRAPHS")) c->graphs = std::atoi(e) != 0;
    CK(cudaStreamSynchronize(c->st));
    *out = c;
    return IFOS_OK;
}

// ----------------------------------------------------------------------------
template <typename T>
static void upload_plane(std::vector<T> &host, const ifos_ctx *c, long long off, const std::vector<float> &src) {
    const ifos_params &p = c->p;
    for (int j = 1; j <= p.ny; j++)
        for (int i = 1; i <= p.nx; i++)
            host[off + pidx(c->g, j, i)] = (T)src[(size_t)(j - 1) * p.nx + (i - 1)];
}

template <typename T>
static int model_upload_t(ifos_ctx *c, int model, const ModelPlanes &mp) {
    const Layout L = layout_of(c->p);
    std::vector<T> h((size_t)L.model_elems, (T)0);
    auto put = [&](int id, const std::vector<float> &v) {
        if (c->mplane[id] && !v.empty()) upload_plane<T>(h, c, c->moff[id], v);
    };
    put(M_RHO, mp.rho);
    put(M_VP, mp.vp);
    put(M_VS, mp.vs);
    put(M_RIP, mp.rip);
    put(M_RJP, mp.rjp);
    put(M_UIPJP, mp.uipjp);
    put(M_F, mp.f_el);
    put(M_G, mp.g_el);
    put(M_GAC, mp.g_ac);
    put(M_MM, mp.mm);
    put(M_LL, mp.ll);
    put(M_FIPJPV, mp.fipjp_v);
    put(M_FV, mp.f_v);
    put(M_GV, mp.g_v);
    put(M_MUR, mp.mu_r);
    put(M_PIR, mp.pi_r);
    put(M_MUIPJPR, mp.muipjp_r);
    put(M_TAUS, mp.taus);
    put(M_TAUP, mp.taup);
    put(M_TAUSIPJP, mp.tausipjp);
    ifos_ctx *cc = c;
    {
        ifos_ctx *c = cc;
        CK(cudaMemcpyAsync((char *)c->models.p + (size_t)model * L.model_elems * sizeof(T), h.data(),
                           h.size() * sizeof(T), cudaMemcpyHostToDevice, c->st));
        std::vector<T> s((size_t)4 * c->p.nx, (T)0);
        for (int i = 0; i < c->p.nx; i++) {
            if (!mp.srf_fjm.empty()) s[i] = mp.srf_fjm[i];
            if (!mp.srf_g.empty()) s[c->p.nx + i] = mp.srf_g[i];
            if (!mp.srf_djm.empty()) s[2 * c->p.nx + i] = mp.srf_djm[i];
            if (!mp.srf_e.empty()) s[3 * c->p.nx + i] = mp.srf_e[i];
        }
        CK(cudaMemcpyAsync((char *)c->srf.p + (size_t)model * 4 * c->p.nx * sizeof(T), s.data(), s.size() * sizeof(T),
                           cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    return IFOS_OK;
}

extern "C" int ifos_model_upload(ifos_ctx *c, int model, const float *vp, const float *vs, const float *rho,
                                 const float *taup, const float *taus) {
    if (!c) return IFOS_ERR_ARG;
    if (model < 0 || model >= c->p.max_models) return fail(c, IFOS_ERR_ARG, "model index out of range");
    ModelPlanes mp;
    if (!build_model(c->p, vp, vs, rho, taup, taus, mp)) return fail(c, IFOS_ERR_ARG, "missing model arrays");
    for (size_t k = 0; k < mp.rho.size(); k++)
        if (!(mp.rho[k] > 0) || !std::isfinite(mp.vp[k]) || !std::isfinite(mp.vs[k]))
            return fail(c, IFOS_ERR_ARG, "model has non-finite values or non-positive density");
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed");
    if (c->p.L) {
        // all models of a context share the tau representation of the first upload
        if (!mp.tau_uniform) c->tau_planes = true;
        c->g.taus0 = mp.taus0;
        c->g.taup0 = mp.taup0;
        c->g.tausipjp0 = mp.tausipjp0;
        if (mp.tau_uniform) {
            // planes stay in the table but are ignored (the kernels read the scalars)
            mp.taus.assign(mp.rho.size(), mp.taus0);
            mp.taup.assign(mp.rho.size(), mp.taup0);
            mp.tausipjp.assign(mp.rho.size(), mp.tausipjp0);
        }
    }
    c->snaps_valid = false;
    return c->dbl ? model_upload_t<double>(c, model, mp) : model_upload_t<float>(c, model, mp);
}

extern "C" int ifos_shot_setup(ifos_ctx *c, int slot, int model, int nsrc, const float *srcpos, const float *signals,
                               int ntr, const int *recpos) {
    if (!c) return IFOS_ERR_ARG;
    const ifos_params &p = c->p;
    if (slot < 0 || slot >= p.max_shots) return fail(c, IFOS_ERR_ARG, "slot out of range");
    if (model < 0 || model >= p.max_models) return fail(c, IFOS_ERR_ARG, "model out of range");
    if (nsrc < 0 || nsrc > p.max_src) return fail(c, IFOS_ERR_ARG, "nsrc exceeds max_src");
    if (ntr < 0 || ntr > p.max_rec) return fail(c, IFOS_ERR_ARG, "ntr exceeds max_rec");
    if ((nsrc && (!srcpos || !signals)) || (ntr && !recpos)) return fail(c, IFOS_ERR_ARG, "null geometry");
    for (int l = 0; l < nsrc; l++) {
        const int i = (int)srcpos[l], j = (int)srcpos[nsrc + l];
        if (i < 1 || i > p.nx || j < 1 || j > p.ny)
            return fail(c, IFOS_ERR_ARG, "source " + std::to_string(l) + " outside the grid");
    }
    for (int l = 0; l < ntr; l++) {
        const int i = recpos[l], j = recpos[ntr + l];
        if (i < 1 || i > p.nx || j < 1 || j > p.ny)
            return fail(c, IFOS_ERR_ARG, "receiver " + std::to_string(l) + " outside the grid");
        for (int m = 0; m < l; m++)
            if (recpos[m] == i && recpos[ntr + m] == j)
                return fail(c, IFOS_ERR_ARG, "receivers must be unique per cell (src/receiver.c:73-88)");
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed");
    const int ms = std::max(1, p.max_src), mr = std::max(1, p.max_rec);
    std::vector<float> pos((size_t)8 * ms, 0.0f);
    for (int r = 0; r < 8; r++)
        for (int l = 0; l < nsrc; l++) pos[(size_t)r * ms + l] = srcpos[(size_t)r * nsrc + l];
    std::vector<int> rp((size_t)2 * mr, 1);
    for (int r = 0; r < 2; r++)
        for (int l = 0; l < ntr; l++) rp[(size_t)r * mr + l] = recpos[(size_t)r * ntr + l];
    CK(cudaMemcpyAsync((char *)c->src_pos.p + (size_t)slot * 8 * ms * 4, pos.data(), pos.size() * 4,
                       cudaMemcpyHostToDevice, c->st));
    if (nsrc)
        CK(cudaMemcpyAsync((char *)c->src_sig.p + (size_t)slot * ms * p.nt * 4, signals, (size_t)nsrc * p.nt * 4,
                           cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((char *)c->rec_pos.p + (size_t)slot * 2 * mr * 4, rp.data(), rp.size() * 4,
                       cudaMemcpyHostToDevice, c->st));
    // the slot's cell -> receiver map for the in-stencil sampling and injection
    const size_t mstride = (size_t)p.ny + (size_t)kRecMapRows * p.nx;
    std::vector<int> rm(mstride, -1);
    int lo = p.ny + 1, hi = 0, nrows = 0;
    bool mapped = true;
    for (int l = 0; l < ntr; l++) {
        const int i = recpos[l], j = recpos[ntr + l];
        lo = std::min(lo, j);
        hi = std::max(hi, j);
        if (rm[j - 1] < 0) {
            if (nrows == kRecMapRows) {
                mapped = false;
                continue;
            }
            rm[j - 1] = nrows++;
        }
        rm[(size_t)p.ny + (size_t)rm[j - 1] * p.nx + (i - 1)] = l;
    }
    CK(cudaMemcpyAsync((char *)c->rec_map.p + (size_t)slot * mstride * 4, rm.data(), rm.size() * 4,
                       cudaMemcpyHostToDevice, c->st));
    c->rec_mapped[slot] = mapped;
    c->rec_row_lo[slot] = lo;
    c->rec_row_hi[slot] = hi;
    c->nsrc_h[slot] = nsrc;
    c->ntr_h[slot] = ntr;
    c->slot_model_h[slot] = model;
    std::copy(pos.begin(), pos.end(), c->srcpos_h.begin() + (size_t)slot * 8 * ms);
    CK(cudaMemcpyAsync((char *)c->src_n.p + slot * 4, &c->nsrc_h[slot], 4, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((char *)c->rec_n.p + slot * 4, &c->ntr_h[slot], 4, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((char *)c->slot_model.p + slot * 4, &c->slot_model_h[slot], 4, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->snaps_valid = false;
    return IFOS_OK;
}


static bool any_force_source(const ifos_ctx *c, int nshots) {
    const int ms = std::max(1, c->p.max_src);
    for (int s = 0; s < nshots; s++)
        for (int l = 0; l < c->nsrc_h[s]; l++) {
            int t = (int)c->srcpos_h[(size_t)s * 8 * ms + 7 * ms + l];
            if (t == 2 || t == 3 || t == 4) return true;
        }
    return false;
}

// error codes >= 16 in the status word come from a bounded barrier wait of a
// pipelined kernel that gave up (16/17: a consumer on a stage's loads, 18: the
// producer on a stage's release)
static int pipeline_timeout(ifos_ctx *c, int code) {
    return fail(c, IFOS_ERR_CUDA, "pipelined stencil kernel: barrier wait timed out (code " + std::to_string(code) + ")");
}

template <typename T>
static int zero_state(ifos_ctx *c, int nshots) {
    CK(cudaMemsetAsync(c->state.p, 0, (size_t)nshots * c->slot_stride * sizeof(T), c->st));
    CK(cudaMemsetAsync(c->psi.p, 0, (size_t)nshots * c->psi_slot * sizeof(T), c->st));
    return IFOS_OK;
}

// Run one time loop; enqueue() issues its launches on c->st.  With graphs
// on, the loop is captured once per launch sequence (key) on the capture
// stream and the instantiated graph is replayed on c->st by every later call
// with the same key: every per-shot input the kernels read (sources,
// receivers, adjoint sources, model index) lives in device buffers that
// ifos_shot_setup / ifos_stage_adjoint rewrite in place.
template <typename F>
static int run_loop(ifos_ctx *c, LoopGraph &lg, const std::string &key, F &&enqueue) {
    if (!c->graphs) {
        enqueue();
        CK(cudaGetLastError());
        return IFOS_OK;
    }
    if (lg.key != key || !lg.exec) {
        drop_graph(lg);
        cudaStream_t user = c->st;
        const long long l0 = c->launches;
        const size_t e_first = c->ev_used, p_first = c->ev_pairs.size();
        c->st = c->cap_st;
        cudaError_t e = cudaStreamBeginCapture(c->cap_st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            c->capturing = true;
            enqueue();
            c->capturing = false;
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(c->cap_st, &g);
            if (e == cudaSuccess) {
                e = cudaGraphInstantiate(&lg.exec, g, 0);
                cudaGraphDestroy(g);
            }
        }
        c->st = user;
        lg.launches = c->launches - l0;
        c->launches = l0;
        // the graph owns the timing events it records
        lg.events.assign(c->ev_pool.begin() + e_first, c->ev_pool.begin() + c->ev_used);
        c->ev_pool.erase(c->ev_pool.begin() + e_first, c->ev_pool.begin() + c->ev_used);
        c->ev_used = e_first;
        lg.pairs.assign(c->ev_pairs.begin() + p_first, c->ev_pairs.end());
        c->ev_pairs.resize(p_first);
        if (e != cudaSuccess) {
            drop_graph(lg);
            cudaGetLastError();
            return fail(c, IFOS_ERR_CUDA, std::string("time-loop graph capture: ") + cudaGetErrorString(e));
        }
        lg.key = key;
    }
    CK(cudaGraphLaunch(lg.exec, c->st));
    c->launches += lg.launches;
    c->ev_pairs.insert(c->ev_pairs.end(), lg.pairs.begin(), lg.pairs.end());
    return IFOS_OK;
}

static std::string loop_key(const ifos_ctx *c, std::initializer_list<long long> v) {
    std::string k;
    for (long long x : v) k += std::to_string(x) + ",";
    k += std::to_string(c->prof_stride) + "," + std::to_string(c->pdl) + "," + std::to_string(c->blocks_per_sm) + "," +
         std::to_string(c->g.tile_order) + "," + std::to_string(c->g.prod_polls);
    return k;
}

template <typename T>
static int forward_t(ifos_ctx *c, int nshots, int store, int nsteps) {
    const ifos_params &p = c->p;
    Launcher<T> Lr(c, nshots);
    if (int rc = zero_state<T>(c, nshots)) return rc;
    CK(cudaMemsetAsync(c->sec.p, 0, (size_t)nshots * IFOS_NS * std::max(1, p.max_rec) * p.nt * 4, c->st));
    CK(cudaMemsetAsync(c->bad.p, 0, 4, c->st));
    const bool snaps = store && c->with_snap;
    const int ntd = p.nt / p.dtinv;
    if (snaps && (p.snap_format == IFOS_SNAP_BF16 || p.snap_format == IFOS_SNAP_F16))
        CK(cudaMemsetAsync(c->snap_scale.p, 0, (size_t)nshots * ntd * c->ncomp * 4, c->st));
    const bool force = (c->psv && !c->ac && any_force_source(c, nshots)) || c->sh ||
                       (c->ac && any_force_source(c, nshots));
    KSnap sn = ksnap(c);
    // snapshots stored by the stencil kernels; the source and surface kernel
    // patches the fp32 cells it changes afterwards, and the fp16 segments
    // holding them are stored again after it
    const bool fused = snaps && c->pipe && c->fused_snap;
    const bool f16s = p.snap_format == IFOS_SNAP_F16S || p.snap_format == IFOS_SNAP_I16S;  // 16-bit segments
    // P-SV elastic / viscoelastic: the stress kernel applies the explosive
    // sources and the free surface, so nothing changes a stress after it
    // (no surface kernel, no snapshot patches)
    const bool in_stress = c->pipe && c->psv && !c->ac && !c->sh;
    Lr.fps = in_stress ? 1 : 0;
    Lr.fsurf = (in_stress && p.free_surf) ? 1 : 0;
    // P-SV without force sources, SEISMO 1: vx, vy are final when the velocity
    // op stores them, so it samples the receivers itself (and probes for NaN)
    const bool rec_ok = Lr.receiver_rows();
    const bool seis_fused = std::is_same<T, float>::value && in_stress && !force && p.seismo == 1 && rec_ok;
    Lr.seis_fused = seis_fused;
    {
        const int ms = std::max(1, p.max_src);
        int lo = p.ny + 1, hi = 0;
        for (int s = 0; s < nshots; s++)
            for (int l = 0; l < c->nsrc_h[s]; l++) {
                const int j = (int)c->srcpos_h[(size_t)s * 8 * ms + ms + l];
                lo = std::min(lo, j);
                hi = std::max(hi, j);
            }
        Lr.src_j0 = lo;
        Lr.src_j1 = hi;
    }
    const int segs = (p.nx + 63) / 64;
    KSnapPatch pt{};
    pt.slot_floats = c->snap_slot_bytes / 4;
    pt.n = (long long)p.nx * p.ny;
    auto comp_of = [&](int plane) {
        for (int k = 0; k < c->ncomp; k++)
            if (c->comp_plane[k] == plane) return k;
        return -1;
    };
    pt.c_sxx = comp_of(P_SXX);
    pt.c_syy = comp_of(P_SYY);
    pt.c_sp = comp_of(P_SP);
    pt.c_syz = comp_of(P_SYZ);
    CK(cudaEventRecord(c->ev0, c->st));
    auto enqueue = [&]() {
    int hin = 0;
    for (int nt = 1; nt <= nsteps; nt++) {
        const bool snap_now = snaps && ((nt - 1) % p.dtinv == 0) && hin < ntd;
        const bool sample = c->prof_stride > 0 && (nt % c->prof_stride) == 0;
        const int fhin = (fused && snap_now) ? hin : -1;
        pt.base = (fhin >= 0 && !f16s && !in_stress) ? (float *)((char *)c->snap.p + (size_t)hin * c->snap_bytes)
                                                     : nullptr;
        Lr.nt_cur = nt;
        {
            KTimer t(c, 0, sample);
            Lr.rec_mode = seis_fused ? 1 : 0;
            Lr.v_step(0, snap_now ? 1 : 0, fhin);
            Lr.rec_mode = 0;
        }
        if (force) {
            launch_dep(c->st, c->pdl, k_inject_v_fwd<T>, dim3(nshots), dim3(32), 0, c->g, Lr.S, Lr.M, Lr.src, nt, c->psv && !c->ac ? 1 : (c->ac ? 1 : 0),
                                                        c->sh);
            c->launches++;
        }
        {
            KTimer t(c, 1, sample);
            Lr.s_step(fhin);
        }
        Lr.post_fwd(nt, c->psv != 0, pt);
        if (snap_now && fused) {
            if (f16s && !in_stress && (p.free_surf || c->psv)) {
                const int4 patched = make_int4(pt.c_sxx, pt.c_syy, pt.c_sp, pt.c_syz);
                launch_dep(c->st, c->pdl, k_snap_fix16<T>, dim3(segs + std::max(1, p.max_src), 1, nshots), dim3(32),
                           0, c->g, Lr.S, sn, hin, Lr.src, p.free_surf ? 1 : 0, patched);
                c->launches++;
            }
            hin++;
        } else if (snap_now) {
            KTimer t(c, 2, sample);
            if (f16s) {
                launch_dep(c->st, c->pdl, k_snap_seg16<T>, dim3(segs, (p.ny + 7) / 8, nshots), dim3(32, 8), 0, c->g,
                           Lr.S, sn, hin);
                c->launches++;
            } else if (p.snap_format == 0) {
                launch_dep(c->st, c->pdl, k_snap_store<T>, dim3(Lr.grd), dim3(Lr.blk), 0, c->g, Lr.S, sn, hin);
                c->launches++;
            } else {
                launch_dep(c->st, c->pdl, k_snap_absmax<T>, dim3(Lr.grd), dim3(Lr.blk), 0, c->g, Lr.S, sn, hin);
                launch_dep(c->st, c->pdl, k_snap_quant<T>, dim3(Lr.grd), dim3(Lr.blk), 0, c->g, Lr.S, sn, hin);
                c->launches += 2;
            }
            hin++;
        }
    }
    };
    // the source rows are launch parameters of the stress kernels: part of the captured sequence
    if (int rc = run_loop(c, c->gfwd, loop_key(c, {0, nshots, snaps, nsteps, force, fused, Lr.src_j0, Lr.src_j1,
                                                    seis_fused, Lr.rec_j0, Lr.rec_j1}),
                          enqueue))
        return rc;
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(c->ev1));
    CK(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    collect_kernel_times(c);
    int bad = 0;
    CK(cudaMemcpy(&bad, c->bad.p, 4, cudaMemcpyDeviceToHost));
    c->snaps_valid = snaps && nsteps == p.nt;
    c->fwd_nshots = nshots;
    if (bad >= 16) return pipeline_timeout(c, bad);
    if (bad) return fail(c, IFOS_ERR_UNSTABLE, "simulation is unstable (NaN at the grid centre)");
    return IFOS_OK;
}

template <typename T>
static int adjoint_t(ifos_ctx *c, int nshots) {
    const ifos_params &p = c->p;
    Launcher<T> Lr(c, nshots);
    // P-SV elastic / viscoelastic without the pressure residual source: the
    // stress kernel applies the free surface (no surface kernel)
    Lr.fsurf = (c->pipe && c->psv && !c->ac && !c->sh && p.free_surf && p.adjoint_type != 4) ? 1 : 0;
    if (int rc = zero_state<T>(c, nshots)) return rc;
    const long long N = (long long)p.nx * p.ny;
    CK(cudaMemsetAsync(c->gacc.p, 0, (size_t)nshots * 5 * N * 4, c->st));
    if (c->gacc64.p) CK(cudaMemsetAsync(c->gacc64.p, 0, (size_t)nshots * 5 * N * 8, c->st));
    CK(cudaMemsetAsync(c->bad.p, 0, 4, c->st));
    KSnap sn = ksnap(c);
    KGrad gr{(float *)c->gacc.p, (float *)c->gout.p, N, (double *)c->gacc64.p};
    const int ntd = p.nt / p.dtinv;
    const int mr = std::max(1, p.max_rec);
    dim3 gr_rec((mr + 127) / 128, nshots);
    // P-SV (elastic or viscoelastic) on the pipelined path: the velocity op
    // adds the residual sources itself
    const bool rec_ok = Lr.receiver_rows();
    const bool inj_fused = std::is_same<T, float>::value && c->pipe && c->psv && !c->ac && !c->sh &&
                           p.adjoint_type >= 1 && p.adjoint_type <= 3 && rec_ok;
    CK(cudaEventRecord(c->ev0, c->st));
    auto enqueue = [&]() {
    int hin_a = 1;
    for (int nt = 1; nt <= p.nt; nt++) {
        const bool sample = c->prof_stride > 0 && (nt % c->prof_stride) == 0;
        Lr.nt_cur = nt;
        {
            KTimer t(c, 0, sample);
            Lr.rec_mode = inj_fused ? 2 : 0;
            Lr.v_step(1, 0);
            Lr.rec_mode = 0;
        }
        if (!inj_fused && ((c->psv && p.adjoint_type >= 1 && p.adjoint_type <= 3) || c->sh)) {
            launch_dep(c->st, c->pdl, k_inject_v_adj<T>, dim3(gr_rec), dim3(128), 0, c->g, Lr.S, Lr.rec, nt, c->psv ? 1 : 0, c->sh && !c->ac);
            c->launches++;
        }
        const int fstep = p.nt - nt + 1;  // forward step this adjoint step meets
        const bool snap_step = (fstep - 1) % p.dtinv == 0;
        {
            KTimer t(c, 1, sample);
            Lr.s_step();
        }
        Lr.post_adj(nt, p.adjoint_type == 4);
        if (snap_step) {
            KTimer t(c, 3, sample);
            bool pairs = false;
            if constexpr (std::is_same<T, float>::value) {
                const bool f16s = p.snap_format == IFOS_SNAP_F16S, i16s = p.snap_format == IFOS_SNAP_I16S;
                if ((p.snap_format == IFOS_SNAP_F32 || f16s || i16s) && p.nx % 2 == 0) {
                    const dim3 gc((unsigned)((p.nx / 2 + 127) / 128), (unsigned)p.ny, (unsigned)nshots);
                    const int h = ntd - hin_a;
                    auto corr = [&](auto kern) {
                        launch_dep(c->st, c->pdl, kern, dim3(gc), dim3(128), 0, c->g, Lr.S, Lr.M, sn, gr, h);
                    };
                    if (gr.acc64) {  // the sums in double (grad_acc64)
                        if (f16s) {
                            if (c->ac) corr(k_correlate_pairs<1, 0, 1, 1, true>);
                            else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 1, true>);
                            else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 1, true>);
                            else corr(k_correlate_pairs<0, 1, 0, 1, true>);
                        } else if (i16s) {
                            if (c->ac) corr(k_correlate_pairs<1, 0, 1, 2, true>);
                            else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 2, true>);
                            else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 2, true>);
                            else corr(k_correlate_pairs<0, 1, 0, 2, true>);
                        } else {
                            if (c->ac) corr(k_correlate_pairs<1, 0, 1, 0, true>);
                            else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 0, true>);
                            else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 0, true>);
                            else corr(k_correlate_pairs<0, 1, 0, 0, true>);
                        }
                    } else if (f16s) {
                        if (c->ac) corr(k_correlate_pairs<1, 0, 1, 1>);
                        else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 1>);
                        else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 1>);
                        else corr(k_correlate_pairs<0, 1, 0, 1>);
                    } else if (i16s) {
                        if (c->ac) corr(k_correlate_pairs<1, 0, 1, 2>);
                        else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 2>);
                        else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 2>);
                        else corr(k_correlate_pairs<0, 1, 0, 2>);
                    } else {
                        if (c->ac) corr(k_correlate_pairs<1, 0, 1, 0>);
                        else if (c->psv && c->sh) corr(k_correlate_pairs<1, 1, 0, 0>);
                        else if (c->psv) corr(k_correlate_pairs<1, 0, 0, 0>);
                        else corr(k_correlate_pairs<0, 1, 0, 0>);
                    }
                    pairs = true;
                }
            }
            if (!pairs)
                launch_dep(c->st, c->pdl, k_correlate<T>, dim3(Lr.grd), dim3(Lr.blk), 0, c->g, Lr.S, Lr.M, sn, gr, ntd - hin_a, c->psv, c->sh,
                                                            c->ac);
            c->launches++;
            hin_a++;
        }
    }
    launch_dep(c->st, c->pdl, k_assemble<T>, dim3(Lr.grd), dim3(Lr.blk), 0, c->g, Lr.M, gr, c->psv, c->sh, c->ac);
    c->launches++;
    };
    if (int rc = run_loop(c, c->gadj, loop_key(c, {1, nshots, inj_fused, Lr.rec_j0, Lr.rec_j1}), enqueue))
        return rc;
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(c->ev1));
    CK(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    collect_kernel_times(c);
    int bad = 0;
    CK(cudaMemcpy(&bad, c->bad.p, 4, cudaMemcpyDeviceToHost));
    if (bad >= 16) return pipeline_timeout(c, bad);
    return IFOS_OK;
}

// Orders the context's stream after the asynchronous fetches still reading
// the seismogram (sec) or gradient (grads) buffers, before work that
// overwrites them; the host does not wait.
static int order_after_fetches(ifos_ctx *c, bool sec, bool grads) {
    if (sec && c->sec_pending) {
        CK(cudaStreamWaitEvent(c->st, c->ev_sec_done, 0));
        c->sec_pending = false;
    }
    if (grads && c->grad_pending) {
        CK(cudaStreamWaitEvent(c->st, c->ev_grad_done, 0));
        c->grad_pending = false;
    }
    return IFOS_OK;
}

extern "C" int ifos_forward(ifos_ctx *c, int nshots, int store, float *sections) {
    if (!c) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed");
    if (int rc = order_after_fetches(c, true, false)) return rc;
    int rc = c->dbl ? forward_t<double>(c, nshots, store, c->p.nt) : forward_t<float>(c, nshots, store, c->p.nt);
    if (rc == IFOS_OK && sections) rc = ifos_fetch_sections(c, nshots, sections);
    return rc;
}

extern "C" int ifos_stage_adjoint(ifos_ctx *c, int nshots, const float *adj) {
    if (!c) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots || !adj) return fail(c, IFOS_ERR_ARG, "bad adjoint staging");
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed");
    CK(cudaMemcpyAsync(c->adj.p, adj, (size_t)nshots * 3 * std::max(1, c->p.max_rec) * c->p.nt * 4,
                       cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->adj_staged = true;
    return IFOS_OK;
}

extern "C" int ifos_adjoint(ifos_ctx *c, int nshots, const float *adj, float *grads) {
    if (!c) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    if (!c->snaps_valid || nshots > c->fwd_nshots)
        return fail(c, IFOS_ERR_STATE, "adjoint needs a preceding forward run that stored snapshots");
    if (adj) {
        if (int rc = ifos_stage_adjoint(c, nshots, adj)) return rc;
    } else if (!c->adj_staged) {
        return fail(c, IFOS_ERR_STATE, "no adjoint sources staged");
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, IFOS_ERR_CUDA, "cudaSetDevice failed");
    if (int rc = order_after_fetches(c, false, true)) return rc;
    int rc = c->dbl ? adjoint_t<double>(c, nshots) : adjoint_t<float>(c, nshots);
    if (rc == IFOS_OK && grads) rc = ifos_fetch_grads(c, nshots, grads);
    return rc;
}

extern "C" int ifos_fetch_sections(ifos_ctx *c, int nshots, float *sections) {
    if (!c || !sections) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(sections, c->sec.p, (size_t)nshots * IFOS_NS * std::max(1, c->p.max_rec) * c->p.nt * 4,
                       cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_fetch_grads(ifos_ctx *c, int nshots, float *grads) {
    if (!c || !grads) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(grads, c->gout.p, (size_t)nshots * IFOS_NG * c->p.nx * c->p.ny * 4, cudaMemcpyDeviceToHost,
                       c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

// An asynchronous device-to-host copy on the context's copy stream, after the
// work already on its stream; *done marks its completion.
static int fetch_async(ifos_ctx *c, void *dst, const void *src, size_t bytes, cudaEvent_t done, bool *pending) {
    CK(cudaEventRecord(c->ev_ready, c->st));
    CK(cudaStreamWaitEvent(c->cp_st, c->ev_ready, 0));
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->cp_st));
    CK(cudaEventRecord(done, c->cp_st));
    *pending = true;
    return IFOS_OK;
}

static int copy_stream(ifos_ctx *c) {
    if (c->cp_st) return IFOS_OK;
    CK(cudaStreamCreateWithFlags(&c->cp_st, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&c->ev_ready, &c->ev_sec_done, &c->ev_grad_done})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return IFOS_OK;
}

extern "C" int ifos_fetch_sections_async(ifos_ctx *c, int nshots, float *sections) {
    if (!c || !sections) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    if (int rc = copy_stream(c)) return rc;
    return fetch_async(c, sections, c->sec.p, (size_t)nshots * IFOS_NS * std::max(1, c->p.max_rec) * c->p.nt * 4,
                       c->ev_sec_done, &c->sec_pending);
}

extern "C" int ifos_fetch_grads_async(ifos_ctx *c, int nshots, float *grads) {
    if (!c || !grads) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    if (int rc = copy_stream(c)) return rc;
    return fetch_async(c, grads, c->gout.p, (size_t)nshots * IFOS_NG * c->p.nx * c->p.ny * 4, c->ev_grad_done,
                       &c->grad_pending);
}

extern "C" int ifos_fetch_wait(ifos_ctx *c) {
    if (!c) return IFOS_ERR_ARG;
    if (!c->cp_st) return IFOS_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->cp_st));
    c->sec_pending = c->grad_pending = false;
    return IFOS_OK;
}

extern "C" int ifos_host_alloc(size_t bytes, void **out) {
    if (!out) return IFOS_ERR_ARG;
    *out = nullptr;
    const cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        ifos_internal_set_error(std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
        return IFOS_ERR_NOMEM;
    }
    return IFOS_OK;
}

extern "C" int ifos_host_free(void *p) {
    if (!p) return IFOS_OK;
    const cudaError_t e = cudaFreeHost(p);
    if (e != cudaSuccess) {
        ifos_internal_set_error(std::string("cudaFreeHost: ") + cudaGetErrorString(e));
        return IFOS_ERR_CUDA;
    }
    return IFOS_OK;
}

extern "C" int ifos_grad_sum(ifos_ctx *c, int nshots, float *out) {
    if (!c || !out) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    const long long N = (long long)c->p.nx * c->p.ny;
    void *tmp = nullptr;
    if (int rc = scratch(c, (size_t)5 * N * 4, &tmp)) return rc;
    k_grad_sum<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>((const float *)c->gout.p, nshots, N, (float *)tmp);
    c->launches++;
    CK(cudaMemcpyAsync(out, tmp, (size_t)5 * N * 4, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

template <typename T>
__global__ void k_fields_out(KGrid g, KState<T> S, int slot, const int *ids, int nid, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    const long long c = pidx(g, j, i), q = (long long)(j - 1) * g.nx + (i - 1), n = (long long)g.nx * g.ny;
    for (int k = 0; k < nid; k++) out[k * n + q] = ids[k] >= 0 ? (float)fieldp(S, slot, ids[k])[c] : 0.0f;
}

template <typename T>
static int fetch_fields_t(ifos_ctx *c, int slot, float *fields) {
    const long long N = (long long)c->p.nx * c->p.ny;
    void *tmp = nullptr;
    const size_t fb = (size_t)IFOS_NF * N * 4;
    if (int rc = scratch(c, fb + 256, &tmp)) return rc;
    int *ids = (int *)((char *)tmp + fb);
    int idh[IFOS_NF];
    const int map[IFOS_NF] = {P_VX, P_VY, P_SXX, P_SYY, P_SXY, P_VXP1, P_VYP1, P_VZ, P_SXZ, P_SYZ, P_VZP1, P_SP};
    for (int k = 0; k < IFOS_NF; k++) idh[k] = c->off[map[k]] >= 0 ? map[k] : -1;
    CK(cudaMemcpyAsync(ids, idh, sizeof idh, cudaMemcpyHostToDevice, c->st));
    dim3 blk(32, 8), grd((c->p.nx + 31) / 32, (c->p.ny + 7) / 8);
    k_fields_out<T><<<grd, blk, 0, c->st>>>(c->g, kstate<T>(c), slot, ids, IFOS_NF, (float *)tmp);
    c->launches++;
    CK(cudaMemcpyAsync(fields, tmp, fb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_fetch_fields(ifos_ctx *c, int slot, float *fields) {
    if (!c || !fields) return IFOS_ERR_ARG;
    if (slot < 0 || slot >= c->p.max_shots) return fail(c, IFOS_ERR_ARG, "slot out of range");
    CK(cudaSetDevice(c->device));
    return c->dbl ? fetch_fields_t<double>(c, slot, fields) : fetch_fields_t<float>(c, slot, fields);
}

template <typename T>
__global__ void k_snap_out(KSnap sn, int slot, int snap, float *out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= sn.n) return;
    for (int k = 0; k < sn.ncomp; k++) out[k * sn.n + q] = (float)snap_load<T>(sn, slot, snap, k, q);
}

extern "C" int ifos_fetch_snapshot(ifos_ctx *c, int slot, int index, float *out) {
    if (!c || !out) return IFOS_ERR_ARG;
    if (!c->with_snap) return fail(c, IFOS_ERR_STATE, "context has no snapshots");
    if (slot < 0 || slot >= c->p.max_shots || index < 0 || index >= c->p.nt / c->p.dtinv)
        return fail(c, IFOS_ERR_ARG, "slot or snapshot index out of range");
    CK(cudaSetDevice(c->device));
    const long long N = (long long)c->p.nx * c->p.ny;
    const size_t bytes = (size_t)c->ncomp * N * 4;
    void *tmp = nullptr;
    if (int rc = scratch(c, bytes, &tmp)) return rc;
    const unsigned nb = (unsigned)((N + 255) / 256);
    if (c->dbl) k_snap_out<double><<<nb, 256, 0, c->st>>>(ksnap(c), slot, index, (float *)tmp);
    else k_snap_out<float><<<nb, 256, 0, c->st>>>(ksnap(c), slot, index, (float *)tmp);
    c->launches++;
    CK(cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_forward_steps(ifos_ctx *c, int nsteps, float *fields) {
    if (!c) return IFOS_ERR_ARG;
    if (nsteps < 1 || nsteps > c->p.nt) return fail(c, IFOS_ERR_ARG, "nsteps out of range");
    CK(cudaSetDevice(c->device));
    if (int rc = order_after_fetches(c, true, false)) return rc;
    int rc = c->dbl ? forward_t<double>(c, 1, 0, nsteps) : forward_t<float>(c, 1, 0, nsteps);
    if (rc == IFOS_OK && fields) rc = ifos_fetch_fields(c, 0, fields);
    return rc;
}

extern "C" int ifos_dot_f64(ifos_ctx *c, const float *a, const float *b, size_t n, int device_ptrs, double *out) {
    if (!c || !a || !out) return IFOS_ERR_ARG;
    CK(cudaSetDevice(c->device));
    const float *da = a, *db = b;
    DevBuf ta, tb;
    if (!device_ptrs) {
        if (int rc = dev_alloc(c, ta, n * 4 + 4)) return rc;
        CK(cudaMemcpyAsync(ta.p, a, n * 4, cudaMemcpyHostToDevice, c->st));
        da = (const float *)ta.p;
        if (b) {
            if (int rc = dev_alloc(c, tb, n * 4 + 4)) {
                dev_free(ta);
                return rc;
            }
            CK(cudaMemcpyAsync(tb.p, b, n * 4, cudaMemcpyHostToDevice, c->st));
            db = (const float *)tb.p;
        }
    }
    const int nb = 592;  // 4 blocks per SM on 148 SMs; <= 1024 partials
    k_dot_partial<<<nb, 256, 0, c->st>>>(da, db, (long long)n, (double *)c->dot_partial.p);
    k_dot_final<<<1, 256, 0, c->st>>>((const double *)c->dot_partial.p, nb, (double *)c->dot_out.p);
    c->launches += 2;
    cudaError_t e = cudaMemcpyAsync(out, c->dot_out.p, sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dev_free(ta);
    dev_free(tb);
    if (e != cudaSuccess) return fail(c, IFOS_ERR_CUDA, cudaGetErrorString(e));
    return IFOS_OK;
}

// Vector updates of the L-BFGS two-loop recursion (src/LBFGS.c:285-321), each
// the reference's float operation: mode 0 x = x - a*y, mode 1 x = a*y,
// mode 2 x = x + y*a (a: alpha, h0, or alpha - beta, rounded to float).
__global__ void k_lbfgs_vec(float *x, const float *y, float a, long long n, int mode) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        if (mode == 0) x[k] = x[k] - a * y[k];
        else if (mode == 1) x[k] = a * y[k];
        else x[k] = x[k] + y[k] * a;
    }
}

// sum(a*b) in double over n device floats, on the context's stream, to the host
static int dot_dev(ifos_ctx *c, const float *a, const float *b, long long n, double *out) {
    const int nb = 592;
    k_dot_partial<<<nb, 256, 0, c->st>>>(a, b, n, (double *)c->dot_partial.p);
    k_dot_final<<<1, 256, 0, c->st>>>((const double *)c->dot_partial.p, nb, (double *)c->dot_out.p);
    c->launches += 2;
    CK(cudaMemcpyAsync(out, c->dot_out.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_lbfgs_core(ifos_ctx *c, int iteration, int n_lbfgs, size_t npar, const float *s, const float *y,
                               float *rho, float *q, float *alpha, float *r, int device_ptrs) {
    if (!c || !s || !y || !rho || !q || !alpha || !r || n_lbfgs < 1 || iteration < 2 || npar < 1)
        return IFOS_ERR_ARG;
    CK(cudaSetDevice(c->device));
    const long long n = (long long)npar;
    const size_t vb = npar * sizeof(float), mb = (size_t)n_lbfgs * vb;
    DevBuf ts, ty, tq, tr;
    struct Frees {  // the staging copies of host arrays, freed on every return
        DevBuf *b[4];
        ~Frees() {
            for (DevBuf *x : b) dev_free(*x);
        }
    } frees{{&ts, &ty, &tq, &tr}};
    const float *ds = s, *dy = y;
    float *dq = q, *dr = r;
    if (!device_ptrs) {
        int rc = dev_alloc(c, ts, mb);
        if (!rc) rc = dev_alloc(c, ty, mb);
        if (!rc) rc = dev_alloc(c, tq, vb);
        if (!rc) rc = dev_alloc(c, tr, vb);
        if (rc) return rc;
        CK(cudaMemcpyAsync(ts.p, s, mb, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(ty.p, y, mb, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(tq.p, q, vb, cudaMemcpyHostToDevice, c->st));
        ds = (const float *)ts.p;
        dy = (const float *)ty.p;
        dq = (float *)tq.p;
        dr = (float *)tr.p;
    }
    auto row = [&](const float *m, int w) { return m + (size_t)(w - 1) * npar; };  // pair w = 1..n_lbfgs
    const unsigned nb = 4 * (unsigned)c->num_sms;
    int rc = IFOS_OK;
    int m = iteration - n_lbfgs;
    if (m < 1) m = 1;
    // H0 and rho of the newest pair (src/LBFGS.c:240-256)
    int w = (iteration - 1) % n_lbfgs;
    if (w == 0) w = n_lbfgs;
    double d1 = 0.0, d2 = 0.0;
    if (!rc) rc = dot_dev(c, row(dy, w), row(ds, w), n, &d1);
    if (!rc) rc = dot_dev(c, row(dy, w), row(dy, w), n, &d2);
    const float buf1 = (float)d1, buf2 = (float)d2;
    rho[w - 1] = 1 / buf1;
    const float h0 = buf1 / buf2;
    // loop 1, newest pair first (:271-290)
    for (int v = iteration - 1; v >= m && !rc; v--) {
        int wv = v % n_lbfgs;
        if (wv == 0) wv = n_lbfgs;
        double sq = 0.0;
        rc = dot_dev(c, row(ds, wv), dq, n, &sq);
        alpha[wv - 1] = (float)((double)rho[wv - 1] * sq);
        if (!rc) {
            k_lbfgs_vec<<<nb, 256, 0, c->st>>>(dq, row(dy, wv), alpha[wv - 1], n, 0);
            c->launches++;
        }
    }
    // r = H0 q (:295-297), then loop 2, oldest pair first (:302-321)
    if (!rc) {
        k_lbfgs_vec<<<nb, 256, 0, c->st>>>(dr, dq, h0, n, 1);
        c->launches++;
    }
    for (int v = m; v <= iteration - 1 && !rc; v++) {
        int wv = v % n_lbfgs;
        if (wv == 0) wv = n_lbfgs;
        double yr = 0.0;
        rc = dot_dev(c, row(dy, wv), dr, n, &yr);
        const float beta = (float)((double)rho[wv - 1] * yr);
        if (!rc) {
            k_lbfgs_vec<<<nb, 256, 0, c->st>>>(dr, row(ds, wv), alpha[wv - 1] - beta, n, 2);
            c->launches++;
        }
    }
    if (!rc && !device_ptrs) {
        cudaError_t e = cudaMemcpyAsync(q, dq, vb, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(r, dr, vb, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess) rc = fail(c, IFOS_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess) rc = fail(c, IFOS_ERR_CUDA, cudaGetErrorString(e));
    }
    return rc;
}

extern "C" int ifos_calc_res(ifos_ctx *c, int ntr, const float *obs, const float *syn, float *diff, double *l2,
                             double *energy) {
    if (!c || !obs || !syn || ntr < 1) return IFOS_ERR_ARG;
    CK(cudaSetDevice(c->device));
    const int ns = c->p.nt;
    const size_t bytes = (size_t)ntr * ns * 4, tb = (size_t)2 * ntr * sizeof(double);
    void *scr = nullptr;
    if (int rc = scratch(c, tb + 3 * bytes, &scr)) return rc;
    double *tr = (double *)scr;
    float *d_obs = (float *)((char *)scr + tb), *d_syn = d_obs + (size_t)ntr * ns, *d_diff = d_syn + (size_t)ntr * ns;
    CK(cudaMemcpyAsync(d_obs, obs, bytes, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(d_syn, syn, bytes, cudaMemcpyHostToDevice, c->st));
    k_calc_res<<<(ntr + 127) / 128, 128, 0, c->st>>>(d_obs, d_syn, d_diff, ntr, ns, c->p.dt, tr, tr + ntr);
    c->launches++;
    std::vector<double> h((size_t)2 * ntr);
    if (diff) CK(cudaMemcpyAsync(diff, d_diff, bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(h.data(), tr, tb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    double a = 0, b = 0;
    for (int k = 0; k < ntr; k++) {
        a += h[k];
        b += h[ntr + k];
    }
    if (l2) *l2 = a;
    if (energy) *energy = b;
    return IFOS_OK;
}

// The adjoint sources of slots [0, nshots) from their synthetic seismograms
// (kept on the device by ifos_forward) and the observed ones: per active
// component the residual of calc_res (src/calc_res.c, LNORM=2) is written
// time-reversed into the staged adjoint sources, and the FP64 misfit and
// energy are summed per slot.
extern "C" int ifos_residual_adjoint(ifos_ctx *c, int nshots, const float *obs, const int *kill,
                                     const ifos_window *win, double *l2, double *energy) {
    if (!c || !obs) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    if (c->fwd_nshots < nshots) return fail(c, IFOS_ERR_STATE, "no forward seismograms for these slots");
    CK(cudaSetDevice(c->device));
    const ifos_params &p = c->p;
    const int mr = std::max(1, p.max_rec), ns = p.nt;
    // adjoint-source component -> seismogram plane (-1 unused)
    int plane[3] = {-1, -1, -1};
    if (c->ac || (c->psv && p.adjoint_type == 4)) {
        plane[2] = IFOS_S_P;
    } else {
        if (c->psv && (p.adjoint_type == 1 || p.adjoint_type == 3)) plane[0] = IFOS_S_VX;
        if (c->psv && (p.adjoint_type == 1 || p.adjoint_type == 2)) plane[1] = IFOS_S_VY;
        if (c->sh) plane[2] = IFOS_S_VZ;
    }
    const size_t comp = (size_t)mr * ns, obs_bytes = (size_t)nshots * 3 * comp * 4;
    const size_t tb = (size_t)nshots * 3 * mr * 2 * sizeof(double);
    const size_t kb = kill ? ((size_t)nshots * mr * sizeof(int) + 255) / 256 * 256 : 0;
    int np = 0;
    if (win) {
        if (!win->picks || win->tw_ind < 0 || win->tw_ind > 2) return fail(c, IFOS_ERR_ARG, "bad time window");
        np = win->tw_ind == 0 ? 1 : (win->tw_ind == 1 ? 3 : 6);
    }
    const size_t pb = ((size_t)nshots * np * mr * sizeof(float) + 255) / 256 * 256;
    void *scr = nullptr;
    if (int rc = scratch(c, tb + kb + pb + obs_bytes, &scr)) return rc;
    double *tr = (double *)scr;
    int *d_kill = kill ? (int *)((char *)scr + tb) : nullptr;
    float *d_picks = win ? (float *)((char *)scr + tb + kb) : nullptr;
    float *d_obs = (float *)((char *)scr + tb + kb + pb);
    CK(cudaMemcpyAsync(d_obs, obs, obs_bytes, cudaMemcpyHostToDevice, c->st));
    if (kill) CK(cudaMemcpyAsync(d_kill, kill, (size_t)nshots * mr * sizeof(int), cudaMemcpyHostToDevice, c->st));
    if (win)
        CK(cudaMemcpyAsync(d_picks, win->picks, (size_t)nshots * np * mr * sizeof(float), cudaMemcpyHostToDevice,
                           c->st));
    CK(cudaMemsetAsync(c->adj.p, 0, obs_bytes, c->st));
    CK(cudaMemsetAsync(tr, 0, tb, c->st));
    for (int s = 0; s < nshots; s++) {
        const int ntr = c->ntr_h[s];
        if (ntr < 1) continue;
        for (int k = 0; k < 3; k++) {
            if (plane[k] < 0) continue;
            const float *syn = (const float *)c->sec.p + ((size_t)s * IFOS_NS + plane[k]) * comp;
            float *adj = (float *)c->adj.p + ((size_t)s * 3 + k) * comp;
            double *t = tr + ((size_t)s * 3 + k) * mr * 2;
            KWindow kw{};
            if (win) {
                kw.picks = d_picks + (size_t)s * np * mr;
                kw.stride = mr;
                kw.tw_ind = win->tw_ind;
                kw.gamma = win->gamma;
                kw.twl_plus = win->twl_plus;
                kw.twl_minus = win->twl_minus;
            }
            k_calc_res<<<(ntr + 127) / 128, 128, 0, c->st>>>(d_obs + ((size_t)s * 3 + k) * comp, syn, adj, ntr, ns,
                                                             p.dt, t, t + mr, d_kill ? d_kill + (size_t)s * mr : nullptr,
                                                             kw);
            c->launches++;
        }
    }
    std::vector<double> h(tb / sizeof(double));
    CK(cudaMemcpyAsync(h.data(), tr, tb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int s = 0; s < nshots; s++) {
        double a = 0, b = 0;
        for (int k = 0; k < 3; k++) {
            const double *t = h.data() + ((size_t)s * 3 + k) * mr * 2;
            for (int r = 0; r < c->ntr_h[s]; r++) {
                a += t[r];
                b += t[mr + r];
            }
        }
        if (l2) l2[s] = a;
        if (energy) energy[s] = b;
    }
    c->adj_staged = true;
    return IFOS_OK;
}

extern "C" double ifos_last_ms(const ifos_ctx *c) { return c ? c->last_ms : 0.0; }
extern "C" long long ifos_launch_count(const ifos_ctx *c) { return c ? c->launches : 0; }
extern "C" int ifos_status(ifos_ctx *c) {
    if (!c) return IFOS_ERR_ARG;
    int code = c->last_code;
    c->last_code = IFOS_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return IFOS_ERR_CUDA;
    for (cudaStream_t s : {c->st, c->cp_st}) {
        if (!s) continue;
        const cudaError_t e = cudaStreamQuery(s);
        if (e != cudaSuccess && e != cudaErrorNotReady) {
            c->err = std::string("stream failed: ") + cudaGetErrorString(e);
            code = IFOS_ERR_CUDA;
        }
    }
    return code;
}

extern "C" int ifos_sync(ifos_ctx *c) {
    if (!c) return IFOS_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_trkill_table(ifos_ctx *c, int ntr, const int *rx, const int *ry, int nsrc, const float *sx,
                                 const float *sy, float lower, float upper, int *killtable) {
    if (!c) return IFOS_ERR_ARG;
    if (ntr < 0 || nsrc < 0 || (ntr && (!rx || !ry)) || (nsrc && (!sx || !sy)) || (ntr && nsrc && !killtable))
        return fail(c, IFOS_ERR_ARG, "bad trace-kill arguments");
    if (!ntr || !nsrc) return IFOS_OK;
    CK(cudaSetDevice(c->device));
    DevBuf b_rx, b_ry, b_sx, b_sy, b_k;
    const size_t nk = (size_t)ntr * nsrc;
    int rc = IFOS_OK;
    if ((rc = dev_alloc(c, b_rx, ntr * sizeof(int))) || (rc = dev_alloc(c, b_ry, ntr * sizeof(int))) ||
        (rc = dev_alloc(c, b_sx, nsrc * sizeof(float))) || (rc = dev_alloc(c, b_sy, nsrc * sizeof(float))) ||
        (rc = dev_alloc(c, b_k, nk * sizeof(int)))) {
        dev_free(b_rx), dev_free(b_ry), dev_free(b_sx), dev_free(b_sy), dev_free(b_k);
        return rc;
    }
    cudaError_t e = cudaMemcpyAsync(b_rx.p, rx, ntr * sizeof(int), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_ry.p, ry, ntr * sizeof(int), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_sx.p, sx, nsrc * sizeof(float), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_sy.p, sy, nsrc * sizeof(float), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_k.p, killtable, nk * sizeof(int), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        k_trkill<<<(unsigned)((nk + 255) / 256), 256, 0, c->st>>>(ntr, (const int *)b_rx.p, (const int *)b_ry.p, nsrc,
                                                                  (const float *)b_sx.p, (const float *)b_sy.p,
                                                                  c->p.dh, lower, upper, (int *)b_k.p);
        c->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(killtable, b_k.p, nk * sizeof(int), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dev_free(b_rx), dev_free(b_ry), dev_free(b_sx), dev_free(b_sy), dev_free(b_k);
    if (e != cudaSuccess) return fail(c, IFOS_ERR_CUDA, std::string("ifos_trkill_table: ") + cudaGetErrorString(e));
    return IFOS_OK;
}

extern "C" int ifos_time_window(ifos_ctx *c, int ntr, int ns, float *sections, int tw_ind, const float *picks,
                                float gamma, float twl_plus, float twl_minus, unsigned char *mask) {
    if (!c) return IFOS_ERR_ARG;
    if (ntr < 0 || ns < 0 || tw_ind < 0 || tw_ind > 2 || (ntr && ns && (!sections || !picks)))
        return fail(c, IFOS_ERR_ARG, "bad time-window arguments");
    if (!ntr || !ns) return IFOS_OK;
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)ntr * ns;
    const int np = tw_ind == 1 ? 3 : (tw_ind == 2 ? 6 : 1);
    DevBuf b_s, b_p, b_m;
    int rc = IFOS_OK;
    if ((rc = dev_alloc(c, b_s, n * sizeof(float))) || (rc = dev_alloc(c, b_p, (size_t)np * ntr * sizeof(float))) ||
        (mask && (rc = dev_alloc(c, b_m, n)))) {
        dev_free(b_s), dev_free(b_p), dev_free(b_m);
        return rc;
    }
    cudaError_t e = cudaMemcpyAsync(b_s.p, sections, n * sizeof(float), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b_p.p, picks, (size_t)np * ntr * sizeof(float), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        k_time_window<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>((float *)b_s.p, ntr, ns, tw_ind,
                                                                      (const float *)b_p.p, c->p.dt, gamma, twl_plus,
                                                                      twl_minus, (unsigned char *)b_m.p);
        c->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(sections, b_s.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess && mask) e = cudaMemcpyAsync(mask, b_m.p, n, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    dev_free(b_s), dev_free(b_p), dev_free(b_m);
    if (e != cudaSuccess) return fail(c, IFOS_ERR_CUDA, std::string("ifos_time_window: ") + cudaGetErrorString(e));
    return IFOS_OK;
}

// The parabola fit of the line search (src/calc_opt_step.c:73-112): the
// misfits of the three test steps define a + b e + c e^2, solved by Gaussian
// elimination without pivoting in the order of src/solvelin.c:55-68; the
// step is the extremum -b/(2c) with the reference's clamps.
template <typename T>
static float opt_step_t(const float *l2t, const float *epst) {
    T A[3][3], b[3], x[3];
    for (int i = 0; i < 3; i++) {
        A[i][2] = (T)epst[i] * (T)epst[i];
        A[i][1] = (T)epst[i];
        A[i][0] = (T)1.0;
        b[i] = (T)l2t[i];
    }
    for (int k = 0; k < 2; k++)
        for (int n = k; n < 2; n++) {
            const T a = A[n + 1][k] / A[k][k];
            for (int m = 0; m < 3; m++) A[n + 1][m] = A[n + 1][m] - a * A[k][m];
            b[n + 1] = b[n + 1] - a * b[k];
        }
    for (int k = 2; k >= 0; k--) {
        T c = b[k];
        for (int m = 2; m >= k + 1; m--) c = c - A[k][m] * x[m];
        x[k] = c / A[k][k];
    }
    // the reference divides in double (2.0 is a double literal)
    float opteps = (float)(-(double)x[1] / (2.0 * (double)x[2]));
    if ((2.0 * (double)x[2]) < 0.0 && l2t[1] > l2t[2]) opteps = epst[2];
    if (opteps > epst[2]) opteps = epst[2];
    if (opteps < 0.0f) opteps = epst[0];
    return opteps;
}

extern "C" int ifos_opt_step(const float *l2t, const float *epst, int fp64, float *opteps) {
    if (!l2t || !epst || !opteps) return IFOS_ERR_ARG;
    *opteps = fp64 ? opt_step_t<double>(l2t, epst) : opt_step_t<float>(l2t, epst);
    return IFOS_OK;
}

// The taper matrix of src/taper_grad_shot.c:62-111 (gp x gp floats, row j
// then column i), with the reference's float/double promotions.
static std::vector<float> shot_taper_matrix(float srtradius, int srtshape, float dh, int &gp) {
    gp = (int)(std::ceil(2.0 * srtradius / dh));
    if (gp < 5) gp = 5;
    std::vector<float> m((size_t)gp * gp);
    const float a = 1.0f;
    const float maxrad = (float)std::sqrt(2.0 * srtradius * srtradius);
    for (int j = 1; j <= gp; j++)
        for (int i = 1; i <= gp; i++) {
            const float x = (float)(((float)i - ((float)gp) / 2.0 - 0.5) * dh);
            const float y = (float)(((float)j - ((float)gp) / 2.0 - 0.5) * dh);
            // the reference calls the double sqrt / erf / log on float arguments
            const float rad = (float)std::sqrt((double)(x * x + y * y));
            float v = 0.0f;
            if (srtshape == 1) v = (float)std::erf((double)(a * rad / maxrad));
            else if (rad > 0) v = (float)std::log((double)rad);
            m[(size_t)(j - 1) * gp + (i - 1)] = v;
        }
    // minimum_m / maximum_m of src/util.c:56-90: start at [1][1], then compare
    auto at = [&](int j, int i) -> float & { return m[(size_t)(j - 1) * gp + (i - 1)]; };
    float minm = at(1, 1);
    for (int i = 1; i <= gp; i++)
        for (int j = 1; j <= gp; j++)
            if (i * j != 1 && at(j, i) < minm) minm = at(j, i);
    for (float &v : m) v -= minm;
    const float edge[4] = {at(1, gp / 2), at(gp / 2, 1), at(gp / 2, gp), at(gp, gp / 2)};
    float maxm = edge[0];
    for (int k = 1; k < 4; k++)
        if (edge[k] > maxm) maxm = edge[k];
    for (float &v : m) {
        v /= maxm;
        if (v > 1.0f) v = 1.0f;
    }
    return m;
}

extern "C" int ifos_taper_grad_shot(ifos_ctx *c, int nshots, const float *src_xy, float srtradius, int srtshape,
                                    int filtsize, unsigned planes) {
    if (!c || !src_xy || nshots < 1 || nshots > c->p.max_shots) return IFOS_ERR_ARG;
    if (srtshape != 1 && srtshape != 2) return fail(c, IFOS_ERR_ARG, "SRTSHAPE must be 1 or 2");
    CK(cudaSetDevice(c->device));
    if (int rc = order_after_fetches(c, false, true)) return rc;
    const ifos_params &p = c->p;
    const float dh = p.dh;
    int gp = 0;
    const std::vector<float> mat = shot_taper_matrix(srtradius, srtshape, dh, gp);
    const int ijc = (int)std::ceil((float)gp / 2);
    std::vector<KTaperShot> tp(nshots);
    std::vector<float> mats((size_t)nshots * gp * gp);
    for (int s = 0; s < nshots; s++) {
        KTaperShot &t = tp[s];
        t.i0 = (int)std::floor(src_xy[2 * s] / dh + 0.5);  // iround(srcpos[1][n]/DH)
        t.j0 = (int)std::floor(src_xy[2 * s + 1] / dh + 0.5);
        t.ijc = ijc;
        t.gp = gp;
        t.filtsize = filtsize;
        std::copy(mat.begin(), mat.end(), mats.begin() + (size_t)s * gp * gp);
        // the field's minimum over every cell (1 outside the taper, which is at most 1 inside)
        bool outside = (long long)p.nx * p.ny > 0;
        int inside = 0;
        float minm = 1.0f;
        for (int iy = 1; iy <= gp; iy++)
            for (int ix = 1; ix <= gp; ix++) {
                const int xx = t.i0 + ix - ijc, yy = t.j0 + iy - ijc;
                if (xx < 1 || xx > p.nx || yy < 1 || yy > p.ny) continue;
                inside++;
                const float v = std::min(1.0f, mat[(size_t)(iy - 1) * gp + (ix - 1)]);
                if (v < minm) minm = v;
            }
        outside = inside < p.nx * p.ny;
        float maxm = outside ? 1.0f - minm : -INFINITY;
        for (int iy = 1; iy <= gp; iy++)
            for (int ix = 1; ix <= gp; ix++) {
                const int xx = t.i0 + ix - ijc, yy = t.j0 + iy - ijc;
                if (xx < 1 || xx > p.nx || yy < 1 || yy > p.ny) continue;
                const float v = std::min(1.0f, mat[(size_t)(iy - 1) * gp + (ix - 1)]) - minm;
                if (v > maxm) maxm = v;
            }
        t.minm = minm;
        t.maxm = maxm;
    }
    const size_t tb = ((size_t)nshots * sizeof(KTaperShot) + 255) / 256 * 256;
    void *scr = nullptr;
    if (int rc = scratch(c, tb + mats.size() * 4, &scr)) return rc;
    CK(cudaMemcpyAsync(scr, tp.data(), nshots * sizeof(KTaperShot), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync((char *)scr + tb, mats.data(), mats.size() * 4, cudaMemcpyHostToDevice, c->st));
    const long long N = (long long)p.nx * p.ny;
    k_taper_shot<<<dim3((unsigned)((N + 255) / 256), (unsigned)nshots), 256, 0, c->st>>>(
        (float *)c->gout.p, N, p.nx, p.ny, planes, (const KTaperShot *)scr, (const float *)((char *)scr + tb));
    c->launches++;
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_taper_grad_coeff(ifos_ctx *c, int slot, unsigned planes, const float *coeff) {
    if (!c || !coeff || slot < 0 || slot >= c->p.max_shots) return IFOS_ERR_ARG;
    if (planes >> IFOS_NG) return fail(c, IFOS_ERR_ARG, "planes is a mask over the IFOS_NG gradient planes");
    CK(cudaSetDevice(c->device));
    if (int rc = order_after_fetches(c, false, true)) return rc;
    const long long N = (long long)c->p.nx * c->p.ny;
    void *scr = nullptr;
    if (int rc = scratch(c, (size_t)N * 4, &scr)) return rc;
    CK(cudaMemcpyAsync(scr, coeff, (size_t)N * 4, cudaMemcpyHostToDevice, c->st));
    k_taper_coeff<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>((float *)c->gout.p + (long long)slot * IFOS_NG * N,
                                                                  N, planes, (const float *)scr);
    c->launches++;
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_mat_change_test(ifos_ctx *c, const ifos_mat_change *mc, float *vp, float *vs, float *rho,
                                    const float *g_vp, const float *g_vs, const float *g_rho, const float *vp_start,
                                    const float *vs_start, const float *rho_start, float *vp1, float *vs1,
                                    float *rho1, float *s_lbfgs, float *eps, int *ratio_hit) {
    if (!c || !mc) return IFOS_ERR_ARG;
    const bool ac = c->ac;
    if (!vp || !rho || !g_vp || !g_rho || !vp1 || !rho1 || (!ac && (!vs || !g_vs || !vs1)))
        return fail(c, IFOS_ERR_ARG, "missing model, search-direction or output planes");
    if (mc->limit_update == 1 && (!vp_start || !rho_start || (!ac && !vs_start)))
        return fail(c, IFOS_ERR_ARG, "the limited update needs the start model");
    KMatChange m{};
    m.nx = c->p.nx;
    m.ny = c->p.ny;
    m.n = (long long)m.nx * m.ny;
    m.acoustic = ac ? 1 : 0;
    m.eps_scale = mc->eps_scale;
    m.iter = mc->iter;
    m.itest = mc->itest;
    m.inv_vp_iter = mc->inv_vp_iter;
    m.inv_vs_iter = mc->inv_vs_iter;
    m.inv_rho_iter = mc->inv_rho_iter;
    m.lbfgs_unnormalised = mc->lbfgs_unnormalised;
    m.vp_lower = mc->vp_lower, m.vp_upper = mc->vp_upper;
    m.vs_lower = mc->vs_lower, m.vs_upper = mc->vs_upper;
    m.rho_lower = mc->rho_lower, m.rho_upper = mc->rho_upper;
    m.vp_vs_ratio = mc->vp_vs_ratio;
    m.limit_update = mc->limit_update;
    m.s_vp = mc->s_vp, m.s_vs = mc->s_vs, m.s_rho = mc->s_rho;
    m.lbfgs_npar = s_lbfgs ? std::max(0, std::min(3, mc->lbfgs_npar)) : 0;
    m.vs_avg = mc->vs_avg, m.rho_avg = mc->rho_avg, m.vp_avg = mc->vp_avg;
    CK(cudaSetDevice(c->device));
    const long long N = m.n;
    const size_t pb = (size_t)N * 4;
    void *scr = nullptr;
    if (int rc = scratch(c, 15 * pb + 64, &scr)) return rc;
    float *d = (float *)scr;
    float *d_vp = d, *d_vs = d + N, *d_rho = d + 2 * N, *d_gvp = d + 3 * N, *d_gvs = d + 4 * N, *d_grho = d + 5 * N;
    float *d_vp0 = d + 6 * N, *d_vs0 = d + 7 * N, *d_rho0 = d + 8 * N;
    float *d_vp1 = d + 9 * N, *d_vs1 = d + 10 * N, *d_rho1 = d + 11 * N, *d_s = d + 12 * N;
    unsigned *d_mx = (unsigned *)(d + 15 * N);
    float *d_eps = (float *)(d_mx + 8);
    int *d_hit = (int *)(d_eps + 4);
    auto h2d = [&](float *dst, const float *src) -> cudaError_t {
        return src ? cudaMemcpyAsync(dst, src, pb, cudaMemcpyHostToDevice, c->st) : cudaSuccess;
    };
    const bool lim = mc->limit_update == 1;
    CK(h2d(d_vp, vp));
    CK(h2d(d_rho, rho));
    CK(h2d(d_gvp, g_vp));
    CK(h2d(d_grho, g_rho));
    if (!ac) {
        CK(h2d(d_vs, vs));
        CK(h2d(d_gvs, g_vs));
    }
    if (lim) {
        CK(h2d(d_vp0, vp_start));
        CK(h2d(d_rho0, rho_start));
        if (!ac) CK(h2d(d_vs0, vs_start));
    }
    CK(cudaMemsetAsync(d_mx, 0, 64, c->st));
    k_mc_maxima<<<(unsigned)std::min<long long>((N + 255) / 256, 148 * 8), 256, 0, c->st>>>(
        m, d_vp, d_gvp, d_vs, d_gvs, d_rho, d_grho, d_mx);
    k_mc_update<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>(m, d_mx, d_vp, d_vs, d_rho, d_gvp, d_gvs, d_grho,
                                                                 d_vp0, d_vs0, d_rho0, d_vp1, d_vs1, d_rho1,
                                                                 m.lbfgs_npar ? d_s : nullptr, d_eps, d_hit);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(vp1, d_vp1, pb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(rho1, d_rho1, pb, cudaMemcpyDeviceToHost, c->st));
    if (!ac) CK(cudaMemcpyAsync(vs1, d_vs1, pb, cudaMemcpyDeviceToHost, c->st));
    if (m.itest == 0) {
        CK(cudaMemcpyAsync(vp, d_vp, pb, cudaMemcpyDeviceToHost, c->st));
        CK(cudaMemcpyAsync(rho, d_rho, pb, cudaMemcpyDeviceToHost, c->st));
        if (!ac) CK(cudaMemcpyAsync(vs, d_vs, pb, cudaMemcpyDeviceToHost, c->st));
        if (m.lbfgs_npar) CK(cudaMemcpyAsync(s_lbfgs, d_s, (size_t)m.lbfgs_npar * pb, cudaMemcpyDeviceToHost, c->st));
    }
    float e[3];
    int hit = 0;
    CK(cudaMemcpyAsync(e, d_eps, sizeof e, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&hit, d_hit, sizeof hit, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (eps) std::memcpy(eps, e, sizeof e);
    if (ratio_hit) *ratio_hit = hit;
    return IFOS_OK;
}

extern "C" int ifos_median_smooth(ifos_ctx *c, float *mat, int filt_size) {
    if (!c || !mat) return IFOS_ERR_ARG;
    if (filt_size == 0) return IFOS_OK;  // src/smooth.c:78 returns unchanged
    int fs = filt_size;
    if (!(fs % 2)) fs += fs > 0 ? 1 : -1;  // an even size grows away from zero (src/smooth.c:79-82)
    fs = std::abs(fs);
    if (fs * fs + 1 > kMedianMax) return fail(c, IFOS_ERR_ARG, "filter size above 31");
    CK(cudaSetDevice(c->device));
    const long long N = (long long)c->p.nx * c->p.ny;
    void *scr = nullptr;
    if (int rc = scratch(c, (size_t)2 * N * 4, &scr)) return rc;
    float *d_in = (float *)scr, *d_out = d_in + N;
    CK(cudaMemcpyAsync(d_in, mat, (size_t)N * 4, cudaMemcpyHostToDevice, c->st));
    k_median_smooth<<<(unsigned)((N + 127) / 128), 128, 0, c->st>>>(d_in, d_out, c->p.nx, c->p.ny, fs);
    c->launches++;
    CK(cudaMemcpyAsync(mat, d_out, (size_t)N * 4, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

// The cascade of a Butterworth filter of order `m` (contrib/libcseife/
// cseife.c:164-193 with the section coefficients of cseife_rfk.c): a first-
// order section when m is odd, then m/2 second-order sections with damping
// sin(pi/2 (2j-1)/m); t0 = period / sample interval.
static int butterworth_sections(bool highpass, double t0, int m, KIIR &f) {
    f.n = 0;
    if (m < 1 || m / 2 + (m % 2) > 8) return IFOS_ERR_ARG;
    const double one = 1., two = 2., four = 4., eight = 8.;
    const double zpi = eight * atan(one);
    const double eps = zpi / t0;
    if (m > 2 * (m / 2)) {
        double *c = f.c[f.n++];
        c[2] = 0.;
        c[4] = 0.;
        c[3] = (two - eps) / (two + eps);
        if (highpass) {
            c[0] = two / (two + eps);
            c[1] = -(c[0]);
        } else {
            c[0] = eps / (two + eps);
            c[1] = c[0];
        }
    }
    const double pih = 2. * atan(1.);
    for (int j = 1; j <= m / 2; ++j) {
        const double h = sin(pih * (2 * j - 1) / m);
        const double epsq = eps * eps;
        const double a = one - eps * h + epsq / four;
        const double b = -two + epsq / two;
        const double cc = one + eps * h + epsq / four;
        double *c = f.c[f.n++];
        c[3] = -b / cc;
        c[4] = -a / cc;
        if (highpass) {
            c[0] = one / cc;
            c[1] = -(c[0]) - c[0];
        } else {
            c[0] = epsq / four / cc;
            c[1] = c[0] + c[0];
        }
        c[2] = c[0];
    }
    return IFOS_OK;
}

extern "C" int ifos_timedomain_filt(ifos_ctx *c, float *data, int ntr, int ns, float fc, int order, int method,
                                    float f_high_pass) {
    if (!c || !data || ntr < 1 || ns < 1 || (method != 1 && method != 2)) return IFOS_ERR_ARG;
    if (!(fc > 0.0f) || order < 1) return fail(c, IFOS_ERR_ARG, "corner frequency and order must be positive");
    CK(cudaSetDevice(c->device));
    const double dt = (double)c->p.dt;
    KIIR lp{}, hp{};
    // src/timedomain_filt.c:53-84: a lowpass at fc (method 1), then a highpass
    // at F_HIGH_PASS when it is set; method 2 is a highpass at fc
    if (method == 1 && butterworth_sections(false, (1.0 / (double)fc) / dt, order, lp))
        return fail(c, IFOS_ERR_ARG, "filter order too high");
    const double t0_hp = method == 2 ? 1.0 / (double)fc : (f_high_pass != 0.0f ? 1.0 / (double)f_high_pass : 0.0);
    if ((method == 2 || f_high_pass != 0.0f) && butterworth_sections(true, t0_hp / dt, order, hp))
        return fail(c, IFOS_ERR_ARG, "filter order too high");
    const size_t db = (size_t)ntr * ns * 4, wb = (size_t)ntr * (ns + 1) * sizeof(double);
    void *scr = nullptr;
    if (int rc = scratch(c, wb + db, &scr)) return rc;
    double *work = (double *)scr;
    float *d_data = (float *)((char *)scr + wb);
    CK(cudaMemcpyAsync(d_data, data, db, cudaMemcpyHostToDevice, c->st));
    k_butterworth<<<(ntr + 63) / 64, 64, 0, c->st>>>(d_data, work, ntr, ns, lp, hp);
    c->launches++;
    CK(cudaMemcpyAsync(data, d_data, db, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_fd_coeffs(const ifos_params *p, float *hc7) {
    if (!p || !hc7) return IFOS_ERR_ARG;
    return fd_coefficients(p->fdorder, p->maxrelerror, hc7) ? IFOS_OK : IFOS_ERR_ARG;
}

extern "C" int ifos_cpml_profiles(const ifos_params *p, float *out) {
    if (!p || !out || p->fw < 0) return IFOS_ERR_ARG;
    CpmlProfiles pr = cpml_profiles(*p);
    for (int a = 0; a < 12; a++)
        for (int h = 0; h <= 2 * p->fw; h++) out[(size_t)a * (2 * p->fw + 1) + h] = pr.arr[a][h];
    return IFOS_OK;
}

extern "C" int ifos_kernel_timing(ifos_ctx *c, int stride) {
    if (!c || stride < 0) return IFOS_ERR_ARG;
    c->prof_stride = stride;
    return IFOS_OK;
}

extern "C" int ifos_kernel_times(ifos_ctx *c, double *ms4, long long *count4, int reset) {
    if (!c) return IFOS_ERR_ARG;
    for (int k = 0; k < 4; k++) {
        if (ms4) ms4[k] = c->kt_ms[k];
        if (count4) count4[k] = c->kt_n[k];
        if (reset) {
            c->kt_ms[k] = 0;
            c->kt_n[k] = 0;
        }
    }
    return IFOS_OK;
}

extern "C" int ifos_grad_sum_device(ifos_ctx *c, int nshots, float *dev_out) {
    if (!c || !dev_out) return IFOS_ERR_ARG;
    if (nshots < 1 || nshots > c->p.max_shots) return fail(c, IFOS_ERR_ARG, "nshots out of range");
    CK(cudaSetDevice(c->device));
    const long long N = (long long)c->p.nx * c->p.ny;
    k_grad_sum<<<(unsigned)((N + 255) / 256), 256, 0, c->st>>>((const float *)c->gout.p, nshots, N, dev_out);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    return IFOS_OK;
}

extern "C" int ifos_set_option(ifos_ctx *c, int option, int value) {
    if (!c) return IFOS_ERR_ARG;
    switch (option) {
        case IFOS_OPT_GRAPHS: c->graphs = value != 0; break;
        case IFOS_OPT_PDL: c->pdl = value != 0; break;
        case IFOS_OPT_BLOCKS_PER_SM:
            if (value < 0 || value > 32) return fail(c, IFOS_ERR_ARG, "blocks per SM must be in 0..32");
            c->blocks_per_sm = value;
            break;
        case IFOS_OPT_TILE_ORDER:
            if (value < 0 || value > 3) return fail(c, IFOS_ERR_ARG, "tile order must be 0..3");
            c->g.tile_order = value;
            break;
        case IFOS_OPT_WAIT_LIMIT:
            if (value < 0) return fail(c, IFOS_ERR_ARG, "the wait limit must be >= 0");
            c->g.prod_polls = value;
            break;
        default: return fail(c, IFOS_ERR_ARG, "unknown option " + std::to_string(option));
    }
    return IFOS_OK;
}

extern "C" int ifos_get_option(const ifos_ctx *c, int option, int *value) {
    if (!c || !value) return IFOS_ERR_ARG;
    switch (option) {
        case IFOS_OPT_GRAPHS: *value = c->graphs ? 1 : 0; break;
        case IFOS_OPT_PDL: *value = c->pdl ? 1 : 0; break;
        case IFOS_OPT_BLOCKS_PER_SM: *value = c->blocks_per_sm; break;
        case IFOS_OPT_TILE_ORDER: *value = c->g.tile_order; break;
        case IFOS_OPT_WAIT_LIMIT: *value = c->g.prod_polls; break;
        default: return IFOS_ERR_ARG;
    }
    return IFOS_OK;
}

extern "C" int ifos_set_stream(ifos_ctx *c, void *stream) {
    if (!c) return IFOS_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->st));
    c->st = stream ? (cudaStream_t)stream : c->own_st;
    return IFOS_OK;
}
