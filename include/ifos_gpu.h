/*
 * ifos_gpu.h -- C ABI of the B200 shot solver (libifos_b200.so).
 *
 * Replaces the device-side work of the IFOS2D shot loop:
 *   forward time loop   src/IFOS2D.c:1651-1894  (update_v_PML, update_s_*_PML,
 *                       psource, surface_*_PML, seismo_ssg, snapshot store)
 *   adjoint time loop   src/IFOS2D.c:2224-2438  (same kernels with sw=1 and the
 *                       zero-lag correlation at :2379-2419)
 *   gradient assembly   src/IFOS2D.c:2471-2611  (PARAMETERIZATION 1 and 3)
 *   model set-up        src/IFOS2D.c:906-943 (matcopy_elastic, av_mue, av_rho,
 *                       av_tau, prepare_update_s) and :816 (PML_pro)
 * The reference exposes these as void C functions over float** arrays plus
 * global scalars (src/fd.h:206-560); its shot loop, snapshot store, correlation
 * and assembly are inline in main().  This ABI keeps their roles behind plain
 * pointers and sizes: the caller owns every host buffer, the library owns the
 * device state, every call returns an int status and never exits.
 *
 * Array conventions
 *   model / gradient planes: NY x NX floats, row-major, x fastest; element
 *     (j,i) of the reference's 1-based grid at [(j-1)*NX + (i-1)]
 *   srcpos: 8 x nsrc floats, row r = the reference's srcpos_loc[r+1][*]
 *     (x, y as 1-based grid indices, 0, tshift, fc, amp, azimuth, type)
 *   recpos: 2 x ntr ints, grid x row then grid y row (1-based)
 *   signals: nsrc x NT; sections: IFOS_NS x ntr x NT (vx, vy, vz, p, curl,
 *     div); adjoint sources: 3 x ntr x NT (vx, vy, vz-or-p), time-reversed as
 *     calc_res writes them (src/calc_res.c:220-281)
 * A context holds `max_shots` shot slots stepped together (batching).  One
 * context must not be used from two host threads at once; distinct contexts
 * are independent and each owns its own CUDA stream.
 */
#ifndef IFOS_GPU_H
#define IFOS_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFOS_OK 0
#define IFOS_ERR_ARG 1      /* invalid argument or parameter combination */
#define IFOS_ERR_CUDA 2     /* CUDA runtime error (message via ifos_last_error) */
#define IFOS_ERR_NOMEM 3    /* device allocation failed / admission refused */
#define IFOS_ERR_UNSTABLE 4 /* NaN/Inf found in the wavefield (src/IFOS2D.c:1660-1672) */
#define IFOS_ERR_STATE 5    /* call out of order (e.g. adjoint without stored snapshots) */

#define IFOS_MAX_L 8
#define IFOS_NS 6  /* seismogram planes */
#define IFOS_NG 10 /* gradient planes, see IFOS_G_* */
#define IFOS_NF 12 /* field planes, see IFOS_F_* */

enum { IFOS_S_VX = 0, IFOS_S_VY, IFOS_S_VZ, IFOS_S_P, IFOS_S_CURL, IFOS_S_DIV };
enum {
    IFOS_G_LAM_RAW = 0, /* waveconv_shot before assembly   (src/IFOS2D.c:2390) */
    IFOS_G_MU_RAW,      /* waveconv_u_shot before assembly (src/IFOS2D.c:2398) */
    IFOS_G_RHO_RAW,     /* waveconv_rho_shot before assembly (src/IFOS2D.c:2385) */
    IFOS_G_VP,          /* per-shot vp gradient  (src/IFOS2D.c:2491) */
    IFOS_G_VS,          /* per-shot vs gradient  (src/IFOS2D.c:2520) */
    IFOS_G_RHO,         /* per-shot rho gradient (src/IFOS2D.c:2580) */
    IFOS_G_MU_Z_RAW,    /* SH waveconv_u_shot_z   (src/IFOS2D.c:2412) */
    IFOS_G_RHO_Z_RAW,   /* SH waveconv_rho_shot_z (src/IFOS2D.c:2410) */
    IFOS_G_VS_Z,        /* SH vs gradient  (src/IFOS2D.c:2549) */
    IFOS_G_RHO_Z        /* SH rho gradient (src/IFOS2D.c:2600) */
};
enum {
    IFOS_F_VX = 0, IFOS_F_VY, IFOS_F_SXX, IFOS_F_SYY, IFOS_F_SXY, IFOS_F_VXP1, IFOS_F_VYP1,
    IFOS_F_VZ, IFOS_F_SXZ, IFOS_F_SYZ, IFOS_F_VZP1, IFOS_F_SP
};

/* Snapshot storage formats (the forward wavefield kept for the adjoint). */
#define IFOS_SNAP_F32 0
#define IFOS_SNAP_BF16 1 /* bf16 with one fp32 scale per snapshot and component */
#define IFOS_SNAP_F16 2  /* fp16 with one fp32 scale per snapshot and component */
/* fp16 with an fp32 scale per snapshot, component and 64-cell row segment,
 * written by the stencil kernels themselves (no extra pass over the
 * wavefield); the scale maps each segment's maximum to 65472. */
#define IFOS_SNAP_F16S 3
/* int16 with the scale layout of IFOS_SNAP_F16S: the segment maximum maps to
 * 32767 and values round to the nearest integer, so the absolute error is at
 * most about max/65534 (32x below fp16's at the top of a segment) */
#define IFOS_SNAP_I16S 4

/* Parameters: the reference's global scalars of the propagation path
 * (src/globvar.h; read by src/update_v_PML.c:41-48, src/PML_pro.c:88-98,
 * src/prepare_update_s.c:24-26, src/seismo_ssg.c:30-32) plus the
 * device-side choices of this library. */
typedef struct ifos_params {
    int nx, ny, nt;
    float dh, dt;
    int fdorder, maxrelerror;
    int fw, free_surf, boundary;
    float vppml, fpml, npower, k_max_pml;
    int L;
    float f_ref, tau;
    float fl[IFOS_MAX_L];
    int wavetype;         /* 1 P-SV, 2 SH, 3 both */
    int acoustic;         /* 1: pressure formulation (WAVETYPE 1 only) */
    int parameterization; /* 1: vp, vs, rho; 3: lambda, mu, rho (elastic and visco,
                             not acoustic): the vp and vs planes of ifos_model_upload
                             then hold lambda and mu, as the reference's ppi and pu
                             do, and the vp / vs / rho gradients are the lambda / mu /
                             rho ones (src/IFOS2D.c:2498-2608).  2 is rejected: the
                             reference's stress updates leave it undefined */
    int velocity;         /* must be 0 */
    int seismo;           /* 0..5 as SEISMO */
    int source_type;      /* default forward source type */
    int adjoint_type;     /* 1 vx+vy, 2 vy, 3 vx, 4 p */
    int dtinv;            /* snapshot interval; NT % DTINV == 0 */
    /* --- device-side choices --- */
    int hi_order_corrected; /* 1: FDORDER 10/12 P-SV/acoustic use the CPML form of
                               orders 2-8; 0: the reference's 10/12 branches */
    int precision;          /* 0: fp32 arithmetic, 1: fp64 (the error oracle) */
    int snap_format;        /* IFOS_SNAP_* */
    int max_shots;          /* shot slots stepped together, >= 1 */
    int max_models;         /* model slots, >= 1 */
    int max_src, max_rec;   /* per-shot source / receiver capacity */
    int grad_acc64;         /* 1: the fp32 path accumulates the correlation sums in double and
                               rounds them to float once, before the assembly (needs fp32
                               arithmetic, an even NX and IFOS_SNAP_F32/F16S/I16S); 0: in float,
                               as the reference does (default) */
    int mu_corrected;       /* 1: the mu correlation as (f_xx+f_yy)(s_xx+s_yy) and (f_xx-f_yy)(s_xx-s_yy)
                               (a documented deviation: src/IFOS2D.c:2398-2404 multiplies before it
                               adds, so the forward stresses enter alone and cancel only over time);
                               0: the reference's expression (default) */
} ifos_params;

typedef struct ifos_ctx ifos_ctx;

/* Fill `p` with the defaults of the reference's JSON reader. */
void ifos_params_default(ifos_params *p);

/* Create a context on CUDA device `device`; allocates all device state,
 * including max_shots snapshot buffers when `with_snapshots` is non-zero.
 * Replaces the allocations of src/IFOS2D.c:371-645. */
int ifos_ctx_create(const ifos_params *p, int device, int with_snapshots, ifos_ctx **out);
int ifos_ctx_destroy(ifos_ctx *ctx);
/* Last error message of this context (or of the last failed create when ctx is NULL). */
const char *ifos_last_error(const ifos_ctx *ctx);
/* Status of a context for a driver that checks once per shot or iteration:
 * the code of the last failed call since the previous ifos_status (IFOS_OK
 * when none), or IFOS_ERR_CUDA when its stream or copy stream has failed;
 * clears the recorded code.  The message stays in ifos_last_error.  The
 * reference aborts instead (declare_error, src/util.c:26-35). */
int ifos_status(ifos_ctx *ctx);
/* Bytes of device memory a context with these parameters needs. */
size_t ifos_ctx_bytes(const ifos_params *p, int with_snapshots);

/* Upload model `model` (vp, vs, rho, or lambda, mu, rho under PARAMETERIZATION
 * 3; taup/taus may be NULL meaning TAU) and
 * rebuild its coefficients: ghost ring, rip/rjp, uipjp, viscoelastic
 * coefficients.  Replaces src/IFOS2D.c:906-943 / :3240-3265. */
int ifos_model_upload(ifos_ctx *ctx, int model, const float *vp, const float *vs, const float *rho,
                      const float *taup, const float *taus);

/* Describe shot `slot`: its model, sources (+ signals nsrc x NT) and receivers. */
int ifos_shot_setup(ifos_ctx *ctx, int slot, int model, int nsrc, const float *srcpos, const float *signals,
                    int ntr, const int *recpos);

/* Forward time loop for slots [0, nshots): zero state, step NT times.
 * Stores snapshots when the context has them and store != 0.  Sections of
 * slot s go to sections + s * IFOS_NS*max_rec*NT (NULL: keep on device). */
int ifos_forward(ifos_ctx *ctx, int nshots, int store, float *sections);

/* Adjoint time loop for slots [0, nshots) with adjoint sources
 * adj + s * 3*max_rec*NT (NULL: use the ones staged by ifos_stage_adjoint),
 * correlation with the stored snapshots, and per-shot gradient assembly.
 * Gradients of slot s go to grads + s * IFOS_NG*NY*NX (NULL: keep on device). */
int ifos_adjoint(ifos_ctx *ctx, int nshots, const float *adj, float *grads);

/* Device-resident pieces of the two calls above, for callers that keep
 * inputs resident: stage adjoint sources, then run and fetch separately. */
int ifos_stage_adjoint(ifos_ctx *ctx, int nshots, const float *adj);
int ifos_fetch_sections(ifos_ctx *ctx, int nshots, float *sections);
int ifos_fetch_grads(ifos_ctx *ctx, int nshots, float *grads);
/* Asynchronous device-to-host staging of the same buffers (the driver's
 * seismogram and gradient output, src/saveseis_glob.c and the gradient
 * writers, without the host waiting on the device): the copy is queued on
 * the context's copy stream after the work already queued and the call
 * returns at once, so it overlaps the next forward or adjoint.  A later call
 * that overwrites the buffer (ifos_forward / ifos_forward_steps for the
 * seismograms, ifos_adjoint / ifos_taper_grad_shot for the gradients) is
 * ordered after the copy on the device.  The host memory must stay valid,
 * and is not to be read, until ifos_fetch_wait returns; it overlaps only
 * when pinned (ifos_host_alloc). */
int ifos_fetch_sections_async(ifos_ctx *ctx, int nshots, float *sections);
int ifos_fetch_grads_async(ifos_ctx *ctx, int nshots, float *grads);
int ifos_fetch_wait(ifos_ctx *ctx);
/* Pinned (page-locked) host memory for asynchronous fetches; no context. */
int ifos_host_alloc(size_t bytes, void **out);
int ifos_host_free(void *p);
/* Sum of the assembled per-shot gradients (vp, vs, rho, vs_z, rho_z) over
 * slots [0, nshots), as src/IFOS2D.c:2703-2724: out is 5 x NY x NX. */
int ifos_grad_sum(ifos_ctx *ctx, int nshots, float *out);

/* Run `nsteps` forward steps of slot 0 from zero state without snapshots and
 * copy the IFOS_NF field planes to `fields` (parity checks of single steps). */
int ifos_forward_steps(ifos_ctx *ctx, int nsteps, float *fields);
/* Stored forward snapshot `index` (0 .. NT/DTINV-1) of `slot`, read back as
 * the correlation reads it (dequantised for the 2-byte formats): ncomp x NY x
 * NX floats, components in the order vxp1, vyp1, sxx, syy, sxy (P-SV; acoustic
 * vxp1, vyp1, p), then vzp1, sxz, syz (SH). */
int ifos_fetch_snapshot(ifos_ctx *ctx, int slot, int index, float *out);
/* Copy the current IFOS_NF field planes of `slot` to host. */
int ifos_fetch_fields(ifos_ctx *ctx, int slot, float *fields);

/* FP64 reductions (misfit, energy, dot products) over n floats on the
 * device: returns sum(a*b) (b NULL: sum(a*a)) accumulated in double. */
int ifos_dot_f64(ifos_ctx *ctx, const float *a, const float *b, size_t n, int device_ptrs, double *out);

/* The L-BFGS two-loop recursion (src/LBFGS.c:226-323, lbfgs_core, one rank)
 * on the device.  s and y hold n_lbfgs rows of npar floats, row w-1 being
 * the reference's s_LBFGS[w] / y_LBFGS[w] (w = 1..n_lbfgs, the ring the
 * driver fills); q (npar) is the preconditioned gradient, changed in place as
 * the reference changes it; r (npar) receives the direction; rho and alpha
 * are host arrays of n_lbfgs floats: rho[w-1] of the newest pair
 * (w = (iteration-1) % n_lbfgs, 0 read as n_lbfgs) is set, the others are
 * read, and alpha is filled.  iteration >= 2.  device_ptrs: s, y, q and r are
 * device pointers, else host arrays (copied in and out).  Every dot product
 * is accumulated in double (the reference sums in float); its result is
 * rounded to float where the reference keeps a float (rho, H0, alpha, beta),
 * and the vector updates are the reference's float operations. */
int ifos_lbfgs_core(ifos_ctx *ctx, int iteration, int n_lbfgs, size_t npar, const float *s, const float *y,
                    float *rho, float *q, float *alpha, float *r, int device_ptrs);

/* Residuals of one component, LNORM=2, VELOCITY=0 (src/calc_res.c:137-281):
 * integrates both sections, writes the time-reversed residual to diff
 * (ntr x NT) and the misfit/energy sums in double. */
int ifos_calc_res(ifos_ctx *ctx, int ntr, const float *obs, const float *syn, float *diff, double *l2,
                  double *energy);

/* The residual step between the loops (src/IFOS2D.c:2115-2180, which calls
 * calc_res per component): for slots [0, nshots) of the last ifos_forward,
 * forms the residual of each component the adjoint uses (vx/vy by
 * ADJOINT_TYPE 1-3, vz for SH, p for ADJOINT_TYPE 4 / acoustic) against the
 * observed seismograms `obs` (slot x 3 x max_rec x NT, host; components
 * vx, vy, vz-or-p) on the device, stages them as the adjoint sources of the
 * next ifos_adjoint(ctx, nshots, NULL, ...) and returns each slot's FP64
 * misfit and energy in l2[nshots] / energy[nshots] (either may be NULL).
 * kill (slot x max_rec ints, or NULL) marks traces killed for this shot (a
 * column of the trace-kill table): they keep a zero residual and add nothing
 * to the sums, as calc_res skips them (src/calc_res.c:196-197).  win (or
 * NULL) applies the time windows of TIMEWIN=1 to the integrated synthetic
 * and observed traces before the residual (src/calc_res.c:157-160), as
 * ifos_time_window does. */
typedef struct ifos_window {
    int tw_ind;          /* TW_IND: 0 one pick + TWLENGTH_PLUS/MINUS, 1 pick + lengths, 2 two windows */
    const float *picks;  /* host, slot x np x max_rec with np = 1, 3, 6 for tw_ind 0, 1, 2 */
    float gamma;         /* GAMMA */
    float twl_plus, twl_minus; /* TWLENGTH_PLUS, TWLENGTH_MINUS (tw_ind 0) */
} ifos_window;
int ifos_residual_adjoint(ifos_ctx *ctx, int nshots, const float *obs, const int *kill, const ifos_window *win,
                          double *l2, double *energy);

/* Offset-based trace-kill table (src/create_trkill_table.c:21-46), on the
 * device and bit-identical to the reference: killtable (ntr_glob x nsrc_glob,
 * row-major [receiver][source], host, in/out) gets 1 where the offset between
 * source s at (sx[s], sy[s]) metres and receiver r at grid point
 * (rx[r], ry[r]) (times DH) lies strictly between lower and upper; other
 * entries keep their values (the driver zeroes the table first or adds the
 * offset kill to a table read from file). */
int ifos_trkill_table(ifos_ctx *ctx, int ntr_glob, const int *rx, const int *ry, int nsrc_glob, const float *sx,
                      const float *sy, float lower, float upper, int *killtable);

/* Time windows around picked first arrivals (src/time_window.c:24-224) on
 * ntr traces of ns samples (host, row-major, in/out), samples 2..ns as the
 * reference: tw_ind 0 takes picks[ntr] with twl_plus/twl_minus, 1 takes
 * picks[3][ntr] (pick, length+, length-), 2 takes picks[6][ntr] (two windows).
 * The picks are those of the local traces (the reference's recpos_loc[3]
 * mapping is the caller's).  mask (NULL or ntr x ns) receives per sample the
 * tapers applied (bits 0/1: late/early taper of the first window, 2/3: of the
 * second).  The sample selection is bit-identical to the reference; the taper
 * values use the device's exp(). */
int ifos_time_window(ifos_ctx *ctx, int ntr, int ns, float *sections, int tw_ind, const float *picks, float gamma,
                     float twl_plus, float twl_minus, unsigned char *mask);

/* Host-only set-up queries (no device needed): the FD weights hc[0..6]
 * (src/holbergcoeff.c:37-108) and the CPML profiles as 12 arrays of 2*FW+1
 * floats, 1-based, in the order K_x a_x b_x K_x_half a_x_half b_x_half K_y a_y
 * b_y K_y_half a_y_half b_y_half (src/PML_pro.c:83-316). */
int ifos_fd_coeffs(const ifos_params *p, float *hc7);
int ifos_cpml_profiles(const ifos_params *p, float *out);

/* Per-kernel timing: every `stride`-th time step (0 = off) the velocity and
 * stress kernels are bracketed by CUDA events on the context's stream; the
 * accumulated milliseconds and launch counts of the kernel classes
 * {velocity, stress, snapshot, correlation} are returned (4 each) and reset. */
int ifos_kernel_timing(ifos_ctx *ctx, int stride);
int ifos_kernel_times(ifos_ctx *ctx, double *ms4, long long *count4, int reset);

/* Sum of the assembled gradients written to DEVICE memory (5 x NY x NX
 * floats at dev_out), for callers that reduce it across GPUs in place. */
int ifos_grad_sum_device(ifos_ctx *ctx, int nshots, float *dev_out);

/* Launch on the caller's CUDA stream (a cudaStream_t passed as void*), e.g.
 * to time the library with the caller's events; NULL returns to the
 * context's own stream.  The caller keeps ownership of its stream. */
int ifos_set_stream(ifos_ctx *ctx, void *stream);

/* Execution options of a context (no counterpart in the reference; they
 * change how the loops run, never what they compute: every setting of the
 * first four gives bit-identical results).  A change takes effect at the
 * next loop and discards the loops captured so far. */
enum {
    /* 1 (default): each time loop (ifos_forward, ifos_adjoint) is captured
     * once into a CUDA graph per launch sequence and replayed for every
     * later call with the same shot count; 0: launched step by step. */
    IFOS_OPT_GRAPHS = 0,
    /* 1 (default): the loop's kernels are programmatic dependent launches
     * (each starts its independent loads while its predecessor drains). */
    IFOS_OPT_PDL = 1,
    /* persistent stencil CTAs per SM; 0 (default): as many as fit. */
    IFOS_OPT_BLOCKS_PER_SM = 2,
    /* 0: the stencil launches walk all tiles of slot 0, then of slot 1, ...;
     * 1: the same tile of consecutive slots on consecutive CTAs, so that
     * shots over one model share its coefficient tiles in L2.  2 (default)
     * and 3: orders 0 and 1 with the tiles that meet a CPML strip ranked
     * before the interior, so that every persistent CTA gets the same share
     * of the slower strip tiles (one shot per launch: 10 % faster loops on
     * the 2000 x 600 workload). */
    IFOS_OPT_TILE_ORDER = 3,
    /* polls of the pipelined stencils' stage-release wait (the producer
     * waiting for the compute warps to free a ring stage); 0 (default): about
     * a second.  A wait that runs out stops the launch: its block issues no
     * more copies, waits for those in flight, and the loop returns
     * IFOS_ERR_CUDA ("barrier wait timed out", also reported by ifos_status)
     * with the context still usable.  A limit of a few polls makes that
     * happen on purpose, to test the error path. */
    IFOS_OPT_WAIT_LIMIT = 4
};
int ifos_set_option(ifos_ctx *ctx, int option, int value);
int ifos_get_option(const ifos_ctx *ctx, int option, int *value);

/* Butterworth filtering of ntr traces of ns samples (host, in place), as
 * src/timedomain_filt.c does with the vendored libcseife: method 1 a lowpass
 * of `order` at corner frequency fc, followed by a highpass at f_high_pass
 * when that is non-zero (F_HIGH_PASS); method 2 a highpass at fc.  Each
 * trace is filtered in double with a zero sample before it, as the
 * reference's dvector provides; the context's DT is the sample interval.
 * Orders up to 16. */
int ifos_timedomain_filt(ifos_ctx *ctx, float *data, int ntr, int ns, float fc, int order, int method,
                         float f_high_pass);

/* Per-shot gradient taper around the source (src/taper_grad_shot.c, sws=1)
 * applied on the device to the stored per-shot gradients of slots
 * [0, nshots) (the planes of `planes`, a bit mask over IFOS_G_*), as the
 * driver applies it before summing the shots (src/IFOS2D.c:2683-2687):
 * src_xy holds each slot's source x, y in metres (srcpos rows 1-2);
 * srtradius, srtshape and filtsize are SRTRADIUS, SRTSHAPE and FILTSIZE. */
int ifos_taper_grad_shot(ifos_ctx *ctx, int nshots, const float *src_xy, float srtradius, int srtshape,
                         int filtsize, unsigned planes);

/* Per-shot gradient taper read from a file (src/taper_grad_shot.c:206-289,
 * sws 2-4; the driver's SWS_TAPER_FILE_PER_SHOT, src/IFOS2D.c:2669-2697):
 * the planes of `planes` (a bit mask over IFOS_G_*) of slot `slot`'s stored
 * gradients are multiplied cell by cell by `coeff`, an NY x NX host plane --
 * the TAPER_FILE_NAME.shot<n>.vp / .vs / .rho values, which the reference
 * reads x-major (ifos_b200.modelio.read_taper_file reads them so).  The
 * driver applies .vp to IFOS_G_VP, .vs to IFOS_G_VS and IFOS_G_VS_Z, .rho to
 * IFOS_G_RHO and IFOS_G_RHO_Z. */
int ifos_taper_grad_coeff(ifos_ctx *ctx, int slot, unsigned planes, const float *coeff);

/* Median smoothing of an NY x NX plane (host, in place) as src/smooth.c
 * does for gradients (FILT_SIZE_GRAD) and models (FILT_SIZE): filt_size 0
 * leaves the plane unchanged, an even size grows away from zero, |size| up
 * to 31; bit-identical to the reference's median2d selection. */
int ifos_median_smooth(ifos_ctx *ctx, float *mat, int filt_size);

/* Test model of a step-length trial, or the model update itself
 * (src/calc_mat_change_test.c:26-334, PARAMETERIZATION 1 or 3, which share
 * the update at :228, one rank): each
 * parameter's step is eps_scale * max(model) / max|search direction| (0
 * before its INV_*_ITER iteration; eps_scale itself under unnormalised
 * L-BFGS steps), then the reference's bounds, Vp/Vs ratio, limited-update
 * (S) and sign rules, in its float/double arithmetic.  The search
 * directions are the driver's waveconv, waveconv_u, waveconv_rho. */
typedef struct ifos_mat_change {
    float eps_scale;                       /* eps_scale: the trial's scale */
    int iter, itest;                       /* iter; itest 0 updates vp/vs/rho in place */
    int inv_vp_iter, inv_vs_iter, inv_rho_iter;  /* INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER */
    int lbfgs_unnormalised;                /* GRAD_METHOD==2 && iter > LBFGS_iter_start && LBFGS_STEP_LENGTH */
    float vp_lower, vp_upper, vs_lower, vs_upper, rho_lower, rho_upper; /* VPLOWERLIM ... RHOUPPERLIM */
    float vp_vs_ratio;                     /* VP_VS_RATIO (checked when > 1) */
    int limit_update;                      /* S */
    float s_vp, s_vs, s_rho;               /* S_VP, S_VS, S_RHO (percent) */
    int lbfgs_npar;                        /* LBFGS_NPAR of the difference vectors (itest 0), 0: none */
    float vs_avg, rho_avg, vp_avg;         /* Vs_avg, rho_avg, Vp_avg of the difference vectors */
} ifos_mat_change;
/* Host NY x NX planes.  vs, g_vs, vs_start and vs1 are unused (may be NULL)
 * when the context is acoustic; the *_start planes are read only when
 * limit_update is set.  vp1, vs1, rho1 receive the test model; with itest 0
 * vp, vs, rho are also replaced by it and, when s_lbfgs is not NULL, the
 * difference vectors (vs, rho, vp planes of NX*NY, in the reference's
 * column-major order) are written there.  eps[3] receives EPSILON,
 * EPSILON_u, EPSILON_rho; *ratio_hit is set when the Vp/Vs bound moved vp. */
int ifos_mat_change_test(ifos_ctx *ctx, const ifos_mat_change *mc, float *vp, float *vs, float *rho,
                         const float *g_vp, const float *g_vs, const float *g_rho, const float *vp_start,
                         const float *vs_start, const float *rho_start, float *vp1, float *vs1, float *rho1,
                         float *s_lbfgs, float *eps, int *ratio_hit);

/* Step length of the line search (src/calc_opt_step.c:73-112, solving with
 * src/solvelin.c:53-70): fits the parabola a + b*eps + c*eps^2 through the
 * misfits l2t[0..2] of the test steps epst[0..2] by Gaussian elimination
 * without pivoting and returns its extremum -b/(2c) in *opteps, clamped as
 * the reference clamps it (epst[2] when the parabola opens downward with
 * l2t[1] > l2t[2] or when the extremum lies beyond epst[2]; epst[0] when it
 * is negative).  fp64 = 1 solves in double (this library's line search);
 * fp64 = 0 in float with the reference's operation order, bit-identical to
 * it.  Host code: needs no context or device. */
int ifos_opt_step(const float *l2t, const float *epst, int fp64, float *opteps);

/* FP64 dot product without any device allocation.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc -- code whose
 * device memory is owned and fully budgeted by another framework, or a
 * latency-bound loop where an allocation would synchronise the device -- and
 * already hold the data on the device.  Returns sum(a*b) (b NULL: sum(a*a))
 * over n floats at DEVICE pointers a, b of `device`, accumulated in double,
 * in *out (host).  Needs no context.  Its scratch is a static array of
 * IFOS_NOALLOC_MAX_BLOCKS+1 doubles that every device loading the library
 * keeps until exit; n is limited to IFOS_NOALLOC_MAX_N (IFOS_ERR_ARG above
 * it, message in ifos_last_error(NULL)).  Launches go to `stream` (NULL:
 * the default stream); the call copies the result to host memory and
 * synchronises `stream` before it returns, so it can be called neither from
 * a host function enqueued on a stream nor while any stream capture is in
 * progress.  The calling thread's
 * current device is restored before returning.  All calls on a device share
 * the scratch, so calls that overlap on the GPU (other host threads, other
 * streams) race. */
#define IFOS_NOALLOC_MAX_BLOCKS 4096
#define IFOS_NOALLOC_MAX_N (4096LL * 256 * 32)
int ifos_dot_f64_noalloc(int device, const float *a, const float *b, size_t n, void *stream, double *out);

/* Milliseconds of device time of the last ifos_forward / ifos_adjoint call. */
double ifos_last_ms(const ifos_ctx *ctx);
/* Kernel launches issued by this context since creation. */
long long ifos_launch_count(const ifos_ctx *ctx);
int ifos_sync(ifos_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
