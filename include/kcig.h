/*
 * kcig.h -- C ABI of the B200 adjoint angle-domain Kirchhoff CIG migration.
 *
 * Drop-in replacement for the adjoint (adj=1) path of the reference tool
 * kirchmig2d_cig (src/kirchmig2d_cig.cpp) and of the library routines it
 * calls (SERECKIRCH/include/kirmig.h, SERECKIRCH/include/tinterpsr.h).  All
 * arguments are plain pointers and sizes.  No entry point exits the process:
 * every function returns KCIG_OK (0) or a negative KCIG_ERR_* status, and
 * kcig_last_error() gives the message the reference would have printed.
 *
 * Array layouts follow the reference files exactly:
 *   data   [ns][nh][nt]   (time fastest)                 seismic_data=
 *   tables [npos][nx][nz] (depth fastest, index ix*nz+iz) stable= sderiv= rtable= rderiv=
 *   image  [ng][nx][nz]                                   migration=
 */
#ifndef KCIG_H
#define KCIG_H

#ifdef __cplusplus
extern "C" {
#endif

#define KCIG_OK 0
#define KCIG_ERR_ARG (-1)         /* invalid parameter or size                    */
#define KCIG_ERR_CUDA (-2)        /* a CUDA call failed                           */
#define KCIG_ERR_IO (-3)          /* file missing, truncated or malformed         */
#define KCIG_ERR_UNSUPPORTED (-4) /* valid for the reference, not built here      */
#define KCIG_ERR_NOMEM (-5)       /* device or host allocation failed             */
#define KCIG_ERR_DEVICE (-6)      /* a kernel reported a bounded-wait or bounds fault */

#define KCIG_MEM_HOST 0   /* pointer is ordinary or pinned host memory         */
#define KCIG_MEM_DEVICE 1 /* pointer is device memory of the plan's device      */
#define KCIG_MEM_HOST_STREAM 2 /* tables only: stay in host memory, slices copied per leg batch */

/* Parameters of kirchmig2d_cig.  Field meanings and defaults are those of
 * src/kirchmig2d_cig.cpp:494-958; kcig_params_init() fills the defaults. */
typedef struct kcig_params {
    int adj;                 /* 1 = migration, 0 = forward modelling          :565-568 */
    int cig;                 /* 0 stack, 1 common-image gathers               :569-572 */
    int cig_is_angle;        /* mode=angle (1) or mode=offset (0)             :554-563 */
    int cmp;                 /* receiver position = s+h (1) or h (0)          :573-576 */
    int half_angle;          /* 0 full opening angle, 1 half                  :585-586 */
    int isdiff;              /* diff=1: central derivative after doubint      :599     */
    int interp_type;         /* 'h' Hermite, 'l' linear, 'p' partial          :952-958 */
    int angle_interp;        /* two-bin linear (1) or nearest-bin (0)          :845-846 */
    int angle_grad_radius;   /* finite-difference radius, >=1                  :851-854 */
    int angle_smooth;        /* triangle smoothing radius, 0 = off             :855-858 */
    int aperture_trace;      /* -1 = no trace-index aperture                   :544-548 */
    int aperture_trace_taper;/*                                                 :859-862 */
    int direct_mute;         /*                                                 :707-762 */
    int direct_mute_invert;
    int direct_mute_qc_shot; /* -1 = no QC dump (CLI only)                      */
    float tau, aperture, aperture_taper, aperture_rmin, aperture_rtaper, antialias;
    float angle_taper_start, angle_taper_end;
    float oazmin, oazmax, oaztaper;
    float direct_mute_slope, direct_mute_intercept, direct_mute_taper;
    /* output axis as given (parse_output_axis, :323-368); resolved per plan */
    int axis_min_given, axis_max_given, axis_step_given, axis_n_given;
    float axis_min, axis_max, axis_step;
    int axis_n;
    /* which tool's semantics: 0 kirchmig2d_cig (above), 1 kirchmig2d
     * (src/kirchmig2d.cpp): cone aperture on both legs, cig=1 gives one
     * image per trace offset index, no mute, no angle gathers */
    int tool;
} kcig_params;

/* Axes of the data cube and of the traveltime tables (header values as the
 * reference reads them, cast to float: :651-661, :765-802). */
typedef struct kcig_geometry {
    int nt, nh, ns;
    float t0, dt, h0, dh, s0, ds;
    int nz, nx;
    float z0, dz, x0, dx;
    int sny;
    float sy0, sdy;
    int rny;
    float ry0, rdy;
} kcig_geometry;

typedef struct kcig_plan kcig_plan;

/* Message of the last failing call on this thread (never NULL). */
const char *kcig_last_error(void);

/* Reference defaults (kirchmig2d_cig.cpp:494-958 with mode=angle unset). */
int kcig_params_init(kcig_params *p);

/* Parse key=value tokens and par=<file> exactly as se_par_init +
 * kirchmig2d_cig's parameter block do (SEFILESYSTEM/src/se_par_sep.cpp:185-340,
 * src/kirchmig2d_cig.cpp:494-958), including the validation errors of the
 * direct mute.  argv[0] is skipped.  File keys (seismic_data=, ...) are
 * ignored here; kcig_run_cli handles them. */
int kcig_params_parse(int argc, char **argv, kcig_params *p);

/* The parameter block of kirchmig2d (src/kirchmig2d.cpp:55-340) into
 * kcig_params with tool = 1: adj (1), cig (0; 1 = common-offset gathers, one
 * image per offset index), cmp (1), diff (0), aperture_trace (-1, hard cut),
 * tau (0), aperture (90 deg, hard cone), antialias (1), type (hermit). */
int kcig_params_parse_kirchmig2d(int argc, char **argv, kcig_params *p);

/* Resolve the output (n3,o3,d3) axis for these data axes, as
 * parse_output_axis (src/kirchmig2d_cig.cpp:323-368). */
int kcig_output_axis(const kcig_params *p, const kcig_geometry *g, int *ng, float *g0, float *dg);

/* Create a migration plan on the current CUDA device.  Validates sizes like
 * the reference's dimension checks (:651-661, :765-802).  scratch_bytes caps
 * the plan's device scratch (0 = choose from free device memory). */
int kcig_plan_create(const kcig_params *p, const kcig_geometry *g, unsigned long long scratch_bytes,
                     kcig_plan **out);
int kcig_plan_destroy(kcig_plan *plan);

/* Use this CUDA stream (cudaStream_t) for all work of the plan (0 = legacy). */
int kcig_plan_set_stream(kcig_plan *plan, void *stream);

/* Traveltime tables and their position derivatives ([npos][nx][nz]).  Host
 * tables are copied to the device; device tables are used in place and must
 * outlive the plan.  Passing the same stable/rtable pointers shares one copy.
 * KCIG_MEM_HOST_STREAM keeps host tables where they are (they must stay valid
 * while the plan uses them; pinned memory copies fastest): each batch of leg
 * fields copies only the slices it interpolates into a staging buffer, so
 * tables larger than the device memory can be migrated.  Results are
 * identical to device-resident tables.  kcig_migrate, kcig_model and
 * kcig_leg_fields_device take streamed tables; kcig_migrate_prepared does
 * not (KCIG_ERR_UNSUPPORTED). */
int kcig_plan_set_tables(kcig_plan *plan, const float *stable, const float *sderiv,
                         const float *rtable, const float *rderiv, int memory);

/* Optional spatial gradient volumes sgradx/sgradz/rgradx/rgradz (all four or
 * none, :627-642), same layout as the tables. */
int kcig_plan_set_gradients(kcig_plan *plan, const float *sgradx, const float *sgradz,
                            const float *rgradx, const float *rgradz, int memory);

/* Adjoint migration: image[ng][nx][nz] = sum over traces (zeroed first, as
 * the reference memsets out, :964-965).  data and image are both host or both
 * device pointers (memory).  Replaces the shot/trace loop :979-1339. */
int kcig_migrate(kcig_plan *plan, const float *data, float *image, int memory);

/* Shot positions of the survey axis (s0 + is * ds, ds = 0 for one shot) for
 * shots first .. first + count - 1, both as the migration uses them: in FP64
 * for continuous quantities (pos) and in the reference's float expression
 * s0 + (float)is * ds for its discrete decisions (posf, :980).  Host-only;
 * either output may be NULL. */
int kcig_shot_positions(const kcig_geometry *g, int first, int count, double *pos, float *posf);

/* Restrict kcig_migrate to shots first .. first + count - 1 of the plan's
 * survey (first = 0, count = -1: all).  The data then holds only those shots
 * ([count][nh][nt]), while every shot keeps the position and antialias
 * spacing it has in the whole survey (kcig_shot_positions), so images of a
 * partition of the shots add up to the whole survey's image -- the shot
 * sharding of one survey over ranks, whose images are then summed (one
 * all-reduce).  The image is zeroed first as always.  No counterpart in the
 * reference, which migrates a whole file. */
int kcig_plan_set_shot_range(kcig_plan *plan, int first, int count);

/* Number of summation-kernel launches and the device time (ms, CUDA events)
 * of the last kcig_migrate; either pointer may be NULL. */
int kcig_plan_last_stats(const kcig_plan *plan, int *sum_launches, float *sum_ms, int *all_launches);

/* The drop-in executable: same argv, files, defaults, messages and exit
 * status as kirchmig2d_cig adj=1.  Returns 0 on success, else a KCIG_ERR_*. */
int kcig_run_cli(int argc, char **argv);

/* The drop-in kirchmig2d (src/kirchmig2d.cpp:35-612), adj=1: same keys,
 * defaults, error texts and output header; adj=0 returns
 * KCIG_ERR_UNSUPPORTED. */
int kcig_run_kirchmig2d_cli(int argc, char **argv);

/* ---- building blocks, device buffers, on `stream` ----------------------- */

/* SERECKIRCH/src/kirmig.cpp:8-24 doubint (+ :381-394 diff2 when isdiff=1)
 * for ntr traces of nt samples: in [ntr][nt] float, out [ntr][nt] double
 * (each causal/anticausal running sum accumulated in FP64). */
int kcig_doubint_device(const float *in, double *out, int ntr, int nt, int isdiff, float dt,
                        void *stream);

/* Leg fields of one source (is_source=1) or receiver position of a plan with
 * tables set, [nx][nz] each: traveltime T (double), position derivative Tx
 * (float, not scaled by the data spacing), direction phi = atan2(gz, gx) of
 * the stabilised traveltime gradient (double; NaN where the gradient
 * vanishes) and the aperture leg weight w (float) --
 * src/kirchmig2d_cig.cpp:987-1052 (source), :1148-1201 (receiver), :226-269.
 * Any output pointer may be NULL. */
int kcig_leg_fields_device(kcig_plan *plan, int is_source, double pos, double *T, float *Tx,
                           double *phi, float *w);

/* Allocation-free variant of kcig_leg_fields_device; it has no counterpart in
 * the reference.  For callers that cannot allocate device memory -- a host
 * application whose device memory belongs to its own allocator or is budgeted
 * to the byte, or code running where a cudaMalloc would synchronise the device
 * or fail -- it computes the same T, Tx, phi and w for one position without any
 * allocation, using a fixed 16 MiB scratch array built into the library (each
 * device that loads the library holds it until the process exits).  Limit:
 * nz*nx <= 262144 points, else KCIG_ERR_ARG.  p/g give the parameters and the
 * axes (the source or receiver position axis of g is used); table/deriv are
 * the device tables [npos][nx][nz]; gradx/gradz are the optional device
 * gradient volumes (both or NULL); outputs are caller-owned device arrays
 * [nx][nz] (any may be NULL).  The first call on a device looks up the
 * scratch array's device address.  The address is kept for the life of the process: do not call
 * this entry point again after cudaDeviceReset on that device.  All calls share the one array and leave the last call's contents
 * in it (every value is written before it is read, so nothing needs clearing);
 * calls that overlap on the GPU -- from other threads or other streams --
 * race and must be serialised by the caller.  Runs on `stream` and returns
 * after it completes. */
int kcig_leg_fields_noalloc(const kcig_params *p, const kcig_geometry *g, const float *table,
                            const float *deriv, const float *gradx, const float *gradz,
                            int is_source, double pos, double *T, float *Tx, double *phi, float *w,
                            void *stream);

/* Options of kcig_eikods (the eikods2d parameters of src/eikods2d.cpp:149-300). */
typedef struct kcig_eikods_opts {
    int order;            /* 1 or 2: accuracy order of the upwind update (order=, default 2) */
    int b1, b2;           /* constant-slowness box half-widths in samples along depth and lateral
                             (b1=, b2=; values below 1 become 1) */
    int l;                /* source perturbation axis of tdl1/tds1: 1 lateral (l=, default), 0 depth */
    int vel_is_slowness2; /* 0: vel is velocity (vel=1, default); 1: slowness squared (vel=0) */
    int max_iter;         /* bound on sweep iterations (4 sweeps each) per source; 0 = 256 */
} kcig_eikods_opts;

/* First-arrival traveltime tables, the computation of eikods2d
 * (src/eikods2d.cpp:149-765; SERECKIRCH/src/eikods.cpp:66-211 and
 * neighbors.cpp) on a 2-D grid: vel [nx][nz] (device, depth fastest) with
 * origins o1 (depth), o2 (lateral), samplings d1, d2, and the third-axis
 * origin/sampling o3/d3 of the velocity header (o3=0, d3=1 for a 2-D file);
 * shots [nshot][3] (host) as in the shot file: depth, lateral, third axis.
 * Writes time [nshot][nx][nz] (device) and, where not NULL, tdl1/tds1 (the
 * first derivatives with respect to the source position; both or neither),
 * gradz/gradx (the branch-aware upwind gradients of eikods2d.cpp:30-68), all
 * [nshot][nx][nz] (device), and iters [nshot] (host): the sweeps each source
 * took.  nz in 3..1400, nx >= 3; the call allocates 4 bytes of scratch per
 * output sample.  The same local problem as the marching code, solved by
 * sweeps to the fixed point: identical results for order 1, within ~2.5e-4 s
 * for order 2 (whose marching result depends on the heap's acceptance
 * order).  KCIG_ERR_DEVICE if a source has no fixed point within max_iter. */
int kcig_eikods(const float *vel, int nz, int nx, float o1, float o2, float d1, float d2, float o3, float d3,
                const float *shots, int nshot, const kcig_eikods_opts *opt, float *time, float *tdl1,
                float *tds1, float *gradz, float *gradx, int *iters, void *stream);

/* The drop-in eikods2d (src/eikods2d.cpp:149-765) for 2-D velocity files:
 * same keys (in= out= tdl1= tds1= shotfile= gradz= gradx= order= b1= b2= br1=
 * br2= vel= l= zshot= yshot= xshot=), required outputs, error texts and
 * output headers; the tables are computed by kcig_eikods.  efmm=1,
 * plane-wave sources, tdl2=/tds2= and 3-D volumes return
 * KCIG_ERR_UNSUPPORTED.  Returns 0 or a KCIG_ERR_* (message logged). */
int kcig_run_eikods_cli(int argc, char **argv);

/* Tables for sources at depth zsrc and lateral positions p0 + k*dp
 * (k < npos), as the shot files of shotgen give them: kcig_eikods with
 * order 2, boxes (b1, b2), l = 1; deriv (may be NULL) receives tds1.
 * iterations bounds the sweep iterations (0 = 256). */
int kcig_eikonal_tables(const float *vel, int nz, int nx, float dz, float dx, float z0, float x0,
                        int npos, float p0, float dp, float zsrc, int b1, int b2, int iterations,
                        float *time, float *deriv, void *stream);

/* Self-test of the tensor-core operand layouts used by the traveltime
 * surrogate (no counterpart in the reference, which has no surrogate): for
 * two 128x128 BF16 row-major device matrices X and W writes, as FP32
 * [3][128][128], X W^T, X W and X^T W computed by tcgen05 MMAs.  *status
 * (device int) becomes 1 if the kernel gave up waiting for the tensor core. */
int kcig_tc_selftest(const void *X, const void *W, float *D, int *status, void *stream);

/* Forward modelling (kirchmig2d_cig adj=0, src/kirchmig2d_cig.cpp:1300-1351,
 * SERECKIRCH/src/kirmig.cpp:59-68): data [ns][nh][nt] from image
 * [ng][nx][nz] with the plan's geometry and parameters (host or device, as
 * `memory`).  The exact adjoint of kcig_migrate when direct_mute = 0 and
 * diff = 0 (the reference's forward branch applies neither; direct_mute=1
 * is rejected with the reference's message). */
int kcig_model(kcig_plan *plan, const float *image, float *data, int memory);

/* ---------------------------------------------------------------------------
 * Shots of uneven receiver count and trace length (the recursive-layer
 * workflow's windows, run_salt_adcig.sh:131-149, migrate such gathers one
 * file at a time).  Each shot is migrated as kirchmig2d_cig migrates a
 * one-shot file (ns = 1, so the source term of the antialias width uses
 * ds = 0): the image is the sum of those per-shot images.  The plan's
 * geometry supplies the image grid, the table axes, t0, dt and the largest
 * nt; its ns/nh/s0/ds/h0/dh are not used here. */
typedef struct {
    float sx;           /* source position (km)                                   */
    int nh;             /* receivers of this shot                                 */
    float h0, dh;       /* receiver axis h0 + k*dh: offsets (cmp=1) or positions   */
    int nt;             /* samples per trace of this shot, <= the plan's nt        */
    const float *data;  /* [nh][nt], host or device as `memory` says               */
    const float *h;     /* optional host array [nh]: the receiver axis values (in
                           place of h0 + k*dh), e.g. positions on a survey grid;
                           receivers with equal values then share one leg.  The
                           values are used as given (FP32), where h0 + k*dh is
                           rebuilt in FP64 for the continuous quantities      */
} kcig_shot;

/* Uploads the shots and every per-batch table to the device (batches sized
 * to the plan's scratch budget; receivers at the same position and spacing
 * share one leg within a batch). */
int kcig_shots_prepare(kcig_plan *plan, int nshots, const kcig_shot *shots, int memory);
/* Migrates the prepared shots into image [ng][nx][nz] (host or device).  The
 * launch sequence needs no host work; with kcig_plan_set_graph(plan, 1) it
 * is captured once into a CUDA graph (per image buffer) and replayed. */
int kcig_migrate_prepared(kcig_plan *plan, float *image, int memory);
int kcig_migrate_shots(kcig_plan *plan, int nshots, const kcig_shot *shots, float *image, int memory);
int kcig_plan_set_graph(kcig_plan *plan, int enable);
/* Image points x traces of the prepared shots (the throughput unit). */
long long kcig_shots_pairs(const kcig_plan *plan);
/* Times the summation kernel's tile variants (tile shape, shots per block)
 * on the first batch of the prepared shots and keeps the fastest for this
 * plan.  choice: the variant kept; ms: float[5], [0] the kept variant's
 * time, [1..4] each variant's (either may be NULL). */
int kcig_plan_autotune(kcig_plan *plan, int *choice, float *ms);
/* One CUDA graph over several prepared plans (e.g. the five depth windows of
 * the recursive workflow, each with its own tables, mute and image): create
 * runs every plan once directly, then captures the same sequence; launch
 * replays it asynchronously on `stream` (the caller synchronises).  The
 * plans, their prepared shots and the images must outlive the graph. */
typedef struct kcig_graph kcig_graph;
int kcig_graph_create(int nplans, kcig_plan *const *plans, float *const *images, kcig_graph **out);
int kcig_graph_launch(kcig_graph *graph, void *stream);
void kcig_graph_destroy(kcig_graph *graph);

/* ---------------------------------------------------------------------------
 * Learned traveltime surrogate (no counterpart in the reference, which reads
 * eikods2d tables).  A network T(xs, z, x) = Tb + residual_ms * 1e-3 * out
 * (or Tb * (1 + out) when residual_ms = 0), with Tb the closed-form first
 * arrival of the background medium v(z) = vref + vgrad * (z - zsrc) (straight
 * rays |(x, z) - (xs, zsrc)| / vref when vgrad = 0) and out a 4x128 SiLU MLP
 * on 64-frequency Fourier features of the normalised inputs, BF16
 * tensor-core GEMMs with FP32 accumulation.  Trained on a table volume by the
 * library's own forward and backward kernels (Adam, loss
 * mean((1000 (T - T_table))^2) in ms^2, fixed-order gradient sums: a run is
 * reproducible bit for bit); plugged into a plan it replaces the table
 * interpolation of every leg (kcig_plan_set_surrogate_options says which
 * leg quantities it supplies). */
typedef struct kcig_surrogate kcig_surrogate;
typedef struct {
    float lo[3], hi[3]; /* domain of (xs, z, x) in km, mapped to [-1, 1]      */
    float fmax;         /* highest Fourier frequency (half-waves over the domain) */
    float vref, zsrc;   /* background velocity at the source depth (km/s) and source depth (km) */
    float vgrad;        /* background velocity gradient (1/s): 0 = constant velocity */
    float residual_ms;  /* > 0: T = Tb + residual_ms * 1e-3 * out; 0: T = Tb * (1 + out) */
} kcig_surrogate_config;

int kcig_surrogate_nparams(void);
/* Seeded initial parameters on the current device. */
int kcig_surrogate_create(const kcig_surrogate_config *cfg, unsigned long long seed, kcig_surrogate **out);
void kcig_surrogate_destroy(kcig_surrogate *s);
/* Parameters as a host float vector of kcig_surrogate_nparams() entries:
 * W1 [128][384], W2..W4 [128][128] (row = output), b1..b4 [128], wo [128], bo.
 * set_params also resets the optimiser state. */
int kcig_surrogate_set_params(kcig_surrogate *s, const float *params);
int kcig_surrogate_get_params(const kcig_surrogate *s, float *params);
/* T and its derivatives at n points (all device float arrays). */
int kcig_surrogate_eval(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x, float *T,
                        float *dTdxs, float *dTdz, float *dTdx, void *stream);
/* Diagnostics of the tensor-core evaluation: the FP32 accumulators of the
 * first 128-point tile as device float [5][128][128] (row = point): layer 4
 * before its bias, then d tau/d h_3, d tau/d h_2, d tau/d h_1 before the
 * activation derivative, and d tau/d f of the xs features. */
int kcig_surrogate_eval_stages(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x,
                               float *stages, void *stream);
/* Loss of one batch (device float *loss) and its gradient with respect to
 * the parameters (device float grad[nparams]); no update. */
int kcig_surrogate_loss_grad(kcig_surrogate *s, int n, const float *xs, const float *z, const float *x,
                             const float *Ttrue, float *loss, float *grad, void *stream);
/* `steps` Adam steps on batches of `batch` (multiple of 128) points drawn
 * uniformly from the device table volume [npos][nx][nz] (positions
 * p0 + k*dp), learning rate decaying from lr to lr_final (cosine).  losses:
 * host float[steps] or NULL. */
int kcig_surrogate_train(kcig_surrogate *s, const float *table, int npos, float p0, float dp, int nz, int nx,
                         float z0, float dz, float x0, float dx, int steps, int batch, float lr, float lr_final,
                         unsigned long long seed, float *losses, void *stream);
/* Device time of the last kcig_migrate spent in leg-field computation (tables
 * or surrogate) and in the summation kernel, from CUDA events on the plan's
 * stream (ms). */
int kcig_plan_last_timing(const kcig_plan *plan, float *fields_ms, float *sum_ms);
/* Device ms of the trace prelude (mute, integration) in the last uncaptured
 * kcig_migrate_prepared. */
float kcig_plan_last_prelude_ms(const kcig_plan *plan);
/* Leg fields of the plan's source (src) and receiver (rcv) legs from
 * surrogates instead of tables (either may be NULL: that side uses its
 * tables).  The surrogates must outlive the plan's migrations. */
int kcig_plan_set_surrogate(kcig_plan *plan, kcig_surrogate *src, kcig_surrogate *rcv);
/* Which leg quantities a plan's surrogates supply (the traveltime always):
 *   angle KCIG_SG_ANGLE_FD (default): the gradient direction comes from the
 *     surrogate traveltime field by the tables' own centred differences and
 *     triangle smoothing (src/kirchmig2d_cig.cpp:130-152, :424-492), so a
 *     surrogate that matches the tables gives the tables' angles;
 *     KCIG_SG_ANGLE_NETWORK: from the network's input gradient dT/dz, dT/dx.
 *   tx KCIG_SG_TX_NETWORK (default): the source-position derivative (the
 *     antialias width, :1264-1266) from the network's backward pass;
 *     KCIG_SG_TX_TABLE: from the plan's sderiv/rderiv tables, interpolated as
 *     the table path does (the tables must be set and on the device). */
#define KCIG_SG_ANGLE_FD 0
#define KCIG_SG_ANGLE_NETWORK 1
#define KCIG_SG_TX_NETWORK 0
#define KCIG_SG_TX_TABLE 1
int kcig_plan_set_surrogate_options(kcig_plan *plan, int angle, int tx);

/* ---- ADCIG stitching of depth windows (src/layercom_cig.cpp) ------------ */

/* One depth window of layercom_cig's stitch loop (src/layercom_cig.cpp:
 * 473-533), on the device.  out: full-depth volume [n3][n2][n1] (device);
 * layer: the window's volume [n3][n2][end-start+1] (device), covering depth
 * rows start..end.  Every sample is scaled by layer_scale, times the
 * lateral taper of scalex_aper / scalex_scale when use_lateral (:455-466,
 * applied to every window but the first); non-finite products become 0 and
 * are counted in *nonfinite (host).  previous_end: last row of the window
 * above (-1 for the first window).  Rows shared with it keep the upper value
 * for the first overlap - blend rows and are blended over the other blend
 * rows with complementary raised-cosine weights, where blend =
 * min(stitch_blend, overlap) (stitch_blend = -1: the whole overlap).  The
 * other rows are written.  Synchronous on `stream`; the result equals the
 * reference's float arithmetic bit for bit. */
int kcig_stitch_window(float *out, int n1, int n2, int n3, const float *layer, int start, int end,
                       int previous_end, int stitch_blend, float layer_scale, int use_lateral, int scalex_aper,
                       double scalex_scale, long long *nonfinite, void *stream);

/* All nwin depth windows of one stitch in a single device pass (the loop of
 * src/layercom_cig.cpp:473-535 over every window): window k is layers[k]
 * [n3][n2][ends[k]-starts[k]+1] (device) covering depth rows
 * starts[k]..ends[k] (host arrays), scaled by scales[k] and, for k > 0 when
 * use_lateral, by the lateral taper; each window shares rows with the one
 * before it, as in kcig_stitch_window.  Every output sample is formed from
 * the windows covering its row in window order, so out equals nwin calls of
 * kcig_stitch_window on a zeroed volume bit for bit (rows no window covers
 * are 0); each window sample is read once and each output sample written
 * once, with one weight upload and one counter read-back for the whole
 * stitch.  nonfinite: host long long[nwin], the non-finite products of each
 * window.  Synchronous on `stream`. */
int kcig_stitch_windows(float *out, int n1, int n2, int n3, int nwin, const float *const *layers, const int *starts,
                        const int *ends, int stitch_blend, const float *scales, int use_lateral, int scalex_aper,
                        double scalex_scale, long long *nonfinite, void *stream);

/* The drop-in layercom_cig (src/layercom_cig.cpp:412-556): the same keys
 * (full_model= layer_image_base= layer_txt= output_file= nlayers= nangle=
 * scale= stitch_blend= scalex_aper= scalex_scale=), layer file rules,
 * checks, INFO lines, "ERROR: ..." texts and output header; the windows are
 * stitched on the device by kcig_stitch_window.  Returns 0 or KCIG_ERR_ARG
 * (the message printed to stderr). */
int kcig_run_layercom_cig_cli(int argc, char **argv);

/* ---- datuming between depth levels (greensol_auto, kirchdat2d_freq) ----- */

/* The datum-depth slice of a traveltime table (src/greensol_auto.cpp:71-93):
 * tgreen[igx1][igx2] = table[igx1][ix2][idatum], ix2 = (int)((ogx + igx2 dgx
 * - ox) / dx + 0.5), idatum = (int)((datum - oz) / dz + 0.5), every index in
 * the reference's float arithmetic.  table: [ngx][nx][nz], tgreen:
 * [ngx][ngx], both host (memory = KCIG_MEM_HOST) or both device
 * (KCIG_MEM_DEVICE: a gather kernel on `stream`, synchronous).  Errors:
 * "Datum out of range.", "Receiver table too small." (KCIG_ERR_ARG). */
int kcig_green_slice(const float *table, int nz, int nx, int ngx, float oz, float ox, float dz, float dx, float ogx,
                     float dgx, float datum, float *tgreen, int memory, void *stream);

/* Parameters of kirchdat2d_freq (src/kirchdat2d_frequency_cs.cpp:37-52 and
 * :1177-1290).  The input cube is [ns][nh][nt] (time fastest) with axes
 * (0, dt), (h0, dh), (s0, ds): h is the absolute receiver position when
 * cmp = 0 and the offset when cmp = 1.  Green's tables are square,
 * [nsg][nsg] (origin sg0, step dsg) and [nrg][nrg], indexed [cc][c] as the
 * reference reads them.  use_bf and the bf_* values are validated as the
 * reference validates them; the device always applies the exact operator
 * that the reference's butterfly (use_bf = 1) approximates. */
typedef struct kcig_datum_params {
    int nt, nh, ns;
    float dt, h0, dh, s0, ds;
    int nsg, nrg;
    float sg0, dsg, rg0, drg;
    float sdatum, rdatum;
    int aperture, taper, data_taper, cmp;
    float antialias, length;
    int use_bf, bf_p, bf_n_leaf, bf_panel_levels;
    float bf_amp_eps, bf_phase_tol;
} kcig_datum_params;

/* The reference's defaults (:1215-1263): aperture 50, taper 10,
 * data_taper 0, cmp 1, antialias 1, length 0.025, use_bf 1, bf_p 12,
 * bf_n_leaf 16, bf_panel_levels 1, bf_amp_eps 1e-20, bf_phase_tol 2; every
 * size and table field 0. */
int kcig_datum_params_init(kcig_datum_params *p);

/* FFT length and filter length of a run (:82-96, :1343-1346): nsam =
 * (int)(length / dt) + 2, nfft = the next power of two >= nt + ceil(max tau /
 * dt) + nsam. tables: host arrays. */
int kcig_datum_sizes(const kcig_datum_params *p, const float *stable, const float *rtable, int *nsam, int *nfft);

/* Datuming of one shot-gather cube from the recording surface to the datum
 * (src/kirchdat2d_frequency_cs.cpp:1327-1392): each trace reversed in time,
 * edge-tapered (data_taper) and transformed to nfft/2+1 frequencies; per
 * frequency the receiver-side Kirchhoff sum (:493-546) and then the
 * source-side sum (:548-672, the common-receiver walk for cmp = 1), each term
 * w(aperture taper, distance) x anti-alias weight x H(tau, w); back to time,
 * / nfft, reversed.  out: [ns][nh][nt]; interm (may be NULL): the
 * receiver-side result [ns][nh][nt], not reversed (the reference's interm=).
 * stable, rtable, in, out, interm: all host (KCIG_MEM_HOST) or all device
 * (KCIG_MEM_DEVICE) memory.  Synchronous on `stream`.  Errors with the
 * reference's texts ("cmp must be 0 or 1.", "Receiver table too small.",
 * "Source table too small.", ...: KCIG_ERR_ARG), KCIG_ERR_NOMEM when the
 * spectra do not fit the device.  The device buffers (the spectra: nfft/2+1
 * x ns x nh x 8 bytes, the chunk buffers, the cubes of host-memory calls) and
 * the cuFFT plans stay allocated for the next call on the same device: they
 * only grow, a call that cannot allocate frees them and tries once more, and
 * calls on one device run one at a time. */
int kcig_datum_freq(const kcig_datum_params *p, const float *stable, const float *rtable, const float *in, float *out,
                    float *interm, int memory, void *stream);

/* Frees the buffers and plans kcig_datum_freq keeps for the calling thread's
 * current device (the next call allocates them again). */
int kcig_datum_release(void);

/* Device time of the stages of the last kcig_datum_freq call on this thread
 * (ms): forward transforms, operator tables, receiver side, source side,
 * inverse transforms; and the number of kernel launches of the call. */
int kcig_datum_last_timing(float *ms5, int *launches);

/* The drop-in greensol_auto (src/greensol_auto.cpp:23-101) and
 * kirchdat2d_freq (src/kirchdat2d_frequency_cs.cpp:1177-1413): the same keys,
 * defaults, checks, INFO lines, "ERROR:" texts and output headers.  Return 0
 * or the KCIG_ERR_* code (the message printed to stderr). */
int kcig_run_greensol_auto_cli(int argc, char **argv);
int kcig_run_kirchdat2d_freq_cli(int argc, char **argv);

#ifdef __cplusplus
}
#endif
#endif /* KCIG_H */
