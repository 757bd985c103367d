/*
 * cosenu_b200.h -- C ABI of the B200 time-stepping path for COSEnu.
 *
 * The reference advances its state with the C++ member call
 * NuOsc::step_rk4() (src/nuosc.hpp:166 declaration, :320-348 body, called once
 * per iteration from src/main.cpp:175-177) on host arrays owned by NuOsc
 * (FieldVar, src/structures.hpp:5-37).  This header is the boundary that
 * replaces that call: a context owns the state in GPU memory, host arrays in
 * the reference's own layout go in and out, and the driver advances any number
 * of RK4 steps between analysis and snapshot events.
 *
 * Conventions
 *  - Every function returns COSENU_OK (0) or an error code; nothing calls
 *    exit() (the reference exits on bad input, src/parser.hpp:220-243,
 *    src/snaps.hpp:88-92).  cosenu_last_error() gives the message.
 *  - Host arrays use the reference layout: one array per component,
 *    v-major rows of length ld = nz + 2*gz, interior cell (i, j) at
 *    i*ld + j + gz (NuOsc::idx, src/nuosc.hpp:145-148).  Component order is
 *    ee, xx, ex_re, ex_im, bee, bxx, bex_re, bex_im (src/structures.hpp:6-13).
 *  - Work is queued on the context's CUDA stream; functions that return host
 *    data synchronise that stream first.
 *  - One host thread per context.
 */
#ifndef COSENU_B200_H
#define COSENU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COSENU_NCOMP 8
#define COSENU_ABI_VERSION 1

/* status codes */
enum {
    COSENU_OK = 0,
    COSENU_ERR_ARG = 1,       /* invalid argument or unsupported combination   */
    COSENU_ERR_CUDA = 2,      /* CUDA runtime error (message in last_error)    */
    COSENU_ERR_STATE = 3,     /* call out of order (e.g. step before upload)   */
    COSENU_ERR_NONFINITE = 4, /* NaN/Inf detected in the evolved state         */
    COSENU_ERR_NOMEM = 5      /* device allocation failed                       */
};

/* scheme: src/presets.hpp FV / FD (manage.py:167-173) */
enum { COSENU_FV = 0, COSENU_FD = 1 };
/* boundary: PERIODIC_BC / OPEN_BC (src/nuosc.hpp:214-277) */
enum { COSENU_PERIODIC = 0, COSENU_OPEN = 1 };
/* physics switches: VAC_OSC_ON, MAT_OSC_ON, COLL_OSC_ON, ADVEC_OFF
 * (src/rhs_fv.hpp:143-233, src/rhs_fd.hpp:31-126) */
enum { COSENU_VAC = 1u, COSENU_MAT = 2u, COSENU_COLL = 4u, COSENU_ADVEC_OFF = 8u };
/* FD advection stencil: ADVEC_CENTER_FD / ADVEC_UPWIND / lopsided
 * (src/rhs_fd.hpp:53-73) */
enum { COSENU_FD_CENTER = 0, COSENU_FD_UPWIND = 1, COSENU_FD_LOPSIDED = 2 };
/* arithmetic: plain FP64, or FP32-bulk: the RK4 stage increments stored in
 * FP32 over an FP64 base state, with FP64 velocity moments, accumulation and
 * diagnostics (FV evaluates its WENO7 weights in FP32 on FP64 differences) */
enum { COSENU_FP64 = 0, COSENU_FP32_BULK = 1 };

/* Simulation parameters.  Field meanings follow the job.config keys parsed by
 * Params (src/parser.hpp:46-256) plus the compile-time switches of
 * src/presets.hpp, which are run-time choices here. */
typedef struct cosenu_params {
    int nz, nvz;          /* grid (nz must be a multiple of 8)                   */
    int gz;               /* ghost width of the HOST layout (job.config "gz")    */
    double z0, z1;        /* spatial box                                          */
    double v0, v1;        /* velocity range                                       */
    double cfl;           /* dt = CFL*dz (src/nuosc.hpp:80)                       */
    double pmo, omega;    /* vacuum: mass ordering, omega (set_vac_pars)          */
    double theta_deg;     /* mixing angle in DEGREES (src/nuosc.hpp:135)          */
    double mu;            /* collective strength (set_collective_pars)            */
    int scheme;           /* COSENU_FV / COSENU_FD                                */
    int bc;               /* COSENU_PERIODIC / COSENU_OPEN                        */
    unsigned flags;       /* COSENU_VAC | COSENU_MAT | COSENU_COLL | ...          */
    int fd_advec;         /* COSENU_FD_* (FD only)                                */
    int ko_order;         /* 3 (KO_ORD_3) or 5 (FD only)                          */
    int precision;        /* COSENU_FP64 / COSENU_FP32_BULK                       */
    int device;           /* CUDA device ordinal                                  */
    int tile_z, tile_v;   /* kernel tile (0 = choose automatically)              */
} cosenu_params;

/* Fills p with the defaults of src/presets.hpp (periodic FV, vacuum and
 * collective terms on) and the grid of cosenu_configs.yaml. */
void cosenu_params_default(cosenu_params *p);

typedef struct cosenu_ctx cosenu_ctx;

/* Replaces NuOsc::NuOsc(Params) (src/nuosc.hpp:47-118) together with
 * set_vac_pars / set_collective_pars (src/nuosc.hpp:132-143): validates the
 * parameters and allocates the device state. */
int cosenu_create(const cosenu_params *p, cosenu_ctx **out);

/* Replaces NuOsc::~NuOsc (src/nuosc.hpp:119-130). */
int cosenu_destroy(cosenu_ctx *ctx);

/* Message of the last error on this context ("" if none); with ctx == NULL,
 * the last error of a failed cosenu_create on this thread. */
const char *cosenu_last_error(const cosenu_ctx *ctx);

/* NuOsc::set_vac_pars (src/nuosc.hpp:132-139, theta in degrees) and
 * NuOsc::set_collective_pars (src/nuosc.hpp:141-144): change the vacuum and
 * collective parameters of an existing context. */
int cosenu_set_vac_pars(cosenu_ctx *ctx, double pmo, double omega, double theta_deg);
int cosenu_set_collective_pars(cosenu_ctx *ctx, double mu);

/* Uses the given cudaStream_t for all later work (NULL: the context's own
 * stream).  The stream must belong to the context's device. */
int cosenu_set_stream(cosenu_ctx *ctx, void *cuda_stream);

/* Grid values the reference derives in its constructor (src/nuosc.hpp:78-96):
 * out = {dz, dv, dt, ct, st}. */
int cosenu_grid(const cosenu_ctx *ctx, double out[5]);

/* Host -> device copy of the evolved state v_stat (the arrays that
 * NuOsc::read_state / initialize fill, src/snaps.hpp:75-124).  comp[c] points
 * at component c in the reference layout with ghost width gz (>= 0).  Ghost
 * cells on the device are refilled (updateBufferZone, src/nuosc.hpp:212-278). */
int cosenu_upload(cosenu_ctx *ctx, const double *const comp[8], int gz);

/* Device -> host copy of the evolved state into the reference layout
 * (interior and gz ghost cells per side, as updateBufferZone would leave
 * them).  Synchronises. */
int cosenu_download(cosenu_ctx *ctx, double *const comp[8], int gz);

/* Initial angular profiles G0 (Profile, src/structures.hpp:116-130; read by
 * NuOsc::read_G0, src/snaps.hpp:153-183) used by the analysis. */
int cosenu_set_profile(cosenu_ctx *ctx, const double *G, const double *bG, int gz);

/* The initial state v_stat0 the analysis compares against (src/main.cpp:129-151).
 * cosenu_mark_state0 takes the current device state instead (no host copy). */
int cosenu_set_state0(cosenu_ctx *ctx, const double *const comp[8], int gz);
int cosenu_mark_state0(cosenu_ctx *ctx);

/* Replaces `nsteps` calls of NuOsc::step_rk4() (src/nuosc.hpp:320-348): each
 * RK4 step is four fused stage kernels (ghost fill, right-hand side of
 * src/rhs_fv.hpp or src/rhs_fd.hpp, stage combine).  Asynchronous. */
int cosenu_step(cosenu_ctx *ctx, int nsteps);

/* One RK4 stage (stage = 0..3, in order) -- the same kernels as cosenu_step,
 * exposed so that a caller can time the stages separately. */
int cosenu_step_stage(cosenu_ctx *ctx, int stage);

/* Captures the CUDA graphs cosenu_step launches (a chunk of 16 steps and a
 * single step, for each state-buffer parity the precision uses) now rather
 * than on first use, so that no later call pays for a capture.  Launches
 * nothing; a no-op where graphs are off (COSENU_NO_GRAPH=1). */
int cosenu_prepare_graphs(cosenu_ctx *ctx);

/* Waits for the context's stream.  COSENU_ERR_CUDA when a pipeline wait of a
 * stage kernel ran out of time (its results are not to be trusted); that
 * report repeats on every later check until a new state is uploaded or
 * initialised.  The reference has no such watchdog (its loops cannot stall). */
int cosenu_synchronize(cosenu_ctx *ctx);

/* Time limit of every wait inside the TMA-pipelined stage kernels (default
 * 2 s; range [1e-6, 600] s).  No counterpart in the reference. */
int cosenu_set_wait_limit(cosenu_ctx *ctx, double seconds);

/* Test hook for the watchdog (no counterpart in the reference): with on != 0
 * the TMA stage kernels issue no copies, so their consumers' waits run out
 * after the wait limit and the next check returns COSENU_ERR_CUDA.  Nothing
 * faults or hangs: every wait is bounded and nothing is in flight.
 * COSENU_ERR_STATE if the context does not use the TMA kernel. */
int cosenu_test_stall_pipeline(cosenu_ctx *ctx, int on);

/* Simulated time and number of completed RK4 steps (NuOsc::phy_time). */
int cosenu_time(const cosenu_ctx *ctx, double *phy_time, long long *steps);

/* Diagnostics of src/analysis.hpp, reduced on the device. */
typedef struct cosenu_diag {
    double dP_max;  /* max over cells of |d|P|| and |d|bP||  (dcon, :108-125)     */
    double avdP;    /* sum |d|P|| G / sum G                                        */
    double avbdP;   /* sum |d|bP|| bG / sum bG                                     */
    double M0;      /* |M0|                              (cal_Mn n = 0, :50-67)   */
    double M0_e1, M0_e2, M0_e3;
    double Pee;     /* sum ee / sum ee0                   (surv_prob, :169-182)   */
    double Pbee;    /* sum bee / sum bee0                                          */
    double trace;   /* sum (ee + xx) dz dv  (conserved)                            */
    double btrace;  /* sum (bee + bxx) dz dv  (conserved)                          */
    double eln;     /* sum (ee - bee) dz dv                                        */
} cosenu_diag;

/* Replaces NuOsc::analyse + surv_prob (src/analysis.hpp:3-25, 134-185)
 * without copying the state to the host.  Needs set_profile and state0.
 * Synchronises.  Returns COSENU_ERR_NONFINITE if the state holds NaN/Inf. */
int cosenu_analyse(cosenu_ctx *ctx, cosenu_diag *out);

/* Angle-resolved survival probabilities P_ee(v) = sum_z ee / sum_z ee0 and
 * the same for nubar (arrays of nvz). Synchronises. */
int cosenu_pee_v(cosenu_ctx *ctx, double *pee, double *pbee);

/* On-device initial conditions.  cosenu_init_seeded: G = g(v,1,sig_nu),
 * bG = alpha*g(v,1,sig_nubar) (g of src/miscellaneous_funcs.hpp:57-62) and a
 * per-cell Philox-4x32-10 draw of (Re, Im) ex in [-amp, amp] for nu and nubar,
 * shaped like src/initialize.hpp:30-38.  cosenu_init_reference: the
 * reference's own NuOsc::initialize() (src/initialize.hpp:6-47).  Both set
 * the profile and state0 as well and reset the time to zero. */
int cosenu_init_seeded(cosenu_ctx *ctx, uint64_t seed, uint32_t instance, double sig_nu,
                       double sig_nubar, double alpha, double amp);
int cosenu_init_reference(cosenu_ctx *ctx, double perturbation_size);

/* Device addresses of the evolved state for zero-copy use (e.g. from a
 * framework tensor): comp[c] points at interior cell (0,0) of component c,
 * rows are `ld` elements apart.  Valid until the next cosenu_* call that
 * steps.  The pointed-to type is double (COSENU_FP64 and FP32_BULK keep the
 * base state in FP64). */
int cosenu_device_state(cosenu_ctx *ctx, double *comp[8], int *ld);

/* Device <-> device variants of upload/download: comp[c] are device
 * pointers with row pitch `ld` elements, interior only. */
int cosenu_upload_device(cosenu_ctx *ctx, const double *const comp[8], int ld);
int cosenu_download_device(cosenu_ctx *ctx, double *const comp[8], int ld);

/* Snapshots for output written while stepping continues.  The reference's
 * dump_rho and write_state (src/snaps.hpp:6-39,187-218) read the state on the
 * host at the dump step, which stops the run for the whole file write.
 * cosenu_snapshot queues on the context's stream a device copy of the current
 * state (taken before any later step touches it), then, on a second stream,
 * its copy to pinned host memory, and returns at once; *steps (if not NULL)
 * receives the number of RK4 steps the snapshot is taken after.
 * cosenu_snapshot_wait blocks until that host copy is complete and stores in
 * *data the interior cells: 8 components of nvz rows of nz doubles, cell
 * (v, z) of component c at data[((size_t)c * nvz + v) * nz + z].  The data
 * stay valid until the next cosenu_snapshot or cosenu_destroy.
 * cosenu_snapshot_wait touches only the snapshot's own buffers and events and
 * sets no error text, so it may be called from another host thread while this
 * one keeps stepping.  The two buffers (device and pinned host, 64 * nz * nvz
 * bytes each) are allocated by the first cosenu_snapshot. */
int cosenu_snapshot(cosenu_ctx *ctx, long long *steps);
int cosenu_snapshot_wait(cosenu_ctx *ctx, const double **data);

/* ---------------------------------------------------------------------------
 * Ensembles (no counterpart in the reference, which runs one configuration per
 * process: manage.py:361-428 submits one job per (nz, nvz, CFL)).  Many
 * independent simulations of uneven nz, nvz and physics advance together:
 * one launch per RK4 stage covers every member with steps left.  Members are
 * ordinary contexts (cosenu_batch_member) for initial conditions, analysis and
 * download.  Members must share scheme, FD variant, precision and device, and
 * need nz % 32 == 0, nvz <= 1024. */
typedef struct cosenu_batch cosenu_batch;
int cosenu_batch_create(int n, const cosenu_params *params, cosenu_batch **out);
int cosenu_batch_destroy(cosenu_batch *b);
const char *cosenu_batch_last_error(const cosenu_batch *b);
int cosenu_batch_size(const cosenu_batch *b);
/* Runs the ensemble (and its members) on the given cudaStream_t. */
int cosenu_batch_set_stream(cosenu_batch *b, void *cuda_stream);
cosenu_ctx *cosenu_batch_member(cosenu_batch *b, int i);
/* cosenu_init_seeded for every member (instance number = member index). */
int cosenu_batch_init_seeded(cosenu_batch *b, const uint64_t *seeds, const double *sig_nu,
                             const double *sig_nubar, const double *alpha, double amp);
/* Advances member i by nsteps[i] RK4 steps (asynchronous). */
int cosenu_batch_run(cosenu_batch *b, const long long *nsteps);
int cosenu_batch_synchronize(cosenu_batch *b);
/* Times trial_steps ensemble steps for each candidate kernel family and tile
 * (TMA-pipelined; register-tiled with z tile 32/16/8 and a v tile per nvz
 * class) and keeps the fastest; member states are restored.  A text report of
 * the timings goes to `report` (may be NULL). */
int cosenu_batch_autotune(cosenu_batch *b, int trial_steps, char *report, size_t report_len);
/* Current / explicit kernel choice (use_tma 1: TMA-pipelined; 0: register-
 * tiled with z tile tz and v tile tv_per_member[i]). */
int cosenu_batch_config(const cosenu_batch *b, int *use_tma, int *tz, int *tv_per_member);
int cosenu_batch_set_config(cosenu_batch *b, int use_tma, int tz, const int *tv_per_member);

/* ---------------------------------------------------------------------------
 * Surrogate network (no counterpart in the reference): fully connected,
 * n_in -> n_hidden x n_hidden_layers -> n_out with GELU between layers, BF16
 * weights and activations on the tensor cores with FP32 accumulation, FP32
 * master weights trained by AdamW on the mean-squared error.  Parameters are
 * one flat FP32 vector: for each layer W [out][in] (in padded to a multiple
 * of 16, padding columns zero) then b [out].  n_hidden must be a multiple of
 * 16 and n_out of 8.  The GEMMs run on tcgen05 (tensor-memory accumulator);
 * with the environment variable COSENU_MLP_GEMM=mma at cosenu_mlp_create the
 * net uses the warp-level mma.sync kernel instead (the same sums in the same
 * order, kept for comparison).  A GEMM whose bounded internal wait expires
 * makes the next synchronising call return COSENU_ERR_CUDA. */
typedef struct cosenu_mlp cosenu_mlp;
int cosenu_mlp_create(int n_in, int n_hidden, int n_hidden_layers, int n_out, uint64_t seed,
                      int device, cosenu_mlp **out);
int cosenu_mlp_destroy(cosenu_mlp *net);
const char *cosenu_mlp_last_error(const cosenu_mlp *net);
int cosenu_mlp_num_params(const cosenu_mlp *net, size_t *n);
int cosenu_mlp_get_params(cosenu_mlp *net, float *host);
int cosenu_mlp_set_params(cosenu_mlp *net, const float *host);
/* y [rows][n_out] for x [rows][n_in] (host arrays). */
int cosenu_mlp_forward(cosenu_mlp *net, const float *x_host, int rows, float *y_host);
/* Loss 1/(rows*n_out) sum (y - t)^2 and its gradient (flat, like the params). */
int cosenu_mlp_loss_grad(cosenu_mlp *net, const float *x_host, const float *t_host, int rows,
                         float *loss, float *grad_host);
/* Training data held on the device, then minibatch AdamW epochs over it. */
int cosenu_mlp_set_data(cosenu_mlp *net, const float *x_host, const float *t_host, int n);
int cosenu_mlp_train(cosenu_mlp *net, int epochs, int batch, float lr, float weight_decay,
                     float beta1, float beta2, float eps, uint64_t shuffle_seed, float *epoch_loss);
/* Timing mode: with on != 0 every later launch is bracketed by CUDA events and
 * its device time added to one of three classes, read by cosenu_mlp_timing as
 * ms[0] GEMMs (forward, dX, dW), ms[1] elementwise kernels (gather, MSE,
 * GELU backward, bias column sums), ms[2] AdamW updates.  Setting the mode
 * clears the totals. */
int cosenu_mlp_set_timing(cosenu_mlp *net, int on);
int cosenu_mlp_timing(const cosenu_mlp *net, double ms[3]);

/* For callers that must not allocate device memory (a host application whose
 * device memory all comes from its own pool, or a loop that cannot afford the
 * device synchronisation cudaMalloc/cudaFree may cause).  No counterpart in the
 * reference.  Advances a state the caller holds in device memory by `nsteps`
 * RK4 steps without any device allocation: state[c] points at component c,
 * interior cell (v, z) at state[c][v*ld + z] (no ghost cells; ld >= nz), read
 * and overwritten in place; p gives the grid and physics as for cosenu_create.
 * Working memory is one fixed device array inside the library (20.5 MB, held by
 * every GPU that loads the library until exit): grids need
 * nvz * (nz + 32 rounded up to a multiple of 16) <= 69632 and nz <= 16384
 * (the 1024 x 64 grid fits), and p->tile_v <= 64 (0 picks min(nvz, 64));
 * larger grids or v tiles return COSENU_ERR_ARG with the limit in
 * cosenu_last_error(NULL).  The first call on a device (and the first after
 * the device's context was re-created, e.g. by cudaDeviceReset) looks up that
 * array's address; make it before any stream capture.  Calls share the
 * array, so calls whose GPU work overlaps race; order them.  Work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream) and not waited for. */
int cosenu_step_noalloc(const cosenu_params *p, double *const state[8], int ld, int nsteps,
                        void *stream);

/* Number of kernel launches one cosenu_step(ctx, 1) issues. */
int cosenu_launches_per_step(const cosenu_ctx *ctx);

/* Tile shape in use (z cells x v rows per thread block). */
int cosenu_tile(const cosenu_ctx *ctx, int *tile_z, int *tile_v);

/* Bytes of device memory held by the context. */
int cosenu_device_bytes(const cosenu_ctx *ctx, size_t *bytes);

#ifdef __cplusplus
}
#endif
#endif /* COSENU_B200_H */
