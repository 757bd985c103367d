// C ABI of the B200 RK4 path (declarations and reference citations in
// include/cosenu_b200.h).  A context owns the device state of one simulation
// and replays the four stage kernels of an RK4 step, captured once into CUDA
// graphs, for as many steps as the driver asks for.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

namespace cosenu {
int diag_blocks();
int diag_slots();
cudaError_t launch_diag(const double *Y, const double *S0, const double *G, const double *bG,
                        long long cs, int ld, int nz, int nvz, double dz, double dv, double *part,
                        double *out, cudaStream_t s);
cudaError_t launch_pee_v(const double *Y, const double *S0, long long cs, int ld, int nz, int nvz,
                         double *out, cudaStream_t s);
cudaError_t launch_init_seeded(double *Y, double *G, double *bG, const double *Gv,
                               const double *bGv, long long cs, int ld, int nz, int nvz,
                               uint64_t seed, uint32_t instance, double amp, cudaStream_t s);
cudaError_t launch_init_reference(double *Y, double *G, double *bG, const double *Gv,
                                  const double *bGv, const double *ez, const double *ez_,
                                  long long cs, int ld, int nz, int nvz, cudaStream_t s);
}  // namespace cosenu

using namespace cosenu;

// message for cosenu_last_error(NULL): failures that have no context
thread_local std::string g_create_error;

static const int GRAPH_CHUNK = 16;  // even
static_assert(GRAPH_CHUNK % 2 == 0, "a chunk leaves the buffer parity unchanged");

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
            return COSENU_ERR_CUDA;                                                           \
        }                                                                                     \
    } while (0)

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int fail(cosenu_ctx *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

// normalised Gaussian angular profile, src/miscellaneous_funcs.hpp:57-62
double gprof(double v, double v0, double sigma)
{
    double e = (v - v0) * (v - v0) / (2.0 * sigma * sigma);
    double N = sigma * sqrt(M_PI / 2.0) *
               (erf((1.0 + v0) / sigma / sqrt(2.0)) + erf((1.0 - v0) / sigma / sqrt(2.0)));
    return exp(-e) / N;
}

int alloc(cosenu_ctx *ctx, void **p, size_t n)
{
    cudaError_t e = cudaMalloc(p, n);
    if (e != cudaSuccess) {
        ctx->err = "cudaMalloc(" + std::to_string(n) + " B): " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? COSENU_ERR_NOMEM : COSENU_ERR_CUDA;
    }
    ctx->bytes += n;
    return COSENU_OK;
}

void choose_tile(cosenu_ctx *ctx, int layout = 0)
{
    const cosenu_params &p = ctx->p;
    const char *kenv = getenv("COSENU_KERNEL");
    bool force_ldg = kenv && std::string(kenv) == "ldg";
    bool force_tma = kenv && std::string(kenv) == "tma";
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p.device);
    if (p.nz % 32 == 0 && p.nvz <= tma_max_nvz() &&
        (layout == 1 || ((p.nz / 32 >= nsm || force_tma) && p.tile_z == 0 && p.tile_v == 0 &&
                         !force_ldg))) {
        // TMA path (grids with at least one 32-cell z tile per SM): tiles span all rows
        ctx->use_tma = true;
        ctx->tz = 32;
        ctx->tv = p.nvz;
        ctx->nvt = 1;
        return;
    }
    int tz = p.tile_z;
    if (tz == 0) tz = (p.nz % 32 == 0) ? 32 : (p.nz % 16 == 0 ? 16 : 8);
    int rp = NTHREADS / tz;
    int tv = p.tile_v;
    if (tv == 0) {
        tv = std::min(p.nvz, 64);
        // enough blocks to fill 148 SMs several times over
        while (tv > rp && (long long)(p.nz / tz) * ((p.nvz + tv - 1) / tv) < 8 * 148) tv /= 2;
        if (tv < 1) tv = 1;
    }
    ctx->tz = tz;
    ctx->tv = tv;
    ctx->nvt = (p.nvz + tv - 1) / tv;
}

StageArgs stage_args(const cosenu_ctx *ctx, int stage, int par)
{
    if (par < 0) par = ctx->ypar;
    StageArgs a{};
    a.vz = ctx->vz;
    a.rowfac = ctx->rowfac;
    a.Hm = ctx->Hm;
    a.cs = ctx->cs;
    a.nz = ctx->p.nz;
    a.nvz = ctx->p.nvz;
    a.ld = ctx->ld;
    a.tv = ctx->tv;
    a.nvt = ctx->nvt;
    a.H = ctx->H;
    a.bc = ctx->p.bc;
    a.flags = (int)ctx->p.flags;
    a.fd_advec = ctx->p.fd_advec;
    a.ko_order = ctx->p.ko_order;
    a.dt = ctx->dt;
    a.dv = ctx->dv;
    a.v0 = ctx->p.v0;
    a.dz = ctx->dz;
    a.mu = ctx->p.mu;
    a.ct = ctx->ct;
    a.st = ctx->st;
    a.pmo = ctx->p.pmo;
    // omega = 0 (or no mass-ordering sign): the vacuum terms are exact zeros,
    // and the stage kernels skip them
    if ((a.ct == 0.0 && a.st == 0.0) || a.pmo == 0.0) a.flags &= ~F_VAC;
    const double ko = 1.0e-1;  // src/nuosc.hpp:60
    a.ko_eps = ctx->p.ko_order == 5 ? -ko / ctx->dz / 64.0 : -ko / ctx->dz / 16.0;
    a.wait_ns = ctx->wait_ns;
    a.stall = ctx->stall;
    double *Y = ctx->Yb[par];
    a.Y = Y;
    if (!ctx->fp32) {
        // FP64 stage values; the accumulator lives in Yb[1] (par is always 0)
        a.A = ctx->Yb[1];
        switch (stage) {
        case 1: a.X = Y; a.U = ctx->U0; a.Min = ctx->M[2]; a.Mout = ctx->M[0]; break;
        case 2: a.X = ctx->U0; a.U = ctx->U1; a.Min = ctx->M[0]; a.Mout = ctx->M[1]; break;
        case 3: a.X = ctx->U1; a.U = ctx->U0; a.Min = ctx->M[1]; a.Mout = ctx->M[0]; break;
        case 4: a.X = ctx->U0; a.U = Y; a.Min = ctx->M[0]; a.Mout = ctx->M[2]; break;
        }
    } else {
        // FP32-bulk increments D1, D2, D3 in U0, U1, U2; the new state goes to
        // the other FP64 buffer
        a.T1 = static_cast<const float *>(ctx->U0);
        a.T2 = static_cast<const float *>(ctx->U1);
        switch (stage) {
        case 1: a.X = Y; a.U = ctx->U0; a.Min = ctx->M[2]; a.Mout = ctx->M[0]; break;
        case 2: a.X = ctx->U0; a.U = ctx->U1; a.Min = ctx->M[0]; a.Mout = ctx->M[1]; break;
        case 3: a.X = ctx->U1; a.U = ctx->U2; a.Min = ctx->M[1]; a.Mout = ctx->M[0]; break;
        case 4: a.X = ctx->U2; a.U = ctx->Yb[par ^ 1]; a.Min = ctx->M[0]; a.Mout = ctx->M[2]; break;
        }
    }
    return a;
}

void flip(cosenu_ctx *ctx)
{
    if (!ctx->fp32) return;
    ctx->ypar ^= 1;
    ctx->Y = ctx->Yb[ctx->ypar];
    ctx->A = ctx->Yb[ctx->ypar ^ 1];
}

// Launches one stage; after stage 4 of the FP32-bulk form the state is in the
// other buffer.
cudaError_t launch_stage(cosenu_ctx *ctx, int stage, cudaStream_t s)
{
    StageArgs a = stage_args(ctx, stage, -1);
    cudaError_t e;
    if (ctx->use_tma) {
        int nblk = std::min(ctx->p.nz / tma_box_tile(),
                            tma_blocks_per_sm(ctx->p.scheme) * ctx->nsm);
        const CUtensorMap *mX, *mY, *mA, *mB;
        if (!ctx->fp32) {
            // stage 3 reads U at its own cells in the A slot
            mX = stage == 1 ? &ctx->mYb40[0] : (stage == 3 ? &ctx->mU1_40 : &ctx->mU0_40);
            mY = &ctx->mY32;
            mA = stage == 3 ? &ctx->mU0_32 : &ctx->mA32;
            mB = &ctx->mY32;  // unused
        } else {
            // input Y + D with the halo; stage 4 also reads D1, D2 at its own cells
            mY = stage == 4 ? &ctx->mYb40s4[ctx->ypar] : &ctx->mYb40[ctx->ypar];
            mX = stage == 1 ? &ctx->mYb40[ctx->ypar]
                            : (stage == 2 ? &ctx->mU0_40 : (stage == 3 ? &ctx->mU1_40
                                                                       : &ctx->mU2_40));
            mA = &ctx->mU0_32;
            mB = &ctx->mU1_32;
        }
        e = launch_rk4_stage_tma(*mX, *mY, *mA, *mB, a, ctx->p.scheme, stage, ctx->fp32,
                                 ctx->err_flag, nblk, s);
    } else {
        e = launch_rk4_stage(a, ctx->p.scheme, stage, ctx->tz, ctx->fp32, s);
    }
    if (e == cudaSuccess && stage == 4) flip(ctx);
    return e;
}

// Reads the device error word; non-zero means a bounded wait in a stage
// kernel expired (the results of that launch are not to be trusted).  The
// word stays set, and every later check reports it, until a new state is
// uploaded or initialised (prepare_state clears it).
int check_err_flag(cosenu_ctx *ctx)
{
    if (!ctx->use_tma) return COSENU_OK;
    int h = 0;
    CK(cudaMemcpyAsync(&h, ctx->err_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h != 0) {
        ctx->err = "stage kernel pipeline wait timed out (code " + std::to_string(h) + ")";
        return COSENU_ERR_CUDA;
    }
    return COSENU_OK;
}

cudaError_t launch_steps(cosenu_ctx *ctx, int n, cudaStream_t s)
{
    for (int i = 0; i < n; ++i)
        for (int st = 1; st <= 4; ++st) {
            cudaError_t e = launch_stage(ctx, st, s);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

// Captures `n` steps from the current buffer parity into an executable graph
// (on a private stream); the context's parity is left as it was, since nothing
// ran yet.
cudaError_t capture(cosenu_ctx *ctx, int n, cudaGraphExec_t *out)
{
    struct Restore {
        cosenu_ctx *c;
        int par;
        ~Restore()
        {
            if (c->ypar != par) flip(c);
        }
    } restore{ctx, ctx->ypar};
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t le = launch_steps(ctx, n, cs);
        e = cudaStreamEndCapture(cs, &g);
        if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return e;
}

// Refreshes ghosts and input moments of Y after Y changed outside the stages;
// a new state also clears the error word of an earlier expired wait.
int prepare_state(cosenu_ctx *ctx)
{
    if (ctx->err_flag) CK(cudaMemsetAsync(ctx->err_flag, 0, sizeof(int), ctx->stream));
    CK(launch_ghost_fill(ctx->Y, ctx->cs, ctx->ld, ctx->p.nz, ctx->p.nvz, ctx->H, ctx->p.bc,
                         ctx->stream));
    if (ctx->p.flags & COSENU_COLL)
        CK(launch_moments(ctx->Y, ctx->M[2], ctx->vz, ctx->cs, ctx->ld, ctx->p.nz, ctx->p.nvz,
                          ctx->tz, ctx->tv, ctx->stream));
    ctx->have_state = true;
    ctx->next_stage = 0;
    return COSENU_OK;
}

int copy_planes_h2d(cosenu_ctx *ctx, double *dst, const double *const *src, int ncomp, int gz)
{
    const int nz = ctx->p.nz, nvz = ctx->p.nvz;
    for (int c = 0; c < ncomp; ++c) {
        if (!src[c]) return fail(ctx, COSENU_ERR_ARG, "null component pointer");
        CK(cudaMemcpy2DAsync(dst + (long long)c * ctx->cs + HP, (size_t)ctx->ld * 8, src[c] + gz,
                             (size_t)(nz + 2 * gz) * 8, (size_t)nz * 8, nvz,
                             cudaMemcpyHostToDevice, ctx->stream));
    }
    return COSENU_OK;
}

void drop_graphs(cosenu_ctx *ctx)
{
    for (int k = 0; k < 2; ++k) {
        if (ctx->g1[k]) cudaGraphExecDestroy(ctx->g1[k]);
        if (ctx->gN[k]) cudaGraphExecDestroy(ctx->gN[k]);
        ctx->g1[k] = ctx->gN[k] = nullptr;
    }
}

}  // namespace

extern "C" {

void cosenu_params_default(cosenu_params *p)
{
    std::memset(p, 0, sizeof(*p));
    p->nz = 2400;
    p->nvz = 32;
    p->gz = 4;
    p->z0 = -600.0;
    p->z1 = 600.0;
    p->v0 = -1.0;
    p->v1 = 1.0;
    p->cfl = 0.4;
    p->pmo = 1.0;
    p->omega = 1e-2;
    p->theta_deg = 37.0;
    p->mu = 1.0;
    p->scheme = COSENU_FV;
    p->bc = COSENU_PERIODIC;
    p->flags = COSENU_VAC | COSENU_COLL;
    p->fd_advec = COSENU_FD_CENTER;
    p->ko_order = 3;
    p->precision = COSENU_FP64;
}

const char *cosenu_last_error(const cosenu_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int cosenu_create(const cosenu_params *pp, cosenu_ctx **out) { return ctx_create(pp, out, 0); }

}  // extern "C"

int ctx_create(const cosenu_params *pp, cosenu_ctx **out, int layout)
{
    g_create_error.clear();
    if (!pp || !out) {
        g_create_error = "null argument";
        return COSENU_ERR_ARG;
    }
    *out = nullptr;
    const cosenu_params &p = *pp;
    std::string why;
    if (p.nz < 16 || p.nz % 8 != 0) why = "nz must be a multiple of 8 and >= 16";
    else if (p.nvz < 1) why = "nvz must be >= 1";
    else if (p.gz < 0 || p.gz > HP) why = "gz must be in [0, 16]";
    else if (p.scheme != COSENU_FV && p.scheme != COSENU_FD) why = "unknown scheme";
    else if (p.bc != COSENU_PERIODIC && p.bc != COSENU_OPEN) why = "unknown boundary";
    else if (p.precision != COSENU_FP64 && p.precision != COSENU_FP32_BULK) why = "unknown precision";
    else if (p.fd_advec < 0 || p.fd_advec > 2) why = "unknown FD advection stencil";
    else if (p.ko_order != 3 && p.ko_order != 5) why = "ko_order must be 3 or 5";
    else if (!(p.z1 > p.z0) || !(p.v1 > p.v0) || !(p.cfl > 0)) why = "empty box or non-positive CFL";
    else if (p.tile_z != 0 && p.tile_z != 8 && p.tile_z != 16 && p.tile_z != 32) why = "tile_z must be 8, 16 or 32";
    else if (p.tile_z != 0 && p.nz % p.tile_z != 0) why = "tile_z must divide nz";
    else if (p.tile_v < 0 || p.tile_v > MAX_TV) why = "tile_v must be in [0, 256]";
    if (!why.empty()) {
        g_create_error = why;
        return COSENU_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_create_error = "no CUDA device";
        return COSENU_ERR_CUDA;
    }
    if (p.device < 0 || p.device >= ndev) {
        g_create_error = "device ordinal out of range";
        return COSENU_ERR_ARG;
    }
    cosenu_ctx *ctx = new cosenu_ctx();
    ctx->p = p;
    DeviceGuard dg(p.device);
    ctx->fp32 = p.precision == COSENU_FP32_BULK;
    ctx->ld = padded_ld(p.nz);
    ctx->cs = (long long)p.nvz * ctx->ld;
    ctx->H = std::max(4, p.gz);
    choose_tile(ctx, layout);
    if (layout == 1 && !ctx->use_tma) {
        g_create_error = "ensemble members need nz % 32 == 0 and nvz <= 1024";
        delete ctx;
        return COSENU_ERR_ARG;
    }
    // grid exactly as NuOsc::NuOsc and set_vac_pars (src/nuosc.hpp:78-96,132-138)
    ctx->dz = (p.z1 - p.z0) / p.nz;
    ctx->dv = (p.v1 - p.v0) / (p.nvz);
    ctx->dt = p.cfl * ctx->dz;
    double th = p.theta_deg * M_PI / 180.0;
    ctx->ct = (1.0 / 2.0) * p.omega * cos(2.0 * th);
    ctx->st = (1.0 / 2.0) * p.omega * sin(2.0 * th);
    ctx->h_Z.resize(p.nz);
    ctx->h_Hm.resize(p.nz);
    for (int j = 0; j < p.nz; ++j) {
        ctx->h_Z[j] = p.z0 + (j + 0.5) * ctx->dz;
        ctx->h_Hm[j] = -1.0e-3 * (ctx->h_Z[j] + 600.0);
    }
    ctx->h_vz.resize(p.nvz);
    ctx->h_rowfac.resize(p.nvz);
    for (int i = 0; i < p.nvz; ++i) {
        double v = p.v0 + (i + 0.5) * ctx->dv;
        ctx->h_vz[i] = v;
        int sv = (0.0 < v) - (v < 0.0);
        double f;
        if (p.scheme == COSENU_FV) f = -v / ctx->dz;                       // rhs_fv.hpp:145
        else if (p.fd_advec == COSENU_FD_CENTER) f = -v / (12 * ctx->dz);  // rhs_fd.hpp:57
        else if (p.fd_advec == COSENU_FD_UPWIND) f = -sv * v / (12 * ctx->dz);
        else f = sv * v / (12 * ctx->dz);
        ctx->h_rowfac[i] = f;
    }

    int rc;
    const size_t plane = (size_t)ctx->cs * sizeof(double);
    const size_t state = plane * NCOMP;
    const size_t ustate = ctx->fp32 ? state / 2 : state;  // U0, U1 (and U2: FP32-bulk)
    // ensemble members may later be re-tiled down to 8-row v tiles
    ctx->mom_nvt_cap = layout == 1 ? (p.nvz + 7) / 8 : ctx->nvt;
    const size_t mom = (size_t)ctx->mom_nvt_cap * NMOM * p.nz * sizeof(double);
#define AL(ptr, n)                                                              \
    if ((rc = alloc(ctx, (void **)&(ptr), (n))) != COSENU_OK) {                 \
        g_create_error = ctx->err;                                              \
        cosenu_destroy(ctx);                                                    \
        return rc;                                                              \
    }
    AL(ctx->Yb[0], state);
    AL(ctx->Yb[1], state);
    ctx->Y = ctx->Yb[0];
    ctx->A = ctx->Yb[1];
    AL(ctx->S0, state);
    AL(ctx->U0, ustate);
    AL(ctx->U1, ustate);
    if (ctx->fp32) AL(ctx->U2, ustate);
    AL(ctx->G, plane);
    AL(ctx->bG, plane);
    for (int k = 0; k < 3; ++k) AL(ctx->M[k], mom);
    AL(ctx->vz, p.nvz * sizeof(double));
    AL(ctx->rowfac, p.nvz * sizeof(double));
    AL(ctx->Hm, p.nz * sizeof(double));
    AL(ctx->diag_part, (size_t)diag_blocks() * diag_slots() * sizeof(double));
    AL(ctx->diag_out, 16 * sizeof(double));
    AL(ctx->pee, 2 * (size_t)p.nvz * sizeof(double));
    AL(ctx->tmp, (2 * (size_t)p.nvz + 2 * (size_t)p.nz) * sizeof(double));
    AL(ctx->err_flag, 64);
#undef AL
    auto bail = [&](void) {
        g_create_error = ctx->err;
        cosenu_destroy(ctx);
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMallocHost((void **)&ctx->h_pinned, 4096 + 2 * (size_t)p.nvz * 8)) != cudaSuccess) {
        ctx->err = cudaGetErrorString(e);
        bail();
        return COSENU_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    // zero everything once so ghost pads and unused partials are defined
    for (void *q : {(void *)ctx->Yb[0], (void *)ctx->Yb[1], (void *)ctx->S0})
        cudaMemsetAsync(q, 0, state, ctx->stream);
    for (void *q : {ctx->U0, ctx->U1, ctx->U2})
        if (q) cudaMemsetAsync(q, 0, ustate, ctx->stream);
    cudaMemsetAsync(ctx->G, 0, plane, ctx->stream);
    cudaMemsetAsync(ctx->bG, 0, plane, ctx->stream);
    for (int k = 0; k < 3; ++k) cudaMemsetAsync(ctx->M[k], 0, mom, ctx->stream);
    cudaMemcpyAsync(ctx->vz, ctx->h_vz.data(), p.nvz * 8, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(ctx->rowfac, ctx->h_rowfac.data(), p.nvz * 8, cudaMemcpyHostToDevice,
                    ctx->stream);
    cudaMemcpyAsync(ctx->Hm, ctx->h_Hm.data(), p.nz * 8, cudaMemcpyHostToDevice, ctx->stream);
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        ctx->err = cudaGetErrorString(e);
        bail();
        return COSENU_ERR_CUDA;
    }
    cudaMemsetAsync(ctx->err_flag, 0, 64, ctx->stream);
    if (ctx->use_tma) {
        // box rows follow the row count of the stages that read each map (the TMA
        // kernel's rows(): 12 for the latency-bound FD stages, else 8)
        const int ub = ctx->fp32 ? 4 : 8, bx = tma_box_x(8), bxu = tma_box_x(ub),
                  bt = tma_box_tile(), rw = tma_box_rows(p.scheme, true),
                  rn = tma_box_rows(p.scheme, false), ru = ctx->fp32 ? rw : rn;
        int r = make_state_map(&ctx->mYb40[0], ctx->Yb[0], 8, ctx->ld, p.nvz, ctx->cs, bx, rw);
        if (!r) r = make_state_map(&ctx->mYb40[1], ctx->Yb[1], 8, ctx->ld, p.nvz, ctx->cs, bx, rw);
        if (!r) r = make_state_map(&ctx->mYb40s4[0], ctx->Yb[0], 8, ctx->ld, p.nvz, ctx->cs, bx, rn);
        if (!r) r = make_state_map(&ctx->mYb40s4[1], ctx->Yb[1], 8, ctx->ld, p.nvz, ctx->cs, bx, rn);
        if (!r) r = make_state_map(&ctx->mU0_40, ctx->U0, ub, ctx->ld, p.nvz, ctx->cs, bxu, ru);
        // (FP64 stage 3 reads U1 in 40-cell rows, see the TMA kernel's Layout)
        if (!r) r = make_state_map(&ctx->mU1_40, ctx->U1, ub, ctx->ld, p.nvz, ctx->cs,
                                   ctx->fp32 ? bxu : bt + 8, ru);
        if (!r) r = make_state_map(&ctx->mY32, ctx->Yb[0], 8, ctx->ld, p.nvz, ctx->cs, bt, rn);
        if (!r) r = make_state_map(&ctx->mA32, ctx->Yb[1], 8, ctx->ld, p.nvz, ctx->cs, bt, rn);
        if (!r) r = make_state_map(&ctx->mU0_32, ctx->U0, ub, ctx->ld, p.nvz, ctx->cs, bt, rn);
        if (!r) r = make_state_map(&ctx->mU1_32, ctx->U1, ub, ctx->ld, p.nvz, ctx->cs, bt, rn);
        if (!r && ctx->U2)
            r = make_state_map(&ctx->mU2_40, ctx->U2, ub, ctx->ld, p.nvz, ctx->cs, bxu, rn);
        if (!ctx->U2) ctx->mU2_40 = ctx->mU1_40;  // unused in FP64
        if (!r && tma_prepare() != cudaSuccess) r = -2;
        if (r) {
            // no tensor-map support: fall back to the register-tiled kernel
            ctx->use_tma = false;
            ctx->p.tile_z = ctx->p.tile_v = 0;
            choose_tile(ctx);
        }
        cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, p.device);
    }
    const char *ng = getenv("COSENU_NO_GRAPH");
    ctx->use_graphs = !(ng && ng[0] == '1');
    *out = ctx;
    return COSENU_OK;
}

StageArgs ctx_stage_args(const cosenu_ctx *ctx, int stage, int par)
{
    return stage_args(ctx, stage, par);
}
int ctx_prepare_state(cosenu_ctx *ctx) { return prepare_state(ctx); }
void ctx_flip(cosenu_ctx *ctx) { flip(ctx); }

int ctx_normalise_parity(cosenu_ctx *ctx)
{
    if (ctx->ypar == 0) return COSENU_OK;
    CK(cudaMemcpyAsync(ctx->Yb[0], ctx->Yb[1], (size_t)ctx->cs * 8 * NCOMP,
                       cudaMemcpyDeviceToDevice, ctx->stream));
    flip(ctx);
    return COSENU_OK;
}

int ctx_set_tiling(cosenu_ctx *ctx, int tz, int tv)
{
    if (tz == 0) {
        ctx->tz = 32;
        ctx->tv = ctx->p.nvz;
        ctx->nvt = 1;
        ctx->use_tma = true;
    } else {
        int nvt = (ctx->p.nvz + tv - 1) / tv;
        if (ctx->p.nz % tz != 0 || nvt > ctx->mom_nvt_cap || tv > MAX_TV)
            return fail(ctx, COSENU_ERR_ARG, "tile does not fit this member");
        ctx->tz = tz;
        ctx->tv = tv;
        ctx->nvt = nvt;
        ctx->use_tma = false;
    }
    drop_graphs(ctx);
    return ctx->have_state ? prepare_state(ctx) : COSENU_OK;
}

extern "C" {

int cosenu_destroy(cosenu_ctx *ctx)
{
    if (!ctx) return COSENU_OK;
    DeviceGuard dg(ctx->p.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
    void *bufs[] = {ctx->Yb[0], ctx->Yb[1], ctx->S0, ctx->U0, ctx->U1, ctx->U2, ctx->G, ctx->bG, ctx->M[0],
                    ctx->M[1], ctx->M[2], ctx->vz, ctx->rowfac, ctx->Hm, ctx->diag_part,
                    ctx->diag_out, ctx->pee, ctx->tmp, ctx->err_flag};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->snap_stream) {
        cudaStreamSynchronize(ctx->snap_stream);
        cudaStreamDestroy(ctx->snap_stream);
    }
    if (ctx->snap_taken) cudaEventDestroy(ctx->snap_taken);
    if (ctx->snap_done) cudaEventDestroy(ctx->snap_done);
    if (ctx->snap_d) cudaFree(ctx->snap_d);
    if (ctx->snap_h) cudaFreeHost(ctx->snap_h);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return COSENU_OK;
}

int cosenu_set_vac_pars(cosenu_ctx *ctx, double pmo, double omega, double theta_deg)
{
    if (!ctx) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->p.pmo = pmo;
    ctx->p.omega = omega;
    ctx->p.theta_deg = theta_deg;
    double th = theta_deg * M_PI / 180.0;
    ctx->ct = (1.0 / 2.0) * omega * cos(2.0 * th);
    ctx->st = (1.0 / 2.0) * omega * sin(2.0 * th);
    drop_graphs(ctx);
    return COSENU_OK;
}

int cosenu_set_collective_pars(cosenu_ctx *ctx, double mu)
{
    if (!ctx) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->p.mu = mu;
    drop_graphs(ctx);
    return COSENU_OK;
}

int cosenu_set_wait_limit(cosenu_ctx *ctx, double seconds)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!(seconds >= 1e-6 && seconds <= 600.0))
        return fail(ctx, COSENU_ERR_ARG, "wait limit must be in [1e-6, 600] s");
    DeviceGuard dg(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->wait_ns = (unsigned long long)(seconds * 1e9);
    drop_graphs(ctx);
    return COSENU_OK;
}

int cosenu_test_stall_pipeline(cosenu_ctx *ctx, int on)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!ctx->use_tma) return fail(ctx, COSENU_ERR_STATE, "the context does not use the TMA kernel");
    DeviceGuard dg(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stall = on ? 1 : 0;
    drop_graphs(ctx);
    return COSENU_OK;
}

int cosenu_set_stream(cosenu_ctx *ctx, void *stream)
{
    if (!ctx) return COSENU_ERR_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return COSENU_OK;
}

int cosenu_grid(const cosenu_ctx *ctx, double out[5])
{
    if (!ctx || !out) return COSENU_ERR_ARG;
    out[0] = ctx->dz;
    out[1] = ctx->dv;
    out[2] = ctx->dt;
    out[3] = ctx->ct;
    out[4] = ctx->st;
    return COSENU_OK;
}

int cosenu_upload(cosenu_ctx *ctx, const double *const comp[8], int gz)
{
    if (!ctx || !comp) return COSENU_ERR_ARG;
    if (gz < 0 || gz > HP) return fail(ctx, COSENU_ERR_ARG, "gz must be in [0, 16]");
    DeviceGuard dg(ctx->p.device);
    int rc = copy_planes_h2d(ctx, ctx->Y, comp, NCOMP, gz);
    if (rc) return rc;
    return prepare_state(ctx);
}

int cosenu_upload_device(cosenu_ctx *ctx, const double *const comp[8], int ld)
{
    if (!ctx || !comp || ld < ctx->p.nz) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    for (int c = 0; c < NCOMP; ++c)
        CK(cudaMemcpy2DAsync(ctx->Y + (long long)c * ctx->cs + HP, (size_t)ctx->ld * 8, comp[c],
                             (size_t)ld * 8, (size_t)ctx->p.nz * 8, ctx->p.nvz,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    return prepare_state(ctx);
}

int cosenu_download(cosenu_ctx *ctx, double *const comp[8], int gz)
{
    if (!ctx || !comp) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    if (gz < 0 || gz > ctx->H) return fail(ctx, COSENU_ERR_ARG, "gz larger than the device ghost zone");
    DeviceGuard dg(ctx->p.device);
    const int nz = ctx->p.nz;
    for (int c = 0; c < NCOMP; ++c) {
        if (!comp[c]) return fail(ctx, COSENU_ERR_ARG, "null component pointer");
        CK(cudaMemcpy2DAsync(comp[c], (size_t)(nz + 2 * gz) * 8,
                             ctx->Y + (long long)c * ctx->cs + HP - gz, (size_t)ctx->ld * 8,
                             (size_t)(nz + 2 * gz) * 8, ctx->p.nvz, cudaMemcpyDeviceToHost,
                             ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_err_flag(ctx);
}

int cosenu_snapshot(cosenu_ctx *ctx, long long *steps)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    DeviceGuard dg(ctx->p.device);
    const int nz = ctx->p.nz, nvz = ctx->p.nvz;
    const size_t n = (size_t)NCOMP * nvz * nz;
    if (!ctx->snap_d) {
        CK(cudaMalloc(&ctx->snap_d, n * sizeof(double)));
        CK(cudaMallocHost(&ctx->snap_h, n * sizeof(double)));
        CK(cudaStreamCreateWithFlags(&ctx->snap_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->snap_taken, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->snap_done, cudaEventDisableTiming));
    }
    // the previous host copy must be out of the device buffer before it is
    // overwritten (ordered on the device; the caller is done with the host
    // buffer by contract)
    if (ctx->snap_pending) CK(cudaStreamWaitEvent(ctx->stream, ctx->snap_done, 0));
    for (int c = 0; c < NCOMP; ++c)
        CK(cudaMemcpy2DAsync(ctx->snap_d + (size_t)c * nvz * nz, (size_t)nz * 8,
                             ctx->Y + (long long)c * ctx->cs + HP, (size_t)ctx->ld * 8,
                             (size_t)nz * 8, nvz, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->snap_taken, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->snap_stream, ctx->snap_taken, 0));
    CK(cudaMemcpyAsync(ctx->snap_h, ctx->snap_d, n * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->snap_stream));
    CK(cudaEventRecord(ctx->snap_done, ctx->snap_stream));
    ctx->snap_pending = true;
    if (steps) *steps = ctx->steps;
    return COSENU_OK;
}

int cosenu_snapshot_wait(cosenu_ctx *ctx, const double **data)
{
    if (!ctx || !data || !ctx->snap_pending) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    if (cudaEventSynchronize(ctx->snap_done) != cudaSuccess) return COSENU_ERR_CUDA;
    *data = ctx->snap_h;
    return COSENU_OK;
}

int cosenu_download_device(cosenu_ctx *ctx, double *const comp[8], int ld)
{
    if (!ctx || !comp || ld < ctx->p.nz) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    DeviceGuard dg(ctx->p.device);
    for (int c = 0; c < NCOMP; ++c)
        CK(cudaMemcpy2DAsync(comp[c], (size_t)ld * 8, ctx->Y + (long long)c * ctx->cs + HP,
                             (size_t)ctx->ld * 8, (size_t)ctx->p.nz * 8, ctx->p.nvz,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    return COSENU_OK;
}

int cosenu_set_profile(cosenu_ctx *ctx, const double *G, const double *bG, int gz)
{
    if (!ctx || !G || !bG) return COSENU_ERR_ARG;
    if (gz < 0 || gz > HP) return fail(ctx, COSENU_ERR_ARG, "gz must be in [0, 16]");
    DeviceGuard dg(ctx->p.device);
    const double *g[1] = {G}, *bg[1] = {bG};
    int rc = copy_planes_h2d(ctx, ctx->G, g, 1, gz);
    if (!rc) rc = copy_planes_h2d(ctx, ctx->bG, bg, 1, gz);
    if (rc) return rc;
    ctx->have_profile = true;
    return COSENU_OK;
}

int cosenu_set_state0(cosenu_ctx *ctx, const double *const comp[8], int gz)
{
    if (!ctx || !comp) return COSENU_ERR_ARG;
    if (gz < 0 || gz > HP) return fail(ctx, COSENU_ERR_ARG, "gz must be in [0, 16]");
    DeviceGuard dg(ctx->p.device);
    int rc = copy_planes_h2d(ctx, ctx->S0, comp, NCOMP, gz);
    if (rc) return rc;
    ctx->have_state0 = true;
    return COSENU_OK;
}

int cosenu_mark_state0(cosenu_ctx *ctx)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    DeviceGuard dg(ctx->p.device);
    CK(cudaMemcpyAsync(ctx->S0, ctx->Y, (size_t)ctx->cs * 8 * NCOMP, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    ctx->have_state0 = true;
    return COSENU_OK;
}

int cosenu_step_stage(cosenu_ctx *ctx, int stage)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    if (stage != ctx->next_stage) return fail(ctx, COSENU_ERR_STATE, "stages must run in order 0..3");
    DeviceGuard dg(ctx->p.device);
    CK(launch_stage(ctx, stage + 1, ctx->stream));
    ctx->next_stage = (stage + 1) % 4;
    if (ctx->next_stage == 0) ctx->steps++;
    return COSENU_OK;
}

int cosenu_step(cosenu_ctx *ctx, int nsteps)
{
    if (!ctx || nsteps < 0) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    if (nsteps == 0) return COSENU_OK;
    DeviceGuard dg(ctx->p.device);
    if (!ctx->use_graphs || nsteps == 1) {
        CK(launch_steps(ctx, nsteps, ctx->stream));
    } else {
        // graphs start from a given buffer parity (FP32-bulk alternates it;
        // GRAPH_CHUNK is even, so the long graph leaves it unchanged)
        int n = nsteps;
        if (n >= GRAPH_CHUNK) {
            cudaGraphExec_t &g = ctx->gN[ctx->ypar];
            if (!g) CK(capture(ctx, GRAPH_CHUNK, &g));
            while (n >= GRAPH_CHUNK) {
                CK(cudaGraphLaunch(g, ctx->stream));
                n -= GRAPH_CHUNK;
            }
        }
        while (n-- > 0) {
            cudaGraphExec_t &g = ctx->g1[ctx->ypar];
            if (!g) CK(capture(ctx, 1, &g));
            CK(cudaGraphLaunch(g, ctx->stream));
            flip(ctx);
        }
    }
    ctx->steps += nsteps;
    return COSENU_OK;
}

int cosenu_prepare_graphs(cosenu_ctx *ctx)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    if (!ctx->use_graphs) return COSENU_OK;
    DeviceGuard dg(ctx->p.device);
    // FP32-bulk: graphs for both parities of the state buffer; the context's
    // parity is put back whatever happens
    const int npar = ctx->fp32 ? 2 : 1, par0 = ctx->ypar;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < npar && e == cudaSuccess; ++i) {
        if (i) flip(ctx);
        if (!ctx->gN[ctx->ypar]) e = capture(ctx, GRAPH_CHUNK, &ctx->gN[ctx->ypar]);
        if (e == cudaSuccess && !ctx->g1[ctx->ypar]) e = capture(ctx, 1, &ctx->g1[ctx->ypar]);
    }
    if (ctx->ypar != par0) flip(ctx);
    CK(e);
    return COSENU_OK;
}

int cosenu_synchronize(cosenu_ctx *ctx)
{
    if (!ctx) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    CK(cudaStreamSynchronize(ctx->stream));
    return check_err_flag(ctx);
}

int cosenu_time(const cosenu_ctx *ctx, double *phy_time, long long *steps)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (phy_time) *phy_time = (double)ctx->steps * ctx->dt;
    if (steps) *steps = ctx->steps;
    return COSENU_OK;
}

int cosenu_analyse(cosenu_ctx *ctx, cosenu_diag *out)
{
    if (!ctx || !out) return COSENU_ERR_ARG;
    if (!ctx->have_state) return fail(ctx, COSENU_ERR_STATE, "no state uploaded");
    if (!ctx->have_profile || !ctx->have_state0)
        return fail(ctx, COSENU_ERR_STATE, "analysis needs set_profile and state0");
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    DeviceGuard dg(ctx->p.device);
    CK(launch_diag(ctx->Y, ctx->S0, ctx->G, ctx->bG, ctx->cs, ctx->ld, ctx->p.nz, ctx->p.nvz,
                   ctx->dz, ctx->dv, ctx->diag_part, ctx->diag_out, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_pinned, ctx->diag_out, 13 * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (int rc = check_err_flag(ctx)) return rc;
    const double *r = ctx->h_pinned;
    out->dP_max = r[0];
    out->avdP = r[1];
    out->avbdP = r[2];
    out->M0 = r[3];
    out->M0_e1 = r[4];
    out->M0_e2 = r[5];
    out->M0_e3 = r[6];
    out->Pee = r[7];
    out->Pbee = r[8];
    out->trace = r[9];
    out->btrace = r[10];
    out->eln = r[11];
    if (r[12] != 0.0) return fail(ctx, COSENU_ERR_NONFINITE, "non-finite values in the state");
    return COSENU_OK;
}

int cosenu_pee_v(cosenu_ctx *ctx, double *pee, double *pbee)
{
    if (!ctx || !pee || !pbee) return COSENU_ERR_ARG;
    if (!ctx->have_state || !ctx->have_state0) return fail(ctx, COSENU_ERR_STATE, "needs state and state0");
    if (ctx->next_stage != 0) return fail(ctx, COSENU_ERR_STATE, "RK4 step in progress");
    DeviceGuard dg(ctx->p.device);
    const int nvz = ctx->p.nvz;
    CK(launch_pee_v(ctx->Y, ctx->S0, ctx->cs, ctx->ld, ctx->p.nz, nvz, ctx->pee, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_pinned + 16, ctx->pee, 2 * (size_t)nvz * 8, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::memcpy(pee, ctx->h_pinned + 16, nvz * 8);
    std::memcpy(pbee, ctx->h_pinned + 16 + nvz, nvz * 8);
    return COSENU_OK;
}

int cosenu_init_seeded(cosenu_ctx *ctx, uint64_t seed, uint32_t instance, double sig_nu,
                       double sig_nubar, double alpha, double amp)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (!(sig_nu > 0) || !(sig_nubar > 0) || !(amp >= 0) || !(amp <= 1))
        return fail(ctx, COSENU_ERR_ARG, "sigma must be > 0 and amp in [0, 1]");
    DeviceGuard dg(ctx->p.device);
    const int nvz = ctx->p.nvz;
    std::vector<double> tab(2 * nvz);
    for (int i = 0; i < nvz; ++i) {
        tab[i] = gprof(ctx->h_vz[i], 1.0, sig_nu);
        tab[nvz + i] = alpha * gprof(ctx->h_vz[i], 1.0, sig_nubar);
    }
    CK(cudaMemcpyAsync(ctx->tmp, tab.data(), 2 * nvz * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_init_seeded(ctx->Y, ctx->G, ctx->bG, ctx->tmp, ctx->tmp + nvz, ctx->cs, ctx->ld,
                          ctx->p.nz, nvz, seed, instance, amp, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));  // tab goes out of scope
    int rc = prepare_state(ctx);
    if (rc) return rc;
    ctx->have_profile = true;
    ctx->steps = 0;
    return cosenu_mark_state0(ctx);
}

int cosenu_init_reference(cosenu_ctx *ctx, double perturbation_size)
{
    if (!ctx) return COSENU_ERR_ARG;
    DeviceGuard dg(ctx->p.device);
    const int nvz = ctx->p.nvz, nz = ctx->p.nz;
    const double signu = 0.6, sigbnu = 0.6, alpha = 0.90;  // src/initialize.hpp:12-14
    std::vector<double> tab(2 * nvz + 2 * nz);
    for (int i = 0; i < nvz; ++i) {
        tab[i] = gprof(ctx->h_vz[i], 1.0, signu);
        tab[nvz + i] = alpha * gprof(ctx->h_vz[i], 1.0, sigbnu);
    }
    for (int j = 0; j < nz; ++j) {
        double z = ctx->h_Z[j];
        double e = perturbation_size * exp(-(z - 0.0) * (z - 0.0) / 50.0);  // eps()
        tab[2 * nvz + j] = e;
        tab[2 * nvz + nz + j] = sqrt(1.0 - e * e);  // eps_()
    }
    CK(cudaMemcpyAsync(ctx->tmp, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_init_reference(ctx->Y, ctx->G, ctx->bG, ctx->tmp, ctx->tmp + nvz,
                             ctx->tmp + 2 * nvz, ctx->tmp + 2 * nvz + nz, ctx->cs, ctx->ld, nz,
                             nvz, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    int rc = prepare_state(ctx);
    if (rc) return rc;
    ctx->have_profile = true;
    ctx->steps = 0;
    return cosenu_mark_state0(ctx);
}

int cosenu_device_state(cosenu_ctx *ctx, double *comp[8], int *ld)
{
    if (!ctx || !comp) return COSENU_ERR_ARG;
    for (int c = 0; c < NCOMP; ++c) comp[c] = ctx->Y + (long long)c * ctx->cs + HP;
    if (ld) *ld = ctx->ld;
    return COSENU_OK;
}

int cosenu_launches_per_step(const cosenu_ctx *ctx) { return ctx ? 4 : 0; }

int cosenu_tile(const cosenu_ctx *ctx, int *tile_z, int *tile_v)
{
    if (!ctx) return COSENU_ERR_ARG;
    if (tile_z) *tile_z = ctx->tz;
    if (tile_v) *tile_v = ctx->tv;
    return COSENU_OK;
}

int cosenu_device_bytes(const cosenu_ctx *ctx, size_t *bytes)
{
    if (!ctx || !bytes) return COSENU_ERR_ARG;
    *bytes = ctx->bytes;
    return COSENU_OK;
}

}  // extern "C"
