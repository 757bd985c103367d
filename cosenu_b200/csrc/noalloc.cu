// cosenu_step_noalloc: RK4 steps on a caller-owned state without allocating.
//
// Some callers cannot let a library call cudaMalloc: a host application that
// hands out all device memory from its own pool (a framework's caching
// allocator, a service with a fixed memory budget) would see an allocation it
// did not plan for, and cudaMalloc/cudaFree can synchronise the device in the
// middle of a latency-sensitive loop.  This entry point lets such a caller
// advance a state it already holds in device memory.  Its working memory
// (a padded copy of the state with ghost cells, the RK4 stage buffers -- U0,
// U1, A in FP64; a second state buffer and the increments D1, D2, D3 in
// FP32-bulk --, the velocity-moment partials and the per-row tables) lives in one
// file-scope device array of fixed size, NOALLOC_SCRATCH_DOUBLES doubles
// (20.5 MB), which every GPU that loads this library holds until the process
// exits.
//
// The first call on a device looks up that array's device address with
// cudaGetSymbolAddress (the array's name in host code is only a host-side
// stand-in); make that first call before any stream capture.  The address is
// kept per device together with the identity of the device's current context,
// and looked up again when that context changes (after cudaDeviceReset, for
// instance): the first call in a new context is again a set-up call.  All calls share
// the one array: calls whose work overlaps on the GPU (different streams, or
// different host threads on the same device) race on it and must be ordered by
// the caller.  Each call clears the part of the array it uses, so nothing from
// an earlier call leaks into the next one.
//
// The kernels are the ones cosenu_step runs (register-tiled stage kernels,
// ghost fill, moments); only their buffers differ.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include <cuda.h>

#include "../../include/cosenu_b200.h"
#include "common.cuh"

extern thread_local std::string g_create_error;

namespace cosenu {
cudaError_t launch_rk4_stage(const StageArgs &a, int scheme, int stage, int tz, int fp32,
                             cudaStream_t s);
cudaError_t launch_ghost_fill(double *buf, long long cs, int ld, int nz, int nvz, int H, int bc,
                              cudaStream_t s);
cudaError_t launch_moments(const double *X, double *M, const double *vz, long long cs, int ld,
                           int nz, int nvz, int tz, int tv, cudaStream_t s);
}  // namespace cosenu

using namespace cosenu;

// Capacity: nvz * ld_padded <= NOALLOC_MAX_PLANE cells per component plane
// (ld_padded = nz + 32 rounded up to a multiple of 16; the 1024 x 64 FV
// grid needs 67 584) and nz <= NOALLOC_MAX_NZ.
#define NOALLOC_MAX_PLANE 69632
#define NOALLOC_MAX_NZ 16384
#define NOALLOC_MAX_NVZ 4096
#define NOALLOC_MAX_TV 64
#define NOALLOC_MOM_CAP (3 * NMOM * (NOALLOC_MAX_PLANE / NOALLOC_MAX_TV + NOALLOC_MAX_NZ))
#define NOALLOC_SCRATCH_DOUBLES \
    (4LL * NCOMP * NOALLOC_MAX_PLANE + NOALLOC_MOM_CAP + 2 * NOALLOC_MAX_NVZ + NOALLOC_MAX_NZ)

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Per-row velocity and advection factor, per-cell matter potential: the
// values cosenu_create computes on the host (src/nuosc.hpp:78-96), with
// round-to-nearest operations so the bits are the same.
__global__ void noalloc_tables_kernel(double *vz, double *rowfac, double *Hm, int nz, int nvz,
                                      double z0, double v0, double dz, double dv, int scheme,
                                      int fd_advec)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nvz) {
        double v = __dadd_rn(v0, __dmul_rn(__dadd_rn((double)i, 0.5), dv));
        int sv = (0.0 < v) - (v < 0.0);
        double f;
        if (scheme == COSENU_FV) f = __ddiv_rn(-v, dz);
        else if (fd_advec == COSENU_FD_CENTER) f = __ddiv_rn(-v, __dmul_rn(12.0, dz));
        else if (fd_advec == COSENU_FD_UPWIND) f = __ddiv_rn(__dmul_rn((double)(-sv), v), __dmul_rn(12.0, dz));
        else f = __ddiv_rn(__dmul_rn((double)sv, v), __dmul_rn(12.0, dz));
        vz[i] = v;
        rowfac[i] = f;
    }
    if (i < nz) {
        double Z = __dadd_rn(z0, __dmul_rn(__dadd_rn((double)i, 0.5), dz));
        Hm[i] = __dmul_rn(-1.0e-3, __dadd_rn(Z, 600.0));
    }
}

namespace {

std::mutex g_addr_mutex;
double *g_addr[64] = {nullptr};
unsigned long long g_addr_ctx[64] = {0};  // context the cached address belongs to

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the current context (0 if the driver cannot say: the address
// is then looked up on every call).
unsigned long long current_ctx_id()
{
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)p;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)p;
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

int noalloc_fail(int code, const std::string &msg)
{
    g_create_error = "cosenu_step_noalloc: " + msg;
    return code;
}

}  // namespace

extern "C" int cosenu_step_noalloc(const cosenu_params *pp, double *const state[8], int ld,
                                   int nsteps, void *stream)
{
    g_create_error.clear();
    if (!pp || !state) return noalloc_fail(COSENU_ERR_ARG, "null argument");
    const cosenu_params &p = *pp;
    if (p.nz < 16 || p.nz % 8 != 0) return noalloc_fail(COSENU_ERR_ARG, "nz must be a multiple of 8 and >= 16");
    if (p.nvz < 1) return noalloc_fail(COSENU_ERR_ARG, "nvz must be >= 1");
    if (p.scheme != COSENU_FV && p.scheme != COSENU_FD) return noalloc_fail(COSENU_ERR_ARG, "unknown scheme");
    if (p.bc != COSENU_PERIODIC && p.bc != COSENU_OPEN) return noalloc_fail(COSENU_ERR_ARG, "unknown boundary");
    if (p.precision != COSENU_FP64 && p.precision != COSENU_FP32_BULK)
        return noalloc_fail(COSENU_ERR_ARG, "unknown precision");
    if (p.fd_advec < 0 || p.fd_advec > 2) return noalloc_fail(COSENU_ERR_ARG, "unknown FD advection stencil");
    if (p.ko_order != 3 && p.ko_order != 5) return noalloc_fail(COSENU_ERR_ARG, "ko_order must be 3 or 5");
    if (!(p.z1 > p.z0) || !(p.v1 > p.v0) || !(p.cfl > 0))
        return noalloc_fail(COSENU_ERR_ARG, "empty box or non-positive CFL");
    if (p.gz < 0 || p.gz > HP) return noalloc_fail(COSENU_ERR_ARG, "gz must be in [0, 16]");
    if (ld < p.nz) return noalloc_fail(COSENU_ERR_ARG, "ld must be >= nz");
    if (nsteps < 0) return noalloc_fail(COSENU_ERR_ARG, "nsteps must be >= 0");
    for (int c = 0; c < NCOMP; ++c)
        if (!state[c]) return noalloc_fail(COSENU_ERR_ARG, "null component pointer");
    const int ldp = padded_ld(p.nz);
    const long long plane = (long long)p.nvz * ldp;
    if (p.nz > NOALLOC_MAX_NZ || p.nvz > NOALLOC_MAX_NVZ || plane > NOALLOC_MAX_PLANE)
        return noalloc_fail(COSENU_ERR_ARG,
                            "grid too large for the fixed scratch: needs nvz*(nz+32 rounded up to 16) = " +
                                std::to_string(plane) + " <= " + std::to_string(NOALLOC_MAX_PLANE) +
                                " and nz <= " + std::to_string(NOALLOC_MAX_NZ) +
                                "; use cosenu_create/cosenu_step for larger grids");
    // tile: explicit, else the widest z tile that divides nz and up to 64 rows
    int tz = p.tile_z ? p.tile_z : (p.nz % 32 == 0 ? 32 : (p.nz % 16 == 0 ? 16 : 8));
    int tv = p.tile_v ? p.tile_v : std::min(p.nvz, NOALLOC_MAX_TV);
    if ((tz != 8 && tz != 16 && tz != 32) || p.nz % tz != 0 || tv < 1 || tv > NOALLOC_MAX_TV)
        return noalloc_fail(COSENU_ERR_ARG, "tile_z must be 8/16/32 dividing nz, tile_v in [1, 64]");
    const int nvt = (p.nvz + tv - 1) / tv;
    const long long mom = (long long)nvt * NMOM * p.nz;
    if (3 * mom > NOALLOC_MOM_CAP)
        return noalloc_fail(COSENU_ERR_ARG, "tile_v too small for the fixed scratch (moment "
                                            "partials of ceil(nvz/tile_v) v tiles)");
    if (nsteps == 0) return COSENU_OK;

    int prev = -1;
    cudaGetDevice(&prev);
    if (p.device < 0 || p.device >= 64) return noalloc_fail(COSENU_ERR_ARG, "device ordinal out of range");
    cudaError_t e = cudaSetDevice(p.device);
    if (e != cudaSuccess) return noalloc_fail(COSENU_ERR_CUDA, cudaGetErrorString(e));
    auto done = [&](int code, const char *what, cudaError_t err) -> int {
        if (prev >= 0 && prev != p.device) cudaSetDevice(prev);
        if (code != COSENU_OK) return noalloc_fail(code, std::string(what) + ": " + cudaGetErrorString(err));
        return COSENU_OK;
    };
    // set-up, once per device (and again in a new context) with that device current
    double *base;
    {
        std::lock_guard<std::mutex> lk(g_addr_mutex);
        const unsigned long long ctx_id = current_ctx_id();
        if (!g_addr[p.device] || ctx_id == 0 || ctx_id != g_addr_ctx[p.device]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) return done(COSENU_ERR_CUDA, "cudaGetSymbolAddress", e);
            g_addr[p.device] = static_cast<double *>(ptr);
            g_addr_ctx[p.device] = ctx_id;
        }
        base = g_addr[p.device];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long long cs = plane;
    const int fp32 = p.precision == COSENU_FP32_BULK;
    // FP64: Y, stage values U0, U1, accumulator A.  FP32-bulk: two state
    // buffers Y, Y2 (the new state goes to the other one each step) and the
    // FP32 increments D1, D2, D3.
    double *Y = base, *A = base + 3 * NCOMP * cs, *Y2 = base + NCOMP * cs;
    void *U0 = base + NCOMP * cs, *U1 = base + 2 * NCOMP * cs;
    float *D1 = reinterpret_cast<float *>(base + 2 * NCOMP * cs);
    float *D2 = D1 + NCOMP * cs, *D3 = D2 + NCOMP * cs;
    double *M[3] = {base + 4 * NCOMP * cs, base + 4 * NCOMP * cs + mom, base + 4 * NCOMP * cs + 2 * mom};
    double *vz = base + 4 * NCOMP * cs + 3 * mom, *rowfac = vz + p.nvz, *Hm = rowfac + p.nvz;
    const size_t used = (size_t)((Hm + p.nz) - base) * sizeof(double);

    if ((e = cudaMemsetAsync(base, 0, used, s)) != cudaSuccess) return done(COSENU_ERR_CUDA, "clear", e);
    const double dz = (p.z1 - p.z0) / p.nz, dv = (p.v1 - p.v0) / (p.nvz);
    const int n = std::max(p.nz, p.nvz);
    noalloc_tables_kernel<<<(n + 127) / 128, 128, 0, s>>>(vz, rowfac, Hm, p.nz, p.nvz, p.z0, p.v0,
                                                          dz, dv, p.scheme, p.fd_advec);
    if ((e = cudaGetLastError()) != cudaSuccess) return done(COSENU_ERR_CUDA, "tables", e);
    for (int c = 0; c < NCOMP; ++c) {
        e = cudaMemcpy2DAsync(Y + c * cs + HP, (size_t)ldp * 8, state[c], (size_t)ld * 8,
                              (size_t)p.nz * 8, p.nvz, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return done(COSENU_ERR_CUDA, "copy in", e);
    }
    const int H = std::max(4, std::min(p.gz, HP));
    if ((e = launch_ghost_fill(Y, cs, ldp, p.nz, p.nvz, H, p.bc, s)) != cudaSuccess)
        return done(COSENU_ERR_CUDA, "ghost fill", e);
    if ((p.flags & COSENU_COLL) &&
        (e = launch_moments(Y, M[2], vz, cs, ldp, p.nz, p.nvz, tz, tv, s)) != cudaSuccess)
        return done(COSENU_ERR_CUDA, "moments", e);

    StageArgs a{};
    a.vz = vz;
    a.rowfac = rowfac;
    a.Hm = Hm;
    a.cs = cs;
    a.nz = p.nz;
    a.nvz = p.nvz;
    a.ld = ldp;
    a.tv = tv;
    a.nvt = nvt;
    a.H = H;
    a.bc = p.bc;
    a.flags = (int)p.flags;
    a.fd_advec = p.fd_advec;
    a.ko_order = p.ko_order;
    a.dt = p.cfl * dz;
    a.dv = dv;
    a.v0 = p.v0;
    a.dz = dz;
    a.mu = p.mu;
    const double th = p.theta_deg * M_PI / 180.0;
    a.ct = (1.0 / 2.0) * p.omega * cos(2.0 * th);
    a.st = (1.0 / 2.0) * p.omega * sin(2.0 * th);
    a.pmo = p.pmo;
    const double ko = 1.0e-1;
    a.ko_eps = p.ko_order == 5 ? -ko / dz / 64.0 : -ko / dz / 16.0;
    a.Y = Y;
    a.A = A;
    a.T1 = D1;
    a.T2 = D2;
    double *ycur = Y, *ynext = Y2;
    for (int it = 0; it < nsteps; ++it) {
        for (int st = 1; st <= 4; ++st) {
            if (!fp32) {
                switch (st) {
                case 1: a.X = Y; a.U = U0; a.Min = M[2]; a.Mout = M[0]; break;
                case 2: a.X = U0; a.U = U1; a.Min = M[0]; a.Mout = M[1]; break;
                case 3: a.X = U1; a.U = U0; a.Min = M[1]; a.Mout = M[0]; break;
                case 4: a.X = U0; a.U = Y; a.Min = M[0]; a.Mout = M[2]; break;
                }
            } else {
                a.Y = ycur;
                switch (st) {
                case 1: a.X = ycur; a.U = D1; a.Min = M[2]; a.Mout = M[0]; break;
                case 2: a.X = D1; a.U = D2; a.Min = M[0]; a.Mout = M[1]; break;
                case 3: a.X = D2; a.U = D3; a.Min = M[1]; a.Mout = M[0]; break;
                case 4: a.X = D3; a.U = ynext; a.Min = M[0]; a.Mout = M[2]; break;
                }
            }
            if ((e = launch_rk4_stage(a, p.scheme, st, tz, fp32, s)) != cudaSuccess)
                return done(COSENU_ERR_CUDA, "stage", e);
        }
        if (fp32) std::swap(ycur, ynext);
    }
    Y = ycur;
    for (int c = 0; c < NCOMP; ++c) {
        e = cudaMemcpy2DAsync(state[c], (size_t)ld * 8, Y + c * cs + HP, (size_t)ldp * 8,
                              (size_t)p.nz * 8, p.nvz, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return done(COSENU_ERR_CUDA, "copy out", e);
    }
    return done(COSENU_OK, "", cudaSuccess);
}
