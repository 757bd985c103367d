// Internal definitions shared by the C-ABI translation units (context layout,
// launchers).  Not part of the public interface.
#pragma once

#include <cuda.h>

#include <string>
#include <vector>

#include "../../include/cosenu_b200.h"
#include "common.cuh"

namespace cosenu {
cudaError_t launch_rk4_stage(const StageArgs &a, int scheme, int stage, int tz, int fp32,
                             cudaStream_t s);
cudaError_t launch_ghost_fill(double *buf, long long cs, int ld, int nz, int nvz, int H, int bc,
                              cudaStream_t s);
cudaError_t launch_moments(const double *X, double *M, const double *vz, long long cs, int ld,
                           int nz, int nvz, int tz, int tv, cudaStream_t s);
int make_state_map(CUtensorMap *map, const void *base, int elem_bytes, int ld, int nvz,
                   long long cs, int box_cells, int box_rows);
int tma_box_rows(int scheme, bool wide);
int tma_box_x(int elem_bytes);
int tma_box_tile();
int tma_max_nvz();
int tma_blocks_per_sm(int scheme);
cudaError_t tma_prepare();
cudaError_t launch_rk4_stage_tma(const CUtensorMap &mX, const CUtensorMap &mY,
                                 const CUtensorMap &mA, const CUtensorMap &mB, const StageArgs &a,
                                 int scheme, int stage, int fp32, int *err, int nblocks,
                                 cudaStream_t s);
cudaError_t launch_rk4_stage_tma_batch(const BatchDev &bd, const StageArgs &a, int scheme,
                                       int stage, int fp32, int *err, int nblocks, int max_nvz,
                                       cudaStream_t s);
cudaError_t launch_rk4_stage_batch(const BatchDev &bd, int scheme, int stage, int tz, int fp32,
                                   cudaStream_t s);
}  // namespace cosenu

// One simulation on one GPU.
struct cosenu_ctx {
    cosenu_params p{};
    int ld = 0, H = 4, tz = 32, tv = 64, nvt = 1;
    long long cs = 0;
    double dz = 0, dv = 0, dt = 0, ct = 0, st = 0;
    int fp32 = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    // device memory.  Two FP64 state buffers Yb[0], Yb[1]: FP64 keeps the state
    // in Yb[0] and the RK4 accumulator in Yb[1]; FP32-bulk writes each step's
    // new state into the other buffer, so the state sits in Yb[ypar].  Y and A
    // always name the current state and the other buffer.
    double *Yb[2] = {nullptr, nullptr};
    int ypar = 0;
    double *Y = nullptr, *A = nullptr, *S0 = nullptr, *G = nullptr, *bG = nullptr;
    // stage values U0, U1 (FP64) or increments D1, D2, D3 in U0, U1, U2 (FP32-bulk)
    void *U0 = nullptr, *U1 = nullptr, *U2 = nullptr;
    double *M[3] = {nullptr, nullptr, nullptr};
    double *vz = nullptr, *rowfac = nullptr, *Hm = nullptr;
    double *diag_part = nullptr, *diag_out = nullptr, *pee = nullptr, *tmp = nullptr;
    size_t bytes = 0;
    // host mirrors
    std::vector<double> h_vz, h_rowfac, h_Hm, h_Z;
    double *h_pinned = nullptr;  // small pinned buffer for results
    // TMA-pipelined path: tensor maps, "40" = input box with halo, "32" = tile
    bool use_tma = false;
    int nsm = 148;
    CUtensorMap mYb40[2], mU0_40, mU1_40, mU2_40, mY32, mA32, mU0_32, mU1_32;
    CUtensorMap mYb40s4[2];  // FP32-bulk stage 4's view of Yb (its own row count)
    int *err_flag = nullptr;  // device word set by bounded waits that expired
    unsigned long long wait_ns = 2000000000ull;  // limit of each pipeline wait
    int stall = 0;            // test hook: TMA producers issue no copies
    // graphs of 1 and GRAPH_CHUNK steps, per parity of the state buffer
    cudaGraphExec_t g1[2] = {nullptr, nullptr}, gN[2] = {nullptr, nullptr};
    bool use_graphs = true;
    // status
    bool have_state = false, have_profile = false, have_state0 = false;
    int next_stage = 0;
    long long steps = 0;
    int mom_nvt_cap = 1;  // v tiles the moment buffers have room for
    // snapshot: device copy of the interior state, its pinned host copy, the
    // stream of the device-to-host copy and the events ordering the two
    double *snap_d = nullptr, *snap_h = nullptr;
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
    bool snap_pending = false;
    std::string err;
};


// Context creation; layout 1 forces the TMA layout (32-cell z tiles spanning
// all rows, tensor maps built) whatever the grid size, as ensemble members
// need it.
int ctx_create(const cosenu_params *p, cosenu_ctx **out, int layout);
// Arguments of stage 1..4 of a context with its state in Yb[par] (par < 0:
// where it is now).
cosenu::StageArgs ctx_stage_args(const cosenu_ctx *ctx, int stage, int par = -1);
// FP32-bulk: makes Yb[0] hold the state again (copies it over when it is in
// Yb[1]), so that members of an ensemble start a run with the same parity.
int ctx_normalise_parity(cosenu_ctx *ctx);
// After a stage-4 launch (or a graph of an odd number of steps) in FP32-bulk:
// the new state is in the other buffer.
void ctx_flip(cosenu_ctx *ctx);
// Ghost cells and input moments of Y after Y changed outside the stages.
int ctx_prepare_state(cosenu_ctx *ctx);
// Re-tiles an ensemble member for the register-tiled kernel (tz x tv) or back
// to the TMA layout (tz = 0); recomputes the input moments of Y.
int ctx_set_tiling(cosenu_ctx *ctx, int tz, int tv);
