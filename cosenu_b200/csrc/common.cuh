// Shared definitions of the B200 kernels for COSEnu's RK4 path.
//
// Device layout of one state buffer: 8 component planes, each nvz rows of
// `ld` cells; the interior cell (v, z) of component c sits at
//     c*cs + v*ld + HP + z,   cs = nvz*ld,   ld = round_up(nz + 2*HP, 16).
// HP = 16 cells (128 B) of padding on each side of a row keeps the interior
// start of every row 128-byte aligned and holds the ghost cells (up to HP of
// them) that the stencils read.  This is the reference's FieldVar layout
// (v-major rows, z contiguous, src/nuosc.hpp:145-148) with a wider,
// aligned ghost zone.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cosenu {

constexpr int NCOMP = 8;
constexpr int HP = 16;         // pad cells per row side
constexpr int NTHREADS = 256;  // threads per stage block
constexpr int MAX_TV = 256;    // max v rows per tile
constexpr int NMOM = 6;        // velocity moments per z

enum Comp { EE = 0, XX, EXR, EXI, BEE, BXX, BEXR, BEXI };
enum Scheme { FV = 0, FD = 1 };
enum Flags { F_VAC = 1, F_MAT = 2, F_COLL = 4, F_ADVEC_OFF = 8 };

// Arguments of one RK4 stage launch (passed by value).
struct StageArgs {
    const void *X;       // stage input, TIN, with ghosts: U or Y (FP64); D or Y (FP32-bulk)
    const double *Y;     // RK4 base state (FP64 stages 2, 3; FP32-bulk stages 2-4, with ghosts)
    double *A;           // RK4 accumulator (FP64)
    void *U;             // stage output, TOUT (U', U'' or the new Y; D1, D2, D3 or the new Y)
    const float *T1, *T2;  // FP32-bulk stage 4: the increments D1, D2 at its own cells
    const double *Min;   // [nvt][6][nz] per-v-tile moments of X
    double *Mout;        // [nvt][6][nz] per-v-tile moments of U
    const double *vz;    // [nvz] velocities
    const double *rowfac;// [nvz] advection factor per row (scheme specific)
    const double *Hm;    // [nz] matter potential
    long long cs;        // component stride (elements)
    unsigned long long wait_ns;  // time limit of each pipeline wait (TMA kernel)
    int nz, nvz, ld, tv, nvt;
    int H;               // ghost cells written per side
    int bc, flags, fd_advec, ko_order;
    int stall;           // test hook: the TMA producer issues no copies
    double dt, dv, mu, ct, st, pmo, ko_eps;
    double v0, dz;       // velocity grid origin, cell width (rows recompute vz)
};

// Ensemble launch: one stage launch covers every active instance.  Entry t of
// `table` names (instance, z tile, v tile, rows: nvz in the TMA family); `args` holds the four stage
// arguments of every instance and `maps` its six tensor maps (Y and U0/U1
// input boxes; Y, A and U0 tile boxes).
struct BatchDev {
    const int4 *table;
    int ntiles;
    const StageArgs *args;      // [instances][4]
    const CUtensorMap *maps;    // [instances][5]
    const int *range;           // TMA family: block b owns table entries [range[b], range[b+1])
};

// Layout helpers shared by host and device code.
__host__ __device__ inline long long dev_index(long long cs, int ld, int c, int v, int z)
{
    return (long long)c * cs + (long long)v * ld + HP + z;
}

inline int padded_ld(int nz) { return ((nz + 2 * HP + 15) / 16) * 16; }

// RK4 with FP64 stage values moves 832 B per cell-update instead of 1024:
// differences of stored stage values stand in for k1 and k2 in the
// accumulator (U - Y = dt/2 k1 and U' - Y = dt/2 k2 to rounding), so A is
// written once, by stage 3, and only stage 3 writes two arrays:
//   stage 1: U   = Y + dt/2 k1                          (reads Y, writes U)
//   stage 2: U'  = Y + dt/2 k2                          (reads U, Y, writes U')
//   stage 3: U'' = Y + dt k3,
//            A   = Y + (U - Y)/3 + 2 (U' - Y)/3 + dt/3 k3
//            (reads U', Y and U at its own cells; writes U'' over U, and A)
//   stage 4: Y   = A + dt/6 k4                          (reads U'', A, writes Y)
//
// FP32-bulk keeps the base state Y in FP64 and stores the stage increments,
// not the stage values, in FP32: D1 = dt/2 k1, D2 = dt/2 k2, D3 = dt k3.  They
// are small, so FP32 holds them to ~6e-8 of dt*k rather than of U, and each
// stage reads its input as Y + D in FP64:
//   stage 1: D1 = dt/2 k1(Y)                             (reads Y, writes D1)
//   stage 2: D2 = dt/2 k2(Y + D1)                        (reads Y, D1, writes D2)
//   stage 3: D3 = dt k3(Y + D2)                          (reads Y, D2, writes D3)
//   stage 4: Y' = Y + (D1 + 2 D2 + D3)/3 + dt/6 k4(Y + D3)
//            (reads Y, D3, and D1, D2 at its own cells; writes Y')
// 576 B per cell-update.  Stage 4 reads Y around its cells while it writes the
// new state, so Y' goes to the second FP64 buffer and the two swap roles every
// step.  inc_form: a launch of this form (an FP32 operand is involved).
template <class TIN, class TOUT>
__host__ __device__ constexpr bool inc_form()
{
    return sizeof(TIN) == 4 || sizeof(TOUT) == 4;
}

}  // namespace cosenu
