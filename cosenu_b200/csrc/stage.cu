// Fused RK4 stage kernels for COSEnu's time-stepping path on sm_100a.
//
// One launch = one RK4 stage of NuOsc::step_rk4 (src/nuosc.hpp:320-348):
// it reads the stage input X with its ghost cells, evaluates the right-hand
// side of src/rhs_fv.hpp:115-236 (FV, WENO7) or src/rhs_fd.hpp:6-148 (FD),
// and applies the stage combine of a three-register RK4 (state Y, stage value
// U, accumulator A) in the same pass.  With FP32 stage values the accumulator
// is updated as the reference's vectorize does
//     stage 1:  U  = Y + dt/2 k1,   A  = Y + dt/6 k1
//     stage 2:  U' = Y + dt/2 k2,   A += dt/3 k2
//     stage 3:  U''= Y + dt   k3,   A += dt/3 k3
//     stage 4:  Y  = A + dt/6 k4
// and with FP64 stage values stage 3 writes A once from differences of the
// stored stage values (a_deferred in common.cuh: 832 B per cell-update).  The epilogue also writes the ghost cells of its output
// (updateBufferZone, src/nuosc.hpp:212-278, periodic or open) and the six
// per-z velocity moments of its output that the next stage's collective term
// needs, so no separate ghost-fill, flux or combine kernels exist.
//
// Block = 256 threads over a tile of TZ consecutive z cells x tv v rows.
// Thread (lz, rr) owns column z0+lz and rows rr, rr+RP, ... (RP = 256/TZ);
// the TZ lanes of one row segment sit in one warp, so z-neighbour values move
// by warp shuffle.  Loads of the stencil go through L1 (the same 128-byte
// lines serve all lanes of a segment).
//
// FV: only the upwind WENO7 reconstruction is evaluated (sign(v) is uniform
// along a row); each lane computes the one face it owns, takes the other from
// its neighbour lane, and the block computes the single extra face per row
// up front.  The right-biased reconstruction at face j-1/2 is the
// left-biased one applied to the mirrored stencil, so one routine serves both.
//
// Collective term (rhs_fv.hpp:188-233, rhs_fd.hpp:85-126): its sum over v'
// depends on v' only through A=ex_im+bex_im, B=ex_re-bex_re,
// C=ee-xx-bee+bxx, and sum_k (1 - v_i v_k) X_k = M0[X] - v_i M1[X], so it is
// built from six per-z moments.  Each block writes its per-v-tile partial
// moments; the consumer sums the partials in a fixed order, so results are
// bitwise reproducible run to run.
#include <type_traits>

#include "common.cuh"
#include "weno.cuh"

namespace cosenu {

template <class T> __device__ __forceinline__ T ld_nc(const T *p) { return __ldg(p); }

template <class T> __device__ __forceinline__ T shfl_idx(T x, int src, int width)
{
    return __shfl_sync(0xffffffffu, x, src, width);
}

// Face centred at row pointer p (cell z) with stencil direction dir (+1:
// left-biased face z+1/2; -1: right-biased face z-1/2).
template <class TC, class TIN>
__device__ __forceinline__ TC face_at(const TIN *__restrict__ p, int dir)
{
    TC u[7];
#pragma unroll
    for (int k = -3; k <= 3; ++k) u[k + 3] = (TC)ld_nc(p + k * dir);
    return weno7_face(u[0], u[1], u[2], u[3], u[4], u[5], u[6]);
}

// FD advection (src/rhs_fd.hpp:53-73) and Kreiss-Oliger dissipation
// (:128-145) of one component at cell pointer p.
template <class TC, class TIN>
__device__ __forceinline__ void fd_terms(const TIN *__restrict__ p, int fd_advec, int ko_order,
                                         int sv, TC factor, TC ko_eps, bool advec, TC &adv, TC &ko)
{
    TC m2 = (TC)ld_nc(p - 2), m1 = (TC)ld_nc(p - 1), c0 = (TC)ld_nc(p), p1 = (TC)ld_nc(p + 1),
       p2 = (TC)ld_nc(p + 2);
    adv = TC(0);
    if (advec) {
        if (fd_advec == 0) {
            adv = factor * ((m2 - p2) - TC(8) * (m1 - p1));
        } else if (fd_advec == 1) {
            adv = factor * (TC(-4) * (TC)ld_nc(p - 3 * sv) + TC(18) * (TC)ld_nc(p - 2 * sv) -
                            TC(36) * (TC)ld_nc(p - sv) + TC(22) * c0);
        } else {
            adv = factor * ((TC)ld_nc(p - 3 * sv) - TC(6) * (TC)ld_nc(p - 2 * sv) +
                            TC(18) * (TC)ld_nc(p - sv) - TC(10) * c0 - TC(3) * (TC)ld_nc(p + sv));
        }
    }
    if (ko_order == 5) {
        ko = ko_eps * ((TC)ld_nc(p - 3) + (TC)ld_nc(p + 3) - TC(6) * (m2 + p2) +
                       TC(15) * (m1 + p1) - TC(20) * c0);
    } else {
        ko = ko_eps * (m2 + p2 - TC(4) * (m1 + p1) + TC(6) * c0);
    }
}

// ---------------------------------------------------------------------------
template <int SCHEME, int STAGE, int TZ, class TC, class TIN, class TOUT, bool BATCHED>
__global__ void __launch_bounds__(NTHREADS, 2)
    rk4_stage_kernel(const __grid_constant__ StageArgs a0, const BatchDev bd)
{
    // tile: (z tile, v tile) from the grid, or (instance, z tile, v tile) from
    // the ensemble table
    int zt = blockIdx.x, vt = blockIdx.y, inst = 0;
    if (BATCHED) {
        const int4 e = bd.table[blockIdx.x];
        inst = e.x;
        zt = e.y;
        vt = e.z;
    }
    const StageArgs &a = BATCHED ? bd.args[inst * 4 + STAGE - 1] : a0;
    constexpr int RP = NTHREADS / TZ;
    __shared__ double s_mom[NMOM][TZ];
    __shared__ double s_red[RP][NMOM][TZ];
    __shared__ TC s_edge[SCHEME == FV ? MAX_TV : 1][NCOMP];

    const TIN *__restrict__ X = static_cast<const TIN *>(a.X);
    TOUT *__restrict__ U = static_cast<TOUT *>(a.U);
    const int tid = threadIdx.x;
    const int lz = tid % TZ;
    const int rr = tid / TZ;
    const int z0 = zt * TZ;
    const int z = z0 + lz;
    const int vbeg = vt * a.tv;
    const int vend = min(vbeg + a.tv, a.nvz);
    const int nrows = vend - vbeg;
    const bool coll = (a.flags & F_COLL) != 0;
    const bool advec = (a.flags & F_ADVEC_OFF) == 0;
    const bool open_bc = a.bc != 0;

    // moments of the stage input at this tile's columns (fixed-order sum of
    // the per-v-tile partials)
    if (coll) {
        for (int q = tid; q < NMOM * TZ; q += NTHREADS) {
            int m = q / TZ, zz = q % TZ;
            double s = 0.0;
            for (int t = 0; t < a.nvt; ++t) s += a.Min[((long long)t * NMOM + m) * a.nz + z0 + zz];
            s_mom[m][zz] = s;
        }
    }
    // FV: the one face per row that lies outside this tile's lanes
    if (SCHEME == FV && advec) {
        for (int r = tid; r < nrows; r += NTHREADS) {
            int v = vbeg + r;
            int dir = (a.vz[v] >= 0.0) ? 1 : -1;
            int zc = dir > 0 ? z0 - 1 : z0 + TZ;
            bool overridden = open_bc && ((dir > 0 && z0 == 0) || (dir < 0 && z0 + TZ == a.nz));
#pragma unroll
            for (int c = 0; c < NCOMP; ++c) {
                s_edge[r][c] = overridden ? TC(0)
                                          : face_at<TC>(X + dev_index(a.cs, a.ld, c, v, zc), dir);
            }
        }
    }
    __syncthreads();

    double macc[NMOM];
#pragma unroll
    for (int m = 0; m < NMOM; ++m) macc[m] = 0.0;

    const double dt = a.dt;
    const int npass = (nrows + RP - 1) / RP;
    for (int pass = 0; pass < npass; ++pass) {
        const int r = pass * RP + rr;
        const bool valid = r < nrows;
        const int v = vbeg + (valid ? r : nrows - 1);  // clamp: shuffles stay uniform
        const double vzv = a.vz[v];
        const TC rowfac = (TC)a.rowfac[v];
        const long long rowoff = (long long)v * a.ld + HP + z;

        // own cell values: RHS arithmetic in TC, combine in double
        TC c[NCOMP];
        double x0[NCOMP];
#pragma unroll
        for (int k = 0; k < NCOMP; ++k) {
            x0[k] = (double)ld_nc(X + k * a.cs + rowoff);
            c[k] = (TC)x0[k];
        }

        TC o[NCOMP];
        if (SCHEME == FV) {
            // advection: upwind flux difference (rhs_fv.hpp:143-162)
            const int dir = (vzv >= 0.0) ? 1 : -1;
            const int src = lz - dir;
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) {
                TC adv = TC(0);
                if (advec) {
                    TC fown = face_at<TC>(X + k * a.cs + rowoff, dir);
                    TC fnb = shfl_idx(fown, src < 0 ? 0 : (src >= TZ ? TZ - 1 : src), TZ);
                    TC fm1 = shfl_idx(fown, lz > 0 ? lz - 1 : 0, TZ);
                    if (dir > 0 && lz == 0) fnb = s_edge[valid ? r : nrows - 1][k];
                    if (dir < 0 && lz == TZ - 1) fnb = s_edge[valid ? r : nrows - 1][k];
                    if (open_bc) {
                        // flux ghosts under OPEN_BC (updateBufferZone on rflux/lflux,
                        // rhs_fv.hpp:118-119): rflux[-1] = rflux[0],
                        // lflux[nz] = 2 lflux[nz-1] - lflux[nz-2]
                        if (dir > 0 && z == 0) fnb = fown;
                        if (dir < 0 && z == a.nz - 1) fnb = fown * TC(2) - fm1;
                    }
                    adv = dir > 0 ? rowfac * (fown - fnb) : rowfac * (fnb - fown);
                }
                o[k] = adv;
            }
            if (a.flags & F_VAC) {
                const TC pmo = (TC)a.pmo, ct = (TC)a.ct, st = (TC)a.st;
                o[EE] += TC(-2) * st * c[EXI] * pmo;
                o[XX] += TC(2) * st * c[EXI] * pmo;
                o[EXR] += TC(-2) * ct * c[EXI] * pmo;
                o[EXI] += (TC(2) * ct * c[EXR] + st * (c[EE] - c[XX])) * pmo;
                o[BEE] += TC(-2) * st * c[BEXI] * pmo;
                o[BXX] += TC(2) * st * c[BEXI] * pmo;
                o[BEXR] += TC(-2) * ct * c[BEXI] * pmo;
                o[BEXI] += (TC(2) * ct * c[BEXR] + st * (c[BEE] - c[BXX])) * pmo;
            }
        } else {
            TC adv[NCOMP], ko[NCOMP];
            const int sv = (vzv > 0.0) - (vzv < 0.0);
#pragma unroll
            for (int k = 0; k < NCOMP; ++k)
                fd_terms<TC>(X + k * a.cs + rowoff, a.fd_advec, a.ko_order, sv, rowfac,
                             (TC)a.ko_eps, advec, adv[k], ko[k]);
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) o[k] = TC(0);
            if (a.flags & F_VAC) {
                const TC pmo = (TC)a.pmo, ct = (TC)a.ct, st = (TC)a.st;
                o[EE] = -pmo * TC(2) * st * c[EXI];
                o[XX] = pmo * TC(2) * st * c[EXI];
                o[EXR] = -pmo * TC(2) * ct * c[EXI];
                o[EXI] = pmo * (TC(2) * ct * c[EXR] + st * (c[EE] - c[XX]));
                o[BEE] = -pmo * TC(2) * st * c[BEXI];
                o[BXX] = pmo * TC(2) * st * c[BEXI];
                o[BEXR] = -pmo * TC(2) * ct * c[BEXI];
                o[BEXI] = pmo * (TC(2) * ct * c[BEXR] + st * (c[BEE] - c[BXX]));
            }
            if (a.flags & F_MAT) {
                TC h = (TC)a.Hm[z];
                o[EXR] += h * c[EXI];
                o[EXI] += -h * c[EXR];
                o[BEXR] += -h * c[BEXI];
                o[BEXI] += h * c[BEXR];
            }
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) o[k] += adv[k];
            // KO dissipation is added after the collective term below
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) c[k] = c[k];  // keep own values live
            if (coll) {
                TC SA = (TC)(s_mom[0][lz] - vzv * s_mom[3][lz]);
                TC SB = (TC)(s_mom[1][lz] - vzv * s_mom[4][lz]);
                TC SC = (TC)(s_mom[2][lz] - vzv * s_mom[5][lz]);
                TC f = (TC)(a.mu * a.dv);
                TC Iee = TC(2) * (c[EXR] * SA - c[EXI] * SB);
                TC Ibee = TC(2) * (c[BEXR] * SA + c[BEXI] * SB);
                o[EE] += f * Iee;
                o[XX] += f * (-Iee);
                o[EXR] += f * ((c[XX] - c[EE]) * SA + c[EXI] * SC);
                o[EXI] += f * (-(c[XX] - c[EE]) * SB - c[EXR] * SC);
                o[BEE] += f * Ibee;
                o[BXX] += f * (-Ibee);
                o[BEXR] += f * ((c[BXX] - c[BEE]) * SA - c[BEXI] * SC);
                o[BEXI] += f * ((c[BXX] - c[BEE]) * SB + c[BEXR] * SC);
            }
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) o[k] += ko[k];
        }
        if (SCHEME == FV) {
            if (a.flags & F_MAT) {
                TC h = (TC)a.Hm[z];
                o[EXR] += h * c[EXI];
                o[EXI] += -h * c[EXR];
                o[BEXR] += -h * c[BEXI];
                o[BEXI] += h * c[BEXR];
            }
            if (coll) {
                TC SA = (TC)(s_mom[0][lz] - vzv * s_mom[3][lz]);
                TC SB = (TC)(s_mom[1][lz] - vzv * s_mom[4][lz]);
                TC SC = (TC)(s_mom[2][lz] - vzv * s_mom[5][lz]);
                TC f = (TC)(a.mu * a.dv);
                TC Iee = TC(2) * (c[EXR] * SA - c[EXI] * SB);
                TC Ibee = TC(2) * (c[BEXR] * SA + c[BEXI] * SB);
                o[EE] += f * Iee;
                o[XX] += f * (-Iee);
                o[EXR] += f * ((c[XX] - c[EE]) * SA + c[EXI] * SC);
                o[EXI] += f * (-(c[XX] - c[EE]) * SB - c[EXR] * SC);
                o[BEE] += f * Ibee;
                o[BXX] += f * (-Ibee);
                o[BEXR] += f * ((c[BXX] - c[BEE]) * SA - c[BEXI] * SC);
                o[BEXI] += f * ((c[BXX] - c[BEE]) * SB + c[BEXR] * SC);
            }
        }

        // stage combine (a_deferred, common.cuh: with FP64 stage values A is
        // written once, by stage 3)
        constexpr bool AD = a_deferred<STAGE, TIN, TOUT>();
        TOUT u[NCOMP];
#pragma unroll
        for (int k = 0; k < NCOMP; ++k) {
            const double kk = (double)o[k];
            const long long idx = k * a.cs + rowoff;
            if (STAGE == 1) {
                u[k] = (TOUT)(x0[k] + (0.5 * dt) * kk);
                if (!AD && valid) a.A[idx] = x0[k] + (dt / 6.0) * kk;
            } else if (STAGE == 2 || STAGE == 3) {
                const double y = a.Y[idx];
                // stage 3 (FP64): U at this thread's own cell, read before U'' replaces it
                const double u0 = (STAGE == 3 && AD) ? (double)static_cast<const TOUT *>(a.U)[idx]
                                                     : 0.0;
                u[k] = (TOUT)(y + (STAGE == 2 ? 0.5 * dt : dt) * kk);
                if (valid) {
                    if (!AD)
                        a.A[idx] = a.A[idx] + (dt / 3.0) * kk;
                    else if (STAGE == 3)
                        a.A[idx] = y + (u0 - y) * (1.0 / 3.0) + (x0[k] - y) * (2.0 / 3.0) +
                                   (dt / 3.0) * kk;
                }
            } else {
                u[k] = (TOUT)(a.A[idx] + (dt / 6.0) * kk);
            }
        }

        // open-boundary extrapolation needs the value of the cell to the left
        TOUT uleft[NCOMP];
        if (open_bc) {
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) uleft[k] = shfl_idx(u[k], lz > 0 ? lz - 1 : 0, TZ);
        }

        if (valid) {
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) {
                TOUT *row = U + k * a.cs + (long long)v * a.ld + HP;
                row[z] = u[k];
                if (!open_bc) {
                    if (z < a.H) row[z + a.nz] = u[k];
                    if (z >= a.nz - a.H) row[z - a.nz] = u[k];
                } else {
                    if (z == 0)
                        for (int g = 1; g <= a.H; ++g) row[-g] = u[k];
                    if (z == a.nz - 1) {
                        TOUT p0 = uleft[k], p1 = u[k];
                        for (int g = 0; g < a.H; ++g) {
                            TOUT gh = p1 * TOUT(2) - p0;
                            row[a.nz + g] = gh;
                            p0 = p1;
                            p1 = gh;
                        }
                    }
                }
            }
            if (coll) {
                const double Am = (double)u[EXI] + (double)u[BEXI];
                const double Bm = (double)u[EXR] - (double)u[BEXR];
                const double Cm = (double)u[EE] - (double)u[XX] - (double)u[BEE] + (double)u[BXX];
                macc[0] += Am;
                macc[1] += Bm;
                macc[2] += Cm;
                macc[3] += vzv * Am;
                macc[4] += vzv * Bm;
                macc[5] += vzv * Cm;
            }
        }
    }

    if (coll) {
#pragma unroll
        for (int m = 0; m < NMOM; ++m) s_red[rr][m][lz] = macc[m];
        __syncthreads();
        for (int q = tid; q < NMOM * TZ; q += NTHREADS) {
            int m = q / TZ, zz = q % TZ;
            double s = 0.0;
#pragma unroll 4
            for (int t = 0; t < RP; ++t) s += s_red[t][m][zz];
            a.Mout[((long long)vt * NMOM + m) * a.nz + z0 + zz] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// host launcher

template <int SCHEME, int TZ, class TC, class TIN1, class TU, bool B>
static cudaError_t launch_t(const StageArgs &a, int stage, cudaStream_t s, const BatchDev &bd)
{
    dim3 grid = B ? dim3(bd.ntiles) : dim3(a.nz / TZ, a.nvt), block(NTHREADS);
    if (grid.x == 0) return cudaSuccess;
    // FP32-bulk FD stage 1 keeps FP64 arithmetic: its input is the FP64 state
    // and narrowing the 5-point stencil costs more issue than FP64 saves
    using TC1 = std::conditional_t<SCHEME == FD, double, TC>;
    switch (stage) {
    case 1: rk4_stage_kernel<SCHEME, 1, TZ, TC1, TIN1, TU, B><<<grid, block, 0, s>>>(a, bd); break;
    case 2: rk4_stage_kernel<SCHEME, 2, TZ, TC, TU, TU, B><<<grid, block, 0, s>>>(a, bd); break;
    case 3: rk4_stage_kernel<SCHEME, 3, TZ, TC, TU, TU, B><<<grid, block, 0, s>>>(a, bd); break;
    case 4: rk4_stage_kernel<SCHEME, 4, TZ, TC, TU, double, B><<<grid, block, 0, s>>>(a, bd); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int SCHEME, int TZ, bool B>
static cudaError_t launch_p(const StageArgs &a, int stage, int fp32, cudaStream_t s,
                            const BatchDev &bd)
{
    return fp32 ? launch_t<SCHEME, TZ, float, double, float, B>(a, stage, s, bd)
                : launch_t<SCHEME, TZ, double, double, double, B>(a, stage, s, bd);
}

template <bool B>
static cudaError_t launch_s(const StageArgs &a, int scheme, int stage, int tz, int fp32,
                            cudaStream_t s, const BatchDev &bd)
{
    if (scheme == FV) {
        switch (tz) {
        case 8: return launch_p<FV, 8, B>(a, stage, fp32, s, bd);
        case 16: return launch_p<FV, 16, B>(a, stage, fp32, s, bd);
        case 32: return launch_p<FV, 32, B>(a, stage, fp32, s, bd);
        }
    } else {
        switch (tz) {
        case 8: return launch_p<FD, 8, B>(a, stage, fp32, s, bd);
        case 16: return launch_p<FD, 16, B>(a, stage, fp32, s, bd);
        case 32: return launch_p<FD, 32, B>(a, stage, fp32, s, bd);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_rk4_stage(const StageArgs &a, int scheme, int stage, int tz, int fp32,
                             cudaStream_t s)
{
    return launch_s<false>(a, scheme, stage, tz, fp32, s, BatchDev{});
}

// Ensemble launch: one block per table entry (instance, z tile, v tile); the
// z tile width tz is shared by the launch, the v tile is per instance.
cudaError_t launch_rk4_stage_batch(const BatchDev &bd, int scheme, int stage, int tz, int fp32,
                                   cudaStream_t s)
{
    StageArgs a{};
    return launch_s<true>(a, scheme, stage, tz, fp32, s, bd);
}

}  // namespace cosenu
