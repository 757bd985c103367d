// Fused RK4 stage kernels for COSEnu's time-stepping path on sm_100a.
//
// One launch = one RK4 stage of NuOsc::step_rk4 (src/nuosc.hpp:320-348):
// it reads the stage input with its ghost cells, evaluates the right-hand
// side of src/rhs_fv.hpp:115-236 (FV, WENO7) or src/rhs_fd.hpp:6-148 (FD),
// and applies the stage combine in the same pass, in one of the two forms of
// common.cuh: FP64 stage values with the accumulator written once by stage 3
// (832 B per cell-update), or FP32-bulk increments over an FP64 base state
// (576 B).  The epilogue also writes the ghost cells of its output
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
// its neighbour lane, and the block computes the extra face per row and
// component up front, one (row, component) pair per thread.  The right-biased
// reconstruction at face j-1/2 is the left-biased one applied to the mirrored
// stencil, so one routine serves both.
//
// Collective term (rhs_fv.hpp:188-233, rhs_fd.hpp:85-126): its sum over v'
// depends on v' only through A=ex_im+bex_im, B=ex_re-bex_re,
// C=ee-xx-bee+bxx, and sum_k (1 - v_i v_k) X_k = M0[X] - v_i M1[X], so it is
// built from six per-z moments.  Each block writes its per-v-tile partial
// moments; the consumer sums the partials in a fixed order, so results are
// bitwise reproducible run to run.
#include "common.cuh"
#include "weno.cuh"

namespace cosenu {

template <class T> __device__ __forceinline__ T ld_nc(const T *p) { return __ldg(p); }

template <class T> __device__ __forceinline__ T shfl_idx(T x, int src, int width)
{
    return __shfl_sync(0xffffffffu, x, src, width);
}

// The stage input at element offset `i` of a component plane: the stage value
// (FP64 form; or Y at FP32-bulk stage 1), or Y + D (FP32-bulk stages 2-4).
template <bool YPLUS, class TIN>
__device__ __forceinline__ double in_at(const TIN *__restrict__ X, const double *__restrict__ Y,
                                        long long i)
{
    if constexpr (YPLUS)
        return ld_nc(Y + i) + (double)ld_nc(X + i);
    else
        return (double)ld_nc(X + i);
}

// Upwind WENO7 face about element offset i with stencil direction dir (+1:
// left-biased face z+1/2; -1: right-biased face z-1/2).  FP32-bulk (INC):
// FP32 weights on the FP64 stencil differences.
template <bool INC, bool YPLUS, class TIN>
__device__ __forceinline__ double face_at(const TIN *__restrict__ X, const double *__restrict__ Y,
                                          long long i, int dir)
{
    if constexpr (INC) {
        // stencil differences as (Y difference in FP64, rounded) + (D
        // difference in FP32); the face is Y + (D + correction)
        float d[7];
        const double y0 = YPLUS ? ld_nc(Y + i) : (double)ld_nc(X + i);
        const float x0 = YPLUS ? (float)ld_nc(X + i) : 0.f;
#pragma unroll
        for (int k = -3; k <= 3; ++k) {
            if (k == 0) continue;
            const long long j = i + k * dir;
            if constexpr (YPLUS)
                d[k + 3] = (float)(ld_nc(Y + j) - y0) + ((float)ld_nc(X + j) - x0);
            else
                d[k + 3] = (float)((double)ld_nc(X + j) - y0);
        }
        const float corr = weno7_corr(d[0], d[1], d[2], d[4], d[5], d[6]);
        return y0 + (double)(x0 + corr);
    } else {
        double u[7];
#pragma unroll
        for (int k = -3; k <= 3; ++k) u[k + 3] = in_at<YPLUS>(X, Y, i + k * dir);
        return weno7_face(u[0], u[1], u[2], u[3], u[4], u[5], u[6]);
    }
}

// FD advection (src/rhs_fd.hpp:53-73) and Kreiss-Oliger dissipation
// (:128-145) of one component at element offset i.
template <bool YPLUS, class TIN>
__device__ __forceinline__ void fd_terms(const TIN *__restrict__ X, const double *__restrict__ Y,
                                         long long i, int fd_advec, int ko_order, int sv,
                                         double factor, double ko_eps, bool advec, double &adv,
                                         double &ko)
{
    auto u = [&](int k) { return in_at<YPLUS>(X, Y, i + k); };
    const double m2 = u(-2), m1 = u(-1), c0 = u(0), p1 = u(1), p2 = u(2);
    adv = 0.0;
    if (advec) {
        if (fd_advec == 0) {
            adv = factor * ((m2 - p2) - 8.0 * (m1 - p1));
        } else if (fd_advec == 1) {
            adv = factor * (-4.0 * u(-3 * sv) + 18.0 * u(-2 * sv) - 36.0 * u(-sv) + 22.0 * c0);
        } else {
            adv = factor * (u(-3 * sv) - 6.0 * u(-2 * sv) + 18.0 * u(-sv) - 10.0 * c0 -
                            3.0 * u(sv));
        }
    }
    if (ko_order == 5) {
        ko = ko_eps * (u(-3) + u(3) - 6.0 * (m2 + p2) + 15.0 * (m1 + p1) - 20.0 * c0);
    } else {
        ko = ko_eps * (m2 + p2 - 4.0 * (m1 + p1) + 6.0 * c0);
    }
}

// ---------------------------------------------------------------------------
template <int SCHEME, int STAGE, int TZ, class TIN, class TOUT, bool BATCHED>
__global__ void __launch_bounds__(NTHREADS, 2)
    rk4_stage_kernel(const __grid_constant__ StageArgs a0, const BatchDev bd)
{
    constexpr bool INC = inc_form<TIN, TOUT>();
    constexpr bool YPLUS = INC && STAGE >= 2;
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
    __shared__ double s_edge[SCHEME == FV ? MAX_TV : 1][NCOMP];

    const TIN *__restrict__ X = static_cast<const TIN *>(a.X);
    const double *__restrict__ Yb = a.Y;
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
    // FV: the one face per row and component that lies outside this tile's
    // lanes, one (row, component) pair per thread
    if (SCHEME == FV && advec) {
        for (int e = tid; e < nrows * NCOMP; e += NTHREADS) {
            const int r = e / NCOMP, c = e % NCOMP;
            const int v = vbeg + r;
            const int dir = (a.vz[v] >= 0.0) ? 1 : -1;
            const int zc = dir > 0 ? z0 - 1 : z0 + TZ;
            const bool overridden =
                open_bc && ((dir > 0 && z0 == 0) || (dir < 0 && z0 + TZ == a.nz));
            s_edge[r][c] = overridden
                               ? 0.0
                               : face_at<INC, YPLUS>(X, Yb, dev_index(a.cs, a.ld, c, v, zc), dir);
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
        const double rowfac = a.rowfac[v];
        const long long rowoff = (long long)v * a.ld + HP + z;

        // own cell values
        double c[NCOMP];
#pragma unroll
        for (int k = 0; k < NCOMP; ++k) c[k] = in_at<YPLUS>(X, Yb, k * a.cs + rowoff);

        double o[NCOMP];
        if (SCHEME == FV) {
            // advection: upwind flux difference (rhs_fv.hpp:143-162)
            const int dir = (vzv >= 0.0) ? 1 : -1;
            const int src = lz - dir;
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) {
                double adv = 0.0;
                if (advec) {
                    double fown = face_at<INC, YPLUS>(X, Yb, k * a.cs + rowoff, dir);
                    double fnb = shfl_idx(fown, src < 0 ? 0 : (src >= TZ ? TZ - 1 : src), TZ);
                    double fm1 = shfl_idx(fown, lz > 0 ? lz - 1 : 0, TZ);
                    if (dir > 0 && lz == 0) fnb = s_edge[valid ? r : nrows - 1][k];
                    if (dir < 0 && lz == TZ - 1) fnb = s_edge[valid ? r : nrows - 1][k];
                    if (open_bc) {
                        // flux ghosts under OPEN_BC (updateBufferZone on rflux/lflux,
                        // rhs_fv.hpp:118-119): rflux[-1] = rflux[0],
                        // lflux[nz] = 2 lflux[nz-1] - lflux[nz-2]
                        if (dir > 0 && z == 0) fnb = fown;
                        if (dir < 0 && z == a.nz - 1) fnb = fown * 2.0 - fm1;
                    }
                    adv = dir > 0 ? rowfac * (fown - fnb) : rowfac * (fnb - fown);
                }
                o[k] = adv;
            }
            if (a.flags & F_VAC) {
                const double pmo = a.pmo, ct = a.ct, st = a.st;
                o[EE] += -2.0 * st * c[EXI] * pmo;
                o[XX] += 2.0 * st * c[EXI] * pmo;
                o[EXR] += -2.0 * ct * c[EXI] * pmo;
                o[EXI] += (2.0 * ct * c[EXR] + st * (c[EE] - c[XX])) * pmo;
                o[BEE] += -2.0 * st * c[BEXI] * pmo;
                o[BXX] += 2.0 * st * c[BEXI] * pmo;
                o[BEXR] += -2.0 * ct * c[BEXI] * pmo;
                o[BEXI] += (2.0 * ct * c[BEXR] + st * (c[BEE] - c[BXX])) * pmo;
            }
        } else {
            double adv[NCOMP], ko[NCOMP];
            const int sv = (vzv > 0.0) - (vzv < 0.0);
#pragma unroll
            for (int k = 0; k < NCOMP; ++k)
                fd_terms<YPLUS>(X, Yb, k * a.cs + rowoff, a.fd_advec, a.ko_order, sv, rowfac,
                                a.ko_eps, advec, adv[k], ko[k]);
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) o[k] = 0.0;
            if (a.flags & F_VAC) {
                const double pmo = a.pmo, ct = a.ct, st = a.st;
                o[EE] = -pmo * 2.0 * st * c[EXI];
                o[XX] = pmo * 2.0 * st * c[EXI];
                o[EXR] = -pmo * 2.0 * ct * c[EXI];
                o[EXI] = pmo * (2.0 * ct * c[EXR] + st * (c[EE] - c[XX]));
                o[BEE] = -pmo * 2.0 * st * c[BEXI];
                o[BXX] = pmo * 2.0 * st * c[BEXI];
                o[BEXR] = -pmo * 2.0 * ct * c[BEXI];
                o[BEXI] = pmo * (2.0 * ct * c[BEXR] + st * (c[BEE] - c[BXX]));
            }
            if (a.flags & F_MAT) {
                double h = a.Hm[z];
                o[EXR] += h * c[EXI];
                o[EXI] += -h * c[EXR];
                o[BEXR] += -h * c[BEXI];
                o[BEXI] += h * c[BEXR];
            }
#pragma unroll
            for (int k = 0; k < NCOMP; ++k) o[k] += adv[k];
            // KO dissipation is added after the collective term below
            if (coll) {
                double SA = s_mom[0][lz] - vzv * s_mom[3][lz];
                double SB = s_mom[1][lz] - vzv * s_mom[4][lz];
                double SC = s_mom[2][lz] - vzv * s_mom[5][lz];
                double f = a.mu * a.dv;
                double Iee = 2.0 * (c[EXR] * SA - c[EXI] * SB);
                double Ibee = 2.0 * (c[BEXR] * SA + c[BEXI] * SB);
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
                double h = a.Hm[z];
                o[EXR] += h * c[EXI];
                o[EXI] += -h * c[EXR];
                o[BEXR] += -h * c[BEXI];
                o[BEXI] += h * c[BEXR];
            }
            if (coll) {
                double SA = s_mom[0][lz] - vzv * s_mom[3][lz];
                double SB = s_mom[1][lz] - vzv * s_mom[4][lz];
                double SC = s_mom[2][lz] - vzv * s_mom[5][lz];
                double f = a.mu * a.dv;
                double Iee = 2.0 * (c[EXR] * SA - c[EXI] * SB);
                double Ibee = 2.0 * (c[BEXR] * SA + c[BEXI] * SB);
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

        // stage combine (common.cuh)
        TOUT u[NCOMP];
        double um[NCOMP];  // the output as a stage value (for the moments)
#pragma unroll
        for (int k = 0; k < NCOMP; ++k) {
            const double kk = o[k];
            const long long idx = k * a.cs + rowoff;
            if constexpr (INC) {
                const double y = STAGE == 1 ? c[k] : ld_nc(Yb + idx);
                if (STAGE <= 3) {
                    u[k] = (TOUT)((STAGE == 3 ? dt : 0.5 * dt) * kk);
                    um[k] = y + (double)u[k];
                } else {
                    const double d1 = (double)ld_nc(a.T1 + idx), d2 = (double)ld_nc(a.T2 + idx);
                    const double d3 = (double)ld_nc(X + idx);
                    const double yn = y + (d1 + 2.0 * d2 + d3) * (1.0 / 3.0) + (dt / 6.0) * kk;
                    u[k] = (TOUT)yn;
                    um[k] = yn;
                }
            } else {
                if (STAGE == 1) {
                    u[k] = (TOUT)(c[k] + (0.5 * dt) * kk);
                } else if (STAGE == 2 || STAGE == 3) {
                    const double y = a.Y[idx];
                    // stage 3: U at this thread's own cell, read before U'' replaces it
                    const double u0 = STAGE == 3 ? (double)static_cast<const TOUT *>(a.U)[idx] : 0.0;
                    u[k] = (TOUT)(y + (STAGE == 2 ? 0.5 * dt : dt) * kk);
                    if (STAGE == 3 && valid)
                        a.A[idx] = y + (u0 - y) * (1.0 / 3.0) + (c[k] - y) * (2.0 / 3.0) +
                                   (dt / 3.0) * kk;
                } else {
                    u[k] = (TOUT)(a.A[idx] + (dt / 6.0) * kk);
                }
                um[k] = (double)u[k];
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
                const double Am = um[EXI] + um[BEXI];
                const double Bm = um[EXR] - um[BEXR];
                const double Cm = um[EE] - um[XX] - um[BEE] + um[BXX];
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

template <int SCHEME, int TZ, bool B>
static cudaError_t launch_p(const StageArgs &a, int stage, int fp32, cudaStream_t s,
                            const BatchDev &bd)
{
    dim3 grid = B ? dim3(bd.ntiles) : dim3(a.nz / TZ, a.nvt), block(NTHREADS);
    if (grid.x == 0) return cudaSuccess;
    if (fp32) {
        // FP32-bulk: Y in, D1 out; Y + D1 in, D2 out; Y + D2 in, D3 out; Y + D3 in, Y' out
        switch (stage) {
        case 1: rk4_stage_kernel<SCHEME, 1, TZ, double, float, B><<<grid, block, 0, s>>>(a, bd); break;
        case 2: rk4_stage_kernel<SCHEME, 2, TZ, float, float, B><<<grid, block, 0, s>>>(a, bd); break;
        case 3: rk4_stage_kernel<SCHEME, 3, TZ, float, float, B><<<grid, block, 0, s>>>(a, bd); break;
        case 4: rk4_stage_kernel<SCHEME, 4, TZ, float, double, B><<<grid, block, 0, s>>>(a, bd); break;
        default: return cudaErrorInvalidValue;
        }
    } else {
        switch (stage) {
        case 1: rk4_stage_kernel<SCHEME, 1, TZ, double, double, B><<<grid, block, 0, s>>>(a, bd); break;
        case 2: rk4_stage_kernel<SCHEME, 2, TZ, double, double, B><<<grid, block, 0, s>>>(a, bd); break;
        case 3: rk4_stage_kernel<SCHEME, 3, TZ, double, double, B><<<grid, block, 0, s>>>(a, bd); break;
        case 4: rk4_stage_kernel<SCHEME, 4, TZ, double, double, B><<<grid, block, 0, s>>>(a, bd); break;
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
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
