// Auxiliary kernels around the RK4 stages: ghost fill after an upload,
// velocity moments of a state, the analysis reductions of src/analysis.hpp,
// P_ee(v), and on-device initial conditions.
//
// All reductions use a fixed grid and a fixed summation tree, so their
// results are bitwise reproducible from run to run.
#include "common.cuh"

namespace cosenu {

constexpr int DIAG_BLOCKS = 592;  // fixed (4 x 148) so the reduction tree never changes
enum DiagSlot {
    S_DPMAX = 0, S_DBPMAX, S_AVDP, S_AVBDP, S_N0, S_BN0, S_E1, S_E2, S_E3, S_NEE, S_NBEE,
    S_NEE0, S_NBEE0, S_TR, S_BTR, S_ELN, S_BAD, NSLOT
};

// ---------------------------------------------------------------------------
// Ghost cells of every row of an 8-component buffer, as updateBufferZone
// (src/nuosc.hpp:212-278) leaves them: periodic copies, or (open) the first
// interior value on the left and a running linear extrapolation on the right.
__global__ void ghost_fill_kernel(double *buf, long long cs, int ld, int nz, int nvz, int H, int bc)
{
    int row = blockIdx.x * blockDim.x + threadIdx.x;  // c * nvz + v
    if (row >= NCOMP * nvz) return;
    int c = row / nvz, v = row % nvz;
    double *r = buf + (long long)c * cs + (long long)v * ld + HP;
    if (bc == 0) {
        for (int g = 1; g <= H; ++g) {
            r[-g] = r[nz - g];
            r[nz + g - 1] = r[g - 1];
        }
    } else {
        for (int g = 1; g <= H; ++g) r[-g] = r[0];
        double p0 = r[nz - 2], p1 = r[nz - 1];
        for (int g = 0; g < H; ++g) {
            double gh = p1 * 2 - p0;
            r[nz + g] = gh;
            p0 = p1;
            p1 = gh;
        }
    }
}

// Per-v-tile partial velocity moments of a state (the layout the stage
// kernels consume): M[(vt*6 + m)*nz + z].
template <int TZ>
__global__ void __launch_bounds__(NTHREADS) moments_kernel(const double *__restrict__ X,
                                                           double *__restrict__ M,
                                                           const double *__restrict__ vz,
                                                           long long cs, int ld, int nz, int nvz,
                                                           int tv)
{
    constexpr int RP = NTHREADS / TZ;
    __shared__ double s_red[RP][NMOM][TZ];
    int lz = threadIdx.x % TZ, rr = threadIdx.x / TZ;
    int z0 = blockIdx.x * TZ, z = z0 + lz, vt = blockIdx.y;
    int vbeg = vt * tv, vend = min(vbeg + tv, nvz);
    double acc[NMOM] = {0, 0, 0, 0, 0, 0};
    for (int v = vbeg + rr; v < vend; v += RP) {
        long long o = (long long)v * ld + HP + z;
        double A = X[EXI * cs + o] + X[BEXI * cs + o];
        double B = X[EXR * cs + o] - X[BEXR * cs + o];
        double C = X[EE * cs + o] - X[XX * cs + o] - X[BEE * cs + o] + X[BXX * cs + o];
        double w = vz[v];
        acc[0] += A; acc[1] += B; acc[2] += C;
        acc[3] += w * A; acc[4] += w * B; acc[5] += w * C;
    }
#pragma unroll
    for (int m = 0; m < NMOM; ++m) s_red[rr][m][lz] = acc[m];
    __syncthreads();
    for (int q = threadIdx.x; q < NMOM * TZ; q += NTHREADS) {
        int m = q / TZ, zz = q % TZ;
        double s = 0.0;
        for (int t = 0; t < RP; ++t) s += s_red[t][m][zz];
        M[((long long)vt * NMOM + m) * nz + z0 + zz] = s;
    }
}

// ---------------------------------------------------------------------------
// Analysis (src/analysis.hpp): per cell the polarisation vectors of the
// current state and of state0 (cal_pol, :27-46, note the + sign of bP2),
// |dP| statistics (dcon, :71-130), the M0 moment (cal_Mn n = 0, :50-67) and
// the survival-probability sums (surv_prob, :134-185), plus trace and ELN
// sums and a count of non-finite values.

struct DiagIn {
    const double *Y, *S0, *G, *bG;  // G, bG: one plane [nvz][ld]
    long long cs;
    int ld, nz, nvz;
    double dz, dv;
};

__device__ __forceinline__ void diag_cell(const DiagIn &d, int v, int z, double *acc)
{
    long long o = (long long)v * d.ld + HP + z;
    double c[NCOMP], c0[NCOMP];
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) {
        c[k] = d.Y[k * d.cs + o];
        c0[k] = d.S0[k * d.cs + o];
    }
    double G = d.G[o], bG = d.bG[o];
    double P1 = 2.0 * c[EXR] / G, P2 = -2.0 * c[EXI] / G, P3 = (c[EE] - c[XX]) / G;
    double bP1 = 2.0 * c[BEXR] / bG, bP2 = 2.0 * c[BEXI] / bG, bP3 = (c[BEE] - c[BXX]) / bG;
    double n = fabs(sqrt(P1 * P1 + P2 * P2 + P3 * P3));
    double bn = fabs(sqrt(bP1 * bP1 + bP2 * bP2 + bP3 * bP3));
    double Q1 = 2.0 * c0[EXR] / G, Q2 = -2.0 * c0[EXI] / G, Q3 = (c0[EE] - c0[XX]) / G;
    double bQ1 = 2.0 * c0[BEXR] / bG, bQ2 = 2.0 * c0[BEXI] / bG, bQ3 = (c0[BEE] - c0[BXX]) / bG;
    double n0 = fabs(sqrt(Q1 * Q1 + Q2 * Q2 + Q3 * Q3));
    double bn0 = fabs(sqrt(bQ1 * bQ1 + bQ2 * bQ2 + bQ3 * bQ3));
    double dP = fabs(n - n0), dbP = fabs(bn - bn0);
    acc[S_DPMAX] = fmax(acc[S_DPMAX], dP);
    acc[S_DBPMAX] = fmax(acc[S_DBPMAX], dbP);
    acc[S_AVDP] += dP * G;
    acc[S_AVBDP] += dbP * bG;
    acc[S_N0] += G;
    acc[S_BN0] += bG;
    acc[S_E1] += (G * P1 - bG * bP1) * d.dz * d.dv;
    acc[S_E2] += (G * P2 - bG * bP2) * d.dz * d.dv;
    acc[S_E3] += (G * P3 - bG * bP3) * d.dz * d.dv;
    acc[S_NEE] += c[EE] * d.dz * d.dv;
    acc[S_NBEE] += c[BEE] * d.dz * d.dv;
    acc[S_NEE0] += c0[EE] * d.dz * d.dv;
    acc[S_NBEE0] += c0[BEE] * d.dz * d.dv;
    double dzdv = d.dz * d.dv;
    acc[S_TR] += (c[EE] + c[XX]) * dzdv;
    acc[S_BTR] += (c[BEE] + c[BXX]) * dzdv;
    acc[S_ELN] += (c[EE] - c[BEE]) * dzdv;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NCOMP; ++k) s += c[k];
    if (!isfinite(s)) acc[S_BAD] += 1.0;
}

__device__ __forceinline__ bool slot_is_max(int s) { return s == S_DPMAX || s == S_DBPMAX; }

// block-wide fixed-order reduction of NSLOT values; result in thread 0
__device__ void block_reduce_slots(double *acc, double (*sh)[NSLOT])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        double x = acc[s];
        for (int off = 16; off > 0; off >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, x, off);
            x = slot_is_max(s) ? fmax(x, y) : x + y;
        }
        if (lane == 0) sh[warp][s] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < NSLOT; ++s) {
            double x = sh[0][s];
            for (int w = 1; w < NTHREADS / 32; ++w) x = slot_is_max(s) ? fmax(x, sh[w][s]) : x + sh[w][s];
            acc[s] = x;
        }
    }
}

__global__ void __launch_bounds__(NTHREADS) diag_partial_kernel(const DiagIn d, double *part)
{
    __shared__ double sh[NTHREADS / 32][NSLOT];
    double acc[NSLOT];
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) acc[s] = 0.0;
    const long long ncell = (long long)d.nvz * d.nz;
    for (long long q = blockIdx.x * (long long)NTHREADS + threadIdx.x; q < ncell;
         q += (long long)gridDim.x * NTHREADS) {
        int v = (int)(q / d.nz), z = (int)(q % d.nz);
        diag_cell(d, v, z, acc);
    }
    block_reduce_slots(acc, sh);
    if (threadIdx.x == 0)
        for (int s = 0; s < NSLOT; ++s) part[(long long)blockIdx.x * NSLOT + s] = acc[s];
}

// out: dP_max avdP avbdP M0 e1 e2 e3 Pee Pbee trace btrace eln bad
__global__ void diag_final_kernel(const double *part, int nblk, double *out)
{
    __shared__ double sh[NTHREADS / 32][NSLOT];
    double acc[NSLOT];
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) acc[s] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += NTHREADS)
        for (int s = 0; s < NSLOT; ++s)
            acc[s] = slot_is_max(s) ? fmax(acc[s], part[(long long)b * NSLOT + s])
                                    : acc[s] + part[(long long)b * NSLOT + s];
    block_reduce_slots(acc, sh);
    if (threadIdx.x == 0) {
        out[0] = fmax(acc[S_DPMAX], acc[S_DBPMAX]);
        out[1] = acc[S_AVDP] / acc[S_N0];
        out[2] = acc[S_AVBDP] / acc[S_BN0];
        out[3] = sqrt(acc[S_E1] * acc[S_E1] + acc[S_E2] * acc[S_E2] + acc[S_E3] * acc[S_E3]);
        out[4] = acc[S_E1];
        out[5] = acc[S_E2];
        out[6] = acc[S_E3];
        out[7] = acc[S_NEE] / acc[S_NEE0];
        out[8] = acc[S_NBEE] / acc[S_NBEE0];
        out[9] = acc[S_TR];
        out[10] = acc[S_BTR];
        out[11] = acc[S_ELN];
        out[12] = acc[S_BAD];
    }
}

// P_ee(v): one block per row, fixed-order reduction over z.
__global__ void __launch_bounds__(NTHREADS) pee_v_kernel(const double *__restrict__ Y,
                                                         const double *__restrict__ S0,
                                                         long long cs, int ld, int nz,
                                                         double *out /* [2][nvz] */, int nvz)
{
    __shared__ double sh[4][NTHREADS / 32];
    int v = blockIdx.x;
    double a[4] = {0, 0, 0, 0};
    for (int z = threadIdx.x; z < nz; z += NTHREADS) {
        long long o = (long long)v * ld + HP + z;
        a[0] += Y[EE * cs + o];
        a[1] += S0[EE * cs + o];
        a[2] += Y[BEE * cs + o];
        a[3] += S0[BEE * cs + o];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 4; ++k) {
        double x = a[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4];
        for (int k = 0; k < 4; ++k) {
            t[k] = sh[k][0];
            for (int w = 1; w < NTHREADS / 32; ++w) t[k] += sh[k][w];
        }
        out[v] = t[0] / t[1];
        out[nvz + v] = t[2] / t[3];
    }
}

// ---------------------------------------------------------------------------
// Initial conditions.

// Philox-4x32-10 (Salmon et al., SC'11): published round constants and
// Weyl key increments.
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Seeded state: Gv/bGv per row from the host (normalised Gaussian profiles);
// per cell four uniform draws in [-amp, amp].  Written with round-to-nearest
// intrinsics so the bits equal those of the host recipe.
__global__ void init_seeded_kernel(double *Y, double *G, double *bG, const double *Gv,
                                   const double *bGv, long long cs, int ld, int nz, int nvz,
                                   uint32_t k0, uint32_t k1, uint32_t instance, double amp)
{
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz * nvz) return;
    int i = (int)(q / nz), j = (int)(q % nz);
    uint32_t c[4] = {(uint32_t)j, (uint32_t)i, instance, 0u};
    philox4x32_10(c, k0, k1);
    double e[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        double u = __dmul_rn(__dadd_rn((double)c[t], 0.5), 1.0 / 4294967296.0);
        e[t] = __dmul_rn(amp, __dsub_rn(__dmul_rn(2.0, u), 1.0));
    }
    double s = __dsqrt_rn(__dsub_rn(__dsub_rn(1.0, __dmul_rn(e[0], e[0])), __dmul_rn(e[1], e[1])));
    double bs = __dsqrt_rn(__dsub_rn(__dsub_rn(1.0, __dmul_rn(e[2], e[2])), __dmul_rn(e[3], e[3])));
    double gv = Gv[i], bgv = bGv[i];
    long long o = (long long)i * ld + HP + j;
    double h = __dmul_rn(0.5, gv), bh = __dmul_rn(0.5, bgv);
    G[o] = gv;
    bG[o] = bgv;
    Y[EE * cs + o] = __dmul_rn(h, __dadd_rn(1.0, s));
    Y[XX * cs + o] = __dmul_rn(h, __dsub_rn(1.0, s));
    Y[EXR * cs + o] = __dmul_rn(h, e[0]);
    Y[EXI * cs + o] = __dmul_rn(h, e[1]);
    Y[BEE * cs + o] = __dmul_rn(bh, __dadd_rn(1.0, bs));
    Y[BXX * cs + o] = __dmul_rn(bh, __dsub_rn(1.0, bs));
    Y[BEXR * cs + o] = __dmul_rn(bh, e[2]);
    Y[BEXI * cs + o] = __dmul_rn(bh, e[3]);
}

// The reference's default initial condition (src/initialize.hpp:6-47); the
// per-z perturbation e(z), sqrt(1-e^2) and the per-v profiles come from the
// host.
__global__ void init_reference_kernel(double *Y, double *G, double *bG, const double *Gv,
                                      const double *bGv, const double *ez, const double *ez_,
                                      long long cs, int ld, int nz, int nvz)
{
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)nz * nvz) return;
    int i = (int)(q / nz), j = (int)(q % nz);
    long long o = (long long)i * ld + HP + j;
    double g = Gv[i], bg = bGv[i], e = ez[j], e_ = ez_[j];
    G[o] = g;
    bG[o] = bg;
    Y[EE * cs + o] = __dmul_rn(__dmul_rn(0.5, g), __dadd_rn(1.0, e_));
    Y[XX * cs + o] = __dmul_rn(__dmul_rn(0.5, g), __dsub_rn(1.0, e_));
    Y[EXR * cs + o] = __dmul_rn(__dmul_rn(0.5, g), __dadd_rn(0.0, e));
    Y[EXI * cs + o] = -0.0;
    Y[BEE * cs + o] = __dmul_rn(__dmul_rn(0.5, bg), __dadd_rn(1.0, e_));
    Y[BXX * cs + o] = __dmul_rn(__dmul_rn(0.5, bg), __dsub_rn(1.0, e_));
    Y[BEXR * cs + o] = __dmul_rn(__dmul_rn(0.5, bg), __dadd_rn(0.0, e));
    Y[BEXI * cs + o] = 0.0;
}

// ---------------------------------------------------------------------------
// host launchers

cudaError_t launch_ghost_fill(double *buf, long long cs, int ld, int nz, int nvz, int H, int bc,
                              cudaStream_t s)
{
    int rows = NCOMP * nvz;
    ghost_fill_kernel<<<(rows + 127) / 128, 128, 0, s>>>(buf, cs, ld, nz, nvz, H, bc);
    return cudaGetLastError();
}

cudaError_t launch_moments(const double *X, double *M, const double *vz, long long cs, int ld,
                           int nz, int nvz, int tz, int tv, cudaStream_t s)
{
    dim3 grid(nz / tz, (nvz + tv - 1) / tv);
    switch (tz) {
    case 8: moments_kernel<8><<<grid, NTHREADS, 0, s>>>(X, M, vz, cs, ld, nz, nvz, tv); break;
    case 16: moments_kernel<16><<<grid, NTHREADS, 0, s>>>(X, M, vz, cs, ld, nz, nvz, tv); break;
    case 32: moments_kernel<32><<<grid, NTHREADS, 0, s>>>(X, M, vz, cs, ld, nz, nvz, tv); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int diag_blocks() { return DIAG_BLOCKS; }
int diag_slots() { return NSLOT; }

cudaError_t launch_diag(const double *Y, const double *S0, const double *G, const double *bG,
                        long long cs, int ld, int nz, int nvz, double dz, double dv, double *part,
                        double *out, cudaStream_t s)
{
    DiagIn d{Y, S0, G, bG, cs, ld, nz, nvz, dz, dv};
    diag_partial_kernel<<<DIAG_BLOCKS, NTHREADS, 0, s>>>(d, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    diag_final_kernel<<<1, NTHREADS, 0, s>>>(part, DIAG_BLOCKS, out);
    return cudaGetLastError();
}

cudaError_t launch_pee_v(const double *Y, const double *S0, long long cs, int ld, int nz, int nvz,
                         double *out, cudaStream_t s)
{
    pee_v_kernel<<<nvz, NTHREADS, 0, s>>>(Y, S0, cs, ld, nz, out, nvz);
    return cudaGetLastError();
}

cudaError_t launch_init_seeded(double *Y, double *G, double *bG, const double *Gv,
                               const double *bGv, long long cs, int ld, int nz, int nvz,
                               uint64_t seed, uint32_t instance, double amp, cudaStream_t s)
{
    long long n = (long long)nz * nvz;
    init_seeded_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        Y, G, bG, Gv, bGv, cs, ld, nz, nvz, (uint32_t)seed, (uint32_t)(seed >> 32), instance, amp);
    return cudaGetLastError();
}

cudaError_t launch_init_reference(double *Y, double *G, double *bG, const double *Gv,
                                  const double *bGv, const double *ez, const double *ez_,
                                  long long cs, int ld, int nz, int nvz, cudaStream_t s)
{
    long long n = (long long)nz * nvz;
    init_reference_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Y, G, bG, Gv, bGv, ez, ez_,
                                                                       cs, ld, nz, nvz);
    return cudaGetLastError();
}

}  // namespace cosenu
