// BF16 GEMM of the surrogate network on the fifth-generation tensor cores:
// tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in tensor memory),
// issued by one thread per CTA, with the operands staged in shared memory by
// all threads and the accumulator read back with tcgen05.ld for the epilogue
// (bias, FP32 pre-activation, optional GELU into BF16).
//
// C[M][N] = sum_k A(m,k) B(k,n) + bias[n].  Each operand is either K-major
// (8 consecutive k values contiguous in global memory) or M/N-major (8
// consecutive rows contiguous: the transposed operands of the backward pass);
// both are written to shared memory in the canonical K-major, no-swizzle UMMA
// layout, the M/N-major ones transposed in registers on the way.
//
// Shared-memory layout of one operand tile of R rows x 64 k per stage: eight
// 8-wide k chunks, chunk c at c * LBO, row r of a chunk at r * 16 bytes
// (8 rows x 16 bytes form one 128-byte core matrix; core matrices adjacent
// in M/N are SBO = 128 bytes apart, in K LBO = R * 16 + 16 bytes apart: the
// extra 16 bytes rotate the banks of the k chunks so the staging stores of a
// quarter-warp hit distinct banks).  One MMA of K 16 reads chunks 2s and
// 2s + 1 (start address + 2s * LBO).
//
// CTA tile 128 (M, one TMEM lane per row) x 64 (N, TMEM columns) x 64 (K per
// stage), a ring of four stages.  K-major operands go from global memory to
// their place in the ring with cp.async, two stages ahead of the tensor
// core; M/N-major operands go through registers one stage ahead (their
// transpose needs them there).  A stage is refilled only after the
// tcgen05.commit of the MMAs that read it has arrived on its mbarrier.
// Every wait is bounded (one second); on expiry the kernel records an error
// word and carries on, and the host reports it.
#include <cuda_bf16.h>

#include <cstdint>
#include <type_traits>

namespace mlpgemm {

constexpr int TBM = 128;  // rows of the tile = TMEM lanes
constexpr int TBN = 64;   // columns of the tile = TMEM columns allocated
constexpr int TBK = 64;   // k per stage (4 MMAs of K 16)
constexpr int NST = 4;    // stages in the ring
constexpr int PRE = 2;    // stages in flight ahead of the tensor core (cp.async)
constexpr int NTHR = 128;
constexpr unsigned long long WAIT_NS = 1000000000ull;

template <int R>
struct Tile {
    static constexpr uint32_t LBO = R * 16 + 16;
    static constexpr uint32_t BYTES = 8 * LBO;
};
using TA = Tile<TBM>;
using TB = Tile<TBN>;
constexpr uint32_t OFF_B = NST * TA::BYTES;
constexpr uint32_t OFF_BAR = OFF_B + NST * TB::BYTES;
constexpr uint32_t SMEM_BYTES = OFF_BAR + 8 * NST + 16;  // two CTAs per SM
static_assert(PRE < NST, "the stage refilled is not the one being consumed");
static_assert(OFF_B % 16 == 0 && OFF_BAR % 16 == 0, "16-byte aligned tiles");

// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
// (bits 7-9 = 1) and B (bits 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TBN >> 3) << 17) |
                           ((uint32_t)(TBM >> 4) << 24);

struct Args {
    const __nv_bfloat16 *A;  // A(m,k) = A[m*lda + k] (K-major) or A[k*lda + m]
    const __nv_bfloat16 *B;  // B(k,n) = B[n*ldb + k] (K-major) or B[k*ldb + n]
    long long lda, ldb;
    int M, N, K;
    float *C;
    int ldc;
    const float *bias;
    __nv_bfloat16 *H;
    int ldh, act, vec;
    int *err;
};

__device__ __forceinline__ uint32_t su32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gtime()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void bar_wait(uint32_t bar, uint32_t parity, int *err)
{
    if (bar_try(bar, parity)) return;
    const unsigned long long t0 = gtime();
    for (uint32_t n = 1;; ++n) {
        if (bar_try(bar, parity)) return;
        if ((n & 63) == 0 && gtime() - t0 > WAIT_NS) {
            atomicCAS(err, 0, 1);
            return;
        }
    }
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo)
{
    // start address >> 4 (bits 0-13), LBO >> 4 (16-29), SBO >> 4 (32-45),
    // descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0)
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
           ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ uint32_t word(const uint4 &v, int w)
{
    return w == 0 ? v.x : w == 1 ? v.y : w == 2 ? v.z : v.w;
}

// K-major operand: R rows x 8 chunks; item q -> chunk q & 7 of row q >> 3
// (8 lanes read one row's 128 contiguous bytes).
template <int R>
struct KMajor {
    static constexpr int NI = R * 8 / NTHR;
    uint4 v[NI];
    __device__ __forceinline__ void load(const __nv_bfloat16 *X, long long ld, int rtot, int ktot,
                                         int r0, int k0)
    {
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int q = threadIdx.x + NTHR * i, kc = q & 7, r = q >> 3;
            const int rg = r0 + r, kg = k0 + kc * 8;
            v[i] = (rg < rtot && kg < ktot)
                       ? __ldg(reinterpret_cast<const uint4 *>(X + (long long)rg * ld + kg))
                       : make_uint4(0, 0, 0, 0);
        }
    }
    __device__ __forceinline__ void store(unsigned char *s) const
    {
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int q = threadIdx.x + NTHR * i, kc = q & 7, r = q >> 3;
            *reinterpret_cast<uint4 *>(s + kc * Tile<R>::LBO + r * 16) = v[i];
        }
    }
    // the same chunks straight to their place in the stage (cp.async, 16
    // bytes each; out of range: a zero-filled chunk and no global read)
    static __device__ __forceinline__ void copy_async(unsigned char *s, const __nv_bfloat16 *X,
                                                      long long ld, int rtot, int ktot, int r0,
                                                      int k0)
    {
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int q = threadIdx.x + NTHR * i, kc = q & 7, r = q >> 3;
            const int rg = r0 + r, kg = k0 + kc * 8;
            const bool in = rg < rtot && kg < ktot;
            const __nv_bfloat16 *src = in ? X + (long long)rg * ld + kg : X;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                             su32(s + kc * Tile<R>::LBO + r * 16)),
                         "l"(src), "r"(in ? 16 : 0)
                         : "memory");
        }
    }
};

// M/N-major operand: blocks of 8 rows x 8 k; block q -> k chunk q & 7, row
// group q >> 3; a thread reads 8 k-rows of 16 bytes and writes 8 rows of
// 16 bytes after an 8 x 8 transpose of BF16 pairs in registers.
template <int R>
struct MNMajor {
    static constexpr int NB = (R + NTHR - 1) / NTHR;
    uint4 v[NB][8];
    __device__ __forceinline__ void load(const __nv_bfloat16 *X, long long ld, int rtot, int ktot,
                                         int r0, int k0)
    {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int q = threadIdx.x + NTHR * b;
            const int kc = q & 7, rg = r0 + (q >> 3) * 8;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int kg = k0 + kc * 8 + j;
                v[b][j] = (q < R && rg < rtot && kg < ktot)
                              ? __ldg(reinterpret_cast<const uint4 *>(X + (long long)kg * ld + rg))
                              : make_uint4(0, 0, 0, 0);
            }
        }
    }
    __device__ __forceinline__ void store(unsigned char *s) const
    {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int q = threadIdx.x + NTHR * b;
            if (q >= R) continue;
            const int kc = q & 7, r = (q >> 3) * 8;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                // row r + i: k values 0..7 of this chunk = element i of v[0..7]
                const uint32_t sel = (i & 1) ? 0x7632u : 0x5410u;
                uint4 o;
                o.x = __byte_perm(word(v[b][0], i >> 1), word(v[b][1], i >> 1), sel);
                o.y = __byte_perm(word(v[b][2], i >> 1), word(v[b][3], i >> 1), sel);
                o.z = __byte_perm(word(v[b][4], i >> 1), word(v[b][5], i >> 1), sel);
                o.w = __byte_perm(word(v[b][6], i >> 1), word(v[b][7], i >> 1), sel);
                *reinterpret_cast<uint4 *>(s + kc * Tile<R>::LBO + (r + i) * 16) = o;
            }
        }
    }
};

template <bool AK, bool BK>
__global__ void __launch_bounds__(NTHR) gemm_tc_kernel(Args p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + OFF_BAR + 8 * NST);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * TBN;
    const int nk = (p.K + TBK - 1) / TBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         su32(tslot)),
                     "r"(TBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < NST; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bars[b])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    // M/N-major operands: staged through registers (the K-major members of
    // ra / rb stay unused)
    typename std::conditional<AK, KMajor<TBM>, MNMajor<TBM>>::type ra;
    typename std::conditional<BK, KMajor<TBN>, MNMajor<TBN>>::type rb;
    // one cp.async group per stage (empty where no operand is K-major or the
    // stage is past the end), so that group n is stage n
    auto fill_async = [&](int st) {
        if (st < nk) {
            const int b = st % NST;
            if (AK)
                KMajor<TBM>::copy_async(smem + b * TA::BYTES, p.A, p.lda, p.M, p.K, m0, st * TBK);
            if (BK)
                KMajor<TBN>::copy_async(smem + OFF_B + b * TB::BYTES, p.B, p.ldb, p.N, p.K, n0,
                                        st * TBK);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
#pragma unroll
    for (int st = 0; st < PRE; ++st) fill_async(st);
    if (!AK) ra.load(p.A, p.lda, p.M, p.K, m0, 0);
    if (!BK) rb.load(p.B, p.ldb, p.N, p.K, n0, 0);
    const uint32_t sbase = su32(smem);
    for (int kb = 0; kb < nk; ++kb) {
        const int buf = kb % NST;
        // refill the stage PRE ahead once the MMAs that last read its buffer
        // (stage kb + PRE - NST) are done; that wait also frees stage kb + PRE
        // for the register-staged operands when their turn comes
        const int st = kb + PRE;
        if (st < nk && st >= NST) bar_wait(su32(&bars[st % NST]), ((st - NST) / NST) & 1, p.err);
        fill_async(st);
        asm volatile("cp.async.wait_group %0;" ::"n"(PRE) : "memory");  // stage kb landed
        if (!AK) {
            ra.store(smem + buf * TA::BYTES);
            if (kb + 1 < nk) ra.load(p.A, p.lda, p.M, p.K, m0, (kb + 1) * TBK);
        }
        if (!BK) {
            rb.store(smem + OFF_B + buf * TB::BYTES);
            if (kb + 1 < nk) rb.load(p.B, p.ldb, p.N, p.K, n0, (kb + 1) * TBK);
        }
        // the tensor core reads shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = sbase + buf * TA::BYTES, sb = sbase + OFF_B + buf * TB::BYTES;
#pragma unroll
            for (int s = 0; s < TBK / 16; ++s) {
                const uint64_t da = sdesc(sa + 2 * s * TA::LBO, TA::LBO);
                const uint64_t db = sdesc(sb + 2 * s * TB::LBO, TB::LBO);
                const uint32_t acc = (kb > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(IDESC), "r"(acc));
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    su32(&bars[buf]))
                : "memory");
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the last commit of each stage: all MMAs done
    for (int b = 0; b < NST && b < nk; ++b)
        bar_wait(su32(&bars[b]), ((nk - 1 - b) / NST) & 1, p.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // epilogue: warp w holds rows 32w..32w+31 (TMEM lanes), 16 columns per load
    const int m = m0 + warp * 32 + lane;
#pragma unroll
    for (int c = 0; c < TBN / 16; ++c) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + c * 16;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (m >= p.M) continue;
        const int nb = n0 + c * 16;
        if (nb >= p.N) continue;
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
            v[j] = __uint_as_float(r[j]) + ((p.bias && nb + j < p.N) ? p.bias[nb + j] : 0.f);
        float *crow = p.C + (long long)m * p.ldc + nb;
        __nv_bfloat16 *hrow = p.H ? p.H + (long long)m * p.ldh + nb : nullptr;
        if (p.vec && nb + 16 <= p.N) {
#pragma unroll
            for (int j = 0; j < 16; j += 4)
                *reinterpret_cast<float4 *>(crow + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            if (hrow) {
                uint32_t h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float a = p.act ? gelu(v[2 * j]) : v[2 * j];
                    const float b = p.act ? gelu(v[2 * j + 1]) : v[2 * j + 1];
                    h[j] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(a)) |
                           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(b)) << 16);
                }
                *reinterpret_cast<uint4 *>(hrow) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4 *>(hrow + 8) = make_uint4(h[4], h[5], h[6], h[7]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                if (nb + j >= p.N) continue;
                crow[j] = v[j];
                if (hrow) hrow[j] = __float2bfloat16(p.act ? gelu(v[j]) : v[j]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TBN));
    }
}

template <bool AK, bool BK>
cudaError_t launch(const Args &a, cudaStream_t s)
{
    static unsigned long long ready = 0;  // devices whose attribute is set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !(ready >> dev & 1)) {
        e = cudaFuncSetAttribute(gemm_tc_kernel<AK, BK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SMEM_BYTES);
        if (e != cudaSuccess) return e;
        if (dev < 64) ready |= 1ull << dev;
    }
    dim3 grid((a.N + TBN - 1) / TBN, (a.M + TBM - 1) / TBM);
    gemm_tc_kernel<AK, BK><<<grid, NTHR, SMEM_BYTES, s>>>(a);
    return cudaPeekAtLastError();  // left pending for the caller's check
}

}  // namespace mlpgemm

// C = A B (+ bias, GELU into H) with A(m,k) = A[m*sam + k*sak] and B(k,n) =
// B[k*sbk + n*sbn] on the tcgen05 path.  Returns cudaErrorNotSupported when
// the operands do not fit it (a unit stride on each operand, the other
// stride and the contiguous extent multiples of 8 elements, 16-byte aligned
// bases); the caller then uses its mma.sync kernel.
cudaError_t mlp_gemm_tc(const __nv_bfloat16 *A, long long sam, long long sak,
                        const __nv_bfloat16 *B, long long sbk, long long sbn, int M, int N, int K,
                        float *C, int ldc, const float *bias, __nv_bfloat16 *H, int ldh, int act,
                        int *err, cudaStream_t s)
{
    using namespace mlpgemm;
    if (M < 1 || N < 1 || K < 1) return cudaErrorNotSupported;
    const bool ak = sak == 1, bk = sbk == 1;
    const long long lda = ak ? sam : sak, ldb = bk ? sbn : sbk;
    if (!ak && sam != 1) return cudaErrorNotSupported;
    if (!bk && sbn != 1) return cudaErrorNotSupported;
    if (lda % 8 || ldb % 8) return cudaErrorNotSupported;
    if ((ak ? K : M) % 8 || (bk ? K : N) % 8) return cudaErrorNotSupported;
    if (((uintptr_t)A | (uintptr_t)B) & 15) return cudaErrorNotSupported;
    Args a;
    a.A = A;
    a.B = B;
    a.lda = lda;
    a.ldb = ldb;
    a.M = M;
    a.N = N;
    a.K = K;
    a.C = C;
    a.ldc = ldc;
    a.bias = bias;
    a.H = H;
    a.ldh = ldh;
    a.act = act;
    a.vec = (ldc % 4 == 0 && ((uintptr_t)C & 15) == 0 &&
             (!H || (ldh % 8 == 0 && ((uintptr_t)H & 15) == 0)))
                ? 1
                : 0;
    a.err = err;
    if (ak && bk) return launch<true, true>(a, s);
    if (ak) return launch<true, false>(a, s);
    if (bk) return launch<false, true>(a, s);
    return launch<false, false>(a, s);
}
