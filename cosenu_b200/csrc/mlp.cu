// Surrogate network: a fully connected net (n_in -> hidden x L -> n_out, GELU
// between layers) that maps the initial angular distributions and (alpha, mu)
// of a simulation to its late-time, angle-resolved survival probability.
// BF16 weights and activations feed the tensor cores with FP32 accumulation;
// FP32 master weights are updated by AdamW.  Everything here is hand written:
// the GEMMs (tcgen05.mma with the accumulator in tensor memory, mlp_gemm.cu;
// the warp-level mma.sync m16n8k16 kernel below stays for operands that do
// not fit that path and as the comparison the surrogate timing reports with
// COSENU_MLP_GEMM=mma), the GELU forward/backward, the loss, the bias
// reductions and the optimizer.
//
// Layout: activations are batch-major rows; layer l has W_l [out][in] and b_l
// [out]; the input width is padded to a multiple of 16 with zero columns.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cosenu_b200.h"

cudaError_t mlp_gemm_tc(const __nv_bfloat16 *A, long long sam, long long sak,
                        const __nv_bfloat16 *B, long long sbk, long long sbn, int M, int N, int K,
                        float *C, int ldc, const float *bias, __nv_bfloat16 *H, int ldh, int act,
                        int *err, cudaStream_t s);

namespace {

// ---------------------------------------------------------------------------
// C[M][N] = sum_k A(m,k) B(k,n)  (+ bias[n]) with A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn] (BF16).  Epilogue: FP32 C (ldc), optionally
// GELU(C) as BF16 (ldh).  64x64 block tile, 4 warps of 32x32, K step 32.
constexpr int GT = 64, GK = 32;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
           x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(
    const __nv_bfloat16 *__restrict__ A, long long sam, long long sak,
    const __nv_bfloat16 *__restrict__ B, long long sbk, long long sbn, int M, int N, int K,
    float *__restrict__ C, int ldc, const float *__restrict__ bias,
    __nv_bfloat16 *__restrict__ H, int ldh, int act)
{
    __shared__ __nv_bfloat16 As[GT][GK + 8];
    __shared__ __nv_bfloat16 Bs[GK][GT + 8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int q = tid; q < GT * GK; q += 128) {
            int r = q / GK, c = q % GK;
            int m = m0 + r, k = k0 + c;
            As[r][c] = (m < M && k < K) ? A[m * sam + k * sak] : zero;
            int kk = q / GT, nn = q % GT;
            int k2 = k0 + kk, n = n0 + nn;
            Bs[kk][nn] = (k2 < K && n < N) ? B[k2 * sbk + n * sbn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < GK; ks += 16) {
            uint32_t af[2][4], bfr[4][2];
            const int r = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int mr = wm + i * 16 + r;
                af[i][0] = pack2(As[mr][ks + c], As[mr][ks + c + 1]);
                af[i][1] = pack2(As[mr + 8][ks + c], As[mr + 8][ks + c + 1]);
                af[i][2] = pack2(As[mr][ks + c + 8], As[mr][ks + c + 9]);
                af[i][3] = pack2(As[mr + 8][ks + c + 8], As[mr + 8][ks + c + 9]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int nc = wn + j * 8 + r;
                bfr[j][0] = pack2(Bs[ks + c][nc], Bs[ks + c + 1][nc]);
                bfr[j][1] = pack2(Bs[ks + c + 8][nc], Bs[ks + c + 9][nc]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]),
                          "+f"(acc[i][j][3])
                        : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]),
                          "r"(bfr[j][0]), "r"(bfr[j][1]));
        }
        __syncthreads();
    }
    const int r = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int m = m0 + wm + i * 16 + r + h * 8;
                if (m >= M) continue;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int n = n0 + wn + j * 8 + c + e;
                    if (n >= N) continue;
                    float v = acc[i][j][2 * h + e] + (bias ? bias[n] : 0.f);
                    C[(long long)m * ldc + n] = v;
                    if (H) H[(long long)m * ldh + n] = __float2bfloat16(act ? gelu(v) : v);
                }
            }
}

// tcgen05 path when `tc` and the operands fit it; a launch error stays
// pending for the caller's next cudaGetLastError.
void gemm(const __nv_bfloat16 *A, long long sam, long long sak, const __nv_bfloat16 *B,
          long long sbk, long long sbn, int M, int N, int K, float *C, int ldc, const float *bias,
          __nv_bfloat16 *H, int ldh, int act, bool tc, int *err, cudaStream_t s)
{
    if (tc && mlp_gemm_tc(A, sam, sak, B, sbk, sbn, M, N, K, C, ldc, bias, H, ldh, act, err, s) !=
                  cudaErrorNotSupported)
        return;
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    gemm_bf16_kernel<<<grid, 128, 0, s>>>(A, sam, sak, B, sbk, sbn, M, N, K, C, ldc, bias, H, ldh,
                                          act);
}

// MSE loss 1/(B*N) sum (y - t)^2: gradient in BF16 (for the next GEMM) and
// FP32, per-block partial loss.
__global__ void mse_kernel(const float *Y, const float *T, int n, float scale, float *dY,
                           __nv_bfloat16 *dYb, float *partial)
{
    __shared__ float sh[256];
    float l = 0.f;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        float d = Y[i] - T[i];
        l += d * d;
        float g = 2.f * d * scale;
        dY[i] = g;
        dYb[i] = __float2bfloat16(g);
    }
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// dZ = dH * gelu'(Z) (FP32 dH from the GEMM), written in FP32 and BF16.
__global__ void gelu_back_kernel(const float *dH, const float *Z, int n, float *dZ,
                                 __nv_bfloat16 *dZb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float g = dH[i] * gelu_grad(Z[i]);
    dZ[i] = g;
    dZb[i] = __float2bfloat16(g);
}

// db[n] = sum over rows of dZ[m][n] (fixed order).
__global__ void colsum_kernel(const float *dZ, int M, int N, float *db)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; ++m) s += dZ[(long long)m * N + n];
    db[n] = s;
}

// AdamW on FP32 master parameters; refreshes the BF16 copy of weights.
__global__ void adamw_kernel(float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb,
                             long long n, float lr, float b1, float b2, float eps, float wd,
                             float c1, float c2)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float mh = mi / c1, vh = vi / c2;
    float wi = w[i];
    wi -= lr * (mh / (sqrtf(vh) + eps) + wd * wi);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float *x, __nv_bfloat16 *y, long long n)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// rows idx[r] of X [*, kin] (FP32) -> BF16 [r][kpad] (zero padded) and T rows.
__global__ void gather_kernel(const float *X, const float *T, const int *idx, int rows, int kin,
                              int kpad, int nout, __nv_bfloat16 *Xb, float *Tb)
{
    int r = blockIdx.x;
    if (r >= rows) return;
    const long long src = idx ? idx[r] : r;
    for (int k = threadIdx.x; k < kpad; k += blockDim.x)
        Xb[(long long)r * kpad + k] = __float2bfloat16(k < kin ? X[src * kin + k] : 0.f);
    if (T)
        for (int k = threadIdx.x; k < nout; k += blockDim.x)
            Tb[(long long)r * nout + k] = T[src * nout + k];
}

}  // namespace

// ---------------------------------------------------------------------------
// eacc += sum of the nb per-block partial losses (fixed order).
__global__ void loss_accumulate_kernel(const float *partial, int nb, double *eacc)
{
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < nb; ++i) s += partial[i];
        *eacc += s;
    }
}

struct cosenu_mlp {
    int nin = 0, kpad = 0, nh = 0, nl = 0, nout = 0, device = 0;
    std::vector<int> din, dout;      // per layer
    std::vector<size_t> woff, boff;  // offsets into the flat parameter vector
    size_t nparam = 0;
    float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;  // FP32 flat
    __nv_bfloat16 *wb = nullptr;                                      // BF16 copy (flat)
    // activations for up to `cap` rows
    int cap = 0;
    __nv_bfloat16 *xb = nullptr;
    std::vector<float *> Z;           // pre-activations [cap][dout]
    std::vector<__nv_bfloat16 *> Hb;  // activations [cap][dout]
    float *dA = nullptr, *dB = nullptr;
    __nv_bfloat16 *dAb = nullptr;
    float *T = nullptr, *partial = nullptr;  // partial: 1024 floats, then eacc
    double *eacc = nullptr;                   // epoch loss sum, on the device
    // resident training data
    float *dX = nullptr, *dT = nullptr;
    int *didx = nullptr;
    int ndata = 0;
    long long t_step = 0;
    cudaStream_t stream = nullptr;
    bool tc = true;        // GEMMs on tcgen05 (COSENU_MLP_GEMM=mma: the mma.sync kernel)
    int *derr = nullptr;   // error word of the tcgen05 GEMM's bounded waits
    // host inputs of forward / loss_grad staged here (grown on demand)
    float *dxin = nullptr, *dtin = nullptr;
    size_t xin_cap = 0, tin_cap = 0;
    // timing mode: CUDA events around every launch, by kernel class
    bool timing = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev;  // (class, (start, stop))
    std::vector<cudaEvent_t> ev_pool;
    double ms[3] = {0, 0, 0};  // GEMM, elementwise, AdamW
    std::string err;
};

namespace {

enum { K_GEMM = 0, K_ELEM = 1, K_ADAMW = 2 };

cudaEvent_t pool_event(cosenu_mlp *net)
{
    if (!net->ev_pool.empty()) {
        cudaEvent_t e = net->ev_pool.back();
        net->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when timing is on: tstart before the
// launch, tstop after it.
struct Timed {
    cosenu_mlp *net;
    int cls;
    cudaEvent_t a = nullptr;
    Timed(cosenu_mlp *n, int c) : net(n), cls(c)
    {
        if (net->timing) {
            a = pool_event(net);
            cudaEventRecord(a, net->stream);
        }
    }
    ~Timed()
    {
        if (net->timing) {
            cudaEvent_t b = pool_event(net);
            cudaEventRecord(b, net->stream);
            net->ev.push_back({cls, {a, b}});
        }
    }
};

// After a synchronisation: adds the recorded intervals to the class totals.
void collect_times(cosenu_mlp *net)
{
    for (auto &e : net->ev) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, e.second.first, e.second.second) == cudaSuccess)
            net->ms[e.first] += t;
        net->ev_pool.push_back(e.second.first);
        net->ev_pool.push_back(e.second.second);
    }
    net->ev.clear();
}

int mfail(cosenu_mlp *n, int code, const std::string &msg)
{
    if (n) n->err = msg;
    return code;
}

#define MCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return mfail(net, COSENU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// After a synchronisation of the stream: a pending launch error, or an
// expired wait recorded by the tcgen05 GEMM (the word is cleared).
int check_device(cosenu_mlp *net)
{
    MCK(cudaGetLastError());
    int h = 0;
    MCK(cudaMemcpy(&h, net->derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        MCK(cudaMemset(net->derr, 0, sizeof(int)));
        return mfail(net, COSENU_ERR_CUDA, "tensor-core GEMM: a pipeline wait timed out");
    }
    return COSENU_OK;
}

// Host rows (and targets) copied into the staging buffers, grown on demand.
int stage_inputs(cosenu_mlp *net, const float *x_host, const float *t_host, int rows)
{
    const size_t nx = (size_t)rows * net->nin, nt = (size_t)rows * net->nout;
    if (nx > net->xin_cap) {
        cudaStreamSynchronize(net->stream);
        if (net->dxin) cudaFree(net->dxin);
        net->dxin = nullptr;
        MCK(cudaMalloc(&net->dxin, nx * 4));
        net->xin_cap = nx;
    }
    if (t_host && nt > net->tin_cap) {
        cudaStreamSynchronize(net->stream);
        if (net->dtin) cudaFree(net->dtin);
        net->dtin = nullptr;
        MCK(cudaMalloc(&net->dtin, nt * 4));
        net->tin_cap = nt;
    }
    MCK(cudaMemcpyAsync(net->dxin, x_host, nx * 4, cudaMemcpyHostToDevice, net->stream));
    if (t_host)
        MCK(cudaMemcpyAsync(net->dtin, t_host, nt * 4, cudaMemcpyHostToDevice, net->stream));
    return COSENU_OK;
}

int ensure_cap(cosenu_mlp *net, int rows)
{
    if (rows <= net->cap) return COSENU_OK;
    cudaStreamSynchronize(net->stream);
    auto fr = [](void *p) { if (p) cudaFree(p); };
    fr(net->xb);
    for (auto p : net->Z) fr(p);
    for (auto p : net->Hb) fr(p);
    fr(net->dA); fr(net->dB); fr(net->dAb); fr(net->T);
    int wmax = std::max(net->kpad, std::max(net->nh, net->nout));
    MCK(cudaMalloc(&net->xb, (size_t)rows * net->kpad * 2));
    for (int l = 0; l < net->nl; ++l) {
        MCK(cudaMalloc(&net->Z[l], (size_t)rows * net->dout[l] * 4));
        MCK(cudaMalloc(&net->Hb[l], (size_t)rows * net->dout[l] * 2));
    }
    MCK(cudaMalloc(&net->dA, (size_t)rows * wmax * 4));
    MCK(cudaMalloc(&net->dB, (size_t)rows * wmax * 4));
    MCK(cudaMalloc(&net->dAb, (size_t)rows * wmax * 2));
    MCK(cudaMalloc(&net->T, (size_t)rows * net->nout * 4));
    net->cap = rows;
    return COSENU_OK;
}

// forward over `rows` rows already in net->xb; output pre-activation of the
// last layer in Z[nl-1]
void forward(cosenu_mlp *net, int rows)
{
    const __nv_bfloat16 *x = net->xb;
    int kin = net->kpad;
    for (int l = 0; l < net->nl; ++l) {
        const bool last = l == net->nl - 1;
        Timed tm(net, K_GEMM);
        gemm(x, kin, 1, net->wb + net->woff[l], 1, kin, rows, net->dout[l], kin, net->Z[l],
             net->dout[l], net->w + net->boff[l], last ? nullptr : net->Hb[l], net->dout[l],
             last ? 0 : 1, net->tc, net->derr, net->stream);
        x = net->Hb[l];
        kin = net->dout[l];
    }
}

// loss gradient of the rows in xb / T; fills net->g; returns partial losses
void backward(cosenu_mlp *net, int rows, int nblk_loss)
{
    const int L = net->nl;
    const int nout = net->nout;
    {
        Timed tm(net, K_ELEM);
        mse_kernel<<<nblk_loss, 256, 0, net->stream>>>(net->Z[L - 1], net->T, rows * nout,
                                                       1.f / ((float)rows * nout), net->dA,
                                                       net->dAb, net->partial);
    }
    // dA (FP32) / dAb (BF16) hold dZ of layer l
    for (int l = L - 1; l >= 0; --l) {
        const int din = net->din[l], dout = net->dout[l];
        const __nv_bfloat16 *xin = l == 0 ? net->xb : net->Hb[l - 1];
        // dW[n][k] = sum_m dZ[m][n] X[m][k]
        {
            Timed tm(net, K_GEMM);
            gemm(net->dAb, 1, dout, xin, din, 1, dout, din, rows, net->g + net->woff[l], din,
                 nullptr, nullptr, 0, 0, net->tc, net->derr, net->stream);
        }
        {
            Timed tm(net, K_ELEM);
            colsum_kernel<<<(dout + 127) / 128, 128, 0, net->stream>>>(net->dA, rows, dout,
                                                                       net->g + net->boff[l]);
        }
        if (l > 0) {
            // dH[m][k] = sum_n dZ[m][n] W[n][k]; then dZ_{l-1} = dH * gelu'(Z_{l-1})
            {
                Timed tm(net, K_GEMM);
                gemm(net->dAb, dout, 1, net->wb + net->woff[l], din, 1, rows, din, dout, net->dB,
                     din, nullptr, nullptr, 0, 0, net->tc, net->derr, net->stream);
            }
            int n = rows * din;
            Timed tm(net, K_ELEM);
            gelu_back_kernel<<<(n + 255) / 256, 256, 0, net->stream>>>(net->dB, net->Z[l - 1], n,
                                                                       net->dA, net->dAb);
        }
    }
}

}  // namespace

extern "C" {

int cosenu_mlp_create(int n_in, int n_hidden, int n_hidden_layers, int n_out, uint64_t seed,
                      int device, cosenu_mlp **out)
{
    if (!out || n_in < 1 || n_hidden < 16 || n_hidden_layers < 1 || n_out < 1 ||
        n_hidden % 16 || n_out % 8)
        return COSENU_ERR_ARG;
    *out = nullptr;
    cosenu_mlp *net = new cosenu_mlp();
    net->nin = n_in;
    net->kpad = (n_in + 15) / 16 * 16;
    net->nh = n_hidden;
    net->nl = n_hidden_layers + 1;
    net->nout = n_out;
    net->device = device;
    cudaSetDevice(device);
    for (int l = 0; l < net->nl; ++l) {
        net->din.push_back(l == 0 ? net->kpad : n_hidden);
        net->dout.push_back(l == net->nl - 1 ? n_out : n_hidden);
    }
    for (int l = 0; l < net->nl; ++l) {
        net->woff.push_back(net->nparam);
        net->nparam += (size_t)net->din[l] * net->dout[l];
        net->boff.push_back(net->nparam);
        net->nparam += net->dout[l];
    }
    net->Z.assign(net->nl, nullptr);
    net->Hb.assign(net->nl, nullptr);
    // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a 64-bit LCG
    // (Knuth's MMIX constants); padded input columns are zero; biases zero
    std::vector<float> h(net->nparam, 0.f);
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    for (int l = 0; l < net->nl; ++l) {
        const int fan = l == 0 ? n_in : net->din[l];
        const float a = 1.f / std::sqrt((float)fan);
        for (int o = 0; o < net->dout[l]; ++o)
            for (int k = 0; k < net->din[l]; ++k) {
                st = st * 6364136223846793005ull + 1442695040888963407ull;
                float u = (float)((st >> 11) * (1.0 / 9007199254740992.0));
                h[net->woff[l] + (size_t)o * net->din[l] + k] =
                    (l == 0 && k >= n_in) ? 0.f : a * (2.f * u - 1.f);
            }
    }
    if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&net->w, net->nparam * 4) != cudaSuccess ||
        cudaMalloc(&net->g, net->nparam * 4) != cudaSuccess ||
        cudaMalloc(&net->m1, net->nparam * 4) != cudaSuccess ||
        cudaMalloc(&net->m2, net->nparam * 4) != cudaSuccess ||
        cudaMalloc(&net->wb, net->nparam * 2) != cudaSuccess ||
        cudaMalloc(&net->partial, 1024 * 4 + 8) != cudaSuccess ||
        cudaMalloc(&net->derr, sizeof(int)) != cudaSuccess ||
        cudaMemset(net->derr, 0, sizeof(int)) != cudaSuccess) {
        cosenu_mlp_destroy(net);
        return COSENU_ERR_NOMEM;
    }
    net->eacc = reinterpret_cast<double *>(net->partial + 1024);
    const char *gk = std::getenv("COSENU_MLP_GEMM");
    net->tc = !(gk && std::strcmp(gk, "mma") == 0);
    *out = net;
    return cosenu_mlp_set_params(net, h.data());
}

int cosenu_mlp_destroy(cosenu_mlp *net)
{
    if (!net) return COSENU_OK;
    if (net->stream) cudaStreamSynchronize(net->stream);
    void *bufs[] = {net->w, net->g, net->m1, net->m2, net->wb, net->partial, net->xb, net->dA,
                    net->dB, net->dAb, net->T, net->dX, net->dT, net->didx, net->dxin, net->dtin,
                    net->derr};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (auto p : net->Z)
        if (p) cudaFree(p);
    for (auto p : net->Hb)
        if (p) cudaFree(p);
    collect_times(net);
    for (cudaEvent_t e : net->ev_pool) cudaEventDestroy(e);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return COSENU_OK;
}

const char *cosenu_mlp_last_error(const cosenu_mlp *net) { return net ? net->err.c_str() : ""; }

int cosenu_mlp_num_params(const cosenu_mlp *net, size_t *n)
{
    if (!net || !n) return COSENU_ERR_ARG;
    *n = net->nparam;
    return COSENU_OK;
}

int cosenu_mlp_get_params(cosenu_mlp *net, float *host)
{
    if (!net || !host) return COSENU_ERR_ARG;
    MCK(cudaMemcpyAsync(host, net->w, net->nparam * 4, cudaMemcpyDeviceToHost, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    return COSENU_OK;
}

// Sets the FP32 master parameters (and their BF16 copy); resets AdamW state.
int cosenu_mlp_set_params(cosenu_mlp *net, const float *host)
{
    if (!net || !host) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    MCK(cudaMemcpyAsync(net->w, host, net->nparam * 4, cudaMemcpyHostToDevice, net->stream));
    to_bf16_kernel<<<(unsigned)((net->nparam + 255) / 256), 256, 0, net->stream>>>(net->w, net->wb,
                                                                                  (long long)net->nparam);
    MCK(cudaMemsetAsync(net->m1, 0, net->nparam * 4, net->stream));
    MCK(cudaMemsetAsync(net->m2, 0, net->nparam * 4, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    net->t_step = 0;
    return COSENU_OK;
}

int cosenu_mlp_forward(cosenu_mlp *net, const float *x_host, int rows, float *y_host)
{
    if (!net || !x_host || !y_host || rows < 1) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    int rc = ensure_cap(net, rows);
    if (rc) return rc;
    if ((rc = stage_inputs(net, x_host, nullptr, rows)) != COSENU_OK) return rc;
    {
        Timed tm(net, K_ELEM);
        gather_kernel<<<rows, 128, 0, net->stream>>>(net->dxin, nullptr, nullptr, rows, net->nin,
                                                     net->kpad, net->nout, net->xb, nullptr);
    }
    forward(net, rows);
    MCK(cudaMemcpyAsync(y_host, net->Z[net->nl - 1], (size_t)rows * net->nout * 4,
                        cudaMemcpyDeviceToHost, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    collect_times(net);
    return check_device(net);
}

// Mean-squared-error loss and its gradient with respect to the FP32 master
// parameters (flat, per layer W then b), for the rows given.
int cosenu_mlp_loss_grad(cosenu_mlp *net, const float *x_host, const float *t_host, int rows,
                         float *loss, float *grad_host)
{
    if (!net || !x_host || !t_host || rows < 1) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    int rc = ensure_cap(net, rows);
    if (rc) return rc;
    if ((rc = stage_inputs(net, x_host, t_host, rows)) != COSENU_OK) return rc;
    gather_kernel<<<rows, 128, 0, net->stream>>>(net->dxin, net->dtin, nullptr, rows, net->nin,
                                                 net->kpad, net->nout, net->xb, net->T);
    forward(net, rows);
    const int nb = 64;
    backward(net, rows, nb);
    std::vector<float> part(nb);
    MCK(cudaMemcpyAsync(part.data(), net->partial, nb * 4, cudaMemcpyDeviceToHost, net->stream));
    if (grad_host)
        MCK(cudaMemcpyAsync(grad_host, net->g, net->nparam * 4, cudaMemcpyDeviceToHost, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    collect_times(net);
    if ((rc = check_device(net)) != COSENU_OK) return rc;
    double s = 0;
    for (float p : part) s += p;
    if (loss) *loss = (float)(s / ((double)rows * net->nout));
    return COSENU_OK;
}

// Training data kept in device memory for cosenu_mlp_train.
int cosenu_mlp_set_data(cosenu_mlp *net, const float *x_host, const float *t_host, int n)
{
    if (!net || !x_host || !t_host || n < 1) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    if (net->dX) cudaFree(net->dX);
    if (net->dT) cudaFree(net->dT);
    if (net->didx) cudaFree(net->didx);
    net->dX = net->dT = nullptr;
    net->didx = nullptr;
    MCK(cudaMalloc(&net->dX, (size_t)n * net->nin * 4));
    MCK(cudaMalloc(&net->dT, (size_t)n * net->nout * 4));
    MCK(cudaMalloc(&net->didx, (size_t)n * 4));
    MCK(cudaMemcpyAsync(net->dX, x_host, (size_t)n * net->nin * 4, cudaMemcpyHostToDevice, net->stream));
    MCK(cudaMemcpyAsync(net->dT, t_host, (size_t)n * net->nout * 4, cudaMemcpyHostToDevice, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    net->ndata = n;
    return COSENU_OK;
}

// Minibatch AdamW over the resident data for `epochs` epochs (shuffled with
// a 64-bit LCG seeded by shuffle_seed); epoch_loss[e] = mean training loss.
int cosenu_mlp_train(cosenu_mlp *net, int epochs, int batch, float lr, float weight_decay,
                     float beta1, float beta2, float eps, uint64_t shuffle_seed, float *epoch_loss)
{
    if (!net || epochs < 1 || batch < 1 || net->ndata < 1) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    int rc = ensure_cap(net, batch);
    if (rc) return rc;
    std::vector<int> perm(net->ndata);
    uint64_t st = shuffle_seed * 6364136223846793005ull + 1442695040888963407ull;
    const int nb = 32;
    double esum = 0;
    for (int e = 0; e < epochs; ++e) {
        for (int i = 0; i < net->ndata; ++i) perm[i] = i;
        for (int i = net->ndata - 1; i > 0; --i) {  // Fisher-Yates
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            int j = (int)((st >> 33) % (uint64_t)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        MCK(cudaMemcpyAsync(net->didx, perm.data(), (size_t)net->ndata * 4, cudaMemcpyHostToDevice,
                            net->stream));
        MCK(cudaMemsetAsync(net->eacc, 0, sizeof(double), net->stream));
        long long ecount = 0;
        for (int b0 = 0; b0 < net->ndata; b0 += batch) {
            const int rows = std::min(batch, net->ndata - b0);
            {
                Timed tm(net, K_ELEM);
                gather_kernel<<<rows, 128, 0, net->stream>>>(net->dX, net->dT, net->didx + b0,
                                                             rows, net->nin, net->kpad, net->nout,
                                                             net->xb, net->T);
            }
            forward(net, rows);
            backward(net, rows, nb);
            net->t_step++;
            const float c1 = 1.f - std::pow(beta1, (float)net->t_step);
            const float c2 = 1.f - std::pow(beta2, (float)net->t_step);
            Timed *tm = new Timed(net, K_ADAMW);
            for (int l = 0; l < net->nl; ++l) {
                const long long nw = (long long)net->din[l] * net->dout[l];
                adamw_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, net->stream>>>(
                    net->w + net->woff[l], net->g + net->woff[l], net->m1 + net->woff[l],
                    net->m2 + net->woff[l], net->wb + net->woff[l], nw, lr, beta1, beta2, eps,
                    weight_decay, c1, c2);
                adamw_kernel<<<(net->dout[l] + 255) / 256, 256, 0, net->stream>>>(
                    net->w + net->boff[l], net->g + net->boff[l], net->m1 + net->boff[l],
                    net->m2 + net->boff[l], net->wb + net->boff[l], net->dout[l], lr, beta1, beta2,
                    eps, 0.f, c1, c2);
            }
            delete tm;  // the AdamW updates of all layers
            loss_accumulate_kernel<<<1, 32, 0, net->stream>>>(net->partial, nb, net->eacc);
            ecount += (long long)rows * net->nout;
        }
        // one host synchronisation per epoch (the shuffle buffer is reused)
        MCK(cudaMemcpyAsync(&esum, net->eacc, sizeof(double), cudaMemcpyDeviceToHost, net->stream));
        MCK(cudaStreamSynchronize(net->stream));
        collect_times(net);
        if ((rc = check_device(net)) != COSENU_OK) return rc;
        if (epoch_loss) epoch_loss[e] = (float)(esum / ecount);
    }
    return COSENU_OK;
}

int cosenu_mlp_set_timing(cosenu_mlp *net, int on)
{
    if (!net) return COSENU_ERR_ARG;
    cudaSetDevice(net->device);
    MCK(cudaStreamSynchronize(net->stream));
    collect_times(net);
    net->timing = on != 0;
    net->ms[0] = net->ms[1] = net->ms[2] = 0.0;
    return COSENU_OK;
}

int cosenu_mlp_timing(const cosenu_mlp *net, double ms[3])
{
    if (!net || !ms) return COSENU_ERR_ARG;
    for (int k = 0; k < 3; ++k) ms[k] = net->ms[k];
    return COSENU_OK;
}

}  // extern "C"
