// Ensembles: many independent simulations of uneven nz / nvz / physics
// advanced together.  Each member is an ordinary context (its own buffers,
// initial condition, analysis); stepping is shared: one launch per RK4 stage
// covers every member that still has steps to do, through a table of
// (member, z tile, v tile) entries and per-member stage arguments held in
// device memory.  Two kernel families serve the launch: the TMA-pipelined
// kernel (persistent blocks over 32-cell z tiles spanning all rows) and the
// register-tiled kernel (one block per z tile x v tile, tile width shared,
// v tile per member).  cosenu_batch_autotune times the candidates on the
// ensemble itself and keeps the fastest.
//
// Step counts are known up front, so a run is a sequence of phases: each
// phase advances the members that are still active by the smallest remaining
// count, with the per-step launches captured once into a CUDA graph and
// replayed; finished members drop out of the table between phases.
//
// FP32-bulk members write each step's new state into their other FP64 buffer
// (common.cuh), so stage arguments and tensor maps exist per buffer parity.
// A run starts every member from parity 0; active members then advance
// together and keep a common parity, so each launch picks one set.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "ctx.h"

using namespace cosenu;

extern thread_local std::string g_create_error;

struct cosenu_batch {
    int n = 0;
    int device = 0;
    int scheme = 0, fp32 = 0;
    std::vector<cosenu_ctx *> m;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    int nsm = 148;
    // device arrays: per-parity, per-member stage args [2][n][4] and tensor
    // maps [2][n][NMAP_B]; two tile tables
    StageArgs *d_args = nullptr;
    CUtensorMap *d_maps = nullptr;
    int4 *d_table[2] = {nullptr, nullptr};
    int4 *h_table[2] = {nullptr, nullptr};  // pinned staging (table, then block ranges)
    cudaEvent_t table_ev[2] = {nullptr, nullptr};
    size_t table_cap = 0;
    int phase = 0;
    int *err_flag = nullptr;
    // kernel choice
    int use_tma = 1;   // 1: TMA family; 0: register-tiled family
    int tz = 32;       // register-tiled z tile
    std::vector<int> tv;  // register-tiled v tile per member
    int max_nvz = 0;
    std::vector<cudaGraphExec_t> graphs;  // executed graphs, released after a synchronize
    std::string err;
};

namespace {

constexpr int NMAP_B = 8;  // tensor maps per member (the TMA kernel's NMAP)

int bfail(cosenu_batch *b, int code, const std::string &msg)
{
    if (b) b->err = msg;
    return code;
}

#define BCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return bfail(b, COSENU_ERR_CUDA, std::string(#call) + ": " +  \
                                                                    cudaGetErrorString(e_));   \
    } while (0)

// Per-member stage arguments for the current kernel choice, to the device
// (both buffer parities).
int upload_args(cosenu_batch *b)
{
    std::vector<StageArgs> args(8 * (size_t)b->n);
    for (int par = 0; par < 2; ++par)
        for (int i = 0; i < b->n; ++i)
            for (int s = 1; s <= 4; ++s)
                args[4 * ((size_t)par * b->n + i) + s - 1] =
                    ctx_stage_args(b->m[i], s, b->fp32 ? par : 0);
    BCK(cudaMemcpyAsync(b->d_args, args.data(), args.size() * sizeof(StageArgs),
                        cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return COSENU_OK;
}

// Table of tiles of the members in `active`.  TMA family: member by member
// (a block then streams consecutive z tiles of one member), with `ranges`
// splitting the table into nblk contiguous pieces of equal work; register-
// tiled family: heaviest tiles first (one block per entry).
size_t build_table(cosenu_batch *b, const std::vector<int> &active, std::vector<int4> &out,
                   std::vector<int> *ranges = nullptr, int nblk = 0)
{
    out.clear();
    if (b->use_tma) {
        std::vector<long long> w;
        for (int i : active) {
            const cosenu_params &p = b->m[i]->p;
            for (int zt = 0; zt < p.nz / 32; ++zt) {
                out.push_back(make_int4(i, zt, 0, p.nvz));  // .w: rows, read by the kernel
                w.push_back((long long)(p.nvz + 7) / 8 + 1);  // chunks + per-tile overhead
            }
        }
        if (ranges) {
            long long total = 0;
            for (long long x : w) total += x;
            ranges->assign(nblk + 1, (int)out.size());
            (*ranges)[0] = 0;
            long long acc = 0;
            int blk = 1;
            for (size_t t = 0; t < out.size() && blk < nblk; ++t) {
                acc += w[t];
                while (blk < nblk && acc * nblk >= total * blk) (*ranges)[blk++] = (int)t + 1;
            }
        }
        return out.size();
    }
    std::vector<std::pair<long long, int4>> t;
    for (int i : active) {
        const cosenu_params &p = b->m[i]->p;
        if (b->use_tma) {
            for (int zt = 0; zt < p.nz / 32; ++zt)
                t.push_back({(long long)p.nvz * 32, make_int4(i, zt, 0, 0)});
        } else {
            const int tv = b->tv[i], nvt = (p.nvz + tv - 1) / tv;
            for (int vt = 0; vt < nvt; ++vt)
                for (int zt = 0; zt < p.nz / b->tz; ++zt)
                    t.push_back({(long long)std::min(tv, p.nvz - vt * tv) * b->tz,
                                 make_int4(i, zt, vt, 0)});
        }
    }
    std::stable_sort(t.begin(), t.end(),
                     [](const std::pair<long long, int4> &x, const std::pair<long long, int4> &y) {
                         return x.first > y.first;
                     });
    for (auto &e : t) out.push_back(e.second);
    return out.size();
}

int ensure_table_cap(cosenu_batch *b, size_t n)
{
    if (n <= b->table_cap) return COSENU_OK;
    for (int k = 0; k < 2; ++k) {
        if (b->table_ev[k]) cudaEventSynchronize(b->table_ev[k]);
        if (b->d_table[k]) cudaFree(b->d_table[k]);
        if (b->h_table[k]) cudaFreeHost(b->h_table[k]);
        BCK(cudaMalloc(&b->d_table[k], n * sizeof(int4)));
        BCK(cudaMallocHost(&b->h_table[k], n * sizeof(int4)));
    }
    b->table_cap = n;
    return COSENU_OK;
}

// Queues `nsteps` RK4 steps of the members in `active`.
int run_phase(cosenu_batch *b, const std::vector<int> &active, long long nsteps)
{
    std::vector<int4> tab;
    std::vector<int> ranges;
    size_t ntiles_all = 0;
    for (int i : active) ntiles_all += b->m[i]->p.nz / 32;
    const int per_sm = b->use_tma ? tma_blocks_per_sm(b->scheme) : 1;
    const int nblk = (int)std::min<size_t>(std::max<size_t>(ntiles_all, 1), (size_t)(per_sm * b->nsm));
    size_t nt = build_table(b, active, tab, &ranges, nblk);
    if (nt == 0 || nsteps <= 0) return COSENU_OK;
    // table entries, then (TMA family) the nblk + 1 block range starts
    const size_t nrange_int4 = b->use_tma ? (ranges.size() + 3) / 4 : 0;
    int rc = ensure_table_cap(b, nt + nrange_int4);
    if (rc) return rc;
    const int k = b->phase++ & 1;
    BCK(cudaEventSynchronize(b->table_ev[k]));  // staging buffer free again
    std::memcpy(b->h_table[k], tab.data(), nt * sizeof(int4));
    if (nrange_int4) std::memcpy(b->h_table[k] + nt, ranges.data(), ranges.size() * sizeof(int));
    BCK(cudaMemcpyAsync(b->d_table[k], b->h_table[k], (nt + nrange_int4) * sizeof(int4),
                        cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->table_ev[k], b->stream));
    BatchDev bd0{b->d_table[k], (int)nt, b->d_args, b->d_maps,
                 reinterpret_cast<const int *>(b->d_table[k] + nt)};
    if (getenv("COSENU_BATCH_RR")) bd0.range = nullptr;
    int max_nvz = 0;
    for (int i : active) max_nvz = std::max(max_nvz, b->m[i]->p.nvz);
    const StageArgs a0 = ctx_stage_args(b->m[active[0]], 1);
    // the active members' common buffer parity (0 for FP64)
    int par = b->m[active[0]]->ypar;
    auto launch_step = [&](cudaStream_t s, int p) -> cudaError_t {
        BatchDev bd = bd0;
        bd.args += (size_t)p * 4 * b->n;
        bd.maps += (size_t)p * NMAP_B * b->n;
        for (int st = 1; st <= 4; ++st) {
            cudaError_t e;
            if (b->use_tma)
                e = launch_rk4_stage_tma_batch(bd, a0, b->scheme, st, b->fp32, b->err_flag, nblk,
                                               max_nvz, s);
            else
                e = launch_rk4_stage_batch(bd, b->scheme, st, b->tz, b->fp32, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    // one graph of up to 16 steps for this phase, replayed (FP32-bulk: an even
    // number of steps, so that every replay starts from the same parity)
    int chunk = (int)std::min<long long>(16, nsteps);
    if (b->fp32 && chunk > 1) chunk &= ~1;
    cudaGraphExec_t ge = nullptr;
    {
        cudaStream_t cs;
        BCK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = cudaSuccess;
            for (int i = 0; i < chunk && le == cudaSuccess; ++i) le = launch_step(cs, par ^ (i & 1));
            e = cudaStreamEndCapture(cs, &g);
            if (le != cudaSuccess) e = le;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return bfail(b, COSENU_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    }
    long long left = nsteps;
    cudaError_t e = cudaSuccess;
    while (left >= chunk && e == cudaSuccess) {
        e = cudaGraphLaunch(ge, b->stream);
        left -= chunk;
        if (chunk & 1) par ^= b->fp32;  // (an odd chunk is a single replay)
    }
    while (left-- > 0 && e == cudaSuccess) {
        e = launch_step(b->stream, par);
        par ^= b->fp32;
    }
    b->graphs.push_back(ge);  // released once the stream has drained
    if (e != cudaSuccess) return bfail(b, COSENU_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    for (int i : active) {
        b->m[i]->steps += nsteps;
        if (nsteps & 1) ctx_flip(b->m[i]);
    }
    return COSENU_OK;
}

int apply_tiling(cosenu_batch *b)
{
    for (int i = 0; i < b->n; ++i) {
        int rc = b->use_tma ? ctx_set_tiling(b->m[i], 0, 0) : ctx_set_tiling(b->m[i], b->tz, b->tv[i]);
        if (rc) return bfail(b, rc, cosenu_last_error(b->m[i]));
    }
    return upload_args(b);
}

}  // namespace

extern "C" {

int cosenu_batch_create(int n, const cosenu_params *params, cosenu_batch **out)
{
    g_create_error.clear();
    if (n < 1 || !params || !out) {
        g_create_error = "need n >= 1 parameter sets";
        return COSENU_ERR_ARG;
    }
    *out = nullptr;
    for (int i = 1; i < n; ++i)
        if (params[i].scheme != params[0].scheme || params[i].precision != params[0].precision ||
            params[i].device != params[0].device ||
            (params[i].scheme == COSENU_FD && (params[i].fd_advec != params[0].fd_advec ||
                                               params[i].ko_order != params[0].ko_order))) {
            g_create_error = "ensemble members must share scheme, FD variant, precision and device";
            return COSENU_ERR_ARG;
        }
    cosenu_batch *b = new cosenu_batch();
    b->n = n;
    b->device = params[0].device;
    b->scheme = params[0].scheme;
    b->fp32 = params[0].precision == COSENU_FP32_BULK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    auto bail = [&](int rc) {
        g_create_error = b->err.empty() ? g_create_error : b->err;
        cosenu_batch_destroy(b);
        if (prev >= 0) cudaSetDevice(prev);
        return rc;
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(COSENU_ERR_CUDA);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device);
    b->m.assign(n, nullptr);
    b->tv.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        int rc = ctx_create(&params[i], &b->m[i], 1);
        if (rc != COSENU_OK) {
            b->err = "member " + std::to_string(i) + ": " + cosenu_last_error(nullptr);
            return bail(rc);
        }
        cosenu_set_stream(b->m[i], b->stream);
        b->max_nvz = std::max(b->max_nvz, params[i].nvz);
        b->tv[i] = std::min(params[i].nvz, 64);
    }
    if (cudaMalloc(&b->d_args, 8 * (size_t)n * sizeof(StageArgs)) != cudaSuccess ||
        cudaMalloc(&b->d_maps, 2 * NMAP_B * (size_t)n * sizeof(CUtensorMap)) != cudaSuccess ||
        cudaMalloc(&b->err_flag, 64) != cudaSuccess)
        return bail(COSENU_ERR_NOMEM);
    // per parity and member, in the order of the TMA kernel's MapIdx.  FP64:
    // Y, U0, U1 input boxes (with halo), Y, A, U0 tiles.  FP32-bulk: the
    // current Y, D1, D2 input boxes, the D2 tile, -, the D1 tile, the D3 box,
    // the current Y in stage 4's rows.
    std::vector<CUtensorMap> maps(2 * NMAP_B * (size_t)n);
    for (int par = 0; par < 2; ++par)
        for (int i = 0; i < n; ++i) {
            const cosenu_ctx *c = b->m[i];
            CUtensorMap *mp = &maps[NMAP_B * ((size_t)par * n + i)];
            mp[0] = c->mYb40[b->fp32 ? par : 0];
            mp[1] = c->mU0_40;
            mp[2] = c->mU1_40;
            mp[3] = b->fp32 ? c->mU1_32 : c->mY32;
            mp[4] = c->mA32;
            mp[5] = c->mU0_32;
            mp[6] = c->mU2_40;
            mp[7] = c->mYb40s4[b->fp32 ? par : 0];
        }
    cudaMemcpyAsync(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                    cudaMemcpyHostToDevice, b->stream);
    cudaMemsetAsync(b->err_flag, 0, 64, b->stream);
    for (int k = 0; k < 2; ++k)
        if (cudaEventCreateWithFlags(&b->table_ev[k], cudaEventDisableTiming) != cudaSuccess)
            return bail(COSENU_ERR_CUDA);
    if (upload_args(b) != COSENU_OK) return bail(COSENU_ERR_CUDA);
    if (prev >= 0) cudaSetDevice(prev);
    *out = b;
    return COSENU_OK;
}

int cosenu_batch_destroy(cosenu_batch *b)
{
    if (!b) return COSENU_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (cudaGraphExec_t g : b->graphs) cudaGraphExecDestroy(g);
    for (cosenu_ctx *c : b->m)
        if (c) cosenu_destroy(c);
    for (int k = 0; k < 2; ++k) {
        if (b->d_table[k]) cudaFree(b->d_table[k]);
        if (b->h_table[k]) cudaFreeHost(b->h_table[k]);
        if (b->table_ev[k]) cudaEventDestroy(b->table_ev[k]);
    }
    if (b->d_args) cudaFree(b->d_args);
    if (b->d_maps) cudaFree(b->d_maps);
    if (b->err_flag) cudaFree(b->err_flag);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    else if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return COSENU_OK;
}

const char *cosenu_batch_last_error(const cosenu_batch *b) { return b ? b->err.c_str() : ""; }

cosenu_ctx *cosenu_batch_member(cosenu_batch *b, int i)
{
    return (b && i >= 0 && i < b->n) ? b->m[i] : nullptr;
}

int cosenu_batch_size(const cosenu_batch *b) { return b ? b->n : 0; }

int cosenu_batch_set_stream(cosenu_batch *b, void *stream)
{
    if (!b || !stream) return COSENU_ERR_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    if (b->own_stream == nullptr) b->own_stream = b->stream;
    b->stream = (cudaStream_t)stream;
    for (cosenu_ctx *c : b->m) cosenu_set_stream(c, stream);
    return COSENU_OK;
}

int cosenu_batch_init_seeded(cosenu_batch *b, const uint64_t *seeds, const double *sig_nu,
                             const double *sig_nubar, const double *alpha, double amp)
{
    if (!b || !seeds || !sig_nu || !sig_nubar || !alpha) return COSENU_ERR_ARG;
    for (int i = 0; i < b->n; ++i) {
        int rc = cosenu_init_seeded(b->m[i], seeds[i], (uint32_t)i, sig_nu[i], sig_nubar[i],
                                    alpha[i], amp);
        if (rc) return bfail(b, rc, "member " + std::to_string(i) + ": " + cosenu_last_error(b->m[i]));
    }
    return COSENU_OK;
}

int cosenu_batch_run(cosenu_batch *b, const long long *nsteps)
{
    if (!b || !nsteps) return COSENU_ERR_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    std::vector<long long> left(nsteps, nsteps + b->n);
    int rc = COSENU_OK;
    for (int i = 0; i < b->n; ++i)
        if (left[i] < 0 || (left[i] > 0 && !b->m[i]->have_state)) {
            rc = bfail(b, COSENU_ERR_ARG, "member " + std::to_string(i) + ": negative steps or no state");
            break;
        }
    // every member starts from buffer parity 0 (FP32-bulk)
    for (int i = 0; i < b->n && rc == COSENU_OK; ++i)
        if (ctx_normalise_parity(b->m[i]) != COSENU_OK)
            rc = bfail(b, COSENU_ERR_CUDA, cosenu_last_error(b->m[i]));
    while (rc == COSENU_OK) {
        std::vector<int> active;
        long long d = 0;
        for (int i = 0; i < b->n; ++i)
            if (left[i] > 0) {
                active.push_back(i);
                d = d == 0 ? left[i] : std::min(d, left[i]);
            }
        if (active.empty()) break;
        rc = run_phase(b, active, d);
        for (int i : active) left[i] -= d;
    }
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

int cosenu_batch_synchronize(cosenu_batch *b)
{
    if (!b) return COSENU_ERR_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    for (cudaGraphExec_t g : b->graphs) cudaGraphExecDestroy(g);
    b->graphs.clear();
    int h = 0;
    BCK(cudaMemcpy(&h, b->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) return bfail(b, COSENU_ERR_CUDA, "ensemble stage pipeline wait timed out");
    return COSENU_OK;
}

// Chooses the kernel family and tiles by timing `trial_steps` ensemble steps
// per candidate (the state is saved first and restored afterwards).
int cosenu_batch_autotune(cosenu_batch *b, int trial_steps, char *report, size_t report_len)
{
    if (!b || trial_steps < 1) return COSENU_ERR_ARG;
    for (int i = 0; i < b->n; ++i)
        if (!b->m[i]->have_state) return bfail(b, COSENU_ERR_STATE, "autotune needs a state");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    // save every member's state and step count
    std::vector<double *> saved(b->n, nullptr);
    std::vector<long long> saved_steps(b->n);
    for (int i = 0; i < b->n; ++i) saved_steps[i] = b->m[i]->steps;
    for (int i = 0; i < b->n; ++i) {
        size_t bytes = (size_t)b->m[i]->cs * 8 * NCOMP;
        BCK(cudaMalloc(&saved[i], bytes));
        BCK(cudaMemcpyAsync(saved[i], b->m[i]->Y, bytes, cudaMemcpyDeviceToDevice, b->stream));
    }
    std::vector<int> all(b->n);
    std::iota(all.begin(), all.end(), 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::ostringstream rep;
    auto trial = [&](void) -> float {
        if (apply_tiling(b) != COSENU_OK) return 1e30f;
        for (int i = 0; i < b->n; ++i)
            if (ctx_normalise_parity(b->m[i]) != COSENU_OK) return 1e30f;
        if (run_phase(b, all, 1) != COSENU_OK) return 1e30f;  // warm-up (graph capture)
        cudaEventRecord(e0, b->stream);
        if (run_phase(b, all, trial_steps) != COSENU_OK) return 1e30f;
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / trial_steps;
    };
    // register-tiled family: coordinate search, z tile width then v tile per nvz class
    std::map<int, std::vector<int>> classes;
    for (int i = 0; i < b->n; ++i) classes[b->m[i]->p.nvz].push_back(i);
    b->use_tma = 0;
    b->tz = 32;
    for (int i = 0; i < b->n; ++i) b->tv[i] = std::min(b->m[i]->p.nvz, 64);
    float best_ldg = trial();
    rep << "register-tiled tz=32 tv=min(nvz,64): " << best_ldg << " ms/step\n";
    for (auto &c : classes) {
        const int nvz = c.first;
        int best_tv = b->tv[c.second[0]];
        for (int tv : {8, 16, 32, 64, 128, 256}) {
            if (tv > nvz || tv == best_tv || (nvz + tv - 1) / tv > (nvz + 7) / 8) continue;
            for (int i : c.second) b->tv[i] = tv;
            float t = trial();
            rep << "  nvz=" << nvz << " tv=" << tv << ": " << t << " ms/step\n";
            if (t < best_ldg) {
                best_ldg = t;
                best_tv = tv;
            }
        }
        for (int i : c.second) b->tv[i] = best_tv;
    }
    int best_tz = 32;
    for (int tz : {16, 8}) {
        bool ok = true;
        for (int i = 0; i < b->n; ++i) ok = ok && b->m[i]->p.nz % tz == 0;
        if (!ok) continue;
        b->tz = tz;
        float t = trial();
        rep << "  tz=" << tz << ": " << t << " ms/step\n";
        if (t < best_ldg) {
            best_ldg = t;
            best_tz = tz;
        }
    }
    b->tz = best_tz;
    std::vector<int> best_tvs = b->tv;
    // TMA family
    b->use_tma = 1;
    float t_tma = trial();
    rep << "TMA-pipelined: " << t_tma << " ms/step\n";
    if (best_ldg < t_tma) {
        b->use_tma = 0;
        b->tv = best_tvs;
    }
    rep << "chosen: " << (b->use_tma ? "TMA-pipelined" : "register-tiled tz=" + std::to_string(b->tz))
        << "\n";
    int rc = apply_tiling(b);
    // restore the saved states
    for (int i = 0; i < b->n && rc == COSENU_OK; ++i) {
        size_t bytes = (size_t)b->m[i]->cs * 8 * NCOMP;
        cudaMemcpyAsync(b->m[i]->Y, saved[i], bytes, cudaMemcpyDeviceToDevice, b->stream);
        rc = ctx_prepare_state(b->m[i]);
        b->m[i]->steps = saved_steps[i];
    }
    cudaStreamSynchronize(b->stream);
    for (cudaGraphExec_t g : b->graphs) cudaGraphExecDestroy(g);
    b->graphs.clear();
    for (double *p : saved) cudaFree(p);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (report && report_len) {
        std::string r = rep.str();
        std::strncpy(report, r.c_str(), report_len - 1);
        report[report_len - 1] = 0;
    }
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

int cosenu_batch_config(const cosenu_batch *b, int *use_tma, int *tz, int *tv_per_member)
{
    if (!b) return COSENU_ERR_ARG;
    if (use_tma) *use_tma = b->use_tma;
    if (tz) *tz = b->tz;
    if (tv_per_member)
        for (int i = 0; i < b->n; ++i) tv_per_member[i] = b->use_tma ? b->m[i]->p.nvz : b->tv[i];
    return COSENU_OK;
}

int cosenu_batch_set_config(cosenu_batch *b, int use_tma, int tz, const int *tv_per_member)
{
    if (!b) return COSENU_ERR_ARG;
    if (!use_tma) {
        if (tz != 8 && tz != 16 && tz != 32) return bfail(b, COSENU_ERR_ARG, "tz must be 8, 16 or 32");
        if (!tv_per_member) return bfail(b, COSENU_ERR_ARG, "need a v tile per member");
        b->tz = tz;
        for (int i = 0; i < b->n; ++i) b->tv[i] = tv_per_member[i];
    }
    b->use_tma = use_tma ? 1 : 0;
    return apply_tiling(b);
}

}  // extern "C"
