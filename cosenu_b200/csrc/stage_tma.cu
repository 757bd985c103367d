// TMA-pipelined RK4 stage kernel for the FV (src/rhs_fv.hpp:115-236) and FD
// (src/rhs_fd.hpp:6-148) schemes.
//
// Same arithmetic and epilogue as rk4_stage_kernel (stage.cu); what changes
// is how the operands reach the SM.  Each block is persistent over z-tiles of
// 32 cells that span all nvz rows.  One producer warp streams chunks of 8 rows
// x (32 + 2*4) cells of all 8 components of the stage input, and the matching
// 8 x 32 cells of Y and A, into a ring of NBUF shared-memory buffers with
// cp.async.bulk.tensor (one 3-D tensor-map copy per operand and chunk, box
// {cells, rows, components}); eight consumer warps take one row each, read
// their stencil from shared memory and write the results with coalesced
// stores.  Full/empty mbarriers order the ring.  With up to NBUF-1 chunks in
// flight (~100 KB per SM) the kernel keeps HBM busy without depending on
// occupancy, which the register-heavy FP64 right-hand side limits.  FD runs
// one block per SM; FV, bound by FP64 issue rather than HBM, runs two (each
// with half the shared memory) so that twice the warps hide the latency of the
// WENO7 arithmetic.  FV launches have no producer warp: the last consumer
// warp to release a buffer issues its next copies, so a block is 8 warps and
// gets 128 registers per thread.  Per-row velocities and
// advection factors equal the host's tables (src/nuosc.hpp:88-92,
// rhs_fv.hpp:145, rhs_fd.hpp:57): FV reads them once per chunk through the
// read-only cache, FD recomputes them in registers.
//
// FV: a warp holds one row, so every lane reconstructs the upwind WENO7 face it
// owns from the shared-memory stencil and takes its neighbour's face by
// shuffle; the one face per row and component outside the tile is computed,
// for all rows of a chunk at once, by R*8/32 warps in turn and published in
// shared memory (Layout::NE).  FD: the common variant of manage.py (central
// FD4 + KO3) is a compile-time fast path; the upwind / lopsided / KO5 variants
// take the generic path.
//
// Every wait is bounded in time (globaltimer, limit StageArgs::wait_ns): on
// expiry the kernel records a code in *err and carries on along the same
// control path, so no barrier is left waiting and the host reports the error.
// After a failed wait a consumer warp does not release its buffer, so the
// producer's next wait on that buffer fails too and it stops issuing copies
// (without a producer warp the buffer's release count never completes and no
// warp refills it); before the block exits one thread waits (bounded again)
// for the copies in flight, so no block ends while a bulk copy still writes
// into its shared memory.
#include <cuda.h>

#include <type_traits>

#include "common.cuh"
#include "weno.cuh"

namespace cosenu {

namespace tma {

constexpr int TZ = 32;           // cells per tile (one warp lane each)
constexpr int HALO = 4;          // cells each side in the input box
// Width of an input box row: the tile plus HALO cells each side, rounded up so
// that the row is a multiple of 16 bytes (TMA) and the component rows of one
// v row start in distinct shared-memory banks: the edge faces of a row read
// the same cell of all 8 components at once (42 doubles = 84 words: banks
// 0, 20, 8, 28, ... for components 0..7; 44 floats = 44 words: 0, 12, 24, ...).
template <class T> constexpr int xw() { return sizeof(T) == 8 ? 42 : 44; }
// v rows per chunk = consumer warps.  FV runs two blocks per SM with 8.  FD runs one block per SM: the stages that move
// few bytes per cell (FP64 stage 1, FP32-bulk stages 1-3) are bound by latency
// and run 12 (13 warps, ~126 registers, no spills: 0.230 -> 0.205 ms for FP64
// stage 1 at nz 32768 x nvz 256); the HBM-bound stages keep 8, whose smaller
// chunks keep fewer bytes in flight (12 rows: FP64 stage 3 0.436 -> 0.490 ms).
template <int SCHEME, int STAGE, bool INC> constexpr int rows()
{
    return (SCHEME == FD && ((!INC && STAGE == 1) || (INC && STAGE <= 3))) ? 12 : 8;
}
// tensor maps per ensemble member (MapIdx lists them)
constexpr int NMAP = 8;
#define TMA_MAX_NVZ 1024

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; returns false (and records `code`) when `limit_ns` passes.
// Once any wait in the grid has expired (*err != 0) later waits give up
// at once, so a broken pipeline ends within one time limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code,
                                          unsigned long long limit_ns)
{
    if (mbar_try(bar, parity)) return true;
    volatile int *verr = err;
    if (*verr != 0) return false;
    const unsigned long long t0 = gtimer();
    for (uint32_t n = 1;; ++n) {
        if (mbar_try(bar, parity)) return true;
        if ((n & 63) == 0 && (*verr != 0 || gtimer() - t0 > limit_ns)) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
}

// Wait for the completion of copies already issued, whatever *err says
// (bounded by `limit_ns`, code 3 on expiry): the producer's last act.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity, int *err,
                                           unsigned long long limit_ns)
{
    if (mbar_try(bar, parity)) return;
    const unsigned long long t0 = gtimer();
    for (uint32_t n = 1;; ++n) {
        if (mbar_try(bar, parity)) return;
        if ((n & 63) == 0 && gtimer() - t0 > limit_ns) {
            atomicCAS(err, 0, 3);
            return;
        }
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Brings a tensor map held in global memory into the TMA unit's cache.
__device__ __forceinline__ void prefetch_map(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

template <int NCONS> __device__ __forceinline__ void consumer_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(NCONS) : "memory");
}

// One ring buffer holds, for R rows, boxes laid out [row][component][cell]
// (the tensor maps put components before rows): the input box X, then Y, then
// the own-cell tiles A (and B).
template <int SCHEME, class TIN, class TOUT, int STAGE> struct Layout {
    static constexpr bool INC = inc_form<TIN, TOUT>();
    static constexpr int R = rows<SCHEME, STAGE, INC>();
    static constexpr int NTHR = R * 32 + 32;  // consumer warps + producer warp
    // without a producer warp (see producer_warp)
    static constexpr int NTHR_NP = R * 32;
    // FP64 stage 3 streams the most bytes per chunk: its 40-cell rows keep a
    // two-buffer ring within half an SM's shared memory (two blocks per SM)
    static constexpr int XW = (!INC && STAGE == 3) ? TZ + 2 * HALO : xw<TIN>();
    static constexpr int XB = NCOMP * R * XW * (int)sizeof(TIN);
    // Y: FP64 stages 2-3 read it at their own cells; FP32-bulk stages 2-4 read
    // it with the halo (their input is Y + D)
    static constexpr int YW =
        INC ? (STAGE >= 2 ? xw<double>() : 0) : ((STAGE == 2 || STAGE == 3) ? TZ : 0);
    static constexpr int YB = NCOMP * R * YW * 8;
    // FP64 stage 3: U at its own cells (about to be overwritten by U''); stage
    // 4: A.  FP32-bulk stage 4: D1 then D2 at its own cells.
    static constexpr int AB = INC ? (STAGE == 4 ? 2 * NCOMP * R * TZ * 4 : 0)
                                  : (STAGE >= 3 ? NCOMP * R * TZ * 8 : 0);
    static constexpr int BUF = ((XB + YB + AB) + 127) / 128 * 128;
    // FV (two blocks per SM, 96-128 registers): each consumer warp accumulates
    // the output moments of its rows in shared memory rather than in 12
    // registers, where half an SM leaves room (all but FP64 stage 3); the
    // other kernels keep them in registers and pair warps at the tile's end
    static constexpr bool MSM = SCHEME == FV && (INC || STAGE != 3);
    static constexpr int NRED = MSM ? R : R / 2;  // moment slots in shared memory
    // FV: the face of each row and component at the tile's upwind edge lies
    // outside the warp's 32 lanes.  Each chunk, NE = R * NCOMP / 32 warps (in
    // turn) compute all of them at full lane occupancy and publish them in
    // shared memory (one slot array and one mbarrier per ring buffer), rather
    // than every warp spending a ninth WENO7 pass with 8 of 32 lanes active.
    static constexpr int NE = SCHEME == FV ? R * NCOMP / 32 : 0;
    static_assert(NE == 0 || (R * NCOMP % 32 == 0 && (R & (R - 1)) == 0),
                  "edge warps: whole warps, rows a power of two");
};

// FD launches stream through a producer warp.  FV launches (single
// simulations and ensembles) run without one: the last consumer warp to
// release a ring buffer issues that buffer's next copies itself.  Its block is
// then 8 warps, and two blocks per SM get 128 registers per thread instead of
// the 96 that two 9-warp blocks leave (FP64 stage 3 spilled at 96).
template <int SCHEME, bool BATCHED> __host__ __device__ constexpr bool producer_warp()
{
    return SCHEME == FD;
}

// Arrival counter of a ring buffer without a producer warp: acquire-release
// add, so the last warp's refill is ordered after every warp's reads.
__device__ __forceinline__ uint32_t ring_release_count(uint32_t *cnt)
{
    uint32_t old;
    asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
                 : "=r"(old)
                 : "r"(smem_u32(cnt))
                 : "memory");
    return old;
}

// Orders this thread's generic-proxy view of shared memory before the bulk
// copies it issues next.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// The copies of one ring buffer: the stage input box (X) and, where the
// stage reads them, Y and the own-cell tiles A (and B), all completing on
// `bar`.  Coordinates: (cell, component 0, first row of the chunk).
template <class L>
__device__ __forceinline__ void issue_chunk(unsigned char *buf, uint64_t *bar, const CUtensorMap *px,
                                            const CUtensorMap *py, const CUtensorMap *pa,
                                            const CUtensorMap *pb, int z0, int row0)
{
    mbar_expect_tx(bar, L::XB + L::YB + L::AB);
    tma_load_3d(buf, px, HP + z0 - HALO, 0, row0, bar);
    if (L::YB) tma_load_3d(buf + L::XB, py, HP + z0 - (L::INC ? HALO : 0), 0, row0, bar);
    if (L::AB && !L::INC) tma_load_3d(buf + L::XB + L::YB, pa, HP + z0, 0, row0, bar);
    if (L::AB && L::INC) {
        tma_load_3d(buf + L::XB + L::YB, pa, HP + z0, 0, row0, bar);
        tma_load_3d(buf + L::XB + L::YB + L::AB / 2, pb, HP + z0, 0, row0, bar);
    }
}

// Index of each operand's tensor map among a member's NMAP maps (ensembles).
// FP64:      0 Y (halo box), 1 U0 (halo), 2 U1 (halo), 3 Y (tile), 4 A (tile), 5 U0 (tile)
// FP32-bulk: 0 current Y (halo), 1 D1 (halo), 2 D2 (halo), 3 D2 (tile), 5 D1 (tile), 6 D3 (halo),
//            7 current Y (halo) in the row count of stage 4
template <bool INC, int STAGE> struct MapIdx {
    static constexpr int X = STAGE == 1 ? 0 : (STAGE == 3 ? 2 : (INC && STAGE == 4 ? 6 : 1));
    static constexpr int Y = INC ? (STAGE == 4 ? 7 : 0) : 3;
    static constexpr int A = INC ? 5 : (STAGE == 3 ? 5 : 4);
    static constexpr int B = 3;
};

}  // namespace tma

static_assert(sizeof(StageArgs) % 8 == 0, "StageArgs is copied to shared memory in 8-byte words");

template <bool BATCHED>
__device__ __forceinline__ void tma_tile(const BatchDev &bd, int t, int &inst, int &zt)
{
    if (BATCHED) {
        const int4 e = bd.table[t];
        inst = e.x;
        zt = e.y;
    } else {
        inst = 0;
        zt = t;
    }
}

// FD: velocity and advection factor of row i, recomputed with round-to-nearest
// operations so the bits equal the host tables (capi.cu, src/nuosc.hpp:88-92,
// rhs_fd.hpp:57).  The FD stages are bound by memory latency, and a table load
// per chunk slowed them (FP64 stages 1, 2, 4 at nz 32768 x nvz 256 by 8 %); the
// FP64-bound FV stages read the tables instead.
__device__ __forceinline__ void fd_row_values(double v0, double dv, double dz, int fd_advec, int i,
                                              double &v, double &f)
{
    v = __dadd_rn(v0, __dmul_rn(__dadd_rn((double)i, 0.5), dv));
    const double sv = (double)((0.0 < v) - (v < 0.0));
    const double d12 = __dmul_rn(12.0, dz);
    if (fd_advec == 0) f = __ddiv_rn(-v, d12);                      // centre
    else if (fd_advec == 1) f = __ddiv_rn(__dmul_rn(-sv, v), d12);  // upwind
    else f = __ddiv_rn(__dmul_rn(sv, v), d12);                       // lopsided
}

// TIN: type of the streamed stage input (FP64: the stage value U or Y;
// FP32-bulk: Y at stage 1, the increment D after).  TOUT: type of the output
// (FP64: U', U'' or Y; FP32-bulk: D1, D2, D3, then the new Y).  The
// right-hand side is evaluated in FP64 in both forms, except the FP32-bulk
// WENO7 weights and candidates (FP32 on FP64 stencil differences).
template <int SCHEME, bool GEN, int STAGE, class TIN, class TOUT, int NBUF, bool BATCHED, int MINB>
__global__ void __launch_bounds__(tma::producer_warp<SCHEME, BATCHED>()
                                      ? tma::Layout<SCHEME, TIN, TOUT, STAGE>::NTHR
                                      : tma::Layout<SCHEME, TIN, TOUT, STAGE>::NTHR_NP,
                                  MINB)
    rk4_stage_tma_kernel(const __grid_constant__ CUtensorMap mX,
                         const __grid_constant__ CUtensorMap mY,
                         const __grid_constant__ CUtensorMap mA,
                         const __grid_constant__ CUtensorMap mB,
                         const __grid_constant__ StageArgs a0, int *err, const BatchDev bd)
{
    using namespace tma;
    using L = Layout<SCHEME, TIN, TOUT, STAGE>;
    constexpr int R = L::R;
    auto consumer_sync = tma::consumer_sync<R * 32>;
    using MI = MapIdx<L::INC, STAGE>;
    constexpr bool INC = L::INC;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + NBUF * L::BUF);
    uint64_t *empty = full + NBUF;
    uint64_t *ebar = empty + NBUF;  // FV: edge faces of buffer b published
    double(*s_mom)[TZ] =
        reinterpret_cast<double(*)[TZ]>(ebar + (L::NE ? NBUF : 0));  // [6][TZ]
    double(*s_red)[NMOM][TZ] = reinterpret_cast<double(*)[NMOM][TZ]>(s_mom + NMOM);  // [NRED]
    StageArgs *s_args = reinterpret_cast<StageArgs *>(s_red + L::NRED);  // batched: current member
    // FV: [NBUF][R][NCOMP] edge faces
    double(*s_edge)[R][NCOMP] = reinterpret_cast<double(*)[R][NCOMP]>(s_args + 1);
    // without a producer warp: per ring buffer, the warps' release count and
    // the last chunk whose copies went into it
    constexpr bool PW = producer_warp<SCHEME, BATCHED>();
    uint32_t *s_cnt = reinterpret_cast<uint32_t *>(s_edge + (L::NE ? NBUF : 0));
    int *s_last = reinterpret_cast<int *>(s_cnt + NBUF);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nzt = BATCHED ? bd.ntiles : a0.nz / TZ;
    // without a producer warp: the block's chunks in order (its z tiles or
    // table entries, each in chunks of R rows); chunk ch of tile t is the
    // block's n-th chunk, and its copies go into buffer n % NBUF
    const bool rr0 = !BATCHED || bd.range == nullptr;
    const int te0 = rr0 ? nzt : bd.range[blockIdx.x + 1];
    const int ts0 = rr0 ? gridDim.x : 1;
    auto nch_of = [&](int t) { return ((BATCHED ? bd.table[t].w : a0.nvz) + R - 1) / R; };
    auto issue_at = [&](int t, int ch, uint32_t n) {
        if (a0.stall) return;
        const int b = n % NBUF;
        if constexpr (BATCHED) {
            const int4 e = bd.table[t];
            const CUtensorMap *m = &bd.maps[e.x * NMAP];
            issue_chunk<L>(smem + b * L::BUF, &full[b], &m[MI::X], &m[MI::Y], &m[MI::A],
                           &m[MI::B], e.y * TZ, ch * R);
        } else {
            issue_chunk<L>(smem + b * L::BUF, &full[b], &mX, &mY, &mA, &mB, t * TZ, ch * R);
        }
        s_last[b] = (int)n;
    };
    // (t, ch) moved k chunks on; false past the block's last tile
    auto advance = [&](int &t, int &ch, int k) -> bool {
        for (; k > 0; --k) {
            if (++ch == nch_of(t)) {
                ch = 0;
                t += ts0;
                if (t >= te0) return false;
            }
        }
        return true;
    };

    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) {
            tma::mbar_init(&full[b], 1);
            tma::mbar_init(&empty[b], R);
            if (L::NE) tma::mbar_init(&ebar[b], L::NE * 32);
            if constexpr (!PW) {
                s_cnt[b] = 0;
                s_last[b] = -1;
            }
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if constexpr (!PW) {
            int t = rr0 ? blockIdx.x : bd.range[blockIdx.x], ch = 0;
            if (t < te0)
                for (uint32_t n = 0; n < (uint32_t)NBUF; ++n) {
                    issue_at(t, ch, n);
                    if (!advance(t, ch, 1)) break;
                }
        }
    }
    __syncthreads();

    if (PW && warp == R) {
        // ------------------------------------------------------------ producer
        if (lane == 0 && !a0.stall) {
            uint32_t it = 0;
            bool issuing = true;  // false once a wait has failed: no further copies
            const bool rr = !BATCHED || bd.range == nullptr;  // interleaved tiles
            const int t_first = rr ? blockIdx.x : bd.range[blockIdx.x];
            const int t_end = rr ? nzt : bd.range[blockIdx.x + 1];
            const int t_step = rr ? gridDim.x : 1;
            // batched: table entries (member, z tile, -, nvz) are read one tile
            // ahead, and a new member's tensor maps (global memory) are
            // prefetched while the previous tile streams
            int4 cur = make_int4(0, 0, 0, 0);
            if (BATCHED && t_first < t_end) cur = bd.table[t_first];
            for (int t = t_first; t < t_end && issuing; t += t_step) {
                const bool has_next = t + t_step < t_end;
                int4 nxt = cur;
                if (BATCHED && has_next) nxt = bd.table[t + t_step];
                const int inst = BATCHED ? cur.x : 0, zt = BATCHED ? cur.y : t;
                const CUtensorMap *px = BATCHED ? &bd.maps[inst * NMAP + MI::X] : &mX;
                const CUtensorMap *py = BATCHED ? &bd.maps[inst * NMAP + MI::Y] : &mY;
                const CUtensorMap *pa = BATCHED ? &bd.maps[inst * NMAP + MI::A] : &mA;
                const CUtensorMap *pb = BATCHED ? &bd.maps[inst * NMAP + MI::B] : &mB;
                const int z0 = zt * TZ;
                const int nch = ((BATCHED ? cur.w : a0.nvz) + R - 1) / R;
                for (int ch = 0; ch < nch; ++ch, ++it) {
                    if (BATCHED && ch == 0 && has_next && nxt.x != inst) {
                        const CUtensorMap *m = &bd.maps[nxt.x * NMAP];
                        tma::prefetch_map(&m[MI::X]);
                        if (L::YB) tma::prefetch_map(&m[MI::Y]);
                        if (L::AB) tma::prefetch_map(&m[MI::A]);
                        if (INC && L::AB) tma::prefetch_map(&m[MI::B]);
                    }
                    const int b = it % NBUF;
                    if (it >= (uint32_t)NBUF &&
                        !tma::mbar_wait(&empty[b], ((it / NBUF) - 1) & 1, err, 1, a0.wait_ns)) {
                        issuing = false;  // a consumer gave up: buffer b may still be in use
                        break;
                    }
                    issue_chunk<L>(smem + b * L::BUF, &full[b], px, py, pa, pb, z0, ch * R);
                }
                cur = nxt;
            }
            // the last copy issued into each buffer has landed before the block
            // may exit (in normal operation the consumers have waited for it)
            for (uint32_t j = it > (uint32_t)NBUF ? it - NBUF : 0; j < it; ++j)
                tma::mbar_drain(&full[j % NBUF], (j / NBUF) & 1, err, a0.wait_ns);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    // this block's tiles: a contiguous range of the ensemble table, or every
    // gridDim.x-th z tile of a single simulation
    const bool rr = !BATCHED || bd.range == nullptr;
    const int t_first = rr ? blockIdx.x : bd.range[blockIdx.x];
    const int t_end = rr ? nzt : bd.range[blockIdx.x + 1];
    const int t_step = rr ? gridDim.x : 1;
    // moments of the stage input for the first tile
    if (t_first < t_end && tid < NMOM * TZ) {
        int inst, zt;
        tma_tile<BATCHED>(bd, t_first, inst, zt);
        const StageArgs &a = BATCHED ? bd.args[inst * 4 + STAGE - 1] : a0;
        if (a.flags & F_COLL)
            s_mom[tid / TZ][tid % TZ] = a.Min[(long long)(tid / TZ) * a.nz + zt * TZ + tid % TZ];
    }
    consumer_sync();

    uint32_t it = 0;
    int s_inst = -1;  // member whose arguments s_args holds
    int4 cur = make_int4(0, 0, 0, 0);
    if (BATCHED && t_first < t_end) cur = bd.table[t_first];
    for (int t = t_first; t < t_end; t += t_step) {
        const int inst = BATCHED ? cur.x : 0, zt = BATCHED ? cur.y : t;
        const int tn = t + t_step;
        int4 nxt = cur;
        if (BATCHED && tn < t_end) nxt = bd.table[tn];  // next tile's entry, one tile ahead
        if (BATCHED && inst != s_inst) {
            // a new member: its arguments into shared memory.  Read from there
            // (like a0 from parameter space) they cost no registers across the
            // chunk loop and cannot alias the stores to U and A.  The previous
            // tile's epilogue ended with a consumer barrier.
            if (tid < (int)(sizeof(StageArgs) / 8))
                reinterpret_cast<long long *>(s_args)[tid] =
                    reinterpret_cast<const long long *>(&bd.args[inst * 4 + STAGE - 1])[tid];
            consumer_sync();
            s_inst = inst;
        }
        const StageArgs &a = BATCHED ? *s_args : a0;
        const int nch = (a.nvz + R - 1) / R;
        const bool coll = (a.flags & F_COLL) != 0;
        const bool advec = (a.flags & F_ADVEC_OFF) == 0;
        const bool open_bc = a.bc != 0;
        const int z0 = zt * TZ;
        const int z = z0 + lane;
        // prefetch the next tile's input moments into a register
        double mnext = 0.0;
        if (tid < NMOM * TZ && tn < t_end) {
            const int in2 = BATCHED ? nxt.x : 0, zn = BATCHED ? nxt.y : tn;
            const StageArgs &an = BATCHED ? bd.args[in2 * 4 + STAGE - 1] : a0;
            if (an.flags & F_COLL)
                mnext = an.Min[(long long)(tid / TZ) * an.nz + zn * TZ + tid % TZ];
        }
        double macc[NMOM] = {0, 0, 0, 0, 0, 0};
        if constexpr (L::MSM) {
            // this warp's moment slots (the previous tile's epilogue has read them)
#pragma unroll
            for (int m = 0; m < NMOM; ++m) s_red[warp][m][lane] = 0.0;
        }

        for (int ch = 0; ch < nch; ++ch, ++it) {
            const int b = it % NBUF;
            const int v = ch * R + warp;
            const bool valid = v < a.nvz;
            const int vr = valid ? v : a.nvz - 1;
            // the row's velocity and advection factor: FV from the host tables
            // (read before the wait, so the load overlaps it), FD recomputed
            double vzv, factor;
            if constexpr (SCHEME == FV) {
                vzv = __ldg(&a.vz[vr]);
                factor = __ldg(&a.rowfac[vr]);
            } else {
                fd_row_values(a.v0, a.dv, a.dz, a.fd_advec, vr, vzv, factor);
            }
            const bool landed = tma::mbar_wait(&full[b], (it / NBUF) & 1, err, 2, a0.wait_ns);
            const unsigned char *buf = smem + b * L::BUF;
            // row r of component 0 in the input box (HALO cells each side); a
            // row's components are XW cells apart
            constexpr int XW = L::XW, YW = L::YW;
            auto xrow_of = [&](int r) {
                return reinterpret_cast<const TIN *>(buf) + r * (NCOMP * XW) + HALO;
            };
            auto yrow_of = [&](int r) {
                return reinterpret_cast<const double *>(buf + L::XB) + r * (NCOMP * YW) +
                       (INC ? HALO : 0);
            };
            const TIN *xrow = xrow_of(warp);  // this warp's row
            const double *yrow = yrow_of(warp);
            // the stage input at cell j of row x / y (j in [-HALO, TZ + HALO))
            auto in_r = [&](const TIN *x, const double *y, int q, int j) -> double {
                if constexpr (INC && STAGE >= 2)
                    return y[q * YW + j] + (double)x[q * XW + j];
                else
                    return (double)x[q * XW + j];
            };
            auto in = [&](int q, int j) -> double { return in_r(xrow, yrow, q, j); };
            // FP32-bulk: the stencil difference u(j + k) - u(j) as
            // (Y difference in FP64, rounded) + (D difference in FP32)
            auto dif = [&](const TIN *x, const double *y, int q, int j, int k) -> float {
                if constexpr (INC && STAGE >= 2)
                    return (float)(y[q * YW + j + k] - y[q * YW + j]) +
                           ((float)x[q * XW + j + k] - (float)x[q * XW + j]);
                else
                    return (float)((double)x[q * XW + j + k] - (double)x[q * XW + j]);
            };
            // upwind WENO7 face of component q about cell j of row x / y,
            // stencil direction dir
            auto face_r = [&](const TIN *x, const double *y, int q, int j, int dir) -> double {
                if constexpr (INC) {
                    const float corr =
                        weno7_corr(dif(x, y, q, j, -3 * dir), dif(x, y, q, j, -2 * dir),
                                   dif(x, y, q, j, -dir), dif(x, y, q, j, dir),
                                   dif(x, y, q, j, 2 * dir), dif(x, y, q, j, 3 * dir));
                    if constexpr (STAGE >= 2)  // Y + (D + correction)
                        return y[q * YW + j] + (double)((float)x[q * XW + j] + corr);
                    else
                        return (double)x[q * XW + j] + (double)corr;
                } else {
                    return weno7_face(in_r(x, y, q, j - 3 * dir), in_r(x, y, q, j - 2 * dir),
                                      in_r(x, y, q, j - dir), in_r(x, y, q, j),
                                      in_r(x, y, q, j + dir), in_r(x, y, q, j + 2 * dir),
                                      in_r(x, y, q, j + 3 * dir));
                }
            };
            // FP64: numerator and denominator of that face (face = centre +
            // num / den); the faces of components 0-3 and 4-7 of a row then
            // share one division (recip4)
            auto parts_r = [&](const TIN *x, const double *y, int q, int j, int dir, double &num,
                               double &den) {
                weno7_parts(in_r(x, y, q, j - 3 * dir), in_r(x, y, q, j - 2 * dir),
                            in_r(x, y, q, j - dir), in_r(x, y, q, j), in_r(x, y, q, j + dir),
                            in_r(x, y, q, j + 2 * dir), in_r(x, y, q, j + 3 * dir), num, den);
            };

            if constexpr (L::NE > 0) {
                // edge faces of this chunk: warps 2ch, 2ch + 1 (mod R) in turn,
                // lane -> (row 4h + lane / 8, component lane % 8).  Every lane
                // arrives, also without advection, so the barrier's phases
                // follow the ring.
                const int h = (warp - L::NE * ch) & (R - 1);
                if (h < L::NE) {
                    const int r = h * (32 / NCOMP) + (lane >> 3), q = lane & (NCOMP - 1);
                    if (advec) {
                        const double v2 = __ldg(&a.vz[min(ch * R + r, a.nvz - 1)]);
                        const int d2 = (v2 >= 0.0) ? 1 : -1;
                        const int je = d2 > 0 ? -1 : TZ;
                        if constexpr (INC) {
                            s_edge[b][r][q] = face_r(xrow_of(r), yrow_of(r), q, je, d2);
                        } else {
                            // the row's four denominators of this component group
                            // sit in lanes 4k..4k+3: the same division as the
                            // neighbouring tile's own face, bit for bit
                            double num, den, i[4];
                            parts_r(xrow_of(r), yrow_of(r), q, je, d2, num, den);
                            recip4(__shfl_sync(0xffffffffu, den, 0, 4),
                                   __shfl_sync(0xffffffffu, den, 1, 4),
                                   __shfl_sync(0xffffffffu, den, 2, 4),
                                   __shfl_sync(0xffffffffu, den, 3, 4), i[0], i[1], i[2], i[3]);
                            const int k = q & 3;
                            const double inv = k == 0 ? i[0] : k == 1 ? i[1] : k == 2 ? i[2] : i[3];
                            s_edge[b][r][q] = __fma_rn(num, inv, in_r(xrow_of(r), yrow_of(r), q, je));
                        }
                    }
                    tma::mbar_arrive(&ebar[b]);
                }
            }

            double c[NCOMP], o[NCOMP], ko[NCOMP];
#pragma unroll
            for (int q = 0; q < NCOMP; ++q) c[q] = in(q, lane);
            if (SCHEME == FV) {
                // upwind flux difference (rhs_fv.hpp:143-162): this lane's face
                // and its neighbour's; the face at the tile's upwind edge comes
                // from the chunk's edge warps (o[] holds the own faces meanwhile)
                const int dir = (vzv >= 0.0) ? 1 : -1;
                const int src = min(max(lane - dir, 0), TZ - 1);
                if constexpr (INC) {
#pragma unroll
                    for (int q = 0; q < NCOMP; ++q)
                        o[q] = advec ? face_r(xrow, yrow, q, lane, dir) : 0.0;
                } else {
                    double den[NCOMP];
#pragma unroll
                    for (int q = 0; q < NCOMP; ++q) {
                        o[q] = 0.0;
                        den[q] = 1.0;
                        if (advec) parts_r(xrow, yrow, q, lane, dir, o[q], den[q]);
                    }
#pragma unroll
                    for (int g = 0; g < NCOMP; g += 4) {
                        double i[4];
                        recip4(den[g], den[g + 1], den[g + 2], den[g + 3], i[0], i[1], i[2], i[3]);
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            o[g + k] = advec ? __fma_rn(o[g + k], i[k], c[g + k]) : 0.0;
                    }
                }
                if (advec) tma::mbar_wait(&ebar[b], (it / NBUF) & 1, err, 2, a0.wait_ns);
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) {
                    double adv = 0.0;
                    if (advec) {
                        const double fown = o[q];
                        double fnb = __shfl_sync(0xffffffffu, fown, src);
                        if ((dir > 0 && lane == 0) || (dir < 0 && lane == TZ - 1))
                            fnb = s_edge[b][warp][q];
                        if (open_bc) {
                            // flux ghosts under OPEN_BC (updateBufferZone on rflux/lflux,
                            // rhs_fv.hpp:118-119): rflux[-1] = rflux[0],
                            // lflux[nz] = 2 lflux[nz-1] - lflux[nz-2]
                            const double fm1 =
                                __shfl_sync(0xffffffffu, fown, lane > 0 ? lane - 1 : 0);
                            if (dir > 0 && z == 0) fnb = fown;
                            if (dir < 0 && z == a.nz - 1) fnb = fown * 2.0 - fm1;
                        }
                        adv = dir > 0 ? factor * (fown - fnb) : factor * (fnb - fown);
                    }
                    o[q] = adv;
                }
                if (a.flags & F_VAC) {
                    // read where used: batched, a is in shared memory and a
                    // per-tile copy would hold registers across the chunk loop
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
                if (a.flags & F_MAT) {
                    const double hm = a.Hm[z];
                    o[EXR] += hm * c[EXI];
                    o[EXI] += -hm * c[EXR];
                    o[BEXR] += -hm * c[BEXI];
                    o[BEXI] += hm * c[BEXR];
                }
            } else {
                // FD: vacuum, matter, advection, (collective below), dissipation
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) o[q] = 0.0;
                if (a.flags & F_VAC) {
                    // read where used: batched, a is in shared memory and a
                    // per-tile copy would hold registers across the chunk loop
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
                    const double hm = a.Hm[z];
                    o[EXR] += hm * c[EXI];
                    o[EXI] += -hm * c[EXR];
                    o[BEXR] += -hm * c[BEXI];
                    o[BEXI] += hm * c[BEXR];
                }
                const int sv = (vzv > 0.0) - (vzv < 0.0);
                const double ko_eps = a.ko_eps;
                // one pass over each stencil: advection now, dissipation kept
                // for after the collective term (the reference's order)
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) {
                    const double m2 = in(q, lane - 2), m1 = in(q, lane - 1), p1 = in(q, lane + 1),
                                 p2 = in(q, lane + 2);
                    if (advec) {
                        double adv;
                        if (!GEN || a.fd_advec == 0) {
                            adv = factor * ((m2 - p2) - 8.0 * (m1 - p1));
                        } else if (a.fd_advec == 1) {
                            adv = factor * (-4.0 * in(q, lane - 3 * sv) + 18.0 * in(q, lane - 2 * sv) -
                                            36.0 * in(q, lane - sv) + 22.0 * c[q]);
                        } else {
                            adv = factor * (in(q, lane - 3 * sv) - 6.0 * in(q, lane - 2 * sv) +
                                            18.0 * in(q, lane - sv) - 10.0 * c[q] -
                                            3.0 * in(q, lane + sv));
                        }
                        o[q] += adv;
                    }
                    if (GEN && a.ko_order == 5)
                        ko[q] = ko_eps * (in(q, lane - 3) + in(q, lane + 3) - 6.0 * (m2 + p2) +
                                          15.0 * (m1 + p1) - 20.0 * c[q]);
                    else
                        ko[q] = ko_eps * (m2 + p2 - 4.0 * (m1 + p1) + 6.0 * c[q]);
                }
            }
            if (coll) {
                // this tile's input moments, read where used (they stay in
                // shared memory until the tile epilogue replaces them)
                const double mudv = a.mu * a.dv;
                const double SA = s_mom[0][lane] - vzv * s_mom[3][lane],
                             SB = s_mom[1][lane] - vzv * s_mom[4][lane],
                             SC = s_mom[2][lane] - vzv * s_mom[5][lane];
                const double Iee = 2.0 * (c[EXR] * SA - c[EXI] * SB);
                const double Ibee = 2.0 * (c[BEXR] * SA + c[BEXI] * SB);
                o[EE] += mudv * Iee;
                o[XX] += mudv * (-Iee);
                o[EXR] += mudv * ((c[XX] - c[EE]) * SA + c[EXI] * SC);
                o[EXI] += mudv * (-(c[XX] - c[EE]) * SB - c[EXR] * SC);
                o[BEE] += mudv * Ibee;
                o[BXX] += mudv * (-Ibee);
                o[BEXR] += mudv * ((c[BXX] - c[BEE]) * SA - c[BEXI] * SC);
                o[BEXI] += mudv * ((c[BXX] - c[BEE]) * SB + c[BEXR] * SC);
            }
            if (SCHEME == FD) {
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) o[q] += ko[q];
            }

            // stage combine.  FP64 (stage values, A written once by stage 3 from
            // U in the A slot, U' and Y) or FP32-bulk (increments, common.cuh).
            const double dt = a.dt;
            // own-cell tiles: [row][component][TZ cells]
            const double *ys =
                reinterpret_cast<const double *>(buf + L::XB) + warp * (NCOMP * TZ) + lane;
            const double *as =
                reinterpret_cast<const double *>(buf + L::XB + L::YB) + warp * (NCOMP * TZ) + lane;
            const float *d1s =
                reinterpret_cast<const float *>(buf + L::XB + L::YB) + warp * (NCOMP * TZ) + lane;
            TOUT u[NCOMP];
            double anew[NCOMP];  // FP64 stage 3: the accumulator
            double um[NCOMP];    // the output as a stage value (for the moments)
#pragma unroll
            for (int q = 0; q < NCOMP; ++q) {
                const double kk = o[q];
                if constexpr (INC) {
                    // the base state at this cell: stage 1 reads Y itself
                    const double y = STAGE == 1 ? c[q] : yrow[q * YW + lane];
                    if (STAGE <= 3) {
                        u[q] = (TOUT)((STAGE == 3 ? dt : 0.5 * dt) * kk);
                        um[q] = y + (double)u[q];
                    } else {
                        const double d1 = (double)d1s[q * TZ];
                        const double d2 = (double)d1s[NCOMP * R * TZ + q * TZ];
                        const double d3 = (double)xrow[q * XW + lane];
                        const double yn = y + (d1 + 2.0 * d2 + d3) * (1.0 / 3.0) + (dt / 6.0) * kk;
                        u[q] = (TOUT)yn;
                        um[q] = yn;
                    }
                    anew[q] = 0.0;
                } else {
                    if (STAGE == 1) {
                        u[q] = (TOUT)(c[q] + (0.5 * dt) * kk);
                        anew[q] = 0.0;
                    } else if (STAGE == 2 || STAGE == 3) {
                        const double y = ys[q * TZ];
                        u[q] = (TOUT)(y + (STAGE == 2 ? 0.5 * dt : dt) * kk);
                        anew[q] = STAGE == 3 ? y + (as[q * TZ] - y) * (1.0 / 3.0) +
                                                   (c[q] - y) * (2.0 / 3.0) + (dt / 3.0) * kk
                                             : 0.0;  // stage 2 leaves A alone
                    } else {
                        u[q] = (TOUT)(as[q * TZ] + (dt / 6.0) * kk);
                        anew[q] = 0.0;
                    }
                    um[q] = (double)u[q];
                }
            }
            // this warp is done with the buffer (after a failed wait it keeps
            // the buffer: the producer's wait on it fails and it stops issuing;
            // without a producer, the count never completes and no warp
            // refills the buffer)
            __syncwarp();
            if (lane == 0 && landed) {
                if constexpr (PW) {
                    tma::mbar_arrive(&empty[b]);
                } else if (ring_release_count(&s_cnt[b]) == (it / NBUF) * R + (R - 1)) {
                    // the last of the R warps to release buffer b: its next chunk
                    fence_proxy_async_smem();
                    int t2 = t, ch2 = ch;
                    if (advance(t2, ch2, NBUF)) issue_at(t2, ch2, it + NBUF);
                }
            }

            TOUT uleft[NCOMP];
            if (open_bc) {
#pragma unroll
                for (int q = 0; q < NCOMP; ++q)
                    uleft[q] = __shfl_sync(0xffffffffu, u[q], lane > 0 ? lane - 1 : 0);
            }
            if (valid) {
                TOUT *U = static_cast<TOUT *>(a.U);
                const long long ro = (long long)v * a.ld + HP;
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) {
                    TOUT *row = U + q * a.cs + ro;
                    row[z] = u[q];
                    if (!INC && STAGE == 3) a.A[q * a.cs + ro + z] = anew[q];
                    if (!open_bc) {
                        if (z < a.H) row[z + a.nz] = u[q];
                        if (z >= a.nz - a.H) row[z - a.nz] = u[q];
                    } else {
                        if (z == 0)
                            for (int g = 1; g <= a.H; ++g) row[-g] = u[q];
                        if (z == a.nz - 1) {
                            TOUT p0 = uleft[q], p1 = u[q];
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
                    if constexpr (L::MSM) {
                        s_red[warp][0][lane] += Am;
                        s_red[warp][1][lane] += Bm;
                        s_red[warp][2][lane] += Cm;
                        s_red[warp][3][lane] += vzv * Am;
                        s_red[warp][4][lane] += vzv * Bm;
                        s_red[warp][5][lane] += vzv * Cm;
                    } else {
                        macc[0] += Am;
                        macc[1] += Bm;
                        macc[2] += Cm;
                        macc[3] += vzv * Am;
                        macc[4] += vzv * Bm;
                        macc[5] += vzv * Cm;
                    }
                }
            }
        }
        // tile epilogue: output moments (fixed-order sum over warps) and the
        // next tile's input moments
        if ((coll || BATCHED) && L::MSM) {
            consumer_sync();
            if (tid < NMOM * TZ) {
                const int m = tid / TZ, zz = tid % TZ;
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < R; ++w) s += s_red[w][m][zz];
                if (coll) a.Mout[(long long)m * a.nz + z0 + zz] = s;
                s_mom[m][zz] = mnext;  // every consumer read this tile's values above
            }
            consumer_sync();
        } else if (coll || BATCHED) {
            // warps w and w + R/2 pair up, then the R/2 pair sums are added
            // in a fixed order
            if (warp >= R / 2) {
#pragma unroll
                for (int m = 0; m < NMOM; ++m) s_red[warp - R / 2][m][lane] = macc[m];
            }
            consumer_sync();
            if (warp < R / 2) {
#pragma unroll
                for (int m = 0; m < NMOM; ++m) s_red[warp][m][lane] += macc[m];
            }
            consumer_sync();
            if (tid < NMOM * TZ) {
                const int m = tid / TZ, zz = tid % TZ;
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < R / 2; ++w) s += s_red[w][m][zz];
                if (coll) a.Mout[(long long)m * a.nz + z0 + zz] = s;
                s_mom[m][zz] = mnext;  // every consumer read this tile's values above
            }
            consumer_sync();
        }
        cur = nxt;
    }
    if constexpr (!PW) {
        // the last copies issued into each buffer have landed before the block
        // exits (in normal operation the consumers have waited for them)
        consumer_sync();
        if (tid == 0)
            for (int b = 0; b < NBUF; ++b)
                if (s_last[b] >= 0)
                    tma::mbar_drain(&full[b], ((uint32_t)s_last[b] / NBUF) & 1, err, a0.wait_ns);
    }
}

// ---------------------------------------------------------------------------
// host side

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// 3-D map over one 8-component buffer: (cells of a padded row, components,
// rows), so that a box lands in shared memory as [row][component][cell]
int make_state_map(CUtensorMap *map, const void *base, int elem_bytes, int ld, int nvz,
                   long long cs, int box_cells, int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return -1;
    cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)NCOMP, (cuuint64_t)nvz};
    cuuint64_t strides[2] = {(cuuint64_t)cs * elem_bytes, (cuuint64_t)ld * elem_bytes};
    cuuint32_t box[3] = {(cuuint32_t)box_cells, (cuuint32_t)NCOMP, (cuuint32_t)box_rows};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                    3, const_cast<void *>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

int tma_box_x(int elem_bytes) { return elem_bytes == 8 ? tma::xw<double>() : tma::xw<float>(); }
int tma_box_tile() { return tma::TZ; }
// Rows of a map's box: `wide` for the operands of the 12-row FD stages.
int tma_box_rows(int scheme, bool wide) { return scheme == FD && wide ? 12 : 8; }
// largest nvz the TMA layout is offered for (the range its tests cover; the
// kernel itself keeps no per-row state in shared memory)
int tma_max_nvz() { return TMA_MAX_NVZ; }

static const int TMA_SMEM_MAX = 232448;  // opt-in shared memory per block on sm_100
static const int TMA_SMEM_SM = 233472;   // shared memory per SM (1 KB reserved per block)

// Shared memory of one block with an NB-deep ring.
template <int SCHEME, class TIN, class TOUT, int STAGE>
static int tma_smem(int NB)
{
    using L = tma::Layout<SCHEME, TIN, TOUT, STAGE>;
    return NB * L::BUF + (2 + (L::NE ? 1 : 0)) * NB * 8 + (1 + L::NRED) * NMOM * tma::TZ * 8 +
           (L::NE ? NB * L::R * NCOMP * 8 : 0) +
           (int)sizeof(StageArgs) + NB * 8;  // + release counts, last chunks
}

static int tma_smem_limit(int minb)
{
    return minb == 1 ? TMA_SMEM_MAX : TMA_SMEM_SM / minb - 1024;
}

// The operand maps of one launch: X (stage input with halo), Y, A and B (see
// Layout; unused ones are ignored).
struct StageMaps {
    const CUtensorMap *x, *y, *a, *b;
};

template <int SCHEME, bool GEN, int STAGE, class TIN, class TOUT, int NB, int MINB>
static cudaError_t launch_nb(const StageMaps &m, const StageArgs &a, int *err, int nblocks,
                             cudaStream_t s, const BatchDev *bd)
{
    auto kern = rk4_stage_tma_kernel<SCHEME, GEN, STAGE, TIN, TOUT, NB, false, MINB>;
    auto kernb = rk4_stage_tma_kernel<SCHEME, GEN, STAGE, TIN, TOUT, NB, true, MINB>;
    if (nblocks <= 0) {  // preparation call: shared-memory limit and carveout
        for (auto k : {kern, kernb}) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 TMA_SMEM_MAX);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const int shmem = tma_smem<SCHEME, TIN, TOUT, STAGE>(NB);
    using L = tma::Layout<SCHEME, TIN, TOUT, STAGE>;
    constexpr int NT = tma::producer_warp<SCHEME, false>() ? L::NTHR : L::NTHR_NP;
    if (bd)
        kernb<<<nblocks, NT, shmem, s>>>(*m.x, *m.y, *m.a, *m.b, a, err, *bd);
    else
        kern<<<nblocks, NT, shmem, s>>>(*m.x, *m.y, *m.a, *m.b, a, err, BatchDev{});
    return cudaGetLastError();
}

// Ring depth of the FD kernel (one block per SM): the deepest ring of at most
// 4 buffers that total at most 144 KB.  Measured at nz 32768 x nvz 256:
// stages of 53-54 KB chunks (FP64 stage 3) are fastest with 2 buffers
// (0.441 / 0.534 / 0.545 ms with 2 / 3 / 4), FP64 stages 2 and 4 (38 KB) with
// 3, the FP32-bulk stages (48 KB chunks) with 3 (stage 4: 0.358 ms with 2,
// 0.320 ms with 3).
// COSENU_TMA_RING=n (2..4) overrides the depth where it fits.
static int tma_ring_env()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("COSENU_TMA_RING");
        v = (e && e[0] >= '2' && e[0] <= '4' && e[1] == 0) ? e[0] - '0' : 0;
    }
    return v;
}

template <class TIN, class TOUT, int STAGE>
static int tma_fd_ring()
{
    using L = tma::Layout<FD, TIN, TOUT, STAGE>;
    int nb = 2;
    while (nb < 4 && (nb + 1) * L::BUF <= 144 * 1024) ++nb;
    const int e = tma_ring_env();
    if (e) nb = e;
    while (nb > 2 && tma_smem<FD, TIN, TOUT, STAGE>(nb) > tma_smem_limit(1)) --nb;
    return nb;
}

// Blocks per SM.  FD (memory bound): one, with the deepest ring that fits.
// FV (FP64 bound, 8 warps per block): two, to hide FP64 and shared-memory
// latency with twice the warps, each with the deepest ring that fits in half
// the SM (COSENU_TMA_MINB=1 selects one block per SM with a 4-deep ring).
static int tma_minb_env()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("COSENU_TMA_MINB");
        v = (e && e[0] == '1') ? 1 : 2;
    }
    return v;
}

// FD: COSENU_TMA_MINB_FD=2 runs two blocks per SM (<= 112 registers each,
// half the shared memory) instead of one.
static int tma_minb_fd_env()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("COSENU_TMA_MINB_FD");
        v = (e && e[0] == '2') ? 2 : 1;
    }
    return v;
}

int tma_blocks_per_sm(int scheme) { return scheme == FV ? tma_minb_env() : tma_minb_fd_env(); }

template <int SCHEME, bool GEN, int STAGE, class TIN, class TOUT>
static cudaError_t launch_one(const StageMaps &m, const StageArgs &a, int *err, int nblocks,
                              cudaStream_t s, const BatchDev *bd)
{
#define LNB(NB, MINB) launch_nb<SCHEME, GEN, STAGE, TIN, TOUT, NB, MINB>(m, a, err, nblocks, s, bd)
    if constexpr (SCHEME == FD) {
        if (nblocks <= 0) {
            cudaError_t e = LNB(2, 1);
            if (e == cudaSuccess) e = LNB(3, 1);
            if (e == cudaSuccess) e = LNB(4, 1);
            if (e == cudaSuccess) e = LNB(2, 2);
            if (e == cudaSuccess) e = LNB(3, 2);
            if (e == cudaSuccess) e = LNB(4, 2);
            return e;
        }
        if (tma_minb_fd_env() == 2) {
            const int lim = tma_smem_limit(2);
            if (tma_smem<SCHEME, TIN, TOUT, STAGE>(4) <= lim) return LNB(4, 2);
            if (tma_smem<SCHEME, TIN, TOUT, STAGE>(3) <= lim) return LNB(3, 2);
            return LNB(2, 2);
        }
        switch (tma_fd_ring<TIN, TOUT, STAGE>()) {
        case 2: return LNB(2, 1);
        case 3: return LNB(3, 1);
        default: return LNB(4, 1);
        }
    } else {
        if (nblocks <= 0) {
            cudaError_t e = LNB(4, 1);
            if (e == cudaSuccess) e = LNB(4, 2);
            if (e == cudaSuccess) e = LNB(3, 2);
            if (e == cudaSuccess) e = LNB(2, 2);
            return e;
        }
        if (tma_minb_env() == 1) return LNB(4, 1);
        const int lim = tma_smem_limit(2);
        if (tma_smem<SCHEME, TIN, TOUT, STAGE>(4) <= lim) return LNB(4, 2);
        if (tma_smem<SCHEME, TIN, TOUT, STAGE>(3) <= lim) return LNB(3, 2);
        return LNB(2, 2);
    }
#undef LNB
}

template <int SCHEME, bool GEN>
static cudaError_t launch_p(const StageMaps &m, const StageArgs &a, int stage, int fp32, int *err,
                            int nblocks, cudaStream_t s, const BatchDev *bd)
{
    if (fp32) {
        // FP32-bulk: Y in, D1 out; Y + D1 in, D2 out; Y + D2 in, D3 out; Y + D3 in, Y' out
        switch (stage) {
        case 1: return launch_one<SCHEME, GEN, 1, double, float>(m, a, err, nblocks, s, bd);
        case 2: return launch_one<SCHEME, GEN, 2, float, float>(m, a, err, nblocks, s, bd);
        case 3: return launch_one<SCHEME, GEN, 3, float, float>(m, a, err, nblocks, s, bd);
        case 4: return launch_one<SCHEME, GEN, 4, float, double>(m, a, err, nblocks, s, bd);
        }
    } else {
        switch (stage) {
        case 1: return launch_one<SCHEME, GEN, 1, double, double>(m, a, err, nblocks, s, bd);
        case 2: return launch_one<SCHEME, GEN, 2, double, double>(m, a, err, nblocks, s, bd);
        case 3: return launch_one<SCHEME, GEN, 3, double, double>(m, a, err, nblocks, s, bd);
        case 4: return launch_one<SCHEME, GEN, 4, double, double>(m, a, err, nblocks, s, bd);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_rk4_stage_tma(const CUtensorMap &mX, const CUtensorMap &mY,
                                 const CUtensorMap &mA, const CUtensorMap &mB, const StageArgs &a,
                                 int scheme, int stage, int fp32, int *err, int nblocks,
                                 cudaStream_t s)
{
    const StageMaps m{&mX, &mY, &mA, &mB};
    if (scheme == FV) return launch_p<FV, false>(m, a, stage, fp32, err, nblocks, s, nullptr);
    const bool gen = a.fd_advec != 0 || a.ko_order == 5;
    return gen ? launch_p<FD, true>(m, a, stage, fp32, err, nblocks, s, nullptr)
               : launch_p<FD, false>(m, a, stage, fp32, err, nblocks, s, nullptr);
}

// Ensemble launch: `a` carries the variant switches shared by every instance
// (scheme variant, precision); per-instance values come from bd.
cudaError_t launch_rk4_stage_tma_batch(const BatchDev &bd, const StageArgs &a, int scheme,
                                       int stage, int fp32, int *err, int nblocks, int max_nvz,
                                       cudaStream_t s)
{
    CUtensorMap z{};
    const StageMaps m{&z, &z, &z, &z};
    if (scheme == FV) return launch_p<FV, false>(m, a, stage, fp32, err, nblocks, s, &bd);
    const bool gen = a.fd_advec != 0 || a.ko_order == 5;
    return gen ? launch_p<FD, true>(m, a, stage, fp32, err, nblocks, s, &bd)
               : launch_p<FD, false>(m, a, stage, fp32, err, nblocks, s, &bd);
}

// Sets the shared-memory attribute of every instantiation on the current device.
cudaError_t tma_prepare()
{
    CUtensorMap m{};
    StageArgs a{};
    for (int sch = 0; sch < 2; ++sch)
        for (int gen = 0; gen < 2; ++gen)
            for (int fp32 = 0; fp32 < 2; ++fp32)
                for (int st = 1; st <= 4; ++st) {
                    a.fd_advec = gen;
                    a.ko_order = 3;
                    cudaError_t e = launch_rk4_stage_tma(m, m, m, m, a, sch, st, fp32, nullptr, 0,
                                                         nullptr);
                    if (e != cudaSuccess) return e;
                }
    return cudaSuccess;
}

}  // namespace cosenu
