// dsmc_persist.cuh - every case of a context stepped by ONE persistent kernel.
//
// k_persistent runs n time steps of all cases in a single cooperative launch
// (all CTAs resident at once, grid = CTAs per SM x SMs).  Each step is the
// phase sequence of the step graph, phase for phase the same device code
// (the bodies of dsmc_kernels.cuh), with a grid barrier where the graph has
// a kernel boundary:
//
//   plan (CTA 0) | move tiles, inject units | move_near | dead-count scan |
//   holes (+ tail plan) | tail | cell scan, tile-count scan |
//   out-of-range lists, collision select | cell fix | scatter |
//   collision pairs | sample (+ end of step, CTA 0) |
//
// so every result is the graph's, bit for bit.  Work is dealt as in the
// graph kernels: static tile schedules over the resident CTAs, tickets, or
// virtual blocks (the chunked scans).  A CTA is TILE_THREADS wide in every
// phase; sampling uses blocks of TILE_THREADS / 2 cells (two threads a cell).
//
// Every barrier wait is bounded: after wait_ns nanoseconds (or GRID_SPIN_LIMIT
// polls) the CTA reports DSMC_ERR_TIMEOUT, raises the launch's abort flag and
// leaves; the other CTAs see the flag at their next barrier and leave too,
// so the context stays usable and the host reads the status.  A phase whose
// staged copies timed out raises the flag the same way.
#pragma once

#include <cstdint>

#include "dsmc_kernels.cuh"

namespace dsmc {

// Barrier state of one launch, zeroed before it (a memset node of the graph).
// Arrivals and the released generation sit on separate 128-byte lines, so
// the CTAs that poll do not contend with the ones still arriving.
struct GridSync {
    unsigned long long count; // arrivals over all barriers of the launch
    unsigned long long pad0[15];
    unsigned long long gen;   // barriers released so far
    int abort;                // raised by a CTA that gave up or failed a phase
    int pad1[29];
};
static_assert(sizeof(GridSync) == 256, "two lines");

constexpr int PERSIST_THREADS = TILE_THREADS;
// Sampling in the persistent step: blocks of 128 cells, two threads a cell,
// one stage (the step graph's k_sample runs more, narrower CTAs per SM).
#ifndef DSMC_PERSIST_SAMPLE_SPLIT
#define DSMC_PERSIST_SAMPLE_SPLIT 2
#endif
#ifndef DSMC_PERSIST_SAMPLE_STAGES
#define DSMC_PERSIST_SAMPLE_STAGES 1
#endif
constexpr int PERSIST_SAMPLE_SPLIT = DSMC_PERSIST_SAMPLE_SPLIT;
constexpr int PERSIST_SAMPLE_CELLS = PERSIST_THREADS / PERSIST_SAMPLE_SPLIT;
constexpr int PERSIST_SAMPLE_STAGES = DSMC_PERSIST_SAMPLE_STAGES;
constexpr uint32_t GRID_SPIN_LIMIT = 1u << 22; // polls of a wait (besides its time bound)
#ifndef DSMC_GRID_SLEEP_NS
#define DSMC_GRID_SLEEP_NS 512
#endif

// Pipeline depths and CTAs per SM of the persistent kernel: the deepest
// staging that leaves room for the occupancy (dynamic shared memory is the
// largest of the three staged phases).
#ifndef DSMC_PERSIST_MOVE_STAGES_F32
#define DSMC_PERSIST_MOVE_STAGES_F32 3
#endif
template <class T> __host__ __device__ constexpr int persist_move_stages()
{
    return sizeof(T) == 4 ? DSMC_PERSIST_MOVE_STAGES_F32 : 2;
}
template <class T> __host__ __device__ constexpr int persist_scatter_stages() { return 2; }
#ifndef DSMC_PERSIST_MIN_BLOCKS_F32
#define DSMC_PERSIST_MIN_BLOCKS_F32 3
#endif
template <class T> __host__ __device__ constexpr int persist_min_blocks()
{
    return sizeof(T) == 4 ? DSMC_PERSIST_MIN_BLOCKS_F32 : 2;
}
template <class T> __host__ __device__ constexpr size_t persist_smem()
{
    const size_t a = sizeof(MoveStage<T>) * persist_move_stages<T>();
    const size_t b = sizeof(ScatterStage<T>) * persist_scatter_stages<T>();
    const size_t c = sample_smem<T, PERSIST_SAMPLE_CELLS, PERSIST_SAMPLE_STAGES>();
    return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void grid_abort(GridSync *g)
{
    if (threadIdx.x == 0)
        atomicExch(&g->abort, 1);
}

__device__ __forceinline__ void st_release_gpu(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// All CTAs of the launch meet here.  `target` counts the arrivals this CTA
// waits for (it advances by the grid size per barrier): the CTA whose
// arrival makes the count reach it releases the barrier by advancing the
// generation word, which the others poll.  Every write made before the
// barrier by any thread of any CTA is visible after it; thread 0 also orders
// the CTA's earlier shared-memory accesses before the async proxy's next
// writes (the next phase's staged copies reuse the memory).  False when the
// launch is abandoned: the caller returns.
__device__ __forceinline__ bool grid_sync(GridSync *g, unsigned long long &target,
                                          uint64_t wait_ns, int *err)
{
    __shared__ int s_go;
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        const unsigned long long gen = target / gridDim.x; // this barrier's number
        __threadfence();
        int go = 1;
        if (atomicAdd(&g->count, 1ull) + 1 == target) {
            __threadfence(); // every arrival (and what preceded it) is seen ...
            st_release_gpu(&g->gen, gen); // ... and released with the generation
        } else {
            const uint64_t t0 = globaltimer_ns();
            for (uint32_t spins = 0;; ++spins) {
                if (ld_acquire_gpu(&g->gen) >= gen)
                    break;
                if (*reinterpret_cast<volatile int *>(&g->abort)) {
                    go = 0;
                    break;
                }
                if (spins >= GRID_SPIN_LIMIT || globaltimer_ns() - t0 > wait_ns) {
                    report_error(err, DSMC_ERR_TIMEOUT);
                    atomicExch(&g->abort, 1);
                    go = 0;
                    break;
                }
                if (DSMC_GRID_SLEEP_NS > 0)
                    __nanosleep(DSMC_GRID_SLEEP_NS); // spare the memory system while waiting
            }
        }
        __threadfence();
        fence_proxy_async_smem();
        s_go = go;
    }
    __syncthreads();
    return s_go != 0;
}

// Everything a step of the context reads and writes.  The two particle
// buffers are separate members: indexing a parameter array by the run-time
// side would copy it to local memory.
template <class T> struct StepArgs {
    const CaseDev *cases;
    CaseState *st;
    StepScratch *sc;
    TileTables tt;
    Slots<T> buf0, buf1;
    uint32_t *key;
    Cells cells;
    int32_t *tile_in, *tile_prefix, *tile_dead, *tile_dprefix, *itile_dead, *itile_dprefix;
    uint64_t *tail_chain, *cell_chain;
    int32_t *hole_pos, *hole_oc;
    uint32_t *obuf, *near_list;
    int32_t *olist;
    uint32_t *coll_list;
    dsmc_counters *rec; // every case's counters at the end of each step
    int32_t *tmp;       // 2 x ncase
    const int64_t *pbases;
    int total_cells, ncase;
    int scan_chunks; // chunks of PERSIST_THREADS * SCAN_VEC tile counts per case
    int *err;
    GridSync *gsync;
    uint64_t wait_ns;               // bound of one barrier wait
    unsigned long long *phase_ns;   // PERSIST_PHASES sums of phase durations (CTA 0's view)
};

// The phases of a step, in order (each ends at a grid barrier).
constexpr int PERSIST_PHASES = 12;

// n_steps steps from buffer side0.  Between phases the kernel keeps almost
// nothing in registers (the barrier count, the phase timer and the buffer
// side live in shared memory; the arguments in the parameter bank), so each
// phase has the register budget to itself.
template <class T>
__global__ void __launch_bounds__(PERSIST_THREADS, persist_min_blocks<T>())
    k_persistent(const StepArgs<T> a, int n_steps, int side0)
{
    constexpr int NT = PERSIST_THREADS;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ unsigned long long s_target; // arrivals awaited (thread 0)
    __shared__ uint64_t s_tprev;            // CTA 0: end of the previous phase
    __shared__ int s_phase, s_side;
    // CTA 0 times each phase from barrier to barrier: a barrier opens when
    // the last CTA reaches it, so that is the phase's device time.
    if (threadIdx.x == 0) {
        s_target = 0;
        s_tprev = globaltimer_ns();
        s_phase = 0;
    }
#define DSMC_GRID_SYNC()                                                   \
    if (!grid_sync(a.gsync, s_target, a.wait_ns, a.err))                   \
        return;                                                            \
    if (blockIdx.x == 0 && threadIdx.x == 0) {                             \
        const uint64_t t_now = globaltimer_ns();                           \
        a.phase_ns[s_phase] += t_now - s_tprev;                            \
        s_tprev = t_now;                                                   \
        s_phase = s_phase + 1 == PERSIST_PHASES ? 0 : s_phase + 1;         \
    }
#define DSMC_OR_ABORT(call)                                                \
    if (!(call)) {                                                         \
        grid_abort(a.gsync);                                               \
        return;                                                            \
    }
// The buffers of this step, read again in every phase.
#define DSMC_SIDE() (*reinterpret_cast<volatile int *>(&s_side))
#define DSMC_CUR() (DSMC_SIDE() ? a.buf1 : a.buf0)
#define DSMC_NXT() (DSMC_SIDE() ? a.buf0 : a.buf1)
    for (int s = 0; s < n_steps; ++s) {
        if (threadIdx.x == 0)
            s_side = (side0 + s) & 1; // read after the next barrier
        // MoveParticles, with the inflow strips of BoundaryConditions (their
        // slots follow the moved ones).
        if (blockIdx.x == 0)
            plan_step(a.cases, a.st, a.sc, a.tt, a.tmp, a.itile_dead, a.cell_chain, a.ncase, 0,
                      a.err);
        DSMC_GRID_SYNC();
        DSMC_OR_ABORT((move_tiles<T, persist_move_stages<T>()>(
            a.cases, a.st, a.sc, a.tt, DSMC_CUR(), a.key, a.cells, a.tile_in, a.tile_dead, a.obuf,
            a.near_list, a.ncase, a.err, smem_raw, blockIdx.x, gridDim.x)));
        inject_units<T>(a.cases, a.st, a.sc, a.tt, DSMC_CUR(), a.key, a.cells, a.itile_dead,
                        a.obuf, a.ncase, a.err);
        DSMC_GRID_SYNC();
        move_near<T>(a.cases, a.st, a.sc, a.tt, DSMC_CUR(), a.key, a.cells, a.tile_in,
                     a.tile_dead, a.obuf, a.near_list, a.ncase, a.err, blockIdx.x, gridDim.x);
        DSMC_GRID_SYNC();
        // The swap-with-last removal: removed-slot prefix, holes, tail.
        for (int v = blockIdx.x; v < a.scan_chunks * a.ncase; v += gridDim.x)
            dead_scan_chunk<NT>(a.st, a.tile_dead, a.tile_dprefix, a.itile_dead, a.itile_dprefix,
                                v % a.scan_chunks, v / a.scan_chunks);
        DSMC_GRID_SYNC();
        holes_blocks(a.cases, a.st, a.sc, a.tt, a.key, a.tile_dead, a.tile_dprefix, a.itile_dead,
                     a.itile_dprefix, a.hole_pos, a.hole_oc, a.tmp, a.tail_chain, a.ncase,
                     blockIdx.x, gridDim.x);
        DSMC_GRID_SYNC();
        tail_tiles<T>(a.cases, a.st, a.sc, a.tt, DSMC_CUR(), a.key, a.cells, a.tile_in,
                      a.tail_chain, a.hole_pos, a.hole_oc, a.obuf, a.ncase, a.err);
        DSMC_GRID_SYNC();
        // Indexing: the stable counting sort into the other buffer.
        cell_scan_tiles(a.cases, a.sc, a.tt, a.cells, DSMC_SIDE() ^ 1, a.cell_chain, a.ncase,
                        a.err);
        for (int v = blockIdx.x; v < a.scan_chunks * a.ncase; v += gridDim.x)
            tile_scan_chunk<NT>(a.st, a.tile_in, a.tile_prefix, v % a.scan_chunks,
                                v / a.scan_chunks);
        DSMC_GRID_SYNC();
        olist_blocks(a.cases, a.st, a.sc, a.obuf, a.key, a.cells, a.olist, a.pbases, a.ncase,
                     a.err, blockIdx.x, gridDim.x);
        collide_select_blocks(a.cases, a.st, a.sc, a.tt, a.cells, DSMC_SIDE() ^ 1, a.coll_list,
                              a.total_cells, a.ncase, blockIdx.x, gridDim.x);
        DSMC_GRID_SYNC();
        cell_fix_blocks(a.cases, a.st, a.tt, a.cells, DSMC_SIDE(), a.key, a.olist, a.total_cells,
                        a.ncase, a.err, blockIdx.x, gridDim.x);
        DSMC_GRID_SYNC();
        DSMC_OR_ABORT((scatter_tiles<T, persist_scatter_stages<T>()>(
            a.cases, a.st, a.tt, DSMC_CUR(), DSMC_NXT(), a.key, a.cells, a.tile_prefix, a.ncase,
            a.err, smem_raw, blockIdx.x, gridDim.x)));
        DSMC_GRID_SYNC();
        // CollideParticles, then Sampling, which also ends the step.
        collide_pairs_blocks<T>(a.cases, a.st, a.sc, a.tt, DSMC_NXT(), a.cells, DSMC_SIDE() ^ 1,
                                a.coll_list, a.ncase, blockIdx.x, gridDim.x);
        DSMC_GRID_SYNC();
        DSMC_OR_ABORT((sample_blocks<T, PERSIST_SAMPLE_CELLS, PERSIST_SAMPLE_SPLIT,
                                     PERSIST_SAMPLE_STAGES>(
            a.cases, a.st, a.tt, DSMC_NXT(), a.cells, DSMC_SIDE() ^ 1, a.ncase, 1, a.rec, a.err,
            smem_raw, blockIdx.x, gridDim.x)));
        DSMC_GRID_SYNC();
    }
#undef DSMC_NXT
#undef DSMC_CUR
#undef DSMC_SIDE
#undef DSMC_OR_ABORT
#undef DSMC_GRID_SYNC
}

// One CTA at a barrier that `missing` more arrivals would open: it can never
// complete, so its bounded wait runs out.  The test of the timeout path (the
// status comes back, the context stays usable).
__global__ void k_grid_sync_probe(GridSync *g, int missing, uint64_t wait_ns, int *err)
{
    unsigned long long target = static_cast<unsigned long long>(missing); // never reached
    (void)grid_sync(g, target, wait_ns, err);
}

} // namespace dsmc
