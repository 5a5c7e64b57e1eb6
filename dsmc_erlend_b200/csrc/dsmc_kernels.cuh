// dsmc_kernels.cuh - the kernels of one DSMC time step.
//
// A step over all cases of a context is this fixed launch sequence (every
// size lives on the device, so the sequence is captured once in a CUDA graph):
//
//   k_plan      1 CTA    per case: sampling mode, inflow counts (the count
//                        draws of GenerateNewParticles), tile tables
//   k_move      tiles    MoveParticles + the new cell of every slot, removal
//                        flag, in-range flag, per-cell counts, hole list
//   k_inject    tiles    GenerateNewParticles for the four strips, appended
//   k_dead_scan chunks   prefix of removed-slot counts per tile
//   k_holes     tiles    removed-slot list in slot order; its last CTA:
//                        survivors K, hole count H, tail tiles
//   k_tail      tiles    swap-with-last: alive tail slots refill the holes
//   k_cell_scan tiles    per-cell offsets (stable counting sort)
//   k_tile_scan chunks   prefix of in-range counts per tile
//   k_olist     grid     lists of the particles that changed cell
//   k_cell_fix  grid     orders those lists, places them, per-cell bases
//   k_scatter   tiles    places every in-range particle
//   k_collide_select  cells  NTC pair counts, list of cells with candidates
//   k_collide_pairs   list   NTC + VHS collisions of the listed cells
//   k_sample    cells    moment sampling, two threads per cell; in a full
//                        step its first CTA also ends the step (Step++,
//                        NP = K); the staged calls use k_finish for that
//
// Particle order contract (the reference's, made parallel):
//   * at the start of a step slots [0, n_old) are sorted by cell, each cell
//     keeping the order its particles had before the sort;
//   * injected particles are appended in strip order L, R, B, T;
//   * removal is the reference's swap-with-last loop (Boundary.cpp:181-202):
//     survivors below K stay, and the m-th removed slot below K receives the
//     m-th survivor at or above K counted from the end;
//   * Indexing's lists are stable in slot order (Geometry.cpp:168), so the
//     sort is a stable counting sort by cell.
#pragma once

#include <cstdint>

#include "dsmc_device.cuh"
#include "dsmc_bulk.cuh"
#include "dsmc_scan.cuh"

namespace dsmc {

// Tile bases of every case for each tiled kernel: entry i is the first
// global tile of case i, entry ncase the total.  The last three are static:
// cell-scan tiles, collide blocks and global cell ids (ncell + 1 per case).
struct TileTables {
    int32_t *move0, *inject0, *tail0, *scatter0, *cell0, *cblock0, *cellbase;
};

// Particle arrays of one buffer.
template <class T> struct Slots {
    T *x, *y, *vx, *vy, *vz;
};

// Per-cell arrays, indexed by global cell id (each case owns ncell + 1 ids).
struct Cells {
    int32_t *n_in, *n_o, *o_fill;
    int32_t *fin, *ostart, *base_in;
    int32_t *start[2];   // cell start offsets, ping-pong: old and new
    double *acc;         // 14 moment sums per cell, one array per moment
    int64_t acc_stride;  // elements per moment array
};

// The start offsets of buffer `side`.  A select, not an index: indexing the
// kernel parameter with a run-time value would copy it to local memory.
__device__ __forceinline__ int32_t *start_of(const Cells &c, int side)
{
    return side ? c.start[1] : c.start[0];
}

// Moments kept per cell.  The reference's CELL (include/Cell.h:4-10) holds
// CountVV as a 3x3 tensor; it is symmetric and stored once here.
enum : int {
    ACC_NP = 0,
    ACC_V0, ACC_V1, ACC_V2,
    ACC_VV00, ACC_VV01, ACC_VV02, ACC_VV11, ACC_VV12, ACC_VV22,
    ACC_V2V0, ACC_V2V1, ACC_V2V2,
    ACC_NC,
    ACC_COUNT
};

__device__ __forceinline__ int case_of(const int32_t *base, int ncase, int t)
{
    int lo = 0, hi = ncase - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Exclusive scan over cases of one count per case (<= 1024 threads, any
// number of cases); writes base[0..ncase] and returns nothing.
__device__ __forceinline__ void case_scan(int32_t *base, const int32_t *count_of_case_smem,
                                          int ncase)
{
    // Single-thread scan: the number of cases is at most a few thousand and
    // this runs once per step in a 1-CTA kernel.
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int i = 0; i < ncase; ++i) {
            base[i] = run;
            run += count_of_case_smem[i];
        }
        base[ncase] = run;
    }
}

// ---------------------------------------------------------------------------
// k_plan: start of a step (or of the cold start when init_mode is set).
// ---------------------------------------------------------------------------
// It first clears the step's scratch counters and the look-back status
// words of the cell scan (the first kernel of a step: nothing reads them
// before), so the step needs no memset of its own.  One CTA, any width.
__device__ __forceinline__ void plan_step(const CaseDev *cases, CaseState *st, StepScratch *sc,
                                          TileTables tt, int32_t *tmp, int32_t *itile_dead,
                                          uint64_t *cell_chain, int ncase, int init_mode,
                                          int *err)
{
    {
        uint32_t *words = reinterpret_cast<uint32_t *>(sc);
        for (int i = threadIdx.x; i < static_cast<int>(sizeof(StepScratch) / 4); i += blockDim.x)
            words[i] = 0u;
        for (int i = threadIdx.x; i < tt.cell0[ncase]; i += blockDim.x)
            cell_chain[i] = 0ull;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < ncase; i += blockDim.x) {
        const CaseDev &c = cases[i];
        CaseState &s = st[i];
        if (init_mode) {
            s.n_old = 0;
            s.sampling_mode = 0;
        } else {
            // Simulation.cpp:139-146
            s.sampling_mode =
                (s.step > c.first_sampling_step && s.step % c.sampling_period == 0) ? 1 : 0;
            if (s.step > c.first_sampling_step)
                s.drag_time += c.dt;
        }
        // The count draws of GenerateNewParticles (Boundary.cpp:62-71).
        const int s0 = init_mode ? 4 : 0;
        const int s1 = init_mode ? 5 : 4;
        int64_t total = 0;
        for (int k = 0; k < 5; ++k) {
            s.inj_count[k] = 0;
            s.inj_c0[k] = 0;
        }
        for (int k = s0; k < s1; ++k) {
            dsmc_stream r;
            if (init_mode)
                open_stream(r, c, DSMC_RNG_INIT, 0, 0);
            else
                open_stream(r, c, DSMC_RNG_INJECT, s.step, static_cast<uint32_t>(k));
            int draws;
            const int n = inflow_count(r, c.strip_navg[k], &draws);
            s.inj_count[k] = n;
            s.inj_c0[k] = draws;
            total += n;
        }
        if (s.n_old + total > c.cap) {
            // Boundary.cpp:73-80 exits; the step injects nothing and reports.
            report_error(err, DSMC_ERR_CAPACITY);
            for (int k = 0; k < 5; ++k)
                s.inj_count[k] = 0;
            total = 0;
        }
        s.inj_off[0] = 0;
        for (int k = 0; k < 5; ++k)
            s.inj_off[k + 1] = s.inj_off[k] + s.inj_count[k];
        s.n_total = s.n_old + total;
        s.dead_old = 0;
        s.dead_total = 0;
        s.nc_step = 0;
        s.n_move_tiles = static_cast<int32_t>((s.n_old + TILE - 1) / TILE);
        s.n_inject_tiles = static_cast<int32_t>((total + TILE - 1) / TILE);
        tmp[i] = s.n_move_tiles;
        tmp[ncase + i] = s.n_inject_tiles;
    }
    __syncthreads();
    case_scan(tt.move0, tmp, ncase);
    __syncthreads();
    case_scan(tt.inject0, tmp + ncase, ncase);
    __syncthreads();
    if (threadIdx.x == 0) {
        sc->total_move_tiles = tt.move0[ncase];
        sc->total_inject_tiles = tt.inject0[ncase];
        sc->init_mode = init_mode;
    }
    // k_inject adds the removed slots of each quarter of an inject tile.
    for (int i = threadIdx.x; i < tt.inject0[ncase]; i += blockDim.x)
        itile_dead[i] = 0;
    for (int i = threadIdx.x; i < ncase; i += blockDim.x) {
        st[i].move_tile0 = tt.move0[i];
        st[i].inject_tile0 = tt.inject0[i];
    }
}

__global__ void k_plan(const CaseDev *cases, CaseState *st, StepScratch *sc, TileTables tt,
                       int32_t *tmp, int32_t *itile_dead, uint64_t *cell_chain, int ncase,
                       int init_mode, int *err)
{
    plan_step(cases, st, sc, tt, tmp, itile_dead, cell_chain, ncase, init_mode, err);
}

// The impact branch of MoveParticles (Boundary.cpp:301-326) for slot q (global
// slot g): wall interaction drawn from the slot's stream, new velocity stored,
// post-impact position returned; the result is the drag impulse of the hit.
// Kept out of line: impacts are rare and the transcendental code would
// otherwise set the register budget of the whole move loop.
template <class T>
__device__ __noinline__ double wall_hit(const CaseDev &c, int64_t step, int64_t q, int64_t g,
                                        Slots<T> p, double x0, double y0, double dx, double dy,
                                        double t_hit, double nx, double ny, T &xn, T &yn)
{
    const double x_hit = x0 + t_hit * dx;
    const double y_hit = y0 + t_hit * dy;
    double v[3] = {static_cast<double>(p.vx[g]), static_cast<double>(p.vy[g]),
                   static_cast<double>(p.vz[g])};
    const double vx_in = v[0];
    dsmc_stream r;
    open_stream(r, c, DSMC_RNG_MOVE, step, static_cast<uint32_t>(q));
    wall_interaction(r, c, v, nx, ny);
    p.vx[g] = Store<T>::rn(v[0]);
    p.vy[g] = Store<T>::rn(v[1]);
    p.vz[g] = Store<T>::rn(v[2]);
    const double remaining = c.dt * (1.0 - t_hit);
    constexpr double epsilon = 1e-12;
    xn = round_out<T>(x_hit + remaining * v[0] + epsilon * nx, nx);
    yn = round_out<T>(y_hit + remaining * v[1] + epsilon * ny, ny);
    return c.drag_scale * (vx_in - v[0]);
}

// ---------------------------------------------------------------------------
// k_move: MoveParticles (Boundary.cpp:284-328) over the sorted slots, plus the
// per-slot bookkeeping of BoundaryConditions' removal and of Indexing.
// ---------------------------------------------------------------------------
// Four consecutive slots, 16-byte aligned (case bases and tiles are
// multiples of TILE).
__device__ __forceinline__ void load4(const float *p, float v[4])
{
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
}
__device__ __forceinline__ void load4(const double *p, double v[4])
{
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void store4(float *p, const float v[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double *p, const double v[4])
{
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void store4(uint32_t *p, const uint32_t v[4])
{
    *reinterpret_cast<uint4 *>(p) = make_uint4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void load4(const uint32_t *p, uint32_t v[4])
{
    const uint4 t = *reinterpret_cast<const uint4 *>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
}

// Classification of a moved slot: the key, the old and new global cells and
// whether it is removed, in range (same cell) or out of range (new cell).
struct MoveClass {
    uint32_t key;
    int32_t ocg;
    bool dead, out, in;
};

// Removal (Boundary.cpp:183-188) and the new cell of a slot, given its old
// cell `oc`, whether its new position lies outside the domain (`gone`) and
// otherwise its new cell `nc` (NO_CELL outside the grid).
__device__ __forceinline__ MoveClass classify_cells(const CaseDev &c, int32_t oc, bool gone,
                                                    int32_t nc, int *err)
{
    MoveClass m;
    m.dead = m.out = m.in = false;
    m.key = KEY_DEAD;
    m.ocg = oc < 0 ? NO_CELL : c.cbase + oc;
    if (gone) {
        m.dead = true;
    } else if (nc < 0) {
        // Inside the domain bounds but in no cell (rounding, NaN): the
        // reference aborts in ExchangeParticles, status 30.
        report_error(err, DSMC_ERR_EXCHANGE);
        m.dead = true;
    } else if (nc == oc) {
        m.key = static_cast<uint32_t>(c.cbase + nc) | KEY_IN;
        m.in = true;
    } else {
        m.key = static_cast<uint32_t>(c.cbase + nc);
        m.out = true;
    }
    if (m.dead)
        m.key = KEY_DEAD | (m.ocg == NO_CELL ? KEY_CELL : static_cast<uint32_t>(m.ocg));
    return m;
}

// Exact form: the cells by the reference's FP64 expressions.
template <class T>
__device__ __forceinline__ MoveClass classify(const CaseDev &c, double x0, double y0, T xn, T yn,
                                              int *err)
{
    const int32_t oc = cell_of(c, x0, y0);
    const bool gone = outside_domain(c, static_cast<double>(xn), static_cast<double>(yn));
    const int32_t nc = gone ? NO_CELL
                            : cell_of(c, static_cast<double>(xn), static_cast<double>(yn));
    return classify_cells(c, oc, gone, nc, err);
}

// Free flight of one slot, without the impact test and with estimated cell
// indices: false when the segment is near the box or a cell index is not
// certain from its estimate (the slot then takes the exact body), else the
// stored end point, the old cell, whether the end point left the domain and
// otherwise its new cell.  Same results as the exact body for every slot it
// accepts.
__device__ __forceinline__ bool free_flight(const CaseDev &c, double x0, double y0, double vx,
                                            double vy, double &xn, double &yn, int32_t &oc,
                                            bool &gone, int32_t &nc)
{
    xn = x0 + c.dt * vx;
    yn = y0 + c.dt * vy;
    if (near_box(c, x0, y0, xn, yn) || !cell_of_fast(c, x0, y0, oc))
        return false;
    gone = outside_domain(c, xn, yn);
    nc = NO_CELL;
    return gone || cell_of_fast(c, xn, yn, nc);
}

// FP32 slots: the end point is rounded from the FP64 sum as in the exact
// body; the box, domain and cell tests run on floats (exact or conservative,
// as their helpers state), with the FP64 estimate as a second chance for a
// cell the float estimate leaves open.  A certain float estimate also decides
// the removal test: its floors are those of (x - X1) / DX and (y - Y1) / DY,
// at least the window's margin (far above the ulps between X2 and X1 + NX DX)
// away from an integer, so the position lies strictly inside the domain
// exactly when that cell is in the grid.  Only an open estimate takes the
// exact domain test.
__device__ __forceinline__ bool free_flight(const CaseDev &c, float x0, float y0, float vx,
                                            float vy, float &xn, float &yn, int32_t &oc,
                                            bool &gone, int32_t &nc)
{
    xn = __double2float_rn(static_cast<double>(x0) + c.dt * static_cast<double>(vx));
    yn = __double2float_rn(static_cast<double>(y0) + c.dt * static_cast<double>(vy));
    const bool near = near_box_f(c, x0, y0, xn, yn);
    bool ok_o = cell_of_fast_f(c, x0, y0, oc);
    bool ok_n = cell_of_fast_f(c, xn, yn, nc);
    gone = nc == NO_CELL;
    if (!ok_o)
        ok_o = cell_of_fast(c, static_cast<double>(x0), static_cast<double>(y0), oc);
    if (!ok_n) {
        gone = outside_domain_f(c, xn, yn);
        nc = NO_CELL;
        ok_n = gone || cell_of_fast(c, static_cast<double>(xn), static_cast<double>(yn), nc);
    }
    return !near & ok_o & ok_n;
}

// Stores the key of a classified slot and moves the cell counters: every
// cell starts the step with its old count as its in-range count, so only
// slots that leave it touch a counter.
__device__ __forceinline__ void commit_class(const MoveClass &m, uint32_t *key, int64_t g,
                                             Cells cells)
{
    key[g] = m.key;
    if ((m.dead || m.out) && m.ocg != NO_CELL)
        atomicSub(cells.n_in + m.ocg, 1);
    if (m.out)
        atomicAdd(cells.n_o + (m.key & KEY_CELL), 1);
}

// The full MoveParticles body (Boundary.cpp:284-328) for one slot: impact
// test, wall interaction, FP32 placement outside the box, exact cell index.
// Runs in its own kernel, so its register demand stays out of k_move.
template <class T>
__device__ __forceinline__ MoveClass move_near_box(const CaseDev &c, int64_t step, int64_t q,
                                                int64_t g, Slots<T> p, uint32_t *key, Cells cells,
                                                double &impulse, int &n_hit, int *err)
{
    const double x0 = static_cast<double>(p.x[g]);
    const double y0 = static_cast<double>(p.y[g]);
    const double dx = c.dt * static_cast<double>(p.vx[g]);
    const double dy = c.dt * static_cast<double>(p.vy[g]);
    const double xe = x0 + dx;
    const double ye = y0 + dy;
    double t_hit = 0.0, hnx = 0.0, hny = 0.0;
    T xn, yn;
    if (may_hit_box(c, x0, y0, xe, ye) && intersect_box(c, x0, y0, dx, dy, t_hit, hnx, hny)) {
        impulse += wall_hit<T>(c, step, q, g, p, x0, y0, dx, dy, t_hit, hnx, hny, xn, yn);
        n_hit++;
    } else {
        xn = Store<T>::rn(xe);
        yn = Store<T>::rn(ye);
        keep_outside<T>(c, xn, yn);
    }
    p.x[g] = xn;
    p.y[g] = yn;
    const MoveClass m = classify<T>(c, x0, y0, xn, yn, err);
    commit_class(m, key, g, cells);
    return m;
}

// Slot mapping of a move tile: iteration k of thread t handles slot
// tile + k * TILE_THREADS + t, so every load and store of a warp is one
// contiguous 128-byte (FP32) access, and ranks in slot order come from warp
// ballots: (iteration, warp) pairs are in slot order.
constexpr int MOVE_WARPS = TILE_THREADS / 32;
static_assert(TILE_VEC * MOVE_WARPS == 32, "one warp scans the (iteration, warp) counts");

// Tiles are staged in shared memory by bulk asynchronous copies, MOVE
// stages deep, so the loads of the next tiles of a CTA are in flight while it
// moves the current one.  Tiles are dealt to CTAs statically (no tile waits on
// another, so no ticket order is needed).  k_move moves every slot that
// free_flight accepts and queues the other few for k_move_near, which runs
// the exact body; both give the exact body's result for every slot.
template <class T> struct MoveStage {
    T v[4][TILE]; // x, y, vx, vy
};
// Pipeline depths (build-time settings, -DDSMC_MOVE_STAGES=... etc.; the
// defaults were chosen by measurement on B200).
#ifndef DSMC_MOVE_STAGES
#define DSMC_MOVE_STAGES 3
#endif
#ifndef DSMC_SCATTER_STAGES
#define DSMC_SCATTER_STAGES 3
#endif
#ifndef DSMC_SAMPLE_STAGES
#define DSMC_SAMPLE_STAGES 1
#endif
#ifndef DSMC_SAMPLE_UNROLL // unroll of k_sample's per-cell loop
#define DSMC_SAMPLE_UNROLL 8
#endif
#ifndef DSMC_MOVE_MIN_BLOCKS // CTAs per SM k_move is compiled for (register budget)
#define DSMC_MOVE_MIN_BLOCKS 4
#endif
// k_move and k_scatter need two stages at least: a stage's tile is rewritten
// by thread 0 after the tile's barrier and read by the others one full
// iteration later, which another barrier separates only when the next tile
// uses another stage.  k_sample adds that barrier when it runs one stage.
static_assert(DSMC_MOVE_STAGES >= 2 && DSMC_SCATTER_STAGES >= 2 && DSMC_SAMPLE_STAGES >= 1,
              "the tile pipelines need two or more stages");
template <class T> __host__ __device__ constexpr int move_stages()
{
    return sizeof(T) == 4 ? DSMC_MOVE_STAGES : 2;
}
template <class T> __host__ __device__ constexpr size_t move_smem()
{
    return sizeof(MoveStage<T>) * move_stages<T>();
}

// The move tiles of block bx of nbx (tiles bx, bx + nbx, ...); smem_raw holds
// S * sizeof(MoveStage<T>) bytes.  False when a staged copy never completed (reported;
// the block's copies in flight were waited for, its barriers stay live).
template <class T, int S = move_stages<T>()>
__device__ __forceinline__ bool
    move_tiles(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
               Slots<T> p, uint32_t *__restrict__ key, Cells cells,
               int32_t *__restrict__ tile_in, int32_t *__restrict__ tile_dead,
               uint32_t *__restrict__ obuf, uint32_t *__restrict__ near_list, int ncase, int *err,
               unsigned char *smem_raw, int bx, int nbx)
{
    static_assert(TILE == 1024, "near_list packs the slot in tile into 10 bits");
    static_assert(S >= 2, "see the stage rule above");
    constexpr int NB = 3; // ballot buffers: a tile's are read until the next tile's barrier
    MoveStage<T> *stage = reinterpret_cast<MoveStage<T> *>(smem_raw);
    __shared__ uint64_t bar[S];
    __shared__ CaseDev s_case; // constants of the current tile's case
    __shared__ unsigned s_dead[NB][32], s_out[NB][32]; // per (iteration, warp)
    __shared__ unsigned s_opre[NB][32];                // exclusive prefix of s_out
    __shared__ uint32_t s_obase[NB];
    __shared__ int s_nnear[NB]; // slots of the tile queued for k_move_near
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const int total = sc->total_move_tiles;

    // Thread 0 only: the copies of tile t into stage sidx.
    auto issue = [&](int t, int sidx) {
        const int ci = case_of(tt.move0, ncase, t);
        const int64_t g0 = cases[ci].pbase + static_cast<int64_t>(t - tt.move0[ci]) * TILE;
        constexpr uint32_t vb = TILE * sizeof(T);
        mbar_arrive_expect_tx(&bar[sidx], 4 * vb);
        bulk_g2s(stage[sidx].v[0], p.x + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[1], p.y + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[2], p.vx + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[3], p.vy + g0, vb, &bar[sidx]);
    };
    // All threads: the out-of-range list entries of the tile at global slot
    // gt whose ballots are in buffer nb (counted by warp 0 after its barrier).
    auto append = [&](int nb, int64_t gt) {
        for (int k = 0; k < TILE_VEC; ++k) {
            const int i = k * MOVE_WARPS + warp;
            const unsigned bo = s_out[nb][i];
            if ((bo >> lane) & 1u)
                obuf[s_obase[nb] + s_opre[nb][i] + __popc(bo & lanes_below)] =
                    static_cast<uint32_t>(gt + k * TILE_THREADS + threadIdx.x);
        }
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i)
            mbar_init(&bar[i], 1);
        fence_mbar_init();
        for (int i = 0; i < S; ++i)
            if (bx + i * nbx < total)
                issue(bx + i * nbx, i);
    }
    if (threadIdx.x < NB)
        s_nnear[threadIdx.x] = 0;
    __syncthreads();

    int cur_case = -1;
    int64_t prev_gt = 0;
    int it = 0;
    for (;; ++it) {
        const int t = bx + it * nbx;
        if (t >= total)
            break;
        const int sidx = it % S;
        const int nb = it % NB;
        const int ci = case_of(tt.move0, ncase, t);
        if (ci != cur_case) {
            // No thread reads s_case between a tile's barrier and the next
            // tile's top, so the copy needs only the barrier after it.
            const uint32_t *src = reinterpret_cast<const uint32_t *>(cases + ci);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s_case);
            for (int w = threadIdx.x; w < static_cast<int>(sizeof(CaseDev) / 4); w += TILE_THREADS)
                dst[w] = src[w];
            __syncthreads();
            cur_case = ci;
        }
        const CaseDev &c = s_case;
        const bool ok = mbar_wait(&bar[sidx], static_cast<uint32_t>((it / S) & 1));
        const int local_tile = t - tt.move0[ci];
        const int64_t tile0 = static_cast<int64_t>(local_tile) * TILE;
        const int64_t left = st[ci].n_old - tile0;
        const int n_here = ok ? (left < TILE ? static_cast<int>(left) : TILE) : 0;
        const int64_t gt = c.pbase + tile0;
        T *px = p.x + gt;
        T *py = p.y + gt;
        uint32_t *pkey = key + gt;
        const MoveStage<T> &sg = stage[sidx];

        unsigned near = 0; // bit k: the slot of iteration k takes the exact body
#pragma unroll
        for (int k = 0; k < TILE_VEC; ++k) {
            const int e = k * TILE_THREADS + threadIdx.x;
            MoveClass m;
            m.dead = m.out = m.in = false;
            if (e < n_here) {
                T xn, yn;
                int32_t oc, nc;
                bool gone;
                if (free_flight(c, sg.v[0][e], sg.v[1][e], sg.v[2][e], sg.v[3][e], xn, yn, oc,
                                gone, nc)) {
                    px[e] = xn;
                    py[e] = yn;
                    m = classify_cells(c, oc, gone, nc, err);
                    commit_class(m, pkey, e, cells);
                } else {
                    near |= 1u << k;
                }
            }
            const unsigned bd = __ballot_sync(0xffffffffu, m.dead);
            const unsigned bo = __ballot_sync(0xffffffffu, m.out);
            if (lane == 0) {
                s_dead[nb][k * MOVE_WARPS + warp] = bd;
                s_out[nb][k * MOVE_WARPS + warp] = bo;
            }
        }
        // Slots for the exact body go to k_move_near's queue as (tile, slot
        // in tile); their ballots, counts and list entries are added there.
        const unsigned nq = __ballot_sync(0xffffffffu, near != 0);
        if (nq) {
            int n_mine = __popc(near);
            if (n_mine)
                atomicAdd(&s_nnear[nb], n_mine);
            int incl = n_mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += v;
            }
            uint32_t qbase = 0;
            if (lane == 31)
                qbase = atomicAdd(&sc->near_count, static_cast<uint32_t>(incl));
            qbase = __shfl_sync(0xffffffffu, qbase, 31) + static_cast<uint32_t>(incl - n_mine);
            for (int k = 0; k < TILE_VEC; ++k)
                if ((near >> k) & 1u)
                    near_list[qbase++] = (static_cast<uint32_t>(t) << 10) |
                                         static_cast<uint32_t>(k * TILE_THREADS + threadIdx.x);
        }
        // The one barrier of the tile: the stage is consumed, this tile's
        // ballots are complete and the previous tile's list base is visible.
        if (__syncthreads_or(!ok)) {
            // A copy never completed (nothing of this tile was written).
            if (threadIdx.x == 0) {
                report_error(err, DSMC_ERR_TIMEOUT);
                for (int j = it; j < it + S; ++j)
                    if (bx + j * nbx < total)
                        mbar_wait(&bar[j % S], static_cast<uint32_t>((j / S) & 1));
            }
            return false;
        }
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            const int tn = t + S * nbx;
            if (tn < total)
                issue(tn, sidx);
        }
        if (warp == 0) {
            // Lane i holds the counts of (iteration, warp) pair i; pairs are
            // in slot order, so an exclusive scan gives list ranks in slot
            // order.  Removed slots are only counted here: their ranks come
            // from k_dead_scan and k_holes, so no tile waits on another.
            const unsigned o = __popc(s_out[nb][lane]);
            unsigned oi = o;
#pragma unroll
            for (int sft = 1; sft < 32; sft <<= 1) {
                const unsigned b = __shfl_up_sync(0xffffffffu, oi, sft);
                if (lane >= sft)
                    oi += b;
            }
            s_opre[nb][lane] = oi - o;
            const unsigned out_tile = __shfl_sync(0xffffffffu, oi, 31);
            const unsigned dead_tile =
                static_cast<unsigned>(warp_sum_u64(__popc(s_dead[nb][lane])));
            if (lane == 0) {
                // Every slot this kernel moved is removed, out of range or in
                // range; k_move_near counts the queued ones.
                const int in_tile = n_here - s_nnear[nb] - static_cast<int>(dead_tile) -
                                    static_cast<int>(out_tile);
                s_nnear[nb] = 0; // rewritten for the tile NB iterations on
                tile_in[t] = static_cast<int32_t>(in_tile);
                tile_dead[t] = static_cast<int32_t>(dead_tile);
                s_obase[nb] = out_tile ? atomicAdd(&sc->obuf_count, out_tile) : 0u;
            }
        }
        // The previous tile's list entries (its base was set before this
        // tile's barrier).
        if (it > 0)
            append((it + NB - 1) % NB, prev_gt);
        prev_gt = gt;
    }
    if (it > 0) {
        __syncthreads();
        append((it + NB - 1) % NB, prev_gt);
    }
    // Every copy issued was consumed: the barriers can be retired.
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < S; ++i)
            mbar_inval(&bar[i]);
    return true;
}

template <class T>
__global__ void __launch_bounds__(TILE_THREADS, DSMC_MOVE_MIN_BLOCKS)
    k_move(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
           Slots<T> p, uint32_t *__restrict__ key, Cells cells, int32_t *__restrict__ tile_in,
           int32_t *__restrict__ tile_dead, uint32_t *__restrict__ obuf,
           uint32_t *__restrict__ near_list, int ncase, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (void)move_tiles<T>(cases, st, sc, tt, p, key, cells, tile_in, tile_dead, obuf, near_list,
                        ncase, err, smem_raw, blockIdx.x, gridDim.x);
}

// k_move_near: the exact MoveParticles body for the slots k_move queued
// (near the box, or a cell index not certain from its estimate), then their
// share of the tile counts, the out-of-range list and the drag diagnostics.
template <class T>
__device__ __forceinline__ void
    move_near(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
              Slots<T> p, uint32_t *__restrict__ key, Cells cells, int32_t *__restrict__ tile_in,
              int32_t *__restrict__ tile_dead, uint32_t *__restrict__ obuf,
              const uint32_t *__restrict__ near_list, int ncase, int *err, int bx, int nbx)
{
    const uint32_t n = sc->near_count;
    for (uint32_t i = bx * blockDim.x + threadIdx.x; i < n; i += nbx * blockDim.x) {
        const uint32_t w = near_list[i];
        const int t = static_cast<int>(w >> 10);
        const int e = static_cast<int>(w & 1023u);
        const int ci = case_of(tt.move0, ncase, t);
        const CaseDev &c = cases[ci];
        const int64_t q = static_cast<int64_t>(t - tt.move0[ci]) * TILE + e;
        double impulse = 0.0;
        int n_hit = 0;
        const MoveClass m = move_near_box<T>(c, st[ci].step, q, c.pbase + q, p, key, cells,
                                             impulse, n_hit, err);
        if (m.in)
            atomicAdd(tile_in + t, 1);
        if (m.dead)
            atomicAdd(tile_dead + t, 1);
        if (m.out)
            obuf[atomicAdd(&sc->obuf_count, 1u)] = static_cast<uint32_t>(c.pbase + q);
        if (n_hit) {
            atomicAdd(&st[ci].drag_impulse, impulse);
            atomicAdd(&st[ci].drag_count, static_cast<unsigned long long>(n_hit));
            if (st[ci].step > c.first_sampling_step) { // the DragSamplingTime window
                atomicAdd(&st[ci].drag_impulse_window, impulse);
                atomicAdd(&st[ci].drag_count_window, static_cast<unsigned long long>(n_hit));
            }
        }
    }
}

template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_move_near(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc,
                TileTables tt, Slots<T> p, uint32_t *__restrict__ key, Cells cells,
                int32_t *__restrict__ tile_in, int32_t *__restrict__ tile_dead,
                uint32_t *__restrict__ obuf, const uint32_t *__restrict__ near_list, int ncase,
                int *err)
{
    move_near<T>(cases, st, sc, tt, p, key, cells, tile_in, tile_dead, obuf, near_list, ncase,
                 err, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_inject: GenerateNewParticles (Boundary.cpp:60-92) for every strip of every
// case, written after the case's n_old slots.  In init mode the single strip
// is the cold-start fill of InitialConditions (Initialization.cpp:302-310),
// without the pre-move, and the removal predicate is InsideBox
// (RemoveParticlesInsideBox, Geometry.cpp:231-247).
// ---------------------------------------------------------------------------
// Inject units are dealt by ticket: any number of CTAs of TILE_THREADS.
template <class T>
__device__ __forceinline__ void
    inject_units(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
                 Slots<T> p, uint32_t *__restrict__ key, Cells cells,
                 int32_t *__restrict__ itile_dead, uint32_t *__restrict__ obuf, int ncase,
                 int *err)
{
    __shared__ int s_unit;
    const int init_mode = sc->init_mode;
    const int lane = threadIdx.x & 31;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_unit = static_cast<int>(atomicAdd(&sc->inject_ticket, 1u));
        __syncthreads();
        // A unit is a quarter of an inject tile, one slot per thread, so the
        // long per-particle chain (stream seek, five draws) runs once per
        // thread.
        const int u = s_unit;
        if (u >= sc->total_inject_tiles * TILE_VEC)
            return;
        const int t = u / TILE_VEC;
        const int ci = case_of(tt.inject0, ncase, t);
        const CaseDev &c = cases[ci];
        const CaseState &s = st[ci];
        const int64_t n_inj = s.inj_off[5];
        const int local_tile = t - tt.inject0[ci];
        const int64_t j = static_cast<int64_t>(local_tile) * TILE +
                          (u % TILE_VEC) * TILE_THREADS + threadIdx.x;
        uint32_t kw = KEY_DEAD | KEY_CELL;
        int n_dead = 0;
        if (j < n_inj) {
            int strip = 0;
            while (strip < 4 && j >= s.inj_off[strip + 1])
                ++strip;
            const int64_t js = j - s.inj_off[strip];
            dsmc_stream r;
            if (init_mode)
                open_stream(r, c, DSMC_RNG_INIT, 0, 0);
            else
                open_stream(r, c, DSMC_RNG_INJECT, s.step, static_cast<uint32_t>(strip));
            dsmc_stream_seek(&r, static_cast<uint64_t>(s.inj_c0[strip]) + 8ull * js);
            const double *b = c.strip[strip];
            double x, y, vx, vy, vz;
            new_particle(r, b, c.ux_free, c.uy_free, c.rt_free, x, y, vx, vy, vz);
            if (!init_mode) {
                x += c.dt * vx;
                y += c.dt * vy;
            }
            T xs = Store<T>::rn(x), ys = Store<T>::rn(y);
            if (init_mode) {
                // The fill box ends at LocalX2 = X1 + NX DX, which can exceed
                // X2 by an ulp; a float rounded up to X2 itself would then
                // index cell NX.  Keep FP32 positions below both.
                xs = clamp_into<T>(xs, b[0], fmin(b[2], c.x2));
                ys = clamp_into<T>(ys, b[1], fmin(b[3], c.y2));
            }
            const int64_t q = s.n_old + j;
            const int64_t g = c.pbase + q;
            p.x[g] = xs;
            p.y[g] = ys;
            p.vx[g] = Store<T>::rn(vx);
            p.vy[g] = Store<T>::rn(vy);
            p.vz[g] = Store<T>::rn(vz);
            const double xd = static_cast<double>(xs), yd = static_cast<double>(ys);
            const bool dead = init_mode ? inside_box(c, xd, yd) : outside_domain(c, xd, yd);
            if (dead) {
                n_dead = 1;
            } else {
                const int32_t nc = cell_of(c, xd, yd);
                if (nc < 0) {
                    report_error(err, DSMC_ERR_EXCHANGE);
                    n_dead = 1;
                } else {
                    kw = static_cast<uint32_t>(c.cbase + nc);
                }
            }
            key[g] = kw;
        }
        const bool alive = !(kw & KEY_DEAD);
        const int32_t cg = static_cast<int32_t>(kw & KEY_CELL);
        warp_aggregated_inc(cells.n_o, cg, alive);
        const unsigned m = __ballot_sync(0xffffffffu, alive);
        if (m) {
            uint32_t base = 0;
            if (lane == __ffs(m) - 1)
                base = atomicAdd(&sc->obuf_count, static_cast<uint32_t>(__popc(m)));
            base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
            if (alive)
                obuf[base + __popc(m & ((1u << lane) - 1u))] =
                    static_cast<uint32_t>(c.pbase + s.n_old + j);
        }
        int dead_total;
        (void)block_exclusive<int>(n_dead, dead_total);
        if (threadIdx.x == 0 && dead_total > 0)
            atomicAdd(itile_dead + t, dead_total);
    }
}

template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_inject(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
             Slots<T> p, uint32_t *__restrict__ key, Cells cells,
             int32_t *__restrict__ itile_dead, uint32_t *__restrict__ obuf, int ncase, int *err)
{
    inject_units<T>(cases, st, sc, tt, p, key, cells, itile_dead, obuf, ncase, err);
}

// ---------------------------------------------------------------------------
// Threads of a CTA of the per-case scans (also k_warm_scan).
constexpr int SCAN_THREADS = 1024;

// The tile-count scans (k_dead_scan, k_tile_scan): the exclusive prefix of a
// case's sequence of per-tile counts, cut into chunks of SCAN_CHUNK counts,
// one CTA each, all at once.  A CTA first sums every count before its chunk
// (read directly: no CTA waits for another), then scans its chunk, SCAN_VEC
// consecutive counts per thread.
constexpr int SCAN_VEC = 4;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_VEC;

// Count i of the sequence a[0, na) followed by b.
__device__ __forceinline__ int32_t seq_count(const int32_t *a, int na, const int32_t *b, int i)
{
    return i < na ? a[i] : b[i - na];
}

// Sum of counts [0, c0) of the sequence, in every thread.
template <int NT = SCAN_THREADS>
__device__ __forceinline__ int32_t seq_before(const int32_t *a, int na, const int32_t *b, int c0)
{
    int32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0; // four loads in flight per round
    int i = threadIdx.x;
    for (; i + 3 * NT < c0; i += 4 * NT) {
        s0 += seq_count(a, na, b, i);
        s1 += seq_count(a, na, b, i + NT);
        s2 += seq_count(a, na, b, i + 2 * NT);
        s3 += seq_count(a, na, b, i + 3 * NT);
    }
    for (; i < c0; i += NT)
        s0 += seq_count(a, na, b, i);
    int32_t tot;
    (void)block_exclusive<int32_t, NT>(s0 + s1 + s2 + s3, tot);
    return tot;
}

// Exclusive prefixes of chunk [c0, c0 + NT * SCAN_VEC) of the sequence of
// length n (from `carry`) into oa / ob; returns the prefix of each of this
// thread's counts in pre[] and carry plus the chunk's total.
template <int NT = SCAN_THREADS>
__device__ __forceinline__ int32_t seq_chunk(const int32_t *a, int32_t *oa, int na,
                                             const int32_t *b, int32_t *ob, int n, int c0,
                                             int32_t carry, int32_t pre[SCAN_VEC])
{
    const int i0 = c0 + static_cast<int>(threadIdx.x) * SCAN_VEC;
    int32_t v[SCAN_VEC];
    int32_t sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_VEC; ++k) {
        v[k] = i0 + k < n ? seq_count(a, na, b, i0 + k) : 0;
        sum += v[k];
    }
    int32_t tot;
    int32_t run = carry + block_exclusive<int32_t, NT>(sum, tot);
#pragma unroll
    for (int k = 0; k < SCAN_VEC; ++k) {
        const int i = i0 + k;
        pre[k] = run;
        if (i < n) {
            if (i < na)
                oa[i] = run;
            else
                ob[i - na] = run;
        }
        run += v[k];
    }
    return carry + tot;
}

// k_dead_scan: grid (chunks, cases).  Exclusive prefix of the removed-slot
// counts of a case's move tiles, then of its inject tiles (their ranks
// continue the count, in slot order); sets dead_old and dead_total.
// dead_scan_chunk: chunk `chunk` of case `ci` by a CTA of NT threads.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void dead_scan_chunk(CaseState *st, const int32_t *tile_dead,
                                                int32_t *tile_dprefix, const int32_t *itile_dead,
                                                int32_t *itile_dprefix, int chunk, int ci)
{
    constexpr int CHUNK = NT * SCAN_VEC;
    CaseState &s = st[ci];
    const int na = s.n_move_tiles;
    const int n = na + s.n_inject_tiles;
    const int c0 = chunk * CHUNK;
    if (c0 >= n)
        return; // uniform over the CTA
    const int32_t *a = tile_dead + s.move_tile0, *b = itile_dead + s.inject_tile0;
    const int32_t carry = seq_before<NT>(a, na, b, c0);
    int32_t pre[SCAN_VEC];
    const int32_t total = seq_chunk<NT>(a, tile_dprefix + s.move_tile0, na, b,
                                        itile_dprefix + s.inject_tile0, n, c0, carry, pre);
    const int i0 = c0 + static_cast<int>(threadIdx.x) * SCAN_VEC;
#pragma unroll
    for (int k = 0; k < SCAN_VEC; ++k)
        if (i0 + k == na && na < n) // the first inject tile: all move tiles before it
            s.dead_old = pre[k];
    if (c0 + CHUNK >= n && threadIdx.x == 0) { // the last chunk
        s.dead_total = total;
        if (na == n)
            s.dead_old = total;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS)
    k_dead_scan(CaseState *st, const int32_t *tile_dead, int32_t *tile_dprefix,
                const int32_t *itile_dead, int32_t *itile_dprefix)
{
    dead_scan_chunk<SCAN_THREADS>(st, tile_dead, tile_dprefix, itile_dead, itile_dprefix,
                                  blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Survivors, holes and the tail of every case, once the removed-slot list is
// complete (run by the last CTA of k_holes).
// ---------------------------------------------------------------------------
__device__ void plan_tail(const CaseDev *cases, CaseState *st, StepScratch *sc, TileTables tt,
                          const int32_t *hole_pos, int32_t *tmp, uint64_t *tail_chain, int ncase)
{
    // One warp per case: a 33-way search (32 probes a round) for the number
    // of removed slots below K (the holes); the list is in slot order.  The
    // list was written by other CTAs of this kernel: read through L2.
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i < ncase; i += nwarps) {
        CaseState &s = st[i];
        const int64_t keep = s.n_total - s.dead_total; // dead_total: k_dead_scan
        const int32_t *hp = hole_pos + cases[i].pbase;
        int64_t lo = 0, hi = s.dead_total; // first index with hp >= keep is in [lo, hi]
        while (lo < hi) {
            const int64_t span = hi - lo;
            const int64_t idx = lo + ((lane + 1) * span) / 33; // < hi
            const bool below = __ldcg(hp + idx) < keep;
            const unsigned bl = __ballot_sync(0xffffffffu, below);
            const int j = __popc(bl); // probes 0..j-1 are below (monotone)
            const int64_t lo_n = j > 0 ? __shfl_sync(0xffffffffu, idx, j - 1) + 1 : lo;
            const int64_t hi_n = j < 32 ? __shfl_sync(0xffffffffu, idx, j < 32 ? j : 31) : hi;
            lo = lo_n;
            hi = hi_n;
        }
        if (lane == 0) {
            s.n_keep = keep;
            s.n_holes = lo;
            s.n_tail_tiles = static_cast<int32_t>((s.n_total - keep + TILE - 1) / TILE);
            tmp[i] = s.n_tail_tiles;
            tmp[ncase + i] = static_cast<int32_t>((keep + TILE - 1) / TILE);
        }
    }
    __syncthreads();
    case_scan(tt.tail0, tmp, ncase);
    __syncthreads();
    case_scan(tt.scatter0, tmp + ncase, ncase);
    __syncthreads();
    if (threadIdx.x == 0)
        sc->total_tail_tiles = tt.tail0[ncase];
    for (int i = threadIdx.x; i < ncase; i += blockDim.x)
        st[i].tail_tile0 = tt.tail0[i];
    // The look-back status words k_tail is about to use.
    for (int i = threadIdx.x; i < tt.tail0[ncase]; i += blockDim.x)
        tail_chain[i] = 0ull;
}

// ---------------------------------------------------------------------------
// k_holes: the removed-slot list in slot order (hole_pos, and the old cell of
// each removed slot in hole_oc), from the tiles that have removed slots.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void
    holes_blocks(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
                 const uint32_t *__restrict__ key, const int32_t *tile_dead,
                 const int32_t *tile_dprefix, const int32_t *itile_dead,
                 const int32_t *itile_dprefix, int32_t *__restrict__ hole_pos,
                 int32_t *__restrict__ hole_oc, int32_t *tmp, uint64_t *tail_chain, int ncase,
                 int bx, int nbx)
{
    __shared__ bool s_last;
    __shared__ int s_list[TILE_THREADS];
    const int n_move = sc->total_move_tiles;
    const int total = n_move + sc->total_inject_tiles;
    for (int T0 = bx; T0 < total; T0 += nbx * TILE_THREADS) {
        // The counts of this CTA's next TILE_THREADS tiles are read at once
        // and the tiles with removed slots listed: most tiles have none.
        const int Tm = T0 + static_cast<int>(threadIdx.x) * nbx;
        int cnt = 0;
        if (Tm < total)
            cnt = Tm < n_move ? tile_dead[Tm] : itile_dead[Tm - n_move];
        int n_list;
        const int pos = block_exclusive<int>(cnt > 0 ? 1 : 0, n_list);
        if (cnt > 0)
            s_list[pos] = Tm;
        __syncthreads();
        for (int li = 0; li < n_list; ++li) {
            const int T = s_list[li];
            const bool moved = T < n_move;
            const int t = moved ? T : T - n_move;
            const int ci = case_of(moved ? tt.move0 : tt.inject0, ncase, t);
            const CaseDev &c = cases[ci];
            const CaseState &s = st[ci];
            const int local_tile = t - (moved ? tt.move0[ci] : tt.inject0[ci]);
            const int64_t first = moved ? 0 : s.n_old;
            const int64_t end = moved ? s.n_old : s.n_total;
            const int64_t q0 =
                first + static_cast<int64_t>(local_tile) * TILE + threadIdx.x * TILE_VEC;
            uint32_t keys[TILE_VEC];
            int n_dead = 0;
#pragma unroll
            for (int k = 0; k < TILE_VEC; ++k) {
                keys[k] = q0 + k < end ? key[c.pbase + q0 + k] : 0u;
                n_dead += (keys[k] & KEY_DEAD) ? 1 : 0;
            }
            int tot;
            int64_t rank = (moved ? tile_dprefix[t] : itile_dprefix[t]) +
                           block_exclusive<int>(n_dead, tot);
#pragma unroll
            for (int k = 0; k < TILE_VEC; ++k) {
                if (!(keys[k] & KEY_DEAD))
                    continue;
                const uint32_t oc = keys[k] & KEY_CELL;
                hole_pos[c.pbase + rank] = static_cast<int32_t>(q0 + k);
                hole_oc[c.pbase + rank] = oc == KEY_CELL ? NO_CELL : static_cast<int32_t>(oc);
                ++rank;
            }
        }
        __syncthreads(); // s_list is rewritten by the next group
    }
    // The last CTA to finish plans the tail: every hole is listed by then.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        s_last = atomicAdd(&sc->holes_done, 1u) == static_cast<unsigned>(nbx - 1);
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    plan_tail(cases, st, sc, tt, hole_pos, tmp, tail_chain, ncase);
}

__global__ void __launch_bounds__(TILE_THREADS)
    k_holes(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
            const uint32_t *__restrict__ key, const int32_t *tile_dead,
            const int32_t *tile_dprefix, const int32_t *itile_dead, const int32_t *itile_dprefix,
            int32_t *__restrict__ hole_pos, int32_t *__restrict__ hole_oc, int32_t *tmp,
            uint64_t *tail_chain, int ncase)
{
    holes_blocks(cases, st, sc, tt, key, tile_dead, tile_dprefix, itile_dead, itile_dprefix,
                 hole_pos, hole_oc, tmp, tail_chain, ncase, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_tail: the swap-with-last removal (Boundary.cpp:181-202) as a permutation.
// The r-th surviving slot of the tail [K, n_total), counted from its end,
// moves into the r-th hole.
// ---------------------------------------------------------------------------
// Tail tiles are dealt by ticket: any number of CTAs of TILE_THREADS.
template <class T>
__device__ __forceinline__ void
    tail_tiles(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
               Slots<T> p, uint32_t *__restrict__ key, Cells cells,
               int32_t *__restrict__ tile_in, uint64_t *lb, const int32_t *__restrict__ hole_pos,
               const int32_t *__restrict__ hole_oc, uint32_t *__restrict__ obuf, int ncase,
               int *err)
{
    __shared__ int s_tile;
    __shared__ uint64_t s_excl;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_tile = static_cast<int>(atomicAdd(&sc->tail_ticket, 1u));
        __syncthreads();
        const int t = s_tile;
        if (t >= sc->total_tail_tiles)
            return;
        const int ci = case_of(tt.tail0, ncase, t);
        const CaseDev &c = cases[ci];
        const CaseState &s = st[ci];
        const int local_tile = t - tt.tail0[ci];
        const int64_t q0 = s.n_keep + static_cast<int64_t>(local_tile) * TILE +
                           threadIdx.x * TILE_VEC;
        uint32_t keys[TILE_VEC];
        int n_alive = 0;
#pragma unroll
        for (int k = 0; k < TILE_VEC; ++k) {
            keys[k] = KEY_DEAD;
            if (q0 + k < s.n_total)
                keys[k] = key[c.pbase + q0 + k];
            n_alive += (keys[k] & KEY_DEAD) ? 0 : 1;
        }
        int alive_total;
        const int alive_excl = block_exclusive<int>(n_alive, alive_total);
        if (threadIdx.x < 32) {
            const uint64_t excl = lookback_warp(lb, t, t - local_tile, alive_total, err);
            if (threadIdx.x == 0)
                s_excl = excl;
        }
        __syncthreads();
        int64_t r = static_cast<int64_t>(s_excl) + alive_excl;
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < TILE_VEC; ++k) {
            const bool alive = !(keys[k] & KEY_DEAD);
            int64_t m = -1;
            if (alive) {
                m = s.n_holes - 1 - r;
                ++r;
                if (m < 0)
                    report_error(err, DSMC_ERR_STATE);
            }
            const bool go = alive && m >= 0;
            int64_t h = 0;
            int32_t hoc = NO_CELL;
            if (go) {
                h = hole_pos[c.pbase + m];
                hoc = hole_oc[c.pbase + m];
            }
            const int32_t cg = static_cast<int32_t>(keys[k] & KEY_CELL);
            const bool was_in = (keys[k] & KEY_IN) != 0;
            const bool now_in = go && hoc == cg;
            const bool listed = go && !now_in;
            // One increment of the list counter per warp.
            const unsigned lm = __ballot_sync(0xffffffffu, listed);
            uint32_t lbase = 0;
            if (lm) {
                const int lead = __ffs(lm) - 1;
                if (lane == lead)
                    lbase = atomicAdd(&sc->obuf_count, static_cast<uint32_t>(__popc(lm)));
                lbase = __shfl_sync(0xffffffffu, lbase, lead);
            }
            if (!go)
                continue;
            if (was_in && !now_in) {
                atomicSub(cells.n_in + cg, 1);
                atomicAdd(cells.n_o + cg, 1);
            } else if (!was_in && now_in) {
                atomicSub(cells.n_o + cg, 1);
                atomicAdd(cells.n_in + cg, 1);
            }
            if (now_in)
                atomicAdd(tile_in + s.move_tile0 + static_cast<int>(h / TILE), 1);
            else
                obuf[lbase + __popc(lm & ((1u << lane) - 1u))] =
                    static_cast<uint32_t>(c.pbase + h);
            const int64_t gs = c.pbase + q0 + k, gd = c.pbase + h;
            p.x[gd] = p.x[gs];
            p.y[gd] = p.y[gs];
            p.vx[gd] = p.vx[gs];
            p.vy[gd] = p.vy[gs];
            p.vz[gd] = p.vz[gs];
            key[gd] = static_cast<uint32_t>(cg) | (now_in ? KEY_IN : 0u);
        }
    }
}

template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_tail(const CaseDev *__restrict__ cases, CaseState *st, StepScratch *sc, TileTables tt,
           Slots<T> p, uint32_t *__restrict__ key, Cells cells, int32_t *__restrict__ tile_in,
           uint64_t *lb, const int32_t *__restrict__ hole_pos,
           const int32_t *__restrict__ hole_oc, uint32_t *__restrict__ obuf, int ncase, int *err)
{
    tail_tiles<T>(cases, st, sc, tt, p, key, cells, tile_in, lb, hole_pos, hole_oc, obuf, ncase,
                  err);
}

// ---------------------------------------------------------------------------
// k_cell_scan: per case, exclusive sums over its cells of the in-range and
// out-of-range counts (Fin, ostart) and the new cell starts.
// ---------------------------------------------------------------------------
// Cells per tile of k_cell_scan: each warp takes 32 x CELL_VEC consecutive
// cells as CELL_VEC rows of 32 (a row per load, so every load and store of a
// warp is contiguous), scanned row by row with warp shuffles.
#ifndef DSMC_CELL_VEC
#define DSMC_CELL_VEC 4
#endif
constexpr int CELL_VEC = DSMC_CELL_VEC;
constexpr int CELL_TILE = TILE_THREADS * CELL_VEC;

// Cell tiles are dealt by ticket: any number of CTAs of TILE_THREADS.
__device__ __forceinline__ void cell_scan_tiles(const CaseDev *__restrict__ cases,
                                                StepScratch *sc, TileTables tt, Cells cells,
                                                int new_side, uint64_t *lb, int ncase, int *err)
{
    __shared__ int s_tile;
    int32_t *start = start_of(cells, new_side);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_tile = static_cast<int>(atomicAdd(&sc->cell_ticket, 1u));
        __syncthreads();
        const int t = s_tile;
        if (t >= tt.cell0[ncase])
            return;
        const int ci = case_of(tt.cell0, ncase, t);
        const CaseDev &c = cases[ci];
        const int local_tile = t - tt.cell0[ci];
        const int w0 = local_tile * CELL_TILE + warp * (32 * CELL_VEC); // warp's first cell
        unsigned long long v[CELL_VEC]; // pack2(in-range, out-of-range) of row k's cell
        unsigned long long mine = 0;
#pragma unroll
        for (int k = 0; k < CELL_VEC; ++k) {
            const int cc = w0 + k * 32 + lane;
            uint32_t a = 0, b = 0;
            if (cc < c.ncell) {
                a = static_cast<uint32_t>(cells.n_in[c.cbase + cc]);
                b = static_cast<uint32_t>(cells.n_o[c.cbase + cc]);
            }
            v[k] = pack2(a, b);
            mine += v[k];
        }
        // Warps in cell order: the exclusive prefix of lane 0 of a warp is
        // the sum of the warps before it.
        unsigned long long tot;
        const unsigned long long ex = block_exclusive<unsigned long long>(mine, tot);
        const unsigned long long wex = __shfl_sync(0xffffffffu, ex, 0);
        unsigned long long run =
            lookback_block<TILE_THREADS>(lb, t, t - local_tile, tot, err) + wex;
#pragma unroll
        for (int k = 0; k < CELL_VEC; ++k) {
            unsigned long long inc = v[k];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o)
                    inc += u;
            }
            const unsigned long long base = run + inc - v[k];
            const int cc = w0 + k * 32 + lane;
            const uint32_t ra = pack2_a(base), rb = pack2_b(base);
            if (cc < c.ncell) {
                cells.fin[c.cbase + cc] = static_cast<int32_t>(ra);
                cells.ostart[c.cbase + cc] = static_cast<int32_t>(rb);
                start[c.cbase + cc] = static_cast<int32_t>(ra + rb);
            }
            if (cc == c.ncell - 1) {
                const unsigned long long end = base + v[k];
                start[c.cbase + c.ncell] = static_cast<int32_t>(pack2_a(end) + pack2_b(end));
            }
            run += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
}

__global__ void __launch_bounds__(TILE_THREADS)
    k_cell_scan(const CaseDev *__restrict__ cases, StepScratch *sc, TileTables tt, Cells cells,
                int new_side, uint64_t *lb, int ncase, int *err)
{
    cell_scan_tiles(cases, sc, tt, cells, new_side, lb, ncase, err);
}

// ---------------------------------------------------------------------------
// k_tile_scan: grid (chunks, cases).  Exclusive prefix of the in-range
// counts of a case's move tiles into tile_prefix.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void tile_scan_chunk(const CaseState *st, const int32_t *tile_in,
                                                int32_t *tile_prefix, int chunk, int ci)
{
    const CaseState &s = st[ci];
    const int n = s.n_move_tiles;
    const int c0 = chunk * NT * SCAN_VEC;
    if (c0 >= n)
        return; // uniform over the CTA
    const int32_t *a = tile_in + s.move_tile0;
    const int32_t carry = seq_before<NT>(a, n, a, c0);
    int32_t pre[SCAN_VEC];
    (void)seq_chunk<NT>(a, tile_prefix + s.move_tile0, n, a, tile_prefix + s.move_tile0, n, c0,
                        carry, pre);
}

__global__ void __launch_bounds__(SCAN_THREADS)
    k_tile_scan(const CaseState *st, const int32_t *tile_in, int32_t *tile_prefix)
{
    tile_scan_chunk<SCAN_THREADS>(st, tile_in, tile_prefix, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// k_olist: buckets the particles that are not in range (changed cell, were
// injected, or refilled a hole) into per-cell lists; order is fixed later.
// ---------------------------------------------------------------------------
// Each thread takes OLIST_BATCH entries at a time, one phase of dependent
// accesses (list entry, key, counter, list slot) for all of them before the
// next, so that their memory latencies overlap.
constexpr int OLIST_BATCH = 4;
__device__ __forceinline__ void olist_blocks(const CaseDev *__restrict__ cases,
                                             const CaseState *st, const StepScratch *sc,
                                             const uint32_t *__restrict__ obuf,
                                             const uint32_t *__restrict__ key, Cells cells,
                                             int32_t *__restrict__ olist,
                                             const int64_t *__restrict__ pbases, int ncase,
                                             int *err, int bx, int nbx)
{
    const uint32_t n = sc->obuf_count;
    const uint32_t stride = nbx * blockDim.x;
    for (uint32_t i0 = bx * blockDim.x + threadIdx.x; i0 < n;
         i0 += OLIST_BATCH * stride) {
        uint32_t g[OLIST_BATCH], kw[OLIST_BATCH];
        int64_t q[OLIST_BATCH];
        int32_t cg[OLIST_BATCH], j[OLIST_BATCH];
        int ci[OLIST_BATCH];
#pragma unroll
        for (int k = 0; k < OLIST_BATCH; ++k) {
            const uint32_t i = i0 + k * stride;
            g[k] = i < n ? obuf[i] : 0u;
            kw[k] = i < n ? key[g[k]] : KEY_DEAD;
        }
#pragma unroll
        for (int k = 0; k < OLIST_BATCH; ++k) {
            int lo = 0, hi = ncase - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (pbases[mid] <= static_cast<int64_t>(g[k]))
                    lo = mid;
                else
                    hi = mid - 1;
            }
            ci[k] = lo;
            q[k] = static_cast<int64_t>(g[k]) - pbases[lo];
            // Not listed: removed, in range, or a tail slot that moved into
            // a hole (listed there).
            const bool listed = !(kw[k] & (KEY_DEAD | KEY_IN)) && q[k] < st[lo].n_keep;
            cg[k] = listed ? static_cast<int32_t>(kw[k] & KEY_CELL) : -1;
        }
        // The cell's count and list offset do not depend on the increment:
        // loaded before it, so both latencies overlap.
        int32_t no[OLIST_BATCH], os[OLIST_BATCH];
#pragma unroll
        for (int k = 0; k < OLIST_BATCH; ++k) {
            no[k] = cg[k] >= 0 ? cells.n_o[cg[k]] : 0;
            os[k] = cg[k] >= 0 ? cells.ostart[cg[k]] : 0;
        }
#pragma unroll
        for (int k = 0; k < OLIST_BATCH; ++k)
            j[k] = cg[k] >= 0 ? atomicAdd(cells.o_fill + cg[k], 1) : 0;
#pragma unroll
        for (int k = 0; k < OLIST_BATCH; ++k) {
            if (cg[k] < 0)
                continue;
            if (j[k] >= no[k]) {
                report_error(err, DSMC_ERR_STATE); // counts and list disagree
                continue;
            }
            olist[pbases[ci[k]] + os[k] + j[k]] = static_cast<int32_t>(q[k]);
        }
    }
}

__global__ void k_olist(const CaseDev *__restrict__ cases, const CaseState *st,
                        const StepScratch *sc, const uint32_t *__restrict__ obuf,
                        const uint32_t *__restrict__ key, Cells cells,
                        int32_t *__restrict__ olist, const int64_t *__restrict__ pbases,
                        int ncase, int *err)
{
    olist_blocks(cases, st, sc, obuf, key, cells, olist, pbases, ncase, err, blockIdx.x,
                 gridDim.x);
}

// ---------------------------------------------------------------------------
// k_cell_fix: per cell, orders its out-of-range list by slot, gives each of
// those particles its final slot (written into its key word, bit 31 clear),
// and computes the base offset of the cell's in-range particles.
// ---------------------------------------------------------------------------
// The j-th particle, in slot order, of a cell's out-of-range list (old slot
// q) gets its final slot: after the cell's `ni` in-range particles when it
// lies above the cell's old slot range [o_lo, o_hi).  Returns 1 when it lies
// below that range.
__device__ __forceinline__ int fix_place(int32_t q, int j, int32_t start, int32_t ni,
                                         int32_t o_lo, int32_t o_hi, int64_t keep,
                                         uint32_t *key, int64_t pbase, int *err)
{
    const int64_t fin = start + j + (q >= o_hi ? ni : 0);
    if (q < 0 || q >= keep || fin < 0 || fin >= keep)
        report_error(err, DSMC_ERR_STATE); // counts and list disagree
    else
        key[pbase + q] = static_cast<uint32_t>(fin);
    return q < o_lo ? 1 : 0;
}

// Lists of up to FIX_REG entries (nearly all: a few particles enter a cell
// per step) are sorted in registers; longer ones in place.
constexpr int FIX_REG = 8;

__device__ __forceinline__ void cell_fix_blocks(const CaseDev *__restrict__ cases,
                                                const CaseState *st, TileTables tt, Cells cells,
                                                int old_side, uint32_t *__restrict__ key,
                                                int32_t *__restrict__ olist, int total_cells,
                                                int ncase, int *err, int bx, int nbx)
{
    const int32_t *os = start_of(cells, old_side);
    const int32_t *ns = start_of(cells, old_side ^ 1);
    for (int cg = bx * blockDim.x + threadIdx.x; cg < total_cells; cg += nbx * blockDim.x) {
        const int ci = case_of(tt.cellbase, ncase, cg);
        const CaseDev &c = cases[ci];
        const int cl = cg - c.cbase;
        if (cl >= c.ncell)
            continue;
        // Every per-cell word first, so that their loads overlap.
        const int32_t n = cells.n_o[cg];
        const int32_t ost = cells.ostart[cg];
        const int32_t fin_cell = cells.fin[cg];
        const int32_t nend = ns[cg + 1];
        const int32_t ni = cells.n_in[cg];
        const int32_t start = ns[cg];
        const int32_t o_lo = os[cg], o_hi = os[cg + 1];
        int32_t lo = 0;
        if (n > 0) {
            int32_t *seg = olist + c.pbase + ost;
            const int64_t keep = st[ci].n_keep;
            if (n <= FIX_REG) {
                int32_t v[FIX_REG];
#pragma unroll
                for (int a = 0; a < FIX_REG; ++a)
                    v[a] = a < n ? seg[a] : INT32_MAX;
                // Odd-even transposition sort: FIX_REG rounds sort FIX_REG
                // values (slots are distinct; the padding sorts last).
#pragma unroll
                for (int r = 0; r < FIX_REG; ++r)
#pragma unroll
                    for (int a = r & 1; a + 1 < FIX_REG; a += 2) {
                        const int32_t x = v[a], y = v[a + 1];
                        v[a] = min(x, y);
                        v[a + 1] = max(x, y);
                    }
#pragma unroll
                for (int j = 0; j < FIX_REG; ++j)
                    if (j < n)
                        lo += fix_place(v[j], j, start, ni, o_lo, o_hi, keep, key, c.pbase, err);
            } else {
                // Insertion sort by slot, in place.
                for (int a = 1; a < n; ++a) {
                    const int32_t v = seg[a];
                    int b = a - 1;
                    while (b >= 0 && seg[b] > v) {
                        seg[b + 1] = seg[b];
                        --b;
                    }
                    seg[b + 1] = v;
                }
                for (int j = 0; j < n; ++j)
                    lo += fix_place(seg[j], j, start, ni, o_lo, o_hi, keep, key, c.pbase, err);
            }
        }
        cells.base_in[cg] = start + lo - fin_cell;
        // The next step starts with every particle of the cell counted as
        // in range; k_move subtracts the ones that leave.
        cells.n_in[cg] = nend - start;
        cells.n_o[cg] = 0;
        cells.o_fill[cg] = 0;
    }
}

__global__ void k_cell_fix(const CaseDev *__restrict__ cases, const CaseState *st,
                           TileTables tt, Cells cells, int old_side, uint32_t *__restrict__ key,
                           int32_t *__restrict__ olist, int total_cells, int ncase, int *err)
{
    cell_fix_blocks(cases, st, tt, cells, old_side, key, olist, total_cells, ncase, err,
                    blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_scatter: moves every particle of slots [0, K) to its sorted slot.  An
// in-range particle goes to base_in[cell] + (number of in-range particles at
// lower slots of its case); any other particle's key word already holds its
// slot (k_cell_fix).
//
// Tiles are staged whole in shared memory by bulk asynchronous copies, SCATTER
// stages deep: while the warps place tile i, the copies of the next tiles of
// this CTA are in flight, so the kernel keeps HBM busy without holding the
// loads in registers.  Iteration k of thread t takes slot k * SC_THREADS + t
// of the tile (SC_THREADS threads, SC_VEC slots each), so the 32 lanes of a
// warp store 32 consecutive destinations when they share a cell.  One
// barrier per tile: it publishes the in-range
// counts of the (iteration, warp) chunks and frees the stage for its refill.
// ---------------------------------------------------------------------------
template <class T> struct ScatterStage {
    uint32_t key[TILE];
    T v[5][TILE];
};
// Threads of a k_scatter CTA: each takes TILE / SC_THREADS slots of a tile.
#ifndef DSMC_SCATTER_THREADS
#define DSMC_SCATTER_THREADS 256
#endif
constexpr int SC_THREADS = DSMC_SCATTER_THREADS;
constexpr int SC_VEC = TILE / SC_THREADS;
constexpr int SC_WARPS = SC_THREADS / 32;
static_assert(SC_VEC * SC_WARPS == 32, "one warp scans the (iteration, warp) chunk counts");

template <class T> __host__ __device__ constexpr int scatter_stages()
{
    return sizeof(T) == 4 ? DSMC_SCATTER_STAGES : 2;
}
template <class T> __host__ __device__ constexpr size_t scatter_smem()
{
    return sizeof(ScatterStage<T>) * scatter_stages<T>();
}

// The scatter tiles of block bx of nbx; smem_raw holds
// S * sizeof(ScatterStage<T>) bytes.  False when a staged copy never completed (reported; the copies in
// flight were waited for, the barriers stay live).
template <class T, int S = scatter_stages<T>()>
__device__ __forceinline__ bool
    scatter_tiles(const CaseDev *__restrict__ cases, const CaseState *st, TileTables tt,
                  Slots<T> src, Slots<T> dst, const uint32_t *__restrict__ key, Cells cells,
                  const int32_t *__restrict__ tile_prefix, int ncase, int *err,
                  unsigned char *smem_raw, int bx, int nbx)
{
    static_assert(S >= 2, "see the stage rule above");
    ScatterStage<T> *stage = reinterpret_cast<ScatterStage<T> *>(smem_raw);
    __shared__ uint64_t bar[S];
    __shared__ int s_cnt[2][32]; // in-range counts per (iteration, warp), two buffers
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const int total = tt.scatter0[ncase];

    // Thread 0 only: starts the copies of tile t into stage sidx.
    auto issue = [&](int t, int sidx) {
        const int ci = case_of(tt.scatter0, ncase, t);
        const int64_t g0 = cases[ci].pbase + static_cast<int64_t>(t - tt.scatter0[ci]) * TILE;
        constexpr uint32_t kb = TILE * sizeof(uint32_t), vb = TILE * sizeof(T);
        mbar_arrive_expect_tx(&bar[sidx], kb + 5 * vb);
        bulk_g2s(stage[sidx].key, key + g0, kb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[0], src.x + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[1], src.y + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[2], src.vx + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[3], src.vy + g0, vb, &bar[sidx]);
        bulk_g2s(stage[sidx].v[4], src.vz + g0, vb, &bar[sidx]);
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i)
            mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncthreads();
    int issued = 0;
    if (threadIdx.x == 0)
        for (; issued < S && bx + issued * nbx < total; ++issued)
            issue(bx + issued * nbx, issued);

    int it = 0;
    bool failed = false;
    for (int t = bx; t < total; t += nbx, ++it) {
        const int sidx = it % S;
        const bool ok = mbar_wait(&bar[sidx], static_cast<uint32_t>((it / S) & 1));
        const int ci = case_of(tt.scatter0, ncase, t);
        const CaseDev &c = cases[ci];
        const CaseState &s = st[ci];
        const int local_tile = t - tt.scatter0[ci];
        const int64_t keep = s.n_keep;
        const ScatterStage<T> &sg = stage[sidx];
        const int64_t tile0 = static_cast<int64_t>(local_tile) * TILE;
        uint32_t keys[SC_VEC];
        T x[SC_VEC], y[SC_VEC], vx[SC_VEC], vy[SC_VEC], vz[SC_VEC];
        unsigned bin[SC_VEC];
#pragma unroll
        for (int k = 0; k < SC_VEC; ++k) {
            const int e = k * SC_THREADS + threadIdx.x;
            keys[k] = (ok && tile0 + e < keep) ? sg.key[e] : KEY_DEAD;
            x[k] = sg.v[0][e];
            y[k] = sg.v[1][e];
            vx[k] = sg.v[2][e];
            vy[k] = sg.v[3][e];
            vz[k] = sg.v[4][e];
            bin[k] = __ballot_sync(0xffffffffu, (keys[k] & KEY_IN) != 0);
            if (lane == 0)
                s_cnt[it & 1][k * SC_WARPS + warp] = __popc(bin[k]);
        }
        // Every thread has copied its part of the stage into registers.
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            const int tn = t + S * nbx;
            if (tn < total) {
                issue(tn, sidx);
                ++issued;
            }
        }
        // Lane i: in-range count of (iteration, warp) chunk i; chunks are in
        // slot order, so their exclusive scan ranks them within the tile.
        const int cnt = s_cnt[it & 1][lane];
        int cinc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, cinc, o);
            if (lane >= o)
                cinc += v;
        }
        const int cexcl = cinc - cnt;
        const int tile_total = __shfl_sync(0xffffffffu, cinc, 31);
        const int64_t base = tile_total > 0 ? tile_prefix[s.move_tile0 + local_tile] : 0;
        int64_t fin[SC_VEC];
#pragma unroll
        for (int k = 0; k < SC_VEC; ++k) {
            const int pre = __shfl_sync(0xffffffffu, cexcl, k * SC_WARPS + warp);
            if (keys[k] & KEY_DEAD)
                fin[k] = -1;
            else if (keys[k] & KEY_IN)
                fin[k] = cells.base_in[keys[k] & KEY_CELL] + base + pre +
                         __popc(bin[k] & lanes_below);
            else
                fin[k] = keys[k];
        }
#pragma unroll
        for (int k = 0; k < SC_VEC; ++k) {
            if (keys[k] & KEY_DEAD)
                continue;
            if (fin[k] < 0 || fin[k] >= keep) {
                report_error(err, DSMC_ERR_STATE); // counts and keys disagree
                continue;
            }
            const int64_t gd = c.pbase + fin[k];
            dst.x[gd] = x[k];
            dst.y[gd] = y[k];
            dst.vx[gd] = vx[k];
            dst.vy[gd] = vy[k];
            dst.vz[gd] = vz[k];
        }
    }
    if (failed) {
        // A copy never completed: report, then wait (bounded) for the copies
        // this CTA still has in flight before its shared memory goes away.
        if (threadIdx.x == 0) {
            report_error(err, DSMC_ERR_TIMEOUT);
            for (int j = it; j < issued; ++j)
                mbar_wait(&bar[j % S], static_cast<uint32_t>((j / S) & 1));
        }
        return false;
    }
    // Every copy issued was consumed: the barriers can be retired.
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < S; ++i)
            mbar_inval(&bar[i]);
    return true;
}

template <class T>
__global__ void __launch_bounds__(SC_THREADS)
    k_scatter(const CaseDev *__restrict__ cases, const CaseState *st, TileTables tt,
              Slots<T> src, Slots<T> dst, const uint32_t *__restrict__ key, Cells cells,
              const int32_t *__restrict__ tile_prefix, int ncase, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (void)scatter_tiles<T>(cases, st, tt, src, dst, key, cells, tile_prefix, ncase, err,
                           smem_raw, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Collisions, BinaryCollisionsInCell (Collision.cpp:21-44) with one stream
// per cell, in two passes.  k_collide_select makes every cell's first draw
// (the Bernoulli rounding of the pair count) and lists the cells that have
// candidate pairs; at the reference's rarefaction that is about one cell in
// a thousand.  k_collide_pairs then runs the candidate loop of the listed
// cells only, continuing each cell's stream at draw 1.  The expensive code
// (pow, sin, cos, the elastic collision) thus sets neither the register
// budget nor the occupancy of the passes that touch every cell.
// ---------------------------------------------------------------------------
constexpr int COLLIDE_CELLS = 128;

// NTC pair count of a cell with n particles (Collision.cpp:23-27) and the
// draw that rounds it.
__device__ __forceinline__ int ntc_pairs(const CaseDev &c, int n, dsmc_stream &r)
{
    const double npair = 0.5 * n * (n - 1) * c.weight * c.sc_max * c.dt / c.dv;
    int nn = static_cast<int>(npair);
    const double frac = npair - nn;
    return (uniform(r) < frac) ? nn + 1 : nn;
}

// ElasticCollision (Collision.cpp:7-19) of velocities vi, vj with relative
// speed cr, drawing v3rand_isotropic (rng/IsotropicVectorRNG.cxx:11-19) from
// r; the new velocities replace vi and vj.
__device__ __forceinline__ void elastic_collision(dsmc_stream &r, double vi[3], double vj[3],
                                                  double cr)
{
    const double cos_t = 1.0 - 2.0 * uniform(r);
    const double sin_t = sqrt(1.0 - cos_t * cos_t);
    const double e = 2.0 * PI_D * uniform(r);
    const double nv[3] = {cos_t, sin_t * cos(e), sin_t * sin(e)};
    const double half = cr * 0.5;
    const double vc0 = 0.5 * (vj[0] + vi[0]), vc1 = 0.5 * (vj[1] + vi[1]),
                 vc2 = 0.5 * (vj[2] + vi[2]);
    const double d0 = half * nv[0], d1 = half * nv[1], d2 = half * nv[2];
    vi[0] = vc0 + d0;
    vi[1] = vc1 + d1;
    vi[2] = vc2 + d2;
    vj[0] = vc0 - d0;
    vj[1] = vc1 - d1;
    vj[2] = vc2 - d2;
}

// The particles of one cell's list IPC: entry i is slot base + i, or
// base + ipc[i] when a list is given.  Velocities are read as doubles and
// stored rounded to the state's precision.
template <class T> struct SlotRun {
    Slots<T> p;
    int64_t base;
    const int32_t *ipc;
    __device__ __forceinline__ int64_t at(int i) const { return base + (ipc ? ipc[i] : i); }
    __device__ __forceinline__ void load(int i, double v[3]) const
    {
        const int64_t g = at(i);
        v[0] = static_cast<double>(p.vx[g]);
        v[1] = static_cast<double>(p.vy[g]);
        v[2] = static_cast<double>(p.vz[g]);
    }
    __device__ __forceinline__ void store(int i, const double v[3]) const
    {
        const int64_t g = at(i);
        p.vx[g] = Store<T>::rn(v[0]);
        p.vy[g] = Store<T>::rn(v[1]);
        p.vz[g] = Store<T>::rn(v[2]);
    }
};

// The candidate loop of BinaryCollisionsInCell (Collision.cpp:29-42): nn
// candidate pairs of the cell's n particles drawn from r (which continues
// after the pair-count draw), VHS acceptance, elastic collision of the
// accepted ones.  Returns the number of collisions.
template <class Run>
__device__ __forceinline__ int ntc_candidates(const CaseDev &c, int n, int nn, dsmc_stream &r,
                                              const Run &run)
{
    int ncc = 0;
    for (int kk = 0; kk < nn; ++kk) {
        const int i = irand_uniform(r, n);
        int j;
        do {
            j = irand_uniform(r, n);
        } while (j == i);
        double vi[3], vj[3];
        run.load(i, vi);
        run.load(j, vj);
        const double vr0 = vj[0] - vi[0], vr1 = vj[1] - vi[1], vr2 = vj[2] - vi[2];
        const double cr = sqrt(vr0 * vr0 + vr1 * vr1 + vr2 * vr2);
        const double sigma = c.sigma_ref * pow(c.cr_ref / cr, c.omega);
        if (uniform(r) < sigma * cr / c.sc_max) {
            elastic_collision(r, vi, vj, cr);
            run.store(i, vi);
            run.store(j, vj);
            ncc++;
        }
    }
    return ncc;
}

__device__ __forceinline__ void
    collide_select_blocks(const CaseDev *__restrict__ cases, const CaseState *st,
                          StepScratch *sc, TileTables tt, Cells cells, int side,
                          uint32_t *__restrict__ coll_list, int total_cells, int ncase, int bx,
                          int nbx)
{
    const int32_t *start = start_of(cells, side);
    for (int base = bx * blockDim.x; base < total_cells; base += nbx * blockDim.x) {
        const int cg = base + threadIdx.x;
        bool listed = false;
        if (cg < total_cells) {
            const int ci = case_of(tt.cellbase, ncase, cg);
            const CaseDev &c = cases[ci];
            const int cl = cg - c.cbase;
            if (cl < c.ncell) {
                const int n = start[cg + 1] - start[cg];
                if (n >= 2) {
                    dsmc_stream r;
                    open_stream(r, c, DSMC_RNG_COLLIDE, st[ci].step, static_cast<uint32_t>(cl));
                    listed = ntc_pairs(c, n, r) > 0;
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, listed);
        if (m) {
            const int lane = threadIdx.x & 31;
            uint32_t b = 0;
            if (lane == __ffs(m) - 1)
                b = atomicAdd(&sc->coll_count, static_cast<uint32_t>(__popc(m)));
            b = __shfl_sync(0xffffffffu, b, __ffs(m) - 1);
            if (listed)
                coll_list[b + __popc(m & ((1u << lane) - 1u))] = static_cast<uint32_t>(cg);
        }
    }
}

__global__ void __launch_bounds__(256)
    k_collide_select(const CaseDev *__restrict__ cases, const CaseState *st, StepScratch *sc,
                     TileTables tt, Cells cells, int side, uint32_t *__restrict__ coll_list,
                     int total_cells, int ncase)
{
    collide_select_blocks(cases, st, sc, tt, cells, side, coll_list, total_cells, ncase,
                          blockIdx.x, gridDim.x);
}

template <class T>
__device__ __forceinline__ void
    collide_pairs_blocks(const CaseDev *__restrict__ cases, CaseState *st,
                         const StepScratch *sc, TileTables tt, Slots<T> p, Cells cells, int side,
                         const uint32_t *__restrict__ coll_list, int ncase, int bx, int nbx)
{
    const int32_t *start = start_of(cells, side);
    const uint32_t count = sc->coll_count;
    for (uint32_t w = bx * blockDim.x + threadIdx.x; w < count; w += nbx * blockDim.x) {
        const int cg = static_cast<int>(coll_list[w]);
        const int ci = case_of(tt.cellbase, ncase, cg);
        const CaseDev &c = cases[ci];
        CaseState &s = st[ci];
        const int cl = cg - c.cbase;
        const int64_t a0 = c.pbase + start[cg];
        const int n = start[cg + 1] - start[cg];
        dsmc_stream r;
        open_stream(r, c, DSMC_RNG_COLLIDE, s.step, static_cast<uint32_t>(cl));
        const int nn = ntc_pairs(c, n, r); // draw 0 again: the same value
        SlotRun<T> run{p, a0, nullptr};
        const int ncc = ntc_candidates(c, n, nn, r, run);
        if (ncc > 0) {
            if (s.sampling_mode == 1) // CollideParticles, Collision.cpp:53
                cells.acc[ACC_NC * cells.acc_stride + cg] += ncc;
            atomicAdd(reinterpret_cast<unsigned long long *>(&s.nc_step),
                      static_cast<unsigned long long>(ncc));
        }
    }
}

template <class T>
__global__ void __launch_bounds__(128)
    k_collide_pairs(const CaseDev *__restrict__ cases, CaseState *st, const StepScratch *sc,
                    TileTables tt, Slots<T> p, Cells cells, int side,
                    const uint32_t *__restrict__ coll_list, int ncase)
{
    collide_pairs_blocks<T>(cases, st, sc, tt, p, cells, side, coll_list, ncase, blockIdx.x,
                            gridDim.x);
}

// ---------------------------------------------------------------------------
// k_sample: Sampling's accumulation (Sampling.cpp:14-31) in the reference's
// order: each sum of a cell is made by one thread that walks the cell's
// particles sequentially, so every FP64 sum is bit-identical to the
// reference's.  A sample block is CELLS consecutive cells of one case with
// SPLIT threads per cell: thread t takes cell t % CELLS and part t / CELLS
// of its sums (each part a fixed set of sums, so a thread's chains are
// short and independent).  The velocities of a block are one contiguous
// slot range, staged in shared memory by bulk asynchronous copies, S stages
// per CTA; a block whose range exceeds a stage is read from global memory
// directly.  The step graph's k_sample: SAMPLE_CELLS x SAMPLE_SPLIT threads,
// SAMPLE_STAGES stages (one stage measured fastest: more CTAs fit on an SM
// and overlap each other's copies); the persistent step uses its own shape.
// ---------------------------------------------------------------------------
constexpr int SAMPLE_STAGES = DSMC_SAMPLE_STAGES;
constexpr int SAMPLE_UNROLL = DSMC_SAMPLE_UNROLL;
#ifndef DSMC_SAMPLE_CELLS
#define DSMC_SAMPLE_CELLS 64
#endif
#ifndef DSMC_SAMPLE_SPLIT
#define DSMC_SAMPLE_SPLIT 2
#endif
constexpr int SAMPLE_CELLS = DSMC_SAMPLE_CELLS;
constexpr int SAMPLE_SPLIT = DSMC_SAMPLE_SPLIT;
constexpr int SAMPLE_THREADS = SAMPLE_SPLIT * SAMPLE_CELLS;
#ifndef DSMC_SAMPLE_MIN_BLOCKS // k_sample's register budget: 1024 threads per SM
#define DSMC_SAMPLE_MIN_BLOCKS (1024 / SAMPLE_THREADS)
#endif
template <int CELLS> __host__ __device__ constexpr int sample_sub()
{
    static_assert(CELLS % 32 == 0 && COLLIDE_CELLS % CELLS == 0,
                  "whole warps per part, whole sample blocks per collision block");
    return COLLIDE_CELLS / CELLS; // sample blocks per collision block
}
// Staging capacity of a block: 24 (FP32) or 12 (FP64) particles per cell.
template <class T, int CELLS = SAMPLE_CELLS> __host__ __device__ constexpr int sample_pcl()
{
    return 12288 / sizeof(T) / sample_sub<CELLS>();
}
// First cell (in its case) of sample block b of case ci.
template <int CELLS>
__device__ __forceinline__ int sample_cell0(const TileTables &tt, int ci, int b)
{
    constexpr int SUB = sample_sub<CELLS>();
    return (b / SUB - tt.cblock0[ci]) * COLLIDE_CELLS + (b % SUB) * CELLS;
}
template <class T, int CELLS = SAMPLE_CELLS> struct SampleStage {
    T v[3][sample_pcl<T, CELLS>() + 16 / sizeof(T)];
};
template <class T, int CELLS = SAMPLE_CELLS, int S = SAMPLE_STAGES>
__host__ __device__ constexpr size_t sample_smem()
{
    return sizeof(SampleStage<T, CELLS>) * S;
}

// End of the step (Simulation.cpp:160-161) and Sampling's counters
// (Sampling.cpp:17-18) when the step sampled, by the threads of one CTA.
// k_sample's first CTA runs it in a full step: nothing k_sample reads is
// changed by it.
__device__ __forceinline__ void finish_cases(const CaseDev *cases, CaseState *st, int ncase,
                                             int init_mode, int did_sample, int end_step,
                                             dsmc_counters *rec = nullptr)
{
    for (int i = threadIdx.x; i < ncase; i += blockDim.x) {
        CaseState &s = st[i];
        s.n_old = s.n_keep;
        if (init_mode)
            continue;
        if (did_sample && s.sampling_mode == 1) {
            s.sample_step++;
            s.sample_time += cases[i].dt;
        }
        if (end_step) {
            s.nc_last = s.nc_step;
            s.nc_total += s.nc_step;
            s.particle_steps += s.n_keep;
            s.step++;
            s.time += cases[i].dt;
        }
        if (rec) { // the counters of the ended step, as dsmc_get_counters gives them
            dsmc_counters &r = rec[i];
            r.np = s.n_old;
            r.step = s.step;
            r.sample_step = s.sample_step;
            r.collisions_last_step = s.nc_last;
            r.collisions_total = s.nc_total;
            r.drag_collision_count = static_cast<int64_t>(s.drag_count);
            r.particle_steps = s.particle_steps;
            r.drag_impulse_total = s.drag_impulse;
            r.time = s.time;
            r.sample_time = s.sample_time;
            r.drag_sampling_time = s.drag_time;
            r.drag_collision_count_window = static_cast<int64_t>(s.drag_count_window);
            r.drag_impulse_window = s.drag_impulse_window;
        }
    }
}

// The part of a cell's threads that owns moment m, SPLIT threads per cell:
//   2: NP, V, VV00, VV01, VV02, VV11 | VV12, VV22, V2V
//   4: NP, V | VV00, VV01, VV02 | VV11, VV12, VV22 | V2V
__host__ __device__ constexpr int sample_part_of(int split, int m)
{
    return split == 2 ? (m <= ACC_VV11 ? 0 : 1)
                      : (m <= ACC_V2 ? 0 : m <= ACC_VV02 ? 1 : m <= ACC_VV22 ? 2 : 3);
}

// One particle's terms (Sampling.cpp:24-30) of the sums that part P owns.
// FP64 velocities: products rounded, then added.  FP32 velocities: the
// product of two floats is exact in FP64 (24 + 24 significand bits), so
// s + u * v rounds once either way and a fused multiply-add gives the same
// bits as the separate product and sum, with one FP64 operation instead of
// two; vv * v is not exact and keeps its rounding.  Either way every sum has
// the same bits whichever part layout computes it.
template <int SPLIT, int P>
__device__ __forceinline__ void sample_add(double a[ACC_NC], double v0, double v1, double v2)
{
#define DSMC_OWN(m) (sample_part_of(SPLIT, m) == P)
    if (DSMC_OWN(ACC_V0)) {
        a[ACC_V0] += v0;
        a[ACC_V1] += v1;
        a[ACC_V2] += v2;
    }
    if (DSMC_OWN(ACC_VV00))
        a[ACC_VV00] += v0 * v0;
    if (DSMC_OWN(ACC_VV01))
        a[ACC_VV01] += v0 * v1;
    if (DSMC_OWN(ACC_VV02))
        a[ACC_VV02] += v0 * v2;
    if (DSMC_OWN(ACC_VV11))
        a[ACC_VV11] += v1 * v1;
    if (DSMC_OWN(ACC_VV12))
        a[ACC_VV12] += v1 * v2;
    if (DSMC_OWN(ACC_VV22))
        a[ACC_VV22] += v2 * v2;
    if (DSMC_OWN(ACC_V2V0)) {
        const double vv = v0 * v0 + v1 * v1 + v2 * v2;
        a[ACC_V2V0] += vv * v0;
        a[ACC_V2V1] += vv * v1;
        a[ACC_V2V2] += vv * v2;
    }
}
template <int SPLIT, int P>
__device__ __forceinline__ void sample_add(double a[ACC_NC], float f0, float f1, float f2)
{
    const double v0 = f0, v1 = f1, v2 = f2;
    if (DSMC_OWN(ACC_V0)) {
        a[ACC_V0] += v0;
        a[ACC_V1] += v1;
        a[ACC_V2] += v2;
    }
    if (DSMC_OWN(ACC_VV00))
        a[ACC_VV00] += v0 * v0;
    if (DSMC_OWN(ACC_VV01))
        a[ACC_VV01] = __fma_rn(v0, v1, a[ACC_VV01]);
    if (DSMC_OWN(ACC_VV02))
        a[ACC_VV02] = __fma_rn(v0, v2, a[ACC_VV02]);
    if (DSMC_OWN(ACC_VV11))
        a[ACC_VV11] = __fma_rn(v1, v1, a[ACC_VV11]);
    if (DSMC_OWN(ACC_VV12))
        a[ACC_VV12] = __fma_rn(v1, v2, a[ACC_VV12]);
    if (DSMC_OWN(ACC_VV22))
        a[ACC_VV22] = __fma_rn(v2, v2, a[ACC_VV22]);
    if (DSMC_OWN(ACC_V2V0)) {
        const double vv = __fma_rn(v2, v2, __fma_rn(v1, v1, v0 * v0));
        a[ACC_V2V0] += vv * v0;
        a[ACC_V2V1] += vv * v1;
        a[ACC_V2V2] += vv * v2;
    }
#undef DSMC_OWN
}

// The sums that part `part` owns of cell cg, read into a[] (issued before the
// wait for the staged velocities, so that their latency overlaps it).
template <int SPLIT>
__device__ __forceinline__ void sample_load(int part, double a[ACC_NC], Cells cells, int cg)
{
#pragma unroll
    for (int m = 0; m < ACC_NC; ++m)
        if (sample_part_of(SPLIT, m) == part)
            a[m] = cells.acc[m * cells.acc_stride + cg];
}

// Part P's sums a[] of one cell of n particles (velocities vx, vy, vz, in
// slot order): accumulated in order and written back.  The count NP is a
// sum of n ones: exact, so one add of n.
template <class T, int SPLIT, int P>
__device__ __forceinline__ void sample_cell(double a[ACC_NC], Cells cells, int cg, int n,
                                            const T *vx, const T *vy, const T *vz)
{
    if (sample_part_of(SPLIT, ACC_NP) == P)
        a[ACC_NP] += static_cast<double>(n);
    // Unrolled so that the loads and products of the next particles overlap
    // the adds of this one (the sums keep their order: only the adds chain).
#pragma unroll SAMPLE_UNROLL
    for (int i = 0; i < n; ++i)
        sample_add<SPLIT, P>(a, vx[i], vy[i], vz[i]);
#pragma unroll
    for (int m = 0; m < ACC_NC; ++m)
        if (sample_part_of(SPLIT, m) == P)
            cells.acc[m * cells.acc_stride + cg] = a[m];
}

// The sample blocks bx, bx + nbx, ... (CELLS cells, SPLIT x CELLS threads,
// S stages); smem_raw holds sample_smem<T, CELLS, S>() bytes.  Its block
// bx == 0 also ends the step when `finish` is set.  False when a staged copy
// never completed (reported; copies in flight waited for).
template <class T, int CELLS, int SPLIT, int S>
__device__ __forceinline__ bool sample_blocks(const CaseDev *__restrict__ cases, CaseState *st,
                                              TileTables tt, Slots<T> p, Cells cells, int side,
                                              int ncase, int finish, dsmc_counters *rec,
                                              int *err, unsigned char *smem_raw, int bx,
                                              int nbx)
{
    static_assert(SPLIT == 2 || SPLIT == 4, "two or four threads per cell");
    if (finish && bx == 0)
        finish_cases(cases, st, ncase, 0, 1, 1, rec);
    constexpr int A = 16 / sizeof(T); // elements per 16 bytes
    constexpr int SUB = sample_sub<CELLS>();
    SampleStage<T, CELLS> *stage = reinterpret_cast<SampleStage<T, CELLS> *>(smem_raw);
    __shared__ uint64_t bar[S];
    __shared__ int s_staged[S];
    __shared__ int64_t s_r0[S]; // first staged slot (rounded down to A)
    const int32_t *start = start_of(cells, side);
    const int nblocks = tt.cblock0[ncase] * SUB;

    // Thread 0 only: stages the velocities of block b in stage sidx when its
    // case samples this step and the range fits.
    auto issue = [&](int b, int sidx) {
        s_staged[sidx] = 0;
        const int ci = case_of(tt.cblock0, ncase, b / SUB);
        if (st[ci].sampling_mode != 1)
            return;
        const CaseDev &c = cases[ci];
        const int cl0 = sample_cell0<CELLS>(tt, ci, b);
        if (cl0 >= c.ncell)
            return;
        const int cl1 = min(cl0 + CELLS, c.ncell);
        const int64_t r0 = start[c.cbase + cl0] & ~static_cast<int64_t>(A - 1);
        const int64_t r1 = (start[c.cbase + cl1] + A - 1) & ~static_cast<int64_t>(A - 1);
        const int64_t n = r1 - r0;
        if (n <= 0 || n > sample_pcl<T, CELLS>() + A)
            return;
        const uint32_t bytes = static_cast<uint32_t>(n * sizeof(T));
        mbar_arrive_expect_tx(&bar[sidx], 3 * bytes);
        bulk_g2s(stage[sidx].v[0], p.vx + c.pbase + r0, bytes, &bar[sidx]);
        bulk_g2s(stage[sidx].v[1], p.vy + c.pbase + r0, bytes, &bar[sidx]);
        bulk_g2s(stage[sidx].v[2], p.vz + c.pbase + r0, bytes, &bar[sidx]);
        s_r0[sidx] = r0;
        s_staged[sidx] = 1;
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i)
            mbar_init(&bar[i], 1);
        fence_mbar_init();
        for (int i = 0; i < S; ++i)
            if (bx + i * nbx < nblocks)
                issue(bx + i * nbx, i);
    }
    __syncthreads();

    uint32_t phase = 0; // bit i: parity of the next completion of stage i
    for (int it = 0;; ++it) {
        const int b = bx + it * nbx;
        if (b >= nblocks)
            break;
        const int sidx = it % S;
        const int ci = case_of(tt.cblock0, ncase, b / SUB);
        const bool staged = s_staged[sidx] != 0;
        const int part = threadIdx.x / CELLS; // uniform over a warp
        bool ok = true;
        if (st[ci].sampling_mode == 1) {
            const CaseDev &c = cases[ci];
            const int cl = sample_cell0<CELLS>(tt, ci, b) + static_cast<int>(threadIdx.x % CELLS);
            const int cg = c.cbase + cl;
            const bool mine = cl < c.ncell;
            int64_t a0 = 0;
            int n = 0;
            double a[ACC_NC];
            if (mine) {
                a0 = start[cg];
                n = static_cast<int>(start[cg + 1] - a0);
                sample_load<SPLIT>(part, a, cells, cg);
            }
            const T *vx = p.vx + c.pbase + a0, *vy = p.vy + c.pbase + a0,
                    *vz = p.vz + c.pbase + a0;
            if (staged) {
                ok = mbar_wait(&bar[sidx], (phase >> sidx) & 1u);
                phase ^= 1u << sidx;
                const int64_t off = a0 - s_r0[sidx];
                vx = stage[sidx].v[0] + off;
                vy = stage[sidx].v[1] + off;
                vz = stage[sidx].v[2] + off;
            }
            if (mine && n > 0 && ok) {
                if (part == 0)
                    sample_cell<T, SPLIT, 0>(a, cells, cg, n, vx, vy, vz);
                else if (part == 1)
                    sample_cell<T, SPLIT, 1>(a, cells, cg, n, vx, vy, vz);
                else if (SPLIT == 4 && part == 2)
                    sample_cell<T, SPLIT, 2>(a, cells, cg, n, vx, vy, vz);
                else if (SPLIT == 4)
                    sample_cell<T, SPLIT, 3>(a, cells, cg, n, vx, vy, vz);
            }
        }
        // The stage is consumed: refill it with this CTA's block it + S.
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                report_error(err, DSMC_ERR_TIMEOUT);
                for (int j = 0; j < S; ++j)
                    if (s_staged[j])
                        mbar_wait(&bar[j], (phase >> j) & 1u);
            }
            return false;
        }
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            const int bn = b + S * nbx;
            s_staged[sidx] = 0;
            if (bn < nblocks)
                issue(bn, sidx);
        }
        if (S == 1) // the next block reads this stage's flags: publish them first
            __syncthreads();
    }
    // No copy is in flight after the last block (each issued stage was
    // consumed): the barriers can be retired.
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < S; ++i)
            mbar_inval(&bar[i]);
    return true;
}

template <class T>
__global__ void __launch_bounds__(SAMPLE_THREADS, DSMC_SAMPLE_MIN_BLOCKS)
    k_sample(const CaseDev *__restrict__ cases, CaseState *st, TileTables tt, Slots<T> p,
             Cells cells, int side, int ncase, int finish, dsmc_counters *rec, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (void)sample_blocks<T, SAMPLE_CELLS, SAMPLE_SPLIT, SAMPLE_STAGES>(
        cases, st, tt, p, cells, side, ncase, finish, rec, err, smem_raw, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_finish: end of the step (Simulation.cpp:160-161), Sampling's counters
// (Sampling.cpp:17-18) when the step sampled.
// ---------------------------------------------------------------------------
__global__ void k_finish(const CaseDev *cases, CaseState *st, int ncase, int init_mode,
                         int did_sample, int end_step)
{
    finish_cases(cases, st, ncase, init_mode, did_sample, end_step);
}

} // namespace dsmc
