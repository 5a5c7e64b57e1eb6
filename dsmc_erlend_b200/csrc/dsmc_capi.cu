// dsmc_capi.cu - the C ABI of include/dsmc.h over the kernels of
// dsmc_kernels.cuh: context and device memory, the launch sequence of a
// step, its CUDA graphs, and the upload/download paths.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dsmc.h"
#include "dsmc_kernels.cuh"
#include "dsmc_persist.cuh"
#include "dsmc_units.cuh"

using namespace dsmc;

namespace {

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "dsmc: %s failed: %s (%s:%d)\n", #call,                  \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                     \
            return DSMC_ERR_CUDA;                                                         \
        }                                                                                 \
    } while (0)

enum KernelId {
    KID_PLAN, KID_MOVE, KID_MOVE_NEAR, KID_INJECT, KID_DEAD_SCAN, KID_HOLES, KID_TAIL,
    KID_CELL_SCAN, KID_TILE_SCAN,
    KID_OLIST, KID_CELL_FIX, KID_SCATTER, KID_COLLIDE_SELECT, KID_COLLIDE, KID_SAMPLE,
    KID_FINISH, KID_COUNT
};
const char *kKernelNames[KID_COUNT] = {
    "k_plan",      "k_move",   "k_move_near",      "k_inject",         "k_dead_scan",     "k_holes",
    "k_tail",
    "k_cell_scan", "k_tile_scan", "k_olist",       "k_cell_fix",      "k_scatter",
    "k_collide_select", "k_collide_pairs", "k_sample", "k_finish"};

struct Timed {
    int kid;
    cudaEvent_t a, b;
};


} // namespace

struct dsmc_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // The step graph's second branch: kernels that depend on neither
    // neighbour on the main stream run there (captured only, see `par`).
    cudaStream_t side_stream = nullptr;
    cudaEvent_t branch_ev[6] = {nullptr};
    // Pinned chunks of the field read-back into pageable host memory
    // (allocated by the first large read-back).
    void *field_stage[2] = {nullptr, nullptr};
    cudaEvent_t field_ev[2] = {nullptr, nullptr};
    bool par = false; // true while the full step is captured into a graph
    int ncase = 0;
    int precision = DSMC_FP64;
    std::vector<dsmc_params> params;
    std::vector<dsmc_derived> derived;
    std::vector<CaseDev> hcases;
    int64_t total_slots = 0;
    int total_cells = 0; // global cell ids, ncell + 1 per case
    int max_slot_tiles = 0;
    int64_t max_case_tiles = 0; // most move + inject tiles of one case
    int total_cell_tiles = 0;

    CaseDev *d_cases = nullptr;
    CaseState *d_state = nullptr;
    StepScratch *d_scratch = nullptr;
    int *d_err = nullptr;
    int32_t *d_tables = nullptr; // 7 x (ncase + 1)
    int32_t *d_tmp = nullptr;    // 2 x ncase
    int64_t *d_pbases = nullptr;
    TileTables tt{};

    void *arena = nullptr; // the one device allocation all buffers below are carved from
    void *buf[2][5] = {{nullptr}};
    uint32_t *key = nullptr;
    Cells cells{};
    int32_t *tile_in = nullptr, *tile_prefix = nullptr;
    int32_t *tile_dead = nullptr, *tile_dprefix = nullptr;   // removed slots per move tile
    int32_t *itile_dead = nullptr, *itile_dprefix = nullptr; // ... per inject tile
    uint64_t *lb = nullptr; // 4 chains: move, inject, tail, cell
    size_t lb_words = 0;
    int32_t *hole_pos = nullptr, *hole_oc = nullptr;
    uint32_t *obuf = nullptr;
    uint32_t *near_list = nullptr; // slots queued by k_move for k_move_near
    int32_t *olist = nullptr;
    uint32_t *coll_list = nullptr; // cells with candidate pairs, per step
    dsmc_counters *d_counters = nullptr; // every case's counters at the end of the last full step

    int cur = 0;
    bool initialized = false;
    int stage = 0; // staged calls: 0 idle, 1 moved, 2 boundary, 3 indexed, 4 collided, 5 sampled
    bool sampled = false;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};

    // The persistent step (DSMC_STEP_PERSISTENT): one cooperative launch of
    // k_persistent for all steps of a dsmc_step call, the kernel node of a
    // graph (memset of the barrier state, then the kernel); one instantiated
    // graph per (steps, buffer side) pair met, the most recent few kept.
    int step_mode = DSMC_STEP_GRAPH;
    GridSync *d_gsync = nullptr;
    int *d_probe_err = nullptr;
    unsigned long long *d_phase_ns = nullptr; // PERSIST_PHASES sums
    int p_ctas = 0, p_ctas_max = 0; // CTAs per SM of k_persistent
    bool coop = false;              // the device supports cooperative launches
    bool p_graph = true;            // launched through graphs (else directly)
    uint64_t p_wait_ns = 2000000000ull;
    struct PGraph {
        int n_steps, side;
        cudaGraph_t g;
        cudaGraphExec_t exec;
    };
    std::vector<PGraph> pgraphs;

    // CTAs per SM of each kernel's grid (the tunable launch shape), and the
    // most that fit (occupancy); zero for kernels with a fixed grid.
    int ctas[KID_COUNT] = {0};
    int ctas_max[KID_COUNT] = {0};

    bool profiling = false;
    std::vector<Timed> timed;
    double kernel_ms[KID_COUNT] = {0};
    int64_t kernel_launches[KID_COUNT] = {0};
    std::vector<cudaEvent_t> event_pool;
};

namespace {

cudaEvent_t take_event(dsmc_ctx *c)
{
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when profiling (eager mode only).
struct Span {
    dsmc_ctx *c;
    int kid;
    cudaEvent_t a = nullptr;
    Span(dsmc_ctx *ctx, int k) : c(ctx), kid(k)
    {
        if (c->profiling) {
            a = take_event(c);
            cudaEventRecord(a, c->stream);
        }
    }
    ~Span()
    {
        if (c->profiling) {
            cudaEvent_t b = take_event(c);
            cudaEventRecord(b, c->stream);
            c->timed.push_back({kid, a, b});
        }
    }
};

int grid(const dsmc_ctx *c, int kid) { return std::max(1, c->ctas[kid]) * c->sms; }

// Bytes per pinned chunk of the field read-back.
constexpr size_t FIELD_CHUNK = size_t(8) << 20;

// Chunks of the tile-count scans: enough for the most tiles a case can have
// (its slots, move and inject tiles rounded up separately).
int scan_chunks(const dsmc_ctx *c)
{
    return static_cast<int>((c->max_case_tiles + SCAN_CHUNK - 1) / SCAN_CHUNK);
}

template <class T> Slots<T> slots(dsmc_ctx *c, int side)
{
    Slots<T> s;
    s.x = static_cast<T *>(c->buf[side][0]);
    s.y = static_cast<T *>(c->buf[side][1]);
    s.vx = static_cast<T *>(c->buf[side][2]);
    s.vy = static_cast<T *>(c->buf[side][3]);
    s.vz = static_cast<T *>(c->buf[side][4]);
    return s;
}

uint64_t *lb_chain(dsmc_ctx *c, int i) { return c->lb + static_cast<size_t>(i) * c->lb_words / 4; }

int clear_step_scratch(dsmc_ctx *c)
{
    CK(cudaMemsetAsync(c->d_scratch, 0, sizeof(StepScratch), c->stream));
    CK(cudaMemsetAsync(c->lb, 0, c->lb_words * sizeof(uint64_t), c->stream));
    return DSMC_OK;
}

// Branch points of the step graph.  Captured into the graph (never run
// eagerly), the side stream holds kernels whose inputs and outputs are
// disjoint from those of the main-stream kernels they overlap:
//   k_inject         || k_move, k_move_near   (slots [n_old, n_total) against
//                       [0, n_old); commutative cell counters; the
//                       out-of-range list is ordered by slot later)
//   k_tile_scan      || k_cell_scan, k_olist, k_cell_fix (tile counts only)
//   k_collide_select || k_olist, k_cell_fix, k_scatter (the new cell starts,
//                       final after k_cell_scan; no particle data)
enum { EV_PLAN, EV_INJECT, EV_TAIL, EV_TILE_SCAN, EV_CELL_SCAN, EV_SELECT };

// `to` waits for what `from` has enqueued so far (event `ev`).
int branch(dsmc_ctx *c, int ev, cudaStream_t from, cudaStream_t to)
{
    CK(cudaEventRecord(c->branch_ev[ev], from));
    CK(cudaStreamWaitEvent(to, c->branch_ev[ev], 0));
    return DSMC_OK;
}

template <class T> void launch_inject(dsmc_ctx *c, cudaStream_t stream)
{
    Span sp(c, KID_INJECT);
    k_inject<T><<<grid(c, KID_INJECT), TILE_THREADS, 0, stream>>>(
        c->d_cases, c->d_state, c->d_scratch, c->tt, slots<T>(c, c->cur), c->key, c->cells,
        c->itile_dead, c->obuf, c->ncase, c->d_err);
}

void launch_tile_scan(dsmc_ctx *c, cudaStream_t stream)
{
    Span sp(c, KID_TILE_SCAN);
    k_tile_scan<<<dim3(scan_chunks(c), c->ncase), SCAN_THREADS, 0, stream>>>(
        c->d_state, c->tile_in, c->tile_prefix);
}

// `side`: the buffer that holds the sorted particles of this step.
void launch_collide_select(dsmc_ctx *c, int side, cudaStream_t stream)
{
    Span sp(c, KID_COLLIDE_SELECT);
    k_collide_select<<<grid(c, KID_COLLIDE_SELECT), 256, 0, stream>>>(
        c->d_cases, c->d_state, c->d_scratch, c->tt, c->cells, side, c->coll_list,
        c->total_cells, c->ncase);
}

// MoveParticles: plan + move.
template <class T> int enqueue_move(dsmc_ctx *c, int init_mode)
{
    int s; // k_plan clears the step's scratch and the cell scan's chain
    {
        Span sp(c, KID_PLAN);
        k_plan<<<1, 1024, 0, c->stream>>>(c->d_cases, c->d_state, c->d_scratch, c->tt, c->d_tmp,
                                          c->itile_dead, lb_chain(c, 3), c->ncase, init_mode,
                                          c->d_err);
    }
    if (!init_mode && c->par) {
        if ((s = branch(c, EV_PLAN, c->stream, c->side_stream)))
            return s;
        launch_inject<T>(c, c->side_stream);
        CK(cudaEventRecord(c->branch_ev[EV_INJECT], c->side_stream));
    }
    if (!init_mode) {
        Span sp(c, KID_MOVE);
        k_move<T><<<grid(c, KID_MOVE), TILE_THREADS, move_smem<T>(), c->stream>>>(
            c->d_cases, c->d_state, c->d_scratch, c->tt, slots<T>(c, c->cur), c->key, c->cells,
            c->tile_in, c->tile_dead, c->obuf, c->near_list, c->ncase, c->d_err);
    }
    if (!init_mode) {
        Span sp(c, KID_MOVE_NEAR);
        k_move_near<T><<<c->sms, TILE_THREADS, 0, c->stream>>>(
            c->d_cases, c->d_state, c->d_scratch, c->tt, slots<T>(c, c->cur), c->key, c->cells,
            c->tile_in, c->tile_dead, c->obuf, c->near_list, c->ncase, c->d_err);
    }
    CK(cudaGetLastError());
    return DSMC_OK;
}

// BoundaryConditions: inflow strips, then the swap-with-last removal.
template <class T> int enqueue_boundary(dsmc_ctx *c)
{
    if (c->par) // launched on the side stream by enqueue_move
        CK(cudaStreamWaitEvent(c->stream, c->branch_ev[EV_INJECT], 0));
    else
        launch_inject<T>(c, c->stream);
    {
        Span sp(c, KID_DEAD_SCAN);
        k_dead_scan<<<dim3(scan_chunks(c), c->ncase), SCAN_THREADS, 0, c->stream>>>(
            c->d_state, c->tile_dead, c->tile_dprefix, c->itile_dead, c->itile_dprefix);
    }
    {
        Span sp(c, KID_HOLES);
        k_holes<<<grid(c, KID_HOLES), TILE_THREADS, 0, c->stream>>>(
            c->d_cases, c->d_state, c->d_scratch, c->tt, c->key, c->tile_dead, c->tile_dprefix,
            c->itile_dead, c->itile_dprefix, c->hole_pos, c->hole_oc, c->d_tmp, lb_chain(c, 2),
            c->ncase);
    }
    {
        Span sp(c, KID_TAIL);
        k_tail<T><<<grid(c, KID_TAIL), TILE_THREADS, 0, c->stream>>>(
            c->d_cases, c->d_state, c->d_scratch, c->tt, slots<T>(c, c->cur), c->key, c->cells,
            c->tile_in, lb_chain(c, 2), c->hole_pos, c->hole_oc, c->obuf, c->ncase, c->d_err);
    }
    CK(cudaGetLastError());
    return DSMC_OK;
}

// Indexing: the stable counting sort into the other buffer, then flip.
template <class T> int enqueue_index(dsmc_ctx *c)
{
    const int side = c->cur;
    int s;
    if (c->par) {
        if ((s = branch(c, EV_TAIL, c->stream, c->side_stream)))
            return s;
        launch_tile_scan(c, c->side_stream);
        CK(cudaEventRecord(c->branch_ev[EV_TILE_SCAN], c->side_stream));
    }
    {
        Span sp(c, KID_CELL_SCAN);
        k_cell_scan<<<grid(c, KID_CELL_SCAN), TILE_THREADS, 0, c->stream>>>(
            c->d_cases, c->d_scratch, c->tt, c->cells, side ^ 1, lb_chain(c, 3), c->ncase,
            c->d_err);
    }
    if (c->par) {
        if ((s = branch(c, EV_CELL_SCAN, c->stream, c->side_stream)))
            return s;
        launch_collide_select(c, side ^ 1, c->side_stream);
        CK(cudaEventRecord(c->branch_ev[EV_SELECT], c->side_stream));
    } else {
        launch_tile_scan(c, c->stream);
    }
    {
        Span sp(c, KID_OLIST);
        k_olist<<<grid(c, KID_OLIST), 256, 0, c->stream>>>(c->d_cases, c->d_state, c->d_scratch,
                                                      c->obuf, c->key, c->cells, c->olist,
                                                      c->d_pbases, c->ncase, c->d_err);
    }
    {
        Span sp(c, KID_CELL_FIX);
        k_cell_fix<<<grid(c, KID_CELL_FIX), 256, 0, c->stream>>>(c->d_cases, c->d_state, c->tt,
                                                             c->cells, side, c->key, c->olist,
                                                             c->total_cells, c->ncase, c->d_err);
    }
    if (c->par)
        CK(cudaStreamWaitEvent(c->stream, c->branch_ev[EV_TILE_SCAN], 0));
    {
        Span sp(c, KID_SCATTER);
        k_scatter<T><<<grid(c, KID_SCATTER), SC_THREADS, scatter_smem<T>(), c->stream>>>(
            c->d_cases, c->d_state, c->tt, slots<T>(c, side), slots<T>(c, side ^ 1), c->key,
            c->cells, c->tile_prefix, c->ncase, c->d_err);
    }
    CK(cudaGetLastError());
    c->cur ^= 1;
    return DSMC_OK;
}

// `finish`: k_sample also ends the step (a full step; the staged calls end
// it with k_finish).
template <class T> int enqueue_collide(dsmc_ctx *c, int do_collide, int do_sample, int finish = 0)
{
    if (do_collide) {
        if (c->par) // launched on the side stream by enqueue_index
            CK(cudaStreamWaitEvent(c->stream, c->branch_ev[EV_SELECT], 0));
        else
            launch_collide_select(c, c->cur, c->stream);
        {
            Span sp(c, KID_COLLIDE);
            k_collide_pairs<T><<<2 * c->sms, 128, 0, c->stream>>>(
                c->d_cases, c->d_state, c->d_scratch, c->tt, slots<T>(c, c->cur), c->cells,
                c->cur, c->coll_list, c->ncase);
        }
    }
    if (do_sample) {
        Span sp(c, KID_SAMPLE);
        k_sample<T><<<grid(c, KID_SAMPLE), SAMPLE_THREADS, sample_smem<T>(), c->stream>>>(
            c->d_cases, c->d_state, c->tt, slots<T>(c, c->cur), c->cells, c->cur, c->ncase,
            finish, finish ? c->d_counters : nullptr, c->d_err);
    }
    CK(cudaGetLastError());
    return DSMC_OK;
}

int enqueue_finish(dsmc_ctx *c, int init_mode, int did_sample, int end_step)
{
    Span sp(c, KID_FINISH);
    k_finish<<<1, 256, 0, c->stream>>>(c->d_cases, c->d_state, c->ncase, init_mode, did_sample,
                                        end_step);
    CK(cudaGetLastError());
    return DSMC_OK;
}

template <class T> int enqueue_step(dsmc_ctx *c)
{
    int s;
    if ((s = enqueue_move<T>(c, 0)))
        return s;
    if ((s = enqueue_boundary<T>(c)))
        return s;
    if ((s = enqueue_index<T>(c)))
        return s;
    return enqueue_collide<T>(c, 1, 1, 1); // k_sample ends the step
}

int dispatch_step(dsmc_ctx *c)
{
    return c->precision == DSMC_FP32 ? enqueue_step<float>(c) : enqueue_step<double>(c);
}

int build_graphs(dsmc_ctx *c)
{
    if (c->side_stream == nullptr) {
        CK(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
        for (auto &e : c->branch_ev)
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    for (int side = 0; side < 2; ++side) {
        const int saved = c->cur;
        c->cur = side;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->par = true;
        const int s = dispatch_step(c);
        c->par = false;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->cur = saved;
        if (s)
            return s;
        if (e != cudaSuccess)
            return DSMC_ERR_CUDA;
        e = cudaGraphInstantiate(&c->graph[side], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess)
            return DSMC_ERR_CUDA;
    }
    return DSMC_OK;
}

// ---- the persistent step ---------------------------------------------------

template <class T> StepArgs<T> step_args(dsmc_ctx *c)
{
    StepArgs<T> a{};
    a.cases = c->d_cases;
    a.st = c->d_state;
    a.sc = c->d_scratch;
    a.tt = c->tt;
    a.buf0 = slots<T>(c, 0);
    a.buf1 = slots<T>(c, 1);
    a.key = c->key;
    a.cells = c->cells;
    a.tile_in = c->tile_in;
    a.tile_prefix = c->tile_prefix;
    a.tile_dead = c->tile_dead;
    a.tile_dprefix = c->tile_dprefix;
    a.itile_dead = c->itile_dead;
    a.itile_dprefix = c->itile_dprefix;
    a.tail_chain = lb_chain(c, 2);
    a.cell_chain = lb_chain(c, 3);
    a.hole_pos = c->hole_pos;
    a.hole_oc = c->hole_oc;
    a.obuf = c->obuf;
    a.near_list = c->near_list;
    a.olist = c->olist;
    a.coll_list = c->coll_list;
    a.rec = c->d_counters;
    a.tmp = c->d_tmp;
    a.pbases = c->d_pbases;
    a.total_cells = c->total_cells;
    a.ncase = c->ncase;
    constexpr int64_t chunk = PERSIST_THREADS * SCAN_VEC;
    a.scan_chunks = static_cast<int>((c->max_case_tiles + chunk - 1) / chunk);
    a.err = c->d_err;
    a.gsync = c->d_gsync;
    a.wait_ns = c->p_wait_ns;
    a.phase_ns = c->d_phase_ns;
    return a;
}

// The graph of one persistent launch: zero the barrier state, then the
// cooperative kernel for n_steps steps from buffer `side`.
template <class T> int persistent_graph(dsmc_ctx *c, int n_steps, int side, cudaGraphExec_t *out)
{
    for (const auto &pg : c->pgraphs)
        if (pg.n_steps == n_steps && pg.side == side) {
            *out = pg.exec;
            return DSMC_OK;
        }
    StepArgs<T> a = step_args<T>(c);
    void *args[] = {&a, &n_steps, &side};
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaMemsetParams mp{};
    mp.dst = c->d_gsync;
    mp.value = 0;
    mp.elementSize = 4;
    mp.width = sizeof(GridSync) / 4;
    mp.height = 1;
    mp.pitch = sizeof(GridSync);
    cudaGraphNode_t mn = nullptr, kn = nullptr;
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void *>(k_persistent<T>);
    kp.gridDim = dim3(c->p_ctas * c->sms);
    kp.blockDim = dim3(PERSIST_THREADS);
    kp.sharedMemBytes = static_cast<unsigned>(persist_smem<T>());
    kp.kernelParams = args;
    cudaLaunchAttributeValue v{};
    v.cooperative = 1;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphAddMemsetNode(&mn, g, nullptr, 0, &mp);
    if (e == cudaSuccess)
        e = cudaGraphAddKernelNode(&kn, g, &mn, 1, &kp);
    if (e == cudaSuccess)
        e = cudaGraphKernelNodeSetAttribute(kn, cudaLaunchAttributeCooperative, &v);
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&exec, g, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        return DSMC_ERR_UNSUPPORTED;
    }
    if (c->pgraphs.size() >= 8) { // keep the most recent few
        cudaGraphExecDestroy(c->pgraphs.front().exec);
        cudaGraphDestroy(c->pgraphs.front().g);
        c->pgraphs.erase(c->pgraphs.begin());
    }
    c->pgraphs.push_back({n_steps, side, g, exec});
    *out = exec;
    return DSMC_OK;
}

// n_steps full steps of every case in one persistent launch.
template <class T> int persistent_steps(dsmc_ctx *c, int n_steps)
{
    if (n_steps == 0)
        return DSMC_OK;
    if (c->p_graph) {
        cudaGraphExec_t exec = nullptr;
        const int s = persistent_graph<T>(c, n_steps, c->cur, &exec);
        if (s == DSMC_OK) {
            CK(cudaGraphLaunch(exec, c->stream));
            c->cur = (c->cur + n_steps) & 1;
            return DSMC_OK;
        }
        c->p_graph = false; // graphs of cooperative kernels refused: launch directly
    }
    const StepArgs<T> a = step_args<T>(c);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(c->p_ctas * c->sms);
    cfg.blockDim = dim3(PERSIST_THREADS);
    cfg.dynamicSmemBytes = persist_smem<T>();
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaMemsetAsync(c->d_gsync, 0, sizeof(GridSync), c->stream));
    CK(cudaLaunchKernelEx(&cfg, k_persistent<T>, a, n_steps, c->cur));
    c->cur = (c->cur + n_steps) & 1;
    return DSMC_OK;
}

// Constants of one case, computed on the host with the reference expressions.
// Largest float <= v and smallest float >= v.
float float_down(double v)
{
    float f = static_cast<float>(v);
    if (static_cast<double>(f) > v)
        f = std::nextafter(f, -INFINITY);
    return f;
}
float float_up(double v)
{
    float f = static_cast<float>(v);
    if (static_cast<double>(f) < v)
        f = std::nextafter(f, INFINITY);
    return f;
}

// FP32 constants of the free-flight pass (see CaseDev).  The float cell
// estimate q' differs from (x - X1) / DX by at most e inside the grid: the
// float difference, the product and 1/DX each round by at most 2^-24
// relative (3 |q| 2^-24 in all), and X1 rounded to float adds 2^-24 |X1| / DX;
// e is doubled, plus 1e-9 for the FP64 quotient of the reference.
void set_float_bounds(CaseDev &c, const dsmc_params &p)
{
    c.fx1 = static_cast<float>(c.x1);
    c.fy1 = static_cast<float>(c.y1);
    c.finv_dx = static_cast<float>(c.inv_dx);
    c.finv_dy = static_cast<float>(c.inv_dy);
    const double qmax = static_cast<double>(std::max(p.nx, p.ny)) + 1.0;
    const double shift = std::max(std::fabs(c.x1) / c.dx, std::fabs(c.y1) / c.dy);
    const double err = std::ldexp(3.01 * qmax + 1.01 * shift + 1.0, -24);
    // Half-width of the certain window of r - 0.5, less 2^-20 for the
    // rounding of that difference; off (negative) for grids of 2^20 cells or
    // more per side, where the rounding constant's range is not assured.
    c.fcell_hw = std::max(p.nx, p.ny) < (1 << 20)
                     ? static_cast<float>(0.5 - (2.0 * err + 1e-9) - std::ldexp(1.0, -20))
                     : -1.0f;
    c.dom_lo[0] = float_down(c.x1);
    c.dom_lo[1] = float_down(c.y1);
    c.dom_hi[0] = float_up(c.x2);
    c.dom_hi[1] = float_up(c.y2);
    c.fnear_lo[0] = float_down(c.near_lo[0]);
    c.fnear_lo[1] = float_down(c.near_lo[1]);
    c.fnear_hi[0] = float_up(c.near_hi[0]);
    c.fnear_hi[1] = float_up(c.near_hi[1]);
}

CaseDev make_case(const dsmc_params &p, const dsmc_derived &d)
{
    CaseDev c{};
    c.x1 = p.x1;
    c.x2 = p.x2;
    c.y1 = p.y1;
    c.y2 = p.y2;
    c.dz = p.dz;
    c.dx = d.dx;
    c.dy = d.dy;
    c.dv = d.dv;
    c.dt = p.dt;
    c.inv_dx = 1.0 / d.dx;
    c.inv_dy = 1.0 / d.dy;
    double near_margin;
    {
        double mag = 1.0;
        const double v[] = {p.x1, p.x2, p.y1, p.y2, p.box_x - p.box_width / 2.0,
                            p.box_x + p.box_width / 2.0, p.box_y - p.box_height / 2.0,
                            p.box_y + p.box_height / 2.0};
        for (double a : v)
            mag = std::max(mag, std::fabs(a));
        c.cull = 1e-9 * mag;
        near_margin = c.cull + std::ldexp(mag, -20);
    }
    c.box_lo[0] = p.box_x - p.box_width / 2.0; // Geometry.cpp:184
    c.box_lo[1] = p.box_y - p.box_height / 2.0;
    c.box_hi[0] = p.box_x + p.box_width / 2.0; // Geometry.cpp:185
    c.box_hi[1] = p.box_y + p.box_height / 2.0;
    {
        const double m = near_margin;
        c.near_lo[0] = c.box_lo[0] - m;
        c.near_lo[1] = c.box_lo[1] - m;
        c.near_hi[0] = c.box_hi[0] + m;
        c.near_hi[1] = c.box_hi[1] + m;
    }
    c.box_x = p.box_x;
    c.box_y = p.box_y;
    c.box_hw = p.box_width / 2.0; // Geometry.cpp:175-176
    c.box_hh = p.box_height / 2.0;
    const double m = d.molecule_mass;
    c.rtw = K_BOLTZMANN * p.t_wall / m; // Boundary.cpp:213 (and :258)
    c.sqrt_rtw = std::sqrt(c.rtw);
    c.cll_an = p.cll_normal;
    c.cll_at = p.cll_tangential;
    c.cll_var_n = p.cll_normal * c.rtw; // Boundary.cpp:268
    c.cll_var_t = p.cll_tangential * c.rtw; // Boundary.cpp:276
    c.cll_keep_n = std::sqrt(1.0 - p.cll_normal);
    c.cll_keep_t = std::sqrt(1.0 - p.cll_tangential);
    c.mass = m;
    c.drag_scale = d.weight * m; // Boundary.cpp:318
    c.weight = d.weight;
    c.sigma_ref = d.sigma_ref;
    c.omega = d.omega;
    c.cr_ref = d.cr_ref;
    c.sc_max = d.sc_max;
    c.ux_free = d.ux_free;
    c.uy_free = d.uy_free;
    c.rt_free = K_BOLTZMANN * p.t_free / m; // Boundary.cpp:53
    // One rank owns all cells: LocalX1 = X1 + 0 * DX, LocalX2 = X1 + NX * DX
    // (MPIManager.cpp:216-229).
    const double lx1 = p.x1 + 0 * d.dx, lx2 = p.x1 + p.nx * d.dx;
    const double ly1 = p.y1 + 0 * d.dy, ly2 = p.y1 + p.ny * d.dy;
    const double strips[5][4] = {
        {p.x1 - p.dl, ly1, p.x1, ly2},  // Boundary.cpp:100-113
        {p.x2, ly1, p.x2 + p.dl, ly2},  // :120-133
        {lx1, p.y1 - p.dl, lx2, p.y1},  // :140-153
        {lx1, p.y2, lx2, p.y2 + p.dl},  // :160-173
        {lx1, ly1, lx2, ly2},           // Initialization.cpp:302-310
    };
    for (int s = 0; s < 5; ++s) {
        for (int k = 0; k < 4; ++k)
            c.strip[s][k] = strips[s][k];
        // Boundary.cpp:62-63
        const double v = (strips[s][2] - strips[s][0]) * (strips[s][3] - strips[s][1]) * p.dz;
        c.strip_navg[s] = p.n_free * v / d.weight;
    }
    c.nx = p.nx;
    c.ny = p.ny;
    c.wall_model = p.wall_model;
    c.first_sampling_step = p.first_sampling_step;
    c.sampling_period = p.sampling_period;
    c.max_per_cell = p.max_particles_in_cell;
    c.ncell = p.nx * p.ny;
    c.key0 = static_cast<uint32_t>(p.seed);
    c.key1 = static_cast<uint32_t>(p.seed >> 32);
    set_float_bounds(c, p);
    return c;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

template <class T> int occupancy_grids(dsmc_ctx *c)
{
    int b = 0;
    auto occ = [&](int kid, int occupancy) {
        c->ctas_max[kid] = std::max(1, occupancy);
        c->ctas[kid] = c->ctas_max[kid];
    };
    CK(cudaFuncSetAttribute(k_move<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(move_smem<T>())));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_move<T>, TILE_THREADS,
                                                     move_smem<T>()));
    occ(KID_MOVE, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_inject<T>, TILE_THREADS, 0));
    occ(KID_INJECT, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_tail<T>, TILE_THREADS, 0));
    occ(KID_TAIL, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cell_scan, TILE_THREADS, 0));
    occ(KID_CELL_SCAN, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_holes, TILE_THREADS, 0));
    occ(KID_HOLES, b);
    CK(cudaFuncSetAttribute(k_scatter<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(scatter_smem<T>())));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_scatter<T>, SC_THREADS,
                                                     scatter_smem<T>()));
    occ(KID_SCATTER, b);
    CK(cudaFuncSetAttribute(k_sample<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(sample_smem<T>())));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sample<T>, SAMPLE_THREADS,
                                                     sample_smem<T>()));
    occ(KID_SAMPLE, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_collide_select, 256, 0));
    occ(KID_COLLIDE_SELECT, b);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_olist, 256, 0));
    occ(KID_OLIST, b);
    c->ctas[KID_OLIST] = std::min(4, c->ctas_max[KID_OLIST]);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cell_fix, 256, 0));
    occ(KID_CELL_FIX, b);
    c->ctas[KID_CELL_FIX] = std::min(8, c->ctas_max[KID_CELL_FIX]);
    // The persistent step: every CTA of its grid must be resident at once.
    int coop = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    c->coop = coop != 0;
    CK(cudaFuncSetAttribute(k_persistent<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(persist_smem<T>())));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_persistent<T>, PERSIST_THREADS,
                                                     persist_smem<T>()));
    c->p_ctas_max = b;
    c->p_ctas = b;
    return DSMC_OK;
}

void free_ctx(dsmc_ctx *c)
{
    for (auto &g : c->graph)
        if (g)
            cudaGraphExecDestroy(g);
    for (auto &pg : c->pgraphs) {
        cudaGraphExecDestroy(pg.exec);
        cudaGraphDestroy(pg.g);
    }
    for (auto e : c->branch_ev)
        if (e)
            cudaEventDestroy(e);
    for (auto e : c->field_ev)
        if (e)
            cudaEventDestroy(e);
    for (void *h : c->field_stage)
        if (h)
            cudaFreeHost(h);
    if (c->side_stream)
        cudaStreamDestroy(c->side_stream);
    for (auto &t : c->timed) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : c->event_pool)
        cudaEventDestroy(e);
    if (c->arena) // every device buffer of the context lives in it
        cudaFree(c->arena);
    if (c->own_stream && c->stream)
        cudaStreamDestroy(c->stream);
    delete c;
}

int read_state(dsmc_ctx *c, std::vector<CaseState> &st)
{
    st.resize(c->ncase);
    CK(cudaMemcpyAsync(st.data(), c->d_state, sizeof(CaseState) * c->ncase,
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int device_error(dsmc_ctx *c)
{
    int err = 0;
    CK(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return err;
}

// ---- upload: convert host FP64 state into one case's slots, then re-sort ---

template <class T>
__global__ void k_upload_case(const double *x, const double *y, const double *vx, const double *vy,
                              const double *vz, int64_t n, Slots<T> p, int64_t pbase)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        p.x[pbase + i] = Store<T>::rn(x[i]);
        p.y[pbase + i] = Store<T>::rn(y[i]);
        p.vx[pbase + i] = Store<T>::rn(vx[i]);
        p.vy[pbase + i] = Store<T>::rn(vy[i]);
        p.vz[pbase + i] = Store<T>::rn(vz[i]);
    }
}

// Every slot of every case becomes an out-of-range particle of its cell, so
// the sort orders all cases from scratch (stable in slot order).
template <class T>
__global__ void k_rekey(const CaseDev *cases, CaseState *st, StepScratch *sc, Slots<T> p,
                        uint32_t *key, Cells cells, uint32_t *obuf, int ncase, int *err)
{
    for (int ci = 0; ci < ncase; ++ci) {
        const CaseDev &c = cases[ci];
        const int64_t n = st[ci].n_old;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
             i += (int64_t)gridDim.x * blockDim.x) {
            const int64_t g = c.pbase + i;
            const int32_t cl = cell_of(c, static_cast<double>(p.x[g]), static_cast<double>(p.y[g]));
            if (cl < 0) {
                report_error(err, DSMC_ERR_EXCHANGE);
                key[g] = KEY_DEAD | KEY_CELL;
                continue;
            }
            key[g] = static_cast<uint32_t>(c.cbase + cl);
            atomicAdd(cells.n_o + c.cbase + cl, 1);
            obuf[atomicAdd(&sc->obuf_count, 1u)] = static_cast<uint32_t>(g);
        }
    }
}

__global__ void k_resort_plan(CaseState *st, StepScratch *sc, TileTables tt, int ncase)
{
    if (threadIdx.x != 0)
        return;
    int32_t run = 0;
    for (int i = 0; i < ncase; ++i) {
        CaseState &s = st[i];
        s.n_total = s.n_old;
        s.dead_old = s.dead_total = 0;
        s.n_keep = s.n_old;
        s.n_holes = 0;
        s.n_move_tiles = 0;
        s.move_tile0 = 0;
        s.n_tail_tiles = 0;
        tt.scatter0[i] = run;
        run += static_cast<int32_t>((s.n_keep + TILE - 1) / TILE);
    }
    tt.scatter0[ncase] = run;
    sc->total_tail_tiles = 0;
}

template <class T> int resort_all(dsmc_ctx *c)
{
    int s = clear_step_scratch(c);
    if (s)
        return s;
    const int side = c->cur;
    CK(cudaMemsetAsync(c->cells.start[side], 0, sizeof(int32_t) * c->total_cells, c->stream));
    CK(cudaMemsetAsync(c->cells.n_in, 0, sizeof(int32_t) * c->total_cells, c->stream));
    k_resort_plan<<<1, 32, 0, c->stream>>>(c->d_state, c->d_scratch, c->tt, c->ncase);
    k_rekey<T><<<4 * c->sms, 256, 0, c->stream>>>(c->d_cases, c->d_state, c->d_scratch,
                                                   slots<T>(c, side), c->key, c->cells, c->obuf,
                                                   c->ncase, c->d_err);
    CK(cudaGetLastError());
    if ((s = enqueue_index<T>(c)))
        return s;
    return enqueue_finish(c, 1, 0, 0);
}

// ---- warm start: particles from the local Maxwellian of a field ------------
//
// Cell l of a case (x-major, k * NY + m) with field (n, ux, uy, T) gets
// floor(n DV / W) + Bernoulli(rest) candidates (draw 0 of the cell's WARM
// stream, step 0); candidate j sits at X1 + (k + u) DX, Y1 + (m + u') DY
// (draws 1 + 2j, 2 + 2j) and moves with ux, uy, 0 plus Gaussians of variance
// k T / m (the cell's WARM stream at step 1, as vrand_MB draws them).  A
// candidate whose stored position is inside the box is dropped, as
// RemoveParticlesInsideBox does after the cold fill.

__device__ __forceinline__ int warm_candidates(const CaseDev &c, const double *f, int cl)
{
    const double lam = f[0] * c.dv / c.weight;
    if (!(lam > 0.0) || !(lam < 1e9))
        return 0;
    dsmc_stream r;
    open_stream(r, c, DSMC_RNG_WARM, 0, static_cast<uint32_t>(cl));
    const double fl = floor(lam);
    return static_cast<int>(fl) + (uniform(r) < lam - fl ? 1 : 0);
}

template <class T>
__device__ __forceinline__ void warm_position(const CaseDev &c, int cl, dsmc_stream &r, T &x, T &y)
{
    const int k = cl / c.ny, m = cl % c.ny;
    x = clamp_into<T>(Store<T>::rn(c.x1 + (k + uniform(r)) * c.dx), c.x1, c.x2);
    y = clamp_into<T>(Store<T>::rn(c.y1 + (m + uniform(r)) * c.dy), c.y1, c.y2);
}

// Survivors per cell into cnt[global cell].  `stride` doubles per cell.
template <class T>
__global__ void k_warm_count(const CaseDev *cases, int ncase, const double *field, int stride,
                             int32_t *cnt)
{
    int64_t f0 = 0;
    for (int ci = 0; ci < ncase; ++ci) {
        const CaseDev &c = cases[ci];
        for (int cl = blockIdx.x * blockDim.x + threadIdx.x; cl < c.ncell;
             cl += gridDim.x * blockDim.x) {
            const double *f = field + stride * (f0 + cl);
            const int nc = warm_candidates(c, f, cl);
            dsmc_stream r;
            open_stream(r, c, DSMC_RNG_WARM, 0, static_cast<uint32_t>(cl));
            uniform(r); // the count draw
            int keep = 0;
            for (int j = 0; j < nc; ++j) {
                T x, y;
                warm_position<T>(c, cl, r, x, y);
                keep += inside_box(c, static_cast<double>(x), static_cast<double>(y)) ? 0 : 1;
            }
            cnt[c.cbase + cl] = keep;
        }
        f0 += c.ncell;
    }
}

// Per case (one CTA each): exclusive prefix of the survivors and n_old.
__global__ void __launch_bounds__(SCAN_THREADS)
    k_warm_scan(const CaseDev *cases, CaseState *st, const int32_t *cnt, int32_t *off, int *err)
{
    constexpr int PER = 8;
    const CaseDev &c = cases[blockIdx.x];
    int64_t carry = 0;
    for (int b = 0; b < c.ncell; b += SCAN_THREADS * PER) {
        const int i0 = b + threadIdx.x * PER;
        int v[PER];
        int sum = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            v[k] = i0 + k < c.ncell ? cnt[c.cbase + i0 + k] : 0;
            sum += v[k];
        }
        int tot;
        int64_t run = carry + block_exclusive<int, SCAN_THREADS>(sum, tot);
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            if (i0 + k < c.ncell)
                off[c.cbase + i0 + k] = static_cast<int32_t>(run);
            run += v[k];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) {
        if (carry > c.cap) {
            report_error(err, DSMC_ERR_CAPACITY);
            carry = 0;
        }
        st[blockIdx.x].n_old = carry;
    }
}

// Writes the survivors of every cell from its offset, in cell order.
// With stride 4 the velocity is (ux, uy, 0) plus isotropic Gaussians of
// variance k T / m; with stride 7 the field gives the temperature tensor
// (Txx, Tyy, Tzz, Txy) and the Gaussians are correlated through its
// Cholesky factor (the xz and yz entries vanish in this 2-D flow).  With
// stride 8 the field is (n, alpha, ux_r, uy_r, Txx_r, Tyy_r, Tzz_r, Txy_r),
// a mixture of two populations: with probability alpha (one uniform of the
// velocity stream first) a particle is drawn from the case's freestream
// Maxwellian, else from the Gaussian of mean (ux_r, uy_r, 0) whose
// covariance is k / m times that temperature tensor (Cholesky as above).
template <class T>
__global__ void k_warm_fill(const CaseDev *cases, const CaseState *st, int ncase,
                            const double *field, int stride, const int32_t *off, Slots<T> p)
{
    int64_t f0 = 0;
    for (int ci = 0; ci < ncase; ++ci) {
        const CaseDev &c = cases[ci];
        const bool fits = st[ci].n_old > 0;
        for (int cl = blockIdx.x * blockDim.x + threadIdx.x; fits && cl < c.ncell;
             cl += gridDim.x * blockDim.x) {
            const double *f = field + stride * (f0 + cl);
            const int nc = warm_candidates(c, f, cl);
            if (nc == 0)
                continue;
            const bool mix = stride == 8;
            const double ux = mix ? f[2] : f[1], uy = mix ? f[3] : f[2];
            const double var = K_BOLTZMANN * fmax(f[3], 0.0) / c.mass;
            const double alpha = mix ? f[1] : 0.0;
            double l11 = 0.0, l21 = 0.0, l22 = 0.0, l33 = 0.0;
            if (stride == 7 || mix) {
                const double *tt = f + (mix ? 4 : 3); // Txx, Tyy, Tzz, Txy
                const double kb = K_BOLTZMANN / c.mass;
                l11 = sqrt(fmax(kb * tt[0], 0.0));
                l21 = l11 > 0.0 ? kb * tt[3] / l11 : 0.0;
                l22 = sqrt(fmax(kb * tt[1] - l21 * l21, 0.0));
                l33 = sqrt(fmax(kb * tt[2], 0.0));
            }
            dsmc_stream r, rv;
            open_stream(r, c, DSMC_RNG_WARM, 0, static_cast<uint32_t>(cl));
            open_stream(rv, c, DSMC_RNG_WARM, 1, static_cast<uint32_t>(cl));
            uniform(r);
            int64_t g = c.pbase + off[c.cbase + cl];
            for (int j = 0; j < nc; ++j) {
                T x, y;
                warm_position<T>(c, cl, r, x, y);
                double vx, vy, vz;
                if (mix && uniform(rv) < alpha) { // the freestream population
                    vx = frand_gaussian(rv, c.ux_free, c.rt_free);
                    vy = frand_gaussian(rv, c.uy_free, c.rt_free);
                    vz = frand_gaussian(rv, 0.0, c.rt_free);
                } else if (stride == 7 || mix) {
                    const double z1 = frand_gaussian(rv, 0.0, 1.0);
                    const double z2 = frand_gaussian(rv, 0.0, 1.0);
                    const double z3 = frand_gaussian(rv, 0.0, 1.0);
                    vx = ux + l11 * z1;
                    vy = uy + l21 * z1 + l22 * z2;
                    vz = l33 * z3;
                } else {
                    vx = frand_gaussian(rv, ux, var);
                    vy = frand_gaussian(rv, uy, var);
                    vz = frand_gaussian(rv, 0.0, var);
                }
                if (inside_box(c, static_cast<double>(x), static_cast<double>(y)))
                    continue;
                p.x[g] = x;
                p.y[g] = y;
                p.vx[g] = Store<T>::rn(vx);
                p.vy[g] = Store<T>::rn(vy);
                p.vz[g] = Store<T>::rn(vz);
                ++g;
            }
        }
        f0 += c.ncell;
    }
}

template <class T>
int warm_fill(dsmc_ctx *c, const double *dfield, int stride, int32_t *cnt, int32_t *off)
{
    const int grid = 4 * c->sms;
    k_warm_count<T><<<grid, 256, 0, c->stream>>>(c->d_cases, c->ncase, dfield, stride, cnt);
    k_warm_scan<<<c->ncase, SCAN_THREADS, 0, c->stream>>>(c->d_cases, c->d_state, cnt, off,
                                                           c->d_err);
    k_warm_fill<T><<<grid, 256, 0, c->stream>>>(c->d_cases, c->d_state, c->ncase, dfield, stride,
                                                off, slots<T>(c, c->cur));
    CK(cudaGetLastError());
    return resort_all<T>(c);
}

__global__ void k_fields_out(const Cells cells, int cbase, int ncell, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += gridDim.x * blockDim.x) {
        const int64_t cg = cbase + i;
        const int64_t S = cells.acc_stride;
        auto A = [&](int m) { return cells.acc[m * S + cg]; };
        double *o = out + 17 * static_cast<int64_t>(i);
        o[0] = A(ACC_NP);
        o[1] = A(ACC_V0);
        o[2] = A(ACC_V1);
        o[3] = A(ACC_V2);
        o[4] = A(ACC_VV00);
        o[5] = A(ACC_VV01);
        o[6] = A(ACC_VV02);
        o[7] = A(ACC_VV01);
        o[8] = A(ACC_VV11);
        o[9] = A(ACC_VV12);
        o[10] = A(ACC_VV02);
        o[11] = A(ACC_VV12);
        o[12] = A(ACC_VV22);
        o[13] = A(ACC_V2V0);
        o[14] = A(ACC_V2V1);
        o[15] = A(ACC_V2V2);
        o[16] = A(ACC_NC);
    }
}

__global__ void k_fields_in(Cells cells, int cbase, int ncell, const double *in)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += gridDim.x * blockDim.x) {
        const int64_t cg = cbase + i;
        const int64_t S = cells.acc_stride;
        const double *o = in + 17 * static_cast<int64_t>(i);
        const int map[ACC_COUNT] = {0, 1, 2, 3, 4, 5, 6, 8, 9, 12, 13, 14, 15, 16};
        for (int m = 0; m < ACC_COUNT; ++m)
            cells.acc[m * S + cg] = o[map[m]];
    }
}

__global__ void k_download_case(Slots<float> p, int64_t pbase, int64_t n, double *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        out[i] = p.x[pbase + i];
        out[n + i] = p.y[pbase + i];
        out[2 * n + i] = p.vx[pbase + i];
        out[3 * n + i] = p.vy[pbase + i];
        out[4 * n + i] = p.vz[pbase + i];
    }
}

// ---- unit kernels ------------------------------------------------------------

__global__ void k_unit_intersect(CaseDev c, int64_t n, const double *x, const double *y,
                                 const double *dx, const double *dy, int32_t *hit, double *t,
                                 double *nx, double *ny)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double th = 0.0, a = 0.0, b = 0.0;
        const bool h = intersect_box(c, x[i], y[i], dx[i], dy[i], th, a, b);
        hit[i] = h ? 1 : 0;
        t[i] = h ? th : 0.0;
        nx[i] = h ? a : 0.0;
        ny[i] = h ? b : 0.0;
    }
}

__global__ void k_unit_inside(CaseDev c, int64_t n, const double *x, const double *y,
                              int32_t *inside)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        inside[i] = inside_box(c, x[i], y[i]) ? 1 : 0;
}

__global__ void k_unit_scatter(CaseDev c, int64_t n, double *v, const double *nx,
                               const double *ny, uint32_t kind, uint32_t step,
                               const uint32_t *entity)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double w[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        dsmc_stream r;
        open_stream(r, c, kind, step, entity[i]);
        wall_interaction(r, c, w, nx[i], ny[i]);
        v[3 * i] = w[0];
        v[3 * i + 1] = w[1];
        v[3 * i + 2] = w[2];
    }
}

int resolve_timings(dsmc_ctx *c)
{
    if (c->timed.empty())
        return DSMC_OK;
    CK(cudaStreamSynchronize(c->stream));
    for (auto &t : c->timed) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, t.a, t.b));
        c->kernel_ms[t.kid] += ms;
        c->kernel_launches[t.kid] += 1;
        c->event_pool.push_back(t.a);
        c->event_pool.push_back(t.b);
    }
    c->timed.clear();
    return DSMC_OK;
}


void drop_graphs(dsmc_ctx *c)
{
    for (auto &g : c->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto &pg : c->pgraphs) {
        cudaGraphExecDestroy(pg.exec);
        cudaGraphDestroy(pg.g);
    }
    c->pgraphs.clear();
}

} // namespace

extern "C" {

int dsmc_ctx_create(const dsmc_params *cases, const dsmc_derived *derived, int n_cases,
                    void *cuda_stream, dsmc_ctx **out)
{
    if (cases == nullptr || out == nullptr || n_cases < 1 || n_cases > 65535)
        return DSMC_ERR_ARGUMENT; // 65535: the cases are a grid dimension of the scans
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return DSMC_ERR_NO_DEVICE;
    auto *c = new dsmc_ctx();
    c->ncase = n_cases;
    c->precision = cases[0].precision;
    c->params.assign(cases, cases + n_cases);
    c->derived.resize(n_cases);
    for (int i = 0; i < n_cases; ++i) {
        if (cases[i].precision != c->precision) {
            delete c;
            return DSMC_ERR_ARGUMENT; // one storage precision per context
        }
        const int s = dsmc_setup(&cases[i], &c->derived[i]);
        if (s) {
            delete c;
            return s;
        }
        if (derived != nullptr)
            c->derived[i] = derived[i];
    }
    cudaGetDevice(&c->device);
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    if (cuda_stream != nullptr) {
        c->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return DSMC_ERR_CUDA;
        }
        c->own_stream = true;
    }

    // Layout: each case owns a TILE-aligned slot range and ncell + 1 cell ids.
    c->hcases.resize(n_cases);
    int64_t slot = 0;
    int cell = 0, cell_tiles = 0, cblocks = 0;
    std::vector<int32_t> cell0(n_cases + 1), cblock0(n_cases + 1), cellbase(n_cases + 1);
    std::vector<int64_t> pbases(n_cases);
    int max_tiles = 0;
    int64_t max_cap = 0;
    for (int i = 0; i < n_cases; ++i) {
        const dsmc_params &p = cases[i];
        CaseDev cd = make_case(p, c->derived[i]);
        int64_t cap = p.capacity;
        if (cap <= 0) {
            // Freestream count plus room for compression near the box and
            // one step of inflow per strip.
            double inflow = 0.0;
            for (int s = 0; s < 4; ++s)
                inflow += cd.strip_navg[s] + 10.0 * std::sqrt(cd.strip_navg[s] + 1.0);
            cap = static_cast<int64_t>(1.5 * p.npc_free * p.nx * p.ny + 2.0 * inflow +
                                       cd.strip_navg[4] * 0.0) + 4096;
            cap = std::max<int64_t>(cap, static_cast<int64_t>(
                                              cd.strip_navg[4] + 10.0 * std::sqrt(cd.strip_navg[4]) +
                                              4096));
        }
        cap = round_up(cap, TILE);
        max_cap = std::max(max_cap, cap);
        cd.pbase = slot;
        cd.cap = cap;
        cd.cbase = cell;
        pbases[i] = slot;
        cellbase[i] = cell;
        cell0[i] = cell_tiles;
        cblock0[i] = cblocks;
        slot += cap;
        cell += cd.ncell + 1;
        cell_tiles += (cd.ncell + CELL_TILE - 1) / CELL_TILE;
        cblocks += (cd.ncell + COLLIDE_CELLS - 1) / COLLIDE_CELLS;
        max_tiles += static_cast<int>(cap / TILE) + 1;
        c->max_case_tiles = std::max<int64_t>(c->max_case_tiles, cap / TILE + 2);
        c->hcases[i] = cd;
    }
    cellbase[n_cases] = cell;
    cell0[n_cases] = cell_tiles;
    cblock0[n_cases] = cblocks;
    c->total_slots = slot;
    c->total_cells = cell;
    c->total_cell_tiles = cell_tiles;
    c->max_slot_tiles = max_tiles;
    // Keys hold cell ids and slots in 30 bits; global slots fit 32 bits.
    if (slot >= (int64_t(1) << 32) - 1 || cell >= (1 << 30) - 1 || max_cap >= (int64_t(1) << 30)) {
        free_ctx(c);
        return DSMC_ERR_ARGUMENT;
    }

    const size_t esz = c->precision == DSMC_FP32 ? sizeof(float) : sizeof(double);
    // Every device buffer of the context is carved from one allocation (one
    // cudaMalloc maps the whole range at once: creating and destroying a
    // context of a few GB then takes about a millisecond instead of tens).
    // Buffers start on 256-byte boundaries.
    std::vector<std::pair<void **, size_t>> carve;
    auto alloc = [&](void **p, size_t bytes) -> bool {
        carve.emplace_back(p, (std::max<size_t>(bytes, 16) + 255) & ~size_t(255));
        return true;
    };
    bool ok = true;
    ok &= alloc(reinterpret_cast<void **>(&c->d_cases), sizeof(CaseDev) * n_cases);
    ok &= alloc(reinterpret_cast<void **>(&c->d_state), sizeof(CaseState) * n_cases);
    ok &= alloc(reinterpret_cast<void **>(&c->d_scratch), sizeof(StepScratch));
    ok &= alloc(reinterpret_cast<void **>(&c->d_err), sizeof(int));
    ok &= alloc(reinterpret_cast<void **>(&c->d_tables), sizeof(int32_t) * 7 * (n_cases + 1));
    ok &= alloc(reinterpret_cast<void **>(&c->d_tmp), sizeof(int32_t) * 2 * n_cases);
    ok &= alloc(reinterpret_cast<void **>(&c->d_pbases), sizeof(int64_t) * n_cases);
    for (auto &side : c->buf)
        for (void *&p : side)
            ok &= alloc(&p, esz * slot);
    ok &= alloc(reinterpret_cast<void **>(&c->key), sizeof(uint32_t) * slot);
    int32_t **cell_arrays[] = {&c->cells.n_in, &c->cells.n_o, &c->cells.o_fill, &c->cells.fin,
                               &c->cells.ostart, &c->cells.base_in, &c->cells.start[0],
                               &c->cells.start[1]};
    for (auto pp : cell_arrays)
        ok &= alloc(reinterpret_cast<void **>(pp), sizeof(int32_t) * cell);
    ok &= alloc(reinterpret_cast<void **>(&c->cells.acc), sizeof(double) * ACC_COUNT * cell);
    c->cells.acc_stride = cell;
    ok &= alloc(reinterpret_cast<void **>(&c->tile_in), sizeof(int32_t) * max_tiles);
    ok &= alloc(reinterpret_cast<void **>(&c->tile_prefix), sizeof(int32_t) * max_tiles);
    ok &= alloc(reinterpret_cast<void **>(&c->tile_dead), sizeof(int32_t) * max_tiles);
    ok &= alloc(reinterpret_cast<void **>(&c->tile_dprefix), sizeof(int32_t) * max_tiles);
    ok &= alloc(reinterpret_cast<void **>(&c->itile_dead), sizeof(int32_t) * max_tiles);
    ok &= alloc(reinterpret_cast<void **>(&c->itile_dprefix), sizeof(int32_t) * max_tiles);
    const size_t chain = static_cast<size_t>(std::max(max_tiles, cell_tiles)) + 1;
    c->lb_words = 4 * chain;
    ok &= alloc(reinterpret_cast<void **>(&c->lb), sizeof(uint64_t) * c->lb_words);
    ok &= alloc(reinterpret_cast<void **>(&c->hole_pos), sizeof(int32_t) * slot);
    ok &= alloc(reinterpret_cast<void **>(&c->hole_oc), sizeof(int32_t) * slot);
    // Appends per step and case: out-of-range moved slots + injected
    // survivors (n_old + n_inj <= cap) + refilled holes (<= n_old): <= 2 cap.
    ok &= alloc(reinterpret_cast<void **>(&c->obuf), sizeof(uint32_t) * 2 * slot);
    ok &= alloc(reinterpret_cast<void **>(&c->near_list), sizeof(uint32_t) * slot);
    ok &= alloc(reinterpret_cast<void **>(&c->olist), sizeof(int32_t) * slot);
    ok &= alloc(reinterpret_cast<void **>(&c->coll_list), sizeof(uint32_t) * cell);
    ok &= alloc(reinterpret_cast<void **>(&c->d_counters), sizeof(dsmc_counters) * n_cases);
    ok &= alloc(reinterpret_cast<void **>(&c->d_gsync), sizeof(GridSync));
    ok &= alloc(reinterpret_cast<void **>(&c->d_probe_err), sizeof(int));
    ok &= alloc(reinterpret_cast<void **>(&c->d_phase_ns),
                sizeof(unsigned long long) * PERSIST_PHASES);

    size_t arena_bytes = 0;
    for (const auto &b : carve)
        arena_bytes += b.second;
    ok &= cudaMalloc(&c->arena, arena_bytes) == cudaSuccess;
    if (!ok) {
        c->arena = nullptr;
        free_ctx(c);
        return DSMC_ERR_CUDA;
    }
    {
        char *at = static_cast<char *>(c->arena);
        for (const auto &b : carve) {
            *b.first = at;
            at += b.second;
        }
    }
    int32_t *t = c->d_tables;
    const int w = n_cases + 1;
    c->tt = TileTables{t, t + w, t + 2 * w, t + 3 * w, t + 4 * w, t + 5 * w, t + 6 * w};
    auto fail = [&]() {
        free_ctx(c);
        return DSMC_ERR_CUDA;
    };
    if (cudaMemcpy(c->d_cases, c->hcases.data(), sizeof(CaseDev) * n_cases,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->tt.cell0, cell0.data(), sizeof(int32_t) * w, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->tt.cblock0, cblock0.data(), sizeof(int32_t) * w, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->tt.cellbase, cellbase.data(), sizeof(int32_t) * w,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_pbases, pbases.data(), sizeof(int64_t) * n_cases,
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return fail();
    if (cudaMemset(c->d_state, 0, sizeof(CaseState) * n_cases) != cudaSuccess ||
        cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->cells.n_in, 0, sizeof(int32_t) * cell) != cudaSuccess ||
        cudaMemset(c->cells.n_o, 0, sizeof(int32_t) * cell) != cudaSuccess ||
        cudaMemset(c->cells.o_fill, 0, sizeof(int32_t) * cell) != cudaSuccess ||
        cudaMemset(c->cells.start[0], 0, sizeof(int32_t) * cell) != cudaSuccess ||
        cudaMemset(c->cells.start[1], 0, sizeof(int32_t) * cell) != cudaSuccess ||
        cudaMemset(c->cells.acc, 0, sizeof(double) * ACC_COUNT * cell) != cudaSuccess ||
        cudaMemset(c->d_phase_ns, 0, sizeof(unsigned long long) * PERSIST_PHASES) != cudaSuccess)
        return fail();
    const int g = c->precision == DSMC_FP32 ? occupancy_grids<float>(c) : occupancy_grids<double>(c);
    if (g)
        return fail();

    *out = c;
    return DSMC_OK;
}

int dsmc_ctx_destroy(dsmc_ctx *ctx)
{
    if (ctx == nullptr)
        return DSMC_ERR_ARGUMENT;
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    return DSMC_OK;
}

int dsmc_init_cold(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    CK(cudaMemsetAsync(c->d_state, 0, sizeof(CaseState) * c->ncase, c->stream));
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream)); // a new run starts clean
    CK(cudaMemsetAsync(c->cells.acc, 0, sizeof(double) * ACC_COUNT * c->total_cells, c->stream));
    CK(cudaMemsetAsync(c->cells.start[c->cur], 0, sizeof(int32_t) * c->total_cells, c->stream));
    // Every particle of the cold start is out of range (no previous sort).
    CK(cudaMemsetAsync(c->cells.n_in, 0, sizeof(int32_t) * c->total_cells, c->stream));
    int s;
    if (c->precision == DSMC_FP32) {
        if ((s = enqueue_move<float>(c, 1)) || (s = enqueue_boundary<float>(c)) ||
            (s = enqueue_index<float>(c)))
            return s;
    } else {
        if ((s = enqueue_move<double>(c, 1)) || (s = enqueue_boundary<double>(c)) ||
            (s = enqueue_index<double>(c)))
            return s;
    }
    if ((s = enqueue_finish(c, 1, 0, 0)))
        return s;
    c->initialized = true;
    c->stage = 0;
    return DSMC_OK;
}

namespace {

int init_warm(dsmc_ctx *c, const double *host_field, int stride)
{
    if (c == nullptr || host_field == nullptr)
        return DSMC_ERR_ARGUMENT;
    int64_t cells = 0;
    for (const CaseDev &cd : c->hcases)
        cells += cd.ncell;
    CK(cudaMemsetAsync(c->d_state, 0, sizeof(CaseState) * c->ncase, c->stream));
    CK(cudaMemsetAsync(c->cells.acc, 0, sizeof(double) * ACC_COUNT * c->total_cells, c->stream));
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    double *dfield = nullptr;
    int32_t *tmp = nullptr;
    const size_t bytes = sizeof(double) * stride * cells;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dfield), bytes, c->stream));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(int32_t) * 2 * c->total_cells,
                       c->stream));
    CK(cudaMemcpyAsync(dfield, host_field, bytes, cudaMemcpyHostToDevice, c->stream));
    const int s = c->precision == DSMC_FP32
                      ? warm_fill<float>(c, dfield, stride, tmp, tmp + c->total_cells)
                      : warm_fill<double>(c, dfield, stride, tmp, tmp + c->total_cells);
    CK(cudaFreeAsync(dfield, c->stream));
    CK(cudaFreeAsync(tmp, c->stream));
    if (s)
        return s;
    CK(cudaStreamSynchronize(c->stream));
    c->initialized = true;
    c->stage = 0;
    return device_error(c);
}

} // namespace

int dsmc_init_warm(dsmc_ctx *c, const double *host_field) { return init_warm(c, host_field, 4); }

int dsmc_init_warm_tensor(dsmc_ctx *c, const double *host_field)
{
    return init_warm(c, host_field, 7);
}

int dsmc_init_warm_mixture(dsmc_ctx *c, const double *host_field)
{
    return init_warm(c, host_field, 8);
}

int dsmc_step_read(dsmc_ctx *c, int n_steps, dsmc_counters *host_out)
{
    if (c == nullptr || host_out == nullptr || n_steps < 0)
        return DSMC_ERR_ARGUMENT;
    for (int k = 0; k < n_steps; ++k) {
        const int s = dsmc_step(c, 1);
        if (s)
            return s;
        CK(cudaMemcpyAsync(host_out + static_cast<size_t>(k) * c->ncase, c->d_counters,
                           sizeof(dsmc_counters) * c->ncase, cudaMemcpyDeviceToHost, c->stream));
    }
    return DSMC_OK;
}

int dsmc_step(dsmc_ctx *c, int n_steps)
{
    if (c == nullptr || n_steps < 0)
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || c->stage != 0)
        return DSMC_ERR_STATE;
    if (c->profiling) {
        for (int i = 0; i < n_steps; ++i) {
            const int s = dispatch_step(c);
            if (s)
                return s;
        }
        return DSMC_OK;
    }
    if (c->step_mode == DSMC_STEP_PERSISTENT)
        return c->precision == DSMC_FP32 ? persistent_steps<float>(c, n_steps)
                                         : persistent_steps<double>(c, n_steps);
    if (c->graph[0] == nullptr) {
        const int s = build_graphs(c);
        if (s)
            return s;
    }
    for (int i = 0; i < n_steps; ++i) {
        CK(cudaGraphLaunch(c->graph[c->cur], c->stream));
        c->cur ^= 1;
    }
    return DSMC_OK;
}

#define STAGE_DISPATCH(fn, ...)                                                   \
    (c->precision == DSMC_FP32 ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

int dsmc_stage_move(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || c->stage != 0)
        return DSMC_ERR_STATE;
    const int s = STAGE_DISPATCH(enqueue_move, c, 0);
    c->stage = s ? c->stage : 1;
    c->sampled = false;
    return s;
}

int dsmc_stage_boundary(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 1)
        return DSMC_ERR_STATE;
    const int s = STAGE_DISPATCH(enqueue_boundary, c);
    c->stage = s ? c->stage : 2;
    return s;
}

int dsmc_stage_index(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 2)
        return DSMC_ERR_STATE;
    const int s = STAGE_DISPATCH(enqueue_index, c);
    c->stage = s ? c->stage : 3;
    return s;
}

int dsmc_stage_collide(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 3)
        return DSMC_ERR_STATE;
    const int s = STAGE_DISPATCH(enqueue_collide, c, 1, 0);
    c->stage = s ? c->stage : 4;
    return s;
}

int dsmc_stage_sample(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 4)
        return DSMC_ERR_STATE;
    const int s = STAGE_DISPATCH(enqueue_collide, c, 0, 1);
    c->stage = s ? c->stage : 5;
    c->sampled = s == 0;
    return s;
}

int dsmc_stage_end_step(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage < 3)
        return DSMC_ERR_STATE;
    const int s = enqueue_finish(c, 0, c->sampled ? 1 : 0, 1);
    if (s == 0)
        c->stage = 0;
    return s;
}

int dsmc_synchronize(dsmc_ctx *c)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return device_error(c);
}

int dsmc_get_counters(dsmc_ctx *c, int i, dsmc_counters *out)
{
    if (c == nullptr || out == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    std::vector<CaseState> st;
    const int s = read_state(c, st);
    if (s)
        return s;
    const CaseState &x = st[i];
    // After BoundaryConditions the valid slots are the survivors [0, K).
    out->np = c->stage >= 2 ? x.n_keep : x.n_old;
    out->step = x.step;
    out->sample_step = x.sample_step;
    out->collisions_last_step = c->stage >= 4 ? x.nc_step : x.nc_last;
    out->collisions_total = x.nc_total;
    out->drag_collision_count = static_cast<int64_t>(x.drag_count);
    out->particle_steps = x.particle_steps;
    out->drag_impulse_total = x.drag_impulse;
    out->time = x.time;
    out->sample_time = x.sample_time;
    out->drag_sampling_time = x.drag_time;
    out->drag_collision_count_window = static_cast<int64_t>(x.drag_count_window);
    out->drag_impulse_window = x.drag_impulse_window;
    return DSMC_OK;
}

int dsmc_get_fields_device(dsmc_ctx *c, int i, double *device_out)
{
    if (c == nullptr || device_out == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    const CaseDev &cd = c->hcases[i];
    k_fields_out<<<std::max(1, std::min(1024, (cd.ncell + 255) / 256)), 256, 0, c->stream>>>(
        c->cells, cd.cbase, cd.ncell, device_out);
    CK(cudaGetLastError());
    return DSMC_OK;
}

int dsmc_get_fields(dsmc_ctx *c, int i, dsmc_cell *host_out)
{
    if (c == nullptr || host_out == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    const CaseDev &cd = c->hcases[i];
    const size_t bytes = sizeof(double) * 17 * cd.ncell;
    // A pinned destination is copied into directly; pageable memory, which
    // the driver would copy through its own small bounce buffers, goes
    // through two pinned chunks of the context instead, the device copy of
    // one overlapping the host copy of the other.
    cudaPointerAttributes pa{};
    const bool pinned =
        cudaPointerGetAttributes(&pa, host_out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError(); // an unregistered pointer is not an error to keep
    const bool staged = !pinned && bytes > FIELD_CHUNK;
    if (staged && c->field_stage[0] == nullptr) {
        for (int k = 0; k < 2; ++k) {
            CK(cudaMallocHost(&c->field_stage[k], FIELD_CHUNK));
            CK(cudaEventCreateWithFlags(&c->field_ev[k], cudaEventDisableTiming));
        }
    }
    // The gathered cells go to the changed-cell list buffer when it is large
    // enough and no staged step is in progress: it is rebuilt within every
    // step, and this call is ordered on the context's stream between steps.
    const bool in_scratch = c->stage == 0 &&
                            bytes <= sizeof(uint32_t) * 2 * static_cast<size_t>(c->total_slots);
    double *tmp = nullptr;
    if (in_scratch)
        tmp = reinterpret_cast<double *>(c->obuf);
    else
        CK(cudaMallocAsync(reinterpret_cast<void **>(&tmp), bytes, c->stream));
    int s = dsmc_get_fields_device(c, i, tmp);
    if (s == 0 && !staged) {
        CK(cudaMemcpyAsync(host_out, tmp, bytes, cudaMemcpyDeviceToHost, c->stream));
    } else if (s == 0) {
        const size_t n = (bytes + FIELD_CHUNK - 1) / FIELD_CHUNK;
        auto span = [&](size_t k) { return std::min(FIELD_CHUNK, bytes - k * FIELD_CHUNK); };
        auto issue = [&](size_t k) -> int {
            CK(cudaMemcpyAsync(c->field_stage[k & 1], reinterpret_cast<char *>(tmp) + k * FIELD_CHUNK,
                               span(k), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaEventRecord(c->field_ev[k & 1], c->stream));
            return DSMC_OK;
        };
        for (size_t k = 0; k < n && k < 2 && s == 0; ++k)
            s = issue(k);
        for (size_t k = 0; k < n && s == 0; ++k) {
            CK(cudaEventSynchronize(c->field_ev[k & 1]));
            std::memcpy(reinterpret_cast<char *>(host_out) + k * FIELD_CHUNK, c->field_stage[k & 1],
                        span(k));
            if (k + 2 < n)
                s = issue(k + 2);
        }
    }
    if (!in_scratch)
        CK(cudaFreeAsync(tmp, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return s;
}

} // extern "C"

// Staging array of dsmc_get_fields_noalloc: 17 doubles per cell.
static __device__ __align__(256) double g_fields_noalloc[17 * DSMC_FIELDS_NOALLOC_MAX_CELLS];

namespace {
// Device address of g_fields_noalloc on each device.  In host code the name
// g_fields_noalloc is a host-side stand-in, not a device address, so the
// kernel receives the address cudaGetSymbolAddress reports, looked up once
// per device with that device current.
constexpr int kMaxDevices = 64;
double *g_fields_noalloc_addr[kMaxDevices] = {nullptr};
std::mutex g_fields_noalloc_lock;

int fields_noalloc_address(int device, double **out)
{
    if (device < 0 || device >= kMaxDevices)
        return DSMC_ERR_ARGUMENT;
    std::lock_guard<std::mutex> guard(g_fields_noalloc_lock);
    if (g_fields_noalloc_addr[device] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_fields_noalloc);
        if (e != cudaSuccess || p == nullptr) {
            std::fprintf(stderr, "dsmc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return DSMC_ERR_CUDA;
        }
        g_fields_noalloc_addr[device] = static_cast<double *>(p);
    }
    *out = g_fields_noalloc_addr[device];
    return DSMC_OK;
}
} // namespace

// ---- checkpoint ----------------------------------------------------------------

namespace {

constexpr char kCheckpointMagic[8] = {'D', 'S', 'M', 'C', 'C', 'K', 'P', '1'};

// The run counters of one case, as stored in a checkpoint.
struct CheckpointCase {
    int64_t n, step, sample_step, nc_last, nc_total, particle_steps;
    uint64_t drag_count, drag_count_window;
    double drag_impulse, drag_impulse_window, time, sample_time, drag_time;
};

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f)
            std::fclose(f);
    }
};

bool put(FILE *f, const void *p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
bool get(FILE *f, void *p, size_t n) { return std::fread(p, 1, n, f) == n; }

} // namespace

extern "C" {

int dsmc_get_fields_noalloc(dsmc_ctx *c, int i, dsmc_cell *host_out)
{
    if (c == nullptr || host_out == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    const CaseDev &cd = c->hcases[i];
    if (cd.ncell > DSMC_FIELDS_NOALLOC_MAX_CELLS) {
        std::fprintf(stderr,
                     "dsmc_get_fields_noalloc: %d cells exceed the static maximum of %d; "
                     "use dsmc_get_fields\n",
                     cd.ncell, DSMC_FIELDS_NOALLOC_MAX_CELLS);
        return DSMC_ERR_TOO_LARGE;
    }
    int prev = 0;
    CK(cudaGetDevice(&prev));
    if (prev != c->device)
        CK(cudaSetDevice(c->device));
    double *staging = nullptr;
    int s = fields_noalloc_address(c->device, &staging);
    if (s == DSMC_OK) {
        k_fields_out<<<std::max(1, std::min(1024, (cd.ncell + 255) / 256)), 256, 0, c->stream>>>(
            c->cells, cd.cbase, cd.ncell, staging);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host_out, staging, sizeof(double) * 17 * cd.ncell,
                                cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "dsmc_get_fields_noalloc: %s\n", cudaGetErrorString(e));
            s = DSMC_ERR_CUDA;
        }
    }
    if (prev != c->device)
        cudaSetDevice(prev);
    return s;
}

int dsmc_set_fields_device(dsmc_ctx *c, int i, const double *device_in, int64_t sample_step)
{
    if (c == nullptr || device_in == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    const CaseDev &cd = c->hcases[i];
    k_fields_in<<<std::max(1, std::min(1024, (cd.ncell + 255) / 256)), 256, 0, c->stream>>>(
        c->cells, cd.cbase, cd.ncell, device_in);
    CK(cudaGetLastError());
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    st[i].sample_step = sample_step;
    CK(cudaMemcpyAsync(c->d_state + i, &st[i], sizeof(CaseState), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_download_particles(dsmc_ctx *c, int i, double *x, double *y, double *vx, double *vy,
                            double *vz, int64_t capacity, int64_t *n_out)
{
    if (c == nullptr || i < 0 || i >= c->ncase || n_out == nullptr)
        return DSMC_ERR_ARGUMENT;
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    // Valid slots: [0, n_old) at rest and after MoveParticles, the survivors
    // [0, K) from BoundaryConditions on.
    const int64_t n = c->stage >= 2 ? st[i].n_keep : st[i].n_old;
    *n_out = n;
    if (n > capacity)
        return DSMC_ERR_CAPACITY;
    if (n == 0)
        return DSMC_OK;
    const CaseDev &cd = c->hcases[i];
    double *tmp = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(double) * 5 * n, c->stream));
    if (c->precision == DSMC_FP32) {
        k_download_case<<<std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256)), 256, 0,
                          c->stream>>>(slots<float>(c, c->cur), cd.pbase, n, tmp);
    } else {
        Slots<double> p = slots<double>(c, c->cur);
        double *dsts[5] = {tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, tmp + 4 * n};
        double *srcs[5] = {p.x, p.y, p.vx, p.vy, p.vz};
        for (int k = 0; k < 5; ++k)
            CK(cudaMemcpyAsync(dsts[k], srcs[k] + cd.pbase, sizeof(double) * n,
                               cudaMemcpyDeviceToDevice, c->stream));
    }
    double *outs[5] = {x, y, vx, vy, vz};
    for (int k = 0; k < 5; ++k)
        if (outs[k] != nullptr)
            CK(cudaMemcpyAsync(outs[k], tmp + k * n, sizeof(double) * n, cudaMemcpyDeviceToHost,
                               c->stream));
    CK(cudaFreeAsync(tmp, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_upload_particles(dsmc_ctx *c, int i, const double *x, const double *y, const double *vx,
                          const double *vy, const double *vz, int64_t n)
{
    if (c == nullptr || i < 0 || i >= c->ncase || n < 0 || !x || !y || !vx || !vy || !vz)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 0)
        return DSMC_ERR_STATE;
    const CaseDev &cd = c->hcases[i];
    if (n > cd.cap)
        return DSMC_ERR_CAPACITY;
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    double *tmp = nullptr;
    if (n > 0) {
        CK(cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(double) * 5 * n, c->stream));
        const double *ins[5] = {x, y, vx, vy, vz};
        for (int k = 0; k < 5; ++k)
            CK(cudaMemcpyAsync(tmp + k * n, ins[k], sizeof(double) * n, cudaMemcpyHostToDevice,
                               c->stream));
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256)));
        if (c->precision == DSMC_FP32)
            k_upload_case<float><<<grid, 256, 0, c->stream>>>(tmp, tmp + n, tmp + 2 * n,
                                                              tmp + 3 * n, tmp + 4 * n, n,
                                                              slots<float>(c, c->cur), cd.pbase);
        else
            k_upload_case<double><<<grid, 256, 0, c->stream>>>(tmp, tmp + n, tmp + 2 * n,
                                                               tmp + 3 * n, tmp + 4 * n, n,
                                                               slots<double>(c, c->cur), cd.pbase);
        CK(cudaGetLastError());
    }
    st[i].n_old = n;
    CK(cudaMemcpyAsync(c->d_state + i, &st[i], sizeof(CaseState), cudaMemcpyHostToDevice,
                       c->stream));
    s = c->precision == DSMC_FP32 ? resort_all<float>(c) : resort_all<double>(c);
    if (tmp)
        CK(cudaFreeAsync(tmp, c->stream));
    if (s)
        return s;
    CK(cudaStreamSynchronize(c->stream));
    c->initialized = true;
    return device_error(c);
}


int dsmc_checkpoint_save(dsmc_ctx *c, const char *path)
{
    if (c == nullptr || path == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 0 || !c->initialized)
        return DSMC_ERR_STATE;
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    File out;
    out.f = std::fopen(path, "wb");
    if (out.f == nullptr)
        return DSMC_ERR_ARGUMENT;
    const int32_t head[4] = {1, c->ncase, c->precision, static_cast<int32_t>(sizeof(dsmc_params))};
    bool ok = put(out.f, kCheckpointMagic, 8) && put(out.f, head, sizeof(head));
    for (int i = 0; i < c->ncase && ok; ++i) {
        const CaseDev &cd = c->hcases[i];
        const CaseState &x = st[i];
        const CheckpointCase k{x.n_old,        x.step,         x.sample_step,      x.nc_last,
                               x.nc_total,     x.particle_steps, x.drag_count,      x.drag_count_window,
                               x.drag_impulse, x.drag_impulse_window, x.time,       x.sample_time,
                               x.drag_time};
        ok = put(out.f, &c->params[i], sizeof(dsmc_params)) && put(out.f, &k, sizeof(k));
        std::vector<double> v(5 * static_cast<size_t>(std::max<int64_t>(k.n, 1)));
        int64_t n = 0;
        s = dsmc_download_particles(c, i, v.data(), v.data() + k.n, v.data() + 2 * k.n,
                                    v.data() + 3 * k.n, v.data() + 4 * k.n, k.n, &n);
        if (s)
            return s;
        ok = ok && put(out.f, v.data(), sizeof(double) * 5 * k.n);
        std::vector<double> acc(static_cast<size_t>(ACC_COUNT) * cd.ncell);
        for (int m = 0; m < ACC_COUNT; ++m)
            CK(cudaMemcpyAsync(acc.data() + static_cast<size_t>(m) * cd.ncell,
                               c->cells.acc + static_cast<size_t>(m) * c->cells.acc_stride + cd.cbase,
                               sizeof(double) * cd.ncell, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        ok = ok && put(out.f, acc.data(), sizeof(double) * acc.size());
    }
    return ok ? DSMC_OK : DSMC_ERR_ARGUMENT;
}

int dsmc_checkpoint_load(dsmc_ctx *c, const char *path)
{
    if (c == nullptr || path == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 0)
        return DSMC_ERR_STATE;
    File in;
    in.f = std::fopen(path, "rb");
    if (in.f == nullptr)
        return DSMC_ERR_ARGUMENT;
    char magic[8];
    int32_t head[4];
    if (!get(in.f, magic, 8) || std::memcmp(magic, kCheckpointMagic, 8) != 0 ||
        !get(in.f, head, sizeof(head)) || head[0] != 1 || head[1] != c->ncase ||
        head[2] != c->precision || head[3] != static_cast<int32_t>(sizeof(dsmc_params)))
        return DSMC_ERR_ARGUMENT;
    std::vector<CheckpointCase> ks(c->ncase);
    for (int i = 0; i < c->ncase; ++i) {
        const CaseDev &cd = c->hcases[i];
        dsmc_params p;
        CheckpointCase &k = ks[i];
        if (!get(in.f, &p, sizeof(p)))
            return DSMC_ERR_ARGUMENT;
        p.n_step = c->params[i].n_step; // the run length may grow on a restart
        if (std::memcmp(&p, &c->params[i], sizeof(p)) != 0 || !get(in.f, &k, sizeof(k)) ||
            k.n < 0 || k.n > cd.cap)
            return DSMC_ERR_ARGUMENT;
        std::vector<double> v(5 * static_cast<size_t>(std::max<int64_t>(k.n, 1)));
        std::vector<double> acc(static_cast<size_t>(ACC_COUNT) * cd.ncell);
        if (!get(in.f, v.data(), sizeof(double) * 5 * k.n) ||
            !get(in.f, acc.data(), sizeof(double) * acc.size()))
            return DSMC_ERR_ARGUMENT;
        int s = dsmc_upload_particles(c, i, v.data(), v.data() + k.n, v.data() + 2 * k.n,
                                      v.data() + 3 * k.n, v.data() + 4 * k.n, k.n);
        if (s)
            return s;
        for (int m = 0; m < ACC_COUNT; ++m)
            CK(cudaMemcpyAsync(c->cells.acc + static_cast<size_t>(m) * c->cells.acc_stride + cd.cbase,
                               acc.data() + static_cast<size_t>(m) * cd.ncell,
                               sizeof(double) * cd.ncell, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    for (int i = 0; i < c->ncase; ++i) {
        const CheckpointCase &k = ks[i];
        CaseState &x = st[i];
        x.step = k.step;
        x.sample_step = k.sample_step;
        x.nc_last = k.nc_last;
        x.nc_total = k.nc_total;
        x.particle_steps = k.particle_steps;
        x.drag_count = k.drag_count;
        x.drag_count_window = k.drag_count_window;
        x.drag_impulse = k.drag_impulse;
        x.drag_impulse_window = k.drag_impulse_window;
        x.time = k.time;
        x.sample_time = k.sample_time;
        x.drag_time = k.drag_time;
    }
    CK(cudaMemcpyAsync(c->d_state, st.data(), sizeof(CaseState) * c->ncase,
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_get_cell_starts(dsmc_ctx *c, int i, int32_t *host_out)
{
    if (c == nullptr || host_out == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    const CaseDev &cd = c->hcases[i];
    CK(cudaMemcpyAsync(host_out, c->cells.start[c->cur] + cd.cbase,
                       sizeof(int32_t) * (cd.ncell + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_set_profiling(dsmc_ctx *c, int enabled)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    int s = resolve_timings(c);
    if (s)
        return s;
    c->profiling = enabled != 0;
    for (int k = 0; k < KID_COUNT; ++k) {
        c->kernel_ms[k] = 0.0;
        c->kernel_launches[k] = 0;
    }
    return DSMC_OK;
}

int dsmc_get_kernel_times(dsmc_ctx *c, double *ms_out, int64_t *launches_out, int max_kernels,
                          int *n_kernels, const char **names_out)
{
    if (c == nullptr || n_kernels == nullptr)
        return DSMC_ERR_ARGUMENT;
    const int s = resolve_timings(c);
    if (s)
        return s;
    *n_kernels = KID_COUNT;
    for (int k = 0; k < KID_COUNT && k < max_kernels; ++k) {
        if (ms_out)
            ms_out[k] = c->kernel_ms[k];
        if (launches_out)
            launches_out[k] = c->kernel_launches[k];
        if (names_out)
            names_out[k] = kKernelNames[k];
    }
    return DSMC_OK;
}

int dsmc_get_launch_config(dsmc_ctx *c, int32_t *ctas_per_sm, int32_t *max_ctas_per_sm,
                           int max_kernels, int *n_kernels, const char **names_out)
{
    if (c == nullptr || n_kernels == nullptr)
        return DSMC_ERR_ARGUMENT;
    *n_kernels = KID_COUNT;
    for (int k = 0; k < KID_COUNT && k < max_kernels; ++k) {
        if (ctas_per_sm)
            ctas_per_sm[k] = c->ctas[k];
        if (max_ctas_per_sm)
            max_ctas_per_sm[k] = c->ctas_max[k];
        if (names_out)
            names_out[k] = kKernelNames[k];
    }
    return DSMC_OK;
}

int dsmc_set_launch_config(dsmc_ctx *c, const int32_t *ctas_per_sm, int n)
{
    if (c == nullptr || ctas_per_sm == nullptr || n < 0 || n > KID_COUNT)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 0)
        return DSMC_ERR_STATE;
    for (int k = 0; k < n; ++k)
        if (c->ctas_max[k] > 0 && ctas_per_sm[k] > 0)
            c->ctas[k] = std::min(ctas_per_sm[k], c->ctas_max[k]);
    drop_graphs(c); // rebuilt with the new shapes at the next dsmc_step
    return DSMC_OK;
}

int dsmc_set_step_mode(dsmc_ctx *c, int mode, int ctas_per_sm)
{
    if (c == nullptr || (mode != DSMC_STEP_GRAPH && mode != DSMC_STEP_PERSISTENT) ||
        ctas_per_sm < 0)
        return DSMC_ERR_ARGUMENT;
    if (c->stage != 0)
        return DSMC_ERR_STATE;
    if (mode == DSMC_STEP_PERSISTENT) {
        if (!c->coop || c->p_ctas_max < 1)
            return DSMC_ERR_UNSUPPORTED;
        const int want = ctas_per_sm == 0 ? c->p_ctas_max : std::min(ctas_per_sm, c->p_ctas_max);
        if (want != c->p_ctas)
            drop_graphs(c);
        c->p_ctas = want;
    }
    c->step_mode = mode;
    return DSMC_OK;
}

int dsmc_get_step_mode(dsmc_ctx *c, int *mode, int *ctas_per_sm, int *max_ctas_per_sm,
                       int *graph_launch)
{
    if (c == nullptr)
        return DSMC_ERR_ARGUMENT;
    if (mode)
        *mode = c->step_mode;
    if (ctas_per_sm)
        *ctas_per_sm = c->p_ctas;
    if (max_ctas_per_sm)
        *max_ctas_per_sm = c->coop ? c->p_ctas_max : 0;
    if (graph_launch)
        *graph_launch = c->p_graph ? 1 : 0;
    return DSMC_OK;
}

const char *kPhaseNames[PERSIST_PHASES] = {
    "plan", "move+inject", "move_near", "dead_scan", "holes", "tail",
    "cell_scan+tile_scan", "olist+collide_select", "cell_fix", "scatter", "collide_pairs",
    "sample"};

int dsmc_get_phase_times(dsmc_ctx *c, double *ms_out, int max_phases, int *n_phases,
                         const char **names_out, int reset)
{
    if (c == nullptr || n_phases == nullptr || max_phases < 0)
        return DSMC_ERR_ARGUMENT;
    unsigned long long ns[PERSIST_PHASES];
    CK(cudaMemcpyAsync(ns, c->d_phase_ns, sizeof(ns), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (reset)
        CK(cudaMemsetAsync(c->d_phase_ns, 0, sizeof(ns), c->stream));
    *n_phases = PERSIST_PHASES;
    for (int k = 0; k < PERSIST_PHASES && k < max_phases; ++k) {
        if (ms_out)
            ms_out[k] = static_cast<double>(ns[k]) * 1e-6;
        if (names_out)
            names_out[k] = kPhaseNames[k];
    }
    return DSMC_OK;
}

int dsmc_grid_sync_probe(dsmc_ctx *c, int64_t wait_ns)
{
    if (c == nullptr || wait_ns < 0)
        return DSMC_ERR_ARGUMENT;
    CK(cudaMemsetAsync(c->d_gsync, 0, sizeof(GridSync), c->stream));
    CK(cudaMemsetAsync(c->d_probe_err, 0, sizeof(int), c->stream));
    k_grid_sync_probe<<<1, 32, 0, c->stream>>>(c->d_gsync, 1, static_cast<uint64_t>(wait_ns),
                                               c->d_probe_err);
    CK(cudaGetLastError());
    int err = 0;
    CK(cudaMemcpyAsync(&err, c->d_probe_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return err;
}

int dsmc_autotune(dsmc_ctx *c, int steps_per_trial)
{
    if (c == nullptr || steps_per_trial < 1)
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || c->stage != 0)
        return DSMC_ERR_STATE;
    const bool was_profiling = c->profiling;
    int s = dsmc_set_profiling(c, 1);
    if (s)
        return s;
    for (int k = 0; k < KID_COUNT; ++k) {
        if (c->ctas_max[k] <= 0)
            continue;
        const int mx = c->ctas_max[k];
        std::vector<int> cand;
        for (int v : {mx, mx / 2, mx / 4, 1, 2, 4, 8, 16})
            if (v >= 1 && v <= mx && std::find(cand.begin(), cand.end(), v) == cand.end())
                cand.push_back(v);
        int best = c->ctas[k];
        double best_ms = 1e300;
        for (int v : cand) {
            c->ctas[k] = v;
            if ((s = resolve_timings(c)))
                return s;
            c->kernel_ms[k] = 0.0;
            c->kernel_launches[k] = 0;
            for (int i = 0; i < steps_per_trial; ++i)
                if ((s = dispatch_step(c)))
                    return s;
            if ((s = resolve_timings(c)))
                return s;
            const double ms = c->kernel_launches[k] ? c->kernel_ms[k] / c->kernel_launches[k] : 0.0;
            if (ms < best_ms * 0.98) { // keep the larger grid unless clearly slower
                best_ms = ms;
                best = v;
            }
        }
        c->ctas[k] = best;
    }
    drop_graphs(c);
    if ((s = dsmc_set_profiling(c, was_profiling ? 1 : 0)))
        return s;
    return device_error(c);
}

} // extern "C"

namespace {

// Removes, in the reference's swap-with-last order, the slots of [q0, n) of
// case i that `pred` selects (slots below q0 all survive) and sets the case's
// particle count; the caller re-sorts.  Temporary buffers come from the
// stream-ordered allocator (these edits run between steps, rarely).
template <class T> int edit_case(dsmc_ctx *c, int i, int64_t q0, int64_t n, int pred)
{
    const int64_t m = n - q0;
    if (m <= 0)
        return DSMC_OK;
    const int64_t ntile = (m + TILE - 1) / TILE;
    int32_t *tiles = nullptr;
    int64_t *alive = nullptr, *holes = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&tiles), sizeof(int32_t) * ntile, c->stream));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&alive), sizeof(int64_t), c->stream));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&holes), sizeof(int64_t) * m, c->stream));
    const Slots<T> p = slots<T>(c, c->cur);
    const int g = static_cast<int>(std::min<int64_t>(ntile, 4 * c->sms));
    k_edit_count<T><<<g, TILE_THREADS, 0, c->stream>>>(c->d_cases, i, p, q0, n, pred, tiles);
    k_edit_scan<<<1, 1024, 0, c->stream>>>(tiles, ntile, alive);
    k_edit_holes<T><<<g, TILE_THREADS, 0, c->stream>>>(c->d_cases, i, p, q0, n, pred, tiles,
                                                        alive, holes);
    k_edit_fill<T><<<g, TILE_THREADS, 0, c->stream>>>(c->d_cases, i, p, q0, n, pred, tiles, alive,
                                                       holes, c->d_err);
    k_edit_commit<<<1, 1, 0, c->stream>>>(c->d_state, i, q0, alive);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(tiles, c->stream));
    CK(cudaFreeAsync(alive, c->stream));
    CK(cudaFreeAsync(holes, c->stream));
    return DSMC_OK;
}

// Appends n FP64 particles (device arrays) to case i, drops those outside the
// domain as BoundaryConditions would, and re-sorts.
template <class T>
int append_case(dsmc_ctx *c, int i, int64_t n_old, const double *x, const double *y,
                const double *vx, const double *vy, const double *vz, int64_t n)
{
    if (n > 0) {
        const int g = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256)));
        k_upload_case<T><<<g, 256, 0, c->stream>>>(x, y, vx, vy, vz, n, slots<T>(c, c->cur),
                                                    c->hcases[i].pbase + n_old);
        CK(cudaGetLastError());
    }
    int s = edit_case<T>(c, i, n_old, n_old + n, EDIT_OUTSIDE_DOMAIN);
    return s ? s : resort_all<T>(c);
}

template <class T> int remove_inside_case(dsmc_ctx *c, int i, int64_t n_old)
{
    int s = edit_case<T>(c, i, 0, n_old, EDIT_INSIDE_BOX);
    return s ? s : resort_all<T>(c);
}

template <class T>
int collide_list_case(dsmc_ctx *c, const CaseDev &cd, const int32_t *d_buf, uint32_t kind,
                      uint32_t step, int32_t *d_nc)
{
    // d_buf: start[2], entity, then the list.
    k_unit_collide<T><<<1, 32, 0, c->stream>>>(cd, 1, d_buf, d_buf + 3, slots<T>(c, c->cur),
                                               cd.pbase, kind, step,
                                               reinterpret_cast<const uint32_t *>(d_buf + 2),
                                               d_nc);
    CK(cudaGetLastError());
    return DSMC_OK;
}

} // namespace

extern "C" {

int dsmc_append_particles_device(dsmc_ctx *c, int i, const double *x, const double *y,
                                 const double *vx, const double *vy, const double *vz, int64_t n)
{
    if (c == nullptr || i < 0 || i >= c->ncase || n < 0 ||
        (n > 0 && (!x || !y || !vx || !vy || !vz)))
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || c->stage != 0)
        return DSMC_ERR_STATE;
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    if (st[i].n_old + n > c->hcases[i].cap)
        return DSMC_ERR_CAPACITY;
    s = c->precision == DSMC_FP32
            ? append_case<float>(c, i, st[i].n_old, x, y, vx, vy, vz, n)
            : append_case<double>(c, i, st[i].n_old, x, y, vx, vy, vz, n);
    if (s)
        return s;
    CK(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int dsmc_remove_inside_box(dsmc_ctx *c, int i)
{
    if (c == nullptr || i < 0 || i >= c->ncase)
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || c->stage != 0)
        return DSMC_ERR_STATE;
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    s = c->precision == DSMC_FP32 ? remove_inside_case<float>(c, i, st[i].n_old)
                                  : remove_inside_case<double>(c, i, st[i].n_old);
    if (s)
        return s;
    CK(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int dsmc_collide_list(dsmc_ctx *c, int i, double cell_volume, int32_t n, const int32_t *ipc,
                      uint32_t kind, uint32_t step, uint32_t entity, int32_t *n_collisions)
{
    if (c == nullptr || i < 0 || i >= c->ncase || n < 0 || (n > 0 && ipc == nullptr) ||
        n_collisions == nullptr || !(cell_volume > 0.0))
        return DSMC_ERR_ARGUMENT;
    if (!c->initialized || (c->stage != 0 && c->stage < 3))
        return DSMC_ERR_STATE; // slots are a sorted population only between steps or after Indexing
    std::vector<CaseState> st;
    int s = read_state(c, st);
    if (s)
        return s;
    const int64_t np = c->stage >= 2 ? st[i].n_keep : st[i].n_old;
    for (int32_t k = 0; k < n; ++k)
        if (ipc[k] < 0 || ipc[k] >= np)
            return DSMC_ERR_ARGUMENT;
    std::vector<int32_t> buf(3 + static_cast<size_t>(n));
    buf[0] = 0;
    buf[1] = n;
    buf[2] = static_cast<int32_t>(entity);
    std::copy(ipc, ipc + n, buf.begin() + 3);
    CaseDev cd = c->hcases[i];
    cd.dv = cell_volume; // BinaryCollisionsInCell's CellVolume argument
    int32_t *d = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&d), sizeof(int32_t) * (buf.size() + 1),
                       c->stream));
    CK(cudaMemcpyAsync(d, buf.data(), sizeof(int32_t) * buf.size(), cudaMemcpyHostToDevice,
                       c->stream));
    s = c->precision == DSMC_FP32 ? collide_list_case<float>(c, cd, d, kind, step, d + buf.size())
                                  : collide_list_case<double>(c, cd, d, kind, step, d + buf.size());
    if (s)
        return s;
    int32_t nc = 0;
    CK(cudaMemcpyAsync(&nc, d + buf.size(), sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(d, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *n_collisions = nc;
    return device_error(c);
}

int dsmc_k_intersect(const dsmc_params *p, int64_t n, const double *x, const double *y,
                     const double *dx, const double *dy, int32_t *hit, double *t_hit, double *nx,
                     double *ny, void *cuda_stream)
{
    if (p == nullptr || n < 0)
        return DSMC_ERR_ARGUMENT;
    dsmc_derived d;
    const int s = dsmc_setup(p, &d);
    if (s)
        return s;
    if (n == 0)
        return DSMC_OK;
    const CaseDev c = make_case(*p, d);
    const int grid = static_cast<int>(std::min<int64_t>(4096, (n + 255) / 256));
    k_unit_intersect<<<grid, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(c, n, x, y, dx, dy,
                                                                               hit, t_hit, nx, ny);
    CK(cudaGetLastError());
    return DSMC_OK;
}

int dsmc_k_inside_box(const dsmc_params *p, int64_t n, const double *x, const double *y,
                      int32_t *inside, void *cuda_stream)
{
    if (p == nullptr || n < 0)
        return DSMC_ERR_ARGUMENT;
    dsmc_derived d;
    const int s = dsmc_setup(p, &d);
    if (s)
        return s;
    if (n == 0)
        return DSMC_OK;
    const CaseDev c = make_case(*p, d);
    const int grid = static_cast<int>(std::min<int64_t>(4096, (n + 255) / 256));
    k_unit_inside<<<grid, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(c, n, x, y, inside);
    CK(cudaGetLastError());
    return DSMC_OK;
}

int dsmc_k_scatter(const dsmc_params *p, const dsmc_derived *d, int64_t n, double *v,
                   const double *nx, const double *ny, uint32_t kind, uint32_t step,
                   const uint32_t *entity, void *cuda_stream)
{
    if (p == nullptr || n < 0)
        return DSMC_ERR_ARGUMENT;
    dsmc_derived dd;
    const int s = dsmc_setup(p, &dd);
    if (s)
        return s;
    if (d != nullptr)
        dd = *d;
    if (n == 0)
        return DSMC_OK;
    const CaseDev c = make_case(*p, dd);
    const int grid = static_cast<int>(std::min<int64_t>(4096, (n + 255) / 256));
    k_unit_scatter<<<grid, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(c, n, v, nx, ny, kind,
                                                                             step, entity);
    CK(cudaGetLastError());
    return DSMC_OK;
}


int dsmc_k_inject(const dsmc_params *p, const dsmc_derived *d, const double *rect, double n_gas,
                  double ux_gas, double uy_gas, double t_gas, int move_flag, uint32_t kind,
                  uint32_t step, uint32_t entity, int64_t capacity, double *x, double *y,
                  double *vx, double *vy, double *vz, int64_t *n_out, void *cuda_stream)
{
    if (p == nullptr || rect == nullptr || n_out == nullptr || capacity < 0)
        return DSMC_ERR_ARGUMENT;
    dsmc_derived dd;
    const int s = dsmc_setup(p, &dd);
    if (s)
        return s;
    if (d != nullptr)
        dd = *d;
    const CaseDev c = make_case(*p, dd);
    // Boundary.cpp:62-63 and :53
    const double v = (rect[2] - rect[0]) * (rect[3] - rect[1]) * p->dz;
    const double navg = n_gas * v / dd.weight;
    const double rt = K_BOLTZMANN * t_gas / dd.molecule_mass;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    int32_t *cnt = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&cnt), 2 * sizeof(int32_t), st));
    k_unit_inject_count<<<1, 1, 0, st>>>(c, navg, kind, step, entity, cnt);
    int32_t h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *n_out = h[0];
    int status = DSMC_OK;
    if (h[0] > capacity) {
        status = DSMC_ERR_CAPACITY;
    } else if (h[0] > 0) {
        if (!x || !y || !vx || !vy || !vz) {
            status = DSMC_ERR_ARGUMENT;
        } else {
            const int g = static_cast<int>(std::min<int64_t>(4096, (h[0] + 255) / 256));
            k_unit_inject_fill<<<g, 256, 0, st>>>(c, make_double4(rect[0], rect[1], rect[2], rect[3]),
                                                  ux_gas, uy_gas, rt, move_flag, kind, step,
                                                  entity, cnt, x, y, vx, vy, vz);
            CK(cudaGetLastError());
        }
    }
    CK(cudaFreeAsync(cnt, st));
    return status;
}

int dsmc_k_collide(const dsmc_params *p, const dsmc_derived *d, double cell_volume,
                   int32_t n_lists, const int32_t *list_start, const int32_t *ipc, double *vx,
                   double *vy, double *vz, uint32_t kind, uint32_t step, const uint32_t *entity,
                   int32_t *n_collisions, void *cuda_stream)
{
    if (p == nullptr || n_lists < 0 || !(cell_volume > 0.0) ||
        (n_lists > 0 && (list_start == nullptr || !vx || !vy || !vz)))
        return DSMC_ERR_ARGUMENT;
    dsmc_derived dd;
    const int s = dsmc_setup(p, &dd);
    if (s)
        return s;
    if (d != nullptr)
        dd = *d;
    if (n_lists == 0)
        return DSMC_OK;
    CaseDev c = make_case(*p, dd);
    c.dv = cell_volume; // BinaryCollisionsInCell's CellVolume argument
    Slots<double> sl{nullptr, nullptr, vx, vy, vz};
    const int g = static_cast<int>(std::min<int32_t>(4096, (n_lists + 127) / 128));
    k_unit_collide<double><<<g, 128, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
        c, n_lists, list_start, ipc, sl, 0, kind, step, entity, n_collisions);
    CK(cudaGetLastError());
    return DSMC_OK;
}

int dsmc_k_elastic(const dsmc_params *p, int64_t n, double *v1, double *v2, const double *cr,
                   uint32_t kind, uint32_t step, const uint32_t *entity, void *cuda_stream)
{
    if (p == nullptr || n < 0 || (n > 0 && (!v1 || !v2 || !cr)))
        return DSMC_ERR_ARGUMENT;
    dsmc_derived dd;
    const int s = dsmc_setup(p, &dd);
    if (s)
        return s;
    if (n == 0)
        return DSMC_OK;
    const CaseDev c = make_case(*p, dd);
    const int g = static_cast<int>(std::min<int64_t>(4096, (n + 255) / 256));
    k_unit_elastic<<<g, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(c, n, v1, v2, cr, kind,
                                                                          step, entity);
    CK(cudaGetLastError());
    return DSMC_OK;
}

} // extern "C"
