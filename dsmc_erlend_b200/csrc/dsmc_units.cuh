// dsmc_units.cuh - kernels behind the single-routine entry points of the C
// ABI (GenerateNewParticles, BinaryCollisionsInCell, ElasticCollision) and
// behind the between-step population edits (particles appended, particles
// inside the box removed) that the reference-named surface offers.
#pragma once

#include <cstdint>

#include "dsmc_kernels.cuh"

namespace dsmc {

// ---- GenerateNewParticles (Boundary.cpp:60-92) on one rectangle -------------

// The count draw of a rectangle with mean navg; writes the count and the
// uniforms it used.  One thread.
__global__ void k_unit_inject_count(CaseDev c, double navg, uint32_t kind, uint32_t step,
                                    uint32_t entity, int32_t *out)
{
    dsmc_stream r;
    open_stream(r, c, kind, step, entity);
    int draws = 0;
    out[0] = inflow_count(r, navg, &draws);
    out[1] = draws;
}

// Particle j of the rectangle: the stream continues at draw c0 + 8 j, the
// draws a sequential GenerateNewParticles gives it.  MoveFlag 1 pre-moves by
// Dt (Boundary.cpp:87-90).
__global__ void k_unit_inject_fill(CaseDev c, double4 rect, double ux, double uy, double rt,
                                   int move_flag, uint32_t kind, uint32_t step, uint32_t entity,
                                   const int32_t *count, double *x, double *y, double *vx,
                                   double *vy, double *vz)
{
    const int64_t n = count[0];
    const uint64_t c0 = static_cast<uint64_t>(count[1]);
    const double b[4] = {rect.x, rect.y, rect.z, rect.w};
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        dsmc_stream r;
        open_stream(r, c, kind, step, entity);
        dsmc_stream_seek(&r, c0 + 8ull * static_cast<uint64_t>(j));
        double px, py, pvx, pvy, pvz;
        new_particle(r, b, ux, uy, rt, px, py, pvx, pvy, pvz);
        if (move_flag == 1) {
            px += c.dt * pvx;
            py += c.dt * pvy;
        }
        x[j] = px;
        y[j] = py;
        vx[j] = pvx;
        vy[j] = pvy;
        vz[j] = pvz;
    }
}

// ---- BinaryCollisionsInCell (Collision.cpp:21-44) over cell lists ------------

// List l holds entries [start[l], start[l + 1]) of ipc (slot indices), or
// those slots themselves when ipc is null; it draws from stream (kind, step,
// entity[l] or l).  One thread per list.  c.dv is the CellVolume argument.
template <class T>
__global__ void k_unit_collide(CaseDev c, int32_t n_lists, const int32_t *start,
                               const int32_t *ipc, Slots<T> p, int64_t pbase, uint32_t kind,
                               uint32_t step, const uint32_t *entity, int32_t *n_collisions)
{
    for (int32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < n_lists;
         l += gridDim.x * blockDim.x) {
        const int32_t s0 = start[l];
        const int n = start[l + 1] - s0;
        int ncc = 0;
        if (n >= 2) {
            dsmc_stream r;
            open_stream(r, c, kind, step, entity ? entity[l] : static_cast<uint32_t>(l));
            const int nn = ntc_pairs(c, n, r);
            const SlotRun<T> run{p, ipc ? pbase : pbase + s0, ipc ? ipc + s0 : nullptr};
            ncc = ntc_candidates(c, n, nn, r, run);
        }
        if (n_collisions)
            n_collisions[l] = ncc;
    }
}

// ---- ElasticCollision (Collision.cpp:7-19) -----------------------------------

__global__ void k_unit_elastic(CaseDev c, int64_t n, double *v1, double *v2, const double *cr,
                               uint32_t kind, uint32_t step, const uint32_t *entity)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double a[3] = {v1[3 * i], v1[3 * i + 1], v1[3 * i + 2]};
        double b[3] = {v2[3 * i], v2[3 * i + 1], v2[3 * i + 2]};
        dsmc_stream r;
        open_stream(r, c, kind, step, entity ? entity[i] : static_cast<uint32_t>(i));
        elastic_collision(r, a, b, cr[i]);
        for (int k = 0; k < 3; ++k) {
            v1[3 * i + k] = a[k];
            v2[3 * i + k] = b[k];
        }
    }
}

// ---- population edits between steps -------------------------------------------
//
// The reference removes particles with its swap-with-last loop
// (BoundaryConditions, Boundary.cpp:181-202; RemoveParticlesInsideBox,
// Geometry.cpp:231-247): with A survivors among slots [q0, n) the count
// becomes K = q0 + A; survivors below K stay; the m-th removed slot below K
// receives the m-th survivor at or above K counted from the end.  Slots
// below q0 are known to survive.  Three passes over tiles of TILE slots
// (counts, holes, refills) and a one-CTA scan of the tile counts.

enum : int { EDIT_OUTSIDE_DOMAIN = 0, EDIT_INSIDE_BOX = 1 };

template <class T>
__device__ __forceinline__ bool edit_removed(const CaseDev &c, Slots<T> p, int64_t g, int pred)
{
    const double x = static_cast<double>(p.x[g]), y = static_cast<double>(p.y[g]);
    return pred == EDIT_INSIDE_BOX ? inside_box(c, x, y) : outside_domain(c, x, y);
}

// Survivors per tile of [q0, n).
template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_edit_count(const CaseDev *cases, int ci, Slots<T> p, int64_t q0, int64_t n, int pred,
                 int32_t *tile_alive)
{
    const CaseDev &c = cases[ci];
    const int64_t ntile = (n - q0 + TILE - 1) / TILE;
    for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
        int alive = 0;
        for (int k = 0; k < TILE_VEC; ++k) {
            const int64_t q = q0 + t * TILE + k * TILE_THREADS + threadIdx.x;
            if (q < n && !edit_removed(c, p, c.pbase + q, pred))
                ++alive;
        }
        int total;
        (void)block_exclusive<int>(alive, total);
        if (threadIdx.x == 0)
            tile_alive[t] = total;
        __syncthreads(); // block_exclusive's shared words are reused by the next tile
    }
}

// Exclusive prefix of the tile counts (in place) and the survivor total.
__global__ void __launch_bounds__(1024)
    k_edit_scan(int32_t *tile_alive, int64_t ntile, int64_t *alive_total)
{
    int64_t carry = 0;
    for (int64_t base = 0; base < ntile; base += 1024) {
        const int64_t t = base + threadIdx.x;
        const int32_t v = t < ntile ? tile_alive[t] : 0;
        int32_t total;
        const int32_t ex = block_exclusive<int32_t, 1024>(v, total);
        if (t < ntile)
            tile_alive[t] = static_cast<int32_t>(carry + ex);
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *alive_total = carry;
}

// Rank of slot q among the survivors of [q0, n) (its tile's prefix plus the
// survivors before it in the tile), for every slot of tile t at once.  The
// slot order inside a tile is k * TILE_THREADS + thread, scanned per k.
template <class T, class F>
__device__ __forceinline__ void edit_tile(const CaseDev &c, Slots<T> p, int64_t q0, int64_t n,
                                          int pred, int64_t t, int64_t tile_pre, F &&visit)
{
    int64_t run = tile_pre;
    for (int k = 0; k < TILE_VEC; ++k) {
        const int64_t q = q0 + t * TILE + k * TILE_THREADS + threadIdx.x;
        const bool valid = q < n;
        const bool alive = valid && !edit_removed(c, p, c.pbase + q, pred);
        int total;
        const int ex = block_exclusive<int>(alive ? 1 : 0, total);
        if (valid)
            visit(q, alive, run + ex);
        run += total;
        __syncthreads();
    }
}

// Removed slots below K into hole_pos, in slot order.
template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_edit_holes(const CaseDev *cases, int ci, Slots<T> p, int64_t q0, int64_t n, int pred,
                 const int32_t *tile_pre, const int64_t *alive_total, int64_t *hole_pos)
{
    const CaseDev &c = cases[ci];
    const int64_t keep = q0 + *alive_total;
    const int64_t ntile = (n - q0 + TILE - 1) / TILE;
    for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x)
        edit_tile(c, p, q0, n, pred, t, tile_pre[t], [&](int64_t q, bool alive, int64_t rank) {
            if (!alive && q < keep)
                hole_pos[(q - q0) - rank] = q; // removed slots before q
        });
}

// The survivors at or above K move into the holes: the r-th from the end
// into hole r.
template <class T>
__global__ void __launch_bounds__(TILE_THREADS)
    k_edit_fill(const CaseDev *cases, int ci, Slots<T> p, int64_t q0, int64_t n, int pred,
                const int32_t *tile_pre, const int64_t *alive_total, const int64_t *hole_pos,
                int *err)
{
    const CaseDev &c = cases[ci];
    const int64_t a = *alive_total;
    const int64_t keep = q0 + a;
    const int64_t ntile = (n - q0 + TILE - 1) / TILE;
    for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x)
        edit_tile(c, p, q0, n, pred, t, tile_pre[t], [&](int64_t q, bool alive, int64_t rank) {
            if (!alive || q < keep)
                return;
            const int64_t r = a - 1 - rank;
            if (r < 0 || r >= keep - q0) {
                report_error(err, DSMC_ERR_STATE);
                return;
            }
            const int64_t gs = c.pbase + q, gd = c.pbase + hole_pos[r];
            p.x[gd] = p.x[gs];
            p.y[gd] = p.y[gs];
            p.vx[gd] = p.vx[gs];
            p.vy[gd] = p.vy[gs];
            p.vz[gd] = p.vz[gs];
        });
}

// The new particle count of case ci after an edit.
__global__ void k_edit_commit(CaseState *st, int ci, int64_t q0, const int64_t *alive_total)
{
    st[ci].n_old = q0 + *alive_total;
}

} // namespace dsmc
