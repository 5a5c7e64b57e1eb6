// dsmc_device.cuh - device-side data layout and per-particle physics of the
// B200 DSMC engine.
//
// Arithmetic follows the reference expressions operation by operation (the
// library is compiled with --fmad=false so no multiply-add is contracted);
// sqrt and division are IEEE, log/cos/sin/pow/hypot are CUDA's double
// functions, which differ from the host's libm by at most a few ulp.
#pragma once

#include <cstdint>

#include "../../include/dsmc.h"
#include "../../include/dsmc_philox.h"

namespace dsmc {

// include/Constants.h:9 - bit-identical physical constant.
constexpr double K_BOLTZMANN = 1.380662E-23;
constexpr double PI_D = 3.14159265358979323846; // the value of M_PI

// A particle tile: 256 threads x 4 consecutive slots each.
constexpr int TILE_THREADS = 256;
constexpr int TILE_VEC = 4;
constexpr int TILE = TILE_THREADS * TILE_VEC;

// Sort key of a slot: bit 31 marks an "in-range" particle (still inside the
// slot range its cell owned after the previous sort), bit 30 a removed one,
// bits 0-29 hold the global cell id (for a removed particle its old cell, or
// all ones when it had none).  Cell ids and slots stay below 2^30.
constexpr uint32_t KEY_IN = 0x80000000u;
constexpr uint32_t KEY_DEAD = 0x40000000u;
constexpr uint32_t KEY_CELL = 0x3FFFFFFFu;
constexpr int32_t NO_CELL = -1;

// Bounded spin for the decoupled look-back chains (iterations of ~100 ns).
constexpr uint32_t SPIN_LIMIT = 1u << 22;

// Per-case constants, computed on the host with the reference expressions.
struct CaseDev {
    double x1, x2, y1, y2, dz;
    double dx, dy, dv, dt;
    double inv_dx, inv_dy;         // 1 / DX, 1 / DY (fast path of the cell index)
    double cull;                   // margin of the box pre-test (may_hit_box)
    double near_lo[2], near_hi[2]; // box widened by cull + 2^-20 of the coordinates
    // FP32 forms for the free-flight pass of FP32 slots: X1, Y1 and 1/DX, 1/DY
    // rounded to float; the bound on the error of the float cell estimate;
    // the domain bounds rounded inwards-exclusive (a float x is <= X1 iff it
    // is <= dom_lo[0], >= X2 iff >= dom_hi[0]); the near bounds rounded out.
    float fx1, fy1, finv_dx, finv_dy, fcell_hw; // fcell_hw: half-width of the certain window
    float dom_lo[2], dom_hi[2];
    float fnear_lo[2], fnear_hi[2];
    double box_lo[2], box_hi[2];   // IntersectBox bounds (Geometry.cpp:184-185)
    double box_x, box_y;           // InsideBox centre (Geometry.cpp:175-176)
    double box_hw, box_hh;         // BoxWidth / 2.0, BoxHeight / 2.0
    double rtw, sqrt_rtw;          // k Tw / m and its root (Boundary.cpp:213,216)
    double cll_an, cll_at;         // accommodation coefficients
    double cll_var_n, cll_var_t;   // an k Tw/m, at k Tw/m (Boundary.cpp:258,268,276)
    double cll_keep_n, cll_keep_t; // sqrt(1 - an), sqrt(1 - at) (Boundary.cpp:269,277)
    double mass, drag_scale;       // MoleculeMass, Weight * MoleculeMass
    double weight, sigma_ref, omega, cr_ref, sc_max;
    double ux_free, uy_free, rt_free; // freestream velocity, k TFree / m
    double strip[5][4];            // inflow strips L R B T and the cold-start box
    double strip_navg[5];          // Ngas V / Weight of each (Boundary.cpp:62-63)
    int32_t nx, ny, wall_model, first_sampling_step, sampling_period, max_per_cell;
    int32_t ncell, cbase;          // cells and first global cell id
    int64_t pbase, cap;            // first global slot and slot count
    uint32_t key0, key1;           // Philox key
};

// Per-case running state, updated on the device.
struct CaseState {
    int64_t n_old;        // particles at the start of the step (cell-sorted)
    int64_t step;
    int64_t sample_step;
    int64_t nc_last, nc_total, nc_step;
    int64_t particle_steps;
    unsigned long long drag_count;
    double drag_impulse;
    unsigned long long drag_count_window; // impacts of moves after FirstSamplingStep
    double drag_impulse_window;
    double time, sample_time, drag_time;
    int32_t sampling_mode;
    int32_t inj_count[5], inj_c0[5], inj_off[6];
    int64_t n_total;      // n_old + injected
    int64_t dead_old;     // removed particles among [0, n_old)
    int64_t dead_total;   // removed particles among [0, n_total)
    int64_t n_keep;       // survivors K
    int64_t n_holes;      // removed slots below K, refilled from the tail
    int32_t move_tile0, n_move_tiles;
    int32_t inject_tile0, n_inject_tiles;
    int32_t tail_tile0, n_tail_tiles;
    int32_t cell_tile0, n_cell_tiles;
    int32_t otile0, n_otiles;   // tiles of the per-case move-tile counts
};

// Whole-context counters of one step, cleared before each step.
struct StepScratch {
    uint32_t inject_ticket, tail_ticket, cell_ticket, otile_ticket;
    int32_t total_move_tiles, total_inject_tiles, total_tail_tiles;
    int32_t total_cell_tiles, total_otiles;
    uint32_t obuf_count;
    uint32_t near_count;  // slots queued by k_move for k_move_near
    uint32_t coll_count;  // cells listed by k_collide_select
    uint32_t holes_done;  // CTAs of k_holes that have finished
    int32_t init_mode;
};

// ---- random numbers --------------------------------------------------------

__device__ __forceinline__ double uniform(dsmc_stream &s) { return dsmc_stream_uniform(&s); }

__device__ __forceinline__ void open_stream(dsmc_stream &s, const CaseDev &c, uint32_t kind,
                                            int64_t step, uint32_t entity)
{
    s.key0 = c.key0;
    s.key1 = c.key1;
    s.kind = kind;
    s.step = static_cast<uint32_t>(step);
    s.entity = entity;
    s.next = 0;
    s.used = 4;
}

// frand_Gaussian, Boundary.cpp:49-50: the logarithm's draw first.
__device__ __forceinline__ double frand_gaussian(dsmc_stream &s, double mean, double var)
{
    const double u_log = uniform(s);
    const double u_angle = uniform(s);
    return mean + sqrt(-2.0 * var * log(u_log)) * cos(2.0 * PI_D * u_angle);
}

// frand_Rayleigh, rng/RayleighRNG.cxx:11-15
__device__ __forceinline__ double frand_rayleigh(dsmc_stream &s, double sigma)
{
    return sigma * sqrt(-2.0 * log(uniform(s)));
}

// irand_uniform, rng/DiscreteUniformRNG.cxx:11-14
__device__ __forceinline__ int irand_uniform(dsmc_stream &s, int n)
{
    return static_cast<int>(n * uniform(s));
}

// irand_Poisson, rng/PoissonRNG.cxx:11-22; *draws receives the draws used.
__device__ __forceinline__ int irand_poisson(dsmc_stream &s, double e, int *draws)
{
    const double exp_e = exp(-e);
    double prod = 1.0;
    int i = 0;
    do {
        i++;
        prod *= uniform(s);
    } while (prod >= exp_e && i < (1 << 30));
    *draws = i;
    return i - 1;
}

// The particle count of GenerateNewParticles (Boundary.cpp:62-71) for a mean
// of navg: floor plus a Bernoulli draw above 20, a Poisson draw otherwise;
// *draws receives the uniforms it used (the particles' draws follow them).
__device__ __forceinline__ int inflow_count(dsmc_stream &r, double navg, int *draws)
{
    if (navg > 20.0) {
        int n = static_cast<int>(navg);
        if (uniform(r) < navg - n)
            n++;
        *draws = 1;
        return n;
    }
    return irand_poisson(r, navg, draws);
}

// One particle of GenerateNewParticles (Boundary.cpp:85-90): a uniform
// position in the rectangle rect = (x1, y1, x2, y2) (v2rand_uniform_rect,
// :44-47), then a Maxwellian velocity around (ux, uy, 0) of variance rt =
// k T / m per component (vrand_MB, :52-57).  Eight draws.
__device__ __forceinline__ void new_particle(dsmc_stream &r, const double *rect, double ux,
                                             double uy, double rt, double &x, double &y,
                                             double &vx, double &vy, double &vz)
{
    x = rect[0] + (rect[2] - rect[0]) * uniform(r);
    y = rect[1] + (rect[3] - rect[1]) * uniform(r);
    vx = frand_gaussian(r, ux, rt);
    vy = frand_gaussian(r, uy, rt);
    vz = frand_gaussian(r, 0.0, rt);
}

// SampleGaussianPair, Boundary.cpp:27-41
__device__ __forceinline__ void gaussian_pair(dsmc_stream &s, double variance, double &first,
                                              double &second)
{
    if (variance == 0.0) {
        first = second = 0.0;
        return;
    }
    double u;
    do {
        u = uniform(s);
    } while (u <= 0.0 || u >= 1.0);
    const double radius = sqrt(-2.0 * variance * log(u));
    const double angle = 2.0 * PI_D * uniform(s);
    first = radius * cos(angle);
    second = radius * sin(angle);
}

// ---- wall interaction --------------------------------------------------------

// SpecularScattering, Boundary.cpp:235-241
__device__ __forceinline__ void specular(double v[3], double nx, double ny)
{
    const double vn = v[0] * nx + v[1] * ny;
    v[0] -= 2.0 * vn * nx;
    v[1] -= 2.0 * vn * ny;
}

// DiffuseScattering, Boundary.cpp:205-233
__device__ __forceinline__ void diffuse(dsmc_stream &s, const CaseDev &c, double v[3], double nx,
                                        double ny)
{
    const double vn = frand_rayleigh(s, c.sqrt_rtw);
    const double vt = frand_gaussian(s, 0.0, c.rtw);
    const double vz = frand_gaussian(s, 0.0, c.rtw);
    const double tx = -ny;
    const double ty = nx;
    v[0] = vn * nx + vt * tx;
    v[1] = vn * ny + vt * ty;
    v[2] = vz;
}

// CLLScattering, Boundary.cpp:243-282.  The coefficients are validated on the
// host before a context accepts them.
__device__ __forceinline__ void cll(dsmc_stream &s, const CaseDev &c, double v[3], double nx,
                                    double ny)
{
    if (c.cll_an == 0.0 && c.cll_at == 0.0) {
        specular(v, nx, ny);
        return;
    }
    const double in_normal = v[0] * nx + v[1] * ny;
    const double tx = -ny;
    const double ty = nx;
    const double in_tangent = v[0] * tx + v[1] * ty;
    const double in_z = v[2];
    double n1, n2;
    gaussian_pair(s, c.cll_var_n, n1, n2);
    const double retained_normal = c.cll_keep_n * fabs(in_normal);
    const double out_normal = hypot(retained_normal + n1, n2);
    double t_noise, z_noise;
    gaussian_pair(s, c.cll_var_t, t_noise, z_noise);
    const double out_tangent = c.cll_keep_t * in_tangent + t_noise;
    v[0] = out_normal * nx + out_tangent * tx;
    v[1] = out_normal * ny + out_tangent * ty;
    v[2] = c.cll_keep_t * in_z + z_noise;
}

__device__ __forceinline__ void wall_interaction(dsmc_stream &s, const CaseDev &c, double v[3],
                                                 double nx, double ny)
{
    if (c.wall_model == DSMC_WALL_SPECULAR)
        specular(v, nx, ny);
    else if (c.wall_model == DSMC_WALL_DIFFUSE)
        diffuse(s, c, v, nx, ny);
    else
        cll(s, c, v, nx, ny);
}

// ---- geometry ----------------------------------------------------------------

// InsideBox, Geometry.cpp:173-177
__device__ __forceinline__ bool inside_box(const CaseDev &c, double x, double y)
{
    return fabs(x - c.box_x) < c.box_hw && fabs(y - c.box_y) < c.box_hh;
}

// IntersectBox, Geometry.cpp:179-229: slab intervals; an exact corner entry
// goes to the x face; touching an edge or corner is not a hit.
__device__ __forceinline__ bool intersect_box(const CaseDev &c, double x, double y, double dx,
                                              double dy, double &t_hit, double &nxo, double &nyo)
{
    const double pos[2] = {x, y};
    const double disp[2] = {dx, dy};
    double entry = -INFINITY;
    double exit_t = INFINITY;
    int face_axis = -1;
    double face_normal = 0.0;
#pragma unroll
    for (int axis = 0; axis < 2; ++axis) {
        if (disp[axis] == 0.0) {
            if (pos[axis] <= c.box_lo[axis] || pos[axis] >= c.box_hi[axis])
                return false;
            continue;
        }
        double near_t = (c.box_lo[axis] - pos[axis]) / disp[axis];
        double far_t = (c.box_hi[axis] - pos[axis]) / disp[axis];
        double normal = -1.0;
        if (near_t > far_t) {
            const double tmp = near_t;
            near_t = far_t;
            far_t = tmp;
            normal = 1.0;
        }
        if (near_t > entry) {
            entry = near_t;
            face_axis = axis;
            face_normal = normal;
        }
        exit_t = (far_t < exit_t) ? far_t : exit_t; // std::min(exit, far)
    }
    if (face_axis < 0 || entry < 0.0 || entry > 1.0 || entry >= exit_t)
        return false;
    t_hit = entry;
    nxo = face_axis == 0 ? face_normal : 0.0;
    nyo = face_axis == 1 ? face_normal : 0.0;
    return true;
}

// Removal predicate of BoundaryConditions, Boundary.cpp:183-188.
__device__ __forceinline__ bool outside_domain(const CaseDev &c, double x, double y)
{
    return x <= c.x1 || x >= c.x2 || y <= c.y1 || y >= c.y2;
}

// floor(u / d) with the IEEE quotient, as the reference computes it.  The
// quotient is first estimated as u * (1/d), which is within a few ulp of it;
// unless the estimate lies within 1e-9 of an integer (or |u/d| is huge, or
// NaN), both floors are the same integer and the division is skipped.
__device__ __forceinline__ double floor_div(double u, double d, double inv_d)
{
    const double q = u * inv_d;
    const double f = floor(q);
    const double r = q - f;
    if (r > 1e-9 && r < 1.0 - 1e-9 && fabs(q) < 1e6)
        return f;
    return floor(u / d);
}

// Cell of a position (Geometry.cpp:47-59); -1 when outside the grid or NaN,
// where the reference aborts (MPIManager.cpp:602-632).
__device__ __forceinline__ int32_t cell_of(const CaseDev &c, double x, double y)
{
    const double fk = floor_div(x - c.x1, c.dx, c.inv_dx);
    const double fl = floor_div(y - c.y1, c.dy, c.inv_dy);
    if (!(fk >= 0.0 && fk < c.nx && fl >= 0.0 && fl < c.ny))
        return NO_CELL;
    return static_cast<int32_t>(fk) * c.ny + static_cast<int32_t>(fl);
}

// Estimate-only form of cell_of for the free-flight pass: false when either
// floor is not certain from the estimate (the exact form then decides), else
// the cell (NO_CELL outside the grid) in `cell`.
__device__ __forceinline__ bool cell_of_fast(const CaseDev &c, double x, double y, int32_t &cell)
{
    const double qk = (x - c.x1) * c.inv_dx;
    const double ql = (y - c.y1) * c.inv_dy;
    const double fk = floor(qk);
    const double fl = floor(ql);
    const double rk = qk - fk;
    const double rl = ql - fl;
    if (!(rk > 1e-9 && rk < 1.0 - 1e-9 && rl > 1e-9 && rl < 1.0 - 1e-9 && fabs(qk) < 1e6 &&
          fabs(ql) < 1e6))
        return false;
    cell = (fk >= 0.0 && fk < c.nx && fl >= 0.0 && fl < c.ny)
               ? static_cast<int32_t>(fk) * c.ny + static_cast<int32_t>(fl)
               : NO_CELL;
    return true;
}

// FP32 estimate of the cell of a float position for the free-flight pass.
// The estimate q' = (x - fx1) * finv_dx differs from (x - X1) / DX by less
// than a bound e inside the grid (float rounding of X1, 1/DX, the difference
// and the product; computed on the host), so when q' is more than e from an
// integer its floor is the reference's FP64 floor.  Returns false when not
// certain.
//
// floor(q') comes from rounding q' - 0.5 to an integer with the 1.5 * 2^23
// constant; r = q' - floor is then certain when |r - 0.5| < fcell_hw
// (= 0.5 - e, less a margin for the rounding of r - 0.5).  A tie or
// any |q'| >= 2^21 gives r outside that window, so no separate range check
// is needed; the host keeps the grid below 2^20 cells per side for this
// path (fcell_hw < 0 turns it off).
__device__ __forceinline__ bool floor_fast_f(float q, float hw, int32_t &n)
{
    const float t = (q - 0.5f) + 12582912.0f;
    const float f = t - 12582912.0f;
    n = __float_as_int(t) - 0x4B400000;
    return fabsf((q - f) - 0.5f) < hw;
}

__device__ __forceinline__ bool cell_of_fast_f(const CaseDev &c, float x, float y, int32_t &cell)
{
    int32_t k, l;
    const bool ok = floor_fast_f((x - c.fx1) * c.finv_dx, c.fcell_hw, k) &
                    floor_fast_f((y - c.fy1) * c.finv_dy, c.fcell_hw, l);
    const bool in = (static_cast<uint32_t>(k) < static_cast<uint32_t>(c.nx)) &
                    (static_cast<uint32_t>(l) < static_cast<uint32_t>(c.ny));
    cell = in ? static_cast<int32_t>(static_cast<uint32_t>(k) * static_cast<uint32_t>(c.ny) +
                                     static_cast<uint32_t>(l))
              : NO_CELL;
    return ok;
}

// Removal predicate of BoundaryConditions (Boundary.cpp:183-188) for a float
// position, exact: compares against the float bounds described in CaseDev.
__device__ __forceinline__ bool outside_domain_f(const CaseDev &c, float x, float y)
{
    return (x <= c.dom_lo[0]) | (x >= c.dom_hi[0]) | (y <= c.dom_lo[1]) | (y >= c.dom_hi[1]);
}

// near_box for a float segment (start, rounded end): the float near bounds
// contain the FP64 ones, and the end point's rounding (2^-24 of it) is far
// inside the 2^-20 widening, so "not near" here implies "not near" in FP64.
__device__ __forceinline__ bool near_box_f(const CaseDev &c, float x0, float y0, float x1, float y1)
{
    return (fmaxf(x0, x1) > c.fnear_lo[0]) & (fminf(x0, x1) < c.fnear_hi[0]) &
           (fmaxf(y0, y1) > c.fnear_lo[1]) & (fminf(y0, y1) < c.fnear_hi[1]);
}

// False only when IntersectBox cannot report an impact: the segment's
// bounding box is more than `cull` clear of the box.  An impact needs the
// slab entry time <= 1 and the exit time >= 0, i.e. the segment reaching the
// box to within a few ulp of its coordinates; `cull` (1e-9 m plus 1e-9 of the
// coordinates) is many orders above that, so skipping the slab test here
// never changes a result.
__device__ __forceinline__ bool may_hit_box(const CaseDev &c, double x0, double y0, double x1,
                                            double y1)
{
    return fmax(x0, x1) > c.box_lo[0] - c.cull && fmin(x0, x1) < c.box_hi[0] + c.cull &&
           fmax(y0, y1) > c.box_lo[1] - c.cull && fmin(y0, y1) < c.box_hi[1] + c.cull;
}

// False when the segment's bounding box is clear of the box widened to
// near_lo / near_hi.  The widening (cull plus 2^-20 of the largest coordinate)
// covers both the margin of may_hit_box and the FP32 rounding of the end
// point (at most 2^-24 of it), so a segment that is not near the box neither
// hits it nor ends, rounded to storage precision, inside it.
__device__ __forceinline__ bool near_box(const CaseDev &c, double x0, double y0, double x1,
                                         double y1)
{
    return fmax(x0, x1) > c.near_lo[0] && fmin(x0, x1) < c.near_hi[0] &&
           fmax(y0, y1) > c.near_lo[1] && fmin(y0, y1) < c.near_hi[1];
}

// ---- storage precision ---------------------------------------------------------

template <class T> struct Store;

template <> struct Store<double> {
    __device__ __forceinline__ static double rn(double v) { return v; }
    __device__ __forceinline__ static double down(double v) { return v; }
    __device__ __forceinline__ static double up(double v) { return v; }
};

template <> struct Store<float> {
    __device__ __forceinline__ static float rn(double v) { return __double2float_rn(v); }
    __device__ __forceinline__ static float down(double v) { return __double2float_rd(v); }
    __device__ __forceinline__ static float up(double v) { return __double2float_ru(v); }
};

// Rounds a post-impact coordinate to storage precision away from the face it
// left (normal component n = -1, 0 or +1), so an FP32 particle never lands on
// or inside the box.  Identity for FP64.
template <class T> __device__ __forceinline__ T round_out(double v, double n)
{
    return n < 0.0 ? Store<T>::down(v) : (n > 0.0 ? Store<T>::up(v) : Store<T>::rn(v));
}

// Keeps a stored coordinate inside [lo, hi).  The cold-start fill draws in
// [X1, X2) in FP64; rounded to FP32 a draw just below X2 can become X2
// itself, which lies in no cell.  In FP64 the largest draw stays ~1e-8 m
// inside (u <= 1 - 4.7e-10), so the double version is the identity.
template <class T> __device__ __forceinline__ T clamp_into(T v, double, double) { return v; }

template <> __device__ __forceinline__ float clamp_into<float>(float v, double lo, double hi)
{
    if (static_cast<double>(v) < lo)
        v = __double2float_ru(lo);
    for (int i = 0; i < 4 && static_cast<double>(v) >= hi; ++i)
        v = nextafterf(v, -INFINITY);
    return v;
}

// FP32 only: a free-flight end point rounded to float can fall inside a box
// whose faces are not floats.  Push it to the nearest face's outside.
template <class T>
__device__ __forceinline__ void keep_outside(const CaseDev &c, T &x, T &y)
{
    if (sizeof(T) == sizeof(double))
        return;
    if (!inside_box(c, static_cast<double>(x), static_cast<double>(y)))
        return;
    const double dl = static_cast<double>(x) - c.box_lo[0];
    const double dr = c.box_hi[0] - static_cast<double>(x);
    const double db = static_cast<double>(y) - c.box_lo[1];
    const double dt = c.box_hi[1] - static_cast<double>(y);
    const double m = fmin(fmin(dl, dr), fmin(db, dt));
    if (m == dl)
        x = Store<T>::down(c.box_lo[0] - c.box_hw * 1e-7);
    else if (m == dr)
        x = Store<T>::up(c.box_hi[0] + c.box_hw * 1e-7);
    else if (m == db)
        y = Store<T>::down(c.box_lo[1] - c.box_hh * 1e-7);
    else
        y = Store<T>::up(c.box_hi[1] + c.box_hh * 1e-7);
}

// ---- warp helpers ------------------------------------------------------------------

// Adds 1 to counter[key] for every active lane, with one atomic per distinct
// key in the warp (cell-sorted particles share keys, so this is usually one
// or two atomics per warp).  All 32 lanes must call it.
__device__ __forceinline__ void warp_aggregated_inc(int32_t *counter, int32_t key, bool active)
{
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active)
        return;
    const unsigned peers = __match_any_sync(mask, key);
    if ((threadIdx.x & 31) == __ffs(peers) - 1)
        atomicAdd(counter + key, __popc(peers));
}

} // namespace dsmc
