/*
 * dsmc_oracle.c - CPU restatement of the reference DSMC time step.
 *
 * TEST INFRASTRUCTURE ONLY (see dsmc_oracle.h).  Plain C99, FP64, single
 * threaded, compiled with -ffp-contract=off so every expression is the IEEE
 * operation sequence written here, in the order the reference writes it.
 * Each function names the reference lines it restates.
 */
#include "dsmc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/dsmc_philox.h"

/* include/Constants.h:9-10 - physical constants, bit-identical. */
#define K_BOLTZMANN 1.380662E-23
#define N_AVOGADRO 6.022045E+23
#define PI_D 3.14159265358979323846 /* the value of M_PI */

struct dsmc_oracle {
    dsmc_params p;
    dsmc_derived d;
    int64_t cap, np;
    double *x, *y, *vx, *vy, *vz;
    double *sx, *sy, *svx, *svy, *svz; /* reorder scratch */
    int32_t ncell;
    int32_t *cell_start; /* ncell + 1, valid after the index stage */
    int32_t *cell_of;    /* per particle, scratch of the index stage */
    int32_t *fill;
    double *acc; /* 17 doubles per cell, CELL layout (include/Cell.h:4-10) */
    int64_t step, sample_step;
    int sampling_mode;
    double time, sample_time, drag_impulse, drag_sampling_time;
    int64_t drag_count, last_nc, total_nc, particle_steps;
    double drag_impulse_window; /* impacts of moves after FirstSamplingStep */
    int64_t drag_count_window;
    double box_lo[2], box_hi[2];
    double local[4]; /* LocalX1 LocalY1 LocalX2 LocalY2 (MPIManager.cpp:216-229) */
    dsmc_stream rng;
};

/* ---- random numbers ----------------------------------------------------- */

static void select_stream(dsmc_oracle *o, uint32_t kind, uint64_t step, uint32_t entity)
{
    dsmc_stream_init(&o->rng, o->p.seed, kind, (uint32_t)step, entity);
}

/* brng(), rng/BRNG.cxx:30-34, drawn from the selected keyed stream. */
static double brng(dsmc_oracle *o) { return dsmc_stream_uniform(&o->rng); }

/* irand_uniform, rng/DiscreteUniformRNG.cxx:11-14 */
static int irand_uniform(dsmc_oracle *o, int n) { return (int)(n * brng(o)); }

/* irand_Poisson, rng/PoissonRNG.cxx:11-22 (Knuth's product method) */
static int irand_poisson(dsmc_oracle *o, double e)
{
    const double exp_e = exp(-e);
    double prod = 1.0;
    int i = 0;
    do {
        i++;
        prod *= brng(o);
    } while (prod >= exp_e);
    return i - 1;
}

/* frand_Rayleigh, rng/RayleighRNG.cxx:11-15 */
static double frand_rayleigh(dsmc_oracle *o, double s) { return s * sqrt(-2.0 * log(brng(o))); }

/* v3rand_isotropic, rng/IsotropicVectorRNG.cxx:11-19 */
static void v3rand_isotropic(dsmc_oracle *o, double *r)
{
    const double cos_t = 1.0 - 2.0 * brng(o);
    const double sin_t = sqrt(1.0 - cos_t * cos_t);
    const double e = 2.0 * PI_D * brng(o);
    r[0] = cos_t;
    r[1] = sin_t * cos(e);
    r[2] = sin_t * sin(e);
}

/* frand_Gaussian, src/Boundary.cpp:49-50.  The two draws sit in one
 * expression; the reference compiler evaluates the logarithm's draw first. */
static double frand_gaussian(dsmc_oracle *o, double mean, double var)
{
    const double u_log = brng(o);
    const double u_angle = brng(o);
    return mean + sqrt(-2.0 * var * log(u_log)) * cos(2.0 * PI_D * u_angle);
}

/* vrand_MB, src/Boundary.cpp:52-57 */
static void vrand_mb(dsmc_oracle *o, double *v, double m, const double *u, double t)
{
    const double rt = K_BOLTZMANN * t / m;
    v[0] = frand_gaussian(o, u[0], rt);
    v[1] = frand_gaussian(o, u[1], rt);
    v[2] = frand_gaussian(o, u[2], rt);
}

/* SampleGaussianPair, src/Boundary.cpp:27-41 */
static void sample_gaussian_pair(dsmc_oracle *o, double variance, double *first, double *second)
{
    if (variance == 0.0) {
        *first = *second = 0.0;
        return;
    }
    double u;
    do {
        u = brng(o);
    } while (u <= 0.0 || u >= 1.0);
    const double radius = sqrt(-2.0 * variance * log(u));
    const double angle = 2.0 * PI_D * brng(o);
    *first = radius * cos(angle);
    *second = radius * sin(angle);
}

/* ---- wall interaction --------------------------------------------------- */

/* SpecularScattering, src/Boundary.cpp:235-241 */
static void specular(double *v, double nx, double ny)
{
    const double vn = v[0] * nx + v[1] * ny;
    v[0] -= 2.0 * vn * nx;
    v[1] -= 2.0 * vn * ny;
}

/* DiffuseScattering, src/Boundary.cpp:205-233 */
static void diffuse(dsmc_oracle *o, double *v, double m, double tw, double nx, double ny)
{
    const double rtw = K_BOLTZMANN * tw / m;
    const double vn = frand_rayleigh(o, sqrt(rtw));
    const double vt = frand_gaussian(o, 0.0, rtw);
    const double vz = frand_gaussian(o, 0.0, rtw);
    const double tx = -ny;
    const double ty = nx;
    v[0] = vn * nx + vt * tx;
    v[1] = vn * ny + vt * ty;
    v[2] = vz;
}

static int cll_valid(double an, double at)
{
    return isfinite(an) && an >= 0.0 && an <= 1.0 && isfinite(at) && at >= 0.0 && at <= 1.0;
}

/* CLLScattering, src/Boundary.cpp:243-282 */
static int cll(dsmc_oracle *o, double *v, double m, double tw, double nx, double ny, double an,
               double at)
{
    if (!cll_valid(an, at))
        return DSMC_ERR_BAD_CLL;
    if (an == 0.0 && at == 0.0) {
        specular(v, nx, ny);
        return DSMC_OK;
    }
    const double thermal_variance = K_BOLTZMANN * tw / m;
    const double in_normal = v[0] * nx + v[1] * ny;
    const double tx = -ny;
    const double ty = nx;
    const double in_tangent = v[0] * tx + v[1] * ty;
    const double in_z = v[2];
    double n1, n2;
    sample_gaussian_pair(o, an * thermal_variance, &n1, &n2);
    const double retained_normal = sqrt(1.0 - an) * fabs(in_normal);
    const double out_normal = hypot(retained_normal + n1, n2);
    double t_noise, z_noise;
    sample_gaussian_pair(o, at * thermal_variance, &t_noise, &z_noise);
    const double retained_tangent = sqrt(1.0 - at);
    const double out_tangent = retained_tangent * in_tangent + t_noise;
    v[0] = out_normal * nx + out_tangent * tx;
    v[1] = out_normal * ny + out_tangent * ty;
    v[2] = retained_tangent * in_z + z_noise;
    return DSMC_OK;
}

static int wall_interaction(dsmc_oracle *o, double *v, double nx, double ny)
{
    switch (o->p.wall_model) {
    case DSMC_WALL_SPECULAR:
        specular(v, nx, ny);
        return DSMC_OK;
    case DSMC_WALL_DIFFUSE:
        diffuse(o, v, o->d.molecule_mass, o->p.t_wall, nx, ny);
        return DSMC_OK;
    case DSMC_WALL_CLL:
        return cll(o, v, o->d.molecule_mass, o->p.t_wall, nx, ny, o->p.cll_normal,
                   o->p.cll_tangential);
    }
    return DSMC_ERR_ARGUMENT;
}

/* ---- geometry ----------------------------------------------------------- */

/* InsideBox, src/Geometry.cpp:173-177 */
static int inside_box(const dsmc_oracle *o, double x, double y)
{
    return fabs(x - o->p.box_x) < o->p.box_width / 2.0 &&
           fabs(y - o->p.box_y) < o->p.box_height / 2.0;
}

/* IntersectBox, src/Geometry.cpp:179-229: slab test, corner ties go to x. */
static int intersect_box(const dsmc_oracle *o, double x, double y, double dx, double dy,
                         double *t_hit, double *nxo, double *nyo)
{
    const double pos[2] = {x, y};
    const double disp[2] = {dx, dy};
    double entry = -INFINITY;
    double exit_t = INFINITY;
    int face_axis = -1;
    double face_normal = 0.0;
    for (int axis = 0; axis < 2; ++axis) {
        if (disp[axis] == 0.0) {
            if (pos[axis] <= o->box_lo[axis] || pos[axis] >= o->box_hi[axis])
                return 0;
            continue;
        }
        double near_t = (o->box_lo[axis] - pos[axis]) / disp[axis];
        double far_t = (o->box_hi[axis] - pos[axis]) / disp[axis];
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
        exit_t = (far_t < exit_t) ? far_t : exit_t; /* std::min(exit, far) */
    }
    if (face_axis < 0 || entry < 0.0 || entry > 1.0 || entry >= exit_t)
        return 0;
    *t_hit = entry;
    *nxo = face_axis == 0 ? face_normal : 0.0;
    *nyo = face_axis == 1 ? face_normal : 0.0;
    return 1;
}

/* ---- storage ------------------------------------------------------------ */

static void swap_last(dsmc_oracle *o, int64_t i)
{
    const int64_t last = o->np - 1;
    if (i < last) {
        o->x[i] = o->x[last];
        o->y[i] = o->y[last];
        o->vx[i] = o->vx[last];
        o->vy[i] = o->vy[last];
        o->vz[i] = o->vz[last];
    }
    o->np--;
}

/* ---- stages ------------------------------------------------------------- */

/* One particle of MoveParticles, src/Boundary.cpp:286-327. */
static int move_one(dsmc_oracle *o, int64_t i)
{
    const double dt = o->p.dt;
    const double x0 = o->x[i];
    const double y0 = o->y[i];
    const double dx = dt * o->vx[i];
    const double dy = dt * o->vy[i];
    double t_hit, nx, ny;
    if (!intersect_box(o, x0, y0, dx, dy, &t_hit, &nx, &ny)) {
        o->x[i] = x0 + dx;
        o->y[i] = y0 + dy;
        return DSMC_OK;
    }
    const double x_hit = x0 + t_hit * dx;
    const double y_hit = y0 + t_hit * dy;
    double v[3] = {o->vx[i], o->vy[i], o->vz[i]};
    const double vx_in = v[0];
    select_stream(o, DSMC_RNG_MOVE, o->step, (uint32_t)i);
    const int s = wall_interaction(o, v, nx, ny);
    if (s != DSMC_OK)
        return s;
    o->vx[i] = v[0];
    o->vy[i] = v[1];
    o->vz[i] = v[2];
    o->drag_impulse += o->d.weight * o->d.molecule_mass * (vx_in - v[0]);
    o->drag_count++;
    if (o->step > o->p.first_sampling_step) {
        o->drag_impulse_window += o->d.weight * o->d.molecule_mass * (vx_in - v[0]);
        o->drag_count_window++;
    }
    const double remaining = dt * (1.0 - t_hit);
    const double eps = 1e-12;
    o->x[i] = x_hit + remaining * v[0] + eps * nx;
    o->y[i] = y_hit + remaining * v[1] + eps * ny;
    return DSMC_OK;
}

/* GenerateNewParticles, src/Boundary.cpp:60-92, with v2rand_uniform_rect
 * (:44-47) inlined.  Draws come from the stream selected by the caller. */
static int generate_gas(dsmc_oracle *o, double gx1, double gy1, double gx2, double gy2,
                        double n_gas, double ux_gas, double uy_gas, double t_gas, int move_flag)
{
    const double v = (gx2 - gx1) * (gy2 - gy1) * o->p.dz;
    const double n_avg = n_gas * v / o->d.weight;
    int n_new;
    if (n_avg > 20.0) {
        n_new = (int)n_avg;
        if (brng(o) < n_avg - n_new)
            n_new++;
    } else {
        n_new = irand_poisson(o, n_avg);
    }
    if (o->np + n_new > o->cap)
        return DSMC_ERR_CAPACITY;
    const double u_gas[3] = {ux_gas, uy_gas, 0.0};
    for (int64_t i = o->np; i < o->np + n_new; ++i) {
        o->x[i] = gx1 + (gx2 - gx1) * brng(o);
        o->y[i] = gy1 + (gy2 - gy1) * brng(o);
        double vel[3];
        vrand_mb(o, vel, o->d.molecule_mass, u_gas, t_gas);
        o->vx[i] = vel[0];
        o->vy[i] = vel[1];
        o->vz[i] = vel[2];
        if (move_flag == 1) {
            o->x[i] += o->p.dt * o->vx[i];
            o->y[i] += o->p.dt * o->vy[i];
        }
    }
    o->np += n_new;
    return DSMC_OK;
}

/* The freestream form that BoundaryConditions and InitialConditions use. */
static int generate(dsmc_oracle *o, double gx1, double gy1, double gx2, double gy2, int move_flag)
{
    return generate_gas(o, gx1, gy1, gx2, gy2, o->p.n_free, o->d.ux_free, o->d.uy_free,
                        o->p.t_free, move_flag);
}

int dsmc_oracle_stage_move(dsmc_oracle *o)
{
    /* Simulation.cpp:139-142 */
    o->sampling_mode =
        (o->step > o->p.first_sampling_step && o->step % o->p.sampling_period == 0) ? 1 : 0;
    for (int64_t i = 0; i < o->np; ++i) {
        const int s = move_one(o, i);
        if (s != DSMC_OK)
            return s;
    }
    if (o->step > o->p.first_sampling_step) /* Simulation.cpp:144-146 */
        o->drag_sampling_time += o->p.dt;
    return DSMC_OK;
}

/* BoundaryConditions, src/Boundary.cpp:94-203: the four inflow strips (no
 * corner strips), one stream each, then swap-with-last removal. */
int dsmc_oracle_stage_boundary(dsmc_oracle *o)
{
    const dsmc_params *p = &o->p;
    const double *lc = o->local;
    const double strips[4][4] = {
        {p->x1 - p->dl, lc[1], p->x1, lc[3]},
        {p->x2, lc[1], p->x2 + p->dl, lc[3]},
        {lc[0], p->y1 - p->dl, lc[2], p->y1},
        {lc[0], p->y2, lc[2], p->y2 + p->dl},
    };
    for (uint32_t s = 0; s < 4; ++s) {
        select_stream(o, DSMC_RNG_INJECT, o->step, s);
        const int st = generate(o, strips[s][0], strips[s][1], strips[s][2], strips[s][3], 1);
        if (st != DSMC_OK)
            return st;
    }
    return dsmc_oracle_remove_outside_domain(o);
}

/* The removal loop of BoundaryConditions, src/Boundary.cpp:181-202. */
int dsmc_oracle_remove_outside_domain(dsmc_oracle *o)
{
    const dsmc_params *p = &o->p;
    for (int64_t i = 0; i < o->np;) {
        if (o->x[i] <= p->x1 || o->x[i] >= p->x2 || o->y[i] <= p->y1 || o->y[i] >= p->y2)
            swap_last(o, i);
        else
            i++;
    }
    return DSMC_OK;
}

/* Indexing, src/Geometry.cpp:37-170, then the stable reorder into cell order
 * k*NY + l that keeps each cell's particles in particle order (the order of
 * the reference's IPC lists). */
int dsmc_oracle_stage_index(dsmc_oracle *o)
{
    const dsmc_params *p = &o->p;
    memset(o->cell_start, 0, sizeof(int32_t) * (size_t)(o->ncell + 1));
    for (int64_t i = 0; i < o->np; ++i) {
        const int k = (int)floor((o->x[i] - p->x1) / o->d.dx);
        const int l = (int)floor((o->y[i] - p->y1) / o->d.dy);
        /* The reference checks this first in ExchangeParticles
         * (src/MPIManager.cpp:602-632, code 30), then in Indexing (code 20). */
        if (k < 0 || k >= p->nx || l < 0 || l >= p->ny)
            return DSMC_ERR_EXCHANGE;
        const int32_t c = k * p->ny + l;
        o->cell_of[i] = c;
        o->cell_start[c + 1]++;
    }
    if (p->max_particles_in_cell > 0)
        for (int32_t c = 0; c < o->ncell; ++c)
            if (o->cell_start[c + 1] > p->max_particles_in_cell)
                return DSMC_ERR_CELL_OVERFLOW;
    for (int32_t c = 0; c < o->ncell; ++c)
        o->cell_start[c + 1] += o->cell_start[c];
    memcpy(o->fill, o->cell_start, sizeof(int32_t) * (size_t)o->ncell);
    for (int64_t i = 0; i < o->np; ++i) {
        const int32_t dst = o->fill[o->cell_of[i]]++;
        o->sx[dst] = o->x[i];
        o->sy[dst] = o->y[i];
        o->svx[dst] = o->vx[i];
        o->svy[dst] = o->vy[i];
        o->svz[dst] = o->vz[i];
    }
    double *t;
    t = o->x; o->x = o->sx; o->sx = t;
    t = o->y; o->y = o->sy; o->sy = t;
    t = o->vx; o->vx = o->svx; o->svx = t;
    t = o->vy; o->vy = o->svy; o->svy = t;
    t = o->vz; o->vz = o->svz; o->svz = t;
    return DSMC_OK;
}

/* ElasticCollision, src/Collision.cpp:7-19 */
static void elastic_v(dsmc_oracle *o, double *v1, double *v2, double cr)
{
    double n[3];
    v3rand_isotropic(o, n);
    cr *= 0.5;
    const double vc[3] = {0.5 * (v2[0] + v1[0]), 0.5 * (v2[1] + v1[1]), 0.5 * (v2[2] + v1[2])};
    const double vcr[3] = {cr * n[0], cr * n[1], cr * n[2]};
    v1[0] = vc[0] + vcr[0];
    v1[1] = vc[1] + vcr[1];
    v1[2] = vc[2] + vcr[2];
    v2[0] = vc[0] - vcr[0];
    v2[1] = vc[1] - vcr[1];
    v2[2] = vc[2] - vcr[2];
}

static void elastic(dsmc_oracle *o, int64_t a, int64_t b, double cr)
{
    double v1[3] = {o->vx[a], o->vy[a], o->vz[a]};
    double v2[3] = {o->vx[b], o->vy[b], o->vz[b]};
    elastic_v(o, v1, v2, cr);
    o->vx[a] = v1[0];
    o->vy[a] = v1[1];
    o->vz[a] = v1[2];
    o->vx[b] = v2[0];
    o->vy[b] = v2[1];
    o->vz[b] = v2[2];
}

/* BinaryCollisionsInCell, src/Collision.cpp:21-44: NTC with fixed SCMax and
 * VHS acceptance.  The cell's list IPC is ids[0, n) when ids is given, else
 * the contiguous run [start, start+n); cell_volume is the CellVolume
 * argument (DV in CollideParticles). */
static int collide_ids(dsmc_oracle *o, int64_t start, const int32_t *ids, int n,
                       double cell_volume)
{
    if (n < 2)
        return 0;
    const double sc_max = 9.0 * o->d.sigma_ref *
                          sqrt(K_BOLTZMANN * o->p.t_free / o->d.molecule_mass);
    const double npair = 0.5 * n * (n - 1) * o->d.weight * sc_max * o->p.dt / cell_volume;
    int nn = (int)npair;
    const double frac = npair - nn;
    nn = (brng(o) < frac) ? nn + 1 : nn;
    int nc = 0;
    for (int k = 0; k < nn; k++) {
        int i = irand_uniform(o, n);
        int j;
        do {
            j = irand_uniform(o, n);
        } while (j == i);
        const int64_t a = ids ? ids[i] : start + i;
        const int64_t b = ids ? ids[j] : start + j;
        const double vr[3] = {o->vx[b] - o->vx[a], o->vy[b] - o->vy[a], o->vz[b] - o->vz[a]};
        const double cr = sqrt(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
        const double sigma = o->d.sigma_ref * pow(o->d.cr_ref / cr, o->d.omega);
        if (brng(o) < sigma * cr / sc_max) {
            elastic(o, a, b, cr);
            nc++;
        }
    }
    return nc;
}

static int collide_cell(dsmc_oracle *o, int64_t start, int n)
{
    return collide_ids(o, start, NULL, n, o->d.dv);
}

/* CollideParticles, src/Collision.cpp:45-56, one stream per cell. */
int dsmc_oracle_stage_collide(dsmc_oracle *o)
{
    int64_t nc = 0;
    for (int32_t c = 0; c < o->ncell; ++c) {
        select_stream(o, DSMC_RNG_COLLIDE, o->step, (uint32_t)c);
        const int ncc =
            collide_cell(o, o->cell_start[c], o->cell_start[c + 1] - o->cell_start[c]);
        nc += ncc;
        if (o->sampling_mode == 1)
            o->acc[17 * (int64_t)c + 16] += ncc;
    }
    o->last_nc = nc;
    o->total_nc += nc;
    return DSMC_OK;
}

/* Sampling, src/Sampling.cpp:14-31 */
int dsmc_oracle_stage_sample(dsmc_oracle *o)
{
    if (o->sampling_mode != 1)
        return DSMC_OK;
    o->sample_step++;
    o->sample_time += o->p.dt;
    for (int32_t c = 0; c < o->ncell; ++c) {
        double *a = o->acc + 17 * (int64_t)c;
        for (int64_t i = o->cell_start[c]; i < o->cell_start[c + 1]; ++i) {
            const double v[3] = {o->vx[i], o->vy[i], o->vz[i]};
            a[0] += 1.0;
            const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            for (int m = 0; m < 3; m++) {
                a[1 + m] += v[m];
                a[13 + m] += v2 * v[m];
                for (int n = 0; n < 3; n++)
                    a[4 + 3 * m + n] += v[m] * v[n];
            }
        }
    }
    return DSMC_OK;
}

/* Simulation.cpp:160-161 */
int dsmc_oracle_stage_end_step(dsmc_oracle *o)
{
    o->particle_steps += o->np;
    o->step++;
    o->time += o->p.dt;
    return DSMC_OK;
}

int dsmc_oracle_step(dsmc_oracle *o)
{
    int s;
    if ((s = dsmc_oracle_stage_move(o)) != DSMC_OK) return s;
    if ((s = dsmc_oracle_stage_boundary(o)) != DSMC_OK) return s;
    if ((s = dsmc_oracle_stage_index(o)) != DSMC_OK) return s;
    if ((s = dsmc_oracle_stage_collide(o)) != DSMC_OK) return s;
    if ((s = dsmc_oracle_stage_sample(o)) != DSMC_OK) return s;
    return dsmc_oracle_stage_end_step(o);
}

/* RemoveParticlesInsideBox, src/Geometry.cpp:231-247 (swap-with-last). */
int dsmc_oracle_remove_inside_box(dsmc_oracle *o)
{
    for (int64_t i = 0; i < o->np;) {
        if (inside_box(o, o->x[i], o->y[i]))
            swap_last(o, i);
        else
            i++;
    }
    return DSMC_OK;
}

/* InitialConditions, src/Initialization.cpp:290-313, with
 * RemoveParticlesInsideBox (src/Geometry.cpp:231-247), then the cell sort. */
int dsmc_oracle_init_cold(dsmc_oracle *o)
{
    o->step = 0;
    o->time = 0.0;
    o->np = 0;
    o->sample_step = 0;
    o->sample_time = 0.0;
    memset(o->acc, 0, sizeof(double) * 17 * (size_t)o->ncell);
    select_stream(o, DSMC_RNG_INIT, 0, 0);
    int s = generate(o, o->local[0], o->local[1], o->local[2], o->local[3], 0);
    if (s != DSMC_OK)
        return s;
    dsmc_oracle_remove_inside_box(o);
    return dsmc_oracle_stage_index(o);
}

/* ---- setup -------------------------------------------------------------- */

/* Gamma(x), x > 0, src/Initialization.cpp:111-207: the reference's private
 * routine, restated from the published method it follows.  Below 0.001 the
 * two-term series of 1/Gamma; on [0.001, 12) W. J. Cody's rational
 * approximation Gamma(1 + z) = 1 + z P(z) / Q(z) on (1, 2) (SPECFUN; the
 * degree-8 coefficient table as published) with the recurrence outside
 * (1, 2); from 12 Stirling's series, Abramowitz and Stegun 6.1.41.  The
 * operation order is the reference's, so the result has its bits. */
static double gamma_fn(double x)
{
    static const double P[8] = {-1.71618513886549492533811E+0, 2.47656508055759199108314E+1,
                                -3.79804256470945635097577E+2, 6.29331155312818442661052E+2,
                                8.66966202790413211295064E+2, -3.14512729688483675254357E+4,
                                -3.61444134186911729807069E+4, 6.64561438202405440627855E+4};
    static const double Q[8] = {-3.08402300119738975254353E+1, 3.15350626979604161529144E+2,
                                -1.01515636749021914166146E+3, -3.10777167157231109440444E+3,
                                2.25381184209801510330112E+4, 4.75584627752788110767815E+3,
                                -1.34659959864969306392456E+5, -1.15132259675553483497211E+5};
    static const double B[8] = {1.0 / 12.0, -1.0 / 360.0, 1.0 / 1260.0, -1.0 / 1680.0,
                                1.0 / 1188.0, -691.0 / 360360.0, 1.0 / 156.0,
                                -3617.0 / 122400.0};
    if (x < 0.001)
        return 1.0 / (x * (1.0 + 0.577215664901532860606512090 * x));
    if (x < 12.0) {
        double y = x, num = 0.0, den = 1.0, r;
        int n = 0, i;
        const int small = y < 1.0;
        if (small)
            y += 1.0;
        else {
            n = (int)floor(y) - 1;
            y -= n;
        }
        for (i = 0; i < 8; ++i) {
            num = (num + P[i]) * (y - 1);
            den = den * (y - 1) + Q[i];
        }
        r = num / den + 1.0;
        if (small)
            r /= (y - 1.0);
        else
            for (i = 0; i < n; ++i)
                r *= y++;
        return r;
    }
    if (x > 171.624)
        return DBL_MAX * 2.0;
    {
        const double z = 1.0 / (x * x);
        double sum = B[7];
        int i;
        for (i = 6; i >= 0; --i) {
            sum *= z;
            sum += B[i];
        }
        return exp((x - 0.5) * log(x) - x + 0.91893853320467274178032973640562 + sum / x);
    }
}

/* Setup, src/Initialization.cpp:210-265, with the reference's Gamma. */
int dsmc_oracle_setup(const dsmc_params *p, dsmc_derived *d)
{
    if (p->wall_model == DSMC_WALL_CLL && !cll_valid(p->cll_normal, p->cll_tangential))
        return DSMC_ERR_BAD_CLL;
    if (p->nx < 1 || p->ny < 1 || !(p->x2 > p->x1) || !(p->y2 > p->y1) || !(p->dt > 0.0) ||
        p->sampling_period < 1)
        return DSMC_ERR_ARGUMENT;
    const double k = K_BOLTZMANN;
    d->molecule_mass = p->molar_mass / N_AVOGADRO;
    const double m = d->molecule_mass;
    d->p_free = p->n_free * (k * p->t_free);
    d->u_free = p->ma_free * sqrt((5.0 / 3.0) * k * p->t_free / m);
    d->ux_free = d->u_free * cos(PI_D * p->attack_angle / 180.0);
    d->uy_free = -d->u_free * sin(PI_D * p->attack_angle / 180.0);
    d->dx = (p->x2 - p->x1) / p->nx;
    d->dy = (p->y2 - p->y1) / p->ny;
    d->dv = d->dx * d->dy * p->dz;
    d->weight = d->dv * p->n_free / p->npc_free;
    d->sigma_ref = PI_D * p->d_ref * p->d_ref;
    d->omega = 2.0 * p->viscosity_index - 1.0;
    d->cr_ref = sqrt(4.0 * k * p->t_ref / m) / pow(gamma_fn(2.5 - p->viscosity_index), 1.0 / d->omega);
    const double q = 1.0 - d->omega;
    const double mean_rel = pow(4.0 * k * p->t_free / m, q / 2.0) * gamma_fn((q + 3.0) / 2.0) /
                            gamma_fn(1.5);
    const double rate_coeff = d->sigma_ref * pow(d->cr_ref, d->omega) * mean_rel;
    const double freq = p->n_free * rate_coeff;
    d->mft_free = 1.0 / freq;
    const double mean_speed = sqrt(8.0 * k * p->t_free / (PI_D * m));
    d->mfp_free = mean_speed * d->mft_free;
    d->kn_free = d->mfp_free / p->box_height;
    d->sc_max = 9.0 * d->sigma_ref * sqrt(k * p->t_free / m);
    return DSMC_OK;
}

/* ---- lifecycle and accessors -------------------------------------------- */

dsmc_oracle *dsmc_oracle_create(const dsmc_params *p, const dsmc_derived *d, int64_t capacity)
{
    dsmc_oracle *o = (dsmc_oracle *)calloc(1, sizeof(dsmc_oracle));
    if (!o)
        return NULL;
    o->p = *p;
    if (d)
        o->d = *d;
    else if (dsmc_oracle_setup(p, &o->d) != DSMC_OK) {
        free(o);
        return NULL;
    }
    if (capacity <= 0)
        capacity = (int64_t)(2.0 * p->npc_free * p->nx * p->ny) + 100000;
    o->cap = capacity;
    o->ncell = p->nx * p->ny;
    const size_t n = (size_t)capacity;
    double **arrays[10] = {&o->x, &o->y, &o->vx, &o->vy, &o->vz,
                           &o->sx, &o->sy, &o->svx, &o->svy, &o->svz};
    for (int i = 0; i < 10; ++i)
        *arrays[i] = (double *)malloc(sizeof(double) * n);
    o->cell_of = (int32_t *)malloc(sizeof(int32_t) * n);
    o->cell_start = (int32_t *)calloc((size_t)o->ncell + 1, sizeof(int32_t));
    o->fill = (int32_t *)malloc(sizeof(int32_t) * ((size_t)o->ncell + 1));
    o->acc = (double *)calloc(17 * (size_t)o->ncell, sizeof(double));
    o->box_lo[0] = p->box_x - p->box_width / 2.0;
    o->box_lo[1] = p->box_y - p->box_height / 2.0;
    o->box_hi[0] = p->box_x + p->box_width / 2.0;
    o->box_hi[1] = p->box_y + p->box_height / 2.0;
    /* One rank owns cells [0, NX) x [0, NY). */
    o->local[0] = p->x1 + 0 * o->d.dx;
    o->local[1] = p->y1 + 0 * o->d.dy;
    o->local[2] = p->x1 + p->nx * o->d.dx;
    o->local[3] = p->y1 + p->ny * o->d.dy;
    return o;
}

void dsmc_oracle_destroy(dsmc_oracle *o)
{
    if (!o)
        return;
    double *arrays[10] = {o->x, o->y, o->vx, o->vy, o->vz, o->sx, o->sy, o->svx, o->svy, o->svz};
    for (int i = 0; i < 10; ++i)
        free(arrays[i]);
    free(o->cell_of);
    free(o->cell_start);
    free(o->fill);
    free(o->acc);
    free(o);
}

int dsmc_oracle_get_counters(dsmc_oracle *o, dsmc_counters *c)
{
    c->np = o->np;
    c->step = o->step;
    c->sample_step = o->sample_step;
    c->collisions_last_step = o->last_nc;
    c->collisions_total = o->total_nc;
    c->drag_collision_count = o->drag_count;
    c->particle_steps = o->particle_steps;
    c->drag_impulse_total = o->drag_impulse;
    c->time = o->time;
    c->sample_time = o->sample_time;
    c->drag_sampling_time = o->drag_sampling_time;
    c->drag_collision_count_window = o->drag_count_window;
    c->drag_impulse_window = o->drag_impulse_window;
    return DSMC_OK;
}

int64_t dsmc_oracle_np(dsmc_oracle *o) { return o->np; }

int dsmc_oracle_get_particles(dsmc_oracle *o, double *x, double *y, double *vx, double *vy,
                              double *vz)
{
    const size_t n = sizeof(double) * (size_t)o->np;
    memcpy(x, o->x, n);
    memcpy(y, o->y, n);
    memcpy(vx, o->vx, n);
    memcpy(vy, o->vy, n);
    memcpy(vz, o->vz, n);
    return DSMC_OK;
}

int dsmc_oracle_set_particles_raw(dsmc_oracle *o, const double *x, const double *y,
                                  const double *vx, const double *vy, const double *vz, int64_t n)
{
    if (n < 0 || n > o->cap)
        return DSMC_ERR_CAPACITY;
    const size_t b = sizeof(double) * (size_t)n;
    memcpy(o->x, x, b);
    memcpy(o->y, y, b);
    memcpy(o->vx, vx, b);
    memcpy(o->vy, vy, b);
    memcpy(o->vz, vz, b);
    o->np = n;
    return DSMC_OK;
}

int dsmc_oracle_set_particles(dsmc_oracle *o, const double *x, const double *y, const double *vx,
                              const double *vy, const double *vz, int64_t n)
{
    const int s = dsmc_oracle_set_particles_raw(o, x, y, vx, vy, vz, n);
    return s != DSMC_OK ? s : dsmc_oracle_stage_index(o);
}

int dsmc_oracle_set_step(dsmc_oracle *o, int64_t step)
{
    o->step = step;
    return DSMC_OK;
}

int dsmc_oracle_get_cell_starts(dsmc_oracle *o, int32_t *out)
{
    memcpy(out, o->cell_start, sizeof(int32_t) * ((size_t)o->ncell + 1));
    return DSMC_OK;
}

int dsmc_oracle_get_fields(dsmc_oracle *o, double *out)
{
    memcpy(out, o->acc, sizeof(double) * 17 * (size_t)o->ncell);
    return DSMC_OK;
}

int dsmc_oracle_set_fields(dsmc_oracle *o, const double *in, int64_t sample_step)
{
    memcpy(o->acc, in, sizeof(double) * 17 * (size_t)o->ncell);
    o->sample_step = sample_step;
    return DSMC_OK;
}

int dsmc_oracle_intersect(dsmc_oracle *o, double x, double y, double dx, double dy, double *t,
                          double *nx, double *ny)
{
    return intersect_box(o, x, y, dx, dy, t, nx, ny);
}

int dsmc_oracle_inside_box(dsmc_oracle *o, double x, double y) { return inside_box(o, x, y); }

int dsmc_oracle_scatter(dsmc_oracle *o, double *v, double nx, double ny, uint32_t kind,
                        uint32_t step, uint32_t entity)
{
    select_stream(o, kind, step, entity);
    return wall_interaction(o, v, nx, ny);
}

/* ---- unit forms of single routines (parity of the ABI's unit kernels) -- */

/* GenerateNewParticles(X1, Y1, X2, Y2, Ngas, Ugasx, Ugasy, Tgas, MoveFlag),
 * src/Boundary.cpp:60-92, on stream (kind, step, entity); the particles are
 * appended to the oracle's (unsorted) array. */
int dsmc_oracle_generate(dsmc_oracle *o, const double *rect, double n_gas, double ux_gas,
                         double uy_gas, double t_gas, int move_flag, uint32_t kind, uint32_t step,
                         uint32_t entity)
{
    select_stream(o, kind, step, entity);
    return generate_gas(o, rect[0], rect[1], rect[2], rect[3], n_gas, ux_gas, uy_gas, t_gas,
                        move_flag);
}

/* BinaryCollisionsInCell(CellVolume, NPC, IPC), src/Collision.cpp:21-44, on
 * stream (kind, step, entity) over the oracle's particles ipc[0, n); returns
 * the number of collisions in *nc. */
int dsmc_oracle_collide_list(dsmc_oracle *o, double cell_volume, int n, const int32_t *ipc,
                             uint32_t kind, uint32_t step, uint32_t entity, int *nc)
{
    select_stream(o, kind, step, entity);
    *nc = collide_ids(o, 0, ipc, n, cell_volume);
    return DSMC_OK;
}

/* ElasticCollision(V1, V2, Cr), src/Collision.cpp:7-19, on stream
 * (kind, step, entity). */
int dsmc_oracle_elastic(dsmc_oracle *o, double *v1, double *v2, double cr, uint32_t kind,
                        uint32_t step, uint32_t entity)
{
    select_stream(o, kind, step, entity);
    elastic_v(o, v1, v2, cr);
    return DSMC_OK;
}
