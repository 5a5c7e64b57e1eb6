// C API over the reference solver's own routines, compiled from the reference
// sources (src/*.cpp, rng/*.cxx) with the single-rank MPI stub and the keyed
// Philox brng() of this directory.
//
// TEST INFRASTRUCTURE ONLY: it pins the CPU restatement in oracle/ and
// generates golden vectors.  It is never part of the product path.
//
// One time step follows the reference loop (src/Simulation.cpp:138-199) and
// calls the reference functions for every piece of physics.  The differences
// are the ones the engine's design fixes, applied identically here:
//   * each entity draws from its own Philox stream, so MoveParticles runs
//     once per particle with that particle's stream selected, and the
//     collision loop of CollideParticles (src/Collision.cpp:45-56) is
//     written out here so the stream can be selected per cell;
//   * the four inflow strips of BoundaryConditions (src/Boundary.cpp:100-173)
//     are generated by calling GenerateNewParticles with one stream per strip;
//     the reference BoundaryConditions is then called with NFree = 0, which
//     generates nothing and runs its own swap-with-last removal;
//   * after Indexing (src/Geometry.cpp:37-170) the particle array is reordered
//     into cell order, keeping the in-cell order of IPC, so the next step
//     starts from a cell-sorted array exactly as the engine's does.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "Boundary.h"
#include "Collision.h"
#include "Geometry.h"
#include "Initialization.h"
#include "MPIManager.h"
#include "RNG.h"
#include "Sampling.h"
#include "SimulationState.h"

#include "../../include/dsmc.h"
#include "../../include/dsmc_philox.h"

extern "C" void dsmc_ref_rng_select(std::uint32_t kind, std::uint32_t step, std::uint32_t entity);
extern "C" std::uint64_t dsmc_ref_rng_draws();
extern "C" void dsmc_ref_rng_set_seed64(std::uint64_t seed);
double frand_Gaussian(double E, double V); // src/Boundary.cpp:49, external linkage

namespace {
struct AbortCode {
    int code;
};
std::string g_results_dir = "results";
long long g_last_nc = 0;
long long g_total_nc = 0;
long long g_particle_steps = 0;
bool g_configured = false;

template <class F> int guarded(F &&f)
{
    try {
        f();
        return DSMC_OK;
    } catch (const AbortCode &a) {
        return a.code;
    } catch (const std::invalid_argument &) {
        return DSMC_ERR_BAD_CLL;
    } catch (...) {
        return DSMC_ERR_ARGUMENT;
    }
}

void sort_by_cell()
{
    // IPC holds, per cell, the particle indices in particle order.  Laying
    // the cells out k-major (the field layout k*NY + l) gives the engine's
    // cell-sorted array; Indexing() then rebuilds IPC for the new order.
    std::vector<PCL> sorted;
    sorted.reserve(NP);
    for (int k = 0; k < LocalNX; ++k)
        for (int l = 0; l < LocalNY; ++l)
            for (int i = 0; i < NPC[k][l]; ++i)
                sorted.push_back(P[IPC[k][l][i]]);
    for (int i = 0; i < NP; ++i)
        P[i] = sorted[i];
    Indexing();
}
} // namespace

[[noreturn]] void dsmc_ref_mpi_abort(int code) { throw AbortCode{code}; }

const char *dsmc_ref_results_dir() { return g_results_dir.c_str(); }

extern "C" {

int dsmc_ref_configure(const dsmc_params *p)
{
    return guarded([&] {
        if (p->nx < 1 || p->ny < 1 || p->nx > MAX_CELL_X || p->ny > MAX_CELL_Y)
            throw AbortCode{DSMC_ERR_ARGUMENT};
        X1 = p->x1;
        X2 = p->x2;
        Y1 = p->y1;
        Y2 = p->y2;
        DZ = p->dz;
        DL = p->dl;
        NX = p->nx;
        NY = p->ny;
        BoxX = p->box_x;
        BoxY = p->box_y;
        BoxWidth = p->box_width;
        BoxHeight = p->box_height;
        Dt = p->dt;
        NStep = p->n_step;
        FirstSamplingStep = p->first_sampling_step;
        SamplingPeriod = p->sampling_period;
        NPCFree = p->npc_free;
        MolarMass = p->molar_mass;
        MaFree = p->ma_free;
        NFree = p->n_free;
        TFree = p->t_free;
        AttackAngle = p->attack_angle;
        Tw = p->t_wall;
        DRef = p->d_ref;
        ViscosityIndex = p->viscosity_index;
        Tref = p->t_ref;
        WallInteraction = static_cast<WallModel>(p->wall_model);
        CLLNormalAccommodation = p->cll_normal;
        CLLTangentialAccommodation = p->cll_tangential;
        dsmc_ref_rng_set_seed64(p->seed);
        MPI_Comm_size(MPI_COMM_WORLD, &MPISize); // as RunSimulation does (Simulation.cpp:70-71)
        CreateMPICellType();
        CreateMPIParticleType();
        MPIRank = 1; // Setup() prints on rank 0 only; keep test output quiet
        Setup();
        SetupMPIDomain(); // resets MPIRank to 0 and fills the Local* globals
        DragImpulseTotal = 0.0;
        DragCollisionCount = 0;
        DragSamplingTime = 0.0;
        g_last_nc = g_total_nc = g_particle_steps = 0;
        g_configured = true;
    });
}

int dsmc_ref_get_derived(dsmc_derived *d)
{
    d->molecule_mass = MoleculeMass;
    d->p_free = PFree;
    d->u_free = UFree;
    d->ux_free = UxFree;
    d->uy_free = UyFree;
    d->dx = DX;
    d->dy = DY;
    d->dv = DV;
    d->weight = Weight;
    d->sigma_ref = SigmaRef;
    d->omega = Omega;
    d->cr_ref = CrRef;
    d->mft_free = MFTFree;
    d->mfp_free = MFPFree;
    d->kn_free = KnFree;
    d->sc_max = 9.0 * SigmaRef * std::sqrt(BOLTZMANN_CONSTANT * TFree / MoleculeMass);
    return DSMC_OK;
}

// Overrides derived constants (e.g. to align with another Setup()).
int dsmc_ref_set_derived(const dsmc_derived *d)
{
    MoleculeMass = d->molecule_mass;
    PFree = d->p_free;
    UFree = d->u_free;
    UxFree = d->ux_free;
    UyFree = d->uy_free;
    DX = d->dx;
    DY = d->dy;
    DV = d->dv;
    Weight = d->weight;
    SigmaRef = d->sigma_ref;
    Omega = d->omega;
    CrRef = d->cr_ref;
    MFTFree = d->mft_free;
    MFPFree = d->mfp_free;
    KnFree = d->kn_free;
    return DSMC_OK;
}

int dsmc_ref_init_cold()
{
    if (!g_configured)
        return DSMC_ERR_STATE;
    return guarded([] {
        dsmc_ref_rng_select(DSMC_RNG_INIT, 0, 0);
        InitialConditions();
        Indexing();
        sort_by_cell();
    });
}

int dsmc_ref_stage_move()
{
    return guarded([] {
        SamplingMode = (Step > FirstSamplingStep && Step % SamplingPeriod == 0) ? 1 : 0;
        const int n = NP;
        std::vector<PCL> saved(P, P + n);
        for (int i = 0; i < n; ++i) {
            dsmc_ref_rng_select(DSMC_RNG_MOVE, static_cast<std::uint32_t>(Step),
                                static_cast<std::uint32_t>(i));
            NP = 1;
            P[0] = saved[i];
            MoveParticles();
            saved[i] = P[0];
        }
        NP = n;
        for (int i = 0; i < n; ++i)
            P[i] = saved[i];
        if (Step > FirstSamplingStep)
            DragSamplingTime += Dt;
    });
}

int dsmc_ref_stage_boundary()
{
    return guarded([] {
        const std::uint32_t step = static_cast<std::uint32_t>(Step);
        // The four strips of BoundaryConditions, in its order.
        dsmc_ref_rng_select(DSMC_RNG_INJECT, step, 0);
        GenerateNewParticles(X1 - DL, LocalY1, X1, LocalY2, NFree, UxFree, UyFree, TFree, 1);
        dsmc_ref_rng_select(DSMC_RNG_INJECT, step, 1);
        GenerateNewParticles(X2, LocalY1, X2 + DL, LocalY2, NFree, UxFree, UyFree, TFree, 1);
        dsmc_ref_rng_select(DSMC_RNG_INJECT, step, 2);
        GenerateNewParticles(LocalX1, Y1 - DL, LocalX2, Y1, NFree, UxFree, UyFree, TFree, 1);
        dsmc_ref_rng_select(DSMC_RNG_INJECT, step, 3);
        GenerateNewParticles(LocalX1, Y2, LocalX2, Y2 + DL, NFree, UxFree, UyFree, TFree, 1);
        // The reference's own removal loop; with NFree = 0 its four
        // GenerateNewParticles calls add nothing.
        const double nfree = NFree;
        NFree = 0.0;
        dsmc_ref_rng_select(0, 0, 0);
        BoundaryConditions();
        NFree = nfree;
    });
}

int dsmc_ref_stage_index()
{
    return guarded([] {
        ExchangeParticles();
        Indexing();
        sort_by_cell();
    });
}

int dsmc_ref_stage_collide()
{
    return guarded([] {
        // CollideParticles (src/Collision.cpp:45-56), one stream per cell.
        long long nc = 0;
        for (int k = 0; k < LocalNX; ++k)
            for (int l = 0; l < LocalNY; ++l) {
                dsmc_ref_rng_select(DSMC_RNG_COLLIDE, static_cast<std::uint32_t>(Step),
                                    static_cast<std::uint32_t>(k * NY + l));
                const int ncc = BinaryCollisionsInCell(DV, NPC[k][l], IPC[k][l]);
                nc += ncc;
                if (SamplingMode == 1)
                    C[k][l].CountNC += ncc;
            }
        g_last_nc = nc;
        g_total_nc += nc;
    });
}

int dsmc_ref_stage_sample()
{
    return guarded([] {
        if (SamplingMode == 1)
            Sampling();
    });
}

int dsmc_ref_stage_end_step()
{
    g_particle_steps += NP;
    Step++;
    Time += Dt;
    return DSMC_OK;
}

int dsmc_ref_step()
{
    int s;
    if ((s = dsmc_ref_stage_move()) != 0) return s;
    if ((s = dsmc_ref_stage_boundary()) != 0) return s;
    if ((s = dsmc_ref_stage_index()) != 0) return s;
    if ((s = dsmc_ref_stage_collide()) != 0) return s;
    if ((s = dsmc_ref_stage_sample()) != 0) return s;
    return dsmc_ref_stage_end_step();
}

int dsmc_ref_get_counters(dsmc_counters *c)
{
    c->np = NP;
    c->step = Step;
    c->sample_step = SampleStep;
    c->collisions_last_step = g_last_nc;
    c->collisions_total = g_total_nc;
    c->drag_collision_count = DragCollisionCount;
    c->particle_steps = g_particle_steps;
    c->drag_impulse_total = DragImpulseTotal;
    c->time = Time;
    c->sample_time = SampleTime;
    c->drag_sampling_time = DragSamplingTime;
    // The reference keeps no per-window drag counters.
    c->drag_collision_count_window = -1;
    c->drag_impulse_window = -1.0;
    return DSMC_OK;
}

long long dsmc_ref_np() { return NP; }

int dsmc_ref_get_particles(double *x, double *y, double *vx, double *vy, double *vz)
{
    for (int i = 0; i < NP; ++i) {
        x[i] = P[i].X[0];
        y[i] = P[i].X[1];
        vx[i] = P[i].V[0];
        vy[i] = P[i].V[1];
        vz[i] = P[i].V[2];
    }
    return DSMC_OK;
}

// Replaces the particles and sorts them by cell (Indexing + reorder).
int dsmc_ref_set_particles(const double *x, const double *y, const double *vx, const double *vy,
                           const double *vz, long long n)
{
    if (n < 0 || n > MAX_PCL)
        return DSMC_ERR_CAPACITY;
    for (long long i = 0; i < n; ++i) {
        P[i].X[0] = x[i];
        P[i].X[1] = y[i];
        P[i].V[0] = vx[i];
        P[i].V[1] = vy[i];
        P[i].V[2] = vz[i];
    }
    NP = static_cast<int>(n);
    return guarded([] {
        Indexing();
        sort_by_cell();
    });
}

// Particles are stored without sorting (for stage-level tests).
int dsmc_ref_set_particles_raw(const double *x, const double *y, const double *vx,
                               const double *vy, const double *vz, long long n)
{
    if (n < 0 || n > MAX_PCL)
        return DSMC_ERR_CAPACITY;
    for (long long i = 0; i < n; ++i) {
        P[i].X[0] = x[i];
        P[i].X[1] = y[i];
        P[i].V[0] = vx[i];
        P[i].V[1] = vy[i];
        P[i].V[2] = vz[i];
    }
    NP = static_cast<int>(n);
    return DSMC_OK;
}

int dsmc_ref_set_step(long long step)
{
    Step = static_cast<int>(step);
    return DSMC_OK;
}

int dsmc_ref_get_npc(int *out)
{
    for (int k = 0; k < NX; ++k)
        for (int l = 0; l < NY; ++l)
            out[k * NY + l] = NPC[k][l];
    return DSMC_OK;
}

int dsmc_ref_get_fields(double *out)
{
    for (int k = 0; k < NX; ++k)
        for (int l = 0; l < NY; ++l)
            std::memcpy(out + 17 * (k * NY + l), &C[k][l], sizeof(CELL));
    return DSMC_OK;
}

int dsmc_ref_set_fields(const double *in, long long sample_step)
{
    for (int k = 0; k < NX; ++k)
        for (int l = 0; l < NY; ++l)
            std::memcpy(&C[k][l], in + 17 * (k * NY + l), sizeof(CELL));
    SampleStep = static_cast<int>(sample_step);
    return DSMC_OK;
}

// Printing() of the gathered field into <dir>/<wall>/.
int dsmc_ref_write_field(const char *dir)
{
    return guarded([&] {
        g_results_dir = dir;
        const std::vector<CELL> field = GatherGlobalField();
        Printing(field);
    });
}

int dsmc_ref_intersect(double x, double y, double dx, double dy, double *t, double *nx, double *ny)
{
    return IntersectBox(x, y, dx, dy, *t, *nx, *ny) ? 1 : 0;
}

int dsmc_ref_inside_box(double x, double y) { return InsideBox(x, y) ? 1 : 0; }

// One wall interaction with the configured wall model and the given stream.
int dsmc_ref_scatter(double *v, double nx, double ny, std::uint32_t kind, std::uint32_t step,
                     std::uint32_t entity)
{
    return guarded([&] {
        dsmc_ref_rng_select(kind, step, entity);
        switch (WallInteraction) {
        case WallModel::Specular: SpecularScattering(v, nx, ny); break;
        case WallModel::Diffuse: DiffuseScattering(v, MoleculeMass, Tw, nx, ny); break;
        case WallModel::CLL:
            CLLScattering(v, MoleculeMass, Tw, nx, ny, CLLNormalAccommodation,
                          CLLTangentialAccommodation);
            break;
        }
    });
}

// CLLScattering with explicit arguments (the reference test's entry).
int dsmc_ref_cll(double *v, double m, double tw, double nx, double ny, double an, double at)
{
    return guarded([&] { CLLScattering(v, m, tw, nx, ny, an, at); });
}

int dsmc_ref_select_stream(std::uint32_t kind, std::uint32_t step, std::uint32_t entity)
{
    dsmc_ref_rng_select(kind, step, entity);
    return DSMC_OK;
}

unsigned long long dsmc_ref_draws() { return dsmc_ref_rng_draws(); }

double dsmc_ref_brng() { return brng(); }

// The reference's 2-draw Gaussian (src/Boundary.cpp:49-50), to pin the order
// in which g++ evaluates its two brng() calls.
double dsmc_ref_gaussian(double e, double v) { return frand_Gaussian(e, v); }

int dsmc_ref_poisson(double e) { return irand_Poisson(e); }

// The reference's GenerateNewParticles (src/Boundary.cpp:60-92) on stream
// (kind, step, entity): appends to P, NP grows.
int dsmc_ref_generate(const double *rect, double n_gas, double ux, double uy, double t_gas,
                      int move_flag, std::uint32_t kind, std::uint32_t step, std::uint32_t entity)
{
    return guarded([&] {
        dsmc_ref_rng_select(kind, step, entity);
        GenerateNewParticles(rect[0], rect[1], rect[2], rect[3], n_gas, ux, uy, t_gas, move_flag);
    });
}

// The reference's BinaryCollisionsInCell (src/Collision.cpp:21-44) over P on
// stream (kind, step, entity); the list is copied since the routine takes it
// as int *.
int dsmc_ref_collide_list(double cell_volume, int n, const int *ipc, std::uint32_t kind,
                          std::uint32_t step, std::uint32_t entity, int *nc)
{
    return guarded([&] {
        dsmc_ref_rng_select(kind, step, entity);
        std::vector<int> ids(ipc, ipc + n);
        *nc = BinaryCollisionsInCell(cell_volume, n, ids.data());
    });
}

// The reference's ElasticCollision (src/Collision.cpp:7-19).
int dsmc_ref_elastic(double *v1, double *v2, double cr, std::uint32_t kind, std::uint32_t step,
                     std::uint32_t entity)
{
    return guarded([&] {
        dsmc_ref_rng_select(kind, step, entity);
        ElasticCollision(v1, v2, cr);
    });
}

// The reference's RemoveParticlesInsideBox (src/Geometry.cpp:231-247) on P as
// it stands (no sort).
int dsmc_ref_remove_inside_box()
{
    return guarded([] { RemoveParticlesInsideBox(); });
}

} // extern "C"
