// surface.cpp - the reference solver's C++ functions and globals
// (include/dsmc_reference_api.h) on top of the C ABI.  Nothing here computes
// physics: every stage and every wall interaction runs on the GPU.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/dsmc.h"
#include "../../include/dsmc_philox.h"
#include "../../include/dsmc_reference_api.h"

// ---- globals with the reference's defaults ---------------------------------
// src/Boundary.cpp:11-13
WallModel WallInteraction = WallModel::CLL;
double CLLNormalAccommodation = 0.8;
double CLLTangentialAccommodation = 0.8;
// src/Geometry.cpp:11-28
double X1 = -20.0, X2 = 20.0, Y1 = -20.0, Y2 = 20.0, DZ = 0.1;
int NX = 100, NY = 100;
double DL = 0.1;
double BoxX = 0.0, BoxY = 0.0, BoxWidth = 4.0, BoxHeight = 4.0;
double DX, DY, DV;
// src/Initialization.cpp:11-37
double Dt = 1.0e-05;
int NStep = 100000;
int FirstSamplingStep = 10000;
int SamplingPeriod = 1;
int PrintPeriod = 10000;
double NPCFree = 10;
double MolarMass = 0.040;
double MaFree = 4;
double NFree = 1e17;
double TFree = 200;
double AttackAngle = 0;
double Tw = 300.0;
double Omega, SigmaRef, CrRef, MFTFree, MFPFree, KnFree;
double DRef = 4.17e-10;
double ViscosityIndex = 0.81;
double Tref = 273.0;
long long DragCollisionCount = 0;
double DragImpulseTotal = 0.0;
double DragSamplingTime = 0.0;
int SampleStep = 0;
int NP = 0;
double Weight, MoleculeMass, PFree, UFree, UxFree, UyFree;
double SampleTime = 0.0;
int Step = 0;
double Time = 0.0;
int SamplingMode = 0;

namespace dsmc {
int Precision = DSMC_FP64;
std::string ResultsDirectory = "results";
} // namespace dsmc

namespace {
dsmc_ctx *g_ctx = nullptr;
dsmc_params g_params{};
dsmc_derived g_derived{};
uint64_t g_seed = 0x5EED;
dsmc_stream g_user;
uint32_t g_user_calls = 0;
bool g_step_open = false;

void fail(int code, const char *what)
{
    throw dsmc::Error(code, std::string(what) + ": " + dsmc_status_string(code));
}

void check(int code, const char *what)
{
    if (code != DSMC_OK)
        fail(code, what);
}

dsmc_params params_from_globals()
{
    dsmc_params p;
    dsmc_default_params(&p);
    p.x1 = X1;
    p.x2 = X2;
    p.y1 = Y1;
    p.y2 = Y2;
    p.dz = DZ;
    p.dl = DL;
    p.nx = NX;
    p.ny = NY;
    p.box_x = BoxX;
    p.box_y = BoxY;
    p.box_width = BoxWidth;
    p.box_height = BoxHeight;
    p.dt = Dt;
    p.n_step = NStep;
    p.first_sampling_step = FirstSamplingStep;
    p.sampling_period = SamplingPeriod;
    p.wall_model = static_cast<int32_t>(WallInteraction);
    p.npc_free = NPCFree;
    p.molar_mass = MolarMass;
    p.ma_free = MaFree;
    p.n_free = NFree;
    p.t_free = TFree;
    p.attack_angle = AttackAngle;
    p.t_wall = Tw;
    p.d_ref = DRef;
    p.viscosity_index = ViscosityIndex;
    p.t_ref = Tref;
    p.cll_normal = CLLNormalAccommodation;
    p.cll_tangential = CLLTangentialAccommodation;
    p.seed = g_seed;
    p.precision = dsmc::Precision;
    return p;
}

void pull_counters()
{
    if (g_ctx == nullptr)
        return;
    dsmc_counters c;
    check(dsmc_get_counters(g_ctx, 0, &c), "dsmc_get_counters");
    NP = static_cast<int>(c.np);
    Step = static_cast<int>(c.step);
    SampleStep = static_cast<int>(c.sample_step);
    DragCollisionCount = c.drag_collision_count;
    DragImpulseTotal = c.drag_impulse_total;
    DragSamplingTime = c.drag_sampling_time;
    Time = c.time;
    SampleTime = c.sample_time;
}

dsmc_ctx *ctx()
{
    if (g_ctx == nullptr)
        fail(DSMC_ERR_STATE, "Setup() has not been called");
    return g_ctx;
}

// The engine advances Step when a step's stages are complete; the
// reference's caller does Step++ itself after Sampling().  A step left open
// is closed before the next MoveParticles() or a field read.
void close_open_step()
{
    if (g_step_open) {
        check(dsmc_stage_end_step(ctx()), "end of step");
        g_step_open = false;
    }
}

// One-element device buffers for the scalar entry points.
struct Scratch {
    double *d = nullptr; // 8 doubles
    int32_t *i = nullptr;
    uint32_t *u = nullptr;
    Scratch()
    {
        if (cudaMalloc(&d, 8 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&i, 4 * sizeof(int32_t)) != cudaSuccess ||
            cudaMalloc(&u, 4 * sizeof(uint32_t)) != cudaSuccess)
            fail(DSMC_ERR_CUDA, "device scratch");
    }
};

Scratch &scratch()
{
    static Scratch s;
    return s;
}
} // namespace

dsmc_ctx *dsmc::Context() { return g_ctx; }
const dsmc_params &dsmc::Parameters() { return g_params; }

// WallModelName, src/Boundary.cpp:15-24
const char *WallModelName()
{
    const char *n = dsmc_wall_model_name(static_cast<int>(WallInteraction));
    if (n == nullptr)
        throw std::invalid_argument("Unknown wall model");
    return n;
}

// SetupGeometry, src/Geometry.cpp:30-35
void SetupGeometry()
{
    DX = (X2 - X1) / NX;
    DY = (Y2 - Y1) / NY;
    DV = DX * DY * DZ;
}

// Setup, src/Initialization.cpp:210-288: derived constants, the printed
// freestream summary, and a device context for the case.
void Setup()
{
    g_params = params_from_globals();
    const int s = dsmc_setup(&g_params, &g_derived);
    if (s == DSMC_ERR_BAD_CLL)
        std::cerr << "ERROR: CLL accommodation coefficients must be in [0, 1]\n";
    check(s, "Setup");
    MoleculeMass = g_derived.molecule_mass;
    PFree = g_derived.p_free;
    UFree = g_derived.u_free;
    UxFree = g_derived.ux_free;
    UyFree = g_derived.uy_free;
    SetupGeometry();
    Weight = g_derived.weight;
    SigmaRef = g_derived.sigma_ref;
    Omega = g_derived.omega;
    CrRef = g_derived.cr_ref;
    MFTFree = g_derived.mft_free;
    MFPFree = g_derived.mfp_free;
    KnFree = g_derived.kn_free;
    std::cout << "\nFreestream properties\n-----------------------------\n"
              << "Box size    = " << BoxWidth << " x " << BoxHeight << " m\n"
              << "Wall model  = " << WallModelName() << '\n';
    if (WallInteraction == WallModel::CLL)
        std::cout << "CLL normal  = " << CLLNormalAccommodation << '\n'
                  << "CLL tangent = " << CLLTangentialAccommodation << '\n';
    std::cout << "Angle       = " << AttackAngle << " degrees\n"
              << "P_inf       = " << PFree << " Pa\n"
              << "U_inf       = " << UFree << " m/s\n"
              << "MFT_inf     = " << MFTFree << " s\n"
              << "MFP_inf     = " << MFPFree << " m\n"
              << "Kn_inf      = " << KnFree << "\n"
              << "DX / lambda = " << DX / MFPFree << "\n"
              << "DY / lambda = " << DY / MFPFree << "\n"
              << "Dt / MFT    = " << Dt / MFTFree << "\n";
    if (g_ctx != nullptr) {
        dsmc_ctx_destroy(g_ctx);
        g_ctx = nullptr;
    }
    g_step_open = false;
    check(dsmc_ctx_create(&g_params, &g_derived, 1, nullptr, &g_ctx), "dsmc_ctx_create");
}

// InitialConditions, src/Initialization.cpp:290-313
void InitialConditions()
{
    check(dsmc_init_cold(ctx()), "InitialConditions");
    g_step_open = false;
    pull_counters();
}

// MoveParticles, src/Boundary.cpp:284-328 (also starts a step)
void MoveParticles()
{
    close_open_step();
    SamplingMode = (Step > FirstSamplingStep && Step % SamplingPeriod == 0) ? 1 : 0;
    check(dsmc_stage_move(ctx()), "MoveParticles");
    g_step_open = true;
    pull_counters();
}

// BoundaryConditions, src/Boundary.cpp:94-203
void BoundaryConditions()
{
    check(dsmc_stage_boundary(ctx()), "BoundaryConditions");
    pull_counters();
}

// Indexing, src/Geometry.cpp:37-170
void Indexing()
{
    check(dsmc_stage_index(ctx()), "Indexing");
    const int s = dsmc_synchronize(ctx());
    if (s != DSMC_OK)
        fail(s, "Indexing");
}

// CollideParticles, src/Collision.cpp:45-56
int CollideParticles()
{
    check(dsmc_stage_collide(ctx()), "CollideParticles");
    dsmc_counters c;
    check(dsmc_get_counters(ctx(), 0, &c), "dsmc_get_counters");
    return static_cast<int>(c.collisions_last_step);
}

// Sampling, src/Sampling.cpp:14-31
void Sampling()
{
    check(dsmc_stage_sample(ctx()), "Sampling");
    SampleStep++;
    SampleTime += Dt;
}

// ExchangeParticles, src/MPIManager.cpp:592-824: with one device owning every
// cell no particle changes owner; the out-of-domain check it performs is made
// by the device sort (status 30).
void ExchangeParticles() { ctx(); }

// GatherGlobalField, src/MPIManager.cpp:305-499 (one process holds it all)
std::vector<CELL> GatherGlobalField()
{
    close_open_step();
    std::vector<CELL> field(static_cast<size_t>(NX) * NY);
    check(dsmc_get_fields(ctx(), 0, field.data()), "GatherGlobalField");
    pull_counters();
    return field;
}

// Printing, src/Sampling.cpp:36-268
void Printing(const std::vector<CELL> &GlobalField)
{
    if (GlobalField.size() != static_cast<size_t>(NX) * NY) {
        std::cerr << "ERROR: GlobalField has wrong size\nExpected = " << NX * NY
                  << "\nReceived = " << GlobalField.size() << '\n';
        return;
    }
    dsmc_params p = g_params;
    p.n_step = NStep;
    const int s = dsmc_write_field(&p, &g_derived, SampleStep, GlobalField.data(),
                                   dsmc::ResultsDirectory.c_str());
    if (s != DSMC_OK) {
        std::cerr << "ERROR: Could not write the field to " << dsmc::ResultsDirectory << '\n';
        return;
    }
    std::cout << "Global field written to " << dsmc::ResultsDirectory << '/' << WallModelName()
              << "/DSMC2D_Field.plt\n";
}

// InsideBox, src/Geometry.cpp:173-177 (on the device)
bool InsideBox(double x, double y)
{
    dsmc_params p = params_from_globals();
    Scratch &s = scratch();
    const double in[2] = {x, y};
    if (cudaMemcpy(s.d, in, sizeof in, cudaMemcpyHostToDevice) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "InsideBox");
    check(dsmc_k_inside_box(&p, 1, s.d, s.d + 1, s.i, nullptr), "InsideBox");
    int32_t r = 0;
    if (cudaMemcpy(&r, s.i, sizeof r, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "InsideBox");
    return r != 0;
}

// IntersectBox, src/Geometry.cpp:179-229 (on the device)
bool IntersectBox(double x, double y, double dx, double dy, double &tHit, double &normalX,
                  double &normalY)
{
    dsmc_params p = params_from_globals();
    Scratch &s = scratch();
    const double in[4] = {x, y, dx, dy};
    if (cudaMemcpy(s.d, in, sizeof in, cudaMemcpyHostToDevice) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "IntersectBox");
    check(dsmc_k_intersect(&p, 1, s.d, s.d + 1, s.d + 2, s.d + 3, s.i, s.d + 4, s.d + 5, s.d + 6,
                           nullptr),
          "IntersectBox");
    double out[3];
    int32_t hit = 0;
    if (cudaMemcpy(out, s.d + 4, sizeof out, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&hit, s.i, sizeof hit, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "IntersectBox");
    if (!hit)
        return false;
    tHit = out[0];
    normalX = out[1];
    normalY = out[2];
    return true;
}

namespace {
// One wall interaction on the device, drawing from the user stream.
void scatter_one(double *v, double m, double tw, double nx, double ny, int model, double an,
                 double at)
{
    dsmc_params p = params_from_globals();
    p.wall_model = model;
    p.t_wall = tw;
    p.cll_normal = an;
    p.cll_tangential = at;
    dsmc_derived d;
    check(dsmc_setup(&p, &d), "wall interaction");
    d.molecule_mass = m;
    Scratch &s = scratch();
    const double in[5] = {v[0], v[1], v[2], nx, ny};
    const uint32_t entity = 0;
    if (cudaMemcpy(s.d, in, sizeof in, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s.u, &entity, sizeof entity, cudaMemcpyHostToDevice) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "wall interaction");
    check(dsmc_k_scatter(&p, &d, 1, s.d, s.d + 3, s.d + 4, DSMC_RNG_USER, g_user_calls++, s.u,
                         nullptr),
          "wall interaction");
    if (cudaMemcpy(v, s.d, 3 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "wall interaction");
}
} // namespace

// SpecularScattering, src/Boundary.cpp:235-241
void SpecularScattering(double *v, double Nx, double Ny)
{
    scatter_one(v, MoleculeMass > 0 ? MoleculeMass : MolarMass / 6.022045E+23, Tw, Nx, Ny,
                DSMC_WALL_SPECULAR, 0.0, 0.0);
}

// DiffuseScattering, src/Boundary.cpp:205-233
void DiffuseScattering(double *v, double m, double tw, double Nx, double Ny)
{
    scatter_one(v, m, tw, Nx, Ny, DSMC_WALL_DIFFUSE, 0.0, 0.0);
}

// CLLScattering, src/Boundary.cpp:243-282
void CLLScattering(double *v, double m, double wallTemperature, double Nx, double Ny,
                   double normalAccommodation, double tangentialAccommodation)
{
    if (!std::isfinite(normalAccommodation) || normalAccommodation < 0.0 ||
        normalAccommodation > 1.0 || !std::isfinite(tangentialAccommodation) ||
        tangentialAccommodation < 0.0 || tangentialAccommodation > 1.0)
        throw std::invalid_argument("CLL accommodation coefficients must be in [0, 1]");
    scatter_one(v, m, wallTemperature, Nx, Ny, DSMC_WALL_CLL, normalAccommodation,
                tangentialAccommodation);
}

// rng/BRNG.cxx:17-21: the seed becomes the Philox key of the next Setup().
void SetSeed(unsigned int u, unsigned int v)
{
    g_seed = static_cast<uint64_t>(u) | (static_cast<uint64_t>(v) << 32);
    dsmc_stream_init(&g_user, g_seed, DSMC_RNG_USER, 0xFFFFFFFFu, 0);
    g_user_calls = 0;
}

// rng/BRNG.cxx:30-34: the next uniform of the host-side user stream.
double brng()
{
    static bool ready = false;
    if (!ready) {
        dsmc_stream_init(&g_user, g_seed, DSMC_RNG_USER, 0xFFFFFFFFu, 0);
        ready = true;
    }
    return dsmc_stream_uniform(&g_user);
}

// ---- single routines of the reference headers -----------------------------------
namespace {
// The population edits need the step's sort done: between steps they run
// at once; after Indexing the open step is ended first; between
// MoveParticles and Indexing the particles are mid-step and the call fails.
void settle_population(const char *what)
{
    dsmc_ctx *c = ctx();
    (void)c;
    if (g_step_open) {
        const int s = dsmc_stage_end_step(g_ctx);
        if (s == DSMC_ERR_STATE)
            fail(s, (std::string(what) + " between MoveParticles() and Indexing()").c_str());
        check(s, what);
        g_step_open = false;
    }
}

// Device buffers of the generated particles, grown as needed.
struct InjectBuffers {
    double *d = nullptr;
    int64_t cap = 0;
    void reserve(int64_t n)
    {
        if (n <= cap)
            return;
        if (d != nullptr)
            cudaFree(d);
        d = nullptr;
        cap = 0;
        if (cudaMalloc(&d, sizeof(double) * 5 * static_cast<size_t>(n)) != cudaSuccess)
            fail(DSMC_ERR_CUDA, "GenerateNewParticles buffers");
        cap = n;
    }
};
} // namespace

// GenerateNewParticles, src/Boundary.cpp:60-92: the particles are drawn on
// the device from the user stream, then join the population (those outside
// the domain are dropped as BoundaryConditions would drop them) and are
// sorted by cell as the next Indexing orders them.
void GenerateNewParticles(double x1, double y1, double x2, double y2, double Ngas,
                          double Ugasx, double Ugasy, double Tgas, int MoveFlag)
{
    settle_population("GenerateNewParticles");
    static InjectBuffers buf;
    const double rect[4] = {x1, y1, x2, y2};
    const uint32_t step = g_user_calls++;
    const double navg = Ngas * ((x2 - x1) * (y2 - y1) * DZ) / Weight;
    buf.reserve(std::max<int64_t>(64, static_cast<int64_t>(navg + 10.0 * std::sqrt(navg)) + 64));
    int64_t n = 0;
    for (int attempt = 0;; ++attempt) {
        const int64_t cap = buf.cap;
        double *d = buf.d;
        const int s = dsmc_k_inject(&g_params, &g_derived, rect, Ngas, Ugasx, Ugasy, Tgas,
                                    MoveFlag, DSMC_RNG_USER, step, 0, cap, d, d + cap,
                                    d + 2 * cap, d + 3 * cap, d + 4 * cap, &n, nullptr);
        if (s == DSMC_ERR_CAPACITY && attempt == 0) { // the same draws again, more room
            buf.reserve(n);
            continue;
        }
        check(s, "GenerateNewParticles");
        break;
    }
    const int64_t cap = buf.cap;
    check(dsmc_append_particles_device(ctx(), 0, buf.d, buf.d + cap, buf.d + 2 * cap,
                                       buf.d + 3 * cap, buf.d + 4 * cap, n),
          "GenerateNewParticles");
    pull_counters();
}

// RemoveParticlesInsideBox, src/Geometry.cpp:231-247
void RemoveParticlesInsideBox()
{
    settle_population("RemoveParticlesInsideBox");
    check(dsmc_remove_inside_box(ctx(), 0), "RemoveParticlesInsideBox");
    pull_counters();
}

// ElasticCollision, src/Collision.cpp:7-19 (on the device, user stream)
void ElasticCollision(double *V1, double *V2, double Cr)
{
    dsmc_params p = params_from_globals();
    Scratch &s = scratch();
    const double in[7] = {V1[0], V1[1], V1[2], V2[0], V2[1], V2[2], Cr};
    if (cudaMemcpy(s.d, in, sizeof in, cudaMemcpyHostToDevice) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "ElasticCollision");
    check(dsmc_k_elastic(&p, 1, s.d, s.d + 3, s.d + 6, DSMC_RNG_USER, g_user_calls++, nullptr,
                         nullptr),
          "ElasticCollision");
    double out[6];
    if (cudaMemcpy(out, s.d, sizeof out, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(DSMC_ERR_CUDA, "ElasticCollision");
    std::copy(out, out + 3, V1);
    std::copy(out + 3, out + 6, V2);
}

// BinaryCollisionsInCell, src/Collision.cpp:21-44: IPC holds slot indices of
// the current cell-sorted population (slot i is the i-th particle of
// dsmc_download_particles); the pairs are drawn from the user stream.
int BinaryCollisionsInCell(double CellVolume, int NPC, int *IPC)
{
    if (NPC < 2)
        return 0;
    int32_t nc = 0;
    check(dsmc_collide_list(ctx(), 0, CellVolume, NPC, IPC, DSMC_RNG_USER, g_user_calls++, 0,
                            &nc),
          "BinaryCollisionsInCell");
    return nc;
}

// ---- RunSimulation, src/Simulation.cpp:18-247 --------------------------------
namespace {
enum class ArgumentResult { Run, Help, Error };

bool parse_number(const char *s, double &out)
{
    char *end = nullptr;
    errno = 0;
    out = std::strtod(s, &end);
    return !(end == s || *end != '\0' || errno == ERANGE || !std::isfinite(out));
}

// The reference's flags (--angle-of-attack/--aoa, -h/--help, exit codes 0/2)
// plus run-time settings it fixes at compile time; defaults are its values.
// Run controls beyond the reference's flags.
struct RunControls {
    int print_period = 0;      // intermediate fields (the reference's commented PrintPeriod)
    int checkpoint_period = 0; // checkpoints during the run
    std::string checkpoint;    // checkpoint file
    std::string restart;       // resume from this checkpoint
    bool drag = false;         // print the drag block at the end
};
RunControls g_run;

ArgumentResult ParseArguments(int argc, char **argv)
{
    for (int i = 1; i < argc; ++i) {
        const std::string option = argv[i];
        if (option == "--help" || option == "-h") {
            std::cout
                << "Usage: dsmc [--angle-of-attack DEGREES] [options]\n"
                << "  --angle-of-attack, --aoa  Flow angle in [-180, 180] degrees\n"
                << "  Positive angles tilt the flow toward negative y.\n"
                << "  The box remains aligned with the x/y axes.\n"
                << "  --wall specular|diffuse|cll   wall interaction (default cll)\n"
                << "  --acc-n A, --acc-t A          CLL accommodation coefficients\n"
                << "  --nx N, --ny N, --npc N       grid and particles per cell\n"
                << "  --dt S, --steps N, --first-sampling-step N\n"
                << "  --box-width W, --box-height H, --mach M, --density N\n"
                << "  --seed N, --precision fp64|fp32, --results DIR\n"
                << "  --print-period N      also write the field every N steps after\n"
                << "                        FirstSamplingStep, into DIR/step_<Step>\n"
                << "  --checkpoint FILE     write a checkpoint at the end (and every\n"
                << "  --checkpoint-period N   N steps)\n"
                << "  --restart FILE        resume from a checkpoint instead of\n"
                << "                        InitialConditions\n"
                << "  --drag                print the drag block (mean force, Cd)\n";
            return ArgumentResult::Help;
        }
        const bool known =
            option == "--angle-of-attack" || option == "--aoa" || option == "--wall" ||
            option == "--acc-n" || option == "--acc-t" || option == "--nx" || option == "--ny" ||
            option == "--npc" || option == "--dt" || option == "--steps" ||
            option == "--first-sampling-step" || option == "--seed" || option == "--precision" ||
            option == "--results" || option == "--box-width" || option == "--box-height" ||
            option == "--mach" || option == "--density" || option == "--print-period" ||
            option == "--checkpoint" || option == "--checkpoint-period" || option == "--restart";
        if (option == "--drag") {
            g_run.drag = true;
            continue;
        }
        if (!known) {
            std::cerr << "Unknown option: " << option << ". Use --help.\n";
            return ArgumentResult::Error;
        }
        if (++i == argc) {
            // The angle flags keep the reference's message (Simulation.cpp:44).
            if (option == "--angle-of-attack" || option == "--aoa")
                std::cerr << option << " requires an angle in degrees.\n";
            else
                std::cerr << option << " requires a value.\n";
            return ArgumentResult::Error;
        }
        const std::string value = argv[i];
        double x = 0.0;
        if (option == "--angle-of-attack" || option == "--aoa") {
            if (!parse_number(argv[i], x) || x < -180.0 || x > 180.0) {
                std::cerr << "Invalid angle: " << value
                          << ". Expected a finite number in [-180, 180].\n";
                return ArgumentResult::Error;
            }
            AttackAngle = x;
        } else if (option == "--wall") {
            if (value == "specular")
                WallInteraction = WallModel::Specular;
            else if (value == "diffuse")
                WallInteraction = WallModel::Diffuse;
            else if (value == "cll")
                WallInteraction = WallModel::CLL;
            else {
                std::cerr << "Invalid wall model: " << value << '\n';
                return ArgumentResult::Error;
            }
        } else if (option == "--precision") {
            if (value == "fp64")
                dsmc::Precision = DSMC_FP64;
            else if (value == "fp32")
                dsmc::Precision = DSMC_FP32;
            else {
                std::cerr << "Invalid precision: " << value << '\n';
                return ArgumentResult::Error;
            }
        } else if (option == "--results") {
            dsmc::ResultsDirectory = value;
        } else if (option == "--checkpoint") {
            g_run.checkpoint = value;
        } else if (option == "--restart") {
            g_run.restart = value;
        } else {
            if (!parse_number(argv[i], x)) {
                std::cerr << "Invalid value for " << option << ": " << value << '\n';
                return ArgumentResult::Error;
            }
            if (option == "--acc-n") CLLNormalAccommodation = x;
            else if (option == "--acc-t") CLLTangentialAccommodation = x;
            else if (option == "--nx") NX = static_cast<int>(x);
            else if (option == "--ny") NY = static_cast<int>(x);
            else if (option == "--npc") NPCFree = x;
            else if (option == "--dt") Dt = x;
            else if (option == "--steps") NStep = static_cast<int>(x);
            else if (option == "--first-sampling-step") FirstSamplingStep = static_cast<int>(x);
            else if (option == "--seed") {
                const uint64_t s = static_cast<uint64_t>(x);
                SetSeed(static_cast<unsigned>(s), static_cast<unsigned>(s >> 32));
            } else if (option == "--box-width") BoxWidth = x;
            else if (option == "--box-height") BoxHeight = x;
            else if (option == "--mach") MaFree = x;
            else if (option == "--density") NFree = x;
            else if (option == "--print-period" || option == "--checkpoint-period") {
                if (x < 1.0 || x != std::floor(x)) {
                    std::cerr << "Invalid value for " << option << ": " << value << '\n';
                    return ArgumentResult::Error;
                }
                (option == "--print-period" ? g_run.print_period : g_run.checkpoint_period) =
                    static_cast<int>(x);
            }
        }
    }
    return ArgumentResult::Run;
}
} // namespace

int RunSimulation(int argc, char **argv)
{
    const ArgumentResult arguments = ParseArguments(argc, argv);
    if (arguments != ArgumentResult::Run)
        return arguments == ArgumentResult::Help ? 0 : 2;
    try {
        Setup();
        std::cout << "Setup\n";
        if (!g_run.restart.empty()) {
            check(dsmc_checkpoint_load(ctx(), g_run.restart.c_str()), "restart");
            pull_counters();
            std::cout << "Restarted from " << g_run.restart << " at step " << Step << '\n';
        } else {
            InitialConditions();
            std::cout << "Total particles across all ranks = " << NP << "\nInitialConditions\n";
        }
        const std::string results = dsmc::ResultsDirectory;
        // The loop of src/Simulation.cpp:138-199 as CUDA graphs, with the
        // reference's progress line every 100 steps.
        while (Step < NStep) {
            int chunk = std::min(100 - Step % 100, NStep - Step);
            for (int period : {g_run.print_period, g_run.checkpoint_period})
                if (period > 0)
                    chunk = std::min(chunk, period - Step % period);
            check(dsmc_step(ctx(), chunk), "time step");
            const int s = dsmc_synchronize(ctx());
            if (s != DSMC_OK)
                fail(s, "time step");
            pull_counters();
            if (Step % 100 == 0) {
                dsmc_counters c;
                check(dsmc_get_counters(ctx(), 0, &c), "dsmc_get_counters");
                std::cout << "Time step " << Step << ", Number of particles " << NP
                          << ", Number of collisions " << c.collisions_last_step << '\n';
            }
            // The reference's commented-out intermediate output
            // (Simulation.cpp:198), one directory per output step.
            if (g_run.print_period > 0 && Step > FirstSamplingStep &&
                Step % g_run.print_period == 0 && Step < NStep) {
                dsmc::ResultsDirectory = results + "/step_" + std::to_string(Step);
                Printing(GatherGlobalField());
                dsmc::ResultsDirectory = results;
            }
            if (g_run.checkpoint_period > 0 && !g_run.checkpoint.empty() &&
                Step % g_run.checkpoint_period == 0 && Step < NStep)
                check(dsmc_checkpoint_save(ctx(), g_run.checkpoint.c_str()), "checkpoint");
        }
        Printing(GatherGlobalField());
        if (!g_run.checkpoint.empty())
            check(dsmc_checkpoint_save(ctx(), g_run.checkpoint.c_str()), "checkpoint");
        if (g_run.drag) {
            // Simulation.cpp:210-237 (commented out in the reference).
            dsmc_counters c;
            dsmc_drag dr;
            check(dsmc_get_counters(ctx(), 0, &c), "dsmc_get_counters");
            if (dsmc_drag_report(&g_params, &g_derived, &c, &dr) == DSMC_OK) {
                std::cout << "\n====================================\n"
                          << "Box collisions = " << dr.box_collisions_window << "\n"
                          << "Sampling time = " << dr.sampling_time << " s\n"
                          << "Mean drag force = " << dr.mean_force << " N\n"
                          << "Drag coefficient Cd = " << dr.cd << "\n"
                          << "====================================\n";
            } else {
                std::cout << "No drag sampling time yet (Step <= FirstSamplingStep)\n";
            }
        }
    } catch (const dsmc::Error &e) {
        std::cerr << "ERROR: " << e.what() << '\n';
        return e.code();
    }
    if (g_ctx != nullptr) {
        dsmc_ctx_destroy(g_ctx);
        g_ctx = nullptr;
    }
    return 0;
}
