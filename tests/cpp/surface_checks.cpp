// Drives the engine only through the reference's C++ names
// (include/dsmc_reference_api.h), as code written for the reference would:
// geometry predicates, wall models, the CLL coefficient rule, the stage loop
// of src/Simulation.cpp:138-199, the field gather and Printing(), and the
// single routines GenerateNewParticles, RemoveParticlesInsideBox,
// BinaryCollisionsInCell and ElasticCollision checked against the CPU oracle
// (oracle/dsmc_oracle.h, test infrastructure) on the same streams.
// Exit status 0 when every check holds.  Built and run by
// tests/test_gpu_surface.py.
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "dsmc_oracle.h"
#include "dsmc_philox.h"
#include "dsmc_reference_api.h"

namespace {
int failures = 0;
void expect(bool ok, const char *what)
{
    if (!ok) {
        std::cerr << "FAILED: " << what << '\n';
        ++failures;
    }
}

// Units in the last place between two doubles.
long long ulps(double a, double b)
{
    long long ia, ib;
    std::memcpy(&ia, &a, 8);
    std::memcpy(&ib, &b, 8);
    if (ia < 0)
        ia = static_cast<long long>(0x8000000000000000ull) - ia;
    if (ib < 0)
        ib = static_cast<long long>(0x8000000000000000ull) - ib;
    return ia > ib ? ia - ib : ib - ia;
}

struct State {
    std::vector<double> a[5];
    size_t size() const { return a[0].size(); }
};

State engine_state()
{
    State s;
    dsmc_counters c;
    dsmc_get_counters(dsmc::Context(), 0, &c);
    for (auto &v : s.a)
        v.resize(static_cast<size_t>(c.np));
    int64_t n = 0;
    dsmc_download_particles(dsmc::Context(), 0, s.a[0].data(), s.a[1].data(), s.a[2].data(),
                            s.a[3].data(), s.a[4].data(), c.np, &n);
    return s;
}

State oracle_state(dsmc_oracle *o)
{
    State s;
    for (auto &v : s.a)
        v.resize(static_cast<size_t>(dsmc_oracle_np(o)));
    dsmc_oracle_get_particles(o, s.a[0].data(), s.a[1].data(), s.a[2].data(), s.a[3].data(),
                              s.a[4].data());
    return s;
}

// Positions within pos_ulp, velocities within vel_ulp (the transcendental
// functions of the device and the host differ in their last bits).
bool same_state(const State &g, const State &o, long long pos_ulp, long long vel_ulp)
{
    if (g.size() != o.size())
        return false;
    for (int k = 0; k < 5; ++k)
        for (size_t i = 0; i < g.size(); ++i)
            if (ulps(g.a[k][i], o.a[k][i]) > (k < 2 ? pos_ulp : vel_ulp))
                return false;
    return true;
}
} // namespace

int main(int argc, char **argv)
{
    const std::string out = argc > 1 ? argv[1] : "surface_results";

    // Geometry predicates on a 6 x 6 box.
    BoxX = BoxY = 0.0;
    BoxWidth = BoxHeight = 6.0;
    expect(InsideBox(0.0, 0.0) && InsideBox(2.9, -2.9), "interior points");
    expect(!InsideBox(3.0, 0.0) && !InsideBox(0.0, 3.1), "surface and exterior");
    double t = 0, nx = 0, ny = 0;
    expect(IntersectBox(-4, 0, 2, 0, t, nx, ny) && std::abs(t - 0.5) < 1e-12 && nx == -1 &&
               ny == 0,
           "x-face impact");
    expect(IntersectBox(-4, -4, 2, 2, t, nx, ny) && nx == -1 && ny == 0,
           "corner entry resolved to the x face");
    expect(!IntersectBox(-4, 2, 2, 2, t, nx, ny), "corner touch is not an impact");

    // Wall models.
    MolarMass = 0.040;
    const double m = MolarMass / 6.022045E+23;
    const double d = std::sqrt(0.5);
    double a[3] = {-3, -4, 5}, b[3] = {-3, -4, 5};
    SpecularScattering(a, d, d);
    expect(std::abs(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] - 50) < 1e-12 && a[2] == 5,
           "specular keeps energy and z velocity");
    CLLScattering(b, m, 300, d, d, 0.0, 0.0);
    expect(a[0] == b[0] && a[1] == b[1] && a[2] == b[2], "CLL (0, 0) is specular");
    const double invalid[] = {-0.1, 1.1, std::numeric_limits<double>::quiet_NaN()};
    for (double c : invalid) {
        bool thrown = false;
        double v[3] = {-2, 3, 1.5};
        try {
            CLLScattering(v, m, 300, 1, 0, c, 0.8);
        } catch (const std::invalid_argument &) {
            thrown = true;
        }
        expect(thrown, "invalid CLL coefficient rejected");
    }
    double v[3] = {-500, 20, 10};
    DiffuseScattering(v, m, 300, -1, 0);
    expect(v[0] < 0, "diffuse reflection leaves the -x face outward");

    // The reference's time loop on a small case.
    WallInteraction = WallModel::CLL;
    CLLNormalAccommodation = 0.5;
    CLLTangentialAccommodation = 0.9;
    expect(std::string(WallModelName()) == "cll", "wall model name");
    NX = 40;
    NY = 32;
    NPCFree = 6;
    Dt = 2e-5;
    NStep = 60;
    FirstSamplingStep = 20;
    AttackAngle = 15.0;
    BoxWidth = 3.0;
    BoxHeight = 5.0;
    SetSeed(7, 11);
    Setup();
    expect(UxFree > 0 && UyFree < 0, "positive angle tilts the flow toward negative y");
    InitialConditions();
    const int np0 = NP;
    expect(np0 > 0.9 * NPCFree * NX * NY && np0 < NPCFree * NX * NY, "cold start count");
    long long collisions = 0;
    do {
        SamplingMode = (Step > FirstSamplingStep && Step % SamplingPeriod == 0) ? 1 : 0;
        MoveParticles();
        BoundaryConditions();
        ExchangeParticles();
        Indexing();
        collisions += CollideParticles();
        if (SamplingMode == 1)
            Sampling();
        Step++;
        Time += Dt;
    } while (Step < NStep);
    const std::vector<CELL> field = GatherGlobalField();
    expect(Step == NStep, "step counter");
    expect(SampleStep == NStep - FirstSamplingStep - 1, "sampling steps");
    expect(DragCollisionCount > 0, "wall impacts counted");
    expect(collisions >= 0, "collision count");
    double np = 0;
    for (const CELL &c : field)
        np += c.count_np;
    expect(std::abs(np / SampleStep - NP) < 0.1 * NP, "sampled particles per step");
    dsmc::ResultsDirectory = out;
    Printing(field);
    std::ifstream plt(out + "/cll/DSMC2D_Field.plt");
    std::string header;
    std::getline(plt, header);
    expect(header == "VARIABLES = \"X\" \"Y\" \"N\" \"Ux\" \"Uy\" \"Tx\" \"Ty\" \"T\"",
           "field header");

    // The single routines of the reference headers, against the oracle with
    // the same streams: the user stream (kind 5) keyed by the seed, one step
    // number per call, counted from SetSeed.
    {
        dsmc_oracle *o = dsmc_oracle_create(&dsmc::Parameters(), nullptr, 0);
        State g0 = engine_state();
        dsmc_oracle_set_particles_raw(o, g0.a[0].data(), g0.a[1].data(), g0.a[2].data(),
                                      g0.a[3].data(), g0.a[4].data(),
                                      static_cast<int64_t>(g0.size()));
        SetSeed(7, 11); // the user-stream call counter starts again at 0
        const double strip[4] = {X1 - 0.7, -6.0, X1 + 1.5, 6.0}; // partly outside the domain
        GenerateNewParticles(strip[0], strip[1], strip[2], strip[3], 3 * NFree, UxFree, UyFree,
                             400.0, 1);
        dsmc_oracle_generate(o, strip, 3 * NFree, UxFree, UyFree, 400.0, 1, DSMC_RNG_USER, 0, 0);
        dsmc_oracle_remove_outside_domain(o);
        dsmc_oracle_stage_index(o);
        const State g1 = engine_state(), o1 = oracle_state(o);
        expect(g1.size() > g0.size() && static_cast<int64_t>(g1.size()) == NP,
               "GenerateNewParticles adds particles");
        expect(same_state(g1, o1, 1, 8), "GenerateNewParticles matches the oracle");

        const double cover[4] = {BoxX - 2.0, BoxY - 3.0, BoxX + 2.0, BoxY + 3.0}; // the box
        GenerateNewParticles(cover[0], cover[1], cover[2], cover[3], NFree, 0.0, 0.0, TFree, 0);
        dsmc_oracle_generate(o, cover, NFree, 0.0, 0.0, TFree, 0, DSMC_RNG_USER, 1, 0);
        dsmc_oracle_remove_outside_domain(o);
        dsmc_oracle_stage_index(o);
        const int with_box = NP;
        RemoveParticlesInsideBox();
        dsmc_oracle_remove_inside_box(o);
        dsmc_oracle_stage_index(o);
        expect(NP < with_box && NP == dsmc_oracle_np(o), "RemoveParticlesInsideBox count");
        expect(same_state(engine_state(), oracle_state(o), 1, 8),
               "RemoveParticlesInsideBox matches the oracle");

        // The densest cell's list, collided in a volume small enough for many pairs.
        std::vector<int32_t> starts(static_cast<size_t>(NX) * NY + 1);
        dsmc_get_cell_starts(dsmc::Context(), 0, starts.data());
        size_t best = 0;
        for (size_t k = 0; k + 1 < starts.size(); ++k)
            if (starts[k + 1] - starts[k] > starts[best + 1] - starts[best])
                best = k;
        std::vector<int> ipc;
        for (int32_t q = starts[best + 1] - 1; q >= starts[best]; --q)
            ipc.push_back(q);
        const int nc = BinaryCollisionsInCell(DV * 1e-3, static_cast<int>(ipc.size()), ipc.data());
        int onc = 0;
        std::vector<int32_t> ids(ipc.begin(), ipc.end());
        dsmc_oracle_collide_list(o, DV * 1e-3, static_cast<int>(ids.size()), ids.data(),
                                 DSMC_RNG_USER, 2, 0, &onc);
        expect(nc > 0 && nc == onc, "BinaryCollisionsInCell pairs");
        expect(same_state(engine_state(), oracle_state(o), 1, 8),
               "BinaryCollisionsInCell matches the oracle");

        double v1[3] = {310.0, -45.0, 12.0}, v2[3] = {-150.0, 220.0, -80.0};
        double w1[3] = {310.0, -45.0, 12.0}, w2[3] = {-150.0, 220.0, -80.0};
        const double cr = std::sqrt(460.0 * 460.0 + 265.0 * 265.0 + 92.0 * 92.0);
        ElasticCollision(v1, v2, cr);
        dsmc_oracle_elastic(o, w1, w2, cr, DSMC_RNG_USER, 3, 0);
        bool same = true;
        for (int k = 0; k < 3; ++k)
            same = same && ulps(v1[k], w1[k]) <= 8 && ulps(v2[k], w2[k]) <= 8;
        expect(same, "ElasticCollision matches the oracle");
        dsmc_oracle_destroy(o);
    }

    // RunSimulation's argument handling.
    char prog[] = "dsmc", help[] = "--help", bad[] = "--bogus", aoa[] = "--aoa",
         big[] = "200";
    char *h[] = {prog, help};
    char *e[] = {prog, bad};
    char *r[] = {prog, aoa, big};
    expect(RunSimulation(2, h) == 0, "--help exits 0");
    expect(RunSimulation(2, e) == 2, "unknown option exits 2");
    expect(RunSimulation(3, r) == 2, "angle outside [-180, 180] exits 2");

    if (failures == 0)
        std::cout << "surface checks passed\n";
    return failures == 0 ? 0 : 1;
}
