// Drives the engine only through the reference's C++ names
// (include/dsmc_reference_api.h), as code written for the reference would:
// geometry predicates, wall models, the CLL coefficient rule, the stage loop
// of src/Simulation.cpp:138-199, the field gather and Printing().
// Exit status 0 when every check holds.  Built and run by
// tests/test_gpu_surface.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>

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
