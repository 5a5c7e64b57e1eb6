// CPU baseline: the reference solver, built from its own sources with its own
// multiply-with-carry RNG (rng/BRNG.cxx) and the single-rank MPI stub, timed
// around its time loop.
//
// TEST INFRASTRUCTURE ONLY (the CPU arm of the benchmark).
//
// The loop body is the one of RunSimulation (src/Simulation.cpp:138-161):
// MoveParticles, BoundaryConditions, ExchangeParticles, Indexing,
// CollideParticles and, in sampling steps, Sampling.  Parameters that the
// reference fixes at compile time are set through its globals before Setup().
//
// usage: dsmc_ref_baseline NX NY NPCFREE WARMUP STEPS WALL AN AT AOA DT SEED
//        [FIRST_SAMPLING_STEP [FIELD_OUT]]
//   WALL: 0 diffuse, 1 specular, 2 cll (the reference's WallModel order)
//   FIELD_OUT: file receiving GatherGlobalField() as raw doubles (17 per
//   cell, x-major) followed by SampleStep as one double
// prints one JSON line: {"particle_steps": ..., "seconds": ..., ...}
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Boundary.h"
#include "Collision.h"
#include "Geometry.h"
#include "Initialization.h"
#include "MPIManager.h"
#include "RNG.h"
#include "Sampling.h"
#include "SimulationState.h"

[[noreturn]] void dsmc_ref_mpi_abort(int code)
{
    std::fprintf(stderr, "reference aborted with code %d\n", code);
    std::exit(code);
}

const char *dsmc_ref_results_dir() { return "/tmp"; }

int main(int argc, char **argv)
{
    if (argc < 12) {
        std::fprintf(stderr,
                     "usage: %s NX NY NPCFREE WARMUP STEPS WALL AN AT AOA DT SEED [FIRST]\n",
                     argv[0]);
        return 2;
    }
    NX = std::atoi(argv[1]);
    NY = std::atoi(argv[2]);
    NPCFree = std::atof(argv[3]);
    const int warmup = std::atoi(argv[4]);
    const int steps = std::atoi(argv[5]);
    WallInteraction = static_cast<WallModel>(std::atoi(argv[6]));
    CLLNormalAccommodation = std::atof(argv[7]);
    CLLTangentialAccommodation = std::atof(argv[8]);
    AttackAngle = std::atof(argv[9]);
    Dt = std::atof(argv[10]);
    const unsigned seed = static_cast<unsigned>(std::strtoul(argv[11], nullptr, 10));
    FirstSamplingStep = argc > 12 ? std::atoi(argv[12]) : 0;
    NStep = warmup + steps;

    MPI_Init(&argc, &argv);
    MPI_Comm_rank(MPI_COMM_WORLD, &MPIRank);
    MPI_Comm_size(MPI_COMM_WORLD, &MPISize);
    CreateMPICellType();
    CreateMPIParticleType();
    // Distinct seeds per copy, as RunSimulation derives them per rank
    // (src/Simulation.cpp:84-90).
    SetSeed(seed * 7919u + 12345u, 362436069u + 104729u * seed);
    MPIRank = 1; // silence Setup()
    Setup();
    SetupMPIDomain();
    InitialConditions();

    long long particle_steps = 0;
    long long collisions = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < warmup + steps; ++s) {
        if (s == warmup) {
            particle_steps = 0;
            collisions = 0;
            t0 = std::chrono::steady_clock::now();
        }
        SamplingMode = (Step > FirstSamplingStep && Step % SamplingPeriod == 0) ? 1 : 0;
        MoveParticles();
        if (Step > FirstSamplingStep)
            DragSamplingTime += Dt;
        BoundaryConditions();
        ExchangeParticles();
        Indexing();
        collisions += CollideParticles();
        if (SamplingMode == 1)
            Sampling();
        particle_steps += NP;
        Step++;
        Time += Dt;
    }
    const auto t1 = std::chrono::steady_clock::now();
    const double seconds = std::chrono::duration<double>(t1 - t0).count();
    if (argc > 13) {
        const std::vector<CELL> field = GatherGlobalField();
        std::FILE *f = std::fopen(argv[13], "wb");
        if (f == nullptr)
            return 3;
        const double ss = SampleStep;
        std::fwrite(field.data(), sizeof(CELL), field.size(), f);
        std::fwrite(&ss, sizeof ss, 1, f);
        std::fclose(f);
    }
    std::printf("{\"particle_steps\": %lld, \"seconds\": %.6f, \"np\": %d, \"collisions\": %lld, "
                "\"nx\": %d, \"ny\": %d, \"steps\": %d}\n",
                particle_steps, seconds, NP, collisions, NX, NY, steps);
    return 0;
}
