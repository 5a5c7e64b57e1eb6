// dsmc_reference_api.h - the reference solver's C++ surface, served by the
// B200 engine.
//
// Code written against the reference's headers (include/Simulation.h,
// Initialization.h, Boundary.h, Geometry.h, Collision.h, Sampling.h, RNG.h,
// SimulationState.h) keeps its calls: set the same globals, call Setup(),
// InitialConditions(), then MoveParticles(), BoundaryConditions(), Indexing(),
// CollideParticles(), Sampling() per step, or RunSimulation(argc, argv).
// Every function runs on the GPU through include/dsmc.h; the globals are a
// host-side mirror (particle state lives in device memory and is never
// copied to a host P[] array).  Errors the reference turns into MPI_Abort or
// exit() are thrown as dsmc::Error carrying the same code; CLLScattering
// throws std::invalid_argument as the reference does (src/Boundary.cpp:247-250).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "dsmc.h"

// include/Cell.h: identical layout (17 doubles).
typedef dsmc_cell CELL;

// include/Boundary.h:3-21
enum class WallModel { Diffuse, Specular, CLL };
extern WallModel WallInteraction;
extern double CLLNormalAccommodation;
extern double CLLTangentialAccommodation;
const char *WallModelName();
void DiffuseScattering(double *v, double m, double Tw, double Nx, double Ny);
void SpecularScattering(double *v, double Nx, double Ny);
void CLLScattering(double *v, double m, double wallTemperature, double Nx, double Ny,
                   double normalAccommodation, double tangentialAccommodation);
void MoveParticles();
void BoundaryConditions();
// Particles joining the case (Boundary.cpp:60-92).  Between steps or after
// Indexing(): drawn on the device from the user stream, those outside
// [X1, X2] x [Y1, Y2] dropped as BoundaryConditions() drops them, the rest
// sorted by cell with the population (NP grows).
void GenerateNewParticles(double X1, double Y1, double X2, double Y2, double Ngas, double Ugasx,
                          double Ugasy, double Tgas, int MoveFlag);

// include/Geometry.h
extern double X1, X2;
extern double Y1, Y2;
extern double DZ;
extern int NX, NY;
extern double DL;
extern double BoxX, BoxY, BoxWidth, BoxHeight;
extern double DX, DY;
extern double DV;
void SetupGeometry();
void Indexing();
bool InsideBox(double x, double y);
// Geometry.cpp:231-247, with the swap-with-last order; between steps or
// after Indexing(), then the population is sorted by cell again.
void RemoveParticlesInsideBox();
bool IntersectBox(double x, double y, double dx, double dy, double &tHit, double &normalX,
                  double &normalY);

// include/Initialization.h
void Setup();
void InitialConditions();

// include/Collision.h
// Collision.cpp:7-19, drawing from the user stream.
void ElasticCollision(double *V1, double *V2, double Cr);
// Collision.cpp:21-44 on the particles whose slots IPC lists (indices into
// the cell-sorted population, as dsmc_download_particles orders it), drawing
// from the user stream; returns NC.
int BinaryCollisionsInCell(double CellVolume, int NPC, int *IPC);
int CollideParticles();

// include/Sampling.h
void Sampling();
void Printing(const std::vector<CELL> &GlobalField);

// include/MPIManager.h: one device owns the whole domain, so the exchange
// between BoundaryConditions() and Indexing() moves nothing; the field is
// gathered from the device.
void ExchangeParticles();
std::vector<CELL> GatherGlobalField();

// include/Simulation.h
int RunSimulation(int argc, char **argv);

// rng/RNG.h: the seed is the Philox key of the next Setup(); brng() draws
// from a host-side user stream of the same generator.
void SetSeed(unsigned int u, unsigned int v);
double brng();

// include/SimulationState.h (the parameters and counters a caller uses)
extern double Dt;
extern int NStep;
extern int FirstSamplingStep;
extern int SamplingPeriod;
extern int PrintPeriod;
extern double NPCFree;
extern double MolarMass;
extern double MaFree;
extern double NFree;
extern double TFree;
extern double AttackAngle;
extern double Tw;
extern double Omega;
extern double SigmaRef;
extern double CrRef;
extern double MFTFree;
extern double MFPFree;
extern double KnFree;
extern double DRef;
extern double ViscosityIndex;
extern double Tref;
extern long long DragCollisionCount;
extern double DragImpulseTotal;
extern double DragSamplingTime;
extern int SampleStep;
extern int NP;
extern double Weight;
extern double MoleculeMass;
extern double PFree;
extern double UFree;
extern double UxFree, UyFree;
extern double SampleTime;
extern int Step;
extern double Time;
extern int SamplingMode;

namespace dsmc {

// An engine error with the reference's exit/abort code (dsmc.h status).
class Error : public std::runtime_error {
  public:
    Error(int code, const std::string &what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

// Engine settings the reference fixes at compile time.
extern int Precision;            // DSMC_FP64 (default) or DSMC_FP32
extern std::string ResultsDirectory; // Printing() writes <dir>/<wall>/ ("results")

// The device context behind the surface (null before Setup()), and the
// parameters the last Setup() gave it.
dsmc_ctx *Context();
const dsmc_params &Parameters();

} // namespace dsmc
