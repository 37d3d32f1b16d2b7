// TEST INFRASTRUCTURE: the reference's own SPH/CRKSPH fluid path, run on one node set.
//
// Links the reference's SPHHydroBase or CRKSPHHydroBase,
// MonaghanGingoldViscosity or CRKSPHMonaghanGingoldViscosity,
// SPHSmoothingScale, TableKernel, GammaLawGas, FluidNodeList,
// NestedGridNeighbor, ConnectivityMap, PeriodicBoundary, DataBase, State,
// the update policies and CheapSynchronousRK2, all compiled from the
// reference source tree (oracle/build_ref.py) against the stand-in headers and
// stand-in entry points of oracle/refshim, and drives them the way the
// reference's controller does (src/SimulationControl/SpheralController.py:
// 133-188): ghost nodes, initializeProblemStartup, State/StateDerivatives,
// preStepInitialize, initializeDerivatives, one evaluateDerivatives +
// finalizeDerivatives at the start time, then CheapSynchronousRK2 steps.
//
// usage: ref_sph input.bin outdir
//        ref_sph --time WARMUP input.bin [IDEALH_MAXITER IDEALH_TOLERANCE]
//        ref_sph --ideal-h MAXITER TOLERANCE input.bin outdir
//        ref_sph --restart-dump input.bin restart.txt
//        ref_sph --restart-load input.bin restart.txt outdir
// The second form times the reference's CheapSynchronousRK2 steps instead of
// writing fields: after the start-up and WARMUP untimed steps it runs the
// input's step count, timing each step, and prints one JSON line with the
// steps, the seconds they took and the pair interactions they evaluated (the
// reference's ncalc: internal pairs j > i plus every ghost pair).  The third
// form runs the reference's iterateIdealH (src/Utilities/iterateIdealH.cc) the
// way SpheralController.iterateIdealH calls it (SPHSmoothingScale, no nPerh
// rescaling, no spherical start, no fixed determinant) after the start-up
// ghosts, and writes the relaxed H and the iteration count and last change it
// reports.  --restart-dump runs the start-up, the evaluation and the input's
// steps, then writes the reference's restart file: RestartRegistrar::dumpState
// (src/DataOutput/RestartRegistrar.cc) into a FlatFileIO ascii file
// (src/FileIO/FlatFileIO.cc), every registered object under its unique label.
// --restart-load runs the start-up, then restores every registered object
// from such a file the way SpheralController.loadRestartFile does
// (src/SimulationControl/SpheralController.py:514-550), runs the input's
// steps and writes the steps/ fields; the input's node arrays only size the
// problem.
// input.bin: int64 n, int64 nsteps, sphgpu_config (raw struct), then the
// internal nodes' position[3n], velocity[3n], mass[n], mass density[n],
// specific thermal energy[n], H[6n] (float64, the reference Field layouts).
// Writes raw little-endian arrays (name.f64 / name.i64) into outdir.
// Built a second time with -DREF_SPH_GPU (oracle/_ref/ref_sph_gpu): the same
// driver with GpuSPHHydroBase, the reference's SPHHydroBase whose
// evaluateDerivatives runs on the GPU through libsphgpu.so, in place of
// SPHHydroBase: the reference's integrator, policies and boundaries driving
// the device derivatives.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "Geometry/Dimension.hh"
#include "Geometry/GeomPlane.hh"
#include "Material/PhysicalConstants.hh"
#include "Material/GammaLawGas.hh"
#include "NodeList/FluidNodeList.hh"
#include "NodeList/SPHSmoothingScale.hh"
#include "Neighbor/NestedGridNeighbor.hh"
#include "Neighbor/ConnectivityMap.hh"
#include "DataBase/DataBase.hh"
#include "DataBase/State.hh"
#include "DataBase/StateDerivatives.hh"
#include "Boundary/PeriodicBoundary.hh"
#include "Kernel/TableKernel.hh"
#include "Kernel/BSplineKernel.hh"
#include "Kernel/WendlandC4Kernel.hh"
#include "ArtificialViscosity/MonaghanGingoldViscosity.hh"
#include "SPH/SPHHydroBase.hh"
#include "CRKSPH/CRKSPHHydroBase.hh"
#include "ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.hh"
#include "Geometry/GeomThirdRankTensor.hh"
#include "Integrator/CheapSynchronousRK2.hh"
#include "Utilities/iterateIdealH.hh"
#include "FileIO/FlatFileIO.hh"
#include "DataOutput/RestartRegistrar.hh"

#include "sphgpu.h"
#ifdef REF_SPH_GPU
#include "GpuSPHHydroBase.hh"
#endif

using namespace Spheral;
typedef Dim<3> D;
typedef D::Vector Vector;
typedef D::Tensor Tensor;
typedef D::SymTensor SymTensor;

namespace {

std::string g_dir;
bool g_timing = false;
int g_warmup = 0;
int g_idealHMax = -1;          // >= 0: run iterateIdealH instead of the steps
double g_idealHTol = 0.0;
int g_timeIdealHMax = 0;        // --time: iterateIdealH before the run (0: none)
double g_timeIdealHTol = 0.0;
std::string g_restartOut;       // --restart-dump: restart file written after the steps
std::string g_restartIn;        // --restart-load: restart file restored before the steps
bool g_quiet = false;           // no field dumps

template<typename T>
void dumpRaw(const std::string& name, const std::vector<T>& v, const char* ext) {
  if (g_timing || g_quiet) return;
  const std::string path = g_dir + "/" + name + ext;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::perror(path.c_str()); std::exit(1); }
  if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
  std::fclose(f);
}
void dump(const std::string& name, const std::vector<double>& v) { dumpRaw(name, v, ".f64"); }
void dumpI(const std::string& name, const std::vector<int64_t>& v) { dumpRaw(name, v, ".i64"); }

void put(std::vector<double>& out, double x) { out.push_back(x); }
void put(std::vector<double>& out, const Vector& x) { for (int k = 0; k < 3; ++k) out.push_back(x(k)); }
void put(std::vector<double>& out, const Tensor& x) { for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) out.push_back(x(r, c)); }
void put(std::vector<double>& out, const D::ThirdRankTensor& x) {
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) out.push_back(x(i, j, k));
}
void put(std::vector<double>& out, const SymTensor& x) {
  out.push_back(x.xx()); out.push_back(x.xy()); out.push_back(x.xz());
  out.push_back(x.yy()); out.push_back(x.yz()); out.push_back(x.zz());
}

// Internal-node values of a one-NodeList FieldList.
template<typename Value>
void dumpField(const std::string& name, const FieldSpace::FieldList<D, Value>& fl, int n) {
  if (g_timing) return;
  std::vector<double> out;
  const FieldSpace::Field<D, Value>& f = *fl[0];
  for (int i = 0; i < n; ++i) put(out, f(i));
  dump(name, out);
}
template<typename Value>
void dumpField(const std::string& name, const FieldSpace::Field<D, Value>& f, int n) {
  if (g_timing) return;
  std::vector<double> out;
  for (int i = 0; i < n; ++i) put(out, f(i));
  dump(name, out);
}



struct Input {
  int n = 0;
  int64_t nsteps = 0;
  sphgpu_config cfg;
  std::vector<double> pos, vel, mass, rho, eps, H;
};

// Fields every hydro form provides.
template<typename Hydro>
void dumpCommon(const Hydro& hydro, int n) {
  dumpField("eval/pressure", hydro.pressure(), n);
  dumpField("eval/sound speed", hydro.soundSpeed(), n);
  dumpField("eval/delta position", hydro.DxDt(), n);
  dumpField("eval/delta mass density", hydro.DmassDensityDt(), n);
  dumpField("eval/delta velocity hydro", hydro.DvDt(), n);
  dumpField("eval/delta specific thermal energy", hydro.DspecificThermalEnergyDt(), n);
  dumpField("eval/velocity gradient", hydro.DvDx(), n);
  dumpField("eval/internal velocity gradient", hydro.internalDvDx(), n);
  dumpField("eval/delta H", hydro.DHDt(), n);
  dumpField("eval/new H", hydro.Hideal(), n);
  dumpField("eval/max viscous pressure", hydro.maxViscousPressure(), n);
  dumpField("eval/effective viscous pressure", hydro.effectiveViscousPressure(), n);
  dumpField("eval/viscous work rate", hydro.viscousWork(), n);
  dumpField("eval/XSPH delta vi", hydro.XSPHDeltaV(), n);
  dumpField("eval/weighted neighbor sum", hydro.weightedNeighborSum(), n);
  dumpField("eval/mass second moment", hydro.massSecondMoment(), n);
  std::vector<double> pa;
  const FieldSpace::Field<D, std::vector<Vector> >& f = *hydro.pairAccelerations()[0];
  for (int i = 0; i < n; ++i) for (const Vector& a : f(i)) put(pa, a);
  dump("eval/pair accelerations", pa);
}
void dumpForm(const SPHSpace::SPHHydroBase<D>& hydro, int n) {
  dumpCommon(hydro, n);
  dumpField("eval/grad h corrections", hydro.omegaGradh(), n);
  dumpField("eval/new mass density", hydro.massDensitySum(), n);
  dumpField("eval/normalization", hydro.normalization(), n);
  dumpField("eval/M SPH gradient correction", hydro.M(), n);
  dumpField("eval/local M SPH gradient correction", hydro.localM(), n);
  dumpField("eval/XSPH weight sum", hydro.XSPHWeightSum(), n);
}
void dumpForm(const CRKSPHSpace::CRKSPHHydroBase<D>& hydro, int n) {
  dumpCommon(hydro, n);
  dumpField("eval/node volume", hydro.volume(), n);
  dumpField("eval/mass density gradient", hydro.massDensityGradient(), n);
  dumpField("eval/A CRKSPH correction", hydro.A(), n);
  dumpField("eval/B CRKSPH correction", hydro.B(), n);
  dumpField("eval/grad A CRKSPH correction", hydro.gradA(), n);
  dumpField("eval/grad B CRKSPH correction", hydro.gradB(), n);
  dumpField("eval/m0 CRKSPH moment", hydro.m0(), n);
  dumpField("eval/m1 CRKSPH moment", hydro.m1(), n);
  dumpField("eval/m2 CRKSPH moment", hydro.m2(), n);
  dumpField("eval/grad m0 CRKSPH moment", hydro.gradm0(), n);
  dumpField("eval/grad m1 CRKSPH moment", hydro.gradm1(), n);
  dumpField("eval/grad m2 CRKSPH moment", hydro.gradm2(), n);
}
void dumpStepForm(const SPHSpace::SPHHydroBase<D>&, int) {}
void dumpStepForm(const CRKSPHSpace::CRKSPHHydroBase<D>& hydro, int n) { dumpField("steps/node volume", hydro.volume(), n); }

// The controller's start-up, one evaluation, then the RK2 steps
// (src/SimulationControl/SpheralController.py:133-188; no iterateIdealH).
template<typename Hydro>
int run(const Input& in, Hydro& hydro, NodeSpace::FluidNodeList<D>& nodes, DataBaseSpace::DataBase<D>& db) {
  const sphgpu_config& cfg = in.cfg;
  const int n = in.n;
  // Periodic boundaries in x, y, z order, planes (xmin, +e) and (xmax, -e).
  std::vector<BoundarySpace::PeriodicBoundary<D>*> bcs;
  const Vector xmin(cfg.xmin[0], cfg.xmin[1], cfg.xmin[2]), xmax(cfg.xmax[0], cfg.xmax[1], cfg.xmax[2]);
  for (int axis = 0; axis < 3; ++axis) {
    if (!cfg.periodic[axis]) continue;
    Vector n0 = Vector::zero, n1 = Vector::zero;
    n0(axis) = 1.0; n1(axis) = -1.0;
    bcs.push_back(new BoundarySpace::PeriodicBoundary<D>(GeomPlane<D>(xmin, n0), GeomPlane<D>(xmax, n1)));
    hydro.appendBoundary(*bcs.back());
  }
  IntegratorSpace::CheapSynchronousRK2<D> integ(db);
  integ.appendPhysicsPackage(hydro);
  integ.dtMin(cfg.dtMin);
  integ.dtMax(cfg.dtMax);
  integ.dtGrowth(cfg.dtGrowth);
  integ.lastDt(cfg.lastDt);
  integ.currentTime(0.0);

  integ.setGhostNodes();
  if (g_timing && g_timeIdealHMax > 0) {
    // the controller's start-up with iterateInitialH (its default): H
    // relaxed to the ideal smoothing scale before the run, untimed
    // (src/SimulationControl/SpheralController.py:186-187,718-731)
    NodeSpace::SPHSmoothingScale<D> method;
    std::stringstream log;
    std::streambuf* old = std::cerr.rdbuf(log.rdbuf());
    iterateIdealH(db, integ.uniqueBoundaryConditions(), hydro.kernel(), method, g_timeIdealHMax,
                  g_timeIdealHTol, 0.0, false, false);
    std::cerr.rdbuf(old);
    integ.setGhostNodes();
  }
  if (g_idealHMax >= 0) {
    // SpheralController.iterateIdealH (src/SimulationControl/SpheralController.py:718-731)
    NodeSpace::SPHSmoothingScale<D> method;
    std::stringstream log;
    std::streambuf* old = std::cerr.rdbuf(log.rdbuf());
    iterateIdealH(db, integ.uniqueBoundaryConditions(), hydro.kernel(), method, g_idealHMax, g_idealHTol,
                  0.0, false, false);
    std::cerr.rdbuf(old);
    // its progress lines: "iterateIdealH: (iteration, deltaH) = (itr, maxDeltaH)"
    double itr = -1.0, dh = -1.0;
    std::string line;
    while (std::getline(log, line)) {
      const size_t k = line.find(") = (");
      if (k != std::string::npos) std::sscanf(line.c_str() + k + 5, "%lf, %lf", &itr, &dh);
    }
    dumpField("idealh/H", nodes.Hfield(), n);
    dump("idealh/iterations_delta", std::vector<double>{itr, dh});
    for (auto* bc : bcs) delete bc;
    std::printf("ok %d nodes, %g iterations\n", n, itr);
    return 0;
  }
  std::vector<PhysicsSpace::Physics<D>*> packages(1, &hydro);
  hydro.initializeProblemStartup(db);
  for (auto* bc : bcs) bc->initializeProblemStartup();
  State<D> state(db, packages);
  StateDerivatives<D> derivs(db, packages);
  integ.preStepInitialize(state, derivs);
  integ.initializeDerivatives(0.0, 0.0, state, derivs);

  if (!g_restartIn.empty()) {
    FileIOSpace::FlatFileIO file(g_restartIn, FileIOSpace::AccessType::Read, FileIOSpace::FlatFileFormat::ascii);
    DataOutput::RestartRegistrar::instance().restoreState(file);
    file.close();
  } else {
  // Ghosts: root internal node and position of every ghost.
  const int numNodes = nodes.numNodes();
  std::vector<int64_t> root(numNodes);
  for (int i = 0; i < numNodes; ++i) root[i] = i;
  for (auto* bc : bcs) {
    const std::vector<int>& control = bc->controlNodes(nodes);
    const std::vector<int>& ghosts = bc->ghostNodes(nodes);
    for (size_t k = 0; k < ghosts.size(); ++k) root[ghosts[k]] = root[control[k]];
  }
  std::vector<int64_t> groot;
  std::vector<double> gpos;
  for (int g = n; g < numNodes; ++g) { groot.push_back(root[g]); put(gpos, nodes.positions()(g)); }
  dumpI("ghost_root", groot);
  dump("ghost_position", gpos);
  // ConnectivityMap rows (node indices as the reference numbers them).
  const NeighborSpace::ConnectivityMap<D>& cm = db.connectivityMap();
  std::vector<int64_t> offsets(1, 0), nbrs;
  for (int i = 0; i < n; ++i) {
    const std::vector<int>& row = cm.connectivityForNode(&nodes, i)[0];
    for (int j : row) nbrs.push_back(j);
    offsets.push_back(int64_t(nbrs.size()));
  }
  dumpI("conn_offsets", offsets);
  dumpI("conn_neighbors", nbrs);

  // One evaluation at the start time, and the time step it votes for.
  integ.evaluateDerivatives(0.0, 0.0, db, state, derivs);
  integ.finalizeDerivatives(0.0, 0.0, db, state, derivs);
  dumpForm(hydro, n);
  dump("eval/hydro dt", std::vector<double>(1, hydro.dt(db, state, derivs, 0.0).first));
  }

  if (g_timing) {
    for (int s = 0; s < g_warmup; ++s) integ.step(1e30);
    double seconds = 0.0;
    int64_t pairs = 0;
    for (int64_t s = 0; s < in.nsteps; ++s) {
      const auto t0 = std::chrono::steady_clock::now();
      integ.step(1e30);
      seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      const NeighborSpace::ConnectivityMap<D>& cmap = db.connectivityMap();
      for (int i = 0; i < n; ++i)
        for (int j : cmap.connectivityForNode(&nodes, i)[0]) pairs += (j > i);
    }
    for (auto* bc : bcs) delete bc;
    std::printf("{\"steps\": %lld, \"seconds\": %.6f, \"pairs\": %lld, \"nodes\": %d}\n",
                (long long)in.nsteps, seconds, (long long)pairs, n);
    return 0;
  }

  // CheapSynchronousRK2 steps.
  std::vector<double> tdt;
  for (int64_t s = 0; s < in.nsteps; ++s) {
    integ.step(1e30);
    tdt.push_back(integ.currentTime());
    tdt.push_back(integ.lastDt());
  }
  if (!g_restartOut.empty()) {
    FileIOSpace::FlatFileIO file(g_restartOut, FileIOSpace::AccessType::Create, FileIOSpace::FlatFileFormat::ascii);
    DataOutput::RestartRegistrar::instance().dumpState(file);
    file.close();
    for (const std::string& l : DataOutput::RestartRegistrar::instance().uniqueLabels()) std::printf("label %s\n", l.c_str());
  }
  dump("steps/time_dt", tdt);
  dumpField("steps/position", nodes.positions(), n);
  dumpField("steps/velocity", nodes.velocity(), n);
  dumpField("steps/mass density", nodes.massDensity(), n);
  dumpField("steps/specific thermal energy", nodes.specificThermalEnergy(), n);
  dumpField("steps/H", nodes.Hfield(), n);
  dumpField("steps/pressure", hydro.pressure(), n);
  dumpField("steps/sound speed", hydro.soundSpeed(), n);
  dumpStepForm(hydro, n);
  for (auto* bc : bcs) delete bc;
  std::printf("ok %d nodes, %d ghosts\n", n, nodes.numNodes() - n);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const char* inputPath = nullptr;
  if (argc == 6 && std::string(argv[1]) == "--ideal-h") {
    g_idealHMax = std::atoi(argv[2]);
    g_idealHTol = std::atof(argv[3]);
    inputPath = argv[4];
    g_dir = argv[5];
  } else if ((argc == 4 || argc == 6) && std::string(argv[1]) == "--time") {
    g_timing = true;
    g_warmup = std::atoi(argv[2]);
    inputPath = argv[3];
    if (argc == 6) {
      g_timeIdealHMax = std::atoi(argv[4]);
      g_timeIdealHTol = std::atof(argv[5]);
    }
  } else if (argc == 4 && std::string(argv[1]) == "--restart-dump") {
    inputPath = argv[2];
    g_restartOut = argv[3];
    g_quiet = true;
  } else if (argc == 5 && std::string(argv[1]) == "--restart-load") {
    inputPath = argv[2];
    g_restartIn = argv[3];
    g_dir = argv[4];
  } else if (argc == 3) {
    g_dir = argv[2];
    inputPath = argv[1];
  } else {
    std::fprintf(stderr, "usage: %s input.bin outdir | %s --time WARMUP input.bin [IDEALH_MAXITER IDEALH_TOL] | "
                         "%s --ideal-h MAXITER TOL input.bin outdir | %s --restart-dump input.bin restart.txt | "
                         "%s --restart-load input.bin restart.txt outdir\n", argv[0], argv[0], argv[0], argv[0], argv[0]);
    return 2;
  }
  Input in;
  FILE* fin = std::fopen(inputPath, "rb");
  if (!fin) { std::perror(inputPath); return 1; }
  int64_t n64 = 0;
  if (std::fread(&n64, 8, 1, fin) != 1 || std::fread(&in.nsteps, 8, 1, fin) != 1 ||
      std::fread(&in.cfg, sizeof(in.cfg), 1, fin) != 1) { std::fprintf(stderr, "short input\n"); return 1; }
  const int n = in.n = int(n64);
  in.pos.resize(3*n); in.vel.resize(3*n); in.mass.resize(n); in.rho.resize(n); in.eps.resize(n); in.H.resize(6*n);
  const bool ok = std::fread(in.pos.data(), 8, 3*n, fin) == size_t(3*n) && std::fread(in.vel.data(), 8, 3*n, fin) == size_t(3*n) &&
                  std::fread(in.mass.data(), 8, n, fin) == size_t(n) && std::fread(in.rho.data(), 8, n, fin) == size_t(n) &&
                  std::fread(in.eps.data(), 8, n, fin) == size_t(n) && std::fread(in.H.data(), 8, 6*n, fin) == size_t(6*n);
  std::fclose(fin);
  if (!ok) { std::fprintf(stderr, "short input arrays\n"); return 1; }
  const sphgpu_config& cfg = in.cfg;

  // Material and kernel (the drivers' GammaLawGasMKS(gamma, mu) and
  // TableKernel(K(), numPoints), src/Material/MaterialEquationsOfState.py:20-31).
  Material::PhysicalConstants units(1.0, 1.0, 1.0);
  Material::GammaLawGas<D> eos(cfg.gamma, 1.0, units, -1e200, 1e200, Material::MaterialPressureMinType::PressureFloor);
  KernelSpace::BSplineKernel<D> bspline;
  KernelSpace::WendlandC4Kernel<D> wendland;
  KernelSpace::TableKernel<D> WT = cfg.kernel == SPHGPU_KERNEL_BSPLINE ? KernelSpace::TableKernel<D>(bspline, cfg.num_points)
                                                                        : KernelSpace::TableKernel<D>(wendland, cfg.num_points);

  // makeFluidNodeList (src/NodeList/FluidNodeLists.py:11-45).
  NodeSpace::FluidNodeList<D> nodes("nodes", eos, n, 0, cfg.hmin, cfg.hmax, cfg.hminratio, cfg.nPerh,
                                    cfg.max_neighbors > 0 ? cfg.max_neighbors : 500, cfg.rhoMin, cfg.rhoMax);
  NeighborSpace::NestedGridNeighbor<D> neighbor(nodes, NeighborSpace::NeighborSearchType::GatherScatter, 31, 100.0,
                                                Vector::zero, WT.kernelExtent(), 1);
  nodes.registerNeighbor(neighbor);
  for (int i = 0; i < n; ++i) {
    nodes.positions()(i) = Vector(in.pos[3*i], in.pos[3*i + 1], in.pos[3*i + 2]);
    nodes.velocity()(i) = Vector(in.vel[3*i], in.vel[3*i + 1], in.vel[3*i + 2]);
    nodes.mass()(i) = in.mass[i];
    nodes.massDensity()(i) = in.rho[i];
    nodes.specificThermalEnergy()(i) = in.eps[i];
    const double* h = &in.H[6*i];
    nodes.Hfield()(i) = SymTensor(h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]);
  }
  nodes.neighbor().updateNodes();
  DataBaseSpace::DataBase<D> db;
  db.appendNodeList(nodes);
  NodeSpace::SPHSmoothingScale<D> smooth;
  const PhysicsSpace::MassDensityType densityUpdate = cfg.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM
      ? PhysicsSpace::MassDensityType::RigorousSumDensity : PhysicsSpace::MassDensityType::IntegrateDensity;
  const PhysicsSpace::HEvolutionType HUpdate = cfg.HUpdate == SPHGPU_H_IDEAL
      ? PhysicsSpace::HEvolutionType::IdealH : PhysicsSpace::HEvolutionType::IntegrateH;

  if (cfg.hydro == SPHGPU_HYDRO_SPH) {
    if (cfg.qType != SPHGPU_Q_MONAGHAN_GINGOLD) { std::fprintf(stderr, "SPH runs with the Monaghan-Gingold Q\n"); return 2; }
    ArtificialViscositySpace::MonaghanGingoldViscosity<D> Q(cfg.Cl, cfg.Cq, cfg.linearInExpansion != 0,
                                                            cfg.quadraticInExpansion != 0);
    Q.epsilon2(cfg.epsilon2);
    Q.balsaraShearCorrection(cfg.balsaraShearCorrection != 0);
    // SPHHydroBase (src/SPH/SPHHydroBase.hh:53-71): filter 0, total energy off,
    // sumMassDensityOverAllNodeLists (one NodeList), unbounded box.
#ifdef REF_SPH_GPU
    // the same package with its evaluateDerivatives on the GPU (the drop-in
    // adapter llnl-spheral_b200/spheral/GpuSPHHydroBase.hh); everything else
    // stays the reference's
    SPHSpace::GpuSPHHydroBase<D> hydro(cfg, smooth, Q, WT, WT, 0.0, cfg.cfl, cfg.useVelocityMagnitudeForDt != 0,
#else
    SPHSpace::SPHHydroBase<D> hydro(smooth, Q, WT, WT, 0.0, cfg.cfl, cfg.useVelocityMagnitudeForDt != 0,
#endif
                                    cfg.compatibleEnergyEvolution != 0, false, cfg.gradhCorrection != 0, cfg.XSPH != 0,
                                    cfg.correctVelocityGradient != 0, true, densityUpdate, HUpdate,
                                    cfg.epsTensile, cfg.nTensile, Vector(-1e100, -1e100, -1e100), Vector(1e100, 1e100, 1e100));
    return run(in, hydro, nodes, db);
  }
#ifdef REF_SPH_GPU
  std::fprintf(stderr, "the GPU adapter covers SPHHydroBase only\n");
  return 2;
#endif
  // CRKSPHHydroBase (src/CRKSPH/CRKSPHHydroBase.hh:59-78): filter 0, linear
  // order, no surface detection.
  std::unique_ptr<ArtificialViscositySpace::ArtificialViscosity<D> > Q;
  if (cfg.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD)
    Q.reset(new ArtificialViscositySpace::CRKSPHMonaghanGingoldViscosity<D>(cfg.Cl, cfg.Cq, cfg.linearInExpansion != 0,
                                                                           cfg.quadraticInExpansion != 0,
                                                                           cfg.etaCritFrac, cfg.etaFoldFrac));
  else
    Q.reset(new ArtificialViscositySpace::MonaghanGingoldViscosity<D>(cfg.Cl, cfg.Cq, cfg.linearInExpansion != 0,
                                                                     cfg.quadraticInExpansion != 0));
  Q->epsilon2(cfg.epsilon2);
  CRKSPHSpace::CRKSPHHydroBase<D> hydro(smooth, *Q, WT, WT, 0.0, cfg.cfl, cfg.useVelocityMagnitudeForDt != 0,
                                        cfg.compatibleEnergyEvolution != 0, false, cfg.XSPH != 0, densityUpdate, HUpdate,
                                        CRKSPHSpace::CRKOrder::LinearOrder,
                                        cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME ? CRKSPHSpace::CRKVolumeType::CRKSumVolume
                                                                                  : CRKSPHSpace::CRKVolumeType::CRKMassOverDensity,
                                        false, 0.05, 0.8, 1.0, cfg.epsTensile, cfg.nTensile);
  return run(in, hydro, nodes, db);
}
