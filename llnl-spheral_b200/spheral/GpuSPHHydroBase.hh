// GpuSPHHydroBase: the reference's SPHHydroBase with its derivative
// evaluation on the B200 through libsphgpu (include/sphgpu.h).
//
// A drop-in physics package for Spheral's own integrators and drivers.  It is
// an SPHHydroBase<Dim<3>> in every respect (registerState,
// registerDerivatives, initialize, finalizeDerivatives, finalize, dt,
// dumpState / restoreState, boundaries and policies all stay the reference's,
// src/SPH/SPHHydroBase.cc) except evaluateDerivatives
// (src/SPH/SPHHydroBase.cc:471-928), which this class replaces:
//
//   1. at the start of each step (preStepInitialize, right after the
//      integrator's setGhostNodes rebuilt the reference's ConnectivityMap)
//      the internal nodes' position, velocity, mass, mass density, specific
//      thermal energy and H go to the device as they lie in the Fields
//      (sphgpu_set_state: GeomVector / GeomSymmetricTensor records, no
//      repacking) and the device builds the periodic ghosts and its
//      ConnectivityMap from them (sphgpu_build_neighbors: bit-identical to
//      the reference's);
//   2. at each evaluation (the RK2 mid point) the evolving state, with the
//      pressure and sound speed the reference's policies set, goes to the
//      device by field (sphgpu_set_field) and the device evaluates the
//      grad-h correction and the derivatives on that connectivity, as the
//      reference evaluates on the connectivity of the step's start
//      (sphgpu_initialize, sphgpu_evaluate_derivatives);
//   3. every StateDerivatives field the reference's evaluateDerivatives
//      writes is read back into the internal elements of its Field
//      (sphgpu_get_field, by the reference's own field names), and the
//      pair-wise accelerations into the reference's per-node vectors.
//
// The ghost entries of the derivative Fields stay zero: the reference's
// finalizeDerivatives copies the accelerations and energy rates of the roots
// to the ghosts (src/SPH/SPHHydroBase.cc:936-957), and nothing reads the other
// ghost derivatives.  Pair accelerations: for node i the vector holds one
// entry per neighbor in ConnectivityMap order, as the reference's pair loop
// pushes them; the entries of the pairs node i owns (neighbor j > i, or a
// ghost) are the reference's values bit for bit, the entries of the pairs a
// lower node owns hold that pair's acceleration scaled to node i's side
// (m_owner deltaDvDt, rounded differently: SpecificThermalEnergyPolicy reads
// only the owner's entry, src/Hydro/SpecificThermalEnergyPolicy.cc:145-176).
// A ghost node's vector is sized from the reference's ConnectivityMap (the
// policy's counter steps through it) and holds zeros.
//
// One FluidNodeList, periodic boundaries only, SPH (not CRKSPH); the
// sphgpu_config given to the constructor must describe the same problem as
// the SPHHydroBase arguments (kernel, nPerh, Q coefficients, options, box).
// Errors of the device path throw std::runtime_error with the library's
// message (the reference's VERIFY throws).
#ifndef SPHGPU_GPU_SPH_HYDRO_BASE_HH
#define SPHGPU_GPU_SPH_HYDRO_BASE_HH

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "SPH/SPHHydroBase.hh"
#include "DataBase/DataBase.hh"
#include "DataBase/State.hh"
#include "DataBase/StateDerivatives.hh"
#include "Hydro/HydroFieldNames.hh"
#include "Neighbor/ConnectivityMap.hh"

#include "sphgpu.h"

namespace Spheral {
namespace SPHSpace {

template<typename Dimension>
class GpuSPHHydroBase: public SPHHydroBase<Dimension> {
public:
  typedef typename Dimension::Scalar Scalar;
  typedef typename Dimension::Vector Vector;
  typedef typename Dimension::Tensor Tensor;
  typedef typename Dimension::SymTensor SymTensor;

  // cfg: the device problem's description; the rest: SPHHydroBase's own
  // constructor arguments (src/SPH/SPHHydroBase.hh:53-71).
  template<typename... Args>
  GpuSPHHydroBase(const sphgpu_config& cfg, Args&&... args):
    SPHHydroBase<Dimension>(std::forward<Args>(args)...),
    mConfig(cfg) {}

  virtual ~GpuSPHHydroBase() {
    if (mProblem != nullptr) sphgpu_destroy(mProblem);
  }

  // Physics::preStepInitialize (src/Physics/Physics.hh:110): the state of the
  // step's start to the device and its ConnectivityMap built there.
  virtual
  void preStepInitialize(const DataBaseSpace::DataBase<Dimension>& dataBase,
                         State<Dimension>& state,
                         StateDerivatives<Dimension>& derivs) override {
    SPHHydroBase<Dimension>::preStepInitialize(dataBase, state, derivs);
    startStep(state);
  }

  virtual
  void evaluateDerivatives(const Scalar time,
                           const Scalar dt,
                           const DataBaseSpace::DataBase<Dimension>& dataBase,
                           const State<Dimension>& state,
                           StateDerivatives<Dimension>& derivatives) const override {
    if (mProblem == nullptr) startStep(state);
    const int64_t n = mNodes;
    // the evolving state of this evaluation (the step's start, or its mid point)
    put<Vector>(state, HydroFieldNames::position, n);
    put<Vector>(state, HydroFieldNames::velocity, n);
    put<Scalar>(state, HydroFieldNames::massDensity, n);
    put<Scalar>(state, HydroFieldNames::specificThermalEnergy, n);
    put<SymTensor>(state, HydroFieldNames::H, n);
    put<Scalar>(state, HydroFieldNames::pressure, n);
    put<Scalar>(state, HydroFieldNames::soundSpeed, n);
    check(sphgpu_initialize(mProblem, time, dt), "sphgpu_initialize");
    check(sphgpu_evaluate_derivatives(mProblem, time, dt), "sphgpu_evaluate_derivatives");

    // the fields src/SPH/SPHHydroBase.cc:520-539 fetches, by the same names
    const std::string replace = "new ", increment = "delta ";
    fetch<Scalar>(derivatives, replace + HydroFieldNames::massDensity, n);
    fetch<Scalar>(derivatives, HydroFieldNames::normalization, n);
    fetch<Vector>(derivatives, increment + HydroFieldNames::position, n);
    fetch<Scalar>(derivatives, increment + HydroFieldNames::massDensity, n);
    fetch<Vector>(derivatives, HydroFieldNames::hydroAcceleration, n);
    fetch<Scalar>(derivatives, increment + HydroFieldNames::specificThermalEnergy, n);
    fetch<Tensor>(derivatives, HydroFieldNames::velocityGradient, n);
    fetch<Tensor>(derivatives, HydroFieldNames::internalVelocityGradient, n);
    fetch<Tensor>(derivatives, HydroFieldNames::M_SPHCorrection, n);
    fetch<Tensor>(derivatives, "local " + HydroFieldNames::M_SPHCorrection, n);
    fetch<SymTensor>(derivatives, increment + HydroFieldNames::H, n);
    fetch<SymTensor>(derivatives, replace + HydroFieldNames::H, n);
    fetch<Scalar>(derivatives, HydroFieldNames::maxViscousPressure, n);
    fetch<Scalar>(derivatives, HydroFieldNames::effectiveViscousPressure, n);
    fetch<Scalar>(derivatives, HydroFieldNames::viscousWork, n);
    fetch<Scalar>(derivatives, HydroFieldNames::XSPHWeightSum, n);
    fetch<Vector>(derivatives, HydroFieldNames::XSPHDeltaV, n);
    fetch<Scalar>(derivatives, HydroFieldNames::weightedNeighborSum, n);
    fetch<SymTensor>(derivatives, HydroFieldNames::massSecondMoment, n);
    if (this->compatibleEnergyEvolution()) pairAccelerations(dataBase, derivatives, n);
  }

private:
  sphgpu_config mConfig;
  mutable sphgpu_problem* mProblem = nullptr;
  mutable int64_t mNodes = -1;

  // The problem (re)made for the NodeList's internal nodes, their state
  // uploaded, ghosts and ConnectivityMap built.
  void startStep(const State<Dimension>& state) const {
    const auto position = state.fields(HydroFieldNames::position, Vector::zero);
    const auto velocity = state.fields(HydroFieldNames::velocity, Vector::zero);
    const auto mass = state.fields(HydroFieldNames::mass, 0.0);
    const auto massDensity = state.fields(HydroFieldNames::massDensity, 0.0);
    const auto eps = state.fields(HydroFieldNames::specificThermalEnergy, 0.0);
    const auto H = state.fields(HydroFieldNames::H, SymTensor::zero);
    if (position.numFields() != 1) throw std::runtime_error("GpuSPHHydroBase: exactly one NodeList");
    const int64_t n = position[0]->nodeList().numInternalNodes();
    if (mProblem == nullptr || n != mNodes) {
      if (mProblem != nullptr) sphgpu_destroy(mProblem);
      mProblem = nullptr;
      check(sphgpu_create(&mConfig, n, &mProblem), "sphgpu_create");
      mNodes = n;
    }
    check(sphgpu_set_state(mProblem, data(*position[0]), data(*velocity[0]), data(*mass[0]),
                           data(*massDensity[0]), data(*eps[0]), data(*H[0])), "sphgpu_set_state");
    check(sphgpu_build_neighbors(mProblem), "sphgpu_build_neighbors");
  }

  // Internal elements of one State Field to the device.
  template<typename Value>
  void put(const State<Dimension>& state, const std::string& key, const int64_t n) const {
    const auto fl = state.fields(key, Value());
    const int64_t count = n*(int64_t)(sizeof(Value)/sizeof(double));
    check(sphgpu_set_field(mProblem, key.c_str(), data(*fl[0]), count), key.c_str());
  }

  static void check(int rc, const char* what) {
    if (rc != SPHGPU_OK) throw std::runtime_error(std::string("GpuSPHHydroBase: ") + what + ": " + sphgpu_last_error());
  }

  // A Field's elements are records of doubles (GeomVector, GeomTensor,
  // GeomSymmetricTensor) stored contiguously.
  template<typename Value>
  static double* data(FieldSpace::Field<Dimension, Value>& f) { return reinterpret_cast<double*>(&f(0)); }
  template<typename Value>
  static const double* data(const FieldSpace::Field<Dimension, Value>& f) {
    return reinterpret_cast<const double*>(&f(0));
  }

  // Internal elements of one derivative Field from the device.
  template<typename Value>
  void fetch(StateDerivatives<Dimension>& derivs, const std::string& key, const int64_t n) const {
    auto fl = derivs.fields(key, Value());
    const int64_t count = n*(int64_t)(sizeof(Value)/sizeof(double));
    check(sphgpu_get_field(mProblem, key.c_str(), data(*fl[0]), count), key.c_str());
  }

  void pairAccelerations(const DataBaseSpace::DataBase<Dimension>& dataBase, StateDerivatives<Dimension>& derivs,
                         const int64_t n) const {
    int64_t G = 0, E = 0;
    check(sphgpu_connectivity_size(mProblem, &G, &E), "sphgpu_connectivity_size");
    std::vector<int64_t> offsets(n + 1);
    std::vector<int32_t> nbrs(E), roots(G);
    check(sphgpu_get_connectivity(mProblem, offsets.data(), nbrs.data(), roots.data()), "sphgpu_get_connectivity");
    std::vector<double> pa(3*E);
    check(sphgpu_get_pair_accelerations(mProblem, pa.data(), 3*E), "sphgpu_get_pair_accelerations");
    auto fl = derivs.fields(HydroFieldNames::pairAccelerations, std::vector<Vector>());
    FieldSpace::Field<Dimension, std::vector<Vector> >& f = *fl[0];
    for (int64_t i = 0; i < n; ++i) {
      std::vector<Vector>& v = f(i);
      v.clear();
      for (int64_t k = offsets[i]; k < offsets[i + 1]; ++k) v.push_back(Vector(pa[3*k], pa[3*k + 1], pa[3*k + 2]));
    }
    // ghost nodes: one entry per internal node whose row holds them, in the
    // reference's own ConnectivityMap (its ghost numbering)
    const auto& cm = dataBase.connectivityMap();
    const auto& nodeList = f.nodeList();
    for (int g = (int)n; g < (int)nodeList.numNodes(); ++g) f(g).clear();
    for (int64_t i = 0; i < n; ++i)
      for (int j : cm.connectivityForNode(&nodeList, (int)i)[0])
        if (j >= (int)n) f(j).push_back(Vector::zero);
  }
};

}  // namespace SPHSpace
}  // namespace Spheral

#endif
