/*
 * sphgpu.h -- C ABI of the B200 SPH/CRKSPH hydro derivative path.
 *
 * This is the drop-in boundary for Spheral's fluid-hydro hot path.  A thin
 * C++ adapter (a GpuSPHHydroBase<Dim<3>> derived from GenericHydro<Dim<3>>)
 * implements the Physics<Dim<3>> virtuals of the reference by calling these
 * entry points, so the reference's integrators and drivers keep working
 * unchanged.
 *
 * Conventions (all entry points):
 *   - every call returns SPHGPU_OK (0) or a negative SPHGPU_ERR_* code; no
 *     C++ exception crosses the ABI.  sphgpu_last_error() returns a
 *     thread-local description of the last failure.
 *   - host arrays use the reference's Field storage order: one AoS record
 *     per node, internal nodes only.  Vector = (x,y,z); SymTensor =
 *     (xx,xy,xz,yy,yz,zz) (GeomSymmetricTensor<3> element order,
 *     src/Geometry/GeomSymmetricTensorBase.hh); Tensor = row major
 *     (xx,xy,xz,yx,yy,yz,zx,zy,zz) (src/Geometry/GeomTensorBase.hh).
 *   - the handle owns all device memory; the caller owns the handle.
 *   - calls are synchronous with respect to the host unless stated.
 */
#ifndef SPHGPU_H
#define SPHGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace Spheral::dbc::VERIFYError, src/Utilities/DBC.hh:20-40) */
#define SPHGPU_OK                 0
#define SPHGPU_ERR_ARG           -1  /* bad argument / unknown field key        */
#define SPHGPU_ERR_CUDA          -2  /* CUDA runtime failure                    */
#define SPHGPU_ERR_CAPACITY      -3  /* neighbor/ghost capacity exceeded        */
#define SPHGPU_ERR_STATE         -4  /* call out of order (e.g. no neighbors)   */
#define SPHGPU_ERR_UNSUPPORTED   -5  /* option outside the implemented subset   */
#define SPHGPU_ERR_NUMERIC       -6  /* non-finite / non-positive state         */
#define SPHGPU_ERR_NOMEM         -7  /* device allocation failed                */
#define SPHGPU_ERR_ADMISSION     -8  /* serving: request exceeds memory budget  */

/* ---- enumerations mirroring the reference's Python factory options ---- */
#define SPHGPU_HYDRO_SPH          0  /* SPHHydroBase   (src/SPH/SPHHydroBase.hh:40)      */
#define SPHGPU_HYDRO_CRKSPH       1  /* CRKSPHHydroBase (src/CRKSPH/CRKSPHHydroBase.hh:59) */

#define SPHGPU_KERNEL_BSPLINE     0  /* BSplineKernel<Dim<3>>    (src/Kernel/BSplineKernelInline.hh) */
#define SPHGPU_KERNEL_WENDLANDC4  1  /* WendlandC4Kernel<Dim<3>> (src/Kernel/WendlandC4KernelInline.hh) */

#define SPHGPU_DENSITY_RIGOROUS_SUM 0 /* MassDensityType::RigorousSumDensity */
#define SPHGPU_DENSITY_INTEGRATE    1 /* MassDensityType::IntegrateDensity   */

#define SPHGPU_H_IDEAL            0  /* HEvolutionType::IdealH      */
#define SPHGPU_H_INTEGRATE        1  /* HEvolutionType::IntegrateH  */

#define SPHGPU_PRECISION_FP64     0  /* plain all-FP64 pair arithmetic                     */
#define SPHGPU_PRECISION_MIXED    1  /* FP32 pair arithmetic, Kahan FP32 sums, FP64 state  */

#define SPHGPU_CRK_SUMVOLUME      0  /* CRKVolumeType::CRKSumVolume       */
#define SPHGPU_CRK_MASSOVERDENSITY 1 /* CRKVolumeType::CRKMassOverDensity */

#define SPHGPU_Q_MONAGHAN_GINGOLD 0  /* MonaghanGingoldViscosity (src/ArtificialViscosity/MonaghanGingoldViscosity.cc) */
#define SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD 1 /* CRKSPHMonaghanGingoldViscosity: limited, gradient-reconstructed
                                       (src/ArtificialViscosity/CRKSPHMonaghanGingoldViscosity.cc:60-313);
                                       CRKSPH problems only */

/* Problem configuration: every physics switch of SPHHydroBase's constructor
 * (src/SPH/SPHHydroBase.cc:82-141), MonaghanGingoldViscosity
 * (src/ArtificialViscosity/MonaghanGingoldViscosity.cc:43-50), GammaLawGas,
 * the FluidNodeList limits (src/NodeList/FluidNodeLists.py:11-35), the periodic
 * box (PeriodicBoundary pairs, src/Boundary/PeriodicBoundary.cc:67-73) and the
 * integrator time-step controls (src/Integrator/Integrator.cc:166-212). */
typedef struct sphgpu_config {
  int32_t hydro;                 /* SPHGPU_HYDRO_*                       */
  int32_t kernel;                /* SPHGPU_KERNEL_*                      */
  int32_t num_points;            /* TableKernel numPoints (drivers: 1000) */
  int32_t precision;             /* SPHGPU_PRECISION_*                   */
  double  nPerh;                 /* nodes per smoothing scale            */
  double  Cl, Cq, epsilon2;      /* Q coefficients, eps^2 (C++ default 1e-2) */
  int32_t linearInExpansion;
  int32_t quadraticInExpansion;
  double  cfl;
  double  epsTensile, nTensile;
  double  hmin, hmax, hminratio;
  double  rhoMin, rhoMax;
  double  gamma;                 /* GammaLawGas gamma (mu irrelevant for P, cs) */
  int32_t compatibleEnergyEvolution;
  int32_t gradhCorrection;
  int32_t XSPH;
  int32_t correctVelocityGradient;
  int32_t densityUpdate;         /* SPHGPU_DENSITY_*                     */
  int32_t HUpdate;               /* SPHGPU_H_*                           */
  int32_t useVelocityMagnitudeForDt;
  int32_t crkVolumeType;         /* SPHGPU_CRK_* (CRKSPH only)            */
  double  xmin[3], xmax[3];      /* periodic box planes                  */
  int32_t periodic[3];           /* 1 = PeriodicBoundary along that axis */
  int32_t max_neighbors;         /* per-node neighbor capacity (0 = 1024) */
  double  dtMin, dtMax, dtGrowth, lastDt;  /* Integrator controls       */
  int32_t qType;                 /* SPHGPU_Q_*                           */
  int32_t balsaraShearCorrection; /* ArtificialViscosity::balsaraShearCorrection
                                     (src/ArtificialViscosity/ArtificialViscosity.cc:123-148),
                                     off by default; SPH problems only */
  double  etaCritFrac, etaFoldFrac;  /* CRKSPH Q: full Q below etaCritFrac/nPerh,
                                        fold width etaFoldFrac/nPerh (defaults 1, 0.2) */
} sphgpu_config;

typedef struct sphgpu_problem sphgpu_problem;

/* Thread-local text of the last error (never NULL). */
const char* sphgpu_last_error(void);

/* Replaces the SPHHydroBase / CRKSPHHydroBase constructors plus
 * initializeProblemStartup (src/SPH/SPHHydroBase.cc:82-230): builds the
 * TableKernel, W(0) and nPerh tables and reserves device storage for
 * n_internal nodes of one FluidNodeList on the current CUDA device. */
int sphgpu_create(const sphgpu_config* cfg, int64_t n_internal, sphgpu_problem** out);
void sphgpu_destroy(sphgpu_problem* p);

/* Host -> device copy of the evolved state of the internal nodes, AoS as in
 * the reference Fields ("position", "velocity", "mass", "mass density",
 * "specific thermal energy", "H"); pressure and sound speed are recomputed
 * from the EOS (SPHHydroBase::initializeProblemStartup, :194-197). */
int sphgpu_set_state(sphgpu_problem* p, const double* position, const double* velocity,
                     const double* mass, const double* massDensity,
                     const double* specificThermalEnergy, const double* H);
/* Same, from device pointers already resident on this GPU (no host copy). */
int sphgpu_set_state_device(sphgpu_problem* p, const double* position, const double* velocity,
                            const double* mass, const double* massDensity,
                            const double* specificThermalEnergy, const double* H);
int sphgpu_get_state(sphgpu_problem* p, double* position, double* velocity, double* mass,
                     double* massDensity, double* specificThermalEnergy, double* H);

/* State / StateDerivatives lookup by the reference's field key
 * (src/Hydro/HydroFieldNames.cc), e.g. "delta velocity hydro",
 * "delta specific thermal energy", "delta mass density", "new H",
 * "velocity gradient", "pressure", "sound speed".  `count` is the number of
 * doubles in `out` and must equal n_internal * components. */
int sphgpu_get_field(sphgpu_problem* p, const char* key, double* out, int64_t count);
int sphgpu_field_components(const char* key, int32_t* components);
/* Write a field by the same keys (host AoS, count = n_internal * components):
 * the State or StateDerivatives value a caller carries in, e.g. a domain's
 * derivatives from the last evaluation (FieldList assignment, as the
 * reference's DistributedBoundary fills its ghost Fields).  A CRKSPH "node
 * volume" written here stands for the start-up volume. */
int sphgpu_set_field(sphgpu_problem* p, const char* key, const double* values, int64_t count);
/* Integrator::dtMin / dtMax (src/Integrator/Integrator.hh) after creation,
 * e.g. both set to a time step agreed between domains. */
int sphgpu_set_dt_bounds(sphgpu_problem* p, double dt_min, double dt_max);

/* Integrator::setGhostNodes (src/Integrator/Integrator.cc:445-597) without
 * ghost culling: periodic ghost images in boundary order x, y, z, then
 * ConnectivityMap::computeConnectivity (src/Neighbor/ConnectivityMap.cc:521-890). */
int sphgpu_build_neighbors(sphgpu_problem* p);
int sphgpu_connectivity_size(sphgpu_problem* p, int64_t* num_ghosts, int64_t* num_entries);
/* CSR of the ConnectivityMap: offsets[n_internal+1], neighbors[num_entries]
 * sorted ascending per node (ghost j >= n_internal), and for each ghost the
 * internal node it images (ghost_root[num_ghosts]).  Any pointer may be NULL. */
int sphgpu_get_connectivity(sphgpu_problem* p, int64_t* offsets, int32_t* neighbors,
                            int32_t* ghost_root);
/* The pair-wise accelerations of the last derivative evaluation on the
 * current ConnectivityMap (the reference's HydroFieldNames::pairAccelerations
 * derivative, filled by SPHHydroBase::evaluateDerivatives,
 * src/SPH/SPHHydroBase.cc:773-777): out[3k..3k+2] for ConnectivityMap entry k
 * (node i's row in the order of sphgpu_get_connectivity).  Where node i owns
 * the pair (neighbor j > i or a ghost) the value is the reference's
 * -m_j deltaDvDt bit for bit; otherwise it is m_j deltaDvDt formed from the
 * owner's value (the reference's SpecificThermalEnergyPolicy reads only the
 * owner's entries).  count must be 3 x the entries.  Only problems that
 * evolve energy compatibly keep them (SPHGPU_ERR_UNSUPPORTED otherwise);
 * after a neighbor build without an evaluation, SPHGPU_ERR_STATE. */
int sphgpu_get_pair_accelerations(sphgpu_problem* p, double* out, int64_t count);
/* Positions of the ghost nodes of the current connectivity (3 doubles per
 * ghost, in ghost order): the NodeList's ghost "position" values, each its
 * root's position mapped through the periodic planes as
 * PlanarBoundary::setGhostNodes / updateGhostNodes do
 * (src/Boundary/PlanarBoundary.cc:114-181,361-395). */
int sphgpu_get_ghost_positions(sphgpu_problem* p, double* positions);

/* Physics::initialize (SPHHydroBase::initialize, src/SPH/SPHHydroBase.cc:430-466;
 * CRKSPHHydroBase::initialize, src/CRKSPH/CRKSPHHydroBase.cc:583-641). */
int sphgpu_initialize(sphgpu_problem* p, double time, double dt);
/* Physics::evaluateDerivatives (src/SPH/SPHHydroBase.cc:471-928;
 * src/CRKSPH/CRKSPHHydroBase.cc:646-1102).  Derivatives are zeroed first
 * (StateDerivatives::Zero, src/DataBase/StateDerivatives.cc:155). */
int sphgpu_evaluate_derivatives(sphgpu_problem* p, double time, double dt);
/* Physics::finalizeDerivatives (src/SPH/SPHHydroBase.cc:933-957). */
int sphgpu_finalize_derivatives(sphgpu_problem* p, double time, double dt);
/* Physics::finalize (src/SPH/SPHHydroBase.cc:962-1105; CRK :1192-1332). */
int sphgpu_finalize(sphgpu_problem* p, double time, double dt);
/* GenericHydro::dt (src/Physics/GenericHydro.cc:114-331): cfl * min dt. */
int sphgpu_dt(sphgpu_problem* p, double* dt_out);
/* CheapSynchronousRK2::step (src/Integrator/CheapSynchronousRK2.cc:81-143),
 * nsteps times; *time advances, *last_dt receives the last step size. */
int sphgpu_step_rk2(sphgpu_problem* p, double* time, int64_t nsteps, double* last_dt);
/* One CheapSynchronousRK2::step (src/Integrator/CheapSynchronousRK2.cc:81-143)
 * of a state that lives in host arrays, as the reference's integrator holds
 * it in its Fields: the state in (as sphgpu_set_state; all six inputs
 * required), one step, the new state out (as sphgpu_get_state; a NULL
 * output is skipped; outputs may alias the inputs).  Same results as those
 * three calls.  The position and H copies go first; for SPH problems the
 * ghost and connectivity rebuild, which reads only those, is queued before
 * the rest of the state is copied on a second stream.  Synchronous. */
int sphgpu_step_rk2_host(sphgpu_problem* p, const double* position, const double* velocity, const double* mass,
                         const double* massDensity, const double* specificThermalEnergy, const double* H,
                         double* position_out, double* velocity_out, double* mass_out, double* massDensity_out,
                         double* specificThermalEnergy_out, double* H_out, double* time, double* last_dt);
/* Integrator::currentTime and lastDt (src/Integrator/Integrator.hh) of the problem. */
int sphgpu_time(sphgpu_problem* p, double* time, double* last_dt);
/* iterateIdealH (src/Utilities/iterateIdealH.cc:26-349) as the reference's
 * controller calls it at start-up (SpheralController.iterateIdealH: at most
 * max_iterations iterations, tolerance on the relative change of H, no
 * nPerh rescaling, no spherical start, no fixed determinant) with
 * SPHSmoothingScale.  Each iteration rebuilds the ghosts and the
 * ConnectivityMap from the current H and replaces the H of every node not
 * yet converged by its ideal H.  Returns the iterations done and the
 * largest change of the last one; the connectivity must be rebuilt
 * afterwards (sphgpu_build_neighbors or the next step). */
int sphgpu_iterate_ideal_h(sphgpu_problem* p, int32_t max_iterations, double tolerance, int32_t* iterations,
                           double* max_delta_h);
/* Checkpoint and restart (SPHHydroBase::dumpState/restoreState,
 * src/SPH/SPHHydroBase.cc:1283-1357, with the NodeList state and the
 * integrator's time, last dt and cycle).  The image is a self-describing
 * byte buffer: a header (format tag, node count, hydro form, precision, field
 * counts, time, last dt, cycle) followed by the FP64 state, the
 * StateDerivatives and, for CRKSPH, the corrections and moments.  Restoring
 * it into a problem created with the same configuration and node count
 * continues the run bit for bit (the next step rebuilds the connectivity, as
 * every step does).  A size, tag or layout mismatch returns SPHGPU_ERR_ARG. */
int sphgpu_checkpoint_size(sphgpu_problem* p, int64_t* bytes);
int sphgpu_checkpoint_save(sphgpu_problem* p, void* buffer, int64_t bytes);
int sphgpu_checkpoint_load(sphgpu_problem* p, const void* buffer, int64_t bytes);
/* Restart files in the reference's own layout: what RestartRegistrar::dumpState
 * (src/DataOutput/RestartRegistrar.cc:155-171) writes through FlatFileIO in
 * ascii form (src/FileIO/FlatFileIO.cc; "path value" lines at precision 20,
 * Fields as "path n v0 v1 ...", FieldLists as path/NodeListNames + path/Field0)
 * for the objects of a one-NodeList problem, in registration order under their
 * unique labels: FluidNodeList (NodeList::dumpState + FluidNodeList::dumpState,
 * src/NodeList/NodeList.cc:606-621, FluidNodeList.cc:180-189), the artificial
 * viscosity (src/ArtificialViscosity/ArtificialViscosity.cc:173-179),
 * SPHHydroBase (src/SPH/SPHHydroBase.cc:1286-1318) or CRKSPHHydroBase
 * (src/CRKSPH/CRKSPHHydroBase.cc:1455-1485), PeriodicBoundary and its two
 * PlanarBoundary planes per periodic axis (src/Boundary/PlanarBoundary.cc:
 * 297-301), CheapSynchronousRK2 (src/Integrator/Integrator.cc:798-806).  The
 * reference's FlatFileIO and RestartRegistrar::restoreState read the file into
 * a reference problem of the same configuration; the NodeList's per-node
 * "work" timing field is written as 0.
 * sphgpu_restart_dump: node_list_name is the NodeList's name (NULL: "nodes").
 * sphgpu_restart_restore: reads such a file (written by this library or by the
 * reference) into a problem of the same configuration and node count: state,
 * derivatives, CRKSPH corrections, time, last dt and cycle; the next step
 * continues the run as SpheralController.loadRestartFile does
 * (src/SimulationControl/SpheralController.py:514-550).  A missing key or
 * another node count returns SPHGPU_ERR_ARG and leaves the problem unchanged.
 * sphgpu_restart_labels: the labels a dump of `cfg` writes, one per line
 * (host only, no device work). */
int sphgpu_restart_dump(sphgpu_problem* p, const char* path, const char* node_list_name);
int sphgpu_restart_restore(sphgpu_problem* p, const char* path);
int sphgpu_restart_labels(const sphgpu_config* cfg, char* buffer, int64_t bytes);
/* SpheralConservation (src/SimulationControl/SpheralConservation.py:27-63):
 * out = {mass, px, py, pz, kinetic E, thermal E, total E, total E low part},
 * FP64 on device.  The total energy is summed as a double-double (two-sum
 * compensation): out[6] is its rounded value and out[6] + out[7] the total to
 * about 2^-100 relative, so an energy drift below the rounding of a plain FP64
 * sum is still resolved. */
int sphgpu_conservation(sphgpu_problem* p, double out[8]);
/* The same sums over caller-owned DEVICE arrays (reference Field layout:
 * mass[n], velocity[3n] AoS, specificThermalEnergy[n]) with no problem
 * handle and no allocation: no counterpart in the reference.  For callers
 * that must not allocate device memory when they ask for the sums (state in
 * their own buffers under a fixed HBM budget).  Scratch is a fixed device
 * array inside the library, so n <= 16,777,216 (larger n returns
 * SPHGPU_ERR_CAPACITY).  The first call on each device looks up the scratch
 * address (set-up) and keeps it for the life of the process; make it before
 * any stream capture, and do not call the entry point again on a device
 * after a cudaDeviceReset of that device (the kept address is stale then).
 * Work is issued on `stream` (cudaStream_t as void*, NULL = default stream).
 * The call is synchronous: it waits for `stream` and returns with the results
 * in `out` (host memory), so it must not be called while `stream` is being
 * captured.  Calls that overlap in time on one device share the scratch and
 * race. */
int sphgpu_conservation_noalloc(const double* mass, const double* velocity,
                                const double* specificThermalEnergy, int64_t n, void* stream,
                                double out[8]);

/* Pair interactions (the reference's ncalc summed over nodes,
 * src/SPH/SPHHydroBase.cc:674) of the current connectivity. */
int sphgpu_num_pairs(sphgpu_problem* p, int64_t* pairs);
/* sphgpu_num_pairs of each RK2 step's connectivity, summed over the steps
 * taken so far (counted on the device, so it stays exact when many steps run
 * in one call). */
int sphgpu_pairs_evaluated(sphgpu_problem* p, int64_t* pairs);
/* Number of CUDA kernels this problem has launched so far (diagnostics; the
 * reference's per-node "work" timing field, src/SPH/SPHHydroBase.cc:598,905-925,
 * has no device counterpart). */
int sphgpu_kernel_launches(sphgpu_problem* p, int64_t* launches);
/* Kernel schedules (no counterpart in the reference, whose loops are serial).
 * stage "neighbor walk": 0 = automatic (thread per node while the 27-cell
 * candidate set is small, warp per node otherwise), 1 = thread per node,
 * 2 = warp per node.  Every schedule yields the same ConnectivityMap.
 * stage "pair loop": threads per block of the derivative kernels, 64 or 128.
 * stage "neighbor filter": 1 (default) = an FP32 pre-test decides the pairs
 * clearly inside or outside the kernel support and the exact FP64 test the
 * rest (used only while every H has condition number <= 100, where the FP32
 * error is far inside the band, so the ConnectivityMap is unchanged); 0 = the
 * FP64 test for every candidate.  stage "step graph": 1 (default) = a whole RK2 step
 * (ghost and connectivity rebuild, records, dt, updates, derivatives,
 * compatible energy, sum density, boundaries) is captured once as a CUDA
 * graph and sphgpu_step_rk2(p, n) replays it n times with no host round trip
 * between steps; the rebuild's capacities are checked on the device and a
 * conditional node skips the rest of the step when one overflows, after
 * which the library grows the buffer, takes that step eagerly and captures
 * again.  The graph is captured the second time a buffer layout recurs (a
 * first step of a new layout runs eagerly).  Results are bit-identical to
 * eager launches.  0 = eager launches.  stage "neighbor passes": 1 (default) = the counting
 * walk also builds each node's sorted list and parks it in the
 * pair-acceleration buffer (free until the next derivative evaluation), and
 * a compaction moves the lists into the ConnectivityMap, so the candidates
 * are walked once; used when the problem evolves energy compatibly (it has
 * that buffer) and the lists fit in it, otherwise 2 = a counting walk, then
 * a filling walk.  Both give the same ConnectivityMap.  stage "neighbor
 * cells": cells per kernel reach of the walk's grid, 0 = automatic (1),
 * 1 = cells of one reach (27-cell window), 2 = cells of half a reach
 * (125-cell window, rows and cells beyond the reach skipped).  Same
 * ConnectivityMap either way.  stage "ghost passes": the six periodic
 * boundary passes of the ghost build, 0 = automatic (2 for a problem or a
 * batch of at most 4 members, else 1), 1 = four launches and a prefix sum
 * per pass, 2 = all six passes in one cooperative launch with grid
 * barriers.  Same ghosts in the same order either way.
 * sphgpu_get_schedule reports what the last call used. */
int sphgpu_set_schedule(sphgpu_problem* p, const char* stage, int32_t schedule);
int sphgpu_get_schedule(sphgpu_problem* p, const char* stage, int32_t* schedule);
/* Autotuner: times every schedule of the neighbor walk (thread or warp per
 * node, then cells of one or half a kernel reach) and of the pair loop on
 * the problem's own data (CUDA events, median of three) and keeps the
 * fastest.  Results do not depend on the schedule; the call leaves the
 * connectivity rebuilt and the derivatives evaluated at the current state (as
 * sphgpu_build_neighbors, sphgpu_initialize and sphgpu_evaluate_derivatives
 * do).  report (may be NULL) = {neighbor schedule, ms thread, ms warp,
 * pair-loop threads, ms 64, ms 128, cells per kernel reach, ms with
 * half-reach cells}. */
int sphgpu_autotune(sphgpu_problem* p, double report[8]);
/* ---- batches (no counterpart in the reference, which advances one problem
 * at a time).  A batch advances many independent problems together: each
 * stage of a call is ONE kernel launch over all members, whose blocks are
 * dealt to the members through a per-member block-offset table.  Members keep
 * their own device state and may differ in size, kernel, gamma, hydro form
 * and precision; a member's results are bit-identical to running it alone.
 * Members must live on the current device.  A batch works on its own stream
 * and first waits for work pending on its members' streams. */
typedef struct sphgpu_batch sphgpu_batch;
int sphgpu_batch_create(sphgpu_problem* const* members, int32_t count, sphgpu_batch** out);
void sphgpu_batch_destroy(sphgpu_batch* b);
int sphgpu_batch_size(sphgpu_batch* b, int32_t* count);
/* sphgpu_build_neighbors for every member. */
int sphgpu_batch_build_neighbors(sphgpu_batch* b);
/* sphgpu_initialize + sphgpu_evaluate_derivatives for every member. */
int sphgpu_batch_evaluate_derivatives(sphgpu_batch* b);
/* nsteps CheapSynchronousRK2 steps of every member, each with its own dt;
 * every member's time and last dt advance as with sphgpu_step_rk2. */
int sphgpu_batch_step_rk2(sphgpu_batch* b, int64_t nsteps);
/* Pair interactions of the members' current connectivity, summed. */
int sphgpu_batch_pairs(sphgpu_batch* b, int64_t* pairs);
/* sphgpu_pairs_evaluated summed over the members. */
int sphgpu_batch_pairs_evaluated(sphgpu_batch* b, int64_t* pairs);
int sphgpu_batch_kernel_launches(sphgpu_batch* b, int64_t* launches);
/* Schedule for all members that have not set their own (see sphgpu_set_schedule). */
int sphgpu_batch_set_schedule(sphgpu_batch* b, const char* stage, int32_t schedule);
/* sphgpu_autotune over the whole batch (one schedule per stage for all members). */
int sphgpu_batch_autotune(sphgpu_batch* b, double report[8]);
int sphgpu_batch_get_stream(sphgpu_batch* b, void** stream);

/* ---- serving (no counterpart in the reference).  A continuous-batching
 * request loop: simulations are submitted as they arrive, admitted first come
 * first served while their device-memory footprint fits under the budget
 * (and at most max_members run at once), advanced together by one batched
 * RK2 step per tick with their state resident on the device, and retired
 * when they reach their step count.  A request larger than the whole budget
 * fails with SPHGPU_ERR_ADMISSION (reported through sphgpu_server_status). */
typedef struct sphgpu_server sphgpu_server;
#define SPHGPU_REQ_QUEUED  0
#define SPHGPU_REQ_RUNNING 1
#define SPHGPU_REQ_DONE    2
#define SPHGPU_REQ_FAILED  3
#define SPHGPU_REQ_CANCELLED 4
/* Device bytes the server charges for a request before it runs (host only;
 * positions and H as for sphgpu_set_state). */
int sphgpu_estimate_footprint(const sphgpu_config* cfg, int64_t n, const double* position, const double* H,
                              int64_t* bytes);
int sphgpu_server_create(double hbm_budget_bytes, int32_t max_members, sphgpu_server** out);
void sphgpu_server_destroy(sphgpu_server* s);
/* Queue a simulation: configuration, initial state (host AoS arrays as for
 * sphgpu_set_state, copied at submission) and its number of RK2 steps. */
int sphgpu_server_submit(sphgpu_server* s, const sphgpu_config* cfg, int64_t n, const double* position,
                         const double* velocity, const double* mass, const double* massDensity,
                         const double* specificThermalEnergy, const double* H, int64_t nsteps, int64_t* id);
/* Admit what fits, advance every running simulation by one RK2 step, retire
 * the finished ones.  Returns the running and queued counts afterwards. */
int sphgpu_server_tick(sphgpu_server* s, int32_t* running, int32_t* queued);
/* Withdraw a queued or running request (between ticks).  A running one
 * gives its device memory back to the budget at once; the other running
 * simulations are unaffected.  The request is reported as finished with
 * state SPHGPU_REQ_CANCELLED; fetching it returns SPHGPU_ERR_STATE and
 * releases it.  A finished request returns SPHGPU_ERR_STATE. */
int sphgpu_server_cancel(sphgpu_server* s, int64_t id);
/* Requests finished (done, failed or cancelled) since the last call, up to `capacity`. */
int sphgpu_server_finished(sphgpu_server* s, int64_t* ids, int32_t capacity, int32_t* count);
int sphgpu_server_status(sphgpu_server* s, int64_t id, int32_t* state, int64_t* steps_done, int64_t* pairs);
/* Final state of a finished request (any pointer may be NULL); releases it. */
int sphgpu_server_fetch(sphgpu_server* s, int64_t id, double* position, double* velocity, double* mass,
                        double* massDensity, double* specificThermalEnergy, double* H, double* time);
/* {bytes in use, peak bytes in use, budget, pair interactions, ticks,
 *  completed requests, simulation steps, kernel launches} */
int sphgpu_server_stats(sphgpu_server* s, double out[8]);

/* Synchronise the problem's stream; returns the first device error. */
int sphgpu_synchronize(sphgpu_problem* p);
/* CUDA stream the problem launches on (cudaStream_t as void*). */
int sphgpu_get_stream(sphgpu_problem* p, void** stream);
int sphgpu_set_stream(sphgpu_problem* p, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPHGPU_H */
