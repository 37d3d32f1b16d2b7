// Device data layout of one hydro problem (one FluidNodeList, one GPU).
//
// HBM layout (FP64 unless noted):
//   S    [NSTATE][n]      evolved + EOS state of the internal nodes, SoA
//   S0   [NSTATE][n]      start-of-step copy (CheapSynchronousRK2 state0)
//   D    [NDERIV][n]      StateDerivatives of the internal nodes, SoA
//   rec  [n+G][RECW]      packed pair records (state gathered for a neighbor
//                         walk; ghosts are images of their root), 160 B each
//   groot/gcode [G]       ghost -> internal root node, per-axis image code
//   offsets [n+1] (i64), nbr [E] (i32)   ConnectivityMap as CSR, ascending j
//   pacc [3][E]           owner-oriented pair acceleration per CSR entry
//                         (the reference's "pair-wise accelerations"); FP32
//                         in the mixed form
// Ghost nodes are never stored as state: every ghost quantity is read from
// its root, positions are re-mapped through the periodic planes.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <functional>
#include <vector>

#include <cuda_runtime.h>

#include "devmath.cuh"
#include "mixed.cuh"
#include "../../include/sphgpu.h"

// Blocks of 128 threads per SM the derivative pair kernels are compiled for
// (the register budget follows: 65,536 / (128 x blocks)).  The FP64 pair
// kernel keeps node i's record and its two tensor sums in shared memory
// (SPH_FP64_SHARED_I, SPH_FP64_SHARED_ACC), which brings it to 4 blocks: on
// Kelvin-Helmholtz 128^3 and Sod 256x32x32 that evaluates 15-17% faster than
// the all-register form at 2 blocks, with the same bits.
#ifndef SPH_FP64_MIN_BLOCKS
#define SPH_FP64_MIN_BLOCKS 4
#endif
#ifndef SPH_MIXED_MIN_BLOCKS
#define SPH_MIXED_MIN_BLOCKS 3
#endif
// 1: the FP64 pair kernel keeps node i's record in shared memory
#ifndef SPH_FP64_SHARED_I
#define SPH_FP64_SHARED_I 1
#endif
// 1: ... and accumulates its two tensor sums there
#ifndef SPH_FP64_SHARED_ACC
#define SPH_FP64_SHARED_ACC 1
#endif

namespace sphgpu {

enum StateField {
  S_X = 0, S_Y, S_Z, S_VX, S_VY, S_VZ, S_M, S_RHO, S_EPS, S_P, S_CS, S_OMEGA,
  S_H = 12,            // 6 components xx,xy,xz,yy,yz,zz
  S_VOL = 18,          // CRKSPH "node volume"
  NSTATE = 19
};
// Columns of the start-of-step copy S0 that no step reads, kept for the
// restart files: the mass column (mass is constant within a step) holds the
// entropy (the EOS's at the state the caller set; CRKSPH's EntropyPolicy
// updates it every full update), and S_EPS holds the specific thermal energy
// at the start of the last step (the reference's specificThermalEnergy0).
constexpr int S0_ENTROPY = S_M;

// CRKSPH corrections and moments of the internal nodes, SoA [NCRK][n].
enum CrkField {
  K_A = 0,             // 1  "A CRKSPH correction"
  K_B = 1,             // 3  "B CRKSPH correction"
  K_GRADA = 4,         // 3  "grad A CRKSPH correction"
  K_GRADB = 7,         // 9  "grad B CRKSPH correction" (row major)
  K_M0 = 16,           // 1  "m0 CRKSPH moment"
  K_M1 = 17,           // 3  "m1 CRKSPH moment"
  K_M2 = 20,           // 6  "m2 CRKSPH moment"
  K_GRADM0 = 26,       // 3  "grad m0 CRKSPH moment"
  K_GRADM1 = 29,       // 9  "grad m1 CRKSPH moment"
  K_GRADM2 = 38,       // 27 "grad m2 CRKSPH moment" (i*9 + j*3 + k)
  K_GRADRHO = 65,      // 3  "mass density gradient"
  NCRK = 68
};

// CRKSPH pair record: the SPH record fields plus volume and corrections.
enum CrkRecField {
  C_X = 0, C_Y, C_Z, C_VX, C_VY, C_VZ, C_M, C_RHO, C_CS, C_P, C_HDET, C_VOL,
  C_H = 12,            // 6
  C_A = 18,
  C_B = 19,            // 3
  C_GRADA = 22,        // 3
  C_GRADB = 25,        // 9
  CRECW = 34           // 272 bytes
};

// StateDerivatives of the internal nodes.  With one NodeList the reference's
// "internal velocity gradient" and "local M SPH gradient correction" equal
// the velocity gradient and M (every pair is internal to the material), so
// those two keys read D_DVDX and D_M.
enum DerivField {
  D_DXDT = 0,          // 3  "delta position"
  D_DVDT = 3,          // 3  "delta velocity hydro"
  D_DRHODT = 6,        // 1  "delta mass density"
  D_DEPSDT = 7,        // 1  "delta specific thermal energy"
  D_DHDT = 8,          // 6  "delta H"
  D_HIDEAL = 14,       // 6  "new H"
  D_DVDX = 20,         // 9  "velocity gradient", "internal velocity gradient"
  D_M = 29,            // 9  "M SPH gradient correction", "local M SPH gradient correction"
  D_RHOSUM = 38,       // 1  "new mass density"
  D_NORM = 39,         // 1  "normalization"
  D_WNS = 40,          // 1  "weighted neighbor sum"
  D_M2 = 41,           // 6  "mass second moment"
  D_XSPHW = 47,        // 1  "XSPH weight sum"
  D_XSPHDV = 48,       // 3  "XSPH delta vi"
  D_MAXVP = 51,        // 1  "max viscous pressure"
  D_EFFVP = 52,        // 1  "effective viscous pressure"
  D_VISCW = 53,        // 1  "viscous work rate"
  NDERIV = 54
};

// Packed pair record: everything one side of a pair needs.
enum RecField {
  // position, m, det H and H first: the summed density and the CRKSPH
  // volumes read the first 96 bytes (three sectors) of a neighbor's record
  R_X = 0, R_Y, R_Z, R_M, R_HDET,
  R_H = 5,             // 6
  R_VX = 11, R_VY, R_VZ, R_RHO, R_CS,
  R_PRHO = 16,         // safeOmega*P/(rho*rho)  (tensile-free P/rho^2 term)
  R_MRHO = 17,         // m/rho
  R_P = 18,
  R_SOMEGA = 19,       // safeInv(omega)
  RECW = 20
};

// The pair records of one node, from its state.  Written by the record
// pack kernels and by the update kernel (which packs the internal nodes as
// it advances them); every writer is compiled in the same translation unit
// (sph.cu, -fmad=false), so a node's record has the same bits whoever wrote it.
__device__ __forceinline__ void writeRecord(double* rec, int64_t k, const V3& x, const V3& v, double m, double rho,
                                            double cs, double P, double omega, const Sym& H) {
  const double somega = safeInv(omega, 1.0e-30);
  double2* q = reinterpret_cast<double2*>(rec + k*RECW);
  q[0] = make_double2(x.x, x.y);
  q[1] = make_double2(x.z, m);
  q[2] = make_double2(sdet(H), H.xx);
  q[3] = make_double2(H.xy, H.xz);
  q[4] = make_double2(H.yy, H.yz);
  q[5] = make_double2(H.zz, v.x);
  q[6] = make_double2(v.y, v.z);
  q[7] = make_double2(rho, cs);
  q[8] = make_double2(somega*P/(rho*rho), m/rho);
  q[9] = make_double2(P, somega);
}

// Mixed-precision record (MRECW doubles): FP64 position and velocity, FP32
// m, rho, cs, det H, H, P/rho^2 term, m/rho, P, safeOmega, isotropy flag.
__device__ __forceinline__ void writeMixedRecord(double* mrec, int64_t k, const V3& x, const V3& v, double m,
                                                 double rho, double cs, double P, double omega, const Sym& H) {
  const double somega = safeInv(omega, 1.0e-30);
  double2* q = reinterpret_cast<double2*>(mrec + k*MRECW);
  q[0] = make_double2(x.x, x.y);
  q[1] = make_double2(x.z, v.x);
  q[2] = make_double2(v.y, v.z);
  float4* f = reinterpret_cast<float4*>(q + 3);
  f[0] = make_float4((float)m, (float)rho, (float)cs, (float)sdet(H));
  f[1] = make_float4((float)H.xx, (float)H.xy, (float)H.xz, (float)H.yy);
  f[2] = make_float4((float)H.yz, (float)H.zz, (float)(somega*P/(rho*rho)), (float)(m/rho));
  const bool iso = H.xy == 0.0 && H.xz == 0.0 && H.yz == 0.0 && H.xx == H.yy && H.xx == H.zz;
  f[3] = make_float4((float)P, (float)somega, iso ? 1.0f : 0.0f, 0.0f);
}

// Read-only physics parameters of one problem (in its Member descriptor).
struct Params {
  TableDev W;
  const double* nperh;     // TableKernel nPerh table
  const double* wsum;      // TableKernel Wsum table
  // Bracket table of the Wsum bisection (ascending tables only, else null):
  // wsumBins[b] = last index j with wsum[j] <= wsumBin0 + b/wsumBinInv.
  const int32_t* wsumBins;
  int wsumNbins;
  double wsumBin0, wsumBinInv;
  double W0;               // W.kernelValue(0, 1)
  double WnPerh;           // W.kernelValue(1/nPerh, 1)
  double nPerh, Cl, Cq, eps2, epsTensile, gamma, cfl;
  double hmin, hmax, rhoMin, rhoMax;
  double kernelExtent;
  int compatible, XSPH, correctVelGrad, linearInExp, quadInExp, useVelMagDt;
  int HUpdate, densityUpdate, gradh;
  int balsara;             // Balsara shear correction of the Q (SPH)
  int hydro;               // SPHGPU_HYDRO_*
  int qType;               // SPHGPU_Q_*
  int precision;           // SPHGPU_PRECISION_*
  double etaCrit, etaFold; // CRKSPH Q: etaCritFrac/nPerh, etaFoldFrac/nPerh
  double dtMin, dtMax, dtGrowth;   // Integrator time-step controls
  BoxBCs bcs;
};

// Uniform cell grid of one member's neighbor search.
struct Grid {
  double lo[3];
  double cell;
  int dim[3];
  float filterTol;     // relative band of the FP32 neighbor pre-test (0: exact test only)
  int stashCap;        // lists built in the count pass, at most this long, kept in the
                       // pair-acceleration buffer until compacted (0: separate fill pass)
  int64_t stashStride; // thread schedule: element c of sorted slot s at c*stashStride + s
  int sub;             // cells per kernel reach (1: 27-cell walk, 2: 125-cell walk with pruning)
  float reach;         // kernel reach kappa*max(1/min(eig(H))) in cells (device-side, per build)
};

struct Batch;

struct Problem {
  sphgpu_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  int64_t n = 0;            // internal nodes
  int64_t G = 0;            // ghosts
  int64_t gcap = 0;
  int64_t E = 0, ecap = 0;  // CSR entries
  int64_t pairs = 0;        // unordered pairs (ncalc)
  int64_t pairsEvaluated = 0;  // pair interactions of every evaluation in the RK2 steps so far
  int maxNbr = 1024;
  int maxCount = 0;         // largest neighbor count of the current connectivity
  int nbrSchedule = 0;      // NBR_SCHEDULE_* requested for the neighbor walk
  int lastNbrSchedule = 0;  // schedule the last build used
  bool nbrFilter = true;    // FP32 pre-test in the neighbor walk (exact either way)
  bool nbrStash = true;     // single-pass neighbor walk when the lists fit the stash
  int nbrCells = 0;         // cells per kernel reach requested (0 auto, 1, 2)
  int lastNbrCells = 0;     // cells per kernel reach of the last build
  int lastNbrPasses = 0;    // walks over the candidates the last build made (1 or 2)
  int fillCap = 0;          // neighbor-list capacity planned for the fill pass
  int fillSchedule = 0;     // schedule planned for this build (NBR_SCHEDULE_THREAD/WARP)
  // sizes the first neighbor build plans its buffers from (0: built-in guesses)
  int64_t hintG = 0, hintE = 0, hintCells = 0;

  double* S = nullptr;
  double* S0 = nullptr;
  double* D = nullptr;
  double* K = nullptr;          // [NCRK][n] CRKSPH fields (CRKSPH problems only)
  double* Kheld = nullptr;      // [K_M0][n] the corrections A, B, grad A, grad B as the
                                // reference's State holds them between RK2 steps: those of
                                // the last initialize outside a step (each step's state0
                                // copy restores them after its mid-point evaluation);
                                // written to restart files only
  bool omegaResetByStep = false; // the reference's omegaGradh is 1 after an RK2 step (each step's
                                 // State construction resets it, its state0 copy restores that);
                                 // a restart file written then holds 1
  double* qgrad = nullptr;      // [n][QGRADW] velocity gradient cached by the CRKSPH Q's initialize
  double* fshear = nullptr;     // [n] Balsara shear correction of the Q's initialize
  double* crec = nullptr;       // [n+G][CRECW] CRKSPH pair records
  int64_t creccap = 0;
  bool crkVolumeReady = false;
  double* rec = nullptr;
  int64_t reccap = 0;

  int32_t* groot = nullptr;
  uint32_t* gcode = nullptr;
  double* gpos = nullptr;   // [3][gcap] ghost positions during creation

  // cell list
  double* cand = nullptr;       // cell order, CAND_DOUBLES per slot: FP32 pre-test records
                                // (cell offsets, min eig(H)), FP32 max eig(H)
  int32_t* cidx = nullptr;      // [candcap] cell index of each node (unsorted)
  int32_t* sortedIdx = nullptr; // [candcap]
  int64_t candcap = 0;
  int64_t* cellStart = nullptr; // [ncells+1]
  int32_t* cellFill = nullptr;  // [ncells]
  int64_t cellcap = 0;
  int64_t ncells = 0;
  int64_t cellsWanted = 0;      // cells of the last grid at its natural size
  bool cellsMeasured = false;   // cellcap has been planned from a measured cell count
  int64_t ntot = 0;             // n + ghosts created so far (ghost passes)
  Grid grid{};

  int32_t* counts = nullptr;    // [n]
  int64_t* offsets = nullptr;   // [n+1]
  int32_t* nbr = nullptr;       // [ecap]
  double* pacc = nullptr;       // [3][ecap]

  double* tableCoef = nullptr;
  float* coefF = nullptr;       // FP32 copy of the table (mixed form)
  double* mrec = nullptr;       // [n+G][MRECW] mixed-precision records
  int64_t mreccap = 0;
  double* nperhTab = nullptr;
  int32_t* wsumBinsTab = nullptr;   // [kWsumBins + 1] Params::wsumBins
  double* wsumTab = nullptr;
  Params prm{};

  // scratch
  int64_t* blockSums = nullptr; // scan scratch
  int64_t blockSumsCap = 0;
  int* d_err = nullptr;         // device error word
  double* d_scal = nullptr;     // NSCAL scalar slots (ScalSlot)
  double* d_red = nullptr;      // reduction partials
  int64_t redcap = 0;
  double* staging = nullptr;    // host<->device AoS staging, 9*n doubles
  double* hmaxi = nullptr;      // [2][n] 1/min(eig(H)), max(eig(H)) of each internal node, per build
  double* pinned = nullptr;     // pinned host staging for get/set
  int64_t pinnedcap = 0;
  // sphgpu_step_rk2_host (made on its first call): a copy stream, its
  // events and a second staging buffer (6 n doubles) for the state that
  // crosses the host link while the connectivity is rebuilt
  cudaStream_t copyStream = nullptr;
  cudaEvent_t evCopyStart = nullptr, evCopyDone = nullptr;
  double* stagingB = nullptr;

  Batch* solo = nullptr;        // this problem as a batch of one
  int64_t launches = 0;         // kernels launched for this problem (diagnostics)
  bool haveNbrs = false;
  bool haveDerivs = false;
  bool paccReady = false;       // pacc holds the pair accelerations of an evaluation on the current connectivity
  double time = 0.0;
  double lastDt = 1e-5;
  int64_t cycle = 0;
};

// Device error bits (d_err).
enum DevError {
  DERR_NBR_CAPACITY = 1,
  DERR_GHOST_CHAIN = 2,
  DERR_NONPOSITIVE = 8,
  DERR_GHOST_CAPACITY = 16,   // more ghosts than the ghost buffers hold (build is redone)
  DERR_ENTRY_CAPACITY = 32,   // more CSR entries than the entry buffers hold (build is redone)
  DERR_LIST_CAPACITY = 64,    // a neighbor list longer than the fill pass's list (build is redone)
  DERR_BARRIER = 128,         // a grid barrier of the fused ghost passes waited past its limit
};

// Neighbor-walk schedules (values of sphgpu_set_schedule's "neighbor walk").
enum NbrSchedule {
  NBR_SCHEDULE_AUTO = 0,     // thread per node for small candidate sets, else warp
  NBR_SCHEDULE_THREAD = 1,   // thread per node, cell-sorted order
  NBR_SCHEDULE_WARP = 2,     // warp per node
};

// ---- batched launches -------------------------------------------------
//
// Every kernel runs over a set of independent problems ("members") in one
// launch.  A member is described on the device by a Member record (its
// buffers, sizes and parameters); the blocks of a launch are dealt to the
// members by a block map: first[m] is the first block of member m and
// first[nmem] the grid size.  A single problem is a batch of one member.

// Slots of a member's small device scalar array (64-bit words).
// Doubles per node of the CRKSPH Q's cached velocity gradient (9, padded
// to 80 bytes for 16-byte loads).
constexpr int QGRADW = 10;

// Doubles per slot of the cell-ordered candidate arrays (Problem::cand):
// 16-byte pre-test record + 4-byte FP32 max eig(H), rounded up.
constexpr int CAND_DOUBLES = 3;

enum ScalSlot {
  SC_HMAX = 0,         // ghost hmax of the current boundary (double bits)
  SC_BOUNDS = 1,       // 7 ordered-bit words: lo[3], hi[3], max h
  SC_PAIRS = 8,        // unordered pairs of the connectivity (u64)
  SC_MAXCOUNT = 9,     // largest neighbor count (int)
  SC_MINDT = 10,       // min dt vote before the Courant factor (double bits)
  SC_VOTE = 11,        // cfl * min dt
  SC_DT = 12,          // dt of the current step
  SC_LASTDT = 13,      // dt of the previous step
  SC_DTOUT = 14,       // sphgpu_dt result
  SC_TOTAL = 15,       // total of the last prefix sum (i64)
  SC_CONS = 16,        // 8 conservation sums
  SC_LMAXALL = 24,     // largest eigenvalue of H over the internal nodes (double bits)
  // sizes of the current connectivity, produced and read on the device (i64)
  SC_NTOT = 25,        // internal nodes + ghosts made so far (ghost passes)
  SC_G = 26,           // ghosts
  SC_NCELLS = 27,      // cells of the grid
  SC_GRID = 28,        // lo[3], cell (doubles), dim[3] (i64), pre-test tolerance
  SC_NNEAR = 36,       // internal nodes near a periodic plane (the boundary passes' list)
  SC_REACH = 37,       // kernel reach in cells of the current grid
  SC_CELLSWANTED = 38, // cells of the grid at its natural cell size (i64)
  SC_DELTAH = 39,      // largest H change of an iterateIdealH iteration (double bits)
  // step bookkeeping kept on the device, so that steps replayed from a CUDA
  // graph need no host read-back in between
  SC_TIME = 40,        // current time (advanced by every completed step)
  SC_STEPS = 41,       // completed steps since the host last reset it (i64)
  SC_PAIRSUM = 42,     // pair interactions evaluated by all completed steps (i64)
  SC_PHMAX = 43,       // 6 ghost hmax words, one per boundary pass (fused ghost passes, double bits)
  NSCAL = 49
};

// Sizes and grid of the current connectivity (device side).
// A gathered scalar slot that holds integer bits, on the host.
inline int64_t asI64(double stored) {
  int64_t v;
  std::memcpy(&v, &stored, sizeof(v));
  return v;
}
inline int asI32(double stored) {
  int v;
  std::memcpy(&v, &stored, sizeof(v));
  return v;
}
__device__ __forceinline__ int64_t scalI(const double* scal, int slot) {
  return reinterpret_cast<const int64_t*>(scal)[slot];
}
__device__ __forceinline__ void setScalI(double* scal, int slot, int64_t v) {
  reinterpret_cast<int64_t*>(scal)[slot] = v;
}

struct Member {
  Params prm;
  double* S; double* S0; double* D; double* K;
  double* rec; double* crec; double* mrec;
  double* gpos; double* pacc; double* scal; double* red; double* hmaxi; double* qgrad; double* fshear;
  int32_t* groot; int32_t* cidx; int32_t* sortedIdx; int32_t* counts; int32_t* nbr; int32_t* cellFill;
  uint32_t* gcode;
  int64_t* offsets; int64_t* cellStart; int64_t* blockSums;
  void* cand;
  const float* coefF;
  int* err;
  int64_t n, G, ntot, gcap, E, ecap, candcap, ncells, cellcap;
  Grid grid;
};

struct BlockMap {
  const int32_t* first;
  int nmem;
};

struct MemberBlock {
  int m;            // member index
  int64_t block;    // block index within the member
  int blocks;       // blocks of the member in this launch
};

// The member owning this block: the largest m with first[m] <= blockIdx.x
// (members with no blocks are skipped by construction).
__device__ __forceinline__ MemberBlock memberBlock(const BlockMap& bm) {
  // a single member needs no table (the launch carries no map)
  if (bm.nmem == 1) return MemberBlock{0, (int64_t)blockIdx.x, (int)gridDim.x};
  int lo = 0, hi = bm.nmem - 1;
  const int b = (int)blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(bm.first + mid) <= b) lo = mid; else hi = mid - 1;
  }
  const int f0 = __ldg(bm.first + lo);
  return MemberBlock{lo, (int64_t)(b - f0), __ldg(bm.first + lo + 1) - f0};
}

struct Batch {
  std::vector<Problem*> mem;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  Member* d_mem = nullptr;       // device descriptors of the latest upload
  // Descriptor uploads rotate through kMemSlots slots (pinned host + device),
  // so an upload never waits for the kernels that read an earlier one.
  static constexpr int kMemSlots = 8;
  Member* d_memRing = nullptr;
  Member* h_memRing = nullptr;
  int memcap = 0;                // members per slot
  int memSlot = 0;
  cudaEvent_t memEvents[kMemSlots] = {};
  bool memDirty = true;
  int32_t* d_maps = nullptr;     // block-map ring (device)
  int32_t* h_maps = nullptr;     // pinned host side of the ring
  int64_t mapcap = 0, mappos = 0;
  double* d_gather = nullptr;    // gathered member scalars
  double* h_gather = nullptr;
  int64_t gathercap = 0;
  int64_t launches = 0;
  int nbrSchedule = 0;           // requested neighbor-walk schedule
  int nbrCells = 0;              // requested cells per kernel reach (0 auto)
  int lastNbrSchedule = 0;
  int evalThreads = 128;         // threads per block of the pair-loop kernels (64, 128 or 256)
  int packedByUpdate = 0;        // records the last update kernel wrote (PackNeed), 0: none
  bool midInS0 = false;          // a record-only mid-point update ran: its packed SPH
                                 // members' mid-point H and mass density are in S0
  // CUDA-graph replay of the whole RK2 step, rebuild included (api.cu):
  // captured once per buffer layout, replayed for every step of a call
  // (on unless the "step graph" schedule is set to 0).
  bool useGraph = true;
  // boundary passes of the ghost build: 0 = automatic (one cooperative
  // launch for batches of at most kFusedGhostMembers members), 1 = four
  // launches and a prefix sum per pass, 2 = one cooperative launch
  int ghostPasses = 0;
  int lastGhostPasses = 0;        // what the last build used (1 or 2; 0 before any periodic build)
  unsigned int* d_fuse = nullptr; // fused ghost passes: grid barrier (2 words), then per-block counts
  // the next build's capacities are planned and its descriptors uploaded
  // already (sphgpu_step_rk2_host does both before its copy stream starts)
  bool buildPlanned = false;
  // called once right after the next build's launches are enqueued, before
  // its read-back (sphgpu_step_rk2_host enqueues its second copy group there)
  std::function<int()> afterBuildLaunch;
  uint64_t graphCandidate = 0;   // buffer layout of the last eager step (capture when it recurs)
  bool capturing = false;        // stream capture in progress: maps go to the arena
  bool capacityGrids = false;    // (n + ghosts)-sized kernels sized for the buffer capacity
  cudaGraphExec_t graphExec = nullptr;
  int64_t graphBuildLaunches = 0;  // kernels of the captured rebuild
  uint64_t graphKey = 0;
  int64_t graphLaunches = 0;     // kernel nodes of the captured graph
  cudaStream_t sideStream = nullptr;
  int32_t* d_mapArena = nullptr; // block maps referenced by the captured graph
  int64_t mapArenaCap = 0, mapArenaPos = 0;
  Member* d_memGraph = nullptr;  // descriptor slot read by the captured graph
  Member* h_memGraph = nullptr;
  int memGraphCap = 0;
  cudaEvent_t memGraphEvent = nullptr;
};

// batch.cu
int batch_init(Batch& b, cudaStream_t stream);

// Device buffers of problems and batches come from one stream-ordered memory
// pool per device that keeps freed blocks (release threshold unlimited), so
// creating, growing and destroying problems maps no new memory once the pool
// has grown.  dev_alloc orders the allocation on the legacy stream and
// synchronises it: the block is ready for every stream on return.  dev_free
// synchronises the device first, as cudaFree does, so no kernel still reads
// the block when it returns to the pool; dev_free_all does that once for
// several blocks.  An allocation that fails trims the pool and retries once.
cudaError_t dev_alloc(void** ptr, size_t bytes);
void dev_free(void* ptr);
void dev_free_all(void* const* ptrs, int count);
void batch_free(Batch& b);
int batch_upload(Batch& b);                                  // member descriptors -> device (if dirty)
Member describe_member(const Problem& p);                    // a problem's descriptor (host)
// block map from per-member block counts; *grid = total blocks
int batch_map(Batch& b, const std::vector<int64_t>& blocks, BlockMap* bm, unsigned* grid);
template<class F>
int batch_map_items(Batch& b, F items, int threads, BlockMap* bm, unsigned* grid) {
  std::vector<int64_t> blocks(b.mem.size());
  for (size_t m = 0; m < b.mem.size(); ++m) {
    const int64_t k = items(*b.mem[m]);
    blocks[m] = k > 0 ? (k + threads - 1)/threads : 0;
  }
  return batch_map(b, blocks, bm, grid);
}
// member scalar slots -> host, out[m*nslots + s]; synchronises the stream
int batch_gather(Batch& b, const int* slots, int nslots, std::vector<double>& out);
void batch_count_launch(Batch& b);
// zero (or set) one scalar slot of every member
void batch_set_scal(Batch& b, int slot, double value);
// exclusive prefix sums of every member (in/out chosen by `which`), totals in SC_TOTAL
enum ScanWhich { SCAN_FLAGS = 0, SCAN_CELLS = 1, SCAN_COUNTS = 2 };
// A scan runs on at most kScanBlocks blocks per member, each over a
// contiguous run of tiles, so its grid does not grow with the capacity
// (blockSums holds kScanBlocks + 1 entries).
constexpr int kScanBlocks = 148*2;
int batch_scan(Batch& b, int which);

// ---- stages (ghosts/neighbors: nbrs.cu; SPH: sph.cu; mixed: sph_mixed.cu; CRKSPH: crk.cu)
int build_connectivity(Batch& b);     // ghosts + ConnectivityMap, device-sized
int plan_build(Batch& b);             // capacities and schedules of the next build
int launch_build_captured(Batch& b);  // the build's launches, sized on the device, no read-back
// FP64 pair records of the members that read them next (PACK_ALL: every member)
enum PackNeed { PACK_ALL = 0, PACK_FOR_EVAL = 1, PACK_FOR_FINALIZE = 2 };
int pack_records(Batch& b, int need = PACK_ALL);
// mixed records of the mixed-form SPH members (of those with a summed
// density only, for finalize); sph.cu
int pack_mixed(Batch& b, bool rigorousSumOnly);
// members whose internal records the last update kernel wrote (packMode 1:
// mid-point evaluation, 2: end-of-step summed density); their packs then
// cover the ghosts only
bool packedByUpdate(const Problem& p, int packMode);
int launch_gradh(Batch& b);
int launch_balsara(Batch& b);
int launch_eval_sph_fp64(Batch& b);
int launch_eval_sph_mixed(Batch& b);
// summed density of the plain FP64 / mixed-precision SPH members; enforce:
// also apply the step's periodic wrap to those members' positions
int launch_sum_density(Batch& b, bool enforce = false);
int launch_sum_density_mixed(Batch& b, bool enforce = false);
// mode: 0 in place, 1 save state0 first (mid point), 2 from state0 (full step);
// packMode (PackNeed): also write the internal nodes' records for the next
// evaluation (1) or summed density (2), 0: none; recordMid: the RK2 step's
// record-only mid point for the members the update packs (update_kernel)
int launch_update(Batch& b, double scale, bool timeAdvanceOnly, int mode, int packMode = 0,
                  bool recordMid = false);
// skipSummed: leave out the SPH members whose summed density already wrapped them
int launch_enforce_boundaries(Batch& b, bool skipSummed = false);
int launch_eos(Batch& b);
int launch_dt(Batch& b, int slot, bool cachedEig);
// one iterateIdealH iteration of a single problem; deltaH[n] per-node changes
int launch_ideal_h_iteration(Batch& b, double tolerance, double* deltaH);          // min dt vote bits -> slot
int launch_select_dt(Batch& b);                             // SC_DT from the vote and SC_LASTDT
int launch_finish_step(Batch& b);                           // SC_LASTDT = SC_DT
int launch_conservation(Batch& b);                          // SC_CONS
int launch_zero_derivs(Batch& b);
int prepare_mixed(Batch& b);
int crk_prepare(Batch& b);
int launch_crk_sum_volume(Batch& b, bool startupOnly);      // CRKSumVolume members
int launch_crk_volume_from_density(Batch& b, bool startupOnly);  // CRKMassOverDensity members
int launch_crk_sum_density(Batch& b);
int launch_crk_initialize(Batch& b);
int launch_crk_eval(Batch& b);                              // plain FP64 CRKSPH members
int launch_crk_eval_mixed(Batch& b);                        // mixed-precision CRKSPH members (crk_mixed.cu)

// one CheapSynchronousRK2 step of every member (api.cu)
int batch_step_rk2(Batch& b);
int batch_steps_rk2(Batch& b, int64_t nsteps);   // graph replays where the schedule allows
// TableKernel::equivalentNodesPerSmoothingScale (src/Kernel/TableKernel.cc:
// 402-430): bisectSearch of the Wsum table, then linear interpolation of the
// nPerh table.  The bisection starts from the bracket table's interval for w
// (a few entries) instead of the whole table; every bracket satisfies the
// bisection's invariant wsum[jl] <= w < wsum[ju], so it ends on the same
// index as the full search.
constexpr int kWsumBins = 4096;
__device__ __forceinline__ double equivalentNodesPerSmoothingScale(const Params& P, double w) {
  const int nt = P.W.n;
  const bool ascnd = __ldg(P.wsum + nt - 1) >= __ldg(P.wsum);
  int jl = -1, ju = nt;
  if (P.wsumBins != nullptr && w >= P.wsumBin0) {
    const double q = (w - P.wsumBin0)*P.wsumBinInv;
    const int b = q < (double)(P.wsumNbins - 1) ? (int)q : P.wsumNbins - 1;
    jl = b >= 1 ? __ldg(P.wsumBins + b - 1) : -1;
    ju = __ldg(P.wsumBins + (b + 2 < P.wsumNbins ? b + 2 : P.wsumNbins)) + 1;
  }
  while (ju - jl > 1) {
    const int jm = (ju + jl)/2;
    if ((w >= __ldg(P.wsum + jm)) == ascnd) jl = jm; else ju = jm;
  }
  if (jl == -1) return __ldg(P.nperh);
  if (jl + 1 == nt) return __ldg(P.nperh + nt - 1);
  const double nl = __ldg(P.nperh + jl), nu = __ldg(P.nperh + jl + 1);
  const double wl = __ldg(P.wsum + jl), wu = __ldg(P.wsum + jl + 1);
  return dmin(nu, dmax(nl, nl + (w - wl)/(wu - wl)*(nu - nl)));
}

// device bytes held by a problem, from its buffer capacities (api.cu)
int64_t problem_bytes(const Problem& p);
// device bytes a new problem holds after its first neighbor build, when that
// build is planned from G ghosts, E entries and ncells cells and needs no more
// (the capacity rules of sphgpu_create and plan_capacities; nbrs.cu)
int64_t planned_bytes(const sphgpu_config& cfg, int64_t n, int64_t G, int64_t E, int64_t ncells);

// device buffer helpers (api.cu)
int ensure_capacity_ghosts(Problem& p, int64_t gcap);
int ensure_capacity_entries(Problem& p, int64_t ecap);
int ensure_block_sums(Problem& p, int64_t nblocks);
void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* where);

#define SPH_CHECK(call)                                                 \
  do {                                                                  \
    const cudaError_t e__ = (call);                                     \
    if (e__ != cudaSuccess) return cuda_status(e__, #call);             \
  } while (0)

#define SPH_TRY(expr)                                                   \
  do {                                                                  \
    const int rc__ = (expr);                                            \
    if (rc__ != SPHGPU_OK) return rc__;                                 \
  } while (0)

// host TableKernel construction (table.cc)
void build_table_kernel(int kernelType, int numPoints, std::vector<double>& coef6, std::vector<double>& nperh,
                        std::vector<double>& wsum, double& stepSize, double& extent);
double table_kernel_value(const std::vector<double>& coef6, int n, double stepSize, double extent,
                          double eta, double Hdet);

}  // namespace sphgpu

// Handle types of the C-ABI (include/sphgpu.h).
struct sphgpu_problem : public sphgpu::Problem {};
struct sphgpu_batch : public sphgpu::Batch {};
