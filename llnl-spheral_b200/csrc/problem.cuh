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
//                         (the reference's "pair-wise accelerations")
// Ghost nodes are never stored as state: every ghost quantity is read from
// its root, positions are re-mapped through the periodic planes.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "devmath.cuh"
#include "../../include/sphgpu.h"

namespace sphgpu {

enum StateField {
  S_X = 0, S_Y, S_Z, S_VX, S_VY, S_VZ, S_M, S_RHO, S_EPS, S_P, S_CS, S_OMEGA,
  S_H = 12,            // 6 components xx,xy,xz,yy,yz,zz
  S_VOL = 18,          // CRKSPH "node volume"
  NSTATE = 19
};

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

enum DerivField {
  D_DXDT = 0,          // 3  "delta position"
  D_DVDT = 3,          // 3  "delta velocity hydro"
  D_DRHODT = 6,        // 1  "delta mass density"
  D_DEPSDT = 7,        // 1  "delta specific thermal energy"
  D_DHDT = 8,          // 6  "delta H"
  D_HIDEAL = 14,       // 6  "new H"
  D_DVDX = 20,         // 9  "velocity gradient"
  D_LDVDX = 29,        // 9  "internal velocity gradient"
  D_M = 38,            // 9  "M SPH gradient correction"
  D_LM = 47,           // 9  "local M SPH gradient correction"
  D_RHOSUM = 56,       // 1  "new mass density"
  D_NORM = 57,         // 1  "normalization"
  D_WNS = 58,          // 1  "weighted neighbor sum"
  D_M2 = 59,           // 6  "mass second moment"
  D_XSPHW = 65,        // 1  "XSPH weight sum"
  D_XSPHDV = 66,       // 3  "XSPH delta vi"
  D_MAXVP = 69,        // 1  "max viscous pressure"
  D_EFFVP = 70,        // 1  "effective viscous pressure"
  D_VISCW = 71,        // 1  "viscous work rate"
  NDERIV = 72
};

// Packed pair record: everything one side of a pair needs.
enum RecField {
  R_X = 0, R_Y, R_Z, R_VX, R_VY, R_VZ, R_M, R_RHO, R_CS, R_HDET,
  R_H = 10,            // 6
  R_PRHO = 16,         // safeOmega*P/(rho*rho)  (tensile-free P/rho^2 term)
  R_MRHO = 17,         // m/rho
  R_P = 18,
  R_SOMEGA = 19,       // safeInv(omega)
  RECW = 20
};

// Read-only physics parameters, passed by value to kernels.
struct Params {
  TableDev W;
  const double* nperh;     // TableKernel nPerh table
  const double* wsum;      // TableKernel Wsum table
  double W0;               // W.kernelValue(0, 1)
  double WnPerh;           // W.kernelValue(1/nPerh, 1)
  double nPerh, Cl, Cq, eps2, epsTensile, gamma, cfl;
  double hmin, hmax, rhoMin, rhoMax;
  double kernelExtent;
  int compatible, XSPH, correctVelGrad, linearInExp, quadInExp, useVelMagDt;
  int HUpdate, densityUpdate, gradh;
  int hydro;               // SPHGPU_HYDRO_*
  BoxBCs bcs;
};

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
  int maxNbr = 1024;
  int maxCount = 0;         // largest neighbor count of the current connectivity
  int nbrSchedule = 0;      // NBR_SCHEDULE_* requested for the neighbor walk
  int lastNbrSchedule = 0;  // schedule the last build used

  double* S = nullptr;
  double* S0 = nullptr;
  double* D = nullptr;
  double* K = nullptr;          // [NCRK][n] CRKSPH fields (CRKSPH problems only)
  double* crec = nullptr;       // [n+G][CRECW] CRKSPH pair records
  int64_t creccap = 0;
  bool crkVolumeReady = false;
  double* rec = nullptr;
  int64_t reccap = 0;

  int32_t* groot = nullptr;
  uint32_t* gcode = nullptr;
  double* gpos = nullptr;   // [3][gcap] ghost positions during creation

  // cell list
  double* cand = nullptr;       // [candcap] 80-byte records x,y,z,H6,index (cell order)
  int32_t* cidx = nullptr;      // [candcap] cell index of each node (unsorted)
  int32_t* sortedIdx = nullptr; // [candcap]
  int64_t candcap = 0;
  int32_t* cellStart = nullptr; // [ncells+1]
  int32_t* cellFill = nullptr;  // [ncells]
  int64_t cellcap = 0;
  int gdim[3] = {1, 1, 1};
  double glo[3] = {0, 0, 0};
  double gcell = 1.0;

  int32_t* counts = nullptr;    // [n]
  int64_t* offsets = nullptr;   // [n+1]
  int32_t* nbr = nullptr;       // [ecap]
  double* pacc = nullptr;       // [3][ecap]

  double* tableCoef = nullptr;
  float* coefF = nullptr;       // FP32 copy of the table (mixed form)
  double* mrec = nullptr;       // [n+G][MRECW] mixed-precision records
  int64_t mreccap = 0;
  double* nperhTab = nullptr;
  double* wsumTab = nullptr;
  Params prm{};

  // scratch
  int64_t* blockSums = nullptr; // scan scratch
  int64_t blockSumsCap = 0;
  int* d_err = nullptr;         // device error word
  double* d_scal = nullptr;     // small reduction results (16 doubles)
  double* d_red = nullptr;      // reduction partials
  int64_t redcap = 0;
  double* staging = nullptr;    // host<->device AoS staging, 9*n doubles
  double* pinned = nullptr;     // pinned host staging for get/set
  int64_t pinnedcap = 0;

  int64_t launches = 0;         // kernels launched by this problem (diagnostics)
  bool haveNbrs = false;
  bool haveDerivs = false;
  double time = 0.0;
  double lastDt = 1e-5;
  int64_t cycle = 0;
};

// Device error bits (d_err).
enum DevError {
  DERR_NBR_CAPACITY = 1,
  DERR_GHOST_CHAIN = 2,
  DERR_H_CLAMP = 4,
  DERR_NONPOSITIVE = 8,
};

// Neighbor-walk schedules (values of sphgpu_set_schedule's "neighbor walk").
enum NbrSchedule {
  NBR_SCHEDULE_AUTO = 0,     // thread per node for small candidate sets, else warp
  NBR_SCHEDULE_THREAD = 1,   // thread per node, cell-sorted order
  NBR_SCHEDULE_WARP = 2,     // warp per node
};

// ---- launchers (ghosts/neighbors: nbrs.cu; physics: sph.cu) ----
int build_ghosts(Problem& p);
int build_cells_and_csr(Problem& p);
void pack_records(Problem& p);
void launch_gradh(Problem& p);
void launch_eval_sph_fp64(Problem& p);
void launch_eval_sph_mixed(Problem& p);
void launch_sum_density(Problem& p);
void launch_update(Problem& p, const double* d_dt, double scale, bool timeAdvanceOnly);
void launch_compatible_energy(Problem& p, const double* d_dt, double scale);
void launch_enforce_boundaries(Problem& p);
void launch_eos(Problem& p);
void launch_dt(Problem& p, double* d_out);
void launch_select_dt(Problem& p, double* d_dt, double* d_lastDt);
void launch_conservation(Problem& p, double* d_out8);
void launch_zero_derivs(Problem& p);
// CRKSPH (crk.cu)
int crk_prepare(Problem& p);
void launch_crk_sum_volume(Problem& p);
void launch_crk_volume_from_density(Problem& p);
void launch_crk_sum_density(Problem& p);
void launch_crk_initialize(Problem& p);
void launch_crk_eval(Problem& p);

// device buffer helpers (api.cu)
int ensure_capacity_ghosts(Problem& p, int64_t gcap);
int ensure_capacity_entries(Problem& p, int64_t ecap);
int ensure_block_sums(Problem& p, int64_t nblocks);
// exclusive prefix sum of int32 counts into out[0..n] (int64), total returned on the host
int exclusive_scan_i32(Problem& p, const int32_t* in, int64_t n, int64_t* out, int64_t* total);
void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* where);

// host TableKernel construction (table.cc)
void build_table_kernel(int kernelType, int numPoints, std::vector<double>& coef6, std::vector<double>& nperh,
                        std::vector<double>& wsum, double& stepSize, double& extent);
double table_kernel_value(const std::vector<double>& coef6, int n, double stepSize, double extent,
                          double eta, double Hdet);

}  // namespace sphgpu
