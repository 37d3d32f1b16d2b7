// C-ABI of the B200 SPH hydro path and the host-side orchestration of one
// CheapSynchronousRK2 step (src/Integrator/CheapSynchronousRK2.cc:81-143),
// for one problem or for a batch of independent problems.
//
// A problem's own calls run as a batch of one member on the problem's
// stream; a batch runs every stage as one launch over all its members on
// the batch's stream.  Each call returns SPHGPU_OK or a negative status (no
// exceptions cross the ABI); the text of the last failure is kept per host
// thread.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "problem.cuh"
#include "mixed.cuh"

namespace sphgpu {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SPHGPU_OK;
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? SPHGPU_ERR_NOMEM : SPHGPU_ERR_CUDA;
}


namespace {

template<typename T>
int dalloc(T*& ptr, int64_t count) {
  ptr = nullptr;
  if (count <= 0) count = 1;
  const cudaError_t e = dev_alloc(reinterpret_cast<void**>(&ptr), sizeof(T)*(size_t)count);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_status(e, "device allocation");
  }
  return SPHGPU_OK;
}

template<typename T>
int grow_preserve(T*& ptr, int64_t oldCount, int64_t newCount, cudaStream_t st) {
  T* np = nullptr;
  SPH_TRY(dalloc(np, newCount));
  if (ptr != nullptr && oldCount > 0) {
    const cudaError_t e = cudaMemcpyAsync(np, ptr, sizeof(T)*(size_t)oldCount, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) { dev_free(np); return cuda_status(e, "grow copy"); }
  }
  cudaStreamSynchronize(st);
  dev_free(ptr);
  ptr = np;
  return SPHGPU_OK;
}

__global__ void aos_to_soa_kernel(const double* src, int comps, int64_t n, double* dst) {
  for (int64_t t = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; t < n*comps; t += (int64_t)gridDim.x*blockDim.x) {
    const int64_t i = t/comps;
    const int c = (int)(t - i*comps);
    dst[(int64_t)c*n + i] = src[t];
  }
}

__global__ void soa_to_aos_kernel(const double* src, int comps, int64_t n, double* dst) {
  for (int64_t t = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; t < n*comps; t += (int64_t)gridDim.x*blockDim.x) {
    const int64_t i = t/comps;
    const int c = (int)(t - i*comps);
    dst[t] = src[(int64_t)c*n + i];
  }
}

__global__ void fill_kernel(double* dst, int64_t n, double v) {
  for (int64_t t = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x*blockDim.x) dst[t] = v;
}

// The restart-file values of the state the caller set (the reference's
// start-up): the EOS entropy, GammaLawGas::setEntropy
// (src/Material/GammaLawGas.cc:151-158, DataBase::fluidEntropy at the
// hydro's construction), and specificThermalEnergy0 = the specific thermal
// energy with the compatible energy, else 0
// (src/SPH/SPHHydroBase.cc:262-272).
__global__ void startup_restart_kernel(const double* S, double* S0, int64_t n, double gamma, int compatible) {
  for (int64_t i = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x*blockDim.x) {
    const double rho = S[S_RHO*n + i], eps = S[S_EPS*n + i];
    const double P = (gamma - 1.0)*rho*eps;
    S0[S0_ENTROPY*n + i] = P*safeInvVar(pow(rho, gamma));
    S0[S_EPS*n + i] = compatible ? eps : 0.0;
  }
}

__global__ void check_state_kernel(const double* S, int64_t n, int* err) {
  for (int64_t i = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x*blockDim.x) {
    const double m = S[S_M*n + i], rho = S[S_RHO*n + i];
    const Sym H{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
                S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
    bool ok = m > 0.0 && rho > 0.0 && sdet(H) > 0.0 && isfinite(S[S_EPS*n + i]);
    for (int c = 0; c < 6; ++c) ok = ok && isfinite(S[c*n + i]);
    if (!ok) atomicOr(err, DERR_NONPOSITIVE);
  }
}

inline int grid1(int64_t work, int threads = 256) {
  int64_t b = (work + threads - 1)/threads;
  if (b < 1) b = 1;
  if (b > 148*16) b = 148*16;
  return (int)b;
}

struct FieldSpec {
  const char* key;
  int array;      // 0 = state S, 1 = derivatives D, 2 = CRKSPH fields K
  int field;
  int comps;
};

const FieldSpec kFields[] = {
    {"position", 0, S_X, 3},
    {"velocity", 0, S_VX, 3},
    {"mass", 0, S_M, 1},
    {"mass density", 0, S_RHO, 1},
    {"specific thermal energy", 0, S_EPS, 1},
    {"pressure", 0, S_P, 1},
    {"sound speed", 0, S_CS, 1},
    {"grad h corrections", 0, S_OMEGA, 1},
    {"H", 0, S_H, 6},
    {"delta position", 1, D_DXDT, 3},
    {"delta velocity hydro", 1, D_DVDT, 3},
    {"delta mass density", 1, D_DRHODT, 1},
    {"delta specific thermal energy", 1, D_DEPSDT, 1},
    {"delta H", 1, D_DHDT, 6},
    {"new H", 1, D_HIDEAL, 6},
    {"velocity gradient", 1, D_DVDX, 9},
    {"internal velocity gradient", 1, D_DVDX, 9},
    {"M SPH gradient correction", 1, D_M, 9},
    {"local M SPH gradient correction", 1, D_M, 9},
    {"new mass density", 1, D_RHOSUM, 1},
    {"normalization", 1, D_NORM, 1},
    {"weighted neighbor sum", 1, D_WNS, 1},
    {"mass second moment", 1, D_M2, 6},
    {"XSPH weight sum", 1, D_XSPHW, 1},
    {"XSPH delta vi", 1, D_XSPHDV, 3},
    {"max viscous pressure", 1, D_MAXVP, 1},
    {"effective viscous pressure", 1, D_EFFVP, 1},
    {"viscous work rate", 1, D_VISCW, 1},
    {"node volume", 0, S_VOL, 1},
    {"A CRKSPH correction", 2, K_A, 1},
    {"B CRKSPH correction", 2, K_B, 3},
    {"grad A CRKSPH correction", 2, K_GRADA, 3},
    {"grad B CRKSPH correction", 2, K_GRADB, 9},
    {"m0 CRKSPH moment", 2, K_M0, 1},
    {"m1 CRKSPH moment", 2, K_M1, 3},
    {"m2 CRKSPH moment", 2, K_M2, 6},
    {"grad m0 CRKSPH moment", 2, K_GRADM0, 3},
    {"grad m1 CRKSPH moment", 2, K_GRADM1, 9},
    {"grad m2 CRKSPH moment", 2, K_GRADM2, 27},
    {"mass density gradient", 2, K_GRADRHO, 3},
};

const FieldSpec* findField(const char* key) {
  if (key == nullptr) return nullptr;
  for (const auto& f : kFields) if (std::strcmp(f.key, key) == 0) return &f;
  return nullptr;
}

int validate_config(const sphgpu_config& c) {
  if (c.hydro != SPHGPU_HYDRO_SPH && c.hydro != SPHGPU_HYDRO_CRKSPH) { set_error("unknown hydro"); return SPHGPU_ERR_ARG; }
  if (c.crkVolumeType != SPHGPU_CRK_SUMVOLUME && c.crkVolumeType != SPHGPU_CRK_MASSOVERDENSITY) {
    set_error("unknown crkVolumeType"); return SPHGPU_ERR_ARG;
  }
  if (c.kernel != SPHGPU_KERNEL_BSPLINE && c.kernel != SPHGPU_KERNEL_WENDLANDC4) { set_error("unknown kernel"); return SPHGPU_ERR_ARG; }
  if (c.num_points < 4) { set_error("num_points must be >= 4"); return SPHGPU_ERR_ARG; }
  if (c.precision != SPHGPU_PRECISION_FP64 && c.precision != SPHGPU_PRECISION_MIXED) { set_error("unknown precision"); return SPHGPU_ERR_ARG; }
  if (!(c.nPerh > 0.0) || !(c.gamma > 1.0)) { set_error("nPerh must be > 0 and gamma > 1"); return SPHGPU_ERR_ARG; }
  if (c.compatibleEnergyEvolution && c.densityUpdate != SPHGPU_DENSITY_RIGOROUS_SUM && c.densityUpdate != SPHGPU_DENSITY_INTEGRATE) {
    set_error("unknown densityUpdate"); return SPHGPU_ERR_ARG;
  }
  if (c.HUpdate != SPHGPU_H_IDEAL && c.HUpdate != SPHGPU_H_INTEGRATE) { set_error("unknown HUpdate"); return SPHGPU_ERR_ARG; }
  for (int a = 0; a < 3; ++a) if (c.periodic[a] && !(c.xmax[a] > c.xmin[a])) { set_error("empty periodic box"); return SPHGPU_ERR_ARG; }
  if (c.max_neighbors < 0 || c.max_neighbors > 4096) { set_error("max_neighbors must be in [0, 4096]"); return SPHGPU_ERR_ARG; }
  if (c.qType != SPHGPU_Q_MONAGHAN_GINGOLD && c.qType != SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD) {
    set_error("unknown qType"); return SPHGPU_ERR_ARG;
  }
  if (c.balsaraShearCorrection != 0 && c.hydro != SPHGPU_HYDRO_SPH) {
    set_error("the Balsara shear correction is implemented for SPH problems"); return SPHGPU_ERR_UNSUPPORTED;
  }
  if (c.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD && c.hydro != SPHGPU_HYDRO_CRKSPH) {
    set_error("the CRKSPH Monaghan-Gingold Q is implemented for CRKSPH problems"); return SPHGPU_ERR_UNSUPPORTED;
  }
  if (c.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD && !(c.etaCritFrac >= 0.0 && c.etaFoldFrac > 0.0)) {
    set_error("etaCritFrac must be >= 0 and etaFoldFrac > 0"); return SPHGPU_ERR_ARG;
  }
  return SPHGPU_OK;
}

void free_problem(Problem* p) {
  if (p == nullptr) return;
  void* ptrs[] = {p->S, p->S0, p->D, p->rec, p->groot, p->gcode, p->gpos, p->cand, p->cidx, p->sortedIdx,
                  p->cellStart, p->cellFill, p->counts, p->offsets, p->nbr, p->pacc, p->tableCoef, p->nperhTab,
                  p->wsumTab, p->blockSums, p->d_err, p->d_scal, p->d_red, p->staging, p->coefF, p->mrec, p->K, p->crec, p->hmaxi,
                  p->wsumBinsTab, p->qgrad, p->Kheld, p->fshear};
  dev_free_all(ptrs, (int)(sizeof(ptrs)/sizeof(ptrs[0])));
  if (p->pinned) cudaFreeHost(p->pinned);
  if (p->stagingB) { void* sb[] = {p->stagingB}; dev_free_all(sb, 1); }
  if (p->evCopyStart) cudaEventDestroy(p->evCopyStart);
  if (p->evCopyDone) cudaEventDestroy(p->evCopyDone);
  if (p->copyStream) cudaStreamDestroy(p->copyStream);
  if (p->solo) { batch_free(*p->solo); delete p->solo; p->solo = nullptr; }
  if (p->ownStream && p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

// The problem as a batch of one.  Its descriptor is re-uploaded on every
// call: another batch holding the same problem may have moved its buffers.
Batch& solo(Problem* p) {
  p->solo->memDirty = true;
  p->solo->packedByUpdate = 0;      // records written by an update belong to that step only
  p->solo->midInS0 = false;
  return *p->solo;
}

// AoS host arrays -> SoA fields of S (via the device staging buffer).  The
// host-to-device copies go back to back into the staging buffer (9 n
// doubles: position, velocity, mass, density and energy at once, then H), a
// transpose kernel follows each group, and the call synchronises once, at
// its end (the caller's arrays are free again then).
struct AosField { const double* host; int comps; int field; };

int upload_group(Problem& p, const AosField* f, int nf, bool device, double* staging, cudaStream_t st,
                 cudaEvent_t copied = nullptr) {
  int64_t off = 0;
  const double* src[6];
  for (int k = 0; k < nf; ++k) {
    src[k] = f[k].host;
    if (f[k].host == nullptr || device) continue;
    const int64_t cnt = p.n*f[k].comps;
    SPH_CHECK(cudaMemcpyAsync(staging + off, f[k].host, sizeof(double)*(size_t)cnt, cudaMemcpyHostToDevice, st));
    src[k] = staging + off;
    off += cnt;
  }
  if (copied) SPH_CHECK(cudaEventRecord(copied, st));
  for (int k = 0; k < nf; ++k) {
    if (f[k].host == nullptr) continue;
    const int64_t cnt = p.n*f[k].comps;
    aos_to_soa_kernel<<<grid1(cnt), 256, 0, st>>>(src[k], f[k].comps, p.n, p.S + (int64_t)f[k].field*p.n);
    ++p.launches;
  }
  return cuda_status(cudaGetLastError(), "set_state (transpose)");
}

int upload_state(Problem& p, const double* pos, const double* vel, const double* mass, const double* rho,
                 const double* eps, const double* H, bool device) {
  const AosField g1[5] = {{pos, 3, S_X}, {vel, 3, S_VX}, {mass, 1, S_M}, {rho, 1, S_RHO}, {eps, 1, S_EPS}};
  const AosField g2[1] = {{H, 6, S_H}};
  SPH_TRY(upload_group(p, g1, 5, device, p.staging, p.stream));
  SPH_TRY(upload_group(p, g2, 1, device, p.staging, p.stream));   // reuses the staging buffer after the first transposes
  return SPHGPU_OK;
}

// SoA fields -> AoS host arrays: transpose into the staging buffer, then the
// device-to-host copies back to back; one synchronisation at the end.
int download_group(Problem& p, const double* base, const AosField* f, int nf) {
  int64_t off = 0;
  int64_t at[6];
  for (int k = 0; k < nf; ++k) {
    at[k] = off;
    if (f[k].host == nullptr) continue;
    const int64_t cnt = p.n*f[k].comps;
    soa_to_aos_kernel<<<grid1(cnt), 256, 0, p.stream>>>(base + (int64_t)f[k].field*p.n, f[k].comps, p.n,
                                                        p.staging + off);
    ++p.launches;
    off += cnt;
  }
  SPH_CHECK(cudaGetLastError());
  for (int k = 0; k < nf; ++k) {
    if (f[k].host == nullptr) continue;
    SPH_CHECK(cudaMemcpyAsync(const_cast<double*>(f[k].host), p.staging + at[k],
                              sizeof(double)*(size_t)(p.n*f[k].comps), cudaMemcpyDeviceToHost, p.stream));
  }
  return SPHGPU_OK;
}

int download_aos(Problem& p, const double* base, int comps, int field, double* host) {
  if (host == nullptr) return SPHGPU_OK;
  const AosField f[1] = {{host, comps, field}};
  SPH_TRY(download_group(p, base, f, 1));
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  return SPHGPU_OK;
}

// Every member's device error word; reports and clears the words that are set.
int batch_check_errors(Batch& b, const char* where) {
  const int slot = -1;
  std::vector<double> errs;
  SPH_TRY(batch_gather(b, &slot, 1, errs));
  int rc = SPHGPU_OK;
  std::string msg;
  for (size_t m = 0; m < b.mem.size(); ++m) {
    const int herr = (int)errs[m];
    if (herr == 0) continue;
    cudaMemsetAsync(b.mem[m]->d_err, 0, sizeof(int), b.stream);
    msg = std::string(where) + ":";
    if (b.mem.size() > 1) msg += " member " + std::to_string(m) + ":";
    int r = SPHGPU_ERR_NUMERIC;
    if (herr & DERR_NBR_CAPACITY) { msg += " neighbor capacity exceeded;"; r = SPHGPU_ERR_CAPACITY; }
    if (herr & DERR_GHOST_CHAIN) { msg += " ghost imaged twice on one axis;"; r = SPHGPU_ERR_UNSUPPORTED; }
    if (herr & DERR_NONPOSITIVE) { msg += " non-positive mass/density/det(H) or non-finite state;"; r = SPHGPU_ERR_NUMERIC; }
    if (herr & DERR_BARRIER) {
      msg += " a grid barrier of the fused ghost passes timed out;";
      r = SPHGPU_ERR_CUDA;
      if (b.d_fuse) cudaMemsetAsync(b.d_fuse, 0, 2*sizeof(unsigned int), b.stream);
    }
    if (rc == SPHGPU_OK) rc = r;
  }
  if (rc != SPHGPU_OK) {
    cudaStreamSynchronize(b.stream);
    set_error(msg);
  }
  return rc;
}

// initializeProblemStartup after new state: omega = 1, P and cs from the
// EOS, the state checked, the restart copies of the compatible energy.
int startup_after_upload(Problem& p, const char* where) {
  fill_kernel<<<grid1(p.n), 256, 0, p.stream>>>(p.S + (int64_t)S_OMEGA*p.n, p.n, 1.0); ++p.launches;
  SPH_TRY(launch_eos(solo(&p)));
  check_state_kernel<<<grid1(p.n), 256, 0, p.stream>>>(p.S, p.n, p.d_err); ++p.launches;
  startup_restart_kernel<<<grid1(p.n), 256, 0, p.stream>>>(p.S, p.S0, p.n, p.cfg.gamma,
                                                           p.cfg.compatibleEnergyEvolution); ++p.launches;
  SPH_CHECK(cudaGetLastError());
  return batch_check_errors(solo(&p), where);
}

int set_state_impl(Problem& p, const double* pos, const double* vel, const double* mass, const double* rho,
                   const double* eps, const double* H, bool device) {
  SPH_TRY(upload_state(p, pos, vel, mass, rho, eps, H, device));
  SPH_TRY(startup_after_upload(p, "set_state"));
  p.haveNbrs = false;
  p.crkVolumeReady = false;
  p.omegaResetByStep = false;
  return SPHGPU_OK;
}

bool anyMember(const Batch& b, bool (*pred)(const Problem&)) {
  for (const Problem* p : b.mem) if (pred(*p)) return true;
  return false;
}
bool isCrkP(const Problem& p) { return p.prm.hydro == SPHGPU_HYDRO_CRKSPH; }
bool needsStartupVolume(const Problem& p) { return isCrkP(p) && !p.crkVolumeReady; }
bool isMixedSph(const Problem& p) { return !isCrkP(p) && p.cfg.precision == SPHGPU_PRECISION_MIXED; }
bool isMixedCrk(const Problem& p) { return isCrkP(p) && p.cfg.precision == SPHGPU_PRECISION_MIXED; }
bool hasGradh(const Problem& p) { return !isCrkP(p) && p.prm.gradh; }

// CRKSPH volume (CRKSumVolume or mass/density) of the CRKSPH members;
// `startupOnly` restricts it to members that have none yet.
int crk_volume(Batch& b, bool startupOnly) {
  SPH_TRY(launch_crk_sum_volume(b, startupOnly));
  SPH_TRY(launch_crk_volume_from_density(b, startupOnly));
  return SPHGPU_OK;
}

// Ghosts and connectivity of every member (Integrator::setGhostNodes +
// ConnectivityMap::computeConnectivity), then the CRKSPH start-up volume
// (CRKSPHHydroBase::initializeProblemStartup, src/CRKSPH/CRKSPHHydroBase.cc:279-300).
int build_neighbors_impl(Batch& b) {
  SPH_TRY(build_connectivity(b));
  for (Problem* p : b.mem) p->haveNbrs = true;
  if (anyMember(b, isCrkP)) {
    SPH_TRY(crk_prepare(b));
    if (anyMember(b, needsStartupVolume)) {
      SPH_TRY(pack_records(b));
      SPH_TRY(crk_volume(b, true));
      for (Problem* p : b.mem) if (isCrkP(*p)) p->crkVolumeReady = true;
    }
  }
  return SPHGPU_OK;
}

// Physics::initialize: grad-h (SPH) or the CRKSPH moments and corrections.
int initialize_impl(Batch& b) {
  // ArtificialViscosity::initialize: the Balsara shear correction from the
  // last evaluation's velocity gradient (before the derivatives are zeroed)
  if (anyMember(b, [](const Problem& p) { return p.prm.balsara != 0; })) SPH_TRY(launch_balsara(b));
  if (anyMember(b, isCrkP)) {
    SPH_TRY(crk_prepare(b));
    SPH_TRY(launch_crk_initialize(b));
  }
  if (anyMember(b, hasGradh)) {
    SPH_TRY(launch_gradh(b));
    SPH_TRY(pack_records(b, PACK_FOR_EVAL));
  }
  return cuda_status(cudaGetLastError(), "initialize");
}

// After an initialize outside an RK2 step: the restart-file state the
// reference's State then holds (Problem::Kheld, Problem::omegaResetByStep).
int hold_restart_state(Batch& b) {
  for (Problem* p : b.mem) {
    p->omegaResetByStep = false;
    if (!isCrkP(*p) || p->K == nullptr) continue;
    const size_t bytes = sizeof(double)*K_M0*(size_t)p->n;
    if (p->Kheld == nullptr && dev_alloc(reinterpret_cast<void**>(&p->Kheld), bytes) != cudaSuccess) {
      set_error("CRKSPH correction copy allocation failed");
      return SPHGPU_ERR_NOMEM;
    }
    SPH_CHECK(cudaMemcpyAsync(p->Kheld, p->K, bytes, cudaMemcpyDeviceToDevice, b.stream));
  }
  return SPHGPU_OK;
}

// Physics::finalize: CRK volumes then the summed density, or the SPH sum.
// enforce: the step's enforceBoundaries follows; the summed-density
// kernels apply it to their members
int finalize_impl(Batch& b, bool enforce) {
  if (anyMember(b, isCrkP)) {
    SPH_TRY(crk_volume(b, false));
    SPH_TRY(launch_crk_sum_density(b));
  }
  SPH_TRY(launch_sum_density(b, enforce));
  if (anyMember(b, isMixedSph)) SPH_TRY(launch_sum_density_mixed(b, enforce));
  return SPHGPU_OK;
}

int require_nbrs(Batch& b) {
  for (Problem* p : b.mem)
    if (!p->haveNbrs) { set_error("connectivity not built (call sphgpu_build_neighbors)"); return SPHGPU_ERR_STATE; }
  return SPHGPU_OK;
}

int launch_eval(Batch& b) {
  for (Problem* p : b.mem) p->paccReady = p->pacc != nullptr;
  if (anyMember(b, isCrkP)) {
    SPH_TRY(crk_prepare(b));
    SPH_TRY(launch_crk_eval(b));
    if (anyMember(b, isMixedCrk)) {
      SPH_TRY(prepare_mixed(b));
      SPH_TRY(launch_crk_eval_mixed(b));
    }
  }
  if (anyMember(b, isMixedSph)) {
    SPH_TRY(prepare_mixed(b));
    SPH_TRY(launch_eval_sph_mixed(b));
  }
  SPH_TRY(launch_eval_sph_fp64(b));
  return cuda_status(cudaGetLastError(), "evaluate");
}

// CheapSynchronousRK2::step for every member, each with its own dt.
// The part of the step after the connectivity: no host synchronisation and
// no allocation, so it can be captured as a CUDA graph.
int step_after_connectivity(Batch& b) {
  // selectDt with the previous derivatives, state at the step start
  // (reads the state and derivatives directly: no records needed yet).
  SPH_TRY(launch_select_dt(b));
  if (anyMember(b, isMixedSph)) SPH_TRY(prepare_mixed(b));   // the update writes mixed records
  // state0 = state; trial advance to the mid point (updateAsIncrement for
  // every policy) and the internal nodes' pair records, one kernel; the
  // record passes then cover the ghosts (and the members the update does
  // not pack)
  SPH_TRY(launch_update(b, 0.5, true, 1, PACK_FOR_EVAL, true));
  SPH_TRY(pack_records(b, PACK_FOR_EVAL));
  // initializeDerivatives + derivs.Zero + evaluateDerivatives at the mid point
  SPH_TRY(initialize_impl(b));
  SPH_TRY(launch_eval(b));
  // full step from state0 with the mid-point derivatives (the restore of
  // state0 and the compatible energy are folded into the update kernel),
  // with the records of the summed density
  SPH_TRY(launch_update(b, 1.0, false, 2, PACK_FOR_FINALIZE, true));
  // applyGhostBoundaries; postStepFinalize (sum density); enforceBoundaries
  SPH_TRY(pack_records(b, PACK_FOR_FINALIZE));
  SPH_TRY(finalize_impl(b, true));
  b.packedByUpdate = 0;
  SPH_TRY(launch_enforce_boundaries(b, true));
  SPH_TRY(launch_finish_step(b));
  return SPHGPU_OK;
}

// A key of everything the captured graph depends on: buffer addresses and
// capacities, sizes fixed per problem, the schedules.
uint64_t graph_key(const Batch& b) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](uint64_t v) { h ^= v; h *= 1099511628211ULL; };
  mix(b.mem.size());
  mix((uint64_t)b.evalThreads);
  for (const Problem* p : b.mem) {
    const void* ptrs[] = {p->S, p->S0, p->D, p->K, p->qgrad, p->fshear, p->rec, p->crec, p->mrec, p->groot, p->gcode,
                          p->gpos, p->cand, p->cidx, p->sortedIdx, p->cellStart, p->cellFill, p->counts,
                          p->offsets, p->nbr, p->pacc, p->tableCoef, p->coefF, p->blockSums, p->d_scal,
                          p->d_red, p->d_err, p->hmaxi, p};
    for (const void* q : ptrs) mix((uint64_t)(uintptr_t)q);
    // sizes and plans that set launch shapes, kernel variants and shared memory
    const int64_t sizes[] = {p->n, p->gcap, p->ecap, p->candcap, p->cellcap, p->reccap, p->creccap,
                             p->mreccap, p->blockSumsCap, p->redcap, p->maxNbr, p->fillCap, p->fillSchedule,
                             p->grid.sub, p->grid.stashCap, p->grid.stashStride};
    for (int64_t v : sizes) mix((uint64_t)v);
  }
  return h;
}

int enable_graph(Batch& b) {
  if (b.sideStream == nullptr) SPH_CHECK(cudaStreamCreateWithFlags(&b.sideStream, cudaStreamNonBlocking));
  if (b.memGraphEvent == nullptr) SPH_CHECK(cudaEventCreateWithFlags(&b.memGraphEvent, cudaEventDisableTiming));
  if (b.d_mapArena == nullptr) {
    b.mapArenaCap = 1 << 18;
    SPH_CHECK(dev_alloc(reinterpret_cast<void**>(&b.d_mapArena), sizeof(int32_t)*b.mapArenaCap));
  }
  return SPHGPU_OK;
}

// Descriptors of this step into the slot the captured graph reads.
int upload_graph_descriptors(Batch& b) {
  const int nm = (int)b.mem.size();
  if (nm > b.memGraphCap) {
    cudaStreamSynchronize(b.stream);
    dev_free(b.d_memGraph); cudaFreeHost(b.h_memGraph);
    b.d_memGraph = nullptr; b.h_memGraph = nullptr;
    b.memGraphCap = nm + 16;
    if (dev_alloc(reinterpret_cast<void**>(&b.d_memGraph), sizeof(Member)*b.memGraphCap) != cudaSuccess ||
        cudaMallocHost(&b.h_memGraph, sizeof(Member)*b.memGraphCap) != cudaSuccess) {
      b.memGraphCap = 0;
      set_error("graph descriptor allocation failed");
      return SPHGPU_ERR_NOMEM;
    }
  }
  SPH_CHECK(cudaEventSynchronize(b.memGraphEvent));
  for (int m = 0; m < nm; ++m) b.h_memGraph[m] = describe_member(*b.mem[m]);
  SPH_CHECK(cudaMemcpyAsync(b.d_memGraph, b.h_memGraph, sizeof(Member)*nm, cudaMemcpyHostToDevice, b.stream));
  SPH_CHECK(cudaEventRecord(b.memGraphEvent, b.stream));
  b.d_mem = b.d_memGraph;
  b.memDirty = false;
  return SPHGPU_OK;
}

// Capture of one whole RK2 step, rebuild included, as a CUDA graph:
//   [open] -> IF(no error so far) { ghosts + ConnectivityMap launches }
//   -> [gate] -> IF(no error) { dt vote, mid-point update, records,
//   initialize, derivatives, full update with the compatible energy,
//   finalize, boundaries, step bookkeeping }
// The build is sized on the device and checks its capacities there; the gate
// turns the rest of the step off (a conditional graph node) when a capacity
// overflowed, so the state is left as it was, and the open kernel of every
// later replay of the same call turns that replay off, rebuild included.  The
// host redoes the overflowing step eagerly, with grown buffers, after the
// call's one read-back.  Any other error bit (set by a build or by a step)
// stops the replays the same way, and the call reports it.
__global__ void step_gate_kernel(const Member* mem, int nmem, cudaGraphConditionalHandle handle) {
  int bad = 0;
  for (int m = threadIdx.x; m < nmem; m += blockDim.x) bad |= *mem[m].err != 0;
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) cudaGraphSetConditional(handle, bad ? 0u : 1u);
}

// Per member: the device time from the host's, the step and pair counters zeroed.
__global__ void step_counters_kernel(const Member* mem, int nmem, const double* times) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  double* s = mem[m].scal;
  s[SC_TIME] = times[m];
  reinterpret_cast<int64_t*>(s)[SC_STEPS] = 0;
  reinterpret_cast<int64_t*>(s)[SC_PAIRSUM] = 0;
}

namespace {
// Nodes of `g` with no dependents.
int graph_leaves(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves) {
  size_t nnodes = 0;
  SPH_CHECK(cudaGraphGetNodes(g, nullptr, &nnodes));
  std::vector<cudaGraphNode_t> nodes(nnodes);
  SPH_CHECK(cudaGraphGetNodes(g, nodes.data(), &nnodes));
  leaves.clear();
  for (cudaGraphNode_t nd : nodes) {
    size_t nout = 0;
    SPH_CHECK(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
    if (nout == 0) leaves.push_back(nd);
  }
  return SPHGPU_OK;
}

// An IF node on `handle` after every leaf of `g`; its body graph in *body.
int add_if_node(cudaGraph_t g, cudaGraphConditionalHandle handle, cudaGraphNode_t* node, cudaGraph_t* body) {
  std::vector<cudaGraphNode_t> leaves;
  SPH_TRY(graph_leaves(g, leaves));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  SPH_CHECK(cudaGraphAddNode(node, g, leaves.data(), leaves.size(), &cp));
  *body = cp.conditional.phGraph_out[0];
  return SPHGPU_OK;
}

// Launches of `fn` captured into `g` (after `dep` when given).
template <class F>
int capture_into(Batch& b, cudaGraph_t g, const cudaGraphNode_t* dep, F&& fn, const char* what) {
  cudaError_t e = cudaStreamBeginCaptureToGraph(b.stream, g, dep, nullptr, dep ? 1 : 0,
                                                cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return cuda_status(e, what);
  const int rc = fn();
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(b.stream, &captured);
  if (rc != SPHGPU_OK) return rc;
  return e == cudaSuccess ? SPHGPU_OK : cuda_status(e, what);
}
}  // namespace

int capture_full_step(Batch& b) {
  if (b.graphExec) { cudaGraphExecDestroy(b.graphExec); b.graphExec = nullptr; }
  // everything the replay touches must exist before the capture
  if (anyMember(b, isCrkP)) SPH_TRY(crk_prepare(b));
  if (anyMember(b, isMixedSph) || anyMember(b, isMixedCrk)) SPH_TRY(prepare_mixed(b));
  SPH_TRY(plan_build(b));
  SPH_TRY(enable_graph(b));
  SPH_TRY(upload_graph_descriptors(b));
  b.mapArenaPos = 0;
  const int64_t l0 = b.launches;
  std::vector<int64_t> m0;
  for (Problem* p : b.mem) m0.push_back(p->launches);
  cudaGraph_t graph = nullptr;
  SPH_CHECK(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle hBuild, hStep;
  cudaError_t e = cudaGraphConditionalHandleCreate(&hBuild, graph, 0u, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hStep, graph, 0u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return cuda_status(e, "graph conditional handle"); }
  const int nm = (int)b.mem.size();
  int rc = SPHGPU_OK;
  b.capturing = true;
  b.capacityGrids = true;
  do {
    // the open kernel: no error left by an earlier replay of this call
    rc = capture_into(b, graph, nullptr, [&]() {
      step_gate_kernel<<<1, 128, 0, b.stream>>>(b.d_mem, nm, hBuild);
      batch_count_launch(b);
      return cuda_status(cudaGetLastError(), "step open");
    }, "graph capture (open)");
    if (rc != SPHGPU_OK) break;
    cudaGraphNode_t ifBuild, ifStep;
    cudaGraph_t buildBody, stepBody;
    if ((rc = add_if_node(graph, hBuild, &ifBuild, &buildBody)) != SPHGPU_OK) break;
    // the rebuild, in the first conditional's body
    const int64_t lb = b.launches;
    rc = capture_into(b, buildBody, nullptr, [&]() { return launch_build_captured(b); }, "graph capture (build)");
    if (rc != SPHGPU_OK) break;
    b.graphBuildLaunches = b.launches - lb;
    // the gate, after the first conditional
    rc = capture_into(b, graph, &ifBuild, [&]() {
      step_gate_kernel<<<1, 128, 0, b.stream>>>(b.d_mem, nm, hStep);
      batch_count_launch(b);
      return cuda_status(cudaGetLastError(), "step gate");
    }, "graph capture (gate)");
    if (rc != SPHGPU_OK) break;
    if ((rc = add_if_node(graph, hStep, &ifStep, &stepBody)) != SPHGPU_OK) break;
    // the step after the rebuild, in the second conditional's body
    rc = capture_into(b, stepBody, nullptr, [&]() { return step_after_connectivity(b); }, "graph capture (step)");
  } while (false);
  b.capturing = false;
  b.capacityGrids = false;
  // launches are counted when the graph is replayed
  b.graphLaunches = b.launches - l0;
  b.launches = l0;
  for (size_t m = 0; m < b.mem.size(); ++m) b.mem[m]->launches = m0[m];
  if (rc == SPHGPU_OK) {
    e = cudaGraphInstantiate(&b.graphExec, graph, 0);
    if (e != cudaSuccess) { b.graphExec = nullptr; rc = cuda_status(e, "graph instantiate"); }
  }
  cudaGraphDestroy(graph);
  if (rc == SPHGPU_OK) b.graphKey = graph_key(b);
  return rc;
}

// One eager CheapSynchronousRK2 step of every member (host read-backs after
// the rebuild and after the step).
int step_finish(Batch& b);

int step_impl(Batch& b) {
  // preStepInitialize: ghosts + connectivity every cycle, then ghost state.
  SPH_TRY(build_neighbors_impl(b));
  return step_finish(b);
}

// The step after the connectivity, then the host's step bookkeeping.
int step_finish(Batch& b) {
  SPH_TRY(step_after_connectivity(b));
  const int slots[2] = {SC_DT, -1};
  std::vector<double> res;
  SPH_TRY(batch_gather(b, slots, 2, res));
  for (size_t m = 0; m < b.mem.size(); ++m) {
    if ((int)res[2*m + 1] != 0) return batch_check_errors(b, "step_rk2");
  }
  for (size_t m = 0; m < b.mem.size(); ++m) {
    Problem& p = *b.mem[m];
    p.time += res[2*m];
    p.lastDt = res[2*m];
    p.cycle += 1;
    p.haveDerivs = true;
    p.omegaResetByStep = true;
    p.pairsEvaluated += p.pairs;
  }
  return SPHGPU_OK;
}

// `count` steps as replays of the captured graph with no host synchronisation
// in between, then one read-back.  *done: steps completed (fewer when a
// rebuild outgrew its buffers; the state is then the one before that step).
int run_graph_steps(Batch& b, int64_t count, int64_t* done) {
  *done = 0;
  const int nm = (int)b.mem.size();
  SPH_TRY(upload_graph_descriptors(b));
  {
    // device time from the host's, counters zeroed (one small upload)
    std::vector<double> t(nm);
    for (int m = 0; m < nm; ++m) t[m] = b.mem[m]->time;
    std::vector<double> unused;
    if ((int64_t)nm > b.gathercap) {
      const int s0 = SC_DT;
      SPH_TRY(batch_gather(b, &s0, 1, unused));      // sizes the gather buffers
    }
    SPH_CHECK(cudaMemcpyAsync(b.d_gather, t.data(), sizeof(double)*nm, cudaMemcpyHostToDevice, b.stream));
    step_counters_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm, b.d_gather);
    batch_count_launch(b);
    SPH_CHECK(cudaGetLastError());
  }
  for (int64_t s = 0; s < count; ++s) SPH_CHECK(cudaGraphLaunch(b.graphExec, b.stream));
  b.memDirty = true;     // the next eager call uploads to the rotating slots again
  const int s1[8] = {SC_STEPS, -1, SC_TIME, SC_DT, SC_G, SC_TOTAL, SC_MAXCOUNT, SC_PAIRS};
  const int s2[3] = {SC_NCELLS, SC_CELLSWANTED, SC_PAIRSUM};
  std::vector<double> r1, r2;
  SPH_TRY(batch_gather(b, s1, 8, r1));
  SPH_TRY(batch_gather(b, s2, 3, r2));
  int64_t ran = count;
  for (int m = 0; m < nm; ++m) ran = asI64(r1[8*m]) < ran ? asI64(r1[8*m]) : ran;
  // kernels run: every completed replay; the open kernel of each one that
  // stopped, and the rebuild and gate of the one that overflowed
  const int64_t launched = b.graphLaunches*ran + (ran < count ? (count - ran) + b.graphBuildLaunches + 1 : 0);
  bool overflow = false;
  for (int m = 0; m < nm; ++m) {
    Problem& p = *b.mem[m];
    const double* a = &r1[8*m];
    const int64_t steps = asI64(a[0]);
    const int herr = (int)a[1];
    p.launches += launched;
    p.time = a[2];
    if (steps > 0) {
      p.lastDt = a[3];
      p.cycle += steps;
      p.haveNbrs = true;
      p.haveDerivs = true;
      p.omegaResetByStep = true;
    }
    p.G = asI64(a[4]);
    p.ntot = p.n + p.G;
    p.E = asI64(a[5]);
    p.maxCount = asI32(a[6]);
    p.pairs = asI64(a[7]);
    p.ncells = asI64(r2[3*m]);
    p.cellsWanted = asI64(r2[3*m + 1]);
    p.pairsEvaluated += asI64(r2[3*m + 2]);
    if (herr & (DERR_GHOST_CAPACITY | DERR_ENTRY_CAPACITY | DERR_LIST_CAPACITY | DERR_NBR_CAPACITY)) overflow = true;
    else if (herr) return batch_check_errors(b, "step_rk2");
  }
  b.launches += launched;
  if (overflow) {
    // the steps from the overflowing rebuild on did nothing; the next eager
    // step replans the buffers (and reports a real neighbor-capacity error)
    for (Problem* p : b.mem) SPH_CHECK(cudaMemsetAsync(p->d_err, 0, sizeof(int), b.stream));
    b.graphCandidate = 0;
  }
  *done = ran;
  return SPHGPU_OK;
}

// nsteps CheapSynchronousRK2 steps of every member.  Eager steps unless the
// "step graph" schedule is on; then every step runs as one replay of the
// captured whole-step graph, captured once the buffer layout of an eager step
// recurs (so a batch whose membership keeps changing stays eager).
int steps_impl(Batch& b, int64_t nsteps) {
  int64_t done = 0;
  while (done < nsteps) {
    // (a CRKSPH start-up volume, after new state, is an eager step's work)
    if (!b.useGraph || anyMember(b, needsStartupVolume)) { SPH_TRY(step_impl(b)); ++done; continue; }
    const uint64_t key = graph_key(b);
    if (b.graphExec == nullptr || key != b.graphKey) {
      if (key != b.graphCandidate) {
        SPH_TRY(step_impl(b));
        b.graphCandidate = graph_key(b);
        ++done;
        continue;
      }
      SPH_TRY(capture_full_step(b));
    }
    const int64_t want = nsteps - done;
    int64_t ran = 0;
    SPH_TRY(run_graph_steps(b, want, &ran));
    done += ran;
    if (ran < want) {
      // an overflow stopped the replays: one eager step regrows the buffers
      SPH_TRY(step_impl(b));
      b.graphCandidate = graph_key(b);
      ++done;
    }
  }
  return SPHGPU_OK;
}

// One RK2 step with the state in and out of host arrays: what
// set_state + step_rk2(1) + get_state do, with the position and H copies
// first and, for SPH problems, the ghost/connectivity rebuild (which reads
// only those) queued before velocity, mass, density and energy are copied
// on the copy stream.  Same results as the three calls.  (Measured on B200
// with pinned host arrays, the copy and the rebuild do not overlap: the call
// is 0.1-0.2 ms faster than the three calls, not the rebuild's 1.2 ms.)
int step_host_impl(Problem& p, const double* const in[6], double* const out[6]) {
  for (int k = 0; k < 6; ++k) {
    if (in[k] == nullptr) { set_error("sphgpu_step_rk2_host: every input array is required"); return SPHGPU_ERR_ARG; }
  }
  if (p.copyStream == nullptr) {
    SPH_CHECK(cudaStreamCreateWithFlags(&p.copyStream, cudaStreamNonBlocking));
    SPH_CHECK(cudaEventCreateWithFlags(&p.evCopyStart, cudaEventDisableTiming));
    SPH_CHECK(cudaEventCreateWithFlags(&p.evCopyDone, cudaEventDisableTiming));
  }
  if (p.stagingB == nullptr && dev_alloc(reinterpret_cast<void**>(&p.stagingB), sizeof(double)*6*(size_t)p.n) != cudaSuccess) {
    p.stagingB = nullptr;
    set_error("sphgpu_step_rk2_host: staging allocation failed");
    return SPHGPU_ERR_NOMEM;
  }
  const bool overlap = p.cfg.hydro != SPHGPU_HYDRO_CRKSPH;
  // the copy stream starts after the position and H copies (and everything
  // queued before them on the problem's stream), so that the two groups do
  // not split the host link's bandwidth
  const AosField ga[2] = {{in[0], 3, S_X}, {in[5], 6, S_H}};
  const AosField gb[4] = {{in[1], 3, S_VX}, {in[2], 1, S_M}, {in[3], 1, S_RHO}, {in[4], 1, S_EPS}};
  SPH_TRY(upload_group(p, ga, 2, false, p.staging, p.stream, p.evCopyStart));
  SPH_CHECK(cudaStreamWaitEvent(p.copyStream, p.evCopyStart, 0));
  Batch& b = solo(&p);
  bool second = false;
  auto copySecond = [&]() {
    second = true;
    SPH_TRY(upload_group(p, gb, 4, false, p.stagingB, p.copyStream));
    return cuda_status(cudaEventRecord(p.evCopyDone, p.copyStream), "step_rk2_host (copy event)");
  };
  if (overlap) {
    // the rebuild's host-to-device traffic (its descriptors) goes first, and
    // its kernels are queued before the second copy group is issued
    SPH_TRY(plan_build(b));
    SPH_TRY(batch_upload(b));
    b.buildPlanned = true;
    b.afterBuildLaunch = copySecond;
    p.haveNbrs = false;
    const int rc = build_neighbors_impl(b);
    b.buildPlanned = false;
    b.afterBuildLaunch = nullptr;
    if (!second) SPH_TRY(copySecond());
    SPH_TRY(rc);
    SPH_CHECK(cudaStreamWaitEvent(p.stream, p.evCopyDone, 0));
    SPH_TRY(startup_after_upload(p, "step_rk2_host"));
  } else {
    // CRKSPH: the start-up volume of the build reads the whole state
    SPH_TRY(copySecond());
    SPH_CHECK(cudaStreamWaitEvent(p.stream, p.evCopyDone, 0));
    SPH_TRY(startup_after_upload(p, "step_rk2_host"));
    p.haveNbrs = false;
    p.crkVolumeReady = false;
    SPH_TRY(build_neighbors_impl(solo(&p)));
  }
  p.omegaResetByStep = false;
  SPH_TRY(step_finish(solo(&p)));
  const AosField o1[5] = {{out[0], 3, S_X}, {out[1], 3, S_VX}, {out[2], 1, S_M}, {out[3], 1, S_RHO},
                          {out[4], 1, S_EPS}};
  const AosField o2[1] = {{out[5], 6, S_H}};
  SPH_TRY(download_group(p, p.S, o1, 5));
  SPH_TRY(download_group(p, p.S, o2, 1));
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  return SPHGPU_OK;
}

int set_schedule_impl(Batch& b, int* nbrSchedule, int* nbrCells, const char* stage, int32_t schedule) {
  if (std::strcmp(stage, "neighbor cells") == 0) {
    if (schedule < 0 || schedule > 2) {
      set_error("neighbor cells is 0 (auto), 1 (cells of one kernel reach) or 2 (half a reach)");
      return SPHGPU_ERR_ARG;
    }
    *nbrCells = schedule;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor walk") == 0) {
    if (schedule < NBR_SCHEDULE_AUTO || schedule > NBR_SCHEDULE_WARP) {
      set_error("neighbor walk schedule must be 0 (auto), 1 (thread per node) or 2 (warp per node)");
      return SPHGPU_ERR_ARG;
    }
    *nbrSchedule = schedule;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "pair loop") == 0) {
    if (schedule != 64 && schedule != 128) {
      set_error("pair loop schedule is the threads per block: 64 or 128");
      return SPHGPU_ERR_ARG;
    }
    b.evalThreads = schedule;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor filter") == 0) {
    if (schedule != 0 && schedule != 1) {
      set_error("neighbor filter is 0 (exact FP64 test only) or 1 (FP32 pre-test)");
      return SPHGPU_ERR_ARG;
    }
    for (Problem* p : b.mem) p->nbrFilter = schedule != 0;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor passes") == 0) {
    if (schedule != 1 && schedule != 2) {
      set_error("neighbor passes is 1 (lists built in the counting walk when they fit) or 2 (count, then fill)");
      return SPHGPU_ERR_ARG;
    }
    for (Problem* p : b.mem) p->nbrStash = schedule == 1;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "ghost passes") == 0) {
    if (schedule < 0 || schedule > 2) {
      set_error("ghost passes is 0 (auto), 1 (launches per pass) or 2 (one cooperative launch)");
      return SPHGPU_ERR_ARG;
    }
    b.ghostPasses = schedule;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "step graph") == 0) {
    if (schedule != 0 && schedule != 1) {
      set_error("step graph is 0 (eager launches) or 1 (CUDA-graph replay)");
      return SPHGPU_ERR_ARG;
    }
    b.useGraph = schedule != 0;
    return SPHGPU_OK;
  }
  set_error(std::string("unknown schedule stage: ") + stage);
  return SPHGPU_ERR_ARG;
}

// Autotuner: every candidate schedule of a stage is run on the batch's own
// data and timed with CUDA events on the batch stream (one warm run, then the
// median of three); the fastest is kept.  All schedules give bit-identical
// results, so tuning changes speed only.  report = {neighbor schedule,
// ms thread, ms warp, pair-loop threads, ms 64, ms 128, cells per kernel
// reach, ms with half-reach cells}.
int autotune_impl(Batch& b, double* report) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SPH_CHECK(cudaEventCreate(&e0));
  SPH_CHECK(cudaEventCreate(&e1));
  auto timeit = [&](auto fn, double* ms) -> int {
    SPH_TRY(fn());
    double t[3];
    for (int r = 0; r < 3; ++r) {
      SPH_CHECK(cudaEventRecord(e0, b.stream));
      SPH_TRY(fn());
      SPH_CHECK(cudaEventRecord(e1, b.stream));
      SPH_CHECK(cudaEventSynchronize(e1));
      float f = 0.0f;
      SPH_CHECK(cudaEventElapsedTime(&f, e0, e1));
      t[r] = f;
    }
    std::sort(t, t + 3);
    *ms = t[1];
    return SPHGPU_OK;
  };
  double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int rc = SPHGPU_OK;
  do {
    // neighbor walk: thread per node vs warp per node
    const int schedules[2] = {NBR_SCHEDULE_THREAD, NBR_SCHEDULE_WARP};
    double best = 1e300;
    int bestS = NBR_SCHEDULE_AUTO;
    for (int k = 0; k < 2 && rc == SPHGPU_OK; ++k) {
      b.nbrSchedule = schedules[k];
      double ms = 0.0;
      rc = timeit([&]() { return build_neighbors_impl(b); }, &ms);
      out[1 + k] = ms;
      if (ms < best) { best = ms; bestS = schedules[k]; }
    }
    if (rc != SPHGPU_OK) break;
    b.nbrSchedule = bestS;
    out[0] = bestS;
    // cells of one kernel reach (the times above) vs half a reach
    b.nbrCells = 2;
    double ms2 = 0.0;
    if ((rc = timeit([&]() { return build_neighbors_impl(b); }, &ms2)) != SPHGPU_OK) break;
    b.nbrCells = ms2 < best ? 2 : 1;
    out[6] = b.nbrCells;
    out[7] = ms2;
    if ((rc = build_neighbors_impl(b)) != SPHGPU_OK) break;
    if ((rc = pack_records(b)) != SPHGPU_OK) break;
    if ((rc = initialize_impl(b)) != SPHGPU_OK) break;
    if ((rc = hold_restart_state(b)) != SPHGPU_OK) break;
    // pair loop: threads per block
    const int widths[2] = {64, 128};
    best = 1e300;
    int bestW = 128;
    for (int k = 0; k < 2 && rc == SPHGPU_OK; ++k) {
      b.evalThreads = widths[k];
      double ms = 0.0;
      rc = timeit([&]() { return launch_eval(b); }, &ms);
      out[4 + k] = ms;
      if (ms < best) { best = ms; bestW = widths[k]; }
    }
    b.evalThreads = bestW;
    out[3] = bestW;
  } while (false);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == SPHGPU_OK && report) for (int k = 0; k < 8; ++k) report[k] = out[k];
  return rc;
}

}  // namespace

int batch_step_rk2(Batch& b) { return batch_steps_rk2(b, 1); }

int batch_steps_rk2(Batch& b, int64_t nsteps) {
  b.memDirty = true;
  for (Problem* p : b.mem) SPH_CHECK(cudaStreamSynchronize(p->stream));
  return steps_impl(b, nsteps);
}

// Device bytes a problem holds, from its buffer capacities.
int64_t problem_bytes(const Problem& p) {
  const int64_t n = p.n;
  const int stagingComps = p.cfg.hydro == SPHGPU_HYDRO_CRKSPH ? 27 : 9;
  int64_t b = 8*(2*(int64_t)NSTATE*n + (int64_t)NDERIV*n + stagingComps*n + 2*n + NSCAL + 148*4*8) + 16;
  b += 8*(6 + 2)*(int64_t)p.prm.W.n + 4*(kWsumBins + 1);              // tables
  b += p.gcap*(4 + 4 + 24);                                           // groot, gcode, gpos
  b += p.candcap*(4 + 4 + 4 + 8*CAND_DOUBLES + 8*RECW) + 8*(p.candcap + 1);  // counts, cidx, sortedIdx, cand, rec, offsets
  b += p.ecap*(4 + (p.pacc ? 24 : 0));                                // nbr, pacc
  b += p.cellcap*(8 + 4) + 8 + 8*p.blockSumsCap;
  b += 8*(int64_t)(p.cfg.hydro == SPHGPU_HYDRO_CRKSPH ? CMRECW : MRECW)*p.mreccap +
       (p.coefF ? 4*6*(int64_t)p.prm.W.n : 0);
  b += 8*(int64_t)CRECW*p.creccap + (p.K ? 8*(int64_t)NCRK*n : 0) + (p.Kheld ? 8*(int64_t)K_M0*n : 0);
  b += p.cfg.qType == SPHGPU_Q_CRKSPH_MONAGHAN_GINGOLD ? 8*(int64_t)QGRADW*n : 0;
  b += p.cfg.balsaraShearCorrection ? 8*n : 0;                        // fshear
  return b;
}

int ensure_block_sums(Problem& p, int64_t nblocks) {
  if (nblocks <= p.blockSumsCap) return SPHGPU_OK;
  dev_free(p.blockSums);
  p.blockSums = nullptr;
  p.blockSumsCap = nblocks + 64;
  return dalloc(p.blockSums, p.blockSumsCap);
}

// Ghost arrays and every (n + ghosts)-sized buffer; contents are preserved
// because the ghost build grows them between passes.
int ensure_capacity_ghosts(Problem& p, int64_t need) {
  if (need <= p.gcap && p.candcap >= p.n + need) return SPHGPU_OK;
  const int64_t ng = need + need/2 + 1024;
  const int64_t oldg = p.gcap, oldc = p.candcap;
  const int64_t nc = p.n + ng;
  // ghost arrays
  SPH_TRY(grow_preserve(p.groot, oldg, ng, p.stream));
  SPH_TRY(grow_preserve(p.gcode, oldg, ng, p.stream));
  double* np = nullptr;
  SPH_TRY(dalloc(np, 3*ng));
  if (p.gpos) {
    for (int c = 0; c < 3; ++c)
      SPH_CHECK(cudaMemcpyAsync(np + c*ng, p.gpos + c*oldg, sizeof(double)*(size_t)oldg, cudaMemcpyDeviceToDevice, p.stream));
    SPH_CHECK(cudaStreamSynchronize(p.stream));
    dev_free(p.gpos);
  }
  p.gpos = np;
  p.gcap = ng;
  // (n + ghost)-sized buffers
  SPH_TRY(grow_preserve(p.counts, oldc, nc, p.stream));
  SPH_TRY(grow_preserve(p.offsets, oldc ? oldc + 1 : 0, nc + 1, p.stream));
  SPH_TRY(grow_preserve(p.cidx, 0, nc, p.stream));
  SPH_TRY(grow_preserve(p.sortedIdx, 0, nc, p.stream));
  dev_free(p.cand);
  SPH_TRY(dalloc(p.cand, CAND_DOUBLES*nc));
  dev_free(p.rec);
  SPH_TRY(dalloc(p.rec, RECW*nc));
  p.candcap = nc;
  p.reccap = nc;
  return SPHGPU_OK;
}

int ensure_capacity_entries(Problem& p, int64_t need) {
  if (need <= p.ecap) return SPHGPU_OK;
  const int64_t ne = need + need/8 + 1024;
  void* old[] = {p.nbr, p.pacc};
  dev_free_all(old, 2);
  p.nbr = nullptr;
  p.pacc = nullptr;
  SPH_TRY(dalloc(p.nbr, ne));
  if (p.cfg.compatibleEnergyEvolution) SPH_TRY(dalloc(p.pacc, 3*ne));
  p.ecap = ne;
  return SPHGPU_OK;
}

}  // namespace sphgpu

// ================================================================== C ABI
using namespace sphgpu;

extern "C" {


const char* sphgpu_last_error(void) { return g_last_error.c_str(); }

int sphgpu_create(const sphgpu_config* cfg, int64_t n_internal, sphgpu_problem** out) {
  if (cfg == nullptr || out == nullptr || n_internal <= 0) { set_error("sphgpu_create: bad arguments"); return SPHGPU_ERR_ARG; }
  *out = nullptr;
  SPH_TRY(validate_config(*cfg));
  if (n_internal > (int64_t)1 << 30) { set_error("sphgpu_create: too many nodes"); return SPHGPU_ERR_CAPACITY; }
  sphgpu_problem* p = new (std::nothrow) sphgpu_problem();
  if (p == nullptr) { set_error("host allocation failed"); return SPHGPU_ERR_NOMEM; }
  p->cfg = *cfg;
  p->n = n_internal;
  int rc = SPHGPU_OK;
  do {
    if ((rc = cuda_status(cudaGetDevice(&p->device), "cudaGetDevice")) != SPHGPU_OK) break;
    if ((rc = cuda_status(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream")) != SPHGPU_OK) break;
    p->ownStream = true;
    int mx = cfg->max_neighbors > 0 ? cfg->max_neighbors : 1024;
    int m2 = 32;
    while (m2 < mx) m2 <<= 1;
    p->maxNbr = m2;
    // TableKernel (host construction, device tables)
    std::vector<double> coef6, nperh, wsum;
    double stepSize = 0.0, extent = 0.0;
    build_table_kernel(cfg->kernel, cfg->num_points, coef6, nperh, wsum, stepSize, extent);
    const int nt = cfg->num_points;
    if ((rc = dalloc(p->tableCoef, 6*(int64_t)nt)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->nperhTab, nt)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->wsumTab, nt)) != SPHGPU_OK) break;
    cudaMemcpy(p->tableCoef, coef6.data(), sizeof(double)*coef6.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p->nperhTab, nperh.data(), sizeof(double)*nt, cudaMemcpyHostToDevice);
    cudaMemcpy(p->wsumTab, wsum.data(), sizeof(double)*nt, cudaMemcpyHostToDevice);
    // bracket table of the Wsum bisection (ascending Wsum)
    if (nt >= 2 && wsum[nt - 1] > wsum[0]) {
      std::vector<int32_t> bins(kWsumBins + 1);
      const double w0 = wsum[0], width = (wsum[nt - 1] - wsum[0])/kWsumBins;
      int j = -1;
      for (int b = 0; b <= kWsumBins; ++b) {
        const double edge = b == kWsumBins ? wsum[nt - 1] : w0 + b*width;
        while (j + 1 < nt && wsum[j + 1] <= edge) ++j;
        bins[b] = j;
      }
      bool ascending = true;
      for (int k = 1; k < nt; ++k) ascending = ascending && wsum[k] >= wsum[k - 1];
      if (ascending) {
        if ((rc = dalloc(p->wsumBinsTab, kWsumBins + 1)) != SPHGPU_OK) break;
        cudaMemcpy(p->wsumBinsTab, bins.data(), sizeof(int32_t)*(kWsumBins + 1), cudaMemcpyHostToDevice);
        p->prm.wsumBins = p->wsumBinsTab;
        p->prm.wsumNbins = kWsumBins;
        p->prm.wsumBin0 = w0;
        p->prm.wsumBinInv = 1.0/width;
      }
    }
    Params& P = p->prm;
    P.W.coef = p->tableCoef;
    P.W.n = nt;
    P.W.stepSize = stepSize;
    P.W.extent = extent;
    P.nperh = p->nperhTab;
    P.wsum = p->wsumTab;
    P.W0 = table_kernel_value(coef6, nt, stepSize, extent, 0.0, 1.0);
    P.WnPerh = table_kernel_value(coef6, nt, stepSize, extent, 1.0/cfg->nPerh, 1.0);
    P.nPerh = cfg->nPerh; P.Cl = cfg->Cl; P.Cq = cfg->Cq; P.eps2 = cfg->epsilon2;
    P.epsTensile = cfg->epsTensile; P.gamma = cfg->gamma; P.cfl = cfg->cfl;
    P.hmin = cfg->hmin; P.hmax = cfg->hmax; P.rhoMin = cfg->rhoMin; P.rhoMax = cfg->rhoMax;
    P.kernelExtent = extent;
    P.compatible = cfg->compatibleEnergyEvolution; P.XSPH = cfg->XSPH; P.correctVelGrad = cfg->correctVelocityGradient;
    P.linearInExp = cfg->linearInExpansion; P.quadInExp = cfg->quadraticInExpansion;
    P.useVelMagDt = cfg->useVelocityMagnitudeForDt; P.HUpdate = cfg->HUpdate; P.densityUpdate = cfg->densityUpdate;
    P.gradh = cfg->gradhCorrection;
    P.hydro = cfg->hydro;
    P.qType = cfg->qType;
    P.balsara = cfg->balsaraShearCorrection != 0;
    P.precision = cfg->precision;
    P.etaCrit = cfg->etaCritFrac/cfg->nPerh;
    P.etaFold = cfg->etaFoldFrac/cfg->nPerh;
    P.dtMin = cfg->dtMin; P.dtMax = cfg->dtMax; P.dtGrowth = cfg->dtGrowth;
    // periodic planes: PeriodicBoundary(plane1 = (xmin, +e_a), plane2 = (xmax, -e_a))
    for (int a = 0; a < 3; ++a) {
      P.bcs.periodic[a] = cfg->periodic[a] ? 1 : 0;
      V3 n0{0, 0, 0}, n1{0, 0, 0};
      (&n0.x)[a] = 1.0; (&n1.x)[a] = -1.0;
      const PlaneD plane1{V3{cfg->xmin[0], cfg->xmin[1], cfg->xmin[2]}, unitVector(n0)};
      const PlaneD plane2{V3{cfg->xmax[0], cfg->xmax[1], cfg->xmax[2]}, unitVector(n1)};
      P.bcs.bc[2*a] = PlanarBC{plane1, plane2};
      P.bcs.bc[2*a + 1] = PlanarBC{plane2, plane1};
    }
    const int64_t n = p->n;
    if ((rc = dalloc(p->S, NSTATE*n)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->S0, NSTATE*n)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->D, NDERIV*n)) != SPHGPU_OK) break;
    // widest field: Tensor (9) for SPH, the third-rank grad m2 (27) for CRKSPH
    if ((rc = dalloc(p->staging, (cfg->hydro == SPHGPU_HYDRO_CRKSPH ? 27 : 9)*n)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->d_err, 4)) != SPHGPU_OK) break;
    if ((rc = dalloc(p->hmaxi, 2*n)) != SPHGPU_OK) break;
    if (cfg->balsaraShearCorrection) {
      // no correction (1) until the first initialize computes it
      if ((rc = dalloc(p->fshear, n)) != SPHGPU_OK) break;
      fill_kernel<<<grid1(n), 256>>>(p->fshear, n, 1.0); ++p->launches;
    }
    if ((rc = dalloc(p->d_scal, NSCAL)) != SPHGPU_OK) break;
    p->redcap = 148*4*8;
    if ((rc = dalloc(p->d_red, p->redcap)) != SPHGPU_OK) break;
    cudaMemset(p->d_err, 0, 4*sizeof(int));
    cudaMemset(p->D, 0, sizeof(double)*NDERIV*(size_t)n);
    cudaMemset(p->S, 0, sizeof(double)*NSTATE*(size_t)n);
    p->lastDt = cfg->lastDt;
    cudaMemset(p->d_scal, 0, sizeof(double)*NSCAL);
    cudaMemcpy(p->d_scal + SC_LASTDT, &p->lastDt, sizeof(double), cudaMemcpyHostToDevice);
    if ((rc = ensure_capacity_ghosts(*p, n/2 + 4096)) != SPHGPU_OK) break;
    p->solo = new (std::nothrow) Batch();
    if (p->solo == nullptr) { set_error("host allocation failed"); rc = SPHGPU_ERR_NOMEM; break; }
    if ((rc = batch_init(solo(p), p->stream)) != SPHGPU_OK) break;
    p->solo->mem.push_back(p);
    if ((rc = cuda_status(cudaDeviceSynchronize(), "create")) != SPHGPU_OK) break;
  } while (false);
  if (rc != SPHGPU_OK) {
    free_problem(p);
    return rc;
  }
  *out = p;
  return SPHGPU_OK;
}

void sphgpu_destroy(sphgpu_problem* p) {
  if (p == nullptr) return;
  cudaStreamSynchronize(p->stream);
  free_problem(p);
}

int sphgpu_set_state(sphgpu_problem* p, const double* position, const double* velocity, const double* mass,
                     const double* massDensity, const double* specificThermalEnergy, const double* H) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  return set_state_impl(*p, position, velocity, mass, massDensity, specificThermalEnergy, H, false);
}

int sphgpu_set_state_device(sphgpu_problem* p, const double* position, const double* velocity, const double* mass,
                            const double* massDensity, const double* specificThermalEnergy, const double* H) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  return set_state_impl(*p, position, velocity, mass, massDensity, specificThermalEnergy, H, true);
}

int sphgpu_get_state(sphgpu_problem* p, double* position, double* velocity, double* mass, double* massDensity,
                     double* specificThermalEnergy, double* H) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  const AosField g1[5] = {{position, 3, S_X}, {velocity, 3, S_VX}, {mass, 1, S_M}, {massDensity, 1, S_RHO},
                          {specificThermalEnergy, 1, S_EPS}};
  const AosField g2[1] = {{H, 6, S_H}};
  SPH_TRY(download_group(*p, p->S, g1, 5));
  SPH_TRY(download_group(*p, p->S, g2, 1));     // stream order: after the first group's copies
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return SPHGPU_OK;
}

int sphgpu_field_components(const char* key, int32_t* components) {
  const FieldSpec* f = findField(key);
  if (f == nullptr || components == nullptr) { set_error(std::string("unknown field key: ") + (key ? key : "(null)")); return SPHGPU_ERR_ARG; }
  *components = f->comps;
  return SPHGPU_OK;
}

int sphgpu_get_field(sphgpu_problem* p, const char* key, double* out, int64_t count) {
  if (p == nullptr || out == nullptr) return SPHGPU_ERR_ARG;
  const FieldSpec* f = findField(key);
  if (f == nullptr) { set_error(std::string("unknown field key: ") + (key ? key : "(null)")); return SPHGPU_ERR_ARG; }
  if (count != p->n*f->comps) { set_error("sphgpu_get_field: count mismatch"); return SPHGPU_ERR_ARG; }
  if (f->array == 2 && p->K == nullptr) { set_error("CRKSPH fields exist for CRKSPH problems only"); return SPHGPU_ERR_STATE; }
  return download_aos(*p, f->array == 0 ? p->S : (f->array == 1 ? p->D : p->K), f->comps, f->field, out);
}

int sphgpu_set_field(sphgpu_problem* p, const char* key, const double* values, int64_t count) {
  if (p == nullptr || values == nullptr) return SPHGPU_ERR_ARG;
  const FieldSpec* f = findField(key);
  if (f == nullptr) { set_error(std::string("unknown field key: ") + (key ? key : "(null)")); return SPHGPU_ERR_ARG; }
  if (count != p->n*f->comps) { set_error("sphgpu_set_field: count mismatch"); return SPHGPU_ERR_ARG; }
  const bool crk = p->cfg.hydro == SPHGPU_HYDRO_CRKSPH;
  if (f->array == 2) {
    if (!crk) { set_error("CRKSPH fields exist for CRKSPH problems only"); return SPHGPU_ERR_STATE; }
    if (p->K == nullptr) {
      if (dev_alloc(reinterpret_cast<void**>(&p->K), sizeof(double)*NCRK*(size_t)p->n) != cudaSuccess) {
        set_error("CRKSPH field allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
      SPH_CHECK(cudaMemsetAsync(p->K, 0, sizeof(double)*NCRK*(size_t)p->n, p->stream));
    }
  }
  double* base = f->array == 0 ? p->S : (f->array == 1 ? p->D : p->K);
  const int64_t cnt = count;
  SPH_CHECK(cudaMemcpyAsync(p->staging, values, sizeof(double)*(size_t)cnt, cudaMemcpyHostToDevice, p->stream));
  aos_to_soa_kernel<<<grid1(cnt), 256, 0, p->stream>>>(p->staging, f->comps, p->n, base + (int64_t)f->field*p->n);
  ++p->launches;
  SPH_CHECK(cudaGetLastError());
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  if (f->array == 1) p->haveDerivs = true;
  // a CRKSPH node volume given by the caller replaces the start-up volume
  if (f->array == 0 && f->field == S_VOL && crk) p->crkVolumeReady = true;
  return SPHGPU_OK;
}

int sphgpu_set_dt_bounds(sphgpu_problem* p, double dt_min, double dt_max) {
  if (p == nullptr || !(dt_min > 0.0) || !(dt_max >= dt_min)) {
    set_error("sphgpu_set_dt_bounds: need 0 < dt_min <= dt_max");
    return SPHGPU_ERR_ARG;
  }
  p->cfg.dtMin = dt_min;
  p->cfg.dtMax = dt_max;
  p->prm.dtMin = dt_min;
  p->prm.dtMax = dt_max;
  return SPHGPU_OK;
}

int sphgpu_build_neighbors(sphgpu_problem* p) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(build_neighbors_impl(solo(p)));
  SPH_TRY(pack_records(solo(p)));
  return batch_check_errors(solo(p), "build_neighbors");
}

int sphgpu_connectivity_size(sphgpu_problem* p, int64_t* num_ghosts, int64_t* num_entries) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  if (num_ghosts) *num_ghosts = p->G;
  if (num_entries) *num_entries = p->E;
  return SPHGPU_OK;
}

int sphgpu_get_connectivity(sphgpu_problem* p, int64_t* offsets, int32_t* neighbors, int32_t* ghost_root) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  if (offsets) SPH_CHECK(cudaMemcpyAsync(offsets, p->offsets, sizeof(int64_t)*(size_t)(p->n + 1), cudaMemcpyDeviceToHost, p->stream));
  if (neighbors && p->E) SPH_CHECK(cudaMemcpyAsync(neighbors, p->nbr, sizeof(int32_t)*(size_t)p->E, cudaMemcpyDeviceToHost, p->stream));
  if (ghost_root && p->G) SPH_CHECK(cudaMemcpyAsync(ghost_root, p->groot, sizeof(int32_t)*(size_t)p->G, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return SPHGPU_OK;
}

int sphgpu_get_pair_accelerations(sphgpu_problem* p, double* out, int64_t count) {
  if (p == nullptr || (out == nullptr && count > 0)) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  if (p->pacc == nullptr) {
    set_error("pair accelerations are kept only with compatible energy evolution");
    return SPHGPU_ERR_UNSUPPORTED;
  }
  if (!p->paccReady) {
    set_error("no derivative evaluation on the current connectivity");
    return SPHGPU_ERR_STATE;
  }
  if (count != 3*p->E) {
    set_error("pair accelerations: count must be 3 x the ConnectivityMap entries");
    return SPHGPU_ERR_ARG;
  }
  const int64_t n = p->n, E = p->E;
  std::vector<int64_t> off((size_t)n + 1);
  std::vector<int32_t> nb((size_t)E);
  std::vector<double> m((size_t)n), pa(3*(size_t)E);
  std::vector<float> paF;
  const bool mixed = p->cfg.precision == SPHGPU_PRECISION_MIXED;
  SPH_CHECK(cudaMemcpyAsync(off.data(), p->offsets, sizeof(int64_t)*(size_t)(n + 1), cudaMemcpyDeviceToHost, p->stream));
  if (E) SPH_CHECK(cudaMemcpyAsync(nb.data(), p->nbr, sizeof(int32_t)*(size_t)E, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaMemcpyAsync(m.data(), p->S + S_M*n, sizeof(double)*(size_t)n, cudaMemcpyDeviceToHost, p->stream));
  if (mixed) paF.resize(3*(size_t)E);
  for (int a = 0; a < 3 && E; ++a) {
    if (mixed)
      SPH_CHECK(cudaMemcpyAsync(paF.data() + a*E, reinterpret_cast<const float*>(p->pacc) + a*p->ecap,
                                sizeof(float)*(size_t)E, cudaMemcpyDeviceToHost, p->stream));
    else
      SPH_CHECK(cudaMemcpyAsync(pa.data() + a*E, p->pacc + a*p->ecap, sizeof(double)*(size_t)E,
                                cudaMemcpyDeviceToHost, p->stream));
  }
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  if (mixed) for (size_t t = 0; t < paF.size(); ++t) pa[t] = (double)paF[t];
  // entry k of node i's row stores the owner's pair acceleration
  // -m_other deltaDvDt; the reference's vector of node i holds that for the
  // pairs i owns and m_owner deltaDvDt for the others
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = off[i]; k < off[i + 1]; ++k) {
      const int32_t j = nb[k];
      const double s = j > (int32_t)i ? 1.0 : -(m[j]/m[i]);
      for (int a = 0; a < 3; ++a) out[3*k + a] = s == 1.0 ? pa[a*E + k] : pa[a*E + k]*s;
    }
  }
  return SPHGPU_OK;
}

int sphgpu_get_ghost_positions(sphgpu_problem* p, double* positions) {
  if (p == nullptr || (positions == nullptr && p->G > 0)) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  if (p->G == 0) return SPHGPU_OK;
  const int64_t n = p->n, G = p->G;
  std::vector<double> x(3*(size_t)n);
  std::vector<int32_t> root((size_t)G);
  std::vector<uint32_t> code((size_t)G);
  for (int a = 0; a < 3; ++a)
    SPH_CHECK(cudaMemcpyAsync(x.data() + a*n, p->S + (S_X + a)*n, sizeof(double)*(size_t)n, cudaMemcpyDeviceToHost,
                              p->stream));
  SPH_CHECK(cudaMemcpyAsync(root.data(), p->groot, sizeof(int32_t)*(size_t)G, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaMemcpyAsync(code.data(), p->gcode, sizeof(uint32_t)*(size_t)G, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  for (int64_t g = 0; g < G; ++g) {
    const int64_t r = root[g];
    const V3 q = ghostPosition(p->prm.bcs, V3{x[r], x[n + r], x[2*n + r]}, code[g]);
    positions[3*g] = q.x; positions[3*g + 1] = q.y; positions[3*g + 2] = q.z;
  }
  return SPHGPU_OK;
}

int sphgpu_initialize(sphgpu_problem* p, double time, double dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  (void)time; (void)dt;
  SPH_TRY(require_nbrs(solo(p)));
  SPH_TRY(pack_records(solo(p)));
  SPH_TRY(initialize_impl(solo(p)));
  return hold_restart_state(solo(p));
}

int sphgpu_evaluate_derivatives(sphgpu_problem* p, double time, double dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  (void)time; (void)dt;
  SPH_TRY(require_nbrs(solo(p)));
  SPH_TRY(pack_records(solo(p), PACK_FOR_EVAL));   // the mixed form packs its own records
  SPH_TRY(launch_eval(solo(p)));
  p->haveDerivs = true;
  return SPHGPU_OK;
}

int sphgpu_finalize_derivatives(sphgpu_problem* p, double time, double dt) {
  // Ghost copies of DvDt/DepsDt are read through the ghost roots; nothing to do.
  (void)time; (void)dt;
  return p == nullptr ? SPHGPU_ERR_ARG : SPHGPU_OK;
}

int sphgpu_finalize(sphgpu_problem* p, double time, double dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  (void)time; (void)dt;
  SPH_TRY(require_nbrs(solo(p)));
  SPH_TRY(pack_records(solo(p)));
  return finalize_impl(solo(p), false);
}

int sphgpu_dt(sphgpu_problem* p, double* dt_out) {
  if (p == nullptr || dt_out == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  SPH_TRY(launch_dt(solo(p), SC_DTOUT, false));
  const int slot = SC_DTOUT;
  std::vector<double> v;
  SPH_TRY(batch_gather(solo(p), &slot, 1, v));
  *dt_out = p->cfg.cfl*v[0];
  return SPHGPU_OK;
}

int sphgpu_step_rk2(sphgpu_problem* p, double* time, int64_t nsteps, double* last_dt) {
  if (p == nullptr || nsteps < 0) return SPHGPU_ERR_ARG;
  if (time) p->time = *time;
  SPH_TRY(steps_impl(solo(p), nsteps));
  if (time) *time = p->time;
  if (last_dt) *last_dt = p->lastDt;
  return SPHGPU_OK;
}

int sphgpu_step_rk2_host(sphgpu_problem* p, const double* position, const double* velocity, const double* mass,
                         const double* massDensity, const double* specificThermalEnergy, const double* H,
                         double* position_out, double* velocity_out, double* mass_out, double* massDensity_out,
                         double* specificThermalEnergy_out, double* H_out, double* time, double* last_dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  const double* const in[6] = {position, velocity, mass, massDensity, specificThermalEnergy, H};
  double* const out[6] = {position_out, velocity_out, mass_out, massDensity_out, specificThermalEnergy_out, H_out};
  if (time) p->time = *time;
  SPH_TRY(step_host_impl(*p, in, out));
  if (time) *time = p->time;
  if (last_dt) *last_dt = p->lastDt;
  return SPHGPU_OK;
}

int sphgpu_time(sphgpu_problem* p, double* time, double* last_dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  if (time) *time = p->time;
  if (last_dt) *last_dt = p->lastDt;
  return SPHGPU_OK;
}

namespace {
// Checkpoint image header; the arrays follow in this order: S, D, K (CRKSPH).
struct CheckpointHeader {
  char tag[8];                 // "SPHGPUC1"
  int64_t n;
  int32_t hydro, precision, nstate, nderiv, ncrk, haveDerivs, crkVolumeReady, pad;
  double time, lastDt;
  int64_t cycle;
};
constexpr char kCheckpointTag[8] = {'S', 'P', 'H', 'G', 'P', 'U', 'C', '1'};

int64_t checkpoint_bytes(const Problem& p) {
  const int64_t ncrk = p.cfg.hydro == SPHGPU_HYDRO_CRKSPH ? NCRK : 0;
  return (int64_t)sizeof(CheckpointHeader) + 8*p.n*((int64_t)NSTATE + NDERIV + ncrk);
}
}  // namespace

int sphgpu_iterate_ideal_h(sphgpu_problem* p, int32_t max_iterations, double tolerance, int32_t* iterations,
                           double* max_delta_h) {
  if (p == nullptr || max_iterations < 0 || !(tolerance >= 0.0)) return SPHGPU_ERR_ARG;
  Batch& b = solo(p);
  // per-node change of H: the staging buffer (free between calls), start 2*tolerance
  double* deltaH = p->staging;
  fill_kernel<<<grid1(p->n), 256, 0, b.stream>>>(deltaH, p->n, 2.0*tolerance);
  batch_count_launch(b);
  int itr = 0;
  double maxDeltaH = 2.0*tolerance;
  while (itr < max_iterations && maxDeltaH > tolerance) {
    ++itr;
    SPH_TRY(build_neighbors_impl(b));
    SPH_TRY(launch_ideal_h_iteration(b, tolerance, deltaH));
    const int slot = SC_DELTAH;
    std::vector<double> v;
    SPH_TRY(batch_gather(b, &slot, 1, v));
    maxDeltaH = v[0];
  }
  // the connectivity of the last iteration belongs to the previous H
  p->haveNbrs = false;
  p->haveDerivs = false;
  if (iterations) *iterations = itr;
  if (max_delta_h) *max_delta_h = maxDeltaH;
  return batch_check_errors(b, "iterate ideal H");
}

int sphgpu_checkpoint_size(sphgpu_problem* p, int64_t* bytes) {
  if (p == nullptr || bytes == nullptr) return SPHGPU_ERR_ARG;
  *bytes = checkpoint_bytes(*p);
  return SPHGPU_OK;
}

int sphgpu_checkpoint_save(sphgpu_problem* p, void* buffer, int64_t bytes) {
  if (p == nullptr || buffer == nullptr) return SPHGPU_ERR_ARG;
  if (bytes < checkpoint_bytes(*p)) { set_error("checkpoint buffer too small"); return SPHGPU_ERR_ARG; }
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  CheckpointHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.tag, kCheckpointTag, sizeof(h.tag));
  h.n = p->n;
  h.hydro = p->cfg.hydro;
  h.precision = p->cfg.precision;
  h.nstate = NSTATE;
  h.nderiv = NDERIV;
  h.ncrk = p->cfg.hydro == SPHGPU_HYDRO_CRKSPH ? NCRK : 0;
  h.haveDerivs = p->haveDerivs ? 1 : 0;
  h.crkVolumeReady = p->crkVolumeReady ? 1 : 0;
  h.time = p->time;
  h.lastDt = p->lastDt;
  h.cycle = p->cycle;
  char* out = static_cast<char*>(buffer);
  std::memcpy(out, &h, sizeof(h));
  double* d = reinterpret_cast<double*>(out + sizeof(h));
  SPH_CHECK(cudaMemcpy(d, p->S, sizeof(double)*NSTATE*(size_t)p->n, cudaMemcpyDeviceToHost));
  SPH_CHECK(cudaMemcpy(d + NSTATE*p->n, p->D, sizeof(double)*NDERIV*(size_t)p->n, cudaMemcpyDeviceToHost));
  if (h.ncrk) {
    if (p->K) {
      SPH_CHECK(cudaMemcpy(d + (NSTATE + NDERIV)*p->n, p->K, sizeof(double)*NCRK*(size_t)p->n,
                           cudaMemcpyDeviceToHost));
    } else {
      std::memset(d + (NSTATE + NDERIV)*p->n, 0, sizeof(double)*NCRK*(size_t)p->n);
    }
  }
  return SPHGPU_OK;
}

int sphgpu_checkpoint_load(sphgpu_problem* p, const void* buffer, int64_t bytes) {
  if (p == nullptr || buffer == nullptr) return SPHGPU_ERR_ARG;
  if (bytes < (int64_t)sizeof(CheckpointHeader)) { set_error("checkpoint image too small"); return SPHGPU_ERR_ARG; }
  CheckpointHeader h;
  std::memcpy(&h, buffer, sizeof(h));
  if (std::memcmp(h.tag, kCheckpointTag, sizeof(h.tag)) != 0) { set_error("not a checkpoint image"); return SPHGPU_ERR_ARG; }
  const int32_t ncrk = p->cfg.hydro == SPHGPU_HYDRO_CRKSPH ? NCRK : 0;
  if (h.n != p->n || h.hydro != p->cfg.hydro || h.nstate != NSTATE || h.nderiv != NDERIV || h.ncrk != ncrk) {
    set_error("checkpoint image does not match the problem (node count, hydro form or field layout)");
    return SPHGPU_ERR_ARG;
  }
  if (bytes < checkpoint_bytes(*p)) { set_error("checkpoint image truncated"); return SPHGPU_ERR_ARG; }
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  const double* d = reinterpret_cast<const double*>(static_cast<const char*>(buffer) + sizeof(h));
  SPH_CHECK(cudaMemcpy(p->S, d, sizeof(double)*NSTATE*(size_t)p->n, cudaMemcpyHostToDevice));
  SPH_CHECK(cudaMemcpy(p->D, d + NSTATE*p->n, sizeof(double)*NDERIV*(size_t)p->n, cudaMemcpyHostToDevice));
  if (ncrk) {
    if (p->K == nullptr && dev_alloc(reinterpret_cast<void**>(&p->K), sizeof(double)*NCRK*(size_t)p->n) != cudaSuccess) {
      p->K = nullptr;
      set_error("CRKSPH field allocation failed");
      return SPHGPU_ERR_NOMEM;
    }
    SPH_CHECK(cudaMemcpy(p->K, d + (NSTATE + NDERIV)*p->n, sizeof(double)*NCRK*(size_t)p->n,
                         cudaMemcpyHostToDevice));
  }
  p->time = h.time;
  p->lastDt = h.lastDt;
  p->cycle = h.cycle;
  p->haveDerivs = h.haveDerivs != 0;
  p->crkVolumeReady = h.crkVolumeReady != 0;
  p->haveNbrs = false;
  SPH_CHECK(cudaMemcpy(p->d_scal + SC_LASTDT, &p->lastDt, sizeof(double), cudaMemcpyHostToDevice));
  solo(p).memDirty = true;
  return SPHGPU_OK;
}

int sphgpu_conservation(sphgpu_problem* p, double out[8]) {
  if (p == nullptr || out == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(launch_conservation(solo(p)));
  const int slots[8] = {SC_CONS, SC_CONS + 1, SC_CONS + 2, SC_CONS + 3, SC_CONS + 4, SC_CONS + 5, SC_CONS + 6,
                        SC_CONS + 7};
  std::vector<double> v;
  SPH_TRY(batch_gather(solo(p), slots, 8, v));
  for (int c = 0; c < 8; ++c) out[c] = v[c];
  return SPHGPU_OK;
}

int sphgpu_num_pairs(sphgpu_problem* p, int64_t* pairs) {
  if (p == nullptr || pairs == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(solo(p)));
  *pairs = p->pairs;
  return SPHGPU_OK;
}

int sphgpu_pairs_evaluated(sphgpu_problem* p, int64_t* pairs) {
  if (p == nullptr || pairs == nullptr) return SPHGPU_ERR_ARG;
  *pairs = p->pairsEvaluated;
  return SPHGPU_OK;
}

int sphgpu_kernel_launches(sphgpu_problem* p, int64_t* launches) {
  if (p == nullptr || launches == nullptr) return SPHGPU_ERR_ARG;
  *launches = p->launches;
  return SPHGPU_OK;
}

int sphgpu_set_schedule(sphgpu_problem* p, const char* stage, int32_t schedule) {
  if (p == nullptr || stage == nullptr) return SPHGPU_ERR_ARG;
  return set_schedule_impl(*p->solo, &p->nbrSchedule, &p->nbrCells, stage, schedule);
}

int sphgpu_get_schedule(sphgpu_problem* p, const char* stage, int32_t* schedule) {
  if (p == nullptr || stage == nullptr || schedule == nullptr) return SPHGPU_ERR_ARG;
  if (std::strcmp(stage, "neighbor walk") == 0) {
    *schedule = p->lastNbrSchedule;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "pair loop") == 0) {
    *schedule = p->solo->evalThreads;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "step graph") == 0) {
    *schedule = p->solo->useGraph ? 1 : 0;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "ghost passes") == 0) {
    *schedule = p->solo->lastGhostPasses;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor passes") == 0) {
    *schedule = p->lastNbrPasses;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor cells") == 0) {
    *schedule = p->lastNbrCells;
    return SPHGPU_OK;
  }
  if (std::strcmp(stage, "neighbor filter") == 0) {
    *schedule = p->nbrFilter ? 1 : 0;
    return SPHGPU_OK;
  }
  set_error(std::string("unknown schedule stage: ") + stage);
  return SPHGPU_ERR_ARG;
}

int sphgpu_autotune(sphgpu_problem* p, double report[8]) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  return autotune_impl(solo(p), report);
}

int sphgpu_synchronize(sphgpu_problem* p) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return batch_check_errors(solo(p), "synchronize");
}

int sphgpu_get_stream(sphgpu_problem* p, void** stream) {
  if (p == nullptr || stream == nullptr) return SPHGPU_ERR_ARG;
  *stream = (void*)p->stream;
  return SPHGPU_OK;
}

int sphgpu_set_stream(sphgpu_problem* p, void* stream) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  if (p->ownStream) cudaStreamDestroy(p->stream);
  p->stream = (cudaStream_t)stream;
  p->ownStream = false;
  p->solo->stream = p->stream;
  return SPHGPU_OK;
}

// ---------------------------------------------------------------- batches

namespace {

// A member may have pending work on its own stream: order the batch after it.
int batch_begin(Batch& b) {
  // members' buffers may have moved under their own calls since the last upload
  b.memDirty = true;
  b.packedByUpdate = 0;
  b.midInS0 = false;
  for (Problem* p : b.mem) SPH_CHECK(cudaStreamSynchronize(p->stream));
  return SPHGPU_OK;
}

}  // namespace

int sphgpu_batch_create(sphgpu_problem* const* members, int32_t count, sphgpu_batch** out) {
  if (members == nullptr || out == nullptr || count <= 0) { set_error("sphgpu_batch_create: bad arguments"); return SPHGPU_ERR_ARG; }
  *out = nullptr;
  int dev = 0;
  SPH_CHECK(cudaGetDevice(&dev));
  for (int32_t m = 0; m < count; ++m) {
    if (members[m] == nullptr) { set_error("sphgpu_batch_create: null member"); return SPHGPU_ERR_ARG; }
    if (members[m]->device != dev) { set_error("sphgpu_batch_create: members must live on the current device"); return SPHGPU_ERR_ARG; }
    for (int32_t k = 0; k < m; ++k)
      if (members[k] == members[m]) { set_error("sphgpu_batch_create: a problem appears twice"); return SPHGPU_ERR_ARG; }
  }
  sphgpu_batch* b = new (std::nothrow) sphgpu_batch();
  if (b == nullptr) { set_error("host allocation failed"); return SPHGPU_ERR_NOMEM; }
  cudaStream_t st = nullptr;
  int rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "batch stream");
  if (rc == SPHGPU_OK) {
    b->ownStream = true;
    rc = batch_init(*b, st);
    b->ownStream = true;
  }
  if (rc != SPHGPU_OK) {
    if (st && !b->stream) cudaStreamDestroy(st);
    batch_free(*b);
    delete b;
    return rc;
  }
  for (int32_t m = 0; m < count; ++m) b->mem.push_back(members[m]);
  b->memDirty = true;
  *out = b;
  return SPHGPU_OK;
}

void sphgpu_batch_destroy(sphgpu_batch* b) {
  if (b == nullptr) return;
  batch_free(*b);
  delete b;
}

int sphgpu_batch_size(sphgpu_batch* b, int32_t* count) {
  if (b == nullptr || count == nullptr) return SPHGPU_ERR_ARG;
  *count = (int32_t)b->mem.size();
  return SPHGPU_OK;
}

int sphgpu_batch_build_neighbors(sphgpu_batch* b) {
  if (b == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(batch_begin(*b));
  SPH_TRY(build_neighbors_impl(*b));
  SPH_TRY(pack_records(*b));
  return batch_check_errors(*b, "batch build_neighbors");
}

int sphgpu_batch_evaluate_derivatives(sphgpu_batch* b) {
  if (b == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(batch_begin(*b));
  SPH_TRY(require_nbrs(*b));
  SPH_TRY(pack_records(*b));
  SPH_TRY(initialize_impl(*b));
  SPH_TRY(hold_restart_state(*b));
  SPH_TRY(launch_eval(*b));
  for (Problem* p : b->mem) p->haveDerivs = true;
  return batch_check_errors(*b, "batch evaluate_derivatives");
}

int sphgpu_batch_step_rk2(sphgpu_batch* b, int64_t nsteps) {
  if (b == nullptr || nsteps < 0) return SPHGPU_ERR_ARG;
  SPH_TRY(batch_begin(*b));
  SPH_TRY(steps_impl(*b, nsteps));
  return SPHGPU_OK;
}

int sphgpu_batch_pairs(sphgpu_batch* b, int64_t* pairs) {
  if (b == nullptr || pairs == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(*b));
  int64_t t = 0;
  for (Problem* p : b->mem) t += p->pairs;
  *pairs = t;
  return SPHGPU_OK;
}

int sphgpu_batch_pairs_evaluated(sphgpu_batch* b, int64_t* pairs) {
  if (b == nullptr || pairs == nullptr) return SPHGPU_ERR_ARG;
  int64_t t = 0;
  for (Problem* p : b->mem) t += p->pairsEvaluated;
  *pairs = t;
  return SPHGPU_OK;
}

int sphgpu_batch_kernel_launches(sphgpu_batch* b, int64_t* launches) {
  if (b == nullptr || launches == nullptr) return SPHGPU_ERR_ARG;
  *launches = b->launches;
  return SPHGPU_OK;
}

int sphgpu_batch_set_schedule(sphgpu_batch* b, const char* stage, int32_t schedule) {
  if (b == nullptr || stage == nullptr) return SPHGPU_ERR_ARG;
  return set_schedule_impl(*b, &b->nbrSchedule, &b->nbrCells, stage, schedule);
}

int sphgpu_batch_autotune(sphgpu_batch* b, double report[8]) {
  if (b == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(batch_begin(*b));
  return autotune_impl(*b, report);
}

int sphgpu_batch_get_stream(sphgpu_batch* b, void** stream) {
  if (b == nullptr || stream == nullptr) return SPHGPU_ERR_ARG;
  *stream = (void*)b->stream;
  return SPHGPU_OK;
}

}  // extern "C"
