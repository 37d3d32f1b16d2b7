// C-ABI of the B200 SPH hydro path and the host-side orchestration of one
// CheapSynchronousRK2 step (src/Integrator/CheapSynchronousRK2.cc:81-143).
//
// All device work of a problem is issued on the problem's stream.  Each call
// returns SPHGPU_OK or a negative status (no exceptions cross the ABI); the
// text of the last failure is kept per host thread.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "problem.cuh"
#include "scan.cuh"
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

namespace {

template<typename T>
int dalloc(T*& ptr, int64_t count) {
  ptr = nullptr;
  if (count <= 0) count = 1;
  const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), sizeof(T)*(size_t)count);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_status(e, "cudaMalloc");
  }
  return SPHGPU_OK;
}

template<typename T>
int grow_preserve(T*& ptr, int64_t oldCount, int64_t newCount, cudaStream_t st) {
  T* np = nullptr;
  SPH_TRY(dalloc(np, newCount));
  if (ptr != nullptr && oldCount > 0) {
    const cudaError_t e = cudaMemcpyAsync(np, ptr, sizeof(T)*(size_t)oldCount, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) { cudaFree(np); return cuda_status(e, "grow copy"); }
  }
  cudaStreamSynchronize(st);
  cudaFree(ptr);
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
    {"internal velocity gradient", 1, D_LDVDX, 9},
    {"M SPH gradient correction", 1, D_M, 9},
    {"local M SPH gradient correction", 1, D_LM, 9},
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

int check_device_error(Problem& p, const char* where) {
  int herr = 0;
  SPH_CHECK(cudaMemcpyAsync(&herr, p.d_err, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  if (herr == 0) return SPHGPU_OK;
  cudaMemsetAsync(p.d_err, 0, sizeof(int), p.stream);
  std::string msg = std::string(where) + ":";
  int rc = SPHGPU_ERR_NUMERIC;
  if (herr & DERR_NBR_CAPACITY) { msg += " neighbor capacity exceeded;"; rc = SPHGPU_ERR_CAPACITY; }
  if (herr & DERR_GHOST_CHAIN) { msg += " ghost imaged twice on one axis;"; rc = SPHGPU_ERR_UNSUPPORTED; }
  if (herr & DERR_H_CLAMP) { msg += " H eigenvalue clamp (hmin/hmax) would be active;"; rc = SPHGPU_ERR_UNSUPPORTED; }
  if (herr & DERR_NONPOSITIVE) { msg += " non-positive mass/density/det(H) or non-finite state;"; rc = SPHGPU_ERR_NUMERIC; }
  set_error(msg);
  return rc;
}

int validate_config(const sphgpu_config& c) {
  if (c.hydro != SPHGPU_HYDRO_SPH && c.hydro != SPHGPU_HYDRO_CRKSPH) { set_error("unknown hydro"); return SPHGPU_ERR_ARG; }
  if (c.hydro == SPHGPU_HYDRO_CRKSPH && c.precision != SPHGPU_PRECISION_FP64) {
    set_error("CRKSPH runs in the plain FP64 form only"); return SPHGPU_ERR_UNSUPPORTED;
  }
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
  return SPHGPU_OK;
}

void free_problem(Problem* p) {
  if (p == nullptr) return;
  void* ptrs[] = {p->S, p->S0, p->D, p->rec, p->groot, p->gcode, p->gpos, p->cand, p->cidx, p->sortedIdx,
                  p->cellStart, p->cellFill, p->counts, p->offsets, p->nbr, p->pacc, p->tableCoef, p->nperhTab,
                  p->wsumTab, p->blockSums, p->d_err, p->d_scal, p->d_red, p->staging, p->coefF, p->mrec, p->K, p->crec};
  for (void* q : ptrs) if (q) cudaFree(q);
  if (p->pinned) cudaFreeHost(p->pinned);
  if (p->ownStream && p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

// AoS host array -> SoA fields of S (via the device staging buffer).
int upload_aos(Problem& p, const double* host, int comps, int field, bool device) {
  if (host == nullptr) return SPHGPU_OK;
  const int64_t cnt = p.n*comps;
  const double* src = host;
  if (!device) {
    SPH_CHECK(cudaMemcpyAsync(p.staging, host, sizeof(double)*(size_t)cnt, cudaMemcpyHostToDevice, p.stream));
    src = p.staging;
  }
  aos_to_soa_kernel<<<grid1(cnt), 256, 0, p.stream>>>(src, comps, p.n, p.S + (int64_t)field*p.n); ++p.launches;
  SPH_CHECK(cudaGetLastError());
  if (!device) SPH_CHECK(cudaStreamSynchronize(p.stream));
  return SPHGPU_OK;
}

int download_aos(Problem& p, const double* base, int comps, int field, double* host) {
  if (host == nullptr) return SPHGPU_OK;
  const int64_t cnt = p.n*comps;
  soa_to_aos_kernel<<<grid1(cnt), 256, 0, p.stream>>>(base + (int64_t)field*p.n, comps, p.n, p.staging); ++p.launches;
  SPH_CHECK(cudaGetLastError());
  SPH_CHECK(cudaMemcpyAsync(host, p.staging, sizeof(double)*(size_t)cnt, cudaMemcpyDeviceToHost, p.stream));
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  return SPHGPU_OK;
}

int set_state_impl(Problem& p, const double* pos, const double* vel, const double* mass, const double* rho,
                   const double* eps, const double* H, bool device) {
  SPH_TRY(upload_aos(p, pos, 3, S_X, device));
  SPH_TRY(upload_aos(p, vel, 3, S_VX, device));
  SPH_TRY(upload_aos(p, mass, 1, S_M, device));
  SPH_TRY(upload_aos(p, rho, 1, S_RHO, device));
  SPH_TRY(upload_aos(p, eps, 1, S_EPS, device));
  SPH_TRY(upload_aos(p, H, 6, S_H, device));
  // initializeProblemStartup: omega = 1, P and cs from the EOS.
  fill_kernel<<<grid1(p.n), 256, 0, p.stream>>>(p.S + (int64_t)S_OMEGA*p.n, p.n, 1.0); ++p.launches;
  launch_eos(p);
  check_state_kernel<<<grid1(p.n), 256, 0, p.stream>>>(p.S, p.n, p.d_err); ++p.launches;
  SPH_CHECK(cudaGetLastError());
  SPH_TRY(check_device_error(p, "set_state"));
  p.haveNbrs = false;
  p.crkVolumeReady = false;
  return SPHGPU_OK;
}

// CRKSPH volume: CRKSumVolume or mass/density (records must be packed).
void crk_volume(Problem& p) {
  if (p.cfg.crkVolumeType == SPHGPU_CRK_SUMVOLUME) launch_crk_sum_volume(p);
  else launch_crk_volume_from_density(p);
}

int build_neighbors_impl(Problem& p) {
  SPH_TRY(build_ghosts(p));
  SPH_TRY(build_cells_and_csr(p));
  SPH_TRY(check_device_error(p, "build_neighbors"));
  p.haveNbrs = true;
  if (p.prm.hydro == SPHGPU_HYDRO_CRKSPH) {
    SPH_TRY(crk_prepare(p));
    if (!p.crkVolumeReady) {
      // CRKSPHHydroBase::initializeProblemStartup (src/CRKSPH/CRKSPHHydroBase.cc:279-300)
      pack_records(p);
      crk_volume(p);
      p.crkVolumeReady = true;
    }
  }
  return SPHGPU_OK;
}

// Physics::initialize: grad-h (SPH) or the CRKSPH moments and corrections.
int initialize_impl(Problem& p) {
  if (p.prm.hydro == SPHGPU_HYDRO_CRKSPH) {
    SPH_TRY(crk_prepare(p));
    launch_crk_initialize(p);
  } else if (p.prm.gradh) {
    launch_gradh(p);
    pack_records(p);
  }
  return cuda_status(cudaGetLastError(), "initialize");
}

// Physics::finalize: CRK volumes then the summed density, or the SPH sum.
void finalize_impl(Problem& p) {
  if (p.prm.hydro == SPHGPU_HYDRO_CRKSPH) {
    crk_volume(p);
    if (p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM) launch_crk_sum_density(p);
  } else if (p.prm.densityUpdate == SPHGPU_DENSITY_RIGOROUS_SUM) {
    launch_sum_density(p);
  }
}

int require_nbrs(Problem& p) {
  if (!p.haveNbrs) { set_error("connectivity not built (call sphgpu_build_neighbors)"); return SPHGPU_ERR_STATE; }
  return SPHGPU_OK;
}

int launch_eval(Problem& p) {
  if (p.prm.hydro == SPHGPU_HYDRO_CRKSPH) {
    SPH_TRY(crk_prepare(p));
    launch_crk_eval(p);
  } else if (p.cfg.precision == SPHGPU_PRECISION_MIXED) {
    SPH_TRY(prepare_mixed(p));
    launch_eval_sph_mixed(p);
  } else {
    launch_eval_sph_fp64(p);
  }
  return cuda_status(cudaGetLastError(), "evaluate");
}

// CheapSynchronousRK2::step.
int step_impl(Problem& p) {
  double* d_dt = p.d_scal + 12;
  double* d_lastDt = p.d_scal + 13;
  // preStepInitialize: ghosts + connectivity every cycle, then ghost state.
  SPH_TRY(build_neighbors_impl(p));
  pack_records(p);
  // selectDt with the previous derivatives, state at the step start.
  launch_select_dt(p, d_dt, d_lastDt);
  // state0 copy
  SPH_CHECK(cudaMemcpyAsync(p.S0, p.S, sizeof(double)*NSTATE*(size_t)p.n, cudaMemcpyDeviceToDevice, p.stream));
  // trial advance to the mid point (updateAsIncrement for every policy)
  launch_update(p, d_dt, 0.5, true);
  pack_records(p);
  // initializeDerivatives + derivs.Zero + evaluateDerivatives at the mid point
  SPH_TRY(initialize_impl(p));
  SPH_TRY(launch_eval(p));
  // full step from state0 with the mid-point derivatives
  SPH_CHECK(cudaMemcpyAsync(p.S, p.S0, sizeof(double)*NSTATE*(size_t)p.n, cudaMemcpyDeviceToDevice, p.stream));
  if (p.prm.compatible) launch_compatible_energy(p, d_dt, 1.0);
  launch_update(p, d_dt, 1.0, false);
  // applyGhostBoundaries; postStepFinalize (sum density); enforceBoundaries
  pack_records(p);
  finalize_impl(p);
  launch_enforce_boundaries(p);
  SPH_CHECK(cudaMemcpyAsync(d_lastDt, d_dt, sizeof(double), cudaMemcpyDeviceToDevice, p.stream));
  SPH_CHECK(cudaGetLastError());
  double dt = 0.0;
  SPH_CHECK(cudaMemcpyAsync(&dt, d_dt, sizeof(double), cudaMemcpyDeviceToHost, p.stream));
  SPH_TRY(check_device_error(p, "step_rk2"));
  p.time += dt;
  p.lastDt = dt;
  p.cycle += 1;
  p.haveDerivs = true;
  return SPHGPU_OK;
}

}  // namespace

int ensure_block_sums(Problem& p, int64_t nblocks) {
  if (nblocks <= p.blockSumsCap) return SPHGPU_OK;
  cudaFree(p.blockSums);
  p.blockSumsCap = nblocks + 64;
  return dalloc(p.blockSums, p.blockSumsCap);
}

int exclusive_scan_i32(Problem& p, const int32_t* in, int64_t n, int64_t* out, int64_t* total) {
  const int64_t tiles = (n + SCAN_TILE - 1)/SCAN_TILE;
  SPH_TRY(ensure_block_sums(p, tiles + 1));
  int64_t* dtotal = p.blockSums + tiles;
  if (tiles > 0) scan_tile_sums_kernel<<<(unsigned)tiles, SCAN_THREADS, 0, p.stream>>>(in, n, p.blockSums); p.launches += (tiles > 0);
  scan_sums_kernel<<<1, SCAN_THREADS, 0, p.stream>>>(p.blockSums, tiles, dtotal); ++p.launches;
  scan_apply_kernel<<<(unsigned)(tiles > 0 ? tiles : 1), SCAN_THREADS, 0, p.stream>>>(in, n, p.blockSums, out, dtotal); ++p.launches;
  SPH_CHECK(cudaGetLastError());
  SPH_CHECK(cudaMemcpyAsync(total, dtotal, sizeof(int64_t), cudaMemcpyDeviceToHost, p.stream));
  SPH_CHECK(cudaStreamSynchronize(p.stream));
  return SPHGPU_OK;
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
    cudaFree(p.gpos);
  }
  p.gpos = np;
  p.gcap = ng;
  // (n + ghost)-sized buffers
  SPH_TRY(grow_preserve(p.counts, oldc, nc, p.stream));
  SPH_TRY(grow_preserve(p.offsets, oldc ? oldc + 1 : 0, nc + 1, p.stream));
  SPH_TRY(grow_preserve(p.cidx, 0, nc, p.stream));
  SPH_TRY(grow_preserve(p.sortedIdx, 0, nc, p.stream));
  cudaFree(p.cand);
  SPH_TRY(dalloc(p.cand, 10*nc));
  cudaFree(p.rec);
  SPH_TRY(dalloc(p.rec, RECW*nc));
  p.candcap = nc;
  p.reccap = nc;
  return SPHGPU_OK;
}

int ensure_capacity_entries(Problem& p, int64_t need) {
  if (need <= p.ecap) return SPHGPU_OK;
  const int64_t ne = need + need/8 + 1024;
  cudaFree(p.nbr);
  cudaFree(p.pacc);
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

struct sphgpu_problem : public Problem {};

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
    if ((rc = dalloc(p->d_scal, 32)) != SPHGPU_OK) break;
    p->redcap = 148*4*8;
    if ((rc = dalloc(p->d_red, p->redcap)) != SPHGPU_OK) break;
    cudaMemset(p->d_err, 0, 4*sizeof(int));
    cudaMemset(p->D, 0, sizeof(double)*NDERIV*(size_t)n);
    cudaMemset(p->S, 0, sizeof(double)*NSTATE*(size_t)n);
    p->lastDt = cfg->lastDt;
    cudaMemcpy(p->d_scal + 13, &p->lastDt, sizeof(double), cudaMemcpyHostToDevice);
    if ((rc = ensure_capacity_ghosts(*p, n/2 + 4096)) != SPHGPU_OK) break;
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
  SPH_TRY(download_aos(*p, p->S, 3, S_X, position));
  SPH_TRY(download_aos(*p, p->S, 3, S_VX, velocity));
  SPH_TRY(download_aos(*p, p->S, 1, S_M, mass));
  SPH_TRY(download_aos(*p, p->S, 1, S_RHO, massDensity));
  SPH_TRY(download_aos(*p, p->S, 1, S_EPS, specificThermalEnergy));
  SPH_TRY(download_aos(*p, p->S, 6, S_H, H));
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

int sphgpu_build_neighbors(sphgpu_problem* p) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(build_neighbors_impl(*p));
  pack_records(*p);
  return cuda_status(cudaGetLastError(), "pack_records");
}

int sphgpu_connectivity_size(sphgpu_problem* p, int64_t* num_ghosts, int64_t* num_entries) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(*p));
  if (num_ghosts) *num_ghosts = p->G;
  if (num_entries) *num_entries = p->E;
  return SPHGPU_OK;
}

int sphgpu_get_connectivity(sphgpu_problem* p, int64_t* offsets, int32_t* neighbors, int32_t* ghost_root) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(*p));
  if (offsets) SPH_CHECK(cudaMemcpyAsync(offsets, p->offsets, sizeof(int64_t)*(size_t)(p->n + 1), cudaMemcpyDeviceToHost, p->stream));
  if (neighbors && p->E) SPH_CHECK(cudaMemcpyAsync(neighbors, p->nbr, sizeof(int32_t)*(size_t)p->E, cudaMemcpyDeviceToHost, p->stream));
  if (ghost_root && p->G) SPH_CHECK(cudaMemcpyAsync(ghost_root, p->groot, sizeof(int32_t)*(size_t)p->G, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return SPHGPU_OK;
}

int sphgpu_initialize(sphgpu_problem* p, double time, double dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  (void)time; (void)dt;
  SPH_TRY(require_nbrs(*p));
  pack_records(*p);
  return initialize_impl(*p);
}

int sphgpu_evaluate_derivatives(sphgpu_problem* p, double time, double dt) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  (void)time; (void)dt;
  SPH_TRY(require_nbrs(*p));
  pack_records(*p);
  SPH_TRY(launch_eval(*p));
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
  SPH_TRY(require_nbrs(*p));
  pack_records(*p);
  finalize_impl(*p);
  return cuda_status(cudaGetLastError(), "finalize");
}

int sphgpu_dt(sphgpu_problem* p, double* dt_out) {
  if (p == nullptr || dt_out == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(*p));
  double* bits = p->d_scal + 14;
  launch_dt(*p, bits);
  SPH_CHECK(cudaGetLastError());
  double minDt = 0.0;
  SPH_CHECK(cudaMemcpyAsync(&minDt, bits, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  *dt_out = p->cfg.cfl*minDt;
  return SPHGPU_OK;
}

int sphgpu_step_rk2(sphgpu_problem* p, double* time, int64_t nsteps, double* last_dt) {
  if (p == nullptr || nsteps < 0) return SPHGPU_ERR_ARG;
  if (time) p->time = *time;
  for (int64_t s = 0; s < nsteps; ++s) SPH_TRY(step_impl(*p));
  if (time) *time = p->time;
  if (last_dt) *last_dt = p->lastDt;
  return SPHGPU_OK;
}

int sphgpu_conservation(sphgpu_problem* p, double out[8]) {
  if (p == nullptr || out == nullptr) return SPHGPU_ERR_ARG;
  launch_conservation(*p, p->d_scal + 16);
  SPH_CHECK(cudaGetLastError());
  SPH_CHECK(cudaMemcpyAsync(out, p->d_scal + 16, sizeof(double)*8, cudaMemcpyDeviceToHost, p->stream));
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return SPHGPU_OK;
}

int sphgpu_num_pairs(sphgpu_problem* p, int64_t* pairs) {
  if (p == nullptr || pairs == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(require_nbrs(*p));
  *pairs = p->pairs;
  return SPHGPU_OK;
}

int sphgpu_kernel_launches(sphgpu_problem* p, int64_t* launches) {
  if (p == nullptr || launches == nullptr) return SPHGPU_ERR_ARG;
  *launches = p->launches;
  return SPHGPU_OK;
}

int sphgpu_set_schedule(sphgpu_problem* p, const char* stage, int32_t schedule) {
  if (p == nullptr || stage == nullptr) return SPHGPU_ERR_ARG;
  if (std::strcmp(stage, "neighbor walk") == 0) {
    if (schedule < NBR_SCHEDULE_AUTO || schedule > NBR_SCHEDULE_WARP) {
      set_error("neighbor walk schedule must be 0 (auto), 1 (thread per node) or 2 (warp per node)");
      return SPHGPU_ERR_ARG;
    }
    p->nbrSchedule = schedule;
    return SPHGPU_OK;
  }
  set_error(std::string("unknown schedule stage: ") + stage);
  return SPHGPU_ERR_ARG;
}

int sphgpu_get_schedule(sphgpu_problem* p, const char* stage, int32_t* schedule) {
  if (p == nullptr || stage == nullptr || schedule == nullptr) return SPHGPU_ERR_ARG;
  if (std::strcmp(stage, "neighbor walk") == 0) {
    *schedule = p->lastNbrSchedule;
    return SPHGPU_OK;
  }
  set_error(std::string("unknown schedule stage: ") + stage);
  return SPHGPU_ERR_ARG;
}

int sphgpu_synchronize(sphgpu_problem* p) {
  if (p == nullptr) return SPHGPU_ERR_ARG;
  SPH_CHECK(cudaStreamSynchronize(p->stream));
  return check_device_error(*p, "synchronize");
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
  return SPHGPU_OK;
}

}  // extern "C"
