// Periodic ghost images, cell list and ConnectivityMap CSR on the device,
// for every member of a batch in one launch per stage.
//
// Replaces, for one FluidNodeList in a periodic box:
//   PlanarBoundary::setGhostNodes     src/Boundary/PlanarBoundary.cc:114-181
//   PlanarBoundary::updateGhostNodes  src/Boundary/PlanarBoundary.cc:361-395
//   NestedGridNeighbor + Neighbor precull (superset generation only)
//   ConnectivityMap::computeConnectivity src/Neighbor/ConnectivityMap.cc:521-890
//
// Compiled with -fmad=false: the ghost positions and the neighbor predicate
// |H_i r_ij|^2 <= kappa^2 || |H_j r_ij|^2 <= kappa^2 are evaluated in the
// reference's FP64 operation order, so neighbor sets are bit-identical.
//
// The build is sized on the device: the ghost counts, the cell grid, the
// entry count and the longest list are produced by kernels into each member's
// scalar slots and read there by the next kernels; launches are sized for the
// buffer capacities.  The host plans the capacities from the previous build,
// launches every stage, and reads the sizes back once at the end; a capacity
// overflow sets an error bit and the build is redone with larger buffers.
//
// Kernels and their bounds (see the roofline notes in the design document):
//   ghost_hmax / ghost_flag / ghost_scatter  O(N+G) streaming, HBM bound
//   node_bounds / cell_index / cell_scatter  O(N+G) streaming + atomics
//   nbr_thread<COUNT|FILL>                   thread per node (cell-sorted
//                                            order) over the 27 neighbouring
//                                            cells; 64-byte candidate records
//                                            shared by a warp through L1
//   nbr_walk<COUNT|FILL>                     warp per node, for large
//                                            candidate sets
#include <cstdio>
#include <cstring>
#include <climits>

#include "problem.cuh"

namespace sphgpu {

namespace {

constexpr int kGhostThreads = 256;
constexpr float kFilterTol = 1.0e-3f;
// shared memory for the per-thread lists of a 32-thread block (larger lists
// take the warp schedule)
constexpr size_t kMaxListSmem = 200*1024;

__device__ __forceinline__ unsigned long long orderedBits(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double fromOrderedBits(unsigned long long b) {
  const unsigned long long r = (b & 0x8000000000000000ULL) ? (b & 0x7fffffffffffffffULL) : ~b;
  return __longlong_as_double((long long)r);
}

__device__ __forceinline__ V3 nodePos(const Member& M, int64_t k) {
  const int64_t n = M.n;
  if (k < n) return V3{M.S[S_X*n + k], M.S[S_Y*n + k], M.S[S_Z*n + k]};
  const int64_t g = k - n;
  return V3{M.gpos[g], M.gpos[M.gcap + g], M.gpos[2*M.gcap + g]};
}
__device__ __forceinline__ Sym nodeH(const Member& M, int64_t k) {
  const int64_t n = M.n;
  const int64_t r = k < n ? k : M.groot[k - n];
  const double* S = M.S;
  return Sym{S[(S_H + 0)*n + r], S[(S_H + 1)*n + r], S[(S_H + 2)*n + r],
             S[(S_H + 3)*n + r], S[(S_H + 4)*n + r], S[(S_H + 5)*n + r]};
}

// internal + ghost nodes of the current build
__device__ __forceinline__ int64_t allNodes(const Member& M) { return M.n + scalI(M.scal, SC_G); }

__device__ __forceinline__ Grid loadGrid(const Member& M) {
  const double* s = M.scal + SC_GRID;
  Grid g;
  g.lo[0] = s[0]; g.lo[1] = s[1]; g.lo[2] = s[2];
  g.cell = s[3];
  g.dim[0] = (int)scalI(M.scal, SC_GRID + 4);
  g.dim[1] = (int)scalI(M.scal, SC_GRID + 5);
  g.dim[2] = (int)scalI(M.scal, SC_GRID + 6);
  g.filterTol = (float)s[7];
  return g;
}

// ---------------------------------------------------------------- ghosts
// Start of a build: no ghosts yet.
__global__ void build_init_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  double* s = mem[m].scal;
  setScalI(s, SC_NTOT, mem[m].n);
  setScalI(s, SC_G, 0);
  s[SC_HMAX] = 0.0;
  s[SC_MAXCOND] = 0.0;
}

// 1/min(eig(H)) of every internal node, once per build (ghosts share their
// root's H, so every boundary pass and the cell size read it from here), and
// the largest condition number of H (bounds the FP32 pre-test error).
__global__ void __launch_bounds__(kGhostThreads) node_hmax_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t i = mb.block*blockDim.x + threadIdx.x;
  double cond = 0.0;
  if (i < M.n) {
    const V3 ev = eigenValues(nodeH(M, i));
    M.hmaxi[i] = 1.0/vmin(ev);
    cond = vmax(ev)/vmin(ev);
    if (!(cond < 1.0e300)) cond = 1.0e300;     // degenerate H: no FP32 pre-test
  }
  for (int o = 16; o > 0; o >>= 1) cond = dmax(cond, __shfl_xor_sync(0xffffffffu, cond, o));
  if ((threadIdx.x & 31) == 0 && cond > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(M.scal + SC_MAXCOND),
              (unsigned long long)__double_as_longlong(cond));
}

__device__ __forceinline__ double nodeHmax(const Member& M, int64_t k) {
  return M.hmaxi[k < M.n ? k : M.groot[k - M.n]];
}

// hmax of PlanarBoundary::setGhostNodes: max 1/min(eig(H)) over nodes within
// kernelExtent*hmaxi of either plane.
__global__ void __launch_bounds__(kGhostThreads) ghost_hmax_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  double best = 0.0;
  if (k < scalI(M.scal, SC_NTOT) && M.prm.bcs.periodic[b >> 1]) {
    const PlanarBC& bc = M.prm.bcs.bc[b];
    const V3 r = nodePos(M, k);
    const double hmaxi = nodeHmax(M, k);
    if (dmin(minimumDistance(bc.exit, r), minimumDistance(bc.enter, r)) < M.prm.kernelExtent*hmaxi) best = hmaxi;
  }
  for (int o = 16; o > 0; o >>= 1) best = dmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(M.scal + SC_HMAX), (unsigned long long)__double_as_longlong(best));
}

__global__ void __launch_bounds__(kGhostThreads) ghost_flag_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  if (k >= scalI(M.scal, SC_NTOT)) return;
  int f = 0;
  const double hmax = M.scal[SC_HMAX];
  if (M.prm.bcs.periodic[b >> 1] && hmax > 0.0) {
    const V3 r = nodePos(M, k);
    const double disti = signedDistance(M.prm.bcs.bc[b].exit, r)/hmax;
    f = (disti >= 0.0 && disti <= M.prm.kernelExtent) ? 1 : 0;
  }
  M.counts[k] = f;
}

__global__ void __launch_bounds__(kGhostThreads) ghost_scatter_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  const int64_t ntot = scalI(M.scal, SC_NTOT);
  if (k >= ntot || !M.counts[k]) return;
  const int64_t n = M.n;
  const int64_t g = (ntot - n) + M.offsets[k];     // ghost index of the new image
  if (g >= M.gcap) {
    atomicOr(M.err, DERR_GHOST_CAPACITY);
    return;
  }
  const PlanarBC& bc = M.prm.bcs.bc[b];
  const V3 gp = mapPositionThroughPlanes(nodePos(M, k), bc.exit, bc.enter);
  const int32_t root = k < n ? (int32_t)k : M.groot[k - n];
  uint32_t code = k < n ? 0u : M.gcode[k - n];
  const int axis = b >> 1;
  if ((code >> (2*axis)) & 3u) atomicOr(M.err, DERR_GHOST_CHAIN);
  code |= (uint32_t)((b & 1) + 1) << (2*axis);
  M.groot[g] = root;
  M.gcode[g] = code;
  M.gpos[g] = gp.x; M.gpos[M.gcap + g] = gp.y; M.gpos[2*M.gcap + g] = gp.z;
}

// After a boundary pass: the new images join the node set (at most up to the
// ghost capacity; beyond it the build is redone), hmax restarts.
__global__ void ghost_advance_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const Member& M = mem[m];
  int64_t g = scalI(M.scal, SC_NTOT) - M.n + scalI(M.scal, SC_TOTAL);
  if (g > M.gcap) {
    atomicOr(M.err, DERR_GHOST_CAPACITY);
    g = M.gcap;
  }
  setScalI(M.scal, SC_NTOT, M.n + g);
  setScalI(M.scal, SC_G, g);
  M.scal[SC_HMAX] = 0.0;
}

// ---------------------------------------------------------------- cells
__global__ void bounds_init_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  unsigned long long* bb = reinterpret_cast<unsigned long long*>(mem[m].scal + SC_BOUNDS);
  for (int a = 0; a < 3; ++a) { bb[a] = ~0ULL; bb[3 + a] = 0ULL; }
  bb[6] = 0ULL;
}

// Bounding box of all nodes and max of 1/min(eig(H)) (cell size).
__global__ void __launch_bounds__(kGhostThreads) node_bounds_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, h = 0.0;
  if (k < allNodes(M)) {
    const V3 r = nodePos(M, k);
    lo[0] = r.x; lo[1] = r.y; lo[2] = r.z;
    hi[0] = r.x; hi[1] = r.y; hi[2] = r.z;
    if (k < M.n) h = M.hmaxi[k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    h = fmax(h, __shfl_xor_sync(0xffffffffu, h, o));
  }
  __shared__ double sh[kGhostThreads/32][7];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) { sh[w][a] = lo[a]; sh[w][3 + a] = hi[a]; }
    sh[w][6] = h;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) {
      for (int a = 0; a < 3; ++a) { lo[a] = fmin(lo[a], sh[ww][a]); hi[a] = fmax(hi[a], sh[ww][3 + a]); }
      h = fmax(h, sh[ww][6]);
    }
    unsigned long long* out = reinterpret_cast<unsigned long long*>(M.scal + SC_BOUNDS);
    for (int a = 0; a < 3; ++a) {
      atomicMin(out + a, orderedBits(lo[a]));
      atomicMax(out + 3 + a, orderedBits(hi[a]));
    }
    atomicMax(out + 6, orderedBits(h));
  }
}

// Uniform grid of cells of edge >= kappa*max(1/lambda_min(H)) (the margin
// covers the libm difference of the eigenvalue solve for anisotropic H),
// enlarged until the cells fit the cell buffers (larger cells only widen the
// candidate set).  Also resets the walk's counters and sets the FP32
// pre-test tolerance: only when every H has condition number <= 100.
__global__ void grid_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const Member& M = mem[m];
  const unsigned long long* bb = reinterpret_cast<const unsigned long long*>(M.scal + SC_BOUNDS);
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) { lo[a] = fromOrderedBits(bb[a]); hi[a] = fromOrderedBits(bb[3 + a]); }
  const double hmaxAll = fromOrderedBits(bb[6]);
  double cell = M.prm.kernelExtent*hmaxAll*1.001;
  if (!(cell > 0.0) || !(cell < 1.0e300)) {
    atomicOr(M.err, DERR_NONPOSITIVE);
    cell = 1.0;
  }
  const int64_t maxCells = M.cellcap < ((int64_t)1 << 26) ? M.cellcap : ((int64_t)1 << 26);
  int64_t dim[3] = {1, 1, 1}, ncells = 1;
  for (int attempt = 0; attempt < 200; ++attempt) {
    ncells = 1;
    for (int a = 0; a < 3; ++a) {
      const double d = (hi[a] - lo[a])/cell;
      const int64_t mm = d < 1.0e6 ? (int64_t)d + 1 : (int64_t)1 << 20;
      dim[a] = mm < (1 << 20) ? mm : (1 << 20);
      ncells *= dim[a];
    }
    if (ncells <= maxCells) break;
    cell *= 1.26;
  }
  double* s = M.scal + SC_GRID;
  s[0] = lo[0]; s[1] = lo[1]; s[2] = lo[2];
  s[3] = cell;
  for (int a = 0; a < 3; ++a) setScalI(M.scal, SC_GRID + 4 + a, dim[a]);
  const double cond = M.scal[SC_MAXCOND];
  s[7] = (M.grid.filterTol > 0.0f && cond > 0.0 && cond <= 100.0) ? (double)M.grid.filterTol : 0.0;
  setScalI(M.scal, SC_NCELLS, ncells);
  setScalI(M.scal, SC_MAXCOUNT, 0);
  setScalI(M.scal, SC_PAIRS, 0);
}

__device__ __forceinline__ int cellCoord(double x, double lo, double cell, int dim) {
  int c = int((x - lo)/cell);
  return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

__global__ void __launch_bounds__(kGhostThreads) cell_zero_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t c = mb.block*blockDim.x + threadIdx.x;
  if (c < scalI(M.scal, SC_NCELLS)) M.cellFill[c] = 0;
}

__global__ void __launch_bounds__(kGhostThreads) cell_index_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  if (k >= allNodes(M)) return;
  const Grid g = loadGrid(M);
  const V3 r = nodePos(M, k);
  const int cx = cellCoord(r.x, g.lo[0], g.cell, g.dim[0]);
  const int cy = cellCoord(r.y, g.lo[1], g.cell, g.dim[1]);
  const int cz = cellCoord(r.z, g.lo[2], g.cell, g.dim[2]);
  const int c = (cz*g.dim[1] + cy)*g.dim[0] + cx;
  M.cidx[k] = c;
  atomicAdd(M.cellFill + c, 1);
}

// Candidate record of the cell-sorted node list, 64 bytes read as four
// 16-byte loads: FP64 position, node index, FP32 copy of H.  The FP64 H of
// the same slot sits in a second array (48 bytes) and is read only when the
// FP32 pre-test cannot decide.
struct __align__(16) NbrCand {
  double x, y, z;
  int32_t idx;
  float h[6];
  float pad;
};
static_assert(sizeof(NbrCand) == 64, "candidate record is four 16-byte words");

__device__ __forceinline__ NbrCand loadCand(const NbrCand* c) {
  const double2* q = reinterpret_cast<const double2*>(c);
  const double2 a = __ldg(q);
  const double2 b = __ldg(q + 1);
  const float4 f = __ldg(reinterpret_cast<const float4*>(q + 2));
  const float4 g = __ldg(reinterpret_cast<const float4*>(q + 3));
  NbrCand r;
  r.x = a.x; r.y = a.y; r.z = b.x;
  const uint64_t w = (uint64_t)__double_as_longlong(b.y);
  r.idx = (int32_t)(uint32_t)(w & 0xffffffffu);
  r.h[0] = __uint_as_float((uint32_t)(w >> 32));
  r.h[1] = f.x; r.h[2] = f.y; r.h[3] = f.z; r.h[4] = f.w; r.h[5] = g.x;
  r.pad = 0.0f;
  return r;
}

__device__ __forceinline__ const double* candHArray(const Member& M) {
  return static_cast<const double*>(M.cand) + 8*M.candcap;
}

__device__ __forceinline__ Sym loadCandH(const double* candH, int64_t k) {
  const double2* q = reinterpret_cast<const double2*>(candH + 6*k);
  const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
  return Sym{a.x, a.y, b.x, b.y, c.x, c.y};
}

__device__ __forceinline__ float symEta2F(const float* h, float x, float y, float z) {
  const float ex = __fmaf_rn(h[0], x, __fmaf_rn(h[1], y, h[2]*z));
  const float ey = __fmaf_rn(h[1], x, __fmaf_rn(h[3], y, h[4]*z));
  const float ez = __fmaf_rn(h[2], x, __fmaf_rn(h[4], y, h[5]*z));
  return __fmaf_rn(ex, ex, __fmaf_rn(ey, ey, ez*ez));
}

// ConnectivityMap predicate |H_i r_ij|^2 <= kappa^2 || |H_j r_ij|^2 <= kappa^2.
// A FP32 pre-test on r_ij = r_i - r_j (formed in FP64, rounded once) decides
// every pair whose eta^2 lies outside the band kappa^2 (1 -+ tol); inside the
// band the test is the exact FP64 one in the reference's operation order.
// The FP32 error of eta^2 is below 1e-6 cond(H) relative, and tol is only set
// (1e-3) when every H has cond(H) <= 100, so the result equals the exact test.
__device__ __forceinline__ bool neighborTest(const V3& ri, const Sym& Hi, const float* hif, const NbrCand& c,
                                             const double* candH, int64_t k, double k2, float tol) {
  const double dx = ri.x - c.x, dy = ri.y - c.y, dz = ri.z - c.z;
  if (tol > 0.0f) {
    const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
    const float e2i = symEta2F(hif, fx, fy, fz);
    const float e2j = symEta2F(c.h, fx, fy, fz);
    const float k2f = (float)k2;
    const float lo = k2f*(1.0f - tol), hi = k2f*(1.0f + tol);
    if (e2i <= lo || e2j <= lo) return true;
    if (e2i > hi && e2j > hi) return false;
  }
  const V3 rij{dx, dy, dz};
  return mag2(sdot(Hi, rij)) <= k2 || mag2(sdot(loadCandH(candH, k), rij)) <= k2;
}

__global__ void __launch_bounds__(kGhostThreads) cell_scatter_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t k = mb.block*blockDim.x + threadIdx.x;
  if (k >= allNodes(M)) return;
  const int c = M.cidx[k];
  const int64_t slot = M.cellStart[c] + atomicAdd(M.cellFill + c, 1);
  M.sortedIdx[slot] = (int32_t)k;
  const V3 r = nodePos(M, k);
  const Sym H = nodeH(M, k);
  double2* q = reinterpret_cast<double2*>(static_cast<NbrCand*>(M.cand) + slot);
  const uint64_t w = (uint64_t)(uint32_t)k | ((uint64_t)__float_as_uint((float)H.xx) << 32);
  q[0] = make_double2(r.x, r.y);
  q[1] = make_double2(r.z, __longlong_as_double((long long)w));
  float4* f = reinterpret_cast<float4*>(q + 2);
  f[0] = make_float4((float)H.xy, (float)H.xz, (float)H.yy, (float)H.yz);
  f[1] = make_float4((float)H.zz, 0.0f, 0.0f, 0.0f);
  double2* h = reinterpret_cast<double2*>(const_cast<double*>(candHArray(M)) + 6*slot);
  h[0] = make_double2(H.xx, H.xy);
  h[1] = make_double2(H.xz, H.yy);
  h[2] = make_double2(H.yz, H.zz);
}

// Thread per internal node, nodes taken in cell-sorted order so that the
// threads of a warp share their candidate rows (L1 broadcast).  The 27
// neighbouring cells are walked as 9 x-rows (three cells each, contiguous in
// the sorted order) and the exact ConnectivityMap predicate is applied.
// COUNT pass: per-node counts and their maximum.  FILL pass: the neighbor
// indices are insertion-sorted into a per-thread shared-memory list of
// capacity `cap` (element c of thread t at lst[c*blockDim + t], conflict
// free) and stored ascending at offsets[i].
// A member with a stash (Grid::stashCap > 0) builds its lists in the COUNT
// pass too and stores them ascending in the stash, element c of sorted slot s
// at stash[c*stashStride + s]; nbr_compact_thread_kernel then moves them to
// offsets[i], and the FILL pass does not run for it.
template<bool FILL>
__global__ void __launch_bounds__(256) nbr_thread_kernel(const Member* mem, BlockMap bm, int cap, int maxNbr) {
  extern __shared__ int32_t lst[];
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int tid = threadIdx.x;
  const int bd = blockDim.x;
  const int64_t s = mb.block*bd + tid;
  const int64_t n = M.n;
  const NbrCand* cand = static_cast<const NbrCand*>(M.cand);
  NbrCand me;
  bool active = s < allNodes(M);
  if (active) {
    me = loadCand(cand + s);
    active = me.idx < n;
  }
  // list capacity: the shared-memory list (FILL) or the member's stash (COUNT)
  const int lcap = FILL ? cap : M.grid.stashCap;
  const bool collect = FILL || lcap > 0;
  int count = 0, above = 0;
  if (active) {
    const Grid g = loadGrid(M);
    const double kernelExtent2 = M.prm.kernelExtent*M.prm.kernelExtent;
    const int64_t* cellStart = M.cellStart;
    const double* candH = candHArray(M);
    const int32_t i = me.idx;
    const V3 ri{me.x, me.y, me.z};
    const Sym Hi = loadCandH(candH, s);
    const int cx = cellCoord(ri.x, g.lo[0], g.cell, g.dim[0]);
    const int cy = cellCoord(ri.y, g.lo[1], g.cell, g.dim[1]);
    const int cz = cellCoord(ri.z, g.lo[2], g.cell, g.dim[2]);
    const int x0 = cx > 0 ? cx - 1 : 0;
    const int x1 = cx + 1 < g.dim[0] ? cx + 1 : g.dim[0] - 1;
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = cz + dz;
      if (z < 0 || z >= g.dim[2]) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= g.dim[1]) continue;
        const int cbase = (z*g.dim[1] + y)*g.dim[0];
        const int64_t start = cellStart[cbase + x0];
        const int64_t end = cellStart[cbase + x1 + 1];
        for (int64_t k = start; k < end; ++k) {
          const NbrCand c = loadCand(cand + k);
          if (c.idx != i && neighborTest(ri, Hi, me.h, c, candH, k, kernelExtent2, g.filterTol)) {
            if (collect) {
              if (count < lcap) {
                int p = count;
                while (p > 0) {
                  const int32_t prev = lst[(p - 1)*bd + tid];
                  if (prev < c.idx) break;
                  lst[p*bd + tid] = prev;
                  --p;
                }
                lst[p*bd + tid] = c.idx;
              }
              above += (c.idx > i);
            }
            ++count;
          }
        }
      }
    }
    if (!FILL) {
      M.counts[i] = count;
      if (count > maxNbr) atomicOr(M.err, DERR_NBR_CAPACITY);
      if (lcap > 0) {
        const int64_t stride = M.grid.stashStride;
        if (count > lcap || s >= stride) {
          atomicOr(M.err, DERR_LIST_CAPACITY);
        } else {
          int32_t* stash = reinterpret_cast<int32_t*>(M.pacc);
          for (int c = 0; c < count; ++c) stash[c*stride + s] = lst[c*bd + tid];
        }
      }
    } else {
      const int64_t o = M.offsets[i];
      if (count > cap) atomicOr(M.err, DERR_LIST_CAPACITY);
      else if (o + count > M.ecap) atomicOr(M.err, DERR_ENTRY_CAPACITY);
      else for (int c = 0; c < count; ++c) M.nbr[o + c] = lst[c*bd + tid];
    }
  }
  if (!FILL) {
    int m = count;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0 && m > 0) atomicMax(reinterpret_cast<int*>(M.scal + SC_MAXCOUNT), m);
  }
  if (collect) {
    unsigned long long a = (unsigned long long)above;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((tid & 31) == 0 && a) atomicAdd(reinterpret_cast<unsigned long long*>(M.scal + SC_PAIRS), a);
  }
}

// Stashed lists (thread schedule) to the CSR: thread per sorted slot.
__global__ void __launch_bounds__(256) nbr_compact_thread_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t s = mb.block*blockDim.x + threadIdx.x;
  if (s >= allNodes(M)) return;
  const int32_t i = M.sortedIdx[s];
  if (i >= M.n) return;
  const int count = M.counts[i];
  const int64_t stride = M.grid.stashStride;
  if (count > M.grid.stashCap || s >= stride) return;   // not stashed: the count pass flagged it
  const int64_t o = M.offsets[i];
  if (o + count > M.ecap) {
    atomicOr(M.err, DERR_ENTRY_CAPACITY);
    return;
  }
  const int32_t* stash = reinterpret_cast<const int32_t*>(M.pacc);
  for (int c = 0; c < count; ++c) M.nbr[o + c] = stash[c*stride + s];
}

// Stashed lists (warp schedule) to the CSR: warp per internal node, the list
// of node i at stash[i*stashCap : i*stashCap + count].
__global__ void __launch_bounds__(256) nbr_compact_warp_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int lane = threadIdx.x & 31;
  const int64_t i = (mb.block*(int64_t)blockDim.x + threadIdx.x) >> 5;
  if (i >= M.n) return;
  const int count = M.counts[i];
  if (count > M.grid.stashCap) return;       // not stashed: the count pass flagged it
  const int64_t o = M.offsets[i];
  if (o + count > M.ecap) {
    if (lane == 0) atomicOr(M.err, DERR_ENTRY_CAPACITY);
    return;
  }
  const int32_t* stash = reinterpret_cast<const int32_t*>(M.pacc) + i*(int64_t)M.grid.stashCap;
  for (int t = lane; t < count; t += 32) M.nbr[o + t] = stash[t];
}

// Warp per internal node: walk the 27 neighbouring cells, apply the exact
// ConnectivityMap predicate, count (FILL=false) or collect, sort ascending
// and store (FILL=true) the neighbor indices.  Used when the candidate sets
// are large (many nodes per cell), where a warp per node keeps the SMs full.
// `cap` is the per-warp list capacity (a power of two >= 32).  A member with
// a stash (Grid::stashCap > 0) collects and sorts in the COUNT pass and
// stores the list of node i at stash[i*stashCap]; nbr_compact_warp_kernel
// moves it to offsets[i].
template<bool FILL>
__global__ void __launch_bounds__(256) nbr_walk_kernel(const Member* mem, BlockMap bm, int cap, int maxNbr) {
  extern __shared__ int32_t sbuf_all[];
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int scap = FILL ? 0 : M.grid.stashCap;
  const bool collect = FILL || scap > 0;
  int32_t* sbuf = sbuf_all + (collect ? wib*cap : 0);
  const int64_t n = M.n;
  const int64_t i = (mb.block*(int64_t)blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const double* S = M.S;
  const Grid g = loadGrid(M);
  const NbrCand* cand = static_cast<const NbrCand*>(M.cand);
  const double kernelExtent2 = M.prm.kernelExtent*M.prm.kernelExtent;
  const V3 ri{S[S_X*n + i], S[S_Y*n + i], S[S_Z*n + i]};
  const Sym Hi{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
               S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
  const float hif[6] = {(float)Hi.xx, (float)Hi.xy, (float)Hi.xz, (float)Hi.yy, (float)Hi.yz, (float)Hi.zz};
  const double* candH = candHArray(M);
  const int cx = cellCoord(ri.x, g.lo[0], g.cell, g.dim[0]);
  const int cy = cellCoord(ri.y, g.lo[1], g.cell, g.dim[1]);
  const int cz = cellCoord(ri.z, g.lo[2], g.cell, g.dim[2]);
  int count = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = cz + dz;
    if (z < 0 || z >= g.dim[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = cy + dy;
      if (y < 0 || y >= g.dim[1]) continue;
      // the three x-cells of a row are contiguous in the sorted order
      const int x0 = cx > 0 ? cx - 1 : 0;
      const int x1 = cx + 1 < g.dim[0] ? cx + 1 : g.dim[0] - 1;
      const int cbase = (z*g.dim[1] + y)*g.dim[0];
      const int64_t start = M.cellStart[cbase + x0];
      const int64_t end = M.cellStart[cbase + x1 + 1];
      for (int64_t base = start; base < end; base += 32) {
        const int64_t k = base + lane;
        bool pass = false;
        int32_t j = -1;
        if (k < end) {
          const NbrCand c = loadCand(cand + k);
          j = c.idx;
          pass = j != (int32_t)i && neighborTest(ri, Hi, hif, c, candH, k, kernelExtent2, g.filterTol);
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, pass);
        if (collect && pass) {
          const int pos = count + __popc(ballot & ((1u << lane) - 1u));
          if (pos < cap) sbuf[pos] = j;
        }
        count += __popc(ballot);
      }
    }
  }
  if (!FILL) {
    if (lane == 0) {
      M.counts[i] = count;
      if (count > maxNbr) atomicOr(M.err, DERR_NBR_CAPACITY);
      atomicMax(reinterpret_cast<int*>(M.scal + SC_MAXCOUNT), count);
    }
    if (scap == 0) return;
    if (count > scap) {
      if (lane == 0) atomicOr(M.err, DERR_LIST_CAPACITY);
      return;
    }
  }
  const int64_t o = FILL ? M.offsets[i] : 0;
  if (FILL && (count > cap || o + count > M.ecap)) {
    if (lane == 0) atomicOr(M.err, count > cap ? DERR_LIST_CAPACITY : DERR_ENTRY_CAPACITY);
    return;
  }
  int32_t* out = FILL ? M.nbr + o : reinterpret_cast<int32_t*>(M.pacc) + i*(int64_t)scap;
  // bitonic sort of sbuf[0:count] (padded to a power of two)
  int size = 32;
  while (size < count) size <<= 1;
  for (int t = count + lane; t < size; t += 32) sbuf[t] = INT_MAX;
  __syncwarp();
  for (int k = 2; k <= size; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int t = lane; t < size; t += 32) {
        const int ixj = t ^ jj;
        if (ixj > t) {
          const int32_t a = sbuf[t], b = sbuf[ixj];
          const bool up = (t & k) == 0;
          if ((a > b) == up) { sbuf[t] = b; sbuf[ixj] = a; }
        }
      }
      __syncwarp();
    }
  }
  int above = 0;
  for (int t = lane; t < count; t += 32) {
    const int32_t j = sbuf[t];
    out[t] = j;
    above += (j > (int32_t)i);
  }
  for (int s = 16; s > 0; s >>= 1) above += __shfl_xor_sync(0xffffffffu, above, s);
  if (lane == 0 && above)
    atomicAdd(reinterpret_cast<unsigned long long*>(M.scal + SC_PAIRS), (unsigned long long)above);
}

int64_t asI64(double stored) {
  int64_t v;
  std::memcpy(&v, &stored, sizeof(v));
  return v;
}

int asI32(double stored) {
  int v;
  std::memcpy(&v, &stored, sizeof(v));
  return v;
}

int64_t grow(int64_t v) { return v + v/4 + 1024; }

// Capacities for the next build, from the previous one (or first estimates).
int plan_capacities(Batch& b) {
  for (Problem* pp : b.mem) {
    Problem& p = *pp;
    const int64_t oldg = p.gcap, oldc = p.candcap, olde = p.ecap, oldcells = p.cellcap;
    // sizes of the last build, else the caller's hints, else built-in guesses
    const int64_t G = p.G > 0 ? p.G : p.hintG;
    const int64_t E = p.E > 0 ? p.E : p.hintE;
    const int64_t cells = p.ncells > 0 ? p.ncells : p.hintCells;
    if (G > 0) SPH_TRY(ensure_capacity_ghosts(p, grow(G)));
    const int64_t cellsNeed = cells > 0 ? grow(cells) : p.candcap/2 + 64;
    if (cellsNeed + 1 > p.cellcap) {
      cudaStreamSynchronize(b.stream);
      cudaFree(p.cellStart); cudaFree(p.cellFill);
      p.cellStart = nullptr; p.cellFill = nullptr;
      p.cellcap = cellsNeed + 1;
      if (cudaMalloc(&p.cellStart, sizeof(int64_t)*(p.cellcap + 1)) != cudaSuccess ||
          cudaMalloc(&p.cellFill, sizeof(int32_t)*p.cellcap) != cudaSuccess) {
        p.cellcap = 0;
        set_error("cell list allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
    }
    // without a hint the first build guesses 32 entries per node; an overflow redoes it
    SPH_TRY(ensure_capacity_entries(p, E > 0 ? E + E/8 : 32*p.n));
    if (p.fillCap < 8) p.fillCap = p.maxCount > 0 ? p.maxCount + p.maxCount/4 + 8 : 64;
    const int64_t tiles = ((p.candcap > p.cellcap ? p.candcap : p.cellcap) + 1023)/1024 + 2;
    if (tiles > p.blockSumsCap) SPH_TRY(ensure_block_sums(p, tiles));
    if (p.gcap != oldg || p.candcap != oldc || p.ecap != olde || p.cellcap != oldcells) b.memDirty = true;
    // schedule: a warp per node once the 27-cell candidate set of the last
    // build kept 32 lanes busy, or once a thread's list would not fit in
    // shared memory
    const double candPerNode = p.ncells > 0 ? 27.0*(double)(p.n + p.G)/(double)p.ncells : 0.0;
    const int req = p.nbrSchedule != NBR_SCHEDULE_AUTO ? p.nbrSchedule : b.nbrSchedule;
    p.fillSchedule = (req == NBR_SCHEDULE_WARP || (req == NBR_SCHEDULE_AUTO && candPerNode > 384.0) ||
                      sizeof(int32_t)*32*(size_t)p.fillCap > kMaxListSmem)
                         ? NBR_SCHEDULE_WARP : NBR_SCHEDULE_THREAD;
    p.grid.filterTol = p.nbrFilter ? kFilterTol : 0.0f;
    // single pass: the lists go to the pair-acceleration buffer (free until
    // the next derivative evaluation rewrites it) when they fit there
    // (thread schedule: one row per sorted slot, internal and ghost, sized
    // from the last build's ghosts; a slot beyond it flags the build for a redo)
    const int64_t rows = G > 0 ? p.n + grow(G) : p.candcap;
    p.grid.stashStride = rows < p.candcap ? rows : p.candcap;
    const int64_t slots = p.fillSchedule == NBR_SCHEDULE_WARP ? p.n : p.grid.stashStride;
    p.grid.stashCap = (p.pacc != nullptr && p.nbrStash && (int64_t)p.fillCap*slots <= 6*p.ecap) ? p.fillCap : 0;
  }
  b.memDirty = true;
  return SPHGPU_OK;
}

}  // namespace

// Mirrors the capacity rules a new problem goes through: sphgpu_create sizes
// the ghost and (n + ghost) buffers for n/2 + 4096 ghosts, plan_capacities
// grows them from the planned sizes, ensure_capacity_* add their own slack,
// and the mixed and CRKSPH records follow the (n + ghost) capacity.
int64_t planned_bytes(const sphgpu_config& cfg, int64_t n, int64_t G, int64_t E, int64_t ncells) {
  auto ghostCap = [](int64_t need) { return need + need/2 + 1024; };  // ensure_capacity_ghosts
  Problem p;
  p.cfg = cfg;
  p.n = n;
  p.prm.W.n = cfg.num_points;
  p.gcap = ghostCap(n/2 + 4096);
  if (G > 0 && grow(G) > p.gcap) p.gcap = ghostCap(grow(G));
  p.candcap = n + p.gcap;
  p.cellcap = (ncells > 0 ? grow(ncells) : p.candcap/2 + 64) + 1;
  const int64_t eneed = E > 0 ? E + E/8 : 32*n;
  p.ecap = eneed + eneed/8 + 1024;                                       // ensure_capacity_entries
  p.blockSumsCap = ((p.candcap > p.cellcap ? p.candcap : p.cellcap) + 1023)/1024 + 2 + 64;
  if (cfg.precision == SPHGPU_PRECISION_MIXED) p.mreccap = p.candcap;
  if (cfg.hydro == SPHGPU_HYDRO_CRKSPH) p.creccap = p.candcap;
  double marker = 0.0;                          // problem_bytes only tests these for null
  if (cfg.compatibleEnergyEvolution) p.pacc = &marker;
  if (cfg.precision == SPHGPU_PRECISION_MIXED) p.coefF = reinterpret_cast<float*>(&marker);
  if (cfg.hydro == SPHGPU_HYDRO_CRKSPH) p.K = &marker;
  const int64_t b = problem_bytes(p);
  p.pacc = nullptr; p.coefF = nullptr; p.K = nullptr;
  return b;
}

namespace {

int launch_build(Batch& b) {
  cudaStream_t st = b.stream;
  const int nm = (int)b.mem.size();
  SPH_TRY(batch_upload(b));
  BlockMap bm;
  unsigned grid = 0;
  // ---- ghosts: six planar boundaries in order, sizes kept on the device
  build_init_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return p.n; }, kGhostThreads, &bm, &grid));
  if (grid) { node_hmax_kernel<<<grid, kGhostThreads, 0, st>>>(b.d_mem, bm); batch_count_launch(b); }
  BlockMap cap;
  unsigned capGrid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return p.candcap; }, kGhostThreads, &cap, &capGrid));
  for (int bnd = 0; bnd < 6; ++bnd) {
    bool any = false;
    for (Problem* p : b.mem) any = any || p->prm.bcs.periodic[bnd >> 1];
    if (!any) continue;
    ghost_hmax_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap, bnd); batch_count_launch(b);
    ghost_flag_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap, bnd); batch_count_launch(b);
    SPH_TRY(batch_scan(b, SCAN_FLAGS));
    ghost_scatter_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap, bnd); batch_count_launch(b);
    ghost_advance_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  }
  // ---- cell grid and counting sort of all nodes by cell
  bounds_init_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  node_bounds_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap); batch_count_launch(b);
  grid_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  BlockMap cm;
  unsigned cgrid = 0;
  SPH_TRY(batch_map_items(b, [](const Problem& p) { return p.cellcap; }, kGhostThreads, &cm, &cgrid));
  cell_zero_kernel<<<cgrid, kGhostThreads, 0, st>>>(b.d_mem, cm); batch_count_launch(b);
  cell_index_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap); batch_count_launch(b);
  SPH_TRY(batch_scan(b, SCAN_CELLS));
  cell_zero_kernel<<<cgrid, kGhostThreads, 0, st>>>(b.d_mem, cm); batch_count_launch(b);
  cell_scatter_kernel<<<capGrid, kGhostThreads, 0, st>>>(b.d_mem, cap); batch_count_launch(b);
  // ---- neighbor counts, offsets, lists
  int maxNbr = 0, tcap = 1, wmax = 0;
  bool tstash = false, wstash = false;
  for (Problem* p : b.mem) {
    maxNbr = p->maxNbr > maxNbr ? p->maxNbr : maxNbr;
    if (p->fillSchedule == NBR_SCHEDULE_WARP) {
      wmax = p->fillCap > wmax ? p->fillCap : wmax;
      wstash = wstash || p->grid.stashCap > 0;
    } else {
      tcap = p->fillCap > tcap ? p->fillCap : tcap;
      tstash = tstash || p->grid.stashCap > 0;
    }
  }
  const int wthreads = 256;
  // a thread's list lives in shared memory: fewer threads per block for long lists
  int fthreads = 256;
  while (fthreads > 32 && sizeof(int32_t)*(size_t)fthreads*tcap > 96*1024) fthreads >>= 1;
  const int tthreads = tstash ? fthreads : 256;
  // bitonic sort pads each warp's list to a power of two >= 32
  int wcap = 32;
  while (wcap < wmax) wcap <<= 1;
  auto thread = [](const Problem& p) { return p.fillSchedule != NBR_SCHEDULE_WARP; };
  BlockMap tmap, wmap, fmap, wfmap, ctmap, cwmap;
  unsigned tgrid = 0, wgrid = 0, fgrid = 0, wfgrid = 0, ctgrid = 0, cwgrid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return thread(p) ? p.candcap : (int64_t)0; },
                          tthreads, &tmap, &tgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return thread(p) ? (int64_t)0 : 32*p.n; }, wthreads, &wmap, &wgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return thread(p) && !p.grid.stashCap ? p.candcap : (int64_t)0; },
                          fthreads, &fmap, &fgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return !thread(p) && !p.grid.stashCap ? 32*p.n : (int64_t)0; },
                          wthreads, &wfmap, &wfgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return thread(p) && p.grid.stashCap ? p.candcap : (int64_t)0; },
                          256, &ctmap, &ctgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return !thread(p) && p.grid.stashCap ? 32*p.n : (int64_t)0; },
                          256, &cwmap, &cwgrid));
  for (Problem* p : b.mem) {
    p->lastNbrSchedule = p->fillSchedule;
    p->lastNbrPasses = p->grid.stashCap > 0 ? 1 : 2;
  }
  b.lastNbrSchedule = nm ? b.mem[0]->lastNbrSchedule : 0;
  const size_t tsmem = sizeof(int32_t)*(size_t)fthreads*tcap;
  const size_t wsmem = sizeof(int32_t)*(wthreads/32)*(size_t)wcap;
  if (tsmem > 48*1024) {
    for (auto* k : {nbr_thread_kernel<false>, nbr_thread_kernel<true>}) {
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem);
      if (e != cudaSuccess) return cuda_status(e, "nbr smem attribute");
    }
  }
  if (wsmem > 48*1024) {
    for (auto* k : {nbr_walk_kernel<false>, nbr_walk_kernel<true>}) {
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem);
      if (e != cudaSuccess) return cuda_status(e, "nbr smem attribute");
    }
  }
  // count pass (and the lists of members with a stash)
  if (tgrid) {
    nbr_thread_kernel<false><<<tgrid, tthreads, tstash ? tsmem : 0, st>>>(b.d_mem, tmap, tstash ? tcap : 0, maxNbr);
    batch_count_launch(b);
  }
  if (wgrid) {
    nbr_walk_kernel<false><<<wgrid, wthreads, wstash ? wsmem : 0, st>>>(b.d_mem, wmap, wstash ? wcap : 0, maxNbr);
    batch_count_launch(b);
  }
  SPH_TRY(batch_scan(b, SCAN_COUNTS));
  // lists to the CSR: compaction of the stashes, fill pass for the rest
  if (ctgrid) { nbr_compact_thread_kernel<<<ctgrid, 256, 0, st>>>(b.d_mem, ctmap); batch_count_launch(b); }
  if (cwgrid) { nbr_compact_warp_kernel<<<cwgrid, 256, 0, st>>>(b.d_mem, cwmap); batch_count_launch(b); }
  if (fgrid) { nbr_thread_kernel<true><<<fgrid, fthreads, tsmem, st>>>(b.d_mem, fmap, tcap, maxNbr); batch_count_launch(b); }
  if (wfgrid) { nbr_walk_kernel<true><<<wfgrid, wthreads, wsmem, st>>>(b.d_mem, wfmap, wcap, maxNbr); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "neighbor build");
}

}  // namespace

// Ghosts and ConnectivityMap of every member: all stages launched with the
// sizes kept on the device, then one read-back of the sizes; a capacity
// overflow grows the buffers and repeats the build.
int build_connectivity(Batch& b) {
  const int nm = (int)b.mem.size();
  for (Problem* p : b.mem) {
    if (p->n + p->gcap > INT_MAX) { set_error("too many nodes for 32-bit neighbor indices"); return SPHGPU_ERR_CAPACITY; }
  }
  for (int attempt = 0; attempt < 6; ++attempt) {
    SPH_TRY(plan_capacities(b));
    SPH_TRY(launch_build(b));
    const int slots[6] = {SC_G, SC_TOTAL, SC_MAXCOUNT, SC_PAIRS, SC_NCELLS, -1};
    std::vector<double> r;
    SPH_TRY(batch_gather(b, slots, 6, r));
    bool redo = false;
    for (int m = 0; m < nm; ++m) {
      Problem& p = *b.mem[m];
      const int herr = (int)r[m*6 + 5];
      p.G = asI64(r[m*6]);
      p.ntot = p.n + p.G;
      p.E = asI64(r[m*6 + 1]);
      p.maxCount = asI32(r[m*6 + 2]);
      p.pairs = asI64(r[m*6 + 3]);
      p.ncells = asI64(r[m*6 + 4]);
      if (herr) cudaMemsetAsync(p.d_err, 0, sizeof(int), b.stream);
      if ((herr & DERR_NBR_CAPACITY) || p.maxCount > p.maxNbr) {
        set_error("a node has more neighbors than max_neighbors");
        return SPHGPU_ERR_CAPACITY;
      }
      if (herr & DERR_GHOST_CHAIN) {
        set_error("a ghost image was imaged twice through one periodic axis");
        return SPHGPU_ERR_UNSUPPORTED;
      }
      if (herr & DERR_NONPOSITIVE) {
        set_error("non-positive or non-finite smoothing scale");
        return SPHGPU_ERR_NUMERIC;
      }
      if (herr & DERR_GHOST_CAPACITY) { p.G = 2*p.gcap; redo = true; }        // ghost count unknown: double
      if (herr & DERR_ENTRY_CAPACITY) redo = true;                           // p.E is the true entry count
      if (herr & DERR_LIST_CAPACITY) { p.fillCap = p.maxCount + p.maxCount/4 + 8; redo = true; }
      else if (p.fillCap > 2*p.maxCount + 64) p.fillCap = 0;                 // re-plan a tighter list
    }
    if (!redo) return SPHGPU_OK;
    SPH_CHECK(cudaStreamSynchronize(b.stream));
  }
  set_error("neighbor build: capacities did not converge");
  return SPHGPU_ERR_CAPACITY;
}

}  // namespace sphgpu
