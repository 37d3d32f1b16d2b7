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
// blocks per member of the streaming passes (member-local grid stride)
constexpr int64_t kStreamBlocks = 148*4;
constexpr float kFilterTol = 1.0e-3f;
// shared memory for the per-thread lists of a 32-thread block (larger lists
// take the warp schedule)
constexpr size_t kMaxListSmem = 200*1024;
// blocks of 256 threads per SM the thread walk is compiled for
#ifndef NBR_THREAD_MIN_BLOCKS
#define NBR_THREAD_MIN_BLOCKS 4
#endif

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
  g.reach = (float)M.scal[SC_REACH];
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
  for (int b = 0; b < 6; ++b) s[SC_PHMAX + b] = 0.0;
  s[SC_LMAXALL] = 0.0;
  unsigned long long* bb = reinterpret_cast<unsigned long long*>(s + SC_BOUNDS);
  for (int a = 0; a < 3; ++a) { bb[a] = ~0ULL; bb[3 + a] = 0ULL; }
  bb[6] = 0ULL;
}

// 1/min(eig(H)) (hmaxi[i]) and max(eig(H)) (hmaxi[n + i]) of every internal
// node, once per build (ghosts share their root's H, so every boundary pass,
// the cell size and the pre-test records read them from here); the bounding
// box of the internal nodes and the largest 1/min(eig(H)) (SC_BOUNDS); the
// largest max(eig(H)) of the problem (with the largest 1/min(eig(H)) it
// bounds the FP32 pre-test error).
// Fixed grid (member-local grid stride): each thread accumulates its nodes'
// bounds, then one set of atomics per block.
__global__ void __launch_bounds__(kGhostThreads) node_hmax_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  double lmax = 0.0, h = 0.0;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = mb.block*(int64_t)blockDim.x + threadIdx.x; i < M.n; i += (int64_t)mb.blocks*blockDim.x) {
    const V3 ev = eigenValues(nodeH(M, i));
    const double hi1 = 1.0/vmin(ev);
    M.hmaxi[i] = hi1;
    h = fmax(h, hi1);
    double l = vmax(ev);
    M.hmaxi[M.n + i] = l;
    if (!(l < 1.0e300)) l = 1.0e300;           // degenerate H: no FP32 pre-test
    lmax = dmax(lmax, l);
    const V3 r = nodePos(M, i);
    lo[0] = fmin(lo[0], r.x); lo[1] = fmin(lo[1], r.y); lo[2] = fmin(lo[2], r.z);
    hi[0] = fmax(hi[0], r.x); hi[1] = fmax(hi[1], r.y); hi[2] = fmax(hi[2], r.z);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lmax = dmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    h = fmax(h, __shfl_xor_sync(0xffffffffu, h, o));
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  __shared__ double sh[kGhostThreads/32][8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) { sh[w][a] = lo[a]; sh[w][3 + a] = hi[a]; }
    sh[w][6] = h;
    sh[w][7] = lmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) {
      for (int a = 0; a < 3; ++a) { lo[a] = fmin(lo[a], sh[ww][a]); hi[a] = fmax(hi[a], sh[ww][3 + a]); }
      h = fmax(h, sh[ww][6]);
      lmax = dmax(lmax, sh[ww][7]);
    }
    unsigned long long* out = reinterpret_cast<unsigned long long*>(M.scal + SC_BOUNDS);
    if (h > 0.0) {
      for (int a = 0; a < 3; ++a) {
        atomicMin(out + a, orderedBits(lo[a]));
        atomicMax(out + 3 + a, orderedBits(hi[a]));
      }
      atomicMax(out + 6, orderedBits(h));
    }
    if (lmax > 0.0)
      atomicMax(reinterpret_cast<unsigned long long*>(M.scal + SC_LMAXALL),
                (unsigned long long)__double_as_longlong(lmax));
  }
}

__device__ __forceinline__ double nodeHmax(const Member& M, int64_t k) {
  return M.hmaxi[k < M.n ? k : M.groot[k - M.n]];
}

// Items of a member in a fixed grid: member-local grid stride.
#define FOR_ITEMS(t, count) \
  for (int64_t t = mb.block*(int64_t)blockDim.x + threadIdx.x; t < (count); t += (int64_t)mb.blocks*blockDim.x)

// Internal nodes within kernelExtent*max(1/min(eig(H))) of a periodic plane
// (with a relative margin): the only internal nodes a boundary pass can
// image or count into its hmax.  Flags into counts[0:n].
__global__ void __launch_bounds__(kGhostThreads) near_flag_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const unsigned long long* bb = reinterpret_cast<const unsigned long long*>(M.scal + SC_BOUNDS);
  const double reach = M.prm.kernelExtent*fromOrderedBits(bb[6])*(1.0 + 1.0e-6);
  FOR_ITEMS(i, M.n) {
    const V3 r = nodePos(M, i);
    int f = 0;
    for (int a = 0; a < 3; ++a) {
      if (!M.prm.bcs.periodic[a]) continue;
      const PlanarBC& bc = M.prm.bcs.bc[2*a];
      if (dmin(minimumDistance(bc.exit, r), minimumDistance(bc.enter, r)) <= reach) f = 1;
    }
    M.counts[i] = f;
  }
}

// The near-plane list, ascending, into cidx[0:nnear] (cidx is free until
// the cell pass), and its length.
__global__ void __launch_bounds__(kGhostThreads) near_list_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  FOR_ITEMS(i, M.n) {
    if (M.counts[i]) M.cidx[M.offsets[i]] = (int32_t)i;
  }
  if (mb.block == 0 && threadIdx.x == 0) setScalI(M.scal, SC_NNEAR, M.offsets[M.n]);
}

// Item t of a boundary pass: the near-plane internal nodes in ascending
// order, then the ghosts made so far in creation order (the order in which
// the reference visits a NodeList's nodes).
__device__ __forceinline__ int64_t passItems(const Member& M) {
  return scalI(M.scal, SC_NNEAR) + scalI(M.scal, SC_NTOT) - M.n;
}
__device__ __forceinline__ int64_t passNode(const Member& M, int64_t t, int64_t nnear) {
  return t < nnear ? (int64_t)M.cidx[t] : M.n + (t - nnear);
}

// hmax of PlanarBoundary::setGhostNodes: max 1/min(eig(H)) over nodes within
// kernelExtent*hmaxi of either plane.
__global__ void __launch_bounds__(kGhostThreads) ghost_hmax_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  double best = 0.0;
  if (M.prm.bcs.periodic[b >> 1]) {
    const PlanarBC& bc = M.prm.bcs.bc[b];
    const int64_t nnear = scalI(M.scal, SC_NNEAR);
    FOR_ITEMS(t, passItems(M)) {
      const int64_t k = passNode(M, t, nnear);
      const V3 r = nodePos(M, k);
      const double hmaxi = nodeHmax(M, k);
      if (dmin(minimumDistance(bc.exit, r), minimumDistance(bc.enter, r)) < M.prm.kernelExtent*hmaxi)
        best = dmax(best, hmaxi);
    }
  }
  for (int o = 16; o > 0; o >>= 1) best = dmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(M.scal + SC_HMAX), (unsigned long long)__double_as_longlong(best));
}

__global__ void __launch_bounds__(kGhostThreads) ghost_flag_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const double hmax = M.scal[SC_HMAX];
  const bool on = M.prm.bcs.periodic[b >> 1] && hmax > 0.0;
  const int64_t nnear = scalI(M.scal, SC_NNEAR);
  FOR_ITEMS(t, passItems(M)) {
    int f = 0;
    if (on) {
      const V3 r = nodePos(M, passNode(M, t, nnear));
      const double disti = signedDistance(M.prm.bcs.bc[b].exit, r)/hmax;
      f = (disti >= 0.0 && disti <= M.prm.kernelExtent) ? 1 : 0;
    }
    M.counts[t] = f;
  }
}

__global__ void __launch_bounds__(kGhostThreads) ghost_scatter_kernel(const Member* mem, BlockMap bm, int b) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int64_t n = M.n;
  const int64_t ntot = scalI(M.scal, SC_NTOT);
  const int64_t nnear = scalI(M.scal, SC_NNEAR);
  const PlanarBC& bc = M.prm.bcs.bc[b];
  const int axis = b >> 1;
  FOR_ITEMS(t, passItems(M)) {
    if (!M.counts[t]) continue;
    const int64_t k = passNode(M, t, nnear);
    const int64_t g = (ntot - n) + M.offsets[t];     // ghost index of the new image
    if (g >= M.gcap) {
      atomicOr(M.err, DERR_GHOST_CAPACITY);
      continue;
    }
    const V3 gp = mapPositionThroughPlanes(nodePos(M, k), bc.exit, bc.enter);
    const int32_t root = k < n ? (int32_t)k : M.groot[k - n];
    uint32_t code = k < n ? 0u : M.gcode[k - n];
    if ((code >> (2*axis)) & 3u) atomicOr(M.err, DERR_GHOST_CHAIN);
    code |= (uint32_t)((b & 1) + 1) << (2*axis);
    M.groot[g] = root;
    M.gcode[g] = code;
    M.gpos[g] = gp.x; M.gpos[M.gcap + g] = gp.y; M.gpos[2*M.gcap + g] = gp.z;
  }
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

// ---------------------------------------------------------------- fused ghost passes
// The six boundary passes in one cooperative launch, for a batch of a few
// members: the per-pass hmax, the flags, their prefix sum and the scatter
// of the new images, separated by grid barriers.  An item's share of a
// pass's hmax depends on the item alone, so the near-plane nodes give their
// shares to every pass before the first one, and each new image to the
// passes after its own as it is made; a pass then needs two barriers (after
// its block counts, after its scatter).  Block k takes the k-th contiguous
// chunk of a pass's items and numbers its images in item order, so the
// images, their order and the error bits are those of the per-pass launches.
__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
constexpr int kFusedGhostMembers = 4;
#ifndef FUSED_GHOST_MIN_BLOCKS
#define FUSED_GHOST_MIN_BLOCKS 2
#endif
constexpr int kFusedGhostBlocks = 148*FUSED_GHOST_MIN_BLOCKS;
constexpr int kBarrierPolls = 1 << 21;

// Grid barrier of a cooperative launch (every block resident).  bar[0]
// counts arrivals, bar[1] is the generation.  A block that polls more than
// kBarrierPolls times records DERR_BARRIER in every member and returns
// false; its launch then ends without finishing the passes.
__device__ bool grid_barrier(unsigned int* bar, const Member* mem, int nm) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int* gen = bar + 1;
    const unsigned int g0 = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      int polls = 0;
      while (*gen == g0) {
        if (++polls > kBarrierPolls) {
          for (int m = 0; m < nm; ++m) atomicOr(mem[m].err, DERR_BARRIER);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// position of item node k (ghost positions are written during the launch:
// read through L2)
__device__ __forceinline__ V3 fusedPos(const Member& M, int64_t k) {
  const int64_t n = M.n;
  if (k < n) return V3{M.S[S_X*n + k], M.S[S_Y*n + k], M.S[S_Z*n + k]};
  const int64_t g = k - n;
  return V3{__ldcg(M.gpos + g), __ldcg(M.gpos + M.gcap + g), __ldcg(M.gpos + 2*M.gcap + g)};
}
__device__ __forceinline__ int32_t fusedRoot(const Member& M, int64_t k) {
  return k < M.n ? (int32_t)k : __ldcg(M.groot + (k - M.n));
}

// an item's shares of the hmax of passes [from, 6) (ghost_hmax_kernel's test)
__device__ __forceinline__ void hmaxShares(const Member& M, const V3& r, double hmaxi, int from, double* loc) {
#pragma unroll
  for (int b = 0; b < 6; ++b) {
    if (b < from || !M.prm.bcs.periodic[b >> 1]) continue;
    const PlanarBC& bc = M.prm.bcs.bc[b];
    if (dmin(minimumDistance(bc.exit, r), minimumDistance(bc.enter, r)) < M.prm.kernelExtent*hmaxi)
      loc[b] = dmax(loc[b], hmaxi);
  }
}

// block maxima of the shares into the member's pass hmax words
__device__ void hmaxFlush(const Member& M, double* loc, int from) {
  __shared__ double red[6][kGhostThreads/32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int b = 0; b < 6; ++b) {
    double v = loc[b];
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) red[b][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6 && (int)threadIdx.x >= from) {
    double v = 0.0;
    for (int k = 0; k < kGhostThreads/32; ++k) v = dmax(v, red[threadIdx.x][k]);
    if (v > 0.0)
      atomicMax(reinterpret_cast<unsigned long long*>(M.scal + SC_PHMAX + threadIdx.x),
                (unsigned long long)__double_as_longlong(v));
  }
  __syncthreads();
}

// ghost_flag_kernel's test of item t for pass b
__device__ __forceinline__ bool ghostFlag(const Member& M, int b, double hmax, int64_t t, int64_t nnear) {
  if (!M.prm.bcs.periodic[b >> 1] || !(hmax > 0.0)) return false;
  const V3 r = fusedPos(M, passNode(M, t, nnear));
  const double disti = signedDistance(M.prm.bcs.bc[b].exit, r)/hmax;
  return disti >= 0.0 && disti <= M.prm.kernelExtent;
}

__global__ void __launch_bounds__(kGhostThreads, FUSED_GHOST_MIN_BLOCKS) ghost_passes_fused_kernel(const Member* mem, int nm, unsigned int* fuse) {
  unsigned int* bar = fuse;
  int64_t* blk = reinterpret_cast<int64_t*>(fuse + 2);      // [member][block] counts of a pass
  const int nb = gridDim.x, kb = blockIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ int64_t wsum[kGhostThreads/32];
  __shared__ int64_t sG[kFusedGhostMembers];
  __shared__ int64_t sPre, sTot;
  if (threadIdx.x < kFusedGhostMembers) sG[threadIdx.x] = 0;
  // the near-plane nodes' shares of every pass's hmax
  for (int m = 0; m < nm; ++m) {
    const Member& M = mem[m];
    const int64_t nnear = scalI(M.scal, SC_NNEAR);
    double loc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t t = kb*(int64_t)blockDim.x + threadIdx.x; t < nnear; t += (int64_t)nb*blockDim.x) {
      const int64_t k = M.cidx[t];
      hmaxShares(M, nodePos(M, k), M.hmaxi[k], 0, loc);
    }
    hmaxFlush(M, loc, 0);
  }
  if (!grid_barrier(bar, mem, nm)) return;
  for (int b = 0; b < 6; ++b) {
    bool any = false;
    for (int m = 0; m < nm; ++m) any = any || mem[m].prm.bcs.periodic[b >> 1];
    if (!any) continue;
    // flags of this block's chunk: the block's count
    for (int m = 0; m < nm; ++m) {
      const Member& M = mem[m];
      const int64_t nnear = scalI(M.scal, SC_NNEAR);
      const int64_t items = nnear + sG[m];
      const int64_t chunk = (items + nb - 1)/nb;
      const int64_t c0 = imin64(items, kb*chunk), c1 = imin64(items, c0 + chunk);
      const double hmax = __longlong_as_double((long long)__ldcg(reinterpret_cast<const unsigned long long*>(M.scal + SC_PHMAX + b)));
      int64_t cnt = 0;
      for (int64_t t = c0 + threadIdx.x; t < c1; t += blockDim.x) cnt += ghostFlag(M, b, hmax, t, nnear) ? 1 : 0;
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      if (lane == 0) wsum[w] = cnt;
      __syncthreads();
      if (threadIdx.x == 0) {
        int64_t s = 0;
        for (int k = 0; k < kGhostThreads/32; ++k) s += wsum[k];
        blk[m*nb + kb] = s;
      }
      __syncthreads();
    }
    if (!grid_barrier(bar, mem, nm)) return;
    // the block's offset among the chunks, the pass total, the scatter
    for (int m = 0; m < nm; ++m) {
      const Member& M = mem[m];
      const int64_t n = M.n;
      const int64_t nnear = scalI(M.scal, SC_NNEAR);
      const int64_t G = sG[m];
      const int64_t items = nnear + G;
      const int64_t chunk = (items + nb - 1)/nb;
      const int64_t c0 = imin64(items, kb*chunk), c1 = imin64(items, c0 + chunk);
      const double hmax = __longlong_as_double((long long)__ldcg(reinterpret_cast<const unsigned long long*>(M.scal + SC_PHMAX + b)));
      int64_t pre = 0, tot = 0;
      for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const int64_t c = __ldcg(blk + m*nb + k);
        tot += c;
        if (k < kb) pre += c;
      }
      for (int o = 16; o > 0; o >>= 1) {
        pre += __shfl_xor_sync(0xffffffffu, pre, o);
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
      }
      __shared__ int64_t wpre[kGhostThreads/32];
      if (lane == 0) { wsum[w] = tot; wpre[w] = pre; }
      __syncthreads();
      if (threadIdx.x == 0) {
        int64_t a = 0, c = 0;
        for (int k = 0; k < kGhostThreads/32; ++k) { a += wpre[k]; c += wsum[k]; }
        sPre = a;
        sTot = c;
      }
      __syncthreads();
      int64_t next = G + sPre;                         // ghost index of this block's first image
      const PlanarBC& bc = M.prm.bcs.bc[b];
      const int axis = b >> 1;
      double loc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      for (int64_t base = c0; base < c1; base += blockDim.x) {
        const int64_t t = base + threadIdx.x;
        const bool f = t < c1 && ghostFlag(M, b, hmax, t, nnear);
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wsum[w] = __popc(bal);
        __syncthreads();
        int64_t off = 0, tileTot = 0;
        for (int k = 0; k < kGhostThreads/32; ++k) {
          if (k < w) off += wsum[k];
          tileTot += wsum[k];
        }
        off += __popc(bal & ((1u << lane) - 1u));
        if (f) {
          const int64_t k = passNode(M, t, nnear);
          const int64_t g = next + off;
          if (g >= M.gcap) {
            atomicOr(M.err, DERR_GHOST_CAPACITY);
          } else {
            const V3 gp = mapPositionThroughPlanes(fusedPos(M, k), bc.exit, bc.enter);
            const int32_t root = fusedRoot(M, k);
            uint32_t code = k < n ? 0u : __ldcg(M.gcode + (k - n));
            if ((code >> (2*axis)) & 3u) atomicOr(M.err, DERR_GHOST_CHAIN);
            code |= (uint32_t)((b & 1) + 1) << (2*axis);
            M.groot[g] = root;
            M.gcode[g] = code;
            M.gpos[g] = gp.x; M.gpos[M.gcap + g] = gp.y; M.gpos[2*M.gcap + g] = gp.z;
            hmaxShares(M, gp, M.hmaxi[root], b + 1, loc);
          }
        }
        next += tileTot;
        __syncthreads();
      }
      hmaxFlush(M, loc, b + 1);
      if (threadIdx.x == 0) {
        int64_t g = G + sTot;
        if (g > M.gcap) {
          if (kb == 0) atomicOr(M.err, DERR_GHOST_CAPACITY);
          g = M.gcap;
        }
        sG[m] = g;
      }
      __syncthreads();
    }
    if (!grid_barrier(bar, mem, nm)) return;
  }
  if (kb == 0 && threadIdx.x < nm) {
    const Member& M = mem[threadIdx.x];
    setScalI(M.scal, SC_NTOT, M.n + sG[threadIdx.x]);
    setScalI(M.scal, SC_G, sG[threadIdx.x]);
    M.scal[SC_HMAX] = 0.0;
  }
}

// ---------------------------------------------------------------- cells
// Uniform grid of cells of edge >= kappa*max(1/lambda_min(H)) (the margin
// covers the libm difference of the eigenvalue solve for anisotropic H),
// enlarged until the cells fit the cell buffers (larger cells only widen the
// candidate set).  Also resets the walk's counters and sets the FP32
// pre-test tolerance: only when max h / min h over the problem is <= 100.
__global__ void grid_kernel(const Member* mem, int nmem) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const Member& M = mem[m];
  const unsigned long long* bb = reinterpret_cast<const unsigned long long*>(M.scal + SC_BOUNDS);
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) { lo[a] = fromOrderedBits(bb[a]); hi[a] = fromOrderedBits(bb[3 + a]); }
  const double hmaxAll = fromOrderedBits(bb[6]);
  // ghosts lie within kappa*hmax (<= kappa*hmaxAll) beyond the periodic
  // planes; elsewhere they share their root's coordinates
  const double reach = M.prm.kernelExtent*hmaxAll*1.001 + 1.0e-300;
  for (int a = 0; a < 3; ++a) {
    if (!M.prm.bcs.periodic[a]) continue;
    const PlanarBC& bc = M.prm.bcs.bc[2*a];
    const double p0 = (&bc.enter.point.x)[a], p1 = (&bc.exit.point.x)[a];
    lo[a] = fmin(lo[a], fmin(p0, p1) - reach);
    hi[a] = fmax(hi[a], fmax(p0, p1) + reach);
  }
  const int sub = M.grid.sub > 1 ? M.grid.sub : 1;
  double cell = M.prm.kernelExtent*hmaxAll*1.001/sub;
  if (!(cell > 0.0) || !(cell < 1.0e300)) {
    atomicOr(M.err, DERR_NONPOSITIVE);
    cell = 1.0;
  }
  const int64_t maxCells = M.cellcap < ((int64_t)1 << 26) ? M.cellcap : ((int64_t)1 << 26);
  int64_t dim[3] = {1, 1, 1}, ncells = 1;
  {
    // cells at the natural size, for the next build's capacity
    double want = 1.0;
    for (int a = 0; a < 3; ++a) want *= fmin((hi[a] - lo[a])/cell + 1.0, (double)(1 << 20));
    setScalI(M.scal, SC_CELLSWANTED, want < 1.0e15 ? (int64_t)want : (int64_t)1 << 50);
  }
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
  // largest h over smallest h of the problem (>= every node's condition number)
  const double spread = hmaxAll*M.scal[SC_LMAXALL];
  s[7] = (M.grid.filterTol > 0.0f && spread > 0.0 && spread <= 100.0) ? (double)M.grid.filterTol : 0.0;
  // the largest kernel reach in cells (<= sub), for the walks' pruning
  M.scal[SC_REACH] = M.prm.kernelExtent*hmaxAll/cell;
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
  FOR_ITEMS(c, scalI(M.scal, SC_NCELLS)) M.cellFill[c] = 0;
}

__global__ void __launch_bounds__(kGhostThreads) cell_index_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const Grid g = loadGrid(M);
  FOR_ITEMS(k, allNodes(M)) {
    const V3 r = nodePos(M, k);
    const int cx = cellCoord(r.x, g.lo[0], g.cell, g.dim[0]);
    const int cy = cellCoord(r.y, g.lo[1], g.cell, g.dim[1]);
    const int cz = cellCoord(r.z, g.lo[2], g.cell, g.dim[2]);
    const int c = (cz*g.dim[1] + cy)*g.dim[0] + cx;
    M.cidx[k] = c;
    atomicAdd(M.cellFill + c, 1);
  }
}

// Cell-ordered candidate arrays (Problem::cand), one slot per node:
//   pre     [candcap] float4:   FP32 offsets of the position from the lower
//                               corner of the node's cell, and
//                               k2hi/min eig(H)^2 (k2hi the upper edge of the
//                               pre-test band): beyond that r^2 the node's own
//                               eta^2 lies above the band
//   lmax    [candcap] float:    FP32 max eig(H)
// and sortedIdx[slot], the node of each slot.  The walks read only `pre` for
// most candidates; `lmax` when the i-side test alone does not decide, and
// the FP64 position and H of the node (state, ghost positions) for the
// candidates the FP32 pre-test cannot decide.
struct NbrArrays {
  const float4* pre;
  const float* lmax;
};

__device__ __forceinline__ NbrArrays nbrArrays(const Member& M) {
  const double* c = static_cast<const double*>(M.cand);
  NbrArrays a;
  a.pre = reinterpret_cast<const float4*>(c);
  a.lmax = reinterpret_cast<const float*>(c + 2*M.candcap);
  return a;
}

__device__ __forceinline__ float symEta2F(const float* h, float x, float y, float z) {
  const float ex = __fmaf_rn(h[0], x, __fmaf_rn(h[1], y, h[2]*z));
  const float ey = __fmaf_rn(h[1], x, __fmaf_rn(h[3], y, h[4]*z));
  const float ez = __fmaf_rn(h[2], x, __fmaf_rn(h[4], y, h[5]*z));
  return __fmaf_rn(ex, ex, __fmaf_rn(ey, ey, ez*ez));
}

// The walking node: FP32 H and cell offsets for the pre-test, its cell, its
// sorted slot and node index (the exact test re-reads its FP64 state).
struct Walker {
  float hf[6];
  float lam2;          // isotropic H = lam I: lam^2 (then eta_i^2 = lam^2 |r|^2)
  float T;             // k2hi/min eig(H)^2: beyond r^2 = T the node's own eta^2 exceeds the band
  bool iso;
  float ox, oy, oz;
  int cx, cy, cz;
  int32_t slot;
  int32_t idx;
};

// Walker of sorted slot s; idx >= n marks a ghost slot (no walk).
__device__ __forceinline__ Walker makeWalker(const Member& M, const NbrArrays& a, const Grid& g, int32_t s) {
  Walker w;
  w.slot = s;
  w.idx = __ldg(M.sortedIdx + s);
  if (w.idx >= M.n) return w;
  const V3 r = nodePos(M, w.idx);
  const Sym H = nodeH(M, w.idx);
  w.hf[0] = (float)H.xx; w.hf[1] = (float)H.xy; w.hf[2] = (float)H.xz;
  w.hf[3] = (float)H.yy; w.hf[4] = (float)H.yz; w.hf[5] = (float)H.zz;
  w.iso = H.xy == 0.0 && H.xz == 0.0 && H.yz == 0.0 && H.xx == H.yy && H.xx == H.zz;
  w.lam2 = w.hf[0]*w.hf[0];
  const float4 p = __ldg(a.pre + s);
  w.ox = p.x; w.oy = p.y; w.oz = p.z;
  w.T = p.w;
  w.cx = cellCoord(r.x, g.lo[0], g.cell, g.dim[0]);
  w.cy = cellCoord(r.y, g.lo[1], g.cell, g.dim[1]);
  w.cz = cellCoord(r.z, g.lo[2], g.cell, g.dim[2]);
  return w;
}

// Distance, in cells, from a walker at fraction f of its cell to the cell d
// cells away along one axis (0 for its own cell); a lower bound for every
// node of that cell.
__device__ __forceinline__ float axisGap(int d, float f) {
  return d > 0 ? fmaxf(0.0f, (float)d - f) : (d < 0 ? fmaxf(0.0f, (float)(-d - 1) + f) : 0.0f);
}

// One x-row of the walk window: the candidate slot range [start, end) of its
// cells x0..x1 (contiguous in the sorted order), trimmed with SUB > 1 to
// the cells within the kernel reach, and the ends of its first cells (a
// candidate's cell follows from its slot).
template<int SUB>
struct Row {
  int32_t start, end;  // slots (every slot index fits in 32 bits)
  int32_t e[2*SUB];
  int x0;
};

template<int SUB>
__device__ __forceinline__ Row<SUB> loadRow(const Member& M, const Grid& g, const Walker& w, int y, int z,
                                            float fx, float gyz, float rc2) {
  int x0 = w.cx - SUB > 0 ? w.cx - SUB : 0;
  int x1 = w.cx + SUB < g.dim[0] - 1 ? w.cx + SUB : g.dim[0] - 1;
  if (SUB > 1) {
    // the gaps grow with |x - cx|: trim the far cells at both ends
    while (x0 < w.cx) { const float gx = axisGap(x0 - w.cx, fx); if (gx*gx + gyz <= rc2) break; ++x0; }
    while (x1 > w.cx) { const float gx = axisGap(x1 - w.cx, fx); if (gx*gx + gyz <= rc2) break; --x1; }
  }
  const int64_t* cs = M.cellStart + (int64_t)(z*g.dim[1] + y)*g.dim[0] + x0;
  const int nx = x1 - x0 + 1;
  Row<SUB> r;
  r.x0 = x0;
  r.start = (int32_t)cs[0];
  r.end = (int32_t)cs[nx];
#pragma unroll
  for (int c = 0; c < 2*SUB; ++c) r.e[c] = c + 1 < nx ? (int32_t)cs[c + 1] : r.end;
  return r;
}

template<int SUB>
__device__ __forceinline__ float rowDxc(const Row<SUB>& r, const Walker& w, int32_t k, float cellf) {
  int xc = r.x0 - w.cx;
#pragma unroll
  for (int c = 0; c < 2*SUB; ++c) xc += (k >= r.e[c]);
  return (float)xc*cellf;
}

// The exact FP64 predicate for nodes i and j (the walks reach it for the
// few candidates the pre-test leaves undecided).
__device__ __forceinline__ bool exactTest(const Member& M, int32_t i, int32_t j, double k2) {
  const int64_t n = M.n;
  const double* S = M.S;
  const V3 ri{S[S_X*n + i], S[S_Y*n + i], S[S_Z*n + i]};     // the walker is an internal node
  const V3 rj = nodePos(M, j);
  const V3 rij{ri.x - rj.x, ri.y - rj.y, ri.z - rj.z};
  const Sym Hi{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
               S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
  return mag2(sdot(Hi, rij)) <= k2 || mag2(sdot(nodeH(M, j), rij)) <= k2;
}

// ConnectivityMap predicate |H_i r_ij|^2 <= kappa^2 || |H_j r_ij|^2 <= kappa^2
// (src/Neighbor/ConnectivityMapInline.hh:169-186) for candidate slot k, whose
// cell corner lies at (dxc, dyc, dzc) from the walker's (FP32).
// With tol > 0 a FP32 pre-test decides every pair whose eta^2 lies clearly
// outside the band kappa^2 (1 -+ tol): eta_i^2 from the FP32 H_i, eta_j^2
// bounded by min/max eig(H_j)^2 |r_ij|^2, r_ij from the cell offsets.  The
// pre-test error is below 1e-6 (max h/min h over the problem) relative, and
// tol (1e-3) is only set when that ratio is <= 100, so it never decides a
// pair the exact test would decide otherwise.  Undecided pairs take the
// exact FP64 test in the reference's operation order.  eta^2 of either node
// lies in [min eig(H)^2 r^2, max eig(H)^2 r^2]: a candidate beyond the band
// for the smaller of the two minimum eigenvalues is rejected from r^2 alone
// (most candidates of the window); each record carries that r^2 bound,
// k2hi/min eig(H)^2, so the test is one comparison with the larger of the
// two nodes' bounds.
__device__ __forceinline__ bool candTest(const Member& M, const NbrArrays& a, const Walker& w, int32_t k,
                                         float dxc, float dyc, float dzc, double k2, float k2lo, float k2hi,
                                         bool pretest) {
  if (pretest) {
    const float4 c = __ldg(a.pre + k);
    const float fx = (w.ox - c.x) - dxc, fy = (w.oy - c.y) - dyc, fz = (w.oz - c.z) - dzc;
    const float r2 = __fmaf_rn(fx, fx, __fmaf_rn(fy, fy, fz*fz));
    if (r2 > fmaxf(w.T, c.w)) return false;
    float e2i;
    if (w.iso) e2i = w.lam2*r2;          // the common case: H = lam I
    else e2i = symEta2F(w.hf, fx, fy, fz);
    if (e2i <= k2lo) return true;
    if (e2i > k2hi && r2 > c.w) return false;
    const float lm = __ldg(a.lmax + k);
    if (lm*lm*r2 <= k2lo) return true;
  }
  return exactTest(M, w.idx, __ldg(M.sortedIdx + k), k2);
}

__global__ void __launch_bounds__(kGhostThreads) cell_scatter_kernel(const Member* mem, BlockMap bm) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const Grid g = loadGrid(M);
  double* base = static_cast<double*>(M.cand);
  float4* pre = reinterpret_cast<float4*>(base);
  float* lmax = reinterpret_cast<float*>(base + 2*M.candcap);
  // the pre-test's upper band edge, as the walks form it
  const float k2f = (float)(M.prm.kernelExtent*M.prm.kernelExtent);
  const double k2hi = (double)(k2f*(1.0f + g.filterTol));
  FOR_ITEMS(k, allNodes(M)) {
    const int c = M.cidx[k];
    const int64_t slot = M.cellStart[c] + atomicAdd(M.cellFill + c, 1);
    M.sortedIdx[slot] = (int32_t)k;
    const V3 r = nodePos(M, k);
    const int cx = cellCoord(r.x, g.lo[0], g.cell, g.dim[0]);
    const int cy = cellCoord(r.y, g.lo[1], g.cell, g.dim[1]);
    const int cz = cellCoord(r.z, g.lo[2], g.cell, g.dim[2]);
    const int64_t root = k < M.n ? k : M.groot[k - M.n];
    const double hm = M.hmaxi[root];
    pre[slot] = make_float4((float)(r.x - (g.lo[0] + cx*g.cell)), (float)(r.y - (g.lo[1] + cy*g.cell)),
                            (float)(r.z - (g.lo[2] + cz*g.cell)), (float)(k2hi*hm*hm));
    lmax[slot] = (float)M.hmaxi[M.n + root];
  }
}

// Thread per internal node, nodes taken in cell-sorted order so that the
// threads of a warp share their candidate rows (L1 broadcast).  The 27
// neighbouring cells are walked as 9 x-rows (three cells each, contiguous in
// the sorted order) and the ConnectivityMap predicate is applied.
// COUNT pass: per-node counts and their maximum.  FILL pass: the neighbor
// indices are insertion-sorted into a per-thread shared-memory list of
// capacity `cap` (element c of thread t at lst[c*blockDim + t], conflict
// free) and stored ascending at offsets[i].
// A member with a stash (Grid::stashCap > 0) builds its lists in the COUNT
// pass too and stores them ascending in the stash, element c of sorted slot s
// at stash[c*stashStride + s]; nbr_compact_thread_kernel then moves them to
// offsets[i], and the FILL pass does not run for it.
template<bool FILL, int SUB>
__global__ void __launch_bounds__(256, SUB == 1 ? NBR_THREAD_MIN_BLOCKS : 1) nbr_thread_kernel(const Member* mem, BlockMap bm, int cap, int maxNbr) {
  extern __shared__ int32_t lst[];
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int tid = threadIdx.x;
  const int bd = blockDim.x;
  const int64_t s = mb.block*bd + tid;
  const int64_t n = M.n;
  const NbrArrays a = nbrArrays(M);
  const Grid g = loadGrid(M);
  bool active = s < allNodes(M);
  Walker me;
  if (active) {
    me = makeWalker(M, a, g, (int32_t)s);
    active = me.idx < n;
  }
  // list capacity: the shared-memory list (FILL) or the member's stash (COUNT)
  const int lcap = FILL ? cap : M.grid.stashCap;
  const bool collect = FILL || lcap > 0;
  int count = 0, above = 0;
  if (active) {
    const double k2 = M.prm.kernelExtent*M.prm.kernelExtent;
    const float k2f = (float)k2;
    const bool pretest = g.filterTol > 0.0f;
    const float k2lo = k2f*(1.0f - g.filterTol), k2hi = k2f*(1.0f + g.filterTol);
    const float cellf = (float)g.cell;
    const int32_t i = me.idx;
    // window of +-SUB cells; with SUB > 1 the rows and cells farther than the
    // largest kernel reach (in cells, with a margin) are skipped
    const float rc2 = g.reach*g.reach*1.0001f;
    auto accept = [&](int32_t k) {
      if (collect) {
        const int32_t j = __ldg(M.sortedIdx + k);
        if (count < lcap) {
          int p = count;
          while (p > 0) {
            const int32_t prev = lst[(p - 1)*bd + tid];
            if (prev < j) break;
            lst[p*bd + tid] = prev;
            --p;
          }
          lst[p*bd + tid] = j;
        }
        above += (j > i);
      }
      ++count;
    };
    {
      const float fx = me.ox/cellf, fy = me.oy/cellf, fz = me.oz/cellf;
      for (int dz = -SUB; dz <= SUB; ++dz) {
        const int z = me.cz + dz;
        if (z < 0 || z >= g.dim[2]) continue;
        const float gz = axisGap(dz, fz);
        const float dzc = (float)dz*cellf;
        for (int dy = -SUB; dy <= SUB; ++dy) {
          const int y = me.cy + dy;
          if (y < 0 || y >= g.dim[1]) continue;
          const float gy = axisGap(dy, fy);
          const float gyz = gy*gy + gz*gz;
          if (SUB > 1 && gyz > rc2) continue;
          const float dyc = (float)dy*cellf;
          const Row<SUB> row = loadRow<SUB>(M, g, me, y, z, fx, gyz, rc2);
          for (int32_t k = row.start; k < row.end; ++k) {
            if (k != s && candTest(M, a, me, k, rowDxc<SUB>(row, me, k, cellf), dyc, dzc, k2, k2lo, k2hi, pretest))
              accept(k);
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
    unsigned long long b = (unsigned long long)above;
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
    if ((tid & 31) == 0 && b) atomicAdd(reinterpret_cast<unsigned long long*>(M.scal + SC_PAIRS), b);
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

// Warp per internal node (warps dealt over the sorted slots, ghost slots
// idle): walk the 27 neighbouring cells, apply the ConnectivityMap
// predicate, count (FILL=false) or collect, sort ascending and store
// (FILL=true) the neighbor indices.  Used when the candidate sets are large
// (many nodes per cell), where a warp per node keeps the SMs full.  `cap` is
// the per-warp list capacity (a power of two >= 32).  A member with a stash
// (Grid::stashCap > 0) collects and sorts in the COUNT pass and stores the
// list of node i at stash[i*stashCap]; nbr_compact_warp_kernel moves it to
// offsets[i].
template<bool FILL, int SUB>
__global__ void __launch_bounds__(256, SUB == 1 ? 3 : 1) nbr_walk_kernel(const Member* mem, BlockMap bm, int cap, int maxNbr) {
  extern __shared__ int32_t sbuf_all[];
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int scap = FILL ? 0 : M.grid.stashCap;
  const bool collect = FILL || scap > 0;
  int32_t* sbuf = sbuf_all + (collect ? wib*cap : 0);
  const int64_t s = (mb.block*(int64_t)blockDim.x + threadIdx.x) >> 5;
  if (s >= allNodes(M)) return;
  const NbrArrays a = nbrArrays(M);
  const Grid g = loadGrid(M);
  const Walker me = makeWalker(M, a, g, (int32_t)s);
  if (me.idx >= M.n) return;
  const int32_t i = me.idx;
  const double k2 = M.prm.kernelExtent*M.prm.kernelExtent;
  const float k2f = (float)k2;
  const bool pretest = g.filterTol > 0.0f;
  const float k2lo = k2f*(1.0f - g.filterTol), k2hi = k2f*(1.0f + g.filterTol);
  const float cellf = (float)g.cell;
  const float rc2 = g.reach*g.reach*1.0001f;
  const float fx = me.ox/cellf, fy = me.oy/cellf, fz = me.oz/cellf;
  // The window's rows, one per lane (rows outside the grid or, with SUB > 1,
  // beyond the kernel reach are empty), their candidates numbered in one
  // sequence by a warp scan: the lanes then take 32 consecutive candidates at
  // a time across row ends, so a warp iteration tests 32 candidates however
  // short the rows are.
  constexpr int NR = (2*SUB + 1)*(2*SUB + 1);
  constexpr int RW = 3 + 2*SUB;                       // start, first candidate number, x0, cell ends
  __shared__ int32_t rowTab[256/32][NR*RW];
  int32_t* R = rowTab[wib];
  int len = 0;
  if (lane < NR) {
    const int dy = lane % (2*SUB + 1) - SUB, dz = lane/(2*SUB + 1) - SUB;
    const int y = me.cy + dy, z = me.cz + dz;
    if (y >= 0 && y < g.dim[1] && z >= 0 && z < g.dim[2]) {
      const float gy = axisGap(dy, fy), gz = axisGap(dz, fz);
      const float gyz = gy*gy + gz*gz;
      if (SUB == 1 || gyz <= rc2) {
        const Row<SUB> row = loadRow<SUB>(M, g, me, y, z, fx, gyz, rc2);
        len = row.end > row.start ? row.end - row.start : 0;
        R[lane*RW] = row.start;
        R[lane*RW + 2] = row.x0;
#pragma unroll
        for (int c = 0; c < 2*SUB; ++c) R[lane*RW + 3 + c] = row.e[c];
      }
    }
  }
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane < NR) R[lane*RW + 1] = incl - len;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  __syncwarp();
  int count = 0;
  int r = 0;                                          // the lane's row (lanes only move forward)
  for (int base = 0; base < total; base += 32) {
    const int t = base + lane;
    bool pass = false;
    int32_t k = 0;
    if (t < total) {
      while (r + 1 < NR && R[(r + 1)*RW + 1] <= t) ++r;
      const int32_t* row = R + r*RW;
      k = row[0] + (t - row[1]);
      if (k != s) {
        int xc = row[2] - me.cx;
#pragma unroll
        for (int c = 0; c < 2*SUB; ++c) xc += (k >= row[3 + c]);
        const float dyc = (float)(r % (2*SUB + 1) - SUB)*cellf, dzc = (float)(r/(2*SUB + 1) - SUB)*cellf;
        pass = candTest(M, a, me, k, (float)xc*cellf, dyc, dzc, k2, k2lo, k2hi, pretest);
      }
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, pass);
    if (collect && pass) {
      const int pos = count + __popc(ballot & ((1u << lane) - 1u));
      if (pos < cap) sbuf[pos] = __ldg(M.sortedIdx + k);
    }
    count += __popc(ballot);
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
          const int32_t u = sbuf[t], v = sbuf[ixj];
          const bool up = (t & k) == 0;
          if ((u > v) == up) { sbuf[t] = v; sbuf[ixj] = u; }
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
  for (int sh = 16; sh > 0; sh >>= 1) above += __shfl_xor_sync(0xffffffffu, above, sh);
  if (lane == 0 && above)
    atomicAdd(reinterpret_cast<unsigned long long*>(M.scal + SC_PAIRS), (unsigned long long)above);
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
    if (G > 0) SPH_TRY(ensure_capacity_ghosts(p, grow(G)));
    // schedule: a warp per node once the 27-cell candidate set of the last
    // build kept 32 lanes busy, or once a thread's list would not fit in
    // shared memory
    const int lastSub = p.lastNbrCells > 0 ? p.lastNbrCells : 1;
    const double cells1 = p.cellsWanted > 0 ? (double)p.cellsWanted/(double)(lastSub*lastSub*lastSub) : 0.0;
    const double candPerNode = cells1 > 0.0 ? 27.0*(double)(p.n + p.G)/cells1 : 0.0;
    const int req = p.nbrSchedule != NBR_SCHEDULE_AUTO ? p.nbrSchedule : b.nbrSchedule;
    p.fillSchedule = (req == NBR_SCHEDULE_WARP || (req == NBR_SCHEDULE_AUTO && candPerNode > 384.0) ||
                      sizeof(int32_t)*32*(size_t)(p.fillCap > 8 ? p.fillCap : 64) > kMaxListSmem)
                         ? NBR_SCHEDULE_WARP : NBR_SCHEDULE_THREAD;
    // cells per kernel reach: one unless requested (half-reach cells test
    // fewer candidates but walk more rows; the autotuner measures both)
    const int reqCells = p.nbrCells != 0 ? p.nbrCells : b.nbrCells;
    p.grid.sub = reqCells != 0 ? reqCells : 1;
    const int sub = p.grid.sub;
    // cells the grid wants at this subdivision (the last build's, rescaled), else the hint
    const int64_t cells = cells1 > 0.0 ? (int64_t)(cells1*sub*sub*sub) + 1 : p.hintCells;
    // grow (with slack) when the buffers hold less than the wanted cells, and
    // once when the first measured count replaces the first build's guess (so
    // that a later small drift of h does not reallocate mid-run)
    const int64_t cellsNeed = cells > 0 ? grow(cells) : p.candcap/2 + 64;
    const int64_t cellsMin = cells > 0 ? cells + cells/32 + 64 : cellsNeed;
    const bool firstMeasured = cells > 0 && !p.cellsMeasured;
    if (cells > 0) p.cellsMeasured = true;
    if (cellsMin + 1 > p.cellcap || (firstMeasured && cellsNeed + 1 > p.cellcap)) {
      cudaStreamSynchronize(b.stream);
      void* old[] = {p.cellStart, p.cellFill};
      dev_free_all(old, 2);
      p.cellStart = nullptr; p.cellFill = nullptr;
      p.cellcap = cellsNeed + 1;
      if (dev_alloc(reinterpret_cast<void**>(&p.cellStart), sizeof(int64_t)*(p.cellcap + 1)) != cudaSuccess ||
          dev_alloc(reinterpret_cast<void**>(&p.cellFill), sizeof(int32_t)*p.cellcap) != cudaSuccess) {
        p.cellcap = 0;
        set_error("cell list allocation failed");
        return SPHGPU_ERR_NOMEM;
      }
    }
    // without a hint the first build guesses 32 entries per node; an overflow redoes it
    SPH_TRY(ensure_capacity_entries(p, E > 0 ? E + E/8 : 32*p.n));
    if (p.fillCap < 8) p.fillCap = p.maxCount > 0 ? p.maxCount + p.maxCount/4 + 8 : 64;
    if (kScanBlocks + 1 > p.blockSumsCap) SPH_TRY(ensure_block_sums(p, kScanBlocks + 1));
    if (p.gcap != oldg || p.candcap != oldc || p.ecap != olde || p.cellcap != oldcells) b.memDirty = true;
    if (p.fillSchedule == NBR_SCHEDULE_THREAD && sizeof(int32_t)*32*(size_t)p.fillCap > kMaxListSmem)
      p.fillSchedule = NBR_SCHEDULE_WARP;
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
  p.blockSumsCap = kScanBlocks + 1 + 64;                                // ensure_block_sums
  if (cfg.precision == SPHGPU_PRECISION_MIXED) p.mreccap = p.candcap;
  if (cfg.hydro == SPHGPU_HYDRO_CRKSPH) p.creccap = p.candcap;
  double marker = 0.0;                          // problem_bytes only tests these for null
  if (cfg.compatibleEnergyEvolution) p.pacc = &marker;
  if (cfg.precision == SPHGPU_PRECISION_MIXED) p.coefF = reinterpret_cast<float*>(&marker);
  if (cfg.hydro == SPHGPU_HYDRO_CRKSPH) { p.K = &marker; p.Kheld = &marker; }
  const int64_t b = problem_bytes(p);
  p.pacc = nullptr; p.coefF = nullptr; p.K = nullptr; p.Kheld = nullptr;
  return b;
}

namespace {

// Grid of the fused ghost passes: every block must be resident at once.
int fused_ghost_grid() {
  static int grid = -1;
  if (grid < 0) {
    int dev = 0, sms = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ghost_passes_fused_kernel, kGhostThreads, 0) != cudaSuccess) {
      cudaGetLastError();
      grid = 0;
    } else {
      grid = sms*occ < kFusedGhostBlocks ? sms*occ : kFusedGhostBlocks;
    }
  }
  return grid;
}

// The fused passes for this build: by the schedule, or (automatic) for a
// batch of at most kFusedGhostMembers members.  Their scratch is allocated
// outside a capture; a captured build without it takes the per-pass launches.
bool use_fused_ghost_passes(Batch& b) {
  const int nm = (int)b.mem.size();
  if (b.ghostPasses == 1 || nm > kFusedGhostMembers || fused_ghost_grid() <= 0) return false;
  if (b.d_fuse == nullptr) {
    if (b.capturing) return false;
    const size_t bytes = 2*sizeof(unsigned int) + sizeof(int64_t)*(size_t)kFusedGhostMembers*kFusedGhostBlocks + 8;
    if (dev_alloc(reinterpret_cast<void**>(&b.d_fuse), bytes) != cudaSuccess) { cudaGetLastError(); return false; }
    if (cudaMemset(b.d_fuse, 0, bytes) != cudaSuccess) { cudaGetLastError(); return false; }
  }
  return true;
}

int launch_fused_ghost_passes(Batch& b) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3((unsigned)fused_ghost_grid());
  lc.blockDim = dim3(kGhostThreads);
  lc.dynamicSmemBytes = 0;
  lc.stream = b.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  const int nm = (int)b.mem.size();
  return cuda_status(cudaLaunchKernelEx(&lc, ghost_passes_fused_kernel, (const Member*)b.d_mem, nm, b.d_fuse),
                     "fused ghost passes");
}

int launch_build(Batch& b) {
  cudaStream_t st = b.stream;
  const int nm = (int)b.mem.size();
  for (Problem* p : b.mem) p->paccReady = false;   // the walk parks its lists in pacc
  // (a captured build reads the descriptor slot uploaded before the capture)
  if (!b.capturing && !b.buildPlanned) SPH_TRY(batch_upload(b));
  b.buildPlanned = false;
  // ---- ghosts: six planar boundaries in order, sizes kept on the device
  build_init_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  // fixed grids: at most kStreamBlocks blocks per member, member-local stride
  auto fixedItems = [](int64_t cap) { return cap < kStreamBlocks*kGhostThreads ? cap : kStreamBlocks*kGhostThreads; };
  BlockMap nmap, cap;
  unsigned ngrid = 0, capGrid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return fixedItems(p.n); }, kGhostThreads, &nmap, &ngrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return fixedItems(p.candcap); }, kGhostThreads, &cap, &capGrid));
  if (ngrid) { node_hmax_kernel<<<ngrid, kGhostThreads, 0, st>>>(b.d_mem, nmap); batch_count_launch(b); }
  bool anyPeriodic = false;
  for (Problem* p : b.mem) for (int a = 0; a < 3; ++a) anyPeriodic = anyPeriodic || p->prm.bcs.periodic[a];
  if (anyPeriodic) {
    // the boundary passes visit only the internal nodes near a periodic plane
    near_flag_kernel<<<ngrid, kGhostThreads, 0, st>>>(b.d_mem, nmap); batch_count_launch(b);
    SPH_TRY(batch_scan(b, SCAN_COUNTS));
    near_list_kernel<<<ngrid, kGhostThreads, 0, st>>>(b.d_mem, nmap); batch_count_launch(b);
  }
  const bool fused = anyPeriodic && use_fused_ghost_passes(b);
  if (anyPeriodic) b.lastGhostPasses = fused ? 2 : 1;
  if (fused) {
    // (the barrier's arrival counter is back at zero after every completed
    // barrier; a build that reported a timed-out barrier clears it)
    SPH_TRY(launch_fused_ghost_passes(b));
    batch_count_launch(b);
  }
  for (int bnd = 0; bnd < 6 && !fused; ++bnd) {
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
  grid_kernel<<<(nm + 127)/128, 128, 0, st>>>(b.d_mem, nm); batch_count_launch(b);
  BlockMap cm;
  unsigned cgrid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return fixedItems(p.cellcap); }, kGhostThreads, &cm, &cgrid));
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
  // bitonic sort pads each warp's list to a power of two >= 32
  int wcap = 32;
  while (wcap < wmax) wcap <<= 1;
  auto thread = [](const Problem& p) { return p.fillSchedule != NBR_SCHEDULE_WARP; };
  for (Problem* p : b.mem) {
    p->lastNbrSchedule = p->fillSchedule;
    p->lastNbrPasses = p->grid.stashCap > 0 ? 1 : 2;
  }
  b.lastNbrSchedule = nm ? b.mem[0]->lastNbrSchedule : 0;
  const size_t tsmem = sizeof(int32_t)*(size_t)fthreads*tcap;
  const size_t wsmem = sizeof(int32_t)*(wthreads/32)*(size_t)wcap;
  auto smemAttr = [](auto* kernel, size_t bytes) -> int {
    if (bytes <= 48*1024) return SPHGPU_OK;
    return cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                       "nbr smem attribute");
  };
  SPH_TRY(smemAttr(nbr_thread_kernel<false, 1>, tsmem)); SPH_TRY(smemAttr(nbr_thread_kernel<true, 1>, tsmem));
  SPH_TRY(smemAttr(nbr_thread_kernel<false, 2>, tsmem)); SPH_TRY(smemAttr(nbr_thread_kernel<true, 2>, tsmem));
  SPH_TRY(smemAttr(nbr_walk_kernel<false, 1>, wsmem)); SPH_TRY(smemAttr(nbr_walk_kernel<true, 1>, wsmem));
  SPH_TRY(smemAttr(nbr_walk_kernel<false, 2>, wsmem)); SPH_TRY(smemAttr(nbr_walk_kernel<true, 2>, wsmem));
  // One walk launch per (schedule, cell subdivision) present.  pass 0: count
  // (and the lists of members with a stash); pass 1: fill (members without).
  auto walk = [&](bool threadSched, int sub, bool fill) -> int {
    BlockMap map;
    unsigned grid = 0;
    const int threads = threadSched ? (fill || tstash ? fthreads : 256) : wthreads;
    SPH_TRY(batch_map_items(b, [&](const Problem& p) {
      if (thread(p) != threadSched || p.grid.sub != sub || (fill && p.grid.stashCap)) return (int64_t)0;
      return threadSched ? p.candcap : 32*p.candcap; }, threads, &map, &grid));
    if (!grid) return SPHGPU_OK;
    if (threadSched) {
      const bool lists = fill || tstash;
      const size_t smem = lists ? tsmem : 0;
      const int c = lists ? tcap : 0;
      if (sub == 1) {
        if (fill) nbr_thread_kernel<true, 1><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
        else nbr_thread_kernel<false, 1><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
      } else {
        if (fill) nbr_thread_kernel<true, 2><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
        else nbr_thread_kernel<false, 2><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
      }
    } else {
      const bool lists = fill || wstash;
      const size_t smem = lists ? wsmem : 0;
      const int c = lists ? wcap : 0;
      if (sub == 1) {
        if (fill) nbr_walk_kernel<true, 1><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
        else nbr_walk_kernel<false, 1><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
      } else {
        if (fill) nbr_walk_kernel<true, 2><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
        else nbr_walk_kernel<false, 2><<<grid, threads, smem, st>>>(b.d_mem, map, c, maxNbr);
      }
    }
    batch_count_launch(b);
    return SPHGPU_OK;
  };
  for (int sub = 1; sub <= 2; ++sub) {
    SPH_TRY(walk(true, sub, false));
    SPH_TRY(walk(false, sub, false));
  }
  SPH_TRY(batch_scan(b, SCAN_COUNTS));
  // lists to the CSR: compaction of the stashes, fill pass for the rest
  BlockMap ctmap, cwmap;
  unsigned ctgrid = 0, cwgrid = 0;
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return thread(p) && p.grid.stashCap ? p.candcap : (int64_t)0; },
                          256, &ctmap, &ctgrid));
  SPH_TRY(batch_map_items(b, [&](const Problem& p) { return !thread(p) && p.grid.stashCap ? 32*p.n : (int64_t)0; },
                          256, &cwmap, &cwgrid));
  if (ctgrid) { nbr_compact_thread_kernel<<<ctgrid, 256, 0, st>>>(b.d_mem, ctmap); batch_count_launch(b); }
  if (cwgrid) { nbr_compact_warp_kernel<<<cwgrid, 256, 0, st>>>(b.d_mem, cwmap); batch_count_launch(b); }
  for (int sub = 1; sub <= 2; ++sub) {
    SPH_TRY(walk(true, sub, true));
    SPH_TRY(walk(false, sub, true));
  }
  return cuda_status(cudaGetLastError(), "neighbor build");
}

}  // namespace

// The build's launches alone, for a CUDA-graph capture of the whole step:
// capacities planned beforehand (plan_build), no read-back; a capacity
// overflow sets the member's error flag on the device instead.
int plan_build(Batch& b) { return plan_capacities(b); }
int launch_build_captured(Batch& b) { return launch_build(b); }

// Ghosts and ConnectivityMap of every member: all stages launched with the
// sizes kept on the device, then one read-back of the sizes; a capacity
// overflow grows the buffers and repeats the build.
int build_connectivity(Batch& b) {
  const int nm = (int)b.mem.size();
  for (Problem* p : b.mem) {
    if (p->n + p->gcap > INT_MAX) { set_error("too many nodes for 32-bit neighbor indices"); return SPHGPU_ERR_CAPACITY; }
  }
  for (int attempt = 0; attempt < 6; ++attempt) {
    if (!(attempt == 0 && b.buildPlanned)) SPH_TRY(plan_capacities(b));
    SPH_TRY(launch_build(b));
    if (b.afterBuildLaunch) {
      const std::function<int()> f = std::move(b.afterBuildLaunch);
      b.afterBuildLaunch = nullptr;
      SPH_TRY(f());
    }
    const int slots[7] = {SC_G, SC_TOTAL, SC_MAXCOUNT, SC_PAIRS, SC_NCELLS, SC_CELLSWANTED, -1};
    std::vector<double> r;
    SPH_TRY(batch_gather(b, slots, 7, r));
    bool redo = false;
    for (int m = 0; m < nm; ++m) {
      Problem& p = *b.mem[m];
      const int herr = (int)r[m*7 + 6];
      p.G = asI64(r[m*7]);
      p.ntot = p.n + p.G;
      p.E = asI64(r[m*7 + 1]);
      p.maxCount = asI32(r[m*7 + 2]);
      p.pairs = asI64(r[m*7 + 3]);
      p.ncells = asI64(r[m*7 + 4]);
      p.cellsWanted = asI64(r[m*7 + 5]);
      p.lastNbrCells = p.grid.sub;
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
      if (herr & DERR_BARRIER) {
        if (b.d_fuse) cudaMemsetAsync(b.d_fuse, 0, 2*sizeof(unsigned int), b.stream);
        set_error("neighbor build: a grid barrier of the fused ghost passes timed out");
        return SPHGPU_ERR_CUDA;
      }
      if (herr & DERR_GHOST_CAPACITY) { p.G = 2*p.gcap; redo = true; }        // ghost count unknown: double
      if (herr & DERR_ENTRY_CAPACITY) redo = true;                           // p.E is the true entry count
      if (herr & DERR_LIST_CAPACITY) { p.fillCap = p.maxCount + p.maxCount/4 + 8; redo = true; }
      else if (p.fillCap > p.maxCount + p.maxCount/2 + 16) p.fillCap = 0;   // re-plan a tighter list
    }
    if (!redo) return SPHGPU_OK;
    SPH_CHECK(cudaStreamSynchronize(b.stream));
  }
  set_error("neighbor build: capacities did not converge");
  return SPHGPU_ERR_CAPACITY;
}

}  // namespace sphgpu
