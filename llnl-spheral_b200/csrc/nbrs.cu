// Periodic ghost images, cell list and ConnectivityMap CSR on the device.
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
// Kernels and their bounds (see the roofline notes in the design document):
//   ghost_hmax / ghost_flag / ghost_scatter  O(N+G) streaming, HBM bound
//   node_bounds / cell_index / cell_scatter  O(N+G) streaming + atomics
//   nbr_thread<COUNT|FILL>                   thread per node (cell-sorted
//                                            order) over the 27 neighbouring
//                                            cells; 80-byte candidate records
//                                            shared by a warp through L1
//   nbr_walk<COUNT|FILL>                     warp per node, for large
//                                            candidate sets
#include <cstdio>
#include <climits>

#include "problem.cuh"

namespace sphgpu {

namespace {

__device__ __forceinline__ unsigned long long orderedBits(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

__device__ __forceinline__ V3 nodePos(const double* S, int64_t n, const double* gpos, int64_t gcap, int64_t k) {
  if (k < n) return V3{S[S_X*n + k], S[S_Y*n + k], S[S_Z*n + k]};
  const int64_t g = k - n;
  return V3{gpos[g], gpos[gcap + g], gpos[2*gcap + g]};
}
__device__ __forceinline__ Sym nodeH(const double* S, int64_t n, const int32_t* groot, int64_t k) {
  const int64_t r = k < n ? k : groot[k - n];
  return Sym{S[(S_H + 0)*n + r], S[(S_H + 1)*n + r], S[(S_H + 2)*n + r],
             S[(S_H + 3)*n + r], S[(S_H + 4)*n + r], S[(S_H + 5)*n + r]};
}

// hmax of PlanarBoundary::setGhostNodes: max 1/min(eig(H)) over nodes within
// kernelExtent*hmaxi of either plane.
__global__ void ghost_hmax_kernel(const double* S, int64_t n, const double* gpos, int64_t gcap,
                                  const int32_t* groot, int64_t ntot, PlanarBC bc, double kernelExtent,
                                  unsigned long long* out) {
  double best = 0.0;
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    const V3 r = nodePos(S, n, gpos, gcap, k);
    const Sym H = nodeH(S, n, groot, k);
    const double hmaxi = 1.0/vmin(eigenValues(H));
    if (hmaxi > best && dmin(minimumDistance(bc.exit, r), minimumDistance(bc.enter, r)) < kernelExtent*hmaxi)
      best = hmaxi;
  }
  for (int o = 16; o > 0; o >>= 1) best = dmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

__global__ void ghost_flag_kernel(const double* S, int64_t n, const double* gpos, int64_t gcap, int64_t ntot,
                                  PlanarBC bc, double kernelExtent, const unsigned long long* hmaxBits,
                                  int32_t* flags) {
  const double hmax = __longlong_as_double((long long)*hmaxBits);
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    int f = 0;
    if (hmax > 0.0) {
      const V3 r = nodePos(S, n, gpos, gcap, k);
      const double disti = signedDistance(bc.exit, r)/hmax;
      f = (disti >= 0.0 && disti <= kernelExtent) ? 1 : 0;
    }
    flags[k] = f;
  }
}

__global__ void ghost_scatter_kernel(const double* S, int64_t n, double* gpos, int64_t gcap,
                                     int32_t* groot, uint32_t* gcode, int64_t ntot,
                                     const int32_t* flags, const int64_t* slots, PlanarBC bc, int b,
                                     int* err) {
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    if (!flags[k]) continue;
    const int64_t g = (ntot - n) + slots[k];     // ghost index of the new image
    const V3 r = nodePos(S, n, gpos, gcap, k);
    const V3 gp = mapPositionThroughPlanes(r, bc.exit, bc.enter);
    const int32_t root = k < n ? (int32_t)k : groot[k - n];
    uint32_t code = k < n ? 0u : gcode[k - n];
    const int axis = b >> 1;
    if ((code >> (2*axis)) & 3u) atomicOr(err, DERR_GHOST_CHAIN);
    code |= (uint32_t)((b & 1) + 1) << (2*axis);
    groot[g] = root;
    gcode[g] = code;
    gpos[g] = gp.x; gpos[gcap + g] = gp.y; gpos[2*gcap + g] = gp.z;
  }
}

// Global bounding box of all nodes and max of 1/min(eig(H)) (cell size).
__global__ void node_bounds_kernel(const double* S, int64_t n, const double* gpos, int64_t gcap,
                                   const int32_t* groot, int64_t ntot, unsigned long long* out) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, h = 0.0;
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    const V3 r = nodePos(S, n, gpos, gcap, k);
    lo[0] = fmin(lo[0], r.x); lo[1] = fmin(lo[1], r.y); lo[2] = fmin(lo[2], r.z);
    hi[0] = fmax(hi[0], r.x); hi[1] = fmax(hi[1], r.y); hi[2] = fmax(hi[2], r.z);
    if (k < n) h = fmax(h, 1.0/vmin(eigenValues(nodeH(S, n, groot, k))));
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    h = fmax(h, __shfl_xor_sync(0xffffffffu, h, o));
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(out + a, orderedBits(lo[a]));
      atomicMax(out + 3 + a, orderedBits(hi[a]));
    }
    atomicMax(out + 6, orderedBits(h));
  }
}

struct Grid {
  double lo[3];
  double cell;
  int dim[3];
};

__device__ __forceinline__ int cellCoord(double x, double lo, double cell, int dim) {
  int c = int((x - lo)/cell);
  return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

__global__ void cell_index_kernel(const double* S, int64_t n, const double* gpos, int64_t gcap, int64_t ntot,
                                  Grid g, int32_t* cidx, int32_t* cellCount) {
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    const V3 r = nodePos(S, n, gpos, gcap, k);
    const int cx = cellCoord(r.x, g.lo[0], g.cell, g.dim[0]);
    const int cy = cellCoord(r.y, g.lo[1], g.cell, g.dim[1]);
    const int cz = cellCoord(r.z, g.lo[2], g.cell, g.dim[2]);
    const int c = (cz*g.dim[1] + cy)*g.dim[0] + cx;
    cidx[k] = c;
    atomicAdd(cellCount + c, 1);
  }
}

// Candidate record of the cell-sorted node list: position, H and the node
// index, 80 bytes, read as five 16-byte loads.
struct __align__(16) NbrCand {
  double x, y, z;
  double hxx, hxy, hxz, hyy, hyz, hzz;
  int32_t idx, pad;
};
static_assert(sizeof(NbrCand) == 80, "candidate record is five 16-byte words");

__device__ __forceinline__ NbrCand loadCand(const NbrCand* c) {
  const double2* q = reinterpret_cast<const double2*>(c);
  const double2 a = __ldg(q), b = __ldg(q + 1), d = __ldg(q + 2), e = __ldg(q + 3), f = __ldg(q + 4);
  NbrCand r;
  r.x = a.x; r.y = a.y; r.z = b.x; r.hxx = b.y; r.hxy = d.x; r.hxz = d.y; r.hyy = e.x; r.hyz = e.y; r.hzz = f.x;
  r.idx = __double_as_longlong(f.y) & 0xffffffff;
  r.pad = 0;
  return r;
}

__global__ void cell_scatter_kernel(const double* S, int64_t n, const double* gpos, int64_t gcap,
                                    const int32_t* groot, int64_t ntot, const int32_t* cidx,
                                    const int64_t* cellStart, int32_t* cellFill, int32_t* sortedIdx,
                                    NbrCand* cand) {
  for (int64_t k = blockIdx.x*(int64_t)blockDim.x + threadIdx.x; k < ntot; k += (int64_t)gridDim.x*blockDim.x) {
    const int c = cidx[k];
    const int64_t slot = cellStart[c] + atomicAdd(cellFill + c, 1);
    sortedIdx[slot] = (int32_t)k;
    const V3 r = nodePos(S, n, gpos, gcap, k);
    const Sym H = nodeH(S, n, groot, k);
    double2* q = reinterpret_cast<double2*>(cand + slot);
    q[0] = make_double2(r.x, r.y);
    q[1] = make_double2(r.z, H.xx);
    q[2] = make_double2(H.xy, H.xz);
    q[3] = make_double2(H.yy, H.yz);
    q[4] = make_double2(H.zz, __longlong_as_double((long long)(uint32_t)k));
  }
}

// Thread per internal node, nodes taken in cell-sorted order so that the
// threads of a warp share their candidate rows (L1 broadcast).  The 27
// neighbouring cells are walked as 9 x-rows (three cells each, contiguous in
// the sorted order) and the exact ConnectivityMap predicate is applied.
// COUNT pass: per-node counts and their maximum.  FILL pass: the neighbor
// indices are insertion-sorted into a per-thread shared-memory list of
// capacity `cap` (element c of thread t at lst[c*blockDim + t], conflict
// free) and stored ascending at offsets[i].
template<bool FILL>
__global__ void __launch_bounds__(256) nbr_thread_kernel(int64_t n, int64_t ntot, Grid g, const int64_t* cellStart,
                                                         const NbrCand* cand, double kernelExtent2, int32_t* counts,
                                                         const int64_t* offsets, int32_t* nbr, int cap,
                                                         int* maxCount, int* err,
                                                         unsigned long long* pairCount) {
  extern __shared__ int32_t lst[];
  const int tid = threadIdx.x;
  const int bd = blockDim.x;
  const int64_t s = blockIdx.x*(int64_t)bd + tid;
  NbrCand me;
  bool active = s < ntot;
  if (active) {
    me = loadCand(cand + s);
    active = me.idx < n;
  }
  int count = 0, above = 0;
  if (active) {
    const int32_t i = me.idx;
    const V3 ri{me.x, me.y, me.z};
    const Sym Hi{me.hxx, me.hxy, me.hxz, me.hyy, me.hyz, me.hzz};
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
          const V3 rij = vsub(ri, V3{c.x, c.y, c.z});
          const double eta2i = mag2(sdot(Hi, rij));
          const double eta2j = mag2(sdot(Sym{c.hxx, c.hxy, c.hxz, c.hyy, c.hyz, c.hzz}, rij));
          if ((eta2i <= kernelExtent2 || eta2j <= kernelExtent2) && c.idx != i) {
            if (FILL) {
              if (count < cap) {
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
      counts[i] = count;
    } else if (count <= cap) {
      const int64_t o = offsets[i];
      for (int c = 0; c < count; ++c) nbr[o + c] = lst[c*bd + tid];
    } else {
      atomicOr(err, DERR_NBR_CAPACITY);
    }
  }
  if (!FILL) {
    int m = count;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0 && m > 0) atomicMax(maxCount, m);
  } else {
    unsigned long long a = (unsigned long long)above;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((tid & 31) == 0 && a) atomicAdd(pairCount, a);
  }
}

// Warp per internal node: walk the 27 neighbouring cells, apply the exact
// ConnectivityMap predicate, count (FILL=false) or collect, sort ascending
// and store (FILL=true) the neighbor indices.  Used when the candidate sets
// are large (many nodes per cell), where a warp per node keeps the SMs full.
template<bool FILL>
__global__ void __launch_bounds__(256) nbr_walk_kernel(const double* S, int64_t n, Grid g,
                                                       const int64_t* cellStart, const NbrCand* cand,
                                                       double kernelExtent2,
                                                       int32_t* counts, const int64_t* offsets, int32_t* nbr,
                                                       int maxNbr, int* err, int* maxCount,
                                                       unsigned long long* pairCount) {
  extern __shared__ int32_t sbuf_all[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  int32_t* sbuf = sbuf_all + (FILL ? wib*maxNbr : 0);
  const int64_t i = (blockIdx.x*(int64_t)blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const V3 ri{S[S_X*n + i], S[S_Y*n + i], S[S_Z*n + i]};
  const Sym Hi{S[(S_H + 0)*n + i], S[(S_H + 1)*n + i], S[(S_H + 2)*n + i],
               S[(S_H + 3)*n + i], S[(S_H + 4)*n + i], S[(S_H + 5)*n + i]};
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
      const int64_t start = cellStart[cbase + x0];
      const int64_t end = cellStart[cbase + x1 + 1];
      for (int64_t base = start; base < end; base += 32) {
        const int64_t k = base + lane;
        bool pass = false;
        int32_t j = -1;
        if (k < end) {
          const NbrCand c = loadCand(cand + k);
          j = c.idx;
          const V3 rj{c.x, c.y, c.z};
          const Sym Hj{c.hxx, c.hxy, c.hxz, c.hyy, c.hyz, c.hzz};
          const V3 rij = vsub(ri, rj);
          const double eta2i = mag2(sdot(Hi, rij));
          const double eta2j = mag2(sdot(Hj, rij));
          pass = (eta2i <= kernelExtent2 || eta2j <= kernelExtent2) && (j != (int32_t)i);
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, pass);
        if (FILL && pass) {
          const int pos = count + __popc(ballot & ((1u << lane) - 1u));
          if (pos < maxNbr) sbuf[pos] = j;
        }
        count += __popc(ballot);
      }
    }
  }
  if (!FILL) {
    if (lane == 0) {
      counts[i] = count;
      if (count > maxNbr) atomicOr(err, DERR_NBR_CAPACITY);
      atomicMax(maxCount, count);
    }
    return;
  }
  if (count > maxNbr) return;
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
  const int64_t o = offsets[i];
  int above = 0;
  for (int t = lane; t < count; t += 32) {
    const int32_t j = sbuf[t];
    nbr[o + t] = j;
    above += (j > (int32_t)i);
  }
  for (int s = 16; s > 0; s >>= 1) above += __shfl_xor_sync(0xffffffffu, above, s);
  if (lane == 0) atomicAdd(pairCount, (unsigned long long)above);
}

inline int nblocks(int64_t work, int threads, int cap = 148*32) {
  int64_t b = (work + threads - 1)/threads;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}

}  // namespace

int build_ghosts(Problem& p) {
  cudaStream_t st = p.stream;
  p.G = 0;
  int64_t ntot = p.n;
  unsigned long long* hbits = reinterpret_cast<unsigned long long*>(p.d_scal);
  for (int b = 0; b < 6; ++b) {
    if (!p.prm.bcs.periodic[b >> 1]) continue;
    const PlanarBC bc = p.prm.bcs.bc[b];
    if (cudaMemsetAsync(hbits, 0, sizeof(unsigned long long), st) != cudaSuccess) return cuda_status(cudaGetLastError(), "memset");
    ghost_hmax_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, p.groot, ntot, bc,
                                                           p.prm.kernelExtent, hbits); ++p.launches;
    ghost_flag_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, ntot, bc, p.prm.kernelExtent,
                                                           hbits, p.counts); ++p.launches;
    int64_t total = 0;
    int rc = exclusive_scan_i32(p, p.counts, ntot, p.offsets, &total);
    if (rc) return rc;
    if (total == 0) continue;
    rc = ensure_capacity_ghosts(p, (ntot - p.n) + total);
    if (rc) return rc;
    ghost_scatter_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, p.groot, p.gcode, ntot,
                                                              p.counts, p.offsets, bc, b, p.d_err); ++p.launches;
    ntot += total;
  }
  p.G = ntot - p.n;
  return cuda_status(cudaGetLastError(), "build_ghosts");
}

int build_cells_and_csr(Problem& p) {
  cudaStream_t st = p.stream;
  const int64_t ntot = p.n + p.G;
  if (ntot > INT_MAX) { set_error("too many nodes for 32-bit neighbor indices"); return SPHGPU_ERR_CAPACITY; }
  // ---- grid
  unsigned long long* bb = reinterpret_cast<unsigned long long*>(p.d_scal);
  unsigned long long init[7];
  for (int a = 0; a < 3; ++a) { init[a] = ~0ULL; init[3 + a] = 0ULL; }
  init[6] = 0ULL;
  cudaMemcpyAsync(bb, init, sizeof(init), cudaMemcpyHostToDevice, st);
  node_bounds_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, p.groot, ntot, bb); ++p.launches;
  unsigned long long res[7];
  cudaMemcpyAsync(res, bb, sizeof(res), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_status(cudaGetLastError(), "bounds");
  auto fromBits = [](unsigned long long b) {
    const unsigned long long r = (b & 0x8000000000000000ULL) ? (b & 0x7fffffffffffffffULL) : ~b;
    double d; memcpy(&d, &r, sizeof(d)); return d;
  };
  Grid g;
  double hi[3];
  for (int a = 0; a < 3; ++a) { g.lo[a] = fromBits(res[a]); hi[a] = fromBits(res[3 + a]); }
  const double hmaxAll = fromBits(res[6]);
  // cell size >= interaction radius kappa*max(1/lambda_min); the margin
  // covers the libm difference of the eigenvalue solve for anisotropic H.
  g.cell = p.prm.kernelExtent*hmaxAll*1.001;
  if (!(g.cell > 0.0)) { set_error("non-positive smoothing scale"); return SPHGPU_ERR_NUMERIC; }
  // Larger cells only widen the candidate set; cap the cell count so that
  // 32-bit cell indices cannot overflow.
  int64_t ncells = 1;
  for (int attempt = 0; attempt < 64; ++attempt) {
    ncells = 1;
    for (int a = 0; a < 3; ++a) {
      const double d = (hi[a] - g.lo[a])/g.cell;
      const int64_t m = (int64_t)d + 1;
      g.dim[a] = (int)(m < (1 << 20) ? m : (1 << 20));
      ncells *= g.dim[a];
    }
    if (ncells <= ((int64_t)1 << 26)) break;
    g.cell *= 1.26;
  }
  if (ncells > ((int64_t)1 << 26)) { set_error("cell grid too large"); return SPHGPU_ERR_CAPACITY; }
  if (ncells + 1 > p.cellcap) {
    cudaFree(p.cellStart); cudaFree(p.cellFill);
    p.cellcap = ncells + 1;
    if (cudaMalloc(&p.cellStart, sizeof(int64_t)*(p.cellcap + 1)) != cudaSuccess ||
        cudaMalloc(&p.cellFill, sizeof(int32_t)*p.cellcap) != cudaSuccess) {
      set_error("cell list allocation failed"); return SPHGPU_ERR_NOMEM;
    }
  }
  int64_t* cellStart = reinterpret_cast<int64_t*>(p.cellStart);
  for (int a = 0; a < 3; ++a) { p.gdim[a] = g.dim[a]; p.glo[a] = g.lo[a]; }
  p.gcell = g.cell;
  // ---- counting sort of all nodes by cell
  cudaMemsetAsync(p.cellFill, 0, sizeof(int32_t)*ncells, st);
  cell_index_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, ntot, g, p.cidx, p.cellFill); ++p.launches;
  int64_t tot = 0;
  int rc = exclusive_scan_i32(p, p.cellFill, ncells, cellStart, &tot);
  if (rc) return rc;
  cudaMemsetAsync(p.cellFill, 0, sizeof(int32_t)*ncells, st);
  NbrCand* cand = reinterpret_cast<NbrCand*>(p.cand);
  cell_scatter_kernel<<<nblocks(ntot, 256), 256, 0, st>>>(p.S, p.n, p.gpos, p.gcap, p.groot, ntot, p.cidx,
                                                           cellStart, p.cellFill, p.sortedIdx, cand); ++p.launches;
  // ---- neighbor counts, offsets, fill
  const double k2 = p.prm.kernelExtent*p.prm.kernelExtent;
  // Schedule: a thread per node while the 27-cell candidate set is small, a
  // warp per node once it is large enough to keep 32 lanes busy.
  const double candPerNode = 27.0*(double)ntot/(double)ncells;
  const bool warpSchedule = p.nbrSchedule == NBR_SCHEDULE_WARP ||
                            (p.nbrSchedule == NBR_SCHEDULE_AUTO && candPerNode > 384.0);
  p.lastNbrSchedule = warpSchedule ? NBR_SCHEDULE_WARP : NBR_SCHEDULE_THREAD;
  int* dMaxCount = reinterpret_cast<int*>(p.d_scal + 10);
  cudaMemsetAsync(dMaxCount, 0, sizeof(int), st);
  const int wthreads = 256;
  const int64_t wblocks = (p.n*32 + wthreads - 1)/wthreads;
  const int tthreads = 256;
  const int64_t tblocks = (ntot + tthreads - 1)/tthreads;
  if (warpSchedule) {
    nbr_walk_kernel<false><<<(unsigned)wblocks, wthreads, 0, st>>>(p.S, p.n, g, cellStart, cand, k2, p.counts,
                                                                     nullptr, nullptr, p.maxNbr, p.d_err,
                                                                     dMaxCount, nullptr); ++p.launches;
  } else {
    nbr_thread_kernel<false><<<(unsigned)tblocks, tthreads, 0, st>>>(p.n, ntot, g, cellStart, cand, k2, p.counts,
                                                                       nullptr, nullptr, 0, dMaxCount, p.d_err,
                                                                       nullptr); ++p.launches;
  }
  int64_t E = 0;
  rc = exclusive_scan_i32(p, p.counts, p.n, p.offsets, &E);
  if (rc) return rc;
  int herr = 0, maxCount = 0;
  cudaMemcpyAsync(&herr, p.d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&maxCount, dMaxCount, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_status(cudaGetLastError(), "nbr count");
  if (herr & (DERR_NBR_CAPACITY | DERR_GHOST_CHAIN)) cudaMemsetAsync(p.d_err, 0, sizeof(int), st);
  if ((herr & DERR_NBR_CAPACITY) || maxCount > p.maxNbr) {
    set_error("a node has more neighbors than max_neighbors");
    return SPHGPU_ERR_CAPACITY;
  }
  if (herr & DERR_GHOST_CHAIN) {
    set_error("a ghost image was imaged twice through one periodic axis");
    return SPHGPU_ERR_UNSUPPORTED;
  }
  p.maxCount = maxCount;
  rc = ensure_capacity_entries(p, E);
  if (rc) return rc;
  unsigned long long* pc = reinterpret_cast<unsigned long long*>(p.d_scal + 8);
  cudaMemsetAsync(pc, 0, sizeof(unsigned long long), st);
  // per-thread list capacity: shrink the block until the lists fit
  int fthreads = tthreads;
  const int tcap = maxCount > 0 ? maxCount : 1;
  while (fthreads > 32 && sizeof(int32_t)*(size_t)fthreads*tcap > 96*1024) fthreads >>= 1;
  const bool threadFill = !warpSchedule && sizeof(int32_t)*(size_t)fthreads*tcap <= 200*1024;
  if (threadFill) {
    const size_t smem = sizeof(int32_t)*(size_t)fthreads*tcap;
    if (smem > 48*1024) {
      const cudaError_t e = cudaFuncSetAttribute(nbr_thread_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
      if (e != cudaSuccess) return cuda_status(e, "nbr smem attribute");
    }
    const int64_t fblocks = (ntot + fthreads - 1)/fthreads;
    nbr_thread_kernel<true><<<(unsigned)fblocks, fthreads, smem, st>>>(p.n, ntot, g, cellStart, cand, k2, p.counts,
                                                                         p.offsets, p.nbr, tcap, nullptr, p.d_err,
                                                                         pc); ++p.launches;
  } else {
    // bitonic sort pads each warp's list to a power of two >= 32
    int wcap = 32;
    while (wcap < maxCount) wcap <<= 1;
    const size_t smem = sizeof(int32_t)*(wthreads/32)*(size_t)wcap;
    if (smem > 48*1024) {
      const cudaError_t e = cudaFuncSetAttribute(nbr_walk_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
      if (e != cudaSuccess) return cuda_status(e, "nbr smem attribute");
    }
    nbr_walk_kernel<true><<<(unsigned)wblocks, wthreads, smem, st>>>(p.S, p.n, g, cellStart, cand, k2, p.counts,
                                                                       p.offsets, p.nbr, wcap, p.d_err, nullptr,
                                                                       pc); ++p.launches;
  }
  unsigned long long pairs = 0;
  cudaMemcpyAsync(&pairs, pc, sizeof(pairs), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_status(cudaGetLastError(), "nbr fill");
  p.E = E;
  p.pairs = (int64_t)pairs;
  return SPHGPU_OK;
}

}  // namespace sphgpu
