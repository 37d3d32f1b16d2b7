// Batched launches: member descriptors, block maps, gathered scalars and
// the per-member prefix sums used by the neighbor build.
//
// A batch is a set of independent problems advanced together.  Each stage
// is one kernel launch over all members: the grid is the concatenation of
// the members' grids, and a block finds its member in the block map (a
// prefix table of per-member block counts).  Each member keeps its own
// buffers, so a member's results do not depend on the other members.
#include <cstring>
#include <map>
#include <mutex>

#include "problem.cuh"

namespace sphgpu {

namespace {

cudaMemPool_t device_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = ~0ULL;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = pool;
  return pool;
}

}  // namespace

cudaError_t dev_alloc(void** ptr, size_t bytes) {
  *ptr = nullptr;
  if (bytes == 0) bytes = 1;
  cudaMemPool_t pool = device_pool();
  if (pool == nullptr) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, cudaStreamLegacy);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(ptr, bytes, pool, cudaStreamLegacy);
  }
  if (e != cudaSuccess) { *ptr = nullptr; return e; }
  return cudaStreamSynchronize(cudaStreamLegacy);
}

void dev_free_all(void* const* ptrs, int count) {
  bool any = false;
  for (int k = 0; k < count; ++k) any = any || ptrs[k] != nullptr;
  if (!any) return;
  cudaDeviceSynchronize();
  for (int k = 0; k < count; ++k) if (ptrs[k]) cudaFreeAsync(ptrs[k], cudaStreamLegacy);
}

void dev_free(void* ptr) { dev_free_all(&ptr, 1); }


namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS*SCAN_ITEMS;

constexpr int64_t kMapRing = 1 << 20;

Member member_of(const Problem& p) {
  Member M;
  std::memset(&M, 0, sizeof(M));
  M.prm = p.prm;
  M.S = p.S; M.S0 = p.S0; M.D = p.D; M.K = p.K;
  M.rec = p.rec; M.crec = p.crec; M.mrec = p.mrec;
  M.gpos = p.gpos; M.pacc = p.pacc; M.scal = p.d_scal; M.red = p.d_red; M.hmaxi = p.hmaxi;
  M.qgrad = p.qgrad;
  M.fshear = p.fshear;
  M.groot = p.groot; M.cidx = p.cidx; M.sortedIdx = p.sortedIdx; M.counts = p.counts; M.nbr = p.nbr;
  M.cellFill = p.cellFill;
  M.gcode = p.gcode;
  M.offsets = p.offsets; M.cellStart = p.cellStart; M.blockSums = p.blockSums;
  M.cand = p.cand;
  M.coefF = p.coefF;
  M.err = p.d_err;
  M.n = p.n; M.G = p.G; M.ntot = p.ntot; M.gcap = p.gcap; M.E = p.E; M.ecap = p.ecap;
  M.candcap = p.candcap; M.ncells = p.ncells; M.cellcap = p.cellcap;
  M.grid = p.grid;
  return M;
}

__global__ void gather_scal_kernel(const Member* mem, int nmem, int4 slotsA, int4 slotsB, int nslots,
                                   double* out) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m >= nmem) return;
  const int slots[8] = {slotsA.x, slotsA.y, slotsA.z, slotsA.w, slotsB.x, slotsB.y, slotsB.z, slotsB.w};
  // slot -1 reads the member's device error word
  for (int s = 0; s < nslots; ++s)
    out[(int64_t)m*nslots + s] = slots[s] >= 0 ? mem[m].scal[slots[s]] : (double)mem[m].err[0];
}

__global__ void set_scal_kernel(const Member* mem, int nmem, int slot, double v) {
  const int m = blockIdx.x*blockDim.x + threadIdx.x;
  if (m < nmem) mem[m].scal[slot] = v;
}

__device__ __forceinline__ void scanIO(const Member& M, int which, const int32_t*& in, int64_t& n,
                                       int64_t*& out) {
  // lengths from the device-side sizes of the build in progress
  if (which == SCAN_FLAGS) {
    // a boundary pass: the near-plane internal nodes, then the ghosts so far
    in = M.counts; n = scalI(M.scal, SC_NNEAR) + scalI(M.scal, SC_NTOT) - M.n; out = M.offsets;
  }
  else if (which == SCAN_CELLS) { in = M.cellFill; n = scalI(M.scal, SC_NCELLS); out = M.cellStart; }
  else { in = M.counts; n = M.n; out = M.offsets; }
}

// Upper bound of a scan's length (host and device).
__host__ __device__ __forceinline__ int64_t scanCapacity(int64_t n, int64_t candcap, int64_t cellcap, int which) {
  return which == SCAN_FLAGS ? candcap : (which == SCAN_CELLS ? cellcap : n);
}

// Blocks of a member's scan: one per tile up to kScanBlocks.
__host__ __device__ __forceinline__ int scanBlocks(int64_t cap) {
  const int64_t t = (cap + SCAN_TILE - 1)/SCAN_TILE;
  return (int)(t < 1 ? 1 : (t > kScanBlocks ? kScanBlocks : t));
}

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan; returns the exclusive prefix of `v`, sets *total.
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* total) {
  __shared__ int64_t wsum[SCAN_THREADS/32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t inc = warp_incl_scan(v);
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < SCAN_THREADS/32 ? wsum[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < SCAN_THREADS/32) wsum[lane] = s;
  }
  __syncthreads();
  const int64_t before = (w > 0 ? wsum[w - 1] : 0) + inc - v;
  *total = wsum[SCAN_THREADS/32 - 1];
  __syncthreads();
  return before;
}

// Tile range [t0, t1) of block `blk` of `nblk` over a scan of length n.
__device__ __forceinline__ void blockTiles(int64_t n, int blk, int nblk, int64_t& t0, int64_t& t1) {
  const int64_t tiles = (n + SCAN_TILE - 1)/SCAN_TILE;
  const int64_t per = (tiles + nblk - 1)/nblk;
  t0 = (int64_t)blk*per;
  t1 = t0 + per < tiles ? t0 + per : tiles;
}

// Pass 1: the sum of each block's run of tiles.
__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_sums_kernel(const Member* mem, BlockMap bm, int which) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int32_t* in; int64_t n; int64_t* out;
  scanIO(M, which, in, n, out);
  int64_t t0, t1;
  blockTiles(n, (int)mb.block, mb.blocks, t0, t1);
  int64_t s = 0;
  for (int64_t t = t0; t < t1; ++t) {
    const int64_t base = t*SCAN_TILE + (int64_t)threadIdx.x*SCAN_ITEMS;
    for (int k = 0; k < SCAN_ITEMS; ++k)
      if (base + k < n) s += in[base + k];
  }
  int64_t total;
  block_excl_scan(s, &total);
  if (threadIdx.x == 0) M.blockSums[mb.block] = total;
}

// Pass 2: one block per member scans its block sums; writes out[n] and the total.
__global__ void __launch_bounds__(SCAN_THREADS) scan_sums_kernel(const Member* mem, BlockMap bm, int which) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int32_t* in; int64_t n; int64_t* out;
  scanIO(M, which, in, n, out);
  const int nblk = scanBlocks(scanCapacity(M.n, M.candcap, M.cellcap, which));
  int64_t carry = 0;
  for (int base = 0; base < nblk; base += SCAN_THREADS) {
    const int idx = base + threadIdx.x;
    const int64_t v = idx < nblk ? M.blockSums[idx] : 0;
    int64_t total;
    const int64_t ex = block_excl_scan(v, &total);
    if (idx < nblk) M.blockSums[idx] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) {
    out[n] = carry;
    reinterpret_cast<int64_t*>(M.scal)[SC_TOTAL] = carry;
  }
}

// Pass 3: each block rescans its run of tiles from its block's offset.
__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const Member* mem, BlockMap bm, int which) {
  const MemberBlock mb = memberBlock(bm);
  const Member& M = mem[mb.m];
  const int32_t* in; int64_t n; int64_t* out;
  scanIO(M, which, in, n, out);
  int64_t t0, t1;
  blockTiles(n, (int)mb.block, mb.blocks, t0, t1);
  int64_t carry = M.blockSums[mb.block];
  for (int64_t t = t0; t < t1; ++t) {
    const int64_t base = t*SCAN_TILE + (int64_t)threadIdx.x*SCAN_ITEMS;
    int32_t v[SCAN_ITEMS];
    int64_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      v[k] = base + k < n ? in[base + k] : 0;
      s += v[k];
    }
    int64_t total;
    int64_t run = block_excl_scan(s, &total) + carry;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      if (base + k < n) out[base + k] = run;
      run += v[k];
    }
    carry += total;
  }
}

// Launch sizes: the capacities bound the device-side lengths.
int64_t scan_items(const Problem& p, int which) { return scanCapacity(p.n, p.candcap, p.cellcap, which); }

}  // namespace

Member describe_member(const Problem& p) { return member_of(p); }

int batch_init(Batch& b, cudaStream_t stream) {
  b.stream = stream;
  for (int k = 0; k < Batch::kMemSlots; ++k)
    if (cudaEventCreateWithFlags(&b.memEvents[k], cudaEventDisableTiming) != cudaSuccess)
      return cuda_status(cudaGetLastError(), "batch event");
  if (dev_alloc(reinterpret_cast<void**>(&b.d_maps), sizeof(int32_t)*kMapRing) != cudaSuccess ||
      cudaMallocHost(&b.h_maps, sizeof(int32_t)*kMapRing) != cudaSuccess) {
    set_error("batch block-map ring allocation failed");
    return SPHGPU_ERR_NOMEM;
  }
  b.mapcap = kMapRing;
  b.mappos = 0;
  return SPHGPU_OK;
}

void batch_free(Batch& b) {
  if (b.stream) cudaStreamSynchronize(b.stream);
  void* dev[] = {b.d_memRing, b.d_maps, b.d_gather, b.d_mapArena, b.d_memGraph, b.d_fuse};
  dev_free_all(dev, 6);
  cudaFreeHost(b.h_memRing);
  cudaFreeHost(b.h_maps);
  cudaFreeHost(b.h_gather);
  for (int k = 0; k < Batch::kMemSlots; ++k) if (b.memEvents[k]) cudaEventDestroy(b.memEvents[k]);
  if (b.graphExec) cudaGraphExecDestroy(b.graphExec);
  if (b.sideStream) cudaStreamDestroy(b.sideStream);
  cudaFreeHost(b.h_memGraph);
  if (b.memGraphEvent) cudaEventDestroy(b.memGraphEvent);
  if (b.ownStream && b.stream) cudaStreamDestroy(b.stream);
  b = Batch();
}

int batch_upload(Batch& b) {
  if (b.capturing) {
    set_error("descriptor upload inside a graph capture (a buffer changed during the step)");
    return SPHGPU_ERR_STATE;
  }
  const int nm = (int)b.mem.size();
  if (nm > b.memcap) {
    cudaStreamSynchronize(b.stream);
    dev_free(b.d_memRing); cudaFreeHost(b.h_memRing);
    b.d_memRing = nullptr; b.h_memRing = nullptr; b.d_mem = nullptr;
    const int cap = nm + 16;
    if (dev_alloc(reinterpret_cast<void**>(&b.d_memRing), sizeof(Member)*cap*Batch::kMemSlots) != cudaSuccess ||
        cudaMallocHost(&b.h_memRing, sizeof(Member)*cap*Batch::kMemSlots) != cudaSuccess) {
      set_error("batch descriptor allocation failed");
      b.memcap = 0;
      return SPHGPU_ERR_NOMEM;
    }
    b.memcap = cap;
  }
  // The next slot's host side must have been copied out (its upload, kMemSlots
  // uploads ago, has completed); kernels still reading its device side run
  // before the new copy because both are on the batch stream.
  const int slot = (b.memSlot + 1) % Batch::kMemSlots;
  cudaError_t e = cudaEventSynchronize(b.memEvents[slot]);
  if (e != cudaSuccess) return cuda_status(e, "batch descriptor event");
  Member* h = b.h_memRing + (size_t)slot*b.memcap;
  Member* d = b.d_memRing + (size_t)slot*b.memcap;
  for (int m = 0; m < nm; ++m) h[m] = member_of(*b.mem[m]);
  e = cudaMemcpyAsync(d, h, sizeof(Member)*nm, cudaMemcpyHostToDevice, b.stream);
  if (e != cudaSuccess) return cuda_status(e, "batch descriptor upload");
  e = cudaEventRecord(b.memEvents[slot], b.stream);
  if (e != cudaSuccess) return cuda_status(e, "batch descriptor event");
  b.memSlot = slot;
  b.d_mem = d;
  b.memDirty = false;
  return SPHGPU_OK;
}

int batch_map(Batch& b, const std::vector<int64_t>& blocks, BlockMap* bm, unsigned* grid) {
  const int nm = (int)blocks.size();
  if (nm == 1) {
    // one member: the kernel takes its block index directly
    if (blocks[0] > 0x7fffffffLL) { set_error("launch grid too large"); return SPHGPU_ERR_CAPACITY; }
    bm->first = nullptr;
    bm->nmem = 1;
    *grid = (unsigned)blocks[0];
    return SPHGPU_OK;
  }
  if (b.capturing) {
    // a captured graph keeps the map pointer: place the map in the arena,
    // copied synchronously on the side stream (outside the capture)
    std::vector<int32_t> h(nm + 1);
    int64_t total = 0;
    for (int m = 0; m < nm; ++m) { h[m] = (int32_t)total; total += blocks[m]; }
    if (total > 0x7fffffffLL) { set_error("launch grid too large"); return SPHGPU_ERR_CAPACITY; }
    h[nm] = (int32_t)total;
    const int64_t needA = ((int64_t)nm + 1 + 31) & ~(int64_t)31;
    if (b.mapArenaPos + needA > b.mapArenaCap) { set_error("graph block-map arena full"); return SPHGPU_ERR_CAPACITY; }
    int32_t* d = b.d_mapArena + b.mapArenaPos;
    cudaError_t e = cudaMemcpyAsync(d, h.data(), sizeof(int32_t)*(nm + 1), cudaMemcpyHostToDevice, b.sideStream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b.sideStream);
    if (e != cudaSuccess) return cuda_status(e, "graph map upload");
    b.mapArenaPos += needA;
    bm->first = d;
    bm->nmem = nm;
    *grid = (unsigned)total;
    return SPHGPU_OK;
  }
  const int64_t need = ((int64_t)nm + 1 + 31) & ~(int64_t)31;
  if (need > b.mapcap) { set_error("batch too large for the block-map ring"); return SPHGPU_ERR_CAPACITY; }
  if (b.mappos + need > b.mapcap) {
    // every earlier map copy has been consumed once the stream is idle
    const cudaError_t e = cudaStreamSynchronize(b.stream);
    if (e != cudaSuccess) return cuda_status(e, "batch map ring");
    b.mappos = 0;
  }
  int32_t* h = b.h_maps + b.mappos;
  int64_t total = 0;
  for (int m = 0; m < nm; ++m) {
    h[m] = (int32_t)total;
    total += blocks[m];
  }
  if (total > 0x7fffffffLL) { set_error("launch grid too large"); return SPHGPU_ERR_CAPACITY; }
  h[nm] = (int32_t)total;
  const cudaError_t e = cudaMemcpyAsync(b.d_maps + b.mappos, h, sizeof(int32_t)*(nm + 1), cudaMemcpyHostToDevice,
                                        b.stream);
  if (e != cudaSuccess) return cuda_status(e, "batch map upload");
  bm->first = b.d_maps + b.mappos;
  bm->nmem = nm;
  *grid = (unsigned)total;
  b.mappos += need;
  return SPHGPU_OK;
}

int batch_gather(Batch& b, const int* slots, int nslots, std::vector<double>& out) {
  const int nm = (int)b.mem.size();
  if (nslots < 1 || nslots > 8) { set_error("batch_gather: 1..8 slots"); return SPHGPU_ERR_ARG; }
  const int64_t need = (int64_t)nm*nslots;
  if (need > b.gathercap) {
    cudaStreamSynchronize(b.stream);
    dev_free(b.d_gather); cudaFreeHost(b.h_gather);
    b.d_gather = nullptr; b.h_gather = nullptr;
    const int64_t cap = need + 256;
    if (dev_alloc(reinterpret_cast<void**>(&b.d_gather), sizeof(double)*cap) != cudaSuccess ||
        cudaMallocHost(&b.h_gather, sizeof(double)*cap) != cudaSuccess) {
      b.gathercap = 0;
      set_error("batch gather allocation failed");
      return SPHGPU_ERR_NOMEM;
    }
    b.gathercap = cap;
  }
  if (b.memDirty) { const int rc = batch_upload(b); if (rc) return rc; }
  int s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < nslots; ++k) s[k] = slots[k];
  gather_scal_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm, make_int4(s[0], s[1], s[2], s[3]),
                                                           make_int4(s[4], s[5], s[6], s[7]), nslots,
                                                           b.d_gather);
  batch_count_launch(b);
  cudaError_t e = cudaMemcpyAsync(b.h_gather, b.d_gather, sizeof(double)*need, cudaMemcpyDeviceToHost, b.stream);
  if (e != cudaSuccess) return cuda_status(e, "batch gather copy");
  e = cudaStreamSynchronize(b.stream);
  if (e != cudaSuccess) return cuda_status(e, "batch gather");
  out.assign(b.h_gather, b.h_gather + need);
  return SPHGPU_OK;
}

void batch_count_launch(Batch& b) {
  ++b.launches;
  for (Problem* p : b.mem) ++p->launches;
}

void batch_set_scal(Batch& b, int slot, double value) {
  const int nm = (int)b.mem.size();
  set_scal_kernel<<<(nm + 127)/128, 128, 0, b.stream>>>(b.d_mem, nm, slot, value);
  batch_count_launch(b);
}

int batch_scan(Batch& b, int which) {
  std::vector<int64_t> tiles(b.mem.size()), ones(b.mem.size(), 1);
  for (size_t m = 0; m < b.mem.size(); ++m) {
    Problem& p = *b.mem[m];
    tiles[m] = scanBlocks(scan_items(p, which));
    if (tiles[m] + 1 > p.blockSumsCap) {
      const int rc = ensure_block_sums(p, kScanBlocks + 1);
      if (rc) return rc;
      b.memDirty = true;
    }
  }
  if (b.memDirty) { const int rc = batch_upload(b); if (rc) return rc; }
  BlockMap tm, om;
  unsigned tgrid = 0, ogrid = 0;
  int rc = batch_map(b, tiles, &tm, &tgrid);
  if (rc) return rc;
  rc = batch_map(b, ones, &om, &ogrid);
  if (rc) return rc;
  if (tgrid) { scan_tile_sums_kernel<<<tgrid, SCAN_THREADS, 0, b.stream>>>(b.d_mem, tm, which); batch_count_launch(b); }
  scan_sums_kernel<<<ogrid, SCAN_THREADS, 0, b.stream>>>(b.d_mem, om, which); batch_count_launch(b);
  if (tgrid) { scan_apply_kernel<<<tgrid, SCAN_THREADS, 0, b.stream>>>(b.d_mem, tm, which); batch_count_launch(b); }
  return cuda_status(cudaGetLastError(), "batch scan");
}

}  // namespace sphgpu
