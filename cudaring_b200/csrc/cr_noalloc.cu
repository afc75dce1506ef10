// Neighbour-list build that allocates nothing.
//
// Some callers cannot allocate device memory from inside their own code: a
// host framework that owns a fixed device memory budget and hands out only
// pre-sized buffers, or code that must not call cudaMalloc/cudaFree because
// those calls synchronise the whole device and stall every other stream.
// cr_neighbor_list_noalloc serves them: it runs the same cell-list kernels as
// cr_calc_neighbor_list on device buffers the caller passes, and keeps every
// temporary in one static device array of this file, so it never calls
// cudaMalloc, cudaFree or any allocating library routine.
//
// Limits and rules of use:
//   * at most CR_NOALLOC_MAX_VERTICES vertices (the scratch array is sized
//     for these; every GPU that loads the library keeps it, about 4.2 MB,
//     until the process exits); larger inputs return CR_EINVAL before any
//     buffer is touched.  The cell grid is coarsened to at most
//     CR_NOALLOC_MAX_CELLS cells (larger cells hold every pair the finer grid
//     did, so the list is the same);
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device) and keeps it for the life of the
//     process; make that first call before any stream capture.  After
//     cudaDeviceReset on that device the kept address is stale: do not call
//     this entry point on a device that was reset;
//   * the call waits for its stream (it reads the largest count back);
//   * all calls share the one array, so calls that overlap on the GPU (other
//     streams, other host threads) race; serialise them.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "cr_launch.h"
#include "cr_tile.cuh"

namespace {

constexpr long kMaxVertices = CR_NOALLOC_MAX_VERTICES;
constexpr long kMaxCells = CR_NOALLOC_MAX_CELLS;

// Layout of the scratch array (byte offsets, each 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffStatus = 0;
constexpr size_t kOffCellOf = align256(kOffStatus + sizeof(cr::DevStatus));
constexpr size_t kOffSlot = align256(kOffCellOf + kMaxVertices * sizeof(int));
constexpr size_t kOffCellVid = align256(kOffSlot + kMaxVertices * sizeof(int));
constexpr size_t kOffCellRing = align256(kOffCellVid + kMaxVertices * sizeof(int));
constexpr size_t kOffCellPos = align256(kOffCellRing + kMaxVertices * sizeof(int));
constexpr size_t kOffCellRad = align256(kOffCellPos + kMaxVertices * sizeof(double2));
constexpr size_t kOffLastPos = align256(kOffCellRad + kMaxVertices * sizeof(double));
constexpr size_t kOffCellCnt = align256(kOffLastPos + kMaxVertices * sizeof(double2));
constexpr size_t kOffCellStart = align256(kOffCellCnt + kMaxCells * sizeof(int));
constexpr size_t kScratchBytes = align256(kOffCellStart + (kMaxCells + 1) * sizeof(int));

}  // namespace

// The scratch memory itself: file scope, fixed size, one copy per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_mu;
void* g_scratch_addr[128] = {nullptr};

// Device address of g_noalloc_scratch on the current device (host code may
// not use the symbol itself as a pointer).
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return CR_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CR_ECUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return CR_OK;
}

}  // namespace

extern "C" int cr_neighbor_list_noalloc(const double* pos, const double* rad, const int* ring_of,
                                        long numVertices, const double* boxSize, double maxRad,
                                        double cutDistance, long capacity, int* neighbors, int* counts,
                                        long* maxCount, void* stream) {
  if (!pos || !rad || !ring_of || !boxSize || !neighbors || !counts || !maxCount) return CR_EINVAL;
  if (numVertices <= 0 || numVertices > kMaxVertices || capacity < 0 || capacity > (1L << 20)) return CR_EINVAL;
  if (!(boxSize[0] > 0) || !(boxSize[1] > 0) || !(maxRad > 0) || !(cutDistance > -1.0)) return CR_EINVAL;
  cr::SysParams p{};
  p.nv = (int)numVertices;
  p.lx = boxSize[0];
  p.ly = boxSize[1];
  p.inv_lx = 1.0 / p.lx;
  p.inv_ly = 1.0 / p.ly;
  // the same cell rule as the context's build: cells no smaller than the
  // largest neighbour distance, brute force below three cells per side
  const double cmin = (1.0 + cutDistance) * 2.0 * maxRad * (1.0 + 1e-9);
  long ncx = (long)std::min(p.lx / cmin, 1048576.0), ncy = (long)std::min(p.ly / cmin, 1048576.0);
  cr::CellGrid g{0, 0, 0.0, 0.0};
  if (ncx >= 3 && ncy >= 3) {
    if (ncx * ncy > kMaxCells) {
      // coarsen to the scratch array's cell budget, at least three cells a side
      const double f = std::sqrt((double)kMaxCells / (double)(ncx * ncy));
      ncx = std::max(3L, (long)std::floor((double)ncx * f));
      ncy = std::max(3L, (long)std::floor((double)ncy * f));
      if (ncx * ncy > kMaxCells) {
        if (ncx > ncy) ncx = std::max(3L, kMaxCells / ncy);
        else ncy = std::max(3L, kMaxCells / ncx);
      }
    }
    g = cr::CellGrid{(int)ncx, (int)ncy, p.lx / ncx, p.ly / ncy};
  }
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char* s = static_cast<unsigned char*>(base);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cr::NbrArgs n;
  n.pos = reinterpret_cast<const double2*>(pos);
  n.rad = rad;
  n.ring_of = ring_of;
  n.nbr = neighbors;
  n.nbr_cnt = counts;
  n.cap = (int)capacity;
  n.cut_distance = cutDistance;
  n.last_pos = reinterpret_cast<double2*>(s + kOffLastPos);
  n.cell_of = reinterpret_cast<int*>(s + kOffCellOf);
  n.slot = reinterpret_cast<int*>(s + kOffSlot);
  n.cell_cnt = reinterpret_cast<int*>(s + kOffCellCnt);
  n.cell_start = reinterpret_cast<int*>(s + kOffCellStart);
  n.cell_vid = reinterpret_cast<int*>(s + kOffCellVid);
  n.cell_pos = reinterpret_cast<double2*>(s + kOffCellPos);
  n.cell_rad = reinterpret_cast<double*>(s + kOffCellRad);
  n.cell_ring = reinterpret_cast<int*>(s + kOffCellRing);
  n.status = reinterpret_cast<cr::DevStatus*>(s + kOffStatus);
  n.count_op = 0;
  n.count_update = 0;
  // the status block and the per-cell counters must start at zero; the array
  // keeps whatever the previous call left in it
  if (cudaMemsetAsync(s + kOffStatus, 0, sizeof(cr::DevStatus), st) != cudaSuccess) return CR_ECUDA;
  if (g.ncx && cudaMemsetAsync(s + kOffCellCnt, 0, (size_t)g.ncx * g.ncy * sizeof(int), st) != cudaSuccess)
    return CR_ECUDA;
  cr::launch_nbr_build(st, p, g, n);
  if (cudaGetLastError() != cudaSuccess) return CR_ECUDA;
  int mc = 0;
  if (cudaMemcpyAsync(&mc, s + kOffStatus + offsetof(cr::DevStatus, max_count), sizeof(int),
                      cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CR_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CR_ECUDA;
  *maxCount = mc;
  return mc > capacity ? CR_ENBR_OVERFLOW : CR_OK;
}
