// Neighbour-list build on a periodic cell grid.
//
// Rule (kernelCalcNeighborList, include/cudaKernel.cuh:1735-1763): j is a
// neighbour of i iff ring(j) != ring(i) and -(1 - d_ij/(r_i + r_j)) <
// cutDistance, d_ij the minimum-image distance.  The host picks cells no
// smaller than (1 + cutDistance) * 2 * max(rad) (plus a relative margin), so
// every such pair lies in the 3x3 cell stencil and the set equals the
// reference's O(Nv^2) scan; the test itself is evaluated with the same
// expression.  Systems with fewer than 3 cells per side use the brute-force
// kernel.
//
// Kernels (all graph-capturable, no host synchronisation):
//   k_cell_count   cell of each vertex + slot inside the cell (atomic)
//   k_cell_scan    exclusive scan of the cell counts (one CTA), zeroes counts
//   k_cell_fill    scatter vertex ids by cell
//   k_cell_sort    sort each cell's ids ascending (in registers up to 16)
//   k_cell_gather  copy pos/rad/ring/offsets into cell order (SoA)
//   k_nbr_cells    stencil search, 16 lanes per vertex (one stencil cell per
//                  lane, counts scanned across lanes) -> slot-major list (and its companion of
//                  packed ring-predecessor offsets), counts, overflow flag,
//                  lastPos = pos; the last CTA publishes the build to status
#include <algorithm>

#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

__device__ __forceinline__ int cell_coord(double x, double L, double invL, int nc) {
  double w = x - L * floor(x * invL);          // wrap into [0, L]
  int c = (int)(w * (nc * invL));
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_cell_count(const __grid_constant__ SysParams p, int ncx, int ncy, const double2* pos, int* cell_of,
                             int* slot, int* cell_cnt) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < p.nv) {
    const double2 x = pos[v];
    const int cx = cell_coord(x.x, p.lx, p.inv_lx, ncx);
    const int cy = cell_coord(x.y, p.ly, p.inv_ly, ncy);
    const int c = cy * ncx + cx;
    cell_of[v] = c;
    slot[v] = atomicAdd(cell_cnt + c, 1);
  }
}

// One CTA of 1024 threads: chunked exclusive scan over ncells counts.
__global__ void __launch_bounds__(1024) k_cell_scan(int ncells, int* cell_cnt, int* cell_start) {
  __shared__ int s_w[32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int chunk = (ncells + 1023) / 1024;
  const int b = t * chunk, e = min(ncells, b + chunk);
  int sum = 0;
  for (int c = b; c < e; c++) sum += cell_cnt[c];
  // block-wide inclusive scan of the chunk sums: warp shuffles, then the 32 warp totals
  int incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = s_w[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_w[lane] = w;
  }
  __syncthreads();
  int run = incl - sum + (warp > 0 ? s_w[warp - 1] : 0);  // exclusive prefix of this chunk
  for (int c = b; c < e; c++) {
    const int n = cell_cnt[c];
    cell_start[c] = run;
    run += n;
    cell_cnt[c] = 0;
  }
  if (t == 1023) cell_start[ncells] = s_w[31];
}

__global__ void k_cell_fill(int nv, const int* cell_of, const int* slot, const int* cell_start, int* cell_vid) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) cell_vid[cell_start[cell_of[v]] + slot[v]] = v;
}

// Ascending ids in cell entries [b, e) (the atomic slots of k_cell_count come
// in scheduling order): cells of up to 16 vertices are sorted in registers.
__device__ __forceinline__ void sort_cell(int b, int e, int* cell_vid) {
  const int n = e - b;
  if (n <= 1) return;
  if (n <= 16) {
    int ids[16];
#pragma unroll
    for (int i = 0; i < 16; i++) ids[i] = (i < n) ? cell_vid[b + i] : 0x7fffffff;
#pragma unroll
    for (int i = 1; i < 16; i++) {
#pragma unroll
      for (int j = i; j > 0; j--) {
        const int lo = min(ids[j - 1], ids[j]), hi = max(ids[j - 1], ids[j]);
        ids[j - 1] = lo;
        ids[j] = hi;
      }
    }
#pragma unroll
    for (int i = 0; i < 16; i++)
      if (i < n) cell_vid[b + i] = ids[i];
    return;
  }
  for (int i = b + 1; i < e; i++) {
    const int key = cell_vid[i];
    int j = i - 1;
    while (j >= b && cell_vid[j] > key) {
      cell_vid[j + 1] = cell_vid[j];
      j--;
    }
    cell_vid[j + 1] = key;
  }
}

__global__ void k_cell_sort(int ncells, const int* cell_start, int* cell_vid) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncells) sort_cell(cell_start[c], cell_start[c + 1], cell_vid);
}

// SoA copies in cell order for the stencil search, one thread per entry.
__global__ void k_cell_gather(int nv, const int* cell_start_end, const int* cell_vid, const double2* pos,
                              const double* rad, const int* ring_of, const int* pq_pack, double2* cell_pos,
                              double* cell_rad, int* cell_ring, int* cell_pq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv || i >= *cell_start_end) return;
  const int v = cell_vid[i];
  cell_pos[i] = pos[v];
  cell_rad[i] = rad[v];
  cell_ring[i] = ring_of[v];
  if (cell_pq) cell_pq[i] = pq_pack[v];
}

__device__ __forceinline__ bool is_neighbor(const SysParams& p, double2 xi, double2 xj, double rsum, double cut) {
  // -calcOverlap(thisPos, otherPos, radSum) < cutDistance (include/cudaKernel.cuh:1752)
  const double d = dist_of(pbc2(p, xi, xj));
  return -(1.0 - d / rsum) < cut;
}

__device__ __forceinline__ void publish_build(const NbrArgs& n, int my_max, int my_overflow) {
  DevStatus* st = n.status;
  if (my_overflow) atomicOr(&st->overflow, 1);
  if (my_max > 0) atomicMax(&st->max_count, my_max);
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      __threadfence();
      if (st->max_count > st->max_ever) st->max_ever = st->max_count;
      if (st->abort) {
        // an earlier op of this sequence failed; leave its state alone
      } else if (st->overflow) {
        st->abort = 1;
      } else {
        st->rebuild = 0;
        if (n.count_update) st->update_count += 1;
        if (n.count_op) st->ops_done += 1;
      }
      st->bar_count = 0;  // every CTA is past the one-launch build's last barrier
      st->done_ctr = 0;
    }
  }
}

// 16 lanes per vertex (two vertices per warp): lane l < 9 scans stencil cell
// l (dy = l / 3 - 1, dx = l % 3 - 1, the sequential order), counts its
// neighbours, and after an exclusive scan of the counts over the lanes writes
// them at its offset, so a vertex's list has the sequential scan's order.
constexpr int kNbrLanes = 16;

// The stencil search of vertex g by the 16 lanes of its group (all 16 lanes
// call it; valid = g < nv); ids[k] is the vertex at cell-order entry k.
// Writes the list, count and lastPos; returns the count on lane 0, 0
// elsewhere.
__device__ __forceinline__ int stencil_vertex(const SysParams& p, int ncx, int ncy, const NbrArgs& n,
                                              const int* ids, int g, int lane, bool valid) {
  int mine = 0, kb = 0, ke = 0;
  unsigned int hits = 0u;  // neighbours among the cell's first 32 entries
  double2 xi = make_double2(0.0, 0.0);
  double ri = 0.0;
  int ring = -1;
  if (valid && lane < 9) {
    xi = n.pos[g];
    ri = n.rad[g];
    ring = n.ring_of[g];
    const int c = n.cell_of[g];
    const int cx = c % ncx, cy = c / ncx;
    int yy = cy + lane / 3 - 1;
    yy += (yy < 0) ? ncy : 0;
    yy -= (yy >= ncy) ? ncy : 0;
    int xx = cx + lane % 3 - 1;
    xx += (xx < 0) ? ncx : 0;
    xx -= (xx >= ncx) ? ncx : 0;
    const int cc = yy * ncx + xx;
    kb = n.cell_start[cc];
    ke = n.cell_start[cc + 1];
    // entries in groups of four, loaded before any is tested (the last
    // group re-reads entry ke - 1 in its unused slots and ignores it)
    for (int k0 = kb; k0 < ke; k0 += 4) {
      int rj[4];
      double2 xj[4];
      double rr[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = min(k0 + u, ke - 1);
        rj[u] = n.cell_ring[k];
        xj[u] = n.cell_pos[k];
        rr[u] = n.cell_rad[k];
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = k0 + u;
        if (k < ke && rj[u] != ring && is_neighbor(p, xi, xj[u], ri + rr[u], n.cut_distance)) {
          if (k - kb < 32) hits |= 1u << (k - kb);
          mine++;
        }
      }
    }
  }
  // exclusive scan of the lane counts inside the 16-lane group
  int incl = mine;
  for (int o = 1; o < kNbrLanes; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o, kNbrLanes);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(0xffffffffu, incl, kNbrLanes - 1, kNbrLanes);
  int slot = incl - mine;
  if (valid && lane < 9 && mine > 0) {
    if (ke - kb <= 32) {
      while (hits) {
        const int k = kb + __ffs(hits) - 1;
        hits &= hits - 1u;
        if (slot < n.cap) {
          n.nbr[(size_t)slot * p.nv + g] = ids[k];
          if (n.nbr_pq) n.nbr_pq[(size_t)slot * p.nv + g] = n.cell_pq[k];
        }
        slot++;
      }
    } else {
      for (int k = kb; k < ke; k++) {
        if (n.cell_ring[k] != ring && is_neighbor(p, xi, n.cell_pos[k], ri + n.cell_rad[k], n.cut_distance)) {
          if (slot < n.cap) {
            n.nbr[(size_t)slot * p.nv + g] = ids[k];
            if (n.nbr_pq) n.nbr_pq[(size_t)slot * p.nv + g] = n.cell_pq[k];
          }
          slot++;
        }
      }
    }
  }
  if (valid && lane == 0) {
    n.nbr_cnt[g] = total;
    n.last_pos[g] = n.pos[g];
    return total;
  }
  return 0;
}

// CTA-wide maximum of m (every thread calls it); the result on thread 0.
__device__ __forceinline__ int block_max(int m) {
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ int s_max[32];
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  int bm = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) bm = max(bm, s_max[w]);
  return bm;
}

__global__ void __launch_bounds__(256) k_nbr_cells(const __grid_constant__ SysParams p, int ncx, int ncy,
                                                   const __grid_constant__ NbrArgs n) {
  const int g = blockIdx.x * (256 / kNbrLanes) + threadIdx.x / kNbrLanes;  // vertex
  const int lane = threadIdx.x % kNbrLanes;
  const int m = stencil_vertex(p, ncx, ncy, n, n.cell_vid, g, lane, g < p.nv);
  const int bm = block_max(m);
  publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap);
}

// Brute force for boxes with fewer than three cells per side.
__device__ __forceinline__ int brute_vertex(const SysParams& p, const NbrArgs& n, int i) {
  const double2 xi = n.pos[i];
  const double ri = n.rad[i];
  const int ring = n.ring_of[i];
  int cnt = 0;
  for (int j = 0; j < p.nv; j++) {
    if (n.ring_of[j] == ring) continue;
    if (is_neighbor(p, xi, n.pos[j], ri + n.rad[j], n.cut_distance)) {
      if (cnt < n.cap) {
        n.nbr[(size_t)cnt * p.nv + i] = j;
        if (n.nbr_pq) n.nbr_pq[(size_t)cnt * p.nv + i] = n.pq_pack[j];
      }
      cnt++;
    }
  }
  n.nbr_cnt[i] = cnt;
  n.last_pos[i] = xi;
  return cnt;
}

__global__ void __launch_bounds__(256) k_nbr_brute(const __grid_constant__ SysParams p,
                                                   const __grid_constant__ NbrArgs n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int bm = block_max(i < p.nv ? brute_vertex(p, n, i) : 0);
  publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap);
}

// The build skips itself when an earlier op aborted the sequence.
__global__ void k_nbr_guard_reset(DevStatus* st) {
  if (threadIdx.x == 0) {
    st->overflow = 0;
    st->max_count = 0;
  }
}

void launch_cell_scan(cudaStream_t st, int ncells, int* cell_cnt, int* cell_start) {
  k_cell_scan<<<1, 1024, 0, st>>>(ncells, cell_cnt, cell_start);
}

void launch_cell_sort(cudaStream_t st, int ncells, int nv, const NbrArgs& n) {
  k_cell_sort<<<(ncells + 127) / 128, 128, 0, st>>>(ncells, n.cell_start, n.cell_vid);
  k_cell_gather<<<(nv + 255) / 256, 256, 0, st>>>(nv, n.cell_start + ncells, n.cell_vid, n.pos, n.rad, n.ring_of,
                                                  n.nbr_pq ? n.pq_pack : nullptr, n.cell_pos, n.cell_rad,
                                                  n.cell_ring, n.nbr_pq ? n.cell_pq : nullptr);
}

void launch_nbr_build(cudaStream_t stream, const SysParams& p, const CellGrid& g, const NbrArgs& n) {
  const int nb = (p.nv + 255) / 256;
  k_nbr_guard_reset<<<1, 32, 0, stream>>>(n.status);
  if (g.ncx >= 3 && g.ncy >= 3) {
    const int ncells = g.ncx * g.ncy;
    k_cell_count<<<nb, 256, 0, stream>>>(p, g.ncx, g.ncy, n.pos, n.cell_of, n.slot, n.cell_cnt);
    k_cell_scan<<<1, 1024, 0, stream>>>(ncells, n.cell_cnt, n.cell_start);
    k_cell_fill<<<nb, 256, 0, stream>>>(p.nv, n.cell_of, n.slot, n.cell_start, n.cell_vid);
    launch_cell_sort(stream, ncells, p.nv, n);
    k_nbr_cells<<<(p.nv + 256 / kNbrLanes - 1) / (256 / kNbrLanes), 256, 0, stream>>>(p, g.ncx, g.ncy, n);
  } else {
    k_nbr_brute<<<nb, 256, 0, stream>>>(p, n);
  }
}

// ------------------------------------------------------- one-launch build
//
// The phases above in one launch, for step sequences captured in graphs: the
// kernel follows every op that may arm a rebuild and returns at once unless
// the op armed one, so a step that needs no rebuild pays one early-exit launch
// instead of a conditional graph node.  When armed, the phases run back to
// back with grid-wide barriers between them:
//   1 cell + slot of every vertex             (k_cell_count)
//   2 per-CTA totals of a contiguous cell range
//   3 exclusive scan: CTA offset from the totals, then the range (k_cell_scan)
//   4 scatter ids by cell                     (k_cell_fill)
//   5 per vertex: rank in its cell by id, copy to that entry
//                                             (k_cell_sort + k_cell_gather)
//   6 stencil search, 16 lanes per vertex     (k_nbr_cells)
// and the last CTA publishes the build exactly as the multi-kernel path does,
// so both paths produce the same list.  The grid never exceeds the CTAs the
// GPU holds at once (occupancy x SMs, nbr_fused_max_blocks), so every CTA is
// resident while the others wait.  Every wait is bounded: a barrier that does
// not complete within about a second (2^20 polls) sets status.stalled and
// abort, and the CTAs return without finishing the build.

constexpr int kFusedBlock = 1024;
constexpr int kFusedMinBlocks = 1;
constexpr long kBarrierSpins = 1L << 20;

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* a) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int atom_add_release_u32(unsigned int* a, unsigned int x) {
  unsigned int old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(a), "r"(x) : "memory");
  return old;
}

// Grid barrier on one counter: bar_count is zero when the build starts (the
// publishing CTA clears it after every CTA has passed the last barrier), and
// barrier i completes when it reaches i * gridDim.x.  Arrival is a release
// add (this CTA's writes, ordered before it by __syncthreads, become visible
// first); the wait is an acquire load, so what the other CTAs wrote before
// arriving is visible after it.
__device__ bool grid_barrier(DevStatus* st) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int prev = atom_add_release_u32(&st->bar_count, 1u);
    const unsigned int target = (prev / gridDim.x + 1u) * gridDim.x;
    long it = 0;
    while (ld_acquire_u32(&st->bar_count) < target) {
      if (++it > kBarrierSpins || *(volatile int*)&st->stalled) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    if (!ok) {
      atomicExch(&st->stalled, 1);
      atomicExch(&st->abort, 1);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Inclusive CTA-wide scan of x; *total receives the CTA's sum.
__device__ __forceinline__ int block_scan(int x, int* total) {
  __shared__ int s_w[kFusedBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = x;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kFusedBlock / 32 ? s_w[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kFusedBlock / 32) s_w[lane] = w;
  }
  __syncthreads();
  const int r = incl + (warp > 0 ? s_w[warp - 1] : 0);
  *total = s_w[kFusedBlock / 32 - 1];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kFusedBlock, kFusedMinBlocks)
    k_nbr_fused(const __grid_constant__ SysParams p, int ncx, int ncy, const __grid_constant__ NbrArgs n, int force) {
  DevStatus* st = n.status;
  if (!force) {
    const volatile DevStatus* vs = st;
    if (!vs->rebuild || vs->abort || vs->converged) return;
  }
  const int nv = p.nv;
  const int nthreads = gridDim.x * kFusedBlock;
  const int gt = blockIdx.x * kFusedBlock + threadIdx.x;
  if (ncx < 3 || ncy < 3) {
    int m = 0;
    for (int i = gt; i < nv; i += nthreads) m = max(m, brute_vertex(p, n, i));
    const int bm = block_max(m);
    publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap);
    return;
  }
  const int ncells = ncx * ncy;
  // 1: cells and slots (the counts are zero between builds)
  if (gt == 0) {
    st->overflow = 0;
    st->max_count = 0;
  }
  for (int v = gt; v < nv; v += nthreads) {
    const double2 x = n.pos[v];
    const int c = cell_coord(x.y, p.ly, p.inv_ly, ncy) * ncx + cell_coord(x.x, p.lx, p.inv_lx, ncx);
    n.cell_of[v] = c;
    n.slot[v] = atomicAdd(n.cell_cnt + c, 1);
  }
  if (!grid_barrier(st)) return;
  // 2: this CTA's cells [cb, ce), this thread's [tb, te)
  const int per_block = (ncells + gridDim.x - 1) / gridDim.x;
  const int cb = min(ncells, (int)blockIdx.x * per_block), ce = min(ncells, cb + per_block);
  const int per_thread = (ce - cb + kFusedBlock - 1) / kFusedBlock;
  const int tb = min(ce, cb + (int)threadIdx.x * per_thread), te = min(ce, tb + per_thread);
  int sum = 0;
  for (int c = tb; c < te; c++) sum += n.cell_cnt[c];
  int cta_total = 0;
  const int incl = block_scan(sum, &cta_total);
  if (threadIdx.x == 0) n.block_sum[blockIdx.x] = cta_total;
  if (!grid_barrier(st)) return;
  // 3: offset of this CTA = totals of the CTAs before it
  int part = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += kFusedBlock) part += n.block_sum[b];
  int offset = 0;
  block_scan(part, &offset);
  int run = offset + incl - sum;
  for (int c = tb; c < te; c++) {
    const int k = n.cell_cnt[c];
    n.cell_start[c] = run;
    run += k;
    n.cell_cnt[c] = 0;
  }
  if (tb < te && te == ncells) n.cell_start[ncells] = run;
  if (!grid_barrier(st)) return;
  // 4: scatter
  for (int v = gt; v < nv; v += nthreads) n.cell_vid[n.cell_start[n.cell_of[v]] + n.slot[v]] = v;
  if (!grid_barrier(st)) return;
  // 5: every vertex takes entry cell_start + (members of its cell with a
  // smaller id), the ascending order k_cell_sort produces; the ids in cell
  // order go to `slot`, whose per-vertex slots phase 4 has consumed
  for (int v = gt; v < nv; v += nthreads) {
    const int b = n.cell_start[n.cell_of[v]], e = n.cell_start[n.cell_of[v] + 1];
    int rank = 0;
#pragma unroll 4
    for (int i = b; i < e; i++) rank += (n.cell_vid[i] < v) ? 1 : 0;
    const int k = b + rank;
    n.slot[k] = v;
    n.cell_pos[k] = n.pos[v];
    n.cell_rad[k] = n.rad[v];
    n.cell_ring[k] = n.ring_of[v];
    if (n.nbr_pq) n.cell_pq[k] = n.pq_pack[v];
  }
  if (!grid_barrier(st)) return;
  // 6: stencil search; the loop bound is uniform over a warp (two vertices
  // per warp) so the 16-lane shuffles see full warps
  const int lane = threadIdx.x % kNbrLanes, half = (threadIdx.x / kNbrLanes) & 1;
  const int nwarps = nthreads / 32;
  int m = 0;
  for (int g0 = 2 * (gt / 32); g0 < nv; g0 += 2 * nwarps) {
    const int g = g0 + half;
    m = max(m, stencil_vertex(p, ncx, ncy, n, n.slot, g, lane, g < nv));
  }
  const int bm = block_max(m);
  publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap);
}

int nbr_fused_max_blocks() {
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_nbr_fused, kFusedBlock, 0) != cudaSuccess) return 0;
  return occ * sms;
}

int nbr_fused_blocks(int nv, int max_blocks) {
  const long want = ((long)nv * kNbrLanes + kFusedBlock - 1) / kFusedBlock;
  return (int)std::max(1L, std::min<long>(want, max_blocks));
}

void launch_nbr_fused(cudaStream_t st, const SysParams& p, const CellGrid& g, const NbrArgs& n, int blocks,
                      int force) {
  k_nbr_fused<<<blocks, kFusedBlock, 0, st>>>(p, g.ncx, g.ncy, n, force);
}

}  // namespace cr
