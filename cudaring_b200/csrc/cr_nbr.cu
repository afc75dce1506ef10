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
//   k_nbr_cells    stencil search, one warp per home cell (candidates one per
//                  lane, home vertices staged in shared memory) -> slot-major
//                  list (and its companion of packed ring-predecessor
//                  offsets), counts, overflow flag, lastPos = pos; the last
//                  CTA publishes the build to status
#include <algorithm>

#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

// CTA size of the one-launch build (one CTA per SM)
constexpr int kFusedBlock = 1024;
constexpr int kFusedMinBlocks = 1;

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

// -calcOverlap(thisPos, otherPos, radSum) < cutDistance
// (include/cudaKernel.cuh:1752), i.e. d < (1 + cut) * rsum.  The squared
// distance decides every pair outside a relative band of 1e-9 around the
// threshold (rounding moves either side by ~1e-16), the reference expression
// decides the pairs inside it, so the decisions are those of the reference
// expression while most pairs skip its square root and division.
__device__ __forceinline__ double pair_sq(const SysParams& p, double2 xi, double2 xj) {
  const double2 dl = pbc2(p, xi, xj);
  double sq = dl.x * dl.x;
  return fma(dl.y, dl.y, sq);
}
// 1: neighbour, 0: not, -1: inside the band (the reference expression decides)
__device__ __forceinline__ int pre_test(double sq, double rsum, double cut) {
  if (!(cut > -0.5)) return -1;
  const double t = (1.0 + cut) * rsum;
  const double t2 = t * t;
  return (sq < t2 * (1.0 - 1e-9)) ? 1 : ((sq > t2 * (1.0 + 1e-9)) ? 0 : -1);
}
__device__ __forceinline__ bool exact_test(double sq, double rsum, double cut) {
  return -(1.0 - sqrt(sq) / rsum) < cut;
}
__device__ __forceinline__ bool is_neighbor(const SysParams& p, double2 xi, double2 xj, double rsum, double cut) {
  const double sq = pair_sq(p, xi, xj);
  const int pt = pre_test(sq, rsum, cut);
  return pt >= 0 ? pt == 1 : exact_test(sq, rsum, cut);
}

// ctl (bucket form of the one-launch build): the control words after the two
// count arrays; the last CTA makes the other array current when this build
// left counts in the current one (bucket_pass), and clears the bucket
// overflow word.
__device__ __forceinline__ void publish_build(const NbrArgs& n, int my_max, int my_overflow, int* ctl = nullptr,
                                              bool bucket_pass = false) {
  DevStatus* st = n.status;
  if (my_overflow) atomicOr(&st->overflow, 1);
  if (my_max > 0) atomicMax(&st->max_count, my_max);
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      __threadfence();
      if (ctl) {
        if (bucket_pass) ctl[0] ^= 1;
        ctl[1] = 0;
      }
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

// Per-warp shared staging of the home vertices (32 at a time): positions
// relative to the home cell's corner and radii in single precision for the
// pre-test, ring and id.
struct HomeStage {
  float2 x[32];
  float r[32];
  int ring[32];
  int id[32];
};

// Single-precision pre-test.  Positions are taken relative to the home
// cell's corner o (each candidate shifted by the box length its stencil
// cell was wrapped by, which is its minimum image whenever it lies within
// range: cells are no smaller than the largest neighbour distance and there
// are at least three per side), so every coordinate is below R = 3 cells in
// magnitude and carries an absolute rounding error below e = 2^-22 R after
// the conversion.  With t = (1 + cut) rsum, the squared distance then lies
// within M = 1e-5 t^2 + 4 t e + 4 e^2 of the exact one wherever the exact
// one is below (t^2 + M): pairs with sq < t^2 - M are neighbours, pairs with
// sq > t^2 + M are not, and the few in between take the double-precision
// test, whose decisions are the reference expression's.
struct PreTest {
  double ox, oy;     // home cell corner
  float e4, ee4;     // 4 e, 4 e^2
  float opc;         // 1 + cut
  bool on;           // cut > -0.5 (else every pair takes the exact test)
};

__device__ __forceinline__ float2 rel_f(const SysParams& p, const PreTest& pt, double2 x, double sx, double sy) {
  const double wx = x.x - p.lx * floor(x.x * p.inv_lx) + sx;
  const double wy = x.y - p.ly * floor(x.y * p.inv_ly) + sy;
  return make_float2((float)(wx - pt.ox), (float)(wy - pt.oy));
}

// One warp per home cell.  The candidates are the entries of the 3x3 stencil
// cells concatenated in the sequential scan's order (stencil cell l = 0..8,
// dy = l / 3 - 1, dx = l % 3 - 1; inside a cell, cell order), 32 at a time,
// one per lane.  For each home vertex h of the cell (staged in shared
// memory) the lanes test their candidate, a ballot marks the hits, and hit
// lanes write at h's running count plus the hits on lower lanes, so every
// vertex's list has the sequential scan's order.  ids[k] is the vertex at
// cell-order entry k.  Writes lists, counts and lastPos of the cell's
// vertices; returns the largest count on the lanes that held a home vertex
// (0 elsewhere).
__device__ __forceinline__ int stencil_cell(const SysParams& p, int ncx, int ncy, const NbrArgs& n, const int* ids,
                                            int c, int lane, HomeStage& hs) {
  constexpr unsigned kAll = 0xffffffffu;
  const int cx = c % ncx, cy = c / ncx;
  int sb = 0, se = 0;
  if (lane < 9) {
    int yy = cy + lane / 3 - 1;
    yy += (yy < 0) ? ncy : 0;
    yy -= (yy >= ncy) ? ncy : 0;
    int xx = cx + lane % 3 - 1;
    xx += (xx < 0) ? ncx : 0;
    xx -= (xx >= ncx) ? ncx : 0;
    const int cc = yy * ncx + xx;
    sb = n.cell_start[cc];
    se = n.cell_start[cc + 1];
  }
  const int len = se - sb;
  int incl = len;  // inclusive offsets of the nine segments
  for (int o = 1; o < 16; o <<= 1) {
    const int y = __shfl_up_sync(kAll, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(kAll, incl, 8);
  const int off = incl - len;
  const int hb = __shfl_sync(kAll, sb, 4), he = __shfl_sync(kAll, se, 4);  // the home cell
  PreTest pt;
  {
    const double cw = p.lx / ncx, ch = p.ly / ncy;
    pt.ox = cx * cw;
    pt.oy = cy * ch;
    const float e = (float)(3.0 * fmax(cw, ch) * 0x1p-22);
    pt.e4 = 4.0f * e;
    pt.ee4 = 4.0f * e * e;
    pt.opc = (float)(1.0 + n.cut_distance);
    pt.on = n.cut_distance > -0.5;
  }
  // candidate q of the concatenated stencil list (k = -1 past its end)
  auto load = [&](int q, int& k, int& rj, float2& xf, float& rf, int& idj, int& pqj) {
    k = -1;
    int seg = 0;
#pragma unroll
    for (int sg = 0; sg < 9; sg++) {
      const int o_s = __shfl_sync(kAll, off, sg), b_s = __shfl_sync(kAll, sb, sg), l_s = __shfl_sync(kAll, len, sg);
      if (q >= o_s && q < o_s + l_s) {
        k = b_s + (q - o_s);
        seg = sg;
      }
    }
    rj = -1;
    idj = 0;
    pqj = 0;
    xf = make_float2(0.0f, 0.0f);
    rf = 0.0f;
    if (k >= 0) {
      const int ux = cx + seg % 3 - 1, uy = cy + seg / 3 - 1;  // unwrapped stencil cell
      const double sx = ux < 0 ? -p.lx : (ux >= ncx ? p.lx : 0.0);
      const double sy = uy < 0 ? -p.ly : (uy >= ncy ? p.ly : 0.0);
      rj = n.cell_ring[k];
      xf = rel_f(p, pt, n.cell_pos[k], sx, sy);
      rf = (float)n.cell_rad[k];
      idj = ids[k];
      if (n.nbr_pq) pqj = n.cell_pq[k];
    }
  };
  int maxc = 0;
  for (int h0 = hb; h0 < he; h0 += 32) {
    const int nh = min(32, he - h0);
    double2 xh = make_double2(0.0, 0.0);
    double rh = 0.0;
    int ringh = -1, gh = 0;
    // the home vertices and the first 32 candidates are loaded together,
    // and every later group of 32 while the one before is tested
    if (lane < nh) {
      xh = n.cell_pos[h0 + lane];
      rh = n.cell_rad[h0 + lane];
      ringh = n.cell_ring[h0 + lane];
      gh = ids[h0 + lane];
    }
    int k, rj, idj, pqj;
    float2 xf;
    float rf;
    load(lane, k, rj, xf, rf, idj, pqj);
    __syncwarp();  // the previous chunk's readers are done with hs
    if (lane < nh) {
      hs.x[lane] = rel_f(p, pt, xh, 0.0, 0.0);
      hs.r[lane] = (float)rh;
      hs.ring[lane] = ringh;
      hs.id[lane] = gh;
    }
    __syncwarp();
    int cnt = 0;  // on lane h: neighbours of home vertex h so far
    for (int q0 = 0; q0 < total; q0 += 32) {
      int k2 = -1, rj2 = -1, idj2 = 0, pqj2 = 0;
      float2 xf2 = make_float2(0.0f, 0.0f);
      float rf2 = 0.0f;
      if (q0 + 32 < total) load(q0 + 32 + lane, k2, rj2, xf2, rf2, idj2, pqj2);
      // four home vertices at a time: their tests are independent
      for (int h4 = 0; h4 < nh; h4 += 4) {
        int dec[4];  // 1 neighbour, 0 not, -1 exact test
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int h = min(h4 + u, nh - 1);
          const float2 xi = hs.x[h];
          const float dx = xf.x - xi.x, dy = xf.y - xi.y;
          const float sq = fmaf(dy, dy, dx * dx);
          const float t = (hs.r[h] + (n.self_rsum ? hs.r[h] : rf)) * pt.opc;
          const float t2 = t * t;
          const float m = fmaf(1e-5f, t2, fmaf(pt.e4, t, pt.ee4));
          const int d = !pt.on ? -1 : (sq < t2 - m ? 1 : (sq > t2 + m ? 0 : -1));
          dec[u] = (k >= 0 && h4 + u < nh && rj != hs.ring[h]) ? d : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int h = h4 + u;
          if (dec[u] < 0) {
            // inside the band: the reference expression on double positions
            const double rh = n.cell_rad[h0 + h];
            dec[u] = is_neighbor(p, n.cell_pos[h0 + h], n.cell_pos[k], rh + (n.self_rsum ? rh : n.cell_rad[k]),
                                 n.cut_distance) ? 1 : 0;
          }
          const bool hit = dec[u] == 1;
          const unsigned int m = __ballot_sync(kAll, hit);
          if (m) {
            const int base = __shfl_sync(kAll, cnt, h & 31);
            if (hit) {
              const int g = hs.id[h];
              const int slot = base + __popc(m & ((1u << lane) - 1u));
              if (slot < n.cap) {
                n.nbr[(size_t)slot * p.nv + g] = idj;
                if (n.nbr_pq) n.nbr_pq[(size_t)slot * p.nv + g] = pqj;
              }
            }
            if (lane == h) cnt += __popc(m);
          }
        }
      }
      k = k2;
      rj = rj2;
      xf = xf2;
      rf = rf2;
      idj = idj2;
      pqj = pqj2;
    }
    if (lane < nh) {
      n.nbr_cnt[gh] = cnt;
      n.last_pos[gh] = xh;
      maxc = max(maxc, cnt);
    }
  }
  return maxc;
}

// Bucket form of the stencil search.  The home cells are dealt to the CTAs
// in square tiles of T x T cells (T from the host: the smallest tile whose
// count fits the grid, up to kStageTileMax).  A CTA stages its tile's cells
// and their one-cell halo from the buckets into shared memory (cp.async,
// every bucket slot and the counts), then converts: ids, rings, packed
// offsets, radii in single precision and positions in single precision
// relative to the tile's corner, each shifted by the box lengths its staged
// cell was wrapped by (its minimum image whenever it lies within range of a
// home vertex).  Every staged row of cells becomes one list, cell after cell
// and ascending id inside a cell (bucket slots come in atomic order), so the
// three stencil cells of a home vertex on one row are one contiguous run in
// the sequential scan's order.  Three threads per home vertex, one per row
// (dy = row - 1), ten vertices per warp (lanes 30 and 31 idle): pass 1 tests
// the row's run with the single-precision pre-test of the sorted-cell search
// (PreTest, here over T + 2 cells) and, inside its rounding band, with the
// reference expression on the double positions (band_test), one bit per
// hit; the rows' hit counts give each row its first slot (row 0 first);
// pass 2 writes the hits in run order.  The list is the sorted-cell search's,
// entry for entry.  Returns the largest count among the vertices this thread
// completed.
constexpr int kStageTileMax = 12;
constexpr size_t kStageEntryBytes =
    sizeof(double2) + sizeof(double) + sizeof(float2) + sizeof(float) + 4 * sizeof(int);
__host__ __device__ constexpr size_t bucket_stage_bytes(int t) {
  return (size_t)(t + 2) * (t + 2) * kCellBucket * kStageEntryBytes + (size_t)(t + 2) * (t + 2) * sizeof(int) +
         (size_t)(t + 2) * (t + 3) * sizeof(int) + ((size_t)t * t + 1) * sizeof(int);
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// staged cell sl of a tile with corner (ox, oy): its grid cell and the
// number of box lengths it was wrapped by along x and y
template <int SW>
__device__ __forceinline__ int staged_cell(int sl, int ox, int oy, int ncx, int ncy, int& wx, int& wy) {
  const int ux = ox - 1 + sl % SW, uy = oy - 1 + sl / SW;  // unwrapped cell
  wx = ux < 0 ? -1 : (ux < ncx ? 0 : ux / ncx);
  wy = uy < 0 ? -1 : (uy < ncy ? 0 : uy / ncy);
  return (uy - wy * ncy) * ncx + (ux - wx * ncx);
}

// Inside the pre-test's rounding band: the reference expression on the
// double positions of home vertex v and candidate c.  Out of line, so the
// candidate loop branches over it instead of carrying it on every pass.
__device__ __noinline__ int band_test(const SysParams& p, const NbrArgs& n, int v, int c) {
  const double rv = n.rad[v];
  return is_neighbor(p, n.pos[v], n.pos[c], rv + (n.self_rsum ? rv : n.rad[c]), n.cut_distance) ? 1 : 0;
}

template <int T>
__device__ __forceinline__ int bucket_tiles(const SysParams& p, int ncx, int ncy, const NbrArgs& n, const int* cnt,
                                            unsigned char* smem) {
  constexpr unsigned kAll = 0xffffffffu;
  constexpr int SW = T + 2, S = SW * SW, E = S * kCellBucket, H = T * T, RL = SW * kCellBucket;
  double2* s_rpos = reinterpret_cast<double2*>(smem);  // bucket copies as stored
  double* s_rrad = reinterpret_cast<double*>(s_rpos + E);
  float2* s_xf = reinterpret_cast<float2*>(s_rrad + E);
  float* s_rf = reinterpret_cast<float*>(s_xf + E);
  int* s_ring = reinterpret_cast<int*>(s_rf + E);
  int* s_id = s_ring + E;
  int* s_pq = s_id + E;
  int* s_row = s_pq + E;     // [SW][RL]: staged entries of each row of cells, in scan order
  int* s_cnt = s_row + E;    // [S]
  int* s_roff = s_cnt + S;   // [SW][SW + 1]: first run position of each cell in its row
  int* s_pref = s_roff + SW * (SW + 1);  // [H + 1]: exclusive prefix of the home cells' counts
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row = lane % 3, grp = lane - row;  // lanes grp .. grp + 2 share a home vertex
  const int ntx = (ncx + T - 1) / T, nty = (ncy + T - 1) / T;
  const double cw = p.lx / ncx, ch = p.ly / ncy;
  // rounding of a staged coordinate (at most T + 2 cells from the corner)
  const float e = (float)((T + 2) * fmax(cw, ch) * 0x1p-22);
  const float e4 = 4.0f * e, ee4 = 4.0f * e * e;
  const float opc = (float)(1.0 + n.cut_distance);
  const bool pre_on = n.cut_distance > -0.5;
  int maxc = 0;
  for (int tile = blockIdx.x; tile < ntx * nty; tile += gridDim.x) {
    const int ox = (tile % ntx) * T, oy = (tile / ntx) * T;
    const int hxn = min(T, ncx - ox), hyn = min(T, ncy - oy);
    const double cox = ox * cw, coy = oy * ch;
    __syncthreads();  // the previous tile's readers are done with the stage
    // every bucket slot and count of the staged cells, copied asynchronously
    for (int i = threadIdx.x; i < E; i += kFusedBlock) {
      const int sl = i / kCellBucket, el = i % kCellBucket;
      int wx, wy;
      const int cell = staged_cell<SW>(sl, ox, oy, ncx, ncy, wx, wy);
      const size_t k = (size_t)cell * kCellBucket + el;
      if (el == 0) cp_async4(s_cnt + sl, cnt + cell);
      cp_async16(s_rpos + i, n.bucket_pos + k);
      cp_async8(s_rrad + i, n.bucket_rad + k);
      cp_async4(s_ring + i, n.bucket_ring + k);
      cp_async4(s_id + i, n.bucket + k);
      if (n.nbr_pq) cp_async4(s_pq + i, n.bucket_pq + k);
    }
    cp_async_wait_all();
    __syncthreads();
    if (warp < SW) {
      // run offsets of the cells of staged row `warp`
      const int c = lane < SW ? s_cnt[warp * SW + lane] : 0;
      int incl = c;
      for (int o = 1; o < 16; o <<= 1) {
        const int y = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < SW) s_roff[warp * (SW + 1) + lane] = incl - c;
      if (lane == SW - 1) s_roff[warp * (SW + 1) + SW] = incl;
    } else if (warp == 31) {
      // exclusive prefix of the home cells' counts, tile row-major (cells
      // past the grid's edge hold none); s_pref[H] = home vertices of the tile
      constexpr int per = (H + 31) / 32;
      const int hb = min(H, lane * per), he = min(H, hb + per);
      int loc = 0;
      for (int h = hb; h < he; h++)
        loc += (h % T < hxn && h / T < hyn) ? s_cnt[(h / T + 1) * SW + h % T + 1] : 0;
      int incl = loc;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += y;
      }
      int run = incl - loc;
      for (int h = hb; h < he; h++) {
        s_pref[h] = run;
        run += (h % T < hxn && h / T < hyn) ? s_cnt[(h / T + 1) * SW + h % T + 1] : 0;
      }
      if (lane == 31) s_pref[H] = incl;
    }
    __syncthreads();
    // single-precision positions relative to the tile's corner, in the
    // staged cell's image; each entry to its place in its row's run
    for (int i = threadIdx.x; i < E; i += kFusedBlock) {
      const int sl = i / kCellBucket, el = i % kCellBucket, c = s_cnt[sl];
      if (el < c) {
        int wx, wy;
        staged_cell<SW>(sl, ox, oy, ncx, ncy, wx, wy);
        const double2 x = s_rpos[i];
        const double xw = x.x - p.lx * floor(x.x * p.inv_lx) + wx * p.lx;
        const double yw = x.y - p.ly * floor(x.y * p.inv_ly) + wy * p.ly;
        s_xf[i] = make_float2((float)(xw - cox), (float)(yw - coy));
        s_rf[i] = (float)s_rrad[i];
        const int id = s_id[i];
        int r = 0;
        for (int k = 0; k < c; k++) r += s_id[sl * kCellBucket + k] < id ? 1 : 0;
        const int y = sl / SW, x_ = sl % SW;
        s_row[y * RL + s_roff[y * (SW + 1) + x_] + r] = i;
      }
    }
    __syncthreads();
    const int nhome = s_pref[H];
    for (int m0 = 0; m0 < nhome; m0 += 10 * (kFusedBlock / 32)) {
      const int m = m0 + warp * 10 + lane / 3;
      const bool live = lane < 30 && m < nhome;
      unsigned long long hit = 0ull;
      int hq = 0, rb = 0;  // home entry; first run position of the row's three cells
      if (live) {
        // home cell: the last h with s_pref[h] <= m; the home vertex is its
        // member of rank m - s_pref[h]
        int lo = 0, hi = H - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_pref[mid] <= m) lo = mid;
          else hi = mid - 1;
        }
        const int hx = lo % T, hy = lo / T;
        hq = s_row[(hy + 1) * RL + s_roff[(hy + 1) * (SW + 1) + hx + 1] + (m - s_pref[lo])];
        const int y = hy + row;
        rb = y * RL + s_roff[y * (SW + 1) + hx];
        const int re = y * RL + s_roff[y * (SW + 1) + hx + 3];
        const float2 xh = s_xf[hq];
        const float rh = s_rf[hq];
        const int ringh = s_ring[hq];
        for (int q = rb; q < re; q++) {
          const int c = s_row[q];
          const float2 xc = s_xf[c];
          const float ddx = xc.x - xh.x, ddy = xc.y - xh.y;
          const float sq = fmaf(ddy, ddy, ddx * ddx);
          const float t = (rh + (n.self_rsum ? rh : s_rf[c])) * opc;
          const float t2 = t * t;
          const float mg = fmaf(1e-5f, t2, fmaf(e4, t, ee4));
          int d = !pre_on ? -1 : (sq < t2 - mg ? 1 : (sq > t2 + mg ? 0 : -1));
          if (d < 0) d = band_test(p, n, s_id[hq], s_id[c]);
          if (d && s_ring[c] != ringh) hit |= 1ull << (q - rb);
        }
      }
      const int nh = __popcll(hit);
      const int h0 = __shfl_sync(kAll, nh, grp), h1 = __shfl_sync(kAll, nh, grp + 1),
                h2 = __shfl_sync(kAll, nh, grp + 2);
      if (live) {
        const int v = s_id[hq];
        int slot = row == 0 ? 0 : (row == 1 ? h0 : h0 + h1);
        for (unsigned long long r = hit; r; r &= r - 1ull) {
          const int c = s_row[rb + __ffsll((long long)r) - 1];
          if (slot < n.cap) {
            n.nbr[(size_t)slot * p.nv + v] = s_id[c];
            if (n.nbr_pq) n.nbr_pq[(size_t)slot * p.nv + v] = s_pq[c];
          }
          slot++;
        }
        if (row == 0) {
          const int tot = h0 + h1 + h2;
          n.nbr_cnt[v] = tot;
          n.last_pos[v] = n.pos[v];
          maxc = max(maxc, tot);
        }
      }
    }
  }
  return maxc;
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
  __shared__ HomeStage s_home[8];
  const int c = blockIdx.x * 8 + threadIdx.x / 32;  // home cell of this warp
  const int m =
      (c < ncx * ncy) ? stencil_cell(p, ncx, ncy, n, n.cell_vid, c, threadIdx.x & 31, s_home[threadIdx.x / 32]) : 0;
  const int bm = block_max(m);
  publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap);
}

__device__ __forceinline__ int brute_vertex(const SysParams& p, const NbrArgs& n, int i) {
  const double2 xi = n.pos[i];
  const double ri = n.rad[i];
  const int ring = n.ring_of[i];
  int cnt = 0;
  for (int j = 0; j < p.nv; j++) {
    if (n.ring_of[j] == ring) continue;
    if (is_neighbor(p, xi, n.pos[j], ri + (n.self_rsum ? ri : n.rad[j]), n.cut_distance)) {
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
    k_nbr_cells<<<(ncells + 7) / 8, 256, 0, stream>>>(p, g.ncx, g.ncy, n);
  } else {
    k_nbr_brute<<<nb, 256, 0, stream>>>(p, n);
  }
}

// ------------------------------------------------------- one-launch build
//
// The build in one launch, for step sequences captured in graphs: the kernel
// follows every op that may arm a rebuild and returns at once unless the op
// armed one, so a step that needs no rebuild pays one early-exit launch
// instead of a conditional graph node.  When armed:
//   1 cell + slot of every vertex (atomic count, as k_cell_count); with
//     buckets, the vertex and its data also go to its cell's bucket slot,
//     and the other count array is cleared for the next build
//   -- grid barrier --
//   2 every cell within its bucket: the tiled search on the buckets
//     (bucket_tiles), then publish.  Otherwise the sorted-cell form:
//   2' per-CTA totals of a contiguous cell range
//   3' exclusive scan: CTA offset from the totals, then the range (k_cell_scan)
//   4' scatter ids by cell                     (k_cell_fill)
//   5' per vertex: rank in its cell by id, copy to that entry
//                                              (k_cell_sort + k_cell_gather)
//   6' stencil search, one warp per home cell  (k_nbr_cells)
//     with grid barriers between them,
// and the last CTA publishes the build exactly as the multi-kernel path does,
// so every path produces the same list.  The grid never exceeds the CTAs the
// GPU holds at once (occupancy x SMs, nbr_fused_max_blocks), so every CTA is
// resident while the others wait.  Every wait is bounded: a barrier that does
// not complete within status.spin_limit polls (default 2^20, about a second)
// sets status.stalled and abort, and the CTAs return without finishing the
// build.


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
    const long long lim = barrier_poll_limit(st);
    long long it = 0;
    while (ld_acquire_u32(&st->bar_count) < target) {
      if (++it > lim || *(volatile int*)&st->stalled) {
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
    k_nbr_fused(const __grid_constant__ SysParams p, int ncx, int ncy, const __grid_constant__ NbrArgs n, int force,
                int stage_tile) {
  // the status block and positions come from the step kernel before this
  // launch; the next kernel starts when this one exits (no early trigger, so
  // no later grid can take the SMs that the grid barriers need)
  pdl_wait();
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
  __shared__ HomeStage s_home[kFusedBlock / 32];
  // bucket form: this build counts into the current count array and clears
  // the other one, which the next build counts into
  const bool dual = n.bucket != nullptr && n.cell_stride > 0;
  int* ctl = dual ? n.cell_cnt + 2 * (size_t)n.cell_stride : nullptr;
  const int sel = dual ? *(volatile int*)ctl : 0;
  int* cnt = n.cell_cnt + (size_t)sel * n.cell_stride;
  // 1: cells and slots (the current counts are zero between builds)
  if (gt == 0) {
    st->overflow = 0;
    st->max_count = 0;
  }
  bool full = false;
  // a contiguous range of vertices per CTA, so every CTA takes a share
  const int per_cta = (nv + gridDim.x - 1) / gridDim.x;
  const int vb = min(nv, (int)blockIdx.x * per_cta), ve = min(nv, vb + per_cta);
  for (int v = vb + threadIdx.x; v < ve; v += kFusedBlock) {
    const double2 x = n.pos[v];
    const int c = cell_coord(x.y, p.ly, p.inv_ly, ncy) * ncx + cell_coord(x.x, p.lx, p.inv_lx, ncx);
    n.cell_of[v] = c;
    const int s = atomicAdd(cnt + c, 1);
    n.slot[v] = s;
    if (dual) {
      if (s < kCellBucket) {
        const size_t k = (size_t)c * kCellBucket + s;
        n.bucket[k] = v;
        n.bucket_pos[k] = x;
        n.bucket_rad[k] = n.rad[v];
        n.bucket_ring[k] = n.ring_of[v];
        if (n.nbr_pq) n.bucket_pq[k] = n.pq_pack[v];
      } else {
        full = true;
      }
    }
  }
  if (dual) {
    if (full) atomicOr(ctl + 1, 1);
    int* other = n.cell_cnt + (size_t)(sel ^ 1) * n.cell_stride;
    for (int i = gt; i < n.cell_stride; i += nthreads) other[i] = 0;
  }
  if (!grid_barrier(st)) return;
  if (dual && *(volatile int*)(ctl + 1) == 0) {
    // 2 (every cell within its bucket): the search on the buckets
    extern __shared__ __align__(16) unsigned char s_stage[];
    int m = 0;
    switch (stage_tile) {
      case 4: m = bucket_tiles<4>(p, ncx, ncy, n, cnt, s_stage); break;
      case 6: m = bucket_tiles<6>(p, ncx, ncy, n, cnt, s_stage); break;
      case 8: m = bucket_tiles<8>(p, ncx, ncy, n, cnt, s_stage); break;
      case 9: m = bucket_tiles<9>(p, ncx, ncy, n, cnt, s_stage); break;
      case 10: m = bucket_tiles<10>(p, ncx, ncy, n, cnt, s_stage); break;
      default: m = bucket_tiles<kStageTileMax>(p, ncx, ncy, n, cnt, s_stage); break;
    }
    const int bm = block_max(m);
    publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap, ctl, true);
    return;
  }
  // 2 (a cell beyond its bucket, or no buckets): sort by cell.  This CTA's
  // cells [cb, ce), this thread's [tb, te)
  const int per_block = (ncells + gridDim.x - 1) / gridDim.x;
  const int cb = min(ncells, (int)blockIdx.x * per_block), ce = min(ncells, cb + per_block);
  const int per_thread = (ce - cb + kFusedBlock - 1) / kFusedBlock;
  const int tb = min(ce, cb + (int)threadIdx.x * per_thread), te = min(ce, tb + per_thread);
  int sum = 0;
  for (int c = tb; c < te; c++) sum += cnt[c];
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
    const int k = cnt[c];
    n.cell_start[c] = run;
    run += k;
    cnt[c] = 0;
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
  // 6: stencil search, one warp per home cell
  int m = 0;
  for (int c = gt / 32; c < ncells; c += nthreads / 32)
    m = max(m, stencil_cell(p, ncx, ncy, n, n.slot, c, gt & 31, s_home[threadIdx.x / 32]));
  const int bm = block_max(m);
  publish_build(n, threadIdx.x == 0 ? bm : 0, threadIdx.x == 0 && bm > n.cap, ctl, false);
}

int nbr_fused_max_blocks() {
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  const int smem = (int)bucket_stage_bytes(kStageTileMax);
  if (cudaFuncSetAttribute(k_nbr_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_nbr_fused, kFusedBlock, smem) != cudaSuccess) return 0;
  return occ * sms;
}

int nbr_fused_blocks(int nv, int max_blocks) {
  const long want = ((long)nv * 4 + kFusedBlock - 1) / kFusedBlock;
  return (int)std::max(1L, std::min<long>(want, max_blocks));
}

// Side of the bucket search's tiles: the smallest whose tiles number no more
// than the CTAs, else the largest the stage allows.
static int stage_tile(int ncx, int ncy, int blocks) {
  for (int t : {4, 6, 8, 9, 10})
    if ((long)((ncx + t - 1) / t) * ((ncy + t - 1) / t) <= blocks) return t;
  return kStageTileMax;
}

void launch_nbr_fused(cudaStream_t st, const SysParams& p, const CellGrid& g, const NbrArgs& n, int blocks,
                      int force, bool pdl) {
  const int t = stage_tile(g.ncx, g.ncy, blocks);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kFusedBlock);
  cfg.dynamicSmemBytes = (n.bucket && g.ncx >= 3 && g.ncy >= 3) ? bucket_stage_bytes(t) : 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_nbr_fused, p, g.ncx, g.ncy, n, force, t);
}

}  // namespace cr
