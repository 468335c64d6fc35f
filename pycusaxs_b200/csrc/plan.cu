// pycusaxs_b200: B200-native per-frame SAXS path.
//
// Pipeline of one batch of frames (all kernels hand-written for sm_100a):
//
//   k_sort_atoms    one thread-block cluster per (type, frame): atoms ->
//                   float32 grid coordinates (the reference's float steps,
//                   saxsDeviceKernels.cu:355-368), counting sort into
//                   (type, home tile) order with shared-memory counters shared
//                   across the cluster, per-type FP64 z-border sums for the
//                   padding mean (saxsDeviceKernels.cu:446-465 evaluated per
//                   atom instead of per voxel).
//   k_spread_zdft   one CTA per (frame, type, 8x8 column tile): B-spline
//                   spreading into a shared-memory column tile (no global
//                   atomics), mean padding folded in as "subtract the mean",
//                   then the z-axis DFT of every column restricted to the
//                   kz values the q-cut can reach.
//   k_ydft          y-axis DFT restricted to the ky range (complex GEMM-shaped
//                   tiles in shared memory, FP32 FMA).
//   k_xdft_post     x-axis DFT restricted to the kx range, then per k-point:
//                   form factor f_t(|q|), complex sum over types, |F|^2 times
//                   the B-spline moduli (saxsDeviceKernels.cu:142-216).
//   k_hist          mirror-weighted radial histogram with the reference's
//                   float32 bin rule (saxsDeviceKernels.cu:67-125), FP64
//                   shared-memory bins, one global flush per CTA.
//
// Why no full FFT: the reference zero-pads (mean-pads) the nx^3 grid into an
// nn^3 supercell and runs a full R2C FFT, but only k-points with |q| <= qcut
// ever reach the histogram, and qcut is clamped so that these form a small
// ellipsoid around the origin (|m| <= ~20 of 256 at 100k atoms / 256^3).  The
// padded transform is F = DFT(g - mean over the corner block) + mean*nn^3 at
// k = 0, evaluated exactly by three pruned DFT passes that never touch the
// zero region.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched at run time)
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pycusaxs_b200.h"
#include "scratch_forward.h"
#include "setup.h"

namespace {

constexpr int kTile = 8;                  // spread tile edge (columns per axis)
constexpr int kCols = kTile * kTile;      // columns per tile
constexpr int kThreads = 256;
constexpr int kGeom = 24;                 // floats of per-frame geometry: oc[9], ocs[9]
constexpr int kRing = 4;                  // pinned geometry slots in flight
constexpr int kKzThread = 6;              // kz outputs (complex) per thread in k_spread_zdft
constexpr int kKyGroup = 10;              // ky outputs per warp in k_ydft
constexpr int kKyPass = 8 * kKyGroup;     // ky outputs per pass (eight warps)
constexpr int kYChunk = 32;               // y values staged per step in k_ydft
constexpr int kYRows = 64;                // x rows per CTA in k_ydft
constexpr int kYStride = kYRows + 2;      // padded shared row (float2), 16-byte aligned
constexpr int kXRows = 4;                 // ky rows per CTA in k_xdft_post
constexpr int kHistSmemBins = 2048;       // bins held in shared memory by k_hist

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(x)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess)                                                            \
      return fail(SAXS_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));      \
  } while (0)

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Everything a kernel needs, passed by value.
struct DevArgs {
  int n[3], nn[3], ext[3];
  int order, ntaps;
  int T, M;
  int tiles[2], stiles[2], nbins;
  int bin_w;  // home-bin width (columns) of the atom counting sort: 4, or 8 when 4 would
              // need more than four bins per spread tile and axis
  int kx_lo, nkx, ky_lo, nky, nkz, nkzp, nkxp, nkyp;
  int zc;  // z rows of twiddles k_spread_zdft holds in shared memory at once
  // tensor-core z-DFT (k_spread_zdft_tc): GEMM N, K, spread rows, stages, TMEM columns
  int tcN, tcK, tcR, tcS, tcCols, tcRB, tcCap;
  int tcG;  // producer groups of k_spread_zdft_tc (1, or 2 with two operand stages)
  // wide-tile variant (k_spread_zdft_tcw): tile row stride (floats), record buffer,
  // atom table entries, producer groups; y tiles of 16 rows
  int twN, twRS, twRB, twCap, twG, stw;
  int xtcKyb;  // tensor-core x-axis DFT: ky values per item (rows (ky, type), T per ky)
  int nf[3];
  int dz;
  float dq, qcut;
  int num_bins;
  double border_count;
  double nn3;
  int64_t frame_stride;
  const float *xyz;
  const int32_t *entry_atom;
  const int32_t *entry_type;
  const int *type_start;  // [T + 1]: entries are grouped by type, type t owns [type_start[t], type_start[t+1])
  const float *geom;
  const float2 *twz;  // [ez][nkzp], nkzp a multiple of kKzThread
  const float2 *twy;  // [ey][nkyp]
  const float2 *twx;  // [ex][nkxp]
  const float *modx, *mody, *modz;
  const float *ff;    // [T][9]
  const float *twz_sum; // [2*nkzp]: sum over z < ez of the z twiddles (re, im)
  const float *twz_tc;  // [2][tcK x tcN]: z twiddles as TF32 head / remainder, K-major
  const float *twz_tcw; // [tcK x 2*twN] f16 (wide tiles): head and remainder side by side
  const int4 *home_x; // per spread tile along x: home tiles whose atoms reach it (-1 padded)
  const int4 *home_y;
  const int4 *home_yw; // per 16-row y tile: up to eight home tiles (two int4, -1 padded)
  int2 *key;
  int *offsets;
  float4 *rec;
  double *border;
  const float *pad_val;  // [T] given padding densities (atoms per grid point); null: z-border mean
  float2 *Z;
  float2 *Y;
  float *ibox;
  double *hist, *nhist;
  double *iacc;
  int *status;
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

// Grid coordinate r = n * frac(oc_row . x), written as the reference writes it
// (saxsDeviceKernels.cu:355-361) so that nvcc evaluates it the same way.
__device__ __forceinline__ float grid_coord(const float *oc, float x0, float y0, float z0, int n) {
  float x1 = oc[0] * x0 + oc[1] * y0 + oc[2] * z0;
  return static_cast<float>(n * (x1 - rint(x1 - 0.5)));
}

// |q| of the k-point with signed indices (ia, ja, ka), in the reference's
// float32 form (saxsDeviceKernels.cu:85-92): the dot products in float, the
// 2*pi factor applied in double, then sqrtf of the sum of squares.
__device__ __forceinline__ float kpoint_q(const float *oc, int ia, int ja, int ka) {
  float mw1, mw2, mw3, mw;
  mw1 = oc[0] * ia + oc[1] * ja + oc[2] * ka;
  mw1 = 2.0 * M_PI * mw1;
  mw2 = oc[3] * ia + oc[4] * ja + oc[5] * ka;
  mw2 = 2.0 * M_PI * mw2;
  mw3 = oc[6] * ia + oc[7] * ja + oc[8] * ka;
  mw3 = 2.0 * M_PI * mw3;
  mw = sqrtf(mw1 * mw1 + mw2 * mw2 + mw3 * mw3);
  return mw;
}

// Cubic (order-4) cardinal B-spline weights of the four taps at fractional
// offset u in [0, 1]: tap 0 is the farthest-left grid point.
__device__ __forceinline__ void cubic_weights(float u, float w[4]) {
  const float v = 1.0f - u;
  const float u2 = u * u, u3 = u2 * u;
  const float s = 1.0f / 6.0f;
  w[0] = v * v * v * s;
  w[1] = (3.0f * u3 - 6.0f * u2 + 4.0f) * s;
  w[2] = (-3.0f * u3 + 3.0f * u2 + 3.0f * u + 1.0f) * s;
  w[3] = u3 * s;
}

// Form factor sum_i a_i exp(-b_i s2) + c at s2 = (q/4pi)^2 (opsfact.cu:30-35).
__device__ __forceinline__ float form_factor(const float *c, float q2) {
  return c[0] * expf(-c[4] * q2) + c[1] * expf(-c[5] * q2) + c[2] * expf(-c[6] * q2) +
         c[3] * expf(-c[7] * q2) + c[8];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int signed_k(int k, int nn, int nf) { return k < nf ? k : k - nn; }

// Padding density of type t in frame f: the plan's given value, or the mean of
// the type's z-border planes (saxsKernel.cu:150-162).
__device__ __forceinline__ float padding_mean(const DevArgs &a, int f, int t) {
  return a.pad_val ? a.pad_val[t]
                   : static_cast<float>(a.border[static_cast<int64_t>(f) * a.T + t] / a.border_count);
}

// Programmatic dependent launch: the forward's kernels after the first are
// launched with programmatic stream serialization, so a kernel's grid may start
// while the previous one drains.  Each such kernel lets its own successor launch
// at once (every CTA is then resident, so the successor cannot starve it of
// SMs) and waits for its predecessor's completion and memory before it reads
// anything the predecessor wrote; only set-up that touches plan constants,
// shared and tensor memory runs before the wait.  Both are no-ops for kernels
// launched without the attribute.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Thread-block cluster helpers (PTX ISA: %cluster_ctarank, mapa,
// ld/st.shared::cluster, barrier.cluster).  A kernel launched without a
// cluster dimension is a cluster of one CTA.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_ctas() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
// shared::cluster address of `p` (this CTA's shared memory) in CTA `rank`
__device__ __forceinline__ uint32_t cluster_map(const void *p, uint32_t rank) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(a), "r"(rank));
  return out;
}
__device__ __forceinline__ int cluster_ld(uint32_t addr) {
  int v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void cluster_st(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}

// grid (T * C, frames), cluster (C, 1, 1), block kSortThreads: counting sort of
// one type's atoms of one frame by home bin, shared among the C CTAs of a
// cluster (C = 1..kSortMaxCluster, chosen per launch so that the largest type
// does not hold one SM while the others idle).  CTA r of the cluster takes the
// r-th contiguous slice of the type's entries:
//   pass 1   grid coordinates, home bin, rank within the CTA's bin counter
//            (shared-memory atomics), the slice's z-border share;
//   prefix   per bin, the counts of all C CTAs read through distributed shared
//            memory: the bin's total (scanned over the type's bins: its records
//            start at type_start[t], fixed by the grouping of the entries) and
//            the counts of the CTAs before r, so that the slices' records follow
//            each other inside a bin;
//   pass 2   records (rx, ry, rz, entry) written in bin order.
// CTA 0 writes the offsets (per global bin t * bins_t + local bin, and the total
// at offsets[nbins]) and the type's border sum, added in CTA order.  No global
// atomics and no separate scan or scatter launch.
// Dynamic shared memory: 2 * bins_t ints.
//
// Geometry: with `in_params`, frame f0 + j's kGeom floats arrive as kernel
// parameters (gp.g[j]) and CTA 0 of type 0 stores them to a.geom for the later
// kernels, so that no host-to-device copy of them queues behind other transfers
// on the copy engines; otherwise a.geom already holds them.
constexpr int kSortThreads = 512, kSortU = 4, kSortMaxCluster = 8, kSortParamFrames = 128;
struct SortGeom {
  float g[kSortParamFrames * kGeom];
};
__global__ void __launch_bounds__(kSortThreads, 2)
    k_sort_atoms(DevArgs a, const __grid_constant__ SortGeom gp, int in_params, int f0) {
  pdl_release();
  extern __shared__ int scnt[];  // [bins_t] counts of this CTA, then [bins_t] bases
  __shared__ double wsum[kSortThreads / 32];
  __shared__ double csum[kSortMaxCluster];
  __shared__ int wscan[kSortThreads / 32];
  __shared__ float oc[9];
  const int C = static_cast<int>(cluster_ctas()), r = static_cast<int>(cluster_rank());
  const int t = blockIdx.x / C, f = f0 + blockIdx.y;
  const int nb = a.tiles[0] * a.tiles[1];
  int *sbase = scnt + nb;
  const int e0 = a.type_start[t], e1 = a.type_start[t + 1];
  const int s0e = e0 + static_cast<int>(static_cast<int64_t>(e1 - e0) * r / C);
  const int s1e = e0 + static_cast<int>(static_cast<int64_t>(e1 - e0) * (r + 1) / C);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int b = tid; b < nb; b += kSortThreads) scnt[b] = 0;
  pdl_wait();
  if (in_params) {
    if (tid < 9) oc[tid] = gp.g[blockIdx.y * kGeom + tid];
    if (t == 0 && r == 0 && tid < kGeom) const_cast<float *>(a.geom)[f * kGeom + tid] = gp.g[blockIdx.y * kGeom + tid];
  } else if (tid < 9) {
    oc[tid] = a.geom[f * kGeom + tid];
  }
  __syncthreads();
  const float *xyz = a.xyz + f * a.frame_stride;
  int2 *key = a.key + static_cast<int64_t>(f) * a.M;
  const int bsh = __ffs(a.bin_w) - 1;  // bins are 4 or 8 columns wide
  double contrib = 0.0;
  // kSortU entries per thread per round, their loads issued before any of their
  // arithmetic so that the position gathers overlap
  for (int eb = s0e + tid; eb < s1e; eb += kSortU * kSortThreads) {
    int at[kSortU];
    float px[kSortU][3];
#pragma unroll
    for (int u = 0; u < kSortU; ++u) {
      const int e = eb + u * kSortThreads;
      at[u] = e < s1e ? a.entry_atom[e] : -1;
    }
#pragma unroll
    for (int u = 0; u < kSortU; ++u)
      if (at[u] >= 0) {
        const float *p = xyz + 3ll * at[u];
        px[u][0] = p[0];
        px[u][1] = p[1];
        px[u][2] = p[2];
      }
#pragma unroll
    for (int u = 0; u < kSortU; ++u) {
      if (at[u] < 0) continue;
      float rr[3];
      int m[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        rr[d] = grid_coord(oc + 3 * d, px[u][0], px[u][1], px[u][2], a.n[d]);
        m[d] = static_cast<int>(rr[d]);
      }
      int xf = m[0] - a.order;
      if (xf < 0) xf += a.n[0];
      int yf = m[1] - a.order;
      if (yf < 0) yf += a.n[1];
      const int bin = (yf >> bsh) * a.tiles[0] + (xf >> bsh);
      key[eb + u * kSortThreads] = make_int2(bin, atomicAdd(&scnt[bin], 1));
      // the atom's share of its type's z-border planes: (sum of x weights) *
      // (sum of y weights) * (sum of z weights on border planes)
      float wx[4], wy[4], wz[4];
      cubic_weights(rr[0] - static_cast<float>(m[0]), wx);
      cubic_weights(rr[1] - static_cast<float>(m[1]), wy);
      cubic_weights(rr[2] - static_cast<float>(m[2]), wz);
      float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (o < a.ntaps) {
          sx += wx[o];
          sy += wy[o];
          int z = m[2] - a.order + o;
          if (z < 0) z += a.n[2];
          if (z <= a.dz || z >= a.n[2] - a.dz) sz += wz[o];
        }
      }
      contrib += static_cast<double>(sx) * static_cast<double>(sy) * static_cast<double>(sz);
    }
  }
  contrib = warp_sum(contrib);
  if (lane == 0) wsum[warp] = contrib;
  __syncthreads();
  if (warp == 0) {
    double b = lane < kSortThreads / 32 ? wsum[lane] : 0.0;
    b = warp_sum(b);
    if (lane == 0) cluster_st(cluster_map(&csum[r], 0), b);
  }
  // every CTA's counts final and its border share in CTA 0
  cluster_arrive();
  cluster_wait();
  uint32_t rcnt[kSortMaxCluster];
#pragma unroll
  for (int c = 0; c < kSortMaxCluster; ++c) rcnt[c] = c < C ? cluster_map(scnt, c) : 0u;
  // exclusive scan of the bins' totals: a contiguous segment per thread
  const int per = (nb + kSortThreads - 1) / kSortThreads, b0 = tid * per;
  int local = 0;
  for (int i = 0; i < per; ++i) {
    const int b = b0 + i;
    if (b < nb) {
#pragma unroll
      for (int c = 0; c < kSortMaxCluster; ++c)
        if (c < C) local += cluster_ld(rcnt[c] + 4u * b);
    }
  }
  int inc = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += v;
  }
  if (lane == 31) wscan[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kSortThreads / 32 ? wscan[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += v;
    }
    if (lane < kSortThreads / 32) wscan[lane] = w;
    if (r == 0) {
      double b = lane < C ? csum[lane] : 0.0;
      // CTA order, so that the sum does not depend on scheduling
#pragma unroll
      for (int c = 1; c < kSortMaxCluster; ++c) {
        const double v = __shfl_sync(0xffffffffu, b, c);
        if (lane == 0 && c < C) b += v;
      }
      if (lane == 0) a.border[static_cast<int64_t>(f) * a.T + t] = b;
    }
  }
  __syncthreads();
  int run = (warp > 0 ? wscan[warp - 1] : 0) + inc - local;
  int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1) + static_cast<int64_t>(t) * nb;
  for (int i = 0; i < per; ++i) {
    const int b = b0 + i;
    if (b < nb) {
      int tot = 0, before = 0;
#pragma unroll
      for (int c = 0; c < kSortMaxCluster; ++c)
        if (c < C) {
          const int v = cluster_ld(rcnt[c] + 4u * b);
          tot += v;
          if (c < r) before += v;
        }
      sbase[b] = e0 + run + before;
      if (r == 0) off[b] = e0 + run;
      run += tot;
    }
  }
  if (t == a.T - 1 && r == 0 && tid == 0) a.offsets[static_cast<int64_t>(f) * (a.nbins + 1) + a.nbins] = e1;
  // the other CTAs' reads of this CTA's counts end before its exit (wait below)
  cluster_arrive();
  __syncthreads();
  float4 *rec = a.rec + static_cast<int64_t>(f) * a.M;
  for (int eb = s0e + tid; eb < s1e; eb += kSortU * kSortThreads) {
    int at[kSortU];
    int2 k[kSortU];
    float px[kSortU][3];
#pragma unroll
    for (int u = 0; u < kSortU; ++u) {
      const int e = eb + u * kSortThreads;
      at[u] = -1;
      if (e < s1e) {
        at[u] = a.entry_atom[e];
        k[u] = key[e];
      }
    }
#pragma unroll
    for (int u = 0; u < kSortU; ++u)
      if (at[u] >= 0) {
        const float *p = xyz + 3ll * at[u];
        px[u][0] = p[0];
        px[u][1] = p[1];
        px[u][2] = p[2];
      }
#pragma unroll
    for (int u = 0; u < kSortU; ++u)
      if (at[u] >= 0)
        rec[sbase[k[u].x] + k[u].y] = make_float4(grid_coord(oc + 0, px[u][0], px[u][1], px[u][2], a.n[0]),
                                                  grid_coord(oc + 3, px[u][0], px[u][1], px[u][2], a.n[1]),
                                                  grid_coord(oc + 6, px[u][0], px[u][1], px[u][2], a.n[2]),
                                                  __int_as_float(eb + u * kSortThreads));
  }
  cluster_wait();
}

// The atoms of up to 16 home bins of one tile, as one flat range: bin j holds
// records [start[j], start[j] + cum[j+1] - cum[j]).  Filled by threads 0..15.
struct TileAtoms {
  int start[16];
  int cum[17];
  int nb;
};

__device__ __forceinline__ void tile_atom_ranges(const DevArgs &a, TileAtoms &ta, int f, int t,
                                                 int x0, int y0) {
  if (threadIdx.x == 0) {
    const int4 hxv = a.home_x[x0 / kTile], hyv = a.home_y[y0 / kTile];
    const int hx[4] = {hxv.x, hxv.y, hxv.z, hxv.w}, hy[4] = {hyv.x, hyv.y, hyv.z, hyv.w};
    const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
    int nb = 0;
    ta.cum[0] = 0;
    for (int ix = 0; ix < 4; ++ix) {
      for (int iy = 0; iy < 4; ++iy) {
        if (hx[ix] >= 0 && hy[iy] >= 0) {
          const int bin = (t * a.tiles[1] + hy[iy]) * a.tiles[0] + hx[ix];
          const int s0 = off[bin];
          ta.start[nb] = s0;
          ta.cum[nb + 1] = ta.cum[nb] + (off[bin + 1] - s0);
          ++nb;
        }
      }
    }
    ta.nb = nb;
  }
}

// Spreading of one column tile into shared memory (float atomics on the tile).
__device__ __forceinline__ void spread_tile(const DevArgs &a, const TileAtoms &ta, float *tile,
                                            int f, int x0, int y0, int cw, int ch) {
  const float4 *rec = a.rec + static_cast<int64_t>(f) * a.M;
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  const int total = ta.cum[ta.nb];
  {
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
      int j = 0;
      while (k >= ta.cum[j + 1]) ++j;
      const int i = ta.start[j] + (k - ta.cum[j]);
        const float4 q = rec[i];
        const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y),
                  m2 = static_cast<int>(q.z);
        float wx[4], wy[4], wz[4];
        cubic_weights(q.x - static_cast<float>(m0), wx);
        cubic_weights(q.y - static_cast<float>(m1), wy);
        cubic_weights(q.z - static_cast<float>(m2), wz);
        int zs[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          int z = m2 - P + o;
          if (z < 0) z += nz;
          zs[o] = z * kCols;
        }
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          if (o >= nt) break;
          int x = m0 - P + o;
          if (x < 0) x += a.n[0];
          const int lx = x - x0;
          if (static_cast<unsigned>(lx) >= static_cast<unsigned>(cw)) continue;
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            if (p >= nt) break;
            int y = m1 - P + p;
            if (y < 0) y += a.n[1];
            const int ly = y - y0;
            if (static_cast<unsigned>(ly) >= static_cast<unsigned>(ch)) continue;
            const float wxy = wx[o] * wy[p];
            float *col = tile + lx * kTile + ly;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              if (r >= nt) break;
              atomicAdd(col + zs[r], wxy * wz[r]);
            }
          }
        }
      }
    }
}

// Persistent: grid = min(work items, resident CTAs); block 256.  A work item is
// one (frame, type, 8x8 column tile).  Dynamic shared memory:
//   twiddles  ez x NP floats   (NP = 2*nkzq; row z holds exp(-2 pi i kz z/nnz) as re,im)
//   tile      max(nz*64, 64*NP) floats (z-major: 64 columns contiguous per z)
// The z-axis DFT of the 64 columns is a small GEMM  out[c][n] = sum_z g[z][c] tw[z][n]
// done with 4 columns x 6 kz (12 floats) per thread and the z range split
// `ks` ways across the block, reduced deterministically in shared memory.
__global__ void __launch_bounds__(kThreads, 2) k_spread_zdft(DevArgs a, int items) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int nz = a.n[2], ez = a.ext[2];
  const int NP = 2 * a.nkzp;
  float *tws = reinterpret_cast<float *>(smem);
  float *tile = tws + static_cast<size_t>(a.zc) * NP;
  const int tid = threadIdx.x;
  const bool all_rows = a.zc >= ez;
  if (all_rows) {
    const float4 *src = reinterpret_cast<const float4 *>(a.twz);
    float4 *dst = reinterpret_cast<float4 *>(tws);
    const int n4 = ez * NP / 4;
    for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
  }
  const int ngroups = a.nkzp / kKzThread;      // kz groups of kKzThread
  const int tps = (kCols / 4) * ngroups;       // tasks per z split
  // Small k-boxes: every task runs once and the z range is split `ks` ways.
  // Large k-boxes (tps > block): ks = 1 and the block walks the tasks in rounds.
  const int ks = max(1, min(8, static_cast<int>(blockDim.x) / tps));
  const int rounds = (tps + blockDim.x - 1) / blockDim.x;
  const int split = rounds > 1 ? 0 : tid / tps;
  const int st = a.stiles[0] * a.stiles[1];
  const int ex = a.ext[0], ey = a.ext[1];
  const int64_t zplane = static_cast<int64_t>(ex) * ey;
  const int tile_floats = max(nz * kCols, kCols * NP);

  __shared__ TileAtoms ta;
  for (int w = blockIdx.x; w < items; w += gridDim.x) {
    const int f = w / (a.T * st);
    const int t = (w / st) % a.T;
    const int tl = w % st;
    const int x0 = (tl % a.stiles[0]) * kTile, y0 = (tl / a.stiles[0]) * kTile;
    const int cw = min(kTile, ex - x0), ch = min(kTile, ey - y0);
    {
      float4 *t4 = reinterpret_cast<float4 *>(tile);
      for (int i = tid; i < tile_floats / 4; i += blockDim.x) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    tile_atom_ranges(a, ta, f, t, x0, y0);
    __syncthreads();
    spread_tile(a, ta, tile, f, x0, y0, cw, ch);
    __syncthreads();
    // mean padding: the supercell is g on the corner block and the border mean
    // elsewhere = (g - mean) on the corner + a constant whose transform is k = 0
    // only.  The column DFT of -mean over z < ez is -mean * sum_z tw[z][n].
    const float mean = padding_mean(a, f, t);
    float2 *Zft = a.Z + (static_cast<int64_t>(f) * a.T + t) * a.nkz * zplane;
    for (int rd = 0; rd < rounds; ++rd) {
      const int task = rounds > 1 ? rd * blockDim.x + tid : tid % tps;
      const bool worker = rounds > 1 ? task < tps : split < ks;
      const int cg = task % (kCols / 4), kg = task / (kCols / 4);
      float acc[4][2 * kKzThread];
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int n = 0; n < 2 * kKzThread; ++n) acc[c][n] = 0.f;
      for (int z0 = 0; z0 < ez; z0 += a.zc) {
        const int zn = min(a.zc, ez - z0);
        if (!all_rows) {
          __syncthreads();
          const float4 *src = reinterpret_cast<const float4 *>(a.twz) + static_cast<size_t>(z0) * NP / 4;
          float4 *dst = reinterpret_cast<float4 *>(tws);
          const int n4 = zn * NP / 4;
          for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
          __syncthreads();
        }
        if (worker) {
          const float4 *g4 = reinterpret_cast<const float4 *>(tile) + cg;
          const float *twr = tws + kg * 2 * kKzThread;
          const int zlo = z0 + split * zn / ks, zhi = z0 + (split + 1) * zn / ks;
          for (int z = zlo; z < zhi; ++z) {
            const float4 g = g4[z * (kCols / 4)];
            const float4 *w4 = reinterpret_cast<const float4 *>(twr + (z - z0) * NP);
            const float4 w0 = w4[0], w1 = w4[1], w2 = w4[2];
            const float wv[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
            const float gv[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
              for (int n = 0; n < 12; ++n) acc[c][n] = fmaf(gv[c], wv[n], acc[c][n]);
          }
        }
      }
      if (worker && split == 0) {
#pragma unroll
        for (int n = 0; n < 2 * kKzThread; ++n) {
          const float d = a.twz_sum[kg * 2 * kKzThread + n];
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[c][n] = fmaf(-mean, d, acc[c][n]);
        }
      }
      if (rounds > 1) {
        // the tile is still read by later rounds: results go straight to Z
        if (worker) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int col = 4 * cg + c, lx = col / kTile, ly = col % kTile;
            if (lx >= cw || ly >= ch) continue;
#pragma unroll
            for (int j = 0; j < kKzThread; ++j) {
              const int kz = kg * kKzThread + j;
              if (kz < a.nkz)
                Zft[kz * zplane + static_cast<int64_t>(x0 + lx) * ey + (y0 + ly)] =
                    make_float2(acc[c][2 * j], acc[c][2 * j + 1]);
            }
          }
        }
        continue;
      }
      __syncthreads();  // tile contents are dead: reuse the region as out[NP][64]
      float *out = tile;
      for (int r = 0; r < ks; ++r) {
        if (worker && split == r) {
#pragma unroll
          for (int n = 0; n < 2 * kKzThread; ++n) {
            float4 *o = reinterpret_cast<float4 *>(out + (kg * 2 * kKzThread + n) * kCols) + cg;
            float4 v = make_float4(acc[0][n], acc[1][n], acc[2][n], acc[3][n]);
            if (r > 0) {
              const float4 u = *o;
              v.x += u.x;
              v.y += u.y;
              v.z += u.z;
              v.w += u.w;
            }
            *o = v;
          }
        }
        __syncthreads();
      }
      for (int i = tid; i < a.nkz * kCols; i += blockDim.x) {
        const int kz = i / kCols, col = i % kCols;
        const int lx = col / kTile, ly = col % kTile;
        if (lx < cw && ly < ch) {
          const float2 v = make_float2(out[(2 * kz) * kCols + col], out[(2 * kz + 1) * kCols + col]);
          Zft[kz * zplane + static_cast<int64_t>(x0 + lx) * ey + (y0 + ly)] = v;
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tensor-core z-axis DFT (tcgen05, 3xTF32)
// ---------------------------------------------------------------------------
//
// The column DFT of one 8x8 column tile is the GEMM D[c][n] = sum_z g[z][c] B[z][n]
// with M = 64 columns, N = 2*nkz (re, im interleaved, padded to a multiple of 8)
// and K = the z extent.  Both operands sit in shared memory in the K-major
// no-swizzle canonical layout of tcgen05 (core matrices of 8 rows x 16 bytes):
//   A (64 x K):  float offset (z/4)*256 + (c/8)*32 + (c%8)*4 + z%4
//                 (LBO = 1024 B between z quads, SBO = 128 B between 8-column groups)
//   B (N x K):   float offset (z/4)*(N/8)*32 + (n/8)*32 + (n%8)*4 + z%4
//                 (LBO = N*16 B, SBO = 128 B)
// Column c of the tile is (lx, ly) = (c/8, c%8).  FP32 accuracy comes from
// splitting each operand into a TF32 head (low 13 mantissa bits cleared) and the
// exact FP32 remainder: A*B ~ Ah*Bh + Ah*Bl + Al*Bh, accumulated in FP32 in
// tensor memory.  The dropped Al*Bl term and the TF32 rounding of the remainders
// are below 2^-19 of each product.
constexpr int kTcProducerWarps = 24;
constexpr int kTcProducers = 32 * kTcProducerWarps;
constexpr int kTcMmaWarp = kTcProducerWarps;
constexpr int kTcLoaderWarp = kTcProducerWarps + 1;
constexpr int kTcThreads = 32 * (kTcProducerWarps + 6);  // producers, MMA, loader, 4 epilogue warps

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, leading/stride byte offsets (>> 4),
// descriptor version 1 at bit 46, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (static_cast<uint64_t>(1) << 46);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The same with A read from tensor memory (row m of A in lane m, K along columns).
__device__ __forceinline__ void umma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The same with kind::f16 (f16 A and B, FP32 D, K = 16): A in tensor memory
// holds two K-consecutive halves per 32-bit column, the even one in the low half.
__device__ __forceinline__ void umma_f16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the given phase parity of an mbarrier: each try suspends the
// thread until the phase completes or 0.1 ms pass (so waiting warps do not take
// issue slots from working ones); gives up after 2^16 tries or 2 s, whichever
// comes first, and returns false.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity), "r"(100000)
      : "memory");
  return done != 0;
}

// Bounded wait: at most 2^16 + 1 tries and 2 s.  The global timer is read only
// once the first try has failed (a read of it costs hundreds of cycles, and most
// waits in the pipelines below find their phase already complete).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (int it = 0; it < (1 << 16); ++it) {
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

__device__ __forceinline__ float tf32_head(float v) {
  return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
}

// Shared-memory bytes per entry of the spreading pre-pass atom table (the plan
// sizes the table, DevArgs::tcCap entries).
constexpr int kTcAtomBytes = 3 * 16 + 16 + 2 * 4;  // wx, wy, wz (float4), z offsets (int4), lx, ly

// What the loader publishes with an item's records: the home-bin record ranges,
// the item's frame, type and tile, and its padding mean.
struct TcSlot {
  TileAtoms ta;
  int f, t, x0, y0, cw, ch;
  float mean;
};

// Grid-stride walk over work items w = ((f*T + t)*sy + ty)*sx + tx without
// divisions after the first item: each step adds the grid size digit by digit.
struct ItemIter {
  int tx, ty, t, f;
  int dtx, dty, dt, df;
  int sx, sy, T;
  __device__ __forceinline__ void init(const DevArgs &a, int w0, int g) {
    init_dims(w0, g, a.stiles[0], a.stiles[1], a.T);
  }
  __device__ __forceinline__ void init_dims(int w0, int g, int sx_, int sy_, int T_) {
    sx = sx_;
    sy = sy_;
    T = T_;
    const int st = sx * sy;
    tx = (w0 % st) % sx;
    ty = (w0 % st) / sx;
    t = (w0 / st) % T;
    f = (w0 / st) / T;
    dtx = (g % st) % sx;
    dty = (g % st) / sx;
    dt = (g / st) % T;
    df = (g / st) / T;
  }
  __device__ __forceinline__ void next() {
    tx += dtx;
    int c = tx >= sx;
    if (c) tx -= sx;
    ty += dty + c;
    c = ty >= sy;
    if (c) ty -= sy;
    t += dt + c;
    c = t >= T;
    if (c) t -= T;
    f += df + c;
  }
};

// Loader, first half: lane 4*iy + ix of the calling warp loads the record range
// of home bin (hx[ix], hy[iy]) (bins adjacent in x are adjacent in memory).
__device__ __forceinline__ void home_ranges_load(const DevArgs &a, const int4 *home_x,
                                                 const int4 *home_y, int f, int t, int x0, int y0,
                                                 int &s0, int &cnt, bool &valid) {
  const int lane = threadIdx.x & 31;
  const int4 hxv = home_x[x0 / kTile], hyv = home_y[y0 / kTile];
  const int iy = (lane >> 2) & 3, ix = lane & 3;
  const int hx = ix == 0 ? hxv.x : ix == 1 ? hxv.y : ix == 2 ? hxv.z : hxv.w;
  const int hy = iy == 0 ? hyv.x : iy == 1 ? hyv.y : iy == 2 ? hyv.z : hyv.w;
  valid = lane < 16 && hx >= 0 && hy >= 0;
  s0 = 0;
  cnt = 0;
  if (valid) {
    const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
    const int bin = (t * a.tiles[1] + hy) * a.tiles[0] + hx;
    s0 = off[bin];
    cnt = off[bin + 1] - s0;
  }
}

// Loader, second half: compaction and prefix sum of the ranges into `ta`.
__device__ __forceinline__ void home_ranges_publish(TileAtoms &ta, int s0, int cnt, bool valid) {
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, valid);
  const int pos = __popc(bal & ((1u << lane) - 1u));
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += v;
  }
  if (valid) {
    ta.start[pos] = s0;
    ta.cum[pos + 1] = inc;
  }
  if (lane == 0) {
    ta.cum[0] = 0;
    ta.nb = __popc(bal);
  }
}

// Shared-memory atom table of the spreading pre-pass (struct of arrays).
struct AtomTab {
  float4 *wx, *wy, *wz;  // B-spline weights of the four taps per axis
  int4 *zo;              // A-tile offsets (z/4)*256 + z%4 of the four z taps
  int *lx, *ly;          // tile column of each x / y tap, one byte each, 0xFF outside
};

// Atom table of the wide kernel: x weights pre-multiplied by the item's
// fixed-point scale, and the four x taps' tile offsets (lx * 16 * row stride,
// -1 outside) precomputed, so that a tap costs no byte extraction or multiply.
struct AtomTabW {
  float4 *wxs, *wy, *wz;  // scale * x weights, y and z weights
  int4 *zo;               // z row of each z tap
  int4 *xo;               // tile offset of each x tap's column, -1 outside
  int *ly;                // tile row (16 * lx + ly) y part of each y tap, one byte each, 0xFF outside
};
constexpr int kTwAtomBytes = 5 * 16 + 4;

// Spreading pre-pass: atom v0 + i (i < nv) -> weights, z offsets and in-tile tap
// columns.  Records [0, nrec_smem) come from the staged copy, the rest from
// global memory.
__device__ __forceinline__ void spread_prepass(const DevArgs &a, const TileAtoms &ta,
                                               const float4 *srec, int nrec_smem, int f, int v0,
                                               int nv, const AtomTab &tab, int x0, int y0, int cw,
                                               int ch, int tid, int nthreads) {
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  for (int i = tid; i < nv; i += nthreads) {
    const int v = v0 + i;
    float4 q;
    if (v < nrec_smem) {
      q = srec[v];
    } else {
      int j = 0;
      while (v >= ta.cum[j + 1]) ++j;
      q = a.rec[static_cast<int64_t>(f) * a.M + ta.start[j] + (v - ta.cum[j])];
    }
    const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y), m2 = static_cast<int>(q.z);
    float wx[4], wy[4], wz[4];
    cubic_weights(q.x - static_cast<float>(m0), wx);
    cubic_weights(q.y - static_cast<float>(m1), wy);
    cubic_weights(q.z - static_cast<float>(m2), wz);
    int lxp = 0, lyp = 0, zo[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      int bx = 0xFF, by = 0xFF, zz = 0;
      if (o < nt) {
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw)) bx = x - x0;
        int y = m1 - P + o;
        if (y < 0) y += a.n[1];
        if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch)) by = y - y0;
        int z = m2 - P + o;
        if (z < 0) z += nz;
        zz = (z >> 2) * 256 + (z & 3);
      }
      lxp |= bx << (8 * o);
      lyp |= by << (8 * o);
      zo[o] = zz;
    }
    tab.wx[i] = make_float4(wx[0], wx[1], wx[2], wx[3]);
    tab.wy[i] = make_float4(wy[0], wy[1], wy[2], wy[3]);
    tab.wz[i] = make_float4(wz[0], wz[1], wz[2], wz[3]);
    tab.zo[i] = make_int4(zo[0], zo[1], zo[2], zo[3]);
    tab.lx[i] = lxp;
    tab.ly[i] = lyp;
  }
}

// Spreading taps: one lane per (atom, y tap, z tap), four x taps each.  The 16
// lanes of an atom write 16 different banks (bank = 4*ly + z%4).
__device__ __forceinline__ void spread_taps(const AtomTab &tab, int nv, int nt, float *A, int tid,
                                            int nthreads) {
  for (int u = tid; u < nv * 16; u += nthreads) {
    const int i = u >> 4, p = (u >> 2) & 3, r = u & 3;
    if (p >= nt || r >= nt) continue;
    const int ly = (tab.ly[i] >> (8 * p)) & 0xFF;
    const int lxp = tab.lx[i];
    if (ly == 0xFF || lxp == -1) continue;
    const float wy = reinterpret_cast<const float *>(&tab.wy[i])[p];
    const float wz = reinterpret_cast<const float *>(&tab.wz[i])[r];
    const int zo = reinterpret_cast<const int *>(&tab.zo[i])[r];
    const float4 wx4 = tab.wx[i];
    const float wx[4] = {wx4.x, wx4.y, wx4.z, wx4.w};
    float *col = A + zo + ly * 4;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const int lx = (lxp >> (8 * o)) & 0xFF;
      if (lx != 0xFF) atomicAdd(col + lx * 32, (wx[o] * wy) * wz);
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Named barrier `id` over `count` producer threads.
__device__ __forceinline__ void producers_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// The same barrier, also returning the OR of `v` over its threads.
__device__ __forceinline__ bool producers_sync_or(bool v, int id, int count) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}\n"
      : "=r"(out)
      : "r"(static_cast<uint32_t>(v)), "r"(id), "r"(count)
      : "memory");
  return out != 0;
}

// Persistent, warp-specialized: grid = min(work items, resident CTAs), block
// kTcThreads.  Work items as in k_spread_zdft, in the same order in every role:
//   producer warps (kTcProducerWarps): zero the stage's A tile, spread the
//               item's atoms into it (a per-atom pre-pass, then shared-memory
//               atomics per tap), subtract the padding mean and split it into
//               the TF32 head (in place) and remainder.  With two operand
//               stages they form two groups that take alternate items (group g:
//               items j = g mod 2, stage and record slot g, named barrier 1 + g,
//               its own atom table), so one group's barriers and waits overlap
//               the other group's work
//   next warp   one lane issues the 3xTF32 MMAs of an item into its TMEM stage
//   next warp   loader: home-bin record ranges, frame/type/tile and padding mean
//               of an item, and bulk copies (cp.async.bulk) of its atom records
//               into a staging buffer
//   last 4      epilogue: TMEM accumulator -> Z (warp w reads lane quarter w%4)
// Hand-offs are mbarriers, every wait bounded:
//   rec_full[b]   loader -> producers (records + item data of slot b landed)
//   rec_empty[b]  producers -> loader (slot b spread)
//   full[s]       producers -> MMA (stage s operands written)
//   done[s]       MMA commit -> epilogue (accumulator ready) and producers
//                 (stage s operands free again)
//   tmem_empty[s] epilogue -> MMA (TMEM stage s read out)
// Dynamic shared memory: Bh, Bl (tcK x tcN floats each), tcS stages of
// A32 (tcR x 64) + Al (tcK x 64), two record buffers of tcRB float4, the
// home-bin tables (stiles[0] + stiles[1] int4) and one atom table per producer
// group.
__global__ void __launch_bounds__(kTcThreads, 1) k_spread_zdft_tc(DevArgs a, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];  // no-swizzle operands need 16 B
  __shared__ TcSlot slot[2];
  __shared__ __align__(8) uint64_t bars[10];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int N = a.tcN, KT = a.tcK, R = a.tcR, S = a.tcS, RB = a.tcRB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float *bh = reinterpret_cast<float *>(smem);
  float *bl = bh + KT * N;
  float *stages = bl + KT * N;
  float4 *recs = reinterpret_cast<float4 *>(stages + static_cast<size_t>(S) * (R + KT) * 64);
  int4 *home_x = reinterpret_cast<int4 *>(recs + 2 * RB);
  int4 *home_y = home_x + a.stiles[0];
  // producer groups: two when there are two operand stages
  const int G = (S == 2 && a.tcG == 2) ? 2 : 1;
  const int group = warp < kTcProducerWarps ? warp / (kTcProducerWarps / G) : 0;
  const int gthreads = kTcProducers / G, gtid = tid - group * gthreads;
  const int cap = a.tcCap;
  AtomTab tab;
  tab.wx = reinterpret_cast<float4 *>(reinterpret_cast<unsigned char *>(home_y + a.stiles[1]) +
                                      static_cast<size_t>(group) * cap * kTcAtomBytes);
  tab.wy = tab.wx + cap;
  tab.wz = tab.wy + cap;
  tab.zo = reinterpret_cast<int4 *>(tab.wz + cap);
  tab.lx = reinterpret_cast<int *>(tab.zo + cap);
  tab.ly = tab.lx + cap;
  uint64_t *rec_full = bars, *rec_empty = bars + 2, *full = bars + 4, *done = bars + 6,
           *tmem_empty = bars + 8;
  {
    const float4 *src = reinterpret_cast<const float4 *>(a.twz_tc);
    float4 *dst = reinterpret_cast<float4 *>(bh);
    for (int i = tid; i < KT * N / 2; i += blockDim.x) dst[i] = src[i];
    for (int i = tid; i < a.stiles[0]; i += blockDim.x) home_x[i] = a.home_x[i];
    for (int i = tid; i < a.stiles[1]; i += blockDim.x) home_y[i] = a.home_y[i];
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(a.tcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    const int counts[10] = {1, 1, 1, 1, kTcProducerWarps / G, kTcProducerWarps / G, 1, 1, 4, 4};
    for (int i = 0; i < 10; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bars[i])), "r"(counts[i]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  // bounded wait; on a timeout the whole block switches to skipping its work
  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicExch(a.status, 1);
    }
  };

  if (warp < kTcProducerWarps) {
    const int bar_id = 1 + group;
    for (int j = group, w = blockIdx.x + group * gridDim.x; w < items; j += G, w += G * gridDim.x) {
      const int b = j & 1, s = S == 2 ? (j & 1) : 0;
      float *A32 = stages + static_cast<size_t>(s) * (R + KT) * 64;
      float *Al = A32 + static_cast<size_t>(R) * 64;
      if (j >= S) wait(&done[s], (j - S) / S);  // the stage's previous MMAs are finished
      {
        float4 *t4 = reinterpret_cast<float4 *>(A32);
        for (int i = gtid; i < R * 16; i += gthreads) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      wait(&rec_full[b], j >> 1);
      // one decision for all producers: the spreading below has barriers inside
      const bool skip = producers_sync_or(abort_flag != 0, bar_id, gthreads);
      const TcSlot &sl = slot[b];
      const float mean = sl.mean;
      if (!skip) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        const int nrec = min(nvis, RB);
        for (int v0 = 0; v0 < nvis; v0 += cap) {
          const int nv = min(cap, nvis - v0);
          if (v0 > 0) producers_sync(bar_id, gthreads);  // the previous chunk's taps have read the table
          spread_prepass(a, sl.ta, recs + static_cast<size_t>(b) * RB, nrec, sl.f, v0, nv, tab, sl.x0,
                         sl.y0, sl.cw, sl.ch, gtid, gthreads);
          producers_sync(bar_id, gthreads);
          spread_taps(tab, nv, a.ntaps, A32, gtid, gthreads);
        }
      }
      producers_sync(bar_id, gthreads);
      if (gtid == 0) mbar_arrive(smem_addr(&rec_empty[b]));
      {
        // padding mean applied before the TF32 split: the tensor cores see
        // g - mean (rows z >= ez meet zero twiddles)
        float4 *h4 = reinterpret_cast<float4 *>(A32);
        float4 *l4 = reinterpret_cast<float4 *>(Al);
        for (int i = gtid; i < KT * 16; i += gthreads) {
          float4 v = h4[i];
          v.x -= mean;
          v.y -= mean;
          v.z -= mean;
          v.w -= mean;
          const float4 h = make_float4(tf32_head(v.x), tf32_head(v.y), tf32_head(v.z), tf32_head(v.w));
          h4[i] = h;
          l4[i] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&full[s]));
    }
  } else if (warp == kTcMmaWarp) {
    if (lane == 0) {
      // kind::tf32 instruction descriptor: D f32 (bits 4-5 = 1), A and B tf32 (2),
      // both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 64).
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) |
                             (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(64 >> 4) << 24);
      const uint32_t bstep = static_cast<uint32_t>(N) * 32;  // bytes per 8 z of B
      const uint64_t dbh0 = umma_desc(smem_addr(bh), N * 16, 128);
      const uint64_t dbl0 = umma_desc(smem_addr(bl), N * 16, 128);
      int j = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++j) {
        const int s = S == 2 ? (j & 1) : 0;
        const float *A32 = stages + static_cast<size_t>(s) * (R + KT) * 64;
        const float *Al = A32 + static_cast<size_t>(R) * 64;
        wait(&full[s], j / S);
        if (j >= S) wait(&tmem_empty[s], (j - S) / S);
        if (abort_flag) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + static_cast<uint32_t>(s * N);
        const uint64_t dah0 = umma_desc(smem_addr(A32), 1024, 128);
        const uint64_t dal0 = umma_desc(smem_addr(Al), 1024, 128);
        // descriptor start addresses are in 16-byte units: one k step of A is
        // 2048 B (+128), of B N*32 B (+N*2)
        for (int kk = 0; kk < KT / 8; ++kk) {
          const uint64_t dah = dah0 + static_cast<uint64_t>(kk * 128);
          const uint64_t dal = dal0 + static_cast<uint64_t>(kk * 128);
          const uint64_t dbh = dbh0 + static_cast<uint64_t>(kk * (bstep >> 4));
          const uint64_t dbl = dbl0 + static_cast<uint64_t>(kk * (bstep >> 4));
          umma_tf32(d, dal, dbh, idesc, kk > 0 ? 1u : 0u);
          umma_tf32(d, dah, dbl, idesc, 1u);
          umma_tf32(d, dah, dbh, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&done[s]))
                     : "memory");
        last_bar = smem_addr(&done[s]);
        last_parity = j / S;
      }
      // a wait ran out somewhere: let the newest MMAs finish (bounded) before the
      // tensor memory is released
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else if (warp == kTcLoaderWarp) {
    ItemIter it;
    it.init(a, blockIdx.x, gridDim.x);
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int b = j & 1;
      const int x0 = it.tx * kTile, y0 = it.ty * kTile;
      int s0, cnt;
      bool valid;
      // the range and mean loads are issued before the wait for the slot
      home_ranges_load(a, home_x, home_y, it.f, it.t, x0, y0, s0, cnt, valid);
      const float pmean = a.pad_val ? a.pad_val[it.t] : 0.0f;
      const double bsum = a.pad_val ? 0.0 : a.border[static_cast<int64_t>(it.f) * a.T + it.t];
      if (j >= 2) wait(&rec_empty[b], (j - 2) >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      TcSlot &sl = slot[b];
      home_ranges_publish(sl.ta, s0, cnt, valid);
      if (lane == 0) {
        sl.f = it.f;
        sl.t = it.t;
        sl.x0 = x0;
        sl.y0 = y0;
        sl.cw = min(kTile, a.ext[0] - x0);
        sl.ch = min(kTile, a.ext[1] - y0);
        sl.mean = a.pad_val ? pmean : static_cast<float>(bsum / a.border_count);
      }
      __syncwarp();
      if (lane == 0) {
        const TileAtoms &tb = sl.ta;
        const int nrec = min(tb.cum[tb.nb], RB);
        const uint32_t bar = smem_addr(&rec_full[b]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(nrec * 16)
                     : "memory");
        const float4 *src = a.rec + static_cast<int64_t>(it.f) * a.M;
        const uint32_t dst = smem_addr(recs + static_cast<size_t>(b) * RB);
        // one bulk copy per run of ranges that are contiguous in global memory
        int r = 0;
        while (r < tb.nb && tb.cum[r] < nrec) {
          int e = r;
          while (e + 1 < tb.nb && tb.start[e + 1] == tb.start[e] + (tb.cum[e + 1] - tb.cum[e])) ++e;
          const int lo = tb.cum[r], hi = min(tb.cum[e + 1], nrec);
          if (hi > lo)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dst + static_cast<uint32_t>(lo) * 16),
                "l"(src + tb.start[r]), "r"((hi - lo) * 16), "r"(bar)
                : "memory");
          r = e + 1;
        }
      }
    }
  } else {
    // epilogue warps
    const int quarter = warp & 3;
    ItemIter it;
    it.init(a, blockIdx.x, gridDim.x);
    const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int s = S == 2 ? (j & 1) : 0;
      wait(&done[s], j / S);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int x0 = it.tx * kTile, y0 = it.ty * kTile;
      float2 *Zft = a.Z + (static_cast<int64_t>(it.f) * a.T + it.t) * a.nkz * zplane;
      // with M = 64, row c of D sits in TMEM lane (c % 16) + 32 * (c / 16)
      const int c = 16 * quarter + lane, lx = c >> 3, ly = c & 7;
      const bool valid = lane < 16 && lx < min(kTile, a.ext[0] - x0) && ly < min(kTile, a.ext[1] - y0);
      const int64_t cell = static_cast<int64_t>(x0 + lx) * a.ext[1] + (y0 + ly);
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + static_cast<uint32_t>(s * N);
      for (int c0 = 0; c0 < N; c0 += 8) {
        uint32_t r[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                       "=r"(r[6]), "=r"(r[7])
                     : "r"(lane_base + c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int kz = c0 / 2 + jj;
            if (kz < a.nkz)
              Zft[kz * zplane + cell] = make_float2(__uint_as_float(r[2 * jj]), __uint_as_float(r[2 * jj + 1]));
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&tmem_empty[s]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kTcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tcCols));
}


// ---------------------------------------------------------------------------
// Wide-tile tensor-core spreading + z-axis DFT (k_spread_zdft_tcw)
// ---------------------------------------------------------------------------
// The same GEMM as k_spread_zdft_tc with M = 128 columns per work item (a tile
// of 8 x-columns by 16 y-rows, column m = 16*lx + ly in TMEM lane m): twice the
// columns per item halve the per-item fixed work and the halo share of the
// atoms, and M = 128 runs the tensor core at its full rate.  The tile is
// accumulated in shared memory in 32-bit fixed point (integer atomics; see
// tw_scale) as [m][z] rows of twRS words (twRS = tcR + 4, so that 8 consecutive
// rows of 16-byte loads and the 16 taps of one atom fall in distinct banks),
// then split into an f16 head and remainder straight into tensor memory, where
// the kind::f16 MMAs (K = 16) read A.
// An MMA costs about the same up to N = 192 (it is bound by its issue and
// accumulator latency, not by its N), so B holds the twiddle head and
// remainder side by side, B' = [Bh | Bl] (N' = 2*twN), and one k step is two
// MMAs, D += Ah * B' and D += Al * B', where three were needed with separate
// operands; the epilogue adds the two halves of D:
// D[:, n] + D[:, twN + n] = (Ah + Al)(Bh + Bl), all four products, and scales
// the sum back by 2^17 / scale.
// Tensor memory (512 columns):
//   [0, 256)    A ring: kTwRing = 8 slots of kTwChunk z (f16 pairs), head in
//               the first 16 columns of a slot, remainder in the next 16
//   [256, 512)  two accumulator stages of 2*twN <= 128 columns
constexpr int kTwX = 8, kTwY = 16;  // wide tile: x-columns, y-rows (M = 128)
constexpr int kTwProducerWarps = 24;
constexpr int kTwMmaWarp = kTwProducerWarps;
constexpr int kTwLoaderWarp = kTwProducerWarps + 1;
constexpr int kTwReleaseWarp = kTwProducerWarps + 6;
constexpr int kTwThreads = 32 * (kTwProducerWarps + 7);  // producers, MMA, loader, 4 epilogue, release
constexpr int kTwChunk = 32; // z per A ring slot
constexpr int kTwSlotCols = 32;  // tensor-memory columns of an A ring slot: 16 head + 16 remainder (f16 pairs)
constexpr int kTwRing = 8;   // A ring slots (two items of 128 z in flight)
static_assert(kTwRing * kTwSlotCols <= 256, "A ring and accumulator stages share 512 TMEM columns");

// Record ranges of an item's home bins (up to 4 along x times 8 along y).
struct TileAtomsW {
  int start[32];
  int cum[33];
  int nb;
};

struct TwSlot {
  TileAtomsW ta;
  int f, t, x0, y0, cw, ch;
  float mean;
  float scale;    // fixed-point scale of the item's tile (see tw_scale)
  float mean_fx;  // mean * scale
};

// The wide kernel accumulates its tile in 32-bit fixed point: shared-memory
// integer atomics issue about three times faster than FP32 ones on sm_100
// (1.97 against 6.6 cycles per warp-wide add per SM, measured).  A voxel of
// column (x, y) receives taps only from atoms whose home columns lie within
// four columns of it in x and in y: at most 3 x 3 home bins (2 x 2 unless a
// partial bin at the periodic edge is crossed), and each tap is a product of
// three B-spline weights: at most (2/3)^3 with two or more taps per axis, and
// (1/6)^3 with one (only the first cubic weight is used).  With `most` the
// largest home-bin count of the item, no voxel exceeds
// min(nvis, 9 * most) * tapmax and each rounded tap adds at most 1/2, so the
// scale 2^e with 2^e * (tapmax * bound + |mean|) <= 2e9 keeps every sum, and
// every sum minus mean * 2^e, below 2^31 in magnitude.  The scale is also kept
// at or below 2^22 / tapmax, so that a tap (below 2^22 units) can be rounded to
// an integer by adding 1.5 * 2^23 in FP32 (tap_fixed).  Each tap is rounded to
// 1/scale; at the 100k-atom workload (bound ~700, scale 2^23) that is an
// absolute error of at most 6e-8 per tap.
__device__ __forceinline__ float tw_scale(int nvis, int most, float mean, int ntaps) {
  const float tapmax = ntaps >= 2 ? 0.2964f : 0.00464f;
  const float bound = static_cast<float>(max(1, min(nvis, 9 * most)));
  const float e = floorf(log2f(2.0e9f / (tapmax * bound + fabsf(mean))));
  const float cap = floorf(log2f(4194304.0f / tapmax));
  return exp2f(fminf(e, cap));
}

// round(a * b) for 0 <= a * b < 2^22: one FMA with 1.5 * 2^23 leaves the rounded
// integer in the low mantissa bits (round to nearest even, as __float2int_rn).
__device__ __forceinline__ int tap_fixed(float a, float b) {
  return __float_as_int(fmaf(a, b, 12582912.0f)) - 0x4B400000;
}

// Padding mean of the item's type and frame, and the item's fixed-point scale:
// the loader and the epilogue evaluate the same expressions (one full warp).
__device__ __forceinline__ float tw_item_mean(const DevArgs &a, int f, int t) {
  return a.pad_val ? a.pad_val[t] : static_cast<float>(a.border[static_cast<int64_t>(f) * a.T + t] / a.border_count);
}

// Loader, first half, for wide tiles: lane 4*iy + ix loads the record range of
// home bin (hx[ix], hy[iy]); home_y holds eight bins per wide y tile.
__device__ __forceinline__ void home_ranges_load_w(const DevArgs &a, const int4 *home_x, const int4 *home_y,
                                                   int f, int t, int tx, int ty, int &s0, int &cnt,
                                                   bool &valid) {
  const int lane = threadIdx.x & 31;
  const int ix = lane & 3, iy = lane >> 2;
  const int4 hxv = home_x[tx], hyv = home_y[2 * ty + (iy >> 2)];
  const int hx = ix == 0 ? hxv.x : ix == 1 ? hxv.y : ix == 2 ? hxv.z : hxv.w;
  const int jy = iy & 3;
  const int hy = jy == 0 ? hyv.x : jy == 1 ? hyv.y : jy == 2 ? hyv.z : hyv.w;
  valid = hx >= 0 && hy >= 0;
  s0 = 0;
  cnt = 0;
  if (valid) {
    const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
    const int bin = (t * a.tiles[1] + hy) * a.tiles[0] + hx;
    s0 = off[bin];
    cnt = off[bin + 1] - s0;
  }
}

__device__ __forceinline__ void home_ranges_publish_w(TileAtomsW &ta, int s0, int cnt, bool valid) {
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, valid);
  const int pos = __popc(bal & ((1u << lane) - 1u));
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += v;
  }
  if (valid) {
    ta.start[pos] = s0;
    ta.cum[pos + 1] = inc;
  }
  if (lane == 0) {
    ta.cum[0] = 0;
    ta.nb = __popc(bal);
  }
}

// Pre-pass for wide tiles: as spread_prepass, with z offsets that are plain z
// rows of the [m][z] tile, and only the atoms whose stencil reaches the tile
// kept: each warp appends its reaching atoms to the table at *count (a
// shared-memory counter that starts at 0).
__device__ __forceinline__ void spread_prepass_w(const DevArgs &a, const TileAtomsW &ta, const float4 *srec,
                                                 int nrec_smem, int f, int v0, int nv, const AtomTabW &tab,
                                                 int x0, int y0, int cw, int ch, int rs, float scale, int tid,
                                                 int nthreads, int *count) {
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  const int lane = tid & 31;
  for (int i0 = tid - lane; i0 < nv; i0 += nthreads) {
    const int i = i0 + lane;
    const int v = v0 + min(i, nv - 1);
    float4 q;
    if (v < nrec_smem) {
      q = srec[v];
    } else {
      int j = 0;
      while (v >= ta.cum[j + 1]) ++j;
      q = a.rec[static_cast<int64_t>(f) * a.M + ta.start[j] + (v - ta.cum[j])];
    }
    const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y), m2 = static_cast<int>(q.z);
    float wx[4], wy[4], wz[4];
    cubic_weights(q.x - static_cast<float>(m0), wx);
    cubic_weights(q.y - static_cast<float>(m1), wy);
    cubic_weights(q.z - static_cast<float>(m2), wz);
    int xo[4], lyp = 0, zo[4];
    bool anyx = false;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      int by = 0xFF, zz = 0;
      xo[o] = -1;
      if (o < nt) {
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw)) {
          xo[o] = (x - x0) * kTwY * rs;
          anyx = true;
        }
        int y = m1 - P + o;
        if (y < 0) y += a.n[1];
        if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch)) by = y - y0;
        int z = m2 - P + o;
        if (z < 0) z += nz;
        zz = z;
      } else {
        wz[o] = 0.0f;  // a missing z tap adds 0 at row 0; a missing y tap is outside
      }
      lyp |= by << (8 * o);
      zo[o] = zz;
    }
    const bool reach = i < nv && anyx && lyp != -1;
    const unsigned m = __ballot_sync(0xffffffffu, reach);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (reach) {
      const int e = base + __popc(m & ((1u << lane) - 1u));
      tab.wxs[e] = make_float4(wx[0] * scale, wx[1] * scale, wx[2] * scale, wx[3] * scale);
      tab.wy[e] = make_float4(wy[0], wy[1], wy[2], wy[3]);
      tab.wz[e] = make_float4(wz[0], wz[1], wz[2], wz[3]);
      tab.zo[e] = make_int4(zo[0], zo[1], zo[2], zo[3]);
      tab.xo[e] = make_int4(xo[0], xo[1], xo[2], xo[3]);
      tab.ly[e] = lyp;
    }
  }
}

// Taps for wide tiles: one lane per (atom, y tap, z tap), four x taps each, into
// the [m][z] tile (row stride rs, m = 16*lx + ly).  With rs = 4 (mod 32) the 16
// lanes of an atom write banks 4*ly + z (mod 32), all distinct.  Each thread
// takes two units per round and reads both units' table entries before either
// unit's atomics, so the shared-memory loads of one overlap the other.
struct TapUnit {
  int *col;  // tile row start of the unit's (y tap, z tap), or null when outside
  int i;     // the atom's table entry
  float w;   // wy * wz
};

__device__ __forceinline__ TapUnit tap_unit(const AtomTabW &tab, int u, int nu, int *A, int rs) {
  TapUnit t;
  t.col = nullptr;
  if (u >= nu) return t;
  const int i = u >> 4, p = (u >> 2) & 3, r = u & 3;
  const int ly = reinterpret_cast<const unsigned char *>(&tab.ly[i])[p];  // byte p
  if (ly == 0xFF) return t;
  const float wy = reinterpret_cast<const float *>(&tab.wy[i])[p];
  const float wz = reinterpret_cast<const float *>(&tab.wz[i])[r];
  const int zo = reinterpret_cast<const int *>(&tab.zo[i])[r];
  t.i = i;
  t.w = wy * wz;
  t.col = A + zo + ly * rs;
  return t;
}

__device__ __forceinline__ void tap_apply(const AtomTabW &tab, const TapUnit &t) {
  if (!t.col) return;
  const float4 w4 = tab.wxs[t.i];
  const int4 x4 = tab.xo[t.i];
  const float wx[4] = {w4.x, w4.y, w4.z, w4.w};
  const int xo[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
  for (int o = 0; o < 4; ++o)
    if (xo[o] >= 0) atomicAdd(t.col + xo[o], tap_fixed(wx[o], t.w));
}

__device__ __forceinline__ void spread_taps_w(const AtomTabW &tab, int nv, int *A, int rs, int tid,
                                              int nthreads) {
  const int nu = nv * 16;
  for (int u = tid; u < nu; u += 2 * nthreads) {
    const TapUnit t0 = tap_unit(tab, u, nu, A, rs);
    const TapUnit t1 = tap_unit(tab, u + nthreads, nu, A, rs);
    tap_apply(tab, t0);
    tap_apply(tab, t1);
  }
}

// Persistent, warp-specialized like k_spread_zdft_tc; grid = min(work items,
// SMs), block kTwThreads.  Work items w = ((f*T + t)*stw + ty)*stiles[0] + tx.
//   producer warps: twG groups on alternate items, each with its own fixed-point
//               tile and atom table: pre-pass and shared-memory taps into the
//               tile, then the split, chunk by chunk of kTwChunk z: chunk q
//               (q = j*CH + c over the CTA's items j) goes to ring slot
//               q % kTwRing once the MMAs of chunk q - kTwRing are complete;
//               warp q (mod 4) with rank h < 2 among the group's warps of that
//               lane quarter converts rows 32q..32q+31, z in [32c + 16h, +16)
//               ((tile - mean) * 2^-17 -> f16 head and remainder) with
//               tcgen05.st and zeroes what it read
//   MMA warp    one lane issues per chunk 2 x (kTwChunk/16) kind::f16 MMAs with A
//               from tensor memory (M = 128, N = 2*twN, K = 16) into the item's
//               accumulator stage, chunk by chunk as the split delivers them
//   loader warp home-bin record ranges (up to 32 bins), item data, bulk copies
//   4 epilogue  accumulator halves summed -> Z (lane m = column 16*lx + ly)
//   release     one lane waits for the MMA completion of every chunk in order
//               and publishes the count of completed chunks (`released`)
// Hand-offs (mbarriers, every wait bounded):
//   rec_full[b] / rec_empty[b]   loader <-> producers, record slot b
//   a_full[s]                    8 split units (4 lane quarters x 2) -> MMA
//   a_empty[s]                   MMA commit -> release lane
//   released                     release lane -> split warps (a counter)
//   acc_full[d] / acc_empty[d]   MMA commit -> epilogue -> MMA, stage d
// Each mbarrier has waiters that observe every one of its phases in order and
// can neither fall two phases behind nor run two ahead (parity waits cannot
// tell those apart); the ring slots, filled by both groups, are handed back
// through the monotonic counter instead.
// Dynamic shared memory: B' (tcK x 2*twN halves), twG tiles of 128 x twRS
// words, two record buffers of twRB float4, the home-bin tables (stiles[0] +
// 2*stw int4) and twG atom tables of twCap entries (kTwAtomBytes each).
__global__ void __launch_bounds__(kTwThreads, 1) k_spread_zdft_tcw(DevArgs a, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ TwSlot slot[2];
  __shared__ __align__(8) uint64_t bars[4 + 2 * kTwRing + 4];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  __shared__ volatile int released;
  __shared__ int tab_count[2][2][2];  // reaching atoms in the table: [group][item parity][chunk parity]
  const int NB = a.twN, N = 2 * a.twN, KT = a.tcK, R = a.tcR, RB = a.twRB, RS = a.twRS, G = a.twG;
  const int SR = 2;  // split warps per lane quarter (16 z of a chunk each); 4 measured no faster
  const int CH = (KT + kTwChunk - 1) / kTwChunk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float *bh = reinterpret_cast<float *>(smem);  // B' = [Bh | Bl], f16, K-major, N columns
  float *tiles = bh + KT * N / 2;
  float4 *recs = reinterpret_cast<float4 *>(tiles + static_cast<size_t>(G) * 128 * RS);
  int4 *home_x = reinterpret_cast<int4 *>(recs + 2 * RB);
  int4 *home_y = home_x + a.stiles[0];
  const int gwarps = kTwProducerWarps / G;
  const int group = warp < kTwProducerWarps ? warp / gwarps : 0;
  const int gthreads = 32 * gwarps, gtid = tid - group * gthreads;
  const int cap = a.twCap;
  AtomTabW tab;
  tab.wxs = reinterpret_cast<float4 *>(reinterpret_cast<unsigned char *>(home_y + 2 * a.stw) +
                                       static_cast<size_t>(group) * cap * kTwAtomBytes);
  tab.wy = tab.wxs + cap;
  tab.wz = tab.wy + cap;
  tab.zo = reinterpret_cast<int4 *>(tab.wz + cap);
  tab.xo = tab.zo + cap;
  tab.ly = reinterpret_cast<int *>(tab.xo + cap);
  uint64_t *rec_full = bars, *rec_empty = bars + 2, *a_full = bars + 4, *a_empty = bars + 4 + kTwRing,
           *acc_full = bars + 4 + 2 * kTwRing, *acc_empty = acc_full + 2;
  {
    const float4 *src = reinterpret_cast<const float4 *>(a.twz_tcw);
    float4 *dst = reinterpret_cast<float4 *>(bh);
    for (int i = tid; i < KT * N / 8; i += blockDim.x) dst[i] = src[i];
    float4 *t4 = reinterpret_cast<float4 *>(tiles);
    for (int i = tid; i < G * 32 * RS; i += blockDim.x) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < a.stiles[0]; i += blockDim.x) home_x[i] = a.home_x[i];
    for (int i = tid; i < 2 * a.stw; i += blockDim.x) home_y[i] = a.home_yw[i];
  }
  if (warp == kTwMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < 4 + 2 * kTwRing + 4; ++i) {
      int cnt = 1;
      if (i >= 4 && i < 4 + kTwRing) cnt = 4 * SR;  // a_full: 4 lane quarters x SR split warps
      if (i >= 4 + 2 * kTwRing + 2) cnt = 4;   // acc_empty: 4 epilogue warps
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bars[i])), "r"(cnt));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    released = 0;
    for (int i = 0; i < 8; ++i) (&tab_count[0][0][0])[i] = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicExch(a.status, 1);
    }
  };
  // bounded wait until the MMAs of the first `n` chunks are complete: an acquire
  // load of the counter the release lane publishes with a release store (a
  // fence here would also wait for this warp's outstanding tap reductions)
  const uint32_t released_addr = smem_addr(const_cast<const int *>(&released));
  auto released_acquire = [&]() {
    int v;
    asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(released_addr) : "memory");
    return v;
  };
  auto wait_released = [&](int n) {
    if (released_acquire() >= n || abort_flag) return;
    const uint64_t t0 = global_ns();
    while (released_acquire() < n && !abort_flag) {
      if (global_ns() - t0 > 2000000000ull) {
        abort_flag = 1;
        atomicExch(a.status, 1);
      }
      __nanosleep(64);
    }
  };

  if (warp < kTwProducerWarps) {
    const int bar_id = 1 + group;
    float *A = tiles + static_cast<size_t>(group) * 128 * RS;
    const int gw = warp - group * gwarps;          // warp within the group (groups start at multiples of 4)
    const int quarter = warp & 3, rq = gw >> 2;
    const int m = 32 * quarter + lane;             // the tile row this lane splits
    float *row = A + static_cast<size_t>(m) * RS;
    // split warps: rank < SR in their lane quarter (group threads 0..128*SR-1);
    // the group's other warps pre-pass the next item's first table chunk while
    // the split warps split the current item
    const bool splitter = rq < SR;
    const int ns_tid = gtid - 128 * SR, ns_threads = gthreads - 128 * SR;
    for (int j = group, w = blockIdx.x + group * gridDim.x; w < items; j += G, w += G * gridDim.x) {
      const int b = j & 1, ip = (j / G) & 1;
      wait(&rec_full[b], j >> 1);
      const TwSlot &sl = slot[b];
      // chunk k of an item's visible atoms counts its reaching atoms in
      // tab_count[group][item parity][k & 1]
      if (!splitter && !__any_sync(0xffffffffu, abort_flag != 0)) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        spread_prepass_w(a, sl.ta, recs + static_cast<size_t>(b) * RB, min(nvis, RB), sl.f, 0, min(cap, nvis),
                         tab, sl.x0, sl.y0, sl.cw, sl.ch, RS, sl.scale, ns_tid, ns_threads, &tab_count[group][ip][0]);
      }
      // the first chunk's table is complete and the previous item's split done
      const bool skip = producers_sync_or(abort_flag != 0, bar_id, gthreads);
      if (gtid == 0) tab_count[group][ip ^ 1][0] = tab_count[group][ip ^ 1][1] = 0;  // the next item's
      const float mean_fx = sl.mean_fx;
      if (!skip) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        const int nrec = min(nvis, RB);
        for (int v0 = 0, k = 0; v0 < nvis; v0 += cap, ++k) {
          if (k > 0) {
            // further chunks: all producer warps; the counter of chunk k - 1's
            // predecessor is free (its readers passed the barrier above)
            producers_sync(bar_id, gthreads);
            if (gtid == 0) tab_count[group][ip][(k + 1) & 1] = 0;
            spread_prepass_w(a, sl.ta, recs + static_cast<size_t>(b) * RB, nrec, sl.f, v0, min(cap, nvis - v0),
                             tab, sl.x0, sl.y0, sl.cw, sl.ch, RS, sl.scale, gtid, gthreads,
                             &tab_count[group][ip][k & 1]);
            producers_sync(bar_id, gthreads);
          }
          spread_taps_w(tab, tab_count[group][ip][k & 1], reinterpret_cast<int *>(A), RS, gtid, gthreads);
        }
      }
      producers_sync(bar_id, gthreads);
      if (gtid == 0) mbar_arrive(smem_addr(&rec_empty[b]));
      if (!splitter) continue;
      // rows z in [tcK, tcR) meet no twiddle: cleared for the next item
      for (int i = gtid; i < 128 * ((R - KT) / 4); i += 128 * SR) {
        const int mm = i / ((R - KT) / 4), zq = i % ((R - KT) / 4);
        reinterpret_cast<float4 *>(A + static_cast<size_t>(mm) * RS + KT)[zq] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      // split, chunk by chunk through the A ring
      for (int c = 0; c < CH; ++c) {
        const int q = j * CH + c, s = q % kTwRing;
        if (q >= kTwRing) wait_released(q - kTwRing + 1);
        __syncwarp();  // converged for the .sync.aligned tensor-memory stores
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int h = rq;
        // 16 z per split warp: (tile - mean) * 2^-17 in fixed-point units, split
        // into an f16 head and remainder; two halves per tensor-memory column,
        // head to the slot's first 16 columns, remainder to the next 16
        {
          const int z0 = kTwChunk * c + 16 * h;
          uint32_t hi[8], lo[8];
          // all four loads, then the zeroing stores, then the arithmetic
          int4 iv[4];
          int4 *p = reinterpret_cast<int4 *>(row + z0);
          const int nq = z0 < KT ? 4 : 0;  // KT is a multiple of 16: all or none of the 16 z
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4) iv[k4] = k4 < nq ? p[k4] : make_int4(0, 0, 0, 0);
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4)
            if (k4 < nq) p[k4] = make_int4(0, 0, 0, 0);
          const float mz = z0 < KT ? mean_fx : 0.0f;
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4) {
            const float v[4] = {(__int2float_rn(iv[k4].x) - mz) * 0x1p-17f, (__int2float_rn(iv[k4].y) - mz) * 0x1p-17f,
                                (__int2float_rn(iv[k4].z) - mz) * 0x1p-17f, (__int2float_rn(iv[k4].w) - mz) * 0x1p-17f};
#pragma unroll
            for (int e = 0; e < 4; e += 2) {
              const __half2 hh = __floats2half2_rn(v[e], v[e + 1]);
              const float2 hf = __half22float2(hh);
              const __half2 ll = __floats2half2_rn(v[e] - hf.x, v[e + 1] - hf.y);
              hi[2 * k4 + e / 2] = *reinterpret_cast<const uint32_t *>(&hh);
              lo[2 * k4 + e / 2] = *reinterpret_cast<const uint32_t *>(&ll);
            }
          }
          const uint32_t dst = tmem + (static_cast<uint32_t>(32 * quarter) << 16) +
                               static_cast<uint32_t>(kTwSlotCols * s + 8 * h);
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(dst),
                       "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]),
                       "r"(hi[7])
                       : "memory");
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(dst + 16),
                       "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]),
                       "r"(lo[7])
                       : "memory");
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&a_full[s]));
      }
    }
  } else if (warp == kTwMmaWarp) {
    if (lane == 0) {
      // kind::f16 (f16 A and B), D f32, A from tensor memory, B' K-major, N >> 3 at bit 17, M = 128
      const uint32_t idesc = (1u << 4) | (static_cast<uint32_t>(N >> 3) << 17) |
                             (static_cast<uint32_t>(128 >> 4) << 24);
      const uint64_t db0 = umma_desc(smem_addr(bh), N * 16, 128);
      const uint64_t bstep = static_cast<uint64_t>(N) * 2;  // 16 z of f16 B' in 16-byte units
      int j = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++j) {
        const int d = j & 1;
        const uint32_t dcol = tmem + 256u + static_cast<uint32_t>(128 * d);
        for (int c = 0; c < CH; ++c) {
          const int q = j * CH + c, s = q % kTwRing;
          wait(&a_full[s], q / kTwRing);
          if (c == 0 && j >= 2) wait(&acc_empty[d], (j - 2) >> 1);
          if (abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int ks = min(kTwChunk, KT - kTwChunk * c) / 16;
          for (int kk = 0; kk < ks; ++kk) {
            const uint32_t ahi = tmem + static_cast<uint32_t>(kTwSlotCols * s + 8 * kk);
            const uint64_t db = db0 + static_cast<uint64_t>(kTwChunk / 16 * c + kk) * bstep;
            umma_f16_ts(dcol, ahi + 16, db, idesc, (c | kk) ? 1u : 0u);
            umma_f16_ts(dcol, ahi, db, idesc, 1u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&a_empty[s]))
                       : "memory");
        }
        if (abort_flag) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&acc_full[d]))
                     : "memory");
        last_bar = smem_addr(&acc_full[d]);
        last_parity = j >> 1;
      }
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else if (warp == kTwLoaderWarp) {
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.T);
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int b = j & 1;
      const int x0 = it.tx * kTwX, y0 = it.ty * kTwY;
      int s0, cnt;
      bool valid;
      home_ranges_load_w(a, home_x, home_y, it.f, it.t, it.tx, it.ty, s0, cnt, valid);
      const int most = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
      const int nall = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
      const float mean = tw_item_mean(a, it.f, it.t);
      if (j >= 2) wait(&rec_empty[b], (j - 2) >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      TwSlot &sl = slot[b];
      home_ranges_publish_w(sl.ta, s0, cnt, valid);
      if (lane == 0) {
        sl.f = it.f;
        sl.t = it.t;
        sl.x0 = x0;
        sl.y0 = y0;
        sl.cw = min(kTwX, a.ext[0] - x0);
        sl.ch = min(kTwY, a.ext[1] - y0);
        sl.mean = mean;
        sl.scale = tw_scale(nall, most, mean, a.ntaps);
        sl.mean_fx = mean * sl.scale;
      }
      __syncwarp();
      if (lane == 0) {
        const TileAtomsW &tb = sl.ta;
        const int nrec = min(tb.cum[tb.nb], RB);
        const uint32_t bar = smem_addr(&rec_full[b]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(nrec * 16)
                     : "memory");
        const float4 *src = a.rec + static_cast<int64_t>(it.f) * a.M;
        const uint32_t dst = smem_addr(recs + static_cast<size_t>(b) * RB);
        int r = 0;
        while (r < tb.nb && tb.cum[r] < nrec) {
          int e = r;
          while (e + 1 < tb.nb && tb.start[e + 1] == tb.start[e] + (tb.cum[e + 1] - tb.cum[e])) ++e;
          const int lo = tb.cum[r], hi = min(tb.cum[e + 1], nrec);
          if (hi > lo)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dst + static_cast<uint32_t>(lo) * 16),
                "l"(src + tb.start[r]), "r"((hi - lo) * 16), "r"(bar)
                : "memory");
          r = e + 1;
        }
      }
    }
  } else if (warp == kTwReleaseWarp) {
    if (lane == 0) {
      const int mine = items > static_cast<int>(blockIdx.x)
                           ? (items - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1
                           : 0;
      for (int q = 0; q < mine * CH && !abort_flag; ++q) {
        wait(&a_empty[q % kTwRing], q / kTwRing);
        if (abort_flag) break;
        asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(released_addr), "r"(q + 1) : "memory");
      }
    }
  } else {
    const int quarter = warp & 3;
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.T);
    const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int d = j & 1;
      // the item's fixed-point scale, as the loader computed it (before the wait,
      // so that its loads overlap it): Z = D * 2^17 / scale
      float unscale;
      {
        int s0, cnt;
        bool valid;
        home_ranges_load_w(a, home_x, home_y, it.f, it.t, it.tx, it.ty, s0, cnt, valid);
        const int most = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
        const int nall = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
        unscale = 131072.0f / tw_scale(nall, most, tw_item_mean(a, it.f, it.t), a.ntaps);
      }
      wait(&acc_full[d], j >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int x0 = it.tx * kTwX, y0 = it.ty * kTwY;
      float2 *Zft = a.Z + (static_cast<int64_t>(it.f) * a.T + it.t) * a.nkz * zplane;
      const int m = 32 * quarter + lane, lx = m >> 4, ly = m & 15;
      const bool valid = lx < min(kTwX, a.ext[0] - x0) && ly < min(kTwY, a.ext[1] - y0);
      const int64_t cell = static_cast<int64_t>(x0 + lx) * a.ext[1] + (y0 + ly);
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + 256u +
                                 static_cast<uint32_t>(128 * d);
      for (int c0 = 0; c0 < NB; c0 += 8) {
        uint32_t r[8], t[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(lane_base + c0));
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]),
                       "=r"(t[7])
                     : "r"(lane_base + NB + c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int kz = c0 / 2 + jj;
            if (kz < a.nkz)
              Zft[kz * zplane + cell] =
                  make_float2((__uint_as_float(r[2 * jj]) + __uint_as_float(t[2 * jj])) * unscale,
                              (__uint_as_float(r[2 * jj + 1]) + __uint_as_float(t[2 * jj + 1])) * unscale);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&acc_empty[d]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kTwMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

// grid (ceil(ex/64), nkz, frames*T), block 256: y-axis DFT.
// Y[f,t,kz][ky][x] = sum_y Z[f,t,kz][x][y] * exp(-2 pi i ja y / nny).
__global__ void __launch_bounds__(kThreads) k_ydft(DevArgs a) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *zs = reinterpret_cast<float2 *>(smem);        // [kYChunk][kYStride]
  float2 *tys = zs + kYChunk * kYStride;                // [kYChunk][nkyp]
  const int ft = blockIdx.z, kz = blockIdx.y;
  const int xb = blockIdx.x * kYRows;
  const int ex = a.ext[0], ey = a.ext[1];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float2 *Zp = a.Z + (static_cast<int64_t>(ft) * a.nkz + kz) * ex * ey;
  float2 *Yp = a.Y + (static_cast<int64_t>(ft) * a.nkz + kz) * a.nky * ex;
  const int xr0 = xb + 2 * lane;
  for (int kp = 0; kp * kKyPass < a.nky; ++kp) {
    const int kbase = kp * kKyPass + warp * kKyGroup;
    float2 acc0[kKyGroup], acc1[kKyGroup];
#pragma unroll
    for (int j = 0; j < kKyGroup; ++j) acc0[j] = acc1[j] = make_float2(0.f, 0.f);
    for (int y0 = 0; y0 < ey; y0 += kYChunk) {
      const int yn = min(kYChunk, ey - y0);
      for (int i = tid; i < kYRows * kYChunk; i += blockDim.x) {
        const int row = i / kYChunk, yy = i % kYChunk;
        const int x = xb + row, y = y0 + yy;
        zs[yy * kYStride + row] =
            (x < ex && yy < yn) ? Zp[static_cast<int64_t>(x) * ey + y] : make_float2(0.f, 0.f);
      }
      {
        const float4 *src = reinterpret_cast<const float4 *>(a.twy + static_cast<size_t>(y0) * a.nkyp);
        float4 *dst = reinterpret_cast<float4 *>(tys);
        const int n4 = yn * a.nkyp / 2;
        for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
      }
      __syncthreads();
      if (kbase < a.nky) {
        for (int yy = 0; yy < yn; ++yy) {
          const float4 z2 = *reinterpret_cast<const float4 *>(zs + yy * kYStride + 2 * lane);
          const float4 *w4 = reinterpret_cast<const float4 *>(tys + yy * a.nkyp + kbase);
#pragma unroll
          for (int j = 0; j < kKyGroup / 2; ++j) {
            const float4 w = w4[j];
            // (z.x + i z.y)(w.x + i w.y)
            acc0[2 * j].x = fmaf(z2.x, w.x, fmaf(-z2.y, w.y, acc0[2 * j].x));
            acc0[2 * j].y = fmaf(z2.x, w.y, fmaf(z2.y, w.x, acc0[2 * j].y));
            acc1[2 * j].x = fmaf(z2.z, w.x, fmaf(-z2.w, w.y, acc1[2 * j].x));
            acc1[2 * j].y = fmaf(z2.z, w.y, fmaf(z2.w, w.x, acc1[2 * j].y));
            acc0[2 * j + 1].x = fmaf(z2.x, w.z, fmaf(-z2.y, w.w, acc0[2 * j + 1].x));
            acc0[2 * j + 1].y = fmaf(z2.x, w.w, fmaf(z2.y, w.z, acc0[2 * j + 1].y));
            acc1[2 * j + 1].x = fmaf(z2.z, w.z, fmaf(-z2.w, w.w, acc1[2 * j + 1].x));
            acc1[2 * j + 1].y = fmaf(z2.z, w.w, fmaf(z2.w, w.z, acc1[2 * j + 1].y));
          }
        }
      }
      __syncthreads();
    }
    if (kbase < a.nky) {
#pragma unroll
      for (int j = 0; j < kKyGroup; ++j) {
        const int ky = kbase + j;
        if (ky < a.nky) {
          if (xr0 < ex) Yp[static_cast<int64_t>(ky) * ex + xr0] = acc0[j];
          if (xr0 + 1 < ex) Yp[static_cast<int64_t>(ky) * ex + xr0 + 1] = acc1[j];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Tensor-core y- and x-axis DFTs (tcgen05, 3xTF32)
// ---------------------------------------------------------------------------
//
// Both passes are real GEMMs  D[r][n'] = sum_k' A[r][k'] B'[k'][n']  over blocks
// of 128 rows, with complex data read as real:
//   A[r][2u + c] = component c (0 re, 1 im) of the row's complex values at u
//                  (each row is contiguous in memory, so A is that memory read
//                  as floats), K' = 2 * (extent of u),
//   B'[2u + c][2k + d] = { Wr, Wi ; -Wi, Wr }[c][d] of the twiddle W[u][k],
//   D[r][2k + d] = component d of the transformed row at k,  N' = 2 * (number
//                  of k) padded to 16.
// y pass: rows are the x rows of one z-transformed plane Z[x][y] (u = y, k =
//   ky), 128 per item; the epilogue writes Y[ky][x].
// x pass: rows are (ky, type) pairs of one (frame, kz), row = (ky - ky0) * T +
//   type, kyb = 128 / T ky per item (rows beyond T*kyb unused), u = x, k = kx;
//   the epilogue applies the form factors, then the four warps of an epilogue
//   slot sum the types of each ky through shared memory, square and multiply by
//   the B-spline moduli (the SIMT kernel's k_xdft_post), writing
//   ibox[kz][ky][kx].
// K is streamed in chunks of kDtcChunk values of u: per chunk the loader warp
// issues one tensor copy (cp.async.bulk.tensor, no multicast, 128-byte swizzle)
// of the 128 rows x 32 floats into a raw staging tile (rows outside the data
// zero-filled by the tensor map) and one bulk copy of the B' chunk.  The
// producers split the raw rows into a TF32 head and remainder and store them to
// tensor memory, where the MMA reads A: row r of A is TMEM lane r, element k'
// column a0 + k'.  B' stays in shared memory, K-major no-swizzle (core matrices
// of 8 rows x 16 B): element (n', k') at (k'/4)*(N'/8)*32 + (n'/8)*32 + (n'%8)*4
// + k'%4 floats (LBO N'*16 B, SBO 128 B), split on the host.
constexpr int kDtcChunk = 16;                  // u values per K chunk (K' = 32)
constexpr int kDtcProducerWarps = 8;
constexpr int kDtcMmaWarp = kDtcProducerWarps;
constexpr int kDtcLoaderWarp = kDtcProducerWarps + 1;
// epilogue warps: 4 for the y pass (stores only), 12 for the x pass (form factors
// per element), a multiple of 4 so each TMEM lane quarter has the same number
template <bool kX>
__host__ __device__ constexpr int dtc_epi_warps() { return kX ? 12 : 4; }
template <bool kX>
__host__ __device__ constexpr int dtc_threads() { return 32 * (kDtcProducerWarps + 2 + dtc_epi_warps<kX>()); }
constexpr int kDtcMaxStages = 4;

// One pass's GEMM shape: N', K chunks, stages, TMEM columns, B' table.
// With `lo_smem` (when 2N' <= 256): only A's TF32 head goes to tensor memory (32
// columns per stage); the producers write A's remainder back in place into the
// 128-byte-swizzled tensor-copy tile, which the MMA reads as a K-major SWIZZLE_128B
// shared-memory operand, and B' holds head and remainder side by side (2N'
// columns).  A k step is then two MMAs, D += Ah [Bh|Bl] and D += Al [Bh|Bl] (a
// tf32 MMA costs about the same up to N = 192), instead of three; the epilogue
// adds the two halves of D.
struct DtcShape {
  int N, chunks, S, cols;
  int lo_smem;
  const float *B;  // [chunk]: head block then remainder block (N' x 2*kDtcChunk
                   // each), or one block of 2N' x 2*kDtcChunk with lo_smem
};

// Tensor copy of chunk c of item w's 128 rows into `dst`, 1024-byte aligned
// (128-byte swizzle: the 16-byte piece j of row r lands at piece j ^ (r % 8) of
// the row) (y pass: 3-D map
// {2*ey floats, ex rows, planes}; x pass: 5-D map {2*ex floats, type, ky, kz,
// frame} whose box {32, T, kyb, 1, 1} lands rows in (ky, type) order).
template <bool kX>
__device__ __forceinline__ void dtc_tensor_copy(const DevArgs &a, const CUtensorMap *map, int w, int c,
                                                uint32_t dst, uint32_t bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const int u0 = c * 2 * kDtcChunk;
  if (!kX) {
    const int xblocks = (a.ext[0] + 127) / 128;
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(m), "r"(u0), "r"((w % xblocks) * 128), "r"(w / xblocks), "r"(bar)
        : "memory");
  } else {
    const int kyb = a.xtcKyb;
    const int nblk = (a.nky + kyb - 1) / kyb;
    const int f = w / (a.nkz * nblk), kz = (w / nblk) % a.nkz;
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4, %5, %6}], [%7];" ::"r"(dst),
        "l"(m), "r"(u0), "r"(0), "r"((w % nblk) * kyb), "r"(kz), "r"(f), "r"(bar)
        : "memory");
  }
}

// Persistent, warp-specialized: grid = min(items, resident CTAs), block
// dtc_threads<kX>() (producers, MMA warp, loader warp, epilogue warps).  Items: y pass (plane, block of 128 x rows), planes ordered
// (frame, type, kz) like Z and Y; x pass (frame, kz, block of 128/TP ky).
// Barriers (all waits bounded):
//   bfull[st] loader copies -> producers and MMA (raw A rows and B' landed)
//   afull[st] producers -> MMA (A chunk of stage st split and written)
//   empty[st] MMA commit -> loader (stage st read)
//   dfull[d]  MMA commit -> epilogue (accumulator d complete)
//   dempty[d] epilogue -> MMA (accumulator d read out)
// Dynamic shared memory: S stages of { raw A rows (128 x K'), B' head, B'
// remainder (N' x K') } floats, 1024-byte aligned.  Tensor memory (512
// columns): accumulators d at columns d*N', A stage st at 2N' + 64*st (head) and
// + 32 (remainder).
template <bool kX>
__global__ void __launch_bounds__(dtc_threads<kX>(), 1)
    k_dft_tc(DevArgs a, DtcShape sh, const __grid_constant__ CUtensorMap amap, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];
  // x pass: per epilogue slot, the 128 rows x 8 kx of f_t * F summed over types
  __shared__ float2 xsum[kX ? 3 * 128 * 8 : 1];
  __shared__ __align__(8) uint64_t bars[3 * kDtcMaxStages + 4];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int N = sh.N, NS = sh.S, NC = sh.chunks;
  const int NM = sh.lo_smem ? 2 * N : N;             // MMA N, accumulator stage width
  const int AW = sh.lo_smem ? 32 : 64;               // tensor-memory columns of an A stage
  const int KP = 2 * kDtcChunk;                      // K' per chunk
  const int a_floats = 128 * KP, b_floats = N * KP;  // raw A tile; B' head or remainder
  const int stage_floats = a_floats + 2 * b_floats;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // swizzled tensor copies need a 1024-byte aligned destination: the stages
  // start at the first 1024-byte boundary of the dynamic shared memory
  float *stages = reinterpret_cast<float *>(smem + ((1024u - (smem_addr(smem) & 1023u)) & 1023u));
  uint64_t *afull = bars, *bfull = bars + kDtcMaxStages, *empty = bars + 2 * kDtcMaxStages,
           *dfull = bars + 3 * kDtcMaxStages, *dempty = dfull + 2;
  if (warp == kDtcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(sh.cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&afull[i])), "r"(kDtcProducerWarps));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bfull[i])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[i])), "r"(1));
    }
    for (int d = 0; d < 2; ++d) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&dfull[d])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&dempty[d])), "r"(dtc_epi_warps<kX>()));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicExch(a.status, 1);
    }
  };

  if (warp < kDtcProducerWarps) {
    // warp w owns TMEM lane quarter w % 4 (rows 32*(w%4) + lane) and K' columns
    // 16*(w/4) .. +15 of each chunk: four 16-byte reads of its row (swizzled
    // pieces, conflict-free across the 8 rows of a 1024-byte block), split, two
    // 16-column stores to tensor memory
    static_assert(kDtcProducerWarps == 8 && kDtcChunk == 16, "8 producer warps cover 128 rows x 32 columns");
    const int quarter = warp & 3, half = warp >> 2;
    const int r = 32 * quarter + lane;
    const uint32_t lane_off = static_cast<uint32_t>(32 * quarter) << 16;
    int g = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x) {
      for (int c = 0; c < NC; ++c, ++g) {
        const int st = g % NS;
        if (g >= NS) wait(&empty[st], g / NS - 1);  // the stage's MMAs have read its TMEM columns
        wait(&bfull[st], g / NS);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float *raw = stages + static_cast<size_t>(st) * stage_floats;
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = 4 * half + jj;
          float4 *p = reinterpret_cast<float4 *>(raw + r * KP + 4 * (j ^ (r & 7)));
          const float4 v = *p;
          const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float h = tf32_head(vv[e]);
            hi[4 * jj + e] = __float_as_uint(h);
            lo[4 * jj + e] = __float_as_uint(vv[e] - h);
          }
          if (sh.lo_smem)  // the remainder replaces the raw values in the swizzled tile
            *p = make_float4(__uint_as_float(lo[4 * jj]), __uint_as_float(lo[4 * jj + 1]),
                             __uint_as_float(lo[4 * jj + 2]), __uint_as_float(lo[4 * jj + 3]));
        }
        const uint32_t col = tmem + lane_off + static_cast<uint32_t>(2 * NM + AW * st + 16 * half);
        if (sh.lo_smem) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
            "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(col),
            "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]), "r"(hi[7]),
            "r"(hi[8]), "r"(hi[9]), "r"(hi[10]), "r"(hi[11]), "r"(hi[12]), "r"(hi[13]), "r"(hi[14]), "r"(hi[15]));
        if (!sh.lo_smem)
          asm volatile(
              "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
              "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(col + 32),
              "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]),
              "r"(lo[8]), "r"(lo[9]), "r"(lo[10]), "r"(lo[11]), "r"(lo[12]), "r"(lo[13]), "r"(lo[14]), "r"(lo[15]));
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&afull[st]));
      }
    }
  } else if (warp == kDtcLoaderWarp) {
    if (lane == 0) {
      const uint32_t bbytes = static_cast<uint32_t>(2 * b_floats * sizeof(float));
      // the tensor copy lands T*kyb rows in the x pass (128 in the y pass)
      const int arows = kX ? a.T * a.xtcKyb : 128;
      const uint32_t abytes = static_cast<uint32_t>(arows * KP * sizeof(float));
      int g = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x) {
        for (int c = 0; c < NC; ++c, ++g) {
          const int st = g % NS;
          if (g >= NS) wait(&empty[st], g / NS - 1);
          if (abort_flag) break;
          const uint32_t bar = smem_addr(&bfull[st]);
          float *sb = stages + static_cast<size_t>(st) * stage_floats;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bbytes + abytes)
                       : "memory");
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  smem_addr(sb + a_floats)),
              "l"(sh.B + static_cast<size_t>(c) * 2 * b_floats), "r"(bbytes), "r"(bar)
              : "memory");
          dtc_tensor_copy<kX>(a, &amap, w, c, smem_addr(sb), bar);
        }
      }
    }
  } else if (warp == kDtcMmaWarp) {
    if (lane == 0) {
      // kind::tf32: D f32, A and B tf32, both K-major, N >> 3 at bit 17, M = 128
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) |
                             (static_cast<uint32_t>(NM >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
      int g = 0, i = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++i) {
        const int d = i & 1;
        if (i >= 2) wait(&dempty[d], (i - 2) >> 1);
        const uint32_t dcol = tmem + static_cast<uint32_t>(d * NM);
        for (int c = 0; c < NC; ++c, ++g) {
          const int st = g % NS;
          wait(&bfull[st], g / NS);
          wait(&afull[st], g / NS);
          if (abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const float *sb = stages + static_cast<size_t>(st) * stage_floats;
          const uint32_t ah0 = tmem + static_cast<uint32_t>(2 * NM + AW * st);
          if (sh.lo_smem) {
            // B' = [Bh | Bl] (2N' columns); Al is the swizzled tile itself: a K-major
            // SWIZZLE_128B descriptor (layout type 2, 8-row groups 1024 B apart) whose
            // start advances 32 B per k step of 8 floats within the 128-byte rows
            const uint64_t db0 = umma_desc(smem_addr(sb + a_floats), NM * 16, 128);
            const uint64_t dal0 = umma_desc(smem_addr(sb), 16, 1024) | (static_cast<uint64_t>(2) << 61);
            for (int kk = 0; kk < KP / 8; ++kk) {
              const uint64_t db = db0 + static_cast<uint64_t>(kk * 2 * NM);
              umma_tf32_ts(dcol, ah0 + 8 * kk, db, idesc, (c > 0 || kk > 0) ? 1u : 0u);
              umma_tf32(dcol, dal0 + static_cast<uint64_t>(2 * kk), db, idesc, 1u);
            }
          } else {
            const uint64_t dbh0 = umma_desc(smem_addr(sb + a_floats), N * 16, 128);
            const uint64_t dbl0 = umma_desc(smem_addr(sb + a_floats + b_floats), N * 16, 128);
            // one k step (8 of K'): A advances 8 TMEM columns, B' N*32 B (+N*2)
            for (int kk = 0; kk < KP / 8; ++kk) {
              const uint32_t ah = ah0 + 8 * kk, al = ah + 32;
              const uint64_t dbh = dbh0 + static_cast<uint64_t>(kk * 2 * N);
              const uint64_t dbl = dbl0 + static_cast<uint64_t>(kk * 2 * N);
              umma_tf32_ts(dcol, al, dbh, idesc, (c > 0 || kk > 0) ? 1u : 0u);
              umma_tf32_ts(dcol, ah, dbl, idesc, 1u);
              umma_tf32_ts(dcol, ah, dbh, idesc, 1u);
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&empty[st]))
                       : "memory");
          last_bar = smem_addr(&empty[st]);
          last_parity = g / NS;
        }
        if (abort_flag) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&dfull[d]))
                     : "memory");
      }
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w%4).. = rows of the block; the
    // epilogue warps of one lane quarter take every EQ-th 16-column group
    constexpr int EQ = dtc_epi_warps<kX>() / 4;
    const int quarter = warp & 3;
    const int eslot = (warp - (kDtcLoaderWarp + 1)) / 4;
    const int r = 32 * quarter + lane;
    int i = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++i) {
      const int d = i & 1;
      wait(&dfull[d], i >> 1);
      // x pass: the four warps of a slot meet at named barriers, so they decide together
      if (kX ? producers_sync_or(abort_flag != 0, 1 + eslot, 128) : __any_sync(0xffffffffu, abort_flag != 0))
        break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + static_cast<uint32_t>(d * NM);
      // 16 accumulator columns from c0 (with lo_smem: the sum of the two halves)
      auto load16 = [&](int c0, uint32_t v[16]) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(lane_base + c0));
        if (sh.lo_smem) {
          uint32_t u[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
              "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
                "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
              : "r"(lane_base + N + c0));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] = __float_as_uint(__uint_as_float(v[q]) + __uint_as_float(u[q]));
        } else {
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
      };
      if (!kX) {
        const int ex = a.ext[0];
        const int xblocks = (ex + 127) / 128;
        const int64_t plane = w / xblocks;
        const int x = (w % xblocks) * 128 + r;
        float2 *Yp = a.Y + plane * a.nky * ex;
        for (int c0 = 16 * eslot; c0 < N; c0 += 16 * EQ) {
          uint32_t v[16];
          load16(c0, v);
          if (x < ex) {
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const int ky = c0 / 2 + jj;
              if (ky < a.nky)
                Yp[static_cast<int64_t>(ky) * ex + x] =
                    make_float2(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1]));
            }
          }
        }
      } else {
        // rows r = kyl * T + t (kyl < kyb); each lane finishes f_t * F for its row,
        // the four warps of this epilogue slot (one per lane quarter) meet in
        // shared memory to sum the types of each ky, square and scale
        const int T = a.T, kyb = a.xtcKyb;
        const int nblk = (a.nky + kyb - 1) / kyb;
        const int f = w / (a.nkz * nblk), kz = (w / nblk) % a.nkz;
        const int ky0 = (w % nblk) * kyb;
        const int kyl = r / T, t = r % T, ky = ky0 + kyl;
        const bool row_ok = r < T * kyb && ky < a.nky;
        float ocs[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) ocs[q] = a.geom[f * kGeom + 9 + q];
        const int ka = signed_k(kz, a.nn[2], a.nf[2]);
        const int ja = a.ky_lo + min(ky, a.nky - 1);
        const float mean = row_ok ? padding_mean(a, f, t) : 0.0f;
        float ff[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) ff[q] = a.ff[9 * t + q];
        float2 *red = xsum + eslot * 128 * 8;  // [row][8 kx]
        const int rid = 32 * quarter + lane;    // 0..127 over the slot's four warps
        const uint32_t bar_id = 1 + eslot;
        for (int c0 = 16 * eslot; c0 < N; c0 += 16 * EQ) {
          uint32_t v[16];
          load16(c0, v);
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int kx = c0 / 2 + jj;
            const int ia = a.kx_lo + min(kx, a.nkx - 1);
            const float mw = kpoint_q(ocs, ia, ja, ka);
            const bool inside = row_ok && kx < a.nkx && !(mw > a.qcut);
            float2 F = make_float2(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1]));
            // the padding mean's constant over the whole supercell lands at k = 0
            if (ka == 0 && ja == 0 && ia == 0)
              F.x += static_cast<float>(static_cast<double>(mean) * a.nn3);
            float2 A = make_float2(0.f, 0.f);
            if (inside) {
              const float q = mw / (4.0 * M_PI);
              const float ft = form_factor(ff, q * q);
              A.x = ft * F.x;
              A.y = ft * F.y;
            }
            red[r * 8 + jj] = A;
          }
          asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");
          for (int p = rid; p < kyb * 8; p += 128) {
            const int kl = p >> 3, jj = p & 7;
            const int kyy = ky0 + kl, kx = c0 / 2 + jj;
            if (kyy < a.nky && kx < a.nkx) {
              float2 A = make_float2(0.f, 0.f);
              for (int tt = 0; tt < T; ++tt) {
                const float2 e = red[(kl * T + tt) * 8 + jj];
                A.x += e.x;
                A.y += e.y;
              }
              const int ia = a.kx_lo + kx, jb = a.ky_lo + kyy;
              const float mw = kpoint_q(ocs, ia, jb, ka);
              const int iw = ia < 0 ? ia + a.nn[0] : ia, jw = jb < 0 ? jb + a.nn[1] : jb;
              a.ibox[((static_cast<int64_t>(f) * a.nkz + kz) * a.nky + kyy) * a.nkx + kx] =
                  !(mw > a.qcut) ? (A.x * A.x + A.y * A.y) * (a.modx[iw] * (a.mody[jw] * a.modz[kz])) : 0.0f;
            }
          }
          asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");  // before the next group's writes
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&dempty[d]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kDtcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(sh.cols));
}

// grid (ceil(nky/4), nkz, frames), block 256: x-axis DFT, form factors, type
// sum, modulus.  Dynamic shared memory, for an x chunk of `xc` values:
// twx xc*nkxp | Y rows T*xc | F T*nkxp (all float2).
__global__ void __launch_bounds__(kThreads) k_xdft_post(DevArgs a, int xc) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int ex = a.ext[0];
  float2 *txs = reinterpret_cast<float2 *>(smem);
  float2 *ys = txs + static_cast<size_t>(xc) * a.nkxp;
  float2 *fs = ys + static_cast<size_t>(a.T) * xc;
  __shared__ float ocs[9];
  __shared__ float means[64];
  const int f = blockIdx.z, kz = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid < 9) ocs[tid] = a.geom[f * kGeom + 9 + tid];
  for (int t = tid; t < a.T && t < 64; t += blockDim.x)
    means[t] = padding_mean(a, f, t);
  const bool one_chunk = xc >= ex;
  if (one_chunk) {
    const float4 *src = reinterpret_cast<const float4 *>(a.twx);
    float4 *dst = reinterpret_cast<float4 *>(txs);
    const int n4 = ex * a.nkxp / 2;
    for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
  }
  const int ka = signed_k(kz, a.nn[2], a.nf[2]);
  const int npairs = a.T * a.nkx;
  for (int r = 0; r < kXRows; ++r) {
    const int ky = blockIdx.x * kXRows + r;
    if (ky >= a.nky) break;
    const int ja = a.ky_lo + ky;
    for (int p0 = 0; p0 < npairs; p0 += blockDim.x) {
      const int i = p0 + tid;
      const int t = i / a.nkx, kx = i % a.nkx;
      float2 acc = make_float2(0.f, 0.f);
      for (int x0 = 0; x0 < ex; x0 += xc) {
        const int xn = min(xc, ex - x0);
        __syncthreads();
        for (int j = tid; j < a.T * xn; j += blockDim.x) {
          const int tt = j / xn, x = j % xn;
          ys[tt * xc + x] = a.Y[((static_cast<int64_t>(f) * a.T + tt) * a.nkz + kz) * a.nky * ex +
                                static_cast<int64_t>(ky) * ex + x0 + x];
        }
        if (!one_chunk) {
          const float4 *src = reinterpret_cast<const float4 *>(a.twx + static_cast<size_t>(x0) * a.nkxp);
          float4 *dst = reinterpret_cast<float4 *>(txs);
          const int n4 = xn * a.nkxp / 2;
          for (int j = tid; j < n4; j += blockDim.x) dst[j] = src[j];
        }
        __syncthreads();
        if (i < npairs) {
          const float2 *yr = ys + t * xc;
          for (int x = 0; x < xn; ++x) {
            const float2 v = yr[x];
            const float2 w = txs[x * a.nkxp + kx];
            acc.x = fmaf(v.x, w.x, fmaf(-v.y, w.y, acc.x));
            acc.y = fmaf(v.x, w.y, fmaf(v.y, w.x, acc.y));
          }
        }
      }
      if (i < npairs) {
        if (ka == 0 && ja == 0 && a.kx_lo + kx == 0)
          acc.x += static_cast<float>(static_cast<double>(means[t < 64 ? t : 63]) * a.nn3);
        fs[t * a.nkxp + kx] = acc;
      }
    }
    __syncthreads();
    for (int kx = tid; kx < a.nkx; kx += blockDim.x) {
      const int ia = a.kx_lo + kx;
      const float mw = kpoint_q(ocs, ia, ja, ka);
      float I = 0.0f;
      if (!(mw > a.qcut)) {
        const float q = mw / (4.0 * M_PI);
        const float q2 = q * q;
        float2 A = make_float2(0.f, 0.f);
        for (int t = 0; t < a.T; ++t) {
          const float ft = form_factor(a.ff + 9 * t, q2);
          const float2 F = fs[t * a.nkxp + kx];
          A.x = fmaf(ft, F.x, A.x);
          A.y = fmaf(ft, F.y, A.y);
        }
        const int i = ia < 0 ? ia + a.nn[0] : ia;
        const int j = ja < 0 ? ja + a.nn[1] : ja;
        const float bsp = a.modx[i] * a.mody[j] * a.modz[kz];
        I = (A.x * A.x + A.y * A.y) * bsp;
      }
      a.ibox[((static_cast<int64_t>(f) * a.nkz + kz) * a.nky + ky) * a.nkx + kx] = I;
    }
  }
}

// grid (nkz, planes), block 256: mirror-weighted histogram of one kz plane.
// `vals` holds nkz*nky*nkx values per plane; `geom` the frame geometry.
template <typename V>
__global__ void __launch_bounds__(kThreads)
    k_hist(DevArgs a, const V *vals, const float *geom, int geom_stride, double fact,
           double *hist, double *nhist) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int npts = a.nky * a.nkx;
  const bool in_smem = a.num_bins <= kHistSmemBins;
  double *sh = reinterpret_cast<double *>(smem);
  double *sn = sh + (in_smem ? a.num_bins : 0);
  __shared__ float ocs[9];
  const int kz = blockIdx.x, f = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid < 9) ocs[tid] = geom[f * geom_stride + 9 + tid];
  if (in_smem)
    for (int b = tid; b < 2 * a.num_bins; b += blockDim.x) sh[b] = 0.0;
  const V *pl = vals + (static_cast<int64_t>(f) * a.nkz + kz) * npts;
  __syncthreads();
  const int ka = signed_k(kz, a.nn[2], a.nf[2]);
  const int kx_hi = a.kx_lo + a.nkx - 1, ky_hi = a.ky_lo + a.nky - 1;
  double *dh = in_smem ? sh : hist;
  double *dn = in_smem ? sn : nhist;
  // Neighbouring k-points (consecutive lanes) mostly fall in the same bin: each
  // warp sums runs of equal bins in lane order (a segmented shuffle scan) and
  // the last lane of a run adds the run's sums, so the FP64 atomics contend
  // far less.
  const int lane = tid & 31;
  for (int p0 = tid - lane; p0 < npts; p0 += blockDim.x) {
    const int p = p0 + lane;
    int h0 = -1;
    double v = 0.0, c = 0.0;
    if (p < npts && a.dq > 0.0f) {
      const int ky = p / a.nkx, kx = p % a.nkx;
      const int ia = a.kx_lo + kx, ja = a.ky_lo + ky;
      const float mw = kpoint_q(ocs, ia, ja, ka);
      const int hb = static_cast<int>(mw / a.dq);
      if (!(mw > a.qcut) && hb >= 0 && hb < a.num_bins) {
        h0 = hb;
        if (ia == 0 && ja == 0 && ka == 0) {
          v = static_cast<double>(pl[p]) * fact;
          c = 1.0;
        } else {
          int ib = -ia, jb = -ja;
          if (ib > kx_hi) ib = ia;
          if (jb > ky_hi) jb = ja;
          const int pm = (jb - a.ky_lo) * a.nkx + (ib - a.kx_lo);
          if (sizeof(V) == 4)
            v = static_cast<double>(static_cast<float>(pl[p]) + static_cast<float>(pl[pm])) * fact;
          else
            v = (static_cast<double>(pl[p]) + static_cast<double>(pl[pm])) * fact;
          c = 2.0;
        }
      }
    }
    // first lane of this lane's run of equal bins
    const int hprev = __shfl_up_sync(0xffffffffu, h0, 1);
    int start = (lane == 0 || hprev != h0) ? lane : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) start = max(start, __shfl_up_sync(0xffffffffu, start, d));
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double vo = __shfl_up_sync(0xffffffffu, v, d);
      const double co = __shfl_up_sync(0xffffffffu, c, d);
      if (lane - d >= start) {
        v += vo;
        c += co;
      }
    }
    const int hnext = __shfl_down_sync(0xffffffffu, h0, 1);
    if (h0 >= 0 && (lane == 31 || hnext != h0)) {
      atomicAdd(dh + h0, v);
      atomicAdd(dn + h0, c);
    }
  }
  if (in_smem) {
    __syncthreads();
    for (int b = tid; b < a.num_bins; b += blockDim.x) {
      if (sn[b] != 0.0) {
        atomicAdd(hist + b, sh[b]);
        atomicAdd(nhist + b, sn[b]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// adjoint (reverse mode) kernels: dL/dI(bin) -> dL/dxyz for one frame
// ---------------------------------------------------------------------------

// Extra device buffers of the adjoint, allocated on first use.
struct AdjArgs {
  const double *dl;   // [num_bins] dL/d hist
  float2 *G;          // [T][nkz][nky][nkx] dL/dF_t (Re + i Im)
  float2 *H1;         // [T][nkz][nky][ex]  (the layout of Y)
  float2 *H2;         // [T][nkz][ex][ey]   (the layout of Z)
  const float2 *twyT; // [nky][eyp]: exp(-2 pi i ky y / nny) transposed
  const float2 *twzT; // [nkz][ezp]: exp(-2 pi i kz z / nnz) transposed
  int eyp, ezp;
  float *dg;          // [T][ex][ey][ez] dL/dg' on the corner block
  double *S;          // [T] sum of dg over the corner block
  float *dcg;         // [T] nn^3 * Re G_t(k = 0)
  float *grad;        // [natoms * 3] output
};

__device__ __forceinline__ double bin_weight(const DevArgs &a, const AdjArgs &j, const float *ocs,
                                             int ia, int ja, int ka) {
  const float mw = kpoint_q(ocs, ia, ja, ka);
  if (mw > a.qcut || a.dq <= 0.0f) return 0.0;
  const int h0 = static_cast<int>(mw / a.dq);
  if (h0 < 0 || h0 >= a.num_bins) return 0.0;
  return j.dl[h0];
}

// grid (ceil(nky/4), nkz), block 256: x-axis DFT of the recomputed Y rows, then
// G_t(p) = 2 w(p) M(p) f_t(p) A(p) with w(p) = g[bin(p)] + g[bin(mirror(p))].
__global__ void __launch_bounds__(kThreads) k_xdft_grad(DevArgs a, AdjArgs j, int xc) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int ex = a.ext[0];
  float2 *txs = reinterpret_cast<float2 *>(smem);
  float2 *ys = txs + static_cast<size_t>(xc) * a.nkxp;
  float2 *fs = ys + static_cast<size_t>(a.T) * xc;
  __shared__ float ocs[9];
  __shared__ float means[64];
  const int kz = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid < 9) ocs[tid] = a.geom[9 + tid];
  for (int t = tid; t < a.T && t < 64; t += blockDim.x)
    means[t] = padding_mean(a, 0, t);
  const int ka = signed_k(kz, a.nn[2], a.nf[2]);
  const int npairs = a.T * a.nkx;
  const int kx_hi = a.kx_lo + a.nkx - 1, ky_hi = a.ky_lo + a.nky - 1;
  for (int r = 0; r < kXRows; ++r) {
    const int ky = blockIdx.x * kXRows + r;
    if (ky >= a.nky) break;
    const int ja = a.ky_lo + ky;
    for (int p0 = 0; p0 < npairs; p0 += blockDim.x) {
      const int i = p0 + tid;
      const int t = i / a.nkx, kx = i % a.nkx;
      float2 acc = make_float2(0.f, 0.f);
      for (int x0 = 0; x0 < ex; x0 += xc) {
        const int xn = min(xc, ex - x0);
        __syncthreads();
        for (int q = tid; q < a.T * xn; q += blockDim.x) {
          const int tt = q / xn, x = q % xn;
          ys[tt * xc + x] = a.Y[(static_cast<int64_t>(tt) * a.nkz + kz) * a.nky * ex +
                                static_cast<int64_t>(ky) * ex + x0 + x];
        }
        {
          const float4 *src = reinterpret_cast<const float4 *>(a.twx + static_cast<size_t>(x0) * a.nkxp);
          float4 *dst = reinterpret_cast<float4 *>(txs);
          const int n4 = xn * a.nkxp / 2;
          for (int q = tid; q < n4; q += blockDim.x) dst[q] = src[q];
        }
        __syncthreads();
        if (i < npairs) {
          const float2 *yr = ys + t * xc;
          for (int x = 0; x < xn; ++x) {
            const float2 v = yr[x];
            const float2 w = txs[x * a.nkxp + kx];
            acc.x = fmaf(v.x, w.x, fmaf(-v.y, w.y, acc.x));
            acc.y = fmaf(v.x, w.y, fmaf(v.y, w.x, acc.y));
          }
        }
      }
      if (i < npairs) {
        if (ka == 0 && ja == 0 && a.kx_lo + kx == 0)
          acc.x += static_cast<float>(static_cast<double>(means[t < 64 ? t : 63]) * a.nn3);
        fs[t * a.nkxp + kx] = acc;
      }
    }
    __syncthreads();
    for (int kx = tid; kx < a.nkx; kx += blockDim.x) {
      const int ia = a.kx_lo + kx;
      const float mw = kpoint_q(ocs, ia, ja, ka);
      double w = 0.0;
      float q2 = 0.f;
      if (!(mw > a.qcut)) {
        const float q = mw / (4.0 * M_PI);
        q2 = q * q;
        w = bin_weight(a, j, ocs, ia, ja, ka);
        if (!(ia == 0 && ja == 0 && ka == 0)) {
          int ib = -ia, jb = -ja;
          if (ib > kx_hi) ib = ia;
          if (jb > ky_hi) jb = ja;
          w += bin_weight(a, j, ocs, ib, jb, ka);
        }
      }
      float2 A = make_float2(0.f, 0.f);
      if (w != 0.0) {
        for (int t = 0; t < a.T; ++t) {
          const float ft = form_factor(a.ff + 9 * t, q2);
          const float2 F = fs[t * a.nkxp + kx];
          A.x = fmaf(ft, F.x, A.x);
          A.y = fmaf(ft, F.y, A.y);
        }
      }
      const int ii = ia < 0 ? ia + a.nn[0] : ia;
      const int jj = ja < 0 ? ja + a.nn[1] : ja;
      const float bsp = a.modx[ii] * a.mody[jj] * a.modz[kz];
      const float s = static_cast<float>(2.0 * w) * bsp;
      for (int t = 0; t < a.T; ++t) {
        float2 g = make_float2(0.f, 0.f);
        if (w != 0.0) {
          const float ft = form_factor(a.ff + 9 * t, q2);
          g = make_float2(s * ft * A.x, s * ft * A.y);
        }
        j.G[((static_cast<int64_t>(t) * a.nkz + kz) * a.nky + ky) * a.nkx + kx] = g;
        if (ka == 0 && ja == 0 && ia == 0) j.dcg[t] = static_cast<float>(g.x * a.nn3);
      }
    }
  }
}

// H1[t][kz][ky][x] = sum_kx G[t][kz][ky][kx] conj(exp(-2 pi i kx x / nnx)); thread per output.
__global__ void k_xadj(DevArgs a, AdjArgs j) {
  const int ex = a.ext[0];
  const int64_t total = static_cast<int64_t>(a.T) * a.nkz * a.nky * ex;
  const int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= total) return;
  const int x = o % ex;
  const int64_t row = o / ex;  // (t, kz, ky)
  const float2 *g = j.G + row * a.nkx;
  const float2 *w = a.twx + static_cast<size_t>(x) * a.nkxp;
  float2 acc = make_float2(0.f, 0.f);
  for (int kx = 0; kx < a.nkx; ++kx) {
    const float2 v = g[kx], c = w[kx];        // v * conj(c)
    acc.x = fmaf(v.x, c.x, fmaf(v.y, c.y, acc.x));
    acc.y = fmaf(v.y, c.x, fmaf(-v.x, c.y, acc.y));
  }
  j.H1[o] = acc;
}

// H2[t][kz][x][y] = sum_ky H1[t][kz][ky][x] conj(exp(-2 pi i ky y / nny)); thread per output
// (used when the tiled version does not fit shared memory).
__global__ void k_yadj(DevArgs a, AdjArgs j) {
  const int ex = a.ext[0], ey = a.ext[1];
  const int64_t total = static_cast<int64_t>(a.T) * a.nkz * ex * ey;
  const int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= total) return;
  const int y = o % ey;
  const int x = (o / ey) % ex;
  const int64_t tk = o / (static_cast<int64_t>(ey) * ex);
  const float2 *h = j.H1 + tk * a.nky * ex + x;
  const float2 *w = a.twy + static_cast<size_t>(y) * a.nkyp;
  float2 acc = make_float2(0.f, 0.f);
  for (int ky = 0; ky < a.nky; ++ky) {
    const float2 v = h[static_cast<int64_t>(ky) * ex], c = w[ky];
    acc.x = fmaf(v.x, c.x, fmaf(v.y, c.y, acc.x));
    acc.y = fmaf(v.y, c.x, fmaf(-v.x, c.y, acc.y));
  }
  j.H2[o] = acc;
}

// grid (ceil(ex/64), nkz, T), block 256: the same contraction in shared-memory tiles.
// Thread: 2 x rows x 16 y values.  Dynamic smem: H1 tile nky x 64 | twyT nky x eyp (float2).
__global__ void __launch_bounds__(kThreads) k_yadj_tile(DevArgs a, AdjArgs j) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *h1 = reinterpret_cast<float2 *>(smem);
  float2 *tw = h1 + static_cast<size_t>(a.nky) * 64;
  const int t = blockIdx.z, kz = blockIdx.y, xb = blockIdx.x * 64;
  const int ex = a.ext[0], ey = a.ext[1];
  const int tid = threadIdx.x, lane = tid & 31, yg = tid >> 5;
  const float2 *src = j.H1 + (static_cast<int64_t>(t) * a.nkz + kz) * a.nky * ex;
  for (int i = tid; i < a.nky * 64; i += blockDim.x) {
    const int ky = i / 64, xl = i % 64;
    h1[i] = (xb + xl < ex) ? src[static_cast<int64_t>(ky) * ex + xb + xl] : make_float2(0.f, 0.f);
  }
  {
    const float4 *s4 = reinterpret_cast<const float4 *>(j.twyT);
    float4 *d4 = reinterpret_cast<float4 *>(tw);
    const int n4 = a.nky * j.eyp / 2;
    for (int i = tid; i < n4; i += blockDim.x) d4[i] = s4[i];
  }
  __syncthreads();
  float2 *dst = j.H2 + (static_cast<int64_t>(t) * a.nkz + kz) * ex * ey;
  const int x = xb + 2 * lane;
  for (int yb = yg * 16; yb < ey; yb += 128) {
    float2 acc0[16], acc1[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc0[q] = acc1[q] = make_float2(0.f, 0.f);
    for (int ky = 0; ky < a.nky; ++ky) {
      const float4 hv = *reinterpret_cast<const float4 *>(h1 + ky * 64 + 2 * lane);
      const float4 *w4 = reinterpret_cast<const float4 *>(tw + static_cast<size_t>(ky) * j.eyp + yb);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 w = w4[q];
        // h * conj(w): re = hr wr + hi wi, im = hi wr - hr wi
        acc0[2 * q].x = fmaf(hv.x, w.x, fmaf(hv.y, w.y, acc0[2 * q].x));
        acc0[2 * q].y = fmaf(hv.y, w.x, fmaf(-hv.x, w.y, acc0[2 * q].y));
        acc1[2 * q].x = fmaf(hv.z, w.x, fmaf(hv.w, w.y, acc1[2 * q].x));
        acc1[2 * q].y = fmaf(hv.w, w.x, fmaf(-hv.z, w.y, acc1[2 * q].y));
        acc0[2 * q + 1].x = fmaf(hv.x, w.z, fmaf(hv.y, w.w, acc0[2 * q + 1].x));
        acc0[2 * q + 1].y = fmaf(hv.y, w.z, fmaf(-hv.x, w.w, acc0[2 * q + 1].y));
        acc1[2 * q + 1].x = fmaf(hv.z, w.z, fmaf(hv.w, w.w, acc1[2 * q + 1].x));
        acc1[2 * q + 1].y = fmaf(hv.w, w.z, fmaf(-hv.z, w.w, acc1[2 * q + 1].y));
      }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int y = yb + q;
      if (y < ey) {
        if (x < ex) dst[static_cast<int64_t>(x) * ey + y] = acc0[q];
        if (x + 1 < ex) dst[static_cast<int64_t>(x + 1) * ey + y] = acc1[q];
      }
    }
  }
}

// dg[t][x][y][z] = Re sum_kz H2[t][kz][x][y] conj(exp(-2 pi i kz z / nnz)); thread per output
// (used when the fused tiled version does not fit shared memory).
__global__ void k_zadj(DevArgs a, AdjArgs j) {
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  const int64_t total = static_cast<int64_t>(a.T) * ex * ey * ez;
  const int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= total) return;
  const int z = o % ez;
  const int64_t col = o / ez;  // (t, x, y)
  const int64_t xy = col % (static_cast<int64_t>(ex) * ey);
  const int t = static_cast<int>(col / (static_cast<int64_t>(ex) * ey));
  const float2 *h = j.H2 + static_cast<int64_t>(t) * a.nkz * ex * ey + xy;
  const float2 *w = a.twz + static_cast<size_t>(z) * a.nkzp;
  float acc = 0.f;
  for (int kz = 0; kz < a.nkz; ++kz) {
    const float2 v = h[static_cast<int64_t>(kz) * ex * ey], c = w[kz];
    acc = fmaf(v.x, c.x, fmaf(v.y, c.y, acc));
  }
  j.dg[o] = acc;
}

// grid (blocks, T), block 256: S_t = sum of dg_t over the corner block (FP64).
__global__ void __launch_bounds__(kThreads) k_sum_dg(DevArgs a, AdjArgs j) {
  __shared__ double red[kThreads / 32];
  const int t = blockIdx.y;
  const int64_t per = static_cast<int64_t>(a.ext[0]) * a.ext[1] * a.ext[2];
  const float *d = j.dg + t * per;
  double s = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < per;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += d[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) tot += red[w];
    atomicAdd(j.S + t, tot);
  }
}

// One thread per entry: B-spline derivative gather of dL/dg, then dL/dx.
__global__ void __launch_bounds__(kThreads) k_gather(DevArgs a, AdjArgs j) {
  __shared__ float oc[9];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (threadIdx.x < 9) oc[threadIdx.x] = a.geom[threadIdx.x];
  __syncthreads();
  if (e >= a.M) return;
  const int at = a.entry_atom[e];
  const int t = a.entry_type[e];
  const float *p = a.xyz + 3ll * at;
  const float x0 = p[0], y0 = p[1], z0 = p[2];
  float r[3], w[3][4], dw[3][4];
  int m[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r[d] = grid_coord(oc + 3 * d, x0, y0, z0, a.n[d]);
    m[d] = static_cast<int>(r[d]);
    const float u = r[d] - static_cast<float>(m[d]);
    cubic_weights(u, w[d]);
    const float v = 1.0f - u;
    dw[d][0] = -0.5f * v * v;
    dw[d][1] = 1.5f * u * u - 2.0f * u;
    dw[d][2] = -1.5f * u * u + u + 0.5f;
    dw[d][3] = 0.5f * u * u;
  }
  const int P = a.order, nt = a.ntaps;
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  const float *dgt = j.dg + static_cast<int64_t>(t) * ex * ey * ez;
  float gr[3] = {0.f, 0.f, 0.f};
  // taps on the corner block
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    if (o >= nt) break;
    int x = m[0] - P + o;
    if (x < 0) x += a.n[0];
    if (x >= ex) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q >= nt) break;
      int y = m[1] - P + q;
      if (y < 0) y += a.n[1];
      if (y >= ey) continue;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        if (s >= nt) break;
        int z = m[2] - P + s;
        if (z < 0) z += a.n[2];
        if (z >= ez) continue;
        const float v = dgt[(static_cast<int64_t>(x) * ey + y) * ez + z];
        gr[0] = fmaf(v, dw[0][o] * w[1][q] * w[2][s], gr[0]);
        gr[1] = fmaf(v, w[0][o] * dw[1][q] * w[2][s], gr[1]);
        gr[2] = fmaf(v, w[0][o] * w[1][q] * dw[2][s], gr[2]);
      }
    }
  }
  // the border mean: every border voxel carries (nn^3 Re G(0) - S_t) / count
  // (a given padding does not depend on the positions)
  const float cm = a.pad_val ? 0.0f
                             : static_cast<float>((static_cast<double>(j.dcg[t]) - j.S[t]) / a.border_count);
  float sx = 0.f, sy = 0.f, szb = 0.f, dsx = 0.f, dsy = 0.f, dszb = 0.f;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    if (o < nt) {
      sx += w[0][o];
      sy += w[1][o];
      dsx += dw[0][o];
      dsy += dw[1][o];
      int z = m[2] - P + o;
      if (z < 0) z += a.n[2];
      if (z <= a.dz || z >= a.n[2] - a.dz) {
        szb += w[2][o];
        dszb += dw[2][o];
      }
    }
  }
  gr[0] = fmaf(cm, dsx * sy * szb, gr[0]);
  gr[1] = fmaf(cm, sx * dsy * szb, gr[1]);
  gr[2] = fmaf(cm, sx * sy * dszb, gr[2]);
  // r_d = n_d * (oc_d . x) + const
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float g = gr[0] * a.n[0] * oc[c] + gr[1] * a.n[1] * oc[3 + c] + gr[2] * a.n[2] * oc[6 + c];
    atomicAdd(j.grad + 3ll * at + c, g);
  }
}

__device__ __forceinline__ void spline_and_derivative(float u, float w[4], float dw[4]) {
  cubic_weights(u, w);
  const float v = 1.0f - u;
  dw[0] = -0.5f * v * v;
  dw[1] = 1.5f * u * u - 2.0f * u;
  dw[2] = -1.5f * u * u + u + 0.5f;
  dw[3] = 0.5f * u * u;
}

// dL/dr (grid units) -> dL/dxyz of the atom: r_d = n_d (oc_d . x) + const.
__device__ __forceinline__ void add_position_gradient(const DevArgs &a, const float *oc,
                                                      const float gr[3], float *g) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float v = gr[0] * a.n[0] * oc[c] + gr[1] * a.n[1] * oc[3 + c] + gr[2] * a.n[2] * oc[6 + c];
    atomicAdd(g + c, v);
  }
}

// Persistent over (type, 8x8 column tile) of frame 0; block 256.  The z-axis
// adjoint of the tile's 64 columns into shared memory (a small GEMM: 4 columns x
// 8 z per thread), its sum into S_t, then the B-spline derivative gather of every
// atom whose stencil reaches the tile.  Dynamic smem:
//   twzT nkz x ezp float2 | H2 columns nkz x 64 float2 | dg tile ez x 64 float.
__global__ void __launch_bounds__(kThreads) k_zadj_gather(DevArgs a, AdjArgs j, int items) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  float2 *tw = reinterpret_cast<float2 *>(smem);
  float2 *hz = tw + static_cast<size_t>(a.nkz) * j.ezp;
  float *dgt = reinterpret_cast<float *>(hz + static_cast<size_t>(a.nkz) * kCols);
  __shared__ TileAtoms ta;
  __shared__ float oc[9];
  __shared__ double red[kThreads / 32];
  const int tid = threadIdx.x;
  {
    const float4 *s4 = reinterpret_cast<const float4 *>(j.twzT);
    float4 *d4 = reinterpret_cast<float4 *>(tw);
    const int n4 = a.nkz * j.ezp / 2;
    for (int i = tid; i < n4; i += blockDim.x) d4[i] = s4[i];
  }
  if (tid < 9) oc[tid] = a.geom[tid];
  const int st = a.stiles[0] * a.stiles[1];
  const int cg = tid % 16, zg = tid / 16;
  const float4 *hz4 = reinterpret_cast<const float4 *>(hz);
  const float4 *tw4 = reinterpret_cast<const float4 *>(tw);
  const float4 *rec = a.rec;
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  for (int w = blockIdx.x; w < items; w += gridDim.x) {
    const int t = w / st, tl = w % st;
    const int x0 = (tl % a.stiles[0]) * kTile, y0 = (tl / a.stiles[0]) * kTile;
    const int cw = min(kTile, ex - x0), ch = min(kTile, ey - y0);
    const float2 *src = j.H2 + static_cast<int64_t>(t) * a.nkz * ex * ey;
    for (int i = tid; i < a.nkz * kCols; i += blockDim.x) {
      const int kz = i / kCols, col = i % kCols, lx = col / kTile, ly = col % kTile;
      hz[i] = (lx < cw && ly < ch)
                  ? src[(static_cast<int64_t>(kz) * ex + x0 + lx) * ey + y0 + ly]
                  : make_float2(0.f, 0.f);
    }
    tile_atom_ranges(a, ta, 0, t, x0, y0);
    __syncthreads();
    double part = 0.0;
    for (int zb = zg * 8; zb < ez; zb += 128) {
      float acc[4][8];
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[c][q] = 0.f;
      for (int kz = 0; kz < a.nkz; ++kz) {
        const float4 h01 = hz4[kz * (kCols / 2) + 2 * cg];
        const float4 h23 = hz4[kz * (kCols / 2) + 2 * cg + 1];
        const float hr[4] = {h01.x, h01.z, h23.x, h23.z};
        const float hi[4] = {h01.y, h01.w, h23.y, h23.w};
        const float4 *w4 = tw4 + (static_cast<size_t>(kz) * j.ezp + zb) / 2;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 wv = w4[q];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            acc[c][2 * q] = fmaf(hr[c], wv.x, fmaf(hi[c], wv.y, acc[c][2 * q]));
            acc[c][2 * q + 1] = fmaf(hr[c], wv.z, fmaf(hi[c], wv.w, acc[c][2 * q + 1]));
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int z = zb + q;
        if (z < ez) {
          *reinterpret_cast<float4 *>(dgt + z * kCols + 4 * cg) =
              make_float4(acc[0][q], acc[1][q], acc[2][q], acc[3][q]);
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int col = 4 * cg + c;
            if ((col / kTile) < cw && (col % kTile) < ch) part += acc[c][q];
          }
        }
      }
    }
    part = warp_sum(part);
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double tot = 0.0;
      for (int q = 0; q < kThreads / 32; ++q) tot += red[q];
      if (tot != 0.0) atomicAdd(j.S + t, tot);
    }
    // gather dL/dg' at the taps of every atom whose stencil reaches this tile
    const int total = ta.cum[ta.nb];
    for (int k = tid; k < total; k += blockDim.x) {
      int jb = 0;
      while (k >= ta.cum[jb + 1]) ++jb;
      const float4 q = rec[ta.start[jb] + (k - ta.cum[jb])];
      const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y), m2 = static_cast<int>(q.z);
      float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
      spline_and_derivative(q.x - static_cast<float>(m0), wx, dx);
      spline_and_derivative(q.y - static_cast<float>(m1), wy, dy);
      spline_and_derivative(q.z - static_cast<float>(m2), wz, dz);
      float gr[3] = {0.f, 0.f, 0.f};
      bool hit = false;
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (o >= nt) break;
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        const int lx = x - x0;
        if (static_cast<unsigned>(lx) >= static_cast<unsigned>(cw)) continue;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          if (p >= nt) break;
          int y = m1 - P + p;
          if (y < 0) y += a.n[1];
          const int ly = y - y0;
          if (static_cast<unsigned>(ly) >= static_cast<unsigned>(ch)) continue;
          const float *colp = dgt + lx * kTile + ly;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (r >= nt) break;
            int z = m2 - P + r;
            if (z < 0) z += nz;
            if (z >= ez) continue;
            const float v = colp[z * kCols];
            gr[0] = fmaf(v, dx[o] * wy[p] * wz[r], gr[0]);
            gr[1] = fmaf(v, wx[o] * dy[p] * wz[r], gr[1]);
            gr[2] = fmaf(v, wx[o] * wy[p] * dz[r], gr[2]);
            hit = true;
          }
        }
      }
      if (hit) {
        const int e = __float_as_int(q.w);
        add_position_gradient(a, oc, gr, j.grad + 3ll * a.entry_atom[e]);
      }
    }
    __syncthreads();
  }
}

// One thread per sorted record of frame 0: the border-mean part of dL/dx,
// (nn^3 Re G_t(0) - S_t) / count per border voxel.
__global__ void __launch_bounds__(kThreads) k_mean_grad(DevArgs a, AdjArgs j) {
  __shared__ float oc[9];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (threadIdx.x < 9) oc[threadIdx.x] = a.geom[threadIdx.x];
  __syncthreads();
  if (i >= a.M) return;
  const float4 q = a.rec[i];
  const int e = __float_as_int(q.w);
  const int t = a.entry_type[e];
  const float cm = a.pad_val ? 0.0f
                             : static_cast<float>((static_cast<double>(j.dcg[t]) - j.S[t]) / a.border_count);
  if (cm == 0.0f) return;
  const int m[3] = {static_cast<int>(q.x), static_cast<int>(q.y), static_cast<int>(q.z)};
  float w[3][4], dw[3][4];
  spline_and_derivative(q.x - static_cast<float>(m[0]), w[0], dw[0]);
  spline_and_derivative(q.y - static_cast<float>(m[1]), w[1], dw[1]);
  spline_and_derivative(q.z - static_cast<float>(m[2]), w[2], dw[2]);
  float sx = 0.f, sy = 0.f, szb = 0.f, dsx = 0.f, dsy = 0.f, dszb = 0.f;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    if (o < a.ntaps) {
      sx += w[0][o];
      sy += w[1][o];
      dsx += dw[0][o];
      dsy += dw[1][o];
      int z = m[2] - a.order + o;
      if (z < 0) z += a.n[2];
      if (z <= a.dz || z >= a.n[2] - a.dz) {
        szb += w[2][o];
        dszb += dw[2][o];
      }
    }
  }
  const float gr[3] = {cm * dsx * sy * szb, cm * sx * dsy * szb, cm * sx * sy * dszb};
  add_position_gradient(a, oc, gr, j.grad + 3ll * a.entry_atom[e]);
}

// grid (ceil(points/256)), block 256: nvt intensity sum over the batch's frames.
__global__ void k_accumulate(DevArgs a, int nframes) {
  const int64_t npl = static_cast<int64_t>(a.nkz) * a.nky * a.nkx;
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npl) return;
  double s = a.iacc[p];
  for (int f = 0; f < nframes; ++f) s += static_cast<double>(a.ibox[f * npl + p]);
  a.iacc[p] = s;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Ring {
  float *host = nullptr;
  cudaEvent_t ev[kRing] = {};
  int next = 0;
};

// Timed stages of saxs_forward, in launch order.
enum Stage { kStSort, kStSpread, kStYdft, kStXdft, kStHist, kStages };
const char *kStageNames[kStages] = {"k_sort_atoms", "k_spread_zdft", "k_ydft", "k_xdft_post", "k_hist"};

struct StageRecord {
  cudaEvent_t start[kStages] = {};
  cudaEvent_t stop[kStages] = {};
  bool used[kStages] = {};
};

}  // namespace

struct SaxsPlan {
  int device = 0;
  SaxsParams p{};
  std::vector<float> ff;
  std::vector<float> pad;  // given padding densities per type (empty: z-border mean)
  DevArgs a{};
  int ensemble = SAXS_NPT;
  long long half[3] = {0, 0, 0};
  bool full_axis[3] = {false, false, false};
  float sigma_scale = 1.0f;  // nx / nnx
  int frames = 0;            // frames accumulated
  int last_frame_batch = 0;  // frames in the last forward batch
  size_t bytes = 0;
  size_t smem_spread = 0, smem_ydft = 0, smem_xdft = 0, smem_hist = 0;
  std::vector<void *> allocations;
  Ring ring;
  float *d_geom0 = nullptr;
  double *d_tmp_hist = nullptr;
  // adjoint buffers, allocated by the first saxs_backward
  double *d_adj_dl = nullptr, *d_adj_S = nullptr;
  float2 *d_adj_G = nullptr, *d_adj_twyT = nullptr, *d_adj_twzT = nullptr;
  float *d_adj_dg = nullptr, *d_adj_dcg = nullptr;
  int adj_eyp = 0, adj_ezp = 0, zadj_ctas = 1;
  bool adj_tiled_y = false, adj_tiled_z = false;
  size_t smem_yadj = 0, smem_zadj = 0;
  int spread_ctas = 1;  // resident CTAs of the persistent spreading kernel
  int sort_slots = 1;    // resident k_sort_atoms CTAs on the device
  int sort_max_type = 0; // entries of the largest type
  bool use_tc = false;   // z-axis DFT on the tensor cores
  bool use_tcw = false;  // ... with the wide-tile kernel (k_spread_zdft_tcw), else k_spread_zdft_tc
  size_t smem_spread_tc = 0, smem_spread_tcw = 0;
  int tc_ctas = 1, tcw_ctas = 1;
  bool tcn_ok = false, tcw_ok = false;  // z kernels the plan can run: 64- and 128-column tiles
  int twG_max = 1;                      // producer groups the wide kernel's shared memory allows
  int tw_cap[2] = {0, 0}, tw_rb[2] = {0, 0};  // wide kernel atom table / record buffer, 1 or 2 groups
  size_t tw_smem[2] = {0, 0};
  bool tc_ok = false, ytc_ok = false, xtc_ok = false;  // tensor-core kernels the plan can run
  bool use_ytc = false;  // y-axis DFT on the tensor cores (k_dft_tc<false>)
  bool use_xtc = false;  // x-axis DFT + post on the tensor cores (k_dft_tc<true>)
  DtcShape yshape{}, xshape{};
  size_t smem_ydft_tc = 0, smem_xdft_tc = 0;
  int ytc_ctas = 1, xtc_ctas = 1;
  int xc = 1;           // x values per shared-memory chunk in k_xdft_post
  bool profiling = false;
  std::vector<StageRecord> prof_pending;
  std::vector<cudaEvent_t> event_pool;
};

namespace {

// The wide kernel's producer groups with the table sizes planned for them.
void set_wide_groups(SaxsPlan *pl, int g) {
  pl->a.twG = g;
  pl->a.twCap = pl->tw_cap[g - 1];
  pl->a.twRB = pl->tw_rb[g - 1];
  pl->smem_spread_tcw = pl->tw_smem[g - 1];
}

int optin_smem() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return 48 * 1024;
  }
  return v;
}

template <typename K>
size_t static_smem(K kernel) {
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1024;
  }
  return fa.sharedSizeBytes;
}

template <typename K>
cudaError_t raise_smem_limit(K kernel) {
  const int lim = optin_smem() - static_cast<int>(static_smem(kernel));
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

template <typename T>
int dalloc(SaxsPlan *pl, T **ptr, size_t count) {
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(ptr), bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    return fail(SAXS_E_NOMEM, "device allocation of " + std::to_string(bytes) +
                                  " bytes failed (" + cudaGetErrorString(e) + "; free " +
                                  std::to_string(fr) + " of " + std::to_string(tot) + ")");
  }
  pl->allocations.push_back(*ptr);
  pl->bytes += bytes;
  return SAXS_OK;
}

// Distinct home bins (width bin_w) whose atoms can reach the columns
// [c0, c0+cw) of each spread tile along an axis of length n, for stencils of
// `order` taps that start at an atom's home column.  Returns false when a tile
// would need more than four bins.
bool home_tile_table(int ext, int n, int order, int bin_w, std::vector<int4> *out) {
  out->clear();
  for (int c0 = 0; c0 < ext; c0 += kTile) {
    const int cw = std::min(kTile, ext - c0);
    int h[4] = {-1, -1, -1, -1}, cnt = 0;
    for (int d = 0; d < cw + order - 1; ++d) {
      int x = (c0 - order + 1 + d) % n;
      if (x < 0) x += n;
      const int t = x / bin_w;
      bool seen = false;
      for (int k = 0; k < cnt; ++k) seen |= (h[k] == t);
      if (!seen) {
        if (cnt == 4) return false;
        h[cnt++] = t;
      }
    }
    out->push_back(make_int4(h[0], h[1], h[2], h[3]));
  }
  return true;
}

// The same for the 16-row y tiles of k_spread_zdft_tcw: up to eight bins per
// tile, two int4 each.  Returns false when a tile would need more.
bool home_tile_table_w(int ext, int n, int order, int bin_w, std::vector<int4> *out) {
  out->clear();
  for (int c0 = 0; c0 < ext; c0 += kTwY) {
    const int cw = std::min(kTwY, ext - c0);
    int h[8] = {-1, -1, -1, -1, -1, -1, -1, -1}, cnt = 0;
    for (int d = 0; d < cw + order - 1; ++d) {
      int x = (c0 - order + 1 + d) % n;
      if (x < 0) x += n;
      const int t = x / bin_w;
      bool seen = false;
      for (int k = 0; k < cnt; ++k) seen |= (h[k] == t);
      if (!seen) {
        if (cnt == 8) return false;
        h[cnt++] = t;
      }
    }
    out->push_back(make_int4(h[0], h[1], h[2], h[3]));
    out->push_back(make_int4(h[4], h[5], h[6], h[7]));
  }
  return true;
}

// Per-frame geometry: g[0..9) = oc, the map from Cartesian to fractional
// coordinates (rows); g[9..18) = the map from k indices to q / 2pi used by the
// k-point code (rows).  Reference parity: oc from the box's upper triangle and
// q rows = sigma' oc.  Triclinic mode: oc = H^-T and q = 2 pi (sigma' oc)^T m,
// so the q rows are the transpose.
void frame_geometry(const SaxsPlan *pl, const float box[9], float g[kGeom]) {
  float oc[9];
  if (pl->p.box_mode == SAXS_BOX_TRICLINIC)
    saxs::cell_oc_triclinic(box, oc);
  else
    saxs::cell_oc(box, oc);
  const bool tr = pl->p.box_mode == SAXS_BOX_TRICLINIC;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      g[3 * r + c] = oc[3 * r + c];
      g[9 + 3 * r + c] = pl->sigma_scale * (tr ? oc[3 * c + r] : oc[3 * r + c]);
    }
  for (int i = 18; i < kGeom; ++i) g[i] = 0.0f;
}

int check_box(const float box[9]) {
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(box[i])) return fail(SAXS_E_INVALID, "box contains a non-finite value");
  if (!(box[0] > 0.f) || !(box[4] > 0.f) || !(box[8] > 0.f))
    return fail(SAXS_E_INVALID, "box diagonal must be positive");
  return SAXS_OK;
}

void destroy(SaxsPlan *pl) {
  if (!pl) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(pl->device);
  for (void *p : pl->allocations) cudaFree(p);
  for (int i = 0; i < kRing; ++i)
    if (pl->ring.ev[i]) cudaEventDestroy(pl->ring.ev[i]);
  for (auto &r : pl->prof_pending)
    for (int k = 0; k < kStages; ++k) {
      if (r.start[k]) cudaEventDestroy(r.start[k]);
      if (r.stop[k]) cudaEventDestroy(r.stop[k]);
    }
  for (cudaEvent_t e : pl->event_pool) cudaEventDestroy(e);
  if (pl->ring.host) cudaFreeHost(pl->ring.host);
  cudaSetDevice(prev);
  delete pl;
}

// GEMM shape of a tensor-core DFT pass over `extent` values of u to `nk` values
// of k: N' = 2*nk padded to 16 (at most 256), two to four K-chunk stages in
// `avail` bytes of shared memory.  Returns false when the pass does not fit.
bool dtc_shape(int nk, int extent, size_t avail, DtcShape *sh, size_t *smem, bool allow_lo_smem) {
  const int N = round_up(2 * nk, 16);
  const size_t stage_bytes = (128 + 2 * static_cast<size_t>(N)) * 2 * kDtcChunk * sizeof(float);
  const int S_smem = static_cast<int>((avail - 1024) / stage_bytes);
  // tensor memory: two accumulators of N' columns and 64 columns of A per stage;
  // with the A remainder in shared memory (2N' <= 256): two accumulators of 2N'
  // columns and 32 columns per stage.  PYCUSAXS_DTC=split keeps the first form.
  // Measured on the 100k-atom workload: the y pass 0.60 ms per 100 frames with
  // the remainder in shared memory against 0.65 ms; the x pass, whose epilogue
  // then reads twice the accumulator columns, 0.34 against 0.33 ms, so it keeps
  // the first form.
  const char *mode = std::getenv("PYCUSAXS_DTC");
  int S = std::min({kDtcMaxStages, S_smem, (512 - 2 * N) / 64});
  sh->lo_smem = 0;
  if (allow_lo_smem && !(mode && std::strcmp(mode, "split") == 0) && 2 * N <= 256) {
    const int Sl = std::min({kDtcMaxStages, S_smem, (512 - 4 * N) / 32});
    if (Sl >= 2) {
      sh->lo_smem = 1;
      S = Sl;
    }
  }
  if (N > 256 || S < 2) return false;
  sh->N = N;
  sh->chunks = (extent + kDtcChunk - 1) / kDtcChunk;
  sh->S = S;
  sh->cols = 512;
  *smem = S * stage_bytes + 1024;  // + alignment slack of the stage base
  return true;
}

// B' operand of a tensor-core DFT pass from twiddles tw[u * stride + k] (u <
// extent, k < nk): per K chunk a head block then a remainder block, each N' x
// 2*kDtcChunk K-major, B'[2u + c][2k + d] = {Wr, Wi ; -Wi, Wr}[c][d].
std::vector<float> dtc_bprime(const std::vector<float2> &tw, int stride, int extent, int nk,
                              const DtcShape &sh) {
  const int KP = 2 * kDtcChunk, Np = sh.N;
  const size_t blk = static_cast<size_t>(Np) * KP;
  std::vector<float> out(static_cast<size_t>(sh.chunks) * 2 * blk, 0.0f);
  // element (n', k') of the head (part 0) or remainder (part 1) of chunk c: two
  // N'-column blocks, or one 2N'-column block with the parts side by side
  auto at = [&](int c, int part, int np, int kp) {
    const int n2 = sh.lo_smem ? np + part * Np : np, N2 = sh.lo_smem ? 2 * Np : Np;
    const size_t off = static_cast<size_t>(c) * 2 * blk + (sh.lo_smem ? 0 : part * blk);
    return off + static_cast<size_t>(kp / 4) * (N2 / 8) * 32 + (n2 / 8) * 32 + (n2 % 8) * 4 + kp % 4;
  };
  for (int c = 0; c < sh.chunks; ++c)
    for (int uu = 0; uu < kDtcChunk; ++uu) {
      const int u = c * kDtcChunk + uu;
      if (u >= extent) continue;
      for (int k = 0; k < nk; ++k) {
        const float2 w = tw[static_cast<size_t>(u) * stride + k];
        const float vals[2][2] = {{w.x, w.y}, {-w.y, w.x}};
        for (int cz = 0; cz < 2; ++cz)
          for (int d = 0; d < 2; ++d) {
            const int kp = 2 * uu + cz, np = 2 * k + d;
            const float v = vals[cz][d];
            uint32_t bits;
            std::memcpy(&bits, &v, sizeof(bits));
            bits &= 0xFFFFE000u;
            float head;
            std::memcpy(&head, &bits, sizeof(head));
            out[at(c, 0, np, kp)] = head;
            out[at(c, 1, np, kp)] = v - head;
          }
      }
    }
  return out;
}

int create(const SaxsParams *prm, SaxsPlan **out) {
  if (!prm || !out) return fail(SAXS_E_INVALID, "null argument");
  *out = nullptr;
  const SaxsParams &p = *prm;
  for (int d = 0; d < 3; ++d)
    if (p.grid[d] <= 0) return fail(SAXS_E_INVALID, "Grid dimensions must be positive");
  if (p.order < 1 || p.order > 8)
    return fail(SAXS_E_INVALID, "Spline order must be between 1 and 8");
  if (p.ntypes < 1 || !p.form_factors) return fail(SAXS_E_INVALID, "at least one atom type is required");
  if (p.natoms < 0 || p.nentries < 0) return fail(SAXS_E_INVALID, "negative atom count");
  if (p.nentries > 0 && (!p.entry_atom || !p.entry_type))
    return fail(SAXS_E_INVALID, "atom lists missing");
  if (p.max_frames < 1) return fail(SAXS_E_INVALID, "max_frames must be >= 1");
  if (p.ensemble != SAXS_NPT && p.ensemble != SAXS_NVT)
    return fail(SAXS_E_INVALID, "ensemble must be npt or nvt");
  if (int rc = check_box(p.box0)) return rc;
  if (p.box_mode != SAXS_BOX_PARITY && p.box_mode != SAXS_BOX_TRICLINIC)
    return fail(SAXS_E_INVALID, "box_mode must be parity (0) or triclinic (1)");
  if (p.padding_mode != SAXS_PAD_AVERAGE && p.padding_mode != SAXS_PAD_GIVEN)
    return fail(SAXS_E_INVALID, "padding_mode must be average (0) or given (1)");
  if (p.padding_mode == SAXS_PAD_GIVEN) {
    if (!p.padding_values) return fail(SAXS_E_INVALID, "given padding needs padding_values");
    for (int t = 0; t < p.ntypes; ++t)
      if (!std::isfinite(p.padding_values[t]) || p.padding_values[t] < 0.0f)
        return fail(SAXS_E_INVALID, "padding values must be finite and non-negative");
  }
  for (int i = 0; i < p.nentries; ++i) {
    if (p.entry_atom[i] < 0 || p.entry_atom[i] >= p.natoms)
      return fail(SAXS_E_INVALID, "atom index " + std::to_string(p.entry_atom[i]) +
                                      " out of range [0, " + std::to_string(p.natoms) + ")");
    if (p.entry_type[i] < 0 || p.entry_type[i] >= p.ntypes)
      return fail(SAXS_E_INVALID, "type index out of range");
  }
  const bool scaled = p.scaled_grid[0] > 0 || p.scaled_grid[1] > 0 || p.scaled_grid[2] > 0;
  int nn[3];
  for (int d = 0; d < 3; ++d) {
    if (scaled) {
      if (p.scaled_grid[d] <= 0) return fail(SAXS_E_INVALID, "Scaled grid dimensions must be positive");
      nn[d] = p.scaled_grid[d];
    } else {
      if (!(p.scale_factor > 0.0f))
        return fail(SAXS_E_INVALID, "Scale factor must be positive when scaled grid is not provided");
      const long long v = saxs::closest_product(p.grid[d], p.scale_factor);
      if (v < 1 || v > (1 << 20)) return fail(SAXS_E_INVALID, "scaled grid out of range");
      nn[d] = static_cast<int>(v);
    }
  }
  const int ntaps = std::min(p.order, 4);
  for (int d = 0; d < 3; ++d) {
    if (p.grid[d] < p.order)
      return fail(SAXS_E_INVALID, "grid dimension smaller than the spline order");
    if (nn[d] < 2) return fail(SAXS_E_INVALID, "scaled grid dimension must be >= 2");
  }

  SaxsPlan *pl = new SaxsPlan();
  cudaGetDevice(&pl->device);
  pl->p = p;
  if (p.padding_mode == SAXS_PAD_GIVEN) pl->pad.assign(p.padding_values, p.padding_values + p.ntypes);
  pl->p.padding_values = nullptr;  // the caller's array is not kept
  pl->ensemble = p.ensemble;
  pl->ff.assign(p.form_factors, p.form_factors + 9 * p.ntypes);
  DevArgs &a = pl->a;
  for (int d = 0; d < 3; ++d) {
    a.n[d] = p.grid[d];
    a.nn[d] = nn[d];
    a.ext[d] = std::min(p.grid[d], nn[d]);
    a.nf[d] = saxs::nf_of(nn[d]);
  }
  a.order = p.order;
  a.ntaps = ntaps;
  a.T = p.ntypes;
  a.M = p.nentries;
  // home bins 4 columns wide cut the atoms an item visits without reaching its
  // tile (about half with 8-wide bins, a sixth with 4-wide ones)
  std::vector<int4> hxt, hyt;
  a.bin_w = 4;
  if (!home_tile_table(a.ext[0], a.n[0], a.order, 4, &hxt) ||
      !home_tile_table(a.ext[1], a.n[1], a.order, 4, &hyt)) {
    a.bin_w = 8;
    if (!home_tile_table(a.ext[0], a.n[0], a.order, 8, &hxt) ||
        !home_tile_table(a.ext[1], a.n[1], a.order, 8, &hyt)) {
      destroy(pl);
      return fail(SAXS_E_INVALID, "spline order too large for the spread tiles");
    }
  }
  a.tiles[0] = (a.n[0] + a.bin_w - 1) / a.bin_w;
  a.tiles[1] = (a.n[1] + a.bin_w - 1) / a.bin_w;
  a.stiles[0] = (a.ext[0] + kTile - 1) / kTile;
  a.stiles[1] = (a.ext[1] + kTile - 1) / kTile;
  std::vector<int4> hywt;
  a.stw = home_tile_table_w(a.ext[1], a.n[1], a.order, a.bin_w, &hywt) ? (a.ext[1] + kTwY - 1) / kTwY : 0;
  a.nbins = a.T * a.tiles[0] * a.tiles[1];
  a.dz = static_cast<int>(0.07f * a.n[2] / 2);  // borderBins (saxsKernel.h:107-110)
  {
    int planes = 0;
    for (int z = 0; z < a.n[2]; ++z)
      if (!(z > a.dz && z < a.n[2] - a.dz)) ++planes;
    a.border_count = static_cast<double>(a.n[0]) * a.n[1] * planes;
  }
  a.nn3 = static_cast<double>(nn[0]) * nn[1] * nn[2];

  pl->sigma_scale = static_cast<float>(a.n[0]) / static_cast<float>(nn[0]);
  float geo0[kGeom];
  frame_geometry(pl, p.box0, geo0);
  float oc0[9], ocs0[9];
  for (int i = 0; i < 9; ++i) {
    oc0[i] = geo0[i];
    ocs0[i] = geo0[9 + i];
  }
  saxs::histogram_parameters(nn, oc0, p.scale_factor, p.bin_size, p.qcut, &a.dq, &a.qcut,
                             &a.num_bins);
  if (a.num_bins < 1) a.num_bins = 1;

  // k-box: every integer k with |2 pi ocs k| <= qcut for the first frame and
  // for boxes up to `box_margin` smaller.
  const double margin = std::max(0.0f, p.box_margin) + 1e-5;
  saxs::kbox_halfwidths(ocs0, a.qcut, margin, pl->half);
  for (int d = 0; d < 2; ++d) {
    const long long hmax = a.nf[d] - 1;
    if (pl->half[d] >= hmax) {
      pl->full_axis[d] = true;
      pl->half[d] = hmax;
    }
  }
  a.kx_lo = pl->full_axis[0] ? a.nf[0] - nn[0] : -static_cast<int>(pl->half[0]);
  a.nkx = pl->full_axis[0] ? nn[0] : 2 * static_cast<int>(pl->half[0]) + 1;
  a.ky_lo = pl->full_axis[1] ? a.nf[1] - nn[1] : -static_cast<int>(pl->half[1]);
  a.nky = pl->full_axis[1] ? nn[1] : 2 * static_cast<int>(pl->half[1]) + 1;
  if (pl->half[2] >= nn[2] / 2) {
    pl->full_axis[2] = true;
    pl->half[2] = nn[2] / 2;
  }
  a.nkz = static_cast<int>(pl->half[2]) + 1;
  a.nkzp = round_up(a.nkz, kKzThread);
  a.nkxp = round_up(a.nkx, 2);
  a.nkyp = round_up(a.nky, kKyGroup);

  // shared-memory budgets (rows of twiddles / x chunks shrink to fit)
  const size_t optin = static_cast<size_t>(optin_smem());
  {
    const size_t NP = 2 * static_cast<size_t>(a.nkzp);
    const size_t tile = std::max<size_t>(static_cast<size_t>(a.n[2]) * kCols, kCols * NP) * sizeof(float);
    const size_t avail = optin - static_smem(k_spread_zdft);
    size_t zc = a.ext[2];
    while (zc > 8 && zc * NP * sizeof(float) + tile > avail) zc = (zc > 16) ? zc / 2 : 8;
    a.zc = static_cast<int>(zc);
    pl->smem_spread = zc * NP * sizeof(float) + tile;
  }
  pl->smem_ydft = static_cast<size_t>(kYChunk) * kYStride * sizeof(float2) +
                  static_cast<size_t>(kYChunk) * a.nkyp * sizeof(float2);
  {
    const size_t avail = optin - static_smem(k_xdft_post);
    const size_t fixed = static_cast<size_t>(a.T) * a.nkxp * sizeof(float2);
    const size_t per_x = (static_cast<size_t>(a.nkxp) + a.T) * sizeof(float2);
    size_t xc = a.ext[0];
    if (fixed + xc * per_x > avail) xc = avail > fixed + 2 * per_x ? (avail - fixed) / per_x : 2;
    xc = std::max<size_t>(2, xc & ~static_cast<size_t>(1));
    pl->xc = static_cast<int>(std::min<size_t>(xc, a.ext[0]));
    pl->smem_xdft = fixed + static_cast<size_t>(pl->xc) * per_x;
  }
  {
    // tensor-core z-DFT: N = 2*nkz padded to 8 (<= 256; to 16 and <= 128 for wide tiles),
    // K = ez padded to 8, two operand stages when they fit, else one.
    // PYCUSAXS_ZDFT=simt keeps the FP32 SIMT kernel, PYCUSAXS_ZDFT=narrow the
    // 64-column tensor-core kernel.
    const char *mode = std::getenv("PYCUSAXS_ZDFT");
    const bool simt_only = mode && std::strcmp(mode, "simt") == 0;
    const bool narrow_only = mode && std::strcmp(mode, "narrow") == 0;
    const int N = round_up(2 * a.nkz, 8);
    const int NW = round_up(2 * a.nkz, 16);  // M = 128 needs N a multiple of 16
    const int KT = round_up(a.ext[2], 16);  // K = 16 per f16 MMA of the wide kernel
    const int R = std::max(KT, round_up(a.n[2], 8));
    const size_t avail = optin - static_smem(k_spread_zdft_tc);
    const size_t b_bytes = 2 * static_cast<size_t>(KT) * N * sizeof(float);
    const size_t stage_bytes = static_cast<size_t>(R + KT) * 64 * sizeof(float);
    const size_t home_bytes = static_cast<size_t>(a.stiles[0] + a.stiles[1]) * sizeof(int4);
    // two operand stages before larger record buffers before a larger atom
    // table; records beyond the staging buffer are read from global memory,
    // atoms beyond the table are spread in further chunks
    // (one atom table per producer group: two groups with two stages)
    int S = 0, RB = 0, CAP = 0;
    for (int s_try = 2; s_try >= 1 && S == 0; --s_try)
      for (int cap = 256; cap >= 64 && S == 0; cap /= 2)
        for (int rb = 1024; rb >= 128 && S == 0; rb /= 2)
          if (b_bytes + s_try * stage_bytes + 2 * static_cast<size_t>(rb) * 16 + home_bytes +
                  static_cast<size_t>(s_try) * cap * kTcAtomBytes <= avail) {
            S = s_try;
            RB = rb;
            CAP = cap;
          }
    // wide tiles, for one and for two producer groups: twG fixed-point tiles of
    // 128 x (R + 4) words, then the largest atom table (each table chunk costs a
    // latency-bound pre-pass and two barriers), then the largest record buffer
    // that fit beside them
    const int RSW = R + 4;
    const size_t home_w = static_cast<size_t>(a.stiles[0] + 2 * a.stw) * sizeof(int4);
    const size_t bw_bytes = 2 * static_cast<size_t>(KT) * NW * sizeof(uint16_t);  // f16 B''
    auto wide_bytes = [&](int g, int rb, int cap) {
      return bw_bytes + static_cast<size_t>(g) * 128 * RSW * sizeof(float) + 2 * static_cast<size_t>(rb) * 16 +
             home_w + static_cast<size_t>(g) * cap * kTwAtomBytes;
    };
    int GW = 0;
    if (a.stw > 0 && NW <= 64) {  // two accumulator stages of 2*NW columns
      const size_t avail_w = optin - static_smem(k_spread_zdft_tcw);
      static const int cand[][2] = {{1024, 1024}, {1024, 512}, {512, 1024}, {512, 512}, {1024, 256},
                                    {512, 256},   {256, 1024}, {256, 512},  {256, 256}, {128, 512},
                                    {128, 256},   {128, 128},  {64, 128}};  // {cap, records}
      for (int g = 1; g <= 2; ++g)
        for (const auto &c : cand)
          if (pl->tw_cap[g - 1] == 0 && wide_bytes(g, c[1], c[0]) <= avail_w) {
            pl->tw_cap[g - 1] = c[0];
            pl->tw_rb[g - 1] = c[1];
            GW = g;
          }
    }
    pl->tcn_ok = !simt_only && N <= 256 && S > 0;
    pl->tcw_ok = !simt_only && !narrow_only && GW > 0;
    if (pl->tcn_ok || pl->tcw_ok) {
      pl->use_tc = true;
      pl->use_tcw = pl->tcw_ok;
      a.tcN = N;
      a.tcK = KT;
      a.tcR = R;
    }
    if (pl->tcw_ok) {
      a.twN = NW;
      a.twRS = RSW;
      pl->twG_max = GW;
      for (int g = 1; g <= GW; ++g) pl->tw_smem[g - 1] = wide_bytes(g, pl->tw_rb[g - 1], pl->tw_cap[g - 1]);
      // one group by default: its larger atom table measured faster than two
      // groups on the 100k-atom trajectory workload (2.95 vs 3.42 ms per 100 frames)
      set_wide_groups(pl, 1);
    }
    if (pl->tcn_ok) {
      a.tcS = S;
      a.tcRB = RB;
      a.tcCap = CAP;
      a.tcG = S == 2 ? 2 : 1;
      int cols = 32;
      while (cols < S * N) cols *= 2;
      a.tcCols = cols;
      pl->smem_spread_tc = b_bytes + S * stage_bytes + 2 * static_cast<size_t>(RB) * 16 + home_bytes +
                           static_cast<size_t>(S) * CAP * kTcAtomBytes;
    }
  }
  {
    // tensor-core y- and x-axis DFTs when their shapes fit; the x pass needs at
    // most 16 types.  PYCUSAXS_YDFT=simt / PYCUSAXS_XDFT=simt keep the FP32
    // SIMT kernels.
    const char *ym = std::getenv("PYCUSAXS_YDFT");
    const char *xm = std::getenv("PYCUSAXS_XDFT");
    // the tensor maps need row strides that are multiples of 16 bytes: even extents
    if (!(ym && std::strcmp(ym, "simt") == 0) && a.ext[1] % 2 == 0)
      pl->use_ytc = dtc_shape(a.nky, a.ext[1], optin - static_smem(k_dft_tc<false>), &pl->yshape,
                              &pl->smem_ydft_tc, true);
    a.xtcKyb = 128 / a.T;
    if (!(xm && std::strcmp(xm, "simt") == 0) && a.T <= 16 && a.ext[0] % 2 == 0)
      pl->use_xtc = dtc_shape(a.nkx, a.ext[0], optin - static_smem(k_dft_tc<true>), &pl->xshape,
                              &pl->smem_xdft_tc, false);
  }
  pl->tc_ok = pl->use_tc;
  pl->ytc_ok = pl->use_ytc;
  pl->xtc_ok = pl->use_xtc;
  pl->smem_hist = a.num_bins <= kHistSmemBins ? 2 * sizeof(double) * a.num_bins : 0;
  const size_t smem_sort = 2 * sizeof(int) * static_cast<size_t>(a.tiles[0]) * a.tiles[1];
  if (pl->smem_spread + static_smem(k_spread_zdft) > optin ||
      pl->smem_ydft + static_smem(k_ydft) > optin ||
      pl->smem_xdft + static_smem(k_xdft_post) > optin ||
      pl->smem_hist + static_smem(k_hist<double>) > optin || smem_sort + static_smem(k_sort_atoms) > optin) {
    destroy(pl);
    return fail(SAXS_E_INVALID,
                "grid / q-cut combination exceeds the shared-memory budget (z extent " +
                    std::to_string(a.n[2]) + ", k-box " + std::to_string(a.nkx) + "x" +
                    std::to_string(a.nky) + "x" + std::to_string(a.nkz) + ")");
  }
  if (a.T > 64) {
    destroy(pl);
    return fail(SAXS_E_INVALID, "at most 64 element types are supported");
  }

  const int B = p.max_frames;
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  int rc = SAXS_OK;
  int32_t *d_ea = nullptr, *d_et = nullptr;
  float2 *d_twz = nullptr, *d_twy = nullptr, *d_twx = nullptr;
  float *d_modx = nullptr, *d_mody = nullptr, *d_modz = nullptr, *d_ff = nullptr, *d_geom = nullptr;
  int *d_status = nullptr;
#define ALLOC(ptr, cnt)                       \
  do {                                        \
    if ((rc = dalloc(pl, &(ptr), (cnt)))) {   \
      destroy(pl);                            \
      return rc;                              \
    }                                         \
  } while (0)
  ALLOC(d_ea, a.M);
  ALLOC(d_et, a.M);
  int *d_ts = nullptr;
  ALLOC(d_ts, a.T + 1);
  // entries grouped by type (stable), the sort kernel's per-type ranges
  std::vector<int32_t> ea_sorted(a.M), et_sorted(a.M);
  std::vector<int> type_start(a.T + 1, 0);
  for (int i = 0; i < a.M; ++i) ++type_start[p.entry_type[i] + 1];
  for (int t = 0; t < a.T; ++t) {
    pl->sort_max_type = std::max(pl->sort_max_type, type_start[t + 1]);
    type_start[t + 1] += type_start[t];
  }
  {
    std::vector<int> fill(type_start.begin(), type_start.end() - 1);
    for (int i = 0; i < a.M; ++i) {
      const int k = fill[p.entry_type[i]]++;
      ea_sorted[k] = p.entry_atom[i];
      et_sorted[k] = p.entry_type[i];
    }
  }
  ALLOC(d_twz, static_cast<size_t>(ez) * a.nkzp);
  ALLOC(d_twy, static_cast<size_t>(ey) * a.nkyp);
  ALLOC(d_twx, static_cast<size_t>(ex) * a.nkxp);
  ALLOC(d_modx, nn[0]);
  ALLOC(d_mody, nn[1]);
  ALLOC(d_modz, nn[2]);
  ALLOC(d_ff, 9 * a.T);
  float *d_pad = nullptr;
  if (!pl->pad.empty()) ALLOC(d_pad, a.T);
  int4 *d_hx = nullptr, *d_hy = nullptr;
  float *d_twzs = nullptr, *d_twztc = nullptr, *d_twytc = nullptr, *d_twxtc = nullptr;
  ALLOC(d_twzs, 2 * a.nkzp);
  int4 *d_hyw = nullptr;
  float *d_twztcw = nullptr;
  if (pl->tcn_ok) ALLOC(d_twztc, 2 * static_cast<size_t>(a.tcK) * a.tcN);
  if (pl->tcw_ok) ALLOC(d_twztcw, 2 * static_cast<size_t>(a.tcK) * a.twN);
  if (pl->tcw_ok) ALLOC(d_hyw, 2 * static_cast<size_t>(a.stw));
  if (pl->use_ytc) ALLOC(d_twytc, static_cast<size_t>(pl->yshape.chunks) * 4 * pl->yshape.N * kDtcChunk);
  if (pl->use_xtc) ALLOC(d_twxtc, static_cast<size_t>(pl->xshape.chunks) * 4 * pl->xshape.N * kDtcChunk);
  ALLOC(d_hx, a.stiles[0]);
  ALLOC(d_hy, a.stiles[1]);
  ALLOC(d_geom, static_cast<size_t>(B) * kGeom);
  ALLOC(pl->d_geom0, kGeom);
  ALLOC(d_status, 4);
  ALLOC(a.key, static_cast<size_t>(B) * a.M);
  ALLOC(a.offsets, static_cast<size_t>(B) * (a.nbins + 1));
  ALLOC(a.rec, static_cast<size_t>(B) * a.M);
  ALLOC(a.border, static_cast<size_t>(B) * a.T);
  ALLOC(a.Z, static_cast<size_t>(B) * a.T * a.nkz * ex * ey);
  ALLOC(a.Y, static_cast<size_t>(B) * a.T * a.nkz * a.nky * ex);
  ALLOC(a.ibox, static_cast<size_t>(B) * a.nkz * a.nky * a.nkx);
  ALLOC(a.hist, a.num_bins);
  ALLOC(a.nhist, a.num_bins);
  ALLOC(pl->d_tmp_hist, 2 * a.num_bins);
  if (pl->ensemble == SAXS_NVT) ALLOC(a.iacc, static_cast<size_t>(a.nkz) * a.nky * a.nkx);
#undef ALLOC
  a.entry_atom = d_ea;
  a.type_start = d_ts;
  a.entry_type = d_et;
  a.twz = d_twz;
  a.twy = d_twy;
  a.twx = d_twx;
  a.modx = d_modx;
  a.mody = d_mody;
  a.modz = d_modz;
  a.ff = d_ff;
  a.pad_val = d_pad;
  a.twz_sum = d_twzs;
  a.twz_tc = d_twztc;
  a.twz_tcw = d_twztcw;
  pl->yshape.B = d_twytc;
  pl->xshape.B = d_twxtc;
  a.home_x = d_hx;
  a.home_y = d_hy;
  a.home_yw = d_hyw;
  a.geom = d_geom;
  a.status = d_status;

  // host tables
  std::vector<float2> twz(static_cast<size_t>(ez) * a.nkzp, make_float2(0.f, 0.f));
  for (int z = 0; z < ez; ++z)
    for (int k = 0; k < a.nkz; ++k) saxs::twiddle(k, z, nn[2], &twz[z * a.nkzp + k].x, &twz[z * a.nkzp + k].y);
  std::vector<float> twzs(2 * a.nkzp, 0.0f);
  for (int k = 0; k < a.nkz; ++k) {
    double re = 0.0, im = 0.0;
    for (int z = 0; z < ez; ++z) {
      long long r = (static_cast<long long>(k) * z) % nn[2];
      const double ang = -2.0 * M_PI * static_cast<double>(r) / nn[2];
      re += std::cos(ang);
      im += std::sin(ang);
    }
    twzs[2 * k] = static_cast<float>(re);
    twzs[2 * k + 1] = static_cast<float>(im);
  }
  // the same z twiddles in the tensor-core B layout, split into a TF32 head and
  // the exact remainder
  // B operand of the tensor-core z passes, N columns: the z twiddles split into a
  // TF32 head and remainder, K-major canonical layout
  auto z_operand = [&](int N) {
    std::vector<float> out(2 * static_cast<size_t>(a.tcK) * N, 0.0f);
    const size_t half = static_cast<size_t>(a.tcK) * N;
    for (int z = 0; z < ez; ++z)
      for (int n = 0; n < 2 * a.nkz; ++n) {
        const float2 w = twz[z * a.nkzp + n / 2];
        const float v = (n & 1) ? w.y : w.x;
        uint32_t bits;
        std::memcpy(&bits, &v, sizeof(bits));
        bits &= 0xFFFFE000u;
        float head;
        std::memcpy(&head, &bits, sizeof(head));
        const size_t o = static_cast<size_t>(z / 4) * (N / 8) * 32 + (n / 8) * 32 + (n % 8) * 4 + z % 4;
        out[o] = head;
        out[half + o] = v - head;
      }
    return out;
  };
  const std::vector<float> twtc = pl->tcn_ok ? z_operand(a.tcN) : std::vector<float>();
  // wide tiles: B' = [Bh | Bl] as one K-major operand of 2*twN columns
  // wide kernel: B' = [Bh | Bl] in f16, Bh the twiddle rounded to f16 and Bl the
  // rounded remainder; element (z, n) at half ((z / 8) * 2twN + n) * 8 + z % 8
  // (K-major, 16-byte K blocks of 2twN rows)
  std::vector<__half> twtcw;
  if (pl->tcw_ok) {
    const int NB = a.twN, N2 = 2 * a.twN;
    twtcw.assign(static_cast<size_t>(a.tcK) * N2, __float2half_rn(0.0f));
    for (int z = 0; z < ez; ++z)
      for (int n = 0; n < 2 * a.nkz; ++n) {
        const float2 w = twz[z * a.nkzp + n / 2];
        const float v = (n & 1) ? w.y : w.x;
        const __half h = __float2half_rn(v);
        const __half l = __float2half_rn(v - __half2float(h));
        twtcw[(static_cast<size_t>(z / 8) * N2 + n) * 8 + z % 8] = h;
        twtcw[(static_cast<size_t>(z / 8) * N2 + n + NB) * 8 + z % 8] = l;
      }
  }
  std::vector<float2> twy(static_cast<size_t>(ey) * a.nkyp, make_float2(0.f, 0.f));
  for (int y = 0; y < ey; ++y)
    for (int k = 0; k < a.nky; ++k)
      saxs::twiddle(a.ky_lo + k, y, nn[1], &twy[y * a.nkyp + k].x, &twy[y * a.nkyp + k].y);
  std::vector<float2> twx(static_cast<size_t>(ex) * a.nkxp, make_float2(0.f, 0.f));
  for (int x = 0; x < ex; ++x)
    for (int k = 0; k < a.nkx; ++k)
      saxs::twiddle(a.kx_lo + k, x, nn[0], &twx[x * a.nkxp + k].x, &twx[x * a.nkxp + k].y);
  const std::vector<float> twytc =
      pl->use_ytc ? dtc_bprime(twy, a.nkyp, ey, a.nky, pl->yshape) : std::vector<float>();
  const std::vector<float> twxtc =
      pl->use_xtc ? dtc_bprime(twx, a.nkxp, ex, a.nkx, pl->xshape) : std::vector<float>();
  const int ndim = std::max(nn[0], std::max(nn[1], nn[2]));
  std::vector<float> mx(nn[0]), my(nn[1]), mz(nn[2]);
  saxs::bspline_moduli(nn[0], ndim, mx.data());
  saxs::bspline_moduli(nn[1], ndim, my.data());
  saxs::bspline_moduli(nn[2], ndim, mz.data());
  float g0[kGeom];
  frame_geometry(pl, p.box0, g0);

  auto up = [&](void *dst, const void *src, size_t bytes) -> int {
    if (bytes == 0) return SAXS_OK;
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    return SAXS_OK;
  };
  if ((rc = up(d_ea, ea_sorted.data(), sizeof(int32_t) * a.M)) ||
      (rc = up(d_et, et_sorted.data(), sizeof(int32_t) * a.M)) ||
      (rc = up(d_ts, type_start.data(), sizeof(int) * (a.T + 1))) ||
      (rc = up(d_twz, twz.data(), sizeof(float2) * twz.size())) ||
      (rc = up(d_twy, twy.data(), sizeof(float2) * twy.size())) ||
      (rc = up(d_twx, twx.data(), sizeof(float2) * twx.size())) ||
      (rc = up(d_modx, mx.data(), sizeof(float) * nn[0])) ||
      (rc = up(d_mody, my.data(), sizeof(float) * nn[1])) ||
      (rc = up(d_modz, mz.data(), sizeof(float) * nn[2])) ||
      (rc = up(d_ff, pl->ff.data(), sizeof(float) * pl->ff.size())) ||
      (rc = up(d_pad, pl->pad.data(), sizeof(float) * pl->pad.size())) ||
      (rc = up(d_hx, hxt.data(), sizeof(int4) * hxt.size())) ||
      (rc = up(d_twzs, twzs.data(), sizeof(float) * twzs.size())) ||
      (rc = up(d_twztc, twtc.data(), sizeof(float) * twtc.size())) ||
      (rc = up(d_twztcw, twtcw.data(), sizeof(__half) * twtcw.size())) ||
      (rc = up(d_twytc, twytc.data(), sizeof(float) * twytc.size())) ||
      (rc = up(d_twxtc, twxtc.data(), sizeof(float) * twxtc.size())) ||
      (rc = up(d_hy, hyt.data(), sizeof(int4) * hyt.size())) ||
      (rc = up(d_hyw, hywt.data(), pl->tcw_ok ? sizeof(int4) * hywt.size() : 0)) ||
      (rc = up(pl->d_geom0, g0, sizeof(g0)))) {
    destroy(pl);
    return rc;
  }
  cudaError_t e = cudaMemset(a.hist, 0, sizeof(double) * a.num_bins);
  if (e == cudaSuccess) e = cudaMemset(a.nhist, 0, sizeof(double) * a.num_bins);
  if (e == cudaSuccess && a.iacc)
    e = cudaMemset(a.iacc, 0, sizeof(double) * a.nkz * a.nky * a.nkx);
  if (e == cudaSuccess) e = cudaMemset(d_status, 0, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&pl->ring.host),
                                           sizeof(float) * kRing * B * kGeom);
  for (int i = 0; e == cudaSuccess && i < kRing; ++i)
    e = cudaEventCreateWithFlags(&pl->ring.ev[i], cudaEventDisableTiming);
  // The dynamic shared-memory limit is per kernel function, not per plan, so
  // it is raised once to the largest value each kernel allows (the opt-in
  // per-block limit minus the kernel's static shared memory).
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft);
  if (e == cudaSuccess) e = raise_smem_limit(k_sort_atoms);
  if (e == cudaSuccess) e = raise_smem_limit(k_ydft);
  if (e == cudaSuccess) e = raise_smem_limit(k_xdft_post);
  if (e == cudaSuccess) e = raise_smem_limit(k_hist<float>);
  if (e == cudaSuccess) e = raise_smem_limit(k_hist<double>);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_tc);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_tcw);
  if (e == cudaSuccess) e = raise_smem_limit(k_dft_tc<false>);
  if (e == cudaSuccess) e = raise_smem_limit(k_dft_tc<true>);
  if (e == cudaSuccess) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spread_zdft, kThreads,
                                                      pl->smem_spread);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pl->device);
    pl->spread_ctas = std::max(1, per_sm) * std::max(1, sms);
    int sort_per_sm = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sort_per_sm, k_sort_atoms, kSortThreads,
                                                        2 * sizeof(int) * a.tiles[0] * a.tiles[1]);
    pl->sort_slots = std::max(1, sort_per_sm) * std::max(1, sms);
    if (e == cudaSuccess && pl->tcw_ok) pl->tcw_ctas = std::max(1, sms);  // 512 TMEM columns: one per SM
    if (e == cudaSuccess && pl->tcn_ok) {
      // resident CTAs whose tensor-memory allocations fit the SM's 512 columns together
      int tc_per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tc_per_sm, k_spread_zdft_tc, kTcThreads,
                                                        pl->smem_spread_tc);
      tc_per_sm = std::min(std::max(1, tc_per_sm), 512 / a.tcCols);
      pl->tc_ctas = tc_per_sm * std::max(1, sms);
    }
    if (e == cudaSuccess && pl->use_ytc) {
      int per = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dft_tc<false>, dtc_threads<false>(),
                                                        pl->smem_ydft_tc);
      per = std::min(std::max(1, per), 512 / pl->yshape.cols);
      pl->ytc_ctas = per * std::max(1, sms);
    }
    if (e == cudaSuccess && pl->use_xtc) {
      int per = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dft_tc<true>, dtc_threads<true>(),
                                                        pl->smem_xdft_tc);
      per = std::min(std::max(1, per), 512 / pl->xshape.cols);
      pl->xtc_ctas = per * std::max(1, sms);
    }
  }
  if (e != cudaSuccess) {
    destroy(pl);
    return fail(SAXS_E_CUDA, std::string("plan setup: ") + cudaGetErrorString(e));
  }
  *out = pl;
  return SAXS_OK;
}

int launch_check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return SAXS_OK;
}

cudaEvent_t pooled_event(SaxsPlan *pl) {
  if (!pl->event_pool.empty()) {
    cudaEvent_t e = pl->event_pool.back();
    pl->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records CUDA events around one stage when profiling is on.
struct StageTimer {
  SaxsPlan *pl;
  StageRecord *rec;
  cudaStream_t st;
  void begin(int k) {
    if (!rec) return;
    rec->start[k] = pooled_event(pl);
    rec->stop[k] = pooled_event(pl);
    rec->used[k] = true;
    cudaEventRecord(rec->start[k], st);
  }
  void end(int k) {
    if (rec) cudaEventRecord(rec->stop[k], st);
  }
};

// Launch with programmatic stream serialization (see pdl_wait).
template <typename... KArgs, typename... Args>
int launch_pdl(const char *name, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  static const bool off = [] {
    const char *v = std::getenv("PYCUSAXS_PDL");  // PYCUSAXS_PDL=0: plain launches
    return v && std::strcmp(v, "0") == 0;
  }();
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = off ? 0 : 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string(name) + ": " + cudaGetErrorString(e));
  return launch_check(name);
}

// Counting sort of `nframes` frames' atoms into home-bin order (the first kernel
// of a batch: launched without programmatic serialization).  The cluster size C
// is the smallest power of two for which the largest type's slice (max_type / C
// entries) is no more than an even share of the launch's entries over the
// device's resident CTAs, capped at kSortMaxCluster.
int launch_sort(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st,
                const float *host_geom = nullptr) {
  static_assert(sizeof(DevArgs) + sizeof(SortGeom) + 2 * sizeof(int) <= 32764, "kernel parameter space");
  SortGeom gp{};
  const int step = host_geom ? kSortParamFrames : nframes;
  for (int f0 = 0; f0 < nframes; f0 += step) {
    const int n = std::min(step, nframes - f0);
    if (host_geom) std::memcpy(gp.g, host_geom + static_cast<size_t>(f0) * kGeom, sizeof(float) * n * kGeom);
    int C = 1;
    const long long total = static_cast<long long>(a.M) * n;
    while (C < kSortMaxCluster &&
           static_cast<long long>(pl->sort_max_type) * pl->sort_slots > static_cast<long long>(C) * total)
      C *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.T * C, n);
    cfg.blockDim = dim3(kSortThreads);
    cfg.dynamicSmemBytes = 2 * sizeof(int) * a.tiles[0] * a.tiles[1];
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_sort_atoms, a, gp, host_geom ? 1 : 0, f0);
    if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string("k_sort_atoms: ") + cudaGetErrorString(e));
    if (int rc = launch_check("k_sort_atoms")) return rc;
  }
  return SAXS_OK;
}

// Spreading + z-axis DFT of `nframes` frames: the wide-tile or 64-column
// tensor-core kernel the plan is configured for, else the FP32 SIMT kernel.
int launch_spread(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st) {
  if (pl->use_tc && pl->use_tcw) {
    const int items = a.stiles[0] * a.stw * a.T * nframes;
    return launch_pdl("k_spread_zdft_tcw", k_spread_zdft_tcw, dim3(std::max(1, std::min(items, pl->tcw_ctas))),
                      dim3(kTwThreads), pl->smem_spread_tcw, st, a, items);
  }
  const int items = a.stiles[0] * a.stiles[1] * a.T * nframes;
  if (pl->use_tc) {
    return launch_pdl("k_spread_zdft_tc", k_spread_zdft_tc, dim3(std::max(1, std::min(items, pl->tc_ctas))),
                      dim3(kTcThreads), pl->smem_spread_tc, st, a, items);
  }
  return launch_pdl("k_spread_zdft", k_spread_zdft, dim3(std::max(1, std::min(items, pl->spread_ctas))),
                    dim3(kThreads), pl->smem_spread, st, a, items);
}

// cuTensorMapEncodeTiled, fetched from the driver once (no link to libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Float32 tiled tensor map over `base` (128-byte swizzle, zero fill outside).
int encode_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
               const cuuint32_t *box) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return fail(SAXS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, static_cast<cuuint32_t>(rank), const_cast<void *>(base),
                        dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SAXS_E_CUDA, "tensor map encoding failed (" + std::to_string(r) + ")");
  return SAXS_OK;
}

// y-axis DFT of `planes` z-transformed planes: the tensor-core kernel when the
// plan has it, else the FP32 SIMT kernel.
int launch_ydft(const SaxsPlan *pl, const DevArgs &a, int planes, cudaStream_t st) {
  if (pl->use_ytc) {
    const int items = planes * ((a.ext[0] + 127) / 128);
    // Z[plane][x][y] as {2*ey floats, x, plane}
    const cuuint64_t ex = a.ext[0], ey = a.ext[1];
    const cuuint64_t dims[3] = {2 * ey, ex, static_cast<cuuint64_t>(planes)};
    const cuuint64_t strides[2] = {8 * ey, 8 * ey * ex};
    const cuuint32_t box[3] = {2 * kDtcChunk, 128, 1};
    CUtensorMap map;
    if (int rc = encode_map(&map, a.Z, 3, dims, strides, box)) return rc;
    return launch_pdl("k_dft_tc<y>", k_dft_tc<false>, dim3(std::max(1, std::min(items, pl->ytc_ctas))),
                      dim3(dtc_threads<false>()), pl->smem_ydft_tc, st, a, pl->yshape, map, items);
  }
  dim3 gy((a.ext[0] + kYRows - 1) / kYRows, a.nkz, planes / a.nkz);
  return launch_pdl("k_ydft", k_ydft, gy, dim3(kThreads), pl->smem_ydft, st, a);
}

// x-axis DFT, form factors, type sum and moduli of `nframes` frames into ibox:
// the tensor-core kernel when the plan has it, else the FP32 SIMT kernel.
int launch_xdft(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st) {
  if (pl->use_xtc) {
    const int kyb = a.xtcKyb;
    const int items = nframes * a.nkz * ((a.nky + kyb - 1) / kyb);
    // Y[f][t][kz][ky][x] as {2*ex floats, t, ky, kz, f}
    const cuuint64_t ex = a.ext[0];
    const cuuint64_t dims[5] = {2 * ex, static_cast<cuuint64_t>(a.T), static_cast<cuuint64_t>(a.nky),
                                static_cast<cuuint64_t>(a.nkz), static_cast<cuuint64_t>(nframes)};
    const cuuint64_t row = 8 * ex;
    const cuuint64_t strides[4] = {row * a.nky * a.nkz, row, row * a.nky, row * a.nky * a.nkz * a.T};
    const cuuint32_t box[5] = {2 * kDtcChunk, static_cast<cuuint32_t>(a.T), static_cast<cuuint32_t>(kyb), 1, 1};
    CUtensorMap map;
    if (int rc = encode_map(&map, a.Y, 5, dims, strides, box)) return rc;
    return launch_pdl("k_dft_tc<x>", k_dft_tc<true>, dim3(std::max(1, std::min(items, pl->xtc_ctas))),
                      dim3(dtc_threads<true>()), pl->smem_xdft_tc, st, a, pl->xshape, map, items);
  }
  dim3 gx((a.nky + kXRows - 1) / kXRows, a.nkz, nframes);
  return launch_pdl("k_xdft_post", k_xdft_post, gx, dim3(kThreads), pl->smem_xdft, st, a, pl->xc);
}

// Enqueue the memsets and kernels of one batch of `nframes` frames whose
// geometry is already in (or queued for) a.geom.  Host work free, so that it can
// be captured in a CUDA graph.
int enqueue_batch(SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st, bool timed,
                  const float *host_geom = nullptr) {
  StageTimer tm{pl, nullptr, st};
  if (timed && pl->profiling) {
    pl->prof_pending.emplace_back();
    tm.rec = &pl->prof_pending.back();
  }
  {
    tm.begin(kStSort);
    const int rc = launch_sort(pl, a, nframes, st, host_geom);
    tm.end(kStSort);
    if (rc) return rc;
  }
  {
    tm.begin(kStSpread);
    const int rc = launch_spread(pl, a, nframes, st);
    tm.end(kStSpread);
    if (rc) return rc;
  }
  {
    tm.begin(kStYdft);
    const int rc = launch_ydft(pl, a, nframes * a.T * a.nkz, st);
    tm.end(kStYdft);
    if (rc) return rc;
  }
  {
    tm.begin(kStXdft);
    const int rc = launch_xdft(pl, a, nframes, st);
    tm.end(kStXdft);
    if (rc) return rc;
  }
  tm.begin(kStHist);
  if (pl->ensemble == SAXS_NPT) {
    dim3 gh(a.nkz, nframes);
    if (int rc = launch_pdl("k_hist", k_hist<float>, gh, dim3(kThreads), pl->smem_hist, st, a, a.ibox, a.geom,
                            kGeom, 1.0, a.hist, a.nhist))
      return rc;
  } else {
    const int64_t npl = static_cast<int64_t>(a.nkz) * a.nky * a.nkx;
    k_accumulate<<<static_cast<unsigned>((npl + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, nframes);
  }
  tm.end(kStHist);
  if (int rc = launch_check("k_hist")) return rc;
  return SAXS_OK;
}

int forward(SaxsPlan *pl, const float *xyz, int64_t stride, int nframes, const float *boxes,
            cudaStream_t st) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  if (nframes < 1 || nframes > pl->p.max_frames)
    return fail(SAXS_E_INVALID, "nframes must be in [1, max_frames]");
  if (!boxes || (!xyz && pl->a.M > 0)) return fail(SAXS_E_INVALID, "null positions or boxes");
  if (stride < 3ll * pl->p.natoms) return fail(SAXS_E_INVALID, "frame stride smaller than 3*natoms");
  DevArgs a = pl->a;
  a.xyz = xyz;
  a.frame_stride = stride;
  // geometry of each frame, checked against the planned k-box
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  for (int f = 0; f < nframes; ++f) {
    const float *box = boxes + 9 * f;
    if (int rc = check_box(box)) return rc;
    frame_geometry(pl, box, g + f * kGeom);
    long long h[3];
    saxs::kbox_halfwidths(g + f * kGeom + 9, a.qcut, 1e-5, h);
    for (int d = 0; d < 3; ++d) {
      if (!pl->full_axis[d] && h[d] > pl->half[d])
        return fail(SAXS_E_RANGE, "frame box shrank beyond the planned k-box margin; "
                                  "create the plan with a larger box_margin");
    }
  }
  // the geometry travels as k_sort_atoms' kernel parameters
  if (int rc = enqueue_batch(pl, a, nframes, st, true, g)) return rc;
  pl->frames += nframes;
  pl->last_frame_batch = nframes;
  return SAXS_OK;
}

}  // namespace

struct SaxsGraph {
  std::vector<SaxsPlan *> plans;
  std::vector<DevArgs> args;
  std::vector<int> nframes;
  std::vector<int> offset;  // first frame of each plan in the geometry slots
  int total = 0;
  int device = 0;
  float *pinned[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int next = 0;
};

namespace {

void graph_destroy(SaxsGraph *g) {
  if (!g) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  for (int k = 0; k < 2; ++k) {
    if (g->done[k]) {
      cudaEventSynchronize(g->done[k]);
      cudaEventDestroy(g->done[k]);
    }
    if (g->exec[k]) cudaGraphExecDestroy(g->exec[k]);
    if (g->pinned[k]) cudaFreeHost(g->pinned[k]);
  }
  cudaSetDevice(prev);
  delete g;
}

int graph_create(SaxsPlan *const *plans, const float *const *xyz, const int64_t *stride,
                 const int *nframes, int count, SaxsGraph **out) {
  if (!plans || !xyz || !stride || !nframes || !out || count < 1)
    return fail(SAXS_E_INVALID, "null argument or empty plan list");
  *out = nullptr;
  SaxsGraph *g = new SaxsGraph();
  g->device = plans[0] ? plans[0]->device : 0;
  for (int i = 0; i < count; ++i) {
    SaxsPlan *pl = plans[i];
    if (!pl) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "null plan in the list");
    }
    for (int k = 0; k < i; ++k)
      if (plans[k] == pl) {
        graph_destroy(g);
        return fail(SAXS_E_INVALID, "a plan appears twice in one graph");
      }
    if (pl->device != g->device) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "all plans of a graph must be on one device");
    }
    if (nframes[i] < 1 || nframes[i] > pl->p.max_frames || stride[i] < 3ll * pl->p.natoms ||
        (!xyz[i] && pl->a.M > 0)) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "bad frame count, stride or positions for plan " + std::to_string(i));
    }
    DevArgs a = pl->a;
    a.xyz = xyz[i];
    a.frame_stride = stride[i];
    g->plans.push_back(pl);
    g->args.push_back(a);
    g->nframes.push_back(nframes[i]);
    g->offset.push_back(g->total);
    g->total += nframes[i];
  }
  cudaStream_t origin = nullptr;
  std::vector<cudaStream_t> br(count, nullptr);
  std::vector<cudaEvent_t> fork(count, nullptr), join(count, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking);
  for (int i = 0; e == cudaSuccess && i < count; ++i) {
    e = cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
  }
  int rc = SAXS_OK;
  for (int k = 0; e == cudaSuccess && rc == SAXS_OK && k < 2; ++k) {
    e = cudaMallocHost(reinterpret_cast<void **>(&g->pinned[k]), sizeof(float) * g->total * kGeom);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal);
    for (int i = 0; e == cudaSuccess && rc == SAXS_OK && i < count; ++i) {
      const DevArgs &a = g->args[i];
      e = cudaEventRecord(fork[i], origin);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(br[i], fork[i], 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<float *>(a.geom), g->pinned[k] + g->offset[i] * kGeom,
                            sizeof(float) * g->nframes[i] * kGeom, cudaMemcpyHostToDevice, br[i]);
      if (e == cudaSuccess) rc = enqueue_batch(g->plans[i], a, g->nframes[i], br[i], false);
      if (e == cudaSuccess && rc == SAXS_OK) e = cudaEventRecord(join[i], br[i]);
      if (e == cudaSuccess && rc == SAXS_OK) e = cudaStreamWaitEvent(origin, join[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(origin, &graph);
    if (e == cudaSuccess) e = ee;
    if (e == cudaSuccess && rc == SAXS_OK) e = cudaGraphInstantiate(&g->exec[k], graph, 0);
    if (graph) cudaGraphDestroy(graph);
  }
  for (int i = 0; i < count; ++i) {
    if (br[i]) cudaStreamDestroy(br[i]);
    if (fork[i]) cudaEventDestroy(fork[i]);
    if (join[i]) cudaEventDestroy(join[i]);
  }
  if (origin) cudaStreamDestroy(origin);
  if (e != cudaSuccess || rc != SAXS_OK) {
    graph_destroy(g);
    if (rc != SAXS_OK) return rc;
    cudaGetLastError();
    return fail(SAXS_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  }
  *out = g;
  return SAXS_OK;
}

int graph_launch(SaxsGraph *g, const float *boxes, cudaStream_t st) {
  if (!g || !boxes) return fail(SAXS_E_INVALID, "null argument");
  const int slot = g->next;
  g->next ^= 1;
  CUDA_TRY(cudaEventSynchronize(g->done[slot]));
  for (size_t i = 0; i < g->plans.size(); ++i) {
    SaxsPlan *pl = g->plans[i];
    for (int f = 0; f < g->nframes[i]; ++f) {
      const int k = g->offset[i] + f;
      const float *box = boxes + 9 * k;
      if (int rc = check_box(box)) return rc;
      float *geo = g->pinned[slot] + static_cast<size_t>(k) * kGeom;
      frame_geometry(pl, box, geo);
      long long h[3];
      saxs::kbox_halfwidths(geo + 9, pl->a.qcut, 1e-5, h);
      for (int d = 0; d < 3; ++d)
        if (!pl->full_axis[d] && h[d] > pl->half[d])
          return fail(SAXS_E_RANGE, "frame box shrank beyond the planned k-box margin");
    }
  }
  CUDA_TRY(cudaGraphLaunch(g->exec[slot], st));
  CUDA_TRY(cudaEventRecord(g->done[slot], st));
  for (size_t i = 0; i < g->plans.size(); ++i) {
    g->plans[i]->frames += g->nframes[i];
    g->plans[i]->last_frame_batch = g->nframes[i];
  }
  return SAXS_OK;
}

int histogram(SaxsPlan *pl, double *hist, double *nhist, cudaStream_t st) {
  if (!pl || !hist || !nhist) return fail(SAXS_E_INVALID, "null argument");
  const DevArgs &a = pl->a;
  const size_t nb = static_cast<size_t>(a.num_bins);
  if (pl->ensemble == SAXS_NVT) {
    double *th = pl->d_tmp_hist, *tn = pl->d_tmp_hist + nb;
    CUDA_TRY(cudaMemsetAsync(th, 0, 2 * nb * sizeof(double), st));
    if (pl->frames > 0) {
      const float fact = static_cast<float>(1.0 / static_cast<float>(pl->frames));
      dim3 gh(a.nkz, 1);
      k_hist<double><<<gh, kThreads, pl->smem_hist, st>>>(a, a.iacc, pl->d_geom0, kGeom,
                                                          static_cast<double>(fact), th, tn);
      if (int rc = launch_check("k_hist(nvt)")) return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(hist, th, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(nhist, tn, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
  } else {
    CUDA_TRY(cudaMemcpyAsync(hist, a.hist, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(nhist, a.nhist, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  int status = 0;
  CUDA_TRY(cudaMemcpyAsync(&status, a.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (status != 0)
    return fail(SAXS_E_CUDA, "tensor-core z-DFT: an MMA completion wait ran out; results are invalid");
  return SAXS_OK;
}


int ensure_adjoint(SaxsPlan *pl) {
  if (pl->d_adj_G) return SAXS_OK;
  const DevArgs &a = pl->a;
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  pl->adj_eyp = round_up(ey, 16);
  pl->adj_ezp = round_up(ez, 8);
  int rc;
  if ((rc = dalloc(pl, &pl->d_adj_dl, a.num_bins)) ||
      (rc = dalloc(pl, &pl->d_adj_S, a.T)) ||
      (rc = dalloc(pl, &pl->d_adj_dcg, a.T)) ||
      (rc = dalloc(pl, &pl->d_adj_G, static_cast<size_t>(a.T) * a.nkz * a.nky * a.nkx)) ||
      (rc = dalloc(pl, &pl->d_adj_twyT, static_cast<size_t>(a.nky) * pl->adj_eyp)) ||
      (rc = dalloc(pl, &pl->d_adj_twzT, static_cast<size_t>(a.nkz) * pl->adj_ezp)))
    return rc;
  std::vector<float2> ty(static_cast<size_t>(a.nky) * pl->adj_eyp, make_float2(0.f, 0.f));
  for (int k = 0; k < a.nky; ++k)
    for (int y = 0; y < ey; ++y)
      saxs::twiddle(a.ky_lo + k, y, a.nn[1], &ty[k * pl->adj_eyp + y].x, &ty[k * pl->adj_eyp + y].y);
  std::vector<float2> tz(static_cast<size_t>(a.nkz) * pl->adj_ezp, make_float2(0.f, 0.f));
  for (int k = 0; k < a.nkz; ++k)
    for (int z = 0; z < ez; ++z)
      saxs::twiddle(k, z, a.nn[2], &tz[k * pl->adj_ezp + z].x, &tz[k * pl->adj_ezp + z].y);
  CUDA_TRY(cudaMemcpy(pl->d_adj_twyT, ty.data(), sizeof(float2) * ty.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(pl->d_adj_twzT, tz.data(), sizeof(float2) * tz.size(), cudaMemcpyHostToDevice));
  const size_t optin = static_cast<size_t>(optin_smem());
  pl->smem_yadj = (static_cast<size_t>(a.nky) * 64 + static_cast<size_t>(a.nky) * pl->adj_eyp) *
                  sizeof(float2);
  pl->smem_zadj = (static_cast<size_t>(a.nkz) * pl->adj_ezp + static_cast<size_t>(a.nkz) * kCols) *
                      sizeof(float2) + static_cast<size_t>(ez) * kCols * sizeof(float);
  pl->adj_tiled_y = pl->smem_yadj + static_smem(k_yadj_tile) <= optin;
  pl->adj_tiled_z = pl->smem_zadj + static_smem(k_zadj_gather) <= optin;
  CUDA_TRY(raise_smem_limit(k_xdft_grad));
  if (pl->adj_tiled_y) CUDA_TRY(raise_smem_limit(k_yadj_tile));
  if (pl->adj_tiled_z) {
    CUDA_TRY(raise_smem_limit(k_zadj_gather));
    int per_sm = 0, sms = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zadj_gather, kThreads,
                                                           pl->smem_zadj));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pl->device));
    pl->zadj_ctas = std::max(1, per_sm) * std::max(1, sms);
  } else {
    if ((rc = dalloc(pl, &pl->d_adj_dg, static_cast<size_t>(a.T) * ex * ey * ez))) return rc;
  }
  return SAXS_OK;
}

int backward(SaxsPlan *pl, const float *xyz, const float *box, const double *dl, float *grad,
             cudaStream_t st) {
  if (!pl || !box || !dl || !grad || (!xyz && pl->a.M > 0)) return fail(SAXS_E_INVALID, "null argument");
  if (int rc = check_box(box)) return rc;
  if (int rc = ensure_adjoint(pl)) return rc;
  DevArgs a = pl->a;
  a.xyz = xyz;
  a.frame_stride = 3ll * pl->p.natoms;
  AdjArgs j{};
  j.dl = pl->d_adj_dl;
  j.G = pl->d_adj_G;
  j.H1 = a.Y;  // Y is consumed by k_xdft_grad before k_xadj overwrites it
  j.H2 = a.Z;  // Z is consumed by k_ydft before the y adjoint overwrites it
  j.twyT = pl->d_adj_twyT;
  j.twzT = pl->d_adj_twzT;
  j.eyp = pl->adj_eyp;
  j.ezp = pl->adj_ezp;
  j.dg = pl->d_adj_dg;
  j.S = pl->d_adj_S;
  j.dcg = pl->d_adj_dcg;
  j.grad = grad;
  // geometry of the frame through the pinned ring, checked against the k-box
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  frame_geometry(pl, box, g);
  long long h[3];
  saxs::kbox_halfwidths(g + 9, a.qcut, 1e-5, h);
  for (int d = 0; d < 3; ++d)
    if (!pl->full_axis[d] && h[d] > pl->half[d])
      return fail(SAXS_E_RANGE, "frame box shrank beyond the planned k-box margin");
  CUDA_TRY(cudaMemcpyAsync(const_cast<float *>(a.geom), g, sizeof(float) * kGeom,
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(ring.ev[slot], st));
  CUDA_TRY(cudaMemcpyAsync(pl->d_adj_dl, dl, sizeof(double) * a.num_bins, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(pl->d_adj_S, 0, sizeof(double) * a.T, st));
  CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(float) * 3 * static_cast<size_t>(pl->p.natoms), st));
  // recompute the frame's y-transformed planes (nothing is kept from the forward)
  if (int rc = launch_sort(pl, a, 1, st)) return rc;
  if (int rc = launch_spread(pl, a, 1, st)) return rc;
  if (int rc = launch_ydft(pl, a, a.T * a.nkz, st)) return rc;
  const int items = a.stiles[0] * a.stiles[1] * a.T;  // 8 x 8 column tiles of the z adjoint
  // adjoint passes
  dim3 gx((a.nky + kXRows - 1) / kXRows, a.nkz, 1);
  k_xdft_grad<<<gx, kThreads, pl->smem_xdft, st>>>(a, j, pl->xc);
  const int64_t n1 = static_cast<int64_t>(a.T) * a.nkz * a.nky * a.ext[0];
  k_xadj<<<static_cast<unsigned>((n1 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
  if (pl->adj_tiled_y) {
    dim3 gya((a.ext[0] + 63) / 64, a.nkz, a.T);
    k_yadj_tile<<<gya, kThreads, pl->smem_yadj, st>>>(a, j);
  } else {
    const int64_t n2 = static_cast<int64_t>(a.T) * a.nkz * a.ext[0] * a.ext[1];
    k_yadj<<<static_cast<unsigned>((n2 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
  }
  if (pl->adj_tiled_z) {
    k_zadj_gather<<<std::max(1, std::min(items, pl->zadj_ctas)), kThreads, pl->smem_zadj, st>>>(
        a, j, items);
  } else {
    const int64_t n3 = static_cast<int64_t>(a.T) * a.ext[0] * a.ext[1] * a.ext[2];
    k_zadj<<<static_cast<unsigned>((n3 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
    k_sum_dg<<<dim3(64, a.T), kThreads, 0, st>>>(a, j);
    if (a.M > 0) k_gather<<<(a.M + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, j);
  }
  if (pl->adj_tiled_z && a.M > 0)
    k_mean_grad<<<(a.M + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, j);
  return launch_check("backward");
}

}  // namespace

// ---------------------------------------------------------------------------
// single frame into caller scratch (used by the allocation-free entry point)
// ---------------------------------------------------------------------------
namespace saxs {

namespace {

// Byte offsets of the per-frame buffers inside one scratch block.
struct ScratchLayout {
  size_t geom, key, offsets, rec, border, Z, Y, ibox, total;
};

ScratchLayout scratch_layout(const DevArgs &a) {
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  ScratchLayout L{};
  size_t o = 0;
  L.geom = o;
  o = up(o + sizeof(float) * kGeom);
  L.key = o;
  o = up(o + sizeof(int2) * static_cast<size_t>(a.M));
  L.offsets = o;
  o = up(o + sizeof(int) * (static_cast<size_t>(a.nbins) + 1));
  L.rec = o;
  o = up(o + sizeof(float4) * static_cast<size_t>(a.M));
  L.border = o;
  o = up(o + sizeof(double) * static_cast<size_t>(a.T));
  L.Z = o;
  o = up(o + sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * a.ext[0] * a.ext[1]);
  L.Y = o;
  o = up(o + sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * a.nky * a.ext[0]);
  L.ibox = o;
  o = up(o + sizeof(float) * static_cast<size_t>(a.nkz) * a.nky * a.nkx);
  L.total = o;
  return L;
}

}  // namespace

int plan_device(const SaxsPlan *plan) { return plan->device; }

size_t single_frame_scratch_bytes(const SaxsPlan *plan) { return scratch_layout(plan->a).total; }

int record_error(int code, const char *msg) { return fail(code, msg); }

int forward_into_scratch(SaxsPlan *pl, const float *xyz, const float *box, unsigned char *scratch,
                         size_t scratch_bytes, double *hist, double *nhist, cudaStream_t st) {
  if (!pl || !box || !scratch || !hist || !nhist || (!xyz && pl->a.M > 0))
    return fail(SAXS_E_INVALID, "null argument");
  if (int rc = check_box(box)) return rc;
  DevArgs a = pl->a;
  const ScratchLayout L = scratch_layout(a);
  if (L.total > scratch_bytes) return fail(SAXS_E_RANGE, "scratch too small for this plan");
  a.xyz = xyz;
  a.frame_stride = 3ll * pl->p.natoms;
  a.geom = reinterpret_cast<const float *>(scratch + L.geom);
  a.key = reinterpret_cast<int2 *>(scratch + L.key);
  a.offsets = reinterpret_cast<int *>(scratch + L.offsets);
  a.rec = reinterpret_cast<float4 *>(scratch + L.rec);
  a.border = reinterpret_cast<double *>(scratch + L.border);
  a.Z = reinterpret_cast<float2 *>(scratch + L.Z);
  a.Y = reinterpret_cast<float2 *>(scratch + L.Y);
  a.ibox = reinterpret_cast<float *>(scratch + L.ibox);
  a.hist = hist;
  a.nhist = nhist;
  // frame geometry, checked against the k-box, staged through the plan's pinned ring
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  frame_geometry(pl, box, g);
  long long h[3];
  kbox_halfwidths(g + 9, a.qcut, 1e-5, h);
  for (int d = 0; d < 3; ++d)
    if (!pl->full_axis[d] && h[d] > pl->half[d])
      return fail(SAXS_E_RANGE, "frame box shrank beyond the planned k-box margin");
  CUDA_TRY(cudaMemcpyAsync(const_cast<float *>(a.geom), g, sizeof(float) * kGeom,
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(ring.ev[slot], st));
  // the block keeps the previous call's contents: clear what accumulates
  CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(double) * a.num_bins, st));
  CUDA_TRY(cudaMemsetAsync(nhist, 0, sizeof(double) * a.num_bins, st));
  if (int rc = launch_sort(pl, a, 1, st)) return rc;
  if (int rc = launch_spread(pl, a, 1, st)) return rc;
  if (int rc = launch_ydft(pl, a, a.T * a.nkz, st)) return rc;
  if (int rc = launch_xdft(pl, a, 1, st)) return rc;
  dim3 gh(a.nkz, 1);
  k_hist<float><<<gh, kThreads, pl->smem_hist, st>>>(a, a.ibox, a.geom, kGeom, 1.0, hist, nhist);
  return launch_check("k_hist");
}

}  // namespace saxs

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int saxs_plan_create(const SaxsParams *params, SaxsPlan **plan) {
  g_err.clear();
  return create(params, plan);
}

void saxs_plan_destroy(SaxsPlan *plan) { destroy(plan); }

int saxs_plan_info(const SaxsPlan *pl, SaxsPlanInfo *info) {
  if (!pl || !info) return fail(SAXS_E_INVALID, "null argument");
  const DevArgs &a = pl->a;
  for (int d = 0; d < 3; ++d) {
    info->grid[d] = a.n[d];
    info->scaled_grid[d] = a.nn[d];
  }
  info->bin_size = a.dq;
  info->qcut = a.qcut;
  info->num_bins = a.num_bins;
  info->kbox[0] = a.nkx;
  info->kbox[1] = a.nky;
  info->kbox[2] = a.nkz;
  info->kz_count = a.nkz;
  info->path = (pl->use_tc ? 1 : 0) | (pl->use_ytc ? 2 : 0) | (pl->use_xtc ? 4 : 0) |
               (pl->use_tc && pl->use_tcw ? 8 : 0);
  info->device_bytes = pl->bytes;
  info->frames_accumulated = pl->frames;
  return SAXS_OK;
}

int saxs_plan_config(const SaxsPlan *pl, SaxsPlanConfig *cfg) {
  if (!pl || !cfg) return fail(SAXS_E_INVALID, "null argument");
  cfg->z_tensor_cores = pl->use_tc ? 1 : 0;
  cfg->y_tensor_cores = pl->use_ytc ? 1 : 0;
  cfg->x_tensor_cores = pl->use_xtc ? 1 : 0;
  cfg->z_wide_tiles = pl->use_tc && pl->use_tcw ? 1 : 0;
  cfg->z_producer_groups = !pl->use_tc ? 1 : pl->use_tcw ? pl->a.twG : pl->a.tcG;
  cfg->z_tensor_cores_available = pl->tc_ok ? 1 : 0;
  cfg->y_tensor_cores_available = pl->ytc_ok ? 1 : 0;
  cfg->x_tensor_cores_available = pl->xtc_ok ? 1 : 0;
  cfg->z_narrow_tiles_available = pl->tcn_ok ? 1 : 0;
  cfg->z_wide_tiles_available = pl->tcw_ok ? 1 : 0;
  cfg->z_producer_groups_max = (pl->tcn_ok && pl->a.tcS == 2) ? 2 : 1;
  cfg->z_wide_producer_groups_max = pl->tcw_ok ? pl->twG_max : 1;
  return SAXS_OK;
}

int saxs_plan_set_config(SaxsPlan *pl, const SaxsPlanConfig *cfg) {
  if (!pl || !cfg) return fail(SAXS_E_INVALID, "null argument");
  const bool z = cfg->z_tensor_cores != 0, wide = z && cfg->z_wide_tiles != 0;
  if ((z && !(wide ? pl->tcw_ok : pl->tcn_ok)) || (cfg->y_tensor_cores && !pl->ytc_ok) ||
      (cfg->x_tensor_cores && !pl->xtc_ok))
    return fail(SAXS_E_INVALID, "a tensor-core pass the plan cannot run was requested");
  const int gmax = !z ? 1 : wide ? pl->twG_max : (pl->a.tcS == 2 ? 2 : 1);
  if (cfg->z_producer_groups < 1 || cfg->z_producer_groups > gmax)
    return fail(SAXS_E_INVALID, "z_producer_groups must be 1.." + std::to_string(gmax));
  pl->use_tc = z;
  pl->use_tcw = wide;
  pl->use_ytc = cfg->y_tensor_cores != 0;
  pl->use_xtc = cfg->x_tensor_cores != 0;
  if (wide)
    set_wide_groups(pl, cfg->z_producer_groups);
  else if (z)
    pl->a.tcG = cfg->z_producer_groups;
  return SAXS_OK;
}

int saxs_forward(SaxsPlan *plan, const float *xyz_dev, int64_t frame_stride, int nframes,
                 const float *boxes_host, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = forward(plan, xyz_dev, frame_stride, nframes, boxes_host,
                         static_cast<cudaStream_t>(stream));
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_histogram(SaxsPlan *plan, double *hist_host, double *nhist_host, void *stream) {
  g_err.clear();
  return histogram(plan, hist_host, nhist_host, static_cast<cudaStream_t>(stream));
}

int saxs_reset(SaxsPlan *pl, void *stream) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const DevArgs &a = pl->a;
  CUDA_TRY(cudaMemsetAsync(a.hist, 0, sizeof(double) * a.num_bins, st));
  CUDA_TRY(cudaMemsetAsync(a.nhist, 0, sizeof(double) * a.num_bins, st));
  if (a.iacc) CUDA_TRY(cudaMemsetAsync(a.iacc, 0, sizeof(double) * a.nkz * a.nky * a.nkx, st));
  pl->frames = 0;
  return SAXS_OK;
}

int saxs_debug_kbox_intensity(SaxsPlan *pl, float *out, void *stream) {
  if (!pl || !out) return fail(SAXS_E_INVALID, "null argument");
  if (pl->last_frame_batch < 1) return fail(SAXS_E_INVALID, "no frame processed yet");
  const DevArgs &a = pl->a;
  const size_t npl = static_cast<size_t>(a.nkz) * a.nky * a.nkx;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, a.ibox + (pl->last_frame_batch - 1) * npl, npl * sizeof(float),
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return SAXS_OK;
}

int saxs_debug_border_sums(SaxsPlan *pl, double *out, void *stream) {
  if (!pl || !out) return fail(SAXS_E_INVALID, "null argument");
  if (pl->last_frame_batch < 1) return fail(SAXS_E_INVALID, "no frame processed yet");
  const DevArgs &a = pl->a;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, a.border + static_cast<size_t>(pl->last_frame_batch - 1) * a.T,
                           a.T * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return SAXS_OK;
}

int saxs_backward(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                  const double *dl_dprofile_host, float *grad_xyz_dev, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = backward(plan, xyz_dev, box_host, dl_dprofile_host, grad_xyz_dev,
                          static_cast<cudaStream_t>(stream));
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_graph_create(SaxsPlan *const *plans, const float *const *xyz_dev,
                      const int64_t *frame_stride, const int *nframes, int count, SaxsGraph **graph) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  const int dev = (plans && count > 0 && plans[0]) ? plans[0]->device : prev;
  if (prev != dev) cudaSetDevice(dev);
  const int rc = graph_create(plans, xyz_dev, frame_stride, nframes, count, graph);
  if (prev != dev) cudaSetDevice(prev);
  return rc;
}

int saxs_graph_launch(SaxsGraph *graph, const float *boxes_host, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (graph && prev != graph->device) cudaSetDevice(graph->device);
  const int rc = graph_launch(graph, boxes_host, static_cast<cudaStream_t>(stream));
  if (graph && prev != graph->device) cudaSetDevice(prev);
  return rc;
}

void saxs_graph_destroy(SaxsGraph *graph) { graph_destroy(graph); }

int saxs_profile_stages(void) { return kStages; }

const char *saxs_profile_stage_name(int i) {
  return (i >= 0 && i < kStages) ? kStageNames[i] : "";
}

int saxs_profile_enable(SaxsPlan *pl, int enable) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  pl->profiling = enable != 0;
  return SAXS_OK;
}

int saxs_profile_read(SaxsPlan *pl, double *ms_out, int *launches_out) {
  if (!pl || !ms_out) return fail(SAXS_E_INVALID, "null argument");
  for (auto &r : pl->prof_pending) {
    for (int k = 0; k < kStages; ++k) {
      if (!r.used[k]) continue;
      CUDA_TRY(cudaEventSynchronize(r.stop[k]));
      float ms = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms, r.start[k], r.stop[k]));
      ms_out[k] += ms;
      if (launches_out) launches_out[k] += 1;
      pl->event_pool.push_back(r.start[k]);
      pl->event_pool.push_back(r.stop[k]);
      r.start[k] = r.stop[k] = nullptr;
    }
  }
  pl->prof_pending.clear();
  return SAXS_OK;
}

int64_t saxs_closest_product(int n, float sigma) { return saxs::closest_product(n, sigma); }

int saxs_cell_oc(const float box[9], float oc_out[9]) {
  if (!box || !oc_out) return fail(SAXS_E_INVALID, "null argument");
  saxs::cell_oc(box, oc_out);
  return SAXS_OK;
}

int saxs_histogram_parameters(const int nn[3], const float oc[9], float sigma, float bin_size,
                              float qcut, float *bin_out, float *qcut_out, int *num_bins_out) {
  if (!nn || !oc || !bin_out || !qcut_out || !num_bins_out) return fail(SAXS_E_INVALID, "null argument");
  saxs::histogram_parameters(nn, oc, sigma, bin_size, qcut, bin_out, qcut_out, num_bins_out);
  return SAXS_OK;
}

int saxs_bspline_moduli(int n, int ndim, float *out) {
  if (n < 1 || !out) return fail(SAXS_E_INVALID, "bad argument");
  saxs::bspline_moduli(n, ndim, out);
  return SAXS_OK;
}

const char *saxs_last_error(void) { return g_err.c_str(); }

const char *saxs_version(void) { return "pycusaxs_b200 0.1 (sm_100a)"; }

}  // extern "C"
