// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// k_sort_atoms: the cluster counting sort of a batch's atoms by (type, home bin).

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
  bool bad = false;  // a NaN or infinite position among this thread's atoms
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
        rr[d] = grid_coord_checked(oc + 3 * d, px[u][0], px[u][1], px[u][2], a.n[d], bad);
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
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.status, kStatusInput);
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
    // (a non-finite coordinate was reported in pass 1; here it only becomes 0)
#pragma unroll
    for (int u = 0; u < kSortU; ++u)
      if (at[u] >= 0)
        rec[sbase[k[u].x] + k[u].y] =
            make_float4(grid_coord_checked(oc + 0, px[u][0], px[u][1], px[u][2], a.n[0], bad),
                        grid_coord_checked(oc + 3, px[u][0], px[u][1], px[u][2], a.n[1], bad),
                        grid_coord_checked(oc + 6, px[u][0], px[u][1], px[u][2], a.n[2], bad),
                        __int_as_float(eb + u * kSortThreads));
  }
  cluster_wait();
}

