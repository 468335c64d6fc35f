// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// k_spread_zdft: the FP32 SIMT spreading + z-DFT kernel (fallback).

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

