// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// The adjoint (reverse-mode) kernels: dL/dI(bin) -> dL/dxyz.

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
  bool bad = false;  // a non-finite position: placed at 0 (the forward reports it)
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r[d] = grid_coord_checked(oc + 3 * d, x0, y0, z0, a.n[d], bad);
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

