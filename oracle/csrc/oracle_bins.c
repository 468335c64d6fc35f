/*
 * Float32 k-point binning rule of the reference, restated in C (test infrastructure only).
 *
 * Follows saxsDeviceKernels.cu:80-101 (calculate_histogram) and :195-207
 * (scatterKernel): signed frequencies by the nf rule, mw_d = 2*pi*(ocs_d . k)
 * in float with the 2*pi product taken in double, mw = sqrtf(sum of squares),
 * a point is kept if mw <= qcut, its bin is (int)(mw / bin_size).
 *
 * The reference is compiled by nvcc with its default floating-point
 * contraction, so the dot products and the sum of squares may be evaluated
 * with fused multiply-adds.  Which pairing nvcc chooses is pinned by the GPU
 * tests; this file offers the candidates explicitly (fmaf is correctly
 * rounded) and is built with -ffp-contract=off so that the host compiler adds
 * no contraction of its own.
 *
 *   mode 0: no fused operations          r(r(a*b) + r(c*d)) + r(e*f)
 *   mode 1: fma(e, f, fma(a, b, r(c*d)))  (first product fused)
 *   mode 2: fma(e, f, fma(c, d, r(a*b)))  (second product fused)
 */
#include <math.h>
#include <stdint.h>

static inline float dot3(float a, float b, float c, float d, float e, float f, int mode) {
  switch (mode) {
    case 1:
      return fmaf(e, f, fmaf(a, b, c * d));
    case 2:
      return fmaf(e, f, fmaf(c, d, a * b));
    default: {
      float s = a * b + c * d;
      return s + e * f;
    }
  }
}

static inline int signed_freq(int i, int n) {
  int nf = (n % 2 == 0) ? n / 2 : n / 2 + 1;
  return (i < nf) ? i : i - n;
}

/* For raw half-spectrum indices (i, j, k) compute mw and the bin (-1 if the
 * point is beyond qcut or the bin is out of range).  ocs is the scaled inverse
 * cell, row-major 3x3.  Returns the number of points kept. */
int64_t oracle_bins(int64_t npts, const int32_t *ii, const int32_t *jj, const int32_t *kk,
                    int nnx, int nny, int nnz, const float ocs[9], float bin_size, float qcut,
                    int num_bins, int mode, float *mw_out, int32_t *bin_out) {
  int64_t kept = 0;
  for (int64_t p = 0; p < npts; ++p) {
    int ia = signed_freq(ii[p], nnx);
    int ja = signed_freq(jj[p], nny);
    int ka = signed_freq(kk[p], nnz);
    float fa = (float)ia, fb = (float)ja, fc = (float)ka;
    float mw1 = dot3(ocs[0], fa, ocs[1], fb, ocs[2], fc, mode);
    float mw2 = dot3(ocs[3], fa, ocs[4], fb, ocs[5], fc, mode);
    float mw3 = dot3(ocs[6], fa, ocs[7], fb, ocs[8], fc, mode);
    mw1 = (float)(2.0 * M_PI * (double)mw1);
    mw2 = (float)(2.0 * M_PI * (double)mw2);
    mw3 = (float)(2.0 * M_PI * (double)mw3);
    float mw = sqrtf(dot3(mw1, mw1, mw2, mw2, mw3, mw3, mode));
    mw_out[p] = mw;
    int32_t b = -1;
    if (!(mw > qcut) && bin_size > 0.0f) {
      int h0 = (int)(mw / bin_size);
      if (h0 >= 0 && h0 < num_bins) {
        b = h0;
        ++kept;
      }
    }
    bin_out[p] = b;
  }
  return kept;
}

/* Fractional grid coordinate of saxsDeviceKernels.cu:355-368 for one axis:
 * x1 = ocs_row . r in float (contraction mode as above), then
 * r1 = (float)(n * (x1 - rint(x1 - 0.5))) in double. */
void oracle_grid_coords(int64_t natoms, const float *xyz, const float oc[9], int nx, int ny,
                        int nz, int mode, float *r_out) {
  const int n[3] = {nx, ny, nz};
  for (int64_t a = 0; a < natoms; ++a) {
    const float x0 = xyz[3 * a], y0 = xyz[3 * a + 1], z0 = xyz[3 * a + 2];
    for (int d = 0; d < 3; ++d) {
      float x1 = dot3(oc[3 * d], x0, oc[3 * d + 1], y0, oc[3 * d + 2], z0, mode);
      double xd = (double)x1;
      r_out[3 * a + d] = (float)((double)n[d] * (xd - rint(xd - 0.5)));
    }
  }
}
