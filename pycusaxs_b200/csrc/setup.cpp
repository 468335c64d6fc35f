// Host-side setup numerics of the SAXS path (grid sizing, inverse cell,
// Delta-q / q-cut reset, B-spline moduli, DFT twiddles).
//
// These run once per plan (and the inverse cell once per frame).  They keep the
// reference's float32 evaluation order so that the effective bin width, q-cut,
// bin count and moduli match the reference's to the last bit where the
// reference is deterministic.  Compiled with -ffp-contract=off: the reference's
// host code is built for baseline x86-64, where the compiler emits no fused
// multiply-adds.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace saxs {

// All 2^a 3^b 5^c 7^d <= limit, ascending (saxsKernel.cu:377-436).
static std::vector<long long> smooth_numbers(long long limit) {
  std::vector<long long> out;
  for (long long p2 = 1; p2 <= limit; p2 *= 2)
    for (long long p3 = p2; p3 <= limit; p3 *= 3)
      for (long long p5 = p3; p5 <= limit; p5 *= 5)
        for (long long p7 = p5; p7 <= limit; p7 *= 7) out.push_back(p7);
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// saxsKernel::findClosestProduct (saxsKernel.cu:449-469): target is
// std::round of the float product n*sigma; the first (smallest) candidate at
// minimal distance wins.
long long closest_product(int n, float sigma) {
  const float prod = static_cast<float>(n) * sigma;
  const long long target = static_cast<long long>(std::round(prod));
  long long closest = target;
  long long best = std::numeric_limits<long long>::max();
  for (long long m : smooth_numbers(target * 2)) {
    const long long d = std::llabs(m - target);
    if (d < best) {
      best = d;
      closest = m;
    }
  }
  return closest;
}

// Cell::calculateMatrices(3x3) (Cell.cpp:111-126): only the upper triangle of
// the box enters; the lower triangle of oc stays zero.
void cell_oc(const float co[9], float oc[9]) {
  for (int i = 0; i < 9; ++i) oc[i] = 0.0f;
  oc[0] = static_cast<float>(1.0 / co[0]);
  oc[1] = -co[1] / (co[0] * co[4]);
  oc[2] = (co[1] * co[5] - co[2] * co[4]) / (co[0] * co[4] * co[8]);
  oc[4] = static_cast<float>(1.0 / co[4]);
  oc[5] = -co[5] / (co[4] * co[8]);
  oc[8] = static_cast<float>(1.0 / co[8]);
}

void cell_oc_triclinic(const float co[9], float oc[9]) {
  const double h[9] = {co[0], co[1], co[2], co[3], co[4], co[5], co[6], co[7], co[8]};
  // cofactors of H; H^-1 = adj(H) / det, and oc = (H^-1)^T = cof(H) / det
  const double c00 = h[4] * h[8] - h[5] * h[7], c01 = h[5] * h[6] - h[3] * h[8], c02 = h[3] * h[7] - h[4] * h[6];
  const double c10 = h[2] * h[7] - h[1] * h[8], c11 = h[0] * h[8] - h[2] * h[6], c12 = h[1] * h[6] - h[0] * h[7];
  const double c20 = h[1] * h[5] - h[2] * h[4], c21 = h[2] * h[3] - h[0] * h[5], c22 = h[0] * h[4] - h[1] * h[3];
  const double det = h[0] * c00 + h[1] * c01 + h[2] * c02;
  const double cof[9] = {c00, c01, c02, c10, c11, c12, c20, c21, c22};
  for (int i = 0; i < 9; ++i) oc[i] = static_cast<float>(cof[i] / det);
}

int nf_of(int n) { return (n % 2 == 0) ? n / 2 : n / 2 + 1; }

// saxsKernel::resetHistogramParameters (saxsKernel.cu:489-526) and num_bins
// (saxsKernel.cu:247).
void histogram_parameters(const int nn[3], const float oc[9], float sigma, float dq_req,
                          float qcut_req, float *dq_out, float *qcut_out, int *nbins_out) {
  const float argx = 2.0f * static_cast<float>(M_PI) * oc[0] / sigma;
  const float argy = 2.0f * static_cast<float>(M_PI) * oc[4] / sigma;
  const float argz = 2.0f * static_cast<float>(M_PI) * oc[8] / sigma;
  const float fx[3] = {static_cast<float>(nf_of(nn[0])) - 1, static_cast<float>(nf_of(nn[1])) - 1,
                       static_cast<float>(nf_of(nn[2])) - 1};
  const float dq0[4] = {argx, argy, argz, dq_req};
  const float cut0[4] = {argx * fx[0], argy * fx[1], argz * fx[2], qcut_req};
  float dq = dq0[0], qc = cut0[0];
  for (int i = 1; i < 4; ++i) {
    if (dq0[i] > dq) dq = dq0[i];
    if (cut0[i] < qc) qc = cut0[i];
  }
  *dq_out = dq;
  *qcut_out = qc;
  *nbins_out = static_cast<int>(qc / dq) + 1;
}

// Cubic B-spline weights at w by the reference's recurrence
// (BSpline.cpp:26-34 / Splines.cu:11-73, order fixed at 4).
static void cubic_weights(float w, float x[4]) {
  x[2] = 0.0f;
  x[3] = 0.0f;
  x[1] = w;
  x[0] = static_cast<float>(1.0 - w);
  for (int k1 = 2; k1 <= 3; ++k1) {
    const int k = k1 + 1;
    const float div = static_cast<float>(1.0 / static_cast<float>(k - 1));
    x[k - 1] = div * w * x[k - 2];
    for (int j = 1; j <= k - 2; ++j)
      x[k - j - 1] = div * ((w + j) * x[k - j - 2] + (k - j - w) * x[k - j - 1]);
    x[0] = static_cast<float>(div * (1.0 - w) * x[0]);
  }
}

// BSpmod (BSpmod.cpp:45-129): |DFT of the order-4 spline at the knots|^2, the
// tiny-value fill, the 50-term aliasing (Gamma) correction, then inversion.
void bspline_moduli(int n, int ndim, float *out) {
  const int order = 4;
  const float twopi = static_cast<float>(M_PI * 2.0);
  const float tiny = 1.0e-7f;
  if (ndim < order + 1) ndim = order + 1;
  float d[4];
  cubic_weights(0.0f, d);
  std::vector<float> a0(ndim, 0.0f);
  for (int o = 1; o < order + 1; ++o) a0[o] = d[o - 1];
  std::vector<float> bsp(n, 0.0f);
  for (int o = 0; o < n; ++o) {
    float s1 = 0.0f, s2 = 0.0f;
    for (int p = 0; p < order + 1; ++p) {
      const float arg = twopi * static_cast<float>(o * p) / static_cast<float>(n);
      s1 += a0[p] * std::cos(arg);
      s2 += a0[p] * std::sin(arg);
    }
    bsp[o] = s1 * s1 + s2 * s2;
  }
  for (int o = 1; o < n - 1; ++o) bsp[o] = bsp[o] > tiny ? bsp[o] : 0.5f * (bsp[o - 1] + bsp[o + 1]);
  const int nf = n / 2;
  auto gamma_sum = [n](int m, int p) -> float {
    if (!m) return 1.0f;
    float g = 1.0f;
    const float x = static_cast<float>(M_PI * static_cast<float>(m) / static_cast<float>(n));
    for (int k = 1; k <= 50; ++k)
      g += static_cast<float>(std::pow(x / (x + M_PI * k), p) + std::pow(x / (x - M_PI * k), p));
    return g;
  };
  for (int k = 0; k < n; ++k) {
    float lambda = 1.0f;
    const int m = k < nf ? k : k - n;
    if (m != 0) lambda = gamma_sum(m, order) / gamma_sum(m, 2 * order);
    bsp[k] /= (lambda * lambda);
  }
  for (int k = 0; k < n; ++k) out[k] = static_cast<float>(1.0 / bsp[k]);
}

// exp(-2 pi i k x / n) in double with the angle reduced exactly, rounded to float.
void twiddle(long long k, long long x, long long n, float *re, float *im) {
  long long r = (k * x) % n;
  if (r < 0) r += n;
  const double ang = -2.0 * M_PI * static_cast<double>(r) / static_cast<double>(n);
  *re = static_cast<float>(std::cos(ang));
  *im = static_cast<float>(std::sin(ang));
}

// Half-extent of the k-box along each axis: the largest |m_d| of any integer
// point inside the ellipsoid |2 pi ocs m| <= qcut, with a relative margin for
// float rounding and box fluctuation.  A = 2 pi ocs is upper triangular, so the
// bound along axis d is qcut * || row d of A^-1 ||.
void kbox_halfwidths(const float ocs[9], float qcut, double margin, long long half[3]) {
  double a[9];
  for (int i = 0; i < 9; ++i) a[i] = 2.0 * M_PI * static_cast<double>(ocs[i]);
  // inverse of an upper-triangular 3x3
  double inv[9] = {0};
  inv[0] = 1.0 / a[0];
  inv[4] = 1.0 / a[4];
  inv[8] = 1.0 / a[8];
  inv[1] = -a[1] * inv[4] * inv[0];
  inv[5] = -a[5] * inv[8] * inv[4];
  inv[2] = -(a[1] * inv[5] + a[2] * inv[8]) * inv[0];
  for (int d = 0; d < 3; ++d) {
    const double rn = std::sqrt(inv[3 * d] * inv[3 * d] + inv[3 * d + 1] * inv[3 * d + 1] +
                                inv[3 * d + 2] * inv[3 * d + 2]);
    const double b = static_cast<double>(qcut) * rn * (1.0 + margin) + 1e-6;
    half[d] = static_cast<long long>(std::floor(b));
  }
}

}  // namespace saxs
