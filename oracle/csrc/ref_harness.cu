// Kernel harness around the reference's own device kernels (test infrastructure only).
//
// Compiled by oracle/build_ref.sh against the reference sources where they lie
// (cpp-src/Saxs/saxsDeviceKernels.cu, Splines.cu, opsfact.cu are #included
// unmodified).  It exposes the reference's histogram-binning kernel
// (saxsDeviceKernels.cu:67-125) and its spreading kernel
// (saxsDeviceKernels.cu:338-398) behind plain C entry points so that tests can
// pin the float32 bin rule and the B-spline stencil of the new kernels against
// the reference's compiled code on the same GPU.  Launch shapes follow
// saxsKernel.cu:87-99 and :141-147 (dim3(8,8,8) blocks; 256-thread 1D blocks).
#include "saxsDeviceKernels.cu"
#include "Splines.cu"
#include "opsfact.cu"

#include <cstdio>
#include <vector>

#define HCHECK(x)                                                              \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "ref_harness: %s -> %s\n", #x, cudaGetErrorString(e_)); \
      return (int)e_;                                                          \
    }                                                                          \
  } while (0)

extern "C" {

// hist/nhist (num_bins doubles each) from the reference's npt histogram kernel
// given the real parts of the modulus grid (nnx*nny*(nnz/2+1) floats, z fastest).
int ref_histogram(const float *ireal, const float ocs[9], int nnx, int nny, int nnz,
                  float bin_size, float qcut, int num_bins, double *hist, double *nhist) {
  const size_t npz = (size_t)nnz / 2 + 1;
  const size_t h = (size_t)nnx * nny * npz;
  std::vector<cuFloatComplex> host(h);
  for (size_t i = 0; i < h; ++i) host[i] = make_cuComplex(ireal[i], 0.0f);
  cuFloatComplex *d_arr = nullptr;
  double *d_hist = nullptr, *d_nhist = nullptr;
  float *d_oc = nullptr;
  HCHECK(cudaMalloc(&d_arr, h * sizeof(cuFloatComplex)));
  HCHECK(cudaMalloc(&d_hist, num_bins * sizeof(double)));
  HCHECK(cudaMalloc(&d_nhist, num_bins * sizeof(double)));
  HCHECK(cudaMalloc(&d_oc, 9 * sizeof(float)));
  HCHECK(cudaMemcpy(d_arr, host.data(), h * sizeof(cuFloatComplex), cudaMemcpyHostToDevice));
  HCHECK(cudaMemcpy(d_oc, ocs, 9 * sizeof(float), cudaMemcpyHostToDevice));
  HCHECK(cudaMemset(d_hist, 0, num_bins * sizeof(double)));
  HCHECK(cudaMemset(d_nhist, 0, num_bins * sizeof(double)));
  dim3 block(8, 8, 8);
  dim3 grid((nnx + 7) / 8, (nny + 7) / 8, (unsigned)((npz + 7) / 8));
  calculate_histogram<<<grid, block>>>(d_arr, d_hist, d_nhist, d_oc, nnx, nny, nnz,
                                       bin_size, qcut, num_bins);
  HCHECK(cudaGetLastError());
  HCHECK(cudaMemcpy(hist, d_hist, num_bins * sizeof(double), cudaMemcpyDeviceToHost));
  HCHECK(cudaMemcpy(nhist, d_nhist, num_bins * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d_arr);
  cudaFree(d_hist);
  cudaFree(d_nhist);
  cudaFree(d_oc);
  return 0;
}

// Density grid (nx*ny*nz floats, z fastest) from the reference's rhoCartKernel
// for n atoms (xyz, Angstrom) with the unscaled inverse cell oc (row-major 3x3).
int ref_rho(const float *xyz, int n, const float oc[9], int nx, int ny, int nz, int order,
            float *grid_out) {
  // orders above 4 make the reference read spline taps it never wrote
  // (Splines.h:7-11, saxsDeviceKernels.cu:386); the harness refuses them.
  if (order < 1 || order > 4 || nx < order || ny < order || nz < order) return -1;
  const size_t g = (size_t)nx * ny * nz;
  float *d_xyz = nullptr, *d_grid = nullptr, *d_oc = nullptr;
  HCHECK(cudaMalloc(&d_xyz, (size_t)(n > 0 ? n : 1) * 3 * sizeof(float)));
  HCHECK(cudaMalloc(&d_grid, g * sizeof(float)));
  HCHECK(cudaMalloc(&d_oc, 9 * sizeof(float)));
  if (n > 0) HCHECK(cudaMemcpy(d_xyz, xyz, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice));
  HCHECK(cudaMemcpy(d_oc, oc, 9 * sizeof(float), cudaMemcpyHostToDevice));
  HCHECK(cudaMemset(d_grid, 0, g * sizeof(float)));
  if (n > 0) {
    rhoCartKernel<<<(n + 255) / 256, 256>>>(d_xyz, d_oc, d_grid, order, n, nx, ny, nz);
    HCHECK(cudaGetLastError());
  }
  HCHECK(cudaMemcpy(grid_out, d_grid, g * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d_xyz);
  cudaFree(d_grid);
  cudaFree(d_oc);
  return 0;
}

}  // extern "C"
