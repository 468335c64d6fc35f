// Host-side setup numerics shared by the plan code (see setup.cpp).
#pragma once

namespace saxs {

long long closest_product(int n, float sigma);
void cell_oc(const float co[9], float oc[9]);
// Full inverse-transpose of the box rows, oc = H^-T (fractional s = oc r for any
// triclinic box); computed in double, stored in float.
void cell_oc_triclinic(const float co[9], float oc[9]);
int nf_of(int n);
void histogram_parameters(const int nn[3], const float oc[9], float sigma, float dq_req,
                          float qcut_req, float *dq_out, float *qcut_out, int *nbins_out);
void bspline_moduli(int n, int ndim, float *out);
void twiddle(long long k, long long x, long long n, float *re, float *im);
void kbox_halfwidths(const float ocs[9], float qcut, double margin, long long half[3]);

}  // namespace saxs
