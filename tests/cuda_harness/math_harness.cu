// Host-side harness over the small-matrix math of the CUDA kernels
// (adaptive-gimp_b200/csrc/common.cuh: the same __host__ __device__ source),
// so CPU tests can check it against numpy / scipy.  Test infrastructure only.
#include "../../adaptive-gimp_b200/csrc/common.cuh"

using namespace agimp;

extern "C" {
void h_polar_newton3(const float* F, float* R, int* ok, int n) {
  for (int i = 0; i < n; ++i) ok[i] = polar_newton3(F + 9 * i, R + 9 * i) ? 1 : 0;
}
void h_polar_rot(int dim, const float* F, float* R, int n) {
  for (int i = 0; i < n; ++i) {
    if (dim == 2) polar_rot<2>(F + 4 * i, R + 4 * i);
    else polar_rot<3>(F + 9 * i, R + 9 * i);
  }
}
void h_svd(int dim, const float* A, float* U, float* S, float* V, int n) {
  for (int i = 0; i < n; ++i) {
    if (dim == 2) svd2(A + 4 * i, U + 4 * i, S + 2 * i, V + 4 * i);
    else svd3(A + 9 * i, U + 9 * i, S + 3 * i, V + 9 * i);
  }
}
// the 2^dim corner elements of I0 on a level of nb blocks per axis, through
// Corners and through elem_of / in_store one corner at a time
void h_corners(int dim, int nb, const int* I0, int n, unsigned* idx, int* ok, long long* ref_idx, int* ref_ok) {
  LevelDev V = {};
  V.nb = nb;
  for (int i = 0; i < n; ++i) {
    const int* b = I0 + dim * i;
    for (int a = 0; a < (1 << dim); ++a) {
      int I[3];
      for (int d = 0; d < dim; ++d) I[d] = b[d] + ((a >> (dim - 1 - d)) & 1);
      const int o = (1 << dim) * i + a;
      if (dim == 2) {
        const Corners<2> K(V, b);
        idx[o] = K.idx(a);
        ok[o] = K.ok(a);
        ref_ok[o] = in_store<2>(V, I);
        ref_idx[o] = ref_ok[o] ? elem_of<2>(V, I) : -1;
      } else {
        const Corners<3> K(V, b);
        idx[o] = K.idx(a);
        ok[o] = K.ok(a);
        ref_ok[o] = in_store<3>(V, I);
        ref_idx[o] = ref_ok[o] ? elem_of<3>(V, I) : -1;
      }
    }
  }
}
void h_axis_weights(float t, float r, float* W, float* G) { axis_weights(t, r, W, G); }
void h_axis_weights_half(float t, float* W, float* G) { axis_weights_half(t, W, G); }
// symmetric Kirchhoff stress expanded to full dim x dim matrices
void h_kirchhoff(int dim, const float* F, float mu, float la, float* tau, int n) {
  for (int i = 0; i < n; ++i) {
    if (dim == 2) {
      const float* f = F + 4 * i;
      const float J = det<2>(f);
      float t[3];
      kirchhoff_sym<2>(f, 2.f * mu, la * J * (J - 1.f), t);
      float* o = tau + 4 * i;
      o[0] = t[0]; o[1] = t[1]; o[2] = t[1]; o[3] = t[2];
    } else {
      const float* f = F + 9 * i;
      const float J = det<3>(f);
      float t[6];
      kirchhoff_sym<3>(f, 2.f * mu, la * J * (J - 1.f), t);
      float* o = tau + 9 * i;
      o[0] = t[0]; o[1] = t[1]; o[2] = t[3];
      o[3] = t[1]; o[4] = t[2]; o[5] = t[4];
      o[6] = t[3]; o[7] = t[4]; o[8] = t[5];
    }
  }
}
void h_within(int dim, const float* F, float lo, float hi, int* out, int n) {
  for (int i = 0; i < n; ++i)
    out[i] = dim == 2 ? singular_values_within<2>(F + 4 * i, lo, hi) : singular_values_within<3>(F + 9 * i, lo, hi);
}
}
