// Device tridiagonal eigen-solve shared by the Lanczos drivers: the k lowest
// eigenpairs of T = tridiag(b[1..m-1], a[0..m-1], b[1..m-1]) computed by the
// calling CTA (blockDim.x == kTriThreads): multisection on Sturm counts
// (kTriThreads points per round) for the eigenvalues, then inverse iteration
// with a pivoted tridiagonal LU (thread 0) for the eigenvectors.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace edg {

constexpr int kTriThreads = 256;

__device__ inline int sturm_count(const double* a, const double* b2, int m, double x, double pivmin) {
  int cnt = 0;
  double q = a[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  for (int i = 1; i < m; ++i) {
    q = a[i] - x - b2[i] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// k lowest eigenpairs of the tridiagonal (a[0..m-1], bb[1..m-1]) for the
// calling CTA: multisection on Sturm counts, then inverse iteration (thread 0).
// evals_out[q] (q < k), evecs_out[q * ldv + i] (i < m, may be null),
// wk: 6*m doubles of scratch.
__device__ inline void tridiag_body(const double* __restrict__ a, const double* __restrict__ bb, int m, int k,
                             double* __restrict__ evals_out, double* __restrict__ evecs_out, int ldv,
                             double* __restrict__ wk) {
  double* b2 = wk;
  __shared__ double lo_s, hi_s, xs[kTriThreads + 1];
  __shared__ int cnt_s[kTriThreads + 1];
  __shared__ double gl_s, gu_s, pivmin_s;
  for (int i = threadIdx.x; i < m; i += kTriThreads) b2[i] = i == 0 ? 0.0 : bb[i] * bb[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double gl = 1e300, gu = -1e300, bmax = 0.0;
    for (int i = 0; i < m; ++i) {
      double off = (i > 0 ? fabs(bb[i]) : 0.0) + (i + 1 < m ? fabs(bb[i + 1]) : 0.0);
      gl = fmin(gl, a[i] - off);
      gu = fmax(gu, a[i] + off);
      if (i > 0) bmax = fmax(bmax, b2[i]);
    }
    double span = fmax(fabs(gl), fabs(gu));
    gl_s = gl - 2.0 * span * 1e-15 - 1e-300;
    gu_s = gu + 2.0 * span * 1e-15 + 1e-300;
    pivmin_s = fmax(1e-290, 2.2e-308 * fmax(1.0, bmax));
  }
  __syncthreads();
  for (int e = 0; e < k && e < m; ++e) {
    if (threadIdx.x == 0) {
      lo_s = gl_s;
      hi_s = gu_s;
    }
    __syncthreads();
    for (int round = 0; round < 12; ++round) {
      double lo = lo_s, hi = hi_s;
      if (!(hi - lo > 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300)) break;
      // kTriThreads interior points; count(x) = #eigenvalues < x
      double x = lo + (hi - lo) * (double)(threadIdx.x + 1) / (double)(kTriThreads + 1);
      xs[threadIdx.x] = x;
      cnt_s[threadIdx.x] = sturm_count(a, b2, m, x, pivmin_s);
      __syncthreads();
      if (threadIdx.x == 0) {
        // first point with count >= e+1 bounds eigenvalue e from above
        double nlo = lo, nhi = hi;
        for (int t = 0; t < kTriThreads; ++t) {
          if (cnt_s[t] >= e + 1) {
            nhi = xs[t];
            break;
          }
          nlo = xs[t];
        }
        lo_s = nlo;
        hi_s = nhi;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) evals_out[e] = 0.5 * (lo_s + hi_s);
    __syncthreads();
  }
  // inverse iteration for eigenvectors (thread 0; m is small)
  if (threadIdx.x == 0 && evecs_out != nullptr) {
    double* dl = wk + m;      // LU factors of tridiagonal T - theta
    double* dd = wk + 2 * m;
    double* du = wk + 3 * m;
    double* du2 = wk + 4 * m;
    int* piv = (int*)(wk + 5 * m);
    for (int e = 0; e < k && e < m; ++e) {
      double theta = evals_out[e];
      double* s = evecs_out + (int64_t)e * ldv;
      double scale = 0.0;
      for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(a[i]) + (i > 0 ? fabs(bb[i]) : 0.0));
      double eps_shift = 2.2e-16 * fmax(scale, 1e-300);
      // factor (T - theta I) with partial pivoting (dgttrf)
      for (int i = 0; i < m; ++i) {
        dd[i] = a[i] - theta;
        if (i + 1 < m) {
          dl[i] = bb[i + 1];
          du[i] = bb[i + 1];
        }
        du2[i] = 0.0;
      }
      for (int i = 0; i < m - 1; ++i) {
        if (fabs(dd[i]) >= fabs(dl[i])) {
          piv[i] = i;
          if (dd[i] == 0.0) dd[i] = eps_shift;
          double f = dl[i] / dd[i];
          dl[i] = f;
          dd[i + 1] -= f * du[i];
          if (i + 1 < m - 1) du2[i] = 0.0;
        } else {
          piv[i] = i + 1;
          double f = dd[i] / dl[i];
          dd[i] = dl[i];
          dl[i] = f;
          double tmp = du[i];
          du[i] = dd[i + 1];
          dd[i + 1] = tmp - f * dd[i + 1];
          if (i + 1 < m - 1) {
            du2[i] = du[i + 1];
            du[i + 1] = -f * du[i + 1];
          }
        }
      }
      if (dd[m - 1] == 0.0) dd[m - 1] = eps_shift;
      for (int i = 0; i < m; ++i) s[i] = 1.0 / sqrt((double)m) * (1.0 + 0.01 * (double)((i * 7 + e * 3) % 5));
      for (int it = 0; it < 3; ++it) {
        // solve L U x = P s
        for (int i = 0; i < m - 1; ++i) {
          if (piv[i] == i) {
            s[i + 1] -= dl[i] * s[i];
          } else {
            double t = s[i];
            s[i] = s[i + 1];
            s[i + 1] = t - dl[i] * s[i];
          }
        }
        s[m - 1] /= dd[m - 1];
        if (m > 1) s[m - 2] = (s[m - 2] - du[m - 2] * s[m - 1]) / dd[m - 2];
        for (int i = m - 3; i >= 0; --i) s[i] = (s[i] - du[i] * s[i + 1] - du2[i] * s[i + 2]) / dd[i];
        // orthogonalise against earlier eigenvectors (near-degenerate pairs)
        for (int f = 0; f < e; ++f) {
          const double* sf = evecs_out + (int64_t)f * ldv;
          double p = 0.0;
          for (int i = 0; i < m; ++i) p += sf[i] * s[i];
          for (int i = 0; i < m; ++i) s[i] -= p * sf[i];
        }
        double nn = 0.0;
        for (int i = 0; i < m; ++i) nn += s[i] * s[i];
        nn = 1.0 / sqrt(nn);
        for (int i = 0; i < m; ++i) s[i] *= nn;
      }
      // sign convention: largest component positive
      int imax = 0;
      for (int i = 1; i < m; ++i)
        if (fabs(s[i]) > fabs(s[imax])) imax = i;
      if (s[imax] < 0.0)
        for (int i = 0; i < m; ++i) s[i] = -s[i];
    }
  }
}


}  // namespace edg
