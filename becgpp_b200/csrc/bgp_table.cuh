// Long-range kernel tables: cell-averaged point kernels on the M^d wrap-around
// grid (becgpp/interactions.py:97-151), and the special functions they need.
#pragma once
#include <math.h>
#include "bgp_common.cuh"

BGP_NS_BEGIN

// 4-point Gauss-Legendre rule on [-1, 1] (the reference's table, interactions.py:32-35)
#define BGP_GL4_NODES {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526}
#define BGP_GL4_WTS {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538}

// Exact self-cell averages (interactions.py:41-43); the 3D value is the
// reference's 10-digit constant, kept so both tables agree entry for entry.
constexpr double kSelfNewton3D = 2.3800773640;
constexpr double kSqrt2Pi = 2.5066282746310002;   // sqrt(2 pi)

// e^x K0(x) and e^x K1(x) for x > 0 from the integral representations
//     K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt        (DLMF 10.32.9)
// so that  e^x K_nu(x) = int_0^inf exp(-x (cosh t - 1)) cosh(nu t) dt,
// evaluated by the trapezoidal rule, which converges exponentially for this
// integrand (analytic in a strip around the real axis, double-exponential decay;
// Trefethen & Weideman, SIAM Review 56 (2014)). Step h = min(0.1, 0.4/sqrt(x))
// keeps the discretisation error below 1e-16; the sum runs until the integrand
// falls below 1e-18 of its peak, with compensated (Neumaier) summation;
// cosh t - 1 is formed as 2 sinh^2(t/2) so large x loses no digits.
BGP_HD void k01e(double x, double& k0, double& k1) {
  const double h = fmin(0.1, 0.4 / sqrt(x));
  double s0 = 0.5, c0 = 0.0, s1 = 0.5, c1 = 0.0;
  for (int m = 1; m < 20000; ++m) {
    const double t = m * h;
    const double sh = sinh(0.5 * t);
    const double ch = 1.0 + 2.0 * sh * sh;           // cosh t, with cosh t - 1 = 2 sinh^2(t/2)
    const double e = exp(-2.0 * x * sh * sh);
    if (e < 1e-18) break;
    // Neumaier compensated adds
    double y = e, tt = s0 + y;
    c0 += (fabs(s0) >= fabs(y)) ? (s0 - tt) + y : (y - tt) + s0;
    s0 = tt;
    y = e * ch; tt = s1 + y;
    c1 += (fabs(s1) >= fabs(y)) ? (s1 - tt) + y : (y - tt) + s1;
    s1 = tt;
  }
  k0 = h * (s0 + c0);
  k1 = h * (s1 + c1);
}

BGP_HD double k0e(double x) { double a, b; k01e(x, a, b); return a; }

// quasi-2D kernel K(u) = e^x K0(x) / (sqrt(2 pi) l_z), x = u^2 / (4 l_z^2)  (interactions.py:64-67)
BGP_HD double q2d_point(double u, double lz) {
  const double x = u * u / (4.0 * lz * lz);
  return k0e(x) / (kSqrt2Pi * lz);
}
// virial kernel W(u) = 2 x (e^x K0 - e^x K1) / (sqrt(2 pi) l_z)  (interactions.py:70-74)
BGP_HD double q2d_virial_point(double u, double lz) {
  double x = u * u / (4.0 * lz * lz);
  x = fmax(x, 1e-300);
  double a, b;
  k01e(x, a, b);
  return 2.0 * x * (a - b) / (kSqrt2Pi * lz);
}

// point kernel: which 0 = K, 1 = W
BGP_HD double point_kernel(int kind, int which, double lz, double r2) {
  if (which == 1) return q2d_virial_point(sqrt(r2), lz);
  if (kind == 1) return 1.0 / sqrt(r2);
  if (kind == 2) return -0.5 * log(r2);
  return q2d_point(sqrt(r2), lz);
}

#if defined(__CUDACC__)
// Cell-averaged kernel on the M^d wrap-around grid (real part of a complex array),
// origin cell excluded (set on the host).
__global__ void k_table_fill(double2* out, int ndim, int M, double dx, int kind, int which, double lz) {
  const double gn[4] = BGP_GL4_NODES;
  const double gw[4] = BGP_GL4_WTS;
  const long long total = (ndim == 2) ? (long long)M * M : (long long)M * M * M;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total;
       p += (long long)gridDim.x * blockDim.x) {
    int a, b, c = 0;
    if (ndim == 2) { a = (int)(p / M); b = (int)(p - (long long)a * M); }
    else { a = (int)(p / ((long long)M * M)); const long long rem = p - (long long)a * M * M; b = (int)(rem / M); c = (int)(rem - (long long)b * M); }
    const double da = ((a <= M / 2) ? a : a - M) * dx;
    const double db = ((b <= M / 2) ? b : b - M) * dx;
    const double dc = ((c <= M / 2) ? c : c - M) * dx;
    double ker = 0.0;
    if (ndim == 2) {
      for (int u = 0; u < 4; ++u)
        for (int v = 0; v < 4; ++v) {
          const double x = da + 0.5 * dx * gn[u], y = db + 0.5 * dx * gn[v];
          ker += 0.25 * gw[u] * gw[v] * point_kernel(kind, which, lz, x * x + y * y);
        }
    } else {
      for (int u = 0; u < 4; ++u)
        for (int v = 0; v < 4; ++v)
          for (int w = 0; w < 4; ++w) {
            const double x = da + 0.5 * dx * gn[u], y = db + 0.5 * dx * gn[v], z = dc + 0.5 * dx * gn[w];
            ker += (gw[u] * gw[v] * gw[w] / 8.0) / sqrt(x * x + y * y + z * z);
          }
    }
    out[p] = cmk(ker, 0.0);
  }
}

// Real quadrant of the transformed table: Kq[a][b][c] = Re F[a][b][c], a,b,c <= M/2.
__global__ void k_table_quadrant(const double2* F, double* Kq, int ndim, int M) {
  const int Mh = M / 2 + 1;
  const long long total = (ndim == 2) ? (long long)Mh * Mh : (long long)Mh * Mh * Mh;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total;
       p += (long long)gridDim.x * blockDim.x) {
    long long src;
    if (ndim == 2) { const long long a = p / Mh, b = p - a * Mh; src = a * M + b; }
    else {
      const long long a = p / ((long long)Mh * Mh), rem = p - a * Mh * Mh, b = rem / Mh, c = rem - b * Mh;
      src = (a * M + b) * M + c;
    }
    Kq[p] = F[src].x;
  }
}
#endif

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n (host).
inline void gauss_legendre(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int iter = 0; iter < 100; ++iter) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1; p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1; p1 = p2;
    }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[n - 1 - i] = z;              // ascending order
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Average of a radial kernel over the square cell [-dx/2, dx/2]^2 in polar
// coordinates over its 8 symmetric triangles, n x n Gauss-Legendre nodes and
// r = R t^2 (interactions.py:77-94).
inline double polar_self_cell_2d(int kind, int which, double lz, double dx, int n = 48) {
  double t[128], wt[128];
  gauss_legendre(n, t, wt);
  double total = 0.0;
  for (int j = 0; j < n; ++j) {
    const double th = 0.5 * (M_PI / 4.0) * (t[j] + 1.0);
    const double wth = 0.5 * (M_PI / 4.0) * wt[j];
    const double R = 0.5 * dx / cos(th);
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
      const double tt = 0.5 * (t[i] + 1.0), wtt = 0.5 * wt[i];
      const double r = R * tt * tt;
      const double jac = 2.0 * R * R * tt * tt * tt;
      const double f = (which == 1) ? q2d_virial_point(r, lz) : q2d_point(r, lz);
      s += f * jac * wtt;
    }
    total += wth * s;
  }
  (void)kind;
  return 8.0 * total / (dx * dx);
}

BGP_NS_END  // namespace bgp
