// table_init.cpp -- host FP64 construction of the min-max:KB interpolation
// tables and scaling factors, as st = nufft_init(om, Nd, Jd, Kd, n_shift,
// 'table', Ld, 'minmax:kb') builds them.
//
// Reference lines followed:
//   alpha/beta fit     nufft/nufft_alpha_kb_fit.m:13-54
//   KB FT              nufft/kaiser_bessel_ft.m:70-73 (kb_m = 0, d = 1)
//   KB shape           nufft/kaiser_bessel.m:119-140, nufft/param-data/kaiser,m=0.mat
//   scaling factors    nufft/nufft_scale.m:54-75, outer product nufft/nufft_init.m:214-232
//   T, r, offset       nufft/private/nufft_T.m:45-75, nufft_r.m:32-50, nufft_offset.m:18-19
//   sinc "diric"       nufft/nufft_diric.m:38-40, nufft/nufft_sinc.m
//   1D table           nufft/nufft_table_init.m:111-134 with nufft/nufft_init.m:234-263,287-288
//   newfft kb:minmax   real table nufft/private/newfft_table_init.m:140-184 ('ratio'),
//                      kernel nufft/kaiser_bessel.m:68-69,106-117 (alpha = 2.34 J, kb_m = 0),
//                      sn nufft/newfft.m:340-375 with Nmid (nufft/newfft.m:146-151)
//
// MATLAB built-ins are replaced: mldivide by a Householder QR least-squares
// solve, inv by Gauss-Jordan with partial pivoting, besseli(0, .) by its power
// series, and besselj(1/2, z) / z^(1/2) by the closed form sqrt(2/pi) sin(z)/z.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <vector>

namespace mirt {

using cd = std::complex<double>;

namespace {

// abest.zn of nufft/param-data/kaiser,m=0.mat for J = 2..16 (alpha = J * zn
// at K/N = 2).  Data that must match the reference's file for sn parity.
const double kKbZn[15] = {2.5, 2.27, 2.31, 2.34, 2.32, 2.32, 2.35, 2.34,
                          2.34, 2.35, 2.34, 2.35, 2.35, 2.35, 2.33};

double kb_alpha_best(int J, double K_N) {
  if (K_N != 2.0) return 2.34 * J;
  int idx = J - 2;
  if (idx < 0) idx = 0;
  if (idx > 14) idx = 14;
  return J * kKbZn[idx];
}

// I0(x) by its power series sum (x^2/4)^k / (k!)^2
double bessel_i0(double x) {
  const double q = x * x / 4.0;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; k++) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}

// FT of the KB function with kb_m = 0, d = 1:
//   (2 pi)^(1/2) (J/2) / I0(alpha) * J_{1/2}(z) / z^(1/2),  z = sqrt((pi J u)^2 - alpha^2)
// and J_{1/2}(z)/z^(1/2) = sqrt(2/pi) sin(z)/z (sinh for imaginary z).
double kb_ft(double u, int J, double alpha) {
  const double a = 2 * M_PI * (J / 2.0) * u;
  const double z2 = a * a - alpha * alpha;
  double s;
  if (z2 > 0) {
    const double z = std::sqrt(z2);
    s = std::sin(z) / z;
  } else if (z2 < 0) {
    const double y = std::sqrt(-z2);
    s = std::sinh(y) / y;
  } else {
    s = 1.0;
  }
  return std::sqrt(2 * M_PI) * (J / 2.0) / bessel_i0(alpha) * std::sqrt(2 / M_PI) * s;
}

// least squares min ||X c - y|| for X [n x p] column-major by Householder QR
std::vector<double> lstsq(std::vector<double> X, int n, int p, std::vector<double> y) {
  for (int k = 0; k < p; k++) {
    double nrm = 0;
    for (int i = k; i < n; i++) nrm += X[i + k * n] * X[i + k * n];
    nrm = std::sqrt(nrm);
    if (nrm == 0) continue;
    const double alpha = X[k + k * n] > 0 ? -nrm : nrm;
    std::vector<double> v(n, 0.0);
    for (int i = k; i < n; i++) v[i] = X[i + k * n];
    v[k] -= alpha;
    double vn = 0;
    for (int i = k; i < n; i++) vn += v[i] * v[i];
    if (vn == 0) continue;
    for (int j = k; j < p; j++) {
      double dot = 0;
      for (int i = k; i < n; i++) dot += v[i] * X[i + j * n];
      const double f = 2 * dot / vn;
      for (int i = k; i < n; i++) X[i + j * n] -= f * v[i];
    }
    double dot = 0;
    for (int i = k; i < n; i++) dot += v[i] * y[i];
    const double f = 2 * dot / vn;
    for (int i = k; i < n; i++) y[i] -= f * v[i];
  }
  std::vector<double> c(p, 0.0);
  for (int k = p - 1; k >= 0; k--) {
    double s = y[k];
    for (int j = k + 1; j < p; j++) s -= X[k + j * n] * c[j];
    c[k] = X[k + k * n] != 0 ? s / X[k + k * n] : 0.0;
  }
  return c;
}

// in-place inverse of a J x J real matrix (row-major), Gauss-Jordan with pivoting
bool invert(std::vector<double> &A, int J) {
  std::vector<double> I(J * J, 0.0);
  for (int i = 0; i < J; i++) I[i * J + i] = 1;
  for (int c = 0; c < J; c++) {
    int piv = c;
    for (int r = c + 1; r < J; r++)
      if (std::fabs(A[r * J + c]) > std::fabs(A[piv * J + c])) piv = r;
    if (A[piv * J + c] == 0) return false;
    if (piv != c)
      for (int k = 0; k < J; k++) {
        std::swap(A[c * J + k], A[piv * J + k]);
        std::swap(I[c * J + k], I[piv * J + k]);
      }
    const double d = A[c * J + c];
    for (int k = 0; k < J; k++) {
      A[c * J + k] /= d;
      I[c * J + k] /= d;
    }
    for (int r = 0; r < J; r++) {
      if (r == c) continue;
      const double f = A[r * J + c];
      if (f == 0) continue;
      for (int k = 0; k < J; k++) {
        A[r * J + k] -= f * A[c * J + k];
        I[r * J + k] -= f * I[c * J + k];
      }
    }
  }
  A = I;
  return true;
}

// v as printf's %g prints it (six significant digits): the KB shape that
// MATLAB's sprintf('%g') writes into the inline kernel strings of
// nufft/kaiser_bessel.m:80-82 and nufft/kaiser_bessel_ft.m
double printed_g(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%g", v);
  return std::atof(buf);
}

double nufft_sinc(double x) {
  if (x == 0) return 1.0;
  return std::sin(M_PI * x) / (M_PI * x);
}

double diric(double k, int N, int K) { return nufft_sinc(k / ((double)K / (double)N)); }

// T = inv(C'SS'C) of nufft/private/nufft_T.m (the sinc diric; tol 0, so the
// plain inverse) for real scaling-factor coefficients alpha[0 .. La] and beta,
// row-major [J][J]; false when singular
bool minmax_T(int N, int J, int K, const std::vector<double> &alpha, double beta,
              std::vector<double> &T) {
  const int La = (int)alpha.size() - 1;
  T.assign((size_t)J * J, 0.0);
  for (int a = 0; a < J; a++)
    for (int b = 0; b < J; b++) {
      double s = 0;
      for (int l1 = -La; l1 <= La; l1++)
        for (int l2 = -La; l2 <= La; l2++) {
          const double tmp = (double)(b - a) + beta * (double)(l1 - l2);
          s += alpha[std::abs(l1)] * alpha[std::abs(l2)] * diric(tmp, N, K);
        }
      T[a * J + b] = s;
    }
  return invert(T, J);
}

}  // namespace

// alphas (L+1 real coefficients) and beta of nufft_alpha_kb_fit(N, J, K, 'Nmid', Nmid)
void alpha_kb_fit_nmid(int N, int J, int K, double Nmid, std::vector<double> &alphas,
                       double &beta) {
  beta = 1.0;
  const int L = N > 40 ? 13 : (int)std::ceil(N / 3.0);
  double kb_a = kb_alpha_best(J, (double)K / (double)N);
  // kaiser_bessel_ft('inline', ...) prints alpha with %g into its kernel string
  kb_a = printed_g(kb_a);
  std::vector<double> sn_kaiser(N), X((size_t)N * (L + 1));
  const double gam = 2 * M_PI / K;
  for (int i = 0; i < N; i++) {
    const double nl = i - Nmid;
    sn_kaiser[i] = 1.0 / kb_ft(nl / K, J, kb_a);
    for (int l = 0; l <= L; l++) X[i + (size_t)l * N] = std::cos((beta * gam * nl) * (double)l);
  }
  std::vector<double> coef = lstsq(X, N, L + 1, sn_kaiser);
  alphas.assign(L + 1, 0.0);
  alphas[0] = coef[0];
  for (int l = 1; l <= L; l++) alphas[l] = coef[l] / 2;
}

// nufft_alpha_kb_fit(N, J, K) (its default Nmid = (N - 1) / 2)
void alpha_kb_fit(int N, int J, int K, std::vector<double> &alphas, double &beta) {
  alpha_kb_fit_nmid(N, J, K, (N - 1) / 2.0, alphas, beta);
}

// 1D scaling factors nufft_scale1(N, K, alpha, beta, (N-1)/2)
std::vector<cd> scale1(int N, int K, const std::vector<double> &alpha, double beta) {
  const int L = (int)alpha.size() - 1;
  const double Nmid = (N - 1) / 2.0;
  std::vector<cd> sn(N, cd(0, 0));
  for (int n = 0; n < N; n++) {
    const double g = (2 * M_PI / K) * (n - Nmid) * beta;
    cd s(0, 0);
    for (int l1 = -L; l1 <= L; l1++) {
      const double alf = alpha[std::abs(l1)];  // real alpha: conj is a no-op
      s += alf * std::exp(cd(0, g * l1));
    }
    sn[n] = s;
  }
  return sn;
}

// Complex min-max:KB table for one dimension, length J*L+1.
bool minmax_kb_table(int N, int J, int K, int L, std::vector<cd> &h) {
  std::vector<double> alpha;
  double beta;
  alpha_kb_fit(N, J, K, alpha, beta);
  const int La = (int)alpha.size() - 1;
  std::vector<double> T;  // tol = 0 in nufft_init
  if (!minmax_T(N, J, K, alpha, beta, T)) return false;
  const double gam = 2 * M_PI / K;
  std::vector<cd> p((size_t)L * J, cd(0, 0));  // used columns 0..J-1 of p [L, K]
  std::vector<double> r(J), arg(J);
  for (int l = 0; l < L; l++) {
    const double t1 = (J / 2.0 - 1) + (double)l / L;
    const double om = t1 * 2 * M_PI / K;
    const double koff = std::floor(om / gam - J / 2.0);
    const double dk = om / gam - koff;
    for (int j = 0; j < J; j++) {
      arg[j] = -(double)(j + 1) + dk;
      double s = 0;
      for (int l1 = -La; l1 <= La; l1++) s += alpha[std::abs(l1)] * diric(arg[j] + l1 * beta, N, K);
      r[j] = s;
    }
    for (int j = 0; j < J; j++) {
      double c = 0;
      for (int i = 0; i < J; i++) c += T[j * J + i] * r[i];
      const cd ud = std::exp(cd(0, gam * (N - 1) / 2 * arg[j])) * c;
      long long col = (long long)(koff + (j + 1));
      col = ((col % K) + K) % K;
      if (col < J) p[(size_t)l + (size_t)col * L] += std::conj(ud);
    }
  }
  h.assign((size_t)J * L + 1, cd(0, 0));
  for (int jj = J - 1, blk = 0; jj >= 0; jj--, blk++)
    for (int l = 0; l < L; l++) h[(size_t)blk * L + l] = p[(size_t)l + (size_t)jj * L];
  h[(size_t)J * L] = 0;
  return true;
}

// The real min-max table of newfft's 'minmax:*' interpolators with phasing
// 'real' (nufft/newfft.m:384-395) for scaling-factor Fourier coefficients
// alpha[0..La] and beta: T = inv(C'SS'C) and r of nufft/private/nufft_T.m /
// nufft_r.m (sinc diric, tol 0: the plain inverse), coefficients c = T r
// without phase, read by the 'fast' construction of
// nufft/private/newfft_table_init.m:160-169 (columns J .. 1 of the sparse
// interpolator at t1 = J/2 - 1 + i/L, the last entry repeating the first).
// The coefficients are real.
bool minmax_table_real_ab(int N, int J, int K, int L, const std::vector<double> &alpha, double beta,
                          std::vector<double> &h) {
  const int La = (int)alpha.size() - 1;
  std::vector<double> T;
  if (!minmax_T(N, J, K, alpha, beta, T)) return false;
  const double gam = 2 * M_PI / K;
  std::vector<double> p((size_t)L * J, 0.0);  // used columns 0..J-1 of p [L, K]
  std::vector<double> r(J), arg(J);
  for (int l = 0; l < L; l++) {
    const double t1 = (J / 2.0 - 1) + (double)l / L;
    const double om = t1 * 2 * M_PI / K;
    const double koff = std::floor(om / gam - J / 2.0);
    const double dk = om / gam - koff;
    for (int j = 0; j < J; j++) {
      arg[j] = -(double)(j + 1) + dk;
      double s = 0;
      for (int l1 = -La; l1 <= La; l1++) s += alpha[std::abs(l1)] * diric(arg[j] + l1 * beta, N, K);
      r[j] = s;
    }
    for (int j = 0; j < J; j++) {
      double c = 0;
      for (int i = 0; i < J; i++) c += T[j * J + i] * r[i];
      long long col = (long long)(koff + (j + 1));
      col = ((col % K) + K) % K;
      if (col < J) p[(size_t)l + (size_t)col * L] += c;
    }
  }
  h.assign((size_t)J * L + 1, 0.0);
  for (int jj = J - 1, blk = 0; jj >= 0; jj--, blk++)
    for (int l = 0; l < L; l++) h[(size_t)blk * L + l] = p[(size_t)l + (size_t)jj * L];
  h[(size_t)J * L] = h[0];
  return true;
}

// the real part of nufft_scale1(N, K, alpha, beta, Nmid) (nufft/nufft_scale.m:54-75;
// nufft/newfft.m:360-364 keeps the real part), alpha real
std::vector<double> minmax_scale_real_ab(int N, int K, const std::vector<double> &alpha,
                                         double beta, double Nmid) {
  const int L = (int)alpha.size() - 1;
  std::vector<double> sn(N);
  for (int n = 0; n < N; n++) {
    if (L == 0) {
      sn[n] = alpha[0];
      continue;
    }
    const double g = (2 * M_PI / K) * (n - Nmid) * beta;
    cd s(0, 0);
    for (int l1 = -L; l1 <= L; l1++) s += alpha[std::abs(l1)] * std::exp(cd(0, g * l1));
    sn[n] = s.real();
  }
  return sn;
}

// newfft's ktype 'minmax:kb' (nufft/newfft.m:315-320): the alphas and beta of
// nufft_alpha_kb_fit fitted at Nmid = floor(N/2) for the table, at nmid for
// the scaling factors
bool minmax_kb_table_real(int N, int J, int K, int L, std::vector<double> &h) {
  std::vector<double> alpha;
  double beta;
  alpha_kb_fit_nmid(N, J, K, std::floor(N / 2.0), alpha, beta);
  return minmax_table_real_ab(N, J, K, L, alpha, beta, h);
}

std::vector<double> minmax_kb_scale_real(int N, int J, int K, double Nmid) {
  std::vector<double> alpha;
  double beta;
  alpha_kb_fit_nmid(N, J, K, Nmid, alpha, beta);
  return minmax_scale_real_ab(N, K, alpha, beta, Nmid);
}

// nufft_best_alpha(J, 0, K/N) (nufft/nufft_best_alpha.m), ktype 'minmax:tuned'
// (nufft/newfft.m:322-327): for K/N = 2 the numerically tuned Fourier
// coefficients of the scaling factors -- three-term sets for J = 4 and 6,
// two-term sets for J = 2, 3, 5, 7 .. 10 (the reference's tables, data the
// interpolator's values depend on); for any other K/N alpha = 1, beta = 0.5.
// False for K/N = 2 with a J outside 2..10 (the reference's 'unknown J,K/N').
bool best_alpha(int J, int N, int K, std::vector<double> &alpha, double &beta) {
  if (K != 2 * N) {
    alpha.assign(1, 1.0);
    beta = 0.5;
    return true;
  }
  if (J == 4) {
    alpha = {1, -0.5319, 0.1522, -0.0199};
    beta = 0.6339;
    return true;
  }
  if (J == 6) {
    alpha = {1, -0.6903, 0.2138, -0.0191};
    beta = 0.2254;
    return true;
  }
  static const double two[9][4] = {
      {1, -0.200, -0.04, 0.34},  {1, -0.485, 0.090, 0.48}, {1, -0.470, 0.085, 0.56},
      {1, -0.4825, 0.12, 0.495}, {1, -0.57, 0.14, 0.43},   {1, -0.465, 0.07, 0.65},
      {1, -0.540, 0.16, 0.47},   {1, -0.625, 0.14, 0.325}, {1, -0.57, 0.185, 0.43}};
  if (J < 2 || J > 10) return false;
  const double *row = two[J - 2];
  alpha = {row[0], row[1], row[2]};
  beta = row[3];
  return true;
}

// ktype 'linear' (nufft/newfft.m:268-273): the triangle (1 - |t| / (J/2)) on
// |t| < J/2, sampled by the 'fast' construction at t = -J/2 + i/L, the last
// entry repeating the first (0 at |t| = J/2)
void linear_table(int J, int L, std::vector<double> &h) {
  h.assign((size_t)J * L + 1, 0.0);
  for (long long i = 0; i < (long long)J * L; i++) {
    const double t = -J / 2.0 + (double)i / L;
    h[i] = std::fabs(t) < J / 2.0 ? 1 - std::fabs(t / (J / 2.0)) : 0.0;
  }
  h[(size_t)J * L] = h[0];
}

// its scaling factors, newfft_scale_tri (nufft/newfft.m:535-550): with
// f(x) = J sinc^2(J x / K), sn[n] = f(n - Nmid) / sum_{l = -3..3} f(n - Nmid - l K)^2
// (per dimension: the reference passes the whole Nmid vector, which only
// works in 1D)
std::vector<double> linear_scale(int N, int J, int K, double Nmid) {
  auto f = [&](double x) {
    const double s = nufft_sinc(J * x / K);
    return J * s * s;
  };
  std::vector<double> sn(N);
  for (int n = 0; n < N; n++) {
    const double nc = n - Nmid;
    double tmp = 0;
    for (int l = -3; l <= 3; l++) {
      const double v = f(nc - (double)l * K);
      tmp += v * v;
    }
    sn[n] = f(nc) / tmp;
  }
  return sn;
}

// Real table of newfft's KB interpolators (phasing 'real'): the KB kernel
// (kb_m = 0) of shape alpha sampled at t = -J/2 + i / L, i = 0 .. J*L.  The
// 'ratio' construction reads the sparse interpolator of a fake N = J problem
// column by column; for a kernel that depends only on the offset t that is
// the kernel itself, symmetric, zero at |t| = J/2.  The inline kernel carries
// alpha printed with %g (nufft/kaiser_bessel.m:80-82).  'kb:minmax' (the
// default of 'table0' / 'table1'): alpha = 2.34 J; 'kb:beatty': kb_beatty_alpha.
void kb_table_alpha(int J, int L, double alpha_full, std::vector<double> &h) {
  const double alpha = printed_g(alpha_full);
  const double i0a = bessel_i0(alpha);
  h.assign((size_t)J * L + 1, 0.0);
  for (size_t i = 0; i < h.size(); i++) {
    const double t = -J / 2.0 + (double)i / L;
    if (std::fabs(t) < J / 2.0) {
      const double f = std::sqrt(1 - (t / (J / 2.0)) * (t / (J / 2.0)));
      h[i] = bessel_i0(alpha * f) / i0a;
    }
  }
}

void kb_table(int J, int L, std::vector<double> &h) { kb_table_alpha(J, L, 2.34 * J, h); }

// 1D scaling factors of newfft's KB interpolators: 1 / KB-FT((n - Nmid) / K)
// (alpha as a number, no %g round trip here: st.kb_alf, nufft/newfft.m:352-356).
std::vector<double> kb_scale_alpha(int N, int J, int K, double nmid, double alpha) {
  std::vector<double> s(N);
  for (int n = 0; n < N; n++) s[n] = 1.0 / kb_ft((n - nmid) / K, J, alpha);
  return s;
}

std::vector<double> kb_scale(int N, int J, int K, double nmid) {
  return kb_scale_alpha(N, J, K, nmid, 2.34 * J);
}

// KB shape of ktype 'kb:beatty' (Beatty et al.): pi sqrt(J^2 / r^2 (r - 1/2)^2 - 0.8)
// with r = K / N (nufft/newfft.m:275-283); kb_m = 0.  0 when the root is not real.
double kb_beatty_alpha(int N, int J, int K) {
  const double r = (double)K / (double)N;
  const double a = (double)J * J / (r * r) * (r - 0.5) * (r - 0.5) - 0.8;
  return a > 0 ? M_PI * std::sqrt(a) : 0.0;
}

// I_m(x) for an integer order m >= 0 and x >= 0 by its power series
// sum_k (x/2)^(2k+m) / (k! (k+m)!) (positive terms)
double bessel_in(int m, double x) {
  const double q = x * x / 4.0;
  double term = std::pow(x / 2.0, m) / std::tgamma(m + 1.0), sum = term;
  for (int k = 1; k < 1000; k++) {
    term *= q / ((double)k * (double)(k + m));
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}

// the KB kernel of order m at offset t: f^m I_m(alpha f) / I_m(alpha) with
// f = sqrt(1 - (t / (J/2))^2) on |t| < J/2, else 0 (nufft/kaiser_bessel.m:
// 106-117); den = I_m(alpha)
static double kb_kernel(double t, int J, double alpha, int m, double den) {
  if (!(std::fabs(t) < J / 2.0)) return 0.0;
  const double u = t / (J / 2.0);
  const double f = std::sqrt(1 - u * u);
  return std::pow(f, m) * bessel_in(m, alpha * f) / den;
}

// J_nu(z) / z^nu for nu = m + 1/2 (the 1D KB transform), given z^2 (z
// imaginary when z^2 < 0, where the ratio is I_nu(|z|) / |z|^nu).  Power
// series sum_k (-z^2/4)^k / (k! Gamma(k + nu + 1)) / 2^nu where its terms do
// not cancel (z^2 <= 0, or z below m + 1); above, the spherical Bessel
// function j_m by upward recurrence from sin z / z (J_{m+1/2}(z) =
// sqrt(2 z / pi) j_m(z)), stable for z > m.
double jnu_over_znu(int m, double z2) {
  const double nu = m + 0.5;
  if (z2 <= (double)(m + 1) * (m + 1)) {
    double term = 1.0 / std::tgamma(nu + 1.0), sum = term;
    for (int k = 1; k < 1000; k++) {
      term *= (-z2 / 4.0) / ((double)k * ((double)k + nu));
      sum += term;
      if (std::fabs(term) < std::fabs(sum) * 1e-17) break;
    }
    return sum / std::pow(2.0, nu);
  }
  const double z = std::sqrt(z2);
  double jm = std::sin(z) / z;
  if (m > 0) {
    double jprev = jm;
    jm = std::sin(z) / (z * z) - std::cos(z) / z;
    for (int l = 1; l < m; l++) {
      const double jn = (2 * l + 1) / z * jm - jprev;
      jprev = jm;
      jm = jn;
    }
  }
  return std::sqrt(2 * z / M_PI) * jm / std::pow(z, nu);
}

// ktype 'kb:user' (nufft/newfft.m:300-313): the KB kernel of shape alpha and
// integer order m >= 0, f^m I_m(alpha f) / I_m(alpha) with f = sqrt(1 -
// (t / (J/2))^2) on |t| < J/2 (nufft/kaiser_bessel.m:106-117), both printed
// with %g into the inline kernel (:80-82), sampled at t = -J/2 + i/L as the
// 'ratio' construction reads it
void kb_user_table(int J, int L, double alpha_full, int m, std::vector<double> &h) {
  const double alpha = printed_g(alpha_full);
  const double den = bessel_in(m, alpha);
  h.assign((size_t)J * L + 1, 0.0);
  for (size_t i = 0; i < h.size(); i++) h[i] = kb_kernel(-J / 2.0 + (double)i / L, J, alpha, m, den);
}

// its scaling factors 1 / KB-FT((n - nmid) / K) with the 1D transform
// (2 pi)^(1/2) (J/2) alpha^m / I_m(alpha) J_nu(z) / z^nu, nu = m + 1/2,
// z = sqrt((2 pi (J/2) u)^2 - alpha^2) (nufft/kaiser_bessel_ft.m:70-73)
std::vector<double> kb_user_scale(int N, int J, int K, double nmid, double alpha, int m) {
  const double c = std::sqrt(2 * M_PI) * (J / 2.0) * std::pow(alpha, m) / bessel_in(m, alpha);
  std::vector<double> s(N);
  for (int n = 0; n < N; n++) {
    const double a = 2 * M_PI * (J / 2.0) * ((n - nmid) / K);
    s[n] = 1.0 / (c * jnu_over_znu(m, a * a - alpha * alpha));
  }
  return s;
}

// ---------------------------------------------------------------------------
// newfft's tables for phasing 'complex'
// ---------------------------------------------------------------------------
// The 'fast' construction of nufft/private/newfft_table_init.m:160-169 with
// phasing 'complex': the sparse interpolator of the sample points om = t1 2 pi
// / K, t1 = J/2 - 1 + l/L, has the entries conj(exp(i gam (N - 1)/2 arg) c)
// (nufft/newfft.m:405-411, 446) at grid columns mod(koff + j, K), where c is
// the coefficient of tap j at offset arg = -j + om/gam - koff
// (nufft/private/nufft_coef.m, nufft_r.m); the table is columns J .. 1 of it,
// the last entry repeating the first.  K may be fractional (the 'ratio'
// construction's fake problem).  coef(arg, c) fills the J coefficients of one
// sample point.
template <class Coef>
void table_fast_complex(double N, int J, double K, int L, Coef coef, std::vector<cd> &h) {
  const double gam = 2 * M_PI / K;
  std::vector<cd> p((size_t)L * J, cd(0, 0));  // the used columns 0 .. J-1
  std::vector<double> arg(J), c(J);
  for (int l = 0; l < L; l++) {
    const double t1 = (J / 2.0 - 1) + (double)l / L;
    const double om = t1 * 2 * M_PI / K;
    const double koff = std::floor(om / gam - J / 2.0);
    const double dk = om / gam - koff;
    for (int j = 0; j < J; j++) arg[j] = -(double)(j + 1) + dk;
    coef(arg.data(), c.data());
    for (int j = 0; j < J; j++) {
      const cd ud = std::exp(cd(0, gam * (N - 1) / 2 * arg[j])) * c[j];
      const double col = std::fmod(std::fmod(koff + (j + 1), K) + K, K);
      if (col < J && col == std::floor(col)) p[(size_t)l + (size_t)col * L] += std::conj(ud);
    }
  }
  h.assign((size_t)J * L + 1, cd(0, 0));
  for (int jj = J - 1, blk = 0; jj >= 0; jj--, blk++)
    for (int l = 0; l < L; l++) h[(size_t)blk * L + l] = p[(size_t)l + (size_t)jj * L];
  h[(size_t)J * L] = h[0];
}

// 'kb:*' with phasing 'complex': the 'ratio' construction
// (nufft/private/newfft_table_init.m:173-184): the fake problem N' = J,
// K' = J K / N, then the phase exp(i pi t (1/K - 1/K')) at t = -J/2 + i/L
void kb_table_complex(int N, int J, int K, int L, double alpha_full, int m, std::vector<cd> &h) {
  const double alpha = printed_g(alpha_full);
  const double den = bessel_in(m, alpha);
  const double Kf = (double)J * K / N;
  table_fast_complex((double)J, J, Kf, L, [&](const double *arg, double *c) {
    for (int j = 0; j < J; j++) c[j] = kb_kernel(arg[j], J, alpha, m, den);
  }, h);
  for (size_t i = 0; i < h.size(); i++) {
    const double t = -J / 2.0 + (double)i / L;
    h[i] *= std::exp(cd(0, M_PI * t * (1.0 / K - 1.0 / Kf)));
  }
}

// 'minmax:*' with phasing 'complex': T = inv(C'SS'C), c = T r for the
// scaling-factor coefficients alpha, beta, in the 'fast' construction
bool minmax_table_complex_ab(int N, int J, int K, int L, const std::vector<double> &alpha,
                             double beta, std::vector<cd> &h) {
  const int La = (int)alpha.size() - 1;
  std::vector<double> T;
  if (!minmax_T(N, J, K, alpha, beta, T)) return false;
  std::vector<double> r(J);
  table_fast_complex((double)N, J, (double)K, L, [&](const double *arg, double *c) {
    for (int j = 0; j < J; j++) {
      double s = 0;
      for (int l1 = -La; l1 <= La; l1++) s += alpha[std::abs(l1)] * diric(arg[j] + l1 * beta, N, K);
      r[j] = s;
    }
    for (int j = 0; j < J; j++) {
      double v = 0;
      for (int i = 0; i < J; i++) v += T[j * J + i] * r[i];
      c[j] = v;
    }
  }, h);
  return true;
}

// 'diric' with phasing 'complex' (nufft/newfft.m:256-266 without the odd-N
// trick of phasing 'real'): N/K diric(t, N, K) with the true Dirichlet kernel
// sin(pi t N / K) / (N sin(pi t / K)) (nufft/nufft_diric.m:31-36)
void diric_table_complex(int N, int J, int K, int L, std::vector<cd> &h) {
  table_fast_complex((double)N, J, (double)K, L, [&](const double *arg, double *c) {
    for (int j = 0; j < J; j++) {
      const double t = M_PI / K * arg[j];
      const double f = std::sin(t);
      const double cs = std::cos(t * (N - 1));
      const double d = std::fabs(f) > 1e-12 ? std::sin(N * t) / (N * f)
                                            : (double)((cs > 0) - (cs < 0));
      c[j] = (double)N / K * d;
    }
  }, h);
}

// 'linear' with phasing 'complex'
void linear_table_complex(int N, int J, int K, int L, std::vector<cd> &h) {
  table_fast_complex((double)N, J, (double)K, L, [&](const double *arg, double *c) {
    for (int j = 0; j < J; j++)
      c[j] = std::fabs(arg[j]) < J / 2.0 ? 1 - std::fabs(arg[j] / (J / 2.0)) : 0.0;
  }, h);
}

// ---------------------------------------------------------------------------
// nufft_init's interpolators in table mode
// ---------------------------------------------------------------------------
// nufft/nufft_table_init.m:100-116 reads nufft_init's sparse interpolator
// (entries conj(exp(i gam (N-1)/2 arg) c), nufft/nufft_init.m:262-290) at
// t1 = J/2 - 1 + l/L with the 'fast' construction, columns J .. 1, the last
// entry 0.  kt: 0 'kaiser' (alpha = 2.34 J, m = 0: kaiser_bessel('inline', J),
// nufft/kaiser_bessel.m:68-69), 7 'kaiser' with the caller's alpha and m,
// 3 'minmax:kb', 4 'uniform', 5 'minmax:tuned', 8 'minmax:user', 6 'linear'.
bool nufft_table_ktype(int kt, int N, int J, int K, int L, double kb_alf, int kb_m,
                       const std::vector<double> &alpha, double beta, std::vector<cd> &h) {
  if (kt == 0 || kt == 7) {
    const double a = printed_g(kt == 0 ? 2.34 * J : kb_alf);
    const int m = kt == 0 ? 0 : kb_m;
    const double den = bessel_in(m, a);
    table_fast_complex((double)N, J, (double)K, L, [&](const double *arg, double *c) {
      for (int j = 0; j < J; j++) c[j] = kb_kernel(arg[j], J, a, m, den);
    }, h);
  } else if (kt == 6) {
    linear_table_complex(N, J, K, L, h);
  } else {
    std::vector<double> al{1.0};
    double b = 0.0;
    if (kt == 3) {
      alpha_kb_fit(N, J, K, al, b);
    } else if (kt == 5) {
      if (!best_alpha(J, N, K, al, b)) return false;
    } else if (kt == 8) {
      al = alpha;
      b = beta;
    } else if (kt != 4) {
      return false;
    }
    if (!minmax_table_complex_ab(N, J, K, L, al, b, h)) return false;
  }
  h.back() = 0;
  return true;
}

// the 1D factors whose outer product is nufft_init's st.sn (st.sn(:) *
// tmp', nufft/nufft_init.m:210-230, a conjugate transpose): conj of
// 1 / KB-FT((n - (N-1)/2) / K) for 'kaiser', of nufft_scale(N, K, alpha,
// beta) for the min-max kinds, of 1 / nufft_interp_zn(0, N, J, K, kernel)
// (nufft/private/nufft_interp_zn.m) for 'linear'
bool nufft_scale_ktype(int kt, int N, int J, int K, double kb_alf, int kb_m,
                       const std::vector<double> &alpha, double beta, std::vector<cd> &sn) {
  sn.assign(N, cd(0, 0));
  const double nmid = (N - 1) / 2.0;
  if (kt == 0 || kt == 7) {
    const std::vector<double> s =
        kb_user_scale(N, J, K, nmid, kt == 0 ? 2.34 * J : kb_alf, kt == 0 ? 0 : kb_m);
    for (int n = 0; n < N; n++) sn[n] = s[n];
    return true;
  }
  if (kt == 6) {
    const double gam = 2 * M_PI / K;
    const int j0 = (J % 2 == 0) ? -J / 2 + 1 : -(J - 1) / 2;
    for (int n = 0; n < N; n++) {
      cd zn(0, 0);
      for (int jj = 0; jj < J; jj++) {
        const double jarg = -(double)(j0 + jj);
        const double f = std::fabs(jarg) < J / 2.0 ? 1 - std::fabs(jarg / (J / 2.0)) : 0.0;
        zn += f * std::exp(cd(0, gam * jarg * (n - nmid)));
      }
      sn[n] = std::conj(1.0 / zn);
    }
    return true;
  }
  std::vector<double> al{1.0};
  double b = 0.0;
  if (kt == 3) {
    alpha_kb_fit(N, J, K, al, b);
  } else if (kt == 5) {
    if (!best_alpha(J, N, K, al, b)) return false;
  } else if (kt == 8) {
    al = alpha;
    b = beta;
  } else if (kt != 4) {
    return false;
  }
  const std::vector<cd> s = scale1(N, K, al, b);
  for (int n = 0; n < N; n++) sn[n] = std::conj(s[n]);
  return true;
}

// Table of ktype 'diric' with phasing 'real' (nufft/newfft.m:256-266,
// nufft/nufft_diric.m:31-36): the kernel N' / K diric(k, N', K) with the odd
// N' = 2 floor((K + 1) / 2) - 1 and the true Dirichlet function
// sin(pi k N' / K) / (N' sin(pi k / K)) (sign(cos(pi k (N' - 1) / K)) where
// |sin(pi k / K)| <= 1e-12), read by the 'fast' construction
// (nufft/private/newfft_table_init.m:160-169, nufft/private/nufft_coef.m) at
// t = -J/2 + i / L, i < J L, the last entry repeating the first.
void diric_table(int J, int K, int L, std::vector<double> &h) {
  const int Np = 2 * ((K + 1) / 2) - 1;
  h.assign((size_t)J * L + 1, 0.0);
  for (size_t i = 0; i + 1 < h.size(); i++) {
    const double k = -J / 2.0 + (double)i / L;
    const double t = M_PI / K * k;
    const double sn = std::sin(t);
    double f;
    if (std::fabs(sn) > 1e-12) {
      f = std::sin(Np * t) / (Np * sn);
    } else {
      const double c = std::cos(t * (Np - 1));
      f = c > 0 ? 1.0 : (c < 0 ? -1.0 : 0.0);
    }
    h[i] = (double)Np / K * f;
  }
  h[h.size() - 1] = h[0];
}

}  // namespace mirt
