// Small dense FP64 linear algebra for the Krylov logic of the step (k x k, k <= 65).
//
// The reference calls LAPACK (syevr/syev for the Lanczos tridiagonal, geev for Hessenberg
// eigenvalues; src/BUG/Core/LocalSolvers/krylov.jl:77-98, root_methods.jl:136-141) and Julia's
// matrix `exp` for these. This file holds the engine's own implementations:
//   * eigh_jacobi   -- cyclic Jacobi eigen-decomposition of a real symmetric matrix;
//   * eigh_tridiag  -- eigen-decomposition of a symmetric tridiagonal matrix (the Lanczos
//                      tridiagonal) by the implicit symmetric QR step with Wilkinson shift and
//                      deflation (Golub & Van Loan, "Matrix Computations", Algorithms 8.3.2/8.3.3),
//                      the rotations chased down the diagonal and off-diagonal directly;
//   * expm          -- scaling and squaring with the degree-13 Pade approximant (Higham, "The
//                      scaling and squaring method for the matrix exponential revisited", SIAM J.
//                      Matrix Anal. Appl. 26 (2005)); the Pade coefficients are computed from
//                      their closed form (2m-j)! m! / ((2m)! j! (m-j)!);
//   * eigvals_hess  -- eigenvalues of a complex upper-Hessenberg matrix by the single-shift QR
//                      algorithm with Wilkinson shifts and deflation.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <stdexcept>
#include <vector>

namespace smallla {

using cd = std::complex<double>;

// Row-major dense matrix.
template <class V>
struct Mat {
  int n = 0, m = 0;
  std::vector<V> a;
  Mat() = default;
  Mat(int rows, int cols) : n(rows), m(cols), a(size_t(rows) * cols, V(0)) {}
  V& operator()(int i, int j) { return a[size_t(i) * m + j]; }
  const V& operator()(int i, int j) const { return a[size_t(i) * m + j]; }
};

using CMat = Mat<cd>;
using RMat = Mat<double>;

// z = x y with the complex products written out on the interleaved (re, im) storage: the inner
// loop then vectorises (std::complex's multiply carries a NaN-recovery branch per product)
inline CMat matmul(const CMat& x, const CMat& y) {
  CMat z(x.n, y.m);
  const int m = y.m;
  const double* yd = reinterpret_cast<const double*>(y.a.data());
  double* zd = reinterpret_cast<double*>(z.a.data());
  for (int i = 0; i < x.n; ++i) {
    double* zr = zd + 2 * size_t(i) * m;
    for (int k = 0; k < x.m; ++k) {
      const cd v = x(i, k);
      if (v == cd(0)) continue;
      const double vr = v.real(), vi = v.imag();
      const double* yr = yd + 2 * size_t(k) * m;
      for (int j = 0; j < m; ++j) {
        const double a = yr[2 * j], b = yr[2 * j + 1];
        zr[2 * j] += vr * a - vi * b;
        zr[2 * j + 1] += vr * b + vi * a;
      }
    }
  }
  return z;
}

inline double norm1(const CMat& x) {
  double best = 0.0;
  for (int j = 0; j < x.m; ++j) {
    double s = 0.0;
    for (int i = 0; i < x.n; ++i) s += std::abs(x(i, j));
    best = std::max(best, s);
  }
  return best;
}

inline double frob(const CMat& x) {
  double s = 0.0;
  for (auto& v : x.a) s += std::norm(v);
  return std::sqrt(s);
}

// Symmetric eigen-decomposition: returns eigenvalues (ascending) and eigenvectors as columns of V.
inline void eigh_jacobi(const RMat& A0, std::vector<double>& vals, RMat& V) {
  const int n = A0.n;
  RMat A = A0;
  V = RMat(n, n);
  for (int i = 0; i < n; ++i) V(i, i) = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += A(i, j) * A(i, j);
        if (i != j) off += A(i, j) * A(i, j);
      }
    if (off <= 1e-32 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A(p, q);
        if (apq == 0.0) continue;
        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V(k, p), vkq = V(k, q);
          V(k, p) = c * vkp - s * vkq;
          V(k, q) = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A(x, x) < A(y, y); });
  vals.resize(n);
  RMat W(n, n);
  for (int j = 0; j < n; ++j) {
    vals[j] = A(order[j], order[j]);
    for (int i = 0; i < n; ++i) W(i, j) = V(i, order[j]);
  }
  V = W;
}

// Symmetric tridiagonal eigen-decomposition: diagonal `d` (n), off-diagonal `e` (n - 1). Returns
// eigenvalues ascending and eigenvectors as columns of V. Each implicit QR step on an unreduced
// block [lo, hi] starts with the rotation that takes (d_lo - mu, e_lo) to (r, 0), mu the
// eigenvalue of the trailing 2 x 2 nearer its last entry, and chases the bulge down: the rotation
// in plane (k, k+1) is G = [[c, s], [-s, c]], T <- G^T T G, V <- V G. Off-diagonals below
// eps (|d_i| + |d_i+1|) are set to zero (deflation).
inline void eigh_tridiag(std::vector<double> d, std::vector<double> e, std::vector<double>& vals,
                         RMat& V) {
  const int n = int(d.size());
  V = RMat(n, n);
  for (int i = 0; i < n; ++i) V(i, i) = 1.0;
  e.resize(std::max(n - 1, 0));
  const double eps = 2.220446049250313e-16;
  auto negligible = [&](int i) { return std::fabs(e[i]) <= eps * (std::fabs(d[i]) + std::fabs(d[i + 1])); };
  int hi = n - 1, steps = 0;
  while (hi > 0) {
    if (negligible(hi - 1)) {
      e[hi - 1] = 0.0;
      --hi;
      continue;
    }
    int lo = hi - 1;
    while (lo > 0 && !negligible(lo - 1)) --lo;
    if (lo > 0) e[lo - 1] = 0.0;
    if (++steps > 60 * n) throw std::runtime_error("eigh_tridiag: QR iteration did not converge");
    // Wilkinson shift from the trailing 2 x 2 of the block
    const double a = d[hi - 1], b = e[hi - 1], m = d[hi];
    const double delta = 0.5 * (a - m);
    const double den = delta + (delta >= 0.0 ? 1.0 : -1.0) * std::hypot(delta, b);
    const double mu = den != 0.0 ? m - b * b / den : m;
    double x = d[lo] - mu, z = e[lo], bulge = 0.0;
    for (int k = lo; k < hi; ++k) {
      const double r = std::hypot(x, z);
      const double c = r != 0.0 ? x / r : 1.0, s = r != 0.0 ? -z / r : 0.0;
      if (k > lo) e[k - 1] = c * e[k - 1] - s * bulge;  // the previous bulge is zeroed
      const double dk = d[k], dk1 = d[k + 1], ek = e[k];
      d[k] = c * c * dk - 2.0 * c * s * ek + s * s * dk1;
      d[k + 1] = s * s * dk + 2.0 * c * s * ek + c * c * dk1;
      e[k] = c * s * (dk - dk1) + (c * c - s * s) * ek;
      if (k + 1 < hi) {
        bulge = -s * e[k + 1];
        e[k + 1] = c * e[k + 1];
        x = e[k];
        z = bulge;
      }
      for (int row = 0; row < n; ++row) {
        const double vk = V(row, k), vk1 = V(row, k + 1);
        V(row, k) = c * vk - s * vk1;
        V(row, k + 1) = s * vk + c * vk1;
      }
    }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return d[p] < d[q]; });
  vals.resize(n);
  RMat W(n, n);
  for (int j = 0; j < n; ++j) {
    vals[j] = d[order[j]];
    for (int i = 0; i < n; ++i) W(i, j) = V(i, order[j]);
  }
  V = W;
}

// Least-squares solution of A x = b (A m x n, m >= n) by Householder QR: each reflector
// I - 2 v v^H / (v^H v), v = a + e^{i arg a_kk} |a| e_k, zeroes column k below the diagonal; then
// R x = (Q^H b)[0..n). A zero column leaves its unknown zero.
inline std::vector<cd> lstsq(CMat A, std::vector<cd> b) {
  const int m = A.n, n = A.m;
  for (int k = 0; k < n && k < m; ++k) {
    double nrm2 = 0.0;
    for (int i = k; i < m; ++i) nrm2 += std::norm(A(i, k));
    const double nrm = std::sqrt(nrm2);
    if (nrm == 0.0) continue;
    const cd alpha = A(k, k);
    const cd ph = std::abs(alpha) > 0.0 ? alpha / std::abs(alpha) : cd(1.0);
    std::vector<cd> v(size_t(m - k));
    v[0] = alpha + ph * nrm;
    for (int i = k + 1; i < m; ++i) v[size_t(i - k)] = A(i, k);
    double vv = 0.0;
    for (auto& x : v) vv += std::norm(x);
    auto reflect = [&](auto&& get) {
      cd sdot = 0.0;
      for (int i = k; i < m; ++i) sdot += std::conj(v[size_t(i - k)]) * get(i);
      sdot *= 2.0 / vv;
      for (int i = k; i < m; ++i) get(i) -= v[size_t(i - k)] * sdot;
    };
    for (int j = k; j < n; ++j) reflect([&](int i) -> cd& { return A(i, j); });
    reflect([&](int i) -> cd& { return b[size_t(i)]; });
  }
  std::vector<cd> x(size_t(n), 0.0);
  for (int k = std::min(n, m) - 1; k >= 0; --k) {
    if (A(k, k) == cd(0.0)) continue;
    cd s = b[size_t(k)];
    for (int j = k + 1; j < n; ++j) s -= A(k, j) * x[size_t(j)];
    x[size_t(k)] = s / A(k, k);
  }
  return x;
}

// Solve X from P X = Q (complex, partial pivoting); P is overwritten.
inline CMat solve(CMat P, CMat Q) {
  const int n = P.n;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = std::abs(P(k, k));
    for (int i = k + 1; i < n; ++i)
      if (std::abs(P(i, k)) > best) {
        best = std::abs(P(i, k));
        piv = i;
      }
    if (best == 0.0) throw std::runtime_error("expm: singular Pade denominator");
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(P(k, j), P(piv, j));
      for (int j = 0; j < Q.m; ++j) std::swap(Q(k, j), Q(piv, j));
    }
    for (int i = k + 1; i < n; ++i) {
      const cd f = P(i, k) / P(k, k);
      if (f == cd(0)) continue;
      // x -= f y with the product written out as std::complex forms it for finite values
      const double fr = f.real(), fi = f.imag();
      auto axpy = [fr, fi](cd& x, const cd& y) {
        const double yr = y.real(), yi = y.imag();
        x = cd(x.real() - (fr * yr - fi * yi), x.imag() - (fr * yi + fi * yr));
      };
      for (int j = k; j < n; ++j) axpy(P(i, j), P(k, j));
      for (int j = 0; j < Q.m; ++j) axpy(Q(i, j), Q(k, j));
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    for (int j = 0; j < Q.m; ++j) {
      double sr = Q(k, j).real(), si = Q(k, j).imag();
      for (int i = k + 1; i < n; ++i) {
        const double ar = P(k, i).real(), ai = P(k, i).imag();
        const double br = Q(i, j).real(), bi = Q(i, j).imag();
        sr = sr - (ar * br - ai * bi);
        si = si - (ar * bi + ai * br);
      }
      Q(k, j) = cd(sr, si) / P(k, k);
    }
  }
  return Q;
}

// exp(A) by scaling and squaring with the [13/13] Pade approximant.
inline CMat expm(const CMat& A0) {
  const int n = A0.n;
  CMat I(n, n);
  for (int i = 0; i < n; ++i) I(i, i) = 1.0;
  if (n == 0) return I;
  // Pade coefficients b_j = (2m-j)! m! / ((2m)! j! (m-j)!), m = 13
  const int m = 13;
  double b[m + 1];
  for (int j = 0; j <= m; ++j) {
    long double v = 1.0L;
    for (int k = 1; k <= m; ++k) v *= (long double)k;          // m!
    for (int k = 1; k <= 2 * m - j; ++k) v *= (long double)k;  // (2m-j)!
    for (int k = 1; k <= 2 * m; ++k) v /= (long double)k;      // (2m)!
    for (int k = 1; k <= j; ++k) v /= (long double)k;          // j!
    for (int k = 1; k <= m - j; ++k) v /= (long double)k;      // (m-j)!
    b[j] = double(v);
  }
  const double theta13 = 5.371920351148152;  // Higham (2005), Table 2.3
  const double nrm = norm1(A0);
  int s = 0;
  if (nrm > theta13) s = std::max(0, int(std::ceil(std::log2(nrm / theta13))));
  CMat A = A0;
  const double scale = std::ldexp(1.0, -s);
  for (auto& v : A.a) v *= scale;
  CMat A2 = matmul(A, A), A4 = matmul(A2, A2), A6 = matmul(A4, A2);
  CMat Ut(n, n), V(n, n), W1(n, n), Z1(n, n);
  for (size_t i = 0; i < A.a.size(); ++i) {
    W1.a[i] = b[13] * A6.a[i] + b[11] * A4.a[i] + b[9] * A2.a[i];
    Z1.a[i] = b[12] * A6.a[i] + b[10] * A4.a[i] + b[8] * A2.a[i];
  }
  CMat W = matmul(A6, W1);
  for (size_t i = 0; i < A.a.size(); ++i)
    W.a[i] += b[7] * A6.a[i] + b[5] * A4.a[i] + b[3] * A2.a[i] + b[1] * I.a[i];
  CMat U = matmul(A, W);
  V = matmul(A6, Z1);
  for (size_t i = 0; i < A.a.size(); ++i)
    V.a[i] += b[6] * A6.a[i] + b[4] * A4.a[i] + b[2] * A2.a[i] + b[0] * I.a[i];
  CMat P(n, n), Q(n, n);
  for (size_t i = 0; i < A.a.size(); ++i) {
    P.a[i] = V.a[i] - U.a[i];
    Q.a[i] = V.a[i] + U.a[i];
  }
  CMat R = solve(P, Q);
  for (int k = 0; k < s; ++k) R = matmul(R, R);
  return R;
}

// Eigenvalues of a complex upper-Hessenberg matrix (entries below the subdiagonal are ignored).
inline std::vector<cd> eigvals_hess(const CMat& H0) {
  const int n = H0.n;
  CMat H = H0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j + 1 < i; ++j) H(i, j) = 0.0;
  std::vector<cd> ev(n);
  int hi = n - 1;
  int iter = 0;
  const double eps = 2.220446049250313e-16;
  while (hi >= 0) {
    if (hi == 0) {
      ev[0] = H(0, 0);
      break;
    }
    // deflation search
    int lo = hi;
    while (lo > 0) {
      const double sub = std::abs(H(lo, lo - 1));
      const double diag = std::abs(H(lo, lo)) + std::abs(H(lo - 1, lo - 1));
      if (sub <= eps * (diag > 0 ? diag : 1.0)) {
        H(lo, lo - 1) = 0.0;
        break;
      }
      --lo;
    }
    if (lo == hi) {
      ev[hi] = H(hi, hi);
      --hi;
      iter = 0;
      continue;
    }
    if (++iter > 60 * n) throw std::runtime_error("Hessenberg QR did not converge");
    // Wilkinson shift from the trailing 2x2 block
    const cd a = H(hi - 1, hi - 1), bb = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
    const cd tr = a + d, det = a * d - bb * c;
    const cd disc = std::sqrt(tr * tr / 4.0 - det);
    cd mu1 = tr / 2.0 + disc, mu2 = tr / 2.0 - disc;
    cd mu = (std::abs(mu1 - d) < std::abs(mu2 - d)) ? mu1 : mu2;
    if (iter % 11 == 0) mu += cd(std::abs(H(hi, hi - 1)), 0.0);  // exceptional shift
    // QR step on the active block lo..hi with Givens rotations
    std::vector<cd> cs(hi - lo), sn(hi - lo);
    for (int k = lo; k <= hi; ++k) H(k, k) -= mu;
    for (int k = lo; k < hi; ++k) {
      const cd x = H(k, k), y = H(k + 1, k);
      const double r = std::sqrt(std::norm(x) + std::norm(y));
      cd cc = 1.0, ss = 0.0;
      if (r > 0) {
        cc = x / r;
        ss = y / r;
      }
      cs[k - lo] = cc;
      sn[k - lo] = ss;
      // only the active block's entries are updated: the eigenvalues never read the coupling to
      // rows above `lo` or columns past `hi`, and the block's own arithmetic is unchanged
      // the complex products written out as (ac - bd, ad + bc), the operations and order of
      // std::complex's multiply for finite values, without its per-product NaN branch
      const double cr = cc.real(), ci = cc.imag(), sr = ss.real(), si = ss.imag();
      const double nci = -ci, nsi = -si, nsr = -sr;
      for (int j = k; j <= hi; ++j) {  // rows k, k+1: G^H
        const double ur = H(k, j).real(), ui = H(k, j).imag();
        const double vr = H(k + 1, j).real(), vi = H(k + 1, j).imag();
        // conj(cc) u + conj(ss) v ; -ss u + cc v
        H(k, j) = cd((cr * ur - nci * ui) + (sr * vr - nsi * vi),
                     (cr * ui + nci * ur) + (sr * vi + nsi * vr));
        H(k + 1, j) = cd((nsr * ur - nsi * ui) + (cr * vr - ci * vi),
                         (nsr * ui + nsi * ur) + (cr * vi + ci * vr));
      }
    }
    for (int k = lo; k < hi; ++k) {  // columns k, k+1: G
      const double cr = cs[k - lo].real(), ci = cs[k - lo].imag();
      const double sr = sn[k - lo].real(), si = sn[k - lo].imag();
      const double nci = -ci, nsi = -si;
      for (int i = lo; i <= std::min(k + 2, hi); ++i) {
        const double ur = H(i, k).real(), ui = H(i, k).imag();
        const double vr = H(i, k + 1).real(), vi = H(i, k + 1).imag();
        const double nur = -ur, nui = -ui;
        // u cc + v ss ; (-u) conj(ss) + v conj(cc)
        H(i, k) = cd((ur * cr - ui * ci) + (vr * sr - vi * si), (ur * ci + ui * cr) + (vr * si + vi * sr));
        H(i, k + 1) = cd((nur * sr - nui * nsi) + (vr * cr - vi * nci),
                         (nur * nsi + nui * sr) + (vr * nci + vi * cr));
      }
    }
    for (int k = lo; k <= hi; ++k) H(k, k) += mu;
  }
  return ev;
}

}  // namespace smallla
