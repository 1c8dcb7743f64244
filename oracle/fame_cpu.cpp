// CPU FP64 restatement of the plain band-structure method, C++ with OpenMP.
//
// TEST INFRASTRUCTURE ONLY: the oracle side of the tests and the CPU baseline of
// bench.py (`cpu_baseline`, kind "port").  The product (the CUDA library behind
// include/fame_b200.h) never links or calls it.
//
// What it restates, step for step, for Simple lattices (simple cubic, primitive
// orthorhombic/tetragonal; paths relative to the reference project root):
//   Lambdas, D_k, Pi, Nd         FAME_Main/FAME_Matrix_Lambdas.cu:77-286
//   Q_r / Q_r^* / QBQ            FAME_Main/FAME_Matrix_Vector_Production_Qr.cu:8-40,
//                                ..._Qrs.cu:7-29, ..._Isotropic_QBQ.cu:8-36
//   CG (x0 = 0, absolute tol)    FAME_Main/CG.cu:5-88
//   invAr                        FAME_Main/FAME_Matrix_Vector_Production_Isotropic_invAr.cu:8-48
//   Lanczos decomposition        FAME_Main/Lanczos_decomp_gpu.cu:7-91 (start e_M, :93-107)
//   exact-shift lock/purge       FAME_Main/Lanczos_LockPurge_gpu.cu:7-48, GVqrrq_g :95-190,
//                                given_rotation :245-265
//   restart loop, w = sqrt(1/t)  FAME_Main/Lanczos_Isotropic.cu:7-96
//   Gamma patch                  FAME_Main/FAME_Fast_Algorithms_Isotropic.cu:61-79
// The tridiagonal eigensolve the reference does with LAPACK's zpteqr
// (Lanczos_Isotropic.cu:53) is the implicit QL method with Wilkinson shifts
// (Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11, 1968), eigenvalues
// sorted descending as zpteqr returns them.  The 3-D DFTs are this file's own
// mixed-radix Stockham transforms (radix 4, 2, 3, 5, other factors by a direct
// DFT pass), one line at a time, lines spread over the OpenMP threads.
//
// In QBQ the twiddle D_k of Q_r and conj(D_k) of Q_r^* multiply the same edge and
// cancel (|D_k| = 1, B diagonal), so QBQ x = unmix(DFT(B^-1 IDFT(mix x)) / N); the
// reference applies both factors.
//
// C ABI (ctypes from bench.py and tests):
//   fame_cpu_solve   full solve of a list of k-points
//   fame_cpu_time    seconds per CG iteration and per Lanczos step at one k-point
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <complex>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.141592653589793;  // the reference's `pi` (include/FAME_Internal_Common.h:23)

// ------------------------------------------------------------------ 1-D FFT
struct Plan {
  int n = 1;
  std::vector<int> rad;
  std::vector<cd> w;  // w[m] = e^{-2 pi i m / n}
};

Plan make_plan(int n) {
  Plan p;
  p.n = n;
  int m = n;
  for (int r : {4, 2, 3, 5})
    while (m % r == 0) {
      p.rad.push_back(r);
      m /= r;
    }
  for (int q = 7; m > 1; q++)
    while (m % q == 0) {
      p.rad.push_back(q);
      m /= q;
    }
  p.w.resize(n);
  for (int i = 0; i < n; i++) p.w[i] = cd(cos(2.0 * kPi * i / n), -sin(2.0 * kPi * i / n));
  return p;
}

inline cd rot(cd a, bool inv) { return inv ? cd(-a.imag(), a.real()) : cd(a.imag(), -a.real()); }  // +-i a

// One Stockham pass of radix R, span Ns: src -> dst.
void pass(const Plan& P, int R, int Ns, const cd* src, cd* dst, bool inv) {
  const int n = P.n, nb = n / R, stw = n / (Ns * R);
  cd v[64], o[64];
  for (int j = 0; j < nb; j++) {
    const int k = j % Ns;
    for (int t = 0; t < R; t++) {
      cd a = src[j + t * nb];
      if (t && k) {
        cd w = P.w[(t * k * stw) % n];
        if (inv) w = std::conj(w);
        a *= w;
      }
      v[t] = a;
    }
    if (R == 2) {
      o[0] = v[0] + v[1];
      o[1] = v[0] - v[1];
    } else if (R == 4) {
      const cd s0 = v[0] + v[2], d0 = v[0] - v[2], s1 = v[1] + v[3], d1 = rot(v[1] - v[3], inv);
      o[0] = s0 + s1;
      o[2] = s0 - s1;
      o[1] = d0 + d1;
      o[3] = d0 - d1;
    } else if (R == 3) {
      const double s = 0.86602540378443864676;
      const cd p = v[1] + v[2], q = v[1] - v[2];
      const cd m = v[0] - 0.5 * p, r = rot(q * s, inv);
      o[0] = v[0] + p;
      o[1] = m + r;
      o[2] = m - r;
    } else {
      for (int u = 0; u < R; u++) {
        cd acc = 0;
        for (int t = 0; t < R; t++) {
          cd w = P.w[((long)u * t * (n / R)) % n];
          if (inv) w = std::conj(w);
          acc += v[t] * w;
        }
        o[u] = acc;
      }
    }
    const int base = (j / Ns) * Ns * R + k;
    for (int t = 0; t < R; t++) dst[base + t * Ns] = o[t];
  }
}

// Unnormalised DFT of one contiguous line (forward e^{-i}, inverse e^{+i}); a holds
// the line in and out, b is scratch of the same length.
void fft_line(const Plan& P, cd* a, cd* b, bool inv) {
  int Ns = 1;
  cd *s = a, *d = b;
  for (int r : P.rad) {
    pass(P, r, Ns, s, d, inv);
    std::swap(s, d);
    Ns *= r;
  }
  if (s != a) memcpy(a, s, sizeof(cd) * P.n);
}

struct Grid {
  int Nx, Ny, Nz;
  long N;
  Plan px, py, pz;
};

// 3-D DFT of one component (x fastest), unnormalised.
void fft3(const Grid& g, cd* f, bool inv) {
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  constexpr int B = 8;  // lines gathered per strided batch
#pragma omp parallel
  {
    const int L = std::max(Nx, std::max(Ny, Nz));
    std::vector<cd> buf((size_t)B * L), tmp(L);
#pragma omp for schedule(static)
    for (long yz = 0; yz < (long)Ny * Nz; yz++) fft_line(g.px, f + yz * Nx, tmp.data(), inv);
#pragma omp for schedule(static) collapse(2)
    for (int z = 0; z < Nz; z++)
      for (int x0 = 0; x0 < Nx; x0 += B) {
        const int nb = std::min(B, Nx - x0);
        cd* base = f + (long)z * Nx * Ny + x0;
        for (int y = 0; y < Ny; y++)
          for (int q = 0; q < nb; q++) buf[(size_t)q * Ny + y] = base[(long)y * Nx + q];
        for (int q = 0; q < nb; q++) fft_line(g.py, buf.data() + (size_t)q * Ny, tmp.data(), inv);
        for (int y = 0; y < Ny; y++)
          for (int q = 0; q < nb; q++) base[(long)y * Nx + q] = buf[(size_t)q * Ny + y];
      }
#pragma omp for schedule(static) collapse(2)
    for (int y = 0; y < Ny; y++)
      for (int x0 = 0; x0 < Nx; x0 += B) {
        const int nb = std::min(B, Nx - x0);
        cd* base = f + (long)y * Nx + x0;
        const long sz = (long)Nx * Ny;
        for (int z = 0; z < Nz; z++)
          for (int q = 0; q < nb; q++) buf[(size_t)q * Nz + z] = base[z * sz + q];
        for (int q = 0; q < nb; q++) fft_line(g.pz, buf.data() + (size_t)q * Nz, tmp.data(), inv);
        for (int z = 0; z < Nz; z++)
          for (int q = 0; q < nb; q++) base[z * sz + q] = buf[(size_t)q * Nz + z];
      }
  }
}

// ------------------------------------------------------------------ operator
struct Op {
  const Grid* g;
  long Nd, off;                 // Nd = N or N - 1 (Gamma), off = N - Nd
  std::vector<cd> P;            // Pi_Qr columns, [6][Nd] (FAME_Matrix_Lambdas.cu:184-244)
  std::vector<double> lq_sqrt;  // sqrt(Lambda_q), [Nd]
  const double* invB;           // 1/eps, 3N
  std::vector<cd> T;            // 3-component field, 3N
};

// Construct_Lambdas_Simple for wave vector k (theta_d = k . a_d, no 2 pi).
void setup_op(Op& o, const Grid& g, const double* a, const double* h, const double* k, const double* invB) {
  o.g = &g;
  o.invB = invB;
  const double th[3] = {k[0] * a[0] + k[1] * a[1] + k[2] * a[2], k[0] * a[3] + k[1] * a[4] + k[2] * a[5],
                        k[0] * a[6] + k[1] * a[7] + k[2] * a[8]};
  const double nrm = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
  o.Nd = nrm < 1e-4 ? g.N - 1 : g.N;  // FAME_Matrix_Lambdas.cu:157-169
  o.off = g.N - o.Nd;
  auto lam = [&](int m, int n, double t, double hh) {
    const double ph = 2.0 * kPi * (m + t) / n;
    return cd((cos(ph) - 1.0) / hh, sin(ph) / hh);
  };
  std::vector<cd> lx(g.Nx), ly(g.Ny), lz(g.Nz);
  for (int i = 0; i < g.Nx; i++) lx[i] = lam(i, g.Nx, th[0], h[0]);
  for (int i = 0; i < g.Ny; i++) ly[i] = lam(i, g.Ny, th[1], h[1]);
  for (int i = 0; i < g.Nz; i++) lz[i] = lam(i, g.Nz, th[2], h[2]);
  o.P.assign(6 * o.Nd, 0);
  o.lq_sqrt.assign(o.Nd, 0);
  o.T.assign(3 * g.N, 0);
  const double al = 3.0, be = 5.0;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < o.Nd; i++) {
    const long fi = i + o.off;
    const int x = (int)(fi % g.Nx), y = (int)((fi / g.Nx) % g.Ny), z = (int)(fi / ((long)g.Nx * g.Ny));
    const cd Lx = lx[x], Ly = ly[y], Lz = lz[z];
    const double Lq = std::norm(Lx) + std::norm(Ly) + std::norm(Lz);
    const cd t1 = be * Lz - Ly, t2 = Lx - al * Lz, t3 = al * Ly - be * Lx;
    const double n2 = std::norm(t1) + std::norm(t2) + std::norm(t3);
    const double s1 = sqrt(n2 * Lq), s2 = sqrt(n2);
    o.P[0 * o.Nd + i] = (t3 * std::conj(Ly) - t2 * std::conj(Lz)) / s1;
    o.P[1 * o.Nd + i] = (t1 * std::conj(Lz) - t3 * std::conj(Lx)) / s1;
    o.P[2 * o.Nd + i] = (t2 * std::conj(Lx) - t1 * std::conj(Ly)) / s1;
    o.P[3 * o.Nd + i] = std::conj(t1) / s2;
    o.P[4 * o.Nd + i] = std::conj(t2) / s2;
    o.P[5 * o.Nd + i] = std::conj(t3) / s2;
    o.lq_sqrt[i] = sqrt(Lq);
  }
}

// y = Q_r^* B^-1 Q_r x  (x, y: 2 Nd)
void qbq(Op& o, const cd* x, cd* y) {
  const Grid& g = *o.g;
  const long N = g.N, Nd = o.Nd, off = o.off;
  cd* T = o.T.data();
#pragma omp parallel for schedule(static)
  for (long fi = 0; fi < N; fi++) {
    if (fi < off) {
      for (int c = 0; c < 3; c++) T[c * N + fi] = 0;
      continue;
    }
    const long i = fi - off;
    for (int c = 0; c < 3; c++) T[c * N + fi] = o.P[c * Nd + i] * x[i] + o.P[(3 + c) * Nd + i] * x[Nd + i];
  }
  for (int c = 0; c < 3; c++) fft3(g, T + c * N, true);
  const double invN = 1.0 / (double)N;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < 3 * N; e++) T[e] *= o.invB[e] * invN;
  for (int c = 0; c < 3; c++) fft3(g, T + c * N, false);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < Nd; i++) {
    const long fi = i + off;
    cd a = 0, b = 0;
    for (int c = 0; c < 3; c++) {
      a += std::conj(o.P[c * Nd + i]) * T[c * N + fi];
      b += std::conj(o.P[(3 + c) * Nd + i]) * T[c * N + fi];
    }
    y[i] = a;
    y[Nd + i] = b;
  }
}

cd dotc(const cd* a, const cd* b, long n) {
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
  for (long i = 0; i < n; i++) {
    const cd v = std::conj(a[i]) * b[i];
    re += v.real();
    im += v.imag();
  }
  return cd(re, im);
}

// CG.cu:5-88 on QBQ: returns the reference's counter k (m products -> m + 1).
int cg(Op& o, const cd* rhs, cd* x, double tol, int maxit, std::vector<cd>& r, std::vector<cd>& p,
       std::vector<cd>& Ap) {
  const long n = 2 * o.Nd;
  for (long i = 0; i < n; i++) {
    x[i] = 0;
    r[i] = rhs[i];
  }
  double r1 = dotc(r.data(), r.data(), n).real(), r0 = r1;
  int k = 1;
  while (r1 > tol * tol && k <= maxit) {
    if (k > 1) {
      const double b = r1 / r0;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; i++) p[i] = r[i] + b * p[i];
    } else {
      for (long i = 0; i < n; i++) p[i] = r[i];
    }
    qbq(o, p.data(), Ap.data());
    const cd dot = dotc(p.data(), Ap.data(), n);
    const cd a = r1 / dot;
    double acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * Ap[i];
      acc += std::norm(r[i]);
    }
    r0 = r1;
    r1 = acc;
    k++;
  }
  return k;
}

struct Counters {
  long ls_iter = 0;
  int es_iter = 0;
};

struct Solver {
  Op& o;
  double tol;
  int maxit;
  Counters cnt;
  std::vector<cd> rhs, r, p, Ap, y;
  explicit Solver(Op& op, double t, int m) : o(op), tol(t), maxit(m) {
    const long n = 2 * o.Nd;
    rhs.resize(n);
    r.resize(n);
    p.resize(n);
    Ap.resize(n);
    y.resize(n);
  }
  // w = A_r^-1 u (invAr.cu:8-48)
  void invAr(const cd* u, cd* w) {
    const long Nd = o.Nd, n = 2 * Nd;
    for (long i = 0; i < n; i++) rhs[i] = u[i] / o.lq_sqrt[i < Nd ? i : i - Nd];
    cnt.ls_iter += cg(o, rhs.data(), y.data(), tol, maxit, r, p, Ap);
    cnt.es_iter++;
    for (long i = 0; i < n; i++) w[i] = y[i] / o.lq_sqrt[i < Nd ? i : i - Nd];
  }
};

// ------------------------------------------------------------------ Lanczos
void given_rotation(double a, double b, double& c, double& s, double& r) {
  double t, u;
  if (fabs(a) > fabs(b)) {
    t = b / a;
    u = (fabs(a) / a) * sqrt(1 + t * t);
    c = 1.0 / u;
    s = c * t;
    r = a * u;
    s = -s;
  } else {
    t = a / b;
    u = (fabs(b) / b) * sqrt(1 + t * t);
    s = 1.0 / u;
    c = s * t;
    r = b * u;
    s = -s;
  }
}

// GVqrrq_g: one shifted QR step on the leading n x n tridiagonal, in place.
void gvqrrq(double* T0, double* T1, double shift, int n, std::vector<double>& c, std::vector<double>& s) {
  c.assign(std::max(n - 1, 0), 0.0);
  s.assign(std::max(n - 1, 0), 0.0);
  std::vector<double> T2(std::max(n - 2, 1), 0.0), T3(T1, T1 + std::max(n - 1, 0));
  for (int i = 0; i < n; i++) T0[i] -= shift;
  for (int i = 0; i < n - 1; i++) {
    double r;
    given_rotation(T0[i], T1[i], c[i], s[i], r);
    T0[i] = r;
    T1[i] = 0.0;
    const double a = T3[i], b = T0[i + 1];
    T3[i] = c[i] * a - s[i] * b;
    T0[i + 1] = s[i] * a + c[i] * b;
    if (i < n - 2) {
      T2[i] = -s[i] * T3[i + 1];
      T3[i + 1] = c[i] * T3[i + 1];
    }
  }
  {
    const double R0 = T0[0], R1 = T3[0], R2 = T1[0], R3 = T0[1];
    T0[0] = c[0] * R0 - s[0] * R1;
    T3[0] = s[0] * R0 + c[0] * R1;
    T1[0] = c[0] * R2 - s[0] * R3;
    T0[1] = s[0] * R2 + c[0] * R3;
  }
  for (int i = 1; i < n - 1; i++) {
    const double R[6] = {T3[i - 1], T2[i - 1], T0[i], T3[i], T1[i], T0[i + 1]};
    T3[i - 1] = c[i] * R[0] - s[i] * R[1];
    T2[i - 1] = s[i] * R[0] + c[i] * R[1];
    T0[i] = c[i] * R[2] - s[i] * R[3];
    T3[i] = s[i] * R[2] + c[i] * R[3];
    T1[i] = c[i] * R[4] - s[i] * R[5];
    T0[i + 1] = s[i] * R[4] + c[i] * R[5];
  }
  for (int i = 0; i < n - 1; i++) T1[i] = (T1[i] + T3[i]) / 2.0;
  for (int i = 0; i < n; i++) T0[i] += shift;
}

// cublasZdrot on columns: x' = c x + s y, y' = -s x + c y
void zdrot(cd* x, cd* y, long n, double c, double s) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    const cd a = x[i], b = y[i];
    x[i] = c * a + s * b;
    y[i] = -s * a + c * b;
  }
}

// Eigenpairs of the symmetric tridiagonal (d, e), eigenvalues descending, Z column
// major (z[r + c n]).  Implicit QL with Wilkinson shifts.
bool tridiag_eig(int n, const double* d0, const double* e0, std::vector<double>& w, std::vector<double>& z) {
  std::vector<double> d(d0, d0 + n), e(n, 0.0);
  for (int i = 0; i + 1 < n; i++) e[i] = e0[i];
  z.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) z[i + (size_t)i * n] = 1.0;
  for (int l = 0; l < n; l++) {
    int iter = 0, m;
    do {
      for (m = l; m < n - 1; m++) {
        const double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= 1e-300 || fabs(e[m]) <= 2.2e-16 * dd) break;
      }
      if (m != l) {
        if (iter++ == 60) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; i--) {
          double f = s * e[i], b = c * e[i];
          r = hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; k++) {
            f = z[k + (size_t)(i + 1) * n];
            z[k + (size_t)(i + 1) * n] = s * z[k + (size_t)i * n] + c * f;
            z[k + (size_t)i * n] = c * z[k + (size_t)i * n] - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; i++) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] > d[b]; });
  w.resize(n);
  std::vector<double> zz((size_t)n * n);
  for (int c = 0; c < n; c++) {
    w[c] = d[ord[c]];
    for (int r = 0; r < n; r++) zz[r + (size_t)c * n] = z[r + (size_t)ord[c] * n];
  }
  z.swap(zz);
  return true;
}

struct Lanczos {
  Solver& S;
  long M;
  int nwant, nstep;
  std::vector<cd> U;  // M x (nstep + 1), column major
  std::vector<double> T0, T1;
  cd* col(int j) { return U.data() + (size_t)j * M; }
  Lanczos(Solver& s, int nw, int ns) : S(s), M(2 * s.o.Nd), nwant(nw), nstep(ns) {
    U.assign((size_t)M * (ns + 1), 0);
    T0.assign(ns, 0.0);
    T1.assign(ns, 0.0);
  }
  double norm(const cd* a) { return sqrt(dotc(a, a, M).real()); }
  void scale(cd* a, double s) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) a[i] *= s;
  }
  void axpy(cd al, const cd* x, cd* y) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) y[i] += al * x[i];
  }
  // Lanczos_decomp_gpu (:7-91): one MGS pass after normalisation, no renormalisation
  void step(int j) {
    cd* w = col(j + 1);
    S.invAr(col(j), w);
    T0[j] = dotc(w, col(j), M).real();
    axpy(-T0[j], col(j), w);
    if (j > 0) axpy(-T1[j - 1], col(j - 1), w);
    T1[j] = norm(w);
    scale(w, 1.0 / T1[j]);
    for (int i = 0; i <= j; i++) axpy(-dotc(col(i), w, M), col(i), w);
  }
  void decomp(bool init) {
    int start = nwant;
    if (!init) {
      cd* u = col(0);
      for (long i = 0; i < M; i++) u[i] = 0;
      u[M - 1] = 1.0;
      start = 0;
    }
    for (int j = start; j < nstep; j++) step(j);
  }
  // Lanczos_LockPurge_gpu (:7-48)
  void lock_purge(const std::vector<double>& LT0) {
    std::vector<double> c, s;
    for (int j = 0; j < nstep - nwant; j++) {
      const int n = nstep - j;
      gvqrrq(T0.data(), T1.data(), LT0[nwant + j], n, c, s);
      for (int jj = 0; jj < n - 1; jj++) zdrot(col(jj + 1), col(jj), M, c[jj], s[jj]);
      const int jj = n - 1;
      s[jj - 1] *= T1[jj];
      zdrot(col(jj + 1), col(jj), M, T1[jj - 1], s[jj - 1]);
      T1[jj - 1] = norm(col(jj));
      scale(col(jj), 1.0 / T1[jj - 1]);
      T0[jj] = 0.0;
      T1[jj] = 0.0;
      cd* u = col(jj + 1);
      for (long i = 0; i < M; i++) u[i] = 0;
    }
  }
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

// Full plain-method solve of nk wave vectors on a Simple lattice.  grid[3], mesh_len[3],
// lattice_vec_a[9] (rows a1, a2, a3), B: 3N edge permittivities, k_xyz: nk x 3.
// Outputs (nk x nwant frequencies, with the Gamma patch), per-k ls_iter / es_iter /
// restarts / converged (Lanczos), wall seconds per k.  nthreads <= 0: all cores.
// Returns 0, or 1 when a tridiagonal eigensolve failed.
int fame_cpu_solve(const int* grid, const double* mesh_len, const double* lattice_vec_a, const double* B,
                   const double* k_xyz, int nk, int nwant, int nstep, double es_tol, int es_maxit, double ls_tol,
                   int ls_maxit, int nthreads, double* freq_out, int* ls_iter, int* es_iter, int* restarts,
                   int* converged, double* wall_s) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Grid g;
  g.Nx = grid[0];
  g.Ny = grid[1];
  g.Nz = grid[2];
  g.N = (long)g.Nx * g.Ny * g.Nz;
  g.px = make_plan(g.Nx);
  g.py = make_plan(g.Ny);
  g.pz = make_plan(g.Nz);
  std::vector<double> invB(3 * g.N);
  for (long i = 0; i < 3 * g.N; i++) invB[i] = 1.0 / B[i];
  for (int q = 0; q < nk; q++) {
    const double t0 = now_s();
    Op o;
    setup_op(o, g, lattice_vec_a, mesh_len, k_xyz + 3 * q, invB.data());
    const bool gamma = o.Nd == g.N - 1;
    const int nw = nwant;
    Solver S(o, ls_tol, ls_maxit);
    Lanczos L(S, nw, nstep);
    L.decomp(false);
    std::vector<double> w, z;
    int it = 1;
    bool conv_all = false;
    while (it <= es_maxit) {
      std::vector<double> e(L.T1.begin(), L.T1.end() - 1);
      if (!tridiag_eig(nstep, L.T0.data(), e.data(), w, z)) return 1;
      int conv = 0;
      for (int i = 0; i < nw; i++) {
        if (L.T1[nstep - 1] * fabs(z[(nstep - 1) + (size_t)i * nstep]) < es_tol)
          conv++;
        else
          break;
      }
      if (conv == nw) {
        conv_all = true;
        break;
      }
      L.lock_purge(w);
      L.decomp(true);
      it++;
    }
    double* f = freq_out + (size_t)q * nwant;
    if (gamma) {  // bands shift up by two, w0 = w1 = 0 (FAME_Fast_Algorithms_Isotropic.cu:61-79)
      f[0] = f[1] = 0.0;
      for (int i = 0; i + 2 < nw; i++) f[2 + i] = sqrt(1.0 / w[i]);
    } else {
      for (int i = 0; i < nw; i++) f[i] = sqrt(1.0 / w[i]);
    }
    ls_iter[q] = (int)S.cnt.ls_iter;
    es_iter[q] = S.cnt.es_iter;
    restarts[q] = it - 1;
    converged[q] = conv_all ? 1 : 0;
    wall_s[q] = now_s() - t0;
  }
  return 0;
}

// Time of the plain method's building blocks at one wave vector: seconds per CG
// iteration (one QBQ plus the CG vector updates and dots, mean over `iters`
// iterations of a CG solve from a fixed pseudo-random right-hand side) and per
// Lanczos step j (the A_r^-1-free part: alpha, two axpys, the norm and the j+1
// reorthogonalisation dot/axpy pairs), at j = jstep.
int fame_cpu_time(const int* grid, const double* mesh_len, const double* lattice_vec_a, const double* B,
                  const double* k, int iters, int jstep, int nthreads, double* s_per_cg_iter, double* s_per_lz_step) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Grid g;
  g.Nx = grid[0];
  g.Ny = grid[1];
  g.Nz = grid[2];
  g.N = (long)g.Nx * g.Ny * g.Nz;
  g.px = make_plan(g.Nx);
  g.py = make_plan(g.Ny);
  g.pz = make_plan(g.Nz);
  std::vector<double> invB(3 * g.N);
  for (long i = 0; i < 3 * g.N; i++) invB[i] = 1.0 / B[i];
  Op o;
  setup_op(o, g, lattice_vec_a, mesh_len, k, invB.data());
  const long n = 2 * o.Nd;
  std::vector<cd> rhs(n), x(n), r(n), p(n), Ap(n);
  uint64_t st = 12345;
  for (long i = 0; i < n; i++) {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    rhs[i] = cd((double)(st >> 11) / 9007199254740992.0 - 0.5, 0.0);
  }
  // CG to a tolerance it cannot reach, capped at `iters` products
  const double t0 = now_s();
  const int kk = cg(o, rhs.data(), x.data(), 0.0, iters, r, p, Ap);
  *s_per_cg_iter = (now_s() - t0) / std::max(1, kk - 1);
  Solver S(o, 0.0, 1);
  Lanczos L(S, 1, jstep + 1);
  for (int j = 0; j <= jstep + 1; j++)
    for (long i = 0; i < n; i++) L.col(j)[i] = rhs[(i + 7 * j) % n];
  const double t1 = now_s();
  cd* w = L.col(jstep + 1);
  L.T0[jstep] = dotc(w, L.col(jstep), n).real();
  L.axpy(-L.T0[jstep], L.col(jstep), w);
  L.axpy(-0.5, L.col(jstep - 1 >= 0 ? jstep - 1 : 0), w);
  L.T1[jstep] = L.norm(w);
  L.scale(w, 1.0 / L.T1[jstep]);
  for (int i = 0; i <= jstep; i++) L.axpy(-dotc(L.col(i), w, n), L.col(i), w);
  *s_per_lz_step = now_s() - t1;
  return 0;
}

int fame_cpu_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
