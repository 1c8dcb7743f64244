// Host-side geometry shared by the solver context (solver.cu) and the
// allocation-free operator (qbq_static.cu): FFT plans of the three axes, the
// plane/pencil layout, the per-k table offsets, the Bloch phases theta and the
// reduced size Nd.  Both translation units build their Geom here, so the layout the
// kernels index is the same in both.
#pragma once
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "../../include/fame_b200.h"
#include "op_kernels_decl.h"

namespace fame {

// Radix order of a plan: the listed radices as often as they divide n, in order, then
// the remaining prime factors from 17 up.  kRadixOrders[0] (largest power-of-two
// radix first: fewest passes) is the default; the plan tuner tries the others.
constexpr int kNumRadixOrder = 8;
constexpr int kNumRadixOrders = 4;
constexpr int kRadixOrders[kNumRadixOrders][kNumRadixOrder] = {
    {8, 4, 2, 5, 3, 7, 11, 13},  // 64 = 8 8, 96 = 8 4 3
    {4, 2, 8, 3, 5, 7, 11, 13},  // 64 = 4 4 4, 96 = 4 4 2 3
    {8, 2, 4, 3, 5, 7, 11, 13},  // 64 = 8 8, 32 = 8 2 2
    {3, 5, 7, 11, 13, 4, 8, 2},  // odd radices first: 96 = 3 4 4 2
};
constexpr const int* kRadixOrder = kRadixOrders[0];

inline bool factor_axis(int n, AxisPlan& p, const int* order = kRadixOrder, int norder = kNumRadixOrder) {
  p.n = n;
  p.npass = 0;
  int m = n;
  for (int i = 0; i < norder; i++) {
    const int r = order[i];
    while (m % r == 0) {
      if (p.npass >= kMaxPasses) return false;
      p.radix[p.npass++] = r;
      m /= r;
    }
  }
  for (int q = 17; m > 1 && q <= m; q++) {
    while (m % q == 0) {
      if (p.npass >= kMaxPasses) return false;
      p.radix[p.npass++] = q;
      m /= q;
    }
  }
  if (n == 1) p.npass = 0;
  return m == 1;
}

// Lengths, plans, table and twiddle offsets of lattice L.  Simple lattices walk
// (slow, mid, fast) = (z, y, x); General lattices (x, y, z) in frequency (the
// reference's z-fastest order, FAME_Main/FAME_Matrix_Lambdas.cu:317).  Returns a
// FAME_* status; err receives the reason.  max_points bounds N.
inline int layout_geom(const fame_lattice& L, Geom& g, long max_points, std::string& err, int radix_order = 0) {
  memset(&g, 0, sizeof(g));
  g.Nx = L.grid[0];
  g.Ny = L.grid[1];
  g.Nz = L.grid[2];
  if (g.Nx < 2 || g.Ny < 2 || g.Nz < 2) {
    err = "grid dimensions must be >= 2";
    return FAME_ERR_BAD_INPUT;
  }
  const long N = (long)g.Nx * g.Ny * g.Nz;
  if (N > max_points) {
    err = "grid too large";
    return FAME_ERR_BAD_INPUT;
  }
  g.N = (int)N;
  g.general = L.simple ? 0 : 1;
  g.hx = L.mesh_len[0];
  g.hy = L.mesh_len[1];
  g.hz = L.mesh_len[2];
  g.ihz = 1.0 / g.hz;
  g.tnz = 2.0 / g.Nz;
  g.Ls = g.general ? g.Nx : g.Nz;
  g.Lm = g.Ny;
  g.Lf = g.general ? g.Nz : g.Nx;
  g.P = g.Lm * g.Lf;
  g.S = g.Lf | 1;  // odd row pitch: bank-conflict-free passes along both plane axes
  const int* ord = kRadixOrders[radix_order];
  if (!factor_axis(g.Lf, g.pf, ord) || !factor_axis(g.Lm, g.pm, ord) || !factor_axis(g.Ls, g.ps, ord)) {
    err = "axis length needs more than 10 FFT passes";
    return FAME_ERR_UNSUPPORTED;
  }
  if (plane_smem_bytes<double>(g.Lf, g.Lm, g.S) > 227 * 1024) {
    err = "plane " + std::to_string(g.Lm) + "x" + std::to_string(g.Lf) + " exceeds one CTA";
    return FAME_ERR_UNSUPPORTED;
  }
  int o = 0;
  if (!g.general) {
    g.oLx = o; o += g.Nx;
    g.oLy = o; o += g.Ny;
    g.oLz = o; o += g.Nz;
    g.oDx = o; o += g.Nx;
    g.oDy = o; o += g.Ny;
    g.oDz = o; o += g.Nz;
  } else {
    g.oLx = o; o += g.Nx;
    g.oLy = o; o += g.Nx * g.Ny;
    g.oExy = o; o += g.Nx * g.Ny;
    g.oWz = o; o += g.Nz;
    g.oDky = o; o += g.Nx * g.Ny;
    g.oPhi = o; o += g.Nx * g.Ny;
    g.oDkx = o; o += g.Nx;
  }
  g.tab_stride = (o + 7) / 8 * 8;
  // forward twiddle tables e^{-2 pi i m / n} of the fast, mid and slow axes, back to back
  g.twf = 0;
  g.twm = g.Lf;
  g.tws = g.Lf + g.Lm;
  return FAME_OK;
}

// fft_lines level (kernel instantiation) the three axis plans need.
inline int geom_level(const Geom& g) {
  return std::max(plan_level(g.pf), std::max(plan_level(g.pm), plan_level(g.ps)));
}
// ... the plane stages' axes (fast, mid) and the pencil stage's axis (slow) alone: each
// stage kernel runs the lowest level its own axes need (fewer registers, no spills
// from passes it never runs)
inline int plane_level(const Geom& g) { return std::max(plan_level(g.pf), plan_level(g.pm)); }
inline int pencil_level(const Geom& g) { return plan_level(g.ps); }

// Threads of a runtime-geometry plane CTA: about 8 plane elements per thread, at most
// 512; at most 256 when two planes of precision R fit one SM's shared memory (more,
// smaller CTAs per SM hide the latency of the staged passes better), except FP64
// planes with the prime pass (level 2), whose 128-register budget admits one CTA per SM.
template <typename R>
inline int plane_threads_rule(const Geom& g, int level) {
  const int pt = std::min(512, std::max(64, ((g.P + 7) / 8 + 31) / 32 * 32));
  const size_t kSmemSM = 227 * 1024;
  const bool two = 2 * plane_smem_bytes<R>(g.Lf, g.Lm, g.S) <= kSmemSM;
  if (sizeof(R) == 8 && level >= 2) return pt;
  return two ? std::min(pt, 256) : pt;
}

// theta_x, theta_y(xy), theta_z(xyz) of wave vector k (FAME_Main/FAME_Matrix_Lambdas.cu:43-70)
inline void lattice_thetas(const fame_lattice& L, const double* k, double th[3]) {
  const double* a = L.lattice_vec_a;
  auto dot = [&](const double* v) { return k[0] * v[0] + k[1] * v[1] + k[2] * v[2]; };
  th[0] = dot(a);
  if (L.simple) {
    th[1] = dot(a + 3);
    th[2] = dot(a + 6);
    return;
  }
  double c1 = 0.0;
  if (a[3] > 0)
    c1 = -(double)L.m[0] / (double)L.grid[0];
  else if (a[3] < 0)
    c1 = 1. - (double)L.m[0] / (double)L.grid[0];
  const double c2 = (double)L.m[2] / (double)L.grid[1];
  const double c3 = (double)L.m[1] / (double)L.grid[0];
  double a2h[3], a3h[3];
  for (int i = 0; i < 3; i++) a2h[i] = c1 * a[i] + a[3 + i];
  for (int i = 0; i < 3; i++) a3h[i] = a[6 + i] - c2 * a2h[i] - c3 * a[i] + L.t1[i];
  th[1] = dot(a2h);
  th[2] = dot(a3h);
}

// Nd of wave vector k: N - 1 at the Gamma point, |k| below 1e-4 for Simple lattices
// (FAME_Main/FAME_Matrix_Lambdas.cu:157) and 1e-3 for General ones (:406), else N.
inline int lattice_reduced_size(const fame_lattice& L, const double* k) {
  const int N = L.grid[0] * L.grid[1] * L.grid[2];
  const double nrm = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
  return nrm < (L.simple ? 1e-4 : 1e-3) ? N - 1 : N;
}

// The slot of wave vector k.
inline Slot make_slot(const fame_lattice& L, const double* k) {
  Slot sl;
  memset(&sl, 0, sizeof(sl));
  lattice_thetas(L, k, sl.th);
  sl.Nd = lattice_reduced_size(L, k);
  sl.off = L.grid[0] * L.grid[1] * L.grid[2] - sl.Nd;
  sl.active = 1;
  return sl;
}

}  // namespace fame
