// Mixed-radix FFT passes on data staged in shared memory.
//
// Algorithm: the Stockham autosort formulation of Govindaraju, Lloyd, Dotsenko,
// Smith and Manferdelli, "High Performance Discrete Fourier Transforms on
// Graphics Processors" (SC'08): for span Ns = 1, r1, r1*r2, ... each pass of
// radix R takes butterfly j's inputs x[j + t*n/R] (t < R), multiplies input t by
// w^(t*(j mod Ns)) with w = e^(-/+ 2*pi*i/(Ns*R)), applies an R-point DFT and
// writes output t to (j/Ns)*Ns*R + (j mod Ns) + t*Ns.  The result is in natural
// order after the last pass.  Forward transforms use e^{-i...} (cuFFT
// CUFFT_FORWARD, which the reference's FFT_CUDA uses, FAME_Main/FAME_FFT_CUDA.cu:31)
// and inverse transforms e^{+i...}, both unnormalised.
//
// A "tile" holds `nl` lines of length n; element m of line l sits at
// buf[l*ls + m*es].  Every pass is register staged: each thread reads all inputs
// of its butterflies, the block synchronises, then every thread writes, so the
// transform runs in place in one shared buffer.  Radices 2,3,4,5,7,8 (and odd
// 11, 13 through the symmetric-pair DFT) use butterflies; any other factor (a
// large prime such as 23 or 107) uses a register-blocked symmetric-pair DFT pass
// (prime_pass), or an output-stationary pass where each thread forms its outputs
// as length-R sums when a line needs more threads than the block has.
#pragma once
#include "fame_common.cuh"

namespace fame {

constexpr int kMaxPasses = 10;

struct AxisPlan {
  int n;
  int npass;
  int radix[kMaxPasses];
};

// cos/sin(2*pi*m/R) for the odd radices handled by the symmetric-pair DFT
// (mathematical constants, correctly rounded to double).  m is a compile-time
// constant at every use, so each call folds to a literal.
template <int RAD> struct OddTab;
template <> struct OddTab<5> {
  __device__ __forceinline__ static constexpr double c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.30901699437494745 : m == 2 ? -0.8090169943749475 : m == 3 ? -0.8090169943749475 : 0.30901699437494745;
  }
  __device__ __forceinline__ static constexpr double s(int m) {
    return m == 0 ? 0.0 : m == 1 ? 0.9510565162951535 : m == 2 ? 0.5877852522924731 : m == 3 ? -0.5877852522924731 : -0.9510565162951535;
  }
};
template <> struct OddTab<7> {
  __device__ __forceinline__ static constexpr double c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.6234898018587335 : m == 2 ? -0.2225209339563144 : m == 3 ? -0.9009688679024191 : m == 4 ? -0.9009688679024191 : m == 5 ? -0.2225209339563144 : 0.6234898018587335;
  }
  __device__ __forceinline__ static constexpr double s(int m) {
    return m == 0 ? 0.0 : m == 1 ? 0.7818314824680298 : m == 2 ? 0.9749279121818236 : m == 3 ? 0.4338837391175581 : m == 4 ? -0.4338837391175581 : m == 5 ? -0.9749279121818236 : -0.7818314824680298;
  }
};
template <> struct OddTab<11> {
  __device__ __forceinline__ static constexpr double c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.8412535328311812 : m == 2 ? 0.41541501300188644 : m == 3 ? -0.14231483827328514 : m == 4 ? -0.6548607339452851 : m == 5 ? -0.9594929736144974 : m == 6 ? -0.9594929736144974 : m == 7 ? -0.6548607339452851 : m == 8 ? -0.14231483827328514 : m == 9 ? 0.41541501300188644 : 0.8412535328311812;
  }
  __device__ __forceinline__ static constexpr double s(int m) {
    return m == 0 ? 0.0 : m == 1 ? 0.5406408174555976 : m == 2 ? 0.9096319953545183 : m == 3 ? 0.9898214418809327 : m == 4 ? 0.7557495743542583 : m == 5 ? 0.28173255684142967 : m == 6 ? -0.28173255684142967 : m == 7 ? -0.7557495743542583 : m == 8 ? -0.9898214418809327 : m == 9 ? -0.9096319953545183 : -0.5406408174555976;
  }
};
template <> struct OddTab<13> {
  __device__ __forceinline__ static constexpr double c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.8854560256532099 : m == 2 ? 0.5680647467311558 : m == 3 ? 0.12053668025532305 : m == 4 ? -0.3546048870425356 : m == 5 ? -0.7485107481711011 : m == 6 ? -0.970941817426052 : m == 7 ? -0.970941817426052 : m == 8 ? -0.7485107481711011 : m == 9 ? -0.3546048870425356 : m == 10 ? 0.12053668025532305 : m == 11 ? 0.5680647467311558 : 0.8854560256532099;
  }
  __device__ __forceinline__ static constexpr double s(int m) {
    return m == 0 ? 0.0 : m == 1 ? 0.46472317204376856 : m == 2 ? 0.8229838658936564 : m == 3 ? 0.992708874098054 : m == 4 ? 0.9350162426854148 : m == 5 ? 0.6631226582407952 : m == 6 ? 0.23931566428755777 : m == 7 ? -0.23931566428755777 : m == 8 ? -0.6631226582407952 : m == 9 ? -0.9350162426854148 : m == 10 ? -0.992708874098054 : m == 11 ? -0.8229838658936564 : -0.46472317204376856;
  }
};

// multiply by -i (forward) or +i (inverse)
template <typename T> __device__ __forceinline__ T rot_mi(T a, bool inv) {
  T z;
  if (inv) {
    z.x = -a.y;
    z.y = a.x;
  } else {
    z.x = a.y;
    z.y = -a.x;
  }
  return z;
}

template <typename R, int RAD> struct Dft;

template <typename R> struct Dft<R, 2> {
  __device__ __forceinline__ static void run(cplx<R>* a, bool) {
    cplx<R> t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  }
};

template <typename R> struct Dft<R, 3> {
  __device__ __forceinline__ static void run(cplx<R>* a, bool inv) {
    const R c = (R)-0.5;
    const R s = (R)0.86602540378443864676;  // sin(2*pi/3)
    cplx<R> p = cadd(a[1], a[2]);
    cplx<R> q = csub(a[1], a[2]);
    cplx<R> m = mk<R>(a[0].x + c * p.x, a[0].y + c * p.y);
    cplx<R> r = rot_mi(cscale(q, s), inv);
    a[0] = cadd(a[0], p);
    a[1] = cadd(m, r);
    a[2] = csub(m, r);
  }
};

template <typename R> struct Dft<R, 4> {
  __device__ __forceinline__ static void run(cplx<R>* a, bool inv) {
    cplx<R> s0 = cadd(a[0], a[2]);
    cplx<R> d0 = csub(a[0], a[2]);
    cplx<R> s1 = cadd(a[1], a[3]);
    cplx<R> d1 = rot_mi(csub(a[1], a[3]), inv);
    a[0] = cadd(s0, s1);
    a[2] = csub(s0, s1);
    a[1] = cadd(d0, d1);
    a[3] = csub(d0, d1);
  }
};

template <typename R> struct Dft<R, 8> {
  __device__ __forceinline__ static void run(cplx<R>* a, bool inv) {
    const R h = (R)0.70710678118654752440;  // 1/sqrt(2)
    cplx<R> e[4] = {a[0], a[2], a[4], a[6]};
    cplx<R> o[4] = {a[1], a[3], a[5], a[7]};
    Dft<R, 4>::run(e, inv);
    Dft<R, 4>::run(o, inv);
    // twiddles w8^k for k = 1, 2, 3 (w8 = e^{-/+ i pi/4})
    cplx<R> o1 = inv ? mk<R>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                     : mk<R>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    cplx<R> o2 = rot_mi(o[2], inv);
    cplx<R> o3 = inv ? mk<R>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                     : mk<R>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    a[0] = cadd(e[0], o[0]);
    a[4] = csub(e[0], o[0]);
    a[1] = cadd(e[1], o1);
    a[5] = csub(e[1], o1);
    a[2] = cadd(e[2], o2);
    a[6] = csub(e[2], o2);
    a[3] = cadd(e[3], o3);
    a[7] = csub(e[3], o3);
  }
};

// FP32 butterflies with packed pair arithmetic (sm_100 FADD2 / FMUL2 / FFMA2: one
// instruction updates both parts of a complex value).  Same operations and roundings
// as the generic ones: a - b is formed as b * (-1) + a (exact product, one rounding).
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 pscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float2 pfma(float2 a, float s, float2 c) { return __ffma2_rn(a, make_float2(s, s), c); }

// c + s * a for a complex a and a real s, one rounding per part: one packed FFMA2 in
// FP32, two FMAs in FP64.
__device__ __forceinline__ float2 cfma_r(float2 a, float s, float2 c) { return pfma(a, s, c); }
__device__ __forceinline__ double2 cfma_r(double2 a, double s, double2 c) {
  return make_double2(fma(s, a.x, c.x), fma(s, a.y, c.y));
}

template <> struct Dft<float, 2> {
  __device__ __forceinline__ static void run(float2* a, bool) {
    const float2 t = a[0];
    a[0] = padd(t, a[1]);
    a[1] = psub(t, a[1]);
  }
};

template <> struct Dft<float, 3> {
  __device__ __forceinline__ static void run(float2* a, bool inv) {
    const float s = 0.86602540378443864676f;  // sin(2*pi/3)
    const float2 p = padd(a[1], a[2]), q = psub(a[1], a[2]);
    const float2 m = pfma(p, -0.5f, a[0]);
    a[0] = padd(a[0], p);
    // m -/+ i s q (forward) or m +/- i s q (inverse)
    if (inv) {
      a[1] = make_float2(m.x - s * q.y, m.y + s * q.x);
      a[2] = make_float2(m.x + s * q.y, m.y - s * q.x);
    } else {
      a[1] = make_float2(m.x + s * q.y, m.y - s * q.x);
      a[2] = make_float2(m.x - s * q.y, m.y + s * q.x);
    }
  }
};

template <> struct Dft<float, 4> {
  __device__ __forceinline__ static void run(float2* a, bool inv) {
    const float2 s0 = padd(a[0], a[2]), d0 = psub(a[0], a[2]);
    const float2 s1 = padd(a[1], a[3]), e = psub(a[1], a[3]);
    a[0] = padd(s0, s1);
    a[2] = psub(s0, s1);
    // d0 -/+ i e (forward) or d0 +/- i e (inverse)
    if (inv) {
      a[1] = make_float2(d0.x - e.y, d0.y + e.x);
      a[3] = make_float2(d0.x + e.y, d0.y - e.x);
    } else {
      a[1] = make_float2(d0.x + e.y, d0.y - e.x);
      a[3] = make_float2(d0.x - e.y, d0.y + e.x);
    }
  }
};

template <> struct Dft<float, 8> {
  __device__ __forceinline__ static void run(float2* a, bool inv) {
    const float h = 0.70710678118654752440f;  // 1/sqrt(2)
    float2 e[4] = {a[0], a[2], a[4], a[6]};
    float2 o[4] = {a[1], a[3], a[5], a[7]};
    Dft<float, 4>::run(e, inv);
    Dft<float, 4>::run(o, inv);
    // twiddles w8^k, k = 1, 3 (w8 = e^{-/+ i pi/4}); k = 2 is a rotation folded below
    const float2 x1 = o[1], x3 = o[3];
    const float2 o1 = inv ? pscale(make_float2(x1.x - x1.y, x1.x + x1.y), h)
                          : pscale(make_float2(x1.x + x1.y, x1.y - x1.x), h);
    const float2 o3 = inv ? pscale(make_float2(-(x3.x + x3.y), x3.x - x3.y), h)
                          : pscale(make_float2(x3.y - x3.x, -(x3.x + x3.y)), h);
    a[0] = padd(e[0], o[0]);
    a[4] = psub(e[0], o[0]);
    a[1] = padd(e[1], o1);
    a[5] = psub(e[1], o1);
    const float2 y = o[2];
    if (inv) {
      a[2] = make_float2(e[2].x - y.y, e[2].y + y.x);
      a[6] = make_float2(e[2].x + y.y, e[2].y - y.x);
    } else {
      a[2] = make_float2(e[2].x + y.y, e[2].y - y.x);
      a[6] = make_float2(e[2].x - y.y, e[2].y + y.x);
    }
    a[3] = padd(e[3], o3);
    a[7] = psub(e[3], o3);
  }
};

// Radix 12 as a prime-factor (Good-Thomas) DFT 3 x 4, no internal twiddles:
// input n = (4 n1 + 3 n2) mod 12, output k = (4 k1 + 9 k2) mod 12 with
// k1 = k mod 3, k2 = k mod 4 (Chinese remainder map).
template <typename R> struct Dft<R, 12> {
  __device__ __forceinline__ static void run(cplx<R>* a, bool inv) {
    cplx<R> y[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
#pragma unroll
      for (int n1 = 0; n1 < 3; n1++) y[n2][n1] = a[(4 * n1 + 3 * n2) % 12];
      Dft<R, 3>::run(y[n2], inv);
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
      cplx<R> z[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      Dft<R, 4>::run(z, inv);
#pragma unroll
      for (int k2 = 0; k2 < 4; k2++) a[(4 * k1 + 9 * k2) % 12] = z[k2];
    }
  }
};

// Odd radix via symmetric pairs: X_t = a0 + sum_s c(ts) (a_s + a_{R-s})
//                                       -/+ i sum_s s(ts) (a_s - a_{R-s}).
template <typename R, int RAD> struct DftOdd {
  __device__ __forceinline__ static void run(cplx<R>* a, bool inv) {
    constexpr int H = (RAD - 1) / 2;
    cplx<R> P[H], Q[H];
    cplx<R> x0 = a[0];
    cplx<R> sum = x0;
#pragma unroll
    for (int s = 1; s <= H; s++) {
      P[s - 1] = cadd(a[s], a[RAD - s]);
      Q[s - 1] = csub(a[s], a[RAD - s]);
      sum = cadd(sum, P[s - 1]);
    }
    // a[1..RAD-1] are free now (kept in P, Q): write the outputs in place
    a[0] = sum;
#pragma unroll
    for (int t = 1; t <= H; t++) {
      cplx<R> re = x0, im = mk<R>(0, 0);
#pragma unroll
      for (int s = 1; s <= H; s++) {
        const int m = (t * s) % RAD;
        const R c = (R)OddTab<RAD>::c(m), sn = (R)OddTab<RAD>::s(m);
        re = cfma_r(P[s - 1], c, re);
        im = cfma_r(Q[s - 1], sn, im);
      }
      cplx<R> r = rot_mi(im, inv);  // -i*im (forward) / +i*im (inverse)
      a[t] = cadd(re, r);
      a[RAD - t] = csub(re, r);
    }
  }
};
template <typename R> struct Dft<R, 5> : DftOdd<R, 5> {};
template <typename R> struct Dft<R, 7> : DftOdd<R, 7> {};
template <typename R> struct Dft<R, 11> : DftOdd<R, 11> {};
template <typename R> struct Dft<R, 13> : DftOdd<R, 13> {};

// Lines layout: element m of line l at buf[l*ls + m*es].  Threads are mapped
// lines-fastest: thread t works on line t mod nl, so consecutive threads touch
// words ls apart.  Lines along the contiguous axis therefore use an odd padded
// line stride (the plane row pitch), which makes every pass free of shared memory
// bank conflicts for any radix; lines across the contiguous axis have ls = 1.
struct LineSet {
  int nl, ls, es;
};

// Exact unsigned division by an invariant divisor d for n * d < 2^32:
// floor(n / d) = umulhi(n, ceil(2^32 / d)).
struct Div {
  unsigned m, d;
  __device__ __forceinline__ explicit Div(unsigned dd) : m(0xffffffffu / dd + 1u), d(dd) {}
  __device__ __forceinline__ unsigned q(unsigned n) const { return d == 1 ? n : __umulhi(n, m); }
};

// One radix-RAD Stockham pass over all lines, in place.  Every round stages the
// butterflies of G complete lines in registers (read all, barrier, write all,
// barrier): a line's outputs overwrite positions other butterflies of the same
// line still read, so a line never spans two rounds.  Thread t works on line
// l0 + t mod G and butterflies j = t / G + jstep * q (q < MAXB), with jstep * MAXB
// >= n / RAD; consecutive threads touch consecutive lines.
template <typename R, int RAD, int MAXB>
__device__ __forceinline__ void stockham_pass(cplx<R>* buf, int n, int Ns, LineSet L, const cplx<R>* tw,
                                              bool inv) {
  const int T = blockDim.x;
  const int nb = n / RAD;
  const int stw = n / (Ns * RAD);
  const int per_line = (nb + MAXB - 1) / MAXB;  // threads one line needs
  const int G = min(L.nl, max(1, T / per_line));
  const Div dg(G), dns(Ns);
  const int t = threadIdx.x;
  const int j0 = (int)dg.q(t);
  const int lt = t - j0 * G;
  const int jstep = T / G;
  for (int l0 = 0; l0 < L.nl; l0 += G) {
    const int l = l0 + lt;
    const bool live = j0 < jstep && l < L.nl;
    cplx<R>* base = buf + l * L.ls;
    cplx<R> v[MAXB][RAD];
    int dst[MAXB];
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
      const int j = j0 + jstep * q;
      dst[q] = -1;
      if (live && j < nb) {
        const int jb = (int)dns.q(j);
        const int k = j - jb * Ns;
#pragma unroll
        for (int u = 0; u < RAD; u++) {
          cplx<R> a = base[(j + u * nb) * L.es];
          if (u > 0 && k > 0) {
            cplx<R> w = tw[u * k * stw];
            if (inv) w.y = -w.y;
            a = cmul(a, w);
          }
          v[q][u] = a;
        }
        Dft<R, RAD>::run(v[q], inv);
        dst[q] = (jb * Ns * RAD + k) * L.es;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
      if (dst[q] >= 0) {
#pragma unroll
        for (int u = 0; u < RAD; u++) base[dst[q] + u * Ns * L.es] = v[q][u];
      }
    }
    __syncthreads();
  }
}

// Output-stationary DFT pass for an arbitrary radix r (used for large primes):
// rounds of G complete lines, thread t owns line l0 + t mod G and outputs
// o = t / G + ostep * q.
template <typename R, int MAXE>
__device__ __forceinline__ void generic_pass(cplx<R>* buf, int n, int r, int Ns, LineSet L, const cplx<R>* tw,
                                             bool inv) {
  const int T = blockDim.x;
  const int stw = n / (Ns * r);
  const int nr = n / r;
  const int per_line = (n + MAXE - 1) / MAXE;
  const int G = min(L.nl, max(1, T / per_line));
  const int t = threadIdx.x;
  const int o0 = t / G;
  const int lt = t - o0 * G;
  const int ostep = T / G;
  for (int l0 = 0; l0 < L.nl; l0 += G) {
    const int l = l0 + lt;
    const bool live = o0 < ostep && l < L.nl;
    cplx<R>* base = buf + l * L.ls;
    cplx<R> v[MAXE];
    int dst[MAXE];
#pragma unroll
    for (int q = 0; q < MAXE; q++) {
      const int o = o0 + ostep * q;
      dst[q] = -1;
      if (live && o < n) {
        const int k = o % Ns;
        const int u = (o / Ns) % r;
        const int j = (o / (Ns * r)) * Ns + k;
        const int step = (k * stw + u * nr) % n;
        int idx = 0;
        const cplx<R>* src = base + j * L.es;
        cplx<R> acc = mk<R>(0, 0);
        for (int s = 0; s < r; s++) {
          cplx<R> w = tw[idx];
          if (inv) w.y = -w.y;
          acc = cadd(acc, cmul(src[s * nr * L.es], w));
          idx += step;
          if (idx >= n) idx -= n;
        }
        v[q] = acc;
        dst[q] = o * L.es;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXE; q++)
      if (dst[q] >= 0) base[dst[q]] = v[q];
    __syncthreads();
  }
}

// Odd radix r (a prime >= 17) through symmetric pairs, in two phases.
// Phase A, over all lines at once: butterfly j's inputs a_s = x[j + s*nb] take the
// Stockham twiddle w^(s*k*stw) (k = j mod Ns) and are replaced in place by
// P_s = a_s + a_{r-s} at s and Q_s = a_s - a_{r-s} at r - s (1 <= s <= H).
// Phase B, in rounds of complete lines:
//   X_u = a_0 + sum_s cos(2 pi us/r) P_s -/+ i sum_s sin(2 pi us/r) Q_s,
//   X_{r-u} the same with the sign of the second sum flipped (u = 0..H).
// A thread owns one butterfly j, MU consecutive u and up to ML lines (Gt apart), so
// each loaded P_s, Q_s feeds MU outputs and each cos/sin feeds ML lines: 4*MU*ML
// FMAs per 2*ML + MU shared-memory loads.  cos/sin come from the axis table,
// tw[(us mod r)*nb] = e^{-2 pi i us/r}.  Returns false (nothing done) when one
// line's MU-groups exceed the block; the caller then takes the output-stationary
// pass.  TC > 0: the block's thread count as a compile-time constant (static plans,
// whose kernels launch exactly TC threads), so that the cell and line split, the
// rounds and the shared-memory offsets fold to constants; 0: blockDim.x.
template <typename R, int MU, int ML, int TC = 0>
__device__ __forceinline__ bool prime_pass(cplx<R>* buf, int n, int r, int Ns, LineSet L, const cplx<R>* tw,
                                           bool inv) {
  const int T = TC > 0 ? TC : (int)blockDim.x;
  const int nb = n / r;
  const int stw = n / (Ns * r);
  const int H = (r - 1) / 2;
  const int ug = (H + MU) / MU;  // groups of MU covering u = 0..H
  const int cells = nb * ug;
  if (cells > T) return false;
  // phase A
  {
    const Div dl(L.nl), dnb(nb), dns(Ns);
    const int tot = L.nl * nb * H;
    for (int i = threadIdx.x; i < tot; i += T) {
      const int q = (int)dl.q(i);
      const int l = i - q * L.nl;
      const int sq = (int)dnb.q(q);
      const int j = q - sq * nb;
      const int s = sq + 1;
      const int k = j - (int)dns.q(j) * Ns;
      cplx<R>* base = buf + l * L.ls;
      cplx<R>* pa = base + (j + s * nb) * L.es;
      cplx<R>* pb = base + (j + (r - s) * nb) * L.es;
      cplx<R> a = *pa, b = *pb;
      if (k > 0) {
        cplx<R> wa = tw[s * k * stw], wb = tw[(r - s) * k * stw];
        if (inv) {
          wa.y = -wa.y;
          wb.y = -wb.y;
        }
        a = cmul(a, wa);
        b = cmul(b, wb);
      }
      *pa = cadd(a, b);
      *pb = csub(a, b);
    }
  }
  __syncthreads();
  // phase B: rounds of equal size (a thread's ML line slots beyond the last line
  // would issue FMAs on zeros)
  const int gmax = min(L.nl, T / cells);
  const int rounds = (L.nl + gmax * ML - 1) / (gmax * ML);
  const int Gt = ((L.nl + rounds - 1) / rounds + ML - 1) / ML;
  const int t = threadIdx.x;
  const int cell = t / Gt;
  const int lt = t - cell * Gt;
  const bool live = cell < cells;
  const int ugi = cell / nb;
  const int j = cell - ugi * nb;
  const int u0 = ugi * MU;
  const int jb = j / Ns;
  const int k = j - jb * Ns;
  const int ostep = Ns * L.es;
  const int o0 = (jb * Ns * r + k) * L.es;
  const int dstep = nb * L.es;
  for (int l0 = 0; l0 < L.nl; l0 += Gt * ML) {
    cplx<R> re[ML][MU], im[ML][MU];
    bool lok[ML];
#pragma unroll
    for (int i = 0; i < ML; i++) {
      const int l = l0 + lt + Gt * i;
      lok[i] = live && l < L.nl;
      const cplx<R> a0 = lok[i] ? buf[l * L.ls + j * L.es] : mk<R>(0, 0);
#pragma unroll
      for (int m = 0; m < MU; m++) {
        re[i][m] = a0;
        im[i][m] = mk<R>(0, 0);
      }
    }
    if (live) {
      int idx[MU];
#pragma unroll
      for (int m = 0; m < MU; m++) idx[m] = 0;
      const cplx<R>* pp = buf + (l0 + lt) * L.ls + j * L.es;
      const cplx<R>* pq = pp + r * dstep;
#pragma unroll 4  // loads of the next s issue under the FMAs of this one
      for (int s = 1; s <= H; s++) {
        pp += dstep;
        pq -= dstep;
        cplx<R> P[ML], Q[ML];
#pragma unroll
        for (int i = 0; i < ML; i++) {
          if (lok[i]) {
            P[i] = pp[Gt * i * L.ls];
            Q[i] = pq[Gt * i * L.ls];
          } else {
            P[i] = Q[i] = mk<R>(0, 0);
          }
        }
#pragma unroll
        for (int m = 0; m < MU; m++) {
          idx[m] += (u0 + m) * nb;
          if (idx[m] >= n) idx[m] -= n;
          const cplx<R> w = tw[idx[m]];  // (cos, -sin)(2 pi us / r)
#pragma unroll
          for (int i = 0; i < ML; i++) {
            re[i][m] = cfma_r(P[i], w.x, re[i][m]);
            im[i][m] = cfma_r(Q[i], -w.y, im[i][m]);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ML; i++) {
      if (!lok[i]) continue;
      cplx<R>* base = buf + (l0 + lt + Gt * i) * L.ls + o0;
#pragma unroll
      for (int m = 0; m < MU; m++) {
        const int u = u0 + m;
        if (u > H) break;
        const cplx<R> rr = rot_mi(im[i][m], inv);
        base[u * ostep] = cadd(re[i][m], rr);
        if (u > 0) base[(r - u) * ostep] = csub(re[i][m], rr);
      }
    }
    __syncthreads();
  }
  return true;
}

template <typename R> struct PrimeBlock;
template <> struct PrimeBlock<float> { static constexpr int mu = 4, ml = 3; };
template <> struct PrimeBlock<double> { static constexpr int mu = 2, ml = 2; };

// Passes for radix 7, 11, 13 (LEVEL >= 1) and primes >= 17 (LEVEL 2).
template <typename R, int EMAX, int LEVEL>
__device__ __forceinline__ void rare_pass(cplx<R>* buf, int n, int r, int Ns, LineSet L, const cplx<R>* tw,
                                       bool inv) {
  switch (r) {
    case 7: stockham_pass<R, 7, (EMAX / 7 > 0 ? EMAX / 7 : 1)>(buf, n, Ns, L, tw, inv); break;
    case 11: stockham_pass<R, 11, 1>(buf, n, Ns, L, tw, inv); break;
    case 13: stockham_pass<R, 13, 1>(buf, n, Ns, L, tw, inv); break;
    default:
      if constexpr (LEVEL >= 2) {
        if (!prime_pass<R, PrimeBlock<R>::mu, PrimeBlock<R>::ml>(buf, n, r, Ns, L, tw, inv))
          generic_pass<R, EMAX>(buf, n, r, Ns, L, tw, inv);
      }
      break;
  }
}

// Full transform of all lines along one axis.  RARE selects the passes compiled
// in beyond radix 2, 3, 4, 5, 8: none (0), radix 7, 11, 13 (1), and also primes
// >= 17 (2).  They are register hungry, so each grid runs the lowest level its
// axis plans need (plan_level; the host picks the instantiation).  EMAX bounds
// the elements a thread stages in registers per round.
template <typename R, int EMAX, int RARE>
__device__ __forceinline__ void fft_lines(cplx<R>* buf, const AxisPlan P, LineSet L, const cplx<R>* tw,
                                          bool inv) {
  const int n = P.n;
  constexpr int MB5 = EMAX / 5 > 2 ? 2 : (EMAX / 5 > 0 ? EMAX / 5 : 1);
  int Ns = 1;
  for (int p = 0; p < P.npass; p++) {
    const int r = P.radix[p];
    switch (r) {
      case 2: stockham_pass<R, 2, EMAX / 2>(buf, n, Ns, L, tw, inv); break;
      case 3: stockham_pass<R, 3, EMAX / 3>(buf, n, Ns, L, tw, inv); break;
      case 4: stockham_pass<R, 4, EMAX / 4>(buf, n, Ns, L, tw, inv); break;
      case 5: stockham_pass<R, 5, MB5>(buf, n, Ns, L, tw, inv); break;
      case 8: stockham_pass<R, 8, EMAX / 8>(buf, n, Ns, L, tw, inv); break;
      default:
        if constexpr (RARE >= 1) rare_pass<R, EMAX, RARE>(buf, n, r, Ns, L, tw, inv);
        break;
    }
    Ns *= r;
  }
}


// ---------------------------------------------------------------- compile-time plans
// Static plans: a two-pass split n = r0 * r1 with both radices in {4, 8, 12}
// when one exists (fewest passes, each a single register-staged round), else the
// greedy factorisation into 8, 4, 2, 5, 3, 7, 11, 13 and then the remaining prime
// factors (>= 17), as the runtime plans do.
constexpr int kSplit[][2] = {{8, 12}, {12, 8}, {8, 8}, {4, 12}, {12, 12}, {4, 8}, {8, 4}, {4, 4}};
constexpr int kSRadix[8] = {8, 4, 2, 5, 3, 7, 11, 13};
constexpr int splan_split(int n) {
  for (int i = 0; i < (int)(sizeof(kSplit) / sizeof(kSplit[0])); i++)
    if (kSplit[i][0] * kSplit[i][1] == n) return i;
  return -1;
}
// radix of pass p (p < 0: the number of passes; 0 when n does not factor)
constexpr int splan_walk(int n, int p) {
  int c = 0;
  for (int i = 0; i < 8; i++)
    while (n % kSRadix[i] == 0) {
      if (c == p) return kSRadix[i];
      n /= kSRadix[i];
      c++;
    }
  for (int q = 17; n > 1 && q <= n; q++)
    while (n % q == 0) {
      if (c == p) return q;
      n /= q;
      c++;
    }
  return p < 0 ? c : 0;
}
constexpr int splan_count(int n) {
  if (splan_split(n) >= 0) return 2;
  return splan_walk(n, -1);
}
constexpr int splan_radix(int n, int p) {
  if (splan_split(n) >= 0) return kSplit[splan_split(n)][p];
  return splan_walk(n, p);
}

// One radix-RAD pass with the line length N, line count NL and thread count T
// compile-time: line stride ls, element stride es (constants fold when the caller
// passes literals).  Same round structure as stockham_pass.
template <typename R, int N, int NL, int T, int NS, int RAD, int MAXB>
__device__ __forceinline__ void spass(cplx<R>* buf, int ls, int es, const cplx<R>* tw, bool inv) {
  constexpr int nb = N / RAD;
  constexpr int stw = N / (NS * RAD);
  constexpr int per_line = (nb + MAXB - 1) / MAXB;
  constexpr int G0 = T / per_line;
  constexpr int G = G0 < 1 ? 1 : (G0 > NL ? NL : G0);
  constexpr int jstep = T / G;
  constexpr int rounds = (NL + G - 1) / G;
  const int t = threadIdx.x;
  const int j0 = t / G;
  const int lt = t - j0 * G;
#pragma unroll 1
  for (int rd = 0; rd < rounds; rd++) {
    const int l = rd * G + lt;
    const bool live = j0 < jstep && (rounds * G == NL || l < NL);
    cplx<R>* base = buf + l * ls;
    cplx<R> v[MAXB][RAD];
    bool on[MAXB];
    int jbk[MAXB];
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
      const int j = j0 + jstep * q;
      on[q] = live && (jstep * MAXB == nb || j < nb);
      if (on[q]) {
        const int jb = j / NS;  // compile-time divisor
        const int k = j - jb * NS;
        jbk[q] = jb * NS * RAD + k;
#pragma unroll
        for (int u = 0; u < RAD; u++) {
          cplx<R> a = base[(j + u * nb) * es];
          if (NS > 1 && u > 0) {
            cplx<R> w = tw[u * k * stw];
            if (inv) w.y = -w.y;
            a = cmul(a, w);
          }
          v[q][u] = a;
        }
        Dft<R, RAD>::run(v[q], inv);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; q++) {
      if (on[q]) {
#pragma unroll
        for (int u = 0; u < RAD; u++) base[(jbk[q] + u * NS) * es] = v[q][u];
      }
    }
    __syncthreads();
  }
}

// Butterflies a thread stages per round: enough that all NL lines fit one round
// when T >= NL (T / NL threads per line), capped by EMAX elements in registers.
constexpr int smaxb(int N, int NL, int T, int EMAX, int RAD) {
  const int nb = N / RAD;
  const int tpl = T / NL > 0 ? T / NL : 1;
  const int want = (nb + tpl - 1) / tpl;
  const int cap = EMAX / RAD > 0 ? EMAX / RAD : 1;
  return want < cap ? want : cap;
}

template <typename R, int N, int NL, int T, int EMAX, int P = 0, int NS = 1>
__device__ __forceinline__ void sfft(cplx<R>* buf, int ls, int es, const cplx<R>* tw, bool inv) {
  static_assert(N == 1 || splan_count(N) > 0, "line length without a static plan");
  if constexpr (P < splan_count(N)) {
    constexpr int RAD = splan_radix(N, P);
    if constexpr (RAD >= 17) {
      // a prime factor >= 17: the symmetric-pair pass, its sizes compile-time constants
      const LineSet L{NL, ls, es};
      if (!prime_pass<R, PrimeBlock<R>::mu, PrimeBlock<R>::ml, T>(buf, N, RAD, NS, L, tw, inv))
        generic_pass<R, EMAX>(buf, N, RAD, NS, L, tw, inv);
    } else {
      constexpr int MB = smaxb(N, NL, T, EMAX, RAD);
      spass<R, N, NL, T, NS, RAD, MB>(buf, ls, es, tw, inv);
    }
    sfft<R, N, NL, T, EMAX, P + 1, NS * RAD>(buf, ls, es, tw, inv);
  }
}

// The lowest fft_lines level (RARE) that has a pass for every radix of the plan.
inline int plan_level(const AxisPlan& P) {
  int lv = 0;
  for (int p = 0; p < P.npass; p++) {
    const int r = P.radix[p];
    if (r == 2 || r == 3 || r == 4 || r == 5 || r == 8) continue;
    lv = (r == 7 || r == 11 || r == 13) ? (lv > 1 ? lv : 1) : 2;
  }
  return lv;
}

}  // namespace fame
