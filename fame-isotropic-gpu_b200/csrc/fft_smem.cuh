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
// large prime such as 23 or 107) uses an output-stationary DFT pass where each
// thread forms its outputs as length-R sums.
#pragma once
#include "fame_common.cuh"

namespace fame {

constexpr int kMaxPasses = 10;

struct AxisPlan {
  int n;
  int npass;
  int radix[kMaxPasses];
};

// cos/sin(2*pi*m/R) for the odd radices handled by the symmetric-pair DFT,
// filled once from the host (fame_fft_init_constants) with libm in FP64.
__constant__ double c_cos7[7], c_sin7[7], c_cos11[11], c_sin11[11], c_cos13[13], c_sin13[13];
__constant__ double c_cos5[5], c_sin5[5];

template <int RAD> struct OddTab;
template <> struct OddTab<5> {
  __device__ static double c(int m) { return c_cos5[m]; }
  __device__ static double s(int m) { return c_sin5[m]; }
};
template <> struct OddTab<7> {
  __device__ static double c(int m) { return c_cos7[m]; }
  __device__ static double s(int m) { return c_sin7[m]; }
};
template <> struct OddTab<11> {
  __device__ static double c(int m) { return c_cos11[m]; }
  __device__ static double s(int m) { return c_sin11[m]; }
};
template <> struct OddTab<13> {
  __device__ static double c(int m) { return c_cos13[m]; }
  __device__ static double s(int m) { return c_sin13[m]; }
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
    cplx<R> out[RAD];
    out[0] = sum;
#pragma unroll
    for (int t = 1; t <= H; t++) {
      cplx<R> re = x0, im = mk<R>(0, 0);
#pragma unroll
      for (int s = 1; s <= H; s++) {
        const int m = (t * s) % RAD;
        const R c = (R)OddTab<RAD>::c(m), sn = (R)OddTab<RAD>::s(m);
        re.x += c * P[s - 1].x;
        re.y += c * P[s - 1].y;
        im.x += sn * Q[s - 1].x;
        im.y += sn * Q[s - 1].y;
      }
      cplx<R> r = rot_mi(im, inv);  // -i*im (forward) / +i*im (inverse)
      out[t] = cadd(re, r);
      out[RAD - t] = csub(re, r);
    }
#pragma unroll
    for (int t = 0; t < RAD; t++) a[t] = out[t];
  }
};
template <typename R> struct Dft<R, 5> : DftOdd<R, 5> {};
template <typename R> struct Dft<R, 7> : DftOdd<R, 7> {};
template <typename R> struct Dft<R, 11> : DftOdd<R, 11> {};
template <typename R> struct Dft<R, 13> : DftOdd<R, 13> {};

// Lines layout: element m of line l at buf[l*ls + m*es].  `line_fast` chooses the
// thread->butterfly mapping so that consecutive threads touch consecutive shared
// memory words: lines fastest when the lines are adjacent words (es > 1, ls = 1),
// butterflies fastest when the line itself is contiguous (es = 1).
struct LineSet {
  int nl, ls, es;
  bool line_fast;
};

// One radix-RAD pass over lines [l0, l0 + nlg).
template <typename R, int RAD, int MAXB>
__device__ __noinline__ void stockham_pass(cplx<R>* buf, int n, int Ns, LineSet L, int l0, int nlg,
                                              const cplx<R>* tw, bool inv) {
  const int nb_line = n / RAD;
  const int total = nb_line * nlg;
  const int stw = n / (Ns * RAD);
  cplx<R> v[MAXB][RAD];
  int dst[MAXB];
#pragma unroll
  for (int q = 0; q < MAXB; q++) {
    const int b = threadIdx.x + q * blockDim.x;
    dst[q] = -1;
    if (b < total) {
      int l, j;
      if (L.line_fast) {
        l = b % nlg;
        j = b / nlg;
      } else {
        j = b % nb_line;
        l = b / nb_line;
      }
      l += l0;
      const int k = j % Ns;
      const cplx<R>* src = buf + l * L.ls;
#pragma unroll
      for (int t = 0; t < RAD; t++) {
        cplx<R> a = src[(j + t * nb_line) * L.es];
        if (t > 0 && k > 0) {
          cplx<R> w = tw[t * k * stw];
          if (inv) w.y = -w.y;
          a = cmul(a, w);
        }
        v[q][t] = a;
      }
      Dft<R, RAD>::run(v[q], inv);
      dst[q] = l * L.ls + ((j / Ns) * Ns * RAD + k) * L.es;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MAXB; q++) {
    if (dst[q] >= 0) {
#pragma unroll
      for (int t = 0; t < RAD; t++) buf[dst[q] + t * Ns * L.es] = v[q][t];
    }
  }
  __syncthreads();
}

// Output-stationary DFT pass for an arbitrary radix r (used for large primes).
template <typename R, int MAXE>
__device__ __noinline__ void generic_pass(cplx<R>* buf, int n, int r, int Ns, LineSet L, int l0, int nlg,
                                             const cplx<R>* tw, bool inv) {
  const int total = n * nlg;
  const int stw = n / (Ns * r);
  const int nr = n / r;
  cplx<R> v[MAXE];
  int dst[MAXE];
#pragma unroll
  for (int q = 0; q < MAXE; q++) {
    const int b = threadIdx.x + q * blockDim.x;
    dst[q] = -1;
    if (b < total) {
      int l, o;
      if (L.line_fast) {
        l = b % nlg;
        o = b / nlg;
      } else {
        o = b % n;
        l = b / n;
      }
      l += l0;
      const int k = o % Ns;
      const int t = (o / Ns) % r;
      const int j = (o / (Ns * r)) * Ns + k;
      const int step = (k * stw + t * nr) % n;
      int idx = 0;
      const cplx<R>* src = buf + l * L.ls + j * L.es;
      cplx<R> acc = mk<R>(0, 0);
      for (int s = 0; s < r; s++) {
        cplx<R> w = tw[idx];
        if (inv) w.y = -w.y;
        acc = cadd(acc, cmul(src[s * nr * L.es], w));
        idx += step;
        if (idx >= n) idx -= n;
      }
      v[q] = acc;
      dst[q] = l * L.ls + o * L.es;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MAXE; q++)
    if (dst[q] >= 0) buf[dst[q]] = v[q];
  __syncthreads();
}

// Full transform of all lines along one axis.  Lines are independent, so each
// pass is run over groups of lines small enough that a thread holds at most
// about EMAX elements in registers; every group costs one barrier pair.
template <typename R, int EMAX>
__device__ __forceinline__ void fft_lines(cplx<R>* buf, const AxisPlan P, LineSet L, const cplx<R>* tw,
                                       bool inv) {
  const int n = P.n;
  const int per_group = max(1, (EMAX * (int)blockDim.x) / n);  // lines per group
  int Ns = 1;
  for (int p = 0; p < P.npass; p++) {
    const int r = P.radix[p];
    for (int l0 = 0; l0 < L.nl; l0 += per_group) {
      const int nlg = min(per_group, L.nl - l0);
      switch (r) {
        case 2: stockham_pass<R, 2, (EMAX + 1) / 2>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 3: stockham_pass<R, 3, (EMAX + 2) / 3>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 4: stockham_pass<R, 4, (EMAX + 3) / 4>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 5: stockham_pass<R, 5, (EMAX + 4) / 5>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 7: stockham_pass<R, 7, (EMAX + 6) / 7>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 8: stockham_pass<R, 8, (EMAX + 7) / 8>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 11: stockham_pass<R, 11, (EMAX + 10) / 11>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        case 13: stockham_pass<R, 13, (EMAX + 12) / 13>(buf, n, Ns, L, l0, nlg, tw, inv); break;
        default: generic_pass<R, EMAX>(buf, n, r, Ns, L, l0, nlg, tw, inv); break;
      }
    }
    Ns *= r;
  }
}

}  // namespace fame
