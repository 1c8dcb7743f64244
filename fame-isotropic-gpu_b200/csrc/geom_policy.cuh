// Geometry policies of the operator kernels.
//
// DynGeom takes every length from the runtime Geom and runs the runtime-planned
// FFT passes (any grid).  StatGeom<LF, LM, LS> fixes the fast, mid and slow line
// lengths at compile time: the FFT passes are fully unrolled and all index
// arithmetic folds to constants.  The solver instantiates StatGeom for the grids
// it runs most (cubic 96^3) and falls back to DynGeom elsewhere.
#pragma once
#include "state.cuh"

namespace fame {

constexpr int kPlaneThreads = 512;      // most threads of a plane CTA (runtime geometry)
constexpr int kStatPlaneThreads = 384;  // threads of a plane CTA with a static geometry
constexpr int kPencilThreads = 256;     // threads of a pencil CTA

struct DynGeom {
  static constexpr bool kStatic = false;
  static constexpr int kMaxPlaneThreads = kPlaneThreads;
  // The stage kernels' register budgets (launch bounds in op_kernels.cuh) are
  // sized for two resident plane CTAs per SM (64 registers at 512 threads) and
  // three pencil CTAs (85 registers), except that plane kernels with the prime
  // pass (RARE 2), whose MU x ML accumulator block needs more, take one.
  __device__ __forceinline__ static int plane_threads() { return blockDim.x; }
  // plane CTAs per SM the register budget is sized for (launch bounds)
  template <typename R, int RARE> static constexpr int plane_min_blocks() { return RARE >= 2 ? 1 : 2; }
  __device__ __forceinline__ static int Lf(const Geom& g) { return g.Lf; }
  __device__ __forceinline__ static int Lm(const Geom& g) { return g.Lm; }
  __device__ __forceinline__ static int Ls(const Geom& g) { return g.Ls; }
  __device__ __forceinline__ static int S(const Geom& g) { return g.S; }
  __device__ __forceinline__ static int P(const Geom& g) { return g.P; }
  // lines of a plane (pitch S) along its fast axis (fast = true) or mid axis, and
  // the TW lines of a pencil tile.  One FFT call site per kernel keeps the kernel
  // within its register budget, so the plane axis is a runtime argument.
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_plane(cplx<R>* b, const Geom& g, bool fast, const cplx<R>* tw,
                                                   bool inv) {
    fft_lines<R, Emax<R>::v, RARE>(b, fast ? g.pf : g.pm, fast ? LineSet{g.Lm, g.S, 1} : LineSet{g.Lf, 1, g.S},
                                   tw, inv);
  }
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_slow(cplx<R>* b, const Geom& g, const cplx<R>* tw, bool inv) {
    constexpr int TW = PencilTW<R>::v;
    fft_lines<R, Emax<R>::v, RARE>(b, g.ps, LineSet{TW, 1, TW}, tw, inv);
  }
};

// elements a thread stages per round in the static passes: plane passes (FP32 at
// most 80 registers, two CTAs per SM) and pencil passes
template <typename R> struct SEmax;
template <> struct SEmax<float> { static constexpr int v = 24; };
template <> struct SEmax<double> { static constexpr int v = 12; };
template <typename R> struct SPenEmax;
template <> struct SPenEmax<float> { static constexpr int v = 24; };
template <> struct SPenEmax<double> { static constexpr int v = 12; };
// static plane passes of the runtime-geometry grids (128 registers at two 256-thread
// CTAs per SM, the general-lattice Pi mixing in the same kernel): half the 96^3
// staging in FP32, a third in FP64, which keeps the radix-11 and radix-13 passes of
// the FCC and BCC planes in registers (FCC 64x55x52: FP32 CG iteration 37.5 -> 33.9
// us per k-point; BCC 48x45x39: FP64 plane stages 23.5 -> 20.7 us)
template <typename R> struct PlaneEmax;
template <> struct PlaneEmax<float> { static constexpr int v = 12; };
template <> struct PlaneEmax<double> { static constexpr int v = 4; };
// static slow-axis passes of the runtime-geometry grids (80 registers at three
// pencil CTAs per SM, the general-lattice twiddles in the same kernel): a third of
// the 96^3 pencil staging, which removes the FP32 spills (hexagonal 128-point slow
// axis: FP32 pencil stage 37.6 -> 28.3 us per k-point)
template <typename R> struct SlowEmax;
template <> struct SlowEmax<float> { static constexpr int v = 8; };
template <> struct SlowEmax<double> { static constexpr int v = 4; };

// DynGeom with the slow-axis length fixed at compile time: the pencil stage's
// slow-axis transforms run the static plan (unrolled passes, constant strides and
// twiddle indices); everything else stays runtime.  The solver uses it for the
// pencils of runtime-geometry grids whose slow axis is one of the lengths
// instantiated in ops_slow_static.cu.
template <int LSL>
struct DynGeomSlow : DynGeom {
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_slow(cplx<R>* b, const Geom&, const cplx<R>* tw, bool inv) {
    constexpr int TW = PencilTW<R>::v;
    sfft<R, LSL, TW, kPencilThreads, SlowEmax<R>::v>(b, 1, TW, tw, inv);
  }
};

// DynGeom with the two plane axes' lengths fixed at compile time: the plane stages'
// fast- and mid-axis transforms run static plans (spass, and the prime pass with
// constant sizes); T threads per plane CTA, MB CTAs per SM in the register budget.
// Index arithmetic outside the transforms stays runtime.  The solver uses it for the
// plane stages of the runtime-geometry grids instantiated in ops_plane_static.cu.
template <int LF, int LM, int T, int MB>
struct DynGeomPlane : DynGeom {
  static constexpr int kMaxPlaneThreads = T;
  __device__ __forceinline__ static constexpr int plane_threads() { return T; }
  template <typename R, int RARE> static constexpr int plane_min_blocks() { return MB; }
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_plane(cplx<R>* b, const Geom&, bool fast, const cplx<R>* tw,
                                                   bool inv) {
    if (fast)
      sfft<R, LF, LM, T, PlaneEmax<R>::v>(b, LF | 1, 1, tw, inv);
    else
      sfft<R, LM, LF, T, PlaneEmax<R>::v>(b, 1, LF | 1, tw, inv);
  }
};

template <int LF, int LM, int LSL>
struct StatGeom {
  static constexpr bool kStatic = true;
  static constexpr int kS = LF | 1;
  // 384 = 4 threads per line of a 96 x 96 plane: every pass of the 8 x 12 plan
  // is one round with all threads busy
  static constexpr int kMaxPlaneThreads = kStatPlaneThreads;
  // two FP32 plane CTAs per SM (80 registers), one FP64 plane CTA; three FP32 and
  // two FP64 pencil CTAs
  __device__ __forceinline__ static constexpr int plane_threads() { return kStatPlaneThreads; }
  template <typename R, int RARE> static constexpr int plane_min_blocks() { return sizeof(R) == 4 ? 2 : 1; }
  __device__ __forceinline__ static constexpr int Lf(const Geom&) { return LF; }
  __device__ __forceinline__ static constexpr int Lm(const Geom&) { return LM; }
  __device__ __forceinline__ static constexpr int Ls(const Geom&) { return LSL; }
  __device__ __forceinline__ static constexpr int S(const Geom&) { return kS; }
  __device__ __forceinline__ static constexpr int P(const Geom&) { return LF * LM; }
  static_assert(LF == LM, "a static plane geometry has equal fast and mid lengths");
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_plane(cplx<R>* b, const Geom&, bool fast, const cplx<R>* tw,
                                                   bool inv) {
    sfft<R, LF, LM, kStatPlaneThreads, SEmax<R>::v>(b, fast ? kS : 1, fast ? 1 : kS, tw, inv);
  }
  template <typename R, int RARE>
  __device__ __forceinline__ static void fft_slow(cplx<R>* b, const Geom&, const cplx<R>* tw, bool inv) {
    constexpr int TW = PencilTW<R>::v;
    sfft<R, LSL, TW, kPencilThreads, SPenEmax<R>::v>(b, 1, TW, tw, inv);
  }
  // The same passes with the axis and the direction fixed at compile time: every
  // stride, twiddle sign and rotation folds to a constant (one call site each).
  template <typename R, bool FAST, bool INV>
  __device__ __forceinline__ static void fft_plane_c(cplx<R>* b, const cplx<R>* tw) {
    sfft<R, LF, LM, kStatPlaneThreads, SEmax<R>::v>(b, FAST ? kS : 1, FAST ? 1 : kS, tw, INV);
  }
  template <typename R, bool INV>
  __device__ __forceinline__ static void fft_slow_c(cplx<R>* b, const cplx<R>* tw) {
    constexpr int TW = PencilTW<R>::v;
    sfft<R, LSL, TW, kPencilThreads, SPenEmax<R>::v>(b, 1, TW, tw, INV);
  }
};

using Stat96 = StatGeom<96, 96, 96>;
// static plane plans of the general-lattice benchmark grids (fast, mid, threads, CTAs per SM)
using PlaneFcc64 = DynGeomPlane<52, 55, 256, 2>;
using PlaneBcc48 = DynGeomPlane<39, 45, 256, 2>;
using PlaneHex128f = DynGeomPlane<92, 107, 256, 2>;
using PlaneHex128d = DynGeomPlane<92, 107, 512, 1>;

}  // namespace fame
