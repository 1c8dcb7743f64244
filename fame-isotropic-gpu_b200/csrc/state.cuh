// State, loop conditions and kernel argument structs shared by the operator
// kernels (op_kernels.cuh) and the solver kernels (solver_kernels.cuh).
#pragma once
#include "operator.cuh"

namespace fame {

// complex elements a thread holds in registers during one FFT pass of the runtime
// plans (per precision).  FP32 stages 8: the runtime plane kernels run at 64
// registers, and 16 elements spilled twice as much (FP32 CG iteration on the
// runtime plans of FCC 64x55x52: 38.6 -> 36.3 us per k-point, hex 36x30x26: 14.8 -> 13.6)
template <typename R> struct Emax;
template <> struct Emax<float> { static constexpr int v = 8; };
template <> struct Emax<double> { static constexpr int v = 8; };
// fast-axis positions per pencil CTA: 256-byte rows
template <typename R> struct PencilTW { static constexpr int v = 256 / (int)sizeof(cplx<R>); };

// ------------------------------------------------------------------ state
struct CgState {
  double r1, r0, beta;       // ||r||^2 now / before, r1/r0
  double a_re, a_im;         // CG step a = r1 / <p, Ap>
  double r1_0, tol2;         // initial ||r||^2, stop threshold on ||r||^2
  int iter;                  // the reference's counter k (starts at 1, CG.cu:36)
  int active;
  int maxit;
  int total;                 // CG products accumulated for the profile counter
  // outer iterative refinement (mixed precision)
  double rr, scale;          // ||b - A y||^2, 1/||b - A y|| used to scale the FP32 rhs
  double otol2;              // stop threshold of the refinement on ||b - A y||^2 (ls_tol^2)
  int outer, outer_active, outer_max, outer_total;
};

struct LzState {
  int converged;
  int restarts;
  int nconv;
  int pad;
};

// Condition of one CUDA-graph WHILE node (in host-driven mode only `flag` is used).
// Every loop is fail-safe: the first kernel of the body clears the condition, the
// deciding kernel sets it again only while work remains and the loop's trip count
// (counted on the device) is below `cap`; hitting the cap records an overflow in
// trips[1] and ends the loop, so no data-dependent loop can run unbounded.
struct Cond {
  cudaGraphConditionalHandle handle;
  int* flag;
  int* trips;  // [0] trips of the current loop, [1] overflow marker
  int cap;
};

__device__ __forceinline__ void set_cond(const Cond& c, int v) {
  if (!c.flag) return;
  *c.flag = v;
  if (c.handle) cudaGraphSetConditional(c.handle, (unsigned)v);
}

// decision at the end of a loop body
__device__ __forceinline__ void decide_cond(const Cond& c, int any) {
  if (c.trips) {
    const int t = ++c.trips[0];
    if (any && t >= c.cap) {
      c.trips[1] = 1;
      any = 0;
    }
  }
  set_cond(c, any);
}

// before the loop: reset the trip counter and set the first decision
__device__ __forceinline__ void start_cond(const Cond& c, int any) {
  if (c.trips) c.trips[0] = 0;
  set_cond(c, any);
}

// Ticket counter over the whole grid: true in exactly one CTA, the last one.
__device__ __forceinline__ bool grid_last(unsigned* ctr, unsigned total) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ctr, 1u) == total - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    *ctr = 0u;
  }
  return last;
}

// D_kz(x, y, z) = e^{i 2 pi phi(x,y) z / Nz} (…Lambdas.cu:389-400)
template <typename R>
__device__ __forceinline__ cplx<R> dkz_at(const Geom& g, const double2* tab, int x, int y, int z) {
  const double ph = tab[g.oPhi + x * g.Ny + y].x;
  const double a = ph * z * g.tnz;  // e^{i pi a}, a = 2 ph z / Nz
  if constexpr (sizeof(R) == 8) {
    return expipi(a);
  } else {
    // FP32: the argument reduced to [-1, 1] in FP64 (a - 2n changes nothing), then a
    // single-precision sincospi
    return expipi((float)(a - 2.0 * rint(0.5 * a)));
  }
}

// ------------------------------------------------------------------ plane stage
enum InMode { IN_VEC = 0, IN_CG = 1, IN_REFINE = 2 };
// EPI_CG writes Ap and forms <p, Ap>; EPI_CGR (fused CG) keeps Ap in registers and
// applies r -= a Ap with ||r||^2, the step size a coming from the PEN_QBQ_CG pencil.
enum EpiMode { EPI_OUT = 0, EPI_CG = 1, EPI_RESID = 2, EPI_CGR = 3 };
// PEN_QBQ_CG: PEN_QBQ that also reduces <p, Ap> = (1/N) sum_e |(IDFT v)_e|^2 / eps_e
enum PencilMode { PEN_QBQ = 0, PEN_QR_OUT = 1, PEN_QRS_IN = 2, PEN_QBQ_CG = 3 };

template <typename R>
struct PlaneInArgs {
  Geom g;
  const Slot* slots;
  const double2* tabs;
  const cplx<R>* tw;      // forward twiddle tables, R precision
  long vstride;           // per-slot stride of reduced vectors (elements)
  long fstride;           // per-slot stride of 3N fields (elements)
  int vec_per_slot;       // number of vectors per slot (batched Qr over bands)
  const cplx<R>* in;      // IN_VEC: reduced input
  cplx<R>* p;             // IN_CG: search direction (updated in place)
  const cplx<R>* r;       // IN_CG: residual
  cplx<R>* x;             // IN_CG: solution; takes the previous iteration's a * p here
  CgState* cg;            // IN_CG / IN_REFINE
  double2* y64;           // IN_REFINE: FP64 accumulated solution (updated)
  const float2* x32;      // IN_REFINE: FP32 correction
  const float2* p32;      // IN_REFINE: the FP32 search direction of the inner solve's last update
  int sigma;              // IN_VEC: multiply the input by sqrt(Lambda_q) first (Sigma, …_Isotropic.cu:109)
  cplx<R>* T;             // output field (3 components)
  Cond reset;             // loop condition cleared by this kernel when it starts a loop body
  int pf_dist;            // > 0: each CTA prefetches into L2 the operands of the CTA this
                          // many places later in launch order (about one wave ahead)
  int self_pf;            // IN_CG: L2 prefetch of this CTA's own r, p and x at its start
  int* fault;             // set to 1 if a bounded wait of the component exchange ran out (or NULL)
};

template <typename R>
struct PencilArgs {
  Geom g;
  const Slot* slots;
  const double2* tabs;
  const cplx<R>* tw;
  long fstride;
  int vec_per_slot;
  cplx<R>* T;              // field in frequency-plane layout (in/out)
  const R* invB;           // PEN_QBQ and PEN_QR_OUT (optional): 1/eps per edge, 3N
  int ib_field;            // invB in the field layout (else the spatial layout; same for Simple lattices)
  cplx<R>* out;            // PEN_QR_OUT: spatial field out (3N per vector)
  const cplx<R>* in;       // PEN_QRS_IN: spatial field in
  CgState* cg;             // optional activity gate; PEN_QBQ_CG writes the step size a
  int gate;                // 0 none, 1 CG active, 2 outer refinement active
  double* partials;        // PEN_QBQ_CG: partial sums of <p, Ap>, [slot * pstride + CTA of the slot]
  unsigned* counters;      // (unused by PEN_QBQ_CG)
  long pstride;            // per-slot stride of `partials`
  int TW;                  // fast positions per CTA
  int nslots;              // k-points of the launch (k_pencil_pipe walks all their tiles)
  int pf_dist;             // > 0: L2 prefetch of the tile of the CTA this many places later
};

template <typename R>
struct PlaneOutArgs {
  Geom g;
  const Slot* slots;
  const double2* tabs;
  const cplx<R>* tw;
  long vstride, fstride;
  int vec_per_slot;
  const cplx<R>* T;        // field after the slow-axis forward pass
  cplx<R>* out;            // EPI_OUT: reduced output; EPI_CG: Ap; EPI_RESID: r (FP64)
  const cplx<R>* p;        // EPI_CG: p for <p, Ap>
  cplx<R>* r;              // EPI_CGR: CG residual, updated in place
  const cplx<R>* b;        // EPI_RESID: right-hand side
  CgState* cg;
  double* partials;        // [nslots][blocks per slot][NV]
  unsigned* counters;      // [nslots] ticket counters, plus [nslots] = grid counter
  Cond cond;               // EPI_RESID: outer WHILE condition; EPI_CGR: CG WHILE condition
  int nslots;
  double tol2;             // EPI_RESID: absolute tolerance^2 on ||b - A y||
  int pf_dist;             // > 0: L2 prefetch of the operands of the CTA this many places later
  int self_pf;             // EPI_CGR: L2 prefetch of this CTA's own residual at its start
  long pstride;            // EPI_CGR: per-slot stride of `partials`
  int pen_parts;           // EPI_CGR: the pencil's <p, Ap> partials per slot (at the slot's start);
                           // this kernel's ||r||^2 partials follow them
};

// Ordered sum of p[0], p[stride], ..., p[(n - 1) stride] by one warp (lane-strided,
// then a fixed shuffle tree); valid in all lanes.
__device__ __forceinline__ double warp_sum_strided(const double* p, int n, int stride) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += p[(size_t)i * stride];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// warp_sum_strided over data other CTAs of this grid wrote (loads through L2, not L1).
__device__ __forceinline__ double warp_sum_strided_cg(const double* p, int n, int stride) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += __ldcg(p + (size_t)i * stride);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Ordered sum of n partial sums by one warp (lane-strided, then a fixed shuffle tree):
// every caller gets the same bits, so kernels that need the same CG scalar (the step
// size) agree exactly.  Valid in all lanes.
__device__ __forceinline__ double warp_sum_partials(const double* p, int n) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  // 16 independent loads per lane in flight per round (a few hundred partials take
  // one or two L2 round trips, not one per element)
  for (int b = 0; b < n; b += 32 * 16) {
    double v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int i = b + u * 32 + lane;
      v[u] = i < n ? p[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; u++) s += v[u];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

}  // namespace fame
