// Fused Q_r / Q_r^H / P_r / P_r^H and Q_r^H B^{-1} Q_r kernels.
//
// Reference behaviour (FP64, cuFFT):
//   Q_r  : FAME_Main/FAME_Matrix_Vector_Production_Qr.cu:8-78 (mix 2->3 with Pi_Qr,
//          zero the Gamma-point entry, inverse 3-D DFT, x D_k / N)
//   Q_r^H: FAME_Main/FAME_Matrix_Vector_Production_Qrs.cu:7-58 (x conj(D_k), forward
//          3-D DFT, mix 3->2 with Pi_Qr^H)
//   QBQ  : FAME_Main/FAME_Matrix_Vector_Production_Isotropic_QBQ.cu:8-67
//   General lattices: FAME_Main/FAME_FFT_CUDA.cu:63-160 (1-D passes z -> y -> x
//          with the index-dependent twiddles D_kz, D_ky, D_kx between them)
//
// Layout.  A grid point is (slow s, mid m, fast f); flat index s*P + m*Lf + f with
// P = Lm*Lf.  Simple lattices: (s,m,f) = (z,y,x) in both frequency and space.
// General lattices: (s,m,f) = (x,y,z) in frequency (the reference's z-fastest
// order), while the spatial field keeps x fastest.  Every transform is split in
// a PLANE stage (fast and mid axes, one (s) plane per CTA, the whole plane in
// shared memory) and a PENCIL stage (slow axis, a tile of TW fast positions per
// CTA).  The Pi mixing is evaluated on the fly from 1-D Lambda tables, so no
// 6*Nd Pi array is read from HBM.
//
// The three field components of one plane live in the three CTAs of a thread
// block cluster: the 2->3 mix writes each component into its owner's shared
// memory (distributed shared memory), and the 3->2 unmix reads all three.
#pragma once
#include <cooperative_groups.h>

#include "fft_smem.cuh"

namespace cg = cooperative_groups;

namespace fame {

// ------------------------------------------------------------------ geometry
struct Geom {
  int Nx, Ny, Nz, N;
  int general;
  int Ls, Lm, Lf, P;  // slow / mid / fast lengths, plane size
  int S;              // row pitch of a plane in shared memory: Lf rounded up to odd
  double hx, hy, hz;
  double ihz;  // 1 / hz
  double tnz;  // 2 / Nz
  AxisPlan pf, pm, ps;
  // per-slot table offsets (in double2 units) inside a slot's table block
  int oLx, oLy, oLz, oDx, oDy, oDz, oExy, oWz, oDky, oPhi, oDkx;
  int tab_stride;
  int twf, twm, tws;  // offsets of the forward twiddle tables of each axis (double2 units)
};

// Per k-point scalars.
struct Slot {
  int Nd;   // N or N-1 (Gamma point)
  int off;  // N - Nd
  int active;
  int pad;
  double th[3];  // theta_x, theta_y (or theta_xy), theta_z (or theta_xyz)
};

// Lambda_x, Lambda_y, Lambda_z at (s, m, f) from the slot tables (FP64).
__device__ __forceinline__ void lambdas_at(const Geom& g, const double2* tab, int s, int m, int f,
                                           double2& Lx, double2& Ly, double2& Lz) {
  if (!g.general) {
    Lx = tab[g.oLx + f];
    Ly = tab[g.oLy + m];
    Lz = tab[g.oLz + s];
  } else {
    Lx = tab[g.oLx + s];
    Ly = tab[g.oLy + s * g.Ny + m];
    const double2 e = cmul(tab[g.oExy + s * g.Ny + m], tab[g.oWz + f]);
    Lz = make_double2((e.x - 1.0) * g.ihz, e.y * g.ihz);
  }
}

// Pi_Qr columns (FAME_Main/FAME_Matrix_Lambdas.cu:184-244 Simple, :438-489 General),
// or Pi_Pr = [-conj(Pi2); conj(Pi1)] when pr is set.  P[0..2] multiply x1, P[3..5] x2.
// Lambdas in the operator precision R; the normalisers use rsqrt.
template <typename R>
__device__ __forceinline__ void pi_from(bool general, bool pr, cplx<R> Lx, cplx<R> Ly, cplx<R> Lz, cplx<R>* P) {
  const R Lq = cabs2(Lx) + cabs2(Ly) + cabs2(Lz);
  cplx<R> p1[3], p2[3];
  if (!general) {
    const R al = 3, be = 5;
    const cplx<R> t1 = mk<R>(be * Lz.x - Ly.x, be * Lz.y - Ly.y);
    const cplx<R> t2 = mk<R>(Lx.x - al * Lz.x, Lx.y - al * Lz.y);
    const cplx<R> t3 = mk<R>(al * Ly.x - be * Lx.x, al * Ly.y - be * Lx.y);
    const R n2 = cabs2(t1) + cabs2(t2) + cabs2(t3);
    const R i2 = rsqrt(n2), i1 = i2 * rsqrt(Lq);
    // t x conj(Lambda)
    p1[0] = cscale(csub(cmul(t3, cconj(Ly)), cmul(t2, cconj(Lz))), i1);
    p1[1] = cscale(csub(cmul(t1, cconj(Lz)), cmul(t3, cconj(Lx))), i1);
    p1[2] = cscale(csub(cmul(t2, cconj(Lx)), cmul(t1, cconj(Ly))), i1);
    p2[0] = cscale(cconj(t1), i2);
    p2[1] = cscale(cconj(t2), i2);
    p2[2] = cscale(cconj(t3), i2);
  } else {
    const cplx<R> Ls = cadd(cadd(Lx, Ly), Lz);
    // 3*Lq - |Ls|^2 (the reference's normaliser, …Lambdas.cu:450-451) written as
    // |Lx-Ly|^2 + |Ly-Lz|^2 + |Lz-Lx|^2: the same number without cancellation
    const R d2 = cabs2(csub(Lx, Ly)) + cabs2(csub(Ly, Lz)) + cabs2(csub(Lz, Lx));
    const R i2 = rsqrt(d2), i1 = i2 * rsqrt(Lq);
    const cplx<R> cs = cconj(Ls);
    p1[0] = cscale(csub(mk<R>(Lq, 0), cmul(Lx, cs)), i1);
    p1[1] = cscale(csub(mk<R>(Lq, 0), cmul(Ly, cs)), i1);
    p1[2] = cscale(csub(mk<R>(Lq, 0), cmul(Lz, cs)), i1);
    p2[0] = cscale(csub(cconj(Lz), cconj(Ly)), i2);
    p2[1] = cscale(csub(cconj(Lx), cconj(Lz)), i2);
    p2[2] = cscale(csub(cconj(Ly), cconj(Lx)), i2);
  }
  if (!pr) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      P[c] = p1[c];
      P[3 + c] = p2[c];
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      P[c] = cscale(cconj(p2[c]), (R)-1);
      P[3 + c] = cconj(p1[c]);
    }
  }
}

// sqrt(Lambda_q) at full frequency index fi, in FP64 (invAr scaling,
// FAME_Main/FAME_Matrix_Vector_Production_Isotropic_invAr.cu:50-70).
__device__ __forceinline__ double lq_sqrt_at(const Geom& g, const double2* tab, int fi) {
  const int s = fi / g.P, e = fi - s * g.P, m = e / g.Lf, f = e - m * g.Lf;
  double2 Lx, Ly, Lz;
  lambdas_at(g, tab, s, m, f, Lx, Ly, Lz);
  return sqrt(cabs2(Lx) + cabs2(Ly) + cabs2(Lz));
}

// ------------------------------------------------------------------ reductions
// Deterministic grid reduction: every CTA of a slot stores its partial, the last
// CTA to arrive (ticket counter, threadfence pattern of the CUDA samples'
// threadFenceReduction) sums the partials in a fixed order.
constexpr int kMaxRed = 4;  // values reduced per call

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* sred) {
  // sred: NV * 32 doubles of shared scratch
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sred[q * 32 + wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double x = lane < nw ? sred[q * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[q] = x;
    }
  }
  __syncthreads();
}

// Store this CTA's partials (valid in thread 0) and report whether this CTA is the
// last of the `nblk` CTAs of the slot; if so `out` holds the ordered sum in thread 0.
template <int NV>
__device__ __forceinline__ bool slot_reduce(double (&v)[NV], double* partials, unsigned* counter,
                                            int bid, int nblk, double (&out)[NV]) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) partials[(size_t)bid * NV + q] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == (unsigned)nblk - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // ordered sum by the whole CTA: thread-strided partial sums, then a block reduce
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) acc[q] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; q++) acc[q] += *((volatile double*)&partials[(size_t)b * NV + q]);
  }
  __shared__ double sred[NV * 32];
  block_reduce<NV>(acc, sred);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = acc[q];
    *counter = 0u;
  }
  return true;
}

}  // namespace fame
