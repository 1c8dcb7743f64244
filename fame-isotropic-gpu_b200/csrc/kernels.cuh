// Kernels of the band-structure path: per-k tables, fused operator stages,
// CG (FP64 or FP32 with FP64 iterative refinement) and FP64 Lanczos.
#pragma once
#include "operator.cuh"

namespace fame {

// complex elements a thread holds in registers during one FFT pass (per precision)
template <typename R> struct Emax;
template <> struct Emax<float> { static constexpr int v = 16; };
template <> struct Emax<double> { static constexpr int v = 8; };

// ------------------------------------------------------------------ state
struct CgState {
  double r1, r0, beta;       // ||r||^2 now / before, r1/r0
  double a_re, a_im;         // CG step a = r1 / <p, Ap>
  double r1_0, tol2;         // initial ||r||^2, stop threshold on ||r||^2
  int iter;                  // the reference's counter k (starts at 1, CG.cu:301)
  int active;
  int maxit;
  int total;                 // CG products accumulated for the profile counter
  // outer iterative refinement (mixed precision)
  double rr, scale;          // ||b - A y||^2, 1/||b - A y|| used to scale the FP32 rhs
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

// ------------------------------------------------------------------ tables
// Per-k tables (FAME_Main/FAME_Matrix_Lambdas.cu:77-244 Simple, :288-489 General)
// computed on the device: one thread per table entry, FP64 sincospi.
__global__ void k_tables(Geom g, const Slot* slots, double2* tabs, double m1, double m2, double m3) {
  FAME_COUNT_LAUNCH();
  const int slot = blockIdx.y;
  const Slot sl = slots[slot];
  double2* t = tabs + (size_t)slot * g.tab_stride;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  if (!g.general) {
    // Lambda_d[n] = (e^{i 2 pi (n + theta_d)/N_d} - 1)/h_d,  D_d[n] = e^{i 2 pi theta_d n / N_d}
    if (i < Nx) {
      double2 e = expipi(2.0 * (i + sl.th[0]) / Nx);
      t[g.oLx + i] = make_double2((e.x - 1.0) / g.hx, e.y / g.hx);
      t[g.oDx + i] = expipi(2.0 * sl.th[0] * i / Nx);
    }
    if (i < Ny) {
      double2 e = expipi(2.0 * (i + sl.th[1]) / Ny);
      t[g.oLy + i] = make_double2((e.x - 1.0) / g.hy, e.y / g.hy);
      t[g.oDy + i] = expipi(2.0 * sl.th[1] * i / Ny);
    }
    if (i < Nz) {
      double2 e = expipi(2.0 * (i + sl.th[2]) / Nz);
      t[g.oLz + i] = make_double2((e.x - 1.0) / g.hz, e.y / g.hz);
      t[g.oDz + i] = expipi(2.0 * sl.th[2] * i / Nz);
    }
  } else {
    const double c1 = (m1 * m3) / ((double)Ny * Nx) - (m2 / Nx);
    const double c2 = -(m3 / Ny);
    if (i < Nx) {
      double2 e = expipi(2.0 * (i + sl.th[0]) / Nx);
      t[g.oLx + i] = make_double2((e.x - 1.0) / g.hx, e.y / g.hx);
      t[g.oDkx + i] = expipi(2.0 * sl.th[0] * i / Nx);
    }
    if (i < Nx * Ny) {
      const int x = i / Ny, y = i - x * Ny;
      // mxy = -m1*x/Nx + y (…Lambdas.cu:333-335), Lambda_y over (x, y)
      const double mxy = (-(m1 / Nx) * x) + y;
      double2 e = expipi(2.0 * (mxy + sl.th[1]) / Ny);
      t[g.oLy + i] = make_double2((e.x - 1.0) / g.hy, e.y / g.hy);
      // D_ky[x, y] = e^{i 2 pi (theta_xy - m1 x / Nx) y / Ny} (…Lambdas.cu:382-388)
      t[g.oDky + i] = expipi(2.0 * (sl.th[1] + x * (-m1 / Nx)) * y / Ny);
      // phase base of Lambda_z and D_kz: phi = (theta_xyz + c1 x + c2 y)
      const double ph = sl.th[2] + c1 * x + c2 * y;
      t[g.oExy + i] = expipi(2.0 * ph / Nz);
      t[g.oPhi + i] = make_double2(ph, 0.0);
    }
    if (i < Nz) t[g.oWz + i] = expipi(2.0 * i / Nz);
  }
}

// D_kz(x, y, z) = e^{i 2 pi phi(x,y) z / Nz} (…Lambdas.cu:389-400)
template <typename R>
__device__ __forceinline__ cplx<R> dkz_at(const Geom& g, const double2* tab, int x, int y, int z) {
  const double ph = tab[g.oPhi + x * g.Ny + y].x;
  if constexpr (sizeof(R) == 8) {
    // exact argument reduction of ph*z/Nz: the integer part of ph*z contributes 2*pi*n
    return expipi(2.0 * ph * z / g.Nz);
  } else {
    return to_f(expipi(2.0 * ph * z / g.Nz));
  }
}

// ------------------------------------------------------------------ plane stage
enum InMode { IN_VEC = 0, IN_CG = 1, IN_REFINE = 2 };
enum EpiMode { EPI_OUT = 0, EPI_CG = 1, EPI_RESID = 2 };
enum PencilMode { PEN_QBQ = 0, PEN_QR_OUT = 1, PEN_QRS_IN = 2 };

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
  CgState* cg;            // IN_CG / IN_REFINE
  double2* y64;           // IN_REFINE: FP64 accumulated solution (updated)
  const float2* x32;      // IN_REFINE: FP32 correction
  int sigma;              // IN_VEC: multiply the input by sqrt(Lambda_q) first (Sigma, …_Isotropic.cu:109)
  cplx<R>* T;             // output field (3 components)
  Cond reset;             // loop condition cleared by this kernel when it starts a loop body
};

// One cluster = 3 CTAs = the 3 components of plane s.  grid = (3*Ls, vec_per_slot, nslots)
template <typename R, bool GEN, int IN, bool PR>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(512)
    k_plane_inv(PlaneInArgs<R> a) {
  FAME_COUNT_LAUNCH();
  if ((threadIdx.x | blockIdx.x | blockIdx.y | blockIdx.z) == 0) set_cond(a.reset, 0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* plane = reinterpret_cast<cplx<R>*>(smem_raw);
  const Geom& g = a.g;
  cplx<R>* twf = plane + g.P;
  cplx<R>* twm = twf + g.Lf;
  cg::cluster_group cl = cg::this_cluster();
  const int comp = (int)cl.block_rank();
  const int s = blockIdx.x / 3;
  const int vec = blockIdx.y;
  const int slot = blockIdx.z;
  const Slot sl = a.slots[slot];
  if (!sl.active) return;  // uniform over the cluster
  CgState* st = nullptr;
  if constexpr (IN == IN_CG || IN == IN_REFINE) {
    st = a.cg + slot;
    if constexpr (IN == IN_CG) {
      if (!st->active) return;
    } else {
      if (!st->outer_active) return;
    }
  }
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < g.Lf; i += blockDim.x) twf[i] = a.tw[g.twf + i];
  for (int i = threadIdx.x; i < g.Lm; i += blockDim.x) twm[i] = a.tw[g.twm + i];
  cl.sync();  // every CTA of the cluster is running before remote writes

  const long vb = (long)(slot * a.vec_per_slot + vec) * a.vstride;
  const int Nd = sl.Nd, off = sl.off;
  cplx<R>* dst[3] = {cl.map_shared_rank(plane, 0), cl.map_shared_rank(plane, 1),
                     cl.map_shared_rank(plane, 2)};
  const int per = (g.P + 2) / 3;
  const int e0 = comp * per, e1 = min(g.P, e0 + per);
  R beta = 0;
  bool first = false;
  R rscale = 0;
  if constexpr (IN == IN_CG) {
    first = st->iter == 1;
    beta = (R)st->beta;
  }
  if constexpr (IN == IN_REFINE) rscale = (R)(1.0 / st->scale);
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int fi = s * g.P + e;
    cplx<R> v[3] = {mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0)};
    if (fi >= off) {
      const long i = fi - off;
      const int m = e / g.Lf, f = e - m * g.Lf;
      double2 Lx, Ly, Lz;
      lambdas_at(g, tab, s, m, f, Lx, Ly, Lz);
      cplx<R> x1, x2;
      if constexpr (IN == IN_VEC) {
        x1 = a.in[vb + i];
        x2 = a.in[vb + Nd + i];
        if (a.sigma) {
          const R sc = (R)sqrt(cabs2(Lx) + cabs2(Ly) + cabs2(Lz));
          x1 = cscale(x1, sc);
          x2 = cscale(x2, sc);
        }
      } else if constexpr (IN == IN_CG) {
        const cplx<R> r1 = a.r[vb + i], r2 = a.r[vb + Nd + i];
        if (first) {
          x1 = r1;
          x2 = r2;
        } else {
          const cplx<R> p1 = a.p[vb + i], p2 = a.p[vb + Nd + i];
          x1 = mk<R>(r1.x + beta * p1.x, r1.y + beta * p1.y);
          x2 = mk<R>(r2.x + beta * p2.x, r2.y + beta * p2.y);
        }
        a.p[vb + i] = x1;
        a.p[vb + Nd + i] = x2;
      } else {  // IN_REFINE (R = double): y += x32 / scale, mix y
        const float2 c1 = a.x32[vb + i], c2 = a.x32[vb + Nd + i];
        double2 y1 = a.y64[vb + i], y2 = a.y64[vb + Nd + i];
        y1.x += (double)c1.x * rscale;
        y1.y += (double)c1.y * rscale;
        y2.x += (double)c2.x * rscale;
        y2.y += (double)c2.y * rscale;
        a.y64[vb + i] = y1;
        a.y64[vb + Nd + i] = y2;
        x1 = cvt<R>(y1);
        x2 = cvt<R>(y2);
      }
      cplx<R> P[6];
      pi_at<R>(GEN, PR, Lx, Ly, Lz, P, nullptr);
#pragma unroll
      for (int c = 0; c < 3; c++) v[c] = cadd(cmul(P[c], x1), cmul(P[3 + c], x2));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) dst[c][e] = v[c];
  }
  cl.sync();

  // inverse 2-D transform of this component's plane (unnormalised)
  LineSet rows{g.Lm, g.Lf, 1, false};   // lines along the fast axis
  LineSet cols{g.Lf, 1, g.Lf, true};    // lines along the mid axis
  fft_lines<R, Emax<R>::v>(plane, g.pf, rows, twf, true);
  if constexpr (GEN) {
    // x D_kz(x, y, z) after the z (fast) pass (FAME_FFT_CUDA.cu:278, kernel :452-487)
    for (int e = threadIdx.x; e < g.P; e += blockDim.x) {
      const int m = e / g.Lf, f = e - m * g.Lf;
      plane[e] = cmul(plane[e], dkz_at<R>(g, tab, s, m, f));
    }
    __syncthreads();
  }
  fft_lines<R, Emax<R>::v>(plane, g.pm, cols, twm, true);
  if constexpr (GEN) {
    // x D_ky(x, y) after the y (mid) pass (FAME_FFT_CUDA.cu:284, kernel :367-404)
    for (int e = threadIdx.x; e < g.P; e += blockDim.x) {
      const int m = e / g.Lf;
      plane[e] = cmul(plane[e], cvt<R>(tab[g.oDky + s * g.Ny + m]));
    }
    __syncthreads();
  }
  cplx<R>* T = a.T + (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + (long)s * g.P;
  for (int e = threadIdx.x; e < g.P; e += blockDim.x) T[e] = plane[e];
}

// ------------------------------------------------------------------ pencil stage
template <typename R>
struct PencilArgs {
  Geom g;
  const Slot* slots;
  const double2* tabs;
  const cplx<R>* tw;
  long fstride;
  int vec_per_slot;
  cplx<R>* T;              // field in frequency-plane layout (in/out)
  const R* invB;           // PEN_QBQ: 1/eps per edge (3N, spatial layout); PEN_QR_OUT: optional
  cplx<R>* out;            // PEN_QR_OUT: spatial field out (3N per vector)
  const cplx<R>* in;       // PEN_QRS_IN: spatial field in
  const CgState* cg;       // optional activity gate
  int gate;                // 0 none, 1 CG active, 2 outer refinement active
  int TW;                  // fast positions per CTA
};

// grid = (Lm * ceil(Lf/TW), 3 * vec_per_slot, nslots)
template <typename R, bool GEN, int MODE>
__global__ void __launch_bounds__(256) k_pencil(PencilArgs<R> a) {
  FAME_COUNT_LAUNCH();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  const int TW = a.TW;
  cplx<R>* tile = reinterpret_cast<cplx<R>*>(smem_raw);  // [Ls][TW]
  cplx<R>* tws = tile + g.Ls * TW;
  const int slot = blockIdx.z;
  const Slot sl = a.slots[slot];
  if (!sl.active) return;
  if (a.gate == 1 && !a.cg[slot].active) return;
  if (a.gate == 2 && !a.cg[slot].outer_active) return;
  const int comp = blockIdx.y % 3, vec = blockIdx.y / 3;
  const int nft = (g.Lf + TW - 1) / TW;
  const int m = blockIdx.x / nft;
  const int f0 = (blockIdx.x - m * nft) * TW;
  const int tw_n = min(TW, g.Lf - f0);
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < g.Ls; i += blockDim.x) tws[i] = a.tw[g.tws + i];
  const long fb = (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N;
  const int Ls = g.Ls;
  // ---- load
  for (int q = threadIdx.x; q < Ls * TW; q += blockDim.x) {
    const int s = q / TW, f = q - s * TW;
    cplx<R> v = mk<R>(0, 0);
    if (f < tw_n) {
      if constexpr (MODE == PEN_QRS_IN) {
        // spatial input, x conj(D) before the forward transform
        long sp;
        cplx<R> d;
        if (!GEN) {
          sp = (long)s * g.P + m * g.Lf + f0 + f;
          const double2 dd = cmul(cmul(tab[g.oDz + s], tab[g.oDy + m]), tab[g.oDx + f0 + f]);
          d = cvt<R>(cconj(dd));
        } else {
          sp = ((long)(f0 + f) * g.Ny + m) * g.Nx + s;
          d = cvt<R>(cconj(tab[g.oDkx + s]));
        }
        v = cmul(a.in[(long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + sp], d);
      } else {
        v = a.T[fb + (long)s * g.P + m * g.Lf + f0 + f];
      }
    }
    tile[q] = v;
  }
  __syncthreads();
  LineSet L{TW, 1, TW, true};
  if constexpr (MODE == PEN_QBQ || MODE == PEN_QR_OUT) {
    fft_lines<R, Emax<R>::v>(tile, g.ps, L, tws, true);
    const R invN = (R)(1.0 / g.N);
    for (int q = threadIdx.x; q < Ls * TW; q += blockDim.x) {
      const int s = q / TW, f = q - s * TW;
      if (f < tw_n) {
        long sp;
        if (!GEN)
          sp = (long)s * g.P + m * g.Lf + f0 + f;
        else
          sp = ((long)(f0 + f) * g.Ny + m) * g.Nx + s;
        if constexpr (MODE == PEN_QBQ) {
          tile[q] = cscale(tile[q], a.invB[(long)comp * g.N + sp] * invN);
        } else {
          cplx<R> d;
          if (!GEN)
            d = cvt<R>(cmul(cmul(tab[g.oDz + s], tab[g.oDy + m]), tab[g.oDx + f0 + f]));
          else
            d = cvt<R>(tab[g.oDkx + s]);
          cplx<R> v = cscale(cmul(tile[q], d), invN);
          if (a.invB) v = cscale(v, a.invB[(long)comp * g.N + sp]);
          a.out[(long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + sp] = v;
        }
      }
    }
    __syncthreads();
  }
  if constexpr (MODE == PEN_QBQ || MODE == PEN_QRS_IN) {
    fft_lines<R, Emax<R>::v>(tile, g.ps, L, tws, false);
    for (int q = threadIdx.x; q < Ls * TW; q += blockDim.x) {
      const int s = q / TW, f = q - s * TW;
      if (f < tw_n) a.T[fb + (long)s * g.P + m * g.Lf + f0 + f] = tile[q];
    }
  }
}

// ------------------------------------------------------------------ plane stage (forward)
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
  const cplx<R>* b;        // EPI_RESID: right-hand side
  CgState* cg;
  double* partials;        // [nslots][blocks per slot][NV]
  unsigned* counters;      // [nslots] ticket counters, plus [nslots] = grid counter
  Cond cond;               // EPI_RESID: outer WHILE condition
  int nslots;
  double tol2;             // EPI_RESID: absolute tolerance^2 on ||b - A y||
};

template <typename R, bool GEN, int EPI, bool PR>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(512)
    k_plane_fwd(PlaneOutArgs<R> a) {
  FAME_COUNT_LAUNCH();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* plane = reinterpret_cast<cplx<R>*>(smem_raw);
  const Geom& g = a.g;
  cplx<R>* twf = plane + g.P;
  cplx<R>* twm = twf + g.Lf;
  cg::cluster_group cl = cg::this_cluster();
  const int comp = (int)cl.block_rank();
  const int s = blockIdx.x / 3;
  const int vec = blockIdx.y;
  const int slot = blockIdx.z;
  const Slot sl = a.slots[slot];
  bool live = sl.active;
  if constexpr (EPI == EPI_CG) live = live && a.cg[slot].active;
  if constexpr (EPI == EPI_RESID) live = live && a.cg[slot].outer_active;
  if (!live) {
    if constexpr (EPI == EPI_RESID) {
      if (grid_last(a.counters + a.nslots, gridDim.x * gridDim.y * gridDim.z)) {
        if (threadIdx.x == 0) {
          int any = 0;
          for (int q = 0; q < a.nslots; q++) any |= a.slots[q].active && a.cg[q].outer_active;
          decide_cond(a.cond, any);
        }
      }
    }
    return;
  }
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < g.Lf; i += blockDim.x) twf[i] = a.tw[g.twf + i];
  for (int i = threadIdx.x; i < g.Lm; i += blockDim.x) twm[i] = a.tw[g.twm + i];
  const cplx<R>* T = a.T + (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + (long)s * g.P;
  for (int e = threadIdx.x; e < g.P; e += blockDim.x) plane[e] = T[e];
  __syncthreads();
  LineSet rows{g.Lm, g.Lf, 1, false};
  LineSet cols{g.Lf, 1, g.Lf, true};
  if constexpr (GEN) {
    // T*: x conj(D_ky), y (mid) pass, x conj(D_kz), z (fast) pass (FAME_FFT_CUDA.cu:297-319)
    for (int e = threadIdx.x; e < g.P; e += blockDim.x) {
      const int m = e / g.Lf;
      plane[e] = cmul(plane[e], cvt<R>(cconj(tab[g.oDky + s * g.Ny + m])));
    }
    __syncthreads();
    fft_lines<R, Emax<R>::v>(plane, g.pm, cols, twm, false);
    for (int e = threadIdx.x; e < g.P; e += blockDim.x) {
      const int m = e / g.Lf, f = e - m * g.Lf;
      plane[e] = cmul(plane[e], cconj(dkz_at<R>(g, tab, s, m, f)));
    }
    __syncthreads();
    fft_lines<R, Emax<R>::v>(plane, g.pf, rows, twf, false);
  } else {
    fft_lines<R, Emax<R>::v>(plane, g.pf, rows, twf, false);
    fft_lines<R, Emax<R>::v>(plane, g.pm, cols, twm, false);
  }
  cl.sync();  // all three component planes transformed

  const cplx<R>* src[3] = {cl.map_shared_rank(plane, 0), cl.map_shared_rank(plane, 1),
                           cl.map_shared_rank(plane, 2)};
  const int per = (g.P + 2) / 3;
  const int e0 = comp * per, e1 = min(g.P, e0 + per);
  const int Nd = sl.Nd, off = sl.off;
  const long vb = (long)(slot * a.vec_per_slot + vec) * a.vstride;
  double acc[2] = {0.0, 0.0};
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int fi = s * g.P + e;
    if (fi < off) continue;
    const long i = fi - off;
    const cplx<R> t0 = src[0][e], t1 = src[1][e], t2 = src[2][e];
    const int m = e / g.Lf, f = e - m * g.Lf;
    double2 Lx, Ly, Lz;
    lambdas_at(g, tab, s, m, f, Lx, Ly, Lz);
    cplx<R> P[6];
    pi_at<R>(GEN, PR, Lx, Ly, Lz, P, nullptr);
    const cplx<R> o1 = cadd(cadd(cmulc(P[0], t0), cmulc(P[1], t1)), cmulc(P[2], t2));
    const cplx<R> o2 = cadd(cadd(cmulc(P[3], t0), cmulc(P[4], t1)), cmulc(P[5], t2));
    if constexpr (EPI == EPI_OUT) {
      a.out[vb + i] = o1;
      a.out[vb + Nd + i] = o2;
    } else if constexpr (EPI == EPI_CG) {
      a.out[vb + i] = o1;
      a.out[vb + Nd + i] = o2;
      const cplx<R> p1 = a.p[vb + i], p2 = a.p[vb + Nd + i];
      const cplx<R> d = cadd(cmulc(p1, o1), cmulc(p2, o2));  // conj(p) Ap
      acc[0] += (double)d.x;
      acc[1] += (double)d.y;
    } else {  // EPI_RESID
      const cplx<R> r1 = csub(a.b[vb + i], o1), r2 = csub(a.b[vb + Nd + i], o2);
      a.out[vb + i] = r1;
      a.out[vb + Nd + i] = r2;
      acc[0] += (double)(cabs2(r1) + cabs2(r2));
    }
  }
  cl.sync();  // remote shared memory must outlive the readers

  if constexpr (EPI == EPI_CG || EPI == EPI_RESID) {
    __shared__ double sred[2 * 32];
    block_reduce<2>(acc, sred);
    const int nblk = gridDim.x;  // CTAs of this slot (vec_per_slot == 1 in solves)
    double tot[2];
    if (slot_reduce<2>(acc, a.partials + (size_t)slot * nblk * 2, a.counters + slot, blockIdx.x, nblk,
                       tot)) {
      if (threadIdx.x == 0) {
        CgState* st = a.cg + slot;
        if constexpr (EPI == EPI_CG) {
          // a = r1 / dot  (CG.cu:325-328)
          const double den = tot[0] * tot[0] + tot[1] * tot[1];
          st->a_re = st->r1 * tot[0] / den;
          st->a_im = -st->r1 * tot[1] / den;
        } else {
          st->rr = tot[0];
          st->outer++;
          st->outer_total++;
          st->outer_active = (tot[0] > a.tol2) && (st->outer < st->outer_max);
          st->scale = 1.0 / sqrt(tot[0] > 0 ? tot[0] : 1.0);
        }
        __threadfence();
      }
    }
    if constexpr (EPI == EPI_RESID) {
      if (grid_last(a.counters + a.nslots, gridDim.x * gridDim.y * gridDim.z)) {
        if (threadIdx.x == 0) {
          int any = 0;
          for (int q = 0; q < a.nslots; q++) any |= a.slots[q].active && a.cg[q].outer_active;
          decide_cond(a.cond, any);
        }
      }
    }
  }
}

}  // namespace fame
