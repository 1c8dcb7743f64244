// Operator stage kernels (plane inverse, pencil, plane forward); explicitly
// instantiated per precision, lattice family and geometry policy in ops_*.cu.
//
// GP is the geometry policy (geom_policy.cuh): runtime lengths (DynGeom) or
// compile-time lengths (StatGeom<...>).
#pragma once
#include "geom_policy.cuh"

namespace fame {

// Lambda_x, Lambda_y, Lambda_z at plane element (m, f) of plane s, in precision R.
// Simple lattices read the per-CTA shared tables lx[f], ly[m] and the plane's lz.
template <typename R, bool GEN>
__device__ __forceinline__ void lam_elem(const Geom& g, const double2* tab, const cplx<R>* lx, const cplx<R>* ly,
                                         cplx<R> lz, int s, int m, int f, cplx<R>& Lx, cplx<R>& Ly,
                                         cplx<R>& Lz) {
  if constexpr (!GEN) {
    Lx = lx[f];
    Ly = ly[m];
    Lz = lz;
  } else {
    double2 a, b, c;
    lambdas_at(g, tab, s, m, f, a, b, c);
    Lx = cvt<R>(a);
    Ly = cvt<R>(b);
    Lz = cvt<R>(c);
  }
}

// ------------------------------------------------------------------ L2 prefetch
// The CTAs of a stage kernel run in waves in launch order, and each one spends most of
// its time on shared-memory transforms.  A CTA therefore issues, at its start, bulk L2
// prefetches of the global operands of the CTA pf_dist places later (about one wave
// ahead), so that CTA finds them in L2 instead of waiting on DRAM.  The prefetches only
// cover bytes that CTA will read.

// Linear launch index of this CTA, and the (x, y, z) block of linear index t.
__device__ __forceinline__ long cta_linear() {
  return blockIdx.x + (long)gridDim.x * (blockIdx.y + (long)gridDim.y * blockIdx.z);
}
__device__ __forceinline__ bool cta_of(long t, int& x, int& y, int& z) {
  const long n = (long)gridDim.x * gridDim.y * gridDim.z;
  if (t >= n) return false;
  x = (int)(t % gridDim.x);
  const long r = t / gridDim.x;
  y = (int)(r % gridDim.y);
  z = (int)(r / gridDim.y);
  return true;
}

// The reduced-vector range [e0, e1) of plane s that the component-`comp` CTA of a
// plane cluster mixes, as element offsets (first half; the second starts Nd later).
__device__ __forceinline__ bool plane_vec_range(int P, int s, int comp, const Slot& sl, long& i0, long& i1) {
  const int per = (P + 2) / 3;
  const int e0 = comp * per, e1 = min(P, e0 + per);
  i0 = max(0L, (long)s * P + e0 - sl.off);
  i1 = (long)s * P + e1 - sl.off;
  return i1 > i0;
}

// One cluster = 3 CTAs = the 3 components of plane s.  grid = (3*Ls, vec_per_slot, nslots)
template <typename R, bool GEN, int IN, bool PR, int RARE, class GP>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(GP::kMaxPlaneThreads, GP::template plane_min_blocks<R, RARE>())
    k_plane_inv(PlaneInArgs<R> a) {
  FAME_COUNT_LAUNCH();
  if ((threadIdx.x | blockIdx.x | blockIdx.y | blockIdx.z) == 0) set_cond(a.reset, 0);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  const int Lf = GP::Lf(g), Lm = GP::Lm(g), S = GP::S(g), P = GP::P(g);
  const Div dlf(Lf);  // row of plane element e: e / Lf (folds to a constant for static geometries)
  cplx<R>* plane = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* twf = plane + Lm * S;  // plane rows have the odd pitch S >= Lf
  cplx<R>* twm = twf + Lf;
  cplx<R>* lx = twm + Lm;
  cplx<R>* ly = lx + Lf;
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
  if constexpr (IN == IN_CG) {
    // this CTA's own r, p and x, all at once: the batched loads of the mix below then
    // wait on one DRAM latency and find the rest in L2
    long i0, i1;
    if (a.self_pf && threadIdx.x < (st->iter == 1 ? 2 : 6) && plane_vec_range(P, s, comp, sl, i0, i1)) {
      const cplx<R>* v = threadIdx.x < 2 ? a.r : threadIdx.x < 4 ? a.p : a.x;
      const long base = (long)(slot * a.vec_per_slot + vec) * a.vstride + ((threadIdx.x & 1) ? sl.Nd : 0);
      prefetch_l2(v + base + i0, (i1 - i0) * sizeof(cplx<R>));
    }
  }
  if constexpr (IN == IN_CG) {
    // r, p and x of the CTA one wave ahead (p and x once its k-point is past k = 1)
    int x2, y2, z2;
    if (a.pf_dist > 0 && threadIdx.x < 6 && cta_of(cta_linear() + a.pf_dist, x2, y2, z2)) {
      const Slot s2 = a.slots[z2];
      const CgState* c2 = a.cg + z2;
      long i0, i1;
      const int which = threadIdx.x >> 1;  // 0 r, 1 p, 2 x
      if (s2.active && c2->active && (which == 0 || c2->iter > 1) &&
          plane_vec_range(P, x2 / 3, x2 % 3, s2, i0, i1)) {
        const cplx<R>* v = which == 0 ? a.r : which == 1 ? a.p : a.x;
        const long base = (long)(z2 * a.vec_per_slot + y2) * a.vstride + ((threadIdx.x & 1) ? s2.Nd : 0);
        prefetch_l2(v + base + i0, (i1 - i0) * sizeof(cplx<R>));
      }
    }
  }
  // Static geometries exchange the mixed components with st.async into the owner's
  // plane, counted on the owner's barrier `xbar` (P values arrive per plane); the
  // others use a cluster barrier after the exchange.
  constexpr bool kAsyncMix = GP::kStatic;
  __shared__ __align__(8) unsigned long long xbar;
  const unsigned bar = smem_u32(&xbar);
  // after a failed exchange (the fault marker), later launches skip their work: the
  // cluster's rank-0 CTA reads the marker and all three CTAs act on its value
  __shared__ int skip;
  if (kAsyncMix && threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence_cluster();
    skip = a.fault ? *(volatile int*)a.fault : 0;
  }
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < Lf; i += GP::plane_threads()) {
    twf[i] = a.tw[g.twf + i];
    if constexpr (!GEN) lx[i] = cvt<R>(tab[g.oLx + i]);
  }
  for (int i = threadIdx.x; i < Lm; i += GP::plane_threads()) {
    twm[i] = a.tw[g.twm + i];
    if constexpr (!GEN) ly[i] = cvt<R>(tab[g.oLy + i]);
  }
  const cplx<R> lz = GEN ? mk<R>(0, 0) : cvt<R>(tab[g.oLz + s]);
  cl.sync();  // every CTA of the cluster is running (and the tables and barriers are in place)
  if constexpr (kAsyncMix) {
    if (*cl.map_shared_rank(&skip, 0)) {
      cl.sync();  // rank 0's marker stays readable until all three have read it
      return;
    }
  }
  if (kAsyncMix && threadIdx.x == 0) mbar_arrive_expect_tx(bar, (unsigned)(P * sizeof(cplx<R>)));
  unsigned rplane[3], rbar[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    rplane[c] = kAsyncMix ? mapa_u32(smem_u32(plane), c) : 0u;
    rbar[c] = kAsyncMix ? mapa_u32(bar, c) : 0u;
  }

  const long vb = (long)(slot * a.vec_per_slot + vec) * a.vstride;
  const int Nd = sl.Nd, off = sl.off;
  cplx<R>* dst[3] = {cl.map_shared_rank(plane, 0), cl.map_shared_rank(plane, 1),
                     cl.map_shared_rank(plane, 2)};
  const int per = (P + 2) / 3;
  const int e0 = comp * per, e1 = min(P, e0 + per);
  R beta = 0;
  bool first = false;
  R rscale = 0;
  // CG step size a of the last update: the solution update x += a p is applied here
  // (IN_CG: the previous iteration's, IN_REFINE: the inner solve's last) instead of
  // in the vector update kernel, where it would cost another pass over p and x
  R are = 0, aim = 0;
  if constexpr (IN == IN_CG) {
    first = st->iter == 1;
    beta = (R)st->beta;
    are = (R)st->a_re;
    aim = (R)st->a_im;
  }
  float fre = 0.f, fim = 0.f;
  bool pend = false;
  if constexpr (IN == IN_REFINE) {
    rscale = (R)(1.0 / st->scale);
    pend = st->iter > 1;
    fre = (float)st->a_re;
    fim = (float)st->a_im;
  }
  // Input stage and the 2 -> 3 mix.  IN_CG: p = r + beta p (p = r at k = 1) and the
  // deferred x += a p (CG.cu:39-51, :65-66).  IN_REFINE: y += x32 / scale with the
  // inner solve's last update folded in.  The operands of KB points per thread are
  // loaded up front, so one global-load latency covers KB points.
  // (runtime geometries run at 64 registers: two points)
  constexpr int KB = !GP::kStatic ? 2 : IN == IN_VEC ? 8 : 2;
  const int NT = GP::plane_threads();
  for (int eb = e0 + threadIdx.x; eb < e1; eb += KB * NT) {
    cplx<R> A1[KB], A2[KB], B1[KB], B2[KB], C1[KB], C2[KB];
    float2 F1[KB], F2[KB], G1[KB], G2[KB];
#pragma unroll
    for (int k = 0; k < KB; k++) {
      const int e = eb + k * NT;
      if (e < e1 && s * P + e >= off) {
        const long i = s * P + e - off;
        if constexpr (IN == IN_VEC) {
          A1[k] = a.in[vb + i];
          A2[k] = a.in[vb + Nd + i];
        } else if constexpr (IN == IN_CG) {
          A1[k] = a.r[vb + i];
          A2[k] = a.r[vb + Nd + i];
          if (!first) {
            B1[k] = a.p[vb + i];
            B2[k] = a.p[vb + Nd + i];
            C1[k] = a.x[vb + i];
            C2[k] = a.x[vb + Nd + i];
          }
        } else {  // IN_REFINE (R = double)
          A1[k] = a.y64[vb + i];
          A2[k] = a.y64[vb + Nd + i];
          F1[k] = a.x32[vb + i];
          F2[k] = a.x32[vb + Nd + i];
          if (pend) {
            G1[k] = a.p32[vb + i];
            G2[k] = a.p32[vb + Nd + i];
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < KB; k++) {
      const int e = eb + k * NT;
      if (e >= e1) break;
      const int fi = s * P + e;
      const int m = GP::kStatic ? e / Lf : (int)dlf.q(e), f = e - m * Lf;
      cplx<R> v[3] = {mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0)};
      if (fi >= off) {
        const long i = fi - off;
        cplx<R> Lx, Ly, Lz;
        lam_elem<R, GEN>(g, tab, lx, ly, lz, s, m, f, Lx, Ly, Lz);
        cplx<R> x1 = A1[k], x2 = A2[k];
        if constexpr (IN == IN_VEC) {
          if (a.sigma) {
            const R sc = sqrt(cabs2(Lx) + cabs2(Ly) + cabs2(Lz));
            x1 = cscale(x1, sc);
            x2 = cscale(x2, sc);
          }
        } else if constexpr (IN == IN_CG) {
          if (!first) {
            cplx<R> s1 = C1[k], s2 = C2[k];
            const cplx<R> p1 = B1[k], p2 = B2[k];
            if constexpr (sizeof(R) == 4) {
              // the FP32 CG's step size is real (<p, Ap> from the pencil stage): packed pairs
              s1 = pfma(p1, are, s1);
              s2 = pfma(p2, are, s2);
              x1 = pfma(p1, beta, x1);
              x2 = pfma(p2, beta, x2);
            } else {
              s1.x += are * p1.x - aim * p1.y;
              s1.y += are * p1.y + aim * p1.x;
              s2.x += are * p2.x - aim * p2.y;
              s2.y += are * p2.y + aim * p2.x;
              x1 = mk<R>(x1.x + beta * p1.x, x1.y + beta * p1.y);
              x2 = mk<R>(x2.x + beta * p2.x, x2.y + beta * p2.y);
            }
            a.x[vb + i] = s1;
            a.x[vb + Nd + i] = s2;
          }
          a.p[vb + i] = x1;
          a.p[vb + Nd + i] = x2;
        } else {  // IN_REFINE
          float2 c1 = F1[k], c2 = F2[k];
          if (pend) {
            const float2 q1 = G1[k], q2 = G2[k];
            c1.x += fre * q1.x - fim * q1.y;
            c1.y += fre * q1.y + fim * q1.x;
            c2.x += fre * q2.x - fim * q2.y;
            c2.y += fre * q2.y + fim * q2.x;
          }
          x1.x += (double)c1.x * rscale;
          x1.y += (double)c1.y * rscale;
          x2.x += (double)c2.x * rscale;
          x2.y += (double)c2.y * rscale;
          a.y64[vb + i] = x1;
          a.y64[vb + Nd + i] = x2;
        }
        cplx<R> Pc[6];
        pi_from<R>(GEN, PR, Lx, Ly, Lz, Pc);
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = cadd(cmul(Pc[c], x1), cmul(Pc[3 + c], x2));
      }
      if constexpr (kAsyncMix) {
        const unsigned o = (unsigned)((m * S + f) * sizeof(cplx<R>));
#pragma unroll
        for (int c = 0; c < 3; c++) st_async(rplane[c] + o, v[c], rbar[c]);
      } else {
#pragma unroll
        for (int c = 0; c < 3; c++) dst[c][m * S + f] = v[c];
      }
    }
  }
  if constexpr (kAsyncMix) {
    // this CTA's plane is complete once all P values have arrived.  A wait that runs out
    // (about 0.1 s; it cannot unless the exchange is broken) records the fault and goes
    // on, and later launches return at once (below), so the solve ends with an error.
    if (!mbar_wait(bar, 0, 200000000LL) && a.fault) atomicExch(a.fault, 1);
    __syncthreads();
  } else {
    cl.sync();
  }

  // inverse 2-D transform of this component's plane (unnormalised): fast axis,
  // then mid axis.  One FFT call site per axis loop keeps the kernel within its
  // register budget.
  if constexpr (GP::kStatic && !GEN) {
    GP::template fft_plane_c<R, true, true>(plane, twf);
    GP::template fft_plane_c<R, false, true>(plane, twm);
  }
  for (int ax = 0; !(GP::kStatic && !GEN) && ax < 2; ax++) {
    GP::template fft_plane<R, RARE>(plane, g, ax == 0, ax == 0 ? twf : twm, true);
    if constexpr (GEN) {
      // x D_kz(x,y,z) after the z (fast) pass (FAME_FFT_CUDA.cu:109, kernel :283-317),
      // x D_ky(x,y) after the y (mid) pass (FAME_FFT_CUDA.cu:115, kernel :198-234)
      for (int e = threadIdx.x; e < P; e += GP::plane_threads()) {
        const int m = GP::kStatic ? e / Lf : (int)dlf.q(e), f = e - m * Lf;
        const int q = m * S + f;
        plane[q] = cmul(plane[q], ax == 0 ? dkz_at<R>(g, tab, s, m, f) : cvt<R>(tab[g.oDky + s * g.Ny + m]));
      }
      __syncthreads();
    }
  }
  cplx<R>* T = a.T + (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + (long)s * P;
  for (int e = threadIdx.x; e < P; e += GP::plane_threads()) {
    const int m = GP::kStatic ? e / Lf : (int)dlf.q(e);
    T[e] = plane[e + m * (S - Lf)];
  }
}

// ------------------------------------------------------------------ pencil stage

// grid = (Lm * ceil(Lf/TW), 3 * vec_per_slot, nslots), kPencilThreads threads
template <typename R, bool GEN, int MODE, int RARE, class GP>
__global__ void __launch_bounds__(kPencilThreads, GP::kStatic ? (sizeof(R) == 4 ? 3 : 2) : 3)
    k_pencil(PencilArgs<R> a) {
  FAME_COUNT_LAUNCH();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  constexpr int TW = PencilTW<R>::v;
  const int Lf = GP::Lf(g), Ls = GP::Ls(g), P = GP::P(g);
  // shared memory: tile [Ls][TW] | 1/eps tile [Ls][TW] (PEN_QBQ) | slow-axis twiddles [Ls]
  cplx<R>* tile = reinterpret_cast<cplx<R>*>(smem_raw);
  R* ibt = reinterpret_cast<R*>(tile + Ls * TW);
  cplx<R>* tws = reinterpret_cast<cplx<R>*>(ibt + Ls * TW);
  constexpr bool QBQ = MODE == PEN_QBQ || MODE == PEN_QBQ_CG;
  const int slot = blockIdx.z;
  const Slot sl = a.slots[slot];
  if (!sl.active) return;
  if (a.gate == 1 && !a.cg[slot].active) return;
  if (a.gate == 2 && !a.cg[slot].outer_active) return;
  const int comp = blockIdx.y % 3, vec = blockIdx.y / 3;
  const int nft = (Lf + TW - 1) / TW;
  const int m = blockIdx.x / nft;
  const int f0 = (blockIdx.x - m * nft) * TW;
  const int tw_n = min(TW, Lf - f0);
  if constexpr (MODE == PEN_QBQ_CG) {
    // the field rows and 1/eps rows of the tile of the CTA one wave ahead
    int x2, y2, z2;
    if (a.pf_dist > 0 && threadIdx.x < 2 * Ls && cta_of(cta_linear() + a.pf_dist, x2, y2, z2) &&
        a.slots[z2].active && a.cg[z2].active) {
      const int m2 = x2 / nft, f2 = (x2 - m2 * nft) * TW, c2 = y2 % 3, v2 = y2 / 3;
      const int n2 = min(TW, Lf - f2);
      const int srow = threadIdx.x < Ls ? threadIdx.x : threadIdx.x - Ls;
      const long off = (long)c2 * g.N + (long)srow * P + m2 * Lf + f2;
      if (threadIdx.x < Ls)
        prefetch_l2(a.T + (long)(z2 * a.vec_per_slot + v2) * a.fstride + off, n2 * sizeof(cplx<R>));
      else
        prefetch_l2(a.invB + off, n2 * sizeof(R));
    }
  }
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < Ls; i += kPencilThreads) tws[i] = a.tw[g.tws + i];
  const long fb = (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N;
  // ---- load.  Full tiles of the QBQ stream the field rows (TW contiguous
  // elements at stride P) and the 1/eps rows (1/eps in the field layout) straight
  // into shared memory with 16-byte cp.async copies.
  constexpr int CH = 16 / sizeof(cplx<R>);    // elements per 16-byte copy
  constexpr int CHB = 16 / sizeof(R);         // 1/eps values per 16-byte copy
  const bool ib_field = !GEN || a.ib_field;  // 1/eps rows contiguous along the tile's fast positions
  const bool async_tile = QBQ && ib_field && tw_n == TW && Lf % CHB == 0;
  if (async_tile) {
    for (int q = threadIdx.x; q < Ls * (TW / CH); q += kPencilThreads) {
      const int s = q / (TW / CH), c = q - s * (TW / CH);
      cp_async16(tile + s * TW + c * CH, a.T + fb + (long)s * P + m * Lf + f0 + c * CH);
    }
    for (int q = threadIdx.x; q < Ls * (TW / CHB); q += kPencilThreads) {
      const int s = q / (TW / CHB), c = q - s * (TW / CHB);
      cp_async16(ibt + s * TW + c * CHB, a.invB + (long)comp * g.N + (long)s * P + m * Lf + f0 + c * CHB);
    }
  } else {
  for (int q = threadIdx.x; q < Ls * TW; q += kPencilThreads) {
    const int s = q / TW, f = q - s * TW;
    cplx<R> v = mk<R>(0, 0);
    if (f < tw_n) {
      if constexpr (MODE == PEN_QRS_IN) {
        // spatial input, x conj(D) before the forward transform
        long sp;
        cplx<R> d;
        if (!GEN) {
          sp = (long)s * P + m * Lf + f0 + f;
          const double2 dd = cmul(cmul(tab[g.oDz + s], tab[g.oDy + m]), tab[g.oDx + f0 + f]);
          d = cvt<R>(cconj(dd));
        } else {
          sp = ((long)(f0 + f) * g.Ny + m) * g.Nx + s;
          d = cvt<R>(cconj(tab[g.oDkx + s]));
        }
        v = cmul(a.in[(long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + sp], d);
      } else {
        v = a.T[fb + (long)s * P + m * Lf + f0 + f];
      }
    }
    tile[q] = v;
  }
  }
  if (async_tile) cp_async_wait_all();
  __syncthreads();
  // QBQ: inverse, x B^{-1}/N, forward.  QR_OUT: inverse, x D/N (and B^{-1}), store.
  // QRS_IN: forward only.  One FFT call site (dir loop) for the register budget.
  constexpr int ndir = QBQ ? 2 : 1;
  // PEN_QBQ_CG: sum of |v|^2 / eps over the tile after the inverse transform
  float dot = 0.f;
  constexpr bool kStatQBQ = GP::kStatic && QBQ;  // whole tiles, 1/eps staged in shared memory
  if constexpr (kStatQBQ) {
    GP::template fft_slow_c<R, true>(tile, tws);
    const R invN = (R)(1.0 / g.N);
#pragma unroll 4
    for (int q = threadIdx.x; q < Ls * TW; q += kPencilThreads) {
      const R ib = ibt[q];
      const cplx<R> v = tile[q];
      if constexpr (MODE == PEN_QBQ_CG) dot += (float)(ib * cabs2(v));
      if constexpr (sizeof(R) == 4)
        tile[q] = pscale(v, ib * invN);
      else
        tile[q] = cscale(v, ib * invN);
    }
    __syncthreads();
    GP::template fft_slow_c<R, false>(tile, tws);
  }
  for (int dir = 0; !kStatQBQ && dir < ndir; dir++) {
    const bool inv = MODE == PEN_QRS_IN ? false : dir == 0;
    GP::template fft_slow<R, RARE>(tile, g, tws, inv);
    if (MODE != PEN_QRS_IN && dir == 0) {
      const R invN = (R)(1.0 / g.N);
      for (int q = threadIdx.x; q < Ls * TW; q += kPencilThreads) {
        const int s = q / TW, f = q - s * TW;
        if (f < tw_n) {
          long sp;
          if (!GEN)
            sp = (long)s * P + m * Lf + f0 + f;
          else
            sp = ((long)(f0 + f) * g.Ny + m) * g.Nx + s;
          if constexpr (QBQ) {
            const long ii = ib_field ? (long)s * P + m * Lf + f0 + f : sp;
            const R ib = async_tile ? ibt[q] : a.invB[(long)comp * g.N + ii];
            if constexpr (MODE == PEN_QBQ_CG) dot += (float)(ib * cabs2(tile[q]));
            tile[q] = cscale(tile[q], ib * invN);
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
  }
  if constexpr (QBQ || MODE == PEN_QRS_IN) {
    for (int q = threadIdx.x; q < Ls * TW; q += kPencilThreads) {
      const int s = q / TW, f = q - s * TW;
      if (f < tw_n) a.T[fb + (long)s * P + m * Lf + f0 + f] = tile[q];
    }
  }
  if constexpr (MODE == PEN_QBQ_CG) {
    // <p, Ap> for A = Q_r^* B^-1 Q_r: Q_r^* is N times the adjoint of Q_r (unnormalised
    // forward DFT against the 1/N-scaled inverse), so <p, Ap> = N ||B^-1/2 Q_r p||^2 =
    // (1/N) sum_e |IDFT(Pi p)_e|^2 / eps_e, real and positive (CG.cu:57-63, with
    // Zdotc(p, Ap) formed in the field domain).  This CTA writes its partial sum; the
    // forward plane stage sums the slot's partials in order and forms a = ||r||^2 / <p, Ap>.
    double acc[1] = {(double)dot};
    __shared__ double sred[32];
    block_reduce<1>(acc, sred);
    if (threadIdx.x == 0) a.partials[(size_t)slot * a.pstride + blockIdx.y * gridDim.x + blockIdx.x] = acc[0];
  }
}

// Pipelined Q_r^* B^-1 Q_r pencil stage for the static 96^3 geometry (used in FP64,
// where it takes 26.5 instead of 28.5 us per k-point at batch 20).  Each CTA
// walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ... of all k-points in the
// launch and streams the next tile's field and 1/eps rows into its second buffer
// (16-byte cp.async, one copy group per tile) while it transforms the current one,
// so the memory phase of one tile runs under the transforms of the previous.
// grid = (resident CTAs), kPencilThreads threads.
// Tile t of a pipelined 96^3 pencil launch (t = ((slot * 3 * vec_per_slot + 3 * vec
// + comp) * 96 + m) * nft + fast block): its slot (returned), component, field base
// of that component and offset of its first element in every slow-axis plane.
template <typename R>
__device__ __forceinline__ int pencil_pipe_tile(const PencilArgs<R>& a, int t, long& fb, int& off, int& comp) {
  constexpr int TW = PencilTW<R>::v, nft = 96 / TW, per_vec = 96 * nft;
  const int per_slot = 3 * a.vec_per_slot * per_vec;
  const int slot = t / per_slot;
  const int r = t - slot * per_slot;
  const int y = r / per_vec, x = r - y * per_vec;
  comp = y % 3;
  const int vec = y / 3;
  const int m = x / nft, f0 = (x - m * nft) * TW;
  fb = (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * a.g.N;
  off = m * 96 + f0;
  return slot;
}
template <typename R> __device__ __forceinline__ bool pencil_pipe_live(const PencilArgs<R>& a, int t) {
  const int slot = t / (3 * a.vec_per_slot * 96 * (96 / PencilTW<R>::v));
  if (!a.slots[slot].active) return false;
  if (a.gate == 1 && !a.cg[slot].active) return false;
  if (a.gate == 2 && !a.cg[slot].outer_active) return false;
  return true;
}
// Starts the 16-byte copies of tile t's field rows and 1/eps rows into (tile, ibt).
template <typename R>
__device__ __forceinline__ void pencil_pipe_issue(const PencilArgs<R>& a, int t, int total, cplx<R>* tile, R* ibt) {
  constexpr int TW = PencilTW<R>::v, P = 96 * 96;
  constexpr int CH = 16 / sizeof(cplx<R>), CHB = 16 / sizeof(R);
  if (t >= total || !pencil_pipe_live(a, t)) return;
  long fb;
  int off, comp;
  pencil_pipe_tile<R>(a, t, fb, off, comp);
  const long ib = (long)comp * a.g.N;
  for (int q = threadIdx.x; q < 96 * (TW / CH); q += kPencilThreads) {
    const int s = q / (TW / CH), c = q - s * (TW / CH);
    cp_async16(tile + s * TW + c * CH, a.T + fb + (long)s * P + off + c * CH);
  }
  for (int q = threadIdx.x; q < 96 * (TW / CHB); q += kPencilThreads) {
    const int s = q / (TW / CHB), c = q - s * (TW / CHB);
    cp_async16(ibt + s * TW + c * CHB, a.invB + ib + (long)s * P + off + c * CHB);
  }
}

template <typename R>
__global__ void __launch_bounds__(kPencilThreads, sizeof(R) == 4 ? 3 : 2) k_pencil_pipe(PencilArgs<R> a) {
  FAME_COUNT_LAUNCH();
  using GP = Stat96;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  constexpr int TW = PencilTW<R>::v;
  constexpr int Lf = 96, Lm = 96, Ls = 96, P = Lf * Lm;
  constexpr int nft = Lf / TW;
  constexpr int TILE = Ls * TW;
  constexpr int CHB = 16 / sizeof(R);  // 1/eps values per 16-byte copy
  static_assert(Lf % TW == 0 && TW % CHB == 0, "whole tiles of whole 16-byte copies");
  cplx<R>* tiles = reinterpret_cast<cplx<R>*>(smem_raw);     // [2][TILE]
  R* ibts = reinterpret_cast<R*>(tiles + 2 * TILE);            // [2][TILE]
  cplx<R>* tws = reinterpret_cast<cplx<R>*>(ibts + 2 * TILE);  // [Ls]
  for (int i = threadIdx.x; i < Ls; i += kPencilThreads) tws[i] = a.tw[g.tws + i];
  const int total = a.nslots * 3 * a.vec_per_slot * Lm * nft;
  int t = blockIdx.x;
  pencil_pipe_issue<R>(a, t, total, tiles, ibts);
  cp_async_commit();
  for (int b = 0; t < total; b ^= 1, t += gridDim.x) {
    // buffer b ^ 1 was released at the end of the last iteration
    pencil_pipe_issue<R>(a, t + gridDim.x, total, tiles + (b ^ 1) * TILE, ibts + (b ^ 1) * TILE);
    cp_async_commit();
    cp_async_wait_group<1>();  // this tile's group has landed
    __syncthreads();
    if (pencil_pipe_live(a, t)) {  // uniform over the CTA
      cplx<R>* tile = tiles + b * TILE;
      // inverse, x B^{-1}/N, forward; one FFT call site for the register budget
      for (int dir = 0; dir < 2; dir++) {
        GP::template fft_slow<R, 0>(tile, g, tws, dir == 0);
        if (dir == 0) {
          const R invN = (R)(1.0 / g.N);
          const R* ibt = ibts + b * TILE;
          for (int q = threadIdx.x; q < TILE; q += kPencilThreads) tile[q] = cscale(tile[q], ibt[q] * invN);
          __syncthreads();
        }
      }
      long fb;
      int off, comp;
      pencil_pipe_tile<R>(a, t, fb, off, comp);
      for (int q = threadIdx.x; q < TILE; q += kPencilThreads) {
        const int s = q / TW, f = q - s * TW;
        a.T[fb + (long)s * P + off + f] = tile[q];
      }
    }
    __syncthreads();  // every thread is done with buffer b before it is refilled
  }
  cp_async_wait_group<0>();
}

// ------------------------------------------------------------------ plane stage (forward)

// End of a loop body in the forward plane stage: the last CTA of the grid decides
// whether the loop (EPI_RESID: outer refinement, EPI_CGR: CG) runs again.  Every CTA,
// live or not, arrives here once.
template <int EPI, typename R>
__device__ __forceinline__ void plane_fwd_decide(const PlaneOutArgs<R>& a) {
  if (grid_last(a.counters + a.nslots, gridDim.x * gridDim.y * gridDim.z)) {
    if (threadIdx.x == 0) {
      int any = 0;
      for (int q = 0; q < a.nslots; q++)
        any |= a.slots[q].active && (EPI == EPI_RESID ? a.cg[q].outer_active : a.cg[q].active);
      decide_cond(a.cond, any);
    }
  }
}

template <typename R, bool GEN, int EPI, bool PR, int RARE, class GP>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(GP::kMaxPlaneThreads, GP::template plane_min_blocks<R, RARE>())
    k_plane_fwd(PlaneOutArgs<R> a) {
  FAME_COUNT_LAUNCH();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  const int Lf = GP::Lf(g), Lm = GP::Lm(g), S = GP::S(g), P = GP::P(g);
  const Div dlf(Lf);  // row of plane element e: e / Lf (folds to a constant for static geometries)
  cplx<R>* plane = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* twf = plane + Lm * S;  // plane rows have the odd pitch S >= Lf
  cplx<R>* twm = twf + Lf;
  cplx<R>* lx = twm + Lm;
  cplx<R>* ly = lx + Lf;
  cg::cluster_group cl = cg::this_cluster();
  const int comp = (int)cl.block_rank();
  const int s = blockIdx.x / 3;
  const int vec = blockIdx.y;
  const int slot = blockIdx.z;
  const Slot sl = a.slots[slot];
  bool live = sl.active;
  if constexpr (EPI == EPI_CG || EPI == EPI_CGR) live = live && a.cg[slot].active;
  if constexpr (EPI == EPI_RESID) live = live && a.cg[slot].outer_active;
  if (!live) {
    if constexpr (EPI == EPI_RESID) plane_fwd_decide<EPI>(a);
    return;
  }
  if constexpr (EPI == EPI_CGR) {
    // this CTA's own residual, read in the epilogue: it streams into L2 during the transforms
    long i0, i1;
    if (a.self_pf && threadIdx.x < 2 && plane_vec_range(P, s, comp, sl, i0, i1))
      prefetch_l2(a.r + (long)(slot * a.vec_per_slot + vec) * a.vstride + (threadIdx.x ? sl.Nd : 0) + i0,
                  (i1 - i0) * sizeof(cplx<R>));
  }
  if constexpr (EPI == EPI_CGR) {
    // the field plane (4 pieces) and the residual of the CTA one wave ahead
    int x2, y2, z2;
    if (a.pf_dist > 0 && threadIdx.x < 6 && cta_of(cta_linear() + a.pf_dist, x2, y2, z2)) {
      const Slot s2 = a.slots[z2];
      if (s2.active && a.cg[z2].active) {
        const int s2p = x2 / 3, c2 = x2 % 3;
        if (threadIdx.x < 4) {
          const long piece = (P + 3) / 4;
          const long lo = threadIdx.x * piece, hi = min((long)P, lo + piece);
          prefetch_l2(a.T + (long)(z2 * a.vec_per_slot + y2) * a.fstride + (long)c2 * g.N + (long)s2p * P + lo,
                      (hi - lo) * sizeof(cplx<R>));
        } else {
          long i0, i1;
          if (plane_vec_range(P, s2p, c2, s2, i0, i1))
            prefetch_l2(a.r + (long)(z2 * a.vec_per_slot + y2) * a.vstride + ((threadIdx.x & 1) ? s2.Nd : 0) + i0,
                        (i1 - i0) * sizeof(cplx<R>));
        }
      }
    }
  }
  const double2* tab = a.tabs + (size_t)slot * g.tab_stride;
  for (int i = threadIdx.x; i < Lf; i += GP::plane_threads()) {
    twf[i] = a.tw[g.twf + i];
    if constexpr (!GEN) lx[i] = cvt<R>(tab[g.oLx + i]);
  }
  for (int i = threadIdx.x; i < Lm; i += GP::plane_threads()) {
    twm[i] = a.tw[g.twm + i];
    if constexpr (!GEN) ly[i] = cvt<R>(tab[g.oLy + i]);
  }
  const cplx<R> lz = GEN ? mk<R>(0, 0) : cvt<R>(tab[g.oLz + s]);
  const cplx<R>* T = a.T + (long)(slot * a.vec_per_slot + vec) * a.fstride + (long)comp * g.N + (long)s * P;
  for (int e = threadIdx.x; e < P; e += GP::plane_threads()) {
    const int m = GP::kStatic ? e / Lf : (int)dlf.q(e);
    cp_async_elem(plane + e + m * (S - Lf), T + e);
  }
  __shared__ R s_step;
  if constexpr (EPI == EPI_CGR) {
    // the CG step a = ||r||^2 / <p, Ap> from the pencil stage's partial sums of this
    // k-point, summed in order by one warp while the plane streams in (k_cg_decide forms
    // the same sum for the solution update and the CG state)
    if (threadIdx.x < 32) {
      const double pAp = warp_sum_partials(a.partials + (size_t)slot * a.pstride, a.pen_parts) / g.N;
      if (threadIdx.x == 0) s_step = (R)(pAp > 0 ? a.cg[slot].r1 / pAp : 0.0);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // forward 2-D transform.  General lattices (T*, FAME_FFT_CUDA.cu:128-150):
  // x conj(D_ky), y (mid) pass, x conj(D_kz), z (fast) pass.  Simple lattices:
  // fast then mid axis, no twiddles.
  if constexpr (GP::kStatic && !GEN) {
    GP::template fft_plane_c<R, true, false>(plane, twf);
    GP::template fft_plane_c<R, false, false>(plane, twm);
  }
  for (int ax = 0; !(GP::kStatic && !GEN) && ax < 2; ax++) {
    const bool fast = GEN ? ax == 1 : ax == 0;
    if constexpr (GEN) {
      for (int e = threadIdx.x; e < P; e += GP::plane_threads()) {
        const int m = GP::kStatic ? e / Lf : (int)dlf.q(e), f = e - m * Lf;
        const int q = m * S + f;
        plane[q] = cmul(plane[q], ax == 0 ? cvt<R>(cconj(tab[g.oDky + s * g.Ny + m]))
                                          : cconj(dkz_at<R>(g, tab, s, m, f)));
      }
      __syncthreads();
    }
    GP::template fft_plane<R, RARE>(plane, g, fast, fast ? twf : twm, false);
  }
  cl.sync();  // all three component planes transformed

  const cplx<R>* src[3] = {cl.map_shared_rank(plane, 0), cl.map_shared_rank(plane, 1),
                           cl.map_shared_rank(plane, 2)};
  const int per = (P + 2) / 3;
  const int e0 = comp * per, e1 = min(P, e0 + per);
  const int Nd = sl.Nd, off = sl.off;
  const long vb = (long)(slot * a.vec_per_slot + vec) * a.vstride;
  double acc[2] = {0.0, 0.0};
  // 3 -> 2 unmix and the epilogue.  The three components (remote shared memory) and
  // the vector operand of KB points per thread are read up front, so one latency of
  // each kind covers KB points.
  constexpr int KB = GP::kStatic ? 4 : 2;
  const int NT = GP::plane_threads();
  R are = 0, aim = 0;
  if constexpr (EPI == EPI_CGR) are = s_step;  // real: <p, Ap> > 0
  for (int eb = e0 + threadIdx.x; eb < e1; eb += KB * NT) {
    cplx<R> t[KB][3], va[KB], vb2[KB];
#pragma unroll
    for (int k = 0; k < KB; k++) {
      const int e = eb + k * NT;
      const int fi = s * P + e;
      if (e < e1 && fi >= off) {
        const long i = fi - off;
        const int m = GP::kStatic ? e / Lf : (int)dlf.q(e), q = m * S + (e - m * Lf);
#pragma unroll
        for (int c = 0; c < 3; c++) t[k][c] = src[c][q];
        if constexpr (EPI == EPI_CG) {
          va[k] = a.p[vb + i];
          vb2[k] = a.p[vb + Nd + i];
        } else if constexpr (EPI == EPI_RESID) {
          va[k] = a.b[vb + i];
          vb2[k] = a.b[vb + Nd + i];
        } else if constexpr (EPI == EPI_CGR) {
          va[k] = a.r[vb + i];
          vb2[k] = a.r[vb + Nd + i];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < KB; k++) {
      const int e = eb + k * NT;
      const int fi = s * P + e;
      if (e >= e1 || fi < off) continue;
      const long i = fi - off;
      const int m = GP::kStatic ? e / Lf : (int)dlf.q(e), f = e - m * Lf;
      cplx<R> Lx, Ly, Lz;
      lam_elem<R, GEN>(g, tab, lx, ly, lz, s, m, f, Lx, Ly, Lz);
      cplx<R> Pc[6];
      pi_from<R>(GEN, PR, Lx, Ly, Lz, Pc);
      const cplx<R> t0 = t[k][0], t1 = t[k][1], t2 = t[k][2];
      const cplx<R> o1 = cadd(cadd(cmulc(Pc[0], t0), cmulc(Pc[1], t1)), cmulc(Pc[2], t2));
      const cplx<R> o2 = cadd(cadd(cmulc(Pc[3], t0), cmulc(Pc[4], t1)), cmulc(Pc[5], t2));
      if constexpr (EPI == EPI_OUT) {
        a.out[vb + i] = o1;
        a.out[vb + Nd + i] = o2;
      } else if constexpr (EPI == EPI_CG) {
        a.out[vb + i] = o1;
        a.out[vb + Nd + i] = o2;
        const cplx<R> d = cadd(cmulc(va[k], o1), cmulc(vb2[k], o2));  // conj(p) Ap
        acc[0] += (double)d.x;
        acc[1] += (double)d.y;
      } else if constexpr (EPI == EPI_RESID) {
        const cplx<R> r1 = csub(va[k], o1), r2 = csub(vb2[k], o2);
        a.out[vb + i] = r1;
        a.out[vb + Nd + i] = r2;
        acc[0] += (double)(cabs2(r1) + cabs2(r2));
      } else {  // EPI_CGR: r -= a Ap and ||r||^2 (CG.cu:71-76); Ap is never stored
        cplx<R> r1 = va[k], r2 = vb2[k];
        if constexpr (sizeof(R) == 4) {  // real step size: packed pairs
          r1 = pfma(o1, -are, r1);
          r2 = pfma(o2, -are, r2);
        } else {
          r1.x -= are * o1.x - aim * o1.y;
          r1.y -= are * o1.y + aim * o1.x;
          r2.x -= are * o2.x - aim * o2.y;
          r2.y -= are * o2.y + aim * o2.x;
        }
        a.r[vb + i] = r1;
        a.r[vb + Nd + i] = r2;
        acc[0] += (double)(cabs2(r1) + cabs2(r2));
      }
    }
  }
  // This CTA is done reading the other CTAs' planes.  A relaxed arrival (no wait for
  // this CTA's global stores to drain); the matching wait below keeps every plane alive
  // until all three CTAs have read it.
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");

  if constexpr (EPI == EPI_CGR) {
    // this CTA's part of ||r||^2; k_cg_decide sums the slot's parts in order
    __shared__ double sred[32];
    double acc1[1] = {acc[0]};
    block_reduce<1>(acc1, sred);
    if (threadIdx.x == 0) a.partials[(size_t)slot * a.pstride + a.pen_parts + blockIdx.x] = acc1[0];
  }
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
          // a = r1 / dot  (CG.cu:60-63)
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
    if constexpr (EPI == EPI_RESID) plane_fwd_decide<EPI>(a);
  }
  asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");  // every CTA has read this plane
}

}  // namespace fame
