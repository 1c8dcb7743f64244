// Host orchestration and the C ABI (include/fame_b200.h).
//
// One context = one device, one grid and lattice, one set of edge permittivities.
// fame_solve_kpoints splits the k list into batches of `batch` k-points ("slots").
// A batch runs the reference's whole per-k solve (FAME_Main/FAME_Fast_Algorithms_
// Isotropic.cu:20-86: restarted Lanczos on A_r^{-1}, invAr by CG, Ritz vectors,
// eigenvector restoration, Gamma patch) for all its slots in lockstep: every kernel
// carries the slot in blockIdx.z and slots that finished skip their work.  The whole
// batch is recorded once as a CUDA graph with WHILE nodes for the CG, refinement and
// restart loops and replayed for every batch.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include <utility>

#include "../../include/fame_b200.h"
#include "geometry.h"
#include "op_kernels_decl.h"
#include "program.h"
#include "solver_kernels.cuh"

namespace fame {

unsigned long long launches_ops_f32_simple();
unsigned long long launches_ops_f32_general();
unsigned long long launches_ops_f64_simple();
unsigned long long launches_ops_f64_general();
unsigned long long launches_ops_f32_simple_rare();
unsigned long long launches_ops_f32_general_rare();
unsigned long long launches_ops_f64_simple_rare();
unsigned long long launches_ops_f64_general_rare();
unsigned long long launches_ops_f32_simple_prime();
unsigned long long launches_ops_f32_general_prime();
unsigned long long launches_ops_f64_simple_prime();
unsigned long long launches_ops_f64_general_prime();
unsigned long long launches_ops_stat96_f32();
unsigned long long launches_ops_stat96_f64();
unsigned long long launches_ops_slow_static();
unsigned long long launches_ops_plane_static();
unsigned long long launches_material_locate();
FAME_DEFINE_LAUNCH_GETTER(launches_solver)

static thread_local std::string g_err;
static void set_err(const std::string& s) { g_err = s; }
// error text of the entry points defined in other translation units
void set_last_error(const std::string& s) { g_err = s; }

// ------------------------------------------------------------------ device buffers
template <typename T> struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void ensure(size_t count) {
    if (count <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    FAME_CK(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

}  // namespace fame

using namespace fame;

struct fame_ctx {
  int device = 0;
  fame_lattice lat;
  Geom g;
  cudaStream_t stream = nullptr;
  int plane_threads = 512;    // threads of a runtime-geometry plane CTA
  int plane_threads32 = 512;  // the same for FP32 kernels
  template <typename R> int plane_nt() const { return sizeof(R) == 4 ? plane_threads32 : plane_threads; }
  int pipe_ctas64 = 0;  // resident k_pencil_pipe<double> CTAs on the device
  int prefetch = 0;     // L2 prefetch one wave ahead in the CG stage kernels (fame_set_option; measured slower)
  int self_prefetch = 1;  // CG plane stages: L2 prefetch of the CTA's own operands at its start
  int radix_order = 0;  // kRadixOrders index of the runtime-geometry axis plans
  int threads32_opt = 0, threads64_opt = 0;  // plane CTA sizes set by fame_set_option (0: rule)
  std::map<const void*, int> waves;  // resident CTAs of a stage kernel on the device
  int rare = 0;      // fft_lines level the plane axes need: 0 radix 2-8, 1 + 7/11/13, 2 + primes >= 17
  int rare_pen = 0;  // the same for the pencil (slow) axis
  int static_planes = 1;  // static plane plans where instantiated (option "static_planes")
  // An automatic batch of at least 4 k-points per lane is split into `lanes` contiguous
  // blocks solved concurrently, each by a lane context on its own stream and host
  // thread, so one block's FP64 refinement and Lanczos phases run under another's FP32
  // CG (option "lanes").  Lane 0 is this context; the others share its lattice, its
  // permittivity (copied device to device when eps_ver changes) and its options.
  int lanes = 2;
  int eps_ver = 0;
  std::vector<fame_ctx*> lane_ctx;
  std::vector<int> lane_eps_ver;
  bool stat96 = false;  // Simple lattice on a 96^3 grid: compile-time geometry kernels
  int loop_cap = 0;     // fame_set_loop_cap: bound on every device loop's trips (0: defaults)
  bool have_eps = false;
  // persistent data
  DBuf<double2> tw64;
  DBuf<float2> tw32;
  DBuf<double> invB64, B64;
  DBuf<float> invB32;
  // General lattices: 1/eps also in the field layout (x, y, z; z fastest) that the
  // pencil stage of Q_r^* B^-1 Q_r walks, so its loads are contiguous rows
  DBuf<double> invB64q;
  DBuf<float> invB32q;
  const double* ibq64() const { return g.general ? invB64q.p : invB64.p; }
  const float* ibq32() const { return g.general ? invB32q.p : invB32.p; }
  // per-batch workspace
  int cap_slots = 0, cap_nstep = 0, cap_nwant = 0;
  long part_stride = 0;  // doubles of `partials` per slot
  bool cap_mixed = false, cap_vec = false;
  DBuf<Slot> slots;
  DBuf<double2> tabs;
  DBuf<CgState> cg;
  DBuf<LzState> lz;
  DBuf<double> partials, T0, T1, hcoef, theta, Z, G, stats;
  DBuf<unsigned> counters, tri_ctr;
  DBuf<int> map, prof, status, flags;
  DBuf<double2> U, r64, x64, b64, p64, Ap64, T64, EV, AV, Tb, E;
  DBuf<float2> r32, x32, p32, T32;
  int* hflag = nullptr;  // pinned
  // eigenvectors kept on the device by the last solve (evec_out NULL): its k-points,
  // whether each is the Gamma point (Gamma keeps nwant - 2 restored bands), nwant
  int dev_vec_nk = 0, dev_vec_nwant = 0;
  std::vector<int> dev_vec_gamma;
  DBuf<double> adj;  // fame_adjoint_vjp: [nwant] w, [nwant] grad_w, [nwant] denominators
  DBuf<double> bpart;     // per-band partial sums of the solve's split reductions (kBandSplit per band)
  DBuf<double> adj_part;  // the same for the adjoint entry points (never read by a recorded solve)
  DBuf<int> eps_bad;  // fame_set_eps_device: [0] bad count, [1] first bad edge
  // recorded programs keyed by configuration
  std::map<std::string, std::unique_ptr<Program>> progs;
};

namespace fame {

static int vec_blocks(const fame_ctx* c, int nslots) {
  const long n = 2L * c->g.N;
  long b = (n + 2047) / 2048;
  const long cap = std::max<long>(1, 1184 / std::max(1, nslots));
  return (int)std::max<long>(1, std::min(b, cap));
}

template <typename R> static size_t plane_smem(const Geom& g) { return plane_smem_bytes<R>(g.Lf, g.Lm, g.S); }
template <typename R> static int pencil_tw() { return PencilTW<R>::v; }
template <typename R> static size_t pencil_smem(const Geom& g) { return pencil_smem_bytes<R>(g.Ls); }

template <typename K> static void allow_smem(K* k, size_t bytes) {
  if (bytes > 48 * 1024) FAME_CK(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// CTAs of a stage kernel resident on the whole device at once (one wave): clusters of
// three CTAs for the plane kernels (cluster = 3), single CTAs for the pencil kernels.
// Cached per kernel in the context; 0 if the occupancy query fails.
template <typename K> static int wave_ctas(fame_ctx* c, K* k, int threads, size_t smem, int cluster) {
  auto it = c->waves.find((const void*)k);
  if (it != c->waves.end()) return it->second;
  int n = 0, dev = 0, sms = 0;
  if (cluster > 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster * 64, 1, 1);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, (const void*)k, &cfg) == cudaSuccess) n = ncl * cluster;
  } else {
    int per = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ==
                                                   cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, threads, smem) == cudaSuccess)
      n = per * sms;
  }
  cudaGetLastError();  // a failed query only disables the prefetch
  c->waves[(const void*)k] = n;
  return n;
}

// CTAs of kernel k (kPencilThreads threads, `smem` dynamic shared bytes) resident on
// the whole current device at once
template <typename K> static int resident_ctas(K* k, size_t smem) {
  allow_smem(k, smem);
  int dev = 0, sms = 0, per = 0;
  FAME_CK(cudaGetDevice(&dev));
  FAME_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  FAME_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, kPencilThreads, smem));
  return std::max(1, per) * sms;
}

// Device ints of the context (c->flags): the condition flag of loop i at flags[i], its
// trip counter and overflow marker at flags[kTrips + 2i], and a kernel fault marker
// (a bounded wait that ran out) at flags[kFaultFlag].
// CTAs per band of the split per-band reductions (band statistics, norms, adjoint)
constexpr int kBandSplit = 64;
constexpr int kLoopCG = 0, kLoopOuter = 1, kLoopInner = 2, kLoopRestart = 4, kFaultFlag = 30, kTrips = 32;

struct Ops {
  fame_ctx* c;
  Program& P;
  int nslots;

  const Geom& g() const { return c->g; }

  VecArgs va(Cond cond) const {
    VecArgs v;
    v.g = c->g;
    v.slots = c->slots.p;
    v.tabs = c->tabs.p;
    v.vstride = 2L * c->g.N;
    v.cg = c->cg.p;
    v.partials = c->partials.p;
    v.counters = c->counters.p;
    v.cond = cond;
    v.nslots = nslots;
    return v;
  }

  template <typename R> const cplx<R>* tw() const;

  // static plane plans (ops_plane_static.cu) for the runtime-geometry grids they cover:
  // 1 FCC 64x55x52, 2 BCC 48x45x39, 3 hexagonal 128x107x92, 0 none (or switched off)
  int plane_plan() const {
    const Geom& q = g();
    if (!q.general || !c->static_planes) return 0;
    if (q.Lf == 52 && q.Lm == 55) return 1;
    if (q.Lf == 39 && q.Lm == 45) return 2;
    if (q.Lf == 92 && q.Lm == 107) return 3;
    return 0;
  }

  // partial sums per slot of the fused FP32 CG kernels: the pencil stage's <p, Ap>
  // (one per CTA of a slot), then the forward plane stage's ||r||^2
  int cg_pen_parts() const { return 3 * g().Lm * ((g().Lf + pencil_tw<float>() - 1) / pencil_tw<float>()); }
  int cg_fwd_parts() const { return 3 * g().Ls; }

  // end of a fused FP32 CG iteration: step size, r1, beta, counters, loop decision
  void cg_decide(Cond cond) {
    CgDecideArgs d;
    d.slots = c->slots.p;
    d.cg = c->cg.p;
    d.partials = c->partials.p;
    d.pstride = c->part_stride;
    d.pen_parts = cg_pen_parts();
    d.fwd_parts = cg_fwd_parts();
    d.N = g().N;
    d.counters = c->counters.p;
    d.cond = cond;
    d.nslots = nslots;
    P.launch(k_cg_decide, dim3(nslots), dim3(32), 0, d);
  }

  // plane inverse stage
  template <typename R, int IN, bool PR>
  void plane_inv(const cplx<R>* in, cplx<R>* T, int nvec, long vstride, long fstride, int sigma,
                 cplx<R>* p = nullptr, const cplx<R>* r = nullptr, double2* y64 = nullptr,
                 const float2* x32 = nullptr, Cond reset = Cond{}, cplx<R>* x = nullptr,
                 const float2* p32 = nullptr) {
    PlaneInArgs<R> a;
    a.reset = reset;
    a.g = g();
    a.slots = c->slots.p;
    a.tabs = c->tabs.p;
    a.tw = tw<R>();
    a.vstride = vstride;
    a.fstride = fstride;
    a.vec_per_slot = nvec;
    a.in = in;
    a.p = p;
    a.r = r;
    a.cg = c->cg.p;
    a.y64 = y64;
    a.x32 = x32;
    a.x = x;
    a.p32 = p32;
    a.sigma = sigma;
    a.T = T;
    a.fault = c->flags.p ? c->flags.p + kFaultFlag : nullptr;
    const size_t sm = plane_smem<R>(g());
    dim3 grid(3 * g().Ls, nvec, nslots);
    if (g().general) {
      auto k = c->rare == 2   ? k_plane_inv<R, true, IN, PR, 2, DynGeom>
               : c->rare == 1 ? k_plane_inv<R, true, IN, PR, 1, DynGeom>
                              : k_plane_inv<R, true, IN, PR, 0, DynGeom>;
      int nt = c->template plane_nt<R>();
      if constexpr (kPlanInv<R, IN, PR>) {
        const int pp = plane_plan();
        if (pp == 1) k = k_plane_inv<R, true, IN, PR, 0, PlaneFcc64>, nt = PlaneFcc64::kMaxPlaneThreads;
        if (pp == 2) k = k_plane_inv<R, true, IN, PR, 0, PlaneBcc48>, nt = PlaneBcc48::kMaxPlaneThreads;
        if (pp == 3) {
          if constexpr (sizeof(R) == 4)
            k = k_plane_inv<R, true, IN, PR, 0, PlaneHex128f>, nt = PlaneHex128f::kMaxPlaneThreads;
          else
            k = k_plane_inv<R, true, IN, PR, 0, PlaneHex128d>, nt = PlaneHex128d::kMaxPlaneThreads;
        }
      }
      allow_smem(k, sm);
      a.pf_dist = IN == IN_CG && c->prefetch ? wave_ctas(c, k, nt, sm, 3) : 0;
      a.self_pf = c->self_prefetch;
      P.launch(k, grid, dim3(nt), sm, a);
    } else {
      auto k = c->rare == 2   ? k_plane_inv<R, false, IN, PR, 2, DynGeom>
               : c->rare == 1 ? k_plane_inv<R, false, IN, PR, 1, DynGeom>
                              : k_plane_inv<R, false, IN, PR, 0, DynGeom>;
      int nt = c->template plane_nt<R>();
      if constexpr (kStatInv<R, IN, PR>)
        if (c->stat96) {
          k = k_plane_inv<R, false, IN, PR, 0, Stat96>;
          nt = kStatPlaneThreads;
        }
      allow_smem(k, sm);
      a.pf_dist = IN == IN_CG && c->prefetch ? wave_ctas(c, k, nt, sm, 3) : 0;
      a.self_pf = c->self_prefetch;
      P.launch(k, grid, dim3(nt), sm, a);
    }
  }

  template <typename R, int MODE>
  void pencil(cplx<R>* T, int nvec, long fstride, const R* invB, int gate, cplx<R>* out = nullptr,
              const cplx<R>* in = nullptr) {
    PencilArgs<R> a;
    a.g = g();
    a.slots = c->slots.p;
    a.tabs = c->tabs.p;
    a.tw = tw<R>();
    a.fstride = fstride;
    a.vec_per_slot = nvec;
    a.T = T;
    a.invB = invB;
    a.ib_field = MODE == PEN_QBQ || MODE == PEN_QBQ_CG ? 1 : 0;
    a.out = out;
    a.in = in;
    a.cg = c->cg.p;
    a.gate = gate;
    a.partials = c->partials.p;
    a.counters = c->counters.p;
    a.pstride = c->part_stride;
    a.TW = pencil_tw<R>();
    a.nslots = nslots;
    const size_t sm = pencil_smem<R>(g());
    const int nft = (g().Lf + a.TW - 1) / a.TW;
    dim3 grid(g().Lm * nft, 3 * nvec, nslots);
    a.pf_dist = 0;
    if (g().general) {
      auto k = c->rare_pen == 2   ? k_pencil<R, true, MODE, 2, DynGeom>
               : c->rare_pen == 1 ? k_pencil<R, true, MODE, 1, DynGeom>
                              : k_pencil<R, true, MODE, 0, DynGeom>;
      if constexpr (!(sizeof(R) == 8 && MODE == PEN_QBQ_CG))
        if (c->rare_pen == 0) {  // static slow-axis plans (ops_slow_static.cu)
          if (g().Ls == 48) k = k_pencil<R, true, MODE, 0, DynGeomSlow<48>>;
          if (g().Ls == 64) k = k_pencil<R, true, MODE, 0, DynGeomSlow<64>>;
          if (g().Ls == 128) k = k_pencil<R, true, MODE, 0, DynGeomSlow<128>>;
        }
      allow_smem(k, sm);
      if (MODE == PEN_QBQ_CG && c->prefetch) a.pf_dist = wave_ctas(c, k, kPencilThreads, sm, 1);
      P.launch(k, grid, dim3(kPencilThreads), sm, a);
    } else {
      auto k = c->rare_pen == 2   ? k_pencil<R, false, MODE, 2, DynGeom>
               : c->rare_pen == 1 ? k_pencil<R, false, MODE, 1, DynGeom>
                              : k_pencil<R, false, MODE, 0, DynGeom>;
      if constexpr (kStatPen<R, MODE> && sizeof(R) == 4)
        if (c->stat96) k = k_pencil<R, false, MODE, 0, Stat96>;
      if constexpr (kStatPen<R, MODE> && sizeof(R) == 8)
        if (c->stat96) {
          // FP64: pipelined, as many CTAs as are resident, each walking tiles (the FP32
          // stage measured no faster this way: 13.5 against 13.1 us per k-point)
          auto kp = k_pencil_pipe<R>;
          const size_t smp = pencil_pipe_smem_bytes<R>(g().Ls);
          allow_smem(kp, smp);
          const int total = (int)(grid.x * grid.y * grid.z);
          P.launch(kp, dim3(std::min(total, c->pipe_ctas64)), dim3(kPencilThreads), smp, a);
          return;
        }
      allow_smem(k, sm);
      if (MODE == PEN_QBQ_CG && c->prefetch) a.pf_dist = wave_ctas(c, k, kPencilThreads, sm, 1);
      P.launch(k, grid, dim3(kPencilThreads), sm, a);
    }
  }

  template <typename R, int EPI, bool PR>
  void plane_fwd(const cplx<R>* T, cplx<R>* out, int nvec, long vstride, long fstride,
                 const cplx<R>* p = nullptr, const cplx<R>* b = nullptr, Cond cond = Cond{},
                 double tol2 = 0, cplx<R>* r = nullptr) {
    PlaneOutArgs<R> a;
    a.r = r;
    a.g = g();
    a.slots = c->slots.p;
    a.tabs = c->tabs.p;
    a.tw = tw<R>();
    a.vstride = vstride;
    a.fstride = fstride;
    a.vec_per_slot = nvec;
    a.T = T;
    a.out = out;
    a.p = p;
    a.b = b;
    a.cg = c->cg.p;
    a.partials = c->partials.p;
    a.counters = c->counters.p;
    a.cond = cond;
    a.nslots = nslots;
    a.tol2 = tol2;
    a.pstride = c->part_stride;
    a.pen_parts = cg_pen_parts();
    const size_t sm = plane_smem<R>(g());
    dim3 grid(3 * g().Ls, nvec, nslots);
    if (g().general) {
      auto k = c->rare == 2   ? k_plane_fwd<R, true, EPI, PR, 2, DynGeom>
               : c->rare == 1 ? k_plane_fwd<R, true, EPI, PR, 1, DynGeom>
                              : k_plane_fwd<R, true, EPI, PR, 0, DynGeom>;
      int nt = c->template plane_nt<R>();
      if constexpr (kPlanFwd<R, EPI, PR>) {
        const int pp = plane_plan();
        if (pp == 1) k = k_plane_fwd<R, true, EPI, PR, 0, PlaneFcc64>, nt = PlaneFcc64::kMaxPlaneThreads;
        if (pp == 2) k = k_plane_fwd<R, true, EPI, PR, 0, PlaneBcc48>, nt = PlaneBcc48::kMaxPlaneThreads;
        if (pp == 3) {
          if constexpr (sizeof(R) == 4)
            k = k_plane_fwd<R, true, EPI, PR, 0, PlaneHex128f>, nt = PlaneHex128f::kMaxPlaneThreads;
          else
            k = k_plane_fwd<R, true, EPI, PR, 0, PlaneHex128d>, nt = PlaneHex128d::kMaxPlaneThreads;
        }
      }
      allow_smem(k, sm);
      a.pf_dist = EPI == EPI_CGR && c->prefetch ? wave_ctas(c, k, nt, sm, 3) : 0;
      a.self_pf = c->self_prefetch;
      P.launch(k, grid, dim3(nt), sm, a);
    } else {
      auto k = c->rare == 2   ? k_plane_fwd<R, false, EPI, PR, 2, DynGeom>
               : c->rare == 1 ? k_plane_fwd<R, false, EPI, PR, 1, DynGeom>
                              : k_plane_fwd<R, false, EPI, PR, 0, DynGeom>;
      int nt = c->template plane_nt<R>();
      if constexpr (kStatFwd<R, EPI, PR>)
        if (c->stat96) {
          k = k_plane_fwd<R, false, EPI, PR, 0, Stat96>;
          nt = kStatPlaneThreads;
        }
      allow_smem(k, sm);
      a.pf_dist = EPI == EPI_CGR && c->prefetch ? wave_ctas(c, k, nt, sm, 3) : 0;
      a.self_pf = c->self_prefetch;
      P.launch(k, grid, dim3(nt), sm, a);
    }
  }
};
template <> const double2* Ops::tw<double>() const { return c->tw64.p; }
template <> const float2* Ops::tw<float>() const { return c->tw32.p; }

// ------------------------------------------------------------------ geometry
static int setup_geom(fame_ctx* c) {
  Geom& g = c->g;
  std::string err;
  for (int i = 0; i < 3; i++)
    if (!(c->lat.mesh_len[i] > 0.0) || !std::isfinite(c->lat.mesh_len[i])) {
      set_err("mesh lengths must be finite and positive");
      return FAME_ERR_BAD_INPUT;
    }
  bool finite = true;
  for (double v : c->lat.lattice_vec_a) finite = finite && std::isfinite(v);
  for (double v : c->lat.t1) finite = finite && std::isfinite(v);
  if (!finite) {
    set_err("lattice vectors and shifts must be finite");
    return FAME_ERR_BAD_INPUT;
  }
  const int rc = layout_geom(c->lat, g, 1L << 28, err);
  if (rc != FAME_OK) {
    set_err(err);
    return rc;
  }
  c->rare = plane_level(g);
  c->rare_pen = pencil_level(g);
  c->plane_threads32 = plane_threads_rule<float>(g, c->rare);
  c->plane_threads = plane_threads_rule<double>(g, c->rare);
  c->stat96 = !g.general && g.Nx == 96 && g.Ny == 96 && g.Nz == 96;
  if (c->stat96) c->pipe_ctas64 = resident_ctas(k_pencil_pipe<double>, pencil_pipe_smem_bytes<double>(g.Ls));
  // twiddles e^{-2 pi i m / n} for the fast, mid and slow axes
  std::vector<double2> tw;
  for (int n : {g.Lf, g.Lm, g.Ls})  // at g.twf, g.twm, g.tws
    for (int m = 0; m < n; m++) tw.push_back(make_double2(cos(2.0 * M_PI * m / n), -sin(2.0 * M_PI * m / n)));
  std::vector<float2> tw32(tw.size());
  for (size_t i = 0; i < tw.size(); i++) tw32[i] = make_float2((float)tw[i].x, (float)tw[i].y);
  c->tw64.ensure(tw.size());
  c->tw32.ensure(tw.size());
  FAME_CK(cudaMemcpy(c->tw64.p, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));
  FAME_CK(cudaMemcpy(c->tw32.p, tw32.data(), tw32.size() * sizeof(float2), cudaMemcpyHostToDevice));
  return FAME_OK;
}

static void ensure_workspace(fame_ctx* c, int nslots, int nstep, int nwant, bool mixed, bool vec) {
  if (nslots <= c->cap_slots && nstep <= c->cap_nstep && nwant <= c->cap_nwant &&
      (!mixed || c->cap_mixed) && (!vec || c->cap_vec))
    return;
  const Geom& g = c->g;
  const size_t N = g.N, M = 2 * N;
  nslots = std::max(nslots, c->cap_slots);
  nstep = std::max(nstep, c->cap_nstep);
  nwant = std::max(nwant, c->cap_nwant);
  mixed = mixed || c->cap_mixed;
  vec = vec || c->cap_vec;
  c->progs.clear();
  c->slots.ensure(nslots);
  c->tabs.ensure((size_t)nslots * g.tab_stride);
  c->cg.ensure(nslots);
  c->lz.ensure(nslots);
  const size_t lzblk = (M + kLzRows - 1) / kLzRows;
  const size_t part = std::max({lzblk * (2 * 64 + 1), (size_t)3 * g.Ls * 2 * 16, (size_t)1184 * 4,
                                 (size_t)3 * g.Lm * g.Lf + 3 * g.Ls});
  c->partials.ensure((size_t)nslots * part);
  c->part_stride = (long)part;
  c->counters.ensure(nslots + 1);
  FAME_CK(cudaMemset(c->counters.p, 0, (nslots + 1) * sizeof(unsigned)));
  c->tri_ctr.ensure(1);
  FAME_CK(cudaMemset(c->tri_ctr.p, 0, sizeof(unsigned)));
  c->T0.ensure((size_t)nslots * nstep);
  c->T1.ensure((size_t)nslots * nstep);
  c->hcoef.ensure((size_t)nslots * 2 * (nstep + 2));
  c->theta.ensure((size_t)nslots * nstep);
  c->Z.ensure((size_t)nslots * nstep * nstep);
  c->G.ensure((size_t)nslots * (nstep + 1) * (nwant + 1));
  c->stats.ensure((size_t)nslots * nwant * 8);
  c->map.ensure((size_t)nslots * (nstep + 1) + (size_t)nslots * (nwant + 1));
  c->prof.ensure((size_t)nslots * 3);
  c->status.ensure(nslots);
  c->flags.ensure(64);
  const int nphys = nstep + 1 + nwant + 1;
  c->U.ensure((size_t)nslots * nphys * M);
  c->r64.ensure((size_t)nslots * M);
  c->x64.ensure((size_t)nslots * M);
  c->T64.ensure((size_t)nslots * 3 * N);
  c->EV.ensure((size_t)nslots * nwant * M);
  c->AV.ensure((size_t)nslots * nwant * M);
  c->Tb.ensure((size_t)nslots * nwant * 3 * N);
  if (mixed) {
    c->b64.ensure((size_t)nslots * M);
    c->r32.ensure((size_t)nslots * M);
    c->x32.ensure((size_t)nslots * M);
    c->p32.ensure((size_t)nslots * M);
    c->T32.ensure((size_t)nslots * 3 * N);
  }
  // FP64 CG vectors: every context may run FP64 solves and A_r^-1 applies, whatever
  // precision it started with, so they grow with the slot count in both modes
  c->p64.ensure((size_t)nslots * M);
  c->Ap64.ensure((size_t)nslots * M);
  if (vec) c->E.ensure((size_t)nslots * nwant * 3 * N);
  c->bpart.ensure((size_t)nslots * nwant * kBandSplit * 4);
  c->cap_slots = nslots;
  c->cap_nstep = nstep;
  c->cap_nwant = nwant;
  c->cap_mixed = mixed;
  c->cap_vec = vec;
}

// ------------------------------------------------------------------ statistics kernels
// Per-band sums over a reduced or field vector split over kBandSplit CTAs per band: each CTA
// writes its partial sums, and one warp per band adds them in a fixed order
// (k_rows_sum), so the sums are deterministic and every band's work spreads over the SMs.

// [nrows][nsplit][nq] partials -> [nrows][nq] sums, one warp per row (blockIdx.x band,
// blockIdx.y slot; row = slot * nband + band).  slots == nullptr: every row is live.
__global__ void __launch_bounds__(32) k_rows_sum(const Slot* slots, int nband, const double* part, int nsplit,
                                                 int nq, double* out) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.x, slot = blockIdx.y;
  if (slots && !slots[slot].active) return;
  const size_t row = (size_t)slot * nband + band;
  for (int q = 0; q < nq; q++) {
    const double v = warp_sum_strided(part + row * nsplit * nq + q, nsplit, nq);
    if (threadIdx.x == 0) out[row * nq + q] = v;
  }
}

// Per (slot, band): y = Ritz vector, v = QBQ(Sigma y).  Partial sums of
// ||Sigma (Sigma v - lambda y)||^2, ||Sigma y||^2, Re<Sigma y, v>, ||y||^2 over this
// CTA's chunk of the 2 Nd entries (k_rows_sum adds them).
__global__ void __launch_bounds__(256) k_band_stats(VecArgs va, const double2* EV, const double2* AV,
                                                    long vstride, int nwant, const double* theta,
                                                    int nstep, double* part) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.y, slot = blockIdx.z;
  const Slot sl = va.slots[slot];
  if (!sl.active) return;
  const double lam = 1.0 / theta[slot * nstep + band];
  const double2* tab = va.tabs + (size_t)slot * va.g.tab_stride;
  const long base = (long)(slot * nwant + band) * vstride;
  const int n = 2 * sl.Nd;
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  double acc[4] = {0, 0, 0, 0};
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const double s = lq_sqrt_at(va.g, tab, full_index(i, sl.Nd, sl.off));
    const double2 y = EV[base + i], v = AV[base + i];
    const double rx = s * (s * v.x - lam * y.x), ry = s * (s * v.y - lam * y.y);
    acc[0] += rx * rx + ry * ry;
    acc[1] += s * s * (y.x * y.x + y.y * y.y);
    acc[2] += s * (y.x * v.x + y.y * v.y);
    acc[3] += y.x * y.x + y.y * y.y;
  }
  __shared__ double sred[4 * 32];
  block_reduce<4>(acc, sred);
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; q++) part[(((size_t)slot * nwant + band) * gridDim.x + blockIdx.x) * 4 + q] = acc[q];
}

// Partial sums of ||E||^2 per (slot, band) over this CTA's chunk of the 3N entries.
__global__ void __launch_bounds__(256) k_band_norm_part(const Slot* slots, const double2* E, long fstride,
                                                        int nwant, long n3, double* part) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.y, slot = blockIdx.z;
  if (!slots[slot].active) return;
  const double2* e = E + (long)(slot * nwant + band) * fstride;
  const long chunk = (n3 + gridDim.x - 1) / gridDim.x;
  const long i0 = blockIdx.x * chunk, i1 = min(n3, i0 + chunk);
  double acc[1] = {0.0};
  for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) acc[0] += cabs2(e[i]);
  __shared__ double sred[32];
  block_reduce<1>(acc, sred);
  if (threadIdx.x == 0) part[((size_t)slot * nwant + band) * gridDim.x + blockIdx.x] = acc[0];
}

// The reference's scaling E *= ||E|| (FAME_Fast_Algorithms_Isotropic.cu:119-121): every
// CTA forms ||E|| from the nsplit partials in the same order, then scales its chunk.
__global__ void __launch_bounds__(256) k_band_scale(const Slot* slots, double2* E, long fstride, int nwant,
                                                    long n3, const double* part, int nsplit, double* norms) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.y, slot = blockIdx.z;
  if (!slots[slot].active) return;
  const size_t row = (size_t)slot * nwant + band;
  __shared__ double nrm;
  if (threadIdx.x < 32) {
    const double v = sqrt(warp_sum_strided(part + row * nsplit, nsplit, 1));
    if (threadIdx.x == 0) {
      nrm = v;
      if (blockIdx.x == 0) norms[row] = v;
    }
  }
  __syncthreads();
  const double s = nrm;
  double2* e = E + (long)row * fstride;
  const long chunk = (n3 + gridDim.x - 1) / gridDim.x;
  const long i0 = blockIdx.x * chunk, i1 = min(n3, i0 + chunk);
  for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) e[i] = cscale(e[i], s);
}

// ------------------------------------------------------------------ adjoint
// Hellmann-Feynman for C^H C E = w^2 B E with diagonal B: d(w^2)/dB_e =
// -w^2 |E_e|^2 / (E^H B E), so dw/dB_e = -(w/2) |E_e|^2 / (E^H B E).  With one
// permittivity per voxel (B_x = B_y = B_z = eps) the voxel gradient sums its three
// edges.  Bands with w = 0 (Gamma patch) get zero gradient.
// Partial sums of E^H B E per band (blockIdx.y) over this CTA's chunk of the 3N edges;
// k_rows_sum adds the gridDim.x partials of a band in order.
__global__ void __launch_bounds__(256) k_adj_den(const double2* E, const double* B, long n3, double* part) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.y;
  const double2* e = E + (long)band * n3;
  const long chunk = (n3 + gridDim.x - 1) / gridDim.x;
  const long i0 = blockIdx.x * chunk, i1 = min(n3, i0 + chunk);
  double acc[1] = {0.0};
  for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) acc[0] += B[i] * cabs2(e[i]);
  __shared__ double sred[32];
  block_reduce<1>(acc, sred);
  if (threadIdx.x == 0) part[(size_t)band * gridDim.x + blockIdx.x] = acc[0];
}

__global__ void __launch_bounds__(256) k_adj_grad(const double2* E, const double* w, const double* den, long N,
                                                  double* grad) {
  FAME_COUNT_LAUNCH();
  const int band = blockIdx.y;
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  const double2* e = E + (long)band * 3 * N;
  const double s = cabs2(e[v]) + cabs2(e[N + v]) + cabs2(e[2 * N + v]);
  grad[(long)band * N + v] = w[band] > 0 ? -0.5 * w[band] * s / den[band] : 0.0;
}

// Sum over bands of c_i |E_i|^2 on the three edges of voxel v, with
// c_i = -(w_i / 2) g_i / (E_i^H B E_i) (zero for w_i = 0): the vector-Jacobian
// product sum_i g_i dw_i/deps_v.  E holds nvec bands from band `first` (the Gamma
// point keeps the two patched zero bands off the device).
__global__ void __launch_bounds__(256) k_adj_vjp(const double2* E, const double* wgd, int nwant, int first,
                                                 long N, double* grad) {
  FAME_COUNT_LAUNCH();
  __shared__ double coef[64];
  if (threadIdx.x < nwant) {
    const int i = threadIdx.x;
    const double w = wgd[i], g = wgd[nwant + i];
    coef[i] = (i >= first && w > 0) ? -0.5 * w * g / wgd[2 * nwant + i - first] : 0.0;
  }
  __syncthreads();
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  double acc = 0.0;
  for (int i = first; i < nwant; i++) {
    const double2* e = E + (long)(i - first) * 3 * N;
    acc += coef[i] * (cabs2(e[v]) + cabs2(e[N + v]) + cabs2(e[2 * N + v]));
  }
  grad[v] = acc;
}

// Edge permittivities from device memory: count and locate entries that are not
// finite and positive (pass 0), then write B, 1/B in FP64 and FP32 and, for General
// lattices, 1/B in the field layout (x, y, z; z fastest) of the pencil stage (pass 1).
__global__ void __launch_bounds__(256) k_eps_device(Geom g, const double* B, int pass, int* bad, double* B64,
                                                    double* ib64, float* ib32, double* ib64q, float* ib32q) {
  FAME_COUNT_LAUNCH();
  const long n3 = 3L * g.N;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n3; e += (long)gridDim.x * blockDim.x) {
    const double b = B[e];
    if (pass == 0) {
      if (!(b > 0.0) || !isfinite(b)) {
        atomicAdd(bad, 1);
        atomicMin(bad + 1, (int)e);
      }
      continue;
    }
    const double ib = 1.0 / b;
    B64[e] = b;
    ib64[e] = ib;
    ib32[e] = (float)ib;
    if (g.general) {
      const long comp = e / g.N, r = e - comp * g.N;
      const long x = r % g.Nx, y = (r / g.Nx) % g.Ny, z = r / ((long)g.Nx * g.Ny);
      const long q = comp * g.N + (x * g.Ny + y) * g.Nz + z;
      ib64q[q] = ib;
      ib32q[q] = (float)ib;
    }
  }
}

// ------------------------------------------------------------------ recording
struct SolveCfg {
  int nslots, nstep, nwant, es_maxit, ls_maxit, mixed, vec, inner_maxit;
  int enorm;     // restore E (norms only) for the reference-scaled residual
  int loop_cap;  // bound on every device loop's trips (0: the defaults)
  double es_tol, ls_tol, inner_tol;
};

static std::string cfg_key(const SolveCfg& s, bool graph) {
  char b[256];
  snprintf(b, sizeof b, "%d/%d/%d/%d/%d/%d/%d/%d/%d/%.17g/%.17g/%.17g/%d/%d", s.nslots, s.nstep, s.nwant,
           s.es_maxit, s.ls_maxit, s.mixed, s.vec, s.enorm, s.inner_maxit, s.es_tol, s.ls_tol, s.inner_tol,
           (int)graph, s.loop_cap);
  return b;
}

// invAr (FAME_Main/FAME_Matrix_Vector_Production_Isotropic_invAr.cu:8-48) for the
// Lanczos vector u_j of every live slot, leaving w in U[:, j+1]; then one Lanczos step.
static Cond loop_cond(Program& P, int* flags, int id, int cap, int loop_cap = 0) {
  return P.make_cond(flags + id, flags + kTrips + 2 * id, loop_cap > 0 ? std::min(cap, loop_cap) : cap);
}

static void emit_step(Ops& o, const SolveCfg& s, LzArgs L, int j, int* flag_base) {
  fame_ctx* c = o.c;
  Program& P = o.P;
  const Geom& g = c->g;
  const int nvb = vec_blocks(c, s.nslots);
  const long M = 2L * g.N;
  const long F = 3L * g.N;
  const double tol2 = s.ls_tol * s.ls_tol;
  if (!s.mixed) {
    Cond cc = loop_cond(P, flag_base, kLoopCG, s.ls_maxit + 2, s.loop_cap);
    P.launch(k_invar_pro<false>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(cc), L, j, c->r64.p, c->x64.p,
             (double2*)nullptr, tol2, s.ls_maxit);
    P.while_loop(cc, [&] {
      o.plane_inv<double, IN_CG, false>(nullptr, c->T64.p, 1, M, F, 0, c->p64.p, c->r64.p, nullptr, nullptr, cc,
                                        c->x64.p);
      o.pencil<double, PEN_QBQ>(c->T64.p, 1, F, c->ibq64(), 1);
      o.plane_fwd<double, EPI_CG, false>(c->T64.p, c->Ap64.p, 1, M, F, c->p64.p);
      P.launch(k_cg_update<double>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(cc), c->r64.p,
               (const double2*)c->Ap64.p);
    });
    P.launch(k_invar_epi<false>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L, j,
             (const double2*)c->x64.p, (const double2*)c->p64.p);
  } else {
    Cond outer = loop_cond(P, flag_base, kLoopOuter, 42, s.loop_cap);
    Cond inner = loop_cond(P, flag_base, kLoopInner, s.inner_maxit + 2, s.loop_cap);
    P.launch(k_invar_pro<true>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(outer), L, j, c->r64.p, c->x64.p,
             c->b64.p, tol2, s.ls_maxit);
    P.while_loop(outer, [&] {
      P.launch(k_cg32_init, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(inner), (const double2*)c->r64.p,
               c->r32.p, c->x32.p, s.inner_tol * s.inner_tol, s.inner_maxit, tol2, outer);
      // FP32 CG per iteration: p and the deferred x update with the 2 -> 3 mix; the
      // slow-axis transforms with the partial sums of <p, Ap>; the 3 -> 2 unmix with
      // r -= a Ap and the partial sums of ||r||^2 (Ap is never stored); a one-warp-per-slot
      // kernel that ends the iteration (step size, beta, loop decision)
      P.while_loop(inner, [&] {
        o.plane_inv<float, IN_CG, false>(nullptr, c->T32.p, 1, M, F, 0, c->p32.p, c->r32.p, nullptr, nullptr,
                                         inner, c->x32.p);
        o.pencil<float, PEN_QBQ_CG>(c->T32.p, 1, F, c->ibq32(), 1);
        o.plane_fwd<float, EPI_CGR, false>(c->T32.p, nullptr, 1, M, F, nullptr, nullptr, inner, 0.0, c->r32.p);
        o.cg_decide(inner);
      });
      o.plane_inv<double, IN_REFINE, false>(nullptr, c->T64.p, 1, M, F, 0, nullptr, nullptr, c->x64.p,
                                            c->x32.p, Cond{}, nullptr, c->p32.p);
      o.pencil<double, PEN_QBQ>(c->T64.p, 1, F, c->ibq64(), 2);
      o.plane_fwd<double, EPI_RESID, false>(c->T64.p, c->r64.p, 1, M, F, nullptr, c->b64.p, outer, tol2);
    });
    P.launch(k_invar_epi<true>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L, j,
             (const double2*)c->x64.p, (const double2*)nullptr);
  }
  const int ndots = (int)((M + kLzRows - 1) / kLzRows);
  P.launch(k_lz_dots, dim3(ndots, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L, j);
  P.launch(k_lz_update, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L, j);
}

static void record_solve(fame_ctx* c, Program& P, const SolveCfg& s) {
  Ops o{c, P, s.nslots};
  const Geom& g = c->g;
  const long M = 2L * g.N;
  const long F = 3L * g.N;
  const int nvb = vec_blocks(c, s.nslots);
  const int nphys = s.nstep + 1 + s.nwant + 1;
  LzArgs L;
  L.U = c->U.p;
  L.ustride = M;
  L.nphys = nphys;
  L.map = c->map.p;
  L.nstep = s.nstep;
  L.nwant = s.nwant;
  L.T0 = c->T0.p;
  L.T1 = c->T1.p;
  L.h = c->hcoef.p;
  L.lz = c->lz.p;
  L.prof = c->prof.p;
  L.status = c->status.p;
  int* flags = c->flags.p;
  const int tmax = std::max({g.Nx * g.Ny, g.Nx, g.Ny, g.Nz});
  P.launch(k_tables, dim3((tmax + 255) / 256, s.nslots), dim3(256), 0, g, (const Slot*)c->slots.p, c->tabs.p,
           (double)c->lat.m[0], (double)c->lat.m[1], (double)c->lat.m[2]);
  P.launch(k_lz_init, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L);
  for (int j = 0; j < s.nstep; j++) emit_step(o, s, L, j, flags);
  Cond restart = loop_cond(P, flags, kLoopRestart, s.es_maxit + 2, s.loop_cap);
  TriArgs ta;
  ta.L = L;
  ta.slots = c->slots.p;
  ta.theta = c->theta.p;
  ta.Z = c->Z.p;
  ta.G = c->G.p;
  ta.tol = s.es_tol;
  ta.maxit = s.es_maxit;
  ta.cond = restart;
  ta.nslots = s.nslots;
  ta.status = c->status.p;
  ta.ctr = c->tri_ctr.p;
  ta.first = 1;
  const size_t tsm = tridiag_smem(s.nstep);
  allow_smem(k_tridiag, tsm);
  P.launch(k_tridiag, dim3(s.nslots), dim3(32), tsm, ta);
  ta.first = 0;
  P.while_loop(restart, [&] {
    for (int c0 = 0; c0 <= s.nwant; c0 += 8)
      P.launch(k_ugemm<8>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(restart), L, (const double*)c->G.p,
               s.nstep + 1, s.nstep + 1, s.nwant + 1, 0, (double2*)nullptr, c0);
    P.launch(k_remap, dim3(s.nslots), dim3(32), 0, L, (const Slot*)c->slots.p, s.nslots);
    for (int j = s.nwant; j < s.nstep; j++) emit_step(o, s, L, j, flags);
    P.launch(k_tridiag, dim3(s.nslots), dim3(32), tsm, ta);
  });
  // Ritz vectors ev = U(:, 0:nstep) z(:, 0:nwant)   (Lanczos_Isotropic.cu:93)
  for (int c0 = 0; c0 < s.nwant; c0 += 8)
    P.launch(k_ugemm<8>, dim3(nvb, 1, s.nslots), dim3(256), 0, o.va(Cond{}), L, (const double*)c->Z.p,
             s.nstep, s.nstep, s.nwant, 1, c->EV.p, c0);
  // FP64 residual and Rayleigh quotient per band: v = QBQ(Sigma y)
  o.plane_inv<double, IN_VEC, false>(c->EV.p, c->Tb.p, s.nwant, M, F, 1);
  o.pencil<double, PEN_QBQ>(c->Tb.p, s.nwant, F, c->ibq64(), 0);
  o.plane_fwd<double, EPI_OUT, false>(c->Tb.p, c->AV.p, s.nwant, M, F);
  P.launch(k_band_stats, dim3(kBandSplit, s.nwant, s.nslots), dim3(256), 0, o.va(Cond{}),
           (const double2*)c->EV.p, (const double2*)c->AV.p, M, s.nwant, (const double*)c->theta.p, s.nstep,
           c->bpart.p);
  P.launch(k_rows_sum, dim3(s.nwant, s.nslots), dim3(32), 0, (const Slot*)c->slots.p, s.nwant,
           (const double*)c->bpart.p, kBandSplit, 4, c->stats.p);
  if (s.vec || s.enorm) {
    // E = B^{-1} Q_r (Sigma ev), scaled by its norm (FAME_Fast_Algorithms_Isotropic.cu:107-122);
    // the norms go after the band statistics
    o.plane_inv<double, IN_VEC, false>(c->EV.p, c->Tb.p, s.nwant, M, F, 1);
    o.pencil<double, PEN_QR_OUT>(c->Tb.p, s.nwant, F, c->invB64.p, 0, c->E.p);
    P.launch(k_band_norm_part, dim3(kBandSplit, s.nwant, s.nslots), dim3(256), 0, (const Slot*)c->slots.p,
             (const double2*)c->E.p, F, s.nwant, F, c->bpart.p);
    P.launch(k_band_scale, dim3(4 * kBandSplit, s.nwant, s.nslots), dim3(256), 0, (const Slot*)c->slots.p, c->E.p, F,
             s.nwant, F, (const double*)c->bpart.p, kBandSplit, c->stats.p + (size_t)s.nslots * s.nwant * 4);
  }
}

// Device bytes of one slot's workspace (the per-slot buffers of ensure_workspace).
static double slot_bytes(const fame_ctx* c, int nstep, int nwant, bool mixed, bool vec) {
  const double N = c->g.N, M = 2.0 * N, z = 16.0;
  double b = (nstep + 1 + nwant + 1) * M * z   // Lanczos basis U
             + 2 * M * z + 3 * N * z           // r64, x64, T64
             + 2 * nwant * M * z + nwant * 3 * N * z  // EV, AV, Tb
             + 2 * M * z;                      // p64, Ap64
  if (mixed) b += M * z + 3 * M * 8 + 3 * N * 8;  // b64, r32, x32, p32, T32
  if (vec) b += nwant * 3 * N * z;               // E
  return b;
}

// k-points per batch.  The stage kernels of one k-point do not fill the GPU (a 96^3
// plane stage is 96 three-CTA clusters, slightly more than fit at once), so several
// k-points per launch pay: as many as 60% of the free device memory holds, at most 64.
// Slots of workspace the context already holds for this configuration (0 if a solve
// with it would have to reallocate).
static int held_slots(const fame_ctx* c, int nstep, int nwant, bool mixed, bool vec) {
  const bool fits = c->cap_nstep >= nstep && c->cap_nwant >= nwant && (!mixed || c->cap_mixed) && (!vec || c->cap_vec);
  return fits ? c->cap_slots : 0;
}

// Automatic batch: what 60% of the free device memory holds, or the slots the context
// already holds if more (free memory no longer counts them), at most 64 and nk.
static int choose_batch(const fame_ctx* c, int nk, const fame_solver_params* p, bool vec) {
  if (p->batch > 0) return std::min(p->batch, nk);
  size_t free_b = 0, total_b = 0;
  FAME_CK(cudaMemGetInfo(&free_b, &total_b));
  const bool mixed = p->precision == FAME_MIXED;
  const double per = slot_bytes(c, p->nstep, p->nwant, mixed, vec);
  const int b = std::max((int)std::max(1.0, floor(0.6 * (double)free_b / per)),
                         held_slots(c, p->nstep, p->nwant, mixed, vec));
  return std::max(1, std::min({b, nk, 64}));
}

}  // namespace fame

// ================================================================== C ABI
extern "C" {

const char* fame_last_error(void) { return g_err.c_str(); }
const char* fame_version(void) { return "fame-b200 0.1 (sm_100a)"; }

int fame_ctx_create(int device, const fame_lattice* lat, fame_ctx** out) {
  if (!lat || !out) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_err("no CUDA device");
    return FAME_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_err("device index out of range");
    return FAME_ERR_BAD_INPUT;
  }
  fame_ctx* c = new fame_ctx();
  try {
    c->device = device;
    c->lat = *lat;
    FAME_CK(cudaSetDevice(device));
    int rc = setup_geom(c);
    if (rc) {
      delete c;
      return rc;
    }
    FAME_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    FAME_CK(cudaMallocHost(&c->hflag, sizeof(int)));
    c->invB64.ensure(3L * c->g.N);
    c->B64.ensure(3L * c->g.N);
    c->invB32.ensure(3L * c->g.N);
    if (c->g.general) {
      c->invB64q.ensure(3L * c->g.N);
      c->invB32q.ensure(3L * c->g.N);
    }
  } catch (const CudaError& e) {
    set_err(e.what());
    delete c;
    return FAME_ERR_CUDA;
  }
  *out = c;
  return FAME_OK;
}

void fame_ctx_destroy(fame_ctx* c) {
  if (!c) return;
  for (fame_ctx* l : c->lane_ctx) fame_ctx_destroy(l);
  c->lane_ctx.clear();
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->progs.clear();
  for (auto* b : {&c->tw64, &c->tabs, &c->U, &c->r64, &c->x64, &c->b64, &c->p64, &c->Ap64, &c->T64, &c->EV,
                  &c->AV, &c->Tb, &c->E})
    b->release();
  for (auto* b : {&c->r32, &c->x32, &c->p32, &c->T32, &c->tw32}) b->release();
  for (auto* b : {&c->invB64, &c->invB64q, &c->B64, &c->partials, &c->T0, &c->T1, &c->hcoef, &c->theta, &c->Z, &c->G,
                  &c->stats, &c->adj, &c->bpart, &c->adj_part})
    b->release();
  c->eps_bad.release();
  c->invB32.release();
  c->invB32q.release();
  c->slots.release();
  c->cg.release();
  c->lz.release();
  c->counters.release();
  c->tri_ctr.release();
  c->map.release();
  c->prof.release();
  c->status.release();
  c->flags.release();
  if (c->hflag) cudaFreeHost(c->hflag);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int fame_ctx_sizes(const fame_ctx* c, long long* N_out) {
  if (!c || !N_out) return FAME_ERR_BAD_INPUT;
  *N_out = c->g.N;
  return FAME_OK;
}

int fame_set_eps(fame_ctx* c, const double* B) {
  if (!c || !B) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  const long n3 = 3L * c->g.N;
  std::vector<double> ib(n3);
  std::vector<float> ib32(n3);
  for (long i = 0; i < n3; i++) {
    if (!(B[i] > 0.0) || !isfinite(B[i])) {
      set_err("permittivity must be finite and positive (edge " + std::to_string(i) + ")");
      return FAME_ERR_BAD_INPUT;
    }
    ib[i] = 1.0 / B[i];
    ib32[i] = (float)ib[i];
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    FAME_CK(cudaMemcpy(c->B64.p, B, n3 * sizeof(double), cudaMemcpyHostToDevice));
    FAME_CK(cudaMemcpy(c->invB64.p, ib.data(), n3 * sizeof(double), cudaMemcpyHostToDevice));
    FAME_CK(cudaMemcpy(c->invB32.p, ib32.data(), n3 * sizeof(float), cudaMemcpyHostToDevice));
    if (c->g.general) {
      // spatial edge index (z*Ny + y)*Nx + x  ->  field index (x*Ny + y)*Nz + z
      const Geom& g = c->g;
      std::vector<double> q(n3);
      std::vector<float> q32(n3);
      for (int comp = 0; comp < 3; comp++) {
        const long cb = (long)comp * g.N;
        for (int z = 0; z < g.Nz; z++)
          for (int y = 0; y < g.Ny; y++)
            for (int x = 0; x < g.Nx; x++) {
              const long src = cb + ((long)z * g.Ny + y) * g.Nx + x;
              const long dst = cb + ((long)x * g.Ny + y) * g.Nz + z;
              q[dst] = ib[src];
              q32[dst] = ib32[src];
            }
      }
      FAME_CK(cudaMemcpy(c->invB64q.p, q.data(), n3 * sizeof(double), cudaMemcpyHostToDevice));
      FAME_CK(cudaMemcpy(c->invB32q.p, q32.data(), n3 * sizeof(float), cudaMemcpyHostToDevice));
    }
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  c->have_eps = true;
  c->eps_ver++;
  return FAME_OK;
}

int fame_set_material(fame_ctx* c, const int* binout, int material_num, const double* eps_in, double eps_out) {
  if (!c || !binout || (material_num > 0 && !eps_in)) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  const long N = c->g.N;
  std::vector<double> B(3 * N, eps_out);
  for (int comp = 0; comp < 3; comp++)
    for (long i = 0; i < N; i++)
      for (int j = 0; j < material_num; j++)
        if (binout[i + j * N + (long)comp * material_num * N] == 1) B[comp * N + i] = eps_in[j];
  return fame_set_eps(c, B.data());
}

// false when any of the n wave vectors has a NaN or infinite component
static bool finite_k(const double* k, long n) {
  for (long i = 0; i < 3 * n; i++)
    if (!std::isfinite(k[i])) return false;
  return true;
}

// One context's solve of nk k-points in batches (the body of fame_solve_kpoints).
static int solve_batched(fame_ctx* c, const double* k_xyz, int nk, const fame_solver_params* prm,
                         double* freq_out, double* relres_out, double* relerr_out, double* resabs_out,
                         double* evec_out, fame_kcounters* counters) {
  if (!c || !k_xyz || !prm || !freq_out || nk <= 0) {
    set_err("null or empty argument");
    return FAME_ERR_BAD_INPUT;
  }
  if (!finite_k(k_xyz, nk)) {
    set_err("wave vector with a NaN or infinite component");
    return FAME_ERR_BAD_INPUT;
  }
  if (!c->have_eps) {
    set_err("permittivity not set (fame_set_eps / fame_set_material)");
    return FAME_ERR_BAD_INPUT;
  }
  const fame_solver_params& p = *prm;
  if (p.nwant < 1 || p.nstep <= p.nwant || p.nstep > kMaxStep || p.es_maxit < 0 || p.ls_maxit < 1 ||
      !(p.es_tol > 0) || !(p.ls_tol > 0) || (p.precision != FAME_FP64 && p.precision != FAME_MIXED)) {
    set_err("invalid solver parameters (need 1 <= nwant < nstep <= 64, positive tolerances)");
    return FAME_ERR_BAD_INPUT;
  }
  const bool vec_device = p.want_vectors && !evec_out;  // eigenvectors kept on the device
  if (vec_device && p.batch > 0 && p.batch < nk) {
    set_err("eigenvectors kept on the device (evec_out NULL) need all k-points in one batch");
    return FAME_ERR_BAD_INPUT;
  }
  c->dev_vec_nk = 0;
  int rc_all = FAME_OK;
  int status_any = 0;
  try {
    FAME_CK(cudaSetDevice(c->device));
    SolveCfg s;
    s.nslots = choose_batch(c, nk, &p, p.want_vectors || resabs_out);
    if (vec_device && s.nslots < nk) {
      set_err("eigenvectors kept on the device (evec_out NULL) need all k-points in one batch; " +
              std::to_string(nk) + " k-points exceed the " + std::to_string(s.nslots) + " that fit");
      return FAME_ERR_BAD_INPUT;
    }
    s.nstep = p.nstep;
    s.nwant = p.nwant;
    s.es_maxit = p.es_maxit;
    s.ls_maxit = p.ls_maxit;
    s.mixed = p.precision == FAME_MIXED;
    s.vec = p.want_vectors ? 1 : 0;
    s.enorm = resabs_out ? 1 : 0;
    s.es_tol = p.es_tol;
    s.ls_tol = p.ls_tol;
    s.inner_tol = p.inner_tol > 0 ? p.inner_tol : 2e-6;  // two FP64 refinement steps reach 1e-12
    s.inner_maxit = p.inner_maxit > 0 ? p.inner_maxit : 200;
    s.loop_cap = c->loop_cap;
    const bool graph = p.use_graph != 0;
    ensure_workspace(c, s.nslots, s.nstep, s.nwant, s.mixed, s.vec || s.enorm);
    const std::string key = cfg_key(s, graph);
    auto it = c->progs.find(key);
    Program* P = nullptr;
    if (graph) {
      if (it == c->progs.end()) {
        auto prog = std::make_unique<Program>(c->stream, true, c->hflag, 0);
        record_solve(c, *prog, s);
        prog->instantiate();
        P = prog.get();
        c->progs[key] = std::move(prog);
      } else {
        P = it->second.get();
      }
    }
    const long N = c->g.N;
    std::vector<Slot> hs(s.nslots);
    std::vector<double> theta((size_t)s.nslots * s.nstep), stats((size_t)s.nslots * s.nwant * 5);
    std::vector<LzState> lz(s.nslots);
    std::vector<int> prof(3 * s.nslots), status(s.nslots);
    for (int b0 = 0; b0 < nk; b0 += s.nslots) {
      const int nb = std::min(s.nslots, nk - b0);
      for (int q = 0; q < s.nslots; q++) {
        Slot& sl = hs[q];
        memset(&sl, 0, sizeof(sl));
        if (q < nb) {
          const double* k = k_xyz + 3L * (b0 + q);
          sl = make_slot(c->lat, k);
        } else {
          sl.Nd = (int)N;
          sl.active = 0;
        }
      }
      FAME_CK(cudaMemcpyAsync(c->slots.p, hs.data(), s.nslots * sizeof(Slot), cudaMemcpyHostToDevice, c->stream));
      FAME_CK(cudaMemsetAsync(c->status.p, 0, s.nslots * sizeof(int), c->stream));
      FAME_CK(cudaMemsetAsync(c->flags.p, 0, 64 * sizeof(int), c->stream));
      if (graph) {
        P->run();
      } else {
        Program hp(c->stream, false, c->hflag, 100000);
        record_solve(c, hp, s);
      }
      FAME_CK(cudaMemcpyAsync(theta.data(), c->theta.p, theta.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
      FAME_CK(cudaMemcpyAsync(stats.data(), c->stats.p, stats.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
      FAME_CK(cudaMemcpyAsync(lz.data(), c->lz.p, lz.size() * sizeof(LzState), cudaMemcpyDeviceToHost, c->stream));
      FAME_CK(cudaMemcpyAsync(prof.data(), c->prof.p, prof.size() * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      FAME_CK(cudaMemcpyAsync(status.data(), c->status.p, status.size() * sizeof(int), cudaMemcpyDeviceToHost,
                              c->stream));
      int hflags[64];
      FAME_CK(cudaMemcpyAsync(hflags, c->flags.p, sizeof(hflags), cudaMemcpyDeviceToHost, c->stream));
      FAME_CK(cudaStreamSynchronize(c->stream));
      for (int id = 0; id < 8; id++)
        if (hflags[kTrips + 2 * id + 1]) {
          set_err("a device loop reached its trip cap (loop " + std::to_string(id) + ")");
          return FAME_ERR_WATCHDOG;
        }
      if (hflags[kFaultFlag]) {
        set_err("a bounded device wait ran out (shared-memory exchange of a plane cluster)");
        return FAME_ERR_WATCHDOG;
      }
      for (int q = 0; q < nb; q++) {
        const int kk = b0 + q;
        const bool gamma = hs[q].Nd == N - 1;
        std::vector<double> f(s.nwant), rr(s.nwant), re(s.nwant), ra(s.nwant);
        for (int i = 0; i < s.nwant; i++) {
          const double th = theta[(size_t)q * s.nstep + i];
          f[i] = sqrt(1.0 / th);
          const double* st = &stats[((size_t)q * s.nwant + i) * 4];
          const double lam = 1.0 / th;
          rr[i] = sqrt(st[0]) / (lam * sqrt(st[1]));
          const double rho = st[2] / st[3];
          re[i] = fabs(lam - rho) / rho;
          // ||C^H C E - w^2 B E|| = sqrt(st[0] / N) for E = B^-1 Q_r Sigma y (Q_r carries
          // the 1/N of the unnormalised inverse DFT, so ||Q_r z|| = ||z|| / sqrt(N)); the
          // reference restores s E with s = ||E|| (FAME_Fast_Algorithms_Isotropic.cu:119-121)
          ra[i] = s.enorm ? stats[(size_t)s.nslots * s.nwant * 4 + (size_t)q * s.nwant + i] * sqrt(st[0] / N) : 0.0;
        }
        // Gamma patch: bands shift up by two, w0 = w1 = 0 (FAME_Fast_Algorithms_Isotropic.cu:61-79)
        std::vector<double> fo(f), ro(rr), eo(re), ao(ra);
        if (gamma) {
          for (int i = s.nwant - 1; i >= 2; i--) {
            fo[i] = f[i - 2];
            ro[i] = rr[i - 2];
            eo[i] = re[i - 2];
            ao[i] = ra[i - 2];
          }
          fo[0] = fo[1] = 0.0;
          ro[0] = ro[1] = 0.0;
          eo[0] = eo[1] = 0.0;
          ao[0] = ao[1] = 0.0;  // constant E: C E = 0
        }
        for (int i = 0; i < s.nwant; i++) {
          freq_out[(size_t)kk * s.nwant + i] = fo[i];
          if (relres_out) relres_out[(size_t)kk * s.nwant + i] = ro[i];
          if (relerr_out) relerr_out[(size_t)kk * s.nwant + i] = eo[i];
          if (resabs_out) resabs_out[(size_t)kk * s.nwant + i] = ao[i];
        }
        if (counters) {
          fame_kcounters& kc = counters[kk];
          kc.ls_iter = prof[3 * q];
          kc.es_iter = prof[3 * q + 1];
          kc.restarts = lz[q].restarts;
          kc.status = status[q] == 0 ? FAME_OK : FAME_ERR_NO_CONVERGENCE;
          kc.detail = status[q];
          kc.Nd = hs[q].Nd;
          kc.refine = prof[3 * q + 2];
        }
        if (status[q] != 0) rc_all = FAME_ERR_NO_CONVERGENCE;
        status_any |= status[q];
        if (s.vec && vec_device) {
          if (q == 0) {
            c->dev_vec_nk = nb;
            c->dev_vec_nwant = s.nwant;
            c->dev_vec_gamma.assign(nb, 0);
          }
          c->dev_vec_gamma[q] = gamma ? 1 : 0;
        } else if (s.vec) {
          const size_t n3 = 3 * (size_t)N;
          double2* dst = reinterpret_cast<double2*>(evec_out) + (size_t)kk * s.nwant * n3;
          const double2* src = c->E.p + (size_t)q * s.nwant * n3;
          if (!gamma) {
            FAME_CK(cudaMemcpy(dst, src, s.nwant * n3 * sizeof(double2), cudaMemcpyDeviceToHost));
          } else {
            if (s.nwant > 2)
              FAME_CK(cudaMemcpy(dst + 2 * n3, src, (s.nwant - 2) * n3 * sizeof(double2), cudaMemcpyDeviceToHost));
            const double v = 1.0 / sqrt(3.0 * N);
            for (size_t i = 0; i < 2 * n3; i++) dst[i] = make_double2(v, 0.0);
          }
        }
      }
    }
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  } catch (const std::exception& e) {
    set_err(e.what());
    return FAME_ERR_WATCHDOG;
  }
  if (rc_all) {
    std::string m = "no convergence for some k-point:";
    if (status_any & kStatusCG) m += " an A_r^-1 solve stopped above ls_tol (ls_maxit or the refinement cap);";
    if (status_any & kStatusLanczos) m += " Lanczos did not converge within es_maxit restarts;";
    if (status_any & kStatusQL) m += " the tridiagonal eigensolve failed;";
    set_err(m);
  }
  return rc_all;
}

// Lane contexts 1 .. G-1 of c: created on first use with c's lattice, given c's
// permittivity (device to device) whenever it changed, and c's execution options.
static int sync_lanes(fame_ctx* c, int G) {
  while ((int)c->lane_ctx.size() < G - 1) {
    fame_ctx* l = nullptr;
    const int rc = fame_ctx_create(c->device, &c->lat, &l);
    if (rc != FAME_OK) return rc;
    c->lane_ctx.push_back(l);
    c->lane_eps_ver.push_back(-1);
  }
  for (int i = 0; i < G - 1; i++) {
    fame_ctx* l = c->lane_ctx[i];
    if (c->lane_eps_ver[i] != c->eps_ver) {
      const int rc = fame_set_eps_device(l, c->B64.p);
      if (rc != FAME_OK) return rc;
      c->lane_eps_ver[i] = c->eps_ver;
    }
    const struct {
      const char* name;
      int want, have;
    } opts[] = {{"prefetch", c->prefetch, l->prefetch},
                {"self_prefetch", c->self_prefetch, l->self_prefetch},
                {"static_planes", c->static_planes, l->static_planes},
                {"radix_order", c->radix_order, l->radix_order},
                {"plane_threads32", c->threads32_opt, l->threads32_opt},
                {"plane_threads64", c->threads64_opt, l->threads64_opt}};
    for (const auto& o : opts)
      if (o.want != o.have) {
        const int rc = fame_set_option(l, o.name, o.want);
        if (rc != FAME_OK) return rc;
      }
    l->loop_cap = c->loop_cap;
  }
  return FAME_OK;
}

int fame_solve_kpoints(fame_ctx* c, const double* k_xyz, int nk, const fame_solver_params* prm,
                       double* freq_out, double* relres_out, double* relerr_out, double* resabs_out,
                       double* evec_out, fame_kcounters* counters) {
  int G = 1;
  if (c && k_xyz && prm && freq_out && nk > 0 && finite_k(k_xyz, nk) && c->have_eps && prm->batch == 0 &&
      !(prm->want_vectors && !evec_out) && c->lanes > 1)
    G = std::min(c->lanes, nk / 4);
  if (G <= 1)
    return solve_batched(c, k_xyz, nk, prm, freq_out, relres_out, relerr_out, resabs_out, evec_out, counters);
  std::vector<fame_solver_params> pl(G, *prm);
  try {
    FAME_CK(cudaSetDevice(c->device));
    // without its lane contexts (say, no device memory for one) the call runs as one batch
    if (sync_lanes(c, G) != FAME_OK)
      return solve_batched(c, k_xyz, nk, prm, freq_out, relres_out, relerr_out, resabs_out, evec_out, counters);
    // each lane's batch: its k-points, at most what 60% of the free memory holds over
    // the G lanes (lane contexts allocate their workspace on their first solve)
    size_t free_b = 0, total_b = 0;
    FAME_CK(cudaMemGetInfo(&free_b, &total_b));
    const bool mixed = prm->precision == FAME_MIXED, vec = prm->want_vectors || resabs_out;
    const double per = slot_bytes(c, prm->nstep, prm->nwant, mixed, vec);
    const int cap = (int)std::max(1.0, std::min(64.0, floor(0.6 * (double)free_b / (G * per))));
    for (int i = 0; i < G; i++) {
      const fame_ctx* l = i == 0 ? c : c->lane_ctx[i - 1];
      const int held = std::min(64, held_slots(l, prm->nstep, prm->nwant, mixed, vec));
      pl[i].batch = std::min(std::max(cap, held), (int)((long)nk * (i + 1) / G - (long)nk * i / G));
    }
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  const size_t nw = (size_t)prm->nwant, n3 = 3 * (size_t)c->g.N;
  std::vector<int> rcs(G, FAME_OK);
  std::vector<std::string> errs(G);
  auto run = [&](int i) {
    fame_ctx* l = i == 0 ? c : c->lane_ctx[i - 1];
    const long a = (long)nk * i / G, b = (long)nk * (i + 1) / G;
    cudaSetDevice(c->device);
    rcs[i] = solve_batched(l, k_xyz + 3 * a, (int)(b - a), &pl[i], freq_out + a * nw,
                           relres_out ? relres_out + a * nw : nullptr, relerr_out ? relerr_out + a * nw : nullptr,
                           resabs_out ? resabs_out + a * nw : nullptr, evec_out ? evec_out + a * nw * n3 * 2 : nullptr,
                           counters ? counters + a : nullptr);
    if (rcs[i] != FAME_OK) errs[i] = fame_last_error();
  };
  std::vector<std::thread> th;
  for (int i = 1; i < G; i++) th.emplace_back(run, i);
  run(0);
  for (auto& t : th) t.join();
  // a failure outranks a k-point that did not converge
  int out = FAME_OK;
  for (int pass = 0; pass < 2 && out == FAME_OK; pass++)
    for (int i = 0; i < G; i++)
      if (rcs[i] != FAME_OK && (pass == 1 || rcs[i] != FAME_ERR_NO_CONVERGENCE)) {
        out = rcs[i];
        set_err(errs[i]);
        break;
      }
  return out;
}

int fame_apply(fame_ctx* c, int op, const double* k, const void* in, void* out, int precision,
               const fame_solver_params* prm, int* Nd_out) {
  if (!c || !k || !in || !out) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  if (op < FAME_OP_QR || op > FAME_OP_INVAR || (precision != FAME_FP64 && precision != FAME_MIXED) ||
      (op == FAME_OP_INVAR && (precision != FAME_FP64 || !prm))) {
    set_err("unsupported operator/precision combination");
    return FAME_ERR_BAD_INPUT;
  }
  if ((op == FAME_OP_QBQ || op == FAME_OP_INVAR) && !c->have_eps) {
    set_err("permittivity not set");
    return FAME_ERR_BAD_INPUT;
  }
  if (!finite_k(k, 1)) {
    set_err("wave vector with a NaN or infinite component");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    ensure_workspace(c, 1, std::max(2, c->cap_nstep), std::max(1, c->cap_nwant), c->cap_mixed, c->cap_vec);
    if (precision == FAME_MIXED) ensure_workspace(c, 1, c->cap_nstep, c->cap_nwant, true, c->cap_vec);
    const Slot sl = make_slot(c->lat, k);
    if (Nd_out) *Nd_out = sl.Nd;
    FAME_CK(cudaMemcpyAsync(c->slots.p, &sl, sizeof(Slot), cudaMemcpyHostToDevice, c->stream));
    Program P(c->stream, false, c->hflag, 100000);
    Ops o{c, P, 1};
    const Geom& g = c->g;
    const long M = 2L * g.N, F = 3L * g.N;
    const int tmax = std::max({g.Nx * g.Ny, g.Nx, g.Ny, g.Nz});
    P.launch(k_tables, dim3((tmax + 255) / 256, 1), dim3(256), 0, g, (const Slot*)c->slots.p, c->tabs.p,
             (double)c->lat.m[0], (double)c->lat.m[1], (double)c->lat.m[2]);
    if (precision == FAME_FP64) {
      const double2* x = (const double2*)in;
      double2* y = (double2*)out;
      switch (op) {
        case FAME_OP_QR:
        case FAME_OP_PR:
          if (op == FAME_OP_QR)
            o.plane_inv<double, IN_VEC, false>(x, c->T64.p, 1, M, F, 0);
          else
            o.plane_inv<double, IN_VEC, true>(x, c->T64.p, 1, M, F, 0);
          o.pencil<double, PEN_QR_OUT>(c->T64.p, 1, F, (const double*)nullptr, 0, y);
          break;
        case FAME_OP_QRS:
        case FAME_OP_PRS:
          o.pencil<double, PEN_QRS_IN>(c->T64.p, 1, F, (const double*)nullptr, 0, nullptr, x);
          if (op == FAME_OP_QRS)
            o.plane_fwd<double, EPI_OUT, false>(c->T64.p, y, 1, M, F);
          else
            o.plane_fwd<double, EPI_OUT, true>(c->T64.p, y, 1, M, F);
          break;
        case FAME_OP_QBQ:
          o.plane_inv<double, IN_VEC, false>(x, c->T64.p, 1, M, F, 0);
          o.pencil<double, PEN_QBQ>(c->T64.p, 1, F, c->ibq64(), 0);
          o.plane_fwd<double, EPI_OUT, false>(c->T64.p, y, 1, M, F);
          break;
        case FAME_OP_INVAR: {
          // one A_r^{-1} apply through the solver's own invAr kernels (U column 0 -> 1)
          ensure_workspace(c, 1, std::max(2, c->cap_nstep), std::max(1, c->cap_nwant), c->cap_mixed, c->cap_vec);
          const int nstep = c->cap_nstep, nwant = c->cap_nwant;
          LzArgs L;
          L.U = c->U.p;
          L.ustride = M;
          L.nphys = nstep + 1 + nwant + 1;
          L.map = c->map.p;
          L.nstep = nstep;
          L.nwant = nwant;
          L.T0 = c->T0.p;
          L.T1 = c->T1.p;
          L.h = c->hcoef.p;
          L.lz = c->lz.p;
          L.prof = c->prof.p;
          L.status = c->status.p;
          P.launch(k_lz_init, dim3(1, 1, 1), dim3(256), 0, o.va(Cond{}), L);
          FAME_CK(cudaMemcpyAsync(c->U.p, x, 2L * sl.Nd * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
          SolveCfg s;
          memset(&s, 0, sizeof(s));
          s.nslots = 1;
          s.ls_maxit = prm->ls_maxit;
          s.ls_tol = prm->ls_tol;
          s.mixed = 0;
          const int nvb = vec_blocks(c, 1);
          Cond cc = loop_cond(P, c->flags.p, kLoopCG, s.ls_maxit + 2);
          P.launch(k_invar_pro<false>, dim3(nvb, 1, 1), dim3(256), 0, o.va(cc), L, 0, c->r64.p, c->x64.p,
                   (double2*)nullptr, s.ls_tol * s.ls_tol, s.ls_maxit);
          P.while_loop(cc, [&] {
            o.plane_inv<double, IN_CG, false>(nullptr, c->T64.p, 1, M, F, 0, c->p64.p, c->r64.p, nullptr, nullptr,
                                              cc, c->x64.p);
            o.pencil<double, PEN_QBQ>(c->T64.p, 1, F, c->ibq64(), 1);
            o.plane_fwd<double, EPI_CG, false>(c->T64.p, c->Ap64.p, 1, M, F, c->p64.p);
            P.launch(k_cg_update<double>, dim3(nvb, 1, 1), dim3(256), 0, o.va(cc), c->r64.p,
                     (const double2*)c->Ap64.p);
          });
          P.launch(k_invar_epi<false>, dim3(nvb, 1, 1), dim3(256), 0, o.va(Cond{}), L, 0,
                   (const double2*)c->x64.p, (const double2*)c->p64.p);
          FAME_CK(cudaMemcpyAsync(y, c->U.p + M, 2L * sl.Nd * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
          break;
        }
      }
    } else {
      const float2* x = (const float2*)in;
      float2* y = (float2*)out;
      switch (op) {
        case FAME_OP_QR:
        case FAME_OP_PR:
          if (op == FAME_OP_QR)
            o.plane_inv<float, IN_VEC, false>(x, c->T32.p, 1, M, F, 0);
          else
            o.plane_inv<float, IN_VEC, true>(x, c->T32.p, 1, M, F, 0);
          o.pencil<float, PEN_QR_OUT>(c->T32.p, 1, F, (const float*)nullptr, 0, y);
          break;
        case FAME_OP_QRS:
        case FAME_OP_PRS:
          o.pencil<float, PEN_QRS_IN>(c->T32.p, 1, F, (const float*)nullptr, 0, nullptr, x);
          if (op == FAME_OP_QRS)
            o.plane_fwd<float, EPI_OUT, false>(c->T32.p, y, 1, M, F);
          else
            o.plane_fwd<float, EPI_OUT, true>(c->T32.p, y, 1, M, F);
          break;
        case FAME_OP_QBQ:
          o.plane_inv<float, IN_VEC, false>(x, c->T32.p, 1, M, F, 0);
          o.pencil<float, PEN_QBQ>(c->T32.p, 1, F, c->ibq32(), 0);
          o.plane_fwd<float, EPI_OUT, false>(c->T32.p, y, 1, M, F);
          break;
      }
    }
    FAME_CK(cudaStreamSynchronize(c->stream));
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  } catch (const std::exception& e) {
    set_err(e.what());
    return FAME_ERR_WATCHDOG;
  }
  return FAME_OK;
}

void* fame_ctx_stream(fame_ctx* c) { return c ? (void*)c->stream : nullptr; }

int fame_set_option(fame_ctx* c, const char* name, int value) {
  if (!c || !name) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  const std::string n(name);
  const bool threads_ok = value == 0 || (value >= 64 && value <= kPlaneThreads && value % 32 == 0);
  if (n == "prefetch" && (value == 0 || value == 1)) {
    c->prefetch = value;
  } else if (n == "self_prefetch" && (value == 0 || value == 1)) {
    c->self_prefetch = value;
  } else if (n == "static_planes" && (value == 0 || value == 1)) {
    c->static_planes = value;
  } else if (n == "lanes" && value >= 1 && value <= 8) {
    c->lanes = value;
    // lane contexts beyond the new count are released with their device memory
    while ((int)c->lane_ctx.size() > value - 1) {
      fame_ctx_destroy(c->lane_ctx.back());
      c->lane_ctx.pop_back();
      c->lane_eps_ver.pop_back();
    }
    return FAME_OK;  // no recorded graph changes
  } else if (n == "radix_order" && value >= 0 && value < kNumRadixOrders) {
    Geom g;
    std::string err;
    if (layout_geom(c->lat, g, 1L << 28, err, value) != FAME_OK || plane_level(g) != c->rare ||
        pencil_level(g) != c->rare_pen) {
      set_err("radix order " + std::to_string(value) + " gives no plan for this grid");
      return FAME_ERR_BAD_INPUT;
    }
    c->radix_order = value;
    c->g.pf = g.pf;
    c->g.pm = g.pm;
    c->g.ps = g.ps;
  } else if (n == "plane_threads32" && threads_ok) {
    c->threads32_opt = value;
    c->plane_threads32 = value ? value : plane_threads_rule<float>(c->g, c->rare);
  } else if (n == "plane_threads64" && threads_ok) {
    c->threads64_opt = value;
    c->plane_threads = value ? value : plane_threads_rule<double>(c->g, c->rare);
  } else {
    set_err("unknown option or value: " + n + " = " + std::to_string(value));
    return FAME_ERR_BAD_INPUT;
  }
  c->progs.clear();  // recorded graphs carry the old launch parameters
  c->waves.clear();
  return FAME_OK;
}

int fame_get_option(fame_ctx* c, const char* name, int* value) {
  if (!c || !name || !value) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  const std::string n(name);
  if (n == "prefetch") {
    *value = c->prefetch;
  } else if (n == "self_prefetch") {
    *value = c->self_prefetch;
  } else if (n == "static_planes") {
    *value = c->static_planes;
  } else if (n == "lanes") {
    *value = c->lanes;
  } else if (n == "radix_order") {
    *value = c->radix_order;
  } else if (n == "plane_threads32") {
    *value = c->plane_threads32;
  } else if (n == "plane_threads64") {
    *value = c->plane_threads;
  } else if (n == "static96") {
    *value = c->stat96 ? 1 : 0;
  } else if (n == "general") {
    *value = c->g.general;
  } else if (n == "grid_x" || n == "grid_y" || n == "grid_z") {
    *value = n == "grid_x" ? c->g.Nx : n == "grid_y" ? c->g.Ny : c->g.Nz;
  } else if (n == "level") {
    *value = std::max(c->rare, c->rare_pen);
  } else if (n == "plan_signature") {
    // the radix lists of the three axis plans, hashed (equal plans, equal values)
    unsigned h = 2166136261u;
    for (const AxisPlan* a : {&c->g.pf, &c->g.pm, &c->g.ps})
      for (int i = 0; i < a->npass; i++) h = (h ^ (unsigned)a->radix[i]) * 16777619u;
    *value = (int)(h & 0x7fffffff);
  } else {
    set_err("unknown option: " + n);
    return FAME_ERR_BAD_INPUT;
  }
  return FAME_OK;
}

int fame_set_loop_cap(fame_ctx* c, int max_trips) {
  if (!c || max_trips < 0) {
    set_err("null context or negative loop cap");
    return FAME_ERR_BAD_INPUT;
  }
  c->loop_cap = max_trips;
  return FAME_OK;
}

int fame_launch_count(fame_ctx* c, unsigned long long* out) {
  if (!c || !out) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    FAME_CK(cudaStreamSynchronize(c->stream));
    *out = launches_solver() + launches_ops_f32_simple() + launches_ops_f32_general() + launches_ops_f64_simple() +
           launches_ops_f64_general() + launches_ops_f32_simple_rare() + launches_ops_f32_general_rare() +
           launches_ops_f64_simple_rare() + launches_ops_f64_general_rare() + launches_ops_f32_simple_prime() +
           launches_ops_f32_general_prime() + launches_ops_f64_simple_prime() + launches_ops_f64_general_prime() +
           launches_ops_stat96_f32() +
           launches_ops_stat96_f64() + launches_ops_slow_static() + launches_ops_plane_static() +
           launches_material_locate();
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

int fame_bench_qbq(fame_ctx* c, const double* k, int precision, int reps, int nbatch, double* ms_out,
                   double* stage_ms) {
  if (!c || !k || !ms_out || reps < 1 || nbatch < 1 || nbatch > 64 ||
      (precision != FAME_FP64 && precision != FAME_MIXED)) {
    set_err("bad argument");
    return FAME_ERR_BAD_INPUT;
  }
  if (!c->have_eps) {
    set_err("permittivity not set");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    ensure_workspace(c, nbatch, std::max(2, c->cap_nstep), std::max(1, c->cap_nwant), precision == FAME_MIXED,
                     c->cap_vec);
    const Slot sl = make_slot(c->lat, k);
    std::vector<Slot> hs(nbatch, sl);  // the same k-point in every slot of the batch
    FAME_CK(cudaMemcpyAsync(c->slots.p, hs.data(), nbatch * sizeof(Slot), cudaMemcpyHostToDevice, c->stream));
    Program P(c->stream, false, c->hflag, 1);
    Ops o{c, P, nbatch};
    const Geom& g = c->g;
    const long M = 2L * g.N, F = 3L * g.N;
    const int tmax = std::max({g.Nx * g.Ny, g.Nx, g.Ny, g.Nz});
    P.launch(k_tables, dim3((tmax + 255) / 256, nbatch), dim3(256), 0, g, (const Slot*)c->slots.p, c->tabs.p,
             (double)c->lat.m[0], (double)c->lat.m[1], (double)c->lat.m[2]);
    DBuf<unsigned char> flush;
    const size_t fl = 256ull << 20;
    flush.ensure(fl);
    cudaEvent_t ev[4];
    for (auto& e : ev) FAME_CK(cudaEventCreate(&e));
    double tot[3] = {0, 0, 0};
    // input: r64 / r32 hold arbitrary finite data after a memset
    if (precision == FAME_FP64)
      FAME_CK(cudaMemsetAsync(c->r64.p, 0, nbatch * M * sizeof(double2), c->stream));
    else
      FAME_CK(cudaMemsetAsync(c->r32.p, 0, nbatch * M * sizeof(float2), c->stream));
    for (int it = 0; it < reps + 1; it++) {
      FAME_CK(cudaMemsetAsync(flush.p, it & 0xff, fl, c->stream));
      FAME_CK(cudaEventRecord(ev[0], c->stream));
      if (precision == FAME_FP64) {
        o.plane_inv<double, IN_VEC, false>(c->r64.p, c->T64.p, 1, M, F, 0);
        FAME_CK(cudaEventRecord(ev[1], c->stream));
        o.pencil<double, PEN_QBQ>(c->T64.p, 1, F, c->ibq64(), 0);
        FAME_CK(cudaEventRecord(ev[2], c->stream));
        o.plane_fwd<double, EPI_OUT, false>(c->T64.p, c->x64.p, 1, M, F);
      } else {
        o.plane_inv<float, IN_VEC, false>(c->r32.p, c->T32.p, 1, M, F, 0);
        FAME_CK(cudaEventRecord(ev[1], c->stream));
        o.pencil<float, PEN_QBQ>(c->T32.p, 1, F, c->ibq32(), 0);
        FAME_CK(cudaEventRecord(ev[2], c->stream));
        o.plane_fwd<float, EPI_OUT, false>(c->T32.p, c->x32.p, 1, M, F);
      }
      FAME_CK(cudaEventRecord(ev[3], c->stream));
      FAME_CK(cudaEventSynchronize(ev[3]));
      if (it == 0) continue;  // warm-up
      for (int q = 0; q < 3; q++) {
        float ms = 0;
        FAME_CK(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
        tot[q] += ms;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    flush.release();
    *ms_out = (tot[0] + tot[1] + tot[2]) / reps;
    if (stage_ms)
      for (int q = 0; q < 3; q++) stage_ms[q] = tot[q] / reps;
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

int fame_bench_cg(fame_ctx* c, const double* k, int reps, int nbatch, double* ms_out, double* stage_ms) {
  if (!c || !k || !ms_out || reps < 1 || nbatch < 1 || nbatch > 64) {
    set_err("bad argument");
    return FAME_ERR_BAD_INPUT;
  }
  if (!c->have_eps) {
    set_err("permittivity not set");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    ensure_workspace(c, nbatch, std::max(2, c->cap_nstep), std::max(1, c->cap_nwant), true, c->cap_vec);
    const Slot sl = make_slot(c->lat, k);
    std::vector<Slot> hs(nbatch, sl);
    FAME_CK(cudaMemcpyAsync(c->slots.p, hs.data(), nbatch * sizeof(Slot), cudaMemcpyHostToDevice, c->stream));
    const Geom& g = c->g;
    const long M = 2L * g.N, F = 3L * g.N;
    // r: a fixed pseudo-random residual; p = x = 0; the first iteration takes p = r
    std::vector<float2> hr((size_t)nbatch * M);
    unsigned long long z = 0x9e3779b97f4a7c15ull;
    for (auto& v : hr) {
      z = z * 6364136223846793005ull + 1442695040888963407ull;
      v.x = (float)((double)(z >> 11) / 9007199254740992.0 - 0.5);
      z = z * 6364136223846793005ull + 1442695040888963407ull;
      v.y = (float)((double)(z >> 11) / 9007199254740992.0 - 0.5);
    }
    FAME_CK(cudaMemcpyAsync(c->r32.p, hr.data(), hr.size() * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    FAME_CK(cudaMemsetAsync(c->x32.p, 0, (size_t)nbatch * M * sizeof(float2), c->stream));
    FAME_CK(cudaMemsetAsync(c->p32.p, 0, (size_t)nbatch * M * sizeof(float2), c->stream));
    std::vector<CgState> cs(nbatch);
    for (auto& s : cs) {
      memset(&s, 0, sizeof(s));
      s.iter = 1;
      s.active = 1;
      s.maxit = 1 << 30;
      s.r1 = 1.0;
      s.tol2 = 0.0;
    }
    FAME_CK(cudaMemcpyAsync(c->cg.p, cs.data(), nbatch * sizeof(CgState), cudaMemcpyHostToDevice, c->stream));
    Program P(c->stream, false, c->hflag, 1);
    Ops o{c, P, nbatch};
    const int tmax = std::max({g.Nx * g.Ny, g.Nx, g.Ny, g.Nz});
    P.launch(k_tables, dim3((tmax + 255) / 256, nbatch), dim3(256), 0, g, (const Slot*)c->slots.p, c->tabs.p,
             (double)c->lat.m[0], (double)c->lat.m[1], (double)c->lat.m[2]);
    DBuf<unsigned char> flush;
    const size_t fl = 256ull << 20;
    flush.ensure(fl);
    cudaEvent_t ev[4];
    for (auto& e : ev) FAME_CK(cudaEventCreate(&e));
    double tot[3] = {0, 0, 0};
    for (int it = 0; it < reps + 1; it++) {
      FAME_CK(cudaMemsetAsync(flush.p, it & 0xff, fl, c->stream));
      FAME_CK(cudaEventRecord(ev[0], c->stream));
      o.plane_inv<float, IN_CG, false>(nullptr, c->T32.p, 1, M, F, 0, c->p32.p, c->r32.p, nullptr, nullptr, Cond{},
                                       c->x32.p);
      FAME_CK(cudaEventRecord(ev[1], c->stream));
      o.pencil<float, PEN_QBQ_CG>(c->T32.p, 1, F, c->ibq32(), 1);
      FAME_CK(cudaEventRecord(ev[2], c->stream));
      o.plane_fwd<float, EPI_CGR, false>(c->T32.p, nullptr, 1, M, F, nullptr, nullptr, Cond{}, 0.0, c->r32.p);
      o.cg_decide(Cond{});
      FAME_CK(cudaEventRecord(ev[3], c->stream));
      FAME_CK(cudaEventSynchronize(ev[3]));
      if (it == 0) continue;  // warm-up (the p = r iteration)
      for (int q = 0; q < 3; q++) {
        float ms = 0;
        FAME_CK(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
        tot[q] += ms;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    flush.release();
    *ms_out = (tot[0] + tot[1] + tot[2]) / reps;
    if (stage_ms)
      for (int q = 0; q < 3; q++) stage_ms[q] = tot[q] / reps;
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

int fame_set_eps_device(fame_ctx* c, const double* B) {
  if (!c || !B) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    c->eps_bad.ensure(2);
    const int init[2] = {0, 0x7fffffff};
    FAME_CK(cudaMemcpyAsync(c->eps_bad.p, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
    const Geom& g = c->g;
    const int blocks = (int)std::min<long>(4096, (3L * g.N + 255) / 256);
    k_eps_device<<<blocks, 256, 0, c->stream>>>(g, B, 0, c->eps_bad.p, nullptr, nullptr, nullptr, nullptr, nullptr);
    FAME_CK(cudaGetLastError());
    int bad[2];
    FAME_CK(cudaMemcpyAsync(bad, c->eps_bad.p, sizeof(bad), cudaMemcpyDeviceToHost, c->stream));
    FAME_CK(cudaStreamSynchronize(c->stream));
    if (bad[0]) {
      set_err("permittivity must be finite and positive (" + std::to_string(bad[0]) + " edges, first " +
              std::to_string(bad[1]) + ")");
      return FAME_ERR_BAD_INPUT;
    }
    k_eps_device<<<blocks, 256, 0, c->stream>>>(g, B, 1, c->eps_bad.p, c->B64.p, c->invB64.p, c->invB32.p,
                                                  c->invB64q.p, c->invB32q.p);
    FAME_CK(cudaGetLastError());
    FAME_CK(cudaStreamSynchronize(c->stream));
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  c->have_eps = true;
  c->eps_ver++;
  return FAME_OK;
}

int fame_adjoint_vjp(fame_ctx* c, int kidx, const double* freq, const double* grad_w, int nwant, double rel_gap,
                     double* grad_dev) {
  if (!c || !freq || !grad_w || !grad_dev || nwant < 1 || nwant > 64 || !(rel_gap >= 0)) {
    set_err("null argument, nwant outside 1..64 or negative gap");
    return FAME_ERR_BAD_INPUT;
  }
  if (kidx < 0 || kidx >= c->dev_vec_nk || nwant != c->dev_vec_nwant) {
    set_err("no eigenvectors of this k-point on the device (solve with want_vectors and evec_out NULL first)");
    return FAME_ERR_BAD_INPUT;
  }
  // degenerate groups: a derivative of one band of a group is not defined, the sum
  // over the group is; so the weights of a group's bands must be equal
  double gmax = 0;
  for (int i = 0; i < nwant; i++) gmax = std::max(gmax, fabs(grad_w[i]));
  for (int i = 0; i < nwant; i++)
    for (int j = i + 1; j < nwant; j++) {
      const double wi = freq[i], wj = freq[j];
      if (wi <= 0 || wj <= 0) continue;
      if (fabs(wi - wj) <= rel_gap * std::max(wi, wj) && fabs(grad_w[i] - grad_w[j]) > 1e-12 * gmax) {
        set_err("bands " + std::to_string(i) + " and " + std::to_string(j) +
                " are degenerate (relative gap below " + std::to_string(rel_gap) +
                ") but weighted differently; the derivative of one band of a degenerate group is not defined, "
                "weight the whole group equally");
        return FAME_ERR_BAD_INPUT;
      }
    }
  try {
    FAME_CK(cudaSetDevice(c->device));
    const long N = c->g.N;
    const int gamma = c->dev_vec_gamma[kidx];
    const int first = gamma ? 2 : 0;
    const int nvec = nwant - first;
    const double2* E = c->E.p + (size_t)kidx * nwant * 3 * N;
    c->adj.ensure(3 * 64);
    std::vector<double> wg(2 * nwant);
    for (int i = 0; i < nwant; i++) {
      wg[i] = freq[i];
      wg[nwant + i] = grad_w[i];
    }
    FAME_CK(cudaMemcpyAsync(c->adj.p, wg.data(), wg.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (nvec > 0) {
      c->adj_part.ensure((size_t)nvec * kBandSplit);
      k_adj_den<<<dim3(kBandSplit, nvec), 256, 0, c->stream>>>(E, c->B64.p, 3 * N, c->adj_part.p);
      FAME_CK(cudaGetLastError());
      k_rows_sum<<<nvec, 32, 0, c->stream>>>(nullptr, nvec, c->adj_part.p, kBandSplit, 1, c->adj.p + 2 * nwant);
      FAME_CK(cudaGetLastError());
    }
    k_adj_vjp<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(E, c->adj.p, nwant, first, N, grad_dev);
    FAME_CK(cudaGetLastError());
    FAME_CK(cudaStreamSynchronize(c->stream));
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

int fame_adjoint(fame_ctx* c, const double* freq, const double* evec, int nwant, int host, double* grad_out) {
  if (!c || !freq || !evec || !grad_out || nwant < 1) {
    set_err("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  if (!c->have_eps) {
    set_err("permittivity not set");
    return FAME_ERR_BAD_INPUT;
  }
  try {
    FAME_CK(cudaSetDevice(c->device));
    const long N = c->g.N;
    const double2* E = reinterpret_cast<const double2*>(evec);
    DBuf<double2> tmp;
    if (host) {
      tmp.ensure((size_t)nwant * 3 * N);
      FAME_CK(cudaMemcpyAsync(tmp.p, evec, (size_t)nwant * 3 * N * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
      E = tmp.p;
    }
    DBuf<double> w, den, grad;
    w.ensure(nwant);
    den.ensure(nwant);
    grad.ensure((size_t)nwant * N);
    FAME_CK(cudaMemcpyAsync(w.p, freq, nwant * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->adj_part.ensure((size_t)nwant * kBandSplit);
    k_adj_den<<<dim3(kBandSplit, nwant), 256, 0, c->stream>>>(E, c->B64.p, 3 * N, c->adj_part.p);
    FAME_CK(cudaGetLastError());
    k_rows_sum<<<nwant, 32, 0, c->stream>>>(nullptr, nwant, c->adj_part.p, kBandSplit, 1, den.p);
    FAME_CK(cudaGetLastError());
    k_adj_grad<<<dim3((unsigned)((N + 255) / 256), nwant), 256, 0, c->stream>>>(E, w.p, den.p, N, grad.p);
    FAME_CK(cudaGetLastError());
    FAME_CK(cudaMemcpyAsync(grad_out, grad.p, (size_t)nwant * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FAME_CK(cudaStreamSynchronize(c->stream));
    tmp.release();
    w.release();
    den.release();
    grad.release();
  } catch (const CudaError& e) {
    set_err(e.what());
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

}  // extern "C"
