// fame_qbq_static: Q_r^* B^{-1} Q_r in FP64 with no device allocation.
//
// Callers that cannot allocate device memory use this entry point: a host
// framework that owns the whole device budget through its own pool (the
// reference's FAME_Main_Code allocates its work arrays up front), and code that
// runs where cudaMalloc is not allowed or must not block other streams (cudaMalloc
// and cudaFree synchronise the device).  It needs no fame_ctx, whose creation
// allocates the twiddle, table and workspace buffers of the solver.
//
// Scratch: one file-scope device array of kScratchBytes (4 MiB).  A call lays out
// in it the k-point slot, the FFT twiddles, the Lambda/D_k tables and the
// 3-component intermediate field T (3N complex doubles, 48 B per grid point), so
// grids up to about 85,000 points fit; larger grids are rejected with
// FAME_ERR_UNSUPPORTED and a message giving the bytes needed.
//
// Sharing: every call on every stream of a device uses the same array, and the
// array keeps what the last call left in it.  Nothing in it has to start at zero:
// each call writes the slot, twiddles, tables and T before any kernel reads them.
// Two calls that may overlap in time (different streams, or different host threads
// on one stream without ordering) race on the array; the caller serialises them.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's address with cudaGetSymbolAddress (once per device, checked; the address
// is cached).  Make that first call before any stream capture.  Every call also
// sets the dynamic shared-memory limit of the stage kernels it launches
// (cudaFuncSetAttribute, which allocates nothing).
//
// Errors are reported by the return code and the text of fame_last_error().
//
// The computation is the one of fame_apply(FAME_OP_QBQ, FAME_FP64): the same
// plane / pencil / plane kernels and the same table kernel, launched on the
// caller's stream; only where their scratch lives differs.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/fame_b200.h"
#include "geometry.h"
#include "op_kernels_decl.h"

namespace fame {

// defined with the solver (solver_kernels.cuh, solver.cu)
__global__ void k_tables(Geom g, const Slot* slots, double2* tabs, double m1, double m2, double m3);
void set_last_error(const std::string& s);

namespace {

constexpr size_t kScratchBytes = FAME_QBQ_STATIC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_qbq_scratch[kScratchBytes];

// per-device set-up: address of the scratch array
std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices];

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// The slot and the forward twiddles e^{-2 pi i m / n} of the three axes.
__global__ void k_static_prep(Slot sl, Geom g, Slot* slot, double2* tw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *slot = sl;
  const int n[3] = {g.Lf, g.Lm, g.Ls};
  const int o[3] = {g.twf, g.twm, g.tws};
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (i < n[a]) {
      double s, c;
      sincospi(2.0 * i / n[a], &s, &c);
      tw[o[a] + i] = make_double2(c, -s);
    }
}

template <typename K> cudaError_t raise_smem(K* k, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <bool GEN, int RARE>
cudaError_t launch_qbq(const Geom& g, int threads, const Slot* slot, const double2* tabs, const double2* tw,
                       const double2* x, const double* invB, double2* T, double2* y, cudaStream_t st) {
  const long M = 2L * g.N, F = 3L * g.N;
  auto kin = k_plane_inv<double, GEN, IN_VEC, false, RARE, DynGeom>;
  auto kpen = k_pencil<double, GEN, PEN_QBQ, RARE, DynGeom>;
  auto kout = k_plane_fwd<double, GEN, EPI_OUT, false, RARE, DynGeom>;
  const size_t sm_plane = plane_smem_bytes<double>(g.Lf, g.Lm, g.S);
  const int TW = PencilTW<double>::v;
  const size_t sm_pen = pencil_smem_bytes<double>(g.Ls);
  cudaError_t e;
  if ((e = raise_smem(kin, sm_plane)) != cudaSuccess) return e;
  if ((e = raise_smem(kpen, sm_pen)) != cudaSuccess) return e;
  if ((e = raise_smem(kout, sm_plane)) != cudaSuccess) return e;

  PlaneInArgs<double> ai;
  memset(&ai, 0, sizeof(ai));
  ai.g = g;
  ai.slots = slot;
  ai.tabs = tabs;
  ai.tw = tw;
  ai.vstride = M;
  ai.fstride = F;
  ai.vec_per_slot = 1;
  ai.in = x;
  ai.T = T;
  kin<<<dim3(3 * g.Ls, 1, 1), dim3(threads), sm_plane, st>>>(ai);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;

  PencilArgs<double> ap;
  memset(&ap, 0, sizeof(ap));
  ap.g = g;
  ap.slots = slot;
  ap.tabs = tabs;
  ap.tw = tw;
  ap.fstride = F;
  ap.vec_per_slot = 1;
  ap.T = T;
  ap.invB = invB;
  ap.ib_field = 0;  // the caller's 1/eps is in the spatial layout
  ap.nslots = 1;
  ap.TW = TW;
  const int nft = (g.Lf + TW - 1) / TW;
  kpen<<<dim3(g.Lm * nft, 3, 1), dim3(kPencilThreads), sm_pen, st>>>(ap);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;

  PlaneOutArgs<double> ao;
  memset(&ao, 0, sizeof(ao));
  ao.g = g;
  ao.slots = slot;
  ao.tabs = tabs;
  ao.tw = tw;
  ao.vstride = M;
  ao.fstride = F;
  ao.vec_per_slot = 1;
  ao.T = T;
  ao.out = y;
  ao.nslots = 1;
  kout<<<dim3(3 * g.Ls, 1, 1), dim3(threads), sm_plane, st>>>(ao);
  return cudaGetLastError();
}

}  // namespace
}  // namespace fame

using namespace fame;

extern "C" {

int fame_qbq_static(const fame_lattice* lat, const double* k, const double* inv_b, const void* x, void* y,
                    void* stream) {
  if (!lat || !k || !inv_b || !x || !y) {
    set_last_error("null argument");
    return FAME_ERR_BAD_INPUT;
  }
  Geom g;
  std::string err;
  const int rc = layout_geom(*lat, g, 1L << 24, err);
  if (rc != FAME_OK) {
    set_last_error(err);
    return rc;
  }
  const int rare = geom_level(g);
  const int threads = plane_threads_rule<double>(g, rare);
  const size_t off_tw = align256(sizeof(Slot));
  const size_t off_tab = off_tw + align256(sizeof(double2) * (size_t)(g.Lf + g.Lm + g.Ls));
  const size_t off_T = off_tab + align256(sizeof(double2) * (size_t)g.tab_stride);
  const size_t need = off_T + sizeof(double2) * 3 * (size_t)g.N;
  if (need > kScratchBytes) {
    set_last_error("grid of " + std::to_string(g.N) + " points needs " + std::to_string(need) +
            " bytes of scratch; the static array holds " + std::to_string(kScratchBytes));
    return FAME_ERR_UNSUPPORTED;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_last_error(std::string("cudaGetDevice: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "device index out of range"));
    return FAME_ERR_CUDA;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_qbq_scratch);
      if (e != cudaSuccess) {
        set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return FAME_ERR_CUDA;
      }
      g_scratch_ptr[dev] = p;
    }
    base = (unsigned char*)g_scratch_ptr[dev];
  }
  const Slot sl = make_slot(*lat, k);
  Slot* slot = (Slot*)base;
  double2* tw = (double2*)(base + off_tw);
  double2* tabs = (double2*)(base + off_tab);
  double2* T = (double2*)(base + off_T);
  cudaStream_t st = (cudaStream_t)stream;

  const int nprep = std::max({g.Lf, g.Lm, g.Ls, 1});
  k_static_prep<<<(nprep + 255) / 256, 256, 0, st>>>(sl, g, slot, tw);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    set_last_error(std::string("prep launch: ") + cudaGetErrorString(e));
    return FAME_ERR_CUDA;
  }
  const int tmax = std::max({g.Nx * g.Ny, g.Nx, g.Ny, g.Nz});
  k_tables<<<dim3((tmax + 255) / 256, 1), dim3(256), 0, st>>>(g, slot, tabs, (double)lat->m[0], (double)lat->m[1],
                                                              (double)lat->m[2]);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    set_last_error(std::string("table launch: ") + cudaGetErrorString(e));
    return FAME_ERR_CUDA;
  }
  const double2* xd = (const double2*)x;
  double2* yd = (double2*)y;
  if (g.general)
    e = rare == 2   ? launch_qbq<true, 2>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st)
        : rare == 1 ? launch_qbq<true, 1>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st)
                    : launch_qbq<true, 0>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st);
  else
    e = rare == 2   ? launch_qbq<false, 2>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st)
        : rare == 1 ? launch_qbq<false, 1>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st)
                    : launch_qbq<false, 0>(g, threads, slot, tabs, tw, xd, inv_b, T, yd, st);
  if (e != cudaSuccess) {
    set_last_error(std::string("QBQ launch: ") + cudaGetErrorString(e));
    return FAME_ERR_CUDA;
  }
  return FAME_OK;
}

}  // extern "C"
