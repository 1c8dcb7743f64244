// fame_material_locate: the material index map Binout on the GPU, bit-exact.
//
// Reference: FAME_Preprocessing/FAME_Material_Locate_Index.cpp:6-113 (fold each Yee
// edge point into the unit cell of the original lattice), FAME_Material_Handle.cpp:4-87
// (spheres and cylinders over the 27 neighbouring cell images; the first material
// with a hit wins) and FAME_Matrix_Grid.cpp:4-53 (edge point (i + s_x, j + s_y,
// k + s_z) * h with s = 1/2 along the edge's own axis).  The reference runs this on one
// CPU core inside its preprocessing.
//
// Bit-exactness: every product, sum and quotient is an explicit round-to-nearest
// double intrinsic in the reference's operation order, so nothing is contracted into
// a fused multiply-add (the reference's x86-64 build has none) and floor() sees the
// same coefficients; pow(x, 2) of the reference is the correctly rounded square x*x.
// The lattice matrices (Omega' a, its inverse by the adjugate formula of
// FAME_Tools/inv3.cpp:8-23, and the permuted basis) are formed the same way by one
// thread on the device.
#include <cuda_runtime.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/fame_b200.h"
#include "fame_common.cuh"

namespace fame {

void set_last_error(const std::string& s);

namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double sq(double a) { return __dmul_rn(a, a); }
// x*a0 + y*a1 + z*a2, summed left to right
__device__ __forceinline__ double dot3(double x, double a0, double y, double a1, double z, double a2) {
  return add(add(mul(x, a0), mul(y, a1)), mul(z, a2));
}

struct LocGeom {
  double AP[9];     // lattice_vec_a_orig_P = Omega' * lattice_vec_a (…Locate_Index.cpp:44-52)
  double invAP[9];  // inv3(AP)
  double A[9];      // lattice_vec_a_orig: AP with its columns permuted back (:54-83)
};

// One thread: the lattice matrices of FAME_Material_Locate_Index_Print.
__global__ void k_locate_setup(const double* Om, const double* a, const int* perm, LocGeom* out) {
  if (threadIdx.x | blockIdx.x) return;
  LocGeom G;
  int cnt = 0;
  for (int i = 0; i < 3; i++) {
    G.AP[i] = dot3(Om[cnt], a[0], Om[cnt + 1], a[1], Om[cnt + 2], a[2]);
    G.AP[i + 3] = dot3(Om[cnt], a[3], Om[cnt + 1], a[4], Om[cnt + 2], a[5]);
    G.AP[i + 6] = dot3(Om[cnt], a[6], Om[cnt + 1], a[7], Om[cnt + 2], a[8]);
    cnt += 3;
  }
  const double* A = G.AP;
  const double det = add(sub(mul(A[0], sub(mul(A[4], A[8]), mul(A[5], A[7]))),
                             mul(A[3], sub(mul(A[1], A[8]), mul(A[7], A[2])))),
                         mul(A[6], sub(mul(A[1], A[5]), mul(A[4], A[2]))));
  const double inv = __ddiv_rn(1.0, det);
  G.invAP[0] = mul(sub(mul(A[4], A[8]), mul(A[5], A[7])), inv);
  G.invAP[1] = mul(-sub(mul(A[1], A[8]), mul(A[2], A[7])), inv);
  G.invAP[2] = mul(sub(mul(A[1], A[5]), mul(A[2], A[4])), inv);
  G.invAP[3] = mul(-sub(mul(A[3], A[8]), mul(A[6], A[5])), inv);
  G.invAP[4] = mul(sub(mul(A[0], A[8]), mul(A[6], A[2])), inv);
  G.invAP[5] = mul(-sub(mul(A[0], A[5]), mul(A[2], A[3])), inv);
  G.invAP[6] = mul(sub(mul(A[3], A[7]), mul(A[6], A[4])), inv);
  G.invAP[7] = mul(-sub(mul(A[0], A[7]), mul(A[1], A[6])), inv);
  G.invAP[8] = mul(sub(mul(A[0], A[4]), mul(A[1], A[3])), inv);
  int invP[3] = {perm[0], perm[1], perm[2]};
  if (perm[0] == 2 && perm[1] == 3 && perm[2] == 1) {
    invP[0] = 3; invP[1] = 1; invP[2] = 2;
  } else if (perm[0] == 3 && perm[1] == 1 && perm[2] == 2) {
    invP[0] = 2; invP[1] = 3; invP[2] = 1;
  }
  for (int q = 0; q < 3; q++)
    for (int c = 0; c < 3; c++) G.A[3 * q + c] = G.AP[(invP[q] - 1) * 3 + c];
  *out = G;
}

// Image centres of every shape, the same for all points (sphere_handle /
// cylinder_handle compute them inside the point loop): per (shape, shift) a sphere
// stores (cx, cy, cz, r^2) and a cylinder (tx, ty, tz, bx-tx, by-ty, bz-tz, den, r^2).
constexpr int kSph = 4, kCyl = 8;

__global__ void k_locate_shapes(const LocGeom* G, int ns, const double* sc, const double* sr, int nc,
                                const double* tc, const double* bc, const double* cr, double* stab,
                                double* ctab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double* A = G->A;
  if (t < ns * 27) {
    const int i = t / 27, s = t % 27;
    const double sx = s / 9 - 1, sy = (s / 3) % 3 - 1, sz = s % 3 - 1;
    const double u = add(sc[3 * i], sx), v = add(sc[3 * i + 1], sy), w = add(sc[3 * i + 2], sz);
    double* o = stab + (size_t)t * kSph;
    o[0] = dot3(u, A[0], v, A[3], w, A[6]);
    o[1] = dot3(u, A[1], v, A[4], w, A[7]);
    o[2] = dot3(u, A[2], v, A[5], w, A[8]);
    o[3] = sq(sr[i]);
  } else if (t < ns * 27 + nc * 27) {
    const int t2 = t - ns * 27, i = t2 / 27, s = t2 % 27;
    const double sx = s / 9 - 1, sy = (s / 3) % 3 - 1, sz = s % 3 - 1;
    double u = add(tc[3 * i], sx), v = add(tc[3 * i + 1], sy), w = add(tc[3 * i + 2], sz);
    const double tx = dot3(u, A[0], v, A[3], w, A[6]);
    const double ty = dot3(u, A[1], v, A[4], w, A[7]);
    const double tz = dot3(u, A[2], v, A[5], w, A[8]);
    u = add(bc[3 * i], sx);
    v = add(bc[3 * i + 1], sy);
    w = add(bc[3 * i + 2], sz);
    const double bx = dot3(u, A[0], v, A[3], w, A[6]);
    const double by = dot3(u, A[1], v, A[4], w, A[7]);
    const double bz = dot3(u, A[2], v, A[5], w, A[8]);
    double* o = ctab + (size_t)t2 * kCyl;
    o[0] = tx;
    o[1] = ty;
    o[2] = tz;
    o[3] = sub(bx, tx);
    o[4] = sub(by, ty);
    o[5] = sub(bz, tz);
    o[6] = add(add(sq(o[3]), sq(o[4])), sq(o[5]));
    o[7] = sq(cr[i]);
  }
}

struct LocArgs {
  int Nx, Ny, Nz, N;
  double h[3];
  double Om[9];
  int nm;                      // material_num
  const int* sph_first;        // [nm + 1] first sphere of each material
  const int* cyl_first;        // [nm + 1]
  const double* stab;
  const double* ctab;
  const LocGeom* G;
  int* binout;                 // [3][nm][N]
};

// One thread per (edge component, grid point).
__global__ void __launch_bounds__(256) k_locate(LocArgs a) {
  FAME_COUNT_LAUNCH();
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3L * a.N) return;
  const int comp = (int)(t / a.N);
  const int idx = (int)(t - (long)comp * a.N);
  const int i = idx % a.Nx, j = (idx / a.Nx) % a.Ny, k = idx / (a.Nx * a.Ny);
  // FAME_Matrix_Grid: (index + shift) * mesh_len, shift 1/2 on the edge's own axis
  const double p0 = mul(add((double)i, comp == 0 ? 0.5 : 0.0), a.h[0]);
  const double p1 = mul(add((double)j, comp == 1 ? 0.5 : 0.0), a.h[1]);
  const double p2 = mul(add((double)k, comp == 2 ? 0.5 : 0.0), a.h[2]);
  const double* Om = a.Om;
  const LocGeom& G = *a.G;
  // FAME_Material_Locate: to the original frame, coefficients, fold into the cell
  const double o0 = dot3(p0, Om[0], p1, Om[1], p2, Om[2]);
  const double o1 = dot3(p0, Om[3], p1, Om[4], p2, Om[5]);
  const double o2 = dot3(p0, Om[6], p1, Om[7], p2, Om[8]);
  const double c0 = dot3(o0, G.invAP[0], o1, G.invAP[3], o2, G.invAP[6]);
  const double c1 = dot3(o0, G.invAP[1], o1, G.invAP[4], o2, G.invAP[7]);
  const double c2 = dot3(o0, G.invAP[2], o1, G.invAP[5], o2, G.invAP[8]);
  const double s1 = floor(c0), s2 = floor(c1), s3 = floor(c2);
  const double* AP = G.AP;
  const double px = sub(o0, dot3(s1, AP[0], s2, AP[3], s3, AP[6]));
  const double py = sub(o1, dot3(s1, AP[1], s2, AP[4], s3, AP[7]));
  const double pz = sub(o2, dot3(s1, AP[2], s2, AP[5], s3, AP[8]));
  // FAME_Material_Handle: first material whose spheres or cylinders contain the point
  int hit = -1;
  for (int m = 0; m < a.nm && hit < 0; m++) {
    bool in = false;
    for (int q = a.sph_first[m] * 27; q < a.sph_first[m + 1] * 27 && !in; q++) {
      const double* s = a.stab + (size_t)q * kSph;
      const double d = add(add(sq(sub(s[0], px)), sq(sub(s[1], py))), sq(sub(s[2], pz)));
      in = d <= s[3];
    }
    for (int q = a.cyl_first[m] * 27; q < a.cyl_first[m + 1] * 27 && !in; q++) {
      const double* c = a.ctab + (size_t)q * kCyl;
      const double num = add(add(mul(sub(px, c[0]), c[3]), mul(sub(py, c[1]), c[4])), mul(sub(pz, c[2]), c[5]));
      const double tt = __ddiv_rn(num, c[6]);
      if (0.0 <= tt && tt <= 1.0) {
        const double d = add(add(sq(sub(add(c[0], mul(tt, c[3])), px)), sq(sub(add(c[1], mul(tt, c[4])), py))),
                             sq(sub(add(c[2], mul(tt, c[5])), pz)));
        in = d <= c[7];
      }
    }
    if (in) hit = m;
  }
  int* out = a.binout + (size_t)comp * a.nm * a.N + idx;
  for (int m = 0; m < a.nm; m++) out[(size_t)m * a.N] = (m == hit);
}

template <typename T> struct DevArray {
  T* p = nullptr;
  cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, (n ? n : 1) * sizeof(T)); }
  ~DevArray() {
    if (p) cudaFree(p);
  }
};

}  // namespace

FAME_DEFINE_LAUNCH_GETTER(launches_material_locate)

}  // namespace fame

using namespace fame;

extern "C" int fame_material_locate(int device, const fame_locate_geometry* geo, const fame_material_shapes* mat,
                                    int* binout) {
  if (!geo || !mat || !binout || mat->material_num < 1) {
    set_last_error("null argument or no material");
    return FAME_ERR_BAD_INPUT;
  }
  const int Nx = geo->grid[0], Ny = geo->grid[1], Nz = geo->grid[2], nm = mat->material_num;
  if (Nx < 1 || Ny < 1 || Nz < 1 || (long)Nx * Ny * Nz > (1L << 28)) {
    set_last_error("bad grid");
    return FAME_ERR_BAD_INPUT;
  }
  const int N = Nx * Ny * Nz;
  std::vector<int> sf(nm + 1, 0), cf(nm + 1, 0);
  for (int m = 0; m < nm; m++) {
    const int ns = mat->sphere_num ? mat->sphere_num[m] : 0, nc = mat->cylinder_num ? mat->cylinder_num[m] : 0;
    if (ns < 0 || nc < 0) {
      set_last_error("negative shape count");
      return FAME_ERR_BAD_INPUT;
    }
    sf[m + 1] = sf[m] + ns;
    cf[m + 1] = cf[m] + nc;
  }
  const int ns = sf[nm], nc = cf[nm];
  if ((ns && (!mat->sphere_centers || !mat->sphere_radius)) ||
      (nc && (!mat->cylinder_top_centers || !mat->cylinder_bot_centers || !mat->cylinder_radius))) {
    set_last_error("shape arrays missing");
    return FAME_ERR_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_last_error("no CUDA device");
    return FAME_ERR_NO_DEVICE;
  }
  cudaError_t e = cudaSetDevice(device);
  auto ck = [&](cudaError_t r, const char* what) {
    if (r != cudaSuccess && e == cudaSuccess) {
      e = r;
      set_last_error(std::string(what) + ": " + cudaGetErrorString(r));
    }
    return e == cudaSuccess;
  };
  if (!ck(e, "cudaSetDevice")) return FAME_ERR_CUDA;
  DevArray<double> dOm, da, dsc, dsr, dtc, dbc, dcr, dst, dct;
  DevArray<int> dperm, dsf, dcf, dout;
  DevArray<LocGeom> dG;
  const size_t nout = 3 * (size_t)nm * N;
  bool ok = ck(dOm.alloc(9), "cudaMalloc") && ck(da.alloc(9), "cudaMalloc") && ck(dperm.alloc(3), "cudaMalloc") &&
            ck(dsc.alloc(3 * ns), "cudaMalloc") && ck(dsr.alloc(ns), "cudaMalloc") &&
            ck(dtc.alloc(3 * nc), "cudaMalloc") && ck(dbc.alloc(3 * nc), "cudaMalloc") &&
            ck(dcr.alloc(nc), "cudaMalloc") && ck(dst.alloc(27 * (size_t)ns * kSph), "cudaMalloc") &&
            ck(dct.alloc(27 * (size_t)nc * kCyl), "cudaMalloc") && ck(dsf.alloc(nm + 1), "cudaMalloc") &&
            ck(dcf.alloc(nm + 1), "cudaMalloc") && ck(dout.alloc(nout), "cudaMalloc") && ck(dG.alloc(1), "cudaMalloc");
  if (!ok) return FAME_ERR_CUDA;
  const auto H2D = cudaMemcpyHostToDevice;
  ok = ck(cudaMemcpy(dOm.p, geo->Omega, 9 * sizeof(double), H2D), "cudaMemcpy") &&
       ck(cudaMemcpy(da.p, geo->lattice_vec_a, 9 * sizeof(double), H2D), "cudaMemcpy") &&
       ck(cudaMemcpy(dperm.p, geo->permutation, 3 * sizeof(int), H2D), "cudaMemcpy") &&
       ck(cudaMemcpy(dsf.p, sf.data(), (nm + 1) * sizeof(int), H2D), "cudaMemcpy") &&
       ck(cudaMemcpy(dcf.p, cf.data(), (nm + 1) * sizeof(int), H2D), "cudaMemcpy");
  if (ok && ns)
    ok = ck(cudaMemcpy(dsc.p, mat->sphere_centers, 3 * ns * sizeof(double), H2D), "cudaMemcpy") &&
         ck(cudaMemcpy(dsr.p, mat->sphere_radius, ns * sizeof(double), H2D), "cudaMemcpy");
  if (ok && nc)
    ok = ck(cudaMemcpy(dtc.p, mat->cylinder_top_centers, 3 * nc * sizeof(double), H2D), "cudaMemcpy") &&
         ck(cudaMemcpy(dbc.p, mat->cylinder_bot_centers, 3 * nc * sizeof(double), H2D), "cudaMemcpy") &&
         ck(cudaMemcpy(dcr.p, mat->cylinder_radius, nc * sizeof(double), H2D), "cudaMemcpy");
  if (!ok) return FAME_ERR_CUDA;
  k_locate_setup<<<1, 32>>>(dOm.p, da.p, dperm.p, dG.p);
  const int nsh = 27 * (ns + nc);
  if (nsh) k_locate_shapes<<<(nsh + 127) / 128, 128>>>(dG.p, ns, dsc.p, dsr.p, nc, dtc.p, dbc.p, dcr.p, dst.p, dct.p);
  LocArgs a;
  a.Nx = Nx;
  a.Ny = Ny;
  a.Nz = Nz;
  a.N = N;
  memcpy(a.h, geo->mesh_len, sizeof(a.h));
  memcpy(a.Om, geo->Omega, sizeof(a.Om));
  a.nm = nm;
  a.sph_first = dsf.p;
  a.cyl_first = dcf.p;
  a.stab = dst.p;
  a.ctab = dct.p;
  a.G = dG.p;
  a.binout = dout.p;
  const long nt = 3L * N;
  k_locate<<<(unsigned)((nt + 255) / 256), 256>>>(a);
  ok = ck(cudaGetLastError(), "k_locate launch") &&
       ck(cudaMemcpy(binout, dout.p, nout * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
  return ok ? FAME_OK : FAME_ERR_CUDA;
}
