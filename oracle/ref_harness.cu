// Test-infrastructure driver for the UNMODIFIED reference build (oracle/_ref).
//
// It is linked against the reference's own objects (every .o except Main.o) and
// calls only the reference's public functions, in the order FAME_Main_Code uses
// them (FAME_Main/FAME_Main_Code.cu:37-140), minus the CPU self-checks
// (Check_Eigendecomp / Check_Residual), so that a run measures the solver alone.
// It never runs in the product path: it produces golden fixtures and serves as
// the reference arm of bench.py.
//
// Modes (workdir holds Popt.txt and FAME_Material_Data/<name>.txt, as Main.out
// expects, FAME_Preprocessing/FAME_Set_User_Option.cpp:10):
//   fame_ref_harness pre   <workdir> <out.bin>            preprocessing only (CPU)
//   fame_ref_harness solve <workdir> <out.jsonl> [--k kfile] [--eps epsfile]
//                          [--kidx i,j,..] [--evec prefix]
//   fame_ref_harness apply <workdir> <in.bin> <out.bin> [--k kfile] [--eps epsfile]
//
// kfile: text, first line nk, then nk lines "kx ky kz" (Cartesian WaveVector, the
// reference's convention without 2*pi, FAME_Matrix_Lambdas.cu:43-45).
// epsfile: raw little-endian float64, 3N edge permittivities B (x, y, z blocks).
#include "FAME_Internal_Common.h"
#include "FAME_CUDA.h"
#include "FAME_Preprocessing.h"
#include "FAME_Create_cublas.cuh"
#include "FAME_Create_Buffer.cuh"
#include "FAME_Matrix_B_Isotropic.cuh"
#include "FAME_Matrix_Lambdas.cuh"
#include "FAME_Profile.h"
#include "FAME_Matrix_Vector_Production_Qr.cuh"
#include "FAME_Matrix_Vector_Production_Qrs.cuh"
#include "FAME_Matrix_Vector_Production_Isotropic_QBQ.cuh"
#include "FAME_Matrix_Vector_Production_Isotropic_invAr.cuh"
#include <unistd.h>
#include <time.h>
#include <string>
#include <vector>

void FAME_Fast_Algorithms_Driver(double* Freq_array, cmpx* Ele_field_mtx, CULIB_HANDLES cuHandles,
                                 LANCZOS_BUFFER lBuffer, FFT_BUFFER fft_buffer,
                                 LAMBDAS_CUDA Lambdas_cuda, MTX_B mtx_B, ES es, LS ls, int Nx,
                                 int Ny, int Nz, int Nd, int N, char* material_type,
                                 char* lattice_type, PROFILE* Profile);
void Destroy_Lambdas(LAMBDAS Lambdas, LAMBDAS_CUDA Lambdas_cuda, char* lattice_type);

static double now_s() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

static bool is_simple(const char* lt) {
  return !strcmp(lt, "simple_cubic") || !strcmp(lt, "primitive_orthorhombic") ||
         !strcmp(lt, "primitive_tetragonal");
}

static void die(const char* m) {
  fprintf(stderr, "fame_ref_harness: %s\n", m);
  exit(2);
}

static std::vector<double> read_k(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) die("cannot open k file");
  int nk = 0;
  if (fscanf(f, "%d", &nk) != 1 || nk <= 0) die("bad k file");
  std::vector<double> k(3 * nk);
  for (int i = 0; i < 3 * nk; i++)
    if (fscanf(f, "%lf", &k[i]) != 1) die("short k file");
  fclose(f);
  return k;
}

static std::vector<double> read_raw(const char* path, size_t n) {
  std::vector<double> v(n);
  FILE* f = fopen(path, "rb");
  if (!f) die("cannot open raw file");
  if (fread(v.data(), sizeof(double), n, f) != n) die("short raw file");
  fclose(f);
  return v;
}

// Binary dump of the preprocessing result: a sequence of (name, dtype, count, data)
// records that tests/golden/make_golden.py parses.
static void put(FILE* f, const char* name, char dt, long n, const void* data) {
  int len = (int)strlen(name);
  fwrite(&len, 4, 1, f);
  fwrite(name, 1, len, f);
  fwrite(&dt, 1, 1, f);
  fwrite(&n, 8, 1, f);
  fwrite(data, dt == 'i' ? 4 : 8, n, f);
}

static int mode_pre(const char* out) {
  PAR Par;
  memset(&Par, 0, sizeof(Par));
  FAME_Preprocessing(&Par);
  FILE* f = fopen(out, "wb");
  if (!f) die("cannot write pre output");
  const int N = Par.mesh.grid_nums[0] * Par.mesh.grid_nums[1] * Par.mesh.grid_nums[2];
  put(f, "grid_nums", 'i', 3, Par.mesh.grid_nums);
  put(f, "edge_len", 'd', 3, Par.mesh.edge_len);
  put(f, "mesh_len", 'd', 3, Par.mesh.mesh_len);
  put(f, "lattice_vec_a", 'd', 9, Par.lattice.lattice_vec_a);
  put(f, "lattice_vec_a_orig", 'd', 9, Par.lattice.lattice_vec_a_orig);
  put(f, "Omega", 'd', 9, Par.lattice.Omega);
  put(f, "Permutation", 'i', 3, Par.lattice.Permutation);
  int m[4] = {Par.lattice.lattice_constant.m1, Par.lattice.lattice_constant.m2,
              Par.lattice.lattice_constant.m3, Par.lattice.lattice_constant.m4};
  put(f, "m", 'i', 4, m);
  double t[12] = {0};
  if (Par.lattice.lattice_constant.t1) memcpy(t + 0, Par.lattice.lattice_constant.t1, 24);
  if (Par.lattice.lattice_constant.t2) memcpy(t + 3, Par.lattice.lattice_constant.t2, 24);
  if (Par.lattice.lattice_constant.t3) memcpy(t + 6, Par.lattice.lattice_constant.t3, 24);
  if (Par.lattice.lattice_constant.t4) memcpy(t + 9, Par.lattice.lattice_constant.t4, 24);
  put(f, "t", 'd', 12, t);
  put(f, "reciprocal_lattice_vector_b", 'd', 9, Par.recip_lattice.reciprocal_lattice_vector_b);
  put(f, "WaveVector", 'd', 3L * Par.recip_lattice.Wave_vec_num, Par.recip_lattice.WaveVector);
  int simple = is_simple(Par.lattice.lattice_type);
  put(f, "simple", 'i', 1, &simple);
  put(f, "material_num", 'i', 1, &Par.material.material_num);
  put(f, "Binout", 'i', 3L * Par.material.material_num * N, Par.material.Binout);
  put(f, "ele_permitt_in", 'd', Par.material.num_ele_permitt_in, Par.material.ele_permitt_in);
  put(f, "ele_permitt_out", 'd', 1, &Par.material.ele_permitt_out);
  fclose(f);
  return 0;
}

struct Ctx {
  PAR Par;
  PROFILE Profile;
  CULIB_HANDLES cu;
  FFT_BUFFER fft;
  LANCZOS_BUFFER lb;
  MTX_B B;
  int Nx, Ny, Nz, N;
  std::vector<double> k;
};

static void setup(Ctx& c, const char* kfile, const char* epsfile) {
  memset(&c.Par, 0, sizeof(c.Par));
  FAME_Preprocessing(&c.Par);
  c.Nx = c.Par.mesh.grid_nums[0];
  c.Ny = c.Par.mesh.grid_nums[1];
  c.Nz = c.Par.mesh.grid_nums[2];
  c.N = c.Nx * c.Ny * c.Nz;
  if (kfile) {
    c.k = read_k(kfile);
  } else {
    c.k.assign(c.Par.recip_lattice.WaveVector,
               c.Par.recip_lattice.WaveVector + 3 * c.Par.recip_lattice.Wave_vec_num);
  }
  c.Par.recip_lattice.Wave_vec_num = (int)(c.k.size() / 3);
  FAME_Set_Profile(&c.Profile, c.Par);
  cudaSetDevice(c.Par.flag.device);
  FAME_Create_cublas(&c.cu, c.Nx, c.Ny, c.Nz);
  FAME_Create_Buffer(&c.cu, &c.fft, &c.lb, c.N, c.Par.es.nstep);
  checkCudaErrors(cudaMalloc((void**)&c.B.B_eps, 3L * c.N * sizeof(double)));
  checkCudaErrors(cudaMalloc((void**)&c.B.invB_eps, 3L * c.N * sizeof(double)));
  FAME_Matrix_B_Isotropic(c.B.B_eps, c.B.invB_eps, c.Par.material, c.N);
  if (epsfile) {
    std::vector<double> b = read_raw(epsfile, 3L * c.N), ib(3L * c.N);
    for (size_t i = 0; i < b.size(); i++) ib[i] = 1.0 / b[i];
    checkCudaErrors(cudaMemcpy(c.B.B_eps, b.data(), b.size() * 8, cudaMemcpyHostToDevice));
    checkCudaErrors(cudaMemcpy(c.B.invB_eps, ib.data(), ib.size() * 8, cudaMemcpyHostToDevice));
  }
}

static int mode_solve(const char* out, const char* kfile, const char* epsfile,
                      const char* kidx, const char* evec_prefix) {
  Ctx c;
  setup(c, kfile, epsfile);
  const int nk = (int)(c.k.size() / 3), Nwant = c.Par.es.nwant;
  std::vector<int> which;
  if (kidx) {
    std::string s(kidx);
    size_t p = 0;
    while (p < s.size()) {
      size_t q = s.find(',', p);
      if (q == std::string::npos) q = s.size();
      which.push_back(atoi(s.substr(p, q - p).c_str()));
      p = q + 1;
    }
  } else {
    for (int i = 0; i < nk; i++) which.push_back(i);
  }
  FILE* f = fopen(out, "w");
  if (!f) die("cannot write solve output");
  std::vector<double> freq(Nwant);
  std::vector<cmpx> E(3L * c.N * Nwant);
  for (int i : which) {
    if (i < 0 || i >= nk) die("k index out of range");
    c.Profile.idx = i;
    // the reference accumulates its counters per k index: a k solved again in this
    // run (bench warm-up and timed steps) reports its own counts
    c.Profile.ls_iter[i] = 0;
    c.Profile.es_iter[i] = 0;
    double wv[3] = {c.k[3 * i], c.k[3 * i + 1], c.k[3 * i + 2]};
    LAMBDAS L;
    LAMBDAS_CUDA Lc;
    int Nd = FAME_Matrix_Lambdas(&Lc, wv, c.Par.mesh.grid_nums, c.Par.mesh.mesh_len,
                                 c.Par.lattice.lattice_vec_a, &c.Par, &L);
    cudaDeviceSynchronize();
    double t0 = now_s();
    FAME_Fast_Algorithms_Driver(freq.data(), E.data(), c.cu, c.lb, c.fft, Lc, c.B, c.Par.es,
                                c.Par.ls, c.Nx, c.Ny, c.Nz, Nd, c.N, c.Par.material.material_type,
                                c.Par.lattice.lattice_type, &c.Profile);
    cudaDeviceSynchronize();
    double t1 = now_s();
    cudaError_t err = cudaGetLastError();
    fprintf(f, "{\"k\": %d, \"wave_vec\": [%.17g, %.17g, %.17g], \"Nd\": %d, \"wall_s\": %.6f, "
               "\"ls_iter\": %d, \"es_iter\": %d, \"cuda\": \"%s\", \"freq\": [",
            i, wv[0], wv[1], wv[2], Nd, t1 - t0, c.Profile.ls_iter[i], c.Profile.es_iter[i],
            cudaGetErrorString(err));
    for (int b = 0; b < Nwant; b++) fprintf(f, "%s%.17g", b ? ", " : "", freq[b]);
    fprintf(f, "]}\n");
    fflush(f);
    if (evec_prefix) {
      char name[512];
      snprintf(name, sizeof(name), "%s_k%03d.bin", evec_prefix, i);
      FILE* g = fopen(name, "wb");
      if (!g) die("cannot write evec");
      fwrite(E.data(), sizeof(cmpx), E.size(), g);
      fclose(g);
    }
    Destroy_Lambdas(L, Lc, c.Par.lattice.lattice_type);
  }
  fclose(f);
  return 0;
}

// Applies the reference operators to the vectors in <in.bin> (raw complex128:
// x0 of length 2N, then v0 of length 3N) for every k, writing per k:
// Qr(x0) [3N], Qrs(v0) [2Nd], QBQ(x0) [2Nd], invAr(x0) [2Nd], Nd as a double.
static int mode_apply(const char* in, const char* out, const char* kfile, const char* epsfile) {
  Ctx c;
  setup(c, kfile, epsfile);
  const int N = c.N, nk = (int)(c.k.size() / 3);
  std::vector<double> raw = read_raw(in, 2L * (2 * N + 3 * N));
  cuDoubleComplex *dx, *dv, *dy, *d3;
  checkCudaErrors(cudaMalloc((void**)&dx, 2L * N * 16));
  checkCudaErrors(cudaMalloc((void**)&dv, 3L * N * 16));
  checkCudaErrors(cudaMalloc((void**)&dy, 2L * N * 16));
  checkCudaErrors(cudaMalloc((void**)&d3, 3L * N * 16));
  for (int nd = 0; nd < 4; nd++) {
    cuDoubleComplex** t = nd == 0 ? &c.cu.Nd2_temp1
                        : nd == 1 ? &c.cu.Nd2_temp2
                        : nd == 2 ? &c.cu.Nd2_temp3
                                  : &c.cu.Nd2_temp4;
    checkCudaErrors(cudaMalloc((void**)t, 2L * N * 16));
  }
  FILE* f = fopen(out, "wb");
  if (!f) die("cannot write apply output");
  std::vector<cuDoubleComplex> h(3L * N);
  for (int i = 0; i < nk; i++) {
    double wv[3] = {c.k[3 * i], c.k[3 * i + 1], c.k[3 * i + 2]};
    LAMBDAS L;
    LAMBDAS_CUDA Lc;
    int Nd = FAME_Matrix_Lambdas(&Lc, wv, c.Par.mesh.grid_nums, c.Par.mesh.mesh_len,
                                 c.Par.lattice.lattice_vec_a, &c.Par, &L);
    const bool simple = is_simple(c.Par.lattice.lattice_type);
    std::string ct = simple ? "Simple" : "General";
    double ndd = Nd;
    fwrite(&ndd, 8, 1, f);
    // Qr(x0)
    checkCudaErrors(cudaMemcpy(dx, raw.data(), 2L * Nd * 16, cudaMemcpyHostToDevice));
    if (simple)
      FAME_Matrix_Vector_Production_Qr(d3, dx, c.cu, c.fft, Lc.dD_k, Lc.dPi_Qr, c.Nx, c.Ny, c.Nz,
                                       Nd, &c.Profile);
    else
      FAME_Matrix_Vector_Production_Qr(d3, dx, c.cu, c.fft, Lc.dD_kx, Lc.dD_ky, Lc.dD_kz,
                                       Lc.dPi_Qr, c.Nx, c.Ny, c.Nz, Nd, &c.Profile);
    checkCudaErrors(cudaMemcpy(h.data(), d3, 3L * N * 16, cudaMemcpyDeviceToHost));
    fwrite(h.data(), 16, 3L * N, f);
    // Qrs(v0) (the reference overwrites its input, FAME_Matrix_Vector_Production_Qrs.cu:23)
    checkCudaErrors(cudaMemcpy(dv, raw.data() + 4L * N, 3L * N * 16, cudaMemcpyHostToDevice));
    if (simple)
      FAME_Matrix_Vector_Production_Qrs(dy, dv, c.cu, c.fft, Lc.dD_ks, Lc.dPi_Qrs, c.Nx, c.Ny,
                                        c.Nz, Nd, &c.Profile);
    else
      FAME_Matrix_Vector_Production_Qrs(dy, dv, c.cu, c.fft, Lc.dD_kx, Lc.dD_ky, Lc.dD_kz,
                                        Lc.dPi_Qrs, c.Nx, c.Ny, c.Nz, Nd, &c.Profile);
    checkCudaErrors(cudaMemcpy(h.data(), dy, 2L * Nd * 16, cudaMemcpyDeviceToHost));
    fwrite(h.data(), 16, 2L * Nd, f);
    // QBQ(x0)
    if (simple)
      FAME_Matrix_Vector_Production_Isotropic_QBQ(dy, dx, c.cu, c.fft, c.B, Lc.dD_k, Lc.dD_ks,
                                                  Lc.dPi_Qr, Lc.dPi_Qrs, c.Nx, c.Ny, c.Nz, Nd,
                                                  &c.Profile);
    else
      FAME_Matrix_Vector_Production_Isotropic_QBQ(dy, dx, c.cu, c.fft, c.B, Lc.dD_kx, Lc.dD_ky,
                                                  Lc.dD_kz, Lc.dPi_Qr, Lc.dPi_Qrs, c.Nx, c.Ny,
                                                  c.Nz, Nd, &c.Profile);
    checkCudaErrors(cudaMemcpy(h.data(), dy, 2L * Nd * 16, cudaMemcpyDeviceToHost));
    fwrite(h.data(), 16, 2L * Nd, f);
    // invAr(x0)
    c.Profile.idx = i;
    FAME_Matrix_Vector_Production_Isotropic_invAr(dy, dx, c.cu, c.fft, Lc, c.B, c.Par.ls, c.Nx,
                                                  c.Ny, c.Nz, Nd, ct, &c.Profile);
    checkCudaErrors(cudaMemcpy(h.data(), dy, 2L * Nd * 16, cudaMemcpyDeviceToHost));
    fwrite(h.data(), 16, 2L * Nd, f);
    Destroy_Lambdas(L, Lc, c.Par.lattice.lattice_type);
  }
  fclose(f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 4) die("usage: pre|solve|apply <workdir> ...");
  const std::string mode = argv[1];
  // Output paths are resolved before changing into the work directory.
  std::vector<std::string> abs;
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) die("getcwd failed");
  auto absolute = [&](const char* p) -> std::string {
    return p[0] == '/' ? std::string(p) : std::string(cwd) + "/" + p;
  };
  const char *kfile = nullptr, *epsfile = nullptr, *kidx = nullptr, *evec = nullptr;
  std::string ks, es, ev;
  int pos_end = argc;
  for (int a = 3; a < argc; a++) {
    if (!strcmp(argv[a], "--k") && a + 1 < argc) {
      ks = absolute(argv[++a]);
      kfile = ks.c_str();
      pos_end = pos_end == argc ? a - 1 : pos_end;
    } else if (!strcmp(argv[a], "--eps") && a + 1 < argc) {
      es = absolute(argv[++a]);
      epsfile = es.c_str();
      pos_end = pos_end == argc ? a - 1 : pos_end;
    } else if (!strcmp(argv[a], "--kidx") && a + 1 < argc) {
      kidx = argv[++a];
      pos_end = pos_end == argc ? a - 1 : pos_end;
    } else if (!strcmp(argv[a], "--evec") && a + 1 < argc) {
      ev = absolute(argv[++a]);
      evec = ev.c_str();
      pos_end = pos_end == argc ? a - 1 : pos_end;
    }
  }
  std::string p3 = absolute(argv[3]);
  std::string p4 = argc > 4 ? absolute(argv[4]) : std::string();
  if (chdir(argv[2]) != 0) die("cannot chdir to workdir");
  if (mode == "pre") return mode_pre(p3.c_str());
  if (mode == "solve") return mode_solve(p3.c_str(), kfile, epsfile, kidx, evec);
  if (mode == "apply") {
    if (pos_end < 5) die("apply needs <in.bin> <out.bin>");
    return mode_apply(p3.c_str(), p4.c_str(), kfile, epsfile);
  }
  die("unknown mode");
  return 2;
}
