// FAME_Main_Code(PAR, PROFILE*) over the fame_b200 C ABI.
//
// The reference's Main.cpp (Main.cpp:32) calls FAME_Main_Code with C++ linkage.
// This file provides that function, so Main.cpp, the reference's preprocessing
// (Popt.txt and the material description) and its output writers link unchanged
// against libfame_b200.so instead of FAME_Main/*.cu.  It is compiled with the
// reference's include/ directory on the include path (build_main.sh), which
// supplies PAR and PROFILE (include/FAME_Internal_Common.h:150-211).
//
// Behaviour kept from FAME_Main/FAME_Main_Code.cu:35-140:
//   * device Par.flag.device; B from Par.material (isotropic materials only), and,
//     as in FAME_Matrix_B_Isotropic (FAME_Main/FAME_Matrix_B_Isotropic.cu:69-72),
//     Par.material.Binout and Par.material.ele_permitt_in are freed here;
//   * Profile->ls_iter[i] / es_iter[i] / es_time[i] per wave vector, Profile->idx
//     left at the last wave vector, the profile table printed per wave vector;
//   * Data_Omega_array.txt written by the reference's FAME_Create_Frequency_txt and,
//     when Par.flag.save_eigen_vector is set, Data_EV_*.txt in FAME_Save_Eigenvector's
//     format by fame_write_eigenvectors (formatted on all host threads) on a
//     background thread: one batch's files while the next batch is solved;
//   * the sign convention of Check_Residual (FAME_Main_Code.cu:383-421): a frequency
//     whose residual ||C^H C E - w^2 B E|| (E scaled as the reference restores it)
//     exceeds 1e-10 is stored negated.  The residual comes from the solver's FP64
//     band statistics on the device (fame_solve_kpoints resabs_out) instead of the
//     reference's CPU sparse product; the per-band lines are printed the same way.
// Differences: all wave vectors are solved in batches by fame_solve_kpoints (the
// per-k time is the batch time divided evenly, ls_time is 0) and the CPU check of
// the FFT eigendecomposition (Check_Eigendecomp) is not run.  The
// precision comes from the environment variable FAME_B200_PRECISION: "mixed"
// (default: FP32 operator and CG with FP64 refinement, FP64 Lanczos) or "fp64".
// Errors are printed with fame_last_error() and returned as the fame status.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "FAME_Internal_Common.h"
#include "FAME_Create_Frequency_txt.h"
#include "FAME_Profile.h"
#include "fame_b200.h"

namespace {

bool is_simple(const char* lattice_type) {
  // the reference's Simple dispatch (FAME_Main/FAME_Main_Code.cu:158-160)
  return !strcmp(lattice_type, "simple_cubic") || !strcmp(lattice_type, "primitive_orthorhombic") ||
         !strcmp(lattice_type, "primitive_tetragonal");
}

double now_s() {
  timespec t;
  clock_gettime(CLOCK_REALTIME, &t);
  return t.tv_sec + t.tv_nsec * 1e-9;
}

int fail(int rc, const char* what) {
  fprintf(stderr, "FAME_Main_Code: %s: %s\n", what, fame_last_error());
  return rc;
}

}  // namespace

int FAME_Main_Code(PAR Par, PROFILE* Profile) {
  const int Nx = Par.mesh.grid_nums[0], Ny = Par.mesh.grid_nums[1], Nz = Par.mesh.grid_nums[2];
  const long N = (long)Nx * Ny * Nz;
  const int Nwant = Par.es.nwant;
  const int nk = Par.recip_lattice.Wave_vec_num;

  fame_lattice lat;
  memset(&lat, 0, sizeof(lat));
  for (int i = 0; i < 3; i++) {
    lat.grid[i] = Par.mesh.grid_nums[i];
    lat.mesh_len[i] = Par.mesh.mesh_len[i];
  }
  memcpy(lat.lattice_vec_a, Par.lattice.lattice_vec_a, sizeof(lat.lattice_vec_a));
  lat.simple = is_simple(Par.lattice.lattice_type) ? 1 : 0;
  const LATTICE_CONSTANT& lc = Par.lattice.lattice_constant;
  lat.m[0] = lc.m1;
  lat.m[1] = lc.m2;
  lat.m[2] = lc.m3;
  lat.m[3] = lc.m4;
  if (lc.t1) memcpy(lat.t1, lc.t1, sizeof(lat.t1));

  if (strcmp(Par.material.material_type, "isotropic") != 0) {
    fprintf(stderr, "FAME_Main_Code: material type %s is not supported\n", Par.material.material_type);
    return FAME_ERR_UNSUPPORTED;
  }
  if (Par.material.num_ele_permitt_in < Par.material.material_num) {
    // The reference prompts on stdin for the missing values here
    // (FAME_Main/FAME_Matrix_B_Isotropic.cu:13-24); a library call must not, so the
    // run ends with a status.  Binout and ele_permitt_in are released as the
    // reference's FAME_Matrix_B_Isotropic releases them (:69-72).
    fprintf(stderr,
            "FAME_Main_Code: %d inner permittivities given for %d materials (Popt.txt "
            "\"# Permittivity (inner material)\" needs one per material)\n",
            Par.material.num_ele_permitt_in, Par.material.material_num);
    free(Par.material.Binout);
    free(Par.material.ele_permitt_in);
    return FAME_ERR_BAD_INPUT;
  }
  fame_ctx* ctx = nullptr;
  int rc = fame_ctx_create(Par.flag.device, &lat, &ctx);
  if (rc != FAME_OK) return fail(rc, "fame_ctx_create");
  rc = fame_set_material(ctx, Par.material.Binout, Par.material.material_num, Par.material.ele_permitt_in,
                         Par.material.ele_permitt_out);
  free(Par.material.Binout);
  free(Par.material.ele_permitt_in);
  if (rc != FAME_OK) {
    fame_ctx_destroy(ctx);
    return fail(rc, "fame_set_material");
  }

  fame_solver_params p;
  memset(&p, 0, sizeof(p));
  p.nwant = Nwant;
  p.nstep = Par.es.nstep;
  p.es_maxit = Par.es.maxit;
  p.es_tol = Par.es.tol;
  p.ls_maxit = Par.ls.maxit;
  p.ls_tol = Par.ls.tol;
  const char* prec = getenv("FAME_B200_PRECISION");
  p.precision = (prec && !strcmp(prec, "fp64")) ? FAME_FP64 : FAME_MIXED;
  p.use_graph = 1;
  // With eigenvectors to save, the wave vectors are solved in batches of `chunk` into
  // two host buffers of chunk x Nwant x 3N complex values: the files of one batch are
  // written on a background thread while the next batch is solved into the other
  // buffer.  chunk: what a quarter of the available host memory holds for the two
  // buffers, or the environment variable FAME_B200_SAVE_BATCH.
  const bool save = Par.flag.save_eigen_vector != 0;
  p.want_vectors = save ? 1 : 0;
  const size_t per_k = (size_t)Nwant * 3 * N * 2;  // doubles of one wave vector's eigenvectors
  int chunk = nk;
  if (save) {
    const long pages = sysconf(_SC_AVPHYS_PAGES), psz = sysconf(_SC_PAGESIZE);
    const double avail = pages > 0 && psz > 0 ? (double)pages * (double)psz : 8e9;
    chunk = (int)std::max(1.0, std::min((double)nk, floor(0.25 * avail / (2.0 * per_k * sizeof(double)))));
    const char* env = getenv("FAME_B200_SAVE_BATCH");
    if (env && atoi(env) > 0) chunk = std::min(nk, atoi(env));
  }

  std::vector<double> freq((size_t)nk * Nwant), relres((size_t)nk * Nwant), resabs((size_t)nk * Nwant);
  std::vector<fame_kcounters> cnt(nk);
  std::vector<double> evec[2];
  if (save)
    for (auto& e : evec) e.resize((size_t)chunk * per_k);
  // the background writer of the last batch: writes its wave vectors' files in order
  std::thread writer;
  int writer_rc = FAME_OK;
  std::string writer_err;
  auto finish_writer = [&]() -> int {
    if (writer.joinable()) writer.join();
    const int wrc = writer_rc;
    writer_rc = FAME_OK;
    return wrc;
  };
  int status = FAME_OK;
  for (int k0 = 0; k0 < nk; k0 += chunk) {
    const int n = nk - k0 < chunk ? nk - k0 : chunk;
    std::vector<double>& ev = evec[(k0 / chunk) & 1];
    const double t0 = now_s();
    rc = fame_solve_kpoints(ctx, Par.recip_lattice.WaveVector + 3L * k0, n, &p, freq.data() + (size_t)k0 * Nwant,
                            relres.data() + (size_t)k0 * Nwant, nullptr, resabs.data() + (size_t)k0 * Nwant,
                            save ? ev.data() : nullptr, cnt.data() + k0);
    const double dt = now_s() - t0;
    if (rc != FAME_OK && rc != FAME_ERR_NO_CONVERGENCE) {
      const std::string msg = fame_last_error();
      finish_writer();
      fame_ctx_destroy(ctx);
      fprintf(stderr, "FAME_Main_Code: fame_solve_kpoints: %s\n", msg.c_str());
      return rc;
    }
    if (rc != FAME_OK) status = rc;
    for (int i = k0; i < k0 + n; i++) {
      Profile->idx = i;
      Profile->ls_iter[i] = cnt[i].ls_iter;
      Profile->es_iter[i] = cnt[i].es_iter;
      Profile->ls_time[i] = 0.0;
      Profile->es_time[i] = dt / n;
      const double* w = Par.recip_lattice.WaveVector + 3L * i;
      printf("= = WaveVector (%3d/%3d) = [ % .6f % .6f % .6f ] = =\n", i + 1, nk, w[0], w[1], w[2]);
      for (int b = 0; b < Nwant; b++) {
        double& f = freq[(size_t)i * Nwant + b];
        const double res = resabs[(size_t)i * Nwant + b];
        printf("                 Freq(%2d) = %10.8f, residual = %e, relative residual = %.2e.\n", b, f, res,
               relres[(size_t)i * Nwant + b]);
        if (res > 1e-10) f = -f;
      }
      FAME_Print_Profile(*Profile);
    }
    if (save) {
      // Data_EV_*.txt as FAME_Save_Eigenvector writes them (FAME_Main_Code.cu:127), byte
      // for byte: the previous batch's writer has finished with the other buffer, this
      // batch's files are written while the next batch solves
      const int wrc = finish_writer();
      if (wrc != FAME_OK) {
        fame_ctx_destroy(ctx);
        fprintf(stderr, "FAME_Main_Code: writing eigenvectors: %s\n", writer_err.c_str());
        return wrc;
      }
      const double* evp = ev.data();
      writer = std::thread([&writer_rc, &writer_err, evp, per_k, Nwant, N, k0, n]() {
        for (int i = k0; i < k0 + n && writer_rc == FAME_OK; i++) {
          writer_rc = fame_write_eigenvectors(nullptr, evp + (size_t)(i - k0) * per_k, Nwant, 3LL * N, i, 0);
          if (writer_rc != FAME_OK) writer_err = fame_last_error();
        }
      });
    }
  }
  const int wrc = finish_writer();
  if (wrc != FAME_OK) {
    fame_ctx_destroy(ctx);
    fprintf(stderr, "FAME_Main_Code: writing eigenvectors: %s\n", writer_err.c_str());
    return wrc;
  }
  FAME_Create_Frequency_txt(freq.data(), Nwant, Profile->idx);
  fame_ctx_destroy(ctx);
  if (status != FAME_OK) fprintf(stderr, "FAME_Main_Code: %s\n", fame_last_error());
  return status;
}
