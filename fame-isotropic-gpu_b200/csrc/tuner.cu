// fame_tune: the FFT plan autotuner.
//
// The reference fixes its transforms once per run (cufftPlan1d / cufftPlan3d in
// FAME_Main/FAME_Create_cublas.cu:16-25) and leaves the choice to cuFFT.  Here the
// plan of a context's runtime-geometry grids (every grid but the compile-time 96^3
// one) has free parameters: the radix order of the axis plans, the threads of a plane
// CTA in FP32 and FP64, and the L2 prefetch of the mixed-precision CG kernels.  The
// tuner times candidates with CUDA events on the context's stream (fame_bench_cg for
// FAME_MIXED: one FP32 CG iteration, its three kernels; fame_bench_qbq for FAME_FP64:
// one Q_r^* B^-1 Q_r apply), each on `batch` copies of the k-point with the L2 flushed
// before every repetition, and keeps the fastest by coordinate descent: radix order,
// then CTA size, then prefetch, from the context's current options.  The winner is applied to the context and appended to
// a plain-text cache file under a key of grid, lattice family, precision and batch, so
// a later run with the same key applies it without timing.
//
// Built only on the public C ABI (include/fame_b200.h).
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fame_b200.h"

namespace fame {
void set_last_error(const std::string& s);
}

namespace {

struct Plan {
  int radix_order = 0, threads32 = 0, threads64 = 0, prefetch = 1;
};

std::string plan_text(const Plan& p) {
  char b[160];
  snprintf(b, sizeof b, "radix_order=%d plane_threads32=%d plane_threads64=%d prefetch=%d", p.radix_order,
           p.threads32, p.threads64, p.prefetch);
  return b;
}

bool parse_plan(const std::string& s, Plan& p) {
  return sscanf(s.c_str(), "radix_order=%d plane_threads32=%d plane_threads64=%d prefetch=%d", &p.radix_order,
                &p.threads32, &p.threads64, &p.prefetch) == 4;
}

int apply(fame_ctx* c, const Plan& p) {
  int rc;
  if ((rc = fame_set_option(c, "radix_order", p.radix_order)) != FAME_OK) return rc;
  if ((rc = fame_set_option(c, "plane_threads32", p.threads32)) != FAME_OK) return rc;
  if ((rc = fame_set_option(c, "plane_threads64", p.threads64)) != FAME_OK) return rc;
  return fame_set_option(c, "prefetch", p.prefetch);
}

int get(fame_ctx* c, const char* name) {
  int v = 0;
  fame_get_option(c, name, &v);
  return v;
}

// Device ms of the candidate (the better of two timings), or a negative status.
double time_plan(fame_ctx* c, const Plan& p, const double* k, int precision, int batch, int reps) {
  if (apply(c, p) != FAME_OK) return -1;
  double best = 1e30;
  for (int t = 0; t < 2; t++) {
    double ms = 0;
    const int rc = precision == FAME_MIXED ? fame_bench_cg(c, k, reps, batch, &ms, nullptr)
                                           : fame_bench_qbq(c, k, precision, reps, batch, &ms, nullptr);
    if (rc != FAME_OK) return -2;
    best = ms < best ? ms : best;
  }
  return best;
}

std::string tune_key(fame_ctx* c, int precision, int batch) {
  char b[160];
  snprintf(b, sizeof b, "grid=%dx%dx%d general=%d precision=%s batch=%d", get(c, "grid_x"), get(c, "grid_y"),
           get(c, "grid_z"), get(c, "general"), precision == FAME_MIXED ? "mixed" : "fp64", batch);
  return b;
}

}  // namespace

extern "C" int fame_tune(fame_ctx* c, const double* k, int precision, int batch, const char* cache_file,
                         char* plan_out, int plan_len) {
  if (!c || !k || batch < 1 || batch > 64 || (precision != FAME_FP64 && precision != FAME_MIXED)) {
    fame::set_last_error("bad argument");
    return FAME_ERR_BAD_INPUT;
  }
  const std::string key = tune_key(c, precision, batch);
  Plan best;
  bool cached = false;
  if (cache_file) {
    std::ifstream in(cache_file);
    std::string line;
    while (std::getline(in, line)) {  // the last entry of the key wins
      const size_t bar = line.find(" | ");
      Plan p;
      if (bar != std::string::npos && line.compare(0, bar, key) == 0 && parse_plan(line.substr(bar + 3), p)) {
        best = p;
        cached = true;
      }
    }
  }
  if (cached) {
    const int rc = apply(c, best);
    if (rc != FAME_OK) return rc;
  } else {
    const bool stat = get(c, "static96") != 0;
    const int reps = 5;
    Plan cur;  // the context's current choices (the built-in ones unless tuned before)
    cur.radix_order = get(c, "radix_order");
    cur.threads32 = get(c, "plane_threads32");
    cur.threads64 = get(c, "plane_threads64");
    cur.prefetch = get(c, "prefetch");
    double t_best = time_plan(c, cur, k, precision, batch, reps);
    if (t_best < 0) return t_best == -1 ? FAME_ERR_BAD_INPUT : FAME_ERR_CUDA;
    best = cur;
    if (!stat) {
      // radix order (distinct plans only)
      std::vector<int> sigs;
      apply(c, best);
      sigs.push_back(get(c, "plan_signature"));
      for (int o = 1; o < 4; o++) {
        Plan p = best;
        p.radix_order = o;
        if (apply(c, p) != FAME_OK) continue;
        const int sg = get(c, "plan_signature");
        bool seen = false;
        for (int v : sigs) seen = seen || v == sg;
        if (seen) continue;
        sigs.push_back(sg);
        const double t = time_plan(c, p, k, precision, batch, reps);
        if (t > 0 && t < t_best) {
          t_best = t;
          best = p;
        }
      }
      // plane CTA size of the precision the timed kernels run in
      for (int th : {128, 192, 256, 384, 512}) {
        Plan p = best;
        (precision == FAME_MIXED ? p.threads32 : p.threads64) = th;
        const double t = time_plan(c, p, k, precision, batch, reps);
        if (t > 0 && t < t_best) {
          t_best = t;
          best = p;
        }
      }
    }
    if (precision == FAME_MIXED) {
      Plan p = best;
      p.prefetch = 1 - best.prefetch;
      const double t = time_plan(c, p, k, precision, batch, reps);
      if (t > 0 && t < t_best) {
        t_best = t;
        best = p;
      }
    }
    const int rc = apply(c, best);
    if (rc != FAME_OK) return rc;
    if (cache_file) {
      std::ofstream out(cache_file, std::ios::app);
      if (!out) {
        fame::set_last_error(std::string("cannot append to ") + cache_file);
        return FAME_ERR_IO;
      }
      out << key << " | " << plan_text(best) << "\n";
    }
  }
  if (plan_out && plan_len > 0) {
    const std::string t = plan_text(best) + (cached ? " (cached)" : "");
    snprintf(plan_out, (size_t)plan_len, "%s", t.c_str());
  }
  return FAME_OK;
}
