// Eigenvector text files in the reference's format (FAME_Save_Eigenvector,
// FAME_Tools/FAME_Save_Eigenvector.cpp:7-45): host code only.  Each line is
// formatted with the same format string and the same C library as the reference's
// writer, so the files are byte for byte the same; the formatting of a band is split
// over host threads and the pieces are written in order.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fame_b200.h"

namespace fame {
void set_last_error(const std::string& s);
}

struct fame_writer {
  std::thread th;
  int rc = FAME_OK;
  std::string err;
};

namespace {

struct EvJob {
  std::string dir;
  const double* evec;
  int nwant;
  long long n3;
  int kidx;
  int nthreads;
};

std::string ev_file(const std::string& dir, int kidx, int band) {
  char b[64];
  snprintf(b, sizeof b, "Data_EV_%02d_%02d.txt", kidx + 1, band + 1);  // FAME_Save_Eigenvector.cpp:17-35
  return dir.empty() ? std::string(b) : dir + "/" + b;
}

// lines [i0, i1) of one band: "(% e) + (% e * 1i)\n" per complex entry (…Eigenvector.cpp:39-40)
void format_lines(const double* v, long long i0, long long i1, std::string& out) {
  out.clear();
  out.reserve((size_t)(i1 - i0) * 40);
  char b[96];
  for (long long i = i0; i < i1; i++) {
    const int n = snprintf(b, sizeof b, "(% e) + (% e * 1i)\n", v[2 * i], v[2 * i + 1]);
    out.append(b, (size_t)n);
  }
}

int run_job(const EvJob& j, std::string& err) {
  int nt = j.nthreads > 0 ? j.nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  // below ~64k lines per thread the threads cost more than they save
  nt = (int)std::max(1LL, std::min((long long)nt, j.n3 / 65536 + 1));
  std::vector<std::string> part((size_t)nt);
  for (int b = 0; b < j.nwant; b++) {
    const double* v = j.evec + (size_t)b * (size_t)j.n3 * 2;
    if (nt == 1) {
      format_lines(v, 0, j.n3, part[0]);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < nt; t++) {
        const long long i0 = j.n3 * t / nt, i1 = j.n3 * (t + 1) / nt;
        th.emplace_back(format_lines, v, i0, i1, std::ref(part[(size_t)t]));
      }
      for (auto& x : th) x.join();
    }
    const std::string name = ev_file(j.dir, j.kidx, b);
    FILE* fp = fopen(name.c_str(), "w");
    if (!fp) {
      err = "cannot open " + name + ": " + strerror(errno);
      return FAME_ERR_IO;
    }
    bool ok = fprintf(fp, "Ele_field_mtx{%d}(:, %d) = [\n", j.kidx + 1, b + 1) > 0;
    for (int t = 0; t < nt && ok; t++) ok = fwrite(part[(size_t)t].data(), 1, part[(size_t)t].size(), fp) ==
                                             part[(size_t)t].size();
    ok = ok && fputs("];\n", fp) >= 0;
    ok = (fclose(fp) == 0) && ok;
    if (!ok) {
      err = "write failed: " + name;
      return FAME_ERR_IO;
    }
  }
  return FAME_OK;
}

int check(const double* evec, int nwant, long long n3, int kidx) {
  if (!evec || nwant < 1 || n3 < 1 || kidx < 0) {
    fame::set_last_error("bad argument (evec, nwant >= 1, n3 >= 1, kidx >= 0)");
    return FAME_ERR_BAD_INPUT;
  }
  return FAME_OK;
}

}  // namespace

extern "C" {

int fame_write_eigenvectors(const char* dir, const double* evec, int nwant, long long n3, int kidx, int nthreads) {
  int rc = check(evec, nwant, n3, kidx);
  if (rc) return rc;
  std::string err;
  try {
    rc = run_job(EvJob{dir ? dir : "", evec, nwant, n3, kidx, nthreads}, err);
  } catch (const std::exception& e) {  // thread creation or allocation
    err = std::string("eigenvector writer: ") + e.what();
    rc = FAME_ERR_IO;
  }
  if (rc) fame::set_last_error(err);
  return rc;
}

int fame_writer_start(const char* dir, const double* evec, int nwant, long long n3, int kidx, int nthreads,
                      fame_writer** writer_out) {
  if (!writer_out) {
    fame::set_last_error("null writer_out");
    return FAME_ERR_BAD_INPUT;
  }
  *writer_out = nullptr;
  int rc = check(evec, nwant, n3, kidx);
  if (rc) return rc;
  fame_writer* w = nullptr;
  try {
    w = new fame_writer;
    const EvJob job{dir ? dir : "", evec, nwant, n3, kidx, nthreads};
    w->th = std::thread([w, job] {
      try {
        w->rc = run_job(job, w->err);
      } catch (const std::exception& e) {
        w->err = std::string("eigenvector writer: ") + e.what();
        w->rc = FAME_ERR_IO;
      }
    });
  } catch (const std::exception& e) {
    delete w;
    fame::set_last_error(std::string("eigenvector writer: ") + e.what());
    return FAME_ERR_IO;
  }
  *writer_out = w;
  return FAME_OK;
}

int fame_writer_finish(fame_writer* w) {
  if (!w) {
    fame::set_last_error("null writer");
    return FAME_ERR_BAD_INPUT;
  }
  w->th.join();
  const int rc = w->rc;
  if (rc) fame::set_last_error(w->err);
  delete w;
  return rc;
}

}  // extern "C"
