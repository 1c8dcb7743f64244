// Test driver for the reference's eigenvector writer (test infrastructure; the
// product never runs it): calls FAME_Save_Eigenvector
// (FAME_Tools/FAME_Save_Eigenvector.cpp:7-45, compiled from the reference's source
// by oracle/build_ref.sh) on values read from a file.
//
//   fame_ref_evwriter NWANT N3 KIDX INFILE
//
// INFILE holds NWANT * N3 complex128 values (band-major, little-endian); the
// Data_EV_*.txt files go to the working directory.
#include <cstdio>
#include <cstdlib>
#include <vector>

int FAME_Save_Eigenvector(double _Complex* Ele_field_mtx, int Nwant, int N3, int idx);

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s NWANT N3 KIDX INFILE\n", argv[0]);
    return 2;
  }
  const int nwant = atoi(argv[1]), n3 = atoi(argv[2]), kidx = atoi(argv[3]);
  std::vector<double _Complex> v((size_t)nwant * n3);
  FILE* f = fopen(argv[4], "rb");
  if (!f || fread(v.data(), sizeof(double _Complex), v.size(), f) != v.size()) {
    fprintf(stderr, "cannot read %s\n", argv[4]);
    return 1;
  }
  fclose(f);
  return FAME_Save_Eigenvector(v.data(), nwant, n3, kidx);
}
