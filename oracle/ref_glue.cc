// Host-program symbols the reference library expects its caller to provide
// (qws_bqcd.cc:56-57 declares them extern; in BQCD they come from Fortran).
// Linked only into oracle/_ref builds of the reference sources: test
// infrastructure, never part of the product.
//
// Convention (shared with the product's own loaders): sites are split by
// parity eo = (x+y+z+t) % 2, and inside a parity they are numbered
// lexicographically (x fastest) starting at 1, i.e. i = lex/2 + 1 with
// lex = x + nx*(y + ny*(z + nz*t)); this is a bijection when nx is even.
#include <cstdio>

extern "C" {
extern int nx, ny, nz, nt;

int std_xyzt2i_(int* j) {
  int lex = j[0] + nx * (j[1] + ny * (j[2] + nz * j[3]));
  return lex / 2 + 1;
}

int e_o_(int* j) { return (j[0] + j[1] + j[2] + j[3]) % 2; }

// Small accessors so a ctypes caller can drive the reference's global state.
extern double kappa, kappa2, mkappa;
void ref_set_kappa(double k) {
  kappa = k;
  kappa2 = k * k;
  mkappa = -k;
}

// The reference's own call counters (timing.c, compiled with _CHECK_TIMING):
// print_timing_ writes its table -- routine, calls, total and average
// seconds -- to para_outputfile when that is set (timing.c:82-100).  Used to
// read the inner-iteration count of a solve, which the reference does not
// return (bicgstab_precdd_s_ counts it only under _DEBUG_).  print_timing_
// frees the table but keeps its head pointer, so this may run once per
// process, at the end, as main.cc:376-384 does.
extern FILE* para_outputfile;
void print_timing_(void);
int ref_timing_dump(const char* path) {
  FILE* f = fopen(path, "w");
  if (!f) return 1;
  FILE* keep = para_outputfile;
  para_outputfile = f;
  print_timing_();
  para_outputfile = keep;
  fclose(f);
  return 0;
}
}
