// Host-program symbols the reference library expects its caller to provide
// (qws_bqcd.cc:56-57 declares them extern; in BQCD they come from Fortran).
// Linked only into oracle/_ref builds of the reference sources: test
// infrastructure, never part of the product.
//
// Convention (shared with the product's own loaders): sites are split by
// parity eo = (x+y+z+t) % 2, and inside a parity they are numbered
// lexicographically (x fastest) starting at 1, i.e. i = lex/2 + 1 with
// lex = x + nx*(y + ny*(z + nz*t)); this is a bijection when nx is even.
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
}
