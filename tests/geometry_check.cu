// Host-side check of the site indexing the kernels use (lattice.cuh): the
// functions are __host__ __device__, so the exact device code runs here on
// the CPU, over every site of each lattice given on the command line
// ("Lx,Ly,Lz,Lt/NBx,NBy,NBz,NBt ...", or "planted:..." to check that a
// planted mistake is caught).  For every site g:
//   * decode_site(g) gives in-range block and in-block coordinates, and
//     dd_index of the site's coordinates is g again (the DD order is a
//     bijection of [0, V));
//   * for each of the eight hops, the neighbour's index -- g + rot_step(...)
//     when it lies in the same block, nbr_across(...) when it crosses a block
//     face (periodic wrap included) -- equals dd_index of the neighbour's
//     coordinates and lies in [0, V), and the colour nbr_across reports is
//     the neighbour's block colour;
//   * on_block_face(g), which makes the face kernels' site lists, holds
//     exactly when some hop of g leaves its block.
// It prints one line per lattice and exits non-zero on the first failure.
// Built and run by tests/test_geometry_host.py (nvcc, no GPU needed).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../qws_b200/csrc/lattice.cuh"

using namespace qwsg;

static int fail(const char* what, const int L[4], const int NB[4], long g, int mu, int dir) {
  std::printf("FAIL %s: lattice %dx%dx%dx%d blocks %d,%d,%d,%d site %ld mu %d dir %d\n", what,
              L[0], L[1], L[2], L[3], NB[0], NB[1], NB[2], NB[3], g, mu, dir);
  return 1;
}

// planted: a mistake put in on purpose (two in-block strides swapped after
// the layout is made), which the checks must catch
static int check(const int L[4], const int NB[4], bool planted) {
  Geom G{};
  for (int mu = 0; mu < 4; mu++) {
    G.L[mu] = L[mu];
    G.NB[mu] = NB[mu];
    G.B[mu] = L[mu] / NB[mu];
  }
  G.tbc = -1;
  G.nr = 1;
  geom_layout(G);
  if (planted) {
    const int t = G.str[0];
    G.str[0] = G.str[1];
    G.str[1] = t;
  }
  for (long g = 0; g < G.V; g++) {
    Site s;
    decode_site(G, (int)g, s);
    int x[4];
    for (int mu = 0; mu < 4; mu++) {
      if (s.lc[mu] < 0 || s.lc[mu] >= G.B[mu] || s.bc[mu] < 0 || s.bc[mu] >= G.NB[mu])
        return fail("decoded coordinates out of range", L, NB, g, mu, 0);
      x[mu] = s.bc[mu] * G.B[mu] + s.lc[mu];
    }
    if ((s.bc[0] + s.bc[1] + s.bc[2] + s.bc[3]) % 2 != s.col)
      return fail("block colour", L, NB, g, -1, 0);
    if (dd_index(G, x) != g) return fail("dd_index(decode_site(g)) != g", L, NB, g, -1, 0);
    bool face = false;  // some hop leaves the block
    for (int mu = 0; mu < 4; mu++) face |= s.lc[mu] == 0 || s.lc[mu] == G.B[mu] - 1;
    if (on_block_face(G, (int)g) != face) return fail("face-site test", L, NB, g, -1, 0);
    for (int mu = 0; mu < 4; mu++)
      for (int dir = -1; dir <= 1; dir += 2) {
        int y[4] = {x[0], x[1], x[2], x[3]};
        y[mu] = (y[mu] + dir + G.L[mu]) % G.L[mu];
        const long want = dd_index(G, y);
        const int l = s.lc[mu] + dir;
        long got;
        if (l >= 0 && l < G.B[mu]) {
          got = g + rot_step(G, mu, s.lc[mu], dir);
        } else {
          int ncol = -1;
          got = nbr_across(G, s, mu, dir, &ncol);
          const int yb = (y[0] / G.B[0] + y[1] / G.B[1] + y[2] / G.B[2] + y[3] / G.B[3]) % 2;
          if (ncol != yb) return fail("nbr_across colour", L, NB, g, mu, dir);
        }
        if (got < 0 || got >= G.V) return fail("neighbour index out of [0, V)", L, NB, g, mu, dir);
        if (got != want) return fail("neighbour index", L, NB, g, mu, dir);
      }
  }
  std::printf("ok %dx%dx%dx%d blocks %d,%d,%d,%d (rotated direction %d, strides %d %d %d %d)\n",
              L[0], L[1], L[2], L[3], NB[0], NB[1], NB[2], NB[3], G.rot, G.str[0], G.str[1],
              G.str[2], G.str[3]);
  return 0;
}

int main(int argc, char** argv) {
  for (int i = 1; i < argc; i++) {
    int L[4], NB[4];
    const bool planted = std::strncmp(argv[i], "planted:", 8) == 0;
    if (std::sscanf(argv[i] + (planted ? 8 : 0), "%d,%d,%d,%d/%d,%d,%d,%d", &L[0], &L[1], &L[2],
                    &L[3], &NB[0], &NB[1], &NB[2], &NB[3]) != 8) {
      std::printf("FAIL bad argument %s\n", argv[i]);
      return 2;
    }
    if (check(L, NB, planted)) return 1;
  }
  return 0;
}
