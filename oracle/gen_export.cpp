// C export of the seeded synthetic-configuration generator for the checkers.
// TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles general_code_b200/csrc/gc_generator.cpp (the
// generator's only source) with this file into oracle/libgen.so, with the
// same g++ flags the product library uses for it, so that the reference arm
// of the benchmark and the fixture scripts build their input without loading
// the product library. Output: the host link array, link index 4*site+mu,
// row-major element order (the layout of gc_generate_host).
namespace gc {
int generate_host(const int dims[4], int nc, double eps, unsigned seed, unsigned cfg,
                  int gauge, double *out);
}

extern "C" int og_generate_host(const int dims[4], int nc, double eps, unsigned seed,
                                unsigned cfg, int gauge, double *out) {
  if (!dims || !out || (nc != 2 && nc != 3))
    return -1;
  for (int d = 0; d < 4; d++)
    if (dims[d] <= 0)
      return -1;
  return gc::generate_host(dims, nc, eps, seed, cfg, gauge, out);
}
