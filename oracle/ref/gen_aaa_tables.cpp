// Test infrastructure only (oracle build step).
// Regenerates the three translation-coefficient headers that the reference
// includes but does not ship (lib/include/lib_multipole_expansion_constants.hpp:43-45;
// listed in .MISSING_LARGE_BLOBS):  AAA_M2M_FMM.hpp, AAA_M2L_FMM.hpp, AAA_L2L_FMM.hpp.
// Formulas: Greengard & Rokhlin (1997), see ../aaa_coeffs.hpp.  Layout and names follow
// the reference's use sites: AAA_*_FMM[j][k+N][n][m+N] of std::complex<double>, with
// N_AAA_*_FMM = N (moments.hpp:200-270).  Output goes to the directory given as argv[1].
#include <cstdio>
#include <string>

#include "../aaa_coeffs.hpp"

static void emit(const std::string& dir, const char* name, int N, double (*f)(int, int, int, int)) {
  std::string path = dir + "/AAA_" + name + "_FMM.hpp";
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) {
    std::perror(path.c_str());
    std::exit(1);
  }
  int W = 2 * N + 1;
  std::fprintf(fp, "#pragma once\n#include <array>\n#include <complex>\n");
  std::fprintf(fp, "static const int N_AAA_%s_FMM = %d;\n", name, N);
  std::fprintf(fp,
               "static const std::array<std::array<std::array<std::array<std::complex<double>, %d>, %d>, %d>, %d> AAA_%s_FMM = {{\n",
               W, N + 1, W, N + 1, name);
  for (int j = 0; j <= N; ++j) {
    std::fprintf(fp, "{{");
    for (int kk = 0; kk < W; ++kk) {
      int k = kk - N;
      std::fprintf(fp, "{{");
      for (int n = 0; n <= N; ++n) {
        std::fprintf(fp, "{{");
        for (int mm = 0; mm < W; ++mm) {
          int m = mm - N;
          double v = (std::abs(k) <= j && std::abs(m) <= n) ? f(j, k, n, m) : 0.0;
          std::fprintf(fp, "std::complex<double>(%.17g,0.)%s", v, mm + 1 < W ? "," : "");
        }
        std::fprintf(fp, "}}%s", n < N ? "," : "");
      }
      std::fprintf(fp, "}}%s", kk + 1 < W ? "," : "");
    }
    std::fprintf(fp, "}}%s\n", j < N ? "," : "");
  }
  std::fprintf(fp, "}};\n");
  std::fclose(fp);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s OUTDIR N\n", argv[0]);
    return 2;
  }
  int N = std::atoi(argv[2]);
  emit(argv[1], "M2M", N, bem_oracle_aaa::m2m);
  emit(argv[1], "M2L", N, bem_oracle_aaa::m2l);
  emit(argv[1], "L2L", N, bem_oracle_aaa::l2l);
  return 0;
}
