// output_potential through the drop-in: reads n, then x, y, z, pot (n doubles each) from
// the binary file argv[1], fills the reference's PARTICLE array and writes argv[2] with
// output_potential, as a program written against src/tree3d.h would.
#include <cstdio>
#include <vector>

#include "tree3d_b200.h"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  long long n = 0;
  if (std::fread(&n, sizeof(n), 1, f) != 1 || n < 0) return 2;
  std::vector<double> a(4 * n);
  if (std::fread(a.data(), sizeof(double), a.size(), f) != a.size()) return 2;
  std::fclose(f);
  std::vector<PARTICLE> part(n);
  for (long long i = 0; i < n; i++) {
    part[i].x = a[i];
    part[i].y = a[n + i];
    part[i].z = a[2 * n + i];
  }
  output_potential((int)n, part.data(), a.data() + 3 * n, argv[2]);
  if (*bit_tree3d_last_error()) {
    std::printf("%s\n", bit_tree3d_last_error());
    return 1;
  }
  return 0;
}
