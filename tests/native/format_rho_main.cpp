// Writes rho_<t>.dat text with cosenu::format_rho from a binary input:
//   int32 nz, int32 nvz, int32 nthreads, double Z[nz], double vz[nvz],
//   double state[8][nvz][nz]
// usage: format_rho_main <in.bin> <out.dat>
#include <cstdio>
#include <vector>

#include "cosenu_format.hpp"

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int h[3];
    if (std::fread(h, sizeof(int), 3, f) != 3) return 2;
    const int nz = h[0], nvz = h[1], nthreads = h[2];
    std::vector<double> Z(nz), vz(nvz), s((size_t)8 * nvz * nz);
    bool ok = std::fread(Z.data(), 8, nz, f) == (size_t)nz &&
              std::fread(vz.data(), 8, nvz, f) == (size_t)nvz &&
              std::fread(s.data(), 8, s.size(), f) == s.size();
    std::fclose(f);
    if (!ok) return 2;
    const double *comp[8];
    for (int c = 0; c < 8; ++c) comp[c] = s.data() + (size_t)c * nvz * nz;
    return cosenu::format_rho(argv[2], nz, nvz, Z.data(), vz.data(), comp, nz, nthreads) ? 0 : 1;
}
