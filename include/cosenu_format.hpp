// cosenu_format.hpp -- text formats of the reference's snapshot files, written
// fast (header-only C++17, no CUDA).
//
// rho_<t>.dat (NuOsc::dump_rho, src/snaps.hpp:187-218): for every z (outer)
// and v (inner) a line "Z vz ee xx ex_re ex_im bee bxx bex_re bex_im" with tab
// separators, a blank line after each z block.  The reference streams with
// std::ofstream and sets setprecision(16) after the first "Z vz" pair, so the
// very first Z and vz print with the default precision 6 and every later value
// with 16 significant digits in the default float format -- i.e. printf's
// "%.6g" and "%.16g".  format_rho builds the same bytes with snprintf, the z
// blocks split across threads, and writes them in order.
#pragma once

#include <algorithm>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

namespace cosenu {

// One z block (all v lines of z index j, then the blank line) appended to out.
// comp[c] points at interior cell (0, 0) of component c; rows are ld apart.
inline void format_rho_block(std::string &out, int j, int nvz, const double *Z, const double *vz,
                             const double *const comp[8], long long ld, bool first_block)
{
    char buf[512];
    for (int i = 0; i < nvz; ++i) {
        const long long q = (long long)i * ld + j;
        const bool first = first_block && i == 0;
        int n = std::snprintf(buf, sizeof buf, first ? "%.6g\t%.6g\t" : "%.16g\t%.16g\t", Z[j],
                              vz[i]);
        n += std::snprintf(buf + n, sizeof buf - n,
                           "%.16g\t%.16g\t%.16g\t%.16g\t%.16g\t%.16g\t%.16g\t%.16g\n",
                           comp[0][q], comp[1][q], comp[2][q], comp[3][q], comp[4][q], comp[5][q],
                           comp[6][q], comp[7][q]);
        out.append(buf, n);
    }
    out.push_back('\n');
}

// Writes rho_<t>.dat to `path` with up to `nthreads` formatting threads (0:
// one per hardware thread); returns false if the file cannot be written.
inline bool format_rho(const std::string &path, int nz, int nvz, const double *Z, const double *vz,
                       const double *const comp[8], long long ld, int nthreads = 0)
{
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    nthreads = std::max(1, std::min(nthreads, std::max(1, nz / 16)));
    std::vector<std::string> parts(nthreads);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) {
        th.emplace_back([&, t] {
            const int j0 = (int)((long long)nz * t / nthreads);
            const int j1 = (int)((long long)nz * (t + 1) / nthreads);
            parts[t].reserve((size_t)(j1 - j0) * nvz * 200);
            for (int j = j0; j < j1; ++j) format_rho_block(parts[t], j, nvz, Z, vz, comp, ld, j == 0);
        });
    }
    for (auto &x : th) x.join();
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = true;
    for (auto &p : parts) ok = ok && std::fwrite(p.data(), 1, p.size(), f) == p.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace cosenu
