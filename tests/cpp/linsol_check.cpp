// Drives the C ABI through the C++ linsol mirror (nga2_b200/csrc/bbmg_linsol.hpp)
// the way an NGA2 flow solver drives its pressure solver: fill stc/opr, init,
// setup, fill rhs/sol, solve, read it/rerr.  Prints "it rerr" on success;
// exit code 2 when no CUDA device is present.
#include <cmath>
#include <cstdio>
#include <exception>

#include "../../nga2_b200/csrc/bbmg_linsol.hpp"

int main() {
    const int n = 16, no = 2;
    nga2::bbmg_linsol ps("Pressure", n, n, n, true, true, true, no, 7);
    const int stc[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int st = 0; st < 7; st++)
        for (int d = 0; d < 3; d++) ps.stc[3 * st + d] = stc[st][d];
    const int m = n + 2 * no;
    const double h = 1.0 / n, pi = 3.14159265358979323846;
    for (int k = 0; k < m; k++)
        for (int j = 0; j < m; j++)
            for (int i = 0; i < m; i++) {
                size_t c = ((size_t)k * m + j) * m + i;
                // -vol * Laplacian with vol = h^3 (incomp_class.f90:766-785 on a uniform grid)
                ps.opr[7 * c + 0] = 6.0 * h;
                for (int st = 1; st < 7; st++) ps.opr[7 * c + st] = -h;
                double x = (i - no + 0.5) * h, y = (j - no + 0.5) * h, z = (k - no + 0.5) * h;
                ps.rhs[c] = std::sin(2 * pi * x) * std::cos(4 * pi * y) * std::sin(2 * pi * z);
                ps.sol[c] = 0.0;
            }
    try {
        ps.maxit = 50;
        ps.rcvg = 1e-10;
        ps.init(nga2::bbmg_linsol::pcg_bbox);
        ps.setup();
        ps.solve();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    std::printf("%d %.3e\n", ps.it, ps.rerr);
    return (ps.rerr <= 1e-10 && ps.it > 0) ? 0 : 1;
}
