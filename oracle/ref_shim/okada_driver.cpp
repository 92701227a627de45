// ORACLE test infrastructure: runs the reference's okada::okadamapFull
// (src/okada.cpp, compiled where it lies) on points read from a file.
// Usage: okada_driver points.bin out.bin   (points: n, then n x, n y as
// doubles in Mercator km).  The reference loops over five fault files of
// which only data/indianOceanFault1.txt ships; it throws when it reaches the
// second, after the first fault's uplift has been added -- which is the
// displacement recorded here.
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "okada.h"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    double nd = 0;
    if (std::fread(&nd, sizeof(double), 1, f) != 1) return 2;
    const int n = (int)nd;
    std::vector<double> x(n), y(n), q(3 * (size_t)n, 0.0);
    if (std::fread(x.data(), sizeof(double), n, f) != (size_t)n) return 2;
    if (std::fread(y.data(), sizeof(double), n, f) != (size_t)n) return 2;
    std::fclose(f);
    okada o(n);
    try {
        o.okadamapFull(1, x.data(), y.data(), q.data());
    } catch (const std::invalid_argument&) {
        // data/indianOceanFault2.txt is absent: fault 1 has been applied
    }
    FILE* g = std::fopen(argv[2], "wb");
    for (int i = 0; i < n; ++i) std::fwrite(&q[3 * (size_t)i], sizeof(double), 1, g);
    std::fclose(g);
    return 0;
}
