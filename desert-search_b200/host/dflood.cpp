// dflood SEED X Z [STEP=4]: exact bridged desert flood at Y=256 on the GPU (tools/dflood.cpp).
// X, Z are block coordinates; STEP is the flood lattice in quarts (1 = exact, MC-Measure's count).
// Same arguments, output line, messages and exit codes as the reference tool; the flood runs in
// libdsgpu (dsg_flood) instead of a CPU DFS.
#include "dsgpu.h"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

int main(int argc, char **argv) {
    if (argc < 4) { fprintf(stderr, "dflood SEED X Z [STEP=4]\n"); return 2; }
    const uint64_t seed = std::stoull(argv[1]);
    const int qx = std::stoi(argv[2]) >> 2, qz = std::stoi(argv[3]) >> 2, step = argc > 4 ? std::stoi(argv[4]) : 4;
    if (step < 1) { fprintf(stderr, "dflood: STEP must be >= 1\n"); return 2; }
    if (dsg_init(0, 0.35f) != DSG_OK) { fprintf(stderr, "dflood: %s\n", dsg_last_error()); return 3; }
    const int32_t xz[2] = {qx, qz};
    int8_t st = 0;
    if (dsg_points(seed, DSG_PRED_DESERT, 0.f, xz, 1, &st) != DSG_OK) { fprintf(stderr, "dflood: %s\n", dsg_last_error()); return 3; }
    if (st != 2) { fprintf(stderr, "(%d, %d) is not desert at Y=256\n", qx * 4, qz * 4); return 1; }
    dsg_flood_req q{seed, qx, qz, step, 20000 / step, 0, DSG_PRED_DESERT, 0.35f, 0};
    dsg_area a{};
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = dsg_flood(&q, &a);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != DSG_OK) { fprintf(stderr, "dflood: %s\n", dsg_last_error()); return 3; }
    const double cells = double(a.cells) * step * step;
    printf("Desert at step %d: %.0f cells (1:4) = %.0f blocks^2%s  [%.1f s]\n", step, cells, cells * 16, a.edge ? " (hit flood window edge)" : "", sec);
    return 0;
}
