// mcmeasure SEED X Z: exact area of the desert at block (X, 256, Z), the measurement deploy/gpipe.sh runs
// for every CANDIDATE line (deploy/gpipe.sh:9).  MC-Measure itself is an un-vendored submodule of the
// reference; this tool gives the same number -- the 4-connected flood on the 1:4 grid with rivers bridged
// but not counted, area x16 (the step-1 flood of tools/dflood.cpp, which reproduces MC-Measure's counts) --
// computed on the GPU, and prints it in the fields the fleet scripts parse ("1:4 Size: N | Blocks^2 Size: M",
// scripts/log_finds.py:13, deploy/status.py:9).
#include "dsgpu.h"
#include <cstdio>
#include <string>

int main(int argc, char **argv) {
    if (argc < 4) { fprintf(stderr, "mcmeasure SEED X Z\n"); return 2; }
    const uint64_t seed = std::stoull(argv[1]);
    const int x = std::stoi(argv[2]), z = std::stoi(argv[3]);
    if (dsg_init(0, 0.35f) != DSG_OK) { fprintf(stderr, "mcmeasure: %s\n", dsg_last_error()); return 3; }
    const int32_t xz[2] = {x >> 2, z >> 2};
    int8_t st = 0;
    if (dsg_points(seed, DSG_PRED_DESERT, 0.f, xz, 1, &st) != DSG_OK) { fprintf(stderr, "mcmeasure: %s\n", dsg_last_error()); return 3; }
    if (st != 2) { printf("Biome at (%d, 256, %d) is not Desert | 1:4 Size: 0 | Blocks^2 Size: 0\n", x, z); return 1; }
    dsg_flood_req q{seed, x >> 2, z >> 2, 1, 20000, 0, DSG_PRED_DESERT, 0.35f, 0};
    dsg_area a{};
    if (dsg_flood(&q, &a) != DSG_OK) { fprintf(stderr, "mcmeasure: %s\n", dsg_last_error()); return 3; }
    printf("Biome: Desert at (%d, 256, %d) | 1:4 Size: %llu | Blocks^2 Size: %llu%s\n", x, z, (unsigned long long)a.cells,
           (unsigned long long)(a.cells * 16), a.edge ? " | window edge reached" : "");
    return 0;
}
