#!/usr/bin/env python3
"""Regenerate worldgen.bin, the constant game data the pipeline needs.

The data is the Minecraft 26.3 overworld biome parameter tree, its parameter
intervals, the terrain-offset spline graph and the tree's level strides (all
generated from Cubiomes, MIT), plus the measured 40x40 desert-probability
table of the low-octave proxy.  The reference keeps them as C++ arrays in
src/worldgen_data.hpp and src/desert_dtable.hpp.  Rather than parse C++ text,
this script lets the C++ compiler read those headers and dump the values
bit for bit into a small sectioned binary file (layout below), which the GPU
library and the host tools embed at build time.

Layout (little endian):
  b"DSWG", u32 version=1
  sections, each: 4-byte tag, u32 count, payload
    SPLN  count=N   i32 axis[N], i32 npts[N], f32 value[N], f32 knot[N*12],
                    f32 slope[N*12], i32 kid[N*12]
    PARM  count=M   i32 lo_hi[M*2]
    TREE  count=K   u64 node[K]
    STEP  count=S   i32 stride[S]
    DPRB  count=1600 f32 prob[40*40]   (row = C bin, column = E bin)

Usage: python extract_worldgen.py REFERENCE_ROOT [OUT]
"""
import os
import subprocess
import sys
import tempfile

DUMPER = r'''
#include <cstdio>
#include <cstdint>
#include <iterator>
#include "worldgen_data.hpp"
#include "desert_dtable.hpp"
using namespace standalone;
static void put(const void *p, size_t n) { fwrite(p, 1, n, stdout); }
static void tag(const char *t, uint32_t n) { put(t, 4); put(&n, 4); }
int main() {
    put("DSWG", 4); uint32_t ver = 1; put(&ver, 4);
    const uint32_t N = std::size(splines);
    tag("SPLN", N);
    for (uint32_t i = 0; i < N; i++) { int32_t v = splines[i].axis; put(&v, 4); }
    for (uint32_t i = 0; i < N; i++) { int32_t v = splines[i].n; put(&v, 4); }
    for (uint32_t i = 0; i < N; i++) { float v = splines[i].value; put(&v, 4); }
    for (uint32_t i = 0; i < N; i++) put(splines[i].x, 48);
    for (uint32_t i = 0; i < N; i++) put(splines[i].slope, 48);
    for (uint32_t i = 0; i < N; i++) put(splines[i].child, 48);
    tag("PARM", std::size(parameters)); put(parameters, sizeof(parameters));
    tag("TREE", std::size(tree)); put(tree, sizeof(tree));
    tag("STEP", std::size(steps)); put(steps, sizeof(steps));
    tag("DPRB", 1600); put(desert_pass_prob, sizeof(desert_pass_prob));
    return 0;
}
'''


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF")
    if not ref:
        sys.exit("usage: extract_worldgen.py REFERENCE_CHECKOUT [OUT] (or REF=... in the environment)")
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "worldgen.bin")
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "dump.cpp")
        exe = os.path.join(td, "dump")
        with open(src, "w") as f:
            f.write(DUMPER)
        subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ref, "src"), src, "-o", exe])
        blob = subprocess.check_output([exe])
    with open(out, "wb") as f:
        f.write(blob)
    print(f"wrote {out}: {len(blob)} bytes")


if __name__ == "__main__":
    main()
