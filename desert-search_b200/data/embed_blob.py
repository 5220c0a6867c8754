#!/usr/bin/env python3
"""Turn a binary file into a C translation unit: `const unsigned char SYM[]` and `SYM_len`.

Usage: python embed_blob.py IN.bin OUT.c SYMBOL
"""
import sys


def main():
    src, dst, sym = sys.argv[1], sys.argv[2], sys.argv[3]
    data = open(src, "rb").read()
    with open(dst, "w") as f:
        f.write(f"/* generated from {src.split('/')[-1]} by embed_blob.py */\n")
        f.write(f"const unsigned char {sym}[{len(data)}] __attribute__((aligned(16))) = {{\n")
        for i in range(0, len(data), 24):
            f.write(",".join(str(b) for b in data[i:i + 24]) + ",\n")
        f.write("};\n")
        f.write(f"const unsigned long {sym}_len = {len(data)};\n")


if __name__ == "__main__":
    main()
