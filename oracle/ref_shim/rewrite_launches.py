"""Mechanical rewrite of CUDA launch syntax for the host build of the
reference's engine (test infrastructure only).

Reads a .cu file and writes a C++ file that first includes the CPU runtime
emulation (cuda_host_shim.h) and then the original text, with every
``kernel<<<grid, block>>>(args)`` turned into
``shim_launch(grid, block, kernel, args)``. Nothing else is changed.

Usage: python rewrite_launches.py <in.cu> <out.cpp>
"""
import re
import sys

LAUNCH = re.compile(r"(\w+)\s*<<<\s*(.+?)\s*>>>\s*\(", re.S)


def rewrite(text: str) -> str:
    out, n = LAUNCH.subn(lambda m: f"shim_launch({m.group(2)}, {m.group(1)}, ", text)
    if n == 0:
        raise SystemExit("no kernel launches found")
    return '#include "cuda_host_shim.h"\n' + out


def main() -> None:
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        text = f.read()
    with open(dst, "w") as f:
        f.write(f"// generated from {src} by rewrite_launches.py -- do not edit\n")
        f.write(rewrite(text))


if __name__ == "__main__":
    main()
