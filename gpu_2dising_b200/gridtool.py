"""Headless gridstates.bin / gridinput.bin tool.

The reference selects a committor start grid interactively: its pygame
viewer shows gridstates.bin frames and its `w` key writes the grid on screen
to gridinput.bin (tools/vis_gridstates.py:109-114).  This does the same
without a display:

    python -m gpu_2dising_b200.gridtool info gridstates.bin
    python -m gpu_2dising_b200.gridtool extract gridstates.bin FRAME GRID [-o gridinput.bin]
    python -m gpu_2dising_b200.gridtool show gridstates.bin FRAME GRID

FRAME counts frames from 0 in file order; GRID is the replica index.  `show`
prints the grid as text ('#' for +1, '.' for -1) with its magnetisation.
"""
from __future__ import annotations

import argparse
import sys

from . import engine


def frames(path):
    """(index, L, ngrids, isweep) of every frame in a gridstates.bin file."""
    out, k = [], 0
    while True:
        try:
            L, ng, isw, _ = engine.read_frame(path, k, grids=False)
        except Exception:
            return out
        out.append((k, L, ng, isw))
        k += 1


def extract(path, iframe, igrid, out="gridinput.bin"):
    """Writes grid `igrid` of frame `iframe` as gridinput.bin; returns it."""
    L, ng, isw, g = engine.read_frame(path, iframe)
    if not 0 <= igrid < ng:
        raise ValueError(f"grid index {igrid} out of range (frame has {ng} grids)")
    engine.write_input_grid(out, g[igrid])
    return g[igrid]


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m gpu_2dising_b200.gridtool",
                                 description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("info")
    a.add_argument("gridstates")
    for name in ("extract", "show"):
        b = sub.add_parser(name)
        b.add_argument("gridstates")
        b.add_argument("frame", type=int)
        b.add_argument("grid", type=int)
        if name == "extract":
            b.add_argument("-o", "--output", default="gridinput.bin")
    args = ap.parse_args(argv)
    if args.cmd == "info":
        fr = frames(args.gridstates)
        for k, L, ng, isw in fr:
            print(f"frame {k:5d}  isweep {isw:10d}  L {L}  ngrids {ng}")
        return 0 if fr else 1
    if args.cmd == "extract":
        g = extract(args.gridstates, args.frame, args.grid, args.output)
        print(f"grid {args.grid} of frame {args.frame} written to {args.output} "
              f"(m = {g.mean():.6f})")
        return 0
    L, ng, isw, g = engine.read_frame(args.gridstates, args.frame)
    if not 0 <= args.grid < ng:
        print(f"grid index {args.grid} out of range (frame has {ng} grids)", file=sys.stderr)
        return 1
    x = g[args.grid]
    print(f"# frame {args.frame}, isweep {isw}, grid {args.grid}, m = {x.mean():.6f}")
    for row in x:
        print("".join("#" if v == 1 else "." for v in row))
    return 0


if __name__ == "__main__":
    sys.exit(main())
