"""Reading the text dumps of driver/shared.cpp:96-189 (the driver's --dump).

A dump lists, per tile, the state fields, the seven work arrays, the 1-D
geometry and volume / xarea / yarea, each as a block that starts with a
header line "name(rank) [extents]".  The work arrays are scratch that a
phase fills and the next overwrites (the b200 model keeps them on chip and
reports zeros), so comparisons drop their blocks: filtered().  parse_arrays()
returns the 2-D blocks as numpy arrays, indexed [i][j] (x, then y) as the
dump writes them.
"""
import re

import numpy as np

HEADER = re.compile(r"^(\w+)\((\d)\) \[(\d+)(?:x(\d+))?\]$")


def blocks(text):
    """(name, rank, extents, lines) of every array block, in order; other lines as (None, ...)."""
    out, cur = [], None
    for line in text.split("\n"):
        m = HEADER.match(line)
        if m:
            cur = [m.group(1), int(m.group(2)), tuple(int(x) for x in m.group(3, 4) if x), [line]]
            out.append(cur)
        elif line.startswith("\tTile[") or line.startswith("info.") or "=" in line and cur is None:
            cur = None
            out.append([None, 0, (), [line]])
        elif cur is not None:
            cur[3].append(line)
        else:
            out.append([None, 0, (), [line]])
    return out


def filtered(text):
    """The dump text without the work_array blocks."""
    keep = []
    for name, _, _, lines in blocks(text):
        if name is not None and name.startswith("work_array"):
            continue
        keep.extend(lines)
    return "\n".join(keep)


def parse_arrays(text):
    """{name: array} of the rank-2 blocks (all-zero blocks, printed "(0.0)", as zeros)."""
    out = {}
    for name, rank, ext, lines in blocks(text):
        if name is None or rank != 2:
            continue
        body = " ".join(lines[1:])
        if "(0.0)" in body:
            out[name] = np.zeros(ext)
            continue
        vals = [float(x) for x in body.replace("\t", " ").split(",") if x.strip()]
        out[name] = np.array(vals).reshape(ext)
    return out
