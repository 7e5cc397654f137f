"""Test infrastructure: build-time copy of the reference's Setka.cpp whose
constructor sorts the three tracked-face lines once instead of once per face.

``Setka::Setka(N1..M4)`` (Setka.cpp:1008-1049) walks ``All_Gran`` and, inside
that loop, re-sorts ``Line_Contact``, ``Line_Inner`` and ``Line_Outer`` by the
polar angle of the face centres after every face, so the constructor costs
O(faces x line length x log) comparisons, each two ``atan`` calls: ~70 s at
200k cells and ~14 min at 938k cells.  Sorting a list whose keys are distinct
gives one order whatever the order it starts from, so sorting each list once,
at the last face of the loop, gives the same lists.  This script writes a
copy with each of those three ``sort(`` calls guarded by "this is the loop's
last face"; nothing else changes, and the step functions are untouched.

The copy is written under ``oracle/_ref`` (git-ignored) and compiled into the
CPU-baseline library only (``libgelios_ref_fast.so``); the parity library is
built from the unmodified file.  ``tests/test_oracle_pin.py`` checks that the
two constructors export identical grids.

    python hoist_line_sort.py <reference Setka.cpp> <output Setka.cpp>
"""
from __future__ import annotations

import sys
from pathlib import Path

LINES = (b"Line_Contact", b"Line_Inner", b"Line_Outer")
GUARD = b"if (&i == &this->All_Gran.back()) "
END_OF_CONSTRUCTOR = b'"Vsego tochek = "'


def patch(src: bytes) -> bytes:
    end = src.find(END_OF_CONSTRUCTOR)
    if end < 0:
        raise SystemExit("constructor end marker not found")
    head, tail = src[:end], src[end:]
    for name in LINES:
        call = b"sort(this->" + name + b".begin()"
        if head.count(call) != 1:
            raise SystemExit(f"expected one {call!r} in the constructor, found {head.count(call)}")
        k = head.find(call)
        loop = head.rfind(b"for (auto& i : this->All_Gran)", 0, k)
        if loop < 0 or head.find(b"for (", loop + 1, k) >= 0:
            raise SystemExit(f"{call!r} is not directly inside the All_Gran loop")
        head = head[:k] + GUARD + head[k:]
    return head + tail


def main(argv: list[str]) -> None:
    src, dst = Path(argv[1]), Path(argv[2])
    out = patch(src.read_bytes())
    dst.parent.mkdir(parents=True, exist_ok=True)
    dst.write_bytes(out)


if __name__ == "__main__":
    main(sys.argv)
