"""Result files in the reference's formats, so that results served or solved here can be compared
with reference runs file for file.

WriterHomogenization (src/WriterHomogenization.cpp:40-88): one CSV row per written load step,
``t, eps_macro(t)..., <sigma>...`` (the current macroscale strain, then the homogenized stress,
both in Voigt order), every value as a C++ stream with precision 16 prints it (%.16g).  The file
is truncated at step 0 and appended to afterwards.
"""
from __future__ import annotations

from typing import Sequence


def _f16(x: float) -> str:
    """A double as std::ostream prints it after precision(16) (default float field: %.16g)."""
    return "%.16g" % x


def homogenization_row(t: float, macro: Sequence[float], homogenized: Sequence[float] = ()) -> str:
    """WriterHomogenization::writeFromStream: the row of one load step (with its newline).
    Without homogenized values the row holds t and the macroscale strain only."""
    vals = [_f16(t)] + [_f16(v) for v in macro] + [_f16(v) for v in homogenized]
    return ",".join(vals) + "\n"


def write_homogenization(filename: str, t: float, step: int, macro: Sequence[float],
                         homogenized: Sequence[float] = ()) -> None:
    """WriterHomogenization::writeConsecutive: step 0 starts the file, later steps append."""
    with open(filename, "w" if step == 0 else "a") as f:
        f.write(homogenization_row(t, macro, homogenized))


def homogenization_table(t: float, strains: Sequence[Sequence[float]], stresses: Sequence[Sequence[float]]) -> str:
    """The rows of several load cases solved at the same load fraction t (e.g. the unit
    macroscale strains of a homogenization request), one row per case."""
    return "".join(homogenization_row(t, e, s) for e, s in zip(strains, stresses))
