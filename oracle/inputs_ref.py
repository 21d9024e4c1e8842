"""Restatement of the reference's input reading (TEST INFRASTRUCTURE ONLY: imported by
tests/ as the checker of the library's dft.in / solute.in readers, never by the product).

  put_input_in_character_array   src/module_input.f90:654-732
  input_dp / input_int / ...     src/module_input.f90:60-557 (value from columns len+4..len+50)
  input_log                      src/module_input.f90:386-427 (first character T/t or F/f)
  read_solute                    src/module_solute.f90:36-52
  mv_solute_to_center            src/module_solute.f90:146-187
"""
from __future__ import annotations

import math


def clean_lines(text: str) -> list[str]:
    out = []
    for raw in text.split("\n"):
        rec = raw.rstrip("\r")[:100].strip(" ")
        if "#" in rec:
            rec = rec[:rec.index("#")]
        rec = rec.strip(" ")
        if rec:
            out.append(rec)
    return out


def field_of(lines: list[str], tag: str):
    j = len(tag)
    for l in lines:
        rec = l.ljust(100)
        if rec[:j] == tag and rec[j] == " ":
            return rec[j + 3:j + 50]
    return None


def items_of(field: str) -> list[str]:
    out = []
    for tok in field.split("/")[0].replace(",", " ").replace("\t", " ").split():
        if "*" in tok and tok.split("*")[0].isdigit():
            r, c = tok.split("*", 1)
            out += [c] * int(r)
        else:
            out.append(tok)
    return out


def real_of(tok: str) -> float:
    t = tok
    for c in "dDqQ":
        t = t.replace(c, "e")
    return float(t)


def int_of(tok: str) -> int:
    if not tok.lstrip("+-").isdigit():
        raise ValueError(tok)
    return int(tok)


def log_of(field: str) -> bool:
    it = items_of(field)
    c = it[0][0] if it and it[0] else " "
    if c in "Tt":
        return True
    if c in "Ff":
        return False
    raise ValueError(field)


def read_solute(text: str, scale: float = 1.0):
    lines = text.split("\n")[1:]
    k = 0
    while not lines[k].split():
        k += 1
    n = int(lines[k].split()[0])
    rest = lines[k + 2:]
    sites, buf, li = [], [], 0
    while len(sites) < n:
        while len(buf) < 8:
            buf += rest[li].replace(",", " ").split()
            li += 1
        sites.append((int(buf[0]), *[real_of(x) for x in buf[1:7]], int(buf[7])))
        buf = []
    q = [s[1] * scale for s in sites]
    return q, [s[2] for s in sites], [s[3] for s in sites], [list(s[4:7]) for s in sites], [s[7] for s in sites]


def center(xyz, box, translate=True):
    out = [list(r) for r in xyz]
    n = len(out)
    if translate and n:
        for d in range(3):
            mean = 0.0
            for r in out:  # sequential, as Fortran SUM; Python's sum() compensates since 3.12
                mean += r[d]
            mean /= float(n)
            for r in out:
                r[d] = r[d] + box[d] / 2.0 - mean
    for r in out:
        for d in range(3):
            # MODULO for reals as gfortran evaluates it: fmod, then + P when the signs differ
            m = math.fmod(r[d], box[d])
            if m != 0.0 and (m < 0.0) != (box[d] < 0.0):
                m += box[d]
            r[d] = m
    return out
