#!/usr/bin/env python
"""Generate tips2011_data.h: the TIPS-2011 partition-sum tables.

The HITRAN reader of the reference takes Q(T) from the TIPS-2011 Fortran
routine BD_TIPS_2011 (Readers/HITRAN/BD_TIPS_2011_v1p0.for, called at
Readers/HITRAN/HITRANStateReader.cpp:62,95,128).  Its data are, per
molecule subroutine QT_<name>, the state-independent degeneracies xgj(iso)
and the partition sums QofT(iso, 1..119) at the 119 temperatures Tdat =
60, 85, ..., 3010 K, written as DATA statements; the molecule number of each
subroutine is the dispatch `IF(MOL.EQ.n) THEN / CALL QT_<name>` (:73-345).
Molecules 34 and 39 are dispatched to gi = 0, Q = 0 (:253-258, :280-284).

The literals carry no D exponent, so a Fortran compiler stores each as a
default (single precision) REAL converted to the DOUBLE PRECISION array:
the header keeps that widened float value (written as a float literal with
an f suffix, widened by the C++ compiler the same way).

    python gexs_b200/host/gen_tips2011.py <path of BD_TIPS_2011_v1p0.for> [output]
(output defaults to tips2011_data.h beside this script)
"""
import os
import re
import sys

NT = 119


def parse(path):
    lines = open(path, encoding="latin-1").read().split("\n")
    # dispatch: molecule number -> subroutine
    disp = {}
    for i, l in enumerate(lines):
        m = re.match(r"\s+IF\s*\(\s*MOL\s*\.EQ\.\s*(\d+)\s*\)\s*THEN", l, re.I)
        if m:
            c = re.search(r"CALL\s+(QT_\w+)", lines[i + 1], re.I)
            disp[int(m.group(1))] = c.group(1).upper() if c else None
    # join fixed-form continuation lines (non-blank in column 6)
    stmts = []
    for l in lines:
        if not l or l[0] in "cC*!":
            continue
        if len(l) > 5 and l[5] not in " 0" and stmts:
            stmts[-1] += " " + l[6:]
        else:
            stmts.append(l)
    subs = {}
    cur = None
    for s in stmts:
        m = re.match(r"\s+Subroutine\s+(QT_\w+)", s, re.I)
        if m:
            cur = m.group(1).upper()
            subs[cur] = {"gi": None, "q": {}}
            continue
        if cur is None:
            continue
        m = re.match(r"\s+data\s+xgj\s*/(.*)/", s, re.I)
        if m:
            subs[cur]["gi"] = [float(v) for v in m.group(1).replace(",", " ").split()]
            continue
        m = re.match(r"\s+data\s+\(QofT\(\s*(\d+)\s*,J\)\s*,\s*J\s*=\s*1\s*,\s*119\)\s*/(.*)/", s, re.I)
        if m:
            vals = m.group(2).replace(",", " ").split()
            assert len(vals) == NT, (cur, m.group(1), len(vals))
            subs[cur]["q"][int(m.group(1))] = vals
    return disp, subs


def main():
    src = sys.argv[1]
    disp, subs = parse(src)
    mols = []
    for mol in range(1, max(disp) + 1):
        name = disp.get(mol)
        if name is None:
            mols.append((mol, None, [], []))
            continue
        d = subs[name]
        niso = len(d["gi"])
        assert sorted(d["q"]) == list(range(1, niso + 1)), (name, sorted(d["q"]), niso)
        mols.append((mol, name, d["gi"], [d["q"][i] for i in range(1, niso + 1)]))
    out = sys.argv[2] if len(sys.argv) > 2 else \
        os.path.join(os.path.dirname(os.path.abspath(__file__)), "tips2011_data.h")
    w = []
    w.append("/* tips2011_data.h - generated by gen_tips2011.py from the TIPS-2011 DATA")
    w.append(" * statements (Readers/HITRAN/BD_TIPS_2011_v1p0.for); do not edit.")
    w.append(" * Per molecule (HITRAN number, dispatch of BD_TIPS_2011): the")
    w.append(" * isotopologue count, gi per isotopologue and Q at the 119 temperatures")
    w.append(" * 60, 85, ..., 3010 K, each value the single-precision literal widened")
    w.append(" * to double as the Fortran DATA statement stores it. */")
    w.append("#pragma once")
    w.append("namespace gexs_tips {")
    w.append("constexpr int kNT = %d;" % NT)
    w.append("constexpr int kMolecules = %d;" % len(mols))
    total = sum(len(m[2]) for m in mols)
    w.append("constexpr int kIsotopologues = %d;" % total)
    offs, o = [], 0
    for m in mols:
        offs.append(o)
        o += len(m[2])
    w.append("/* first row of molecule m (1-based) is kFirst[m - 1]; its count kCount[m - 1]")
    w.append(" * (0: molecule dispatched to gi = 0, Q = 0) */")
    w.append("constexpr int kFirst[kMolecules] = {%s};" % ", ".join(str(v) for v in offs))
    w.append("constexpr int kCount[kMolecules] = {%s};" % ", ".join(str(len(m[2])) for m in mols))
    w.append("constexpr float kGi[kIsotopologues] = {")
    gis = []
    for m in mols:
        gis += ["%sf" % repr(float(g)) for g in m[2]]
    for i in range(0, len(gis), 8):
        w.append("    " + ", ".join(gis[i:i + 8]) + ",")
    w.append("};")
    w.append("constexpr float kQ[kIsotopologues][kNT] = {")
    for m in mols:
        for iso, row in enumerate(m[3]):
            w.append("    /* molecule %d %s, isotopologue %d */ {" % (m[0], m[1], iso + 1))
            for i in range(0, NT, 6):
                w.append("        " + ", ".join(v.upper().replace("E+", "e+").replace("E-", "e-") + "f"
                                                for v in row[i:i + 6]) + ",")
            w.append("    },")
    w.append("};")
    w.append("}  // namespace gexs_tips")
    open(out, "w").write("\n".join(w) + "\n")
    print(out, len(mols), "molecules", total, "isotopologues")


if __name__ == "__main__":
    main()
