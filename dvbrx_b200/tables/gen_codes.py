"""Generate ``dvbrx_b200/csrc/codes_gen.h``: the DVB-S2 / S2X / T2 LDPC parity
address tables and the FEC parameter rows, in this project's own layout.

The tables are normative data of ETSI EN 302 307-1 (Annexes B and C),
EN 302 307-2 and EN 302 755 (Annexes A and B).  This script extracts them from
the reference receiver's generated headers (libdvbrx/src/ldpc_tables.h and
libdvbrx/src/fec_table.h, which the reference itself generates from
gr-dvbs2rx) and re-emits them as:

* per table: N, K and a list of 360-bit column groups, each group given by the
  parity-accumulator addresses of its first bit (the standard's own form);
* the rate-string -> table maps for normal and short frames
  (reference: libdvbrx/src/ldpc_tables.h:2345-2407);
* the rate-string -> (kbch, nbch, t) rows used by drx_fec_lookup
  (reference: libdvbrx/src/fec_table.h:3-63, libdvbrx/src/bch.c:25-41);
* the DVB-S2/S2X constellations by PLS code with their bit-interleaver column
  orders (reference: libdvbrx/src/const_tables.h, consumed by
  libdvbrx/src/demap.c:164-200), used by this project's channel model.

Usage: python gen_codes.py <reference root> <output header>
"""
import re
import sys


def parse_ldpc(text):
    arrays = {}
    for m in re.finditer(r"static const uint16_t (\w+)\[\] = \{([^}]*)\};", text):
        arrays[m.group(1)] = [int(v) for v in m.group(2).replace("\n", " ").split(",") if v.strip()]
    tables = {}
    for m in re.finditer(
        r"static const struct ldpc_table (\w+) = \{\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\w+),\s*(\w+),\s*(\w+)\s*\};",
        text,
    ):
        name = m.group(1)
        M, N, K, lmc, lt, dmax = (int(m.group(i)) for i in range(2, 8))
        deg, ln, pos = arrays[m.group(8)], arrays[m.group(9)], arrays[m.group(10)]
        runs = []
        for d, l in zip(deg, ln):
            if l == 0:
                break
            runs.append((d, l))
        assert M == 360
        assert sum(d * l for d, l in runs) == len(pos), name
        assert sum(l for _, l in runs) * 360 == K, name
        tables[name] = dict(N=N, K=K, links_max_cn=lmc, links_total=lt, deg_max=dmax, runs=runs, pos=pos)
    maps = {}
    for which in ("normal", "short"):
        m = re.search(r"static const struct ldpc_map ldpc_map_%s\[\] = \{(.*?)\};" % which, text, re.S)
        maps[which] = re.findall(r'\{\s*"(\w+)",\s*&(\w+)\s*\}', m.group(1))
    return tables, maps


def parse_fec(text):
    rows = {}
    for which in ("normal", "short"):
        m = re.search(r"static const struct fec_row fec_%s\[\] = \{(.*?)\};" % which, text, re.S)
        rows[which] = [
            (r, int(a), int(b), int(c))
            for r, a, b, c in re.findall(r'\{\s*"(\w+)",\s*(\d+),\s*(\d+),\s*(\d+)\s*\}', m.group(1))
        ]
    return rows


def parse_const(text):
    """Constellation rows: PLS code, name, rate, short flag, bits per symbol,
    interleaver column order and the points by bit label (MSB first)."""
    rows = []
    for m in re.finditer(
        r'\{\s*(0x[0-9a-f]+),\s*"(\w+)",\s*"(\w+)",\s*(\d),\s*(\d),\s*\{([^}]*)\},\s*\{(.*?)\}\s*\}\s*\},',
        text, re.S,
    ):
        order = [int(v) for v in m.group(6).split(",")]
        pts = [float(v.rstrip("f")) for v in re.findall(r"-?\d+\.\d+f", m.group(7))]
        bits = int(m.group(5))
        assert len(pts) == 2 << bits, (m.group(1), len(pts))
        rows.append((int(m.group(1), 16), m.group(2), m.group(3), int(m.group(4)), bits, order, pts))
    return rows


def emit(tables, maps, fec, out, consts=()):
    names = sorted(tables)
    idx = {n: i for i, n in enumerate(names)}
    w = out.write
    w("/* Generated by dvbrx_b200/tables/gen_codes.py: ETSI EN 302 307-1/-2 and\n"
      " * EN 302 755 LDPC parity-accumulator address tables and FEC rows.\n"
      " * Do not edit. */\n#pragma once\n#include \"codes_types.h\"\n\n")
    for n in names:
        t = tables[n]
        w("static const uint16_t CG_%s_RUNS[] = { " % n)
        w(", ".join("%d, %d" % r for r in t["runs"]))
        w(" };\nstatic const uint16_t CG_%s_ADDR[] = {\n" % n)
        pos = t["pos"]
        for i in range(0, len(pos), 16):
            w("    " + ", ".join(str(v) for v in pos[i:i + 16]) + ",\n")
        w("};\n")
    w("\nstatic const struct cg_table cg_tables[] = {\n")
    for n in names:
        t = tables[n]
        w('    { "%s", %d, %d, %d, CG_%s_RUNS, CG_%s_ADDR },\n' % (n, t["N"], t["K"], len(t["runs"]), n, n))
    w("};\n#define CG_NTABLES %d\n\n" % len(names))
    for which in ("normal", "short"):
        w("static const struct cg_rate cg_rates_%s[] = {\n" % which)
        for rate, tab in maps[which]:
            w('    { "%s", %d },\n' % (rate, idx[tab]))
        w("};\n")
    for which in ("normal", "short"):
        w("static const struct cg_fec cg_fec_%s[] = {\n" % which)
        for r, kbch, nbch, t in fec[which]:
            w('    { "%s", %d, %d, %d },\n' % (r, kbch, nbch, t))
        w("};\n")
    w("\nstatic const struct cg_const cg_consts[] = {\n")
    for pls, name, rate, short, bits, order, pts in consts:
        w('    { 0x%02x, "%s", "%s", %d, %d, { %s },\n      { %s } },\n' % (
            pls, name, rate, short, bits, ", ".join(str(o) for o in order),
            ", ".join("%.9ff" % v for v in pts)))
    w("};\n#define CG_NCONSTS %d\n" % len(consts))


def main():
    root, out = sys.argv[1], sys.argv[2]
    with open(root + "/libdvbrx/src/ldpc_tables.h") as f:
        tables, maps = parse_ldpc(f.read())
    with open(root + "/libdvbrx/src/fec_table.h") as f:
        fec = parse_fec(f.read())
    with open(root + "/libdvbrx/src/const_tables.h") as f:
        consts = parse_const(f.read())
    with open(out, "w") as f:
        emit(tables, maps, fec, f, consts)


if __name__ == "__main__":
    main()
