"""Generate dvbrx_b200/csrc/bb_tables.h: the DVB-S2 BBFRAME scrambling
sequence and the CRC-8 table, from their definitions in EN 302 307-1.

    python dvbrx_b200/tables/gen_bb.py dvbrx_b200/csrc/bb_tables.h

* Scrambler (5.2.2): PRBS of 1 + x^14 + x^15, initial register
  100101010000000, restarted on every BBFRAME; one byte per 8 bits, MSB
  first, for the longest BBFRAME (normal rate 9/10, kbch = 58192 bits).
* CRC-8 (5.1.4, Annex F): generator x^8 + x^7 + x^6 + x^4 + x^2 + 1 (0xD5),
  register starting at 0, one table entry per input byte.
"""
import sys

KBCH_MAX_BYTES = 58192 // 8


def prbs_bytes(n):
    reg, out = 0x4A80, []  # bits 1..15 of the register: 100101010000000
    for _ in range(n):
        byte = 0
        for _ in range(8):
            bit = ((reg >> 1) ^ reg) & 1  # taps x^14 and x^15
            reg = (reg >> 1) | (bit << 14)
            byte = (byte << 1) | bit
        out.append(byte)
    return out


def crc8_table():
    tab = []
    for v in range(256):
        c = v
        for _ in range(8):
            c = ((c << 1) ^ 0xD5) & 0xFF if c & 0x80 else (c << 1) & 0xFF
        tab.append(c)
    return tab


def emit(name, vals):
    lines = ["static __device__ const uint8_t %s[%d] = {" % (name, len(vals))]
    for i in range(0, len(vals), 16):
        lines.append("    " + ", ".join("0x%02x" % v for v in vals[i:i + 16]) + ",")
    lines.append("};")
    return "\n".join(lines)


def main(out):
    with open(out, "w") as f:
        f.write("/* Generated by dvbrx_b200/tables/gen_bb.py: DVB-S2 BBFRAME scrambling sequence\n"
                " * (EN 302 307-1 5.2.2) and CRC-8 table (5.1.4). Do not edit. */\n#pragma once\n#include <stdint.h>\n\n")
        f.write("#define DRXG_KBCH_MAX_BYTES %d\n\n" % KBCH_MAX_BYTES)
        f.write(emit("g_bb_prbs", prbs_bytes(KBCH_MAX_BYTES)) + "\n\n")
        f.write(emit("g_bb_crc8", crc8_table()) + "\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "dvbrx_b200/csrc/bb_tables.h")
