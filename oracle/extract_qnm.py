"""Build step for the oracle: read the QNM ringdown table (final spin,
fring, fdamp; 1003 points) from the reference's IMRPhenomD_internals.h
(QNMData_a / QNMData_fring / QNMData_fdamp, lines 176-640) and write it as a
C initialiser into oracle/_build/qnm_table.h (git-ignored build output).

Usage: python extract_qnm.py <reference dir> <output header>
"""
import re
import sys


def read_tables(ref_dir):
    src = open(f"{ref_dir}/IMRPhenomD_internals.h").read()
    out = {}
    for name in ("QNMData_a", "QNMData_fring", "QNMData_fdamp"):
        m = re.search(r"static const double " + name + r"\[\]\s*=\s*\{(.*?)\};", src, re.S)
        body = m.group(1).replace("\\", " ")
        out[name] = [float(x) for x in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?", body)]
    n = {len(v) for v in out.values()}
    assert len(n) == 1, "QNM tables differ in length"
    return out


def main():
    ref_dir, dst = sys.argv[1], sys.argv[2]
    t = read_tables(ref_dir)
    n = len(t["QNMData_a"])
    with open(dst, "w") as f:
        f.write("/* generated by oracle/extract_qnm.py from the reference header; not committed */\n")
        f.write(f"#define ORA_QNM_N {n}\n")
        for name, key in (("ORA_QNM_A", "QNMData_a"), ("ORA_QNM_FRING", "QNMData_fring"),
                          ("ORA_QNM_FDAMP", "QNMData_fdamp")):
            vals = ",".join(repr(v) for v in t[key])
            f.write(f"static const double {name}[{n}] = {{{vals}}};\n")


if __name__ == "__main__":
    main()
