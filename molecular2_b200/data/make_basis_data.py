"""Extract the basis-set data this engine needs from a molecular2 checkout.

Run once, in a container that has the molecular2 sources, to (re)generate
``basis_sets.json`` beside this file:

    python molecular2_b200/data/make_basis_data.py <molecular2 checkout>

Basis sets are published data (EMSL Basis Set Exchange); molecular2 ships
them in two formats and this script reads both the way molecular2 does:

* XML library ``basislibrary/bases/build/<kind><N>.xml`` with the name→N map
  in ``basislibrary/<kind>.list`` (reader: ``src/basisreader.cpp:46-90``).
  One ``<Shell>`` element is one contracted shell.
* the legacy Molpro-style ``basissets/<NAME>first.basis`` files.  cc-pVDZ for
  H/C/O exists only here (``basis13.xml`` holds Na–Ar only).  Each ``c, i.j``
  contraction line becomes its own shell over exponents ``i..j``, which is the
  rule of ``basislibrary/parsebasis.py:55-68``.

Coefficients are stored exactly as printed (coefficients of normalised
primitives); normalisation is the engine's job, as it is libint2::Shell's in
molecular2 (``src/basis.cpp:49-61``).
"""
import json
import os
import sys
import xml.etree.ElementTree as ET

LVAL = {"s": 0, "p": 1, "sp": 1, "d": 2, "f": 3, "g": 4, "h": 5, "i": 6}

# (our name, kind, list key) for the XML library
XML_SETS = [
    ("6-311g**", "basis", "6-311gdp"),
    ("aug-cc-pvdz", "basis", "aug-cc-pvdz"),
    ("sto-3g", "basis", "sto-3g"),
    ("test", "basis", "test"),
    ("vdz-jkfit", "jkfit", "cc-pvdz"),
    ("avdz-jkfit", "jkfit", "aug-cc-pvdz"),
]
LEGACY_SETS = [("cc-pvdz", "CC-PVDZfirst.basis")]
ELEMENTS = ["h", "he", "c", "o"]


def read_list(ref, kind):
    root = ET.parse(os.path.join(ref, "basislibrary", kind + ".list")).getroot()
    return {it.get("key"): int(it.get("value")) for it in root.findall("Item")}


def read_xml(ref, kind, key):
    idx = read_list(ref, kind)[key]
    path = os.path.join(ref, "basislibrary", "bases", "build", f"{kind}{idx}.xml")
    root = ET.parse(path).getroot()
    out = {}
    for el in ELEMENTS:
        node = root.find(el)
        if node is None:
            continue
        shells = []
        for sh in node.findall("Shell"):
            exps = [float(xc.get("x")) for xc in sh.findall("xc")]
            coefs = [float(xc.get("c")) for xc in sh.findall("xc")]
            shells.append({"l": LVAL[sh.get("lval").strip()], "exps": exps, "coefs": coefs})
        out[el] = shells
    return out


def read_legacy(ref, fname):
    lines = open(os.path.join(ref, "basissets", fname)).read().splitlines()
    out = {}
    i = 0
    while i < len(lines):
        toks = [t.strip() for t in lines[i].strip().split(",")]
        if len(toks) > 1 and toks[0] in ("s", "p", "d", "f", "g", "h", "i"):
            l = LVAL[toks[0]]
            el = toks[1].lower()
            exps = [float(t) for t in toks[2:] if t]
            i += 1
            while i < len(lines):
                ct = [t.strip() for t in lines[i].strip().split(",")]
                if len(ct) > 1 and ct[0] == "c":
                    a, b = ct[1].split(".")
                    s, e = int(a) - 1, int(b) - 1
                    coefs = [float(t) for t in ct[2:] if t]
                    if el in ELEMENTS:
                        out.setdefault(el, []).append(
                            {"l": l, "exps": exps[s:e + 1], "coefs": coefs})
                    i += 1
                else:
                    break
            continue
        i += 1
    return out


def main(ref):
    data = {}
    for name, kind, key in XML_SETS:
        data[name] = read_xml(ref, kind, key)
    for name, fname in LEGACY_SETS:
        data[name] = read_legacy(ref, fname)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_sets.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of a molecular2 checkout>")
    main(sys.argv[1])
