"""Extract molecular2's recorded outputs into ``reference_pins.json``.

Run in a container that has the molecular2 sources:

    python tests/golden/make_golden.py <molecular2 checkout>

molecular2 has no automated tests; its only expected values are hand-run
outputs kept in ``test/``.  This script copies the numbers out of them:
  * ``test/h2otest.out_1:124``   RHF/cc-pVDZ H2O energy (Cartesian d: the run
    printed 25 orbital energies), geometry ``test/h2otest.mol:8-10`` in bohr;
  * ``test/benzene.out_1:104``   RHF/cc-pVDZ benzene energy (Cartesian d:
    "d 6.00 CGBFs" at :47), geometry ``test/benzene-dz.mol`` in angstrom;
  * ``test/h2otest.opt:7-15``    first gradient block at the h2otest geometry
    (its energy -75.9898 is the spherical cc-pVDZ one);
  * ``test/cdthe.ints``          weighted ERIs of He in the 5-primitive "test"
    basis, printed by ``IntegralEngine::printERI`` (src/integrals.cpp:203-233).
"""
import json
import os
import re
import sys


def main(ref):
    t = os.path.join(ref, "test")
    out = {}
    txt = open(os.path.join(t, "h2otest.out_1")).read()
    out["h2otest_energy"] = float(re.search(r"RHF Energy = (-?\d+\.\d+)", txt).group(1))
    geo = []
    for line in open(os.path.join(t, "h2otest.mol")).read().splitlines()[7:10]:
        sym, *xyz = [x.strip() for x in line.split(",")]
        geo.append([sym.lower()] + [float(v) for v in xyz])
    out["h2otest_geometry_bohr"] = geo
    # the final row of the SCF table carries 9 decimals (the summary line only 6)
    rows = re.findall(r"^\s+(\d+)\s+(-\d+\.\d{9})\s", open(os.path.join(t, "benzene.out_1")).read(), re.M)
    out["benzene_energy"] = float(rows[-1][1])
    geo = []
    lines = open(os.path.join(t, "benzene-dz.mol")).read().splitlines()
    for line in lines:
        m = re.match(r"\s*([CH]),\s*(-?[\d.]+),\s*(-?[\d.]+),\s*(-?[\d.]+)", line)
        if m:
            geo.append([m.group(1).lower()] + [float(m.group(i)) for i in (2, 3, 4)])
    out["benzene_geometry_angstrom"] = geo
    grad = {}
    seen = 0
    for line in open(os.path.join(t, "h2otest.opt")).read().splitlines():
        if line.startswith("ITERATION"):
            seen += 1
            if seen > 1:
                break
        m = re.match(r"\s*([XYZ])(\d)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)", line)
        if m:
            grad[m.group(1) + m.group(2)] = float(m.group(5))
    out["h2otest_gradient_first"] = grad
    ints = []
    for line in open(os.path.join(t, "cdthe.ints")).read().splitlines():
        p = line.split()
        if len(p) == 5 and all(x.isdigit() for x in p[:4]):
            ints.append([int(x) for x in p[:4]] + [float(p[4])])
    out["cdthe_weighted_eris"] = ints
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_pins.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of a molecular2 checkout>")
    main(sys.argv[1])
