"""The frozen per-class work table of the direct J/K kernel
(molecular2_b200/data/flop_table.json) is what make_flop_table.py produces."""
import importlib.util
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_flop_table_is_reproducible(tmp_path):
    path = os.path.join(ROOT, "molecular2_b200", "data", "make_flop_table.py")
    spec = importlib.util.spec_from_file_location("make_flop_table", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    committed = json.load(open(os.path.join(ROOT, "molecular2_b200", "data", "flop_table.json")))["table"]
    assert len(committed) == 21
    for A, (la, lb) in enumerate(mod.PAIR_CLASSES):
        for B, (lc, ld) in enumerate(mod.PAIR_CLASSES):
            if B > A:
                continue
            bra, q, dig = mod.quartet_flops(la, lb, lc, ld)
            t = committed[f"{A},{B}"]
            assert (t["bra"], t["quartet"], t["digest"]) == (bra, q, dig)
            assert dig == 12 * mod.ncart(la) * mod.ncart(lb) * mod.ncart(lc) * mod.ncart(ld)
