"""Frozen per-class FP64 work table of the direct J/K kernel (the roofline's
numerator).

    python molecular2_b200/data/make_flop_table.py

Counts the floating-point operations (an FMA counts 2) that the
McMurchie-Davidson quartet evaluation of csrc/jk_kernels.cuh (quartet_cart,
with md_E1, boys and md_R of csrc/md.cuh) performs for one shell quartet of
angular class (LA LB | LC LD), split into
  * bra: work done once per bra primitive pair (its three E tables),
  * quartet: work done once per primitive quartet (ket E tables, Boys
    function, Hermite R table, the two contraction stages),
and the J/K digestion, 6 FMAs (12 flops) per Cartesian integral and density.
The counts follow the loop structure of the kernel source term by term
(exp, sqrt and divisions count 1 each).  The work model of one build is
  sum over classes  bra * (bra primitive pairs) + quartet * (primitive quartets)
                    + digest * (quartets)
with the class counts reported by jk_last_class_work.  Written to
flop_table.json beside this file.
"""
import json
import os


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nherm(L):
    return (L + 1) * (L + 2) * (L + 3) // 6


def cart(l):
    out = []
    for a in range(l, -1, -1):
        for b in range(l - a, -1, -1):
            out.append((a, b, l - a - b))
    return out


def herm(L):
    return [c for k in range(L + 1) for c in cart(k)]


def e1_flops(LA, LB):
    """md_E1<LA, LB>: one Cartesian direction."""
    f = 0
    for i in range(LA + 1):
        for j in range(LB + 1):
            if i == 0 and j == 0:
                continue
            for t in range(i + j + 1):
                f += 1                                   # PA * E (or PB * E)
                if t > 0:
                    f += 2                               # + oo2p * E
                if (j == 0 and t + 1 <= i - 1) or (j > 0 and t + 1 <= i + j - 1):
                    f += 2                               # + (t + 1) * E
    return f


def boys_flops(M):
    return 1 + 6 * 3 + 1 + 1 + 4 * M                    # grid index, Taylor, exp, downward recursion


def r_flops(L):
    f = L                                                # powers of -2a
    for n in range(L - 1, -1, -1):
        for k in range(L - n, 0, -1):
            for (t, u, v) in cart(k):
                lead = t if t > 0 else (u if u > 0 else v)
                f += 1 + (2 if lead > 1 else 0)
        f += 1
    return f + 1


def quartet_flops(LA, LB, LC, LD):
    LAB, LCD = LA + LB, LC + LD
    L = LAB + LCD
    bra = 3 * e1_flops(LA, LB) + 1                       # three directions, 0.5 / p
    q = 3 * e1_flops(LC, LD) + 1                         # ket E tables, 0.5 / q
    q += 1 + 2 + 6 + 3 + 6                               # p + q, alpha, prefactor, PQ, T
    q += boys_flops(L) + r_flops(L)
    # W[h] = sum_{tau nu phi} (+-) E^cd_tau E_nu E_phi R[h + (tau nu phi)]
    for (cx, cy, cz) in cart(LC):
        for (dx, dy, dz) in cart(LD):
            terms = (cx + dx + 1) * (cy + dy + 1) * (cz + dz + 1)
            q += nherm(LAB) * terms * 4
    # out[ab][cd] += pref * sum_{tuv} E^ab_t E_u E_v W[tuv]
    for (ax, ay, az) in cart(LA):
        for (bx, by, bz) in cart(LB):
            terms = (ax + bx + 1) * (ay + by + 1) * (az + bz + 1)
            q += ncart(LC) * ncart(LD) * (terms * 4 + 2)
    digest = 12 * ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)
    return bra, q, digest


PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]  # ss ps pp ds dp dd


def main():
    table = {}
    for A, (la, lb) in enumerate(PAIR_CLASSES):
        for B, (lc, ld) in enumerate(PAIR_CLASSES):
            if B > A:
                continue
            bra, q, dig = quartet_flops(la, lb, lc, ld)
            table[f"{A},{B}"] = {"class": f"({'spd'[la]}{'spd'[lb]}|{'spd'[lc]}{'spd'[ld]})", "bra": bra,
                                 "quartet": q, "digest": dig}
    out = {"model": "flops per bra primitive pair (bra), per primitive quartet (quartet) and per quartet "
                    "(digest, one density) of the direct J/K kernel; keys 'bra class,ket class' in the order "
                    "ss ps pp ds dp dd",
           "table": table}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "flop_table.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
