"""Vectorised constraint evaluation over many rows at once, for the front-end
tests: walks an UNLOWERED IR program (constraint_ir/interp.rs semantics) with
every value a triple of numpy object arrays (Fp3 coordinates, one entry per
row) of Python ints, so a program of tens of thousands of nodes is checked on
a few hundred rows in seconds. Test infrastructure."""
import numpy as np

import oracle as O

P = O.P
W = 2  # Fp3 = Fp[w] / (w^3 - 2)


def _mul3(a, b):
    a0, a1, a2 = a
    b0, b1, b2 = b
    c0 = (a0 * b0 + W * (a1 * b2 + a2 * b1)) % P
    c1 = (a0 * b1 + a1 * b0 + W * a2 * b2) % P
    c2 = (a0 * b2 + a1 * b1 + a2 * b0) % P
    return (c0, c1, c2)


def eval_rows(prog, main, aux, rap, apows, offset, rows):
    """Value of every root of `prog` on each of `rows` (list of row indices):
    a list of (c0, c1, c2) object arrays. main: (n, w) u64; aux: (n, 3 a) u64
    or None."""
    n = main.shape[0]
    rows = np.asarray(rows)
    zero = np.zeros(len(rows), dtype=object)
    base = [True] * len(prog["nodes"])
    v = []
    for i, nd in enumerate(prog["nodes"]):
        k = nd[0]
        if k == "var":
            _, is_main, off, col = nd
            r = (rows + off) % n
            if is_main:
                v.append(main[r, col].astype(object))
            else:
                base[i] = False
                v.append(tuple(aux[r, 3 * col + j].astype(object) for j in range(3)))
        elif k == "cb":
            v.append(zero + prog["base_consts"][nd[1]])
        elif k in ("ce", "rap", "alpha", "off"):
            base[i] = False
            c = {"ce": lambda: prog["ext_consts"][nd[1]], "rap": lambda: rap[nd[1]],
                 "alpha": lambda: apows[nd[1]], "off": lambda: offset}[k]()
            v.append(tuple(zero + int(c[j]) for j in range(3)))
        elif k in ("add", "sub", "mul"):
            x, y = v[nd[1]], v[nd[2]]
            bx, by = base[nd[1]], base[nd[2]]
            if bx and by:
                v.append((x + y) % P if k == "add" else (x - y) % P if k == "sub" else (x * y) % P)
                continue
            base[i] = False
            x = (x, zero, zero) if bx else x
            y = (y, zero, zero) if by else y
            if k == "add":
                v.append(tuple((x[j] + y[j]) % P for j in range(3)))
            elif k == "sub":
                v.append(tuple((x[j] - y[j]) % P for j in range(3)))
            else:
                v.append(_mul3(x, y))
        elif k == "neg":
            x = v[nd[1]]
            base[i] = base[nd[1]]
            v.append((-x) % P if base[i] else tuple((-x[j]) % P for j in range(3)))
        else:
            base[i] = base[nd[1]]
            v.append(v[nd[1]])
    out = []
    for r in prog["roots"]:
        out.append((v[r], zero, zero) if base[r] else v[r])
    return out


def bad_constraints(prog, main, aux, rap, apows, offset, rows):
    """{(constraint index, row)} of every root that does not vanish."""
    vals = eval_rows(prog, main, aux, rap, apows, offset, rows)
    bad = set()
    for ci, (c0, c1, c2) in enumerate(vals):
        nz = np.nonzero((c0 != 0) | (c1 != 0) | (c2 != 0))[0]
        bad |= {(ci, int(rows[j])) for j in nz}
    return bad
