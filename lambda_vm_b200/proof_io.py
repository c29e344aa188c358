"""Canonical byte serialization of a multi-table proof.

The reference serializes proofs with rkyv (crypto/stark/src/proof/stark.rs);
this module defines a plain canonical layout of the same logical content —
every root, challenge-derived value, OOD value, FRI layer commitment and
opening, terminal coefficient, nonce and query index — so "the same proof"
means "the same bytes". All integers are little-endian; field elements are
canonical (in [0, p)) u64; ext3 elements are (c0, c1, c2).

    proof   := b"SGPF" u32:version=1 ext3[2]:challenges u32:tables table*
    table   := root:main root:aux root:comp ext3:table_contribution
               u32:W ext3[2*W]:trace_ood ext3[2]:parts_ood
               u32:F root[F]:fri_roots u32:T ext3[T]:fri_final_coeffs
               u64:nonce u32:Q u64[Q]:iotas
               mat:open_main mat:open_aux mat:open_parts
               paths:path_main paths:path_aux paths:path_parts
               (mat paths)[F]:fri_open, fri_paths
    mat     := u32:rows u32:cols u64[rows*cols]
    paths   := u32:queries u32:depth bytes[queries*depth*32]
"""
import struct

import numpy as np

P = 0xFFFFFFFF00000001
MAGIC = b"SGPF"
VERSION = 1


def _u64s(vals):
    a = np.asarray(vals, dtype=np.uint64).reshape(-1)
    a = np.where(a >= np.uint64(P), a - np.uint64(P), a)
    return a.astype("<u8").tobytes()


def _mat(m):
    m = np.asarray(m, dtype=np.uint64)
    rows, cols = m.shape
    return struct.pack("<II", rows, cols) + _u64s(m)


def _paths(p):
    p = np.asarray(p, dtype=np.uint8)
    q, d = p.shape[0], (p.shape[1] if p.ndim == 3 else 0)
    return struct.pack("<II", q, d) + p.reshape(-1).tobytes()


def serialize(proof):
    out = [MAGIC, struct.pack("<I", VERSION), _u64s(proof["challenges"]), struct.pack("<I", len(proof["tables"]))]
    for t in proof["tables"]:
        out += [bytes(t["main_root"]), bytes(t["aux_root"]), bytes(t["comp_root"]), _u64s(t["table_contribution"])]
        W = len(t["trace_ood"][0])
        out += [struct.pack("<I", W), _u64s(t["trace_ood"]), _u64s(t["parts_ood"])]
        out += [struct.pack("<I", len(t["fri_roots"]))] + [bytes(r) for r in t["fri_roots"]]
        out += [struct.pack("<I", len(t["fri_final_coeffs"])), _u64s(t["fri_final_coeffs"])]
        out += [struct.pack("<Q", int(t["nonce"])), struct.pack("<I", len(t["iotas"])), _u64s(t["iotas"])]
        out += [_mat(t["open_main"]), _mat(t["open_aux"]), _mat(t["open_parts"])]
        out += [_paths(t["path_main"]), _paths(t["path_aux"]), _paths(t["path_parts"])]
        for fo, fp in zip(t["fri_open"], t["fri_paths"]):
            out += [_mat(fo), _paths(fp)]
    return b"".join(out)


class _Reader:
    def __init__(self, b):
        self.b, self.o = memoryview(b), 0

    def take(self, n):
        if self.o + n > len(self.b):
            raise ValueError("truncated proof")
        v = self.b[self.o:self.o + n]
        self.o += n
        return bytes(v)

    def u32(self):
        return struct.unpack("<I", self.take(4))[0]

    def u64s(self, n):
        return np.frombuffer(self.take(8 * n), dtype="<u8").astype(np.uint64)

    def ext3s(self, n):
        return [tuple(int(x) for x in row) for row in self.u64s(3 * n).reshape(n, 3)] if n else []

    def mat(self):
        r, c = self.u32(), self.u32()
        return self.u64s(r * c).reshape(r, c)

    def paths(self):
        q, d = self.u32(), self.u32()
        return np.frombuffer(self.take(q * d * 32), dtype=np.uint8).reshape(q, d, 32).copy()


def deserialize(b):
    r = _Reader(b)
    if r.take(4) != MAGIC or r.u32() != VERSION:
        raise ValueError("not a serialized proof of this version")
    challenges = r.ext3s(2)
    tables = []
    for _ in range(r.u32()):
        t = {"main_root": r.take(32), "aux_root": r.take(32), "comp_root": r.take(32),
             "table_contribution": r.ext3s(1)[0]}
        W = r.u32()
        flat = r.ext3s(2 * W)
        t["trace_ood"] = [flat[:W], flat[W:]]
        t["parts_ood"] = r.ext3s(2)
        F = r.u32()
        t["fri_roots"] = [r.take(32) for _ in range(F)]
        t["fri_final_coeffs"] = r.ext3s(r.u32())
        t["nonce"] = struct.unpack("<Q", r.take(8))[0]
        t["iotas"] = [int(x) for x in r.u64s(r.u32())]
        t["open_main"], t["open_aux"], t["open_parts"] = r.mat(), r.mat(), r.mat()
        t["path_main"], t["path_aux"], t["path_parts"] = r.paths(), r.paths(), r.paths()
        t["fri_open"], t["fri_paths"] = [], []
        for _ in range(F):
            t["fri_open"].append(r.mat())
            t["fri_paths"].append(r.paths())
        tables.append(t)
    if r.o != len(r.b):
        raise ValueError("trailing bytes after the proof")
    return {"tables": tables, "challenges": challenges}
