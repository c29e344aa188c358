"""Synthetic chip-table AIR for multi-table proofs.

A table of `width` base columns over n = 2^log_n rows:
  * columns [0, width-2): seeded uniform Goldilocks data;
  * column width-2: a LogUp multiplicity column with values in [0, 2^16);
  * column width-1: a checksum, c[w-1](r) = sum_{j<k} c[j](r) * c[j](r+1 mod n).
Constraints (all cyclic over the n rows, zerofier x^n - 1):
  * T0 (base, degree 2): c[w-1](r) - sum_{j<k} c[j](r) c[j](r+1);
  * LogUp (crypto/stark/src/lookup.rs:2185-2290): interactions come in
    send/receive pairs of the same tuple on the same bus (so each table's bus
    contribution is zero), committed pairs get a batched term column
    (c fp_a fp_b - s_a m_a fp_b - s_b m_b fp_a), the last 1-2 interactions are
    absorbed into the accumulated column's constraint; fingerprints are
    fp = z - (bus + sum_i alpha^(i+1) v_i) (lookup.rs:2160-2183).
Boundary: the accumulated column is 0 at row 0 (lookup.rs:1330-1340).
Composition degree 3 -> two composition parts; H = C/Z has degree < 2n, so
blowup 2 already gives enough evaluation points.
"""
import numpy as np

from . import field as F
from .ir import Builder

P = F.P
NEG_ONE = P - 1


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def split_interactions(k):
    """lookup.rs:117-125: (committed pairs, absorbed count)."""
    if k <= 2:
        return 0, k
    if k % 2 == 1:
        return (k - 1) // 2, 1
    return (k - 2) // 2, 2


class SynthTableAir:
    def __init__(self, log_n, width, num_interactions=4, k_checksum=4, bus_base=100):
        assert width >= 6, "need at least 6 columns"
        assert num_interactions % 2 == 0 and num_interactions >= 2
        self.log_n, self.n, self.width = log_n, 1 << log_n, width
        self.k = min(k_checksum, width - 2)
        self.mult_col, self.sum_col = width - 2, width - 1
        data_cols = width - 2
        # interactions: pair p sends (c[a], c[b]) and receives the same tuple
        self.interactions = []
        for p in range(num_interactions // 2):
            a, b = (2 * p) % data_cols, (2 * p + 1) % data_cols
            for sender in (True, False):
                self.interactions.append({"bus": bus_base + p, "cols": (a, b), "sender": sender})
        self.num_committed, self.num_absorbed = split_interactions(num_interactions)
        self.aux_width = self.num_committed + 1  # ext3 columns
        self.acc_col = self.num_committed
        self.max_alpha = 3  # alpha^0..alpha^2 used (two values per tuple)
        self.program = self._build_program()
        self.num_transition = len(self.program["roots"])
        # the GPU prover's program: the checksum walked, the LogUp constraints
        # evaluated by the library from the descriptor
        self.device_program = self._build_program(logup=False)
        self.device_program["logup"] = (1, self.logup_descriptor())
        self.device_program["num_roots"] = self.num_transition
        self.boundary = [(self.acc_col, True, 0)]  # (column, is_aux, row)
        self.num_parts = 2

    # ---------------------------------------------------------- constraints
    def _fingerprint(self, b, it):
        z = b.challenge(0)
        fp = b.neg(b.sub(b.const_base(it["bus"]), z))  # z - bus
        for i, col in enumerate(it["cols"]):
            fp = b.sub(fp, b.mul(b.alpha_pow(i + 1), b.main(0, col)))
        return fp

    def _signed_mult_times(self, b, it, other_fp):
        t = b.mul(b.main(0, self.mult_col), other_fp)
        return t if it["sender"] else b.neg(t)

    def _build_program(self, logup=True):
        b = Builder()
        # T0: checksum (base)
        s = None
        for j in range(self.k):
            prod = b.mul(b.main(0, j), b.main(1, j))
            s = prod if s is None else b.add(s, prod)
        b.emit(b.sub(b.main(0, self.sum_col), s))
        if not logup:
            return b.program()
        # batched committed terms
        for p in range(self.num_committed):
            ia, ib = self.interactions[2 * p], self.interactions[2 * p + 1]
            c = b.aux(0, p)
            fa, fb = self._fingerprint(b, ia), self._fingerprint(b, ib)
            main = b.mul(b.mul(c, fa), fb)
            b.emit(b.sub(b.sub(main, self._signed_mult_times(b, ia, fb)), self._signed_mult_times(b, ib, fa)))
        # accumulated
        acc_c, acc_n = b.aux(0, self.acc_col), b.aux(1, self.acc_col)
        delta = b.sub(acc_n, acc_c)
        for p in range(self.num_committed):
            delta = b.sub(delta, b.aux(0, p))
        delta = b.add(delta, b.table_offset())
        ab = self.interactions[2 * self.num_committed:]
        if len(ab) == 1:
            f = self._fingerprint(b, ab[0])
            m = b.main(0, self.mult_col)
            mt = m if ab[0]["sender"] else b.neg(m)
            b.emit(b.neg(b.sub(mt, b.mul(delta, f))))
        else:
            f1, f2 = self._fingerprint(b, ab[0]), self._fingerprint(b, ab[1])
            root = b.mul(b.mul(delta, f1), f2)
            root = b.sub(root, self._signed_mult_times(b, ab[0], f2))
            root = b.sub(root, self._signed_mult_times(b, ab[1], f1))
            b.emit(root)
        return b.program()

    # ---------------------------------------------------------- LogUp descriptor
    def logup_descriptor(self):
        """CSR descriptor (crypto/math-cuda/src/logup.rs:26-44)."""
        K = len(self.interactions)
        eo, ea, ec, to, tc, tl = [0], [], [], [0], [], []
        mc, mo, mk, ml = [], [0], [], []
        for it in self.interactions:
            for i, col in enumerate(it["cols"]):
                ea.append(i + 1)
                ec.append(0)
                tc.append(1)
                tl.append(col)
                to.append(len(tc))
            eo.append(len(ea))
            mc.append(0)
            mk.append(1 if it["sender"] else NEG_ONE)
            ml.append(self.mult_col)
            mo.append(len(mk))
        oo, oi = [0], []
        for c in range(self.num_committed):
            oi += [2 * c, 2 * c + 1]
            oo.append(len(oi))
        oi += list(range(2 * self.num_committed, K))  # absorbed: one virtual column
        oo.append(len(oi))
        u32 = lambda x: np.array(x, np.uint32)
        u64 = lambda x: np.array(x, np.uint64)
        return {"num_interactions": K, "bus_ids": u64([it["bus"] for it in self.interactions]),
                "elem_offsets": u32(eo), "elem_alpha_idx": u32(ea), "elem_consts": u64(ec), "term_offsets": u32(to),
                "term_coefs": u64(tc), "term_cols": u32(tl), "num_out_cols": self.num_committed + 1,
                "out_col_offsets": u32(oo), "out_col_interactions": u32(oi), "mult_consts": u64(mc),
                "mult_term_offsets": u32(mo), "mult_term_coefs": u64(mk), "mult_term_cols": u32(ml),
                "num_committed": self.num_committed}

    # ---------------------------------------------------------- trace
    def trace(self, seed):
        """Counter-based synthetic trace (identical to sg_synth_trace on the device)."""
        n, w = self.n, self.width
        key = splitmix64(np.array([seed], np.uint64))[0]
        with np.errstate(over="ignore"):
            idx = key + np.arange(n * w, dtype=np.uint64)
        v = splitmix64(idx).reshape(n, w)
        t = F.canon(v)
        t[:, self.mult_col] = v[:, self.mult_col] & np.uint64(0xFFFF)
        s = np.zeros(n, np.uint64)
        for j in range(self.k):
            s = F.add(s, F.mul(t[:, j], np.roll(t[:, j], -1)))
        t[:, self.sum_col] = s
        return np.ascontiguousarray(t)

    def trace_random(self, seed):
        rng = np.random.default_rng(seed)
        n, w = self.n, self.width
        t = rng.integers(0, 2**64, size=(n, w), dtype=np.uint64)
        t = F.canon(t)
        t[:, self.mult_col] = rng.integers(0, 1 << 16, size=n, dtype=np.uint64)
        s = np.zeros(n, np.uint64)
        for j in range(self.k):
            s = F.add(s, F.mul(t[:, j], np.roll(t[:, j], -1)))
        t[:, self.sum_col] = s
        return np.ascontiguousarray(t)
